// Test infrastructure (reference harness only).  Force-included in front of
// the reference's vfRayKernelCPU.cc for the counting build: it wraps exp(),
// which the reference calls exactly once per compositing step
// (vfRayKernelCPU.cc:458), to count steps without editing the source.  The
// wrapper returns std::exp of the same double argument, so results are those
// of the plain strict build.
#include <cassert>
#include <cmath>
#include <cstdio>
extern "C" unsigned long long vfref_exp_calls;
static inline double vfref_counted_exp(double x) {
  ++vfref_exp_calls;
  return std::exp(x);
}
#define exp(x) vfref_counted_exp(x)
