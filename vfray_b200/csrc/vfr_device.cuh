// Device-side arithmetic of the VF-Ray render path (sm_100a).
//
// Every operation that decides which faces are visible, which pixels a face
// covers, which face a ray leaves a tet through, and which colour it adds is
// written with explicit round-to-nearest intrinsics (__fadd_rn, __fmul_rn,
// __fdiv_rn, __dadd_rn, ...), so nvcc can neither contract it into an FMA nor
// reorder it: each one is the single IEEE operation the reference's C++
// expression performs (vfRayKernelCPU.cc), including the places where a double
// literal (1.0, 0.5, RDELTA) promotes a float expression to double.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vfr {

constexpr double kRDelta = 1e-12;  // vfRayKernelCPU.h:28 (a double)

// Packed tet record: 4 vertex ids + 4 neighbour ids (conTet row), 32 bytes.
struct __align__(16) TetRec {
  uint4 v;
  uint4 n;
};

struct Plane {
  float zx, zy, zz, sx, sy, sz;
};

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// ABS(n) ((n) < 0 ? -(n) : (n)) compared against the double RDELTA
__device__ __forceinline__ bool below_rdelta(float v) {
  float a = v < 0.0f ? -v : v;
  return (double)a < kRDelta;
}

__device__ __forceinline__ uint32_t sel4(uint4 v, uint32_t i) {
  uint32_t r = v.x;
  r = (i == 1) ? v.y : r;
  r = (i == 2) ? v.z : r;
  r = (i == 3) ? v.w : r;
  return r;
}

__device__ __forceinline__ float4 sel4(const float4 (&v)[4], uint32_t i) {
  float4 r = v[0];
  if (i == 1) r = v[1];
  if (i == 2) r = v[2];
  if (i == 3) r = v[3];
  return r;
}

// Cramer solve of the plane through a, b, c for z(x, y) and s(x, y)
// (vfRayKernelCPU.cc:73-122, repeated at :380-429), same operand order.
__device__ __forceinline__ void face_plane(float4 a, float4 b, float4 c, Plane& p) {
  const float c0x = a.x, c0y = b.x, c0z = c.x;
  const float c1x = a.y, c1y = b.y, c1z = c.y;
  const float cross = fsub(fmul(c0y, c1z), fmul(c1y, c0z));
  float det = fadd(fsub(fmul(c0x, fsub(c1y, c1z)), fmul(c1x, fsub(c0y, c0z))), cross);
  det = below_rdelta(det) ? (float)kRDelta : det;
  const float d1 = fsub(c1y, c1z), d0 = fsub(c0y, c0z);
  {
    const float tx = a.z, ty = b.z, tz = c.z;
    const float mx = fsub(ty, tz);
    const float my = fsub(fmul(ty, c1z), fmul(c1y, tz));
    const float mz = fsub(fmul(c0y, tz), fmul(ty, c0z));
    p.zx = fdiv(fadd(fsub(fmul(tx, d1), fmul(c1x, mx)), my), det);
    p.zy = fdiv(fadd(fsub(fmul(c0x, mx), fmul(tx, d0)), mz), det);
    p.zz = fdiv(fadd(fsub(fmul(c0x, -my), fmul(c1x, mz)), fmul(tx, cross)), det);
  }
  {
    const float tx = a.w, ty = b.w, tz = c.w;
    const float mx = fsub(ty, tz);
    const float my = fsub(fmul(ty, c1z), fmul(c1y, tz));
    const float mz = fsub(fmul(c0y, tz), fmul(ty, c0z));
    p.sx = fdiv(fadd(fsub(fmul(tx, d1), fmul(c1x, mx)), my), det);
    p.sy = fdiv(fadd(fsub(fmul(c0x, mx), fmul(tx, d0)), mz), det);
    p.sz = fdiv(fadd(fsub(fmul(c0x, -my), fmul(c1x, mz)), fmul(tx, cross)), det);
  }
}

// a*x + b*y + c, left to right, no FMA
__device__ __forceinline__ float plane_eval(float x, float y, float a, float b, float c) {
  return fadd(fadd(fmul(x, a), fmul(y, b)), c);
}

// obj = (pix*2)/(float)(res-1) - 1.0 (vfRayKernelCPU.cc:250,254): float
// quotient, double subtraction, stored as float.
__device__ __forceinline__ float obj_coord(uint32_t pix, uint32_t res) {
  float q = fdiv((float)(pix * 2u), (float)(res - 1u));
  return (float)dsub((double)q, 1.0);
}

// (uint)((res - 1.0) * (x + 1.0) / 2.0) in double (vfRayKernelCPU.cc:158-159),
// converted the way the x86-64 reference binary converts: truncate to a
// 64-bit integer and keep the low 32 bits.
__device__ __forceinline__ uint32_t to_pixel(float x, uint32_t res) {
  double d = ddiv(dmul(dsub((double)res, 1.0), dadd((double)x, 1.0)), 2.0);
  return (uint32_t)(unsigned long long)__double2ll_rz(d);
}

// Entry-face edge vectors and doubled area (vfRayKernelCPU.cc:195-216).
struct EntryEdges {
  float v0x, v0y, e1x, e1y, e2x, e2y, cx;
};

__device__ __forceinline__ EntryEdges entry_edges(float4 v0, float4 v1, float4 v2) {
  EntryEdges E;
  float ax = fsub(v1.x, v0.x), ay = fsub(v1.y, v0.y);
  float bx = fsub(v2.x, v0.x), by = fsub(v2.y, v0.y);
  float cx = fsub(fmul(ax, by), fmul(ay, bx));
  cx = below_rdelta(cx) ? (float)kRDelta : cx;
  if (cx < 0.0f) {
    float tx = ax, ty = ay;
    ax = bx; ay = by; bx = tx; by = ty;
    cx = -cx;
  }
  E.v0x = v0.x; E.v0y = v0.y;
  E.e1x = ax; E.e1y = ay; E.e2x = bx; E.e2y = by; E.cx = cx;
  return E;
}

// Inclusive inside test of the entry face, no slack (vfRayKernelCPU.cc:258-268).
__device__ __forceinline__ bool entry_inside(const EntryEdges& E, float ox, float oy) {
  float px = fsub(ox, E.v0x), py = fsub(oy, E.v0y);
  float cy = fsub(fmul(E.e1x, py), fmul(E.e1y, px));
  float cz = fsub(fmul(px, E.e2y), fmul(py, E.e2x));
  return (cy >= 0.0f) && (cz >= 0.0f) && (fadd(cy, cz) <= E.cx);
}

// Exit-face search among the 3 faces other than the entry face
// (vfRayKernelCPU.cc:312-350): 2-D edge functions with +RDELTA slack on the
// sum, faces with |cross| < RDELTA skipped.  Returns the entry face itself
// when no face qualifies (the reference's "anomaly" end of the ray).
__device__ __forceinline__ uint32_t find_exit(const float4 (&fv)[4], uint32_t entry, float ox,
                                              float oy) {
#pragma unroll
  for (uint32_t i = 1; i < 4; ++i) {
    const uint32_t id = (entry + i) & 3u;
    const float4 a = sel4(fv, id), b = sel4(fv, (id + 1) & 3u), c = sel4(fv, (id + 2) & 3u);
    float v1x = fsub(b.x, a.x), v1y = fsub(b.y, a.y);
    float v2x = fsub(c.x, a.x), v2y = fsub(c.y, a.y);
    float cr = fsub(fmul(v1x, v2y), fmul(v1y, v2x));
    if (below_rdelta(cr)) continue;
    if (cr < 0.0f) {
      float tx = v1x, ty = v1y;
      v1x = v2x; v1y = v2y; v2x = tx; v2y = ty;
      cr = -cr;
    }
    const float v0x = fsub(ox, a.x), v0y = fsub(oy, a.y);
    const float c1 = fsub(fmul(v1x, v0y), fmul(v1y, v0x));
    const float c2 = fsub(fmul(v0x, v2y), fmul(v0y, v2x));
    if ((c1 >= 0.0f) && (c2 >= 0.0f) && ((double)fadd(c1, c2) <= dadd((double)cr, kRDelta)))
      return id;
  }
  return entry;
}

// Orderable encoding of floats for atomicMin/atomicMax on unsigned ints.
__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
  uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  return __uint_as_float(b);
}

}  // namespace vfr
