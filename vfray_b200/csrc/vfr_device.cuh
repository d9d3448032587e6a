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

// The checked build (`make checked`: -DVFR_CHECKED) compares every id a
// kernel reads from memory with the extent of the array it is about to
// index: the mesh's tet, vertex and neighbour ids, and the visible-face,
// bin, ray and entry ids the stages write for one another.  A bad id sets
// VFR_DEV_RANGE in its job's status and the access is skipped (the face
// counts as invisible, the pixel or the ray is dropped), so a corrupt input
// or a stage bug shows as a status instead of a fault.  The product build
// leaves the checks out: mesh ids are validated when the mesh is uploaded,
// and the stages' ids are in range by construction.
#ifdef VFR_CHECKED
constexpr bool kChecked = true;
#else
constexpr bool kChecked = false;
#endif
constexpr uint32_t kDevRange = 4u;  // VFR_DEV_RANGE

__host__ __device__ __forceinline__ bool id_bad(uint32_t id, uint32_t n) {
  return kChecked && id >= n;
}

// Walk record of a tet, 32 bytes: the 4 neighbour ids (the conTet row, self
// = boundary) and, per face f, one packed word q[f] describing the neighbour
// n across f: bits 0-26 the id of n's vertex opposite the shared face (the
// only vertex of n a ray entering n through that face does not already
// hold), bits 27-28 the face of n it is entered through (the first k with
// conTet[4n+k] == t, as vfRayKernelCPU.cc:361-364 finds it), bits 29-31 how
// n orders the shared face's vertices: a permutation code 0-5 (perm_code), 6 if
// the ids do not match (the walk then reloads n's vertices), 7 for a
// boundary face.  The walk reads only these records; vertex ids of a tet
// come from the plain tet array (uint4 per tet) when a ray starts.
struct __align__(16) WalkRec {
  uint4 n;
  uint4 q;
};

// perm_code(k) packs, for j = 0..2, which vertex of the exit face (0, 1, 2
// in the current tet's order) sits at slot (fn + j) of the next tet, 2 bits
// each, for the 6 permutations k = (012, 021, 102, 120, 201, 210).
__host__ __device__ __forceinline__ uint32_t perm_code(uint32_t k) {
  // 6-bit fields: 0b100100, 0b011000, 0b100001, 0b001001, 0b010010, 0b000110
  constexpr unsigned long long kLut = 0x24ull | 0x18ull << 6 | 0x21ull << 12 | 0x09ull << 18 |
                                      0x12ull << 24 | 0x06ull << 30;
  return (uint32_t)(kLut >> (6 * k)) & 63u;
}

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

// ABS(n) ((n) < 0 ? -(n) : (n)) compared against the double RDELTA: for a
// float a, (double)a < 1e-12 exactly when a <= 0x2b8cbccc (9.9999996e-13, the
// largest float below 1e-12), so the comparison needs no conversion.
__device__ __forceinline__ bool below_rdelta(float v) {
  return fabsf(v) <= __uint_as_float(0x2b8cbcccu);
}

__device__ __forceinline__ uint32_t sel4(uint4 v, uint32_t i) {
  uint32_t r = v.x;
  r = (i == 1) ? v.y : r;
  r = (i == 2) ? v.z : r;
  r = (i == 3) ? v.w : r;
  return r;
}

// RN(a / b) for floats through a double reciprocal shared by every quotient
// with the same divisor: y = __drcp_rn((double)b) is the correctly rounded
// 1/b, so (double)a * y is within 2^-52 (relative) of a / b.  A quotient of
// two floats in the normal range never lies within 2^-49 (relative) of a
// half-way point between floats: with a = A 2^i, b = B 2^j (A, B odd, below
// 2^24) and the half-way point M 2^k (M odd, at least 2^24), a - M 2^k b is
// a nonzero multiple of 2^min(i, k+j), since A = M B is impossible.  So
// rounding that double to float gives RN(a / b), the IEEE float division
// the reference performs, whenever the quotient is in the normal range
// (subnormal quotients can sit exactly half-way): the callers check that.
__device__ __forceinline__ float div_by(float a, double recip_b) {
  return __double2float_rn(__dmul_rn((double)a, recip_b));
}

// Cramer solve of the plane through a, b, c for z(x, y) and s(x, y)
// (vfRayKernelCPU.cc:73-122, repeated at :380-429), same operand order, with
// IEEE float divisions.
__device__ __forceinline__ void face_plane_ieee(float4 a, float4 b, float4 c, Plane& p) {
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

// The same plane with the six divisions by det sharing one reciprocal
// (div_by).  A coefficient of at least 2^-125 in magnitude is a quotient in
// the normal range, so div_by gave it exactly.  When any coefficient is
// smaller (zero included: rare, a face with an exactly constant depth or
// scalar along an axis), this returns false and the plane must be solved
// again with IEEE divisions (face_plane does so).
__device__ __forceinline__ bool face_plane_fast(float4 a, float4 b, float4 c, Plane& p) {
  const float c0x = a.x, c0y = b.x, c0z = c.x;
  const float c1x = a.y, c1y = b.y, c1z = c.y;
  const float cross = fsub(fmul(c0y, c1z), fmul(c1y, c0z));
  float det = fadd(fsub(fmul(c0x, fsub(c1y, c1z)), fmul(c1x, fsub(c0y, c0z))), cross);
  det = below_rdelta(det) ? (float)kRDelta : det;
  const double rdet = __drcp_rn((double)det);
  const float d1 = fsub(c1y, c1z), d0 = fsub(c0y, c0z);
  {
    const float tx = a.z, ty = b.z, tz = c.z;
    const float mx = fsub(ty, tz);
    const float my = fsub(fmul(ty, c1z), fmul(c1y, tz));
    const float mz = fsub(fmul(c0y, tz), fmul(ty, c0z));
    p.zx = div_by(fadd(fsub(fmul(tx, d1), fmul(c1x, mx)), my), rdet);
    p.zy = div_by(fadd(fsub(fmul(c0x, mx), fmul(tx, d0)), mz), rdet);
    p.zz = div_by(fadd(fsub(fmul(c0x, -my), fmul(c1x, mz)), fmul(tx, cross)), rdet);
  }
  {
    const float tx = a.w, ty = b.w, tz = c.w;
    const float mx = fsub(ty, tz);
    const float my = fsub(fmul(ty, c1z), fmul(c1y, tz));
    const float mz = fsub(fmul(c0y, tz), fmul(ty, c0z));
    p.sx = div_by(fadd(fsub(fmul(tx, d1), fmul(c1x, mx)), my), rdet);
    p.sy = div_by(fadd(fsub(fmul(c0x, mx), fmul(tx, d0)), mz), rdet);
    p.sz = div_by(fadd(fsub(fmul(c0x, -my), fmul(c1x, mz)), fmul(tx, cross)), rdet);
  }
  const float m = fminf(fminf(fminf(fabsf(p.zx), fabsf(p.zy)), fminf(fabsf(p.zz), fabsf(p.sx))),
                        fminf(fabsf(p.sy), fabsf(p.sz)));
  return m >= 0x1p-125f;
}

__device__ __forceinline__ void face_plane(float4 a, float4 b, float4 c, Plane& p) {
  if (!face_plane_fast(a, b, c, p)) face_plane_ieee(a, b, c, p);
}

// a*x + b*y + c, left to right, no FMA
__device__ __forceinline__ float plane_eval(float x, float y, float a, float b, float c) {
  return fadd(fadd(fmul(x, a), fmul(y, b)), c);
}

// obj = (pix*2)/(float)(res-1) - 1.0 (vfRayKernelCPU.cc:250,254): float
// quotient, then a double subtraction stored as float, which is the float
// subtraction (q - 1 is exact in double; one rounding to float either way).
// pix*2 < 2^24 is exact as a float.
__device__ __forceinline__ float obj_coord(uint32_t pix, uint32_t res) {
  return fsub(fdiv((float)(pix * 2u), (float)(res - 1u)), 1.0f);
}

// The same with the division through rres = __drcp_rn((double)(float)(res-1))
// (div_by: the quotient is 0 or at least 2/(res-1), in the normal range).
__device__ __forceinline__ float obj_coord_r(uint32_t pix, double rres) {
  return fsub(div_by((float)(pix * 2u), rres), 1.0f);
}

// (uint)((res - 1.0) * (x + 1.0) / 2.0) in double (vfRayKernelCPU.cc:158-159),
// converted the way the x86-64 reference binary converts: truncate to a
// 64-bit integer and keep the low 32 bits.
__device__ __forceinline__ uint32_t to_pixel(float x, uint32_t res) {
  // halving is exact, so the division by 2.0 is a multiplication by 0.5
  double d = dmul(dmul(dsub((double)res, 1.0), dadd((double)x, 1.0)), 0.5);
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

// psi-table coordinate of one extinction tau (vfRayKernelCPU.cc:462-471):
// gamma = tau / (1.0 + tau) in double, stored to float; tc = gamma + 0.5/512;
// the step ends when tc is outside [0, 1]; the coordinate is (uint)(tc*512).
// Returns that coordinate (at most 511), or -1 when the step ends.
//
// The quotient only selects an integer, so it is first estimated in float:
// for 0 < tau < 2^20, g = __fdividef(tau, 1 + tau) is within 2^-21.4 of
// tau / (1 + tau) (2 ulp for the quotient, half an ulp for the float sum),
// and so is the reference's double quotient (within 2^-52).  The floats
// lo = RD(g - 2^-20) and hi = RU(g + 2^-20) then bracket the reference's
// (float)gamma, and tc and the coordinate are non-decreasing in gamma: when
// lo and hi give the same coordinate (all but about one case in 2^10) it is
// the reference's.  The other cases take the double division, as written
// in the reference.  floor(tc * 512) for tc in [0, 1] is read off
// RD(tc * 512 + 2^23) (tc * 512 is exact), which needs no conversion unit.
static __device__ __noinline__ int psi_coord_double(float tau) {
  const double t = (double)tau;
  const float g = t == 0.0 ? 0.0f : (float)ddiv(t, dadd(1.0, t));
  const float tc = fadd(g, 0.5f / 512.0f);  // one float rounding either way
  if ((tc < 0.0f) || (tc > 1.0f)) return -1;
  return (int)min((uint32_t)fmul(tc, 512.0f), 511u);
}

// The bracket alone: the coordinate (-1 to 511 whatever tau is, so it can
// index the table), and in ok whether it is the reference's.
__device__ __forceinline__ int psi_coord_fast(float tau, bool& ok) {
  // the bracket, computed for every tau (tau = 0 gives coordinate 0 here,
  // as gamma = 0 and tc = 2^-10 do in the reference); only its verdict
  // depends on the domain 0 <= tau < 2^20
  const float g = __fdividef(tau, fadd(1.0f, tau));
  const float tlo = fadd(__fsub_rd(g, 0x1p-20f), 0x1p-10f);
  const float thi = fadd(__fadd_ru(g, 0x1p-20f), 0x1p-10f);
  const float flo = __fmaf_rd(tlo, 512.0f, 0x1p23f);
  const float fhi = __fmaf_rd(thi, 512.0f, 0x1p23f);
  const bool out = tlo > 1.0f;
  ok = tau >= 0.0f && tau < 1048576.0f && (out || (thi <= 1.0f && flo == fhi));
  return out ? -1 : (int)min(__float_as_uint(flo) - 0x4b000000u, 511u);
}

__device__ __forceinline__ int psi_coord(float tau) {
  bool ok;
  int r = psi_coord_fast(tau, ok);
  if (!ok) r = psi_coord_double(tau);
  return r;
}

// zeta = (float)exp(x) for the double x = -(tau_f*0.5 + tau_b*0.5)
// (vfRayKernelCPU.cc:459).  Table-driven exponential (P. T. P. Tang, "Table-
// driven implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15(2), 1989): x = (64m + j) ln2/64 + r with
// |r| <= ln2/128, exp(x) = 2^m * 2^(j/64) * p(r), p the degree-4 Taylor
// polynomial.  Its relative error is below 2^-44.4 (truncation
// (ln2/128)^5/120, plus a few roundings), i.e. under 360 units in the last
// place of the double result, and the reference's double exp is within
// 0.52 of those units of the true value.  Rounded to float, the estimate
// then gives the reference's zeta unless the 29 bits that rounding drops
// lie within 1024 units of the half-way pattern 2^28 (about one case in
// 2^18): those cases, and x outside [-80, 0], take the double exp.
// e2tab holds 2^(j/64), j = 0..63, rounded to double.  zeta_fast returns the
// estimate rounded to float and, in ok, whether it is the reference's zeta;
// zeta_of takes the double exp when it is not.
__device__ __forceinline__ float zeta_fast(double x, const double* e2tab, bool& ok) {
  // computed for every x (e2tab is indexed in range whatever x is); only
  // the verdict depends on the domain -80 <= x <= 0
  const double kShift = 0x1.8p52;  // adding 1.5 * 2^52 rounds to an integer
  const double t = __fma_rn(x, 0x1.71547652b82fep+6 /* 64 / ln2 */, kShift);
  const int k = __double2loint(t);  // round(x * 64 / ln2), -7400 <= k <= 0 in the domain
  const double kd = dsub(t, kShift);
  double r = __fma_rn(-kd, 0x1.62e42fefa39efp-7, x);   // ln2/64, leading part
  r = __fma_rn(-kd, 0x1.abc9e3b39803fp-62, r);         // ln2/64, trailing part
  double p = __fma_rn(r, 1.0 / 24.0, 1.0 / 6.0);
  p = __fma_rn(p, r, 0.5);
  p = __fma_rn(p, r, 1.0);
  p = __fma_rn(p, r, 1.0);
  double e = dmul(e2tab[k & 63], p);
  // times 2^(k >> 6): the exponent field stays far above the subnormals
  e = __hiloint2double(__double2hiint(e) + (k >> 6) * (1 << 20), __double2loint(e));
  const uint32_t dropped = (uint32_t)__double2loint(e) & 0x1fffffffu;
  ok = x >= -80.0 && x <= 0.0 && dropped - (0x10000000u - 1024u) > 2048u;
  return (float)e;
}

__device__ __forceinline__ float zeta_of(double x, const double* e2tab) {
  bool ok;
  float z = zeta_fast(x, e2tab, ok);
  if (!ok) z = (float)exp(x);
  return z;
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
