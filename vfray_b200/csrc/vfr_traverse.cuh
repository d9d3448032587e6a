// Stage (c): tet-to-tet traversal with partial pre-integration
// (vfRayKernelCPU.cc:173-566), one lane per ray, persistent warps.
//
// Per-lane state machine: a lane walks up to two tets per loop pass; when its
// ray ends it writes the pixel, and once enough lanes of the warp are idle
// the warp refills them from the batch's single ray queue (one
// warp-aggregated atomicAdd), so lanes do not wait for the longest ray of
// their warp.  The kernel is bound by instruction issue, so the step is
// written to keep lanes converged: its arithmetic is branch-free, its rare
// exact fallbacks (psi coordinate, exp, plane re-solve) are taken in one
// block after the fast path, and every way a step can end is a status
// rather than an early return.  The current tet's 4 vertices live in
// shared memory, one slot each per thread, and a per-ray map names the slot
// of each vertex in the entry face's rotation (r_j = local vertex
// (f + j) & 3): the three exit candidates (f+1, f+2, f+3) read r_1..r_3
// through it, candidate i using (r_i, r_i+1, r_i+2).  Moving to the next tet
// stores its one new vertex in the slot of the vertex left behind and
// rewrites the map, a permutation of slot numbers where registers rotated
// by the entry face took 48 selects per step (2.4 % faster, and no
// spills at 3 CTAs per SM).  Once the exit face is known, a step issues its
// two loads together: the next tet's 32-byte walk record and the one vertex
// the next tet does not share with this one (its id is in this tet's record),
// so one memory round trip per step.
#pragma once
#include "vfr_jobs.cuh"

namespace vfr {

// One exit candidate (vfRayKernelCPU.cc:312-348), branch-free.  The slack
// test (double)(c1+c2) <= (double)cr + 1e-12 (:341-342) is decided in float:
// for a float sum s and cr >= 0x2b8cbccd (faces below RDELTA are skipped) it
// holds exactly when s - cr rounded to float is at most 0x2b8cbccc, the
// largest float below 1e-12.  For s <= cr both hold; for cr < s <= 2cr the
// difference is exact (Sterbenz) and a multiple of ulp(cr) >= 2^-63, and no
// such multiple lies within the double rounding error of cr + 1e-12 (below
// 2^(k-28) for multiples of 2^k) of 1e-12, whose distance to the multiples of
// 2^-63 is 2^-67.8; for s > 2cr the difference exceeds cr > 1e-12.
//
// The reference swaps v1 and v2 and negates cr when cr < 0 (:323-330).  Its
// products then become c1' = v2x v0y - v2y v0x = -c2 and c2' = -c1 exactly
// (rounded products and differences are symmetric), and its sum and slack
// difference are the negations of the unswapped ones.  So the swap is a sign
// flip of (c1, c2, sum - cr): applied by xor-ing the sign of cr into them.
//
// v2 = c - a is passed in: candidate 3's (r1 - r3) is the negation of
// candidate 1's (r3 - r1), exact under round-to-nearest but for the sign of
// a zero, and that sign cannot change the test: a zero v2 component only
// changes the sign of a product that is zero, so of a sum or difference
// that is zero; cr = 0 is skipped, and c1, c2 and the slack difference are
// only compared with 0 and with 0x2b8cbccc, where -0 and +0 agree.
__device__ __forceinline__ bool exit_test_v2(const float4& a, const float4& b, float v2x,
                                             float v2y, float ox, float oy) {
  const float v1x = fsub(b.x, a.x), v1y = fsub(b.y, a.y);
  const float cr = fsub(fmul(v1x, v2y), fmul(v1y, v2x));
  const bool skip = below_rdelta(cr);
  const float v0x = fsub(ox, a.x), v0y = fsub(oy, a.y);
  const float c1 = fsub(fmul(v1x, v0y), fmul(v1y, v0x));
  const float c2 = fsub(fmul(v0x, v2y), fmul(v0y, v2x));
  const float d = fsub(fadd(c1, c2), cr);
  const uint32_t sg = __float_as_uint(cr) & 0x80000000u;
  const float c1s = __uint_as_float(__float_as_uint(c1) ^ sg);
  const float c2s = __uint_as_float(__float_as_uint(c2) ^ sg);
  const float ds = __uint_as_float(__float_as_uint(d) ^ sg);
  return !skip && (c1s >= 0.0f) && (c2s >= 0.0f) && (ds <= __uint_as_float(0x2b8cbcccu));
}

__device__ __forceinline__ bool exit_test(const float4& a, const float4& b, const float4& c,
                                          float ox, float oy) {
  return exit_test_v2(a, b, fsub(c.x, a.x), fsub(c.y, a.y), ox, oy);
}

// Per-CTA copies of the small tables: the transfer function's alpha in float
// and its colour promoted to double (the compositing multiplies colours in
// double, vfRayKernelCPU.cc:473-476, so the promotion is done once here), and
// 2^(j/64), j = 0..63, for zeta_of.
struct SharedTables {
  double2 rg[256];
  double b[256];
  float a[256];
  double e2[64];
};

// A ray's walk is a function of its state (tet, entry face) alone: the pixel
// is fixed, so a state that comes back means the reference's while loop
// never ends (a cycle among tets around a projected edge, which the
// inclusive exit tests with slack allow on meshes whose tets list their
// vertices in arbitrary order).  Rays longer than kWatchSteps iterations are
// watched: the state is saved at every power-of-two iteration count and
// compared with the state of every later iteration (Brent), which stops a
// cycling ray within about two periods.  Shorter rays pay one comparison
// per pass of two steps.  The oracle applies the same rule, so steps stay
// comparable.
constexpr uint32_t kWatchSteps = 4095;

// The watched state of each thread's ray (tet << 2 | entry face, ~0 =
// none), in shared memory: it is written when a segment starts and read
// only by watched iterations, so it takes no register of the step.
__shared__ uint32_t s_watch_saved[256];

// The current tet's 4 vertices, per thread, in 4 slots; a ray's map says
// which slot holds the vertex the entry-face rotation calls j (r_j =
// vertex (f + j) & 3).  Moving to the next tet stores the one new vertex in
// the slot of the vertex it replaces and rewrites the map, instead of
// permuting 16 registers with selects.
__shared__ float4 s_vtx[4][256];
constexpr uint32_t kIdentityMap = 0u | 1u << 2 | 2u << 4 | 3u << 6;
__device__ __forceinline__ uint32_t slot_of(uint32_t m, uint32_t j) { return (m >> (2u * (j & 3u))) & 3u; }
__device__ __forceinline__ float4 vtx(uint32_t slot) { return s_vtx[slot][threadIdx.x]; }
__device__ __forceinline__ float4 vtx_xy(uint32_t slot) {
  const float2 v = *reinterpret_cast<const float2*>(&s_vtx[slot][threadIdx.x]);
  return make_float4(v.x, v.y, 0.0f, 0.0f);
}

struct Ray {
  uint32_t map;                // slot of rotated vertex j in s_vtx: bits 2j..2j+1
  WalkRec w;                   // walk record of the current tet
  const WalkRec* walk;         // this job's mesh and view vertices
  const float4* vert;
  uint32_t j, nT;
  uint32_t nV;                 // checked build: vertex ids are compared with it
  uint32_t watch;              // min(kWatchSteps, step cap): longer rays are checked
  double rmaxEdge;             // 1 / maxEdgeLength, correctly rounded (div_by)
  uint32_t cbi;                // colorBack: its transfer-function entry
  uint32_t t, f, p, iters;
  float ox, oy, zp;
  float ar, ag, ab, tr, lastZ;
  // composited mode: this pixel's entry list and the next entry to take
  uint32_t ea, en, de;
  float exitZ;
  // served form: the job (its table entry lives in the server's arena) and
  // its completion flag
  const JobDev* jp;
  uint32_t* done;
};

// Read-only loads of the mesh through the non-coherent path (the arrays are
// not written while the traversal runs).
__device__ __forceinline__ WalkRec ldg_walk(const WalkRec* w, uint32_t t) {
  const uint4* p = reinterpret_cast<const uint4*>(w + t);
  WalkRec r;
  r.n = __ldg(p);
  r.q = __ldg(p + 1);
  return r;
}

// Start a segment in tet t through its face f, with entry depth zp and the
// back colour's transfer-function entry cbi (:256-279).  False (checked build
// only): the tet or one of its vertex ids is out of range, and nothing was
// loaded.
__device__ __forceinline__ bool begin_segment_at(const JobDev& J, Ray& R, uint32_t t, uint32_t f,
                                                 float zp, uint32_t cbi) {
  if (id_bad(t, J.nT)) return false;
  R.t = t;
  R.f = f;
  const uint4 id = __ldg(J.tet + t);
  if (id_bad(id.x, J.nV) || id_bad(id.y, J.nV) || id_bad(id.z, J.nV) || id_bad(id.w, J.nV))
    return false;
  R.w = ldg_walk(R.walk, t);
  s_vtx[0][threadIdx.x] = __ldg(R.vert + sel4(id, f));
  s_vtx[1][threadIdx.x] = __ldg(R.vert + sel4(id, (f + 1) & 3u));
  s_vtx[2][threadIdx.x] = __ldg(R.vert + sel4(id, (f + 2) & 3u));
  s_vtx[3][threadIdx.x] = __ldg(R.vert + sel4(id, (f + 3) & 3u));
  R.map = kIdentityMap;
  R.zp = zp;
  R.lastZ = zp;
  R.cbi = cbi;
  s_watch_saved[threadIdx.x] = 0xffffffffu;  // a new segment walks other states
  return true;
}


// Composited mode: the pixel's next entry in its list, which stage (b)
// wrote in descending (depth, face) order, skipping entries above the depth
// where the previous segment left the mesh.  Returns false when the list is
// done (or, checked build only, holds an id out of range: VFR_DEV_RANGE).
__device__ __forceinline__ bool next_entry(const TraverseParams& P, const JobDev& J, Ray& R,
                                           uint32_t& status) {
  bool bad = false;
  while (R.de < R.en) {
    if (id_bad(R.ea + R.de, J.ent_cap)) {
      bad = true;
      break;
    }
    const uint4 q = J.ent[R.ea + R.de];
    ++R.de;
    const float z = __uint_as_float(q.x);
    if (z > R.exitZ) continue;  // behind the ray already
    // stage (b) resolved the segment's start: tet << 2 | entry face, and the
    // back colour's transfer-function entry
    if (begin_segment_at(J, R, q.z >> 2, q.z & 3u, z, q.w)) return true;
    bad = true;
    break;
  }
  if (bad) status |= kDevRange;
  return false;
}

__device__ __forceinline__ void finish_pixel(const JobDev& J, const Ray& R) {
  float c[3] = {R.ar, R.ag, R.ab};
#pragma unroll
  for (int k = 0; k < 3; ++k) c[k] = (c[k] > 1.0f) ? 1.0f : c[k];  // :546-548
  if (J.rgb8) {
    uint8_t* o = J.rgb8 + 3 * (size_t)R.p;
#pragma unroll
    for (int k = 0; k < 3; ++k) o[k] = (uint8_t)__float2int_rz(fmul(255.0f, c[k]));  // :550-552
  }
  if (J.rgba) J.rgba[R.p] = make_float4(c[0], c[1], c[2], fsub(1.0f, R.tr));
  if (J.steps) J.steps[R.p] = R.iters;
}

enum StepResult : uint32_t { kContinue = 0, kSegmentEnd = 1, kCycle = 2, kCap = 3, kRange = 4 };

// The step cap of a ray of this job: the option, or 4 nT + 64 (a walk that
// repeats no state has at most 4 nT iterations).
__device__ __forceinline__ uint32_t step_cap_of(const TraverseParams& P, uint32_t nT) {
  return P.step_cap ? P.step_cap : min(4u * nT + 64u, 0x7fffffffu);
}

// Rare: an iteration beyond the watch threshold.  The cap, then Brent's
// check of the state this iteration starts from (R.t, R.f are still the
// current tet and entry face).
__device__ __forceinline__ uint32_t watched_step(const TraverseParams& P, Ray& R) {
  if (R.iters > step_cap_of(P, R.nT)) return kCap;
  const uint32_t key = (R.t << 2) | R.f;  // nT < 2^30 (checked at upload)
  uint32_t& saved = s_watch_saved[threadIdx.x];
  if (key == saved) return kCycle;
  if ((R.iters & (R.iters - 1u)) == 0u) saved = key;
  return kContinue;
}

// The step's depth difference and extinctions from the exit face's depth zn
// and scalar sn at the pixel (:437-457): dz = |zPrev - zNext| (0 below
// RDELTA) / maxEdgeLength, the front's transfer-function entry, tau of the
// front and of the back.  The step ends when sn is outside [0, 1] (:446).
__device__ __forceinline__ void extinction(const SharedTables& S, const Ray& R, float zn, float sn,
                                           bool& end, uint32_t& tfi, float& taux,
                                           float& tauy) {
  float dz = fsub(R.zp, zn);
  dz = dz < 0.0f ? -dz : dz;
  dz = below_rdelta(dz) ? 0.0f : dz;
  end = end || (sn < 0.0f) || (sn > 1.0f);
  // dz /= maxEdgeLength (:450): dz is 0 or at least 1e-12 and maxEdgeLength
  // below 2^80 (checked at upload; view set-up gives at most 2 sqrt 3), so
  // the quotient is never subnormal and div_by is exact
  dz = div_by(dz, R.rmaxEdge);
  tfi = min((uint32_t)fmul(255.0f, sn), 255u);  // colorFront (:452)
  taux = fmul(S.a[tfi], dz);
  tauy = fmul(S.a[R.cbi], dz);
}

// zeta's argument -(tau_f*0.5 + tau_b*0.5), in double (:459).  Halving is
// exact and commutes with rounding (a double sum of two floats is never
// subnormal), so it is the sum times -0.5: one multiplication fewer.
__device__ __forceinline__ double zeta_arg(float taux, float tauy) {
  return dmul(dadd((double)taux, (double)tauy), -0.5);
}

struct StepColour {
  float r, g, b, t;
};

// The step's colour and transparency (:461-483) from the front's
// transfer-function entry, zeta and the psi coordinates (any of -1..511:
// the table is indexed in range whatever they are).  kUnitZeta: zeta is
// known to lie in [0, 1] (the fast path's certified zeta), which lets
// 1 - a be formed without a conversion.
template <bool kUnitZeta>
__device__ __forceinline__ StepColour composite(const TraverseParams& P, const SharedTables& S,
                                               const Ray& R, uint32_t tfi, float zeta, int ci,
                                               int cj) {
  const double psi = (double)__ldg(P.psi + (uint32_t)max(ci, 0) * 512u + (uint32_t)max(cj, 0));
  const double dzeta = (double)zeta;
  const double ca = dsub(1.0, psi), cbk = dsub(psi, dzeta);
  const double2 frg = S.rg[tfi], brg = S.rg[R.cbi];
  const double fbl = S.b[tfi], bbl = S.b[R.cbi];
  const float fr = (float)dadd(dmul(frg.x, ca), dmul(brg.x, cbk));
  const float fg = (float)dadd(dmul(frg.y, ca), dmul(brg.y, cbk));
  const float fb = (float)dadd(dmul(fbl, ca), dmul(bbl, cbk));
  // keep = 1 - a with a = (float)(1.0 - zeta) (innocuous double rounding);
  // 1 - a is exact.  For zeta in [0, 1], a is 1 - zeta exactly when
  // zeta >= 0.5 and otherwise 1 - zeta rounded to the 2^-24 grid of the
  // floats in [0.5, 1]; either way 1 - a is zeta rounded to a multiple of
  // 2^-24, ties to even, which adding and removing 1.5 * 2^28 in double
  // gives.
  double keep;
  if (kUnitZeta) {
    keep = dsub(dadd(dzeta, 0x1.8p28), 0x1.8p28);
  } else {
    const float fw = fsub(1.0f, zeta);
    keep = dsub(1.0, (double)fw);
  }
  StepColour o;
  o.r = (float)dadd((double)fr, dmul(keep, (double)R.ar));
  o.g = (float)dadd((double)fg, dmul(keep, (double)R.ag));
  o.b = (float)dadd((double)fb, dmul(keep, (double)R.ab));
  o.t = fmul(R.tr, zeta);
  return o;
}

// One iteration of the reference's while loop (:302-542).  The ways it can
// end before compositing (no exit face, scalar or psi coordinate out of
// range; a cycle or the step cap in watched iterations; an id out of range
// in the checked build) are folded into one flag and the arithmetic runs on
// for every lane; the colour is only committed while the flag says to go
// on, so no lane takes an early branch.  The exact fallbacks of the
// plane, zeta and the psi coordinates are gathered into one rare block
// after the fast path, so the step from the exit tests to the advance is
// one straight run of code that the compiler schedules as a whole.
//
// kWatched: the iteration is past the watch threshold and checked for a
// cycle first (its verdict ends the step like the cap: nothing of it is
// committed).  The loop below takes the unwatched form, which carries no
// trace of the check, for every pass that stays below the threshold.
template <bool kWatched, bool kServe = false>
__device__ __forceinline__ uint32_t step(const TraverseParams& P, const SharedTables& S, Ray& R) {
  ++R.iters;
  const uint32_t wst = kWatched ? watched_step(P, R) : (uint32_t)kContinue;
  bool end = wst != kContinue;
  const uint32_t m = R.map;
  const float4 r0 = vtx_xy(slot_of(m, 0)), r1 = vtx_xy(slot_of(m, 1)), r2 = vtx_xy(slot_of(m, 2)),
               r3 = vtx_xy(slot_of(m, 3));
  const float e13x = fsub(r3.x, r1.x), e13y = fsub(r3.y, r1.y);
  const bool h1 = exit_test_v2(r1, r2, e13x, e13y, R.ox, R.oy);
  const bool h2 = exit_test(r2, r3, r0, R.ox, R.oy);
  const bool h3 = exit_test_v2(r3, r0, -e13x, -e13y, R.ox, R.oy);
  const uint32_t i = h1 ? 1u : (h2 ? 2u : (h3 ? 3u : 0u));
  end = end || i == 0;  // :353 no exit face
  const uint32_t ex = (R.f + i) & 3u;
  const bool xo = (ex & 1u) != 0u, xh = (ex & 2u) != 0u;
  const uint32_t tn = xh ? (xo ? R.w.n.w : R.w.n.z) : (xo ? R.w.n.y : R.w.n.x);
  const uint32_t q = xh ? (xo ? R.w.q.w : R.w.q.z) : (xo ? R.w.q.y : R.w.q.x);
  const bool leaving = (tn == R.t);
  // both loads of the step, issued before the plane solve that hides them,
  // whatever the exit: tn and the vertex word are valid ids for every face
  // (a boundary face's record names the tet itself and vertex 0; the mesh's
  // ids were validated at upload), so no branch cuts the step.  The checked
  // build compares them first.
  bool bad = id_bad(tn, R.nT) || id_bad(q & 0x07ffffffu, R.nV);
  end = end || bad;
  WalkRec N = R.w;
  float4 nv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (!bad) {
    N = ldg_walk(R.walk, tn);
    nv = __ldg(R.vert + (q & 0x07ffffffu));
  }
  // exit face (ex, ex+1, ex+2) = (r_i, r_i+1, r_i+2)
  const float4 a = vtx(slot_of(m, i)), b = vtx(slot_of(m, i + 1u)), c = vtx(slot_of(m, i + 2u));
  // fast path: every quantity from its branch-free estimate, with a flag
  // where the estimate may differ from the reference's value
  Plane nf;
  const bool plane_ok = face_plane_fast(a, b, c, nf);
  float zn = plane_eval(R.ox, R.oy, nf.zx, nf.zy, nf.zz);
  const bool end0 = end;
  uint32_t tfi;
  float taux, tauy;
  extinction(S, R, zn, plane_eval(R.ox, R.oy, nf.sx, nf.sy, nf.sz), end, tfi, taux, tauy);
  bool z_ok, i_ok, j_ok;
  float zeta = zeta_fast(zeta_arg(taux, tauy), S.e2, z_ok);
  int ci = psi_coord_fast(taux, i_ok), cj = psi_coord_fast(tauy, j_ok);
  StepColour col = composite<true>(P, S, R, tfi, zeta, ci, cj);
  // rare: the exact path for the lanes whose plane, zeta or psi coordinate
  // was not certified (a plane with a tiny coefficient; about one psi
  // coordinate in 2^10), before anything is committed
  if ((!plane_ok && !end0) || (!end && !(z_ok && i_ok && j_ok))) {
    if (!plane_ok) {
      face_plane_ieee(a, b, c, nf);
      zn = plane_eval(R.ox, R.oy, nf.zx, nf.zy, nf.zz);
      end = end0;
      extinction(S, R, zn, plane_eval(R.ox, R.oy, nf.sx, nf.sy, nf.sz), end, tfi, taux, tauy);
    }
    zeta = zeta_of(zeta_arg(taux, tauy), S.e2);
    ci = psi_coord(taux);
    cj = psi_coord(tauy);
    col = composite<false>(P, S, R, tfi, zeta, ci, cj);
  }
  end = end || (ci | cj) < 0;  // :468
  if (!end) {
    R.ar = col.r;
    R.ag = col.g;
    R.ab = col.b;
    R.tr = col.t;
    R.lastZ = zn;
    R.cbi = tfi;
  }
  const bool go_on = !end && !leaving;  // :535
  // advance to tn through its face fn: slots fn..fn+2 are the exit face's
  // vertices in tn's order (permutation code), slot fn+3 is the loaded
  // vertex.  Done whatever the status: once a ray's segment ends, nothing
  // reads its walk state before begin_segment sets it again.
  const uint32_t fn = (q >> 27) & 3u, code = q >> 29;
  {
    // the exit face's vertices are rotated i, i + 1, i + 2; slot fn + k of
    // the next tet holds the one the permutation code names, and the new
    // vertex takes the slot of the one left behind (rotated i + 3)
    const uint32_t pc = perm_code(code);
    const uint32_t s0 = slot_of(m, i + (pc & 3u)), s1 = slot_of(m, i + ((pc >> 2) & 3u));
    const uint32_t s2 = slot_of(m, i + ((pc >> 4) & 3u)), sd = slot_of(m, i + 3u);
    s_vtx[sd][threadIdx.x] = nv;
    R.map = s0 | (s1 << 2) | (s2 << 4) | (sd << 6);
  }
  if (go_on && code >= 6) {
    // shared face not matched by vertex ids: reload the tet's vertices
    const uint4 id = __ldg((kServe ? R.jp->tet : P.jobs[R.j].tet) + tn);
    bad = id_bad(id.x, R.nV) || id_bad(id.y, R.nV) || id_bad(id.z, R.nV) || id_bad(id.w, R.nV);
    if (!bad) {
      s_vtx[0][threadIdx.x] = __ldg(R.vert + sel4(id, fn));
      s_vtx[1][threadIdx.x] = __ldg(R.vert + sel4(id, (fn + 1) & 3u));
      s_vtx[2][threadIdx.x] = __ldg(R.vert + sel4(id, (fn + 2) & 3u));
      s_vtx[3][threadIdx.x] = __ldg(R.vert + sel4(id, (fn + 3) & 3u));
      R.map = kIdentityMap;
    }
  }
  R.w = N;
  R.t = tn;
  R.f = fn;
  R.zp = zn;
  if (wst != kContinue) return wst;
  if (bad) return kRange;
  return go_on ? (uint32_t)kContinue : (uint32_t)kSegmentEnd;
}

// Start the ray of the job's local ray index `local`: its pixel, the
// pixel's object coordinates, and its first segment -- the winning entry
// face's, from the start record stage (b) wrote (reference mode: three
// levels of dependent loads, the record, then the tet and its walk record,
// then the vertices), or the first entry of the pixel's list (composited
// mode; kMode 2 takes the mode from the job).  Returns whether the ray
// walks; a composited pixel without a usable entry is finished here.
template <int kMode>
__device__ __forceinline__ bool start_ray(const TraverseParams& P, const JobDev& J, Ray& R,
                                          uint32_t local, uint32_t& status) {
  R.walk = J.walk;
  R.vert = J.vert;
  R.nT = J.nT;
  R.nV = J.nV;
  R.watch = min(kWatchSteps, step_cap_of(P, J.nT));
  R.rmaxEdge = __drcp_rn((double)job_maxedge(J));
  const RayStart rs = J.rays[local];
  R.p = rs.p;
  if (id_bad(R.p, J.W * J.H)) {
    status |= kDevRange;
    return false;
  }
  const uint32_t x = R.p % J.W, y = R.p / J.W;
  R.ox = obj_coord(x, J.W);
  R.oy = obj_coord(y, J.H);
  R.ar = R.ag = R.ab = 0.0f;
  R.tr = 1.0f;
  R.iters = 0;
  const bool ref = kMode == 0 || (kMode == 2 && J.mode == 0);
  if (ref) {  // stage (b) resolved the winning face's segment start
    if (!begin_segment_at(J, R, rs.tf >> 2, rs.tf & 3u, __uint_as_float(rs.zp), rs.cbi)) {
      status |= kDevRange;
      return false;
    }
    return true;
  }
  R.ea = J.ent_off[R.p];
  R.en = J.ent_cnt[R.p];
  R.exitZ = INFINITY;
  R.de = 0;
  if (next_entry(P, J, R, status)) return true;
  finish_pixel(J, R);
  return false;
}

// Per-lane tallies of tet-walk steps and status bits, flushed to the job's
// counters when the lane moves to another job and at the end.
struct Tally {
  uint32_t j;
  unsigned long long steps;
  uint32_t status;
};

__device__ __forceinline__ void flush(const TraverseParams& P, Tally& T) {
  if (T.j != 0xffffffffu) {
    ViewCounters* c = P.jobs[T.j].ctr;
    if (T.steps) atomicAdd(&c->steps, T.steps);
    if (T.status) atomicOr(&c->status, T.status);
  }
  T.steps = 0;
  T.status = 0;
}

// kMinBlocks: CTAs of 256 threads the register budget must allow per SM
// (2: no spills; 3: 80 registers, a few spilled to L1).
__device__ __forceinline__ void load_tables(const TraverseParams& P, SharedTables& S) {
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
    const float4 c = P.tf[i];
    S.rg[i] = make_double2((double)c.x, (double)c.y);
    S.b[i] = (double)c.z;
    S.a[i] = c.w;
  }
  for (uint32_t i = threadIdx.x; i < 64; i += blockDim.x) S.e2[i] = P.e2tab[i];
  __syncthreads();
}

template <int kMode, int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) traverse_kernel(TraverseParams P) {
  __shared__ SharedTables S;
  load_tables(P, S);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint32_t nrays = P.ray_pref[P.njobs];
  const uint32_t refill = P.refill ? P.refill : 1u;
  Tally T = {0xffffffffu, 0ull, 0u};
  bool active = false, exhausted = false;
  Ray R;
  for (;;) {
    const uint32_t idle = __ballot_sync(0xffffffffu, !active);
    if (idle && !exhausted && ((uint32_t)__popc(idle) >= refill || idle == 0xffffffffu)) {
      const uint32_t leader = __ffs(idle) - 1u, k = __popc(idle);
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(P.queue, k);
      base = __shfl_sync(0xffffffffu, base, leader);
      if (base + k >= nrays) exhausted = true;
      if (!active) {
        const uint32_t g = base + __popc(idle & lt_mask);
        if (g < nrays) {
          const uint32_t j = job_of(P.ray_pref, P.njobs, g);
          const JobDev& J = P.jobs[j];
          if (j != T.j) {
            flush(P, T);
            T.j = j;
          }
          R.j = j;
          active = start_ray<kMode>(P, J, R, g - P.ray_pref[j], T.status);
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (!active) continue;
    // two steps per pass of the loop: the refill test runs half as often.
    // A pass that would reach the watch threshold takes one watched step
    // instead (rare: rays longer than kWatchSteps iterations).
    uint32_t res;
    if (R.iters + 2u <= R.watch) {
      res = step<false>(P, S, R);
      if (res == kContinue) res = step<false>(P, S, R);
    } else {
      res = step<true>(P, S, R);
    }
    if (res == kContinue) continue;
    if (res == kSegmentEnd) {
      if (kMode == 1) {
        R.exitZ = R.lastZ;
        if (next_entry(P, P.jobs[R.j], R, T.status)) continue;
      }
      finish_pixel(P.jobs[R.j], R);
    } else if (res == kCycle || res == kCap) {
      // the pixel keeps what the ray composited before it was stopped
      T.status |= res == kCycle ? 32u : 2u;  // VFR_DEV_CYCLE, VFR_DEV_STEP_CAP
      finish_pixel(P.jobs[R.j], R);
    } else {
      T.status |= 4u;
    }
    T.steps += R.iters;
    active = false;
  }
  flush(P, T);
}

// ---------------------------------------------------------------- served

// A served ray has ended: its steps and status go to its job's counters,
// then its count of finished rays; the lane that finishes the job's last ray
// sets the job's completion flag in mapped host memory.  Each lane's pixel
// and counter writes are fenced before its count, and the last lane fences
// at system scope before the flag, so everything the job wrote is visible
// to the host's copy once the flag is.
__device__ __forceinline__ void served_ray_done(const Ray& R, uint32_t status) {
  ViewCounters* c = R.jp->ctr;
  atomicAdd(&c->steps, (unsigned long long)R.iters);
  if (status) atomicOr(&c->status, status);
  __threadfence();
  const uint32_t n = atomicAdd(&c->rays_done, 1u) + 1u;
  if (n == *(volatile const uint32_t*)&c->nrays) {
    __threadfence_system();
    *(volatile uint32_t*)R.done = 1u;
  }
}

// A segment-table entry read through L2 only (ld.global.cg): entries are
// 40 bytes, several to a cache line, and each is written (once per epoch)
// after this launch may already have cached the line for an earlier entry.
__device__ __forceinline__ SegDev load_seg(const SegDev* p) {
  static_assert(sizeof(SegDev) == 40, "segment-table entry layout");
  const unsigned long long* w = reinterpret_cast<const unsigned long long*>(p);
  SegDev d;
  unsigned long long* o = reinterpret_cast<unsigned long long*>(&d);
#pragma unroll
  for (int i = 0; i < 5; ++i) o[i] = __ldcg(w + i);
  return d;
}

// The same for every lane of the warp whose ray ended in this pass (fin),
// aggregated per job: one fence and one atomic per job and pass.  Called by
// the whole warp.  The lanes' pixel writes are ordered before the leader's
// fence by __syncwarp, and the leader's count after its fence.
__device__ __forceinline__ void served_rays_done(const Ray& R, bool fin, uint32_t status) {
  const uint32_t finm = __ballot_sync(0xffffffffu, fin);
  if (!finm) return;
  if (fin) {
    const uint32_t peers = __match_any_sync(finm, (unsigned long long)(uintptr_t)R.jp);
    // steps as two 16-bit halves, so the 32-bit warp sums cannot overflow
    const uint32_t lo = __reduce_add_sync(peers, R.iters & 0xffffu);
    const uint32_t hi = __reduce_add_sync(peers, R.iters >> 16);
    const uint32_t st = __reduce_or_sync(peers, status);
    __syncwarp(peers);
    if ((threadIdx.x & 31u) == (uint32_t)(__ffs(peers) - 1)) {
      ViewCounters* c = R.jp->ctr;
      atomicAdd(&c->steps, ((unsigned long long)hi << 16) + lo);
      if (st) atomicOr(&c->status, st);
      __threadfence();
      const uint32_t n = atomicAdd(&c->rays_done, (uint32_t)__popc(peers)) + __popc(peers);
      if (n == *(volatile const uint32_t*)&c->nrays) {
        __threadfence_system();
        *(volatile uint32_t*)R.done = 1u;
      }
    }
  }
}

// The served form's persistent traversal: one long-lived launch whose warps
// take rays from the published segments in order, oldest first, while the
// host publishes new ones (requests admitted while this launch runs fold
// into it).  A warp holds its place in the segment table: it takes rays from
// its current entry with one atomicAdd on the entry's head and moves on once
// the entry is drained.  Jobs of either mode may be mixed (kMode 2 per job).
// A warp with nothing to do polls for newly published segments: it leaves
// when the host's stop flag is set, or sets VFR_DEV_QUEUE in the control
// word and leaves when it has found nothing for idle_limit microseconds
// (%globaltimer) -- a bounded wait, so a launch never outlives its work by
// much more than that.  The host relaunches it when work arrives after it
// left.
template <int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) serve_kernel(ServeParams SP) {
  const TraverseParams& P = SP.T;
  __shared__ SharedTables S;
  load_tables(P, S);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint32_t refill = P.refill ? P.refill : 1u;
  uint32_t cur = SP.first;  // this warp's entry of the segment table
  // Polling costs: a warp with nothing to do polls the publication count and
  // the stop word (device memory) with plain loads by one lane, backing off
  // from 256 ns to 256 us between polls, and a warp whose claim found
  // nothing while some of its lanes still walk waits 32 passes before it
  // tries again -- thousands of warps polling back to back would make those
  // L2 lines hot spots that slow everything, the preparation kernels beside
  // this launch included.
  unsigned long long idle_since = 0;  // %globaltimer (ns) when the warp found nothing (0: busy)
  uint32_t backoff = 256, quiet = 0;
  bool active = false;
  Ray R;
  for (;;) {
    const uint32_t idle = __ballot_sync(0xffffffffu, !active);
    uint32_t seg = 0xffffffffu;
    if (quiet) --quiet;
    if (idle && (idle == 0xffffffffu || ((uint32_t)__popc(idle) >= refill && quiet == 0))) {
      const uint32_t leader = __ffs(idle) - 1u, k = __popc(idle);
      uint32_t base = 0, nr = 0;
      if (lane == leader) {
        const uint32_t pub = *(volatile const uint32_t*)&SP.ctl->published;
        if (cur < pub) {
          // with the publisher's release, the entries below pub are visible
          __threadfence();
          while (cur < pub) {
            SegDev* sg = SP.segs + cur;
            const uint32_t b = atomicAdd(&sg->head, k);
            const uint32_t n = __ldcg(&sg->nrays);  // written before the entry was published
            if (b < n) {
              base = b;
              nr = n;
              seg = cur;
              break;
            }
            ++cur;  // drained: the next entry
          }
        }
      }
      cur = __shfl_sync(0xffffffffu, cur, leader);
      seg = __shfl_sync(0xffffffffu, seg, leader);
      base = __shfl_sync(0xffffffffu, base, leader);
      nr = __shfl_sync(0xffffffffu, nr, leader);
      __syncwarp();  // the leader's fence after the publication orders the lanes' reads
      if (seg == 0xffffffffu) quiet = 32;
      if (seg != 0xffffffffu && !active) {
        const uint32_t g = base + __popc(idle & lt_mask);
        if (g < nr) {
          const SegDev sg = load_seg(SP.segs + seg);
          const uint32_t j = job_of(sg.ray_pref, sg.njobs, g);
          R.jp = sg.jobs + j;
          R.done = sg.done + j;
          uint32_t status = 0;
          active = start_ray<2>(P, *R.jp, R, g - sg.ray_pref[j], status);
          if (!active) served_ray_done(R, status);
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (seg == 0xffffffffu) {  // nothing published to take: wait, boundedly
        // lane 0's reads decide for the warp, which leaves together
        unsigned long long now;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
        now = __shfl_sync(0xffffffffu, now, 0);
        const uint32_t stop = lane == 0 ? *(volatile const uint32_t*)&SP.ctl->stop : 0u;
        if (__shfl_sync(0xffffffffu, stop, 0)) break;
        if (!idle_since) {
          idle_since = now;
        } else if (now - idle_since > 1000ull * SP.idle_limit) {
          if (lane == 0) atomicOr(&SP.ctl->status, 8u);  // VFR_DEV_QUEUE
          break;
        }
        __nanosleep(backoff);
        backoff = min(2u * backoff, 262144u);
      }
      continue;
    }
    idle_since = 0;
    backoff = 256;
    // every lane goes on to served_rays_done, which syncs the whole warp
    uint32_t res = kContinue;
    if (active) {
      if (R.iters + 2u <= R.watch) {
        res = step<false, true>(P, S, R);
        if (res == kContinue) res = step<false, true>(P, S, R);
      } else {
        res = step<true, true>(P, S, R);
      }
    }
    uint32_t status = 0;
    bool fin = false;
    if (active && res != kContinue) {
      fin = true;
      if (res == kSegmentEnd) {
        if (R.jp->mode == 1) {
          R.exitZ = R.lastZ;
          fin = !next_entry(P, *R.jp, R, status);
        }
        if (fin) finish_pixel(*R.jp, R);
      } else if (res == kCycle || res == kCap) {
        status = res == kCycle ? 32u : 2u;
        finish_pixel(*R.jp, R);
      } else {
        status = 4u;
      }
    }
    served_rays_done(R, fin, status);
    active = active && !fin;
  }
}

// Publishes a prepared segment: its table entry, then (release) the count
// of published entries the served launch acquires.  Jobs without rays are
// complete now: their pixels were cleared by stage (b).
__global__ void publish_kernel(SegDev* segs, ServeCtl* ctl, uint32_t seq, const JobDev* jobs,
                               const uint32_t* ray_pref, uint32_t* done, uint32_t njobs) {
  if (threadIdx.x == 0) {
    SegDev d;
    d.jobs = jobs;
    d.ray_pref = ray_pref;
    d.done = done;
    d.njobs = njobs;
    d.nrays = ray_pref[njobs];
    d.head = 0;
    d.pad = 0;
    segs[seq] = d;
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x)
    if (ray_pref[j + 1] == ray_pref[j]) {
      __threadfence_system();
      *(volatile uint32_t*)(done + j) = 1u;
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&ctl->published), "r"(seq + 1u) : "memory");
  }
}

}  // namespace vfr
