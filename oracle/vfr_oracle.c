/* Test infrastructure: the CPU oracle for the VF-Ray render path.
 *
 * Restates vfRayKernelCPU.cc (findVisibleFaces :51-132, projectVisibleFaces
 * :136-169, vfRay :173-566, with USEPARTIALPREINT 1) and the driver sequence
 * of main.cc:73-224 in plain C.  Every expression keeps the reference's
 * operand order and its float/double mix: float * float stays float, while
 * any operand that is a double literal (1.0, 0.5, RDELTA) promotes the
 * expression to double before the result is stored back into a float.
 * Built with -ffp-contract=off and without fast-math (oracle/Makefile).
 *
 * The reference's 512-slot face cache (vfRayKernelCPU.cc:234-245,369-435) is
 * left out: a hit returns the same plane the code would recompute.
 */
#define _GNU_SOURCE
#include "vfr_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define RDELTA 1e-12 /* vfRayKernelCPU.h:28, a double */
#define ABSF(n) ((n) < 0 ? -(n) : (n))

typedef struct { float x, y, z, w; } f4;

static inline f4 vget(const vo_mesh* m, uint32_t id) {
  const float* p = m->vert + 4 * (size_t)id;
  f4 r = {p[0], p[1], p[2], p[3]};
  return r;
}

static inline f4 tfget(const vo_mesh* m, float s) {
  /* (uint)(255*s), vfRayKernelCPU.cc:279,452; s is in [0,1] here */
  uint32_t i = (uint32_t)(255 * s);
  if (i > 255) i = 255;
  const float* p = m->tf + 4 * i;
  f4 r = {p[0], p[1], p[2], p[3]};
  return r;
}

/* Cramer solve of the face plane through a, b, c for z and s
 * (vfRayKernelCPU.cc:73-122 and :380-429). */
static void plane(f4 a, f4 b, f4 c, vo_face* f) {
  float c0x = a.x, c0y = b.x, c0z = c.x; /* fmCol0: x of the 3 vertices */
  float c1x = a.y, c1y = b.y, c1z = c.y; /* fmCol1: y */
  float det = c0x * (c1y - c1z) - c1x * (c0y - c0z) + ((c0y * c1z) - (c1y * c0z));
  det = (ABSF(det) < RDELTA) ? RDELTA : det;
  float tx = a.z, ty = b.z, tz = c.z;
  float mx = ty - tz;
  float my = (ty * c1z) - (c1y * tz);
  float mz = (c0y * tz) - (ty * c0z);
  f->zx = (tx * (c1y - (c1z)) - (c1x * mx) + my) / det;
  f->zy = ((c0x * mx) - tx * (c0y - (c0z)) + mz) / det;
  f->zz = (c0x * (-my) - (c1x * mz) + tx * (c0y * c1z - c1y * c0z)) / det;
  tx = a.w; ty = b.w; tz = c.w;
  mx = ty - tz;
  my = (ty * c1z) - (c1y * tz);
  mz = (c0y * tz) - (ty * c0z);
  f->sx = (tx * (c1y - (c1z)) - (c1x * mx) + my) / det;
  f->sy = ((c0x * mx) - tx * (c0y - (c0z)) + mz) / det;
  f->sz = (c0x * (-my) - (c1x * mz) + tx * (c0y * c1z - c1y * c0z)) / det;
}

static int mesh_ok(const vo_mesh* m) {
  if (!m || !m->vert || !m->tet || !m->con || !m->extf || !m->tf || !m->psi) return 0;
  if (m->nT >= (1u << 30)) return 0; /* walk states are packed as tet << 2 | face */
  for (size_t i = 0; i < 4 * (size_t)m->nT; ++i)
    if (m->tet[i] >= m->nV || m->con[i] >= m->nT) return 0;
  for (uint32_t e = 0; e < m->nExt; ++e)
    if (m->extf[2 * e] >= m->nT || m->extf[2 * e + 1] > 3) return 0;
  return 1;
}

static inline void face_verts(const vo_mesh* m, uint32_t t, uint32_t f, f4* v0, f4* v1, f4* v2) {
  *v0 = vget(m, m->tet[4 * (size_t)t + ((f + 0) & 3)]);
  *v1 = vget(m, m->tet[4 * (size_t)t + ((f + 1) & 3)]);
  *v2 = vget(m, m->tet[4 * (size_t)t + ((f + 2) & 3)]);
}

void vo_find_visible(const vo_mesh* m, vo_face* out) {
  for (uint32_t e = 0; e < m->nExt; ++e) {
    uint32_t t = m->extf[2 * e], f = m->extf[2 * e + 1];
    f4 v0, v1, v2;
    face_verts(m, t, f, &v0, &v1, &v2);
    f4 op = vget(m, m->tet[4 * (size_t)t + ((f + 3) & 3)]);
    vo_face F;
    plane(v0, v1, v2, &F);
    float faceZ = op.x * F.zx + op.y * F.zy + F.zz;
    if (faceZ < op.z) F.sx = -1.0f; /* :128 invisible sentinel */
    out[e] = F;
  }
}

uint32_t vo_compact(const vo_face* faces, uint32_t nExt, uint32_t* visExt) {
  uint32_t n = 0;
  for (uint32_t e = 0; e < nExt; ++e)
    if (faces[e].sx != -1.0) visExt[n++] = e;
  return n;
}

static inline uint32_t to_pix(double d) {
  /* x86-64 double->uint as the reference binary does it: truncate to int64,
   * keep the low 32 bits */
  return (uint32_t)(int64_t)d;
}

void vo_project(const vo_mesh* m, const uint32_t* visExt, uint32_t nVis, uint32_t W,
                uint32_t H, uint32_t* bb) {
  for (uint32_t i = 0; i < nVis; ++i) {
    uint32_t e = visExt[i], t = m->extf[2 * e], f = m->extf[2 * e + 1];
    uint32_t b[4] = {W - 1, H - 1, 0, 0};
    for (uint32_t k = 0; k < 3; ++k) {
      f4 v = vget(m, m->tet[4 * (size_t)t + ((f + k) & 3)]);
      uint32_t ix = to_pix((W - 1.0) * (v.x + 1.0) / 2.0);
      uint32_t iy = to_pix((H - 1.0) * (v.y + 1.0) / 2.0);
      if (ix < b[0]) b[0] = ix;
      if (iy < b[1]) b[1] = iy;
      if (ix > b[2]) b[2] = ix;
      if (iy > b[3]) b[3] = iy;
    }
    memcpy(bb + 4 * (size_t)i, b, sizeof b);
  }
}

/* Entry-face edge setup, vfRayKernelCPU.cc:190-216. */
typedef struct { f4 v0; float e1x, e1y, e2x, e2y, cx; vo_face F; uint32_t t, f; } entry_face;

static void entry_setup(const vo_mesh* m, uint32_t e, entry_face* E) {
  E->t = m->extf[2 * e]; E->f = m->extf[2 * e + 1];
  f4 v0, v1, v2;
  face_verts(m, E->t, E->f, &v0, &v1, &v2);
  plane(v0, v1, v2, &E->F);
  E->v0 = v0;
  float ax = v1.x - v0.x, ay = v1.y - v0.y, bx = v2.x - v0.x, by = v2.y - v0.y;
  float cx = (ax * by) - (ay * bx);
  cx = (ABSF(cx) < RDELTA) ? RDELTA : cx;
  if (cx < 0.0) {
    float tx = ax, ty = ay;
    ax = bx; ay = by; bx = tx; by = ty;
    cx = -cx;
  }
  E->e1x = ax; E->e1y = ay; E->e2x = bx; E->e2y = by; E->cx = cx;
}

static inline float obj_coord(uint32_t p, uint32_t res) {
  return (p * 2) / (float)(res - 1) - 1.0; /* :250,254 */
}

/* Inclusive inside test of the entry face, :258-268. */
static inline int entry_inside(const entry_face* E, float ox, float oy) {
  float px = ox - E->v0.x, py = oy - E->v0.y;
  float cy = (E->e1x * py) - (E->e1y * px);
  float cz = (px * E->e2y) - (py * E->e2x);
  return (cy >= 0.0) && (cz >= 0.0) && ((cy + cz) <= E->cx);
}

typedef struct {
  float acc[3], trans;
  uint32_t iters, comps;
  float lastZ;
} ray_state;

/* FP64 rerun of a ray: the tet sequence and every decision come from the
 * float traversal; along that same path the colour is recomputed entirely
 * in double (planes, depths, tau, zeta, gamma and the psi index, the sum),
 * from the double pixel coordinate.  The tables (TF, psi) are the same. */
typedef struct {
  double ox, oy, acc[3], trans, zp, cb[4];
} ray64;

typedef struct { double zx, zy, zz, sx, sy, sz; } face64;

static void plane64(f4 a, f4 b, f4 c, face64* f) {
  double c0x = a.x, c0y = b.x, c0z = c.x, c1x = a.y, c1y = b.y, c1z = c.y;
  double det = c0x * (c1y - c1z) - c1x * (c0y - c0z) + (c0y * c1z - c1y * c0z);
  if (fabs(det) < RDELTA) det = RDELTA;
  double t[2][3] = {{a.z, b.z, c.z}, {a.w, b.w, c.w}};
  double o[2][3];
  for (int k = 0; k < 2; ++k) {
    double tx = t[k][0], ty = t[k][1], tz = t[k][2];
    double mx = ty - tz, my = ty * c1z - c1y * tz, mz = c0y * tz - ty * c0z;
    o[k][0] = (tx * (c1y - c1z) - c1x * mx + my) / det;
    o[k][1] = (c0x * mx - tx * (c0y - c0z) + mz) / det;
    o[k][2] = (c0x * (-my) - c1x * mz + tx * (c0y * c1z - c1y * c0z)) / det;
  }
  f->zx = o[0][0]; f->zy = o[0][1]; f->zz = o[0][2];
  f->sx = o[1][0]; f->sy = o[1][1]; f->sz = o[1][2];
}

static void tf64(const vo_mesh* m, double s, double* c) {
  if (!(s >= 0.0)) s = 0.0;
  if (s > 1.0) s = 1.0;
  uint32_t i = (uint32_t)(255.0 * s);
  if (i > 255) i = 255;
  for (int k = 0; k < 4; ++k) c[k] = m->tf[4 * i + k];
}

static uint32_t psi_index64(double tau) {
  double tc = tau / (1.0 + tau) + 0.5 / 512;
  if (!(tc >= 0.0)) tc = 0.0;
  uint32_t i = (uint32_t)(tc * 512);
  return i > 511 ? 511 : i;
}

static void ray64_begin(const vo_mesh* m, uint32_t t, uint32_t f, ray64* D) {
  f4 v0 = vget(m, m->tet[4 * (size_t)t + f]);
  f4 v1 = vget(m, m->tet[4 * (size_t)t + ((f + 1) & 3)]);
  f4 v2 = vget(m, m->tet[4 * (size_t)t + ((f + 2) & 3)]);
  face64 F;
  plane64(v0, v1, v2, &F);
  D->zp = D->ox * F.zx + D->oy * F.zy + F.zz;
  tf64(m, D->ox * F.sx + D->oy * F.sy + F.sz, D->cb);
}

static void ray64_step(const vo_mesh* m, f4 a, f4 b, f4 c, ray64* D) {
  face64 F;
  plane64(a, b, c, &F);
  double zn = D->ox * F.zx + D->oy * F.zy + F.zz;
  double sn = D->ox * F.sx + D->oy * F.sy + F.sz;
  double dz = fabs(D->zp - zn);
  if (dz < RDELTA) dz = 0.0;
  dz /= m->maxEdge;
  double cf[4];
  tf64(m, sn, cf);
  double tf = cf[3] * dz, tb = D->cb[3] * dz;
  double zeta = exp(-(tf * 0.5 + tb * 0.5));
  double psi = m->psi[psi_index64(tf) * 512 + psi_index64(tb)];
  for (int k = 0; k < 3; ++k)
    D->acc[k] = cf[k] * (1.0 - psi) + D->cb[k] * (psi - zeta) + zeta * D->acc[k];
  D->trans *= zeta;
  for (int k = 0; k < 4; ++k) D->cb[k] = cf[k];
  D->zp = zn;
}

/* Iterations a ray runs before its walk is watched for a repeated state,
 * and its cap (4 nT + 64, or the mesh's step_cap).  The walk from a state
 * (tet, entry face) is fixed for a pixel, so a state that comes back means
 * the reference's loop never ends.  Past the threshold the state is saved at
 * every power-of-two iteration count and compared with every later one
 * (Brent).  The CUDA traversal applies the same rule. */
#define WATCH_STEPS 4095u

static uint32_t step_cap(const vo_mesh* m) {
  if (m->step_cap) return m->step_cap;
  uint64_t c = 4ull * m->nT + 64u;
  return c > 0x7fffffffu ? 0x7fffffffu : (uint32_t)c;
}

/* One ray segment from entry (t, f) with entry depth/scalar (zp, sp),
 * :276-542.  Returns 0; -1 on the :365 `return` (adjacency that does not
 * point back); TRACE_CAP or TRACE_CYCLE when the ray was stopped (the
 * reference would go on forever). */
#define TRACE_CAP 1
#define TRACE_CYCLE 2
static int trace(const vo_mesh* m, float ox, float oy, uint32_t t, uint32_t f, float zpx,
                 float zpy, ray_state* R, ray64* D) {
  f4 cb = tfget(m, zpy);
  if (D) ray64_begin(m, t, f, D);
  uint32_t tpx = t, tpy = f;
  const uint32_t cap = step_cap(m), watch = cap < WATCH_STEPS ? cap : WATCH_STEPS;
  uint32_t saved = 0xffffffffu;
  R->lastZ = zpx;
  for (;;) {
    R->iters++;
    if (R->iters > watch) {
      if (R->iters > cap) return TRACE_CAP;
      const uint32_t key = (tpx << 2) | tpy;
      if (key == saved) return TRACE_CYCLE;
      if ((R->iters & (R->iters - 1u)) == 0u) saved = key;
    }
    uint32_t tny = tpy, tnx;
    f4 fv[4];
    for (int k = 0; k < 4; ++k) fv[k] = vget(m, m->tet[4 * (size_t)tpx + k]);
    for (uint32_t i = 1; i < 4; ++i) {
      uint32_t id = (tpy + i) & 3;
      float v1x = fv[(id + 1) & 3].x - fv[(id + 0) & 3].x;
      float v1y = fv[(id + 1) & 3].y - fv[(id + 0) & 3].y;
      float v2x = fv[(id + 2) & 3].x - fv[(id + 0) & 3].x;
      float v2y = fv[(id + 2) & 3].y - fv[(id + 0) & 3].y;
      float c = (v1x * v2y) - (v1y * v2x);
      if (ABSF(c) < RDELTA) continue;
      if (c < 0.0) {
        float sx = v1x, sy = v1y;
        v1x = v2x; v1y = v2y; v2x = sx; v2y = sy;
        c = -c;
      }
      float v0x = ox - fv[(id + 0) & 3].x;
      float v0y = oy - fv[(id + 0) & 3].y;
      float c1 = (v1x * v0y) - (v1y * v0x);
      float c2 = (v0x * v2y) - (v0y * v2x);
      if ((c1 >= 0.0) && (c2 >= 0.0) && ((c1 + c2) <= c + RDELTA)) {
        tny = id;
        break;
      }
    }
    if (tny == tpy) break; /* :353 no exit face found */
    tnx = m->con[4 * (size_t)tpx + tny];
    if (tnx != tpx) {
      const uint32_t* cn = m->con + 4 * (size_t)tnx;
      if (cn[0] == tpx) tpy = 0;
      else if (cn[1] == tpx) tpy = 1;
      else if (cn[2] == tpx) tpy = 2;
      else if (cn[3] == tpx) tpy = 3;
      else return -1;
    }
    vo_face nf;
    plane(fv[(tny + 0) & 3], fv[(tny + 1) & 3], fv[(tny + 2) & 3], &nf);
    float znx = ox * nf.zx + oy * nf.zy + nf.zz;
    float zny = ox * nf.sx + oy * nf.sy + nf.sz;
    float dz = ABSF(zpx - znx);
    dz = (dz < RDELTA) ? 0.0 : dz;
    if ((zny < 0.0) || (zny > 1.0)) break;
    dz /= m->maxEdge;
    f4 cf = tfget(m, zny);
    float taux = cf.w * dz, tauy = cb.w * dz;
    float zeta = exp(-(taux * 0.5 + tauy * 0.5));
    float gx = taux / (1.0 + taux), gy = tauy / (1.0 + tauy);
    float tcx = gx + (0.5 / 512), tcy = gy + (0.5 / 512);
    if ((tcx < 0.0) || (tcx > 1.0) || (tcy < 0.0) || (tcy > 1.0)) break;
    uint32_t pi = (uint32_t)(tcx * 512), pj = (uint32_t)(tcy * 512);
    if (pi > 511) pi = 511; /* tc == 1.0 would index row 512 */
    if (pj > 511) pj = 511;
    float psi = m->psi[pi * 512 + pj];
    float fx = cf.x * (1.0 - psi) + cb.x * (psi - zeta);
    float fy = cf.y * (1.0 - psi) + cb.y * (psi - zeta);
    float fz = cf.z * (1.0 - psi) + cb.z * (psi - zeta);
    float fw = 1.0 - zeta;
    R->acc[0] = fx + (1.0 - fw) * R->acc[0];
    R->acc[1] = fy + (1.0 - fw) * R->acc[1];
    R->acc[2] = fz + (1.0 - fw) * R->acc[2];
    R->trans = R->trans * zeta;
    R->comps++;
    R->lastZ = znx;
    if (D) ray64_step(m, fv[(tny + 0) & 3], fv[(tny + 1) & 3], fv[(tny + 2) & 3], D);
    cb = cf;
    if (tnx == tpx) break; /* :535 left the mesh */
    tpx = tnx;
    zpx = znx;
    zpy = zny;
  }
  return 0;
}

static inline void finalize(const ray_state* R, uint8_t* rgb, float* rgba) {
  float a[3] = {R->acc[0], R->acc[1], R->acc[2]};
  for (int k = 0; k < 3; ++k) {
    if (a[k] > 1.0) a[k] = 1.0;
    if (rgb) rgb[k] = (uint8_t)(int32_t)(255 * a[k]); /* :550-552 */
    if (rgba) rgba[k] = a[k];
  }
  if (rgba) rgba[3] = 1.0f - R->trans;
}

static int prepare(const vo_mesh* m, uint32_t W, uint32_t H, uint32_t** visExt,
                   uint32_t** bbox, vo_face** faces) {
  if (!mesh_ok(m) || W < 2 || H < 2) return -1;
  *faces = malloc(sizeof(vo_face) * (m->nExt ? m->nExt : 1));
  *visExt = malloc(sizeof(uint32_t) * (m->nExt ? m->nExt : 1));
  *bbox = malloc(sizeof(uint32_t) * 4 * (m->nExt ? m->nExt : 1));
  vo_find_visible(m, *faces);
  uint32_t n = vo_compact(*faces, m->nExt, *visExt);
  vo_project(m, *visExt, n, W, H, *bbox);
  return (int)n;
}

static inline int in_image(uint32_t x, uint32_t y, uint32_t W, uint32_t H) { return x < W && y < H; }

static int render_ref(const vo_mesh* m, uint32_t W, uint32_t H, uint8_t* rgb8, float* rgba,
                      int32_t* writer, uint32_t* steps, uint64_t* faceComp,
                      uint8_t* faceAbandon, double* rgba64) {
  uint32_t *vis, *bb;
  vo_face* faces;
  int nv = prepare(m, W, H, &vis, &bb, &faces);
  if (nv < 0) return nv;
  size_t np = (size_t)W * H;
  if (rgb8) memset(rgb8, 0, np * 3);
  if (rgba) memset(rgba, 0, np * 4 * sizeof(float));
  if (writer) for (size_t p = 0; p < np; ++p) writer[p] = -1;
  if (steps) memset(steps, 0, np * sizeof(uint32_t));
  if (rgba64) memset(rgba64, 0, np * 4 * sizeof(double));
  for (int i = 0; i < nv; ++i) {
    uint32_t e = vis[i];
    entry_face E;
    entry_setup(m, e, &E);
    const uint32_t* b = bb + 4 * (size_t)i;
    uint64_t comps = 0;
    int abandoned = 0;
    for (uint32_t px = b[0]; px <= b[2] && !abandoned; ++px) {
      float ox = obj_coord(px, W);
      for (uint32_t py = b[1]; py <= b[3]; ++py) {
        float oy = obj_coord(py, H);
        if (!entry_inside(&E, ox, oy)) continue;
        float zpx = ox * E.F.zx + oy * E.F.zy + E.F.zz;
        float zpy = ox * E.F.sx + oy * E.F.sy + E.F.sz;
        if ((zpy < 0.0) || (zpy > 1.0)) break; /* :274 rest of the column */
        ray_state R = {{0, 0, 0}, 1.0f, 0, 0, 0};
        ray64 D = {px * 2.0 / (W - 1.0) - 1.0, py * 2.0 / (H - 1.0) - 1.0, {0, 0, 0}, 1.0, 0,
                   {0, 0, 0, 0}};
        int rc = trace(m, ox, oy, E.t, E.f, zpx, zpy, &R, rgba64 ? &D : NULL);
        comps += R.comps;
        if (rc < 0) { abandoned = 1; break; } /* :365 rest of the face */
        if (!in_image(px, py, W, H)) continue;
        size_t p = (size_t)py * W + px;
        finalize(&R, rgb8 ? rgb8 + 3 * p : NULL, rgba ? rgba + 4 * p : NULL);
        if (writer) writer[p] = (int32_t)e;
        if (steps) steps[p] = R.iters;
        if (rgba64) {
          for (int k = 0; k < 3; ++k) rgba64[4 * p + k] = D.acc[k] > 1.0 ? 1.0 : D.acc[k];
          rgba64[4 * p + 3] = 1.0 - D.trans;
        }
      }
    }
    if (faceComp) faceComp[i] = comps;
    if (faceAbandon) faceAbandon[i] = (uint8_t)abandoned;
  }
  free(vis); free(bb); free(faces);
  return nv;
}

int vo_render_ref(const vo_mesh* m, uint32_t W, uint32_t H, uint8_t* rgb8, float* rgba,
                  int32_t* writer, uint32_t* steps, uint64_t* faceComp, uint8_t* faceAbandon) {
  return render_ref(m, W, H, rgb8, rgba, writer, steps, faceComp, faceAbandon, NULL);
}

int vo_render_ref_fp64(const vo_mesh* m, uint32_t W, uint32_t H, double* rgba64) {
  return render_ref(m, W, H, NULL, NULL, NULL, NULL, NULL, NULL, rgba64);
}

int vo_winners(const vo_mesh* m, uint32_t W, uint32_t H, int32_t* writer) {
  uint32_t *vis, *bb;
  vo_face* faces;
  int nv = prepare(m, W, H, &vis, &bb, &faces);
  if (nv < 0) return nv;
  for (size_t p = 0; p < (size_t)W * H; ++p) writer[p] = -1;
  for (int i = 0; i < nv; ++i) {
    entry_face E;
    entry_setup(m, vis[i], &E);
    const uint32_t* b = bb + 4 * (size_t)i;
    for (uint32_t px = b[0]; px <= b[2]; ++px) {
      float ox = obj_coord(px, W);
      for (uint32_t py = b[1]; py <= b[3]; ++py) {
        float oy = obj_coord(py, H);
        if (!entry_inside(&E, ox, oy)) continue;
        float zpy = ox * E.F.sx + oy * E.F.sy + E.F.sz;
        if ((zpy < 0.0) || (zpy > 1.0)) break;
        if (in_image(px, py, W, H)) writer[(size_t)py * W + px] = (int32_t)vis[i];
      }
    }
  }
  free(vis); free(bb); free(faces);
  return nv;
}

/* ---- threaded helpers ---- */

typedef struct {
  void (*fn)(void* ctx, size_t lo, size_t hi);
  void* ctx;
  size_t n, chunk;
  size_t next; /* guarded by the mutex */
  pthread_mutex_t mu;
} pool_job;

static void* pool_worker(void* arg) {
  pool_job* j = (pool_job*)arg;
  for (;;) {
    pthread_mutex_lock(&j->mu);
    size_t lo = j->next;
    j->next += j->chunk;
    pthread_mutex_unlock(&j->mu);
    if (lo >= j->n) break;
    size_t hi = lo + j->chunk < j->n ? lo + j->chunk : j->n;
    j->fn(j->ctx, lo, hi);
  }
  return NULL;
}

static void parallel_for(size_t n, size_t chunk, int threads,
                         void (*fn)(void*, size_t, size_t), void* ctx) {
  if (threads <= 0) {
    long c = sysconf(_SC_NPROCESSORS_ONLN);
    threads = c > 0 ? (int)c : 1;
  }
  pool_job j = {fn, ctx, n, chunk ? chunk : 1, 0, PTHREAD_MUTEX_INITIALIZER};
  pthread_t* tid = malloc(sizeof(pthread_t) * (size_t)threads);
  int started = 0;
  for (int t = 1; t < threads; ++t)
    if (pthread_create(&tid[started], NULL, pool_worker, &j) == 0) ++started;
  pool_worker(&j);
  for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
  free(tid);
}

typedef struct {
  const vo_mesh* m;
  uint32_t W, H;
  const uint32_t *pix, *entry;
  uint8_t* rgb8;
  float* rgba;
  uint32_t* steps;
  int err; /* written with __atomic */
} trace_ctx;

static void trace_range(void* c_, size_t lo, size_t hi) {
  trace_ctx* c = (trace_ctx*)c_;
  for (size_t k = lo; k < hi; ++k) {
    uint32_t p = c->pix[k], x = p % c->W, y = p / c->W;
    entry_face E;
    entry_setup(c->m, c->entry[k], &E);
    float ox = obj_coord(x, c->W), oy = obj_coord(y, c->H);
    float zpx = ox * E.F.zx + oy * E.F.zy + E.F.zz;
    float zpy = ox * E.F.sx + oy * E.F.sy + E.F.sz;
    ray_state R = {{0, 0, 0}, 1.0f, 0, 0, 0};
    if (trace(c->m, ox, oy, E.t, E.f, zpx, zpy, &R, NULL) < 0) __atomic_store_n(&c->err, 1, __ATOMIC_RELAXED);
    finalize(&R, c->rgb8 ? c->rgb8 + 3 * k : NULL, c->rgba ? c->rgba + 4 * k : NULL);
    if (c->steps) c->steps[k] = R.iters;
  }
}

int vo_trace_pixels(const vo_mesh* m, uint32_t W, uint32_t H, uint32_t n, const uint32_t* pix,
                    const uint32_t* entryExt, uint8_t* rgb8, float* rgba, uint32_t* steps,
                    int threads) {
  if (!mesh_ok(m) || W < 2 || H < 2) return -2;
  for (uint32_t k = 0; k < n; ++k)
    if (pix[k] >= W * H || entryExt[k] >= m->nExt) return -2;
  trace_ctx c = {m, W, H, pix, entryExt, rgb8, rgba, steps, 0};
  parallel_for(n, 256, threads, trace_range, &c);
  return c.err ? -1 : 0;
}

/* ---- depth-composited mode ---- */

typedef struct { float z, s; uint32_t e; } comp_entry;

typedef struct {
  const vo_mesh* m;
  uint32_t W, H;
  const size_t* off;
  const comp_entry* ent;
  uint8_t* rgb8;
  float* rgba;
  uint32_t *steps, *nseg;
  int err;
} comp_ctx;

static void comp_range(void* c_, size_t lo, size_t hi) {
  comp_ctx* c = (comp_ctx*)c_;
  comp_entry buf[64];
  for (size_t p = lo; p < hi; ++p) {
    size_t a = c->off[p], b = c->off[p + 1], n = b - a;
    if (n == 0) continue;
    comp_entry* L = n <= 64 ? buf : malloc(sizeof(comp_entry) * n);
    memcpy(L, c->ent + a, sizeof(comp_entry) * n);
    for (size_t i = 1; i < n; ++i) { /* insertion sort: z desc, then e desc */
      comp_entry k = L[i];
      size_t j = i;
      while (j > 0 && (L[j - 1].z < k.z || (L[j - 1].z == k.z && L[j - 1].e < k.e))) {
        L[j] = L[j - 1];
        --j;
      }
      L[j] = k;
    }
    uint32_t x = (uint32_t)(p % c->W), y = (uint32_t)(p / c->W);
    float ox = obj_coord(x, c->W), oy = obj_coord(y, c->H);
    ray_state R = {{0, 0, 0}, 1.0f, 0, 0, 0};
    float exitZ = INFINITY;
    uint32_t segs = 0;
    for (size_t i = 0; i < n; ++i) {
      if (L[i].z > exitZ) continue;
      uint32_t e = L[i].e;
      int rc = trace(c->m, ox, oy, c->m->extf[2 * e], c->m->extf[2 * e + 1], L[i].z, L[i].s, &R, NULL);
      if (rc < 0) __atomic_store_n(&c->err, 1, __ATOMIC_RELAXED);
      exitZ = R.lastZ;
      ++segs;
      if (rc > 0) break; /* stopped: the ray ends with what it composited */
    }
    finalize(&R, c->rgb8 ? c->rgb8 + 3 * p : NULL, c->rgba ? c->rgba + 4 * p : NULL);
    if (c->steps) c->steps[p] = R.iters;
    if (c->nseg) c->nseg[p] = segs;
    if (L != buf) free(L);
  }
}

int vo_render_composited(const vo_mesh* m, uint32_t W, uint32_t H, uint8_t* rgb8, float* rgba,
                         uint32_t* steps, uint32_t* nseg, int threads) {
  uint32_t *vis, *bb;
  vo_face* faces;
  int nv = prepare(m, W, H, &vis, &bb, &faces);
  if (nv < 0) return nv;
  size_t np = (size_t)W * H;
  if (rgb8) memset(rgb8, 0, np * 3);
  if (rgba) memset(rgba, 0, np * 4 * sizeof(float));
  if (steps) memset(steps, 0, np * sizeof(uint32_t));
  if (nseg) memset(nseg, 0, np * sizeof(uint32_t));
  size_t* off = calloc(np + 1, sizeof(size_t));
  comp_entry* ent = NULL;
  for (int pass = 0; pass < 2; ++pass) {
    size_t* cur = NULL;
    if (pass == 1) {
      for (size_t p = 0; p < np; ++p) off[p + 1] += off[p];
      ent = malloc(sizeof(comp_entry) * (off[np] ? off[np] : 1));
      cur = malloc(sizeof(size_t) * np);
      memcpy(cur, off, sizeof(size_t) * np);
    }
    for (int i = 0; i < nv; ++i) {
      entry_face E;
      entry_setup(m, vis[i], &E);
      const uint32_t* b = bb + 4 * (size_t)i;
      for (uint32_t px = b[0]; px <= b[2]; ++px) {
        float ox = obj_coord(px, W);
        for (uint32_t py = b[1]; py <= b[3]; ++py) {
          float oy = obj_coord(py, H);
          if (!in_image(px, py, W, H) || !entry_inside(&E, ox, oy)) continue;
          float zpx = ox * E.F.zx + oy * E.F.zy + E.F.zz;
          float zpy = ox * E.F.sx + oy * E.F.sy + E.F.sz;
          if ((zpy < 0.0) || (zpy > 1.0)) continue;
          size_t p = (size_t)py * W + px;
          if (pass == 0) off[p + 1]++;
          else { comp_entry q = {zpx, zpy, vis[i]}; ent[cur[p]++] = q; }
        }
      }
    }
    free(cur);
  }
  comp_ctx c = {m, W, H, off, ent, rgb8, rgba, steps, nseg, 0};
  parallel_for(np, 1024, threads, comp_range, &c);
  free(off); free(ent); free(vis); free(bb); free(faces);
  return c.err ? -1 : nv;
}
