// Kernels of the VF-Ray render path: view set-up, stage (a) visible faces +
// ordered compaction, stage (b) projection + per-pixel entry faces, ray-list
// compaction, and stage (c) tet-walk traversal with partial pre-integration.
#pragma once
#include "vfr_device.cuh"

namespace vfr {

// Per-view device counters (one 64-byte block per view/job).
struct __align__(16) ViewCounters {
  uint32_t nvis;         // visible faces
  uint32_t nrays;        // rays in the ray list
  uint32_t queue;        // traversal work-queue head
  uint32_t status;       // VFR_DEV_* bits
  unsigned long long steps;  // tet-walk iterations, all rays
  uint32_t nentries;     // entry-list entries (composited mode)
  uint32_t maxedge_bits; // view maxEdgeLength (float bits, >= 0)
  uint32_t mm[8];        // orderable min x y z s, max x y z s (view set-up)
};

struct TraverseParams {
  const uint4* tet;
  const WalkRec* walk;
  const float4* vert;
  const uint2* extf;
  const float4* planes;   // 2 float4 per ext face: (zx zy zz sx) (sy sz - -)
  const int32_t* winner;  // W*H ext index (reference mode)
  const uint32_t* rays;   // pixel ids
  const uint32_t* ent_off;  // composited: W*H+1 offsets
  const uint2* ent;         // composited: (z bits, ext index)
  ViewCounters* ctr;
  const float4* tf;       // 256 RGBA
  const float* psi;       // 512x512
  uint8_t* rgb8;
  float4* rgba;
  uint32_t* steps;
  uint32_t W, H, nT, nV;
  float maxEdge;          // used when use_view_maxedge == 0
  int use_view_maxedge;
  uint32_t step_cap;
  uint32_t chunk;         // rays per warp fetch (unused by the refill kernel)
  uint32_t ent_cap;       // composited: capacity of ent
  uint32_t refill;        // refill a warp's idle lanes once at least this many are idle
  uint32_t psi_one;       // psi table[0][0] == 1.0f (enables the zero-extinction shortcut)
};

// ---------------------------------------------------------------- view set-up

// rotateVolume (vfRayPreComp.cc:886-906) + min/max for normalizeVertices.
__global__ void view_rotate_kernel(const float4* __restrict__ base, uint32_t nV, float4 m0,
                                   float4 m1, float4 m2, float4* __restrict__ out,
                                   ViewCounters* ctr) {
  float mn[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
  float mx[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nV; i += gridDim.x * blockDim.x) {
    float4 v = base[i];
    float r[3];
    const float4 rows[3] = {m0, m1, m2};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float acc = 0.0f;
      acc = fadd(acc, fmul(rows[a].x, v.x));
      acc = fadd(acc, fmul(rows[a].y, v.y));
      acc = fadd(acc, fmul(rows[a].z, v.z));
      acc = fadd(acc, fmul(rows[a].w, 1.0f));
      r[a] = acc;
    }
    float4 o = make_float4(r[0], r[1], r[2], v.w);
    out[i] = o;
    const float c[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      mn[k] = fminf(mn[k], c[k]);
      mx[k] = fmaxf(mx[k], c[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    for (int o = 16; o; o >>= 1) {
      mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
      mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      atomicMin(&ctr->mm[k], f2ord(mn[k]));
      atomicMax(&ctr->mm[4 + k], f2ord(mx[k]));
    }
  }
}

// normalizeVertices (vfRayPreComp.cc:84-145) with the view's min/max.
__global__ void view_normalize_kernel(float4* __restrict__ v, uint32_t nV, const ViewCounters* ctr) {
  float mn[4], mx[4], cen[3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    mn[k] = ord2f(ctr->mm[k]);
    mx[k] = ord2f(ctr->mm[4 + k]);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    cen[k] = (float)ddiv((double)fadd(mn[k], mx[k]), 2.0);
    mx[k] = fsub(mx[k], cen[k]);
    mn[k] = fsub(mn[k], cen[k]);
  }
  float maxCoord = (mx[1] > mx[2]) ? mx[1] : mx[2];
  maxCoord = (mx[0] > maxCoord) ? mx[0] : maxCoord;
  const float sc = (float)ddiv(1.0, (double)maxCoord);
  const float ss = (float)ddiv(1.0, (double)fsub(mx[3], mn[3]));
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nV; i += gridDim.x * blockDim.x) {
    float4 p = v[i];
    p.x = fmul(fsub(p.x, cen[0]), sc);
    p.y = fmul(fsub(p.y, cen[1]), sc);
    p.z = fmul(fsub(p.z, cen[2]), sc);
    p.w = fmul(fsub(p.w, mn[3]), ss);
    v[i] = p;
  }
}

// buildLmt's maxEdgeLength (vfRayPreComp.cc:810-836) over the view's vertices.
__global__ void view_maxedge_kernel(const uint4* __restrict__ tet, const float4* __restrict__ v,
                                    uint32_t nT, ViewCounters* ctr) {
  float best = 0.0f;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nT; t += gridDim.x * blockDim.x) {
    const uint4 id = tet[t];
    const float4 p[4] = {v[id.x], v[id.y], v[id.z], v[id.w]};
    const int E[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const float4 a = p[E[j][0]], b = p[E[j][1]];
      float e0 = fsub(a.x, b.x), e1 = fsub(a.y, b.y), e2 = fsub(a.z, b.z);
      float len = __fsqrt_rn(fadd(fadd(fmul(e0, e0), fmul(e1, e1)), fmul(e2, e2)));
      if (len > best) best = len;
    }
  }
  for (int o = 16; o; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&ctr->maxedge_bits, __float_as_uint(best));
}

// ------------------------------------------------------------------ stage (a)

// findVisibleFaces (vfRayKernelCPU.cc:51-132), one thread per external face;
// writes the face planes and the per-block count of visible faces.
__global__ void __launch_bounds__(1024) visible_kernel(const float4* __restrict__ vert,
                                                       const uint4* __restrict__ tet,
                                                       const uint2* __restrict__ extf,
                                                       uint32_t nExt, float4* __restrict__ planes,
                                                       uint32_t* __restrict__ blk_cnt) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  int vis = 0;
  if (e < nExt) {
    const uint2 tf = extf[e];
    const uint4 id = tet[tf.x];
    const float4 v0 = vert[sel4(id, tf.y & 3u)];
    const float4 v1 = vert[sel4(id, (tf.y + 1) & 3u)];
    const float4 v2 = vert[sel4(id, (tf.y + 2) & 3u)];
    const float4 op = vert[sel4(id, (tf.y + 3) & 3u)];
    Plane P;
    face_plane(v0, v1, v2, P);
    const float faceZ = plane_eval(op.x, op.y, P.zx, P.zy, P.zz);
    if (faceZ < op.z) P.sx = -1.0f;  // :128 invisible sentinel
    vis = (P.sx != -1.0f);
    planes[2 * (size_t)e] = make_float4(P.zx, P.zy, P.zz, P.sx);
    planes[2 * (size_t)e + 1] = make_float4(P.sy, P.sz, 0.0f, 0.0f);
  }
  const int cnt = __syncthreads_count(vis);
  if (threadIdx.x == 0) blk_cnt[blockIdx.x] = (uint32_t)cnt;
}

// Ordered compaction of the visible faces (the host loop of main.cc:93-138
// and vfRay.cu:355-388): a block's output offset is the sum of the counts of
// the blocks before it; inside the block, warp ballots and a warp-count
// prefix place each face at its rank.  No inter-block waiting.
__global__ void __launch_bounds__(1024) compact_kernel(const float4* __restrict__ planes,
                                                       uint32_t nExt,
                                                       const uint32_t* __restrict__ blk_cnt,
                                                       uint32_t* __restrict__ vis_ext,
                                                       ViewCounters* ctr) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_base;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  // offset of this block
  uint32_t part = 0;
  for (uint32_t b = threadIdx.x; b < blockIdx.x; b += blockDim.x) part += blk_cnt[b];
  for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if (lane == 0) s_warp[warp] = part;
  __syncthreads();
  if (warp == 0) {
    uint32_t x = lane < (blockDim.x >> 5) ? s_warp[lane] : 0u;
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) s_base = x;
  }
  __syncthreads();
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  const bool vis = e < nExt && planes[2 * (size_t)e].w != -1.0f;
  const uint32_t m = __ballot_sync(0xffffffffu, vis);
  if (lane == 0) s_warp[warp] = __popc(m);
  __syncthreads();
  if (warp == 0) {
    uint32_t c = lane < (blockDim.x >> 5) ? s_warp[lane] : 0u, x = c;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    s_warp[lane] = x - c;  // exclusive prefix of warp counts
    if (blockIdx.x == gridDim.x - 1 && lane == 31) ctr->nvis = s_base + x;
  }
  __syncthreads();
  if (vis) vis_ext[s_base + s_warp[warp] + __popc(m & ((1u << lane) - 1u))] = e;
}

// ------------------------------------------------------------------ stage (b)

// projectVisibleFaces (vfRayKernelCPU.cc:136-169) + the pixel coverage of
// vfRay's face loop (:248-274): one warp per visible face, one lane per
// bounding-box column, y ascending; an out-of-range entry scalar ends the
// column (:274).  The reference lets the last visible face in order write a
// pixel; visible order is ext-face order, so the winner is the largest
// ext-face index that reaches the pixel: atomicMax.  Pixels outside the image
// are clipped (the reference would write past its buffer there).
template <bool kCount, bool kFill>
__global__ void __launch_bounds__(256) raster_kernel(
    const float4* __restrict__ vert, const uint4* __restrict__ tet, const uint2* __restrict__ extf,
    const float4* __restrict__ planes, const uint32_t* __restrict__ vis_ext, ViewCounters* ctr,
    uint32_t W, uint32_t H, uint4* __restrict__ bbox, int32_t* __restrict__ winner,
    uint32_t* __restrict__ ent_cnt, const uint32_t* __restrict__ ent_off,
    uint32_t* __restrict__ ent_cur, uint2* __restrict__ ent, uint32_t ent_cap) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nvis = ctr->nvis;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nvis; i += nwarps) {
    const uint32_t e = vis_ext[i];
    const uint2 tf = extf[e];
    const uint4 id = tet[tf.x];
    const float4 v0 = vert[sel4(id, tf.y & 3u)];
    const float4 v1 = vert[sel4(id, (tf.y + 1) & 3u)];
    const float4 v2 = vert[sel4(id, (tf.y + 2) & 3u)];
    uint32_t bx = W - 1, by = H - 1, bz = 0, bw = 0;
    const float4 vv[3] = {v0, v1, v2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const uint32_t ix = to_pixel(vv[k].x, W), iy = to_pixel(vv[k].y, H);
      if (ix < bx) bx = ix;
      if (iy < by) by = iy;
      if (ix > bz) bz = ix;
      if (iy > bw) bw = iy;
    }
    if (bbox && lane == 0) bbox[i] = make_uint4(bx, by, bz, bw);
    const EntryEdges E = entry_edges(v0, v1, v2);
    const float4 p0 = planes[2 * (size_t)e], p1 = planes[2 * (size_t)e + 1];
    const uint32_t xe = min(bz, W - 1), ye = min(bw, H - 1);
    if (bx > xe || by > ye) continue;  // box entirely outside the image
    for (uint32_t px = bx + lane; px <= xe; px += 32) {
      const float ox = obj_coord(px, W);
      for (uint32_t py = by; py <= ye; ++py) {
        const float oy = obj_coord(py, H);
        if (!entry_inside(E, ox, oy)) continue;
        const float sp = plane_eval(ox, oy, p0.w, p1.x, p1.y);
        if (kCount || kFill) {
          if ((sp < 0.0f) || (sp > 1.0f)) continue;  // composited: only this pixel
          const uint32_t p = py * W + px;
          if (kCount) {
            atomicAdd(&ent_cnt[p], 1u);
          } else {
            const float zp = plane_eval(ox, oy, p0.x, p0.y, p0.z);
            const uint32_t slot = ent_off[p] + atomicAdd(&ent_cur[p], 1u);
            if (slot < ent_cap) ent[slot] = make_uint2(__float_as_uint(zp), e);
          }
        } else {
          if ((sp < 0.0f) || (sp > 1.0f)) break;  // :274 rest of the column
          atomicMax(&winner[py * W + px], (int32_t)e);
        }
      }
    }
  }
}

// Ray list: pixels with an entry face, in 8x4 screen tiles (one warp per
// tile) so that neighbouring rays, which walk neighbouring tets, share a warp.
__global__ void __launch_bounds__(256) raylist_kernel(const int32_t* __restrict__ winner,
                                                      const uint32_t* __restrict__ ent_cnt,
                                                      uint32_t W, uint32_t H,
                                                      uint32_t* __restrict__ rays,
                                                      ViewCounters* ctr) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t tx = (W + 7) >> 3, ty = (H + 3) >> 2;
  if (tile >= tx * ty) return;
  const uint32_t x = (tile % tx) * 8 + (lane & 7), y = (tile / tx) * 4 + (lane >> 3);
  bool has = false;
  if (x < W && y < H) {
    const uint32_t p = y * W + x;
    has = winner ? (winner[p] >= 0) : (ent_cnt[p] > 0);
  }
  const uint32_t m = __ballot_sync(0xffffffffu, has);
  if (!m) return;
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(&ctr->nrays, (uint32_t)__popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (has) rays[base + __popc(m & ((1u << lane) - 1u))] = y * W + x;
}

// Exclusive scan helpers for the composited entry lists.
__global__ void __launch_bounds__(1024) scan_blocks_kernel(const uint32_t* __restrict__ in,
                                                           uint32_t n, uint32_t* __restrict__ out,
                                                           uint32_t* __restrict__ sums) {
  __shared__ uint32_t s[32];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t v = i < n ? in[i] : 0u;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) s[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t c = s[lane], z = c;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= (uint32_t)o) z += y;
    }
    s[lane] = z - c;
    if (lane == 31) sums[blockIdx.x] = z;
  }
  __syncthreads();
  if (i < n) out[i] = x - v + s[warp];
}

// Adds the prefix of the block sums (each block sums the ones before it).
__global__ void __launch_bounds__(1024) scan_add_kernel(uint32_t* __restrict__ out, uint32_t n,
                                                        const uint32_t* __restrict__ sums,
                                                        uint32_t* __restrict__ total) {
  __shared__ uint32_t s[32];
  __shared__ uint32_t s_base;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t part = 0;
  for (uint32_t b = threadIdx.x; b < blockIdx.x; b += blockDim.x) part += sums[b];
  for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if (lane == 0) s[warp] = part;
  __syncthreads();
  if (warp == 0) {
    uint32_t x = s[lane];
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) s_base = x;
  }
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += s_base;
  if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
    *total = s_base + sums[blockIdx.x];
}

}  // namespace vfr

#include "vfr_traverse.cuh"
