// Stages (a) and (b) over a table of render jobs.
//
// A job is one (mesh, camera, resolution) view.  Every kernel here covers
// all jobs of a batch in one launch: items of all jobs share one index space
// (vertices, tets, external-face blocks, visible faces, screen tiles), and a
// binary search over a prefix of per-job counts maps an item to its job.
// Counts known on the host (vertices, tets, faces, tiles) are prefixed on the
// host; counts produced on the device (visible faces, rays) by
// prefix_kernel.  Nothing waits on the host between stages, so a batch is one
// stream-ordered chain of launches (and can be captured as a CUDA graph).
#pragma once
#include "vfr_types.cuh"

namespace vfr {

// Largest j with pref[j] <= g (pref[0] = 0, pref has n+1 entries, g < pref[n]).
__device__ __forceinline__ uint32_t job_of(const uint32_t* __restrict__ pref, uint32_t n, uint32_t g) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(pref + mid) <= g) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ float job_maxedge(const JobDev& J) {
  return J.use_mv ? __uint_as_float(J.ctr->maxedge_bits) : J.maxEdge_in;
}

__global__ void init_jobs_kernel(const JobDev* __restrict__ jobs, uint32_t njobs,
                                 uint32_t* __restrict__ queue) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j == 0) {
    queue[0] = 0;  // the traversal's ray queue
    queue[1] = 0;  // the composited mode's entry-arena cursor
  }
  if (j >= njobs) return;
  ViewCounters v;
  v.nvis = 0; v.nrays = 0; v.nentries = 0; v.status = 0; v.steps = 0;
  v.maxedge_bits = 0; v.rays_done = 0; v.nbins = 0;
  for (int k = 0; k < 4; ++k) { v.mm[k] = 0xffffffffu; v.mm[4 + k] = 0u; }
  *jobs[j].ctr = v;
}

// ------------------------------------------------------------ view set-up

// The view set-up kernels give each job a range of blocks (bpref: prefix of
// blocks per job), so a block reduces within one job and ends with one
// atomic per counter.

__device__ __forceinline__ float warp_min(float v) {
  for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// rotateVolume (vfRayPreComp.cc:886-906) + the min/max normalizeVertices
// needs, over the vertices of every job with a model-view.
__global__ void __launch_bounds__(256) view_rotate_kernel(const JobDev* __restrict__ jobs,
                                                          uint32_t njobs,
                                                          const uint32_t* __restrict__ bpref) {
  const uint32_t j = job_of(bpref, njobs, blockIdx.x);
  const JobDev& J = jobs[j];
  const uint32_t lb = blockIdx.x - bpref[j], nb = bpref[j + 1] - bpref[j];
  const float4 rows[3] = {J.m0, J.m1, J.m2};
  float mn[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
  float mx[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = lb * blockDim.x + threadIdx.x; i < J.nV; i += nb * blockDim.x) {
    const float4 v = J.vert_in[i];
    float r[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float acc = 0.0f;
      acc = fadd(acc, fmul(rows[a].x, v.x));
      acc = fadd(acc, fmul(rows[a].y, v.y));
      acc = fadd(acc, fmul(rows[a].z, v.z));
      acc = fadd(acc, fmul(rows[a].w, 1.0f));
      r[a] = acc;
    }
    const float4 o = make_float4(r[0], r[1], r[2], v.w);
    J.vview[i] = o;
    const float c[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      mn[k] = fminf(mn[k], c[k]);
      mx[k] = fmaxf(mx[k], c[k]);
    }
  }
  // one pair of atomics per block and coordinate: warps reduce, then the
  // block through shared memory
  __shared__ float s_mm[8][8];
  const uint32_t w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float a = warp_min(mn[k]), b = warp_max(mx[k]);
    if ((threadIdx.x & 31u) == 0) {
      s_mm[w][k] = a;
      s_mm[w][4 + k] = b;
    }
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    const uint32_t k = threadIdx.x;
    float v = s_mm[0][k];
    for (uint32_t i = 1; i < (blockDim.x >> 5); ++i)
      v = k < 4 ? fminf(v, s_mm[i][k]) : fmaxf(v, s_mm[i][k]);
    if (k < 4) atomicMin(&J.ctr->mm[k], f2ord(v));
    else atomicMax(&J.ctr->mm[k], f2ord(v));
  }
}

// normalizeVertices (vfRayPreComp.cc:84-145) with each view's min/max.
__global__ void __launch_bounds__(256) view_normalize_kernel(const JobDev* __restrict__ jobs,
                                                             uint32_t njobs,
                                                             const uint32_t* __restrict__ bpref) {
  const uint32_t j = job_of(bpref, njobs, blockIdx.x);
  const JobDev& J = jobs[j];
  const uint32_t lb = blockIdx.x - bpref[j], nb = bpref[j + 1] - bpref[j];
  float mn[4], mx[4], cen[3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    mn[k] = ord2f(J.ctr->mm[k]);
    mx[k] = ord2f(J.ctr->mm[4 + k]);
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
  for (uint32_t i = lb * blockDim.x + threadIdx.x; i < J.nV; i += nb * blockDim.x) {
    float4 p = J.vview[i];
    p.x = fmul(fsub(p.x, cen[0]), sc);
    p.y = fmul(fsub(p.y, cen[1]), sc);
    p.z = fmul(fsub(p.z, cen[2]), sc);
    p.w = fmul(fsub(p.w, mn[3]), ss);
    J.vview[i] = p;
  }
}

// buildLmt's maxEdgeLength (vfRayPreComp.cc:810-836) over each view's
// vertices.  The reference visits the 6 edges of every tet; an edge shared by
// several tets gives the same length in each (its difference vector at most
// changes sign), so the maximum over the mesh's distinct edges is the same
// float, at about a seventh of the work.
__global__ void __launch_bounds__(256) view_maxedge_kernel(const JobDev* __restrict__ jobs,
                                                           uint32_t njobs,
                                                           const uint32_t* __restrict__ bpref) {
  const uint32_t j = job_of(bpref, njobs, blockIdx.x);
  const JobDev& J = jobs[j];
  const uint32_t lb = blockIdx.x - bpref[j], nb = bpref[j + 1] - bpref[j];
  // the rounded square root is monotone, so the largest rounded length is
  // the rounded root of the largest squared length: one root per thread
  float best_sq = 0.0f;
  for (uint32_t e = lb * blockDim.x + threadIdx.x; e < J.nEdges; e += nb * blockDim.x) {
    const uint2 ed = __ldg(J.edges + e);
    if (id_bad(ed.x, J.nV) || id_bad(ed.y, J.nV)) {
      atomicOr(&J.ctr->status, kDevRange);
      continue;
    }
    const float4 a = J.vview[ed.x], b = J.vview[ed.y];
    const float e0 = fsub(a.x, b.x), e1 = fsub(a.y, b.y), e2 = fsub(a.z, b.z);
    const float sq = fadd(fadd(fmul(e0, e0), fmul(e1, e1)), fmul(e2, e2));
    if (sq > best_sq) best_sq = sq;
  }
  float best = __fsqrt_rn(best_sq);
  __shared__ float s_best[8];
  best = warp_max(best);
  if ((threadIdx.x & 31u) == 0) s_best[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t i = 1; i < (blockDim.x >> 5); ++i) best = fmaxf(best, s_best[i]);
    atomicMax(&J.ctr->maxedge_bits, __float_as_uint(best));
  }
}

// Keys of the 6 edges of every tet, (min id << 32) | max id, to be sorted and
// made unique into the mesh's distinct edges.
__global__ void __launch_bounds__(256) edge_keys_kernel(const uint4* __restrict__ tet, uint32_t nT,
                                                        unsigned long long* __restrict__ keys) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nT) return;
  const uint4 id = tet[t];
  const uint32_t v[4] = {id.x, id.y, id.z, id.w};
  const int E[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const uint32_t a = v[E[k][0]], b = v[E[k][1]];
    keys[6 * (size_t)t + k] = (unsigned long long)min(a, b) << 32 | max(a, b);
  }
}

// ------------------------------------------------------------ stage (a)

// findVisibleFaces (vfRayKernelCPU.cc:51-132), one thread per external face;
// each block of 1024 faces belongs to one job (bpref: blocks per job).
__global__ void __launch_bounds__(1024) visible_kernel(const JobDev* __restrict__ jobs,
                                                       uint32_t njobs,
                                                       const uint32_t* __restrict__ bpref) {
  const uint32_t j = job_of(bpref, njobs, blockIdx.x);
  const JobDev& J = jobs[j];
  const uint32_t lb = blockIdx.x - bpref[j];
  const uint32_t e = lb * blockDim.x + threadIdx.x;
  int vis = 0;
  if (e < J.nExt) {
    const uint2 tf = J.extf[e];
    bool bad = id_bad(tf.x, J.nT);
    uint4 id = J.tet[bad ? 0u : tf.x];
    bad = bad || id_bad(id.x, J.nV) || id_bad(id.y, J.nV) || id_bad(id.z, J.nV) ||
          id_bad(id.w, J.nV);
    if (bad) {
      id = make_uint4(0u, 0u, 0u, 0u);
      atomicOr(&J.ctr->status, kDevRange);
    }
    const float4 v0 = J.vert[sel4(id, tf.y & 3u)];
    const float4 v1 = J.vert[sel4(id, (tf.y + 1) & 3u)];
    const float4 v2 = J.vert[sel4(id, (tf.y + 2) & 3u)];
    const float4 op = J.vert[sel4(id, (tf.y + 3) & 3u)];
    Plane P;
    face_plane(v0, v1, v2, P);
    const float faceZ = plane_eval(op.x, op.y, P.zx, P.zy, P.zz);
    if (faceZ < op.z || bad) P.sx = -1.0f;  // :128 invisible sentinel
    vis = (P.sx != -1.0f);
    float4* pl = J.planes + kPlaneStride * (size_t)e;
    pl[0] = make_float4(P.zx, P.zy, P.zz, P.sx);
    pl[1] = make_float4(P.sy, P.sz, v0.x, v0.y);
    pl[2] = make_float4(v1.x, v1.y, v2.x, v2.y);
  }
  const int cnt = __syncthreads_count(vis);
  if (threadIdx.x == 0) J.blk[lb] = (uint32_t)cnt;
}

// Ordered compaction (main.cc:93-138, vfRay.cu:355-388): a block's offset is
// the sum of the counts of the job's blocks before it; inside the block,
// warp ballots and a warp-count prefix place each face at its rank.
__global__ void __launch_bounds__(1024) compact_kernel(const JobDev* __restrict__ jobs,
                                                       uint32_t njobs,
                                                       const uint32_t* __restrict__ bpref) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_base;
  const uint32_t j = job_of(bpref, njobs, blockIdx.x);
  const JobDev& J = jobs[j];
  const uint32_t lb = blockIdx.x - bpref[j];
  const uint32_t nb = bpref[j + 1] - bpref[j];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t part = 0;
  const uint32_t nwarps = blockDim.x >> 5;  // blocks of 256 or 1024 threads
  for (uint32_t b = threadIdx.x; b < lb; b += blockDim.x) part += J.blk[b];
  for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if (lane == 0) s_warp[warp] = part;
  __syncthreads();
  if (warp == 0) {
    uint32_t x = lane < nwarps ? s_warp[lane] : 0u;
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) s_base = x;
  }
  __syncthreads();
  const uint32_t e = lb * blockDim.x + threadIdx.x;
  const bool vis = e < J.nExt && J.planes[kPlaneStride * (size_t)e].w != -1.0f;
  const uint32_t m = __ballot_sync(0xffffffffu, vis);
  if (lane == 0) s_warp[warp] = __popc(m);
  __syncthreads();
  if (warp == 0) {
    const uint32_t c = lane < nwarps ? s_warp[lane] : 0u;
    uint32_t x = c;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    s_warp[lane] = x - c;
    if (lb == nb - 1 && lane == 31) J.ctr->nvis = s_base + x;
  }
  __syncthreads();
  if (vis) J.vis_ext[s_base + s_warp[warp] + __popc(m & ((1u << lane) - 1u))] = e;
}

// Exclusive prefix of a per-job device count (0: visible faces, 1: rays,
// 2: entry-list entries) into out[0..njobs]; one block.
__global__ void __launch_bounds__(1024) prefix_kernel(const JobDev* __restrict__ jobs, uint32_t njobs,
                                                      int which, uint32_t* __restrict__ out) {
  __shared__ uint32_t s[32];
  __shared__ uint32_t s_carry;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < njobs; base += blockDim.x) {
    const uint32_t j = base + threadIdx.x;
    uint32_t v = 0;
    if (j < njobs) {
      const ViewCounters* c = jobs[j].ctr;
      v = which == 0 ? c->nvis : (which == 1 ? c->nrays : c->nentries);
    }
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s[warp] = x;
    __syncthreads();
    if (warp == 0) {
      const uint32_t c = lane < (blockDim.x >> 5) ? s[lane] : 0u;
      uint32_t z = c;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
        if (lane >= (uint32_t)o) z += y;
      }
      s[lane] = z - c;
    }
    __syncthreads();
    const uint32_t carry = s_carry;
    if (j < njobs) out[j] = carry + s[warp] + x - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = carry + s[warp] + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[njobs] = s_carry;
}

// ------------------------------------------------------------ stage (b)

// projectVisibleFaces (vfRayKernelCPU.cc:136-169): the pixel bounding box of
// a face from its vertex xy, which stage (a) stores with the plane (p1.zw,
// p2.xy, p2.zw); min starts at res - 1 and max at 0 as in the reference.
__device__ __forceinline__ uint4 face_box(const float4& p1, const float4& p2, uint32_t W,
                                          uint32_t H) {
  uint32_t bx = W - 1, by = H - 1, bz = 0, bw = 0;
  const float xs[3] = {p1.z, p2.x, p2.z}, ys[3] = {p1.w, p2.y, p2.w};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const uint32_t ix = to_pixel(xs[k], W), iy = to_pixel(ys[k], H);
    if (ix < bx) bx = ix;
    if (iy < by) by = iy;
    if (ix > bz) bz = ix;
    if (iy > bw) bw = iy;
  }
  return make_uint4(bx, by, bz, bw);
}

// projectVisibleFaces (vfRayKernelCPU.cc:136-169) + the pixel coverage of
// vfRay's face loop (:248-274): persistent warps over the visible faces of
// all jobs, covering one face at a time with their lanes over the pixels of
// the face's bounding box in chunks of rh rows x (32 / rh) columns (rh = the box height
// rounded up to a power of two, at most 32).  The reference walks a column
// y-ascending and stops it at the first covered pixel whose entry scalar is
// out of [0,1] (:274); here the lanes of a column ballot that condition and a
// pixel is dropped if it or a pixel above it in its column has it (carried
// across row chunks of taller boxes).  The reference lets the last visible
// face in order write a pixel; visible order is ext-face order, so the
// winner is the largest ext-face index reaching it: atomicMax.  Pixels
// outside the image are clipped (the reference would write past its buffer
// there).  Reference mode; the composited mode's entry lists come from the
// screen-tile kernels below.
__global__ void __launch_bounds__(256, 4) raster_kernel(const JobDev* __restrict__ jobs, uint32_t njobs,
                                                     const uint32_t* __restrict__ vpref) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t total = vpref[njobs];
  // A warp takes 32 consecutive visible faces at a time.  Each lane loads and
  // sets up one of them (plane, box, entry edges: 32 independent load
  // chains in flight instead of one), then the warp covers the faces one
  // after another with the setup broadcast from the lane that made it
  // (1.25 -> 0.83 ms for 64 views at 512^2 against one warp per face; the
  // register bound of 4 CTAs per SM spills 20 bytes and beats the unbounded
  // 70 registers at 3 CTAs).
  for (uint32_t g0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; g0 < total;
       g0 += nwarps * 32u) {
    const uint32_t g = g0 + lane;
    bool has = false;
    uint32_t j = 0, e = 0, bx = 0, by = 0, xe = 0, ye = 0;
    EntryEdges E = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    float sa = 0.0f, sb = 0.0f, sc = 0.0f;
    double rW = 0.0, rH = 0.0;
    if (g < total) {
      j = job_of(vpref, njobs, g);
      const JobDev& J = jobs[j];
      const uint32_t i = g - vpref[j];
      const uint32_t W = J.W, H = J.H;
      e = J.vis_ext[i];
      if (id_bad(e, J.nExt)) {
        atomicOr(&J.ctr->status, kDevRange);
      } else {
        // the face's plane and vertex xy, written by stage (a): one dependent
        // load after the visible list instead of the face -> tet -> vertex chain
        const float4* pl = J.planes + kPlaneStride * (size_t)e;
        const float4 p0 = pl[0], p1 = pl[1], p2 = pl[2];
        const uint4 box = face_box(p1, p2, W, H);
        J.bbox[i] = box;
        bx = box.x;
        by = box.y;
        xe = min(box.z, W - 1);
        ye = min(box.w, H - 1);
        has = bx <= xe && by <= ye;  // else the box lies entirely outside the image
        E = entry_edges(make_float4(p1.z, p1.w, 0.0f, 0.0f), make_float4(p2.x, p2.y, 0.0f, 0.0f),
                        make_float4(p2.z, p2.w, 0.0f, 0.0f));
        sa = p0.w;
        sb = p1.x;
        sc = p1.y;
        rW = __drcp_rn((double)(float)(W - 1u));
        rH = __drcp_rn((double)(float)(H - 1u));
      }
    }
    for (uint32_t todo = __ballot_sync(0xffffffffu, has); todo; todo &= todo - 1u) {
      const int src = __ffs(todo) - 1;
      const uint32_t fj = __shfl_sync(0xffffffffu, j, src), fe = __shfl_sync(0xffffffffu, e, src);
      const uint32_t fbx = __shfl_sync(0xffffffffu, bx, src), fby = __shfl_sync(0xffffffffu, by, src);
      const uint32_t fxe = __shfl_sync(0xffffffffu, xe, src), fye = __shfl_sync(0xffffffffu, ye, src);
      EntryEdges F;
      F.v0x = __shfl_sync(0xffffffffu, E.v0x, src);
      F.v0y = __shfl_sync(0xffffffffu, E.v0y, src);
      F.e1x = __shfl_sync(0xffffffffu, E.e1x, src);
      F.e1y = __shfl_sync(0xffffffffu, E.e1y, src);
      F.e2x = __shfl_sync(0xffffffffu, E.e2x, src);
      F.e2y = __shfl_sync(0xffffffffu, E.e2y, src);
      F.cx = __shfl_sync(0xffffffffu, E.cx, src);
      const float fsa = __shfl_sync(0xffffffffu, sa, src), fsb = __shfl_sync(0xffffffffu, sb, src),
                  fsc = __shfl_sync(0xffffffffu, sc, src);
      const double frW = __shfl_sync(0xffffffffu, rW, src), frH = __shfl_sync(0xffffffffu, rH, src);
      const uint32_t W = jobs[fj].W;
      int32_t* const winner = jobs[fj].winner;
      const uint32_t h = fye - fby + 1;
      const uint32_t rh = h >= 32 ? 32u : (h <= 1 ? 1u : 1u << (32 - __clz(h - 1)));
      const uint32_t cw = 32u / rh;
      const uint32_t r = lane % rh, c = lane / rh;
      const uint32_t seg = (rh == 32 ? 0xffffffffu : ((1u << rh) - 1u)) << (c * rh);  // my column
      const uint32_t upto = seg & (lane == 31 ? 0xffffffffu : ((2u << lane) - 1u));   // rows <= mine
      for (uint32_t x0 = fbx; x0 <= fxe; x0 += cw) {
        const uint32_t px = x0 + c;
        const float ox = obj_coord_r(px, frW);
        bool carried = false;  // a kill in an earlier row chunk of this column (rh == 32)
        for (uint32_t y0 = fby; y0 <= fye; y0 += rh) {
          const uint32_t py = y0 + r;
          const bool live = px <= fxe && py <= fye;
          bool inside = false, ok = false;
          if (live) {
            const float oy = obj_coord_r(py, frH);
            inside = entry_inside(F, ox, oy);
            const float sp = plane_eval(ox, oy, fsa, fsb, fsc);
            ok = (sp >= 0.0f) && (sp <= 1.0f);
          }
          const uint32_t kill = __ballot_sync(0xffffffffu, live && inside && !ok);
          if (live && inside && ok && !carried && !(kill & upto))
            atomicMax(&winner[py * W + px], (int32_t)fe);
          carried = carried || (kill & seg);
        }
      }
    }
  }
}

// ------------------------------------------------------------ stage (b), composited mode
//
// Every visible face covering a pixel (entry scalar in [0, 1]) is an entry
// of that pixel's ray.  The faces are binned into screen tiles of 16 x 16
// pixels (count, scan, fill: one atomic per face and tile), then one CTA per
// tile stages the tile's faces in shared memory, and each thread tests its
// pixel against them and writes its pixel's entry list in descending
// (depth, face) order -- the order the traversal takes the segments in.

constexpr uint32_t kTile = 16;

// Bin pass over the visible faces of all jobs: kFill = false counts the
// screen tiles each face's box overlaps (and stores the box), kFill = true
// writes the face's visible index into each tile's bin.  tpref: prefix of
// the jobs' tile counts.
template <bool kFill>
__global__ void __launch_bounds__(256) bin_kernel(const JobDev* __restrict__ jobs, uint32_t njobs,
                                                  const uint32_t* __restrict__ vpref,
                                                  const uint32_t* __restrict__ tpref,
                                                  uint32_t* __restrict__ tile_cnt,
                                                  const uint32_t* __restrict__ tile_off,
                                                  uint32_t* __restrict__ tile_cur,
                                                  uint32_t* __restrict__ bins, uint32_t bin_cap) {
  const uint32_t total = vpref[njobs];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t g0 = blockIdx.x * blockDim.x; g0 < total; g0 += stride) {
    const uint32_t g = g0 + threadIdx.x;
    uint32_t j = 0, n = 0;
    if (g < total) {
      j = job_of(vpref, njobs, g);
      const JobDev& J = jobs[j];
      const uint32_t i = g - vpref[j];
      const uint32_t e = J.vis_ext[i];
      const bool bad = id_bad(e, J.nExt);
      if (bad) atomicOr(&J.ctr->status, kDevRange);
      const float4* pl = J.planes + kPlaneStride * (size_t)(bad ? 0u : e);
      uint4 b = face_box(pl[1], pl[2], J.W, J.H);
      if (bad) b = make_uint4(1u, 1u, 0u, 0u);  // an empty box: no tiles
      if (!kFill) J.bbox[i] = b;
      const uint32_t xe = min(b.z, J.W - 1), ye = min(b.w, J.H - 1);
      if (b.x <= xe && b.y <= ye) {
        const uint32_t tpx = (J.W + kTile - 1) / kTile, base = tpref[j];
        for (uint32_t ty = b.y / kTile; ty <= ye / kTile; ++ty)
          for (uint32_t tx = b.x / kTile; tx <= xe / kTile; ++tx) {
            const uint32_t t = base + ty * tpx + tx;
            if (!kFill) {
              atomicAdd(&tile_cnt[t], 1u);
            } else {
              const uint32_t slot = tile_off[t] + atomicAdd(&tile_cur[t], 1u);
              if (slot < bin_cap) bins[slot] = i;
            }
            ++n;
          }
      }
    }
    if (!kFill) {  // per job the (face, tile) pairs, one atomic per job and warp
      const uint32_t act = __activemask();
      const uint32_t peers = __match_any_sync(act, g < total ? j : 0xffffffffu);
      const uint32_t sum = __reduce_add_sync(peers, n);
      if (g < total && (threadIdx.x & 31u) == (uint32_t)(__ffs(peers) - 1) && sum)
        atomicAdd(&jobs[j].ctr->nbins, sum);
    }
  }
}

// A face as the tile kernel tests it: its box, entry edges, depth and
// scalar planes, ext-face index, and the tet and entry face a segment
// starting at it enters (tet << 2 | face).
struct TileFace {
  uint4 box;
  EntryEdges E;
  float zx, zy, zz, sx, sy, sz;
  uint32_t e, tf;
};

// One CTA per screen tile (a block-stride loop over the tiles of all jobs),
// one thread per pixel.  Pass 1 counts each pixel's entries; a block scan
// and one atomic on the batch's entry cursor give each pixel its list's
// place; pass 2 inserts each entry into its pixel's list in descending
// (depth, face) order.  The entry test is the rasteriser's own: the pixel in
// the face's box (clipped to the image), inside the entry face (inclusive,
// vfRayKernelCPU.cc:258-268), entry scalar in [0, 1].  Lists that do not
// fit the arena are left empty and counted, and the caller renders again
// with room (as with bins past their capacity).
__global__ void __launch_bounds__(256) tile_kernel(const JobDev* __restrict__ jobs, uint32_t njobs,
                                                   const uint32_t* __restrict__ tpref,
                                                   const uint32_t* __restrict__ tile_off,
                                                   const uint32_t* __restrict__ bins,
                                                   uint32_t bin_cap, uint4* __restrict__ ent,
                                                   uint32_t ent_cap, uint32_t* __restrict__ cursor) {
  __shared__ TileFace F[256];
  __shared__ uint32_t s_warp[8];
  __shared__ uint32_t s_base;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t ntiles = tpref[njobs];
  for (uint32_t g = blockIdx.x; g < ntiles; g += gridDim.x) {
    const uint32_t j = job_of(tpref, njobs, g);
    const JobDev& J = jobs[j];
    const uint32_t lt = g - tpref[j], W = J.W, H = J.H;
    const uint32_t tpx = (W + kTile - 1) / kTile;
    const uint32_t px = (lt % tpx) * kTile + (tid % kTile), py = (lt / tpx) * kTile + tid / kTile;
    const bool live = px < W && py < H;
    const double rW = __drcp_rn((double)(float)(W - 1u)), rH = __drcp_rn((double)(float)(H - 1u));
    const float ox = obj_coord_r(px, rW), oy = obj_coord_r(py, rH);
    const uint32_t b0 = min(tile_off[g], bin_cap), b1 = min(tile_off[g + 1], bin_cap);
    auto covers = [&](const TileFace& f) {
      return px >= f.box.x && px <= min(f.box.z, W - 1) && py >= f.box.y &&
             py <= min(f.box.w, H - 1) && entry_inside(f.E, ox, oy) && [&] {
               const float sp = plane_eval(ox, oy, f.sx, f.sy, f.sz);
               return (sp >= 0.0f) && (sp <= 1.0f);
             }();
    };
    auto stage = [&](uint32_t c) {  // faces c .. c+255 of the bin into shared memory
      __syncthreads();
      if (c + tid < b1) {
        uint32_t i = bins[c + tid];
        bool bad = id_bad(i, J.ctr->nvis);
        uint32_t e = J.vis_ext[bad ? 0u : i];
        bad = bad || id_bad(e, J.nExt);
        if (bad) {
          i = e = 0;
          atomicOr(&J.ctr->status, kDevRange);
        }
        const float4* pl = J.planes + kPlaneStride * (size_t)e;
        const float4 p0 = pl[0], p1 = pl[1], p2 = pl[2];
        TileFace f;
        f.box = bad ? make_uint4(1u, 1u, 0u, 0u) : J.bbox[i];  // bad: covers nothing
        f.E = entry_edges(make_float4(p1.z, p1.w, 0.0f, 0.0f), make_float4(p2.x, p2.y, 0.0f, 0.0f),
                          make_float4(p2.z, p2.w, 0.0f, 0.0f));
        f.zx = p0.x;
        f.zy = p0.y;
        f.zz = p0.z;
        f.sx = p0.w;
        f.sy = p1.x;
        f.sz = p1.y;
        f.e = e;
        const uint2 tf = J.extf[e];
        f.tf = (tf.x << 2) | (tf.y & 3u);
        F[tid] = f;
      }
      __syncthreads();
      return min(256u, b1 - c);
    };
    // pass 1: entries per pixel.  A tile whose bin fits one staged chunk
    // (the common case) also keeps which of the chunk's faces cover each
    // pixel, as a 256-bit mask in registers, so that pass 2 neither stages
    // nor tests the faces again.
    const bool one_chunk = b1 - b0 <= 256u;
    uint32_t cov[8];
    uint32_t count = 0;
    for (uint32_t c = b0; c < b1; c += 256) {
      const uint32_t staged = stage(c);  // every thread: stage() synchronises the block
      const uint32_t m = live ? staged : 0u;
#pragma unroll
      for (uint32_t w = 0; w < 8; ++w) {  // w is a constant after unrolling: cov stays in registers
        uint32_t bits = 0;
        const uint32_t kn = min(m, 32u * w + 32u);
        for (uint32_t k = 32u * w; k < kn; ++k)
          if (covers(F[k])) bits |= 1u << (k & 31u);
        cov[w] = bits;
        count += __popc(bits);
      }
    }
    if (b1 == b0) {
#pragma unroll
      for (uint32_t w = 0; w < 8; ++w) cov[w] = 0;
    }
    // block scan of the counts
    uint32_t x = count;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
      const uint32_t c = lane < 8 ? s_warp[lane] : 0u;
      uint32_t z = c;
      for (int o = 1; o < 8; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
        if (lane >= (uint32_t)o) z += y;
      }
      if (lane < 8) s_warp[lane] = z - c;
      if (lane == 7) {
        s_base = atomicAdd(cursor, z);
        atomicAdd(&J.ctr->nentries, z);
      }
    }
    __syncthreads();
    const uint32_t off = s_base + s_warp[warp] + x - count;
    const bool fits = off + count <= ent_cap;
    // VFR_DEV_OVERFLOW: a list or this tile's bin did not fit
    if ((live && count && !fits) || (tid == 0 && tile_off[g + 1] > bin_cap))
      atomicOr(&J.ctr->status, 16u);
    if (live) {
      const uint32_t p = py * W + px;
      J.ent_off[p] = fits ? off : 0u;
      J.ent_cnt[p] = fits ? count : 0u;
    }
    // pass 2: each pixel's entries, inserted in descending (depth, face) order
    uint32_t n = 0;
    // each entry also carries what its segment starts from (the face's tet
    // and entry face, the back colour's TF entry), so the traversal starts a
    // segment without going back through the plane and the external face
    auto insert = [&](const TileFace& f) {
      const float z = plane_eval(ox, oy, f.zx, f.zy, f.zz);
      const uint32_t cbi = (uint32_t)fmul(255.0f, plane_eval(ox, oy, f.sx, f.sy, f.sz));
      uint32_t q = n++;
      while (q > 0) {
        const uint4 a = ent[off + q - 1];
        const float za = __uint_as_float(a.x);
        if (za > z || (za == z && a.y > f.e)) break;
        ent[off + q] = a;
        --q;
      }
      ent[off + q] = make_uint4(__float_as_uint(z), f.e, f.tf, cbi);
    };
    if (one_chunk) {  // F still holds the chunk pass 1 staged
      if (live && fits && count) {
#pragma unroll
        for (uint32_t w = 0; w < 8; ++w)
          for (uint32_t bits = cov[w]; bits; bits &= bits - 1u)
            insert(F[32u * w + (uint32_t)(__ffs(bits) - 1)]);
      }
    } else {
      for (uint32_t c = b0; c < b1; c += 256) {
        const uint32_t m = stage(c);
        if (live && fits && count)
          for (uint32_t k = 0; k < m; ++k)
            if (covers(F[k])) insert(F[k]);
      }
    }
  }
}

// Ray lists: the pixels with an entry face, as start records (RayStart),
// in screen tiles of 32 pixels
// (tw x 32/tw, one warp per tile, tiles of all jobs in one index space) so
// that neighbouring rays, which walk neighbouring tets, are neighbours in the
// list and share warps.  Pixels without one are cleared in the outputs here
// (the reference zero-fills its image, main.cc:194).
__global__ void __launch_bounds__(256) raylist_kernel(const JobDev* __restrict__ jobs, uint32_t njobs,
                                                      const uint32_t* __restrict__ tpref, int mode,
                                                      uint32_t tw) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= tpref[njobs]) return;
  const uint32_t j = job_of(tpref, njobs, g);
  const JobDev& J = jobs[j];
  const uint32_t tile = g - tpref[j];
  const uint32_t th = 32u / tw;
  const uint32_t tx = (J.W + tw - 1) / tw;
  const uint32_t x = (tile % tx) * tw + (lane % tw), y = (tile / tx) * th + (lane / tw);
  bool has = false;
  uint32_t p = 0;
  RayStart rs = {0u, 0u, 0u, 0u};
  const bool inside = x < J.W && y < J.H;
  if (inside) {
    p = y * J.W + x;
    rs.p = p;
    if (mode == 0) {
      // the winning face's segment start, computed as the traversal would
      // (vfRayKernelCPU.cc:250-279): object coordinates of the pixel, the
      // plane's depth and scalar there, the face's tet and entry face
      const int32_t w = J.winner[p];
      has = w >= 0;
      if (has && id_bad((uint32_t)w, J.nExt)) {
        atomicOr(&J.ctr->status, kDevRange);
        has = false;
      }
      if (has) {
        const float4* pl = J.planes + kPlaneStride * (size_t)w;
        const float4 p0 = pl[0], p1 = pl[1];
        const float ox = obj_coord(x, J.W), oy = obj_coord(y, J.H);
        const uint2 tf = J.extf[w];
        rs.tf = (tf.x << 2) | (tf.y & 3u);
        rs.zp = __float_as_uint(plane_eval(ox, oy, p0.x, p0.y, p0.z));
        rs.cbi = (uint32_t)fmul(255.0f, plane_eval(ox, oy, p0.w, p1.x, p1.y));
        if (id_bad(tf.x, J.nT)) {
          atomicOr(&J.ctr->status, kDevRange);
          has = false;
        }
      }
    } else {
      has = J.ent_cnt[p] > 0;
    }
  }
  const uint32_t m = __ballot_sync(0xffffffffu, has);
  if (m) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&J.ctr->nrays, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (has) J.rays[base + __popc(m & ((1u << lane) - 1u))] = rs;
  }
  if (inside && !has) {
    if (J.rgb8) {
      uint8_t* o = J.rgb8 + 3 * (size_t)p;
      o[0] = 0; o[1] = 0; o[2] = 0;
    }
    if (J.rgba) J.rgba[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (J.steps) J.steps[p] = 0;
  }
}

// Exclusive scan of the batch's entry-count arena (composited mode): block
// scans, then each block adds the sums of the blocks before it.
__global__ void __launch_bounds__(1024) scan_blocks_kernel(const uint32_t* __restrict__ in,
                                                           uint32_t n, uint32_t* __restrict__ out,
                                                           uint32_t* __restrict__ sums) {
  __shared__ uint32_t s[32];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t v = i < n ? in[i] : 0u;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) s[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const uint32_t c = lane < (blockDim.x >> 5) ? s[lane] : 0u;
    uint32_t z = c;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= (uint32_t)o) z += y;
    }
    s[lane] = z - c;
    if (lane == 31) sums[blockIdx.x] = z;
  }
  __syncthreads();
  if (i < n) out[i] = x - v + s[warp];
}

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
    uint32_t x = lane < (blockDim.x >> 5) ? s[lane] : 0u;
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) s_base = x;
  }
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += s_base;
  if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total = s_base + sums[blockIdx.x];
}

}  // namespace vfr
