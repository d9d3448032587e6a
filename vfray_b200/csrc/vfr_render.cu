// The C ABI of the VF-Ray render path (include/vfray.h): contexts, resident
// meshes and tables, and batches of views run as stream-ordered launches.
//
// Replaces the host driver of the reference (vfRay.cu:165-594): there the
// stages communicate through globals, texture bindings and a host round trip
// for the visible-face compaction; here a batch of views is one chain of
// kernels on one stream whose intermediate counts stay on the device, so
// nothing waits on the host between stages and the chain can be captured as a
// CUDA graph.  A single view is a batch of one job.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "vfr_internal.h"
#include "vfr_traverse.cuh"
#include "vfray.h"

namespace vfr {

const char* status_string(int s) {
  switch (s) {
    case VFR_OK: return "ok";
    case VFR_ERR_INVALID: return "invalid argument";
    case VFR_ERR_CUDA: return "CUDA error";
    case VFR_ERR_MESH: return "mesh failed validation";
    case VFR_ERR_NOMEM: return "out of memory";
    case VFR_ERR_DEVICE: return "device kernel reported an error";
    case VFR_ERR_STATE: return "call out of order or unknown handle";
    case VFR_ERR_IO: return "file error";
    case VFR_ERR_BUDGET: return "request exceeds the memory budget";
    case VFR_ERR_TIMEOUT: return "bounded device wait gave up";
    default: return "unknown status";
  }
}

// ------------------------------------------------------------------ Ctx

Ctx::~Ctx() {
  cudaStreamSynchronize(stream ? stream : own_stream);
  meshes.clear();
  if (d_tf) cudaFree(d_tf);
  if (d_psi) cudaFree(d_psi);
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  for (auto* v : {&prof_pool, &prof_live})
    for (auto& s : *v)
      for (auto& e : s.e)
        if (e) cudaEventDestroy(e);
  if (own_stream) cudaStreamDestroy(own_stream);
}

int Ctx::fail(int code, const std::string& msg) {
  err = msg;
  return code;
}

int Ctx::cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return VFR_OK;
  cudaGetLastError();
  return fail(e == cudaErrorMemoryAllocation ? VFR_ERR_NOMEM : VFR_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

int Ctx::grow(Buf& b, size_t bytes, const char* what) {
  if (bytes == 0) bytes = 16;
  if (b.cap >= bytes && b.p) return VFR_OK;
  if (b.p) {
    cudaDeviceSynchronize();  // in-flight work (any stream) may still use the old buffer
    cudaFree(b.p);
  }
  b.p = nullptr;
  b.cap = 0;
  // half again as much as asked: a buffer that keeps growing (a server's
  // batches of varying size) settles after a few steps, and every growth
  // waits for the device
  const size_t want = bytes + bytes / 2 + 256;
  int rc = cuda(cudaMalloc(&b.p, want), what);
  if (rc) return rc;
  b.cap = want;
  return VFR_OK;
}

Mesh* Ctx::mesh(int id) {
  if (id < 0 || id >= (int)meshes.size() || !meshes[id]) return nullptr;
  return meshes[id].get();
}

void Ctx::prof_mark(int k, cudaStream_t on) {
  if (!profile) return;
  if (k == 0) {
    StageEvents s;
    if (!prof_pool.empty()) {
      s = prof_pool.back();
      prof_pool.pop_back();
    } else {
      for (auto& e : s.e) cudaEventCreate(&e);
    }
    prof_live.push_back(s);
  }
  cudaEventRecord(prof_live.back().e[k], on ? on : stream);
}

const void* Ctx::traverse_fn(int mode, uint32_t variant) {
  if (mode == VFR_MODE_REF)
    return variant ? (const void*)traverse_kernel<0, 3> : (const void*)traverse_kernel<0, 2>;
  return variant ? (const void*)traverse_kernel<1, 3> : (const void*)traverse_kernel<1, 2>;
}

int Ctx::traverse_blocks_per_sm(int mode) {
  if (tune.blocks_per_sm) return (int)tune.blocks_per_sm;
  int& cached = occ[(mode ? 2 : 0) + (tune.variant ? 1 : 0)];
  if (!cached) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, traverse_fn(mode, tune.variant), 256, 0);
    cached = std::max(1, n);
  }
  return cached;
}

int Ctx::check_status(uint32_t status, uint32_t overflow) {
  if (overflow) return fail(VFR_ERR_DEVICE, "entry lists or tile bins overflowed; render again");
  if (status & (VFR_DEV_CYCLE | VFR_DEV_RANGE | VFR_DEV_STEP_CAP | VFR_DEV_OVERFLOW)) {
    char buf[128];
    std::snprintf(buf, sizeof buf, "device status 0x%x (step-cap=2 range=4 overflow=16 cycle=32)",
                  status);
    return fail(VFR_ERR_DEVICE, buf);
  }
  return VFR_OK;
}

// ------------------------------------------------------------------ Batch

Batch::~Batch() {
  drop_graph();
  if (stage) cudaFreeHost(stage);
  if (stage_done) cudaEventDestroy(stage_done);
}

cudaStream_t Batch::st() const { return stream ? stream : ctx->stream; }

void Batch::drop_graph() {
  if (exec) cudaGraphExecDestroy(exec);
  exec = nullptr;
}

static uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// The mesh's distinct edges, once per mesh: the 6 edge keys of every tet,
// sorted (CUB radix sort over the bits the vertex ids use) and made unique.
// Temporaries are freed before returning; the stream is synchronised.
int Ctx::mesh_edges(Mesh* m, cudaStream_t st) {
  if (m->edges) return VFR_OK;
  const size_t n = 6 * (size_t)m->nT;
  int bits = 1;
  while (bits < 32 && (1ull << bits) < m->nV) ++bits;
  unsigned long long *keys = nullptr, *sorted = nullptr, *uniq = nullptr;
  unsigned long long* count = nullptr;
  void* tmp = nullptr;
  size_t tmp_sort = 0, tmp_uniq = 0;
  int rc = cuda(cudaMalloc(&keys, n * 8), "edge keys");
  if (!rc) rc = cuda(cudaMalloc(&sorted, n * 8), "edge keys");
  if (!rc) rc = cuda(cudaMalloc(&uniq, n * 8), "edge keys");
  if (!rc) rc = cuda(cudaMalloc(&count, sizeof(unsigned long long)), "edge count");
  if (!rc) {
    cub::DeviceRadixSort::SortKeys(nullptr, tmp_sort, keys, sorted, n, 0, 32 + bits, st);
    cub::DeviceSelect::Unique(nullptr, tmp_uniq, sorted, uniq, count, n, st);
    rc = cuda(cudaMalloc(&tmp, std::max(tmp_sort, tmp_uniq)), "edge sort scratch");
  }
  if (!rc) {
    edge_keys_kernel<<<cdiv(m->nT, 256), 256, 0, st>>>(m->tet, m->nT, keys);
    rc = cuda(cub::DeviceRadixSort::SortKeys(tmp, tmp_sort, keys, sorted, n, 0, 32 + bits, st),
              "edge sort");
  }
  if (!rc) rc = cuda(cub::DeviceSelect::Unique(tmp, tmp_uniq, sorted, uniq, count, n, st), "edge unique");
  unsigned long long ne = 0;
  if (!rc)
    rc = cuda(cudaMemcpyAsync(&ne, count, sizeof(ne), cudaMemcpyDeviceToHost, st), "edge count");
  if (!rc) rc = cuda(cudaStreamSynchronize(st), "edge build");
  if (!rc) rc = cuda(cudaMalloc(&m->edges, sizeof(uint2) * std::max<size_t>(ne, 1)), "edges");
  if (!rc) rc = cuda(cudaMemcpyAsync(m->edges, uniq, sizeof(uint2) * ne, cudaMemcpyDeviceToDevice, st),
                     "edges");
  if (!rc) rc = cuda(cudaStreamSynchronize(st), "edge build");
  for (void* p : {(void*)keys, (void*)sorted, (void*)uniq, (void*)count, tmp})
    if (p) cudaFree(p);
  if (rc) {
    if (m->edges) cudaFree(m->edges);
    m->edges = nullptr;
    return rc;
  }
  m->nEdges = (uint32_t)ne;
  m->bytes += sizeof(uint2) * ne;
  return VFR_OK;
}

// Lays the jobs out in the batch's arenas (allocating what is missing) and
// fills the job table on the host.
// A buffer of the layout: grown (the batch's own memory) or the next piece
// of the arena, 256-byte aligned.
int Batch::place(Buf& b, size_t bytes, const char* what) {
  if (!arena) return ctx->grow(b, bytes, what);
  const size_t need = (std::max<size_t>(bytes, 16) + 255) & ~(size_t)255;
  if (arena->off + need > arena->cap) return ctx->fail(VFR_ERR_BUDGET, std::string(what) + ": arena full");
  b.release();
  b.p = arena->base + arena->off;
  b.cap = need;
  b.owned = false;
  arena->off += need;
  return VFR_OK;
}

// The arena bytes layout() places for these jobs: every buffer kind's total
// rounded up to 256 bytes (the same sizes, in the same order).
size_t Batch::arena_bytes(Ctx& C, const std::vector<JobSpec>& s, int mode, uint32_t fb,
                          bool rgb8_only) {
  const size_t nj = s.size();
  size_t nv_mv = 0, next = 0, nblk = 0, pix = 0, stiles = 0;
  for (const JobSpec& q : s) {
    const Mesh* m = C.mesh(q.mesh);
    if (!m) continue;
    nv_mv += q.use_mv ? m->nV : 0;
    next += m->nExt;
    nblk += cdiv(m->nExt, fb);
    pix += (size_t)q.W * q.H;
    stiles += (size_t)cdiv(q.W, kTile) * cdiv(q.H, kTile);
  }
  auto a = [](size_t b) { return (std::max<size_t>(b, 16) + 255) & ~(size_t)255; };
  size_t t = a(sizeof(JobDev) * nj) + a(sizeof(uint32_t) * 5 * (nj + 1)) +
             a(sizeof(uint32_t) * (2 * (nj + 1) + 4)) + a(sizeof(ViewCounters) * nj) +
             a(sizeof(float4) * nv_mv) + a(sizeof(float4) * kPlaneStride * next) +
             a(sizeof(uint32_t) * nblk) + a(sizeof(uint32_t) * next) + a(sizeof(uint4) * next) +
             a(sizeof(RayStart) * pix);
  if (mode == VFR_MODE_REF) t += a(sizeof(int32_t) * pix);
  if (mode == VFR_MODE_COMPOSITED)
    t += 2 * a(sizeof(uint32_t) * pix) + 2 * a(sizeof(uint32_t) * (stiles + 1)) +
         a(sizeof(uint32_t) * stiles) + a(sizeof(uint32_t) * (cdiv(stiles + 1, fb) + 1)) +
         a(sizeof(uint32_t) * (32 * stiles + 4 * next)) + a(sizeof(uint4) * (pix * 4 + 1024));
  t += a(3 * pix);
  if (!rgb8_only) t += a(sizeof(float4) * pix) + a(sizeof(uint32_t) * pix);
  return t;
}

int Batch::layout(const std::vector<JobSpec>& s, int m, bool own_outputs) {
  Ctx& C = *ctx;
  specs = s;
  mode = m;
  tile_w = C.tune.tile_w;
  njobs = (uint32_t)s.size();
  jobs.assign(njobs, JobDev{});
  pref.assign(5 * (size_t)(njobs + 1), 0);
  uint32_t* pr = pref.data();
  uint32_t* pe = pr + (njobs + 1);
  uint32_t* px = pe + (njobs + 1);
  uint32_t* pt = px + (njobs + 1);
  uint32_t* ps = pt + (njobs + 1);  // composited: 16 x 16 screen tiles
  size_t nv_mv = 0, next = 0, nblk = 0, pix = 0;
  for (uint32_t j = 0; j < njobs; ++j) {
    Mesh* mesh = C.mesh(s[j].mesh);
    if (!mesh) return C.fail(VFR_ERR_STATE, "unknown mesh id in job");
    const JobSpec& q = s[j];
    if (q.W < 2 || q.H < 2 || (uint64_t)q.W * q.H > (1ull << 28))
      return C.fail(VFR_ERR_INVALID, "image size out of range");
    const uint32_t rb =
        q.use_mv ? std::max<uint32_t>(1, std::min<uint32_t>(cdiv(mesh->nV, 1024), 2 * C.num_sms)) : 0;
    if (q.use_mv && !mesh->edges) {
      // built once per mesh (allocates and waits): a server builds them all
      // before its launch starts
      if (arena) return C.fail(VFR_ERR_STATE, "mesh edges missing for an arena layout");
      const int rc = C.mesh_edges(mesh, st());
      if (rc) return rc;
    }
    const uint32_t eb =
        q.use_mv ? std::max<uint32_t>(1, std::min<uint32_t>(cdiv(mesh->nEdges, 1024), 4 * C.num_sms))
                 : 0;
    const uint32_t xb = cdiv(mesh->nExt, fb);
    const uint32_t tl = cdiv(q.W, C.tune.tile_w) * cdiv(q.H, 32 / C.tune.tile_w);
    pr[j + 1] = pr[j] + rb;
    pe[j + 1] = pe[j] + eb;
    px[j + 1] = px[j] + xb;
    pt[j + 1] = pt[j] + tl;
    ps[j + 1] = ps[j] + cdiv(q.W, kTile) * cdiv(q.H, kTile);
    nv_mv += q.use_mv ? mesh->nV : 0;
    next += mesh->nExt;
    nblk += xb;
    pix += (size_t)q.W * q.H;
  }
  rot_blocks = pr[njobs];
  edge_blocks = pe[njobs];
  ext_blocks = px[njobs];
  tiles = pt[njobs];
  stiles = ps[njobs];
  pixels = pix;
  ext_total = next;
  if (pix > 0xffffffffull || next > 0xffffffffull) return C.fail(VFR_ERR_BUDGET, "batch too large");
  const size_t old_sig = (size_t)vview.p ^ (size_t)planes.p ^ (size_t)winner.p ^ (size_t)rays.p ^
                         (size_t)ent.p ^ (size_t)d_jobs.p;
  int rc = place(d_jobs, sizeof(JobDev) * njobs, "job table");
  if (!rc) rc = place(d_pref, sizeof(uint32_t) * pref.size(), "job prefixes");
  if (!rc) rc = place(d_dev_pref, sizeof(uint32_t) * (2 * (size_t)(njobs + 1) + 4), "device prefixes");
  if (!rc) rc = place(d_ctr, sizeof(ViewCounters) * njobs, "view counters");
  if (!rc) rc = place(vview, sizeof(float4) * nv_mv, "view vertices");
  if (!rc) rc = place(planes, sizeof(float4) * kPlaneStride * next, "planes");
  if (!rc) rc = place(blk, sizeof(uint32_t) * nblk, "block counts");
  if (!rc) rc = place(vis, sizeof(uint32_t) * next, "visible lists");
  if (!rc) rc = place(bbox, sizeof(uint4) * next, "bboxes");
  if (!rc) rc = place(rays, sizeof(RayStart) * pix, "ray lists");
  if (!rc && mode == VFR_MODE_REF) rc = place(winner, sizeof(int32_t) * pix, "winner maps");
  if (!rc && mode == VFR_MODE_COMPOSITED) {
    if (ent_cap == 0) ent_cap = (C.ent_cap_hint && !arena) ? C.ent_cap_hint : pix * 4 + 1024;
    if (bin_cap == 0)
      bin_cap = (C.bin_cap_hint && !arena) ? C.bin_cap_hint : 32 * (size_t)stiles + 4 * next;
    rc = place(ent_cnt, sizeof(uint32_t) * pix, "entry counts");
    if (!rc) rc = place(ent_off, sizeof(uint32_t) * pix, "entry offsets");
    if (!rc) rc = place(tile_cnt, sizeof(uint32_t) * (stiles + 1), "tile counts");
    if (!rc) rc = place(tile_off, sizeof(uint32_t) * (stiles + 1), "tile offsets");
    if (!rc) rc = place(tile_cur, sizeof(uint32_t) * stiles, "tile cursors");
    if (!rc) rc = place(scan, sizeof(uint32_t) * (cdiv(stiles + 1, fb) + 1), "scan sums");
    if (!rc) rc = place(bins, sizeof(uint32_t) * bin_cap, "tile bins");
    if (!rc) rc = place(ent, sizeof(uint4) * ent_cap, "entries");
  }
  if (!rc && own_outputs) {
    rc = place(out_rgb8, 3 * pix, "rgb8 outputs");
    if (!rc && !rgb8_only) rc = place(out_rgba, sizeof(float4) * pix, "rgba outputs");
    if (!rc && !rgb8_only) rc = place(out_steps, sizeof(uint32_t) * pix, "steps outputs");
  }
  if (rc) return rc;
  const size_t new_sig = (size_t)vview.p ^ (size_t)planes.p ^ (size_t)winner.p ^ (size_t)rays.p ^
                         (size_t)ent.p ^ (size_t)d_jobs.p;
  if (new_sig != old_sig) drop_graph();
  scratch_bytes = vview.cap + planes.cap + blk.cap + vis.cap + bbox.cap + rays.cap + winner.cap +
                  ent_cnt.cap + ent_off.cap + tile_cnt.cap + tile_off.cap + tile_cur.cap + bins.cap +
                  ent.cap + scan.cap + d_ctr.cap;
  size_t ov = 0, oe = 0, ob = 0, op = 0;
  for (uint32_t j = 0; j < njobs; ++j) {
    Mesh* mesh = C.mesh(s[j].mesh);
    const JobSpec& q = s[j];
    JobDev& J = jobs[j];
    J.m0 = make_float4(q.mv[0], q.mv[1], q.mv[2], q.mv[3]);
    J.m1 = make_float4(q.mv[4], q.mv[5], q.mv[6], q.mv[7]);
    J.m2 = make_float4(q.mv[8], q.mv[9], q.mv[10], q.mv[11]);
    J.tet = mesh->tet;
    J.edges = mesh->edges;
    J.nEdges = mesh->nEdges;
    J.walk = mesh->walk;
    J.vert_in = mesh->vert;
    J.extf = mesh->extf;
    J.vview = q.use_mv ? vview.as<float4>(sizeof(float4) * ov) : nullptr;
    J.vert = q.use_mv ? J.vview : mesh->vert;
    J.planes = planes.as<float4>(sizeof(float4) * kPlaneStride * oe);
    J.blk = blk.as<uint32_t>(sizeof(uint32_t) * ob);
    J.vis_ext = vis.as<uint32_t>(sizeof(uint32_t) * oe);
    J.bbox = bbox.as<uint4>(sizeof(uint4) * oe);
    J.winner = mode == VFR_MODE_REF ? winner.as<int32_t>(sizeof(int32_t) * op) : nullptr;
    J.rays = rays.as<RayStart>(sizeof(RayStart) * op);
    J.ent_cnt = mode == VFR_MODE_COMPOSITED ? ent_cnt.as<uint32_t>(sizeof(uint32_t) * op) : nullptr;
    J.ent_off = mode == VFR_MODE_COMPOSITED ? ent_off.as<uint32_t>(sizeof(uint32_t) * op) : nullptr;
    J.ctr = d_ctr.as<ViewCounters>(sizeof(ViewCounters) * j);
    J.ent = mode == VFR_MODE_COMPOSITED ? ent.as<uint4>() : nullptr;
    J.ent_cap = (uint32_t)std::min<size_t>(ent_cap, 0xffffffffu);
    J.mode = (uint32_t)mode;
    if (own_outputs) {
      specs[j].rgb8 = out_rgb8.as<uint8_t>(3 * op);
      specs[j].rgba = rgb8_only ? nullptr : out_rgba.as<float4>(sizeof(float4) * op);
      specs[j].steps = rgb8_only ? nullptr : out_steps.as<uint32_t>(sizeof(uint32_t) * op);
    }
    J.rgb8 = specs[j].rgb8;
    J.rgba = specs[j].rgba;
    J.steps = specs[j].steps;
    J.nV = mesh->nV;
    J.nT = mesh->nT;
    J.nExt = mesh->nExt;
    J.W = q.W;
    J.H = q.H;
    J.use_mv = q.use_mv ? 1u : 0u;
    J.maxEdge_in = mesh->maxEdge;
    J.pix_base = (uint32_t)op;
    ov += q.use_mv ? mesh->nV : 0;
    oe += mesh->nExt;
    ob += cdiv(mesh->nExt, fb);
    op += (size_t)q.W * q.H;
  }
  return VFR_OK;
}

// Uploads the job table and prefixes; async: through pinned staging, stream
// ordered (the staging is reused only after the previous copy has run).
int Batch::upload(bool async) {
  Ctx& C = *ctx;
  const size_t bj = sizeof(JobDev) * njobs, bp = sizeof(uint32_t) * pref.size();
  if (!async) {
    int rc = C.cuda(cudaMemcpyAsync(d_jobs.p, jobs.data(), bj, cudaMemcpyHostToDevice, st()),
                    "job table upload");
    if (!rc)
      rc = C.cuda(cudaMemcpyAsync(d_pref.p, pref.data(), bp, cudaMemcpyHostToDevice, st()),
                  "prefix upload");
    if (!rc) rc = C.cuda(cudaStreamSynchronize(st()), "upload");
    return rc;
  }
  if (ext_stage) {  // the caller's pinned staging, used once (no allocation, no wait)
    if (ext_stage_cap < bj + bp) return C.fail(VFR_ERR_INVALID, "staging too small");
    std::memcpy(ext_stage, jobs.data(), bj);
    std::memcpy(ext_stage + bj, pref.data(), bp);
    int rc = C.cuda(cudaMemcpyAsync(d_jobs.p, ext_stage, bj, cudaMemcpyHostToDevice, st()),
                    "job table upload");
    if (!rc)
      rc = C.cuda(cudaMemcpyAsync(d_pref.p, ext_stage + bj, bp, cudaMemcpyHostToDevice, st()),
                  "prefix upload");
    return rc;
  }
  if (!stage_done) cudaEventCreateWithFlags(&stage_done, cudaEventDisableTiming);
  if (stage_cap < bj + bp) {
    cudaEventSynchronize(stage_done);
    if (stage) cudaFreeHost(stage);
    stage = nullptr;
    stage_cap = 0;
    if (cudaMallocHost(&stage, bj + bp + 4096) != cudaSuccess) return C.fail(VFR_ERR_NOMEM, "staging");
    stage_cap = bj + bp + 4096;
  }
  cudaEventSynchronize(stage_done);
  std::memcpy(stage, jobs.data(), bj);
  std::memcpy((char*)stage + bj, pref.data(), bp);
  int rc = C.cuda(cudaMemcpyAsync(d_jobs.p, stage, bj, cudaMemcpyHostToDevice, st()),
                  "job table upload");
  if (!rc)
    rc = C.cuda(cudaMemcpyAsync(d_pref.p, (char*)stage + bj, bp, cudaMemcpyHostToDevice, st()),
                "prefix upload");
  cudaEventRecord(stage_done, st());
  return rc;
}

int Batch::enqueue_a() {
  Ctx& C = *ctx;
  const cudaStream_t st = Batch::st();
  const JobDev* J = d_jobs.as<JobDev>();
  const uint32_t* P = d_pref.as<uint32_t>();
  const uint32_t n1 = njobs + 1;
  init_jobs_kernel<<<cdiv(njobs, 128), 128, 0, st>>>(J, njobs, queue());
  if (rot_blocks) {
    view_rotate_kernel<<<rot_blocks, 256, 0, st>>>(J, njobs, P);
    view_normalize_kernel<<<rot_blocks, 256, 0, st>>>(J, njobs, P);
    view_maxedge_kernel<<<edge_blocks, 256, 0, st>>>(J, njobs, P + n1);
  }
  if (ext_blocks) {
    visible_kernel<<<ext_blocks, fb, 0, st>>>(J, njobs, P + 2 * n1);
    compact_kernel<<<ext_blocks, fb, 0, st>>>(J, njobs, P + 2 * n1);
  }
  prefix_kernel<<<1, fb, 0, st>>>(J, njobs, 0, vis_pref());
  return C.cuda(cudaGetLastError(), "stage (a) launch");
}

int Batch::enqueue_b() {
  Ctx& C = *ctx;
  const cudaStream_t st = Batch::st();
  const JobDev* J = d_jobs.as<JobDev>();
  const uint32_t* P = d_pref.as<uint32_t>();
  const uint32_t n1 = njobs + 1;
  const uint32_t rb = std::max(1, C.num_sms * (int)C.tune.raster_warps_per_sm / 8);
  if (mode == VFR_MODE_REF) {
    cudaMemsetAsync(winner.p, 0xff, sizeof(int32_t) * pixels, st);
    raster_kernel<<<rb, 256, 0, st>>>(J, njobs, vis_pref());
  } else {
    // faces binned into 16 x 16 screen tiles, then per tile the pixels'
    // depth-ordered entry lists
    const uint32_t n = stiles + 1, nsb = cdiv(n, fb);
    const uint32_t* ps = P + 4 * n1;
    const uint32_t bcap = (uint32_t)std::min<size_t>(bin_cap, 0xffffffffu);
    cudaMemsetAsync(tile_cnt.p, 0, sizeof(uint32_t) * n, st);
    cudaMemsetAsync(tile_cur.p, 0, sizeof(uint32_t) * stiles, st);
    bin_kernel<false><<<rb, 256, 0, st>>>(J, njobs, vis_pref(), ps, tile_cnt.as<uint32_t>(), nullptr,
                                          nullptr, nullptr, 0);
    scan_blocks_kernel<<<nsb, fb, 0, st>>>(tile_cnt.as<uint32_t>(), n, tile_off.as<uint32_t>(),
                                             scan.as<uint32_t>());
    scan_add_kernel<<<nsb, fb, 0, st>>>(tile_off.as<uint32_t>(), n, scan.as<uint32_t>(), nullptr);
    bin_kernel<true><<<rb, 256, 0, st>>>(J, njobs, vis_pref(), ps, nullptr, tile_off.as<uint32_t>(),
                                         tile_cur.as<uint32_t>(), bins.as<uint32_t>(), bcap);
    if (stiles)
      tile_kernel<<<std::min<uint32_t>(stiles, (uint32_t)C.num_sms * 8), 256, 0, st>>>(
          J, njobs, ps, tile_off.as<uint32_t>(), bins.as<uint32_t>(), bcap, ent.as<uint4>(),
          (uint32_t)std::min<size_t>(ent_cap, 0xffffffffu), queue() + 1);
  }
  if (tiles) raylist_kernel<<<cdiv(tiles, 8), 256, 0, st>>>(J, njobs, P + 3 * n1, mode, tile_w);
  prefix_kernel<<<1, fb, 0, st>>>(J, njobs, 1, ray_pref());
  return C.cuda(cudaGetLastError(), "stage (b) launch");
}

int Batch::enqueue_c() {
  Ctx& C = *ctx;
  TraverseParams P;
  P.jobs = d_jobs.as<JobDev>();
  P.njobs = njobs;
  P.ray_pref = ray_pref();
  P.queue = queue();
  P.tf = C.d_tf;
  P.psi = C.d_psi;
  P.e2tab = reinterpret_cast<const double*>(C.d_tf + 256);
  P.step_cap = C.step_cap;
  P.refill = C.tune.refill;
  const int blocks = C.num_sms * C.traverse_blocks_per_sm(mode);
  void* args[] = {&P};
  return C.cuda(cudaLaunchKernel(C.traverse_fn(mode, C.tune.variant), dim3(blocks), dim3(256), args,
                                 0, st()),
                "stage (c) launch");
}

int Batch::capture() {
  Ctx& C = *ctx;
  drop_graph();
  cudaGraph_t g = nullptr;
  int rc = C.cuda(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal), "capture");
  if (rc) return rc;
  rc = enqueue_all();
  cudaError_t e = cudaStreamEndCapture(st(), &g);
  if (!rc) rc = C.cuda(e, "end capture");
  if (!rc) rc = C.cuda(cudaGraphInstantiate(&exec, g, 0), "graph instantiate");
  if (g) cudaGraphDestroy(g);
  if (rc) exec = nullptr;
  return rc;
}

int Batch::run() {
  if (exec) return ctx->cuda(cudaGraphLaunch(exec, st()), "graph launch");
  return enqueue_all();
}

// Composited mode: whether the entry lists or the tile bins of the last run
// needed more room than the layout gave them; if so the context's hints are
// raised to the need (the next layout of a batch with ent_cap / bin_cap 0
// sizes for it).
bool Batch::overflowed(const std::vector<ViewCounters>& k) {
  if (mode != VFR_MODE_COMPOSITED) return false;
  uint64_t ents = 0, bns = 0;
  for (const ViewCounters& x : k) {
    ents += x.nentries;
    bns += x.nbins;
  }
  const bool over = ents > ent_cap || bns > bin_cap;
  if (over && ctx) {
    ctx->ent_cap_hint = std::max<size_t>(ctx->ent_cap_hint, ents + ents / 8 + 1024);
    ctx->bin_cap_hint = std::max<size_t>(ctx->bin_cap_hint, bns + bns / 8 + 1024);
  }
  return over;
}

int Batch::counters(std::vector<ViewCounters>& out) {
  Ctx& C = *ctx;
  out.resize(njobs);
  int rc = C.cuda(cudaMemcpyAsync(out.data(), d_ctr.p, sizeof(ViewCounters) * njobs,
                                  cudaMemcpyDeviceToHost, st()),
                  "counter read");
  if (!rc) rc = C.cuda(cudaStreamSynchronize(st()), "stream sync");
  return rc;
}

int serve_blocks_per_sm(int* n) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, serve_kernel<3>, 256, 0) == cudaSuccess
             ? VFR_OK
             : VFR_ERR_CUDA;
}

cudaError_t launch_serve(const ServeParams& sp, int grid, cudaStream_t st) {
  serve_kernel<3><<<grid, 256, 0, st>>>(sp);
  return cudaGetLastError();
}

cudaError_t launch_publish(SegDev* segs, ServeCtl* ctl, uint32_t seq, const JobDev* jobs,
                           const uint32_t* ray_pref, uint32_t* done, uint32_t njobs,
                           cudaStream_t st) {
  publish_kernel<<<1, 256, 0, st>>>(segs, ctl, seq, jobs, ray_pref, done, njobs);
  return cudaGetLastError();
}

}  // namespace vfr

using vfr::Batch;
using vfr::Ctx;
using vfr::JobSpec;
using vfr::Mesh;

struct vfr_batch {
  vfr_ctx* owner = nullptr;
  Batch b;
};

// Waits for the context stream and for the streams of the context's batches
// (a batch may run on a stream of its own): done before memory that their
// launches may read is freed or overwritten.
static void sync_context(Ctx& C) {
  cudaStreamSynchronize(C.stream);
  for (void* p : C.batches) cudaStreamSynchronize(static_cast<vfr_batch*>(p)->b.st());
}

#define CTX_OR_FAIL(c)              \
  if (!(c)) return VFR_ERR_INVALID; \
  Ctx& C = (c)->impl;               \
  (void)C;                          \
  cudaSetDevice(C.device);

namespace {

void fill_stats(const vfr::ViewCounters& k, uint32_t next, vfr_render_stats* s) {
  s->num_ext = next;
  s->num_vis = k.nvis;
  s->num_rays = k.nrays;
  s->num_entries = k.nentries;
  s->num_steps = k.steps;
  s->device_status = k.status;
}

// The single-view calls run the context's one-job batch.
int single(Ctx& C, int mesh, const float* mv16, uint32_t W, uint32_t H, int mode, bool own,
           uint8_t* rgb8, float4* rgba, uint32_t* steps) {
  JobSpec q;
  q.mesh = mesh;
  q.W = W;
  q.H = H;
  q.use_mv = mv16 != nullptr;
  if (mv16) std::memcpy(q.mv, mv16, sizeof q.mv);
  q.rgb8 = rgb8;
  q.rgba = rgba;
  q.steps = steps;
  C.plain.ctx = &C;
  int rc = C.plain.layout({q}, mode, own);
  if (!rc) rc = C.plain.upload(true);
  return rc;
}

int copy_out(Ctx& C, uint8_t* rgb8, float* rgba, uint32_t* steps, size_t np) {
  Batch& B = C.plain;
  int rc = VFR_OK;
  if (rgb8)
    rc = C.cuda(cudaMemcpyAsync(rgb8, B.out_rgb8.p, np * 3, cudaMemcpyDeviceToHost, C.stream),
                "rgb8 read");
  if (!rc && rgba)
    rc = C.cuda(cudaMemcpyAsync(rgba, B.out_rgba.p, np * sizeof(float4), cudaMemcpyDeviceToHost,
                                C.stream),
                "rgba read");
  if (!rc && steps)
    rc = C.cuda(cudaMemcpyAsync(steps, B.out_steps.p, np * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, C.stream),
                "steps read");
  if (!rc) rc = C.cuda(cudaStreamSynchronize(C.stream), "output read");
  return rc;
}

}  // namespace

extern "C" {

const char* vfr_status_string(int s) { return vfr::status_string(s); }

int vfr_create(vfr_ctx** out, int device) {
  if (!out) return VFR_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return VFR_ERR_CUDA;
  }
  std::unique_ptr<vfr_ctx> c(new vfr_ctx);
  Ctx& C = c->impl;
  C.device = device;
  if (cudaSetDevice(device) != cudaSuccess) return VFR_ERR_CUDA;
  cudaDeviceGetAttribute(&C.num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&C.own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return VFR_ERR_CUDA;
  C.stream = C.own_stream;
  C.plain.ctx = &C;
  for (auto& e : C.ev) cudaEventCreate(&e);
  *out = c.release();
  return VFR_OK;
}

void vfr_destroy(vfr_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->impl.device);
  sync_context(c->impl);
  // batches that outlive their context keep only their own memory; any call
  // on them but vfr_batch_destroy then returns VFR_ERR_STATE
  for (void* p : c->impl.batches) {
    vfr_batch* b = static_cast<vfr_batch*>(p);
    b->owner = nullptr;
    b->b.ctx = nullptr;
  }
  delete c;
}

const char* vfr_last_error(const vfr_ctx* c) { return c ? c->impl.err.c_str() : "null context"; }

int vfr_set_stream(vfr_ctx* c, void* stream) {
  CTX_OR_FAIL(c);
  cudaStreamSynchronize(C.stream);
  C.stream = stream ? (cudaStream_t)stream : C.own_stream;
  C.plain.drop_graph();
  return VFR_OK;
}

int vfr_synchronize(vfr_ctx* c) {
  CTX_OR_FAIL(c);
  return C.cuda(cudaStreamSynchronize(C.stream), "synchronize");
}

int vfr_set_option(vfr_ctx* c, int option, int64_t value) {
  CTX_OR_FAIL(c);
  if (value < 0 || value > 0x7fffffff) return C.fail(VFR_ERR_INVALID, "option value out of range");
  switch (option) {
    case VFR_OPT_STEP_CAP: C.step_cap = (uint32_t)value; return VFR_OK;
    case VFR_OPT_BLOCKS_PER_SM: C.tune.blocks_per_sm = (uint32_t)value; return VFR_OK;
    case VFR_OPT_PROFILE: C.profile = value != 0; return VFR_OK;
    case VFR_OPT_TRAVERSE_VARIANT:
      if (value > 1) return C.fail(VFR_ERR_INVALID, "traversal variant is 0 or 1");
      C.tune.variant = (uint32_t)value;
      return VFR_OK;
    case VFR_OPT_REFILL:
      if (value < 1 || value > 32) return C.fail(VFR_ERR_INVALID, "refill is 1..32");
      C.tune.refill = (uint32_t)value;
      return VFR_OK;
    case VFR_OPT_TILE_WIDTH:
      if (value != 4 && value != 8 && value != 16 && value != 32)
        return C.fail(VFR_ERR_INVALID, "tile width is 4, 8, 16 or 32");
      C.tune.tile_w = (uint32_t)value;
      return VFR_OK;
    case VFR_OPT_RASTER_WARPS:
      if (value < 1 || value > 64) return C.fail(VFR_ERR_INVALID, "raster warps per SM is 1..64");
      C.tune.raster_warps_per_sm = (uint32_t)value;
      return VFR_OK;
    default: return C.fail(VFR_ERR_INVALID, "unknown option");
  }
}

int vfr_profile_read(vfr_ctx* c, float* ms3, int cap, int* count) {
  CTX_OR_FAIL(c);
  if (!count || (cap > 0 && !ms3)) return C.fail(VFR_ERR_INVALID, "bad profile buffer");
  int n = 0;
  for (auto& s : C.prof_live) {
    int rc = C.cuda(cudaEventSynchronize(s.e[3]), "profile event");
    if (rc) return rc;
    if (n < cap) {
      for (int k = 0; k < 3; ++k) cudaEventElapsedTime(&ms3[3 * n + k], s.e[k], s.e[k + 1]);
      ++n;
    }
    C.prof_pool.push_back(s);
  }
  C.prof_live.clear();
  *count = n;
  return VFR_OK;
}

int vfr_tables_upload(vfr_ctx* c, const float* tf, const float* psi) {
  vfr::Range nvtx("vfr_tables_upload");
  CTX_OR_FAIL(c);
  if (!tf) return C.fail(VFR_ERR_INVALID, "transfer function is NULL");
  std::vector<float> ref;
  if (!psi) {  // the reference's own table, the drop-in default
    ref.resize(512 * 512);
    if (vfr_psi_table_reference(ref.data()) != VFR_OK)
      return C.fail(VFR_ERR_IO,
                    "the reference psi table (data/psiGammaTable512.bin beside the library, or "
                    "$VFRAY_PSI_TABLE) is missing; pass vfr_psi_table's generated table instead");
    psi = ref.data();
  }
  // the transfer function (256 float4) is followed by the 64 doubles
  // 2^(j/64) of the traversal's table-driven exponential
  if (!C.d_tf) {
    int rc = C.cuda(cudaMalloc(&C.d_tf, sizeof(float4) * 256 + sizeof(double) * 64), "tf alloc");
    if (!rc) rc = C.cuda(cudaMalloc(&C.d_psi, sizeof(float) * 512 * 512), "psi alloc");
    if (rc) return rc;
  }
  sync_context(C);
  double e2[64];
  for (int j = 0; j < 64; ++j) e2[j] = (double)std::exp2l((long double)j / 64.0L);
  int rc = C.cuda(cudaMemcpy(C.d_tf, tf, sizeof(float) * 1024, cudaMemcpyHostToDevice), "tf upload");
  if (!rc)
    rc = C.cuda(cudaMemcpy(C.d_tf + 256, e2, sizeof(e2), cudaMemcpyHostToDevice), "exp2 upload");
  if (!rc)
    rc = C.cuda(cudaMemcpy(C.d_psi, psi, sizeof(float) * 512 * 512, cudaMemcpyHostToDevice),
                "psi upload");
  return rc;
}

int vfr_mesh_upload(vfr_ctx* c, const float* vert4, uint32_t nV, const uint32_t* tet4,
                    const uint32_t* con4, uint32_t nT, const uint32_t* extf2, uint32_t nExt,
                    float maxEdge, float maxZ, float minZ, int* mesh_id) {
  vfr::Range nvtx("vfr_mesh_upload");
  CTX_OR_FAIL(c);
  if (!vert4 || !tet4 || !con4 || (!extf2 && nExt) || !mesh_id || nV == 0 || nT == 0)
    return C.fail(VFR_ERR_INVALID, "mesh arrays missing or empty");
  if ((uint64_t)nExt > 4ull * nT) return C.fail(VFR_ERR_INVALID, "more external faces than faces");
  // the traversal packs a walk state (tet, entry face) into 32 bits
  if (nT >= (1u << 30)) return C.fail(VFR_ERR_INVALID, "2^30 tets or more");
  // the traversal divides depth steps (at least 1e-12) by it through a
  // reciprocal, exact while no quotient falls below 2^-126
  if (!(maxEdge < 0x1p80f)) return C.fail(VFR_ERR_INVALID, "maxEdgeLength not below 2^80");
  std::string why;
  if (!vfr::validate_mesh(tet4, con4, nV, nT, extf2, nExt, why)) return C.fail(VFR_ERR_MESH, why);
  std::vector<uint32_t> walk(8 * (size_t)nT);
  if (!vfr::build_walk(tet4, con4, nV, nT, walk.data(), why)) return C.fail(VFR_ERR_MESH, why);
  std::unique_ptr<Mesh> m(new Mesh);
  m->nV = nV;
  m->nT = nT;
  m->nExt = nExt;
  m->maxEdge = maxEdge;
  m->maxZ = maxZ;
  m->minZ = minZ;
  int rc = C.cuda(cudaMalloc(&m->tet, sizeof(uint4) * (size_t)nT), "tets");
  if (!rc) rc = C.cuda(cudaMalloc(&m->walk, sizeof(vfr::WalkRec) * (size_t)nT), "walk records");
  if (!rc) rc = C.cuda(cudaMalloc(&m->vert, sizeof(float4) * (size_t)nV), "vertices");
  if (!rc) rc = C.cuda(cudaMalloc(&m->extf, sizeof(uint2) * std::max<size_t>(nExt, 1)), "ext faces");
  if (!rc)
    rc = C.cuda(cudaMemcpy(m->tet, tet4, sizeof(uint4) * (size_t)nT, cudaMemcpyHostToDevice),
                "tet upload");
  if (!rc)
    rc = C.cuda(cudaMemcpy(m->walk, walk.data(), sizeof(vfr::WalkRec) * (size_t)nT,
                           cudaMemcpyHostToDevice),
                "walk upload");
  if (!rc)
    rc = C.cuda(cudaMemcpy(m->vert, vert4, sizeof(float4) * (size_t)nV, cudaMemcpyHostToDevice),
                "vertex upload");
  if (!rc && nExt)
    rc = C.cuda(cudaMemcpy(m->extf, extf2, sizeof(uint2) * (size_t)nExt, cudaMemcpyHostToDevice),
                "ext-face upload");
  if (rc) return rc;
  m->bytes = (sizeof(uint4) + sizeof(vfr::WalkRec)) * (size_t)nT + sizeof(float4) * (size_t)nV +
             sizeof(uint2) * (size_t)nExt;
  for (size_t i = 0; i < C.meshes.size(); ++i)
    if (!C.meshes[i]) {
      C.meshes[i] = std::move(m);
      *mesh_id = (int)i;
      return VFR_OK;
    }
  C.meshes.push_back(std::move(m));
  *mesh_id = (int)C.meshes.size() - 1;
  return VFR_OK;
}

int vfr_mesh_release(vfr_ctx* c, int id) {
  CTX_OR_FAIL(c);
  if (!C.mesh(id)) return C.fail(VFR_ERR_STATE, "unknown mesh id");
  sync_context(C);
  if (C.plain.njobs && C.plain.specs[0].mesh == id) {
    C.plain.njobs = 0;
    C.stage = 0;
  }
  C.meshes[id].reset();
  return VFR_OK;
}

int vfr_mesh_bytes(vfr_ctx* c, int id, uint64_t* bytes) {
  CTX_OR_FAIL(c);
  Mesh* m = C.mesh(id);
  if (!m || !bytes) return C.fail(VFR_ERR_STATE, "unknown mesh id");
  *bytes = m->bytes;
  return VFR_OK;
}

int vfr_find_visible(vfr_ctx* c, int id, uint32_t* num_vis, uint32_t* visExt, float* faceData) {
  vfr::Range nvtx("vfr_find_visible");
  CTX_OR_FAIL(c);
  Mesh* m = C.mesh(id);
  if (!m) return C.fail(VFR_ERR_STATE, "unknown mesh id");
  C.stage = 0;
  int rc = single(C, id, nullptr, 2, 2, VFR_MODE_REF, true, nullptr, nullptr, nullptr);
  if (!rc) rc = C.plain.enqueue_a();
  std::vector<vfr::ViewCounters> k;
  if (!rc) rc = C.plain.counters(k);
  if (rc) return rc;
  if (num_vis) *num_vis = k[0].nvis;
  const vfr::JobDev& J = C.plain.jobs[0];
  if (visExt && k[0].nvis)
    rc = C.cuda(cudaMemcpy(visExt, J.vis_ext, sizeof(uint32_t) * k[0].nvis, cudaMemcpyDeviceToHost),
                "visible list read");
  if (!rc && faceData && m->nExt) {
    std::vector<float4> pl(vfr::kPlaneStride * (size_t)m->nExt);
    rc = C.cuda(cudaMemcpy(pl.data(), J.planes, sizeof(float4) * pl.size(), cudaMemcpyDeviceToHost),
                "plane read");
    for (size_t e = 0; e < m->nExt && !rc; ++e) {
      const float4 a = pl[vfr::kPlaneStride * e], b = pl[vfr::kPlaneStride * e + 1];
      float* o = faceData + 6 * e;
      o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = b.x; o[5] = b.y;
    }
  }
  if (!rc) C.stage = 1;
  return rc;
}

int vfr_project(vfr_ctx* c, int id, uint32_t W, uint32_t H, uint32_t* bbox, int32_t* writer) {
  vfr::Range nvtx("vfr_project");
  CTX_OR_FAIL(c);
  Mesh* m = C.mesh(id);
  if (!m || C.stage < 1 || !C.plain.njobs || C.plain.specs[0].mesh != id)
    return C.fail(VFR_ERR_STATE, "vfr_project needs vfr_find_visible of the same mesh first");
  if (W < 2 || H < 2 || (uint64_t)W * H > (1ull << 28))
    return C.fail(VFR_ERR_INVALID, "image size out of range");
  // the planes and visible list of stage (a) stay where they are: same mesh,
  // so the same arena offsets; only the pixel arenas grow
  int rc = single(C, id, nullptr, W, H, VFR_MODE_REF, true, nullptr, nullptr, nullptr);
  if (!rc) rc = C.plain.enqueue_b();
  std::vector<vfr::ViewCounters> k;
  if (!rc) rc = C.plain.counters(k);
  if (rc) return rc;
  const vfr::JobDev& J = C.plain.jobs[0];
  if (bbox && k[0].nvis)
    rc = C.cuda(cudaMemcpy(bbox, J.bbox, sizeof(uint4) * k[0].nvis, cudaMemcpyDeviceToHost),
                "bbox read");
  if (!rc && writer)
    rc = C.cuda(cudaMemcpy(writer, J.winner, sizeof(int32_t) * (size_t)W * H, cudaMemcpyDeviceToHost),
                "winner read");
  if (!rc) C.stage = 2;
  return rc;
}

int vfr_traverse(vfr_ctx* c, int id, uint8_t* rgb8, float* rgba, uint32_t* steps,
                 vfr_render_stats* stats) {
  vfr::Range nvtx("vfr_traverse");
  CTX_OR_FAIL(c);
  Mesh* m = C.mesh(id);
  if (!m || C.stage < 2 || !C.plain.njobs || C.plain.specs[0].mesh != id)
    return C.fail(VFR_ERR_STATE, "vfr_traverse needs vfr_project of the same mesh first");
  if (!C.d_tf) return C.fail(VFR_ERR_STATE, "tables not uploaded");
  const size_t np = (size_t)C.plain.specs[0].W * C.plain.specs[0].H;
  cudaEventRecord(C.ev[0], C.stream);
  int rc = C.plain.enqueue_c();
  cudaEventRecord(C.ev[1], C.stream);
  std::vector<vfr::ViewCounters> k;
  if (!rc) rc = C.plain.counters(k);
  if (!rc) rc = copy_out(C, rgb8, rgba, steps, np);
  if (rc) return rc;
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    fill_stats(k[0], m->nExt, stats);
    cudaEventElapsedTime(&stats->ms_traverse, C.ev[0], C.ev[1]);
    stats->ms_total = stats->ms_traverse;
  }
  C.stage = 1;  // the ray queue is consumed; project again before another traverse
  return C.check_status(k[0].status, 0);
}

static int render_one(Ctx& C, int id, const float* mv16, uint32_t W, uint32_t H, int mode, bool own,
                      uint8_t* rgb8, float4* rgba, uint32_t* steps, bool timed) {
  if (!C.mesh(id)) return C.fail(VFR_ERR_STATE, "unknown mesh id");
  if (!C.d_tf) return C.fail(VFR_ERR_STATE, "tables not uploaded");
  if (mode != VFR_MODE_REF && mode != VFR_MODE_COMPOSITED)
    return C.fail(VFR_ERR_INVALID, "unknown mode");
  C.stage = 0;
  int rc = single(C, id, mv16, W, H, mode, own, rgb8, rgba, steps);
  if (rc) return rc;
  if (timed) cudaEventRecord(C.ev[0], C.stream);
  C.prof_mark(0);
  rc = C.plain.enqueue_a();
  if (timed) cudaEventRecord(C.ev[1], C.stream);
  C.prof_mark(1);
  if (!rc) rc = C.plain.enqueue_b();
  if (timed) cudaEventRecord(C.ev[2], C.stream);
  C.prof_mark(2);
  if (!rc) rc = C.plain.enqueue_c();
  if (timed) cudaEventRecord(C.ev[3], C.stream);
  C.prof_mark(3);
  return rc;
}

int vfr_render(vfr_ctx* c, int id, const float* mv16, uint32_t W, uint32_t H, int mode,
               uint8_t* rgb8, float* rgba, uint32_t* steps, vfr_render_stats* stats) {
  vfr::Range nvtx("vfr_render");
  CTX_OR_FAIL(c);
  for (int attempt = 0; attempt < 4; ++attempt) {
    int rc = render_one(C, id, mv16, W, H, mode, true, nullptr, nullptr, nullptr, true);
    std::vector<vfr::ViewCounters> k;
    if (!rc) rc = C.plain.counters(k);
    if (rc) return rc;
    if (C.plain.overflowed(k)) {
      // entry lists or tile bins overflowed: grow to the need and render again
      C.plain.ent_cap = 0;
      C.plain.bin_cap = 0;
      continue;
    }
    rc = copy_out(C, rgb8, rgba, steps, (size_t)W * H);
    if (rc) return rc;
    if (stats) {
      std::memset(stats, 0, sizeof *stats);
      fill_stats(k[0], C.mesh(id)->nExt, stats);
      cudaEventElapsedTime(&stats->ms_visible, C.ev[0], C.ev[1]);
      cudaEventElapsedTime(&stats->ms_project, C.ev[1], C.ev[2]);
      cudaEventElapsedTime(&stats->ms_traverse, C.ev[2], C.ev[3]);
      cudaEventElapsedTime(&stats->ms_total, C.ev[0], C.ev[3]);
    }
    return C.check_status(k[0].status, 0);
  }
  return C.fail(VFR_ERR_DEVICE, "entry lists or tile bins kept overflowing");
}

int vfr_render_device(vfr_ctx* c, int id, const float* mv16, uint32_t W, uint32_t H, int mode,
                      uint8_t* rgb8_dev, float* rgba_dev, uint32_t* steps_dev, int32_t* writer_dev) {
  vfr::Range nvtx("vfr_render_device");
  CTX_OR_FAIL(c);
  int rc = render_one(C, id, mv16, W, H, mode, false, rgb8_dev, (float4*)rgba_dev, steps_dev, false);
  if (!rc && writer_dev && mode == VFR_MODE_REF)
    rc = C.cuda(cudaMemcpyAsync(writer_dev, C.plain.jobs[0].winner, sizeof(int32_t) * (size_t)W * H,
                                cudaMemcpyDeviceToDevice, C.stream),
                "winner copy");
  return rc;
}

int vfr_device_status(vfr_ctx* c, uint32_t* status) {
  CTX_OR_FAIL(c);
  if (!C.plain.njobs) {
    if (status) *status = 0;
    return VFR_OK;
  }
  std::vector<vfr::ViewCounters> k;
  int rc = C.plain.counters(k);
  if (rc) return rc;
  if (status) *status = k[0].status;
  const uint32_t over = C.plain.overflowed(k);
  if (over) {
    C.plain.ent_cap = 0;
    C.plain.bin_cap = 0;
  }
  return C.check_status(k[0].status, over);
}

// ---- batches ----

int vfr_batch_create(vfr_ctx* c, vfr_batch** out) {
  CTX_OR_FAIL(c);
  if (!out) return C.fail(VFR_ERR_INVALID, "null batch pointer");
  vfr_batch* b = new vfr_batch;
  b->owner = c;
  b->b.ctx = &C;
  C.batches.push_back(b);
  *out = b;
  return VFR_OK;
}

void vfr_batch_destroy(vfr_batch* b) {
  if (!b) return;
  if (b->owner) {
    Ctx& C = b->owner->impl;
    cudaSetDevice(C.device);
    cudaStreamSynchronize(C.stream);
    cudaStreamSynchronize(b->b.st());
    C.batches.erase(std::remove(C.batches.begin(), C.batches.end(), (void*)b), C.batches.end());
  }
  delete b;
}

int vfr_batch_set_jobs(vfr_batch* b, const vfr_job* jobs, uint32_t n, int mode) {
  vfr::Range nvtx("vfr_batch_set_jobs");
  if (!b) return VFR_ERR_INVALID;
  if (!b->owner) return VFR_ERR_STATE;
  Ctx& C = b->owner->impl;
  cudaSetDevice(C.device);
  if (!jobs || n == 0) return C.fail(VFR_ERR_INVALID, "empty job list");
  if (mode != VFR_MODE_REF && mode != VFR_MODE_COMPOSITED)
    return C.fail(VFR_ERR_INVALID, "unknown mode");
  std::vector<JobSpec> s(n);
  bool own = false;
  for (uint32_t j = 0; j < n; ++j) {
    s[j].mesh = jobs[j].mesh_id;
    s[j].W = jobs[j].W;
    s[j].H = jobs[j].H;
    s[j].use_mv = jobs[j].use_mv != 0;
    std::memcpy(s[j].mv, jobs[j].mv, sizeof s[j].mv);
    s[j].rgb8 = jobs[j].rgb8_dev;
    s[j].rgba = (float4*)jobs[j].rgba_dev;
    s[j].steps = jobs[j].steps_dev;
    own = own || (!jobs[j].rgb8_dev && !jobs[j].rgba_dev && !jobs[j].steps_dev);
  }
  cudaStreamSynchronize(C.stream);
  cudaStreamSynchronize(b->b.st());  // its own stream's runs read the arenas the layout may grow
  int rc = b->b.layout(s, mode, own);
  if (!rc) rc = b->b.upload(false);
  return rc;
}

int vfr_batch_capture(vfr_batch* b) {
  vfr::Range nvtx("vfr_batch_capture");
  if (!b || !b->b.njobs) return VFR_ERR_STATE;
  if (!b->owner) return VFR_ERR_STATE;
  Ctx& C = b->owner->impl;
  cudaSetDevice(C.device);
  if (!C.d_tf) return C.fail(VFR_ERR_STATE, "tables not uploaded");
  return b->b.capture();
}

int vfr_batch_run(vfr_batch* b) {
  vfr::Range nvtx("vfr_batch_run");
  if (!b || !b->b.njobs) return VFR_ERR_STATE;
  if (!b->owner) return VFR_ERR_STATE;
  Ctx& C = b->owner->impl;
  cudaSetDevice(C.device);
  if (!C.d_tf) return C.fail(VFR_ERR_STATE, "tables not uploaded");
  if (C.profile && !b->b.exec) {  // per-stage events need the direct launches
    C.prof_mark(0, b->b.st());
    int rc = b->b.enqueue_a();
    C.prof_mark(1, b->b.st());
    if (!rc) rc = b->b.enqueue_b();
    C.prof_mark(2, b->b.st());
    if (!rc) rc = b->b.enqueue_c();
    C.prof_mark(3, b->b.st());
    return rc;
  }
  C.prof_mark(0, b->b.st());
  C.prof_mark(1, b->b.st());
  C.prof_mark(2, b->b.st());
  int rc = b->b.run();
  C.prof_mark(3, b->b.st());
  return rc;
}

int vfr_batch_stats(vfr_batch* b, vfr_render_stats* per_job, uint32_t n) {
  if (!b || !b->b.njobs) return VFR_ERR_STATE;
  if (!b->owner) return VFR_ERR_STATE;
  Ctx& C = b->owner->impl;
  cudaSetDevice(C.device);
  std::vector<vfr::ViewCounters> k;
  int rc = b->b.counters(k);
  if (rc) return rc;
  uint32_t status = 0, over = 0;
  for (uint32_t j = 0; j < b->b.njobs; ++j) {
    status |= k[j].status;
    if (j < n && per_job) {
      std::memset(&per_job[j], 0, sizeof per_job[j]);
      fill_stats(k[j], b->b.jobs[j].nExt, &per_job[j]);
    }
  }
  over = b->b.overflowed(k);
  return C.check_status(status, over);
}

int vfr_batch_output(vfr_batch* b, uint32_t job, uint8_t** rgb8_dev, float** rgba_dev,
                     uint32_t** steps_dev) {
  if (!b || job >= b->b.njobs) return VFR_ERR_STATE;
  if (rgb8_dev) *rgb8_dev = b->b.specs[job].rgb8;
  if (rgba_dev) *rgba_dev = (float*)b->b.specs[job].rgba;
  if (steps_dev) *steps_dev = b->b.specs[job].steps;
  return VFR_OK;
}

// Autotuner: times stages (b) and (c) of the batch (direct launches, events
// on the context stream, best of `reps`) over a grid of the knobs --
// traversal register budget, refill threshold, traversal CTAs per SM, ray
// tile shape, stage (b) warps per SM -- and keeps the fastest on the context.
int vfr_batch_autotune(vfr_batch* b, int reps, vfr_tuning* out) {
  vfr::Range nvtx("vfr_batch_autotune");
  if (!b || !b->b.njobs) return VFR_ERR_STATE;
  if (!b->owner) return VFR_ERR_STATE;
  Ctx& C = b->owner->impl;
  cudaSetDevice(C.device);
  if (!C.d_tf) return C.fail(VFR_ERR_STATE, "tables not uploaded");
  if (reps < 1) reps = 1;
  const vfr::Tuning saved = C.tune;
  const std::vector<JobSpec> specs = b->b.specs;
  const int mode = b->b.mode;
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&e2);
  int occ_max = 0;
  vfr::Tuning best = saved;
  float best_ms = 1e30f;
  int rc = VFR_OK;
  const uint32_t variants[] = {0, 1}, refills[] = {4, 6}, tiles[] = {4, 8, 16},
                 rasters[] = {16, 64};
  for (uint32_t var : variants)
    for (uint32_t rf : refills)
      for (uint32_t tw : tiles)
        for (uint32_t rw : rasters)
          for (int bsm = 0; bsm < 2 && !rc; ++bsm) {
            vfr::Tuning t = saved;
            t.variant = var;
            t.refill = rf;
            t.tile_w = tw;
            t.raster_warps_per_sm = rw;
            t.blocks_per_sm = 0;
            C.tune = t;
            if (bsm) {
              occ_max = C.traverse_blocks_per_sm(mode);
              if (occ_max < 2) continue;
              C.tune.blocks_per_sm = occ_max - 1;
            }
            rc = b->b.layout(specs, mode, false);
            if (!rc) rc = b->b.upload(false);
            float ms = 1e30f;
            for (int r = 0; r < reps + 1 && !rc; ++r) {
              rc = b->b.enqueue_a();
              cudaEventRecord(e0, b->b.st());
              if (!rc) rc = b->b.enqueue_b();
              cudaEventRecord(e1, b->b.st());
              if (!rc) rc = b->b.enqueue_c();
              cudaEventRecord(e2, b->b.st());
              if (!rc) rc = C.cuda(cudaEventSynchronize(e2), "autotune");
              float m = 0;
              cudaEventElapsedTime(&m, e0, e2);
              if (r > 0) ms = std::min(ms, m);  // the first run warms up
            }
            if (!rc && ms < best_ms) {
              best_ms = ms;
              best = C.tune;
            }
          }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  C.tune = rc ? saved : best;
  int rc2 = b->b.layout(specs, mode, false);
  if (!rc2) rc2 = b->b.upload(false);
  b->b.drop_graph();
  if (rc) return rc;
  if (out) {
    out->variant = best.variant;
    out->refill = best.refill;
    out->blocks_per_sm = best.blocks_per_sm;
    out->tile_w = best.tile_w;
    out->raster_warps_per_sm = best.raster_warps_per_sm;
    out->ms = best_ms;
  }
  return rc2;
}

int vfr_batch_set_cameras(vfr_batch* b, const float* mv16, uint32_t n) {
  vfr::Range nvtx("vfr_batch_set_cameras");
  if (!b || !b->b.njobs) return VFR_ERR_STATE;
  if (!b->owner) return VFR_ERR_STATE;
  Ctx& C = b->owner->impl;
  cudaSetDevice(C.device);
  Batch& B = b->b;
  if (!mv16 || n != B.njobs) return C.fail(VFR_ERR_INVALID, "one camera per job");
  // the host copies follow, so a later layout of the same jobs keeps them
  for (uint32_t j = 0; j < n; ++j) {
    const float* m = mv16 + 16 * (size_t)j;
    std::memcpy(B.specs[j].mv, m, sizeof B.specs[j].mv);
    B.jobs[j].m0 = make_float4(m[0], m[1], m[2], m[3]);
    B.jobs[j].m1 = make_float4(m[4], m[5], m[6], m[7]);
    B.jobs[j].m2 = make_float4(m[8], m[9], m[10], m[11]);
  }
  // rows 0..2 of each matrix are the job table entry's first 48 bytes
  static_assert(offsetof(vfr::JobDev, m0) == 0 && offsetof(vfr::JobDev, m2) == 32,
                "job table camera layout");
  return C.cuda(cudaMemcpy2DAsync(B.d_jobs.p, sizeof(vfr::JobDev), mv16, 16 * sizeof(float),
                                  3 * sizeof(float4), n, cudaMemcpyHostToDevice, B.st()),
                "camera upload");
}

// The batch's outputs into host buffers: enqueued on the batch's stream,
// then (wait) a synchronisation of that stream.
static int batch_read(vfr_batch* b, uint8_t* rgb8_host, float* rgba_host, uint32_t* steps_host,
               bool wait) {
  if (!b || !b->b.njobs) return VFR_ERR_STATE;
  if (!b->owner) return VFR_ERR_STATE;
  Ctx& C = b->owner->impl;
  cudaSetDevice(C.device);
  const std::vector<JobSpec>& sp = b->b.specs;
  const uint32_t nj = b->b.njobs;
  // one copy per run of jobs whose outputs of this kind lie back to back on
  // the device (all of them when the batch owns its outputs)
  auto read = [&](char* host, size_t bpp, auto dev_of, const char* what) -> int {
    if (!host) return VFR_OK;
    size_t off = 0;
    for (uint32_t j = 0; j < nj;) {
      const char* d0 = (const char*)dev_of(sp[j]);
      size_t bytes = 0, h0 = off;
      uint32_t k = j;
      for (; k < nj; ++k) {
        const char* d = (const char*)dev_of(sp[k]);
        const size_t nb = bpp * sp[k].W * sp[k].H;
        if (!d0 || d != d0 + bytes) break;
        bytes += nb;
      }
      if (k == j) {  // no device output of this kind for job j: skipped
        off += bpp * sp[j].W * sp[j].H;
        ++j;
        continue;
      }
      int rc = C.cuda(cudaMemcpyAsync(host + h0, d0, bytes, cudaMemcpyDeviceToHost, b->b.st()), what);
      if (rc) return rc;
      off += bytes;
      j = k;
    }
    return VFR_OK;
  };
  int rc = read((char*)rgb8_host, 3, [](const JobSpec& q) { return (const void*)q.rgb8; }, "rgb8 read");
  if (!rc)
    rc = read((char*)rgba_host, sizeof(float4), [](const JobSpec& q) { return (const void*)q.rgba; },
              "rgba read");
  if (!rc)
    rc = read((char*)steps_host, sizeof(uint32_t),
              [](const JobSpec& q) { return (const void*)q.steps; }, "steps read");
  if (!rc && wait) rc = C.cuda(cudaStreamSynchronize(b->b.st()), "batch read");
  return rc;
}

int vfr_batch_read(vfr_batch* b, uint8_t* rgb8_host, float* rgba_host, uint32_t* steps_host) {
  vfr::Range nvtx("vfr_batch_read");
  return batch_read(b, rgb8_host, rgba_host, steps_host, true);
}

int vfr_batch_read_async(vfr_batch* b, uint8_t* rgb8_host, float* rgba_host,
                         uint32_t* steps_host) {
  vfr::Range nvtx("vfr_batch_read_async");
  return batch_read(b, rgb8_host, rgba_host, steps_host, false);
}

int vfr_batch_synchronize(vfr_batch* b) {
  if (!b || !b->owner) return VFR_ERR_STATE;
  Ctx& C = b->owner->impl;
  cudaSetDevice(C.device);
  return C.cuda(cudaStreamSynchronize(b->b.st()), "batch synchronize");
}

int vfr_batch_set_stream(vfr_batch* b, void* stream) {
  if (!b || !b->owner) return VFR_ERR_STATE;
  Ctx& C = b->owner->impl;
  cudaSetDevice(C.device);
  // work already enqueued on the old stream is not ordered with the new one
  if (int rc = C.cuda(cudaStreamSynchronize(b->b.st()), "batch stream switch")) return rc;
  b->b.stream = static_cast<cudaStream_t>(stream);
  return VFR_OK;
}

int vfr_batch_scratch_bytes(vfr_batch* b, uint64_t* bytes) {
  if (!b || !bytes) return VFR_ERR_INVALID;
  *bytes = b->b.scratch_bytes;
  return VFR_OK;
}

#ifdef VFR_CHECKED
// Test hook of the checked build only (declared in no header: the product
// library does not have it).  Overwrites one id of a resident mesh on the
// device, past the validation at upload, so that a test can show the range
// checks turning it into VFR_DEV_RANGE.  what: 0 = a neighbour id of a walk
// record (index = 4 tet + face), 1 = a vertex id of the tet array (index =
// 4 tet + corner), 2 = the tet id of an external face (index = the face).
__attribute__((visibility("default"))) int vfr_checked_set_id(vfr_ctx* c, int id, int what,
                                                              uint64_t index, uint32_t value) {
  CTX_OR_FAIL(c);
  Mesh* m = C.mesh(id);
  if (!m) return C.fail(VFR_ERR_STATE, "unknown mesh id");
  uint32_t* dst = nullptr;
  if (what == 0 && index < 4ull * m->nT)
    dst = reinterpret_cast<uint32_t*>(m->walk + index / 4) + index % 4;
  else if (what == 1 && index < 4ull * m->nT)
    dst = reinterpret_cast<uint32_t*>(m->tet) + index;
  else if (what == 2 && index < m->nExt)
    dst = reinterpret_cast<uint32_t*>(m->extf + index);
  if (!dst) return C.fail(VFR_ERR_INVALID, "checked_set_id: no such id");
  if (int rc = C.cuda(cudaDeviceSynchronize(), "checked_set_id")) return rc;
  return C.cuda(cudaMemcpy(dst, &value, sizeof value, cudaMemcpyHostToDevice), "checked_set_id");
}
#endif

}  // extern "C"
