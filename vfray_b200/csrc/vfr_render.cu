// The C ABI of the VF-Ray render path (include/vfray.h): context, resident
// meshes and tables, and the three stages of a view as stream-ordered launches.
//
// Replaces the host driver of the reference (vfRay.cu:165-594): there the
// stages communicate through globals, texture bindings and a host round trip
// for the visible-face compaction; here a view is a chain of kernels on one
// stream whose intermediate counts stay on the device, so a whole view can be
// enqueued without a host synchronisation (and captured in a CUDA graph).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "vfray.h"
#include "vfr_kernels.cuh"
#include "vfr_internal.h"

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
  if (b.cap >= bytes && b.p) return VFR_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t want = bytes + bytes / 8 + 256;
  int rc = cuda(cudaMalloc(&b.p, want), what);
  if (rc) return rc;
  b.cap = want;
  return VFR_OK;
}

Mesh* Ctx::mesh(int id) {
  if (id < 0 || id >= (int)meshes.size() || !meshes[id]) return nullptr;
  return meshes[id].get();
}

__global__ void init_counters_kernel(ViewCounters* c, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ViewCounters v;
  v.nvis = 0; v.nrays = 0; v.queue = 0; v.status = 0; v.steps = 0; v.nentries = 0;
  v.maxedge_bits = 0;
  for (int k = 0; k < 4; ++k) { v.mm[k] = 0xffffffffu; v.mm[4 + k] = 0u; }
  c[i] = v;
}

// Enqueue stage (a) (and the view set-up when mv16 is given).
int Ctx::enqueue_visible(Mesh& m, const float* mv16, View& v) {
  v.mesh = &m;
  v.vert = m.vert;
  v.use_view_maxedge = 0;
  v.maxEdge = m.maxEdge;
  init_counters_kernel<<<1, 32, 0, stream>>>(v.ctr, 1);
  if (mv16) {
    int rc = grow(v.vview, sizeof(float4) * (size_t)m.nV, "view vertices");
    if (rc) return rc;
    float4* vv = (float4*)v.vview.p;
    const int blocks = std::max(1, std::min(num_sms * 4, (int)((m.nV + 255) / 256)));
    view_rotate_kernel<<<blocks, 256, 0, stream>>>(
        m.vert, m.nV, make_float4(mv16[0], mv16[1], mv16[2], mv16[3]),
        make_float4(mv16[4], mv16[5], mv16[6], mv16[7]),
        make_float4(mv16[8], mv16[9], mv16[10], mv16[11]), vv, v.ctr);
    view_normalize_kernel<<<blocks, 256, 0, stream>>>(vv, m.nV, v.ctr);
    const int tb = std::max(1, std::min(num_sms * 4, (int)((m.nT + 255) / 256)));
    view_maxedge_kernel<<<tb, 256, 0, stream>>>(m.tet, vv, m.nT, v.ctr);
    v.vert = vv;
    v.use_view_maxedge = 1;
  }
  const uint32_t nblk = std::max<uint32_t>(1, (m.nExt + 1023) / 1024);
  int rc = grow(v.planes, sizeof(float4) * 2 * (size_t)std::max<uint32_t>(m.nExt, 1), "planes");
  if (!rc) rc = grow(v.blk, sizeof(uint32_t) * nblk, "block counts");
  if (!rc) rc = grow(v.vis_ext, sizeof(uint32_t) * std::max<uint32_t>(m.nExt, 1), "visible list");
  if (rc) return rc;
  if (m.nExt) {
    visible_kernel<<<nblk, 1024, 0, stream>>>(v.vert, m.tet, m.extf, m.nExt, (float4*)v.planes.p,
                                             (uint32_t*)v.blk.p);
    compact_kernel<<<nblk, 1024, 0, stream>>>((const float4*)v.planes.p, m.nExt,
                                             (const uint32_t*)v.blk.p, (uint32_t*)v.vis_ext.p,
                                             v.ctr);
  }
  return cuda(cudaGetLastError(), "stage (a) launch");
}

// Enqueue stage (b): coverage (winner or entry lists) + ray list.
int Ctx::enqueue_project(View& v, uint32_t W, uint32_t H, int mode) {
  Mesh& m = *v.mesh;
  v.W = W; v.H = H; v.mode = mode;
  const size_t np = (size_t)W * H;
  int rc = grow(v.bbox, sizeof(uint4) * std::max<uint32_t>(m.nExt, 1), "bbox");
  if (!rc) rc = grow(v.rays, sizeof(uint32_t) * np, "ray list");
  if (rc) return rc;
  const uint32_t warps = std::max<uint32_t>(8, std::min<uint32_t>(m.nExt, (uint32_t)num_sms * 64));
  const uint32_t rb = (warps + 7) / 8;
  const float4* planes = (const float4*)v.planes.p;
  const uint32_t* vis = (const uint32_t*)v.vis_ext.p;
  if (mode == VFR_MODE_REF) {
    rc = grow(v.winner, sizeof(int32_t) * np, "winner map");
    if (rc) return rc;
    cudaMemsetAsync(v.winner.p, 0xff, sizeof(int32_t) * np, stream);
    if (m.nExt)
      raster_kernel<false, false><<<rb, 256, 0, stream>>>(
          v.vert, m.tet, m.extf, planes, vis, v.ctr, W, H, (uint4*)v.bbox.p,
          (int32_t*)v.winner.p, nullptr, nullptr, nullptr, nullptr, 0);
  } else {
    const uint32_t nsb = (uint32_t)((np + 1 + 1023) / 1024);
    rc = grow(v.ent_cnt, sizeof(uint32_t) * (np + 1), "entry counts");
    if (!rc) rc = grow(v.ent_off, sizeof(uint32_t) * (np + 1), "entry offsets");
    if (!rc) rc = grow(v.ent_cur, sizeof(uint32_t) * np, "entry cursors");
    if (!rc) rc = grow(v.scan, sizeof(uint32_t) * nsb, "scan sums");
    if (!rc) rc = grow(v.ent, sizeof(uint2) * std::max<size_t>(v.ent_cap, 1), "entries");
    if (rc) return rc;
    cudaMemsetAsync(v.ent_cnt.p, 0, sizeof(uint32_t) * (np + 1), stream);
    cudaMemsetAsync(v.ent_cur.p, 0, sizeof(uint32_t) * np, stream);
    if (m.nExt)
      raster_kernel<true, false><<<rb, 256, 0, stream>>>(
          v.vert, m.tet, m.extf, planes, vis, v.ctr, W, H, (uint4*)v.bbox.p, nullptr,
          (uint32_t*)v.ent_cnt.p, nullptr, nullptr, nullptr, 0);
    scan_blocks_kernel<<<nsb, 1024, 0, stream>>>((const uint32_t*)v.ent_cnt.p, (uint32_t)(np + 1),
                                                 (uint32_t*)v.ent_off.p, (uint32_t*)v.scan.p);
    scan_add_kernel<<<nsb, 1024, 0, stream>>>((uint32_t*)v.ent_off.p, (uint32_t)(np + 1),
                                              (const uint32_t*)v.scan.p, &v.ctr->nentries);
    if (m.nExt)
      raster_kernel<false, true><<<rb, 256, 0, stream>>>(
          v.vert, m.tet, m.extf, planes, vis, v.ctr, W, H, nullptr, nullptr, nullptr,
          (const uint32_t*)v.ent_off.p, (uint32_t*)v.ent_cur.p, (uint2*)v.ent.p,
          (uint32_t)std::min<size_t>(v.ent_cap, 0xffffffffu));
  }
  const uint32_t tiles = ((W + 7) / 8) * ((H + 3) / 4);
  raylist_kernel<<<(tiles + 7) / 8, 256, 0, stream>>>(
      mode == VFR_MODE_REF ? (const int32_t*)v.winner.p : nullptr,
      mode == VFR_MODE_REF ? nullptr : (const uint32_t*)v.ent_cnt.p, W, H, (uint32_t*)v.rays.p,
      v.ctr);
  return cuda(cudaGetLastError(), "stage (b) launch");
}

// Enqueue stage (c) into the given output buffers (device pointers).
int Ctx::enqueue_traverse(View& v, uint8_t* rgb8, float4* rgba, uint32_t* steps) {
  Mesh& m = *v.mesh;
  const size_t np = (size_t)v.W * v.H;
  if (rgb8) cudaMemsetAsync(rgb8, 0, np * 3, stream);
  if (rgba) cudaMemsetAsync(rgba, 0, np * sizeof(float4), stream);
  if (steps) cudaMemsetAsync(steps, 0, np * sizeof(uint32_t), stream);
  TraverseParams P;
  P.tet = m.tet; P.walk = m.walk; P.vert = v.vert; P.extf = m.extf;
  P.planes = (const float4*)v.planes.p;
  P.winner = (const int32_t*)v.winner.p;
  P.rays = (const uint32_t*)v.rays.p;
  P.ent_off = (const uint32_t*)v.ent_off.p;
  P.ent = (const uint2*)v.ent.p;
  P.ctr = v.ctr;
  P.tf = d_tf; P.psi = d_psi;
  P.rgb8 = rgb8; P.rgba = rgba; P.steps = steps;
  P.W = v.W; P.H = v.H; P.nT = m.nT; P.nV = m.nV;
  P.maxEdge = v.maxEdge;
  P.use_view_maxedge = v.use_view_maxedge;
  P.step_cap = step_cap ? step_cap : (uint32_t)std::min<uint64_t>(4ull * m.nT + 64, 0x7fffffffull);
  P.chunk = tune.chunk;
  P.refill = tune.refill;
  P.psi_one = psi_one ? 1u : 0u;
  P.ent_cap = (uint32_t)std::min<size_t>(v.ent_cap, 0xffffffffu);
  const int blocks = num_sms * traverse_blocks_per_sm(v.mode);
  const void* fn = traverse_fn(v.mode, tune.variant);
  void* args[] = {&P};
  return cuda(cudaLaunchKernel(fn, dim3(blocks), dim3(256), args, 0, stream), "stage (c) launch");
}

const void* Ctx::traverse_fn(int mode, uint32_t variant) {
  if (mode == VFR_MODE_REF)
    return variant ? (const void*)traverse_kernel<0, 3> : (const void*)traverse_kernel<0, 2>;
  return variant ? (const void*)traverse_kernel<1, 3> : (const void*)traverse_kernel<1, 2>;
}

void Ctx::prof_mark(int k) {
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
  cudaEventRecord(prof_live.back().e[k], stream);
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

int Ctx::read_counters(View& v, ViewCounters& out) {
  int rc = cuda(cudaMemcpyAsync(h_ctr, v.ctr, sizeof(ViewCounters), cudaMemcpyDeviceToHost, stream),
                "counter read");
  if (!rc) rc = cuda(cudaStreamSynchronize(stream), "stream sync");
  if (!rc) out = *h_ctr;
  return rc;
}

int Ctx::check_status(const ViewCounters& c) {
  if (c.status & (VFR_DEV_ABANDON | VFR_DEV_RANGE | VFR_DEV_STEP_CAP | VFR_DEV_OVERFLOW)) {
    char buf[128];
    std::snprintf(buf, sizeof buf, "device status 0x%x (abandon=1 step-cap=2 range=4 overflow=16)",
                  c.status);
    return fail(VFR_ERR_DEVICE, buf);
  }
  return VFR_OK;
}

}  // namespace vfr

using vfr::Ctx;
using vfr::Mesh;

struct vfr_ctx {
  Ctx impl;
};

#define CTX_OR_FAIL(c)                  \
  if (!(c)) return VFR_ERR_INVALID;     \
  Ctx& C = (c)->impl;                   \
  (void)C;                              \
  cudaSetDevice(C.device);

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
  if (cudaMallocHost(&C.h_ctr, sizeof(vfr::ViewCounters)) != cudaSuccess) return VFR_ERR_NOMEM;
  if (cudaMalloc(&C.view.ctr, sizeof(vfr::ViewCounters)) != cudaSuccess) return VFR_ERR_NOMEM;
  for (auto& e : C.ev) cudaEventCreate(&e);
  *out = c.release();
  return VFR_OK;
}

void vfr_destroy(vfr_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->impl.device);
  cudaStreamSynchronize(c->impl.stream);
  delete c;
}

const char* vfr_last_error(const vfr_ctx* c) { return c ? c->impl.err.c_str() : "null context"; }

int vfr_set_stream(vfr_ctx* c, void* stream) {
  CTX_OR_FAIL(c);
  C.stream = stream ? (cudaStream_t)stream : C.own_stream;
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
    case VFR_OPT_QUEUE_CHUNK:
      if (value < 1) return C.fail(VFR_ERR_INVALID, "queue chunk must be >= 1");
      C.tune.chunk = (uint32_t)value;
      return VFR_OK;
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
  CTX_OR_FAIL(c);
  if (!tf) return C.fail(VFR_ERR_INVALID, "transfer function is NULL");
  std::vector<float> gen;
  if (!psi) {
    gen.resize(512 * 512);
    vfr_psi_table(gen.data());
    psi = gen.data();
  }
  if (!C.d_tf) {
    int rc = C.cuda(cudaMalloc(&C.d_tf, sizeof(float4) * 256), "tf alloc");
    if (!rc) rc = C.cuda(cudaMalloc(&C.d_psi, sizeof(float) * 512 * 512), "psi alloc");
    if (rc) return rc;
  }
  C.psi_one = psi[0] == 1.0f;
  int rc = C.cuda(cudaMemcpyAsync(C.d_tf, tf, sizeof(float) * 1024, cudaMemcpyHostToDevice, C.stream),
                  "tf upload");
  if (!rc)
    rc = C.cuda(cudaMemcpyAsync(C.d_psi, psi, sizeof(float) * 512 * 512, cudaMemcpyHostToDevice,
                                C.stream),
                "psi upload");
  if (!rc) rc = C.cuda(cudaStreamSynchronize(C.stream), "table upload");
  return rc;
}

int vfr_mesh_upload(vfr_ctx* c, const float* vert4, uint32_t nV, const uint32_t* tet4,
                    const uint32_t* con4, uint32_t nT, const uint32_t* extf2, uint32_t nExt,
                    float maxEdge, float maxZ, float minZ, int* mesh_id) {
  CTX_OR_FAIL(c);
  if (!vert4 || !tet4 || !con4 || (!extf2 && nExt) || !mesh_id || nV == 0 || nT == 0)
    return C.fail(VFR_ERR_INVALID, "mesh arrays missing or empty");
  if ((uint64_t)nExt > 4ull * nT) return C.fail(VFR_ERR_INVALID, "more external faces than faces");
  std::string why;
  if (!vfr::validate_mesh(tet4, con4, nV, nT, extf2, nExt, why)) return C.fail(VFR_ERR_MESH, why);
  std::vector<uint32_t> walk(8 * (size_t)nT);
  if (!vfr::build_walk(tet4, con4, nV, nT, walk.data(), why)) return C.fail(VFR_ERR_MESH, why);
  std::unique_ptr<Mesh> m(new Mesh);
  m->nV = nV; m->nT = nT; m->nExt = nExt;
  m->maxEdge = maxEdge; m->maxZ = maxZ; m->minZ = minZ;
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
  cudaStreamSynchronize(C.stream);
  if (C.view.mesh == C.mesh(id)) { C.view.mesh = nullptr; C.view.stage = 0; }
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
  CTX_OR_FAIL(c);
  Mesh* m = C.mesh(id);
  if (!m) return C.fail(VFR_ERR_STATE, "unknown mesh id");
  C.view.stage = 0;
  int rc = C.enqueue_visible(*m, nullptr, C.view);
  vfr::ViewCounters k;
  if (!rc) rc = C.read_counters(C.view, k);
  if (rc) return rc;
  if (num_vis) *num_vis = k.nvis;
  if (visExt && k.nvis)
    rc = C.cuda(cudaMemcpy(visExt, C.view.vis_ext.p, sizeof(uint32_t) * k.nvis,
                           cudaMemcpyDeviceToHost),
                "visible list read");
  if (!rc && faceData && m->nExt) {
    std::vector<float4> pl(2 * (size_t)m->nExt);
    rc = C.cuda(cudaMemcpy(pl.data(), C.view.planes.p, sizeof(float4) * pl.size(),
                           cudaMemcpyDeviceToHost),
                "plane read");
    for (size_t e = 0; e < m->nExt && !rc; ++e) {
      const float4 a = pl[2 * e], b = pl[2 * e + 1];
      float* o = faceData + 6 * e;
      o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = b.x; o[5] = b.y;
    }
  }
  if (!rc) C.view.stage = 1;
  return rc;
}

int vfr_project(vfr_ctx* c, int id, uint32_t W, uint32_t H, uint32_t* bbox, int32_t* writer) {
  CTX_OR_FAIL(c);
  Mesh* m = C.mesh(id);
  if (!m || C.view.mesh != m || C.view.stage < 1)
    return C.fail(VFR_ERR_STATE, "vfr_project needs vfr_find_visible of the same mesh first");
  if (W < 2 || H < 2 || (uint64_t)W * H > (1ull << 31))
    return C.fail(VFR_ERR_INVALID, "image size out of range");
  int rc = C.enqueue_project(C.view, W, H, VFR_MODE_REF);
  vfr::ViewCounters k;
  if (!rc) rc = C.read_counters(C.view, k);
  if (rc) return rc;
  if (bbox && k.nvis)
    rc = C.cuda(cudaMemcpy(bbox, C.view.bbox.p, sizeof(uint4) * k.nvis, cudaMemcpyDeviceToHost),
                "bbox read");
  if (!rc && writer)
    rc = C.cuda(cudaMemcpy(writer, C.view.winner.p, sizeof(int32_t) * (size_t)W * H,
                           cudaMemcpyDeviceToHost),
                "winner read");
  if (!rc) C.view.stage = 2;
  return rc;
}

static int copy_outputs(Ctx& C, uint8_t* rgb8, float* rgba, uint32_t* steps, size_t np) {
  int rc = VFR_OK;
  if (rgb8)
    rc = C.cuda(cudaMemcpyAsync(rgb8, C.out_rgb8.p, np * 3, cudaMemcpyDeviceToHost, C.stream),
                "rgb8 read");
  if (!rc && rgba)
    rc = C.cuda(cudaMemcpyAsync(rgba, C.out_rgba.p, np * sizeof(float4), cudaMemcpyDeviceToHost,
                                C.stream),
                "rgba read");
  if (!rc && steps)
    rc = C.cuda(cudaMemcpyAsync(steps, C.out_steps.p, np * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, C.stream),
                "steps read");
  if (!rc) rc = C.cuda(cudaStreamSynchronize(C.stream), "output read");
  return rc;
}

static int ensure_outputs(Ctx& C, size_t np, bool rgb8, bool rgba, bool steps) {
  int rc = VFR_OK;
  if (rgb8) rc = C.grow(C.out_rgb8, np * 3, "rgb8 output");
  if (!rc && rgba) rc = C.grow(C.out_rgba, np * sizeof(float4), "rgba output");
  if (!rc && steps) rc = C.grow(C.out_steps, np * sizeof(uint32_t), "steps output");
  return rc;
}

static void fill_stats(const vfr::ViewCounters& k, const Mesh& m, vfr_render_stats* s) {
  s->num_ext = m.nExt;
  s->num_vis = k.nvis;
  s->num_rays = k.nrays;
  s->num_entries = k.nentries;
  s->num_steps = k.steps;
  s->device_status = k.status;
}

int vfr_traverse(vfr_ctx* c, int id, uint8_t* rgb8, float* rgba, uint32_t* steps,
                 vfr_render_stats* stats) {
  CTX_OR_FAIL(c);
  Mesh* m = C.mesh(id);
  if (!m || C.view.mesh != m || C.view.stage < 2)
    return C.fail(VFR_ERR_STATE, "vfr_traverse needs vfr_project of the same mesh first");
  if (!C.d_tf) return C.fail(VFR_ERR_STATE, "tables not uploaded");
  const size_t np = (size_t)C.view.W * C.view.H;
  int rc = ensure_outputs(C, np, rgb8 != nullptr, rgba != nullptr, steps != nullptr);
  if (rc) return rc;
  cudaEventRecord(C.ev[0], C.stream);
  rc = C.enqueue_traverse(C.view, rgb8 ? (uint8_t*)C.out_rgb8.p : nullptr,
                          rgba ? (float4*)C.out_rgba.p : nullptr,
                          steps ? (uint32_t*)C.out_steps.p : nullptr);
  cudaEventRecord(C.ev[1], C.stream);
  vfr::ViewCounters k;
  if (!rc) rc = C.read_counters(C.view, k);
  if (!rc) rc = copy_outputs(C, rgb8, rgba, steps, np);
  if (rc) return rc;
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    fill_stats(k, *m, stats);
    cudaEventElapsedTime(&stats->ms_traverse, C.ev[0], C.ev[1]);
    stats->ms_total = stats->ms_traverse;
  }
  C.view.stage = 1;  // the ray queue is consumed; project again before another traverse
  return C.check_status(k);
}

static int render_common(Ctx& C, int id, const float* mv16, uint32_t W, uint32_t H, int mode,
                         uint8_t* rgb8, float4* rgba, uint32_t* steps, int32_t* writer_dev,
                         bool timed) {
  Mesh* m = C.mesh(id);
  if (!m) return C.fail(VFR_ERR_STATE, "unknown mesh id");
  if (!C.d_tf) return C.fail(VFR_ERR_STATE, "tables not uploaded");
  if (W < 2 || H < 2 || (uint64_t)W * H > (1ull << 31))
    return C.fail(VFR_ERR_INVALID, "image size out of range");
  if (mode != VFR_MODE_REF && mode != VFR_MODE_COMPOSITED)
    return C.fail(VFR_ERR_INVALID, "unknown mode");
  if (mode == VFR_MODE_COMPOSITED) {
    size_t want = C.ent_cap_hint ? C.ent_cap_hint : (size_t)W * H * 4;
    C.view.ent_cap = want;
  }
  if (timed) cudaEventRecord(C.ev[0], C.stream);
  C.prof_mark(0);
  int rc = C.enqueue_visible(*m, mv16, C.view);
  if (timed) cudaEventRecord(C.ev[1], C.stream);
  C.prof_mark(1);
  if (!rc) rc = C.enqueue_project(C.view, W, H, mode);
  if (timed) cudaEventRecord(C.ev[2], C.stream);
  C.prof_mark(2);
  if (!rc) rc = C.enqueue_traverse(C.view, rgb8, rgba, steps);
  if (timed) cudaEventRecord(C.ev[3], C.stream);
  C.prof_mark(3);
  if (!rc && writer_dev && mode == VFR_MODE_REF)
    rc = C.cuda(cudaMemcpyAsync(writer_dev, C.view.winner.p, sizeof(int32_t) * (size_t)W * H,
                                cudaMemcpyDeviceToDevice, C.stream),
                "winner copy");
  C.view.stage = 0;
  return rc;
}

int vfr_render(vfr_ctx* c, int id, const float* mv16, uint32_t W, uint32_t H, int mode,
               uint8_t* rgb8, float* rgba, uint32_t* steps, vfr_render_stats* stats) {
  CTX_OR_FAIL(c);
  const size_t np = (size_t)W * H;
  int rc = ensure_outputs(C, np, rgb8 != nullptr, rgba != nullptr, steps != nullptr);
  if (rc) return rc;
  rc = render_common(C, id, mv16, W, H, mode, rgb8 ? (uint8_t*)C.out_rgb8.p : nullptr,
                     rgba ? (float4*)C.out_rgba.p : nullptr,
                     steps ? (uint32_t*)C.out_steps.p : nullptr, nullptr, true);
  vfr::ViewCounters k;
  if (!rc) rc = C.read_counters(C.view, k);
  if (!rc) rc = copy_outputs(C, rgb8, rgba, steps, np);
  if (rc) return rc;
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    fill_stats(k, *C.mesh(id), stats);
    cudaEventElapsedTime(&stats->ms_visible, C.ev[0], C.ev[1]);
    cudaEventElapsedTime(&stats->ms_project, C.ev[1], C.ev[2]);
    cudaEventElapsedTime(&stats->ms_traverse, C.ev[2], C.ev[3]);
    cudaEventElapsedTime(&stats->ms_total, C.ev[0], C.ev[3]);
  }
  if (mode == VFR_MODE_COMPOSITED && k.nentries > C.view.ent_cap) {
    // entry lists overflowed: grow to the exact need and render again
    C.ent_cap_hint = k.nentries + k.nentries / 8;
    return vfr_render(c, id, mv16, W, H, mode, rgb8, rgba, steps, stats);
  }
  return C.check_status(k);
}

int vfr_render_device(vfr_ctx* c, int id, const float* mv16, uint32_t W, uint32_t H, int mode,
                      uint8_t* rgb8_dev, float* rgba_dev, uint32_t* steps_dev, int32_t* writer_dev) {
  CTX_OR_FAIL(c);
  return render_common(C, id, mv16, W, H, mode, rgb8_dev, (float4*)rgba_dev, steps_dev, writer_dev,
                       false);
}

int vfr_device_status(vfr_ctx* c, uint32_t* status) {
  CTX_OR_FAIL(c);
  vfr::ViewCounters k;
  int rc = C.read_counters(C.view, k);
  if (rc) return rc;
  if (status) *status = k.status;
  if (C.view.mode == VFR_MODE_COMPOSITED && k.nentries > C.view.ent_cap) {
    C.ent_cap_hint = k.nentries + k.nentries / 8;
    return C.fail(VFR_ERR_DEVICE, "entry lists overflowed; render again");
  }
  return C.check_status(k);
}

}  // extern "C"
