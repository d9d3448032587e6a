// Internal host-side types of the render library (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "vfr_host.h"
#include "vfr_types.cuh"

namespace vfr {

// A named NVTX range over a host call or stage, for Nsight timelines and
// ncu's --nvtx filters (header-only NVTX 3: a no-op unless a tool is
// attached).
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

// Grow-only device buffer, or a piece of an Arena (owned = false: never
// freed by the buffer).
struct Buf {
  void* p = nullptr;
  size_t cap = 0;
  bool owned = true;
  Buf() = default;
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  ~Buf() { release(); }
  void release() {
    if (p && owned) cudaFree(p);
    p = nullptr;
    cap = 0;
    owned = true;
  }
  template <class T>
  T* as(size_t byte_off = 0) const {
    return reinterpret_cast<T*>(static_cast<char*>(p) + byte_off);
  }
};

// A resident mesh: tets, walk records, vertices, external faces.
struct Mesh {
  uint32_t nV = 0, nT = 0, nExt = 0;
  float maxEdge = 0, maxZ = 0, minZ = 0;
  uint4* tet = nullptr;     // vertex ids per tet (the reference's tetList)
  WalkRec* walk = nullptr;  // neighbour + opposite-vertex words per tet
  float4* vert = nullptr;
  uint2* extf = nullptr;
  // the mesh's distinct edges (min id, max id), built on first use by a view
  // with a model-view (its maxEdgeLength is recomputed per view)
  uint2* edges = nullptr;
  uint32_t nEdges = 0;
  size_t bytes = 0;
  ~Mesh() {
    if (edges) cudaFree(edges);
    if (tet) cudaFree(tet);
    if (walk) cudaFree(walk);
    if (vert) cudaFree(vert);
    if (extf) cudaFree(extf);
  }
};

struct Tuning {
  uint32_t blocks_per_sm = 0;  // traversal CTAs per SM (0: occupancy maximum)
  uint32_t refill = 4;         // refill idle lanes once this many of a warp's are idle
  uint32_t variant = 1;        // traversal register budget: 0 = 2 CTAs/SM, 1 = 3 CTAs/SM
  uint32_t raster_warps_per_sm = 64;
  uint32_t tile_w = 4;          // ray-list tile width (x 32/tile_w rows)
};

struct Ctx;

// A region of device memory that batches are laid out in by bumping an
// offset (the served form's arena): nothing is allocated or freed per batch.
struct Arena {
  char* base = nullptr;
  size_t cap = 0, off = 0;
};

// One render job as the caller describes it.
struct JobSpec {
  int mesh = -1;
  uint32_t W = 0, H = 0;
  bool use_mv = false;
  float mv[16] = {};
  uint8_t* rgb8 = nullptr;  // device outputs (any may be null)
  float4* rgba = nullptr;
  uint32_t* steps = nullptr;
};

// A set of jobs laid out in shared device arenas, run as one chain of
// launches (optionally a CUDA graph).
struct Batch {
  Ctx* ctx = nullptr;
  int mode = 0;
  std::vector<JobSpec> specs;
  std::vector<JobDev> jobs;
  uint32_t njobs = 0;
  // host-known prefixes: view blocks, edge blocks, ext-face blocks, ray-list
  // tiles, screen tiles (composited stage (b))
  std::vector<uint32_t> pref;  // 5 arrays of njobs + 1
  uint32_t rot_blocks = 0, edge_blocks = 0, ext_blocks = 0, tiles = 0, stiles = 0;
  size_t pixels = 0, ext_total = 0;
  uint64_t scratch_bytes = 0;
  Buf d_jobs, d_pref, d_dev_pref, d_ctr;  // d_dev_pref: vis prefix, ray prefix, queue
  Buf vview, planes, blk, vis, bbox, winner, rays, ent_cnt, ent_off, ent, scan;
  Buf tile_cnt, tile_off, tile_cur, bins;  // composited: faces binned by screen tile
  Buf out_rgb8, out_rgba, out_steps;      // outputs owned by the batch (host-output calls)
  size_t ent_cap = 0, bin_cap = 0;  // composited: entry and bin capacities (0: sized at layout)
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;  // null: the context's stream
  cudaStream_t st() const;
  // pinned staging for the per-call upload of a one-job batch
  void* stage = nullptr;
  size_t stage_cap = 0;
  // or the caller's pinned staging (not owned; the served form's pool): a
  // pinned allocation waits for all work on the device, a running served
  // launch included
  char* ext_stage = nullptr;
  size_t ext_stage_cap = 0;
  cudaEvent_t stage_done = nullptr;

  ~Batch();
  uint32_t* vis_pref() const { return d_dev_pref.as<uint32_t>(); }
  uint32_t* ray_pref() const { return d_dev_pref.as<uint32_t>((njobs + 1) * 4); }
  uint32_t* queue() const { return d_dev_pref.as<uint32_t>(2 * (njobs + 1) * 4); }
  uint32_t tile_w = 8;  // the tile shape the layout was made for
  // Where the buffers come from: grow-only allocations of the batch's own,
  // or (arena set) consecutive pieces of the arena from its offset on.
  Arena* arena = nullptr;
  bool rgb8_only = false;  // owned outputs: RGB8 only (no float RGBA, no steps)
  // Threads of the stage (a) and scan blocks: 1024, or 256 so that the
  // chain fits beside the served launch (CTAs of at most 256 threads).
  uint32_t fb = 1024;
  int layout(const std::vector<JobSpec>& s, int mode, bool own_outputs);
  int place(Buf& b, size_t bytes, const char* what);
  // Arena bytes a layout of these jobs takes (an upper bound).
  static size_t arena_bytes(Ctx& C, const std::vector<JobSpec>& s, int mode, uint32_t fb,
                            bool rgb8_only);
  int upload(bool async);
  int enqueue_a();
  int enqueue_b();
  int enqueue_c();
  int enqueue_all() {
    int rc = enqueue_a();
    if (!rc) rc = enqueue_b();
    if (!rc) rc = enqueue_c();
    return rc;
  }
  int capture();
  int run();
  int counters(std::vector<ViewCounters>& out);
  bool overflowed(const std::vector<ViewCounters>& k);
  void drop_graph();
};

struct Ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  std::string err;
  float4* d_tf = nullptr;
  float* d_psi = nullptr;
  std::vector<std::unique_ptr<Mesh>> meshes;
  Batch plain;     // the one-job batch behind the single-view calls
  int stage = 0;   // single-view stage calls: 0 none, 1 visible done, 2 project done
  cudaEvent_t ev[4] = {};
  int occ[4] = {0, 0, 0, 0};
  uint32_t step_cap = 0;
  size_t ent_cap_hint = 0, bin_cap_hint = 0;
  Tuning tune;
  bool profile = false;
  struct StageEvents {
    cudaEvent_t e[4] = {};
  };
  std::vector<StageEvents> prof_pool, prof_live;
  std::vector<void*> batches;  // live vfr_batch handles, detached when the context goes

  ~Ctx();
  void prof_mark(int k, cudaStream_t on = nullptr);  // on: the stream the stages run on (null: the context stream)
  int fail(int code, const std::string& msg);
  int cuda(cudaError_t e, const char* what);
  int grow(Buf& b, size_t bytes, const char* what);
  Mesh* mesh(int id);
  int mesh_edges(Mesh* m, cudaStream_t st);
  int traverse_blocks_per_sm(int mode);
  const void* traverse_fn(int mode, uint32_t variant);
  int check_status(uint32_t status, uint32_t nentries_over);
};

// The served form's launches (vfr_render.cu, where the kernels are
// compiled): the drain, its occupancy, and the publication of a segment.
int serve_blocks_per_sm(int* n);
cudaError_t launch_serve(const ServeParams& sp, int grid, cudaStream_t st);
cudaError_t launch_publish(SegDev* segs, ServeCtl* ctl, uint32_t seq, const JobDev* jobs,
                           const uint32_t* ray_pref, uint32_t* done, uint32_t njobs,
                           cudaStream_t st);

}  // namespace vfr

// The C ABI's context handle.
struct vfr_ctx {
  vfr::Ctx impl;
};
