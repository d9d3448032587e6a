// Internal host-side types of the render library (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "vfr_host.h"
#include "vfr_kernels.cuh"

namespace vfr {

// Grow-only device buffer.
struct Buf {
  void* p = nullptr;
  size_t cap = 0;
  Buf() = default;
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  ~Buf() {
    if (p) cudaFree(p);
  }
};

// A resident mesh: packed 32-byte tet records, float4 vertices, ext faces.
struct Mesh {
  uint32_t nV = 0, nT = 0, nExt = 0;
  float maxEdge = 0, maxZ = 0, minZ = 0;
  uint4* tet = nullptr;     // vertex ids per tet (the reference's tetList)
  WalkRec* walk = nullptr;  // neighbour + opposite-vertex words per tet
  float4* vert = nullptr;
  uint2* extf = nullptr;
  size_t bytes = 0;
  ~Mesh() {
    if (tet) cudaFree(tet);
    if (walk) cudaFree(walk);
    if (vert) cudaFree(vert);
    if (extf) cudaFree(extf);
  }
};

// Scratch and state of one view in flight.
struct View {
  Mesh* mesh = nullptr;
  const float4* vert = nullptr;
  float maxEdge = 0;
  int use_view_maxedge = 0;
  uint32_t W = 0, H = 0;
  int mode = 0;
  int stage = 0;  // 0 none, 1 visible done, 2 project done
  ViewCounters* ctr = nullptr;
  size_t ent_cap = 0;
  Buf vview, planes, blk, vis_ext, bbox, winner, rays, ent_cnt, ent_off, ent_cur, ent, scan;
  ~View() {
    if (ctr) cudaFree(ctr);
  }
};

struct Tuning {
  uint32_t chunk = 32;        // rays per warp fetch from the ray queue
  uint32_t blocks_per_sm = 0; // traversal CTAs per SM (0: occupancy maximum)
  uint32_t refill = 1;        // refill idle lanes once this many of a warp's are idle
  uint32_t variant = 0;       // traversal register budget: 0 = 2 CTAs/SM, 1 = 3 CTAs/SM
};

// Four events bracketing the stages of one view (profiling).
struct StageEvents {
  cudaEvent_t e[4] = {};
};

struct Ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  std::string err;
  float4* d_tf = nullptr;
  float* d_psi = nullptr;
  bool psi_one = false;  // psi[0][0] == 1.0f
  std::vector<std::unique_ptr<Mesh>> meshes;
  View view;
  Buf out_rgb8, out_rgba, out_steps;
  ViewCounters* h_ctr = nullptr;
  cudaEvent_t ev[4] = {};
  int occ[4] = {0, 0, 0, 0};
  uint32_t step_cap = 0;
  size_t ent_cap_hint = 0;
  Tuning tune;
  bool profile = false;
  std::vector<StageEvents> prof_pool;  // recycled events
  std::vector<StageEvents> prof_live;  // recorded, not yet read
  StageEvents* prof_cur = nullptr;
  void prof_mark(int k);

  ~Ctx() {
    meshes.clear();
    if (d_tf) cudaFree(d_tf);
    if (d_psi) cudaFree(d_psi);
    if (h_ctr) cudaFreeHost(h_ctr);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto* v : {&prof_pool, &prof_live})
      for (auto& s : *v)
        for (auto& e : s.e)
          if (e) cudaEventDestroy(e);
    if (own_stream) cudaStreamDestroy(own_stream);
  }

  int fail(int code, const std::string& msg);
  int cuda(cudaError_t e, const char* what);
  int grow(Buf& b, size_t bytes, const char* what);
  Mesh* mesh(int id);
  int enqueue_visible(Mesh& m, const float* mv16, View& v);
  int enqueue_project(View& v, uint32_t W, uint32_t H, int mode);
  int enqueue_traverse(View& v, uint8_t* rgb8, float4* rgba, uint32_t* steps);
  int traverse_blocks_per_sm(int mode);
  const void* traverse_fn(int mode, uint32_t variant);
  int read_counters(View& v, ViewCounters& out);
  int check_status(const ViewCounters& c);
};

}  // namespace vfr
