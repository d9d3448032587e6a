// Stage (a) without allocation: visible-face detection and ordered
// compaction whose scratch lives in a fixed device array of this library.
//
// Some callers cannot let a library allocate device memory: an application
// that has reserved all of the GPU's memory for its own pool (a game engine,
// a serving process with a fixed budget), or a latency-critical frame loop
// in which cudaMalloc/cudaFree, which may synchronise the device, must not
// run.  vfr_find_visible_static takes the mesh and the outputs as the
// caller's device buffers and uses, besides them, only g_scratch below: the
// per-face plane coefficients and the per-block counts of visible faces.
//
// g_scratch is a file-scope __device__ array, so every GPU that loads this
// library holds kStaticScratchBytes of it until the process exits.  Host code
// may not use its name as an address.  Its device address belongs to a CUDA
// context (a host application may make its own driver-API context current,
// and a device reset makes a new one), so every call whose stream is not
// capturing looks it up again with cudaGetSymbolAddress in the current
// context and remembers it for that context; a call under stream capture
// uses the address remembered for its context and is refused if there is
// none.  All calls share the array and it keeps the last call's contents;
// calls that overlap on the GPU race.
#include <cuda.h>  // driver types only: the two context queries come through the runtime
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <utility>
#include <vector>

#include "vfr_device.cuh"
#include "vfray.h"

namespace {

constexpr uint32_t kStaticBlock = 1024;
constexpr size_t kPlaneBytes = sizeof(float4) * 2 * VFR_STATIC_MAX_EXT;
constexpr size_t kCountBytes = sizeof(uint32_t) * (VFR_STATIC_MAX_EXT / kStaticBlock);
constexpr size_t kStaticScratchBytes = kPlaneBytes + kCountBytes;

static __device__ __align__(256) unsigned char g_scratch[kStaticScratchBytes];

// Addresses of g_scratch found so far, per context (by the context's unique
// id, which is not reused after a context is destroyed).  Failed lookups are
// not remembered.
std::mutex g_mu;
std::vector<std::pair<unsigned long long, void*>> g_addr;

// Plane coefficients and back-face test of every external face, as
// vfRayKernelCPU.cc:51-132, and the count of visible faces per block.
__global__ void __launch_bounds__(kStaticBlock)
    visible_static_kernel(const float4* __restrict__ vert, const uint4* __restrict__ tet,
                          const uint2* __restrict__ extf, uint32_t nExt, uint32_t nV, uint32_t nT,
                          unsigned char* scratch) {
  float4* planes = reinterpret_cast<float4*>(scratch);
  uint32_t* blk = reinterpret_cast<uint32_t*>(scratch + kPlaneBytes);
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  int vis = 0;
  if (e < nExt) {
    const uint2 tf = extf[e];
    bool ok = tf.x < nT && tf.y < 4;
    const uint4 id = ok ? tet[tf.x] : make_uint4(0, 0, 0, 0);
    ok = ok && id.x < nV && id.y < nV && id.z < nV && id.w < nV;
    if (!ok) {  // ids out of range: the face counts as not visible
      planes[2 * (size_t)e] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
      planes[2 * (size_t)e + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float4 v0 = ok ? vert[vfr::sel4(id, tf.y & 3u)] : z4;
    const float4 v1 = ok ? vert[vfr::sel4(id, (tf.y + 1) & 3u)] : z4;
    const float4 v2 = ok ? vert[vfr::sel4(id, (tf.y + 2) & 3u)] : z4;
    const float4 op = ok ? vert[vfr::sel4(id, (tf.y + 3) & 3u)] : z4;
    vfr::Plane P;
    vfr::face_plane(v0, v1, v2, P);
    if (vfr::plane_eval(op.x, op.y, P.zx, P.zy, P.zz) < op.z) P.sx = -1.0f;
    vis = ok && (P.sx != -1.0f);
    if (ok) {
      planes[2 * (size_t)e] = make_float4(P.zx, P.zy, P.zz, P.sx);
      planes[2 * (size_t)e + 1] = make_float4(P.sy, P.sz, 0.0f, 0.0f);
    }
  }
  const int cnt = __syncthreads_count(vis);
  if (threadIdx.x == 0) blk[blockIdx.x] = (uint32_t)cnt;
}

// Ordered compaction (main.cc:93-138): block offset = sum of the counts of
// the blocks before it, rank inside the block from warp ballots.
__global__ void __launch_bounds__(kStaticBlock)
    compact_static_kernel(uint32_t nExt, const unsigned char* scratch, uint32_t* __restrict__ vis_ext,
                          uint32_t* __restrict__ num_vis) {
  const float4* planes = reinterpret_cast<const float4*>(scratch);
  const uint32_t* blk = reinterpret_cast<const uint32_t*>(scratch + kPlaneBytes);
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_base;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t part = 0;
  for (uint32_t b = threadIdx.x; b < blockIdx.x; b += blockDim.x) part += blk[b];
  for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if (lane == 0) s_warp[warp] = part;
  __syncthreads();
  if (warp == 0) {
    uint32_t x = s_warp[lane];
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
    uint32_t c = s_warp[lane], x = c;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    s_warp[lane] = x - c;
    if (blockIdx.x == gridDim.x - 1 && lane == 31) *num_vis = s_base + x;
  }
  __syncthreads();
  if (vis) vis_ext[s_base + s_warp[warp] + __popc(m & ((1u << lane) - 1u))] = e;
}

// Unique id of the current CUDA context (cuCtxGetCurrent + cuCtxGetId,
// reached through the runtime's driver entry points, so the library needs no
// link to the driver library).  False when there is none or the query fails.
bool current_context_id(unsigned long long* id) {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      get_current = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      get_id = nullptr;
    cudaGetLastError();
  });
  CUcontext c = nullptr;
  if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c) return false;
  return get_id(c, id) == CUDA_SUCCESS;
}

// Address of g_scratch in the current context.  capturing: the stream is
// under capture, so use the address an earlier call found in this context
// (VFR_ERR_STATE without one); otherwise look it up now and remember it.
int scratch_address(bool capturing, void** out) {
  unsigned long long id = 0;
  if (!current_context_id(&id)) return VFR_ERR_CUDA;
  std::lock_guard<std::mutex> g(g_mu);
  auto it = g_addr.begin();
  while (it != g_addr.end() && it->first != id) ++it;
  if (capturing) {
    if (it == g_addr.end()) return VFR_ERR_STATE;
    *out = it->second;
    return VFR_OK;
  }
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return VFR_ERR_CUDA;
  }
  if (it != g_addr.end()) it->second = p;
  else g_addr.emplace_back(id, p);
  *out = p;
  return VFR_OK;
}

bool aligned(const void* p, size_t a) { return ((uintptr_t)p % a) == 0; }

}  // namespace

extern "C" int vfr_find_visible_static(const float* vert4_dev, uint32_t nV, const uint32_t* tet4_dev,
                                       uint32_t nT, const uint32_t* extf2_dev, uint32_t nExt,
                                       uint32_t* visExt_dev, uint32_t* num_vis_dev, void* stream) {
  if (!vert4_dev || !tet4_dev || !visExt_dev || !num_vis_dev || (!extf2_dev && nExt) || nV == 0 ||
      nT == 0)
    return VFR_ERR_INVALID;
  if (nExt > VFR_STATIC_MAX_EXT) return VFR_ERR_BUDGET;  // beyond the fixed scratch
  if (!aligned(vert4_dev, 16) || !aligned(tet4_dev, 16) || !aligned(extf2_dev, 8) ||
      !aligned(visExt_dev, 4) || !aligned(num_vis_dev, 4))
    return VFR_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
    cudaGetLastError();
    return VFR_ERR_CUDA;
  }
  void* scratch = nullptr;
  const int rc = scratch_address(cs != cudaStreamCaptureStatusNone, &scratch);
  if (rc) return rc;
  if (cudaMemsetAsync(num_vis_dev, 0, sizeof(uint32_t), s) != cudaSuccess) return VFR_ERR_CUDA;
  if (nExt) {
    const uint32_t nblk = (nExt + kStaticBlock - 1) / kStaticBlock;
    visible_static_kernel<<<nblk, kStaticBlock, 0, s>>>(
        reinterpret_cast<const float4*>(vert4_dev), reinterpret_cast<const uint4*>(tet4_dev),
        reinterpret_cast<const uint2*>(extf2_dev), nExt, nV, nT, (unsigned char*)scratch);
    compact_static_kernel<<<nblk, kStaticBlock, 0, s>>>(nExt, (const unsigned char*)scratch,
                                                        visExt_dev, num_vis_dev);
  }
  return cudaGetLastError() == cudaSuccess ? VFR_OK : VFR_ERR_CUDA;
}
