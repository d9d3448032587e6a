// Test infrastructure: a C-ABI harness around the reference's own CPU render
// path, for the parity tests and the CPU baseline only.  Nothing in the
// vfray_b200 product links or loads this file.
//
// It is compiled together with the reference sources exactly where they lie
// (vfRayKernelCPU.cc, vfRayPreComp.cc; see oracle/Makefile) and replaces only
// the reference's driver main.cc:58-238 with code of our own:
//
//  * stages 1-3 are the reference functions findVisibleFaces,
//    projectVisibleFaces and vfRay (vfRayKernelCPU.h:61-80), called per face
//    in index order exactly as main.cc:80-84,171-176,209-218 does, including
//    the padding duplicate of the last visible face (main.cc:124-126);
//  * the face cache inside vfRay indexes a 512-slot stack array by centroid z
//    (vfRayKernelCPU.cc:234-245,369-435) and overflows it when a centroid
//    reaches maxZ (slot 512).  maxZ/minZ feed nothing but that index, and a
//    cache hit returns the identical recomputation, so the harness passes a
//    z range widened by 1% on each side: every slot stays in [0,511] and the
//    image is unchanged;
//  * writer detection (which visible face wrote each pixel last) renders each
//    face twice over two different sentinel fills of its bounding box;
//  * the multi-threaded baseline splits the screen into column strips; each
//    thread calls the unmodified vfRay on every face overlapping its strip,
//    in face order, with the face's bounding box clipped to the strip, so the
//    reference's last-writer order per pixel is kept.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "vfRayPreComp.h"
#include "vfRayKernelCPU.h"

#define API extern "C" __attribute__((visibility("default")))

// Globals the reference precomputation works on (declared extern in
// vfRayPreComp.h:83-94; the reference defines them in main.cc:34-45).
uint numVerts = 0, numTets = 0;
real* h_vertList = nullptr;
uint* h_tetList = nullptr;
uint* h_extFaces = nullptr;
uint* h_conTet = nullptr;
real* h_transferFunction = nullptr;
uint numExtFaces = 0;
real h_maxEdgeLength = 0, h_maxZ = 0, h_minZ = 0;

extern float psiGammaTable[512][512];

#ifdef VFREF_COUNT_EXP
// Incremented by the exp() wrapper that oracle/ref_count_hook.h puts in
// front of vfRayKernelCPU.cc: one call per compositing step
// (vfRayKernelCPU.cc:458), so per-face counts pin the traversal lengths.
extern "C" { unsigned long long vfref_exp_calls = 0; }
#endif

API int ref_variant(void) {
#ifdef VFREF_COUNT_EXP
  return 2;
#elif defined(__FAST_MATH__)
  return 1;
#else
  return 0;
#endif
}

API void ref_set_psi(const float* t) { std::memcpy(psiGammaTable, t, sizeof(psiGammaTable)); }
API void ref_get_psi(float* t) { std::memcpy(t, psiGammaTable, sizeof(psiGammaTable)); }

API int ref_set_mesh(const float* v, uint nv, const uint* t, uint nt) {
  delete[] h_vertList; delete[] h_tetList;
  numVerts = nv; numTets = nt;
  h_vertList = new real[4 * (size_t)nv];
  h_tetList = new uint[4 * (size_t)nt];
  std::memcpy(h_vertList, v, sizeof(real) * 4 * (size_t)nv);
  std::memcpy(h_tetList, t, sizeof(uint) * 4 * (size_t)nt);
  return 0;
}
API void ref_get_vert(float* v) { std::memcpy(v, h_vertList, sizeof(real) * 4 * (size_t)numVerts); }
// Restores the vertices only (same count), e.g. the normalised mesh before
// the next view's rotateVolume.
API void ref_set_vert(const float* v) { std::memcpy(h_vertList, v, sizeof(real) * 4 * (size_t)numVerts); }
API uint ref_num_verts(void) { return numVerts; }
API uint ref_num_tets(void) { return numTets; }
API uint ref_num_ext(void) { return numExtFaces; }

API void ref_normalize(void) { normalizeVertices(); }
API void ref_rotate(const float* mv) {
  real m[16];
  for (int i = 0; i < 16; ++i) m[i] = mv[i];
  rotateVolume(m);
}

// Reference precomputation (O(nV*nT) incidence: small meshes only).  The
// incidence is not freed with deleteIncid: that function deletes the static
// array without clearing the pointer (vfRayPreComp.cc:349-367), so the next
// buildIncid would delete it again; buildIncid frees the previous one itself.
API int ref_build_con(void) {
  if (!buildIncid()) return -1;
  return buildCon() ? 0 : -2;
}
API int ref_build_extf(void) { return buildExtF() ? 0 : -1; }
API int ref_build_lmt(void) { return buildLmt() ? 0 : -1; }
API int ref_build_tf(void) { return buildTF() ? 0 : -1; }

API void ref_set_con(const uint* c, uint next) {
  delete[] h_conTet;
  h_conTet = new uint[4 * (size_t)numTets];
  std::memcpy(h_conTet, c, sizeof(uint) * 4 * (size_t)numTets);
  numExtFaces = next;
}
API void ref_get_con(uint* c) { std::memcpy(c, h_conTet, sizeof(uint) * 4 * (size_t)numTets); }
API void ref_set_extf(const uint* e, uint n) {
  delete[] h_extFaces;
  numExtFaces = n;
  h_extFaces = new uint[2 * (size_t)n + 2];
  std::memcpy(h_extFaces, e, sizeof(uint) * 2 * (size_t)n);
}
API void ref_get_extf(uint* e) { std::memcpy(e, h_extFaces, sizeof(uint) * 2 * (size_t)numExtFaces); }
API void ref_set_lmt(float me, float mz, float nz) { h_maxEdgeLength = me; h_maxZ = mz; h_minZ = nz; }
API void ref_get_lmt(float* o) { o[0] = h_maxEdgeLength; o[1] = h_maxZ; o[2] = h_minZ; }
API void ref_set_tf(const float* tf) {
  delete[] h_transferFunction;
  h_transferFunction = new real[1024];
  std::memcpy(h_transferFunction, tf, sizeof(real) * 1024);
}
API void ref_get_tf(float* tf) { std::memcpy(tf, h_transferFunction, sizeof(real) * 1024); }

// File readers / writers of the reference, for the format pins.
API int ref_read_off(const char* f) { return readOff(f) ? 0 : -1; }
API int ref_read_con(const char* f) { return readCon(f) ? 0 : -1; }
API int ref_read_extf(const char* f) { return readExtF(f) ? 0 : -1; }
API int ref_read_lmt(const char* f) { return readLmt(f) ? 0 : -1; }
API int ref_read_tf(const char* f) { return readTF(f) ? 0 : -1; }
API int ref_write_con(const char* f) { return writeCon(f) ? 0 : -1; }
API int ref_write_extf(const char* f) { return writeExtF(f) ? 0 : -1; }
API int ref_write_lmt(const char* f) { return writeLmt(f) ? 0 : -1; }
API int ref_write_tf(const char* f) { return writeTF(f) ? 0 : -1; }
API int ref_write_ppm(const char* f, const uint8_t* img, uint w, uint h) {
  return ppmWrite(f, img, w, h) ? 0 : -1;
}

namespace {

struct Prepared {
  std::vector<faceData> vis;       // compacted visible faces (+1 duplicate)
  std::vector<uint> extf;          // compacted (tet, face) pairs (+1 duplicate)
  std::vector<uint> visExt;        // ext-face index of each compacted face
  std::vector<projectedFace> proj;
  uint numVis = 0;                 // including the padding duplicate
  real zlo = 0, zhi = 0;
};

// Stage 1 + host compaction + stage 2, as main.cc:73-182 sequences them.
void prepare(Prepared& p, uint W, uint H) {
  std::vector<faceData> all(numExtFaces);
  for (uint i = 0; i < numExtFaces; ++i)
    findVisibleFaces(all.data(), h_vertList, h_tetList, h_extFaces, i);
  p.vis.clear(); p.extf.clear(); p.visExt.clear();
  for (uint i = 0; i < numExtFaces; ++i) {
    if (all[i].sParams.x != -1.0) {
      p.vis.push_back(all[i]);
      p.extf.push_back(h_extFaces[2 * i]);
      p.extf.push_back(h_extFaces[2 * i + 1]);
      p.visExt.push_back(i);
    }
  }
  p.numVis = 0;
  p.proj.clear();
  if (p.vis.empty()) return;
  p.vis.push_back(p.vis.back());
  p.extf.push_back(p.extf[p.extf.size() - 2]);
  p.extf.push_back(p.extf[p.extf.size() - 2]);
  p.visExt.push_back(p.visExt.back());
  p.numVis = (uint)p.vis.size();
  p.proj.resize(p.numVis);
  for (uint i = 0; i < p.numVis; ++i)
    projectVisibleFaces(p.proj.data(), h_vertList, h_tetList, p.extf.data(), p.vis.data(), i, W, H);
  real lo = h_vertList[2], hi = h_vertList[2];
  for (uint i = 1; i < numVerts; ++i) {
    lo = std::min(lo, h_vertList[4 * i + 2]);
    hi = std::max(hi, h_vertList[4 * i + 2]);
  }
  real m = std::max((hi - lo) * 0.01f, 1e-3f);
  p.zlo = lo - m; p.zhi = hi + m;
}

inline void call_vfray(uint8_t* img, const Prepared& p, const projectedFace* proj, uint i, uint W, uint H) {
  vfRay(img, h_vertList, h_tetList, p.extf.data(), p.vis.data(), proj, h_conTet,
        h_transferFunction, i, W, H, h_maxEdgeLength, p.zhi, p.zlo);
}

}  // namespace

// Render one view.  Outputs (any may be null): img W*H*3 RGB8 (zeroed first,
// as main.cc:194), writer W*H (ext-face index of the last visible face that
// wrote the pixel, -1 if none), visExt (ext-face indices of the visible
// faces in compacted order, without the duplicate; capacity numExtFaces),
// bbox (4 per visible face), faceExp (exp calls per visible face, counting
// build only).  Returns the number of visible faces (without the duplicate).
API int ref_render(uint W, uint H, uint8_t* img, int32_t* writer, uint* visExt,
                   uint* bbox, unsigned long long* faceExp, double* seconds) {
  if (!h_vertList || !h_tetList || !h_conTet || !h_extFaces || !h_transferFunction) return -1;
  auto t0 = std::chrono::steady_clock::now();
  Prepared p;
  prepare(p, W, H);
  std::vector<uint8_t> local;
  if (!img) { local.resize((size_t)W * H * 3); img = local.data(); }
  std::memset(img, 0, (size_t)W * H * 3);
  if (writer) std::fill(writer, writer + (size_t)W * H, -1);
  const bool detect = writer != nullptr || faceExp != nullptr;
  std::vector<uint8_t> save, runA;
  for (uint i = 0; i < p.numVis; ++i) {
    if (!detect) { call_vfray(img, p, p.proj.data(), i, W, H); continue; }
    const uint4 b = p.proj[i].bBox;
    if (b.x > b.z || b.y > b.w) { call_vfray(img, p, p.proj.data(), i, W, H); continue; }
    // Save the face's box, render over sentinel A and over sentinel B; a
    // pixel was written iff it differs from its sentinel in either run.
    const uint bw = b.z - b.x + 1, bh = b.w - b.y + 1;
    save.resize((size_t)bw * bh * 3); runA.resize(save.size());
    auto box = [&](uint x, uint y) { return ((size_t)(y - b.y) * bw + (x - b.x)) * 3; };
    auto pix = [&](uint x, uint y) { return ((size_t)y * W + x) * 3; };
    for (uint y = b.y; y <= b.w; ++y)
      for (uint x = b.x; x <= b.z; ++x) std::memcpy(&save[box(x, y)], &img[pix(x, y)], 3);
    const uint8_t A[3] = {0x11, 0x22, 0x33}, B[3] = {0xEE, 0xDD, 0xCC};
    for (uint y = b.y; y <= b.w; ++y)
      for (uint x = b.x; x <= b.z; ++x) std::memcpy(&img[pix(x, y)], A, 3);
#ifdef VFREF_COUNT_EXP
    unsigned long long e0 = vfref_exp_calls;
#endif
    call_vfray(img, p, p.proj.data(), i, W, H);
#ifdef VFREF_COUNT_EXP
    if (faceExp && i + 1 < p.numVis) faceExp[i] = vfref_exp_calls - e0;
#else
    if (faceExp && i + 1 < p.numVis) faceExp[i] = ~0ull;
#endif
    for (uint y = b.y; y <= b.w; ++y)
      for (uint x = b.x; x <= b.z; ++x) {
        std::memcpy(&runA[box(x, y)], &img[pix(x, y)], 3);
        std::memcpy(&img[pix(x, y)], B, 3);
      }
    call_vfray(img, p, p.proj.data(), i, W, H);
    for (uint y = b.y; y <= b.w; ++y)
      for (uint x = b.x; x <= b.z; ++x) {
        uint8_t* q = &img[pix(x, y)];
        const uint8_t* a = &runA[box(x, y)];
        bool wa = std::memcmp(a, A, 3) != 0, wb = std::memcmp(q, B, 3) != 0;
        if (wa || wb) {
          if (wa) std::memcpy(q, a, 3);
          if (writer) writer[(size_t)y * W + x] = (int32_t)p.visExt[i];
        } else {
          std::memcpy(q, &save[box(x, y)], 3);
        }
      }
  }
  uint nvis = p.numVis ? p.numVis - 1 : 0;
  if (visExt) for (uint i = 0; i < nvis; ++i) visExt[i] = p.visExt[i];
  if (bbox)
    for (uint i = 0; i < nvis; ++i) {
      bbox[4 * i + 0] = p.proj[i].bBox.x; bbox[4 * i + 1] = p.proj[i].bBox.y;
      bbox[4 * i + 2] = p.proj[i].bBox.z; bbox[4 * i + 3] = p.proj[i].bBox.w;
    }
  if (seconds)
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return (int)nvis;
}

// Multi-threaded render of one view over column strips (see the header
// comment); returns the number of visible faces, the wall time in *seconds.
API int ref_render_mt(uint W, uint H, uint8_t* img, int threads, int strip, double* seconds) {
  if (!h_vertList || !h_tetList || !h_conTet || !h_extFaces || !h_transferFunction) return -1;
  if (threads < 1) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  if (strip < 1) strip = 8;
  auto t0 = std::chrono::steady_clock::now();
  Prepared p;
  prepare(p, W, H);
  std::vector<uint8_t> local;
  if (!img) { local.resize((size_t)W * H * 3); img = local.data(); }
  std::memset(img, 0, (size_t)W * H * 3);
  const uint nstrips = (W + strip - 1) / strip;
  // per-strip face lists, in face order
  std::vector<std::vector<uint>> lists(nstrips);
  for (uint i = 0; i < p.numVis; ++i) {
    const uint4 b = p.proj[i].bBox;
    if (b.x > b.z) continue;
    for (uint s = b.x / strip; s <= std::min(b.z / strip, nstrips - 1); ++s) lists[s].push_back(i);
  }
  std::atomic<uint> next(0);
  auto work = [&]() {
    std::vector<projectedFace> proj(p.proj);
    for (;;) {
      uint s = next.fetch_add(1);
      if (s >= nstrips) break;
      const uint x0 = s * strip, x1 = std::min(W, x0 + strip) - 1;
      for (uint i : lists[s]) {
        projectedFace c = p.proj[i];
        c.bBox.x = std::max(c.bBox.x, x0);
        c.bBox.z = std::min(c.bBox.z, x1);
        proj[i] = c;
        call_vfray(img, p, proj.data(), i, W, H);
        proj[i] = p.proj[i];
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  if (seconds)
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return p.numVis ? (int)p.numVis - 1 : 0;
}
