// Device-side types shared by the kernels and the host code of the render
// library: per-view counters and the job table entry.
#pragma once
#include "vfr_device.cuh"

namespace vfr {

// Per-view device counters.
struct __align__(16) ViewCounters {
  uint32_t nvis;             // visible faces
  uint32_t nrays;            // rays of this job
  uint32_t nentries;         // entry-list entries (composited mode)
  uint32_t status;           // VFR_DEV_* bits
  unsigned long long steps;  // tet-walk iterations of this job's rays
  uint32_t maxedge_bits;     // view maxEdgeLength (float bits, >= 0)
  uint32_t rays_done;        // served form: rays of this job finished so far
  uint32_t mm[8];            // orderable min x y z s, max x y z s (view set-up)
  uint32_t nbins;            // composited: (face, screen tile) pairs of this job
};

// One job as the kernels see it (device memory, uploaded with the batch).
// A ray's start, written by stage (b) when it lists the rays: the pixel and,
// in reference mode, the winning face's tet and entry face (tet << 2 |
// face), the entry depth (float bits) and the back colour's
// transfer-function entry.  The traversal starts a ray from it without going
// back through the winner map, the face's plane and the external-face list.
struct __align__(16) RayStart {
  uint32_t p, tf, zp, cbi;
};

struct __align__(16) JobDev {
  float4 m0, m1, m2;         // rows of the model-view (use_mv)
  const uint4* tet;          // mesh
  const uint2* edges;        // the mesh's distinct edges (jobs with a model-view)
  uint32_t nEdges;
  const WalkRec* walk;
  const float4* vert_in;     // the mesh's (normalised) vertices
  const uint2* extf;
  const float4* vert;        // vertices this view renders with (vert_in or vview)
  float4* vview;             // rotated + normalised vertices (use_mv)
  float4* planes;            // kPlaneStride per external face
  uint32_t* blk;             // visible count per block of 1024 external faces
  uint32_t* vis_ext;         // visible external faces, in order
  uint4* bbox;               // per visible face
  int32_t* winner;           // W*H, reference mode
  RayStart* rays;            // W*H capacity
  uint32_t* ent_cnt;         // composited: W*H entry counts
  uint32_t* ent_off;         // composited: W*H offsets of the pixels' lists in ent
  const uint4* ent;          // composited: the batch's entry arena (z bits, ext face,
                             // tet << 2 | entry face, back-colour TF entry), each
                             // pixel's list in descending (depth, face) order
  uint32_t ent_cap;          // its capacity in entries
  ViewCounters* ctr;
  uint8_t* rgb8;             // outputs (any may be null)
  float4* rgba;
  uint32_t* steps;
  uint32_t nV, nT, nExt, W, H;
  uint32_t use_mv;
  float maxEdge_in;          // the mesh's maxEdgeLength when !use_mv
  uint32_t pix_base;         // first pixel of this job in the batch's pixel arenas
  uint32_t mode;             // VFR_MODE_REF or VFR_MODE_COMPOSITED
};

// Face planes per external face: three float4, (zx zy zz sx | sy sz v0x v0y |
// v1x v1y v2x v2y), the plane of findVisibleFaces (sx = -1: not visible) and
// the xy of the face's vertices for stage (b).
constexpr uint32_t kPlaneStride = 3;

struct TraverseParams {
  const JobDev* jobs;
  uint32_t njobs;
  const uint32_t* ray_pref;  // njobs + 1, exclusive prefix of the jobs' ray counts
  uint32_t* queue;           // work-queue head over all jobs' rays
  const float4* tf;          // 256 RGBA
  const float* psi;          // 512 x 512
  const double* e2tab;       // 2^(j/64), j = 0..63
  uint32_t step_cap;         // 0: 4 * nT + 64 of each job's mesh
  uint32_t refill;           // refill a warp's idle lanes once this many are idle
};

// ---- served form ----
//
// One long-lived persistent traversal launch draws rays from segments: each
// admitted mini-batch of render jobs, laid out in the server's arena, is
// prepared (stages a and b) on another stream while the launch runs and then
// published into the next entry of the segment table.  Within one launch an
// entry, and the arena memory its jobs use, is written once before its
// publication and never reused; the server starts a new epoch (table and
// arena from the start) only between launches.

struct SegDev {
  const JobDev* jobs;        // the segment's job table
  const uint32_t* ray_pref;  // njobs + 1, exclusive prefix of its jobs' ray counts
  uint32_t* done;            // per job, mapped host memory: set to 1 when its last ray ends
  uint32_t njobs;
  uint32_t nrays;            // ray_pref[njobs]
  uint32_t head;             // rays handed out so far (atomicAdd; may pass nrays)
  uint32_t pad;
};

struct ServeCtl {
  uint32_t published;        // entries of the segment table published in this epoch
  uint32_t status;           // VFR_DEV_QUEUE: an idle warp's bounded wait gave up
  uint32_t stop;             // the host asks idle warps to leave (copied in while the drain runs)
  uint32_t pad;
};

struct ServeParams {
  TraverseParams T;          // tables, step cap, refill (jobs, ray_pref, queue unused)
  SegDev* segs;
  ServeCtl* ctl;
  uint32_t idle_limit;       // microseconds an idle warp waits for new work before it gives up
  uint32_t first;            // the oldest entry with rays left when the launch starts
};

}  // namespace vfr
