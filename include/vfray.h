/* vfray_b200: the VF-Ray render path on B200 (sm_100a), behind a C ABI.
 *
 * Plain pointers and sizes only.  Every entry point returns an int status
 * (VFR_OK = 0, negative on error) and never aborts; vfr_last_error() gives the
 * message of the last failure on a context.  A context is used by one host
 * thread at a time; all GPU work of a context is ordered on its stream.
 *
 * The array layouts at this boundary are the reference's own
 * (vfRayKernelCPU.h:61-80, vfRayPreComp.h:83-94): vertices are float4
 * (x, y, z, s), tets are uint4 vertex ids, the adjacency `conTet` is uint4
 * neighbour ids with the tet's own id marking a boundary face, external faces
 * are uint2 (tet, face), where face f of a tet is its vertices
 * (f, f+1, f+2) mod 4.  The transfer function is 256 x RGBA float and the
 * partial pre-integration table is 512 x 512 float indexed [front][back]
 * (psiGammaTable512.h:10-20).  Images are row-major with row = pixel y,
 * RGB8 as the reference writes them (vfRayKernelCPU.cc:550-552).
 */
#ifndef VFRAY_H
#define VFRAY_H

#include <stdint.h>

#if defined(__GNUC__)
#define VFR_API __attribute__((visibility("default")))
#else
#define VFR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define VFR_OK 0
#define VFR_ERR_INVALID (-1)  /* bad argument or size */
#define VFR_ERR_CUDA (-2)     /* CUDA runtime error */
#define VFR_ERR_MESH (-3)     /* mesh failed validation */
#define VFR_ERR_NOMEM (-4)    /* device or host allocation failed */
#define VFR_ERR_DEVICE (-5)   /* a kernel reported an error in the status word */
#define VFR_ERR_STATE (-6)    /* call out of order / unknown handle */
#define VFR_ERR_IO (-7)       /* file could not be read or written */
#define VFR_ERR_BUDGET (-8)   /* request exceeds the memory budget */
#define VFR_ERR_TIMEOUT (-9)  /* a bounded device wait gave up */

/* Device status word bits (vfr_render_stats.device_status).  Bit 1 is not
 * used: a mesh whose adjacency does not point back, on which the reference
 * abandons the rest of a face (vfRayKernelCPU.cc:359-365), is refused at
 * upload instead (VFR_ERR_MESH). */
#define VFR_DEV_STEP_CAP 2u   /* a ray hit the per-ray step cap (VFR_OPT_STEP_CAP) */
#define VFR_DEV_RANGE 4u      /* an id read on the device was out of range: reported by the
                                 checked build (libvfray_b200_checked.so, -DVFR_CHECKED),
                                 which compares every id a kernel reads with the extent it
                                 indexes; the product build relies on the upload's
                                 validation and does not compare */
#define VFR_DEV_QUEUE 8u      /* a bounded wait of the served kernel for work gave up */
#define VFR_DEV_OVERFLOW 16u  /* an entry list exceeded its capacity */
#define VFR_DEV_CYCLE 32u     /* a ray's walk came back to a (tet, entry face) state it had
                                 left: the reference's loop would never end; the pixel keeps
                                 what the ray composited before it was stopped */

/* Options (vfr_set_option).  Number 2 is not used. */
#define VFR_OPT_STEP_CAP 1        /* per-ray tet-walk cap; 0 = 4*nT + 64 (default) */
#define VFR_OPT_BLOCKS_PER_SM 3   /* traversal CTAs per SM; 0 = occupancy maximum */
#define VFR_OPT_PROFILE 4         /* 1: record per-stage CUDA events of every view */
#define VFR_OPT_TRAVERSE_VARIANT 5 /* traversal register budget: 0 = 2 CTAs/SM, 1 = 3 CTAs/SM (1) */
#define VFR_OPT_REFILL 6          /* queue chunk: a warp takes rays from the work queue once at
                                     least this many of its lanes are idle, one per idle lane (4) */
#define VFR_OPT_RASTER_WARPS 7    /* stage (b) warps per SM (64) */
#define VFR_OPT_TILE_WIDTH 8      /* ray-list screen tile width: 4, 8, 16, 32 (4 = 4x8) */

/* Render modes. */
#define VFR_MODE_REF 0        /* reference semantics: last visible face wins each pixel */
#define VFR_MODE_COMPOSITED 1 /* depth-ordered entry lists; segments composited */

typedef struct vfr_ctx vfr_ctx;

typedef struct {
  uint32_t num_ext;        /* external faces */
  uint32_t num_vis;        /* visible faces (without the reference's padding duplicate) */
  uint32_t num_rays;       /* pixels with an entry face */
  uint32_t num_entries;    /* entry-list entries (composited mode) */
  uint64_t num_steps;      /* tet-walk iterations over all rays */
  uint32_t device_status;  /* VFR_DEV_* bits */
  float ms_visible;        /* stage (a) device time */
  float ms_project;        /* stage (b) device time */
  float ms_traverse;       /* stage (c) device time */
  float ms_total;          /* all three, device time */
} vfr_render_stats;

/* ---- context ---------------------------------------------------------- */

/* Replaces the reference's initCUDA (vfRay.cu:256-288) and its globals
 * (vfRay.cu:110-151): one context per device. */
VFR_API int vfr_create(vfr_ctx** ctx, int device);
VFR_API void vfr_destroy(vfr_ctx* ctx);
VFR_API const char* vfr_last_error(const vfr_ctx* ctx);
VFR_API const char* vfr_status_string(int status);
/* Use a caller-owned cudaStream_t (NULL: the context's own stream). */
VFR_API int vfr_set_stream(vfr_ctx* ctx, void* stream);
VFR_API int vfr_synchronize(vfr_ctx* ctx);
/* Set a VFR_OPT_* option (negative values are invalid). */
VFR_API int vfr_set_option(vfr_ctx* ctx, int option, int64_t value);
/* With VFR_OPT_PROFILE on: per-view device times in ms of stage (a), (b)
 * and (c) of the views enqueued since the last call, 3 floats per view, in
 * order (waits for them); *count = views returned (at most cap). */
VFR_API int vfr_profile_read(vfr_ctx* ctx, float* ms3, int cap, int* count);

/* ---- tables (vfRay.cu:266-285 uploads the TF and the psi cudaArray) ---- */

/* tf256x4: 256 RGBA entries (vfRayPreComp.cc:551-579 reads them).
 * psi512x512: the psi(gamma) table, [front][back]; NULL selects the
 * reference's own table (vfr_psi_table_reference), and fails with
 * VFR_ERR_IO where the library was built without it -- pass the table this
 * library generates (vfr_psi_table) there. */
VFR_API int vfr_tables_upload(vfr_ctx* ctx, const float* tf256x4, const float* psi512x512);

/* ---- meshes ------------------------------------------------------------ */

/* Replaces prepareDevice1 + the initCUDA uploads (vfRay.cu:256-307).  The
 * arrays are copied; the mesh stays resident until released.  Validates ids,
 * adjacency symmetry and the external-face list (VFR_ERR_MESH on failure:
 * the reference would walk such a mesh into its :365 `return`, which
 * abandons the rest of a face; this library refuses the mesh instead).
 * maxZ/minZ are accepted for the .lmt layout; only maxEdge enters the
 * render, and it must be below 2^80 (VFR_ERR_INVALID otherwise; a
 * normalised mesh has at most 2 sqrt 3).  At most 2^27 vertices and fewer
 * than 2^30 tets. */
VFR_API int vfr_mesh_upload(vfr_ctx* ctx, const float* vert4, uint32_t nV, const uint32_t* tet4,
                    const uint32_t* con4, uint32_t nT, const uint32_t* extf2, uint32_t nExt,
                    float maxEdge, float maxZ, float minZ, int* mesh_id);
VFR_API int vfr_mesh_release(vfr_ctx* ctx, int mesh_id);
/* Device bytes the mesh holds (records, vertices, external faces). */
VFR_API int vfr_mesh_bytes(vfr_ctx* ctx, int mesh_id, uint64_t* bytes);

/* ---- the three stages, one view --------------------------------------- */

/* Stage (a): findVisibleFaces + compaction (vfRayKernel.cu:70-168 and the
 * host loop vfRay.cu:345-404; CPU twin vfRayKernelCPU.cc:51-132, main.cc:73-146).
 * Optional host outputs: visExt (ext-face index of each visible face in
 * order, capacity nExt), faceData (nExt x 6 floats: zParams, sParams, with
 * sParams.x = -1 marking back faces exactly as the reference does). */
VFR_API int vfr_find_visible(vfr_ctx* ctx, int mesh_id, uint32_t* num_vis, uint32_t* visExt,
                     float* faceData);

/* Stage (b): projectVisibleFaces + per-pixel entry faces (vfRayKernel.cu:171-228;
 * CPU vfRayKernelCPU.cc:136-169, main.cc:164-182).  Needs stage (a) of the
 * same mesh first.  Optional host outputs: bbox (4 per visible face:
 * xmin, ymin, xmax, ymax) and writer (W*H ext-face index of the face whose
 * ray the reference writes last at each pixel, -1 for none). */
VFR_API int vfr_project(vfr_ctx* ctx, int mesh_id, uint32_t W, uint32_t H, uint32_t* bbox,
                int32_t* writer);

/* Stage (c): traversal + compositing (vfRayKernel.cu:231-852; CPU
 * vfRayKernelCPU.cc:173-566).  Needs stage (b) first.  Optional host
 * outputs: rgb8 (W*H*3), rgba (W*H*4 float: clamped colour, alpha = 1 - prod
 * zeta), steps (W*H tet-walk iterations of each pixel's ray). */
VFR_API int vfr_traverse(vfr_ctx* ctx, int mesh_id, uint8_t* rgb8, float* rgba, uint32_t* steps,
                 vfr_render_stats* stats);

/* All three stages of one view in one call, host outputs (any may be NULL).
 * mv16: optional row-major 4x4 model-view applied as rotateVolume +
 * normalizeVertices + buildLmt of the view on the device (vfRayPreComp.cc:84-145,
 * 808-853, 886-906); NULL renders the mesh as uploaded with its uploaded
 * maxEdge.  mode: VFR_MODE_REF or VFR_MODE_COMPOSITED. */
VFR_API int vfr_render(vfr_ctx* ctx, int mesh_id, const float* mv16, uint32_t W, uint32_t H, int mode,
               uint8_t* rgb8, float* rgba, uint32_t* steps, vfr_render_stats* stats);

/* Same, but asynchronous on the context stream with device outputs (any may
 * be NULL); stats are not filled.  Call vfr_synchronize, then
 * vfr_device_status, before reading the outputs. */
VFR_API int vfr_render_device(vfr_ctx* ctx, int mesh_id, const float* mv16, uint32_t W, uint32_t H,
                      int mode, uint8_t* rgb8_dev, float* rgba_dev, uint32_t* steps_dev,
                      int32_t* writer_dev);
VFR_API int vfr_device_status(vfr_ctx* ctx, uint32_t* status);

/* ---- batches: many (mesh, camera, resolution) views in one launch chain -- */

/* No single counterpart in the reference, whose driver renders one view per
 * call (vfRay.cu:618-641 re-runs the three kernels for each rotation).  A
 * batch lays out all jobs in shared device arenas; each stage is one launch
 * over all jobs, and the traversal is one persistent launch whose warps take
 * rays of any job from one device work queue.  The chain can be captured
 * once as a CUDA graph and replayed. */
typedef struct {
  int mesh_id;
  uint32_t W, H;
  int use_mv;          /* 1: rotate + normalise + recompute the limits with mv */
  float mv[16];        /* row-major model-view (rotateVolume's layout) */
  uint8_t* rgb8_dev;   /* device outputs; all three NULL: the batch owns them */
  float* rgba_dev;
  uint32_t* steps_dev;
} vfr_job;

typedef struct vfr_batch vfr_batch;
VFR_API int vfr_batch_create(vfr_ctx* ctx, vfr_batch** out);
VFR_API void vfr_batch_destroy(vfr_batch* b);
/* Lays out (allocating) and uploads the jobs; mode is for all jobs. */
VFR_API int vfr_batch_set_jobs(vfr_batch* b, const vfr_job* jobs, uint32_t n, int mode);
/* Captures the whole chain as a CUDA graph; vfr_batch_run then replays it. */
VFR_API int vfr_batch_capture(vfr_batch* b);
/* Enqueues the batch on its stream (asynchronous): the context stream, or
 * the one vfr_batch_set_stream gave it. */
VFR_API int vfr_batch_run(vfr_batch* b);
/* Gives the batch a stream of its own (a cudaStream_t of the context's
 * device; NULL: the context stream again) for its runs, camera uploads,
 * reads and stats; waits first for what the batch's previous stream still
 * holds.  Two batches on two streams overlap: one's copies run beside the
 * other's kernels. */
VFR_API int vfr_batch_set_stream(vfr_batch* b, void* stream);
/* Waits, then fills per-job stats (n entries at most); returns the status. */
VFR_API int vfr_batch_stats(vfr_batch* b, vfr_render_stats* per_job, uint32_t n);
/* Device output pointers of a job (the batch's own when it owns them). */
VFR_API int vfr_batch_output(vfr_batch* b, uint32_t job, uint8_t** rgb8_dev, float** rgba_dev,
                             uint32_t** steps_dev);
/* Replaces the model-view of every job (n = the batch's job count): one
 * asynchronous host-to-device copy on the batch's stream of the first three
 * rows of each matrix, after which the next vfr_batch_run -- a replayed
 * graph included -- renders with the new cameras.  mv16: n row-major 4x4
 * matrices in host memory (pinned memory gives a full-speed copy), left
 * unchanged until the copy has run (vfr_batch_read or vfr_synchronize).
 * Only jobs given a model-view at vfr_batch_set_jobs (use_mv) use theirs. */
VFR_API int vfr_batch_set_cameras(vfr_batch* b, const float* mv16, uint32_t n);
/* Copies every job's outputs to host buffers, concatenated in job order
 * (any may be NULL), and waits: the host-buffer end of a batch.  Outputs
 * that lie back to back on the device (those the batch owns) come back in
 * one copy per kind. */
VFR_API int vfr_batch_read(vfr_batch* b, uint8_t* rgb8_host, float* rgba_host,
                           uint32_t* steps_host);
/* The same copies, enqueued on the batch's stream without waiting: the host
 * buffers (pinned memory, for the copies to be asynchronous) hold the
 * outputs once the stream has run them (vfr_batch_synchronize); the next
 * vfr_batch_run of this batch is ordered after them. */
VFR_API int vfr_batch_read_async(vfr_batch* b, uint8_t* rgb8_host, float* rgba_host,
                                 uint32_t* steps_host);
/* Waits for everything enqueued on the batch's stream. */
VFR_API int vfr_batch_synchronize(vfr_batch* b);
/* Autotuner: times stages (b) and (c) of the batch over a grid of the
 * knobs above (traversal register budget, refill threshold, traversal CTAs
 * per SM, ray-tile shape, stage (b) warps per SM), best of `reps` runs each,
 * keeps the fastest on the context and reports it.  Drops a captured graph
 * (capture again). */
typedef struct {
  uint32_t variant, refill, blocks_per_sm, tile_w, raster_warps_per_sm;
  float ms;  /* stages (b) + (c) of the batch with these knobs */
} vfr_tuning;
VFR_API int vfr_batch_autotune(vfr_batch* b, int reps, vfr_tuning* out);
/* Device bytes of the batch's scratch arenas. */
VFR_API int vfr_batch_scratch_bytes(vfr_batch* b, uint64_t* bytes);

/* ---- served form: a request loop with continuous batching -------------- */

/* No counterpart in the reference.  Requests over the context's resident
 * meshes are submitted from any thread.  One long-lived persistent
 * traversal launch (the drain) takes rays from every request admitted so
 * far: a worker thread admits pending requests in arrival order while their
 * memory footprint fits the budget, prepares them (stages a and b) on a
 * second stream beside the running drain, and publishes them into its work
 * table, so requests that arrive while others are on the GPU fold into the
 * running launch, frames of any size mixed.  When a request's last ray
 * ends, its image is copied to rgb8_host and its footprint released.
 * The budget covers the resident meshes of the context (counted once) and,
 * per request in flight, its view's scratch (view vertices, planes, visible
 * list, boxes, winner map or entry lists, ray list) and RGB8 image; the
 * server allocates that as one arena when it starts and nothing afterwards.
 * A request whose footprint can never fit is refused (VFR_ERR_BUDGET).
 * Upload the meshes before creating the server and release them after
 * destroying it; while the drain runs, calls on the same context that free
 * or grow device memory wait until it goes idle (about 50 ms after the last
 * request). */
typedef struct {
  int mesh_id;
  uint32_t W, H;
  int use_mv;
  float mv[16];
  int mode;             /* VFR_MODE_REF or VFR_MODE_COMPOSITED */
  uint8_t* rgb8_host;   /* W*H*3, written before the request completes; may be NULL */
} vfr_request;

typedef struct {
  int status;
  double t_submit_ms, t_start_ms, t_done_ms;  /* since the server started; start = admission */
  uint32_t batch_id, batch_jobs;               /* the admitted group it joined, its size */
  uint32_t num_rays;
  uint64_t num_steps;
  uint32_t device_status;                      /* VFR_DEV_* bits of its job */
  double t_ready_ms;   /* the worker saw its last ray finish, before the image copy */
} vfr_request_info;

typedef struct {
  uint32_t batches, pending;                   /* admitted groups so far; requests waiting */
  uint64_t completed, rejected, budget_used, rays, steps;
  uint32_t launches;        /* drain launches (a new one after each idle period) */
  uint32_t epochs;          /* arena restarts */
  uint32_t queue_timeouts;  /* drain launches whose bounded idle wait ran out (VFR_DEV_QUEUE) */
  uint64_t mesh_bytes;      /* resident mesh bytes counted against the budget */
  uint64_t arena_bytes;     /* the arena for requests in flight */
  double prep_ms;           /* device time of the finished groups' preparation (stages a, b) */
} vfr_server_counters;

typedef struct vfr_server vfr_server;
VFR_API int vfr_server_create(vfr_ctx* ctx, uint64_t budget_bytes, uint32_t max_batch,
                              vfr_server** out);
VFR_API int vfr_server_submit(vfr_server* s, const vfr_request* r, uint64_t* ticket);
/* Waits for a request (timeout_ms < 0: no limit; VFR_ERR_TIMEOUT if it runs
 * out), fills info, forgets the ticket; returns the request's status. */
VFR_API int vfr_server_wait(vfr_server* s, uint64_t ticket, int timeout_ms, vfr_request_info* info);
VFR_API int vfr_server_stats(vfr_server* s, vfr_server_counters* out);
/* Idle behaviour: the drain's bounded wait for new work (microseconds,
 * default 400000; when it runs out the drain sets VFR_DEV_QUEUE, leaves, and
 * is launched again with the next request) and how long the worker lets an
 * idle drain run before it stops it and starts a new arena epoch (default
 * 50 ms).  Applies from the next drain launch. */
VFR_API int vfr_server_set_idle(vfr_server* s, uint32_t drain_idle_us, uint32_t linger_ms);
/* Drains the admitted and pending requests, then stops. */
VFR_API void vfr_server_destroy(vfr_server* s);

/* ---- stage (a) for callers that cannot allocate ------------------------ */

/* No counterpart in the reference.  Stage (a) (findVisibleFaces + ordered
 * compaction) for callers that must not see the library allocate device
 * memory: an application that has reserved the GPU's memory for its own pool
 * (a game engine, a serving process with a fixed budget), or a frame loop in
 * which cudaMalloc/cudaFree, which may synchronise the device, must not run.
 * Inputs and outputs are the caller's device buffers (vert4_dev 16-byte
 * aligned nV x float4, tet4_dev 16-byte aligned nT x uint4, extf2_dev nExt x
 * uint2); writes visExt_dev (visible ext-face indices in order, capacity
 * nExt) and *num_vis_dev, asynchronously on `stream` (a cudaStream_t, NULL =
 * the default stream).  Its scratch is a fixed device array inside the
 * library (32 bytes per external face for up to VFR_STATIC_MAX_EXT faces,
 * about 8 MiB, held on every GPU that loads the library until exit); larger
 * meshes get VFR_ERR_BUDGET.  The array's device address belongs to the
 * current CUDA context: a call whose stream is not capturing looks it up in
 * that context, and a call under stream capture uses the address an earlier
 * call found in the same context (VFR_ERR_STATE if none did).  Calls share
 * the array: calls that overlap on the GPU race.  An external face whose ids
 * are out of range counts as not visible.  Output pointers must be 4-byte
 * aligned (VFR_ERR_INVALID).  Calls no cudaMalloc/cudaFree. */
#define VFR_STATIC_MAX_EXT (1u << 18)
VFR_API int vfr_find_visible_static(const float* vert4_dev, uint32_t nV, const uint32_t* tet4_dev,
                                    uint32_t nT, const uint32_t* extf2_dev, uint32_t nExt,
                                    uint32_t* visExt_dev, uint32_t* num_vis_dev, void* stream);

/* ---- host-side precomputation and files (vfRayPreComp.h:97-279) -------- */

/* The psi(gamma) table this library generates: psi(tf, tb) =
 * int_0^1 exp(-(tf*u + (tb - tf)*u^2/2)) du at gamma = i/512, tau =
 * gamma/(1-gamma), truncated to 7 decimals like psiGammaTable512.h. */
VFR_API int vfr_psi_table(float* out512x512);
/* The reference's own psi table (psiGammaTable512.h:10-20, which
 * vfRay.cu:280-284 uploads), as converted at build time from the reference
 * sources into data/psiGammaTable512.bin beside this library (with the
 * table's copyright notice in data/psiGammaTable512.NOTICE), or read from
 * the file $VFRAY_PSI_TABLE names.  VFR_ERR_IO if there is no such file. */
VFR_API int vfr_psi_table_reference(float* out512x512);
/* normalizeVertices (vfRayPreComp.cc:84-145), in place. */
VFR_API int vfr_normalize(float* vert4, uint32_t nV);
/* rotateVolume (vfRayPreComp.cc:886-906), in place; mv16 row-major. */
VFR_API int vfr_rotate(float* vert4, uint32_t nV, const float* mv16);
/* buildIncid + buildCon (vfRayPreComp.cc:219-501) by hashing sorted face
 * triples: the same neighbour ids, O(nT log nT).  con4: nT*4 out. */
VFR_API int vfr_build_con(const uint32_t* tet4, uint32_t nT, uint32_t nV, uint32_t* con4,
                  uint32_t* num_ext, int threads);
/* buildExtF (vfRayPreComp.cc:710-737): (tet, face) pairs, tet-then-face order. */
VFR_API int vfr_build_extf(const uint32_t* con4, uint32_t nT, uint32_t* extf2, uint32_t cap,
                   uint32_t* num_ext);
/* buildLmt (vfRayPreComp.cc:808-853): out3 = maxEdgeLength, maxZ, minZ. */
VFR_API int vfr_build_lmt(const float* vert4, uint32_t nV, const uint32_t* tet4, uint32_t nT,
                  float* out3);
/* buildTF (vfRayPreComp.cc:595-622): the 4-band default transfer function. */
VFR_API int vfr_default_tf(float* tf256x4);

/* Readers/writers in the reference text formats (vfRayPreComp.cc:29-880).
 * Readers are two-step: call with NULL buffers to get the sizes. */
VFR_API int vfr_read_off(const char* path, float* vert4, uint32_t* nV, uint32_t* tet4, uint32_t* nT);
VFR_API int vfr_read_con(const char* path, uint32_t* con4, uint32_t* nT, uint32_t* num_ext);
VFR_API int vfr_read_extf(const char* path, uint32_t* extf2, uint32_t* num_ext);
VFR_API int vfr_read_lmt(const char* path, float* out3);
VFR_API int vfr_read_tf(const char* path, float* tf256x4);
VFR_API int vfr_write_off(const char* path, const float* vert4, uint32_t nV, const uint32_t* tet4,
                  uint32_t nT);
VFR_API int vfr_write_con(const char* path, const uint32_t* con4, uint32_t nT, uint32_t num_ext);
VFR_API int vfr_write_extf(const char* path, const uint32_t* extf2, uint32_t num_ext);
VFR_API int vfr_write_lmt(const char* path, const float* in3);
VFR_API int vfr_write_tf(const char* path, const float* tf256x4);
/* ppmWrite (vfRayPreComp.cc:915-934): P6, RGB8. */
VFR_API int vfr_write_ppm(const char* path, const uint8_t* rgb8, uint32_t W, uint32_t H);
/* Parse a psiGammaTable512.h-style C source ("float name[512][512] = {...}"). */
VFR_API int vfr_read_psi_source(const char* path, float* out512x512);

/* cleanTF (cleanTF.cc:13-88): converts a transfer function in the old
 * layout (7 header lines, then 256 lines "index r g b a") into the .tf
 * layout, byte for byte as the reference tool writes it. */
VFR_API int vfr_clean_tf(const char* in_path, const char* out_path);

/* Binary mesh cache (no counterpart in the reference, which re-parses its
 * text files on every run, vfRay.cu:745-842): the normalised vertices, tets,
 * conTet, external faces and limits in one file, read back with a few
 * fread calls.  Reading is two-step like the text readers (NULL buffers:
 * sizes only); a file whose length does not match its header is refused
 * with VFR_ERR_IO. */
VFR_API int vfr_write_mesh_cache(const char* path, const float* vert4, uint32_t nV,
                                 const uint32_t* tet4, const uint32_t* con4, uint32_t nT,
                                 const uint32_t* extf2, uint32_t nExt, const float* lmt3);
VFR_API int vfr_read_mesh_cache(const char* path, float* vert4, uint32_t* nV, uint32_t* tet4,
                                uint32_t* con4, uint32_t* nT, uint32_t* extf2, uint32_t* nExt,
                                float* lmt3);

#ifdef __cplusplus
}
#endif
#endif
