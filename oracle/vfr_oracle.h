/* Test infrastructure: the CPU oracle for the VF-Ray render path.
 *
 * A plain-C restatement of the reference's CPU kernels
 * (vfRayKernelCPU.cc:50-566) and of the driver sequence around them
 * (main.cc:73-224), with the same float/double expression order.  It is
 * compiled without fast-math and without FMA contraction, so every operation
 * is one IEEE-rounded float or double operation, exactly as written.  The
 * parity tests check it against the reference build (oracle/_ref) and check
 * the CUDA path against it.  Only tests, the smoke check and the CPU
 * baseline leg of the benchmark load it; the product never does.
 */
#ifndef VFR_ORACLE_H
#define VFR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* faceData of vfRayKernelCPU.h:51-54: z = zx*x + zy*y + zz, s likewise. */
typedef struct { float zx, zy, zz, sx, sy, sz; } vo_face;

typedef struct {
  const float* vert;     /* nV x (x, y, z, s), normalised */
  const uint32_t* tet;   /* nT x 4 vertex ids */
  const uint32_t* con;   /* nT x 4 neighbour ids, self = boundary face */
  const uint32_t* extf;  /* nExt x (tet, face) */
  uint32_t nV, nT, nExt;
  const float* tf;       /* 256 x RGBA */
  const float* psi;      /* 512 x 512, [front][back] */
  float maxEdge;
  uint32_t step_cap;     /* per-ray iteration cap; 0 = 4 nT + 64 */
} vo_mesh;

/* Stage (a), vfRayKernelCPU.cc:51-132: plane coefficients and back-face
 * sentinel (sx == -1) for every external face. */
void vo_find_visible(const vo_mesh* m, vo_face* faces);
/* Host compaction, main.cc:93-138, without the padding duplicate: writes the
 * ext-face indices of the kept faces in order, returns their count. */
uint32_t vo_compact(const vo_face* faces, uint32_t nExt, uint32_t* visExt);
/* Stage (b), vfRayKernelCPU.cc:136-169: pixel bounding box per visible face. */
void vo_project(const vo_mesh* m, const uint32_t* visExt, uint32_t nVis,
                uint32_t W, uint32_t H, uint32_t* bbox4);

/* Every traversal below stops a ray whose walk comes back to a (tet, entry
 * face) state, checked from iteration 4096 on, or that reaches the step cap;
 * the reference's loop never ends on such a ray.  The ray keeps what it
 * composited before the stop, and its steps count the stopping iteration.
 *
 * Stage (c) in reference order (main.cc:209-218, vfRayKernelCPU.cc:173-566):
 * faces in visible order, each over its box, x outer / y inner, with the
 * column break on an out-of-range entry scalar (:274), the face abandon on
 * inconsistent adjacency (:365) and last-writer-wins per pixel.
 * Outputs (any may be NULL): rgb8 W*H*3 (zeroed first), rgba W*H*4 (clamped
 * colour + alpha = 1 - prod(zeta)), writer W*H (ext-face index, -1 none),
 * steps W*H (while-loop iterations of the writing ray), faceComp per visible
 * face (compositing steps over all of that face's rays), faceAbandon per
 * visible face (1 if the face hit the :365 return).
 * Returns the number of visible faces, or a negative value on bad input. */
int vo_render_ref(const vo_mesh* m, uint32_t W, uint32_t H, uint8_t* rgb8,
                  float* rgba, int32_t* writer, uint32_t* steps,
                  uint64_t* faceComp, uint8_t* faceAbandon);

/* FP64 rerun of vo_render_ref: the same faces, pixels, tet sequences and
 * decisions (all taken by the float traversal), with each ray's colour
 * recomputed in double along its path from the double pixel coordinate
 * (double planes, depths, tau, zeta, gamma, psi index and sum).  rgba64
 * W*H*4: clamped colour and 1 - prod(zeta) of the writing ray, 0 elsewhere.
 * Returns as vo_render_ref. */
int vo_render_ref_fp64(const vo_mesh* m, uint32_t W, uint32_t H, double* rgba64);

/* Per-pixel winner under the reference semantics for a mesh whose adjacency
 * is consistent: the last visible face (highest ext index) that writes the
 * pixel, honouring the column break.  writer W*H, -1 for none. */
int vo_winners(const vo_mesh* m, uint32_t W, uint32_t H, int32_t* writer);

/* Trace one ray per listed pixel from the given entry ext face, as the
 * reference does for the face that wins the pixel; threads <= 0 uses all
 * cores.  Outputs per listed pixel (any may be NULL): rgb8 (3), rgba (4),
 * steps.  Returns 0, or -1 if some ray hit inconsistent adjacency. */
int vo_trace_pixels(const vo_mesh* m, uint32_t W, uint32_t H, uint32_t n,
                    const uint32_t* pix, const uint32_t* entryExt, uint8_t* rgb8,
                    float* rgba, uint32_t* steps, int threads);

/* Depth-composited mode: every visible face that covers a pixel (entry
 * scalar in [0,1]) is an entry of that pixel's ray; entries are taken in
 * descending entry depth (ties: higher ext index first), an entry above the
 * depth where the previous segment left the mesh is skipped, and the
 * compositing sum runs on across segments with the back colour reset at
 * each entry.  Outputs as vo_render_ref, plus nseg W*H (segments traced);
 * steps counts iterations over all segments. */
int vo_render_composited(const vo_mesh* m, uint32_t W, uint32_t H, uint8_t* rgb8,
                         float* rgba, uint32_t* steps, uint32_t* nseg, int threads);

#ifdef __cplusplus
}
#endif
#endif
