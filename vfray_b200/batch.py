"""Batched form: many (mesh, camera, resolution) views rendered by one chain
of launches (vfr_batch_* in include/vfray.h), optionally captured as a CUDA
graph, with the traversal as one persistent launch pulling rays of every
view from one device work queue."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Job, RenderStats, Tuning, check, ptr

__all__ = ["BatchRenderer", "job"]


def job(mesh_id: int, W: int, H: int, mv=None, rgb8=None, rgba=None, steps=None) -> Job:
    """A vfr_job; outputs are device buffers (torch CUDA tensors) or None
    (then the batch owns its outputs when all three are None).  The job
    holds references to its output tensors, and a BatchRenderer holds its
    jobs, so the buffers outlive every launch (and captured graph) that
    writes them."""
    j = Job()
    j.mesh_id = mesh_id
    j.W = W
    j.H = H
    j.use_mv = 0 if mv is None else 1
    if mv is not None:
        m = np.ascontiguousarray(mv, np.float32).reshape(16)
        for k in range(16):
            j.mv[k] = float(m[k])
    j.rgb8_dev = None if rgb8 is None else rgb8.data_ptr()
    j.rgba_dev = None if rgba is None else rgba.data_ptr()
    j.steps_dev = None if steps is None else steps.data_ptr()
    j._keep = tuple(t for t in (rgb8, rgba, steps) if t is not None)
    return j


class BatchRenderer:
    """A batch on a Renderer's context.  ``jobs`` are vfr_job structures (see
    ``job``) or tuples (mesh_id, mv, W, H) rendered into outputs the batch
    owns."""

    def __init__(self, renderer, jobs, mode: int = _lib.MODE_REF, graph: bool = True):
        self.r = renderer
        self.lib = renderer.lib
        h = C.c_void_p()
        check(self.lib.vfr_batch_create(renderer.h, C.byref(h)), renderer.h, "vfr_batch_create")
        self.h = h
        self.mode = mode
        self.graph = graph
        self.set_jobs(jobs)

    def set_jobs(self, jobs):
        js = [j if isinstance(j, Job) else job(j[0], j[2], j[3], mv=j[1]) for j in jobs]
        self.jobs = js  # keeps each job's output tensors alive (job())
        arr = (Job * len(js))(*js)
        self._arr = arr
        check(self.lib.vfr_batch_set_jobs(self.h, arr, len(js), self.mode), self.r.h,
              "vfr_batch_set_jobs")
        self.captured = False

    def autotune(self, reps: int = 2) -> dict:
        """Pick the fastest knobs for this batch (kept on the renderer's
        context) and re-capture the graph."""
        t = Tuning()
        check(self.lib.vfr_batch_autotune(self.h, reps, C.byref(t)), self.r.h,
              "vfr_batch_autotune")
        self.captured = False
        self.prepare()
        return t.as_dict()

    def prepare(self):
        """Capture the chain as a CUDA graph (once)."""
        if self.graph and not self.captured:
            check(self.lib.vfr_batch_capture(self.h), self.r.h, "vfr_batch_capture")
            self.captured = True

    def run(self, *unused):
        """Enqueue the batch (asynchronous on the renderer's stream)."""
        check(self.lib.vfr_batch_run(self.h), self.r.h, "vfr_batch_run")

    def stats(self):
        """Wait; per-job stats as dicts.  Raises on a device status."""
        n = len(self.jobs)
        st = (RenderStats * n)()
        check(self.lib.vfr_batch_stats(self.h, st, n), self.r.h, "vfr_batch_stats")
        return [s.as_dict() for s in st]

    def output_ptrs(self, j: int):
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(self.lib.vfr_batch_output(self.h, j, C.byref(a), C.byref(b), C.byref(c)), self.r.h,
              "vfr_batch_output")
        return a.value, b.value, c.value

    def scratch_bytes(self) -> int:
        b = C.c_uint64()
        check(self.lib.vfr_batch_scratch_bytes(self.h, C.byref(b)), self.r.h,
              "vfr_batch_scratch_bytes")
        return int(b.value)

    def launches_per_run(self) -> int:
        # init, rotate, normalize, maxedge, visible, compact, prefix, raster,
        # raylist, prefix, traverse (composited: the raster replaced by two
        # bin passes, a two-kernel scan and the tile kernel)
        return 11 if self.mode == _lib.MODE_REF else 15

    def read(self, rgb8=None, rgba=None, steps=None):
        """Copy every job's outputs (concatenated in job order) into host
        buffers (numpy arrays or pinned torch tensors) and wait."""
        check(self.lib.vfr_batch_read(self.h, ptr(rgb8), ptr(rgba), ptr(steps)), self.r.h,
              "vfr_batch_read")

    def read_async(self, rgb8=None, rgba=None, steps=None):
        """The same copies, enqueued on the batch's stream without waiting
        (pinned host buffers; they hold the outputs after synchronize())."""
        check(self.lib.vfr_batch_read_async(self.h, ptr(rgb8), ptr(rgba), ptr(steps)), self.r.h,
              "vfr_batch_read_async")

    def synchronize(self):
        """Wait for everything enqueued on the batch's stream."""
        check(self.lib.vfr_batch_synchronize(self.h), self.r.h, "vfr_batch_synchronize")

    def set_stream(self, stream):
        """Run this batch on its own stream (a torch.cuda.Stream or a raw
        cudaStream_t handle; None: the renderer's stream again)."""
        handle = getattr(stream, "cuda_stream", stream)
        self._stream = stream  # alive while the batch uses it
        check(self.lib.vfr_batch_set_stream(self.h, C.c_void_p(handle) if handle else None),
              self.r.h, "vfr_batch_set_stream")

    def set_cameras(self, mv):
        """New model-views for every job, (njobs, 4, 4) row-major float32 in
        host memory (a numpy array or a pinned torch tensor): copied to the
        device asynchronously; the next run renders with them.  The buffer
        must stay unchanged until the next read or synchronize."""
        if hasattr(mv, "data_ptr"):
            assert mv.dtype.is_floating_point and mv.element_size() == 4 and mv.is_contiguous()
            assert mv.numel() == 16 * len(self.jobs)
            p = C.c_void_p(mv.data_ptr())
        else:
            mv = np.ascontiguousarray(mv, np.float32).reshape(len(self.jobs), 16)
            self._cams = mv  # alive until the copy has run
            p = ptr(mv)
        check(self.lib.vfr_batch_set_cameras(self.h, p, len(self.jobs)), self.r.h,
              "vfr_batch_set_cameras")

    def run_host(self, rgb8_host, cameras=None):
        """The host-buffer form: cameras in (optional, see set_cameras), run,
        then every job's RGB8 back into ``rgb8_host`` (pinned host memory
        gives full copy bandwidth)."""
        if cameras is not None:
            self.set_cameras(cameras)
        self.run()
        self.read(rgb8=rgb8_host)

    def close(self):
        if getattr(self, "h", None):
            self.lib.vfr_batch_destroy(self.h)  # safe after the renderer closed too
            self.h = None

    def __del__(self):
        self.close()
