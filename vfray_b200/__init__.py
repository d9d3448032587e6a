"""vfray_b200: the VF-Ray render path (visible faces -> projection -> tet
traversal with partial pre-integration) as hand-written sm_100a kernels
behind a C ABI (include/vfray.h).

This module is the Python face of that ABI: host precomputation and files
(the reference's vfRayPreComp), and ``Renderer``, a context holding resident
meshes and tables on one GPU with the three stages of the reference's driver
(``find_visible`` = findVisibleFaces + compaction, ``project`` =
projectVisibleFaces + per-pixel entry faces, ``traverse`` = vfRay) plus the
one-call ``render``.  Batched and served forms live in ``vfray_b200.batch``
and ``vfray_b200.serve``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (MODE_COMPOSITED, MODE_REF, OPT_BLOCKS_PER_SM, OPT_PROFILE, OPT_RASTER_WARPS,
                   OPT_REFILL, OPT_STEP_CAP, OPT_TILE_WIDTH, OPT_TRAVERSE_VARIANT, RenderStats,
                   VfrError, check, load, ptr, VFR_DEV_CYCLE, VFR_DEV_OVERFLOW, VFR_DEV_QUEUE,
                   VFR_DEV_RANGE, VFR_DEV_STEP_CAP)

__all__ = [
    "Renderer", "VfrError", "MODE_REF", "MODE_COMPOSITED", "RenderStats", "load",
    "normalize", "rotate", "build_con", "build_extf", "build_lmt", "psi_table",
    "reference_psi_table", "default_tf",
    "prepare", "read_off", "read_con", "read_extf", "read_lmt", "read_tf", "write_off",
    "write_con", "write_extf", "write_lmt", "write_tf", "write_ppm", "read_psi_source",
    "write_mesh_cache", "read_mesh_cache", "clean_tf",
]


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


def _u32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    if shape is not None:
        a = a.reshape(shape)
    return a


# ---------------------------------------------------------------- precompute

def psi_table() -> np.ndarray:
    """The generated 512x512 psi(gamma) table, [front][back]."""
    out = np.empty((512, 512), np.float32)
    check(load().vfr_psi_table(ptr(out)), what="vfr_psi_table")
    return out


def reference_psi_table() -> np.ndarray:
    """The reference's own 512x512 psi table (psiGammaTable512.h), as the
    build converted it from the reference sources into
    vfray_b200/data/psiGammaTable512.bin (or the file $VFRAY_PSI_TABLE
    names); raises VfrError if the library was built without it."""
    out = np.empty((512, 512), np.float32)
    check(load().vfr_psi_table_reference(ptr(out)), what="vfr_psi_table_reference")
    return out


def default_tf() -> np.ndarray:
    """buildTF's 4-band default transfer function (vfRayPreComp.cc:595-622)."""
    out = np.empty((256, 4), np.float32)
    check(load().vfr_default_tf(ptr(out)), what="vfr_default_tf")
    return out


def normalize(vert) -> np.ndarray:
    """normalizeVertices (vfRayPreComp.cc:84-145) on a copy."""
    v = _f32(vert, (-1, 4)).copy()
    check(load().vfr_normalize(ptr(v), v.shape[0]), what="vfr_normalize")
    return v


def rotate(vert, mv) -> np.ndarray:
    """rotateVolume (vfRayPreComp.cc:886-906) on a copy; mv row-major 4x4."""
    v = _f32(vert, (-1, 4)).copy()
    m = _f32(mv, (16,))
    check(load().vfr_rotate(ptr(v), v.shape[0], ptr(m)), what="vfr_rotate")
    return v


def build_con(tet, n_vert: int, threads: int = 0):
    """buildIncid + buildCon (vfRayPreComp.cc:219-501): (con (nT,4), num_ext)."""
    t = _u32(tet, (-1, 4))
    con = np.empty_like(t)
    n = C.c_uint32()
    check(load().vfr_build_con(ptr(t), t.shape[0], n_vert, ptr(con), C.byref(n), threads),
          what="vfr_build_con")
    return con, int(n.value)


def build_extf(con) -> np.ndarray:
    """buildExtF (vfRayPreComp.cc:710-737): (nExt, 2) (tet, face), tet-then-face."""
    c = _u32(con, (-1, 4))
    n = C.c_uint32()
    L = load()
    check(L.vfr_build_extf(ptr(c), c.shape[0], None, 0, C.byref(n)), what="vfr_build_extf")
    out = np.empty((n.value, 2), np.uint32)
    check(L.vfr_build_extf(ptr(c), c.shape[0], ptr(out), n.value, C.byref(n)),
          what="vfr_build_extf")
    return out


def build_lmt(vert, tet) -> np.ndarray:
    """buildLmt (vfRayPreComp.cc:808-853): [maxEdgeLength, maxZ, minZ]."""
    v = _f32(vert, (-1, 4))
    t = _u32(tet, (-1, 4))
    out = np.empty(3, np.float32)
    check(load().vfr_build_lmt(ptr(v), v.shape[0], ptr(t), t.shape[0], ptr(out)),
          what="vfr_build_lmt")
    return out


def prepare(vert, tet, threads: int = 0) -> dict:
    """The load sequence of the reference driver (vfRay.cu:752-837) without
    files: normalizeVertices, buildCon, buildExtF, buildLmt."""
    v = normalize(vert)
    t = _u32(tet, (-1, 4))
    con, n_ext = build_con(t, v.shape[0], threads)
    extf = build_extf(con)
    assert extf.shape[0] == n_ext
    return dict(vert=v, tet=t, con=con, extf=extf, lmt=build_lmt(v, t))


# ---------------------------------------------------------------- files

def read_off(path):
    L = load()
    nv, nt = C.c_uint32(), C.c_uint32()
    check(L.vfr_read_off(path.encode(), None, C.byref(nv), None, C.byref(nt)), what=path)
    v = np.empty((nv.value, 4), np.float32)
    t = np.empty((nt.value, 4), np.uint32)
    check(L.vfr_read_off(path.encode(), ptr(v), C.byref(nv), ptr(t), C.byref(nt)), what=path)
    return v, t


def read_con(path):
    L = load()
    nt, ne = C.c_uint32(), C.c_uint32()
    check(L.vfr_read_con(path.encode(), None, C.byref(nt), C.byref(ne)), what=path)
    c = np.empty((nt.value, 4), np.uint32)
    check(L.vfr_read_con(path.encode(), ptr(c), C.byref(nt), C.byref(ne)), what=path)
    return c, int(ne.value)


def read_extf(path):
    L = load()
    n = C.c_uint32()
    check(L.vfr_read_extf(path.encode(), None, C.byref(n)), what=path)
    e = np.empty((n.value, 2), np.uint32)
    check(L.vfr_read_extf(path.encode(), ptr(e), C.byref(n)), what=path)
    return e


def read_lmt(path):
    out = np.empty(3, np.float32)
    check(load().vfr_read_lmt(path.encode(), ptr(out)), what=path)
    return out


def read_tf(path):
    out = np.empty((256, 4), np.float32)
    check(load().vfr_read_tf(path.encode(), ptr(out)), what=path)
    return out


def read_psi_source(path):
    out = np.empty((512, 512), np.float32)
    check(load().vfr_read_psi_source(path.encode(), ptr(out)), what=path)
    return out


def clean_tf(in_path, out_path):
    """cleanTF: the old transfer-function layout to the .tf layout."""
    check(load().vfr_clean_tf(in_path.encode(), out_path.encode()), what=in_path)


def write_mesh_cache(path, p):
    """Write a prepared mesh (dict of vert, tet, con, extf, lmt as from
    ``prepare``) to the binary cache."""
    v, t, c = _f32(p["vert"], (-1, 4)), _u32(p["tet"], (-1, 4)), _u32(p["con"], (-1, 4))
    e, lm = _u32(p["extf"], (-1, 2)), _f32(p["lmt"], (3,))
    check(load().vfr_write_mesh_cache(path.encode(), ptr(v), v.shape[0], ptr(t), ptr(c),
                                      t.shape[0], ptr(e), e.shape[0], ptr(lm)), what=path)


def read_mesh_cache(path) -> dict:
    """A prepared mesh back from the binary cache (the dict ``prepare`` gives)."""
    L = load()
    nv, nt, ne = C.c_uint32(), C.c_uint32(), C.c_uint32()
    check(L.vfr_read_mesh_cache(path.encode(), None, C.byref(nv), None, None, C.byref(nt), None,
                                C.byref(ne), None), what=path)
    v = np.empty((nv.value, 4), np.float32)
    t = np.empty((nt.value, 4), np.uint32)
    c = np.empty((nt.value, 4), np.uint32)
    e = np.empty((ne.value, 2), np.uint32)
    lm = np.empty(3, np.float32)
    check(L.vfr_read_mesh_cache(path.encode(), ptr(v), C.byref(nv), ptr(t), ptr(c), C.byref(nt),
                                ptr(e), C.byref(ne), ptr(lm)), what=path)
    return dict(vert=v, tet=t, con=c, extf=e, lmt=lm)


def write_off(path, vert, tet):
    v, t = _f32(vert, (-1, 4)), _u32(tet, (-1, 4))
    check(load().vfr_write_off(path.encode(), ptr(v), v.shape[0], ptr(t), t.shape[0]), what=path)


def write_con(path, con, num_ext):
    c = _u32(con, (-1, 4))
    check(load().vfr_write_con(path.encode(), ptr(c), c.shape[0], num_ext), what=path)


def write_extf(path, extf):
    e = _u32(extf, (-1, 2))
    check(load().vfr_write_extf(path.encode(), ptr(e), e.shape[0]), what=path)


def write_lmt(path, lmt):
    check(load().vfr_write_lmt(path.encode(), ptr(_f32(lmt, (3,)))), what=path)


def write_tf(path, tf):
    check(load().vfr_write_tf(path.encode(), ptr(_f32(tf, (256, 4)))), what=path)


def write_ppm(path, rgb8):
    a = np.ascontiguousarray(rgb8, np.uint8)
    h, w = a.shape[:2]
    check(load().vfr_write_ppm(path.encode(), ptr(a), w, h), what=path)


# ---------------------------------------------------------------- renderer

class Renderer:
    """A vfr context on one GPU: resident tables and meshes, one stream."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.vfr_create(C.byref(h), device), what="vfr_create")
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.vfr_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        check(rc, self.h, what)

    def set_stream(self, stream):
        """Run on a caller's CUDA stream (a torch.cuda.Stream or a raw handle)."""
        handle = getattr(stream, "cuda_stream", stream)
        self._check(self.lib.vfr_set_stream(self.h, C.c_void_p(handle or 0)), "vfr_set_stream")

    def synchronize(self):
        self._check(self.lib.vfr_synchronize(self.h), "vfr_synchronize")

    def set_option(self, option: int, value: int):
        self._check(self.lib.vfr_set_option(self.h, option, int(value)), "vfr_set_option")

    def profile_read(self, cap: int = 4096) -> np.ndarray:
        """Per-view device ms of stages (a), (b), (c) since the last read
        (needs set_option(OPT_PROFILE, 1))."""
        out = np.empty((cap, 3), np.float32)
        n = C.c_int()
        self._check(self.lib.vfr_profile_read(self.h, ptr(out), cap, C.byref(n)),
                    "vfr_profile_read")
        return out[: n.value].copy()

    def upload_tables(self, tf, psi=None):
        """The transfer function and the psi table; psi None: the
        reference's own table (see reference_psi_table)."""
        tf = _f32(tf, (256, 4))
        psi = None if psi is None else _f32(psi, (512, 512))
        self._check(self.lib.vfr_tables_upload(self.h, ptr(tf), ptr(psi)), "vfr_tables_upload")

    def upload_mesh(self, vert, tet, con, extf, lmt) -> int:
        v, t, c = _f32(vert, (-1, 4)), _u32(tet, (-1, 4)), _u32(con, (-1, 4))
        e = _u32(extf, (-1, 2))
        lmt = np.asarray(lmt, np.float32).reshape(3)
        mid = C.c_int(-1)
        self._check(self.lib.vfr_mesh_upload(self.h, ptr(v), v.shape[0], ptr(t), ptr(c),
                                             t.shape[0], ptr(e), e.shape[0], float(lmt[0]),
                                             float(lmt[1]), float(lmt[2]), C.byref(mid)),
                    "vfr_mesh_upload")
        return mid.value

    def release_mesh(self, mesh_id: int):
        self._check(self.lib.vfr_mesh_release(self.h, mesh_id), "vfr_mesh_release")

    def mesh_bytes(self, mesh_id: int) -> int:
        b = C.c_uint64()
        self._check(self.lib.vfr_mesh_bytes(self.h, mesh_id, C.byref(b)), "vfr_mesh_bytes")
        return int(b.value)

    # --- the three stages (reference kernels 1-3) ---
    def find_visible(self, mesh_id: int, n_ext: int):
        """Stage (a): (visible ext-face indices in order, faceData (nExt,6))."""
        n = C.c_uint32()
        vis = np.empty(max(n_ext, 1), np.uint32)
        fd = np.empty((max(n_ext, 1), 6), np.float32)
        self._check(self.lib.vfr_find_visible(self.h, mesh_id, C.byref(n), ptr(vis), ptr(fd)),
                    "vfr_find_visible")
        return vis[: n.value].copy(), fd[:n_ext]

    def project(self, mesh_id: int, W: int, H: int, n_vis: int):
        """Stage (b): (bbox (nVis,4), writer (H,W) ext-face index or -1)."""
        bb = np.empty((max(n_vis, 1), 4), np.uint32)
        wr = np.empty((H, W), np.int32)
        self._check(self.lib.vfr_project(self.h, mesh_id, W, H, ptr(bb), ptr(wr)), "vfr_project")
        return bb[:n_vis], wr

    def traverse(self, mesh_id: int, W: int, H: int, rgba=True, steps=True):
        """Stage (c): dict(rgb8, rgba, steps, stats)."""
        rgb = np.empty((H, W, 3), np.uint8)
        fa = np.empty((H, W, 4), np.float32) if rgba else None
        st = np.empty((H, W), np.uint32) if steps else None
        stats = RenderStats()
        self._check(self.lib.vfr_traverse(self.h, mesh_id, ptr(rgb), ptr(fa), ptr(st),
                                          C.byref(stats)), "vfr_traverse")
        return dict(rgb8=rgb, rgba=fa, steps=st, stats=stats.as_dict())

    def render(self, mesh_id: int, W: int, H: int, mv=None, mode: int = MODE_REF, rgba=True,
               steps=True):
        """All three stages; mv: optional 4x4 model-view (rotate + normalise +
        limits of the view on the device)."""
        m = None if mv is None else _f32(mv, (16,))
        rgb = np.empty((H, W, 3), np.uint8)
        fa = np.empty((H, W, 4), np.float32) if rgba else None
        st = np.empty((H, W), np.uint32) if steps else None
        stats = RenderStats()
        self._check(self.lib.vfr_render(self.h, mesh_id, ptr(m), W, H, mode, ptr(rgb), ptr(fa),
                                        ptr(st), C.byref(stats)), "vfr_render")
        return dict(rgb8=rgb, rgba=fa, steps=st, stats=stats.as_dict())

    def render_into_host(self, mesh_id: int, W: int, H: int, rgb8: np.ndarray, mv=None,
                         mode: int = MODE_REF):
        """The drop-in host call: RGB8 written into the caller's (ideally
        pinned) buffer; returns the stats."""
        assert rgb8.dtype == np.uint8 and rgb8.flags.c_contiguous and rgb8.size == W * H * 3
        m = None if mv is None else _f32(mv, (16,))
        stats = RenderStats()
        self._check(self.lib.vfr_render(self.h, mesh_id, ptr(m), W, H, mode, ptr(rgb8), None,
                                        None, C.byref(stats)), "vfr_render")
        return stats.as_dict()

    def render_device(self, mesh_id: int, W: int, H: int, mv=None, mode: int = MODE_REF,
                      rgb8=None, rgba=None, steps=None, writer=None):
        """Asynchronous render into device buffers (torch CUDA tensors)."""
        m = None if mv is None else _f32(mv, (16,))
        self._check(self.lib.vfr_render_device(self.h, mesh_id, ptr(m), W, H, mode, ptr(rgb8),
                                               ptr(rgba), ptr(steps), ptr(writer)),
                    "vfr_render_device")

    def device_status(self) -> int:
        s = C.c_uint32()
        self._check(self.lib.vfr_device_status(self.h, C.byref(s)), "vfr_device_status")
        return int(s.value)
