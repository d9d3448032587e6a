"""Test infrastructure: Python bindings for the CPU oracle and the reference.

* ``Oracle``: the C restatement of the reference's CPU render path
  (oracle/vfr_oracle.c, built into oracle/_bin/liboracle.so).
* ``Reference``: the reference's own CPU kernels and precomputation
  (vfRayKernelCPU.cc, vfRayPreComp.cc) compiled from the reference sources
  behind our harness (oracle/ref_harness.cc) into oracle/_ref/.

Only the tests, the smoke check and the benchmark's CPU-baseline legs use this
package, and only as the checker or as the timed CPU baseline.  The
vfray_b200 product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_bin", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
# the reference sources (only present where the oracle is built from them)
REF_SOURCES = os.environ.get("VFRAY_REF", "/root/reference")

_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


def build(reference: bool = True) -> None:
    """Compile the oracle, and the reference harness when the reference
    sources are present (they are not on the GPU box, where the prebuilt
    libraries are used)."""
    targets = ["oracle"]
    if reference and os.path.isdir(REF_SOURCES):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"VFRAY_REF={REF_SOURCES}", *targets], check=True)


def ref_available(variant: str = "strict") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libvfref_{variant}.so"))


def _opt(a, dtype):
    if a is None:
        return None
    assert a.dtype == dtype and a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


class _VoMesh(C.Structure):
    _fields_ = [("vert", C.c_void_p), ("tet", C.c_void_p), ("con", C.c_void_p),
                ("extf", C.c_void_p), ("nV", C.c_uint32), ("nT", C.c_uint32),
                ("nExt", C.c_uint32), ("tf", C.c_void_p), ("psi", C.c_void_p),
                ("maxEdge", C.c_float), ("step_cap", C.c_uint32)]


class Oracle:
    """The C restatement; every call takes the mesh arrays explicitly."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(reference=False)
        self.lib = C.CDLL(path)
        L = self.lib
        for name in ("vo_render_ref", "vo_winners", "vo_trace_pixels", "vo_render_composited",
                     "vo_render_ref_fp64"):
            getattr(L, name).restype = C.c_int
        L.vo_compact.restype = C.c_uint32

    @staticmethod
    def mesh(vert, tet, con, extf, tf, psi, max_edge, step_cap=0):
        arrs = [np.ascontiguousarray(vert, np.float32), np.ascontiguousarray(tet, np.uint32),
                np.ascontiguousarray(con, np.uint32), np.ascontiguousarray(extf, np.uint32),
                np.ascontiguousarray(tf, np.float32), np.ascontiguousarray(psi, np.float32)]
        m = _VoMesh(arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data,
                    arrs[3].ctypes.data, arrs[0].size // 4, arrs[1].size // 4,
                    arrs[3].size // 2, arrs[4].ctypes.data, arrs[5].ctypes.data,
                    float(max_edge), int(step_cap))
        m._keep = arrs
        return m

    def find_visible(self, m):
        faces = np.zeros((m.nExt, 6), np.float32)
        self.lib.vo_find_visible(C.byref(m), faces.ctypes.data_as(C.c_void_p))
        vis = np.zeros(max(m.nExt, 1), np.uint32)
        n = self.lib.vo_compact(faces.ctypes.data_as(C.c_void_p), C.c_uint32(m.nExt),
                                vis.ctypes.data_as(C.c_void_p))
        return faces, vis[:n].copy()

    def project(self, m, vis, W, H):
        bb = np.zeros((len(vis), 4), np.uint32)
        v = np.ascontiguousarray(vis, np.uint32)
        self.lib.vo_project(C.byref(m), v.ctypes.data_as(C.c_void_p), C.c_uint32(len(v)),
                            C.c_uint32(W), C.c_uint32(H), bb.ctypes.data_as(C.c_void_p))
        return bb

    def render_ref(self, m, W, H):
        """Reference-order render: dict of rgb8, rgba, writer, steps,
        face_comp, face_abandon, nvis."""
        rgb = np.zeros((H, W, 3), np.uint8)
        rgba = np.zeros((H, W, 4), np.float32)
        wr = np.zeros((H, W), np.int32)
        st = np.zeros((H, W), np.uint32)
        fc = np.zeros(max(m.nExt, 1), np.uint64)
        fa = np.zeros(max(m.nExt, 1), np.uint8)
        n = self.lib.vo_render_ref(C.byref(m), C.c_uint32(W), C.c_uint32(H), _opt(rgb, np.uint8),
                                   _opt(rgba, np.float32), _opt(wr, np.int32), _opt(st, np.uint32),
                                   _opt(fc, np.uint64), _opt(fa, np.uint8))
        if n < 0:
            raise ValueError("oracle rejected the mesh")
        return dict(rgb8=rgb, rgba=rgba, writer=wr, steps=st, face_comp=fc[:n],
                    face_abandon=fa[:n], nvis=n)

    def render_ref_fp64(self, m, W, H):
        """FP64 rerun of render_ref along the same traversal: (H, W, 4)
        float64 clamped colour + alpha of each pixel's writing ray."""
        out = np.zeros((H, W, 4), np.float64)
        n = self.lib.vo_render_ref_fp64(C.byref(m), C.c_uint32(W), C.c_uint32(H),
                                        out.ctypes.data_as(C.c_void_p))
        if n < 0:
            raise ValueError("oracle rejected the mesh")
        return out

    def winners(self, m, W, H):
        wr = np.zeros((H, W), np.int32)
        n = self.lib.vo_winners(C.byref(m), C.c_uint32(W), C.c_uint32(H), _opt(wr, np.int32))
        if n < 0:
            raise ValueError("oracle rejected the mesh")
        return wr

    def trace_pixels(self, m, W, H, pix, entry, threads=0):
        pix = np.ascontiguousarray(pix, np.uint32)
        entry = np.ascontiguousarray(entry, np.uint32)
        n = len(pix)
        rgb = np.zeros((n, 3), np.uint8)
        rgba = np.zeros((n, 4), np.float32)
        st = np.zeros(n, np.uint32)
        rc = self.lib.vo_trace_pixels(C.byref(m), C.c_uint32(W), C.c_uint32(H), C.c_uint32(n),
                                      _opt(pix, np.uint32), _opt(entry, np.uint32),
                                      _opt(rgb, np.uint8), _opt(rgba, np.float32),
                                      _opt(st, np.uint32), C.c_int(threads))
        if rc == -2:
            raise ValueError("oracle rejected the input")
        return dict(rgb8=rgb, rgba=rgba, steps=st, status=rc)

    def render_composited(self, m, W, H, threads=0):
        rgb = np.zeros((H, W, 3), np.uint8)
        rgba = np.zeros((H, W, 4), np.float32)
        st = np.zeros((H, W), np.uint32)
        ns = np.zeros((H, W), np.uint32)
        n = self.lib.vo_render_composited(C.byref(m), C.c_uint32(W), C.c_uint32(H),
                                          _opt(rgb, np.uint8), _opt(rgba, np.float32),
                                          _opt(st, np.uint32), _opt(ns, np.uint32),
                                          C.c_int(threads))
        return dict(rgb8=rgb, rgba=rgba, steps=st, nseg=ns, status=n)


class Reference:
    """The reference CPU path (its own kernels and precomputation) behind the
    harness.  variant: "strict" (IEEE), "fast" (the reference's -ffast-math
    flags) or "count" (strict + compositing-step counter)."""

    def __init__(self, variant: str = "strict"):
        path = os.path.join(REF_DIR, f"libvfref_{variant}.so")
        if not os.path.exists(path):
            build(reference=True)
        self.variant = variant
        self.lib = C.CDLL(path)
        L = self.lib
        for n in ("ref_num_verts", "ref_num_tets", "ref_num_ext"):
            getattr(L, n).restype = C.c_uint32
        L.ref_set_lmt.argtypes = [C.c_float, C.c_float, C.c_float]

    # --- state ---
    def set_mesh(self, vert, tet):
        v = np.ascontiguousarray(vert, np.float32)
        t = np.ascontiguousarray(tet, np.uint32)
        self.lib.ref_set_mesh(v.ctypes.data_as(C.c_void_p), C.c_uint32(v.size // 4),
                              t.ctypes.data_as(C.c_void_p), C.c_uint32(t.size // 4))

    def set_vert(self, vert):
        """Replace the vertices (same count as the current mesh)."""
        v = np.ascontiguousarray(vert, np.float32)
        assert v.size == 4 * self.lib.ref_num_verts()
        self.lib.ref_set_vert(v.ctypes.data_as(C.c_void_p))

    def vert(self):
        out = np.zeros((self.lib.ref_num_verts(), 4), np.float32)
        self.lib.ref_get_vert(out.ctypes.data_as(C.c_void_p))
        return out

    def normalize(self):
        self.lib.ref_normalize()

    def rotate(self, mv):
        m = np.ascontiguousarray(mv, np.float32).reshape(16)
        self.lib.ref_rotate(m.ctypes.data_as(C.c_void_p))

    def build_con(self):
        if self.lib.ref_build_con() != 0:
            raise RuntimeError("reference incidence/adjacency build failed")

    def build_extf(self):
        self.lib.ref_build_extf()

    def build_lmt(self):
        self.lib.ref_build_lmt()

    def build_tf(self):
        self.lib.ref_build_tf()

    def con(self):
        out = np.zeros((self.lib.ref_num_tets(), 4), np.uint32)
        self.lib.ref_get_con(out.ctypes.data_as(C.c_void_p))
        return out, int(self.lib.ref_num_ext())

    def extf(self):
        out = np.zeros((self.lib.ref_num_ext(), 2), np.uint32)
        self.lib.ref_get_extf(out.ctypes.data_as(C.c_void_p))
        return out

    def lmt(self):
        out = np.zeros(3, np.float32)
        self.lib.ref_get_lmt(out.ctypes.data_as(C.c_void_p))
        return out

    def tf(self):
        out = np.zeros((256, 4), np.float32)
        self.lib.ref_get_tf(out.ctypes.data_as(C.c_void_p))
        return out

    def set_con(self, con, n_ext):
        c = np.ascontiguousarray(con, np.uint32)
        self.lib.ref_set_con(c.ctypes.data_as(C.c_void_p), C.c_uint32(n_ext))

    def set_extf(self, extf):
        e = np.ascontiguousarray(extf, np.uint32)
        self.lib.ref_set_extf(e.ctypes.data_as(C.c_void_p), C.c_uint32(e.size // 2))

    def set_lmt(self, max_edge, max_z, min_z):
        self.lib.ref_set_lmt(max_edge, max_z, min_z)

    def set_tf(self, tf):
        t = np.ascontiguousarray(tf, np.float32)
        self.lib.ref_set_tf(t.ctypes.data_as(C.c_void_p))

    def psi(self):
        out = np.zeros((512, 512), np.float32)
        self.lib.ref_get_psi(out.ctypes.data_as(C.c_void_p))
        return out

    def set_psi(self, psi):
        p = np.ascontiguousarray(psi, np.float32)
        self.lib.ref_set_psi(p.ctypes.data_as(C.c_void_p))

    # --- files ---
    def _io(self, fn, path):
        rc = getattr(self.lib, fn)(os.fsencode(path))
        if rc != 0:
            raise IOError(f"{fn}({path}) failed")

    def read_off(self, p): self._io("ref_read_off", p)
    def read_con(self, p): self._io("ref_read_con", p)
    def read_extf(self, p): self._io("ref_read_extf", p)
    def read_lmt(self, p): self._io("ref_read_lmt", p)
    def read_tf(self, p): self._io("ref_read_tf", p)
    def write_con(self, p): self._io("ref_write_con", p)
    def write_extf(self, p): self._io("ref_write_extf", p)
    def write_lmt(self, p): self._io("ref_write_lmt", p)
    def write_tf(self, p): self._io("ref_write_tf", p)

    # --- render ---
    def render(self, W, H, detect=True):
        """Reference render of the current state; with detect, also the
        per-pixel writer (ext index) and per-face compositing-step counts."""
        next_ = int(self.lib.ref_num_ext())
        img = np.zeros((H, W, 3), np.uint8)
        wr = np.zeros((H, W), np.int32) if detect else None
        vis = np.zeros(max(next_, 1), np.uint32)
        bb = np.zeros((max(next_, 1), 4), np.uint32)
        fe = np.zeros(max(next_, 1), np.uint64) if detect else None
        sec = C.c_double(0)
        n = self.lib.ref_render(C.c_uint32(W), C.c_uint32(H), img.ctypes.data_as(C.c_void_p),
                                _opt(wr, np.int32), vis.ctypes.data_as(C.c_void_p),
                                bb.ctypes.data_as(C.c_void_p), _opt(fe, np.uint64), C.byref(sec))
        if n < 0:
            raise RuntimeError("reference harness has incomplete state")
        out = dict(rgb8=img, vis=vis[:n].copy(), bbox=bb[:n].copy(), nvis=n, seconds=sec.value)
        if detect:
            out["writer"] = wr
            out["face_exp"] = fe[:n].copy()
        return out

    def render_mt(self, W, H, threads=0, strip=8):
        img = np.zeros((H, W, 3), np.uint8)
        sec = C.c_double(0)
        n = self.lib.ref_render_mt(C.c_uint32(W), C.c_uint32(H), img.ctypes.data_as(C.c_void_p),
                                   C.c_int(threads), C.c_int(strip), C.byref(sec))
        return dict(rgb8=img, nvis=n, seconds=sec.value)
