"""Generate the golden fixtures of the render path from the reference itself.

Run in a container where the reference sources are present:

    python tests/golden/make_golden.py

Each case is a seeded synthetic mesh (vfray_b200.synth) precomputed by the
reference's own builders (buildIncid/buildCon/buildExtF/buildLmt through the
harness in oracle/ref_harness.cc) and rendered by the reference's own CPU
kernels (vfRayKernelCPU.cc, strict IEEE build) with the psi table that
vfray_b200 generates written into the reference's psiGammaTable array, so the
fixtures can be checked on a machine that has no reference sources.  Stored:
the inputs (small cases) or an input checksum (the 24^3 case, regenerated from
its seeds), and the reference outputs: RGB8 image, per-pixel last writer
(ext-face index), visible ext faces in order, bounding boxes, and per-face
compositing-step counts (from the counting build).

    python tests/golden/make_golden.py reftable

writes reftable.npz: the same cases rendered by the reference with its own
psi table (psiGammaTable512.h), the library's default table.
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from vfray_b200 import psi_table, synth  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # name: (N, carved, view_seed, W, H, store_mesh)
    "convex6_rot": (6, False, 3, 64, 64, True),
    "carved10_rot": (10, True, 7, 96, 72, True),
    "convex5_axis": (5, False, None, 48, 48, True),
    "single_tet": (1, False, 11, 32, 32, True),
    "cfg0_convex24": (24, False, 3, 512, 512, False),
}


def single_tet_mesh(seed):
    rng = np.random.default_rng(seed)
    v = np.zeros((4, 4), np.float32)
    v[:, :3] = rng.uniform(0, 1, size=(4, 3))
    v[:, 3] = rng.uniform(0, 1, size=4)
    return v, np.array([[0, 1, 2, 3]], np.uint32)


def checksum(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def make_inputs(name):
    n, carved, vs, W, H, store = CASES[name]
    if name == "single_tet":
        vert, tet = single_tet_mesh(vs)
    else:
        vert, tet = synth.make_mesh(n, carved=carved, view_seed=vs)
    return vert, tet, synth.transfer_function(2)


def main_reftable():
    """reftable.npz: every case rendered by the reference with its own psi
    table (psiGammaTable512.h as compiled into the reference build), strict
    and fast-math builds, and the table's checksum; the geometry (visible
    set, writers, steps) does not depend on the table and stays in the
    per-case fixtures."""
    refs = {v: oracle.Reference(v) for v in ("strict", "fast")}
    own = refs["strict"].psi()
    assert np.array_equal(own, refs["fast"].psi())
    rec = dict(psi_sha256=checksum(own))
    for name, (n, carved, vs, W, H, store) in CASES.items():
        d = dict(np.load(os.path.join(OUT, f"{name}.npz")))
        if "vert" in d:
            vn, tet, con, extf, tf = d["vert"], d["tet"], d["con"], d["extf"], d["tf"]
        else:
            vert, tet, tf = make_inputs(name)
            R = refs["strict"]
            R.set_mesh(vert, tet)
            R.normalize()
            R.build_con()
            R.build_extf()
            con, _ = R.con()
            extf, vn = R.extf(), R.vert()
        assert checksum(vn, tet, con, extf, tf) == str(d["input_sha256"])
        for k, r in refs.items():
            r.set_psi(own)
            r.set_mesh(vn, tet)
            r.set_con(con, int(d["n_ext"]))
            r.set_extf(extf)
            r.set_lmt(*d["lmt"])
            r.set_tf(tf)
            o = r.render(int(W), int(H), detect=(k == "strict"))
            rec[f"{name}_{k}"] = o["rgb8"]
            if k == "strict":
                assert np.array_equal(o["writer"], d["writer"]), name
    path = os.path.join(OUT, "reftable.npz")
    np.savez_compressed(path, **rec)
    print(f"reftable: {len(CASES)} cases -> {os.path.getsize(path)} bytes")


def main():
    psi = psi_table()
    refs = {v: oracle.Reference(v) for v in ("strict", "count", "fast")}
    for name, (n, carved, vs, W, H, store) in CASES.items():
        vert, tet, tf = make_inputs(name)
        R = refs["strict"]
        R.set_mesh(vert, tet)
        R.normalize()
        R.build_con()
        R.build_extf()
        R.build_lmt()
        con, n_ext = R.con()
        extf, lmt, vn = R.extf(), R.lmt(), R.vert()
        outs = {}
        for k, r in refs.items():
            r.set_psi(psi)
            r.set_mesh(vn, tet)
            r.set_con(con, n_ext)
            r.set_extf(extf)
            r.set_lmt(*lmt)
            r.set_tf(tf)
            outs[k] = r.render(W, H, detect=(k != "fast"))
        s, c, f = outs["strict"], outs["count"], outs["fast"]
        assert np.array_equal(s["rgb8"], c["rgb8"]) and np.array_equal(s["writer"], c["writer"])
        rec = dict(W=W, H=H, rgb8=s["rgb8"], writer=s["writer"], vis=s["vis"], bbox=s["bbox"],
                   face_comp=c["face_exp"], rgb8_fastmath=f["rgb8"], lmt=lmt, n_ext=n_ext,
                   input_sha256=checksum(vn, tet, con, extf, tf),
                   psi_sha256=checksum(psi))
        if store:
            rec.update(vert=vn, tet=tet, con=con, extf=extf, tf=tf)
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(path, **rec)
        print(f"{name}: nT={len(tet)} nExt={n_ext} nVis={s['nvis']} rays={(s['writer'] >= 0).sum()}"
              f" comps={int(c['face_exp'].sum())} -> {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    if sys.argv[1:] == ["reftable"]:
        main_reftable()
    else:
        main()
