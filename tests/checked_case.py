"""Renders through the checked build of the library
(vfray_b200/libvfray_b200_checked.so, built with -DVFR_CHECKED: every id a
kernel reads from memory is compared with the extent of the array it indexes,
and a bad one becomes VFR_DEV_RANGE instead of an out-of-range access), in a
process of its own so that the product library is not loaded beside it:

    python tests/checked_case.py CASE

CASE:
  clean   a golden case in both modes: the same step counts as the oracle,
          the golden image, no device status;
  walk    the four neighbour ids of a tet that rays enter set past nT;
  tet     a vertex id of a visible face's tet set past nV;
  extf    the tet id of a visible external face set past nT.
The last three overwrite the id on the device after the upload validated the
mesh (the checked build's test hook); the render must report VFR_DEV_RANGE,
and a clean mesh must then render correctly in the same context.  Prints one
JSON line.
"""
import ctypes as C
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from vfray_b200 import _lib  # noqa: E402

CHECKED = os.path.join(ROOT, "vfray_b200", "libvfray_b200_checked.so")
WALK, TET, EXTF = 0, 1, 2  # vfr_checked_set_id's arrays


def main(case):
    lib = _lib.load(CHECKED)  # before anything else loads the product library
    lib.vfr_checked_set_id.restype = C.c_int
    lib.vfr_checked_set_id.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_uint32]
    import oracle
    import vfray_b200 as vb
    from tests.conftest import load_golden

    d = load_golden("carved10_rot")
    W, H = d["W"], d["H"]
    o = oracle.Oracle()
    om = o.mesh(d["vert"], d["tet"], d["con"], d["extf"], d["tf"], d["psi"], d["lmt"][0])
    ref = o.render_ref(om, W, H)
    out = {"case": case, "loaded": os.path.basename(lib._name)}

    def clean_render(r):
        m = r.upload_mesh(d["vert"], d["tet"], d["con"], d["extf"], d["lmt"])
        try:
            a = r.render(m, W, H)
            c = r.render(m, W, H, mode=vb.MODE_COMPOSITED)
        finally:
            r.release_mesh(m)
        comp = o.render_composited(om, W, H)
        return {"ref_steps_equal": bool(np.array_equal(a["steps"], ref["steps"])),
                "ref_rgb_maxdiff": int(np.abs(a["rgb8"].astype(int) - d["rgb8"].astype(int)).max()),
                "comp_steps_equal": bool(np.array_equal(c["steps"], comp["steps"])),
                "comp_rgb_maxdiff": int(np.abs(c["rgb8"].astype(int) - comp["rgb8"].astype(int)).max()),
                "status": [a["stats"]["device_status"], c["stats"]["device_status"]]}

    with vb.Renderer(0) as r:
        r.upload_tables(d["tf"], d["psi"])
        if case == "clean":
            out.update(clean_render(r))
        else:
            nT, nV = len(d["tet"]), len(d["vert"])
            # a pixel's entry face, its tet, and the id to overwrite
            p = int(np.argmax(ref["steps"]))
            e = int(d["writer"].reshape(-1)[p])
            t = int(d["extf"][e][0])
            m = r.upload_mesh(d["vert"], d["tet"], d["con"], d["extf"], d["lmt"])
            if case == "walk":
                edits = [(WALK, 4 * t + k, nT + 7 + k) for k in range(4)]
            elif case == "tet":
                edits = [(TET, 4 * t + 1, nV + 5)]
            elif case == "extf":
                edits = [(EXTF, e, nT + 3)]
            else:
                raise SystemExit(f"unknown case {case}")
            for what, index, value in edits:
                _lib.check(lib.vfr_checked_set_id(r.h, m, what, index, value), what="set_id")
            try:
                r.render(m, W, H)
                out["error"] = None
            except vb.VfrError as ex:
                out["error"] = str(ex)
            hit = re.search(r"device status 0x([0-9a-f]+)", out["error"] or "")
            out["status"] = int(hit.group(1), 16) if hit else 0
            r.release_mesh(m)
            out["after"] = clean_render(r)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main(sys.argv[1])
