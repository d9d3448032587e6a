"""Error behaviour of the C ABI on a GPU context.  Every failure here is made
on the host (a bad array, a call out of order) or by a bounded device-side
check that reports through the status word; nothing faults the GPU."""
import numpy as np
import pytest

import vfray_b200 as vb
from tests.conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture
def case(renderer):
    d = load_golden("convex6_rot")
    renderer.upload_tables(d["tf"], d["psi"])
    return d


def expect(status, fn, *args, **kw):
    with pytest.raises(vb.VfrError) as e:
        fn(*args, **kw)
    assert e.value.status == status, str(e.value)
    return e.value


def test_rejects_out_of_range_vertex(renderer, case):
    tet = case["tet"].copy()
    tet[3, 2] = len(case["vert"])
    expect(vb._lib.VFR_ERR_MESH, renderer.upload_mesh, case["vert"], tet, case["con"],
           case["extf"], case["lmt"])


def test_rejects_asymmetric_adjacency(renderer, case):
    con = case["con"].copy()
    t = int(np.argmax((con != np.arange(len(con))[:, None]).all(1)))  # an interior tet
    n = con[t, 0]
    back = np.flatnonzero(con[n] == t)[0]
    con[n, back] = n  # neighbour no longer points back
    e = expect(vb._lib.VFR_ERR_MESH, renderer.upload_mesh, case["vert"], case["tet"], con,
               case["extf"], case["lmt"])
    assert "point back" in str(e)


def test_rejects_interior_face_in_ext_list(renderer, case):
    extf = case["extf"].copy()
    con = case["con"]
    t = int(np.argmax((con != np.arange(len(con))[:, None]).all(1)))
    extf[0] = (t, 0)
    expect(vb._lib.VFR_ERR_MESH, renderer.upload_mesh, case["vert"], case["tet"], con, extf,
           case["lmt"])


def test_rejects_empty_mesh_and_empty_batch(renderer, case):
    """A mesh without vertices or tets is refused at upload; a batch without
    jobs is refused when its jobs are set; the context stays usable."""
    v0 = np.zeros((0, 4), np.float32)
    t0 = np.zeros((0, 4), np.uint32)
    e0 = np.zeros((0, 2), np.uint32)
    expect(vb._lib.VFR_ERR_INVALID, renderer.upload_mesh, v0, case["tet"], case["con"],
           case["extf"], case["lmt"])
    expect(vb._lib.VFR_ERR_INVALID, renderer.upload_mesh, case["vert"], t0, t0, e0, case["lmt"])
    from vfray_b200 import batch as vbatch

    with pytest.raises(vb.VfrError) as e:
        vbatch.BatchRenderer(renderer, [])
    assert e.value.status == vb._lib.VFR_ERR_INVALID
    mid = renderer.upload_mesh(case["vert"], case["tet"], case["con"], case["extf"], case["lmt"])
    try:
        renderer.render(mid, 16, 16)
    finally:
        renderer.release_mesh(mid)


def test_rejects_unusable_max_edge(renderer, case):
    """maxEdgeLength enters the traversal through a reciprocal whose quotients
    must stay normal: values from 2^80 up, and NaN, are refused."""
    for bad in (2.0 ** 80, float("inf"), float("nan")):
        lmt = case["lmt"].copy()
        lmt[0] = bad
        expect(vb._lib.VFR_ERR_INVALID, renderer.upload_mesh, case["vert"], case["tet"],
               case["con"], case["extf"], lmt)


def test_rejects_oversized_and_degenerate_images(renderer, case):
    """More than 2^28 pixels, or a side below 2 (the reference divides by
    res - 1), is refused before anything is allocated or launched."""
    mid = renderer.upload_mesh(case["vert"], case["tet"], case["con"], case["extf"], case["lmt"])
    try:
        for W, H in ((1 << 15, 1 << 14), (1, 64), (64, 1), (0, 0)):
            expect(vb._lib.VFR_ERR_INVALID, renderer.render_device, mid, W, H)
        renderer.render(mid, 16, 16)  # the context is still usable
    finally:
        renderer.release_mesh(mid)


def test_stage_order_and_handles(renderer, case):
    mid = renderer.upload_mesh(case["vert"], case["tet"], case["con"], case["extf"], case["lmt"])
    try:
        # project before find_visible on a fresh view of this mesh
        renderer.render(mid, 16, 16)  # leaves no stage pending
        expect(vb._lib.VFR_ERR_STATE, renderer.project, mid, 16, 16, 1)
        expect(vb._lib.VFR_ERR_STATE, renderer.render, mid + 100, 16, 16)
        expect(vb._lib.VFR_ERR_INVALID, renderer.render, mid, 1, 16)
        expect(vb._lib.VFR_ERR_INVALID, renderer.set_option, 999, 1)
    finally:
        renderer.release_mesh(mid)
    expect(vb._lib.VFR_ERR_STATE, renderer.release_mesh, mid)


def test_step_cap_reports_status(renderer, case):
    """A per-ray step cap that real rays exceed ends those rays early and is
    reported as VFR_ERR_DEVICE with the STEP_CAP bit; the context stays
    usable afterwards."""
    mid = renderer.upload_mesh(case["vert"], case["tet"], case["con"], case["extf"], case["lmt"])
    try:
        renderer.set_option(vb.OPT_STEP_CAP, 3)
        e = expect(vb._lib.VFR_ERR_DEVICE, renderer.render, mid, case["W"], case["H"])
        assert "step-cap" in str(e)
        renderer.set_option(vb.OPT_STEP_CAP, 0)
        out = renderer.render(mid, case["W"], case["H"])
        assert out["stats"]["device_status"] == 0
    finally:
        renderer.set_option(vb.OPT_STEP_CAP, 0)
        renderer.release_mesh(mid)
