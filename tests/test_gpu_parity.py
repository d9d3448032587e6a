"""The sm_100a render path against the oracle and the reference's golden
fixtures, through the C ABI.

Bars (from the reference's CPU path on the same mesh, TF, psi table, view):
visible-face set, bounding boxes, per-pixel entry face and per-ray tet-walk
iterations are bit-exact; RGB8 within 2/255 per channel and the float colour
within RMS 1e-3.  (Every operation that decides geometry is IEEE-identical to
the reference; only exp() differs -- CUDA's and glibc's double exp may round
differently in the last bit -- so colours are compared with the tolerance.)
"""
import numpy as np
import pytest

import vfray_b200 as vb
from vfray_b200 import synth
from tests.conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu

RGB_TOL = 2      # /255, per channel
RMS_TOL = 1e-3   # float colour


def upload(r, d):
    r.upload_tables(d["tf"], d["psi"])
    return r.upload_mesh(d["vert"], d["tet"], d["con"], d["extf"], d["lmt"])


def assert_colour(rgb_gpu, rgb_ref, rgba_gpu=None, rgba_ref=None):
    diff = np.abs(rgb_gpu.astype(int) - rgb_ref.astype(int))
    assert diff.max() <= RGB_TOL, f"max diff {diff.max()} at {np.argwhere(diff == diff.max())[:3]}"
    if rgba_gpu is not None:
        rms = float(np.sqrt(np.mean((rgba_gpu[..., :3] - rgba_ref[..., :3]) ** 2)))
        assert rms <= RMS_TOL, rms


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_stages_match_golden(name, renderer, oracle_lib):
    d = load_golden(name)
    mid = upload(renderer, d)
    try:
        vis, fd = renderer.find_visible(mid, d["n_ext"])
        assert np.array_equal(vis, d["vis"])
        faces, ovis = oracle_lib.find_visible(oracle_lib.mesh(d["vert"], d["tet"], d["con"],
                                                              d["extf"], d["tf"], d["psi"],
                                                              d["lmt"][0]))
        assert np.array_equal(fd.view(np.uint32), faces.view(np.uint32))  # planes, bit for bit
        bb, wr = renderer.project(mid, d["W"], d["H"], len(vis))
        assert np.array_equal(bb, d["bbox"])
        assert np.array_equal(wr, d["writer"])
        out = renderer.traverse(mid, d["W"], d["H"])
        o = oracle_lib.render_ref(oracle_lib.mesh(d["vert"], d["tet"], d["con"], d["extf"],
                                                  d["tf"], d["psi"], d["lmt"][0]),
                                  d["W"], d["H"])
        assert np.array_equal(out["steps"], o["steps"])
        assert_colour(out["rgb8"], d["rgb8"], out["rgba"], o["rgba"])
        assert out["stats"]["num_rays"] == int((d["writer"] >= 0).sum())
        assert out["stats"]["num_steps"] == int(o["steps"].sum())
        assert out["stats"]["device_status"] == 0
    finally:
        renderer.release_mesh(mid)


@pytest.mark.parametrize("name", ["convex6_rot", "carved10_rot", "cfg0_convex24"])
def test_one_call_render_matches_stages(name, renderer):
    d = load_golden(name)
    mid = upload(renderer, d)
    try:
        a = renderer.render(mid, d["W"], d["H"])
        assert_colour(a["rgb8"], d["rgb8"])
        b = renderer.render(mid, d["W"], d["H"])  # idempotent
        assert np.array_equal(a["rgb8"], b["rgb8"]) and np.array_equal(a["steps"], b["steps"])
    finally:
        renderer.release_mesh(mid)


def prepared(n, carved, seed, view_seed=None):
    vert, tet = synth.make_mesh(n, carved=carved, view_seed=view_seed)
    p = vb.prepare(vert, tet)
    p["tf"] = synth.transfer_function(seed)
    p["psi"] = vb.psi_table()
    return p


@pytest.mark.parametrize("n,carved", [(8, False), (12, True)])
def test_device_view_setup_matches_host(n, carved, renderer, oracle_lib):
    """render(mv=...) rotates, normalises and recomputes the limits on the
    device; the host restatement of rotateVolume + normalizeVertices +
    buildLmt (pinned to the reference) gives the same rays."""
    p = prepared(n, carved, 5)
    mid = upload(renderer, p)
    W, H = 120, 96
    try:
        for mv in synth.orbit_views(3, seed=n):
            vv = vb.normalize(vb.rotate(p["vert"], mv))
            lmt = vb.build_lmt(vv, p["tet"])
            m = oracle_lib.mesh(vv, p["tet"], p["con"], p["extf"], p["tf"], p["psi"], lmt[0])
            o = oracle_lib.render_ref(m, W, H)
            g = renderer.render(mid, W, H, mv=mv)
            assert np.array_equal(g["steps"], o["steps"])
            assert_colour(g["rgb8"], o["rgb8"], g["rgba"], o["rgba"])
    finally:
        renderer.release_mesh(mid)


def test_composited_matches_oracle(renderer, oracle_lib):
    d = load_golden("carved10_rot")
    mid = upload(renderer, d)
    try:
        g = renderer.render(mid, d["W"], d["H"], mode=vb.MODE_COMPOSITED)
        m = oracle_lib.mesh(d["vert"], d["tet"], d["con"], d["extf"], d["tf"], d["psi"],
                            d["lmt"][0])
        o = oracle_lib.render_composited(m, d["W"], d["H"], threads=4)
        assert np.array_equal(g["steps"], o["steps"])
        assert_colour(g["rgb8"], o["rgb8"], g["rgba"], o["rgba"])
        assert g["stats"]["num_entries"] >= g["stats"]["num_rays"]
    finally:
        renderer.release_mesh(mid)


@pytest.mark.parametrize("n,W,H,view", [(20, 333, 250, 2), (32, 512, 512, 5), (7, 1000, 37, 1)])
def test_composited_tiles_match_oracle(n, W, H, view, renderer, oracle_lib):
    """Composited mode, whose entry lists come from faces binned into 16 x 16
    screen tiles: images whose edges cut tiles, a model-view rotated on the
    device, meshes where rays re-enter many times.  Per-ray steps over all
    segments bit-exact against the oracle's composited restatement."""
    vert, tet = synth.make_mesh(n, carved=True, view_seed=None)
    p = vb.prepare(vert, tet)
    tf, psi = synth.transfer_function(2), vb.psi_table()
    renderer.upload_tables(tf, psi)
    mid = renderer.upload_mesh(p["vert"], p["tet"], p["con"], p["extf"], p["lmt"])
    try:
        mv = synth.orbit_views(8, seed=4)[view]
        g = renderer.render(mid, W, H, mv=mv, mode=vb.MODE_COMPOSITED)
        v = vb.normalize(vb.rotate(p["vert"], mv))
        m = oracle_lib.mesh(v, p["tet"], p["con"], p["extf"], tf, psi, vb.build_lmt(v, p["tet"])[0])
        o = oracle_lib.render_composited(m, W, H, threads=8)
        assert np.array_equal(g["steps"], o["steps"])
        assert_colour(g["rgb8"], o["rgb8"], g["rgba"], o["rgba"])
        assert g["stats"]["num_rays"] == int((o["nseg"] > 0).sum())  # pixels with an entry
    finally:
        renderer.release_mesh(mid)


def test_full_size_carved_orbit_properties(renderer, oracle_lib):
    """The 64^3 carved mesh at 512^2 (the batched workload's mesh): per-pixel
    entry faces against the oracle's winner pass, a seeded sample of rays
    traced by the oracle, and size-independent properties (step sum, range,
    idempotence)."""
    p = prepared(64, True, 2)
    mid = upload(renderer, p)
    W = H = 512
    rng = np.random.default_rng(0)
    try:
        for mv in synth.orbit_views(64, seed=4)[::21]:
            vv = vb.normalize(vb.rotate(p["vert"], mv))
            lmt = vb.build_lmt(vv, p["tet"])
            m = oracle_lib.mesh(vv, p["tet"], p["con"], p["extf"], p["tf"], p["psi"], lmt[0])
            g = renderer.render(mid, W, H, mv=mv)
            wr = oracle_lib.winners(m, W, H)
            rays = np.flatnonzero(wr.ravel() >= 0)
            assert g["stats"]["num_rays"] == len(rays)
            assert np.all(g["steps"].ravel()[rays] > 0)
            assert np.all(g["steps"].ravel()[wr.ravel() < 0] == 0)
            assert g["stats"]["num_steps"] == int(g["steps"].sum())
            sample = rng.choice(rays, size=min(4000, len(rays)), replace=False).astype(np.uint32)
            t = oracle_lib.trace_pixels(m, W, H, sample, wr.ravel()[sample])
            assert np.array_equal(g["steps"].ravel()[sample], t["steps"])
            assert_colour(g["rgb8"].reshape(-1, 3)[sample], t["rgb8"],
                          g["rgba"].reshape(-1, 4)[sample], t["rgba"])
    finally:
        renderer.release_mesh(mid)


@pytest.mark.parametrize("seed,carved", [(0, False), (1, True), (2, True)])
def test_permuted_tet_vertex_order(seed, carved, renderer, oracle_lib):
    """Tets listing their vertices in random orders, so neighbouring tets
    share faces under every vertex permutation (lattice meshes only ever
    give the identity): every permutation code of the walk records runs,
    mixed within warps.  Bit-exact steps, colour within tolerance,
    in the single-view and the batched path."""
    from vfray_b200 import batch as vbatch

    vert, tet = synth.make_mesh(10, carved=carved, view_seed=seed + 7)
    tet = synth.permute_tet_vertices(tet, seed)
    p = vb.prepare(vert, tet)
    p["tf"], p["psi"] = synth.transfer_function(seed), vb.psi_table()
    mid = upload(renderer, p)
    try:
        m = oracle_lib.mesh(p["vert"], p["tet"], p["con"], p["extf"], p["tf"], p["psi"],
                            p["lmt"][0])
        o = oracle_lib.render_ref(m, 96, 80)
        g = renderer.render(mid, 96, 80)
        assert np.array_equal(g["steps"], o["steps"])
        assert_colour(g["rgb8"], o["rgb8"], g["rgba"], o["rgba"])
        mv = synth.orbit_views(3, seed=seed)[1]
        single = renderer.render(mid, 64, 72, mv=mv)
        B = vbatch.BatchRenderer(renderer, [(mid, None, 96, 80), (mid, mv, 64, 72)])
        try:
            B.prepare()
            B.run()
            B.stats()
            steps = np.empty(96 * 80 + 64 * 72, np.uint32)
            B.read(steps=steps)
            assert np.array_equal(steps[:96 * 80].reshape(80, 96), o["steps"])
            assert np.array_equal(steps[96 * 80:].reshape(72, 64), single["steps"])
        finally:
            B.close()
    finally:
        renderer.release_mesh(mid)


@pytest.mark.parametrize("W,H", [(2, 2), (37, 23), (8, 300)])
def test_ragged_image_sizes(W, H, renderer, oracle_lib):
    d = load_golden("convex6_rot")
    mid = upload(renderer, d)
    try:
        g = renderer.render(mid, W, H)
        m = oracle_lib.mesh(d["vert"], d["tet"], d["con"], d["extf"], d["tf"], d["psi"],
                            d["lmt"][0])
        o = oracle_lib.render_ref(m, W, H)
        assert np.array_equal(g["steps"], o["steps"])
        assert_colour(g["rgb8"], o["rgb8"])
    finally:
        renderer.release_mesh(mid)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_reference_psi_table_is_the_default(name, renderer, oracle_lib):
    """With the library's default psi table -- the reference's own
    psiGammaTable512.h, shipped beside the library -- every golden case
    matches the reference's kernels rendering with that same table: visible
    set, boxes, entry faces and per-ray steps bit for bit (they do not
    depend on the table), RGB8 within 2/255 of the reference's image, and
    the float colour against the oracle run with the same table."""
    import os

    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", "reftable.npz"))
    d = load_golden(name)
    renderer.upload_tables(d["tf"])  # no table given: the reference's own
    mid = renderer.upload_mesh(d["vert"], d["tet"], d["con"], d["extf"], d["lmt"])
    try:
        vis, _ = renderer.find_visible(mid, d["n_ext"])
        assert np.array_equal(vis, d["vis"])
        bb, wr = renderer.project(mid, d["W"], d["H"], len(vis))
        assert np.array_equal(bb, d["bbox"]) and np.array_equal(wr, d["writer"])
        out = renderer.traverse(mid, d["W"], d["H"])
        psi = vb.reference_psi_table()
        o = oracle_lib.render_ref(oracle_lib.mesh(d["vert"], d["tet"], d["con"], d["extf"],
                                                  d["tf"], psi, d["lmt"][0]), d["W"], d["H"])
        assert np.array_equal(out["steps"], o["steps"])
        assert_colour(out["rgb8"], fx[f"{name}_strict"], out["rgba"], o["rgba"])
        assert_colour(o["rgb8"], fx[f"{name}_strict"])
    finally:
        renderer.release_mesh(mid)
