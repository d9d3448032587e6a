"""The large frame at full size: one 2048^2 view of the carved 256^3 mesh
(85.6 M tets, 4.1 GB of records on the device, far beyond L2).  The oracle
cannot render the whole frame in test time, so parity is checked through
properties that do not depend on size: per-pixel entry faces against the
oracle's winner pass (every pixel), tet-walk lengths and colours of a seeded
sample of 4,000 rays against the oracle's tracer, ray and step totals, and
the same frame rendered twice.  Building the mesh on the host takes about
two minutes."""
import numpy as np
import pytest

import vfray_b200 as vb
from vfray_b200 import synth
from tests.test_gpu_parity import assert_colour

pytestmark = pytest.mark.gpu


def test_large_frame_full_size(renderer, oracle_lib):
    vert, tet = synth.make_mesh(256, carved=True, view_seed=3)
    p = vb.prepare(vert, tet)
    tf, psi = synth.transfer_function(2), vb.psi_table()
    W = H = 2048
    renderer.upload_tables(tf, psi)
    mid = renderer.upload_mesh(p["vert"], p["tet"], p["con"], p["extf"], p["lmt"])
    try:
        g = renderer.render(mid, W, H)
        again = renderer.render(mid, W, H)
    finally:
        renderer.release_mesh(mid)
    assert np.array_equal(g["rgb8"], again["rgb8"]) and np.array_equal(g["steps"], again["steps"])
    m = oracle_lib.mesh(p["vert"], p["tet"], p["con"], p["extf"], tf, psi, p["lmt"][0])
    wr = oracle_lib.winners(m, W, H).ravel()
    rays = np.flatnonzero(wr >= 0)
    steps = g["steps"].ravel()
    assert g["stats"]["num_rays"] == len(rays) > 2_000_000
    assert np.all(steps[rays] > 0) and np.all(steps[wr < 0] == 0)
    assert g["stats"]["num_steps"] == int(steps.sum())
    sample = np.random.default_rng(1).choice(rays, size=4000, replace=False).astype(np.uint32)
    t = oracle_lib.trace_pixels(m, W, H, sample, wr[sample])
    assert np.array_equal(steps[sample], t["steps"])
    assert_colour(g["rgb8"].reshape(-1, 3)[sample], t["rgb8"],
                  g["rgba"].reshape(-1, 4)[sample], t["rgba"])
