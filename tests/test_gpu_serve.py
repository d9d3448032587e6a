"""Served form: continuous batching gives every request exactly the image
it gets alone; admission by footprint refuses what can never fit and queues
what does not fit yet; each request reports its latency."""
import threading

import numpy as np
import pytest

import vfray_b200 as vb
from vfray_b200 import serve, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def meshes(renderer):
    renderer.upload_tables(synth.transfer_function(2))
    ids = []
    for n, carved in [(9, True), (6, False), (12, True)]:
        p = vb.prepare(*synth.make_mesh(n, carved=carved, view_seed=None))
        ids.append(renderer.upload_mesh(p["vert"], p["tet"], p["con"], p["extf"], p["lmt"]))
    yield ids
    for m in ids:
        renderer.release_mesh(m)


def _requests(meshes, count, seed):
    rng = np.random.default_rng(seed)
    views = synth.orbit_views(8, seed=seed)
    sizes = [(32, 32), (64, 48), (96, 96), (40, 70)]
    out = []
    for _ in range(count):
        W, H = sizes[rng.integers(len(sizes))]
        mv = views[rng.integers(len(views))] if rng.random() < 0.8 else None
        out.append((meshes[rng.integers(len(meshes))], mv, int(W), int(H)))
    return out


def test_served_results_equal_alone(renderer, meshes):
    reqs = _requests(meshes, 40, 1)
    alone = [renderer.render(m, W, H, mv=mv, rgba=False, steps=False)["rgb8"] for (m, mv, W, H) in reqs]
    with serve.Server(renderer, budget_bytes=4 << 30) as S:
        tickets = []
        # two submitting threads, so requests arrive while batches run
        def submit(part):
            for k in part:
                m, mv, W, H = reqs[k]
                tickets.append((k, S.submit(m, W, H, mv=mv)))
        th = [threading.Thread(target=submit, args=(range(i, len(reqs), 2),)) for i in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        batch_ids = set()
        for k, t in tickets:
            img, info = S.wait(t, timeout_ms=60000)
            assert np.array_equal(img, alone[k]), k
            assert info["t_submit_ms"] <= info["t_start_ms"] <= info["t_done_ms"]
            batch_ids.add(info["batch_id"])
        st = S.stats()
        assert st["completed"] == len(reqs) and st["pending"] == 0 and st["budget_used"] == 0
    assert len(batch_ids) >= 1


def test_admission_refuses_and_queues(renderer, meshes):
    m = meshes[0]
    with serve.Server(renderer, budget_bytes=600_000) as S:
        with pytest.raises(vb.VfrError) as e:
            S.submit(m, 1024, 1024)  # needs far more than the whole budget
        assert e.value.status == vb._lib.VFR_ERR_BUDGET
        # each 64x64 request takes a good part of the budget: they queue
        tickets = [S.submit(m, 64, 64) for _ in range(12)]
        infos = [S.wait(t, timeout_ms=60000)[1] for t in tickets]
        assert all(i["status"] == 0 for i in infos)
        assert len({i["batch_id"] for i in infos}) >= 2  # not all fitted at once
        assert S.stats()["rejected"] == 1


def test_latency_percentiles(renderer, meshes):
    reqs = _requests(meshes, 16, 3)
    with serve.Server(renderer) as S:
        ts = [S.submit(m, W, H, mv=mv) for (m, mv, W, H) in reqs]
        lat = [S.wait(t)[1] for t in ts]
    p = serve.percentiles([i["t_done_ms"] - i["t_submit_ms"] for i in lat])
    assert 0 < p["p50"] <= p["p99"]
