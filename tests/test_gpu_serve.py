"""Served form: continuous batching gives every request exactly the image
it gets alone; requests submitted while others run fold into the same
running drain launch; admission by footprint (the resident meshes counted
once) refuses what can never fit and queues what does not fit yet; the
drain's wait for work is bounded; each request reports its latency."""
import threading
import time

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
        assert st["completed"] == len(reqs) and st["pending"] == 0
        assert st["budget_used"] == st["mesh_bytes"] > 0  # only the resident meshes remain
    assert len(batch_ids) >= 1


def _mesh_total(renderer, meshes):
    # the server also builds each mesh's distinct-edge list: a little more
    return sum(renderer.mesh_bytes(m) for m in meshes) + (4 << 20)


def test_admission_refuses_and_queues(renderer, meshes):
    m = meshes[0]
    with serve.Server(renderer, budget_bytes=_mesh_total(renderer, meshes) + (24 << 20)) as S:
        with pytest.raises(vb.VfrError) as e:
            S.submit(m, 4096, 4096)  # needs far more than the whole budget
        assert e.value.status == vb._lib.VFR_ERR_BUDGET
        # each 1024^2 request takes about half of what the meshes leave: they queue
        tickets = [S.submit(m, 1024, 1024) for _ in range(8)]
        infos = [S.wait(t, timeout_ms=60000)[1] for t in tickets]
        assert all(i["status"] == 0 for i in infos)
        assert len({i["batch_id"] for i in infos}) >= 3  # at most two fitted at a time
        st = S.stats()
        assert st["rejected"] == 1 and st["budget_used"] == st["mesh_bytes"]


def test_requests_fold_into_the_running_drain(renderer, meshes):
    """A request submitted while a large one is on the GPU is admitted
    while it runs and served by the same drain launch, and both images
    equal their single renders."""
    big_mv = synth.orbit_views(4, seed=5)[1]
    big_alone = renderer.render(meshes[2], 2048, 2048, mv=big_mv, rgba=False, steps=False)["rgb8"]
    small_alone = renderer.render(meshes[1], 48, 40, rgba=False, steps=False)["rgb8"]
    with serve.Server(renderer, budget_bytes=4 << 30) as S:
        tb = S.submit(meshes[2], 2048, 2048, mv=big_mv)
        time.sleep(0.002)
        ts = S.submit(meshes[1], 48, 40)
        img_b, ib = S.wait(tb, timeout_ms=60000)
        img_s, is_ = S.wait(ts, timeout_ms=60000)
        st = S.stats()
    assert np.array_equal(img_b, big_alone) and np.array_equal(img_s, small_alone)
    assert ib["batch_id"] != is_["batch_id"]      # two admitted groups ...
    assert st["launches"] == 1                     # ... one running launch
    assert is_["t_start_ms"] < ib["t_done_ms"]     # admitted while the big one ran


def test_two_waiters_on_one_ticket(renderer, meshes):
    """A ticket is waited for once: a second waiter on the same ticket is
    refused (VFR_ERR_STATE), never left reading a request the first one
    has retired."""
    with serve.Server(renderer, budget_bytes=4 << 30) as S:
        t = S.submit(meshes[0], 1024, 1024, mv=synth.orbit_views(2, seed=1)[0])
        results = []

        def waiter():
            try:
                results.append(S.wait(t, timeout_ms=60000)[1]["status"])
            except vb.VfrError as e:
                results.append(e.status)

        th = [threading.Thread(target=waiter) for _ in range(2)]
        for x in th:
            x.start()
        for x in th:
            x.join()
    assert sorted(results) == [vb._lib.VFR_ERR_STATE, 0]


def test_drain_idle_wait_is_bounded(renderer, meshes):
    """With the server told to leave an idle drain running, the drain's own
    bounded wait for work runs out: it records VFR_DEV_QUEUE and leaves, and
    the next request is served by a new launch."""
    with serve.Server(renderer, budget_bytes=4 << 30) as S:
        S.set_idle(2000, 60000)  # a 2 ms bounded wait; the server never stops it
        a = S.wait(S.submit(meshes[0], 64, 64))[1]
        deadline = time.time() + 10
        while S.stats()["queue_timeouts"] < 1 and time.time() < deadline:
            time.sleep(0.01)
        st = S.stats()
        assert st["queue_timeouts"] >= 1 and st["launches"] == 1
        b = S.wait(S.submit(meshes[1], 64, 64))[1]
        assert a["status"] == 0 and b["status"] == 0
        assert S.stats()["launches"] == 2


def test_latency_percentiles(renderer, meshes):
    reqs = _requests(meshes, 16, 3)
    with serve.Server(renderer) as S:
        ts = [S.submit(m, W, H, mv=mv) for (m, mv, W, H) in reqs]
        lat = [S.wait(t)[1] for t in ts]
    p = serve.percentiles([i["t_done_ms"] - i["t_submit_ms"] for i in lat])
    assert 0 < p["p50"] <= p["p99"]
