"""Batched form: every job of a batch (mixed meshes, resolutions, cameras,
run directly or as a captured CUDA graph) gives exactly the image and tet-walk
lengths of the same view rendered alone, which the parity tests tie to the
reference."""
import numpy as np
import pytest

import vfray_b200 as vb
from vfray_b200 import batch as vbatch
from vfray_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene(renderer):
    meshes = []
    for n, carved, seed in [(10, True, 4), (7, False, 5)]:
        vert, tet = synth.make_mesh(n, carved=carved, view_seed=None)
        p = vb.prepare(vert, tet)
        renderer.upload_tables(synth.transfer_function(2))
        meshes.append(renderer.upload_mesh(p["vert"], p["tet"], p["con"], p["extf"], p["lmt"]))
    views = synth.orbit_views(5, seed=9)
    jobs = [(meshes[0], views[0], 96, 80), (meshes[1], views[1], 64, 64),
            (meshes[0], None, 50, 37), (meshes[0], views[2], 128, 128),
            (meshes[1], views[3], 33, 90), (meshes[1], None, 64, 64)]
    yield jobs
    for m in meshes:
        renderer.release_mesh(m)


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("mode", [vb.MODE_REF, vb.MODE_COMPOSITED])
def test_batch_equals_single_views(renderer, scene, graph, mode):
    B = vbatch.BatchRenderer(renderer, scene, mode=mode, graph=graph)
    try:
        B.prepare()
        for rep in range(2):  # a replayed graph gives the same result
            B.run()
            stats = B.stats()
            npx = sum(W * H for (_, _, W, H) in scene)
            rgb = np.empty(npx * 3, np.uint8)
            steps = np.empty(npx, np.uint32)
            B.read(rgb8=rgb, steps=steps)
            off = 0
            for j, (mid, mv, W, H) in enumerate(scene):
                single = renderer.render(mid, W, H, mv=mv, mode=mode)
                n = W * H
                assert np.array_equal(rgb[3 * off:3 * (off + n)].reshape(H, W, 3), single["rgb8"]), j
                assert np.array_equal(steps[off:off + n].reshape(H, W), single["steps"]), j
                assert stats[j]["num_rays"] == single["stats"]["num_rays"]
                assert stats[j]["num_steps"] == single["stats"]["num_steps"]
                off += n
    finally:
        B.close()


def test_batch_device_outputs(renderer, scene):
    """Jobs may render into the caller's device buffers."""
    import torch

    jobs, bufs = [], []
    for (mid, mv, W, H) in scene:
        rgb = torch.full((H, W, 3), 7, dtype=torch.uint8, device="cuda")
        bufs.append(rgb)
        jobs.append(vbatch.job(mid, W, H, mv=mv, rgb8=rgb))
    B = vbatch.BatchRenderer(renderer, jobs)
    try:
        B.prepare()
        B.run()
        B.stats()
        for (mid, mv, W, H), rgb in zip(scene, bufs):
            single = renderer.render(mid, W, H, mv=mv)
            assert np.array_equal(rgb.cpu().numpy(), single["rgb8"])
    finally:
        B.close()


def test_batch_outliving_its_context_is_safe():
    """Destroying the context first detaches its batches: running one then
    reports a state error, and destroying it is still safe."""
    p = vb.prepare(*synth.make_mesh(4, view_seed=1))
    r = vb.Renderer(0)
    r.upload_tables(synth.transfer_function(2))
    mid = r.upload_mesh(p["vert"], p["tet"], p["con"], p["extf"], p["lmt"])
    B = vbatch.BatchRenderer(r, [(mid, None, 16, 16)], graph=False)
    B.run()
    B.stats()
    r.close()
    assert B.lib.vfr_batch_run(B.h) == vb._lib.VFR_ERR_STATE
    B.close()


def test_batch_with_rayless_jobs(renderer):
    """Jobs whose images no face covers (the single tet at 2x2 and 2x5) mixed
    with jobs that have rays, and a batch of rayless jobs only: empty
    segments of the ray queue, zero totals, images zeroed."""
    from tests.conftest import load_golden

    d = load_golden("single_tet")
    renderer.upload_tables(d["tf"], d["psi"])
    mid = renderer.upload_mesh(d["vert"], d["tet"], d["con"], d["extf"], d["lmt"])
    try:
        for jobs in ([(mid, None, 2, 2), (mid, None, 4, 4), (mid, None, 2, 5), (mid, None, 3, 3)],
                     [(mid, None, 2, 2), (mid, None, 2, 5)]):
            for graph in (False, True):
                B = vbatch.BatchRenderer(renderer, jobs, graph=graph)
                try:
                    B.prepare()
                    B.run()
                    stats = B.stats()
                    npx = sum(W * H for (_, _, W, H) in jobs)
                    rgb = np.full(npx * 3, 77, np.uint8)
                    steps = np.full(npx, 77, np.uint32)
                    B.read(rgb8=rgb, steps=steps)
                    off = 0
                    for j, (m_, mv, W, H) in enumerate(jobs):
                        single = renderer.render(m_, W, H)
                        n = W * H
                        assert stats[j]["num_rays"] == single["stats"]["num_rays"]
                        assert np.array_equal(rgb[3 * off:3 * (off + n)].reshape(H, W, 3),
                                              single["rgb8"])
                        assert np.array_equal(steps[off:off + n].reshape(H, W), single["steps"])
                        off += n
                    assert [s["num_rays"] for s in stats][:1] == [0]
                finally:
                    B.close()
    finally:
        renderer.release_mesh(mid)


def test_cameras_change_between_host_runs(renderer, scene):
    """The host-buffer form uploads the step's cameras: a replayed graph
    renders with the model-views of the latest vfr_batch_set_cameras, and
    each job equals the same view rendered alone with that camera."""
    import torch

    jobs = [j for j in scene if j[1] is not None]
    npx = sum(W * H for (_, _, W, H) in jobs)
    B = vbatch.BatchRenderer(renderer, jobs)
    try:
        B.prepare()
        rgb = torch.empty(npx * 3, dtype=torch.uint8, pin_memory=True)
        cams = torch.empty((len(jobs), 4, 4), dtype=torch.float32, pin_memory=True)
        images = []
        for views in (synth.orbit_views(len(jobs), seed=21), synth.orbit_views(len(jobs), seed=22)):
            cams.copy_(torch.from_numpy(views))
            B.run_host(rgb, cameras=cams)
            B.stats()
            img = rgb.numpy().copy()
            images.append(img)
            off = 0
            for j, (mid, _, W, H) in enumerate(jobs):
                single = renderer.render(mid, W, H, mv=views[j])
                n = W * H
                assert np.array_equal(img[3 * off:3 * (off + n)].reshape(H, W, 3), single["rgb8"]), j
                off += n
        assert not np.array_equal(images[0], images[1])
    finally:
        B.close()


def test_two_batches_on_two_streams_take_turns(renderer, scene):
    """A frame loop over two batches of the same jobs, each on a stream of
    its own: per step, cameras in, run, an asynchronous read into that
    batch's pinned buffer.  After both streams are done, each step's images
    equal the same cameras rendered by one batch with a waiting read."""
    import torch

    jobs = [j for j in scene if j[1] is not None]
    npx = sum(W * H for (_, _, W, H) in jobs)
    pair = [vbatch.BatchRenderer(renderer, jobs), vbatch.BatchRenderer(renderer, jobs)]
    ref = vbatch.BatchRenderer(renderer, jobs)
    try:
        streams = [torch.cuda.Stream(), torch.cuda.Stream()]
        for x, s in zip(pair, streams):
            x.prepare()
            x.set_stream(s)
        ref.prepare()
        steps = [synth.orbit_views(len(jobs), seed=31 + k) for k in range(4)]
        cams = [torch.empty((len(jobs), 4, 4), dtype=torch.float32, pin_memory=True)
                for _ in steps]
        outs = [torch.empty(npx * 3, dtype=torch.uint8, pin_memory=True) for _ in steps]
        got = []
        for k, views in enumerate(steps):
            x = pair[k & 1]
            if k >= 2:  # this batch's previous step is read back: keep it
                x.synchronize()
                got.append(outs[k - 2].numpy().copy())
            cams[k].copy_(torch.from_numpy(views))
            x.set_cameras(cams[k])
            x.run()
            x.read_async(rgb8=outs[k])
        for x in pair:
            x.synchronize()
        got += [outs[2].numpy().copy(), outs[3].numpy().copy()]
        want = torch.empty(npx * 3, dtype=torch.uint8, pin_memory=True)
        for k, views in enumerate(steps):
            ref.run_host(want, cameras=torch.from_numpy(views).contiguous())
            assert np.array_equal(got[k], want.numpy()), k
        assert not np.array_equal(got[0], got[1])
        for x in pair:
            x.stats()
    finally:
        for x in pair + [ref]:
            x.close()


def test_cycling_ray_is_stopped(renderer, oracle_lib):
    """A mesh whose tets list their vertices in random order, seen from a
    view where one ray's walk cycles among the tets around an edge (the
    reference's loop never ends on it): the ray is stopped by the exact
    cycle check (its state saved at power-of-two iteration counts from 4096
    on), its pixel keeps what it composited, the status says so, and every
    pixel's step count -- the cycling ray's included -- equals the oracle's,
    which applies the same rule."""
    vert, tet = synth.make_mesh(12, carved=False, view_seed=None)
    tet = synth.permute_tet_vertices(tet, 0)
    p = vb.prepare(vert, tet)
    tf = synth.transfer_function(2)
    psi = vb.psi_table()
    mv = synth.orbit_views(8, seed=3)[5]
    renderer.upload_tables(tf, psi)
    mid = renderer.upload_mesh(p["vert"], p["tet"], p["con"], p["extf"], p["lmt"])
    try:
        v = vb.normalize(vb.rotate(p["vert"], mv))
        m = oracle_lib.mesh(v, p["tet"], p["con"], p["extf"], tf, psi, vb.build_lmt(v, p["tet"])[0])
        o = oracle_lib.render_ref(m, 256, 256)
        assert int((o["steps"] > 4095).sum()) == 1  # the one cycling ray
        B = vbatch.BatchRenderer(renderer, [(mid, mv, 256, 256)])
        try:
            B.prepare()
            B.run()
            with pytest.raises(vb.VfrError, match="cycle=32"):
                B.stats()
            steps = np.empty(256 * 256, np.uint32)
            rgb = np.empty(256 * 256 * 3, np.uint8)
            B.read(rgb8=rgb, steps=steps)
            assert np.array_equal(steps.reshape(256, 256), o["steps"])
            d = np.abs(rgb.reshape(256, 256, 3).astype(int) - o["rgb8"].astype(int)).max()
            assert d <= 2, d
        finally:
            B.close()
        # the context is usable afterwards
        renderer.render(mid, 64, 64)
    finally:
        renderer.release_mesh(mid)


def test_mixed_workload_full_size_sampled_rays(renderer, oracle_lib):
    """The uneven-jobs workload at its extremes, in one batch: a 1024^2 view
    of the carved 128^3 mesh (10.7 M tets) and a 128^2 view of the carved
    16^3 mesh.  Per job: every pixel's entry face against the oracle's
    winner pass (through the ray count and the zero/non-zero steps), 4,000
    seeded rays traced by the oracle (steps bit for bit, colour within
    tolerance), and the step sum."""
    tf, psi = synth.transfer_function(2), vb.reference_psi_table()
    renderer.upload_tables(tf, psi)
    cases = []
    for n, res, seed in [(128, 1024, 7), (16, 128, 3)]:
        vert, tet = synth.make_mesh(n, carved=True, view_seed=None, jitter_seed=7,
                                    scalar_seed=8, carve_seed=11)
        p = vb.prepare(vert, tet)
        mid = renderer.upload_mesh(p["vert"], p["tet"], p["con"], p["extf"], p["lmt"])
        cases.append((p, mid, res, synth.orbit_views(4, seed=seed)[1]))
    try:
        jobs = [(mid, mv, res, res) for (_, mid, res, mv) in cases]
        B = vbatch.BatchRenderer(renderer, jobs)
        try:
            B.prepare()
            B.run()
            stats = B.stats()
            npx = sum(r * r for (_, _, r, _) in cases)
            rgb = np.empty(npx * 3, np.uint8)
            rgba = np.empty(npx * 4, np.float32)
            steps = np.empty(npx, np.uint32)
            B.read(rgb8=rgb, rgba=rgba, steps=steps)
        finally:
            B.close()
        rng = np.random.default_rng(5)
        off = 0
        for j, (p, _, res, mv) in enumerate(cases):
            n = res * res
            vv = vb.normalize(vb.rotate(p["vert"], mv))
            m = oracle_lib.mesh(vv, p["tet"], p["con"], p["extf"], tf, psi,
                                vb.build_lmt(vv, p["tet"])[0])
            wr = oracle_lib.winners(m, res, res).ravel()
            st = steps[off:off + n]
            rays = np.flatnonzero(wr >= 0)
            assert stats[j]["num_rays"] == len(rays)
            assert np.all(st[rays] > 0) and np.all(st[wr < 0] == 0)
            assert stats[j]["num_steps"] == int(st.sum(dtype=np.uint64))
            sample = rng.choice(rays, size=min(4000, len(rays)), replace=False).astype(np.uint32)
            t = oracle_lib.trace_pixels(m, res, res, sample, wr[sample])
            assert np.array_equal(st[sample], t["steps"])
            d = np.abs(rgb[3 * off:3 * (off + n)].reshape(-1, 3)[sample].astype(int) - t["rgb8"].astype(int))
            assert d.max() <= 2
            rms = np.sqrt(np.mean((rgba[4 * off:4 * (off + n)].reshape(-1, 4)[sample, :3] - t["rgba"][:, :3]) ** 2))
            assert rms <= 1e-3
            off += n
    finally:
        for (_, mid, _, _) in cases:
            renderer.release_mesh(mid)


def test_permuted_orbit_mesh_cycles_are_flagged(renderer, oracle_lib):
    """The 64-view workload's carved 64^3 mesh with every tet listing its
    vertices in a seeded random order: two of its ~10 M rays (views 9 and
    45) walk in a cycle around a projected edge, where the reference's loop
    never ends.  The batch stops exactly those two at the iteration where
    the oracle's identical rule stops them (4,100), reports VFR_DEV_CYCLE,
    and every other ray ends normally."""
    vert, tet = synth.make_mesh(64, carved=True, view_seed=None, jitter_seed=0, scalar_seed=1,
                                carve_seed=4)
    p = vb.prepare(vert, synth.permute_tet_vertices(tet, 0))
    tf = synth.transfer_function(2)
    psi = vb.psi_table()
    views = synth.orbit_views(64, seed=3)
    W = H = 512
    renderer.upload_tables(tf, psi)
    mid = renderer.upload_mesh(p["vert"], p["tet"], p["con"], p["extf"], p["lmt"])
    try:
        B = vbatch.BatchRenderer(renderer, [(mid, mv, W, H) for mv in views])
        try:
            B.prepare()
            B.run()
            with pytest.raises(vb.VfrError, match="cycle=32"):
                B.stats()
            steps = np.empty(len(views) * W * H, np.uint32)
            B.read(steps=steps)
        finally:
            B.close()
        steps = steps.reshape(len(views), W * H)
        long_ = np.argwhere(steps > 4095)
        assert [tuple(x) for x in long_.tolist()] == [(9, 162545), (45, 153268)]
        assert np.all(steps[steps > 4095] == 4100)
        for j, pix in long_.tolist():
            vv = vb.normalize(vb.rotate(p["vert"], views[j]))
            m = oracle_lib.mesh(vv, p["tet"], p["con"], p["extf"], tf, psi,
                                vb.build_lmt(vv, p["tet"])[0])
            wr = oracle_lib.winners(m, W, H).ravel()
            t = oracle_lib.trace_pixels(m, W, H, np.array([pix], np.uint32),
                                        np.array([wr[pix]], np.uint32))
            assert int(t["steps"][0]) == int(steps[j, pix]) == 4100
    finally:
        renderer.release_mesh(mid)
