"""Benchmark of the VF-Ray render path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form batched|plain] [--workload orbit64|convex24]

Workload (default ``orbit64``): the carved 64^3 Freudenthal mesh (1,572,864
tets before carving at the 85th percentile of a 16-Gaussian field) seen from
64 seeded orbit views at 512x512, fp32 colour + RGB8.  One step renders all
64 views.  ``convex24`` is the single 512x512 view of the convex 24^3 mesh.

Timing: W untimed warm-up steps, then K steps, each bracketed by CUDA events
on the render stream after an L2 flush (a 256 MiB write) that is not timed;
the step times are summed, the max over ranks is taken (N > 1 runs N
replicas, one per GPU, weak scaling), and ``value`` = rays rendered by all
ranks / that time.  A ray is a pixel with an entry face.  ``e2e`` is the same
metric through the host-buffer API (camera in, RGB8 images out through pinned
host memory, copies inside the timed region).  ``roofline`` divides the
traversal kernel's algorithmic bytes (48 B per tet-walk step: one 32-byte tet
record + one new 16-byte vertex) by its event-timed launch durations.
``cpu_baseline`` times the reference's own CPU kernels (built from the
reference sources into oracle/_ref, -O3 -ffast-math as the reference builds
them) on all host cores over a bounded sample of the same views.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_STEP = 48        # 32-byte tet record + one new 16-byte vertex
FLUSH_BYTES = 256 << 20    # > 126 MB L2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="batched", choices=["batched", "plain"])
    ap.add_argument("--workload", default="orbit64", choices=["orbit64", "convex24"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="bound of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ------------------------------------------------------------------ workload

def make_workload(name):
    import vfray_b200 as vb
    from vfray_b200 import synth

    if name == "orbit64":
        vert, tet = synth.make_mesh(64, carved=True, view_seed=None)
        views = synth.orbit_views(64, seed=3)
        W = H = 512
        desc = "64 orbit views at 512x512 of the carved 64^3 Freudenthal mesh"
    else:
        vert, tet = synth.make_mesh(24, carved=False, view_seed=3)
        views = [None]
        W = H = 512
        desc = "one 512x512 view of the convex 24^3 Freudenthal mesh (seeded rotation)"
    p = vb.prepare(vert, tet)
    p.update(tf=synth.transfer_function(2), psi=vb.psi_table(), views=views, W=W, H=H,
             name=name, desc=desc)
    return p


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the traversal kernel from the committed ncu
    summary, scaled per step of the workload, if present."""
    path = os.path.join(ROOT, "profiles", "traverse_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


class Clocks:
    """nvidia-smi sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"vfr_clocks_{os.getpid()}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return None
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return None
        sm = np.array([r[0] for r in rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[2][k].strip().lower() == "active"})
        loaded = sm[sm >= 0.5 * sm.max()] if sm.max() > 0 else sm
        return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": float(rows[0][1]),
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ ours

def run_ours(args, rank, world, dist):
    import torch

    import vfray_b200 as vb

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    wl = make_workload(args.workload)
    W, H, views = wl["W"], wl["H"], wl["views"]
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    r = vb.Renderer(dev)
    r.set_stream(stream)
    r.upload_tables(wl["tf"], wl["psi"])
    mid = r.upload_mesh(wl["vert"], wl["tet"], wl["con"], wl["extf"], wl["lmt"])
    nv = len(views)

    # reference counts per view (rays, steps) from one checked pass
    rays_v, steps_v = [], []
    for mv in views:
        o = r.render(mid, W, H, mv=mv, rgba=False, steps=False)
        rays_v.append(o["stats"]["num_rays"])
        steps_v.append(o["stats"]["num_steps"])
    rays_step, steps_step = int(sum(rays_v)), int(sum(steps_v))

    rgb_d = torch.empty((nv, H, W, 3), dtype=torch.uint8, device=dev)
    rgba_d = torch.empty((nv, H, W, 4), dtype=torch.float32, device=dev)

    if args.form == "batched":
        from vfray_b200 import batch as vbatch

        runner = vbatch.BatchRenderer(r, [(mid, mv, W, H) for mv in views])
        runner.prepare()

        def step_plain_or_batched():
            runner.run(rgb_d, rgba_d)
        launches_per_step = runner.launches_per_run()
    else:
        def step_plain_or_batched():
            for i, mv in enumerate(views):
                r.render_device(mid, W, H, mv=mv, rgb8=rgb_d[i], rgba=rgba_d[i])
        launches_per_step = 11 * nv

    def plain_step():
        for i, mv in enumerate(views):
            r.render_device(mid, W, H, mv=mv, rgb8=rgb_d[i], rgba=rgba_d[i])

    def timed(fn, K, Wu, profile=False):
        for _ in range(Wu):
            fn()
        stream.synchronize()
        total = 0.0
        if profile:
            r.set_option(vb.OPT_PROFILE, 1)
            r.profile_read()
        for _ in range(K):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            total += s.elapsed_time(e)
        prof = None
        if profile:
            prof = r.profile_read(cap=65536)
            r.set_option(vb.OPT_PROFILE, 0)
        if r.device_status() != 0:
            raise RuntimeError("device status set during the timed run")
        return total, prof

    if dist:
        dist.barrier()
    with Clocks(dev) as clk:
        t_main, _ = timed(step_plain_or_batched, args.steps, args.warmup)
    if args.form == "batched":
        bst = runner.stats()  # raises on any device status of the batch
        assert sum(x["num_rays"] for x in bst) == rays_step, "batched rays differ from single views"
        assert sum(x["num_steps"] for x in bst) == steps_step, "batched steps differ"
    t_plain, prof_plain = timed(plain_step, max(1, min(args.steps, 3)), 1, profile=True)
    if args.form == "batched":
        # stage times of the batched chain: the same batch launched directly
        # (not as a graph) with events between its stages
        runner_p = vbatch.BatchRenderer(r, [(mid, mv, W, H) for mv in views], graph=False)
        _, prof = timed(lambda: runner_p.run(), max(1, min(args.steps, 3)), 1, profile=True)
        runner_p.close()
        launches_per_trav = 1
    else:
        prof = prof_plain
        launches_per_trav = nv

    # e2e through the host API: camera in, RGB8 out (pinned), copies timed
    pinned = torch.empty((nv, H, W, 3), dtype=torch.uint8, pin_memory=True)
    if args.form == "batched":
        def e2e_step():
            runner.run_host(pinned)
    else:
        host_bufs = [pinned[i].numpy() for i in range(nv)]

        def e2e_step():
            for i, mv in enumerate(views):
                r.render_into_host(mid, W, H, host_bufs[i], mv=mv)
    for _ in range(max(1, args.warmup)):
        e2e_step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    t_e2e = (time.perf_counter() - t0) * 1e3

    times = np.array([t_main, t_e2e, t_plain], dtype=np.float64)
    if dist:
        import torch.distributed as td

        tt = torch.tensor(times, device=dev)
        td.all_reduce(tt, op=td.ReduceOp.MAX)
        times = tt.cpu().numpy()
    t_main, t_e2e, t_plain = times
    K = args.steps
    value = rays_step * world * K / (t_main * 1e-3) / 1e6
    e2e = rays_step * world * K / (t_e2e * 1e-3) / 1e6
    plain = rays_step * world * max(1, min(K, 3)) / (t_plain * 1e-3) / 1e6

    # roofline of the traversal kernel: algorithmic bytes of a launch over its
    # event-timed duration (batched: one launch covers all views)
    peak, peak_kind = load_peaks()
    trav_ms = prof[:, 2] if prof is not None and len(prof) else None
    roof = None
    if trav_ms is not None:
        bytes_per_launch = BYTES_PER_STEP * steps_step / launches_per_trav
        achieved = bytes_per_launch * len(trav_ms) / (trav_ms.sum() * 1e-3) / 1e9
        traffic = load_traffic()
        roof = {"bound": "hbm", "achieved": round(float(achieved), 1), "peak": peak, "unit": "GB/s",
                "frac": round(float(achieved / peak), 4),
                "peak_kind": ("measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                              else "fallback 6.65 TB/s"),
                "traffic": None if traffic is None else traffic.get("bytes_per_launch"),
                "algorithmic_bytes_per_launch": int(bytes_per_launch),
                "bytes_per_step": BYTES_PER_STEP,
                "kernel": "vfr::traverse_kernel<0,2>" + (" (one launch for all views)"
                                                        if launches_per_trav == 1 else " (per view)"),
                "launch_ms_mean": round(float(trav_ms.mean()), 4),
                "gsteps_per_s": round(float(steps_step / launches_per_trav * len(trav_ms)
                                            / (trav_ms.sum() * 1e-3) / 1e9), 2),
                "stage_ms_mean": [round(float(x), 4) for x in prof.mean(0)]}
    if args.form == "batched":
        runner.close()
    r.release_mesh(mid)
    r.close()
    if rank != 0:
        return None
    out = {
        "metric": f"Mrays/s ({wl['desc']})", "value": round(value, 2), "unit": "Mrays/s",
        "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": round(t_main / K, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded meshes, TF and views)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "form": args.form,
                   "tets": int(wl["tet"].shape[0]), "verts": int(wl["vert"].shape[0]),
                   "ext_faces": int(wl["extf"].shape[0]), "views": nv,
                   "resolution": f"{W}x{H}", "rays_per_step": rays_step,
                   "tet_steps_per_step": steps_step, "mode": "reference (last visible face wins)",
                   "l2": "flushed between timed steps (256 MiB write, untimed)",
                   "parallelism": f"{world} replica(s), one per GPU"},
        "fps": round(nv * world * K / (t_main * 1e-3), 2),
        "gsteps_per_s": round(steps_step * world * K / (t_main * 1e-3) / 1e9, 3),
        "plain_per_view": {"value": round(plain, 2), "unit": "Mrays/s",
                           "ms_per_step": round(t_plain / max(1, min(K, 3)), 3)},
        "e2e": {"value": round(e2e, 2), "unit": "Mrays/s", "h2d_bytes_per_step": 64 * nv,
                "d2h_bytes_per_step": nv * W * H * 3, "ms_per_step": round(t_e2e / K, 3)},
        "gpu_launches": int(launches_per_step * (K)),
        "roofline": roof,
        "clocks": clk.summary(),
    }
    return out, wl


# ------------------------------------------------------------------ reference (CPU)

def reference_sample(wl, seconds, threads=0):
    """The reference's CPU kernels (oracle/_ref, its own -O3 -ffast-math
    flags) on all host cores over the workload's views, in order, until
    ``seconds`` have passed (at least one view).  Per view: rotateVolume,
    normalizeVertices and buildLmt of the reference, then its three stages."""
    import oracle

    R = oracle.Reference("fast")
    base = wl["vert"]
    nthreads = threads or os.cpu_count() or 1
    done = 0
    t0 = time.perf_counter()
    R.set_tf(wl["tf"])
    for mv in wl["views"]:
        R.set_mesh(base, wl["tet"])
        if mv is not None:
            R.rotate(mv)
            R.normalize()
        R.set_con(wl["con"], wl["extf"].shape[0])
        R.set_extf(wl["extf"])
        R.build_lmt()
        R.render_mt(wl["W"], wl["H"], threads=nthreads)
        done += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return done, dt, nthreads


def count_rays(wl):
    """Rays (pixels with an entry face) per view, from the oracle's winner pass."""
    import oracle
    import vfray_b200 as vb

    Or = oracle.Oracle()
    out = []
    for mv in wl["views"]:
        v = wl["vert"] if mv is None else vb.normalize(vb.rotate(wl["vert"], mv))
        m = Or.mesh(v, wl["tet"], wl["con"], wl["extf"], wl["tf"], wl["psi"], wl["lmt"][0])
        out.append(int((Or.winners(m, wl["W"], wl["H"]) >= 0).sum()))
    return out


def cpu_baseline(wl, seconds, rays_per_view=None):
    done, dt, nthreads = reference_sample(wl, seconds)
    if rays_per_view is None:
        rays_per_view = count_rays({**wl, "views": wl["views"][:done]})
    rays = sum(rays_per_view[:done])
    return {"value": round(rays / dt / 1e6, 4), "unit": "Mrays/s", "cores": nthreads,
            "kind": "reference",
            "sample": f"{done} of {len(wl['views'])} views, reference vfRayKernelCPU.cc "
                      f"(-O3 -ffast-math) on {nthreads} threads (column strips), {dt:.1f} s"}


def run_reference(args, rank):
    if rank != 0:
        return None
    wl = make_workload(args.workload)
    import oracle

    if not oracle.ref_available("fast"):
        return {"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) missing"}
    rays_pv = count_rays(wl)
    per_step_s = max(1.0, args.cpu_seconds / 4)
    for _ in range(args.warmup):
        reference_sample(wl, 0.0)
    total_rays, total_t, nthreads, views_done = 0, 0.0, 1, 0
    for _ in range(args.steps):
        done, dt, nthreads = reference_sample(wl, per_step_s)
        total_rays += sum(rays_pv[:done])
        total_t += dt
        views_done += done
    v = total_rays / total_t / 1e6
    return {"impl": "reference", "metric": f"Mrays/s ({wl['desc']})", "value": round(v, 4),
            "unit": "Mrays/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_t / args.steps * 1e3, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded meshes, TF and views)",
            "config": {"workload": wl["name"], "desc": wl["desc"], "resolution": f"{wl['W']}x{wl['H']}",
                       "views_per_step": "bounded sample (first views of the orbit)"},
            "cpu_baseline": {"value": round(v, 4), "unit": "Mrays/s", "cores": nthreads,
                             "kind": "reference",
                             "sample": f"{views_done} views over {args.steps} steps, reference "
                                       f"vfRayKernelCPU.cc (-O3 -ffast-math) on {nthreads} threads"},
            "e2e": {"value": round(v, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def _json(o):
    return json.dumps(o, default=lambda x: x.item() if hasattr(x, "item") else str(x))


def main():
    import faulthandler

    faulthandler.enable()
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        out = run_reference(args, rank)
        if out is not None:
            print(_json(out))
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td
    try:
        res = run_ours(args, rank, world, dist)
    finally:
        if dist:
            dist.barrier()
    if res is None:
        if dist:
            dist.destroy_process_group()
        return
    out, wl = res
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(wl, args.cpu_seconds)
    if dist:
        dist.destroy_process_group()
    print(_json(out))


if __name__ == "__main__":
    main()
