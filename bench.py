"""Benchmark of the VF-Ray render path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form batched|plain] [--workload orbit64|mixed|served|convex24|large]

Workloads (seeded synthetic meshes, transfer function and cameras):
  orbit64  (default) the carved 64^3 Freudenthal mesh (1,572,864 tets before
           carving at the 85th percentile of a 16-Gaussian field) seen from 64
           seeded orbit views at 512x512; one step renders the 64 views.
  mixed    8 carved meshes with 16..128 cells per side and 256 jobs, each a
           random mesh, resolution in {128^2, 256^2, 512^2, 1024^2} and
           rotation; one step renders the 256 jobs.
  served   32 resident carved meshes, N drawn uniformly from [16, 160] cells
           per side (268 M tets in all), behind the request server: Poisson
           arrivals at 50, 200, 1000 and 2000 requests/s, each request a
           random mesh, resolution in {256^2, 512^2, 1024^2, 2048^2} and
           rotation; p50/p99 latency, per-stage host timestamps and Mrays/s
           per rate, against the same request mix rendered one request at a
           time and as one batch.  Building the meshes on the host takes
           about two minutes.
  convex24 one 512x512 view of the convex 24^3 mesh.
  large    one 2048x2048 view of the carved 256^3 mesh (100.7 M tets before
           carving, 85.6 M after: 4.1 GB of tet and walk records, far beyond
           L2); building the mesh on the host takes about two minutes.
Every workload renders with the reference's own psi table
(psiGammaTable512.h, shipped with the library).

Timing: W untimed warm-up steps, then K steps, each bracketed by CUDA events
on the render stream after an L2 flush (a 256 MiB write) that is not timed;
the step times are summed, the max over ranks is taken (N > 1 runs N
replicas, one per GPU, weak scaling), and ``value`` = rays rendered by all
ranks / that time.  A ray is a pixel with an entry face.  ``e2e`` is the same
metric through the host-buffer API: every step copies the step's cameras from
pinned host memory to the device and the RGB8 images back to pinned host
memory, inside the timed region, as a frame loop does it: two batches of the
same jobs on two streams take turns, so one step's image copy overlaps the
next step's kernels, and the clock stops when both streams are done.
``served_same_jobs`` submits the step's jobs as requests to the request
server (three rounds at once, after an untimed one): the served form at
saturation on the same work, with p50/p99 latency, against the plain
per-view call (``plain_per_view``).  ``roofline`` divides the traversal kernel's
algorithmic bytes (48 B per tet-walk step: one 32-byte walk record + one new
16-byte vertex) by its event-timed launch duration.  ``cpu_baseline`` times
the reference's own CPU kernels (built from the reference sources into
oracle/_ref, -O3 -ffast-math as the reference builds them) on this host over
a bounded sample of the same jobs: single-threaded as the reference is
written, and on all host cores.

``--impl reference`` times the reference's CPU path alone, in a process that
loads none of this repository's product code: the workload's meshes are
generated here, their adjacency computed by the oracle's numpy restatement,
written as the reference's .off/.con/.extf/.tf files and read back through the
reference's own readers; each step then renders every job of the workload
with the reference's per-view sequence (rotateVolume, normalizeVertices,
buildLmt, its three stages) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_STEP = 48        # 32-byte walk record + one new 16-byte vertex
FLUSH_BYTES = 256 << 20    # > 126 MB L2
L2_NOTE = "GPU: flushed between timed steps (256 MiB write, untimed); CPU: not applicable"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="batched", choices=["batched", "plain"])
    ap.add_argument("--workload", default="orbit64",
                    choices=["orbit64", "mixed", "served", "convex24", "large"])
    ap.add_argument("--views", type=int, default=64, help="orbit views (orbit64)")
    ap.add_argument("--mode", default="ref", choices=["ref", "composited"],
                    help="ref: the reference's last-visible-face image; composited: every "
                         "entry segment of each ray, depth-ordered")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="bound of the CPU-baseline sample")
    ap.add_argument("--ref-step-seconds", type=float, default=60.0,
                    help="reference arm: a step stops taking new jobs after this long")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rates", default="50,200,1000,2000", help="served: arrival rates (req/s)")
    ap.add_argument("--served-seconds", type=float, default=2.0)
    ap.add_argument("--served-meshes", type=int, default=32,
                    help="served: resident meshes (the served config has 32)")
    return ap.parse_args()


# ------------------------------------------------------------------ workloads

MIXED_N = (16, 24, 32, 48, 64, 80, 96, 128)


def workload_spec(name, views=64):
    """The workload as seeded inputs, numpy only: raw meshes (vertices not yet
    normalised, tets), jobs (mesh index, model-view or None, W, H), the
    transfer function and a description."""
    from vfray_b200 import synth  # numpy only: loads no native library

    def carved(n, k=0):
        v, t = synth.make_mesh(n, carved=True, view_seed=None, jitter_seed=0 + k,
                               scalar_seed=1 + k, carve_seed=4 + k)
        return dict(n=n, vert=v, tet=t)

    sp = dict(name=name, tf=synth.transfer_function(2))
    if name == "orbit64":
        sp["meshes"] = [carved(64)]
        sp["jobs"] = [(0, mv, 512, 512) for mv in synth.orbit_views(views, seed=3)]
        sp["desc"] = f"{views} orbit views at 512x512 of the carved 64^3 Freudenthal mesh"
    elif name == "large":
        v, t = synth.make_mesh(256, carved=True, view_seed=3)
        sp["meshes"] = [dict(n=256, vert=v, tet=t)]
        sp["jobs"] = [(0, None, 2048, 2048)]
        sp["desc"] = "one 2048x2048 view of the carved 256^3 Freudenthal mesh (seeded rotation)"
    elif name == "convex24":
        v, t = synth.make_mesh(24, carved=False, view_seed=3)
        sp["meshes"] = [dict(n=24, vert=v, tet=t)]
        sp["jobs"] = [(0, None, 512, 512)]
        sp["desc"] = "one 512x512 view of the convex 24^3 Freudenthal mesh (seeded rotation)"
    else:  # mixed
        sp["meshes"] = [carved(n, k) for k, n in enumerate(MIXED_N)]
        rng = np.random.default_rng(5)
        res = (128, 256, 512, 1024)
        jobs = []
        for j in range(256):
            m = int(rng.integers(len(MIXED_N)))
            r = int(res[rng.integers(len(res))])
            q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
            mv = np.eye(4, dtype=np.float32)
            mv[:3, :3] = q * np.sign(np.linalg.det(q))
            jobs.append((m, mv, r, r))
        sp["jobs"] = jobs
        sp["desc"] = ("256 jobs over 8 carved meshes (16..128 cells per side), resolutions "
                      "128^2..1024^2, random rotations")
    return sp


def prepare_ours(sp):
    """The load sequence of the reference driver (normalizeVertices,
    buildCon, buildExtF, buildLmt) through this library, and its default psi
    table (the reference's own)."""
    import vfray_b200 as vb

    meshes = []
    for m in sp["meshes"]:
        p = vb.prepare(m["vert"], m["tet"])
        p["n"] = m["n"]
        meshes.append(p)
    return dict(sp, meshes=meshes, psi=vb.reference_psi_table())


def mesh_info(meshes):
    return [{"cells": p["n"], "tets": int(p["tet"].shape[0]), "verts": int(p["vert"].shape[0]),
             "ext_faces": int(p["extf"].shape[0])} for p in meshes]


def workload_config(wl, rays_per_step, mode):
    """The config both arms report: what the workload is, nothing about how
    an arm runs it."""
    return {"workload": wl["name"], "desc": wl["desc"], "meshes": mesh_info(wl["meshes"]),
            "jobs": len(wl["jobs"]), "pixels_per_step": int(sum(W * H for (_, _, W, H) in wl["jobs"])),
            "rays_per_step": int(rays_per_step),
            "mode": ("composited (every entry segment, depth-ordered)" if mode == "composited"
                     else "reference (last visible face wins)"),
            "psi_table": "the reference's psiGammaTable512.h", "l2": L2_NOTE}


def max_over_ranks(values, dist, device):
    """Element-wise max over ranks of per-rank timings (ms); every rank takes
    part.  Without a process group, the values themselves."""
    if not dist:
        return np.asarray(values, np.float64)
    import torch

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().numpy()


def whole_job_mrays(rays_per_replica_step, world, steps, ms):
    """Whole-job throughput: every replica renders the same workload (weak
    scaling), so the job's rays are world x the replica's, over the slowest
    rank's time."""
    return rays_per_replica_step * world * steps / (ms * 1e-3) / 1e6


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(name):
    """Per-launch DRAM bytes of the traversal kernel from the committed ncu
    summary of this workload, if present."""
    path = os.path.join(ROOT, "profiles", "traverse_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get(name)
    return None


def host_info():
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model}


class Clocks:
    """nvidia-smi sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"vfr_clocks_{os.getpid()}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # the timed region starts once the sampler runs (its start-up takes
        # longer than a short timed region)
        t_end = time.time() + 3.0
        while self.proc and time.time() < t_end and self.proc.poll() is None:
            self.f.flush()
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.06)  # one more sample at the end of the region
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


# ------------------------------------------------------------------ reference (CPU)

class RefRunner:
    """The reference's CPU path (oracle/_ref/libvfref_fast.so: its own
    kernels and precomputation, -O3 -ffast-math as it builds them) over the
    jobs of a workload.  ``meshes``: per mesh the normalised vertices, tets,
    conTet, boundary count, external faces and limits as the reference holds
    them.  A job is its driver's view change -- rotateVolume,
    normalizeVertices and buildLmt of the new view (vfRay.cu:618-641,
    vfRayPreComp.cc:84-145,808-853,886-906) -- then its three stages, on
    ``threads`` host threads (1: the reference's own sequential loop)."""

    def __init__(self, meshes, jobs, tf):
        import oracle

        self.R = oracle.Reference("fast")
        self.R.set_tf(tf)
        self.meshes, self.jobs, self.tf = meshes, jobs, tf
        self.cur = None
        self.rays_of = {}
        self.S = None  # the strict build, for ray counts

    def _load(self, m):
        p = self.meshes[m]
        if self.cur != m:
            self.R.set_mesh(p["vert"], p["tet"])
            self.R.set_con(p["con"], p["n_ext"])
            self.R.set_extf(p["extf"])
            self.cur = m
        else:
            self.R.set_vert(p["vert"])

    def view(self, k):
        m, mv, W, H = self.jobs[k]
        self._load(m)
        if mv is not None:
            self.R.rotate(mv)
            self.R.normalize()
            self.R.build_lmt()
        else:
            self.R.set_lmt(*self.meshes[m]["lmt"])
        return W, H

    def job(self, k, threads):
        W, H = self.view(k)
        if threads == 1:
            self.R.render(W, H, detect=False)
        else:
            self.R.render_mt(W, H, threads=threads)

    def rays(self, k):
        """Pixels with an entry face in job k (not timed): the oracle's
        winner pass over the view as the reference's IEEE build sets it up
        (normalizeVertices of the mesh, then per view rotateVolume +
        normalizeVertices), the workload's own ray count.  The fast-math
        build's set-up moves a handful of pixels in ten million across an
        edge; the count does not follow it."""
        if k not in self.rays_of:
            import oracle

            if self.S is None:
                self.S = oracle.Reference("strict")
            m, mv, W, H = self.jobs[k]
            p = self.meshes[m]
            self.S.set_mesh(p.get("vert_ieee", p["vert"]), p["tet"])
            lmt = p["lmt"]
            if mv is not None:
                self.S.rotate(mv)
                self.S.normalize()
                self.S.build_lmt()
                lmt = self.S.lmt()
            Or = oracle.Oracle()
            om = Or.mesh(self.S.vert(), p["tet"], p["con"], p["extf"], self.tf,
                         np.zeros((512, 512), np.float32), lmt[0])
            self.rays_of[k] = int((Or.winners(om, W, H) >= 0).sum())
        return self.rays_of[k]


def reference_meshes_from_files(sp, tmpdir):
    """Each mesh of the workload as the reference's driver meets it: written
    as .off/.con/.extf/.tf (adjacency from the oracle's numpy restatement of
    buildIncid + buildCon), read back by the reference's readers
    (vfRayPreComp.cc:29-69,375-420,551-590), normalised by its
    normalizeVertices, limits from its buildLmt.  Meshes above 16 M tets are
    handed over as arrays through the same state instead of text files
    (parsing gigabytes of text is not the path being timed)."""
    import oracle
    from oracle import precomp

    out = []
    R = oracle.Reference("fast")
    S = oracle.Reference("strict")
    for i, m in enumerate(sp["meshes"]):
        con, n_ext = precomp.build_con(m["tet"])
        extf = precomp.build_extf(con)
        if m["tet"].shape[0] <= (16 << 20):
            base = os.path.join(tmpdir, f"mesh{i}")
            precomp.write_off(base + ".off", m["vert"], m["tet"])
            precomp.write_con(base + ".con", con, n_ext)
            precomp.write_extf(base + ".extf", extf)
            precomp.write_tf(base + ".tf", sp["tf"])
            R.read_off(base + ".off")
            R.read_con(base + ".con")
            R.read_extf(base + ".extf")
            R.read_tf(base + ".tf")
            inputs = "files"
        else:
            R.set_mesh(m["vert"], m["tet"])
            R.set_con(con, n_ext)
            R.set_extf(extf)
            R.set_tf(sp["tf"])
            inputs = "arrays"
        S.set_mesh(R.vert(), m["tet"])  # as read, before normalisation
        S.normalize()
        R.normalize()
        R.build_lmt()
        rc, rn = R.con()
        out.append(dict(n=m["n"], vert=R.vert(), vert_ieee=S.vert(), tet=m["tet"], con=rc,
                        n_ext=rn, extf=R.extf(), lmt=R.lmt(), tf=R.tf(), inputs=inputs))
    return out


def cpu_baseline(wl, seconds):
    """The reference's CPU kernels on this host over a bounded sample of the
    workload's jobs (in order): a third of the time single-threaded, as the
    reference is written, the rest on all host cores."""
    meshes = [dict(p, n_ext=int(p["extf"].shape[0])) for p in wl["meshes"]]
    run = RefRunner(meshes, wl["jobs"], wl["tf"])
    nthreads = os.cpu_count() or 1
    legs = {}
    for threads, budget in ((1, seconds / 3), (nthreads, 2 * seconds / 3)):
        done, t, k = 0, 0.0, 0
        rays = 0
        while True:
            t0 = time.perf_counter()
            run.job(k, threads)
            t += time.perf_counter() - t0
            rays += run.rays(k)
            done += 1
            k = (k + 1) % len(wl["jobs"])
            if t >= budget:
                break
        legs[threads] = (rays / t / 1e6, done, t)
    v, done, t = legs[nthreads]
    v1, done1, t1 = legs[1]
    return dict({"value": round(v, 4), "unit": "Mrays/s", "cores": nthreads, "kind": "reference",
                 "sample": f"{done} job renders (the workload's {len(wl['jobs'])} jobs in order, "
                           "cycling), reference vfRayKernelCPU.cc "
                           f"(-O3 -ffast-math) on {nthreads} threads (column strips), {t:.1f} s, "
                           "per job rotateVolume + normalizeVertices + buildLmt + the three stages",
                 "single_thread": {"value": round(v1, 4), "unit": "Mrays/s", "cores": 1,
                                   "sample": f"{done1} job(s), the reference's own sequential "
                                             f"loop (main.cc:73-224), {t1:.1f} s"}},
                **host_info())


def product_library_loaded():
    try:
        with open("/proc/self/maps") as f:
            return any("libvfray_b200" in line for line in f)
    except OSError:
        return None


def run_reference(args, rank):
    if rank != 0:
        return None
    import oracle

    if not oracle.ref_available("fast"):
        return {"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) missing"}
    name = "mixed" if args.workload == "served" else args.workload
    sp = workload_spec(name, args.views)
    with tempfile.TemporaryDirectory() as tmp:
        meshes = reference_meshes_from_files(sp, tmp)
    wl = dict(sp, meshes=meshes)
    run = RefRunner(meshes, sp["jobs"], meshes[0]["tf"])
    nthreads = os.cpu_count() or 1
    nj = len(sp["jobs"])
    for w in range(args.warmup):  # the CPU needs no warm-up beyond one job
        run.job(w % nj, nthreads)
    total_t, rendered, full_steps = 0.0, [], 0
    for _ in range(args.steps):
        t_step, k = 0.0, 0
        while k < nj:
            t0 = time.perf_counter()
            run.job(k, nthreads)
            t_step += time.perf_counter() - t0
            rendered.append(k)
            k += 1
            if t_step >= args.ref_step_seconds:
                break
        full_steps += k == nj
        total_t += t_step
    rays = sum(run.rays(k) for k in rendered)
    v = rays / total_t / 1e6
    rays_per_step = sum(run.rays(k) for k in range(nj)) if full_steps == args.steps else rays / args.steps
    loaded = product_library_loaded()
    return {"impl": "reference", "metric": f"Mrays/s ({sp['desc']})", "value": round(v, 4),
            "unit": "Mrays/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_t / args.steps * 1e3, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded meshes, TF and views)",
            "config": workload_config(wl, rays_per_step, args.mode),
            "steps_detail": {"jobs_per_step": len(rendered) / args.steps,
                             "every_step_rendered_all_jobs": full_steps == args.steps,
                             "warmup": "one job per warm-up step",
                             "inputs": sorted({m["inputs"] for m in meshes}),
                             "product_library_loaded": loaded},
            "cpu_baseline": dict({"value": round(v, 4), "unit": "Mrays/s", "cores": nthreads,
                                  "kind": "reference",
                                  "sample": f"{len(rendered)} jobs over {args.steps} steps, "
                                            "reference vfRayKernelCPU.cc (-O3 -ffast-math) on "
                                            f"{nthreads} threads (column strips), per job "
                                            "rotateVolume + normalizeVertices + buildLmt + the "
                                            "three stages"}, **host_info()),
            "e2e": {"value": round(v, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


# ------------------------------------------------------------------ ours

def setup_gpu(wl, dev):
    import torch

    import vfray_b200 as vb

    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    r = vb.Renderer(dev)
    r.set_stream(stream)
    r.upload_tables(wl["tf"], wl["psi"])
    mids = [r.upload_mesh(p["vert"], p["tet"], p["con"], p["extf"], p["lmt"]) for p in wl["meshes"]]
    return r, stream, mids


def served_leg(r, jobs, mode, rounds=3):
    """The step's jobs as requests to the request server (the served form):
    one untimed round, then `rounds` rounds submitted at once, so the server
    runs at saturation on this workload.  Latency is submit to image in the
    caller's host buffer.  Per GPU (each rank measures its own)."""
    from vfray_b200 import serve

    with serve.Server(r, budget_bytes=64 << 30) as S:
        def submit_all(n):
            return [S.submit(mid, W, H, mv=mv, mode=mode)
                    for _ in range(n) for (mid, mv, W, H) in jobs]
        for t in submit_all(1):
            S.wait(t, timeout_ms=600000)
        st0 = S.stats()
        t0 = time.perf_counter()
        infos = [S.wait(t, timeout_ms=600000)[1] for t in submit_all(rounds)]
        dt = time.perf_counter() - t0
        st1 = S.stats()
    assert all(i["status"] == 0 for i in infos)
    lat = [i["t_done_ms"] - i["t_submit_ms"] for i in infos]
    pc = serve.percentiles(lat)
    return {"value": round(sum(i["num_rays"] for i in infos) / dt / 1e6, 2), "unit": "Mrays/s",
            "requests": len(infos), "p50_ms": round(pc["p50"], 3), "p99_ms": round(pc["p99"], 3),
            "drain_launches": st1["launches"] - st0["launches"],
            "admitted_groups": st1["batches"] - st0["batches"],
            "how": (f"the step's {len(jobs)} jobs submitted {rounds} times at once to the request "
                    "server (one persistent drain launch; images into host memory), after one "
                    "untimed round")}


def run_ours(args, rank, world, dist):
    import torch

    import vfray_b200 as vb
    from vfray_b200 import batch as vbatch

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    wl = prepare_ours(workload_spec(args.workload, args.views))
    r, stream, mids = setup_gpu(wl, dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    jobs = [(mids[m], mv, W, H) for (m, mv, W, H) in wl["jobs"]]
    nj = len(jobs)
    mode = vb.MODE_COMPOSITED if args.mode == "composited" else vb.MODE_REF

    # per-job rays and steps from single-view renders (checked below against the batch)
    rays_j, steps_j = [], []
    for (mid, mv, W, H) in jobs:
        o = r.render(mid, W, H, mv=mv, mode=mode, rgba=False, steps=False)
        rays_j.append(o["stats"]["num_rays"])
        steps_j.append(o["stats"]["num_steps"])
    rays_step, steps_step = int(sum(rays_j)), int(sum(steps_j))
    npix = sum(W * H for (_, _, W, H) in jobs)
    offs = np.cumsum([0] + [W * H for (_, _, W, H) in jobs])
    rgb_d = torch.empty(npix * 3, dtype=torch.uint8, device=dev)
    rgba_d = torch.empty(npix * 4, dtype=torch.float32, device=dev)

    def plain_step():
        for i, (mid, mv, W, H) in enumerate(jobs):
            r.render_device(mid, W, H, mv=mv, mode=mode, rgb8=rgb_d[3 * offs[i]:3 * offs[i + 1]],
                            rgba=rgba_d[4 * offs[i]:4 * offs[i + 1]])

    tuning = None
    runner = vbatch.BatchRenderer(r, jobs, mode=mode)
    if not args.no_autotune:
        tuning = runner.autotune(reps=1)
    runner.prepare()

    def batched_step():
        runner.run()

    step = batched_step if args.form == "batched" else plain_step
    launches_per_step = runner.launches_per_run() if args.form == "batched" else 11 * nj

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
        t_main, _ = timed(step, args.steps, args.warmup)
    bst = runner.stats()  # raises on any device status of the batch
    assert sum(x["num_rays"] for x in bst) == rays_step, "batched rays differ from single views"
    assert sum(x["num_steps"] for x in bst) == steps_step, "batched steps differ"
    kp = max(1, min(args.steps, 3))
    t_plain, _ = timed(plain_step, kp, 1)
    prof_plain = timed(plain_step, 1, 0, profile=True)[1] if args.form == "plain" else None
    t_batch, _ = timed(batched_step, kp, 1)
    # stage times of the batched chain: the same batch launched directly
    # (not as a graph) with events between its stages
    runner_p = vbatch.BatchRenderer(r, jobs, mode=mode, graph=False)
    _, prof_batch = timed(lambda: runner_p.run(), kp, 1, profile=True)
    runner_p.close()
    prof, launches_per_trav = (prof_batch, 1) if args.form == "batched" else (prof_plain, nj)

    # e2e through the host API: every step, cameras in from pinned memory,
    # the three stages, RGB8 out to pinned memory
    pinned = torch.empty(npix * 3, dtype=torch.uint8, pin_memory=True)
    cams = torch.empty((nj, 4, 4), dtype=torch.float32, pin_memory=True)
    for i, (_, mv, _, _) in enumerate(jobs):
        cams[i] = torch.from_numpy(np.asarray(mv if mv is not None else np.eye(4), np.float32))
    runner2 = None
    if args.form == "batched":
        # a frame loop as a host application runs it: two batches of the same
        # jobs on two streams take turns, so one step's image copy runs beside
        # the next step's kernels; every step still uploads its cameras and
        # reads all its images back into pinned host memory
        runner2 = vbatch.BatchRenderer(r, jobs, mode=mode)
        runner2.prepare()
        pair = [runner, runner2]
        e2e_streams = [torch.cuda.Stream(dev), torch.cuda.Stream(dev)]
        for x, st_ in zip(pair, e2e_streams):
            x.set_stream(st_)
        outs = [pinned, torch.empty(npix * 3, dtype=torch.uint8, pin_memory=True)]
        turn = [0]

        def e2e_step():
            k = turn[0] & 1
            pair[k].set_cameras(cams)
            pair[k].run()
            pair[k].read_async(rgb8=outs[k])
            turn[0] += 1

        def e2e_wait():
            for x in pair:
                x.synchronize()
        h2d = 48 * nj  # rows 0..2 of each job's model-view
    else:
        host = pinned.numpy()

        def e2e_step():
            for i, (mid, mv, W, H) in enumerate(jobs):
                r.render_into_host(mid, W, H, host[3 * offs[i]:3 * offs[i + 1]], mv=mv, mode=mode)

        def e2e_wait():
            pass
        h2d = None  # each call uploads its one-job table (camera included)
    for _ in range(max(1, args.warmup)):
        e2e_step()
    e2e_wait()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_wait()
    t_e2e = (time.perf_counter() - t0) * 1e3
    if runner2 is not None:
        runner.set_stream(None)
        runner2.close()
    served = served_leg(r, jobs, mode) if args.form == "batched" else None

    times = max_over_ranks([t_main, t_e2e, t_plain, t_batch], dist, dev)
    t_main, t_e2e, t_plain, t_batch = times
    K = args.steps

    def mrays(t, k):
        return whole_job_mrays(rays_step, world, k, t)

    value, e2e = mrays(t_main, K), mrays(t_e2e, K)

    peak, peak_kind = load_peaks()
    # traversal CTAs per SM the register budget allows: 2 + the tuned variant
    # (without the autotuner, the library's default variant 1)
    kmin = 2 + (tuning["variant"] if tuning else 1)
    trav_ms = prof[:, 2] if prof is not None and len(prof) else None
    roof = None
    if trav_ms is not None:
        bytes_per_launch = BYTES_PER_STEP * steps_step / launches_per_trav
        achieved = bytes_per_launch * len(trav_ms) / (trav_ms.sum() * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": round(float(achieved), 1), "peak": peak, "unit": "GB/s",
                "frac": round(float(achieved / peak), 4),
                "peak_kind": ("measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                              else "fallback 6.65 TB/s"),
                "traffic": load_traffic(wl["name"]),
                "algorithmic_bytes_per_launch": int(bytes_per_launch),
                "bytes_per_step": BYTES_PER_STEP,
                "kernel": f"vfr::traverse_kernel<{1 if args.mode == 'composited' else 0},{kmin}>"
                          + (" (one launch for all jobs)" if launches_per_trav == 1 else " (per job)"),
                "launch_ms_mean": round(float(trav_ms.mean()), 4),
                "gsteps_per_s": round(float(steps_step / launches_per_trav * len(trav_ms)
                                            / (trav_ms.sum() * 1e-3) / 1e9), 2),
                "stage_ms_mean": [round(float(x), 4) for x in prof.mean(0)],
                # the same launch counted without the walk's vertex reuse: the
                # record and all 4 vertices of every tet (32 + 4 x 16 B)
                "no_reuse": {"bytes_per_step": 96,
                             "achieved": round(float(achieved * 96 / BYTES_PER_STEP), 1),
                             "frac": round(float(achieved * 96 / BYTES_PER_STEP / peak), 4)}}
    runner.close()
    for m in mids:
        r.release_mesh(m)
    r.close()
    if rank != 0:
        return None
    out = {
        "metric": f"Mrays/s ({wl['desc']})" + (" [composited]" if args.mode == "composited" else ""),
        "value": round(float(value), 2), "unit": "Mrays/s",
        "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": round(float(t_main / K), 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded meshes, TF and views)",
        "config": workload_config(wl, rays_step, args.mode),
        "run": {"form": args.form, "parallelism": f"{world} replica(s), one per GPU",
                "tuning": tuning, "tet_steps_per_step": steps_step},
        "fps": round(float(nj * world * K / (t_main * 1e-3)), 2),
        "gsteps_per_s": round(float(steps_step * world * K / (t_main * 1e-3) / 1e9), 3),
        "batched": {"value": round(float(mrays(t_batch, kp)), 2), "unit": "Mrays/s",
                    "ms_per_step": round(float(t_batch / kp), 3)},
        "plain_per_view": {"value": round(float(mrays(t_plain, kp)), 2), "unit": "Mrays/s",
                           "ms_per_step": round(float(t_plain / kp), 3)},
        "batched_over_plain": round(float(t_plain / t_batch), 3),
        "served_same_jobs": (dict(served, over_plain=round(float(served["value"] / mrays(t_plain, kp)), 3))
                             if served else None),
        "e2e": {"value": round(float(e2e), 2), "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": int(npix * 3), "ms_per_step": round(float(t_e2e / K), 3),
                "copies": ("per step: one 2D copy of the jobs' cameras (host to device), the "
                           "batch graph, one copy of all RGB8 images (device to host); steps "
                           "alternate between two batches of the same jobs on two streams, so one "
                           "step's image copy runs beside the next step's kernels; the timed region "
                           "ends when both streams are done.  It can exceed `value`, which times "
                           "each step alone after an L2 flush: here consecutive steps overlap "
                           "(the next step's stages (a) and (b) run in the traversal's tail)"
                           if args.form == "batched" else
                           "per job: its job table in, its RGB8 image out")},
        "gpu_launches": int(launches_per_step * K),
        "roofline": roof,
        "clocks": clk.summary(),
    }
    return out, wl


# ------------------------------------------------------------------ served

SERVED_RES = (256, 512, 1024, 2048)


def served_spec(seed=13, count=32):
    """The served workload: ``count`` resident carved meshes with N drawn
    uniformly from [16, 160] cells per side (seeded), and a request
    generator (mesh, resolution from {256^2 .. 2048^2}, random rotation)."""
    from vfray_b200 import synth

    from concurrent.futures import ThreadPoolExecutor

    rng = np.random.default_rng(seed)
    ns = [int(x) for x in rng.integers(16, 161, size=count)]

    def one(k):  # numpy releases the interpreter lock: meshes build side by side
        v, t = synth.make_mesh(ns[k], carved=True, view_seed=None, jitter_seed=100 + k,
                               scalar_seed=200 + k, carve_seed=300 + k)
        return dict(n=ns[k], vert=v, tet=t)

    with ThreadPoolExecutor(max_workers=4) as ex:
        meshes = list(ex.map(one, range(count)))
    return dict(name="served", tf=synth.transfer_function(2), meshes=meshes, jobs=[],
                desc=f"{count} resident carved meshes, N uniform in [16,160] (seed {seed}), "
                     "requests at 256^2..2048^2 with random rotations")


def served_requests(n, nmeshes, rng):
    out = []
    for _ in range(n):
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        mv = np.eye(4, dtype=np.float32)
        mv[:3, :3] = q * np.sign(np.linalg.det(q))
        out.append((int(rng.integers(nmeshes)), mv, int(SERVED_RES[rng.integers(len(SERVED_RES))])))
    return out


def run_served(args):
    """Poisson arrivals at each rate for a fixed time over the resident
    meshes; latency = submit to image in the caller's host buffer.  The
    same request mix is also rendered one request at a time through the
    plain per-view call and as one batch, for the served-over-plain ratio."""
    import torch

    import vfray_b200 as vb
    from vfray_b200 import batch as vbatch
    from vfray_b200 import serve

    dev = int(os.environ.get("LOCAL_RANK", "0"))

    def log(*a):
        print(f"[served {time.strftime('%H:%M:%S')}]", *a, file=sys.stderr, flush=True)

    t_gen = time.perf_counter()
    wl = prepare_ours(served_spec(count=args.served_meshes))
    t_gen = time.perf_counter() - t_gen
    log(f"{len(wl['meshes'])} meshes, {sum(p['tet'].shape[0] for p in wl['meshes'])} tets "
        f"built in {t_gen:.1f} s")
    r, stream, mids = setup_gpu(wl, dev)
    nm = len(mids)
    rng = np.random.default_rng(7)
    budget = 120 << 30

    # the same mix, plain (one request at a time, host buffers) and batched
    mix = served_requests(64, nm, np.random.default_rng(99))
    outs = [np.empty((s, s, 3), np.uint8) for (_, _, s) in mix]
    # warm-up, untimed: every mesh once (its distinct edges, which a view
    # with a model-view needs, are built on first use; the server builds
    # them at start), then the first requests of the mix
    for m in range(nm):
        r.render_into_host(mids[m], 64, 64, np.empty((64, 64, 3), np.uint8), mv=mix[0][1])
    for k, (m, mv, s) in enumerate(mix[:4]):
        r.render_into_host(mids[m], s, s, outs[k], mv=mv)
    t0 = time.perf_counter()
    mix_rays = 0
    for k, (m, mv, s) in enumerate(mix):
        mix_rays += r.render_into_host(mids[m], s, s, outs[k], mv=mv)["num_rays"]
    plain_mrays = mix_rays / (time.perf_counter() - t0) / 1e6
    log(f"plain per-view on the mix: {plain_mrays:.1f} Mrays/s")
    B = vbatch.BatchRenderer(r, [(mids[m], mv, s, s) for (m, mv, s) in mix])
    B.prepare()
    pinned = torch.empty(sum(s * s * 3 for (_, _, s) in mix), dtype=torch.uint8, pin_memory=True)
    B.run_host(pinned)
    t0 = time.perf_counter()
    for _ in range(3):
        B.run_host(pinned)
    batched_mrays = 3 * mix_rays / (time.perf_counter() - t0) / 1e6
    B.close()
    log(f"batched on the mix: {batched_mrays:.1f} Mrays/s")

    results = []
    with serve.Server(r, budget_bytes=budget) as S:
        import threading

        done = threading.Event()

        def progress():  # server counters on stderr while the run goes on
            while not done.wait(10.0):
                log("server", S.stats())

        threading.Thread(target=progress, daemon=True).start()
        log("server", S.stats())
        # warm-up, untimed: the pinned staging reaches its working size
        for burst in (16, 64):
            ts = [S.submit(mids[m], s, s, mv=mv) for (m, mv, s) in served_requests(burst, nm, rng)]
            for t in ts:
                S.wait(t, timeout_ms=600000)
        with Clocks(dev) as clk:
            for rate in [float(x) for x in args.rates.split(",")]:
                n = max(8, int(rate * args.served_seconds))
                gaps = rng.exponential(1.0 / rate, size=n)
                reqs = served_requests(n, nm, rng)
                st0 = S.stats()
                tickets = []
                t0 = time.perf_counter()
                due = t0
                for (m, mv, s), g in zip(reqs, gaps):
                    due += g
                    d = due - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    tickets.append(S.submit(mids[m], s, s, mv=mv))
                t_sub = time.perf_counter() - t0
                infos = [S.wait(t, timeout_ms=600000)[1] for t in tickets]
                st1 = S.stats()
                assert all(i["status"] == 0 for i in infos)
                lat = [i["t_done_ms"] - i["t_submit_ms"] for i in infos]
                span = max(i["t_done_ms"] for i in infos) - min(i["t_submit_ms"] for i in infos)
                rays = sum(i["num_rays"] for i in infos)
                groups = {}
                for i in infos:
                    groups[i["batch_id"]] = i["batch_jobs"]
                log(f"rate {rate}: {n} requests done")
                results.append({"rate_req_s": rate, "requests": n,
                                "offered_req_s": round(n / t_sub, 1),
                                "achieved_req_s": round(n / (span * 1e-3), 1),
                                **{k: round(v, 3) for k, v in serve.percentiles(lat).items()},
                                "mrays_s": round(rays / (span * 1e-3) / 1e6, 2),
                                "mean_admitted_group": round(float(np.mean(list(groups.values()))), 1),
                                # host timestamps per stage: queued (submit -> admitted), on the
                                # device (admitted -> last ray seen done), copy-out (-> image in
                                # the caller's buffer); medians and p99 in ms
                                "stages_ms": {
                                    k: {"p50": round(float(np.percentile(v, 50)), 3),
                                        "p99": round(float(np.percentile(v, 99)), 3)}
                                    for k, v in (
                                        ("queued", [i["t_start_ms"] - i["t_submit_ms"] for i in infos]),
                                        ("device", [i["t_ready_ms"] - i["t_start_ms"] for i in infos]),
                                        ("copy_out", [i["t_done_ms"] - i["t_ready_ms"] for i in infos]))},
                                "prep_ms_per_group": round((st1["prep_ms"] - st0["prep_ms"]) /
                                                           max(1, st1["batches"] - st0["batches"]), 3),
                                "drain_launches": st1["launches"] - st0["launches"]})
        stats = S.stats()
        done.set()
    for m in mids:
        r.release_mesh(m)
    r.close()
    best = max(results, key=lambda x: x["mrays_s"])
    return {"metric": "Mrays/s + p50/p99 latency (served: Poisson arrivals over 32 resident carved "
                      "meshes, N in [16,160], requests 256^2..2048^2)",
            "value": best["mrays_s"], "unit": "Mrays/s",
            "n_gpus": 1, "steps": len(results), "warmup": 2, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded meshes, TF, cameras and arrivals)",
            "config": {"workload": "served", "desc": wl["desc"], "meshes": mesh_info(wl["meshes"]),
                       "budget_bytes": budget, "rates": results},
            "served_at_saturation_over_plain": round(best["mrays_s"] / plain_mrays, 3),
            "plain_per_view_same_mix": {"value": round(plain_mrays, 2), "unit": "Mrays/s",
                                        "requests": len(mix),
                                        "how": "one request at a time, vfr_render into host memory"},
            "batched_same_mix": {"value": round(batched_mrays, 2), "unit": "Mrays/s",
                                 "how": "the 64 requests as one batch graph, RGB8 to pinned memory"},
            "server": {k: stats[k] for k in ("launches", "epochs", "queue_timeouts", "mesh_bytes",
                                              "arena_bytes", "batches")},
            "host_seconds_building_meshes": round(t_gen, 1),
            "clocks": clk.summary()}


def _json(o):
    return json.dumps(o, default=lambda x: x.item() if hasattr(x, "item") else str(x))


def main():
    import faulthandler

    faulthandler.enable()
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
        if out is not None:
            print(_json(out))
        return
    if args.workload == "served":
        if os.environ.get("VFRAY_STACK_DUMP_S"):  # Python stacks on stderr before an outer timeout
            faulthandler.dump_traceback_later(float(os.environ["VFRAY_STACK_DUMP_S"]), exit=True)
        if rank == 0:
            print(_json(run_served(args)))
        return
    dist = None
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
    if not args.no_cpu_baseline and world == 1:
        out["cpu_baseline"] = cpu_baseline(wl, args.cpu_seconds)
        if args.mode == "composited":
            out["cpu_baseline"]["sample"] += (" (its own last-visible-face render: the reference "
                                              "has no composited mode)")
    if dist:
        dist.destroy_process_group()
    print(_json(out))


if __name__ == "__main__":
    main()
