"""Benchmark: PartialFSHT.jl's stretched-leaf forward + exact adjoint on B200.

Workload (the configuration the headline metric is quoted on): lmax = 2048, a 20-degree
polar cap with M = round(4 (lmax theta*)^2) = 2,044,253 points (cos theta uniform on the cap,
phi uniform, 1% of the points moved to the cap boundary), tol = 1e-8, plain FP64, ntrans = 1,
coefficients complex N(0,1)/(l+1) in every valid sph_mode slot. One step = one forward
apply mul!(f, plan, alm) plus one adjoint apply mul!(alm, plan', f) on inputs resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU: one process per GPU (torchrun), each GPU runs an independent replica of the
workload (the path does not shard: replicas only); the time is the max over ranks.
`--impl reference` times the CPU restatement of the reference's apply (the oracle port) on
the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

THETA_STAR = np.deg2rad(20.0)


def workload(lmax, seed=2048):
    """Seeded synthetic inputs of the benchmark configuration."""
    rng = np.random.default_rng(seed)
    M = int(round(4 * (lmax * THETA_STAR) ** 2))
    theta = np.arccos(1 - (1 - np.cos(THETA_STAR)) * rng.random(M))
    phi = 2 * np.pi * rng.random(M)
    nb = M // 100  # 1% jittered to the boundary (within 1e-9 theta* of it)
    idx = rng.choice(M, nb, replace=False)
    theta[idx] = THETA_STAR * (1 - 1e-9 * rng.random(nb))
    return M, theta, phi, rng


def rand_alm_host(lmax, rng, ntrans=1):
    """complex N(0,1)/(l+1) in the valid modes, zero padding; Julia layout, column-major."""
    nr, nc = lmax + 1, 2 * lmax + 1
    a = np.zeros((ntrans, nc, nr), dtype=np.complex128)  # memory order = Julia (nr, nc, B)
    l = np.arange(nr)
    for c in range(nc):
        am = (c + 1) // 2
        n = nr - am
        v = rng.standard_normal((ntrans, n)) + 1j * rng.standard_normal((ntrans, n))
        a[:, c, :n] = v / (l[:n] + am + 1)
    return a


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"pfsht_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()),
                                   default=None)}


def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def cpu_port_apply_time(lmax, tol, nthreads, napply=1):
    """Time the CPU restatement (oracle port) of the reference apply on this host."""
    from oracle import oracle as O
    M, theta, phi, rng = workload(lmax)
    alm = np.asfortranarray(rand_alm_host(lmax, rng).transpose(2, 1, 0))
    t0 = time.perf_counter()
    S = O.Stretch(theta, phi, lmax, tol, nufft="es")
    build = time.perf_counter() - t0
    g = np.asfortranarray((rng.standard_normal(M) + 1j * rng.standard_normal(M))[:, None])
    times = []
    for _ in range(napply):
        t0 = time.perf_counter()
        S.forward(alm, nthreads=nthreads)
        S.adjoint(g, nthreads=nthreads)
        times.append(time.perf_counter() - t0)
    return min(times), build, M


def run_reference(args, world, rank):
    """--impl reference: the CPU restatement of the reference apply, all host threads."""
    if rank != 0:
        return 0
    nthreads = os.cpu_count() or 1
    from oracle import oracle as O
    M, theta, phi, rng = workload(args.lmax)
    alm = np.asfortranarray(rand_alm_host(args.lmax, rng).transpose(2, 1, 0))
    S = O.Stretch(theta, phi, args.lmax, args.tol, nufft="es")
    g = np.asfortranarray((rng.standard_normal(M) + 1j * rng.standard_normal(M))[:, None])
    for _ in range(args.warmup):
        S.forward(alm, nthreads=nthreads)
        S.adjoint(g, nthreads=nthreads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        S.forward(alm, nthreads=nthreads)
        S.adjoint(g, nthreads=nthreads)
    T = (time.perf_counter() - t0) * 1e3
    ms = T / args.steps
    line = {
        "impl": "reference", "metric": "ms per fwd+adj apply", "value": ms, "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_dict(args, M),
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": nthreads, "kind": "port",
                         "sample": "full workload, one fwd+adj per step (C restatement of the "
                                   "reference's CPU apply with an ES-kernel NUFFT, OpenMP)"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "Julia and FINUFFT are absent on this image, so the reference's own apply "
                "cannot run; this arm times the repository's C restatement of it",
    }
    print(json.dumps(line), flush=True)
    return 0


def fft_lengths_arg(v):
    """--fft-lengths: "timed", "minimal" or N1xN2."""
    if v in ("timed", "minimal"):
        return v
    a, b = v.lower().split("x")
    return int(a), int(b)


def config_dict(args, M):
    B = getattr(args, "ntrans", 1)
    return {"workload": f"stretched-leaf fwd+adj, lmax={args.lmax}, 20deg polar cap, M={M}, "
                        f"tol={args.tol:g}, {args.precision}, ntrans={B}",
            "lmax": args.lmax, "npts": M, "cap_deg": 20.0, "tol": args.tol,
            "precision": args.precision, "ntrans": B,
            "alm": "complex N(0,1)/(l+1) in valid sph_mode slots",
            "points": "cos(theta) uniform on the cap, phi uniform, 1% on the boundary",
            "l2": "3 rotating input sets, each apply's buffers larger than L2",
            "parallelism": f"replicas x{args.gpus}"}


# the stages of the forward apply (the others are the adjoint's)
FWD_STAGES = ("ring_fwd", "fft_theta_fwd", "nufft_pad", "fft_fine1_fwd", "rows_fwd", "fft_fine2_fwd",
              "interp")


def hbm_peak():
    """HBM bandwidth denominator: MEASURED_PEAKS.json's hbm_gbs (of measured) when present, else
    the pool's earlier measurement of 6650 GB/s (of fallback)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        v = json.load(open(p)).get("hbm_gbs")
        if v:
            return float(v), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, ValueError):
        pass
    return 6650.0, "6650 GB/s (of fallback: MEASURED_PEAKS.json absent)"


def load_traffic():
    p = os.path.join(ROOT, "profiles", "traffic_per_launch.json")
    try:
        return json.load(open(p))
    except (OSError, ValueError):
        return {}


def stage_work(info, stage, B=1):
    """Algorithmic work per launch of a stage: (flops, bytes)."""
    L, M, w = info["lmax"], info["npts"], info["nufft_w"]
    rw = info["ring_work"]
    nth, ncols, nf1, nf2, nrows = info["nth"], info["ncols"], info["nf1"], info["nf2"], info["nrows"]
    touched_alm = sum(2 * (L - m + 1) for m in range(info["mmax"] + 1)) * 16 * B
    H = nth * ncols * 16 * B
    U = nrows * nf2 * 16 * B
    pts = M * (16 + 4)
    if stage in ("ring_fwd", "ring_adj"):
        return 10.0 * rw * B, touched_alm + H
    if stage == "interp":
        return 8.0 * M * w * w * B, U + pts + M * 16 * B
    if stage == "spread":
        return 8.0 * M * w * w * B, U + pts + M * 16 * B
    P = nf1 * ncols * 16 * B       # the padded dim-1 grid
    K = nrows * ncols * 16 * B     # its kept rows, mode columns only
    if stage == "nufft_pad":       # mode columns in, padded grid out (zeros included)
        return 0.0, H + P
    if stage == "nufft_unpad":     # the modes read back out of the padded grid
        return 0.0, 2 * H
    if stage == "rows_fwd":        # kept rows of the mode columns in, fine rows out
        return 0.0, K + U
    if stage == "rows_adj":        # fine rows' mode columns in, kept rows out
        return 0.0, 2 * K
    return 0.0, 0.0


def stage_rooflines(info, stages, fp64_peak, hbm, B=1):
    """Per stage of our own kernels: time per launch, algorithmic FP64 rate and bytes rate against
    the measured peaks, and the DRAM rate from the ncu traffic per launch where one is recorded."""
    traffic = load_traffic()
    out = {}
    for k, (tot, n) in stages.items():
        if k.startswith("fft_"):
            continue
        ms = tot / n
        fl, by = stage_work(info, k, B)
        r = {"ms": round(ms, 4)}
        if fl:
            r["fp64_tflops"] = round(fl / (ms * 1e-3) / 1e12, 2)
            r["frac_fp64"] = round(fl / (ms * 1e-3) / 1e12 / fp64_peak, 3)
        if by:
            r["alg_gbs"] = round(by / (ms * 1e-3) / 1e9, 1)
            r["frac_hbm"] = round(by / (ms * 1e-3) / 1e9 / hbm, 3)
        if k in traffic:
            r["dram_gbs"] = round(traffic[k] / (ms * 1e-3) / 1e9, 1)
        out[k] = r
    return out


def time_applies(pf, plan, alms, fins, fout, aout, steps, warmup, stream):
    """Device time of `steps` fwd+adj applies (CUDA events on the launching stream) and the
    per-stage profile of those applies."""
    import torch
    nset = len(alms)

    def step(i):
        k = i % nset
        pf.mul(fout, plan, alms[k])
        pf.mul(aout, plan.H, fins[k])

    for i in range(warmup):
        step(i)
    torch.cuda.synchronize()
    plan.profile_start(64 * (steps + 2))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(steps):
        step(i)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), plan.profile_stop()


def accuracy(pf, plan, theta, phi, lmax, alm, fin, nsub, rng):
    """Relative l2 error of the forward on a seeded subsample of the points against FP64
    direct evaluation (the library's Direct leaf, which the tests hold to the oracle at 1e-13),
    and the full-size dot-test error <Y a, f> vs <a, Y^H f>."""
    import torch
    dev = alm.device
    f = plan * alm
    a = plan.H * fin
    lhs = torch.vdot(f, fin).item()
    rhs = torch.vdot(alm.T.reshape(-1), a.T.reshape(-1)).item()
    dot = abs(lhs - rhs) / abs(lhs)
    idx = np.sort(rng.choice(len(theta), nsub, replace=False))
    pd = pf.Plan(theta[idx], phi[idx], lmax=lmax, method="direct", device=dev.index)
    fd = pd * alm
    fs = f[torch.from_numpy(idx).to(dev)]
    err = (torch.linalg.vector_norm(fs - fd) / torch.linalg.vector_norm(fd)).item()
    del pd
    return err, dot


def batch_workload(nplans=64, seed=4):
    """Plans of the batched configuration: lmax log-uniform in [128, 1024], cap radius uniform
    in 5-30 degrees, M = round(4 (lmax theta*)^2) points, ntrans uniform in 1..8, tol 1e-6 (the
    mixed form) or 1e-8 (FP64)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nplans):
        L = int(round(np.exp(rng.uniform(np.log(128), np.log(1024)))))
        cap = np.deg2rad(rng.uniform(5.0, 30.0))
        M = max(64, int(round(4 * (L * cap) ** 2)))
        th = np.arccos(1 - (1 - np.cos(cap)) * rng.random(M))
        ph = 2 * np.pi * rng.random(M)
        B = int(rng.integers(1, 9))
        tol = 1e-6 if rng.random() < 0.5 else 1e-8
        out.append((L, th, ph, B, tol))
    return out


def run_batch(args, world, rank, local):
    """--config batch: 64 plans, one launch sequence per plan with default tiles vs the
    autotuned batch graph (both forward + adjoint of every plan per step)."""
    import torch
    from __graft_entry__ import load_package
    pf = load_package()
    import importlib
    autotune = importlib.import_module("pfsht_b200.autotune")
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    specs = batch_workload()
    t0 = time.perf_counter()
    plain = [pf.Plan(th, ph, lmax=L, tol=tol, ntrans=B, precision="mixed" if tol >= 1e-6 else "fp64")
             for (L, th, ph, B, tol) in specs]
    build_plain = time.perf_counter() - t0
    cache = os.path.join("/tmp", f"pfsht_tiles_{os.getpid()}.json")
    t0 = time.perf_counter()
    tuned = [autotune.tuned_plan(th, ph, lmax=L, tol=tol, ntrans=B, cache=cache,
                                 precision="mixed" if tol >= 1e-6 else "fp64")
             for (L, th, ph, B, tol) in specs]
    tune_s = time.perf_counter() - t0
    nclasses = len(json.load(open(cache)))
    alms, fins, fouts, aouts = [], [], [], []
    for p in plain:
        a = pf.zeros_alm(p.lmax, p.ntrans, device=dev)
        a.real.normal_()
        a.imag.normal_()
        f = pf.zeros_field(p.npts, p.ntrans, device=dev)
        f.real.normal_()
        f.imag.normal_()
        alms.append(a)
        fins.append(f)
        fouts.append(pf.zeros_field(p.npts, p.ntrans, device=dev))
        aouts.append(pf.zeros_alm(p.lmax, p.ntrans, device=dev))
    stream = torch.cuda.current_stream(dev)

    def timed(step, n):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    def per_plan():
        for p, a, f, fo, ao in zip(plain, alms, fins, fouts, aouts):
            p.mul(fo, a)
            p.mul_adjoint(ao, f)

    batch = pf.Batch(tuned, nstreams=8)

    def batched():
        batch.forward(fouts, alms)
        batch.adjoint(aouts, fins)

    batch_default = pf.Batch(plain, nstreams=8)

    def batched_default():
        batch_default.forward(fouts, alms)
        batch_default.adjoint(aouts, fins)

    steps = max(3, min(args.steps, 20))
    ms_plain = timed(per_plan, steps)
    ms_batch_default = timed(batched_default, steps)
    ms_batch = timed(batched, steps)
    del batch_default
    info = batch.info()
    triples = sum(p.ring_work() * p.ntrans for p in plain)
    kinds = [p.info["kind"] for p in plain]
    line = {
        "metric": "ms per batch step (fwd+adj of 64 plans)", "value": ms_batch, "unit": "ms",
        "n_gpus": 1, "steps": steps, "warmup": args.warmup, "higher_is_better": False,
        "data": "synthetic", "config": {"workload": "batched: 64 plans, lmax log-uniform in "
                                        "[128, 1024], cap 5-30 deg, M = 4 (lmax theta*)^2, "
                                        "ntrans 1..8, tol 1e-6 (mixed) or 1e-8 (fp64)",
                                        "seed": 4},
        "one_launch_sequence_per_plan_ms": ms_plain, "speedup": ms_plain / ms_batch,
        "batched_default_tiles_ms": ms_batch_default,
        "ns_per_triple_batched": ms_batch * 1e6 / triples,
        "ring_launches": [info["ring_launches_fwd"], info["ring_launches_adj"]],
        "graph_nodes": [info["graph_nodes_fwd"], info["graph_nodes_adj"]],
        "direct_plans": kinds.count("direct"), "mixed_plans": sum(p.info["precision"] == 1 for p in plain),
        "autotune": {"seconds": tune_s, "shape_classes": nclasses}, "plan_build_s": build_plain,
    }
    del batch
    print(json.dumps(line), flush=True)
    return 0


def serve_workload(nplans=32, seed=5):
    """Plans of the serving configuration: lmax cycling through 128..2048, cap radius uniform in
    5-30 degrees, M = round(4 (lmax theta*)^2), alternately FP64 at tol 1e-8 and mixed at 1e-6."""
    rng = np.random.default_rng(seed)
    Ls = (128, 256, 512, 1024, 2048)
    out = []
    for i in range(nplans):
        L = Ls[i % len(Ls)]
        cap = np.deg2rad(rng.uniform(5.0, 30.0))
        M = max(64, int(round(4 * (L * cap) ** 2)))
        th = np.arccos(1 - (1 - np.cos(cap)) * rng.random(M))
        ph = 2 * np.pi * rng.random(M)
        tol, prec = (1e-8, "fp64") if i % 2 == 0 else (1e-6, "mixed")
        out.append((L, th, ph, tol, prec))
    return out


def measure_serving(pf, nreq=160, loads=(0.7, 1.0, 1.5), seed=6):
    """Poisson arrivals of synthesis/adjoint requests (half each) over 32 resident plans, host
    buffers in pinned memory: the serving loop against the unbatched path (each request a
    synchronous host-buffer apply, in arrival order). Loads are multiples of the unbatched
    path's capacity (1 / mean service time)."""
    rng = np.random.default_rng(seed)
    specs = serve_workload()
    t0 = time.perf_counter()
    plans = [pf.Plan(th, ph, lmax=L, tol=tol, precision=prec) for (L, th, ph, tol, prec) in specs]
    build_s = time.perf_counter() - t0
    bufs = []
    for p in plans:
        a = pf.zeros_alm(p.lmax, device="pinned")
        a.real[...] = rng.standard_normal(a.shape)
        f = pf.zeros_field(p.npts, device="pinned")
        f.real[...] = rng.standard_normal(f.shape)
        bufs.append((a, f, pf.zeros_field(p.npts, device="pinned"), pf.zeros_alm(p.lmax, device="pinned")))
    reqs = [(int(rng.integers(len(plans))), bool(rng.integers(2))) for _ in range(nreq)]

    def run_unbatched(arrivals):
        lat = []
        t_start = time.perf_counter()
        for (i, fwd), ta in zip(reqs, arrivals):
            now = time.perf_counter() - t_start
            if now < ta:
                time.sleep(ta - now)
            a, f, fo, ao = bufs[i]
            if fwd:
                plans[i].mul(fo, a)
            else:
                plans[i].mul_adjoint(ao, f)
            lat.append(time.perf_counter() - t_start - ta)
        span = time.perf_counter() - t_start
        return lat, span

    # warm up, then the service time of the unbatched path (back to back)
    run_unbatched([0.0] * nreq)
    lat0, span0 = run_unbatched([0.0] * nreq)
    service = span0 / nreq
    srv = pf.Server(hbm_budget_gb=120, nslots=8)
    ids = [srv.add(p) for p in plans]
    resident = srv.stats()["bytes_resident"]

    def run_server(arrivals):
        rids = []
        t_start = time.perf_counter()
        for (i, fwd), ta in zip(reqs, arrivals):
            now = time.perf_counter() - t_start
            if now < ta:
                time.sleep(ta - now)
            a, f, fo, ao = bufs[i]
            rids.append(srv.submit(ids[i], fwd, a if fwd else f, fo if fwd else ao))
        lat = [srv.wait(r) for r in rids]
        times = [srv.times(r) for r in rids]
        for r in rids:
            srv.release(r)
        span = max(t[2] for t in times) - min(t[0] for t in times)
        return lat, span

    run_server(np.zeros(nreq))
    out = []
    for load in loads:
        rate = load / service
        arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
        lu, su = run_unbatched(arrivals)
        ls, ss = run_server(arrivals)
        pct = lambda v, q: float(np.percentile(np.asarray(v) * 1e3, q))
        out.append({"load": load, "rate_rps": rate,
                    "server": {"p50_ms": pct(ls, 50), "p99_ms": pct(ls, 99), "rps": nreq / ss},
                    "unbatched": {"p50_ms": pct(lu, 50), "p99_ms": pct(lu, 99), "rps": nreq / su}})
    srv.close()
    return {"plans": len(plans), "requests_per_rate": nreq, "hbm_budget_gb": 120,
            "resident_gb": resident / 1e9, "unbatched_service_ms": service * 1e3,
            "plan_build_s": build_s, "rates": out,
            "workload": "32 resident plans (lmax 128..2048, cap 5-30 deg, M = 4 (lmax theta*)^2, "
                        "fp64 at 1e-8 / mixed at 1e-6), Poisson arrivals, half synthesis half "
                        "adjoint, host buffers in pinned memory; unbatched = synchronous "
                        "host-buffer applies in arrival order"}


def run_serve(args, world, rank, local):
    """--config serve: the serving loop alone."""
    import torch
    from __graft_entry__ import load_package
    pf = load_package()
    torch.cuda.set_device(local)
    res = measure_serving(pf)
    mid = res["rates"][1]
    line = {"metric": "serve p50/p99 latency and requests/s", "value": mid["server"]["p99_ms"],
            "unit": "ms (p99 at the unbatched path's capacity)", "n_gpus": 1,
            "higher_is_better": False, "data": "synthetic", "config": {"workload": res["workload"]},
            "serve": res}
    print(json.dumps(line), flush=True)
    return 0


def run_solve(args, world, rank, local):
    """--config solve: solve! (CG) on the device at the headline workload; ms per iteration
    against one fwd+adj apply (the iteration adds two dot products and three vector updates,
    and the host stays out of the loop)."""
    import time

    import torch
    from __graft_entry__ import load_package
    pf = load_package()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    M, theta, phi, rng = workload(args.lmax)
    plan = pf.Plan(theta, phi, lmax=args.lmax, tol=args.tol, precision=args.precision, device=local,
                   fft_lengths=fft_lengths_arg(args.fft_lengths))
    alm = torch.from_numpy(rand_alm_host(args.lmax, rng)).to(dev).permute(2, 1, 0)[:, :, 0]
    f = plan * alm
    fin = pf.zeros_field(M, device=dev)
    aout = pf.zeros_alm(args.lmax, device=dev)
    T_apply, _ = time_applies(pf, plan, [alm], [f], fin, aout, 20, 3, torch.cuda.current_stream(dev))
    ms_apply = T_apply / 20

    def solve_ms(n):
        a = pf.zeros_alm(args.lmax, device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, info = pf.solve(a, plan, f, mode="cg", rtol=1e-30, maxiter=n)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3, info

    solve_ms(2)  # warm-up: workspace, capture, the plan's bounding box for the info
    t_short, i_short = solve_ms(5)
    t_long, i_long = solve_ms(5 + max(100, args.steps // 2))
    per_iter = (t_long - t_short) / (i_long["iters"] - i_short["iters"])
    line = {"metric": "ms per CG iteration (solve!, fwd + adj + 2 dots + 3 updates)",
            "value": per_iter, "unit": "ms", "n_gpus": 1, "higher_is_better": False,
            "data": "synthetic", "dtype": "f64",
            "config": dict(config_dict(args, M), solve="cg, rtol below reach, iterations "
                           f"{i_short['iters']} vs {i_long['iters']} differenced (wall clock)"),
            "ms_per_fwd_adj_apply": ms_apply, "overhead_per_iteration_ms": per_iter - ms_apply,
            "relres_after": i_long["relres"]}
    print(json.dumps(line), flush=True)
    return 0


def rand_spin_alm_host(lmax, spin, rng):
    """Spin coefficients (l, m + lmax) as complex N(0,1)/(l+1) where l >= max(|m|, |s|)."""
    L = lmax
    l = np.arange(L + 1)[:, None]
    m = np.arange(-L, L + 1)[None, :]
    mask = (np.abs(m) <= l) & (l >= abs(spin))
    a = (rng.standard_normal((L + 1, 2 * L + 1)) + 1j * rng.standard_normal((L + 1, 2 * L + 1)))
    return np.asfortranarray(a / np.sqrt(2) / (l + 1) * mask)


def run_spin(args, world, rank, local):
    """--config spin: the spin-s stretched leaf (src/Spin.jl, s = --spin) at the headline
    workload: ms per fwd+adj, stage times, ns per retained (l, m, ring) triple, accuracy against
    the spin Direct leaf on a subsample and the dot test; the CPU restatement of the spin apply
    timed beside it."""
    import torch
    from __graft_entry__ import load_package
    pf = load_package()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    s = args.spin
    M, theta, phi, rng = workload(args.lmax)
    plan = pf.Plan(theta, phi, lmax=args.lmax, tol=args.tol, device=local, spin=s,
                   fft_lengths=fft_lengths_arg(args.fft_lengths))
    info = plan.info
    alms = [torch.from_numpy(np.ascontiguousarray(rand_spin_alm_host(args.lmax, s, rng).T)).to(dev).T
            for _ in range(3)]
    fins = [torch.from_numpy((rng.standard_normal(M) + 1j * rng.standard_normal(M)) / np.sqrt(2)).to(dev)
            for _ in range(3)]
    fout = pf.zeros_field(M, device=dev)
    aout = pf.zeros_alm(args.lmax, device=dev)
    stream = torch.cuda.current_stream(dev)
    n0 = pf._lib.load().pfsht_launch_count()
    T, stages = time_applies(pf, plan, alms, fins, fout, aout, args.steps, args.warmup, stream)
    launches = (pf._lib.load().pfsht_launch_count() - n0) * args.steps // (args.steps + args.warmup)
    ms = T / args.steps
    # accuracy: the spin Direct leaf (FP64, every order on every point) on a seeded subsample
    sub = np.sort(np.random.default_rng(7).choice(M, 4096, replace=False))
    pd = pf.Plan(theta[sub], phi[sub], lmax=args.lmax, tol=args.tol, method="direct", spin=s,
                 device=local)
    f = plan * alms[0]
    fd = pd * alms[0]
    fs = f[torch.from_numpy(sub).to(dev)]
    err = float(torch.linalg.vector_norm(fs - fd) / torch.linalg.vector_norm(fd))
    a = plan.H * fins[0]
    lhs = torch.vdot(f, fins[0]).item()
    rhs = torch.vdot(alms[0].T.reshape(-1), a.T.reshape(-1)).item()
    dot = abs(lhs - rhs) / abs(lhs)
    cpu = None
    if not args.no_cpu:
        from oracle import oracle as O
        nthreads = os.cpu_count() or 1
        S = O.Stretch(theta, phi, args.lmax, args.tol, nufft="es", spin=s)
        ah = rand_spin_alm_host(args.lmax, s, rng)[:, :, None]
        g = np.asfortranarray(fins[0].cpu().numpy()[:, None])
        t0 = time.perf_counter()
        S.forward(ah, nthreads=nthreads)
        S.adjoint(g, nthreads=nthreads)
        cpu = {"value": (time.perf_counter() - t0) * 1e3, "unit": "ms", "cores": nthreads,
               "kind": "port", "sample": "full workload, one spin fwd+adj of the C restatement"}
    line = {"metric": f"ms per spin-{s} fwd+adj apply", "value": ms, "unit": "ms", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "dtype": "f64", "data": "synthetic",
            "config": dict(config_dict(args, M), spin=s,
                           alm="complex N(0,1)/(l+1) where l >= max(|m|, |s|), (l, m + lmax) layout"),
            "ring_work": info["ring_work"], "ns_per_triple": ms * 1e6 / info["ring_work"],
            "stages_ms": {k: round(v[0] / v[1], 4) for k, v in stages.items()},
            "accuracy": {"tol": args.tol, "l2_rel_vs_spin_direct": err, "dot_rel": dot,
                         "sample": "4096 seeded points, spin Direct leaf on the device"},
            "cpu_baseline": cpu, "gpu_launches": launches}
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args, world, rank, local):
    import ctypes as C

    import torch
    from __graft_entry__ import load_package
    pf = load_package()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib = pf._lib.load()

    # FP64 FMA peak on this GPU (the ring pass and NUFFT roof; MEASURED_PEAKS.json has none)
    fl = C.c_double()
    ms = C.c_double()
    pf._lib.check(lib.pfsht_fma_peak(1, 4000, C.byref(fl), C.byref(ms)))
    fp64_peak = fl.value / 1e12

    M, theta, phi, rng = workload(args.lmax)
    B = args.ntrans
    t0 = time.perf_counter()
    plan = pf.Plan(theta, phi, lmax=args.lmax, tol=args.tol, precision=args.precision,
                   device=local, fft_lengths=fft_lengths_arg(args.fft_lengths), ntrans=B)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    # a second build of the same plan: without the process's one-time costs (library loading,
    # the fine-grid FFT length timing, which is cached per process and shape)
    t0 = time.perf_counter()
    p_again = pf.Plan(theta, phi, lmax=args.lmax, tol=args.tol, precision=args.precision,
                      device=local, fft_lengths=fft_lengths_arg(args.fft_lengths), ntrans=B)
    torch.cuda.synchronize()
    build_warm_s = time.perf_counter() - t0
    del p_again
    info = plan.info
    nset = 3
    alms, fins = [], []
    for _ in range(nset):
        ah = rand_alm_host(args.lmax, rng, B)
        a3 = torch.from_numpy(ah).to(dev).permute(2, 1, 0)
        alms.append(a3[:, :, 0] if B == 1 else a3)
        fh = (rng.standard_normal((B, M)) + 1j * rng.standard_normal((B, M))) / np.sqrt(2)
        f2 = torch.from_numpy(fh).to(dev).T  # (M, B), column-major
        fins.append(f2[:, 0] if B == 1 else f2)
    fout = pf.zeros_field(M, B, device=dev)
    aout = pf.zeros_alm(args.lmax, B, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(i):
        k = i % nset
        pf.mul(fout, plan, alms[k])
        pf.mul(aout, plan.H, fins[k])

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    n0 = lib.pfsht_launch_count()
    plan.profile_start(64 * (args.steps + 2))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(args.steps):
        step(i)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = lib.pfsht_launch_count() - n0
    stages = plan.profile_stop()
    clk = clocks.stop()
    T = e0.elapsed_time(e1)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([T], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        T = float(t.item())
        c = torch.tensor([launches], device=dev, dtype=torch.int64)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
        launches = int(c.item())

    # end to end through the public API with pinned host buffers
    ah = torch.from_numpy(rand_alm_host(args.lmax, rng, B)).pin_memory()
    sq = (lambda x: x[:, :, 0]) if B == 1 else (lambda x: x)
    a_host = sq(ah.numpy().transpose(2, 1, 0))
    fq = (lambda x: x[:, 0]) if B == 1 else (lambda x: x)
    f_in = fq(torch.from_numpy(rng.standard_normal((B, M)) + 1j * rng.standard_normal((B, M)))
              .pin_memory().numpy().T)
    f_out = fq(torch.zeros((B, M), dtype=torch.complex128).pin_memory().numpy().T)
    a_out = sq(torch.zeros(ah.shape, dtype=torch.complex128).pin_memory().numpy().transpose(2, 1, 0))
    ne2e = max(3, min(args.steps, 10))

    # each step: the adjoint and the forward issued back to back through the asynchronous
    # host-buffer entry points (their inputs are independent), then one wait for both results.
    # The adjoint goes first: its field upload is the smaller one and its compute the longer,
    # so the forward's coefficient upload overlaps it and the link stays busy both ways
    def e2e_steps(adjoint_first):
        def one():
            if adjoint_first:
                plan.mul_adjoint_async(a_out, f_in)
                plan.mul_async(f_out, a_host)
            else:
                plan.mul_async(f_out, a_host)
                plan.mul_adjoint_async(a_out, f_in)
            plan.host_sync()
        for _ in range(2):
            one()
        t0 = time.perf_counter()
        for _ in range(ne2e):
            one()
        return (time.perf_counter() - t0) * 1e3 / ne2e
    e2e_ms = e2e_steps(True)
    e2e_fwd_first_ms = e2e_steps(False)
    # the same with the synchronous entry points: each call returns with its result
    for _ in range(2):
        plan.mul(f_out, a_host)
        plan.mul_adjoint(a_out, f_in)
    t0 = time.perf_counter()
    for _ in range(ne2e):
        plan.mul(f_out, a_host)
        plan.mul_adjoint(a_out, f_in)
    e2e_sync_ms = (time.perf_counter() - t0) * 1e3 / ne2e
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
        t = torch.tensor([e2e_sync_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_sync_ms = float(t.item())
        t = torch.tensor([e2e_fwd_first_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_fwd_first_ms = float(t.item())

    # accuracy of this form, then the mixed form at tol 1e-6 on the same points and inputs
    acc_rng = np.random.default_rng(7)
    if B == 1:
        err, dot = accuracy(pf, plan, theta, phi, args.lmax, alms[0], fins[0], 4096, acc_rng)
    else:
        # several transforms: the dot test of every column (the l2 error is a B = 1 figure)
        err = None
        fB, aB = plan * alms[0], plan.H * fins[0]
        dot = max(abs(torch.vdot(fB[:, b], fins[0][:, b]).item()
                      - torch.vdot(alms[0][:, :, b].T.reshape(-1), aB[:, :, b].T.reshape(-1)).item())
                  / abs(torch.vdot(fB[:, b], fins[0][:, b]).item()) for b in range(B))
    mixed = None
    if not args.no_mixed and args.precision == "fp64" and B == 1:
        pm = pf.Plan(theta, phi, lmax=args.lmax, tol=1e-6, precision="mixed", device=local)
        Tm, st_m = time_applies(pf, pm, alms, fins, fout, aout, args.steps, args.warmup, stream)
        em, dm = accuracy(pf, pm, theta, phi, args.lmax, alms[0], fins[0], 4096,
                          np.random.default_rng(7))
        mixed = {"tol": 1e-6, "ms_per_step": Tm / args.steps, "speedup_vs_fp64": T / Tm,
                 "l2_rel_vs_direct": em, "dot_rel": dm, "nufft_w": pm.info["nufft_w"],
                 "ns_per_triple": Tm / args.steps * 1e6 / pm.info["ring_work"],
                 "stages_ms": {k: round(v[0] / v[1], 4) for k, v in st_m.items()},
                 "note": "FP64 recurrence and exponents, FP32 compensated ring sums, FP32 "
                         "NUFFT (w=7); same points, inputs and timing as the headline"}
        del pm
    # the workload's two other readings, timed once to show they do not change the speed:
    # coefficients in the m >= 0 slots only, and points theta* sqrt(u) (the reference's
    # benchmark/calibrate.jl:56 draw) instead of cos(theta) uniform
    variants = None
    if not args.no_variants and world == 1 and B == 1:
        nv = max(20, min(args.steps, 50))
        apos = []
        for a in alms:
            b = a.clone()
            b[:, 1::2] = 0  # columns 2|m| - 1 hold m < 0
            apos.append(b)
        Tp, _ = time_applies(pf, plan, apos, fins, fout, aout, nv, args.warmup, stream)
        rs = np.random.default_rng(4096)
        th2 = THETA_STAR * np.sqrt(rs.random(M))
        ph2 = 2 * np.pi * rs.random(M)
        p2 = pf.Plan(th2, ph2, lmax=args.lmax, tol=args.tol, precision=args.precision, device=local,
                     fft_lengths=fft_lengths_arg(args.fft_lengths))
        Ts, _ = time_applies(pf, p2, alms, fins, fout, aout, nv, args.warmup, stream)
        variants = {"steps": nv,
                    "alm_m_nonneg_ms_per_step": Tp / nv,
                    "points_theta_sqrt_u_ms_per_step": Ts / nv,
                    "points_theta_sqrt_u_ring_work": p2.info["ring_work"],
                    "headline_ms_per_step": T / args.steps}
        del p2
    # the benchmark's smaller configurations (lmax 256 and 1024 on the same cap, M = round(4
    # (lmax theta*)^2)), timed the same way on their own plans
    other_workloads = None
    if not args.no_variants and world == 1 and B == 1 and args.lmax == 2048:
        other_workloads = {}
        for Lw in (256, 1024):
            Mw, thw, phw, rw = workload(Lw)
            pw = pf.Plan(thw, phw, lmax=Lw, tol=args.tol, precision=args.precision, device=local)
            aw = [torch.from_numpy(rand_alm_host(Lw, rw)).to(dev).permute(2, 1, 0)[:, :, 0]
                  for _ in range(nset)]
            fw = [torch.from_numpy((rw.standard_normal(Mw) + 1j * rw.standard_normal(Mw))
                                   / np.sqrt(2)).to(dev) for _ in range(nset)]
            fo = pf.zeros_field(Mw, device=dev)
            ao = pf.zeros_alm(Lw, device=dev)
            nw = 100
            Tw, stw = time_applies(pf, pw, aw, fw, fo, ao, nw, args.warmup, stream)
            other_workloads[f"lmax{Lw}"] = {
                "npts": Mw, "ms_per_step": Tw / nw, "steps": nw, "ring_work": pw.info["ring_work"],
                "ns_per_triple": Tw / nw * 1e6 / pw.info["ring_work"],
                "stages_ms": {k: round(v[0] / v[1], 4) for k, v in stw.items()}}
            del pw
    serve = None
    if not args.no_serve and world == 1 and B == 1:
        serve = measure_serving(pf)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()

    if rank != 0:
        return 0

    ms_per_step = T / args.steps
    # each rank runs its own replica of the workload: the time of one fwd+adj (max over ranks)
    value = ms_per_step
    # roofline of the dominant stage of our kernels
    ours = {k: v for k, v in stages.items() if not k.startswith("fft_")}
    dom = max(ours, key=lambda k: ours[k][0])
    dom_ms = ours[dom][0] / ours[dom][1]
    flops, byts = stage_work(info, dom, B)
    hbm, hbm_source = hbm_peak()
    traffic = load_traffic().get(dom)
    if flops / (fp64_peak * 1e12) >= byts / (hbm * 1e9):
        achieved = flops / (dom_ms * 1e-3) / 1e12
        roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak}
    else:
        achieved = byts / (dom_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm}
    roof.update({"kernel": dom, "ms_per_launch": dom_ms, "traffic": traffic,
                 "traffic_source": "stored ncu figure (profiles/traffic_per_launch.json: "
                                   "dram__bytes_read.sum + dram__bytes_write.sum per launch of "
                                   "this kernel at this workload), not measured in this run"
                 if traffic is not None else None,
                 "peak_source": "FP64 FMA microbenchmark pfsht_fma_peak run in this bench "
                                "(MEASURED_PEAKS.json has no FP64 figure)"
                 if roof["bound"] == "fp64" else hbm_source})
    stage_ms = {k: round(v[0] / v[1], 4) for k, v in stages.items()}

    cpu = None
    acc_oracle = None
    if world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        t_cpu, _, _ = cpu_port_apply_time(args.lmax, args.tol, nthreads, napply=2)
        t_ser, _, _ = cpu_port_apply_time(args.lmax, args.tol, 1, napply=1)
        cpu = {"value": t_cpu * 1e3, "unit": "ms", "cores": nthreads, "kind": "port",
               "sample": f"full workload (lmax {args.lmax}, M {M}), best of 2 fwd+adj applies of "
                         "the C restatement of the reference's CPU apply, OpenMP",
               "serial_ms": t_ser * 1e3,
               "serial_sample": "the same workload, one fwd+adj apply on 1 thread",
               "published_reference": {
                   "synthesis_only_ms": {"serial": 538.0, "threads_4": 245.0},
                   "source": "README.md:44 of the reference (lmax 2048, M 2.0e6, tol 1e-8, "
                             "FINUFFT, 4 physical cores; synthesis alone, no adjoint)"}}
        # the oracle checks the device result: FP64 direct evaluation of the same coefficients
        # on a seeded subsample (the CPU leg is where the oracle runs)
        if B == 1:
            from oracle import oracle as O
            sub = np.sort(np.random.default_rng(11).choice(M, 1024, replace=False))
            a_h = np.asfortranarray(alms[0].cpu().numpy())[:, :, None]
            fd = O.Direct(theta[sub], phi[sub], args.lmax).forward(a_h, nthreads=nthreads)[:, 0]
            fs = (plan * alms[0]).cpu().numpy()[sub]
            acc_oracle = float(np.linalg.norm(fs - fd) / np.linalg.norm(fd))

    hb = plan.host_bytes()
    line = {
        "metric": "ms per fwd+adj apply", "value": value, "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": dict(config_dict(args, M), nufft_lengths=[info["nf1"], info["nf2"]],
                       fft_lengths=args.fft_lengths),
        "ns_per_triple": ms_per_step * 1e6 / (info["ring_work"] * B),
        "ms_forward": sum(v[0] / v[1] for k, v in stages.items() if k in FWD_STAGES),
        "ms_adjoint": sum(v[0] / v[1] for k, v in stages.items() if k not in FWD_STAGES),
        "ring_work": info["ring_work"],
        "plan_build_s": build_s,
        "plan_build_warm_s": build_warm_s,
        "roofline": roof,
        "stages_ms": stage_ms,
        "stages_roofline": stage_rooflines(info, stages, fp64_peak, hbm, B),
        "accuracy": {"tol": args.tol, "l2_rel_vs_direct": err, "dot_rel": dot,
                     "sample": "4096 seeded points, FP64 direct evaluation on the device",
                     "l2_rel_vs_oracle_direct": acc_oracle,
                     "oracle_sample": "1024 seeded points, the CPU oracle's Direct leaf"},
        "workloads": other_workloads,
        "mixed": mixed,
        "variants": variants,
        "serve": serve,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_ms, "unit": "ms",
                "h2d_bytes_per_step": hb["h2d_forward"] + hb["h2d_adjoint"],
                "d2h_bytes_per_step": hb["d2h_forward"] + hb["d2h_adjoint"],
                "sync_value": e2e_sync_ms,
                "forward_first_value": e2e_fwd_first_ms,
                "note": "host-buffer C-ABI applies, pinned memory, wall clock per step: "
                        "pfsht_adjoint_host_async and pfsht_forward_host_async issued back to back "
                        "(independent inputs) and one pfsht_host_sync, so one direction's copies "
                        "overlap the other's compute; forward_first_value: the same with the "
                        "forward issued first; sync_value: the synchronous "
                        "pfsht_forward_host / pfsht_adjoint_host one after the other. The "
                        "coefficient array crosses PCIe as its sph_mode staircase of the retained "
                        "orders m <= mmax, in blocks of orders whose ring pass overlaps the next "
                        "block's copy; the field whole"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--lmax", type=int, default=2048)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--ntrans", type=int, default=1, help="transforms per plan (headline config)")
    ap.add_argument("--fft-lengths", default="timed",
                    help='NUFFT fine-grid FFT lengths: "timed" (plan default), "minimal" or N1xN2')
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-form measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving measurement")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the m >= 0 and theta* sqrt(u) workload variants")
    ap.add_argument("--config", default="headline",
                    choices=["headline", "batch", "serve", "solve", "spin"],
                    help="headline (default): the lmax 2048 cap; batch: 64 plans in one graph; "
                         "serve: the request loop; solve: CG iterations of solve!; spin: the "
                         "spin-s leaf on the headline workload")
    ap.add_argument("--spin", type=int, default=2, help="spin weight of --config spin")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        return run_reference(args, world, rank)
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.config == "batch":
            return run_batch(args, world, rank, local) if rank == 0 else 0
        if args.config == "serve":
            return run_serve(args, world, rank, local) if rank == 0 else 0
        if args.config == "solve":
            return run_solve(args, world, rank, local) if rank == 0 else 0
        if args.config == "spin":
            return run_spin(args, world, rank, local) if rank == 0 else 0
        return run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
