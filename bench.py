#!/usr/bin/env python3
"""Benchmark of the colour-gradient LBM step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload ("batch600"): a batched stream of 600 cases drawn from
seed 20261203: square boxes with side log-uniform in 64-512, 80 % static drops (R uniform in 10 to
side/4) and 20 % straight interfaces inclined at atan(q/p), p, q in 1..4; operator uniform over the
seven; tau uniform in 0.51-2; sigma log-uniform in 0.1-2 (A = 9 sigma / 4 tau for class P); FP32
shifted storage -- all advanced together by the batch engine (one CUDA graph of step launches over
the device work table, one CTA per tile).  A "step" is one lattice-Boltzmann time step of every
case.
Beside it, one 4096 x 4096 x 1 static drop (R = 400, P3 chi = 0.5, A = 0.225, tau = 1), the
single-case roofline configuration, in FP32 and in the plain FP64 path (bit-identical to the
reference).

value   MLUPS (million lattice-node updates per second) of the batch, device time from CUDA events
        on the batch's stream around exactly K steps, state resident in HBM (11+ GB, far larger than
        L2, so no flush is needed between steps).
e2e     the same metric through the C ABI as a user runs the batch: itlbm_batch_submit of every case
        (a strip's initial profile is computed on the host and copied up, a drop's on the device),
        advances of up to 500 steps
        with the diagnostics that fall due (each a device-to-host copy of the observables), wall
        clock from the first submit to the last step.
roofline algorithmic bytes per update: 38 populations read + 38 written (304 B in FP32, 608 B in
        FP64) x nodes / mean kernel duration, against the measured copy bandwidth.
fp64_one_at_a_time_mix  the plain FP64 path on the same mixed sweep, one case at a time (every
        10th case of the mix, 40 steps each): the denominator of the batched-vs-plain ratio.
fp64_batched_mix  the same 600-case batch advanced by the batch engine in the plain FP64 path.
latency the served stream (Poisson arrivals, scaled to a bench run) fed into one batch as requests
        arrive, at 70 % of the capacity the batch sustains on that stream (measured first with every
        request submitted at once): p50 / p99 time-to-result, wall clock.
cpu_baseline the reference's own step (Imm_OPS.cpp:252-287, compiled from its sources with its own
        flags into oracle/_ref) on all host cores, on a bounded 1024 x 1024 sample.

Multi-GPU: cases are independent, so N GPUs run N replicas with no collective (weak scaling);
value is the sum of the ranks' node updates over the slowest rank's time.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
PKG_DIR = REPO / "interfacial-tension-operators-lbm_b200"
sys.path.insert(0, str(REPO / "oracle"))  # the CPU baseline legs only


def load_package():
    """Import the package binding (a directory whose name is not an identifier) as `itlbm_b200`."""
    import importlib.util
    if "itlbm_b200" in sys.modules:
        return sys.modules["itlbm_b200"]
    spec = importlib.util.spec_from_file_location("itlbm_b200", PKG_DIR / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["itlbm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod

PEAKS = REPO / "MEASURED_PEAKS.json"
# HBM traffic per node of one FP32 step launch, dram__bytes_read.sum + dram__bytes_write.sum from one
# ncu capture each: a launch over a 100-case subset of the batch mix (1.73 GB for 5 542 507 nodes) and a
# launch over the 4096^2 drop (5.06 GB for 16 777 216 nodes).
TRAFFIC_B_PER_NODE = {"batch600": (912193536 + 813472000) / 5542507, "single": (2552271872 + 2507548928) / 16777216}
HBM_FALLBACK = 6650.0


def hbm_peak():
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def batch_mix(seed=20261203, n=600):
    """The case mix of the batched configuration (see the module docstring)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    ops = [(1, 0.5), (3, -0.4), (3, 0.5), (3, 2.0), (11, 0.5), (12, 0.5), (13, 0.5)]
    cases = []
    for _ in range(n):
        side = int(round(math.exp(rng.uniform(math.log(64), math.log(512)))))
        strip = rng.uniform() < 0.2
        tipo, chi = ops[rng.integers(len(ops))]
        tau = float(rng.uniform(0.51, 2.0))
        sigma = float(math.exp(rng.uniform(math.log(0.1), math.log(2.0))))
        A = 9.0 * sigma / (4.0 * tau) if tipo < 11 else sigma
        p, q = (int(rng.integers(1, 5)), int(rng.integers(1, 5))) if strip else (1, 0)
        radius = float(rng.uniform(10.0, side / 4.0)) if not strip else 0.0
        steps = int(rng.integers(5000, 30001))
        cases.append(dict(nx=side, tipo=tipo, chi=chi, tau=tau, A=A, strip=strip, p=p, q=q, radius=radius,
                          steps=steps))
    return cases


def batch_desc(pkg, c, prec):
    op = pkg.make_op(c["tipo"], c["chi"], 1.569988)
    return pkg.desc(c["nx"], c["nx"], op, tau=c["tau"], beta=0.8, A_fact=c["A"], radius=c["radius"],
                    geometry=pkg.GEOM_STRIP if c["strip"] else pkg.GEOM_DROP, p=c["p"], q=c["q"],
                    precision=prec)


def batch_run(pkg, steps, warmup, world, sample_clocks, local, n_cases=600, prec=None):
    """MLUPS of the batch over exactly `steps` steps of every case (one graph replay)."""
    import torch
    prec = pkg.PREC_F32 if prec is None else prec
    mix = batch_mix(n=n_cases)
    b = pkg.Batch(chunk=steps, diag_every=10 ** 9)
    for k, c in enumerate(mix):
        b.submit(batch_desc(pkg, c, prec), 10 ** 8, k)
    b.advance()  # admission, step 0 and its diagnostic
    st = b.stats()
    # every case is admitted; the stop rule may retire a case at its step-0 diagnostic (as the
    # reference would stop it), so the timed node count is that of the cases still running
    assert st.active + st.finished == n_cases, f"only {st.active + st.finished} of {n_cases} cases admitted"
    b.poll()
    # warm-up: at least `warmup` steps, in whole replays of the graph that is timed (the first full
    # replay also runs the launch-shape autotuning)
    for _ in range(max(1, -(-warmup // steps))):
        b.advance()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    st0 = b.stats()
    sampler = ClockSampler(local) if sample_clocks else None
    if sampler:
        sampler.__enter__()
        time.sleep(0.3)
    b.advance()  # the timed replay: exactly `steps` steps of every case
    torch.cuda.synchronize()
    if sampler:
        sampler.__exit__()
    barrier(world)
    torch.cuda.synchronize()
    st1 = b.stats()
    ms = st1.device_ms - st0.device_ms
    upd = st1.node_updates - st0.node_updates
    assert upd % steps == 0 and st1.active == st0.active
    b.close()
    global LAST_LAUNCH_MODE, LAST_TILING
    LAST_LAUNCH_MODE = st1.launch_mode
    LAST_TILING = st1.narrow_edges
    return upd // steps, ms, (sampler.summary() if sampler else None), st1.active


def served_stream(seed=20261203, n=160):
    """The served-stream configuration, scaled to a bench run: Poisson arrivals of cases with side
    log-uniform in 64-1024, 500-5000 steps (the full stream is 64-2048 and 5 000-100 000 steps),
    10 % FP64, 80 % drops / 20 % inclined strips, operators, tau and sigma as in the batch mix."""
    import numpy as np
    rng = np.random.default_rng(seed + 1)
    ops = [(1, 0.5), (3, -0.4), (3, 0.5), (3, 2.0), (11, 0.5), (12, 0.5), (13, 0.5)]
    reqs = []
    for _ in range(n):
        side = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
        strip = rng.uniform() < 0.2
        tipo, chi = ops[rng.integers(len(ops))]
        tau = float(rng.uniform(0.51, 2.0))
        sigma = float(math.exp(rng.uniform(math.log(0.1), math.log(2.0))))
        A = 9.0 * sigma / (4.0 * tau) if tipo < 11 else sigma
        p, q = (int(rng.integers(1, 5)), int(rng.integers(1, 5))) if strip else (1, 0)
        radius = float(rng.uniform(10.0, side / 4.0)) if not strip else 0.0
        reqs.append(dict(nx=side, tipo=tipo, chi=chi, tau=tau, A=A, strip=strip, p=p, q=q, radius=radius,
                         steps=int(rng.integers(500, 5001)), fp64=bool(rng.uniform() < 0.1)))
    gaps = rng.exponential(1.0, n)
    return reqs, gaps


def stream_capacity(pkg, reqs):
    """MLUPS the batch sustains on the served stream's own mix: every request submitted at once and
    advanced until the last one ends (the tail, where few cases are left, is included)."""
    b = pkg.Batch(chunk=250, diag_every=500)
    t0 = time.perf_counter()
    for k, r in enumerate(reqs):
        b.submit(batch_desc(pkg, r, pkg.PREC_F64 if r["fp64"] else pkg.PREC_F32), r["steps"], k)
    while True:
        b.advance()
        b.poll()
        st = b.stats()
        if st.active == 0 and st.pending == 0:
            break
    wall = time.perf_counter() - t0
    b.close()
    return st.node_updates / wall / 1e6


def served_latency(pkg, load=0.7):
    """Time-to-result of a stream of cases fed into one batch as they arrive (Poisson, offered load
    `load` of the capacity measured on the same stream): from submission to the case's last step and
    diagnostic, wall clock."""
    import numpy as np
    reqs, gaps = served_stream()
    capacity_mlups = stream_capacity(pkg, reqs)
    work = np.mean([r["nx"] ** 2 * r["steps"] for r in reqs])
    rate = load * capacity_mlups * 1e6 / work  # arrivals per second
    arrive = np.cumsum(gaps / rate)
    b = pkg.Batch(chunk=250, diag_every=500)
    t0 = time.perf_counter()
    nxt, lat, done = 0, [], 0
    while done < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and arrive[nxt] <= now:
            r = reqs[nxt]
            b.submit(batch_desc(pkg, r, pkg.PREC_F64 if r["fp64"] else pkg.PREC_F32), r["steps"], nxt)
            nxt += 1
        st = b.stats()
        if st.active == 0 and st.pending == 0:
            if nxt < len(reqs):
                time.sleep(min(0.001, max(0.0, arrive[nxt] - now)))
            continue
        b.advance()
        for e in b.poll():
            if e.kind != pkg.EV_DIAG:
                lat.append(e.t_event - e.t_submit)
                done += 1
    wall = time.perf_counter() - t0
    st = b.stats()
    b.close()
    lat = np.sort(np.array(lat))
    # HBM bytes per node update of the stream, weighted by each request's planned work: 608 B for the
    # FP64 requests, 304 B for the FP32 ones
    planned = [(r["nx"] ** 2 * r["steps"], 608.0 if r["fp64"] else 304.0) for r in reqs]
    bpu = sum(w * b_ for w, b_ in planned) / sum(w for w, _ in planned)
    peak, peak_kind = hbm_peak()
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "max_s": float(lat[-1]), "requests": len(reqs), "offered_load": load,
            "capacity_mlups": capacity_mlups, "bytes_per_update": bpu,
            "capacity_roofline_frac": capacity_mlups * 1e6 * bpu / 1e9 / peak,
            "offered_mlups": load * capacity_mlups,
            "achieved_mlups": st.node_updates / wall / 1e6, "wall_s": wall,
            "workload": "served stream, scaled: Poisson arrivals, side 64-1024, 500-5000 steps, 10% FP64, "
                        "80% drops / 20% strips, 7 operators; offered load relative to the capacity measured "
                        "on the same stream (all requests at once); time-to-result from submission to the "
                        "last step's diagnostic"}


def c5_stream(seed=20261203, n=32):
    """The served-stream configuration at its specified sizes: Poisson arrivals of cases with side
    log-uniform in 64-2048 and 5 000-100 000 steps, 10 % FP64, 80 % drops / 20 % inclined strips,
    operators, tau and sigma as in the batch mix; a bounded number of requests."""
    import numpy as np
    rng = np.random.default_rng(seed + 2)
    ops = [(1, 0.5), (3, -0.4), (3, 0.5), (3, 2.0), (11, 0.5), (12, 0.5), (13, 0.5)]
    reqs = []
    for _ in range(n):
        side = int(round(math.exp(rng.uniform(math.log(64), math.log(2048)))))
        strip = rng.uniform() < 0.2
        tipo, chi = ops[rng.integers(len(ops))]
        tau = float(rng.uniform(0.51, 2.0))
        sigma = float(math.exp(rng.uniform(math.log(0.1), math.log(2.0))))
        A = 9.0 * sigma / (4.0 * tau) if tipo < 11 else sigma
        p, q = (int(rng.integers(1, 5)), int(rng.integers(1, 5))) if strip else (1, 0)
        radius = float(rng.uniform(10.0, side / 4.0)) if not strip else 0.0
        reqs.append(dict(nx=side, tipo=tipo, chi=chi, tau=tau, A=A, strip=strip, p=p, q=q, radius=radius,
                         steps=int(rng.integers(5000, 100001)), fp64=bool(rng.uniform() < 0.1)))
    return reqs, rng.exponential(1.0, n)


def fifo_latency(arrive, service, servers=1):
    """Time-to-result of requests served first come, first served by `servers` identical servers."""
    import heapq
    free = [0.0] * servers
    out = []
    for a, s in zip(arrive, service):
        t = heapq.heappop(free)
        start = max(t, a)
        heapq.heappush(free, start + s)
        out.append(start + s - a)
    return out


def served_latency_c5(pkg, capacity_mlups, load=0.7, n=32):
    """The specified served stream fed into one batch as requests arrive (offered load `load` of the
    capacity the batch reaches on the 600-case mix), time-to-result from submission to the last step's
    diagnostic; beside it, the same arrivals served one case at a time by the plain FP64 path (each
    request's service time from its own CUDA-event-timed FP64 steps, queued first come, first served)."""
    import numpy as np
    import torch
    reqs, gaps = c5_stream(n=n)
    work = np.array([r["nx"] ** 2 * r["steps"] for r in reqs], dtype=float)
    rate = load * capacity_mlups * 1e6 / work.mean()
    arrive = np.cumsum(gaps / rate)
    b = pkg.Batch(chunk=500, diag_every=500)
    t0 = time.perf_counter()
    nxt, lat, done = 0, [], 0
    while done < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and arrive[nxt] <= now:
            r = reqs[nxt]
            b.submit(batch_desc(pkg, r, pkg.PREC_F64 if r["fp64"] else pkg.PREC_F32), r["steps"], nxt)
            nxt += 1
        st = b.stats()
        if st.active == 0 and st.pending == 0:
            if nxt < len(reqs):
                time.sleep(min(0.01, max(0.0, arrive[nxt] - now)))
            continue
        b.advance()
        for e in b.poll():
            if e.kind != pkg.EV_DIAG:
                lat.append(e.t_event - e.t_submit)
                done += 1
    wall = time.perf_counter() - t0
    st = b.stats()
    b.close()
    # the plain FP64 path, one case at a time: each request's own rate over 100 timed steps
    stream = torch.cuda.current_stream()
    service = []
    for r in reqs:
        case = pkg.Case(batch_desc(pkg, r, pkg.PREC_F64))
        case.step(3, stream=stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        case.step(100, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        service.append(e0.elapsed_time(e1) * 1e-3 * r["steps"] / 100.0)
        case.close()
    lat64 = np.array(fifo_latency(arrive, service))
    lat = np.array(lat)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "max_s": float(lat.max()), "requests": len(reqs), "offered_load": load,
            "capacity_mlups": capacity_mlups, "achieved_mlups": st.node_updates / wall / 1e6, "wall_s": wall,
            "node_updates": float(work.sum()), "diag_ms": st.diag_ms,
            "fp64_one_at_a_time": {"p50_s": float(np.percentile(lat64, 50)),
                                   "p99_s": float(np.percentile(lat64, 99)),
                                   "mlups": float(work.sum() / sum(service) / 1e6),
                                   "model": "same arrivals, one FP64 case at a time first come first served; "
                                            "service time of each request from 100 CUDA-event-timed steps of "
                                            "it alone, scaled to its step count"},
            "workload": f"served stream at its specified sizes: {len(reqs)} Poisson arrivals, side 64-2048, "
                        "5000-100000 steps, 10% FP64, 80% drops / 20% strips, 7 operators; offered load "
                        "relative to the batch600 throughput; time-to-result from submission to the last "
                        "step's diagnostic"}, reqs, arrive


def c5_cpu_estimate(reqs, arrive, mlups_1thread, cores):
    """The same requests on the reference's CPU path as rodar_lote.py runs it: one single-threaded
    process per case, `cores` of them at a time, each at the measured one-thread rate of the
    reference's step loop, first come first served (a model, not a run)."""
    import numpy as np
    service = [r["nx"] ** 2 * r["steps"] / (mlups_1thread * 1e6) for r in reqs]
    lat = np.array(fifo_latency(arrive, service, servers=cores))
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "processes": cores, "mlups_per_process": mlups_1thread,
            "model": "the same arrivals, one single-threaded reference process per case on each host core "
                     "(rodar_lote.py's process pool), each at the measured one-thread rate"}


def batch_e2e(pkg, steps, n_cases=600):
    """The batch through the C ABI, wall clock: submit every case, advance until each has run
    `steps` steps (diagnostics every 500 steps fall due on the way), poll the events."""
    import ctypes
    mix = batch_mix(n=n_cases)
    nodes = sum(c["nx"] * c["nx"] for c in mix)
    t0 = time.perf_counter()
    b = pkg.Batch(chunk=500, diag_every=500)
    for k, c in enumerate(mix):
        b.submit(batch_desc(pkg, c, pkg.PREC_F32), steps, k)
    nev = 0
    while True:
        b.advance()
        nev += len(b.poll())
        st = b.stats()
        if st.active == 0 and st.pending == 0:
            break
    dt = time.perf_counter() - t0
    upd = st.node_updates
    b.close()
    diag_rounds = -(-steps // 500)  # diagnostic rounds after step 0: every 500 steps and the last
    # host -> device: each case's descriptor (under 512 B) and work-table entries (8 B a tile), and the
    # initial profile of a strip (one double per distance class; a drop's FP32 profile is formed on
    # the device)
    h2d = sum(512 + 8 * (-(-c["nx"] // 32)) * (-(-c["nx"] // 8)) + (8 * c["nx"] if c["strip"] else 0) for c in mix)
    d2h = nev * ctypes.sizeof(pkg.BatchEvent)
    return {"value": upd / dt / 1e6, "unit": "MLUPS", "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": d2h / steps, "wall_s": dt, "events": nev,
            "device_ms": st.device_ms, "diag_ms": st.diag_ms,
            "diag_ms_per_500_steps": st.diag_ms / (diag_rounds + 1), "admit_ms": st.admit_ms,
            "capture_ms": st.capture_ms, "advance_ms": st.advance_ms,
            "note": "whole batch through itlbm_batch_*, wall clock from creating the batch to the last step: "
                    "case descriptors, work tables and strip profiles up, diagnostics down; unstable cases "
                    "retire early, so node updates are counted, not assumed"}


WORKLOADS = {
    "drop4096": dict(nx=4096, ny=4096, radius=400.0, tipo=3, chi=0.5, xi=1.569988, A=0.225, tau=1.0,
                     beta=0.8, kprof=2.0 * math.log(9.0) / 3.45),
    "drop2048": dict(nx=2048, ny=2048, radius=200.0, tipo=3, chi=0.5, xi=1.569988, A=0.225, tau=1.0,
                     beta=0.8, kprof=2.0 * math.log(9.0) / 3.45),
    "drop1024": dict(nx=1024, ny=1024, radius=100.0, tipo=3, chi=0.5, xi=1.569988, A=0.225, tau=1.0,
                     beta=0.8, kprof=2.0 * math.log(9.0) / 3.45),
}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit())
        mx = max((float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.rows)}


def setup_dist(backend="nccl"):
    """One process per GPU under torchrun: (world, rank, local rank).  The CPU tests of the replica
    path use backend "gloo"."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def _reduce(v, world, op):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def allreduce_max(v, world):
    import torch.distributed as dist
    return _reduce(v, world, dist.ReduceOp.MAX)


def allreduce_sum(v, world):
    import torch.distributed as dist
    return _reduce(v, world, dist.ReduceOp.SUM)


def replica_mlups(updates, ms, world):
    """Whole-job MLUPS of N replicas: every rank's node updates over the slowest rank's device time.
    Returns (mlups, ms_max)."""
    ms_max = allreduce_max(ms, world)
    return allreduce_sum(updates, world) / (ms_max * 1e-3) / 1e6, ms_max


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def make_case(pkg, w, prec):
    op = pkg.make_op(w["tipo"], w["chi"], w["xi"])
    d = pkg.desc(w["nx"], w["ny"], op, tau=w["tau"], beta=w["beta"], A_fact=w["A"], radius=w["radius"],
                 k_profile=w["kprof"], precision=prec)
    return pkg.Case(d)


def fp64_one_at_a_time(pkg, steps=40, every=10):
    """The plain FP64 path on the same mixed sweep, one case at a time as the reference runs it:
    every `every`-th case of the batch mix, each stepped `steps` times alone (CUDA events around its
    steps, creation excluded).  Aggregate MLUPS = all node updates / the sum of the case times."""
    import torch
    mix = batch_mix()[::every]
    upd, ms = 0, 0.0
    stream = torch.cuda.current_stream()
    for c in mix:
        case = pkg.Case(batch_desc(pkg, c, pkg.PREC_F64))
        case.step(3, stream=stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        case.step(steps, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        upd += c["nx"] * c["nx"] * steps
        case.close()
    return {"value": upd / (ms * 1e-3) / 1e6, "unit": "MLUPS", "cases": len(mix), "steps": steps,
            "workload": f"every {every}th case of the batch mix, FP64 plain, one case at a time"}


def device_run(pkg, w, prec, steps, warmup, world, sample_clocks, local):
    """MLUPS of exactly `steps` steps, CUDA events on the launching stream, max over ranks."""
    import torch
    c = make_case(pkg, w, prec)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    c.step(warmup, stream=sp)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local) if sample_clocks else None
    if sampler:
        sampler.__enter__()
        time.sleep(0.3)
    e0.record(stream)
    c.step(steps, stream=sp)
    e1.record(stream)
    torch.cuda.synchronize()
    if sampler:
        sampler.__exit__()
    barrier(world)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    n = w["nx"] * w["ny"]
    c.close()
    return n, ms, (sampler.summary() if sampler else None)


def e2e_run(pkg, w, prec, steps):
    """A whole case through the C ABI with host buffers: create (host profile -> device), steps,
    a diagnostic every 500 steps and at the end (device -> host), destroy.  Wall clock."""
    import ctypes
    t0 = time.perf_counter()
    c = make_case(pkg, w, prec)
    ndiag = 0
    done = 0
    while done < steps:
        chunk = min(500, steps - done)
        c.step(chunk, keep_aux=True)
        done += chunk
        c.diag_drop(done - 1)
        ndiag += 1
    c.close()
    dt = time.perf_counter() - t0
    n = w["nx"] * w["ny"]
    h2d = 8 * n  # the initial profile rho^N(r) per node, double
    d2h = ndiag * ctypes.sizeof(pkg.DropDiag)
    return {"value": n * steps / dt / 1e6, "unit": "MLUPS", "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": d2h / steps, "wall_s": dt}


def host_cpu():
    """Model name and logical core count of the host."""
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count()


def cpu_baseline(threads=0):
    import oracle
    if not oracle.REF_DIR.joinpath("libref_ops_fast.so").exists():
        return None
    nx = 1024
    steps = 8
    mlups, dt, nthr = oracle.time_reference_step(nx, nx, steps=steps, warmup=1, threads=threads)
    # the same loop on one host thread, on a smaller box (a bounded sample)
    n1, s1 = 256, 8
    mlups1, dt1, _ = oracle.time_reference_step(n1, n1, radius=25.0, steps=s1, warmup=1, threads=1)
    model, ncpu = host_cpu()
    return {"value": mlups, "unit": "MLUPS", "cores": nthr, "kind": "reference",
            "sample": f"reference step loop (Imm_OPS.cpp:252-287, oracle/_ref, its own flags), "
                      f"{nx}x{nx} drop P3 chi=0.5, {steps} steps, {nthr} OpenMP threads, {dt:.1f} s",
            "single_thread": {"value": mlups1, "unit": "MLUPS",
                              "sample": f"{n1}x{n1} drop P3 chi=0.5, {s1} steps, 1 thread, {dt1:.1f} s"},
            "host": {"model": model, "logical_cores": ncpu}}


METRIC = "MLUPS & % HBM roofline, batched FP32 vs plain FP64 on 1 B200; p99 case latency"
REF_EVERY = 10  # the reference arm steps every 10th case of the batch mix (60 cases spread over it)


LAST_LAUNCH_MODE = None  # launch shape the batch engine's autotuner chose in the last batch_run
LAST_TILING = None  # and its tiling: 1 narrow tiles at a box's partial last column, 0 32 x 8 throughout


def batch_config(nodes, ncases, world):
    return {"workload": "batch600: 600 cases (seed 20261203), side 64-512 log-uniform, 80% drops / 20% "
                        "inclined strips, 7 operators, tau 0.51-2, sigma 0.1-2, FP32 shifted storage",
            "nodes": nodes, "cases": ncases,
            "l2": "state 11+ GB >> 126 MB L2: no flush needed", "parallelism": f"replicas x{world}"}


def run_reference(args):
    """The reference's own CPU step loop on the host cores, same metric and workload, rank 0 only.
    Each step is one step of each case of a sample spread over the batch mix (every REF_EVERY-th case):
    drops through the Imm_OPS step loop, inclined strips through the Imm_INCL one.  The cases run the
    way the reference runs a batch (rodar_lote.py's pool: one single-threaded run per case, as many at
    a time as there are cores): one host thread per core, each stepping its share of the cases with
    one OpenMP thread, largest cases first; the time is the wall clock of the whole sample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    os.environ["OMP_NUM_THREADS"] = "1"  # before the reference's OpenMP runtime is loaded
    import concurrent.futures
    import oracle
    if args.workload == "batch600":
        mix = batch_mix()
        sample = mix[::REF_EVERY]
        cfg = batch_config(sum(c["nx"] * c["nx"] for c in mix), len(mix), args.gpus)
        names = {1: "P1", 3: "P3", 11: "F1", 12: "F2", 13: "F3"}
        ops = {}
        for c in sample:
            k = names[c["tipo"]] + (f" chi={c['chi']}" if c["tipo"] == 3 else "")
            ops[k] = ops.get(k, 0) + 1
        nstrip = sum(1 for c in sample if c["strip"])
        desc = (f"every {REF_EVERY}th case of the batch mix: {len(sample)} cases, "
                f"{sum(c['nx'] ** 2 for c in sample)} nodes, {len(sample) - nstrip} drops / {nstrip} strips, "
                f"sides {min(c['nx'] for c in sample)}-{max(c['nx'] for c in sample)}, operators "
                + ", ".join(f"{k} x{v}" for k, v in sorted(ops.items())))
    else:
        w = WORKLOADS[args.workload]
        sample = [dict(nx=1024, tipo=w["tipo"], chi=w["chi"], tau=w["tau"], A=w["A"], radius=100.0, strip=False)]
        cfg = {"workload": args.workload, "nodes": w["nx"] * w["ny"], "parallelism": f"replicas x{args.gpus}"}
        desc = f"1024x1024 sample of {args.workload}"
    steppers = []
    for c in sample:
        if c["strip"]:
            steppers.append(oracle.RefStripStepper(c["nx"], c["tipo"], c["p"], c["q"], c["chi"], 1.569988,
                                                   c["tau"], 0.8, c["A"], threads=1))
        else:
            steppers.append(oracle.RefStepper(c["nx"], c["nx"], c["tipo"], c["chi"], 1.569988, c["tau"], 0.8,
                                              c["A"], c["radius"], threads=1))
    nthr = min(os.cpu_count() or 1, len(steppers))
    shares = [[] for _ in range(nthr)]
    load = [0] * nthr
    for r in sorted(steppers, key=lambda r: -r.nodes):  # largest first onto the least loaded thread
        k = load.index(min(load))
        shares[k].append(r)
        load[k] += r.nodes

    def run_all(n):
        with concurrent.futures.ThreadPoolExecutor(nthr) as ex:  # the steps release the interpreter lock
            list(ex.map(lambda sh: [r.step(n) for r in sh], shares))

    run_all(args.warmup)
    t0 = time.perf_counter()
    run_all(args.steps)
    dt = time.perf_counter() - t0
    upd = sum(r.nodes for r in steppers) * args.steps
    for r in steppers:
        r.close()
    mlups = upd / dt / 1e6
    cfg["sample"] = desc
    line = {"impl": "reference", "metric": METRIC, "value": mlups, "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": nthr, "kind": "reference",
                             "sample": f"{desc}; {args.steps} steps each, the reference's step loops "
                                       f"(Imm_OPS.cpp:252-287, Imm_INCL.cpp:364-396; oracle/_ref, its own "
                                       f"flags), one single-threaded case at a time per host thread, "
                                       f"{nthr} threads"},
            "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch600", choices=["batch600"] + sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-latency", action="store_true")
    ap.add_argument("--c5-requests", type=int, default=32, help="requests of the specified served stream (0: skip)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    world, rank, local = setup_dist()
    import torch
    torch.cuda.set_device(local)
    pkg = load_package()
    peak, peak_kind = hbm_peak()

    single = WORKLOADS["drop4096" if args.workload == "batch600" else args.workload]
    if args.workload == "batch600":
        nodes, ms, clocks, ncases = batch_run(pkg, args.steps, args.warmup, world, rank == 0, local)
        mode = LAST_LAUNCH_MODE
        mlups, ms_max = replica_mlups(nodes * args.steps, ms, world)
        achieved = 304.0 * nodes * args.steps / (ms * 1e-3) / 1e9
        launches = args.steps  # one FP32 launch per step; the FP64 table is empty, so nothing is launched for it
        cfg = batch_config(nodes, ncases, world)
        cfg["launch_shape"] = {-1: "one CTA per tile (autotuned)", 0: "persistent CTAs (autotuned)"}.get(mode, mode)
        cfg["tiling"] = {1: "narrow tiles at partial last columns (autotuned)",
                         0: "32x8 tiles throughout (autotuned)"}.get(LAST_TILING, LAST_TILING)
    else:
        nodes, ms, clocks = device_run(pkg, single, pkg.PREC_F32, args.steps, args.warmup, world,
                                       rank == 0, local)
        mlups, ms_max = replica_mlups(nodes * args.steps, ms, world)
        achieved = 304.0 * nodes * args.steps / (ms * 1e-3) / 1e9
        launches = args.steps
        cfg = {"workload": f"{args.workload}: {single['nx']}x{single['ny']}x1 static drop, P3 chi=0.5, FP32",
               "nodes": nodes, "parallelism": f"replicas x{world}"}

    # the single 4096^2 case, FP32 and plain FP64
    ks = max(50, args.steps // 2)
    n1, ms1, _ = device_run(pkg, single, pkg.PREC_F32, ks, args.warmup, world, False, local)
    n64, ms64, _ = device_run(pkg, single, pkg.PREC_F64, ks, args.warmup, world, False, local)
    single32 = {"value": replica_mlups(n1 * ks, ms1, world)[0], "unit": "MLUPS", "steps": ks,
                "roofline_frac": 304.0 * n1 * ks / (ms1 * 1e-3) / 1e9 / peak}
    fp64 = {"value": replica_mlups(n64 * ks, ms64, world)[0], "unit": "MLUPS", "steps": ks,
            "roofline_frac": 608.0 * n64 * ks / (ms64 * 1e-3) / 1e9 / peak,
            "workload": "4096x4096x1 static drop R=400, P3 chi=0.5, FP64 plain (bit-identical to the reference)"}

    fp64_mix = fp64_one_at_a_time(pkg) if args.workload == "batch600" else None
    # the same 600-case batch in the plain FP64 path (bit-identical to the reference): what batching
    # alone gains over one case at a time, at the reference's precision
    fp64_batch = None
    if args.workload == "batch600":
        kb = min(args.steps, 100)
        nb64, msb64, _, ncb64 = batch_run(pkg, kb, args.warmup, world, False, local, prec=pkg.PREC_F64)
        fp64_batch = {"value": replica_mlups(nb64 * kb, msb64, world)[0], "unit": "MLUPS", "steps": kb,
                      "cases": ncb64, "roofline_frac": 608.0 * nb64 * kb / (msb64 * 1e-3) / 1e9 / peak,
                      "workload": "batch600 in the plain FP64 path (bit-identical to the reference)"}
    # the in-plane fold (nine classes per colour, 144 B per update): a separate variant, not the
    # headline D3Q19 number
    fold = None
    if args.workload == "batch600":
        nf, msf, _, ncf = batch_run(pkg, min(args.steps, 200), args.warmup, world, False, local, prec=pkg.PREC_F32_FOLD)
        kf = min(args.steps, 200)
        n4, ms4, _ = device_run(pkg, single, pkg.PREC_F32_FOLD, ks, args.warmup, world, False, local)
        fold = {"batch600_mlups": replica_mlups(nf * kf, msf, world)[0],
                "batch600_roofline_frac": 144.0 * nf * kf / (msf * 1e-3) / 1e9 / peak,
                "single_4096_mlups": replica_mlups(n4 * ks, ms4, world)[0],
                "single_4096_roofline_frac": 144.0 * n4 * ks / (ms4 * 1e-3) / 1e9 / peak,
                "bytes_per_lu": 144.0, "cases": ncf,
                "note": "FP32 storage of the nine in-plane classes of D3Q19 per colour; exact for the "
                        "one-node slab up to rounding; reported beside, never as, the D3Q19 value"}
    e2e = None
    if not args.no_e2e:
        # clocks sampled over the whole end-to-end run (seconds of sustained load, against the
        # headline's short timed region): the power cap lowers the SM clock under sustained load
        e2e_sampler = ClockSampler(local) if rank == 0 else None
        if e2e_sampler:
            e2e_sampler.__enter__()
        e2e = batch_e2e(pkg, 1001) if args.workload == "batch600" else e2e_run(pkg, single, pkg.PREC_F32, args.steps)
        if e2e_sampler:
            e2e_sampler.__exit__()
            e2e["clocks"] = e2e_sampler.summary()
        if world > 1:
            e2e["value"] = allreduce_sum(e2e["value"], world)
    latency = latency_c5 = None
    if not args.no_latency and args.workload == "batch600":
        latency = served_latency(pkg)
        if args.c5_requests > 0:
            latency_c5, c5_reqs, c5_arrive = served_latency_c5(pkg, mlups / world, n=args.c5_requests)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()
        if latency_c5 is not None and cpu is not None:
            latency_c5["reference_cpu"] = c5_cpu_estimate(c5_reqs, c5_arrive, cpu["single_thread"]["value"],
                                                          cpu["host"]["logical_cores"])

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": mlups, "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "bytes_per_lu": 304.0,
                         "traffic": TRAFFIC_B_PER_NODE["batch600" if args.workload == "batch600" else "single"] * nodes,
                         "traffic_note": "bytes per launch: dram__bytes_read.sum + dram__bytes_write.sum of one "
                                         "ncu capture (profiles/k_step_f32_batch100_traffic.md, "
                                         "profiles/k_step_f32_drop4096_traffic.md), per node, times the "
                                         "nodes of one launch"},
            "fp32_single_4096": single32,
            "fp64_plain": fp64,
            "fp64_one_at_a_time_mix": fp64_mix,
            "fp64_batched_mix": fp64_batch,
            "fold_variant": fold,
            "batched_fp32_over_plain_fp64": mlups / fp64["value"],
            "batched_fp32_over_fp64_one_at_a_time_mix": (mlups / fp64_mix["value"]) if fp64_mix else None,
            "gpu_launches": launches,
            "clocks": clocks,
            "e2e": e2e,
            "latency": latency,
            "latency_c5": latency_c5,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
