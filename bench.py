"""Benchmark: CG time-to-solution for the fat+Naik staggered even-odd system.

Workload (one step = one solve): 32^4 lattice, fat+Naik links (fat =
0.8*SU(3) + N(0, 0.2^2) entries, long = SU(3), phases folded in), mass
0.01, Gaussian even-site source, solve stagD2ee(m^2) y = b (QEX's solveEE)
to a true FP64 relative residual of 1e-10 (r2req = 1e-20).  `value` is the
time to solution of the fastest solver configuration on device-resident
inputs; the plain FP64 CG time is reported beside it.  `e2e` is the same
solve through the C ABI with host (QEX-layout) buffers, copies included.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--dims 32,32,32,32]
  python bench.py --rows    (every hot-path row beside the oracle on the host)

With N > 1 (torchrun) the lattice grows with N: 32^3 x (32 N), split along
t into one 32^4 slab per GPU and solved by the domain decomposition's
16-bit CG with NCCL exchanges (weak scaling; --replicas: one independent
32^4 solve per GPU instead); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MASS = 0.01
R2REQ = 1e-20
# FP64 CG iteration count of this workload at 32^4 (seeded fields), as the
# oracle's solve and the GPU FP64 solve both take it.  The CPU reference arm
# cuts its one whole solve into --steps steps of about this count / steps
# iterations; the cpu_baseline of this arm scales its sample by the GPU
# FP64 solve's own count.
FP64_ITERS_32 = 2719
# reliable-update threshold of the mixed-precision solves of the workload
DELTA = 0.1

HBM_FALLBACK_GBS = 6650.0


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def dist_setup(backend="nccl"):
    """One process per GPU (torchrun).  The process group carries the
    barriers around the timed region and the max over ranks of the timings;
    for the domain split also the broadcast of the NCCL id (the library's
    own communicator does the exchanges), or, over gloo, the exchanges
    themselves."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, ws):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_inputs(dims, rank):
    from qex_b200 import fields as F
    g = F.fat_naik_links(dims, 21 + 1000 * rank)
    b = F.even_source(dims, 31 + 1000 * rank)
    return g, b


def cpu_sample(dims, g, b, iters, fp64_iters):
    """Oracle (C, OpenMP, all host threads) FP64 CG sampled for `iters`
    iterations on the full workload; extrapolated to fp64_iters iterations."""
    from oracle import oracle as O
    o = O.Oracle(dims, g)
    y = o.vec()
    o.cg(0, y, b, MASS * MASS, R2REQ, maxits=1)  # warm
    t0 = time.perf_counter()
    its, _ = o.cg(0, y, b, MASS * MASS, R2REQ, maxits=iters)
    dt = time.perf_counter() - t0
    per_it = dt / max(its, 1)
    return per_it * fp64_iters, per_it, its, dt, O.num_threads()


def run_reference(args, dims):
    """The CPU arm: the oracle's FP64 solve (the restatement of QEX's cg.nim
    on stagD2ee, C with OpenMP on all host threads) of the same system, run
    once to convergence.  The solve is cut into steps of a fixed number of
    iterations, sized so that `--steps` steps cover it; every step is timed
    and `value` is their sum, the measured time to solution.  Warm-up steps
    run a few iterations of a separate solve."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return  # the CPU reference arm runs on rank 0 alone
    from oracle import oracle as O
    g, b = make_inputs(dims, 0)
    o = O.Oracle(dims, g)
    m2 = MASS * MASS
    yw = o.vec()
    warm = o.cg_steps(0, yw, b, m2, R2REQ)
    for _ in range(args.warmup):
        warm.run(args.ref_warm_iters)
    warm.end()
    chunk = max(1, -(-args.ref_iters // max(1, args.steps)))
    y = o.vec()
    times = []
    t0 = time.perf_counter()
    run = o.cg_steps(0, y, b, m2, R2REQ)
    while True:
        run.run(chunk)
        done = run.converged or run.iterations >= args.ref_maxits
        if done:
            its, r2_iter = run.end()
            ay = o.vec()
            o.stagD2ee(ay, y, m2)  # the true residual, as solveXX checks it
            r2_true = float(np.linalg.norm(ay[: len(y) // 2] - b[: len(y) // 2]) ** 2
                            / np.linalg.norm(b[: len(y) // 2]) ** 2)
        t1 = time.perf_counter()
        times.append(t1 - t0)
        t0 = t1
        if done:
            break
    val = float(sum(times))
    cores = O.num_threads()
    sample = (f"one whole FP64 CG solve of the oracle (C/OpenMP restatement of QEX cg.nim + stagD2ee, "
              f"{cores} threads) on the full {'x'.join(map(str, dims))} workload from a zero start: "
              f"{its} iterations in {len(times)} timed steps of {chunk} iterations, true r2 {r2_true:.3g}")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "s", "n_gpus": ws,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": val / len(times) * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded numpy: warmSU(0.3) links, Gaussian source)",
            "config": config_dict(dims), "iterations": its, "true_r2": r2_true,
            "steps_requested": args.steps, "iterations_per_step": chunk,
            "cpu_baseline": {"value": val, "unit": "s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


METRIC = "CG time-to-solution, FP64 true residual 1e-10, fat+Naik even-odd, m=0.01"


def config_dict(dims):
    return {"workload": f"fat+Naik staggered even-odd CG, {'x'.join(map(str, dims))}, m={MASS}, "
                        f"Gaussian even source, true r2 <= 1e-20 |b|^2",
            "lattice": list(dims), "mass": MASS, "r2req": R2REQ,
            "reliable_update_delta": DELTA,
            "sloppy_formats": {"fp32": "FP32 links (12-real long links) and vectors",
                               "fp16": "16-bit fixed-point links (12-real long links, one scale per "
                                       "list) and vectors (per-site norm)"},
            "l2": "inputs larger than L2 (links 1.2 GB FP64), no flush needed"}


def timed_solves(s, yd, bd, sp_kw, steps, torch):
    from qex_b200 import stag as S
    times, launches, iters, sps = [], 0, [], []
    for _ in range(steps):
        sp = S.SolverParams(r2req=R2REQ, **sp_kw)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        s.solveEE(yd, bd, MASS, sp)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
        launches += sp.kernel_launches
        iters.append(sp.iterations)
        sps.append(sp)
    return times, launches, iters, sps


def iteration_breakdown(res, k, nh, peak, solver):
    """Where an iteration of the fastest solve goes, from this run's live
    times: the solve's time per iteration against the Schur operator's time
    per call; the rest is the fused update of r, x and p (16-bit solve: r,
    Ap, x in FP32 and p in 16 bits read, r, x and the next p written, 152 B
    per even site, and half sweep 2's read of r for <r, Ap>, 24 B), the
    reliable updates spread over the iterations, and the kernel
    boundaries."""
    it = res["time_s"] / max(res["iterations"], 1)
    rest = it - k["seconds"]
    vec_bytes = {"fp16+fp64": 3 * 24 + 16 + 2 * 24 + 16 + 24, "fp32+fp64": 4 * 24 + 3 * 24,
                 "fp64": 240 + 48 * 4}[solver]
    return {"us_per_iteration": round(it * 1e6, 2), "schur_us": round(k["seconds"] * 1e6, 2),
            "other_us": round(rest * 1e6, 2), "vector_bytes_per_even_site": vec_bytes,
            "vector_GBps_if_all_other_time": round(vec_bytes * nh / max(rest, 1e-12) / 1e9, 1),
            "vector_frac": round(vec_bytes * nh / max(rest, 1e-12) / 1e9 / peak, 4)}


def time_multishift(s, dims, torch):
    """The mixed-precision multi-shift solve on the workload's lattice and
    fields: one Gaussian right-hand side, 12 shifts log-spaced from 1e-4 to
    1 (A + sigma_k, A = stagD2ee(m^2)), true FP64 residual 1e-10 for every
    shift; the SLOPPY_HALF call: FP32 links in the multi-shift iterations,
    then each shift refined by the 16-bit reliable-update CG.  Beside it,
    the same systems by FP64 multi-shift CG and by one plain FP64 CG per
    shift.  One warm-up and one timed call each (CUDA events)."""
    from qex_b200 import fields as F
    from qex_b200 import stag as S
    from qex_b200.multishift_bench import shifts
    V = F.volume(dims)
    sig = shifts(12)
    b = S.to_device_vector(F.even_source(dims, 100))
    ys = [torch.zeros((3, V), dtype=torch.complex128, device="cuda") for _ in sig]

    def timed(fn, reps):
        for i in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            out = fn()
            e1.record()
            torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3, out

    res = {}
    for name, sl in (("mixed_16bit", 2), ("fp64_multishift", 0)):
        sp = S.SolverParams(r2req=R2REQ, sloppySolve=sl, delta=DELTA)
        t, r2 = timed(lambda: s.cgm_ee(MASS, sig, [b], [ys], sp), 2)
        res[name] = {"time_s": t, "iterations": sp.iterations, "max_true_r2": float(r2.max())}

    def separate():
        its, worst = 0, 0.0
        for k, sg in enumerate(sig):
            sp = S.SolverParams(r2req=R2REQ)
            s.solveEE(ys[k], b, float(np.sqrt(MASS * MASS + 0.25 * sg)), sp)
            its += sp.iterations
            worst = max(worst, sp.r2)
        return its, worst

    t, (its, worst) = timed(separate, 1)
    res["fp64_cg_per_shift"] = {"time_s": t, "iterations": its, "max_true_r2": worst}
    m = res["mixed_16bit"]["time_s"]
    return {"workload": f"{'x'.join(map(str, dims))}, m={MASS}, 1 Gaussian right-hand side, 12 shifts "
                        "10^-4..1, true r2 <= 1e-20 per shift", "solvers": res,
            "speedup_vs_fp64_cg_per_shift": res["fp64_cg_per_shift"]["time_s"] / m,
            "speedup_vs_fp64_multishift": res["fp64_multishift"]["time_s"] / m}


def time_stagdn(s, nh, torch, peak):
    """stagDN (FP64 multi-field Dslash) on 1 and 8 fields: device time per
    call and HBM throughput against its compulsory bytes per output site,
    links 16 x 144 B + fields x (48 B own site + 48 B neighbours + 48 B out)."""
    out = {}
    V = 2 * nh
    xs = [torch.randn((3, V), dtype=torch.complex128, device="cuda") for _ in range(8)]
    rs = [torch.zeros_like(x) for x in xs]
    for n in (1, 8):
        for rep in range(2):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(10):
                s.stagDN(0, rs[:n], xs[:n], 0.1)
            e1.record()
            torch.cuda.synchronize()
        t = e0.elapsed_time(e1) * 1e-3 / 10
        byt = (16 * 144 + n * 144) * nh
        out[f"fields_{n}"] = {"us": round(t * 1e6, 1), "GBps": round(byt / t / 1e9, 1),
                              "frac": round(byt / t / 1e9 / peak, 4), "bytes_per_site": 16 * 144 + n * 144}
    return out


def run_rows(args):
    """--rows: each hot-path row of the library on one GPU (device-resident
    inputs, CUDA events on the library's stream) beside the oracle's CPU
    restatement of QEX's code for it, on this box's host threads, on the
    same fields.  Where a whole CPU call takes minutes the CPU leg runs a
    bounded sample and scales it, and says so.  One JSON line."""
    import torch

    from oracle import oracle as O
    from qex_b200 import fields as F
    from qex_b200 import md as MD
    from qex_b200 import smear as SM
    from qex_b200 import stag as S
    from qex_b200.batched_bench import problem_set
    from qex_b200.multishift_bench import shifts
    S.init(0)
    S.set_stream(torch.cuda.current_stream().cuda_stream)

    def gpu(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3 / reps

    def cpu(fn, reps=1):
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            out = fn()
            ts.append(time.perf_counter() - t0)
        return min(ts), out

    rows = {}
    dims = (32, 32, 32, 32)
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 21)
    s = S.Staggered(S.Layout(dims), S.to_device_links(g))
    o = O.Oracle(dims, g)
    # A7: the FP64 Schur operator stagD2ee
    x = F.gaussian_vector(V, 3)
    r = x.copy()
    tc, _ = cpu(lambda: o.stagD2ee(r, x, 1e-4), 3)
    rows["A7 stagD2ee FP64, 32^4 fat+Naik"] = {"gpu_s": s.bench_schur(0, 20, 1e-4), "cpu_s": tc,
                                              "gpu_16bit_s": s.bench_schur(2, 20, 1e-4)}
    # A9: stagDN on 8 fields against 8 oracle stagD2 calls
    xs = [F.gaussian_vector(V, 10 + j) for j in range(8)]
    rs = [v.copy() for v in xs]
    xd = [S.to_device_vector(v) for v in xs]
    rd = [torch.zeros_like(v) for v in xd]
    tg = gpu(lambda: s.stagDN(0, rd, xd, 0.1), 10)
    tc, _ = cpu(lambda: [o.stagD2(0, rr, xx, 0.0, 0.1) for rr, xx in zip(rs, xs)], 2)
    rows["A9 stagDN FP64, 8 fields, 32^4 fat+Naik"] = {"gpu_s": tg, "cpu_s": tc}
    # A14: FP64 multi-shift CG, 12 shifts, one right-hand side
    sig = shifts(12)
    b = F.even_source(dims, 100)
    bd = S.to_device_vector(b)
    ys = [torch.zeros((3, V), dtype=torch.complex128, device="cuda") for _ in sig]
    sp = S.SolverParams(r2req=R2REQ)
    tg = gpu(lambda: s.cgm_ee(MASS, sig, [bd], [ys], sp), 1)
    its_g = sp.iterations
    xo = [o.vec() for _ in sig]
    k = 100
    tc, (its_c, _) = cpu(lambda: o.cgm(0, xo, sig, b, MASS * MASS, R2REQ, maxits=k))
    rows["A14 multi-shift CG FP64, 12 shifts, 32^4"] = {
        "gpu_s": tg, "gpu_iterations": its_g, "cpu_s": tc / max(its_c, 1) * its_g,
        "cpu_sample": f"{its_c} oracle CG-M iterations ({tc:.2f} s), scaled to the GPU's {its_g}"}
    del s, o, ys, xd, rd
    torch.cuda.empty_cache()
    # C3: 64 small lattices, one persistent launch against the oracle's CG per lattice
    stags, bds, ms, probs = [], [], [], problem_set(64)
    for pd, pg, pm, pb in probs:
        stags.append(S.Staggered(S.Layout(pd), S.to_device_links(pg)))
        bds.append(S.to_device_vector(pb))
        ms.append(pm)
    xds = [torch.zeros_like(v) for v in bds]
    S.solve_batched(stags, xds, bds, ms, S.SolverParams(r2req=R2REQ))  # launch configuration
    tg = gpu(lambda: S.solve_batched(stags, xds, bds, ms, S.SolverParams(r2req=R2REQ)), 3)
    tcs = 0.0
    for pd, pg, pm, pb in probs:
        oo = O.Oracle(pd, pg)
        y = oo.vec()
        t, _ = cpu(lambda: oo.cg(0, y, pb, pm * pm, R2REQ))
        tcs += t
        del oo
    rows["C3 64 lattices {8^4, 12^4, 16^4, 8^3x16} to 1e-10"] = {"gpu_s": tg, "cpu_s": tcs}
    del stags, bds, xds
    torch.cuda.empty_cache()
    # A16: the fermion force at 16^4 (solve to 1e-26 and outer products)
    d4 = (16, 16, 16, 16)
    g4 = F.fat_naik_links(d4, 21)
    phi = F.even_source(d4, 33)
    gd4 = S.to_device_links(g4)
    s4 = S.Staggered(S.Layout(d4), gd4)
    fd = torch.zeros_like(gd4)
    phid = S.to_device_vector(phi)
    tg = gpu(lambda: s4.force(fd, phid, 0.05, S.SolverParams(r2req=1e-26)), 2)
    o4 = O.Oracle(d4, g4)
    fo = np.zeros_like(g4)
    tc, _ = cpu(lambda: o4.force(fo, phi, 0.05, 1e-26))
    rows["A16 fermion force, 16^4 fat+Naik, m 0.05"] = {"gpu_s": tg, "cpu_s": tc}
    del s4, o4, fd, gd4
    # F1: HISQ smearing and its chain rule; F4: gauge force, 32^4
    gw = F.apply_phases(dims, F.gauge_warm(dims, 0.3, 17))
    gwd = S.to_device_links(gw)
    lay = S.Layout(dims)
    sm = SM.Smear(lay)
    coef = SM.newHISQ()
    fl, ll = torch.empty_like(gwd), torch.empty_like(gwd)
    tg = gpu(lambda: sm.smear(coef, gwd, fl, ll), 5)
    tc, _ = cpu(lambda: O.hisq_smear(dims, gw))
    rows["F1 HISQ smear, 32^4"] = {"gpu_s": tg, "cpu_s": tc}
    rng = np.random.default_rng(5)
    cf = rng.standard_normal(gw.shape) + 1j * rng.standard_normal(gw.shape)
    cl = np.ascontiguousarray(cf[::-1])
    cfd, cld = S.to_device_links(cf), S.to_device_links(cl)
    dd = torch.empty_like(gwd)
    tg = gpu(lambda: sm.smearDeriv(coef, gwd, cfd, cld, dd), 3)
    tc, _ = cpu(lambda: O.hisq_deriv(dims, gw, cf, cl))
    rows["F1 HISQ chain rule, 32^4"] = {"gpu_s": tg, "cpu_s": tc}
    u = F.gauge_warm(dims, 0.3, 3)
    ud = S.to_device_links(u)
    f = torch.empty_like(ud)
    for name, c1 in (("Wilson", 0.0), ("Symanzik", -1.0 / 12)):
        ga = MD.GaugeAction(lay, 5.6, c1)
        tg = gpu(lambda: ga.force(ud, f), 5)
        tc, _ = cpu(lambda: O.gauge_force(dims, u, 5.6 * (1 - 8 * c1), 5.6 * c1))
        rows[f"F4 gauge force {name}, 32^4"] = {"gpu_s": tg, "cpu_s": tc}
    for v in rows.values():
        v["cpu_over_gpu"] = v["cpu_s"] / v["gpu_s"]
    print(json.dumps({"rows": rows, "cpu_threads": O.num_threads(), "cpu_kind": "port",
                      "device": torch.cuda.get_device_name(0)}), flush=True)


def run_domain(args, dims, ws, rank, local):
    """N > 1: one lattice of dims[0] x dims[1] x dims[2] x (dims[3] N) split
    along t into N slabs of dims, one per rank (weak scaling), solved by the
    domain decomposition's 16-bit reliable-update CG (delta 0.1, FP64 defect
    correction) with its ghost exchanges and sums over NCCL (one GPU per
    rank) or, with --transport host, through host memory over the process
    group (gloo).  Each rank draws its own slab of the fat+Naik field (its
    seed, phases from global coordinates) and of the source.  value: max
    over ranks of the mean device time to solution."""
    import torch
    import torch.distributed as dist

    from qex_b200 import domain as DD
    from qex_b200 import fields as F
    from qex_b200 import stag as S
    gdims = (dims[0], dims[1], dims[2], dims[3] * ws)
    off = (0, 0, 0, dims[3] * rank)
    if args.transport == "nccl":
        obj = [DD.nccl_unique_id() if rank == 0 else None]
        dist.broadcast_object_list(obj, src=0)
        d = DD.DomainSet(gdims, ws, 8, ranks=[rank], nccl_id=obj[0], device=local)
    else:
        d = DD.DomainSet(gdims, ws, 8, ranks=[rank], host_comm=DD.TorchHostComm(), device=local)
    S.set_stream(torch.cuda.current_stream().cuda_stream)
    g = F.fat_naik_slab(gdims, dims, off, 21 + 1000 * rank)
    d.set_links_local([S.to_device_links(g)])
    b_h = F.even_source(dims, 31 + 1000 * rank)
    bd = S.to_device_vector(b_h)
    xd = torch.zeros_like(bd)

    def solve(kw):
        sp = S.SolverParams(r2req=R2REQ, **kw)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        d.solveEE_local([xd], [bd], MASS, sp)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3, sp

    kw16 = {"sloppySolve": 2, "delta": DELTA}
    for _ in range(args.warmup):
        solve(kw16)
    barrier(ws)
    torch.cuda.synchronize()
    times, launches = [], 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            t, sp = solve(kw16)
            times.append(t)
            launches += sp.kernel_launches
    torch.cuda.synchronize()
    barrier(ws)
    value = max_over_ranks(float(np.mean(times)), ws)
    its16, r216 = sp.iterations, sp.r2
    t64, sp64 = solve({"sloppySolve": 0})
    t64 = max_over_ranks(t64, ws)
    # e2e: host buffers in the rank's local V=1 order, copies in the timed region
    bh = np.ascontiguousarray(b_h)
    xh = np.zeros_like(bh)
    e2e_times = []
    for _ in range(max(1, min(args.steps, 3))):
        sp = S.SolverParams(r2req=R2REQ, **kw16)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d.solveEE_local([xh], [bh], MASS, sp)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    e2e = max_over_ranks(float(np.mean(e2e_times)), ws)
    # roofline of the dominant kernel on this rank's slab (the 16-bit Schur
    # operator of the slab's links; the domain solve runs the same kernel on
    # the slab and its ghost slices)
    from qex_b200.kernel_timing import time_schur
    s = S.Staggered(S.Layout(dims), S.to_device_links(g))
    nh = F.volume(dims) // 2
    k = time_schur(s, nh, (2,), nrep=20)["fp16"]
    peak, peak_kind = measured_peaks()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "fp16+fp64",
                "data": "synthetic (seeded numpy per rank: warmSU(0.3) links, Gaussian source)",
                "config": {**config_dict(gdims),
                           "workload": f"fat+Naik staggered even-odd CG, {'x'.join(map(str, gdims))} split along t "
                                       f"into {ws} slabs of {'x'.join(map(str, dims))}, m={MASS}, "
                                       f"Gaussian even source, true r2 <= 1e-20 |b|^2",
                           "parallelism": f"domain decomposition along t, {ws} ranks, {args.transport} exchange"},
                "solver": "fp16+fp64 (domain)", "iterations": its16, "true_r2": r216,
                "fp64_domain_time_s": t64, "fp64_domain_iterations": sp64.iterations,
                "speedup_vs_fp64": t64 / value,
                "roofline": {"kernel": "Schur operator, fp16 fat+Naik, one rank's slab", "bound": "hbm",
                             "achieved": round(k["GBps"], 1), "peak": peak, "unit": "GB/s",
                             "frac": round(k["GBps"] / peak, 4), "peak_source": peak_kind, "traffic": None,
                             "bytes_per_even_site": k["bytes_per_even_site"], "seconds_per_call": k["seconds"]},
                "cpu_baseline": None,
                "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": int(bh.nbytes) // 2,
                        "d2h_bytes_per_step": int(xh.nbytes), "host_memory": "pageable", "per_rank": True},
                "clocks": clk.summary(), "gpu_launches": int(launches)}
        print(json.dumps(line), flush=True)
    del s
    del d


def run_ours(args, dims):
    import torch

    from qex_b200 import fields as F
    from qex_b200 import stag as S
    ws, rank, local = dist_setup("gloo" if args.transport == "host" else "nccl")
    local = local % max(1, torch.cuda.device_count())
    torch.cuda.set_device(local)
    S.init(local)
    if ws > 1 and not args.replicas:
        run_domain(args, dims, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    S.set_stream(torch.cuda.current_stream().cuda_stream)
    g, b = make_inputs(dims, rank)
    V = F.volume(dims)
    nh = V // 2
    lay = S.Layout(dims, device=local)
    s = S.Staggered(lay, S.to_device_links(g))
    bd = S.to_device_vector(b)
    yd = torch.zeros((3, V), dtype=torch.complex128, device="cuda")

    # the workload's solver configurations (reliable updates at delta 0.1);
    # `value` is the fastest of these.  The 16-bit solve at delta 0.3 is
    # timed the same way and reported beside them, not as `value`.
    configs = [("fp64", {"sloppySolve": 0}), ("fp32+fp64", {"sloppySolve": 1, "delta": DELTA}),
               ("fp16+fp64", {"sloppySolve": 2, "delta": DELTA})]
    extra = [("fp16+fp64 delta 0.3", {"sloppySolve": 2, "delta": 0.3})]
    results = {}
    for name, kw in configs + extra:
        # warm-up
        timed_solves(s, yd, bd, kw, args.warmup, torch)
        barrier(ws)
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            times, launches, iters, sps = timed_solves(s, yd, bd, kw, args.steps, torch)
        torch.cuda.synchronize()
        barrier(ws)
        t = max_over_ranks(float(np.mean(times)), ws)
        # true residual of the last solution (FP64, through the library)
        ay = torch.zeros_like(yd)
        s.stagD2ee(ay, yd, MASS * MASS)
        rr = ((ay[:, :nh] - bd[:, :nh]).abs() ** 2).sum().item() / (bd[:, :nh].abs() ** 2).sum().item()
        results[name] = {"time_s": t, "iterations": iters[-1], "true_r2": rr,
                         "outer": sps[-1].outer_iterations, "reliable_updates": sps[-1].reliable_updates,
                         "launches": launches, "clocks": clk.summary()}
    best = min((c[0] for c in configs), key=lambda k: results[k]["time_s"])
    value = results[best]["time_s"]

    # roofline of the dominant kernel: the Schur half sweeps in the precision
    # the fastest solver iterates in, timed with CUDA events in the library
    from qex_b200.kernel_timing import time_schur
    kt = time_schur(s, nh, (0, 1, 2), nrep=20)
    dom = {"fp64": "fp64", "fp32+fp64": "fp32", "fp16+fp64": "fp16"}[best]
    k = kt[dom]
    peak, peak_kind = measured_peaks()
    # DRAM bytes (read + write) of one Schur call = its two half sweeps, from
    # ncu captures of these kernels at 32^4 (per-launch traffic scales with
    # the site count); 16-bit: dslash_x2_kernel half sweep 1 260.08 MB read +
    # 2.93 MB written, half sweep 2 268.49 + 3.95 MB (two launches each)
    ncu_traffic_32 = {"fp64": 1233229000 + 5634048 + 1258927000 + 7406080,
                      "fp32": 515961088 + 7234048 + 528527616 + 5271808,
                      "fp16": 260084500 + 2930000 + 268494000 + 3946500}
    traffic = ncu_traffic_32[dom] * nh / 524288
    roof = {"kernel": f"Schur operator, {dom} fat+Naik (two Dslash half sweeps)", "bound": "hbm",
            "achieved": round(k["GBps"], 1), "peak": peak, "unit": "GB/s",
            "frac": round(k["GBps"] / peak, 4), "peak_source": peak_kind,
            "traffic": traffic, "traffic_unit": "bytes per Schur call (ncu, scaled from 32^4)",
            "bytes_per_even_site": k["bytes_per_even_site"],
            "seconds_per_call": k["seconds"],
            "iteration": iteration_breakdown(results[best], k, nh, peak, best),
            "all_precisions": {n: {"GBps": round(v["GBps"], 1), "frac": round(v["GBps"] / peak, 4),
                                   "GFLOPs": round(v["GFLOPs"], 1), "us": round(v["seconds"] * 1e6, 1),
                                   "GBps_no_reuse": round(v["GBps_no_reuse"], 1),
                                   "no_reuse_bytes_per_even_site": v["no_reuse_bytes_per_even_site"]}
                               for n, v in kt.items()}}
    # the Schur call in SM cycles, so that boxes held at different clocks by
    # the power cap compare (the call is too short to sample on its own)
    sm_mhz = results[best]["clocks"].get("sm_mhz")
    roof["cycles_per_call"] = round(k["seconds"] * sm_mhz * 1e6) if sm_mhz else None
    roof["cycles_clock"] = "median SM clock sampled during the timed headline solves"

    # e2e: the same solve through the C ABI with host buffers in pinned
    # memory: per solve the library copies the source's even half in and
    # the whole solution field out
    bh_t = torch.from_numpy(np.ascontiguousarray(b)).pin_memory()
    yh_t = torch.zeros(b.shape, dtype=torch.complex128).pin_memory()
    bh, yh = bh_t.numpy(), yh_t.numpy()
    kw = configs[[c[0] for c in configs].index(best)][1]
    e2e_times = []
    s.solveEE(yh, bh, MASS, S.SolverParams(r2req=R2REQ, **kw))  # warm-up (staging buffers)
    for i in range(max(1, args.steps)):
        sp = S.SolverParams(r2req=R2REQ, **kw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.solveEE(yh, bh, MASS, sp)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    e2e = max_over_ranks(float(np.mean(e2e_times)), ws)

    multishift = None if args.no_multishift else time_multishift(s, dims, torch)
    stagdn = time_stagdn(s, nh, torch, peak)

    line = None
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu:
            its64 = results["fp64"]["iterations"]
            v, per_it, its, dt, cores = cpu_sample(dims, g, b, args.cpu_iters, its64)
            cpu = {"value": v, "unit": "s", "cores": cores, "kind": "port",
                   "sample": f"{its} FP64 CG iterations of the oracle on the full workload "
                             f"({per_it*1e3:.1f} ms/iteration, {dt:.1f} s), extrapolated to the "
                             f"{its64} iterations the FP64 solve takes"}
        line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if best == "fp64" else best,
                "data": "synthetic (seeded numpy: warmSU(0.3) links, Gaussian source)",
                "config": config_dict(dims), "solver": best,
                "solvers": {k: {kk: vv for kk, vv in v.items() if kk != "clocks"} for k, v in results.items()
                            if k in dict(configs)},
                "solvers_other_delta": {k: {kk: vv for kk, vv in v.items() if kk != "clocks"}
                                        for k, v in results.items() if k not in dict(configs)},
                "fp64_time_s": results["fp64"]["time_s"],
                "speedup_vs_fp64": results["fp64"]["time_s"] / value,
                "roofline": roof, "cpu_baseline": cpu,
                "multishift": multishift, "multi_rhs_dslash": stagdn,
                "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": int(bh.nbytes) // 2,
                        "d2h_bytes_per_step": int(yh.nbytes), "host_memory": "pinned"},
                "clocks": results[best]["clocks"],
                "gpu_launches": int(results[best]["launches"])}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dims", default="32,32,32,32")
    ap.add_argument("--cpu-iters", type=int, default=400,
                    help="oracle CG iterations in the cpu_baseline sample of this arm")
    ap.add_argument("--ref-iters", type=int, default=0,
                    help="expected FP64 iterations of the reference arm's solve (sets its step size)")
    ap.add_argument("--ref-warm-iters", type=int, default=5)
    ap.add_argument("--ref-maxits", type=int, default=100000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-multishift", action="store_true", help="skip the multi-shift comparison")
    ap.add_argument("--rows", action="store_true",
                    help="instead: every hot-path row on the GPU beside the oracle on the host threads")
    ap.add_argument("--transport", default="nccl", choices=["nccl", "host"],
                    help="N > 1: domain exchanges over NCCL, or through host memory over gloo")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: one independent 32^4 solve per GPU instead of the domain split")
    args = ap.parse_args()
    dims = tuple(int(v) for v in args.dims.split(","))
    if args.rows and args.impl == "ours":
        run_rows(args)
        return
    if args.impl == "reference":
        if args.ref_iters <= 0:
            args.ref_iters = FP64_ITERS_32 if dims == (32, 32, 32, 32) else 100 * max(1, args.steps)
        run_reference(args, dims)
    else:
        run_ours(args, dims)


if __name__ == "__main__":
    main()
