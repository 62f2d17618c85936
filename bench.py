"""Benchmark: maxLq Riemannian CG iterations per second on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n 512] [--q 4]
    python bench.py --impl reference ...      # the reference algorithm on the host cores

A step is one full CG iteration of maxdLqdt (optimization.f90:136-446):
GradL2ForLq, Hilbert gradient, tangent projection, Polak-Ribiere beta, the
mnbrak + Brent line search (each trial a full R evaluation), two vector
transports and the retraction.  Workload: N = 512^3, q = 4, B = 1, seeded
divergence-free field with spectrum |j|^-2 exp(-(|j|/(N/32))^2) (synthetic:
the reference ships no input fields).  The headline value is the
mixed-precision path (FP32 fields and FFTs, FP64 state, reductions and
control); the all-FP64 path is timed the same way and reported beside it.

With N > 1 (torchrun) every rank runs an independent replica (seed = rank):
the path does not shard (one GPU holds the whole box), so value = all ranks'
iterations / the slowest rank's time, and there is no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CG iters/s at 512³ q=4: mixed vs FP64 GPU (rel ΔR≤1e-6); FFT HBM GB/s"
# The calls one CG iteration of the reference makes at q >= 4
# (optimization.f90:136-446), each timed as a whole reference-order call of
# the CPU port; the line search adds n_evals calls of eval_J("LineMin")
# (mnbrak 613-778 and brent 784-951).
REF_CALLS = (
    ("GradL2ForLq", 1),                  # 146
    ("HilbertGradient", 2),              # 151, 164
    ("divAvg_free", 2),                  # 153, 165
    ("calcConstraintDerivativeL2", 1),   # 162
    ("H inner product", 12),             # 170-171, 180 (2), 189, 213 (2), 226-227, 245-247
    ("divergence", 1),                   # 188
    ("calc0thFourierModes", 2),          # 251, 257
    ("vectorTransport", 2),              # 324-325
    ("rescaleLqNorm", 1),                # 346
    ("eval_J maxdLqdt", 1),              # 349
    ("calc_global_Lq_norm", 1),          # 421
    ("calc_global_dLqdt_inclParts", 1),  # 423
    ("CG algebra", 1),                   # the array updates 177, 213, 240, 329, 344, 432-436
)
TRIAL_CALL = "eval_J LineMin"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--q", type=float, default=4.0)
    ap.add_argument("--no-fp64", action="store_true", help="skip the all-FP64 comparison path")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the summaries of the 64^3 (c1) and 32-instance (c4) configurations in the line")
    ap.add_argument("--profile-detail", action="store_true", help="key x-stage kernel times by fused functor")
    ap.add_argument("--config", default=None, choices=["c1", "c2", "c3", "c4", "c5"],
                    help="run one of the other workload configurations instead of the headline one")
    ap.add_argument("--max-iter", type=int, default=3000, help="iteration cap per B for --config c2")
    ap.add_argument("--c4-iters", type=int, default=5, help="CG iterations per instance for --config c4")
    return ap.parse_args()


class Dist:
    """Rank bookkeeping; torch.distributed only when WORLD_SIZE > 1."""

    def __init__(self):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        return self._reduce(v, "max")

    def sum(self, v: float) -> float:
        return self._reduce(v, "sum")

    def _reduce(self, v, op):
        if not self.pg:
            return v
        import torch

        dev = f"cuda:{self.local}" if torch.cuda.is_available() else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX if op == "max" else self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def pinned_like(a: np.ndarray) -> np.ndarray:
    """A page-locked host copy of a (plain copy when no GPU is present)."""
    import torch
    if not torch.cuda.is_available():
        return np.ascontiguousarray(a.copy())
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    out = t.numpy()
    out[...] = a
    pinned_like.keep.append(t)  # the numpy view does not own the memory
    return out


pinned_like.keep = []


def device_sync():
    try:
        import torch

        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except Exception:
        pass


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes per algorithmic byte of the pass kernels, from full ncu
# captures of one launch each (the column-pair y passes and z inverse at
# 512^3 on the autotuner's scratch arrays, the x stages at 256^3; traffic
# scales with the work of a launch).
TRAFFIC_PER_ALG_BYTE = {"x_fwd": 0.94, "x_inv": 0.91, "y_fwd": 1.01, "y_inv": 0.99, "z_inv": 0.99}


def load_traffic():
    """Per-kernel DRAM-traffic scale factors measured with ncu."""
    return {k: {"dram_bytes_per_alg_byte": v} for k, v in TRAFFIC_PER_ALG_BYTE.items()}


def run_path(ctx, u0, K, W, dist, profile=False):
    """W warm-up iterations then exactly K timed ones on the resident state."""
    ctx.state_load(u0)
    recs = []
    for _ in range(W):
        _, st, r = ctx.state_iterate(1)
        recs += r
    dist.barrier()
    device_sync()
    l0 = ctx.kernel_launches
    if profile:
        ctx.profile(profile)
        ctx.profile_report(reset=True)
    t0 = time.perf_counter()
    timed = []
    for _ in range(K):
        _, st, r = ctx.state_iterate(1)
        timed += r
        if st != 0:
            break
    device_sync()
    wall = time.perf_counter() - t0
    dist.barrier()
    prof = ctx.profile_report(reset=True) if profile else {}
    if profile:
        ctx.profile(False)
    launches = ctx.kernel_launches - l0
    dev = sum(r["seconds"] for r in timed)
    return {"records": timed, "device_s": dev, "wall_s": wall, "launches": launches, "prof": prof,
            "iters": len(timed)}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class RefCallTimer:
    """Whole reference-order calls of the CPU port (oracle/mlq_oracle.cpp,
    OpenMP on every host core) at one grid size, on the seeded workload
    field u (rescaled to B) and a seeded divergence-free direction d."""

    def __init__(self, n, q, threads):
        from oracle.oracle import Oracle
        from oracle.seedfield import seed_field

        self.n, self.q = n, q
        self.o = Oracle(n, q, 1.0, threads=threads)
        self.u = self.o.rescale(self.o.divavg_free(seed_field(n, 0, 2.0, n / 32.0)))
        d = self.o.divavg_free(seed_field(n, 1, 2.0, n / 32.0))
        self.d = d * np.sqrt(self.o.field_inner(self.u, self.u, "H") / self.o.field_inner(d, d, "H"))
        self.tau = 0.05

    def run(self, name):
        o, u, d, q, tau = self.o, self.u, self.d, self.q, self.tau
        t0 = time.perf_counter()
        if name == "GradL2ForLq":
            o.grad_l2(u)
        elif name == "HilbertGradient":
            o.hilbert_gradient(d, 1.5 - 1.0 / q)
        elif name == "divAvg_free":
            o.divavg_free(d)
        elif name == "calcConstraintDerivativeL2":
            o.normal_l2(u)
        elif name == "H inner product":
            o.field_inner(u, d, "H")
        elif name == "divergence":
            o.divergence(d)
        elif name == "calc0thFourierModes":
            o.zeroth_modes(d)
        elif name == "vectorTransport":
            o.vector_transport(u, tau * d, d)
        elif name == "rescaleLqNorm":
            o.rescale(u)
        elif name == "eval_J maxdLqdt":
            o.eval_J(u, "maxdLqdt")
        elif name == "calc_global_Lq_norm":
            o.lq_norm(u)
        elif name == "calc_global_dLqdt_inclParts":
            o.R_parts(u)
        elif name == TRIAL_CALL:
            o.eval_J(u + tau * d, "LineMin")
        elif name == "CG algebra":
            # gradJproj, the normalisation, d1, uvec0, Uvec + tau d1 and the
            # shift of the CG memory: about ten passes over a vector field
            a = u.copy()
            for _ in range(3):
                a = u - tau * d
                a = tau * a
                a = a + tau * d
        elif name == "dealias_scalar":
            o.dealias_scalar(u[0], 2.0)
        else:
            raise KeyError(name)
        return time.perf_counter() - t0


def compose_iteration(t, n_evals):
    """Seconds of one reference CG iteration from whole-call times t[name]."""
    return sum(c * t[name] for name, c in REF_CALLS) + n_evals * t[TRIAL_CALL]


ALL_CALLS = [name for name, _ in REF_CALLS] + [TRIAL_CALL]


def cpu_reference_baseline(n, q, n_evals, threads, sample_n=256, check_n=64):
    """The reference's CG iteration on the host cores, from timed whole calls.

    Every call of one iteration (REF_CALLS and the n_evals line-search trials)
    is timed once as a whole reference-order call at sample_n^3; the sum is
    scaled to n^3 by the measured ratio of a whole dealias_scalar call at n^3
    and at sample_n^3.  The same composition is checked against one fully
    timed reference-order CG iteration (the oracle's maxdLqdt) at check_n^3."""
    out = {}
    small = RefCallTimer(check_n, q, threads)
    t0 = time.perf_counter()
    _, it, _, rec = small.o.maxdlqdt(small.u, max_iter=1, optim_tol=1e-14)
    t_full = time.perf_counter() - t0
    ne_small = rec[0]["n_evals"] if rec else n_evals
    t_small = {k: min(small.run(k) for _ in range(3)) for k in ALL_CALLS}
    out["c1_full_iteration_iters_per_s"] = 1.0 / t_full
    out["c1_composed_over_measured"] = compose_iteration(t_small, ne_small) / t_full
    del small
    mid = RefCallTimer(sample_n, q, threads)
    t_mid = {k: mid.run(k) for k in ALL_CALLS}
    t_dm = min(mid.run("dealias_scalar") for _ in range(2))
    del mid
    if n != sample_n:
        big = RefCallTimer(n, q, threads)
        t_db = min(big.run("dealias_scalar") for _ in range(2))
        del big
    else:
        t_db = t_dm
    ratio = t_db / t_dm
    it_s = compose_iteration(t_mid, n_evals) * ratio
    out["value"] = 1.0 / it_s
    out["size_ratio"] = ratio
    out["calls_s"] = {k: round(v, 4) for k, v in t_mid.items()}
    out["sample"] = (f"the oracle port (reference order, {threads} host threads): every call of one reference CG "
                     f"iteration timed whole at {sample_n}^3 ({', '.join(f'{c} x {k}' for k, c in REF_CALLS)}, "
                     f"{n_evals:.1f} x eval_J LineMin), scaled to {n}^3 by the measured {n}^3/{sample_n}^3 time "
                     f"ratio {ratio:.2f} of a whole dealias_scalar call; composition checked against one fully timed "
                     f"CG iteration at {check_n}^3 (composed/measured "
                     f"{out['c1_composed_over_measured']:.2f})")
    return out


def workload_name(n, q):
    return (f"maxdLqdt CG iteration, N={n}^3, q={q:g}, B=1, seeded spectrum |j|^-2 exp(-(|j|/{n / 32.0:g})^2), "
            "one independent replica per GPU")


def bench_reference(args, dist):
    """--impl reference: the reference's CG iteration on the host cores (the
    reference-order CPU port, every host thread).  Each step times one whole
    reference-order call of the iteration at 256^3 (cycling through every call
    the iteration makes), or a whole dealias_scalar at the workload size and
    at 256^3 for the size ratio; the iteration is composed from the per-call
    means as in cpu_reference_baseline."""
    if dist.rank != 0:
        dist.close()
        return
    n, q = args.n, args.q
    threads = host_cores()
    sample_n = min(256, n)
    mid = RefCallTimer(sample_n, q, threads)
    big = RefCallTimer(n, q, threads) if n != sample_n else mid
    kinds = ALL_CALLS + ["dealias_scalar@big", "dealias_scalar@mid"]
    times = {k: [] for k in kinds}
    step_s = []
    total = args.warmup + args.steps
    # every kind is timed at least once even when there are fewer steps
    order = [kinds[i % len(kinds)] for i in range(max(total, len(kinds)))]
    for i, k in enumerate(order):
        if k == "dealias_scalar@big":
            dt = big.run("dealias_scalar")
        elif k == "dealias_scalar@mid":
            dt = mid.run("dealias_scalar")
        else:
            dt = mid.run(k)
        times[k].append(dt)
        if i >= args.warmup and len(step_s) < args.steps:
            step_s.append(dt)
    mean = {k: statistics.fmean(v) for k, v in times.items()}
    ratio = mean["dealias_scalar@big"] / mean["dealias_scalar@mid"]
    n_evals = REF_TRIALS_PER_ITER
    it_s = compose_iteration(mean, n_evals) * ratio
    value = 1.0 / it_s
    sample = (f"the oracle port (reference order, {threads} host threads): each step one whole call of the "
              f"reference CG iteration at {sample_n}^3, cycling through all of its calls "
              f"({', '.join(f'{c} x {k}' for k, c in REF_CALLS)}, {n_evals} x eval_J LineMin) and a whole "
              f"dealias_scalar at {n}^3 and {sample_n}^3; iteration = sum of the per-call means x counts, scaled "
              f"to {n}^3 by the measured dealias time ratio {ratio:.2f}")
    line = {"metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.fmean(step_s), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload_name(n, q), "n": n, "q": q,
                       "step": "one whole reference-order call (see cpu_baseline.sample); ms_per_step is its mean",
                       "iteration_s": it_s, "calls_s": {k: round(v, 4) for k, v in mean.items()}},
            "cpu_baseline": {"value": value, "unit": "iters/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    dist.close()


# trials per CG iteration of the reference arm's composition: the mean count
# the GPU run measures on this workload (12.3-12.8) is used in our arm's line
REF_TRIALS_PER_ITER = 12


# ---------------------------------------------------------------------------
# Other workload configurations (one JSON line each; rank 0 only)
# ---------------------------------------------------------------------------
def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _rel2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def config_c1(args):
    """All-FP64 CG at N = 64, q = 4, spectrum |j|^-2 exp(-(|j|/4)^2), seed 0,
    B = 1: 50 iterations or relative improvement 1e-8."""
    import maxlq_b200 as mlq

    n, q = 64, 4.0
    with mlq.MaxLq(n, q, 1.0, max_iter=50, optim_tol=1e-8) as c:
        u0 = c.seed_field(0, 2.0, 4.0)
        t0 = time.perf_counter()
        u, iters, st, rec = c.maxdLqdt(u0.copy())
        wall = time.perf_counter() - t0
        R = c.calc_global_dLqdt_inclParts(u)
        lq = c.calc_global_Lq_norm(u)
        div = float(np.abs(c.divergence(u)).max())
    dev = sum(r["seconds"] for r in rec)
    return {"config": "c1", "workload": "maxdLqdt, N=64^3, q=4, B=1, FP64, seed 0, k0=4, 50 iterations or eps=1e-8",
            "iterations": iters, "status": st, "iters_per_s": len(rec) / max(dev, 1e-12), "wall_s": wall,
            "R_final": R.tolist(), "lq_norm_final": lq, "max_abs_div_final": div,
            "J1_trajectory": [r["J1"] for r in rec], "n_evals": [r["n_evals"] for r in rec]}


def config_c2(args):
    """All-FP64 B-continuation at N = 256, q = 4, k0 = 8: B = 1 then five steps
    B <- 1.1 B, each solved to relative improvement 1e-8 from the previous
    optimum (the reference's continuation loop, maxdLpdt.f90:478-512)."""
    import maxlq_b200 as mlq

    n, q = 256, 4.0
    Bs = [1.1 ** k for k in range(6)]
    steps = []
    with mlq.MaxLq(n, q, Bs[0], max_iter=args.max_iter, optim_tol=1e-8) as c:
        u = c.seed_field(0, 2.0, 8.0)
        for B in Bs:
            c.set_B(B)
            t0 = time.perf_counter()
            u, iters, st, rec = c.maxdLqdt(u)
            wall = time.perf_counter() - t0
            R = c.calc_global_dLqdt_inclParts(u)
            steps.append({"B": B, "iterations": iters, "status": st, "R": R.tolist(),
                          "lq_norm": c.calc_global_Lq_norm(u), "wall_s": wall,
                          "device_s": sum(r["seconds"] for r in rec),
                          "last_rel_improvement": (rec[-1]["deltaJ"] / abs(rec[-1]["J1"])) if rec else None})
    return {"config": "c2", "workload": "B-continuation, N=256^3, q=4, FP64, B=1.1^k k=0..5, eps=1e-8",
            "steps": steps}


def config_c3(args):
    """N = 512, q = 6, B = 4, spectrum |j|^-5/3 exp(-(|j|/16)^2): errors of the
    mixed path (FP32 fields and FFTs, FP64 reductions and retraction) against
    the all-FP64 path for R, the L2 gradient and the first betas, and the
    Taylor test of both gradients along a seeded divergence-free direction."""
    import maxlq_b200 as mlq

    n, q, B = 512, 6.0, 4.0
    d = mlq.MaxLq(n, q, B, optim_tol=0.0)
    m = mlq.MaxLq(n, q, B, precision="mixed", optim_tol=0.0)
    u = d.rescaleLqNorm(d.seed_field(0, 5.0 / 3.0, 16.0), B)
    phi = d.divAvg_free(d.seed_field(1, 5.0 / 3.0, 16.0))
    phi *= np.sqrt(d.global_summed_field_inner_product(u, u) / d.global_summed_field_inner_product(phi, phi))
    out = {"config": "c3", "workload": "N=512^3, q=6, B=4, seed 0, |j|^-5/3 exp(-(|j|/16)^2); direction seed 1"}
    R_d, R_m = d.calc_global_dLqdt_inclParts(u), m.calc_global_dLqdt_inclParts(u)
    g_d = d.GradL2ForLq(u)
    g_m = m.GradL2ForLq(u)
    # R_parts = (R, R1 + R2, R3)
    out["rel_err_mixed_vs_fp64"] = {"R": abs(R_m[0] - R_d[0]) / abs(R_d[0]),
                                    "R12_R3": [abs(a - b) / abs(b) for a, b in zip(R_m[1:], R_d[1:])],
                                    "grad_max": _rel(g_m, g_d), "grad_l2": _rel2(g_m, g_d)}
    taylor = []
    ip_d = d.global_summed_field_inner_product(g_d, phi)
    ip_m = m.global_summed_field_inner_product(g_m, phi)
    J_d0, J_m0 = R_d[0], R_m[0]
    del g_d, g_m
    for e in range(1, 8):
        h = 10.0 ** (-e)
        w = u + h * phi
        kd = (d.calc_global_dLqdt_inclParts(w)[0] - J_d0) / (h * ip_d)
        km = (m.calc_global_dLqdt_inclParts(w)[0] - J_m0) / (h * ip_m)
        taylor.append({"h": h, "kappa_fp64": kd, "kappa_mixed": km})
    out["taylor"] = taylor
    # first CG iterations from the same field: beta, tau, J1
    recs = {}
    for name, ctx in (("fp64", d), ("mixed", m)):
        ctx.state_load(u)
        _, st, rec = ctx.state_iterate(3)
        recs[name] = rec
    out["iterations"] = [{"iter": a["iter"], "beta_fp64": a["beta"], "beta_mixed": b["beta"],
                          "tau_fp64": a["tau"], "tau_mixed": b["tau"], "J1_fp64": a["J1"], "J1_mixed": b["J1"]}
                         for a, b in zip(recs["fp64"], recs["mixed"])]
    d.close()
    m.close()
    return out


def c4_instances(count=32, seed=2026):
    """The batched-instance workload: N cycles through {48, 64, 96, 128}, q
    through {3, 4, 6, 8} (every (N, q) pair twice in 32), B log-uniform in
    [0.5, 8], field seed = instance index, spectrum |j|^-2 exp(-(|j|/(N/16))^2)."""
    rng = np.random.default_rng(seed)
    Ns, qs = (48, 64, 96, 128), (3.0, 4.0, 6.0, 8.0)
    out = []
    for i in range(count):
        B = float(np.exp(rng.uniform(np.log(0.5), np.log(8.0))))
        out.append({"seed": i, "n": Ns[i % 4], "q": qs[(i // 4) % 4], "B": B})
    return out


def run_instances(ctxs, fields, iters, concurrent):
    """CG iterations of every context from its field: one at a time, or all at
    once from one host thread per context (each context has its own stream;
    the library releases the interpreter while it runs)."""
    import threading

    res = [None] * len(ctxs)

    def work(j):
        ctxs[j].state_load(fields[j])
        res[j] = ctxs[j].state_iterate(iters)

    t0 = time.perf_counter()
    if concurrent:
        th = [threading.Thread(target=work, args=(j,)) for j in range(len(ctxs))]
        for t in th:
            t.start()
        for t in th:
            t.join()
    else:
        for j in range(len(ctxs)):
            work(j)
    return time.perf_counter() - t0, res


def config_c4(args):
    """32 independent instances, mixed precision: aggregate CG iterations/s
    with all instances in flight together (one stream and host thread each)
    against running them one at a time; the per-instance trajectories of the
    two runs must be identical (every reduction is deterministic)."""
    import maxlq_b200 as mlq

    spec = c4_instances()
    K = args.c4_iters
    ctxs = [mlq.MaxLq(s["n"], s["q"], s["B"], precision="mixed", optim_tol=0.0) for s in spec]
    fields = [c.seed_field(s["seed"], 2.0, s["n"] / 16.0) for c, s in zip(ctxs, spec)]
    run_instances(ctxs, fields, 1, concurrent=True)  # buffers, tuning, first-touch
    t_seq, r_seq = run_instances(ctxs, fields, K, concurrent=False)
    t_con, r_con = run_instances(ctxs, fields, K, concurrent=True)
    its_seq = sum(len(r[2]) for r in r_seq)
    its_con = sum(len(r[2]) for r in r_con)
    same = all([x["J1"] for x in a[2]] == [x["J1"] for x in b[2]] for a, b in zip(r_seq, r_con))
    for c in ctxs:
        c.close()
    return {"config": "c4", "workload": "32 instances, N in {48,64,96,128} x q in {3,4,6,8}, B log-uniform [0.5, 8], "
                                        f"mixed precision, {K} CG iterations each",
            "instances": spec, "iters_per_s_one_at_a_time": its_seq / t_seq,
            "iters_per_s_concurrent": its_con / t_con, "speedup": (its_con / t_con) / (its_seq / t_seq),
            "iterations": its_con, "identical_trajectories": same,
            "timing": "host wall clock around all instances' iterations (each iteration ends in a stream sync)"}


def config_c5(args):
    """The largest single-GPU size: N = 1024, q = 4, B = 16, spectrum
    |j|^-5/3 exp(-(|j|/32)^2), FP32 fields with FP64 reductions and state; 10
    full CG iterations timed with per-kernel device time.  At this size the
    engine runs in z-slab streaming mode (no N^3 field kept resident)."""
    import maxlq_b200 as mlq

    n, q, B = 1024, 4.0, 16.0
    K, W = args.steps, min(args.warmup, 1)
    # host side: the seeded field (26 GB) and pinned transfer staging (9 GB)
    avail = 0
    with open("/proc/meminfo") as fh:
        for line in fh:
            if line.startswith("MemAvailable:"):
                avail = int(line.split()[1]) * 1024
    if avail < 96 * 2**30:
        return {"config": "c5", "skipped": f"needs about 96 GiB of free host memory, {avail / 2**30:.0f} GiB available"}
    peak, peak_kind = load_peaks()
    c = mlq.MaxLq(n, q, B, precision="mixed", optim_tol=0.0)
    u0 = c.seed_field(0, 5.0 / 3.0, 32.0)
    c.state_load(u0)
    del u0
    for _ in range(W):
        c.state_iterate(1)
    c.profile(True)
    c.profile_report(reset=True)
    t0 = time.perf_counter()
    _, st, rec = c.state_iterate(K)
    wall = time.perf_counter() - t0
    prof = c.profile_report(reset=True)
    c.profile(False)
    dev = sum(r["seconds"] for r in rec)
    per_kernel = {k: {"launches": v["launches"], "ms": round(v["ms"], 2),
                      "GB/s": round(v["bytes"] / max(v["ms"], 1e-9) / 1e6, 1),
                      "frac_of_peak": round(v["bytes"] / max(v["ms"], 1e-9) / 1e6 / peak, 3)} for k, v in prof.items()}
    out = {"config": "c5", "workload": "N=1024^3, q=4, B=16, seed 0, |j|^-5/3 exp(-(|j|/32)^2), mixed precision",
           "iterations": len(rec), "status": st, "iters_per_s": len(rec) / max(dev, 1e-12), "wall_s": wall,
           "device_bytes": c.device_bytes, "kernels": c.kernel_config(), "peak_gbs": peak, "peak_kind": peak_kind,
           "J1": [r["J1"] for r in rec], "n_evals": [r["n_evals"] for r in rec], "per_kernel": per_kernel}
    c.close()
    return out


def main():
    args = parse()
    dist = Dist()
    if args.impl == "reference":
        return bench_reference(args, dist)
    if args.config:
        if dist.rank == 0:
            fn = {"c1": config_c1, "c2": config_c2, "c3": config_c3, "c4": config_c4, "c5": config_c5}[args.config]
            print(json.dumps(fn(args)), flush=True)
        dist.close()
        return

    import maxlq_b200 as mlq

    n, q, K, W = args.n, args.q, args.steps, args.warmup
    k0 = n / 32.0
    dev = dist.local
    seed = dist.rank
    peak, peak_kind = load_peaks()

    mixed = mlq.MaxLq(n, q, 1.0, precision="mixed", device=dev, optim_tol=0.0)
    u0 = mixed.seed_field(seed, 2.0, k0)

    clocks = ClockSampler(dev)
    clocks.start()
    res_m = run_path(mixed, u0, K, W, dist, profile=2 if args.profile_detail else True)
    clk = clocks.stop()

    # the all-FP64 path, and the accuracy of the mixed path against it on the
    # same field: relative |R_mixed - R_fp64| / |R_fp64|
    res_d, rel_dR, acc = None, None, {}
    if not args.no_fp64:
        fp64 = mlq.MaxLq(n, q, 1.0, precision="fp64", device=dev, optim_tol=0.0)
        res_d = run_path(fp64, u0, K, W, dist)
        # after the timed iterations: R of the mixed path's own state, by the
        # mixed and by the FP64 pipeline
        u_end = mixed.state_store()
        R_mK, _ = mixed.state_R()
        fp64.state_load(u_end)
        fp64.state_iterate(0)  # the pre-loop steps only (rescale, projection)
        R_dK, _ = fp64.state_R()
        acc["rel_dR_mixed_vs_fp64_after_timed"] = abs(R_mK[0] - R_dK[0]) / abs(R_dK[0])
        # at the start (u0 after the pre-loop steps), and against the oracle
        fp64.state_load(u0)
        fp64.state_iterate(0)
        R_d0, _ = fp64.state_R()
        mixed.state_load(u0)
        mixed.state_iterate(0)
        R_m0, _ = mixed.state_R()
        rel_dR = abs(R_m0[0] - R_d0[0]) / abs(R_d0[0])
        fx = os.path.join(ROOT, "tests", "golden", f"headline_n{n}_q{q:g}.npz")
        if seed == 0 and os.path.exists(fx):
            R_or = float(np.load(fx)["R_parts"][0])
            acc["rel_dR_mixed_vs_oracle_iter0"] = abs(R_m0[0] - R_or) / abs(R_or)
            acc["rel_dR_fp64_vs_oracle_iter0"] = abs(R_d0[0] - R_or) / abs(R_or)
        fp64.close()

    # e2e: each step copies u host->device from pinned host memory, iterates
    # once, copies u back (the library DMAs a pinned buffer directly)
    e2e = None
    if not args.no_e2e:
        uh = pinned_like(u0)
        mixed.state_load(uh)
        for _ in range(min(W, 1)):
            mixed.state_step(uh)
        dist.barrier()
        device_sync()
        t0 = time.perf_counter()
        ke = 0
        for _ in range(K):
            st, _ = mixed.state_step(uh)
            ke += 1
            if st != 0:
                break
        device_sync()
        te = dist.max(time.perf_counter() - t0)
        e2e = {"value": dist.world * ke / te, "unit": "iters/s", "h2d_bytes_per_step": int(uh.nbytes),
               "d2h_bytes_per_step": int(uh.nbytes)}

    # whole-job throughput: all ranks' iterations over the slowest rank's device time
    t_m = dist.max(res_m["device_s"])
    value = dist.world * res_m["iters"] / t_m
    fp64_value = (dist.world * res_d["iters"] / dist.max(res_d["device_s"])) if res_d else None

    # roofline of the dominant kernel (live CUDA-event timing of the timed region)
    prof = res_m["prof"]
    top = max(prof.items(), key=lambda kv: kv[1]["ms"]) if prof else (None, None)
    traffic = load_traffic()
    roof = None
    if top[0]:
        name, st = top
        achieved = st["bytes"] / (st["ms"] * 1e-3) / 1e9
        per_launch_bytes = st["bytes"] / max(st["launches"], 1)
        tr = traffic.get(name)
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (tr["dram_bytes_per_alg_byte"] * per_launch_bytes) if tr else None,
                "kernel": name, "peak_kind": peak_kind,
                "share": st["ms"] / sum(v["ms"] for v in prof.values()),
                "alg_bytes_per_launch": per_launch_bytes}

    n_evals = [r["n_evals"] for r in res_m["records"]]
    cpu = None
    if dist.rank == 0 and not args.no_cpu:
        threads = host_cores()
        ne = float(np.mean(n_evals)) if n_evals else REF_TRIALS_PER_ITER
        cb = cpu_reference_baseline(n, q, ne, threads, sample_n=min(256, n))
        cpu = {"value": cb["value"], "unit": "iters/s", "cores": threads, "kind": "port", "sample": cb["sample"],
               "c1_full_iteration_iters_per_s": cb["c1_full_iteration_iters_per_s"],
               "c1_composed_over_measured": cb["c1_composed_over_measured"], "calls_s": cb["calls_s"]}

    # the small configurations, summarised in the same line (rank 0)
    configs = None
    if dist.rank == 0 and not args.no_configs:
        configs = {}
        c1 = config_c1(args)
        configs["c1"] = {k: c1[k] for k in ("workload", "iterations", "status", "iters_per_s", "R_final",
                                              "lq_norm_final", "max_abs_div_final")}
        c4 = config_c4(args)
        configs["c4"] = {k: c4[k] for k in ("workload", "iters_per_s_one_at_a_time", "iters_per_s_concurrent",
                                              "speedup", "iterations", "identical_trajectories", "timing")}

    kcfg = mixed.kernel_config()
    per_kernel = {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                      "GB/s": round(v["bytes"] / max(v["ms"], 1e-9) / 1e6, 1)} for k, v in prof.items()}
    if dist.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": dist.world, "steps": K, "warmup": W,
            "ms_per_step": 1000.0 * t_m / max(res_m["iters"], 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": workload_name(n, q),
                       "n": n, "q": q, "precision": "mixed: FP32 fields and FFTs, FP64 state/reductions/control",
                       "fp64_iters_per_s": fp64_value,
                       "mixed_over_fp64": (value / fp64_value) if fp64_value else None,
                       "rel_dR_mixed_vs_fp64": rel_dR, **acc,
                       "line_search_trials_per_iter": float(np.mean(n_evals)) if n_evals else None,
                       "l2": "working set (GBs) far above the 126 MB L2; no flush needed",
                       "parallelism": f"replicas x{dist.world}",
                       "kernels": kcfg},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": res_m["launches"],
            "clocks": clk, "wall_s_timed": res_m["wall_s"], "per_kernel": per_kernel, "configs": configs,
        }
        print(json.dumps(line), flush=True)
    mixed.close()
    dist.close()


if __name__ == "__main__":
    main()
