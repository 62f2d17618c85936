"""Generate the oracle fixtures of the headline workload (512^3, q = 4).

    python tests/golden/gen_headline.py [256] [512]

The workload the benchmark runs is N = 512^3, q = 4, B = 1, seed 0,
spectrum |j|^-2 exp(-(|j|/(N/32))^2).  These fixtures pin the GPU path at
that size (and at 256^3, where one whole reference-order CG iteration also
fits the CPU) to the C++ oracle (oracle/mlq_oracle.cpp, reference order,
OpenMP on every host core), so the compile-time pass kernels, the mixed
precision path and the reuse paths the benchmark runs are checked against
the oracle and not only against other GPU code paths.

Each file holds, for u = rescaleLqNorm(divAvg_free(seed field)):
  R_parts   calc_global_dLqdt_inclParts(u): R, R1 + R2, R3
  lq_norm   calc_global_Lq_norm(u)
  grad_l2norm, grad_maxabs   of v = GradL2ForLq(u) (L2 norm with dV = 1/N^3)
  grad_idx, grad_sample      v.ravel()[grad_idx] at a prime stride
and at 256^3 the first iteration of maxdLqdt from the raw seed field
(iter1_*: J0, J1, tau, tau bracket, line-search trials, R after the update).
The 512^3 case needs about 45 GB of host memory and some tens of minutes
of CPU.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Oracle  # noqa: E402
from oracle.seedfield import seed_field  # noqa: E402

Q, B, SEED, SLOPE = 4.0, 1.0, 0, 2.0
STRIDE = {256: 8191, 512: 65537}  # primes: the sample does not alias with the grid


def path(n: int) -> str:
    return os.path.join(HERE, f"headline_n{n}_q4.npz")


def generate(n: int) -> None:
    t0 = time.time()
    k0 = n / 32.0
    u_raw = seed_field(n, SEED, SLOPE, k0)
    o = Oracle(n, Q, B)
    out = {"n": n, "q": Q, "B": B, "seed": SEED, "slope": SLOPE, "k0": k0}
    if n <= 256:
        uo, it, flag, rec = o.maxdlqdt(u_raw, max_iter=1, optim_tol=1e-14)
        r = rec[0]
        out.update(iter1_J0=r["J0"], iter1_J1=r["J1"], iter1_tau=r["tau"], iter1_tau_a=r["tau_a"],
                   iter1_tau_b=r["tau_b"], iter1_n_evals=r["n_evals"], iter1_R=r["R"], iter1_flag=flag,
                   iter1_unorm_q=r["u_norm_q"])
        print(f"n={n}: one CG iteration, {r['n_evals']} trials, J1 {r['J1']!r} ({time.time() - t0:.0f} s)",
              flush=True)
        del uo
    u = o.rescale(o.divavg_free(u_raw))
    del u_raw
    out["R_parts"] = np.asarray(o.R_parts(u))
    out["lq_norm"] = o.lq_norm(u)
    print(f"n={n}: R {out['R_parts']!r} ({time.time() - t0:.0f} s)", flush=True)
    v = o.grad_l2(u)
    del u
    out["grad_l2norm"] = float(np.sqrt(np.sum(v * v) / float(n) ** 3))
    out["grad_maxabs"] = float(np.abs(v).max())
    idx = np.arange(0, v.size, STRIDE[n], dtype=np.int64)
    out["grad_idx"] = idx
    out["grad_sample"] = v.ravel()[idx].copy()
    np.savez_compressed(path(n), **out)
    print(f"n={n}: wrote {path(n)} ({time.time() - t0:.0f} s)", flush=True)


if __name__ == "__main__":
    for arg in sys.argv[1:] or ["256", "512"]:
        generate(int(arg))
