"""Generate the golden fixtures of this directory.

    python tests/golden/gen_golden.py

The reference publishes no golden vectors and its Fortran build is not
available here, so the fixtures are produced by the independent numpy
transcription of the reference's operators (oracle/ref_numpy.py, reference
order: every dealias / derivative a c2c FFT round trip + REAL()).  Inputs are
the project's seeded fields (oracle/seedfield.py).  Each file holds the input
field u, a second seeded direction d, and the outputs of the reference
routines named in the keys.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.ref_numpy import RefNumpy  # noqa: E402
from oracle.seedfield import seed_field  # noqa: E402

CASES = [
    # (n, q, B, seed, slope, k0)
    (8, 4.0, 1.0, 0, 2.0, 4.0),
    (12, 3.0, 2.0, 1, 2.0, 3.0),
    (12, 6.0, 1.5, 2, 5.0 / 3.0, 4.0),
    (16, 8.0, 0.75, 3, 2.0, 2.0),
]


def make_case(n, q, B, seed, slope, k0):
    r = RefNumpy(n, q, B)
    u = r.rescale(r.divavg_free(seed_field(n, seed, slope, k0)))
    d = r.divavg_free(seed_field(n, seed + 100, slope, k0))
    d = d / np.sqrt(r.field_inner(d, d))
    s = 1.5 - 1.0 / q
    grad = r.grad_l2(u)
    return dict(
        n=n, q=q, B=B, seed=seed, slope=slope, k0=k0, u=u, d=d,
        R_parts=r.R_parts(u),
        lq_norm=r.lq_norm(u),
        J_linemin=r.eval_J(u + 0.05 * d, "LineMin"),
        grad_l2=grad,
        hilbert=r.hilbert(grad, s),
        divavg_hilbert=r.divavg_free(r.hilbert(grad, s)),
        normal_l2=r.normal_l2(u),
        transport=r.vector_transport(u, 0.05 * d, grad),
        inner_hl=r.field_inner(u, d, "H"),
        inner_l2=r.field_inner(u, d, "L2"),
        uk_q2=r.calc_uk(u, q - 2.0),
    )


def main():
    for case in CASES:
        n, q = case[0], case[1]
        out = make_case(*case)
        path = os.path.join(HERE, f"golden_n{n:02d}_q{q:g}.npz")
        np.savez_compressed(path, **out)
        print(path, out["R_parts"], out["lq_norm"])


if __name__ == "__main__":
    main()
