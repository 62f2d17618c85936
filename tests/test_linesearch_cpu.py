"""Host logic of the line search (maxlq_b200/csrc/linesearch.cuh), on the
CPU: the clamp-free intervals of one point's quadratic S(tau) = c + b tau +
q tau^2 checked by sampling, and mnbrak + Brent (optimization.f90:613-951)
on closed-form functions.  A small host program is compiled with nvcc from
the same header the library and its device controller use."""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "maxlq_b200", "csrc")

PROGRAM = r'''
#include <cstdio>
#include <cstdlib>
#include "linesearch.cuh"
using namespace mlq;

struct Quad {  // J(tau) = (tau - t0)^2 + w (tau - t0)^4 + j0
    double t0, w, j0;
    int calls = 0;
    bool operator()(double tau, double* J) {
        ++calls;
        const double d = tau - t0;
        *J = d * d + w * d * d * d * d + j0;
        return true;
    }
};

int main(int argc, char** argv) {
    const char* mode = argv[1];
    if (mode[0] == 'i') {  // intervals: read q b c a per line, print lo0 hi0 lo hi
        double q, b, c, a;
        while (std::scanf("%lf %lf %lf %lf", &q, &b, &c, &a) == 4) {
            const LsRoots r = ls_roots(q, b, c);
            double l0, h0, l1, h1;
            ls_component0(r, q, b, c, l0, h0);
            ls_component(r, q, b, c, a, l1, h1);
            std::printf("%.17g %.17g %.17g %.17g\n", l0, h0, l1, h1);
        }
        return 0;
    }
    // search: read t0 w j0 tB0 per line, print flag x fx calls
    double t0, w, j0, tB0;
    while (std::scanf("%lf %lf %lf %lf", &t0, &w, &j0, &tB0) == 4) {
        Quad f{t0, w, j0};
        double br[2] = {0, 0}, x = 0, fx = 0;
        int flag = 0;
        const int r = ls_mnbrak(f, 0.0, tB0, br, &flag);
        if (r == 0) ls_brent(f, br, &x, &fx);
        std::printf("%d %.17g %.17g %d\n", flag, x, fx, f.calls);
    }
    return 0;
}
'''


@pytest.fixture(scope="module")
def prog(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("ls")
    src = d / "ls_host.cu"
    src.write_text(PROGRAM)
    exe = d / "ls_host"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-I", CSRC, "-I", os.path.join(os.path.dirname(CSRC), "..", "include"),
                    "-o", str(exe), str(src)], check=True, capture_output=True)
    return str(exe)


def _run(exe, mode, rows):
    text = "\n".join(" ".join(repr(float(v)) for v in r) for r in rows) + "\n"
    out = subprocess.run([exe, mode], input=text, capture_output=True, text=True, check=True).stdout
    return np.array([[float(v) for v in line.split()] for line in out.strip().splitlines()])


def _check_interval(q, b, c, lo, hi, a):
    S = lambda t: c + t * (b + t * q)
    if lo > hi:  # empty: S is negative at the anchor
        assert S(a) < 1e-12 * (abs(c) + abs(a * b) + abs(a * a * q)) + 1e-300
        return
    assert lo <= a <= hi
    big = 1e6
    ts = np.linspace(max(lo, -big), min(hi, big), 257)
    scale = abs(c) + np.abs(ts * b) + np.abs(ts * ts * q)
    assert np.all(S(ts) >= -1e-9 * scale), (q, b, c, lo, hi)
    # just outside a finite end, S is negative (the interval is maximal)
    for end, sgn in ((lo, -1), (hi, 1)):
        if abs(end) < big:
            t = end + sgn * 1e-6 * max(1.0, abs(end))
            assert S(t) < 1e-9 * (abs(c) + abs(t * b) + abs(t * t * q)), (q, b, c, end)


def test_clamp_free_intervals_by_sampling(prog):
    rng = np.random.default_rng(0)
    rows = []
    for _ in range(400):
        q, b, c = rng.standard_normal(3)
        a = abs(rng.standard_normal()) * 3.0
        rows.append((q, b, abs(c), a))  # S(0) >= 0: the interval around 0 exists
    # special shapes: linear, constant, double root, no real root
    rows += [(0.0, 1.0, 2.0, 1.0), (0.0, -1.0, 2.0, 1.0), (0.0, 0.0, 3.0, 2.0), (1.0, -2.0, 1.0, 3.0),
             (1.0, 0.0, 1.0, 0.5), (-1.0, 0.0, 4.0, 1.0), (1.0, -5.0, 6.0, 1.0), (1.0, -5.0, 6.0, 4.0),
             (1.0, -5.0, 6.0, 2.5)]
    out = _run(prog, "i", rows)
    assert len(out) == len(rows)
    for (q, b, c, a), (l0, h0, l1, h1) in zip(rows, out):
        _check_interval(q, b, c, l0, h0, 0.0)
        _check_interval(q, b, c, l1, h1, a)
    # 1 - 5 tau + tau^2 ... : S = 6 - 5 tau + tau^2 has roots 2 and 3
    i = rows.index((1.0, -5.0, 6.0, 4.0))
    assert out[i][2] == pytest.approx(3.0) and out[i][3] > 1e299
    i = rows.index((1.0, -5.0, 6.0, 2.5))
    assert out[i][2] > out[i][3]  # S(2.5) < 0: no interval around the anchor


def test_negative_start_gives_no_interval_around_zero(prog):
    out = _run(prog, "i", [(1.0, 0.0, -1.0, 2.0)])
    l0, h0, l1, h1 = out[0]
    assert l0 > h0
    assert l1 == pytest.approx(1.0) and h1 > 1e299  # S >= 0 for tau >= 1


def test_mnbrak_and_brent_find_the_minimum(prog):
    rows = [(0.37, 0.0, -1.0, 100.0), (2.5, 0.3, 4.0, 0.01), (1e-3, 1.0, 0.0, 1.0), (12.0, 0.05, -3.0, 1.0)]
    out = _run(prog, "s", rows)
    for (t0, w, j0, tB0), (flag, x, fx, calls) in zip(rows, out):
        assert flag == 0
        # Brent stops at TOL = 1e-6 relative (plus ZEPS) to the abscissa
        assert x == pytest.approx(t0, rel=1e-5, abs=1e-7)
        assert fx == pytest.approx(j0, abs=1e-9)
        assert calls < 200


def test_mnbrak_flags_an_uphill_direction(prog):
    # the minimum lies behind tau = 0: mnbrak shrinks tau_B below machine epsilon
    out = _run(prog, "s", [(-1.0, 0.0, 0.0, 1.0)])
    assert out[0][0] == 1
