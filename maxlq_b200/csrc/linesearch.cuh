// linesearch.cuh -- the line search of maxdLqdt: mnbrak (optimization.f90:
// 613-778) and brent (784-951) written once over a trial evaluator, for the
// host loop and for the device controller, and the trial values of the
// transform-free path at q = 4.
//
// The evaluator is called as ev(tau, &J) and returns false to suspend the
// search: the device controller replays the search from its start each time
// it runs, with every trial value it has so far in a table keyed by tau, and
// stops at the first tau it has no value for.  Host and device execute the
// same operations in the same order (the device side is compiled without
// multiply-add contraction), so both searches take the same steps.
#pragma once

#include <cmath>

#include "common.cuh"

namespace mlq {

constexpr int LS_SUSPEND = -1;

// Coefficients of a line search along phi = u + tau d at q = 4, from its
// setup: Parseval products of the |phi|^2 coefficient spectra S_i with the
// |grad phi|^2 ones G_a and with each other, the R2 and R3 integrands as
// polynomials in tau, and the interval of tau around 0 on which
// S(tau) >= 0 at every point.
// Besides that interval, the setup finds the clamp-free interval around
// each of LS_ANCHORS anchor steps near the previous step (alo[k] > ahi[k]:
// none), so that most trials away from 0 need no check either.
constexpr int LS_ANCHORS = 6;
struct LsPoly {
    double sx[3][3], ss[3][3];
    double r2[5], r3[6];
    double tlo, thi;
    double alo[LS_ANCHORS], ahi[LS_ANCHORS];
};

// The anchors for a previous step tau0: tau0 * GOLD^k, k = -3..2 (mnbrak's
// first trials from tau0 and Brent's refinements near it); none for tau0 <= 0.
__host__ __device__ inline void ls_anchors(double tau0, double a[LS_ANCHORS]) {
    const double GOLD = (1.0 + sqrt(5.0)) / 2.0;
    double t = tau0 > 0.0 ? tau0 / (GOLD * GOLD * GOLD) : 0.0;
    for (int k = 0; k < LS_ANCHORS; ++k, t *= GOLD) a[k] = t;
}

// One point's S(tau) = c + b tau + q tau^2 >= 0 set, from its roots (found
// once per point): kind 0 linear (q = 0), 1 no real root, 2 roots r1 <= r2.
struct LsRoots {
    int kind;
    double r1, r2;
};
__host__ __device__ inline LsRoots ls_roots(double q, double b, double c) {
    LsRoots r{0, 0.0, 0.0};
    if (q == 0.0) {
        if (b != 0.0) r.r1 = r.r2 = -c / b;
        return r;
    }
    const double disc = b * b - 4.0 * q * c;
    if (disc < 0.0) {
        r.kind = 1;
        return r;
    }
    const double sq = sqrt(disc);
    const double qq = -0.5 * (b + (b >= 0.0 ? sq : -sq));
    double r1 = qq / q, r2 = qq != 0.0 ? c / qq : 0.0;
    if (r1 > r2) {
        const double t = r1;
        r1 = r2;
        r2 = t;
    }
    r.kind = 2;
    r.r1 = r1;
    r.r2 = r2;
    return r;
}

// The point's interval around tau = 0 (empty when S(0) = c < 0).
__host__ __device__ inline void ls_component0(const LsRoots& r, double q, double b, double c, double& lo,
                                              double& hi) {
    const double inf = 1e300;
    lo = -inf;
    hi = inf;
    if (c < 0.0) {
        lo = inf;
        hi = -inf;
        return;
    }
    if (r.kind == 0) {
        if (b > 0.0) lo = r.r1;
        if (b < 0.0) hi = r.r1;
    } else if (r.kind == 2) {
        if (q < 0.0) {  // non-negative between the roots
            lo = r.r1;
            hi = r.r2;
        } else if (r.r2 <= 0.0) {  // opens up: the side of 0
            lo = r.r2;
        } else if (r.r1 >= 0.0) {
            hi = r.r1;
        } else {
            lo = 0.0;
            hi = 0.0;
        }
    }
}

// The point's interval around anchor a (empty when S(a) < 0, or when a
// falls between the roots of an upward S by rounding).
__host__ __device__ inline void ls_component(const LsRoots& r, double q, double b, double c, double a, double& lo,
                                             double& hi) {
    const double inf = 1e300;
    lo = -inf;
    hi = inf;
    if (c + a * (b + a * q) < 0.0) {
        lo = inf;
        hi = -inf;
        return;
    }
    if (r.kind == 0) {
        if (b > 0.0) lo = r.r1;
        if (b < 0.0) hi = r.r1;
    } else if (r.kind == 2) {
        if (q < 0.0) {
            lo = r.r1;
            hi = r.r2;
        } else if (a <= r.r1) {
            hi = r.r1;
        } else if (a >= r.r2) {
            lo = r.r2;
        } else {
            lo = inf;
            hi = -inf;
        }
    }
}

// the anchors by value (a kernel argument)
struct LsAnchorSet {
    double a[LS_ANCHORS];
};

// A trial with no clamp: inside the interval around 0 or inside the
// interval around an anchor (clear of its ends).
__host__ __device__ inline bool ls_free(const LsPoly& c, double tau) {
    if (tau >= c.tlo && tau <= c.thi) return true;
    for (int k = 0; k < LS_ANCHORS; ++k)
        if (tau >= c.alo[k] && tau <= c.ahi[k]) return true;
    return false;
}

// The R2/R3 coefficients from the setup's sums r[0..23] (FLSRed slots) and
// the Parseval products q1[0..8] = <S_i, G_a>, q2[0..5] = <S_i, S_j> (i <= j);
// lo/hi are the interval ends over all points.
__host__ __device__ inline void ls_assemble(const double* r, const double* q1, const double* q2, double lo, double hi,
                                            const double* alo, const double* ahi, const double* anchor, LsPoly& c) {
    const double M[3][3] = {{r[0], r[1], r[2]}, {r[1], r[3], r[4]}, {r[2], r[4], r[5]}};
    for (int k = 0; k < 5; ++k) c.r2[k] = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) c.r2[a + b] += M[a][b];
    for (int k = 0; k < 6; ++k) c.r3[k] = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int cc = 0; cc < 2; ++cc)
            for (int b = 0; b < 3; ++b) c.r3[a + cc + b] += r[6 + 3 * (2 * a + cc) + b];
    int k = 0;
    for (int i = 0; i < 3; ++i)
        for (int a = 0; a < 3; ++a) c.sx[i][a] = q1[k++];
    k = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) c.ss[i][j] = c.ss[j][i] = q2[k++];
    // stay clear of the ends, where the T-precision trial may round either way
    c.tlo = lo <= 0.0 ? lo * (1.0 - 1e-6) : 1.0;
    c.thi = hi >= 0.0 ? hi * (1.0 - 1e-6) : -1.0;
    for (int k = 0; k < LS_ANCHORS; ++k) {
        const bool ok = anchor[k] > 0.0 && alo[k] <= anchor[k] && anchor[k] <= ahi[k];
        c.alo[k] = ok ? alo[k] + 1e-6 * fabs(alo[k]) : 1.0;
        c.ahi[k] = ok ? ahi[k] - 1e-6 * fabs(ahi[k]) : -1.0;
    }
}

// R = (R1 + R2 + R3, R1 + R2, R3) (calc_local_dLqdt_inclParts, function_ops.f90:
// 1304-1358) and ||phi||_4^4 at tau from the two integrals I2, I3 and I1
__host__ __device__ inline void ls_R_from(const LsPoly& c, double q, double cv, double cp, double tau, double I1,
                                          double out[3]) {
    double I2 = 0.0, I3 = 0.0;
    for (int k = 4; k >= 0; --k) I2 = I2 * tau + c.r2[k];
    for (int k = 5; k >= 0; --k) I3 = I3 * tau + c.r3[k];
    const double R1 = -cv * I1;              // -nu <|u|^2, P2 |grad u|^2>  (1318)
    const double R2 = -cv * (q - 2.0) * I2;  // -(q-2) nu <1, P2 sum_j V_j^2> (1333)
    const double R3 = cp * (q - 2.0) * I3;   // (q-2) <p, u.V>  (1352)
    out[0] = R1 + R2 + R3;
    out[1] = R1 + R2;
    out[2] = R3;
}

// a trial inside [tlo, thi]: every product is a polynomial in tau
__host__ __device__ inline void ls_poly_R(const LsPoly& c, double q, double cv, double cp, double tau, double out[3],
                                          double* lqq) {
    const double tp[5] = {1.0, tau, tau * tau, tau * tau * tau, tau * tau * tau * tau};
    double ra[3] = {0, 0, 0}, r0 = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int a = 0; a < 3; ++a) ra[a] += tp[i] * c.sx[i][a];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r0 += tp[i + j] * c.ss[i][j];
    ls_R_from(c, q, cv, cp, tau, ra[0] + tau * (ra[1] + tau * ra[2]), out);
    *lqq = r0;
}

// a transform trial: r[0] = ||A||^2 (= ||phi||_4^4), r[1..3] = <A, G_a>
__host__ __device__ inline void ls_fft_R(const LsPoly& c, double q, double cv, double cp, const double* r, double tau,
                                         double out[3], double* lqq) {
    ls_R_from(c, q, cv, cp, tau, r[1] + tau * (r[2] + tau * r[3]), out);
    *lqq = r[0];
}

// eval_J(phi, "LineMin") (optimization.f90:537-539): the trial field rescaled
// to ||phi||_q = B, J = -(cs^q (R1 + R2) + cs^(q+1) R3), cs = B / ||phi||_q.
// At q = 4 the powers are formed by square roots and products.
__host__ __device__ inline double ls_J(double R12, double R3, double lqq, double q, double B) {
    if (q == 4.0) {
        const double cs = B / sqrt(sqrt(lqq));
        const double c2 = cs * cs;
        const double c4 = c2 * c2;
        return -1.0 * (c4 * R12 + (c4 * cs) * R3);
    }
    const double cs = B / pow(lqq, 1.0 / q);
    return -1.0 * (pow(cs, q) * R12 + pow(cs, q + 1.0) * R3);
}

// mnbrak (optimization.f90:613-778): a bracket [tau_brack[0], tau_brack[1]] of
// a minimum of J along the line.  Returns the flag (0 found, 1 tau_B fell
// below machine epsilon, 2 ITMAX) or LS_SUSPEND.
#pragma nv_exec_check_disable
template <class Ev>
__host__ __device__ int ls_mnbrak(Ev& ev, double tA0, double tB0, double tau_brack[2], int* myflag) {
    const double GOLD = (1.0 + sqrt(5.0)) / 2.0;
    const double CGOLD = 1.0 / GOLD;
    const double GLIMIT = 10.0;
    const int ITMAX = 100;
    double tA = tA0, tB = fmax(tB0, MACH_EPSILON), tC = 0.0, tP, FP, Pmax, R, Q;
    double FA, FB, FC = 0.0;
    if (!ev(tA, &FA)) return LS_SUSPEND;
    if (!ev(tB, &FB)) return LS_SUSPEND;
    int brakIter = 0;
    while (FB > FA && tB > MACH_EPSILON) {
        tB = CGOLD * tB;
        if (!ev(tB, &FB)) return LS_SUSPEND;
    }
    if (tB <= MACH_EPSILON) {
        *myflag = 1;
        return 1;
    }
    tC = GOLD * tB;
    if (!ev(tC, &FC)) return LS_SUSPEND;
    while (FB >= FC && brakIter < ITMAX) {
        brakIter++;
        tC = GOLD * tC;
        if (!ev(tC, &FC)) return LS_SUSPEND;
        R = (tB - tA) * (FB - FC);
        Q = (tB - tC) * (FB - FA);
        tP = tB - 0.5 * ((tB - tC) * Q - (tB - tA) * R) / copysign(fmax(fabs(Q - R), MACH_EPSILON), Q - R);
        Pmax = tB + GLIMIT * (tC - tB);
        if ((tB - tP) * (tP - tC) > 0) {
            if (!ev(tP, &FP)) return LS_SUSPEND;
            if (FP < FC) {
                tA = tB; FA = FB; tB = tP; FB = FP;
                break;
            } else if (FP > FB) {
                tC = tP; FC = FP;
                break;
            }
            tP = tC + GOLD * (tC - tB);
            if (!ev(tP, &FP)) return LS_SUSPEND;
        } else if ((tC - tP) * (tP - Pmax) > 0) {
            if (!ev(tP, &FP)) return LS_SUSPEND;
            if (FP < FC) {
                tB = tC; tC = tP; FB = FC; FC = FP;
                tP = tC + GOLD * (tC - tB);
                if (!ev(tP, &FP)) return LS_SUSPEND;
            }
        } else if ((tP - Pmax) * (Pmax - tC) >= 0) {
            tP = Pmax;
            if (!ev(tP, &FP)) return LS_SUSPEND;
        } else {
            tP = tC + GOLD * (tC - tB);
            if (!ev(tP, &FP)) return LS_SUSPEND;
        }
        tA = tB; tB = tC; tC = tP;
        FA = FB; FB = FC; FC = FP;
    }
    tau_brack[0] = tA;
    tau_brack[1] = tC;
    *myflag = brakIter >= ITMAX ? 2 : 0;
    return *myflag;
}

// brent (optimization.f90:784-951): the minimiser *x_out in the bracket and
// J there (*fx_out).  The constants are the Fortran default-real literals
// TOL = 1E-6, ZEPS = 1E-8, CGOLD = .381966 widened to double (804-806).
// Returns 0 or LS_SUSPEND.
#pragma nv_exec_check_disable
template <class Ev>
__host__ __device__ int ls_brent(Ev& ev, const double tau_brack[2], double* x_out, double* fx_out) {
    const int ITMAX = 300;
    const double TOL = (double)1E-6f;
    const double ZEPS = (double)1E-8f;
    const double CGOLD = (double).381966f;
    double D = 0.0, A = fmin(tau_brack[0], tau_brack[1]), Bb = fmax(tau_brack[0], tau_brack[1]);
    double V = tau_brack[1] * CGOLD, W = V, X = V, E = 0.0, ETEMP, P = 0, Q = 0, R, U, XM, TOL1, TOL2;
    double FX;
    if (!ev(D, &FX)) return LS_SUSPEND;  // value at tau = 0 written to brent-info (833-840)
    if (!ev(X, &FX)) return LS_SUSPEND;
    double FV = FX, FW = FX, FU;
    for (int j = 1; j <= ITMAX; ++j) {
        XM = 0.5 * (A + Bb);
        TOL1 = TOL * fabs(X) + ZEPS;
        TOL2 = 2.0 * TOL1;
        if (fabs(X - XM) <= (TOL2 - 0.5 * (Bb - A))) break;
        int FLAG = 1;
        if (fabs(E) > TOL1) {
            R = (X - W) * (FX - FV);
            Q = (X - V) * (FX - FW);
            P = (X - V) * Q - (X - W) * R;
            Q = 2.0 * (Q - R);
            if (Q > 0.0) P = -P;
            Q = fabs(Q);
            ETEMP = E;
            E = D;
            if ((fabs(P) >= fabs(0.5 * Q * ETEMP)) || (P <= Q * (A - X)) || (P >= Q * (Bb - X)))
                FLAG = 1;
            else
                FLAG = 2;
        }
        if (FLAG == 1) {
            E = (X >= XM) ? A - X : Bb - X;
            D = CGOLD * E;
        } else {
            D = P / Q;
            U = X + D;
            if ((U - A < TOL2) || (Bb - U < TOL2)) D = copysign(TOL1, XM - X);
        }
        U = (fabs(D) >= TOL1) ? X + D : X + copysign(TOL1, D);
        if (!ev(U, &FU)) return LS_SUSPEND;
        if (FU <= FX) {
            if (U >= X) A = X; else Bb = X;
            V = W; FV = FW; W = X; FW = FX; X = U; FX = FU;
        } else {
            if (U < X) A = U; else Bb = U;
            if ((FU <= FW) || (W == X)) {
                V = W; FV = FW; W = U; FW = FU;
            } else if ((FU <= FV) || (V == X) || (V == W)) {
                V = U; FV = FU;
            }
        }
    }
    *x_out = X;
    if (fx_out) *fx_out = FX;
    return 0;
}

// ---- the device line search ---------------------------------------------------
constexpr int LS_MEMO = 512;      // trial values kept per search
constexpr int LS_MAX_LOOPS = 96;  // controller runs per search (each adds one value)
constexpr int LS_RUNNING = 1;
constexpr int LS_ERR_CAP = 2;  // memo or loop bound reached

// Parameters the host writes before each device search.
struct LsParams {
    double q, cv, cp, B;
    double tA0, tB0;
    int transform_trials;  // every trial by transform (a test of that branch)
};

// What one device search leaves for the host.
struct LsOut {
    int status;  // 0 done, LS_RUNNING, LS_ERR_CAP, MLQ_ERR_NAN
    int mflag, evals, loops, checks, npoly, nfft;
    double tb[2], tau1, fx;
    // the accepted trial: R(tau1), ||phi||_4^4 there, and how it was formed
    double R1[3], lqq1;
    int fft1;
};

// Device state of one search: coefficients, parameters, the table of trial
// values and the suspension.
struct LsDevState {
    LsPoly poly;
    LsParams par;
    LsOut out;
    int ntr;
    int need;  // 0 none, 1 check of ptau pending, 2 transform of ptau pending
    double ptau;
    double mtau[LS_MEMO], mR[LS_MEMO][3], mlqq[LS_MEMO];
    int mfft[LS_MEMO];
};

}  // namespace mlq
