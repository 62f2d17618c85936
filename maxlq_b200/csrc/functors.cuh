// functors.cuh -- physical-space point math fused into the x stage.
//
// Each functor F has compile-time NIN inputs, NOUT outputs and NRED FP64
// reduction slots, and is called per grid point with the inputs' values.
// Outputs are forward-transformed by the x stage (or stored, for the map
// kernel); reductions are summed per block.  The products are those the
// reference forms between its FFT round trips (function_ops.f90); which of
// them is later dealiased, and how, is decided by the pipeline.
#pragma once

#include "common.cuh"

namespace mlq {

// identity: one input to one output (forward transform of a stored field)
struct FCopy {
    static constexpr int NIN = 1, NOUT = 1, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const { out[0] = in[0]; }
};

// x * y
struct FMul {
    static constexpr int NIN = 2, NOUT = 1, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const { out[0] = in[0] * in[1]; }
};

// |u|^2 = u1^2+u2^2+u3^2 (calc_uk 2332; calc_pointwiseVectorNorm 1783-1786)
struct FSq3 {
    static constexpr int NIN = 3, NOUT = 1, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        out[0] = in[0] * in[0] + in[1] * in[1] + in[2] * in[2];
    }
};

// g = sqrt(max(S,0)) (calc_uk 2335-2339); output g*g (calc_gk_order2 2309)
struct FGSq {
    static constexpr int NIN = 1, NOUT = 1, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        const T s = in[0];
        const T g = s <= T(0) ? T(0) : sqrt(s);
        out[0] = g * g;
    }
};

// g^k from S (calc_gk_order2 2291-2304 without the dealias): for k < 0 the
// |g| < MACH_EPSILON points are 0.
struct FGPow {
    static constexpr int NIN = 1, NOUT = 1, NRED = 0;
    double k;
    int thresh;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        const T s = in[0];
        const double g = s <= T(0) ? 0.0 : sqrt((double)s);
        double v;
        if (thresh)
            v = fabs(g) < MACH_EPSILON ? 0.0 : pow(g, k);
        else
            v = pow(g, k);
        out[0] = (T)v;
    }
};

// sum of squares of a stored field (for ||.||^2 of a non-band-limited power)
struct FSqRed {
    static constexpr int NIN = 1, NOUT = 0, NRED = 1;
    template <typename T>
    __device__ void operator()(const T* in, T*, double* acc) const { acc[0] += (double)in[0] * (double)in[0]; }
};

// ---- R(u) and GradL2ForLq products -----------------------------------------
// inputs: u0,u1,u2 then D[3i+j] = d_j u_i
#define U(i) in[i]
#define D(i, j) in[3 + 3 * (i) + (j)]

// q >= 4 branch: S=|u|^2, W_j = sum_i u_i d_j u_i (calc_vgraduvgradu 2189-2194,
// calc_vvgradu 2031-2036), Q = d_j u_i d_i u_j (calc_nablaUnablaUt 1933-1938),
// G2 = |grad u|^2 (calc_nablaModSquared 2380-2386)
struct FRProd {
    static constexpr int NIN = 12, NOUT = 6, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        out[0] = U(0) * U(0) + U(1) * U(1) + U(2) * U(2);
#pragma unroll
        for (int j = 0; j < 3; ++j) out[1 + j] = U(0) * D(0, j) + U(1) * D(1, j) + U(2) * D(2, j);
        T q = 0, g2 = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                q += D(j, i) * D(i, j);
                g2 += D(i, j) * D(i, j);
            }
        out[4] = q;
        out[5] = g2;
    }
};

// e_u branch, first products: S, Q, G2
struct FRProdE {
    static constexpr int NIN = 12, NOUT = 3, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        out[0] = U(0) * U(0) + U(1) * U(1) + U(2) * U(2);
        T q = 0, g2 = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                q += D(j, i) * D(i, j);
                g2 += D(i, j) * D(i, j);
            }
        out[1] = q;
        out[2] = g2;
    }
};

// e_u = u / sqrt(|S|), 0 where the norm < MACH_EPSILON (1775-1791, 1836-1840)
template <typename T>
__device__ __forceinline__ void unit_vec(const T* u, T s, T* e) {
    const T nrm = sqrt(fabs(s));
    if ((double)nrm < MACH_EPSILON) {
        e[0] = e[1] = e[2] = T(0);
    } else {
        e[0] = u[0] / nrm;
        e[1] = u[1] / nrm;
        e[2] = u[2] / nrm;
    }
}

// e_u branch: E_j = sum_i e_i d_j u_i.  inputs u(3), D(9), S
struct FRE {
    static constexpr int NIN = 13, NOUT = 3, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        T e[3];
        unit_vec(in, in[12], e);
#pragma unroll
        for (int j = 0; j < 3; ++j) out[j] = e[0] * D(0, j) + e[1] * D(1, j) + e[2] * D(2, j);
    }
};

// ---- diagnostics -------------------------------------------------------------
// (u . grad) u: out_i = sum_j u_j d_j u_i (calc_global_dEnstrophydt 1452-1458).
// inputs u(3), D(9)
struct FUGradU {
    static constexpr int NIN = 12, NOUT = 3, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
#pragma unroll
        for (int i = 0; i < 3; ++i) out[i] = U(0) * D(i, 0) + U(1) * D(i, 1) + U(2) * D(i, 2);
    }
};

// a . b of two stored vector fields (calc_vvgradu 2052-2058).  inputs a(3), b(3)
struct FDot3 {
    static constexpr int NIN = 6, NOUT = 1, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        out[0] = in[0] * in[3] + in[1] * in[4] + in[2] * in[5];
    }
};

// e_u . E with e_u = u / sqrt(|S|) (calc_vvgradu with v = e_u).  inputs u(3), S, E(3)
struct FEDot {
    static constexpr int NIN = 7, NOUT = 1, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        T e[3];
        unit_vec(in, in[3], e);
        out[0] = e[0] * in[4] + e[1] * in[5] + e[2] * in[6];
    }
};

// the pointwise R fields from the dealiased products x1, x2, x3: R_i = c_i x_i
// -> (R1 + R2 + R3, R1 + R2, R3) (calc_local_pointwise_dLqdt_inclParts 1240,
// 1255, 1280, 1286-1288)
struct FRSum {
    static constexpr int NIN = 3, NOUT = 3, NRED = 0;
    double c1, c2, c3;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        const T r1 = (T)c1 * in[0], r2 = (T)c2 * in[1], r3 = (T)c3 * in[2];
        out[0] = r1 + r2 + r3;
        out[1] = r1 + r2;
        out[2] = r3;
    }
};

// q >= 4 with |u|^{q-4} == 1: R2 and R3 integrands from V (dealiased W), p, u.
// inputs V0,V1,V2, p, u0,u1,u2 -> acc0 += sum V^2 ; acc1 += p * u.V
struct FRRed1 {
    static constexpr int NIN = 7, NOUT = 0, NRED = 2;
    template <typename T>
    __device__ void operator()(const T* in, T*, double* acc) const {
        const double v0 = in[0], v1 = in[1], v2 = in[2];
        acc[0] += v0 * v0 + v1 * v1 + v2 * v2;
        acc[1] += (double)in[3] * ((double)in[4] * v0 + (double)in[5] * v1 + (double)in[6] * v2);
    }
};

// general q >= 4: forward outputs sum V^2, p*a4, u.V.  inputs V(3), p, u(3), a4
struct FRProd2 {
    static constexpr int NIN = 8, NOUT = 3, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        out[0] = in[0] * in[0] + in[1] * in[1] + in[2] * in[2];
        out[1] = in[3] * in[7];
        out[2] = in[4] * in[0] + in[5] * in[1] + in[6] * in[2];
    }
};

// e_u branch: sum E^2, p*a2, e.E.  inputs E(3), p, u(3), S, a2
struct FRProd2E {
    static constexpr int NIN = 9, NOUT = 3, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        T e[3];
        unit_vec(in + 4, in[7], e);
        out[0] = in[0] * in[0] + in[1] * in[1] + in[2] * in[2];
        out[1] = in[3] * in[8];
        out[2] = e[0] * in[0] + e[1] * in[1] + e[2] * in[2];
    }
};

// ---- GradL2ForLq (1066-1211) ----------------------------------------------
// S and Q from u, D
struct FG1 {
    static constexpr int NIN = 12, NOUT = 2, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        out[0] = U(0) * U(0) + U(1) * U(1) + U(2) * U(2);
        T q = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) q += D(j, i) * D(i, j);
        out[1] = q;
    }
};
#undef U
#undef D

// non-e_u: T = sum_i u_i (vc nu Lap u_i - pc d_i p) (1131-1133), c_i = a2 u_i (1150-1153)
// inputs u(3), Lu(3), Gp(3), a2
struct FG2 {
    static constexpr int NIN = 10, NOUT = 4, NRED = 0;
    double cvisc, cpress;  // vc*nu, pc
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        T t = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) t += in[i] * ((T)cvisc * in[3 + i] - (T)cpress * in[6 + i]);
        out[0] = t;
#pragma unroll
        for (int i = 0; i < 3; ++i) out[1 + i] = in[9] * in[i];
    }
};

// e_u: T = sum_i e_i (vc nu Lap u_i - pc d_i p) (1118-1120), c_i = a2 u_i
// inputs u(3), Lu(3), Gp(3), a2, S
struct FG2E {
    static constexpr int NIN = 11, NOUT = 4, NRED = 0;
    double cvisc, cpress;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        T e[3];
        unit_vec(in, in[10], e);
        T t = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) t += e[i] * ((T)cvisc * in[3 + i] - (T)cpress * in[6 + i]);
        out[0] = t;
#pragma unroll
        for (int i = 0; i < 3; ++i) out[1 + i] = in[9] * in[i];
    }
};

// Final sum of the dealiased terms (1178-1190) before the common dealias:
// Z_i = (q-2) aux2 v_i - pc a2 d_i p + 2 pc sum_k d_i u_k d_k aux4 + vc nu a2 Lap u_i
// where v = u (q>=4 branch) or e_u.
// inputs: aux2, u(3), a2, Gp(3), D(9), Ga4(3), Lu(3), [S]
template <bool EU>
struct FG3 {
    static constexpr int NIN = EU ? 24 : 23, NOUT = 3, NRED = 0;
    double qm2, cvisc, cpress;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        const T aux2 = in[0];
        const T* u = in + 1;
        const T a2 = in[4];
        const T* gp = in + 5;
        const T* d = in + 8;  // d[3i+j] = d_j u_i
        const T* ga = in + 17;
        const T* lu = in + 20;
        T v[3];
        if (EU)
            unit_vec(u, in[23], v);
        else {
            v[0] = u[0];
            v[1] = u[1];
            v[2] = u[2];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const T a5 = d[0 * 3 + i] * ga[0] + d[1 * 3 + i] * ga[1] + d[2 * 3 + i] * ga[2];
            out[i] = (T)qm2 * (aux2 * v[i]) - (T)cpress * (a2 * gp[i]) + (T)(2.0 * cpress) * a5 +
                     (T)cvisc * (a2 * lu[i]);
        }
    }
};

// c_i = a2 w_i (vectorTransport 1737-1740).  inputs a2, w(3)
struct FC3 {
    static constexpr int NIN = 4, NOUT = 3, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        out[0] = in[0] * in[1];
        out[1] = in[0] * in[2];
        out[2] = in[0] * in[3];
    }
};

// w = x + tau y for three components (a point of the line search from the
// physical fields of u and d).  inputs x(3), y(3)
struct FAxpy3 {
    static constexpr int NIN = 6, NOUT = 3, NRED = 0;
    double tau;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
#pragma unroll
        for (int i = 0; i < 3; ++i) out[i] = in[i] + (T)tau * in[3 + i];
    }
};

// The retracted state u' = cs w, w = u + tau d, its gradient
// cs (grad u + tau grad d), and (with S) P2(|u'|^2) = cs^2 P2(|w|^2) and
// P2(g'^2) = cs^2 P2(g^2).  inputs w(3), Du(9), Dd(9)[, S, A]; outputs u'(3),
// Du'(9)[, S', A'].  cs and tau are read from device memory (coef[0],
// coef[1]), so a captured launch stays valid from one iteration to the next.
template <bool S>
struct FRetract {
    static constexpr int NIN = S ? 23 : 21, NOUT = S ? 14 : 12, NRED = 0;
    const double* coef;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        const T cs = (T)coef[0], ctau = (T)(coef[0] * coef[1]);
#pragma unroll
        for (int i = 0; i < 3; ++i) out[i] = cs * in[i];
#pragma unroll
        for (int k = 0; k < 9; ++k) out[3 + k] = cs * in[3 + k] + ctau * in[12 + k];
        if constexpr (S) {
            const T cs2 = (T)(coef[0] * coef[0]);
            out[12] = cs2 * in[21];
            out[13] = cs2 * in[22];
        }
    }
};

// T of FG2 alone (c given).  inputs u(3), Lu(3), Gp(3)
struct FG2T {
    static constexpr int NIN = 9, NOUT = 1, NRED = 0;
    double cvisc, cpress;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        T t = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) t += in[i] * ((T)cvisc * in[3 + i] - (T)cpress * in[6 + i]);
        out[0] = t;
    }
};

// S(tau) = s0 + tau s1 + tau^2 s2 from the line search's coefficient fields,
// written twice (S and, where S >= 0 everywhere, A = P2(max(S, 0)) = S).
// inputs s0, s1, s2
struct FPolyS {
    static constexpr int NIN = 3, NOUT = 2, NRED = 0;
    double tau;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        const T t = (T)tau;
        const T v = in[0] + t * (in[1] + t * in[2]);
        out[0] = v;
        out[1] = v;
    }
};

// sum (a-b)^2 and sum a^2: energy of a field outside its band projection
struct FDiffSq {
    static constexpr int NIN = 2, NOUT = 0, NRED = 2;
    template <typename T>
    __device__ void operator()(const T* in, T*, double* acc) const {
        const double d = (double)in[0] - (double)in[1];
        acc[0] += d * d;
        acc[1] += (double)in[0] * (double)in[0];
    }
};

// ---- line search along phi = u + tau d (q = 4) -------------------------------
// Every product that R needs is quadratic in tau; these functors form the
// coefficient fields, whose dealias/Poisson images then combine linearly.

// S_a of |phi|^2 = |u|^2 + tau 2 u.d + tau^2 |d|^2.  inputs u(3), d(3)
struct FLSS {
    static constexpr int NIN = 6, NOUT = 3, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        out[0] = in[0] * in[0] + in[1] * in[1] + in[2] * in[2];
        out[1] = T(2) * (in[0] * in[3] + in[1] * in[4] + in[2] * in[5]);
        out[2] = in[3] * in[3] + in[4] * in[4] + in[5] * in[5];
    }
};

// The tau^1 and tau^2 coefficients of |phi|^2 alone (the tau^0 one, |u|^2, is
// the gradient program's S).  inputs u(3), d(3)
struct FLSS12 {
    static constexpr int NIN = 6, NOUT = 2, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        out[0] = T(2) * (in[0] * in[3] + in[1] * in[4] + in[2] * in[5]);
        out[1] = in[3] * in[3] + in[4] * in[4] + in[5] * in[5];
    }
};

// Coefficients of W_j = sum_i phi_i d_j phi_i in tau.  A = 0: v_i d_j v_i,
// inputs v(3), Dv(9) (the tau^0 term with v = u, the tau^2 term with v = d);
// A = 1: the tau^1 term u_i d_j d_i + d_i d_j u_i, inputs u(3), Du(9), d(3), Dd(9).
template <int A>
struct FLSW {
    static constexpr int NIN = A == 1 ? 24 : 12, NOUT = 3, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        const T* u = in;
        const T* du = in + 3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T w = 0;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                if constexpr (A == 1)
                    w += u[i] * in[15 + 3 * i + j] + in[12 + i] * du[3 * i + j];
                else
                    w += u[i] * du[3 * i + j];
            }
            out[j] = w;
        }
    }
};

// tau^a coefficients of Q = d_j phi_i d_i phi_j (out 0..2) and of
// G2 = |grad phi|^2 (out 3..5).  inputs Du(9), Dd(9)
struct FLSQG {
    static constexpr int NIN = 18, NOUT = 6, NRED = 0;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        const T* du = in;
        const T* dd = in + 9;
        T q0 = 0, q1 = 0, q2 = 0, g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const T a = du[3 * i + j], b = dd[3 * i + j];  // d_j u_i, d_j d_i
                const T at = du[3 * j + i], bt = dd[3 * j + i];
                q0 += a * at;
                q1 += a * bt + b * at;
                q2 += b * bt;
                g0 += a * a;
                g1 += a * b;
                g2 += b * b;
            }
        out[0] = q0;
        out[1] = q1;
        out[2] = q2;
        out[3] = g0;
        out[4] = T(2) * g1;
        out[5] = g2;
    }
};

// g^2 at tau: g = sqrt(max(S0 + tau S1 + tau^2 S2, 0)).  inputs S_a (dealiased)
struct FLSA {
    static constexpr int NIN = 3, NOUT = 1, NRED = 0;
    double tau;
    const double* taup = nullptr;  // tau in device memory instead (the device line search)
    template <typename T>
    __device__ void operator()(const T* in, T* out, double*) const {
        const T t = (T)(taup ? *taup : tau);
        const T s = in[0] + t * (in[1] + t * in[2]);
        const T g = s <= T(0) ? T(0) : sqrt(s);
        out[0] = g * g;
    }
};

// Polynomial coefficients of R2 and R3 along the line.  inputs V[a][j] at
// 3a+j (9), p_a (3), u(3), d(3).  Slots: 0..5 sum_j V_aj V_bj for
// (a,b) = 00,01,02,11,12,22; 6 + 3(2a+c) + b: p_a sum_j c_j V_bj, c = u, d.
struct FLSRed {
    static constexpr int NIN = 18, NOUT = 0, NRED = 24;
    template <typename T>
    __device__ void operator()(const T* in, T*, double* acc) const {
        double V[3][3], p[3], c[2][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int j = 0; j < 3; ++j) V[a][j] = (double)in[3 * a + j];
#pragma unroll
        for (int a = 0; a < 3; ++a) p[a] = (double)in[9 + a];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            c[0][j] = (double)in[12 + j];
            c[1][j] = (double)in[15 + j];
        }
        int s = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = a; b < 3; ++b) acc[s++] += V[a][0] * V[b][0] + V[a][1] * V[b][1] + V[a][2] * V[b][2];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
#pragma unroll
                for (int b = 0; b < 3; ++b)
                    acc[6 + 3 * (2 * a + cc) + b] +=
                        p[a] * (c[cc][0] * V[b][0] + c[cc][1] * V[b][1] + c[cc][2] * V[b][2]);
    }
};

// sum of squares of three stored fields (energy check of a loaded field)
struct FEnergy3 {
    static constexpr int NIN = 3, NOUT = 3, NRED = 1;
    template <typename T>
    __device__ void operator()(const T* in, T* out, double* acc) const {
        acc[0] += (double)in[0] * in[0] + (double)in[1] * in[1] + (double)in[2] * in[2];
        out[0] = in[0];
        out[1] = in[1];
        out[2] = in[2];
    }
};

}  // namespace mlq
