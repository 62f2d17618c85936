// kappa.cpp -- the table of the reference's gradient check.
//
// kappa_test (optimization.f90:957-1129) evaluates J at phi and at
// phi + eps_i phi_pert for eps_i = 10^(-7 - n/2 + i), i = 1..n (n = 16), and
// tabulates kappa_i = (J(phi + eps_i phi_pert) - J(phi)) / (eps_i <grad J,
// phi_pert>).  This file restates the host arithmetic that follows the J
// values: kappa, the "best" kappa with the reference's selection rule
// (1041-1044, whose right-hand side compares against |1/kappa_i - 1|, not
// |1/best - 1|), and the adjusted kappa (1063-1081): the window of
// adjAvgSize = 4 consecutive kappas with the smallest sum of
// |1 - kappa_j/kappa_(j+1)| and the table divided by the signed geometric
// mean of that window.  The J evaluations themselves are mlq_eval_J calls.
#include <cfloat>
#include <cmath>

#include "maxlq.h"

extern "C" {

int mlq_kappa_epsilons(int n, double* eps) {
    if (n < 1 || !eps) return MLQ_ERR_BADARG;
    for (int i = 1; i <= n; ++i) eps[i - 1] = std::pow(10.0, -7.0 - (double)n / 2.0 + (double)i);  // 1037-1038
    return MLQ_OK;
}

int mlq_kappa_table(double J0, const double* J1, double inner, int n, double* table, double* adj_factor,
                    int* best_index, double* best_kappa) {
    const int adj = 4;  // adjAvgSize (1063)
    if (!J1 || !table || n < adj + 1) return MLQ_ERR_BADARG;
    double best = DBL_MAX;  // huge(pr) (1031)
    int bi = 0;
    for (int i = 1; i <= n; ++i) {
        const double eps = std::pow(10.0, -7.0 - (double)n / 2.0 + (double)i);
        const double dJ = J1[i - 1] - J0;
        const double kappa = dJ / (eps * inner);
        if (std::fmax(std::fabs(kappa - 1.0), std::fabs(1.0 / kappa - 1.0)) <
            std::fmax(std::fabs(best - 1.0), std::fabs(1.0 / kappa - 1.0))) {
            best = kappa;
            bi = i;
        }
        double* row = table + 5 * (i - 1);
        row[0] = eps;
        row[1] = inner;
        row[2] = dJ;
        row[3] = kappa;
        row[4] = kappa;
    }
    // adjusted kappa (1063-1081)
    int imin = 1;
    double fmin = 9999.0;
    for (int i = 1; i <= n - (adj - 1) - 1; ++i) {
        double f = 0.0;
        for (int j = 0; j < adj; ++j) f += std::fabs(1.0 - table[5 * (i + j - 1) + 4] / table[5 * (i + j) + 4]);
        if (f < fmin) {
            fmin = f;
            imin = i;
        }
    }
    double f = 1.0;
    for (int j = 0; j < adj; ++j) f *= std::fabs(table[5 * (imin + j - 1) + 4]);
    f = std::copysign(std::pow(f, 1.0 / adj), table[5 * (imin - 1) + 4]);
    for (int i = 0; i < n; ++i) table[5 * i + 4] /= f;
    if (adj_factor) *adj_factor = f;
    if (best_index) *best_index = bi;
    if (best_kappa) *best_kappa = best;
    return MLQ_OK;
}

}  // extern "C"
