/*
 * Harness-local replacement for the reference's QMatrixModel.cpp, which needs
 * Eigen (absent here). Written from the mathematics, not from that file:
 *
 *   GetRate        : escape rate of the current micro-state, -Q[s][s]
 *   MakeTransition : pick the next state by inverse CDF over the off-diagonal
 *                    row of Q restricted to the adjacency list
 *   SetMacroState  : stationary distribution p of Q (p Q = 0, sum p = 1),
 *                    obtained as the least-squares solution of p [Q | 1] = [0 | 1],
 *                    i.e. (S S^T) p = S [0|1]^T = 1 with S = [Q | 1]; a micro-state
 *                    of the requested macro-state is then drawn with probability
 *                    proportional to p.
 *
 * Semantics follow CaSim/QMatrixModel.cpp:16-73 (interface in
 * CaSim/QMatrixModel.h). The dense solve is a plain Gaussian elimination with
 * partial pivoting. Only the 60-state SingleSiteMWC* models use this class;
 * the two-state models on the hot path do not.
 */
#include "QMatrixModel.h"
#include <cmath>
#include <vector>

QMatrixModel::QMatrixModel(std::map<std::string, double>&) { cur_state = 0; }
QMatrixModel::QMatrixModel() { cur_state = 0; }

int QMatrixModel::GetNStates() { return (int)states.size(); }

double QMatrixModel::GetRate(const std::unordered_map<std::string, double>& ions) {
    RebuildQMatrixofSingleState(ions);
    return -Q[cur_state][cur_state];
}

void QMatrixModel::MakeTransition(double rand) {
    const double out_rate = -Q[cur_state][cur_state];
    double cum = 0;
    for (int nb : adjacency_list[cur_state]) {
        cum += Q[cur_state][nb];
        if (cum / out_rate >= rand) {
            cur_state = nb;
            return;
        }
    }
}

static std::vector<double> solve_dense(std::vector<std::vector<double>> a, std::vector<double> b) {
    const int n = (int)b.size();
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
        std::swap(a[c], a[piv]);
        std::swap(b[c], b[piv]);
        for (int r = c + 1; r < n; ++r) {
            double f = a[r][c] / a[c][c];
            if (f == 0) continue;
            for (int k = c; k < n; ++k) a[r][k] -= f * a[c][k];
            b[r] -= f * b[c];
        }
    }
    std::vector<double> x(n, 0.0);
    for (int r = n - 1; r >= 0; --r) {
        double s = b[r];
        for (int k = r + 1; k < n; ++k) s -= a[r][k] * x[k];
        x[r] = s / a[r][r];
    }
    return x;
}

void QMatrixModel::SetMacroState(int macro_state, double rand, const std::unordered_map<std::string, double>& ions) {
    RebuildQMatrix(ions);
    const int n = (int)Q.size();
    // M = S S^T with S = [Q | 1]  ->  M_ij = sum_k Q_ik Q_jk + 1
    std::vector<std::vector<double>> m(n, std::vector<double>(n, 0.0));
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 1.0;
            for (int k = 0; k < n; ++k) s += Q[i][k] * Q[j][k];
            m[i][j] = s;
        }
    std::vector<double> p = solve_dense(m, std::vector<double>(n, 1.0));
    double total = 0;
    for (int i = 0; i < n; ++i) total += (states[i] == macro_state) * p[i];
    double cum = 0;
    for (int i = 0; i < n; ++i) {
        cum += (states[i] == macro_state) * p[i];
        if (cum / total >= rand) {
            cur_state = i;
            return;
        }
    }
}

int QMatrixModel::GetMacroState() { return states[cur_state]; }

int QMatrixModel::GetMacroState(int state) {
    if (state < 0 || state >= (int)states.size()) return -1;
    return states[state];
}

bool QMatrixModel::isOpen() { return states[cur_state] > 0; }
