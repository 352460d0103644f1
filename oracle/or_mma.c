/* Test infrastructure, not the product: the oracle's restatement of the method of moving
 * asymptotes (MMA) for one inequality constraint, in FP64 C.  Only tests and the bench's CPU
 * baseline call it; the library's own implementation is robtop_b200/csrc/rt_mma.cu.
 *
 * The reference (optimization/mma_t.cu, optimization/mma_t.cpp, optimization/mma_t.h) is
 * Svanberg's MMA: the convex separable approximation of each function at x^k,
 *   p_ij = (U_j - x_j)^2 (1.001 max(df_ij, 0) + 0.001 max(-df_ij, 0) + 1e-5 / (xmax_j - xmin_j))
 *   q_ij = (x_j - L_j)^2 (0.001 max(df_ij, 0) + 1.001 max(-df_ij, 0) + 1e-5 / (xmax_j - xmin_j))
 * (mma_t.cu:70-81), the subproblem
 *   min  sum_j p_0j / (U_j - x_j) + q_0j / (x_j - L_j) + a0 z + c y + d y^2 / 2
 *   s.t. sum_j p_1j / (U_j - x_j) + q_1j / (x_j - L_j) - a z - y <= b,  alpha <= x <= beta,
 * b = (the approximation's value at x^k) - g (mma_t.cu:83-89), with a0 = 1, a = 0, c = 10,
 * d = 1 (mma_t.h:229-237), then the asymptote update (mma_t.cu:164-226): gamma = 1.2 / 0.7 / 1
 * by the sign of (x^{k+1} - x^k)(x^k - x^{k-1}), L = x^{k+1} - gamma (x^k - L),
 * U = x^{k+1} + gamma (U - x^k), L clamped to [x - 10 D, x - 0.01 D], U to [x + 0.01 D, x + 10 D]
 * (D = xmax - xmin), alpha = max(xmin, L + 0.1f (x - L), x - 0.5 D), beta = min(xmax,
 * U - 0.1f (U - x), x + 0.5 D); initially x = (xmin + xmax) / 2, L = xmin, U = xmax with the
 * same bounds rule (mma_t.cu:740-754, 802-824).
 *
 * The reference solves the subproblem with a primal-dual interior-point method (mma_t.cu:
 * 330-500, epsilon continuation down to 1e-6).  With one constraint and a = 0 the optimal z is 0
 * and the subproblem's dual is a concave function of one multiplier lambda >= 0 whose
 * derivative
 *   h(lambda) = sum_j p_1j / (U_j - x_j(lambda)) + q_1j / (x_j(lambda) - L_j) - y(lambda) - b,
 *   x_j(lambda) = clamp((sqrt(P) L_j + sqrt(Q) U_j) / (sqrt(P) + sqrt(Q)), alpha_j, beta_j),
 *   P = p_0j + lambda p_1j, Q = q_0j + lambda q_1j, y(lambda) = max(0, (lambda - c) / d),
 * decreases monotonically; its root (lambda = 0 when h(0) <= 0) gives the subproblem's exact
 * optimum, which the interior-point iterates approach.  It is found by bracketing and bisection.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define MMA_C 10.0
#define MMA_D 1.0
#define MMA_RAA0 1e-5

static double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* mma_t::set_bound + clamp_asymptotes: the initial state */
void or_mma_init(long n, const double* xmin, const double* xmax, double* x, double* low, double* upp,
                 double* alpha, double* beta, double* lastdx) {
    for (long j = 0; j < n; j++) {
        const double D = xmax[j] - xmin[j];
        x[j] = 0.5 * (xmin[j] + xmax[j]);
        low[j] = clampd(xmin[j], x[j] - 10 * D, x[j] - 0.01 * D);
        upp[j] = clampd(xmax[j], x[j] + 0.01 * D, x[j] + 10 * D);
        double a = xmin[j], t = low[j] + 0.1 * (x[j] - low[j]);
        if (a < t) a = t;
        t = x[j] - 0.5 * D;
        if (a < t) a = t;
        double b = xmax[j];
        t = upp[j] - 0.1 * (upp[j] - x[j]);
        if (b > t) b = t;
        t = x[j] + 0.5 * D;
        if (b > t) b = t;
        alpha[j] = a;
        beta[j] = b;
        lastdx[j] = 0;
    }
}

static double mma_x_of(double lam, double p0, double q0, double p1, double q1, double l, double u, double a,
                       double b) {
    const double sp = sqrt(p0 + lam * p1), sq = sqrt(q0 + lam * q1);
    return clampd((sp * l + sq * u) / (sp + sq), a, b);
}

/* h(lambda) (see above); pq = [p0 | q0 | p1 | q1] */
static double mma_h(long n, double lam, const double* pq, const double* low, const double* upp, const double* alpha,
                    const double* beta, double bconst) {
    const double *p0 = pq, *q0 = pq + n, *p1 = pq + 2 * n, *q1 = pq + 3 * n;
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long j = 0; j < n; j++) {
        const double xj = mma_x_of(lam, p0[j], q0[j], p1[j], q1[j], low[j], upp[j], alpha[j], beta[j]);
        s += p1[j] / (upp[j] - xj) + q1[j] / (xj - low[j]);
    }
    const double y = lam > MMA_C ? (lam - MMA_C) / MMA_D : 0.0;
    return s - y - bconst;
}

/* one mma_t::update: df (objective gradient), dg (constraint gradient), g (constraint value);
 * x, low, upp, alpha, beta, lastdx updated in place; returns the multiplier, *dxnorm = |dx|;
 * work holds 4 n doubles */
double or_mma_update(long n, const double* df, const double* dg, double g, const double* xmin, const double* xmax,
                     double* x, double* low, double* upp, double* alpha, double* beta, double* lastdx,
                     double* dxnorm, double* work) {
    double *p0 = work, *q0 = work + n, *p1 = work + 2 * n, *q1 = work + 3 * n;
    double gk = 0;
    for (long j = 0; j < n; j++) {
        const double ux = upp[j] - x[j], xl = x[j] - low[j], r = MMA_RAA0 / (xmax[j] - xmin[j]);
        const double f0p = df[j] > 0 ? df[j] : 0, f0m = df[j] < 0 ? -df[j] : 0;
        const double f1p = dg[j] > 0 ? dg[j] : 0, f1m = dg[j] < 0 ? -dg[j] : 0;
        p0[j] = ux * ux * (1.001 * f0p + 0.001 * f0m + r);
        q0[j] = xl * xl * (0.001 * f0p + 1.001 * f0m + r);
        p1[j] = ux * ux * (1.001 * f1p + 0.001 * f1m + r);
        q1[j] = xl * xl * (0.001 * f1p + 1.001 * f1m + r);
        gk += p1[j] / ux + q1[j] / xl;
    }
    const double bconst = gk - g;
    double lam = 0;
    if (mma_h(n, 0.0, work, low, upp, alpha, beta, bconst) > 0) {
        double lo = 0, hi = 1;
        for (int k = 0; k < 400 && mma_h(n, hi, work, low, upp, alpha, beta, bconst) > 0; k++) {
            lo = hi;
            hi *= 4;
        }
        for (int k = 0; k < 200 && hi - lo > 1e-15 * hi; k++) {
            const double mid = 0.5 * (lo + hi);
            if (mma_h(n, mid, work, low, upp, alpha, beta, bconst) > 0)
                lo = mid;
            else
                hi = mid;
        }
        lam = 0.5 * (lo + hi);
    }
    double s2 = 0;
    const double tenth = (double)0.1f;  /* the reference's float literal, promoted */
    for (long j = 0; j < n; j++) {
        const double xn = mma_x_of(lam, p0[j], q0[j], p1[j], q1[j], low[j], upp[j], alpha[j], beta[j]);
        const double dx = xn - x[j], D = xmax[j] - xmin[j];
        const double gam = dx * lastdx[j] > 0 ? 1.2 : (dx * lastdx[j] < 0 ? 0.7 : 1.0);
        double nl = xn - gam * (x[j] - low[j]), nu = xn + gam * (upp[j] - x[j]);
        nl = clampd(nl, xn - 10 * D, xn - 0.01 * D);
        nu = clampd(nu, xn + 0.01 * D, xn + 10 * D);
        double a = xmin[j], t = nl + tenth * (xn - nl);
        if (a < t) a = t;
        t = xn - 0.5 * D;
        if (a < t) a = t;
        double b = xmax[j];
        t = nu - tenth * (nu - xn);
        if (b > t) b = t;
        t = xn + 0.5 * D;
        if (b > t) b = t;
        low[j] = nl;
        upp[j] = nu;
        alpha[j] = a;
        beta[j] = b;
        lastdx[j] = dx;
        x[j] = xn;
        s2 += dx * dx;
    }
    if (dxnorm) *dxnorm = sqrt(s2);
    return lam;
}
