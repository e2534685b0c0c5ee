// Divide and conquer for the symmetric tridiagonal eigenproblem: the
// per-merge arithmetic, as __host__ __device__ functions so one definition
// serves the device kernels and any host-side check of them.
//
// The method (Cuppen 1981; Dongarra & Sorensen 1987; Gu & Eisenstat 1995):
// T = diag(T1, T2) + beta v v^T with v = e_{m1-1} + sgn(beta) e_{m1} once
// beta = T[m1-1][m1] is subtracted from the two diagonal entries it couples.
// With T1 = Q1 D1 Q1^T and T2 = Q2 D2 Q2^T known, T = Q (D + rho z z^T) Q^T
// where Q = diag(Q1, Q2), z = (last row of Q1, sgn * first row of Q2) / sqrt 2
// and rho = 2 |beta|.  The eigenvalues of D + rho z z^T are the roots of the
// secular equation 1 + rho sum_i z_i^2 / (d_i - lambda) = 0, one in each gap
// between consecutive poles d_i (the last above d_k-1).  Poles with a
// negligible z_i, and pairs of nearly equal poles (after a rotation that
// zeroes one z_i), deflate: their d_i is an eigenvalue as it stands.  The
// eigenvectors of the rest come from z-hat, the vector for which the computed
// roots are exact (Loewner's formula), which keeps them orthogonal to working
// precision: u_j ~ (z-hat_i / (d_i - lambda_j))_i.
#pragma once

#include <math.h>

namespace nmx {
namespace dc {

constexpr double kEps = 1.1102230246251565e-16;  // 2^-53, the unit roundoff
constexpr int kSecularMaxIter = 400;

// lambda_j - d_i written as the root's offset from its origin pole, so the
// small differences near a pole keep their relative accuracy:
// d_i - lambda_j = (d_i - d_org) - tau.
__host__ __device__ __forceinline__ double delta_ij(const double *d, int i, int org, double tau) {
    return (d[i] - d[org]) - tau;
}

// Root j (0 <= j < k) of 1 + rho sum_i z_i^2 / (d_i - lambda) = 0, d strictly
// ascending, rho > 0, sum z_i^2 <= 1.  The root is returned as its nearer
// pole *org and the offset *tau from it (lambda = d[org] + tau).  In tau,
// g(tau) = 1 + rho sum z_i^2 / ((d_i - d_org) - tau) rises monotonically
// between the poles.  Each step keeps the origin pole's term exact,
// -C / tau with C = rho z_org^2, and replaces the rest, psi, by its tangent
// at the current iterate: 1 + psi + psi' (t - tau) - C / t = 0 is a quadratic
// in t whose root on the origin's side is the next iterate (a one-pole
// rational model, so the steps stay good right next to the pole).  Every
// evaluation also shrinks a bracket around the root, and a step that leaves
// it is replaced by bisection.  Returns the iterations used.
__host__ __device__ inline int secular_root(int k, const double *d, const double *z, double rho,
                                            int j, int *org, double *tau) {
    const bool last = j == k - 1;
    const double gap = last ? rho : d[j + 1] - d[j];
    const double mid = 0.5 * gap;
    int o = j;
    if (!last) {
        double f = 1.0;
        for (int i = 0; i < k; ++i) f += rho * z[i] * z[i] / ((d[i] - d[j]) - mid);
        if (f < 0.0) o = j + 1;
    }
    double lo, hi;
    if (o == j) {
        lo = 0.0;
        hi = last ? gap : mid;
    } else {
        lo = mid - gap;  // relative to d[j+1]
        hi = 0.0;
    }
    const double C = rho * z[o] * z[o];
    double t = 0.5 * (lo + hi);
    int it = 0;
    for (; it < kSecularMaxIter; ++it) {
        if (t == 0.0) break;
        double psi = 0.0, dpsi = 0.0;
        for (int i = 0; i < k; ++i) {
            if (i == o) continue;
            const double q = z[i] / ((d[i] - d[o]) - t);
            psi += rho * z[i] * q;
            dpsi += rho * q * q;
        }
        const double g = 1.0 + psi - C / t;
        // Converged when g is at the rounding level of its terms.
        if (fabs(g) <= 4.0 * kEps * (1.0 + fabs(psi) + fabs(C / t))) break;
        if (g > 0.0)
            hi = t;
        else
            lo = t;
        // Root of dpsi t^2 + A t - C = 0 on the origin's side, in the
        // cancellation-free form.
        const double A = 1.0 + psi - dpsi * t;
        double tn;
        if (dpsi == 0.0) {
            tn = C / A;
        } else {
            const double sq = sqrt(A * A + 4.0 * dpsi * C);
            if (o == j)
                tn = A >= 0.0 ? 2.0 * C / (A + sq) : (sq - A) / (2.0 * dpsi);
            else
                tn = A >= 0.0 ? -(A + sq) / (2.0 * dpsi) : -2.0 * C / (sq - A);
        }
        if (fabs(tn - t) <= 2.0 * kEps * fabs(t)) {
            if (tn > lo && tn < hi) t = tn;
            break;
        }
        if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
        if (hi - lo <= 4.0 * kEps * fmax(fabs(lo), fabs(hi))) {
            t = tn;
            break;
        }
        t = tn;
    }
    *org = o;
    *tau = t;
    return it;
}

// z-hat_i for the computed roots (org[j], tau[j]), j < k:
// z-hat_i^2 = -(d_i - lambda_i) prod_{j != i} (d_i - lambda_j) / (d_i - d_j) / rho,
// the ratios interleaved so the product stays in range; the sign is z_i's.
__host__ __device__ inline double lowner_z(int k, const double *d, const double *z, double rho,
                                           const int *org, const double *tau, int i) {
    double p = delta_ij(d, i, org[i], tau[i]);
    for (int j = 0; j < k; ++j)
        if (j != i) p *= delta_ij(d, i, org[j], tau[j]) / (d[i] - d[j]);
    const double s = sqrt(fmax(-p / rho, 0.0));
    return z[i] < 0.0 ? -s : s;
}

struct Deflation {
    int k;     // non-deflated poles
    int ndef;  // deflated poles (k + ndef = m)
    int nrot;  // plane rotations to apply to Q's columns, in order
};

// The deflation pass of one merge of m = m1 + m2 eigenpairs.  D[0, m1) and
// D[m1, m) are the two halves' eigenvalues, each ascending; z (length m) the
// merge vector, |z| = 1.  Relative column indices 0..m-1 name Q's columns.
// Poles are visited in ascending order (the two halves merged); a pole is
// deflated when rho |z_t| <= tol, or when the rotation G in the plane of it
// and the previous surviving pole (c = z_t / r, s = -z_p / r, r = |(z_p,
// z_t)|) leaves an off-diagonal |(d_t - d_p) c s| <= tol; G moves z_p's
// weight onto z_t and is recorded for Q's columns (col_p, col_t) as
// (x, y) -> (c x + s y, c y - s x).  tol = 8 eps max(max|d|, max|z|).
// Outputs: dl/zl/col_nd (k), ddef/col_def (ndef), rot_* (nrot <= m - 1).
// Scratch: perm, ds, zs (m each).
__host__ __device__ inline Deflation deflate(int m, int m1, const double *D, const double *z,
                                             double rho, int *perm, double *ds, double *zs,
                                             double *dl, double *zl, int *col_nd, double *ddef,
                                             int *col_def, int *rot_a, int *rot_b, double *rot_c,
                                             double *rot_s) {
    int a = 0, b = m1, t = 0;
    while (a < m1 || b < m) {
        if (b >= m || (a < m1 && D[a] <= D[b]))
            perm[t++] = a++;
        else
            perm[t++] = b++;
    }
    double dmax = 0.0, zmax = 0.0;
    for (t = 0; t < m; ++t) {
        ds[t] = D[perm[t]];
        zs[t] = z[perm[t]];
        dmax = fmax(dmax, fabs(ds[t]));
        zmax = fmax(zmax, fabs(zs[t]));
    }
    const double tol = 8.0 * kEps * fmax(dmax, zmax);
    Deflation r{0, 0, 0};
    if (rho * zmax <= tol) {
        for (t = 0; t < m; ++t) {
            ddef[r.ndef] = ds[t];
            col_def[r.ndef++] = perm[t];
        }
        return r;
    }
    int p = -1;
    for (t = 0; t < m; ++t) {
        if (rho * fabs(zs[t]) <= tol) {
            ddef[r.ndef] = ds[t];
            col_def[r.ndef++] = perm[t];
            continue;
        }
        if (p < 0) {
            p = t;
            continue;
        }
        double s = zs[p], c = zs[t];
        const double rr = hypot(c, s);
        const double diff = ds[t] - ds[p];
        c /= rr;
        s = -s / rr;
        if (fabs(diff * c * s) <= tol) {
            zs[t] = rr;
            zs[p] = 0.0;
            rot_a[r.nrot] = perm[p];
            rot_b[r.nrot] = perm[t];
            rot_c[r.nrot] = c;
            rot_s[r.nrot++] = s;
            const double dp = ds[p] * c * c + ds[t] * s * s;
            ds[t] = ds[p] * s * s + ds[t] * c * c;
            ds[p] = dp;
            ddef[r.ndef] = ds[p];
            col_def[r.ndef++] = perm[p];
        } else {
            dl[r.k] = ds[p];
            zl[r.k] = zs[p];
            col_nd[r.k++] = perm[p];
        }
        p = t;
    }
    if (p >= 0) {
        dl[r.k] = ds[p];
        zl[r.k] = zs[p];
        col_nd[r.k++] = perm[p];
    }
    return r;
}

// Position of candidate c among a merge's m eigenvalues: the k roots
// lambda_j (keys 0..k-1) and the ndef deflated values (keys k..m-1), ranked
// by value with ties broken by key, so every candidate gets a distinct slot.
__host__ __device__ inline int merged_rank(int k, int ndef, const double *dl, const int *org,
                                           const double *tau, const double *ddef, int c) {
    const double v = c < k ? dl[org[c]] + tau[c] : ddef[c - k];
    int r = 0;
    for (int j = 0; j < k; ++j) {
        const double w = dl[org[j]] + tau[j];
        r += (w < v) || (w == v && j < c);
    }
    for (int j = 0; j < ndef; ++j) {
        const double w = ddef[j];
        r += (w < v) || (w == v && k + j < c);
    }
    return r;
}

// Eigenvalue k (0-based, ascending) of the symmetric tridiagonal (d, e),
// e[i] coupling i and i+1, inside [lo, hi] (which must hold it), by
// multisection on the Sturm count -- the number of negative pivots of
// T - x I, i.e. of eigenvalues below x.  Each pass counts at three interior
// points at once (three independent division chains) and keeps the quarter
// holding eigenvalue k, until the interval is 2 eps max(|lo|, |hi|) + pivmin
// wide; a pivot smaller than pivmin in magnitude is replaced by -pivmin.
__host__ __device__ inline double sturm_kth(int n, const double *d, const double *e, int k,
                                            double lo, double hi, double pivmin) {
    for (int it = 0; it < 128; ++it) {
        if (hi - lo <= 2.0 * kEps * fmax(fabs(lo), fabs(hi)) + pivmin) break;
        const double w = hi - lo;
        const double x0 = lo + 0.25 * w, x1 = lo + 0.5 * w, x2 = lo + 0.75 * w;
        if (!(lo < x0 && x0 < x1 && x1 < x2 && x2 < hi)) break;
        double q0 = d[0] - x0, q1 = d[0] - x1, q2 = d[0] - x2;
        if (fabs(q0) < pivmin) q0 = -pivmin;
        if (fabs(q1) < pivmin) q1 = -pivmin;
        if (fabs(q2) < pivmin) q2 = -pivmin;
        int c0 = q0 < 0.0, c1 = q1 < 0.0, c2 = q2 < 0.0;
        for (int i = 1; i < n; ++i) {
            const double e2 = e[i - 1] * e[i - 1];
            q0 = (d[i] - x0) - e2 / q0;
            q1 = (d[i] - x1) - e2 / q1;
            q2 = (d[i] - x2) - e2 / q2;
            if (fabs(q0) < pivmin) q0 = -pivmin;
            if (fabs(q1) < pivmin) q1 = -pivmin;
            if (fabs(q2) < pivmin) q2 = -pivmin;
            c0 += q0 < 0.0;
            c1 += q1 < 0.0;
            c2 += q2 < 0.0;
        }
        if (c0 > k) {
            hi = x0;
        } else if (c1 > k) {
            lo = x0;
            hi = x1;
        } else if (c2 > k) {
            lo = x1;
            hi = x2;
        } else {
            lo = x2;
        }
    }
    return 0.5 * (lo + hi);
}

}  // namespace dc
}  // namespace nmx
