// Test infrastructure: the divide and conquer of numax_b200/csrc/tridiag_dc.cuh
// (the per-merge arithmetic the eigh kernels run) driven on the host, merge
// by merge in the kernels' order, so the CPU test suite can check deflation,
// the secular roots and the Loewner vectors against LAPACK without a GPU.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "tridiag_dc.cuh"

using namespace nmx::dc;

namespace {
struct Merge {
    int lo, mid, hi, h;
};
int tree(int lo, int hi, std::vector<Merge> &v) {
    if (hi - lo <= 1) return 0;
    const int mid = lo + (hi - lo) / 2;
    const int h = 1 + std::max(tree(lo, mid, v), tree(mid, hi, v));
    v.push_back({lo, mid, hi, h});
    return h;
}
}  // namespace

// Eigenvalues (ascending) into W and eigenvectors (columns of the n x n
// row-major Z) of the symmetric tridiagonal (d, e[0 .. n-2]).  *max_iter
// receives the most secular iterations any root took.
extern "C" int dc_host_solve(int n, const double *d0, const double *e0, double *W, double *Z,
                             int *max_iter) {
    double scale = 0.0;
    for (int i = 0; i < n; ++i) scale = std::fmax(scale, std::fabs(d0[i]));
    for (int i = 0; i + 1 < n; ++i) scale = std::fmax(scale, std::fabs(e0[i]));
    if (scale == 0.0) scale = 1.0;
    std::vector<double> D(n), e(n, 0.0);
    for (int i = 0; i < n; ++i) D[i] = d0[i] / scale;
    for (int i = 0; i + 1 < n; ++i) e[i] = e0[i] / scale;
    std::vector<Merge> merges;
    tree(0, n, merges);
    for (const Merge &m : merges) {
        const double b = std::fabs(e[m.mid - 1]);
        D[m.mid - 1] -= b;
        D[m.mid] -= b;
    }
    std::stable_sort(merges.begin(), merges.end(),
                     [](const Merge &a, const Merge &b) { return a.h < b.h; });
    std::vector<double> Q((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
    *max_iter = 0;
    for (const Merge &mg : merges) {
        const int lo = mg.lo, mid = mg.mid, hi = mg.hi, m = hi - lo, m1 = mid - lo;
        const double beta = e[mid - 1], rho = 2.0 * std::fabs(beta), sg = beta < 0 ? -1.0 : 1.0;
        std::vector<double> z(m), Dl(D.begin() + lo, D.begin() + hi);
        for (int i = 0; i < m; ++i)
            z[i] = (i < m1 ? Q[(size_t)(mid - 1) * n + lo + i] : sg * Q[(size_t)mid * n + lo + i]) /
                   std::sqrt(2.0);
        std::vector<int> perm(m), cnd(m), cdef(m), ra(m), rb(m);
        std::vector<double> ds(m), zs(m), dl(m), zl(m), ddef(m), rc(m), rs(m);
        const Deflation r = deflate(m, m1, Dl.data(), z.data(), rho, perm.data(), ds.data(),
                                    zs.data(), dl.data(), zl.data(), cnd.data(), ddef.data(),
                                    cdef.data(), ra.data(), rb.data(), rc.data(), rs.data());
        if (r.k + r.ndef != m) return 1;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j)
                if ((i < m1) != (j < m1)) Q[(size_t)(lo + i) * n + lo + j] = 0.0;
        for (int t = 0; t < r.nrot; ++t)
            for (int i = 0; i < m; ++i) {
                double &x = Q[(size_t)(lo + i) * n + lo + ra[t]];
                double &y = Q[(size_t)(lo + i) * n + lo + rb[t]];
                const double xn = rc[t] * x + rs[t] * y, yn = rc[t] * y - rs[t] * x;
                x = xn;
                y = yn;
            }
        const int k = r.k;
        std::vector<int> org(k);
        std::vector<double> tau(k), zh(k), U((size_t)k * k);
        for (int j = 0; j < k; ++j)
            *max_iter = std::max(*max_iter, secular_root(k, dl.data(), zl.data(), rho, j, &org[j], &tau[j]));
        for (int i = 0; i < k; ++i) zh[i] = lowner_z(k, dl.data(), zl.data(), rho, org.data(), tau.data(), i);
        for (int j = 0; j < k; ++j) {
            double s = 0.0;
            for (int i = 0; i < k; ++i) {
                const double u = zh[i] / delta_ij(dl.data(), i, org[j], tau[j]);
                U[(size_t)i * k + j] = u;
                s += u * u;
            }
            s = 1.0 / std::sqrt(s);
            for (int i = 0; i < k; ++i) U[(size_t)i * k + j] *= s;
        }
        std::vector<double> Qo((size_t)m * k, 0.0), Qn((size_t)m * m);
        for (int i = 0; i < m; ++i)
            for (int t = 0; t < k; ++t) {
                const double q = Q[(size_t)(lo + i) * n + lo + cnd[t]];
                for (int j = 0; j < k; ++j) Qo[(size_t)i * k + j] += q * U[(size_t)t * k + j];
            }
        std::vector<double> Dn(m);
        std::vector<int> used(m, 0);
        for (int c = 0; c < m; ++c) {
            const int rk = merged_rank(k, r.ndef, dl.data(), org.data(), tau.data(), ddef.data(), c);
            if (rk < 0 || rk >= m || used[rk]++) return 2;
            Dn[rk] = c < k ? dl[org[c]] + tau[c] : ddef[c - k];
            for (int i = 0; i < m; ++i)
                Qn[(size_t)i * m + rk] =
                    c < k ? Qo[(size_t)i * k + c] : Q[(size_t)(lo + i) * n + lo + cdef[c - k]];
        }
        for (int i = 0; i < m; ++i) {
            D[lo + i] = Dn[i];
            for (int j = 0; j < m; ++j) Q[(size_t)(lo + i) * n + lo + j] = Qn[(size_t)i * m + j];
        }
    }
    for (int i = 0; i < n; ++i) W[i] = D[i] * scale;
    std::memcpy(Z, Q.data(), sizeof(double) * (size_t)n * n);
    return 0;
}

// Every eigenvalue of (d, e[0 .. n-2]) by dc::sturm_kth, as the values-only
// kernel computes them (one call per k, Gershgorin interval).
extern "C" void sturm_host_values(int n, const double *d, const double *e, double *W) {
    double lo = d[0], hi = d[0], emax2 = 0.0;
    for (int i = 0; i < n; ++i) {
        const double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(e[i]) : 0.0);
        lo = std::fmin(lo, d[i] - r);
        hi = std::fmax(hi, d[i] + r);
        if (i + 1 < n) emax2 = std::fmax(emax2, e[i] * e[i]);
    }
    const double pivmin = 2.2250738585072014e-308 * std::fmax(1.0, emax2);
    const double tnorm = std::fmax(std::fabs(lo), std::fabs(hi));
    lo -= 2.0 * kEps * tnorm * n + pivmin;
    hi += 2.0 * kEps * tnorm * n + pivmin;
    for (int k = 0; k < n; ++k) W[k] = sturm_kth(n, d, e, k, lo, hi, pivmin);
}
