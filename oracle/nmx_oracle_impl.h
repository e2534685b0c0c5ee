/*
 * CPU oracle for the dense-factorization path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of numax.linalg's algorithms (numax 0.3.0), used by
 * the test suite, the smoke check and the benchmark's CPU baseline as the
 * thing results are checked against.  Nothing in the shipped library links,
 * loads or calls this code.
 *
 * This header is included twice by nmx_oracle.c, once per element type:
 *   T   the element type (double / float)
 *   FN  the name suffixer (name##_f64 / name##_f32)
 *
 * Every routine names the numax source it follows.  Index conventions are
 * numax's: row-major storage with an explicit leading dimension, 0-based
 * LAPACK-style pivots, 1-based `info`.
 */

/* ---------------------------------------------------------------------- */
/* Branchless helpers: numax/core/numeric.mojo:263-388                     */
/* ---------------------------------------------------------------------- */

/* ge_indicator(x, t): 1 where x >= t (copysign's +1 at exactly zero), else 0.
 * numax/core/numeric.mojo:320-345 */
static inline T FN(ge_indicator)(T x, T threshold) {
    T sign = (T)copysign((T)1, x - threshold);
    return (sign + (T)1) / (T)2;
}

/* max_of(a, b): exact selection, a where a >= b.  numax/core/numeric.mojo:263-300 */
static inline T FN(max_of)(T a, T b) {
    T take_a = FN(ge_indicator)(a, b);
    return a * take_a + b * ((T)1 - take_a);
}

/* guard_nonzero(x, floor) = copysign(max_of(|x|, floor), x).
 * numax/core/numeric.mojo:348-366 */
static inline T FN(guard_nonzero)(T x, T floor_) {
    return (T)copysign(FN(max_of)((T)fabs(x), floor_), x);
}

/* ---------------------------------------------------------------------- */
/* Array tier (one problem per lane): numax/linalg/_array/                 */
/* ---------------------------------------------------------------------- */

/* Left-looking (Crout) Cholesky of the lower triangle; upper of `out` zeroed.
 * numax/linalg/_array/cholesky.mojo:26-65 */
void FN(orc_array_cholesky)(int n, const T *a, T *out) {
    for (int i = 0; i < n * n; ++i) out[i] = (T)0;
    for (int j = 0; j < n; ++j) {
        T diagonal = a[j * n + j];
        for (int k = 0; k < j; ++k) {
            T ljk = out[j * n + k];
            diagonal = diagonal - ljk * ljk;
        }
        T ljj = (T)sqrt(FN(guard_nonzero)(diagonal, (T)NMX_PIVOT_FLOOR));
        out[j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            T total = a[i * n + j];
            for (int k = 0; k < j; ++k) total = total - out[i * n + k] * out[j * n + k];
            out[i * n + j] = total / ljj;
        }
    }
}

/* numax/linalg/_array/triangular.mojo:24-46 (unit_diagonal=False) */
void FN(orc_array_forward)(int n, const T *lower, const T *b, T *x) {
    for (int i = 0; i < n; ++i) {
        T total = b[i];
        for (int j = 0; j < i; ++j) total = total - lower[i * n + j] * x[j];
        x[i] = total / FN(guard_nonzero)(lower[i * n + i], (T)NMX_PIVOT_FLOOR);
    }
}

/* Back substitution against L^T read in place (upper[i*n+j] = lower[j*n+i]).
 * numax/linalg/_array/triangular.mojo:49-63 with the transpose of
 * numax/linalg/_array/cholesky.mojo:83-92 */
void FN(orc_array_back_lt)(int n, const T *lower, const T *y, T *x) {
    for (int step = 0; step < n; ++step) {
        int i = n - 1 - step;
        T total = y[i];
        for (int j = i + 1; j < n; ++j) total = total - lower[j * n + i] * x[j];
        x[i] = total / FN(guard_nonzero)(lower[i * n + i], (T)NMX_PIVOT_FLOOR);
    }
}

/* cholesky_solve(L, b): numax/linalg/_array/cholesky.mojo:68-92 */
void FN(orc_array_cholesky_solve)(int n, const T *lower, const T *b, T *x, T *tmp) {
    FN(orc_array_forward)(n, lower, b, tmp);
    FN(orc_array_back_lt)(n, lower, tmp, x);
}

/* The Jacobi rotation (cosine, sine) annihilating an off-diagonal entry.
 * numax/linalg/_array/eigen.mojo:34-75 */
static inline void FN(jacobi_rotation)(T numerator, T denominator, T *c, T *s) {
    T twice = (T)2 * numerator;
    T radius = (T)sqrt(denominator * denominator + twice * twice);
    T safe = FN(guard_nonzero)((T)fabs(denominator) + radius, (T)NMX_PIVOT_FLOOR);
    T tangent = (T)copysign((T)1, denominator) * twice / safe;
    T cosine = (T)1 / (T)sqrt((T)1 + tangent * tangent);
    *c = cosine;
    *s = tangent * cosine;
}

/* Cyclic-by-row Jacobi eigh, fixed `sweeps`, eigenvalues unsorted (the
 * diagonal), eigenvectors the columns of row-major `vectors`.
 * numax/linalg/_array/eigen.mojo:316-392 */
void FN(orc_jacobi_eigh)(int n, int sweeps, const T *a, T *values, T *vectors, T *work) {
    for (int i = 0; i < n * n; ++i) { work[i] = a[i]; vectors[i] = (T)0; }
    for (int i = 0; i < n; ++i) vectors[i * n + i] = (T)1;
    for (int sw = 0; sw < sweeps; ++sw) {
        for (int p = 0; p < n - 1; ++p) {
            for (int q = p + 1; q < n; ++q) {
                T apq = work[p * n + q], app = work[p * n + p], aqq = work[q * n + q];
                T c, s;
                FN(jacobi_rotation)(apq, aqq - app, &c, &s);
                for (int k = 0; k < n; ++k) {
                    T akp = work[p * n + k], akq = work[q * n + k];
                    work[p * n + k] = c * akp - s * akq;
                    work[q * n + k] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    T apk = work[k * n + p], aqk = work[k * n + q];
                    work[k * n + p] = c * apk - s * aqk;
                    work[k * n + q] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    T vkp = vectors[k * n + p], vkq = vectors[k * n + q];
                    vectors[k * n + p] = c * vkp - s * vkq;
                    vectors[k * n + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    for (int i = 0; i < n; ++i) values[i] = work[i * n + i];
}

/* ---------------------------------------------------------------------- */
/* Tensor tier: panel kernels (numax/linalg/panel.mojo), host rules        */
/* ---------------------------------------------------------------------- */

#define A_(i, j) a[(int64_t)(i) * lda + (j)]

/* Trailing update `C -= L @ R` with MAX matmul's subtracting epilogue: the
 * product of each element is formed first (p ascending), then subtracted.
 * Stands in for linalg.matmul at numax/linalg/lu.mojo:646-673 and
 * numax/linalg/panel.mojo:548-584. */
static void FN(gemm_sub)(int64_t rows, int64_t cols, int64_t depth,
                         const T *l, int64_t ldl, const T *r, int64_t ldr,
                         T *c, int64_t ldc, int parallel) {
#pragma omp parallel for schedule(static) if (parallel && rows * cols * depth > 262144)
    for (int64_t i = 0; i < rows; ++i) {
        for (int64_t j = 0; j < cols; ++j) {
            T product = (T)0;
            for (int64_t p = 0; p < depth; ++p) product += l[i * ldl + p] * r[p * ldr + j];
            c[i * ldc + j] = c[i * ldc + j] - product;
        }
    }
}

/* Unblocked pivoted LU of panel columns k..k+nb over rows k..n; swaps span
 * the full width; first-maximum pivot rule (ties to the lower row index);
 * exact zero pivot floored to 1e-30 for the division, info = first exact
 * zero (1-based).  numax/linalg/panel.mojo:289-431 */
void FN(orc_getrf_panel)(T *a, int64_t lda, int n, int k, int nb, int32_t *piv, int32_t *info) {
    for (int j = 0; j < nb; ++j) {
        int col = k + j;
        int best = col;
        T best_mag = (T)0;
        for (int i = col; i < n; ++i) {
            T mag = (T)fabs(A_(i, col));
            if (mag > best_mag) { best_mag = mag; best = i; }
        }
        piv[col] = best;
        if (best_mag == (T)0 && *info == 0) *info = col + 1;
        if (best != col) {
            for (int c = 0; c < n; ++c) {
                T keep = A_(col, c);
                A_(col, c) = A_(best, c);
                A_(best, c) = keep;
            }
        }
        T pivot = A_(col, col);
        if (pivot == (T)0) pivot = (T)NMX_PIVOT_FLOOR;
        for (int i = col + 1; i < n; ++i) {
            T m = A_(i, col) / pivot;
            A_(i, col) = m;
            for (int c = j + 1; c < nb; ++c) A_(i, k + c) = A_(i, k + c) - m * A_(col, k + c);
        }
    }
}

/* U12 := L11^-1 A12 (unit lower), columns k+nb..cols.
 * numax/linalg/panel.mojo:2411-2463 */
void FN(orc_trsm_left_lower_unit)(T *a, int64_t lda, int k, int nb, int cols) {
    for (int col = k + nb; col < cols; ++col) {
        for (int i = 0; i < nb; ++i) {
            T total = A_(k + i, col);
            for (int p = 0; p < i; ++p) total = total - A_(k + i, k + p) * A_(k + p, col);
            A_(k + i, col) = total;
        }
    }
}

/* Recursive panel: split until nb <= base or nb < 4; left, solve, GEMM,
 * right.  numax/linalg/panel.mojo:434-586 */
void FN(orc_getrf2)(T *a, int64_t lda, int n, int k, int nb, int base, int32_t *piv, int32_t *info) {
    if (nb <= base || nb < NMX_MIN_SPLIT) { FN(orc_getrf_panel)(a, lda, n, k, nb, piv, info); return; }
    int half = nb / 2;
    FN(orc_getrf2)(a, lda, n, k, half, base, piv, info);
    FN(orc_trsm_left_lower_unit)(a, lda, k, half, k + nb);
    int rows = n - k - half, cols = nb - half;
    if (rows > 0 && cols > 0) {
        int r0 = k + half;
        FN(gemm_sub)(rows, cols, half, &A_(r0, k), lda, &A_(k, r0), lda, &A_(r0, r0), lda, 1);
    }
    FN(orc_getrf2)(a, lda, n, k + half, nb - half, base, piv, info);
}

/* Blocked right-looking LU with partial pivoting, in place.  Returns the
 * swap parity (+1/-1).  numax/linalg/lu.mojo:454-701 */
int FN(orc_lu_factor)(T *a, int64_t lda, int n, int block, int base, int32_t *piv, int32_t *info) {
    *info = 0;
    for (int k = 0; k < n; k += block) {
        int nb = n - k < block ? n - k : block;
        FN(orc_getrf2)(a, lda, n, k, nb, base, piv, info);
        FN(orc_trsm_left_lower_unit)(a, lda, k, nb, n);
        int m = n - k - nb;
        if (m > 0) {
            int b0 = k + nb;
            FN(gemm_sub)(m, m, nb, &A_(b0, k), lda, &A_(k, b0), lda, &A_(b0, b0), lda, 1);
        }
    }
    int sign = 1;
    for (int j = 0; j < n; ++j) if (piv[j] != j) sign = -sign;
    return sign;
}

/* Apply the recorded interchanges to an n x rhs row-major block.
 * numax/linalg/panel.mojo:1824-1852 (vector), :2279-2313 (matrix) */
void FN(orc_laswp)(T *b, int64_t ldb, int n, int rhs, const int32_t *piv) {
    for (int c = 0; c < rhs; ++c) {
        for (int j = 0; j < n; ++j) {
            int other = piv[j];
            if (other != j) {
                T keep = b[(int64_t)j * ldb + c];
                b[(int64_t)j * ldb + c] = b[(int64_t)other * ldb + c];
                b[(int64_t)other * ldb + c] = keep;
            }
        }
    }
}

static inline T FN(at)(const T *a, int64_t lda, int trans, int i, int j) {
    return trans ? A_(j, i) : A_(i, j);
}

/* Blocked triangular solve against a vector, in place: trsv_diag on each
 * diagonal block then gemv_sub on the rows that remain.
 * numax/linalg/triangular.mojo:43-111, numax/linalg/panel.mojo:1855-1972 */
void FN(orc_trsv)(const T *a, int64_t lda, T *x, int n, int block, int upper, int unit, int trans) {
    int steps = (n + block - 1) / block;
    for (int step = 0; step < steps; ++step) {
        int k, nb = block;
        if (upper) { k = n - (step + 1) * block; if (k < 0) { nb = block + k; k = 0; } }
        else { k = step * block; nb = n - k < block ? n - k : block; }
        for (int s = 0; s < nb; ++s) {
            int i = upper ? nb - 1 - s : s;
            T total = x[k + i];
            if (upper) for (int p = i + 1; p < nb; ++p) total = total - FN(at)(a, lda, trans, k + i, k + p) * x[k + p];
            else for (int p = 0; p < i; ++p) total = total - FN(at)(a, lda, trans, k + i, k + p) * x[k + p];
            x[k + i] = unit ? total : total / A_(k + i, k + i);
        }
        int row0 = upper ? 0 : k + nb;
        int rows = upper ? k : n - k - nb;
        for (int r = 0; r < rows; ++r) {
            int row = row0 + r;
            T total = x[row];
            for (int j = 0; j < nb; ++j) total = total - FN(at)(a, lda, trans, row, k + j) * x[k + j];
            x[row] = total;
        }
    }
}

/* Blocked triangular solve against an n x rhs row-major matrix, in place:
 * trsm_diag per RHS column, then a GEMM with the subtracting epilogue.
 * numax/linalg/triangular.mojo:114-225, numax/linalg/panel.mojo:2221-2276 */
void FN(orc_trsm)(const T *a, int64_t lda, T *b, int64_t ldb, int n, int rhs, int block,
                  int upper, int unit, int trans) {
    for (int step = 0, steps = (n + block - 1) / block; step < steps; ++step) {
        int k, nb = block;
        if (upper) { k = n - (step + 1) * block; if (k < 0) { nb = block + k; k = 0; } }
        else { k = step * block; nb = n - k < block ? n - k : block; }
        for (int c = 0; c < rhs; ++c) {
            for (int s = 0; s < nb; ++s) {
                int i = upper ? nb - 1 - s : s;
                T total = b[(int64_t)(k + i) * ldb + c];
                if (upper) for (int p = i + 1; p < nb; ++p) total = total - FN(at)(a, lda, trans, k + i, k + p) * b[(int64_t)(k + p) * ldb + c];
                else for (int p = 0; p < i; ++p) total = total - FN(at)(a, lda, trans, k + i, k + p) * b[(int64_t)(k + p) * ldb + c];
                b[(int64_t)(k + i) * ldb + c] = unit ? total : total / A_(k + i, k + i);
            }
        }
        int row0 = upper ? 0 : k + nb;
        int rows = upper ? k : n - k - nb;
        for (int r = 0; r < rows; ++r) {
            for (int c = 0; c < rhs; ++c) {
                T product = (T)0;
                for (int p = 0; p < nb; ++p) product += FN(at)(a, lda, trans, row0 + r, k + p) * b[(int64_t)(k + p) * ldb + c];
                b[(int64_t)(row0 + r) * ldb + c] -= product;
            }
        }
    }
}

/* LU.solve: laswp, unit-lower solve, upper solve.  rhs == 1 takes the
 * vector path (numax/linalg/lu.mojo:222-274), rhs > 1 the matrix path
 * (numax/linalg/lu.mojo:290-354). */
void FN(orc_lu_solve)(const T *a, int64_t lda, const int32_t *piv, T *b, int64_t ldb, int n, int rhs, int block) {
    FN(orc_laswp)(b, ldb, n, rhs, piv);
    if (rhs == 1 && ldb == 1) {
        FN(orc_trsv)(a, lda, b, n, block, 0, 1, 0);
        FN(orc_trsv)(a, lda, b, n, block, 1, 0, 0);
    } else {
        FN(orc_trsm)(a, lda, b, ldb, n, rhs, block, 0, 1, 0);
        FN(orc_trsm)(a, lda, b, ldb, n, rhs, block, 1, 0, 0);
    }
}

/* Unblocked Cholesky of the nb x nb diagonal block; non-positive pivot
 * floored to 1e-30 and recorded (first failure, 1-based).
 * numax/linalg/panel.mojo:216-286 */
void FN(orc_potrf_diag)(T *a, int64_t lda, int k, int nb, int32_t *info) {
    for (int j = 0; j < nb; ++j) {
        T d = A_(k + j, k + j);
        if (d <= (T)0) { if (*info == 0) *info = k + j + 1; d = (T)NMX_PIVOT_FLOOR; }
        A_(k + j, k + j) = (T)sqrt(d);
        T root = A_(k + j, k + j);
        for (int i = j + 1; i < nb; ++i) A_(k + i, k + j) = A_(k + i, k + j) / root;
        for (int i = j + 1; i < nb; ++i) {
            T lij = A_(k + i, k + j);
            for (int c = j + 1; c <= i; ++c) A_(k + i, k + c) = A_(k + i, k + c) - lij * A_(k + c, k + j);
        }
    }
}

/* X := X L^-T for X = a[k+nb:rows, k:k+nb].  numax/linalg/panel.mojo:2316-2408 */
void FN(orc_trsm_right_lower_t)(T *a, int64_t lda, int k, int nb, int rows) {
    for (int row = k + nb; row < rows; ++row) {
        for (int j = 0; j < nb; ++j) {
            T acc = (T)0;
            for (int p = 0; p < j; ++p) acc += A_(row, k + p) * A_(k + j, k + p);
            A_(row, k + j) = (A_(row, k + j) - acc) / A_(k + j, k + j);
        }
    }
}

/* Blocked right-looking Cholesky in place (lower), trailing update tiled
 * over the lower block triangle (`tile` x `tile` GEMMs with transpose_b).
 * numax/linalg/cholesky.mojo:59-230.  info = first non-positive pivot. */
void FN(orc_potrf_blocked)(T *a, int64_t lda, int n, int block, int tile, int32_t *info) {
    *info = 0;
    if (tile <= 0) tile = n > 0 ? n : 1;
    for (int k = 0; k < n; k += block) {
        int nb = n - k < block ? n - k : block;
        FN(orc_potrf_diag)(a, lda, k, nb, info);
        FN(orc_trsm_right_lower_t)(a, lda, k, nb, n);
        int m = n - k - nb;
        if (m <= 0) continue;
        int b0 = k + nb;
        int tiles = (m + tile - 1) / tile;
        for (int ti = 0; ti < tiles; ++ti) {
            int row0 = ti * tile, rows = m - row0 < tile ? m - row0 : tile;
            for (int tj = 0; tj <= ti; ++tj) {
                int col0 = tj * tile, cols = m - col0 < tile ? m - col0 : tile;
#pragma omp parallel for schedule(static) if ((int64_t)rows * cols * nb > 262144)
                for (int i = 0; i < rows; ++i)
                    for (int j = 0; j < cols; ++j) {
                        T product = (T)0;
                        for (int p = 0; p < nb; ++p) product += A_(b0 + row0 + i, k + p) * A_(b0 + col0 + j, k + p);
                        A_(b0 + row0 + i, b0 + col0 + j) -= product;
                    }
            }
        }
    }
}

/* cholesky() = blocked factorization then tril.  numax/linalg/cholesky.mojo:233-396 */
void FN(orc_cholesky)(T *a, int64_t lda, int n, int block, int tile, int32_t *info) {
    FN(orc_potrf_blocked)(a, lda, n, block, tile, info);
    for (int i = 0; i < n; ++i) for (int j = i + 1; j < n; ++j) A_(i, j) = (T)0;
}

/* cholesky_solve(L, B): lower solve, then the upper solve reading L^T in
 * place.  numax/linalg/cholesky.mojo:471-580 (vector and matrix). */
void FN(orc_cholesky_solve)(const T *a, int64_t lda, T *b, int64_t ldb, int n, int rhs, int block) {
    if (rhs == 1 && ldb == 1) {
        FN(orc_trsv)(a, lda, b, n, block, 0, 0, 0);
        FN(orc_trsv)(a, lda, b, n, block, 1, 0, 1);
    } else {
        FN(orc_trsm)(a, lda, b, ldb, n, rhs, block, 0, 0, 0);
        FN(orc_trsm)(a, lda, b, ldb, n, rhs, block, 1, 0, 1);
    }
}

/* Unblocked Householder of panel columns k..k+nb, rows k..m.
 * beta = -sign(alpha)*||x|| (alpha <= 0 -> +||x||), tau = (beta-alpha)/beta,
 * v = x/(alpha-beta), tau = 0 when the sub-column is exactly zero.
 * numax/linalg/panel.mojo:1975-2073 */
void FN(orc_geqr2_panel)(T *a, int64_t lda, int m, int k, int nb, T *tau) {
    for (int j = 0; j < nb; ++j) {
        int col = k + j;
        T below = (T)0;
        for (int i = col + 1; i < m; ++i) { T v = A_(i, col); below += v * v; }
        T alpha = A_(col, col);
        if (below == (T)0) { tau[col] = (T)0; continue; }
        T beta = (T)sqrt(alpha * alpha + below);
        if (alpha > (T)0) beta = -beta;
        T this_tau = (beta - alpha) / beta;
        T scale = (T)1 / (alpha - beta);
        for (int i = col + 1; i < m; ++i) A_(i, col) = A_(i, col) * scale;
        A_(col, col) = beta;
        tau[col] = this_tau;
        for (int c = j + 1; c < nb; ++c) {
            int other = k + c;
            T dot = A_(col, other);
            for (int r = col + 1; r < m; ++r) dot += A_(r, col) * A_(r, other);
            T factor = this_tau * dot;
            A_(col, other) = A_(col, other) - factor;
            for (int r = col + 1; r < m; ++r) A_(r, other) = A_(r, other) - factor * A_(r, col);
        }
    }
}

/* Forward columnwise T of the block reflector (t is nb x nb, row-major).
 * numax/linalg/panel.mojo:2076-2169 */
void FN(orc_larft)(const T *a, int64_t lda, int m, int k, int nb, const T *tau, T *t) {
    for (int e = 0; e < nb * nb; ++e) t[e] = (T)0;
    t[0] = tau[k];
    for (int i = 1; i < nb; ++i) {
        T ti = tau[k + i];
        for (int p = 0; p < i; ++p) {
            T total = A_(k + i, k + p);
            for (int r = k + i + 1; r < m; ++r) total += A_(r, k + p) * A_(r, k + i);
            t[p * nb + i] = -ti * total;
        }
        for (int q = 0; q < i; ++q) {
            T total = (T)0;
            for (int r = q; r < i; ++r) total += t[q * nb + r] * t[r * nb + i];
            t[q * nb + i] = total;
        }
        t[i * nb + i] = ti;
    }
}

/* C := (I - V T' V^T) C for the panel at k, C = c[row0.., col0..] of
 * rows x width, T' = T^T when `transposed`.  numax/linalg/qr.mojo:123-327 */
void FN(orc_apply_block_reflector)(const T *a, int64_t lda, int m, int k, int nb, const T *tau,
                                   T *c, int64_t ldc, int rows, int width, int row0, int col0,
                                   int transposed, T *scratch /* nb*nb + 2*nb*width */) {
    if (rows <= 0 || width <= 0 || nb <= 0) return;
    T *t = scratch, *w = scratch + nb * nb, *y = w + (int64_t)nb * width;
    FN(orc_larft)(a, lda, m, k, nb, tau, t);
    /* W = V^T C, V unit lower trapezoidal rows x nb read from a[k.., k..] */
    for (int p = 0; p < nb; ++p)
        for (int j = 0; j < width; ++j) {
            T total = (T)0;
            for (int i = p; i < rows; ++i) {
                T v = i == p ? (T)1 : A_(k + i, k + p);
                total += v * c[(int64_t)(row0 + i) * ldc + col0 + j];
            }
            w[(int64_t)p * width + j] = total;
        }
    for (int p = 0; p < nb; ++p)
        for (int j = 0; j < width; ++j) {
            T total = (T)0;
            for (int q = 0; q < nb; ++q) total += (transposed ? t[q * nb + p] : t[p * nb + q]) * w[(int64_t)q * width + j];
            y[(int64_t)p * width + j] = total;
        }
#pragma omp parallel for schedule(static) if ((int64_t)rows * width * nb > 262144)
    for (int i = 0; i < rows; ++i)
        for (int j = 0; j < width; ++j) {
            T total = (T)0;
            int top = i < nb - 1 ? i : nb - 1;
            for (int p = 0; p <= top; ++p) {
                T v = i == p ? (T)1 : A_(k + i, k + p);
                total += v * y[(int64_t)p * width + j];
            }
            c[(int64_t)(row0 + i) * ldc + col0 + j] -= total;
        }
}

/* Blocked Householder QR (m >= n) in LAPACK packed form.
 * numax/linalg/qr.mojo:615-743 */
void FN(orc_qr_factor)(T *a, int64_t lda, int m, int n, int block, T *tau, T *scratch) {
    for (int k = 0; k < n; k += block) {
        int nb = n - k < block ? n - k : block;
        FN(orc_geqr2_panel)(a, lda, m, k, nb, tau);
        FN(orc_apply_block_reflector)(a, lda, m, k, nb, tau, a, lda, m - k, n - k - nb, k, k + nb, 1, scratch);
    }
}

/* Thin Q (m x n, row-major ldq): the reflectors replayed last panel first on
 * the identity.  numax/linalg/qr.mojo:405-468 */
void FN(orc_qr_q)(const T *a, int64_t lda, int m, int n, int block, const T *tau, T *q, int64_t ldq, T *scratch) {
    for (int i = 0; i < m; ++i) for (int j = 0; j < n; ++j) q[(int64_t)i * ldq + j] = i == j ? (T)1 : (T)0;
    int steps = (n + block - 1) / block;
    for (int step = 0; step < steps; ++step) {
        int k = (steps - 1 - step) * block;
        int nb = n - k < block ? n - k : block;
        FN(orc_apply_block_reflector)(a, lda, m, k, nb, tau, q, ldq, m - k, n - k, k, k, 0, scratch);
    }
}

/* ---------------------------------------------------------------------- */
/* Batched drivers over a ragged batch (matrix i at offset a_off[i], n_i x n_i
 * row-major; B/X at b_off[i], n_i x nrhs row-major).  The per-problem body is
 * the Array tier, as numax's map_blocks runs it one problem per lane
 * (numax/core/functional.mojo:691-834); OpenMP stands in for parallelize.  */
/* ---------------------------------------------------------------------- */

void FN(orc_batched_cholesky_solve)(int64_t count, const int32_t *ns, const int64_t *a_off, const T *A,
                                    T *L, const int64_t *b_off, const T *B, T *X, int nrhs, int threads) {
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
    {
        T *lfull = (T *)malloc(sizeof(T) * NMX_BATCH_MAX_N * NMX_BATCH_MAX_N);
        T *bcol = (T *)malloc(sizeof(T) * NMX_BATCH_MAX_N * 3);
        T *xcol = bcol + NMX_BATCH_MAX_N, *tmp = xcol + NMX_BATCH_MAX_N;
#pragma omp for schedule(dynamic, 64)
        for (int64_t p = 0; p < count; ++p) {
            int n = ns[p];
            FN(orc_array_cholesky)(n, A + a_off[p], lfull);
            if (L) for (int i = 0; i < n; ++i) for (int j = 0; j <= i; ++j) L[a_off[p] + (int64_t)i * n + j] = lfull[i * n + j];
            for (int r = 0; r < nrhs; ++r) {
                for (int i = 0; i < n; ++i) bcol[i] = B[b_off[p] + (int64_t)i * nrhs + r];
                FN(orc_array_cholesky_solve)(n, lfull, bcol, xcol, tmp);
                for (int i = 0; i < n; ++i) X[b_off[p] + (int64_t)i * nrhs + r] = xcol[i];
            }
        }
        free(lfull);
        free(bcol);
    }
}

void FN(orc_batched_jacobi_eigh)(int64_t count, const int32_t *ns, const int64_t *a_off, const T *A,
                                 const int64_t *w_off, T *W, T *V, int sweeps, int threads) {
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
    {
        T *work = (T *)malloc(sizeof(T) * NMX_BATCH_MAX_N * NMX_BATCH_MAX_N);
#pragma omp for schedule(dynamic, 16)
        for (int64_t p = 0; p < count; ++p) {
            FN(orc_jacobi_eigh)(ns[p], sweeps, A + a_off[p], W + w_off[p], V + a_off[p], work);
        }
        free(work);
    }
}

#undef A_

/* ---------------------------------------------------------------------- */
/* Tensor-tier eigh: numax/linalg/eigen.mojo:1268-1430                    */
/* ---------------------------------------------------------------------- */

/* Symmetric eigendecomposition of the n x n row-major a (lower triangle
 * read), numax's eigh at block = 1 (the unblocked algorithm every block
 * width is pinned against):
 *   sytrd   numax/linalg/eigen.mojo:320-560 with sytd2_column
 *           (numax/linalg/panel.mojo:589-686): column k's reflector
 *           annihilates a[k+2.., k]; beta = sqrt(alpha^2 + |x|^2), negated
 *           when alpha > 0; tau = (beta - alpha) / beta; v = x / (alpha -
 *           beta) below the implicit 1; tau = 0 when |x| = 0.  Then
 *           p = A v, w = tau p - (tau^2 / 2)(p . v) v, A -= v w^T + w v^T.
 *   _tql    implicit QL with Wilkinson shifts (numax/linalg/eigen.mojo:
 *           966-1060, Numerical Recipes' tqli), the rotations applied to Z
 *           as push_rotation defines them (eigen.mojo:724-733): column i
 *           <- c z_i - s z_{i+1}, column i+1 <- s z_i + c z_{i+1}; at most
 *           60 sweeps per eigenvalue (eigen.mojo:564).
 *   sort    insertion sort of the values, the vectors' columns permuted
 *           alike (eigen.mojo:1372-1385); vectors = Q Z (eigen.mojo:1411-1423).
 * w receives the values ascending; z (n x n, may be NULL for values only)
 * the vectors as columns.  work: 2 n^2 + 4 n elements.  Returns 0, or
 * l + 1 when eigenvalue l did not converge. */
int FN(orc_eigh)(int n, const T *a, int lda, T *w, T *z, T *work) {
    T *A = work, *Z = work + (size_t)n * n, *d = Z + (size_t)n * n, *e = d + n, *tau = e + n,
      *p = tau + n;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) A[i * n + j] = j <= i ? a[i * lda + j] : a[j * lda + i];
    for (int k = 0; k + 2 < n; ++k) {
        T below = 0;
        for (int i = k + 2; i < n; ++i) below += A[i * n + k] * A[i * n + k];
        T alpha = A[(k + 1) * n + k];
        tau[k] = 0;
        if (below == 0) continue;
        T beta = (T)sqrt(alpha * alpha + below);
        if (alpha > 0) beta = -beta;
        T t = (beta - alpha) / beta, scale = (T)1 / (alpha - beta);
        for (int i = k + 2; i < n; ++i) A[i * n + k] *= scale;
        A[(k + 1) * n + k] = beta;
        tau[k] = t;
        /* v = (1, A[k+2.., k]) on rows k+1..; p = A22 v; w = t p + aw v. */
        T pv = 0;
        for (int i = k + 1; i < n; ++i) {
            T s = 0;
            for (int j = k + 1; j < n; ++j) s += A[i * n + j] * (j == k + 1 ? (T)1 : A[j * n + k]);
            p[i] = s;
            pv += s * (i == k + 1 ? (T)1 : A[i * n + k]);
        }
        T aw = -(T)0.5 * t * t * pv;
        for (int i = k + 1; i < n; ++i) p[i] = t * p[i] + aw * (i == k + 1 ? (T)1 : A[i * n + k]);
        for (int i = k + 1; i < n; ++i) {
            T vi = i == k + 1 ? (T)1 : A[i * n + k];
            for (int j = k + 1; j < n; ++j) {
                T vj = j == k + 1 ? (T)1 : A[j * n + k];
                A[i * n + j] -= vi * p[j] + p[i] * vj;
            }
        }
    }
    for (int i = 0; i < n; ++i) d[i] = A[i * n + i];
    for (int i = 0; i + 1 < n; ++i) e[i] = A[(i + 1) * n + i];
    e[n - 1] = 0;
    for (int i = 0; i < n * n; ++i) Z[i] = (i / n == i % n) ? (T)1 : (T)0;
    T eps = sizeof(T) == 8 ? (T)2.220446049250313e-16 : (T)1.1920929e-07;
    for (int l = 0; l < n; ++l) {
        int sweeps = 0;
        for (;;) {
            int m = l;
            while (m < n - 1) {
                T sc = (T)fabs(d[m]) + (T)fabs(d[m + 1]);
                if ((T)fabs(e[m]) <= eps * sc) break;
                ++m;
            }
            if (m == l) break;
            if (++sweeps > 60) return l + 1;
            T g = (d[l + 1] - d[l]) / ((T)2 * e[l]);
            T r = (T)hypot(g, (T)1);
            g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            T s = 1, c = 1, pp = 0;
            int i = m - 1, under = 0;
            for (; i >= l; --i) {
                T f = s * e[i], b = c * e[i];
                r = (T)hypot(f, g);
                e[i + 1] = r;
                if (r == 0) {
                    d[i + 1] -= pp;
                    e[m] = 0;
                    under = 1;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - pp;
                r = (d[i] - g) * s + (T)2 * c * b;
                pp = s * r;
                d[i + 1] = g + pp;
                g = c * r - b;
                for (int q = 0; q < n; ++q) {
                    T zi = Z[q * n + i], zj = Z[q * n + i + 1];
                    Z[q * n + i] = c * zi - s * zj;
                    Z[q * n + i + 1] = s * zi + c * zj;
                }
            }
            if (under) continue;
            d[l] -= pp;
            e[l] = g;
            e[m] = 0;
        }
    }
    /* Insertion sort of the values; Z's columns follow. */
    int *order = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) order[i] = i;
    for (int i = 1; i < n; ++i)
        for (int j = i; j > 0 && d[order[j]] < d[order[j - 1]]; --j) {
            int t = order[j];
            order[j] = order[j - 1];
            order[j - 1] = t;
        }
    for (int i = 0; i < n; ++i) w[i] = d[order[i]];
    if (z) {
        /* z = Q Zs, Q = H_0 ... H_{n-3}: the reflectors applied last first. */
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) z[i * n + j] = Z[i * n + order[j]];
        for (int k = n - 3; k >= 0; --k) {
            if (tau[k] == 0) continue;
            for (int j = 0; j < n; ++j) {
                T s = z[(k + 1) * n + j];
                for (int i = k + 2; i < n; ++i) s += A[i * n + k] * z[i * n + j];
                s *= tau[k];
                z[(k + 1) * n + j] -= s;
                for (int i = k + 2; i < n; ++i) z[i * n + j] -= s * A[i * n + k];
            }
        }
    }
    free(order);
    return 0;
}
