/*
 * oracle/tri.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU restatement of sparse triangular solves (forward / backward
 * substitution over CSR rows) and of ILU(0) on a CSR pattern.
 *
 * The reference has no CPU code for these: it calls cuSPARSE csrsv2
 * (common/csr/gpu_matrix.h:142-311; closed library, and removed from
 * CUDA 12, so it neither builds nor runs here) and its
 * csr::gpu_ilu0_preconditioner (common/csr/gpu_ilu0_preconditioner.h:32-80)
 * computes no factors.  Parity is therefore pinned to the textbook
 * algorithms, not to reference outputs:
 *   - triangular solve: x_i = (alpha b_i - sum_{j in triangle} t_ij x_j) / t_ii
 *     in row order (ascending for the lower, descending for the upper
 *     triangle); with a unit diagonal the division is skipped and stored
 *     diagonal entries are ignored (csrsv2's CUSPARSE_DIAG_TYPE_UNIT,
 *     gpu_matrix.h:162, which the reference's csr::preconditioner::apply
 *     uses for L, preconditioner.h:68-70);
 *   - ILU(0): the IKJ variant (Saad, Iterative Methods for Sparse Linear
 *     Systems, 2nd ed., Algorithm 10.4), updates restricted to A's pattern.
 * Each value is formed by the same sequence of roundings as the GPU kernels
 * (one FMA per real product in a - l*u; complex products and quotients by
 * the formulas below), so results agree bit for bit.
 *
 * Complex arrays are interleaved (re, im).
 */
#include <math.h>
#include <stdint.h>

typedef struct { float re, im; } cf_t;
typedef struct { double re, im; } cd_t;

/* a - l*u */
static inline float fms_f(float a, float l, float u) { return fmaf(-l, u, a); }
static inline double fms_d(double a, double l, double u) { return fma(-l, u, a); }
static inline cf_t fms_cf(cf_t a, cf_t l, cf_t u) {
    cf_t r = {fmaf(-l.re, u.re, fmaf(l.im, u.im, a.re)), fmaf(-l.re, u.im, fmaf(-l.im, u.re, a.im))};
    return r;
}
static inline cd_t fms_cd(cd_t a, cd_t l, cd_t u) {
    cd_t r = {fma(-l.re, u.re, fma(l.im, u.im, a.re)), fma(-l.re, u.im, fma(-l.im, u.re, a.im))};
    return r;
}
/* a * b */
static inline float mul_f(float a, float b) { return a * b; }
static inline double mul_d(double a, double b) { return a * b; }
static inline cf_t mul_cf(cf_t a, cf_t b) {
    cf_t r = {fmaf(a.re, b.re, -(a.im * b.im)), fmaf(a.re, b.im, a.im * b.re)};
    return r;
}
static inline cd_t mul_cd(cd_t a, cd_t b) {
    cd_t r = {fma(a.re, b.re, -(a.im * b.im)), fma(a.re, b.im, a.im * b.re)};
    return r;
}
/* a / d = (a conj(d)) / |d|^2 */
static inline float div_f(float a, float d) { return a / d; }
static inline double div_d(double a, double d) { return a / d; }
static inline cf_t div_cf(cf_t a, cf_t d) {
    float den = fmaf(d.re, d.re, d.im * d.im);
    cf_t r = {fmaf(a.re, d.re, a.im * d.im) / den, fmaf(a.im, d.re, -(a.re * d.im)) / den};
    return r;
}
static inline cd_t div_cd(cd_t a, cd_t d) {
    double den = fma(d.re, d.re, d.im * d.im);
    cd_t r = {fma(a.re, d.re, a.im * d.im) / den, fma(a.im, d.re, -(a.re * d.im)) / den};
    return r;
}
static inline int zero_f(float a) { return a == 0.0f; }
static inline int zero_d(double a) { return a == 0.0; }
static inline int zero_cf(cf_t a) { return a.re == 0.0f && a.im == 0.0f; }
static inline int zero_cd(cd_t a) { return a.re == 0.0 && a.im == 0.0; }

static int32_t diag_pos(const int32_t *rp, const int32_t *ci, int32_t i) {
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] == i) return k;
    return -1;
}

/*
 * x := T^-1 (alpha b).  upper = 0: T = lower triangle (entries with column
 * < row, rows ascending); upper = 1: upper triangle (column > row, rows
 * descending).  Dependencies are taken in the row's index order.  x may
 * equal b.  Returns 0, or -1 when a row needed for a non-unit solve stores
 * no diagonal.
 *
 * oro_csr_ilu0_*: val := L\U in place; returns -1, or the first row whose
 * pivot is exactly zero (the factorization still runs to the end), or -2
 * when a row stores no diagonal.
 */
#define ORO_TRI(SUF, T, FMS, MUL, DIV, ZERO)                                                          \
    int oro_csr_trsv_##SUF(int32_t n, const int32_t *rp, const int32_t *ci, const T *val, int upper,     \
                           int unit, const T *alpha, const T *b, T *x) {                                 \
        for (int32_t s = 0; s < n; ++s) {                                                                \
            const int32_t i = upper ? n - 1 - s : s;                                                     \
            T acc = MUL(*alpha, b[i]);                                                                   \
            int32_t dp = -1;                                                                             \
            for (int32_t e = rp[i]; e < rp[i + 1]; ++e) {                                                \
                const int32_t j = ci[e];                                                                 \
                if (j == i) dp = e;                                                                      \
                if (upper ? j > i : j < i) acc = FMS(acc, val[e], x[j]);                                 \
            }                                                                                            \
            if (!unit) {                                                                                 \
                if (dp < 0) return -1;                                                                   \
                acc = DIV(acc, val[dp]);                                                                 \
            }                                                                                            \
            x[i] = acc;                                                                                  \
        }                                                                                                \
        return 0;                                                                                        \
    }                                                                                                    \
    /* Jacobi sweeps: x_0 = 0, x_{k+1} = D^-1 (alpha b - (T - D) x_k), each row over its triangle   \
     * in index order; xprev: n scratch elements.  Returns 0, or -1 for a missing diagonal. */       \
    int oro_csr_trsv_sweeps_##SUF(int32_t n, const int32_t *rp, const int32_t *ci, const T *val,       \
                                  int upper, int unit, const T *alpha, const T *b, int sweeps, T *x,   \
                                  T *xprev) {                                                          \
        for (int k = 0; k <= sweeps; ++k) {                                                             \
            for (int32_t i = 0; i < n; ++i) xprev[i] = x[i];                                           \
            for (int32_t i = 0; i < n; ++i) {                                                          \
                T acc = MUL(*alpha, b[i]);                                                              \
                int32_t dp = -1;                                                                        \
                for (int32_t e = rp[i]; e < rp[i + 1]; ++e) {                                           \
                    const int32_t j = ci[e];                                                            \
                    if (j == i) dp = e;                                                                 \
                    if (k > 0 && (upper ? j > i : j < i)) acc = FMS(acc, val[e], xprev[j]);             \
                }                                                                                       \
                if (!unit) {                                                                            \
                    if (dp < 0) return -1;                                                              \
                    acc = DIV(acc, val[dp]);                                                            \
                }                                                                                       \
                x[i] = acc;                                                                             \
            }                                                                                           \
        }                                                                                               \
        return 0;                                                                                       \
    }                                                                                                   \
    int32_t oro_csr_ilu0_##SUF(int32_t n, const int32_t *rp, const int32_t *ci, T *val) {                \
        int32_t first_zero = -1;                                                                         \
        for (int32_t i = 0; i < n; ++i)                                                                  \
            if (diag_pos(rp, ci, i) < 0) return -2;                                                      \
        for (int32_t i = 0; i < n; ++i) {                                                                \
            const int32_t e_end = rp[i + 1];                                                             \
            for (int32_t e = rp[i]; e < e_end && ci[e] < i; ++e) {                                       \
                const int32_t k = ci[e];                                                                 \
                const int32_t dk = diag_pos(rp, ci, k);                                                  \
                const T lik = DIV(val[e], val[dk]);                                                      \
                val[e] = lik;                                                                            \
                int32_t p = e + 1, q = dk + 1;                                                           \
                while (p < e_end && q < rp[k + 1]) {                                                     \
                    if (ci[p] == ci[q]) {                                                                \
                        val[p] = FMS(val[p], lik, val[q]);                                               \
                        ++p;                                                                             \
                        ++q;                                                                             \
                    } else if (ci[p] < ci[q]) {                                                          \
                        ++p;                                                                             \
                    } else {                                                                             \
                        ++q;                                                                             \
                    }                                                                                    \
                }                                                                                        \
            }                                                                                            \
            if (first_zero < 0 && ZERO(val[diag_pos(rp, ci, i)])) first_zero = i;                        \
        }                                                                                                \
        return first_zero;                                                                               \
    }

ORO_TRI(f32, float, fms_f, mul_f, div_f, zero_f)
ORO_TRI(f64, double, fms_d, mul_d, div_d, zero_d)
ORO_TRI(c64, cf_t, fms_cf, mul_cf, div_cf, zero_cf)
ORO_TRI(c128, cd_t, fms_cd, mul_cd, div_cd, zero_cd)
