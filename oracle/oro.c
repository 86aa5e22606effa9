/*
 * oracle/oro.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU restatement of the reference's compensated BLAS-1 arithmetic plus an
 * exact (Kulisch-style fixed-point) accumulator.  Only tests/, the smoke
 * check and the benchmark's CPU-baseline leg load this library.
 *
 * Parity: pinned.  The sequential Dot2/Sum2 here are checked bit for bit
 * against the reference's own CPU code (common/dot_product.h and
 * common/threaded_reduction.h compiled from the reference sources into
 * oracle/_ref/) on the committed golden vectors in tests/golden/, and the
 * exact accumulator is checked against Python's fractions.Fraction.
 *
 * Build: gcc -O2 -fPIC -shared -ffp-contract=off -fno-fast-math
 * (-ffp-contract=off keeps "s + a*b" from becoming an FMA, which would
 * change the roundings the error-free transformations describe).
 *
 * Complex arrays are interleaved (re, im).  Results:
 *   real dot/sum  -> out[0] = s + c (the Dot2 value), out[1] = s, out[2] = c
 *   complex       -> out[0..1] = s + c, out[2..3] = s, out[4..5] = c
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

/* ------------------------------------------------------------------ */
/* Error-free transformations                                          */
/* (reference: common/dot_product.h:49-66, gpu_reduction_ogita.h:139-153) */
/* ------------------------------------------------------------------ */
static double two_sum_d(double a, double b, double *t) {
    double s = a + b;
    double bs = s - a;
    double as = s - bs;
    *t = (b - bs) + (a - as);
    return s;
}
static float two_sum_f(float a, float b, float *t) {
    float s = a + b;
    float bs = s - a;
    float as = s - bs;
    *t = (b - bs) + (a - as);
    return s;
}
static double two_prod_d(double a, double b, double *t) {
    double p = a * b;
    *t = fma(a, b, -p);
    return p;
}
static float two_prod_f(float a, float b, float *t) {
    float p = a * b;
    *t = fmaf(a, b, -p);
    return p;
}

/* complex conj(a)*b with error terms, common/dot_product.h:124-196 */
#define CPLX_TWO_PROD(R, TP, TS)                                                   \
    static void ctp_##R(R aR, R aI, R bR, R bI, R *pR, R *pI, R *tR, R *tI) {      \
        R tR1, tR2, tI1, tI2, t1 = 0, t2 = 0;                                      \
        R pR1 = TP(aR, bR, &tR1);                                                  \
        R pR2 = TP(aI, bI, &tR2);                                                  \
        R pI1 = TP(aR, bI, &tI1);                                                  \
        R pI2 = TP(-aI, bR, &tI2);                                                 \
        *pR = TS(pR1, pR2, &t1);                                                   \
        *pI = TS(pI1, pI2, &t2);                                                   \
        *tR = tR1 + tR2 + t1;                                                      \
        *tI = tI1 + tI2 + t2;                                                      \
    }
CPLX_TWO_PROD(double, two_prod_d, two_sum_d)
CPLX_TWO_PROD(float, two_prod_f, two_sum_f)

/* ------------------------------------------------------------------ */
/* Sequential Dot2, dot_product<T>::dot_ogita (common/dot_product.h:108-121):
 *   p = TwoProd(x_j, y_j) -> (p, pi); s = TwoSum(s, p) -> (s, t);
 *   c = c + pi + t;  result s + c, all in T.                            */
/* ------------------------------------------------------------------ */
void oro_dot2_seq_f64(int64_t n, const double *x, const double *y, double *out) {
    double s = 0, c = 0, pi = 0, t = 0, p;
    for (int64_t j = 0; j < n; j++) {
        p = two_prod_d(x[j], y[j], &pi);
        s = two_sum_d(s, p, &t);
        c = c + pi + t;
    }
    out[0] = s + c;
    out[1] = s;
    out[2] = c;
}
void oro_dot2_seq_f32(int64_t n, const float *x, const float *y, double *out) {
    float s = 0, c = 0, pi = 0, t = 0, p;
    for (int64_t j = 0; j < n; j++) {
        p = two_prod_f(x[j], y[j], &pi);
        s = two_sum_f(s, p, &t);
        c = c + pi + t;
    }
    out[0] = (float)(s + c);
    out[1] = s;
    out[2] = c;
}
/* complex: thrust::complex arithmetic is componentwise for +/-, so the
 * TwoSum of complex values is two real TwoSums. */
#define CPLX_DOT2(R, SUF, TS)                                                      \
    void oro_dot2_seq_##SUF(int64_t n, const R *x, const R *y, double *out) {      \
        R sR = 0, sI = 0, cR = 0, cI = 0;                                          \
        for (int64_t j = 0; j < n; j++) {                                          \
            R pR, pI, piR, piI, tR, tI;                                            \
            ctp_##R(x[2 * j], x[2 * j + 1], y[2 * j], y[2 * j + 1], &pR, &pI, &piR, &piI); \
            sR = TS(sR, pR, &tR);                                                  \
            sI = TS(sI, pI, &tI);                                                  \
            cR = cR + piR + tR;                                                    \
            cI = cI + piI + tI;                                                    \
        }                                                                          \
        out[0] = (R)(sR + cR);                                                     \
        out[1] = (R)(sI + cI);                                                     \
        out[2] = sR;                                                               \
        out[3] = sI;                                                               \
        out[4] = cR;                                                               \
        out[5] = cI;                                                               \
    }
CPLX_DOT2(double, c128, two_sum_d)
CPLX_DOT2(float, c64, two_sum_f)

/* naive dot, dot_product<T>::dot_naive (common/dot_product.h:94-103);
 * complex uses conj(a)*b (:205-216). */
void oro_dot_naive_f64(int64_t n, const double *x, const double *y, double *out) {
    double s = 0;
    for (int64_t j = 0; j < n; j++) s += x[j] * y[j];
    out[0] = s;
}

/* ------------------------------------------------------------------ */
/* Sum2 / asum2 per part, threaded_reduction<T>::sum_ogita
 * (common/threaded_reduction.h:128-178): s = TwoSum(s, x_j); c = c + t.  */
/* ------------------------------------------------------------------ */
void oro_sum2_seq_f64(int64_t n, const double *x, int use_abs, double *out) {
    double s = 0, c = 0, t = 0;
    for (int64_t j = 0; j < n; j++) {
        double v = use_abs ? fabs(x[j]) : x[j];
        s = two_sum_d(s, v, &t);
        c = c + t;
    }
    out[0] = s + c;
    out[1] = s;
    out[2] = c;
}
void oro_sum2_seq_f32(int64_t n, const float *x, int use_abs, double *out) {
    float s = 0, c = 0, t = 0;
    for (int64_t j = 0; j < n; j++) {
        float v = use_abs ? fabsf(x[j]) : x[j];
        s = two_sum_f(s, v, &t);
        c = c + t;
    }
    out[0] = (float)(s + c);
    out[1] = s;
    out[2] = c;
}

/* ------------------------------------------------------------------ */
/* Threaded Dot2, threaded_reduction<T>::dot with use_high_prec = 1
 * (common/threaded_reduction.h:220-302, :307-349): the vector is cut into
 * `parts` contiguous ranges (bounds(), :413-436: delta = n/parts, the last
 * part takes the remainder), each range runs the sequential recurrence,
 * and the partial results are merged
 *   result = TwoSum(result, s) -> t ; sigma1 = TwoSum(sigma1, c) -> qq ;
 *   sigma2 = sigma2 + t + qq ;   final = result + sigma1 + sigma2.
 * The reference merges under a mutex in thread completion order; here the
 * merge runs in part order, which the reference reaches when the threads
 * finish in order.                                                       */
/* ------------------------------------------------------------------ */
void oro_dot2_threaded_f64(int64_t n, const double *x, const double *y, int parts, double *out) {
    if (parts < 1) parts = 1;
    int64_t delta = n / parts, rem = n % parts;
    double result = 0, sig1 = 0, sig2 = 0;
    int64_t b = 0;
    for (int j = 0; j < parts; j++) {
        int64_t e = b + delta + (j == parts - 1 ? rem : 0);
        double s = 0, c = 0, pi = 0, t = 0, qq = 0, p;
        for (int64_t i = b; i < e; i++) {
            p = two_prod_d(x[i], y[i], &pi);
            s = two_sum_d(s, p, &t);
            c = c + pi + t;
        }
        result = two_sum_d(result, s, &t);
        sig1 = two_sum_d(sig1, c, &qq);
        sig2 = sig2 + t + qq;
        b = e;
    }
    out[0] = result + sig1 + sig2;
}

/* ================================================================== */
/* Exact accumulator                                                   */
/* ================================================================== */
/* A two's-complement fixed-point integer of KL 64-bit limbs; bit 0 has
 * weight 2^-OFF.  Every binary64 product and sum is representable exactly:
 * mantissas are 53-bit integers m with value m*2^(e-53) (frexp), so a
 * product is a 106-bit integer times 2^(e1+e2-106) >= 2^-2252, and sums of
 * up to 2^64 terms below 2^2048 stay below bit OFF+2112 < 64*KL - 1.       */
#define KL 72
#define OFF 2300

typedef struct { uint64_t w[KL]; } xacc;

static void xacc_zero(xacc *a) { memset(a, 0, sizeof(*a)); }

static int xacc_is_neg(const xacc *a) { return (a->w[KL - 1] >> 63) != 0; }

/* add (or subtract) the 128-bit magnitude m shifted left by `sh` bits */
static void xacc_add_shifted(xacc *a, unsigned __int128 m, int sh, int negative) {
    if (m == 0) return;
    int k = sh / 64, b = sh % 64;
    uint64_t part[3];
    /* (m << b) spans at most 3 limbs (m < 2^107, b < 64) */
    unsigned __int128 lo = m << b;               /* low 128 bits */
    uint64_t hi3 = b ? (uint64_t)(m >> (128 - b)) : 0;
    part[0] = (uint64_t)lo;
    part[1] = (uint64_t)(lo >> 64);
    part[2] = hi3;
    if (!negative) {
        unsigned __int128 carry = 0;
        int i;
        for (i = 0; i < 3 && k + i < KL; i++) {
            unsigned __int128 s = (unsigned __int128)a->w[k + i] + part[i] + carry;
            a->w[k + i] = (uint64_t)s;
            carry = s >> 64;
        }
        for (i = k + 3; carry && i < KL; i++) {
            unsigned __int128 s = (unsigned __int128)a->w[i] + carry;
            a->w[i] = (uint64_t)s;
            carry = s >> 64;
        }
    } else {
        uint64_t borrow = 0;
        int i;
        for (i = 0; i < 3 && k + i < KL; i++) {
            uint64_t w = a->w[k + i];
            uint64_t d = part[i];
            uint64_t r = w - d - borrow;
            borrow = (w < d) || (w - d < borrow);
            a->w[k + i] = r;
        }
        for (i = k + 3; borrow && i < KL; i++) {
            uint64_t w = a->w[i];
            a->w[i] = w - 1;
            borrow = (w == 0);
        }
    }
}

/* v = m * 2^e with m a non-negative integer < 2^53 */
static void split_d(double v, uint64_t *m, int *e, int *neg) {
    int ex;
    double f = frexp(fabs(v), &ex); /* f in [0.5, 1) */
    *neg = v < 0;
    *m = (uint64_t)ldexp(f, 53);
    *e = ex - 53;
}

void xacc_add_double(xacc *a, double v) {
    if (v == 0) return;
    uint64_t m;
    int e, neg;
    split_d(v, &m, &e, &neg);
    xacc_add_shifted(a, (unsigned __int128)m, e + OFF, neg);
}

void xacc_add_prod(xacc *a, double x, double y) {
    if (x == 0 || y == 0) return;
    uint64_t mx, my;
    int ex, ey, nx, ny;
    split_d(x, &mx, &ex, &nx);
    split_d(y, &my, &ey, &ny);
    xacc_add_shifted(a, (unsigned __int128)mx * my, ex + ey + OFF, nx ^ ny);
}

/* round the exact value to the nearest double (ties to even) */
double xacc_round(const xacc *a0) {
    xacc a = *a0;
    int neg = xacc_is_neg(&a);
    if (neg) { /* magnitude = two's complement negation */
        unsigned __int128 carry = 1;
        for (int i = 0; i < KL; i++) {
            unsigned __int128 s = (unsigned __int128)(~a.w[i]) + carry;
            a.w[i] = (uint64_t)s;
            carry = s >> 64;
        }
    }
    int top = -1;
    for (int i = KL - 1; i >= 0; i--)
        if (a.w[i]) { top = i * 64 + 63 - __builtin_clzll(a.w[i]); break; }
    if (top < 0) return 0.0;
#define BIT(idx) ((idx) < 0 ? 0 : (int)((a.w[(idx) / 64] >> ((idx) % 64)) & 1))
    int lsb = top - 52;
    const int sub_lsb = OFF - 1074; /* weight 2^-1074 */
    if (lsb < sub_lsb) lsb = sub_lsb;
    if (top - OFF >= 1024) return neg ? -INFINITY : INFINITY;
    uint64_t m = 0;
    for (int i = top; i >= lsb; i--) m = (m << 1) | (uint64_t)BIT(i);
    int rbit = BIT(lsb - 1);
    int sticky = 0;
    for (int i = lsb - 2; i >= 0 && !sticky; i--) {
        if (i % 64 == 63 && a.w[i / 64] == 0) { i -= 63; continue; }
        sticky = BIT(i);
    }
    if (rbit && (sticky || (m & 1))) m += 1;
#undef BIT
    double r = ldexp((double)m, lsb - OFF);
    return neg ? -r : r;
}

/* hi = round(exact), lo = round(exact - hi) */
static void xacc_hilo(const xacc *a, double *hi, double *lo) {
    xacc b = *a;
    *hi = xacc_round(&b);
    if (isinf(*hi)) { *lo = 0; return; }
    xacc_add_double(&b, -*hi);
    *lo = xacc_round(&b);
}

/* exact sum_i x_i*y_i: out[0] = hi, out[1] = lo */
void oro_exact_dot_f64(int64_t n, const double *x, const double *y, double *out) {
    xacc a;
    xacc_zero(&a);
    for (int64_t i = 0; i < n; i++) xacc_add_prod(&a, x[i], y[i]);
    xacc_hilo(&a, &out[0], &out[1]);
}
void oro_exact_dot_f32(int64_t n, const float *x, const float *y, double *out) {
    xacc a;
    xacc_zero(&a);
    for (int64_t i = 0; i < n; i++) xacc_add_prod(&a, (double)x[i], (double)y[i]);
    xacc_hilo(&a, &out[0], &out[1]);
}
/* exact sum_i conj(x_i)*y_i: out = {hi.re, hi.im, lo.re, lo.im} */
void oro_exact_dot_c128(int64_t n, const double *x, const double *y, double *out) {
    xacc ar, ai;
    xacc_zero(&ar);
    xacc_zero(&ai);
    for (int64_t i = 0; i < n; i++) {
        double xr = x[2 * i], xi = x[2 * i + 1], yr = y[2 * i], yi = y[2 * i + 1];
        xacc_add_prod(&ar, xr, yr);
        xacc_add_prod(&ar, xi, yi);
        xacc_add_prod(&ai, xr, yi);
        xacc_add_prod(&ai, -xi, yr);
    }
    xacc_hilo(&ar, &out[0], &out[2]);
    xacc_hilo(&ai, &out[1], &out[3]);
}
void oro_exact_dot_c64(int64_t n, const float *x, const float *y, double *out) {
    xacc ar, ai;
    xacc_zero(&ar);
    xacc_zero(&ai);
    for (int64_t i = 0; i < n; i++) {
        double xr = x[2 * i], xi = x[2 * i + 1], yr = y[2 * i], yi = y[2 * i + 1];
        xacc_add_prod(&ar, xr, yr);
        xacc_add_prod(&ar, xi, yi);
        xacc_add_prod(&ai, xr, yi);
        xacc_add_prod(&ai, -xi, yr);
    }
    xacc_hilo(&ar, &out[0], &out[2]);
    xacc_hilo(&ai, &out[1], &out[3]);
}
/* exact sum (mode 0), sum of |x| (mode 1), sum of |re|+|im| for complex
 * arrays of n elements (ncomp = 2) */
void oro_exact_sum_f64(int64_t n, const double *x, int ncomp, int mode, double *out) {
    xacc a[2];
    xacc_zero(&a[0]);
    xacc_zero(&a[1]);
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < ncomp; k++) {
            double v = x[ncomp * i + k];
            if (mode == 1) xacc_add_double(&a[0], fabs(v));
            else xacc_add_double(&a[k], v);
        }
    if (mode == 1 || ncomp == 1) {
        xacc_hilo(&a[0], &out[0], &out[1]);
    } else {
        xacc_hilo(&a[0], &out[0], &out[2]);
        xacc_hilo(&a[1], &out[1], &out[3]);
    }
}
void oro_exact_sum_f32(int64_t n, const float *x, int ncomp, int mode, double *out) {
    double *d = (double *)malloc(sizeof(double) * (size_t)(n * ncomp + 1));
    for (int64_t i = 0; i < n * ncomp; i++) d[i] = x[i];
    oro_exact_sum_f64(n, d, ncomp, mode, out);
    free(d);
}
/* exact sum of squares (real: x_i^2; complex: re^2 + im^2) */
void oro_exact_sumsq_f64(int64_t n, const double *x, int ncomp, double *out) {
    xacc a;
    xacc_zero(&a);
    for (int64_t i = 0; i < n * ncomp; i++) xacc_add_prod(&a, x[i], x[i]);
    xacc_hilo(&a, &out[0], &out[1]);
}

/* sum |x_i*y_i| rounded (for condition numbers; exact then rounded) */
void oro_exact_absdot_f64(int64_t n, const double *x, const double *y, double *out) {
    xacc a;
    xacc_zero(&a);
    for (int64_t i = 0; i < n; i++) xacc_add_prod(&a, fabs(x[i]), fabs(y[i]));
    xacc_hilo(&a, &out[0], &out[1]);
}

/* |value - exact dot| rounded, computed exactly (value given as hi + lo) */
void oro_abs_err_dot_f64(int64_t n, const double *x, const double *y, double vhi, double vlo, double *out) {
    xacc a;
    xacc_zero(&a);
    for (int64_t i = 0; i < n; i++) xacc_add_prod(&a, x[i], y[i]);
    xacc_add_double(&a, -vhi);
    xacc_add_double(&a, -vlo);
    out[0] = fabs(xacc_round(&a));
}

/* ------------------------------------------------------------------ */
/* A priori relative error bounds, high_prec/error_bounds.hpp:58-277.
 * eps = numeric_limits<T>::epsilon() (= 2u), gamma(n) = n eps/(1-n eps). */
/* ------------------------------------------------------------------ */
static long double gam(long double eps, double n) { return (long double)n * eps / (1.0L - (long double)n * eps); }

/* ogita_dot_bound_real, error_bounds.hpp:254-258 */
double oro_bound_dot2_real(double n, double cond, double eps) {
    long double g = gam(eps, n);
    return (double)(eps + 0.5L * g * g * cond);
}
/* ogita_dot_bound_complex, error_bounds.hpp:259-265 */
double oro_bound_dot2_complex(double n, double cond, double eps) {
    long double g = gam(eps, n), g2 = gam(eps, 2);
    return (double)(eps + 0.5L * (g * g + g * g2 + g2 * g2 + g * g * g2) * cond);
}
/* ogita_sum_bound, error_bounds.hpp:236-240 */
double oro_bound_sum2(double n, double cond, double eps) {
    long double g = gam(eps, n - 1);
    return (double)(eps + g * g * cond);
}
/* comp_block_dot_bound_real, error_bounds.hpp:266-271 (b = ceil(n/k)) */
double oro_bound_dot2_block_real(double b, double k, double cond, double eps) {
    long double gk = gam(eps, k), gb = gam(eps, b);
    return (double)(eps + 0.5L * (2.0L * gk * gk + gb * gb + gk * gb + gk * gb * gb) * cond);
}
/* simple_dot_bound_real (plain recursive dot), error_bounds.hpp:181-186 */
double oro_bound_dot_naive_real(double n, double cond, double eps) {
    return (double)(0.5L * gam(eps, n) * cond);
}
