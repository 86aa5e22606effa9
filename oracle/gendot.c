/*
 * oracle/gendot.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU restatement of the device GenDot generator (hpb_gendot_f64_dev): the
 * same counter-based hash of (seed, index, stream), the same head / tail
 * split and pinned exponents, the same tail recurrence y_j = (t_j - D)/x_j
 * with D carried as a compensated sum.  The one intended difference: D
 * starts from a sequential compensated sum of the head here, from the
 * device's Dot2 (hi, lo) there, so the tail's y values agree to about the
 * double-double accuracy of D, not bit for bit; everything else agrees bit
 * for bit.  Built with -ffp-contract=off (the Makefile), so the arithmetic
 * rounds as written.
 */
#include <math.h>
#include <stdint.h>

static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t draw(uint64_t seed, int64_t i, uint32_t k) {
    return mix64(seed * 0x9E3779B97F4A7C15ull + ((uint64_t)i * 16u + k) * 0xD1B54A32D192ED03ull +
                 0x632BE59BD9B4E019ull);
}
static double uniform01(uint64_t r) { return (double)(r >> 11) * 0x1.0p-53; }
static double mantissa(uint64_t seed, int64_t i, uint32_t k) {
    for (uint32_t t = 0; t < 8; ++t) {
        const double m = 2.0 * uniform01(draw(seed, i, k + 8 * t)) - 1.0;
        if (fabs(m) >= 0x1.0p-30) return m;
    }
    return 0.5;
}

int64_t oro_gendot_dev_nfix(uint64_t seed, int64_t n, double cond) {
    const double B = 0.5 * log2(cond);
    int64_t nfix = 10000 + (int64_t)(draw(seed, n, 7) % 10001ull);
    if (nfix < (int64_t)B) nfix = (int64_t)B;
    const int64_t half = (int64_t)llround(0.5 * (double)n);
    if (nfix > half) nfix = half;
    return nfix;
}

/* x, y: n doubles; returns N_fix */
int64_t oro_gendot_dev_f64(uint64_t seed, int64_t n, double cond, double *x, double *y) {
    if (n <= 0) return 0;
    const double B = 0.5 * log2(cond);
    const int64_t nfix = oro_gendot_dev_nfix(seed, n, cond);
    const double step = nfix > 0 ? B / (double)nfix : 0.0;
    const int64_t head = n - nfix;
    double s = 0.0, c = 0.0;
    for (int64_t i = 0; i < head; ++i) {
        double ex = round(B * uniform01(draw(seed, i, 0)));
        double ey = round(B * uniform01(draw(seed, i, 1)));
        if (i == 0) ex = ey = 0.0;
        if (i == nfix) ex = ey = round(B);
        x[i] = ldexp(mantissa(seed, i, 2), (int)ex);
        y[i] = ldexp(mantissa(seed, i, 3), (int)ey);
        const double p = x[i] * y[i], t = fma(x[i], y[i], -p);
        const double s2 = s + p, bv = s2 - s, av = s2 - bv, e = (p - bv) + (s - av);
        s = s2;
        c = c + (t + e);
    }
    for (int64_t j = 0; j < nfix; ++j) {
        const int64_t i = head + j;
        const double e = round(B - (double)j * step);
        x[i] = ldexp(mantissa(seed, i, 2), (int)e);
        const double target = ldexp(mantissa(seed, i, 3), (int)e);
        const double yi = ((target - s) - c) / x[i];
        y[i] = yi;
        const double p = x[i] * yi, t = fma(x[i], yi, -p);
        const double s2 = s + p, bv = s2 - s, av = s2 - bv, ee = (p - bv) + (s - av);
        s = s2;
        c = c + (t + ee);
    }
    return nfix;
}
