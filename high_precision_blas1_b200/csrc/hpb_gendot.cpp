// Seeded generator of ill-conditioned dot-product pairs (host code).
//
// Follows the scheme of the reference's generate_vector_pair::generate
// (generate_vector_pair.hpp:119-182, kernel generate_vector_pair_helper_impl.cuh:42-58),
// which is Ogita-Rump-Oishi's GenDot adapted to long vectors:
//   b = log2(cond), B = b/2;
//   N_fix = min(max(U{10000..20000}, floor(B)), round(n/2)) tail entries;
//   x_i = m_i * 2^round(e_i), y_i likewise, with m ~ U(-1,1) and
//   e ~ U(0, B) for the head; element 0 gets exponent 0 and element N_fix
//   exponent B (the two entries the reference kernel pins);
//   tail j (position n-N_fix+j): x exponent round(B - j*B/N_fix), and
//   y_j = (m'_j * 2^{e_j} - D) / x_j with D the running dot product,
//   so each tail pair cancels the running sum down to m'_j*2^{e_j}.
// Differences from the reference, on purpose:
//   * seeded (splitmix64) instead of std::random_device / cuRAND, so the
//     same seed gives the same vectors on every machine;
//   * D is carried incrementally as a compensated (double-double) sum over
//     the entries already fixed -- O(n) work instead of the reference's
//     full re-dot per tail entry, O(n*N_fix) -- and excludes the stale
//     random y values of the not-yet-fixed tail entries;
//   * the reference's race on exponent_v[0] / exponent_v[N_fix]
//     (every thread writes them) becomes a plain assignment.
// This file is compiled with -ffp-contract=off (see build.py) so the
// compensated arithmetic rounds as written.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>

#include "../../include/hpblas1.h"

namespace {

struct SplitMix64 {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return double(next() >> 11) * 0x1.0p-53; }  // [0, 1)
    double sym() { return 2.0 * uniform() - 1.0; }                    // [-1, 1)
    int64_t range(int64_t lo, int64_t hi) { return lo + int64_t(next() % uint64_t(hi - lo + 1)); }
};

inline double two_sum(double a, double b, double& e) {
    double s = a + b;
    double bv = s - a;
    double av = s - bv;
    e = (b - bv) + (a - av);
    return s;
}
inline double two_prod(double a, double b, double& e) {
    double p = a * b;
    e = std::fma(a, b, -p);
    return p;
}
struct DD {  // compensated running sum (s, c)
    double s = 0, c = 0;
    void add_prod(double a, double b) {
        double t, e;
        double p = two_prod(a, b, t);
        s = two_sum(s, p, e);
        c += t + e;
    }
    double value() const { return s + c; }
};

inline double nonzero_mantissa(SplitMix64& g) {
    double m;
    do {
        m = g.sym();
    } while (std::fabs(m) < 0x1.0p-30);
    return m;
}

}  // namespace

extern "C" int hpb_gendot_f64(uint64_t seed, int64_t n, double cond, double* x, double* y, int64_t* n_fixed_out) {
    if (n < 0 || (n > 0 && (x == nullptr || y == nullptr)) || !(cond >= 1.0)) return HPB_ERROR_INVALID_VALUE;
    if (n == 0) {
        if (n_fixed_out) *n_fixed_out = 0;
        return HPB_SUCCESS;
    }
    SplitMix64 g{seed * 0x2545F4914F6CDD1Dull + 0x1234567ull};
    const double b = std::log2(cond);
    const double B = 0.5 * b;
    int64_t nfix = g.range(10000, 20000);
    if (nfix < int64_t(B)) nfix = int64_t(B);
    int64_t half = int64_t(std::llround(0.5 * double(n)));
    if (nfix > half) nfix = half;
    const int64_t head = n - nfix;
    const double step = nfix > 0 ? B / double(nfix) : 0.0;

    for (int64_t i = 0; i < n; ++i) {
        double ex = std::round(B * g.uniform());
        double ey = std::round(B * g.uniform());
        if (i == 0) ex = ey = 0.0;
        if (i == nfix && nfix < n) ex = ey = std::round(B);
        x[i] = std::ldexp(nonzero_mantissa(g), int(ex));
        y[i] = std::ldexp(nonzero_mantissa(g), int(ey));
    }
    DD d;
    for (int64_t i = 0; i < head; ++i) d.add_prod(x[i], y[i]);
    for (int64_t j = 0; j < nfix; ++j) {
        const int64_t i = head + j;
        const double e = std::round(B - double(j) * step);
        x[i] = std::ldexp(nonzero_mantissa(g), int(e));
        const double target = std::ldexp(nonzero_mantissa(g), int(e));
        // y_i = (target - D) / x_i, with D as a double-double
        double yi = ((target - d.s) - d.c) / x[i];
        y[i] = yi;
        d.add_prod(x[i], yi);
    }
    if (n_fixed_out) *n_fixed_out = nfix;
    return HPB_SUCCESS;
}

// Complex pairs: x = a + i c, y = b + i d with (a, b) and (c, d) two
// independent real GenDot pairs, so Re conj(x).y = a.b + c.d cancels
// heavily; Im conj(x).y = a.d - c.b is an ordinary random sum.
extern "C" int hpb_gendot_c128(uint64_t seed, int64_t n, double cond, double* x, double* y) {
    if (n < 0 || (n > 0 && (x == nullptr || y == nullptr)) || !(cond >= 1.0)) return HPB_ERROR_INVALID_VALUE;
    if (n == 0) return HPB_SUCCESS;
    double* buf = new (std::nothrow) double[size_t(4 * n)];
    if (buf == nullptr) return HPB_ERROR_OUT_OF_MEMORY;
    int st = hpb_gendot_f64(seed ^ 0xA5A5ull, n, cond, buf, buf + n, nullptr);
    if (st == HPB_SUCCESS) st = hpb_gendot_f64(seed ^ 0x5A5Aull, n, cond, buf + 2 * n, buf + 3 * n, nullptr);
    if (st == HPB_SUCCESS) {
        for (int64_t i = 0; i < n; ++i) {
            x[2 * i] = buf[i];
            y[2 * i] = buf[n + i];
            x[2 * i + 1] = buf[2 * n + i];
            y[2 * i + 1] = buf[3 * n + i];
        }
    }
    delete[] buf;
    return st;
}
