// Convergence monitor for the Krylov solvers in this directory.
//
// Same contract as the reference's default_monitor
// (numerical_algos/lin_solvers/default_monitor.h:53-227): tolerance
// tol = abs_tol + rel_tol * ||rhs||, a finiteness check of the iterate at
// every test, optional convergence history of (iteration, residual norm),
// and "finished" = converged (after min_iters) or max_iters reached.
#ifndef HPBLAS1_SOLVERS_MONITOR_H
#define HPBLAS1_SOLVERS_MONITOR_H

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <utility>
#include <vector>

#include <thrust/complex.h>

namespace hpb {
namespace solvers {

template <class T> struct real_part_type { using type = T; };
template <class R> struct real_part_type<thrust::complex<R> > { using type = R; };

template <class T> inline T conj_of(const T& v) { return v; }
template <class R> inline thrust::complex<R> conj_of(const thrust::complex<R>& v) { return thrust::conj(v); }
template <class T> inline typename real_part_type<T>::type abs_of(const T& v) { return std::abs(v); }
template <class R> inline R abs_of(const thrust::complex<R>& v) { return thrust::abs(v); }
template <class T> inline bool finite_of(const T& v) { return std::isfinite(v); }
template <class R> inline bool finite_of(const thrust::complex<R>& v) {
    return std::isfinite(v.real()) && std::isfinite(v.imag());
}

// A logger that drops everything; any type with info_f / error_f (printf
// style) can be used instead, e.g. a wrapper around the reference's
// utils::log_std.
struct null_log {
    void info_f(const char*, ...) {}
    void error_f(const char*, ...) {}
};

struct stderr_log {
    int level = 1;
    void info_f(const char* fmt, ...) {
        if (level < 2) return;
        va_list ap;
        va_start(ap, fmt);
        std::vfprintf(stderr, fmt, ap);
        va_end(ap);
        std::fputc('\n', stderr);
    }
    void error_f(const char* fmt, ...) {
        va_list ap;
        va_start(ap, fmt);
        std::vfprintf(stderr, fmt, ap);
        va_end(ap);
        std::fputc('\n', stderr);
    }
};

template <class VectorOperations, class Log = null_log>
class default_monitor {
public:
    using scalar_type = typename VectorOperations::scalar_type;
    using vector_type = typename VectorOperations::vector_type;
    using real_type = typename real_part_type<scalar_type>::type;

    explicit default_monitor(const VectorOperations& ops, Log* log = nullptr, int = 0) : ops_(ops), log_(log) {}

    void init(real_type rel_tol, real_type abs_tol = real_type(0), int max_iters = 100, int min_iters = 0,
              bool out_min_resid_norm = false, bool save_history = false, bool divide_by_rel_base = false) {
        rel_tol_ = rel_tol;
        abs_tol_ = abs_tol;
        max_iters_ = max_iters;
        min_iters_ = min_iters;
        (void)out_min_resid_norm;
        save_history_ = save_history;
        divide_by_rel_base_ = divide_by_rel_base;
    }
    void set_save_convergence_history(bool on) { save_history_ = on; }
    void set_divide_out_norms_by_rel_base(bool on) { divide_by_rel_base_ = on; }
    void set_temp_tolerance(real_type t) {
        saved_rel_tol_ = rel_tol_;
        rel_tol_ = t;
    }
    void restore_tolerance() { rel_tol_ = saved_rel_tol_; }
    void set_temp_max_iterations(int m) {
        saved_max_iters_ = max_iters_;
        max_iters_ = m;
    }
    void restore_max_iterations() { max_iters_ = saved_max_iters_; }

    void start(const vector_type& rhs) {
        rhs_norm_ = real_type(ops_.norm(rhs));
        iters_ = 0;
        history_.clear();
    }
    // start from a known right-hand-side norm (no reduction)
    void start_with_norm(real_type rhs_norm) {
        rhs_norm_ = rhs_norm;
        iters_ = 0;
        history_.clear();
    }
    void stop() {}

    real_type rel_tol() const { return rel_tol_; }
    real_type abs_tol() const { return abs_tol_; }
    real_type rel_tol_base() const { return rhs_norm_; }
    real_type tol() const { return abs_tol_ + rel_tol_ * rhs_norm_; }
    int max_iters_num() const { return max_iters_; }
    int min_iters_num() const { return min_iters_; }
    int iters_performed() const { return iters_; }
    bool is_valid_number() const { return valid_; }
    real_type rhs_norm() const { return rhs_norm_; }
    real_type resid_norm() const { return resid_norm_; }
    real_type resid_norm_out() const { return divide_by_rel_base_ ? resid_norm_ / rhs_norm_ : resid_norm_; }
    real_type tol_out() const { return divide_by_rel_base_ ? tol() / rhs_norm_ : tol(); }
    const std::vector<std::pair<int, real_type> >& convergence_history() const { return history_; }

    default_monitor& operator++() {
        ++iters_;
        return *this;
    }
    default_monitor& operator+=(int n) {
        iters_ += n;
        return *this;
    }
    bool converged() const { return valid_ && resid_norm_ <= tol(); }

    bool check_finished(const vector_type& x, const vector_type& r) {
        valid_ = ops_.check_is_valid_number(x);
        if (!valid_) {
            if (log_) log_->info_f("monitor: iterate is not a finite vector at iteration %d", iters_);
            return true;
        }
        return record(real_type(ops_.norm(r)));
    }
    // same test with an externally computed residual norm (device-resident
    // solvers compute it fused with other work); `valid` is the finiteness
    // of the iterate
    bool check_finished_norm(real_type resid_norm, bool valid) {
        valid_ = valid && std::isfinite(resid_norm);
        if (!valid_) return true;
        return record(resid_norm);
    }

private:
    bool record(real_type rn) {
        resid_norm_ = rn;
        if (log_) log_->info_f("monitor: iter = %d resid norm = %0.6e tol = %0.6e", iters_, double(resid_norm_out()),
                               double(tol_out()));
        if (save_history_) history_.emplace_back(iters_, resid_norm_out());
        return (converged() && iters_ >= min_iters_) || iters_ >= max_iters_;
    }

    const VectorOperations& ops_;
    Log* log_;
    real_type rel_tol_ = real_type(1e-6), abs_tol_ = real_type(0), saved_rel_tol_ = real_type(1e-6);
    int max_iters_ = 100, min_iters_ = 0, saved_max_iters_ = 100;
    bool save_history_ = false, divide_by_rel_base_ = false;
    int iters_ = 0;
    bool valid_ = true;
    real_type rhs_norm_ = real_type(0), resid_norm_ = real_type(0);
    std::vector<std::pair<int, real_type> > history_;
};

}  // namespace solvers
}  // namespace hpb

#endif
