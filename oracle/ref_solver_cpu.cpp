// oracle/ref_solver_cpu.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's own Krylov solvers on the CPU: numerical_algos::
// lin_solvers::bicgstabl / gmres (bicgstabl.h, gmres.h) with its
// default_monitor and cpu_vector_operations<double> (sequential or
// std::thread Dot2, common/cpu_vector_operations.h), compiled from the
// reference sources into oracle/_ref/.  The reference has no CPU CSR
// product, so this harness supplies the linear operator (an OpenMP CSR
// SpMV, y = A x with one FMA per nonzero in index order) and an identity
// preconditioner.  Used as the timed CPU solver baseline and to compare
// iteration counts with the GPU solvers.
#include <common/cpu_vector_operations.h>
#include <numerical_algos/lin_solvers/bicgstabl.h>
#include <numerical_algos/lin_solvers/default_monitor.h>
#include <numerical_algos/lin_solvers/gmres.h>
#include <utils/log.h>

#include <chrono>
#include <cmath>
#include <cstdint>

namespace {

struct csr_op {
    int n;
    const int* rp;
    const int* ci;
    const double* v;
    void apply(double* const& x, double*& f) const {
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; ++r) {
            double s = 0.0;
            for (int k = rp[r]; k < rp[r + 1]; ++k) s = std::fma(v[k], x[ci[k]], s);
            f[r] = s;
        }
    }
};

struct identity_prec {
    void set_operator(const csr_op*) {}
    void apply(double*&) const {}
};

struct quiet_log : public utils::log_std {
    quiet_log() { set_verbosity(0); }
};

using vec_ops_t = cpu_vector_operations<double>;
using mon_t = numerical_algos::lin_solvers::default_monitor<vec_ops_t, utils::log_std>;

void copy_history(const std::vector<std::pair<int, double> >& h, double* out, int cap, int* len) {
    if (out == nullptr) return;
    int k = 0;
    for (; k < int(h.size()) && k < cap; ++k) {
        out[2 * k] = double(h[k].first);
        out[2 * k + 1] = h[k].second;
    }
    if (len) *len = k;
}

}  // namespace

extern "C" {

// method 0: BiCGStab(basis), 1: GMRES(basis).  max_iters caps the
// monitor's iteration counter (BiCGStab(l) counts l per cycle).
// threads: 0/1 -> sequential Dot2, >1 -> threaded_reduction with that many
// threads (<0 -> hardware_concurrency).  Returns 1 if converged.
// hist (optional, 2 * hist_cap doubles): the monitor's convergence history,
// (iteration, ||r||) pairs as default_monitor records them
// (default_monitor.h:206-212); *hist_len receives the number of pairs.
int ref_cpu_solve_hist_f64(int method, int n, const int* rp, const int* ci, const double* v, double* b, double* x,
                           int basis, double rel_tol, int max_iters, int high_prec, int threads, int* iters_out,
                           double* resid_out, double* seconds_out, double* hist, int hist_cap, int* hist_len);

int ref_cpu_solve_f64(int method, int n, const int* rp, const int* ci, const double* v, double* b, double* x,
                      int basis, double rel_tol, int max_iters, int high_prec, int threads, int* iters_out,
                      double* resid_out, double* seconds_out) {
    return ref_cpu_solve_hist_f64(method, n, rp, ci, v, b, x, basis, rel_tol, max_iters, high_prec, threads,
                                  iters_out, resid_out, seconds_out, nullptr, 0, nullptr);
}

int ref_cpu_solve_hist_f64(int method, int n, const int* rp, const int* ci, const double* v, double* b, double* x,
                           int basis, double rel_tol, int max_iters, int high_prec, int threads, int* iters_out,
                           double* resid_out, double* seconds_out, double* hist, int hist_cap, int* hist_len) {
    if (threads < 0) threads = int(std::thread::hardware_concurrency());
    vec_ops_t ops(size_t(n), high_prec, threads);
    if (high_prec)
        ops.use_high_precision();
    else
        ops.use_standard_precision();
    csr_op A{n, rp, ci, v};
    identity_prec prec;
    utils::log_std log;
    log.set_verbosity(0);
    auto t0 = std::chrono::steady_clock::now();
    bool ok = false;
    int iters = 0;
    double resid = 0;
    if (method == 0) {
        numerical_algos::lin_solvers::bicgstabl<csr_op, identity_prec, vec_ops_t, mon_t, utils::log_std> s(&ops, &log);
        s.set_basis_size(basis);
        s.monitor().init(rel_tol, 0.0, max_iters, 0, false, hist != nullptr);
        ok = s.solve(A, b, x);
        iters = s.monitor().iters_performed();
        resid = s.monitor().resid_norm();
        copy_history(s.monitor().convergence_history(), hist, hist_cap, hist_len);
    } else {
        numerical_algos::lin_solvers::gmres<csr_op, identity_prec, vec_ops_t, mon_t, utils::log_std> s(&ops, &log);
        s.set_restarts(unsigned(basis));
        s.set_reorthogonalization(false);
        s.monitor().init(rel_tol, 0.0, max_iters, 0, false, hist != nullptr);
        ok = s.solve(A, b, x);
        iters = s.monitor().iters_performed();
        resid = s.monitor().resid_norm();
        copy_history(s.monitor().convergence_history(), hist, hist_cap, hist_len);
    }
    if (seconds_out) *seconds_out = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (iters_out) *iters_out = iters;
    if (resid_out) *resid_out = resid;
    return ok ? 1 : 0;
}

}  // extern "C"
