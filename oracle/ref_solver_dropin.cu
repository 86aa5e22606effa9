// oracle/ref_solver_dropin.cu -- TEST INFRASTRUCTURE ONLY.
//
// The reference's own solver code (numerical_algos/lin_solvers/bicgstabl.h,
// gmres.h, default_monitor.h, utils/log.h), compiled UNCHANGED against this
// repository's C++ drop-in headers (include/hpblas1_dropin: the reference's
// gpu_vector_operations / csr::gpu_matrix / csr::linear_operator /
// csr::preconditioner interfaces) and linked to libhpblas1.so.  Built into
// oracle/_ref/ from the reference sources where they lie (oracle/Makefile).
// A GPU test runs it beside the library's own solvers on the same device
// arrays: same recurrences, same kernels -> same iterates.
#include <common/csr/gpu_ilu0_preconditioner.h>
#include <common/csr/gpu_matrix.h>
#include <common/csr/linear_operator.h>
#include <common/csr/preconditioner.h>
#include <common/gpu_vector_operations.h>
#include <common/ogita/gpu_reduction_ogita.h>
#include <numerical_algos/lin_solvers/bicgstabl.h>
#include <numerical_algos/lin_solvers/default_monitor.h>
#include <numerical_algos/lin_solvers/gmres.h>
#include <utils/log.h>

#include <cstdint>

namespace {
using vec_ops_t = gpu_vector_operations<double>;
using mat_t = csr::gpu_matrix<vec_ops_t, cublas_wrap>;
using lin_op_t = csr::linear_operator<vec_ops_t, mat_t>;
using prec_t = csr::preconditioner<vec_ops_t, lin_op_t, mat_t>;
using ilu_t = csr::gpu_ilu0_preconditioner<vec_ops_t, lin_op_t, mat_t>;
using log_t = utils::log_std;
using mon_t = numerical_algos::lin_solvers::default_monitor<vec_ops_t, log_t>;

template <class Prec>
int run_solver(Prec& prec, vec_ops_t& vec_ops, lin_op_t& lin_op, int method, double* b, double* x, int basis,
               double rel_tol, int max_iters, int* iters_out, double* resid_out) {
    log_t log;
    log.set_verbosity(0);
    bool ok = false;
    if (method == 0) {
        numerical_algos::lin_solvers::bicgstabl<lin_op_t, Prec, vec_ops_t, mon_t, log_t> s(&vec_ops, &log);
        s.set_preconditioner(&prec);
        s.set_basis_size(basis);
        s.monitor().init(rel_tol, 0.0, max_iters);
        ok = s.solve(lin_op, b, x);
        *iters_out = s.monitor().iters_performed();
        *resid_out = s.monitor().resid_norm();
    } else {
        numerical_algos::lin_solvers::gmres<lin_op_t, Prec, vec_ops_t, mon_t, log_t, 300> s(&vec_ops, &log);
        s.set_preconditioner(&prec);
        s.set_restarts(unsigned(basis));
        s.set_reorthogonalization(false);
        s.monitor().init(rel_tol, 0.0, max_iters);
        ok = s.solve(lin_op, b, x);
        *iters_out = s.monitor().iters_performed();
        *resid_out = s.monitor().resid_norm();
    }
    vec_ops.sync();
    return ok ? 1 : 0;
}

}  // namespace

extern "C" {

// method 0: bicgstabl(basis), 1: gmres(basis); precond 0: csr::preconditioner
// without factors (the identity), 1: csr::gpu_ilu0_preconditioner of A.
// Device arrays; x holds the initial guess.  Returns 1 if the reference's
// monitor reports convergence.
int ref_dropin_solve_prec_f64(int method, int precond, int rows, int64_t nnz, const int* rp, const int* ci,
                              const double* val, double* b, double* x, int basis, double rel_tol, int max_iters,
                              int high_prec, int* iters_out, double* resid_out) {
    cublas_wrap cublas(false);
    vec_ops_t vec_ops(size_t(rows), &cublas);
    if (high_prec)
        vec_ops.use_high_precision();
    else
        vec_ops.use_standard_precision();
    mat_t mat(&cublas);
    mat.attach(rows, rows, int(nnz), rp, ci, val);
    lin_op_t lin_op(&vec_ops, &mat);
    if (precond == 1) {
        ilu_t prec(&vec_ops);
        prec.set_matrix(mat);
        return run_solver(prec, vec_ops, lin_op, method, b, x, basis, rel_tol, max_iters, iters_out, resid_out);
    }
    prec_t prec(&vec_ops);
    return run_solver(prec, vec_ops, lin_op, method, b, x, basis, rel_tol, max_iters, iters_out, resid_out);
}

// The drop-in's transposed operations on one matrix (device arrays):
// y = A^T x (csr::gpu_matrix::axpy with transpose_ = true), z solves
// L^T z = x with L the unit lower triangle, w solves U^T w = x with U the
// upper triangle with its diagonal.  Returns 1.
int ref_dropin_transposed_ops_f64(int rows, int64_t nnz, const int* rp, const int* ci, const double* val,
                                  double* x, double* y, double* z, double* w) {
    cublas_wrap cublas(false);
    mat_t mat(&cublas);
    mat.attach(rows, rows, int(nnz), rp, ci, val);
    mat.axpy(1.0, x, 0.0, y, true);
    mat.triangular_solve_lower(x, z, 1.0, true);
    mat.triangular_solve_upper(x, w, 1.0, true);
    cudaDeviceSynchronize();
    return 1;
}

int ref_dropin_solve_f64(int method, int rows, int64_t nnz, const int* rp, const int* ci, const double* val,
                         double* b, double* x, int basis, double rel_tol, int max_iters, int high_prec,
                         int* iters_out, double* resid_out) {
    return ref_dropin_solve_prec_f64(method, 0, rows, nnz, rp, ci, val, b, x, basis, rel_tol, max_iters, high_prec,
                                     iters_out, resid_out);
}

}  // extern "C"

// The drop-in reducer class gpu_reduction_ogita<T, T*> (the reference's
// common/ogita/gpu_reduction_ogita.h interface) on device vectors: what the
// reference's own drivers call (test_vector_operations.cpp:100, :211, :304).
// out: dot, sum (complex: re, im each), asum, norm -- 6 doubles.
namespace {
template <class T>
void reducer_all(int64_t n, const void* x, const void* y, double* out) {
    gpu_reduction_ogita<T, T*> r(static_cast<size_t>(n));
    T* xp = static_cast<T*>(const_cast<void*>(x));
    T* yp = static_cast<T*>(const_cast<void*>(y));
    thrust::complex<double> d(r.dot(xp, yp)), s(r.sum(xp));
    out[0] = d.real();
    out[1] = d.imag();
    out[2] = s.real();
    out[3] = s.imag();
    out[4] = double(r.asum(xp));
    out[5] = double(r.norm(xp));
}
}  // namespace

extern "C" int ref_dropin_reducer(int type, int64_t n, const void* x, const void* y, double* out) {
    try {
        switch (type) {
            case 0: reducer_all<float>(n, x, y, out); break;
            case 1: reducer_all<double>(n, x, y, out); break;
            case 2: reducer_all<thrust::complex<float> >(n, x, y, out); break;
            case 3: reducer_all<thrust::complex<double> >(n, x, y, out); break;
            default: return -1;
        }
    } catch (...) {
        return -2;
    }
    return 0;
}
