// C ABI of the Krylov solvers on CSR matrices, built from the C++ drop-in
// (gpu_vector_operations, csr::gpu_matrix, csr::linear_operator,
// csr::jacobi_preconditioner) and the solver templates of
// include/hpblas1/solvers/.  This is the plain drop-in path: every
// reduction returns its value to the host, exactly as the reference's
// solvers over gpu_vector_operations do (numerical_algos/lin_solvers/*.h
// driven as in test_csr_linear_solver.cpp:101-353).
#include <chrono>
#include <memory>
#include <new>
#include <stdexcept>
#include <type_traits>

#include <common/csr/gpu_ilu0_preconditioner.h>
#include <common/csr/gpu_matrix.h>
#include <common/csr/linear_operator.h>
#include <common/csr/preconditioner.h>
#include <common/gpu_vector_operations.h>

#include <hpblas1/solvers/bicgstab.h>
#include <hpblas1/solvers/bicgstabl.h>
#include <hpblas1/solvers/gmres.h>

#include "hpb_common.cuh"
#include "hpb_fused.cuh"

namespace {

template <class T> struct storage_of { using type = T; };
template <> struct storage_of<thrust::complex<float> > { using type = hpb::cf; };
template <> struct storage_of<thrust::complex<double> > { using type = hpb::cd; };

template <class T>
struct Stack {
    using VO = gpu_vector_operations<T>;
    using MAT = csr::gpu_matrix<VO, cublas_wrap>;
    using LO = csr::linear_operator<VO, MAT>;
    using PJ = csr::jacobi_preconditioner<VO, LO, MAT>;
    using PI = csr::gpu_ilu0_preconditioner<VO, LO, MAT>;
    using MON = hpb::solvers::default_monitor<VO>;
};

// The preconditioner the solver templates are instantiated with: Jacobi
// (D^-1) or ILU(0) ((L U)^-1 by two sparse triangular solves).
template <class S>
struct AnyPrec {
    std::unique_ptr<typename S::PJ> jac;
    std::unique_ptr<typename S::PI> ilu;
    void set_operator(const typename S::LO*) {}
    void apply(typename S::VO::vector_type& x) const {
        if (jac)
            jac->apply(x);
        else if (ilu)
            ilu->apply(x);
    }
};

template <class Solver, class Mon>
void fill_report(const Mon& mon, hpb_solver_report* rep, double* hist, int cap) {
    rep->iters = mon.iters_performed();
    rep->rhs_norm = double(mon.rhs_norm());
    rep->resid_norm = double(mon.resid_norm());
    rep->converged = mon.converged() ? 1 : 0;
    const auto& h = mon.convergence_history();
    int k = 0;
    for (; k < int(h.size()) && k < cap; ++k) {
        hist[2 * k] = double(h[k].first);
        hist[2 * k + 1] = double(h[k].second);
    }
    rep->history_len = k;
}

template <class T>
int solve_device(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
                 const T* val, const T* b, T* x, hpb_solver_report* rep, double* hist, int cap) {
    using S = Stack<T>;
    if (p == nullptr || rep == nullptr || rows < 0 || nnz < 0 || nnz > INT32_MAX || (cap > 0 && hist == nullptr))
        return HPB_ERROR_INVALID_VALUE;
    *rep = hpb_solver_report{};
    if (rows == 0) {
        rep->converged = 1;
        return HPB_SUCCESS;
    }
    if (p->fused) {
        using E = typename storage_of<T>::type;
        if (p->method == HPB_SOLVER_BICGSTABL)
            return hpb::fused::solve_bicgstabl<E>(p, rows, nnz, rp, ci, reinterpret_cast<const E*>(val),
                                                  reinterpret_cast<const E*>(b), reinterpret_cast<E*>(x), rep, hist,
                                                  cap);
        if (p->method == HPB_SOLVER_GMRES) {
            hpb::fused::RightPrec<E> M;
            hpb::fused::IluFactors<E> F;
            if (p->precond == HPB_PRECOND_JACOBI) {
                M.kind = 1;
            } else if (p->precond == HPB_PRECOND_ILU0) {
                const int st = F.build(rows, nnz, rp, ci, reinterpret_cast<const E*>(val));
                if (st != HPB_SUCCESS) return st;
                M.kind = 3;
                M.val = F.lu;
                M.lower = F.lower;
                M.upper = F.upper;
                M.sweeps = p->ilu_sweeps;
            } else if (p->precond != HPB_PRECOND_NONE) {
                return HPB_ERROR_NOT_SUPPORTED;
            }
            return hpb::fused::solve_gmres<E>(p, rows, nnz, rp, ci, reinterpret_cast<const E*>(val), M,
                                              reinterpret_cast<const E*>(b), reinterpret_cast<E*>(x), rep, hist, cap,
                                              0);
        }
        return HPB_ERROR_NOT_SUPPORTED;
    }
    T* bm = const_cast<T*>(b);  // the solver concept takes non-const vector references
    try {
        typename S::VO ops(static_cast<size_t>(rows), nullptr);
        if (p->high_precision)
            ops.use_high_precision();
        else
            ops.use_standard_precision();
        typename S::MAT A;
        A.attach(rows, rows, int(nnz), rp, ci, val);
        typename S::LO op(&ops, &A);
        std::unique_ptr<AnyPrec<S> > jac;
        if (p->precond == HPB_PRECOND_JACOBI) {
            jac.reset(new AnyPrec<S>);
            jac->jac.reset(new typename S::PJ(&ops));
            jac->jac->set_matrix(&A);
        } else if (p->precond == HPB_PRECOND_ILU0) {
            if (p->ilu_sweeps != 0) return HPB_ERROR_NOT_SUPPORTED;  // the drop-in applies the factors exactly
            jac.reset(new AnyPrec<S>);
            jac->ilu.reset(new typename S::PI(&ops));
            jac->ilu->set_matrix(A);
        } else if (p->precond != HPB_PRECOND_NONE) {
            return HPB_ERROR_NOT_SUPPORTED;
        }
        using R = typename hpb::solvers::real_part_type<T>::type;
        ops.sync();
        auto t0 = std::chrono::steady_clock::now();
        bool ok = false;
        if (p->method == HPB_SOLVER_BICGSTABL) {
            hpb::solvers::bicgstabl<typename S::LO, AnyPrec<S>, typename S::VO, typename S::MON> sv(&ops);
            sv.set_basis_size(p->basis > 0 ? p->basis : 2);
            sv.set_resid_recalc_freq(p->resid_recalc_freq);
            if (jac) sv.set_preconditioner(jac.get());
            sv.monitor().init(R(p->rel_tol), R(p->abs_tol), p->max_iters, 0, false, cap > 0);
            ok = sv.solve(op, bm, x);
            rep->breakdown = sv.breakdown_flag() < 0 ? 1 : 0;
            fill_report<decltype(sv)>(sv.monitor(), rep, hist, cap);
        } else if (p->method == HPB_SOLVER_GMRES) {
            hpb::solvers::gmres<typename S::LO, AnyPrec<S>, typename S::VO, typename S::MON> sv(&ops);
            sv.set_restarts(unsigned(p->basis > 0 ? p->basis : 30));
            sv.set_reorthogonalization(p->reorthogonalize != 0);
            sv.set_early_exit(p->early_exit != 0);
            if (jac) sv.set_preconditioner(jac.get());
            sv.monitor().init(R(p->rel_tol), R(p->abs_tol), p->max_iters, 0, false, cap > 0);
            ok = sv.solve(op, bm, x);
            fill_report<decltype(sv)>(sv.monitor(), rep, hist, cap);
        } else if (p->method == HPB_SOLVER_BICGSTAB) {
            hpb::solvers::bicgstab<typename S::LO, AnyPrec<S>, typename S::VO, typename S::MON> sv(&ops);
            sv.set_resid_recalc_freq(p->resid_recalc_freq);
            if (jac) sv.set_preconditioner(jac.get());
            sv.monitor().init(R(p->rel_tol), R(p->abs_tol), p->max_iters, 0, false, cap > 0);
            ok = sv.solve(op, bm, x);
            rep->breakdown = sv.breakdown() ? 1 : 0;
            fill_report<decltype(sv)>(sv.monitor(), rep, hist, cap);
        } else {
            return HPB_ERROR_NOT_SUPPORTED;
        }
        ops.sync();
        rep->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        // true residual ||b - A x|| and ||b|| with compensated reductions
        const bool hp = ops.get_current_precision();
        ops.use_high_precision();
        T* r = nullptr;
        ops.init_vector(r);
        ops.start_use_vector(r);
        op.apply(x, r);
        ops.add_mul(T(1), bm, -T(1), r);
        rep->true_resid_norm = double(ops.norm(r));
        rep->true_rhs_norm = double(ops.norm(bm));
        ops.free_vector(r);
        if (!hp) ops.use_standard_precision();
        (void)ok;
        return rep->converged ? HPB_SUCCESS : (rep->breakdown ? HPB_ERROR_BREAKDOWN : HPB_ERROR_NOT_CONVERGED);
    } catch (const std::bad_alloc&) {
        return HPB_ERROR_OUT_OF_MEMORY;
    } catch (const std::logic_error&) {
        return HPB_ERROR_NOT_SUPPORTED;
    } catch (const std::exception&) {
        return HPB_ERROR_CUDA;
    }
}

template <class T>
int solve_host(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
               const T* val, const T* b, T* x, hpb_solver_report* rep, double* hist, int cap) {
    if (rows < 0 || nnz < 0) return HPB_ERROR_INVALID_VALUE;
    // device copies from the solvers' memory pool, stream-ordered on the
    // legacy default stream (no cudaMalloc/cudaFree per call)
    using hpb::fused::pool_alloc;
    using hpb::fused::pool_free;
    const size_t n = size_t(rows);
    void* d_rp = pool_alloc((n + 1) * 4, nullptr);
    void* d_ci = pool_alloc(size_t(nnz ? nnz : 1) * 4, nullptr);
    void* d_val = pool_alloc(size_t(nnz ? nnz : 1) * sizeof(T), nullptr);
    void* d_b = pool_alloc((n ? n : 1) * sizeof(T), nullptr);
    void* d_x = pool_alloc((n ? n : 1) * sizeof(T), nullptr);
    auto cleanup = [&]() {
        for (void* q : {d_rp, d_ci, d_val, d_b, d_x}) pool_free(q, nullptr);
        cudaStreamSynchronize(nullptr);
    };
    if (!d_rp || !d_ci || !d_val || !d_b || !d_x) {
        cleanup();
        return HPB_ERROR_OUT_OF_MEMORY;
    }
    int st = HPB_SUCCESS;
    if (cudaMemcpy(d_rp, rp, (n + 1) * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_ci, ci, size_t(nnz) * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_val, val, size_t(nnz) * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_b, b, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_x, x, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        st = HPB_ERROR_CUDA;
    if (st == HPB_SUCCESS)
        st = solve_device<T>(p, rows, nnz, static_cast<int32_t*>(d_rp), static_cast<int32_t*>(d_ci),
                             static_cast<T*>(d_val), static_cast<T*>(d_b), static_cast<T*>(d_x), rep, hist, cap);
    if ((st == HPB_SUCCESS || st == HPB_ERROR_NOT_CONVERGED || st == HPB_ERROR_BREAKDOWN) &&
        cudaMemcpy(x, d_x, n * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = HPB_ERROR_CUDA;
    cleanup();
    return st;
}

}  // namespace

using cf = thrust::complex<float>;
using cd = thrust::complex<double>;

extern "C" {

int hpb_solver_params_default(hpb_solver_params* p) {
    if (p == nullptr) return HPB_ERROR_INVALID_VALUE;
    *p = hpb_solver_params{};
    p->method = HPB_SOLVER_BICGSTABL;
    p->basis = 2;
    p->rel_tol = 1e-10;
    p->abs_tol = 0.0;
    p->max_iters = 10000;
    p->precond = HPB_PRECOND_NONE;
    p->high_precision = 1;
    return HPB_SUCCESS;
}

#define HPB_SOLVE_DEF(SUF, T, PT)                                                                              \
    int hpb_csr_solve_##SUF(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,     \
                            const int32_t* col_ind, const PT* val, const PT* b, PT* x, hpb_solver_report* rep,   \
                            double* history, int history_cap) {                                                \
        return solve_device<T>(p, rows, nnz, row_ptr, col_ind, reinterpret_cast<const T*>(val),                \
                               reinterpret_cast<const T*>(b), reinterpret_cast<T*>(x), rep, history, history_cap); \
    }                                                                                                          \
    int hpb_csr_solve_##SUF##_host(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr, \
                                   const int32_t* col_ind, const PT* val, const PT* b, PT* x,                  \
                                   hpb_solver_report* rep, double* history, int history_cap) {                 \
        return solve_host<T>(p, rows, nnz, row_ptr, col_ind, reinterpret_cast<const T*>(val),                  \
                             reinterpret_cast<const T*>(b), reinterpret_cast<T*>(x), rep, history, history_cap); \
    }

HPB_SOLVE_DEF(f32, float, float)
HPB_SOLVE_DEF(f64, double, double)
HPB_SOLVE_DEF(c64, cf, void)
HPB_SOLVE_DEF(c128, cd, void)

}  // extern "C"
