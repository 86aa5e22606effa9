// BiCGStab of van der Vorst over the VectorOperations concept.
//
// Interface of the reference's numerical_algos::lin_solvers::bicgstab
// (numerical_algos/lin_solvers/bicgstab.h:64-254): set_use_precond_resid,
// set_resid_recalc_freq, set_preconditioner, monitor(), solve(A, b, x);
// left preconditioning; one monitor test and one counted iteration per
// BiCGStab step; the step stops when beta, alpha or omega becomes NaN/Inf.
// Unlike the reference (which then returns true), such a breakdown is
// reported through breakdown() and solve() returns the monitor's verdict.
#ifndef HPBLAS1_SOLVERS_BICGSTAB_H
#define HPBLAS1_SOLVERS_BICGSTAB_H

#include <stdexcept>

#include "monitor.h"
#include "vector_pool.h"

namespace hpb {
namespace solvers {

template <class LinearOperator, class Preconditioner, class VectorOperations, class Monitor, class Log = null_log>
class bicgstab {
public:
    using scalar_type = typename VectorOperations::scalar_type;
    using vector_type = typename VectorOperations::vector_type;
    using T = scalar_type;

    explicit bicgstab(const VectorOperations* ops, Log* log = nullptr, int = 3) : ops_(ops), log_(log), monitor_(*ops, log) {}
    ~bicgstab() {
        if (prec_ && own_prec_) delete prec_;
    }
    void set_use_precond_resid(bool on) { use_precond_resid_ = on; }
    void set_resid_recalc_freq(int f) { resid_recalc_freq_ = f; }
    void set_preconditioner(Preconditioner* p, bool own = false) {
        prec_ = p;
        own_prec_ = own;
    }
    Monitor& monitor() { return monitor_; }
    const Monitor& monitor() const { return monitor_; }
    bool breakdown() const { return breakdown_; }

    bool solve(const LinearOperator& A, const vector_type& b, vector_type& x) const {
        if (!use_precond_resid_ && prec_)
            throw std::logic_error("bicgstab::solve: unpreconditioned residual with a preconditioner is not supported");
        if (prec_) prec_->set_operator(&A);
        vector_pool<VectorOperations> pool(ops_, 6);
        vector_type &r = pool[0], &rs = pool[1], &p = pool[2], &v = pool[3], &s = pool[4], &t = pool[5];
        if (prec_) {
            ops_->assign(b, r);
            prec_->apply(r);
            monitor_.start(r);
        } else {
            monitor_.start(b);
        }
        residual(A, x, b, r);
        ops_->assign(r, rs);
        T rho_prev(1), alpha(1), omega(1);
        ops_->assign_scalar(T(0), v);
        ops_->assign_scalar(T(0), p);
        breakdown_ = false;
        while (!monitor_.check_finished(x, r)) {
            T rho = ops_->scalar_prod(rs, r);
            T beta = (rho / rho_prev) * (alpha / omega);
            if (!finite_of(beta)) {
                breakdown_ = true;
                break;
            }
            ops_->add_mul(T(1), r, -beta * omega, v, beta, p);  // p = r + beta (p - omega v)
            A.apply(p, v);
            if (prec_) prec_->apply(v);
            alpha = rho / ops_->scalar_prod(rs, v);
            if (!finite_of(alpha)) {
                breakdown_ = true;
                break;
            }
            ops_->assign_mul(T(1), r, -alpha, v, s);  // s = r - alpha v
            A.apply(s, t);
            if (prec_) prec_->apply(t);
            T omega_new = ops_->scalar_prod(t, s) / ops_->scalar_prod(t, t);
            if (!finite_of(omega_new)) {
                breakdown_ = true;
                break;
            }
            ops_->add_mul(alpha, p, omega_new, s, T(1), x);  // x += alpha p + omega s
            if (resid_recalc_freq_ > 0 && (monitor_.iters_performed() + 1) % resid_recalc_freq_ == 0)
                residual(A, x, b, r);
            else
                ops_->assign_mul(T(1), s, -omega_new, t, r);  // r = s - omega t
            omega = omega_new;
            rho_prev = rho;
            ++monitor_;
        }
        const bool ok = monitor_.converged();
        if (!ok && log_) log_->error_f("bicgstab::solve: linear solver failed to converge");
        return ok;
    }

private:
    void residual(const LinearOperator& A, const vector_type& x, const vector_type& b, vector_type& r) const {
        A.apply(x, r);
        ops_->add_mul(T(1), b, -T(1), r);
        if (prec_) prec_->apply(r);
    }
    const VectorOperations* ops_;
    Log* log_;
    mutable Monitor monitor_;
    Preconditioner* prec_ = nullptr;
    bool own_prec_ = false;
    bool use_precond_resid_ = true;
    int resid_recalc_freq_ = 0;
    mutable bool breakdown_ = false;
};

}  // namespace solvers
}  // namespace hpb

#endif
