// BiCGStab(l) of Sleijpen and Fokkema over the VectorOperations concept.
//
// Interface of the reference's numerical_algos::lin_solvers::bicgstabl
// (numerical_algos/lin_solvers/bicgstabl.h:68-275): template parameters
// <LinearOperator, Preconditioner, VectorOperations, Monitor, Log>,
// set_basis_size / set_use_precond_resid / set_resid_recalc_freq /
// set_preconditioner / monitor() / solve(A, b, x), left preconditioning
// r = P(b - A x), u_{j+1} = P A u_j, one monitor test per BiCG+MR cycle and
// the iteration counter advanced by l per cycle.
//
// The algorithm is the published one: l BiCG steps building r_0..r_l and
// u_0..u_l, then a minimal-residual polynomial step in which r_1..r_l are
// orthogonalised by modified Gram-Schmidt (tau, sigma) and gamma, gamma',
// gamma'' follow from the triangular system.  Inner products are written
// <a, b> = sum conj(a_i) b_i with the left argument being the one the
// algorithm conjugates, so the solver is also correct for complex data; on
// real data the values equal those of the reference's ordering.
#ifndef HPBLAS1_SOLVERS_BICGSTABL_H
#define HPBLAS1_SOLVERS_BICGSTABL_H

#include <stdexcept>
#include <vector>

#include "monitor.h"
#include "vector_pool.h"

namespace hpb {
namespace solvers {

template <class LinearOperator, class Preconditioner, class VectorOperations, class Monitor, class Log = null_log>
class bicgstabl {
public:
    using scalar_type = typename VectorOperations::scalar_type;
    using vector_type = typename VectorOperations::vector_type;
    using T = scalar_type;

    explicit bicgstabl(const VectorOperations* ops, Log* log = nullptr, int = 3)
        : ops_(ops), log_(log), monitor_(*ops, log) {}
    ~bicgstabl() {
        if (prec_ && own_prec_) delete prec_;
    }

    void set_basis_size(int l) {
        if (l < 1 || l > kMaxBasis) throw std::logic_error("bicgstabl::set_basis_size: basis size out of range");
        l_ = l;
    }
    int basis_size() const { return l_; }
    void set_use_precond_resid(bool on) { use_precond_resid_ = on; }
    void set_resid_recalc_freq(int f) { resid_recalc_freq_ = f; }
    void set_preconditioner(Preconditioner* p, bool own = false) {
        prec_ = p;
        own_prec_ = own;
    }
    Monitor& monitor() { return monitor_; }
    const Monitor& monitor() const { return monitor_; }
    int breakdown_flag() const { return flag_; }

    bool solve(const LinearOperator& A, const vector_type& b, vector_type& x) const {
        if (!use_precond_resid_ && prec_)
            throw std::logic_error("bicgstabl::solve: unpreconditioned residual with a preconditioner is not supported");
        if (prec_) prec_->set_operator(&A);
        const int L = l_;
        vector_pool<VectorOperations> pool(ops_, 2 * (L + 1) + 1);
        vector_type* r = &pool[0];      // r[0..L]
        vector_type* u = &pool[L + 1];  // u[0..L]
        vector_type& rt = pool[2 * L + 2];

        if (prec_ && use_precond_resid_) {
            ops_->assign(b, r[0]);
            prec_->apply(r[0]);
            monitor_.start(r[0]);
        } else {
            monitor_.start(b);
        }
        ops_->assign_scalar(T(0), u[0]);
        residual(A, x, b, r[0]);
        ops_->assign(r[0], rt);
        ops_->assign_mul(T(1) / T(ops_->norm(rt)), rt, rt);

        std::vector<T> sigma(L + 1), gam(L + 1), gam1(L + 1), gam2(L + 1);
        std::vector<std::vector<T> > tau(L + 1, std::vector<T>(L + 1));
        T rho = T(1), alpha = T(0), omega = T(1);
        flag_ = 1;
        while (!monitor_.check_finished(x, r[0])) {
            rho = -omega * rho;
            // ---- BiCG part
            for (int j = 0; j < L; ++j) {
                if (rho == T(0)) {
                    flag_ = -1;
                    break;
                }
                T rho1 = ops_->scalar_prod(rt, r[j]);
                T beta = alpha * rho1 / rho;
                rho = rho1;
                for (int i = 0; i <= j; ++i) ops_->add_mul(T(1), r[i], -beta, u[i]);  // u_i = r_i - beta u_i
                A.apply(u[j], u[j + 1]);
                if (prec_) prec_->apply(u[j + 1]);
                alpha = rho / ops_->scalar_prod(rt, u[j + 1]);
                for (int i = 0; i <= j; ++i) ops_->add_mul(-alpha, u[i + 1], T(1), r[i]);  // r_i -= alpha u_{i+1}
                A.apply(r[j], r[j + 1]);
                if (prec_) prec_->apply(r[j + 1]);
                ops_->add_mul(alpha, u[0], T(1), x);
            }
            if (flag_ < 0) break;
            // ---- MR part: modified Gram-Schmidt on r_1..r_L
            for (int j = 1; j <= L; ++j) {
                for (int i = 1; i < j; ++i) {
                    tau[i][j] = ops_->scalar_prod(r[i], r[j]) / sigma[i];
                    ops_->add_mul(-tau[i][j], r[i], T(1), r[j]);
                }
                sigma[j] = ops_->scalar_prod(r[j], r[j]);
                gam1[j] = ops_->scalar_prod(r[j], r[0]) / sigma[j];
            }
            gam[L] = gam1[L];
            omega = gam[L];
            for (int j = L - 1; j >= 1; --j) {
                T g = gam1[j];
                for (int i = j + 1; i <= L; ++i) g -= tau[j][i] * gam[i];
                gam[j] = g;
            }
            for (int j = 1; j < L; ++j) {
                T g = gam[j + 1];
                for (int i = j + 1; i < L; ++i) g += tau[j][i] * gam[i + 1];
                gam2[j] = g;
            }
            ops_->add_mul(gam[1], r[0], T(1), x);
            ops_->add_mul(-gam1[L], r[L], T(1), r[0]);
            ops_->add_mul(-gam[L], u[L], T(1), u[0]);
            for (int j = 1; j < L; ++j) {
                ops_->add_mul(gam2[j], r[j], T(1), x);
                ops_->add_mul(-gam1[j], r[j], T(1), r[0]);
                ops_->add_mul(-gam[j], u[j], T(1), u[0]);
            }
            const bool recalc = resid_recalc_freq_ > 0 &&
                                ((monitor_.iters_performed() / L + 1) % resid_recalc_freq_ == 0);
            if (recalc) residual(A, x, b, r[0]);
            monitor_ += L;
        }
        const bool ok = monitor_.converged();
        if (!ok && log_) log_->error_f("bicgstabl::solve: linear solver failed to converge");
        return ok;
    }

private:
    static constexpr int kMaxBasis = 30;
    void residual(const LinearOperator& A, const vector_type& x, const vector_type& b, vector_type& r) const {
        A.apply(x, r);
        ops_->add_mul(T(1), b, -T(1), r);  // r = b - A x
        if (prec_) prec_->apply(r);
    }

    const VectorOperations* ops_;
    Log* log_;
    mutable Monitor monitor_;
    Preconditioner* prec_ = nullptr;
    bool own_prec_ = false;
    int l_ = 2;
    bool use_precond_resid_ = true;
    int resid_recalc_freq_ = 0;
    mutable int flag_ = 1;
};

}  // namespace solvers
}  // namespace hpb

#endif
