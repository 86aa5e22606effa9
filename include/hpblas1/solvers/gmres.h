// Restarted GMRES(m) over the VectorOperations concept.
//
// Interface of the reference's numerical_algos::lin_solvers::gmres
// (numerical_algos/lin_solvers/gmres.h:65-495): set_restarts (the basis
// size m), set_reorthogonalization, set_use_precond_resid,
// set_preconditioner, monitor(), solve(A, b, x); left preconditioning; a
// cycle of m Arnoldi steps with modified Gram-Schmidt, Givens rotations on
// the Hessenberg matrix, a triangular solve, x += V s, then the true
// (preconditioned) residual and one monitor test per cycle; the iteration
// counter advances once per Arnoldi step.
//
// Differences, all deliberate: the Givens rotation is the complex one
// (conjugates where the reference's conj_ is the identity, gmres.h:219-223,
// which makes its complex GMRES wrong); a happy breakdown (zero new basis
// vector) ends the cycle instead of dividing by zero; with
// set_early_exit(true) a cycle also ends as soon as the rotated residual
// estimate |s_{i+1}| meets the monitor's tolerance (off by default, so the
// iteration counts match the reference's fixed-length cycles).
// The Hessenberg matrix and rotations live on the host in binary64
// (complex<double> for complex data) whatever T is.
#ifndef HPBLAS1_SOLVERS_GMRES_H
#define HPBLAS1_SOLVERS_GMRES_H

#include <cmath>
#include <stdexcept>
#include <vector>

#include <thrust/complex.h>

#include "monitor.h"
#include "vector_pool.h"

namespace hpb {
namespace solvers {

template <class T> struct wide_scalar { using type = double; };
template <class R> struct wide_scalar<thrust::complex<R> > { using type = thrust::complex<double>; };

template <class LinearOperator, class Preconditioner, class VectorOperations, class Monitor, class Log = null_log,
          unsigned MaxBasis = 300>
class gmres {
public:
    using scalar_type = typename VectorOperations::scalar_type;
    using vector_type = typename VectorOperations::vector_type;
    using T = scalar_type;
    using W = typename wide_scalar<T>::type;

    explicit gmres(const VectorOperations* ops, Log* log = nullptr, int = 3) : ops_(ops), log_(log), monitor_(*ops, log) {}
    ~gmres() {
        if (prec_ && own_prec_) delete prec_;
    }

    void set_restarts(unsigned m) {
        if (m < 1 || m >= MaxBasis) throw std::logic_error("gmres::set_restarts: basis size out of range");
        m_ = int(m);
    }
    void set_reorthogonalization(bool on) { reorth_ = on; }
    void set_use_precond_resid(bool on) { use_precond_resid_ = on; }
    void set_resid_recalc_freq(int) {}
    void set_early_exit(bool on) { early_exit_ = on; }
    void set_preconditioner(Preconditioner* p, bool own = false) {
        prec_ = p;
        own_prec_ = own;
    }
    Monitor& monitor() { return monitor_; }
    const Monitor& monitor() const { return monitor_; }

    bool solve(const LinearOperator& A, const vector_type& b, vector_type& x) const {
        if (!use_precond_resid_ && prec_)
            throw std::logic_error("gmres::solve: unpreconditioned residual with a preconditioner is not supported");
        if (prec_) prec_->set_operator(&A);
        const int m = m_;
        vector_pool<VectorOperations> pool(ops_, m + 2);
        vector_type* V = &pool[0];  // V[0..m]
        vector_type& r = pool[m + 1];
        std::vector<W> H(size_t(m + 1) * m), s(m + 1), cs(m), sn(m);
        auto h = [&](int row, int col) -> W& { return H[size_t(row) * m + col]; };

        if (prec_ && use_precond_resid_) {
            ops_->assign(b, r);
            prec_->apply(r);
            monitor_.start(r);
        } else {
            monitor_.start(b);
        }
        residual(A, x, b, r);
        if (!monitor_.check_finished(x, r)) {
            do {
                const double beta = double(ops_->norm(r));
                ops_->assign_mul(T(1.0 / beta), r, V[0]);
                std::fill(s.begin(), s.end(), W(0));
                std::fill(H.begin(), H.end(), W(0));
                s[0] = W(beta);
                int i = -1;
                bool stop = false;
                while (!stop && i + 1 < m) {
                    ++i;
                    ++monitor_;
                    A.apply(V[i], V[i + 1]);
                    if (prec_) prec_->apply(V[i + 1]);
                    for (int k = 0; k <= i; ++k) {  // modified Gram-Schmidt
                        T a = ops_->scalar_prod(V[k], V[i + 1]);
                        ops_->add_mul(-a, V[k], V[i + 1]);
                        W aw = W(a);
                        if (reorth_) {
                            T c = ops_->scalar_prod(V[k], V[i + 1]);
                            ops_->add_mul(-c, V[k], V[i + 1]);
                            aw += W(c);
                        }
                        h(k, i) = aw;
                    }
                    const double hn = double(ops_->norm(V[i + 1]));
                    h(i + 1, i) = W(hn);
                    if (hn > 0.0) ops_->assign_mul(T(1.0 / hn), V[i + 1], V[i + 1]);
                    for (int k = 0; k < i; ++k) rotate(h(k, i), h(k + 1, i), cs[k], sn[k]);
                    make_rotation(h(i, i), h(i + 1, i), cs[i], sn[i]);
                    rotate(h(i, i), h(i + 1, i), cs[i], sn[i]);
                    h(i + 1, i) = W(0);
                    rotate(s[i], s[i + 1], cs[i], sn[i]);
                    if (hn == 0.0) stop = true;  // happy breakdown: the Krylov space is invariant
                    if (early_exit_ && absw(s[i + 1]) <= double(monitor_.tol())) stop = true;
                }
                // back substitution H(0:i,0:i) y = s(0:i), then x += V y
                for (int j = i; j >= 0; --j) {
                    s[j] /= h(j, j);
                    for (int k = j - 1; k >= 0; --k) s[k] -= h(k, j) * s[j];
                }
                for (int j = 0; j <= i; ++j) ops_->add_mul(narrow(s[j]), V[j], x);
                residual(A, x, b, r);
            } while (!monitor_.check_finished(x, r));
        }
        const bool ok = monitor_.converged();
        if (!ok && log_) log_->error_f("gmres::solve: linear solver failed to converge");
        return ok;
    }

private:
    static T narrow(const W& w) { return T(w); }
    static double absw(double v) { return std::fabs(v); }
    static double absw(const thrust::complex<double>& v) { return thrust::abs(v); }

    // real: the textbook rotation with the larger of |dx|, |dy| as pivot
    static void make_rotation(double dx, double dy, double& c, double& sgn) {
        if (dy == 0.0) {
            c = 1.0;
            sgn = 0.0;
        } else if (std::fabs(dy) > std::fabs(dx)) {
            double t = dx / dy;
            sgn = 1.0 / std::sqrt(1.0 + t * t);
            c = t * sgn;
        } else {
            double t = dy / dx;
            c = 1.0 / std::sqrt(1.0 + t * t);
            sgn = t * c;
        }
    }
    static void rotate(double& dx, double& dy, double c, double sgn) {
        double t = c * dx + sgn * dy;
        dy = -sgn * dx + c * dy;
        dx = t;
    }
    // complex: c real >= 0, s complex, [c s; -conj(s) c] zeroes dy
    using CD = thrust::complex<double>;
    static void make_rotation(const CD& dx, const CD& dy, CD& c, CD& sgn) {
        const double ax = thrust::abs(dx), ay = thrust::abs(dy);
        if (ay == 0.0) {
            c = 1.0;
            sgn = 0.0;
        } else if (ax == 0.0) {
            c = 0.0;
            sgn = thrust::conj(dy) / ay;
        } else {
            const double nr = std::hypot(ax, ay);
            c = ax / nr;
            sgn = (dx / ax) * thrust::conj(dy) / nr;
        }
    }
    static void rotate(CD& dx, CD& dy, const CD& c, const CD& sgn) {
        CD t = c * dx + sgn * dy;
        dy = -thrust::conj(sgn) * dx + c * dy;
        dx = t;
    }

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
    int m_ = 2;
    bool reorth_ = false, use_precond_resid_ = true, early_exit_ = false;
};

}  // namespace solvers
}  // namespace hpb

#endif
