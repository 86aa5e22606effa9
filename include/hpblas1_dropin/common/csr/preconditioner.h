// Drop-in replacement of the reference's common/csr/preconditioner.h.
//
// csr::preconditioner keeps the reference's interface (set_operator,
// set_matrix(L, U), in-place apply) (csr/preconditioner.h:32-85).  With no
// factors set, apply is the identity, as in the reference; with factors,
// apply is x := U^-1 L^-1 x by the same two calls the reference makes
// (triangular_solve_lower with a unit diagonal into a work vector, then
// triangular_solve_upper back into x), here on the library's sparse
// triangular-solve kernel instead of csrsv2.  L and U may be the same
// matrix holding both factors (the layout csr::gpu_matrix::ilu0 produces).
//
// csr::jacobi_preconditioner is the diagonal scaling x := D^{-1} x of A,
// the GPU analogue of the reference's constant-diagonal prec_operator for
// its 1-D operator (linear_operator.hpp:59-91); it is the baseline the
// learned preconditioner is compared against.
#ifndef __CSR__PRECONDITIONER_H__
#define __CSR__PRECONDITIONER_H__

#include <stdexcept>

namespace csr {

template <class VectorOperations, class LinearOperator, class Matrix>
struct preconditioner {
    using T = typename VectorOperations::scalar_type;
    using T_vec = typename VectorOperations::vector_type;

    explicit preconditioner(const VectorOperations* vec_ops_) : vec_ops(vec_ops_) {
        vec_ops->init_vector(y);
        vec_ops->start_use_vector(y);
    }
    ~preconditioner() {
        vec_ops->stop_use_vector(y);
        vec_ops->free_vector(y);
    }
    preconditioner(const preconditioner&) = delete;
    preconditioner& operator=(const preconditioner&) = delete;
    void set_operator(const LinearOperator* lin_op_) {
        lin_op = lin_op_;
        operator_set = true;
    }
    void set_matrix(const Matrix* matL_, const Matrix* matU_) {
        matL = matL_;
        matU = matU_;
        matrix_set = true;
    }
    void apply(T_vec& x) const {
        if (!matrix_set) return;
        matL->triangular_solve_lower(x, y);
        matU->triangular_solve_upper(y, x);
    }

private:
    mutable T_vec y = nullptr;
    bool operator_set = false;
    bool matrix_set = false;
    const VectorOperations* vec_ops;
    const LinearOperator* lin_op = nullptr;
    const Matrix* matL = nullptr;
    const Matrix* matU = nullptr;
};

template <class VectorOperations, class LinearOperator, class Matrix>
struct jacobi_preconditioner {
    using T = typename VectorOperations::scalar_type;
    using T_vec = typename VectorOperations::vector_type;

    explicit jacobi_preconditioner(const VectorOperations* vec_ops_) : vec_ops(vec_ops_) {
        vec_ops->init_vector(dinv);
        vec_ops->start_use_vector(dinv);
    }
    ~jacobi_preconditioner() {
        vec_ops->stop_use_vector(dinv);
        vec_ops->free_vector(dinv);
    }
    jacobi_preconditioner(const jacobi_preconditioner&) = delete;
    jacobi_preconditioner& operator=(const jacobi_preconditioner&) = delete;
    // the solvers call this with their operator; the diagonal comes from the
    // matrix given to set_matrix
    void set_operator(const LinearOperator*) {}
    void set_matrix(const Matrix* m) {
        m->diagonal(dinv);  // d := diag(A)
    }
    void apply(T_vec& x) const { vec_ops->div_pointwise(x, T(1.0), dinv); }

private:
    const VectorOperations* vec_ops;
    mutable T_vec dinv = nullptr;
};

}  // namespace csr

#endif
