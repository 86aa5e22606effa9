// Drop-in replacement of the reference's common/csr/gpu_ilu0_preconditioner.h.
//
// Same interface (gpu_ilu0_preconditioner.h:32-80): constructed from the
// vector operations, set_operator, set_matrix(const Matrix) taking a copy of
// the matrix, in-place apply.  The reference's version keeps the copy but
// computes no factors (its apply only copies x into a work vector, i.e. it
// is the identity); here set_matrix factors the copy with ILU(0) on A's
// pattern (csr::gpu_matrix::ilu0, the library's level-scheduled kernel) and
// apply is x := U^-1 L^-1 x with the library's sparse triangular solves.
#ifndef __CSR__GPU_ILU0_PRECONDITIONER_H__
#define __CSR__GPU_ILU0_PRECONDITIONER_H__

#include <memory>
#include <stdexcept>

namespace csr {

template <class VectorOperations, class LinearOperator, class Matrix>
struct gpu_ilu0_preconditioner {
    using T = typename VectorOperations::scalar_type;
    using T_vec = typename VectorOperations::vector_type;

    explicit gpu_ilu0_preconditioner(const VectorOperations* vec_ops_) : vec_ops(vec_ops_) {
        vec_ops->init_vector(y);
        vec_ops->start_use_vector(y);
    }
    ~gpu_ilu0_preconditioner() {
        vec_ops->stop_use_vector(y);
        vec_ops->free_vector(y);
    }
    gpu_ilu0_preconditioner(const gpu_ilu0_preconditioner&) = delete;
    gpu_ilu0_preconditioner& operator=(const gpu_ilu0_preconditioner&) = delete;

    void set_operator(const LinearOperator* lin_op_) {
        lin_op = lin_op_;
        operator_set = true;
    }
    // Copy the matrix and replace the copy's values by its ILU(0) factors
    // (throws on a missing diagonal or a zero pivot).
    void set_matrix(const Matrix& matP_) {
        std::unique_ptr<Matrix> m(new Matrix(matP_));
        m->ilu0();
        mat = std::move(m);
    }
    void apply(T_vec& x) const {
        if (!mat) return;  // no matrix set: the identity, as the reference
        mat->triangular_solve_lower(x, y);
        mat->triangular_solve_upper(y, x);
    }
    const Matrix* factors() const { return mat.get(); }

private:
    mutable T_vec y = nullptr;
    bool operator_set = false;
    const VectorOperations* vec_ops;
    const LinearOperator* lin_op = nullptr;
    std::unique_ptr<Matrix> mat;
};

}  // namespace csr

#endif
