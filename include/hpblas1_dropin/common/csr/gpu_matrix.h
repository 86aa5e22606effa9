// Drop-in replacement of the reference's common/csr/gpu_matrix.h.
//
// csr::gpu_matrix<VectorOperations, CudaBlas, Ordinal> keeps the
// reference's constructors, init / set_dim / set / init_set / get_dim and
// axpy(alpha, x, beta, y, transpose) (csr/gpu_matrix.h:93-375 with the base
// class csr/matrix.h:33-158), but axpy runs the library's CSR kernel
// (hpb_csr_spmv_*) instead of cusparseSpMV with a cudaMalloc'd work buffer
// per call.
//
// Shape contract: the reference hands cuSPARSE size_row = rows+1 and
// size_col = nnz as the matrix dimensions (csr/gpu_matrix.h:389-396), an
// off-by-one.  Here the operator is rows x columns from set_dim(); without
// set_dim the matrix is taken square with rows = size_row - 1.
// Only 0-based int32 indices are supported (the configs' matrices).
// Triangular solves (triangular_solve_lower / _upper, csr/gpu_matrix.h:
// 142-311, there cuSPARSE csrsv2 with an analysis and a cudaMalloc'd buffer
// per call) run the library's level-scheduled kernel (hpb_csr_trsv_*); the
// analysis of each triangle is made on the first solve and kept until the
// matrix is set again or destroyed.  The transposed product and solves
// (transpose_ = true) run on A^T's pattern, built on the device once
// (hpb_csr_transpose_pattern) and kept like the analyses; A^T's values are
// gathered from A's on every transposed call, so in-place value changes are
// seen.
#ifndef __CSR__GPU_MATRIX_H__
#define __CSR__GPU_MATRIX_H__

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>

#include <common/gpu_vector_operations.h>

namespace csr {

template <class VectorOperations, class CudaBlas, class Ordinal = int>
class gpu_matrix {
    static_assert(std::is_same<Ordinal, int>::value || std::is_same<Ordinal, std::int32_t>::value,
                  "csr::gpu_matrix: the drop-in supports int32 indices");

public:
    using T = typename VectorOperations::scalar_type;
    using T_vec = typename VectorOperations::vector_type;
    using I = Ordinal;
    using I_vec = Ordinal*;
    struct dimensions_t {
        int columns = 0;
        int rows = 0;
    };

    explicit gpu_matrix(CudaBlas* cublas_ = nullptr) : cublas(cublas_) { ctx = hpb_dropin::make_context(); }
    gpu_matrix(int nnz_, int size_col_, int size_row_, CudaBlas* cublas_) : cublas(cublas_) {
        ctx = hpb_dropin::make_context();
        init(nnz_, size_col_, size_row_);
    }
    gpu_matrix(const gpu_matrix& m) : cublas(m.cublas), dim(m.dim) {
        ctx = hpb_dropin::make_context();
        if (m.initialized) {
            init(m.nnz, m.size_col, m.size_row);
            copy_d2d(data, m.data, size_t(nnz) * sizeof(T));
            copy_d2d(col_ind, m.col_ind, size_t(size_col) * sizeof(I));
            copy_d2d(row_ptr, m.row_ptr, size_t(size_row) * sizeof(I));
        }
    }
    gpu_matrix& operator=(const gpu_matrix&) = delete;
    ~gpu_matrix() {
        drop_analyses();
        if (owns_) {
            cudaFree(data);
            cudaFree(col_ind);
            cudaFree(row_ptr);
        }
        hpb_destroy(ctx);
    }

    void set_dim(int matrix_columns_, int matrix_rows_) {
        dim.columns = matrix_columns_;
        dim.rows = matrix_rows_;
    }
    // allocate nnz values, size_col column indices and size_row row pointers
    void init(int nnz_, int size_col_, int size_row_) {
        if (initialized) return;
        if (nnz_ < 0 || size_col_ < 0 || size_row_ < 1) throw std::runtime_error("csr::gpu_matrix: invalid sizes");
        nnz = nnz_;
        size_col = size_col_;
        size_row = size_row_;
        data = static_cast<T*>(dalloc(size_t(nnz) * sizeof(T)));
        col_ind = static_cast<I*>(dalloc(size_t(size_col) * sizeof(I)));
        row_ptr = static_cast<I*>(dalloc(size_t(size_row) * sizeof(I)));
        initialized = true;
    }
    dimensions_t get_dim() const {
        dimensions_t d = dim;
        if (d.rows == 0 && initialized) {
            d.rows = size_row - 1;
            d.columns = d.rows;
        }
        return d;
    }
    // upload host arrays (values, column indices, row pointers)
    void set(const T_vec data_, const I_vec col_ind_, const I_vec row_ptr_) {
        if (!initialized) throw std::runtime_error("csr::gpu_matrix: trying to set an uninitialized matrix.");
        drop_analyses();
        h2d(data, data_, size_t(nnz) * sizeof(T));
        h2d(col_ind, col_ind_, size_t(size_col) * sizeof(I));
        h2d(row_ptr, row_ptr_, size_t(size_row) * sizeof(I));
    }
    void init_set(int nnz_, int size_col_, int size_row_, const T_vec data_, const I_vec col_ind_,
                  const I_vec row_ptr_, int matrix_columns_, int matrix_rows_) {
        init(nnz_, size_col_, size_row_);
        set_dim(matrix_columns_, matrix_rows_);
        set(data_, col_ind_, row_ptr_);
    }

    // y := alpha*op(A)*x + beta*y, op(A) = A or A^T
    void axpy(const T& alpha_, const T_vec& x_, const T& beta_, T_vec& y_, bool transpose_ = false) const {
        if (!initialized) throw std::runtime_error("csr::gpu_matrix::axpy: matrix not set");
        dimensions_t d = get_dim();
        using A = hpb_dropin::abi<T>;
        if (transpose_) {
            const Transposed& t = transposed();
            hpb_dropin::check(A::spmv(ctx, d.columns, d.rows, nnz, t.rp, t.ci, t.val, A::s(alpha_), x_, A::s(beta_),
                                      y_),
                              ctx, "csr::gpu_matrix::axpy");
            return;
        }
        hpb_dropin::check(A::spmv(ctx, d.rows, d.columns, nnz, row_ptr, col_ind, data, A::s(alpha_), x_, A::s(beta_),
                                  y_),
                          ctx, "csr::gpu_matrix::axpy");
    }
    // L x = alpha b, L the lower triangle with a unit diagonal (stored
    // diagonal and upper entries ignored), as the reference's csrsv2 call
    // with CUSPARSE_DIAG_TYPE_UNIT (csr/gpu_matrix.h:150-225).
    void triangular_solve_lower(const T_vec& b_, T_vec& x_, const T& alpha_ = T(1.0), bool transpose_ = false) const {
        tri_solve(false, true, b_, x_, alpha_, transpose_, "csr::gpu_matrix::triangular_solve_lower");
    }
    // U x = alpha b, U the upper triangle with its stored diagonal
    // (csr/gpu_matrix.h:236-311).
    void triangular_solve_upper(const T_vec& b_, T_vec& x_, const T& alpha_ = T(1.0), bool transpose_ = false) const {
        tri_solve(true, false, b_, x_, alpha_, transpose_, "csr::gpu_matrix::triangular_solve_upper");
    }

    // ------------------------------------------------------------ extensions
    // Use CSR arrays already resident on the device (not copied, not freed).
    void attach(int rows, int cols, int nnz_, const I* row_ptr_dev, const I* col_ind_dev, const T* val_dev) {
        if (initialized) throw std::runtime_error("csr::gpu_matrix::attach: matrix already initialised");
        nnz = nnz_;
        size_col = nnz_;
        size_row = rows + 1;
        data = const_cast<T*>(val_dev);
        col_ind = const_cast<I*>(col_ind_dev);
        row_ptr = const_cast<I*>(row_ptr_dev);
        set_dim(cols, rows);
        owns_ = false;
        initialized = true;
    }
    const T* values() const { return data; }
    const I* columns() const { return col_ind; }
    const I* row_pointers() const { return row_ptr; }
    int nonzeros() const { return nnz; }
    hpb_context* context() const { return ctx; }
    // diagonal of A into the device vector d (d_i = A_ii)
    void diagonal(T_vec& d) const {
        using A = hpb_dropin::abi<T>;
        hpb_dropin::check(A::diag(ctx, get_dim().rows, row_ptr, col_ind, data, d), ctx, "csr::gpu_matrix::diagonal");
    }
    // Replace the values by the ILU(0) factors on the same pattern (L unit
    // lower in the strictly lower entries, U upper with the diagonal), so
    // that triangular_solve_lower then triangular_solve_upper apply
    // (L U)^-1.  Every row must store its diagonal, the columns of each row
    // must be increasing; a zero pivot throws.  On an attached matrix the
    // caller's value array is overwritten.
    void ilu0() {
        if (!initialized) throw std::runtime_error("csr::gpu_matrix::ilu0: matrix not set");
        using A = hpb_dropin::abi<T>;
        hpb_dropin::check(A::ilu0(ctx, analysis(false), data), ctx, "csr::gpu_matrix::ilu0");
    }

protected:
    T_vec data = nullptr;
    I_vec col_ind = nullptr;
    I_vec row_ptr = nullptr;
    int size_row = 0, size_col = 0, nnz = 0;
    bool initialized = false;
    dimensions_t dim;

private:
    CudaBlas* cublas;
    hpb_context* ctx = nullptr;
    bool owns_ = true;
    mutable hpb_csr_tri* tri_[2] = {nullptr, nullptr};  // analyses of the lower / upper triangle
    struct Transposed {
        int32_t* rp = nullptr;    // pattern of A^T
        int32_t* ci = nullptr;
        int32_t* perm = nullptr;  // position in A of each entry of A^T
        T* val = nullptr;         // values of A^T, gathered per transposed call
        hpb_csr_tri* tri[2] = {nullptr, nullptr};
    };
    mutable Transposed tr_;

    void drop_analyses() {
        for (auto& t : tri_) {
            hpb_csr_tri_destroy(t);
            t = nullptr;
        }
        for (auto& t : tr_.tri) {
            hpb_csr_tri_destroy(t);
            t = nullptr;
        }
        cudaFree(tr_.rp);
        cudaFree(tr_.ci);
        cudaFree(tr_.perm);
        cudaFree(tr_.val);
        tr_.rp = tr_.ci = tr_.perm = nullptr;
        tr_.val = nullptr;
    }
    // A^T's pattern (built once) with A's current values gathered into it
    const Transposed& transposed() const {
        using A = hpb_dropin::abi<T>;
        dimensions_t d = get_dim();
        if (tr_.rp == nullptr) {
            tr_.rp = static_cast<int32_t*>(dalloc(size_t(d.columns + 1) * sizeof(int32_t)));
            tr_.ci = static_cast<int32_t*>(dalloc(size_t(nnz) * sizeof(int32_t)));
            tr_.perm = static_cast<int32_t*>(dalloc(size_t(nnz) * sizeof(int32_t)));
            tr_.val = static_cast<T*>(dalloc(size_t(nnz) * sizeof(T)));
            hpb_dropin::check(hpb_csr_transpose_pattern(ctx, d.rows, d.columns, nnz, row_ptr, col_ind, tr_.rp, tr_.ci,
                                                        tr_.perm),
                              ctx, "csr::gpu_matrix: transpose");
        }
        hpb_dropin::check(A::gather(ctx, nnz, tr_.perm, data, tr_.val), ctx, "csr::gpu_matrix: transpose");
        return tr_;
    }
    hpb_csr_tri* analysis(bool upper) const {
        hpb_csr_tri*& t = tri_[upper ? 1 : 0];
        if (t == nullptr)
            hpb_dropin::check(hpb_csr_tri_create(ctx, upper ? 1 : 0, get_dim().rows, nnz, row_ptr, col_ind, &t), ctx,
                              "csr::gpu_matrix: triangular analysis");
        return t;
    }
    void tri_solve(bool upper, bool unit, const T_vec& b_, T_vec& x_, const T& alpha_, bool transpose_,
                   const char* what) const {
        if (!initialized) throw std::runtime_error(std::string(what) + ": matrix not set");
        using A = hpb_dropin::abi<T>;
        hpb_csr_tri* t = nullptr;
        const T* vals = data;
        if (transpose_) {  // the transpose of a lower triangle is the upper triangle of A^T and vice versa
            const Transposed& tt = transposed();
            hpb_csr_tri*& slot = tr_.tri[upper ? 0 : 1];
            if (slot == nullptr)
                hpb_dropin::check(hpb_csr_tri_create(ctx, upper ? 0 : 1, get_dim().columns, nnz, tt.rp, tt.ci, &slot),
                                  ctx, "csr::gpu_matrix: triangular analysis");
            t = slot;
            vals = tt.val;
        } else {
            t = analysis(upper);
        }
        hpb_dropin::check(A::trsv(ctx, t, unit ? 1 : 0, vals, A::s(alpha_), b_, x_), ctx, what);
        // blocking, like the reference's call (its cudaFree of the work buffer
        // synchronises); also reports a solve whose bounded waits gave up
        hpb_dropin::check(hpb_csr_tri_check(ctx, t), ctx, what);
    }

    static void* dalloc(size_t b) {
        void* p = nullptr;
        if (cudaMalloc(&p, b ? b : 4) != cudaSuccess) throw std::runtime_error("csr::gpu_matrix: cudaMalloc failed");
        return p;
    }
    static void h2d(void* d, const void* h, size_t b) {
        if (b && cudaMemcpy(d, h, b, cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("csr::gpu_matrix: failed to set the gpu_matrix.");
    }
    static void copy_d2d(void* d, const void* s, size_t b) {
        if (b && cudaMemcpy(d, s, b, cudaMemcpyDeviceToDevice) != cudaSuccess)
            throw std::runtime_error("csr::gpu_matrix: copy failed");
    }
};

}  // namespace csr

#endif
