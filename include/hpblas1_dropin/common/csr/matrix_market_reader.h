// Drop-in replacement of the reference's common/csr/matrix_market_reader.h.
//
// csr::matrix_market_reader<T, Ord> keeps the reference's interface
// (matrix_market_reader.h:48-460): read_file, read_file_2_csr_marix (the
// reference's spelling), set_csr_matrix(Matrix*) (init + set_dim + set of a
// csr::gpu_matrix), get_matrix_dim, allocate_set_csr_pointers (malloc'd
// host arrays the caller frees), and its errors (runtime_error on a bad
// file, on a complex file read into a real T, on use before read_file).
// Parsing and the COO -> CSR conversion run in libhpblas1 (hpb_mm_read_csr):
// same accepted files and the same CSR as the reference (stable (row,
// column) order, duplicates kept, symmetric files mirrored).
#ifndef __CSR__MATRIX_MARKET_READER_H__
#define __CSR__MATRIX_MARKET_READER_H__

#include <cstdlib>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include <hpblas1.h>

#include <common/csr/matrix_market_reader_set_val.h>

namespace csr {

template <class T, class Ord = int>
class matrix_market_reader {
public:
    explicit matrix_market_reader(bool verbose_ = false) : verbose(verbose_) {}
    ~matrix_market_reader() = default;
    matrix_market_reader(const matrix_market_reader&) = delete;
    matrix_market_reader& operator=(const matrix_market_reader&) = delete;

    template <class Matrix>
    void read_file_2_csr_marix(const std::string& file_name_, Matrix* mat_) {
        read_file(file_name_);
        set_csr_matrix(mat_);
    }

    template <class Matrix>
    void set_csr_matrix(Matrix* mat_) {
        if (!matrix_file_read)
            throw std::runtime_error(
                "csr::matrix_market_reader::set_csr_matrix: one must read a file before setting a matrix. Call "
                "'read_file' before or 'read_file_2_csr_marix' ");
        mat_->init(nnz, nnz, num_rows + 1);
        mat_->set_dim(num_cols, num_rows);
        mat_->set(data.data(), col.data(), row.data());
    }

    void get_matrix_dim(Ord& size_rows_, Ord& size_cols_) {
        if (!matrix_file_read)
            throw std::runtime_error(
                "csr::matrix_market_reader::get_matrix_dim: one must read a file before. Call 'read_file' before ");
        size_rows_ = num_rows;
        size_cols_ = num_cols;
    }

    // row_p_ = rows + 1, col_i_ = nnz_ = number of stored entries; the three
    // arrays are malloc'd here and belong to the caller (free()).
    void allocate_set_csr_pointers(Ord& row_p_, Ord& col_i_, Ord& nnz_, Ord*& row_data_, Ord*& col_data_,
                                   T*& values_data_) {
        if (row_data_ != nullptr || col_data_ != nullptr || values_data_ != nullptr)
            throw std::runtime_error(
                "csr::matrix_market_reader::allocate_set_csr_pointers: pointers must be 'nullptr' i.e. not set "
                "before this call ");
        if (!matrix_file_read)
            throw std::runtime_error(
                "csr::matrix_market_reader::allocate_set_csr_pointers: one must read a file before setting pinters. "
                "Call 'read_file' before ");
        row_p_ = num_rows + 1;
        col_i_ = nnz;
        nnz_ = nnz;
        row_data_ = static_cast<Ord*>(std::malloc(sizeof(Ord) * size_t(row_p_)));
        col_data_ = static_cast<Ord*>(std::malloc(sizeof(Ord) * size_t(col_i_ > 0 ? col_i_ : 1)));
        values_data_ = static_cast<T*>(std::malloc(sizeof(T) * size_t(nnz_ > 0 ? nnz_ : 1)));
        if (row_data_ == nullptr || col_data_ == nullptr || values_data_ == nullptr) {
            std::free(row_data_);
            std::free(col_data_);
            std::free(values_data_);
            row_data_ = col_data_ = nullptr;
            values_data_ = nullptr;
            throw std::runtime_error("csr::matrix_market_reader::allocate_set_csr_pointers: failed to allocate memory ");
        }
        for (Ord j = 0; j < row_p_; ++j) row_data_[j] = row[size_t(j)];
        for (Ord j = 0; j < nnz_; ++j) {
            col_data_[j] = col[size_t(j)];
            values_data_[j] = data[size_t(j)];
        }
    }

    void read_file(const std::string& file_name_) {
        hpb_mm_csr m{};
        const int st = hpb_mm_read_csr(file_name_.c_str(), &m);
        if (st != HPB_SUCCESS)
            throw std::runtime_error(std::string("csr::matrix_market_reader::read_file: ") + hpb_mm_last_error());
        using R = typename complex_base_type<T>::real;
        if (std::is_same<T, R>::value && m.is_complex) {
            hpb_mm_free(&m);
            throw std::runtime_error(
                "csr::matrix_market_reader::read_file: real data type used for a complex matrix. This will be fixed "
                "later.");
        }
        num_rows = Ord(m.rows);
        num_cols = Ord(m.cols);
        nnz = Ord(m.nnz);
        row.assign(m.row_ptr, m.row_ptr + m.rows + 1);
        col.assign(m.col_ind, m.col_ind + m.nnz);
        data.resize(size_t(m.nnz));
        for (int64_t k = 0; k < m.nnz; ++k)
            set_val(data[size_t(k)], m.is_complex ? m.val[2 * k] : m.val[k], m.is_complex ? m.val[2 * k + 1] : 0.0);
        hpb_mm_free(&m);
        matrix_file_read = true;
    }

private:
    bool matrix_file_read = false;
    bool verbose = false;
    Ord num_rows = 0, num_cols = 0, nnz = 0;
    std::vector<Ord> row, col;
    std::vector<T> data;
};

}  // namespace csr

#endif
