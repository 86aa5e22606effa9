// RAII set of work vectors taken from a VectorOperations object
// (init_vector + start_use_vector on entry, stop_use_vector + free_vector on
// exit), the role of the reference's vectors_arr_wrap_static
// (numerical_algos/detail/vectors_arr_wrap_static.h:53-189).
#ifndef HPBLAS1_SOLVERS_VECTOR_POOL_H
#define HPBLAS1_SOLVERS_VECTOR_POOL_H

#include <vector>

namespace hpb {
namespace solvers {

template <class VectorOperations>
class vector_pool {
public:
    using vector_type = typename VectorOperations::vector_type;
    vector_pool(const VectorOperations* ops, int count) : ops_(ops), v_(count) {
        try {
            for (auto& x : v_) {
                ops_->init_vector(x);
                ops_->start_use_vector(x);
            }
        } catch (...) {
            release();
            throw;
        }
    }
    ~vector_pool() { release(); }
    vector_pool(const vector_pool&) = delete;
    vector_pool& operator=(const vector_pool&) = delete;
    vector_type& operator[](int i) { return v_[i]; }
    int size() const { return int(v_.size()); }

private:
    void release() {
        for (auto& x : v_) {
            ops_->stop_use_vector(x);
            ops_->free_vector(x);
            x = vector_type();
        }
    }
    const VectorOperations* ops_;
    std::vector<vector_type> v_;
};

}  // namespace solvers
}  // namespace hpb

#endif
