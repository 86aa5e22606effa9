// Drop-in stand-in for the reference's external_libraries/cublas_wrap.h.
//
// The reference passes a cublas_wrap* to gpu_vector_operations and
// csr::gpu_matrix (common/gpu_vector_operations.h:98, csr/gpu_matrix.h:98);
// the drop-in runs every operation in libhpblas1, so this type only keeps
// that source compatible: constructing it creates no cuBLAS handle and
// nothing dispatches through it.
#ifndef __CUBLAS_WRAP_H__
#define __CUBLAS_WRAP_H__

class cublas_wrap {
public:
    explicit cublas_wrap(bool plot_info = false) : plot_info_(plot_info) {}
    cublas_wrap(const cublas_wrap&) = delete;
    cublas_wrap& operator=(const cublas_wrap&) = delete;
    bool plot_info() const { return plot_info_; }
    // the reference toggles cuBLAS host/device pointer mode; results of the
    // drop-in always come back by value, so the setting is recorded only
    void set_pointer_location_device(bool on) { device_pointers_ = on; }
    bool pointer_location_device() const { return device_pointers_; }

private:
    bool plot_info_;
    bool device_pointers_ = false;
};

#endif
