// Cross-rank merge of compensated reductions over a vector sharded in
// contiguous slices, one slice per GPU (one process per GPU).
//
// Each rank reduces its own slice with the single-GPU kernels (hpb_dot2_*,
// hpb_sum2_*, hpb_asum2_*, hpb_nrm2_* sums of squares), which leave one
// (hi, lo) result in device memory.  The ranks exchange those results with
// an all-gather (NCCL over NVLink / NVSwitch in
// high_precision_blas1_b200/sharded.py: 16 or 32 bytes per rank) and every
// rank merges the gathered results in rank order with hpb_shard_merge, so
// every rank holds the same bits whatever order the ranks finished in.  An
// all-reduce(sum) is not used: it would drop lo and its summation order is
// not specified.
//
// The merge is the recurrence the reference applies to (value, error)
// partials in a compensated pass (common/ogita/gpu_reduction_ogita_impl.cuh:
// 274-276: main_sum = TwoSum(main_sum, partial), error_sum += error_local +
// err_data): per real component, s = c = 0; for k in rank order
// s = TwoSum(s, hi_k, t), c = c + (t + lo_k); then (hi, lo) = TwoSum(s, c),
// the same normalisation as the single-GPU result (hi the rounded value, lo
// its error).  One result merges to itself bit for bit.
//
// hpb_shard_merge runs it in one device thread (stream-ordered on the
// context's stream, no host synchronisation); hpb_shard_merge_cpu runs the
// same additions on the host (round-to-nearest binary64 additions only, no
// contraction), for callers that gather the results to host memory.
#include "hpb_common.cuh"

namespace hpb {
namespace {

// TwoSum from additions that neither compiler contracts or reorders
// (device: explicit round-to-nearest intrinsics; host: IEEE binary64
// additions, which x86-64 and AArch64 compilers evaluate as written).
__host__ __device__ __forceinline__ double hd_add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ double hd_sub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ double hd_two_sum(double a, double b, double& e) {
    const double s = hd_add(a, b);
    const double bv = hd_sub(s, a);
    const double av = hd_sub(s, bv);
    e = hd_add(hd_sub(b, bv), hd_sub(a, av));
    return s;
}

// parts: count results of `comps` real components each, laid out as the
// reductions write them (real: hi, lo; complex: hi.re, hi.im, lo.re, lo.im)
__host__ __device__ __forceinline__ void merge_results(int count, int comps, const double* parts, double* out) {
    const int stride = 2 * comps;
    for (int q = 0; q < comps; ++q) {
        double s = 0.0, c = 0.0;
        for (int k = 0; k < count; ++k) {
            double t;
            s = hd_two_sum(s, parts[k * stride + q], t);
            c = hd_add(c, hd_add(t, parts[k * stride + comps + q]));
        }
        double lo;
        const double hi = hd_two_sum(s, c, lo);
        out[q] = hi;
        out[comps + q] = lo;
    }
}

__global__ void k_shard_merge(int count, int comps, const double* __restrict__ parts, double* __restrict__ out) {
    if (blockIdx.x == 0 && threadIdx.x == 0) merge_results(count, comps, parts, out);
}

}  // namespace
}  // namespace hpb

extern "C" {

int hpb_shard_merge(hpb_context* ctx, int count, int is_complex, const double* parts, double* out) {
    HPB_CHECK_CTX(ctx);
    if (count < 1 || parts == nullptr || out == nullptr)
        return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_shard_merge: count < 1 or null pointer");
    if ((reinterpret_cast<uintptr_t>(parts) | reinterpret_cast<uintptr_t>(out)) % 8)
        return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_shard_merge: pointer not aligned to double");
    const int comps = is_complex ? 2 : 1;
    hpb::k_shard_merge<<<1, 32, 0, ctx->stream>>>(count, comps, parts, out);
    hpb::count_launch();
    return hpb::check_launch(ctx, "hpb_shard_merge");
}

int hpb_shard_merge_cpu(int count, int is_complex, const double* parts, double* out) {
    if (count < 1 || parts == nullptr || out == nullptr) return HPB_ERROR_INVALID_VALUE;
    hpb::merge_results(count, is_complex ? 2 : 1, parts, out);
    return HPB_SUCCESS;
}

}  // extern "C"
