// Shared device/host helpers of the sm_100a BM3D library.
#pragma once

#include <type_traits>

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace nssb {

// A failed CUDA call; the C ABI turns it into NSSB_ERR_CUDA with this text
// (the reference's CudaError, src/cuda/runtime/error.hpp:14-47).
struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        throw CudaError(std::string("nss_cuda: ") + what + " failed: " + cudaGetErrorString(e) + " (" + file + ":" +
                        std::to_string(line) + ")");
    }
}
#define NSSB_CUDA(call) ::nssb::cuda_check((call), #call, __FILE__, __LINE__)

// Fixed-point scale of the aggregation sums: num and the per-origin weights
// are int64 multiples of 2^-32, so the sums do not depend on the order in
// which groups land (deterministic in any launch shape or batch mix). All of
// it is FP32 and integer arithmetic: a sample w * v is rounded once in FP32,
// scaled by 2^32 (exact: a power of two) and rounded to the nearest integer.
constexpr float kFixedScale = 4294967296.f;
constexpr float kFixedInv = 1.f / 4294967296.f;

#ifdef __CUDACC__
__device__ __forceinline__ long long to_fixed(float x) { return __float2ll_rn(x * kFixedScale); }
// num / den of two fixed-point sums (the common 2^-32 cancels)
__device__ __forceinline__ float fixed_quotient(long long num, long long den) {
    return __fdiv_rn(__ll2float_rn(num), __ll2float_rn(den));
}
#endif

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ inline int grid_count(int extent, int block, int step) {
    return extent < block ? 0 : (extent - block + step - 1) / step + 1;
}
__host__ __device__ inline int grid_pos(int i, int extent, int block, int step) {
    const int p = i * step;
    return p < extent - block ? p : extent - block;
}

// Packed match position: y in the high half, x in the low half.
__host__ __device__ inline int32_t pack_pos(int x, int y) { return static_cast<int32_t>((uint32_t(y) << 16) | uint32_t(x)); }
__host__ __device__ inline int pos_x(int32_t p) { return static_cast<int>(uint32_t(p) & 0xffffu); }
__host__ __device__ inline int pos_y(int32_t p) { return static_cast<int>(uint32_t(p) >> 16); }

// The SSD order of this build: one FMA chain per block column down the
// rows, then the columns added pairwise (halves first, recursively).
template <int N>
__device__ __forceinline__ float column_tree(const float* c) {
    if constexpr (N == 1) {
        return c[0];
    } else {
        return __fadd_rn(column_tree<N / 2>(c), column_tree<N - N / 2>(c + N / 2));
    }
}

#ifdef __CUDACC__
// Compile-time integers and an unrolled loop over them (the matchers' row
// schedules: accumulator slots stay register names).
template <int N>
using IC = std::integral_constant<int, N>;
template <int N>
__device__ __forceinline__ IC<N> ic() { return {}; }
template <int B, int E, class F>
__device__ __forceinline__ void static_for(F&& f) {
    if constexpr (B < E) {
        f(IC<B>{});
        static_for<B + 1, E>(f);
    }
}
#endif

// Asynchronous 4-byte global -> shared copy (LDGSTS): a tile fill issues
// all its copies without waiting on any, then waits once. bytes = 0 writes
// zero and reads nothing (src must still be a valid address).
__device__ __forceinline__ void cp_async4(float* dst, const float* src, int bytes) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

}  // namespace nssb
