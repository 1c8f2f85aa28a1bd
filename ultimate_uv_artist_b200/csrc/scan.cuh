// Exclusive prefix sums over int32 / int64 counts on one stream: a block
// scan per 1024 elements, one block over the block totals, then the carry.
// Header-only (static kernels: one copy per translation unit).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace uva {

static constexpr int kScanThreads = 1024;

template <typename T>
static __device__ __forceinline__ T block_inclusive_scan(T x, T* s) {
    s[threadIdx.x] = x;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {
        const T y = threadIdx.x >= o ? s[threadIdx.x - o] : T(0);
        __syncthreads();
        s[threadIdx.x] += y;
        __syncthreads();
    }
    return s[threadIdx.x];
}

template <typename T>
static __global__ void __launch_bounds__(kScanThreads) k_xscan_local(const T* in, T* out, T* sums, int64_t n) {
    __shared__ T s[kScanThreads];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kScanThreads + threadIdx.x;
    const T x = i < n ? in[i] : T(0);
    const T inc = block_inclusive_scan(x, s);
    if (i < n) out[i] = inc - x;
    if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = inc;
}

template <typename T>
static __global__ void __launch_bounds__(kScanThreads) k_xscan_sums(T* sums, int64_t nb, T* total) {
    __shared__ T s[kScanThreads];
    __shared__ T carry;
    if (threadIdx.x == 0) carry = T(0);
    __syncthreads();
    for (int64_t base = 0; base < nb; base += kScanThreads) {
        const int64_t i = base + threadIdx.x;
        const T x = i < nb ? sums[i] : T(0);
        const T inc = block_inclusive_scan(x, s);
        if (i < nb) sums[i] = carry + inc - x;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry += inc;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <typename T>
static __global__ void __launch_bounds__(kScanThreads) k_xscan_add(T* out, const T* sums, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kScanThreads + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

// Scratch of xscan: one T per 1024 inputs.
static inline int64_t xscan_sums(int64_t n) { return std::max<int64_t>(1, (n + kScanThreads - 1) / kScanThreads); }

// out[i] = in[0] + ... + in[i-1]; *total (device, may be null) = the sum of
// all n. in and out may alias.
template <typename T>
static void xscan(const T* in, T* out, T* sums, T* total, int64_t n, cudaStream_t s) {
    const int64_t nb = xscan_sums(n);
    k_xscan_local<T><<<static_cast<unsigned>(nb), kScanThreads, 0, s>>>(in, out, sums, n);
    k_xscan_sums<T><<<1, kScanThreads, 0, s>>>(sums, nb, total);
    k_xscan_add<T><<<static_cast<unsigned>(nb), kScanThreads, 0, s>>>(out, sums, n);
}

}  // namespace uva
