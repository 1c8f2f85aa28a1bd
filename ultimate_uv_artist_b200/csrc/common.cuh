// Shared device helpers for the uva_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/uva_b200.h"

extern "C" void uva_set_error(const char* msg);
int uva_cuda_status(cudaError_t e, const char* where);

#define UVA_CHECK_LAUNCH(where)                                        \
    do {                                                               \
        cudaError_t e_ = cudaGetLastError();                           \
        if (e_ != cudaSuccess) return uva_cuda_status(e_, where);      \
    } while (0)

namespace uva {

constexpr int kWarp = 32;

__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

__device__ __forceinline__ bool finite2(double2 v) { return isfinite(v.x) && isfinite(v.y); }

// SLIM local step of one 2x2 Jacobian J = [[j00, j01], [j10, j11]]
// (engine/param.py:234-255, mode 1): signed singular values s1 = Q + R,
// s2 = Q - R and first left singular vector at angle phi (closed form),
// weights w = sqrt((|s| - |s|^-3) / (|s| - 1)) (2 when |s| ~ 1, |s| clamped
// at 1e-8), W = U diag(w) U^T (symmetric: w00, w01, w11), and the closest
// rotation R = [[rc, -rs], [rs, rc]].
__device__ __forceinline__ double slim_weight(double s) {
    s = fmax(fabs(s), 1e-8);
    if (fabs(s - 1.0) < 1e-6) return 2.0;
    return sqrt(fmax((s - 1.0 / (s * s * s)) / (s - 1.0), 1e-12));
}

__device__ __forceinline__ void slim_2x2(double j00, double j01, double j10, double j11, double& rc, double& rs,
                                         double& w00, double& w01, double& w11) {
    const double E = 0.5 * (j00 + j11), F = 0.5 * (j00 - j11), G = 0.5 * (j10 + j01), H = 0.5 * (j10 - j01);
    const double Q = sqrt(E * E + H * H), R = sqrt(F * F + G * G);
    if (Q > 0.0) { rc = E / Q; rs = H / Q; } else { rc = 1.0; rs = 0.0; }
    const double phi = 0.5 * (atan2(G, F) + atan2(H, E));
    const double cp = cos(phi), sp = sin(phi);
    const double w1 = slim_weight(Q + R), w2 = slim_weight(Q - R);
    const double d = w1 - w2;
    w00 = w2 + d * cp * cp;
    w01 = d * cp * sp;
    w11 = w2 + d * sp * sp;
}


// Block-wide all-reduce of K values (every thread gets the totals, summed in
// the same order on every thread, so branch decisions stay uniform).
// `red` holds 2 * K * NW slots; `phase` alternates between the two halves so
// that one __syncthreads per reduction suffices.
template <int NT, int K, typename T>
__device__ __forceinline__ void block_sum(T (&v)[K], T* red, int& phase) {
    constexpr int NW = NT / kWarp;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T* buf = red + phase * K * NW;
    phase ^= 1;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        T x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) buf[k * NW + warp] = x;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        T s = T(0);
#pragma unroll
        for (int w = 0; w < NW; ++w) s += buf[k * NW + w];
        v[k] = s;
    }
}

template <int NT, typename T>
__device__ __forceinline__ T block_min(T v, T* red, int& phase) {
    constexpr int NW = NT / kWarp;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T* buf = red + phase * NW;
    phase ^= 1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T y = __shfl_xor_sync(0xffffffffu, v, o);
        v = y < v ? y : v;
    }
    if (lane == 0) buf[warp] = v;
    __syncthreads();
    T s = buf[0];
#pragma unroll
    for (int w = 1; w < NW; ++w) s = buf[w] < s ? buf[w] : s;
    return s;
}

template <int NT>
__device__ __forceinline__ int block_or(int v, int* red, int& phase) {
    constexpr int NW = NT / kWarp;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int* buf = red + phase * NW;
    phase ^= 1;
    v = __any_sync(0xffffffffu, v) ? 1 : 0;
    if (lane == 0) buf[warp] = v;
    __syncthreads();
    int s = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) s |= buf[w];
    return s;
}

// Ordered-bits atomic max of a non-negative double (IEEE order equals integer
// order for non-negative values).
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    if (!(v >= 0.0)) return;
    atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

}  // namespace uva
