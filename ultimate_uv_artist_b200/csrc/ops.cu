// Batch utilities: orientation, flip repair, per-chart flip counts, signed
// areas, Jacobians and target-size shrinking (engine/gpu.py:145-295,
// engine/param.py:477-516). One CTA per island where a per-island reduction
// or an island-local iteration is needed; one thread per triangle otherwise.
#include <cuda_runtime.h>

#include "common.cuh"

using namespace uva;

namespace {

__device__ __forceinline__ double sarea(const double2* U, int v0, int4 tv) {
    const double2 a = U[v0 + tv.x], b = U[v0 + tv.y], c = U[v0 + tv.z];
    return 0.5 * ((b.x - a.x) * (c.y - a.y) - (c.x - a.x) * (b.y - a.y));
}

// gpu.py:275-281: mirror v of islands whose area-weighted orientation is negative.
template <int NT>
__global__ void k_orient(uva_batch b) {
    __shared__ double red[2 * 4 * (NT / 32)];
    int phase = 0;
    const int isl = blockIdx.x;
    const int v0 = b.vofs[isl], f0 = b.tofs[isl], f1 = b.tofs[isl + 1];
    double2* U = reinterpret_cast<double2*>(b.U);
    double s[1] = {0.0};
    for (int f = f0 + threadIdx.x; f < f1; f += NT) {
        const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
        const double sa = sarea(U, v0, tv);
        const double area = b.frame[4 * f + 3];
        s[0] += (sa > 0.0 ? 1.0 : (sa < 0.0 ? -1.0 : 0.0)) * area;
    }
    block_sum<NT, 1>(s, red, phase);
    if (s[0] < 0.0) {
        for (int v = v0 + threadIdx.x; v < b.vofs[isl + 1]; v += NT) U[v].y = -U[v].y;
    }
}

// gpu.py:251-273: synchronous (Jacobi) moves of interior vertices of folded
// triangles to the mean of their unique-edge neighbours, per island until no
// fold is left or `rounds` is reached.
template <int NT>
__global__ void k_repair(uva_batch b, int rounds, uint8_t* mark) {
    __shared__ int redi[2 * (NT / 32)];
    int phase = 0;
    const int isl = blockIdx.x;
    const int v0 = b.vofs[isl], n = b.vofs[isl + 1] - v0, f0 = b.tofs[isl], f1 = b.tofs[isl + 1];
    const int s0 = b.sofs[isl];
    double2* U = reinterpret_cast<double2*>(b.U);
    double2* tmp = reinterpret_cast<double2*>(b.x64);
    for (int r = 0; r < rounds; ++r) {
        for (int i = threadIdx.x; i < n; i += NT) mark[v0 + i] = 0;
        __syncthreads();
        int any = 0;
        for (int f = f0 + threadIdx.x; f < f1; f += NT) {
            const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
            const bool ok = b.wtri[4 * f + 3] != 0.0;
            if (ok && sarea(U, v0, tv) < 0.0) {
                any = 1;
                mark[v0 + tv.x] = 1; mark[v0 + tv.y] = 1; mark[v0 + tv.z] = 1;
            }
        }
        any = block_or<NT>(any, redi, phase);
        if (!any) break;
        for (int i = threadIdx.x; i < n; i += NT) {
            const int v = v0 + i;
            double2 u = U[v];
            if (mark[v] && !(b.vflags[v] & 1)) {
                const int row = b.vert_row[v];   // solver row of vertex i
                const int s = s0 + (row >> 5);
                const int q0 = b.slice_ptr[s] + (row & 31), width = (b.slice_ptr[s + 1] - b.slice_ptr[s]) >> 5;
                double sx = 0.0, sy = 0.0;
                int deg = 0;
                for (int k = 0; k < width; ++k) {
                    const int q = q0 + 32 * k;
                    if (b.slot_edge[q] < 0) continue;
                    const double2 w = U[v0 + b.row_vert[v0 + b.slot_col[q]]];
                    sx += w.x; sy += w.y; ++deg;
                }
                const double dd = deg > 0 ? static_cast<double>(deg) : 1.0;
                u = make_double2(sx / dd, sy / dd);
            }
            tmp[v] = u;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += NT) U[v0 + i] = tmp[v0 + i];
        __syncthreads();
    }
}

// param.py:477-516: Gauss-Seidel repair in triangle order, one thread per
// island (the reference kernel is serial, and its result depends on order).
__global__ void k_repair_serial(uva_batch b, int rounds) {
    const int isl = blockIdx.x * blockDim.x + threadIdx.x;
    if (isl >= b.nc) return;
    const int v0 = b.vofs[isl], f0 = b.tofs[isl], f1 = b.tofs[isl + 1], s0 = b.sofs[isl];
    double2* U = reinterpret_cast<double2*>(b.U);
    for (int r = 0; r < rounds; ++r) {
        int bad = 0;
        for (int f = f0; f < f1; ++f) {
            const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
            const double2 a = U[v0 + tv.x], bb = U[v0 + tv.y], c = U[v0 + tv.z];
            const double ar = (bb.x - a.x) * (c.y - a.y) - (c.x - a.x) * (bb.y - a.y);
            if (ar > 0.0) continue;
            ++bad;
            const int cs[3] = {tv.x, tv.y, tv.z};
            for (int k = 0; k < 3; ++k) {
                const int i = cs[k];
                if (b.vflags[v0 + i] & 2) continue;
                const int row = b.vert_row[v0 + i];   // neighbours in ascending vertex order
                const int s = s0 + (row >> 5);
                const int q0 = b.slice_ptr[s] + (row & 31), width = (b.slice_ptr[s + 1] - b.slice_ptr[s]) >> 5;
                double sx = 0.0, sy = 0.0;
                int cnt = 0;
                for (int kk = 0; kk < width; ++kk) {
                    const int q = q0 + 32 * kk;
                    if (b.slot_edge[q] < 0) continue;
                    const double2 w = U[v0 + b.row_vert[v0 + b.slot_col[q]]];
                    sx += w.x; sy += w.y; ++cnt;
                }
                if (cnt > 0) U[v0 + i] = make_double2(sx / cnt, sy / cnt);
            }
        }
        if (bad == 0) break;
    }
}

__global__ void k_signed_area(uva_batch b, const double2* U, double* out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t) return;
    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
    out[f] = sarea(U, b.vofs[tv.w], tv);
}

__global__ void k_flips(uva_batch b, float* out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t) return;
    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
    const double2* U = reinterpret_cast<const double2*>(b.U);
    if (b.wtri[4 * f + 3] != 0.0 && sarea(U, b.vofs[tv.w], tv) < 0.0) atomicAdd(out + tv.w, 1.0f);
}

// gpu.py:145-151 (x1, y2 already clamped by the setup).
__global__ void k_jacobians(uva_batch b, const double2* U, double* out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t) return;
    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
    const int v0 = b.vofs[tv.w];
    const double4 fr = reinterpret_cast<const double4*>(b.frame)[f];
    const double2 a0 = U[v0 + tv.x], a1 = U[v0 + tv.y], a2 = U[v0 + tv.z];
    const double j00 = (a1.x - a0.x) / fr.x, j10 = (a1.y - a0.y) / fr.x;
    const double j01 = ((a2.x - a0.x) - j00 * fr.y) / fr.z, j11 = ((a2.y - a0.y) - j10 * fr.y) / fr.z;
    reinterpret_cast<double4*>(out)[f] = make_double4(j00, j01, j10, j11);
}

// gpu.py:283-295: grow the selection by `rings` vertex rings, then scale.
__global__ void k_mark_from_sel(uva_batch b, const uint8_t* sel, uint8_t* vmark) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t || !sel[f]) return;
    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
    const int v0 = b.vofs[tv.w];
    vmark[v0 + tv.x] = 1; vmark[v0 + tv.y] = 1; vmark[v0 + tv.z] = 1;
}
__global__ void k_sel_from_mark(uva_batch b, uint8_t* sel, const uint8_t* vmark) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t) return;
    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
    const int v0 = b.vofs[tv.w];
    sel[f] = (vmark[v0 + tv.x] | vmark[v0 + tv.y] | vmark[v0 + tv.z]) ? 1 : 0;
}
__global__ void k_apply_scale(uva_batch b, const uint8_t* sel, float factor, float floor_) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t || !sel[f]) return;
    b.tscale[f] = fmaxf(b.tscale[f] * factor, floor_);
}

inline int blocks(int n, int t) { return (n + t - 1) / t; }

}  // namespace

extern "C" int uva_orient_positive(uva_batch* b, void* stream) {
    if (!b) { uva_set_error("uva_orient_positive: null batch"); return UVA_E_ARG; }
    if (b->nc == 0) return UVA_OK;
    k_orient<256><<<b->nc, 256, 0, static_cast<cudaStream_t>(stream)>>>(*b);
    UVA_CHECK_LAUNCH("uva_orient_positive");
    return UVA_OK;
}

extern "C" int uva_repair_flips(uva_batch* b, int32_t rounds, void* stream) {
    if (!b || rounds < 0) { uva_set_error("uva_repair_flips: bad arguments"); return UVA_E_ARG; }
    if (b->nc == 0 || rounds == 0) return UVA_OK;
    // vertex marks live in the FP32 scratch (n floats >= n bytes)
    uint8_t* mark = reinterpret_cast<uint8_t*>(b->r32);
    k_repair<256><<<b->nc, 256, 0, static_cast<cudaStream_t>(stream)>>>(*b, rounds, mark);
    UVA_CHECK_LAUNCH("uva_repair_flips");
    return UVA_OK;
}

extern "C" int uva_repair_flips_serial(uva_batch* b, int32_t rounds, void* stream) {
    if (!b || rounds < 0) { uva_set_error("uva_repair_flips_serial: bad arguments"); return UVA_E_ARG; }
    if (b->nc == 0 || rounds == 0) return UVA_OK;
    k_repair_serial<<<blocks(b->nc, 64), 64, 0, static_cast<cudaStream_t>(stream)>>>(*b, rounds);
    UVA_CHECK_LAUNCH("uva_repair_flips_serial");
    return UVA_OK;
}

extern "C" int uva_flips_per_chart(const uva_batch* b, float* out, void* stream) {
    if (!b || !out) { uva_set_error("uva_flips_per_chart: bad arguments"); return UVA_E_ARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(out, 0, sizeof(float) * static_cast<size_t>(b->nc), s);
    if (b->t > 0) k_flips<<<blocks(b->t, 256), 256, 0, s>>>(*b, out);
    UVA_CHECK_LAUNCH("uva_flips_per_chart");
    return UVA_OK;
}

extern "C" int uva_signed_area(const uva_batch* b, const double* U, double* out, void* stream) {
    if (!b || !U || !out) { uva_set_error("uva_signed_area: bad arguments"); return UVA_E_ARG; }
    if (b->t > 0)
        k_signed_area<<<blocks(b->t, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(*b, reinterpret_cast<const double2*>(U), out);
    UVA_CHECK_LAUNCH("uva_signed_area");
    return UVA_OK;
}

extern "C" int uva_jacobians(const uva_batch* b, const double* U, double* out, void* stream) {
    if (!b || !U || !out) { uva_set_error("uva_jacobians: bad arguments"); return UVA_E_ARG; }
    if (b->t > 0)
        k_jacobians<<<blocks(b->t, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(*b, reinterpret_cast<const double2*>(U), out);
    UVA_CHECK_LAUNCH("uva_jacobians");
    return UVA_OK;
}

extern "C" int uva_shrink(uva_batch* b, uint8_t* sel, uint8_t* vmark, int32_t rings, float factor, float floor_,
                          void* stream) {
    if (!b || !sel || !vmark || rings < 0) { uva_set_error("uva_shrink: bad arguments"); return UVA_E_ARG; }
    if (b->t == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(vmark, 0, static_cast<size_t>(b->n), s);
    for (int r = 0; r < rings; ++r) {
        k_mark_from_sel<<<blocks(b->t, 256), 256, 0, s>>>(*b, sel, vmark);
        k_sel_from_mark<<<blocks(b->t, 256), 256, 0, s>>>(*b, sel, vmark);
    }
    k_apply_scale<<<blocks(b->t, 256), 256, 0, s>>>(*b, sel, factor, floor_);
    UVA_CHECK_LAUNCH("uva_shrink");
    return UVA_OK;
}
