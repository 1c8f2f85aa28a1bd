// Batched per-island parameterization on B200: setup, LSCM and ARAP.
//
// Design (one island per CTA "team", persistent launch):
//  * A batch holds thousands of independent islands. Every solve is
//    block-diagonal, so no grid-wide synchronisation is ever needed: each CTA
//    pulls the next island (largest first) from an atomic work counter and
//    runs that island's WHOLE solve - all ARAP local/global iterations, every
//    CG iteration, every FP64 refinement and the line search - before taking
//    the next. The host never syncs inside a solve (the reference syncs the
//    host once per CG iteration, engine/gpu.py:196).
//  * The Laplacian is applied in difference form, (L x)_i = sum_j w_ij (x_i -
//    x_j) + [i == pin] wpin x_i, from FP32 edge weights in a sliced-ELL layout.
//    Zero row sums then hold exactly in any precision, which keeps the
//    near-singular soft-pinned system well posed in FP32.
//  * Mixed precision: each global step solves L x = b with FP32 Jacobi-PCG
//    corrections and recomputes the residual b - L x in FP64 (iterative
//    refinement) until ||b - L x|| <= tol ||b|| per column, checked in FP64.
//    x and the UVs are kept in FP64.
//  * Convergence is per island and per column, so small islands stop early
//    and never wait for the largest one (the reference's test is global over
//    the batch, engine/gpu.py:196).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"

using namespace uva;

namespace {

// ------------------------------------------------------------------ setup
// Isometric frame and half-cotangent weights of every triangle.
// BATCH semantics: engine/gpu.py:88-121 (ok mask, 1e-30 clamps).
// PARAM semantics: engine/param.py:19-44 (no mask, 1e-300 clamps).
__global__ void k_frames(uva_batch b, double* wmax_isl) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    int isl = -1;
    double m = 0.0;
    if (f < b.t) {
        const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
        const int v0 = b.vofs[tv.w];
        const double* P = b.P;
        const double p0x = P[3 * (v0 + tv.x)], p0y = P[3 * (v0 + tv.x) + 1], p0z = P[3 * (v0 + tv.x) + 2];
        const double e1x = P[3 * (v0 + tv.y)] - p0x, e1y = P[3 * (v0 + tv.y) + 1] - p0y, e1z = P[3 * (v0 + tv.y) + 2] - p0z;
        const double e2x = P[3 * (v0 + tv.z)] - p0x, e2y = P[3 * (v0 + tv.z) + 1] - p0y, e2z = P[3 * (v0 + tv.z) + 2] - p0z;
        const bool batch = b.semantics == UVA_SEM_BATCH;
        double l1 = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
        const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
        const double dbl = sqrt(nx * nx + ny * ny + nz * nz);
        const double clampl = batch ? 1e-30 : 1e-300;
        if (batch) l1 = fmax(l1, 1e-30);
        const double il = 1.0 / fmax(l1, clampl);
        const double exx = e1x * il, exy = e1y * il, exz = e1z * il;
        const double in = 1.0 / fmax(dbl, clampl);
        const double ux = nx * in, uy = ny * in, uz = nz * in;
        const double eyx = uy * exz - uz * exy, eyy = uz * exx - ux * exz, eyz = ux * exy - uy * exx;
        double X1 = l1, X2 = e2x * exx + e2y * exy + e2z * exz, Y2 = e2x * eyx + e2y * eyy + e2z * eyz;
        bool ok = true;
        if (batch) {
            ok = (dbl > 1e-14 * fmax(l1 * l1, 1e-300)) && isfinite(dbl);
            if (!ok) { X1 = 0.0; X2 = 0.0; Y2 = 0.0; }
        }
        // cotangent of the angle at corner o opposite edge k (corners k+1, k+2)
        const double cx[3] = {0.0, X1, X2}, cy[3] = {0.0, 0.0, Y2};
        double w[3];
        const double crmin = batch ? 1e-30 : 1e-300;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int i = (k + 1) % 3, j = (k + 2) % 3;
            const double ax = cx[i] - cx[k], ay = cy[i] - cy[k], bx = cx[j] - cx[k], by = cy[j] - cy[k];
            const double cr = fmax(fabs(ax * by - ay * bx), crmin);
            double c = (ax * bx + ay * by) / cr;
            c = fmin(fmax(c, -1e4), 1e4);
            w[k] = ok ? 0.5 * c : 0.0;
        }
        if (batch) {
            // Jacobian denominators as engine/gpu.py:117-120 clamps them
            X1 = fmax(X1, 1e-30);
            if (!(fabs(Y2) > 1e-30)) Y2 = 1e-30;
        }
        reinterpret_cast<double4*>(b.frame)[f] = make_double4(X1, X2, Y2, 0.5 * dbl);
        reinterpret_cast<double4*>(b.wtri)[f] = make_double4(w[0], w[1], w[2], ok ? 1.0 : 0.0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int e = b.tri_edge[3 * f + k];
            if (e >= 0) atomicAdd(&b.wedge[e], w[k]);
            m = fmax(m, fabs(w[k]));
        }
        isl = tv.w;
    }
    // the island's max |w|: a segmented maximum over the warp (triangles of
    // an island are contiguous), then one atomic per island and warp instead
    // of one per triangle on the island's slot
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_down_sync(0xffffffffu, m, o);
        const int yi = __shfl_down_sync(0xffffffffu, isl, o);
        if (lane + o < 32 && yi == isl) m = fmax(m, y);
    }
    const int prev = __shfl_up_sync(0xffffffffu, isl, 1);
    if (isl >= 0 && (lane == 0 || prev != isl)) atomic_max_nonneg(&wmax_isl[isl], m);
}

// Pin weight: BATCH one global max |w| clamped at 1e-12 (gpu.py:138);
// PARAM per island max |W| (param.py:394).
__global__ void k_wpin(uva_batch b, const double* wmax_isl) {
    __shared__ double red[64];
    int phase = 0;
    double m = 0.0;
    if (b.semantics == UVA_SEM_BATCH) {
        for (int i = threadIdx.x; i < b.nc; i += blockDim.x) m = fmax(m, wmax_isl[i]);
        m = block_min<1024, double>(-m, red, phase);
        m = fmax(-m, 1e-12);
        for (int i = threadIdx.x; i < b.nc; i += blockDim.x) b.wpin[i] = m;
    } else {
        for (int i = threadIdx.x; i < b.nc; i += blockDim.x) {
            const double v = wmax_isl[i];
            b.wpin[i] = (b.tofs[i + 1] > b.tofs[i]) ? fmax(v, 1e-300) : 1.0;
        }
    }
}

// FP32 slot weights and the Jacobi diagonal (without the pin).
__global__ void k_rows(uva_batch b, const int32_t* vert_isl) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= b.n) return;
    const int isl = vert_isl[v];
    const int i = v - b.vofs[isl];
    const int s = b.sofs[isl] + (i >> 5);
    const int q0 = b.slice_ptr[s] + (i & 31);
    const int width = (b.slice_ptr[s + 1] - b.slice_ptr[s]) >> 5;
    double sum = 0.0;
    for (int k = 0; k < width; ++k) {
        const int q = q0 + 32 * k;
        const int e = b.slot_edge[q];
        const float w32 = e >= 0 ? static_cast<float>(b.wedge[e]) : 0.0f;
        const int c2 = __float2int_rn(2.0f * b.slot_c[q]);   // |c2| <= 127 (checked by the plan)
        reinterpret_cast<int2*>(b.slot_cw)[q] = make_int2((c2 << 24) | b.slot_col[q], __float_as_int(w32));
        sum += static_cast<double>(w32);
    }
    b.wdiag[v] = sum;
    b.dinv[v] = sum > 1e-30 ? static_cast<float>(1.0 / sum) : 1.0f;
    // the island's last row also fills the padding rows of its slice (the
    // plan's zero-weight slots): the solver's slice-wide products read them
    const int n = b.vofs[isl + 1] - b.vofs[isl];
    if (i == n - 1) {
        for (int r = i + 1; r < ((n + 31) & ~31); ++r) {
            const int qr = b.slice_ptr[s] + (r & 31);
            for (int k = 0; k < width; ++k)
                reinterpret_cast<int2*>(b.slot_cw)[qr + 32 * k] = make_int2(b.slot_col[qr + 32 * k], 0);
        }
    }
}

// LSCM pins: the far boundary pair of engine/param.py:172-179, evaluated in
// the same order as numpy (sequential centroid sum, first index on ties).
__global__ void k_far_pair(uva_batch b) {
    const int isl = blockIdx.x * blockDim.x + threadIdx.x;
    if (isl >= b.nc) return;
    const int v0 = b.vofs[isl];
    const int lo = b.bofs[isl], hi = b.bofs[isl + 1];
    b.pins[3 * isl + 0] = 0;
    if (hi <= lo) { b.pins[3 * isl + 1] = -1; b.pins[3 * isl + 2] = -1; return; }
    const double* P = b.P;
    double cx = 0.0, cy = 0.0, cz = 0.0;
    for (int q = lo; q < hi; ++q) {
        const int v = v0 + b.bverts[q];
        cx += P[3 * v]; cy += P[3 * v + 1]; cz += P[3 * v + 2];
    }
    const double cnt = static_cast<double>(hi - lo);
    cx /= cnt; cy /= cnt; cz /= cnt;
    int bi = b.bverts[lo];
    double best = -1.0;
    for (int q = lo; q < hi; ++q) {
        const int v = v0 + b.bverts[q];
        const double dx = P[3 * v] - cx, dy = P[3 * v + 1] - cy, dz = P[3 * v + 2] - cz;
        const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        if (d2 > best) { best = d2; bi = b.bverts[q]; }
    }
    int bj = b.bverts[lo];
    best = -1.0;
    const int vi = v0 + bi;
    for (int q = lo; q < hi; ++q) {
        const int v = v0 + b.bverts[q];
        const double dx = P[3 * v] - P[3 * vi], dy = P[3 * v + 1] - P[3 * vi + 1], dz = P[3 * v + 2] - P[3 * vi + 2];
        const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        if (d2 > best) { best = d2; bj = b.bverts[q]; }
    }
    if (bi == bj) bj = (b.bverts[lo] != bi) ? b.bverts[lo] : b.bverts[hi - 1];
    b.pins[3 * isl + 1] = bi;
    b.pins[3 * isl + 2] = bj;
}

__global__ void k_vert_isl(const int32_t* vofs, int nc, int32_t* vert_isl) {
    const int isl = blockIdx.x;
    if (isl >= nc) return;
    for (int v = vofs[isl] + threadIdx.x; v < vofs[isl + 1]; v += blockDim.x) vert_isl[v] = isl;
}

// ------------------------------------------------------------------ island solver
// One persistent launch of 1024-thread CTAs serves four island size classes
// (islands pre-sorted by vertex count and grouped by class in b.order):
//   G  n > 8192          whole CTA, CG vectors in global memory (L2)
//   A  2048 < n <= 8192  whole CTA, CG vectors p, r, d in shared memory
//   B  256 < n <= 2048   256-thread sub-team (named barrier), shared memory
//   C  n <= 256          one warp, shared memory
// A CTA drains class G, then A, then splits into sub-teams for B and warps
// for C, so small islands fill the SMs while the large ones finish.
constexpr int KB = 1024;              // CTA size
constexpr int RB = 8;                 // rows per thread in the shared-memory classes
constexpr int SUB = 256;              // sub-team size of class B
constexpr size_t kDynSmem = sizeof(float2) * 3 * KB * RB;   // 196,608 bytes

enum Op { OP_ARAP = 0, OP_LSCM = 1 };

// Class W: islands above kWideMin vertices are solved by the whole GPU as
// one team (k_wide: a cooperative launch of kWideCtas 1024-thread CTAs, one
// per SM), one island after another, before the persistent launch takes the
// other islands. A single CTA would keep them for hundreds of milliseconds
// while the rest of the batch is done in tens. The team syncs with a grid
// barrier (in the batch's cpart) and reduces across CTAs through per-CTA
// slots that every CTA adds up in the same order (in the batch's
// coarse_work), so its results are as reproducible as a single CTA's.
constexpr int kWideMin = 16384;
constexpr int kWideCtas = 148;
constexpr int kWideNTT = KB * kWideCtas;
constexpr int kRedMaxW = 10;   // values per reduction (the solver's kRedMax)

struct WideScratch {                    // at the start of the batch's cpart
    unsigned count, gen;                // grid barrier
    int abort, reserved;                // a barrier gave up: later barriers pass at once
};
constexpr int kWideHdr = 16;
// In the batch's coarse_work (the setup's FP64 workspace, free during the
// solves): per-CTA partials of the team's reductions, two sets in turn
// (kWideCtas x kRedMaxW doubles each), then the per-warp residual sums of
// the coarse restriction (one float2 per 32 rows).
constexpr int kWidePart = 2 * kWideCtas * kRedMaxW;

__device__ __forceinline__ unsigned wide_ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long wide_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier of the class-W team (all kWideCtas CTAs resident: a
// cooperative launch). A CTA that waits more than two seconds sets `abort`;
// from then on every barrier passes at once and the island's status says so.
__device__ __noinline__ void wide_sync(WideScratch* ws) {
    __syncthreads();
    if (threadIdx.x == 0 && !*reinterpret_cast<volatile int*>(&ws->abort)) {
        const unsigned g = wide_ld_acquire(&ws->gen);
        __threadfence();
        if (atomicAdd(&ws->count, 1u) == static_cast<unsigned>(kWideCtas) - 1u) {
            atomicExch(&ws->count, 0u);
            __threadfence();
            atomicAdd(&ws->gen, 1u);
        } else {
            const unsigned long long t0 = wide_ns();
            unsigned spins = 0;
            while (wide_ld_acquire(&ws->gen) == g) {
                if ((++spins & 255u) == 0 && wide_ns() - t0 > 2000000000ull) {
                    atomicExch(&ws->abort, 1);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <int NTT>
__device__ __forceinline__ void team_sync(int bar) {
    if constexpr (NTT == 32) {
        __syncwarp();
    } else if constexpr (NTT == KB) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(NTT) : "memory");
    }
}

template <int NTT>
struct Team {
    int tid, bar, phase;
    double* redd;
    float* redf;
    int* redi;
    int* slot;
    float2 *sp, *sr, *sd;   // CG vectors (shared memory, or null for class G)
    float *cg, *cy;         // coarse restriction / coarse solution (shared memory)
    int* sc;                // slice-pointer cache of the current island (shared memory)
    int sc_cap;             // its capacity (slices + 1)
    __nv_bfloat16* dc;      // Jacobi diagonal of the current island (shared memory, or null)
    int dc_cap;             // its capacity (rows)
    WideScratch* ws;        // class W only: grid barrier
    int wph;                // class W only: partial set in use (0, 1; the same on every thread)
    double* wpart;          // class W only: 2 x kWideCtas x kRedMaxW partials
    float2* wgw;            // class W only: per-warp residual sums of the coarse restriction
    __device__ __forceinline__ void sync() {
        if constexpr (NTT == kWideNTT) wide_sync(ws);
        else team_sync<NTT>(bar);
    }
};

// Class W: reduction partials alternate between two sets; a set is written
// again two reductions later, after every CTA has read it and passed a
// barrier since.
template <int NTT>
__device__ __forceinline__ double* wide_slots(Team<NTT>& tm) {
    double* p = tm.wpart + tm.wph * (kWideCtas * kRedMaxW);
    tm.wph ^= 1;
    return p;
}

// All-reduce of K values over the team; every thread gets bitwise-identical
// totals (xor butterflies are symmetric; the cross-warp sum runs in one order).
// The reduction buffers hold 2 * kRedMax values per warp.
constexpr int kRedMax = 10;
template <int NTT, int K, typename T>
__device__ __forceinline__ void team_sum(Team<NTT>& tm, T (&v)[K], T* red) {
    static_assert(K <= kRedMax, "team_sum: more values than the reduction buffers hold");
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    if constexpr (NTT == kWideNTT) {
        // CTA partial (warps in a fixed order) into this CTA's slot; after
        // the barrier every CTA's warp 0 adds the slots in the same order,
        // so every thread of the team gets the same bits
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        T* buf = red + tm.phase * K * 32;
        tm.phase ^= 1;
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) buf[k * 32 + warp] = v[k];
        }
        __syncthreads();
        double* slots = wide_slots(tm);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                double c = 0.0;
                for (int w = 0; w < 32; ++w) c += static_cast<double>(buf[k * 32 + w]);
                slots[blockIdx.x * kRedMaxW + k] = c;
            }
        }
        wide_sync(tm.ws);
        if (warp < K) {   // warp k adds value k: every load of a lane in flight at once
            constexpr int J = (kWideCtas + 31) / 32;
            double part[J];
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int q = lane + 32 * j;
                part[j] = q < kWideCtas ? __ldcg(slots + q * kRedMaxW + warp) : 0.0;
            }
            double c = 0.0;
#pragma unroll
            for (int j = 0; j < J; ++j) c += part[j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0) buf[warp * 32] = static_cast<T>(c);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = buf[k * 32];
    } else if constexpr (NTT > 32) {
        constexpr int NW = NTT / 32;
        const int lane = tm.tid & 31, warp = tm.tid >> 5;
        T* buf = red + tm.phase * K * NW;
        tm.phase ^= 1;
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) buf[k * NW + warp] = v[k];
        }
        tm.sync();
        // every warp folds the per-warp partials with the same butterfly
#pragma unroll
        for (int k = 0; k < K; ++k) {
            T s = lane < NW ? buf[k * NW + lane] : T(0);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            v[k] = s;
        }
    } else {
        __syncwarp();
    }
}

template <int NTT>
__device__ __forceinline__ double team_min(Team<NTT>& tm, double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if constexpr (NTT == kWideNTT) {
        double* buf = tm.redd + tm.phase * 4 * 32;
        tm.phase ^= 1;
        if ((threadIdx.x & 31) == 0) buf[threadIdx.x >> 5] = v;
        __syncthreads();
        double* slots = wide_slots(tm);
        if (threadIdx.x == 0) {
            double c = buf[0];
            for (int w = 1; w < 32; ++w) c = fmin(c, buf[w]);
            slots[blockIdx.x * kRedMaxW] = c;
        }
        wide_sync(tm.ws);
        if (threadIdx.x < 32) {
            double c = 1e300;
#pragma unroll
            for (int q = threadIdx.x; q < kWideCtas; q += 32) c = fmin(c, __ldcg(slots + q * kRedMaxW));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c = fmin(c, __shfl_xor_sync(0xffffffffu, c, o));
            if (threadIdx.x == 0) buf[0] = c;
        }
        __syncthreads();
        v = buf[0];
    } else if constexpr (NTT > 32) {
        constexpr int NW = NTT / 32;
        double* buf = tm.redd + tm.phase * 4 * NW;
        tm.phase ^= 1;
        if ((tm.tid & 31) == 0) buf[tm.tid >> 5] = v;
        tm.sync();
        v = (tm.tid & 31) < NW ? buf[tm.tid & 31] : 1e300;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    } else {
        __syncwarp();
    }
    return v;
}

template <int NTT>
__device__ __forceinline__ int team_or(Team<NTT>& tm, int v) {
    v = __any_sync(0xffffffffu, v) ? 1 : 0;
    if constexpr (NTT == kWideNTT) {
        const int c = __syncthreads_or(v);
        double* slots = wide_slots(tm);
        if (threadIdx.x == 0) slots[blockIdx.x * kRedMaxW] = c ? 1.0 : 0.0;
        wide_sync(tm.ws);
        int any = 0;
        if (threadIdx.x < 32) {
            for (int q = threadIdx.x; q < kWideCtas; q += 32) any |= __ldcg(slots + q * kRedMaxW) != 0.0;
        }
        v = __syncthreads_or(any);
    } else if constexpr (NTT > 32) {
        constexpr int NW = NTT / 32;
        int* buf = tm.redi + tm.phase * NW;
        tm.phase ^= 1;
        if ((tm.tid & 31) == 0) buf[tm.tid >> 5] = v;
        tm.sync();
        v = __any_sync(0xffffffffu, (tm.tid & 31) < NW && buf[tm.tid & 31] != 0) ? 1 : 0;
    } else {
        __syncwarp();
    }
    return v;
}

// Rows of the island owned by this thread: i = tid + j*NTT. R > 0: at most R
// rows (unrolled); R == 0: any number (class G).
template <int NTT, int R, typename F>
__device__ __forceinline__ void for_rows(int tid, int n, F&& f) {
    if constexpr (R > 0) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int i = tid + j * NTT;
            if (i < n) f(i, j);
        }
    } else {
        for (int i = tid; i < n; i += NTT) f(i, 0);
    }
}

// Same rows as for_rows, but every lane of a warp runs every iteration (with
// `valid` false past the island's last row), so warp shuffles are legal:
// the 32 lanes of a warp hold the 32 consecutive rows of one slice.
template <int NTT, int R, typename F>
__device__ __forceinline__ void slice_loop(int tid, int n, F&& f) {
    if constexpr (R > 0) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int i = tid + j * NTT;
            f(i, j, i < n);
        }
    } else {
        for (int base = 0; base < n; base += NTT) f(base + tid, 0, base + tid < n);
    }
}

struct Isl {
    int id, v0, n, f0, nt, s0;
    int pin, p0, p1;          // solver rows of the ARAP pin and the LSCM pins (-1: none)
    int pinv;                 // ARAP pin vertex
    int agg, M, co;           // rows per aggregate, aggregates (0: Jacobi only), coarse offset
    int aggsh;                // log2(agg) when agg is a power of two, else -1
    const int* sptr;          // slot offsets of the island's slices (shared-memory cache or global)
    const __nv_bfloat16* dv;  // Jacobi diagonal in shared memory (null: read b.dinv)
    double wpin;
};

template <Op OP>
__device__ __forceinline__ Isl load_island(const uva_batch& b, int isl) {
    Isl I;
    I.id = isl;
    I.v0 = b.vofs[isl]; I.n = b.vofs[isl + 1] - I.v0;
    I.f0 = b.tofs[isl]; I.nt = b.tofs[isl + 1] - I.f0;
    I.s0 = b.sofs[isl];
    I.pinv = b.pins[3 * isl];
    I.pin = I.n > 0 ? b.vert_row[I.v0 + I.pinv] : -1;
    const int p0 = b.pins[3 * isl + 1], p1 = b.pins[3 * isl + 2];
    I.p0 = p0 >= 0 ? b.vert_row[I.v0 + p0] : -1;
    I.p1 = p1 >= 0 ? b.vert_row[I.v0 + p1] : -1;
    I.agg = b.agg_rows[isl];
    I.M = I.agg > 0 ? (I.n + I.agg - 1) / I.agg : 0;
    I.co = b.cofs[isl];
    I.aggsh = (I.agg > 0 && (I.agg & (I.agg - 1)) == 0) ? __ffs(I.agg) - 1 : -1;
    I.sptr = b.slice_ptr + I.s0;
    I.dv = nullptr;
    I.wpin = b.wpin[isl];
    return I;
}

__device__ __forceinline__ int agg_of(const Isl& I, int i) { return I.aggsh >= 0 ? (i >> I.aggsh) : i / I.agg; }

// Packed slot column: island row in the low 24 bits, twice the LSCM
// boundary coupling (a small integer) in the high 8 bits.
__device__ __forceinline__ int slot_row(int x) { return x & 0xFFFFFF; }
__device__ __forceinline__ float slot_c2(int x) { return static_cast<float>(x >> 24); }

__device__ __forceinline__ void row_slots(const uva_batch&, const Isl& I, int i, int& q0, int& width) {
    const int s = i >> 5;
    const int p = I.sptr[s];
    q0 = p + (i & 31);
    width = (I.sptr[s + 1] - p) >> 5;
}

template <Op OP>
__device__ __forceinline__ bool is_pinned(const Isl& I, int i) {
    return OP == OP_LSCM && (i == I.p0 || i == I.p1);
}

// (A x)_i in FP64 from an FP64 vector (global memory, island-local indices).
template <Op OP>
__device__ __forceinline__ double2 apply64(const uva_batch& b, const Isl& I, int i, const double2* x) {
    int q0, width;
    row_slots(b, I, i, q0, width);
    const int2* cw = reinterpret_cast<const int2*>(b.slot_cw);
    const double2 xi = x[i];
    double ax = 0.0, ay = 0.0;
#pragma unroll 4
    for (int k = 0; k < width; ++k) {
        const int q = q0 + 32 * k;
        const int2 s = __ldg(cw + q);
        const double w = static_cast<double>(__int_as_float(s.y));
        const double2 xj = x[slot_row(s.x)];
        ax += w * (xi.x - xj.x);
        ay += w * (xi.y - xj.y);
        if (OP == OP_LSCM) {
            const double c = 0.5 * static_cast<double>(slot_c2(s.x));
            ax += c * xj.y;
            ay -= c * xj.x;
        }
    }
    if (OP == OP_ARAP && i == I.pin) { ax += I.wpin * xi.x; ay += I.wpin * xi.y; }
    return make_double2(ax, ay);
}

// LSCM boundary coupling of four slots: (A p)_i += c_ij (p_j.y, -p_j.x).
// Only boundary rows have nonzero c, so the products callers take it on
// test the slots' coupling bits first and most groups skip it.
__device__ __forceinline__ void lscm_coupling(const int2 (&s)[4], const float2* p, float& ax, float& ay) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const float c = 0.5f * slot_c2(s[u].x);
        const float2 xj = p[slot_row(s[u].x)];
        ax = fmaf(c, xj.y, ax);
        ay = fmaf(-c, xj.x, ay);
    }
}

// (A p)_i in FP32, four slots per step (slice widths are multiples of 4).
template <Op OP>
__device__ __forceinline__ float2 apply32(const uva_batch& b, const Isl& I, int i, const float2* p, float wpin32) {
    int q0, width;
    row_slots(b, I, i, q0, width);
    const int2* cw = reinterpret_cast<const int2*>(b.slot_cw);
    const float2 xi = p[i];
    float ax = 0.f, ay = 0.f;
    for (int k = 0; k < width; k += 4) {
        int2 s[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) s[u] = __ldg(cw + q0 + 32 * (k + u));
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float2 xj = p[slot_row(s[u].x)];
            const float w = __int_as_float(s[u].y);
            ax = fmaf(w, xi.x - xj.x, ax);
            ay = fmaf(w, xi.y - xj.y, ay);
        }
        if (OP == OP_LSCM && ((s[0].x | s[1].x | s[2].x | s[3].x) >> 24) != 0) lscm_coupling(s, p, ax, ay);
    }
    if (OP == OP_ARAP && i == I.pin) { ax = fmaf(wpin32, xi.x, ax); ay = fmaf(wpin32, xi.y, ay); }
    return make_float2(ax, ay);
}

// Four slots of one row of (A p), accumulated into (ax, ay).
template <Op OP>
__device__ __forceinline__ void row_group4(const int2* cw, int q, const float2* p, float2 x, float& ax, float& ay) {
    int2 s[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) s[u] = __ldg(cw + q + 32 * u);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const float2 y = p[slot_row(s[u].x)];
        const float w = __int_as_float(s[u].y);
        ax = fmaf(w, x.x - y.x, ax);
        ay = fmaf(w, x.y - y.y, ay);
    }
    if (OP == OP_LSCM && ((s[0].x | s[1].x | s[2].x | s[3].x) >> 24) != 0) lscm_coupling(s, p, ax, ay);
}

// (A p) for two rows of one thread at once (rows of different slices):
// the slot loads of both rows are in flight together, which halves the
// chain of dependent L2 round trips of the single-row product. Row ib is
// used only when hb (its slice exists); widths are per slice, so every loop
// bound is the same on all lanes of the warp.
template <Op OP>
__device__ __forceinline__ void apply32_pair(const uva_batch& b, const Isl& I, int ia, int ib, bool hb,
                                             const float2* p, float wpin32, float2& qa, float2& qb) {
    int q0a, wa, q0b = 0, wb = 0;
    row_slots(b, I, ia, q0a, wa);
    if (hb) row_slots(b, I, ib, q0b, wb);
    const int2* cw = reinterpret_cast<const int2*>(b.slot_cw);
    const float2 xa = p[ia], xb = hb ? p[ib] : make_float2(0.f, 0.f);
    float ax = 0.f, ay = 0.f, bx = 0.f, by = 0.f;
    const int wmin = min(wa, wb);
    int k = 0;
    for (; k < wmin; k += 4) {
        int2 sa[4], sb[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            sa[u] = __ldg(cw + q0a + 32 * (k + u));
            sb[u] = __ldg(cw + q0b + 32 * (k + u));
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float2 ya = p[slot_row(sa[u].x)];
            const float wA = __int_as_float(sa[u].y);
            ax = fmaf(wA, xa.x - ya.x, ax);
            ay = fmaf(wA, xa.y - ya.y, ay);
            const float2 yb = p[slot_row(sb[u].x)];
            const float wB = __int_as_float(sb[u].y);
            bx = fmaf(wB, xb.x - yb.x, bx);
            by = fmaf(wB, xb.y - yb.y, by);
        }
        if (OP == OP_LSCM) {
            if (((sa[0].x | sa[1].x | sa[2].x | sa[3].x) >> 24) != 0) lscm_coupling(sa, p, ax, ay);
            if (((sb[0].x | sb[1].x | sb[2].x | sb[3].x) >> 24) != 0) lscm_coupling(sb, p, bx, by);
        }
    }
    for (int ka = k; ka < wa; ka += 4) row_group4<OP>(cw, q0a + 32 * ka, p, xa, ax, ay);
    for (int kb = k; kb < wb; kb += 4) row_group4<OP>(cw, q0b + 32 * kb, p, xb, bx, by);
    if (OP == OP_ARAP && ia == I.pin) { ax = fmaf(wpin32, xa.x, ax); ay = fmaf(wpin32, xa.y, ay); }
    if (OP == OP_ARAP && ib == I.pin) { bx = fmaf(wpin32, xb.x, bx); by = fmaf(wpin32, xb.y, by); }
    qa = is_pinned<OP>(I, ia) ? make_float2(0.f, 0.f) : make_float2(ax, ay);
    qb = (hb && !is_pinned<OP>(I, ib)) ? make_float2(bx, by) : make_float2(0.f, 0.f);
}

// Inverse Jacobi diagonal of row i: 0 on the LSCM hard pins, the ARAP pin
// row includes the soft-pin weight.
template <Op OP>
__device__ __forceinline__ float jacobi_global(const uva_batch& b, const Isl& I, int i) {
    if (is_pinned<OP>(I, i)) return 0.0f;
    if (OP == OP_ARAP && i == I.pin) {
        const double diag = b.wdiag[I.v0 + i] + I.wpin;
        return diag > 1e-30 ? static_cast<float>(1.0 / diag) : 1.0f;
    }
    return __ldg(b.dinv + I.v0 + i);
}

// The preconditioner reads a bfloat16 copy from shared memory when the team
// has room for it (a preconditioner may be approximate; CG stays exact).
template <Op OP>
__device__ __forceinline__ float jacobi(const uva_batch& b, const Isl& I, int i) {
    if (I.dv) return __bfloat162float(I.dv[i]);
    return jacobi_global<OP>(b, I, i);
}

// Inverse coarse operators are stored as FP16, scaled so that the largest
// entry is 1024 (a CPU probe on LSCM islands: same PCG iterations as FP32,
// still positive definite), in the first half of the island's FP32 block;
// the float after the halves holds the inverse of the scale. ARAP: the real
// M x M inverse; LSCM: the complex M x M inverse of the complex Hermitian
// operator whose real representation is the (u, v) system, as (re, im)
// half pairs. Rows are padded (zeros) to an even number of entries: one
// vector load takes 2 entries (4-byte aligned ARAP blocks, 16-byte aligned
// LSCM blocks).
__host__ __device__ __forceinline__ const float* coarse_scale(const float* block, int nhalf) {
    return block + (nhalf + 1) / 2;
}
__host__ __device__ constexpr int coarse_stride(int N, int vec) { return (N + vec - 1) / vec * vec; }

// Two-level additive preconditioner z = D^-1 r + P Ac^-1 P^T r. P is the
// piecewise-constant prolongation over aggregates of `agg` consecutive solver
// rows (compact mesh blobs from the plan; agg is a multiple of 64, so an
// aggregate is agg/32 whole slices), Ac = P^T A P is inverted once per batch
// by the setup.
// y = Ac^-1 P^T r for the residual r (complete: a team barrier precedes the
// call). The restriction g = P^T r is deterministic: T threads per aggregate
// (a power of two, T * M <= NTT where possible) add rows a*agg + t, + T, ...
// and fold with xor shuffles in a fixed order. Ends with a barrier: y complete.
template <Op OP>
__device__ void coarse_solve_wide(const uva_batch& b, Team<kWideNTT>& tm, const Isl& I, const float2* r);

template <int NTT, Op OP>
__device__ __forceinline__ void coarse_solve(const uva_batch& b, Team<NTT>& tm, const Isl& I, const float2* r) {
    if constexpr (NTT == kWideNTT) {
        coarse_solve_wide<OP>(b, tm, I, r);
        return;
    }
    int lt = 5;   // log2 T
    while (lt > 0 && (I.M << lt) > NTT) --lt;
    const int T = 1 << lt, groups = NTT >> lt;
    for (int base = 0; base < I.M; base += groups) {   // the same trip count on every thread
        const int a = base + (tm.tid >> lt), t = tm.tid & (T - 1);
        float gx = 0.f, gy = 0.f;
        if (a < I.M) {
            const int r1 = min((a + 1) * I.agg, I.n);
            for (int i = a * I.agg + t; i < r1; i += T) {
                const float2 v = r[i];
                gx += v.x; gy += v.y;
            }
        }
        for (int o = T >> 1; o > 0; o >>= 1) {
            gx += __shfl_xor_sync(0xffffffffu, gx, o);
            gy += __shfl_xor_sync(0xffffffffu, gy, o);
        }
        if (t == 0 && a < I.M) {
            if (OP == OP_ARAP) { tm.cg[a] = gx; tm.cg[I.M + a] = gy; }
            else { tm.cg[2 * a] = gx; tm.cg[2 * a + 1] = gy; }
        }
    }
    // odd M: the product's last pair reads g one entry past the end (against a
    // zero matrix entry), which must hold a finite value
    if ((I.M & 1) && tm.tid == 0) { tm.cg[2 * I.M] = 0.f; tm.cg[2 * I.M + 1] = 0.f; }
    tm.sync();   // g complete
    // y = Ac^-1 g. ARAP: a real M x M inverse applied to the u and v
    // columns; LSCM: a complex M x M inverse (the real (u, v) operator is the
    // representation of a complex Hermitian one) applied to g_u + i g_v.
    // Eight lanes per coarse row, every row of the team in flight at once: a
    // lane takes a run of consecutive entries (two per load) and the group
    // folds with three xor shuffles.
    constexpr int G = 8;
    const int M = I.M;
    const int S = coarse_stride(M, 2);
    const float* blockf = OP == OP_ARAP ? b.coarse_a + I.co : b.coarse_l + 4 * static_cast<size_t>(I.co);
    const __half* A = reinterpret_cast<const __half*>(blockf);
    const float isc = __ldg(coarse_scale(blockf, (OP == OP_ARAP ? 1 : 2) * M * S));
    const int gl = tm.tid & (G - 1), grow = tm.tid / G;
    const int cpl = ((M + G - 1) / G + 1) & ~1;   // entries per lane, even
    const int c_beg = gl * cpl, c_end = min(c_beg + cpl, M);
    for (int base = 0; base < M; base += NTT / G) {   // the same trip count on every thread
        const int o = base + grow;
        float au = 0.f, av = 0.f;
        if (o < M) {
            for (int c = c_beg; c < c_end; c += 2) {   // c even: entry c + 1 < S (zero past M)
                if constexpr (OP == OP_ARAP) {
                    const unsigned raw = __ldg(reinterpret_cast<const unsigned*>(A + static_cast<size_t>(o) * S + c));
                    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw));
                    au = fmaf(a.x, tm.cg[c], au); au = fmaf(a.y, tm.cg[c + 1], au);
                    av = fmaf(a.x, tm.cg[M + c], av); av = fmaf(a.y, tm.cg[M + c + 1], av);
                } else {   // two complex entries (re, im) against (g_u, g_v) pairs
                    const uint2 raw = __ldg(reinterpret_cast<const uint2*>(A + 2 * (static_cast<size_t>(o) * S + c)));
                    const float2 z0 = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
                    const float2 z1 = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
                    const float4 g = *reinterpret_cast<const float4*>(tm.cg + 2 * c);
                    au = fmaf(z0.x, g.x, au); au = fmaf(-z0.y, g.y, au);
                    av = fmaf(z0.y, g.x, av); av = fmaf(z0.x, g.y, av);
                    au = fmaf(z1.x, g.z, au); au = fmaf(-z1.y, g.w, au);
                    av = fmaf(z1.y, g.z, av); av = fmaf(z1.x, g.w, av);
                }
            }
        }
#pragma unroll
        for (int k = G / 2; k > 0; k >>= 1) {
            au += __shfl_xor_sync(0xffffffffu, au, k);
            av += __shfl_xor_sync(0xffffffffu, av, k);
        }
        if (gl == 0 && o < M) {
            if (OP == OP_ARAP) { tm.cy[o] = au * isc; tm.cy[M + o] = av * isc; }
            else { tm.cy[2 * o] = au * isc; tm.cy[2 * o + 1] = av * isc; }
        }
    }
    tm.sync();   // y complete
}

template <int NTT, Op OP>
__device__ __forceinline__ float2 prolong(const Team<NTT>& tm, const Isl& I, int i) {
    const int a = agg_of(I, i);
    if (OP == OP_ARAP) return make_float2(tm.cy[a], tm.cy[I.M + a]);
    return make_float2(tm.cy[2 * a], tm.cy[2 * a + 1]);
}

// Class W coarse correction with one grid barrier: every warp stores the
// residual sum of its 32 rows (one aggregate: agg is a multiple of 32);
// after the barrier every CTA rebuilds g from those sums in a fixed order
// (the same bits in every CTA) in its shared memory and computes y for the
// aggregates of its own rows, the only ones prolong reads.
template <Op OP>
__device__ void coarse_solve_wide(const uva_batch& b, Team<kWideNTT>& tm, const Isl& I, const float2* r) {
    const int M = I.M;
    slice_loop<kWideNTT, 0>(tm.tid, I.n, [&](int i, int, bool valid) {
        float2 v = valid ? r[i] : make_float2(0.f, 0.f);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        }
        if ((threadIdx.x & 31) == 0 && valid) tm.wgw[i >> 5] = v;
    });
    wide_sync(tm.ws);   // warp sums complete
    float* g = tm.cg;   // shared memory of this CTA
    const int wpa = I.agg >> 5, nw = (I.n + 31) >> 5;
    {   // four threads per aggregate (M <= 256), each a quarter of its warp
        // sums (loads in flight together), folded in a fixed order
        const int a = threadIdx.x >> 2, part = threadIdx.x & 3;
        float gx = 0.f, gy = 0.f;
        if (a < M) {
            const int w0 = a * wpa, w1 = min(w0 + wpa, nw);
            for (int w = w0 + part; w < w1; w += 4) {
                const float2 v = __ldcg(tm.wgw + w);
                gx += v.x; gy += v.y;
            }
        }
        gx += __shfl_xor_sync(0xffffffffu, gx, 1); gy += __shfl_xor_sync(0xffffffffu, gy, 1);
        gx += __shfl_xor_sync(0xffffffffu, gx, 2); gy += __shfl_xor_sync(0xffffffffu, gy, 2);
        if (part == 0 && a < M) {
            if (OP == OP_ARAP) { g[a] = gx; g[M + a] = gy; }
            else { g[2 * a] = gx; g[2 * a + 1] = gy; }
        }
    }
    // the products' last pair may read one entry past the end (against a
    // zero matrix entry): it must hold a finite value
    if (threadIdx.x < 4) g[2 * M + threadIdx.x] = 0.f;
    __syncthreads();
    constexpr int G = 8;
    const int S = coarse_stride(M, 2);
    const float* blockf = OP == OP_ARAP ? b.coarse_a + I.co : b.coarse_l + 4 * static_cast<size_t>(I.co);
    const __half* A = reinterpret_cast<const __half*>(blockf);
    const float isc = __ldg(coarse_scale(blockf, (OP == OP_ARAP ? 1 : 2) * M * S));
    const int gl = threadIdx.x & (G - 1);
    const int cpl = ((M + G - 1) / G + 1) & ~1;   // entries per lane, even
    const int c_beg = gl * cpl, c_end = min(c_beg + cpl, M);
    for (int base = static_cast<int>(blockIdx.x) * KB; base < I.n; base += kWideNTT) {
        const int a0 = base / I.agg, a1 = min(M - 1, (min(base + KB, I.n) - 1) / I.agg);
        const int o = a0 + static_cast<int>(threadIdx.x) / G;   // at most KB / 64 + 1 aggregates: one pass
        float au = 0.f, av = 0.f;
        if (o <= a1) {
            for (int c = c_beg; c < c_end; c += 2) {
                if constexpr (OP == OP_ARAP) {
                    const unsigned raw = __ldg(reinterpret_cast<const unsigned*>(A + static_cast<size_t>(o) * S + c));
                    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw));
                    au = fmaf(a.x, g[c], au); au = fmaf(a.y, g[c + 1], au);
                    av = fmaf(a.x, g[M + c], av); av = fmaf(a.y, g[M + c + 1], av);
                } else {
                    const uint2 raw = __ldg(reinterpret_cast<const uint2*>(A + 2 * (static_cast<size_t>(o) * S + c)));
                    const float2 z0 = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
                    const float2 z1 = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
                    const float4 gg = *reinterpret_cast<const float4*>(g + 2 * c);
                    au = fmaf(z0.x, gg.x, au); au = fmaf(-z0.y, gg.y, au);
                    av = fmaf(z0.y, gg.x, av); av = fmaf(z0.x, gg.y, av);
                    au = fmaf(z1.x, gg.z, au); au = fmaf(-z1.y, gg.w, au);
                    av = fmaf(z1.y, gg.z, av); av = fmaf(z1.x, gg.w, av);
                }
            }
        }
#pragma unroll
        for (int k = G / 2; k > 0; k >>= 1) {
            au += __shfl_xor_sync(0xffffffffu, au, k);
            av += __shfl_xor_sync(0xffffffffu, av, k);
        }
        if (gl == 0 && o <= a1) {
            if (OP == OP_ARAP) { tm.cy[o] = au * isc; tm.cy[M + o] = av * isc; }
            else { tm.cy[2 * o] = au * isc; tm.cy[2 * o + 1] = av * isc; }
        }
    }
    __syncthreads();   // y of this CTA's aggregates complete
}

// The last m updates of the ARAP iterate and their images under A (FP32,
// by solver row, most recent first) for the Galerkin start of the next
// global step; m == 0: start from the given x.
constexpr int kStartMax = 4;
// Kept compact (two ints) because it stays live across the refinement loop:
// the vectors are found from the batch (b.hist, or the class-G buffers).
struct StartSpace {
    int m = 0;       // updates in use
    int slots = 0;   // ring slot of update k (most recent first) in bits 2k..2k+1
    __device__ __forceinline__ int slot(int k) const { return (slots >> (2 * k)) & 3; }
};

// Ring slot k of the ARAP update history of island rows [v0, v0 + n): the
// update (part 0) or its image under A (part 1).
__device__ __forceinline__ float2* start_vec(const uva_batch& b, int v0, int k, int part) {
    if (b.hist) return reinterpret_cast<float2*>(b.hist) + static_cast<size_t>(2 * k + part) * b.n + v0;
    float* base = part == 0 ? (k == 0 ? b.p32 : b.d32) : (k == 0 ? b.q32 : b.r32);
    return reinterpret_cast<float2*>(base) + v0;
}

// t = M^+ g for the m x m Gram matrix M (lower triangle, row-major packed:
// M[k(k+1)/2 + l], l <= k) of one column: LDL^T in FP64 that skips a vector
// whose A-norm is below 1e-8 of its own after the earlier ones are removed
// (near-parallel updates); skipped vectors get t = 0.
__device__ __forceinline__ void start_coeffs(int m, const double* M, const double* g, double* t) {
    double L[kStartMax][kStartMax], Dg[kStartMax], y[kStartMax];
    bool on[kStartMax];
#pragma unroll
    for (int k = 0; k < kStartMax; ++k) {
        on[k] = false; Dg[k] = 0.0; y[k] = 0.0; t[k] = 0.0;
#pragma unroll
        for (int l = 0; l < kStartMax; ++l) L[k][l] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < kStartMax; ++k) {
        if (k >= m) break;
        const double mkk = M[k * (k + 1) / 2 + k];
        double v = mkk;
#pragma unroll
        for (int j = 0; j < kStartMax; ++j)
            if (j < k && on[j]) v -= L[k][j] * L[k][j] * Dg[j];
        if (!(mkk > 0.0) || !(v > 1e-8 * mkk) || !isfinite(v)) continue;
        on[k] = true;
        Dg[k] = v;
#pragma unroll
        for (int i = 0; i < kStartMax; ++i) {
            if (i <= k || i >= m) continue;
            double x = M[i * (i + 1) / 2 + k];
#pragma unroll
            for (int j = 0; j < kStartMax; ++j)
                if (j < k && on[j]) x -= L[i][j] * L[k][j] * Dg[j];
            L[i][k] = x / v;
        }
    }
#pragma unroll
    for (int k = 0; k < kStartMax; ++k) {   // L y = g
        if (k >= m || !on[k]) continue;
        double x = g[k];
#pragma unroll
        for (int j = 0; j < kStartMax; ++j)
            if (j < k && on[j]) x -= L[k][j] * y[j];
        y[k] = x;
    }
#pragma unroll
    for (int k = kStartMax - 1; k >= 0; --k) {   // D L^T t = y
        if (k >= m || !on[k]) continue;
        double x = y[k] / Dg[k];
#pragma unroll
        for (int i = 0; i < kStartMax; ++i)
            if (i > k && i < m && on[i]) x -= L[i][k] * t[i];
        t[k] = isfinite(x) ? x : 0.0;
    }
}

// Solves A x = rhs for one island. x64 (global, FP64, by solver row) holds the
// start on entry and the solution on exit. FP64 residual refinement around
// FP32 PCG corrections; NCOL = 2 (ARAP: u and v separately) or 1 (LSCM: one
// vector of 2n unknowns). Returns the inner CG iterations executed.
template <int NTT, int R, Op OP, int NCOL>
__device__ __forceinline__ int refine_solve(const uva_batch& b, const Isl& I, const uva_solve_params& prm, Team<NTT>& tm,
                            const double bb[2], double res_out[2], int& nref, bool& capped,
                            const StartSpace& gsp = StartSpace{}) {
    double2* x64 = reinterpret_cast<double2*>(b.x64) + I.v0;
    const double2* b64 = reinterpret_cast<const double2*>(b.b64) + I.v0;
    // classes with R > 0 always hold the vectors in shared memory; keeping
    // global memory out of their pointers lets the compiler use shared loads
    float2* sp = R > 0 ? tm.sp : reinterpret_cast<float2*>(b.p32) + I.v0;
    float2* sr = R > 0 ? tm.sr : reinterpret_cast<float2*>(b.r32) + I.v0;
    float2* sd = R > 0 ? tm.sd : reinterpret_cast<float2*>(b.d32) + I.v0;
    float2* sq = reinterpret_cast<float2*>(b.q32) + I.v0;   // class G only
    const float wpin32 = static_cast<float>(I.wpin);
    const int tid = tm.tid, n = I.n;
    const bool two_level = NTT > 32 && I.M > 0;
    float2 qreg[R > 0 ? R : 1];
    int total = 0;
    capped = false;
    nref = 0;
    for (int ref = 0;; ++ref) {
        // ---- FP64 residual r = rhs - A x. The shared-memory classes stage x
        // in the p and d buffers first (adjacent: NTT * R FP64 pairs; both are
        // rewritten before the inner CG reads them), so the product gathers
        // from shared memory instead of L2.
        const double2* xr = x64;
        if constexpr (R > 0) {
            double2* xs = reinterpret_cast<double2*>(sp);
            for_rows<NTT, R>(tid, n, [&](int i, int) { xs[i] = x64[i]; });
            tm.sync();
            xr = xs;
        }
        double rr[2] = {0.0, 0.0};
        for_rows<NTT, R>(tid, n, [&](int i, int) {
            double2 r = make_double2(0.0, 0.0);
            if (!is_pinned<OP>(I, i)) {
                const double2 ax = apply64<OP>(b, I, i, xr);
                const double2 rhs = OP == OP_ARAP ? b64[i] : make_double2(0.0, 0.0);
                r = make_double2(rhs.x - ax.x, rhs.y - ax.y);
            }
            sr[i] = make_float2(static_cast<float>(r.x), static_cast<float>(r.y));
            rr[0] += r.x * r.x;
            rr[1] += r.y * r.y;
        });
        team_sum<NTT, 2>(tm, rr, tm.redd);
        ++nref;
        bool done;
        if (NCOL == 2) {
            res_out[0] = sqrt(rr[0] / fmax(bb[0], 1e-300));
            res_out[1] = sqrt(rr[1] / fmax(bb[1], 1e-300));
            done = rr[0] <= prm.tol * prm.tol * fmax(bb[0], 1e-300) && rr[1] <= prm.tol * prm.tol * fmax(bb[1], 1e-300);
        } else {
            const double s = rr[0] + rr[1];
            res_out[0] = res_out[1] = sqrt(s / fmax(bb[0], 1e-300));
            done = s <= prm.tol * prm.tol * fmax(bb[0], 1e-300);
        }
        if (done || ref >= prm.max_refine || !isfinite(rr[0] + rr[1])) {
            if (!done) capped = true;
            break;
        }
        if (ref == 0 && gsp.m > 0) {
            // Galerkin start: x += D t with D the last m updates of the outer
            // iteration and t minimising the energy norm of the error over
            // x + span(D): (D^T A D) t = D^T r, per column. A D is kept from
            // the updates; r -= A D t follows without a product.
            // one pass per update k: d_k . r and d_k . A d_l (l <= k), per column
            constexpr int NM = kStartMax * (kStartMax + 1) / 2;
            double g[2][kStartMax], M[2][NM];
            const int m = gsp.m;
#pragma unroll
            for (int k = 0; k < kStartMax; ++k) {
                if (k >= m) break;
                double acc[2 * (kStartMax + 1)];
#pragma unroll
                for (int e = 0; e < 2 * (kStartMax + 1); ++e) acc[e] = 0.0;
                for_rows<NTT, R>(tid, n, [&](int i, int) {
                    const float2 d = start_vec(b, I.v0, gsp.slot(k), 0)[i], r = sr[i];
                    acc[0] += static_cast<double>(d.x) * r.x;
                    acc[1] += static_cast<double>(d.y) * r.y;
#pragma unroll
                    for (int l = 0; l <= k; ++l) {
                        const float2 a = start_vec(b, I.v0, gsp.slot(l), 1)[i];
                        acc[2 + 2 * l] += static_cast<double>(d.x) * a.x;
                        acc[3 + 2 * l] += static_cast<double>(d.y) * a.y;
                    }
                });
                team_sum<NTT, 2 * (kStartMax + 1)>(tm, acc, tm.redd);
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    g[c][k] = acc[c];
#pragma unroll
                    for (int l = 0; l <= k; ++l) M[c][k * (k + 1) / 2 + l] = acc[2 + 2 * l + c];
                }
            }
            double t[2][kStartMax];
            start_coeffs(m, M[0], g[0], t[0]);
            start_coeffs(m, M[1], g[1], t[1]);
            for_rows<NTT, R>(tid, n, [&](int i, int) {
                double2 x = x64[i];
                float2 r = sr[i];
                double ax = 0.0, ay = 0.0;
#pragma unroll
                for (int k = 0; k < kStartMax; ++k) {
                    if (k >= m) break;
                    const float2 d = start_vec(b, I.v0, gsp.slot(k), 0)[i], a = start_vec(b, I.v0, gsp.slot(k), 1)[i];
                    x.x += t[0][k] * d.x; x.y += t[1][k] * d.y;
                    ax += t[0][k] * a.x; ay += t[1][k] * a.y;
                }
                x64[i] = x;
                r.x -= static_cast<float>(ax); r.y -= static_cast<float>(ay);
                sr[i] = r;
            });
            tm.sync();   // corrected residual complete (the coarse restriction reads all rows)
        }
        if (two_level) coarse_solve<NTT, OP>(b, tm, I, sr);
        // ---- inner FP32 PCG on A d = r, d0 = 0
        float red4[4] = {0.f, 0.f, 0.f, 0.f};   // r.z (2), r.r (2)
        for_rows<NTT, R>(tid, n, [&](int i, int) {
            const float2 r = sr[i];
            const float m = jacobi<OP>(b, I, i);
            float2 z = make_float2(m * r.x, m * r.y);
            if (two_level && !is_pinned<OP>(I, i)) { const float2 y = prolong<NTT, OP>(tm, I, i); z.x += y.x; z.y += y.y; }
            sd[i] = make_float2(0.f, 0.f);
            sp[i] = z;
            red4[0] += r.x * z.x; red4[1] += r.y * z.y;
            red4[2] += r.x * r.x; red4[3] += r.y * r.y;
        });
        team_sum<NTT, 4>(tm, red4, tm.redf);
        float rz[2], thr2[2];
        bool act[2];
        if (NCOL == 2) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                rz[c] = red4[c];
                const float t = fmaxf(static_cast<float>(prm.inner_eta) * sqrtf(red4[2 + c]),
                                      static_cast<float>(0.8 * prm.tol * sqrt(bb[c])));
                thr2[c] = t * t;
                act[c] = red4[2 + c] > thr2[c] && rz[c] > 0.f;
            }
        } else {
            rz[0] = rz[1] = red4[0] + red4[1];
            const float t = fmaxf(static_cast<float>(prm.inner_eta) * sqrtf(red4[2] + red4[3]),
                                  static_cast<float>(0.8 * prm.tol * sqrt(bb[0])));
            thr2[0] = thr2[1] = t * t;
            act[0] = act[1] = (red4[2] + red4[3]) > thr2[0] && rz[0] > 0.f;
        }
        int it = 0;
        float apend[2] = {0.f, 0.f};   // alpha of the last step not yet added to d
        while ((act[0] || act[1]) && it < prm.max_inner) {
            tm.sync();   // p complete
            float pq[2] = {0.f, 0.f};
            if constexpr (R > 0) {
                // whole slices at a time (a warp's lanes are one slice, so the
                // branch and the widths are the same on every lane); rows past
                // the island's end compute zero-weight padding and are dropped
                const int nsl = (n + 31) >> 5;
                for (int j = 0; j < R; j += 2) {
                    const int ia = tid + j * NTT, ib = ia + NTT;
                    if ((ia >> 5) < nsl) {
                        const bool sb = j + 1 < R && (ib >> 5) < nsl;
                        float2 qa, qb;
                        apply32_pair<OP>(b, I, ia, ib, sb, sp, wpin32, qa, qb);
                        qreg[j] = qa;
                        if (ia < n) {
                            const float2 pa = sp[ia];
                            pq[0] += pa.x * qa.x; pq[1] += pa.y * qa.y;
                        }
                        if (j + 1 < R) {
                            qreg[j + 1] = qb;
                            if (sb && ib < n) {
                                const float2 pb = sp[ib];
                                pq[0] += pb.x * qb.x; pq[1] += pb.y * qb.y;
                            }
                        }
                    }
                }
            } else {
                for_rows<NTT, R>(tid, n, [&](int i, int) {
                    float2 q = make_float2(0.f, 0.f);
                    if (!is_pinned<OP>(I, i)) q = apply32<OP>(b, I, i, sp, wpin32);
                    sq[i] = q;
                    const float2 p = sp[i];
                    pq[0] += p.x * q.x; pq[1] += p.y * q.y;
                });
            }
            team_sum<NTT, 2>(tm, pq, tm.redf);
            float alpha[2];
            if (NCOL == 2) {
                alpha[0] = (act[0] && pq[0] > 0.f) ? rz[0] / pq[0] : 0.f;
                alpha[1] = (act[1] && pq[1] > 0.f) ? rz[1] / pq[1] : 0.f;
            } else {
                const float s = pq[0] + pq[1];
                alpha[0] = alpha[1] = (act[0] && s > 0.f) ? rz[0] / s : 0.f;
            }
            // update r (d takes alpha p in the p update below, which reads p anyway)
            for_rows<NTT, R>(tid, n, [&](int i, int j) {
                float2 q;
                if constexpr (R > 0) q = qreg[j]; else q = sq[i];
                float2 r = sr[i];
                r.x = fmaf(-alpha[0], q.x, r.x); r.y = fmaf(-alpha[1], q.y, r.y);
                sr[i] = r;
            });
            apend[0] = alpha[0]; apend[1] = alpha[1];
            if (two_level) {
                if constexpr (NTT != kWideNTT) tm.sync();   // residual complete (class W reads only its own rows)
                coarse_solve<NTT, OP>(b, tm, I, sr);
            }
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            for_rows<NTT, R>(tid, n, [&](int i, int j) {
                const float2 r = sr[i];
                const float m = jacobi<OP>(b, I, i);
                float zx = m * r.x, zy = m * r.y;
                if (two_level && !is_pinned<OP>(I, i)) { const float2 y = prolong<NTT, OP>(tm, I, i); zx += y.x; zy += y.y; }
                // LSCM keeps z for the p update in the A p registers (ARAP: its
                // register budget is tighter, z is recomputed)
                if constexpr (R > 0 && OP == OP_LSCM) qreg[j] = make_float2(zx, zy);
                acc[0] += r.x * zx; acc[1] += r.y * zy;
                acc[2] += r.x * r.x; acc[3] += r.y * r.y;
            });
            team_sum<NTT, 4>(tm, acc, tm.redf);
            ++it;
            float beta[2];
            if (NCOL == 2) {
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    beta[c] = (act[c] && rz[c] > 0.f) ? acc[c] / rz[c] : 0.f;
                    if (act[c]) rz[c] = acc[c];
                    if (acc[2 + c] <= thr2[c] || !(acc[c] > 0.f)) act[c] = false;
                }
            } else {
                const float s = acc[0] + acc[1];
                beta[0] = beta[1] = (act[0] && rz[0] > 0.f) ? s / rz[0] : 0.f;
                rz[0] = rz[1] = s;
                if (acc[2] + acc[3] <= thr2[0] || !(s > 0.f)) act[0] = act[1] = false;
            }
            if (!(act[0] || act[1])) break;
            for_rows<NTT, R>(tid, n, [&](int i, int j) {
                const float2 p = sp[i];
                float2 d = sd[i];
                d.x = fmaf(apend[0], p.x, d.x); d.y = fmaf(apend[1], p.y, d.y);
                sd[i] = d;
                float zx, zy;
                if constexpr (R > 0 && OP == OP_LSCM) {
                    zx = qreg[j].x; zy = qreg[j].y;
                } else {
                    const float2 r = sr[i];
                    const float m = jacobi<OP>(b, I, i);
                    zx = m * r.x; zy = m * r.y;
                    if (two_level && !is_pinned<OP>(I, i)) { const float2 y = prolong<NTT, OP>(tm, I, i); zx += y.x; zy += y.y; }
                }
                sp[i] = make_float2(fmaf(beta[0], p.x, zx), fmaf(beta[1], p.y, zy));
            });
            apend[0] = 0.f; apend[1] = 0.f;
        }
        if (it >= prm.max_inner) capped = true;
        total += it;
        tm.sync();
        for_rows<NTT, R>(tid, n, [&](int i, int) {   // x += d (+ the last step's alpha p)
            const float2 p = sp[i];
            float2 d = sd[i];
            d.x = fmaf(apend[0], p.x, d.x); d.y = fmaf(apend[1], p.y, d.y);
            double2 x = x64[i];
            x.x += static_cast<double>(d.x); x.y += static_cast<double>(d.y);
            x64[i] = x;
        });
        tm.sync();
    }
    return total;
}

// ---- local step (per triangle): closest rotation + corner RHS terms.
// BATCH: engine/gpu.py:165-182. PARAM: engine/param.py:206-233, 457-474.
__device__ __forceinline__ void local_terms(const uva_batch& b, const Isl& I, int f, const double2* U, bool batch,
                                            double& energy, int& flip) {
    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
    const double4 fr = reinterpret_cast<const double4*>(b.frame)[f];
    const double4 wt = reinterpret_cast<const double4*>(b.wtri)[f];
    const double2 u0 = U[I.v0 + tv.x], u1 = U[I.v0 + tv.y], u2 = U[I.v0 + tv.z];
    const double x1 = fr.x, x2 = fr.y, y2 = fr.z;
    const double du1x = u1.x - u0.x, du1y = u1.y - u0.y, du2x = u2.x - u0.x, du2y = u2.y - u0.y;
    double c = 1.0, s = 0.0;
    const double sar = du1x * du2y - du2x * du1y;
    flip = sar <= 0.0 ? 1 : 0;
    energy = 0.0;
    if (batch) {
        if (wt.w != 0.0) {
            const double j00 = du1x / x1, j10 = du1y / x1;
            const double j01 = (du2x - j00 * x2) / y2, j11 = (du2y - j10 * x2) / y2;
            const double ca = j00 + j11, cb = j10 - j01;
            if (isfinite(ca) && isfinite(cb)) {
                const double h = hypot(ca, cb);
                if (h > 0.0) { c = ca / h; s = cb / h; }
            } else if (!isnan(ca) && !isnan(cb)) {
                const double th = atan2(cb, ca);
                c = cos(th); s = sin(th);
            }
        }
        const double sc = static_cast<double>(b.tscale[f]);
        c *= sc; s *= sc;
    } else if (fabs(x1 * y2) >= 1e-300) {
        const double j00 = du1x / x1, j10 = du1y / x1;
        const double j01 = (du2x - j00 * x2) / y2, j11 = (du2y - j10 * x2) / y2;
        double ca = j00 + j11, cb = j10 - j01;
        double h = sqrt(ca * ca + cb * cb);
        if (h < 1e-300) { ca = 1.0; cb = 0.0; h = 1.0; }
        c = ca / h; s = cb / h;
        const double qe = 0.5 * (j00 + j11), qh = 0.5 * (j10 - j01);
        const double rf = 0.5 * (j00 - j11), rg = 0.5 * (j10 + j01);
        const double q = sqrt(qe * qe + qh * qh), r = sqrt(rf * rf + rg * rg);
        energy = fr.w * ((q + r - 1.0) * (q + r - 1.0) + (q - r - 1.0) * (q - r - 1.0));
    }
    // edge k runs corner k+1 -> k+2; frame corners (0,0), (x1,0), (x2,y2)
    const double cxs[3] = {0.0, x1, x2}, cys[3] = {0.0, 0.0, y2};
    const double wk[3] = {wt.x, wt.y, wt.z};
    double vx[3], vy[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int i = (k + 1) % 3, j = (k + 2) % 3;
        const double dx = cxs[i] - cxs[j], dy = cys[i] - cys[j];
        vx[k] = wk[k] * (c * dx - s * dy);
        vy[k] = wk[k] * (s * dx + c * dy);
    }
    double2* rc = reinterpret_cast<double2*>(b.rc);
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
        const int kp = (cc + 2) % 3, km = (cc + 1) % 3;
        rc[3 * f + cc] = make_double2(vx[kp] - vx[km], vy[kp] - vy[km]);
    }
}

// Flip-safe step bound of one triangle (smallest positive root of the
// signed-area quadratic). BATCH: gpu.py:204-227, PARAM: param.py:259-291.
__device__ __forceinline__ double step_bound(const uva_batch& b, const Isl& I, int f, const double2* U, const double2* X,
                                             bool batch) {
    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
    const double2 u0 = U[I.v0 + tv.x], u1 = U[I.v0 + tv.y], u2 = U[I.v0 + tv.z];
    const int* vr = b.vert_row + I.v0;
    const double2 x0 = X[I.v0 + vr[tv.x]], x1 = X[I.v0 + vr[tv.y]], x2 = X[I.v0 + vr[tv.z]];
    const double2 d0 = make_double2(x0.x - u0.x, x0.y - u0.y), d1 = make_double2(x1.x - u1.x, x1.y - u1.y),
                  d2 = make_double2(x2.x - u2.x, x2.y - u2.y);
    const double ux1 = u1.x - u0.x, uy1 = u1.y - u0.y, ux2 = u2.x - u0.x, uy2 = u2.y - u0.y;
    const double dx1 = d1.x - d0.x, dy1 = d1.y - d0.y, dx2 = d2.x - d0.x, dy2 = d2.y - d0.y;
    const double C = ux1 * uy2 - ux2 * uy1;
    const double B = ux1 * dy2 + dx1 * uy2 - ux2 * dy1 - dx2 * uy1;
    const double A = dx1 * dy2 - dx2 * dy1;
    const double big = 1e30;
    if (!(C > 0.0)) return big;
    if (batch) {
        double t = big;
        if (fabs(A) < 1e-30) {
            if (B < 0.0) t = -C / B;
        } else {
            const double disc = B * B - 4.0 * A * C;
            if (disc >= 0.0) {
                const double sq = sqrt(disc);
                const double r1 = (-B - sq) / (2.0 * A), r2 = (-B + sq) / (2.0 * A);
                if (r1 > 0.0) t = fmin(t, r1);
                if (r2 > 0.0) t = fmin(t, r2);
            }
        }
        return isnan(t) ? big : t;
    }
    if (A == 0.0 || fabs(A) < 1e-30 * fmax(fabs(B), 1e-300)) return B < 0.0 ? -C / B : big;
    const double disc = B * B - 4.0 * A * C;
    if (disc < 0.0) return big;
    const double sq = sqrt(disc);
    const double r1 = (-B - sq) / (2.0 * A), r2 = (-B + sq) / (2.0 * A);
    double t = big;
    if (r1 > 0.0 && r1 < t) t = r1;
    if (r2 > 0.0 && r2 < t) t = r2;
    return t;
}

// 1 if triangle f is folded at U: negative signed UV area with a valid frame
// (engine/hier.py:549)
__device__ __forceinline__ int folded_tri(const uva_batch& b, const Isl& I, int f, const double2* U) {
    if (reinterpret_cast<const double4*>(b.wtri)[f].w == 0.0) return 0;
    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
    const double2 a = U[I.v0 + tv.x], c1 = U[I.v0 + tv.y], c2 = U[I.v0 + tv.z];
    return ((c1.x - a.x) * (c2.y - a.y) - (c2.x - a.x) * (c1.y - a.y)) < 0.0 ? 1 : 0;
}

// ---- ARAP outer iterations of one island (gpu.py:230-249 / param.py:379-414)
template <int NTT, int R>
__device__ __forceinline__ void solve_arap(const uva_batch& b, const uva_solve_params& prm, Team<NTT>& tm, const Isl& I) {
    const int tid = tm.tid;
    const bool batch = b.semantics == UVA_SEM_BATCH;
    double2* U = reinterpret_cast<double2*>(b.U);
    double2* x64 = reinterpret_cast<double2*>(b.x64);
    double2* b64 = reinterpret_cast<double2*>(b.b64);
    const double2* rc = reinterpret_cast<const double2*>(b.rc);
    // the status accumulates in global memory (thread 0 only): nothing of it
    // stays live in registers across the CG loops
    uva_island_status* gst = b.status + I.id;
    if (tid == 0) *gst = uva_island_status{};
    bool use_ls = prm.line_search != 0;
    double prev_e = 0.0;
    // CG start of each global step (shared-memory classes): the outer
    // iterates converge about linearly, so the next solution lies close to
    // U_k + span(U_k - U_{k-1}, U_{k-1} - U_{k-2}); refine_solve takes the
    // best point of that plane in the energy norm (StartSpace). The updates
    // and their images under A live in the class-G CG buffers (FP32, by
    // row), which these classes do not use. Only the work of the solve
    // changes, not its tolerance.
    // History ring: slot k holds an update and its image under A. With the
    // batch's history buffer (b.hist) kStartMax slots, else 2 slots in the
    // class-G CG buffers (the no-allocation entry point's case).
    const int depth = b.hist ? kStartMax : 2;
    auto hist_d = [&](int k) -> float2* { return start_vec(b, I.v0, k, 0); };
    auto hist_a = [&](int k) -> float2* { return start_vec(b, I.v0, k, 1); };
    const float wpin32 = static_cast<float>(I.wpin);
    for (int it = 0; it < prm.iters; ++it) {
        double ev[2] = {0.0, 0.0};
        for (int f = I.f0 + tid; f < I.f0 + I.nt; f += NTT) {
            double e; int fl;
            local_terms(b, I, f, U, batch, e, fl);
            ev[0] += e; ev[1] += fl;
        }
        if (!batch) {
            team_sum<NTT, 2>(tm, ev, tm.redd);
            if (it == 0) {
                use_ls = prm.line_search != 0 && ev[1] == 0.0;
                prev_e = ev[0];
            } else if (prm.energy_tol > 0.0 && fabs(prev_e - ev[0]) <= prm.energy_tol * fmax(prev_e, 1e-300)) {
                if (tid == 0) { gst->flags |= UVA_ST_ENERGYSTOP; gst->energy = ev[0]; }
                break;
            } else {
                prev_e = ev[0];
            }
            if (tid == 0) gst->energy = ev[0];
        }
        tm.sync();   // corner terms complete
        double bb[2] = {0.0, 0.0};
        for_rows<NTT, R>(tid, I.n, [&](int i, int) {
            const int v = I.v0 + __ldg(b.row_vert + I.v0 + i);   // vertex of solver row i
            double bx = 0.0, by = 0.0;
            const int pe = __ldg(b.vt_ptr + v + 1);
            for (int p = __ldg(b.vt_ptr + v); p < pe; ++p) {
                const double2 c = rc[__ldg(b.vt + p)];
                bx += c.x; by += c.y;
            }
            const double2 u = U[v];
            if (i == I.pin) { bx += I.wpin * u.x; by += I.wpin * u.y; }
            b64[I.v0 + i] = make_double2(bx, by);
            x64[I.v0 + i] = u;
            bb[0] += bx * bx; bb[1] += by * by;
        });
        team_sum<NTT, 2>(tm, bb, tm.redd);   // also publishes x64 / b64 to the team
        int nref = 0;
        bool capped = false;
        double res[2];
        StartSpace gsp;
        if (R > 0) {
            gsp.m = min(it, depth);
            for (int k = 0; k < gsp.m; ++k) gsp.slots |= ((it - 1 - k) % depth) << (2 * k);   // most recent first
        }
        const int cgi = refine_solve<NTT, R, OP_ARAP, 2>(b, I, prm, tm, bb, res, nref, capped, gsp);
        if (tid == 0) {
            gst->cg_iters += cgi;
            gst->refinements += nref;
            gst->resid[0] = res[0]; gst->resid[1] = res[1];
            if (capped) gst->flags |= UVA_ST_MAXITER;
            gst->outer_iters = it + 1;
        }
        int bad = 0;
        for_rows<NTT, R>(tid, I.n, [&](int i, int) { bad |= finite2(x64[I.v0 + i]) ? 0 : 1; });
        bad = team_or(tm, bad);
        if (bad) {   // non-finite charts keep their layout (gpu.py:235-240)
            if (tid == 0) gst->flags |= UVA_ST_NONFINITE;
            continue;
        }
        double step = 1.0;
        if (use_ls) {
            double tmin = 1e30;
            int folded = 0;
            for (int f = I.f0 + tid; f < I.f0 + I.nt; f += NTT) {
                tmin = fmin(tmin, step_bound(b, I, f, U, x64, batch));
                if (prm.fold_step) folded |= folded_tri(b, I, f, U);
            }
            tmin = team_min(tm, tmin);
            if (prm.fold_step) folded = team_or(tm, folded);   // folded islands: plain ARAP step
            step = folded ? 1.0 : fmin(0.9 * tmin, 1.0);
        }
        if (tid == 0) gst->step = step;
        tm.sync();   // all line-search reads of U done
        for_rows<NTT, R>(tid, I.n, [&](int i, int) {
            const int v = I.v0 + __ldg(b.row_vert + I.v0 + i);
            const double2 u = U[v], x = x64[I.v0 + i];
            const double2 un = use_ls ? make_double2(u.x + (x.x - u.x) * step, u.y + (x.y - u.y) * step) : x;
            U[v] = un;
            if constexpr (R > 0) {   // update history for the next starts
                const float2 d = make_float2(static_cast<float>(un.x - u.x), static_cast<float>(un.y - u.y));
                hist_d(it % depth)[i] = d;
                tm.sp[i] = d;
            }
        });
        tm.sync();   // U and the update complete; also the barrier before the next local step
        if (R > 0 && it + 1 < prm.iters) {   // A d of the update, the solver's own FP32 product
            float2* ha1 = hist_a(it % depth);
            const int nsl = (I.n + 31) >> 5;
            for (int j = 0; j < R; j += 2) {
                const int ia = tid + j * NTT, ib = ia + NTT;
                if ((ia >> 5) < nsl) {
                    const bool sb = j + 1 < R && (ib >> 5) < nsl;
                    float2 qa, qb;
                    apply32_pair<OP_ARAP>(b, I, ia, ib, sb, tm.sp, wpin32, qa, qb);
                    if (ia < I.n) ha1[ia] = qa;
                    if (sb && ib < I.n) ha1[ib] = qb;
                }
            }
        }
    }
}

// ---- LSCM of one island: hard pins p0 -> (0,0), p1 -> (|P[p1]-P[p0]|, 0);
// start from the projection on the mean-normal plane aligned with the pins.
template <int NTT, int R>
__device__ __forceinline__ void solve_lscm(const uva_batch& b, const uva_solve_params& prm, Team<NTT>& tm, const Isl& I) {
    const int tid = tm.tid;
    double2* x64 = reinterpret_cast<double2*>(b.x64);
    double2* U = reinterpret_cast<double2*>(b.U);
    const double* P = b.P;
    uva_island_status st{};
    if (I.p0 < 0 || I.n == 0) {
        st.flags |= UVA_ST_NOBOUNDARY;
        for_rows<NTT, R>(tid, I.n, [&](int i, int) { U[I.v0 + i] = make_double2(0.0, 0.0); });
        if (tid == 0) b.status[I.id] = st;
        tm.sync();
        return;
    }
    double nrm[3] = {0.0, 0.0, 0.0};
    for (int f = I.f0 + tid; f < I.f0 + I.nt; f += NTT) {
        const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
        const double* a = P + 3 * (I.v0 + tv.x);
        const double* c1 = P + 3 * (I.v0 + tv.y);
        const double* c2 = P + 3 * (I.v0 + tv.z);
        const double e1x = c1[0] - a[0], e1y = c1[1] - a[1], e1z = c1[2] - a[2];
        const double e2x = c2[0] - a[0], e2y = c2[1] - a[1], e2z = c2[2] - a[2];
        nrm[0] += e1y * e2z - e1z * e2y;
        nrm[1] += e1z * e2x - e1x * e2z;
        nrm[2] += e1x * e2y - e1y * e2x;
    }
    team_sum<NTT, 3>(tm, nrm, tm.redd);
    const double* pp0 = P + 3 * (I.v0 + b.pins[3 * I.id + 1]);   // pin vertices
    const double* pp1 = P + 3 * (I.v0 + b.pins[3 * I.id + 2]);
    // every thread derives the same basis from the same totals
    const double nl = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
    double nx = 0.0, ny = 0.0, nz = 1.0;
    if (nl > 0.0 && isfinite(nl)) { nx = nrm[0] / nl; ny = nrm[1] / nl; nz = nrm[2] / nl; }
    double ax = pp1[0] - pp0[0], ay = pp1[1] - pp0[1], az = pp1[2] - pp0[2];
    const double dpin = sqrt(ax * ax + ay * ay + az * az);
    const double dn = ax * nx + ay * ny + az * nz;
    ax -= dn * nx; ay -= dn * ny; az -= dn * nz;
    const double al = sqrt(ax * ax + ay * ay + az * az);
    double s = 1.0;
    if (al > 0.0 && isfinite(al)) { s = dpin / al; ax /= al; ay /= al; az /= al; }
    else { ax = 1.0; ay = 0.0; az = 0.0; }
    const double bx = ny * az - nz * ay, by = nz * ax - nx * az, bz = nx * ay - ny * ax;
    for_rows<NTT, R>(tid, I.n, [&](int i, int) {
        const double* pi = P + 3 * (I.v0 + __ldg(b.row_vert + I.v0 + i));
        const double dx = pi[0] - pp0[0], dy = pi[1] - pp0[1], dz = pi[2] - pp0[2];
        double2 x = make_double2(s * (dx * ax + dy * ay + dz * az), s * (dx * bx + dy * by + dz * bz));
        if (i == I.p0) x = make_double2(0.0, 0.0);
        if (i == I.p1) x = make_double2(dpin, 0.0);
        x64[I.v0 + i] = x;
    });
    // ||rhs||^2 of the reduced system: A applied to the pinned values only
    double bb[2] = {0.0, 0.0};
    const int2* cw = reinterpret_cast<const int2*>(b.slot_cw);
    for_rows<NTT, R>(tid, I.n, [&](int i, int) {
        if (is_pinned<OP_LSCM>(I, i)) return;
        int q0, width;
        row_slots(b, I, i, q0, width);
        double rx = 0.0, ry = 0.0;
        for (int k = 0; k < width; ++k) {
            const int q = q0 + 32 * k;
            const int2 sl = __ldg(cw + q);
            if (slot_row(sl.x) != I.p1) continue;   // p0 sits at the origin
            const double w = static_cast<double>(__int_as_float(sl.y));
            const double c = 0.5 * static_cast<double>(slot_c2(sl.x));
            rx -= w * dpin;
            ry -= c * dpin;
        }
        bb[0] += rx * rx + ry * ry;
    });
    team_sum<NTT, 2>(tm, bb, tm.redd);   // also publishes x64 to the team
    int nref = 0;
    bool capped = false;
    st.cg_iters = refine_solve<NTT, R, OP_LSCM, 1>(b, I, prm, tm, bb, st.resid, nref, capped);
    st.refinements = nref;
    st.outer_iters = 1;
    if (capped) st.flags |= UVA_ST_MAXITER;
    int bad = 0;
    for_rows<NTT, R>(tid, I.n, [&](int i, int) {
        const double2 x = x64[I.v0 + i];
        bad |= finite2(x) ? 0 : 1;
        U[I.v0 + __ldg(b.row_vert + I.v0 + i)] = x;
    });
    bad = team_or(tm, bad);
    if (bad) st.flags |= UVA_ST_NONFINITE;
    if (tid == 0) b.status[I.id] = st;
    tm.sync();
}

__device__ __forceinline__ long long global_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned sm_id() {
    unsigned r;
    asm("mov.u32 %0, %%smid;" : "=r"(r));
    return r;
}

// A class-G island that the class-W team solves: above kWideMin vertices,
// and its coarse g and y fit the batch's cpart after the team's header.
// (Its reduction partials and warp sums fit its own block of the batch's
// coarse_work, 4 M^2 doubles; its coarse vectors fit shared memory, M <= 256.)
__device__ __forceinline__ bool wide_island(const uva_batch&, const Isl& I) {
    return I.n > kWideMin && I.agg > 0 && (I.agg & 31) == 0 && I.M >= 64 && I.M <= 256 &&
           kWidePart + (I.n + 31) / 32 <= 4ll * I.M * I.M;
}

template <int NTT, int R, Op OP>
__device__ __forceinline__ void run_class(const uva_batch& b, const uva_solve_params& prm, Team<NTT>& tm, int cls,
                                          bool skip_wide = false) {
    const int lo = b.class_ofs[cls], hi = b.class_ofs[cls + 1];
    if (lo >= hi) return;
    for (;;) {
        int qi;
        if constexpr (NTT == 32) {
            qi = 0;
            if (tm.tid == 0) qi = atomicAdd(b.work + cls, 1);
            qi = __shfl_sync(0xffffffffu, qi, 0);
        } else {
            if (tm.tid == 0) *tm.slot = atomicAdd(b.work + cls, 1);
            tm.sync();
            qi = *tm.slot;
            tm.sync();
        }
        if (lo + qi >= hi) break;
        Isl I = load_island<OP>(b, b.order[lo + qi]);
        if (R == 0 && skip_wide && wide_island(b, I)) continue;   // solved by k_wide
        if (R > 0 && I.n > NTT * R) {   // the team's shared-memory vectors hold NTT * R rows
            if (tm.tid == 0) {
                uva_island_status st{};
                st.flags = UVA_ST_BADCLASS;
                b.status[I.id] = st;
            }
            continue;
        }
        const long long t0 = global_ns();
        // shared-memory copies of the island's slice pointers and Jacobi
        // diagonal (the previous island ended with a team barrier, so the
        // buffers are free)
        // (classes with R > 0 always fit the caches: their islands have at
        // most NTT * R rows; the choice is then fixed at compile time)
        const int nsl1 = ((I.n + 31) >> 5) + 1;
        bool cached = false;
        if (R > 0 || (tm.sc && nsl1 <= tm.sc_cap)) {
            for (int k = tm.tid; k < nsl1; k += NTT) tm.sc[k] = __ldg(b.slice_ptr + I.s0 + k);
            I.sptr = tm.sc;
            cached = true;
        }
        if (R > 0 || (tm.dc && I.n <= tm.dc_cap)) {
            for (int i = tm.tid; i < I.n; i += NTT) tm.dc[i] = __float2bfloat16(jacobi_global<OP>(b, I, i));
            I.dv = tm.dc;
            cached = true;
        }
        if (cached) tm.sync();
        if (OP == OP_ARAP) solve_arap<NTT, R>(b, prm, tm, I);
        else solve_lscm<NTT, R>(b, prm, tm, I);
        if (tm.tid == 0) {   // the same thread wrote the rest of the status
            uva_island_status& st = b.status[I.id];
            st.t_begin = t0;
            st.t_end = global_ns();
            st.sm = static_cast<int32_t>(sm_id());
            st.team = NTT;
        }
    }
}

// The first `nrev` CTAs take the classes in reverse order (warps first):
// the many small islands are latency bound and long-lived for their size,
// so starting some of them at once keeps them out of the launch's tail,
// while the other CTAs start with the largest islands.
// Class W: every class-G island above kWideMin vertices, one after another,
// each by the whole grid (gridDim.x == kWideCtas, cooperative launch).
template <Op OP>
__global__ void __launch_bounds__(KB, 1) k_wide(uva_batch b, uva_solve_params prm) {
    __shared__ double redd[2 * kRedMax * 32];
    __shared__ float redf[2 * kRedMax * 32];
    __shared__ int redi[2 * 32];
    __shared__ __align__(16) float wg[2 * 256 + 8];   // coarse g (all aggregates)
    __shared__ float wy[2 * 256];                      // coarse y (this CTA's aggregates)
    WideScratch* ws = reinterpret_cast<WideScratch*>(b.cpart);
    double* part = b.coarse_work;
    Team<kWideNTT> tm{static_cast<int>(blockIdx.x * KB + threadIdx.x), 0, 0, redd, redf, redi, nullptr,
                      nullptr, nullptr, nullptr, wg, wy, nullptr, 0, nullptr, 0, ws, 0, part,
                      reinterpret_cast<float2*>(part + kWidePart)};
    const int lo = b.class_ofs[0], hi = b.class_ofs[1];
    for (int q = lo; q < hi; ++q) {
        const Isl I = load_island<OP>(b, b.order[q]);
        if (!wide_island(b, I)) continue;
        const long long t0 = global_ns();
        if (OP == OP_ARAP) solve_arap<kWideNTT, 0>(b, prm, tm, I);
        else solve_lscm<kWideNTT, 0>(b, prm, tm, I);
        tm.sync();   // the status below comes after every thread's part
        if (tm.tid == 0) {
            uva_island_status& st = b.status[I.id];
            st.t_begin = t0;
            st.t_end = global_ns();
            st.sm = static_cast<int32_t>(sm_id());
            st.team = kWideNTT;
            if (*reinterpret_cast<volatile int*>(&ws->abort)) st.flags |= UVA_ST_NONFINITE | UVA_ST_MAXITER;
        }
    }
}

template <Op OP>
__global__ void __launch_bounds__(KB, 1) k_islands(uva_batch b, uva_solve_params prm, int nrev, int wide) {
    extern __shared__ __align__(16) float2 dyn[];   // 16-byte aligned: refine_solve stages FP64 pairs here
    __shared__ double redd[2 * kRedMax * 32];
    __shared__ float redf[2 * kRedMax * 32];
    __shared__ int redi[2 * 32];
    __shared__ int slots[8];
    __shared__ __align__(16) float coarse_buf[1024];   // g and y of the coarse level (CTA: 512 each; sub-team: 128 each)
    __shared__ int sc_buf[288];          // slice pointers (CTA: 288; sub-team: 72 each; warp: 9 each)
    __shared__ __nv_bfloat16 dinv_buf[KB * RB];   // Jacobi (CTA: 8192; sub-team: 2048; warp: 256)
    const bool rev = static_cast<int>(blockIdx.x) < nrev;
    auto whole_cta = [&]() {
        Team<KB> tm{static_cast<int>(threadIdx.x), 0, 0, redd, redf, redi, &slots[0], nullptr, nullptr, nullptr,
                    coarse_buf, coarse_buf + 512, sc_buf, 288, dinv_buf, KB * RB};
        run_class<KB, 0, OP>(b, prm, tm, 0, wide != 0);
        tm.sp = dyn; tm.sd = dyn + KB * RB; tm.sr = dyn + 2 * KB * RB;   // sp, sd adjacent (see refine_solve)
        run_class<KB, RB, OP>(b, prm, tm, 1);
    };
    // a sub-team reuses only its own quarter of the buffers, a warp only its
    // own 1/32 (inside its sub-team's quarter)
    auto sub_teams = [&]() {
        const int s = threadIdx.x / SUB;
        float2* base = dyn + s * (3 * SUB * RB);
        Team<SUB> tm{static_cast<int>(threadIdx.x % SUB), 1 + s, 0, redd + s * (2 * kRedMax * 8),
                     redf + s * (2 * kRedMax * 8), redi + s * 16,
                     &slots[1 + s], base, base + 2 * SUB * RB, base + SUB * RB, coarse_buf + 256 * s,
                     coarse_buf + 256 * s + 128, sc_buf + 72 * s, 72,
                     dinv_buf + SUB * RB * s, SUB * RB};
        run_class<SUB, RB, OP>(b, prm, tm, 2);
    };
    auto warps = [&]() {
        const int w = threadIdx.x / 32;
        float2* base = dyn + w * (3 * 32 * RB);
        Team<32> tm{static_cast<int>(threadIdx.x % 32), 0, 0, nullptr, nullptr, nullptr, nullptr,
                    base, base + 2 * 32 * RB, base + 32 * RB, nullptr, nullptr, sc_buf + 9 * w, 9,
                    dinv_buf + 32 * RB * w, 32 * RB};
        run_class<32, RB, OP>(b, prm, tm, 3);
    };
    // one copy of each phase in the code; the order is decided at run time
    for (int step = 0; step < 3; ++step) {
        const int ph = rev ? 2 - step : step;
        if (ph == 0) {
            if (step > 0) __syncthreads();   // every sub-team and warp is done
            whole_cta();
            if (step < 2) __syncthreads();
        } else if (ph == 1) {
            sub_teams();   // its first barrier waits for the team's 8 warps
        } else {
            warps();
        }
    }
}

// In-place Gauss-Jordan inverse of an SPD N x N FP64 matrix (no pivoting
// needed), one CTA. A non-positive pivot (a singular coarse block, e.g. a
// disconnected island) zeroes that row and column of the result.
__device__ void gauss_jordan(double* W, int N, double* colk, double* rowk) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = 0; k < N; ++k) {
        __syncthreads();   // the previous step's updates are complete
        const double piv = W[static_cast<size_t>(k) * N + k];
        const double ip = (piv > 0.0 && isfinite(piv)) ? 1.0 / piv : 0.0;
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            colk[i] = i == k ? 0.0 : W[static_cast<size_t>(i) * N + k];
            rowk[i] = i == k ? ip : W[static_cast<size_t>(k) * N + i] * ip;   // scaled pivot row
        }
        __syncthreads();
        // one warp per row, lanes along the row: row k becomes the scaled
        // pivot row, row i loses colk[i] times it (its column k becomes
        // -colk[i] / piv)
        for (int i = warp; i < N; i += nw) {
            double* Wi = W + static_cast<size_t>(i) * N;
            if (i == k) {
                for (int j = lane; j < N; j += 32) Wi[j] = rowk[j];
                continue;
            }
            const double f = colk[i];
            if (f == 0.0) continue;
            for (int j = lane; j < N; j += 32) Wi[j] = (j == k ? 0.0 : Wi[j]) - f * rowk[j];
        }
    }
    __syncthreads();
}

// The same for a complex Hermitian positive definite M x M matrix (pivots
// real and positive); W row-major (re, im) pairs.
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ void gauss_jordan_c(double2* W, int M, double2* colk, double2* rowk) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = 0; k < M; ++k) {
        __syncthreads();
        const double2 piv = W[static_cast<size_t>(k) * M + k];
        const double den = piv.x * piv.x + piv.y * piv.y;
        const double2 ip = (piv.x > 0.0 && isfinite(den) && den > 0.0) ? make_double2(piv.x / den, -piv.y / den)
                                                                        : make_double2(0.0, 0.0);
        for (int i = threadIdx.x; i < M; i += blockDim.x) {
            colk[i] = i == k ? make_double2(0.0, 0.0) : W[static_cast<size_t>(i) * M + k];
            rowk[i] = i == k ? ip : cmul(W[static_cast<size_t>(k) * M + i], ip);
        }
        __syncthreads();
        for (int i = warp; i < M; i += nw) {
            double2* Wi = W + static_cast<size_t>(i) * M;
            if (i == k) {
                for (int j = lane; j < M; j += 32) Wi[j] = rowk[j];
                continue;
            }
            const double2 f = colk[i];
            if (f.x == 0.0 && f.y == 0.0) continue;
            for (int j = lane; j < M; j += 32) {
                const double2 base = j == k ? make_double2(0.0, 0.0) : Wi[j];
                const double2 d = cmul(f, rowk[j]);
                Wi[j] = make_double2(base.x - d.x, base.y - d.y);
            }
        }
    }
    __syncthreads();
}

// Coarse operators of every island with aggregates: ARAP Ac = P^T A P (with
// the soft pin) and LSCM Hc = P^T H P over free unknowns (u, v per
// aggregate), accumulated from the FP32 slot weights in FP64, inverted,
// stored in FP32. One thread owns each coarse row and adds its terms in
// slot order, so the operators are the same bits on every run. The
// inversion works in shared memory when the block fits (kCoarseSmemN).
// W (FP64, N x N) -> FP16 halves scaled to a largest entry of 1024, in rows
// of stride S (zero padding), plus the inverse scale after them
// (coarse_scale); `red` is >= 32 doubles of shared memory. Whole CTA.
__device__ void store_half_scaled(const double* W, int N, int S, float* block, double* red) {
    const int cnt = N * N;
    double m = 0.0;
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) m = fmax(m, fabs(W[e]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __syncthreads();   // red may still be read by the caller's last step
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    m = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    const double sc = (m > 0.0 && isfinite(m)) ? 1024.0 / m : 1.0;
    __half* h = reinterpret_cast<__half*>(block);
    for (int e = threadIdx.x; e < N * S; e += blockDim.x) {   // rows padded to the stride S
        const int r = e / S, c = e - r * S;
        h[e] = c < N ? __double2half(W[static_cast<size_t>(r) * N + c] * sc) : __double2half(0.0);
    }
    if (threadIdx.x == 0) *const_cast<float*>(coarse_scale(block, N * S)) = static_cast<float>(1.0 / sc);
    __syncthreads();
}

// The LSCM inverse (complex M x M, FP64) -> its Hermitian part as (re, im)
// FP16 pairs scaled to a largest entry of 1024, rows of stride S (zero
// padding), plus the inverse scale after them. Whole CTA.
__device__ void store_complex_scaled(const double2* W, int M, int S, float* block, double* red) {
    auto cre = [&](int o, int c) { return 0.5 * (W[static_cast<size_t>(o) * M + c].x + W[static_cast<size_t>(c) * M + o].x); };
    auto cim = [&](int o, int c) { return 0.5 * (W[static_cast<size_t>(o) * M + c].y - W[static_cast<size_t>(c) * M + o].y); };
    double m = 0.0;
    for (int e = threadIdx.x; e < M * M; e += blockDim.x) {
        const int o = e / M, c = e - o * M;
        m = fmax(m, fmax(fabs(cre(o, c)), fabs(cim(o, c))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __syncthreads();   // red may still be read by the caller's last step
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    m = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    const double sc = (m > 0.0 && isfinite(m)) ? 1024.0 / m : 1.0;
    __half2* h = reinterpret_cast<__half2*>(block);
    for (int e = threadIdx.x; e < M * S; e += blockDim.x) {
        const int o = e / S, c = e - o * S;
        h[e] = c < M ? __floats2half2_rn(static_cast<float>(cre(o, c) * sc), static_cast<float>(cim(o, c) * sc))
                     : __floats2half2_rn(0.f, 0.f);
    }
    if (threadIdx.x == 0) *const_cast<float*>(coarse_scale(block, 2 * M * S)) = static_cast<float>(1.0 / sc);
    __syncthreads();
}

// shared-memory work matrix: complex LSCM operators up to 118 x 118, real
// ARAP operators up to 166 x 166 (larger ones work in b.coarse_work)
constexpr int kCoarseSmemC = 118;
constexpr size_t kCoarseSmem = sizeof(double2) * kCoarseSmemC * kCoarseSmemC;   // 222,784 bytes
constexpr int kCoarseSmemN = 166;   // sizeof(double) * 166 * 166 <= kCoarseSmem
static_assert(sizeof(double) * kCoarseSmemN * kCoarseSmemN <= kCoarseSmem, "real work matrix must fit");

// One CTA per island of b.order[first, first + count): NT = 1024 with
// kCoarseSmem of dynamic shared memory for the whole-CTA classes (one CTA
// per SM), NT = 256 with kCoarseSmallSmem for the sub-team classes, whose
// operators are at most 32 x 32 (several CTAs per SM).
constexpr int kCoarseSmallM = 32;
constexpr size_t kCoarseSmallSmem = sizeof(double2) * kCoarseSmallM * kCoarseSmallM;   // 16 KB

template <int NT>
__global__ void __launch_bounds__(NT) k_coarse(uva_batch b, int first, int count) {
    extern __shared__ __align__(16) double wsm[];
    __shared__ double2 colk2[256], rowk2[256];   // pivot column / row (complex; the real pass uses 256 doubles of each)
    double* colk = reinterpret_cast<double*>(colk2);
    double* rowk = reinterpret_cast<double*>(rowk2);
    if (static_cast<int>(blockIdx.x) >= count) return;
    const int isl = b.order[first + blockIdx.x];   // largest islands first (b.order is by size)
    const int agg = b.agg_rows[isl];
    if (agg <= 0) return;
    const int v0 = b.vofs[isl], n = b.vofs[isl + 1] - v0, s0 = b.sofs[isl];
    const int M = (n + agg - 1) / agg;
    const int co = b.cofs[isl];
    const int2* cw = reinterpret_cast<const int2*>(b.slot_cw);
    auto row_slots_l = [&](int r, int& q0, int& width) {
        const int s = s0 + (r >> 5);
        const int p0s = __ldg(b.slice_ptr + s), p1s = __ldg(b.slice_ptr + s + 1);
        q0 = p0s + (r & 31);
        width = (p1s - p0s) >> 5;
    };
    constexpr int kRealN = NT == 1024 ? kCoarseSmemN : 45;            // 8 N^2 bytes of shared memory
    constexpr int kCplxN = NT == 1024 ? kCoarseSmemC : kCoarseSmallM;  // 16 N^2 bytes
    auto work = [&](int N) { return N <= kRealN ? wsm : b.coarse_work + 4 * static_cast<size_t>(co); };
    // ---- ARAP
    double* W = work(M);
    for (int e = threadIdx.x; e < M * M; e += blockDim.x) W[e] = 0.0;
    __syncthreads();
    const int pin_agg = b.vert_row[v0 + b.pins[3 * isl]] / agg;
    for (int a = threadIdx.x; a < M; a += blockDim.x) {
        double* Wa = W + static_cast<size_t>(a) * M;
        double dsum = 0.0;
        for (int r = a * agg; r < min(n, (a + 1) * agg); ++r) {
            int q0, width;
            row_slots_l(r, q0, width);
            for (int k = 0; k < width; k += 4) {   // widths are multiples of 4
                int2 s4[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) s4[u] = __ldg(cw + q0 + 32 * (k + u));
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const double w = static_cast<double>(__int_as_float(s4[u].y));
                    if (w == 0.0) continue;
                    const int c = slot_row(s4[u].x) / agg;
                    if (c != a) { dsum += w; Wa[c] -= w; }
                }
            }
        }
        if (a == pin_agg) dsum += b.wpin[isl];
        Wa[a] += dsum;
    }
    gauss_jordan(W, M, colk, rowk);
    store_half_scaled(W, M, coarse_stride(M, 2), b.coarse_a + co, colk);
    __syncthreads();
    // ---- LSCM (free unknowns only; the pins are fixed)
    const int pv0 = b.pins[3 * isl + 1], pv1 = b.pins[3 * isl + 2];
    if (pv0 < 0 || pv1 < 0) return;
    const int p0 = b.vert_row[v0 + pv0], p1 = b.vert_row[v0 + pv1];
    // the (u, v) operator per aggregate is the real form [[P, -Q], [Q, P]] of
    // the complex Hermitian Hc = P + i Q: assembled and inverted as complex
    double2* Wc = M <= kCplxN ? reinterpret_cast<double2*>(wsm)
                              : reinterpret_cast<double2*>(b.coarse_work + 4 * static_cast<size_t>(co));
    for (int e = threadIdx.x; e < M * M; e += blockDim.x) Wc[e] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int a = threadIdx.x; a < M; a += blockDim.x) {
        double2* Wa = Wc + static_cast<size_t>(a) * M;
        double dsum = 0.0, qaa = 0.0;
        for (int r = a * agg; r < min(n, (a + 1) * agg); ++r) {
            if (r == p0 || r == p1) continue;
            int q0, width;
            row_slots_l(r, q0, width);
            for (int k = 0; k < width; k += 4) {
                int2 s4[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) s4[u] = __ldg(cw + q0 + 32 * (k + u));
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int2 sl = s4[u];
                    const double w = static_cast<double>(__int_as_float(sl.y));
                    const double cc = 0.5 * static_cast<double>(slot_c2(sl.x));
                    if (w == 0.0 && cc == 0.0) continue;
                    const int col = slot_row(sl.x);
                    const bool pinned_nb = col == p0 || col == p1;   // no coarse coupling
                    const int c = col / agg;
                    if (pinned_nb || c != a) dsum += w;
                    if (pinned_nb) continue;
                    if (c != a) Wa[c].x -= w;
                    if (cc != 0.0) {
                        if (c == a) qaa -= cc;
                        else Wa[c].y -= cc;
                    }
                }
            }
        }
        Wa[a].x += dsum;
        Wa[a].y += qaa;
    }
    gauss_jordan_c(Wc, M, colk2, rowk2);
    store_complex_scaled(Wc, M, coarse_stride(M, 2), b.coarse_l + 4 * static_cast<size_t>(co), colk);
}

cudaError_t ensure_coarse_attr() {
    static std::mutex mu;
    static std::vector<char> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (static_cast<int>(done.size()) <= dev) done.resize(dev + 1, 0);
    if (done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(k_coarse<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kCoarseSmem));
    if (e == cudaSuccess) done[dev] = 1;
    return e;
}

int sm_count() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    if (static_cast<int>(cache.size()) <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 148;
    }
    return cache[dev];
}

// The island kernel's shared-memory opt-in, once per device and operator (so
// that a launch inside a stream capture issues no attribute call).
template <Op OP>
cudaError_t ensure_islands_attr() {
    static std::mutex mu;
    static std::vector<char> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (static_cast<int>(done.size()) <= dev) done.resize(dev + 1, 0);
    if (done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(k_islands<OP>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kDynSmem));
    if (e == cudaSuccess) done[dev] = 1;
    return e;
}

// The batch's inputs (topology, geometry, coarse operators), without the
// caller's solver scratch.
bool check_batch_inputs(const uva_batch* b) {
    return b && b->nc >= 0 && b->n >= 0 && b->t >= 0 &&
           (b->nc == 0 || (b->vofs && b->tofs && b->sofs && b->order && b->slot_cw && b->row_vert &&
                           b->vert_row && b->agg_rows && b->cofs && b->coarse_a && b->coarse_l));
}

bool check_batch(const uva_batch* b) {
    return check_batch_inputs(b) && (b->nc == 0 || (b->work && b->cpart));
}

bool check_classes(const uva_batch* b) {
    if (b->class_ofs[0] != 0 || b->class_ofs[4] != b->nc) return false;
    for (int c = 0; c < 4; ++c)
        if (b->class_ofs[c + 1] < b->class_ofs[c]) return false;
    return true;
}

template <Op OP>
int launch_islands(const uva_batch* b, const uva_solve_params* prm, cudaStream_t s) {
    if (!check_classes(b)) {
        uva_set_error("uva_arap/uva_lscm: class_ofs must be 0 <= ... <= nc, non-decreasing");
        return UVA_E_ARG;
    }
    cudaError_t e = ensure_islands_attr<OP>();
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_islands/cudaFuncSetAttribute");
    e = cudaMemsetAsync(b->work, 0, sizeof(int32_t) * 4, s);
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_islands/memset");
    const int big = b->class_ofs[2];                        // islands that take a whole CTA
    const int small = b->class_ofs[4] - b->class_ofs[2];    // islands for sub-teams / warps
    const int want = big + (small + 3) / 4;
    const int grid = std::max(1, std::min(sm_count(), want));
    // reverse-order CTAs: one per 128 warp-class islands, at most a quarter
    const int nwarp = b->class_ofs[4] - b->class_ofs[3];
    int nrev = big > 0 ? std::min(grid / 4, (nwarp + 127) / 128) : 0;
    if (prm->rev_ctas != 0) nrev = std::max(0, std::min(grid, prm->rev_ctas));
    // class W first, on the whole GPU (cooperative: every CTA resident)
    int wide = 0;
    if (b->class_ofs[1] > b->class_ofs[0] && b->cpart && b->coarse_work && sm_count() >= kWideCtas) {
        e = cudaMemsetAsync(b->cpart, 0, kWideHdr, s);
        if (e != cudaSuccess) return uva_cuda_status(e, "uva_islands/memset");
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(kWideCtas);
        cfg.blockDim = dim3(KB);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, k_wide<OP>, *b, *prm);
        if (e != cudaSuccess) return uva_cuda_status(e, "uva_islands/k_wide");
        wide = 1;
    }
    k_islands<OP><<<grid, KB, kDynSmem, s>>>(*b, *prm, nrev, wide);
    UVA_CHECK_LAUNCH(OP == OP_ARAP ? "uva_arap" : "uva_lscm");
    return UVA_OK;
}

// ------------------------------------------------------------------ SLIM
// Symmetric-Dirichlet SLIM iterations (engine/param.py:206-256 mode 1,
// 341-377 and 415-454), one 1024-thread CTA per island, FP64 throughout.
//
// Local step per triangle: J = U M^-1 in the triangle's frame, its signed
// singular values s1 = q + r, s2 = q - r and left singular vector u1
// (closed form), SLIM weights w_k = sqrt((|s| - |s|^-3) / (|s| - 1)) (2 at
// |s| ~ 1), W = U diag(w) U^T and the closest rotation R. Global step: the
// reference builds A (4t x 2n) with rows sqrt(area) W (J - R) and solves the
// normal equations (A^T A + reg I) x = A^T b + reg x0, reg = 1e-12 sum(area).
// Here A^T A is applied without forming it: per triangle
//   (A^T A x)_{r,k} = area (W^2 J(x) G)_{r,k},   (A^T b)_{r,k} = area (W^2 R G)_{r,k},
// with G the 2x3 gradient of the linear interpolant; each vertex gathers its
// incident corners (vt), so no atomics and a fixed summation order. CG with
// the diagonal of A^T A (the reference's Jacobi) from x0 = U; the reference
// solves exactly (splu) when 2n <= 220,000 and runs CG to rtol 1e-6, at most
// 500 iterations, above: prm.inner_eta and prm.max_inner carry that choice.
// Then the flip-safe step min(1, 0.9 tmax) and halving while the symmetric
// Dirichlet energy is not below the previous one (at most 12 times).
struct SlimTri {
    double x1, x2, y2, area;
    double g0[3], g1[3];   // rows of G (gradient of the linear interpolant)
    bool live;
};

__device__ __forceinline__ SlimTri slim_tri(const uva_batch& b, int f) {
    const double4 fr = reinterpret_cast<const double4*>(b.frame)[f];
    SlimTri t;
    t.x1 = fr.x; t.x2 = fr.y; t.y2 = fr.z; t.area = fr.w;
    t.live = fabs(t.x1 * t.y2) >= 1e-300;
    const double ix1 = 1.0 / t.x1, iy2 = 1.0 / t.y2;
    t.g0[0] = -ix1; t.g0[1] = ix1; t.g0[2] = 0.0;
    t.g1[0] = (-1.0 + t.x2 * ix1) * iy2; t.g1[1] = (-t.x2 * ix1) * iy2; t.g1[2] = iy2;
    return t;
}

// J (rows u, v; columns c) of corner values q_u, q_v
__device__ __forceinline__ void slim_jac(const SlimTri& t, const double2 q[3], double J[2][2]) {
    J[0][0] = t.g0[0] * q[0].x + t.g0[1] * q[1].x + t.g0[2] * q[2].x;
    J[0][1] = t.g1[0] * q[0].x + t.g1[1] * q[1].x + t.g1[2] * q[2].x;
    J[1][0] = t.g0[0] * q[0].y + t.g0[1] * q[1].y + t.g0[2] * q[2].y;
    J[1][1] = t.g1[0] * q[0].y + t.g1[1] * q[1].y + t.g1[2] * q[2].y;
}

// symmetric Dirichlet energy of one triangle, inf if inverted (param.py:310-318)
__device__ __forceinline__ double sd_energy_tri(const SlimTri& t, const double2 q[3]) {
    if (!t.live) return 0.0;
    const double j00 = (q[1].x - q[0].x) / t.x1, j10 = (q[1].y - q[0].y) / t.x1;
    const double j01 = ((q[2].x - q[0].x) - j00 * t.x2) / t.y2, j11 = ((q[2].y - q[0].y) - j10 * t.x2) / t.y2;
    const double dj = j00 * j11 - j01 * j10;
    if (dj <= 0.0) return INFINITY;
    const double fro = j00 * j00 + j01 * j01 + j10 * j10 + j11 * j11;
    return t.area * (fro + fro / (dj * dj) - 4.0);
}

// local step of one triangle: S = W^2 (symmetric: s00, s01, s11) and the
// closest rotation R = [[rc, -rs], [rs, rc]]
__device__ __forceinline__ void slim_local(const SlimTri& t, const double2 q[3], double S[3], double& rc, double& rs) {
    if (!t.live) { S[0] = 1.0; S[1] = 0.0; S[2] = 1.0; rc = 1.0; rs = 0.0; return; }
    const double j00 = (q[1].x - q[0].x) / t.x1, j10 = (q[1].y - q[0].y) / t.x1;
    const double j01 = ((q[2].x - q[0].x) - j00 * t.x2) / t.y2, j11 = ((q[2].y - q[0].y) - j10 * t.x2) / t.y2;
    double w00, w01, w11;
    slim_2x2(j00, j01, j10, j11, rc, rs, w00, w01, w11);
    S[0] = w00 * w00 + w01 * w01;
    S[1] = w00 * w01 + w01 * w11;
    S[2] = w01 * w01 + w11 * w11;
}

template <Op OP>
__global__ void __launch_bounds__(KB, 1) k_slim(uva_batch b, uva_solve_params prm, double* scratch) {
    __shared__ double redd[2 * kRedMax * 32];
    __shared__ float redf[2 * kRedMax * 32];
    __shared__ int redi[2 * 32];
    Team<KB> tm{static_cast<int>(threadIdx.x), 0, 0, redd, redf, redi, nullptr, nullptr, nullptr, nullptr,
                nullptr, nullptr, nullptr, 0, nullptr, 0};
    const int tid = tm.tid;
    double2* U = reinterpret_cast<double2*>(b.U);
    double2* X = reinterpret_cast<double2*>(b.x64);   // trial solution (by vertex)
    double2* Bv = reinterpret_cast<double2*>(b.b64);  // right-hand side
    double* Sbuf = scratch;                               // 3t: W^2 per triangle
    double2* Rv = reinterpret_cast<double2*>(scratch + ((3 * static_cast<size_t>(b.t) + 1) & ~static_cast<size_t>(1)));   // residual
    double2* Pv = Rv + b.n;
    double2* Qv = Pv + b.n;
    double2* RCS = Qv + b.n;                              // t: rotation (c, s) per triangle
    for (int isl = blockIdx.x; isl < b.nc; isl += gridDim.x) {
        const int v0 = b.vofs[isl], n = b.vofs[isl + 1] - v0, f0 = b.tofs[isl], nt = b.tofs[isl + 1] - f0;
        uva_island_status st{};
        // energy at the start; a non-finite start is returned unchanged (param.py:418-419)
        double acc[2] = {0.0, 0.0};
        for (int f = f0 + tid; f < f0 + nt; f += KB) {
            const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
            const double2 q[3] = {U[v0 + tv.x], U[v0 + tv.y], U[v0 + tv.z]};
            const SlimTri t = slim_tri(b, f);
            acc[0] += sd_energy_tri(t, q);
            acc[1] += t.area;
        }
        team_sum<KB, 2>(tm, acc, tm.redd);
        double prev = acc[0];
        const double reg = 1e-12 * acc[1];
        st.energy = prev;
        if (!isfinite(prev)) {
            st.flags |= UVA_ST_NONFINITE;
            if (tid == 0) b.status[isl] = st;
            __syncthreads();
            continue;
        }
        for (int it = 0; it < prm.iters; ++it) {
            // ---- local step
            for (int f = f0 + tid; f < f0 + nt; f += KB) {
                const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
                const double2 q[3] = {U[v0 + tv.x], U[v0 + tv.y], U[v0 + tv.z]};
                double S[3], rc, rs;
                slim_local(slim_tri(b, f), q, S, rc, rs);
                Sbuf[3 * f] = S[0]; Sbuf[3 * f + 1] = S[1]; Sbuf[3 * f + 2] = S[2];
                RCS[f] = make_double2(rc, rs);
            }
            __syncthreads();
            // ---- right-hand side A^T b + reg x0, Jacobi diagonal, r0 = rhs - M x0
            // per vertex over its incident corners (vt), in corner order
            auto apply = [&](int v, const double2* x, bool with_rhs, double2& mx, double2& rhs, double2& dg) {
                mx = make_double2(0.0, 0.0); rhs = make_double2(0.0, 0.0); dg = make_double2(0.0, 0.0);
                const int pe = __ldg(b.vt_ptr + v + 1);
                for (int pq = __ldg(b.vt_ptr + v); pq < pe; ++pq) {
                    const int c = __ldg(b.vt + pq);
                    const int f = c / 3, k = c - 3 * f;
                    const SlimTri t = slim_tri(b, f);
                    if (!t.live) continue;
                    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
                    const double2 q[3] = {x[v0 + tv.x], x[v0 + tv.y], x[v0 + tv.z]};
                    double J[2][2];
                    slim_jac(t, q, J);
                    const double s00 = Sbuf[3 * f], s01 = Sbuf[3 * f + 1], s11 = Sbuf[3 * f + 2];
                    const double gk0 = t.g0[k], gk1 = t.g1[k];
                    // (S J G)_{r,k} = sum_c (S J)_{r,c} G_{c,k}
                    const double sj00 = s00 * J[0][0] + s01 * J[1][0], sj01 = s00 * J[0][1] + s01 * J[1][1];
                    const double sj10 = s01 * J[0][0] + s11 * J[1][0], sj11 = s01 * J[0][1] + s11 * J[1][1];
                    mx.x += t.area * (sj00 * gk0 + sj01 * gk1);
                    mx.y += t.area * (sj10 * gk0 + sj11 * gk1);
                    if (with_rhs) {
                        const double2 r = RCS[f];   // R = [[c, -s], [s, c]]
                        const double sr00 = s00 * r.x + s01 * r.y, sr01 = -s00 * r.y + s01 * r.x;
                        const double sr10 = s01 * r.x + s11 * r.y, sr11 = -s01 * r.y + s11 * r.x;
                        rhs.x += t.area * (sr00 * gk0 + sr01 * gk1);
                        rhs.y += t.area * (sr10 * gk0 + sr11 * gk1);
                        const double gg = gk0 * gk0 + gk1 * gk1;
                        dg.x += t.area * s00 * gg;
                        dg.y += t.area * s11 * gg;
                    }
                }
                mx.x += reg * x[v].x; mx.y += reg * x[v].y;
            };
            double bb[2] = {0.0, 0.0};   // ||rhs||^2, ||r0||^2
            double rz = 0.0;
            for (int i = tid; i < n; i += KB) {
                const int v = v0 + i;
                double2 mx, rhs, dg;
                apply(v, U, true, mx, rhs, dg);
                rhs.x += reg * U[v].x; rhs.y += reg * U[v].y;
                dg.x += reg; dg.y += reg;
                Bv[v] = make_double2(1.0 / dg.x, 1.0 / dg.y);   // Jacobi (inverse diagonal)
                const double2 r = make_double2(rhs.x - mx.x, rhs.y - mx.y);
                Rv[v] = r;
                X[v] = U[v];
                const double2 z = make_double2(r.x / dg.x, r.y / dg.y);
                Pv[v] = z;
                bb[0] += rhs.x * rhs.x + rhs.y * rhs.y;
                bb[1] += r.x * r.x + r.y * r.y;
                rz += r.x * z.x + r.y * z.y;
            }
            double tot[3] = {bb[0], bb[1], rz};
            team_sum<KB, 3>(tm, tot, tm.redd);
            const double thr2 = prm.inner_eta * prm.inner_eta * tot[0];
            double rr = tot[1];
            rz = tot[2];
            int cg = 0;
            while (rr >= thr2 && cg < prm.max_inner && rz > 0.0) {   // scipy: stop once ||r|| < rtol ||b||
                double pq = 0.0;
                for (int i = tid; i < n; i += KB) {
                    const int v = v0 + i;
                    double2 mx, rhs, dg;
                    apply(v, Pv, false, mx, rhs, dg);
                    Qv[v] = mx;
                    pq += Pv[v].x * mx.x + Pv[v].y * mx.y;
                }
                double t1[1] = {pq};
                team_sum<KB, 1>(tm, t1, tm.redd);
                if (!(t1[0] > 0.0)) break;
                const double alpha = rz / t1[0];
                double t2[2] = {0.0, 0.0};
                for (int i = tid; i < n; i += KB) {
                    const int v = v0 + i;
                    const double2 p = Pv[v], q = Qv[v], m = Bv[v];
                    double2 x = X[v], r = Rv[v];
                    x.x += alpha * p.x; x.y += alpha * p.y;
                    r.x -= alpha * q.x; r.y -= alpha * q.y;
                    X[v] = x; Rv[v] = r;
                    t2[0] += r.x * r.x + r.y * r.y;
                    t2[1] += r.x * r.x * m.x + r.y * r.y * m.y;
                }
                team_sum<KB, 2>(tm, t2, tm.redd);
                ++cg;
                rr = t2[0];
                if (rr < thr2) break;
                const double beta = t2[1] / rz;
                rz = t2[1];
                for (int i = tid; i < n; i += KB) {
                    const int v = v0 + i;
                    const double2 r = Rv[v], m = Bv[v], p = Pv[v];
                    Pv[v] = make_double2(r.x * m.x + beta * p.x, r.y * m.y + beta * p.y);
                }
                __syncthreads();
            }
            st.cg_iters += cg;
            st.resid[0] = st.resid[1] = sqrt(rr / fmax(tot[0], 1e-300));
            if (cg >= prm.max_inner) st.flags |= UVA_ST_MAXITER;
            __syncthreads();
            // ---- flip-safe step and energy backtracking (param.py:436-454)
            double tmin = 1e30;
            for (int f = f0 + tid; f < f0 + nt; f += KB) {
                const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
                const double2 u0 = U[v0 + tv.x], u1 = U[v0 + tv.y], u2 = U[v0 + tv.z];
                const double2 a0 = X[v0 + tv.x], a1 = X[v0 + tv.y], a2 = X[v0 + tv.z];
                const double ux1 = u1.x - u0.x, uy1 = u1.y - u0.y, ux2 = u2.x - u0.x, uy2 = u2.y - u0.y;
                const double dx1 = (a1.x - u1.x) - (a0.x - u0.x), dy1 = (a1.y - u1.y) - (a0.y - u0.y);
                const double dx2 = (a2.x - u2.x) - (a0.x - u0.x), dy2 = (a2.y - u2.y) - (a0.y - u0.y);
                const double C = ux1 * uy2 - ux2 * uy1;
                const double B = ux1 * dy2 + dx1 * uy2 - ux2 * dy1 - dx2 * uy1;
                const double A = dx1 * dy2 - dx2 * dy1;
                if (!(C > 0.0)) continue;
                if (A == 0.0 || fabs(A) < 1e-30 * fmax(fabs(B), 1e-300)) {
                    if (B < 0.0) tmin = fmin(tmin, -C / B);
                    continue;
                }
                const double disc = B * B - 4.0 * A * C;
                if (disc < 0.0) continue;
                const double sq = sqrt(disc);
                const double r1 = (-B - sq) / (2.0 * A), r2 = (-B + sq) / (2.0 * A);
                if (r1 > 0.0) tmin = fmin(tmin, r1);
                if (r2 > 0.0) tmin = fmin(tmin, r2);
            }
            tmin = team_min(tm, tmin);
            double step = fmin(1.0, 0.9 * tmin);
            double e = 0.0;
            for (int k = 0; k <= 12; ++k) {
                double ev[1] = {0.0};
                for (int f = f0 + tid; f < f0 + nt; f += KB) {
                    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
                    const int vv[3] = {v0 + tv.x, v0 + tv.y, v0 + tv.z};
                    double2 q[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        q[c] = make_double2(U[vv[c]].x + step * (X[vv[c]].x - U[vv[c]].x),
                                            U[vv[c]].y + step * (X[vv[c]].y - U[vv[c]].y));
                    ev[0] += sd_energy_tri(slim_tri(b, f), q);
                }
                team_sum<KB, 1>(tm, ev, tm.redd);
                e = ev[0];
                if ((isfinite(e) && e <= prev) || k == 12) break;
                step *= 0.5;
            }
            st.outer_iters = it + 1;
            if (!isfinite(e) || e > prev) break;   // no acceptable step: keep U
            for (int i = tid; i < n; i += KB) {
                const int v = v0 + i;
                const double2 u = U[v], x = X[v];
                U[v] = make_double2(u.x + step * (x.x - u.x), u.y + step * (x.y - u.y));
            }
            __syncthreads();
            st.step = step;
            const bool stop = fabs(prev - e) <= prm.energy_tol * prev;
            prev = e;
            st.energy = e;
            if (stop) break;
        }
        if (tid == 0) b.status[isl] = st;
        __syncthreads();
    }
}

}  // namespace

extern "C" int uva_batch_setup(uva_batch* b, void* stream) {
    if (!check_batch(b)) { uva_set_error("uva_batch_setup: bad batch"); return UVA_E_ARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (b->nc == 0) return UVA_OK;
    // scratch: per-island max |w| (nc doubles) in b64 and the vertex -> island
    // map (n ints) in x64; both are sized max(n, nc) * 2 doubles
    double* wmax = b->b64;
    int32_t* vert_isl = reinterpret_cast<int32_t*>(b->x64);
    cudaMemsetAsync(b->wedge, 0, sizeof(double) * static_cast<size_t>(b->E), s);
    cudaMemsetAsync(wmax, 0, sizeof(double) * static_cast<size_t>(b->nc), s);
    if (b->t > 0) k_frames<<<(b->t + 255) / 256, 256, 0, s>>>(*b, wmax);
    UVA_CHECK_LAUNCH("uva_batch_setup/frames");
    k_wpin<<<1, 1024, 0, s>>>(*b, wmax);
    UVA_CHECK_LAUNCH("uva_batch_setup/wpin");
    k_vert_isl<<<b->nc, 256, 0, s>>>(b->vofs, b->nc, vert_isl);
    if (b->n > 0) k_rows<<<(b->n + 255) / 256, 256, 0, s>>>(*b, vert_isl);
    UVA_CHECK_LAUNCH("uva_batch_setup/rows");
    k_far_pair<<<(b->nc + 127) / 128, 128, 0, s>>>(*b);
    UVA_CHECK_LAUNCH("uva_batch_setup/pins");
    if (b->coarse_a && b->coarse_l && b->coarse_work) {
        const cudaError_t e = ensure_coarse_attr();   // 128 KB of dynamic shared memory
        if (e != cudaSuccess) return uva_cuda_status(e, "uva_batch_setup/coarse attribute");
        // whole-CTA classes (W, G, A: islands above 2048 vertices), then the
        // smaller ones (aggregates of 64 rows: at most 32 x 32 operators)
        const int big = std::min(std::max(b->class_ofs[2], 0), b->nc), rest = b->nc - big;
        if (big > 0) k_coarse<1024><<<big, 1024, kCoarseSmem, s>>>(*b, 0, big);
        if (rest > 0) k_coarse<256><<<rest, 256, kCoarseSmallSmem, s>>>(*b, big, rest);
        UVA_CHECK_LAUNCH("uva_batch_setup/coarse");
    }
    return UVA_OK;
}

extern "C" int uva_arap(uva_batch* b, const uva_solve_params* prm, void* stream) {
    if (!check_batch(b) || !prm) { uva_set_error("uva_arap: bad arguments"); return UVA_E_ARG; }
    if (b->nc == 0 || prm->iters <= 0) return UVA_OK;
    return launch_islands<OP_ARAP>(b, prm, static_cast<cudaStream_t>(stream));
}

extern "C" int uva_slim_scratch_bytes(const uva_batch* b, int64_t* bytes) {
    if (!b || !bytes) { uva_set_error("uva_slim_scratch_bytes: null argument"); return UVA_E_ARG; }
    *bytes = static_cast<int64_t>(sizeof(double)) *
             (3 * static_cast<int64_t>(b->t) + 1 + 6 * static_cast<int64_t>(b->n) + 2 * static_cast<int64_t>(b->t));
    return UVA_OK;
}

extern "C" int uva_slim(uva_batch* b, const uva_solve_params* prm, double* scratch, void* stream) {
    if (!check_batch(b) || !prm || !scratch || !b->status || b->semantics != UVA_SEM_PARAM) {
        uva_set_error("uva_slim: bad arguments (scratch, status and PARAM semantics are required)");
        return UVA_E_ARG;
    }
    if (b->nc == 0 || prm->iters <= 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_slim<OP_ARAP><<<std::min(sm_count(), b->nc), KB, 0, s>>>(*b, *prm, scratch);
    UVA_CHECK_LAUNCH("uva_slim");
    return UVA_OK;
}

extern "C" int uva_lscm(uva_batch* b, const uva_solve_params* prm, void* stream) {
    if (!check_batch(b) || !prm) { uva_set_error("uva_lscm: bad arguments"); return UVA_E_ARG; }
    if (b->nc == 0) return UVA_OK;
    return launch_islands<OP_LSCM>(b, prm, static_cast<cudaStream_t>(stream));
}

// ------------------------------------------------------------------ step graphs
// One batch step (setup, LSCM, ARAP: any subset) captured once into a CUDA
// graph and replayed with one launch. The capture runs on a private stream in
// thread-local mode; the kernels take the uva_batch by value, so the graph
// holds the pointers and parameters given at creation.
struct uva_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

extern "C" int uva_step_graph_create(uva_batch* b, int32_t parts, const uva_solve_params* lscm,
                                     const uva_solve_params* arap, uva_graph** out) {
    if (!out || !check_batch(b) || (parts & ~7) || !parts || ((parts & UVA_STEP_LSCM) && !lscm) ||
        ((parts & UVA_STEP_ARAP) && !arap)) {
        uva_set_error("uva_step_graph_create: bad arguments");
        return UVA_E_ARG;
    }
    *out = nullptr;
    cudaError_t e = ensure_islands_attr<OP_ARAP>();
    if (e == cudaSuccess) e = ensure_islands_attr<OP_LSCM>();
    if (e == cudaSuccess) e = ensure_coarse_attr();
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_step_graph_create/attributes");
    sm_count();
    cudaStream_t cs = nullptr;
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_step_graph_create/stream");
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return uva_cuda_status(e, "uva_step_graph_create/begin");
    }
    int rc = UVA_OK;
    if ((parts & UVA_STEP_SETUP) && rc == UVA_OK) rc = uva_batch_setup(b, cs);
    if ((parts & UVA_STEP_LSCM) && rc == UVA_OK) rc = uva_lscm(b, lscm, cs);
    if ((parts & UVA_STEP_ARAP) && rc == UVA_OK) rc = uva_arap(b, arap, cs);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc != UVA_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_step_graph_create/end");
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return uva_cuda_status(e, "uva_step_graph_create/instantiate");
    }
    *out = new uva_graph{g, x};
    return UVA_OK;
}

extern "C" int uva_graph_launch(uva_graph* g, void* stream) {
    if (!g || !g->exec) { uva_set_error("uva_graph_launch: null graph"); return UVA_E_ARG; }
    const cudaError_t e = cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_graph_launch");
    return UVA_OK;
}

extern "C" int uva_graph_destroy(uva_graph* g) {
    if (!g) return UVA_OK;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return UVA_OK;
}

// ------------------------------------------------------------------ no-allocation ARAP
// Fixed solver scratch for uva_arap_noalloc. Some callers of this library
// cannot allocate device memory while they run ARAP: a host application that
// owns a fixed device pool, or code that must not call cudaMalloc between
// frames. They pass their own inputs and outputs and the solver borrows this
// static array instead of caller-provided scratch. Every GPU that loads the
// library holds the array until the process exits.
namespace {

constexpr int64_t kNoAllocMaxVerts = 32768;
constexpr int64_t kNoAllocMaxTris = 65536;
constexpr size_t kAlignUp(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }
constexpr size_t kNaWork = 256;                                                   // work counter
constexpr size_t kNaX64 = kAlignUp(sizeof(double) * 2 * kNoAllocMaxVerts);        // x64
constexpr size_t kNaB64 = kAlignUp(sizeof(double) * 2 * kNoAllocMaxVerts);        // b64
constexpr size_t kNaRc = kAlignUp(sizeof(double) * 6 * kNoAllocMaxTris);          // rc
constexpr size_t kNaF32 = kAlignUp(sizeof(float) * 2 * kNoAllocMaxVerts);         // r32, d32, p32, q32
constexpr size_t kNaPart = kAlignUp(sizeof(float) * 2 * kNoAllocMaxVerts);        // cpart (nslices <= n)
constexpr size_t kNaHist = kAlignUp(sizeof(float) * 16 * kNoAllocMaxVerts);      // ARAP start history
constexpr size_t kNoAllocBytes = kNaWork + kNaX64 + kNaB64 + kNaRc + 4 * kNaF32 + kNaPart + kNaHist;   // 7,602,432 bytes

static_assert(kNoAllocBytes == 7602432, "documented size of the static scratch");
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (the host-side symbol is only a stand-in for the device array).
int noalloc_scratch(unsigned char** out) {
    static std::mutex mu;
    static std::vector<unsigned char*> cache;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_arap_noalloc/cudaGetDevice");
    std::lock_guard<std::mutex> lk(mu);
    if (static_cast<int>(cache.size()) <= dev) cache.resize(dev + 1, nullptr);
    if (!cache[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return uva_cuda_status(e, "uva_arap_noalloc/cudaGetSymbolAddress");
        cache[dev] = static_cast<unsigned char*>(p);
    }
    *out = cache[dev];
    return UVA_OK;
}

}  // namespace

extern "C" int uva_arap_noalloc(const uva_batch* b, const uva_solve_params* prm, void* stream) {
    // the caller's scratch fields (work, cpart, x64, ...) are not read
    if (!check_batch_inputs(b) || !prm || !b->status || !b->U) {
        uva_set_error("uva_arap_noalloc: bad arguments (status and U are required outputs)");
        return UVA_E_ARG;
    }
    if (b->n > kNoAllocMaxVerts || b->t > kNoAllocMaxTris || b->nslices > kNoAllocMaxVerts ||
        b->nc > kNoAllocMaxVerts) {
        uva_set_error("uva_arap_noalloc: batch above the fixed scratch limit of 32768 vertices / 65536 triangles");
        return UVA_E_TOOBIG;
    }
    if (b->nc == 0 || prm->iters <= 0) return UVA_OK;
    unsigned char* base = nullptr;
    const int rc = noalloc_scratch(&base);
    if (rc != UVA_OK) return rc;
    uva_batch w = *b;
    size_t off = 0;
    w.work = reinterpret_cast<int32_t*>(base + off); off += kNaWork;
    w.x64 = reinterpret_cast<double*>(base + off); off += kNaX64;
    w.b64 = reinterpret_cast<double*>(base + off); off += kNaB64;
    w.rc = reinterpret_cast<double*>(base + off); off += kNaRc;
    w.r32 = reinterpret_cast<float*>(base + off); off += kNaF32;
    w.d32 = reinterpret_cast<float*>(base + off); off += kNaF32;
    w.p32 = reinterpret_cast<float*>(base + off); off += kNaF32;
    w.q32 = reinterpret_cast<float*>(base + off); off += kNaF32;
    w.cpart = reinterpret_cast<float*>(base + off); off += kNaPart;
    w.hist = reinterpret_cast<float*>(base + off);
    // the work counters are the only scratch that must start at zero;
    // launch_islands clears them on the stream before the launch
    return launch_islands<OP_ARAP>(&w, prm, static_cast<cudaStream_t>(stream));
}
