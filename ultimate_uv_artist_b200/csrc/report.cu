// Whole-mesh report passes on the device (built with --fmad=false: the edge
// lengths and areas follow numpy's operation order):
//   * the UV seam report of engine/metrics.py:227-261 (seam_report): weld
//     vertices, group the triangle edges of the welded mesh, and classify
//     every group (boundary, interior with or without a UV seam,
//     non-manifold);
//   * exact per-corner equality of two attribute sets, as np.array_equal
//     decides it (engine/metrics.py:264-286 preservation_report,
//     engine/validate.py:191-199);
//   * a segmented sum (per-island totals of a per-triangle value).
//
// The reference sorts 3t edge keys and the vertex rows (np.unique); here two
// open-addressing hash tables do the grouping in two passes. Group results
// do not depend on which vertex represents a welded class: a group's two
// half-edges are paired corner by corner through their shared endpoints, and
// an edge length is symmetric in its endpoints.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"

using namespace uva;

namespace {

constexpr int kTB = 256;
constexpr int kRedBlocks = 296;   // 2 x 148 SMs: partial sums of the reduction

inline int64_t al(int64_t x) { return (x + 255) & ~static_cast<int64_t>(255); }

inline unsigned blocks_for(int64_t n, int64_t cap = 1 << 20) {
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + kTB - 1) / kTB, cap)));
}

uint32_t pow2_mask(int64_t want) {
    uint64_t m = 1024;
    while (static_cast<int64_t>(m) < want) m <<= 1;
    return static_cast<uint32_t>(m - 1);
}

__device__ __forceinline__ uint32_t hash64(unsigned long long k) {
    k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33;
    return static_cast<uint32_t>(k);
}

// Position key of a vertex: the three coordinates with -0.0 read as +0.0
// (np.unique over rows compares values).
__device__ __forceinline__ unsigned long long canon(double x) {
    return static_cast<unsigned long long>(__double_as_longlong(x == 0.0 ? 0.0 : x));
}

__device__ __forceinline__ bool same_vertex(const double* V, const int64_t* weld, int64_t a, int64_t b) {
    if (weld) return weld[a] == weld[b];
    return canon(V[3 * a]) == canon(V[3 * b]) && canon(V[3 * a + 1]) == canon(V[3 * b + 1]) &&
           canon(V[3 * a + 2]) == canon(V[3 * b + 2]);
}

__device__ __forceinline__ uint32_t vertex_hash(const double* V, const int64_t* weld, int64_t v) {
    if (weld) return hash64(static_cast<unsigned long long>(weld[v]));
    unsigned long long h = canon(V[3 * v]);
    h = h * 0x9e3779b97f4a7c15ull ^ canon(V[3 * v + 1]);
    h = h * 0x9e3779b97f4a7c15ull ^ canon(V[3 * v + 2]);
    return hash64(h);
}

// rep[v]: the vertex that first claimed the hash slot of v's key.
__global__ void k_sr_weld(int64_t n, const double* V, const int64_t* weld, int32_t* table, uint32_t hmask,
                          int32_t* rep) {
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < n;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int32_t r = static_cast<int32_t>(v);
        for (uint32_t probe = 0, s = vertex_hash(V, weld, v) & hmask; probe <= hmask; ++probe, s = (s + 1) & hmask) {
            const int32_t prev = atomicCAS(table + s, -1, static_cast<int32_t>(v));
            if (prev == -1) break;
            if (same_vertex(V, weld, prev, v)) { r = prev; break; }
        }
        rep[v] = r;
    }
}

// Directed triangle edge h = k m + f: corners (k, k+1) of face f
// (engine/metrics.py:234-237).
struct HalfEdge {
    int64_t c0, c1;   // corner vertices
    int32_t r0, r1;   // their representatives
};

// numpy row indexing: -n <= idx < n, negative counts from the end.
__device__ __forceinline__ bool vertex_index(int64_t idx, int64_t n, int64_t& v) {
    if (idx < -n || idx >= n) return false;
    v = idx < 0 ? idx + n : idx;
    return true;
}

// The corners of every face, wrapped into [0, n); out-of-range faces are
// flagged (the reference raises IndexError).
__global__ void k_sr_faces(int64_t m, int64_t n, const int64_t* F, int64_t* Fw, int32_t* status) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < 3 * m;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t v;
        if (!vertex_index(F[i], n, v)) { atomicOr(status, 1); v = 0; }
        Fw[i] = v;
    }
}

__device__ __forceinline__ HalfEdge half_edge(const int64_t* F, const int32_t* rep, int64_t m, int64_t h) {
    const int64_t k = h / m, f = h - k * m;
    HalfEdge e;
    e.c0 = F[3 * f + k];
    e.c1 = F[3 * f + (k + 1) % 3];
    e.r0 = rep[e.c0];
    e.r1 = rep[e.c1];
    return e;
}

__device__ __forceinline__ unsigned long long edge_key(const HalfEdge& e) {
    const uint32_t lo = static_cast<uint32_t>(min(e.r0, e.r1)), hi = static_cast<uint32_t>(max(e.r0, e.r1));
    return (static_cast<unsigned long long>(lo) << 32) | hi;
}

constexpr unsigned long long kEmpty = ~0ull;

__global__ void k_sr_edges(int64_t m, const int64_t* F, const int32_t* rep, unsigned long long* keys, int32_t* cnt,
                           unsigned long long* hmin, unsigned long long* hmax, uint32_t hmask) {
    for (int64_t h = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; h < 3 * m;
         h += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const HalfEdge e = half_edge(F, rep, m, h);
        const unsigned long long key = edge_key(e);
        for (uint32_t probe = 0, s = hash64(key) & hmask; probe <= hmask; ++probe, s = (s + 1) & hmask) {
            const unsigned long long prev = atomicCAS(keys + s, kEmpty, key);
            if (prev == kEmpty || prev == key) {
                atomicAdd(cnt + s, 1);
                atomicMin(hmin + s, static_cast<unsigned long long>(h));
                atomicMax(hmax + s, static_cast<unsigned long long>(h));
                break;
            }
        }
    }
}

// |P[a] - P[b]| as np.linalg.norm(axis=1): sqrt((dx dx + dy dy) + dz dz).
__device__ __forceinline__ double seg_len(const double* P, int64_t a, int64_t b) {
    const double dx = P[3 * a] - P[3 * b], dy = P[3 * a + 1] - P[3 * b + 1], dz = P[3 * a + 2] - P[3 * b + 2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// Corners of a half-edge ordered (lower representative first; in the
// reference: swap = e0 > e1, metrics.py:238-240).
__device__ __forceinline__ void lo_hi(const HalfEdge& e, int64_t& clo, int64_t& chi) {
    const bool swap = e.r0 > e.r1;
    clo = swap ? e.c1 : e.c0;
    chi = swap ? e.c0 : e.c1;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Classify every edge group, and sum the triangle areas; one partial per
// block, folded in block order by k_sr_final.
__global__ void __launch_bounds__(kTB) k_sr_classify(uint32_t hslots, const unsigned long long* keys,
                                                     const int32_t* cnt, const unsigned long long* hmin,
                                                     const unsigned long long* hmax, int64_t m, const int64_t* F,
                                                     const int32_t* rep, const double* P, const double* UV,
                                                     double* part) {
    double sl = 0.0, bl = 0.0, ar = 0.0, ns = 0.0, nb = 0.0, nn = 0.0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; s < hslots; s += stride) {
        if (keys[s] == kEmpty) continue;
        const int c = cnt[s];
        if (c == 1) {
            const HalfEdge e = half_edge(F, rep, m, static_cast<int64_t>(hmin[s]));
            int64_t clo, chi;
            lo_hi(e, clo, chi);
            bl += seg_len(P, clo, chi);
            nb += 1.0;
        } else if (c == 2) {
            const HalfEdge e0 = half_edge(F, rep, m, static_cast<int64_t>(hmin[s]));
            const HalfEdge e1 = half_edge(F, rep, m, static_cast<int64_t>(hmax[s]));
            int64_t a0, b0, a1, b1;
            lo_hi(e0, a0, b0);
            lo_hi(e1, a1, b1);
            // np.any(u[a] != u[b]): NaN compares unequal
            const bool mism = UV[2 * a0] != UV[2 * a1] || UV[2 * a0 + 1] != UV[2 * a1 + 1] ||
                              UV[2 * b0] != UV[2 * b1] || UV[2 * b0 + 1] != UV[2 * b1 + 1];
            if (mism) {
                sl += seg_len(P, a0, b0);
                ns += 1.0;
            }
        } else if (c > 2) {
            nn += 1.0;
        }
    }
    for (int64_t f = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; f < m; f += stride) {
        const double* p0 = P + 3 * F[3 * f];
        const double* p1 = P + 3 * F[3 * f + 1];
        const double* p2 = P + 3 * F[3 * f + 2];
        const double ax = p1[0] - p0[0], ay = p1[1] - p0[1], az = p1[2] - p0[2];
        const double bx = p2[0] - p0[0], by = p2[1] - p0[1], bz = p2[2] - p0[2];
        const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
        ar += 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
    }
    __shared__ double red[6][kTB / 32];
    double v[6] = {sl, bl, ar, ns, nb, nn};
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double x = warp_sum(v[k]);
        if (lane == 0) red[k][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double x = 0.0;
        for (int q = 0; q < kTB / 32; ++q) x += red[threadIdx.x][q];
        part[6 * blockIdx.x + threadIdx.x] = x;
    }
}

// out: seam_edges, seam_length, open_boundary_edges, open_boundary_length,
// nonmanifold_edge_groups, surface_area (counts are exact: below 2^53).
__global__ void k_sr_final(int nparts, const double* part, double* out) {
    if (threadIdx.x != 0) return;
    double t[6] = {0, 0, 0, 0, 0, 0};
    for (int b = 0; b < nparts; ++b)
        for (int k = 0; k < 6; ++k) t[k] += part[6 * b + k];
    out[0] = t[3];
    out[1] = t[0];
    out[2] = t[4];
    out[3] = t[1];
    out[4] = t[5];
    out[5] = t[2];
}

struct SrLayout {
    int64_t off[9];
    int64_t total;
    uint32_t vmask, emask;
};

SrLayout sr_layout(int64_t n, int64_t m) {
    SrLayout L{};
    L.vmask = pow2_mask(2 * std::max<int64_t>(n, 1));
    L.emask = pow2_mask(2 * 3 * std::max<int64_t>(m, 1));
    const int64_t V = static_cast<int64_t>(L.vmask) + 1, E = static_cast<int64_t>(L.emask) + 1;
    const int64_t sz[8] = {al(4 * V), al(4 * std::max<int64_t>(n, 1)), al(8 * E), al(4 * E), al(8 * E), al(8 * E),
                           al(8 * 6 * kRedBlocks), al(8 * 3 * std::max<int64_t>(m, 1))};
    int64_t o = 0;
    for (int i = 0; i < 8; ++i) { L.off[i] = o; o += sz[i]; }
    L.off[8] = o;
    L.total = o;
    return L;
}

// ------------------------------------------------------------------ corner equality
// Element type codes (host numpy dtypes): 0 f32, 1 f64, 2 f16, 3 u8, 4 i8,
// 5 i16, 6 u16, 7 i32, 8 u32, 9 i64, 10 u64, 11 bool (as u8).
__device__ __forceinline__ bool is_float(int dt) { return dt <= 2; }

__device__ __forceinline__ double as_double(const void* p, int dt, int64_t i) {
    switch (dt) {
        case 0: return static_cast<const float*>(p)[i];
        case 1: return static_cast<const double*>(p)[i];
        case 2: return __half2float(static_cast<const __half*>(p)[i]);
        case 3: case 11: return static_cast<const uint8_t*>(p)[i];
        case 4: return static_cast<const int8_t*>(p)[i];
        case 5: return static_cast<const int16_t*>(p)[i];
        case 6: return static_cast<const uint16_t*>(p)[i];
        case 7: return static_cast<const int32_t*>(p)[i];
        case 8: return static_cast<const uint32_t*>(p)[i];
        case 9: return static_cast<double>(static_cast<const int64_t*>(p)[i]);
        default: return static_cast<double>(static_cast<const uint64_t*>(p)[i]);
    }
}

// Integers compared exactly: as int64, or as uint64 when both are u64.
__device__ __forceinline__ long long as_i64(const void* p, int dt, int64_t i) {
    switch (dt) {
        case 3: case 11: return static_cast<const uint8_t*>(p)[i];
        case 4: return static_cast<const int8_t*>(p)[i];
        case 5: return static_cast<const int16_t*>(p)[i];
        case 6: return static_cast<const uint16_t*>(p)[i];
        case 7: return static_cast<const int32_t*>(p)[i];
        case 8: return static_cast<const uint32_t*>(p)[i];
        case 9: return static_cast<const int64_t*>(p)[i];
        default: return static_cast<long long>(static_cast<const uint64_t*>(p)[i]);
    }
}

// numpy indexing of a row: -rows <= idx < rows, negative counts from the end.
__device__ __forceinline__ bool wrap_index(int64_t idx, int64_t rows, int64_t& r) {
    if (idx < -rows || idx >= rows) return false;
    r = idx < 0 ? idx + rows : idx;
    return true;
}

__global__ void k_corners_equal(const void* A, int32_t adt, int64_t na, const int64_t* fa, const void* B,
                                int32_t bdt, int64_t nb, const int64_t* fb, int64_t m, int32_t w, int32_t* result) {
    const bool fl = is_float(adt) || is_float(bdt);
    const bool u64 = adt == 10 && bdt == 10;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < m;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t ra, rb;
        if (!wrap_index(fa[i], na, ra) || !wrap_index(fb[i], nb, rb)) { atomicOr(result, 2); continue; }
        bool eq = true;
        for (int c = 0; c < w && eq; ++c) {
            const int64_t ia = ra * w + c, ib = rb * w + c;
            if (fl) eq = as_double(A, adt, ia) == as_double(B, bdt, ib);
            else if (u64) eq = static_cast<const uint64_t*>(A)[ia] == static_cast<const uint64_t*>(B)[ib];
            else eq = as_i64(A, adt, ia) == as_i64(B, bdt, ib);
        }
        if (!eq) atomicOr(result, 1);
    }
}

// ------------------------------------------------------------------ segmented sum
__global__ void k_segment_sum(int64_t m, const double* x, int64_t stride, const int32_t* seg, int32_t nseg,
                              double* out, int32_t* status) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < m;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t g = seg[i];
        if (g < 0 || g >= nseg) { atomicOr(status, 1); continue; }
        atomicAdd(out + g, x[i * stride]);
    }
}

}  // namespace

// ==================================================================== C ABI
extern "C" int uva_seam_report_scratch_bytes(int64_t n, int64_t m, int64_t* bytes) {
    if (n < 0 || m < 0 || !bytes) { uva_set_error("uva_seam_report_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    *bytes = sr_layout(n, m).total;
    return UVA_OK;
}

extern "C" int uva_seam_report(const double* V, int64_t n, const int64_t* F, int64_t m, const double* UV,
                               const int64_t* weld, double* out, int32_t* status, void* scratch,
                               int64_t scratch_bytes, void* stream) {
    const SrLayout L = sr_layout(n < 0 ? 0 : n, m < 0 ? 0 : m);
    if (n < 0 || m < 0 || !out || !status || n > 0x7fffffffll || 6 * m > 0x7fffffffll ||
        (m > 0 && (!V || !F || !UV || !scratch || scratch_bytes < L.total))) {
        uva_set_error("uva_seam_report: bad arguments or scratch too small");
        return UVA_E_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(out, 0, 8 * 6, s);
    cudaMemsetAsync(status, 0, 4, s);
    if (m == 0) { UVA_CHECK_LAUNCH("uva_seam_report"); return UVA_OK; }
    if (n == 0) { cudaMemsetAsync(status, 0x01, 1, s); UVA_CHECK_LAUNCH("uva_seam_report"); return UVA_OK; }
    auto* base = static_cast<unsigned char*>(scratch);
    auto* vtab = reinterpret_cast<int32_t*>(base + L.off[0]);
    auto* rep = reinterpret_cast<int32_t*>(base + L.off[1]);
    auto* keys = reinterpret_cast<unsigned long long*>(base + L.off[2]);
    auto* cnt = reinterpret_cast<int32_t*>(base + L.off[3]);
    auto* hmin = reinterpret_cast<unsigned long long*>(base + L.off[4]);
    auto* hmax = reinterpret_cast<unsigned long long*>(base + L.off[5]);
    auto* part = reinterpret_cast<double*>(base + L.off[6]);
    auto* Fw = reinterpret_cast<int64_t*>(base + L.off[7]);
    const size_t VS = static_cast<size_t>(L.vmask) + 1, ES = static_cast<size_t>(L.emask) + 1;
    cudaMemsetAsync(vtab, 0xff, 4 * VS, s);
    cudaMemsetAsync(keys, 0xff, 8 * ES, s);
    cudaMemsetAsync(cnt, 0, 4 * ES, s);
    cudaMemsetAsync(hmin, 0xff, 8 * ES, s);
    cudaMemsetAsync(hmax, 0, 8 * ES, s);
    k_sr_faces<<<blocks_for(3 * m), kTB, 0, s>>>(m, n, F, Fw, status);
    k_sr_weld<<<blocks_for(n), kTB, 0, s>>>(n, V, weld, vtab, L.vmask, rep);
    k_sr_edges<<<blocks_for(3 * m), kTB, 0, s>>>(m, Fw, rep, keys, cnt, hmin, hmax, L.emask);
    k_sr_classify<<<kRedBlocks, kTB, 0, s>>>(static_cast<uint32_t>(ES), keys, cnt, hmin, hmax, m, Fw, rep, V, UV,
                                              part);
    k_sr_final<<<1, 32, 0, s>>>(kRedBlocks, part, out);
    UVA_CHECK_LAUNCH("uva_seam_report");
    return UVA_OK;
}

extern "C" int uva_corners_equal(const void* A, int32_t adt, int64_t na, const int64_t* fa, const void* B,
                                 int32_t bdt, int64_t nb, const int64_t* fb, int64_t m, int32_t w, int32_t* result,
                                 void* stream) {
    if (!result || m < 0 || w < 0 || na < 0 || nb < 0 || adt < 0 || adt > 11 || bdt < 0 || bdt > 11 ||
        (m > 0 && (!fa || !fb || (w > 0 && (!A || !B))))) {
        uva_set_error("uva_corners_equal: bad arguments");
        return UVA_E_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(result, 0, 4, s);
    if (m > 0) k_corners_equal<<<blocks_for(m, 4096), kTB, 0, s>>>(A, adt, na, fa, B, bdt, nb, fb, m, w, result);
    UVA_CHECK_LAUNCH("uva_corners_equal");
    return UVA_OK;
}

extern "C" int uva_segment_sum(const double* x, int64_t stride, const int32_t* seg, int64_t m, int32_t nseg,
                               double* out, int32_t* status, void* stream) {
    if (m < 0 || nseg < 0 || stride < 1 || !status || (nseg > 0 && !out) || (m > 0 && (!x || !seg))) {
        uva_set_error("uva_segment_sum: bad arguments");
        return UVA_E_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(status, 0, 4, s);
    if (nseg > 0) cudaMemsetAsync(out, 0, 8 * static_cast<size_t>(nseg), s);
    if (m > 0) k_segment_sum<<<blocks_for(m, 4096), kTB, 0, s>>>(m, x, stride, seg, nseg, out, status);
    UVA_CHECK_LAUNCH("uva_segment_sum");
    return UVA_OK;
}
