// Mesh edge bookkeeping on the device: unique undirected edges of a triangle
// list, the symmetric CSR assembled from them, sparse-matrix products with a
// few dense columns, and the directed boundary half-edges of a chart.
//
// These serve the module functions the reference builds with torch / numpy
// sorts (engine/gpu.py:16-63 csr32 / spmm / unique_edges / sym_csr,
// engine/param.py:59-68 boundary_edges_oriented). Here no general sort is
// used:
//   * unique edges: half-edges are bucketed by their smaller endpoint (a
//     counting sort); inside a bucket (a vertex's incident edges, a handful)
//     every entry finds its distinct rank by scanning the bucket, which
//     yields the ascending (lo, hi) order directly;
//   * symmetric CSR: atomic placement per row, then a per-row heap sort by
//     column;
//   * boundary half-edges: an open-addressing hash of the directed keys and
//     one lookup of each reverse key.
// Every result is deterministic.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "scan.cuh"

using namespace uva;

namespace {

constexpr int kTB = 256;

inline unsigned blocks_for(int64_t n) {
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + kTB - 1) / kTB, 1 << 20)));
}

inline int64_t al(int64_t x) { return (x + 255) & ~static_cast<int64_t>(255); }

__device__ __forceinline__ unsigned long long* ull(int64_t* p) { return reinterpret_cast<unsigned long long*>(p); }

// Half-edge h = k t + f of the unique-edge numbering: corners (k+1, k+2) of
// triangle f (engine/gpu.py:41, edge k opposite corner k).
__device__ __forceinline__ void half_edge_opp(const int64_t* T, int64_t t, int64_t h, int64_t& a, int64_t& b) {
    const int64_t k = h / t, f = h - k * t;
    a = T[3 * f + (k + 1) % 3];
    b = T[3 * f + (k + 2) % 3];
}

// ------------------------------------------------------------------ unique edges
__global__ void k_ue_count(const int64_t* T, int64_t t, int64_t n, int64_t* bcnt, int32_t* bad) {
    const int64_t H = 3 * t;
    for (int64_t h = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; h < H;
         h += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t a, b;
        half_edge_opp(T, t, h, a, b);
        if (a < 0 || b < 0 || a >= n || b >= n) { atomicExch(bad, 1); continue; }
        atomicAdd(ull(bcnt + (a < b ? a : b)), 1ull);
    }
}

__global__ void k_ue_fill(const int64_t* T, int64_t t, int64_t n, int64_t* cursor, int64_t* bucket, int64_t* bhi) {
    const int64_t H = 3 * t;
    for (int64_t h = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; h < H;
         h += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t a, b;
        half_edge_opp(T, t, h, a, b);
        if (a < 0 || b < 0 || a >= n || b >= n) continue;
        const int64_t lo = a < b ? a : b;
        const int64_t p = static_cast<int64_t>(atomicAdd(ull(cursor + lo), 1ull));
        bucket[p] = h;
        bhi[p] = a < b ? b : a;
    }
}

// Smaller endpoint of half-edge h (its bucket).
__device__ __forceinline__ int64_t half_edge_lo(const int64_t* T, int64_t t, int64_t h) {
    int64_t a, b;
    half_edge_opp(T, t, h, a, b);
    return a < b ? a : b;
}

// Per bucket entry: first occurrence of its hi (smallest half-edge index) and
// the number of entries sharing it. Only the bstart[n] bucketed entries are
// visited (half-edges with an index out of range were left out).
__global__ void k_ue_first(const int64_t* T, int64_t t, int64_t n, const int64_t* bstart, const int64_t* bucket,
                           const int64_t* bhi, uint8_t* first, int32_t* same, int64_t* dcnt) {
    const int64_t total = bstart[n];
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < total;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t h = bucket[p], hi = bhi[p];
        const int64_t lo = half_edge_lo(T, t, h);
        const int64_t q0 = bstart[lo], q1 = bstart[lo + 1];
        bool is_first = true;
        int32_t cnt = 0;
        for (int64_t q = q0; q < q1; ++q) {
            if (bhi[q] != hi) continue;
            ++cnt;
            if (bucket[q] < h) is_first = false;
        }
        first[p] = is_first ? 1 : 0;
        same[p] = cnt;
        if (is_first) atomicAdd(ull(dcnt + lo), 1ull);
    }
}

// Rank of the entry's hi among the distinct his of its bucket, then the
// outputs: inv for every half-edge, endpoints and use count per unique edge.
__global__ void k_ue_out(const int64_t* T, int64_t t, int64_t n, const int64_t* bstart, const int64_t* bucket,
                         const int64_t* bhi, const uint8_t* first, const int32_t* same, const int64_t* uofs,
                         int64_t* ea, int64_t* eb, int64_t* inv, int64_t* cnt) {
    const int64_t total = bstart[n];
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < total;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t h = bucket[p], hi = bhi[p];
        const int64_t lo = half_edge_lo(T, t, h);
        const int64_t q0 = bstart[lo], q1 = bstart[lo + 1];
        int64_t rank = 0;
        for (int64_t q = q0; q < q1; ++q) rank += (first[q] && bhi[q] < hi) ? 1 : 0;
        const int64_t uid = uofs[lo] + rank;
        inv[h] = uid;
        if (first[p]) {
            ea[uid] = lo;
            eb[uid] = hi;
            cnt[uid] = same[p];
        }
    }
}

__global__ void k_ue_final(const int64_t* uofs, int64_t n, const int32_t* bad, int64_t* nedges) {
    *nedges = *bad ? -1 : uofs[n];
}

struct UeLayout {
    int64_t off[10];
    int64_t total;
};

UeLayout ue_layout(int64_t n, int64_t t) {
    const int64_t N1 = n + 1, H = std::max<int64_t>(3 * t, 1);
    const int64_t sz[9] = {al(8 * N1), al(8 * N1), al(8 * N1), al(8 * H), al(8 * H), al(H), al(4 * H),
                           al(8 * xscan_sums(N1)), al(256)};
    UeLayout L{};
    int64_t o = 0;
    for (int i = 0; i < 9; ++i) { L.off[i] = o; o += sz[i]; }
    L.off[9] = o;
    L.total = o;
    return L;
}

// ------------------------------------------------------------------ symmetric CSR
__global__ void k_sc_count(int64_t ne, int64_t n, const int64_t* ea, const int64_t* eb, int32_t* rc, int32_t* bad) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < ne + n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (i < ne) {
            const int64_t a = ea[i], b = eb[i];
            if (a < 0 || b < 0 || a >= n || b >= n) { atomicExch(bad, 1); continue; }
            atomicAdd(rc + a, 1);
            atomicAdd(rc + b, 1);
        } else {
            atomicAdd(rc + (i - ne), 1);
        }
    }
}

template <typename V>
__global__ void k_sc_fill(int64_t ne, int64_t n, const int64_t* ea, const int64_t* eb, const V* off, const V* diag,
                          int32_t* cursor, int32_t* col, V* val) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < ne + n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (i < ne) {
            const int64_t a = ea[i], b = eb[i];
            if (a < 0 || b < 0 || a >= n || b >= n) continue;
            const int32_t p = atomicAdd(cursor + a, 1);
            col[p] = static_cast<int32_t>(b);
            val[p] = off[i];
            const int32_t q = atomicAdd(cursor + b, 1);
            col[q] = static_cast<int32_t>(a);
            val[q] = off[i];
        } else {
            const int64_t r = i - ne;
            const int32_t p = atomicAdd(cursor + r, 1);
            col[p] = static_cast<int32_t>(r);
            val[p] = diag[r];
        }
    }
}

template <typename V>
__device__ __forceinline__ bool sc_less(int32_t ca, V va, int32_t cb, V vb) {
    if (ca != cb) return ca < cb;
    // equal columns (repeated edges): order by value bits, so the layout is
    // the same on every run
    if (sizeof(V) == 8)
        return __double_as_longlong(static_cast<double>(va)) < __double_as_longlong(static_cast<double>(vb));
    return __float_as_int(static_cast<float>(va)) < __float_as_int(static_cast<float>(vb));
}

// In-place heap sort of one row's (column, value) pairs by column.
template <typename V>
__global__ void k_sc_sort(int64_t n, const int32_t* crow, int32_t* col, V* val) {
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int32_t* c = col + crow[r];
        V* v = val + crow[r];
        const int len = crow[r + 1] - crow[r];
        auto sift = [&](int root, int end) {
            for (;;) {
                int child = 2 * root + 1;
                if (child >= end) return;
                if (child + 1 < end && sc_less(c[child], v[child], c[child + 1], v[child + 1])) ++child;
                if (!sc_less(c[root], v[root], c[child], v[child])) return;
                const int32_t tc = c[root]; c[root] = c[child]; c[child] = tc;
                const V tv = v[root]; v[root] = v[child]; v[child] = tv;
                root = child;
            }
        };
        for (int s = len / 2 - 1; s >= 0; --s) sift(s, len);
        for (int e = len - 1; e > 0; --e) {
            const int32_t tc = c[0]; c[0] = c[e]; c[e] = tc;
            const V tv = v[0]; v[0] = v[e]; v[e] = tv;
            sift(0, e);
        }
    }
}

// ------------------------------------------------------------------ CSR x dense columns
// G lanes per row (a power of two up to 32), columns in chunks of 4.
template <typename V, int G>
__global__ void k_spmm(int32_t nrows, int32_t k, const int32_t* crow, const int32_t* col, const V* val, const V* X,
                       V* Y) {
    const int lane = threadIdx.x & (G - 1);
    const int64_t groups = static_cast<int64_t>(gridDim.x) * (blockDim.x / G);
    const unsigned mask = G == 32 ? 0xffffffffu : (((1u << (G & 31)) - 1u) << (threadIdx.x & 31 & ~(G - 1)));
    for (int64_t r = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) / G; r < nrows; r += groups) {
        const int32_t j0 = crow[r], j1 = crow[r + 1];
        for (int32_t c0 = 0; c0 < k; c0 += 4) {
            V acc[4] = {V(0), V(0), V(0), V(0)};
            for (int32_t j = j0 + lane; j < j1; j += G) {
                const V a = val[j];
                const V* x = X + static_cast<int64_t>(col[j]) * k + c0;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (c0 + q < k) acc[q] += a * x[q];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
#pragma unroll
                for (int o = G / 2; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(mask, acc[q], o, G);
            }
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (c0 + q < k) Y[r * k + c0 + q] = acc[q];
            }
        }
    }
}

template <typename V>
int launch_spmm(int32_t nrows, int32_t k, int64_t nnz, const int32_t* crow, const int32_t* col, const V* val,
                const V* X, V* Y, cudaStream_t s) {
    const double avg = nrows > 0 ? static_cast<double>(nnz) / nrows : 0.0;
    const int64_t threads_needed = static_cast<int64_t>(nrows) * (avg <= 4 ? 2 : avg <= 8 ? 4 : avg <= 16 ? 8 : avg <= 48 ? 16 : 32);
    const unsigned grid = blocks_for(threads_needed);
    if (avg <= 4) k_spmm<V, 2><<<grid, kTB, 0, s>>>(nrows, k, crow, col, val, X, Y);
    else if (avg <= 8) k_spmm<V, 4><<<grid, kTB, 0, s>>>(nrows, k, crow, col, val, X, Y);
    else if (avg <= 16) k_spmm<V, 8><<<grid, kTB, 0, s>>>(nrows, k, crow, col, val, X, Y);
    else if (avg <= 48) k_spmm<V, 16><<<grid, kTB, 0, s>>>(nrows, k, crow, col, val, X, Y);
    else k_spmm<V, 32><<<grid, kTB, 0, s>>>(nrows, k, crow, col, val, X, Y);
    UVA_CHECK_LAUNCH("uva_csr_spmm");
    return UVA_OK;
}

// ------------------------------------------------------------------ boundary half-edges
constexpr unsigned long long kEmptyKey = ~0ull;

__device__ __forceinline__ uint32_t hash64(unsigned long long k) {
    k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33;
    return static_cast<uint32_t>(k);
}

// Directed half-edge h = k t + f of the boundary numbering: corners (k, k+1)
// of triangle f (engine/param.py:61-62).
__device__ __forceinline__ bool directed_key(const int64_t* T, int64_t t, int64_t h, unsigned long long& key,
                                             unsigned long long& rev) {
    const int64_t k = h / t, f = h - k * t;
    const int64_t a = T[3 * f + k], b = T[3 * f + (k + 1) % 3];
    if (a < 0 || b < 0 || a > 0x7fffffffll || b > 0x7fffffffll) return false;
    key = (static_cast<unsigned long long>(a) << 32) | static_cast<unsigned long long>(b);
    rev = (static_cast<unsigned long long>(b) << 32) | static_cast<unsigned long long>(a);
    return true;
}

__global__ void k_bm_insert(const int64_t* T, int64_t t, unsigned long long* table, uint32_t hmask, int32_t* bad) {
    for (int64_t h = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; h < 3 * t;
         h += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        unsigned long long key, rev;
        if (!directed_key(T, t, h, key, rev)) { atomicExch(bad, 1); continue; }
        for (uint32_t probe = 0, s = hash64(key) & hmask; probe <= hmask; ++probe, s = (s + 1) & hmask) {
            const unsigned long long prev = atomicCAS(table + s, kEmptyKey, key);
            if (prev == kEmptyKey || prev == key) break;
        }
    }
}

__global__ void k_bm_query(const int64_t* T, int64_t t, const unsigned long long* table, uint32_t hmask,
                           uint8_t* keep) {
    for (int64_t h = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; h < 3 * t;
         h += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        unsigned long long key, rev;
        if (!directed_key(T, t, h, key, rev)) { keep[h] = 0; continue; }
        bool twin = false;
        for (uint32_t probe = 0, s = hash64(rev) & hmask; probe <= hmask; ++probe, s = (s + 1) & hmask) {
            const unsigned long long x = table[s];
            if (x == rev) { twin = true; break; }
            if (x == kEmptyKey) break;
        }
        keep[h] = twin ? 0 : 1;
    }
}

uint32_t pow2_mask(int64_t want) {
    uint64_t m = 1024;
    while (static_cast<int64_t>(m) < want) m <<= 1;
    return static_cast<uint32_t>(m - 1);
}

// ------------------------------------------------------------------ batch edges
__global__ void k_batch_edges(uva_batch b, int64_t* ea, int64_t* eb, int64_t* cnt) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < 3 * static_cast<int64_t>(b.t);
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t f = i / 3;
        const int k = static_cast<int>(i - 3 * f);
        const int32_t e = b.tri_edge[i];
        if (e < 0 || e >= b.E) continue;
        const int32_t isl = b.tri4[4 * f + 3];
        const int64_t base = b.vofs[isl];
        const int64_t a = base + b.tri4[4 * f + (k + 1) % 3], c = base + b.tri4[4 * f + (k + 2) % 3];
        ea[e] = a < c ? a : c;   // every half-edge of e writes the same pair
        eb[e] = a < c ? c : a;
        atomicAdd(ull(cnt + e), 1ull);
    }
}

}  // namespace

// ==================================================================== C ABI
extern "C" int uva_unique_edges_scratch_bytes(int64_t n, int64_t t, int64_t* bytes) {
    if (n < 0 || t < 0 || !bytes) { uva_set_error("uva_unique_edges_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    *bytes = ue_layout(n, t).total;
    return UVA_OK;
}

extern "C" int uva_unique_edges(const int64_t* T, int64_t t, int64_t n, int64_t* ea, int64_t* eb, int64_t* inv,
                                int64_t* cnt, int64_t* nedges, void* scratch, int64_t scratch_bytes, void* stream) {
    if (t < 0 || n < 0 || !nedges || (t > 0 && (!T || !ea || !eb || !inv || !cnt || !scratch))) {
        uva_set_error("uva_unique_edges: bad arguments");
        return UVA_E_ARG;
    }
    const UeLayout L = ue_layout(n, t);
    if (t > 0 && scratch_bytes < L.total) { uva_set_error("uva_unique_edges: scratch too small"); return UVA_E_ARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (t == 0) { cudaMemsetAsync(nedges, 0, 8, s); UVA_CHECK_LAUNCH("uva_unique_edges"); return UVA_OK; }
    auto* base = static_cast<unsigned char*>(scratch);
    auto* bstart = reinterpret_cast<int64_t*>(base + L.off[0]);
    auto* cursor = reinterpret_cast<int64_t*>(base + L.off[1]);
    auto* uofs = reinterpret_cast<int64_t*>(base + L.off[2]);
    auto* bucket = reinterpret_cast<int64_t*>(base + L.off[3]);
    auto* bhi = reinterpret_cast<int64_t*>(base + L.off[4]);
    auto* first = reinterpret_cast<uint8_t*>(base + L.off[5]);
    auto* same = reinterpret_cast<int32_t*>(base + L.off[6]);
    auto* sums = reinterpret_cast<int64_t*>(base + L.off[7]);
    auto* bad = reinterpret_cast<int32_t*>(base + L.off[8]);
    const int64_t H = 3 * t;
    cudaMemsetAsync(bstart, 0, 8 * (n + 1), s);
    cudaMemsetAsync(uofs, 0, 8 * (n + 1), s);
    cudaMemsetAsync(bad, 0, 4, s);
    k_ue_count<<<blocks_for(H), kTB, 0, s>>>(T, t, n, bstart, bad);
    xscan<int64_t>(bstart, bstart, sums, nullptr, n + 1, s);
    cudaMemcpyAsync(cursor, bstart, 8 * (n + 1), cudaMemcpyDeviceToDevice, s);
    k_ue_fill<<<blocks_for(H), kTB, 0, s>>>(T, t, n, cursor, bucket, bhi);
    k_ue_first<<<blocks_for(H), kTB, 0, s>>>(T, t, n, bstart, bucket, bhi, first, same, uofs);
    xscan<int64_t>(uofs, uofs, sums, nullptr, n + 1, s);
    k_ue_out<<<blocks_for(H), kTB, 0, s>>>(T, t, n, bstart, bucket, bhi, first, same, uofs, ea, eb, inv, cnt);
    k_ue_final<<<1, 1, 0, s>>>(uofs, n, bad, nedges);
    UVA_CHECK_LAUNCH("uva_unique_edges");
    return UVA_OK;
}

extern "C" int uva_sym_csr_scratch_bytes(int64_t n, int64_t* bytes) {
    if (n < 0 || !bytes) { uva_set_error("uva_sym_csr_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    *bytes = al(4 * (n + 1)) + al(4 * xscan_sums(n + 1)) + al(256);
    return UVA_OK;
}

extern "C" int uva_sym_csr(int64_t n, int64_t ne, const int64_t* ea, const int64_t* eb, const void* off,
                           const void* diag, int32_t dtype, int32_t* crow, int32_t* col, void* val, int32_t* status,
                           void* scratch, int64_t scratch_bytes, void* stream) {
    int64_t need = 0;
    uva_sym_csr_scratch_bytes(n < 0 ? 0 : n, &need);
    if (n < 0 || ne < 0 || (dtype != 0 && dtype != 1) || !crow || !status || !scratch || scratch_bytes < need ||
        (ne > 0 && (!ea || !eb || !off)) || (n > 0 && (!diag || !col || !val)) || 2 * ne + n > 0x7fffffffll) {
        uva_set_error("uva_sym_csr: bad arguments (nnz must fit int32)");
        return UVA_E_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto* base = static_cast<unsigned char*>(scratch);
    auto* cursor = reinterpret_cast<int32_t*>(base);
    auto* sums = reinterpret_cast<int32_t*>(base + al(4 * (n + 1)));
    cudaMemsetAsync(status, 0, 4, s);
    cudaMemsetAsync(crow, 0, 4 * (n + 1), s);
    if (n == 0) { UVA_CHECK_LAUNCH("uva_sym_csr"); return UVA_OK; }
    k_sc_count<<<blocks_for(ne + n), kTB, 0, s>>>(ne, n, ea, eb, crow, status);
    xscan<int32_t>(crow, crow, sums, nullptr, n + 1, s);
    cudaMemcpyAsync(cursor, crow, 4 * (n + 1), cudaMemcpyDeviceToDevice, s);
    if (dtype == 0) {
        k_sc_fill<float><<<blocks_for(ne + n), kTB, 0, s>>>(ne, n, ea, eb, static_cast<const float*>(off),
                                                            static_cast<const float*>(diag), cursor, col,
                                                            static_cast<float*>(val));
        k_sc_sort<float><<<blocks_for(n), kTB, 0, s>>>(n, crow, col, static_cast<float*>(val));
    } else {
        k_sc_fill<double><<<blocks_for(ne + n), kTB, 0, s>>>(ne, n, ea, eb, static_cast<const double*>(off),
                                                             static_cast<const double*>(diag), cursor, col,
                                                             static_cast<double*>(val));
        k_sc_sort<double><<<blocks_for(n), kTB, 0, s>>>(n, crow, col, static_cast<double*>(val));
    }
    UVA_CHECK_LAUNCH("uva_sym_csr");
    return UVA_OK;
}

extern "C" int uva_csr_spmm(int32_t nrows, int32_t k, int64_t nnz, const int32_t* crow, const int32_t* col,
                            const void* val, const void* X, void* Y, int32_t dtype, void* stream) {
    if (nrows < 0 || k < 0 || nnz < 0 || (dtype != 0 && dtype != 1) ||
        (nrows > 0 && k > 0 && (!crow || !Y || (nnz > 0 && (!col || !val || !X))))) {
        uva_set_error("uva_csr_spmm: bad arguments");
        return UVA_E_ARG;
    }
    if (nrows == 0 || k == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == 0)
        return launch_spmm<float>(nrows, k, nnz, crow, col, static_cast<const float*>(val),
                                  static_cast<const float*>(X), static_cast<float*>(Y), s);
    return launch_spmm<double>(nrows, k, nnz, crow, col, static_cast<const double*>(val),
                               static_cast<const double*>(X), static_cast<double*>(Y), s);
}

extern "C" int uva_boundary_mask_scratch_bytes(int64_t t, int64_t* bytes) {
    if (t < 0 || !bytes) { uva_set_error("uva_boundary_mask_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    *bytes = 8 * (static_cast<int64_t>(pow2_mask(2 * 3 * t)) + 1) + 256;
    return UVA_OK;
}

extern "C" int uva_boundary_mask(const int64_t* T, int64_t t, uint8_t* keep, int32_t* status, void* scratch,
                                 int64_t scratch_bytes, void* stream) {
    int64_t need = 0;
    uva_boundary_mask_scratch_bytes(t < 0 ? 0 : t, &need);
    if (t < 0 || !status || (t > 0 && (!T || !keep || !scratch || scratch_bytes < need)) || 6 * t > 0x7fffffffll) {
        uva_set_error("uva_boundary_mask: bad arguments");
        return UVA_E_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(status, 0, 4, s);
    if (t == 0) { UVA_CHECK_LAUNCH("uva_boundary_mask"); return UVA_OK; }
    const uint32_t hmask = pow2_mask(2 * 3 * t);
    auto* table = static_cast<unsigned long long*>(scratch);
    cudaMemsetAsync(table, 0xff, 8 * (static_cast<size_t>(hmask) + 1), s);
    k_bm_insert<<<blocks_for(3 * t), kTB, 0, s>>>(T, t, table, hmask, status);
    k_bm_query<<<blocks_for(3 * t), kTB, 0, s>>>(T, t, table, hmask, keep);
    UVA_CHECK_LAUNCH("uva_boundary_mask");
    return UVA_OK;
}

extern "C" int uva_batch_edges(const uva_batch* b, int64_t* ea, int64_t* eb, int64_t* cnt, void* stream) {
    if (!b || b->t < 0 || b->E < 0 || (b->E > 0 && (!ea || !eb || !cnt || !b->tri_edge || !b->tri4 || !b->vofs))) {
        uva_set_error("uva_batch_edges: bad arguments");
        return UVA_E_ARG;
    }
    if (b->E == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(cnt, 0, 8 * static_cast<size_t>(b->E), s);
    k_batch_edges<<<blocks_for(3 * static_cast<int64_t>(b->t)), kTB, 0, s>>>(*b, ea, eb, cnt);
    UVA_CHECK_LAUNCH("uva_batch_edges");
    return UVA_OK;
}
