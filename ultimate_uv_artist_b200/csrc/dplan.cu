// Topology plan of a batch built on the device from the island-local
// triangle lists: the same arrays as the host plan (plan.cpp, uva_plan_*),
// element for element, without the host's per-island passes or their export
// and upload (the host ships 12 bytes per triangle instead of about 110).
//
// Steps (every id fits 32 bits; the host plan's limits apply):
//   1. tri4 and the global half-edges (corners k+1 -> k+2 of triangle f);
//   2. unique undirected edges in ascending global (lo, hi) order by a
//      counting sort on lo and an in-bucket rank (no general sort): this is
//      the host plan's numbering (island by island, (lo, hi) ascending);
//   3. per-edge use counts by direction, vertex flags, boundary sources;
//   4. vertex adjacency, ascending by neighbour: the edges with lo = v are
//      already in order, the ones with hi = v are placed by atomics and
//      sorted per vertex;
//   5. solver rows: compact breadth-first blobs of agg_rows vertices per
//      island, one warp per island walking the host plan's exact order
//      (lowest unplaced seed, neighbours in ascending order);
//   6. 32-row slices (width: the slice's largest degree rounded up to 4);
//   7. (second call, once the host has sized them) the sliced-ELL slots and
//      the vertex -> corner incidence.
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

#define GRID_STRIDE(i, count)                                                              \
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < (count); \
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)

// status bits
constexpr int kBadIndex = 1;     // a local vertex id outside its island
constexpr int kManyUses = 2;     // an edge used by more than 127 triangles in one direction
constexpr int kBadRows = 4;      // the row walk ran out of vertices (cannot happen for a valid plan)

// Scratch of the two calls (kept by the caller between them).
struct Scratch {
    int32_t* bstart;   // n+1  half-edges per smaller endpoint -> bucket offsets
    int32_t* bcur;     // n+1  fill cursors; later lower-neighbour cursors
    int32_t* bucket;   // H    half-edge of each bucket entry
    int32_t* bhi;      // H    larger endpoint of each entry
    uint8_t* first;    // H    entry is the first of its (lo, hi)
    int32_t* same;     // H    entries sharing the entry's (lo, hi)
    int32_t* uofs;     // n+1  distinct edges per lo -> first edge id of lo
    int32_t* e_lo;     // H    edge endpoints (global), use counts by direction
    int32_t* e_hi;
    int32_t* e_cnt;
    int32_t* e_fwd;
    int32_t* e_rev;
    int32_t* lowcnt;   // n    neighbours below the vertex
    int32_t* deg;      // n+1  neighbours -> row_ptr
    int32_t* adj;      // 2H   neighbour (island-local id) per adjacency entry
    int32_t* adj_e;    // 2H   edge of the entry
    int32_t* vflag32;  // n    vertex flags (32-bit for atomicOr)
    int32_t* isb;      // n+1  boundary source flag -> compact offsets
    uint8_t* bfs;      // n    BFS state: 1 placed, 2 queued
    int32_t* queue;    // n    BFS queue (island segments)
    int32_t* swidth;   // nslices+1  slots per slice -> slice offsets (host array owns them)
    int32_t* vcnt;     // n+1  corners per vertex -> cursor
    int32_t* sums;     // scan partials
    int32_t* status;   // 1
    int32_t* vbase;    // n    first global vertex of the vertex's island
};

struct Layout {
    int64_t off[25];
    int64_t total;
};

Layout layout(int64_t n, int64_t t, int64_t nslices) {
    // per-vertex arrays hold n + 2 entries: [v + 1] stays inside for any v <= n
    const int64_t N1 = n + 2, H = std::max<int64_t>(3 * t, 1), S1 = nslices + 1;
    const int64_t sums = std::max(xscan_sums(std::max(N1, S1)), xscan_sums(N1));
    const int64_t sz[25] = {4 * N1, 4 * N1, 4 * H, 4 * H, H, 4 * H, 4 * N1, 4 * H, 4 * H, 4 * H, 4 * H, 4 * H,
                            4 * N1, 4 * N1, 8 * H, 8 * H, 4 * N1, 4 * N1, N1, 4 * N1, 4 * S1, 4 * N1, 4 * sums, 256,
                            4 * N1};
    Layout L{};
    int64_t o = 0;
    for (int i = 0; i < 25; ++i) { L.off[i] = o; o += al(sz[i]); }
    L.total = o;
    return L;
}

Scratch carve(void* base, const Layout& L) {
    auto* b = static_cast<unsigned char*>(base);
    auto I = [&](int k) { return reinterpret_cast<int32_t*>(b + L.off[k]); };
    Scratch s;
    s.bstart = I(0); s.bcur = I(1); s.bucket = I(2); s.bhi = I(3);
    s.first = reinterpret_cast<uint8_t*>(b + L.off[4]);
    s.same = I(5); s.uofs = I(6); s.e_lo = I(7); s.e_hi = I(8); s.e_cnt = I(9); s.e_fwd = I(10); s.e_rev = I(11);
    s.lowcnt = I(12); s.deg = I(13); s.adj = I(14); s.adj_e = I(15); s.vflag32 = I(16); s.isb = I(17);
    s.bfs = reinterpret_cast<uint8_t*>(b + L.off[18]);
    s.queue = I(19); s.swidth = I(20); s.vcnt = I(21); s.sums = I(22); s.status = I(23); s.vbase = I(24);
    return s;
}

}  // namespace

namespace {

// ------------------------------------------------------------------ 1. triangles
// tri4 = (a, b, c, island); an id outside its island is flagged and read as
// 0, so every later pass stays inside the arrays.
__global__ void k_dp_tri4(int32_t nc, const int32_t* vofs, const int32_t* tofs, const int32_t* T, int32_t* tri4,
                          int32_t* status) {
    for (int32_t i = blockIdx.x; i < nc; i += gridDim.x) {
        const int32_t n = vofs[i + 1] - vofs[i];
        for (int64_t c = 3 * static_cast<int64_t>(tofs[i]) + threadIdx.x; c < 3 * static_cast<int64_t>(tofs[i + 1]);
             c += blockDim.x) {
            int32_t v = T[c];
            if (v < 0 || v >= n) { atomicOr(status, kBadIndex); v = 0; }
            const int64_t f = c / 3;
            tri4[4 * f + (c - 3 * f)] = v;
        }
        for (int64_t f = tofs[i] + threadIdx.x; f < tofs[i + 1]; f += blockDim.x) tri4[4 * f + 3] = i;
    }
}

// Half-edge h = 3 f + k: corners (k+1, k+2) of triangle f, global ids.
__device__ __forceinline__ void half_edge(const int32_t* tri4, const int32_t* vofs, int64_t h, int32_t& a,
                                          int32_t& b) {
    const int64_t f = h / 3;
    const int k = static_cast<int>(h - 3 * f);
    const int4 tv = reinterpret_cast<const int4*>(tri4)[f];
    const int32_t v0 = vofs[tv.w];
    const int32_t c[3] = {tv.x, tv.y, tv.z};
    a = v0 + c[(k + 1) % 3];
    b = v0 + c[(k + 2) % 3];
}

// ------------------------------------------------------------------ 2. unique edges
__global__ void k_dp_count(int64_t H, const int32_t* tri4, const int32_t* vofs, int32_t* bcnt, const int32_t* status) {
    if (*status & kBadIndex) return;   // every later pass stops at a bad index
    GRID_STRIDE(h, H) {
        int32_t a, b;
        half_edge(tri4, vofs, h, a, b);
        atomicAdd(bcnt + min(a, b), 1);
    }
}

__global__ void k_dp_fill(int64_t H, const int32_t* tri4, const int32_t* vofs, int32_t* cursor, int32_t* bucket,
                          int32_t* bhi, const int32_t* status) {
    if (*status & kBadIndex) return;
    GRID_STRIDE(h, H) {
        int32_t a, b;
        half_edge(tri4, vofs, h, a, b);
        const int32_t p = atomicAdd(cursor + min(a, b), 1);
        bucket[p] = static_cast<int32_t>(h);
        bhi[p] = max(a, b);
    }
}

__device__ __forceinline__ int32_t bucket_lo(const int32_t* tri4, const int32_t* vofs, int32_t h) {
    int32_t a, b;
    half_edge(tri4, vofs, h, a, b);
    return min(a, b);
}

// first: the entry is the smallest half-edge of its (lo, hi); same: the
// entries of its (lo, hi); the distinct his of every lo are counted.
__global__ void k_dp_first(int64_t H, const int32_t* tri4, const int32_t* vofs, const int32_t* bstart,
                           const int32_t* bucket, const int32_t* bhi, uint8_t* first, int32_t* same, int32_t* ucnt,
                           const int32_t* status) {
    if (*status & kBadIndex) return;
    GRID_STRIDE(p, H) {
        const int32_t h = bucket[p], hi = bhi[p];
        const int32_t lo = bucket_lo(tri4, vofs, h);
        bool is_first = true;
        int32_t cnt = 0;
        for (int32_t q = bstart[lo]; q < bstart[lo + 1]; ++q) {
            if (bhi[q] != hi) continue;
            ++cnt;
            if (bucket[q] < h) is_first = false;
        }
        first[p] = is_first ? 1 : 0;
        same[p] = cnt;
        if (is_first) atomicAdd(ucnt + lo, 1);
    }
}

// Edge ids (uofs[lo] + rank of hi among lo's distinct his), tri_edge, and the
// per-edge endpoints and use counts by direction (fwd: lo -> hi or a
// self-loop; rev: hi -> lo).
__global__ void k_dp_edges(int64_t H, const int32_t* tri4, const int32_t* vofs, const int32_t* bstart,
                           const int32_t* bucket, const int32_t* bhi, const uint8_t* first, const int32_t* same,
                           const int32_t* uofs, int32_t* tri_edge, int32_t* e_lo, int32_t* e_hi, int32_t* e_cnt,
                           int32_t* e_fwd, int32_t* e_rev, int32_t* status) {
    if (*status & kBadIndex) return;
    GRID_STRIDE(p, H) {
        const int32_t h = bucket[p], hi = bhi[p];
        const int32_t lo = bucket_lo(tri4, vofs, h);
        int32_t rank = 0;
        for (int32_t q = bstart[lo]; q < bstart[lo + 1]; ++q) rank += (first[q] && bhi[q] < hi) ? 1 : 0;
        const int32_t e = uofs[lo] + rank;
        tri_edge[h] = e;
        if (first[p]) {
            int32_t fwd = 0, rev = 0;
            for (int32_t q = bstart[lo]; q < bstart[lo + 1]; ++q) {
                if (bhi[q] != hi) continue;
                int32_t a, b;
                half_edge(tri4, vofs, bucket[q], a, b);
                if (a <= b) ++fwd; else ++rev;
            }
            e_lo[e] = lo;
            e_hi[e] = hi;
            e_cnt[e] = same[p];
            e_fwd[e] = fwd;
            e_rev[e] = rev;
            if (fwd > 127 || rev > 127) atomicOr(status, kManyUses);
        }
    }
}

// ------------------------------------------------------------------ 3. flags and degrees
// vflags bit 0: endpoint of an edge used once; bit 1: endpoint of an edge
// used in one direction only; isb: the source of such an edge's half-edges.
__global__ void k_dp_edge_flags(const int32_t* E_ptr, const int32_t* e_lo, const int32_t* e_hi, const int32_t* e_cnt,
                                const int32_t* e_fwd, const int32_t* e_rev, int32_t* vflag, int32_t* isb,
                                int32_t* lowcnt, int32_t* deg, const int32_t* status) {
    if (*status & kBadIndex) return;
    const int32_t E = *E_ptr;
    GRID_STRIDE(e, E) {
        const int32_t lo = e_lo[e], hi = e_hi[e];
        if (e_cnt[e] == 1) { atomicOr(vflag + lo, 1); atomicOr(vflag + hi, 1); }
        if (lo == hi) continue;
        atomicAdd(deg + lo, 1);
        atomicAdd(deg + hi, 1);
        atomicAdd(lowcnt + hi, 1);
        const int32_t f = e_fwd[e], r = e_rev[e];
        // bit 2 (not exported): the vertex is a boundary source; isb counts it once
        if (f > 0 && r == 0) {
            atomicOr(vflag + lo, 2); atomicOr(vflag + hi, 2);
            if (!(atomicOr(vflag + lo, 4) & 4)) isb[lo] = 1;
        }
        if (r > 0 && f == 0) {
            atomicOr(vflag + lo, 2); atomicOr(vflag + hi, 2);
            if (!(atomicOr(vflag + hi, 4) & 4)) isb[hi] = 1;
        }
    }
}

// ------------------------------------------------------------------ 4. adjacency
// Row v: its lower neighbours (edges with hi = v, placed by atomics, sorted
// below), then its upper ones (edges with lo = v: ids uofs[v].. in ascending
// hi order, the self-loop (v, v) first when present). Neighbours are stored
// as island-local ids.
__global__ void k_dp_adj(const int32_t* E_ptr, const int32_t* e_lo, const int32_t* e_hi, const int32_t* uofs,
                         const int32_t* row_ptr, const int32_t* lowcnt, const int32_t* vert_base, int32_t* lcur,
                         int32_t* adj, int32_t* adj_e, const int32_t* status) {
    if (*status & kBadIndex) return;
    const int32_t E = *E_ptr;
    GRID_STRIDE(e, E) {
        const int32_t lo = e_lo[e], hi = e_hi[e];
        if (lo == hi) continue;
        const int32_t base = vert_base[lo];   // first global vertex of the island
        const int32_t e0 = uofs[lo];
        const int32_t self = e_hi[e0] == lo ? 1 : 0;   // the self-loop of lo sorts first
        const int32_t up = row_ptr[lo] + lowcnt[lo] + (e - e0 - self);
        adj[up] = hi - base;
        adj_e[up] = e;
        const int32_t dn = row_ptr[hi] + atomicAdd(lcur + hi, 1);
        adj[dn] = lo - base;
        adj_e[dn] = e;
    }
}

// Insertion sort of every row's lower part by neighbour (a handful each).
__global__ void k_dp_sort_lower(int64_t n, const int32_t* row_ptr, const int32_t* lowcnt, int32_t* adj,
                                int32_t* adj_e) {
    GRID_STRIDE(v, n) {
        const int32_t a = row_ptr[v], m = lowcnt[v];
        for (int32_t i = 1; i < m; ++i) {
            const int32_t c = adj[a + i], e = adj_e[a + i];
            int32_t j = i - 1;
            while (j >= 0 && adj[a + j] > c) { adj[a + j + 1] = adj[a + j]; adj_e[a + j + 1] = adj_e[a + j]; --j; }
            adj[a + j + 1] = c;
            adj_e[a + j + 1] = e;
        }
    }
}

// island of every vertex (as its first global vertex) and of every row
__global__ void k_dp_vert_base(int32_t nc, const int32_t* vofs, int32_t* vert_base) {
    for (int32_t i = blockIdx.x; i < nc; i += gridDim.x)
        for (int32_t v = vofs[i] + threadIdx.x; v < vofs[i + 1]; v += blockDim.x) vert_base[v] = vofs[i];
}

}  // namespace

namespace {

// ------------------------------------------------------------------ 5. solver rows
// One warp per island. Islands with agg_rows = 0 keep the vertex order.
// Otherwise rows are compact breadth-first blobs: every blob of agg_rows
// rows grows from the lowest unplaced vertex; when its component runs out
// the blob continues from the next lowest one; when the blob is full, the
// queued but unplaced vertices are released for later blobs. A vertex's
// neighbours join the queue in ascending order (a ballot and a prefix count
// keep the order across lanes). st: bit 0 placed, bit 1 queued. Islands of
// up to kBlobCap vertices keep st and the queue in shared memory (the walk
// is one dependent chain per vertex, so each global round trip taken out of
// it counts); larger ones use the global scratch.
constexpr int kBlobCap = 8192;
constexpr size_t kBlobSmem = 5 * static_cast<size_t>(kBlobCap);   // st bytes, then the queue (ints)

__global__ void __launch_bounds__(32) k_dp_blob(int32_t nc, const int32_t* vofs, const int32_t* agg_rows,
                                                const int32_t* row_ptr, const int32_t* adj, uint8_t* st,
                                                int32_t* queue, int32_t* row_vert, int32_t* status) {
    extern __shared__ __align__(16) unsigned char blob_smem[];
    if (*status & kBadIndex) return;
    const int lane = threadIdx.x;
    constexpr unsigned kAll = 0xffffffffu;
    for (int32_t i = blockIdx.x; i < nc; i += gridDim.x) {
        const int32_t v0 = vofs[i], n = vofs[i + 1] - v0, agg = agg_rows[i];
        int32_t* rv = row_vert + v0;
        if (agg <= 0) {
            for (int32_t v = lane; v < n; v += 32) rv[v] = v;
            continue;
        }
        const bool local = n <= kBlobCap;
        uint8_t* s = local ? blob_smem : st + v0;
        int32_t* q = local ? reinterpret_cast<int32_t*>(blob_smem + kBlobCap) : queue + v0;
        if (local) {
            for (int32_t v = lane; v < n; v += 32) s[v] = 0;
            __syncwarp();
        }
        const int32_t* rp = row_ptr + v0;
        int32_t norder = 0, seed = 0;
        while (norder < n) {
            const int32_t target = min(n, norder + agg);
            while (norder < target) {
                bool found = false;
                while (seed < n) {   // the lowest unplaced vertex from seed on (one exists: norder < n)
                    const int32_t c = seed + lane;
                    const bool open = c < n && !(s[c] & 1);
                    const unsigned m = __ballot_sync(kAll, open);
                    if (m) { seed += __ffs(m) - 1; found = true; break; }
                    seed += 32;
                }
                if (!found) {   // cannot happen for a valid plan: stop the island, report it
                    if (lane == 0) atomicOr(status, kBadRows);
                    norder = n;
                    break;
                }
                int32_t qlen = 1, head = 0;
                if (lane == 0) { q[0] = seed; s[seed] |= 2; }
                __syncwarp();
                while (head < qlen && norder < target) {
                    const int32_t v = q[head++];
                    if (lane == 0) { s[v] |= 1; rv[norder] = v; }
                    ++norder;
                    __syncwarp();
                    const int32_t a = __ldg(rp + v), b = __ldg(rp + v + 1);
                    for (int32_t k0 = a; k0 < b; k0 += 32) {
                        const int32_t k = k0 + lane;
                        int32_t w = 0;
                        bool take = false;
                        if (k < b) { w = __ldg(adj + k); take = (s[w] & 3) == 0; }
                        const unsigned m = __ballot_sync(kAll, take);
                        if (take) {
                            q[qlen + __popc(m & ((1u << lane) - 1u))] = w;
                            s[w] |= 2;
                        }
                        qlen += __popc(m);
                        __syncwarp();
                    }
                }
                for (int32_t j = lane; j < qlen; j += 32) s[q[j]] &= static_cast<uint8_t>(~2u);
                __syncwarp();
            }
        }
    }
}

// vert_row = inverse of row_vert inside every island (vert_base: the
// island's first global vertex).
__global__ void k_dp_vert_row(int64_t n, const int32_t* vert_base, const int32_t* row_vert, int32_t* vert_row,
                              const int32_t* status) {
    if (*status & (kBadIndex | kBadRows)) return;
    GRID_STRIDE(g, n) {
        const int32_t b = vert_base[g];
        vert_row[b + row_vert[g]] = static_cast<int32_t>(g - b);
    }
}

// ------------------------------------------------------------------ 6. slices
// One warp per 32-row slice: slots = 32 x (largest degree, rounded up to 4).
__global__ void k_dp_slice_width(int32_t nc, const int32_t* vofs, const int32_t* sofs, const int32_t* row_vert,
                                 const int32_t* row_ptr, int32_t* swidth, const int32_t* status) {
    if (*status & (kBadIndex | kBadRows)) return;
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x / 32);
    const int32_t S = sofs[nc];
    for (int64_t s = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) / 32; s < S; s += warps) {
        int32_t lo = 0, hi = nc;   // island of slice s: sofs[lo] <= s < sofs[lo + 1]
        while (hi - lo > 1) { const int32_t mid = (lo + hi) >> 1; if (sofs[mid] <= s) lo = mid; else hi = mid; }
        const int32_t v0 = vofs[lo], n = vofs[lo + 1] - v0;
        const int32_t row = static_cast<int32_t>(s - sofs[lo]) * 32 + lane;
        int32_t d = 0;
        if (row < n) {
            const int32_t v = v0 + row_vert[v0 + row];
            d = row_ptr[v + 1] - row_ptr[v];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_xor_sync(0xffffffffu, d, o));
        if (lane == 0) swidth[s] = 32 * ((d + 3) & ~3);
    }
}

// ------------------------------------------------------------------ boundary sources and flags
__global__ void k_dp_bverts(int64_t n, const int32_t* vert_base, const int32_t* vflag32, const int32_t* isb_ofs,
                            int32_t* bverts) {
    GRID_STRIDE(v, n) {
        if (vflag32[v] & 4) bverts[isb_ofs[v]] = static_cast<int32_t>(v - vert_base[v]);
    }
}

// bofs[i] = boundary sources before island i (vofs[nc] = n: the total).
__global__ void k_dp_bofs(int32_t nc, const int32_t* vofs, const int32_t* isb_ofs, int32_t* bofs) {
    GRID_STRIDE(i, static_cast<int64_t>(nc) + 1) { bofs[i] = isb_ofs[vofs[i]]; }
}

__global__ void k_dp_vflags(int64_t n, const int32_t* vflag32, uint8_t* vflags) {
    GRID_STRIDE(v, n) { vflags[v] = static_cast<uint8_t>(vflag32[v] & 3); }
}

// ------------------------------------------------------------------ vertex -> corner incidence
__global__ void k_dp_vt_count(int64_t t, const int32_t* tri4, const int32_t* vofs, int32_t* vcnt, const int32_t* status) {
    if (*status & kBadIndex) return;
    GRID_STRIDE(c, 3 * t) {
        const int64_t f = c / 3;
        const int32_t v0 = vofs[tri4[4 * f + 3]];
        atomicAdd(vcnt + v0 + tri4[4 * f + (c - 3 * f)], 1);
    }
}

__global__ void k_dp_vt_fill(int64_t t, const int32_t* tri4, const int32_t* vofs, int32_t* cursor, int32_t* vt,
                             const int32_t* status) {
    if (*status & kBadIndex) return;
    GRID_STRIDE(c, 3 * t) {
        const int64_t f = c / 3;
        const int32_t v0 = vofs[tri4[4 * f + 3]];
        vt[atomicAdd(cursor + v0 + tri4[4 * f + (c - 3 * f)], 1)] = static_cast<int32_t>(c);
    }
}

// corners of a vertex ascending (the host plan fills them in corner order)
__global__ void k_dp_vt_sort(int64_t n, const int32_t* vt_ptr, int32_t* vt) {
    GRID_STRIDE(v, n) {
        const int32_t a = vt_ptr[v], m = vt_ptr[v + 1] - a;
        for (int32_t i = 1; i < m; ++i) {
            const int32_t c = vt[a + i];
            int32_t j = i - 1;
            while (j >= 0 && vt[a + j] > c) { vt[a + j + 1] = vt[a + j]; --j; }
            vt[a + j + 1] = c;
        }
    }
}

// ------------------------------------------------------------------ 7. slots
// Slot k of row r sits at slice_ptr[s] + 32 k + lane: the row's k-th
// neighbour (ascending vertex id) as its solver row, the edge, and the LSCM
// boundary coupling of the pair (half-edges r -> j without a twin give
// -1/2, j -> r without a twin +1/2, as H[i, j+n] of engine/param.py:147-150).
// Padding slots: weight 0, the row itself (0 past the island's end).
__global__ void k_dp_slots(int32_t nc, const int32_t* vofs, const int32_t* sofs, const int32_t* slice_ptr,
                           const int32_t* row_vert, const int32_t* vert_row, const int32_t* row_ptr,
                           const int32_t* adj, const int32_t* adj_e, const int32_t* e_fwd, const int32_t* e_rev,
                           int32_t* slot_col, int32_t* slot_edge, float* slot_c) {
    const int32_t S = sofs[nc];
    GRID_STRIDE(g, static_cast<int64_t>(S) * 32) {
        const int64_t s = g >> 5;
        const int lane = static_cast<int>(g & 31);
        int32_t lo = 0, hi = nc;
        while (hi - lo > 1) { const int32_t mid = (lo + hi) >> 1; if (sofs[mid] <= s) lo = mid; else hi = mid; }
        const int32_t v0 = vofs[lo], n = vofs[lo + 1] - v0;
        const int32_t row = static_cast<int32_t>(s - sofs[lo]) * 32 + lane;
        const int32_t base = slice_ptr[s], w = (slice_ptr[s + 1] - base) / 32;
        int32_t k = 0;
        if (row < n) {
            const int32_t r = row_vert[v0 + row];
            const int32_t a = row_ptr[v0 + r], deg = row_ptr[v0 + r + 1] - a;
            for (; k < deg; ++k) {
                const int64_t q = base + static_cast<int64_t>(k) * 32 + lane;
                const int32_t j = adj[a + k], e = adj_e[a + k];
                slot_col[q] = vert_row[v0 + j];
                slot_edge[q] = e;
                const int32_t nf = e_fwd[e], nr = e_rev[e];
                const int32_t n_rj = r < j ? nf : nr, n_jr = r < j ? nr : nf;
                const int32_t b_rj = n_jr == 0 ? n_rj : 0, b_jr = n_rj == 0 ? n_jr : 0;
                slot_c[q] = -0.5f * static_cast<float>(b_rj) + 0.5f * static_cast<float>(b_jr);
            }
        }
        for (; k < w; ++k) {
            const int64_t q = base + static_cast<int64_t>(k) * 32 + lane;
            slot_col[q] = row < n ? row : 0;
            slot_edge[q] = -1;
            slot_c[q] = 0.0f;
        }
    }
}

__global__ void k_dp_sizes(const int32_t* E_ptr, const int32_t* slice_ptr, int32_t nslices, const int32_t* bofs,
                           int32_t nc, const int32_t* status, int64_t* sizes) {
    sizes[0] = *E_ptr;
    sizes[1] = slice_ptr[nslices];
    sizes[2] = bofs[nc];
    sizes[3] = *status;
}

}  // namespace

// ==================================================================== C ABI
extern "C" int uva_dplan_scratch_bytes(int64_t n, int64_t t, int64_t nslices, int64_t* bytes) {
    if (n < 0 || t < 0 || nslices < 0 || !bytes) {
        uva_set_error("uva_dplan_scratch_bytes: bad arguments");
        return UVA_E_ARG;
    }
    *bytes = layout(n, t, nslices).total;
    return UVA_OK;
}

namespace {
bool dplan_ok(const uva_dplan* d, const char* who) {
    if (!d || d->nc < 0 || d->n < 0 || d->t < 0 || d->nslices < 0 || !d->sizes || !d->scratch ||
        (d->nc > 0 && (!d->vofs || !d->tofs || !d->agg_rows || !d->sofs || !d->row_vert || !d->vert_row ||
                       !d->bofs || !d->vt_ptr || !d->slice_ptr)) ||
        (d->t > 0 && (!d->T || !d->tri4 || !d->tri_edge || !d->vt)) || (d->n > 0 && (!d->vflags || !d->bverts)) ||
        static_cast<int64_t>(d->n) > (int64_t(1) << 30) || 3 * static_cast<int64_t>(d->t) > (int64_t(1) << 30) ||
        d->scratch_bytes < layout(d->n, d->t, d->nslices).total) {
        uva_set_error(who);
        return false;
    }
    return true;
}
}  // namespace

extern "C" int uva_dplan_build(const uva_dplan* d, void* stream) {
    if (!dplan_ok(d, "uva_dplan_build: bad arguments or scratch too small")) return UVA_E_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Layout L = layout(d->n, d->t, d->nslices);
    Scratch s = carve(d->scratch, L);
    const int64_t n = d->n, t = d->t, H = 3 * t;
    const int32_t nc = d->nc;
    cudaMemsetAsync(d->scratch, 0, static_cast<size_t>(L.total), st);
    if (n > 0) cudaMemsetAsync(d->row_vert, 0, 4 * static_cast<size_t>(n), st);   // in range whatever happens
    if (nc == 0) {
        cudaMemsetAsync(d->sizes, 0, 4 * sizeof(int64_t), st);
        UVA_CHECK_LAUNCH("uva_dplan_build");
        return UVA_OK;
    }
    const unsigned gi = static_cast<unsigned>(std::min<int32_t>(nc, 65535));
    // 1. triangles; the island of every vertex
    k_dp_tri4<<<gi, kTB, 0, st>>>(nc, d->vofs, d->tofs, d->T, d->tri4, s.status);
    k_dp_vert_base<<<gi, kTB, 0, st>>>(nc, d->vofs, s.vbase);
    // 2. unique edges
    k_dp_count<<<blocks_for(H), kTB, 0, st>>>(H, d->tri4, d->vofs, s.bstart, s.status);
    xscan<int32_t>(s.bstart, s.bstart, s.sums, nullptr, n + 1, st);
    cudaMemcpyAsync(s.bcur, s.bstart, 4 * static_cast<size_t>(n + 1), cudaMemcpyDeviceToDevice, st);
    k_dp_fill<<<blocks_for(H), kTB, 0, st>>>(H, d->tri4, d->vofs, s.bcur, s.bucket, s.bhi, s.status);
    k_dp_first<<<blocks_for(H), kTB, 0, st>>>(H, d->tri4, d->vofs, s.bstart, s.bucket, s.bhi, s.first, s.same, s.uofs,
                                              s.status);
    xscan<int32_t>(s.uofs, s.uofs, s.sums, nullptr, n + 1, st);   // uofs[n] = E
    k_dp_edges<<<blocks_for(H), kTB, 0, st>>>(H, d->tri4, d->vofs, s.bstart, s.bucket, s.bhi, s.first, s.same, s.uofs,
                                              d->tri_edge, s.e_lo, s.e_hi, s.e_cnt, s.e_fwd, s.e_rev, s.status);
    const int32_t* E_ptr = s.uofs + n;
    // 3. flags, degrees
    k_dp_edge_flags<<<blocks_for(H), kTB, 0, st>>>(E_ptr, s.e_lo, s.e_hi, s.e_cnt, s.e_fwd, s.e_rev, s.vflag32, s.isb,
                                                   s.lowcnt, s.deg, s.status);
    xscan<int32_t>(s.deg, s.deg, s.sums, nullptr, n + 1, st);     // deg -> row_ptr
    const int32_t* row_ptr = s.deg;
    // 4. adjacency (bcur reused as the lower-neighbour cursors)
    cudaMemsetAsync(s.bcur, 0, 4 * static_cast<size_t>(n + 1), st);
    k_dp_adj<<<blocks_for(H), kTB, 0, st>>>(E_ptr, s.e_lo, s.e_hi, s.uofs, row_ptr, s.lowcnt, s.vbase, s.bcur, s.adj,
                                            s.adj_e, s.status);
    k_dp_sort_lower<<<blocks_for(n), kTB, 0, st>>>(n, row_ptr, s.lowcnt, s.adj, s.adj_e);
    // boundary sources and vertex flags
    xscan<int32_t>(s.isb, s.isb, s.sums, nullptr, n + 1, st);     // isb -> offsets (flags in vflag32 bit 2)
    k_dp_bverts<<<blocks_for(n), kTB, 0, st>>>(n, s.vbase, s.vflag32, s.isb, d->bverts);
    k_dp_bofs<<<blocks_for(nc + 1), kTB, 0, st>>>(nc, d->vofs, s.isb, d->bofs);
    k_dp_vflags<<<blocks_for(n), kTB, 0, st>>>(n, s.vflag32, d->vflags);
    UVA_CHECK_LAUNCH("uva_dplan_build/edges");
    // 5. solver rows
    k_dp_blob<<<gi, 32, kBlobSmem, st>>>(nc, d->vofs, d->agg_rows, row_ptr, s.adj, s.bfs, s.queue, d->row_vert,
                                         s.status);
    k_dp_vert_row<<<blocks_for(n), kTB, 0, st>>>(n, s.vbase, d->row_vert, d->vert_row, s.status);
    // 6. slices
    if (d->nslices > 0)
        k_dp_slice_width<<<blocks_for(32 * static_cast<int64_t>(d->nslices)), kTB, 0, st>>>(
            nc, d->vofs, d->sofs, d->row_vert, row_ptr, s.swidth, s.status);
    xscan<int32_t>(s.swidth, d->slice_ptr, s.sums, nullptr, static_cast<int64_t>(d->nslices) + 1, st);
    // vertex -> corner incidence
    k_dp_vt_count<<<blocks_for(H), kTB, 0, st>>>(t, d->tri4, d->vofs, s.vcnt, s.status);
    xscan<int32_t>(s.vcnt, d->vt_ptr, s.sums, nullptr, n + 1, st);
    cudaMemcpyAsync(s.vcnt, d->vt_ptr, 4 * static_cast<size_t>(n + 1), cudaMemcpyDeviceToDevice, st);
    k_dp_vt_fill<<<blocks_for(H), kTB, 0, st>>>(t, d->tri4, d->vofs, s.vcnt, d->vt, s.status);
    k_dp_vt_sort<<<blocks_for(n), kTB, 0, st>>>(n, d->vt_ptr, d->vt);
    k_dp_sizes<<<1, 1, 0, st>>>(E_ptr, d->slice_ptr, d->nslices, d->bofs, nc, s.status, d->sizes);
    UVA_CHECK_LAUNCH("uva_dplan_build");
    return UVA_OK;
}

extern "C" int uva_dplan_slots(const uva_dplan* d, int32_t* slot_col, int32_t* slot_edge, float* slot_c,
                               void* stream) {
    if (!dplan_ok(d, "uva_dplan_slots: bad arguments or scratch too small")) return UVA_E_ARG;
    if (d->nc == 0 || d->nslices == 0) return UVA_OK;
    if (!slot_col || !slot_edge || !slot_c) { uva_set_error("uva_dplan_slots: null slot arrays"); return UVA_E_ARG; }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Scratch s = carve(d->scratch, layout(d->n, d->t, d->nslices));
    k_dp_slots<<<blocks_for(32 * static_cast<int64_t>(d->nslices)), kTB, 0, st>>>(
        d->nc, d->vofs, d->sofs, d->slice_ptr, d->row_vert, d->vert_row, s.deg, s.adj, s.adj_e, s.e_fwd, s.e_rev,
        slot_col, slot_edge, slot_c);
    UVA_CHECK_LAUNCH("uva_dplan_slots");
    return UVA_OK;
}
