// Boundary self-intersection checks of UV charts, batched over charts
// (engine/charts.py:547-608 boundary_intersections / _seg_intersections,
// engine/hier.py:183-266 charts_collide / _hit, used by chart_checks
// :270-353). Modes: COUNT (the capped count), ANY (any crossing, charts whose
// extent is not below 1e300 collide), ANY_ALL (any crossing, no extent test).
//
// Compiled with --fmad=false: the segment predicate rounds every FP64
// operation like the reference's numba kernels, so counts are bit-exact.
//
// The reference bins a chart's segments into a uniform grid and tests every
// pair inside every cell, so a crossing pair is counted once per cell the two
// cell boxes share. A crossing needs intersecting bounding boxes, hence at
// least one shared cell, so the count equals the sum over crossing pairs of
// (shared cells in x) * (shared cells in y), and "any crossing" needs no grid
// at all. Here every pair of a chart is visited once, in tiles:
//   k_seg_prep   one CTA per chart: extent, median segment length (radix
//                select), the reference's grid, the cell box of every segment
//   k_seg_scan   tile pairs per chart -> offsets (one CTA)
//   k_seg_pairs  persistent CTAs over (chart, tile i <= tile j) work items:
//                two tiles of 128 segments in shared memory, 16,384 pair
//                tests, one atomic per item and chart
//   k_seg_final  cap / flags -> out
// Counts stop growing in effect at the cap: a work item of a chart whose
// count has reached it is skipped (the capped result is the same).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"

using namespace uva;

namespace {

constexpr int kTile = 128;          // segments per tile
constexpr int kPrep = 256;          // threads of k_seg_prep
constexpr int kPair = 256;          // threads of k_seg_pairs
constexpr int kScan = 1024;         // threads of k_seg_scan
constexpr int kRankMax = 1024;      // charts up to this many segments: one-pass rank select

enum : int32_t { kFlagNone = 0, kFlagNonFinite = 1, kFlagRange = 2 };

struct ChartGrid {
    double lo0, lo1, cell;
    int32_t nx, ny;
    int32_t tiles;   // tiles of kTile segments to test (0: none)
    int32_t flag;
};

struct Layout {
    size_t grid, hits, tile_ofs, box, len, total;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

Layout layout(int64_t nc, int64_t nseg) {
    Layout L;
    size_t o = 0;
    L.grid = o;     o = align16(o + sizeof(ChartGrid) * static_cast<size_t>(std::max<int64_t>(nc, 1)));
    L.hits = o;     o = align16(o + 8 * static_cast<size_t>(std::max<int64_t>(nc, 1)));
    L.tile_ofs = o; o = align16(o + 8 * static_cast<size_t>(nc + 1));
    L.box = o;      o = align16(o + sizeof(int4) * static_cast<size_t>(std::max<int64_t>(nseg, 1)));
    L.len = o;      o = align16(o + 8 * static_cast<size_t>(std::max<int64_t>(nseg, 1)));
    L.total = o;
    return L;
}

__device__ __forceinline__ bool same_point(double2 p, double2 q) { return p.x == q.x && p.y == q.y; }
__device__ __forceinline__ int g_nx(const ChartGrid* grid, int c) { return grid[c].nx; }

// engine/charts.py:579-591 (the same test as engine/hier.py:251-264): segments
// i (a -> b) and j (c -> d) cross properly; endpoints with identical
// coordinates never count.
__device__ __forceinline__ bool seg_cross(double2 a, double2 b, double2 c, double2 d) {
    if (same_point(a, c) || same_point(a, d) || same_point(b, c) || same_point(b, d)) return false;
    const double d1x = b.x - a.x, d1y = b.y - a.y;
    const double d2x = d.x - c.x, d2y = d.y - c.y;
    const double o1 = d1x * (c.y - a.y) - d1y * (c.x - a.x);
    const double o2 = d1x * (d.y - a.y) - d1y * (d.x - a.x);
    const double o3 = d2x * (a.y - c.y) - d2y * (a.x - c.x);
    const double o4 = d2x * (b.y - c.y) - d2y * (b.x - c.x);
    const double tol1 = 1e-9 * (d1x * d1x + d1y * d1y);
    const double tol2 = 1e-9 * (d2x * d2x + d2y * d2y);
    return ((o1 > tol1 && o2 < -tol1) || (o1 < -tol1 && o2 > tol1)) &&
           ((o3 > tol2 && o4 < -tol2) || (o3 < -tol2 && o4 > tol2));
}

// k-th smallest (0-based) of m non-negative finite doubles: most significant
// byte first over their bit patterns (ordered like the values). Whole CTA;
// `hist` 256 ints and `sh` 2 words of shared memory.
__device__ double select_kth(const double* v, int m, int k, int* hist, unsigned long long* sh) {
    unsigned long long prefix = 0, mask = 0;
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const unsigned long long key = static_cast<unsigned long long>(__double_as_longlong(v[i]));
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = 0, dg = 0;
            for (; dg < 255; ++dg) {
                if (acc + hist[dg] > k) break;
                acc += hist[dg];
            }
            sh[0] = prefix | (static_cast<unsigned long long>(dg) << shift);
            sh[1] = static_cast<unsigned long long>(k - acc);
        }
        __syncthreads();
        prefix = sh[0];
        k = static_cast<int>(sh[1]);
        mask |= 255ull << shift;
        __syncthreads();   // sh and hist are rewritten by the next pass
    }
    return __longlong_as_double(static_cast<long long>(prefix));
}

template <typename T>
__device__ __forceinline__ T block_reduce(T v, T* red, bool is_min) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T y = __shfl_xor_sync(0xffffffffu, v, o);
        v = is_min ? (y < v ? y : v) : (y > v ? y : v);
    }
    __syncthreads();   // red may still be read by the previous reduction
    if (lane == 0) red[warp] = v;
    __syncthreads();
    T s = red[0];
    for (int w = 1; w < nw; ++w) s = is_min ? (red[w] < s ? red[w] : s) : (red[w] > s ? red[w] : s);
    return s;
}

__global__ void __launch_bounds__(kPrep) k_seg_prep(uva_seg_desc d, ChartGrid* grid, unsigned long long* hits,
                                                   int4* box, double* len) {
    __shared__ double redd[kPrep / 32];
    __shared__ int redi[kPrep / 32];
    __shared__ int hist[256];
    __shared__ unsigned long long sh[2];
    __shared__ double slen[kRankMax];
    __shared__ double ssel[2];
    __shared__ ChartGrid g;
    const double2* U = reinterpret_cast<const double2*>(d.U);
    for (int c = blockIdx.x; c < d.nc; c += gridDim.x) {
        const int s0 = d.seg_ofs[c], s1 = d.seg_ofs[c + 1];
        const int v0 = d.vofs ? d.vofs[c] : 0, v1 = d.vofs ? d.vofs[c + 1] : d.n;
        const bool gridded_mode = d.mode == UVA_SEG_COUNT || d.mode == UVA_SEG_FIRST;
        int bad = (s0 < 0 || s1 < s0 || s1 > d.nseg) ? kFlagRange : kFlagNone;
        if (gridded_mode && (v0 < 0 || v1 < v0 || v1 > d.n)) bad = kFlagRange;
        if (d.mode == UVA_SEG_FIRST && s1 - s0 >= (1 << 21)) bad = kFlagRange;   // 21-bit segment ids in the key
        const int m = bad ? 0 : s1 - s0;
        // every row a segment names lies in U (COUNT: in the chart's rows)
        const int lo_row = gridded_mode ? v0 : 0, hi_row = gridded_mode ? v1 : d.n;
        int rb = 0;
        for (int s = threadIdx.x; s < m; s += blockDim.x) {
            const int a = d.seg[2 * (s0 + s)], b = d.seg[2 * (s0 + s) + 1];
            rb |= (a < lo_row || a >= hi_row || b < lo_row || b >= hi_row) ? 1 : 0;
        }
        rb = block_reduce<int>(rb, redi, false);
        if (rb) bad = kFlagRange;
        double lo0 = INFINITY, lo1 = INFINITY, hi0 = -INFINITY, hi1 = -INFINITY;
        int nonfin = 0;
        if (!bad && m >= 3) {
            if (gridded_mode) {   // lo = U.min(0), ext = U.max(0) - lo over the chart's rows
                for (int v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
                    const double2 u = U[v];
                    nonfin |= finite2(u) ? 0 : 1;
                    lo0 = fmin(lo0, u.x); lo1 = fmin(lo1, u.y);
                    hi0 = fmax(hi0, u.x); hi1 = fmax(hi1, u.y);
                }
            } else {                         // over the segments' endpoints
                for (int s = threadIdx.x; s < m; s += blockDim.x) {
                    const double2 a = U[d.seg[2 * (s0 + s)]], b = U[d.seg[2 * (s0 + s) + 1]];
                    nonfin |= (finite2(a) && finite2(b)) ? 0 : 1;
                    lo0 = fmin(lo0, fmin(a.x, b.x)); lo1 = fmin(lo1, fmin(a.y, b.y));
                    hi0 = fmax(hi0, fmax(a.x, b.x)); hi1 = fmax(hi1, fmax(a.y, b.y));
                }
            }
            nonfin = block_reduce<int>(nonfin, redi, false);
            lo0 = block_reduce<double>(lo0, redd, true);
            lo1 = block_reduce<double>(lo1, redd, true);
            hi0 = block_reduce<double>(hi0, redd, false);
            hi1 = block_reduce<double>(hi1, redd, false);
        }
        if (gridded_mode && !bad && m >= 3 && !nonfin) {
            // L = |B - A| (np.linalg.norm(B - A, axis=1)), then its median
            const bool small = m <= kRankMax;
            for (int s = threadIdx.x; s < m; s += blockDim.x) {
                const double2 a = U[d.seg[2 * (s0 + s)]], b = U[d.seg[2 * (s0 + s) + 1]];
                const double dx = b.x - a.x, dy = b.y - a.y;
                const double l = sqrt(dx * dx + dy * dy);
                if (small) slen[s] = l; else len[s0 + s] = l;
            }
            __syncthreads();
            double med;
            if (small) {   // stable rank of every length; the middle one(s) publish their value
                const int k1 = (m & 1) ? m / 2 : m / 2 - 1, k2 = m / 2;
                for (int i = threadIdx.x; i < m; i += blockDim.x) {
                    const double v = slen[i];
                    int r = 0;
                    for (int j = 0; j < m; ++j) {
                        const double w = slen[j];
                        r += (w < v || (w == v && j < i)) ? 1 : 0;
                    }
                    if (r == k1) ssel[0] = v;
                    if (r == k2) ssel[1] = v;
                }
                __syncthreads();
                med = (m & 1) ? ssel[1] : (ssel[0] + ssel[1]) / 2.0;
            } else if (m & 1) {
                med = select_kth(len + s0, m, m / 2, hist, sh);
            } else {
                const double x0 = select_kth(len + s0, m, m / 2 - 1, hist, sh);
                const double x1 = select_kth(len + s0, m, m / 2, hist, sh);
                med = (x0 + x1) / 2.0;
            }
            if (threadIdx.x == 0) {
                const double ext0 = hi0 - lo0, ext1 = hi1 - lo1;
                // max(median * 4, ext.max() / 512, 1e-30); collision (FIRST): / 1024
                double cell = med * 4.0;
                const double e = (ext1 > ext0 ? ext1 : ext0) / (d.mode == UVA_SEG_FIRST ? 1024.0 : 512.0);
                if (e > cell) cell = e;
                if (1e-30 > cell) cell = 1e-30;
                g.lo0 = lo0; g.lo1 = lo1; g.cell = cell;
                g.nx = static_cast<int32_t>(ext0 / cell) + 1;
                g.ny = static_cast<int32_t>(ext1 / cell) + 1;
            }
            __syncthreads();
            const double glo0 = g.lo0, glo1 = g.lo1, gcell = g.cell;
            const int gnx = g.nx, gny = g.ny;
            for (int s = threadIdx.x; s < m; s += blockDim.x) {   // engine/charts.py:556-559
                const double2 a = U[d.seg[2 * (s0 + s)]], b = U[d.seg[2 * (s0 + s) + 1]];
                const int x0 = static_cast<int>((fmin(a.x, b.x) - glo0) / gcell);
                const int x1 = static_cast<int>((fmax(a.x, b.x) - glo0) / gcell);
                const int y0 = static_cast<int>((fmin(a.y, b.y) - glo1) / gcell);
                const int y1 = static_cast<int>((fmax(a.y, b.y) - glo1) / gcell);
                box[s0 + s] = make_int4(max(x0, 0), min(x1, gnx - 1), max(y0, 0), min(y1, gny - 1));
            }
        }
        if (threadIdx.x == 0) {
            ChartGrid& o = grid[c];
            const bool gridded = gridded_mode && !bad && m >= 3 && !nonfin;
            o.lo0 = gridded ? g.lo0 : 0.0; o.lo1 = gridded ? g.lo1 : 0.0; o.cell = gridded ? g.cell : 0.0;
            o.nx = gridded ? g.nx : 0; o.ny = gridded ? g.ny : 0;
            int flag = bad;
            if (!flag && m >= 3) {
                if (gridded_mode) {
                    if (nonfin) flag = kFlagNonFinite;
                } else {
                    const double ext0 = hi0 - lo0, ext1 = hi1 - lo1;
                    const double ext = ext1 > ext0 ? ext1 : ext0;
                    // engine/hier.py:344-346 (chart_checks only; charts_collide tests every pair)
                    if (d.mode == UVA_SEG_ANY && (nonfin || !(ext < 1e300))) flag = kFlagNonFinite;
                }
            }
            o.flag = flag;
            o.tiles = (!flag && m >= 3) ? (m + kTile - 1) / kTile : 0;
            hits[c] = d.mode == UVA_SEG_FIRST ? ~0ull : 0ull;
        }
        __syncthreads();   // g is rewritten for the next chart
    }
}

// tile_ofs[c] = sum over charts before c of T (T + 1) / 2, T = tiles of the chart
__global__ void __launch_bounds__(kScan) k_seg_scan(int nc, const ChartGrid* grid, int64_t* tile_ofs) {
    __shared__ long long part[kScan];
    const int per = (nc + kScan - 1) / kScan;
    const int c0 = threadIdx.x * per, c1 = min(nc, c0 + per);
    long long s = 0;
    for (int c = c0; c < c1; ++c) {
        const long long t = grid[c].tiles;
        s += t * (t + 1) / 2;
    }
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < kScan; o <<= 1) {   // inclusive Hillis-Steele scan
        const long long add = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    long long run = part[threadIdx.x] - s;
    for (int c = c0; c < c1; ++c) {
        tile_ofs[c] = run;
        const long long t = grid[c].tiles;
        run += t * (t + 1) / 2;
    }
    if (threadIdx.x == kScan - 1) tile_ofs[nc] = part[kScan - 1];
}

__global__ void __launch_bounds__(kPair) k_seg_pairs(uva_seg_desc d, const ChartGrid* grid, const int64_t* tile_ofs,
                                                    const int4* box, unsigned long long* hits) {
    __shared__ double2 sa[2][kTile], sb[2][kTile];
    __shared__ int4 sbox[2][kTile];
    __shared__ unsigned long long wsum[kPair / 32];
    __shared__ int item[5];   // chart, tile i, tile j, skip, first segment
    const double2* U = reinterpret_cast<const double2*>(d.U);
    const long long total = tile_ofs[d.nc];
    const unsigned long long cap = static_cast<unsigned long long>(d.max_report > 1 ? d.max_report : 1);
    const bool count = d.mode == UVA_SEG_COUNT, first = d.mode == UVA_SEG_FIRST;
    const bool boxes = count || first;
    for (long long w = blockIdx.x; w < total; w += gridDim.x) {
        __syncthreads();   // the previous item's shared data is consumed
        if (threadIdx.x == 0) {
            int lo = 0, hi = d.nc;   // tile_ofs[lo] <= w < tile_ofs[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (tile_ofs[mid] <= w) lo = mid; else hi = mid;
            }
            const int k = grid[lo].tiles;
            long long l = w - tile_ofs[lo];
            int ti = 0;
            while (ti < k - 1 && l >= k - ti) { l -= k - ti; ++ti; }
            item[0] = lo; item[1] = ti; item[2] = ti + static_cast<int>(l);
            const unsigned long long sofar = *reinterpret_cast<volatile unsigned long long*>(hits + lo);
            item[3] = first ? 0 : count ? (sofar >= cap) : (sofar > 0);
            item[4] = d.seg_ofs[lo];
        }
        __syncthreads();
        if (item[3]) continue;
        const int c = item[0], ti = item[1], tj = item[2], s0 = item[4];
        const int m = d.seg_ofs[c + 1] - s0;
        const int ni = min(kTile, m - ti * kTile), nj = min(kTile, m - tj * kTile);
        if (threadIdx.x < 2 * kTile) {
            const int t = threadIdx.x / kTile, q = threadIdx.x % kTile;
            const int nq = t ? nj : ni, base = (t ? tj : ti) * kTile;
            if (q < nq) {
                const int s = s0 + base + q;
                sa[t][q] = U[d.seg[2 * s]];
                sb[t][q] = U[d.seg[2 * s + 1]];
                if (boxes) sbox[t][q] = box[s];
            }
        }
        __syncthreads();
        unsigned long long acc = first ? ~0ull : 0ull;
        const int i = threadIdx.x % kTile;
        if (i < ni) {
            const double2 a = sa[0][i], b = sb[0][i];
            const int4 bi = boxes ? sbox[0][i] : make_int4(0, 0, 0, 0);
            const double ax0 = fmin(a.x, b.x), ax1 = fmax(a.x, b.x), ay0 = fmin(a.y, b.y), ay1 = fmax(a.y, b.y);
            const int jstart = ti == tj ? i + 1 : 0;
            // j = jstart + (tid / kTile) + 2 r: the two thread halves split the columns
            for (int j = jstart + threadIdx.x / kTile; j < nj; j += kPair / kTile) {
                const double2 c2 = sa[1][j], d2 = sb[1][j];
                if (boxes) {
                    const int4 bj = sbox[1][j];
                    const int ox = min(bi.y, bj.y) - max(bi.x, bj.x) + 1;
                    const int oy = min(bi.w, bj.w) - max(bi.z, bj.z) + 1;
                    if (ox > 0 && oy > 0 && seg_cross(a, b, c2, d2)) {
                        if (count) {
                            acc += static_cast<unsigned long long>(ox) * static_cast<unsigned long long>(oy);
                        } else {   // the reference meets the pair first in its first shared cell
                            const unsigned long long cmin = static_cast<unsigned long long>(max(bi.z, bj.z)) *
                                                                static_cast<unsigned long long>(g_nx(grid, c)) +
                                                            static_cast<unsigned long long>(max(bi.x, bj.x));
                            const unsigned long long gi = static_cast<unsigned long long>(ti * kTile + i);
                            const unsigned long long gj = static_cast<unsigned long long>(tj * kTile + j);
                            const unsigned long long key = (cmin << 42) | (gi << 21) | gj;
                            if (key < acc) acc = key;
                        }
                    }
                } else {
                    if (fmax(c2.x, d2.x) >= ax0 && fmin(c2.x, d2.x) <= ax1 && fmax(c2.y, d2.y) >= ay0 &&
                        fmin(c2.y, d2.y) <= ay1 && seg_cross(a, b, c2, d2))
                        acc += 1;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long y = __shfl_xor_sync(0xffffffffu, acc, o);
            acc = first ? (y < acc ? y : acc) : acc + y;
        }
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long s = first ? ~0ull : 0ull;
            for (int k = 0; k < kPair / 32; ++k) s = first ? (wsum[k] < s ? wsum[k] : s) : s + wsum[k];
            if (first) { if (s != ~0ull) atomicMin(hits + c, s); }
            else if (s) atomicAdd(hits + c, s);
        }
    }
}

__global__ void k_seg_final(uva_seg_desc d, const ChartGrid* grid, const unsigned long long* hits) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.nc) return;
    const int flag = grid[c].flag;
    const unsigned long long h = hits[c];
    int64_t r;
    if (flag == kFlagRange) {
        r = -2;
    } else if (d.mode == UVA_SEG_COUNT) {
        const unsigned long long cap = static_cast<unsigned long long>(d.max_report > 1 ? d.max_report : 1);
        r = flag ? -1 : static_cast<int64_t>(h < cap ? h : cap);
    } else if (d.mode == UVA_SEG_FIRST) {   // (i << 32) | j of the first crossing pair, -3: none
        const unsigned long long mask = (1ull << 21) - 1;
        r = flag ? -1 : (h == ~0ull ? -3 : static_cast<int64_t>((((h >> 21) & mask) << 32) | (h & mask)));
    } else {
        r = (flag || h > 0) ? 1 : 0;
    }
    d.out[c] = r;
}

// ------------------------------------------------------------------ batch boundary
// Directed boundary half-edges of a device batch (engine/param.py:59-68 per
// island): corner edge k of triangle f runs c[k+1] -> c[k+2] on unique edge
// tri_edge[3f + k]; it is a boundary half-edge when no half-edge of the same
// edge runs the other way (self-loops never are).
__device__ __forceinline__ bool half_edge(const uva_batch& b, int f, int k, int& e, int& a, int& c, int& dir) {
    e = b.tri_edge[3 * f + k];
    const int4 t = reinterpret_cast<const int4*>(b.tri4)[f];
    const int v[3] = {t.x, t.y, t.z};
    a = v[(k + 1) % 3];
    c = v[(k + 2) % 3];
    dir = a < c ? 0 : 1;
    return e >= 0 && a != c;
}

__global__ void k_bnd_count(uva_batch b, int* ecnt) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t) return;
    for (int k = 0; k < 3; ++k) {
        int e, a, c, dir;
        if (half_edge(b, f, k, e, a, c, dir)) atomicAdd(ecnt + 2 * e + dir, 1);
    }
}

// pass 0: boundary half-edges per island; pass 1: write them (rows of U)
__global__ void k_bnd_emit(uva_batch b, const int* ecnt, int* icnt, const int32_t* seg_ofs, int* cursor,
                           int32_t* seg, int pass) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t) return;
    const int isl = b.tri4[4 * f + 3];
    for (int k = 0; k < 3; ++k) {
        int e, a, c, dir;
        if (!half_edge(b, f, k, e, a, c, dir) || ecnt[2 * e + (dir ^ 1)] != 0) continue;
        if (pass == 0) {
            atomicAdd(icnt + isl, 1);
        } else {
            const int q = seg_ofs[isl] + atomicAdd(cursor + isl, 1);
            seg[2 * q] = b.vofs[isl] + a;
            seg[2 * q + 1] = b.vofs[isl] + c;
        }
    }
}

// seg_ofs = exclusive prefix of icnt (one CTA)
__global__ void __launch_bounds__(kScan) k_bnd_scan(int nc, const int* icnt, int32_t* seg_ofs) {
    __shared__ long long part[kScan];
    const int per = (nc + kScan - 1) / kScan;
    const int c0 = threadIdx.x * per, c1 = min(nc, c0 + per);
    long long s = 0;
    for (int c = c0; c < c1; ++c) s += icnt[c];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < kScan; o <<= 1) {
        const long long add = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    long long run = part[threadIdx.x] - s;
    for (int c = c0; c < c1; ++c) {
        seg_ofs[c] = static_cast<int32_t>(run);
        run += icnt[c];
    }
    if (threadIdx.x == kScan - 1) seg_ofs[nc] = static_cast<int32_t>(part[kScan - 1]);
}

}  // namespace

extern "C" int uva_batch_boundary_scratch_bytes(const uva_batch* b, int64_t* bytes) {
    if (!b || !bytes || b->nc < 0 || b->E < 0) { uva_set_error("uva_batch_boundary_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    *bytes = 4 * (2 * static_cast<int64_t>(std::max(b->E, 1)) + 2 * static_cast<int64_t>(std::max(b->nc, 1)));
    return UVA_OK;
}

extern "C" int uva_batch_boundary(const uva_batch* b, int32_t* seg_ofs, int32_t* seg, void* scratch,
                                  int64_t scratch_bytes, void* stream) {
    if (!b || b->nc < 0 || b->t < 0 || !seg_ofs || (b->nc > 0 && (!b->tri4 || !b->vofs || !scratch)) ||
        (b->t > 0 && (!b->tri_edge || !seg))) {
        uva_set_error("uva_batch_boundary: bad arguments");
        return UVA_E_ARG;
    }
    if (b->nc == 0) return UVA_OK;
    const int64_t need = 4 * (2 * static_cast<int64_t>(std::max(b->E, 1)) + 2 * static_cast<int64_t>(b->nc));
    if (scratch_bytes < need) { uva_set_error("uva_batch_boundary: scratch too small"); return UVA_E_ARG; }
    if (3 * static_cast<int64_t>(b->t) >= (int64_t(1) << 31)) { uva_set_error("uva_batch_boundary: too many triangles"); return UVA_E_TOOBIG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int* ecnt = static_cast<int*>(scratch);
    int* icnt = ecnt + 2 * static_cast<size_t>(std::max(b->E, 1));
    int* cursor = icnt + b->nc;
    cudaMemsetAsync(scratch, 0, static_cast<size_t>(need), s);
    const int blocks = std::max(1, (b->t + 255) / 256);
    k_bnd_count<<<blocks, 256, 0, s>>>(*b, ecnt);
    k_bnd_emit<<<blocks, 256, 0, s>>>(*b, ecnt, icnt, seg_ofs, cursor, seg, 0);
    k_bnd_scan<<<1, kScan, 0, s>>>(b->nc, icnt, seg_ofs);
    k_bnd_emit<<<blocks, 256, 0, s>>>(*b, ecnt, icnt, seg_ofs, cursor, seg, 1);
    UVA_CHECK_LAUNCH("uva_batch_boundary");
    return UVA_OK;
}

extern "C" int uva_seg_scratch_bytes(int32_t nc, int32_t nseg, int64_t* bytes) {
    if (nc < 0 || nseg < 0 || !bytes) { uva_set_error("uva_seg_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    *bytes = static_cast<int64_t>(layout(nc, nseg).total);
    return UVA_OK;
}

extern "C" int uva_boundary_hits(const uva_seg_desc* d, void* stream) {
    if (!d || d->nc < 0 || d->nseg < 0 || d->n < 0 ||
        (d->mode != UVA_SEG_COUNT && d->mode != UVA_SEG_ANY && d->mode != UVA_SEG_ANY_ALL &&
         d->mode != UVA_SEG_FIRST)) {
        uva_set_error("uva_boundary_hits: bad arguments");
        return UVA_E_ARG;
    }
    if (d->nc == 0) return UVA_OK;
    if (!d->seg_ofs || !d->out || !d->scratch || ((d->mode == UVA_SEG_COUNT || d->mode == UVA_SEG_FIRST) && !d->vofs) ||
        (d->nseg > 0 && (!d->seg || !d->U || d->n == 0))) {
        uva_set_error("uva_boundary_hits: null pointer");
        return UVA_E_ARG;
    }
    const Layout L = layout(d->nc, d->nseg);
    if (d->scratch_bytes < static_cast<int64_t>(L.total)) {
        uva_set_error("uva_boundary_hits: scratch too small");
        return UVA_E_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto* base = static_cast<unsigned char*>(d->scratch);
    auto* grid = reinterpret_cast<ChartGrid*>(base + L.grid);
    auto* hits = reinterpret_cast<unsigned long long*>(base + L.hits);
    auto* tile_ofs = reinterpret_cast<int64_t*>(base + L.tile_ofs);
    auto* box = reinterpret_cast<int4*>(base + L.box);
    auto* len = reinterpret_cast<double*>(base + L.len);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int prep_grid = std::max(1, std::min(d->nc, 8 * sms));
    k_seg_prep<<<prep_grid, kPrep, 0, s>>>(*d, grid, hits, box, len);
    k_seg_scan<<<1, kScan, 0, s>>>(d->nc, grid, tile_ofs);
    k_seg_pairs<<<8 * sms, kPair, 0, s>>>(*d, grid, tile_ofs, box, hits);
    k_seg_final<<<(d->nc + 255) / 256, 256, 0, s>>>(*d, grid, hits);
    UVA_CHECK_LAUNCH("uva_boundary_hits");
    return UVA_OK;
}
