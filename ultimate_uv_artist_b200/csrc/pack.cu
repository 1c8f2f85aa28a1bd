// Raster atlas packing on the device (engine/pack.py:53-363, 537-567): the
// chart masks of one packing attempt, their row runs, the greedy first-fit
// placement of all charts on one page, the page occupancy and the final UVs.
// Built with --fmad=false: the raster and the UV arithmetic follow the
// reference's FP64 operations one by one, so masks, placements and UVs are
// the same bits.
//
// Masks (uva_pack_masks). A mask source is a chart at one pre-rotation
// angle. Its mask has a cell set when the cell corner that maximises each
// edge function lies on the inner side of all three edges of some triangle
// (conservative raster, pack.py:53-79), then every cell within the gutter
// radius of a set cell in the square (Chebyshev) sense is set too
// (pack.py:82-92). One thread rasterises a small triangle; a triangle whose
// box holds more than 64 cells goes to a list that whole blocks take. The
// dilation is separable: rows, then columns.
//
// Runs (uva_pack_variants). A variant is a source turned by 0..3 quarter
// turns (np.rot90). Its rows are stored as runs of set cells with the
// longest run of each row (pack.py:95-119), the set cells of the variant
// (the "area" ordering key, pack.py:392) and the row with the longest run,
// which the placement tests first.
//
// Placement (uva_pack_place), one cooperative launch for all charts. The
// page keeps, per cell, the free run to its right (R = 0: occupied) and, per
// row, the longest free run. For every chart in turn (pack.py:312-359):
//   A1. one thread per (row y, variant k) item tests every row of the
//       variant against the longest free run of the page row it would land
//       on; the items that pass are bits in (y, k) order. Grid barrier.
//   A2. blocks take the passing items by rank (block b: ranks b, b + nb, ...,
//       so in increasing y). Per item every x is a bit of one thread: the
//       widest run of the variant's longest-run row and of seven rows spread
//       over its height must land on free runs at least as long (loads in
//       flight together); the x left are candidates, tested whole in
//       increasing x, one per warp, the lanes taking the rows. A fit lowers
//       ybest[k] (atomic minimum); items below ybest[k] are skipped, and a
//       block stops once every variant fits higher than its next item.
//       ybest[k], bestx[k][ybest[k]] is the reference's first fit (smallest
//       y, then smallest x, pack.py:124-156). Grid barrier.
//   B.  every block picks, from the same values, the variant of smallest
//       (y + h) G + (x + w), the first on ties (pack.py:345-351); none: the
//       attempt fails and every block returns.
//   C.  blocks rebuild the free runs of the rows the chart covers; a grid
//       barrier ends the chart.
// Values written inside the launch are read with ld.global.cg (L2), so no
// block sees a stale line of its own L1. The barrier spins a bounded time
// (two seconds) and reports a timeout in the status instead of waiting for
// good.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "scan.cuh"

using namespace uva;

namespace {

constexpr int kTB = 256;
constexpr int32_t kNone = 0x7f7f7f7f;   // a byte memset of 0x7f
constexpr int kBigTri = 64;             // box cells above which a block rasterises the triangle
constexpr long long kSpinLimit = 1ll << 24;

inline unsigned blocks_for(int64_t n) {
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + kTB - 1) / kTB, 1 << 20)));
}

inline int64_t al(int64_t x) { return (x + 255) & ~static_cast<int64_t>(255); }

#define GRID_STRIDE(i, count)                                                                   \
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < (count); \
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)

// k with ofs[k] <= i < ofs[k + 1] (ofs ascending, n + 1 entries, ofs[0] = 0)
template <typename T>
__device__ __forceinline__ int32_t find_seg(const T* ofs, int32_t n, int64_t i) {
    int32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const int32_t mid = (lo + hi) >> 1;
        if (static_cast<int64_t>(ofs[mid]) <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// ------------------------------------------------------------------ masks
struct RasterTri {
    double ex[3], ey[3], ox[3], oy[3];
    int64_t minx, maxx, miny, maxy;
};

// One triangle of a source at its texel scale: corners V = U * scale + pad
// (two roundings, as numpy), counter-clockwise, edge vectors and cell box.
__device__ __forceinline__ RasterTri raster_setup(const double* U, const int32_t* tri, double sc, double pd,
                                                  int32_t h, int32_t w) {
    double x0 = U[2 * tri[0]] * sc + pd, y0 = U[2 * tri[0] + 1] * sc + pd;
    double x1 = U[2 * tri[1]] * sc + pd, y1 = U[2 * tri[1] + 1] * sc + pd;
    double x2 = U[2 * tri[2]] * sc + pd, y2 = U[2 * tri[2] + 1] * sc + pd;
    const double area = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
    if (area < 0) {
        const double tx = x1, ty = y1;
        x1 = x2; y1 = y2; x2 = tx; y2 = ty;
    }
    RasterTri r;
    r.minx = max(static_cast<int64_t>(floor(fmin(x0, fmin(x1, x2)))), int64_t(0));
    r.maxx = min(static_cast<int64_t>(floor(fmax(x0, fmax(x1, x2)))), int64_t(w - 1));
    r.miny = max(static_cast<int64_t>(floor(fmin(y0, fmin(y1, y2)))), int64_t(0));
    r.maxy = min(static_cast<int64_t>(floor(fmax(y0, fmax(y1, y2)))), int64_t(h - 1));
    r.ex[0] = x1 - x0; r.ex[1] = x2 - x1; r.ex[2] = x0 - x2;
    r.ey[0] = y1 - y0; r.ey[1] = y2 - y1; r.ey[2] = y0 - y2;
    r.ox[0] = x0; r.ox[1] = x1; r.ox[2] = x2;
    r.oy[0] = y0; r.oy[1] = y1; r.oy[2] = y2;
    return r;
}

__device__ __forceinline__ bool raster_inside(const RasterTri& r, int64_t px, int64_t py) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double cx = static_cast<double>(px) + (r.ey[k] > 0 ? 0.0 : 1.0);
        const double cy = static_cast<double>(py) + (r.ex[k] > 0 ? 1.0 : 0.0);
        const double e = r.ex[k] * (cy - r.oy[k]) - r.ey[k] * (cx - r.ox[k]);
        if (e < 0) return false;
    }
    return true;
}

__device__ __forceinline__ int64_t raster_cells(const RasterTri& r) {
    if (r.maxx < r.minx || r.maxy < r.miny) return 0;
    return (r.maxx - r.minx + 1) * (r.maxy - r.miny + 1);
}

__global__ void k_pk_raster(int64_t ntri, int32_t nsrc, const double* V, const int64_t* vofs, const int32_t* T,
                            const int64_t* tofs, const double* scale, const int32_t* hw, const int64_t* mofs,
                            int32_t pad, uint8_t* mask, int32_t* big, int32_t* nbig) {
    GRID_STRIDE(t, ntri) {
        const int32_t s = find_seg(tofs, nsrc, t);
        const int32_t h = hw[2 * s], w = hw[2 * s + 1];
        const RasterTri r = raster_setup(V + 2 * vofs[s], T + 3 * t, scale[s], static_cast<double>(pad), h, w);
        const int64_t cells = raster_cells(r);
        if (cells > kBigTri) {
            big[atomicAdd(nbig, 1)] = static_cast<int32_t>(t);
            continue;
        }
        uint8_t* m = mask + mofs[s];
        for (int64_t py = r.miny; py <= r.maxy; ++py)
            for (int64_t px = r.minx; px <= r.maxx; ++px)
                if (raster_inside(r, px, py)) m[py * w + px] = 1;
    }
}

__global__ void k_pk_raster_big(const int32_t* nbig, const int32_t* big, int32_t nsrc, const double* V,
                                const int64_t* vofs, const int32_t* T, const int64_t* tofs, const double* scale,
                                const int32_t* hw, const int64_t* mofs, int32_t pad, uint8_t* mask) {
    const int32_t count = *nbig;
    for (int32_t b = blockIdx.x; b < count; b += gridDim.x) {
        const int64_t t = big[b];
        const int32_t s = find_seg(tofs, nsrc, t);
        const int32_t h = hw[2 * s], w = hw[2 * s + 1];
        const RasterTri r = raster_setup(V + 2 * vofs[s], T + 3 * t, scale[s], static_cast<double>(pad), h, w);
        const int64_t bw = r.maxx - r.minx + 1, cells = raster_cells(r);
        uint8_t* m = mask + mofs[s];
        for (int64_t c = threadIdx.x; c < cells; c += blockDim.x) {
            const int64_t py = r.miny + c / bw, px = r.minx + c % bw;
            if (raster_inside(r, px, py)) m[py * w + px] = 1;
        }
    }
}

// Square dilation by `pad` cells, separable: AXIS 1 along rows, 0 along columns.
template <int AXIS>
__global__ void k_pk_dilate(int64_t ncells, int32_t nsrc, const int32_t* hw, const int64_t* mofs, int32_t pad,
                            const uint8_t* in, uint8_t* out) {
    GRID_STRIDE(c, ncells) {
        const int32_t s = find_seg(mofs, nsrc, c);
        const int32_t h = hw[2 * s], w = hw[2 * s + 1];
        const int64_t local = c - mofs[s];
        const int32_t y = static_cast<int32_t>(local / w), x = static_cast<int32_t>(local - static_cast<int64_t>(y) * w);
        const uint8_t* m = in + mofs[s];
        uint8_t v = 0;
        if (AXIS == 1) {
            for (int32_t k = max(0, x - pad); k <= min(w - 1, x + pad) && !v; ++k)
                v = m[static_cast<int64_t>(y) * w + k];
        } else {
            for (int32_t k = max(0, y - pad); k <= min(h - 1, y + pad) && !v; ++k)
                v = m[static_cast<int64_t>(k) * w + x];
        }
        out[c] = v;
    }
}

// ------------------------------------------------------------------ variant rows and runs
struct Variant {
    int32_t src, turn, h, w;   // source (-1: none), quarter turns, height and width after the turn
};

__device__ __forceinline__ Variant variant_of(int64_t v, const int32_t* var_src, const int32_t* var_turn,
                                              const int32_t* hw) {
    Variant r;
    r.src = var_src[v];
    r.turn = var_turn[v] & 3;
    r.h = r.w = 0;
    if (r.src >= 0) {
        const int32_t h0 = hw[2 * r.src], w0 = hw[2 * r.src + 1];
        r.h = (r.turn & 1) ? w0 : h0;
        r.w = (r.turn & 1) ? h0 : w0;
    }
    return r;
}

// Cell (i, j) of a source mask (h0 x w0) turned like np.rot90(m, turn):
// 1: m[j][w0-1-i], 2: m[h0-1-i][w0-1-j], 3: m[h0-1-j][i].
__device__ __forceinline__ uint8_t turned_cell(const uint8_t* m, int32_t h0, int32_t w0, int32_t turn, int32_t i,
                                               int32_t j) {
    int32_t y, x;
    switch (turn) {
        case 0: y = i; x = j; break;
        case 1: y = j; x = w0 - 1 - i; break;
        case 2: y = h0 - 1 - i; x = w0 - 1 - j; break;
        default: y = h0 - 1 - j; x = i; break;
    }
    return m[static_cast<int64_t>(y) * w0 + x];
}

// FILL false: runs per row (into run_ofs, scanned afterwards), the longest
// run, the row's set cells into the variant's area and (longest run, first
// row) into the variant's key. FILL true: the runs' first and last cells.
template <bool FILL>
__global__ void k_pk_runs(int64_t nrows, int32_t nvar, const int64_t* var_row, const int32_t* var_src,
                          const int32_t* var_turn, const int32_t* hw, const int64_t* mofs, const uint8_t* mask,
                          int32_t* run_ofs, int32_t* row_need, unsigned long long* var_area,
                          unsigned long long* var_key, int32_t* run_a, int32_t* run_b, int64_t run_cap,
                          int32_t* status) {
    GRID_STRIDE(r, nrows) {
        const int32_t v = find_seg(var_row, nvar, r);
        const Variant vr = variant_of(v, var_src, var_turn, hw);
        const int32_t i = static_cast<int32_t>(r - var_row[v]);
        const int32_t h0 = hw[2 * vr.src], w0 = hw[2 * vr.src + 1];
        const uint8_t* m = mask + mofs[vr.src];
        int32_t cnt = 0, need = 0, cells = 0;
        int64_t q = FILL ? run_ofs[r] : 0;
        int32_t j = 0;
        while (j < vr.w) {
            if (turned_cell(m, h0, w0, vr.turn, i, j)) {
                const int32_t s = j;
                while (j < vr.w && turned_cell(m, h0, w0, vr.turn, i, j)) ++j;
                if (FILL) {
                    if (q < run_cap) { run_a[q] = s; run_b[q] = j - 1; }
                    else atomicOr(status, 1);
                    ++q;
                }
                ++cnt;
                cells += j - s;
                need = max(need, j - s);
            } else {
                ++j;
            }
        }
        if (!FILL) {
            run_ofs[r] = cnt;
            row_need[r] = need;
            if (cells) atomicAdd(var_area + v, static_cast<unsigned long long>(cells));
            atomicMax(var_key + v, (static_cast<unsigned long long>(need) << 32) |
                                       static_cast<unsigned long long>(~static_cast<uint32_t>(i)));
        }
    }
}

// ------------------------------------------------------------------ placement
struct GridBar {
    unsigned count, gen;
    int err, reserved;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier of a cooperative launch (all blocks resident). A block that
// waits longer than two seconds sets the error flag and every block returns
// false from then on.
__device__ bool grid_sync(GridBar* bar, unsigned nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned g = ld_acquire(&bar->gen);
        __threadfence();
        int ok = 1;
        if (atomicAdd(&bar->count, 1u) == nblocks - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            long long spins = 0;
            while (ld_acquire(&bar->gen) == g) {
                if ((++spins & 1023) == 0 && (global_ns() - t0 > 2000000000ull || spins > kSpinLimit)) {
                    atomicExch(&bar->err, 1);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (ld_acquire(reinterpret_cast<const unsigned*>(&bar->err))) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

struct PlaceArgs {
    int32_t G, nc, nk;
    const int64_t* order;
    const int32_t* var_src;
    const int32_t* var_turn;
    const int64_t* var_row;
    const int32_t* hw;
    const int32_t* row_need;
    const int32_t* run_ofs;
    const int32_t* run_a;
    const int32_t* run_b;
    const unsigned long long* var_key;
    int32_t* R;
    int32_t* rowmax;
    int32_t* placement;
    int32_t* status;
    int32_t* bestx;   // nk * G
    int32_t* ybest;   // 2 * nk, alternating per chart
    unsigned* cand;   // 2 * cand_words item bits, alternating per chart
    int64_t cand_words;
    GridBar* bar;
};

constexpr int kMaxVariants = 64;
constexpr int kFilters = 8;   // widest run of the longest-run row and of 7 rows spread over the height
constexpr int kWarps = kTB / 32;

// The variants of one chart, staged in shared memory once per chart: size,
// first row, and the filter runs (row, first cell, length; length 0: none)
// tested for every x before the whole variant is.
struct ChartVariants {
    int32_t h[kMaxVariants], w[kMaxVariants], first[kMaxVariants];
    int64_t r0[kMaxVariants];
    int32_t fy[kMaxVariants][kFilters], fa[kMaxVariants][kFilters], fl[kMaxVariants][kFilters];
};

// Does the variant (h rows from r0) fit with its corner at (x, y)? The
// lanes of one warp take the rows, loads independent of each other.
__device__ __forceinline__ bool warp_fits(const int32_t* R, const int32_t* run_ofs, const int32_t* run_a,
                                          const int32_t* run_b, int32_t G, int32_t y, int32_t x, int32_t h,
                                          int64_t r0, int lane) {
    bool ok = true;
    for (int32_t j = lane; j < h; j += 32) {
        const int32_t* Rrow = R + static_cast<int64_t>(y + j) * G + x;
        const int32_t q1 = __ldg(run_ofs + r0 + j + 1);
        for (int32_t q = __ldg(run_ofs + r0 + j); q < q1; ++q) {
            const int32_t qa = __ldg(run_a + q);
            ok &= __ldcg(Rrow + qa) >= __ldg(run_b + q) - qa + 1;
        }
    }
    return __all_sync(0xffffffffu, ok);
}

// Dynamic shared memory: G free-run ints, then G occupancy bytes.
// Several pages (independent attempts) in one launch: block b works on page
// b % np, as block b / np of that page's b-blocks.
constexpr int kMaxPages = 4;
struct PlaceMulti {
    PlaceArgs page[kMaxPages];
    int32_t np;
};

__global__ void __launch_bounds__(kTB, 4) k_pk_place(PlaceMulti pm) {
    const int32_t g = static_cast<int32_t>(blockIdx.x % static_cast<unsigned>(pm.np));
    const PlaceArgs& a = pm.page[g];
    const unsigned nb = (gridDim.x - static_cast<unsigned>(g) + pm.np - 1) / static_cast<unsigned>(pm.np);
    const unsigned bid = blockIdx.x / static_cast<unsigned>(pm.np);
    extern __shared__ __align__(16) uint8_t s_dyn[];
    int32_t* s_R = reinterpret_cast<int32_t*>(s_dyn);
    uint8_t* s_occ = s_dyn + 4 * static_cast<size_t>(a.G);
    __shared__ ChartVariants cv;
    __shared__ int32_t s_wmin[kTB / 32], s_wmax[kTB / 32];
    __shared__ int32_t s_sel[3];
    __shared__ int32_t s_best;
    __shared__ int64_t s_chart;
    __shared__ unsigned s_cand[kWarps];
    __shared__ unsigned s_slots;
    __shared__ unsigned s_word[kTB];
    __shared__ int32_t s_yb[2][kMaxVariants];
    __shared__ int32_t s_pref[kTB];
    const int32_t G = a.G, nk = a.nk;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int32_t p = 0; p < a.nc; ++p) {
        // ---- the chart's variants: usable ones get h > 0
        __syncthreads();
        if (threadIdx.x == 0) s_chart = a.order[p];
        __syncthreads();
        const int64_t c = s_chart;
        int32_t* yb = a.ybest + (p & 1) * nk;
        for (int32_t k = threadIdx.x; k < nk; k += blockDim.x) {
            const int64_t v = c * nk + k;
            const Variant vr = variant_of(v, a.var_src, a.var_turn, a.hw);
            const bool ok = vr.src >= 0 && vr.h > 0 && vr.h <= G && vr.w <= G;
            cv.h[k] = ok ? vr.h : 0;
            cv.w[k] = vr.w;
            cv.r0[k] = a.var_row[v];
            cv.first[k] = static_cast<int32_t>(~static_cast<uint32_t>(__ldg(a.var_key + v) & 0xffffffffull));
        }
        __syncthreads();
        for (int32_t t = threadIdx.x; t < kFilters * nk; t += blockDim.x) {
            const int32_t k = t / kFilters, i = t - kFilters * k, h = cv.h[k];
            int32_t row = 0, fa = 0, fl = 0;
            if (h > 0) {
                row = i == 0 ? cv.first[k] : static_cast<int32_t>((static_cast<int64_t>(i - 1) * (h - 1)) / 6);
                const int32_t q1 = __ldg(a.run_ofs + cv.r0[k] + row + 1);
                for (int32_t q = __ldg(a.run_ofs + cv.r0[k] + row); q < q1; ++q) {
                    const int32_t qa = __ldg(a.run_a + q), len = __ldg(a.run_b + q) - qa + 1;
                    if (len > fl) { fl = len; fa = qa; }
                }
            }
            cv.fy[k][i] = row;
            cv.fa[k][i] = fa;
            cv.fl[k][i] = fl;
        }
        __syncthreads();
        // ---- A1: the items (y, k) whose rows all fit the longest free runs of
        // the page rows below them, one thread per item, as bits in y-major order
        const int64_t items = static_cast<int64_t>(nk) * G;
        unsigned* cb = a.cand + (p & 1) * a.cand_words;
        for (int32_t i = threadIdx.x; i < G; i += blockDim.x) s_R[i] = __ldcg(a.rowmax + i);   // s_R: rowmax here
        __syncthreads();
        // a warp owns the word of its 32 items (it = warp-aligned base + lane)
        for (int64_t base = (bid * static_cast<int64_t>(blockDim.x) + threadIdx.x) & ~int64_t(31);
             base < items; base += static_cast<int64_t>(nb) * blockDim.x) {
            const int64_t it = base + lane;
            bool ok = false;
            if (it < items) {
                const int32_t y = static_cast<int32_t>(it / nk), k = static_cast<int32_t>(it - static_cast<int64_t>(y) * nk);
                const int32_t h = cv.h[k];
                if (h > 0 && y <= G - h) {
                    const int32_t* need = a.row_need + cv.r0[k];
                    const int32_t* rm = s_R + y;
                    ok = true;
                    for (int32_t j = 0; j < h && ok; j += 4) {   // four rows a step, the last row again past the end
                        const int32_t j1 = min(j + 1, h - 1), j2 = min(j + 2, h - 1), j3 = min(j + 3, h - 1);
                        ok = (__ldg(need + j) <= rm[j]) & (__ldg(need + j1) <= rm[j1]) & (__ldg(need + j2) <= rm[j2]) &
                             (__ldg(need + j3) <= rm[j3]);
                    }
                }
            }
            const unsigned bits = __ballot_sync(0xffffffffu, ok);
            if (lane == 0 && bits) cb[base >> 5] = bits;
        }
        if (!grid_sync(a.bar, nb)) {
            if (bid == 0 && threadIdx.x == 0) atomicOr(a.status, 2);
            return;
        }
        // ---- A2: first fit of every variant over the items of A1, in
        // increasing (y, k); block b takes the items of rank b, b + nb, ...
        int64_t carry = 0;
        bool all_done = false;
        int r_par = 0;
        for (int64_t w0 = 0; w0 < a.cand_words && !all_done; w0 += blockDim.x) {
            __syncthreads();   // s_word / s_pref of the previous tile are read
            const int64_t wi = w0 + threadIdx.x;
            const unsigned word = wi < a.cand_words ? __ldcg(cb + wi) : 0u;
            int32_t incl = __popc(word);
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            if (lane == 31) s_wmin[warp] = incl;
            __syncthreads();
            int32_t wbase = 0, total = 0;
            for (int w2 = 0; w2 < kWarps; ++w2) {
                if (w2 < warp) wbase += s_wmin[w2];
                total += s_wmin[w2];
            }
            s_word[threadIdx.x] = word;
            s_pref[threadIdx.x] = wbase + incl - __popc(word);   // exclusive
            __syncthreads();
            const int64_t r_first = carry + ((static_cast<int64_t>(bid) - carry) % nb + nb) % nb;
            for (int64_t r = r_first; r < carry + total; r += nb) {
                const int32_t rr = static_cast<int32_t>(r - carry);
                int32_t lo = 0, hi = kTB - 1;   // the last thread whose exclusive prefix is <= rr
                while (lo < hi) {
                    const int32_t mid = (lo + hi + 1) >> 1;
                    if (s_pref[mid] <= rr) lo = mid; else hi = mid - 1;
                }
                const int bit = __fns(s_word[lo], 0, rr - s_pref[lo] + 1);
                const int64_t it = (w0 + lo) * 32 + bit;
                const int32_t y = static_cast<int32_t>(it / nk), k = static_cast<int32_t>(it - static_cast<int64_t>(y) * nk);
                const int32_t h = cv.h[k], w = cv.w[k];
                const int64_t r0 = cv.r0[k];
                if (threadIdx.x == 0) { s_best = kNone; s_slots = 0; }
                // every x is a slot bit of one thread (x = m * blockDim.x + tid).
                // One round of loads: the first filter for all slots, and the
                // rows' longest runs against the page rows' longest free runs
                const int32_t nx = G - w + 1, M = (nx + blockDim.x - 1) / blockDim.x;   // M <= 32: G <= 8192
                unsigned cand = 0;
                {
                    const int32_t* Rrow = a.R + static_cast<int64_t>(y + cv.fy[k][0]) * G + cv.fa[k][0];
                    const int32_t fl = cv.fl[k][0];
#pragma unroll 8
                    for (int32_t m = 0; m < M; ++m) {
                        const int32_t x = m * blockDim.x + threadIdx.x;
                        const bool ok = x < nx && __ldcg(Rrow + min(x, nx - 1)) >= fl;
                        cand |= static_cast<unsigned>(ok) << m;
                    }
                }
                // skip: a higher row already fits this variant; done: a higher
                // row fits every variant (this block's later items are lower)
                int32_t* syb = s_yb[r_par];
                r_par ^= 1;
                if (threadIdx.x < nk) syb[threadIdx.x] = __ldcg(yb + threadIdx.x);
                __syncthreads();
                bool done = true;
                for (int32_t kk = 0; kk < nk; ++kk) done &= cv.h[kk] == 0 || syb[kk] < y;
                if (done) { all_done = true; break; }
                if (syb[k] < y) continue;
                // the other filters, all loads of one slot in flight together
                for (unsigned live = cand; live; live &= live - 1) {
                    const int32_t m = __ffs(live) - 1;
                    const int32_t x = m * static_cast<int32_t>(blockDim.x) + static_cast<int32_t>(threadIdx.x);
                    bool ok = true;
#pragma unroll
                    for (int f = 1; f < kFilters; ++f)
                        ok &= __ldcg(a.R + static_cast<int64_t>(y + cv.fy[k][f]) * G + cv.fa[k][f] + x) >= cv.fl[k][f];
                    if (!ok) cand &= ~(1u << m);
                }
                // slot by slot in increasing x, the candidates, one per warp,
                // checked whole by the warp's lanes; the first slot with a fit ends it
                if (cand) atomicOr(&s_slots, cand);
                __syncthreads();
                unsigned slots = s_slots;
                bool found = false;
                while (slots) {
                    const int32_t m = __ffs(slots) - 1;
                    slots &= slots - 1;
                    // word `warp` holds the candidates m * blockDim.x + warp * 32 + lane
                    const unsigned bits = __ballot_sync(0xffffffffu, (cand >> m) & 1u);
                    if (lane == 0) s_cand[warp] = bits;
                    __syncthreads();
                    const unsigned word = lane < kWarps ? s_cand[lane] : 0u;
                    int32_t incl = __popc(word);
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= o) incl += t;
                    }
                    const int32_t ncand = __shfl_sync(0xffffffffu, incl, 31);
                    for (int32_t base = 0; base < ncand; base += kWarps) {
                        const int32_t r = base + warp;
                        bool ok = false;
                        if (r < ncand) {
                            const unsigned above = __ballot_sync(0xffffffffu, incl > r);
                            const int wi = __ffs(above) - 1;
                            const unsigned wbits = __shfl_sync(0xffffffffu, word, wi);
                            const int32_t before = __shfl_sync(0xffffffffu, incl - __popc(word), wi);
                            const int bit = __fns(wbits, 0, r - before + 1);
                            const int32_t x = m * static_cast<int32_t>(blockDim.x) + wi * 32 + bit;
                            ok = warp_fits(a.R, a.run_ofs, a.run_a, a.run_b, G, y, x, h, r0, lane);
                            if (ok && lane == 0) atomicMin(&s_best, x);
                        }
                        found = __syncthreads_or(ok && lane == 0);
                        if (found) break;
                    }
                    if (found) break;
                    __syncthreads();   // s_cand is rewritten for the next slot
                }
                if (threadIdx.x == 0 && s_best != kNone) {
                    a.bestx[static_cast<int64_t>(k) * G + y] = s_best;
                    __threadfence();
                    atomicMin(yb + k, y);
                }
            }
            carry += total;
        }
        if (!grid_sync(a.bar, nb)) {
            if (bid == 0 && threadIdx.x == 0) atomicOr(a.status, 2);
            return;
        }
        // ---- B: the variant of smallest (y + h) G + (x + w), the first on ties (warp 0)
        if (warp == 0) {
            unsigned long long key = ~0ull;
            for (int32_t k = lane; k < nk; k += 32) {
                const int32_t yv = __ldcg(yb + k);
                if (yv == kNone) continue;
                const int32_t xv = __ldcg(a.bestx + static_cast<int64_t>(k) * G + yv);
                const unsigned long long score =
                    static_cast<unsigned long long>(yv + cv.h[k]) * static_cast<unsigned long long>(G) + (xv + cv.w[k]);
                key = min(key, (score << 6) | static_cast<unsigned long long>(k));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) key = min(key, __shfl_xor_sync(0xffffffffu, key, o));
            if (lane == 0) {
                if (key == ~0ull) {
                    s_sel[0] = -1;
                } else {
                    const int32_t k = static_cast<int32_t>(key & 63);
                    s_sel[0] = k;
                    s_sel[2] = __ldcg(yb + k);
                    s_sel[1] = __ldcg(a.bestx + static_cast<int64_t>(k) * G + s_sel[2]);
                }
            }
        }
        __syncthreads();
        const int32_t bk = s_sel[0], bx = s_sel[1], by = s_sel[2];
        if (bk < 0) {
            if (bid == 0 && threadIdx.x == 0) { atomicOr(a.status, 1); a.status[1] = p; }
            return;
        }
        // ---- C: mark the chart's cells, rebuild the free runs of its rows
        const int64_t r0 = cv.r0[bk];
        for (int32_t j = bid; j < cv.h[bk]; j += nb) {
            int32_t* Rrow = a.R + static_cast<int64_t>(by + j) * G;
            __syncthreads();
            for (int32_t i = threadIdx.x; i < G; i += blockDim.x) s_occ[i] = __ldcg(Rrow + i) == 0;
            __syncthreads();
            const int32_t q1 = __ldg(a.run_ofs + r0 + j + 1);
            for (int32_t q = __ldg(a.run_ofs + r0 + j); q < q1; ++q) {
                const int32_t qb = __ldg(a.run_b + q);
                for (int32_t i = __ldg(a.run_a + q) + threadIdx.x; i <= qb; i += blockDim.x) s_occ[bx + i] = 1;
            }
            __syncthreads();
            // chunk per thread: its first occupied cell, the first occupied
            // cell right of it (suffix minimum), then the chunk backwards
            const int32_t chunk = (G + blockDim.x - 1) / blockDim.x;
            const int32_t lo = min(G, static_cast<int32_t>(threadIdx.x) * chunk), hi = min(G, lo + chunk);
            int32_t f = G;
            for (int32_t i = lo; i < hi; ++i)
                if (s_occ[i]) { f = i; break; }
            int32_t suf = f;   // inclusive suffix minimum within the warp
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t t = __shfl_down_sync(0xffffffffu, suf, o);
                if (lane + o < 32) suf = min(suf, t);
            }
            if (lane == 0) s_wmin[warp] = suf;
            int32_t nxt = __shfl_down_sync(0xffffffffu, suf, 1);
            if (lane == 31) nxt = G;
            __syncthreads();
            for (int w2 = warp + 1; w2 < static_cast<int>(blockDim.x >> 5); ++w2) nxt = min(nxt, s_wmin[w2]);
            int32_t mx = 0;
            for (int32_t i = hi - 1; i >= lo; --i) {
                if (s_occ[i]) { nxt = i; s_R[i] = 0; }
                else { s_R[i] = nxt - i; mx = max(mx, nxt - i); }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0) s_wmax[warp] = mx;
            __syncthreads();
            for (int32_t i = threadIdx.x; i < G; i += blockDim.x) Rrow[i] = s_R[i];
            if (threadIdx.x == 0) {
                int32_t m = 0;
                for (int w2 = 0; w2 < static_cast<int>(blockDim.x >> 5); ++w2) m = max(m, s_wmax[w2]);
                a.rowmax[by + j] = m;
            }
        }
        {   // the next chart's item bits, last read before the previous chart's end
            unsigned* nxt = a.cand + ((p + 1) & 1) * a.cand_words;
            for (int64_t i = bid * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < a.cand_words;
                 i += static_cast<int64_t>(nb) * blockDim.x)
                nxt[i] = 0u;
        }
        if (bid == 0 && threadIdx.x == 0) {
            a.placement[3 * c] = bk;
            a.placement[3 * c + 1] = bx;
            a.placement[3 * c + 2] = by;
            int32_t* other = a.ybest + ((p + 1) & 1) * nk;   // last read before the previous chart's end
            for (int32_t k = 0; k < nk; ++k) other[k] = kNone;
        }
        if (!grid_sync(a.bar, nb)) {
            if (bid == 0 && threadIdx.x == 0) atomicOr(a.status, 2);
            return;
        }
    }
}

__global__ void k_pk_page_init(int32_t G, int32_t* R, int32_t* rowmax) {
    GRID_STRIDE(c, static_cast<int64_t>(G) * G) { R[c] = G - static_cast<int32_t>(c % G); }
    GRID_STRIDE(y, G) { rowmax[y] = G; }
}

__global__ void k_pk_occupied(int64_t cells, const int32_t* R, unsigned long long* out) {
    unsigned long long cnt = 0;
    GRID_STRIDE(c, cells) { cnt += R[c] == 0; }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, cnt);
}

// UVs of every chart from its placement (pack.py:541-549): V = (U s) d + pad
// inside the unturned mask, turned like the mask (pack.py:557-567), moved by
// (x, y) and divided by the grid.
__global__ void k_pk_uv(int64_t nv, int32_t nc, int32_t nA, int32_t nr, const int64_t* cofs, const int64_t* vofs,
                        const double* V, const int32_t* hw, const int32_t* placement, double s, const double* dens,
                        int32_t pad, int32_t G, double* out) {
    GRID_STRIDE(i, nv) {
        const int32_t c = find_seg(cofs, nc, i);
        const int64_t local = i - cofs[c];
        const int32_t k = placement[3 * c], x = placement[3 * c + 1], y = placement[3 * c + 2];
        if (k < 0 || k >= nA * nr) {   // chart not placed
            out[2 * i] = out[2 * i + 1] = __longlong_as_double(0x7ff8000000000000ll);
            continue;
        }
        const int32_t ai = k / nr, turn = k - ai * nr;
        const int64_t src = static_cast<int64_t>(c) * nA + ai;
        const double h0 = static_cast<double>(hw[2 * src]), w0 = static_cast<double>(hw[2 * src + 1]);
        const double* U = V + 2 * (vofs[src] + local);
        const double d = dens[c], pd = static_cast<double>(pad);
        const double vx = U[0] * s * d + pd, vy = U[1] * s * d + pd;
        double X, Y;
        switch (turn & 3) {
            case 0: X = vx; Y = vy; break;
            case 1: X = vy; Y = w0 - vx; break;
            case 2: X = w0 - vx; Y = h0 - vy; break;
            default: X = h0 - vy; Y = vx; break;
        }
        out[2 * i] = (X + static_cast<double>(x)) / static_cast<double>(G);
        out[2 * i + 1] = (Y + static_cast<double>(y)) / static_cast<double>(G);
    }
}

struct PackScratch {
    int32_t* big;
    int32_t* nbig;
    uint8_t* tmp;
    int32_t* sums;
    int32_t* bestx;
    int32_t* ybest;
    unsigned* cand;
    int64_t cand_words;
    GridBar* bar;
    int64_t total;
};

PackScratch carve(void* base, int64_t ntri, int64_t ncells, int64_t nrows, int32_t nk, int32_t G) {
    PackScratch s{};
    int64_t o = 0;
    char* b = static_cast<char*>(base);
    auto take = [&](int64_t bytes) {
        char* p = b ? b + o : nullptr;
        o += al(std::max<int64_t>(bytes, 1));
        return p;
    };
    s.big = reinterpret_cast<int32_t*>(take(4 * ntri));
    s.nbig = reinterpret_cast<int32_t*>(take(4));
    s.tmp = reinterpret_cast<uint8_t*>(take(ncells));
    s.sums = reinterpret_cast<int32_t*>(take(4 * xscan_sums(nrows + 1)));
    s.bestx = reinterpret_cast<int32_t*>(take(4 * static_cast<int64_t>(nk) * G));
    s.ybest = reinterpret_cast<int32_t*>(take(8 * static_cast<int64_t>(nk)));
    s.cand_words = (static_cast<int64_t>(nk) * G + 31) / 32;
    s.cand = reinterpret_cast<unsigned*>(take(8 * s.cand_words));
    s.bar = reinterpret_cast<GridBar*>(take(sizeof(GridBar)));
    s.total = o;
    return s;
}

constexpr int32_t kMaxGrid = 8192;

bool attempt_ok(const uva_pack_attempt* a, const char* who, bool place) {
    const bool sizes = a && a->nsrc >= 0 && a->nc >= 0 && a->nk > 0 && a->nk <= 64 && a->G > 0 &&
                       a->G <= kMaxGrid && a->pad >= 0 && a->ntri >= 0 && a->ntri < (int64_t(1) << 31) &&
                       a->ncells >= 0 && a->nrows >= 0 && a->nrows < (int64_t(1) << 31) - 1 && a->run_cap >= 0 &&
                       a->run_cap < (int64_t(1) << 31);
    if (!sizes) { uva_set_error(who); return false; }
    const bool ptrs = a->mofs && a->var_row && a->run_ofs && a->status && a->scratch &&
                      (a->nsrc == 0 || (a->hw && a->scale && a->vofs && a->tofs)) &&
                      (a->nc == 0 || (a->var_src && a->var_turn && a->var_area && a->var_key)) &&
                      (a->ncells == 0 || a->mask) && (a->nrows == 0 || a->row_need) &&
                      (a->ntri == 0 || (a->V && a->T)) && (a->run_cap == 0 || (a->run_a && a->run_b)) &&
                      (!place || (a->R && a->rowmax && a->occupied && (a->nc == 0 || (a->order && a->placement))));
    if (!ptrs) { uva_set_error(who); return false; }
    if (a->scratch_bytes < carve(nullptr, a->ntri, a->ncells, a->nrows, a->nk, a->G).total) {
        uva_set_error(who);
        return false;
    }
    return true;
}

}  // namespace

// ==================================================================== C ABI
extern "C" int uva_pack_scratch_bytes(int64_t ntri, int64_t ncells, int64_t nrows, int32_t nk, int32_t G,
                                      int64_t* bytes) {
    if (ntri < 0 || ncells < 0 || nrows < 0 || nk <= 0 || G <= 0 || !bytes) {
        uva_set_error("uva_pack_scratch_bytes: bad arguments");
        return UVA_E_ARG;
    }
    *bytes = carve(nullptr, ntri, ncells, nrows, nk, G).total;
    return UVA_OK;
}

extern "C" int uva_pack_masks(const uva_pack_attempt* a, void* stream) {
    if (!attempt_ok(a, "uva_pack_masks: bad arguments or scratch too small", false)) return UVA_E_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PackScratch s = carve(a->scratch, a->ntri, a->ncells, a->nrows, a->nk, a->G);
    const int32_t nvar = a->nc * a->nk;
    cudaMemsetAsync(a->status, 0, 4 * sizeof(int32_t), st);
    cudaMemsetAsync(s.nbig, 0, sizeof(int32_t), st);
    if (a->ncells > 0) cudaMemsetAsync(a->mask, 0, static_cast<size_t>(a->ncells), st);
    if (nvar > 0) {
        cudaMemsetAsync(a->var_area, 0, 8 * static_cast<size_t>(nvar), st);
        cudaMemsetAsync(a->var_key, 0, 8 * static_cast<size_t>(nvar), st);
    }
    cudaMemsetAsync(a->run_ofs, 0, 4 * static_cast<size_t>(a->nrows + 1), st);
    if (a->ntri > 0 && a->nsrc > 0) {
        k_pk_raster<<<blocks_for(a->ntri), kTB, 0, st>>>(a->ntri, a->nsrc, a->V, a->vofs, a->T, a->tofs, a->scale,
                                                         a->hw, a->mofs, a->pad, a->mask, s.big, s.nbig);
        k_pk_raster_big<<<4 * 148, kTB, 0, st>>>(s.nbig, s.big, a->nsrc, a->V, a->vofs, a->T, a->tofs, a->scale,
                                                 a->hw, a->mofs, a->pad, a->mask);
    }
    if (a->pad > 0 && a->ncells > 0 && a->nsrc > 0) {
        k_pk_dilate<1><<<blocks_for(a->ncells), kTB, 0, st>>>(a->ncells, a->nsrc, a->hw, a->mofs, a->pad, a->mask,
                                                              s.tmp);
        k_pk_dilate<0><<<blocks_for(a->ncells), kTB, 0, st>>>(a->ncells, a->nsrc, a->hw, a->mofs, a->pad, s.tmp,
                                                              a->mask);
    }
    if (a->nrows > 0) {
        k_pk_runs<false><<<blocks_for(a->nrows), kTB, 0, st>>>(
            a->nrows, nvar, a->var_row, a->var_src, a->var_turn, a->hw, a->mofs, a->mask, a->run_ofs, a->row_need,
            reinterpret_cast<unsigned long long*>(a->var_area), reinterpret_cast<unsigned long long*>(a->var_key),
            nullptr, nullptr, 0, a->status + 2);
        xscan<int32_t>(a->run_ofs, a->run_ofs, s.sums, nullptr, a->nrows + 1, st);
        k_pk_runs<true><<<blocks_for(a->nrows), kTB, 0, st>>>(
            a->nrows, nvar, a->var_row, a->var_src, a->var_turn, a->hw, a->mofs, a->mask, a->run_ofs, a->row_need,
            nullptr, nullptr, a->run_a, a->run_b, a->run_cap, a->status + 2);
    }
    UVA_CHECK_LAUNCH("uva_pack_masks");
    return UVA_OK;
}

namespace {

// Page set-up, one cooperative launch over all pages, occupancy per page.
int place_pages(const uva_pack_attempt* const* as, int32_t np, int32_t blocks_per_sm, cudaStream_t st) {
    PlaceMulti pm{};
    pm.np = np;
    int32_t placing = 0;
    for (int32_t g = 0; g < np; ++g) {
        const uva_pack_attempt* a = as[g];
        if (a->G != as[0]->G) { uva_set_error("uva_pack_place_pages: pages of different sizes"); return UVA_E_ARG; }
        PackScratch s = carve(a->scratch, a->ntri, a->ncells, a->nrows, a->nk, a->G);
        const int64_t cells = static_cast<int64_t>(a->G) * a->G;
        cudaMemsetAsync(a->status, 0, 2 * sizeof(int32_t), st);
        cudaMemsetAsync(a->occupied, 0, sizeof(int64_t), st);
        cudaMemsetAsync(s.ybest, 0x7f, 8 * static_cast<size_t>(a->nk), st);
        cudaMemsetAsync(s.bar, 0, sizeof(GridBar), st);
        cudaMemsetAsync(s.cand, 0, 8 * static_cast<size_t>(s.cand_words), st);
        if (a->nc > 0) cudaMemsetAsync(a->placement, 0xff, 12 * static_cast<size_t>(a->nc), st);
        k_pk_page_init<<<blocks_for(cells), kTB, 0, st>>>(a->G, a->R, a->rowmax);
        PlaceArgs& pa = pm.page[g];
        pa.G = a->G; pa.nc = a->nc; pa.nk = a->nk; pa.order = a->order;
        pa.var_src = a->var_src; pa.var_turn = a->var_turn; pa.var_row = a->var_row; pa.hw = a->hw;
        pa.row_need = a->row_need; pa.run_ofs = a->run_ofs; pa.run_a = a->run_a; pa.run_b = a->run_b;
        pa.var_key = reinterpret_cast<const unsigned long long*>(a->var_key);
        pa.R = a->R; pa.rowmax = a->rowmax; pa.placement = a->placement; pa.status = a->status;
        pa.bestx = s.bestx; pa.ybest = s.ybest; pa.bar = s.bar;
        pa.cand = s.cand; pa.cand_words = s.cand_words;
        placing += a->nc > 0;
    }
    UVA_CHECK_LAUNCH("uva_pack_place/init");
    if (placing > 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t smem = 5 * static_cast<size_t>(as[0]->G);
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(k_pk_place, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pk_place, kTB, smem);
        if (e != cudaSuccess) return uva_cuda_status(e, "uva_pack_place/occupancy");
        if (per_sm < 1) { uva_set_error("uva_pack_place: kernel does not fit one SM"); return UVA_E_CUDA; }
        const int want = blocks_per_sm > 0 ? blocks_per_sm : 4;
        // a multiple of the page count, every page at least one block
        unsigned grid = static_cast<unsigned>(sms * std::min(per_sm, want));
        grid = std::max<unsigned>(static_cast<unsigned>(np), grid - grid % static_cast<unsigned>(np));
        void* args[] = {&pm};
        e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_pk_place), dim3(grid), dim3(kTB), args, smem,
                                        st);
        if (e != cudaSuccess) return uva_cuda_status(e, "uva_pack_place/launch");
    }
    for (int32_t g = 0; g < np; ++g) {
        const int64_t cells = static_cast<int64_t>(as[g]->G) * as[g]->G;
        k_pk_occupied<<<std::min<unsigned>(blocks_for(cells), 1024), kTB, 0, st>>>(
            cells, as[g]->R, reinterpret_cast<unsigned long long*>(as[g]->occupied));
    }
    UVA_CHECK_LAUNCH("uva_pack_place");
    return UVA_OK;
}

}  // namespace

extern "C" int uva_pack_place(const uva_pack_attempt* a, int32_t blocks_per_sm, void* stream) {
    if (!attempt_ok(a, "uva_pack_place: bad arguments or scratch too small", true)) return UVA_E_ARG;
    return place_pages(&a, 1, blocks_per_sm, static_cast<cudaStream_t>(stream));
}

extern "C" int uva_pack_place_pages(const uva_pack_attempt* const* attempts, int32_t n, int32_t blocks_per_sm,
                                    void* stream) {
    if (!attempts || n < 1 || n > kMaxPages) {
        uva_set_error("uva_pack_place_pages: 1 to 4 attempts");
        return UVA_E_ARG;
    }
    for (int32_t g = 0; g < n; ++g)
        if (!attempt_ok(attempts[g], "uva_pack_place_pages: bad arguments or scratch too small", true)) return UVA_E_ARG;
    return place_pages(attempts, n, blocks_per_sm, static_cast<cudaStream_t>(stream));
}

extern "C" int uva_pack_uv(const uva_pack_attempt* a, int32_t nangles, int32_t nturns, const int64_t* cofs,
                           int64_t nv, double s, const double* dens, double* out, void* stream) {
    if (!a || a->nc < 0 || nangles <= 0 || nturns <= 0 || nturns > 4 || nangles * nturns != a->nk ||
        a->nsrc != a->nc * nangles || nv < 0 || a->G <= 0 ||
        (a->nc > 0 && nv > 0 && (!cofs || !dens || !out || !a->V || !a->vofs || !a->hw || !a->placement))) {
        uva_set_error("uva_pack_uv: bad arguments");
        return UVA_E_ARG;
    }
    if (a->nc == 0 || nv == 0) return UVA_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_pk_uv<<<blocks_for(nv), kTB, 0, st>>>(nv, a->nc, nangles, nturns, cofs, a->vofs, a->V, a->hw, a->placement, s,
                                            dens, a->pad, a->G, out);
    UVA_CHECK_LAUNCH("uva_pack_uv");
    return UVA_OK;
}
