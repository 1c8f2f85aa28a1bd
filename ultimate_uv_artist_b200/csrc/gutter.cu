// Gutter between islands and raster coverage (engine/metrics.py:13-62,
// 314-373), compiled with --fmad=false (FP64 raster tests round like the
// reference's numba loops).
//
//  * Labels raster (conservative, half-diagonal tolerance): the reference is
//    serial and the LAST triangle in index order wins a texel; here every
//    triangle does atomicMax(texel, triangle index), then the winner's island
//    label is looked up.
//  * Distance transform: exact squared Euclidean distances to the nearest
//    filled texel, and scipy.ndimage.distance_transform_edt's choice among
//    equidistant features (smallest column, then smallest row). A column pass
//    then a row pass, both windowed to radius R: distances up to R are exact;
//    beyond R a texel is marked unknown. Any pair with an unknown texel sums
//    above R, so a minimum found at or below R is the true one; otherwise the
//    host repeats with a larger R.
//  * gap = min over 4-neighbour texel pairs whose nearest labels differ of
//    d(p) + d(q) (then minus 1 on the host); 0 if two islands touch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"

using namespace uva;

namespace {

constexpr int kSmallTexels = 256;   // triangles with larger boxes go to a block each
constexpr int32_t kNoTri = 0x7f7f7f7f;   // "no triangle" (a byte-wise memset value above every index)

struct RTri {
    double x0, y0, x1, y1, x2, y2;
    int minx, maxx, miny, maxy;
    bool valid;
};

// engine/metrics.py:318-330
__device__ RTri setup_label_tri(const double* UV, const int32_t* F, int t, int res) {
    RTri r;
    const int a = F[3 * t], b = F[3 * t + 1], c = F[3 * t + 2];
    const double R = static_cast<double>(res);
    r.x0 = UV[2 * a] * R; r.y0 = UV[2 * a + 1] * R;
    r.x1 = UV[2 * b] * R; r.y1 = UV[2 * b + 1] * R;
    r.x2 = UV[2 * c] * R; r.y2 = UV[2 * c + 1] * R;
    const double area = (r.x1 - r.x0) * (r.y2 - r.y0) - (r.x2 - r.x0) * (r.y1 - r.y0);
    if (area < 0) {
        double tx = r.x1, ty = r.y1; r.x1 = r.x2; r.y1 = r.y2; r.x2 = tx; r.y2 = ty;
    }
    const double fx0 = floor(fmin(r.x0, fmin(r.x1, r.x2))), fx1 = floor(fmax(r.x0, fmax(r.x1, r.x2)));
    const double fy0 = floor(fmin(r.y0, fmin(r.y1, r.y2))), fy1 = floor(fmax(r.y0, fmax(r.y1, r.y2)));
    r.valid = isfinite(fx0) && isfinite(fx1) && isfinite(fy0) && isfinite(fy1);
    if (!r.valid) return r;
    r.minx = fx0 < 0.0 ? 0 : (fx0 > R ? res : static_cast<int>(fx0));
    r.miny = fy0 < 0.0 ? 0 : (fy0 > R ? res : static_cast<int>(fy0));
    r.maxx = fx1 > R - 1.0 ? res - 1 : (fx1 < -1.0 ? -1 : static_cast<int>(fx1));
    r.maxy = fy1 > R - 1.0 ? res - 1 : (fy1 < -1.0 ? -1 : static_cast<int>(fy1));
    return r;
}

// engine/metrics.py:331-345: inside unless some edge test e < -0.7072 L
__device__ __forceinline__ bool label_inside(const RTri& r, int px, int py) {
    const double ex[3] = {r.x1 - r.x0, r.x2 - r.x1, r.x0 - r.x2}, ey[3] = {r.y1 - r.y0, r.y2 - r.y1, r.y0 - r.y2};
    const double ox[3] = {r.x0, r.x1, r.x2}, oy[3] = {r.y0, r.y1, r.y2};
    const double cx = px + 0.5, cy = py + 0.5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double L = sqrt(ex[k] * ex[k] + ey[k] * ey[k]);
        const double e = ex[k] * (cy - oy[k]) - ey[k] * (cx - ox[k]);
        if (e < -0.7072 * L) return false;
    }
    return true;
}

__global__ void k_raster_labels(const double* UV, const int32_t* F, int m, int res, int32_t* img_t, int32_t* big,
                                int32_t* nbig) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const RTri r = setup_label_tri(UV, F, t, res);
    if (!r.valid || r.minx > r.maxx || r.miny > r.maxy) return;
    const long long area = static_cast<long long>(r.maxx - r.minx + 1) * (r.maxy - r.miny + 1);
    if (area > kSmallTexels) { big[atomicAdd(nbig, 1)] = t; return; }
    for (int py = r.miny; py <= r.maxy; ++py)
        for (int px = r.minx; px <= r.maxx; ++px)
            if (label_inside(r, px, py)) atomicMax(img_t + static_cast<size_t>(py) * res + px, t);
}

__global__ void k_raster_labels_big(const double* UV, const int32_t* F, int res, const int32_t* big, const int32_t* nbig,
                                    int32_t* img_t) {
    for (int k = blockIdx.x; k < *nbig; k += gridDim.x) {
        const int t = big[k];
        const RTri r = setup_label_tri(UV, F, t, res);
        const int w = r.maxx - r.minx + 1;
        const long long area = static_cast<long long>(w) * (r.maxy - r.miny + 1);
        for (long long q = threadIdx.x; q < area; q += blockDim.x) {
            const int px = r.minx + static_cast<int>(q % w), py = r.miny + static_cast<int>(q / w);
            if (label_inside(r, px, py)) atomicMax(img_t + static_cast<size_t>(py) * res + px, t);
        }
    }
}

__global__ void k_texel_labels(const int32_t* img_t, const int32_t* lab, size_t ntex, int32_t* img,
                               unsigned long long* filled) {
    const size_t p = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    bool f = false;
    if (p < ntex) {
        const int t = img_t[p];
        img[p] = t >= 0 ? lab[t] : -1;
        f = t >= 0;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && mask) atomicAdd(filled, static_cast<unsigned long long>(__popc(mask)));
}

// 4-neighbour filled texels with different labels: the islands touch.
__global__ void k_touch(const int32_t* img, int res, int32_t* touch) {
    const size_t p = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= static_cast<size_t>(res) * res) return;
    const int x = static_cast<int>(p % res), y = static_cast<int>(p / res);
    const int a = img[p];
    if (a < 0) return;
    if (x + 1 < res) { const int b = img[p + 1]; if (b >= 0 && b != a) *touch = 1; }
    if (y + 1 < res) { const int b = img[p + res]; if (b >= 0 && b != a) *touch = 1; }
}

// Column pass: nearest filled texel in the same column within R rows; on a
// tie the upper row (smaller index) wins. gcol = R+1 when none.
__global__ void k_colpass(const int32_t* img, int res, int R, int16_t* gcol, int16_t* grow_off) {
    const size_t p = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= static_cast<size_t>(res) * res) return;
    const int x = static_cast<int>(p % res), y = static_cast<int>(p / res);
    int g = R + 1, off = 0;
    if (img[p] >= 0) {
        g = 0;
    } else {
        for (int k = 1; k <= R; ++k) {
            if (y - k >= 0 && img[static_cast<size_t>(y - k) * res + x] >= 0) { g = k; off = -k; break; }
            if (y + k < res && img[static_cast<size_t>(y + k) * res + x] >= 0) { g = k; off = k; break; }
        }
    }
    gcol[p] = static_cast<int16_t>(g);
    grow_off[p] = static_cast<int16_t>(off);
}

// Row pass: D = min over columns j of (x-j)^2 + gcol(j)^2, smallest j on a
// tie; exact when D <= R^2, else marked unknown (-1).
__global__ void k_rowpass(const int32_t* img, const int16_t* gcol, const int16_t* grow_off, int res, int R, int32_t* D,
                          int32_t* near) {
    const size_t p = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= static_cast<size_t>(res) * res) return;
    const int x = static_cast<int>(p % res), y = static_cast<int>(p / res);
    const size_t row = static_cast<size_t>(y) * res;
    int best = 0x7fffffff, bj = -1;
    for (int k = 0; k <= R; ++k) {
        const int k2 = k * k;
        if (k2 > best) break;
        // left candidate first: on equal D the smaller column wins
        const int jl = x - k, jr = x + k;
        if (jl >= 0) {
            const int g = gcol[row + jl];
            if (g <= R) {
                const int v = k2 + g * g;
                if (v < best || (v == best && jl < bj)) { best = v; bj = jl; }
            }
        }
        if (k > 0 && jr < res) {
            const int g = gcol[row + jr];
            if (g <= R) {
                const int v = k2 + g * g;
                if (v < best || (v == best && jr < bj)) { best = v; bj = jr; }
            }
        }
    }
    if (bj < 0 || best > R * R) {
        D[p] = -1;
        near[p] = -1;
        return;
    }
    D[p] = best;
    const int fy = y + grow_off[row + bj];
    near[p] = img[static_cast<size_t>(fy) * res + bj];
}

__device__ __forceinline__ void atomic_min_nonneg(double* addr, double v) {
    atomicMin(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// min over 4-neighbour pairs with different nearest labels of d(p) + d(q).
__global__ void k_gap(const int32_t* D, const int32_t* near, int res, double* gmin) {
    const size_t p = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= static_cast<size_t>(res) * res) return;
    const int x = static_cast<int>(p % res), y = static_cast<int>(p / res);
    const int dp = D[p];
    if (dp < 0) return;
    const double sp = sqrt(static_cast<double>(dp));
    const int lp = near[p];
    double best = 1e300;
    if (x + 1 < res) {
        const int dq = D[p + 1];
        if (dq >= 0 && near[p + 1] != lp) best = fmin(best, sp + sqrt(static_cast<double>(dq)));
    }
    if (y + 1 < res) {
        const int dq = D[p + res];
        if (dq >= 0 && near[p + res] != lp) best = fmin(best, sp + sqrt(static_cast<double>(dq)));
    }
    if (best < 1e300) atomic_min_nonneg(gmin, best);
}

// ---- coverage raster (engine/metrics.py:13-54): top-left rule, counts
// saturate at 255 (order independent: the result is min(total, 255)).
__device__ void cover_tri(const double* uv, const int32_t* F, int t, int res, uint32_t* cnt, bool big_only,
                          int32_t* big, int32_t* nbig) {
    const int a = F[3 * t], b = F[3 * t + 1], c = F[3 * t + 2];
    const double R = static_cast<double>(res);
    double x0 = uv[2 * a] * R, y0 = uv[2 * a + 1] * R, x1 = uv[2 * b] * R, y1 = uv[2 * b + 1] * R;
    double x2 = uv[2 * c] * R, y2 = uv[2 * c + 1] * R;
    const double area = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
    if (area == 0.0) return;
    if (area < 0) { double tx = x1, ty = y1; x1 = x2; y1 = y2; x2 = tx; y2 = ty; }
    const double fx0 = floor(fmin(x0, fmin(x1, x2)) - 0.5), fx1 = ceil(fmax(x0, fmax(x1, x2)) - 0.5);
    const double fy0 = floor(fmin(y0, fmin(y1, y2)) - 0.5), fy1 = ceil(fmax(y0, fmax(y1, y2)) - 0.5);
    if (!(isfinite(fx0) && isfinite(fx1) && isfinite(fy0) && isfinite(fy1))) return;
    const int minx = fx0 < 0.0 ? 0 : (fx0 > R ? res : static_cast<int>(fx0));
    const int miny = fy0 < 0.0 ? 0 : (fy0 > R ? res : static_cast<int>(fy0));
    const int maxx = fx1 > R - 1.0 ? res - 1 : (fx1 < -1.0 ? -1 : static_cast<int>(fx1));
    const int maxy = fy1 > R - 1.0 ? res - 1 : (fy1 < -1.0 ? -1 : static_cast<int>(fy1));
    if (minx > maxx || miny > maxy) return;
    const long long n = static_cast<long long>(maxx - minx + 1) * (maxy - miny + 1);
    if (!big_only && n > kSmallTexels) { big[atomicAdd(nbig, 1)] = t; return; }
    const double ex[3] = {x1 - x0, x2 - x1, x0 - x2}, ey[3] = {y1 - y0, y2 - y1, y0 - y2};
    const double ox[3] = {x0, x1, x2}, oy[3] = {y0, y1, y2};
    const int w = maxx - minx + 1;
    const long long start = big_only ? threadIdx.x : 0, step = big_only ? blockDim.x : 1;
    for (long long q = start; q < n; q += step) {
        const int px = minx + static_cast<int>(q % w), py = miny + static_cast<int>(q / w);
        const double cx = px + 0.5, cy = py + 0.5;
        bool inside = true;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double e = ex[k] * (cy - oy[k]) - ey[k] * (cx - ox[k]);
            if (e < 0.0) { inside = false; break; }
            if (e == 0.0) {
                const bool top_left = (ey[k] == 0.0 && ex[k] < 0.0) || ey[k] > 0.0;
                if (!top_left) { inside = false; break; }
            }
        }
        if (inside) atomicAdd(cnt + static_cast<size_t>(py) * res + px, 1u);
    }
}

__global__ void k_cover(const double* uv, const int32_t* F, int m, int res, uint32_t* cnt, int32_t* big, int32_t* nbig) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) cover_tri(uv, F, t, res, cnt, false, big, nbig);
}

__global__ void k_cover_big(const double* uv, const int32_t* F, int res, uint32_t* cnt, const int32_t* big,
                            const int32_t* nbig) {
    for (int k = blockIdx.x; k < *nbig; k += gridDim.x) cover_tri(uv, F, big[k], res, cnt, true, nullptr, nullptr);
}

__global__ void k_cover_final(const uint32_t* cnt, size_t ntex, uint8_t* out, unsigned long long* stats) {
    const size_t p = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    bool covered = false, over = false;
    if (p < ntex) {
        const uint32_t c = cnt[p];
        out[p] = static_cast<uint8_t>(c < 255u ? c : 255u);
        covered = c > 0;
        over = c > 1;
    }
    unsigned mask = __ballot_sync(0xffffffffu, covered);
    if ((threadIdx.x & 31) == 0 && mask) atomicAdd(stats, static_cast<unsigned long long>(__popc(mask)));
    mask = __ballot_sync(0xffffffffu, over);
    if ((threadIdx.x & 31) == 0 && mask) atomicAdd(stats + 1, static_cast<unsigned long long>(__popc(mask)));
}

// ---- texel-centre overlaps of one chart (engine/overlapfix.py:135-224):
// the coverage rule above; every covered texel centre of triangle t in
// row-major order of its box gets visit(q, texel), q the box-local index. A
// box above kSmallTexels texels is queued on `big` instead (unless big_only,
// where the block's threads split the box).
template <typename Visit>
__device__ void texel_walk(const double* uv, const int32_t* F, int t, int res, bool big_only, int32_t* big,
                           int32_t* nbig, Visit visit) {
    const int a = F[3 * t], b = F[3 * t + 1], c = F[3 * t + 2];
    const double R = static_cast<double>(res);
    double x0 = uv[2 * a] * R, y0 = uv[2 * a + 1] * R, x1 = uv[2 * b] * R, y1 = uv[2 * b + 1] * R;
    double x2 = uv[2 * c] * R, y2 = uv[2 * c + 1] * R;
    const double area = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
    if (area == 0.0) return;
    if (area < 0) { double tx = x1, ty = y1; x1 = x2; y1 = y2; x2 = tx; y2 = ty; }
    const double fx0 = floor(fmin(x0, fmin(x1, x2)) - 0.5), fx1 = ceil(fmax(x0, fmax(x1, x2)) - 0.5);
    const double fy0 = floor(fmin(y0, fmin(y1, y2)) - 0.5), fy1 = ceil(fmax(y0, fmax(y1, y2)) - 0.5);
    if (!(isfinite(fx0) && isfinite(fx1) && isfinite(fy0) && isfinite(fy1))) return;
    const int minx = fx0 < 0.0 ? 0 : (fx0 > R ? res : static_cast<int>(fx0));
    const int miny = fy0 < 0.0 ? 0 : (fy0 > R ? res : static_cast<int>(fy0));
    const int maxx = fx1 > R - 1.0 ? res - 1 : (fx1 < -1.0 ? -1 : static_cast<int>(fx1));
    const int maxy = fy1 > R - 1.0 ? res - 1 : (fy1 < -1.0 ? -1 : static_cast<int>(fy1));
    if (minx > maxx || miny > maxy) return;
    const long long n = static_cast<long long>(maxx - minx + 1) * (maxy - miny + 1);
    if (!big_only && n > kSmallTexels) { if (big) big[atomicAdd(nbig, 1)] = t; return; }
    const double ex[3] = {x1 - x0, x2 - x1, x0 - x2}, ey[3] = {y1 - y0, y2 - y1, y0 - y2};
    const double ox[3] = {x0, x1, x2}, oy[3] = {y0, y1, y2};
    const int w = maxx - minx + 1;
    const long long start = big_only ? threadIdx.x : 0, step = big_only ? blockDim.x : 1;
    for (long long q = start; q < n; q += step) {
        const int px = minx + static_cast<int>(q % w), py = miny + static_cast<int>(q / w);
        const double cx = px + 0.5, cy = py + 0.5;
        bool inside = true;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double e = ex[k] * (cy - oy[k]) - ey[k] * (cx - ox[k]);
            if (e < 0.0) { inside = false; break; }
            if (e == 0.0) {
                const bool top_left = (ey[k] == 0.0 && ex[k] < 0.0) || ey[k] > 0.0;
                if (!top_left) { inside = false; break; }
            }
        }
        if (inside) visit(q, static_cast<size_t>(py) * res + px);
    }
}

// pass 1: coverage counts and the first (smallest) triangle on every texel
__global__ void k_ov_cover(const double* uv, const int32_t* F, int m, int res, uint32_t* cnt, int32_t* owner,
                           int32_t* big, int32_t* nbig) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    texel_walk(uv, F, t, res, false, big, nbig, [&](long long, size_t p) { atomicAdd(cnt + p, 1u); atomicMin(owner + p, t); });
}
__global__ void k_ov_cover_big(const double* uv, const int32_t* F, int res, uint32_t* cnt, int32_t* owner,
                               const int32_t* big, const int32_t* nbig) {
    for (int k = blockIdx.x; k < *nbig; k += gridDim.x) {
        const int t = big[k];
        texel_walk(uv, F, t, res, true, nullptr, nullptr,
                   [&](long long, size_t p) { atomicAdd(cnt + p, 1u); atomicMin(owner + p, t); });
    }
}

// pass 2: flags (a covered texel with two coverers) and the first triangle
// that meets a texel an earlier triangle owns
__global__ void k_ov_check(const double* uv, const int32_t* F, int m, int res, const uint32_t* cnt,
                           const int32_t* owner, uint8_t* flags, int32_t* first_t) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    bool shared = false, earlier = false;
    texel_walk(uv, F, t, res, false, nullptr, nullptr, [&](long long, size_t p) {
        shared |= cnt[p] > 1u;
        earlier |= owner[p] < t;
    });
    if (flags) flags[t] = shared ? 1 : 0;
    if (earlier) atomicMin(first_t, t);
}
__global__ void k_ov_check_big(const double* uv, const int32_t* F, int res, const uint32_t* cnt, const int32_t* owner,
                               const int32_t* big, const int32_t* nbig, uint8_t* flags, int32_t* first_t) {
    __shared__ int s_shared, s_earlier;
    for (int k = blockIdx.x; k < *nbig; k += gridDim.x) {
        const int t = big[k];
        if (threadIdx.x == 0) { s_shared = 0; s_earlier = 0; }
        __syncthreads();
        bool shared = false, earlier = false;
        texel_walk(uv, F, t, res, true, nullptr, nullptr, [&](long long, size_t p) {
            shared |= cnt[p] > 1u;
            earlier |= owner[p] < t;
        });
        if (shared) s_shared = 1;
        if (earlier) s_earlier = 1;
        __syncthreads();
        if (threadIdx.x == 0) {
            if (flags) flags[t] = s_shared ? 1 : 0;
            if (s_earlier) atomicMin(first_t, t);
        }
        __syncthreads();
    }
}

// pass 3 (one block): the first texel, in the scan order of triangle
// first_t, that an earlier triangle owns -> (its owner, first_t). The key
// packs the box-local index (high word) over the owner (low word).
__global__ void k_ov_pair(const double* uv, const int32_t* F, int res, const int32_t* owner, const int32_t* first_t,
                          int32_t* pair) {
    __shared__ unsigned long long s_key;
    const int t = *first_t;
    if (threadIdx.x == 0) s_key = ~0ull;
    __syncthreads();
    if (t != kNoTri) {
        unsigned long long best = ~0ull;
        texel_walk(uv, F, t, res, true, nullptr, nullptr, [&](long long q, size_t p) {
            const int o = owner[p];
            if (o < t) {
                const unsigned long long key = (static_cast<unsigned long long>(q) << 32) | static_cast<uint32_t>(o);
                if (key < best) best = key;
            }
        });
        if (best != ~0ull) atomicMin(&s_key, best);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const bool none = t == kNoTri || s_key == ~0ull;
        pair[0] = none ? -1 : static_cast<int32_t>(s_key & 0xffffffffull);
        pair[1] = none ? -1 : t;
    }
}

__global__ void k_gutter_init(double* out, double radius) {
    out[0] = 1e300; out[1] = 0.0; out[2] = 0.0; out[3] = radius;
}

__global__ void k_gutter_final(const unsigned long long* filled, const int32_t* touch, double* out) {
    out[1] = static_cast<double>(*filled);
    out[2] = *touch ? 1.0 : 0.0;
}

size_t gutter_bytes(int64_t res, int64_t m) {
    const size_t ntex = static_cast<size_t>(res) * res;
    auto al = [](size_t x) { return (x + 255) & ~static_cast<size_t>(255); };
    return al(4 * ntex) * 4 + al(2 * ntex) * 2 + al(4 * static_cast<size_t>(std::max<int64_t>(m, 1))) + 256;
}

}  // namespace

extern "C" int uva_gutter_scratch_bytes(int32_t res, int64_t m, int64_t* bytes) {
    if (res <= 0 || res > 16384 || m < 0 || !bytes) { uva_set_error("uva_gutter_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    *bytes = static_cast<int64_t>(gutter_bytes(res, m));
    return UVA_OK;
}

// Labels raster + windowed exact EDT + gap. out (device, 4 doubles):
// [0] minimum d(p)+d(q) over pairs with both distances exact (1e300: none),
// [1] filled texels, [2] 1 if two islands touch, [3] the radius used.
// img (device, res*res int32) receives the label raster (-1 empty).
extern "C" int uva_gutter(const double* UV, const int32_t* F, const int32_t* labels, int32_t m, int32_t res,
                          int32_t radius, int32_t* img, void* scratch, int64_t scratch_bytes, double* out, void* stream) {
    if (m < 0 || res <= 0 || res > 16384 || radius <= 0 || !img || !out || !scratch ||
        (m > 0 && (!UV || !F || !labels))) {
        uva_set_error("uva_gutter: bad arguments");
        return UVA_E_ARG;
    }
    if (scratch_bytes < static_cast<int64_t>(gutter_bytes(res, m))) { uva_set_error("uva_gutter: scratch too small"); return UVA_E_ARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t ntex = static_cast<size_t>(res) * res;
    auto al = [](size_t x) { return (x + 255) & ~static_cast<size_t>(255); };
    auto* base = static_cast<unsigned char*>(scratch);
    int32_t* img_t = reinterpret_cast<int32_t*>(base); base += al(4 * ntex);
    int32_t* D = reinterpret_cast<int32_t*>(base); base += al(4 * ntex);
    int32_t* nearl = reinterpret_cast<int32_t*>(base); base += al(4 * ntex);
    base += al(4 * ntex);   // reserved
    int16_t* gcol = reinterpret_cast<int16_t*>(base); base += al(2 * ntex);
    int16_t* goff = reinterpret_cast<int16_t*>(base); base += al(2 * ntex);
    int32_t* big = reinterpret_cast<int32_t*>(base); base += al(4 * static_cast<size_t>(std::max(m, 1)));
    int32_t* smalls = reinterpret_cast<int32_t*>(base);
    const int R = std::min(radius, 32000);
    cudaMemsetAsync(img_t, 0xff, 4 * ntex, s);
    cudaMemsetAsync(smalls, 0, 256, s);
    k_gutter_init<<<1, 1, 0, s>>>(out, static_cast<double>(R));
    const int tb = 256;
    const unsigned gtex = static_cast<unsigned>((ntex + tb - 1) / tb);
    if (m > 0) {
        k_raster_labels<<<(m + tb - 1) / tb, tb, 0, s>>>(UV, F, m, res, img_t, big, smalls);
        k_raster_labels_big<<<148, tb, 0, s>>>(UV, F, res, big, smalls, img_t);
    }
    unsigned long long* filled = reinterpret_cast<unsigned long long*>(smalls + 8);
    k_texel_labels<<<gtex, tb, 0, s>>>(img_t, labels, ntex, img, filled);
    k_touch<<<gtex, tb, 0, s>>>(img, res, smalls + 2);
    k_colpass<<<gtex, tb, 0, s>>>(img, res, R, gcol, goff);
    k_rowpass<<<gtex, tb, 0, s>>>(img, gcol, goff, res, R, D, nearl);
    k_gap<<<gtex, tb, 0, s>>>(D, nearl, res, out);
    UVA_CHECK_LAUNCH("uva_gutter");
    k_gutter_final<<<1, 1, 0, s>>>(filled, smalls + 2, out);
    UVA_CHECK_LAUNCH("uva_gutter/final");
    return UVA_OK;
}

// Texel-centre overlaps of one chart (engine/overlapfix.py:135-224, 263-275).
extern "C" int uva_overlap_raster(const double* uv, const int32_t* F, int32_t m, int32_t res, uint8_t* flags,
                                  int32_t* pair, void* scratch, int64_t scratch_bytes, void* stream) {
    if (m < 0 || m >= kNoTri || res <= 0 || res > 16384 || !scratch || (!flags && !pair) || (m > 0 && (!uv || !F))) {
        uva_set_error("uva_overlap_raster: bad arguments");
        return UVA_E_ARG;
    }
    if (scratch_bytes < static_cast<int64_t>(gutter_bytes(res, m))) { uva_set_error("uva_overlap_raster: scratch too small"); return UVA_E_ARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t ntex = static_cast<size_t>(res) * res;
    auto al = [](size_t x) { return (x + 255) & ~static_cast<size_t>(255); };
    auto* base = static_cast<unsigned char*>(scratch);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(base); base += al(4 * ntex);
    int32_t* owner = reinterpret_cast<int32_t*>(base); base += al(4 * ntex) * 3 + al(2 * ntex) * 2;
    int32_t* big = reinterpret_cast<int32_t*>(base); base += al(4 * static_cast<size_t>(std::max(m, 1)));
    int32_t* smalls = reinterpret_cast<int32_t*>(base);   // [0] big count, [1] first triangle
    cudaMemsetAsync(cnt, 0, 4 * ntex, s);
    cudaMemsetAsync(owner, 0x7f, 4 * ntex, s);            // kNoTri on every texel
    cudaMemsetAsync(smalls, 0, 4, s);
    cudaMemsetAsync(smalls + 1, 0x7f, 4, s);
    const int tb = 256;
    if (m > 0) {
        k_ov_cover<<<(m + tb - 1) / tb, tb, 0, s>>>(uv, F, m, res, cnt, owner, big, smalls);
        k_ov_cover_big<<<148, tb, 0, s>>>(uv, F, res, cnt, owner, big, smalls);
        k_ov_check<<<(m + tb - 1) / tb, tb, 0, s>>>(uv, F, m, res, cnt, owner, flags, smalls + 1);
        k_ov_check_big<<<148, tb, 0, s>>>(uv, F, res, cnt, owner, big, smalls, flags, smalls + 1);
    }
    if (pair) k_ov_pair<<<1, tb, 0, s>>>(uv, F, res, owner, smalls + 1, pair);
    UVA_CHECK_LAUNCH("uva_overlap_raster");
    return UVA_OK;
}

// Coverage raster (engine/metrics.py:13-62). counts: res*res uint8 out;
// stats (device, 2 int64): covered texels, texels covered more than once.
extern "C" int uva_raster_counts(const double* uv, const int32_t* F, int32_t m, int32_t res, uint8_t* counts,
                                 int64_t* stats, void* scratch, int64_t scratch_bytes, void* stream) {
    if (m < 0 || res <= 0 || res > 16384 || !counts || !stats || !scratch || (m > 0 && (!uv || !F))) {
        uva_set_error("uva_raster_counts: bad arguments");
        return UVA_E_ARG;
    }
    if (scratch_bytes < static_cast<int64_t>(gutter_bytes(res, m))) { uva_set_error("uva_raster_counts: scratch too small"); return UVA_E_ARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t ntex = static_cast<size_t>(res) * res;
    auto al = [](size_t x) { return (x + 255) & ~static_cast<size_t>(255); };
    auto* base = static_cast<unsigned char*>(scratch);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(base); base += al(4 * ntex) * 4 + al(2 * ntex) * 2;
    int32_t* big = reinterpret_cast<int32_t*>(base); base += al(4 * static_cast<size_t>(std::max(m, 1)));
    int32_t* smalls = reinterpret_cast<int32_t*>(base);
    cudaMemsetAsync(cnt, 0, 4 * ntex, s);
    cudaMemsetAsync(smalls, 0, 256, s);
    cudaMemsetAsync(stats, 0, 16, s);
    const int tb = 256;
    if (m > 0) {
        k_cover<<<(m + tb - 1) / tb, tb, 0, s>>>(uv, F, m, res, cnt, big, smalls);
        k_cover_big<<<148, tb, 0, s>>>(uv, F, res, cnt, big, smalls);
    }
    k_cover_final<<<static_cast<unsigned>((ntex + tb - 1) / tb), tb, 0, s>>>(cnt, ntex, counts,
                                                                            reinterpret_cast<unsigned long long*>(stats));
    UVA_CHECK_LAUNCH("uva_raster_counts");
    return UVA_OK;
}
