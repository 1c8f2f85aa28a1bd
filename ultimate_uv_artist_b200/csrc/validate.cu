// Exact validation of exported float32 UVs (engine/validate.py:139-226).
//
// Compiled with --fmad=false: every FP64 predicate rounds each operation like
// the reference's numba kernels, so verdicts are bit-exact. Pipeline (one
// stream, no host synchronisation):
//   k_v_rows      per vertex: non-finite / outside-[0,1] counts (per UV row)
//   k_v_area3     per face: 3D area (numpy order), global max
//   k_v_classify  per face: signed UV area, sliver, has3d, skip, counts, cell box
//   weld + union-find: islands over vertices welded by identical float32
//                 (position, uv) bytes (engine/metrics.py:91-103)
//   orientation   per island positive / negative area; near-ties are re-summed
//                 in face order (the reference's np.bincount order)
//   overlap       uniform grid; each candidate pair tested once, in the first
//                 cell both cell boxes share; tolerant and strict predicates
//   islands with overlap, flipped triangles
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"

using namespace uva;

namespace {

constexpr int kMaxCells = 16;        // cells per triangle on the binned path
constexpr double kUlp32 = 5.9604644775390625e-08;   // 2^-24

// ------------------------------------------------------------------ predicates
__device__ __forceinline__ double orient(double ax, double ay, double bx, double by, double cx, double cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

__device__ __forceinline__ double maxd(double a, double b) { return a > b ? a : b; }

// engine/validate.py:33-45
__device__ bool strict_inside(double px, double py, double ax, double ay, double bx, double by, double cx, double cy,
                              double rel) {
    const double l = maxd((bx - ax) * (bx - ax) + (by - ay) * (by - ay),
                          maxd((cx - bx) * (cx - bx) + (cy - by) * (cy - by), (ax - cx) * (ax - cx) + (ay - cy) * (ay - cy)));
    const double eps = rel > 0.0 ? maxd(rel * l, 4.0 * kUlp32 * sqrt(l)) : 0.0;
    const double d1 = orient(ax, ay, bx, by, px, py);
    const double d2 = orient(bx, by, cx, cy, px, py);
    const double d3 = orient(cx, cy, ax, ay, px, py);
    if (d1 > eps && d2 > eps && d3 > eps) return true;
    if (d1 < -eps && d2 < -eps && d3 < -eps) return true;
    return false;
}

// engine/validate.py:48-54
__device__ bool proper_cross(double ax, double ay, double bx, double by, double cx, double cy, double dx, double dy,
                             double rel) {
    const double l1 = (bx - ax) * (bx - ax) + (by - ay) * (by - ay);
    const double l2 = (dx - cx) * (dx - cx) + (dy - cy) * (dy - cy);
    const double e1 = maxd(rel * l1, 4.0 * kUlp32 * sqrt(l1));
    const double e2 = maxd(rel * l2, 4.0 * kUlp32 * sqrt(l2));
    const double o1 = orient(ax, ay, bx, by, cx, cy), o2 = orient(ax, ay, bx, by, dx, dy);
    const double o3 = orient(cx, cy, dx, dy, ax, ay), o4 = orient(cx, cy, dx, dy, bx, by);
    return ((o1 > e1 && o2 < -e1) || (o1 < -e1 && o2 > e1)) && ((o3 > e2 && o4 < -e2) || (o3 < -e2 && o4 > e2));
}

struct Tri {
    double x[3], y[3];
};

template <typename UVT>
__device__ __forceinline__ Tri load_tri(const UVT* UV, const int32_t* F, int t) {
    Tri r;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int v = F[3 * t + k];
        r.x[k] = static_cast<double>(UV[2 * v]);
        r.y[k] = static_cast<double>(UV[2 * v + 1]);
    }
    return r;
}

// Tolerant (engine/validate.py:57-91) and strict (:232-255) overlap of one
// pair, evaluated together. bit0: tolerant, bit1: strict.
__device__ int pair_overlap(const Tri& a, const Tri& b, double rel) {
    bool same[3][3];
    int shared = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        bool any = false;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            same[i][j] = a.x[i] == b.x[j] && a.y[i] == b.y[j];
            any |= same[i][j];
        }
        shared += any ? 1 : 0;
    }
    if (shared == 3) return 0;
    int tol = 0, strict = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int p0 = i, p1 = (i + 1) % 3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int q0 = j, q1 = (j + 1) % 3;
            if (same[p0][q0] || same[p0][q1] || same[p1][q0] || same[p1][q1]) continue;
            if (!tol && proper_cross(a.x[p0], a.y[p0], a.x[p1], a.y[p1], b.x[q0], b.y[q0], b.x[q1], b.y[q1], rel)) tol = 1;
            if (!strict) {
                const double o1 = orient(a.x[p0], a.y[p0], a.x[p1], a.y[p1], b.x[q0], b.y[q0]);
                const double o2 = orient(a.x[p0], a.y[p0], a.x[p1], a.y[p1], b.x[q1], b.y[q1]);
                const double o3 = orient(b.x[q0], b.y[q0], b.x[q1], b.y[q1], a.x[p0], a.y[p0]);
                const double o4 = orient(b.x[q0], b.y[q0], b.x[q1], b.y[q1], a.x[p1], a.y[p1]);
                if (o1 * o2 < 0.0 && o3 * o4 < 0.0) strict = 1;
            }
        }
    }
    if (!tol) {
#pragma unroll
        for (int i = 0; i < 3 && !tol; ++i) {
            if (!(same[i][0] || same[i][1] || same[i][2]) &&
                strict_inside(a.x[i], a.y[i], b.x[0], b.y[0], b.x[1], b.y[1], b.x[2], b.y[2], rel)) tol = 1;
            if (!tol && !(same[0][i] || same[1][i] || same[2][i]) &&
                strict_inside(b.x[i], b.y[i], a.x[0], a.y[0], a.x[1], a.y[1], a.x[2], a.y[2], rel)) tol = 1;
        }
    }
    if (!tol) {
        const double cx = (a.x[0] + a.x[1] + a.x[2]) / 3.0, cy = (a.y[0] + a.y[1] + a.y[2]) / 3.0;
        if (strict_inside(cx, cy, b.x[0], b.y[0], b.x[1], b.y[1], b.x[2], b.y[2], rel)) tol = 1;
    }
    if (!tol) {
        const double cx = (b.x[0] + b.x[1] + b.x[2]) / 3.0, cy = (b.y[0] + b.y[1] + b.y[2]) / 3.0;
        if (strict_inside(cx, cy, a.x[0], a.y[0], a.x[1], a.y[1], a.x[2], a.y[2], rel)) tol = 1;
    }
    return tol | (strict << 1);
}

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ void count_add(unsigned long long* c, bool pred) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if ((threadIdx.x & 31) == 0 && mask) atomicAdd(c, static_cast<unsigned long long>(__popc(mask)));
}

// ------------------------------------------------------------------ per vertex / per face
__global__ void k_v_rows(int n, const float* UV, unsigned long long* counts) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    bool nf = false, out = false;
    if (v < n) {
        const double u = UV[2 * v], w = UV[2 * v + 1];
        nf = !isfinite(u) || !isfinite(w);
        out = u < 0.0 || u > 1.0 || w < 0.0 || w > 1.0;
    }
    count_add(counts + UVA_VC_NONFINITE, nf);
    count_add(counts + UVA_VC_OUTSIDE, out);
}

// The maximum is taken over the warp first (bit patterns of non-negative
// doubles order like the values; NaN and negatives are left out, as in
// atomic_max_nonneg), then one atomic per warp: a single address took one
// atomic per face before.
__global__ void k_v_area3(int m, const double* V, const int32_t* F, double* a3, double* amax) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long w = 0;   // +0.0: amax starts there
    if (t < m) {
        const int i0 = F[3 * t], i1 = F[3 * t + 1], i2 = F[3 * t + 2];
        const double ax = V[3 * i1] - V[3 * i0], ay = V[3 * i1 + 1] - V[3 * i0 + 1], az = V[3 * i1 + 2] - V[3 * i0 + 2];
        const double bx = V[3 * i2] - V[3 * i0], by = V[3 * i2 + 1] - V[3 * i0 + 1], bz = V[3 * i2 + 2] - V[3 * i0 + 2];
        const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
        const double a = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
        a3[t] = a;
        if (a >= 0.0) w = static_cast<unsigned long long>(__double_as_longlong(a));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, w, o);
        w = y > w ? y : w;
    }
    if ((threadIdx.x & 31) == 0 && w) atomicMax(reinterpret_cast<unsigned long long*>(amax), w);
}

// engine/validate.py:149-172: signed area, sliver, has3d, skip; cell boxes.
__global__ void k_v_classify(int m, const float* UV, const int32_t* F, const double* a3, const double* amax, int G,
                             double* sa_out, uint8_t* tflags, int4* cbox, unsigned long long* counts) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    bool deg = false, sl = false;
    if (t < m) {
        const Tri r = load_tri(UV, F, t);
        const double sa = 0.5 * ((r.x[1] - r.x[0]) * (r.y[2] - r.y[0]) - (r.x[2] - r.x[0]) * (r.y[1] - r.y[0]));
        const double e0 = sqrt((r.x[1] - r.x[0]) * (r.x[1] - r.x[0]) + (r.y[1] - r.y[0]) * (r.y[1] - r.y[0]));
        const double e1 = sqrt((r.x[2] - r.x[1]) * (r.x[2] - r.x[1]) + (r.y[2] - r.y[1]) * (r.y[2] - r.y[1]));
        const double e2 = sqrt((r.x[0] - r.x[2]) * (r.x[0] - r.x[2]) + (r.y[0] - r.y[2]) * (r.y[0] - r.y[2]));
        // np.maximum propagates NaN
        double edge = e0;
        if (isnan(e1) || e1 > edge) edge = isnan(edge) ? edge : e1;
        if (isnan(e2) || e2 > edge) edge = isnan(edge) ? edge : e2;
        double em = edge;
        if (!(em >= kUlp32) && !isnan(em)) em = kUlp32;
        const bool sliver = fabs(sa) < kUlp32 * em;
        const double amx = *amax;
        const bool has3d = a3[t] > 1e-14 * (amx > 1e-30 ? amx : 1e-30);
        const bool skip = !has3d || sliver || !isfinite(sa);
        deg = has3d && sa == 0.0;
        sl = has3d && sliver;
        sa_out[t] = sa;
        tflags[t] = static_cast<uint8_t>((has3d ? 1 : 0) | (sliver ? 2 : 0) | (skip ? 4 : 0));
        if (!skip) {
            double lx = r.x[0], hx = r.x[0], ly = r.y[0], hy = r.y[0];
#pragma unroll
            for (int k = 1; k < 3; ++k) {
                lx = fmin(lx, r.x[k]); hx = fmax(hx, r.x[k]);
                ly = fmin(ly, r.y[k]); hy = fmax(hy, r.y[k]);
            }
            auto cell = [G](double u) {
                const double s = u * static_cast<double>(G);
                int c = s >= 2147483647.0 ? 2147483647 : (s <= -2147483647.0 ? -2147483647 : static_cast<int>(s));
                return c < 0 ? 0 : (c > G - 1 ? G - 1 : c);
            };
            cbox[t] = make_int4(cell(lx), cell(hx), cell(ly), cell(hy));
        } else {
            cbox[t] = make_int4(1, 0, 1, 0);   // empty
        }
    }
    count_add(counts + UVA_VC_DEGENERATE, deg);
    count_add(counts + UVA_VC_SLIVERS, sl);
}

// ------------------------------------------------------------------ islands
__device__ __forceinline__ uint32_t mix(uint32_t h, uint32_t k) {
    k *= 0xcc9e2d51u; k = (k << 15) | (k >> 17); k *= 0x1b873593u;
    h ^= k; h = (h << 13) | (h >> 19); return h * 5u + 0xe6546b64u;
}

__device__ __forceinline__ void vkey(const double* V, const float* UV, int v, uint32_t (&k)[5]) {
    k[0] = __float_as_uint(__double2float_rn(V[3 * v]));
    k[1] = __float_as_uint(__double2float_rn(V[3 * v + 1]));
    k[2] = __float_as_uint(__double2float_rn(V[3 * v + 2]));
    k[3] = __float_as_uint(UV[2 * v]);
    k[4] = __float_as_uint(UV[2 * v + 1]);
}

// Weld: representative = the first vertex to claim the hash slot of its key.
__global__ void k_weld(int n, const double* V, const float* UV, int32_t* table, uint32_t hmask, int32_t* rep) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    uint32_t k[5];
    vkey(V, UV, v, k);
    uint32_t h = 0x9747b28cu;
#pragma unroll
    for (int i = 0; i < 5; ++i) h = mix(h, k[i]);
    h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13;
    for (uint32_t probe = 0; probe <= hmask; ++probe) {
        const uint32_t s = (h + probe) & hmask;
        const int32_t prev = atomicCAS(table + s, -1, v);
        if (prev == -1) { rep[v] = v; return; }
        uint32_t o[5];
        vkey(V, UV, prev, o);
        if (o[0] == k[0] && o[1] == k[1] && o[2] == k[2] && o[3] == k[3] && o[4] == k[4]) { rep[v] = prev; return; }
    }
    rep[v] = v;   // table full: cannot happen (2x oversized)
}

__device__ __forceinline__ int uf_find(int32_t* parent, int x) {
    int p = parent[x];
    while (p != x) {
        const int g = parent[p];
        if (g != p) parent[x] = g;   // path halving (benign race: g is an ancestor)
        x = p;
        p = g;
    }
    return x;
}

__device__ void uf_union(int32_t* parent, int a, int b) {
    for (;;) {
        a = uf_find(parent, a);
        b = uf_find(parent, b);
        if (a == b) return;
        if (a < b) { const int t = a; a = b; b = t; }   // hook the larger root under the smaller
        if (atomicCAS(parent + a, a, b) == a) return;
    }
}

__global__ void k_identity(int n, int32_t* rep) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) rep[v] = v;
}

__global__ void k_uf_init(int n, const int32_t* rep, int32_t* parent) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) parent[v] = rep[v];
}

__global__ void k_uf_faces(int m, const int32_t* F, const int32_t* rep, int32_t* parent) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int a = rep[F[3 * t]];
    uf_union(parent, a, rep[F[3 * t + 1]]);
    uf_union(parent, a, rep[F[3 * t + 2]]);
}

__global__ void k_uf_roots(int m, const int32_t* F, const int32_t* rep, int32_t* parent, int32_t* froot, int32_t* rflag) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int r = uf_find(parent, rep[F[3 * t]]);
    froot[t] = r;
    rflag[r] = 1;
}

// ------------------------------------------------------------------ scan (exclusive, int32)
constexpr int kScanB = 1024;

__global__ void k_scan_local(const int32_t* in, int32_t* out, int32_t* sums, int n) {
    __shared__ int32_t s[kScanB];
    const int i = blockIdx.x * kScanB + threadIdx.x;
    const int x = i < n ? in[i] : 0;
    s[threadIdx.x] = x;
    __syncthreads();
    for (int o = 1; o < kScanB; o <<= 1) {
        const int y = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += y;
        __syncthreads();
    }
    if (i < n) out[i] = s[threadIdx.x] - x;
    if (threadIdx.x == kScanB - 1) sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void k_scan_sums(int32_t* sums, int nb, int32_t* total) {
    __shared__ int32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    __shared__ int32_t s[kScanB];
    for (int base = 0; base < nb; base += kScanB) {
        const int i = base + threadIdx.x;
        const int x = i < nb ? sums[i] : 0;
        s[threadIdx.x] = x;
        __syncthreads();
        for (int o = 1; o < kScanB; o <<= 1) {
            const int y = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += y;
            __syncthreads();
        }
        if (i < nb) sums[i] = carry + s[threadIdx.x] - x;
        __syncthreads();
        if (threadIdx.x == kScanB - 1) carry += s[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(int32_t* out, const int32_t* sums, int n) {
    const int i = blockIdx.x * kScanB + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

void scan(const int32_t* in, int32_t* out, int32_t* sums, int32_t* total, int n, cudaStream_t s) {
    const int nb = std::max(1, (n + kScanB - 1) / kScanB);
    k_scan_local<<<nb, kScanB, 0, s>>>(in, out, sums, n);
    k_scan_sums<<<1, kScanB, 0, s>>>(sums, nb, total);
    k_scan_add<<<nb, kScanB, 0, s>>>(out, sums, n);
}

// ------------------------------------------------------------------ orientation
__global__ void k_labels(int m, const int32_t* froot, const int32_t* rank, int32_t* labels) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) labels[t] = rank[froot[t]];
}

__global__ void k_orient_sums(int m, const double* sa, const int32_t* labels, double* pos, double* neg, int32_t* cnt) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const double s = sa[t];
    const int l = labels[t];
    if (s > 0.0) atomicAdd(pos + l, s);
    else if (s < 0.0) atomicAdd(neg + l, -s);
    atomicAdd(cnt + l, 1);
}

// dom = pos >= neg. Sums of k non-negative terms in any order are within
// (k-1) 2^-53 (pos + neg) of the exact value, and so are the reference's
// sequential sums: islands closer than twice that are ambiguous and get the
// reference's face-order sum.
__global__ void k_orient_decide(const int32_t* nl, const double* pos, const double* neg, const int32_t* cnt, int8_t* dom,
                                int32_t* amb, int32_t* namb) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= *nl) return;
    const double p = pos[l], q = neg[l];
    const double bound = 4.0 * static_cast<double>(cnt[l]) * 1.1102230246251565e-16 * (p + q);
    if (p == 0.0 && q == 0.0) {
        dom[l] = 1;   // no non-zero term: exact in any order
    } else if (fabs(p - q) <= bound) {
        dom[l] = 0;
        amb[atomicAdd(namb, 1)] = l;
    } else {
        dom[l] = p >= q ? 1 : -1;
    }
}

// Reference order: np.bincount walks faces in index order (one thread per
// ambiguous island, rare).
__global__ void k_orient_exact(int m, const double* sa, const int32_t* labels, const int32_t* amb, const int32_t* namb,
                               int8_t* dom) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < *namb; k += gridDim.x * blockDim.x) {
        const int l = amb[k];
        double p = 0.0, q = 0.0;
        for (int t = 0; t < m; ++t) {
            if (labels[t] != l) continue;
            const double s = sa[t];
            p += s > 0.0 ? fabs(s) : 0.0;
            q += s < 0.0 ? fabs(s) : 0.0;
        }
        dom[l] = p >= q ? 1 : -1;
    }
}

__global__ void k_mirrored(int nmax, const int32_t* nl, const int8_t* dom, unsigned long long* counts) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    count_add(counts + UVA_VC_MIRRORED, l < nmax && l < *nl && dom[l] < 0);
}

// ------------------------------------------------------------------ binning
__global__ void k_bin_count(int m, const int4* cbox, int G, int32_t* ccount, int32_t* big, int32_t* nbig) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int4 c = cbox[t];
    if (c.x > c.y) return;   // skipped
    const int nx = c.y - c.x + 1, ny = c.w - c.z + 1;
    if (nx * ny > kMaxCells) { big[atomicAdd(nbig, 1)] = t; return; }
    for (int gy = c.z; gy <= c.w; ++gy)
        for (int gx = c.x; gx <= c.y; ++gx) atomicAdd(ccount + gy * G + gx, 1);
}

__global__ void k_bin_fill(int m, const int4* cbox, int G, const int32_t* cofs, int32_t* cursor, int32_t* items) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int4 c = cbox[t];
    if (c.x > c.y) return;
    const int nx = c.y - c.x + 1, ny = c.w - c.z + 1;
    if (nx * ny > kMaxCells) return;
    for (int gy = c.z; gy <= c.w; ++gy)
        for (int gx = c.x; gx <= c.y; ++gx) {
            const int cell = gy * G + gx;
            items[cofs[cell] + atomicAdd(cursor + cell, 1)] = t;
        }
}

template <typename UVT>
__device__ __forceinline__ void test_pair(int s, int t, const UVT* UV, const int32_t* F, double rel, uint8_t* tflags,
                                          bool& counted) {
    const Tri a = load_tri(UV, F, s), b = load_tri(UV, F, t);
    double alx = a.x[0], ahx = a.x[0], aly = a.y[0], ahy = a.y[0];
    double blx = b.x[0], bhx = b.x[0], bly = b.y[0], bhy = b.y[0];
#pragma unroll
    for (int k = 1; k < 3; ++k) {
        alx = fmin(alx, a.x[k]); ahx = fmax(ahx, a.x[k]); aly = fmin(aly, a.y[k]); ahy = fmax(ahy, a.y[k]);
        blx = fmin(blx, b.x[k]); bhx = fmax(bhx, b.x[k]); bly = fmin(bly, b.y[k]); bhy = fmax(bhy, b.y[k]);
    }
    if (alx > bhx || blx > ahx || aly > bhy || bly > ahy) return;   // real boxes disjoint: no overlap possible
    counted = true;
    const int r = pair_overlap(a, b, rel);
    if (r) {
        const uint8_t bits = static_cast<uint8_t>(((r & 1) ? 16 : 0) | ((r & 2) ? 32 : 0));
        atomicOr(reinterpret_cast<unsigned int*>(tflags + (s & ~3)), static_cast<unsigned int>(bits) << (8 * (s & 3)));
        atomicOr(reinterpret_cast<unsigned int*>(tflags + (t & ~3)), static_cast<unsigned int>(bits) << (8 * (t & 3)));
    }
}

// One thread per (cell, item): pairs with the later items of the cell, each
// pair once (in the first cell both cell boxes share, engine/validate.py:130).
// Only cells of rows [band_lo, band_hi): a shard's band of the atlas.
template <typename UVT>
__global__ void k_pairs_items(const int32_t* nitems, const int32_t* items, const int32_t* item_cell, const int32_t* cofs,
                              const int4* cbox, int G, const UVT* UV, const int32_t* F, double rel, uint8_t* tflags,
                              unsigned long long* counts, int band_lo, int band_hi) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long npairs = 0;
    if (p < *nitems && item_cell[p] / G >= band_lo && item_cell[p] / G < band_hi) {
        const int cell = item_cell[p];
        const int cx = cell % G, cy = cell / G;
        const int end = cofs[cell + 1];
        const int s = items[p];
        const int4 bs = cbox[s];
        for (int q = p + 1; q < end; ++q) {
            const int t = items[q];
            const int4 bt = cbox[t];
            if (max(bs.x, bt.x) != cx || max(bs.z, bt.z) != cy) continue;
            if (bs.x > bt.y || bt.x > bs.y || bs.z > bt.w || bt.z > bs.w) continue;
            bool counted = false;
            test_pair(s, t, UV, F, rel, tflags, counted);
            npairs += counted ? 1 : 0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
    if ((threadIdx.x & 31) == 0 && npairs) atomicAdd(counts + UVA_VC_PAIRS, npairs);
}

// item -> cell map for k_pairs (cells own contiguous item ranges)
__global__ void k_item_cells(int ncells, const int32_t* cofs, int32_t* item_cell) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    for (int p = cofs[c]; p < cofs[c + 1]; ++p) item_cell[p] = c;
}

// Big triangles (more than kMaxCells cells) against every non-skipped
// triangle; big-big pairs once (lower index first). A pair belongs to the
// band holding the row of its first shared cell, as on the binned path.
template <typename UVT>
__global__ void k_pairs_big(int m, const int32_t* big, const int32_t* nbig, const int4* cbox, const uint8_t* skipf,
                            const UVT* UV, const int32_t* F, double rel, uint8_t* tflags, unsigned long long* counts,
                            int band_lo, int band_hi) {
    const int nb = *nbig;
    unsigned long long npairs = 0;
    for (int k = blockIdx.x; k < nb; k += gridDim.x) {
        const int s = big[k];
        const int4 bs = cbox[s];
        for (int t = threadIdx.x; t < m; t += blockDim.x) {
            if (t == s || (skipf[t] & 4)) continue;
            const int4 bt = cbox[t];
            const int ntc = (bt.y - bt.x + 1) * (bt.w - bt.z + 1);
            if (ntc > kMaxCells && t < s) continue;   // big-big: tested from the lower index
            if (bs.x > bt.y || bt.x > bs.y || bs.z > bt.w || bt.z > bs.w) continue;
            const int cy = max(bs.z, bt.z);
            if (cy < band_lo || cy >= band_hi) continue;
            bool counted = false;
            test_pair(s, t, UV, F, rel, tflags, counted);
            npairs += counted ? 1 : 0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
    if ((threadIdx.x & 31) == 0 && npairs) atomicAdd(counts + UVA_VC_PAIRS, npairs);
}

// ------------------------------------------------------------------ final flags and counts
// After the overlap bits of every shard are merged into tflags: the counts
// that depend on them, again (uva_validate_finish).
__global__ void k_recount(int m, const uint8_t* tflags, const int32_t* labels, int32_t* island_ov,
                          unsigned long long* counts) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    bool ov = false, contact = false;
    if (t < m) {
        const uint8_t f = tflags[t];
        ov = f & 16;
        contact = (f & 32) && !ov;
        if (ov) island_ov[labels[t]] = 1;
    }
    count_add(counts + UVA_VC_OVERLAP, ov);
    count_add(counts + UVA_VC_CONTACTS, contact);
}

__global__ void k_zero_counts(unsigned long long* counts) {
    counts[UVA_VC_OVERLAP] = 0;
    counts[UVA_VC_CONTACTS] = 0;
    counts[UVA_VC_ISLANDS_OV] = 0;
}
__global__ void k_final(int m, const double* sa, const int32_t* labels, const int8_t* dom, uint8_t* tflags,
                        int32_t* island_ov, unsigned long long* counts) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    bool fl = false, ov = false, contact = false;
    if (t < m) {
        uint8_t f = tflags[t];
        const double s = sa[t];
        const int d = dom[labels[t]];
        const bool has3d = f & 1, sliver = f & 2;
        // has3d & ~sliver & (sign(sa) != dom) & (sa != 0); NaN compares unequal
        fl = has3d && !sliver && (isnan(s) || (s > 0.0 && d < 0) || (s < 0.0 && d > 0));
        ov = f & 16;
        contact = (f & 32) && !ov;
        if (fl) f |= 8;
        tflags[t] = f;
        if (ov) island_ov[labels[t]] = 1;
    }
    count_add(counts + UVA_VC_FLIPPED, fl);
    count_add(counts + UVA_VC_OVERLAP, ov);
    count_add(counts + UVA_VC_CONTACTS, contact);
}

__global__ void k_count_flags(int nl, const int32_t* flag, unsigned long long* counts, int slot) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    count_add(counts + slot, l < nl && flag[l]);
}

__global__ void k_store_islands(const int32_t* total, unsigned long long* counts) {
    counts[UVA_VC_ISLANDS] = static_cast<unsigned long long>(*total);
}

__global__ void k_store_count(const int32_t* total, int64_t* out) { *out = static_cast<int64_t>(*total); }

__global__ void k_store_pairs_meta(const int32_t* nbig, const int32_t* namb, unsigned long long* counts) {
    counts[UVA_VC_BIG] = static_cast<unsigned long long>(*nbig);
    counts[UVA_VC_AMBIGUOUS] = static_cast<unsigned long long>(*namb);
}

// engine/validate.py:221-226: FP64 normalised chart UVs, skip |sa| <= 1e-14.
__global__ void k_chart_classify(int m, const double* U, const int32_t* F, int G, uint8_t* tflags, int4* cbox) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const Tri r = load_tri(U, F, t);
    const double sa = 0.5 * ((r.x[1] - r.x[0]) * (r.y[2] - r.y[0]) - (r.x[2] - r.x[0]) * (r.y[1] - r.y[0]));
    const bool skip = fabs(sa) <= 1e-14;
    tflags[t] = skip ? 4 : 0;
    if (skip) { cbox[t] = make_int4(1, 0, 1, 0); return; }
    double lx = r.x[0], hx = r.x[0], ly = r.y[0], hy = r.y[0];
#pragma unroll
    for (int k = 1; k < 3; ++k) {
        lx = fmin(lx, r.x[k]); hx = fmax(hx, r.x[k]);
        ly = fmin(ly, r.y[k]); hy = fmax(hy, r.y[k]);
    }
    auto cell = [G](double u) {
        const int c = static_cast<int>(u * static_cast<double>(G));
        return c < 0 ? 0 : (c > G - 1 ? G - 1 : c);
    };
    cbox[t] = make_int4(cell(lx), cell(hx), cell(ly), cell(hy));
}

struct Layout {
    size_t off[32];
    size_t total;
};

// Scratch carve-up (each region 256-byte aligned).
Layout layout(int64_t n, int64_t m, int64_t G) {
    Layout L{};
    const int64_t H = [&] { int64_t h = 1; while (h < 2 * std::max<int64_t>(n, 1)) h <<= 1; return h; }();
    const int64_t ncell = G * G;
    const int64_t nb = std::max<int64_t>(1, (std::max({n, m, ncell + 1}) + kScanB - 1) / kScanB);
    const int64_t sizes[] = {
        8 * m + 8,                 // 0 a3 + amax
        16 * m,                    // 1 cbox (int4)
        4 * H,                     // 2 hash table
        4 * n,                     // 3 rep
        4 * n,                     // 4 parent
        4 * std::max<int64_t>(n, 1),   // 5 root flags
        4 * std::max<int64_t>(n, 1),   // 6 root rank
        4 * m,                     // 7 face root
        8 * (m + 1),               // 8 pos
        8 * (m + 1),               // 9 neg
        4 * (m + 1),               // 10 count per island
        m + 1,                     // 11 dom (int8)
        4 * (m + 1),               // 12 ambiguous list
        4 * (ncell + 1),           // 13 cell counts
        4 * (ncell + 1),           // 14 cell offsets
        4 * ncell,                 // 15 cursor
        4 * kMaxCells * m,         // 16 items
        4 * kMaxCells * m,         // 17 item -> cell
        4 * m,                     // 18 big list
        4 * (m + 1),               // 19 island overlap flag
        4 * nb,                    // 20 scan block sums
        64,                        // 21 small ints (totals, counters)
    };
    size_t o = 0;
    for (int i = 0; i < 22; ++i) {
        L.off[i] = o;
        o += (static_cast<size_t>(sizes[i]) + 255) & ~static_cast<size_t>(255);
    }
    L.total = o;
    return L;
}

int auto_grid(int m, int grid) {
    if (grid > 0) return std::min(grid, 8192);
    int g = static_cast<int>(sqrt(static_cast<double>(m)) / 2.0);
    return std::max(64, std::min(g, 4096));
}

}  // namespace

extern "C" int uva_validate_scratch_bytes(int64_t n, int64_t m, int32_t grid, int64_t* bytes) {
    if (n < 0 || m < 0 || !bytes) { uva_set_error("uva_validate_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    if (m * kMaxCells > (int64_t(1) << 31) - 1) { uva_set_error("uva_validate: too many triangles"); return UVA_E_TOOBIG; }
    *bytes = static_cast<int64_t>(layout(n, m, auto_grid(static_cast<int>(m), grid)).total);
    return UVA_OK;
}

extern "C" int uva_validate(const uva_val_desc* d, void* stream) {
    if (!d || d->n < 0 || d->m < 0 || !d->counts || (d->m > 0 && (!d->F || !d->UV || !d->V || !d->tflags ||
                                                                      !d->labels || !d->sa || !d->scratch))) {
        uva_set_error("uva_validate: bad arguments");
        return UVA_E_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = d->n, m = d->m;
    const int G = auto_grid(m, d->grid);
    const Layout L = layout(n, m, G);
    if (d->scratch_bytes < static_cast<int64_t>(L.total)) { uva_set_error("uva_validate: scratch too small"); return UVA_E_ARG; }
    auto* base = static_cast<unsigned char*>(d->scratch);
    auto R = [&](int i) { return base + L.off[i]; };
    double* a3 = reinterpret_cast<double*>(R(0));
    double* amax = a3 + m;
    int4* cbox = reinterpret_cast<int4*>(R(1));
    int32_t* table = reinterpret_cast<int32_t*>(R(2));
    int32_t* rep = reinterpret_cast<int32_t*>(R(3));
    int32_t* parent = reinterpret_cast<int32_t*>(R(4));
    int32_t* rflag = reinterpret_cast<int32_t*>(R(5));
    int32_t* rrank = reinterpret_cast<int32_t*>(R(6));
    int32_t* froot = reinterpret_cast<int32_t*>(R(7));
    double* pos = reinterpret_cast<double*>(R(8));
    double* neg = reinterpret_cast<double*>(R(9));
    int32_t* icnt = reinterpret_cast<int32_t*>(R(10));
    int8_t* dom = reinterpret_cast<int8_t*>(R(11));
    int32_t* amb = reinterpret_cast<int32_t*>(R(12));
    int32_t* ccount = reinterpret_cast<int32_t*>(R(13));
    int32_t* cofs = reinterpret_cast<int32_t*>(R(14));
    int32_t* cursor = reinterpret_cast<int32_t*>(R(15));
    int32_t* items = reinterpret_cast<int32_t*>(R(16));
    int32_t* item_cell = reinterpret_cast<int32_t*>(R(17));
    int32_t* big = reinterpret_cast<int32_t*>(R(18));
    int32_t* isl_ov = reinterpret_cast<int32_t*>(R(19));
    int32_t* sums = reinterpret_cast<int32_t*>(R(20));
    int32_t* smalls = reinterpret_cast<int32_t*>(R(21));
    int32_t* n_isl = smalls;        // number of islands
    int32_t* nbig = smalls + 1;
    int32_t* namb = smalls + 2;
    int32_t* nitems = smalls + 3;
    unsigned long long* counts = reinterpret_cast<unsigned long long*>(d->counts);
    const int64_t H = (L.off[3] - L.off[2]) / 4;
    uint32_t hmask = 1;
    while (static_cast<int64_t>(hmask) * 2 <= H) hmask <<= 1;
    hmask -= 1;
    const int ncell = G * G;
    cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * UVA_VC_N, s);
    cudaMemsetAsync(smalls, 0, 64, s);
    auto blocks = [](int x) { return std::max(1, (x + 255) / 256); };
    k_v_rows<<<blocks(n), 256, 0, s>>>(n, d->UV, counts);
    if (m == 0) { UVA_CHECK_LAUNCH("uva_validate"); return UVA_OK; }
    cudaMemsetAsync(amax, 0, sizeof(double), s);
    k_v_area3<<<blocks(m), 256, 0, s>>>(m, d->V, d->F, a3, amax);
    k_v_classify<<<blocks(m), 256, 0, s>>>(m, d->UV, d->F, a3, amax, G, d->sa, d->tflags, cbox, counts);
    UVA_CHECK_LAUNCH("uva_validate/classify");
    // islands
    cudaMemsetAsync(table, 0xff, static_cast<size_t>(hmask + 1) * 4, s);
    k_weld<<<blocks(n), 256, 0, s>>>(n, d->V, d->UV, table, hmask, rep);
    k_uf_init<<<blocks(n), 256, 0, s>>>(n, rep, parent);
    k_uf_faces<<<blocks(m), 256, 0, s>>>(m, d->F, rep, parent);
    cudaMemsetAsync(rflag, 0, 4 * static_cast<size_t>(std::max(n, 1)), s);
    k_uf_roots<<<blocks(m), 256, 0, s>>>(m, d->F, rep, parent, froot, rflag);
    scan(rflag, rrank, sums, n_isl, n, s);
    k_labels<<<blocks(m), 256, 0, s>>>(m, froot, rrank, d->labels);
    k_store_islands<<<1, 1, 0, s>>>(n_isl, counts);
    UVA_CHECK_LAUNCH("uva_validate/islands");
    // orientation per island (labels < number of islands <= m)
    cudaMemsetAsync(pos, 0, 8 * static_cast<size_t>(m + 1), s);
    cudaMemsetAsync(neg, 0, 8 * static_cast<size_t>(m + 1), s);
    cudaMemsetAsync(icnt, 0, 4 * static_cast<size_t>(m + 1), s);
    k_orient_sums<<<blocks(m), 256, 0, s>>>(m, d->sa, d->labels, pos, neg, icnt);
    k_orient_decide<<<blocks(m), 256, 0, s>>>(n_isl, pos, neg, icnt, dom, amb, namb);
    k_orient_exact<<<4, 256, 0, s>>>(m, d->sa, d->labels, amb, namb, dom);
    UVA_CHECK_LAUNCH("uva_validate/orientation");
    // binned overlap pairs
    cudaMemsetAsync(ccount, 0, 4 * static_cast<size_t>(ncell + 1), s);
    cudaMemsetAsync(cursor, 0, 4 * static_cast<size_t>(ncell), s);
    k_bin_count<<<blocks(m), 256, 0, s>>>(m, cbox, G, ccount, big, nbig);
    scan(ccount, cofs, sums, nitems, ncell + 1, s);
    k_bin_fill<<<blocks(m), 256, 0, s>>>(m, cbox, G, cofs, cursor, items);
    k_item_cells<<<blocks(ncell), 256, 0, s>>>(ncell, cofs, item_cell);
    UVA_CHECK_LAUNCH("uva_validate/binning");
    // the number of items is bounded by kMaxCells * m; threads beyond the
    // actual count read cofs[ncell] as the end and do nothing
    const int nsh = std::max(1, d->nshards), sh = nsh > 1 ? d->shard : 0;
    const int band_lo = static_cast<int>(static_cast<int64_t>(G) * sh / nsh);
    const int band_hi = static_cast<int>(static_cast<int64_t>(G) * (sh + 1) / nsh);
    k_pairs_items<float><<<blocks(kMaxCells * m), 256, 0, s>>>(nitems, items, item_cell, cofs, cbox, G, d->UV, d->F,
                                                                d->rel, d->tflags, counts, band_lo, band_hi);
    k_pairs_big<float><<<148, 256, 0, s>>>(m, big, nbig, cbox, d->tflags, d->UV, d->F, d->rel, d->tflags, counts,
                                           band_lo, band_hi);
    UVA_CHECK_LAUNCH("uva_validate/pairs");
    cudaMemsetAsync(isl_ov, 0, 4 * static_cast<size_t>(m + 1), s);
    k_final<<<blocks(m), 256, 0, s>>>(m, d->sa, d->labels, dom, d->tflags, isl_ov, counts);
    k_mirrored<<<blocks(m), 256, 0, s>>>(m, n_isl, dom, counts);
    k_count_flags<<<blocks(m), 256, 0, s>>>(m, isl_ov, counts, UVA_VC_ISLANDS_OV);
    k_store_pairs_meta<<<1, 1, 0, s>>>(nbig, namb, counts);
    UVA_CHECK_LAUNCH("uva_validate/final");
    return UVA_OK;
}

extern "C" int uva_validate_finish(const uva_val_desc* d, void* stream) {
    if (!d || d->n < 0 || d->m < 0 || !d->counts || (d->m > 0 && (!d->tflags || !d->labels || !d->scratch))) {
        uva_set_error("uva_validate_finish: bad arguments");
        return UVA_E_ARG;
    }
    if (d->m == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int m = d->m;
    const Layout L = layout(d->n, m, auto_grid(m, d->grid));
    if (d->scratch_bytes < static_cast<int64_t>(L.total)) {
        uva_set_error("uva_validate_finish: scratch too small");
        return UVA_E_ARG;
    }
    int32_t* isl_ov = reinterpret_cast<int32_t*>(static_cast<unsigned char*>(d->scratch) + L.off[19]);
    unsigned long long* counts = reinterpret_cast<unsigned long long*>(d->counts);
    auto blocks = [](int x) { return std::max(1, (x + 255) / 256); };
    cudaMemsetAsync(isl_ov, 0, 4 * static_cast<size_t>(m + 1), s);
    k_zero_counts<<<1, 1, 0, s>>>(counts);
    k_recount<<<blocks(m), 256, 0, s>>>(m, d->tflags, d->labels, isl_ov, counts);
    k_count_flags<<<blocks(m), 256, 0, s>>>(m, isl_ov, counts, UVA_VC_ISLANDS_OV);
    UVA_CHECK_LAUNCH("uva_validate_finish");
    return UVA_OK;
}

extern "C" int uva_chart_overlaps(const double* U, const int32_t* F, int32_t n, int32_t m, uint8_t* tflags,
                                  void* scratch, int64_t scratch_bytes, void* stream) {
    if (n < 0 || m < 0 || (m > 0 && (!U || !F || !tflags || !scratch))) {
        uva_set_error("uva_chart_overlaps: bad arguments");
        return UVA_E_ARG;
    }
    if (m == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // grid of engine/validate.py:225 is clip(sqrt(t)/2, 4, 2048); any grid gives
    // the same flags, the validation grid is reused for the scratch layout
    const int G = auto_grid(m, 0);
    const Layout L = layout(n, m, G);
    if (scratch_bytes < static_cast<int64_t>(L.total)) { uva_set_error("uva_chart_overlaps: scratch too small"); return UVA_E_ARG; }
    auto* base = static_cast<unsigned char*>(scratch);
    auto R = [&](int i) { return base + L.off[i]; };
    int4* cbox = reinterpret_cast<int4*>(R(1));
    int32_t* ccount = reinterpret_cast<int32_t*>(R(13));
    int32_t* cofs = reinterpret_cast<int32_t*>(R(14));
    int32_t* cursor = reinterpret_cast<int32_t*>(R(15));
    int32_t* items = reinterpret_cast<int32_t*>(R(16));
    int32_t* item_cell = reinterpret_cast<int32_t*>(R(17));
    int32_t* big = reinterpret_cast<int32_t*>(R(18));
    int32_t* sums = reinterpret_cast<int32_t*>(R(20));
    int32_t* smalls = reinterpret_cast<int32_t*>(R(21));
    unsigned long long* counts = reinterpret_cast<unsigned long long*>(smalls + 8);
    const int ncell = G * G;
    auto blocks = [](int x) { return std::max(1, (x + 255) / 256); };
    cudaMemsetAsync(smalls, 0, 64, s);
    cudaMemsetAsync(ccount, 0, 4 * static_cast<size_t>(ncell + 1), s);
    cudaMemsetAsync(cursor, 0, 4 * static_cast<size_t>(ncell), s);
    k_chart_classify<<<blocks(m), 256, 0, s>>>(m, U, F, G, tflags, cbox);
    k_bin_count<<<blocks(m), 256, 0, s>>>(m, cbox, G, ccount, big, smalls + 1);
    scan(ccount, cofs, sums, smalls + 3, ncell + 1, s);
    k_bin_fill<<<blocks(m), 256, 0, s>>>(m, cbox, G, cofs, cursor, items);
    k_item_cells<<<blocks(ncell), 256, 0, s>>>(ncell, cofs, item_cell);
    k_pairs_items<double><<<blocks(kMaxCells * m), 256, 0, s>>>(smalls + 3, items, item_cell, cofs, cbox, G, U, F, 1e-6,
                                                                 tflags, counts, 0, G);
    k_pairs_big<double><<<148, 256, 0, s>>>(m, big, smalls + 1, cbox, tflags, U, F, 1e-6, tflags, counts, 0, G);
    UVA_CHECK_LAUNCH("uva_chart_overlaps");
    return UVA_OK;
}

// engine/metrics.py:91-103: islands of faces connected through shared
// vertices; with weld != 0, vertices with identical float32 (position, uv)
// bytes are one vertex. labels: 0..count-1 ordered by the smallest
// (representative) vertex id of each island.
extern "C" int uva_islands(const double* V, const float* UV, const int32_t* F, int32_t n, int32_t m, int32_t weld,
                           int32_t* labels, int64_t* count, void* scratch, int64_t scratch_bytes, void* stream) {
    if (n < 0 || m < 0 || !count || (m > 0 && (!F || !labels || !scratch)) || (weld && n > 0 && (!V || !UV))) {
        uva_set_error("uva_islands: bad arguments");
        return UVA_E_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Layout L = layout(n, m, auto_grid(m, 0));
    if (scratch_bytes < static_cast<int64_t>(L.total)) { uva_set_error("uva_islands: scratch too small"); return UVA_E_ARG; }
    auto* base = static_cast<unsigned char*>(scratch);
    auto R = [&](int i) { return base + L.off[i]; };
    int32_t* table = reinterpret_cast<int32_t*>(R(2));
    int32_t* rep = reinterpret_cast<int32_t*>(R(3));
    int32_t* parent = reinterpret_cast<int32_t*>(R(4));
    int32_t* rflag = reinterpret_cast<int32_t*>(R(5));
    int32_t* rrank = reinterpret_cast<int32_t*>(R(6));
    int32_t* froot = reinterpret_cast<int32_t*>(R(7));
    int32_t* sums = reinterpret_cast<int32_t*>(R(20));
    int32_t* smalls = reinterpret_cast<int32_t*>(R(21));
    auto blocks = [](int x) { return std::max(1, (x + 255) / 256); };
    cudaMemsetAsync(smalls, 0, 64, s);
    cudaMemsetAsync(count, 0, 8, s);
    if (m == 0 || n == 0) return UVA_OK;
    if (weld) {
        const int64_t H = (L.off[3] - L.off[2]) / 4;
        uint32_t hmask = 1;
        while (static_cast<int64_t>(hmask) * 2 <= H) hmask <<= 1;
        hmask -= 1;
        cudaMemsetAsync(table, 0xff, static_cast<size_t>(hmask + 1) * 4, s);
        k_weld<<<blocks(n), 256, 0, s>>>(n, V, UV, table, hmask, rep);
    } else {
        k_identity<<<blocks(n), 256, 0, s>>>(n, rep);
    }
    k_uf_init<<<blocks(n), 256, 0, s>>>(n, rep, parent);
    k_uf_faces<<<blocks(m), 256, 0, s>>>(m, F, rep, parent);
    cudaMemsetAsync(rflag, 0, 4 * static_cast<size_t>(n), s);
    k_uf_roots<<<blocks(m), 256, 0, s>>>(m, F, rep, parent, froot, rflag);
    scan(rflag, rrank, sums, smalls, n, s);
    k_labels<<<blocks(m), 256, 0, s>>>(m, froot, rrank, labels);
    k_store_count<<<1, 1, 0, s>>>(smalls, count);
    UVA_CHECK_LAUNCH("uva_islands");
    return UVA_OK;
}
