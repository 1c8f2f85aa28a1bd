// UV distortion metrics (engine/metrics.py:106-210) and per-chart quality
// (engine/param.py:520-551) on the device.
//
//  * k_tri_jacobians: closed-form 2x2 singular values of the 3D->UV Jacobian
//    (metrics.py:115-145), signed UV area, 3D area, angle error (:213-223).
//  * reductions: FP64 sums (warp-reduced, then atomics) of the report terms.
//  * weighted quantiles (metrics.py:107-112, param.py:543-546): a segmented
//    weighted radix select over the FP64 bit patterns, 8 bits per pass,
//    returning the smallest value whose cumulative weight reaches q * total
//    (numpy: argsort, cumsum, searchsorted). One segment for the whole mesh,
//    or one per island for batched chart quality.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"

using namespace uva;

namespace {

// ------------------------------------------------------------------ per triangle
struct TriJ {
    double s1, s2, sa, a3, ang;
    bool good;
};

__device__ __forceinline__ double angle(double ux, double uy, double uz, double vx, double vy, double vz) {
    const double nu = sqrt(ux * ux + uy * uy + uz * uz), nv = sqrt(vx * vx + vy * vy + vz * vz);
    double c = (ux * vx + uy * vy + uz * vz) / fmax(nu * nv, 1e-300);
    c = fmin(fmax(c, -1.0), 1.0);
    return acos(c);
}

// engine/metrics.py:115-145 and :213-223 for one triangle.
__device__ TriJ tri_jacobian(const double* P, const double* U) {
    const double e1x = P[3] - P[0], e1y = P[4] - P[1], e1z = P[5] - P[2];
    const double e2x = P[6] - P[0], e2y = P[7] - P[1], e2z = P[8] - P[2];
    const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    TriJ r;
    r.a3 = 0.5 * sqrt(nx * nx + ny * ny + nz * nz);
    const double l1 = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
    const double il = 1.0 / fmax(l1, 1e-30);
    const double exx = e1x * il, exy = e1y * il, exz = e1z * il;
    const double in = 1.0 / fmax(2.0 * r.a3, 1e-30);
    const double ux = nx * in, uy = ny * in, uz = nz * in;
    const double eyx = uy * exz - uz * exy, eyy = uz * exx - ux * exz, eyz = ux * exy - uy * exx;
    const double x1 = l1, x2 = e2x * exx + e2y * exy + e2z * exz, y2 = e2x * eyx + e2y * eyy + e2z * eyz;
    const double d1x = U[2] - U[0], d1y = U[3] - U[1], d2x = U[4] - U[0], d2y = U[5] - U[1];
    const double det = x1 * y2;
    r.good = fabs(det) > 1e-30;
    const double inv = r.good ? 1.0 / det : 0.0;
    const double a = d1x * (y2 * inv), c = d1y * (y2 * inv);
    const double b = d1x * (-x2 * inv) + d2x * (x1 * inv), d = d1y * (-x2 * inv) + d2y * (x1 * inv);
    r.sa = 0.5 * (d1x * d2y - d1y * d2x);
    const double E = (a + d) / 2, F = (a - d) / 2, G = (c + b) / 2, H = (c - b) / 2;
    const double Q = sqrt(E * E + H * H), R = sqrt(F * F + G * G);
    r.s1 = Q + R;
    r.s2 = fabs(Q - R);
    // angle error: 3D corner angles vs UV corner angles, mean |diff| in degrees
    const double A0 = angle(e1x, e1y, e1z, e2x, e2y, e2z);
    const double A1 = angle(-e1x, -e1y, -e1z, P[6] - P[3], P[7] - P[4], P[8] - P[5]);
    const double A2 = angle(-e2x, -e2y, -e2z, -(P[6] - P[3]), -(P[7] - P[4]), -(P[8] - P[5]));
    const double B0 = angle(d1x, d1y, 0.0, d2x, d2y, 0.0);
    const double B1 = angle(-d1x, -d1y, 0.0, U[4] - U[2], U[5] - U[3], 0.0);
    const double B2 = angle(-d2x, -d2y, 0.0, -(U[4] - U[2]), -(U[5] - U[3]), 0.0);
    r.ang = (fabs(A0 - B0) + fabs(A1 - B1) + fabs(A2 - B2)) / 3.0 * (180.0 / 3.141592653589793);
    return r;
}

__device__ __forceinline__ void load_corners(const double* V, const double* UV, const int32_t* F, int t, double* P,
                                             double* U) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int v = F[3 * t + k];
        P[3 * k] = V[3 * v]; P[3 * k + 1] = V[3 * v + 1]; P[3 * k + 2] = V[3 * v + 2];
        U[2 * k] = UV[2 * v]; U[2 * k + 1] = UV[2 * v + 1];
    }
}

template <int K>
__device__ __forceinline__ void warp_atomic_sums(double* dst, double (&v)[K]) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (v[k] != 0.0) atomicAdd(dst + k, v[k]);
    }
}

// Pass A: per-triangle values; global sums of a3 and |sa|; per-island a3,
// |sa|, positive / negative 3D area (metrics.py:160-200).
__global__ void k_met_a(int m, const double* V, const double* UV, const int32_t* F, const int32_t* isl, double* tri,
                        double* sums, double* isum) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (t < m) {
        double P[9], U[6];
        load_corners(V, UV, F, t, P, U);
        const TriJ r = tri_jacobian(P, U);
        double* o = tri + 6 * static_cast<size_t>(t);
        o[0] = r.s1; o[1] = r.s2; o[2] = r.sa; o[3] = r.a3; o[4] = r.good ? 1.0 : 0.0; o[5] = r.ang;
        v[0] = r.a3;
        v[1] = fabs(r.sa);
        if (isl) {
            double* s = isum + 4 * static_cast<size_t>(isl[t]);
            atomicAdd(s, r.a3);
            atomicAdd(s + 1, fabs(r.sa));
            if (r.sa > 0.0) atomicAdd(s + 2, r.a3);
            if (r.sa < 0.0) atomicAdd(s + 3, r.a3);
        }
    }
    warp_atomic_sums<2>(sums, v);
}

// Quantile inputs: value (excluded: +inf) and weight (excluded: 0).
struct QIn {
    double* x;
    double* w;
};

// Pass B (metrics.py:160-205): report sums and the quantile inputs.
// sums layout: 0 sum a3, 1 sum |sa|, 2.. see UVA_MET_* in the host code.
__global__ void k_met_b(int m, const double* tri, const int32_t* isl, const double* isum, double* sums, QIn qa, QIn qg,
                        QIn qc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double v[14] = {0};
    if (t < m) {
        const double* o = tri + 6 * static_cast<size_t>(t);
        const double s1 = o[0], s2 = o[1], sa = o[2], a3 = o[3], ang = o[5];
        const bool good = o[4] != 0.0;
        const double A3 = sums[0], UVA = sums[1];
        const double w = a3 / fmax(A3, 1e-30);
        const double uv_abs = fabs(sa);
        const double scale2 = UVA / fmax(A3, 1e-30);
        const bool valid = good && a3 > 0.0;
        const bool collapsed = valid && uv_abs < 1e-2 * (1.0 / (8192.0 * 8192.0));
        const double aniso = s2 > 0.0 ? s1 / fmax(s2, 1e-300) : INFINITY;
        const bool an_ok = valid && isfinite(aniso) && !collapsed;
        const double ar_g = valid ? (s1 * s2) / fmax(scale2, 1e-300) : 1.0;
        const double lg = fabs(log2(fmax(ar_g, 1e-30)));
        const bool ok = valid && !collapsed;
        const double st = sqrt((s1 * s1 + s2 * s2) / 2.0) / sqrt(fmax(scale2, 1e-300));
        v[0] = collapsed ? 1.0 : 0.0;
        v[1] = collapsed ? w : 0.0;
        v[2] = an_ok ? aniso * w : 0.0;
        v[3] = an_ok ? w : 0.0;
        v[4] = valid ? ang * w : 0.0;
        v[5] = valid ? w : 0.0;
        v[6] = ok ? lg * w : 0.0;
        v[7] = ok ? w : 0.0;
        v[8] = ok ? st * st * w : 0.0;
        qa.x[t] = an_ok ? aniso : INFINITY; qa.w[t] = an_ok ? w : 0.0;
        qg.x[t] = ok ? lg : INFINITY; qg.w[t] = ok ? w : 0.0;
        if (isl) {
            const double* s = isum + 4 * static_cast<size_t>(isl[t]);
            const double isc = s[1] / fmax(s[0], 1e-30);
            const double ar_c = valid ? (s1 * s2) / fmax(isc, 1e-300) : 1.0;
            const double lc = fabs(log2(fmax(ar_c, 1e-30)));
            const double dom = s[2] >= s[3] ? 1.0 : -1.0;
            const double sg = sa > 0.0 ? 1.0 : (sa < 0.0 ? -1.0 : (sa == 0.0 ? 0.0 : NAN));
            const bool flipped = valid && !collapsed && !(sg == dom);
            v[9] = ok ? lc * w : 0.0;
            v[10] = flipped ? 1.0 : 0.0;
            v[11] = flipped ? w : 0.0;
            qc.x[t] = ok ? lc : INFINITY; qc.w[t] = ok ? w : 0.0;
        }
    }
    warp_atomic_sums<14>(sums + 2, v);
}

// Per-island inputs of island_density_ratio_p95 and the mirrored count.
__global__ void k_met_islands(int ni, const double* isum, double* sums, QIn qd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < ni) {
        const double* s = isum + 4 * static_cast<size_t>(i);
        const double scale2 = sums[1] / fmax(sums[0], 1e-30);
        const double isc = s[1] / fmax(s[0], 1e-30);
        const double d = sqrt(isc / fmax(scale2, 1e-300));
        qd.x[i] = fabs(log2(fmax(d, 1e-30)));
        qd.w[i] = s[0];   // ia3 (normalisation does not move the quantile)
        v[0] = s[2] >= s[3] ? 0.0 : 1.0;
        v[1] = s[0];
    }
    warp_atomic_sums<2>(sums + 16, v);
}

// ------------------------------------------------------------------ chart quality
// Per-key sums of K values over a warp whose lanes hold their keys in
// contiguous runs (key -1: none): a segmented reduction, then the first lane
// of each run adds the run's sums at dst + stride * key. Batch triangles are
// grouped by island, so an island takes one atomic per value and warp.
template <int K>
__device__ __forceinline__ void warp_run_sums(double* dst, int stride, int key, double (&v)[K]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int yk = __shfl_down_sync(0xffffffffu, key, o);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double y = __shfl_down_sync(0xffffffffu, v[k], o);
            if (lane + o < 32 && yk == key) v[k] += y;
        }
    }
    const int prev = __shfl_up_sync(0xffffffffu, key, 1);
    if (key >= 0 && (lane == 0 || prev != key)) {
        double* d = dst + static_cast<size_t>(stride) * key;
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (v[k] != 0.0) atomicAdd(d + k, v[k]);
    }
}

// engine/param.py:520-551 for every island of a batch (frames from the setup).
__global__ void k_quality_a(const uva_batch b, double* tri, double* isum) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    int key = -1;
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (f < b.t) {
        const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
        const int v0 = b.vofs[tv.w];
        const double4 fr = reinterpret_cast<const double4*>(b.frame)[f];
        const double2* U = reinterpret_cast<const double2*>(b.U);
        const double2 a0 = U[v0 + tv.x], a1 = U[v0 + tv.y], a2 = U[v0 + tv.z];
        const bool ok = fabs(fr.x * fr.z) > 1e-300;
        const double x1s = ok ? fr.x : 1.0, y2s = ok ? fr.z : 1.0;
        const double j00 = (a1.x - a0.x) / x1s, j10 = (a1.y - a0.y) / x1s;
        const double j01 = ((a2.x - a0.x) - j00 * fr.y) / y2s, j11 = ((a2.y - a0.y) - j10 * fr.y) / y2s;
        const double E = (j00 + j11) / 2, F = (j00 - j11) / 2, G = (j10 + j01) / 2, H = (j10 - j01) / 2;
        const double Q = sqrt(E * E + H * H), R = sqrt(F * F + G * G);
        const double s1 = Q + R, s2 = fabs(Q - R);
        const double sa = 0.5 * ((a1.x - a0.x) * (a2.y - a0.y) - (a2.x - a0.x) * (a1.y - a0.y));
        double* o = tri + 6 * static_cast<size_t>(f);
        o[0] = s1; o[1] = s2; o[2] = sa; o[3] = fr.w;
        key = tv.w;
        v[0] = fr.w;                      // A
        v[1] = fabs(sa);                  // uvA
        v[2] = sa > 0.0 ? 1.0 : 0.0;      // positive count
        v[3] = sa < 0.0 ? 1.0 : 0.0;      // negative count
        v[4] = sa <= 0.0 ? 1.0 : 0.0;     // non-positive count
        v[5] = sa >= 0.0 ? 1.0 : 0.0;     // non-negative count
    }
    warp_run_sums<6>(isum, 8, key, v);
}

__global__ void k_quality_b(const uva_batch b, const double* tri, double* isum, QIn qa, QIn qr, double* per_aniso,
                            double* per_area, double* stretch) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t) return;
    const int isl = reinterpret_cast<const int4*>(b.tri4)[f].w;
    const double* o = tri + 6 * static_cast<size_t>(f);
    double* s = isum + 8 * static_cast<size_t>(isl);
    const double A = s[0];
    const double sc = s[1] / fmax(A, 1e-300);
    const double w = o[3] / fmax(A, 1e-300);
    const double s1 = o[0], s2 = o[1];
    const double an = s1 / fmax(s2, 1e-12);
    const double ar = (s1 * s2) / fmax(sc, 1e-300);
    const double lar = fabs(log2(fmax(ar, 1e-12)));
    const double st2 = (s1 * s1 + s2 * s2) / 2.0 / fmax(sc, 1e-300);
    per_aniso[f] = an;
    per_area[f] = ar;
    qa.x[f] = an; qa.w[f] = w;
    qr.x[f] = lar; qr.w[f] = w;
    atomicAdd(s + 6, an * w);
    atomicAdd(s + 7, lar * w);
    atomicAdd(stretch + isl, st2 * w);
}

// Per island: flips, aniso_p95, aniso_mean, area_p95, area_logdev, stretch, scale, A.
__global__ void k_quality_out(int nc, const double* isum, const double* stretch, const double* q95a, const double* q95r,
                              double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const double* s = isum + 8 * static_cast<size_t>(i);
    double* o = out + 8 * static_cast<size_t>(i);
    o[0] = s[2] >= s[3] ? s[4] : s[5];
    o[1] = q95a[i];
    o[2] = s[6];
    o[3] = exp2(q95r[i]);
    o[4] = s[7];
    o[5] = sqrt(stretch[i]);
    o[6] = sqrt(s[1] / fmax(s[0], 1e-300));
    o[7] = s[0];
}

// ------------------------------------------------------------------ weighted quantile
// Order-preserving map of an FP64 value to uint64.
__device__ __forceinline__ unsigned long long okey(double x) {
    const unsigned long long u = static_cast<unsigned long long>(__double_as_longlong(x));
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

struct QState {
    unsigned long long prefix;   // fixed high bits so far
    double below;                // weight of elements with key < prefix range
    double target;               // q * total
    double total;
    int shift;                   // bits still free below the current digit
    int done;
};

// Totals per segment.
__global__ void k_q_total(int n, const double* w, const int32_t* seg, int sstride, double* total) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = w[i];
    if (x != 0.0) atomicAdd(total + (seg ? seg[static_cast<size_t>(i) * sstride] : 0), x);
}

__global__ void k_q_init(int ns, const double* total, double q, QState* st) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    QState z;
    z.prefix = 0; z.below = 0.0; z.total = total[s]; z.target = q * total[s]; z.shift = 64; z.done = 0;
    st[s] = z;
}

// Histogram of the next 8-bit digit among elements matching the prefix.
__global__ void k_q_hist(int n, const double* x, const double* w, const int32_t* seg, int sstride, const QState* st,
                         double* hist) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double wi = w[i];
    if (wi == 0.0) return;
    const int s = seg ? seg[static_cast<size_t>(i) * sstride] : 0;
    const QState q = st[s];
    if (q.done || q.shift <= 0) return;
    const unsigned long long k = okey(x[i]);
    const int hi = q.shift;   // bits [hi-8, hi) form the digit; bits >= hi must equal the prefix
    if (hi < 64 && (k >> hi) != (q.prefix >> hi)) return;
    const int digit = static_cast<int>((k >> (hi - 8)) & 0xff);
    atomicAdd(hist + 256 * static_cast<size_t>(s) + digit, wi);
}

// Pick the digit whose cumulative weight reaches the target: the first
// bucket with below + cumsum >= target; if rounding leaves the target above
// the total, the last non-empty bucket (numpy clamps to the last element).
__global__ void k_q_pick(int ns, QState* st, double* hist) {
    const int s = blockIdx.x;
    if (s >= ns) return;
    __shared__ double h[256];
    double* hs = hist + 256 * static_cast<size_t>(s);
    h[threadIdx.x] = hs[threadIdx.x];
    hs[threadIdx.x] = 0.0;   // ready for the next pass
    __syncthreads();
    if (threadIdx.x != 0) return;
    QState q = st[s];
    if (q.done || q.shift <= 0) return;
    double c = q.below, clast = q.below;
    int d = -1, last = -1;
    for (int k = 0; k < 256; ++k) {
        if (h[k] == 0.0) continue;
        if (c + h[k] >= q.target) { d = k; break; }
        clast = c;
        c += h[k];
        last = k;
    }
    if (d < 0) {
        if (last < 0) { q.done = 1; st[s] = q; return; }
        d = last;
        c = clast;
    }
    q.below = c;
    q.prefix |= static_cast<unsigned long long>(d) << (q.shift - 8);
    q.shift -= 8;
    if (q.shift == 0) q.done = 1;
    st[s] = q;
}

__global__ void k_q_value(int ns, const QState* st, double* out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const QState q = st[s];
    unsigned long long k = q.prefix;
    // invert okey
    const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    out[s] = q.total > 0.0 ? __longlong_as_double(static_cast<long long>(u)) : NAN;
}

size_t al(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Segmented weighted quantile of x with weights w (q in [0,1]); out[ns].
// scratch: ns*(256*8 + sizeof(QState) + 8) bytes.
int wquantile(int n, const double* x, const double* w, const int32_t* seg, int sstride, int ns, double q, double* out,
              unsigned char* scratch, cudaStream_t s) {
    double* hist = reinterpret_cast<double*>(scratch);
    QState* st = reinterpret_cast<QState*>(scratch + al(sizeof(double) * 256 * ns));
    double* total = reinterpret_cast<double*>(scratch + al(sizeof(double) * 256 * ns) + al(sizeof(QState) * ns));
    cudaMemsetAsync(hist, 0, sizeof(double) * 256 * ns, s);
    cudaMemsetAsync(total, 0, sizeof(double) * ns, s);
    const int tb = 256;
    const int gb = std::max(1, (n + tb - 1) / tb);
    if (n > 0) k_q_total<<<gb, tb, 0, s>>>(n, w, seg, sstride, total);
    k_q_init<<<(ns + tb - 1) / tb, tb, 0, s>>>(ns, total, q, st);
    for (int pass = 0; pass < 8; ++pass) {
        if (n > 0) k_q_hist<<<gb, tb, 0, s>>>(n, x, w, seg, sstride, st, hist);
        k_q_pick<<<ns, 256, 0, s>>>(ns, st, hist);
    }
    k_q_value<<<(ns + tb - 1) / tb, tb, 0, s>>>(ns, st, out);
    UVA_CHECK_LAUNCH("uva_wquantile");
    return UVA_OK;
}

size_t wq_bytes(int ns) { return al(sizeof(double) * 256 * ns) + al(sizeof(QState) * ns) + al(sizeof(double) * ns); }

}  // namespace

extern "C" int uva_wquantile_scratch_bytes(int32_t nseg, int64_t* bytes) {
    if (nseg < 1 || !bytes) { uva_set_error("uva_wquantile_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    *bytes = static_cast<int64_t>(wq_bytes(nseg));
    return UVA_OK;
}

extern "C" int uva_wquantile(const double* x, const double* w, const int32_t* seg, int32_t n, int32_t nseg, double q,
                             double* out, void* scratch, int64_t scratch_bytes, void* stream) {
    if (n < 0 || nseg < 1 || !out || !scratch || (n > 0 && (!x || !w))) { uva_set_error("uva_wquantile: bad arguments"); return UVA_E_ARG; }
    if (scratch_bytes < static_cast<int64_t>(wq_bytes(nseg))) { uva_set_error("uva_wquantile: scratch too small"); return UVA_E_ARG; }
    return wquantile(n, x, w, seg, 1, nseg, q, out, static_cast<unsigned char*>(scratch), static_cast<cudaStream_t>(stream));
}

extern "C" int uva_metrics_scratch_bytes(int64_t m, int64_t n_islands, int64_t* bytes) {
    if (m < 0 || n_islands < 0 || !bytes) { uva_set_error("uva_metrics_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    const int64_t ni = std::max<int64_t>(n_islands, 1);
    *bytes = static_cast<int64_t>(al(48 * std::max<int64_t>(m, 1)) + al(32 * ni) + 6 * al(8 * std::max<int64_t>(m, 1)) +
                                  2 * al(8 * ni) + wq_bytes(std::max<int64_t>(ni, 1)) + al(8 * 64));
    return UVA_OK;
}

// engine/metrics.py:148-210. out (device, UVA_MET_N doubles), per_tri
// (device, m*6 or null): s1, s2, signed UV area, 3D area, good, angle error.
extern "C" int uva_distortion_report(const double* V, const double* UV, const int32_t* F, const int32_t* islands,
                                     int32_t n, int32_t m, int32_t n_islands, double* out, double* per_tri,
                                     void* scratch, int64_t scratch_bytes, void* stream) {
    int64_t need = 0;
    if (n < 0 || m < 0 || !out || !scratch || (m > 0 && (!V || !UV || !F)) ||
        uva_metrics_scratch_bytes(m, n_islands, &need) != UVA_OK || scratch_bytes < need) {
        uva_set_error("uva_distortion_report: bad arguments or scratch too small");
        return UVA_E_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int ni = islands ? std::max(n_islands, 1) : 1;
    auto* base = static_cast<unsigned char*>(scratch);
    const size_t M = std::max(m, 1);
    double* tri = per_tri ? per_tri : reinterpret_cast<double*>(base);
    base += al(48 * M);
    double* isum = reinterpret_cast<double*>(base); base += al(32 * static_cast<size_t>(ni));
    QIn qa{reinterpret_cast<double*>(base), reinterpret_cast<double*>(base + al(8 * M))}; base += 2 * al(8 * M);
    QIn qg{reinterpret_cast<double*>(base), reinterpret_cast<double*>(base + al(8 * M))}; base += 2 * al(8 * M);
    QIn qc{reinterpret_cast<double*>(base), reinterpret_cast<double*>(base + al(8 * M))}; base += 2 * al(8 * M);
    QIn qd{reinterpret_cast<double*>(base), reinterpret_cast<double*>(base + al(8 * static_cast<size_t>(ni)))};
    base += 2 * al(8 * static_cast<size_t>(ni));
    unsigned char* wqs = base; base += wq_bytes(ni);
    double* sums = reinterpret_cast<double*>(base);   // 64 doubles
    cudaMemsetAsync(sums, 0, 8 * 64, s);
    cudaMemsetAsync(isum, 0, 32 * static_cast<size_t>(ni), s);
    const int tb = 256, gb = std::max(1, (m + tb - 1) / tb);
    k_met_a<<<gb, tb, 0, s>>>(m, V, UV, F, islands, tri, sums, isum);
    k_met_b<<<gb, tb, 0, s>>>(m, tri, islands, isum, sums, qa, qg, qc);
    if (islands) k_met_islands<<<(ni + tb - 1) / tb, tb, 0, s>>>(ni, isum, sums, qd);
    UVA_CHECK_LAUNCH("uva_distortion_report");
    // sums: [0] a3, [1] |sa|, [2..15] k_met_b terms, [16] mirrored, [17] ia3 total
    cudaMemcpyAsync(out, sums, sizeof(double) * 24, cudaMemcpyDeviceToDevice, s);
    int rc = wquantile(m, qa.x, qa.w, nullptr, 1, 1, 0.95, out + 24, wqs, s);
    if (rc == UVA_OK) rc = wquantile(m, qg.x, qg.w, nullptr, 1, 1, 0.95, out + 25, wqs, s);
    if (rc == UVA_OK && islands) rc = wquantile(m, qc.x, qc.w, nullptr, 1, 1, 0.95, out + 26, wqs, s);
    if (rc == UVA_OK && islands) rc = wquantile(ni, qd.x, qd.w, nullptr, 1, 1, 0.95, out + 27, wqs, s);
    return rc;
}

extern "C" int uva_quality_scratch_bytes(int64_t t, int64_t nc, int64_t* bytes) {
    if (t < 0 || nc < 0 || !bytes) { uva_set_error("uva_quality_scratch_bytes: bad arguments"); return UVA_E_ARG; }
    const size_t T = std::max<int64_t>(t, 1), C = std::max<int64_t>(nc, 1);
    *bytes = static_cast<int64_t>(al(48 * T) + al(64 * C) + 4 * al(8 * T) + 3 * al(8 * C) + wq_bytes(static_cast<int>(C)));
    return UVA_OK;
}

// engine/param.py:520-551 for every island of a batch (after uva_batch_setup
// with UVA_SEM_PARAM, so frames follow param.local_frames). out (device,
// nc*8 doubles): flips, aniso_p95, aniso_mean, area_p95, area_logdev,
// stretch, scale, 3D area. per_aniso, per_area (device, t doubles).
extern "C" int uva_chart_quality(const uva_batch* b, double* out, double* per_aniso, double* per_area, void* scratch,
                                 int64_t scratch_bytes, void* stream) {
    int64_t need = 0;
    if (!b || !out || !per_aniso || !per_area || !scratch || uva_quality_scratch_bytes(b->t, b->nc, &need) != UVA_OK ||
        scratch_bytes < need) {
        uva_set_error("uva_chart_quality: bad arguments or scratch too small");
        return UVA_E_ARG;
    }
    if (b->nc == 0 || b->t == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t T = b->t, C = b->nc;
    auto* base = static_cast<unsigned char*>(scratch);
    double* tri = reinterpret_cast<double*>(base); base += al(48 * T);
    double* isum = reinterpret_cast<double*>(base); base += al(64 * C);
    QIn qa{reinterpret_cast<double*>(base), reinterpret_cast<double*>(base + al(8 * T))}; base += 2 * al(8 * T);
    QIn qr{reinterpret_cast<double*>(base), reinterpret_cast<double*>(base + al(8 * T))}; base += 2 * al(8 * T);
    double* stretch = reinterpret_cast<double*>(base); base += al(8 * C);
    double* q95a = reinterpret_cast<double*>(base); base += al(8 * C);
    double* q95r = reinterpret_cast<double*>(base); base += al(8 * C);
    unsigned char* wqs = base;
    cudaMemsetAsync(isum, 0, 64 * C, s);
    cudaMemsetAsync(stretch, 0, 8 * C, s);
    const int tb = 256, gb = (b->t + tb - 1) / tb;
    k_quality_a<<<gb, tb, 0, s>>>(*b, tri, isum);
    k_quality_b<<<gb, tb, 0, s>>>(*b, tri, isum, qa, qr, per_aniso, per_area, stretch);
    UVA_CHECK_LAUNCH("uva_chart_quality");
    // per-island quantiles: the island of triangle f is tri4[4 f + 3]
    int rc = wquantile(b->t, qa.x, qa.w, b->tri4 + 3, 4, b->nc, 0.95, q95a, wqs, s);
    if (rc == UVA_OK) rc = wquantile(b->t, qr.x, qr.w, b->tri4 + 3, 4, b->nc, 0.95, q95r, wqs, s);
    if (rc != UVA_OK) return rc;
    k_quality_out<<<(b->nc + tb - 1) / tb, tb, 0, s>>>(b->nc, isum, stretch, q95a, q95r, out);
    UVA_CHECK_LAUNCH("uva_chart_quality/out");
    return UVA_OK;
}
