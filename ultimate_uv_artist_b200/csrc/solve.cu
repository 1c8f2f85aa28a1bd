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
    if (f >= b.t) return;
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
    double m = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int e = b.tri_edge[3 * f + k];
        if (e >= 0) atomicAdd(&b.wedge[e], w[k]);
        m = fmax(m, fabs(w[k]));
    }
    atomic_max_nonneg(&wmax_isl[tv.w], m);
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
        b.slot_w[q] = w32;
        sum += static_cast<double>(w32);
    }
    b.wdiag[v] = sum;
    b.dinv[v] = sum > 1e-30 ? static_cast<float>(1.0 / sum) : 1.0f;
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
struct Isl {
    int id, v0, n, f0, nt, s0, pin;
    double wpin;
};

__device__ __forceinline__ Isl load_island(const uva_batch& b, int isl) {
    Isl I;
    I.id = isl;
    I.v0 = b.vofs[isl]; I.n = b.vofs[isl + 1] - I.v0;
    I.f0 = b.tofs[isl]; I.nt = b.tofs[isl + 1] - I.f0;
    I.s0 = b.sofs[isl];
    I.pin = b.pins[3 * isl];
    I.wpin = b.wpin[isl];
    return I;
}

// Sliced-ELL row cursor: row i of the island lives in slice s0 + i/32, lane i%32.
struct Row {
    int q0, width;
};
__device__ __forceinline__ Row row_of(const uva_batch& b, const Isl& I, int i) {
    const int s = I.s0 + (i >> 5);
    const int p = b.slice_ptr[s];
    Row r;
    r.q0 = p + (i & 31);
    r.width = (b.slice_ptr[s + 1] - p) >> 5;
    return r;
}

// Operator modes of the shared CG machinery.
enum Op { OP_ARAP = 0, OP_LSCM = 1 };

// y = A x for one row (FP64): ARAP Laplacian + soft pin, or the LSCM
// conformal operator H = [[L, C], [-C, L]] (param.py:145-150).
template <Op OP>
__device__ __forceinline__ double2 apply_row64(const uva_batch& b, const Isl& I, int i, const double2* x) {
    const Row r = row_of(b, I, i);
    const double2 xi = x[I.v0 + i];
    double ax = 0.0, ay = 0.0;
    for (int k = 0; k < r.width; ++k) {
        const int q = r.q0 + 32 * k;
        const int j = __ldg(b.slot_col + q);
        const double w = static_cast<double>(__ldg(b.slot_w + q));
        const double2 xj = x[I.v0 + j];
        ax += w * (xi.x - xj.x);
        ay += w * (xi.y - xj.y);
        if (OP == OP_LSCM) {
            const double c = static_cast<double>(__ldg(b.slot_c + q));
            ax += c * xj.y;
            ay -= c * xj.x;
        }
    }
    if (OP == OP_ARAP && i == I.pin) { ax += I.wpin * xi.x; ay += I.wpin * xi.y; }
    return make_double2(ax, ay);
}

template <Op OP>
__device__ __forceinline__ float2 apply_row32(const uva_batch& b, const Isl& I, int i, const float2* x, float wpin32) {
    const Row r = row_of(b, I, i);
    const float2 xi = x[I.v0 + i];
    float ax = 0.0f, ay = 0.0f;
    for (int k = 0; k < r.width; ++k) {
        const int q = r.q0 + 32 * k;
        const int j = __ldg(b.slot_col + q);
        const float w = __ldg(b.slot_w + q);
        const float2 xj = x[I.v0 + j];
        ax = fmaf(w, xi.x - xj.x, ax);
        ay = fmaf(w, xi.y - xj.y, ay);
        if (OP == OP_LSCM) {
            const float c = __ldg(b.slot_c + q);
            ax = fmaf(c, xj.y, ax);
            ay = fmaf(-c, xj.x, ay);
        }
    }
    if (OP == OP_ARAP && i == I.pin) { ax = fmaf(wpin32, xi.x, ax); ay = fmaf(wpin32, xi.y, ay); }
    return make_float2(ax, ay);
}

struct Lscm {
    int p0, p1;   // pinned vertices (local); -1 when unused
};

__device__ __forceinline__ bool pinned(const Lscm& L, int i) { return i == L.p0 || i == L.p1; }

__device__ __forceinline__ float jacobi(const uva_batch& b, const Isl& I, int i, Op op) {
    const float d = b.dinv[I.v0 + i];
    if (op == OP_ARAP && i == I.pin) {
        const double diag = b.wdiag[I.v0 + i] + I.wpin;
        return diag > 1e-30 ? static_cast<float>(1.0 / diag) : 1.0f;
    }
    return d;
}

// Shared-memory workspace of one team.
template <int NT>
struct Smem {
    double redd[2 * 4 * (NT / 32)];
    float redf[2 * 4 * (NT / 32)];
    int redi[2 * (NT / 32)];
    int island;
};

// Solves A x = rhs for one island: x64 holds the start on entry and the
// solution on exit. FP64 residual recomputation (refinement) around FP32
// Jacobi-PCG corrections. NCOL = 2 (ARAP: u and v separately) or 1 (LSCM:
// one vector of 2n unknowns). Returns inner iterations; writes residuals.
template <int NT, Op OP, int NCOL>
__device__ int refine_solve(const uva_batch& b, const Isl& I, const Lscm& LS, const uva_solve_params& prm,
                            const double bb[2], Smem<NT>& sm, int& phase, double res_out[2], int& nref,
                            bool& capped) {
    const int tid = threadIdx.x;
    double2* x64 = reinterpret_cast<double2*>(b.x64);
    const double2* b64 = reinterpret_cast<const double2*>(b.b64);
    float2* r32 = reinterpret_cast<float2*>(b.r32);
    float2* d32 = reinterpret_cast<float2*>(b.d32);
    float2* p32 = reinterpret_cast<float2*>(b.p32);
    float2* q32 = reinterpret_cast<float2*>(b.q32);
    const float wpin32 = static_cast<float>(I.wpin);
    int total = 0;
    capped = false;
    nref = 0;
    for (int ref = 0;; ++ref) {
        // ---- FP64 residual r = rhs - A x
        double rr[2] = {0.0, 0.0};
        for (int i = tid; i < I.n; i += NT) {
            double2 r;
            if (OP == OP_LSCM && pinned(LS, i)) {
                r = make_double2(0.0, 0.0);
            } else {
                const double2 ax = apply_row64<OP>(b, I, i, x64);
                const double2 rhs = OP == OP_ARAP ? b64[I.v0 + i] : make_double2(0.0, 0.0);
                r = rhs - ax;
            }
            r32[I.v0 + i] = make_float2(static_cast<float>(r.x), static_cast<float>(r.y));
            rr[0] += r.x * r.x;
            rr[1] += r.y * r.y;
        }
        block_sum<NT, 2>(rr, sm.redd, phase);
        ++nref;
        double res[2];
        bool done = true;
        if (NCOL == 2) {
            for (int c = 0; c < 2; ++c) {
                res[c] = sqrt(rr[c] / fmax(bb[c], 1e-300));
                if (!(rr[c] <= prm.tol * prm.tol * fmax(bb[c], 1e-300))) done = false;
            }
        } else {
            const double s = rr[0] + rr[1];
            res[0] = res[1] = sqrt(s / fmax(bb[0], 1e-300));
            done = s <= prm.tol * prm.tol * fmax(bb[0], 1e-300);
        }
        res_out[0] = res[0]; res_out[1] = res[1];
        if (done) break;
        if (ref >= prm.max_refine || !isfinite(rr[0] + rr[1])) { capped = true; break; }
        // ---- inner FP32 PCG on A d = r (d0 = 0)
        float rz[2] = {0.f, 0.f}, r0[2] = {0.f, 0.f};
        for (int i = tid; i < I.n; i += NT) {
            const float2 r = r32[I.v0 + i];
            const float m = (OP == OP_LSCM && pinned(LS, i)) ? 0.0f : jacobi(b, I, i, OP);
            const float2 z = make_float2(m * r.x, m * r.y);
            d32[I.v0 + i] = make_float2(0.f, 0.f);
            p32[I.v0 + i] = z;
            rz[0] += r.x * z.x; rz[1] += r.y * z.y;
            r0[0] += r.x * r.x; r0[1] += r.y * r.y;
        }
        float red4[4] = {rz[0], rz[1], r0[0], r0[1]};
        block_sum<NT, 4>(red4, sm.redf, phase);
        float thr[2];
        bool act[2];
        if (NCOL == 2) {
            for (int c = 0; c < 2; ++c) {
                rz[c] = red4[c];
                const float a = static_cast<float>(prm.inner_eta) * sqrtf(red4[2 + c]);
                const float t = static_cast<float>(0.5 * prm.tol * sqrt(bb[c]));
                thr[c] = fmaxf(a, t);
                act[c] = red4[2 + c] > thr[c] * thr[c] && rz[c] > 0.f;
            }
        } else {
            rz[0] = red4[0] + red4[1]; rz[1] = rz[0];
            const float a = static_cast<float>(prm.inner_eta) * sqrtf(red4[2] + red4[3]);
            const float t = static_cast<float>(0.5 * prm.tol * sqrt(bb[0]));
            thr[0] = thr[1] = fmaxf(a, t);
            act[0] = act[1] = (red4[2] + red4[3]) > thr[0] * thr[0] && rz[0] > 0.f;
        }
        int it = 0;
        while ((act[0] || act[1]) && it < prm.max_inner) {
            __syncthreads();   // p complete
            float pq[2] = {0.f, 0.f};
            for (int i = tid; i < I.n; i += NT) {
                float2 q;
                if (OP == OP_LSCM && pinned(LS, i)) q = make_float2(0.f, 0.f);
                else q = apply_row32<OP>(b, I, i, p32, wpin32);
                q32[I.v0 + i] = q;
                const float2 p = p32[I.v0 + i];
                pq[0] += p.x * q.x; pq[1] += p.y * q.y;
            }
            block_sum<NT, 2>(pq, sm.redf, phase);
            float alpha[2];
            if (NCOL == 2) {
                for (int c = 0; c < 2; ++c) alpha[c] = (act[c] && pq[c] > 0.f) ? rz[c] / pq[c] : 0.f;
            } else {
                const float s = pq[0] + pq[1];
                alpha[0] = alpha[1] = (act[0] && s > 0.f) ? rz[0] / s : 0.f;
            }
            float acc[4] = {0.f, 0.f, 0.f, 0.f};   // rz_new (2), rr (2)
            for (int i = tid; i < I.n; i += NT) {
                const float2 p = p32[I.v0 + i], q = q32[I.v0 + i];
                float2 d = d32[I.v0 + i], r = r32[I.v0 + i];
                d.x = fmaf(alpha[0], p.x, d.x); d.y = fmaf(alpha[1], p.y, d.y);
                r.x = fmaf(-alpha[0], q.x, r.x); r.y = fmaf(-alpha[1], q.y, r.y);
                d32[I.v0 + i] = d; r32[I.v0 + i] = r;
                const float m = (OP == OP_LSCM && pinned(LS, i)) ? 0.0f : jacobi(b, I, i, OP);
                acc[0] += r.x * m * r.x; acc[1] += r.y * m * r.y;
                acc[2] += r.x * r.x; acc[3] += r.y * r.y;
            }
            block_sum<NT, 4>(acc, sm.redf, phase);
            ++it;
            float beta[2];
            if (NCOL == 2) {
                for (int c = 0; c < 2; ++c) {
                    const bool conv = acc[2 + c] <= thr[c] * thr[c];
                    beta[c] = (act[c] && rz[c] > 0.f) ? acc[c] / rz[c] : 0.f;
                    if (act[c]) rz[c] = acc[c];
                    if (conv || !(acc[c] > 0.f)) act[c] = false;
                }
            } else {
                const float s = acc[0] + acc[1], rrs = acc[2] + acc[3];
                const bool conv = rrs <= thr[0] * thr[0];
                beta[0] = beta[1] = (act[0] && rz[0] > 0.f) ? s / rz[0] : 0.f;
                rz[0] = rz[1] = s;
                if (conv || !(s > 0.f)) act[0] = act[1] = false;
            }
            if (!(act[0] || act[1])) break;
            for (int i = tid; i < I.n; i += NT) {
                const float2 r = r32[I.v0 + i], p = p32[I.v0 + i];
                const float m = (OP == OP_LSCM && pinned(LS, i)) ? 0.0f : jacobi(b, I, i, OP);
                p32[I.v0 + i] = make_float2(fmaf(beta[0], p.x, m * r.x), fmaf(beta[1], p.y, m * r.y));
            }
        }
        if (it >= prm.max_inner) capped = true;
        total += it;
        __syncthreads();
        for (int i = tid; i < I.n; i += NT) {
            const float2 d = d32[I.v0 + i];
            double2 x = x64[I.v0 + i];
            x.x += static_cast<double>(d.x); x.y += static_cast<double>(d.y);
            x64[I.v0 + i] = x;
        }
        __syncthreads();
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
        energy = 0.0;
    } else {
        energy = 0.0;
        if (fabs(x1 * y2) >= 1e-300) {
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
    }
    // edge k runs corner k+1 -> k+2; frame corners (0,0), (x1,0), (x2,y2)
    const double cxs[3] = {0.0, x1, x2}, cys[3] = {0.0, 0.0, y2};
    double vx[3], vy[3];
    const double wk[3] = {wt.x, wt.y, wt.z};
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
    const double2 d0 = X[I.v0 + tv.x] - u0, d1 = X[I.v0 + tv.y] - u1, d2 = X[I.v0 + tv.z] - u2;
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
    if (A == 0.0 || fabs(A) < 1e-30 * fmax(fabs(B), 1e-300)) {
        return B < 0.0 ? -C / B : big;
    }
    const double disc = B * B - 4.0 * A * C;
    if (disc < 0.0) return big;
    const double sq = sqrt(disc);
    const double r1 = (-B - sq) / (2.0 * A), r2 = (-B + sq) / (2.0 * A);
    double t = big;
    if (r1 > 0.0 && r1 < t) t = r1;
    if (r2 > 0.0 && r2 < t) t = r2;
    return t;
}

template <int NT>
__global__ void __launch_bounds__(NT) k_arap(uva_batch b, uva_solve_params prm, const int32_t* order, int count) {
    __shared__ Smem<NT> sm;
    int phase = 0;
    const int tid = threadIdx.x;
    const bool batch = b.semantics == UVA_SEM_BATCH;
    double2* U = reinterpret_cast<double2*>(b.U);
    double2* x64 = reinterpret_cast<double2*>(b.x64);
    double2* b64 = reinterpret_cast<double2*>(b.b64);
    const double2* rc = reinterpret_cast<const double2*>(b.rc);
    for (;;) {
        if (tid == 0) sm.island = atomicAdd(b.work, 1);
        __syncthreads();
        const int qi = sm.island;
        __syncthreads();
        if (qi >= count) break;
        const Isl I = load_island(b, order[qi]);
        const Lscm LS{-1, -1};
        uva_island_status st{};
        bool use_ls = prm.line_search != 0;
        double prev_e = 0.0;
        for (int it = 0; it < prm.iters; ++it) {
            // ---- local step over the island's triangles
            double e_loc[1] = {0.0};
            int flips = 0;
            for (int f = I.f0 + tid; f < I.f0 + I.nt; f += NT) {
                double e; int fl;
                local_terms(b, I, f, U, batch, e, fl);
                e_loc[0] += e;
                flips += fl;
            }
            if (!batch) {
                double ev[2] = {e_loc[0], static_cast<double>(flips)};
                block_sum<NT, 2>(ev, sm.redd, phase);
                if (it == 0) {
                    use_ls = prm.line_search != 0 && ev[1] == 0.0;
                    prev_e = ev[0];
                } else if (prm.energy_tol > 0.0 && fabs(prev_e - ev[0]) <= prm.energy_tol * fmax(prev_e, 1e-300)) {
                    st.flags |= UVA_ST_ENERGYSTOP;
                    st.energy = ev[0];
                    break;
                } else {
                    prev_e = ev[0];
                }
                st.energy = ev[0];
            }
            __syncthreads();   // corner terms complete
            // ---- gather the right-hand side per vertex, warm start x = U
            double bb[2] = {0.0, 0.0};
            for (int i = tid; i < I.n; i += NT) {
                const int v = I.v0 + i;
                double bx = 0.0, by = 0.0;
                for (int p = b.vt_ptr[v]; p < b.vt_ptr[v + 1]; ++p) {
                    const double2 c = rc[b.vt[p]];
                    bx += c.x; by += c.y;
                }
                const double2 u = U[v];
                if (i == I.pin) { bx += I.wpin * u.x; by += I.wpin * u.y; }
                b64[v] = make_double2(bx, by);
                x64[v] = u;
                bb[0] += bx * bx; bb[1] += by * by;
            }
            block_sum<NT, 2>(bb, sm.redd, phase);
            // ---- global step
            int nref = 0;
            bool capped = false;
            st.cg_iters += refine_solve<NT, OP_ARAP, 2>(b, I, LS, prm, bb, sm, phase, st.resid, nref, capped);
            st.refinements += nref;
            if (capped) st.flags |= UVA_ST_MAXITER;
            // ---- non-finite charts keep their layout (gpu.py:235-240)
            int bad = 0;
            for (int i = tid; i < I.n; i += NT) bad |= finite2(x64[I.v0 + i]) ? 0 : 1;
            bad = block_or<NT>(bad, sm.redi, phase);
            if (bad) {
                st.flags |= UVA_ST_NONFINITE;
                st.outer_iters = it + 1;
                continue;
            }
            double step = 1.0;
            if (use_ls) {
                double tmin = 1e30;
                for (int f = I.f0 + tid; f < I.f0 + I.nt; f += NT) tmin = fmin(tmin, step_bound(b, I, f, U, x64, batch));
                tmin = block_min<NT, double>(tmin, sm.redd, phase);
                step = batch ? fmin(0.9 * tmin, 1.0) : fmin(1.0, 0.9 * tmin);
            }
            st.step = step;
            for (int i = tid; i < I.n; i += NT) {
                const int v = I.v0 + i;
                const double2 u = U[v], x = x64[v];
                U[v] = use_ls ? make_double2(u.x + (x.x - u.x) * step, u.y + (x.y - u.y) * step) : x;
            }
            st.outer_iters = it + 1;
            __syncthreads();
        }
        if (tid == 0) b.status[I.id] = st;
        __syncthreads();
    }
}

// LSCM per island: hard pins p0 -> (0,0), p1 -> (|P[p1]-P[p0]|, 0); start
// from the projection onto the mean-normal plane aligned with the pins.
template <int NT>
__global__ void __launch_bounds__(NT) k_lscm(uva_batch b, uva_solve_params prm, const int32_t* order, int count) {
    __shared__ Smem<NT> sm;
    __shared__ double basis[8];
    int phase = 0;
    const int tid = threadIdx.x;
    double2* x64 = reinterpret_cast<double2*>(b.x64);
    double2* U = reinterpret_cast<double2*>(b.U);
    const double* P = b.P;
    for (;;) {
        if (tid == 0) sm.island = atomicAdd(b.work, 1);
        __syncthreads();
        const int qi = sm.island;
        __syncthreads();
        if (qi >= count) break;
        const Isl I = load_island(b, order[qi]);
        Lscm LS{b.pins[3 * I.id + 1], b.pins[3 * I.id + 2]};
        uva_island_status st{};
        if (LS.p0 < 0 || I.n == 0) {
            st.flags |= UVA_ST_NOBOUNDARY;
            for (int i = tid; i < I.n; i += NT) U[I.v0 + i] = make_double2(0.0, 0.0);
            if (tid == 0) b.status[I.id] = st;
            __syncthreads();
            continue;
        }
        // mean normal (sum of triangle cross products)
        double nrm[3] = {0.0, 0.0, 0.0};
        for (int f = I.f0 + tid; f < I.f0 + I.nt; f += NT) {
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
        block_sum<NT, 3>(nrm, sm.redd, phase);
        const double* pp0 = P + 3 * (I.v0 + LS.p0);
        const double* pp1 = P + 3 * (I.v0 + LS.p1);
        if (tid == 0) {
            double nl = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
            double nx = 0.0, ny = 0.0, nz = 1.0;
            if (nl > 0.0 && isfinite(nl)) { nx = nrm[0] / nl; ny = nrm[1] / nl; nz = nrm[2] / nl; }
            double ax = pp1[0] - pp0[0], ay = pp1[1] - pp0[1], az = pp1[2] - pp0[2];
            const double d = sqrt(ax * ax + ay * ay + az * az);
            const double dn = ax * nx + ay * ny + az * nz;
            ax -= dn * nx; ay -= dn * ny; az -= dn * nz;
            double al = sqrt(ax * ax + ay * ay + az * az);
            double s = 1.0;
            if (al > 0.0 && isfinite(al)) { s = d / al; ax /= al; ay /= al; az /= al; }
            else { ax = 1.0; ay = 0.0; az = 0.0; }
            basis[0] = ax * s; basis[1] = ay * s; basis[2] = az * s;
            basis[3] = (ny * az - nz * ay) * s; basis[4] = (nz * ax - nx * az) * s; basis[5] = (nx * ay - ny * ax) * s;
            basis[6] = d;
        }
        __syncthreads();
        for (int i = tid; i < I.n; i += NT) {
            const double* pi = P + 3 * (I.v0 + i);
            const double dx = pi[0] - pp0[0], dy = pi[1] - pp0[1], dz = pi[2] - pp0[2];
            double2 x = make_double2(dx * basis[0] + dy * basis[1] + dz * basis[2], dx * basis[3] + dy * basis[4] + dz * basis[5]);
            if (i == LS.p0) x = make_double2(0.0, 0.0);
            if (i == LS.p1) x = make_double2(basis[6], 0.0);
            x64[I.v0 + i] = x;
        }
        __syncthreads();
        // ||rhs||^2 of the reduced system: A applied to the pinned values only
        double bb[2] = {0.0, 0.0};
        {
            const double dpin = basis[6];
            for (int i = tid; i < I.n; i += NT) {
                if (pinned(LS, i)) continue;
                const Row r = row_of(b, I, i);
                double ax = 0.0, ay = 0.0;
                for (int k = 0; k < r.width; ++k) {
                    const int q = r.q0 + 32 * k;
                    const int j = b.slot_col[q];
                    if (j != LS.p1) continue;   // p0 sits at the origin
                    const double w = static_cast<double>(b.slot_w[q]);
                    const double c = static_cast<double>(b.slot_c[q]);
                    ax += -w * dpin;
                    ay -= c * dpin;
                }
                bb[0] += ax * ax + ay * ay;
            }
            block_sum<NT, 2>(bb, sm.redd, phase);
        }
        int nref = 0;
        bool capped = false;
        st.cg_iters = refine_solve<NT, OP_LSCM, 1>(b, I, LS, prm, bb, sm, phase, st.resid, nref, capped);
        st.refinements = nref;
        if (capped) st.flags |= UVA_ST_MAXITER;
        int bad = 0;
        for (int i = tid; i < I.n; i += NT) bad |= finite2(x64[I.v0 + i]) ? 0 : 1;
        bad = block_or<NT>(bad, sm.redi, phase);
        if (bad) st.flags |= UVA_ST_NONFINITE;
        for (int i = tid; i < I.n; i += NT) U[I.v0 + i] = x64[I.v0 + i];
        if (tid == 0) b.status[I.id] = st;
        __syncthreads();
    }
}

int sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

bool check_batch(const uva_batch* b) {
    return b && b->nc >= 0 && b->n >= 0 && b->t >= 0 &&
           (b->nc == 0 || (b->vofs && b->tofs && b->sofs && b->order && b->work));
}

template <int NT>
int launch_arap(uva_batch* b, const uva_solve_params* prm, cudaStream_t s, bool lscm) {
    const int32_t* order = b->order;
    cudaMemsetAsync(b->work, 0, sizeof(int32_t) * 4, s);
    int occ = 0;
    if (lscm) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_lscm<NT>, NT, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_arap<NT>, NT, 0);
    const int grid = std::max(1, std::min(b->nc, sm_count() * std::max(occ, 1)));
    if (lscm) k_lscm<NT><<<grid, NT, 0, s>>>(*b, *prm, order, b->nc);
    else k_arap<NT><<<grid, NT, 0, s>>>(*b, *prm, order, b->nc);
    UVA_CHECK_LAUNCH(lscm ? "uva_lscm" : "uva_arap");
    return UVA_OK;
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
    return UVA_OK;
}

extern "C" int uva_arap(uva_batch* b, const uva_solve_params* prm, void* stream) {
    if (!check_batch(b) || !prm) { uva_set_error("uva_arap: bad arguments"); return UVA_E_ARG; }
    if (b->nc == 0 || prm->iters <= 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (prm->threads) {
        case 128: return launch_arap<128>(b, prm, s, false);
        case 512: return launch_arap<512>(b, prm, s, false);
        default: return launch_arap<256>(b, prm, s, false);
    }
}

extern "C" int uva_lscm(uva_batch* b, const uva_solve_params* prm, void* stream) {
    if (!check_batch(b) || !prm) { uva_set_error("uva_lscm: bad arguments"); return UVA_E_ARG; }
    if (b->nc == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (prm->threads) {
        case 128: return launch_arap<128>(b, prm, s, true);
        case 512: return launch_arap<512>(b, prm, s, true);
        default: return launch_arap<256>(b, prm, s, true);
    }
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
constexpr size_t kNoAllocBytes = kNaWork + kNaX64 + kNaB64 + kNaRc + 4 * kNaF32;   // 5,243,136 bytes

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
    if (!check_batch(b) || !prm || !b->status || !b->U) {
        uva_set_error("uva_arap_noalloc: bad arguments (status and U are required outputs)");
        return UVA_E_ARG;
    }
    if (b->n > kNoAllocMaxVerts || b->t > kNoAllocMaxTris) {
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
    w.q32 = reinterpret_cast<float*>(base + off);
    // the work counter is the only scratch that must start at zero; launch_arap
    // clears it on the stream before the launch
    return launch_arap<256>(&w, prm, static_cast<cudaStream_t>(stream), false);
}
