// Distortion energies of engine/param.py:294-319 with hand-written backward
// passes, for every island of a batch.
//
//   kind 0 (ARAP):      E_f = area * ((q + r - 1)^2 + (q - r - 1)^2)
//                           = area * (|J|^2 - 4 q + 2),  dE/dJ = 2 area (J - R)
//   kind 1 (sym. Dir.): E_f = area * (|J|^2 + |J|^2 / det^2 - 4), inf if det <= 0
//                       dE/dJ = area * (2 J (1 + 1/det^2) - 2 |J|^2 / det^3 cof(J))
// J maps the triangle's isometric frame M = [[x1, x2], [0, y2]] to UV edges,
// J = [u1 - u0, u2 - u0] M^-1, with x1 = |e1|, x2 = e1.e2 / |e1|,
// y2 = |e1 x e2| / |e1|, area = |e1 x e2| / 2 (param.local_frames). The
// gradient with respect to the 3D positions goes through the frame:
// dE/dM = -J^T G M^-T, then x1, x2, y2 and area as functions of e1, e2.
// Triangles with |x1 y2| < 1e-300 contribute nothing (param.py:301-303).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"

using namespace uva;

namespace {

struct EnTri {
    double e1[3], e2[3], n[3];
    double l1, nn, x1, x2, y2, area;
    double j00, j01, j10, j11;
    bool live;
};

__device__ __forceinline__ EnTri en_tri(const double* P, const double* U, int v0, int4 tv) {
    EnTri t;
    const double* p0 = P + 3 * (v0 + tv.x);
    const double* p1 = P + 3 * (v0 + tv.y);
    const double* p2 = P + 3 * (v0 + tv.z);
#pragma unroll
    for (int k = 0; k < 3; ++k) { t.e1[k] = p1[k] - p0[k]; t.e2[k] = p2[k] - p0[k]; }
    t.n[0] = t.e1[1] * t.e2[2] - t.e1[2] * t.e2[1];
    t.n[1] = t.e1[2] * t.e2[0] - t.e1[0] * t.e2[2];
    t.n[2] = t.e1[0] * t.e2[1] - t.e1[1] * t.e2[0];
    t.l1 = sqrt(t.e1[0] * t.e1[0] + t.e1[1] * t.e1[1] + t.e1[2] * t.e1[2]);
    t.nn = sqrt(t.n[0] * t.n[0] + t.n[1] * t.n[1] + t.n[2] * t.n[2]);
    const double il = 1.0 / fmax(t.l1, 1e-300);
    t.x1 = t.l1;
    t.x2 = (t.e1[0] * t.e2[0] + t.e1[1] * t.e2[1] + t.e1[2] * t.e2[2]) * il;
    t.y2 = t.nn * il;   // e2 . (n/|n| x e1/|e1|) = |n| / |e1|
    t.area = 0.5 * t.nn;
    t.live = fabs(t.x1 * t.y2) >= 1e-300;
    const double2* UU = reinterpret_cast<const double2*>(U);
    const double2 u0 = UU[v0 + tv.x], u1 = UU[v0 + tv.y], u2 = UU[v0 + tv.z];
    if (t.live) {
        t.j00 = (u1.x - u0.x) / t.x1; t.j10 = (u1.y - u0.y) / t.x1;
        t.j01 = ((u2.x - u0.x) - t.j00 * t.x2) / t.y2; t.j11 = ((u2.y - u0.y) - t.j10 * t.x2) / t.y2;
    } else {
        t.j00 = t.j01 = t.j10 = t.j11 = 0.0;
    }
    return t;
}

// f(J) and dE/dJ per unit area; returns false for an inverted SD triangle.
__device__ __forceinline__ bool en_f(const EnTri& t, int kind, double& f, double (&G)[4]) {
    const double fro = t.j00 * t.j00 + t.j01 * t.j01 + t.j10 * t.j10 + t.j11 * t.j11;
    if (kind == 0) {
        const double qe = 0.5 * (t.j00 + t.j11), qh = 0.5 * (t.j10 - t.j01);
        const double rf = 0.5 * (t.j00 - t.j11), rg = 0.5 * (t.j10 + t.j01);
        const double q = sqrt(qe * qe + qh * qh), r = sqrt(rf * rf + rg * rg);
        f = (q + r - 1.0) * (q + r - 1.0) + (q - r - 1.0) * (q - r - 1.0);
        double c = 0.0, s = 0.0;
        if (q > 0.0) { c = qe / q; s = qh / q; }
        G[0] = 2.0 * (t.j00 - c); G[1] = 2.0 * (t.j01 + s); G[2] = 2.0 * (t.j10 - s); G[3] = 2.0 * (t.j11 - c);
        return true;
    }
    const double det = t.j00 * t.j11 - t.j01 * t.j10;
    if (!(det > 0.0)) {
        f = INFINITY;
        G[0] = G[1] = G[2] = G[3] = 0.0;
        return false;
    }
    const double id2 = 1.0 / (det * det);
    f = fro + fro * id2 - 4.0;
    const double a = 2.0 * (1.0 + id2), b = -2.0 * fro * id2 / det;
    G[0] = a * t.j00 + b * t.j11;
    G[1] = a * t.j01 - b * t.j10;
    G[2] = a * t.j10 - b * t.j01;
    G[3] = a * t.j11 + b * t.j00;
    return true;
}

template <int K>
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Triangles per thread of the forward pass: a thread sums a contiguous run
// of triangles (islands are contiguous in triangle order), then the warp
// folds runs of the same island, so an island's sum takes one FP64 atomic
// per warp and island instead of one per triangle.
constexpr int kFwdItems = 8;

__global__ void k_energy_fwd(const uva_batch b, const double* P, const double* U, int kind, double* e_isl, double* e_tri) {
    const int lane = threadIdx.x & 31;
    const int64_t f0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * kFwdItems;
    int isl = -1;
    double acc = 0.0;
    for (int k = 0; k < kFwdItems; ++k) {
        const int64_t f = f0 + k;
        if (f >= b.t) break;
        const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
        const EnTri t = en_tri(P, U, b.vofs[tv.w], tv);
        double e = 0.0;
        if (t.live) {
            double f_, G[4];
            en_f(t, kind, f_, G);
            e = t.area * f_;
        }
        if (e_tri) e_tri[f] = e;
        if (tv.w != isl) {   // a new island inside the run: flush the previous one
            if (isl >= 0 && acc != 0.0) atomicAdd(e_isl + isl, acc);
            isl = tv.w;
            acc = 0.0;
        }
        acc += e;
    }
    // fold the lanes' last runs: island ids do not decrease along the lanes
    // (idle lanes carry -1 and never match a live run)
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_down_sync(0xffffffffu, acc, o);
        const int yi = __shfl_down_sync(0xffffffffu, isl, o);
        if (lane + o < 32 && yi == isl) acc += y;
    }
    const int prev = __shfl_up_sync(0xffffffffu, isl, 1);
    if (isl >= 0 && (lane == 0 || prev != isl) && acc != 0.0) atomicAdd(e_isl + isl, acc);
}

__global__ void k_energy_bwd(const uva_batch b, const double* P, const double* U, int kind, const double* gscale,
                             double* gU, double* gP) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.t) return;
    const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
    const int v0 = b.vofs[tv.w];
    const EnTri t = en_tri(P, U, v0, tv);
    if (!t.live) return;
    double f_, G[4];
    if (!en_f(t, kind, f_, G)) return;
    const double sc = gscale ? gscale[tv.w] : 1.0;
    const double A = t.area * sc;
    // dE/dJ = A G; J = D M^-1 with D = [du1 du2]: dE/dD = dE/dJ M^-T
    const double g00 = A * G[0], g01 = A * G[1], g10 = A * G[2], g11 = A * G[3];
    // M^-1 = [[1/x1, -x2/(x1 y2)], [0, 1/y2]]; dE/dD = g M^-T
    const double ix1 = 1.0 / t.x1, iy2 = 1.0 / t.y2, m01 = -t.x2 / (t.x1 * t.y2);
    const double d1x = g00 * ix1 + g01 * m01, d2x = g01 * iy2;
    const double d1y = g10 * ix1 + g11 * m01, d2y = g11 * iy2;
    double* gu = gU;
    atomicAdd(gu + 2 * (v0 + tv.y), d1x); atomicAdd(gu + 2 * (v0 + tv.y) + 1, d1y);
    atomicAdd(gu + 2 * (v0 + tv.z), d2x); atomicAdd(gu + 2 * (v0 + tv.z) + 1, d2y);
    atomicAdd(gu + 2 * (v0 + tv.x), -(d1x + d2x)); atomicAdd(gu + 2 * (v0 + tv.x) + 1, -(d1y + d2y));
    if (!gP) return;
    // dE/dM = -J^T (A G) M^-T; M^-T = [[1/x1, 0], [m01, 1/y2]]
    const double jg00 = t.j00 * g00 + t.j10 * g10, jg01 = t.j00 * g01 + t.j10 * g11;
    const double jg10 = t.j01 * g00 + t.j11 * g10, jg11 = t.j01 * g01 + t.j11 * g11;
    const double dM00 = -(jg00 * ix1 + jg01 * m01);    // d/dx1
    const double dM01 = -(jg01 * iy2);                  // d/dx2 (row 0, col 1)
    const double dM11 = -(jg11 * iy2);                  // d/dy2
    (void)jg10;
    const double dArea = sc * f_;
    // x1 = |e1|; x2 = e1.e2/|e1|; y2 = |n|/|e1|; area = |n|/2
    const double l1 = t.l1, nn = t.nn;
    const double dot = t.e1[0] * t.e2[0] + t.e1[1] * t.e2[1] + t.e1[2] * t.e2[2];
    double ge1[3], ge2[3];
    const double nh[3] = {t.n[0] / fmax(nn, 1e-300), t.n[1] / fmax(nn, 1e-300), t.n[2] / fmax(nn, 1e-300)};
    // d|n|/de1 = e2 x nh, d|n|/de2 = nh x e1
    const double dn1[3] = {t.e2[1] * nh[2] - t.e2[2] * nh[1], t.e2[2] * nh[0] - t.e2[0] * nh[2], t.e2[0] * nh[1] - t.e2[1] * nh[0]};
    const double dn2[3] = {nh[1] * t.e1[2] - nh[2] * t.e1[1], nh[2] * t.e1[0] - nh[0] * t.e1[2], nh[0] * t.e1[1] - nh[1] * t.e1[0]};
    const double il = 1.0 / l1, il3 = il * il * il;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double dx1_de1 = t.e1[k] * il;
        const double dx2_de1 = t.e2[k] * il - dot * t.e1[k] * il3, dx2_de2 = t.e1[k] * il;
        const double dy2_de1 = dn1[k] * il - nn * t.e1[k] * il3, dy2_de2 = dn2[k] * il;
        const double da_de1 = 0.5 * dn1[k], da_de2 = 0.5 * dn2[k];
        ge1[k] = dM00 * dx1_de1 + dM01 * dx2_de1 + dM11 * dy2_de1 + dArea * da_de1;
        ge2[k] = dM01 * dx2_de2 + dM11 * dy2_de2 + dArea * da_de2;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        atomicAdd(gP + 3 * (v0 + tv.y) + k, ge1[k]);
        atomicAdd(gP + 3 * (v0 + tv.z) + k, ge2[k]);
        atomicAdd(gP + 3 * (v0 + tv.x) + k, -(ge1[k] + ge2[k]));
    }
}

// ---- p95-stretch refinement: Jacobi-preconditioned descent on the
// symmetric Dirichlet energy, flip-safe and monotone per island.
__global__ void k_descent_dir(int n, const uva_batch b, const int32_t* vert_isl, const double* gU, double* Dd) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int v0 = b.vofs[vert_isl[v]];
    const double d = b.wdiag[v0 + b.vert_row[v]];   // the diagonal is stored by solver row
    const double m = d > 1e-30 ? 1.0 / d : 0.0;
    Dd[2 * v] = -m * gU[2 * v];
    Dd[2 * v + 1] = -m * gU[2 * v + 1];
}

__device__ __forceinline__ void atomic_min_pos(double* addr, double v) {
    if (!(v >= 0.0)) return;
    atomicMin(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// Minimum over the warp's lanes of the same island (island ids do not
// decrease along the lanes), one atomic per island and warp.
__device__ __forceinline__ void island_min_fold(double* tmax, int isl, double t, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_down_sync(0xffffffffu, t, o);
        const int yi = __shfl_down_sync(0xffffffffu, isl, o);
        if (lane + o < 32 && yi == isl && y < t) t = y;
    }
    const int prev = __shfl_up_sync(0xffffffffu, isl, 1);
    if (isl >= 0 && (lane == 0 || prev != isl)) atomic_min_pos(tmax + isl, t);
}

// Per-island flip-safe bound (param.py:259-291 per island).
__global__ void k_island_max_step(const uva_batch b, const double* U, const double* Dd, double* tmax) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int isl = -1;          // idle lanes join the warp's fold with no island
    double t = 1e30;
    if (f < b.t) {
        const int4 tv = reinterpret_cast<const int4*>(b.tri4)[f];
        isl = tv.w;
        const int v0 = b.vofs[tv.w];
        const double2* UU = reinterpret_cast<const double2*>(U);
        const double2* DD = reinterpret_cast<const double2*>(Dd);
        const double2 u0 = UU[v0 + tv.x], u1 = UU[v0 + tv.y], u2 = UU[v0 + tv.z];
        const double2 d0 = DD[v0 + tv.x], d1 = DD[v0 + tv.y], d2 = DD[v0 + tv.z];
        const double ux1 = u1.x - u0.x, uy1 = u1.y - u0.y, ux2 = u2.x - u0.x, uy2 = u2.y - u0.y;
        const double dx1 = d1.x - d0.x, dy1 = d1.y - d0.y, dx2 = d2.x - d0.x, dy2 = d2.y - d0.y;
        const double C = ux1 * uy2 - ux2 * uy1;
        const double B = ux1 * dy2 + dx1 * uy2 - ux2 * dy1 - dx2 * uy1;
        const double A = dx1 * dy2 - dx2 * dy1;
        if (C > 0.0) {
            if (A == 0.0 || fabs(A) < 1e-30 * fmax(fabs(B), 1e-300)) {
                if (B < 0.0) t = -C / B;
            } else {
                const double disc = B * B - 4.0 * A * C;
                if (disc >= 0.0) {
                    const double sq = sqrt(disc);
                    const double r1 = (-B - sq) / (2.0 * A), r2 = (-B + sq) / (2.0 * A);
                    if (r1 > 0.0 && r1 < t) t = r1;
                    if (r2 > 0.0 && r2 < t) t = r2;
                }
            }
        }
    }
    island_min_fold(tmax, isl, t, lane);
}

__global__ void k_trial(int n, const uva_batch b, const double* U, const double* Dd, const double* alpha,
                        const int32_t* vert_isl, double* Ut) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const double a = alpha[vert_isl[v]];
    Ut[2 * v] = U[2 * v] + a * Dd[2 * v];
    Ut[2 * v + 1] = U[2 * v + 1] + a * Dd[2 * v + 1];
}

// Accept per island when the trial energy decreased (Armijo-free monotone
// test), else halve its step; islands that accepted stop shrinking.
__global__ void k_accept(int nc, const double* e_old, const double* e_new, double* alpha, int32_t* accepted) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc || accepted[i]) return;
    if (e_new[i] < e_old[i]) accepted[i] = 1;
    else alpha[i] *= 0.5;
}

__global__ void k_commit(int n, const int32_t* vert_isl, const int32_t* accepted, const double* Ut, double* U) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    if (accepted[vert_isl[v]]) { U[2 * v] = Ut[2 * v]; U[2 * v + 1] = Ut[2 * v + 1]; }
}

__global__ void k_init_alpha(int nc, const double* tmax, double* alpha, int32_t* accepted, double cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    alpha[i] = fmin(cap, 0.9 * tmax[i]);
    accepted[i] = 0;
}

__global__ void k_fill_d(double* p, int n, double v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_vert_isl2(const int32_t* vofs, int nc, int32_t* vert_isl) {
    const int isl = blockIdx.x;
    if (isl >= nc) return;
    for (int v = vofs[isl] + threadIdx.x; v < vofs[isl + 1]; v += blockDim.x) vert_isl[v] = isl;
}

inline int nb(int x) { return std::max(1, (x + 255) / 256); }

}  // namespace

extern "C" int uva_energy_fwd(const uva_batch* b, const double* P, const double* U, int32_t kind, double* e_isl,
                              double* e_tri, void* stream) {
    if (!b || !P || !U || !e_isl || (kind != 0 && kind != 1)) { uva_set_error("uva_energy_fwd: bad arguments"); return UVA_E_ARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(e_isl, 0, sizeof(double) * static_cast<size_t>(std::max(b->nc, 1)), s);
    if (b->t > 0) k_energy_fwd<<<nb((b->t + kFwdItems - 1) / kFwdItems), 256, 0, s>>>(*b, P, U, kind, e_isl, e_tri);
    UVA_CHECK_LAUNCH("uva_energy_fwd");
    return UVA_OK;
}

extern "C" int uva_energy_bwd(const uva_batch* b, const double* P, const double* U, int32_t kind, const double* gscale,
                              double* gU, double* gP, void* stream) {
    if (!b || !P || !U || !gU || (kind != 0 && kind != 1)) { uva_set_error("uva_energy_bwd: bad arguments"); return UVA_E_ARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(gU, 0, sizeof(double) * 2 * static_cast<size_t>(b->n), s);
    if (gP) cudaMemsetAsync(gP, 0, sizeof(double) * 3 * static_cast<size_t>(b->n), s);
    if (b->t > 0) k_energy_bwd<<<nb(b->t), 256, 0, s>>>(*b, P, U, kind, gscale, gU, gP);
    UVA_CHECK_LAUNCH("uva_energy_bwd");
    return UVA_OK;
}

// `steps` iterations of descent on the symmetric Dirichlet energy for every
// island (after uva_batch_setup): direction -D^-1 grad (D: cotangent
// Laplacian diagonal), step = min(cap, 0.9 * flip-safe bound), halved up to
// `halvings` times until the island's energy decreases. U (b->U) is updated
// in place; e_isl (nc) receives the final energies. scratch: 8n + 7nc
// doubles + n ints.
extern "C" int uva_sd_refine(uva_batch* b, int32_t steps, int32_t halvings, double cap, double* e_isl, void* scratch,
                             void* stream) {
    if (!b || !e_isl || !scratch || steps < 0 || halvings < 0) { uva_set_error("uva_sd_refine: bad arguments"); return UVA_E_ARG; }
    if (b->nc == 0 || b->t == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = b->n, nc = b->nc;
    double* gU = static_cast<double*>(scratch);
    double* Dd = gU + 2 * static_cast<size_t>(n);
    double* Ut = Dd + 2 * static_cast<size_t>(n);
    double* tmax = Ut + 2 * static_cast<size_t>(n);
    double* alpha = tmax + nc;
    double* e_new = alpha + nc;
    int32_t* accepted = reinterpret_cast<int32_t*>(e_new + nc);
    int32_t* vert_isl = accepted + nc + (nc & 1);
    k_vert_isl2<<<nc, 256, 0, s>>>(b->vofs, nc, vert_isl);
    for (int it = 0; it < steps; ++it) {
        uva_energy_fwd(b, b->P, b->U, 1, e_isl, nullptr, s);
        uva_energy_bwd(b, b->P, b->U, 1, nullptr, gU, nullptr, s);
        k_descent_dir<<<nb(n), 256, 0, s>>>(n, *b, vert_isl, gU, Dd);
        k_fill_d<<<nb(nc), 256, 0, s>>>(tmax, nc, 1e30);
        k_island_max_step<<<nb(b->t), 256, 0, s>>>(*b, b->U, Dd, tmax);
        k_init_alpha<<<nb(nc), 256, 0, s>>>(nc, tmax, alpha, accepted, cap);
        for (int h = 0; h <= halvings; ++h) {
            k_trial<<<nb(n), 256, 0, s>>>(n, *b, b->U, Dd, alpha, vert_isl, Ut);
            uva_energy_fwd(b, b->P, Ut, 1, e_new, nullptr, s);
            k_accept<<<nb(nc), 256, 0, s>>>(nc, e_isl, e_new, alpha, accepted);
        }
        k_commit<<<nb(n), 256, 0, s>>>(n, vert_isl, accepted, Ut, b->U);
    }
    UVA_CHECK_LAUNCH("uva_sd_refine");
    return uva_energy_fwd(b, b->P, b->U, 1, e_isl, nullptr, s);
}
