// Per-chart helpers of engine/param.py on the device: one per-triangle kernel
// with an operation switch, and a generic FP64 Jacobi-PCG for a CSR SPD
// matrix (SPDSolver, param.py:103-132).
//
//   UVA_OP_FRAMES      local_frames (param.py:19-32): X (t,3,2), area (t)
//   UVA_OP_COTS        cot_weights (param.py:35-44) from X
//   UVA_OP_SIGNED_AREA signed_areas (param.py:97-99)
//   UVA_OP_ROTATIONS   _arap_rotations (param.py:206-256), mode in `arg`: R (t,2,2);
//                      mode 1 also the SLIM weight matrices W (t,2,2) in out2
//   UVA_OP_RHS         _arap_rhs (param.py:457-474): b (n,2), FP64 atomics
//   UVA_OP_MAX_STEP    _max_step (param.py:259-291): one scalar
//   UVA_OP_ENERGY      _energy (param.py:294-319), kind in `arg`: one scalar
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"

using namespace uva;

namespace {

struct ChartArgs {
    const double* P;    // n*3
    const int64_t* T;   // t*3
    const double* U;    // n*2
    const double* D;    // n*2 (max step direction)
    const double* X;    // t*6 (frames)
    const double* cots; // t*3
    const double* R;    // t*4
    const double* area; // t
    double* out;
    double* out2;
    int t, n, op, arg;
};

__device__ __forceinline__ void atomic_min_pos(double* addr, double v) {
    if (!(v >= 0.0)) return;
    atomicMin(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

__global__ void k_chart_op(ChartArgs a) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    double red = 0.0;
    bool has = false;
    if (f < a.t) {
        const int64_t i0 = a.T[3 * f], i1 = a.T[3 * f + 1], i2 = a.T[3 * f + 2];
        switch (a.op) {
            case UVA_OP_FRAMES: {
                const double* P = a.P;
                const double e1x = P[3 * i1] - P[3 * i0], e1y = P[3 * i1 + 1] - P[3 * i0 + 1], e1z = P[3 * i1 + 2] - P[3 * i0 + 2];
                const double e2x = P[3 * i2] - P[3 * i0], e2y = P[3 * i2 + 1] - P[3 * i0 + 1], e2z = P[3 * i2 + 2] - P[3 * i0 + 2];
                const double l1 = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
                const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
                const double nn = sqrt(nx * nx + ny * ny + nz * nz);
                const double il = 1.0 / fmax(l1, 1e-300), in = 1.0 / fmax(nn, 1e-300);
                const double exx = e1x * il, exy = e1y * il, exz = e1z * il;
                const double ux = nx * in, uy = ny * in, uz = nz * in;
                const double eyx = uy * exz - uz * exy, eyy = uz * exx - ux * exz, eyz = ux * exy - uy * exx;
                double* X = a.out + 6 * static_cast<size_t>(f);
                X[0] = 0.0; X[1] = 0.0; X[2] = l1; X[3] = 0.0;
                X[4] = e2x * exx + e2y * exy + e2z * exz;
                X[5] = e2x * eyx + e2y * eyy + e2z * eyz;
                a.out2[f] = 0.5 * nn;
                break;
            }
            case UVA_OP_COTS: {
                const double* X = a.X + 6 * static_cast<size_t>(f);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int i = (k + 1) % 3, j = (k + 2) % 3;
                    const double ax = X[2 * i] - X[2 * k], ay = X[2 * i + 1] - X[2 * k + 1];
                    const double bx = X[2 * j] - X[2 * k], by = X[2 * j + 1] - X[2 * k + 1];
                    const double cr = fabs(ax * by - ay * bx);
                    double c = (ax * bx + ay * by) / fmax(cr, 1e-300);
                    a.out[3 * static_cast<size_t>(f) + k] = fmin(fmax(c, -1e4), 1e4);
                }
                break;
            }
            case UVA_OP_SIGNED_AREA: {
                const double* U = a.U;
                a.out[f] = 0.5 * ((U[2 * i1] - U[2 * i0]) * (U[2 * i2 + 1] - U[2 * i0 + 1]) -
                                  (U[2 * i2] - U[2 * i0]) * (U[2 * i1 + 1] - U[2 * i0 + 1]));
                break;
            }
            case UVA_OP_ROTATIONS: {
                const double* X = a.X + 6 * static_cast<size_t>(f);
                const double* U = a.U;
                const double x1 = X[2], x2 = X[4], y2 = X[5];
                double* R = a.out + 4 * static_cast<size_t>(f);
                double* W = (a.arg == 1 && a.out2) ? a.out2 + 4 * static_cast<size_t>(f) : nullptr;
                if (W) { W[0] = 1.0; W[1] = 0.0; W[2] = 0.0; W[3] = 1.0; }
                if (fabs(x1 * y2) < 1e-300) { R[0] = 1.0; R[1] = 0.0; R[2] = 0.0; R[3] = 1.0; break; }
                const double du1x = U[2 * i1] - U[2 * i0], du1y = U[2 * i1 + 1] - U[2 * i0 + 1];
                const double du2x = U[2 * i2] - U[2 * i0], du2y = U[2 * i2 + 1] - U[2 * i0 + 1];
                const double j00 = du1x / x1, j10 = du1y / x1;
                const double j01 = (du2x - j00 * x2) / y2, j11 = (du2y - j10 * x2) / y2;
                if (W) {   // SVD-based rotation and SLIM weights (param.py:234-255)
                    double rc, rs, w00, w01, w11;
                    slim_2x2(j00, j01, j10, j11, rc, rs, w00, w01, w11);
                    R[0] = rc; R[1] = -rs; R[2] = rs; R[3] = rc;
                    W[0] = w00; W[1] = w01; W[2] = w01; W[3] = w11;
                    break;
                }
                double ca = j00 + j11, cb = j10 - j01;
                double h = sqrt(ca * ca + cb * cb);
                if (h < 1e-300) { ca = 1.0; cb = 0.0; h = 1.0; }
                R[0] = ca / h; R[1] = -cb / h; R[2] = cb / h; R[3] = ca / h;
                break;
            }
            case UVA_OP_RHS: {
                const double* X = a.X + 6 * static_cast<size_t>(f);
                const double* R = a.R + 4 * static_cast<size_t>(f);
                const int64_t tv[3] = {i0, i1, i2};
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int ii = (k + 1) % 3, jj = (k + 2) % 3;
                    const double w = 0.5 * a.cots[3 * static_cast<size_t>(f) + k];
                    const double dx0 = X[2 * ii] - X[2 * jj], dx1 = X[2 * ii + 1] - X[2 * jj + 1];
                    const double rx = R[0] * dx0 + R[1] * dx1, ry = R[2] * dx0 + R[3] * dx1;
                    atomicAdd(a.out + 2 * tv[ii], w * rx); atomicAdd(a.out + 2 * tv[ii] + 1, w * ry);
                    atomicAdd(a.out + 2 * tv[jj], -w * rx); atomicAdd(a.out + 2 * tv[jj] + 1, -w * ry);
                }
                break;
            }
            case UVA_OP_MAX_STEP: {
                const double* U = a.U;
                const double* D = a.D;
                const double ux1 = U[2 * i1] - U[2 * i0], uy1 = U[2 * i1 + 1] - U[2 * i0 + 1];
                const double ux2 = U[2 * i2] - U[2 * i0], uy2 = U[2 * i2 + 1] - U[2 * i0 + 1];
                const double dx1 = D[2 * i1] - D[2 * i0], dy1 = D[2 * i1 + 1] - D[2 * i0 + 1];
                const double dx2 = D[2 * i2] - D[2 * i0], dy2 = D[2 * i2 + 1] - D[2 * i0 + 1];
                const double C = ux1 * uy2 - ux2 * uy1;
                const double B = ux1 * dy2 + dx1 * uy2 - ux2 * dy1 - dx2 * uy1;
                const double A = dx1 * dy2 - dx2 * dy1;
                double t = 1e30;
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
                red = t; has = true;
                break;
            }
            case UVA_OP_ENERGY: {
                const double* X = a.X + 6 * static_cast<size_t>(f);
                const double* U = a.U;
                const double x1 = X[2], x2 = X[4], y2 = X[5];
                if (fabs(x1 * y2) < 1e-300) break;
                const double j00 = (U[2 * i1] - U[2 * i0]) / x1, j10 = (U[2 * i1 + 1] - U[2 * i0 + 1]) / x1;
                const double j01 = ((U[2 * i2] - U[2 * i0]) - j00 * x2) / y2;
                const double j11 = ((U[2 * i2 + 1] - U[2 * i0 + 1]) - j10 * x2) / y2;
                if (a.arg == 0) {
                    const double qe = 0.5 * (j00 + j11), qh = 0.5 * (j10 - j01);
                    const double rf = 0.5 * (j00 - j11), rg = 0.5 * (j10 + j01);
                    const double q = sqrt(qe * qe + qh * qh), r = sqrt(rf * rf + rg * rg);
                    red = a.area[f] * ((q + r - 1.0) * (q + r - 1.0) + (q - r - 1.0) * (q - r - 1.0));
                } else {
                    const double dj = j00 * j11 - j01 * j10;
                    if (dj <= 0.0) { red = INFINITY; }
                    else {
                        const double fro = j00 * j00 + j01 * j01 + j10 * j10 + j11 * j11;
                        red = a.area[f] * (fro + fro / (dj * dj) - 4.0);
                    }
                }
                has = true;
                break;
            }
            default: break;
        }
    }
    if (a.op == UVA_OP_MAX_STEP) {
        double v = has ? red : 1e30;
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0) atomic_min_pos(a.out, v);
    } else if (a.op == UVA_OP_ENERGY) {
        double v = has ? red : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(a.out, v);
    }
}

__global__ void k_fill(double* p, double v) { *p = v; }

constexpr int kPcgNT = 1024;
constexpr size_t kPcgRowBytes = 5 * sizeof(double) + sizeof(int32_t);
constexpr size_t kPcgSmem = 220 * 1024;
constexpr int kPcgCap = static_cast<int>((kPcgSmem - 2 * sizeof(int32_t)) / kPcgRowBytes);

template <int NT>
__device__ void pcg_block_smem(int r0, int n, const int32_t* rp, const int32_t* ci, const double* val,
                               const double* b, double* x, double tol, int maxiter, int32_t* it_out, double* red,
                               double* dsm, int cap) {
    int phase = 0;
    double* X = dsm;
    double* R = X + cap;
    double* P = R + cap;
    double* Q = P + cap;
    double* D = Q + cap;
    int32_t* RP = reinterpret_cast<int32_t*>(D + cap);   // n + 1 row starts, relative to the block's first entry
    const int32_t e0 = rp[r0];
    for (int i = threadIdx.x; i <= n; i += NT) RP[i] = rp[r0 + i] - e0;
    ci += e0;
    val += e0;
    for (int i = threadIdx.x; i < n; i += NT) {
        X[i] = x[r0 + i];
        double d = 0.0;
        for (int k = rp[r0 + i] - e0; k < rp[r0 + i + 1] - e0; ++k)
            if (ci[k] == r0 + i) d += val[k];
        D[i] = 1.0 / (fabs(d) > 1e-300 ? d : 1.0);
    }
    __syncthreads();
    double acc[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += NT) {
        double ax = 0.0;
        for (int k = RP[i]; k < RP[i + 1]; ++k) ax += val[k] * X[ci[k] - r0];
        const double bi = b[r0 + i];
        const double ri = bi - ax;
        R[i] = ri;
        P[i] = ri * D[i];
        acc[0] += ri * P[i];
        acc[1] += bi * bi;
    }
    block_sum<NT, 2>(acc, red, phase);   // also publishes P
    double rz = acc[0];
    const double bb = fmax(acc[1], 1e-300);
    int it = 0;
    for (; it < maxiter; ++it) {
        double pq[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            double sacc = 0.0;
            for (int k = RP[i]; k < RP[i + 1]; ++k) sacc += val[k] * P[ci[k] - r0];
            Q[i] = sacc;
            pq[0] += P[i] * sacc;
        }
        block_sum<NT, 1>(pq, red, phase);
        if (!(pq[0] > 0.0)) break;
        const double alpha = rz / pq[0];
        double nz[2] = {0.0, 0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            X[i] += alpha * P[i];
            const double ri = R[i] - alpha * Q[i];
            R[i] = ri;
            nz[0] += ri * ri * D[i];
            nz[1] += ri * ri;
        }
        block_sum<NT, 2>(nz, red, phase);
        if (nz[1] <= tol * tol * bb) { ++it; break; }
        const double beta = nz[0] / rz;
        rz = nz[0];
        for (int i = threadIdx.x; i < n; i += NT) P[i] = R[i] * D[i] + beta * P[i];
        __syncthreads();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += NT) x[r0 + i] = X[i];
    if (threadIdx.x == 0) *it_out = it;
}

// ---- FP64 Jacobi-PCG for one CSR SPD matrix, ncol right-hand sides, one CTA
// per column (param.py:119-132 with the SuperLU branch replaced by PCG to a
// tight tolerance); matrices of at most `cap` rows iterate in shared memory.
template <int NT>
__global__ void __launch_bounds__(NT) k_csr_pcg(int n, const int32_t* rp, const int32_t* ci, const double* val,
                                                const double* b, double* x, double* r, double* p, double* q,
                                                int ncol, double tol, int maxiter, int32_t* iters_out, int cap) {
    __shared__ double red[2 * 4 * (NT / 32)];
    extern __shared__ double dsm[];
    int phase = 0;
    const int c = blockIdx.x;
    if (c >= ncol) return;
    const double* bc = b + static_cast<size_t>(c) * n;
    double* xc = x + static_cast<size_t>(c) * n;
    if (n <= cap) {
        pcg_block_smem<NT>(0, n, rp, ci, val, bc, xc, tol, maxiter, iters_out + c, red, dsm, cap);
        return;
    }
    double* rc = r + static_cast<size_t>(c) * n;
    double* pc = p + static_cast<size_t>(c) * n;
    double* qc = q + static_cast<size_t>(c) * n;
    auto diag = [&](int i) {
        double d = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) d += val[k];
        return fabs(d) > 1e-300 ? d : 1.0;
    };
    double acc[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += NT) {
        double ax = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) ax += val[k] * xc[ci[k]];
        const double ri = bc[i] - ax;
        rc[i] = ri;
        pc[i] = ri / diag(i);
        acc[0] += ri * pc[i];
        acc[1] += bc[i] * bc[i];
    }
    block_sum<NT, 2>(acc, red, phase);
    double rz = acc[0];
    const double bb = fmax(acc[1], 1e-300);
    int it = 0;
    for (; it < maxiter; ++it) {
        double pq[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            double s = 0.0;
            for (int k = rp[i]; k < rp[i + 1]; ++k) s += val[k] * pc[ci[k]];
            qc[i] = s;
            pq[0] += pc[i] * s;
        }
        block_sum<NT, 1>(pq, red, phase);
        if (!(pq[0] > 0.0)) break;
        const double alpha = rz / pq[0];
        double nz[2] = {0.0, 0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            xc[i] += alpha * pc[i];
            rc[i] -= alpha * qc[i];
            const double z = rc[i] / diag(i);
            nz[0] += rc[i] * z;
            nz[1] += rc[i] * rc[i];
        }
        block_sum<NT, 2>(nz, red, phase);
        if (nz[1] <= tol * tol * bb) { ++it; break; }
        const double beta = nz[0] / rz;
        rz = nz[0];
        for (int i = threadIdx.x; i < n; i += NT) pc[i] = rc[i] / diag(i) + beta * pc[i];
        __syncthreads();
    }
    if (threadIdx.x == 0) iters_out[c] = it;
}

// ---- the same PCG on a block-diagonal CSR matrix, one CTA per diagonal
// block: block s owns rows [so[s], so[s+1]) and its columns lie in the same
// range; it stops at ||r_s|| <= tol ||b_s||. A block of at most `cap` rows
// keeps its iterate, residual, direction, product, inverse diagonal and
// row pointers in shared memory (kPcgRowBytes per row), so each iteration
// reads only its matrix entries from L2 and gathers from shared memory;
// larger blocks run the same iteration on the global scratch, the diagonal
// re-read from the row.
template <int NT>
__global__ void __launch_bounds__(NT) k_csr_pcg_blocks(int nsys, const int32_t* so, const int32_t* rp,
                                                       const int32_t* ci, const double* val, const double* b,
                                                       double* x, double* r, double* p, double* q, double tol,
                                                       int maxiter, int32_t* iters_out, int cap) {
    __shared__ double red[2 * 4 * (NT / 32)];
    extern __shared__ double dsm[];
    int phase = 0;
    const int c = blockIdx.x;
    if (c >= nsys) return;
    const int r0 = so[c], r1 = so[c + 1];
    if (r1 - r0 <= cap) {
        pcg_block_smem<NT>(r0, r1 - r0, rp, ci, val, b, x, tol, maxiter, iters_out + c, red, dsm, cap);
        return;
    }
    auto diag = [&](int i) {
        double d = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) d += val[k];
        return fabs(d) > 1e-300 ? d : 1.0;
    };
    double acc[2] = {0.0, 0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += NT) {
        double ax = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) ax += val[k] * x[ci[k]];
        const double ri = b[i] - ax;
        r[i] = ri;
        p[i] = ri / diag(i);
        acc[0] += ri * p[i];
        acc[1] += b[i] * b[i];
    }
    block_sum<NT, 2>(acc, red, phase);
    double rz = acc[0];
    const double bb = fmax(acc[1], 1e-300);
    int it = 0;
    for (; it < maxiter; ++it) {
        double pq[1] = {0.0};
        for (int i = r0 + threadIdx.x; i < r1; i += NT) {
            double s = 0.0;
            for (int k = rp[i]; k < rp[i + 1]; ++k) s += val[k] * p[ci[k]];
            q[i] = s;
            pq[0] += p[i] * s;
        }
        block_sum<NT, 1>(pq, red, phase);
        if (!(pq[0] > 0.0)) break;
        const double alpha = rz / pq[0];
        double nz[2] = {0.0, 0.0};
        for (int i = r0 + threadIdx.x; i < r1; i += NT) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            const double z = r[i] / diag(i);
            nz[0] += r[i] * z;
            nz[1] += r[i] * r[i];
        }
        block_sum<NT, 2>(nz, red, phase);
        if (nz[1] <= tol * tol * bb) { ++it; break; }
        const double beta = nz[0] / rz;
        rz = nz[0];
        for (int i = r0 + threadIdx.x; i < r1; i += NT) p[i] = r[i] / diag(i) + beta * p[i];
        __syncthreads();
    }
    if (threadIdx.x == 0) iters_out[c] = it;
}

}  // namespace

extern "C" int uva_chart_op(int32_t op, int32_t arg, const double* P, const int64_t* T, const double* U,
                            const double* D, const double* X, const double* cots, const double* R, const double* area,
                            int32_t n, int32_t t, double* out, double* out2, void* stream) {
    if (t < 0 || n < 0 || !T || !out || op < 0 || op > UVA_OP_ENERGY) { uva_set_error("uva_chart_op: bad arguments"); return UVA_E_ARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ChartArgs a{P, T, U, D, X, cots, R, area, out, out2, t, n, op, arg};
    if (op == UVA_OP_RHS) cudaMemsetAsync(out, 0, sizeof(double) * 2 * static_cast<size_t>(n), s);
    if (op == UVA_OP_MAX_STEP) k_fill<<<1, 1, 0, s>>>(out, 1e30);
    if (op == UVA_OP_ENERGY) cudaMemsetAsync(out, 0, sizeof(double), s);
    if (t > 0) k_chart_op<<<(t + 255) / 256, 256, 0, s>>>(a);
    UVA_CHECK_LAUNCH("uva_chart_op");
    return UVA_OK;
}

extern "C" int uva_csr_pcg_blocks(int32_t nsys, const int32_t* sys_ofs, int32_t n, const int32_t* rowptr,
                                  const int32_t* col, const double* val, const double* b, double* x, double tol,
                                  int32_t maxiter, double* scratch, int32_t* iters, void* stream) {
    if (nsys < 0 || n < 0 || (nsys > 0 && (!sys_ofs || !rowptr || !b || !x || !scratch || !iters))) {
        uva_set_error("uva_csr_pcg_blocks: bad arguments");
        return UVA_E_ARG;
    }
    if (nsys == 0 || n == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t N = static_cast<size_t>(n);
    const cudaError_t e = cudaFuncSetAttribute(k_csr_pcg_blocks<kPcgNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(kPcgSmem));
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_csr_pcg_blocks/cudaFuncSetAttribute");
    k_csr_pcg_blocks<kPcgNT><<<nsys, kPcgNT, kPcgSmem, s>>>(nsys, sys_ofs, rowptr, col, val, b, x, scratch,
                                                           scratch + N, scratch + 2 * N, tol, maxiter, iters, kPcgCap);
    UVA_CHECK_LAUNCH("uva_csr_pcg_blocks");
    return UVA_OK;
}

extern "C" int uva_csr_pcg(int32_t n, const int32_t* rowptr, const int32_t* col, const double* val, const double* b,
                           double* x, int32_t ncol, double tol, int32_t maxiter, double* scratch, int32_t* iters,
                           void* stream) {
    if (n < 0 || ncol < 1 || !rowptr || !b || !x || !scratch || !iters) { uva_set_error("uva_csr_pcg: bad arguments"); return UVA_E_ARG; }
    if (n == 0) return UVA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t N = static_cast<size_t>(n) * ncol;
    const cudaError_t e = cudaFuncSetAttribute(k_csr_pcg<kPcgNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(kPcgSmem));
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_csr_pcg/cudaFuncSetAttribute");
    k_csr_pcg<kPcgNT><<<ncol, kPcgNT, kPcgSmem, s>>>(n, rowptr, col, val, b, x, scratch, scratch + N, scratch + 2 * N,
                                                    ncol, tol, maxiter, iters, kPcgCap);
    UVA_CHECK_LAUNCH("uva_csr_pcg");
    return UVA_OK;
}
