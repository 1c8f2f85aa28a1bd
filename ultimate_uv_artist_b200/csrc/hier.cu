// hier.Solver.lscm on the device (engine/hier.py:534-585): the soft-pinned
// LSCM system of every chart assembled from the faces and solved per chart
// by FP64 Jacobi-PCG, one CTA per chart.
//
// The system (2 nv unknowns: u then v of each UV vertex) is the reference's
// COO sum: per face edge e = (corner e+1, corner e+2) with half-cot weight
// w_e, (i,j) -= w, (j,i) -= w, (i,i) += w, (j,j) += w in the u and in the v
// block; per directed boundary edge (a, b), (a_u, b_v) -= 1/2,
// (b_u, a_v) += 1/2, (a_v, b_u) += 1/2, (b_v, a_u) -= 1/2; per chart two
// pins (the boundary vertices of smallest and largest initial u, compared in
// float32, the smallest vertex id on ties) with diagonal weight
// wpin = 10 max(max |w|, 1e-12) and right-hand side wpin U0. Only UV
// vertices that a face names have unknowns; the others keep U0.
//
// Layout: the UV vertices grouped by chart (a stable radix sort by chart, so
// by id inside a chart); vertex slot = position in that list. The u row and
// the v row of a vertex share their Laplacian entries, so each vertex keeps
// one row: the diagonal, then its neighbours in first-seen order (corners in
// face order, duplicates summed in that order), then its boundary couplings
// (edge order; value c for the u row against the neighbour's v, -c for the
// v row against its u). A chart whose vectors and rows fit in shared memory
// (about 165 B per vertex) iterates there; larger charts run the same
// iteration on global scratch.
//
// Steps (one stream, no host round trip):
//   k_hl_faces   half-cot weights per face (engine/hier.py:362-382 restated),
//                max |w|, the last face naming each UV vertex, corner counts
//   k_hl_vchart  chart of each vertex (the last naming face's), chart sizes
//   k_hl_check   consistency (a face's corners and a boundary edge's ends in
//                one chart) and the pins' keys (atomic minima of 64-bit
//                (ordered key, vertex) words)
//   radix sorts  vertices by chart, corners by vertex, boundary ends by vertex
//   k_hl_slot    vertex slots; k_hl_lap<false> (row lengths), scans,
//                k_hl_lap<true> (rows, diagonal, right-hand side, start)
//   k_hl_pcg     the per-chart PCG; k_hl_out: U (nv, 2), U0 where not finite.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "scan.cuh"

using namespace uva;

namespace {

constexpr int kTB = 256;
constexpr uint64_t kNoPin = ~0ull;

unsigned blocks_for(int64_t n) { return static_cast<unsigned>(std::max<int64_t>(1, (n + kTB - 1) / kTB)); }

int bits_for(int64_t maxval) {   // bits holding 0..maxval
    int b = 1;
    while (b < 62 && (int64_t{1} << b) <= maxval) ++b;
    return b;
}

struct HlArgs {
    const double* V;       // mesh positions (nvp, 3)
    const int32_t* F;      // mesh faces (nf, 3)
    const int32_t* faces;  // (t) rows of F
    const int32_t* CV;     // (t, 3) UV vertices of the face corners
    const int32_t* chart;  // (t)
    const double* U0;      // (nv, 2)
    const int32_t* ba;     // (nb) directed boundary edges a -> b
    const int32_t* bb;
    int64_t nvp, nf, t, nv, nb;
    int32_t nchart;
};

// Scratch of one call, carved from one buffer (256-byte aligned pieces).
struct HlScratch {
    int32_t *lastf, *cv, *ccnt, *cofs, *npin, *vcnt, *vofs, *bcnt, *bofs, *slot, *llen, *lrow, *lcol, *clen, *cptr,
        *ccol, *its, *err, *isums;
    uint32_t *vkey, *vkey_s, *vval, *vval_s, *ckey, *ckey_s, *cval, *cval_s, *bkey, *bkey_s, *bval, *bval_s;
    double *w, *lval, *cpl, *dg, *bu, *bv, *xu, *xv, *gvec;
    uint64_t *wmax, *pmin, *pmax;
    void* cub;
    size_t cub_bytes;
};

size_t cub_temp(int64_t n, int end_bit) {
    size_t bytes = 0;
    if (n > 0)
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, static_cast<const uint32_t*>(nullptr),
                                        static_cast<uint32_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
                                        static_cast<uint32_t*>(nullptr), static_cast<int>(n), 0, end_bit);
    return bytes;
}

// Lays the scratch out at `base` (nullptr: sizes only); returns the bytes.
size_t hl_layout(const HlArgs& a, char* base, HlScratch* s) {
    size_t off = 0;
    auto take = [&](size_t bytes) -> char* {
        char* p = base ? base + off : nullptr;
        off += (bytes + 255) & ~static_cast<size_t>(255);
        return p;
    };
    const int64_t nv = a.nv, t = a.t, nb = a.nb, nc = a.nchart;
    HlScratch z{};
    HlScratch& r = s ? *s : z;
    auto i32 = [&](int64_t n) { return reinterpret_cast<int32_t*>(take(4 * n)); };
    auto u32 = [&](int64_t n) { return reinterpret_cast<uint32_t*>(take(4 * n)); };
    auto f64 = [&](int64_t n) { return reinterpret_cast<double*>(take(8 * n)); };
    r.lastf = i32(nv); r.cv = i32(nv); r.ccnt = i32(nc + 1); r.cofs = i32(nc + 1); r.npin = i32(nv);
    r.vcnt = i32(nv + 1); r.vofs = i32(nv + 1); r.bcnt = i32(nv + 1); r.bofs = i32(nv + 1); r.slot = i32(nv);
    r.llen = i32(nv + 1); r.lrow = i32(nv + 1); r.lcol = i32(6 * t); r.clen = i32(nv + 1); r.cptr = i32(nv + 1);
    r.ccol = i32(2 * nb); r.its = i32(std::max<int64_t>(nc, 1)); r.err = i32(1);
    r.isums = i32(xscan_sums(std::max(nv, nc) + 1) + 1);
    r.vkey = u32(nv); r.vkey_s = u32(nv); r.vval = u32(nv); r.vval_s = u32(nv);
    r.ckey = u32(3 * t); r.ckey_s = u32(3 * t); r.cval = u32(3 * t); r.cval_s = u32(3 * t);
    r.bkey = u32(2 * nb); r.bkey_s = u32(2 * nb); r.bval = u32(2 * nb); r.bval_s = u32(2 * nb);
    r.w = f64(3 * t); r.lval = f64(6 * t); r.cpl = f64(2 * nb); r.dg = f64(nv); r.bu = f64(nv); r.bv = f64(nv);
    r.xu = f64(nv); r.xv = f64(nv); r.gvec = f64(6 * nv);
    r.wmax = reinterpret_cast<uint64_t*>(take(8));
    r.pmin = reinterpret_cast<uint64_t*>(take(8 * std::max<int64_t>(nc, 1)));
    r.pmax = reinterpret_cast<uint64_t*>(take(8 * std::max<int64_t>(nc, 1)));
    r.cub_bytes = std::max({cub_temp(nv, bits_for(nc)), cub_temp(3 * t, bits_for(nv)), cub_temp(2 * nb, bits_for(nv))});
    r.cub = take(std::max<size_t>(r.cub_bytes, 16));
    return off;
}

__device__ __forceinline__ void flag(int32_t* err, int bit) { atomicOr(err, bit); }

// Half-cot weights of one mesh face (engine/hier.py:362-382): the face in
// its own frame, corners (0,0), (l1,0), (e2.ex, e2.ey); 0 for faces too thin
// for a frame; cotangents clipped to [-1e4, 1e4] (NaN kept, like np.clip).
__device__ void face_cots(const double* V, const int32_t* Fr, double w[3]) {
    const double* p0 = V + 3 * static_cast<int64_t>(Fr[0]);
    const double* p1 = V + 3 * static_cast<int64_t>(Fr[1]);
    const double* p2 = V + 3 * static_cast<int64_t>(Fr[2]);
    const double e1x = p1[0] - p0[0], e1y = p1[1] - p0[1], e1z = p1[2] - p0[2];
    const double e2x = p2[0] - p0[0], e2y = p2[1] - p0[1], e2z = p2[2] - p0[2];
    const double l1 = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
    const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const double dbl = sqrt(nx * nx + ny * ny + nz * nz);
    const bool ok = dbl > 1e-14 * fmax(l1 * l1, 1e-300) && isfinite(dbl) && l1 > 0.0;
    w[0] = w[1] = w[2] = 0.0;
    if (!ok) return;
    const double ld = fmax(l1, 1e-30), dd = fmax(dbl, 1e-30);
    const double exx = e1x / ld, exy = e1y / ld, exz = e1z / ld;
    const double mx = nx / dd, my = ny / dd, mz = nz / dd;
    const double eyx = my * exz - mz * exy, eyy = mz * exx - mx * exz, eyz = mx * exy - my * exx;
    const double X[3][2] = {{0.0, 0.0}, {l1, 0.0}, {e2x * exx + e2y * exy + e2z * exz, e2x * eyx + e2y * eyy + e2z * eyz}};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int i = (k + 1) % 3, j = (k + 2) % 3;
        const double ax = X[i][0] - X[k][0], ay = X[i][1] - X[k][1];
        const double bx = X[j][0] - X[k][0], by = X[j][1] - X[k][1];
        const double cr = fmax(fabs(ax * by - ay * bx), 1e-30);
        double c = (ax * bx + ay * by) / cr;
        c = c < -1e4 ? -1e4 : (c > 1e4 ? 1e4 : c);
        w[k] = 0.5 * c;
    }
}

__global__ void k_hl_faces(HlArgs a, HlScratch s) {
    const int64_t f = static_cast<int64_t>(blockIdx.x) * kTB + threadIdx.x;
    uint64_t wm = 0;
    if (f < a.t) {
        double w[3] = {0.0, 0.0, 0.0};
        const int32_t fid = a.faces[f];
        if (fid < 0 || fid >= a.nf) {
            flag(s.err, 2);
        } else {
            const int32_t* Fr = a.F + 3 * static_cast<int64_t>(fid);
            if (Fr[0] < 0 || Fr[0] >= a.nvp || Fr[1] < 0 || Fr[1] >= a.nvp || Fr[2] < 0 || Fr[2] >= a.nvp)
                flag(s.err, 2);
            else
                face_cots(a.V, Fr, w);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            s.w[3 * f + k] = w[k];
            const uint64_t bits = static_cast<uint64_t>(__double_as_longlong(fabs(w[k])));
            wm = bits > wm ? bits : wm;   // |w| >= 0: the bit patterns order like the values, NaN above all
            const int32_t c = a.CV[3 * f + k];
            if (c < 0 || c >= a.nv) {
                flag(s.err, 2);
                s.ckey[3 * f + k] = static_cast<uint32_t>(a.nv);   // sorts after every vertex
            } else {
                atomicMax(s.lastf + c, static_cast<int32_t>(f));
                atomicAdd(s.vcnt + c, 1);
                s.ckey[3 * f + k] = static_cast<uint32_t>(c);
            }
            s.cval[3 * f + k] = static_cast<uint32_t>(3 * f + k);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t y = __shfl_xor_sync(0xffffffffu, wm, o);
        wm = y > wm ? y : wm;
    }
    if ((threadIdx.x & 31) == 0 && wm) atomicMax(reinterpret_cast<unsigned long long*>(s.wmax), wm);
}

__global__ void k_hl_vchart(HlArgs a, HlScratch s) {
    const int64_t v = static_cast<int64_t>(blockIdx.x) * kTB + threadIdx.x;
    if (v >= a.nv) return;
    const int32_t lf = s.lastf[v];
    int32_t c = -1;
    if (lf >= 0) {
        c = a.chart[lf];
        if (c < 0 || c >= a.nchart) {
            flag(s.err, 4);
            c = -1;
        }
    }
    s.cv[v] = c;
    s.vkey[v] = static_cast<uint32_t>(c >= 0 ? c : a.nchart);
    s.vval[v] = static_cast<uint32_t>(v);
    if (c >= 0) atomicAdd(s.ccnt + c, 1);
}

// float32 key of a pin candidate as an unsigned word in the order of the
// values (-0 and +0 equal); NaN gets `nan_word`.
__device__ __forceinline__ uint32_t key_word(double u, uint32_t nan_word) {
    float k = __double2float_rn(u);
    if (isnan(k)) return nan_word;
    if (k == 0.0f) k = 0.0f;
    const uint32_t b = __float_as_uint(k);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void k_hl_check(HlArgs a, HlScratch s) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kTB + threadIdx.x;
    if (i < a.t) {   // a face's corners in one chart (else the system couples two charts)
        const int32_t c0 = a.CV[3 * i], c1 = a.CV[3 * i + 1], c2 = a.CV[3 * i + 2];
        if (c0 >= 0 && c0 < a.nv && c1 >= 0 && c1 < a.nv && c2 >= 0 && c2 < a.nv) {
            const int32_t k0 = s.cv[c0], k1 = s.cv[c1], k2 = s.cv[c2];
            if (k0 != k1 || k1 != k2) flag(s.err, 1);
        }
        return;
    }
    const int64_t e = i - a.t;
    if (e >= a.nb) return;
    const int32_t u = a.ba[e], v = a.bb[e];
    const bool uok = u >= 0 && u < a.nv, vok = v >= 0 && v < a.nv;
    if (!uok || !vok) flag(s.err, 2);
    s.bkey[e] = static_cast<uint32_t>(uok ? u : a.nv);
    s.bkey[a.nb + e] = static_cast<uint32_t>(vok ? v : a.nv);
    s.bval[e] = static_cast<uint32_t>(e);
    s.bval[a.nb + e] = static_cast<uint32_t>(a.nb + e);
    if (uok) atomicAdd(s.bcnt + u, 1);
    if (vok) atomicAdd(s.bcnt + v, 1);
    if (!uok || !vok) return;
    const int32_t cu = s.cv[u], cvv = s.cv[v];
    if (cu >= 0 && cvv >= 0 && cu != cvv) flag(s.err, 1);
    if (cu < 0) return;
    // pins: smallest key first, then smallest vertex; largest key first (NaN
    // last), then smallest vertex
    const double u0 = a.U0[2 * static_cast<int64_t>(u)];
    const uint64_t lo = static_cast<uint64_t>(static_cast<uint32_t>(u));
    atomicMin(reinterpret_cast<unsigned long long*>(s.pmin + cu),
              (static_cast<uint64_t>(key_word(u0, 0xFFFFFFFFu)) << 32) | lo);
    atomicMin(reinterpret_cast<unsigned long long*>(s.pmax + cu),
              (static_cast<uint64_t>(0xFFFFFFFFu - key_word(u0, 0u)) << 32) | lo);
}

__global__ void k_hl_pins(HlArgs a, HlScratch s) {
    const int64_t c = static_cast<int64_t>(blockIdx.x) * kTB + threadIdx.x;
    if (c >= a.nchart) return;
    if (s.pmin[c] != kNoPin) atomicAdd(s.npin + static_cast<uint32_t>(s.pmin[c]), 1);
    if (s.pmax[c] != kNoPin) atomicAdd(s.npin + static_cast<uint32_t>(s.pmax[c]), 1);
}

// Slot of every UV vertex: its position in the chart-sorted vertex list
// (chart c owns slots [cofs[c], cofs[c+1])), -1 for vertices no face names.
__global__ void k_hl_slot(HlArgs a, HlScratch s) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kTB + threadIdx.x;
    if (i >= a.nv) return;
    const uint32_t c = s.vkey_s[i], v = s.vval_s[i];
    s.slot[v] = c < static_cast<uint32_t>(a.nchart) ? static_cast<int32_t>(i) : -1;
}

// Laplacian candidate j of a vertex: corner p = first + j / 2 of the vertex
// lies on edge (k+2)%3 (to corner k+1, side 0) and edge (k+1)%3 (to corner
// k+2, side 1).
struct Cand {
    int32_t nb;
    double w;
};

__device__ __forceinline__ Cand lap_cand(const HlArgs& a, const HlScratch& s, int32_t first, int32_t j) {
    const uint32_t cj = s.cval_s[first + (j >> 1)];
    const int64_t f = cj / 3;
    const int k = static_cast<int>(cj - 3 * f);
    const int h = j & 1;
    return Cand{a.CV[3 * f + (h == 0 ? (k + 1) % 3 : (k + 2) % 3)], s.w[3 * f + (h == 0 ? (k + 2) % 3 : (k + 1) % 3)]};
}

// One row per used vertex: FILL false counts the distinct same-chart
// neighbours and the couplings, FILL true writes them with the diagonal,
// the right-hand side and the start. Degenerate faces' self edges fold into
// the diagonal (so the Jacobi diagonal equals the matrix's).
constexpr int kCandBuf = 24;

template <bool FILL>
__global__ void k_hl_lap(HlArgs a, HlScratch s) {
    const int64_t v = static_cast<int64_t>(blockIdx.x) * kTB + threadIdx.x;
    if (v >= a.nv) return;
    const int32_t sl = s.slot[v];
    if (sl < 0) return;
    const int32_t c = s.cv[v], base = s.cofs[c];
    const int32_t first = s.vofs[v], m = 2 * s.vcnt[v];
    Cand buf[kCandBuf];
    const bool cached = m <= kCandBuf;
    if (cached)
        for (int32_t j = 0; j < m; ++j) buf[j] = lap_cand(a, s, first, j);
    auto cand = [&](int32_t j) { return cached ? buf[j] : lap_cand(a, s, first, j); };
    int32_t ko = FILL ? s.lrow[sl] : 0, len = 0;
    double d = 0.0, dself = 0.0;
    for (int32_t j = 0; j < m; ++j) {
        const Cand cj = cand(j);
        d += cj.w;
        if (cj.nb < 0 || cj.nb >= a.nv || s.cv[cj.nb] != c) continue;
        bool dup = false;
        for (int32_t i = 0; i < j && !dup; ++i) dup = cand(i).nb == cj.nb;
        if (dup) continue;   // summed at its first occurrence
        double sum = cj.w;
        for (int32_t i = j + 1; i < m; ++i) {
            const Cand ci = cand(i);
            if (ci.nb == cj.nb) sum += ci.w;
        }
        if (cj.nb == v) {
            dself -= sum;
            continue;
        }
        ++len;
        if (FILL) {
            s.lcol[ko] = s.slot[cj.nb] - base;
            s.lval[ko++] = -sum;
        }
    }
    int32_t kc = FILL ? s.cptr[sl] : 0, clen = 0;
    const int32_t b0 = s.bofs[v], b1 = b0 + s.bcnt[v];
    for (int32_t p = b0; p < b1; ++p) {
        const uint32_t j = s.bval_s[p];
        const bool is_a = j < static_cast<uint32_t>(a.nb);   // v is the edge's start
        const int64_t e = is_a ? j : j - a.nb;
        const int32_t o = is_a ? a.bb[e] : a.ba[e];
        if (o < 0 || o >= a.nv || s.cv[o] != c) continue;
        ++clen;
        if (FILL) {
            s.ccol[kc] = s.slot[o] - base;
            s.cpl[kc++] = is_a ? -0.5 : 0.5;   // u row against o's v; the v row takes the opposite sign against o's u
        }
    }
    if (!FILL) {
        s.llen[sl] = len;
        s.clen[sl] = clen;
        return;
    }
    const double wm = __longlong_as_double(static_cast<long long>(*s.wmax));
    const double wpin = 10.0 * (isnan(wm) ? wm : (wm > 1e-12 ? wm : 1e-12));
    const int np = s.npin[v];
    const double ux = a.U0[2 * v], uy = a.U0[2 * v + 1];
    double bx = 0.0, by = 0.0;
    for (int q = 0; q < np; ++q) {
        d += wpin;
        bx += wpin * ux;
        by += wpin * uy;
    }
    s.dg[sl] = d + dself;
    s.bu[sl] = bx; s.bv[sl] = by;
    s.xu[sl] = ux; s.xv[sl] = uy;
}

// ---- per-chart Jacobi-PCG on the paired rows, one CTA per chart. Shared
// memory, when the chart fits: 9 vectors (x, r, p, q for u and v, the
// diagonal) and the rows (starts relative to the chart's first entry, local
// columns); otherwise the vectors live in global scratch and the rows are
// read in place (absolute starts).
constexpr int kHlNT = 1024;
constexpr size_t kHlSmem = 220 * 1024;

template <int NT>
__global__ void __launch_bounds__(NT) k_hl_pcg(HlArgs a, HlScratch s, double tol, int maxiter) {
    __shared__ double red[2 * 4 * (NT / 32)];
    extern __shared__ double dsm[];
    int phase = 0;
    const int c = blockIdx.x;
    if (c >= a.nchart) return;
    const int32_t s0 = s.cofs[c], n = s.cofs[c + 1] - s0;
    const int32_t e0 = s.lrow[s0], ne = s.lrow[s0 + n] - e0;
    const int32_t f0 = s.cptr[s0], nf = s.cptr[s0 + n] - f0;
    const size_t need = 8 * (9 * static_cast<size_t>(n) + ne + nf) + 4 * (2 * (static_cast<size_t>(n) + 1) + ne + nf);
    const bool fit = need <= kHlSmem;
    double *xu, *xv, *ru, *rv, *pu, *pv, *qu, *qv, *dg;
    const int32_t *lr, *lc, *cr, *cc;
    const double *lv, *cp;
    if (fit) {
        double* p = dsm;
        xu = p; p += n; xv = p; p += n; ru = p; p += n; rv = p; p += n; pu = p; p += n; pv = p; p += n;
        qu = p; p += n; qv = p; p += n; dg = p; p += n;
        double* lvs = p; p += ne;
        double* cps = p; p += nf;
        int32_t* ip = reinterpret_cast<int32_t*>(p);
        int32_t* lrs = ip; ip += n + 1;
        int32_t* crs = ip; ip += n + 1;
        int32_t* lcs = ip; ip += ne;
        int32_t* ccs = ip;
        for (int i = threadIdx.x; i <= n; i += NT) {
            lrs[i] = s.lrow[s0 + i] - e0;
            crs[i] = s.cptr[s0 + i] - f0;
        }
        for (int k = threadIdx.x; k < ne; k += NT) { lcs[k] = s.lcol[e0 + k]; lvs[k] = s.lval[e0 + k]; }
        for (int k = threadIdx.x; k < nf; k += NT) { ccs[k] = s.ccol[f0 + k]; cps[k] = s.cpl[f0 + k]; }
        for (int i = threadIdx.x; i < n; i += NT) {
            xu[i] = s.xu[s0 + i]; xv[i] = s.xv[s0 + i]; dg[i] = s.dg[s0 + i];
        }
        lr = lrs; cr = crs; lc = lcs; cc = ccs; lv = lvs; cp = cps;
        __syncthreads();
    } else {
        const int64_t nv = a.nv;
        xu = s.xu + s0; xv = s.xv + s0; dg = s.dg + s0;
        ru = s.gvec + s0; rv = ru + nv; pu = rv + nv; pv = pu + nv; qu = pv + nv; qv = qu + nv;
        lr = s.lrow + s0; cr = s.cptr + s0; lc = s.lcol; cc = s.ccol; lv = s.lval; cp = s.cpl;
    }
    // (A y)_i for the u and v rows of vertex i
    auto apply = [&](int i, const double* yu, const double* yv, double& ou, double& ov) {
        const double d = dg[i];
        double su = d * yu[i], sv = d * yv[i];
        for (int k = lr[i]; k < lr[i + 1]; ++k) {
            const int j = lc[k];
            const double w = lv[k];
            su += w * yu[j];
            sv += w * yv[j];
        }
        for (int k = cr[i]; k < cr[i + 1]; ++k) {
            const int j = cc[k];
            const double w = cp[k];
            su += w * yv[j];
            sv -= w * yu[j];
        }
        ou = su;
        ov = sv;
    };
    auto jac = [&](int i) { const double d = dg[i]; return fabs(d) > 1e-300 ? d : 1.0; };
    double acc[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += NT) {
        double au, av;
        apply(i, xu, xv, au, av);
        const double bu = s.bu[s0 + i], bv = s.bv[s0 + i];
        const double r0 = bu - au, r1 = bv - av, dj = jac(i);
        ru[i] = r0; rv[i] = r1;
        pu[i] = r0 / dj; pv[i] = r1 / dj;
        acc[0] += r0 * pu[i] + r1 * pv[i];
        acc[1] += bu * bu + bv * bv;
    }
    block_sum<NT, 2>(acc, red, phase);   // also publishes p
    double rz = acc[0];
    const double bb = fmax(acc[1], 1e-300);
    int it = 0;
    for (; it < maxiter; ++it) {
        double pq[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            double a0, a1;
            apply(i, pu, pv, a0, a1);
            qu[i] = a0; qv[i] = a1;
            pq[0] += pu[i] * a0 + pv[i] * a1;
        }
        block_sum<NT, 1>(pq, red, phase);
        if (!(pq[0] > 0.0)) break;
        const double alpha = rz / pq[0];
        double nz[2] = {0.0, 0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            xu[i] += alpha * pu[i];
            xv[i] += alpha * pv[i];
            const double r0 = ru[i] - alpha * qu[i], r1 = rv[i] - alpha * qv[i], dj = jac(i);
            ru[i] = r0; rv[i] = r1;
            nz[0] += (r0 * r0 + r1 * r1) / dj;
            nz[1] += r0 * r0 + r1 * r1;
        }
        block_sum<NT, 2>(nz, red, phase);
        if (nz[1] <= tol * tol * bb) { ++it; break; }
        const double beta = nz[0] / rz;
        rz = nz[0];
        for (int i = threadIdx.x; i < n; i += NT) {
            const double dj = jac(i);
            pu[i] = ru[i] / dj + beta * pu[i];
            pv[i] = rv[i] / dj + beta * pv[i];
        }
        __syncthreads();
    }
    if (fit) {
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += NT) { s.xu[s0 + i] = xu[i]; s.xv[s0 + i] = xv[i]; }
    }
    if (threadIdx.x == 0) s.its[c] = it;
}

__global__ void k_hl_out(HlArgs a, HlScratch s, double* U) {
    const int64_t v = static_cast<int64_t>(blockIdx.x) * kTB + threadIdx.x;
    if (v >= a.nv) return;
    const int32_t sl = s.slot[v];
    const double ux = a.U0[2 * v], uy = a.U0[2 * v + 1];
    double x = ux, y = uy;
    if (sl >= 0) { x = s.xu[sl]; y = s.xv[sl]; }
    U[2 * v] = isfinite(x) ? x : ux;
    U[2 * v + 1] = isfinite(y) ? y : uy;
}

// Boundary corners of hier.chart_checks / boundary_directed
// (engine/hier.py:275-291): corner edge k of local face i is interior when
// the face g across it (FF) is in the subset (loc[g] = j >= 0) and in the
// same chart, and g's first corner on the mesh vertex F[f, k] carries the
// same UV vertex. Also the last corner (face order) naming each UV vertex.
__global__ void k_hl_isb(const int32_t* F, const int32_t* FF, int64_t nf, const int32_t* faces, const int32_t* loc,
                         const int32_t* chart, const int32_t* CV, int64_t n, int64_t nv, uint8_t* isb,
                         int32_t* lastc, int32_t* err) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kTB + threadIdx.x;
    if (i >= n) return;
    const int32_t f = faces[i];
    const bool fok = f >= 0 && f < nf;
    if (!fok) flag(err, 2);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int32_t cvk = CV[3 * i + k];
        if (nv > 0) {   // nv = 0: no vertex charts wanted
            if (cvk < 0 || cvk >= nv) flag(err, 2);
            else atomicMax(lastc + cvk, static_cast<int32_t>(3 * i + k));
        }
        uint8_t b = 1;
        const int32_t g = fok ? FF[3 * static_cast<int64_t>(f) + k] : -1;
        if (g >= nf) {
            flag(err, 2);
        } else if (g >= 0) {
            const int32_t j = loc[g];
            if (j >= n) {
                flag(err, 2);
            } else if (j >= 0 && chart[j] == chart[i]) {
                const int32_t v = F[3 * static_cast<int64_t>(f) + k];
                const int32_t* Fg = F + 3 * static_cast<int64_t>(g);
                const int kk = Fg[0] == v ? 0 : (Fg[1] == v ? 1 : (Fg[2] == v ? 2 : -1));
                if (kk >= 0 && CV[3 * static_cast<int64_t>(j) + kk] == cvk) b = 0;
            }
        }
        isb[3 * i + k] = b;
    }
}

__global__ void k_hl_lastc_chart(int64_t nv, const int32_t* chart, int32_t* vchart) {
    const int64_t v = static_cast<int64_t>(blockIdx.x) * kTB + threadIdx.x;
    if (v >= nv) return;
    const int32_t c = vchart[v];   // the last corner naming v, or -1
    vchart[v] = c >= 0 ? chart[c / 3] : -1;
}

bool hl_args_ok(const HlArgs& a) {
    if (a.nv < 0 || a.t < 0 || a.nb < 0 || a.nchart < 0 || a.nvp < 0 || a.nf < 0) return false;
    if (a.t > 0 && (!a.faces || !a.CV || !a.chart || !a.V || !a.F)) return false;
    if (a.nb > 0 && (!a.ba || !a.bb)) return false;
    if (a.nv > 0 && !a.U0) return false;
    return true;
}

bool hl_fits(const HlArgs& a) {   // int32 rows, entries and sort items
    const int64_t lim = INT32_MAX / 2;
    return a.nv < lim / 2 && 3 * a.t < lim && 2 * a.nb < lim && 2 * (a.nv + 6 * a.t + 2 * a.nb) < lim &&
           a.nchart < lim;
}

}  // namespace

extern "C" int uva_hier_lscm_scratch_bytes(int64_t nv, int64_t t, int64_t nb, int32_t nchart, int64_t* bytes) {
    HlArgs a{};
    a.nv = nv; a.t = t; a.nb = nb; a.nchart = nchart;
    if (!bytes || nv < 0 || t < 0 || nb < 0 || nchart < 0) {
        uva_set_error("uva_hier_lscm_scratch_bytes: bad arguments");
        return UVA_E_ARG;
    }
    if (!hl_fits(a)) { uva_set_error("uva_hier_lscm_scratch_bytes: too large for int32 indices"); return UVA_E_TOOBIG; }
    *bytes = static_cast<int64_t>(hl_layout(a, nullptr, nullptr));
    return UVA_OK;
}

extern "C" int uva_hier_lscm(const double* V, int64_t nvp, const int32_t* F, int64_t nf, const int32_t* faces,
                             const int32_t* CV, const int32_t* chart, int64_t t, int64_t nv, int32_t nchart,
                             const double* U0, const int32_t* ba, const int32_t* bb, int64_t nb, double tol,
                             int32_t maxiter, void* scratch, int64_t scratch_bytes, double* U, int32_t* flags,
                             void* stream) {
    HlArgs a{V, F, faces, CV, chart, U0, ba, bb, nvp, nf, t, nv, nb, nchart};
    if (!hl_args_ok(a) || !flags || (nv > 0 && (!U || !scratch)) || maxiter < 0) {
        uva_set_error("uva_hier_lscm: bad arguments");
        return UVA_E_ARG;
    }
    if (!hl_fits(a)) { uva_set_error("uva_hier_lscm: too large for int32 indices"); return UVA_E_TOOBIG; }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return uva_cuda_status(cudaGetLastError(), "uva_hier_lscm");
    if (nv == 0) return UVA_OK;
    HlScratch s{};
    const size_t need = hl_layout(a, static_cast<char*>(scratch), &s);
    if (scratch_bytes < static_cast<int64_t>(need)) { uva_set_error("uva_hier_lscm: scratch too small"); return UVA_E_ARG; }
    s.err = flags;
    auto zero = [&](void* p, size_t bytes) { return cudaMemsetAsync(p, 0, bytes, st); };
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    ok(cudaMemsetAsync(s.lastf, 0xFF, 4 * nv, st));
    ok(zero(s.ccnt, 4 * (nchart + 1)));
    ok(zero(s.npin, 4 * nv));
    ok(zero(s.vcnt, 4 * (nv + 1)));
    ok(zero(s.bcnt, 4 * (nv + 1)));
    ok(zero(s.llen, 4 * (nv + 1)));
    ok(zero(s.clen, 4 * (nv + 1)));
    ok(zero(s.wmax, 8));
    if (nchart > 0) {
        ok(cudaMemsetAsync(s.pmin, 0xFF, 8 * static_cast<size_t>(nchart), st));
        ok(cudaMemsetAsync(s.pmax, 0xFF, 8 * static_cast<size_t>(nchart), st));
    }
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_hier_lscm/memset");
    if (t > 0) k_hl_faces<<<blocks_for(t), kTB, 0, st>>>(a, s);
    k_hl_vchart<<<blocks_for(nv), kTB, 0, st>>>(a, s);
    if (t + nb > 0) k_hl_check<<<blocks_for(t + nb), kTB, 0, st>>>(a, s);
    if (nchart > 0) k_hl_pins<<<blocks_for(nchart), kTB, 0, st>>>(a, s);
    UVA_CHECK_LAUNCH("uva_hier_lscm/faces");
    // stable radix sorts: vertices by chart (then id), corners and boundary ends by vertex (then position)
    size_t cb = s.cub_bytes;
    ok(cub::DeviceRadixSort::SortPairs(s.cub, cb, s.vkey, s.vkey_s, s.vval, s.vval_s, static_cast<int>(nv), 0,
                                       bits_for(nchart), st));
    if (t > 0) {
        cb = s.cub_bytes;
        ok(cub::DeviceRadixSort::SortPairs(s.cub, cb, s.ckey, s.ckey_s, s.cval, s.cval_s, static_cast<int>(3 * t), 0,
                                           bits_for(nv), st));
    }
    if (nb > 0) {
        cb = s.cub_bytes;
        ok(cub::DeviceRadixSort::SortPairs(s.cub, cb, s.bkey, s.bkey_s, s.bval, s.bval_s, static_cast<int>(2 * nb), 0,
                                           bits_for(nv), st));
    }
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_hier_lscm/sort");
    xscan<int32_t>(s.ccnt, s.cofs, s.isums, nullptr, nchart + 1, st);
    xscan<int32_t>(s.vcnt, s.vofs, s.isums, nullptr, nv + 1, st);
    xscan<int32_t>(s.bcnt, s.bofs, s.isums, nullptr, nv + 1, st);
    k_hl_slot<<<blocks_for(nv), kTB, 0, st>>>(a, s);
    k_hl_lap<false><<<blocks_for(nv), kTB, 0, st>>>(a, s);
    xscan<int32_t>(s.llen, s.lrow, s.isums, nullptr, nv + 1, st);
    xscan<int32_t>(s.clen, s.cptr, s.isums, nullptr, nv + 1, st);
    k_hl_lap<true><<<blocks_for(nv), kTB, 0, st>>>(a, s);
    UVA_CHECK_LAUNCH("uva_hier_lscm/assemble");
    if (nchart > 0) {
        ok(cudaFuncSetAttribute(k_hl_pcg<kHlNT>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kHlSmem)));
        if (e != cudaSuccess) return uva_cuda_status(e, "uva_hier_lscm/cudaFuncSetAttribute");
        k_hl_pcg<kHlNT><<<static_cast<unsigned>(nchart), kHlNT, kHlSmem, st>>>(a, s, tol, maxiter);
        UVA_CHECK_LAUNCH("uva_hier_lscm/pcg");
    }
    k_hl_out<<<blocks_for(nv), kTB, 0, st>>>(a, s, U);
    UVA_CHECK_LAUNCH("uva_hier_lscm/out");
    return UVA_OK;
}

extern "C" int uva_hier_boundary_corners(const int32_t* F, const int32_t* FF, int64_t nf, const int32_t* faces,
                                         const int32_t* loc, const int32_t* chart, const int32_t* CV, int64_t n,
                                         int64_t nv, uint8_t* isb, int32_t* vchart, int32_t* flags, void* stream) {
    if (n < 0 || nv < 0 || nf < 0 || !flags || (n > 0 && (!F || !FF || !faces || !loc || !chart || !CV || !isb)) ||
        (nv > 0 && !vchart)) {
        uva_set_error("uva_hier_boundary_corners: bad arguments");
        return UVA_E_ARG;
    }
    if (3 * n >= INT32_MAX || nf >= INT32_MAX / 3) {
        uva_set_error("uva_hier_boundary_corners: too large for int32 indices");
        return UVA_E_TOOBIG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(flags, 0, sizeof(int32_t), st);
    if (e == cudaSuccess && nv > 0) e = cudaMemsetAsync(vchart, 0xFF, 4 * static_cast<size_t>(nv), st);
    if (e != cudaSuccess) return uva_cuda_status(e, "uva_hier_boundary_corners/memset");
    if (n > 0)
        k_hl_isb<<<blocks_for(n), kTB, 0, st>>>(F, FF, nf, faces, loc, chart, CV, n, nv, isb, vchart, flags);
    if (nv > 0) k_hl_lastc_chart<<<blocks_for(nv), kTB, 0, st>>>(nv, chart, vchart);
    UVA_CHECK_LAUNCH("uva_hier_boundary_corners");
    return UVA_OK;
}
