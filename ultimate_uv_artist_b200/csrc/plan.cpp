// Topology plan of a batch of islands (host, C++17, parallel over islands).
//
// Everything here depends on the triangle lists only, so a plan is built once
// per batch and reused by every solve. It replaces the edge deduplication and
// CSR assembly of engine/gpu.py:39-63 (unique_edges, sym_csr) and the boundary
// searches of engine/param.py:59-68 (boundary_edges_oriented) with per-island
// sorts that run on all host cores, and lays the Laplacian pattern out as a
// sliced-ELL matrix (32-row slices, column-major inside a slice) so that a warp
// reads one slot of 32 consecutive rows with one coalesced load. Slice widths
// are padded to a multiple of 4 slots (padding: weight 0, column = the row).
#include <algorithm>
#include <climits>
#include <atomic>
#include <cstring>
#include <memory>
#include <numeric>
#include <thread>
#include <vector>

#include "../../include/uva_b200.h"

extern "C" void uva_set_error(const char* msg);

namespace {

struct IslandPlan {
    int32_t n = 0, t = 0;
    std::vector<int32_t> tri_edge;     // 3t local edge ids (-1: never)
    std::vector<int32_t> edge_info;    // per local edge: count | fwd<<10 | rev<<20
    std::vector<int32_t> row_ptr;      // n+1 (non-self-loop neighbours)
    std::vector<int32_t> row_col;      // neighbour ids, ascending per row
    std::vector<int32_t> row_edge;     // local edge id of each neighbour entry
    std::vector<uint8_t> vflags;       // n
    std::vector<int32_t> bverts;       // sorted unique boundary sources
    int32_t nedges = 0, nslices = 0, nslots = 0;
    std::vector<int32_t> slice_w;      // per slice width
    std::vector<int32_t> row_vert;     // solver row -> vertex (BFS-blob order)
    std::vector<int32_t> vert_row;     // vertex -> solver row
    int32_t agg_rows = 0;              // rows per coarse aggregate (0: no coarse level)
    int32_t ncoarse = 0;               // aggregates
};

// Rows of the island's solver are ordered so that every run of `agg` rows is
// a compact blob of the mesh: each aggregate grows by breadth-first search
// from the lowest unvisited vertex and continues from the next one when its
// component runs out. Aggregates then match whole 32-row slices, so the
// coarse restriction of a vector is a sum of warp reductions.
void blob_order(const IslandPlan& ip, int32_t n, int32_t agg, std::vector<int32_t>& order) {
    order.clear();
    order.reserve(n);
    std::vector<uint8_t> placed(n, 0), inq(n, 0);
    std::vector<int32_t> queue;
    queue.reserve(n);
    int32_t seed = 0;
    while (static_cast<int32_t>(order.size()) < n) {
        const int32_t target = std::min<int32_t>(n, static_cast<int32_t>(order.size()) + agg);
        while (static_cast<int32_t>(order.size()) < target) {
            while (placed[seed]) ++seed;   // an unplaced vertex exists: order.size() < n
            queue.clear();
            queue.push_back(seed);
            inq[seed] = 1;
            size_t head = 0;
            while (head < queue.size() && static_cast<int32_t>(order.size()) < target) {
                const int32_t v = queue[head++];
                placed[v] = 1;
                order.push_back(v);
                for (int32_t q = ip.row_ptr[v]; q < ip.row_ptr[v + 1]; ++q) {
                    const int32_t w = ip.row_col[q];
                    if (!placed[w] && !inq[w]) { inq[w] = 1; queue.push_back(w); }
                }
            }
            for (const int32_t v : queue) inq[v] = 0;
        }
    }
}

template <typename I>   // int32_t or int64_t island-local vertex ids
void build_island(const I* T, int32_t n, int32_t t, IslandPlan& ip, bool& bad) {
    ip.n = n; ip.t = t;
    // half-edges grouped by (lo, hi, half-edge id): a counting sort by lo
    // into contiguous (hi, 2 h + dir) pairs (dir 1: the half-edge runs lo ->
    // hi, or is a self-loop), then a stable insertion sort by hi inside each
    // (short) bucket; everything after reads the buckets sequentially
    const int32_t nh = 3 * t;
    std::vector<int32_t> bstart(n + 1, 0);
    for (int32_t f = 0; f < t; ++f) {
        for (int k = 0; k < 3; ++k) {
            const int64_t a = static_cast<int64_t>(T[3 * f + (k + 1) % 3]), b = static_cast<int64_t>(T[3 * f + (k + 2) % 3]);
            if (a < 0 || a >= n || b < 0 || b >= n) { bad = true; return; }
            ++bstart[(a < b ? a : b) + 1];
        }
    }
    for (int32_t v = 0; v < n; ++v) bstart[v + 1] += bstart[v];
    std::vector<int32_t> bhi(nh), bhd(nh);
    {
        std::vector<int32_t> fillb(bstart.begin(), bstart.end() - 1);
        for (int32_t f = 0; f < t; ++f) {
            for (int k = 0; k < 3; ++k) {
                const int32_t a = static_cast<int32_t>(T[3 * f + (k + 1) % 3]), b = static_cast<int32_t>(T[3 * f + (k + 2) % 3]);
                const int32_t lo = a < b ? a : b;
                const int32_t q = fillb[lo]++;
                bhi[q] = a < b ? b : a;
                bhd[q] = 2 * (3 * f + k) + (a == lo ? 1 : 0);
            }
        }
    }
    for (int32_t v = 0; v < n; ++v) {
        for (int32_t q = bstart[v] + 1; q < bstart[v + 1]; ++q) {
            const int32_t hi = bhi[q], hd = bhd[q];
            int32_t r = q - 1;
            while (r >= bstart[v] && bhi[r] > hi) { bhi[r + 1] = bhi[r]; bhd[r + 1] = bhd[r]; --r; }
            bhi[r + 1] = hi; bhd[r + 1] = hd;
        }
    }
    ip.tri_edge.assign(static_cast<size_t>(3) * t, -1);
    std::vector<int32_t> deg(n, 0);   // neighbours per vertex (self-loops excluded)
    ip.edge_info.clear();
    ip.edge_info.reserve(nh / 2 + n + 4);
    std::vector<int32_t> elo, ehi;   // endpoints of each unique edge (lo <= hi)
    elo.reserve(nh / 2 + n + 4);
    ehi.reserve(nh / 2 + n + 4);
    for (int32_t lo = 0; lo < n; ++lo) {
        const int32_t qe = bstart[lo + 1];
        for (int32_t q = bstart[lo]; q < qe;) {
            const int32_t hi = bhi[q];
            int32_t fwd = 0, rev = 0, e = q;
            for (; e < qe && bhi[e] == hi; ++e) {
                const int32_t hd = bhd[e];
                if (hd & 1) ++fwd; else ++rev;
                ip.tri_edge[hd >> 1] = static_cast<int32_t>(elo.size());
            }
            const int32_t cnt = e - q;
            ip.edge_info.push_back(std::min(cnt, 1023) | (std::min(fwd, 1023) << 10) | (std::min(rev, 1023) << 20));
            elo.push_back(lo);
            ehi.push_back(hi);
            if (lo != hi) { ++deg[lo]; ++deg[hi]; }
            q = e;
        }
    }
    ip.nedges = static_cast<int32_t>(elo.size());
    // rows: appending in key order keeps each row sorted (see file comment)
    ip.row_ptr.assign(n + 1, 0);
    for (int32_t v = 0; v < n; ++v) ip.row_ptr[v + 1] = ip.row_ptr[v] + deg[v];
    ip.row_col.assign(ip.row_ptr[n], 0);
    ip.row_edge.assign(ip.row_ptr[n], 0);
    std::vector<int32_t> fill(ip.row_ptr.begin(), ip.row_ptr.end() - 1);
    for (int32_t e = 0; e < ip.nedges; ++e) {
        const int32_t lo = elo[e], hi = ehi[e];
        if (lo == hi) continue;
        ip.row_col[fill[lo]] = hi; ip.row_edge[fill[lo]++] = e;
        ip.row_col[fill[hi]] = lo; ip.row_edge[fill[hi]++] = e;
    }
    // the fill above appends hi-entries of row `lo` before lo-entries of rows
    // met later; restore ascending column order per row
    for (int32_t v = 0; v < n; ++v) {
        const int32_t a = ip.row_ptr[v], b = ip.row_ptr[v + 1];
        bool sorted = true;
        for (int32_t q = a + 1; q < b; ++q) if (ip.row_col[q - 1] > ip.row_col[q]) { sorted = false; break; }
        if (!sorted) {
            std::vector<std::pair<int32_t, int32_t>> tmp;
            for (int32_t q = a; q < b; ++q) tmp.emplace_back(ip.row_col[q], ip.row_edge[q]);
            std::sort(tmp.begin(), tmp.end());
            for (int32_t q = a; q < b; ++q) { ip.row_col[q] = tmp[q - a].first; ip.row_edge[q] = tmp[q - a].second; }
        }
    }
    // vertex flags and boundary sources
    ip.vflags.assign(n, 0);
    std::vector<uint8_t> isb(n, 0);
    for (int32_t e = 0; e < ip.nedges; ++e) {
        const int32_t info = ip.edge_info[e];
        const int32_t cnt = info & 1023, fwd = (info >> 10) & 1023, rev = (info >> 20) & 1023;
        const int32_t lo = elo[e], hi = ehi[e];
        if (cnt == 1) { ip.vflags[lo] |= 1; ip.vflags[hi] |= 1; }
        if (lo == hi) continue;
        if (fwd > 0 && rev == 0) { ip.vflags[lo] |= 2; ip.vflags[hi] |= 2; isb[lo] = 1; }
        if (rev > 0 && fwd == 0) { ip.vflags[lo] |= 2; ip.vflags[hi] |= 2; isb[hi] = 1; }
    }
    ip.bverts.clear();
    for (int32_t v = 0; v < n; ++v) if (isb[v]) ip.bverts.push_back(v);
    // solver row order and coarse aggregates (islands above one warp's rows)
    if (n > 256) {
        ip.agg_rows = 64;
        while ((n + ip.agg_rows - 1) / ip.agg_rows > 256) ip.agg_rows += 64;
        ip.ncoarse = (n + ip.agg_rows - 1) / ip.agg_rows;
        blob_order(ip, n, ip.agg_rows, ip.row_vert);
    } else {
        ip.agg_rows = 0;
        ip.ncoarse = 0;
        ip.row_vert.resize(n);
        for (int32_t v = 0; v < n; ++v) ip.row_vert[v] = v;
    }
    ip.vert_row.assign(n, 0);
    for (int32_t r = 0; r < n; ++r) ip.vert_row[ip.row_vert[r]] = r;
    // sliced ELL over solver rows: 32 rows per slice
    ip.nslices = (n + 31) / 32;
    ip.slice_w.assign(ip.nslices, 0);
    ip.nslots = 0;
    for (int32_t s = 0; s < ip.nslices; ++s) {
        int32_t w = 0;
        for (int32_t r = s * 32; r < std::min(n, s * 32 + 32); ++r) w = std::max(w, deg[ip.row_vert[r]]);
        w = (w + 3) & ~3;            // multiple of 4: the SpMV loads slots 4 at a time
        ip.slice_w[s] = w;
        ip.nslots += 32 * w;
    }
}

}  // namespace

struct uva_plan {
    int32_t nc = 0;
    int64_t n = 0, t = 0, E = 0, nslices = 0, nslots = 0, nbverts = 0, maxrows = 0;
    std::vector<int64_t> vofs, tofs;
    std::vector<IslandPlan> isl;
    std::vector<int64_t> eofs, sofs, slotofs, bofs, cofs;
    const int64_t* tris = nullptr;   // not owned; only valid during create
    std::unique_ptr<int32_t[]> tri_local;   // 3t local ids (copied by the island workers)
};

// The plan of every island; island i's triangles come from tri_src(i):
// (pointer to its 3 t_i local ids, true if int64 else int32).
template <typename Src>
int plan_create(Src tri_src, const int64_t* vofs, const int64_t* tofs, int32_t nc, int32_t nthreads, uva_plan** out) {
    if (!out || nc < 0 || (nc > 0 && (!vofs || !tofs))) { uva_set_error("uva_plan_create: bad arguments"); return UVA_E_ARG; }
    *out = nullptr;
    auto* p = new uva_plan();
    p->nc = nc;
    p->vofs.assign(vofs, vofs + nc + 1);
    p->tofs.assign(tofs, tofs + nc + 1);
    for (int32_t i = 0; i < nc; ++i) {
        if (p->vofs[i + 1] < p->vofs[i] || p->tofs[i + 1] < p->tofs[i]) {
            delete p; uva_set_error("uva_plan_create: offsets must be non-decreasing"); return UVA_E_ARG;
        }
        if (p->tofs[i + 1] > p->tofs[i] && !tri_src(i).first) {
            delete p; uva_set_error("uva_plan_create: null triangles"); return UVA_E_ARG;
        }
    }
    p->n = p->vofs[nc] - p->vofs[0];
    p->t = p->tofs[nc] - p->tofs[0];
    if (p->n > (int64_t(1) << 30) || 3 * p->t > (int64_t(1) << 30)) {
        delete p; uva_set_error("uva_plan_create: batch too large for 32-bit indices"); return UVA_E_TOOBIG;
    }
    p->isl.resize(nc);
    p->tri_local.reset(new int32_t[static_cast<size_t>(3 * p->t) + 1]);   // uninitialised; filled per island
    // largest islands first for load balance
    std::vector<int32_t> order(nc);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return (p->tofs[a + 1] - p->tofs[a]) > (p->tofs[b + 1] - p->tofs[b]);
    });
    std::atomic<int32_t> next{0};
    std::atomic<bool> anybad{false};
    auto worker = [&]() {
        for (;;) {
            const int32_t q = next.fetch_add(1);
            if (q >= nc) break;
            const int32_t i = order[q];
            bool bad = false;
            const int64_t t0 = 3 * (p->tofs[i] - p->tofs[0]), tn = 3 * (p->tofs[i + 1] - p->tofs[i]);
            const int32_t ni = static_cast<int32_t>(p->vofs[i + 1] - p->vofs[i]);
            const int32_t ti = static_cast<int32_t>(p->tofs[i + 1] - p->tofs[i]);
            const auto src = tri_src(i);
            if (src.second) {
                const int64_t* tris = static_cast<const int64_t*>(src.first);
                build_island(tris, ni, ti, p->isl[i], bad);
                if (!bad) for (int64_t c = 0; c < tn; ++c) p->tri_local[t0 + c] = static_cast<int32_t>(tris[c]);
            } else {
                const int32_t* tris = static_cast<const int32_t*>(src.first);
                build_island(tris, ni, ti, p->isl[i], bad);
                if (!bad) std::memcpy(p->tri_local.get() + t0, tris, sizeof(int32_t) * static_cast<size_t>(tn));
            }
            if (bad) anybad = true;
        }
    };
    int32_t nt = nthreads > 0 ? nthreads : static_cast<int32_t>(std::thread::hardware_concurrency());
    nt = std::max(1, std::min(nt, std::max(nc, 1)));
    std::vector<std::thread> pool;
    for (int32_t k = 1; k < nt; ++k) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    if (anybad) { delete p; uva_set_error("uva_plan_create: triangle index outside its island"); return UVA_E_ARG; }
    for (int32_t i = 0; i < nc; ++i) {
        // the solver packs an island row in 24 bits and twice the LSCM
        // boundary coupling in 8 (signed)
        const IslandPlan& ip = p->isl[i];
        if (ip.n >= (1 << 24)) { delete p; uva_set_error("uva_plan_create: island above 16M vertices"); return UVA_E_TOOBIG; }
        for (int32_t e = 0; e < ip.nedges; ++e) {
            const int32_t info = ip.edge_info[e];
            if (((info >> 10) & 1023) > 127 || ((info >> 20) & 1023) > 127) {
                delete p; uva_set_error("uva_plan_create: an edge is used by more than 127 triangles in one direction");
                return UVA_E_ARG;
            }
        }
    }
    p->eofs.assign(nc + 1, 0); p->sofs.assign(nc + 1, 0); p->slotofs.assign(nc + 1, 0); p->bofs.assign(nc + 1, 0);
    p->cofs.assign(nc + 1, 0);
    for (int32_t i = 0; i < nc; ++i) {
        p->eofs[i + 1] = p->eofs[i] + p->isl[i].nedges;
        p->sofs[i + 1] = p->sofs[i] + p->isl[i].nslices;
        p->slotofs[i + 1] = p->slotofs[i] + p->isl[i].nslots;
        p->bofs[i + 1] = p->bofs[i] + static_cast<int64_t>(p->isl[i].bverts.size());
        p->cofs[i + 1] = p->cofs[i] + static_cast<int64_t>(p->isl[i].ncoarse) * p->isl[i].ncoarse;
        p->maxrows = std::max<int64_t>(p->maxrows, p->isl[i].n);
    }
    p->E = p->eofs[nc]; p->nslices = p->sofs[nc]; p->nslots = p->slotofs[nc]; p->nbverts = p->bofs[nc];
    if (p->nslots > (int64_t(1) << 31) - 1 || p->E > (int64_t(1) << 31) - 1 || 4 * p->cofs[nc] > (int64_t(1) << 31) - 1) {
        delete p; uva_set_error("uva_plan_create: plan too large for 32-bit offsets"); return UVA_E_TOOBIG;
    }
    *out = p;
    return UVA_OK;
}


extern "C" int uva_plan_create(const int64_t* tris, const int64_t* vofs, const int64_t* tofs, int32_t nc,
                               int32_t nthreads, uva_plan** out) {
    if (nc > 0 && vofs && tofs && tofs[nc] > tofs[0] && !tris) { uva_set_error("uva_plan_create: null triangles"); return UVA_E_ARG; }
    const int64_t base = (nc > 0 && tofs) ? tofs[0] : 0;
    return plan_create([&](int32_t i) { return std::make_pair(static_cast<const void*>(tris + 3 * (tofs[i] - base)), true); },
                       vofs, tofs, nc, nthreads, out);
}

extern "C" int uva_plan_create_charts(const void* const* T, const int8_t* tdt, const int64_t* vofs,
                                      const int64_t* tofs, int32_t nc, int32_t nthreads, uva_plan** out) {
    if (nc > 0 && (!T || !tdt)) { uva_set_error("uva_plan_create_charts: bad arguments"); return UVA_E_ARG; }
    for (int32_t i = 0; i < nc; ++i)
        if (tdt[i] < 0 || tdt[i] > 1) { uva_set_error("uva_plan_create_charts: dtype codes 0/1"); return UVA_E_ARG; }
    return plan_create([&](int32_t i) { return std::make_pair(T[i], tdt[i] == 1); }, vofs, tofs, nc, nthreads, out);
}

extern "C" int uva_plan_sizes(const uva_plan* p, int64_t* s) {
    if (!p || !s) { uva_set_error("uva_plan_sizes: null argument"); return UVA_E_ARG; }
    s[UVA_PLAN_NC] = p->nc; s[UVA_PLAN_N] = p->n; s[UVA_PLAN_T] = p->t; s[UVA_PLAN_E] = p->E;
    s[UVA_PLAN_NSLICES] = p->nslices; s[UVA_PLAN_NSLOTS] = p->nslots; s[UVA_PLAN_NBVERTS] = p->nbverts;
    s[UVA_PLAN_MAXROWS] = p->maxrows;
    s[UVA_PLAN_NCOARSE] = p->cofs[p->nc];
    return UVA_OK;
}

extern "C" int uva_plan_export(const uva_plan* p, int32_t* tri4, int32_t* tri_edge, int32_t* sofs,
                               int32_t* slice_ptr, int32_t* slot_col, int32_t* slot_edge, float* slot_c,
                               int32_t* vt_ptr, int32_t* vt, uint8_t* vflags, int32_t* bofs, int32_t* bverts) {
    if (!p) { uva_set_error("uva_plan_export: null plan"); return UVA_E_ARG; }
    return uva_plan_export_range(p, 0, p->nc, tri4, tri_edge, sofs, slice_ptr, slot_col, slot_edge, slot_c, vt_ptr,
                                 vt, vflags, bofs, bverts);
}

extern "C" int uva_plan_island_offsets(const uva_plan* p, int64_t* out) {
    if (!p || !out) { uva_set_error("uva_plan_island_offsets: null argument"); return UVA_E_ARG; }
    const int32_t nc = p->nc;
    for (int32_t i = 0; i <= nc; ++i) {
        out[i] = p->sofs[i];
        out[(nc + 1) + i] = p->slotofs[i];
        out[2 * (nc + 1) + i] = p->bofs[i];
    }
    return UVA_OK;
}

extern "C" int uva_plan_export_range(const uva_plan* p, int32_t i0, int32_t i1, int32_t* tri4, int32_t* tri_edge,
                                     int32_t* sofs, int32_t* slice_ptr, int32_t* slot_col, int32_t* slot_edge,
                                     float* slot_c, int32_t* vt_ptr, int32_t* vt, uint8_t* vflags, int32_t* bofs,
                                     int32_t* bverts) {
    if (!p) { uva_set_error("uva_plan_export: null plan"); return UVA_E_ARG; }
    const int32_t nc = p->nc;
    if (i0 < 0 || i1 < i0 || i1 > nc) { uva_set_error("uva_plan_export_range: bad island range"); return UVA_E_ARG; }
    const int64_t v0 = p->vofs.empty() ? 0 : p->vofs[0];
    const int64_t t0 = p->tofs.empty() ? 0 : p->tofs[0];
    // islands are independent: every array of island i lands in its own
    // range, so workers take islands from a shared counter, largest first
    std::vector<int32_t> order(i1 - i0);
    std::iota(order.begin(), order.end(), i0);
    std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return p->isl[a].t > p->isl[b].t; });
    const int32_t cnt_isl = i1 - i0;
    std::atomic<int32_t> next{0};
    auto one = [&](int32_t i) {
        const IslandPlan& ip = p->isl[i];
        const int64_t fb = p->tofs[i] - t0, vb = p->vofs[i] - v0;
        const int64_t eb = p->eofs[i], sb = p->sofs[i], slb = p->slotofs[i];
        const int32_t* tl = p->tri_local.get() + 3 * fb;
        for (int32_t f = 0; f < ip.t; ++f) {
            for (int k = 0; k < 3; ++k) {
                tri4[4 * (fb + f) + k] = tl[3 * f + k];
                const int32_t e = ip.tri_edge[3 * f + k];
                tri_edge[3 * (fb + f) + k] = e < 0 ? -1 : static_cast<int32_t>(eb + e);
            }
            tri4[4 * (fb + f) + 3] = i;
        }
        if (sofs) sofs[i] = static_cast<int32_t>(sb);
        // sliced ELL: row by row (its slots sit 32 apart inside the slice)
        int64_t slot = slb;
        for (int32_t s = 0; s < ip.nslices; ++s) {
            slice_ptr[sb + s] = static_cast<int32_t>(slot);
            const int32_t w = ip.slice_w[s];
            for (int32_t lane = 0; lane < 32; ++lane) {
                const int32_t row = s * 32 + lane;
                int32_t k = 0;
                if (row < ip.n) {
                    const int32_t r = ip.row_vert[row];   // vertex of this row
                    const int32_t a = ip.row_ptr[r], deg = ip.row_ptr[r + 1] - a;
                    for (; k < deg; ++k) {
                        const int64_t q = slot + static_cast<int64_t>(k) * 32 + lane;
                        const int32_t j = ip.row_col[a + k];
                        const int32_t e = ip.row_edge[a + k];
                        slot_col[q] = ip.vert_row[j];
                        slot_edge[q] = static_cast<int32_t>(eb + e);
                        const int32_t info = ip.edge_info[e];
                        const int32_t nf = (info >> 10) & 1023, nr = (info >> 20) & 1023;
                        // half-edges r->j and j->r (fwd is lo->hi)
                        const int32_t n_rj = r < j ? nf : nr, n_jr = r < j ? nr : nf;
                        const int32_t b_rj = n_jr == 0 ? n_rj : 0, b_jr = n_rj == 0 ? n_jr : 0;
                        slot_c[q] = -0.5f * static_cast<float>(b_rj) + 0.5f * static_cast<float>(b_jr);
                    }
                }
                for (; k < w; ++k) {   // padding: zero weight, the row itself (0 past the island's end)
                    const int64_t q = slot + static_cast<int64_t>(k) * 32 + lane;
                    slot_col[q] = row < ip.n ? row : 0;
                    slot_edge[q] = -1;
                    slot_c[q] = 0.0f;
                }
            }
            slot += static_cast<int64_t>(w) * 32;
        }
        for (int32_t v = 0; v < ip.n; ++v) vflags[vb + v] = ip.vflags[v];
        if (bofs) bofs[i] = static_cast<int32_t>(p->bofs[i]);
        for (size_t q = 0; q < ip.bverts.size(); ++q) bverts[p->bofs[i] + q] = ip.bverts[q];
        // vertex -> (triangle, corner) incidence, ascending by f*3+corner; an
        // island's corners are its own 3*t entries (offset 3 * tofs[i])
        const int32_t n = ip.n, t = ip.t;
        std::vector<int32_t> cnt(n + 1, 0);
        for (int32_t c = 0; c < 3 * t; ++c) ++cnt[tl[c] + 1];
        for (int32_t v = 0; v < n; ++v) cnt[v + 1] += cnt[v];
        for (int32_t v = 0; v <= n; ++v) vt_ptr[vb + v] = static_cast<int32_t>(3 * fb + cnt[v]);
        for (int32_t c = 0; c < 3 * t; ++c) vt[3 * fb + cnt[tl[c]]++] = static_cast<int32_t>(3 * fb + c);
    };
    auto worker = [&]() {
        for (;;) {
            const int32_t q = next.fetch_add(1);
            if (q >= cnt_isl) break;
            one(order[q]);
        }
    };
    int32_t nt = static_cast<int32_t>(std::thread::hardware_concurrency());
    nt = std::max(1, std::min(nt, std::max(cnt_isl, 1)));
    std::vector<std::thread> pool;
    for (int32_t k = 1; k < nt; ++k) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    if (i1 == nc) {   // the closing offsets, with the last range
        if (sofs) sofs[nc] = static_cast<int32_t>(p->nslices);
        slice_ptr[p->nslices] = static_cast<int32_t>(p->nslots);
        if (bofs) bofs[nc] = static_cast<int32_t>(p->nbverts);
        vt_ptr[p->n] = static_cast<int32_t>(3 * p->t);
    }
    return UVA_OK;
}

extern "C" void uva_plan_destroy(uva_plan* p) { delete p; }

extern "C" int uva_plan_export_rows(const uva_plan* p, int32_t* row_vert, int32_t* vert_row, int32_t* agg_rows,
                                    int32_t* cofs) {
    if (!p || !row_vert || !vert_row || !agg_rows || !cofs) { uva_set_error("uva_plan_export_rows: null argument"); return UVA_E_ARG; }
    const int64_t v0 = p->vofs.empty() ? 0 : p->vofs[0];
    std::atomic<int32_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int32_t i = next.fetch_add(1);
            if (i >= p->nc) break;
            const IslandPlan& ip = p->isl[i];
            const int64_t vb = p->vofs[i] - v0;
            std::memcpy(row_vert + vb, ip.row_vert.data(), sizeof(int32_t) * ip.n);
            std::memcpy(vert_row + vb, ip.vert_row.data(), sizeof(int32_t) * ip.n);
            agg_rows[i] = ip.agg_rows;
            cofs[i] = static_cast<int32_t>(p->cofs[i]);
        }
    };
    int32_t nt = std::max(1, std::min<int32_t>(static_cast<int32_t>(std::thread::hardware_concurrency()), std::max(p->nc, 1)));
    std::vector<std::thread> pool;
    for (int32_t k = 1; k < nt; ++k) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    cofs[p->nc] = static_cast<int32_t>(p->cofs[p->nc]);
    return UVA_OK;
}

// ------------------------------------------------------------------ batch concatenation
// Per-chart host arrays (numpy inputs of any supported dtype) into the batch
// layout, charts in parallel: positions and UVs widened to FP64, triangles to
// int64. Replaces the per-chart copies of engine/gpu.py:69-87.
namespace {

template <typename S, typename D>
void widen(const void* src, D* dst, int64_t count) {
    const S* s = static_cast<const S*>(src);
    for (int64_t k = 0; k < count; ++k) dst[k] = static_cast<D>(s[k]);
}

}  // namespace

extern "C" int uva_concat_charts(int32_t nc, const void* const* P, const int8_t* pdt, const void* const* T,
                                 const int8_t* tdt, const void* const* U, const int8_t* udt, const int64_t* vofs,
                                 const int64_t* tofs, double* P_out, int64_t* T_out, double* U_out,
                                 int32_t nthreads) {
    if (nc < 0 || (nc > 0 && (!P || !pdt || !vofs || !tofs || !P_out || (T_out && (!T || !tdt))))) {
        uva_set_error("uva_concat_charts: bad arguments");
        return UVA_E_ARG;
    }
    for (int32_t i = 0; i < nc; ++i) {
        if (vofs[i + 1] < vofs[i] || tofs[i + 1] < tofs[i] || pdt[i] < 0 || pdt[i] > 1 ||
            (T_out && (tdt[i] < 0 || tdt[i] > 1)) ||
            (U && udt && (udt[i] < -1 || udt[i] > 1))) {
            uva_set_error("uva_concat_charts: offsets must be non-decreasing, dtype codes 0/1 (U: -1/0/1)");
            return UVA_E_ARG;
        }
        if ((vofs[i + 1] > vofs[i] && !P[i]) || (T_out && tofs[i + 1] > tofs[i] && !T[i])) {
            uva_set_error("uva_concat_charts: null chart array");
            return UVA_E_ARG;
        }
    }
    std::atomic<int32_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int32_t i = next.fetch_add(1);
            if (i >= nc) break;
            // sizes were checked non-negative above
            const int64_t nv = std::max<int64_t>(vofs[i + 1] - vofs[i], 0), nt = std::max<int64_t>(tofs[i + 1] - tofs[i], 0);
            double* po = P_out + 3 * (vofs[i] - vofs[0]);
            if (pdt[i] == 0) widen<float>(P[i], po, 3 * nv); else std::memcpy(po, P[i], sizeof(double) * 3 * nv);
            if (T_out) {
                int64_t* to = T_out + 3 * (tofs[i] - tofs[0]);
                if (tdt[i] == 0) widen<int32_t>(T[i], to, 3 * nt); else std::memcpy(to, T[i], sizeof(int64_t) * 3 * nt);
            }
            if (U_out) {
                double* uo = U_out + 2 * (vofs[i] - vofs[0]);
                const int8_t d = (U && udt) ? udt[i] : -1;
                if (d < 0 || !U[i]) std::memset(uo, 0, sizeof(double) * 2 * nv);
                else if (d == 0) widen<float>(U[i], uo, 2 * nv);
                else std::memcpy(uo, U[i], sizeof(double) * 2 * nv);
            }
        }
    };
    int32_t nt = nthreads > 0 ? nthreads : static_cast<int32_t>(std::thread::hardware_concurrency());
    nt = std::max(1, std::min(nt, std::max(nc, 1)));
    std::vector<std::thread> pool;
    for (int32_t k = 1; k < nt; ++k) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return UVA_OK;
}

// Per-chart triangle arrays (int32 / int64 island-local ids) into one int32
// array at tofs, charts in parallel: the upload of the device-built plan
// (csrc/dplan.cu). An id outside the int32 range is an error (the device
// plan checks the island ranges).
extern "C" int uva_concat_tris32(int32_t nc, const void* const* T, const int8_t* tdt, const int64_t* tofs,
                                 int32_t* out, int32_t nthreads) {
    if (nc < 0 || (nc > 0 && (!T || !tdt || !tofs || !out))) {
        uva_set_error("uva_concat_tris32: bad arguments");
        return UVA_E_ARG;
    }
    for (int32_t i = 0; i < nc; ++i) {
        if (tofs[i + 1] < tofs[i] || tdt[i] < 0 || tdt[i] > 1 || (tofs[i + 1] > tofs[i] && !T[i])) {
            uva_set_error("uva_concat_tris32: offsets must be non-decreasing, dtype codes 0/1, arrays non-null");
            return UVA_E_ARG;
        }
    }
    std::atomic<int32_t> next{0};
    std::atomic<bool> wide{false};
    auto worker = [&]() {
        for (;;) {
            const int32_t i = next.fetch_add(1);
            if (i >= nc) break;
            const int64_t cnt = 3 * (tofs[i + 1] - tofs[i]);
            int32_t* o = out + 3 * (tofs[i] - tofs[0]);
            if (tdt[i] == 0) {
                std::memcpy(o, T[i], sizeof(int32_t) * static_cast<size_t>(cnt));
            } else {
                const int64_t* s = static_cast<const int64_t*>(T[i]);
                bool bad = false;
                for (int64_t k = 0; k < cnt; ++k) {
                    const int64_t v = s[k];
                    bad |= v < INT32_MIN || v > INT32_MAX;
                    o[k] = static_cast<int32_t>(v);
                }
                if (bad) wide = true;
            }
        }
    };
    int32_t nt = nthreads > 0 ? nthreads : static_cast<int32_t>(std::thread::hardware_concurrency());
    nt = std::max(1, std::min(nt, std::max(nc, 1)));
    std::vector<std::thread> pool;
    for (int32_t k = 1; k < nt; ++k) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    if (wide) { uva_set_error("uva_concat_tris32: a triangle index outside the int32 range"); return UVA_E_ARG; }
    return UVA_OK;
}

// Per-chart float32 rows (width floats each) into one float32 array at ofs,
// charts in parallel: positions that are float32 already travel to the
// device as they are (half the bytes of the FP64 batch copy).
extern "C" int uva_concat_rows32(int32_t nc, const void* const* src, const int64_t* ofs, int32_t width, float* out,
                                 int32_t nthreads) {
    if (nc < 0 || width <= 0 || (nc > 0 && (!src || !ofs || !out))) {
        uva_set_error("uva_concat_rows32: bad arguments");
        return UVA_E_ARG;
    }
    for (int32_t i = 0; i < nc; ++i) {
        if (ofs[i + 1] < ofs[i] || (ofs[i + 1] > ofs[i] && !src[i])) {
            uva_set_error("uva_concat_rows32: offsets must be non-decreasing, arrays non-null");
            return UVA_E_ARG;
        }
    }
    std::atomic<int32_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int32_t i = next.fetch_add(1);
            if (i >= nc) break;
            std::memcpy(out + width * (ofs[i] - ofs[0]), src[i],
                        sizeof(float) * static_cast<size_t>(width * (ofs[i + 1] - ofs[i])));
        }
    };
    int32_t nt = nthreads > 0 ? nthreads : static_cast<int32_t>(std::thread::hardware_concurrency());
    nt = std::max(1, std::min(nt, std::max(nc, 1)));
    std::vector<std::thread> pool;
    for (int32_t k = 1; k < nt; ++k) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return UVA_OK;
}
