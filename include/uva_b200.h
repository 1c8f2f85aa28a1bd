/*
 * uva_b200.h - C ABI of the B200 (sm_100a) parameterization and validation
 * kernels of Ultimate UV Artist's per-island hot path.
 *
 * Conventions
 *   - Every function returns an int status: UVA_OK (0) or a negative
 *     UVA_E_* code; uva_last_error() gives a message for the calling thread.
 *   - Device pointers are plain pointers into CUDA global memory on the
 *     current device; `stream` is a cudaStream_t passed as void*. Nothing is
 *     synchronised unless the function says so.
 *   - No global mutable state: calls on different streams/threads are
 *     independent (the reference calls its flatten path from thread pools).
 *   - A batch is many charts ("islands") concatenated block-diagonally:
 *     vertices [vofs[i], vofs[i+1]) and triangles [tofs[i], tofs[i+1]) belong
 *     to island i. Triangles hold island-LOCAL vertex indices.
 *
 * Reference interfaces replaced (paths inside the Ultimate UV Artist project):
 *   engine/gpu.py   Batch.__init__ :69-124, _build_laplacian :126-142,
 *                   _rhs :165-182, _cg :184-202, _max_step :204-227,
 *                   arap :230-249, repair_flips :251-273,
 *                   orient_positive :275-281, flips_per_chart :158-163,
 *                   signed_area :153-156, jacobians :145-151, shrink :283-295
 *   engine/param.py local_frames :19-32, cot_weights :35-44, lscm :136-169,
 *                   _far_pair :172-179, refine (arap) :379-414,
 *                   _arap_rotations :206-256, _arap_rhs :457-474,
 *                   _max_step :259-291, _energy :294-319,
 *                   repair_flips :477-516, chart_quality :520-551
 *   engine/validate.py, engine/metrics.py: see the validation block below.
 */
#ifndef UVA_B200_H
#define UVA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UVA_OK            0
#define UVA_E_ARG        -1   /* bad argument (null pointer, negative size) */
#define UVA_E_CUDA       -2   /* a CUDA runtime call failed                 */
#define UVA_E_NOBOUNDARY -3   /* LSCM on an island with no boundary         */
#define UVA_E_TOOBIG     -4   /* size above a documented maximum            */
#define UVA_E_NODEVICE   -5   /* no CUDA device / not sm_100                */

/* Frame / weight semantics: the two reference solvers differ in how they
 * treat thin triangles (gpu.py:102-120 vs param.py:19-44).                 */
#define UVA_SEM_BATCH 0
#define UVA_SEM_PARAM 1

/* Per-island solver status bits (uva_island_status.flags).                 */
#define UVA_ST_MAXITER    1   /* an inner CG or the refinement hit its cap  */
#define UVA_ST_NONFINITE  2   /* the solve went non-finite; U kept          */
#define UVA_ST_ENERGYSTOP 4   /* relative-energy stop (param.refine)        */
#define UVA_ST_NOBOUNDARY 8   /* LSCM: no boundary loop                     */
#define UVA_ST_BADCLASS   16  /* island above its team's capacity (class_ofs
                                  inconsistent with the sizes); not solved      */

typedef struct uva_island_status {
    int32_t cg_iters;      /* inner FP32 CG iterations executed             */
    int32_t refinements;   /* FP64 residual recomputations                  */
    int32_t outer_iters;   /* ARAP local/global iterations executed         */
    int32_t flags;         /* UVA_ST_* bits                                 */
    double  resid[2];      /* last FP64 relative residual per column        */
    double  energy;        /* last ARAP energy (param semantics)            */
    double  step;          /* last line-search step                         */
    int64_t t_begin;       /* %globaltimer (ns) when the island's team took it */
    int64_t t_end;         /* %globaltimer (ns) when the team finished it    */
    int32_t sm;            /* SM that ran the island                        */
    int32_t team;          /* team width that ran it (1024, 256 or 32; the
                              whole GPU, 148 * 1024, for islands above 16,384
                              vertices)                                     */
} uva_island_status;

/* --------------------------------------------------------------------------
 * Topology plan (host). Built from the triangle lists only, in parallel over
 * islands; replaces gpu.unique_edges / sym_csr (gpu.py:39-63) and the
 * boundary searches of param.boundary_edges_oriented (param.py:59-68).
 * ------------------------------------------------------------------------ */
typedef struct uva_plan uva_plan;

enum {
    UVA_PLAN_NC = 0, UVA_PLAN_N, UVA_PLAN_T, UVA_PLAN_E, UVA_PLAN_NSLICES,
    UVA_PLAN_NSLOTS, UVA_PLAN_NBVERTS, UVA_PLAN_MAXROWS, UVA_PLAN_NCOARSE, UVA_PLAN_NSIZES
};

/* tris: t*3 island-LOCAL vertex ids (int64, host); vofs/tofs: nc+1 offsets.
 * Returns UVA_E_ARG if an index is out of its island's range.              */
int uva_plan_create(const int64_t* tris, const int64_t* vofs, const int64_t* tofs,
                    int32_t nc, int32_t nthreads, uva_plan** out);
/* The same from per-chart triangle arrays (island i: T[i], 3 t_i local ids,
 * tdt[i] 0: int32, 1: int64), without concatenating them first.          */
int uva_plan_create_charts(const void* const* T, const int8_t* tdt, const int64_t* vofs, const int64_t* tofs,
                           int32_t nc, int32_t nthreads, uva_plan** out);
int uva_plan_sizes(const uva_plan* plan, int64_t* sizes /* UVA_PLAN_NSIZES */);
/* Copies the plan into caller-owned HOST arrays (sizes from uva_plan_sizes):
 *   tri4      t*4   local a,b,c and island id
 *   tri_edge  t*3   global unique-edge id of edge k (corners k+1 -> k+2)
 *   sofs      nc+1  first SELL slice of each island
 *   slice_ptr nslices+1 first slot of each slice (32 rows per slice, width
 *             padded to a multiple of 4 slots)
 *   slot_col  nslots island-local column = solver ROW of the neighbour
 *             (padding: the row itself); slots of a row in vertex order
 *   slot_edge nslots global unique-edge id (padding: -1)
 *   slot_c    nslots LSCM boundary coupling H[i, j+n] (param.py:147-150)
 *   vt_ptr    n+1   incidence offsets; vt 3t entries f*3+corner, ascending
 *   vflags    n     bit0: endpoint of an edge used once (gpu.py:256-258)
 *                   bit1: endpoint of a twin-less half-edge (param.py:513-514)
 *   bofs      nc+1, bverts: sorted boundary source vertices (param.py:152)  */
int uva_plan_export(const uva_plan* plan, int32_t* tri4, int32_t* tri_edge, int32_t* sofs,
                    int32_t* slice_ptr, int32_t* slot_col, int32_t* slot_edge, float* slot_c,
                    int32_t* vt_ptr, int32_t* vt, uint8_t* vflags, int32_t* bofs, int32_t* bverts);
/* The same for islands [i0, i1) only, into the same full-size arrays (each
 * island's entries land in its own ranges; the closing offsets are written
 * with the range that ends at nc), so a caller can copy finished ranges to
 * the device while the next range is exported. The ranges of island i:
 * uva_plan_island_offsets (3*(nc+1) int64: first slice, first slot, first
 * boundary vertex of every island, then the totals).                       */
int uva_plan_export_range(const uva_plan* plan, int32_t i0, int32_t i1, int32_t* tri4, int32_t* tri_edge,
                          int32_t* sofs, int32_t* slice_ptr, int32_t* slot_col, int32_t* slot_edge, float* slot_c,
                          int32_t* vt_ptr, int32_t* vt, uint8_t* vflags, int32_t* bofs, int32_t* bverts);
int uva_plan_island_offsets(const uva_plan* plan, int64_t* out);
/* Solver row order (island-local): row_vert / vert_row (n each), rows per
 * coarse aggregate per island (0: none) and offsets of each island's m*m
 * coarse block (nc+1). Rows are grouped in compact breadth-first blobs of
 * agg_rows vertices so that aggregates are whole 32-row slices.           */
int uva_plan_export_rows(const uva_plan* plan, int32_t* row_vert, int32_t* vert_row, int32_t* agg_rows,
                         int32_t* cofs);
void uva_plan_destroy(uva_plan* plan);
/* Batch concatenation (host, parallel over charts). Replaces the per-chart
 * copies of gpu.Batch.__init__ (gpu.py:69-87): chart i's P (rows of 3,
 * float32/float64: pdt 0/1), T (rows of 3 local ids, int32/int64: tdt 0/1)
 * and optional U (rows of 2, udt -1: none -> zeros, 0: float32, 1: float64;
 * U or udt may be null: all zeros) land in P_out (n*3 FP64), T_out (t*3
 * int64; may be null, then T and tdt are not read) and U_out (n*2 FP64, may
 * be null) at vofs/tofs (nc+1 offsets).                                    */
int uva_concat_charts(int32_t nc, const void* const* P, const int8_t* pdt, const void* const* T,
                      const int8_t* tdt, const void* const* U, const int8_t* udt, const int64_t* vofs,
                      const int64_t* tofs, double* P_out, int64_t* T_out, double* U_out, int32_t nthreads);

/* --------------------------------------------------------------------------
 * Topology plan built on the device (csrc/dplan.cu): the arrays of
 * uva_plan_export / uva_plan_export_rows (same values, element for element)
 * from the island-local triangle lists, replacing the host plan's passes and
 * their upload (gpu.py:39-63 unique_edges / sym_csr, param.py:59-68 boundary
 * search; rows, slices and incidence have no reference counterpart). All
 * pointers are device memory. The host supplies what follows from the sizes
 * alone: agg_rows (rows per coarse aggregate: 0 up to 256 vertices, else the
 * smallest multiple of 64 giving at most 256 aggregates) and sofs (first
 * 32-row slice of each island). uva_dplan_build writes everything but the
 * slots and reports sizes = {E, nslots, nbverts, status}; status bit 0: a
 * vertex id outside its island, bit 1: an edge used by more than 127
 * triangles in one direction (both: the plan is invalid). uva_dplan_slots,
 * given the slot arrays (nslots each) and the same scratch, writes the
 * sliced-ELL slots. Capacities: tri4 4t, tri_edge 3t, slice_ptr nslices+1,
 * vt_ptr n+1, vt 3t, vflags n, bofs nc+1, bverts n, row_vert / vert_row n. */
typedef struct uva_dplan {
    int32_t nc, n, t, nslices;
    const int32_t* vofs;       /* nc+1, vofs[0] = 0 */
    const int32_t* tofs;       /* nc+1, tofs[0] = 0 */
    const int32_t* T;          /* t*3 island-local vertex ids               */
    const int32_t* agg_rows;   /* nc                                         */
    const int32_t* sofs;       /* nc+1                                       */
    int32_t* tri4;   int32_t* tri_edge; int32_t* slice_ptr; int32_t* vt_ptr; int32_t* vt;
    uint8_t* vflags; int32_t* bofs;     int32_t* bverts;    int32_t* row_vert; int32_t* vert_row;
    int64_t* sizes;            /* 4                                          */
    void* scratch;             /* uva_dplan_scratch_bytes, kept between calls */
    int64_t scratch_bytes;
} uva_dplan;

/* Host side of the upload: per-chart triangle arrays (int32 / int64
 * island-local ids, tdt 0 / 1) into one int32 array at tofs, in parallel;
 * UVA_E_ARG for an id outside the int32 range.                             */
int uva_concat_tris32(int32_t nc, const void* const* T, const int8_t* tdt, const int64_t* tofs, int32_t* out,
                      int32_t nthreads);
/* Per-chart float32 rows (width floats) into one float32 array at ofs, in
 * parallel (positions that are float32 upload as they are).               */
int uva_concat_rows32(int32_t nc, const void* const* src, const int64_t* ofs, int32_t width, float* out,
                      int32_t nthreads);
int uva_dplan_scratch_bytes(int64_t n, int64_t t, int64_t nslices, int64_t* bytes);
int uva_dplan_build(const uva_dplan* d, void* stream);
int uva_dplan_slots(const uva_dplan* d, int32_t* slot_col, int32_t* slot_edge, float* slot_c, void* stream);

/* --------------------------------------------------------------------------
 * Device batch descriptor: plain device pointers, filled by the host layer.
 * ------------------------------------------------------------------------ */
typedef struct uva_batch {
    int32_t nc, n, t, E, nslices, nslots, semantics, maxrows;
    /* topology (from the plan) */
    const int32_t* vofs;      const int32_t* tofs;      const int32_t* sofs;
    const int32_t* tri4;      const int32_t* tri_edge;
    const int32_t* slice_ptr; const int32_t* slot_col;  const int32_t* slot_edge;
    const float*   slot_c;    const int32_t* vt_ptr;    const int32_t* vt;
    const uint8_t* vflags;    const int32_t* bofs;      const int32_t* bverts;
    const int32_t* order;     /* nc island ids by class, largest first        */
    const int32_t* row_vert;  /* n: solver row -> vertex (island-local)       */
    const int32_t* vert_row;  /* n: vertex -> solver row (island-local)       */
    const int32_t* agg_rows;  /* nc: rows per coarse aggregate (0: none)      */
    const int32_t* cofs;      /* nc+1: offset of the island's m*m coarse block */
    float*  coarse_a;         /* cofs[nc] floats: inverse coarse ARAP operators,
                                 FP16 scaled to a largest entry of 1024, then
                                 the inverse scale (FP32)                      */
    float*  coarse_l;         /* 4*cofs[nc] floats: the same for LSCM          */
    double* coarse_work;      /* 4*cofs[nc]: FP64 workspace of the setup        */
    float*  cpart;            /* 2*nslices floats of solve scratch: the whole-GPU
                                 team of islands above 16,384 vertices keeps its
                                 grid barrier here (and its reduction slots in
                                 coarse_work, free after the setup)           */
    int32_t class_ofs[5];     /* host values: class c owns order[ofs[c]..ofs[c+1]) */
    /* geometry, written by uva_batch_setup */
    const double*  P;         /* n*3 positions (FP64)                          */
    double* frame;            /* t*4: x1, x2, y2, area                          */
    double* wtri;             /* t*4: w0, w1, w2 (half cotangents), ok (1/0)    */
    float*  tscale;           /* t: target size (Batch.shrink)                  */
    double* wedge;            /* E: summed edge weight                          */
    int32_t* slot_cw;         /* nslots*2: packed (column, FP32 weight bits)    */
    double* wdiag;            /* n (by solver row): FP64 row sum of the weights */
    float*  dinv;             /* n (by row): inverse of wdiag (pin row on the fly) */
    int32_t* pins;            /* nc*3: ARAP pin, LSCM p0, LSCM p1 (local ids)   */
    double* wpin;             /* nc: soft-pin weight                            */
    double* U;                /* n*2 UVs (FP64 master copy)                     */
    /* scratch (device, sized n / t) */
    double* x64;  double* b64;  double* rc;     /* x64, b64: max(n,nc)*2, by  */
                                                /* solver row;                */
                                                /* rc: t*3*2 corner RHS terms */
    float*  r32;  float*  d32;  float*  p32;  float* q32;
    uva_island_status* status;                  /* nc                         */
    int32_t* work;            /* >= 4 ints, zeroed by the callee per launch     */
    float*  hist;             /* 16*n floats (optional): the last 4 ARAP updates
                                 and their images under the operator, FP32 by
                                 solver row, for the start of each global step;
                                 null: 2 updates kept in p32/d32/q32/r32        */
} uva_batch;

/* Island size classes of one persistent launch (see uva_arap): islands are
 * solved by a whole 1024-thread CTA (more than UVA_CLASS_MID vertices), by a
 * 256-thread sub-team (more than UVA_CLASS_SMALL) or by one warp.           */
#define UVA_CLASS_BIG   8192   /* above: CG vectors in global memory          */
#define UVA_CLASS_MID   2048
#define UVA_CLASS_SMALL 256

typedef struct uva_solve_params {
    int32_t iters;            /* ARAP outer iterations                          */
    int32_t line_search;      /* 1: flip-safe step (param: only if flip-free)   */
    double  tol;              /* FP64 relative residual per column              */
    double  energy_tol;       /* >0: param.refine relative-energy stop          */
    double  inner_eta;        /* inner FP32 CG relative reduction floor         */
    int32_t max_inner;        /* inner CG iteration cap per refinement          */
    int32_t max_refine;       /* refinement cap per global step                 */
    int32_t threads;          /* threads per island team (0: autotuned)         */
    int32_t rev_ctas;         /* CTAs that start with the small-island classes
                                 (0: automatic, < 0: none)                      */
    int32_t fold_step;        /* 1: an island with a folded triangle (negative
                                 UV area, frame ok) at the start of an iteration
                                 takes the full step (engine/hier.py:549-552)   */
} uva_solve_params;

/* Frames, weights, matrix values, Jacobi diagonal, pins and pin weights.
 * Batch semantics: global wpin = max|w| (gpu.py:138); param: per island.   */
int uva_batch_setup(uva_batch* b, void* stream);
/* LSCM of every island (hard pins at the far boundary pair, param.py:136-169)
 * solved by FP32 PCG with FP64 residual refinement; writes b->U.           */
int uva_lscm(uva_batch* b, const uva_solve_params* prm, void* stream);
/* ARAP local/global iterations of every island in one persistent launch
 * (gpu.py:230-249 with semantics BATCH, param.py:379-414 with PARAM).      */
int uva_arap(uva_batch* b, const uva_solve_params* prm, void* stream);

/* Step graphs. No counterpart in the reference, which launches every kernel
 * of gpu.Batch.arap (gpu.py:230-249) from Python, one host sync per CG
 * iteration. Captures any subset of setup + LSCM + ARAP of one batch into a CUDA graph
 * (private stream, thread-local capture mode) and replays it with one
 * launch. The graph holds the batch's pointers and the parameters given at
 * creation: re-create it after changing either. Replays of one graph must
 * not overlap (they share the batch scratch). */
#define UVA_STEP_SETUP 1
#define UVA_STEP_LSCM  2
#define UVA_STEP_ARAP  4
typedef struct uva_graph uva_graph;
int uva_step_graph_create(uva_batch* b, int32_t parts, const uva_solve_params* lscm,
                          const uva_solve_params* arap, uva_graph** out);
int uva_graph_launch(uva_graph* g, void* stream);
int uva_graph_destroy(uva_graph* g);

/* SLIM iterations of every island (param.refine(method="slim"),
 * param.py:415-454 with _arap_rotations mode 1 :206-256 and the normal
 * equations of _assemble_weighted / _slim_system :341-377). PARAM semantics
 * only. prm: iters, energy_tol (refine's tol), inner_eta and max_inner (the
 * CG relative tolerance and iteration cap of each global step; the
 * reference solves exactly when 2n <= 220,000, else CG rtol 1e-6, at most
 * 500 iterations). A start with an inverted triangle is left unchanged
 * (status flag UVA_ST_NONFINITE), as the reference returns early.
 * scratch: uva_slim_scratch_bytes(b) bytes, 16-byte aligned.             */
int uva_slim_scratch_bytes(const uva_batch* b, int64_t* bytes);
int uva_slim(uva_batch* b, const uva_solve_params* prm, double* scratch, void* stream);

/* No counterpart in the reference. The same ARAP iterations as uva_arap, for
 * callers that cannot allocate device memory while they run (for example a
 * host application that owns a fixed device pool, or code that must not call
 * cudaMalloc between frames). It allocates nothing: the solver scratch of `b`
 * (x64, b64, rc, r32, d32, p32, q32, cpart, work, hist) is ignored and replaced by one
 * static device array of 7,602,432 bytes that every GPU loading the library
 * holds until exit. The caller still passes the inputs (topology, geometry,
 * pins, order) and the outputs (U, status). Limits: at most 32768 vertices
 * and 65536 triangles per call, else UVA_E_TOOBIG. The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress); make that first
 * call before any stream capture. All calls share the array and it keeps the
 * last call's contents (the work counter is cleared per call): calls that
 * overlap on the GPU, from any stream or thread, race and must be serialised
 * by the caller.                                                            */
int uva_arap_noalloc(const uva_batch* b, const uva_solve_params* prm, void* stream);

/* Batch utilities (gpu.py:145-299). */
int uva_orient_positive(uva_batch* b, void* stream);
int uva_repair_flips(uva_batch* b, int32_t rounds, void* stream);
int uva_flips_per_chart(const uva_batch* b, float* out /* nc */, void* stream);
int uva_signed_area(const uva_batch* b, const double* U, double* out /* t */, void* stream);
int uva_jacobians(const uva_batch* b, const double* U, double* out /* t*4 */, void* stream);
/* Serial in-order flip repair of param.repair_flips (param.py:477-516). */
int uva_repair_flips_serial(uva_batch* b, int32_t rounds, void* stream);
/* gpu.py:283-295: sel (t bytes, in/out) grown by `rings` vertex rings, then
 * tscale = max(tscale * factor, floor) on the selection; vmark: n bytes.   */
int uva_shrink(uva_batch* b, uint8_t* sel, uint8_t* vmark, int32_t rings, float factor, float floor_,
               void* stream);

/* --------------------------------------------------------------------------
 * Exact validation of exported float32 UVs (engine/validate.py:139-209,
 * _overlaps :95-136, _overlaps_strict :258-300; islands of
 * engine/metrics.py:91-103). Bit-exact FP64 predicates (no FMA contraction).
 * ------------------------------------------------------------------------ */
enum {
    UVA_VC_NONFINITE = 0,   /* UV rows with a non-finite coordinate          */
    UVA_VC_OUTSIDE,         /* UV rows outside [0,1]                         */
    UVA_VC_DEGENERATE,      /* has 3D area, zero UV area                     */
    UVA_VC_SLIVERS,         /* has 3D area, below float32 UV resolution      */
    UVA_VC_FLIPPED,         /* against the island's dominant orientation     */
    UVA_VC_MIRRORED,        /* islands with negative dominant orientation    */
    UVA_VC_ISLANDS,         /* islands                                       */
    UVA_VC_OVERLAP,         /* triangles in a positive-area overlap          */
    UVA_VC_CONTACTS,        /* strict-only overlaps (float32 contacts)       */
    UVA_VC_ISLANDS_OV,      /* islands holding an overlapping triangle       */
    UVA_VC_PAIRS,           /* candidate pairs with intersecting FP64 boxes  */
    UVA_VC_BIG,             /* triangles tested outside the grid (> 16 cells)*/
    UVA_VC_AMBIGUOUS,       /* islands whose orientation was re-summed exactly */
    UVA_VC_N = 16
};

typedef struct uva_val_desc {
    int32_t n, m;           /* vertices, triangles                            */
    int32_t grid;           /* grid cells per side (0: clip(sqrt(m)/2, 64, 4096)) */
    int32_t reserved;
    const double* V;        /* n*3 positions (FP64)                           */
    const float* UV;        /* n*2 exported UVs (float32)                     */
    const int32_t* F;       /* m*3                                            */
    double rel;             /* tolerant predicate, relative to edge^2 (1e-6)  */
    uint8_t* tflags;        /* out, m bytes rounded up to a multiple of 4:
                               1 has3d, 2 sliver, 4 skipped, 8 flipped,
                               16 overlap, 32 strict overlap                  */
    int32_t* labels;        /* out, m: island of each face (0..islands-1, by
                               smallest welded vertex id; the partition is the
                               reference's, its numbering depends on union order) */
    double* sa;             /* out, m: signed UV area                         */
    int64_t* counts;        /* out, UVA_VC_N counters                         */
    void* scratch;          /* device scratch of uva_validate_scratch_bytes   */
    int64_t scratch_bytes;
    int32_t shard, nshards; /* nshards > 1: test only the candidate pairs whose
                               first shared cell lies in cell rows
                               [G shard / nshards, G (shard + 1) / nshards);
                               0 / 0: all pairs                               */
} uva_val_desc;

int uva_validate_scratch_bytes(int64_t n, int64_t m, int32_t grid, int64_t* bytes);
int uva_validate(const uva_val_desc* d, void* stream);
/* Several shards (one per GPU): every shard runs
 * uva_validate with its band, the overlap bits 16 and 32 of tflags are
 * merged across shards (OR: an all-reduce MAX of each bit) and the
 * UVA_VC_PAIRS counts summed; then uva_validate_finish, with the same
 * descriptor and scratch, recounts UVA_VC_OVERLAP, UVA_VC_CONTACTS and
 * UVA_VC_ISLANDS_OV from the merged bits. The other counts, labels and
 * flags do not depend on the band.                                         */
int uva_validate_finish(const uva_val_desc* d, void* stream);
/* engine/metrics.py:91-103: face islands; weld != 0 merges vertices with
 * identical float32 (position, uv) bytes. count: device int64.
 * Scratch: uva_validate_scratch_bytes(n, m, 0).                            */
int uva_islands(const double* V, const float* UV, const int32_t* F, int32_t n, int32_t m, int32_t weld,
                int32_t* labels, int64_t* count, void* scratch, int64_t scratch_bytes, void* stream);
/* engine/validate.py:212-226: overlap flags (bit 16 of tflags, m bytes
 * rounded up to a multiple of 4) of one chart whose FP64 UVs the caller has
 * normalised to [0, 0.999999]; triangles with |area| <= 1e-14 are skipped.
 * Scratch: uva_validate_scratch_bytes(n, m, 0).                            */
int uva_chart_overlaps(const double* U, const int32_t* F, int32_t n, int32_t m, uint8_t* tflags,
                       void* scratch, int64_t scratch_bytes, void* stream);

/* --------------------------------------------------------------------------
 * Gutter and coverage rasters (engine/metrics.py:13-62, 314-373).
 * ------------------------------------------------------------------------ */
int uva_gutter_scratch_bytes(int32_t res, int64_t m, int64_t* bytes);
/* Label raster (last triangle wins, like the reference's serial loop) into
 * img (res*res int32, -1 empty) and the gap between islands from an exact,
 * radius-limited Euclidean distance transform that breaks ties like
 * scipy.ndimage.distance_transform_edt (smallest column, then row).
 * out (device, 4 doubles): [0] min d(p)+d(q) over 4-neighbour pairs with
 * different nearest labels and both distances <= radius (1e300: none),
 * [1] filled texels, [2] 1 if two islands touch, [3] radius. The gap is exact
 * when out[0] <= radius; otherwise call again with a larger radius. UV is
 * FP64 as given (validate_uvs passes float32-rounded values).             */
int uva_gutter(const double* UV, const int32_t* F, const int32_t* labels, int32_t m, int32_t res, int32_t radius,
               int32_t* img, void* scratch, int64_t scratch_bytes, double* out, void* stream);
/* Texel-centre overlaps of one chart (engine/overlapfix.py:135-224 and
 * 263-275): uv (n*2 FP64) already normalised like the reference,
 * (U - lo) / ext * 0.999; F (m*3) rows of uv; the coverage rule of
 * uva_raster_counts. flags (device, m bytes, may be null): 1 if the triangle
 * shares a covered texel centre with another triangle (_raster_all). pair
 * (device, 2 int32, may be null): the first pair the reference's serial
 * raster meets (_raster_pair): (earlier triangle, later triangle), or -1 -1.
 * Scratch: uva_gutter_scratch_bytes(res, m).                               */
int uva_overlap_raster(const double* uv, const int32_t* F, int32_t m, int32_t res, uint8_t* flags, int32_t* pair,
                       void* scratch, int64_t scratch_bytes, void* stream);
/* Coverage counts per texel centre with the top-left rule, saturating at 255
 * (uv: FP64 as given); stats (device, 2 int64): covered, covered twice.    */
int uva_raster_counts(const double* uv, const int32_t* F, int32_t m, int32_t res, uint8_t* counts, int64_t* stats,
                      void* scratch, int64_t scratch_bytes, void* stream);

/* --------------------------------------------------------------------------
 * Distortion metrics (engine/metrics.py:106-210, engine/param.py:520-551).
 * ------------------------------------------------------------------------ */
/* Weighted quantile per segment (argsort, cumsum, searchsorted semantics of
 * metrics._wquantile :107-112): the smallest x whose cumulative weight
 * reaches q * total; weight-0 entries are ignored; seg may be null (one
 * segment). out: nseg doubles (device), NaN for an empty segment.          */
int uva_wquantile_scratch_bytes(int32_t nseg, int64_t* bytes);
int uva_wquantile(const double* x, const double* w, const int32_t* seg, int32_t n, int32_t nseg, double q,
                  double* out, void* scratch, int64_t scratch_bytes, void* stream);
int uva_metrics_scratch_bytes(int64_t m, int64_t n_islands, int64_t* bytes);
/* distortion_report (metrics.py:148-210). out (device, 32 doubles):
 * [0] sum a3, [1] sum |sa|, [2] collapsed, [3] collapsed w, [4] aniso*w (ok),
 * [5] w (aniso ok), [6] angle*w (valid), [7] w (valid), [8] lg*w (ok),
 * [9] w (ok), [10] stretch^2*w (ok), [11] lc*w (ok), [12] flipped,
 * [13] flipped w, [16] mirrored islands, [17] sum ia3, [24] anisotropy p95,
 * [25] log2 density-ratio p95, [26] log2 chart-area p95, [27] log2 island
 * density p95. islands may be null. per_tri (device, m*6, may be null):
 * s1, s2, signed UV area, 3D area, good, angle error (triangle_jacobians). */
int uva_distortion_report(const double* V, const double* UV, const int32_t* F, const int32_t* islands,
                          int32_t n, int32_t m, int32_t n_islands, double* out, double* per_tri,
                          void* scratch, int64_t scratch_bytes, void* stream);
int uva_quality_scratch_bytes(int64_t t, int64_t nc, int64_t* bytes);
/* chart_quality (param.py:520-551) of every island of a PARAM-semantics
 * batch. out (device, nc*8): flips, aniso_p95, aniso_mean, area_p95,
 * area_logdev, stretch, scale, area. per_aniso, per_area: t doubles.       */
int uva_chart_quality(const uva_batch* b, double* out, double* per_aniso, double* per_area, void* scratch,
                      int64_t scratch_bytes, void* stream);

/* --------------------------------------------------------------------------
 * Per-chart helpers of engine/param.py (one chart, global int64 triangles).
 * ------------------------------------------------------------------------ */
enum {
    UVA_OP_FRAMES = 0,      /* local_frames :19-32  -> out X (t*6), out2 area */
    UVA_OP_COTS,            /* cot_weights :35-44   X -> out (t*3)            */
    UVA_OP_SIGNED_AREA,     /* signed_areas :97-99  U -> out (t)              */
    UVA_OP_ROTATIONS,       /* _arap_rotations mode 0 :206-233 -> out (t*4)   */
    UVA_OP_RHS,             /* _arap_rhs :457-474   -> out (n*2)              */
    UVA_OP_MAX_STEP,        /* _max_step :259-291   U, D -> out (1)           */
    UVA_OP_ENERGY           /* _energy :294-319, kind = arg -> out (1)        */
};
/* UVA_OP_ROTATIONS: arg = mode; mode 1 writes the SLIM weight matrices
 * (param.py:234-255) to out2 (t*4).                                      */
int uva_chart_op(int32_t op, int32_t arg, const double* P, const int64_t* T, const double* U, const double* D,
                 const double* X, const double* cots, const double* R, const double* area, int32_t n, int32_t t,
                 double* out, double* out2, void* stream);
/* SPDSolver (param.py:103-132): FP64 Jacobi-PCG on a CSR SPD matrix, one
 * right-hand side per column (b, x: ncol*n column-major), warm start in x,
 * stop at ||r|| <= tol ||b||. scratch: 3*n*ncol doubles; iters: ncol.      */
int uva_csr_pcg(int32_t n, const int32_t* rowptr, const int32_t* col, const double* val, const double* b, double* x,
                int32_t ncol, double tol, int32_t maxiter, double* scratch, int32_t* iters, void* stream);
/* The same on a block-diagonal SPD CSR matrix (n rows): block s owns rows
 * [sys_ofs[s], sys_ofs[s+1]) and only its own columns; each block is solved
 * by its own CTA to ||r_s|| <= tol ||b_s||. scratch: 3n doubles; iters:
 * nsys (device). Used by hier.Solver.lscm, one block per chart.           */
int uva_csr_pcg_blocks(int32_t nsys, const int32_t* sys_ofs, int32_t n, const int32_t* rowptr, const int32_t* col,
                       const double* val, const double* b, double* x, double tol, int32_t maxiter, double* scratch,
                       int32_t* iters, void* stream);

/* hier.Solver.lscm (engine/hier.py:534-585) with the system assembled on
 * the device: half-cot weights of the mesh faces `faces` (rows of F, (nf,3),
 * positions V (nvp,3)), the soft-pinned LSCM system of every chart (UV
 * corners CV (t,3), chart per face, directed boundary edges ba -> bb (nb)),
 * one row per UV vertex shared by its u and v unknowns, then FP64
 * Jacobi-PCG per chart (one CTA) to ||r_c|| <= tol ||b_c|| (at most maxiter
 * iterations). U (nv,2): the solution, U0 for UV vertices no face names and
 * for non-finite values. flags (one device int32, zeroed here): bit 0 a UV
 * vertex or boundary edge joins two charts, bit 1 an index out of range
 * (faces, F, CV, ba, bb), bit 2 a chart id out of range; offending entries
 * are left out, so the solve stays in bounds. Index arrays are int32.
 * scratch: uva_hier_lscm_scratch_bytes.                                    */
int uva_hier_lscm_scratch_bytes(int64_t nv, int64_t t, int64_t nb, int32_t nchart, int64_t* bytes);
int uva_hier_lscm(const double* V, int64_t nvp, const int32_t* F, int64_t nf, const int32_t* faces, const int32_t* CV,
                  const int32_t* chart, int64_t t, int64_t nv, int32_t nchart, const double* U0, const int32_t* ba,
                  const int32_t* bb, int64_t nb, double tol, int32_t maxiter, void* scratch, int64_t scratch_bytes,
                  double* U, int32_t* flags, void* stream);

/* --------------------------------------------------------------------------
 * Distortion energies with backward passes (engine/param.py:294-319):
 * kind 0 ARAP, kind 1 symmetric Dirichlet (inf for inverted triangles),
 * frames from P as param.local_frames; per island.
 * ------------------------------------------------------------------------ */
int uva_energy_fwd(const uva_batch* b, const double* P, const double* U, int32_t kind, double* e_isl,
                   double* e_tri, void* stream);
/* dE/dU (n*2) and, if gP is not null, dE/dP (n*3); gscale (nc, may be null)
 * scales each island's energy (the upstream gradient).                     */
int uva_energy_bwd(const uva_batch* b, const double* P, const double* U, int32_t kind, const double* gscale,
                   double* gU, double* gP, void* stream);
/* p95-stretch refinement: `steps` Jacobi-preconditioned, flip-safe, monotone
 * descent steps on the symmetric Dirichlet energy of every island; updates
 * b->U; e_isl (nc) gets the final energies. scratch: 8n + 8nc + n + 2
 * doubles.                                                                 */
int uva_sd_refine(uva_batch* b, int32_t steps, int32_t halvings, double cap, double* e_isl, void* scratch,
                  void* stream);

/* --------------------------------------------------------------------------
 * Boundary self-intersection checks of UV charts, batched over charts.
 * UVA_SEG_COUNT replaces engine/charts.py:547-608 (boundary_intersections /
 * _seg_intersections): the number of crossing segment pairs counted once per
 * grid cell the pair shares, with the reference's grid (lo and extent over
 * the chart's UV rows, cell = max(4 median length, extent / 512, 1e-30)),
 * capped at max(max_report, 1). UVA_SEG_ANY replaces engine/hier.py:183-266
 * (_hit) as called by chart_checks (:270-353): 1 if any two segments
 * cross, also when the endpoints' extent is not below 1e300.
 * UVA_SEG_ANY_ALL is the same test as called by charts_collide (:183-225),
 * which has no extent check. UVA_SEG_FIRST replaces engine/overlapfix.py:
 * 44-84 (_first_hit, as called by collision :283-296): the first crossing
 * pair in the reference's scan (cells in row-major order, then segment
 * order), with the count's grid at extent / 1024.
 * A crossing: the endpoints share no coordinates exactly and each segment's
 * endpoints lie strictly on both sides of the other, beyond 1e-9 times its
 * squared length (FP64, no fused multiply-add).
 * ------------------------------------------------------------------------ */
#define UVA_SEG_COUNT 0
#define UVA_SEG_ANY   1
#define UVA_SEG_ANY_ALL 2
#define UVA_SEG_FIRST   3

typedef struct uva_seg_desc {
    int32_t nc;             /* charts                                         */
    int32_t nseg;           /* boundary segments of all charts                */
    int32_t n;              /* rows of U                                      */
    int32_t mode;           /* UVA_SEG_COUNT, _ANY, _ANY_ALL or _FIRST        */
    int32_t max_report;     /* UVA_SEG_COUNT: cap of the count                */
    int32_t reserved;
    const double* U;        /* n*2 FP64 UVs                                   */
    const int32_t* vofs;    /* nc+1: UV rows of chart c (UVA_SEG_COUNT grid)  */
    const int32_t* seg_ofs; /* nc+1: segments of chart c                      */
    const int32_t* seg;     /* nseg*2: rows (a, b) of U, segment a -> b       */
    int64_t* out;           /* out, nc. COUNT: the capped count, -1 for a
                               chart with >= 3 segments and non-finite UVs
                               (the reference raises), -2 for rows outside the
                               chart; ANY: 0 or 1 (-2 for rows outside U)     */
    void* scratch;          /* device scratch of uva_seg_scratch_bytes        */
    int64_t scratch_bytes;
} uva_seg_desc;

int uva_seg_scratch_bytes(int32_t nc, int32_t nseg, int64_t* bytes);
int uva_boundary_hits(const uva_seg_desc* d, void* stream);
/* Directed boundary half-edges of every island of a device batch
 * (engine/param.py:59-68 per island): seg_ofs (device, nc+1) and seg
 * (device, capacity 3t*2: rows of U, island by island; the order inside an
 * island is unspecified, which no check depends on). Scratch:
 * uva_batch_boundary_scratch_bytes.                                        */
int uva_batch_boundary_scratch_bytes(const uva_batch* b, int64_t* bytes);
int uva_batch_boundary(const uva_batch* b, int32_t* seg_ofs, int32_t* seg, void* scratch, int64_t scratch_bytes,
                       void* stream);

/* --------------------------------------------------------------------------
 * Mesh edges and sparse helpers of engine/gpu.py:16-63 and
 * engine/param.py:59-68, on the device (csrc/edges.cu).
 * ------------------------------------------------------------------------ */
/* gpu.unique_edges (gpu.py:39-49). T: t*3 int64 vertex ids in [0, n).
 * Writes the E unique undirected edges in ascending (lo, hi) order: ea, eb
 * (lo <= hi) and cnt (triangles using the edge), each of capacity 3t;
 * inv (3t): unique edge of half-edge k*t + f, the edge of triangle f
 * opposite corner k (corners k+1, k+2). *nedges (device int64) = E, or -1
 * when a vertex id is outside [0, n). Scratch:
 * uva_unique_edges_scratch_bytes.                                          */
int uva_unique_edges_scratch_bytes(int64_t n, int64_t t, int64_t* bytes);
int uva_unique_edges(const int64_t* T, int64_t t, int64_t n, int64_t* ea, int64_t* eb, int64_t* inv, int64_t* cnt,
                     int64_t* nedges, void* scratch, int64_t scratch_bytes, void* stream);
/* gpu.sym_csr (gpu.py:52-63): the n x n symmetric matrix with off[e] at
 * (ea[e], eb[e]) and (eb[e], ea[e]) and diag on the diagonal, as CSR with
 * int32 row offsets (crow, n+1) and columns (col, 2 ne + n), rows sorted by
 * column. dtype 0: float32 values, 1: float64. *status (device int32) = 1
 * when an endpoint is outside [0, n).                                      */
int uva_sym_csr_scratch_bytes(int64_t n, int64_t* bytes);
int uva_sym_csr(int64_t n, int64_t ne, const int64_t* ea, const int64_t* eb, const void* off, const void* diag,
                int32_t dtype, int32_t* crow, int32_t* col, void* val, int32_t* status, void* scratch,
                int64_t scratch_bytes, void* stream);
/* gpu.spmm (gpu.py:23-28): Y = A X for an int32 CSR matrix (nrows rows,
 * nnz entries) and k dense columns (X, Y row-major with k columns). dtype
 * 0: float32, 1: float64 (values, X and Y).                               */
int uva_csr_spmm(int32_t nrows, int32_t k, int64_t nnz, const int32_t* crow, const int32_t* col, const void* val,
                 const void* X, void* Y, int32_t dtype, void* stream);
/* param.boundary_edges_oriented (param.py:59-68): keep (3t bytes) = 1 for
 * the directed half-edge k*t + f (corners k -> k+1 of triangle f) whose
 * reverse half-edge is absent. *status = 1 for a vertex id outside
 * [0, 2^31).                                                               */
int uva_boundary_mask_scratch_bytes(int64_t t, int64_t* bytes);
int uva_boundary_mask(const int64_t* T, int64_t t, uint8_t* keep, int32_t* status, void* scratch,
                      int64_t scratch_bytes, void* stream);
/* gpu.Batch._edges (gpu.py:128-129) of a device batch, from the plan's
 * unique-edge numbering (which is the ascending global (lo, hi) order):
 * ea, eb, cnt (b->E int64 each).                                           */
int uva_batch_edges(const uva_batch* b, int64_t* ea, int64_t* eb, int64_t* cnt, void* stream);

/* --------------------------------------------------------------------------
 * Whole-mesh reports of engine/metrics.py:227-311 (csrc/report.cu).
 * ------------------------------------------------------------------------ */
/* metrics.seam_report (metrics.py:227-261). V (n*3 FP64), F (m*3 int64,
 * numpy indexing: -n <= id < n), UV (n*2 FP64), weld (n int64 keys, or null:
 * vertices with equal position values are one vertex). out (device, 6
 * doubles): seam_edges, seam_length, open_boundary_edges,
 * open_boundary_length, nonmanifold_edge_groups, surface_area. *status = 1
 * for a face index out of range.                                           */
int uva_seam_report_scratch_bytes(int64_t n, int64_t m, int64_t* bytes);
int uva_seam_report(const double* V, int64_t n, const int64_t* F, int64_t m, const double* UV, const int64_t* weld,
                    double* out, int32_t* status, void* scratch, int64_t scratch_bytes, void* stream);
/* Exact per-corner equality of attribute rows (metrics.py:264-286,
 * validate.py:191-199): rows A[fa[i]] and B[fb[i]], i < m, w columns each,
 * compared by value as np.array_equal does (NaN unequal, -0.0 == 0.0;
 * floats compared as FP64, integers exactly). Element codes: 0 f32, 1 f64,
 * 2 f16, 3 u8, 4 i8, 5 i16, 6 u16, 7 i32, 8 u32, 9 i64, 10 u64, 11 bool.
 * *result (device int32): bit 0 a row differs, bit 1 an index is outside
 * its array (numpy indexing).                                              */
int uva_corners_equal(const void* A, int32_t adt, int64_t na, const int64_t* fa, const void* B, int32_t bdt,
                      int64_t nb, const int64_t* fb, int64_t m, int32_t w, int32_t* result, void* stream);
/* out[seg[i]] = sum of x[i*stride] (np.bincount with weights,
 * metrics.py:306-307); *status = 1 for a segment id outside [0, nseg).   */
int uva_segment_sum(const double* x, int64_t stride, const int32_t* seg, int64_t m, int32_t nseg, double* out,
                    int32_t* status, void* stream);

/* --------------------------------------------------------------------------
 * Raster atlas packing, one attempt at one texel scale (pack.py:53-363,
 * csrc/pack.cu). A mask source is a chart at one pre-rotation angle
 * (source c * nangles + a); a variant is a source turned by 0..3 quarter
 * turns (variant c * nk + k, k = a * nturns + turn). The host gives what
 * follows from the sizes alone: each source's texel scale and mask size
 * (h = ceil(max y * scale + pad + pad) + 1, w likewise, pack.py:84-86), the
 * mask offsets, the variants (var_src -1: none) and their row offsets.
 * uva_pack_masks writes the masks (conservative raster, square dilation by
 * pad), the runs of every variant row (run_ofs, run_a / run_b first and last
 * cell), the longest run of each row, the set cells of every variant
 * (var_area) and a key naming its row with the longest run; status[2] = 1
 * when run_cap was too small (a row of w cells has at most (w + 1) / 2
 * runs). uva_pack_place places the charts in `order` on a G x G page by
 * first fit (pack.py:124-156, 312-359) in one cooperative launch and
 * writes placement (variant, x, y per chart), R (per cell the free run to
 * its right), rowmax, occupied (cells with R = 0) and status[0]: 0 all
 * placed, bit 0 a chart did not fit (status[1]: its position in order),
 * bit 1 a grid barrier timed out. uva_pack_uv writes the UVs of all charts
 * (pack.py:541-549): (U s) dens + pad inside the mask, turned, moved by
 * (x, y), over G; out is nv x 2 at the chart offsets cofs. All pointers
 * are device memory. G at most 8192, nk at most 64.                       */
typedef struct uva_pack_attempt {
    int32_t nsrc, nc, nk, G, pad, reserved;
    int64_t ntri, ncells, nrows, run_cap;
    const double* V;           /* oriented source coordinates, 2 per vertex  */
    const int64_t* vofs;       /* nsrc+1 vertex offsets of the sources       */
    const int32_t* T;          /* ntri*3 source-local vertex ids             */
    const int64_t* tofs;       /* nsrc+1 triangle offsets                    */
    const double* scale;       /* nsrc texel scales                          */
    const int32_t* hw;         /* nsrc*2 mask height, width                  */
    const int64_t* mofs;       /* nsrc+1 mask byte offsets, mofs[nsrc] = ncells */
    const int32_t* var_src;    /* nc*nk source of every variant, -1: none    */
    const int32_t* var_turn;   /* nc*nk quarter turns                        */
    const int64_t* var_row;    /* nc*nk+1 first row of every variant         */
    const int64_t* order;      /* nc charts in placing order                 */
    uint8_t* mask;             /* ncells                                     */
    int32_t* row_need;         /* nrows longest run                          */
    int32_t* run_ofs;          /* nrows+1                                    */
    int32_t* run_a;            /* run_cap                                    */
    int32_t* run_b;            /* run_cap                                    */
    int64_t* var_area;         /* nc*nk                                      */
    int64_t* var_key;          /* nc*nk                                      */
    int32_t* R;                /* G*G                                        */
    int32_t* rowmax;           /* G                                          */
    int32_t* placement;        /* nc*3                                       */
    int32_t* status;           /* 4                                          */
    int64_t* occupied;         /* 1                                          */
    void* scratch;             /* uva_pack_scratch_bytes                     */
    int64_t scratch_bytes;
} uva_pack_attempt;

int uva_pack_scratch_bytes(int64_t ntri, int64_t ncells, int64_t nrows, int32_t nk, int32_t G, int64_t* bytes);
int uva_pack_masks(const uva_pack_attempt* a, void* stream);
/* blocks_per_sm: resident blocks of the placement launch per SM (0: 4). */
int uva_pack_place(const uva_pack_attempt* a, int32_t blocks_per_sm, void* stream);
/* 1 to 4 independent attempts on the same page size in one cooperative
 * launch, the blocks shared out between them (the probes of one round of
 * the k-ary scale search, pack.py:418-445).                               */
int uva_pack_place_pages(const uva_pack_attempt* const* attempts, int32_t n, int32_t blocks_per_sm, void* stream);
int uva_pack_uv(const uva_pack_attempt* a, int32_t nangles, int32_t nturns, const int64_t* cofs, int64_t nv,
                double s, const double* dens, double* out, void* stream);

/* Library info. */
const char* uva_last_error(void);
int uva_version(void);

#ifdef __cplusplus
}
#endif
#endif /* UVA_B200_H */
