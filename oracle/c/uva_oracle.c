/*
 * Oracle (test infrastructure only): plain C restatement of the reference's
 * serial / numba validation loops, compiled with -ffp-contract=off so every
 * FP64 operation rounds like the reference's numba build (no fused
 * multiply-add). Built by oracle/build_oracle.py into oracle/liboracle_c.so.
 *
 *   uvo_overlaps       engine/validate.py:95-136 (_overlaps) and :258-300
 *                      (_overlaps_strict): cell boxes int(u*G) clamped,
 *                      serial CSR binning, each pair once in the first shared
 *                      cell, cell-box reject, exact predicates :21-91, :232-255
 *   uvo_raster_labels  engine/metrics.py:315-345 (last triangle wins)
 *   uvo_raster_counts  engine/metrics.py:13-54 (top-left rule, saturating)
 *   uvo_pack_raster    engine/pack.py:52-79 (conservative chart raster)
 *   uvo_pack_try       engine/pack.py:123-156, 232-256, 312-359 (greedy
 *                      first fit of every chart, serial, with the free-run
 *                      and occupied-run tables and the run-skipping scan)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static const double ULP = 5.9604644775390625e-08; /* 2^-24 */

static inline double orient(double ax, double ay, double bx, double by, double cx, double cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}
static inline double dmax(double a, double b) { return a > b ? a : b; }

static int same(const double* U, int64_t i, int64_t j) { return U[2 * i] == U[2 * j] && U[2 * i + 1] == U[2 * j + 1]; }

static int strict_inside(double px, double py, double ax, double ay, double bx, double by, double cx, double cy,
                         double rel) {
    double l = dmax((bx - ax) * (bx - ax) + (by - ay) * (by - ay),
                    dmax((cx - bx) * (cx - bx) + (cy - by) * (cy - by), (ax - cx) * (ax - cx) + (ay - cy) * (ay - cy)));
    double eps = rel > 0 ? dmax(rel * l, 4.0 * ULP * sqrt(l)) : 0.0;
    double d1 = orient(ax, ay, bx, by, px, py), d2 = orient(bx, by, cx, cy, px, py), d3 = orient(cx, cy, ax, ay, px, py);
    if (d1 > eps && d2 > eps && d3 > eps) return 1;
    if (d1 < -eps && d2 < -eps && d3 < -eps) return 1;
    return 0;
}

static int proper_cross(double ax, double ay, double bx, double by, double cx, double cy, double dx, double dy,
                        double rel) {
    double l1 = (bx - ax) * (bx - ax) + (by - ay) * (by - ay), l2 = (dx - cx) * (dx - cx) + (dy - cy) * (dy - cy);
    double e1 = dmax(rel * l1, 4.0 * ULP * sqrt(l1)), e2 = dmax(rel * l2, 4.0 * ULP * sqrt(l2));
    double o1 = orient(ax, ay, bx, by, cx, cy), o2 = orient(ax, ay, bx, by, dx, dy);
    double o3 = orient(cx, cy, dx, dy, ax, ay), o4 = orient(cx, cy, dx, dy, bx, by);
    return ((o1 > e1 && o2 < -e1) || (o1 < -e1 && o2 > e1)) && ((o3 > e2 && o4 < -e2) || (o3 < -e2 && o4 > e2));
}

#define X(i) U[2 * (i)]
#define Y(i) U[2 * (i) + 1]

static int tri_overlap(const double* U, const int64_t* F, int64_t s, int64_t t, double rel) {
    const int64_t* a = F + 3 * s;
    const int64_t* b = F + 3 * t;
    int shared = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (same(U, a[i], b[j])) { shared++; break; }
    if (shared == 3) return 0;
    for (int i = 0; i < 3; ++i) {
        int64_t p0 = a[i], p1 = a[(i + 1) % 3];
        for (int j = 0; j < 3; ++j) {
            int64_t q0 = b[j], q1 = b[(j + 1) % 3];
            if (same(U, p0, q0) || same(U, p0, q1) || same(U, p1, q0) || same(U, p1, q1)) continue;
            if (proper_cross(X(p0), Y(p0), X(p1), Y(p1), X(q0), Y(q0), X(q1), Y(q1), rel)) return 1;
        }
    }
    for (int i = 0; i < 3; ++i) {
        int64_t v = a[i];
        if (!(same(U, v, b[0]) || same(U, v, b[1]) || same(U, v, b[2])))
            if (strict_inside(X(v), Y(v), X(b[0]), Y(b[0]), X(b[1]), Y(b[1]), X(b[2]), Y(b[2]), rel)) return 1;
        v = b[i];
        if (!(same(U, v, a[0]) || same(U, v, a[1]) || same(U, v, a[2])))
            if (strict_inside(X(v), Y(v), X(a[0]), Y(a[0]), X(a[1]), Y(a[1]), X(a[2]), Y(a[2]), rel)) return 1;
    }
    double cx = (X(a[0]) + X(a[1]) + X(a[2])) / 3.0, cy = (Y(a[0]) + Y(a[1]) + Y(a[2])) / 3.0;
    if (strict_inside(cx, cy, X(b[0]), Y(b[0]), X(b[1]), Y(b[1]), X(b[2]), Y(b[2]), rel)) return 1;
    cx = (X(b[0]) + X(b[1]) + X(b[2])) / 3.0; cy = (Y(b[0]) + Y(b[1]) + Y(b[2])) / 3.0;
    return strict_inside(cx, cy, X(a[0]), Y(a[0]), X(a[1]), Y(a[1]), X(a[2]), Y(a[2]), rel);
}

static int tri_overlap_strict(const double* U, const int64_t* F, int64_t s, int64_t t) {
    const int64_t* a = F + 3 * s;
    const int64_t* b = F + 3 * t;
    int shared = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (same(U, a[i], b[j])) { shared++; break; }
    if (shared == 3) return 0;
    for (int i = 0; i < 3; ++i) {
        int64_t p0 = a[i], p1 = a[(i + 1) % 3];
        for (int j = 0; j < 3; ++j) {
            int64_t q0 = b[j], q1 = b[(j + 1) % 3];
            if (same(U, p0, q0) || same(U, p0, q1) || same(U, p1, q0) || same(U, p1, q1)) continue;
            double o1 = orient(X(p0), Y(p0), X(p1), Y(p1), X(q0), Y(q0));
            double o2 = orient(X(p0), Y(p0), X(p1), Y(p1), X(q1), Y(q1));
            double o3 = orient(X(q0), Y(q0), X(q1), Y(q1), X(p0), Y(p0));
            double o4 = orient(X(q0), Y(q0), X(q1), Y(q1), X(p1), Y(p1));
            if (o1 * o2 < 0 && o3 * o4 < 0) return 1;
        }
    }
    return 0;
}

static int64_t cell_of(double u, int64_t G) {
    double s = u * (double)G;
    int64_t c;
    if (s != s) c = 0;   /* skipped triangles never reach here */
    else if (s >= 9.2e18) c = G - 1;
    else if (s <= -9.2e18) c = 0;
    else c = (int64_t)s;   /* truncation, like int() */
    return c < 0 ? 0 : (c > G - 1 ? G - 1 : c);
}

/* Returns the number of tested candidate pairs (cell boxes intersecting).
 * Only cells of rows [band_lo, band_hi) are scanned: every pair is tested
 * in its first shared cell, so bands that cover the rows once test every
 * pair once (the sharded validation). */
int64_t uvo_overlaps_band(const double* U, const int64_t* F, const uint8_t* skip, int64_t m, int64_t G, double rel,
                          int strict, int64_t band_lo, int64_t band_hi, uint8_t* flag);

int64_t uvo_overlaps(const double* U, const int64_t* F, const uint8_t* skip, int64_t m, int64_t G, double rel,
                     int strict, uint8_t* flag) {
    return uvo_overlaps_band(U, F, skip, m, G, rel, strict, 0, G, flag);
}

int64_t uvo_overlaps_band(const double* U, const int64_t* F, const uint8_t* skip, int64_t m, int64_t G, double rel,
                          int strict, int64_t band_lo, int64_t band_hi, uint8_t* flag) {
    int64_t* x0 = malloc(sizeof(int64_t) * (size_t)m * 4);
    int64_t *x1 = x0 + m, *y0 = x0 + 2 * m, *y1 = x0 + 3 * m;
    for (int64_t t = 0; t < m; ++t) {
        const int64_t* f = F + 3 * t;
        double mnx = fmin(X(f[0]), fmin(X(f[1]), X(f[2]))), mxx = fmax(X(f[0]), fmax(X(f[1]), X(f[2])));
        double mny = fmin(Y(f[0]), fmin(Y(f[1]), Y(f[2]))), mxy = fmax(Y(f[0]), fmax(Y(f[1]), Y(f[2])));
        x0[t] = cell_of(mnx, G); x1[t] = cell_of(mxx, G); y0[t] = cell_of(mny, G); y1[t] = cell_of(mxy, G);
    }
    int64_t* cnt = calloc((size_t)(G * G + 1), sizeof(int64_t));
    for (int64_t t = 0; t < m; ++t) {
        if (skip[t]) continue;
        for (int64_t gy = y0[t]; gy <= y1[t]; ++gy)
            for (int64_t gx = x0[t]; gx <= x1[t]; ++gx) cnt[gy * G + gx + 1]++;
    }
    for (int64_t k = 1; k <= G * G; ++k) cnt[k] += cnt[k - 1];
    int64_t* items = malloc(sizeof(int64_t) * (size_t)(cnt[G * G] + 1));
    int64_t* fill = malloc(sizeof(int64_t) * (size_t)(G * G));
    memcpy(fill, cnt, sizeof(int64_t) * (size_t)(G * G));
    for (int64_t t = 0; t < m; ++t) {
        if (skip[t]) continue;
        for (int64_t gy = y0[t]; gy <= y1[t]; ++gy)
            for (int64_t gx = x0[t]; gx <= x1[t]; ++gx) { int64_t c = gy * G + gx; items[fill[c]++] = t; }
    }
    memset(flag, 0, (size_t)m);
    int64_t tested = 0;
    /* cells in parallel, like the reference's prange over cells */
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tested)
    for (int64_t c = band_lo * G; c < band_hi * G; ++c) {
        int64_t cy = c / G, cx = c % G;
        for (int64_t p = cnt[c]; p < cnt[c + 1]; ++p) {
            int64_t s = items[p];
            for (int64_t q = p + 1; q < cnt[c + 1]; ++q) {
                int64_t t = items[q];
                if ((x0[s] > x0[t] ? x0[s] : x0[t]) != cx || (y0[s] > y0[t] ? y0[s] : y0[t]) != cy) continue;
                if (x0[s] > x1[t] || x0[t] > x1[s] || y0[s] > y1[t] || y0[t] > y1[s]) continue;
                ++tested;
                int hit = strict ? tri_overlap_strict(U, F, s, t) : tri_overlap(U, F, s, t, rel);
                if (hit) {
                    __atomic_store_n(flag + s, (uint8_t)1, __ATOMIC_RELAXED);
                    __atomic_store_n(flag + t, (uint8_t)1, __ATOMIC_RELAXED);
                }
            }
        }
    }
    free(x0); free(cnt); free(items); free(fill);
    return tested;
}

void uvo_raster_labels(const double* uv, const int64_t* F, const int32_t* lab, int64_t m, int64_t res, int32_t* img) {
    for (int64_t t = 0; t < m; ++t) {
        const int64_t a = F[3 * t], b = F[3 * t + 1], c = F[3 * t + 2];
        double x0 = uv[2 * a] * res, y0 = uv[2 * a + 1] * res;
        double x1 = uv[2 * b] * res, y1 = uv[2 * b + 1] * res;
        double x2 = uv[2 * c] * res, y2 = uv[2 * c + 1] * res;
        double area = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
        if (area < 0) { double tx = x1, ty = y1; x1 = x2; y1 = y2; x2 = tx; y2 = ty; }
        double fx0 = floor(fmin(x0, fmin(x1, x2))), fx1 = floor(fmax(x0, fmax(x1, x2)));
        double fy0 = floor(fmin(y0, fmin(y1, y2))), fy1 = floor(fmax(y0, fmax(y1, y2)));
        if (!(fx0 == fx0) || !(fx1 == fx1) || !(fy0 == fy0) || !(fy1 == fy1)) continue;
        int64_t minx = fx0 < 0 ? 0 : (int64_t)fx0, miny = fy0 < 0 ? 0 : (int64_t)fy0;
        int64_t maxx = fx1 > (double)(res - 1) ? res - 1 : (int64_t)fx1;
        int64_t maxy = fy1 > (double)(res - 1) ? res - 1 : (int64_t)fy1;
        double ex[3] = {x1 - x0, x2 - x1, x0 - x2}, ey[3] = {y1 - y0, y2 - y1, y0 - y2};
        double ox[3] = {x0, x1, x2}, oy[3] = {y0, y1, y2};
        double L[3];
        for (int k = 0; k < 3; ++k) L[k] = sqrt(ex[k] * ex[k] + ey[k] * ey[k]);
        for (int64_t py = miny; py <= maxy; ++py)
            for (int64_t px = minx; px <= maxx; ++px) {
                double cx = px + 0.5, cy = py + 0.5;
                int inside = 1;
                for (int k = 0; k < 3; ++k) {
                    double e = ex[k] * (cy - oy[k]) - ey[k] * (cx - ox[k]);
                    if (e < -0.7072 * L[k]) { inside = 0; break; }
                }
                if (inside) img[py * res + px] = lab[t];
            }
    }
}

void uvo_raster_counts(const double* uv, const int64_t* F, int64_t m, int64_t res, uint8_t* counts) {
    for (int64_t t = 0; t < m; ++t) {
        const int64_t a = F[3 * t], b = F[3 * t + 1], c = F[3 * t + 2];
        double x0 = uv[2 * a] * res, y0 = uv[2 * a + 1] * res;
        double x1 = uv[2 * b] * res, y1 = uv[2 * b + 1] * res;
        double x2 = uv[2 * c] * res, y2 = uv[2 * c + 1] * res;
        double area = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
        if (area == 0.0) continue;
        if (area < 0) { double tx = x1, ty = y1; x1 = x2; y1 = y2; x2 = tx; y2 = ty; }
        double fx0 = floor(fmin(x0, fmin(x1, x2)) - 0.5), fx1 = ceil(fmax(x0, fmax(x1, x2)) - 0.5);
        double fy0 = floor(fmin(y0, fmin(y1, y2)) - 0.5), fy1 = ceil(fmax(y0, fmax(y1, y2)) - 0.5);
        if (!(fx0 == fx0) || !(fx1 == fx1) || !(fy0 == fy0) || !(fy1 == fy1)) continue;
        int64_t minx = fx0 < 0 ? 0 : (int64_t)fx0, miny = fy0 < 0 ? 0 : (int64_t)fy0;
        int64_t maxx = fx1 > (double)(res - 1) ? res - 1 : (int64_t)fx1;
        int64_t maxy = fy1 > (double)(res - 1) ? res - 1 : (int64_t)fy1;
        double ex[3] = {x1 - x0, x2 - x1, x0 - x2}, ey[3] = {y1 - y0, y2 - y1, y0 - y2};
        double ox[3] = {x0, x1, x2}, oy[3] = {y0, y1, y2};
        for (int64_t py = miny; py <= maxy; ++py) {
            double cy = py + 0.5;
            for (int64_t px = minx; px <= maxx; ++px) {
                double cx = px + 0.5;
                int inside = 1;
                for (int k = 0; k < 3; ++k) {
                    double e = ex[k] * (cy - oy[k]) - ey[k] * (cx - ox[k]);
                    if (e < 0) { inside = 0; break; }
                    if (e == 0) {
                        int top_left = (ey[k] == 0 && ex[k] < 0) || ey[k] > 0;
                        if (!top_left) { inside = 0; break; }
                    }
                }
                if (inside && counts[py * res + px] < 255) counts[py * res + px]++;
            }
        }
    }
}

/* Conservative raster of one chart whose corners are already scaled and
 * padded (engine/pack.py:52-79): a cell is set when the cell corner that
 * maximises each edge function of a counter-clockwise triangle is on the
 * inner side of all three edges. */
void uvo_pack_raster(const double* V, const int64_t* T, int64_t t, int64_t h, int64_t w, uint8_t* mask) {
    for (int64_t f = 0; f < t; ++f) {
        double x0 = V[2 * T[3 * f]], y0 = V[2 * T[3 * f] + 1];
        double x1 = V[2 * T[3 * f + 1]], y1 = V[2 * T[3 * f + 1] + 1];
        double x2 = V[2 * T[3 * f + 2]], y2 = V[2 * T[3 * f + 2] + 1];
        double area = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
        if (area < 0) { double tx = x1, ty = y1; x1 = x2; y1 = y2; x2 = tx; y2 = ty; }
        int64_t minx = (int64_t)floor(fmin(x0, fmin(x1, x2))), maxx = (int64_t)floor(fmax(x0, fmax(x1, x2)));
        int64_t miny = (int64_t)floor(fmin(y0, fmin(y1, y2))), maxy = (int64_t)floor(fmax(y0, fmax(y1, y2)));
        if (minx < 0) minx = 0;
        if (miny < 0) miny = 0;
        if (maxx > w - 1) maxx = w - 1;
        if (maxy > h - 1) maxy = h - 1;
        double ex[3] = {x1 - x0, x2 - x1, x0 - x2}, ey[3] = {y1 - y0, y2 - y1, y0 - y2};
        double ox[3] = {x0, x1, x2}, oy[3] = {y0, y1, y2};
        for (int64_t py = miny; py <= maxy; ++py)
            for (int64_t px = minx; px <= maxx; ++px) {
                int inside = 1;
                for (int k = 0; k < 3 && inside; ++k) {
                    double cx = (double)px + (ey[k] > 0 ? 0.0 : 1.0);
                    double cy = (double)py + (ex[k] > 0 ? 1.0 : 0.0);
                    if (ex[k] * (cy - oy[k]) - ey[k] * (cx - ox[k]) < 0) inside = 0;
                }
                if (inside) mask[py * w + px] = 1;
            }
    }
}

/* First fit of one variant: the smallest y, then the smallest x, where
 * every run of every row lands on free cells (engine/pack.py:123-156). The
 * rows are tested in `rows` order (longest run first); a failing run moves
 * x past the occupied run that stopped it. */
static int pk_find(const int32_t* R, const int32_t* O, const int64_t* rowmax, int64_t G, int64_t h, int64_t w,
                   const int64_t* rp, const int64_t* ra, const int64_t* rb, const int64_t* need,
                   const int64_t* rows, int64_t* ox, int64_t* oy) {
    for (int64_t y = 0; y + h <= G; ++y) {
        int ok = 1;
        for (int64_t jj = 0; jj < h && ok; ++jj)
            if (need[rows[jj]] > rowmax[y + rows[jj]]) ok = 0;
        if (!ok) continue;
        int64_t x = 0;
        while (x <= G - w) {
            int fits = 1;
            int64_t skip = 1;
            for (int64_t jj = 0; jj < h && fits; ++jj) {
                const int64_t j = rows[jj];
                for (int64_t q = rp[j]; q < rp[j + 1]; ++q) {
                    const int64_t L = rb[q] - ra[q] + 1;
                    const int64_t r = R[(y + j) * G + x + ra[q]];
                    if (r < L) {
                        const int64_t c = x + ra[q] + r;
                        skip = r + (c < G ? O[(y + j) * G + c] : 1);
                        fits = 0;
                        break;
                    }
                }
            }
            if (fits) { *ox = x; *oy = y; return 1; }
            x += skip;
        }
    }
    return 0;
}

/* Mark one placed variant and rebuild the free-run (R), occupied-run (O)
 * and longest-free-run tables of its rows (engine/pack.py:232-256). */
static void pk_place(uint8_t* occ, int32_t* R, int32_t* O, int64_t* rowmax, int64_t G, int64_t x, int64_t y,
                     int64_t h, const int64_t* rp, const int64_t* ra, const int64_t* rb) {
    for (int64_t j = 0; j < h; ++j) {
        uint8_t* row = occ + (y + j) * G;
        for (int64_t q = rp[j]; q < rp[j + 1]; ++q)
            for (int64_t i = ra[q]; i <= rb[q]; ++i) row[x + i] = 1;
        int32_t run = 0, orun = 0;
        int64_t mx = 0;
        for (int64_t i = G - 1; i >= 0; --i) {
            if (row[i]) { run = 0; ++orun; } else { ++run; orun = 0; }
            R[(y + j) * G + i] = run;
            O[(y + j) * G + i] = orun;
            if (run > mx) mx = run;
        }
        rowmax[y + j] = mx;
    }
}

/* Greedy placement of nc charts in `order` on a G x G page (engine/pack.py
 * :312-359). Variant v = c * nk + k has vh[v] x vw[v] cells (vh 0: none) and
 * rows var_row[v] .. var_row[v + 1] - 1 of the row arrays: run offsets rp
 * (absolute, one more entry than rows, per variant), longest run need and
 * test order rows (variant-local). Per chart the variant of smallest
 * (y + h) G + (x + w) wins, the first on ties. Writes placement (k, x, y per
 * chart) and occ; returns 0, or -1 - p when the chart at position p fits
 * nowhere. */
int64_t uvo_pack_try(int64_t nc, int64_t nk, int64_t G, const int64_t* order, const int64_t* vh, const int64_t* vw,
                     const int64_t* var_row, const int64_t* var_rp, const int64_t* ra, const int64_t* rb,
                     const int64_t* need, const int64_t* rows, int64_t* placement, uint8_t* occ) {
    int32_t* R = (int32_t*)malloc(sizeof(int32_t) * G * G);
    int32_t* O = (int32_t*)calloc((size_t)(G * G), sizeof(int32_t));
    int64_t* rowmax = (int64_t*)malloc(sizeof(int64_t) * G);
    int64_t rc = 0;
    memset(occ, 0, (size_t)(G * G));
    for (int64_t y = 0; y < G; ++y) {
        rowmax[y] = G;
        for (int64_t x = 0; x < G; ++x) R[y * G + x] = (int32_t)(G - x);
    }
    for (int64_t p = 0; p < nc; ++p) {
        const int64_t c = order[p];
        int64_t best = -1, bk = -1, bx = 0, by = 0;
        for (int64_t k = 0; k < nk; ++k) {
            const int64_t v = c * nk + k, h = vh[v], w = vw[v];
            if (h <= 0 || h > G || w > G) continue;
            int64_t x, y;
            const int64_t r0 = var_row[v];
            if (!pk_find(R, O, rowmax, G, h, w, var_rp + r0 + v, ra, rb, need + r0, rows + r0, &x, &y)) continue;
            const int64_t score = (y + h) * G + (x + w);
            if (bk < 0 || score < best) { best = score; bk = k; bx = x; by = y; }
        }
        if (bk < 0) { rc = -1 - p; break; }
        const int64_t v = c * nk + bk;
        pk_place(occ, R, O, rowmax, G, bx, by, vh[v], var_rp + var_row[v] + v, ra, rb);
        placement[3 * c] = bk;
        placement[3 * c + 1] = bx;
        placement[3 * c + 2] = by;
    }
    free(R); free(O); free(rowmax);
    return rc;
}
