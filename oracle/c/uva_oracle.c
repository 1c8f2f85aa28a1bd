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

/* Returns the number of tested candidate pairs (cell boxes intersecting). */
int64_t uvo_overlaps(const double* U, const int64_t* F, const uint8_t* skip, int64_t m, int64_t G, double rel,
                     int strict, uint8_t* flag) {
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
    for (int64_t c = 0; c < G * G; ++c) {
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
