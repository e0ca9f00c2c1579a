/*
 * Nested uniform grid over axis-aligned boxes: a candidate prefilter for rays on the CPU — TEST
 * INFRASTRUCTURE ONLY (the oracle's candidate gathering, the host-core baseline, and the OptiX
 * traversal stand-in of oracle/ref_shim/optix.h).
 *
 * The top level covers the scene box with res^3 cells (res ~ cbrt(n / 8), at most 96 per axis).
 * A cell that receives more than ORC_GRID_LEAF boxes, whose boxes are on average small against its
 * children (mean largest extent below four child cells), and that lies less than ORC_GRID_DEPTH
 * levels down is split into 8^3 child cells; otherwise it keeps its list of boxes.  Unbounded scenes (most
 * Gaussians in a small core, a sparse far field) thereby get fine cells only where they are dense.
 *
 * A query walks the cells that the segment o + t d, t in [t0, t1], passes through (3-D DDA in
 * double, recursing into split cells) and appends every box registered there once.  Boxes are
 * registered in every cell their box, grown by 1e-4 of its coordinates' magnitude plus 1e-3 of the
 * cell size, overlaps, so the result is a superset of the boxes the segment meets: callers apply
 * their own exact box and interval tests to it, in their own order, and get the results of a scan
 * over all boxes.  Boxes with a non-finite coordinate are returned by every query.
 */
#ifndef ORC_GRID_H
#define ORC_GRID_H

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_GRID_LEAF 48
#define ORC_GRID_DEPTH 4
#define ORC_GRID_SUB 8

typedef struct {
    double lo[3], cell[3];
    int res;
    long long cell0;           /* first cell of the level in the cell arrays */
} orc_grid_level;

typedef struct {
    orc_grid_level* lv;
    int n_lv, cap_lv;
    long long* first;          /* per cell: first entry in ids, or -(child level + 1) when split */
    int* count;                /* per cell: entries (0 when split) */
    long long n_cells, cap_cells;
    int* ids;
    long long n_ids, cap_ids;
    int* always;               /* boxes with a non-finite coordinate */
    int n_always;
    const double* box;         /* (n, 6) lo.xyz hi.xyz */
    int n;
} orc_grid;

static void* orc_grid_grow(void* p, long long* cap, long long need, size_t elem) {
    if (need <= *cap) return p;
    long long c = *cap ? *cap : 1024;
    while (c < need) c *= 2;
    p = realloc(p, (size_t)c * elem);
    *cap = c;
    return p;
}

static void orc_grid_pad(const double* b, int a, double cell, double* lo, double* hi) {
    double pad = 1e-4 * (fabs(b[a]) + fabs(b[3 + a])) + 1e-6 + 1e-3 * cell;
    *lo = b[a] - pad;
    *hi = b[3 + a] + pad;
}

static int orc_grid_clampi(long long v, int res) { return v < 0 ? 0 : (v >= res ? res - 1 : (int)v); }

/* cell index range [c0, c1] of box b along axis a at a level (-1 when it misses the level) */
static int orc_grid_range(const orc_grid_level* L, const double* b, int a, int* c0, int* c1) {
    double lo, hi;
    orc_grid_pad(b, a, L->cell[a], &lo, &hi);
    double f0 = (lo - L->lo[a]) / L->cell[a], f1 = (hi - L->lo[a]) / L->cell[a];
    if (f1 < 0.0 || f0 >= (double)L->res) return -1;
    *c0 = orc_grid_clampi((long long)floor(f0), L->res);
    *c1 = orc_grid_clampi((long long)floor(f1), L->res);
    return 0;
}

static void orc_grid_level_build(orc_grid* G, const int* items, int m, const double* lo, const double* hi, int res,
                                 int depth) {
    int li = G->n_lv;
    {
        long long cap = G->cap_lv;
        G->lv = (orc_grid_level*)orc_grid_grow(G->lv, &cap, li + 1, sizeof(orc_grid_level));
        G->cap_lv = (int)cap;
    }
    G->n_lv = li + 1;
    orc_grid_level L;
    for (int a = 0; a < 3; ++a) {
        L.lo[a] = lo[a];
        double ext = hi[a] - lo[a];
        L.cell[a] = (ext > 0.0 ? ext : 1e-9) / res;
    }
    L.res = res;
    L.cell0 = G->n_cells;
    const long long nc = (long long)res * res * res;
    G->first = (long long*)orc_grid_grow(G->first, &G->cap_cells, G->n_cells + nc, sizeof(long long));
    G->count = (int*)realloc(G->count, (size_t)G->cap_cells * sizeof(int));   /* same capacity as first */
    G->n_cells += nc;
    G->lv[li] = L;
    /* count boxes per cell and their mean largest extent */
    int* cnt = (int*)calloc((size_t)nc, sizeof(int));
    double* ext = (double*)calloc((size_t)nc, sizeof(double));
    for (int k = 0; k < m; ++k) {
        const double* b = G->box + 6 * (long long)items[k];
        int r0[3], r1[3], miss = 0;
        for (int a = 0; a < 3 && !miss; ++a) miss = orc_grid_range(&L, b, a, &r0[a], &r1[a]);
        if (miss) continue;
        double e = fmax(b[3] - b[0], fmax(b[4] - b[1], b[5] - b[2]));
        for (int z = r0[2]; z <= r1[2]; ++z)
            for (int y = r0[1]; y <= r1[1]; ++y)
                for (int x = r0[0]; x <= r1[0]; ++x) {
                    long long c = ((long long)z * res + y) * res + x;
                    ++cnt[c];
                    ext[c] += e;
                }
    }
    /* per-cell lists (CSR) */
    long long* off = (long long*)malloc(sizeof(long long) * (size_t)(nc + 1));
    off[0] = 0;
    for (long long c = 0; c < nc; ++c) off[c + 1] = off[c] + cnt[c];
    int* list = (int*)malloc(sizeof(int) * (size_t)(off[nc] > 0 ? off[nc] : 1));
    long long* fill = (long long*)malloc(sizeof(long long) * (size_t)(nc > 0 ? nc : 1));
    memcpy(fill, off, sizeof(long long) * (size_t)nc);
    for (int k = 0; k < m; ++k) {
        const double* b = G->box + 6 * (long long)items[k];
        int r0[3], r1[3], miss = 0;
        for (int a = 0; a < 3 && !miss; ++a) miss = orc_grid_range(&L, b, a, &r0[a], &r1[a]);
        if (miss) continue;
        for (int z = r0[2]; z <= r1[2]; ++z)
            for (int y = r0[1]; y <= r1[1]; ++y)
                for (int x = r0[0]; x <= r1[0]; ++x) list[fill[((long long)z * res + y) * res + x]++] = items[k];
    }
    free(fill);
    const double child_cell = fmax(L.cell[0], fmax(L.cell[1], L.cell[2])) / ORC_GRID_SUB;
    for (long long c = 0; c < nc; ++c) {
        const long long gc = L.cell0 + c;
        const int n_in = cnt[c];
        if (n_in > ORC_GRID_LEAF && depth + 1 < ORC_GRID_DEPTH && ext[c] / n_in < 4.0 * child_cell) {
            int x = (int)(c % res), y = (int)((c / res) % res), z = (int)(c / ((long long)res * res));
            double clo[3] = {L.lo[0] + x * L.cell[0], L.lo[1] + y * L.cell[1], L.lo[2] + z * L.cell[2]};
            double chi[3] = {clo[0] + L.cell[0], clo[1] + L.cell[1], clo[2] + L.cell[2]};
            G->first[gc] = -(long long)(G->n_lv + 1);   /* the child is the next level built */
            G->count[gc] = 0;
            orc_grid_level_build(G, list + off[c], n_in, clo, chi, ORC_GRID_SUB, depth + 1);
        } else {
            G->ids = (int*)orc_grid_grow(G->ids, &G->cap_ids, G->n_ids + n_in, sizeof(int));
            memcpy(G->ids + G->n_ids, list + off[c], sizeof(int) * (size_t)n_in);
            G->first[gc] = G->n_ids;
            G->count[gc] = n_in;
            G->n_ids += n_in;
        }
    }
    free(list);
    free(off);
    free(cnt);
    free(ext);
}

/* Builds the grid over n boxes (n, 6) inside [lo, hi]; `box` must outlive the grid. */
static void orc_grid_build(orc_grid* G, const double* box, int n, const double* lo, const double* hi) {
    memset(G, 0, sizeof(*G));
    G->box = box;
    G->n = n;
    int* items = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    G->always = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int m = 0;
    for (int i = 0; i < n; ++i) {
        const double* b = box + 6 * (long long)i;
        int fin = 1;
        for (int a = 0; a < 6; ++a) fin &= isfinite(b[a]) ? 1 : 0;
        if (fin) items[m++] = i;
        else G->always[G->n_always++] = i;
    }
    double glo[3], ghi[3];
    for (int a = 0; a < 3; ++a) {
        double pad = 1e-4 * (fabs(lo[a]) + fabs(hi[a])) + 1e-6;
        glo[a] = lo[a] - pad;
        ghi[a] = hi[a] + pad;
        if (!(ghi[a] > glo[a])) { glo[a] = -1.0; ghi[a] = 1.0; }
    }
    int res = (int)cbrt((double)m / 8.0);
    res = res < 1 ? 1 : (res > 96 ? 96 : res);
    orc_grid_level_build(G, items, m, glo, ghi, res, 0);
    free(items);
}

static void orc_grid_free(orc_grid* G) {
    free(G->lv);
    free(G->first);
    free(G->count);
    free(G->ids);
    free(G->always);
    memset(G, 0, sizeof(*G));
}

static void orc_grid_take(const orc_grid* G, long long gc, unsigned char* mark, int* out, int* m) {
    const int* p = G->ids + G->first[gc];
    for (int k = 0; k < G->count[gc]; ++k) {
        int id = p[k];
        if (!mark[id]) { mark[id] = 1; out[(*m)++] = id; }
    }
}

static void orc_grid_walk(const orc_grid* G, int li, const double* o, const double* d, double t0, double t1,
                          unsigned char* mark, int* out, int* m) {
    const orc_grid_level* L = &G->lv[li];
    const int res = L->res;
    for (int a = 0; a < 3; ++a) {
        double lo = L->lo[a], hi = L->lo[a] + res * L->cell[a];
        if (d[a] == 0.0) {
            if (o[a] < lo || o[a] > hi) return;
            continue;
        }
        double ta = (lo - o[a]) / d[a], tb = (hi - o[a]) / d[a];
        if (ta > tb) { double s = ta; ta = tb; tb = s; }
        if (ta > t0) t0 = ta;
        if (tb < t1) t1 = tb;
    }
    if (!(t0 <= t1)) return;
    int c[3], step[3];
    double tmax[3], tdel[3];
    for (int a = 0; a < 3; ++a) {
        double p = o[a] + d[a] * t0;
        c[a] = orc_grid_clampi((long long)floor((p - L->lo[a]) / L->cell[a]), res);
        if (d[a] > 0.0) {
            step[a] = 1;
            tmax[a] = (L->lo[a] + (c[a] + 1) * L->cell[a] - o[a]) / d[a];
            tdel[a] = L->cell[a] / d[a];
        } else if (d[a] < 0.0) {
            step[a] = -1;
            tmax[a] = (L->lo[a] + c[a] * L->cell[a] - o[a]) / d[a];
            tdel[a] = -L->cell[a] / d[a];
        } else {
            step[a] = 0;
            tmax[a] = INFINITY;
            tdel[a] = INFINITY;
        }
    }
    double t = t0;
    for (int guard = 0; guard < 3 * res + 3; ++guard) {
        const long long gc = L->cell0 + ((long long)c[2] * res + c[1]) * res + c[0];
        int a = (tmax[0] < tmax[1]) ? (tmax[0] < tmax[2] ? 0 : 2) : (tmax[1] < tmax[2] ? 1 : 2);
        double tx = tmax[a] < t1 ? tmax[a] : t1;
        if (G->first[gc] < 0) {
            double eps = 1e-9 * (fabs(t) + fabs(tx)) + 1e-3 * L->cell[0] / (fabs(d[0]) + fabs(d[1]) + fabs(d[2]));
            orc_grid_walk(G, (int)(-G->first[gc] - 1), o, d, t - eps, tx + eps, mark, out, m);
        } else {
            orc_grid_take(G, gc, mark, out, m);
        }
        if (tmax[a] > t1) break;
        c[a] += step[a];
        if (c[a] < 0 || c[a] >= res) break;
        t = tmax[a];
        tmax[a] += tdel[a];
    }
}

/* Appends to out (capacity: the number of boxes) the boxes registered in the cells that the
 * segment o + t d, t in [t0, t1], passes through, each once; `mark` (one byte per box, zero on
 * entry) flags the appended boxes and must be cleared by the caller (orc_grid_unmark).  Returns
 * the count. */
static int orc_grid_query(const orc_grid* G, const double* o, const double* d, double t0, double t1,
                          unsigned char* mark, int* out) {
    int m = 0;
    if (G->n_lv > 0) orc_grid_walk(G, 0, o, d, t0, t1, mark, out, &m);
    for (int k = 0; k < G->n_always; ++k) {
        int id = G->always[k];
        if (!mark[id]) { mark[id] = 1; out[m++] = id; }
    }
    return m;
}

static void orc_grid_unmark(unsigned char* mark, const int* out, int m) {
    for (int k = 0; k < m; ++k) mark[out[k]] = 0;
}

static int orc_grid_cmp_ll(const void* a, const void* b) {
    long long x = *(const long long*)a, y = *(const long long*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* Sorts ids by rank[id] (by id when rank is NULL); key is scratch for m entries. */
static void orc_grid_sort(int* ids, int m, const int* rank, long long* key) {
    for (int k = 0; k < m; ++k) key[k] = ((long long)(rank ? rank[ids[k]] : ids[k]) << 32) | (unsigned)ids[k];
    qsort(key, (size_t)m, sizeof(long long), orc_grid_cmp_ll);
    for (int k = 0; k < m; ++k) ids[k] = (int)(key[k] & 0xffffffffLL);
}

#endif /* ORC_GRID_H */
