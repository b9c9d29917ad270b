/*
 * ORACLE — test infrastructure only.
 *
 * Literal CPU restatement (C99, single-threaded, IEEE double, no FMA
 * contraction) of the Fortran kernels that goSPL's per-timestep surface
 * process path calls through f2py (`gospl._fortran`, fortran/functions.F90).
 * The reference's own Fortran cannot be compiled in this environment (no
 * Fortran compiler), so each routine below restates the cited Fortran line by
 * line, including its queue disciplines and known quirks, so that the Python
 * orchestration of the reference (and this repository's oracle model) can run
 * against it.  Only tests/, the smoke check and bench.py's CPU-baseline leg
 * use this file; the product never links it.
 *
 * Arrays follow C order: a Fortran (nb,12) array becomes a[k*12 + p].
 * Node ids are 0-based exactly as the Fortran stores them (FVnID = id-1).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAXNB 12

/* ---------------------------------------------------------------------------
 * module meshparams (functions.F90:10-36): mesh state shared by all kernels.
 * ------------------------------------------------------------------------- */
static int g_nb = 0;
static int *FVnNb = NULL;       /* [nb]            */
static int *FVnID = NULL;       /* [nb*12], -1 pad */
static double *FVeLgt = NULL;   /* [nb*12]         */
static double *FVvDist = NULL;  /* [nb*12]         */
static double *FVarea = NULL;   /* [nb]            */
static int curvedmesh = -1;     /* functions.F90:28 */

/* ---------------------------------------------------------------------------
 * Queues (functions.F90:39-308).  Every container keeps the reference's exact
 * discipline because pop order decides watershed labels and graph order.
 * ------------------------------------------------------------------------- */
typedef struct { int id; double Z; } qnode;            /* type node  */
typedef struct { int id, w1, w2; double Z; } wnode;    /* type wnode */

typedef struct { qnode *buf; int n, cap; } pqueue_t;   /* 1-based heap */
typedef struct { qnode *buf; int n, cap; } plainq_t;   /* type queue   */
typedef struct { int *buf; int n, cap; } simpleq_t;    /* type squeue  */

static pqueue_t priorityqueue = {0};
static plainq_t plainqueue = {0};
static simpleq_t simplequeue = {0};

static void *grow(void *p, int *cap, int need, size_t elt)
{
    if (need <= *cap) return p;
    int nc = *cap ? *cap : 16;
    while (nc < need) nc *= 2;
    p = realloc(p, (size_t)nc * elt);
    *cap = nc;
    return p;
}

/* shiftdown (functions.F90:120-141) */
static void pq_shiftdown(pqueue_t *q, int a)
{
    qnode *x = q->buf;
    int parent = a;
    while (parent * 2 <= q->n) {
        int child = parent * 2;
        if (child + 1 <= q->n && x[child + 1].Z < x[child].Z) child = child + 1;
        if (x[parent].Z > x[child].Z) {
            qnode t = x[child]; x[child] = x[parent]; x[parent] = t;
            parent = child;
        } else break;
    }
}
/* PQpop (functions.F90:143-150) */
static qnode pq_pop(pqueue_t *q)
{
    qnode res = q->buf[1];
    q->buf[1] = q->buf[q->n];
    q->n -= 1;
    pq_shiftdown(q, 1);
    return res;
}
/* PQpush (functions.F90:152-184): append then sift up while strictly smaller */
static void pq_push(pqueue_t *q, double Z, int id)
{
    q->n += 1;
    q->buf = (qnode *)grow(q->buf, &q->cap, q->n + 1, sizeof(qnode));
    q->buf[q->n].Z = Z; q->buf[q->n].id = id;
    int ii = q->n;
    while (ii > 1) {
        int parent = ii / 2;
        if (q->buf[ii].Z < q->buf[parent].Z) {
            qnode t = q->buf[ii]; q->buf[ii] = q->buf[parent]; q->buf[parent] = t;
            ii = parent;
        } else break;
    }
}
/* queue%push / queue%pop (functions.F90:288-306, 276-283): pop takes the first
 * element and moves the last one into its place. */
static void plain_push(plainq_t *q, double Z, int id)
{
    q->n += 1;
    q->buf = (qnode *)grow(q->buf, &q->cap, q->n + 1, sizeof(qnode));
    q->buf[q->n].Z = Z; q->buf[q->n].id = id;
}
static qnode plain_pop(plainq_t *q)
{
    qnode res = q->buf[1];
    q->buf[1] = q->buf[q->n];
    q->n -= 1;
    return res;
}
/* squeue%spush / spop (functions.F90:255-273) */
static void simple_push(simpleq_t *q, int id)
{
    q->n += 1;
    q->buf = (int *)grow(q->buf, &q->cap, q->n + 1, sizeof(int));
    q->buf[q->n] = id;
}
static int simple_pop(simpleq_t *q)
{
    int res = q->buf[1];
    q->buf[1] = q->buf[q->n];
    q->n -= 1;
    return res;
}

/* wgraph (functions.F90:186-227).  The reference scans the whole buffer for an
 * existing (w1,w2) pair on every push; an open-addressing index mirrors that
 * scan exactly (same slot positions, same "keep the lower Z" update) in O(1). */
typedef struct {
    wnode *buf; int n, cap;          /* 1-based, like the Fortran buffer */
    int64_t *hkey; int *hpos; int hcap;
} wgraph_t;
static wgraph_t graph = {0};

static uint64_t wkey(int w1, int w2) { return ((uint64_t)(uint32_t)w1 << 32) | (uint32_t)w2; }
static uint64_t hmix(uint64_t x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33; return x;
}
static void wg_rehash(wgraph_t *g, int newcap)
{
    free(g->hkey); free(g->hpos);
    g->hcap = newcap;
    g->hkey = (int64_t *)malloc(sizeof(int64_t) * newcap);
    g->hpos = (int *)malloc(sizeof(int) * newcap);
    for (int i = 0; i < newcap; i++) g->hkey[i] = -1;
    for (int p = 1; p <= g->n; p++) {
        uint64_t k = wkey(g->buf[p].w1, g->buf[p].w2);
        uint64_t h = hmix(k) & (uint64_t)(newcap - 1);
        while (g->hkey[h] != -1) h = (h + 1) & (uint64_t)(newcap - 1);
        g->hkey[h] = (int64_t)k; g->hpos[h] = p;
    }
}
static int wg_find(wgraph_t *g, int w1, int w2, uint64_t *slot)
{
    if (g->hcap == 0) return 0;
    uint64_t k = wkey(w1, w2);
    uint64_t h = hmix(k) & (uint64_t)(g->hcap - 1);
    while (g->hkey[h] != -1) {
        if ((uint64_t)g->hkey[h] == k) { *slot = h; return g->hpos[h]; }
        h = (h + 1) & (uint64_t)(g->hcap - 1);
    }
    *slot = h;
    return 0;
}
static void wg_reset(wgraph_t *g)
{
    g->n = 0;
    if (g->hcap) for (int i = 0; i < g->hcap; i++) g->hkey[i] = -1;
}
static void wpush(wgraph_t *g, int w1, int w2, double Z, int id)
{
    uint64_t slot;
    int pos = wg_find(g, w1, w2, &slot);
    if (pos > 0) {
        if (Z < g->buf[pos].Z) { g->buf[pos].Z = Z; g->buf[pos].id = id; }
        return;
    }
    g->n += 1;
    g->buf = (wnode *)grow(g->buf, &g->cap, g->n + 1, sizeof(wnode));
    g->buf[g->n].Z = Z; g->buf[g->n].id = id; g->buf[g->n].w1 = w1; g->buf[g->n].w2 = w2;
    if (g->hcap == 0 || 2 * g->n > g->hcap) {
        int nc = g->hcap ? g->hcap * 2 : 1024;
        while (2 * g->n > nc) nc *= 2;
        wg_rehash(g, nc);
    } else {
        g->hkey[slot] = (int64_t)wkey(w1, w2); g->hpos[slot] = g->n;
    }
}
/* wpop (functions.F90:187-193): first element out, last element moves in. */
static wnode wpop(wgraph_t *g)
{
    wnode res = g->buf[1];
    uint64_t s;
    int p = wg_find(g, res.w1, res.w2, &s);
    (void)p;
    /* delete res from the index (backward-shift deletion) */
    {
        uint64_t mask = (uint64_t)(g->hcap - 1), i = s, j = s;
        g->hkey[i] = -1;
        for (;;) {
            j = (j + 1) & mask;
            if (g->hkey[j] == -1) break;
            uint64_t k = hmix((uint64_t)g->hkey[j]) & mask;
            if ((j > i && (k <= i || k > j)) || (j < i && (k <= i && k > j))) {
                g->hkey[i] = g->hkey[j]; g->hpos[i] = g->hpos[j]; g->hkey[j] = -1; i = j;
            }
        }
    }
    if (g->n > 1) {
        g->buf[1] = g->buf[g->n];
        uint64_t s2;
        if (wg_find(g, g->buf[1].w1, g->buf[1].w2, &s2) > 0) g->hpos[s2] = 1;
    }
    g->n -= 1;
    return res;
}

/* ---------------------------------------------------------------------------
 * Geometry helpers (functions.F90:316-662).
 * ------------------------------------------------------------------------- */
/* gfortran expands NORM2 with the scaled sum of squares
 * (scale, ssq) recurrence; restated here so lengths round the same way. */
static double norm2_3(const double v[3])
{
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < 3; i++) {
        if (v[i] != 0.0) {
            double ax = fabs(v[i]);
            if (scale < ax) {
                double val = scale / ax;
                ssq = 1.0 + ssq * val * val;
                scale = ax;
            } else {
                double val = ax / scale;
                ssq += val * val;
            }
        }
    }
    return scale * sqrt(ssq);
}
static const double PI_F = 3.1415926535897932;
/* spherical2lonlat (functions.F90:316-335) */
static void spherical2lonlat(const double xyz[3], double *lon, double *lat)
{
    double r = sqrt(xyz[0] * xyz[0] + xyz[1] * xyz[1] + xyz[2] * xyz[2]);
    double la = asin(xyz[2] / r) * (180.0 / PI_F);
    double lo = atan2(xyz[1], xyz[0]) * (180.0 / PI_F);
    *lat = la * PI_F / 180.0;
    *lon = lo * PI_F / 180.0;
}
/* great_circle_distance (functions.F90:337-366) */
static double great_circle_distance(double lon1, double lat1, double lon2, double lat2, double radius)
{
    double c1 = cos(lat1), s1 = sin(lat1), c2 = cos(lat2), s2 = sin(lat2);
    double dlon = lon1 - lon2, clon = cos(dlon), slon = sin(dlon);
    double a = c2 * slon, b = c1 * s2 - s1 * c2 * clon;
    return radius * atan2(sqrt(a * a + b * b), (s1 * s2 + c1 * c2 * clon));
}
/* distance (functions.F90:368-393) */
static double fdistance(const double p1[3], const double p2[3])
{
    if (p2[2] == 0.0 && p1[2] == 0.0) {
        double v[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
        return norm2_3(v);
    }
    double radius = norm2_3(p1), lon1, lat1, lon2, lat2;
    spherical2lonlat(p1, &lon1, &lat1);
    spherical2lonlat(p2, &lon2, &lat2);
    return great_circle_distance(lon1, lat1, lon2, lat2, radius);
}
/* slerpmidpt (functions.F90:425-452) */
static void slerpmidpt(const double p1[3], const double p2[3], double mpt[3])
{
    double n1 = norm2_3(p1), n2 = norm2_3(p2), v1[3], v2[3], pt[3];
    for (int i = 0; i < 3; i++) { v1[i] = p1[i] / n1; v2[i] = p2[i] / n2; }
    double d = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
    double a = acos(d);
    for (int i = 0; i < 3; i++)
        pt[i] = sin(0.5 * a) * v1[i] / sin(a) + sin(0.5 * a) * v2[i] / sin(a);
    double npt = norm2_3(pt);
    for (int i = 0; i < 3; i++) mpt[i] = n1 * pt[i] / npt;
}
/* striarea (functions.F90:538-577) */
static double striarea(const double v1[3], const double v2[3], const double v3[3])
{
    double r = sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
    double lon1, lat1, lon2, lat2, lon3, lat3;
    spherical2lonlat(v1, &lon1, &lat1);
    spherical2lonlat(v2, &lon2, &lat2);
    spherical2lonlat(v3, &lon3, &lat3);
    double a = acos(sin(lat2) * sin(lat3) + cos(lat2) * cos(lat3) * cos(lon3 - lon2));
    double b = acos(sin(lat1) * sin(lat3) + cos(lat1) * cos(lat3) * cos(lon3 - lon1));
    double c = acos(sin(lat1) * sin(lat2) + cos(lat1) * cos(lat2) * cos(lon2 - lon1));
    double alpha = acos((cos(a) - cos(b) * cos(c)) / (sin(b) * sin(c)));
    double beta = acos((cos(b) - cos(a) * cos(c)) / (sin(a) * sin(c)));
    double gamma = acos((cos(c) - cos(a) * cos(b)) / (sin(a) * sin(b)));
    double E = alpha + beta + gamma - PI_F;
    return E * (r * r);
}
/* gtriarea (functions.F90:579-616): planar Heron on x,y only */
static double gtriarea(const double p1[3], const double p2[3], const double p3[3])
{
    double x1 = p1[0], x2 = p2[0], x3 = p3[0], y1 = p1[1], y2 = p2[1], y3 = p3[1];
    if (x1 == x2 && y1 == y2) return 0.0;
    if (x1 == x3 && y1 == y3) return 0.0;
    if (x2 == x3 && y2 == y3) return 0.0;
    double l1 = sqrt((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2));
    double l2 = sqrt((x2 - x3) * (x2 - x3) + (y2 - y3) * (y2 - y3));
    double l3 = sqrt((x3 - x1) * (x3 - x1) + (y3 - y1) * (y3 - y1));
    double p = (l1 + l2 + l3) / 2;
    return sqrt(p * (p - l1) * (p - l2) * (p - l3));
}

/* setcurvedmesh (functions.F90:1000-1017) */
void orc_setcurvedmesh(int flag) { curvedmesh = flag; }

/* definetin (functions.F90:2715-2940).  Outputs the module mesh state and the
 * two area arrays the reference keeps: `narea` (returned to Python before the
 * NaN fix) and the module FVarea (NaN -> 0).  The face vectors and midFace are
 * advection-only and are not built. */
int orc_definetin(int nb, int n, int m, const double *coords, const int *cells_nodes,
                  const int *cells_edges, const int *edges_nodes, const double *circumcenter,
                  int *ngbID, double *narea)
{
    free(FVnNb); free(FVnID); free(FVeLgt); free(FVvDist); free(FVarea);
    g_nb = nb;
    FVnNb = (int *)calloc(nb, sizeof(int));
    FVnID = (int *)malloc(sizeof(int) * nb * MAXNB);
    FVeLgt = (double *)calloc((size_t)nb * MAXNB, sizeof(double));
    FVvDist = (double *)calloc((size_t)nb * MAXNB, sizeof(double));
    FVarea = (double *)calloc(nb, sizeof(double));
    int *edge = (int *)malloc(sizeof(int) * nb * MAXNB);
    int *cell_ids = (int *)malloc(sizeof(int) * nb * MAXNB);
    for (int i = 0; i < nb * MAXNB; i++) { edge[i] = -1; cell_ids[i] = -1; ngbID[i] = -1; }

    double radius = 0.0;
    if (curvedmesh == 1) radius = norm2_3(&coords[0]);
    else if (curvedmesh == -1) { if (coords[2] != 0.0) radius = norm2_3(&coords[0]); }

    /* cells surrounding each vertex (cell order) */
    for (int i = 0; i < n; i++) {
        for (int p = 0; p < 3; p++) {
            int v = cells_nodes[i * 3 + p];
            int inside = 0, k;
            for (k = 0; k < MAXNB; k++) {
                if (cell_ids[v * MAXNB + k] == i) break;
                if (cell_ids[v * MAXNB + k] == -1) { inside = 1; break; }
            }
            if (inside) cell_ids[v * MAXNB + k] = i;
        }
    }
    /* edges connected to each vertex (edge order) */
    for (int i = 0; i < m; i++) {
        int ns[2] = {edges_nodes[i * 2], edges_nodes[i * 2 + 1]};
        for (int t = 0; t < 2; t++) {
            int v = ns[t], inside = 0, k;
            for (k = 0; k < MAXNB; k++) {
                if (edge[v * MAXNB + k] == i) break;
                if (edge[v * MAXNB + k] == -1) { inside = 1; break; }
            }
            if (inside) { edge[v * MAXNB + k] = i; FVnNb[v] += 1; }
        }
    }
    for (int k = 0; k < nb; k++) {
        const double *c0 = &coords[k * 3];
        int l = 0, nbngbs = FVnNb[k];
        for (int eid = 0; eid < nbngbs; eid++) {
            int e = edge[k * MAXNB + eid];
            int n1 = edges_nodes[e * 2], n2 = edges_nodes[e * 2 + 1];
            int other = (n1 == k) ? n2 : n1;
            ngbID[k * MAXNB + l] = other;
            FVeLgt[k * MAXNB + l] = fdistance(c0, &coords[other * 3]);
            l++;
        }
        for (int cid = 0; cid < MAXNB; cid++) {
            int c = cell_ids[k * MAXNB + cid];
            if (c == -1) break;
            for (int e = 0; e < 3; e++) {
                int eg = cells_edges[c * 3 + e];
                int e1 = edges_nodes[eg * 2], e2 = edges_nodes[eg * 2 + 1];
                if (k == e1 || k == e2) {
                    double mid[3];
                    if (radius > 0) slerpmidpt(&coords[e1 * 3], &coords[e2 * 3], mid);
                    else for (int d = 0; d < 3; d++) mid[d] = 0.5 * (coords[e1 * 3 + d] + coords[e2 * 3 + d]);
                    int id = -1, want = (e1 == k) ? e2 : e1;
                    for (int i = 0; i < nbngbs; i++)
                        if (ngbID[k * MAXNB + i] == want) { id = i; break; }
                    double cc[3] = {circumcenter[c * 3], circumcenter[c * 3 + 1], circumcenter[c * 3 + 2]};
                    double dist = fdistance(mid, cc);
                    if (id >= 0) FVvDist[k * MAXNB + id] += dist;
                    double tri = (radius == 0.0) ? gtriarea(c0, mid, cc) : striarea(c0, mid, cc);
                    FVarea[k] += tri;
                }
            }
        }
    }
    for (int i = 0; i < nb * MAXNB; i++) FVnID[i] = ngbID[i];
    for (int k = 0; k < nb; k++) narea[k] = FVarea[k];
    for (int k = 0; k < nb; k++) if (isnan(FVarea[k])) FVarea[k] = 0.0;
    free(edge); free(cell_ids);
    return 0;
}

/* updatearea (functions.F90:2699-2713) */
void orc_updatearea(int nb, const double *narea)
{
    for (int k = 0; k < nb && k < g_nb; k++) FVarea[k] = narea[k];
}

/* Direct mesh state setter: lets tests load a saved mesh without rebuilding. */
int orc_setmesh(int nb, const int *nnb, const int *nid, const double *elgt,
                const double *vdist, const double *area)
{
    free(FVnNb); free(FVnID); free(FVeLgt); free(FVvDist); free(FVarea);
    g_nb = nb;
    FVnNb = (int *)malloc(sizeof(int) * nb);
    FVnID = (int *)malloc(sizeof(int) * nb * MAXNB);
    FVeLgt = (double *)malloc(sizeof(double) * nb * MAXNB);
    FVvDist = (double *)malloc(sizeof(double) * nb * MAXNB);
    FVarea = (double *)malloc(sizeof(double) * nb);
    memcpy(FVnNb, nnb, sizeof(int) * nb);
    memcpy(FVnID, nid, sizeof(int) * nb * MAXNB);
    memcpy(FVeLgt, elgt, sizeof(double) * nb * MAXNB);
    memcpy(FVvDist, vdist, sizeof(double) * nb * MAXNB);
    memcpy(FVarea, area, sizeof(double) * nb);
    return 0;
}
int orc_getmesh(int nb, int *nnb, int *nid, double *elgt, double *vdist, double *area)
{
    if (nb != g_nb) return -1;
    memcpy(nnb, FVnNb, sizeof(int) * nb);
    memcpy(nid, FVnID, sizeof(int) * nb * MAXNB);
    memcpy(elgt, FVeLgt, sizeof(double) * nb * MAXNB);
    memcpy(vdist, FVvDist, sizeof(double) * nb * MAXNB);
    memcpy(area, FVarea, sizeof(double) * nb);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Hillslope helpers (functions.F90:876-938)
 * ------------------------------------------------------------------------- */
int orc_setmaxnb(int nb)
{
    int maxnb = 0;
    for (int k = 0; k < nb; k++)
        if (FVarea[k] > 0 && FVnNb[k] > maxnb) maxnb = FVnNb[k];
    return maxnb;
}
/* sethillslopecoeff: dcoeff[k*13 + 0] diagonal, [k*13 + p+1] off-diagonals */
void orc_sethillslopecoeff(int nb, const double *Kd, double *dcoeff)
{
    memset(dcoeff, 0, sizeof(double) * nb * 13);
    for (int k = 0; k < nb; k++) {
        double s1 = 0.0;
        if (FVarea[k] > 0) {
            double ck = Kd[k];
            for (int p = 0; p < FVnNb[k]; p++) {
                if (FVvDist[k * MAXNB + p] > 0.0) {
                    int nn = FVnID[k * MAXNB + p];
                    double cn = Kd[nn];
                    double c = 0.5 * (ck + cn) / FVarea[k];
                    double v = c * FVvDist[k * MAXNB + p] / FVeLgt[k * MAXNB + p];
                    s1 = s1 + v;
                    dcoeff[k * 13 + p + 1] = -v;
                }
            }
            dcoeff[k * 13] = 1.0 + s1;
        }
    }
}

/* ---------------------------------------------------------------------------
 * quicksort / split (functions.F90:683-762).  `array` and `indices` are the
 * full 12-slot buffers; first/last are 1-based like the Fortran.  The left
 * scan is bounded by the buffer size (12), not by `right`, as in the source.
 * ------------------------------------------------------------------------- */
static void split(double *array, int low, int high, int *mid, int *indices)
{
    int left = low, right = high;
    double pivot = array[low - 1];
    int ipivot = indices[low - 1];
    for (;;) {
        if (left >= right) break;
        for (;;) {
            if (left >= right || array[right - 1] < pivot) break;
            right = right - 1;
        }
        for (;;) {
            if (left > 12) break;
            if (array[left - 1] > pivot) break;
            left = left + 1;
        }
        if (left < right) {
            double sw = array[left - 1]; array[left - 1] = array[right - 1]; array[right - 1] = sw;
            int is = indices[left - 1]; indices[left - 1] = indices[right - 1]; indices[right - 1] = is;
        }
    }
    array[low - 1] = array[right - 1];
    array[right - 1] = pivot;
    *mid = right;
    indices[low - 1] = indices[right - 1];
    indices[right - 1] = ipivot;
}
static void quicksort(double *array, int first, int last, int *indices)
{
    if (first < last) {
        int mid;
        split(array, first, last, &mid, indices);
        quicksort(array, first, mid - 1, indices);
        quicksort(array, mid + 1, last, indices);
    }
}
/* exposed for tests: sorts a 12-slot buffer in place over [1, kk] */
void orc_quicksort12(double *array, int kk, int *indices) { quicksort(array, 1, kk, indices); }

/* ---------------------------------------------------------------------------
 * mfdreceivers (functions.F90:1544-1671).  Outputs C-order [nb][nRcv].
 * `powfn` selects the real-exponent power: NULL = libm pow (what the
 * reference's gfortran build calls).
 * ------------------------------------------------------------------------- */
typedef double (*powfn_t)(double, double);
int orc_mfdreceivers(int nb, int nRcv, double exp_, const double *elev, double sl,
                     const int *gid, int *rcv, double *dist, double *wgt, powfn_t powfn)
{
    if (nRcv < 1 || nRcv > 12) return -1;
    if (!powfn) powfn = pow;
    for (int i = 0; i < nb * nRcv; i++) { rcv[i] = -1; dist[i] = 0.0; wgt[i] = 0.0; }
    for (int k = 0; k < nb; k++) {
        int *r = &rcv[k * nRcv];
        double *d = &dist[k * nRcv], *w = &wgt[k * nRcv];
        if (elev[k] <= sl) {
            for (int p = 0; p < nRcv; p++) r[p] = k;
            continue;
        }
        double e = 0.0, val;
        for (int p = 0; p < FVnNb[k]; p++) {
            int n = FVnID[k * MAXNB + p] + 1;
            if (n > 0 && FVeLgt[k * MAXNB + p] > 0.0) {
                val = (elev[k] - elev[n - 1]) / FVeLgt[k * MAXNB + p];
                e = (val > e) ? val : e;   /* max(val, e) */
            }
        }
        double fexp = (e > 0) ? 5.0 * ((e < 1.0) ? e : 1.0) + exp_ : 1.0;
        double slp[12], dst[12], slope[12];
        int id[12];
        for (int p = 0; p < 12; p++) { slp[p] = 0.0; id[p] = 0; }
        int kk = 0;
        for (int p = 0; p < FVnNb[k]; p++) {
            int n = FVnID[k * MAXNB + p] + 1;
            if (n > 0 && FVeLgt[k * MAXNB + p] > 0.0) {
                val = powfn(elev[k] - elev[n - 1], fexp) / FVeLgt[k * MAXNB + p];
                if (val > 0.0) {
                    kk = kk + 1;
                    slp[kk - 1] = val * (1.0 - 1.0e-15 * (double)gid[n - 1]);
                    id[kk - 1] = n - 1;
                    dst[kk - 1] = FVeLgt[k * MAXNB + p];
                }
            }
        }
        if (kk == 0) {
            for (int p = 0; p < nRcv; p++) r[p] = k;
        } else if (kk <= nRcv) {
            val = 0.0;
            for (int p = 0; p < nRcv; p++) r[p] = k;
            for (int p = 0; p < kk; p++) { r[p] = id[p]; d[p] = dst[p]; val = val + slp[p]; }
            for (int p = 0; p < nRcv; p++) w[p] = slp[p] / val;
        } else {
            for (int p = 0; p < nRcv; p++) r[p] = k;
            quicksort(slp, 1, kk, id);
            int nn = 0;
            val = 0.0;
            for (int p = 0; p < 12; p++) slope[p] = 0.0;
            for (int p = kk; p >= kk - nRcv + 1; p--) {
                nn = nn + 1;
                slope[nn - 1] = slp[p - 1];
                r[nn - 1] = id[p - 1];
                d[nn - 1] = dst[p - 1];   /* dst is not permuted by the sort */
                val = val + slp[p - 1];
            }
            for (int p = 0; p < nRcv; p++) w[p] = slope[p] / val;
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------------
 * Pit filling (functions.F90:1845-2499)
 * ------------------------------------------------------------------------- */
/* edge_tile (2036-2080); border is C-order [nb][2] */
void orc_edge_tile(int nb, double lvl, const int *border, const double *elev, int *ledge)
{
    for (int c = 0; c < nb; c++) {
        ledge[c] = -1;
        if (elev[c] < lvl) {
            double maxe = lvl - 1;
            for (int p = 0; p < FVnNb[c]; p++) {
                int nc = FVnID[c * MAXNB + p] + 1;
                if (nc > 0) {
                    maxe = (elev[nc - 1] > maxe) ? elev[nc - 1] : maxe;
                    if (maxe >= lvl) break;
                }
            }
            if (maxe >= lvl && border[c * 2 + 1] > -1) ledge[c] = border[c * 2 + 1] + 1;
            else if (maxe >= lvl) ledge[c] = 0;
            else ledge[c] = -2;
        } else if (border[c * 2 + 1] > -1) {
            ledge[c] = border[c * 2 + 1] + 1;
        }
    }
}

/* fill_tile (2082-2178); edge is C-order [m][2]. Returns graphnb. */
int orc_fill_tile(int m, int nb, const int *edge, const double *elev, const int *inids,
                  double *fillz, int *labels)
{
    for (int i = 0; i < nb; i++) { labels[i] = -1; fillz[i] = elev[i]; }
    priorityqueue.n = 0; plainqueue.n = 0;
    wg_reset(&graph);
    for (int i = 0; i < m; i++) {
        int c = edge[i * 2];
        pq_push(&priorityqueue, fillz[c], c);
    }
    int nblab = 1;
    while (priorityqueue.n > 0 || plainqueue.n > 0) {
        qnode pt = (plainqueue.n > 0) ? plain_pop(&plainqueue) : pq_pop(&priorityqueue);
        int i = pt.id;
        if (labels[i] <= 0) {
            for (int k = 0; k < FVnNb[i]; k++) {
                int c = FVnID[i * MAXNB + k] + 1;
                if (c > 0 && inids[c - 1] > 0)
                    if (labels[c - 1] > 0 && fillz[c - 1] <= fillz[i]) labels[i] = labels[c - 1];
            }
            if (labels[i] <= 0) { labels[i] = nblab; nblab = nblab + 1; }
        }
        for (int k = 0; k < FVnNb[i]; k++) {
            int c = FVnID[i * MAXNB + k] + 1;
            if (c > 0 && inids[c - 1] > 0) {
                int cc = c - 1;
                if (labels[cc] > 0) {
                    if (labels[cc] != labels[i]) {
                        int lb1 = labels[cc], lb2 = labels[i];
                        if (labels[cc] > labels[i]) { lb1 = labels[i]; lb2 = labels[cc]; }
                        if (fillz[cc] > fillz[i]) wpush(&graph, lb1, lb2, fillz[cc], cc + 1);
                        else wpush(&graph, lb1, lb2, fillz[i], i + 1);
                    }
                } else {
                    labels[cc] = labels[i];
                    if (fillz[cc] <= fillz[i]) {
                        fillz[cc] = fillz[i];
                        plain_push(&plainqueue, fillz[cc], cc);
                    } else {
                        pq_push(&priorityqueue, fillz[cc], cc);
                    }
                }
            }
        }
    }
    for (int i = 0; i < m; i++) {
        if (edge[i * 2 + 1] == 0 || edge[i * 2 + 1] == 2) {
            int c = edge[i * 2];
            wpush(&graph, labels[c], 0, elev[c], c + 1);
        }
    }
    return graph.n;
}

/* graph_nodes (2394-2418): rows (w1, w2, Z, id-1), C-order [graphnb][4] */
void orc_graph_nodes(int graphnb, double *out)
{
    int p = 0;
    while (graph.n > 0) {
        wnode w = wpop(&graph);
        if (p < graphnb) {
            out[p * 4] = w.w1; out[p * 4 + 1] = w.w2; out[p * 4 + 2] = w.Z; out[p * 4 + 3] = w.id - 1;
        }
        p++;
    }
}

/* combine_edges (2331-2392); newgraph C-order [n*12][4]; returns graphnb */
int orc_combine_edges(int m, int n, const double *elev, const int *labels, const int *ins,
                      const int *outs, double *newgraph)
{
    for (int i = 0; i < n; i++) {
        int c = ins[i];
        for (int p = 0; p < FVnNb[c]; p++) {
            int nc = FVnID[c * MAXNB + p] + 1;
            if (nc > 0 && outs[nc - 1] > 0 && labels[c] != labels[nc - 1]) {
                double eo = (elev[c] > elev[nc - 1]) ? elev[c] : elev[nc - 1];
                int lb1, lb2;
                if (labels[c] < labels[nc - 1]) { lb1 = labels[c]; lb2 = labels[nc - 1]; }
                else { lb2 = labels[nc - 1]; lb1 = labels[c]; }
                if (elev[c] > elev[nc - 1]) wpush(&graph, lb1, lb2, eo, c + 1);
                else wpush(&graph, lb1, lb2, eo, nc);
            }
        }
    }
    int graphnb = graph.n, i = 0;
    memset(newgraph, 0, sizeof(double) * (size_t)n * 12 * 4);
    while (graph.n > 0) {
        wnode w = wpop(&graph);
        if (i < n * 12) {
            newgraph[i * 4] = w.w1; newgraph[i * 4 + 1] = w.w2;
            newgraph[i * 4 + 2] = w.Z; newgraph[i * 4 + 3] = w.id - 1;
        }
        i++;
    }
    return graphnb;
}

/* fill_edges (2180-2288); cgraph C-order [m][5]; outputs sized nb */
int orc_fill_edges(int nb, int m, const double *cgraph, int maxnghbs, double *nelev,
                   int *spillrank, int *spillnodes, int *spillid)
{
    char *inFlag = (char *)calloc(nb + 1, 1);
    int *ngbNb = (int *)calloc(nb + 1, sizeof(int));
    int *ranknode = (int *)malloc(sizeof(int) * (nb + 1));
    double *spillz = (double *)malloc(sizeof(double) * (nb + 1));
    size_t W = (size_t)maxnghbs;
    int *rank = (int *)malloc(sizeof(int) * (nb + 1) * W);
    int *ngbhArr = (int *)malloc(sizeof(int) * (nb + 1) * W);
    int *spillnode = (int *)malloc(sizeof(int) * (nb + 1) * W);
    double *spill = (double *)malloc(sizeof(double) * (nb + 1) * W);
    int status = 0;
    for (int k = 0; k < nb; k++) {
        spillnodes[k] = -1; spillrank[k] = -1; nelev[k] = 1.e8; spillz[k + 1] = 1.e8;
        ranknode[k + 1] = -1; spillid[k] = -1;
    }
    nelev[0] = -1.e8;
    for (int k = 0; k < m; k++) {
        int n1 = (int)cgraph[k * 5] + 1, n2 = (int)cgraph[k * 5 + 1] + 1;
        if (n1 < 1 || n1 > nb || n2 < 1 || n2 > nb) { status = -1; goto done; }
        ranknode[n1] = (int)cgraph[k * 5 + 4];
        ngbNb[n1]++; ngbNb[n2]++;
        if (ngbNb[n1] > maxnghbs || ngbNb[n2] > maxnghbs) { status = -2; goto done; }
        size_t a = (size_t)n1 * W + ngbNb[n1] - 1, b = (size_t)n2 * W + ngbNb[n2] - 1;
        ngbhArr[a] = n2; ngbhArr[b] = n1;
        spill[a] = cgraph[k * 5 + 2]; spill[b] = cgraph[k * 5 + 2];
        spillnode[a] = (int)cgraph[k * 5 + 3]; spillnode[b] = (int)cgraph[k * 5 + 3];
        rank[a] = (int)cgraph[k * 5 + 4]; rank[b] = (int)cgraph[k * 5 + 4];
    }
    priorityqueue.n = 0;
    pq_push(&priorityqueue, nelev[0], 1);
    while (priorityqueue.n > 0) {
        qnode pt = pq_pop(&priorityqueue);
        int c = pt.id;
        if (!inFlag[c]) {
            nelev[c - 1] = pt.Z;
            inFlag[c] = 1;
            for (int k = 0; k < ngbNb[c]; k++) {
                size_t a = (size_t)c * W + k;
                int nc = ngbhArr[a];
                if (nc > 0 && !inFlag[nc]) {
                    double z = (spill[a] > nelev[c - 1]) ? spill[a] : nelev[c - 1];
                    pq_push(&priorityqueue, z, nc);
                    if (spillid[nc - 1] >= 0 && z < spillz[nc]) {
                        if (ranknode[c] == rank[a]) {
                            spillnodes[nc - 1] = spillnode[a]; spillid[nc - 1] = c - 1;
                            spillrank[nc - 1] = rank[a]; spillz[nc] = z;
                        }
                    } else if (spillid[nc - 1] < 0) {
                        if (c == 1 || ranknode[c] == rank[a]) {
                            spillnodes[nc - 1] = spillnode[a]; spillid[nc - 1] = c - 1;
                            spillrank[nc - 1] = rank[a]; spillz[nc] = z;
                        }
                    }
                }
            }
        }
    }
done:
    free(inFlag); free(ngbNb); free(ranknode); free(spillz);
    free(rank); free(ngbhArr); free(spillnode); free(spill);
    return status;
}

/* fill_depressions (2290-2329) */
void orc_fill_depressions(int m, int nb, double lvl, const double *dem, const double *fillp,
                          const int *wsh, const double *ggraph, double *elev)
{
    for (int k = 0; k < m; k++) {
        elev[k] = dem[k];
        if (dem[k] > lvl) {
            int n = wsh[k] + 1;
            if (n >= 1 && n <= nb) {
                if (dem[k] < fillp[k] && fillp[k] > ggraph[n - 1]) elev[k] = fillp[k];
                else if (dem[k] <= ggraph[n - 1]) elev[k] = ggraph[n - 1];
            }
        }
    }
}

/* label_pits (2420-2499) */
void orc_label_pits(int nb, double lvl, const double *fill, int *label)
{
    char *flag = (char *)calloc(nb, 1);
    int lbl = 0;
    simplequeue.n = 0;
    for (int i = 0; i < nb; i++) label[i] = -1;
    for (int i = 0; i < nb; i++) {
        if (fill[i] > lvl && !flag[i]) {
            int noflow = 1;
            for (int k = 0; k < FVnNb[i]; k++) {
                int c = FVnID[i * MAXNB + k] + 1;
                if (c > 0 && fill[i] > fill[c - 1]) { noflow = 0; break; }
            }
            if (noflow) {
                flag[i] = 1;
                lbl = lbl + 1;
                label[i] = lbl;
                simple_push(&simplequeue, i);
                while (simplequeue.n > 0) {
                    int p = simple_pop(&simplequeue);
                    for (int k = 0; k < FVnNb[p]; k++) {
                        int c = FVnID[p * MAXNB + k] + 1;
                        if (c > 0 && fill[c - 1] == fill[p] && !flag[c - 1]) {
                            simple_push(&simplequeue, c - 1);
                            label[c - 1] = lbl;
                            flag[c - 1] = 1;
                        }
                    }
                }
            }
        } else {
            flag[i] = 1;
        }
    }
    free(flag);
}

/* pits_cons (2005-2034): 1-based position of each id in pitnb */
void orc_pits_cons(int m, int n, const int *pitids, const int *pitnb, int *npitids)
{
    for (int i = 0; i < m; i++) {
        npitids[i] = pitids[i];
        if (pitids[i] > -1) {
            for (int k = 0; k < n; k++)
                if (pitids[i] == pitnb[k]) { npitids[i] = k + 1; break; }
        }
    }
}

/* fill_dir (1845-1899) */
void orc_fill_dir(int m, int n, const int *spill, const int *pitids, const double *h, int *ptdir)
{
    char *flag = (char *)calloc(n, 1);
    double one = 1.0;
    for (int i = 0; i < n; i++) ptdir[i] = -1;
    priorityqueue.n = 0;
    for (int c = 0; c < m; c++) {
        int i = spill[c];
        flag[i] = 1;
        ptdir[i] = 1;
        pq_push(&priorityqueue, one, i);
    }
    while (priorityqueue.n > 0) {
        qnode pt = pq_pop(&priorityqueue);
        int i = pt.id;
        for (int k = 0; k < FVnNb[i]; k++) {
            int c = FVnID[i * MAXNB + k] + 1;
            if (c > 0 && !flag[c - 1] && pitids[c - 1] > -1 && h[c - 1] >= h[i]) {
                flag[c - 1] = 1;
                if (ptdir[c - 1] < ptdir[i] + 1) {
                    ptdir[c - 1] = ptdir[i] + 1;
                    pq_push(&priorityqueue, pt.Z + one, c - 1);
                }
            }
        }
    }
    free(flag);
}

/* nghb_dir (1901-1969): relaxing label-correcting pass */
void orc_nghb_dir(int n, const int *pitids, const double *h, const int *ptdir, int *nptdir)
{
    priorityqueue.n = 0;
    for (int c = 0; c < n; c++) {
        nptdir[c] = ptdir[c];
        if (nptdir[c] > -1) pq_push(&priorityqueue, (double)nptdir[c], c);
    }
    while (priorityqueue.n > 0) {
        qnode pt = pq_pop(&priorityqueue);
        int i = pt.id, di = nptdir[i];
        if ((int)pt.Z > di) continue;
        for (int k = 0; k < FVnNb[i]; k++) {
            int c = FVnID[i * MAXNB + k] + 1;
            if (c > 0 && pitids[c - 1] > -1 && h[c - 1] >= h[i]) {
                if (nptdir[c - 1] < 0 || di + 1 < nptdir[c - 1]) {
                    nptdir[c - 1] = di + 1;
                    pq_push(&priorityqueue, (double)(di + 1), c - 1);
                }
            }
        }
    }
}

/* getpitvol (1971-2003); hlvl/vol C-order [n][4] */
void orc_getpitvol(int m, int n, const double *hlvl, const double *elev, const int *pit,
                   const int *id, double *vol)
{
    for (int i = 0; i < n * 4; i++) vol[i] = 0.0;
    for (int i = 0; i < m; i++) {
        int p = pit[i];
        if (p > -1 && id[i] > 0 && p < n) {
            for (int k = 0; k < 4; k++)
                if (hlvl[p * 4 + k] > elev[i])
                    vol[p * 4 + k] = vol[p * 4 + k] + (hlvl[p * 4 + k] - elev[i]) * FVarea[i];
        }
    }
}

/* ---------------------------------------------------------------------------
 * Exact solves used in place of PETSc KSP (the oracle defines the exact
 * solution of the assembled systems).
 *
 * Flow system (I - W^T) q = b with W given by receivers: W[i, rcv[i,k]] =
 * wgt[i,k] for rcv[i,k] != i (flowplex.py:429-478).  Solved by one sweep in
 * topological order; each node sums its donors in ascending donor index.
 * Returns the number of nodes that could not be ordered (cycle members).
 * ------------------------------------------------------------------------- */
int orc_flow_solve(int nb, int R, const int *rcv, const double *wgt, const double *b, double *q)
{
    int *indeg = (int *)calloc(nb, sizeof(int));
    int *dptr = (int *)calloc(nb + 1, sizeof(int));
    for (int i = 0; i < nb; i++)
        for (int k = 0; k < R; k++) { int r = rcv[i * R + k]; if (r != i && r >= 0) dptr[r + 1]++; }
    for (int i = 0; i < nb; i++) dptr[i + 1] += dptr[i];
    int nnz = dptr[nb];
    int *don = (int *)malloc(sizeof(int) * (nnz + 1));
    double *dw = (double *)malloc(sizeof(double) * (nnz + 1));
    int *fill = (int *)calloc(nb, sizeof(int));
    for (int i = 0; i < nb; i++)           /* ascending donor index per row */
        for (int k = 0; k < R; k++) {
            int r = rcv[i * R + k];
            if (r != i && r >= 0) { int s = dptr[r] + fill[r]++; don[s] = i; dw[s] = wgt[i * R + k]; }
        }
    for (int i = 0; i < nb; i++) indeg[i] = dptr[i + 1] - dptr[i];
    int *queue = (int *)malloc(sizeof(int) * (nb + 1));
    int head = 0, tail = 0;
    for (int i = 0; i < nb; i++) if (indeg[i] == 0) queue[tail++] = i;
    while (head < tail) {
        int i = queue[head++];
        double s = b[i];
        for (int t = dptr[i]; t < dptr[i + 1]; t++) s = s + dw[t] * q[don[t]];
        q[i] = s;
        for (int k = 0; k < R; k++) {
            int r = rcv[i * R + k];
            if (r != i && r >= 0) { if (--indeg[r] == 0) queue[tail++] = r; }
        }
    }
    int left = nb - tail;
    free(indeg); free(dptr); free(don); free(dw); free(fill); free(queue);
    return left;
}

/* SPL system (SPL.py:45-114, 297): row i is
 *   (1 + sum_k c_ik) h_i - sum_k c_ik h_rcv(i,k) = hOld_i
 * with c already zeroed for self receivers.  Receivers are solved first. */
int orc_spl_solve(int nb, int R, const int *rcv, const double *c, const double *hold, double *h)
{
    int *nout = (int *)calloc(nb, sizeof(int));
    int *dptr = (int *)calloc(nb + 1, sizeof(int));
    for (int i = 0; i < nb; i++)
        for (int k = 0; k < R; k++) {
            int r = rcv[i * R + k];
            if (r != i && r >= 0 && c[i * R + k] != 0.0) { nout[i]++; dptr[r + 1]++; }
        }
    for (int i = 0; i < nb; i++) dptr[i + 1] += dptr[i];
    int *up = (int *)malloc(sizeof(int) * (dptr[nb] + 1));
    int *fill = (int *)calloc(nb, sizeof(int));
    for (int i = 0; i < nb; i++)
        for (int k = 0; k < R; k++) {
            int r = rcv[i * R + k];
            if (r != i && r >= 0 && c[i * R + k] != 0.0) up[dptr[r] + fill[r]++] = i;
        }
    int *queue = (int *)malloc(sizeof(int) * (nb + 1));
    int head = 0, tail = 0;
    for (int i = 0; i < nb; i++) if (nout[i] == 0) queue[tail++] = i;
    while (head < tail) {
        int i = queue[head++];
        double num = hold[i], den = 1.0;
        for (int k = 0; k < R; k++) {
            double ck = c[i * R + k];
            int r = rcv[i * R + k];
            if (r != i && r >= 0 && ck != 0.0) { num = num + ck * h[r]; }
            den = den + ck;
        }
        h[i] = num / den;
        for (int t = dptr[i]; t < dptr[i + 1]; t++) if (--nout[up[t]] == 0) queue[tail++] = up[t];
    }
    int left = nb - tail;
    free(nout); free(dptr); free(up); free(fill); free(queue);
    return left;
}

/* ---------------------------------------------------------------------------
 * Marine routing (seaplex.py:_matOcean, seaplex.py:137-238)
 * ------------------------------------------------------------------------- */
/* mfdrcvrs (functions.F90:1673-1785): receivers of the marine routing,
 * C-order [nb][12].  Every strictly lower neighbour is a receiver (up to
 * nRcv above `sl`, 12 at or below it) with the equal weight `1. / kk`; the
 * literal `1.` is a default (single precision) real in the reference's build
 * (no -fdefault-real-8), so the weight is 1/kk rounded to float, widened. */
int orc_mfdrcvrs(int nb, int nRcv, double exp_, const double *elev, double sl,
                 const int *gid, int *rcv, double *dist, double *wgt, powfn_t powfn)
{
    if (nRcv < 1 || nRcv > 12) return -1;
    if (!powfn) powfn = pow;
    for (int i = 0; i < nb * 12; i++) { rcv[i] = -1; dist[i] = 0.0; wgt[i] = 0.0; }
    for (int k = 0; k < nb; k++) {
        int *r = &rcv[k * 12];
        double *d = &dist[k * 12], *w = &wgt[k * 12];
        int ngbs;
        double fexp;
        if (elev[k] > sl) { ngbs = nRcv; fexp = exp_; }
        else { ngbs = 12; fexp = 0.01; }
        double slp[12], dst[12];
        int id[12];
        for (int p = 0; p < 12; p++) { slp[p] = 0.0; id[p] = 0; dst[p] = 0.0; }
        int kk = 0;
        double val = 0.0;
        for (int p = 0; p < FVnNb[k]; p++) {
            int n = FVnID[k * MAXNB + p] + 1;
            if (n > 0 && FVeLgt[k * MAXNB + p] > 0.0) {
                val = powfn(elev[k] - elev[n - 1], fexp) / FVeLgt[k * MAXNB + p];
                if (val > 0.0) {
                    kk = kk + 1;
                    slp[kk - 1] = val * (1.0 - 1.0e-15 * (double)gid[n - 1]);
                    id[kk - 1] = n - 1;
                    dst[kk - 1] = FVeLgt[k * MAXNB + p];
                }
            }
        }
        const double wk = kk > 0 ? (double)(1.0f / (float)kk) : 0.0;
        if (kk == 0) {
            for (int p = 0; p < 12; p++) r[p] = k;
        } else if (kk <= ngbs) {
            for (int p = 0; p < ngbs; p++) r[p] = k;
            for (int p = 0; p < kk; p++) { r[p] = id[p]; d[p] = dst[p]; }
            for (int p = 0; p < ngbs; p++) if (slp[p] > 0.0) w[p] = wk;
        } else {
            for (int p = 0; p < ngbs; p++) r[p] = k;
            quicksort(slp, 1, kk, id);
            int nn = 0;
            for (int p = kk; p >= kk - ngbs + 1; p--) {
                nn = nn + 1;
                r[nn - 1] = id[p - 1];
                d[nn - 1] = dst[p - 1];
            }
            for (int p = 0; p < ngbs; p++) if (slp[p] > 0.0) w[p] = wk;
        }
    }
    return 0;
}

/* epsfill (functions.F90:2633-2697): priority-flood from the cells below `sl`
 * that touch a cell at or above it; every cell reached is raised to at least
 * the next double above the cell it was reached from (nearest(x, 1.0)), so
 * the filled surface has no flats.  Cells below `sl` keep their value. */
int orc_epsfill(int nb, double sl, const double *elev, double *fillz)
{
    char *flag = (char *)calloc(nb > 0 ? nb : 1, 1);
    if (!flag) return -1;
    for (int i = 0; i < nb; i++) fillz[i] = elev[i];
    priorityqueue.n = 0;
    for (int i = 0; i < nb; i++) {
        if (fillz[i] < sl) {
            flag[i] = 1;
            for (int k = 0; k < FVnNb[i]; k++) {
                int c = FVnID[i * MAXNB + k];
                if (c >= 0 && fillz[c] >= sl) {
                    pq_push(&priorityqueue, fillz[i], i);
                    break;
                }
            }
        }
    }
    while (priorityqueue.n > 0) {
        qnode pt = pq_pop(&priorityqueue);
        int i = pt.id;
        for (int k = 0; k < FVnNb[i]; k++) {
            int c = FVnID[i * MAXNB + k];
            if (c >= 0 && !flag[c]) {
                flag[c] = 1;
                double h = nextafter(fillz[i], INFINITY);
                if (fillz[c] > h) {
                    pq_push(&priorityqueue, fillz[c], c);
                } else {
                    fillz[c] = h;
                    pq_push(&priorityqueue, fillz[c], c);
                }
            }
        }
    }
    free(flag);
    return 0;
}
