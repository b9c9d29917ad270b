// Finite-volume geometry of the mesh on the device: a vertex-parallel
// restatement of the Fortran `definetin` (fortran/functions.F90:2715-2940)
// with its helpers (distance 368-393, great_circle_distance 337-366,
// spherical2lonlat 316-335, slerpmidpt 425-452, striarea 538-577,
// gtriarea 579-616).  One thread per vertex walks its edges in global edge
// order (neighbour order) and its first 12 cells in cell order, accumulating
// Voronoi face lengths and cell areas in the reference's order.
#include "gs_plan.cuh"

namespace gs {

__device__ double g_norm2(double x, double y, double z) {
    double v[3] = {x, y, z};
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

__device__ void g_lonlat(const double* p, double* lon, double* lat) {
    const double pi = 3.1415926535897932;
    double r = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    double la = asin(p[2] / r) * (180.0 / pi);
    double lo = atan2(p[1], p[0]) * (180.0 / pi);
    *lat = la * pi / 180.0;
    *lon = lo * pi / 180.0;
}

__device__ double g_distance(const double* p1, const double* p2) {
    if (p2[2] == 0.0 && p1[2] == 0.0) return g_norm2(p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]);
    double radius = g_norm2(p1[0], p1[1], p1[2]);
    double lon1, lat1, lon2, lat2;
    g_lonlat(p1, &lon1, &lat1);
    g_lonlat(p2, &lon2, &lat2);
    double c1 = cos(lat1), s1 = sin(lat1), c2 = cos(lat2), s2 = sin(lat2);
    double dlon = lon1 - lon2, clon = cos(dlon), slon = sin(dlon);
    double a = c2 * slon, b = c1 * s2 - s1 * c2 * clon;
    return radius * atan2(sqrt(a * a + b * b), (s1 * s2 + c1 * c2 * clon));
}

__device__ void g_slerpmid(const double* p1, const double* p2, double* m) {
    double n1 = g_norm2(p1[0], p1[1], p1[2]), n2 = g_norm2(p2[0], p2[1], p2[2]);
    double v1[3], v2[3], pt[3];
    for (int i = 0; i < 3; i++) { v1[i] = p1[i] / n1; v2[i] = p2[i] / n2; }
    double d = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
    double a = acos(d);
    for (int i = 0; i < 3; i++) pt[i] = sin(0.5 * a) * v1[i] / sin(a) + sin(0.5 * a) * v2[i] / sin(a);
    double np_ = g_norm2(pt[0], pt[1], pt[2]);
    for (int i = 0; i < 3; i++) m[i] = n1 * pt[i] / np_;
}

__device__ double g_striarea(const double* v1, const double* v2, const double* v3) {
    const double pi = 3.1415926535897932;
    double r = sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
    double lon1, lat1, lon2, lat2, lon3, lat3;
    g_lonlat(v1, &lon1, &lat1);
    g_lonlat(v2, &lon2, &lat2);
    g_lonlat(v3, &lon3, &lat3);
    double a = acos(sin(lat2) * sin(lat3) + cos(lat2) * cos(lat3) * cos(lon3 - lon2));
    double b = acos(sin(lat1) * sin(lat3) + cos(lat1) * cos(lat3) * cos(lon3 - lon1));
    double c = acos(sin(lat1) * sin(lat2) + cos(lat1) * cos(lat2) * cos(lon2 - lon1));
    double al = acos((cos(a) - cos(b) * cos(c)) / (sin(b) * sin(c)));
    double be = acos((cos(b) - cos(a) * cos(c)) / (sin(a) * sin(c)));
    double ga = acos((cos(c) - cos(a) * cos(b)) / (sin(a) * sin(b)));
    return (al + be + ga - pi) * (r * r);
}

__device__ double g_heron(const double* p1, const double* p2, const double* p3) {
    double x1 = p1[0], x2 = p2[0], x3 = p3[0], y1 = p1[1], y2 = p2[1], y3 = p3[1];
    if ((x1 == x2 && y1 == y2) || (x1 == x3 && y1 == y3) || (x2 == x3 && y2 == y3)) return 0.0;
    double l1 = sqrt((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2));
    double l2 = sqrt((x2 - x3) * (x2 - x3) + (y2 - y3) * (y2 - y3));
    double l3 = sqrt((x3 - x1) * (x3 - x1) + (y3 - y1) * (y3 - y1));
    double p = (l1 + l2 + l3) / 2;
    return sqrt(p * (p - l1) * (p - l2) * (p - l3));
}

// vptr/vedge: per-vertex edges in edge order; cptr/vcell: per-vertex cells in cell order
__global__ void k_fv_geometry(int n, const double* __restrict__ xyz, const int* __restrict__ edges,
                              const int* __restrict__ vptr, const int* __restrict__ vedge,
                              const int* __restrict__ cells_edges, const double* __restrict__ cc,
                              const int* __restrict__ cptr, const int* __restrict__ vcell, int curved,
                              int* nnb, int* ngb, double* elgt, double* vdist, double* farea, double* narea) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double* c0 = xyz + 3 * (size_t)k;
    int deg = vptr[k + 1] - vptr[k];
    if (deg > 12) deg = 12;
    int nb[12];
    for (int s = 0; s < 12; s++) {
        ngb[(size_t)k * 12 + s] = -1;
        elgt[(size_t)k * 12 + s] = 0.0;
        vdist[(size_t)k * 12 + s] = 0.0;
    }
    for (int s = 0; s < deg; s++) {
        int e = vedge[vptr[k] + s];
        int a = edges[2 * e], b = edges[2 * e + 1];
        int o = (a == k) ? b : a;
        nb[s] = o;
        ngb[(size_t)k * 12 + s] = o;
        elgt[(size_t)k * 12 + s] = g_distance(c0, xyz + 3 * (size_t)o);
    }
    nnb[k] = deg;
    double area = 0.0;
    int ncell = cptr[k + 1] - cptr[k];
    if (ncell > 12) ncell = 12;
    for (int q = 0; q < ncell; q++) {
        int c = vcell[cptr[k] + q];
        for (int e = 0; e < 3; e++) {
            int eg = cells_edges[3 * (size_t)c + e];
            int e1 = edges[2 * eg], e2 = edges[2 * eg + 1];
            if (k != e1 && k != e2) continue;
            double mid[3];
            const double* p1 = xyz + 3 * (size_t)e1;
            const double* p2 = xyz + 3 * (size_t)e2;
            if (curved) g_slerpmid(p1, p2, mid);
            else for (int d = 0; d < 3; d++) mid[d] = 0.5 * (p1[d] + p2[d]);
            int want = (e1 == k) ? e2 : e1;
            int id = -1;
            for (int s = 0; s < deg; s++)
                if (nb[s] == want) { id = s; break; }
            const double* ccp = cc + 3 * (size_t)c;
            double dist = g_distance(mid, ccp);
            if (id >= 0) vdist[(size_t)k * 12 + id] += dist;
            area += curved ? g_striarea(c0, mid, ccp) : g_heron(c0, mid, ccp);
        }
    }
    narea[k] = area;
    farea[k] = (area != area) ? 0.0 : area;
}

}  // namespace gs

extern "C" int gs_mesh_geometry(int64_t n, const double* xyz, int64_t m, const int32_t* edges,
                                const int32_t* vptr, const int32_t* vedge, int64_t ncell,
                                const int32_t* cells_edges, const double* cc, const int32_t* cptr,
                                const int32_t* vcell, int32_t curved, int32_t* nnb, int32_t* ngb,
                                double* elgt, double* vdist, double* farea, double* narea, void* stream) {
    if (n < 0 || m < 0 || ncell < 0) {
        gs::set_error(GS_EINVAL, "gs_mesh_geometry: negative size");
        return GS_EINVAL;
    }
    if (n == 0) return GS_OK;
    if (!xyz || !edges || !vptr || !vedge || !cells_edges || !cc || !cptr || !vcell || !nnb || !ngb || !elgt ||
        !vdist || !farea || !narea) {
        gs::set_error(GS_EINVAL, "gs_mesh_geometry: null argument");
        return GS_EINVAL;
    }
    gs::k_fv_geometry<<<gs::grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
        (int)n, xyz, edges, vptr, vedge, cells_edges, cc, cptr, vcell, curved, nnb, ngb, elgt, vdist, farea,
        narea);
    GS_LAUNCH();
    return GS_OK;
}
