// Per-step forcing: UnstMesh.applyForces (unstructuredmesh.py:743-794) with
// _updateRain (924-972, bl = max(rain, 0) * larea), applyTectonics (903-922,
// h += upsub * dt) and _drainOpenEdges (796-901) for 'o' boundary edges.
#include "gs_plan.cuh"

namespace gs {

__global__ void k_force(int n, double* h, const double* __restrict__ rain, const double* __restrict__ upsub,
                        double dt, const double* __restrict__ larea, double* bl) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double r = rain[i];
    if (r < 0) r = 0.0;
    bl[i] = r * larea[i];
    if (upsub) h[i] = h[i] + upsub[i] * dt;
}

// one round of the label-correcting candidate sweep over open nodes: every
// pending open node takes the minimum over neighbours assigned in the
// previous round (interior nodes start assigned)
__global__ void k_open_round(int m, const int* __restrict__ ids, int n, const int* __restrict__ nbr,
                             const int8_t* __restrict__ nnb, const uint8_t* __restrict__ assigned_in,
                             const double* __restrict__ vals_in, uint8_t* assigned_out, double* vals_out,
                             int* pending) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    int i = ids[t];
    if (assigned_in[i]) return;
    double mn = INFINITY;
    for (int s = 0; s < nnb[i]; s++) {
        int j = nbr[(size_t)s * n + i];
        if (j >= 0 && assigned_in[j] && vals_in[j] < mn) mn = vals_in[j];
    }
    if (mn < INFINITY) {
        vals_out[i] = mn;
        assigned_out[i] = 1;
    } else {
        atomicAdd(pending, 1);
    }
}

__global__ void k_open_init(int n, const uint8_t* __restrict__ is_open, const double* __restrict__ h,
                            uint8_t* a0, uint8_t* a1, double* v0, double* v1) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a0[i] = a1[i] = is_open[i] ? 0 : 1;
    v0[i] = v1[i] = h[i];
}

__global__ void k_open_sync(int m, const int* __restrict__ ids, const uint8_t* __restrict__ a_src,
                            const double* __restrict__ v_src, uint8_t* a_dst, double* v_dst) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    int i = ids[t];
    a_dst[i] = a_src[i];
    v_dst[i] = v_src[i];
}

__global__ void k_open_apply(int m, const int* __restrict__ ids, const double* __restrict__ vals, double sl,
                             double* h) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    int i = ids[t];
    double cur = h[i];
    double runmin = cur < vals[i] ? cur : vals[i];
    h[i] = (cur < sl) ? cur : runmin;
}

int apply_forces(gs_plan* p, double* h, const double* rain, const double* upsub, double dt,
                 double sealevel, double* bl) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    const int B = 256, G = grid_for(n, B);
    launch(p, k_force, G, B, n, h, rain, upsub, dt, (const double*)p->larea, bl);
    GS_LAUNCH();
    if (!p->flat || p->n_open == 0) return GS_OK;
    const int m = p->n_open;
    uint8_t* a0 = (uint8_t*)p->flagbuf;               // n bytes
    uint8_t* a1 = (uint8_t*)p->scanbuf;
    double* v0 = p->q2;
    double* v1 = p->q3;
    launch(p, k_open_init, G, B, n, (const uint8_t*)p->open_mask, (const double*)h, a0, a1, v0, v1);
    GS_LAUNCH();
    for (int round = 0; round <= m; round++) {
        GS_CUDA(cudaMemsetAsync(p->i_scalar + 9, 0, sizeof(int), p->stream));
        launch(p, k_open_round, grid_for(m, B), B, m, (const int*)p->open_ids, n, (const int*)p->nbr,
               (const int8_t*)p->nnb, (const uint8_t*)a0, (const double*)v0, a1, v1, p->i_scalar + 9);
        launch(p, k_open_sync, grid_for(m, B), B, m, (const int*)p->open_ids, (const uint8_t*)a1,
               (const double*)v1, a0, v0);
        GS_LAUNCH();
        int pending = 0;
        GS_CUDA(cudaMemcpyAsync(&pending, p->i_scalar + 9, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        if (pending == 0) break;
    }
    launch(p, k_open_apply, grid_for(m, B), B, m, (const int*)p->open_ids, (const double*)v0, sealevel, h);
    GS_LAUNCH();
    return GS_OK;
}

}  // namespace gs
