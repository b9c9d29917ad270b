// Output fields of one step, packed on the device for the HDF5 writer:
// WriteMesh._outputMesh (outmesh.py:252-478) writes every field as float32
// after two edits, values at or below DISCHARGE_FLOOR (1e-8,
// tools/constants.py:51) raised to it for FA, fillFA and sedLoad, and FA and
// fillFA set to 1 on the sea vertices (seaID of the last mask built:
// hillslope.py:620 after a step, flowplex.py:493 before the first one).  One
// launch reads each field once and writes the float32 rows, so a step's output
// leaves the device as 36 bytes per vertex.
#include "gs_plan.cuh"

namespace gs {

constexpr double DISCHARGE_FLOOR = 1.0e-8;

__global__ void k_output_pack(int n, const double* __restrict__ h, const double* __restrict__ ced,
                              const double* __restrict__ eb, const double* __restrict__ wf,
                              const double* __restrict__ ffa, const double* __restrict__ fa,
                              const double* __restrict__ vsed, const double* __restrict__ up,
                              const double* __restrict__ rain, const uint8_t* __restrict__ sea, float* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t N = (size_t)n;
    const bool s = sea[k] != 0;
    double a = ffa[k];
    if (a <= DISCHARGE_FLOOR) a = DISCHARGE_FLOOR;
    if (s) a = 1.0;
    double b = fa[k];
    if (b <= DISCHARGE_FLOOR) b = DISCHARGE_FLOOR;
    if (s) b = 1.0;
    double c = vsed[k];
    if (c <= DISCHARGE_FLOOR) c = DISCHARGE_FLOOR;
    // double -> float rounds to nearest even, as the HDF5 library's conversion
    out[k] = (float)h[k];
    out[N + k] = (float)ced[k];
    out[2 * N + k] = (float)eb[k];
    out[3 * N + k] = (float)wf[k];
    out[4 * N + k] = (float)a;
    out[5 * N + k] = (float)b;
    out[6 * N + k] = (float)c;
    if (up) out[7 * N + k] = (float)up[k];
    if (rain) out[8 * N + k] = (float)rain[k];
}

int output_fields(gs_plan* p, const double* h, const double* cum_ed, const double* eb, const double* water_filled,
                  const double* fill_fa, const double* fa, const double* vsed, const double* upsub,
                  const double* rain, const uint8_t* sea, float* out) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    if (!sea) {
        if (!p->hill_sea) {
            set_error(GS_EINVAL, "no land/sea mask: pass one, or run gs_hillslope first");
            return GS_EINVAL;
        }
        sea = p->dsea;
    }
    const int B = 256;
    launch(p, k_output_pack, grid_for(n, B), B, n, h, cum_ed, eb, water_filled, fill_fa, fa, vsed, upsub, rain,
           sea, out);
    GS_LAUNCH();
    return GS_OK;
}

}  // namespace gs
