// extern "C" boundary of libgospl_b200.so (declarations in include/gospl_b200.h).
#include <algorithm>
#include <cstring>
#include <exception>
#include <string>

#include "gs_plan.cuh"

namespace gs {

static thread_local std::string g_msg;
static thread_local int g_code = GS_OK;

void set_error(int code, const std::string& msg) {
    g_code = code;
    g_msg = msg;
}
int last_code() { return g_code; }

void prof_begin(gs_plan* p, const void* fn, cudaEvent_t* stop) {
    int idx = -1;
    for (size_t k = 0; k < p->prof_fn.size(); k++)
        if (p->prof_fn[k] == fn) { idx = (int)k; break; }
    if (idx < 0) {
        idx = (int)p->prof_fn.size();
        p->prof_fn.push_back(fn);
    }
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return;
    if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return; }
    cudaEventRecord(a, p->stream);
    p->prof_ev.push_back(a);
    p->prof_ev.push_back(b);
    p->prof_idx.push_back(idx);
    p->prof_stream.push_back(p->stream == p->side_a ? 1 : (p->stream == p->side_b ? 2 : 0));
    *stop = b;
}

int plan_create(int64_t nb, const int32_t* nnb, const int32_t* ngb, const double* elgt, const double* vdist,
                const double* farea, const double* larea, const int32_t* outlet_ids, int64_t n_outlet,
                const int32_t* open_ids, int64_t n_open, int flat, int flow_dir, gs_plan** out);
int plan_destroy(gs_plan* p);

}  // namespace gs

#define GS_GUARD(body)                                                        \
    try {                                                                     \
        body                                                                  \
    } catch (const std::exception& e) {                                       \
        gs::set_error(GS_EINVAL, std::string("exception: ") + e.what());     \
        return GS_EINVAL;                                                     \
    } catch (...) {                                                           \
        gs::set_error(GS_EINVAL, "unknown exception");                       \
        return GS_EINVAL;                                                     \
    }

#define NEED(p)                                                               \
    do {                                                                      \
        if (!(p)) {                                                           \
            gs::set_error(GS_EINVAL, std::string("null argument: ") + #p);    \
            return GS_EINVAL;                                                 \
        }                                                                     \
    } while (0)

extern "C" {

int gs_version(void) { return 100; }

int gs_last_error(char* buf, int64_t len) {
    if (buf && len > 0) {
        std::strncpy(buf, gs::g_msg.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return gs::g_code;
}

int gs_plan_create(int64_t nb, const int32_t* nnb, const int32_t* ngb, const double* elgt,
                   const double* vdist, const double* farea, const double* larea,
                   const int32_t* outlet_ids, int64_t n_outlet, const int32_t* open_ids, int64_t n_open,
                   int32_t flat_model, int32_t flow_dir, gs_plan** out) {
    GS_GUARD(return gs::plan_create(nb, nnb, ngb, elgt, vdist, farea, larea, outlet_ids, n_outlet, open_ids,
                                    n_open, flat_model, flow_dir, out);)
}

int gs_plan_destroy(gs_plan* plan) { GS_GUARD(return gs::plan_destroy(plan);) }

int gs_plan_tune(gs_plan* plan, int32_t knob, int32_t value) {
    NEED(plan);
    GS_GUARD(return gs::plan_tune(plan, knob, value);)
}

int gs_plan_tuning(const gs_plan* plan, int32_t knob) { return plan ? gs::plan_tuning(plan, knob) : -1; }

int gs_plan_set_deposition(gs_plan* plan, double g) {
    NEED(plan);
    if (!(g >= 0.0)) {
        gs::set_error(GS_EINVAL, "deposition coefficient G must be >= 0");
        return GS_EINVAL;
    }
    plan->fdepa = g;
    return GS_OK;
}

int gs_plan_set_precision(gs_plan* plan, int32_t bits, double tol) {
    NEED(plan);
    if ((bits != 32 && bits != 64) || !(tol > 0.0) || !(tol < 1.0)) {
        gs::set_error(GS_EINVAL, "precision: bits must be 32 or 64 and 0 < tol < 1");
        return GS_EINVAL;
    }
    plan->fp32 = bits == 32 ? 1 : 0;
    plan->refine_tol = tol;
    return GS_OK;
}

int gs_plan_record(gs_plan* plan, int32_t nslots) {
    NEED(plan);
    GS_GUARD(return gs::record_setup(plan, nslots);)
}

int gs_plan_record_slot(gs_plan* plan, int32_t slot) {
    NEED(plan);
    GS_GUARD(return gs::record_select(plan, slot);)
}

int gs_adjoint_step(gs_plan* plan, int32_t slot, double* lam, const double* rain, double k_scalar,
                    const double* k_field, double d, double m, double dt, double sealevel, double cda, double cdm,
                    double rtol, int32_t max_iter, double* grad_k, double* grad_u, double* grad_rain,
                    double* grad_bl) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(lam);
        NEED(rain);
    }
    if (!(dt > 0)) {
        gs::set_error(GS_EINVAL, "dt must be positive");
        return GS_EINVAL;
    }
    GS_GUARD(return gs::adjoint_step(plan, slot, lam, rain, k_scalar, k_field, d, m, dt, sealevel, cda, cdm, rtol,
                                     max_iter, grad_k, grad_u, grad_rain, grad_bl);)
}

int gs_plan_set_members(gs_plan* plan, int32_t nmem, const int64_t* start, const double* maxarea) {
    NEED(plan);
    NEED(start);
    NEED(maxarea);
    GS_GUARD(return gs::set_members(plan, nmem, start, maxarea);)
}

int gs_plan_set_stream(gs_plan* plan, void* stream) {
    NEED(plan);
    plan->stream = (cudaStream_t)stream;
    return GS_OK;
}

int64_t gs_plan_launches(const gs_plan* plan) { return plan ? plan->launches : -1; }

int gs_plan_profile(gs_plan* plan, int32_t enable) {
    NEED(plan);
    for (cudaEvent_t e : plan->prof_ev) cudaEventDestroy(e);
    plan->prof_ev.clear();
    plan->prof_idx.clear();
    plan->prof_stream.clear();
    plan->profiling = enable ? 1 : 0;
    return GS_OK;
}

int gs_plan_profile_report(gs_plan* plan, char* buf, int64_t len) {
    NEED(plan);
    GS_CUDA(cudaStreamSynchronize(plan->stream));
    std::vector<double> tot(plan->prof_fn.size(), 0.0);
    std::vector<long> cnt(plan->prof_fn.size(), 0);
    for (size_t q = 0; q + 1 < plan->prof_ev.size(); q += 2) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, plan->prof_ev[q], plan->prof_ev[q + 1]) == cudaSuccess) {
            tot[plan->prof_idx[q / 2]] += ms;
            cnt[plan->prof_idx[q / 2]] += 1;
        }
    }
    std::string out;
    for (size_t k = 0; k < plan->prof_fn.size(); k++) {
        const char* name = "?";
        cudaFuncGetName(&name, plan->prof_fn[k]);
        out += std::string(name) + " " + std::to_string(cnt[k]) + " " + std::to_string(tot[k]) + "\n";
    }
    if (buf && len > 0) {
        std::strncpy(buf, out.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return (int)std::min<size_t>(out.size(), (size_t)0x7fffffff);
}

int gs_plan_profile_trace(gs_plan* plan, char* buf, int64_t len) {
    NEED(plan);
    GS_CUDA(cudaDeviceSynchronize());
    std::string out;
    if (plan->prof_ev.size() >= 2) {
        cudaEvent_t t0 = plan->prof_ev[0];
        for (size_t q = 0; q + 1 < plan->prof_ev.size(); q += 2) {
            float a = 0.f, b = 0.f;
            if (cudaEventElapsedTime(&a, t0, plan->prof_ev[q]) != cudaSuccess) continue;
            if (cudaEventElapsedTime(&b, t0, plan->prof_ev[q + 1]) != cudaSuccess) continue;
            const char* name = "?";
            cudaFuncGetName(&name, plan->prof_fn[plan->prof_idx[q / 2]]);
            out += std::string(name) + " " + std::to_string(plan->prof_stream[q / 2]) + " " +
                   std::to_string(a) + " " + std::to_string(b) + "\n";
        }
    }
    if (buf && len > 0) {
        std::strncpy(buf, out.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return (int)std::min<size_t>(out.size(), (size_t)0x7fffffff);
}

int gs_mfdreceivers(gs_plan* plan, int32_t nrcv, double exp, const double* elev, double sl,
                    const int32_t* gid, int32_t* rcv, double* dist, double* wgt) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(elev);
        NEED(rcv);
        NEED(dist);
        NEED(wgt);
    }
    GS_GUARD(return gs::receivers(plan, nrcv, exp, elev, sl, gid, rcv, dist, wgt, nullptr);)
}

int gs_fill_elevation(gs_plan* plan, const double* h, double sealevel, double ofill, int32_t sed, double* lfill,
                      int32_t* pit_ids, int32_t* flat_dirs, int32_t* npits) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(h);
        NEED(lfill);
        NEED(pit_ids);
        NEED(flat_dirs);
    }
    GS_GUARD({
        gs_stats st{};
        int s = gs::fill_elevation(plan, h, sealevel, ofill, lfill, pit_ids, flat_dirs, &st, false, nullptr,
                                   sed != 0);
        if (npits) *npits = plan->npits;
        return s;
    })
}

int gs_build_flow_direction(gs_plan* plan, const double* h, int32_t down, double sealevel, const double* lfill,
                            const int32_t* pit_ids, const int32_t* flat_dirs, int32_t* rcv, double* dist,
                            double* wgt, uint8_t* lsink, uint8_t* sea) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(h); NEED(lfill); NEED(pit_ids); NEED(flat_dirs); NEED(rcv); NEED(dist); NEED(wgt); NEED(lsink);
        NEED(sea);
    }
    // the plan's live-graph slot table is scratch here: every stage that
    // reads it rebuilds it together with its own receivers first
    GS_GUARD(return gs::flow_direction(plan, h, down != 0, lfill, pit_ids, flat_dirs, sealevel, rcv, dist, wgt,
                                       plan->rslot, lsink, sea);)
}

int gs_pit_tables(gs_plan* plan, double* pit_params, int32_t* pit_info, double* filled_lvl,
                  double* filled_vol) {
    NEED(plan);
    const size_t np1 = (size_t)plan->npits + 1;
    if (pit_params)
        GS_CUDA(cudaMemcpyAsync(pit_params, plan->pit_params, sizeof(double) * 3 * np1, cudaMemcpyDeviceToDevice,
                                plan->stream));
    if (pit_info)
        GS_CUDA(cudaMemcpyAsync(pit_info, plan->pit_info, sizeof(int) * 2 * np1, cudaMemcpyDeviceToDevice,
                                plan->stream));
    if (filled_lvl)
        GS_CUDA(cudaMemcpyAsync(filled_lvl, plan->filled_lvl, sizeof(double) * 5 * np1,
                                cudaMemcpyDeviceToDevice, plan->stream));
    if (filled_vol)
        GS_CUDA(cudaMemcpyAsync(filled_vol, plan->filled_vol, sizeof(double) * 5 * np1,
                                cudaMemcpyDeviceToDevice, plan->stream));
    return GS_OK;
}

int gs_flow_accumulation(gs_plan* plan, const double* h, const double* bl, double sealevel, double ofill,
                         double dt, double* fal, double* fill_fal, double* water_filled, double* lfill,
                         int32_t* pit_ids, int32_t* flat_dirs, int32_t* rcv_i, double* dist_i, double* wgt_i,
                         uint8_t* lsink, uint8_t* sea, gs_stats* stats) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(h); NEED(bl); NEED(fal); NEED(fill_fal); NEED(water_filled); NEED(lfill); NEED(pit_ids);
        NEED(flat_dirs); NEED(rcv_i); NEED(dist_i); NEED(wgt_i); NEED(lsink); NEED(sea);
    }
    if (!(dt > 0)) {
        gs::set_error(GS_EINVAL, "dt must be positive");
        return GS_EINVAL;
    }
    GS_GUARD({
        gs_stats st{};
        int s = gs::flow_accumulation(plan, h, bl, sealevel, ofill, dt, fal, fill_fal, water_filled, lfill,
                                      pit_ids, flat_dirs, rcv_i, dist_i, wgt_i, lsink, sea, &st);
        st.status = s;
        if (stats) *stats = st;
        return s;
    })
}

int gs_erodep_spl(gs_plan* plan, double* h, double* cum_ed, double* eb, const double* fal, const double* rain,
                  double k_scalar, const double* k_field, double d, double m, double dt, const int32_t* rcv_i,
                  const double* dist_i, const double* wgt_i, const uint8_t* lsink, const uint8_t* sea,
                  gs_stats* stats) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(h); NEED(cum_ed); NEED(eb); NEED(fal); NEED(rain); NEED(rcv_i); NEED(dist_i); NEED(wgt_i);
        NEED(lsink); NEED(sea);
    }
    if (!(dt > 0)) {
        gs::set_error(GS_EINVAL, "dt must be positive");
        return GS_EINVAL;
    }
    GS_GUARD(return gs::erodep_spl(plan, h, cum_ed, eb, fal, rain, k_scalar, k_field, d, m, dt, rcv_i, dist_i,
                                   wgt_i, lsink, sea, stats);)
}

int gs_plan_set_lake_diffusion(gs_plan* plan, double k, double inlet_bias, int32_t nsub, int32_t npic) {
    NEED(plan);
    if (!(k >= 0.0) || !(inlet_bias >= 0.0 && inlet_bias <= 1.0) || nsub < 0 || npic < 1) {
        gs::set_error(GS_EINVAL, "lake diffusion: need K >= 0, 0 <= inlet_bias <= 1, nsub >= 0, npic >= 1");
        return GS_EINVAL;
    }
    plan->lake_on = nsub > 0 ? 1 : 0;
    plan->lake_K = k;
    plan->lake_bias = inlet_bias;
    plan->lake_nsub = nsub;
    plan->lake_npic = npic;
    return GS_OK;
}

int gs_sed_change(gs_plan* plan, double* h, double* cum_ed, const double* eb, const double* xyz, double sealevel,
                  double ofill, double dt, double nl_pit_volume, double nl_pit_depth, double* lfill,
                  int32_t* pit_ids, int32_t* flat_dirs, const int32_t* rcv_i, const double* wgt_i, uint8_t* lsink,
                  uint8_t* sea, double* vsed, gs_stats* stats) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(h); NEED(cum_ed); NEED(eb); NEED(xyz); NEED(lfill); NEED(pit_ids); NEED(flat_dirs); NEED(rcv_i);
        NEED(wgt_i); NEED(lsink); NEED(sea); NEED(vsed);
    }
    if (!(dt > 0)) {
        gs::set_error(GS_EINVAL, "dt must be positive");
        return GS_EINVAL;
    }
    GS_GUARD(return gs::sed_change(plan, h, cum_ed, eb, xyz, sealevel, ofill, dt, nl_pit_volume, nl_pit_depth,
                                   lfill, pit_ids, flat_dirs, rcv_i, wgt_i, lsink, sea, vsed, stats);)
}

int gs_sea_change(gs_plan* plan, double* h, double* cum_ed, double* eb, const double* xyz, const double* box,
                  const int32_t* edges, int64_t nedge, double sealevel, double ofill, double dt, double clinslp,
                  double offshore, double nlk, double gmar, const double* lfill, const double* vsed,
                  const uint8_t* sea, gs_stats* stats) {
    NEED(plan);
    NEED(box);
    if (plan->n > 0) {
        NEED(h); NEED(cum_ed); NEED(eb); NEED(xyz); NEED(lfill); NEED(vsed); NEED(sea);
        if (nedge > 0) NEED(edges);
    }
    if (!(dt > 0) || nedge < 0 || !(clinslp >= 0) || !(offshore > 0) || !(nlk >= 0) || !(gmar >= 0)) {
        gs::set_error(GS_EINVAL,
                      "seaChange: need dt > 0, nedge >= 0, clinslp >= 0, offshore > 0, nlk >= 0, gmar >= 0");
        return GS_EINVAL;
    }
    GS_GUARD(return gs::sea_change(plan, h, cum_ed, eb, xyz, box, edges, nedge, sealevel, ofill, dt, clinslp, offshore,
                                   nlk, gmar, lfill, vsed, sea, stats);)
}

int gs_sed_budget(gs_plan* plan, double* out16) {
    NEED(plan);
    NEED(out16);
    for (int k = 0; k < 16; k++) out16[k] = 0.0;
    if (!plan->led) return GS_OK;
    GS_GUARD(return gs::sed_budget(plan, out16);)
}

int gs_hillslope(gs_plan* plan, double* h, double* cum_ed, double* eb, double sealevel, double cda, double cdm,
                 double dt, double rtol, int32_t max_iter, gs_stats* stats) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(h); NEED(cum_ed); NEED(eb);
    }
    if (!(dt > 0) || !(rtol > 0) || max_iter < 1) {
        gs::set_error(GS_EINVAL, "dt, rtol must be positive and max_iter >= 1");
        return GS_EINVAL;
    }
    GS_GUARD(return gs::hillslope(plan, h, cum_ed, eb, sealevel, cda, cdm, dt, rtol, max_iter, stats);)
}

int gs_apply_forces(gs_plan* plan, double* h, const double* rain, const double* upsub, double dt,
                    double sealevel, double* bl) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(h); NEED(rain); NEED(bl);
    }
    GS_GUARD(return gs::apply_forces(plan, h, rain, upsub, dt, sealevel, bl);)
}

int gs_output_fields(gs_plan* plan, const double* h, const double* cum_ed, const double* eb,
                     const double* water_filled, const double* fill_fa, const double* fa, const double* vsed,
                     const double* upsub, const double* rain, const uint8_t* sea, float* out) {
    NEED(plan);
    if (plan->n > 0) {
        NEED(h); NEED(cum_ed); NEED(eb); NEED(water_filled); NEED(fill_fa); NEED(fa); NEED(vsed); NEED(out);
    }
    GS_GUARD(return gs::output_fields(plan, h, cum_ed, eb, water_filled, fill_fa, fa, vsed, upsub, rain, sea, out);)
}

}  // extern "C"
