/*
 * gospl_b200 — C ABI of the B200 (sm_100a) implementation of goSPL's
 * per-timestep surface-process path.
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer (CUDA global memory) owned by the
 *    caller unless stated otherwise; the library never frees caller memory.
 *  - Per-vertex arrays have length nb; per-receiver arrays are receiver-major
 *    ("[nrcv][nb]": element (k, i) at k*nb + i).
 *  - Node ids are 0-based int32, as the reference's f2py module stores them.
 *  - Work is issued on the plan's stream (gs_plan_set_stream, default stream
 *    0).  Functions that must inspect device results (pit counts, cascade
 *    control flow, CG convergence) synchronise that stream before returning.
 *  - Every function returns GS_OK (0) or an error code; gs_last_error() gives
 *    the message of the last failure on the calling host thread.
 *  - A plan is not thread-safe: use one plan per host thread.
 */
#ifndef GOSPL_B200_H
#define GOSPL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_OK 0
#define GS_EINVAL 1      /* bad argument (size, range, null pointer)              */
#define GS_ECUDA 2       /* CUDA runtime error                                    */
#define GS_EMAXITER 3    /* iteration cap reached without convergence             */
#define GS_ENONFINITE 4  /* NaN/Inf met in an input or a reduction                */
#define GS_ECYCLE 5      /* a flow graph that should be acyclic has a cycle       */
#define GS_ETIMEOUT 6    /* a device-side wait exceeded its time budget           */
#define GS_ENOMEM 7      /* device allocation failed                              */

typedef struct gs_plan gs_plan;

/* Counters filled by the flow/erosion entry points (host memory). */
typedef struct gs_stats {
    int32_t npits;            /* depressions found by the fill (P; ids 1..P)          */
    int32_t cascade_passes;   /* _distributeDownstream passes executed                */
    int32_t cascade_solves;   /* cascade flow solves executed                         */
    int32_t fill_rounds;      /* spill-graph relaxation rounds                        */
    int32_t flat_rounds;      /* flat-distance BFS levels                             */
    int32_t cycle_nodes;      /* nodes solved by the cycle fallback (0 when acyclic)  */
    int32_t cg_iters;         /* hillslope CG iterations                              */
    int32_t status;           /* last internal status                                 */
    double cg_relres;         /* final relative residual of the hillslope solve      */
} gs_stats;

int gs_version(void);
int gs_last_error(char* buf, int64_t len);

/*
 * Mesh plan.  The finite-volume arrays are exactly what the reference's
 * `definetin` (fortran/functions.F90:2715-2940) leaves in module `meshparams`:
 * nnb = FVnNb, ngb = FVnID (C-order [nb][12], -1 padded), elgt = FVeLgt,
 * vdist = FVvDist, farea = FVarea; larea is the Python-side cell area
 * (unstructuredmesh.py:165-188).  HOST pointers (copied).  outlet_ids are the
 * draining boundary nodes (`outletIDs`, unstructuredmesh.py:463-518) and
 * open_ids the 'o' edge nodes reset by _drainOpenEdges.
 */
int gs_plan_create(int64_t nb, const int32_t* nnb, const int32_t* ngb, const double* elgt,
                   const double* vdist, const double* farea, const double* larea,
                   const int32_t* outlet_ids, int64_t n_outlet, const int32_t* open_ids,
                   int64_t n_open, int32_t flat_model, int32_t flow_dir, gs_plan** out);
int gs_plan_destroy(gs_plan* plan);
/*
 * Landscape members.  No counterpart in the reference (goSPL runs one
 * landscape per model).  A plan built over the disjoint union of several
 * meshes (member m = vertices [start[m], start[m+1]), no edge between
 * members) advances them all with one launch per stage while each member
 * keeps its own control flow: the lake-cascade loop of
 * FAMesh.flowAccumulation (flowplex.py:850-904: excess, pass limit,
 * stagnation, `resid > maxarea` with the member's own largest cell area
 * maxarea[m]), its own lake zeroing and fillFAL maximum.  HOST arrays,
 * start[0] = 0, start[nmem] = nb.  A new plan has one member.
 */
int gs_plan_set_members(gs_plan* plan, int32_t nmem, const int64_t* start, const double* maxarea);
int gs_plan_set_stream(gs_plan* plan, void* cuda_stream);
/*
 * Launch-shape knobs (no counterpart in the reference).  GS_TUNE_SWEEP_BLOCKS:
 * 128-thread blocks per SM of the ordered dependency sweeps (1..32, default
 * 8).  GS_TUNE_COOP_BLOCKS: 256-thread blocks per SM of the cooperative
 * kernels (basin relaxation, grid BFS, hillslope CG; 1..their co-residency
 * limit, default min(limit, 4)); gs_plan_tuning(plan, GS_TUNE_COOP_BLOCKS + 1)
 * returns that limit.  Results do not depend on the knobs beyond the
 * rounding of the hillslope CG's inner products (block partial sums); speed
 * does (gospl_b200.autotune picks them by timing steps).
 */
#define GS_TUNE_SWEEP_BLOCKS 1
#define GS_TUNE_COOP_BLOCKS 2
#define GS_TUNE_REFINE_PASSES 4   /* gs_plan_tuning only: refinement passes so far */
#define GS_TUNE_SWEEP_NAP 5       /* longest back-off between polls of the ordered sweeps, ns (0..1024, default 32) */
#define GS_TUNE_SWEEP_BUDGET 6    /* wall-clock budget of one dependency sweep, us (1..6e7, default 4e6): a sweep
                                     still waiting on a predecessor after it stops with GS_ETIMEOUT */
#define GS_TUNE_FLAT_BFS 7        /* flat-distance BFS: 0 one block with the visited set in shared memory
                                     (default; tiles when the set does not fit), w in 1..4096 tiles in one
                                     cooperative launch settling distance windows of w levels */
#define GS_TUNE_WARM_START 8      /* 1 (default): the hillslope CG starts from h plus the previous step's
                                     diffusion change and the bathymetry smoothing from the previous
                                     smoothing; 0: both start from their right-hand side, so that a step
                                     depends only on its inputs (the adjoint's runs and their finite-
                                     difference checks).  Setting it forgets the stored starts. */
int gs_plan_tune(gs_plan* plan, int32_t knob, int32_t value);
/*
 * Precision form (no counterpart in the reference, which is FP64 only).
 * bits = 32: the flow-accumulation and SPL sweeps and the hillslope CG run in
 * FP32 inside FP64 iterative refinement (FP64 residuals, corrections solved in
 * FP32) until max|r| <= tol max|b| (sweeps) or |r|_2 <= max(rtol, tol) |b|_2
 * (CG); receivers, pit filling, the cascade and every mass sum stay FP64.
 * bits = 64 (default): the plain FP64 path.
 */
int gs_plan_set_precision(gs_plan* plan, int32_t bits, double tol);
int gs_plan_tuning(const gs_plan* plan, int32_t knob);
/* Number of device kernels this plan launched since creation. */
int64_t gs_plan_launches(const gs_plan* plan);
/* Per-kernel timing: when enabled, every launch of the plan is bracketed by
 * CUDA events on the plan's stream (clears previous records). */
int gs_plan_profile(gs_plan* plan, int32_t enable);
/* Writes "kernel_name launches total_ms" lines for the recorded launches into
 * buf (synchronises the plan's stream); returns the report length. */
int gs_plan_profile_report(gs_plan* plan, char* buf, int64_t len);
/* Writes one "kernel_name stream start_ms end_ms" line per recorded launch
 * (stream 0 = the plan's stream, 1 and 2 = its two internal side streams;
 * times from the first recorded launch; synchronises the device). */
int gs_plan_profile_trace(gs_plan* plan, char* buf, int64_t len);

/*
 * Finite-volume geometry of a triangulated mesh (init-time), replacing the
 * Fortran `definetin` (fortran/functions.F90:2715-2940) called from
 * unstructuredmesh.py:164-170.  Inputs (DEVICE): xyz [n][3]; edges [m][2] in
 * the reference's edge order (meshfunc.py:295-327); vptr/vedge: CSR of each
 * vertex's edges in edge order; cells_edges [ncell][3]; cc [ncell][3]
 * circumcentres (projected on the sphere when curved); cptr/vcell: CSR of
 * each vertex's cells in cell order.  Outputs (DEVICE): nnb [n], ngb
 * [n][12] (-1 padded), elgt/vdist [n][12], farea [n] (NaN -> 0) and narea
 * [n] (raw).  `stream` is a cudaStream_t (NULL = default stream).
 */
int gs_mesh_geometry(int64_t n, const double* xyz, int64_t m, const int32_t* edges,
                     const int32_t* vptr, const int32_t* vedge, int64_t ncell,
                     const int32_t* cells_edges, const double* cc, const int32_t* cptr,
                     const int32_t* vcell, int32_t curved, int32_t* nnb, int32_t* ngb,
                     double* elgt, double* vdist, double* farea, double* narea, void* stream);

/*
 * Multiple-flow-direction receivers.  Replaces `mfdreceivers(nRcv, exp, elev,
 * sl, gid)` (fortran/functions.F90:1544-1671, bound in gospl/_fortran through
 * fortran/functions.pyf) called from flowplex.py:499-501.  Outputs receiver-
 * major [nrcv][nb]: rcv (self id = no receiver), dist, wgt.
 */
int gs_mfdreceivers(gs_plan* plan, int32_t nrcv, double exp, const double* elev, double sl,
                    const int32_t* gid, int32_t* rcv, double* dist, double* wgt);

/*
 * Depression filling.  Replaces PITFill.fillElevation(sed)
 * (gospl/flow/pitfilling.py:849-903) and the Fortran kernels it drives
 * (edge_tile, fill_tile, fill_edges, fill_depressions, label_pits, pits_cons,
 * fill_dir, nghb_dir, getpitvol: functions.F90:1845-2499).  sed != 0 is the
 * sediment fill (pitfilling.py:690-692, 718-721, 828-834, 885-887): marine
 * depressions filled too, pits labelled above the fill level, pit volumes on
 * the unclipped surface.  Outputs per vertex: lFill, pitIDs (-1 or 1..P),
 * flatDirs (-1, self or a neighbour).  The per-pit tables (pitParams,
 * pitInfo, filled_lvl, filled_vol) stay in the plan; read them with
 * gs_pit_tables.  *npits receives P.
 */
int gs_fill_elevation(gs_plan* plan, const double* h, double sealevel, double ofill, int32_t sed,
                      double* lfill, int32_t* pit_ids, int32_t* flat_dirs, int32_t* npits);

/*
 * Flow direction of a surface.  Replaces FAMesh._buildFlowDirection(h, down)
 * (gospl/flow/flowplex.py:480-544; the matrix of matrixFlow, 429-478, is the
 * receiver table itself): mfdreceivers on h, then with down != 0 the
 * pit-flat routing (cells with h == lFill in a depression, a flat receiver
 * and no MFD receiver send all their flow to flatDirs), flat-model outlets
 * made self-sinks, lsink = no receiver weight, not an outlet, not sea, and
 * sea = lFill <= sealevel (seaID).  Reads lfill, pit_ids, flat_dirs of the
 * last fill.  Outputs receiver-major rcv/dist/wgt [R][nb], lsink and sea
 * (uint8 masks [nb]).  All pointers DEVICE.
 */
int gs_build_flow_direction(gs_plan* plan, const double* h, int32_t down, double sealevel,
                            const double* lfill, const int32_t* pit_ids, const int32_t* flat_dirs,
                            int32_t* rcv, double* dist, double* wgt, uint8_t* lsink, uint8_t* sea);
/* Copy the pit tables of the last fill into caller DEVICE buffers sized
 * (P+1) rows: pit_params [P+1][3], pit_info [P+1][2], filled_lvl [P+1][5],
 * filled_vol [P+1][5] (rows as in pitfilling.py:521-555, 810-891). */
int gs_pit_tables(gs_plan* plan, double* pit_params, int32_t* pit_info, double* filled_lvl,
                  double* filled_vol);

/*
 * Flow accumulation.  Replaces FAMesh.flowAccumulation (flowplex.py:752-945)
 * with its fill, _buildFlowDirection(down=False), the (I - W^T) FA solve, the
 * downstream lake cascade (_distributeDownstream, flowplex.py:576-686) and the
 * lake zeroing / fillFAL proxy.  bl = rain * larea (m^3/yr).
 * Outputs: fal, fill_fal, water_filled (= waterFilled - h), lfill, pit_ids,
 * flat_dirs, the snapshots rcv_i/dist_i/wgt_i ([nrcv][nb], the reference's
 * rcvIDi/distRcvi/wghtVali), lsink (uint8, the LIVE lsink after the cascade,
 * as SPL.py:352 reads it) and sea (uint8, lFill <= sealevel).
 */
int gs_flow_accumulation(gs_plan* plan, const double* h, const double* bl, double sealevel,
                         double ofill, double dt, double* fal, double* fill_fal,
                         double* water_filled, double* lfill, int32_t* pit_ids,
                         int32_t* flat_dirs, int32_t* rcv_i, double* dist_i, double* wgt_i,
                         uint8_t* lsink, uint8_t* sea, gs_stats* stats);

/*
 * Implicit linear stream-power erosion (n = 1, G = 0).  Replaces
 * SPL.erodepSPL / _getEroDepRate / _eroMats (gospl/eroder/SPL.py:45-114,
 * 260-366, 402-454).  Kbr = K * rain^d * dt * FAL^m (K a scalar when k_field
 * is NULL, else a per-vertex field); the implicit system is solved exactly by
 * a sweep over the receiver graph.  Updates h and cum_ed in place and writes
 * eb = dz/dt.  Uses the receivers/lsink/sea produced by gs_flow_accumulation.
 */
/*
 * Transport-limited SPL: the deposition coefficient G of goSPL's `spl: G`
 * (inputparser.py:472; default 0).  With G > 0 gs_erodep_spl solves the
 * coupled erosion-deposition system of _getEroDepRate / _coupledEDSystem
 * (SPL.py:116-258, 305-336) instead of the detachment-limited one; its
 * stats then report the solver's operator applications (cg_iters; each is
 * one flow sweep and one SPL sweep) and final relative residual (cg_relres).
 */
int gs_plan_set_deposition(gs_plan* plan, double g);
int gs_erodep_spl(gs_plan* plan, double* h, double* cum_ed, double* eb, const double* fal,
                  const double* rain, double k_scalar, const double* k_field, double d,
                  double m, double dt, const int32_t* rcv_i, const double* dist_i,
                  const double* wgt_i, const uint8_t* lsink, const uint8_t* sea,
                  gs_stats* stats);

/*
 * Linear hillslope diffusion.  Replaces hillSLP.getHillslope with
 * _hillSlope(smooth=0) (gospl/sed/hillslope.py:90-233, 614-649) and the
 * Fortran sethillslopecoeff (functions.F90:901-938): solves (I + L) h = hOld
 * with Jacobi-preconditioned CG to relative residual `rtol`.  Updates h and
 * cum_ed in place and adds dz/dt to eb.
 */
/*
 * Continental sediment routing and deposition in depressions:
 * SEDMesh.sedChange (gospl/sed/sedplex.py:1061-1086) with _getSedFlux
 * (103-188), fillElevation(sed=True) (flow/pitfilling.py:849-903),
 * _distributeSediment / _moveDownstream (190-522) and _updateSinks (982-1059)
 * for one landscape, one lithology, no provenance.  Call it right after
 * gs_flow_accumulation on the same h (goSPL's runProcesses with nodep=False
 * runs flowAccumulation, then sedChange): rcv_i / wgt_i are that call's
 * snapshot receivers and sea its sea mask.  xyz holds the vertex coordinates
 * [nb][3] (the micro-tilt of lake deposits).  Updates h and cum_ed, writes
 * vsed (routed sediment flux, m3/yr), the sediment fill (lfill, pit_ids,
 * flat_dirs and the plan's pit tables, with pitParams volumes left to the
 * unfilled remainder) and lsink.  Partly filled depressions of at least
 * nl_pit_volume (m3) and nl_pit_depth (m), whose deposit goSPL smooths by
 * non-linear diffusion, take gs_plan_set_lake_diffusion's path, or return
 * GS_EINVAL when it is off (stats.status = their count).
 * Ensemble members (gs_plan_set_members) each run their own cascade, with
 * closed-domain deposits for members without an outlet.  stats: npits,
 * cascade passes and solves.  `sea` is goSPL's live seaID: read for the
 * sinks of the snapshot graph, and overwritten (lFill <= sealevel of the
 * sediment fill) when the cascade rebuilds the flow graph, as
 * _buildFlowDirection does (flowplex.py:494).
 */
/*
 * Lake deposits of large deep depressions (gs_sed_change path 3): goSPL's
 * _diffuseLargePit (sedplex.py:679-858) with the lagged-diffusivity solver of
 * marineSolver picard (_diffuseImplicitPicard, hillslope.py:988-1076): an
 * inlet pile (share inlet_bias, pitInletBias) over a bathymetric baseline,
 * nsub backward-Euler sub-steps (picardSub) of npic Picard updates each
 * (picardIts) with diffusivity 1e-4 + k (1 - exp(-0.05 dh)) (nlPitK), then a
 * per-pit rescale to the deposited volume.  nsub = 0 switches it off (the
 * default: goSPL's default adaptive TS solver is not built, and those
 * depressions make gs_sed_change return GS_EINVAL).
 */
int gs_plan_set_lake_diffusion(gs_plan* plan, double k, double inlet_bias, int32_t nsub, int32_t npic);
int gs_sed_change(gs_plan* plan, double* h, double* cum_ed, const double* eb, const double* xyz,
                  double sealevel, double ofill, double dt, double nl_pit_volume, double nl_pit_depth,
                  double* lfill, int32_t* pit_ids, int32_t* flat_dirs, const int32_t* rcv_i,
                  const double* wgt_i, uint8_t* lsink, uint8_t* sea, double* vsed,
                  gs_stats* stats);

/*
 * Sediment budget of the last gs_sed_change (m^3 over the step), summed on
 * the device in a fixed order.  No single counterpart in the reference: it
 * accounts, pass by pass, for where the volume eroded by the step's SPL goes
 * in goSPL's continental routing (sedplex.py:103-522), including the volume
 * that goSPL's own rules drop.  Every flow solve of the routing delivers its
 * input to terminal cells (all weights 0), which are split into depression
 * sinks, stray sinks kept on closed domains (sedplex.py:230-245), stray sinks
 * dropped on domains with an outlet, open outlets and the sea; every pass
 * splits the depressions' inflow into the retained volume, the excess (eV >
 * 0) and inflow equal to the remaining volume (eV == 0, which goSPL drops);
 * the excess is placed at spill nodes (one pit wins a shared spill node, a
 * depression without a spill node places nothing) and routed when it exceeds
 * half the largest cell area (sedplex.py:343-350).
 *   eroded = retained + kept + dropped + outlets + sea + zero_excess
 *            + (excess - placed) + (placed - routed)
 * closes to rounding.  `realised` is the volume the step's deposits add to
 * the surface, sum(larea * dh); it differs from retained + kept by goSPL's
 * bottom-up lake level (np.interp over the depth-volume table) and tilt.
 * out[16] receives the GS_LED_* slots.
 */
#define GS_LED_ERODED 0      /* sum(-Eb * larea) * dt                              */
#define GS_LED_PIT_SINKS 1   /* volume reaching depression sinks (all passes)      */
#define GS_LED_KEPT 2        /* stray sinks, domain without outlet: deposited      */
#define GS_LED_DROPPED 3     /* stray sinks, domain with an outlet: leaves         */
#define GS_LED_OUTLETS 4     /* reaching open outlets: leaves the domain           */
#define GS_LED_SEA 5         /* reaching other terminal cells (sea): leaves        */
#define GS_LED_RETAINED 6    /* kept by depressions                                */
#define GS_LED_EXCESS 7      /* overflow of depressions (eV > 0)                   */
#define GS_LED_ZERO 8        /* inflow of depressions with eV == 0                 */
#define GS_LED_INFLOW 9      /* total inflow of depressions (all passes)           */
#define GS_LED_PLACED 10     /* excess written at spill nodes                      */
#define GS_LED_ROUTED 11     /* placed excess that was routed downstream           */
#define GS_LED_REALISED 12   /* sum(larea * (h_after - h_before)) of sedChange     */
#define GS_LED_KEPT_DEP 13   /* sum of the closed-domain deposit volumes           */
int gs_sed_budget(gs_plan* plan, double* out16);

/*
 * Marine deposition.  Replaces SEAMesh.seaChange (gospl/sed/seaplex.py:738-861)
 * for one lithology, no stratigraphy or provenance, and marineSolver
 * picard (the plan's lake-diffusion settings, gs_plan_set_lake_diffusion,
 * give picardSub and picardIts; nlk is nonlinKm): distance of the sea
 * vertices to the sea-level contour of h (_distanceCoasts, 51-135),
 * clinoform capacity from clinslp, the sediment reaching the sea (vsed * dt
 * where the sediment fill lfill <= sealevel), marine receivers on the
 * epsilon-filled routing surface (_matOcean, 137-238: bathymetry smoothed by
 * one implicit diffusion step on spheres, cells farther than `offshore` or
 * planar outlets at the boundary sentinel; epsfill and mfdrcvrs,
 * functions.F90:2633-2697 and 1673-1785), the capacity-limited cascade
 * (_distOcean, 404-619) and the Picard diffusion of the deposit over the sea
 * cells (_diffuseOcean, hillslope.py:739-787); h, cum_ed and eb are updated.
 * `sea` is goSPL's seaID at this point (lFill <= sealevel of the last flow
 * direction built), `edges` the mesh's unique edges [nedge][2] (DEVICE),
 * `box` (HOST, 6 doubles) the vertices' bounding box as (lo, span).  stats:
 * npits = coastline points, cascade_passes = marine passes (of the last
 * cascade), fill_rounds = epsfill relaxation passes, flat_rounds = CG
 * iterations of the bathymetry smoothing, cg_iters = GMRES operator
 * applications of the coupled system.  gmar > 0 on a spherical mesh
 * (_depMarineSystem, seaplex.py:240-402): the deposit of the first cascade
 * feeds the coupled marine elevation / flux system [[I - G, -G dt/A],
 * [A/dt, (I - W)^T]] [h; q] = [(1 - G) h; dep/dt + h A/dt] with
 * G = min(gmar, 0.99) below sea level, W the marine receivers; its deposit
 * (negatives dropped) goes down the cascade again.  The system is reduced to
 * the elevation and solved by GMRES(30) to 1e-13, each application one
 * ordered marine flow sweep.
 */
int gs_sea_change(gs_plan* plan, double* h, double* cum_ed, double* eb, const double* xyz, const double* box,
                  const int32_t* edges, int64_t nedge, double sealevel, double ofill, double dt, double clinslp,
                  double offshore, double nlk, double gmar, const double* lfill, const double* vsed,
                  const uint8_t* sea, gs_stats* stats);

int gs_hillslope(gs_plan* plan, double* h, double* cum_ed, double* eb, double sealevel,
                 double cda, double cdm, double dt, double rtol, int32_t max_iter,
                 gs_stats* stats);

/*
 * Forcing of one step: UnstMesh.applyForces (unstructuredmesh.py:743-794) with
 * _updateRain (bl = max(rain,0) * larea), applyTectonics (h += upsub * dt) and
 * _drainOpenEdges (796-901).  upsub may be NULL.
 */
int gs_apply_forces(gs_plan* plan, double* h, const double* rain, const double* upsub, double dt,
                    double sealevel, double* bl);

/*
 * Output fields of one step for the HDF5 writer: WriteMesh._outputMesh
 * (outmesh.py:252-478).  out is a device float32 array [9][n] whose rows are
 * elev (h), erodep (cum_ed), EDrate (eb), waterFill, fillFA, FA, sedLoad
 * (vsed), uplift (upsub) and rain, each rounded to nearest from float64; FA,
 * fillFA and sedLoad are raised to DISCHARGE_FLOOR = 1e-8 (tools/constants.py:51)
 * where at or below it, and FA and fillFA are 1 on sea vertices.  sea is the
 * land/sea mask (1 = sea) or NULL for the mask of the elevation the last
 * gs_hillslope call started from (hillslope.py:620; GS_EINVAL if there is none).
 * upsub and rain may be NULL (their rows are left as they are).
 */
int gs_output_fields(gs_plan* plan, const double* h, const double* cum_ed, const double* eb,
                     const double* water_filled, const double* fill_fa, const double* fa, const double* vsed,
                     const double* upsub, const double* rain, const uint8_t* sea, float* out);

/*
 * Adjoint.  No counterpart in the reference (goSPL has no derivatives).
 * gs_plan_record allocates nslots per-step records (0 frees them; single-
 * landscape plans only); after gs_plan_record_slot(plan, s) the forward calls
 * of one step (gs_flow_accumulation, gs_erodep_spl, gs_hillslope) store what
 * the adjoint needs in slot s (-1 stops recording).  gs_adjoint_step reverses
 * the recorded step with its discrete decisions held fixed (receiver choice,
 * pits, flat routing, cascade states, masks): on entry lam = dJ/dh after the
 * step's uplift (h_{t+1}), on return lam = dJ/dh_t; it accumulates dJ/dK
 * (grad_k, per vertex), dJ/dU (grad_u, the uplift rate) and the direct SPL
 * part of dJ/drain (grad_rain, rain^d), and writes dJ/dbL_t (grad_bl: the
 * step's rain volume rain * larea); any output may be NULL.  The level of a
 * partially filled lake is held constant.  Synchronises the plan's stream.
 */
int gs_plan_record(gs_plan* plan, int32_t nslots);
int gs_plan_record_slot(gs_plan* plan, int32_t slot);
int gs_adjoint_step(gs_plan* plan, int32_t slot, double* lam, const double* rain, double k_scalar,
                    const double* k_field, double d, double m, double dt, double sealevel, double cda, double cdm,
                    double rtol, int32_t max_iter, double* grad_k, double* grad_u, double* grad_rain,
                    double* grad_bl);

/*
 * Allocation-free flow solve.  No counterpart in the reference: goSPL always
 * allocates its PETSc matrices and vectors.  For callers that cannot call
 * cudaMalloc (an embedding application that owns every allocation, or one
 * that runs under a fixed device-memory budget), this solves (I - W^T) q = b for the
 * receiver graph rcv/wgt ([nrcv][nb], as gs_mfdreceivers writes them) with
 * all scratch in a fixed file-scope device array, so it allocates nothing.
 * The caller passes inputs and the output q.  Limits: nb <= GS_NOALLOC_MAX_NB,
 * nrcv <= GS_NOALLOC_MAX_RCV, else GS_EINVAL.  Every GPU that loads the
 * library holds the array (about 40 MB) until the process exits.  All calls
 * share it: calls that overlap on the GPU race and must be serialised by the
 * caller.  The first call on each device resolves the array's address (make
 * it before any stream capture).  `stream` must belong to the current device
 * (else GS_EINVAL).  Synchronises `stream` before returning, to read the
 * solve's status (GS_ECYCLE for a receiver graph with a cycle).
 */
#define GS_NOALLOC_MAX_NB 1048576
#define GS_NOALLOC_MAX_RCV 4
int gs_flow_solve_noalloc(int64_t nb, int32_t nrcv, const int32_t* rcv, const double* wgt,
                          const double* b, double* q, void* stream);

#ifdef __cplusplus
}
#endif
#endif
