/*
 * bugdef.h -- C ABI of libbugdef.so, the sm_100a implementation of the coupled
 * laser-tissue epoch of yudovsky/bug-defense (voxel Monte Carlo photon transport,
 * explicit bioheat stencil, enthalpy boiling / char / ablation update, smoke plume).
 *
 * Conventions
 *   - Every entry point returns an int status (BD_OK == 0) and never aborts the
 *     process; bd_last_error() gives the message of the last failure on the
 *     calling thread.
 *   - Grids are C-order (nx, ny, nz) with z fastest: idx = (i*ny + j)*nz + k,
 *     the layout of the reference's numpy arrays (simulation/voxel_mc_metal.py:209-211,
 *     simulation/metal_ablation_solver.py:94-96).
 *   - Array arguments are DEVICE pointers unless a name ends in _host.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Calls only enqueue work; nothing synchronises unless documented.
 *   - Units follow the reference: mm, s, W, J, degC; k in W/(mm K), rho_cp in
 *     J/(mm^3 K), Q in W/mm^3, h_lat in J/mm^3, h_eff in W/(mm^2 K).
 */
#ifndef BUGDEF_H
#define BUGDEF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BD_ABI_VERSION 1

#if defined(__GNUC__)
#define BD_API __attribute__((visibility("default")))
#else
#define BD_API
#endif

/* ---- status codes ---------------------------------------------------------- */
#define BD_OK                 0
#define BD_ERR_INVALID_ARG    1  /* bad size, null pointer, unsupported combination (ValueError) */
#define BD_ERR_CUDA           2  /* a CUDA runtime call failed (RuntimeError)                      */
#define BD_ERR_OUT_OF_MEMORY  3
#define BD_ERR_TIMEOUT        4  /* a bounded device loop gave up                                   */
#define BD_ERR_NO_DEVICE      5  /* no CUDA device (RuntimeError, like engine='gpu' without Metal) */
#define BD_ERR_STATE          6  /* handle used in a wrong state                                    */

/* ---- per-voxel flag byte (one uint8 per voxel) ------------------------------ */
#define BD_FLAG_ABLATED  0x01u  /* voxel is void (reference `ablated`)                        */
#define BD_FLAG_DRY      0x02u  /* dehydrated voxel (reference `dry`)                         */
#define BD_FLAG_VOID     0x04u  /* plume domain (reference `plume_void` / compute_void_mask)  */
#define BD_FLAG_NEWLY    0x08u  /* removed at the last epoch end (plume injection source)     */

/* ---- Monte Carlo energy ledger (FP64, one entry per photon-weight channel) --- */
#define BD_LEDGER_LAUNCHED        0   /* photons launched (weight 1 each)                    */
#define BD_LEDGER_SPECULAR        1   /* entrance Fresnel split                              */
#define BD_LEDGER_DIFFUSE         2   /* exit through the entrance face                      */
#define BD_LEDGER_TRANSMITTED     3   /* exit through the far depth face                     */
#define BD_LEDGER_LATERAL         4   /* lateral faces, r_max cut, launch misses             */
#define BD_LEDGER_ABSORBED        5   /* absorbed in voxels without BD_FLAG_ABLATED          */
#define BD_LEDGER_ABSORBED_VOID   6   /* absorbed in ablated voxels (plume attenuation)      */
#define BD_LEDGER_ROULETTE_GAIN   7   /* weight added by Russian-roulette survivors (9 w)    */
#define BD_LEDGER_ROULETTE_LOSS   8   /* weight removed by Russian-roulette kills            */
#define BD_LEDGER_TRUNCATED       9   /* weight left when a photon hit max_events            */
#define BD_LEDGER_COLLISIONS     10   /* number of interaction events                        */
#define BD_LEDGER_CROSSINGS      11   /* number of voxel-face crossings                      */
#define BD_LEDGER_REFLECTIONS    12   /* Fresnel/TIR reflections at index steps and faces    */
#define BD_LEDGER_LEN            16

/* closure = (SPECULAR+DIFFUSE+TRANSMITTED+LATERAL+ABSORBED+ABSORBED_VOID+TRUNCATED
 *            +ROULETTE_LOSS-ROULETTE_GAIN) / LAUNCHED == 1 to FP64 round-off. */

/* ---- beam profiles (simulation/voxel_mc_3d.py:101-120, :619) ---------------- */
#define BD_BEAM_GAUSSIAN        0
#define BD_BEAM_TOPHAT          1
#define BD_BEAM_KIM_EXP_DISK    2
#define BD_BEAM_KIM_GAUSS_DISK  3

/* ---- MC option bits --------------------------------------------------------- */
#define BD_MC_TALLY_FLUENCE   0x1  /* also tally track length L (reference Phi_3d) */
#define BD_MC_METAL_SEMANTICS 0x2  /* Metal deltas: r_max checked only at collisions,
                                      index threshold 1e-4 (voxel_mc_metal.py:246-252,318) */

typedef struct BdMcParams {
    int32_t nx, ny, nz;
    int32_t launch_axis;     /* 0: inject at z=0 along +z; 1: inject at x=0 along +x   */
    float dx, dy, dz;
    float lx, ly, lz;
    float init_ux, init_uy, init_uz;
    float cos_ph, sin_ph, cos_th_safe;
    float x_center, y_center, z_center;
    float sigma_axis;        /* Gaussian per-axis sigma = spot_dia / 4                 */
    float beam_radius;       /* disk radius for the top-hat / Kim profiles              */
    int32_t beam_profile;    /* BD_BEAM_*                                               */
    float n_ambient;
    float r_max_sq;          /* 0 = domain boundaries only                             */
    int32_t options;         /* BD_MC_* bits                                            */
    int32_t _pad0;
    int64_t n_photons;
    int64_t photon_offset;   /* index of the first photon (batches of one run)          */
    int64_t max_events;      /* per-photon event cap; remaining weight -> TRUNCATED     */
    uint64_t seed;           /* Philox-4x32-10 key                                      */
} BdMcParams;

/* ---- thermal / ablation parameters --------------------------------------- */
#define BD_BC_SERIES  0  /* half-cell conduction in series with h_eff (voxel_thermal_3d.py:97,105) */
#define BD_BC_METAL   1  /* -h_eff (T - T_amb) / dz (metal_ablation_solver.py:141,150)           */

typedef struct BdThermalParams {
    int32_t nx, ny, nz;
    int32_t is_active;       /* 0: source off (passive cooling)                      */
    float dx, dy, dz;
    float dt;
    float h_eff;
    float t_ambient;
    int32_t bc_mode;         /* BD_BC_*                                               */
    float q_scale;           /* heat source = src * q_scale                           */
} BdThermalParams;

typedef struct BdAblationParams {
    int32_t nx, ny, nz;
    int32_t is_active;
    float dx, dy, dz;
    float dt;
    float h_eff;
    float t_ambient;
    float t_abl;
    float t_void;
    int32_t bc_mode;
    int32_t has_arrhenius;
    float arr_A, arr_Ea_over_R;
    int32_t has_char;
    float char_A, char_Ea_over_R;
    float q_scale;           /* heat source = src * q_scale                           */
    int32_t zero_src_in_ablated; /* 1: source is 0 in ablated voxels (coupled_ablation.py:476-478) */
} BdAblationParams;

#define BD_PLUME_DT_AS_GIVEN 0  /* plume.py:79, CPU numba semantics                        */
#define BD_PLUME_DT_METAL    1  /* min(dt, 0.45/(2 d_rate)), metal_ablation_solver.py:235-237 */
#define BD_PLUME_DT_SUBCYCLE 2  /* n_sub stable steps of dt/n_sub per substep                */

typedef struct BdPlumeParams {
    int32_t nx, ny, nz;
    int32_t dt_policy;       /* BD_PLUME_DT_*                                          */
    float dx, dy, dz;
    float dt;                /* thermal substep                                       */
    float D_xy, D_z, vz;
    float tau_linger;        /* <= 0 or inf: no decay                                  */
    int32_t n_sub;           /* sub-cycles per substep for SUBCYCLE (0 = automatic)   */
    int32_t _pad0;
} BdPlumeParams;

/* ---- library ---------------------------------------------------------------- */
BD_API int bd_abi_version(void);
/* Copies the last error message of this thread into buf (always NUL-terminated). */
BD_API int bd_last_error(char* buf, size_t buf_len);
/* Number of CUDA devices; replaces is_metal_available() (voxel_mc_metal.py:23,
 * voxel_thermal_metal.py:24, metal_ablation_solver.py:26). */
BD_API int bd_device_count(int* count);
/* Selects the device for this thread and creates its context. */
BD_API int bd_device_init(int device);
/* Blocks until all work on `stream` is done; reports asynchronous faults. */
BD_API int bd_stream_sync(void* stream);

/* ---- Monte Carlo (simulation/voxel_mc_3d.py:123-422, voxel_mc_metal.py:173-332) --- */
/* Packs four property grids into one float4 per voxel {mu_t, mu_a/mu_t, g, n}, adding
 * optional plume extinction (plume_mu_ext != NULL):
 * mu_a += mu_ext*ratio_a, mu_s += mu_ext*ratio_s, g = g_plume where mu_ext > 0.001 in ablated
 * voxels (coupled_ablation.py:445-452). flags may be NULL when plume_mu_ext is NULL. */
BD_API int bd_mc_pack_props(const float* mu_a, const float* mu_s, const float* g, const float* n,
                     const float* plume_mu_ext, const uint8_t* flags,
                     float ratio_a, float ratio_s, float g_plume,
                     int64_t n_voxels, float* props_out /* float4[n_voxels] */, void* stream);

typedef struct BdMcContext BdMcContext;   /* owns the photon queue and ledger partials */
BD_API int bd_mc_create(BdMcContext** ctx);
BD_API int bd_mc_destroy(BdMcContext* ctx);
/* Traces p->n_photons packets and ADDS their weights into A (and L if
 * BD_MC_TALLY_FLUENCE) and the lateral-escape depth histogram lat_depth (may be NULL).
 * ledger receives BD_LEDGER_LEN doubles (overwritten, not added). flags (may be NULL)
 * splits absorption into ABSORBED / ABSORBED_VOID. Replaces the Metal dispatch of
 * trace_photons (voxel_mc_metal.py:508-530) and _mc3d_trace_photons (voxel_mc_3d.py:340-422). */
BD_API int bd_mc_trace(BdMcContext* ctx, const BdMcParams* p, const float* props, const uint8_t* flags,
                float* A, float* L, double* lat_depth, double* ledger, void* stream);
/* bd_mc_trace without any device allocation. No counterpart in the reference: it is for
 * callers that must not allocate device memory while running -- a fixed-latency control loop
 * (an allocation can synchronise the device or block in the driver) or a host framework that
 * owns all device memory through its own pool. Its scratch (photon-queue counter + one FP64
 * ledger row per block, 256 B + 2048 x 16 doubles = 256.25 KiB) is a static device array that
 * every GPU loading this library holds until the process exits. The first call on a device
 * looks up that device's copy of the array (cached until a cudaDeviceReset of that device, after
 * which this entry point must not be used), so make it before any timing-critical phase. The
 * kernel is persistent, so any photon count runs on a grid capped at 2048 blocks. Every call
 * shares the array: calls that overlap on the GPU (other streams, other host threads on the
 * same device) race and must be serialised by the caller. Its absorbed map is summed with FP32
 * atomics (bd_mc_trace sums exactly in 64-bit fixed point, which needs per-voxel scratch): the
 * same photon histories, with FP32 rounding of the per-voxel sums (~1e-5 relative at 1e5 photons). */
BD_API int bd_mc_trace_noalloc(const BdMcParams* p, const float* props, const uint8_t* flags, float* A, float* L,
                               double* lat_depth, double* ledger, void* stream);
/* dst64[i] += src32[i]; src32[i] = 0 (folds a batch tally into an FP64 accumulator). */
BD_API int bd_fold_f32_to_f64(float* src32, double* dst64, int64_t n, void* stream);

/* ---- bioheat stencil (voxel_thermal_3d.py:30-112, voxel_thermal_metal.py:56-134) --- */
/* n_substeps explicit steps ping-ponging between T_a (input) and T_b; the result is in
 * T_a when n_substeps is even, else in T_b. Replaces run_thermal3d_substeps_metal
 * (voxel_thermal_metal.py:179-285) and MetalThermalContext.advance (:348-376). */
BD_API int bd_thermal_advance(const BdThermalParams* p, float* T_a, float* T_b, int n_substeps,
                       const float* src, const float* k, const float* rho_cp, void* stream);

/* ---- fused ablation substep (metal_ablation_solver.py:71-241; CPU twin
 *      coupled_ablation.py:515-531 = _thermal3d_step_explicit + _apply_latent_heat_plateau
 *      + _accumulate_arrhenius + _accumulate_char) ---------------------------------- */
/* Ping-pong as bd_thermal_advance. H_acc, Omega, chi are updated in place; Omega may be
 * NULL when has_arrhenius == 0 and chi NULL when has_char == 0. Replaces
 * MetalAblationContext.advance_substeps (metal_ablation_solver.py:399-437). */
BD_API int bd_ablation_advance(const BdAblationParams* p, float* T_a, float* T_b, int n_substeps,
                        float* H_acc, float* Omega, float* chi, const uint8_t* flags,
                        const float* src, const float* k, const float* rho_cp, void* stream);

/* ---- plume diffusion (plume.py:18-80; Metal block metal_ablation_solver.py:193-240) --- */
/* Advances n_substeps thermal substeps of plume transport in the BD_FLAG_VOID domain;
 * each substep is 1 step (AS_GIVEN, METAL) or n_sub steps (SUBCYCLE). Result lands in
 * *result_in_b = 0 -> C_a, 1 -> C_b (host int written synchronously from the step count). */
BD_API int bd_plume_advance(const BdPlumeParams* p, float* C_a, float* C_b, int n_substeps,
                     const uint8_t* flags, int* result_in_b, void* stream);
/* Number of plume steps per substep the parameters imply (SUBCYCLE: ceil of dt/dt_stable). */
BD_API int bd_plume_steps_per_substep(const BdPlumeParams* p, int* n_steps, float* dt_step);

/* ---- flags ---------------------------------------------------------------- */
/* flags = ablated | dry<<1 | void<<2 from three uint8 masks (void may be NULL -> ablated). */
BD_API int bd_pack_flags(const uint8_t* ablated, const uint8_t* dry, const uint8_t* void_mask,
                  int64_t n_voxels, uint8_t* flags, void* stream);


/* ---- coupled epoch engine (simulation/coupled_ablation.py:183-667) ---------------- */
/* A per-voxel parameter that is either a grid (ptr != NULL) or one value, like the
 * reference's size-1 / size-N dry_state and char_state arrays (coupled_ablation.py:409-438). */
typedef struct BdGridRef {
    const float* ptr;
    float value;
    int32_t _pad;
} BdGridRef;

/* Epoch-end update: _update_phase_properties_numba (coupled_ablation.py:77-180) or
 * _update_single_stage_ablation_numba (:61-74), _remove with the air-gap breach (:628-660),
 * compute_void_mask (:619-626), plume inject + sync_extinction (plume.py:292-366) and the
 * plume-augmented MC properties of the next epoch (coupled_ablation.py:445-452). */
typedef struct BdPhaseDesc {
    int32_t nx, ny, nz;
    int32_t single_stage;      /* 1: dry_state is None                                   */
    int32_t apply_removal;     /* 1: removed voxels become void (the engine); 0: flag only */
    int32_t has_char_state, has_cs_mu_a, has_cs_mu_s, has_cs_k, has_cs_rho_cp;
    int32_t gap_k0, gap_k1;    /* air_gap_range; gap_k0 <= 0 means none                  */
    int32_t has_plume;
    float t_abl, alpha_max_stable, cs_chi_remove, k_void, rho_cp_void, t_void;
    float plume_delta_mu, plume_mu_max, plume_ratio_a, plume_ratio_s, plume_g;
    float *T, *H_acc, *chi, *mu_a, *mu_s, *g, *n, *k, *rho_cp, *T_peak, *ablation_time;
    const float *h_lat, *wet_mu_a, *wet_k, *wet_rho_cp;
    BdGridRef ds_mu_a, ds_mu_s, ds_g, ds_n, ds_k, ds_rho_cp, ds_t_remove;
    BdGridRef cs_mu_a, cs_mu_s, cs_k, cs_rho_cp, cs_t_remove;
    uint8_t* flags;            /* BD_FLAG_* per voxel                                   */
    uint8_t* to_remove;        /* optional output mask                                  */
    float *plume, *mu_ext;     /* plume raw field and saturated extinction (has_plume)  */
    float* props;              /* optional packed MC properties (float4 per voxel)      */
} BdPhaseDesc;

typedef struct BdEngineDesc {
    BdPhaseDesc phase;
    BdAblationParams substep;  /* q_scale and is_active are set per epoch from the power  */
    int32_t n_substeps;
    int32_t has_plume_transport;
    BdPlumeParams plume;
    BdMcParams mc;             /* n_photons, beam, options; photon_offset is set per epoch */
    float *T_alt, *omega, *plume_alt, *A, *L;
    double* lat_depth;
    double dt_epoch;
    double voxel_volume;
} BdEngineDesc;

typedef struct BdEpochDiag {
    double ledger[BD_LEDGER_LEN];  /* MC ledger of the epoch (zeros when the laser is off) */
    double epoch, time_s, n_new, n_ablated, gap_open;
    double plume_tau;              /* sum of plume mu_a along the centre column x dz       */
    double plume_peak_mu_a;
    double plume_ablated_sum;      /* sum of plume mu_a over ablated voxels                */
    double t_optical_ms, t_thermal_ms, t_epoch_end_ms;  /* device time of the three stages */
    double n_void;                 /* voxels in the plume domain after this epoch           */
    double void_zlimit;            /* 1 + deepest slice holding a void voxel                 */
} BdEpochDiag;

#define BD_EPOCH_SKIP_MC 0x1       /* use the absorbed map already in A (no MC this epoch) */
#define BD_EPOCH_NO_GRAPH 0x2      /* launch the stages directly instead of as CUDA graphs  */
#define BD_EPOCH_SERIAL_PLUME 0x4  /* run the plume stage after the substeps on the caller's stream
                                      instead of beside MC + substeps on the engine's plume stream */
#define BD_EPOCH_EXTERNAL_PLUME 0x8 /* enqueue the epoch's start, MC and substeps only: the caller runs
                                      the plume stage (bd_plume_batch_run) and then the epoch end
                                      (bd_engine_epoch_finish); rejected while stage timing is on */

typedef struct BdEngine BdEngine;
/* Replaces CoupledAblationEngine.__init__ device setup (coupled_ablation.py:184-407);
 * the descriptor's device fields are borrowed, not copied. */
BD_API int bd_engine_create(const BdEngineDesc* desc, BdEngine** out);
BD_API int bd_engine_destroy(BdEngine* e);
/* One coupled epoch (CoupledAblationEngine.step_epoch, coupled_ablation.py:440-617):
 * MC -> n_substeps fused substeps -> plume transport -> epoch-end update, all enqueued. */
BD_API int bd_engine_step_epoch(BdEngine* e, float power, int options, void* stream);
/* Only the epoch-end update (phase, removal, breach, plume sync, MC properties). */
BD_API int bd_engine_epoch_end(BdEngine* e, void* stream);
/* The epoch end of an epoch enqueued with BD_EPOCH_EXTERNAL_PLUME (the stage bd_engine_step_epoch
 * ends with otherwise); enqueue it after that epoch's plume stage. */
BD_API int bd_engine_epoch_finish(BdEngine* e, void* stream);

/* Batched plume stage: the plume stages of up to 32 engines of one grid and one set of plume
 * parameters run as one launch per FTCS step over the live units of every engine (a campaign's
 * instances; no reference counterpart: the reference runs its campaign as sequential processes,
 * run_highres_knowledge_suite.py:633-654). The engines' epochs are enqueued with
 * BD_EPOCH_EXTERNAL_PLUME; bd_plume_batch_run then advances every engine's plume field over one epoch
 * (its results are those of each engine's own stage), after which each engine's epoch end is
 * enqueued with bd_engine_epoch_finish. The stage runs as a CUDA graph captured on the first call. */
typedef struct BdPlumeBatch BdPlumeBatch;
BD_API int bd_plume_batch_create(BdEngine* const* engines, int n, BdPlumeBatch** out);
BD_API int bd_plume_batch_run(BdPlumeBatch* b, void* stream);
BD_API int bd_plume_batch_destroy(BdPlumeBatch* b);
/* Synchronises `stream` and copies the diagnostics of the last epoch to the host. */
BD_API int bd_engine_read_diag(BdEngine* e, BdEpochDiag* out, void* stream);
BD_API int bd_engine_set_time(BdEngine* e, double t, int64_t epoch, void* stream);
/* Replaces the MC launch template (beam centre / angles / photon count changed between
 * epochs, as the reference allows for scanning, coupled_ablation.py:222). */
BD_API int bd_engine_set_mc(BdEngine* e, const BdMcParams* mc);
/* Stage timing across many epochs without a per-epoch synchronisation: while enabled each epoch
 * records CUDA events at its stage boundaries (begin | MC | fused substeps | plume | epoch end).
 * Enabling resets the totals; _read synchronises and returns the summed milliseconds of the
 * four stages and the number of timed epochs. */
#define BD_STAGE_MC         0
#define BD_STAGE_SUBSTEPS   1
#define BD_STAGE_PLUME      2
#define BD_STAGE_EPOCH_END  3
/* Mid-run optics change, as the dual-wavelength runner switches lambda
 * (knowledge/beetle/scripts/run_dual_permutation_suite.py:254-283): new plume extinction constants
 * (plume.py:270-278), then, after the caller has written the new optical grids, a pass that
 * re-derives the plume extinction and the packed MC properties (no plume injection, no change to
 * the epoch's diagnostics). */
BD_API int bd_engine_set_plume_optics(BdEngine* e, float mu_max, float ratio_a, float ratio_s, float delta_mu);
BD_API int bd_engine_refresh_props(BdEngine* e, void* stream);
BD_API int bd_engine_timing(BdEngine* e, int enable);
BD_API int bd_engine_timing_read(BdEngine* e, double* stage_ms /* [4] */, int64_t* epochs);

/* ---- per-epoch recording on the device ----------------------------------------------------------
 * What the production runner pulls from the engine after every epoch
 * (knowledge/beetle/scripts/run_highres_knowledge_suite.py:271-306): the xz slice at y of T, Q,
 * the 4-phase map of compute_phase_map (simulation/run_multispectral_matrix.py:168-192, with the
 * air gap as phase 3), the plume absorption, the crater depth below k_surface in that slice, the
 * peak temperature of three depth bands, and the epoch's diagnostics. bd_engine_record enqueues
 * the kernels that fill a record slot in device memory (no synchronisation); the caller copies the
 * slot to pinned host memory asynchronously. Slot layout: BdRecordHead, padded to 256 bytes, then
 * float T[nx][nz], float Q[nx][nz] (W/mm^3), float plume_mu_a[nx][nz], uint8 phase[nx][nz]. */
typedef struct BdRecordSpec {
    int32_t y;                         /* slice index                                               */
    int32_t k_surface;                 /* first slice below the ambient air (crater depth origin)   */
    int32_t band_k0[3], band_k1[3];    /* z ranges [k0, k1) of the peak temperatures                */
    int32_t gap_k0, gap_k1;            /* air-gap slices (gap_k0 == gap_k1: none)                   */
    float q_scale;                     /* W/mm^3 per unit of raw absorbed weight (0: laser off)     */
    float plume_ratio_a;               /* mu_a share of the saturated plume extinction              */
} BdRecordSpec;
typedef struct BdRecordHead {
    double time_s, epoch, plume_tau, n_new, n_void, absorbed_weight;
    float peak_T[3];                   /* -inf for an empty band                                    */
    int32_t depth_voxels;              /* 1 + deepest ablated slice below k_surface in the slice; 0 */
} BdRecordHead;
BD_API int64_t bd_record_slot_bytes(int nx, int nz);
BD_API int bd_engine_record(BdEngine* e, const BdRecordSpec* spec, void* slot, void* stream);

/* ---- launch-shape tuning ------------------------------------------------------------------------
 * No counterpart in the reference (its kernels have fixed launch shapes). Process-wide knobs read at
 * every launch; results do not depend on them beyond the order of FP32 atomic tally additions. A
 * change bumps a generation counter so engines re-capture their epoch graphs. */
#define BD_TUNE_MC_BLOCKS_PER_SM  0  /* persistent MC grid: 128-thread CTAs per SM, 1..16 (0 = occupancy
                                        limit); photons per thread = n_photons / (grid * 128)          */
#define BD_TUNE_STENCIL_XC        1  /* x-planes per CTA of the TMA substep kernel, 1..64 (default 8)   */
#define BD_TUNE_PLUME_XC          2  /* direct plume kernel: x-planes per CTA, 1..64 (default 4)         */
#define BD_TUNE_PLUME_KERNEL      3  /* plume stage: BD_PLUME_KERNEL_DIRECT (default) or
                                        BD_PLUME_KERNEL_COMPACT (value 5 is not used)                   */
#define BD_PLUME_KERNEL_DIRECT    4  /* one launch per FTCS step: a CTA per 32 (z) x 16 (y) tile column
                                        marching x planes over the column's live z groups              */
#define BD_PLUME_KERNEL_COMPACT   6  /* the direct kernel's per-unit code over a compact list of the live
                                        (column, band) units, one wave of CTAs per step: once per stage
                                        the x planes per unit are chosen on the device (2..12, the
                                        smallest whose unit count fits one wave; BD_TUNE_PLUME_XC is not
                                        used), so no empty CTA is dispatched and no partial second wave
                                        runs. Same results as BD_PLUME_KERNEL_DIRECT; nz % 4 != 0 falls
                                        back to it                                                      */
#define BD_TUNE_STENCIL_CAP       4  /* at most this many substep CTAs per SM (0 = no cap, default): the
                                        plume stage runs beside the substeps and keeps the rest         */
#define BD_TUNE_COUNT             5
BD_API int bd_tune_set(int knob, int value);
BD_API int bd_tune_get(int knob, int* value);

/* Self-test of the bounded-wait failure path (no counterpart in the reference): one thread waits at
 * most max_polls (1..2^20) polls, through the kernels' own bounded mbarrier wait, on a barrier that
 * nothing arrives on (arrive = 0: returns BD_ERR_TIMEOUT) or that it completed itself (arrive = 1:
 * BD_OK). Synchronises `stream`; the context stays usable after the timeout. */
BD_API int bd_selftest_wait_timeout(int max_polls, int arrive, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Absorbed-map denoiser: 3-D convolution layers (tcgen05 BF16 tensor cores, FP32 accumulation).
 * No counterpart in the reference, which has no learned component; these are the building blocks
 * of the U-Net that denoises low-photon absorbed-power maps.
 *
 * Volumes are bf16 with a one-voxel zero pad, stored as 8-channel planes: a level with interior
 * nx x ny x nz has R = bd_conv_plane_rows(nx, ny, nz) rows per plane ((nx+2)(ny+2)(nz+2) padded rows,
 * z fastest, then a zero margin), and channel c of padded row v is element ((c/8)*R + v)*8 + c%8.
 * Buffers must start zeroed; every call keeps the pad and margin rows zero. Taps are ordered t = (dx+1)*9 + (dy+1)*3 + (dz+1) (27 taps) or t = (dx+1)*3 + (dy+1)
 * (9 taps, for an input whose z neighbours are packed into its channels); weights are FP32
 * [taps][cout][cin]. */
#define BD_CONV_FWD_RELU   0  /* out = relu(conv + bias) at this level                               */
#define BD_CONV_FWD_UPADD  1  /* out(finer) = up2(relu(conv + bias)) + aux(finer); out_coarse = relu  */
#define BD_CONV_FWD_HEAD   2  /* 1x1 head + residual on the noisy map, loss and head gradient fused  */
#define BD_CONV_BWD_RAW    3  /* out = conv (transposed weights)                                     */
#define BD_CONV_BWD_MASK   4  /* out = conv * (aux > 0)                                              */
#define BD_CONV_BWD_UPADD  5  /* out(finer) = (aux(finer) + up2(conv)/8) * (aux2(finer) > 0)         */

typedef struct BdConvCall {
    int nx, ny, nz;          /* interior size of the level the convolution runs on                  */
    int cin;                 /* channels per input row (16, 32 or 64)                               */
    int cout_total;          /* channels per output row                                             */
    int n_off, n_slice;      /* output channels [n_off, n_off + n_slice) computed by this call      */
    int taps;                /* 27 or 9                                                             */
    int mode;                /* BD_CONV_*                                                           */
    const void* input;       /* bf16 input planes                                                   */
    const void* wimage;      /* weight image of this slice (bd_conv_pack_weights)                   */
    const float* bias;       /* [n_slice] (forward modes) or NULL                                   */
    void* out;               /* bf16 output planes (finer level for the UPADD modes)                */
    void* out_coarse;        /* FWD_UPADD: optional copy of relu(conv + bias) at this level         */
    const void* aux;         /* see the modes above                                                 */
    const void* aux2;
    /* FWD_HEAD only (n_slice == cout_total == 16): pred = (a_noisy*scale + head.relu(conv+bias)) *
     * mask, written unpadded as pred/scale; with a target, loss += sum (pred - target*scale)^2 and
     * grad_out / head_grad receive the gradients of loss * loss_norm. */
    const float* head;       /* [17] weights then bias                                              */
    const float* a_noisy;    /* fp32 [nx*ny*nz]                                                     */
    const uint8_t* mask;     /* [nx*ny*nz] 0 or 1                                                   */
    float scale;
    float loss_norm;
    float* pred;             /* fp32 [nx*ny*nz]                                                     */
    const float* target;     /* fp32 [nx*ny*nz] or NULL (inference)                                 */
    float* head_grad;        /* [17], accumulated                                                   */
    double* loss;            /* [1], accumulated                                                    */
    void* grad_out;          /* bf16 planes (16 channels): gradient at the head input               */
} BdConvCall;

/* Rows per 8-channel plane of a level (padded rows plus the zero margin the tile copies read). */
BD_API int64_t bd_conv_plane_rows(int nx, int ny, int nz);
/* Bytes of the shared-memory weight image of one output-channel slice. */
BD_API int64_t bd_conv_image_bytes(int taps, int k_channels, int n_slice);
/* FP32 [taps][cout][cin] -> bf16 image for output channels [n_off, n_off + n_slice). transpose=0:
 * the forward convolution (K = cin); transpose=1: the data-gradient convolution, whose outputs are
 * the layer's input channels (K = cout, taps mirrored). */
BD_API int bd_conv_pack_weights(int taps, int cin, int cout, int n_off, int n_slice, int transpose,
                                const float* w, void* wimage, void* stream);
BD_API int bd_conv3d(const BdConvCall* c, void* stream);
/* dw[t][co][ci] += sum over voxels of grad[v][co] * act[v + offset(t)][ci] (FP32 atomics). */
BD_API int bd_conv3d_wgrad(int nx, int ny, int nz, int cin, int cout, int taps, const void* grad,
                           const void* act, float* dw, void* stream);

/* The denoiser network (3-level U-Net, 16/32/64 channels) over an nx x ny x nz MC grid (multiples
 * of 4). Inputs: the noisy absorbed map (fraction of launched weight per voxel, as bd_mc_trace
 * tallies it), the packed MC properties (bd_mc_pack_props: mu_t, mu_a/mu_t, g, n per voxel) and the
 * optional flag bytes; `scale` multiplies the map into the network's working range. Parameters are
 * one FP32 vector of bd_unet_param_count() values: per layer W[taps][cout][cin] then b[cout], the
 * layers (taps, cin, cout) = (9,16,16) (27,16,16) (27,16,32) (27,32,32) (27,32,64) (27,64,64)
 * (27,64,32) (27,32,32) (27,32,16) (27,16,16), then 16 head weights and the head bias. */
typedef struct BdUnet BdUnet;
BD_API int64_t bd_unet_param_count(void);
BD_API int bd_unet_create(int nx, int ny, int nz, int training, BdUnet** out);
BD_API int bd_unet_destroy(BdUnet* net);
BD_API int bd_unet_set_params(BdUnet* net, const float* params, void* stream);   /* resets Adam state */
BD_API int bd_unet_get_params(BdUnet* net, float* params, void* stream);
BD_API int bd_unet_forward(BdUnet* net, const float* a_noisy, const float* props, const uint8_t* flags,
                           float scale, float* pred, void* stream);
/* Training pass: forward, loss = sum (pred - target)^2 * scale^2 over absorbing voxels, and the
 * gradient of loss * loss_norm into the network's gradient vector. */
BD_API int bd_unet_forward_backward(BdUnet* net, const float* a_noisy, const float* props,
                                    const uint8_t* flags, const float* target, float scale,
                                    float loss_norm, float* pred, void* stream);
BD_API int bd_unet_get_grads(BdUnet* net, float* grads, void* stream);
BD_API int bd_unet_adam(BdUnet* net, float lr, float beta1, float beta2, float eps, void* stream);
/* Synchronises `stream`; returns the last training loss and BD_ERR_TIMEOUT if a kernel gave up. */
BD_API int bd_unet_read_loss(BdUnet* net, double* loss, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BUGDEF_H */
