// Internal structures shared by the epoch-end kernels and the engine orchestration.
#pragma once

#include "common.cuh"

namespace bd {

struct GridRef {
    const float* ptr;  // per-voxel values, or nullptr to use `value`
    float value;
};

// Device-resident per-epoch scalars (zeroed at the start of every epoch except t/epoch).
struct EngineDyn {
    double ledger[BD_LEDGER_LEN];
    unsigned long long n_new;
    unsigned int gap_open;
    unsigned int plume_peak_bits;
    double plume_tau_sum;
    double plume_abl_sum;
    double n_ablated;
    double t;             // simulated time after this epoch
    long long epoch;      // epochs completed
    float t_now;          // t as float for the kernels
    float _pad;
    long long mc_offset;  // photon-stream offset of this epoch's MC
    int void_zlimit;      // 1 + deepest slice holding a void voxel (monotone: ablation is irreversible)
    int err;              // set by a kernel whose bounded wait timed out
    unsigned long long n_void;  // voxels in the plume domain after this epoch's update
};

struct PhaseArgs {
    int nx, ny, nz;
    int single_stage, apply_removal;
    int has_cs, has_cs_mu_a, has_cs_mu_s, has_cs_k, has_cs_rho;
    int gap_k0, gap_k1;
    int has_plume;
    float t_abl, alpha_max, cs_chi_rem, k_void, rho_void, t_void;
    float delta_mu, mu_max, ratio_a, ratio_s, g_plume;
    int props_only;
    float *T, *H, *chi, *mu_a, *mu_s, *g, *n, *k, *rho, *T_peak, *ablation_time;
    const float *h_lat, *wet_mu_a, *wet_k, *wet_rho;
    GridRef ds_mu_a, ds_mu_s, ds_g, ds_n, ds_k, ds_rho, ds_t_rem;
    GridRef cs_mu_a, cs_mu_s, cs_k, cs_rho, cs_t_rem;
    uint8_t* flags;
    uint8_t* to_remove;   // optional per-voxel output
    float *plume, *mu_ext;
    float* props;         // float4 per voxel, optional
    EngineDyn* dyn;
};

#define BD_PHASE_FULL 0  // phase update + removal + breach + void/plume/props pass
#define BD_PHASE_INIT 1  // breach check (gap_open) + void/plume/props pass only
#define BD_PHASE_PROPS 2 // void bits, plume extinction and packed MC properties only (no injection,
                         // no diagnostics): after the optics change mid-run
int phase_launch(const PhaseArgs& a, int mode, cudaStream_t st);
int ablation_launch(const BdAblationParams* p, float* Ta, float* Tb, int n, float* H, float* Om, float* Chi,
                    const uint8_t* F, const float* src, const float* K, const float* R, cudaStream_t st, int* err);
int plume_launch(const BdPlumeParams* p, float* Ca, float* Cb, int n_substeps, const uint8_t* F, int* in_b,
                 cudaStream_t st, const int* zlimit, int full_first, uint8_t* mask);
int plume_policy_steps(const BdPlumeParams* p, int* n_steps, float* dt_step, float* decay_step);
// One instance of a batched plume stage (several engines' plume stages in one launch per step).
struct PlumeTab;
struct PlumeInstHost {
    float* Ca;               // the field at the start of the stage
    float* Cb;               // the other ping-pong buffer
    uint8_t* mask;           // the instance's neighbourhood bytes + z lists (plume_mask_bytes)
    const uint8_t* flags;    // voxel flags (void bit)
    const int* zlimit;       // void z-limit on the device
    const BdPlumeParams* params;
    int n_substeps;
};
// Plume stages of n instances of one grid (their diffusivities, and so their weights and step
// counts, may differ): per instance its mask and z lists, then one list of the live (instance,
// column, band) units, then one launch per FTCS step covering every instance still stepping.
// plume_batch_prepare fills the device descriptors (`dev`, plume_batch_desc_bytes(n) bytes) and
// orders the instances by step count (order[r] = instance of rank r); the launch enqueues a stage.
size_t plume_batch_desc_bytes(int n);
size_t plume_batch_units_words(int n, int nx, int ny, int nz);
int plume_batch_prepare(int n, const PlumeInstHost* insts, void* dev, int* order, long long* max_steps);
int plume_batch_launch(int n, const PlumeInstHost* insts, const int* order, const void* dev, long long max_steps,
                       unsigned* units, cudaStream_t st);
// Per-epoch xz recording (record.cu): inputs of one launch.
struct RecordArgs {
    int nx, ny, nz, y, k_surface, gap_k0, gap_k1;
    int band_k0[3], band_k1[3];
    float q_scale, plume_ratio_a;
    const float *T, *H, *chi, *A, *mu_ext;
    const uint8_t* flags;
};
constexpr int64_t kRecordHeadBytes = 256;   // BdRecordHead, padded so the slices stay aligned
int record_launch(const RecordArgs& a, const EngineDyn* dyn, float plume_dz, void* slot, cudaStream_t st);

int mc_launch(const BdMcParams* p, const float* props, const uint8_t* flags, float* A, float* L, double* latz,
              double* ledger, unsigned long long* queue, double* partials, int max_blocks, int sm_count,
              cudaStream_t st, const long long* offset_dev, unsigned long long* tally64);

}  // namespace bd
