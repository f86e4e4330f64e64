// Per-epoch recording on the device: the xz slice and scalars that the production runner pulls
// from the engine after every epoch (run_highres_knowledge_suite.py:271-306): T, Q, the 4-phase map
// of compute_phase_map (run_multispectral_matrix.py:168-192), the plume absorption, the crater depth
// below the dorsal surface and the peak temperatures of three depth bands, plus the epoch's
// diagnostics. One launch writes a compact record slot in device memory; the caller copies it
// asynchronously to pinned host memory, so recording needs no per-epoch synchronisation.
#include "common.cuh"
#include "engine.cuh"

namespace bd {

namespace {

// order-preserving float <-> int map, for atomicMax on floats of any sign
__device__ __forceinline__ int f2o(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void k_record_head(const EngineDyn* dyn, float plume_dz, BdRecordHead* head) {
    if (threadIdx.x != 0) return;
    head->time_s = dyn->t;
    head->epoch = (double)dyn->epoch;
    head->plume_tau = dyn->plume_tau_sum * (double)plume_dz;
    head->n_new = (double)dyn->n_new;
    head->n_void = (double)dyn->n_void;
    head->absorbed_weight = dyn->ledger[BD_LEDGER_ABSORBED] + dyn->ledger[BD_LEDGER_ABSORBED_VOID];
    int* pk = reinterpret_cast<int*>(head->peak_T);
    for (int b = 0; b < 3; ++b) pk[b] = f2o(-INFINITY);
    head->depth_voxels = 0;
}

__global__ void k_record_xz(RecordArgs a, BdRecordHead* head, float* sT, float* sQ, float* sP, uint8_t* sPh) {
    const int n = a.nx * a.nz;
    float best[3] = {-INFINITY, -INFINITY, -INFINITY};
    int depth = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int x = i / a.nz, z = i - x * a.nz;
        const size_t v = ((size_t)x * a.ny + a.y) * a.nz + z;
        const float T = a.T[v], H = a.H[v];
        const float chi = a.chi ? a.chi[v] : 0.f;
        const uint8_t fl = a.flags[v];
        const bool gap = z >= a.gap_k0 && z < a.gap_k1;
        const bool ablated = (fl & BD_FLAG_ABLATED) != 0;
        uint8_t ph = 0;
        if (!gap && (T >= 99.5f || H > 0.f)) ph = 2;
        if (!gap && (fl & BD_FLAG_DRY) && chi >= 0.10f) ph = 1;
        if (ablated || gap) ph = 3;
        sT[i] = T;
        sQ[i] = a.A[v] * a.q_scale;
        sP[i] = a.mu_ext ? a.mu_ext[v] * a.plume_ratio_a : 0.f;
        sPh[i] = ph;
        for (int b = 0; b < 3; ++b)
            if (z >= a.band_k0[b] && z < a.band_k1[b]) best[b] = fmaxf(best[b], T);
        if (ablated && z >= a.k_surface) depth = max(depth, z - a.k_surface + 1);
    }
    for (int o = 16; o; o >>= 1) {
        for (int b = 0; b < 3; ++b) best[b] = fmaxf(best[b], __shfl_xor_sync(0xffffffffu, best[b], o));
        depth = max(depth, __shfl_xor_sync(0xffffffffu, depth, o));
    }
    if ((threadIdx.x & 31) == 0) {
        int* pk = reinterpret_cast<int*>(head->peak_T);
        for (int b = 0; b < 3; ++b)
            if (best[b] > -INFINITY) atomicMax(&pk[b], f2o(best[b]));
        if (depth > 0) atomicMax(&head->depth_voxels, depth);
    }
}

__global__ void k_record_finish(BdRecordHead* head) {
    if (threadIdx.x < 3) {
        int* pk = reinterpret_cast<int*>(head->peak_T);
        head->peak_T[threadIdx.x] = o2f(pk[threadIdx.x]);
    }
}

}  // namespace

int record_launch(const RecordArgs& a, const EngineDyn* dyn, float plume_dz, void* slot, cudaStream_t st) {
    unsigned char* base = static_cast<unsigned char*>(slot);
    BdRecordHead* head = reinterpret_cast<BdRecordHead*>(base);
    const size_t n = (size_t)a.nx * a.nz;
    float* sT = reinterpret_cast<float*>(base + kRecordHeadBytes);
    float* sQ = sT + n;
    float* sP = sQ + n;
    uint8_t* sPh = reinterpret_cast<uint8_t*>(sP + n);
    k_record_head<<<1, 32, 0, st>>>(dyn, plume_dz, head);
    k_record_xz<<<grid_for((int64_t)n, 256, 148 * 4), 256, 0, st>>>(a, head, sT, sQ, sP, sPh);
    k_record_finish<<<1, 32, 0, st>>>(head);
    BD_CHECK_LAUNCH("k_record_xz");
    return BD_OK;
}

}  // namespace bd

extern "C" int64_t bd_record_slot_bytes(int nx, int nz) {
    const int64_t n = (int64_t)nx * nz;
    return bd::kRecordHeadBytes + 12 * n + ((n + 15) / 16) * 16;
}
