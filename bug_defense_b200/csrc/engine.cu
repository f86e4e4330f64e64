// Device-resident coupled epoch (CoupledAblationEngine.step_epoch,
// simulation/coupled_ablation.py:440-617) with no host round trip inside an epoch:
//   epoch begin  -> zero per-epoch counters, t += dt_epoch, photon-stream offset
//   MC           -> bd_mc_trace on the packed properties of the previous epoch end
//   substeps     -> n fused bioheat/plateau/Arrhenius/char substeps, source = A * P/(N V)
//                   with zero source in ablated voxels (coupled_ablation.py:474-478)
//   plume        -> transport in the void domain (dt policy: as given / Metal clamp / subcycle)
//   epoch end    -> phase update, removal, breach, plume inject + saturation, MC properties
// All state lives in device buffers owned by the caller; the engine owns only scratch.
#include "engine.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

struct StageGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> key;
    int tune_gen = -1;   // launch shapes baked into the graph
};

struct BdEngine {
    BdEngineDesc d;
    cudaStream_t cap_stream = nullptr;  // private stream used only to capture stage graphs
    // the plume stage runs on its own (higher-priority) stream, forked after the epoch begins and
    // joined before the epoch end: within an epoch it shares no data with the MC and the substeps
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool ring_concurrent = false;  // the timing ring's plume events come from the side stream
    StageGraph g_mc, g_sub_on, g_sub_off, g_plume, g_end;
    uint8_t* plume_mask = nullptr;      // plume neighbourhood bytes (rebuilt every epoch)
    bd::PhaseArgs pa;
    bd::EngineDyn* dyn = nullptr;      // device
    bd::EngineDyn* dyn_host = nullptr; // pinned
    unsigned long long* queue = nullptr;
    double* partials = nullptr;
    unsigned long long* tally64 = nullptr;   // fixed-point absorbed-weight tally of the MC stage
    int partial_blocks = 0;
    int sm_count = 148;
    long long epochs_enqueued = 0;  // host mirror of the epoch count (photon-stream offsets)
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool timed = false;
    // stage-timing ring: 5 events per timed epoch
    bool ring_on = false;
    std::vector<cudaEvent_t> ring;
    size_t ring_used = 0;
    int ring_error = 0;
};

static void graph_reset(StageGraph& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    g.key.clear();
}

// Launches `enqueue` as a captured graph on `st`, re-capturing when `key` changed.
template <typename F>
static int run_stage(BdEngine* e, StageGraph& g, const void* key, size_t key_len, bool use_graph, cudaStream_t st,
                     F enqueue) {
    if (!use_graph) return enqueue(st);
    const unsigned char* kb = static_cast<const unsigned char*>(key);
    if (!g.exec || g.tune_gen != bd::tune_generation() || g.key.size() != key_len ||
        (key_len && memcmp(g.key.data(), kb, key_len) != 0)) {
        graph_reset(g);
        cudaGraph_t graph = nullptr;
        BD_CUDA(cudaStreamBeginCapture(e->cap_stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue(e->cap_stream);
        cudaError_t ce = cudaStreamEndCapture(e->cap_stream, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return bd::cuda_status(ce, "cudaStreamEndCapture");
        ce = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) {
            g.exec = nullptr;
            return bd::cuda_status(ce, "cudaGraphInstantiate");
        }
        g.key.assign(kb, kb + key_len);
        g.tune_gen = bd::tune_generation();
    }
    BD_CUDA(cudaGraphLaunch(g.exec, st));
    return BD_OK;
}

static cudaEvent_t ring_event(BdEngine* e) {
    if (e->ring_used == e->ring.size()) {
        cudaEvent_t ev = nullptr;
        if (cudaEventCreate(&ev) != cudaSuccess) {
            e->ring_error = 1;
            return nullptr;
        }
        e->ring.push_back(ev);
    }
    return e->ring[e->ring_used++];
}

static void mark(BdEngine* e, cudaStream_t st, int slot) {
    if (e->timed && slot >= 0 && slot < 4 && slot != 3) cudaEventRecord(e->ev[slot], st);
    if (e->ring_on && e->timed) {
        cudaEvent_t ev = ring_event(e);
        if (ev) cudaEventRecord(ev, st);
    }
}

namespace bd {

__global__ void k_epoch_begin(EngineDyn* dyn, double dt_epoch) {
    if (threadIdx.x < BD_LEDGER_LEN) dyn->ledger[threadIdx.x] = 0.0;
    if (threadIdx.x == 0) {
        dyn->n_new = 0ull;
        dyn->gap_open = 0u;
        dyn->plume_peak_bits = 0u;
        dyn->plume_tau_sum = 0.0;
        dyn->plume_abl_sum = 0.0;
        dyn->n_ablated = 0.0;
        dyn->n_void = 0ull;
        dyn->epoch += 1;
        dyn->t += dt_epoch;
        dyn->t_now = (float)dyn->t;
        dyn->mc_offset = dyn->epoch << 32;
    }
}

__global__ void k_epoch_end_only(EngineDyn* dyn) {
    if (threadIdx.x == 0) {
        dyn->n_new = 0ull;
        dyn->gap_open = 0u;
        dyn->plume_peak_bits = 0u;
        dyn->plume_tau_sum = 0.0;
        dyn->plume_abl_sum = 0.0;
        dyn->n_ablated = 0.0;
        dyn->n_void = 0ull;
        dyn->t_now = (float)dyn->t;
    }
}

__global__ void k_set_time(EngineDyn* dyn, double t, long long epoch) {
    dyn->t = t;
    dyn->epoch = epoch;
    dyn->t_now = (float)t;
}

static GridRef gref(const BdGridRef& r) { return GridRef{r.ptr, r.value}; }

static PhaseArgs phase_args(const BdPhaseDesc& p, EngineDyn* dyn) {
    PhaseArgs a;
    a.nx = p.nx; a.ny = p.ny; a.nz = p.nz;
    a.single_stage = p.single_stage; a.apply_removal = p.apply_removal;
    a.has_cs = p.has_char_state; a.has_cs_mu_a = p.has_cs_mu_a; a.has_cs_mu_s = p.has_cs_mu_s;
    a.has_cs_k = p.has_cs_k; a.has_cs_rho = p.has_cs_rho_cp;
    a.gap_k0 = p.gap_k0; a.gap_k1 = p.gap_k1; a.has_plume = p.has_plume;
    a.t_abl = p.t_abl; a.alpha_max = p.alpha_max_stable; a.cs_chi_rem = p.cs_chi_remove;
    a.k_void = p.k_void; a.rho_void = p.rho_cp_void; a.t_void = p.t_void;
    a.delta_mu = p.plume_delta_mu; a.mu_max = p.plume_mu_max; a.ratio_a = p.plume_ratio_a;
    a.ratio_s = p.plume_ratio_s; a.g_plume = p.plume_g;
    a.T = p.T; a.H = p.H_acc; a.chi = p.chi; a.mu_a = p.mu_a; a.mu_s = p.mu_s; a.g = p.g; a.n = p.n;
    a.k = p.k; a.rho = p.rho_cp; a.T_peak = p.T_peak; a.ablation_time = p.ablation_time;
    a.h_lat = p.h_lat; a.wet_mu_a = p.wet_mu_a; a.wet_k = p.wet_k; a.wet_rho = p.wet_rho_cp;
    a.ds_mu_a = gref(p.ds_mu_a); a.ds_mu_s = gref(p.ds_mu_s); a.ds_g = gref(p.ds_g); a.ds_n = gref(p.ds_n);
    a.ds_k = gref(p.ds_k); a.ds_rho = gref(p.ds_rho_cp); a.ds_t_rem = gref(p.ds_t_remove);
    a.cs_mu_a = gref(p.cs_mu_a); a.cs_mu_s = gref(p.cs_mu_s); a.cs_k = gref(p.cs_k); a.cs_rho = gref(p.cs_rho_cp);
    a.cs_t_rem = gref(p.cs_t_remove);
    a.flags = p.flags; a.to_remove = p.to_remove; a.plume = p.plume; a.mu_ext = p.mu_ext; a.props = p.props;
    a.dyn = dyn;
    return a;
}

static int validate(const BdEngineDesc* d) {
    const BdPhaseDesc& p = d->phase;
    BD_REQUIRE(p.nx > 0 && p.ny > 0 && p.nz > 0, "bd_engine_create: grid dims must be positive");
    BD_REQUIRE(p.T && p.H_acc && p.mu_a && p.mu_s && p.g && p.n && p.k && p.rho_cp && p.flags && p.h_lat,
               "bd_engine_create: missing state field");
    BD_REQUIRE(p.single_stage || (p.wet_mu_a && p.wet_k && p.wet_rho_cp),
               "bd_engine_create: dry_state needs the wet property copies");
    BD_REQUIRE(!p.has_plume || (p.plume && p.mu_ext), "bd_engine_create: plume needs raw and extinction fields");
    BD_REQUIRE(p.gap_k0 <= 0 || (p.gap_k0 < p.gap_k1 && p.gap_k1 <= p.nz), "bd_engine_create: bad air_gap_range");
    BD_REQUIRE(d->n_substeps >= 0, "bd_engine_create: n_substeps must be >= 0");
    BD_REQUIRE(d->T_alt != nullptr, "bd_engine_create: T_alt is required");
    BD_REQUIRE(!d->has_plume_transport || (d->plume_alt && p.plume), "bd_engine_create: plume transport fields");
    BD_REQUIRE(!d->substep.has_arrhenius || d->omega, "bd_engine_create: Arrhenius needs omega");
    BD_REQUIRE(!d->substep.has_char || p.chi, "bd_engine_create: char kinetics need chi");
    BD_REQUIRE(d->A != nullptr, "bd_engine_create: absorbed map A is required");
    BD_REQUIRE(d->voxel_volume > 0.0, "bd_engine_create: voxel_volume must be > 0");
    BD_REQUIRE((long long)p.nx * p.ny * p.nz < (1LL << 31), "bd_engine_create: grid exceeds 2^31 voxels");
    BD_REQUIRE(d->mc.n_photons >= 0 && d->mc.n_photons <= kTallyMaxPhotons,
               "bd_engine_create: photons per epoch must be 0..%lld", (long long)kTallyMaxPhotons);
    return BD_OK;
}

}  // namespace bd

using namespace bd;

extern "C" int bd_engine_create(const BdEngineDesc* desc, BdEngine** out) {
    BD_REQUIRE(desc && out, "bd_engine_create: NULL argument");
    int rc = validate(desc);
    if (rc) return rc;
    BdEngine* e = new BdEngine();
    e->d = *desc;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&e->sm_count, cudaDevAttrMultiProcessorCount, dev);
    e->partial_blocks = e->sm_count * 16;
    cudaError_t err = cudaMalloc(&e->dyn, sizeof(EngineDyn));
    if (err == cudaSuccess) err = cudaMallocHost(&e->dyn_host, sizeof(EngineDyn));
    if (err == cudaSuccess) err = cudaMalloc(&e->queue, sizeof(unsigned long long));
    if (err == cudaSuccess) err = cudaMalloc(&e->partials, sizeof(double) * BD_LEDGER_LEN * e->partial_blocks);
    const size_t nv_all = (size_t)desc->phase.nx * desc->phase.ny * desc->phase.nz;
    if (err == cudaSuccess) err = cudaMalloc(&e->tally64, sizeof(unsigned long long) * nv_all);
    if (err == cudaSuccess) err = cudaMemset(e->tally64, 0, sizeof(unsigned long long) * nv_all);
    if (err == cudaSuccess) err = cudaMemset(e->dyn, 0, sizeof(EngineDyn));
    for (int q = 0; q < 4 && err == cudaSuccess; ++q) err = cudaEventCreate(&e->ev[q]);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->cap_stream, cudaStreamNonBlocking);
    if (err == cudaSuccess && desc->has_plume_transport) {
        int lo = 0, hi = 0;
        err = cudaDeviceGetStreamPriorityRange(&lo, &hi);
        if (err == cudaSuccess) err = cudaStreamCreateWithPriority(&e->side, cudaStreamNonBlocking, hi);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming);
    }
    if (err == cudaSuccess && desc->has_plume_transport)
        err = cudaMalloc(&e->plume_mask, plume_mask_bytes(desc->phase.nx, desc->phase.ny, desc->phase.nz));
    if (err != cudaSuccess) {
        bd_engine_destroy(e);
        return cuda_status(err, "bd_engine_create");
    }
    e->pa = phase_args(desc->phase, e->dyn);
    // initial void bits, gap state, plume extinction and packed MC properties for the first
    // epoch (no removal: the reference changes no voxel before its first epoch end)
    rc = phase_launch(e->pa, BD_PHASE_INIT, nullptr);
    if (rc == BD_OK) {
        err = cudaStreamSynchronize(nullptr);
        if (err != cudaSuccess) rc = cuda_status(err, "bd_engine_create: initial pass");
    }
    if (rc) {
        bd_engine_destroy(e);
        return rc;
    }
    *out = e;
    return BD_OK;
}

extern "C" int bd_engine_destroy(BdEngine* e) {
    if (!e) return BD_OK;
    cudaFree(e->dyn);
    cudaFreeHost(e->dyn_host);
    cudaFree(e->queue);
    cudaFree(e->partials);
    cudaFree(e->tally64);
    for (int q = 0; q < 4; ++q)
        if (e->ev[q]) cudaEventDestroy(e->ev[q]);
    for (cudaEvent_t ev : e->ring) cudaEventDestroy(ev);
    graph_reset(e->g_mc); graph_reset(e->g_sub_on); graph_reset(e->g_sub_off);
    graph_reset(e->g_plume); graph_reset(e->g_end);
    if (e->cap_stream) cudaStreamDestroy(e->cap_stream);
    if (e->side) cudaStreamDestroy(e->side);
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->ev_join) cudaEventDestroy(e->ev_join);
    cudaFree(e->plume_mask);
    delete e;
    return BD_OK;
}

extern "C" int bd_engine_set_time(BdEngine* e, double t, int64_t epoch, void* stream) {
    BD_REQUIRE(e != nullptr, "bd_engine_set_time: NULL engine");
    k_set_time<<<1, 1, 0, as_stream(stream)>>>(e->dyn, t, (long long)epoch);
    e->epochs_enqueued = (long long)epoch;
    // a graph-launched MC reads the photon offset from the device; keep it consistent

    BD_CHECK_LAUNCH("k_set_time");
    return BD_OK;
}

extern "C" int bd_engine_step_epoch(BdEngine* e, float power, int options, void* stream) {
    BD_REQUIRE(e != nullptr, "bd_engine_step_epoch: NULL engine");
    BD_REQUIRE(power >= 0.0f, "bd_engine_step_epoch: power must be >= 0");
    const bool external = (options & BD_EPOCH_EXTERNAL_PLUME) != 0;
    BD_REQUIRE(!(external && e->ring_on),
               "bd_engine_step_epoch: BD_EPOCH_EXTERNAL_PLUME epochs are not covered by the stage-timing ring; "
               "turn timing off first");
    cudaStream_t st = as_stream(stream);
    const BdEngineDesc& d = e->d;
    const long long nv = (long long)d.phase.nx * d.phase.ny * d.phase.nz;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    BD_CUDA(cudaStreamIsCapturing(st, &cap));
    e->timed = (cap == cudaStreamCaptureStatusNone);
    // stage graphs unless asked not to, or the caller is itself capturing into a graph
    const bool graphs = !(options & BD_EPOCH_NO_GRAPH) && e->timed;
    k_epoch_begin<<<1, 32, 0, st>>>(e->dyn, d.dt_epoch);
    BD_CHECK_LAUNCH("k_epoch_begin");
    ++e->epochs_enqueued;
    mark(e, st, 0);

    const bool laser = power > 0.0f;
    int rc = BD_OK;
    const bool plume = d.n_substeps > 0 && d.has_plume_transport && !external;
    const bool conc = plume && e->side && !(options & BD_EPOCH_SERIAL_PLUME);
    auto plume_stage = [&](cudaStream_t on) -> int {
        return run_stage(e, e->g_plume, &d.plume, sizeof(d.plume), graphs, on, [&](cudaStream_t s) -> int {
            int in_b = 0;
            int r = plume_launch(&d.plume, d.phase.plume, d.plume_alt, d.n_substeps, d.phase.flags, &in_b, s,
                                 &e->dyn->void_zlimit, 0, e->plume_mask);
            if (r) return r;
            if (in_b)
                BD_CUDA(cudaMemcpyAsync(d.phase.plume, d.plume_alt, sizeof(float) * nv, cudaMemcpyDeviceToDevice, s));
            return BD_OK;
        });
    };
    // ring slots 1..3 (after MC, after substeps, after plume) are reserved up front when the plume
    // runs concurrently, so the ring keeps its per-epoch order
    cudaEvent_t r_mc = nullptr, r_sub = nullptr, r_pl = nullptr;
    if (conc) {
        if (e->ring_on && e->timed) {
            r_mc = ring_event(e);
            r_sub = ring_event(e);
            r_pl = ring_event(e);
            e->ring_concurrent = true;
        }
        BD_CUDA(cudaEventRecord(e->ev_fork, st));
        BD_CUDA(cudaStreamWaitEvent(e->side, e->ev_fork, 0));
        rc = plume_stage(e->side);
        if (rc) return rc;
        if (r_pl) cudaEventRecord(r_pl, e->side);
        BD_CUDA(cudaEventRecord(e->ev_join, e->side));
    } else if (e->ring_on && e->timed) {
        e->ring_concurrent = false;
    }
    if (laser && !(options & BD_EPOCH_SKIP_MC)) {
        BD_REQUIRE(d.phase.props != nullptr, "bd_engine_step_epoch: MC needs the packed property buffer");
        BdMcParams mp = d.mc;
        mp.photon_offset = 0;  // the epoch's offset (epoch << 32) is read from device memory
        rc = run_stage(e, e->g_mc, &mp, sizeof(mp), graphs, st, [&](cudaStream_t s) -> int {
            BD_CUDA(cudaMemsetAsync(d.A, 0, sizeof(float) * nv, s));
            if (d.L && (d.mc.options & BD_MC_TALLY_FLUENCE)) BD_CUDA(cudaMemsetAsync(d.L, 0, sizeof(float) * nv, s));
            return mc_launch(&mp, d.phase.props, d.phase.flags, d.A, d.L, d.lat_depth, e->dyn->ledger, e->queue,
                             e->partials, e->partial_blocks, e->sm_count, s, &e->dyn->mc_offset, e->tally64);
        });
        if (rc) return rc;
    }
    if (conc) {
        if (e->timed) cudaEventRecord(e->ev[1], st);
        if (r_mc) cudaEventRecord(r_mc, st);
    } else {
        mark(e, st, 1);
    }
    if (d.n_substeps > 0) {
        BdAblationParams ap = d.substep;
        ap.is_active = laser ? 1 : 0;
        ap.q_scale = (laser && d.mc.n_photons > 0)
                         ? (float)((double)power / ((double)d.mc.n_photons * d.voxel_volume)) : 0.0f;
        ap.zero_src_in_ablated = 1;
        rc = run_stage(e, laser ? e->g_sub_on : e->g_sub_off, &ap, sizeof(ap), graphs, st, [&](cudaStream_t s) -> int {
            int r = ablation_launch(&ap, d.phase.T, d.T_alt, d.n_substeps, d.phase.H_acc, d.omega, d.phase.chi,
                                    d.phase.flags, d.A, d.phase.k, d.phase.rho_cp, s, &e->dyn->err);
            if (r) return r;
            if (d.n_substeps & 1)
                BD_CUDA(cudaMemcpyAsync(d.phase.T, d.T_alt, sizeof(float) * nv, cudaMemcpyDeviceToDevice, s));
            return BD_OK;
        });
        if (rc) return rc;
    }
    if (conc) {
        if (r_sub) cudaEventRecord(r_sub, st);
        BD_CUDA(cudaStreamWaitEvent(st, e->ev_join, 0));
        if (e->timed) cudaEventRecord(e->ev[2], st);
    } else {
        mark(e, st, -1);
        if (plume) {
            rc = plume_stage(st);
            if (rc) return rc;
        }
        mark(e, st, 2);
    }
    if (external) return BD_OK;  // the caller runs the plume stage, then bd_engine_epoch_finish
    rc = run_stage(e, e->g_end, &e->pa, sizeof(e->pa), graphs, st, [&](cudaStream_t s) -> int {
        return phase_launch(e->pa, BD_PHASE_FULL, s);
    });
    if (e->timed) cudaEventRecord(e->ev[3], st);
    if (e->ring_on && e->timed) {
        cudaEvent_t ev = ring_event(e);
        if (ev) cudaEventRecord(ev, st);
    }
    return rc;
}

extern "C" int bd_engine_record(BdEngine* e, const BdRecordSpec* s, void* slot, void* stream) {
    BD_REQUIRE(e && s && slot, "bd_engine_record: NULL argument");
    const BdPhaseDesc& p = e->d.phase;
    BD_REQUIRE(s->y >= 0 && s->y < p.ny, "bd_engine_record: slice y=%d outside 0..%d", s->y, p.ny - 1);
    BD_REQUIRE(s->k_surface >= 0 && s->k_surface <= p.nz, "bd_engine_record: bad k_surface");
    BD_REQUIRE(((uintptr_t)slot & 15) == 0, "bd_engine_record: slot must be 16-byte aligned");
    RecordArgs a{};
    a.nx = p.nx; a.ny = p.ny; a.nz = p.nz; a.y = s->y; a.k_surface = s->k_surface;
    a.gap_k0 = s->gap_k0; a.gap_k1 = s->gap_k1;
    for (int b = 0; b < 3; ++b) { a.band_k0[b] = s->band_k0[b]; a.band_k1[b] = s->band_k1[b]; }
    a.q_scale = s->q_scale; a.plume_ratio_a = s->plume_ratio_a;
    a.T = p.T; a.H = p.H_acc; a.chi = p.chi; a.A = e->d.A; a.flags = p.flags;
    a.mu_ext = p.has_plume ? p.mu_ext : nullptr;
    return record_launch(a, e->dyn, e->d.plume.dz, slot, as_stream(stream));
}

extern "C" int bd_engine_set_plume_optics(BdEngine* e, float mu_max, float ratio_a, float ratio_s, float delta_mu) {
    BD_REQUIRE(e != nullptr, "bd_engine_set_plume_optics: NULL engine");
    BD_REQUIRE(e->d.phase.has_plume, "bd_engine_set_plume_optics: engine has no plume");
    BD_REQUIRE(mu_max >= 0.f && ratio_a >= 0.f && ratio_s >= 0.f && delta_mu >= 0.f,
               "bd_engine_set_plume_optics: values must be >= 0");
    e->d.phase.plume_mu_max = mu_max; e->d.phase.plume_ratio_a = ratio_a;
    e->d.phase.plume_ratio_s = ratio_s; e->d.phase.plume_delta_mu = delta_mu;
    e->pa.mu_max = mu_max; e->pa.ratio_a = ratio_a; e->pa.ratio_s = ratio_s; e->pa.delta_mu = delta_mu;
    return BD_OK;
}

extern "C" int bd_engine_refresh_props(BdEngine* e, void* stream) {
    BD_REQUIRE(e != nullptr, "bd_engine_refresh_props: NULL engine");
    return phase_launch(e->pa, BD_PHASE_PROPS, as_stream(stream));
}

extern "C" int bd_engine_set_mc(BdEngine* e, const BdMcParams* mc) {
    BD_REQUIRE(e && mc, "bd_engine_set_mc: NULL argument");
    BD_REQUIRE(mc->nx == e->d.phase.nx && mc->ny == e->d.phase.ny && mc->nz == e->d.phase.nz,
               "bd_engine_set_mc: grid differs from the engine's");
    BD_REQUIRE(mc->n_photons >= 0 && mc->n_photons <= kTallyMaxPhotons,
               "bd_engine_set_mc: photons per epoch must be 0..%lld", (long long)kTallyMaxPhotons);
    e->d.mc = *mc;
    return BD_OK;
}

extern "C" int bd_engine_timing(BdEngine* e, int enable) {
    BD_REQUIRE(e != nullptr, "bd_engine_timing: NULL engine");
    e->ring_on = enable != 0;
    e->ring_used = 0;
    e->ring_error = 0;
    return BD_OK;
}

extern "C" int bd_engine_timing_read(BdEngine* e, double* stage_ms, int64_t* epochs) {
    BD_REQUIRE(e && stage_ms && epochs, "bd_engine_timing_read: NULL argument");
    if (e->ring_error) return fail(BD_ERR_OUT_OF_MEMORY, "bd_engine_timing_read: event creation failed");
    for (int q = 0; q < 4; ++q) stage_ms[q] = 0.0;
    const size_t n = e->ring_used / 5;
    *epochs = (int64_t)n;
    if (n == 0) return BD_OK;
    BD_CUDA(cudaEventSynchronize(e->ring[e->ring_used - 1]));
    for (size_t ep = 0; ep < n; ++ep) {
        cudaEvent_t* r = &e->ring[ep * 5];  // begin, after MC, after substeps, after plume, after end
        float ms[4] = {0.f, 0.f, 0.f, 0.f};
        BD_CUDA(cudaEventElapsedTime(&ms[0], r[0], r[1]));
        BD_CUDA(cudaEventElapsedTime(&ms[1], r[1], r[2]));
        if (e->ring_concurrent) {
            // the plume ran beside MC + substeps from the epoch begin; the epoch end starts after both
            float a = 0.f, b = 0.f;
            BD_CUDA(cudaEventElapsedTime(&ms[2], r[0], r[3]));
            BD_CUDA(cudaEventElapsedTime(&a, r[2], r[4]));
            BD_CUDA(cudaEventElapsedTime(&b, r[3], r[4]));
            ms[3] = std::min(a, b);
        } else {
            BD_CUDA(cudaEventElapsedTime(&ms[2], r[2], r[3]));
            BD_CUDA(cudaEventElapsedTime(&ms[3], r[3], r[4]));
        }
        for (int q = 0; q < 4; ++q) stage_ms[q] += ms[q];
    }
    return BD_OK;
}

extern "C" int bd_engine_epoch_finish(BdEngine* e, void* stream) {
    BD_REQUIRE(e != nullptr, "bd_engine_epoch_finish: NULL engine");
    cudaStream_t st = as_stream(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    BD_CUDA(cudaStreamIsCapturing(st, &cap));
    const bool graphs = cap == cudaStreamCaptureStatusNone;
    int rc = run_stage(e, e->g_end, &e->pa, sizeof(e->pa), graphs, st, [&](cudaStream_t s) -> int {
        return phase_launch(e->pa, BD_PHASE_FULL, s);
    });
    if (rc == BD_OK && e->timed) cudaEventRecord(e->ev[3], st);
    return rc;
}

// Several engines' plume stages as one batched stage (one launch per FTCS step for all of them).
struct BdPlumeBatch {
    std::vector<BdEngine*> eng;
    std::vector<bd::PlumeInstHost> host;
    std::vector<int> order;
    void* dev = nullptr;             // device descriptors, ranked by step count
    unsigned* units = nullptr;
    long long max_steps = 0;
    cudaStream_t cap_stream = nullptr;
    StageGraph g;
};

extern "C" int bd_plume_batch_create(BdEngine* const* engines, int n, BdPlumeBatch** out) {
    BD_REQUIRE(engines && out, "bd_plume_batch_create: NULL argument");
    BD_REQUIRE(n >= 1 && n <= 32, "bd_plume_batch_create: 1..32 engines, got %d", n);
    const BdEngine* e0 = engines[0];
    BD_REQUIRE(e0 != nullptr, "bd_plume_batch_create: NULL engine");
    const BdPlumeParams& p0 = e0->d.plume;
    for (int i = 0; i < n; ++i) {
        const BdEngine* e = engines[i];
        BD_REQUIRE(e != nullptr, "bd_plume_batch_create: engine %d is NULL", i);
        BD_REQUIRE(e->d.has_plume_transport && e->d.n_substeps > 0,
                   "bd_plume_batch_create: engine %d has no plume transport", i);
        const BdPlumeParams& p = e->d.plume;
        BD_REQUIRE(p.nx == p0.nx && p.ny == p0.ny && p.nz == p0.nz && p.dx == p0.dx && p.dy == p0.dy && p.dz == p0.dz,
                   "bd_plume_batch_create: engine %d has another grid", i);
        BD_REQUIRE(p.nz % 4 == 0 && p.nz <= 1020, "bd_plume_batch_create: needs nz %% 4 == 0 and nz <= 1020");
    }
    BdPlumeBatch* b = new BdPlumeBatch();
    b->order.resize(n);
    for (int i = 0; i < n; ++i) {
        BdEngine* e = engines[i];
        b->eng.push_back(e);
        b->host.push_back(bd::PlumeInstHost{e->d.phase.plume, e->d.plume_alt, e->plume_mask, e->d.phase.flags,
                                            &e->dyn->void_zlimit, &e->d.plume, e->d.n_substeps});
    }
    cudaError_t err = cudaMalloc(&b->dev, bd::plume_batch_desc_bytes(n));
    if (err == cudaSuccess)
        err = cudaMalloc((void**)&b->units, sizeof(unsigned) * bd::plume_batch_units_words(n, p0.nx, p0.ny, p0.nz));
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    int rc = err == cudaSuccess ? BD_OK : cuda_status(err, "bd_plume_batch_create");
    if (rc == BD_OK) rc = bd::plume_batch_prepare(n, b->host.data(), b->dev, b->order.data(), &b->max_steps);
    if (rc != BD_OK) {
        if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
        cudaFree(b->dev);
        cudaFree(b->units);
        delete b;
        return rc;
    }
    *out = b;
    return BD_OK;
}

extern "C" int bd_plume_batch_run(BdPlumeBatch* b, void* stream) {
    BD_REQUIRE(b != nullptr, "bd_plume_batch_run: NULL batch");
    cudaStream_t st = as_stream(stream);
    const int n = (int)b->eng.size();
    auto enqueue = [&](cudaStream_t s) -> int {
        return bd::plume_batch_launch(n, b->host.data(), b->order.data(), b->dev, b->max_steps, b->units, s);
    };
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    BD_CUDA(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone) return enqueue(st);
    // a captured graph, re-captured when a launch-shape knob changed
    if (!b->g.exec || b->g.tune_gen != bd::tune_generation()) {
        graph_reset(b->g);
        cudaGraph_t graph = nullptr;
        BD_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue(b->cap_stream);
        cudaError_t ce = cudaStreamEndCapture(b->cap_stream, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return cuda_status(ce, "bd_plume_batch_run: capture");
        ce = cudaGraphInstantiate(&b->g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return cuda_status(ce, "bd_plume_batch_run: instantiate");
        b->g.tune_gen = bd::tune_generation();
    }
    BD_CUDA(cudaGraphLaunch(b->g.exec, st));
    return BD_OK;
}

extern "C" int bd_plume_batch_destroy(BdPlumeBatch* b) {
    if (!b) return BD_OK;
    graph_reset(b->g);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    cudaFree(b->dev);
    cudaFree(b->units);
    delete b;
    return BD_OK;
}

extern "C" int bd_engine_epoch_end(BdEngine* e, void* stream) {
    BD_REQUIRE(e != nullptr, "bd_engine_epoch_end: NULL engine");
    cudaStream_t st = as_stream(stream);
    k_epoch_end_only<<<1, 32, 0, st>>>(e->dyn);
    BD_CHECK_LAUNCH("k_epoch_end_only");
    return phase_launch(e->pa, BD_PHASE_FULL, st);
}

extern "C" int bd_engine_read_diag(BdEngine* e, BdEpochDiag* out, void* stream) {
    BD_REQUIRE(e && out, "bd_engine_read_diag: NULL argument");
    cudaStream_t st = as_stream(stream);
    BD_CUDA(cudaMemcpyAsync(e->dyn_host, e->dyn, sizeof(EngineDyn), cudaMemcpyDeviceToHost, st));
    BD_CUDA(cudaStreamSynchronize(st));
    const EngineDyn& h = *e->dyn_host;
    for (int q = 0; q < BD_LEDGER_LEN; ++q) out->ledger[q] = h.ledger[q];
    out->epoch = (double)h.epoch;
    out->time_s = h.t;
    out->n_new = (double)h.n_new;
    out->n_ablated = h.n_ablated;
    out->gap_open = (double)h.gap_open;
    out->plume_tau = h.plume_tau_sum * (double)e->d.plume.dz;
    out->plume_peak_mu_a = (double)__builtin_bit_cast(float, h.plume_peak_bits);
    out->plume_ablated_sum = h.plume_abl_sum;
    out->n_void = (double)h.n_void;
    out->void_zlimit = (double)h.void_zlimit;
    out->t_optical_ms = out->t_thermal_ms = out->t_epoch_end_ms = 0.0;
    if (h.err) return fail(BD_ERR_TIMEOUT, "bd_engine_read_diag: a bounded device wait timed out");
    if (e->timed) {
        float a = 0, b = 0, c = 0;
        if (cudaEventElapsedTime(&a, e->ev[0], e->ev[1]) == cudaSuccess) out->t_optical_ms = a;
        if (cudaEventElapsedTime(&b, e->ev[1], e->ev[2]) == cudaSuccess) out->t_thermal_ms = b;
        if (cudaEventElapsedTime(&c, e->ev[2], e->ev[3]) == cudaSuccess) out->t_epoch_end_ms = c;
        cudaGetLastError();
    }
    return BD_OK;
}
