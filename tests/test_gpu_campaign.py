"""Launch-shape knobs and the batched campaign on the GPU.

Absorbed-weight tallies are exact 64-bit fixed point and every other kernel is deterministic, so
neither the launch shapes nor running instances concurrently may change a single bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _knob(k, v=None):
    import ctypes
    from bug_defense_b200 import _lib
    if v is None:
        out = ctypes.c_int(0)
        _lib.call("bd_tune_get", k, ctypes.byref(out))
        return out.value
    _lib.call("bd_tune_set", k, int(v))


@pytest.fixture
def restore_knobs(gpu):
    from bug_defense_b200 import _lib
    keep = {k: _knob(k) for k in (_lib.TUNE_MC_BLOCKS_PER_SM, _lib.TUNE_STENCIL_XC, _lib.TUNE_PLUME_XC,
                                  _lib.TUNE_PLUME_KERNEL, _lib.TUNE_STENCIL_CAP)}
    yield
    for k, v in keep.items():
        _knob(k, v)


def test_knob_validation(gpu, restore_knobs):
    from bug_defense_b200 import _lib
    with pytest.raises(ValueError):
        _knob(_lib.TUNE_STENCIL_XC, 0)
    with pytest.raises(ValueError):
        _knob(_lib.TUNE_MC_BLOCKS_PER_SM, 17)
    for bad in (0, 3, 5, 7):
        with pytest.raises(ValueError):
            _knob(_lib.TUNE_PLUME_KERNEL, bad)
    for bad in (-1, 17):
        with pytest.raises(ValueError):
            _knob(_lib.TUNE_STENCIL_CAP, bad)
    with pytest.raises(ValueError):
        _knob(7, 1)


def test_launch_shapes_leave_results_bit_identical(gpu, restore_knobs):
    from bug_defense_b200 import _lib, thermal
    rng = np.random.default_rng(5)
    n = (24, 20, 36)
    T0 = 25 + 50 * rng.random(n); Q = rng.random(n) * 1e-3
    K = 1e-4 + 5e-4 * rng.random(n); R = 2e-3 + 2e-3 * rng.random(n)
    outs = []
    for xc, cap in ((4, 0), (8, 1), (16, 2), (1, 0)):
        _knob(_lib.TUNE_STENCIL_XC, xc)
        _knob(_lib.TUNE_STENCIL_CAP, cap)
        outs.append(thermal.run_thermal3d_substeps_gpu(T0, Q, K, R, *n, 0.015, 0.015, 0.015, 5e-5, 9, h_eff=2e-5,
                                                       t_ambient=25.0, is_active=1))
    assert all(np.array_equal(outs[0], o) for o in outs[1:])
    cube = {k: np.full((16, 16, 20), v) for k, v in (("mu_a", 2.0), ("mu_s", 15.0), ("g", 0.85), ("n", 1.4))}
    kw = dict(n_photons=60_000, base_seed=77, Lx=0.24, Ly=0.24, Lz=0.3, Nx=16, Ny=16, Nz=20, custom_3d_props=cube,
              spot_dia=0.1)
    maps = []
    for blocks in (0, 2, 5):
        _knob(_lib.TUNE_MC_BLOCKS_PER_SM, blocks)
        maps.append(gpu.run_voxel_mc3d(**kw)["A_3d"])
    assert np.array_equal(maps[0], maps[1]) and np.array_equal(maps[0], maps[2])


def test_plume_kernel_shapes_leave_results_bit_identical(gpu, restore_knobs):
    """Every plume kernel gives the same bits: the direct kernel in both unit orders (grid over the
    z-list columns with several x-chunk lengths, and the compact unit list), through the context API
    (arbitrary values in non-void voxels, ragged y tiles, scattered void, a partly filled last z
    tile, deep cavities under trimmed and empty columns) and through the engine (void z-limit, partly
    void voxel groups at the crater walls, bulk-void fast path)."""
    from bug_defense_b200 import _lib, campaign
    rng = np.random.default_rng(11)
    scattered = rng.uniform(size=(9, 35, 68)) < 0.7
    slab = np.zeros((12, 70, 96), bool)                 # bulk void above z = 50, scattered pores below
    slab[:, :, :50] = True
    slab |= rng.uniform(size=slab.shape) < 0.1
    cavity = np.zeros((12, 70, 132), bool)              # deep z tiles void only in a small cavity, the
    cavity[:, :, :40] = True                            # deepest none: trimmed and empty columns
    cavity[3:7, 20:41, 70:101] = True
    cavity8 = np.zeros((11, 37, 136), bool)             # last 32-voxel z tile 8 deep, ragged y tiles
    cavity8[:, :, :44] = True
    cavity8[2:9, 5:30, 60:131] = rng.uniform(size=(7, 25, 71)) < 0.8
    for vd in (scattered, slab, cavity, cavity8):
        shape = vd.shape
        C0 = (rng.uniform(0, 1, shape) * vd).astype(np.float32)
        z = np.zeros(shape)
        fields = []
        for kern, xc in ((4, 2), (4, 1), (4, 3), (4, 4), (6, 4)):
            _knob(_lib.TUNE_PLUME_KERNEL, kern)
            _knob(_lib.TUNE_PLUME_XC, xc)
            ctx = gpu.MetalAblationContext(*shape, 0.03, 0.025, 0.02, 1e-5, 0.0, 20.0, 100.0, 300.0,
                                           plume_params={'D_xy': 1.5, 'D_z': 2.5, 'vz': 4.0, 'tau_linger': 0.02},
                                           plume_dt_policy='as_given')
            ctx.set_state(np.full(shape, 20.0), z, z, z, np.zeros(shape, np.uint8), np.zeros(shape, np.uint8), z,
                          z, np.full(shape, 1e-3), plume=C0, plume_void=vd)
            ctx.advance_substeps(7, is_active=0)
            fields.append(ctx.get_plume())
        for f in fields[1:]:
            assert np.array_equal(f, fields[0])
        assert np.any(fields[0] != C0)
    inst = _small(22)                                  # 2940 nm, 80 W: a crater opens
    runs = []
    for kern in (4, 6):
        _knob(_lib.TUNE_PLUME_KERNEL, kern)
        camp = campaign.Campaign([inst])
        camp.run(14, sync_every=14)
        e = camp.engines[0]
        runs.append((e.T.copy(), e.plume.raw.double().cpu().numpy(), e.ablated.copy()))
    assert runs[0][2].sum() > 0 and np.any(runs[0][1] > 0)
    for r in runs[1:]:
        assert all(np.array_equal(a, b) for a, b in zip(r, runs[0]))


def test_concurrent_plume_stage_equals_serial(gpu, restore_knobs):
    """With the per-step plume kernel the plume stage runs on its own stream beside MC + substeps;
    within an epoch the stages share no data, so running it after the substeps on one stream gives
    the same bits. The stage-timing ring stays readable in both modes."""
    import ctypes
    from bug_defense_b200 import _lib, campaign
    _knob(_lib.TUNE_PLUME_KERNEL, _lib.PLUME_KERNEL_DIRECT)
    inst = _small(22)                                  # 2940 nm, 80 W: a crater opens, plume injected
    runs = []
    for serial in (True, False):
        eng = campaign.make_engine(inst)
        eng.serial_plume = serial
        eng.power = eng.laser_power
        _lib.call("bd_engine_timing", eng._handle, 1)
        eng.step_epochs(8)
        ms = (ctypes.c_double * 4)()
        n = ctypes.c_int64(0)
        _lib.call("bd_engine_timing_read", eng._handle, ms, ctypes.byref(n))
        _lib.call("bd_engine_timing", eng._handle, 0)
        assert n.value == 8 and all(v >= 0.0 for v in ms[:]) and ms[2] > 0.0
        eng.power = 0.0
        eng.step_epochs(6)
        runs.append((eng.T.copy(), eng.plume.raw.double().cpu().numpy(), eng.ablated.copy(), eng.H_acc.copy()))
    assert runs[0][2].sum() > 0 and np.any(runs[0][1] > 0)
    assert all(np.array_equal(a, b) for a, b in zip(runs[0], runs[1]))


def _small(index, photons=20_000):
    from bug_defense_b200 import campaign
    inst = campaign.campaign_instances(1, grid=(24, 24, 128), n_plume_air=8)[index]
    return dict(inst, n_photons=photons, pulse_ms=12.0)


@pytest.mark.parametrize("kern,batch", [(4, True), (4, False), (6, False)],
                         ids=["batched-plume", "direct-streams", "compact-streams"])
def test_concurrent_campaign_equals_instances_run_alone(gpu, restore_knobs, kern, batch):
    """Instances run together give the bits of each instance run alone with its own plume stage:
    with the batched plume stage (one launch per FTCS step over every instance's units), and with
    each instance's stages on its own stream (direct and compact plume kernels)."""
    from bug_defense_b200 import _lib, campaign
    _knob(_lib.TUNE_PLUME_KERNEL, kern)
    insts = [_small(i) for i in (1, 10, 23)]           # 532, 1064 and 2940 nm
    camp = campaign.Campaign(insts, batch_plume=batch)
    assert (camp.batch is not None) == batch
    camp.run(30, sync_every=10)
    together = [(e.T.copy(), e.ablated.copy(), e.H_acc.copy(), e.plume.raw.double().cpu().numpy())
                for e in camp.engines]
    camp.close()
    for inst, (T, abl, H, C) in zip(insts, together):
        solo = campaign.Campaign([inst], batch_plume=False)
        solo.run(30, sync_every=30)
        e = solo.engines[0]
        assert np.array_equal(e.T, T) and np.array_equal(e.ablated, abl) and np.array_equal(e.H_acc, H)
        assert np.array_equal(e.plume.raw.double().cpu().numpy(), C)
    # the lasers did work: every instance heated up, the 2940 nm one ablated
    assert all(float(T.max()) > 40.0 for T, _, _, _ in together)
    assert together[2][1].sum() > together[0][1].sum() and np.any(together[2][3] > 0)


def test_autotune_sets_the_fastest_candidates(gpu, restore_knobs):
    from bug_defense_b200 import _lib, campaign
    res = campaign.autotune(_small(4), epochs_per_trial=2,
                            candidates={_lib.TUNE_MC_BLOCKS_PER_SM: [2, 4], _lib.TUNE_STENCIL_XC: [4, 8],
                                        _lib.TUNE_PLUME_KERNEL: [4, 6], _lib.TUNE_PLUME_XC: [2, 4],
                                        _lib.TUNE_STENCIL_CAP: [0, 2]})
    for name, knob in (("mc_ctas_per_sm", _lib.TUNE_MC_BLOCKS_PER_SM), ("stencil_xc", _lib.TUNE_STENCIL_XC),
                       ("stencil_cap", _lib.TUNE_STENCIL_CAP)):
        trials = res["trials"][name]
        assert [v for v, _ in trials] == sorted(v for v, _ in trials) and all(t > 0 for _, t in trials)
        assert res[name] == min(trials, key=lambda t: t[1])[0] == _knob(knob)
    # the plume kernel and the direct kernel's x-planes are searched together; the compact kernel
    # picks its x-planes per stage
    plume = res["trials"]["plume"]
    assert [(k, x) for k, x, _ in plume] == [(4, 2), (4, 4), (6, None)]
    assert all(t > 0 for _, _, t in plume)
    k, x, _ = min(plume, key=lambda t: t[2])
    assert res["plume_kernel"] == k == _knob(_lib.TUNE_PLUME_KERNEL)
    assert res["plume_xc"] == _knob(_lib.TUNE_PLUME_XC) and (x is None or res["plume_xc"] == x)
