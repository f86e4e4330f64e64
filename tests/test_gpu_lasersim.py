"""The LaserSim generator end to end on the GPU (simulation/beetle_sim.py:201-313 semantics): one
'setup', frames at the active / cooling cadence up to the last epoch, one 'done'; each frame carries
the reference's keys, its base64 slices decode to the announced (nz, nx) grid, temperatures rise
under the laser, and the frame energies add up (absorbed + reflected + transmitted <= incident)."""
import base64

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FRAME_KEYS = {'t_ms', 'laser_on', 'progress', 'eta_s', 'Q', 'T', 'plume', 'phase', 'transmission_pct', 'core_peak',
              'core_mean', 'ventral_peak', 'ventral_mean', 'ablated_pct', 'boiled_pct', 'depth_um', 'energy_j'}


def _dec(s, dtype, shape):
    return np.frombuffer(base64.b64decode(s), dtype=dtype).reshape(shape)


def test_lasersim_run_streams_reference_events(gpu):
    from bug_defense_b200 import lasersim as ls
    setup = ls.default_setup()
    laser = dict(setup['laser'], resolution='preview', photons=20_000, pulse_ms=4.0, duration_ms=12.0, power_w=40.0)
    events = list(ls.run(setup['layers'], laser, frame_ms_active=2.0, frame_ms_cooling=5.0))
    assert events[0]['event'] == 'setup' and events[-1]['event'] == 'done'
    frames = [e['data'] for e in events[1:-1]]
    assert all(e['event'] == 'frame' for e in events[1:-1])
    s = events[0]['data']
    nxs, nzs = s['nx'], s['nz']
    assert s['grid'].startswith('100x100x') and s['voxel_um'] == 30.0 and s['photons'] == 20_000
    # the first epoch always gives a frame, then every 2 ms under the laser, 5 ms after, and the last
    assert [f['t_ms'] for f in frames] == [1.0, 3.0, 8.0, 12.0]
    assert [f['laser_on'] for f in frames] == [True, True, False, False]
    for f in frames:
        assert set(f) == FRAME_KEYS
        T = _dec(f['T'], '<f4', (nzs, nxs))
        Q = _dec(f['Q'], '<f4', (nzs, nxs))
        ph = _dec(f['phase'], 'u1', (nzs, nxs))
        pl = _dec(f['plume'], '<f4', (nzs, nxs))
        assert np.all(np.isfinite(T)) and T.min() >= 19.0 and np.all(Q >= 1e-4) and np.all(pl >= 0)
        assert set(np.unique(ph)) <= {0, 1, 2, 3} and np.all(ph[:10] == 3)     # ambient air rows
        en = f['energy_j']
        assert en['absorbed'] + en['reflected'] + en['transmitted'] <= en['incident'] + 1e-3
        assert 0.0 <= f['transmission_pct'] <= 100.0 and f['depth_um'] >= 0.0
    assert frames[1]['energy_j']['incident'] == pytest.approx(0.12)           # 3 laser epochs x 40 mJ
    assert frames[-1]['energy_j']['incident'] == pytest.approx(0.16)
    assert frames[1]['energy_j']['absorbed'] > 0.0
    assert _dec(frames[1]['T'], '<f4', (nzs, nxs)).max() > 30.0
    assert frames[-1]['progress'] == 1.0
