"""Checkpoint / resume in the layout of the framework's SimulationHistory
(tvb_framework/tvb/core/entities/file/simulator/simulation_history_h5.py:32-118):
a run resumed from a stored state continues exactly like an uninterrupted
run, and the stored fields have the reference's shapes and contents."""
import numpy as np
import pytest

import golden_util as G
from tvb_b200 import coupling, integrators, models, monitors, noise
from tvb_b200.connectivity import Connectivity
from tvb_b200.simulator import Simulator


def g2d_sim(length):
    fx = G.load('g2d_76')
    w, L = G.connectome(fx)
    np.random.seed(int(fx['ic_seed']))
    return Simulator(model=models.Generic2dOscillator(), connectivity=Connectivity(w, L, speed=float(fx['speed'])),
                     coupling=coupling.Linear(a=float(fx['coupling_a'])),
                     integrator=integrators.HeunDeterministic(dt=float(fx['dt'])),
                     monitors=[monitors.Raw(), monitors.TemporalAverage(period=1.0)],
                     simulation_length=length).configure()


def rww_sim(length):
    fx = G.load('rww_68_short')
    w, L = G.connectome(fx)
    return Simulator(model=models.ReducedWongWang(), connectivity=Connectivity(w, L, speed=float(fx['speed'])),
                     coupling=coupling.Linear(a=0.3),
                     integrator=integrators.EulerStochastic(dt=0.1, noise=noise.Additive(nsig=[1e-3])),
                     monitors=[monitors.TemporalAverage(period=10.0), monitors.Bold(period=200.0)],
                     simulation_length=length).configure()


def test_history_state_layout_matches_reference_buffers():
    """Fields and shapes of SimulationHistory; the history is the reference's
    configured history.buffer (golden fixture), and a state round-trips."""
    fx = G.load('g2d_76')
    sim = g2d_sim(150.0)
    st = sim.history_state()
    H, n = sim.connectivity.horizon, sim.number_of_nodes
    assert st['history'].shape == (H, 1, n, 1) and st['history'].dtype == np.float32
    np.testing.assert_array_equal(st['history'][..., 0], fx['buffer0'])
    assert st['current_state'].shape == (2, n, 1) and st['current_step'] == 0
    assert st['monitor_names'] == ['Raw', 'TemporalAverage']
    assert st['monitor_stock_1'].shape == () and st['monitor_stock_2'].shape == (10, 1, n, 1)
    sim2 = g2d_sim(150.0).set_history_state(st)
    st2 = sim2.history_state()
    for k in ('history', 'current_state', 'monitor_stock_2'):
        np.testing.assert_array_equal(st2[k], st[k])
    r = rww_sim(100.0).history_state()
    assert r['monitor_names'] == ['TemporalAverage', 'Bold']
    assert r['monitor_stock_2'].shape == (5000, 1, 68, 1) and r['monitor_interim_2'].shape == (1, 68, 1)
    assert r['integrator_noise_rng_state_algo'] == 'MT19937' and r['integrator_noise_rng_state_keys'].size == 624
    with pytest.raises(ValueError):
        g2d_sim(10.0).set_history_state(dict(st, history=st['history'][:-1]))


@pytest.mark.gpu
@pytest.mark.parametrize('which', ['g2d', 'rww'])
def test_resume_matches_uninterrupted_run(which):
    make = g2d_sim if which == 'g2d' else rww_sim
    first, second = (70.3, 80.0) if which == 'g2d' else (123.4, 376.6)
    whole = make(first + second)
    ref = whole.run()
    part = make(first)
    a = part.run()
    st = part.history_state()
    resumed = make(second).set_history_state(st)
    b = resumed.run()
    assert resumed.current_step == whole.current_step
    for (ta, ya), (tb, yb), (tr, yr) in zip(a, b, ref):
        # a part without samples returns empty arrays, as the reference's run() does
        np.testing.assert_array_equal(np.concatenate([t for t in (ta, tb) if t.size]), tr)
        np.testing.assert_array_equal(np.concatenate([y for y in (ya, yb) if y.size]), yr)
    np.testing.assert_array_equal(resumed.history_buffer, whole.history_buffer)


@pytest.mark.gpu
def test_region_major_rings_resume_exactly():
    """A large Epileptor network (998 regions) runs on the cluster kernel's blocked edge runs with region-major
    rings; two run() calls -- the second re-uploads the history exported after the first -- give the bits of
    one uninterrupted run, and the exported history has the reference's time-major layout."""
    from tvb_b200 import synthetic

    def make(length):
        w, L = synthetic.connectome(998, 0.10, 5.0, 300.0, seed=4)
        x0 = np.random.default_rng(14).uniform(-2.4, -1.6, 998)
        np.random.seed(15)
        return Simulator(model=models.Epileptor(x0=x0, Ks=np.array([-0.2]), Kf=np.array([0.05])),
                         connectivity=Connectivity(w, L, speed=3.0), coupling=coupling.Difference(),
                         integrator=integrators.HeunDeterministic(dt=0.05),
                         monitors=[monitors.TemporalAverage(period=1.0)], simulation_length=length).configure()
    whole = make(20.0)
    h0 = whole.history_buffer.copy()
    spec, kind = whole.instance_spec(400)
    from tvb_b200.engine import Batch
    plan = Batch(whole._model_id, whole._cfun_id, whole._scheme_id, kind, 0.05, whole._voi_codes, [spec],
                 allocate=False)
    assert plan.cluster >= 2 and plan.ring_layout == 1 and plan.sync_every % 4 == 0
    (t, y), = whole.run()
    parts = make(20.0)
    np.testing.assert_array_equal(parts.history_buffer, h0)
    (t1, y1), = parts.run(n_steps=147)   # the first call ends inside a block of four steps
    assert parts.history_buffer.shape == h0.shape
    (t2, y2), = parts.run(n_steps=253)
    np.testing.assert_array_equal(np.concatenate([t1, t2]), t)
    np.testing.assert_array_equal(np.concatenate([y1, y2]), y)
    np.testing.assert_array_equal(parts.current_state, whole.current_state)
