"""Region stimulus host logic (CPU): the temporal equations and the spatial
pattern against the reference's own arrays, the stimulus slice handed to the
device, and the argument checks.  The device runs are in test_gpu_parity.py."""
import numpy as np
import pytest

import golden_util as G

EQS = {
    'g2d_pulse': ('PulseTrain', {'T': 12.0, 'tau': 4.0, 'amp': 2.0, 'onset': 5.0}, 0.1, 60.0),
    'g2d_w_sin': ('Sinusoid', {'amp': 0.5, 'frequency': 0.05}, 0.1, 40.0),
    'rww_alpha': ('Alpha', {'onset': 3.0, 'alpha': 0.5, 'beta': 1.0}, 0.1, 40.0),
    'epi_gauss': ('Gaussian', {'amp': 1.5, 'sigma': 4.0, 'midpoint': 10.0, 'offset': 0.0}, 0.05, 20.0),
}


@pytest.mark.parametrize('case', sorted(EQS))
def test_temporal_and_spatial_patterns_match_reference(case):
    """equations.py:150-364 and patterns.py:41-186: the pattern arrays the reference's StimuliRegion made."""
    from tvb_b200 import equations
    from tvb_b200.patterns import StimuliRegion
    fx = G.load('stimulus_40')
    name, params, dt, length = EQS[case]
    stim = StimuliRegion(temporal=equations.EQUATIONS[name](params), weight=fx['stim_weight'])
    stim.configure_space()
    stim.configure_time(np.r_[0.0:length:dt].reshape((1, -1)))
    np.testing.assert_allclose(stim.temporal_pattern.reshape(-1), fx[case + '_temporal'], rtol=1e-15, atol=1e-15)
    np.testing.assert_array_equal(stim.spatial_pattern.reshape(-1), fx[case + '_spatial'])
    k = 7
    np.testing.assert_allclose(stim(k), stim.spatial_pattern * stim.temporal_pattern[0, k], rtol=0, atol=0)


def test_other_equations_defaults():
    """Defaults and shapes of the equations the golden runs do not use."""
    from tvb_b200 import equations as E
    t = np.linspace(0.0, 50.0, 11)
    np.testing.assert_allclose(E.Linear().evaluate(t), t)
    np.testing.assert_allclose(E.Cosine().evaluate(t), np.cos(2 * np.pi * 0.01 * t))
    np.testing.assert_allclose(E.GeneralizedSigmoid().evaluate(np.array([1.0])), [0.5])
    np.testing.assert_allclose(E.Sigmoid().evaluate(np.array([5.0])), [0.5])
    dg = E.DoubleGaussian().evaluate(np.array([0.0]))
    np.testing.assert_allclose(dg, [-0.5])
    np.testing.assert_array_equal(E.DiscreteEquation().evaluate(np.array([[2.0], [3.0]])), [[2.0], [3.0]])
    a = E.Alpha().evaluate(np.array([0.0, 0.5, 1.0]))
    assert a[0] == 0.0 and a[1] == 0.0 and a[2] > 0.0
    p = E.PulseTrain().evaluate(np.array([30.0, 31.0, 43.0, 44.0, 72.0, 73.0]))
    np.testing.assert_array_equal(p, [0, 1, 0, 0, 1, 1])


def _sim(stimulus, length=10.0, model=None):
    from tvb_b200 import coupling, integrators, models, monitors, synthetic
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.simulator import Simulator
    w, L = synthetic.connectome(12, 0.5, 5.0, 30.0, seed=1)
    np.random.seed(3)
    return Simulator(model=model or models.Generic2dOscillator(), connectivity=Connectivity(w, L, speed=3.0),
                     coupling=coupling.Linear(a=0.01), integrator=integrators.HeunDeterministic(dt=0.1),
                     monitors=[monitors.Raw()], simulation_length=length, stimulus=stimulus).configure()


def test_stimulus_spec_slices_the_run():
    """Step s of a run reads temporal index s - (current_step + 1) (simulator.py:301-306); a chunk starting
    later in the same run reads further along the same grid."""
    from tvb_b200.equations import Linear
    from tvb_b200.patterns import StimuliRegion
    w = np.linspace(0.0, 1.0, 12)
    sim = _sim(StimuliRegion(temporal=Linear({'a': 1.0, 'b': 0.0}), weight=w))
    sim._prepare_stimulus()
    st = sim.stimulus_spec(100)
    np.testing.assert_allclose(st['temporal'], np.r_[0.0:10.0:0.1][:100])
    np.testing.assert_array_equal(st['weight'], w)
    np.testing.assert_array_equal(st['vars'], [0])      # stvar defaults to cvar
    sim.current_step += 40                                 # next chunk of the same call
    np.testing.assert_allclose(sim.stimulus_spec(60)['temporal'], np.r_[0.0:10.0:0.1][40:100])
    with pytest.raises(IndexError):
        sim.stimulus_spec(61)


def test_instance_spec_mask_and_checks():
    from tvb_b200.engine import Connectome, InstanceSpec
    from tvb_b200 import _lib
    n = 4
    w = np.ones((n, n)) - np.eye(n)
    idl, H = _lib.idelays(np.full((n, n), 10.0), 3.0, 0.1)
    conn = Connectome(w, idl, 1)
    ring0 = np.zeros((H, 1, n), np.float32)
    base = dict(conn=conn, ring0=ring0, state0=np.zeros((2, n)), params=np.zeros((12, n), np.float32),
                cfun=[0.1, 0.0], n_steps=5)
    s = InstanceSpec(**base, stim=dict(temporal=np.arange(8.0), weight=np.ones(n), vars=[0, 1]))
    assert s.stim['mask'] == 3 and s.stim['temporal'].size == 5 and s.stim['temporal'].dtype == np.float32
    with pytest.raises(IndexError):
        InstanceSpec(**base, stim=dict(temporal=np.arange(4.0), weight=np.ones(n), vars=[0]))
    with pytest.raises(ValueError):
        InstanceSpec(**base, stim=dict(temporal=np.arange(8.0), weight=np.ones(n + 1), vars=[0]))


def test_bad_stvar_and_stimulus_kind_rejected():
    from tvb_b200 import models
    from tvb_b200.patterns import StimuliRegion
    m = models.Generic2dOscillator()
    m.stvar = np.array([2])
    with pytest.raises(ValueError):
        _sim(StimuliRegion(weight=np.ones(12)), model=m)

    class StimuliSurface:
        pass
    with pytest.raises(NotImplementedError):
        _sim(StimuliSurface())
