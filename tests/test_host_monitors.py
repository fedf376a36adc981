"""Host-side monitor logic (CPU): the AfferentCouplingTemporalAverage
reduction of an every-step coupling stream, used when AfferentCoupling
monitors of different periods share a run."""
import numpy as np


def _device_rule(raw, s0, istep, carry):
    """The device's arithmetic: float32 running sum from the carry, divided by
    istep at every step that is a multiple of istep."""
    acc = carry.copy()
    out = []
    for k in range(raw.shape[0]):
        acc = acc + raw[k]
        if (s0 + 1 + k) % istep == 0:
            out.append(acc / np.float32(istep))
            acc = np.zeros_like(acc)
    return (np.stack(out) if out else np.zeros((0,) + raw.shape[1:], np.float32)), acc


def test_afferent_average_matches_the_device_rule_across_chunks():
    from tvb_b200.monitors import AfferentCouplingTemporalAverage
    rng = np.random.default_rng(0)
    m = AfferentCouplingTemporalAverage(period=1.0)
    for istep in (1, 3, 10):
        m.istep = istep
        raw = rng.normal(size=(257, 2, 5)).astype(np.float32)
        for cuts in ([257], [7, 100, 150], [1, 1, 255], [13, 244]):
            carry_m = carry_d = np.zeros((2, 5), np.float32)
            s0 = 4
            got, want = [], []
            for a, b in zip(np.cumsum([0] + cuts[:-1]), np.cumsum(cuts)):
                y, carry_m = m.average(raw[a:b], s0 + a, carry_m)
                z, carry_d = _device_rule(raw[a:b], s0 + a, istep, carry_d)
                got.append(y)
                want.append(z)
            np.testing.assert_array_equal(np.concatenate(got), np.concatenate(want))
            np.testing.assert_array_equal(carry_m, carry_d)


def _projection_setup(fx):
    from tvb_b200 import monitors, sensors
    from tvb_b200.sensors import ProjectionSurfaceEEG, ProjectionSurfaceMEG, ProjectionSurfaceSEEG, RegionMapping

    def labels(k, S):
        return ['%s%d' % (k, i) for i in range(S)]
    eeg = monitors.EEG(period=1e3 / 1024.0, sensors=sensors.SensorsEEG(labels('e', 16), fx['sensors_eeg']),
                       projection=ProjectionSurfaceEEG(fx['lead_eeg']), region_mapping=RegionMapping(fx['rmap']),
                       reference='average')
    meg = monitors.MEG(period=1e3 / 1024.0, sensors=sensors.SensorsMEG(labels('m', 12), fx['sensors_meg']),
                       projection=ProjectionSurfaceMEG(fx['lead_meg']), region_mapping=RegionMapping(fx['rmap']),
                       obsnoise=None)
    ieeg = monitors.iEEG(period=2.0, sensors=sensors.SensorsInternal(labels('i', 10), fx['sensors_ieeg']),
                         projection=ProjectionSurfaceSEEG(fx['lead_ieeg']), region_mapping=RegionMapping(fx['rmap']))
    return eeg, meg, ieeg


def _sim(fx, mons, cortical):
    from tvb_b200 import coupling, integrators, models
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.simulator import Simulator
    conn = Connectivity(fx['weights'], fx['tract_lengths'], speed=float(fx['speed']), centres=fx['centres'],
                        orientations=fx['orientations'], cortical=fx['cortical'] if cortical else None)
    return Simulator(model=models.Generic2dOscillator(), connectivity=conn, coupling=coupling.Linear(a=0.0152),
                     integrator=integrators.HeunDeterministic(dt=0.1), monitors=mons, simulation_length=40.0)


def test_projection_gains_and_analytic_lead_fields_match_reference():
    """Region lead fields (vertex gains summed per region, the analytic field of non-cortical regions) and the
    Sarvas analytic EEG / MEG / iEEG formulas equal the reference's (monitors.py:492-600,699-716,752-784,813-824);
    sampling every int(period / dt) steps."""
    import golden_util as G
    from tvb_b200 import monitors, sensors
    fx = G.load('projection_40')
    eeg, meg, ieeg = _projection_setup(fx)
    _sim(fx, [eeg, meg], False).configure()
    _sim(fx, [ieeg], True).configure()
    np.testing.assert_allclose(eeg.gain, fx['em_m0_gain'], rtol=1e-13, atol=0)
    np.testing.assert_allclose(meg.gain, fx['em_m1_gain'], rtol=1e-13, atol=0)
    np.testing.assert_allclose(ieeg.gain, fx['ieeg_m0_gain'], rtol=1e-13, atol=1e-20)
    assert (eeg.istep, meg.istep, ieeg.istep) == (9, 9, 20)
    src, so = fx['centres'][:8], fx['orientations'][:8]
    for m, key in ((monitors.EEG(sensors=sensors.SensorsEEG(['a'] * 16, fx['sensors_eeg']), sigma=0.7), 'eeg'),
                   (monitors.MEG(sensors=sensors.SensorsMEG(['a'] * 12, fx['sensors_meg'])), 'meg'),
                   (monitors.iEEG(sensors=sensors.SensorsInternal(['a'] * 10, fx['sensors_ieeg']), sigma=0.7), 'ieeg')):
        np.testing.assert_allclose(m.analytic(src, so), fx[key + '_analytic'], rtol=1e-12, atol=0)


def test_projection_finish_noise_and_reference():
    """Observation noise drawn per sample in order as (sensors, nvoi) and the average EEG reference."""
    import golden_util as G
    fx = G.load('projection_40')
    eeg, _, _ = _projection_setup(fx)
    _sim(fx, [eeg], False).configure()
    y = np.random.default_rng(0).normal(size=(5, 1, 16))
    got = eeg.finish(y)
    rs = np.random.RandomState(42)
    want = y + np.stack([np.sqrt(0.1) * rs.normal(size=(16, 1)).T for _ in range(5)])
    want = want - want.mean(axis=2, keepdims=True)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


def test_rawvoi_and_progress_logger_configuration():
    """RawVoi keeps the chosen variables of interest (monitors.py:193-211); ProgressLogger records nothing and
    logs every int(period / dt) steps (monitors.py:1005-1026)."""
    from tvb_b200 import coupling, integrators, models, monitors, synthetic
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.simulator import Simulator
    w, L = synthetic.connectome(10, 0.5, 5.0, 30.0, seed=1)
    mons = [monitors.RawVoi(variables_of_interest=[1, 3]), monitors.Raw(), monitors.ProgressLogger(period=2.0)]
    sim = Simulator(model=models.JansenRit(), connectivity=Connectivity(w, L, speed=3.0),
                    coupling=coupling.SigmoidalJansenRit(), integrator=integrators.HeunDeterministic(dt=0.1),
                    monitors=mons, simulation_length=5.0).configure()
    assert list(mons[0].voi) == [1, 3] and mons[0].istep == 1
    assert len(mons[1].voi) == len(sim.model.variables_of_interest)
    assert mons[2].istep == 20
