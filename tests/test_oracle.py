"""Pin the CPU oracle to the reference: golden vectors from reference runs and
the reference's own known-answer tests.  CPU only."""
import numpy as np
import pytest

import golden_util as G
from golden_util import O


def test_idelays_at_ties():
    """rint((L / speed) / dt), round half to even, horizon = max + 1 (connectivity.py:275,321-323)."""
    fx = G.load('idelays')
    L = fx['tract_lengths']
    n = 0
    for key in fx:
        if key.startswith('idelays_s'):
            speed, dt = key[len('idelays_s'):].split('_dt')
            idl, hz = O.integer_delays(L, float(speed), float(dt))
            np.testing.assert_array_equal(idl, fx[key])
            assert hz == int(fx['horizon_s%s_dt%s' % (speed, dt)])
            n += 1
    assert n == 16


def test_sparse_layout_g2d():
    fx = G.load('g2d_76')
    w, L = G.connectome(fx)
    idl, hz = O.integer_delays(L, float(fx['speed']), float(fx['dt']))
    np.testing.assert_array_equal(idl, fx['idelays'])
    assert hz == int(fx['horizon'])
    lay = O.sparse_layout(w, idl)
    np.testing.assert_array_equal(lay['row'], fx['nnz_row'])
    np.testing.assert_array_equal(lay['col'], fx['nnz_col'])
    np.testing.assert_array_equal(lay['w'], fx['nnz_w'])
    np.testing.assert_array_equal(lay['d'], fx['nnz_d'])


def test_exact_propagation():
    """Reference history_test.py:94-112: 4-node chain, identity coupling, x' = x + c."""
    fx = G.load('propagation_4')
    out, _ = O.simulate('Sum', {}, fx['weights'], fx['tract_lengths'], 1.0, 1.0, 'Linear', {'a': 1.0, 'b': 0.0},
                        'Identity', 10, [O.Monitor('Raw')], fx['buffer0'], fx['state0'], int(fx['step0']))
    np.testing.assert_array_equal(out[0][1][:, 0, :], fx['raw'])
    expected = np.array([[2., 2., 2., 1.], [3., 3., 3., 1.], [5., 4., 4., 1.], [8., 5., 5., 1.],
                         [12., 6., 6., 1.], [17., 7., 7., 1.], [23., 8., 8., 1.], [30., 10., 9., 1.],
                         [38., 13., 10., 1.], [48., 17., 11., 1.]])
    np.testing.assert_array_equal(fx['raw'], expected)


def test_difference_and_linear_coupling_known_answer():
    """Reference coupling_test.py:71-85 on two nodes with states 1 and 2."""
    fx = G.load('difference_2')
    w = fx['weights']
    idl = np.zeros((2, 2), dtype=np.int32)
    lay = O.sparse_layout(w, idl)
    buf = np.array([[[1.0, 2.0]]], dtype=np.float32)  # (H=1, ncvar=1, n=2)
    diff = O.coupling_sparse('Difference', buf, 0, lay, {'a': 0.1})
    np.testing.assert_allclose(diff, fx['difference'], rtol=0, atol=0)
    np.testing.assert_allclose(diff[0], [0.1 * (2 - 1), 0.1 * (1 - 2)], rtol=1e-7)
    lin = O.coupling_sparse('Linear', buf, 0, lay, {'a': 0.5, 'b': 0.25})
    np.testing.assert_allclose(lin, fx['linear'], rtol=0, atol=0)


@pytest.mark.parametrize('model', ['Generic2dOscillator', 'JansenRit', 'ReducedWongWang'])
def test_model_fixed_points(model):
    """Model.stationary_trajectory (models/base.py:164-204): Euler dt 0.01,
    2000 steps, zero coupling, from the middle of each state range; the
    reference's fixed points (models_test.py:226,240-243,277)."""
    fx = G.load('steady_state')
    # stationary_trajectory advances its initial_conditions array in place, so
    # the start is the first trajectory sample (the middle of each range)
    init = fx[model + '_traj'][0].reshape(-1, 1)
    dfun = O.DFUNS[model]
    p = {k: np.asarray(v) for k, v in O.MODEL_DEFAULTS[model].items()}
    ncv = len(O.MODEL_INFO[model]['cvar'])
    state = init.copy()
    c = np.zeros((ncv, 1))
    traj = [state.copy()]
    for i in range(2000):
        state = state + 0.01 * dfun(state, c, p)
        if i % 10 == 0:
            traj.append(state.copy())
    traj = np.array(traj)[:, :, 0]
    np.testing.assert_allclose(traj, fx[model + '_traj'], rtol=1e-10, atol=1e-12)
    fixed = {'Generic2dOscillator': [1.048535, -4.507975],
             'JansenRit': [1.105518e-02, 4.790847e+00, 8.826628e-01, 1.308187e-03, 2.367387e-01, 6.615113e-02],
             'ReducedWongWang': [0.452846]}[model]
    np.testing.assert_allclose(traj[-1], fixed, rtol=1e-6, atol=1e-3)


@pytest.mark.parametrize('variant', ['stock', 'fp64'])
def test_g2d_linear_heun(variant):
    fx = G.load('g2d_76')
    w, L = G.connectome(fx)
    fp64 = variant == 'fp64'
    buf = G.initial_history(fx, 'Generic2dOscillator', 76, fp64=fp64, key='buffer0_fp64' if fp64 else 'buffer0')
    out, _ = O.simulate('Generic2dOscillator', {}, w, L, float(fx['speed']), float(fx['dt']), 'Linear',
                        {'a': float(fx['coupling_a'])}, 'HeunDeterministic', 1500,
                        [O.Monitor('Raw'), O.Monitor('TemporalAverage', 1.0)], buf, fx['state0'],
                        int(fx['step0']), history_dtype=np.float64 if fp64 else np.float32)
    sfx = '_fp64' if fp64 else ''
    np.testing.assert_allclose(out[0][0], fx['raw_t'], rtol=0, atol=0)
    np.testing.assert_allclose(out[1][0], fx['tavg_t'], rtol=0, atol=0)
    np.testing.assert_allclose(out[0][1], fx['raw' + sfx], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(out[1][1], fx['tavg' + sfx], rtol=1e-12, atol=1e-12)


def test_epileptor_difference_coupled():
    fx = G.load('epi_96_coupled')
    w, L = G.connectome(fx)
    gains = dict(zip([str(s) for s in fx['gain_names']], fx['gain_values']))
    params = dict(x0=fx['x0'], **gains)
    buf = G.initial_history(fx, 'Epileptor', 96)
    n_steps = int(round(float(fx['length']) / float(fx['dt'])))
    out, _ = O.simulate('Epileptor', params, w, L, float(fx['speed']), float(fx['dt']), 'Difference', {},
                        'HeunDeterministic', n_steps, [O.Monitor('TemporalAverage', 1.0)], buf, fx['state0'],
                        int(fx['step0']))
    np.testing.assert_allclose(out[0][0], fx['tavg_t'], rtol=0, atol=0)
    np.testing.assert_allclose(out[0][1], fx['tavg'], rtol=1e-10, atol=1e-10)


@pytest.mark.slow
def test_epileptor_998_prefix():
    fx = G.load('epi_998')
    w, L = G.connectome(fx)
    idl, hz = O.integer_delays(L, float(fx['speed']), float(fx['dt']))
    assert G.sha(idl) == str(fx['idelays_sha256'])
    buf = G.initial_history(fx, 'Epileptor', 998)
    out, _ = O.simulate('Epileptor', dict(x0=fx['x0']), w, L, float(fx['speed']), float(fx['dt']), 'Difference', {},
                        'HeunDeterministic', 200, [O.Monitor('TemporalAverage', 1.0)], buf, fx['state0'],
                        int(fx['step0']))
    np.testing.assert_allclose(out[0][1], fx['tavg'][:10], rtol=1e-10, atol=1e-10)


def test_rww_stochastic_fed_noise_prefix():
    """EulerStochastic with the reference's own RandomState stream regenerated
    (initial history first, then one normal per step and region)."""
    fx = G.load('rww_68_short')
    w, L = G.connectome(fx)
    n, n_steps = 68, 20000
    z = G.reference_noise(fx, 'ReducedWongWang', n_steps, n)
    for k in (1, 3):
        buf = G.initial_history(fx, 'ReducedWongWang', n, seed=42, key='buffer0_%d' % k)
        out, _ = O.simulate('ReducedWongWang', {}, w, L, float(fx['speed']), float(fx['dt']), 'Linear',
                            {'a': fx['G'][k]}, 'EulerStochastic', n_steps,
                            [O.Monitor('Bold', 2000.0), O.Monitor('TemporalAverage', 100.0)], buf, fx['state0_%d' % k],
                            0, nsig=[fx['nsig'][k]], noise_z=z)
        np.testing.assert_allclose(out[0][1], fx['bold_%d' % k][:1], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(out[1][1], fx['tavg_%d' % k][:20], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(O.bold_hrf()[0], fx['hrf'], rtol=0, atol=0)


def test_fc_is_corrcoef():
    fx = G.load('rww_68_short')
    bold = fx['bold_3'][:, 0, :]
    np.testing.assert_allclose(O.functional_connectivity(bold), fx['fc_3'], rtol=0, atol=0)


def test_philox_known_answers():
    """Philox4x32-10 test vectors published with Random123 (Salmon et al., SC'11)."""
    cases = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
             ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
             ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
              (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for c, k, want in cases:
        got = O.philox4x32_10(*[np.uint32(v) for v in c], np.uint32(k[0]), np.uint32(k[1]))
        assert tuple(int(x) for x in got) == want


def test_philox_normals_statistics():
    z = O.philox_normals(42, 7, np.arange(1, 4001), 2, 64)
    assert z.shape == (4000, 2, 64)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01
    u = O.uniform_open(np.array([0, 0xFFFFFFFF], dtype=np.uint32))
    assert 0.0 < u[0] < u[1] < 1.0


def test_jansen_rit_sigmoidal_heun_stochastic_prefix():
    """JansenRit + dense SigmoidalJansenRit + HeunStochastic (noise on y4 only),
    the reference's RandomState stream regenerated; first 200 ms."""
    fx = G.load('jr_192')
    w, L = G.connectome(fx)
    n, n_steps = 192, 4000
    z = G.reference_noise(fx, 'JansenRit', n_steps, n)
    buf = G.initial_history(fx, 'JansenRit', n, seed=42)
    out, _ = O.simulate('JansenRit', {}, w, L, float(fx['speed']), float(fx['dt']), 'SigmoidalJansenRit', {},
                        'HeunStochastic', n_steps, [O.Monitor('TemporalAverage', 1.0)], buf, fx['state0'], 0,
                        nsig=fx['nsig'], noise_z=z)
    idx = fx['tavg_index']
    k = int(np.sum(idx < 200))
    np.testing.assert_allclose(out[0][1][idx[:k]], fx['tavg'][:k], rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize('case,coupling,params,integrator', [
    ('scaling', 'Scaling', {'a': 0.02}, 'HeunDeterministic'),
    ('sigmoidal', 'Sigmoidal', {'cmin': -0.5, 'cmax': 0.5, 'midpoint': 0.5, 'a': 1.2, 'sigma': 4.0},
     'HeunDeterministic'),
    ('tanh', 'HyperbolicTangent', {'a': 0.05, 'b': 0.8, 'midpoint': 0.3, 'sigma': 2.0}, 'HeunDeterministic'),
    ('kuramoto', 'Kuramoto', {'a': 0.3}, 'HeunDeterministic'),
    ('rk4', 'Linear', {'a': 0.0152}, 'RungeKutta4thOrderDeterministic')])
def test_more_couplings_and_rk4(case, coupling, params, integrator):
    """Scaling, Sigmoidal, HyperbolicTangent, Kuramoto (coupling.py:203-322,489-508) and
    RungeKutta4thOrderDeterministic (integrators.py:429-480) against reference runs."""
    fx = G.load('couplings_40')
    w, L = fx['weights'], fx['tract_lengths']
    out, _ = O.simulate('Generic2dOscillator', {}, w, L, float(fx['speed']), 0.1, coupling, params, integrator,
                        400, [O.Monitor('Raw')], fx[case + '_buffer0'], fx[case + '_state0'], 0)
    ref = fx[case + '_raw']
    err = np.abs(out[0][1] - ref).max() / np.abs(ref).max()
    assert err < 1e-9, (case, err)


def test_epileptor_hyperbolic_tangent_two_cvars():
    fx = G.load('couplings_40')
    out, _ = O.simulate('Epileptor', {}, fx['weights'], fx['tract_lengths'], float(fx['speed']), 0.05,
                        'HyperbolicTangent', {'a': 0.02, 'b': 1.0, 'midpoint': -1.0, 'sigma': 1.5},
                        'HeunDeterministic', 400, [O.Monitor('TemporalAverage', 1.0)],
                        fx['epi_tanh_buffer0'], fx['epi_tanh_state0'], 0)
    ref = fx['epi_tanh_tavg']
    err = np.abs(out[0][1] - ref).max() / np.abs(ref).max()
    assert err < 1e-9, err


def test_subsample_global_spatial_average_monitors():
    """SubSample, GlobalAverage, SpatialAverage (monitors.py:213-360) against reference runs (G2D, and RWW
    with the reference's own noise stream)."""
    fx = G.load('monitors_40')
    w, L = fx['weights'], fx['tract_lengths']
    mask = fx['spatial_mask']
    mons = [O.Monitor('SubSample', 1.0), O.Monitor('GlobalAverage', 1.0),
            O.Monitor('SpatialAverage', 1.0, spatial_mask=mask), O.Monitor('TemporalAverage', 1.0)]
    out, _ = O.simulate('Generic2dOscillator', {}, w, L, float(fx['speed']), 0.1, 'Linear', {'a': 0.0152},
                        'HeunDeterministic', 400, mons, fx['g2d_buffer0'], fx['g2d_state0'], 0)
    for (t, y), name in zip(out, ('sub', 'glob', 'spat', 'tavg')):
        ref = fx['g2d_' + name]
        assert y.shape == ref.shape, name
        np.testing.assert_allclose(t, fx['g2d_%s_t' % name], rtol=0, atol=1e-12)
        assert np.abs(y - ref).max() / np.abs(ref).max() < 1e-9, name
    H = fx['rww_buffer0'].shape[0]
    z = O.reference_noise(42, [O.MODEL_INFO['ReducedWongWang']['ranges']['S']], H, 40, 1, 400)
    out, _ = O.simulate('ReducedWongWang', {}, w, L, float(fx['speed']), 0.1, 'Linear', {'a': 0.3},
                        'EulerStochastic', 400, mons, fx['rww_buffer0'], fx['rww_state0'], 0, nsig=[1e-3], noise_z=z)
    for (t, y), name in zip(out, ('sub', 'glob', 'spat', 'tavg')):
        ref = fx['rww_' + name]
        assert np.abs(y - ref).max() / np.abs(ref).max() < 1e-9, name


@pytest.mark.parametrize('case', ['nl_rbm_none', 'lin_rbm_sum', 'nl_cbm_absdiff', 'nl_rbm_norm'])
def test_balloon_oracle_vs_reference(case):
    """Balloon-Windkessel BOLD (tvb/analyzers/fmri_balloon.py) restated in the oracle vs the reference."""
    fx = G.load('balloon')
    x = fx['x']
    kw = dict(nl_rbm_none=('none', False, True, True), lin_rbm_sum=('sum', False, False, True),
              nl_cbm_absdiff=('abs_diff', False, True, False), nl_rbm_norm=('none', True, True, True))[case]
    mode, norm, nonlinear, rbm = kw
    if mode == 'none':
        xi = x[:, 0, :, 0]
    elif mode == 'sum':
        xi = x.sum(axis=1)[:, :, 0]
    else:
        xi = np.abs(np.diff(x, axis=0))[:, 0, :, 0]
    if norm:
        xi = xi - xi.mean(axis=0)
    E0, TE, eps, nu0, r0 = 0.4, 0.04, 0.5, 40.3, 25.0
    k = (4.3 * nu0 * E0 * TE, eps * r0 * E0 * TE, 1 - eps) if rbm else (7. * E0, 2. * E0, 1. - eps)
    out = O.balloon_bold(xi, 0.001, k=k, nonlinear=nonlinear)
    ref = fx[case][:, 0, :, 0]
    assert out.shape == ref.shape
    assert np.abs(out - ref).max() / np.abs(ref).max() < 1e-12


STIM_CASES = {
    # case: model, model params, coupling, coupling params, integrator, dt, steps, monitors, nsig
    'g2d_pulse': ('Generic2dOscillator', 'Linear', {'a': 0.0152}, 'HeunDeterministic', 0.1, 600,
                  lambda: [O.Monitor('Raw'), O.Monitor('TemporalAverage', 1.0)], None),
    'g2d_w_sin': ('Generic2dOscillator', 'Linear', {'a': 0.0152}, 'EulerDeterministic', 0.1, 400,
                  lambda: [O.Monitor('Raw')], None),
    'rww_alpha': ('ReducedWongWang', 'Linear', {'a': 0.3}, 'EulerStochastic', 0.1, 400,
                  lambda: [O.Monitor('Raw')], [1e-4]),
    'epi_gauss': ('Epileptor', 'Linear', {'a': 0.01}, 'RungeKutta4thOrderDeterministic', 0.05, 400,
                  lambda: [O.Monitor('Raw')], None),
}


@pytest.mark.parametrize('case', sorted(STIM_CASES))
def test_region_stimulus(case):
    """StimuliRegion through the scheme's stimulus term (simulator.py:290-306, integrators.py:296-530) against
    reference runs: PulseTrain / Sinusoid / Alpha / Gaussian temporal patterns, stvar = cvar and stvar = [1]."""
    fx = G.load('stimulus_40')
    model, cf, cp, integ, dt, n_steps, mons, nsig = STIM_CASES[case]
    z = None
    if nsig is not None:
        H = fx[case + '_buffer0'].shape[0]
        z = O.reference_noise(42, [O.MODEL_INFO[model]['ranges']['S']], H, 40, 1, n_steps)
    stim = (fx[case + '_temporal'], fx[case + '_spatial'], fx[case + '_stvar'])
    out, _ = O.simulate(model, {}, fx['weights'], fx['tract_lengths'], float(fx['speed']), dt, cf, cp, integ, n_steps,
                        mons(), fx[case + '_buffer0'], fx[case + '_state0'], 0, nsig=nsig, noise_z=z, stimulus=stim)
    for k, (t, y) in enumerate(out):
        ref = fx['%s_m%d' % (case, k)]
        np.testing.assert_allclose(t, fx['%s_m%d_t' % (case, k)], rtol=0, atol=1e-12)
        err = np.abs(y - ref).max() / np.abs(ref).max()
        assert err < 1e-9, (case, k, err)
    # the stimulus changes the run: without it the oracle departs from the reference
    out0, _ = O.simulate(model, {}, fx['weights'], fx['tract_lengths'], float(fx['speed']), dt, cf, cp, integ,
                         n_steps, mons(), fx[case + '_buffer0'], fx[case + '_state0'], 0, nsig=nsig, noise_z=z)
    ref = fx['%s_m0' % case]
    assert np.abs(out0[0][1] - ref).max() / np.abs(ref).max() > 1e-4


AFF_CASES = {
    'g2d': ('Generic2dOscillator', 'Linear', {'a': 0.0152}, 0.1, 400,
            lambda: [O.Monitor('AfferentCoupling'), O.Monitor('AfferentCouplingTemporalAverage', 1.0),
                     O.Monitor('Raw')]),
    'epi': ('Epileptor', 'Difference', {'a': 0.1}, 0.05, 400,
            lambda: [O.Monitor('AfferentCoupling'), O.Monitor('AfferentCouplingTemporalAverage', 1.0, voi=[1])]),
    'jr': ('JansenRit', 'SigmoidalJansenRit', {'a': 10.0}, 0.1, 400,
           lambda: [O.Monitor('AfferentCoupling', voi=[0]),
                    O.Monitor('AfferentCouplingTemporalAverage', 2.0, voi=[0])]),
}


@pytest.mark.parametrize('case', sorted(AFF_CASES))
def test_afferent_coupling_monitors(case):
    """AfferentCoupling / AfferentCouplingTemporalAverage (monitors.py:394-433; node_coupling of step + 1,
    simulator.py:314-320,358-361) against reference runs: one, two and the SigmoidalJansenRit single
    coupling row."""
    fx = G.load('afferent_40')
    model, cf, cp, dt, n_steps, mons = AFF_CASES[case]
    out, _ = O.simulate(model, {}, fx['weights'], fx['tract_lengths'], float(fx['speed']), dt, cf, cp,
                        'HeunDeterministic', n_steps, mons(), fx[case + '_buffer0'], fx[case + '_state0'], 0)
    for k, (t, y) in enumerate(out):
        ref = fx['%s_m%d' % (case, k)]
        assert y.shape == ref.shape, (case, k)
        np.testing.assert_allclose(t, fx['%s_m%d_t' % (case, k)], rtol=0, atol=1e-12)
        err = np.abs(y - ref).max() / np.abs(ref).max()
        assert err < 1e-9, (case, k, err)


def test_projection_monitors():
    """EEG (average reference, observation noise), MEG and iEEG (analytic lead field for non-cortical regions)
    sampled every int(period / dt) steps (monitors.py:436-831) against reference runs, with the reference's
    configured gains and its observation-noise stream (RandomState(42), one (sensors, nvoi) draw per sample)."""
    fx = G.load('projection_40')
    w, L = fx['weights'], fx['tract_lengths']

    def obs(S, T):
        rs = np.random.RandomState(42)
        return [rs.normal(size=(S, 1)) for _ in range(T)]
    mons = [O.Monitor('Projection', 1e3 / 1024.0, gain=fx['em_m0_gain'], obs_z=obs(16, 44), ref_vec=np.full(16, 1 / 16)),
            O.Monitor('Projection', 1e3 / 1024.0, gain=fx['em_m1_gain'])]
    out, _ = O.simulate('Generic2dOscillator', {}, w, L, float(fx['speed']), 0.1, 'Linear', {'a': 0.0152},
                        'HeunDeterministic', 400, mons, fx['em_buffer0'], fx['em_state0'], 0)
    for k, (t, y) in enumerate(out):
        ref = fx['em_m%d' % k]
        assert y.shape == ref.shape
        np.testing.assert_allclose(t, fx['em_m%d_t' % k], rtol=0, atol=1e-12)
        assert np.abs(y - ref).max() / np.abs(ref).max() < 1e-9, k
    out, _ = O.simulate('Generic2dOscillator', {}, w, L, float(fx['speed']), 0.1, 'Linear', {'a': 0.0152},
                        'HeunDeterministic', 400,
                        [O.Monitor('Projection', 2.0, gain=fx['ieeg_m0_gain'], obs_z=obs(10, 20))],
                        fx['ieeg_buffer0'], fx['ieeg_state0'], 0)
    (t, y), = out
    np.testing.assert_allclose(t, fx['ieeg_m0_t'], rtol=0, atol=1e-12)
    assert np.abs(y - fx['ieeg_m0']).max() / np.abs(fx['ieeg_m0']).max() < 1e-9
