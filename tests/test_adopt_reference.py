"""The drop-in boundary fed the reference's own component objects.

tvb_b200.simulator.Simulator accepts the reference's model, coupling,
integrator, noise, monitor and connectivity objects and reads them by trait
name (tvb/simulator/simulator.py:58-159).  These tests build each component
twice with the reference's classes -- one set for the reference's own
Simulator, an identical one for the drop-in -- configure both, and check
that the drop-in adopted the same parameters (array-valued traits such as
Linear.a = numpy.array([...]) included), variables of interest, noise
(nsig shapes per integrated variable, seed), integer delays and horizon,
initial history and current state, and monitor step constants / HRF.

They need the reference's tvb_library source tree, located by the
TVB_REFERENCE_LIBRARY environment variable; without it they are skipped.
No device is needed (configure() runs on the host).
"""
import logging
import os
import sys
import warnings

import numpy as np
import pytest

REF = os.environ.get('TVB_REFERENCE_LIBRARY')
pytestmark = pytest.mark.skipif(not REF or not os.path.isdir(REF),
                                reason='set TVB_REFERENCE_LIBRARY to the reference tvb_library tree')


@pytest.fixture(scope='module')
def R():
    sys.path.insert(0, REF)
    warnings.filterwarnings('ignore')
    logging.disable(logging.WARNING)
    import tvb.simulator.coupling as coupling
    import tvb.simulator.integrators as integrators
    import tvb.simulator.models as models
    import tvb.simulator.monitors as monitors
    import tvb.simulator.noise as noise
    import tvb.simulator.simulator as simulator
    from tvb.datatypes.connectivity import Connectivity
    return dict(simulator=simulator, models=models, coupling=coupling, integrators=integrators,
                monitors=monitors, noise=noise, Connectivity=Connectivity)


def _conn(R, n, density, lo, hi, speed, seed):
    from tvb_b200 import synthetic
    w, L = synthetic.connectome(n, density, lo, hi, seed=seed)
    return R['Connectivity'](weights=w, tract_lengths=L, speed=np.array([speed]),
                             region_labels=np.array(['r%d' % i for i in range(n)]), centres=np.zeros((n, 3)))


CASES = {
    # RWW with a changed model trait, Linear.a as an array, EulerStochastic + Additive noise, Bold + TAVG
    'rww_linear_eulerstoch': lambda R: dict(
        connectivity=_conn(R, 68, 0.3, 10.0, 200.0, 5.0, 3),
        model=R['models'].ReducedWongWang(J_N=np.array([0.2609]), I_o=np.array([0.33])),
        coupling=R['coupling'].Linear(a=np.array([0.3]), b=np.array([0.0])),
        integrator=R['integrators'].EulerStochastic(dt=0.1, noise=R['noise'].Additive(nsig=np.array([1e-3]),
                                                                                      noise_seed=17)),
        monitors=(R['monitors'].Bold(period=2000.0), R['monitors'].TemporalAverage(period=1.0)),
        simulation_length=100.0),
    # JansenRit with noise on y4 only (nsig per state variable), SigmoidalJansenRit, HeunStochastic
    'jr_sigmoidal_heunstoch': lambda R: dict(
        connectivity=_conn(R, 40, 0.25, 5.0, 250.0, 4.0, 2),
        model=R['models'].JansenRit(mu=np.array([0.09])),
        coupling=R['coupling'].SigmoidalJansenRit(a=np.array([12.0])),
        integrator=R['integrators'].HeunStochastic(dt=0.05, noise=R['noise'].Additive(
            nsig=np.array([0.0, 0.0, 0.0, 0.0, 1e-5, 0.0]), noise_seed=3)),
        monitors=(R['monitors'].TemporalAverage(period=1.0),),
        simulation_length=50.0),
    # Epileptor with a spatialised x0 (one value per region) and its default VOIs, Difference, HeunDeterministic
    'epileptor_difference_heundet': lambda R: dict(
        connectivity=_conn(R, 48, 0.1, 5.0, 300.0, 3.0, 4),
        model=R['models'].Epileptor(x0=np.linspace(-2.4, -1.6, 48)),
        coupling=R['coupling'].Difference(a=np.array([0.05])),
        integrator=R['integrators'].HeunDeterministic(dt=0.05),
        monitors=(R['monitors'].Raw(), R['monitors'].SubSample(period=0.5)),
        simulation_length=20.0),
    # G2D with changed VOIs, Raw + GlobalAverage
    'g2d_linear_heundet': lambda R: dict(
        connectivity=_conn(R, 76, 0.4, 10.0, 200.0, 3.0, 1),
        model=R['models'].Generic2dOscillator(a=np.array([-0.5]), variables_of_interest=('V', 'W')),
        coupling=R['coupling'].Linear(a=np.array([0.0152])),
        integrator=R['integrators'].HeunDeterministic(dt=0.1),
        monitors=(R['monitors'].Raw(), R['monitors'].GlobalAverage(period=1.0)),
        simulation_length=20.0),
}


@pytest.mark.parametrize('case', sorted(CASES))
def test_reference_components_adopted(R, case):
    from tvb_b200.simulator import Simulator
    seed = 1234
    np.random.seed(seed)
    ref = R['simulator'].Simulator(**CASES[case](R)).configure()
    np.random.seed(seed)
    ours = Simulator(**CASES[case](R)).configure()

    # model parameters by trait name, spatialised like the reference
    rm = ref.model
    for name in type(ours.model)._defaults:
        if hasattr(rm, name):
            np.testing.assert_array_equal(np.broadcast_to(np.asarray(ours.model.__dict__.get(name, getattr(
                ours.model, name)), dtype=np.float64).reshape(-1), np.asarray(getattr(rm, name)).reshape(-1).shape),
                np.asarray(getattr(rm, name), dtype=np.float64).reshape(-1), err_msg=name)
    assert tuple(ours.model.variables_of_interest) == tuple(rm.variables_of_interest)
    # coupling parameters
    for name in type(ours.coupling)._defaults:
        if hasattr(ref.coupling, name):
            assert float(np.asarray(getattr(ours.coupling, name)).reshape(-1)[0]) == \
                float(np.asarray(getattr(ref.coupling, name)).reshape(-1)[0]), name
    # integrator, noise scale per integrated variable, seed
    assert ours.integrator.dt == ref.integrator.dt
    if hasattr(ref.integrator, 'noise'):
        rn, on = ref.integrator.noise, ours.integrator.noise
        assert on.noise_seed == rn.noise_seed
        nsig_ref = np.broadcast_to(np.asarray(rn.nsig, dtype=np.float64).reshape(rn.nsig.shape[0], -1)[:, :1],
                                   (rn.nsig.shape[0], 1))
        np.testing.assert_array_equal(np.asarray(on.nsig, dtype=np.float64).reshape(-1), nsig_ref.reshape(-1))
    # integer delays, horizon, initial history and current state
    np.testing.assert_array_equal(ours.connectivity.idelays, ref.connectivity.idelays)
    assert ours._conn.horizon == ref.connectivity.horizon
    np.testing.assert_array_equal(ours.history_buffer, ref.history.buffer)
    np.testing.assert_array_equal(ours.current_state, ref.current_state)
    assert ours.current_step == ref.current_step
    # monitors: step constants and the Bold kernel
    for mo, mr in zip(ours.monitors, ref.monitors):
        assert type(mo).__name__ == type(mr).__name__
        assert mo.istep == mr.istep
        if type(mr).__name__ == 'Bold':
            np.testing.assert_array_equal(mo.hemodynamic_response_function, mr.hemodynamic_response_function)
            assert mo._interim_istep == mr._interim_istep
        if hasattr(mr, 'voi'):
            np.testing.assert_array_equal(np.asarray(mo.voi).reshape(-1), np.asarray(mr.voi).reshape(-1))
