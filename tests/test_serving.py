"""Continuous-batching server: requests of different sizes, models, schemes,
dt and lengths arrive while others run, are admitted by device footprint
into free slots, and each result is the same as the request run alone."""
import numpy as np
import pytest

from tvb_b200 import coupling, integrators, models, monitors, noise, synthetic
from tvb_b200.connectivity import Connectivity
from tvb_b200.simulator import Simulator

# (regions, density, tract lengths, speed, seed) of the synthetic connectomes
SIZES = {24: (0.4, 10.0, 120.0, 3.0, 1), 48: (0.3, 10.0, 200.0, 5.0, 3), 76: (0.4, 10.0, 200.0, 3.0, 1),
         140: (0.1, 5.0, 250.0, 4.0, 2)}


def make_sim(model, n, dt, length, seed):
    dens, lo, hi, speed, cseed = SIZES[n]
    w, L = synthetic.connectome(n, dens, lo, hi, seed=cseed)
    conn = Connectivity(w, L, speed=speed)
    if model == 'G2D':
        np.random.seed(seed)
        return Simulator(model=models.Generic2dOscillator(), connectivity=conn, coupling=coupling.Linear(a=0.0152),
                         integrator=integrators.HeunDeterministic(dt=dt),
                         monitors=[monitors.Raw(), monitors.TemporalAverage(period=1.0)],
                         simulation_length=length).configure()
    if model == 'RWW':
        return Simulator(model=models.ReducedWongWang(), connectivity=conn, coupling=coupling.Linear(a=0.2),
                         integrator=integrators.EulerStochastic(dt=dt, noise=noise.Additive(nsig=[1e-3],
                                                                                            noise_seed=seed)),
                         monitors=[monitors.TemporalAverage(period=1.0), monitors.Bold(period=100.0)],
                         simulation_length=length).configure()
    nsig = np.array([0.0, 0.0, 0.0, 0.0, 1e-5, 0.0])
    return Simulator(model=models.JansenRit(), connectivity=conn, coupling=coupling.SigmoidalJansenRit(),
                     integrator=integrators.HeunStochastic(dt=dt, noise=noise.Additive(nsig=nsig, noise_seed=seed)),
                     monitors=[monitors.TemporalAverage(period=1.0)], simulation_length=length).configure()


CASES = [('G2D', 24, 0.1, 130.0), ('RWW', 48, 0.1, 260.0), ('JR', 76, 0.05, 60.0), ('RWW', 48, 0.05, 210.0),
         ('G2D', 140, 0.05, 55.0), ('RWW', 48, 0.1, 90.0), ('JR', 24, 0.1, 120.0), ('G2D', 24, 0.1, 40.0),
         ('RWW', 140, 0.1, 150.0), ('G2D', 76, 0.1, 75.0)]


def _serve(cases, arrive_every, budget=None, chunk=300):
    from tvb_b200.serving import SimulationServer
    srv = SimulationServer(memory_budget=budget, chunk_steps=chunk)
    rids = {}

    def submitter(k, case):
        def f(server):
            rids[k] = server.submit(make_sim(*case, seed=100 + k))
        return f

    arrivals = [(arrive_every * k, submitter(k, c)) for k, c in cases]
    srv.run(arrivals=arrivals, timeout=300.0)
    return srv, rids


@pytest.mark.gpu
def test_each_result_same_alone_and_in_the_mix():
    cases = list(enumerate(CASES))
    # the largest single footprint, so the budget admits only part of the mix at a time
    from tvb_b200.serving import SimulationServer
    probe = SimulationServer(memory_budget=1 << 40)
    fps = [probe.requests[probe.submit(make_sim(*c, seed=100 + k))].footprint for k, c in cases]
    budget = int(max(fps) * 2.5)
    mix, rids = _serve(cases, arrive_every=0.002, budget=budget)
    st = mix.stats()
    assert st['completed'] == len(CASES)
    assert st['memory_peak_bytes'] <= budget
    assert st['groups'] >= 5
    for k, _ in cases:
        assert mix.requests[rids[k]].status == 0
    # same request id alone and in the mix: identical results
    for k, case in cases:
        from tvb_b200.serving import SimulationServer
        solo = SimulationServer(chunk_steps=10 ** 7)
        solo.next_id = rids[k]
        rid = solo.submit(make_sim(*case, seed=100 + k))
        solo.run(timeout=120.0)
        for (ta, ya), (tm, ym) in zip(solo.result(rid), mix.result(rids[k])):
            np.testing.assert_array_equal(ta, tm)
            np.testing.assert_array_equal(ya, ym)


@pytest.mark.gpu
def test_server_matches_simulator_run():
    case = ('RWW', 48, 0.1, 260.0)
    from tvb_b200.serving import SimulationServer
    srv = SimulationServer(chunk_steps=700)
    srv.next_id = 7
    rid = srv.submit(make_sim(*case, seed=5))
    srv.run(timeout=120.0)
    sim = make_sim(*case, seed=5)
    sim.stream_id = 7
    ref = sim.run()
    for (ta, ya), (tr, yr) in zip(srv.result(rid), ref):
        np.testing.assert_array_equal(ta, tr)
        np.testing.assert_array_equal(ya, yr)


def test_footprint_plan_needs_no_device():
    from tvb_b200 import _lib
    from tvb_b200.engine import Batch
    sim = make_sim('RWW', 48, 0.1, 260.0, seed=3)
    spec, kind = sim.instance_spec(2600, stream=3)
    plan = Batch(sim._model_id, sim._cfun_id, sim._scheme_id, kind, 0.1, sim._voi_codes, [spec], device='cpu',
                 gather='row', allocate=False)
    n, H = 48, sim._conn.horizon
    ring = (H + plan.sync_every) * n * 4
    stock = 5000 * n * 8
    assert plan.nbytes >= ring + stock
    assert plan.nbytes < ring + stock + 2600 * n * 8 + 64 * 1024
    assert not plan.allocated and kind == _lib.NOISE_PHILOX
