"""Instance sharding of a parameter sweep over processes (one per GPU).

The reference runs a parameter-space exploration as one operation per grid
point (tvb_framework/tvb/core/services/operation_service.py:149-186); here
the grid's instances are split over ranks with no collective while they run,
and the results are gathered once at the end.  These tests run two `gloo`
ranks on the CPU (no device work): the union of the two shards' plans equals
the single-process plan instance by instance (global index, swept values,
noise scale, Philox stream, length), and gather_sweep() reassembles
per-instance results -- arrays and uneven-length lists -- in global order.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _sweep(**kw):
    from tvb_b200 import coupling, integrators, models, monitors, noise, synthetic
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.sweep import ParameterSweep
    w, L = synthetic.connectome(68, 0.3, 10.0, 200.0, seed=3)
    G = np.logspace(-3, 0, 7)
    S = np.logspace(-4, -2, 7)
    lengths = np.linspace(50.0, 110.0, 7)
    return ParameterSweep(model=models.ReducedWongWang(), connectivity=Connectivity(w, L, speed=5.0),
                          coupling=coupling.Linear(), monitors=[monitors.TemporalAverage(period=10.0)],
                          integrator=integrators.EulerStochastic(dt=0.1, noise=noise.Additive(nsig=[1e-3])),
                          simulation_length=110.0,
                          sweep={'coupling.a': G, 'noise.nsig': S, 'simulation_length': lengths}, **kw).configure()


def _plan(sw):
    return [dict(g=int(g), a=float(s.cfun[0]), sigma=np.asarray(s.sigma).copy(), stream=s.stream, steps=s.n_steps,
                 seed=s.seed) for g, s in zip(sw.instances, sw._specs)]


def _fake_results(sw):
    """Per-instance results shaped like ParameterSweep.run()'s, filled with
    the global index (the gather must put each where it belongs)."""
    I = sw.n_instances
    g = sw.instances.astype(np.float64)
    return {'instances': sw.instances.copy(),
            'fc': np.broadcast_to(g[:, None, None], (I, 68, 68)).copy(),
            'status': sw.instances.astype(np.int32) * 10,
            'tavg': [np.full((int(s.n_steps) // 100, 1, 68), gi, dtype=np.float32) for gi, s in zip(g, sw._specs)]}


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    import torch.distributed as dist
    from tvb_b200.sweep import gather_sweep
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        sw = _sweep(shard=(rank, world))
        plans = [None] * world if rank == 0 else None
        dist.gather_object(_plan(sw), plans, dst=0)
        merged = gather_sweep(_fake_results(sw))
        if rank == 0:
            out.put((plans, merged))
        else:
            assert merged is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('world', [2])
def test_shards_union_equals_single_process_plan(world):
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    plans, merged = out.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    whole = _sweep()
    ref = _plan(whole)
    got = [e for part in plans for e in part]
    # disjoint contiguous shards that cover the grid
    assert [e['g'] for e in got] == list(range(whole.n_global))
    assert all(len(part) > 0 for part in plans)
    for a, b in zip(got, ref):
        assert a['g'] == b['g'] and a['stream'] == b['stream'] == a['g']   # Philox keyed by the global index
        assert a['a'] == b['a'] and a['steps'] == b['steps'] and a['seed'] == b['seed']
        np.testing.assert_array_equal(a['sigma'], b['sigma'])
    # the gather reassembles every per-instance result in global order
    np.testing.assert_array_equal(merged['instances'], np.arange(whole.n_global))
    assert (merged['fc'][:, 0, 0] == np.arange(whole.n_global)).all()
    assert (merged['status'] == np.arange(whole.n_global) * 10).all()
    assert [int(t[0, 0, 0]) for t in merged['tavg']] == list(range(whole.n_global))
    assert [t.shape[0] for t in merged['tavg']] == [int(s.n_steps) // 100 for s in whole._specs]


def test_explicit_instances_and_errors():
    from tvb_b200.sweep import shard_instances
    sw = _sweep(instances=[5, 1])
    assert list(sw.instances) == [5, 1] and [s.stream for s in sw._specs] == [5, 1]
    whole = _sweep()
    assert sw._specs[0].cfun == whole._specs[5].cfun and sw._specs[1].n_steps == whole._specs[1].n_steps
    assert [len(shard_instances(7, (r, 3))) for r in range(3)] == [3, 2, 2]
    with pytest.raises(IndexError):
        shard_instances(7, instances=[7])
    with pytest.raises(ValueError):
        shard_instances(7, instances=[1, 1])
    with pytest.raises(ValueError):
        shard_instances(7, shard=(3, 3))
