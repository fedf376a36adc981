"""Bank-conflict-free gather slots of the row kernel (CPU): every row's edges
appear once with their offsets and weights, padding has weight 0 and reads
at least d_min steps back, and in every slot the 32 rows of a warp read 32
different shared-memory banks at every step and ring position."""
import numpy as np
import pytest


@pytest.mark.parametrize('n,density,seed', [(68, 0.3, 3), (76, 0.4, 1), (96, 0.25, 7), (40, 0.5, 2)])
def test_slot_table_is_a_conflict_free_permutation(n, density, seed):
    from tvb_b200 import _lib, synthetic
    from tvb_b200.engine import Connectome
    w, L = synthetic.connectome(n, density, 10.0, 200.0, seed=seed)
    idl, H = _lib.idelays(L, 5.0, 0.1)
    c = Connectome(w, idl, 1)
    width = 32 if np.diff(c.row_ptr).max() <= 32 else 64
    t = c.slot_table(width)
    assert t is not None and t.shape == (n, width, 2)
    off = c.idelay.astype(np.int64) * n - c.col
    wbits = c.weight.astype(np.float32).view(np.int32)
    for r in range(n):
        e = np.arange(c.row_ptr[r], c.row_ptr[r + 1])
        real = t[r, :, 1] != 0
        got = sorted(zip(t[r, real, 0].tolist(), t[r, real, 1].tolist()))
        assert got == sorted(zip(off[e].tolist(), wbits[e].tolist()))
        assert (t[r, ~real, 0] >= c.min_delay * n).all()
    m = 32 // np.gcd(n, 32)
    RL = -(-(H + 20) // m) * m
    ring = RL * n
    assert ring % 32 == 0
    for base_slot in (0, 1, 17, RL - 1):
        base = base_slot * n
        for w0 in range(0, n, 32):
            for k in range(width):
                a = base - t[w0:w0 + 32, k, 0].astype(np.int64)
                a = np.where(a < 0, a + ring, a)
                assert ((a >= 0) & (a < ring)).all()
                words = {}
                for x in a.tolist():
                    words.setdefault(x % 32, set()).add(x)
                assert max(len(v) for v in words.values()) == 1


def test_batch_pads_the_ring_and_keeps_two_ctas_per_sm():
    from tvb_b200 import _lib, synthetic
    from tvb_b200.engine import Batch, Connectome, InstanceSpec
    n = 68
    w, L = synthetic.connectome(n, 0.3, 10.0, 200.0, seed=3)
    idl, H = _lib.idelays(L, 5.0, 0.1)
    c = Connectome(w, idl, 1)
    spec = InstanceSpec(c, np.zeros((H, 1, n), np.float32), np.zeros((1, n)), np.zeros((9, n), np.float32),
                        [0.1, 0.0], 100, sigma=np.full((1, n), 0.01, np.float32))
    b = Batch(_lib.MODEL_IDS['ReducedWongWang'], _lib.CFUN_IDS['Linear'], _lib.SCHEME_IDS['EulerStochastic'],
              _lib.NOISE_PHILOX, 0.1, [0], [spec], device='cpu', allocate=False)
    assert b.ring_in_smem and b.prefetch == 1 and b.slot_width == 32
    RL = b.meta[0]['ring_len']
    assert RL >= H + b.sync_every and RL * n % 32 == 0
    # the ring plus its mirrored guard slots keeps two CTAs per SM resident
    assert b.guard == _lib.RING_GUARD
    assert 228 * 1024 // ((RL + b.guard) * n * 4 + 1024) == 2
    assert 4 <= b.sync_every <= c.min_delay


def test_large_network_batches_plan_cooperative_groups():
    """Region-major Epileptor 998 batches plan one cooperative launch of
    groups: 16 uneven instances on 9 groups of 16 CTAs (144 of 148 SMs, where
    thread-block clusters of 16 fit 7 at a time), a single instance on 64
    CTAs; an explicit cluster or groups=False keeps thread-block clusters."""
    from tvb_b200 import _lib, coupling, integrators, models, monitors, synthetic
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.engine import Batch
    from tvb_b200.sweep import ParameterSweep
    w, L = synthetic.connectome(998, 0.10, 5.0, 300.0, seed=4)
    x0 = np.random.default_rng(14).uniform(-2.4, -1.6, (16, 998))

    def plan(ni, uneven, **kw):
        sweep = {'model.x0': x0[:ni]}
        if uneven:
            sweep['simulation_length'] = np.linspace(20.0, 200.0, ni)
        sw = ParameterSweep(model=models.Epileptor(), connectivity=Connectivity(w, L, speed=3.0),
                            coupling=coupling.Difference(), integrator=integrators.HeunDeterministic(dt=0.05),
                            monitors=[monitors.TemporalAverage(period=1.0)], simulation_length=100.0, sweep=sweep,
                            device='cpu').configure()
        sim = sw._sim
        return Batch(sim._model_id, sim._cfun_id, sim._scheme_id, sw._noise_kind, sw.integrator.dt, sim._voi_codes,
                     sw._specs, device='cpu', allocate=False, **kw)

    b = plan(16, True)
    assert (b.ring_layout, b.groups, b.cluster) == (1, 9, 16) and b.edges_per_thread == 16
    # the group launch keeps four-step blocks (K a multiple of 4 with K <= d_min - 3), thread-block clusters
    # take eight-step blocks (K a multiple of 8 with K <= d_min - 7)
    dmin = min(sp.conn.min_delay for sp in b.specs)
    assert b.block_steps == 4 and b.sync_every % 4 == 0 and 4 <= b.sync_every <= dmin - 3
    b8 = plan(16, True, groups=False)
    assert b8.block_steps == 8 and b8.sync_every % 8 == 0 and 8 <= b8.sync_every <= dmin - 7
    b8 = plan(16, True, block_steps=8)
    assert b8.groups == 9 and b8.block_steps == 8
    assert _lib.group_sync_words(b.groups) == 20
    b = plan(1, False)
    assert (b.groups, b.cluster) == (1, 64) and b.edges_per_thread in (8, 16, 32)
    b = plan(16, True, cluster=16)
    assert (b.groups, b.cluster, b.ring_layout) == (0, 16, 1)
    b = plan(16, True, groups=False)
    assert (b.groups, b.cluster) == (0, 16)
    b = plan(16, True, groups=4)
    assert b.groups == 4 and b.groups * b.cluster <= 148


def test_sigmoidal_jansen_rit_plans_region_major_rings():
    """JansenRit + SigmoidalJansenRit on 998 regions plans region-major rings
    (a region-major ring of sigmoid values beside the state ring) and
    cooperative groups; region_rings=False keeps time-major edge runs."""
    from tvb_b200 import _lib, coupling, integrators, models, monitors, synthetic
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.engine import Batch
    from tvb_b200.sweep import ParameterSweep
    w, L = synthetic.connectome(998, 0.10, 5.0, 300.0, seed=2)

    def plan(**kw):
        sw = ParameterSweep(model=models.JansenRit(), connectivity=Connectivity(w, L, speed=3.0),
                            coupling=coupling.SigmoidalJansenRit(), integrator=integrators.HeunDeterministic(dt=0.05),
                            monitors=[monitors.TemporalAverage(period=1.0)], simulation_length=10.0,
                            sweep={'coupling.a': np.linspace(0.5, 2.0, 8)}, device='cpu').configure()
        sim = sw._sim
        return Batch(sim._model_id, sim._cfun_id, sim._scheme_id, sw._noise_kind, sw.integrator.dt, sim._voi_codes,
                     sw._specs, device='cpu', allocate=False, **kw)

    b = plan()
    assert b.sigma and b.ring_layout == 1 and b.groups == 8 and b.sync_every % 4 == 0
    RL = b.meta[0]['ring_len']
    assert b.zero.regions[('pre_ring', 0)][1] == _lib.ring_region_stride(RL, 1) * 998 * 4
    b = plan(region_rings=False)
    assert b.sigma and b.ring_layout == 0 and b.groups == 0 and b.edges_per_thread in (8, 16, 32)

