"""Generate the golden fixtures for the region simulation loop by running the
reference TVB library (numpy path) on seeded synthetic connectomes.

This script is test infrastructure: it needs the reference source tree (the
``tvb_library`` directory of the-virtual-brain/tvb-root) and its numpy/numba
dependencies, and it is only run where that tree exists.  The fixtures it
writes (``tests/golden/*.npz``) are what the tests read; nothing at test time
imports the reference.

    python tests/golden/make_golden.py --ref /root/reference/tvb_library [--only NAME ...]

Every fixture records the raw inputs (weights, tract lengths, speed, dt,
component parameters), the configured state the reference produced
(idelays, horizon, the float32 history ring, the float64 current state and
step) and the monitor outputs, for the stock reference (float32 history and
weights, see ``tvb/simulator/history.py:49-51,166-172``) and, where noted, for
an all-float64 variant obtained by switching those descriptors to float64.

Stochastic fixtures store a SHA-256 of the noise the reference drew (recorded
by wrapping ``integrator.noise.generate``) plus a flag saying that the stream
is reproduced by ``numpy.random.RandomState(noise_seed)`` after the
initial-condition draws (``tvb/simulator/models/base.py:138-155``,
``tvb/simulator/noise.py:195-198``), so the tests regenerate the exact noise
instead of storing hundreds of MB of it.
"""
import argparse
import hashlib
import logging
import os
import sys
import time
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def synthetic_connectome(n, density, lo, hi, seed):
    """Seeded synthetic connectome: symmetric lognormal(0,1) weights on a random
    upper-triangle mask, normalised to max 1, zero diagonal; symmetric uniform
    tract lengths with zero diagonal."""
    rng = np.random.default_rng(seed)
    w = rng.lognormal(0.0, 1.0, (n, n))
    mask = np.triu(rng.random((n, n)) < density, 1)
    w = np.triu(w * mask, 1)
    w = w + w.T
    w /= w.max()
    lengths = np.triu(rng.uniform(lo, hi, (n, n)), 1)
    lengths = lengths + lengths.T
    return w, lengths


def import_reference(ref):
    sys.path.insert(0, ref)
    warnings.filterwarnings("ignore")
    logging.disable(logging.WARNING)
    import tvb.simulator.simulator as simulator
    import tvb.simulator.models as models
    import tvb.simulator.coupling as coupling
    import tvb.simulator.integrators as integrators
    import tvb.simulator.monitors as monitors
    import tvb.simulator.noise as noise
    import tvb.simulator.history as history
    from tvb.datatypes.connectivity import Connectivity
    from tvb.datatypes import equations, patterns, sensors, projections, region_mapping
    from tvb.basic.neotraits.api import List
    return dict(simulator=simulator, models=models, coupling=coupling,
                integrators=integrators, monitors=monitors, noise=noise,
                history=history, Connectivity=Connectivity, List=List,
                equations=equations, patterns=patterns, sensors=sensors, projections=projections,
                region_mapping=region_mapping)


FP64_FIELDS = {
    'BaseHistory': ['weights', 'delays'],
    'DenseHistory': ['es_weights', 'buffer', 'current_state', 'delayed_state'],
    'SparseHistory': ['nnz_weights'],
}


def set_history_dtype(R, code):
    """Switch the reference history descriptors between float32 ('f', stock)
    and float64 ('d', all-FP64 variant)."""
    for cls_name, fields in FP64_FIELDS.items():
        cls = getattr(R['history'], cls_name)
        for f in fields:
            cls.__dict__[f].dtype = code


def make_conn(R, w, lengths, speed):
    n = w.shape[0]
    return R['Connectivity'](weights=w, tract_lengths=lengths, speed=np.array([speed]),
                             region_labels=np.array(['r%d' % i for i in range(n)]),
                             centres=np.zeros((n, 3)))


class NoiseRecorder:
    def __init__(self, sim, keep=False):
        self.h = hashlib.sha256()
        self.count = 0
        self.keep = keep
        self.kept = []
        noise = sim.integrator.noise
        orig = noise.generate

        def gen(shape, lo=-1.0, hi=1.0):
            z = orig(shape, lo, hi)
            self.h.update(np.ascontiguousarray(z, dtype=np.float64).tobytes())
            self.count += 1
            if self.keep:
                self.kept.append(z.copy())
            return z
        noise.generate = gen


def regen_noise_hash(seed, ic_ranges, horizon, n, nintvar, n_steps, dt, chunk=20000):
    """Re-create the reference noise stream with RandomState(seed): first the
    initial-history uniform draws, then one normal draw of shape
    (nintvar, n, 1) per step scaled by sqrt(dt)."""
    rs = np.random.RandomState(seed)
    for lo, hi in ic_ranges:
        rs.uniform(low=lo, high=hi, size=(horizon, n, 1))
    h = hashlib.sha256()
    left = n_steps
    while left > 0:
        k = min(chunk, left)
        z = np.sqrt(dt) * rs.normal(size=(k, nintvar, n, 1))
        for s in range(k):
            h.update(np.ascontiguousarray(z[s]).tobytes())
        left -= k
    return h.hexdigest()


def configured_state(sim):
    hist = sim.history
    return dict(
        idelays=np.asarray(sim.connectivity.idelays, dtype=np.int32),
        horizon=np.int64(sim.connectivity.horizon),
        buffer0=np.array(hist.buffer[..., 0]),          # (H, ncvar, n)
        state0=np.array(sim.current_state[..., 0]),      # (nsv, n)
        step0=np.int64(sim.current_step),
        nnz_row=np.asarray(hist.nnz_row_el_idx, dtype=np.int32),
        nnz_col=np.asarray(hist.nnz_col_el_idx, dtype=np.int32),
        nnz_w=np.array(hist.nnz_weights),
        nnz_d=np.asarray(hist.nnz_idelays, dtype=np.int32),
    )


def run_sim(R, build, length, fp64, ic_seed=None, record_noise=False):
    set_history_dtype(R, 'd' if fp64 else 'f')
    try:
        sim = build()
        if ic_seed is not None:
            np.random.seed(ic_seed)
        sim.configure()
        cfg = configured_state(sim)
        rec = NoiseRecorder(sim) if record_noise else None
        t0 = time.time()
        out = sim.run(simulation_length=length)
        el = time.time() - t0
    finally:
        set_history_dtype(R, 'f')
    return sim, cfg, out, rec, el


# inputs that the tests regenerate bit-exactly from their recipe (synthetic
# connectome seed, initial-history seed, tract lengths / speed / dt) are kept
# as SHA-256 digests once they are larger than this
HASH_LIMIT = 300 * 1024
HASHABLE = ('weights', 'tract_lengths', 'idelays', 'buffer0', 'buffer0_fp64',
            'nnz_row', 'nnz_col', 'nnz_w', 'nnz_d')


def sha256_array(a):
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.tobytes()).hexdigest()


def compact(arrays):
    out = {}
    for k, v in arrays.items():
        base = k.split('_')[0] if k.startswith('buffer0_') and k[8:].isdigit() else k
        if (k in HASHABLE or base == 'buffer0') and isinstance(v, np.ndarray) and v.nbytes > HASH_LIMIT:
            out[k + '_sha256'] = sha256_array(v)
            out[k + '_dtype'] = str(v.dtype)
            out[k + '_shape'] = np.array(v.shape)
        else:
            out[k] = v
    return out


def save(name, **arrays):
    path = os.path.join(HERE, name + '.npz')
    np.savez_compressed(path, **compact(arrays))
    print('wrote', path, '%.1f KB' % (os.path.getsize(path) / 1024.0), flush=True)


# --------------------------------------------------------------------------- cases

def case_g2d(R):
    """Generic2dOscillator, 76 regions, Linear a=0.0152, HeunDeterministic dt 0.1,
    Raw + TemporalAverage(1 ms), 150 ms (1500 steps)."""
    w, L = synthetic_connectome(76, 0.40, 10.0, 200.0, seed=1)
    speed, dt, length = 3.0, 0.1, 150.0

    def build():
        return R['simulator'].Simulator(
            model=R['models'].Generic2dOscillator(),
            connectivity=make_conn(R, w, L, speed),
            coupling=R['coupling'].Linear(a=np.array([0.0152])),
            integrator=R['integrators'].HeunDeterministic(dt=dt),
            monitors=[R['monitors'].Raw(), R['monitors'].TemporalAverage(period=1.0)],
            simulation_length=length)
    res = {}
    for var in ('stock', 'fp64'):
        sim, cfg, out, _, el = run_sim(R, build, length, var == 'fp64', ic_seed=101)
        (tr, raw), (tt, tavg) = out
        res[var] = dict(cfg=cfg, raw=raw[..., 0], raw_t=tr, tavg=tavg[..., 0], tavg_t=tt, el=el)
    c = res['stock']['cfg']
    save('g2d_76', weights=w, tract_lengths=L, speed=speed, dt=dt, length=length,
         conn_recipe=np.array([76, 0.40, 10.0, 200.0, 1]), ic_seed=101,
         coupling_a=0.0152, **c,
         buffer0_fp64=res['fp64']['cfg']['buffer0'],
         raw=res['stock']['raw'], raw_t=res['stock']['raw_t'],
         tavg=res['stock']['tavg'], tavg_t=res['stock']['tavg_t'],
         raw_fp64=res['fp64']['raw'], tavg_fp64=res['fp64']['tavg'],
         ref_seconds=res['stock']['el'])


def case_g2d_full(R):
    """The plain method at its stated length: Generic2dOscillator, 76 regions,
    Linear a=0.0152, HeunDeterministic dt 0.1, Raw + TemporalAverage(1 ms),
    1000 ms (10 000 steps).  Keeps the TemporalAverage and every 10th Raw row
    (stock and all-float64)."""
    w, L = synthetic_connectome(76, 0.40, 10.0, 200.0, seed=1)
    speed, dt, length = 3.0, 0.1, 1000.0

    def build():
        return R['simulator'].Simulator(
            model=R['models'].Generic2dOscillator(),
            connectivity=make_conn(R, w, L, speed),
            coupling=R['coupling'].Linear(a=np.array([0.0152])),
            integrator=R['integrators'].HeunDeterministic(dt=dt),
            monitors=[R['monitors'].Raw(), R['monitors'].TemporalAverage(period=1.0)],
            simulation_length=length)
    res = {}
    for var in ('stock', 'fp64'):
        sim, cfg, out, _, el = run_sim(R, build, length, var == 'fp64', ic_seed=101)
        (tr, raw), (tt, tavg) = out
        res[var] = dict(cfg=cfg, raw=raw[9::10, ..., 0], raw_t=tr[9::10], tavg=tavg[..., 0], tavg_t=tt, el=el)
    c = res['stock']['cfg']
    save('g2d_76_full', weights=w, tract_lengths=L, speed=speed, dt=dt, length=length,
         conn_recipe=np.array([76, 0.40, 10.0, 200.0, 1]), ic_seed=101, coupling_a=0.0152, **c,
         raw_every10=res['stock']['raw'], raw_every10_t=res['stock']['raw_t'],
         raw_every10_fp64=res['fp64']['raw'],
         tavg=res['stock']['tavg'], tavg_t=res['stock']['tavg_t'], tavg_fp64=res['fp64']['tavg'],
         ref_seconds=res['stock']['el'])


def case_epi_stats(R, k, length=2000.0):
    """Instance k of the large-network batch (Epileptor, 998 regions, 10 %
    density, tract lengths 5-300 mm, speed 3 mm/ms, x0 row k of
    default_rng(14).uniform(-2.4, -1.6, (16, 998)), Difference coupling,
    HeunDeterministic dt 0.05, TemporalAverage(1 ms), initial history drawn
    after numpy.random.seed(15)) over `length` ms.  The trajectory is chaotic
    beyond a few tens of ms, so the fixture keeps statistics over the whole
    run -- per-region mean and variance of each observed variable -- and the
    TemporalAverage of 32 regions (for their FC), for the stock and the
    all-float64 reference, and for the stock reference started from a current
    state changed by 1e-7 relative (the natural scale of the divergence)."""
    w, L = synthetic_connectome(998, 0.10, 5.0, 300.0, seed=4)
    x0 = np.random.default_rng(14).uniform(-2.4, -1.6, (16, 998))[k]
    speed, dt = 3.0, 0.05
    pick = np.linspace(0, 997, 32).round().astype(int)

    def build():
        return R['simulator'].Simulator(
            model=R['models'].Epileptor(x0=x0.copy()), connectivity=make_conn(R, w, L, speed),
            coupling=R['coupling'].Difference(), integrator=R['integrators'].HeunDeterministic(dt=dt),
            monitors=[R['monitors'].TemporalAverage(period=1.0)], simulation_length=length)
    res = {}
    for var in ('stock', 'fp64', 'perturbed'):
        if var == 'perturbed':
            # the scale of chaotic divergence: the stock run from a current state changed by 1e-7 relative
            set_history_dtype(R, 'f')
            sim = build()
            np.random.seed(15)
            sim.configure()
            sim.current_state = sim.current_state * (1.0 + 1e-7)
            t0 = time.time()
            out = sim.run(simulation_length=length)
            el = time.time() - t0
            cfg = None
        else:
            sim, cfg, out, _, el = run_sim(R, build, length, var == 'fp64', ic_seed=15)
        print('epi_stats', k, var, '%.1fs' % el, flush=True)
        (tt, tavg), = out
        y = tavg[..., 0]
        res[var] = dict(cfg=cfg, mean=y.mean(axis=0), var=y.var(axis=0), sub=y[:, 0, pick], t=tt, el=el)
    c = res['stock']['cfg']
    save('epi_998_stats_%d' % k, conn_recipe=np.array([998, 0.10, 5.0, 300.0, 4]), speed=speed, dt=dt,
         length=length, x0=x0, ic_seed=15, instance=k, pick=pick, idelays=c['idelays'],
         buffer0=c['buffer0'], state0=c['state0'], tavg_t=res['stock']['t'],
         mean=res['stock']['mean'], var=res['stock']['var'], sub=res['stock']['sub'],
         mean_fp64=res['fp64']['mean'], var_fp64=res['fp64']['var'], sub_fp64=res['fp64']['sub'],
         mean_perturbed=res['perturbed']['mean'], var_perturbed=res['perturbed']['var'],
         sub_perturbed=res['perturbed']['sub'], ref_seconds=res['stock']['el'])


def case_jr(R, length=4000.0):
    """JansenRit, 192 regions, SigmoidalJansenRit, HeunStochastic dt 0.05 with
    additive nsig 1e-5 on y4 only, TemporalAverage(1 ms) + Bold(2000 ms)."""
    w, L = synthetic_connectome(192, 0.25, 5.0, 250.0, seed=2)
    speed, dt = 4.0, 0.05
    nsig = np.array([0, 0, 0, 0, 1e-5, 0.0])

    def build():
        return R['simulator'].Simulator(
            model=R['models'].JansenRit(),
            connectivity=make_conn(R, w, L, speed),
            coupling=R['coupling'].SigmoidalJansenRit(),
            integrator=R['integrators'].HeunStochastic(
                dt=dt, noise=R['noise'].Additive(nsig=nsig.copy())),
            monitors=[R['monitors'].TemporalAverage(period=1.0), R['monitors'].Bold(period=2000.0)],
            simulation_length=length)
    res = {}
    for var in ('stock', 'fp64'):
        sim, cfg, out, rec, el = run_sim(R, build, length, var == 'fp64', record_noise=True)
        (tt, tavg), (tb, bold) = out
        res[var] = dict(cfg=cfg, tavg=tavg[..., 0], tavg_t=tt, bold=bold[..., 0], bold_t=tb,
                        noise_hash=rec.h.hexdigest(), noise_count=rec.count, el=el)
        print('jr', var, el, flush=True)
    sim_model = R['models'].JansenRit()
    ranges = [sim_model.state_variable_range[sv] for sv in sim_model.state_variables]
    c = res['stock']['cfg']
    n_steps = int(np.ceil(length / dt))
    regen = regen_noise_hash(42, ranges, int(c['horizon']), 192, 6, n_steps, dt)
    assert regen == res['stock']['noise_hash'] == res['fp64']['noise_hash'], 'noise regen mismatch'
    sub = slice(19, None, 20)  # every 20th TemporalAverage sample keeps the fixture small
    save('jr_192', weights=w, tract_lengths=L, speed=speed, dt=dt, length=length, nsig=nsig,
         conn_recipe=np.array([192, 0.25, 5.0, 250.0, 2]),
         noise_seed=42, noise_regen_ok=True, noise_hash=res['stock']['noise_hash'], **c,
         tavg_index=np.arange(len(res['stock']['tavg_t']))[sub],
         tavg=res['stock']['tavg'][sub], tavg_t=res['stock']['tavg_t'][sub],
         tavg_fp64=res['fp64']['tavg'][sub],
         bold=res['stock']['bold'], bold_t=res['stock']['bold_t'], bold_fp64=res['fp64']['bold'],
         ref_seconds=res['stock']['el'])


RWW_G = np.logspace(-3, 0, 32)
RWW_NSIG = np.logspace(-4, -2, 32)


def case_rww(R, name, points, length, with_tavg):
    """ReducedWongWang, 68 regions, Linear a=G, EulerStochastic dt 0.1 with
    additive nsig, Bold(2000 ms) (+ TemporalAverage(100 ms) for short runs),
    one reference simulation per (G, nsig) sweep point."""
    w, L = synthetic_connectome(68, 0.30, 10.0, 200.0, seed=3)
    speed, dt = 5.0, 0.1
    out_arrays = {}
    for k, (gi, si) in enumerate(points):
        G, s = RWW_G[gi], RWW_NSIG[si]

        def build():
            mons = [R['monitors'].Bold(period=2000.0)]
            if with_tavg:
                mons.append(R['monitors'].TemporalAverage(period=100.0))
            return R['simulator'].Simulator(
                model=R['models'].ReducedWongWang(),
                connectivity=make_conn(R, w, L, speed),
                coupling=R['coupling'].Linear(a=np.array([G])),
                integrator=R['integrators'].EulerStochastic(
                    dt=dt, noise=R['noise'].Additive(nsig=np.array([s]))),
                monitors=mons, simulation_length=length)
        for var in ('stock', 'fp64'):
            sim, cfg, out, rec, el = run_sim(R, build, length, var == 'fp64', record_noise=True)
            print(name, k, var, '%.1fs' % el, flush=True)
            tb, bold = out[0]
            sfx = '' if var == 'stock' else '_fp64'
            out_arrays['bold%s_%d' % (sfx, k)] = bold[..., 0]
            if with_tavg:
                out_arrays['tavg%s_%d' % (sfx, k)] = out[1][1][..., 0]
                out_arrays['tavg_t'] = out[1][0]
            out_arrays['bold_t'] = tb
            if var == 'stock':
                out_arrays['noise_hash_%d' % k] = rec.h.hexdigest()
                cfg0 = cfg
                out_arrays['buffer0_%d' % k] = cfg['buffer0']
                out_arrays['state0_%d' % k] = cfg['state0']
                out_arrays['ref_seconds_%d' % k] = el
                hrf = sim.monitors[0].hemodynamic_response_function[0]
        # FC exactly as the framework analyzer does it: corrcoef over time
        out_arrays['fc_%d' % k] = np.corrcoef(out_arrays['bold_%d' % k][:, 0, :].T)
        out_arrays['fc_fp64_%d' % k] = np.corrcoef(out_arrays['bold_fp64_%d' % k][:, 0, :].T)
    ranges = [R['models'].ReducedWongWang().state_variable_range['S']]
    n_steps = int(np.ceil(length / dt))
    regen = regen_noise_hash(42, ranges, int(cfg0['horizon']), 68, 1, n_steps, dt)
    for k in range(len(points)):
        assert out_arrays['noise_hash_%d' % k] == regen, 'noise regen mismatch'
    c = {k: v for k, v in cfg0.items() if k not in ('buffer0', 'state0')}
    save(name, weights=w, tract_lengths=L, speed=speed, dt=dt, length=length,
         conn_recipe=np.array([68, 0.30, 10.0, 200.0, 3]),
         G=np.array([RWW_G[g] for g, _ in points]), nsig=np.array([RWW_NSIG[s] for _, s in points]),
         point_index=np.array(points), noise_seed=42, noise_regen_ok=True, hrf=hrf,
         **c, **out_arrays)


def case_epi(R, name, n, density, length, gains, seed):
    """Epileptor with x0 ~ U[-2.4,-1.6] per region, Difference coupling,
    HeunDeterministic dt 0.05, TemporalAverage(1 ms)."""
    w, L = synthetic_connectome(n, density, 5.0, 300.0, seed=seed)
    x0 = np.random.default_rng(seed + 1000).uniform(-2.4, -1.6, n)
    speed, dt = 3.0, 0.05

    def build():
        m = R['models'].Epileptor(x0=x0.copy(), **{k: np.array([v]) for k, v in gains.items()})
        return R['simulator'].Simulator(
            model=m, connectivity=make_conn(R, w, L, speed),
            coupling=R['coupling'].Difference(),
            integrator=R['integrators'].HeunDeterministic(dt=dt),
            monitors=[R['monitors'].TemporalAverage(period=1.0)],
            simulation_length=length)
    res = {}
    for var in ('stock', 'fp64'):
        sim, cfg, out, _, el = run_sim(R, build, length, var == 'fp64', ic_seed=seed + 200)
        print(name, var, '%.1fs' % el, flush=True)
        (tt, tavg), = out
        res[var] = dict(cfg=cfg, tavg=tavg[..., 0], tavg_t=tt, el=el)
    c = res['stock']['cfg']
    save(name, weights=w, tract_lengths=L, speed=speed, dt=dt, length=length, x0=x0,
         conn_recipe=np.array([n, density, 5.0, 300.0, seed]), ic_seed=seed + 200,
         gain_names=np.array(list(gains.keys())), gain_values=np.array(list(gains.values()), dtype=float),
         **c, tavg=res['stock']['tavg'], tavg_t=res['stock']['tavg_t'],
         tavg_fp64=res['fp64']['tavg'], ref_seconds=res['stock']['el'])


def case_propagation(R):
    """Exact delayed propagation on a 4-node chain: identity coupling, a model
    whose derivative is state + coupling, the Identity integrator, dt = 1,
    tract lengths 0..15 at speed 1 and a provided 16-step initial history of
    ones (this also starts the loop at current_step = 15)."""
    models, coupling = R['models'], R['coupling']

    class PassThrough(coupling.SparseCoupling):
        def pre(self, x_i, x_j):
            return x_j

        def post(self, gx):
            return gx

    class StatePlusInput(models.Model):
        nvar = 1
        _nvar = 1
        state_variable_range = {'x': [0, 100]}
        variables_of_interest = R['List'](of=str, default=('x',), choices=('x',))
        state_variables = ('x',)
        cvar = np.array([0])

        def dfun(self, X, c, local_coupling=0):
            return X + c + local_coupling

    n = 4
    w = np.zeros((n, n))
    for i in range(n - 1):
        w[i, i + 1] = 1.0
    L = np.arange(n * n, dtype=float).reshape((n, n))
    sim = R['simulator'].Simulator(
        conduction_speed=1.0, coupling=PassThrough(), integrator=R['integrators'].Identity(dt=1.0),
        initial_conditions=np.ones((n * n, 1, n, 1)), simulation_length=10.0,
        connectivity=R['Connectivity'](region_labels=np.array(['']), weights=w, tract_lengths=L,
                                       speed=np.array([1.0]), centres=np.array([0.0])),
        model=StatePlusInput(), monitors=(R['monitors'].Raw(),))
    sim.configure()
    cfg = configured_state(sim)
    xs = np.array([raw.flat[:].copy() for (t, raw), in sim(simulation_length=10)])
    save('propagation_4', weights=w, tract_lengths=L, speed=1.0, dt=1.0, **cfg, raw=xs)


def case_steady(R):
    """Single-node fixed points reached by Model.stationary_trajectory (Euler,
    dt 0.01, 2000 steps, zero coupling, start at the middle of each state range)."""
    out = {}
    for name in ('Generic2dOscillator', 'JansenRit', 'ReducedWongWang'):
        model = getattr(R['models'], name)()
        model.configure()
        nv = len(model.state_variables)
        init = np.zeros((nv, 1))
        for i, (lo, hi) in enumerate(model.state_variable_range.values()):
            init[i, :] = (hi + lo) / 2.0
        t, y = model.stationary_trajectory(initial_conditions=init, n_step=2000, dt=0.01)
        out[name + '_init'] = init[:, 0]
        out[name + '_traj'] = y[:, :, 0, 0]
    save('steady_state', **out)


def case_idelays(R):
    """Conduction delays in integration steps at and near rounding ties."""
    rng = np.random.default_rng(7)
    n = 24
    L = rng.uniform(0.0, 60.0, (n, n))
    # exact .5 ties at speed 1, dt 1 and decimal values near ties at dt 0.1 / 0.05
    L[0, :12] = np.arange(12) + 0.5
    L[1, :12] = (np.arange(12) + 0.5) * 0.1
    L[2, :12] = np.round(rng.uniform(0, 30, 12), 2)
    L[3, :12] = (np.arange(12) * 0.05 + 0.025)
    res = {}
    for speed in (1.0, 3.0, 4.0, 5.0):
        for dt in (1.0, 0.1, 0.05, 0.0125):
            c = R['Connectivity'](weights=np.ones((n, n)), tract_lengths=L, speed=np.array([speed]),
                                  region_labels=np.array(['r%d' % i for i in range(n)]),
                                  centres=np.zeros((n, 3)))
            c.configure()
            c.set_idelays(dt)
            res['idelays_s%g_dt%g' % (speed, dt)] = np.asarray(c.idelays, dtype=np.int32)
            res['horizon_s%g_dt%g' % (speed, dt)] = np.int64(c.horizon)
    save('idelays', tract_lengths=L, **res)


def case_difference(R):
    """Difference coupling on two nodes with zero delays (state 1 and 2)."""
    H = R['history']
    w = np.array([[0.0, 1.0], [1.0, 0.0]])
    hist = H.SparseHistory(w, np.zeros((2, 2), dtype=int), np.r_[0], 1)
    hist.update(0, np.array([[[1.0], [2.0]]]))
    k = R['coupling'].Difference()
    k.configure()
    res = k(0 + 1, hist)  # coupling for step 1 reads the state stored at step 0
    lin = R['coupling'].Linear(a=np.array([0.5]), b=np.array([0.25]))
    lin.configure()
    res_lin = lin(1, hist)
    save('difference_2', weights=w, state=np.array([1.0, 2.0]), difference=res[:, :, 0],
         a=0.1, linear=res_lin[:, :, 0], linear_a=0.5, linear_b=0.25)


def case_couplings(R):
    """The couplings beyond Linear / Difference / SigmoidalJansenRit and the
    Runge-Kutta scheme: Generic2dOscillator, 40 regions (40 % density, tract
    lengths 10-120 mm, speed 3 mm/ms), Raw, 40 ms at dt 0.1 with Scaling,
    Sigmoidal, HyperbolicTangent, Kuramoto (HeunDeterministic) and Linear with
    RungeKutta4thOrderDeterministic; Epileptor (two coupling variables) with
    HyperbolicTangent, HeunDeterministic dt 0.05, TemporalAverage 1 ms, 20 ms."""
    w, L = synthetic_connectome(40, 0.40, 10.0, 120.0, seed=21)
    speed = 3.0
    C, I = R['coupling'], R['integrators']
    cases = {
        'scaling': (C.Scaling(a=np.array([0.02])), I.HeunDeterministic(dt=0.1)),
        'sigmoidal': (C.Sigmoidal(cmin=np.array([-0.5]), cmax=np.array([0.5]), midpoint=np.array([0.5]),
                                  a=np.array([1.2]), sigma=np.array([4.0])), I.HeunDeterministic(dt=0.1)),
        'tanh': (C.HyperbolicTangent(a=np.array([0.05]), b=np.array([0.8]), midpoint=np.array([0.3]),
                                     sigma=np.array([2.0])), I.HeunDeterministic(dt=0.1)),
        'kuramoto': (C.Kuramoto(a=np.array([0.3])), I.HeunDeterministic(dt=0.1)),
        'rk4': (C.Linear(a=np.array([0.0152])), I.RungeKutta4thOrderDeterministic(dt=0.1)),
    }
    out = dict(weights=w, tract_lengths=L, speed=speed, conn_recipe=np.array([40, 0.40, 10.0, 120.0, 21]),
               ic_seed=202)
    for name, (cf, integ) in cases.items():
        def build(cf=cf, integ=integ):
            return R['simulator'].Simulator(
                model=R['models'].Generic2dOscillator(), connectivity=make_conn(R, w, L, speed), coupling=cf,
                integrator=integ, monitors=[R['monitors'].Raw()], simulation_length=40.0)
        sim, cfg, res, _, _ = run_sim(R, build, 40.0, False, ic_seed=202)
        (t, raw), = res
        out[name + '_raw'] = raw[..., 0]
        out[name + '_t'] = t
        out[name + '_buffer0'] = cfg['buffer0']
        out[name + '_state0'] = cfg['state0']

    def build_epi():
        return R['simulator'].Simulator(
            model=R['models'].Epileptor(), connectivity=make_conn(R, w, L, speed),
            coupling=C.HyperbolicTangent(a=np.array([0.02]), b=np.array([1.0]), midpoint=np.array([-1.0]),
                                         sigma=np.array([1.5])),
            integrator=I.HeunDeterministic(dt=0.05), monitors=[R['monitors'].TemporalAverage(period=1.0)],
            simulation_length=20.0)
    sim, cfg, res, _, _ = run_sim(R, build_epi, 20.0, False, ic_seed=203)
    (t, tavg), = res
    out.update(epi_tanh_tavg=tavg[..., 0], epi_tanh_t=t, epi_tanh_buffer0=cfg['buffer0'],
               epi_tanh_state0=cfg['state0'])
    save('couplings_40', **out)


def case_monitors(R):
    """SubSample, GlobalAverage and SpatialAverage (period 1 ms) beside Raw and
    TemporalAverage: Generic2dOscillator, the 40-region connectome of
    case_couplings, Linear a=0.0152, HeunDeterministic dt 0.1, 40 ms; and the
    same monitors on ReducedWongWang with EulerStochastic (reference noise)."""
    w, L = synthetic_connectome(40, 0.40, 10.0, 120.0, seed=21)
    speed = 3.0
    mask = np.arange(40) % 3
    M = R['monitors']

    def mons():
        return [M.SubSample(period=1.0), M.GlobalAverage(period=1.0),
                M.SpatialAverage(period=1.0, spatial_mask=mask), M.TemporalAverage(period=1.0)]

    def build():
        return R['simulator'].Simulator(
            model=R['models'].Generic2dOscillator(), connectivity=make_conn(R, w, L, speed),
            coupling=R['coupling'].Linear(a=np.array([0.0152])),
            integrator=R['integrators'].HeunDeterministic(dt=0.1), monitors=mons(), simulation_length=40.0)
    sim, cfg, res, _, _ = run_sim(R, build, 40.0, False, ic_seed=204)
    out = dict(weights=w, tract_lengths=L, speed=speed, spatial_mask=mask, ic_seed=204,
               g2d_buffer0=cfg['buffer0'], g2d_state0=cfg['state0'])
    for name, (t, y) in zip(('sub', 'glob', 'spat', 'tavg'), res):
        out['g2d_%s' % name] = y[..., 0]
        out['g2d_%s_t' % name] = t

    def build_rww():
        return R['simulator'].Simulator(
            model=R['models'].ReducedWongWang(), connectivity=make_conn(R, w, L, speed),
            coupling=R['coupling'].Linear(a=np.array([0.3])),
            integrator=R['integrators'].EulerStochastic(dt=0.1, noise=R['noise'].Additive(nsig=np.array([1e-3]))),
            monitors=mons(), simulation_length=40.0)
    sim, cfg, res, rec, _ = run_sim(R, build_rww, 40.0, False, record_noise=True)
    out.update(rww_buffer0=cfg['buffer0'], rww_state0=cfg['state0'], rww_noise_sha256=rec.h.hexdigest())
    for name, (t, y) in zip(('sub', 'glob', 'spat', 'tavg'), res):
        out['rww_%s' % name] = y[..., 0]
    save('monitors_40', **out)


def case_balloon(R):
    """BalloonModel (tvb/analyzers/fmri_balloon.py) on a seeded smooth random
    series (3000 samples at 1 ms, 2 variables, 6 regions, 1 mode) for the
    non-linear and linear BOLD equations, the classical and revised
    coefficients, and the none / sum / abs_diff input transformations with
    and without mean subtraction."""
    from tvb.datatypes.time_series import TimeSeries
    from tvb.analyzers.fmri_balloon import BalloonModel, BoldModels, NeuralInputTransformations as NIT
    rng = np.random.default_rng(5)
    T, n = 3000, 6
    x = np.cumsum(rng.normal(size=(T, 2, n, 1)), axis=0) * 0.01 + 0.1
    out = dict(x=x)
    cases = {'nl_rbm_none': dict(),
             'lin_rbm_sum': dict(bold_model=BoldModels.LINEAR, neural_input_transformation=NIT.SUM),
             'nl_cbm_absdiff': dict(RBM=False, neural_input_transformation=NIT.ABS_DIFF),
             'nl_rbm_norm': dict(normalize_neural_input=True)}
    for name, kw in cases.items():
        ts = TimeSeries(data=x, sample_period=1.0, sample_period_unit='ms', time=np.arange(T) * 1.0)
        bm = BalloonModel(time_series=ts, **kw)
        res = bm.evaluate()
        out[name] = res.data
        out[name + '_t'] = res.time
    save('balloon', **out)


def case_stimulus(R):
    """Region stimuli (StimuliRegion: temporal equation x region weights) on
    the 40-region connectome of case_couplings: Generic2dOscillator with a
    PulseTrain (HeunDeterministic, Raw + TemporalAverage 1 ms, 60 ms);
    Generic2dOscillator with stvar = [1] and a Sinusoid (EulerDeterministic,
    Raw, 40 ms); ReducedWongWang with an Alpha pulse (EulerStochastic,
    reference noise, Raw, 40 ms); Epileptor with a Gaussian
    (RungeKutta4thOrderDeterministic dt 0.05, Raw, 20 ms).  Each case keeps
    the reference's temporal and spatial patterns."""
    w, L = synthetic_connectome(40, 0.40, 10.0, 120.0, seed=21)
    speed = 3.0
    E, P, M, I, C = R['equations'], R['patterns'], R['models'], R['integrators'], R['coupling']
    rng = np.random.default_rng(31)
    weight = np.where(rng.random(40) < 0.5, rng.uniform(0.5, 2.0, 40), 0.0)
    out = dict(weights=w, tract_lengths=L, speed=speed, stim_weight=weight)

    def g2d_w():
        m = M.Generic2dOscillator()
        m.stvar = np.array([1], dtype=np.int32)
        return m
    cases = {
        'g2d_pulse': (M.Generic2dOscillator, C.Linear(a=np.array([0.0152])), lambda: I.HeunDeterministic(dt=0.1),
                      E.PulseTrain(parameters={'T': 12.0, 'tau': 4.0, 'amp': 2.0, 'onset': 5.0}),
                      lambda: [R['monitors'].Raw(), R['monitors'].TemporalAverage(period=1.0)], 60.0, 301),
        'g2d_w_sin': (g2d_w, C.Linear(a=np.array([0.0152])), lambda: I.EulerDeterministic(dt=0.1),
                      E.Sinusoid(parameters={'amp': 0.5, 'frequency': 0.05}),
                      lambda: [R['monitors'].Raw()], 40.0, 302),
        'rww_alpha': (M.ReducedWongWang, C.Linear(a=np.array([0.3])),
                      lambda: I.EulerStochastic(dt=0.1, noise=R['noise'].Additive(nsig=np.array([1e-4]))),
                      E.Alpha(parameters={'onset': 3.0, 'alpha': 0.5, 'beta': 1.0}),
                      lambda: [R['monitors'].Raw()], 40.0, None),
        'epi_gauss': (M.Epileptor, C.Linear(a=np.array([0.01])), lambda: I.RungeKutta4thOrderDeterministic(dt=0.05),
                      E.Gaussian(parameters={'amp': 1.5, 'sigma': 4.0, 'midpoint': 10.0, 'offset': 0.0}),
                      lambda: [R['monitors'].Raw()], 20.0, 303),
    }
    for name, (model, cf, integ, eq, mons, length, seed) in cases.items():
        def build(model=model, cf=cf, integ=integ, eq=eq, mons=mons, length=length):
            conn = make_conn(R, w, L, speed)
            stim = P.StimuliRegion(temporal=eq, connectivity=conn, weight=weight)
            return R['simulator'].Simulator(model=model(), connectivity=conn, coupling=cf, integrator=integ(),
                                            monitors=mons(), simulation_length=length, stimulus=stim)
        sim, cfg, res, rec, _ = run_sim(R, build, length, False, ic_seed=seed, record_noise=seed is None)
        out[name + '_temporal'] = np.asarray(sim.stimulus.temporal_pattern).reshape(-1)
        out[name + '_spatial'] = np.asarray(sim.stimulus.spatial_pattern).reshape(-1)
        out[name + '_stvar'] = np.asarray(sim.model.stvar, dtype=np.int32)
        out[name + '_buffer0'] = cfg['buffer0']
        out[name + '_state0'] = cfg['state0']
        for k, (t, y) in enumerate(res):
            out['%s_m%d' % (name, k)] = y[..., 0]
            out['%s_m%d_t' % (name, k)] = t
        if rec is not None:
            out[name + '_noise_sha256'] = rec.h.hexdigest()
    # two calls of 30 ms: the reference evaluates the temporal pattern again at each call, from its start
    def build2():
        conn = make_conn(R, w, L, speed)
        stim = P.StimuliRegion(temporal=E.PulseTrain(parameters={'T': 12.0, 'tau': 4.0, 'amp': 2.0, 'onset': 5.0}),
                               connectivity=conn, weight=weight)
        return R['simulator'].Simulator(model=M.Generic2dOscillator(), connectivity=conn,
                                        coupling=C.Linear(a=np.array([0.0152])),
                                        integrator=I.HeunDeterministic(dt=0.1), monitors=[R['monitors'].Raw()],
                                        simulation_length=30.0, stimulus=stim)
    sim, cfg, res, _, _ = run_sim(R, build2, 30.0, False, ic_seed=301)
    (t1, y1), = res
    (t2, y2), = sim.run(simulation_length=30.0)
    out.update(g2d_2x_buffer0=cfg['buffer0'], g2d_2x_state0=cfg['state0'], g2d_2x_t=np.concatenate([t1, t2]),
               g2d_2x_raw=np.concatenate([y1, y2])[..., 0])
    save('stimulus_40', **out)


def case_afferent(R):
    """AfferentCoupling and AfferentCouplingTemporalAverage (the coupling each
    step receives next) on the 40-region connectome of case_couplings:
    Generic2dOscillator with Linear a=0.0152 (HeunDeterministic dt 0.1, 40 ms,
    both monitors and Raw); Epileptor with Difference a=0.1 (two coupling
    variables, HeunDeterministic dt 0.05, 20 ms, AfferentCoupling and the
    period-1 ms average of coupling variable 1); JansenRit with
    SigmoidalJansenRit (one coupling row, HeunDeterministic dt 0.1, 40 ms)."""
    w, L = synthetic_connectome(40, 0.40, 10.0, 120.0, seed=21)
    speed = 3.0
    M, I, C = R['models'], R['integrators'], R['coupling']
    Mo = R['monitors']
    out = dict(weights=w, tract_lengths=L, speed=speed)
    cases = {
        'g2d': (M.Generic2dOscillator, lambda: C.Linear(a=np.array([0.0152])), 0.1, 40.0, 401,
                lambda: [Mo.AfferentCoupling(), Mo.AfferentCouplingTemporalAverage(period=1.0), Mo.Raw()]),
        'epi': (M.Epileptor, lambda: C.Difference(a=np.array([0.1])), 0.05, 20.0, 402,
                lambda: [Mo.AfferentCoupling(),
                         Mo.AfferentCouplingTemporalAverage(period=1.0, variables_of_interest=np.array([1]))]),
        'jr': (M.JansenRit, lambda: C.SigmoidalJansenRit(a=np.array([10.0])), 0.1, 40.0, 403,
               lambda: [Mo.AfferentCoupling(variables_of_interest=np.array([0])),
                        Mo.AfferentCouplingTemporalAverage(period=2.0, variables_of_interest=np.array([0]))]),
    }
    for name, (model, cf, dt, length, seed, mons) in cases.items():
        def build(model=model, cf=cf, dt=dt, mons=mons, length=length):
            return R['simulator'].Simulator(model=model(), connectivity=make_conn(R, w, L, speed), coupling=cf(),
                                            integrator=I.HeunDeterministic(dt=dt), monitors=mons(),
                                            simulation_length=length)
        sim, cfg, res, _, _ = run_sim(R, build, length, False, ic_seed=seed)
        out[name + '_buffer0'] = cfg['buffer0']
        out[name + '_state0'] = cfg['state0']
        for k, (t, y) in enumerate(res):
            out['%s_m%d' % (name, k)] = y[..., 0]
            out['%s_m%d_t' % (name, k)] = t
    save('afferent_40', **out)


def case_projection(R):
    """EEG / MEG / iEEG monitors on Generic2dOscillator (the 40-region
    connectome of case_couplings, Linear a=0.0152, HeunDeterministic dt 0.1,
    40 ms) with seeded synthetic sensors, region centres / orientations and
    lead fields over a 200-vertex source space: EEG (16 sensors, average
    reference, default observation noise) and MEG (12 sensors, no
    observation noise) at period 1000/1024 ms (9 steps); iEEG (10 sensors,
    observation noise, 4 non-cortical regions with the analytic lead field)
    alone at period 2 ms."""
    w, L = synthetic_connectome(40, 0.40, 10.0, 120.0, seed=21)
    speed = 3.0
    n, V = 40, 200
    rng = np.random.default_rng(41)
    centres = rng.normal(size=(n, 3)) * 30.0
    ori = rng.normal(size=(n, 3))
    ori /= np.sqrt((ori ** 2).sum(axis=1))[:, None]
    rmap = np.concatenate([np.arange(n), rng.integers(0, n, V - n)])
    cortical = np.ones(n, dtype=bool)
    cortical[[3, 11, 27, 38]] = False
    sens = {k: rng.normal(size=(S, 3)) * 90.0 for k, S in (('eeg', 16), ('meg', 12), ('ieeg', 10))}
    lead = {'eeg': rng.normal(size=(16, V)), 'meg': rng.normal(size=(12, V)) * 1e-3,
            'ieeg': rng.normal(size=(10, int((~np.isin(rmap, np.flatnonzero(~cortical))).sum())))}
    out = dict(weights=w, tract_lengths=L, speed=speed, centres=centres, orientations=ori, rmap=rmap,
               cortical=cortical, **{'sensors_' + k: v for k, v in sens.items()},
               **{'lead_' + k: v for k, v in lead.items()})
    S_, P_, RM, Mo = R['sensors'], R['projections'], R['region_mapping'], R['monitors']

    def conn(with_cortical):
        c = make_conn(R, w, L, speed)
        c.centres = centres
        c.orientations = ori
        c.cortical = cortical if with_cortical else np.ones(n, dtype=bool)
        return c

    def labels(k, S):
        return np.array(['%s%d' % (k, i) for i in range(S)])

    cases = {
        'em': (False, lambda c: [
            Mo.EEG(period=1e3 / 1024.0, sensors=S_.SensorsEEG(labels=labels('e', 16), locations=sens['eeg']),
                   projection=P_.ProjectionSurfaceEEG(projection_data=lead['eeg']),
                   region_mapping=RM.RegionMapping(array_data=rmap, connectivity=c), reference='average'),
            Mo.MEG(period=1e3 / 1024.0, sensors=S_.SensorsMEG(labels=labels('m', 12), locations=sens['meg'],
                                                               orientations=np.tile([0.0, 0.0, 1.0], (12, 1))),
                   projection=P_.ProjectionSurfaceMEG(projection_data=lead['meg']),
                   region_mapping=RM.RegionMapping(array_data=rmap, connectivity=c), obsnoise=None)], 501),
        'ieeg': (True, lambda c: [
            Mo.iEEG(period=2.0, sensors=S_.SensorsInternal(labels=labels('i', 10), locations=sens['ieeg']),
                    projection=P_.ProjectionSurfaceSEEG(projection_data=lead['ieeg']),
                    region_mapping=RM.RegionMapping(array_data=rmap, connectivity=c))], 502),
    }
    for name, (with_cortical, mons, seed) in cases.items():
        def build(with_cortical=with_cortical, mons=mons):
            c = conn(with_cortical)
            return R['simulator'].Simulator(
                model=R['models'].Generic2dOscillator(), connectivity=c,
                coupling=R['coupling'].Linear(a=np.array([0.0152])),
                integrator=R['integrators'].HeunDeterministic(dt=0.1), monitors=mons(c), simulation_length=40.0)
        sim, cfg, res, _, _ = run_sim(R, build, 40.0, False, ic_seed=seed)
        out[name + '_buffer0'] = cfg['buffer0']
        out[name + '_state0'] = cfg['state0']
        for k, (t, y) in enumerate(res):
            out['%s_m%d' % (name, k)] = y[..., 0]
            out['%s_m%d_t' % (name, k)] = t
            out['%s_m%d_gain' % (name, k)] = np.array(sim.monitors[k].gain)
    # the analytic lead fields (Sarvas 1987) on their own, for 8 sources
    src, so = centres[:8], ori[:8]
    out['eeg_analytic'] = Mo.EEG(sensors=S_.SensorsEEG(labels=labels('e', 16), locations=sens['eeg']),
                                 sigma=0.7).analytic(src, so)
    out['meg_analytic'] = Mo.MEG(sensors=S_.SensorsMEG(labels=labels('m', 12), locations=sens['meg'],
                                                       orientations=np.tile([0.0, 0.0, 1.0], (12, 1)))).analytic(src, so)
    out['ieeg_analytic'] = Mo.iEEG(sensors=S_.SensorsInternal(labels=labels('i', 10), locations=sens['ieeg']),
                                   sigma=0.7).analytic(src, so)
    save('projection_40', **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=os.environ.get('TVB_REFERENCE_LIBRARY'),
                    required='TVB_REFERENCE_LIBRARY' not in os.environ,
                    help='the reference\'s tvb_library source directory (default: $TVB_REFERENCE_LIBRARY)')
    ap.add_argument('--only', nargs='*')
    ap.add_argument('--compact', nargs='*', help='re-save existing fixtures with large inputs hashed')
    args = ap.parse_args()
    if args.compact:
        for path in args.compact:
            d = dict(np.load(path, allow_pickle=False))
            np.savez_compressed(path, **compact(d))
            print('compacted', path, '%.1f KB' % (os.path.getsize(path) / 1024.0))
        return
    R = import_reference(args.ref)
    cases = {
        'propagation': lambda: case_propagation(R),
        'steady': lambda: case_steady(R),
        'idelays': lambda: case_idelays(R),
        'difference': lambda: case_difference(R),
        'g2d': lambda: case_g2d(R),
        'g2d_full': lambda: case_g2d_full(R),
        'epi_stats_0': lambda: case_epi_stats(R, 0),
        'epi_stats_1': lambda: case_epi_stats(R, 1),
        'epi': lambda: case_epi(R, 'epi_998', 998, 0.10, 60.0, {}, seed=4),
        'epi_coupled': lambda: case_epi(R, 'epi_96_coupled', 96, 0.3, 200.0,
                                        {'Ks': -0.2, 'Kf': 0.05, 'Kvf': 0.02}, seed=14),
        'rww_short': lambda: case_rww(R, 'rww_68_short', [(0, 0), (10, 20), (20, 5), (31, 31)],
                                      10000.0, True),
        'rww_full': lambda: case_rww(R, 'rww_68_full', [(16, 16), (31, 8)], 60000.0, False),
        'jr': lambda: case_jr(R),
        'couplings': lambda: case_couplings(R),
        'monitors': lambda: case_monitors(R),
        'balloon': lambda: case_balloon(R),
        'stimulus': lambda: case_stimulus(R),
        'afferent': lambda: case_afferent(R),
        'projection': lambda: case_projection(R),
    }
    for name, fn in cases.items():
        if args.only and name not in args.only:
            continue
        t0 = time.time()
        fn()
        print('case', name, 'done in %.1fs' % (time.time() - t0), flush=True)


if __name__ == '__main__':
    main()
