#!/usr/bin/env python
"""Benchmark of the batched region simulation loop on B200.

Workload (one bench step): the ReducedWongWang parameter sweep -- 68-region
seeded synthetic connectome (30 % density, tract lengths 10-200 mm, speed
5 mm/ms), Linear coupling with G over 32 log-spaced values in [0.001, 1] x
additive noise nsig over 32 log-spaced values in [1e-4, 1e-2] = 1024
instances, EulerStochastic dt 0.1 ms, 60 s each (600 000 steps), Bold
(TR 2000 ms, float64 accumulation) and per-instance FC on the device.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line.  `value` is region-steps/s of the device path with the
inputs resident in HBM (kernel launches of the sweep + FC, CUDA events);
`e2e` is the same metric through the public ParameterSweep API from host
arrays to host results, transfers included.  Under torchrun with N ranks the
global sweep is N x 1024 instances (N independent noise realisations of the
grid: instance g is grid point g % 1024 with Philox stream g) and each rank
runs its own 1024-instance shard (weak scaling, no collective on the data
path); the time is the max over ranks.  At N = 1 the line also carries the
Philox-path parity check against the oracle (Bold, state, FC), the serving
leg (p50/p99 latency at a stated Poisson rate) and the large-network leg
(region-steps/s and per-instance error against the float64 oracle).
`cpu_baseline` runs one instance per host core, spread over the (G, nsig)
grid, for the full 60 s (600 000 steps).  `--impl reference` times the CPU
oracle (a numpy restatement of the reference's numpy path) on the host
cores, each step a shorter sample of the same kind (--ref-sample-steps).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, 'tvb-root_b200'))

import numpy as np  # noqa: E402

METRIC = 'region-steps/sec batched FP32 vs plain, err vs FP64 oracle; p50/p99 sim latency'
PHILOX_SEED = 42      # the sweep's noise_seed (Additive default)
UNIT = 'region-steps/s'
N_REGIONS, DENSITY, L_LO, L_HI, SPEED, SEED = 68, 0.30, 10.0, 200.0, 5.0, 3
DT = 0.1


def sweep_grid():
    G = np.logspace(-3, 0, 32)
    S = np.logspace(-4, -2, 32)
    gg, ss = np.meshgrid(G, S, indexing='ij')
    return gg.reshape(-1), ss.reshape(-1)


def make_sweep(instances, length_ms, rank=0, world=1, chunk=None, gather='auto', lanes=1, select=None):
    """The sweep of `instances` x `world` global instances: global instance g
    is grid point g % 1024 with its own Philox stream g (for world > 1, one
    independent noise realisation of the grid per rank); this process runs
    shard `rank` of `world` (weak scaling: `instances` per rank), or the
    global indices in `select`."""
    from tvb_b200 import coupling, integrators, models, monitors, noise, synthetic
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.sweep import ParameterSweep
    w, L = synthetic.connectome(N_REGIONS, DENSITY, L_LO, L_HI, seed=SEED)
    G, S = sweep_grid()
    idx = np.arange(instances * world) % G.size
    where = dict(instances=select) if select is not None else dict(shard=(rank, world))
    sw = ParameterSweep(model=models.ReducedWongWang(), connectivity=Connectivity(w, L, speed=SPEED),
                        coupling=coupling.Linear(), monitors=[monitors.Bold(period=2000.0)],
                        integrator=integrators.EulerStochastic(dt=DT, noise=noise.Additive(nsig=[1e-3])),
                        simulation_length=length_ms, sweep={'coupling.a': G[idx], 'noise.nsig': S[idx]},
                        chunk_steps=chunk, gather=gather, lanes=lanes, **where)
    return sw


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
              'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
              'clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(',')]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith('active'):
                    reasons.add(nm)
        if not sm:
            return None
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': float(max(mx)), 'reasons': sorted(reasons),
                'samples': len(sm)}


# -------------------------------------------------------------- CPU oracle

def _oracle_worker(args):
    """One sweep instance on the CPU oracle (numpy restatement of the
    reference's numpy path), including its per-step normal draws like the
    reference's RandomState path; returns the seconds it took."""
    g, n_steps, G, nsig = args
    os.environ['OMP_NUM_THREADS'] = '1'
    from oracle import tvb_oracle as O
    from tvb_b200 import synthetic
    w, L = synthetic.connectome(N_REGIONS, DENSITY, L_LO, L_HI, seed=SEED)
    idl, H = O.integer_delays(L, SPEED, DT)
    info = O.MODEL_INFO['ReducedWongWang']
    rs = np.random.RandomState(42)
    hist = O.reference_initial_history(rs, [info['ranges']['S']], H, N_REGIONS)
    t0 = time.perf_counter()
    z = rs.normal(size=(n_steps, 1, N_REGIONS))
    O.simulate('ReducedWongWang', {}, w, L, SPEED, DT, 'Linear', {'a': G}, 'EulerStochastic', n_steps,
               [O.Monitor('Bold', 2000.0)], hist[:, [0]].astype(np.float32), hist[0], 0, nsig=[nsig], noise_z=z)
    return time.perf_counter() - t0


def _warm(_):
    os.environ['OMP_NUM_THREADS'] = '1'
    from oracle import tvb_oracle  # noqa: F401
    from tvb_b200 import synthetic  # noqa: F401
    return os.getpid()


def cpu_sample(pool, cores, n_steps, offset=0):
    """One sample of the sweep on the host: `cores` instances spread over the
    (G, nsig) grid (shifted by `offset` grid points), one per core, n_steps
    each.  Returns (wall seconds of the whole sample, global indices)."""
    G, S = sweep_grid()
    pick = (np.linspace(0, G.size - 1, cores).astype(int) + offset) % G.size
    t0 = time.perf_counter()
    pool.map(_oracle_worker, [(int(i), n_steps, G[i], S[i]) for i in pick])
    return time.perf_counter() - t0, pick


def _sample_text(cores, n_steps):
    return ('%d RWW sweep instances spread over the 32 x 32 (G, nsig) grid, one per core, %d steps (%g ms) each, '
            'oracle numpy path incl. per-step noise draws; value = instances x steps x regions / wall time of the '
            'sample' % (cores, n_steps, n_steps * DT))


def cpu_baseline(n_steps=600000, cores=None):
    import multiprocessing as mp
    cores = cores or os.cpu_count() or 1
    with mp.get_context('spawn').Pool(cores) as pool:
        pool.map(_warm, range(cores))
        wall, _ = cpu_sample(pool, cores, n_steps)
    return {'value': cores * n_steps * N_REGIONS / wall, 'unit': UNIT, 'cores': cores, 'kind': 'port',
            'sample': _sample_text(cores, n_steps), 'wall_s': wall}


def _philox_oracle_worker(args):
    """One sweep instance on the CPU oracle fed the device's Philox normals of
    its global index: the stock variant (float32 history and weights, like
    the reference) or the all-float64 one."""
    g, n_steps, G, nsig, buf0, st0, variant = args
    os.environ['OMP_NUM_THREADS'] = '1'
    from oracle import tvb_oracle as O
    from tvb_b200 import synthetic
    w, L = synthetic.connectome(N_REGIONS, DENSITY, L_LO, L_HI, seed=SEED)
    z = O.philox_normals(PHILOX_SEED, g, np.arange(1, n_steps + 1), 1, N_REGIONS)
    # the initial history as the reference draws it (float64; the stock variant keeps it in float32)
    idl, H = O.integer_delays(L, SPEED, DT)
    h64 = O.reference_initial_history(np.random.RandomState(PHILOX_SEED),
                                      [O.MODEL_INFO['ReducedWongWang']['ranges']['S']], H, N_REGIONS)
    assert np.array_equal(h64[:, [0]].astype(np.float32), buf0) and np.array_equal(h64[0], st0)
    kw = dict(history_dtype=np.float64) if variant == 'fp64' else {}
    hist = h64[:, [0]] if variant == 'fp64' else buf0
    out, fin = O.simulate('ReducedWongWang', {}, w, L, SPEED, DT, 'Linear', {'a': G}, 'EulerStochastic', n_steps,
                          [O.Monitor('Bold', 2000.0)], hist, st0, 0, nsig=[nsig], noise_z=z, **kw)
    bold = np.asarray(out[0][1])
    return g, variant, bold.reshape(bold.shape[0], -1), np.asarray(fin['state']).reshape(-1)


def philox_check(n_inst, n_steps, cores):
    """The timed path's parity: the sweep's own kernel, Philox noise and
    straight-line blocks, on `n_inst` instances spread over the grid for
    `n_steps` steps (at least 3 Bold samples, so FC is defined), against the
    CPU oracle fed the same Philox normals -- the stock and the all-float64
    variants.  Max relative error of Bold and final state per result, and
    max |dFC| (device FC kernel vs numpy.corrcoef of the oracle's Bold)."""
    import multiprocessing as mp
    G, S = sweep_grid()
    pick = np.linspace(0, G.size - 1, n_inst).round().astype(np.int64)
    sw = make_sweep(G.size, n_steps * DT, select=pick).configure()
    buf0 = sw._sim.history_buffer[..., 0].copy()
    st0 = sw._sim.current_state[..., 0].copy()
    res = sw.run(fc=True)
    kern = sw.batch.launch_struct(1)
    dev_state = np.stack([sw.batch.state(k)[0] for k in range(len(pick))])
    tasks = [(int(g), n_steps, float(G[g]), float(S[g]), buf0, st0, v) for g in pick for v in ('stock', 'fp64')]
    t0 = time.perf_counter()
    with mp.get_context('spawn').Pool(min(cores, len(tasks))) as pool:
        outs = pool.map(_philox_oracle_worker, tasks)
    wall = time.perf_counter() - t0
    ref = {(g, v): (bold, st) for g, v, bold, st in outs}
    err = {}
    for v in ('stock', 'fp64'):
        bm = sm = fm = 0.0
        per = []
        for k, g in enumerate(pick):
            rb, rs = ref[(int(g), v)]
            db = res['bold'][k][:, 0, :]
            e_b = float(np.abs(db - rb).max() / np.abs(rb).max())
            e_s = float(np.abs(dev_state[k] - rs).max() / np.abs(rs).max())
            e_f = float(np.abs(res['fc'][k] - np.corrcoef(rb.T)).max()) if rb.shape[0] >= 3 else None
            bm, sm = max(bm, e_b), max(sm, e_s)
            fm = max(fm, e_f) if e_f is not None else fm
            per.append({'instance': int(g), 'bold_max_rel': e_b, 'state_max_rel': e_s, 'fc_max_abs': e_f})
        err[v] = {'bold_max_rel': bm, 'state_max_rel': sm, 'fc_max_abs': fm, 'per_instance': per}
    return {'instances': [int(g) for g in pick], 'steps': n_steps, 'bold_samples': int(res['bold'][0].shape[0]),
            'noise': 'philox (the timed path: straight-line blocks, prefetch %d); the oracle fed the same '
                     'Philox normals' % kern.prefetch,
            'vs_all_fp64_oracle': err['fp64'], 'vs_stock_oracle': err['stock'], 'oracle_wall_s': wall,
            'nonfinite_instances': int((res['status'] != 0).sum())}


# ------------------------------------------------------------ plain form

def plain_form(n_steps, rank, gather):
    """The plain single-instance form: one instance of the same sweep (one
    CTA) through the same kernel and API, device-timed; region-steps/s."""
    import torch
    sw = make_sweep(1, n_steps * DT, rank=rank, gather=gather).configure()
    b = sw.build()
    b.snapshot()
    st = torch.cuda.current_stream()
    times = []
    for k in range(4):
        b.reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        sw.run_device()
        e1.record(st)
        torch.cuda.synchronize()
        if k:
            times.append(e0.elapsed_time(e1) / 1e3)
    t = float(np.median(times))
    return {'value': N_REGIONS * sw.n_steps / t, 'unit': UNIT, 'instances': 1, 'steps': sw.n_steps,
            'ms': 1e3 * t}


# ------------------------------------------------------------------ serving

# per connectome size: density, tract-length range (mm), conduction speed (mm/ms), generator seed
SERVE_SIZES = {68: (0.30, 10.0, 200.0, 5.0, 3), 76: (0.40, 10.0, 200.0, 3.0, 1), 192: (0.25, 5.0, 250.0, 4.0, 2),
               998: (0.10, 5.0, 300.0, 3.0, 4)}


def serving_plan(n_req, rate, seed=5):
    """Poisson arrivals at `rate` requests/s; each request draws a connectome
    size, a model, a duration uniform in 1-60 s and dt in {0.05, 0.1} ms."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_req))
    plan = []
    for k in range(n_req):
        plan.append((float(t[k]), str(rng.choice(['G2D', 'JR', 'RWW'])), int(rng.choice(list(SERVE_SIZES))),
                     float(rng.choice([0.05, 0.1])), float(rng.uniform(1000.0, 60000.0))))
    return plan


def serving_sim(model, n, dt, length, seed):
    from tvb_b200 import coupling, integrators, models, monitors, noise, synthetic
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.simulator import Simulator
    dens, lo, hi, speed, cseed = SERVE_SIZES[n]
    w, L = synthetic.connectome(n, dens, lo, hi, seed=cseed)
    conn = Connectivity(w, L, speed=speed)
    if model == 'G2D':
        np.random.seed(seed)
        return Simulator(model=models.Generic2dOscillator(), connectivity=conn, coupling=coupling.Linear(a=0.0152),
                         integrator=integrators.HeunDeterministic(dt=dt),
                         monitors=[monitors.TemporalAverage(period=1.0)], simulation_length=length).configure()
    if model == 'RWW':
        return Simulator(model=models.ReducedWongWang(), connectivity=conn, coupling=coupling.Linear(a=0.1),
                         integrator=integrators.EulerStochastic(dt=dt, noise=noise.Additive(nsig=[1e-3],
                                                                                            noise_seed=seed)),
                         monitors=[monitors.Bold(period=2000.0)], simulation_length=length).configure()
    nsig = np.array([0.0, 0.0, 0.0, 0.0, 1e-5, 0.0])
    return Simulator(model=models.JansenRit(), connectivity=conn, coupling=coupling.SigmoidalJansenRit(),
                     integrator=integrators.HeunStochastic(dt=dt, noise=noise.Additive(nsig=nsig, noise_seed=seed)),
                     monitors=[monitors.TemporalAverage(period=1.0), monitors.Bold(period=2000.0)],
                     simulation_length=length).configure()


def serving_leg(requests, rate, chunk, local, clocks=True):
    """Serve a Poisson stream of `requests` simulation requests at `rate` per
    second (continuous batching); sims/s with p50/p99 latency (arrival to
    result on the host), region-steps/s and device memory."""
    import torch
    from tvb_b200.serving import SimulationServer
    torch.cuda.set_device(local)
    plan = serving_plan(requests, rate)
    sims = [serving_sim(m, n, dt, length, seed=1000 + k) for k, (_, m, n, dt, length) in enumerate(plan)]
    srv = SimulationServer(chunk_steps=chunk or 4000, device=torch.device('cuda', local))
    arrivals = [(t, (lambda server, s=s: server.submit(s))) for (t, *_), s in zip(plan, sims)]
    sampler = ClockSampler(local) if clocks else None
    if sampler:
        sampler.start()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    srv.run(arrivals=arrivals, timeout=1800.0)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = sampler.stop() if sampler else None
    st = srv.stats()
    bad = [dict(zip(('model', 'regions', 'dt_ms', 'length_ms'), plan[k][1:]), seed=1000 + k, status=r.status)
           for k, r in sorted(srv.requests.items()) if r.status]
    leg = {'requests': requests, 'rate_per_s': rate, 'sims_per_s': st['sims_per_s'],
           'latency_p50_s': st['latency_p50_s'], 'latency_p99_s': st['latency_p99_s'],
           'latency_mean_s': st['latency_mean_s'], 'region_steps_per_s': st['region_steps_per_s'],
           'memory_budget_bytes': st['memory_budget_bytes'], 'memory_peak_bytes': st['memory_peak_bytes'],
           'memory_mean_bytes': st['memory_mean_bytes'], 'groups': st['groups'], 'gpu_launches': st['launches'],
           'nonfinite_requests': len(bad), 'nonfinite': bad[:16], 'wall_s': wall,
           'workload': 'Poisson arrivals; each request: connectome of %s regions, model G2D / JR / RWW, duration '
                       'U(1, 60) s, dt 0.05 or 0.1 ms, float32 state' % sorted(SERVE_SIZES),
           'chunk_steps': srv.chunk_steps}
    if clk:
        leg['clocks'] = clk
    return leg


def run_serving(args, rank, local):
    leg = serving_leg(args.requests, args.rate, args.chunk, local)
    line = {'metric': 'serving sims/s with p50/p99 latency (continuous batching)', 'value': leg['sims_per_s'],
            'unit': 'sims/s', 'n_gpus': 1, 'steps': args.requests, 'warmup': 0,
            'ms_per_step': 1e3 * leg['wall_s'] / args.requests, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': 'serving_poisson', 'requests': args.requests, 'rate_per_s': args.rate,
                       'sizes': sorted(SERVE_SIZES), 'models': ['G2D', 'JR', 'RWW'], 'duration_ms': [1000, 60000],
                       'dt_ms': [0.05, 0.1], 'chunk_steps': leg['chunk_steps'], 'state': 'f32'}}
    line.update({k: v for k, v in leg.items() if k not in ('workload', 'chunk_steps', 'requests', 'rate_per_s')})
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------- large network

EPI_N, EPI_DT = 998, 0.05


def large_network_sweep(length_scale=1.0, check_ms=None, gather='auto', cluster='auto', n_inst=16):
    """Epileptor, 998 regions (10 % density, tract lengths 5-300 mm, speed
    3 mm/ms), Difference coupling, HeunDeterministic dt 0.05 ms, 16 instances
    with x0 uniform in [-2.4, -1.6] per region and uneven lengths of 2-20 s
    (times length_scale) in one launch, TemporalAverage 1 ms.  check_ms: all
    16 instances for the first check_ms ms instead (the error check)."""
    from tvb_b200 import coupling, integrators, models, monitors, synthetic
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.sweep import ParameterSweep
    w, L = synthetic.connectome(EPI_N, 0.10, 5.0, 300.0, seed=4)
    x0 = np.random.default_rng(14).uniform(-2.4, -1.6, (16, EPI_N))[:n_inst]
    lengths = (np.linspace(2000.0, 20000.0, 16) * length_scale)[:n_inst]
    np.random.seed(15)
    sweep = {'model.x0': x0} if check_ms else {'model.x0': x0, 'simulation_length': lengths}
    sw = ParameterSweep(model=models.Epileptor(), connectivity=Connectivity(w, L, speed=3.0),
                        coupling=coupling.Difference(), integrator=integrators.HeunDeterministic(dt=EPI_DT),
                        monitors=[monitors.TemporalAverage(period=1.0)],
                        simulation_length=float(check_ms or lengths.max()), sweep=sweep, gather=gather,
                        cluster=cluster if cluster == 'auto' else int(cluster)).configure()
    return sw, x0, lengths


def _epileptor_oracle_worker(args):
    """One large-network instance on the CPU oracle (TemporalAverage 1 ms),
    stock (float32 history) or all-float64, from the configured history."""
    k, x0, n_steps, buf0, st0, variant = args
    os.environ['OMP_NUM_THREADS'] = '1'
    from oracle import tvb_oracle as O
    from tvb_b200 import synthetic
    w, L = synthetic.connectome(EPI_N, 0.10, 5.0, 300.0, seed=4)
    kw = dict(history_dtype=np.float64) if variant == 'fp64' else {}
    t0 = time.perf_counter()
    out, _ = O.simulate('Epileptor', {'x0': x0}, w, L, 3.0, EPI_DT, 'Difference', {'a': 0.1}, 'HeunDeterministic',
                        n_steps, [O.Monitor('TemporalAverage', 1.0)], buf0, st0, 0, **kw)
    return k, variant, np.asarray(out[0][1]), time.perf_counter() - t0


def large_network_error(check_ms, cores):
    """Per-instance error of the device's float32 run against the oracle
    (stock and all-float64) over the first check_ms ms: max relative error of
    the TemporalAverage within the first 20, 40, ... ms (the coupled
    Epileptor is chaotic, so the error grows with time)."""
    import multiprocessing as mp
    sw, x0, _ = large_network_sweep(check_ms=check_ms)
    buf0 = sw._sim.history_buffer[..., 0].copy()
    st0 = sw._sim.current_state[..., 0].copy()
    res = sw.run(fc=False)
    n_steps = sw.n_steps
    tasks = [(k, x0[k], n_steps, buf0, st0, v) for k in range(len(x0)) for v in ('stock', 'fp64')]
    procs = min(cores, len(tasks))
    t0 = time.perf_counter()
    with mp.get_context('spawn').Pool(procs) as pool:
        outs = pool.map(_epileptor_oracle_worker, tasks)
    wall = time.perf_counter() - t0
    ref = {(k, v): y for k, v, y, _ in outs}
    # the oracle's rate on these cores: each process runs its tasks one after another, every task the same
    # number of steps (the stock task's rate is the reference's numpy path; the float64 one costs about the same)
    t_task = float(np.mean([t for _, v, _, t in outs if v == 'stock']))
    cpu = {'value': procs * n_steps * EPI_N / t_task, 'unit': UNIT, 'cores': procs, 'kind': 'port',
           'sample': '%d processes, each an Epileptor 998 instance on the oracle (stock float32 history), %d steps '
                     '(%g ms); value = processes x steps x regions / mean simulate time of one instance (the '
                     'numpy path costs the same per step whatever the length)' % (procs, n_steps, check_ms)}
    windows = [m for m in range(20, int(check_ms) + 1, 20)]
    per = []
    for k in range(len(x0)):
        dev = res['tavg'][k].astype(np.float64)
        e = {'instance': k}
        for v in ('fp64', 'stock'):
            r = ref[(k, v)].reshape(dev.shape)
            scale = np.abs(r).max()
            e['vs_%s' % ('all_fp64' if v == 'fp64' else 'stock')] = {
                '%dms' % m: float(np.abs(dev[:m] - r[:m]).max() / scale) for m in windows}
        per.append(e)
    worst = {v: {'%dms' % m: max(p[v]['%dms' % m] for p in per) for m in windows}
             for v in ('vs_all_fp64', 'vs_stock')}
    return {'check_ms': check_ms, 'metric': 'max |device - oracle| / max |oracle| of TemporalAverage(1 ms) over '
            'the first t ms, from the same configured history', 'max_over_instances': worst, 'per_instance': per,
            'nonfinite_instances': int((res['status'] != 0).sum()), 'oracle_wall_s': wall, 'cpu_baseline': cpu}


def large_network_leg(steps, warmup, local, length_scale=1.0, gather='auto', cluster='auto', n_inst=16):
    """Region-steps/s of the 16-instance large-network batch on the device
    (n_inst < 16: its first n_inst instances)."""
    import torch
    torch.cuda.set_device(local)
    sw, x0, lengths = large_network_sweep(length_scale, gather=gather, cluster=cluster, n_inst=n_inst)
    b = sw.build()
    b.snapshot()
    st = torch.cuda.current_stream()
    ms = []
    for k in range(warmup + steps):
        b.reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        sw.run_device()
        e1.record(st)
        torch.cuda.synchronize()
        if k >= warmup:
            ms.append(e0.elapsed_time(e1))
    steps_total = int(sw.n_steps_each.sum())
    t = float(np.mean(ms)) / 1e3
    return {'value': float(steps_total * EPI_N / t), 'unit': UNIT, 'ms_per_step': 1e3 * t, 'steps': steps,
            'warmup': warmup, 'instances': n_inst, 'regions': EPI_N, 'edge_runs': b.edges_per_thread, 'nnz': int(sw._sim._conn.nnz), 'dt_ms': EPI_DT,
            'lengths_ms': lengths.tolist(), 'cluster_ctas_per_instance': b.cluster, 'sync_every': b.sync_every,
            'launch': ('cooperative, %d groups of %d CTAs' % (b.groups, b.cluster) if b.groups
                       else 'thread-block clusters of %d CTAs' % b.cluster),
            'nonfinite_instances': int((b.status() != 0).sum()), 'gpu_launches': steps * b.last_launches}


def run_large_network(args, rank, local):
    leg = large_network_leg(args.steps, args.warmup, local, args.length / 60000.0, args.gather, args.cluster,
                            args.ln_instances)
    line = {'metric': 'region-steps/sec, large-network batch', 'value': leg['value'], 'unit': UNIT,
            'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': leg['ms_per_step'],
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': 'epileptor_998r_16i_uneven_2-20s', 'instances': leg['instances'], 'regions': EPI_N,
                       'nnz': leg['nnz'], 'dt_ms': EPI_DT, 'lengths_ms': leg['lengths_ms'],
                       'cluster_ctas_per_instance': leg['cluster_ctas_per_instance'],
                       'sync_every': leg['sync_every'], 'launch': leg['launch']},
            'nonfinite_instances': leg['nonfinite_instances'], 'gpu_launches': leg['gpu_launches']}
    if args.check_ms > 0:
        err = large_network_error(args.check_ms, os.cpu_count() or 1)
        line['cpu_baseline'] = err.pop('cpu_baseline')
        line['error_vs_fp64_oracle'] = err
    print(json.dumps(line), flush=True)


# DRAM bytes per instance-step of the simulation kernel on this workload, from the ncu capture
# of 296 instances x 40 000 steps (dram__bytes_read.sum + dram__bytes_write.sum = 1.786 GB);
# a launch's traffic scales with its instance-steps.
NCU_DRAM_BYTES_PER_INSTANCE_STEP = 1.786e9 / (296 * 40000)


# --------------------------------------------------------------------- main

def run_reference(args, rank):
    """The reference arm: the oracle port of the reference's numpy path on all
    host cores.  Each of the W + K steps is one sample (cpu_sample, a
    different stratified subset of the grid each step); ms_per_step is the
    measured wall time of a timed sample."""
    if rank != 0:
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    walls = []
    with mp.get_context('spawn').Pool(cores) as pool:
        pool.map(_warm, range(cores))
        for k in range(args.warmup + args.steps):
            wall, _ = cpu_sample(pool, cores, args.ref_sample_steps, offset=7 * k)
            if k >= args.warmup:
                walls.append(wall)
    t = float(np.mean(walls))
    value = cores * args.ref_sample_steps * N_REGIONS / t
    full = 1024 * 600000 * N_REGIONS / value
    cb = {'value': value, 'unit': UNIT, 'cores': cores, 'kind': 'port',
          'sample': _sample_text(cores, args.ref_sample_steps)}
    line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': args.gpus, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * t, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic', 'impl': 'reference',
            'config': {'workload': 'rww_sweep_68r_1024i_60s_bold_fc', 'step': 'one sample: ' + cb['sample'],
                       'extrapolation': 'the numpy path costs the same per step whatever the state, so the '
                                        'sample rate is the rate of the full 1024 x 600 000-step sweep, which '
                                        'would take %.0f s on these cores' % full},
            'cpu_baseline': cb, 'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0,
                                        'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--instances', type=int, default=1024)
    ap.add_argument('--length', type=float, default=60000.0, help='simulated ms per instance')
    ap.add_argument('--chunk', type=int, default=None, help='steps per kernel launch')
    ap.add_argument('--cpu-steps', type=int, default=600000,
                    help='steps per instance of the cpu_baseline sample (default: the full 60 s)')
    ap.add_argument('--ref-sample-steps', type=int, default=20000,
                    help='steps per instance of each --impl reference sample (one sample per step)')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--e2e-steps', type=int, default=2)
    ap.add_argument('--gather', default='auto', choices=['auto', 'row', 'edge', 'split', 'tune'],
                    help='coupling gather variant of the simulation kernel')
    ap.add_argument('--lanes', default='1', choices=['auto', '1', '2', '4', '8'],
                    help='instance groups (interleaved rings, one thread per region and instance) or one '
                         'instance per CTA')
    ap.add_argument('--plain-steps', type=int, default=60000,
                    help='steps of the plain single-instance measurement (0 skips it)')
    ap.add_argument('--workload', default='sweep', choices=['sweep', 'serving', 'large-network'])
    ap.add_argument('--cluster', default='auto', help='CTAs per instance (large-network workload)')
    ap.add_argument('--requests', type=int, default=48, help='serving: number of requests')
    ap.add_argument('--rate', type=float, default=4.0, help='serving: Poisson arrival rate (requests/s)')
    ap.add_argument('--check-steps', type=int, default=80000,
                    help='steps of the Philox-path parity check against the oracle (0 skips it)')
    ap.add_argument('--check-ms', type=float, default=60.0,
                    help='large network: ms of the per-instance error check against the oracle (0 skips it)')
    ap.add_argument('--ln-instances', type=int, default=16, choices=range(1, 17), metavar='1..16',
                    help='large network: run the first k of the 16 instances')
    ap.add_argument('--no-legs', action='store_true',
                    help='sweep only: no serving and large-network legs in the line')
    args = ap.parse_args()

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        return run_reference(args, rank)
    if args.workload == 'serving':
        if rank == 0:
            run_serving(args, rank, local)
        return
    if args.workload == 'large-network':
        if rank == 0:
            run_large_network(args, rank, local)
        return

    # CPU baseline first: its spawn pool starts before any GPU work
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(n_steps=args.cpu_steps)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=300), device_id=torch.device('cuda', local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    lanes = args.lanes if args.lanes == 'auto' else int(args.lanes)
    sw = make_sweep(args.instances, args.length, rank=rank, world=world, chunk=args.chunk, gather=args.gather,
                    lanes=lanes).configure()
    batch = sw.build()
    batch.snapshot()
    n_steps = sw.n_steps
    launches_per_step = None   # the simulation launches of one step (Batch.run counts them) + the FC kernel
    nnz = sw._sim._conn.nnz
    st = torch.cuda.current_stream()

    def one_step():
        batch.reset()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(st)
        sw.run_device()
        e1.record(st)
        fc = sw.fc_device()
        e2.record(st)
        return e0, e1, e2, fc

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    launches_per_step = batch.last_launches + 1

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    wall0 = time.perf_counter()
    evs = [one_step() for _ in range(args.steps)]
    barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    step_ms = [e0.elapsed_time(e2) for e0, e1, e2, _ in evs]
    kern_ms = [e0.elapsed_time(e1) for e0, e1, e2, _ in evs]
    t_dev = float(np.sum(step_ms)) / 1e3
    t_kern = float(np.mean(kern_ms)) / 1e3
    status = batch.status()

    # end to end through the public API: host inputs -> host Bold + FC
    e2e_times, h2d, d2h = [], 0, 0
    for _ in range(max(args.e2e_steps, 0)):
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(st)
        sw2 = make_sweep(args.instances, args.length, rank=rank, world=world, chunk=args.chunk,
                         gather=args.gather, lanes=lanes).configure()
        res = sw2.run(fc=True)
        s1.record(st)
        torch.cuda.synchronize()
        e2e_times.append(s0.elapsed_time(s1) / 1e3)
        h2d, d2h = sw2.batch.h2d_bytes, sw2.batch.d2h_bytes + res['fc'].nbytes
        del sw2, res

    if not e2e_times:
        e2e_times = [float('inf')]
    plain = plain_form(args.plain_steps, rank, args.gather) if args.plain_steps > 0 else None
    errs = serving = large = None
    if rank == 0 and world == 1:
        cores = os.cpu_count() or 1
        if args.check_steps > 0:
            errs = philox_check(16, args.check_steps, cores)
        if not args.no_legs:
            serving = serving_leg(args.requests, args.rate, None, local, clocks=False)
            large = large_network_leg(1, 1, local)
            if args.check_ms > 0:
                err = large_network_error(args.check_ms, cores)
                large['cpu_baseline'] = err.pop('cpu_baseline')
                large['error_vs_fp64_oracle'] = err

    if world > 1:
        tt = torch.tensor([t_dev, t_kern, float(np.median(e2e_times))], device='cuda', dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_dev, t_kern, t_e2e = tt.tolist()
    else:
        t_e2e = float(np.median(e2e_times))

    region_steps = float(args.instances) * n_steps * N_REGIONS * world
    value = region_steps * args.steps / t_dev
    gather_bytes = float(args.instances) * n_steps * 4.0 * nnz
    peaks = {}
    try:
        with open(os.path.join(HERE, 'MEASURED_PEAKS.json')) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = float(peaks.get('hbm_gbs', 6650.0))
    peak_src = ('measured HBM copy bandwidth (of measured)' if 'hbm_gbs' in peaks
                else 'the pool\'s earlier HBM measurement, 6650 GB/s (of fallback: no measured peaks file)')
    achieved = gather_bytes / t_kern / 1e9
    # the rings live in shared memory: the same bytes against its nominal bandwidth (128 B per clock per SM)
    sm_mhz = (clocks or {}).get('sm_mhz') or float(peaks.get('sm_max_mhz', 1965.0))
    smem_peak = 148 * 128 * sm_mhz * 1e6 / 1e9
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * t_dev / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': 'rww_sweep_68r_1024i_60s_bold_fc', 'instances_per_gpu': args.instances,
                       'instances_total': args.instances * world,
                       'regions': N_REGIONS, 'nnz': nnz, 'dt_ms': DT, 'sim_ms': args.length, 'steps': n_steps,
                       'bold_tr_ms': 2000.0, 'fc': True, 'noise': 'philox',
                       'parallelism': 'instances sharded over ranks' if world > 1 else 'single gpu',
                       'l2': 'flushed between steps by the per-step state reset (%.1f GB written)'
                             % ((batch.init.size + batch.zero.size + batch.out.size) / 1e9),
                       'ring_in_smem': batch.ring_in_smem, 'sync_every': batch.sync_every,
                       'gather': 'edge-parallel %d/thread, %d threads' % (batch.edges_per_thread, batch.block_threads)
                                 if batch.edges_per_thread else 'row per thread',
                       'lanes': batch.lanes, 'prefetch': batch.prefetch},
            'e2e': {'value': region_steps / t_e2e, 'unit': UNIT, 'h2d_bytes_per_step': int(h2d),
                    'd2h_bytes_per_step': int(d2h)},
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak,
                         'traffic': NCU_DRAM_BYTES_PER_INSTANCE_STEP * args.instances * n_steps,
                         'note': 'algorithmic gather bytes 4*ncvar*nnz per instance-step over the simulation '
                                 'kernel time; peak = %s; traffic = ncu '
                                 'DRAM bytes per launch, scaled from a 296-instance x 40 000-step capture; the '
                                 'rings are staged in shared memory, so DRAM carries only staging and Bold'
                                 % peak_src,
                         'smem': {'achieved': achieved, 'peak': smem_peak, 'unit': 'GB/s', 'frac': achieved / smem_peak,
                                  'note': 'the same algorithmic bytes against the shared-memory bandwidth the '
                                          'gather reads: 148 SMs x 128 B per clock at the sampled SM clock '
                                          '(nominal, not measured)'}},
            'gpu_launches': launches_per_step * args.steps,
            'kernel_ms_per_step': 1e3 * t_kern,
            'nonfinite_instances': int((status != 0).sum()),
            'wall_s_timed': wall,
        }
        if clocks:
            line['clocks'] = clocks
        if plain:
            plain['batched_over_plain'] = value / plain['value']
            line['plain_single_instance'] = plain
        if errs:
            line['error_vs_fp64_oracle'] = errs
        if serving:
            line['serving'] = serving
        if large:
            line['large_network'] = large
        if cb:
            line['cpu_baseline'] = cb
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
