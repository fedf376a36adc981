"""Batched parameter sweeps: many instances of one simulation configuration in
one kernel launch, differing in coupling strength, noise and model
parameters.

Each instance is what the reference would run as a separate
``Simulator(...).configure().run()`` (one process per grid point in the
framework's parameter-space exploration); here they all advance together,
one CTA each, sharing the connectome on the device.  Initial histories are
drawn exactly as the reference draws them for each instance.  The Bold
output of every instance can be reduced to its functional connectivity
(Pearson over time, float64) on the device.
"""
import numpy as np
import torch

from . import _lib
from .engine import Batch, Connectome, InstanceSpec, functional_connectivity
from .simulator import (Simulator, adopt_connectivity, adopt_coupling, adopt_integrator, adopt_model,
                        adopt_monitor, noise_sigma)
from . import monitors as monitors_mod


class ParameterSweep:
    """Sweep of `n_instances` simulations.

    sweep: dict mapping 'coupling.<name>', 'noise.nsig', 'model.<name>' or
    'simulation_length' to arrays of one value per instance (for
    'model.<name>' also an (instances, regions) array: one value per region,
    like the reference's spatialised parameters; 'stimulus.weight' takes an
    (instances, regions) array of stimulus weights, with `stimulus` given);
    'simulation_length' gives
    instances of uneven lengths, which run in the same launch and retire at
    their own last step.  Noise: 'philox' draws an independent
    device stream per instance (key = (noise_seed, instance index));
    'reference' feeds every instance the reference's RandomState stream (the
    same for all, as separate reference runs with the default seed would
    draw), which is for parity checks on short runs.

    Sharding: the swept values define the global instance list, instance g
    being what the framework's parameter-space exploration runs as operation
    g.  `shard=(rank, world)` runs the rank-th of `world` contiguous, balanced
    parts of that list (one process per GPU, no collective while it runs);
    `instances=` runs an explicit list of global indices instead.  An
    instance's Philox stream is keyed by its global index, so it draws the
    same noise whichever process runs it, and results come back in the order
    of `self.instances` ('instances' in run()'s result); gather_sweep()
    reassembles the shards on one rank in global order.

    region_rings: clusters of CTAs per instance keep each region's history
    contiguous (region-major rings) when the delays allow four-step gathers;
    False keeps the time-major ring and the one-step edge-run kernel.
    groups: with region-major rings, 'auto' (and cluster='auto') runs the
    batch as one cooperative launch of groups of CTAs that take instances
    from a device queue, choosing the CTAs per instance; True also with an
    explicit cluster; False keeps thread-block clusters.  block_steps: steps
    per gather block on region-major rings, 4, 8 or 'auto' (8 when the
    smallest delay allows and the batch has no stimulus, AfferentCoupling or
    projection stream).
    """

    def __init__(self, model, connectivity, coupling, integrator, monitors, simulation_length, sweep,
                 noise_source='philox', chunk_steps=None, device=None, sync_every=None, ring_in_smem=None,
                 gather='auto', lanes=1, cluster='auto', stimulus=None, shard=None, instances=None,
                 region_rings=True, groups='auto', block_steps='auto'):
        self.model = adopt_model(model)
        self.stimulus = stimulus
        self.connectivity = adopt_connectivity(connectivity)
        self.coupling = adopt_coupling(coupling)
        self.integrator = adopt_integrator(integrator)
        self.monitors = [adopt_monitor(m) for m in (monitors if isinstance(monitors, (list, tuple)) else [monitors])]
        self.simulation_length = float(simulation_length)
        self.sweep = {k: np.atleast_1d(np.asarray(v, dtype=np.float64)) for k, v in sweep.items()}
        sizes = {len(v) for v in self.sweep.values()}
        if len(sizes) != 1:
            raise ValueError('all swept parameters need the same number of values')
        self.n_global = sizes.pop()
        self.instances = shard_instances(self.n_global, shard, instances)
        self.n_instances = len(self.instances)
        if self.n_instances == 0:
            raise ValueError('this shard holds no instances')
        self.noise_source = noise_source
        self.chunk_steps = chunk_steps
        self.device = device
        self.sync_every = sync_every
        self.ring_in_smem = ring_in_smem
        self.gather = gather
        self.lanes = lanes
        self.cluster = cluster
        self.region_rings = region_rings
        self.groups = groups
        self.block_steps = block_steps
        self.batch = None

    def configure(self):
        # one reference-equivalent simulator resolves delays, history and monitors
        self._sim = Simulator(model=self.model, connectivity=self.connectivity, coupling=self.coupling,
                              integrator=self.integrator, monitors=self.monitors,
                              simulation_length=self.simulation_length, noise_source=self.noise_source,
                              device=self.device, stimulus=self.stimulus).configure()
        sim = self._sim
        if 'stimulus.weight' in self.sweep and self.stimulus is None:
            raise ValueError("sweeping 'stimulus.weight' needs a stimulus")
        self.n_steps = int(np.ceil(self.simulation_length / self.integrator.dt))
        n = sim.number_of_nodes
        conn = sim._conn
        raw, tavg_istep, bspec = sim._monitor_spec()
        base_params = sim._params
        pidx = {name: k for k, name in enumerate(self.model.kernel_param_names)}
        cnames = list(type(self.coupling)._defaults)
        fed = None
        if self.integrator.stochastic and self.noise_source == 'reference':
            z = self.integrator.noise.random_stream.normal(size=(self.n_steps, sim.nint, n)).astype(np.float32)
            fed = torch.from_numpy(z)
        self._fed = fed
        specs = []
        lengths = self.sweep.get('simulation_length')
        if lengths is not None:
            self.n_steps_each = np.ceil(lengths[self.instances] / self.integrator.dt).astype(np.int64)
            self.n_steps = int(self.n_steps_each.max())
        else:
            self.n_steps_each = np.full(self.n_instances, self.n_steps, dtype=np.int64)
        stim = None
        if self.stimulus is not None:
            # one time grid covers every instance: r_[0 : L : dt] agrees on the common steps for any L
            sim.simulation_length = max(self.simulation_length, float(self.n_steps) * self.integrator.dt)
            sim._prepare_stimulus()
            stim = sim.stimulus_spec(self.n_steps)
            sim.simulation_length = self.simulation_length
        for i, g in enumerate(self.instances):
            params = base_params
            cf = self.coupling.kernel_params()
            sigma = sim._sigma
            stim_i = stim
            for key, vals in self.sweep.items():
                part, _, name = key.partition('.')
                if part == 'model':
                    if params is base_params:
                        params = base_params.copy()
                    params[pidx[name]] = np.asarray(vals[g], dtype=np.float32)
                elif part == 'coupling':
                    cf = list(cf)
                    cf[cnames.index(name)] = float(vals[g])
                elif part == 'noise' and name == 'nsig':
                    sigma = noise_sigma(np.array([vals[g]]), sim.nint, n, self.integrator.dt)
                elif key == 'simulation_length':
                    pass
                elif key == 'stimulus.weight':
                    stim_i = dict(stim, weight=np.asarray(vals[g], dtype=np.float64).reshape(-1))
                else:
                    raise ValueError('cannot sweep %s' % key)
            spec = InstanceSpec(conn, sim.history_buffer[..., 0], sim.current_state[..., 0], params, cf,
                                int(self.n_steps_each[i]), step0=sim.current_step, sigma=sigma, noise_fed=None,
                                seed=self.integrator.noise.noise_seed if self.integrator.stochastic else 0,
                                stream=int(g), raw=raw, tavg_istep=tavg_istep, bold=bspec, sub_istep=sim._sub_istep,
                                stim=stim_i, aff_istep=sim._aff_istep, proj_istep=sim._proj_istep)
            specs.append(spec)
        self._specs = specs
        noise_kind = _lib.NOISE_NONE
        if self.integrator.stochastic:
            noise_kind = _lib.NOISE_FED if fed is not None else _lib.NOISE_PHILOX
        self._noise_kind = noise_kind
        return self

    def _make_batch(self, gather, lanes, ring_in_smem, cluster):
        sim = self._sim
        return Batch(sim._model_id, sim._cfun_id, sim._scheme_id, self._noise_kind, self.integrator.dt,
                     sim._voi_codes, self._specs, device=self.device, sync_every=self.sync_every,
                     ring_in_smem=ring_in_smem, gather=gather, lanes=lanes, cluster=cluster,
                     region_rings=self.region_rings, groups=self.groups, block_steps=self.block_steps)

    def projection(self, mons):
        """Sensor signals of projection monitors `mons` for all instances: one
        float64 GEMM per monitor on the device over every instance's period
        means, then each instance's observation noise from the monitor's
        RandomState at its current state (what separate runs would each draw)."""
        from .simulator import project_samples
        dev = torch.stack([self.batch.outputs_device(i)['proj'] for i in range(self.n_instances)])
        I, T = dev.shape[:2]
        out = []
        for m in mons:
            y = project_samples(dev.reshape((I * T,) + dev.shape[2:]), m).cpu().numpy().reshape(I, T, len(m.voi), -1)
            rs = getattr(m.obsnoise, 'random_stream', None)
            st0 = rs.get_state() if rs is not None else None
            for i in range(I):
                if rs is not None:
                    rs.set_state(st0)
                y[i] = m.finish(y[i])
            out.append(y)
        return out

    def build(self):
        """Allocate the device batch and upload inputs (one host-to-device copy).
        With gather='tune' the kernel variant is picked by the autotuner
        (trial runs of this batch, cached per GPU and batch shape)."""
        sim = self._sim
        kw = dict(gather=self.gather, lanes=self.lanes, ring_in_smem=self.ring_in_smem, cluster=self.cluster)
        if self.gather == 'tune' and self._fed is not None:
            kw['gather'] = 'auto'  # trial runs draw no fed noise: fed-noise parity runs keep the default variant
        elif self.gather == 'tune':
            from . import autotune
            dev = torch.device(self.device if self.device is not None else 'cuda')
            key = autotune.shape_key(sim._model_id, sim._cfun_id, sim._scheme_id, self._noise_kind,
                                     self.integrator.dt, sim._voi_codes, self._specs, dev)
            kw, self.tune_ms = autotune.tune(self._make_batch, key, sim.ncvar, sim.number_of_nodes,
                                             self.n_instances, shared_conn=True)
        self.batch = self._make_batch(**kw)
        if self._fed is not None:
            fed = self._fed.to(self.batch.device).contiguous()
            self.batch._fed.append(fed)
            ins = self.batch.insts_host
            ins['noise_fed'] = fed.data_ptr()
            off, _ = self.batch.init.regions[('insts',)]
            self.batch.init_buf[off:off + ins.nbytes].copy_(torch.from_numpy(ins.view(np.uint8)))
        return self.batch

    def run_device(self, graph=None):
        """Advance every instance to the end on the device (inputs already
        resident).  With chunk_steps set, the chunk launches are replayed from
        a CUDA graph (graph=None or True) or launched one by one (False)."""
        if graph is None:
            graph = self.chunk_steps is not None
        self.batch.run(chunk=self.chunk_steps, graph=graph)

    def bold_device(self, voi=0):
        """(I, T, n) float64 device tensor of the Bold series of one observed variable."""
        return self.batch.stacked_output('bold', torch.float64)[:, :, voi, :]

    def fc_device(self, voi=0):
        """Per-instance functional connectivity (I, n, n) float64 on the device."""
        bold = self.bold_device(voi)
        return functional_connectivity(bold)

    def run(self, fc=True):
        """Build, run and return host results: dict with per-monitor arrays
        (I, T, nvoi, n) under 'raw' / 'tavg' / 'bold' / 'sub' (lists of
        (T_i, nvoi, n) arrays for uneven lengths), 'aff' (I, T, ncvar, n) for
        the AfferentCoupling monitors, 'proj' (I, T, nvoi, n) the period means
        of the EEG / MEG / iEEG monitors and 'projection' (one (I, T, nvoi_m, S)
        array per such monitor, in monitor order: the sensor signals, each
        instance with the observation noise a separate run would draw) and
        'fc' (I, n, n)."""
        if self.batch is None:
            self.build()
        self.run_device()
        res = {}
        if fc and any(isinstance(m, monitors_mod.Bold) for m in self.monitors):
            dev = self.fc_device()
            host = torch.empty(dev.shape, dtype=dev.dtype, pin_memory=True)   # pinned: a full-speed copy
            host.copy_(dev, non_blocking=True)
            torch.cuda.current_stream(dev.device).synchronize()
            res['fc'] = host.numpy()
        outs = self.batch.outputs_host()
        proj_mons = [m for m in self.monitors if isinstance(m, monitors_mod.Projection)]
        if proj_mons and len({s.n_steps for s in self._specs}) == 1:
            res['projection'] = self.projection(proj_mons)
        for key in ('raw', 'tavg', 'bold', 'sub', 'aff', 'proj'):
            if key in outs[0]:
                arrs = [o[key] for o in outs]
                # instances of uneven lengths give a list of (T_i, nvoi, n) arrays
                res[key] = np.stack(arrs) if len({a.shape for a in arrs}) == 1 else arrs
        res['status'] = self.batch.status()
        if (res['status'] & _lib.TVBK_STATUS_TIMEOUT).any():
            raise RuntimeError('a barrier of the cooperative launch gave up waiting: the run stopped early')
        res['instances'] = self.instances.copy()
        return res


def shard_instances(n_global, shard=None, instances=None):
    """Global indices of the instances one process runs: all of them, the
    rank-th of `world` contiguous balanced parts (shard=(rank, world)), or an
    explicit list (instances=, each index once, in range)."""
    if instances is not None:
        idx = np.asarray(instances, dtype=np.int64).reshape(-1)
        if idx.size and (idx.min() < 0 or idx.max() >= n_global):
            raise IndexError('instance index out of range 0..%d' % (n_global - 1))
        if np.unique(idx).size != idx.size:
            raise ValueError('instance indices repeat')
        return idx
    if shard is None:
        return np.arange(n_global, dtype=np.int64)
    rank, world = (int(v) for v in shard)
    if not 0 <= rank < world:
        raise ValueError('shard (%d, %d): need 0 <= rank < world' % (rank, world))
    return np.array_split(np.arange(n_global, dtype=np.int64), world)[rank]


_PER_INSTANCE = ('raw', 'tavg', 'bold', 'sub', 'aff', 'proj', 'fc', 'status')


def gather_sweep(res, group=None, dst=0):
    """Collect the run() results of every rank's shard on rank `dst` and
    reassemble them in global instance order (one gather of host objects at
    the end of the run, over the process group's backend: NCCL between GPUs,
    or gloo).  Returns the merged dict on `dst`, None elsewhere."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    objs = [None] * world if rank == dst else None
    dist.gather_object(res, objs, dst=dst, group=group)
    if rank != dst:
        return None
    order = np.concatenate([o['instances'] for o in objs])
    perm = np.argsort(order, kind='stable')
    out = {'instances': order[perm]}
    for key in _PER_INSTANCE:
        if key not in objs[0]:
            continue
        parts = [o[key] for o in objs]
        if all(isinstance(p, np.ndarray) for p in parts) and len({p.shape[1:] for p in parts}) == 1:
            out[key] = np.concatenate(parts)[perm]
        else:   # uneven lengths: per-instance arrays
            flat = [a for p in parts for a in p]
            out[key] = [flat[k] for k in perm]
    if 'projection' in objs[0]:
        out['projection'] = [np.concatenate([o['projection'][m] for o in objs])[perm]
                             for m in range(len(objs[0]['projection']))]
    return out
