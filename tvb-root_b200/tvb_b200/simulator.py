"""Drop-in Simulator for the region simulation loop
(tvb/simulator/simulator.py:55-639), running on the B200 kernels.

    sim = Simulator(model=..., connectivity=..., coupling=..., integrator=...,
                    monitors=[...], simulation_length=...).configure()
    (t_raw, raw), (t_tavg, tavg) = sim.run()

Constructor keywords, ``configure()``, the ``__call__`` generator and
``run()`` follow the reference: the same initial-history draw (from the
noise RandomState for stochastic schemes, numpy's global RNG otherwise), the
same integer delays and horizon, the same monitor step constants and output
times, and outputs shaped (T, nvoi, n, 1).  Components may be this package's
classes or the reference's own objects (read by attribute name).

Differences, by design: state, coupling and integration are float32 with
float32 accumulation (Bold accumulation and its HRF dot are float64); noise
comes from the device's Philox stream unless ``noise_source='reference'``,
which feeds the reference's own RandomState stream; unsupported components
raise NotImplementedError -- there is no CPU fallback.
"""
import math

import numpy as np

from . import _lib
from . import coupling as coupling_mod
from . import integrators as integrators_mod
from . import models as models_mod
from . import monitors as monitors_mod
from .connectivity import Connectivity
from .engine import Batch, Connectome, InstanceSpec, ring_to_reference
from .noise import Additive


def _first(v):
    return float(np.asarray(v, dtype=np.float64).reshape(-1)[0])


def adopt_model(model):
    name = type(model).__name__
    if isinstance(model, models_mod.Model):
        return model
    if name not in models_mod.MODELS:
        raise NotImplementedError('model %s has no device implementation' % name)
    cls = models_mod.MODELS[name]
    kw = {p: np.asarray(getattr(model, p)) for p in cls._defaults if hasattr(model, p)}
    m = cls(**kw)
    m.variables_of_interest = tuple(getattr(model, 'variables_of_interest', cls.variables_of_interest))
    if getattr(model, 'stvar', None) is not None:
        m.stvar = np.asarray(model.stvar, dtype=np.int32).copy()
    return m


def adopt_coupling(cf):
    name = type(cf).__name__
    if isinstance(cf, coupling_mod.Coupling):
        return cf
    if name not in coupling_mod.COUPLINGS:
        raise NotImplementedError('coupling %s has no device implementation' % name)
    cls = coupling_mod.COUPLINGS[name]
    return cls(**{p: np.asarray(getattr(cf, p)) for p in cls._defaults if hasattr(cf, p)})


def adopt_integrator(integ):
    name = type(integ).__name__
    if isinstance(integ, integrators_mod.Integrator):
        return integ
    if name not in integrators_mod.INTEGRATORS:
        raise NotImplementedError('integrator %s has no device implementation' % name)
    cls = integrators_mod.INTEGRATORS[name]
    if cls.stochastic:
        nz = integ.noise
        if type(nz).__name__ != 'Additive' or float(getattr(nz, 'ntau', 0.0)) != 0.0:
            raise NotImplementedError('only additive white noise is supported on the device')
        noise = Additive(nsig=nz.nsig, noise_seed=nz.noise_seed, random_stream=nz.random_stream)
        return cls(dt=integ.dt, noise=noise)
    return cls(dt=integ.dt)


def adopt_monitor(mon):
    if isinstance(mon, monitors_mod.Monitor):
        return mon
    name = type(mon).__name__
    voi = getattr(mon, 'variables_of_interest', None)
    if voi is not None and np.asarray(voi).size == 0:
        voi = None
    if name == 'Raw':
        return monitors_mod.Raw()
    if name == 'RawVoi':
        return monitors_mod.RawVoi(variables_of_interest=voi)
    if name == 'ProgressLogger':
        return monitors_mod.ProgressLogger(period=mon.period)
    if name == 'TemporalAverage':
        return monitors_mod.TemporalAverage(period=mon.period, variables_of_interest=voi)
    if name in ('SubSample', 'GlobalAverage', 'AfferentCouplingTemporalAverage'):
        return monitors_mod.MONITORS[name](period=mon.period, variables_of_interest=voi)
    if name == 'AfferentCoupling':
        return monitors_mod.AfferentCoupling(variables_of_interest=voi)
    if name in ('EEG', 'MEG', 'iEEG'):
        kw = dict(period=mon.period, variables_of_interest=voi, sensors=mon.sensors, projection=mon.projection,
                  region_mapping=mon.region_mapping, obsnoise=mon.obsnoise)
        if name == 'EEG':
            kw.update(reference=mon.reference, sigma=mon.sigma)
        elif name == 'iEEG':
            kw.update(sigma=mon.sigma)
        return monitors_mod.MONITORS[name](**kw)
    if name == 'SpatialAverage':
        return monitors_mod.SpatialAverage(period=mon.period, variables_of_interest=voi,
                                           spatial_mask=getattr(mon, 'spatial_mask', None))
    if name == 'Bold':
        if type(mon.hrf_kernel).__name__ != 'FirstOrderVolterra':
            raise NotImplementedError('Bold on the device supports the FirstOrderVolterra kernel')
        from .equations import FirstOrderVolterra
        return monitors_mod.Bold(period=mon.period, variables_of_interest=voi,
                                 hrf_kernel=FirstOrderVolterra(dict(mon.hrf_kernel.parameters)),
                                 hrf_length=mon.hrf_length)
    raise NotImplementedError('monitor %s has no device implementation' % name)


def adopt_connectivity(conn):
    if isinstance(conn, Connectivity):
        return conn
    cort = getattr(conn, 'cortical', None)
    return Connectivity(weights=conn.weights, tract_lengths=conn.tract_lengths,
                        speed=getattr(conn, 'speed', None), centres=getattr(conn, 'centres', None),
                        orientations=getattr(conn, 'orientations', None),
                        cortical=None if cort is None or np.asarray(cort).size == 0 else cort)


def project_samples(proj, m):
    """(T, nvoi_m, S) = gain . mean for the device stream proj (T, nvoi, n)
    float32 of window means and projection monitor m: the library's float64
    projection kernel (tvbk_project) over all samples at once."""
    import ctypes
    import torch
    proj = proj.contiguous()
    T, nvoi, n = proj.shape
    g = torch.as_tensor(np.ascontiguousarray(m.gain, dtype=np.float64), device=proj.device)   # (S, n)
    voi = torch.as_tensor(np.asarray(m.voi, dtype=np.int32).reshape(-1), device=proj.device)
    S = g.shape[0]
    y = torch.empty((T, voi.numel(), S), dtype=torch.float64, device=proj.device)
    st = torch.cuda.current_stream(proj.device)
    _lib.check(_lib.load().tvbk_project(ctypes.c_void_p(proj.data_ptr()), T, nvoi, n, ctypes.c_void_p(voi.data_ptr()),
                                        voi.numel(), ctypes.c_void_p(g.data_ptr()), S, ctypes.c_void_p(y.data_ptr()),
                                        ctypes.c_void_p(st.cuda_stream)), 'tvbk_project')
    return y


def noise_sigma(nsig, nintvar, n, dt):
    """sqrt(dt) * sqrt(2 nsig) per (integrated variable, region), with the nsig
    shapes the reference accepts (tvb/simulator/simulator.py:372-424)."""
    nsig = np.asarray(nsig, dtype=np.float64)
    if nsig.shape in ((1,), ()):
        full = np.full((nintvar, n), float(nsig.reshape(-1)[0]))
    elif nsig.shape in ((nintvar, n, 1), (nintvar, n)):
        full = nsig.reshape(nintvar, n)
    elif nsig.shape in ((nintvar,), (nintvar, 1, 1), (nintvar, 1)):
        full = np.repeat(nsig.reshape(nintvar, 1), n, axis=1)
    elif nsig.shape in ((n,), (1, n, 1), (1, n)):
        full = np.repeat(nsig.reshape(1, n), nintvar, axis=0)
    else:
        raise ValueError('Bad Simulator.integrator.noise.nsig shape: %s' % (nsig.shape,))
    return (np.sqrt(dt) * np.sqrt(2.0 * full)).astype(np.float32)


class Simulator:
    def __init__(self, connectivity=None, coupling=None, model=None, integrator=None, monitors=None,
                 simulation_length=1000.0, initial_conditions=None, conduction_speed=3.0, surface=None,
                 stimulus=None, noise_source='philox', chunk_steps=200000, device=None, stream_id=0):
        if surface is not None:
            raise NotImplementedError('surface simulations are not supported on the device path')
        if noise_source not in ('philox', 'reference'):
            raise ValueError("noise_source must be 'philox' or 'reference'")
        self.connectivity = connectivity
        self.coupling = coupling if coupling is not None else coupling_mod.Linear()
        self.model = model if model is not None else models_mod.Generic2dOscillator()
        self.integrator = integrator if integrator is not None else integrators_mod.HeunDeterministic()
        self.monitors = monitors if monitors is not None else [monitors_mod.TemporalAverage()]
        self.simulation_length = float(simulation_length)
        self.initial_conditions = initial_conditions
        self.conduction_speed = conduction_speed
        self.stimulus = stimulus
        self.noise_source = noise_source
        self.chunk_steps = int(chunk_steps)
        self.device = device
        self.stream_id = int(stream_id)
        self.current_step = 0
        self.current_state = None
        self.calls = 0
        self._configured = False

    # ------------------------------------------------------------ configure
    @property
    def good_history_shape(self):
        return (self.connectivity.horizon, len(self.model.state_variables),
                self.connectivity.number_of_regions, 1)

    def configure(self, full_configure=True):
        self.connectivity = adopt_connectivity(self.connectivity)
        self.model = adopt_model(self.model)
        self.coupling = adopt_coupling(self.coupling)
        self.integrator = adopt_integrator(self.integrator)
        if not isinstance(self.monitors, (list, tuple)):
            self.monitors = [self.monitors]
        self.monitors = [adopt_monitor(m) for m in self.monitors]
        name = type(self.model).__name__
        self._model_id = _lib.MODEL_IDS[name]
        cname = getattr(type(self.coupling), 'kernel_id', type(self.coupling).__name__)
        if cname not in _lib.CFUN_IDS:
            raise NotImplementedError('coupling %s' % cname)
        self._cfun_id = _lib.CFUN_IDS[cname]
        self._scheme_id = _lib.SCHEME_IDS[type(self.integrator).__name__]
        self.ncvar, self.nsv, self.nint, self.nobs, self.nparam = _lib.model_dims(self._model_id)
        if self._cfun_id == _lib.CFUN_IDS['SigmoidalJansenRit'] and self.ncvar < 2:
            raise NotImplementedError('SigmoidalJansenRit needs two coupling variables')
        self.model.configure()
        self.coupling.configure()
        self.integrator.configure()
        self.connectivity.configure()
        self.number_of_nodes = self.connectivity.number_of_regions
        dt = self.integrator.dt
        self.connectivity.set_idelays(dt)
        if self.integrator.stochastic:
            self.integrator.noise.configure_white(dt)
        self._configure_history()
        for m in self.monitors:
            m.config_for_sim(self)
            # node_coupling has one row per coupling variable, one for SigmoidalJansenRit (coupling.py:370-373)
            ncrows = 1 if self._cfun_id == _lib.CFUN_IDS['SigmoidalJansenRit'] else self.ncvar
            if isinstance(m, monitors_mod.AfferentCoupling) and np.asarray(m.voi).max() >= ncrows:
                raise IndexError('AfferentCoupling variables_of_interest %s: node_coupling has %d rows'
                                 % (np.asarray(m.voi).tolist(), ncrows))
        self._voi_codes = self.model.voi_codes()
        if len(self._voi_codes) > _lib.MAX_VOI:
            raise NotImplementedError('more than %d variables of interest' % _lib.MAX_VOI)
        self._conn = Connectome(self.connectivity.weights, self.connectivity.idelays, self.ncvar)
        self._params = self.model.kernel_params(self.number_of_nodes)
        self._sigma = None
        if self.integrator.stochastic:
            self._sigma = noise_sigma(self.integrator.noise.nsig, self.nint, self.number_of_nodes, dt)
        self._acc = None
        # AfferentCoupling monitors: the device averages over their period when they share one; with several
        # periods it writes every step and the averaging monitors reduce that stream on the host
        aff_periods = sorted({m.istep for m in self.monitors if isinstance(m, monitors_mod.AfferentCoupling)})
        self._aff_istep = aff_periods[0] if len(aff_periods) == 1 else (1 if aff_periods else 0)
        self._aff_carry = {}
        self._stim = None
        if self.stimulus is not None:
            if type(self.stimulus).__name__ != 'StimuliRegion':
                raise NotImplementedError('stimulus %s has no device implementation' % type(self.stimulus).__name__)
            if hasattr(self.stimulus, 'configure'):
                self.stimulus.configure()
            self.stimulus.configure_space()
            stvar = np.asarray(self.model.stvar, dtype=np.int64).reshape(-1)
            if stvar.size == 0 or stvar.min() < 0 or stvar.max() >= self.nsv:
                raise ValueError('model.stvar %s out of range' % stvar.tolist())
        self._configured = True
        return self

    # ------------------------------------------------------------ stimulus
    def _prepare_stimulus(self):
        """Temporal pattern on the grid r_[0 : simulation_length : dt], indexed
        from the step after the current one (simulator.py:290-306): the step
        s of this run reads index s - (current_step + 1)."""
        if self.stimulus is None:
            self._stim = None
            return
        time = np.r_[0.0:self.simulation_length:self.integrator.dt]
        self.stimulus.configure_time(time.reshape((1, -1)))
        self._stim = dict(temporal=np.asarray(self.stimulus.temporal_pattern, dtype=np.float64).reshape(-1),
                          weight=np.asarray(self.stimulus.spatial_pattern, dtype=np.float64).reshape(-1),
                          step0=self.current_step)

    def stimulus_spec(self, n_steps):
        """The stimulus of steps current_step + 1 .. + n_steps for InstanceSpec (None without one)."""
        if self.stimulus is None:
            return None
        if self._stim is None:
            self._prepare_stimulus()
        st = self._stim
        k0 = self.current_step - st['step0']
        if k0 + n_steps > st['temporal'].size:
            raise IndexError('index %d is out of bounds for the stimulus temporal pattern of size %d'
                             % (k0 + n_steps - 1, st['temporal'].size))
        return dict(temporal=st['temporal'][k0:k0 + n_steps], weight=st['weight'], vars=self.model.stvar)

    def _configure_history(self):
        """Initial history as SparseHistory.from_simulator (tvb/simulator/history.py:73-158)."""
        H, nsv, n, nm = self.good_history_shape
        ic = self.initial_conditions
        if ic is None:
            history = self.model.initial_for_simulator(self.integrator, (H, nsv, n, nm))
        else:
            ic = np.asarray(ic, dtype=np.float64)
            if ic.ndim == 3:
                ic = ic[..., None]
            if ic.shape[1:] != (nsv, n, nm):
                raise ValueError('Incorrect history sample shape %s, expected %s' % (ic.shape[1:], (nsv, n, nm)))
            if ic.shape[0] >= H:
                history = ic[-H:].copy()
            else:
                history = self.model.initial_for_simulator(self.integrator, (H, nsv, n, nm))
                shift = self.current_step % H
                history = np.roll(history, -shift, axis=0)
                history[:ic.shape[0]] = ic
                history = np.roll(history, shift, axis=0)
            self.current_step += ic.shape[0] - 1
        for it in range(history.shape[0]):
            self.model.bound(history[it])
        self.current_state = history[self.current_step % H].copy()
        self.history_buffer = history[:, self.model.cvar].astype(np.float32)  # (H, ncvar, n, 1)

    # ----------------------------------------------------------------- loop
    def _monitor_spec(self):
        raw = any(isinstance(m, monitors_mod.Raw) for m in self.monitors)
        tavg = [m for m in self.monitors if isinstance(m, monitors_mod.TemporalAverage)]
        bold = [m for m in self.monitors if isinstance(m, monitors_mod.Bold)]
        sub = [m for m in self.monitors if isinstance(m, monitors_mod.SubSample)]
        proj = [m for m in self.monitors if isinstance(m, monitors_mod.Projection)]
        if len(set(m.istep for m in tavg)) > 1 or len(set(m.istep for m in bold)) > 1 or \
                len(set(m.istep for m in sub)) > 1 or len(set(m.istep for m in proj)) > 1:
            raise NotImplementedError('monitors of one kind must share their period')
        self._sub_istep = sub[0].istep if sub else 0
        self._proj_istep = proj[0].istep if proj else 0
        bspec = None
        if bold:
            b = bold[0]
            bspec = dict(istep=b.istep, ii=b._interim_istep,
                         hrf=np.ascontiguousarray(b.hemodynamic_response_function[0], dtype=np.float64),
                         k1v0=b.k1_V0)
        return raw, (tavg[0].istep if tavg else 0), bspec

    def instance_spec(self, n_steps, stream=None):
        """The device description of the next `n_steps` of this simulation and
        its noise kind: (InstanceSpec, noise kind).  `stream` overrides the
        Philox stream id (default: the simulator's stream_id)."""
        n = self.number_of_nodes
        raw, tavg_istep, bspec = self._monitor_spec()
        fed = None
        noise_kind = _lib.NOISE_NONE
        if self.integrator.stochastic:
            if self.noise_source == 'reference':
                noise_kind = _lib.NOISE_FED
                fed = self.integrator.noise.random_stream.normal(size=(n_steps, self.nint, n)).astype(np.float32)
            else:
                noise_kind = _lib.NOISE_PHILOX
        spec = InstanceSpec(self._conn, self.history_buffer[..., 0], self.current_state[..., 0], self._params,
                            self.coupling.kernel_params(), n_steps, step0=self.current_step, sigma=self._sigma,
                            noise_fed=fed, seed=self.integrator.noise.noise_seed if self.integrator.stochastic else 0,
                            stream=self.stream_id if stream is None else stream, raw=raw, tavg_istep=tavg_istep,
                            bold=bspec, sub_istep=self._sub_istep, stim=self.stimulus_spec(n_steps),
                            aff_istep=self._aff_istep, proj_istep=self._proj_istep)
        if self._acc is not None:
            spec.acc0 = self._acc
        return spec, noise_kind

    def _run_device(self, n_steps):
        spec, noise_kind = self.instance_spec(n_steps)
        batch = Batch(self._model_id, self._cfun_id, self._scheme_id, noise_kind, self.integrator.dt,
                      self._voi_codes, [spec], device=self.device)
        batch.run(chunk=self.chunk_steps)
        st = batch.status()
        if st[0] & _lib.TVBK_STATUS_NONFINITE:
            self.log_nonfinite = True
        if st[0] & _lib.TVBK_STATUS_UNSUPPORTED:
            raise RuntimeError('the kernel variant chosen for this simulation does not write all its monitors')
        if st[0] & _lib.TVBK_STATUS_TIMEOUT:
            raise RuntimeError('a barrier of the cooperative launch gave up waiting: the run stopped early')
        out = batch.outputs_host()[0]
        if self._proj_istep:
            # the sensor projection of every sample: one float64 GEMM per monitor on the device
            dev = batch.outputs_device(0)['proj']
            for k, m in enumerate(self.monitors):
                if isinstance(m, monitors_mod.Projection):
                    out['proj_gain_%d' % k] = project_samples(dev, m).cpu().numpy()
        s0 = self.current_step
        self.current_step = s0 + n_steps
        self.current_state = batch.state(0).astype(np.float64)[..., None]
        self.history_buffer = ring_to_reference(batch.ring(0), self.current_step,
                                                self._conn.horizon)[..., None]
        self._acc = batch.accumulators(0)
        return s0, out

    def _collect(self, s0, n_steps, out):
        """Per-monitor (times, data) in the reference's format."""
        res = []
        steps = np.arange(s0 + 1, s0 + n_steps + 1)
        for k, m in enumerate(self.monitors):
            if isinstance(m, monitors_mod.ProgressLogger):
                m.log_steps(steps)
                res.append((np.array([]), np.array([])))
                continue
            if isinstance(m, monitors_mod.Raw):
                t, y = m.times(steps.astype(np.float64)), out['raw'][:, m.voi]
            elif isinstance(m, monitors_mod.TemporalAverage):
                st = steps[steps % m.istep == 0]
                t, y = m.times(st.astype(np.float64)), out['tavg'][:, m.voi]
            elif isinstance(m, monitors_mod.SubSample):
                st = steps[steps % m.istep == 0]
                t, y = m.times(st.astype(np.float64)), m.reduce(out['sub'][:, m.voi])
            elif isinstance(m, monitors_mod.Projection):
                st = steps[steps % m.istep == 0]
                t, y = m.times(st.astype(np.float64)), m.finish(out['proj_gain_%d' % k])
            elif isinstance(m, monitors_mod.AfferentCoupling):
                st = steps[steps % m.istep == 0]
                if m.istep == self._aff_istep:
                    y = out['aff'][:, m.voi]
                else:
                    carry = self._aff_carry.get(k)
                    if carry is None:
                        carry = np.zeros(out['aff'].shape[1:], dtype=np.float32)
                    y, self._aff_carry[k] = m.average(out['aff'], s0, carry)
                    y = y[:, m.voi]
                t = m.times(st.astype(np.float64))
            else:
                st = steps[steps % m.istep == 0]
                t, y = m.times(st.astype(np.float64)), out['bold'][:, m.voi]
            res.append((t, y.astype(np.float64)[..., None]))
        return res

    def __call__(self, simulation_length=None, random_state=None, n_steps=None):
        """Generator over monitor outputs, one list per step with an output
        (tvb/simulator/simulator.py:322-366); the device runs a block of
        steps at a time and the outputs are replayed step by step."""
        if not self._configured:
            raise RuntimeError('call configure() first')
        self.calls += 1
        if simulation_length is not None:
            self.simulation_length = float(simulation_length)
        if random_state is not None and self.integrator.stochastic:
            self.integrator.noise.random_stream.set_state(random_state)
        if n_steps is None:
            n_steps = int(math.ceil(self.simulation_length / self.integrator.dt))
        elif not np.issubdtype(type(n_steps), np.integer):
            raise TypeError('Incorrect type for n_steps: %s, expected integer' % type(n_steps))
        self._prepare_stimulus()
        left = int(n_steps)
        while left > 0:
            k = min(left, self.chunk_steps)
            s0, out = self._run_device(k)
            per_mon = self._collect(s0, k, out)
            ptr = [0] * len(self.monitors)
            sample_steps = []
            for m in self.monitors:
                steps = np.arange(s0 + 1, s0 + k + 1)
                sample_steps.append(set() if isinstance(m, monitors_mod.ProgressLogger)
                                    else set(steps[steps % m.istep == 0].tolist()))
            for step in range(s0 + 1, s0 + k + 1):
                row = []
                for j, m in enumerate(self.monitors):
                    if step in sample_steps[j]:
                        t, y = per_mon[j]
                        row.append([t[ptr[j]], y[ptr[j]]])
                        ptr[j] += 1
                    else:
                        row.append(None)
                if any(r is not None for r in row):
                    yield row
            left -= k

    # ------------------------------------------------------ checkpoint / resume
    def history_state(self):
        """The simulation's state in the layout of the framework's
        SimulationHistory (tvb_framework/tvb/core/entities/file/simulator/
        simulation_history_h5.py:32-118), as a dict:

        history (H, ncvar, n, 1) float32 and current_state (nsv, n, 1) as the
        reference's history.buffer and current_state; current_step;
        monitor_stock_<k> for the k-th monitor (1-based): Raw an empty array,
        TemporalAverage and AfferentCouplingTemporalAverage (istep, nvoi_k, n, 1)
        holding the current period's sum
        in row 0 (the reference's stock rows are only ever read as their mean
        at the next sample, which this reproduces), Bold the 4 ms stock
        (stock_len, nvoi_k, n, 1) float64; monitor_names; for stochastic
        schemes the noise RandomState as integrator_noise_rng_state_*.  Also
        monitor_interim_<k>, Bold's running 4 ms sum (nvoi_k, n, 1), which the
        reference does not store (it restarts that average on reload).  EEG /
        MEG / iEEG: the stock is the reference's running gain . observed sum
        (sensors, nvoi_k) and monitor_interim_<k> the observed sum (nvoi_k, n)
        that resuming needs; the observation-noise RandomState is not stored.
        """
        if not self._configured:
            raise RuntimeError('call configure() first')
        n = self.number_of_nodes
        st = {'history': self.history_buffer.copy(), 'current_state': np.array(self.current_state, copy=True),
              'current_step': int(self.current_step), 'monitor_names': []}
        acc = self._acc or {}
        for k, m in enumerate(self.monitors):
            name = 'monitor_stock_%d' % (k + 1)
            st['monitor_names'].append(type(m).__name__)
            voi = np.asarray(m.voi, dtype=int)
            if isinstance(m, monitors_mod.TemporalAverage):
                stock = np.zeros((m.istep, voi.size, n, 1))
                if 'tavg_acc' in acc:
                    stock[0, :, :, 0] = acc['tavg_acc'][voi]
                st[name] = stock
            elif isinstance(m, monitors_mod.AfferentCouplingTemporalAverage):
                stock = np.zeros((m.istep, voi.size, n, 1))
                if k in self._aff_carry:
                    stock[0, :, :, 0] = self._aff_carry[k][voi]
                elif 'aff_acc' in acc and m.istep == self._aff_istep:
                    stock[0, :, :, 0] = acc['aff_acc'][voi]
                st[name] = stock
            elif isinstance(m, monitors_mod.Projection):
                # the reference's running sum of gain . observed (sensors, nvoi), and the observed sum itself
                interim = np.zeros((voi.size, n), dtype=np.float32)
                if 'proj_acc' in acc:
                    interim = acc['proj_acc'][voi]
                st[name] = m.gain.dot(interim.astype(np.float64).T)
                st['monitor_interim_%d' % (k + 1)] = interim.copy()
            elif isinstance(m, monitors_mod.Bold):
                SL = m.hemodynamic_response_function.shape[1]
                stock = np.zeros((SL, voi.size, n, 1))
                interim = np.zeros((voi.size, n, 1))
                if 'bold_stock' in acc:
                    stock[..., 0] = acc['bold_stock'][:, voi]
                    interim[..., 0] = acc['bold_acc'][voi]
                st[name] = stock
                st['monitor_interim_%d' % (k + 1)] = interim
            else:
                st[name] = np.empty([])
        if self.integrator.stochastic:
            algo, keys, pos, has_gauss, cached = self.integrator.noise.random_stream.get_state()
            st.update(integrator_noise_rng_state_algo=algo, integrator_noise_rng_state_keys=keys,
                      integrator_noise_rng_state_pos=pos, integrator_noise_rng_state_has_gauss=has_gauss,
                      integrator_noise_rng_state_cached_gauss=cached)
        return st

    def set_history_state(self, st):
        """Resume from a dict produced by ``history_state`` (or a reference
        SimulationHistory's fields): the next run continues from that step."""
        if not self._configured:
            raise RuntimeError('call configure() first')
        n = self.number_of_nodes
        hist = np.asarray(st['history'], dtype=np.float32)
        if hist.ndim == 3:
            hist = hist[..., None]
        if hist.shape != self.history_buffer.shape:
            raise ValueError('history shape %s, expected %s' % (hist.shape, self.history_buffer.shape))
        self.history_buffer = hist.copy()
        cs = np.asarray(st['current_state'], dtype=np.float64)
        self.current_state = (cs if cs.ndim == 3 else cs[..., None]).copy()
        self.current_step = int(st['current_step'])
        nvoi = len(self._voi_codes)
        acc = {}
        names = list(st.get('monitor_names', [type(m).__name__ for m in self.monitors]))
        for k, m in enumerate(self.monitors):
            if k < len(names) and names[k] != type(m).__name__:
                raise ValueError('monitor %d is %s in the stored state, %s here' % (k + 1, names[k], type(m).__name__))
            stock = st.get('monitor_stock_%d' % (k + 1))
            voi = np.asarray(m.voi, dtype=int)
            if isinstance(m, monitors_mod.TemporalAverage) and stock is not None:
                t = np.zeros((nvoi, n), dtype=np.float32)
                ph = self.current_step % m.istep
                t[voi] = np.asarray(stock)[:ph, :, :, 0].sum(axis=0)
                acc['tavg_acc'] = t
            elif isinstance(m, monitors_mod.AfferentCouplingTemporalAverage) and stock is not None:
                t = np.zeros((self.ncvar, n), dtype=np.float32)
                ph = self.current_step % m.istep
                t[voi] = np.asarray(stock)[:ph, :, :, 0].sum(axis=0)
                if m.istep == self._aff_istep:
                    acc['aff_acc'] = t
                else:
                    self._aff_carry[k] = t
            elif isinstance(m, monitors_mod.Projection) and stock is not None:
                interim = st.get('monitor_interim_%d' % (k + 1))
                if interim is None:
                    if self.current_step % m.istep and np.any(np.asarray(stock)):
                        raise NotImplementedError('resuming %s inside a sampling period needs monitor_interim_%d'
                                                  % (type(m).__name__, k + 1))
                    interim = np.zeros((voi.size, n))
                t = acc.get('proj_acc', np.zeros((nvoi, n), dtype=np.float32))
                t[voi] = np.asarray(interim, dtype=np.float32)
                acc['proj_acc'] = t
            elif isinstance(m, monitors_mod.Bold) and stock is not None:
                stock = np.asarray(stock)
                b = np.zeros((stock.shape[0], nvoi, n))
                b[:, voi] = stock[..., 0]
                acc['bold_stock'] = b
                ia = np.zeros((nvoi, n))
                interim = st.get('monitor_interim_%d' % (k + 1))
                if interim is not None:
                    ia[voi] = np.asarray(interim)[..., 0]
                acc['bold_acc'] = ia
        self._acc = acc or None
        if self.integrator.stochastic and st.get('integrator_noise_rng_state_algo') is not None:
            self.integrator.noise.random_stream.set_state((
                st['integrator_noise_rng_state_algo'], st['integrator_noise_rng_state_keys'],
                st['integrator_noise_rng_state_pos'], st['integrator_noise_rng_state_has_gauss'],
                st['integrator_noise_rng_state_cached_gauss']))
        return self

    def run(self, **kwds):
        """All monitor outputs of one call: [(times, data(T, nvoi, n, 1)), ...]
        (tvb/simulator/simulator.py:620-639)."""
        if not self._configured:
            raise RuntimeError('call configure() first')
        simulation_length = kwds.get('simulation_length')
        n_steps = kwds.get('n_steps')
        random_state = kwds.get('random_state')
        self.calls += 1
        if simulation_length is not None:
            self.simulation_length = float(simulation_length)
        if random_state is not None and self.integrator.stochastic:
            self.integrator.noise.random_stream.set_state(random_state)
        if n_steps is None:
            n_steps = int(math.ceil(self.simulation_length / self.integrator.dt))
        self._prepare_stimulus()
        left = int(n_steps)
        parts = [[] for _ in self.monitors]
        while left > 0:
            k = min(left, self.chunk_steps)
            s0, out = self._run_device(k)
            for j, (t, y) in enumerate(self._collect(s0, k, out)):
                parts[j].append((t, y))
            left -= k
        res = []
        for j in range(len(self.monitors)):
            ts = [p[0] for p in parts[j] if len(p[0])]
            ys = [p[1] for p in parts[j] if len(p[0])]
            if ts:
                res.append((np.concatenate(ts), np.concatenate(ys)))
            else:
                res.append((np.array([]), np.array([])))
        return res
