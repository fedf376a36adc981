"""Raw, TemporalAverage, Bold, SubSample, GlobalAverage, SpatialAverage and
AfferentCoupling monitors (tvb/simulator/monitors.py).

Sampling runs inside the simulation kernel; these classes resolve the step
constants exactly as the reference does and shape the outputs.
"""
import numpy as np

from .equations import FirstOrderVolterra


def iround(x):
    """Rounding used for monitor periods (tvb/simulator/backend/ref.py:103-121)."""
    y = round(x) - .5
    return int(y) + (y > 0)


class Monitor:
    default_period = 0.9765625

    def __init__(self, period=None, variables_of_interest=None):
        self.period = float(self.default_period if period is None else period)
        self.variables_of_interest = None if variables_of_interest is None else np.asarray(
            variables_of_interest, dtype=int)
        self.voi = None
        self.istep = None
        self.dt = None

    def _config_vois(self, sim):
        """monitors.py:93-96: indices into the model's variables of interest."""
        vois = self.variables_of_interest
        self.voi = vois if vois is not None and vois.size else np.arange(len(sim.model.variables_of_interest))

    def _config_time(self, sim):
        self.dt = sim.integrator.dt
        self.istep = iround(self.period / self.dt)

    def config_for_sim(self, sim):
        self._config_vois(sim)
        self._config_time(sim)
        return self

    def __repr__(self):
        return '%s(period=%g)' % (type(self).__name__, self.period)


class Raw(Monitor):
    """Every step, all variables of interest (monitors.py:160-190)."""
    default_period = 0.0

    def _config_vois(self, sim):
        self.voi = np.arange(len(sim.model.variables_of_interest))

    def _config_time(self, sim):
        self.dt = sim.integrator.dt
        self.period = sim.integrator.dt
        self.istep = 1

    def times(self, steps):
        return steps * self.dt


class RawVoi(Raw):
    """Every step, the chosen variables of interest (monitors.py:193-211)."""

    def _config_vois(self, sim):
        Monitor._config_vois(self, sim)


class ProgressLogger(Monitor):
    """Logs the step and time every int(period / dt) steps from the first
    step it sees and records nothing (monitors.py:1005-1026)."""
    default_period = 1000.0

    def _config_time(self, sim):
        self.dt = sim.integrator.dt
        self.istep = max(int(self.period / self.dt), 1)
        self._first = None

    def log_steps(self, steps):
        import logging
        log = logging.getLogger(__name__)
        for s in np.asarray(steps):
            if self._first is None:
                self._first = int(s)
            if (int(s) - self._first) % self.istep == 0:
                log.info('step %d time %.4f s', int(s), int(s) * self.dt / 1e3)


class TemporalAverage(Monitor):
    """Mean over each period, stamped at its middle (monitors.py:363-391)."""

    def times(self, steps):
        return (steps - self.istep / 2.0) * self.dt


class Bold(Monitor):
    """HRF-convolved 4 ms averages (monitors.py:834-962) with the
    FirstOrderVolterra kernel; accumulation and the HRF dot are float64."""
    default_period = 2000.0

    def __init__(self, period=None, variables_of_interest=None, hrf_kernel=None, hrf_length=20000.0):
        super().__init__(period, variables_of_interest)
        self.hrf_kernel = hrf_kernel if hrf_kernel is not None else FirstOrderVolterra()
        if not isinstance(self.hrf_kernel, FirstOrderVolterra):
            raise NotImplementedError('Bold on the device supports the FirstOrderVolterra kernel')
        self.hrf_length = float(hrf_length)
        self.hemodynamic_response_function = None

    def compute_hrf(self):
        """monitors.py:903-929."""
        self._stock_sample_rate = 2.0 ** -2
        self._stock_steps = int(np.ceil(self._stock_sample_rate * self.hrf_length))
        stock_time_max = self.hrf_length / 1000.0
        stock_time_step = stock_time_max / self._stock_steps
        self._stock_time = np.arange(0.0, stock_time_max, stock_time_step)
        G = self.hrf_kernel.evaluate(self._stock_time)[::-1]
        self.hemodynamic_response_function = G[np.newaxis, :].copy()
        self._interim_period = 1.0 / self._stock_sample_rate
        self._interim_istep = int(round(self._interim_period / self.dt))

    def _config_time(self, sim):
        super()._config_time(sim)
        self.compute_hrf()

    @property
    def k1_V0(self):
        return self.hrf_kernel.parameters['k_1'] * self.hrf_kernel.parameters['V_0']

    def times(self, steps):
        return steps * self.dt


class SubSample(Monitor):
    """The variables of interest at every step with step % istep == 0,
    stamped step * dt (monitors.py:213-222)."""

    def times(self, steps):
        return steps * self.dt

    def reduce(self, y):
        """(T, nvoi, n) sampled states -> this monitor's data."""
        return y


class GlobalAverage(SubSample):
    """Mean over all regions of the sub-sampled variables of interest,
    (T, nvoi, 1) (monitors.py:342-360)."""

    def reduce(self, y):
        return y.astype(np.float64).mean(axis=2)[:, :, None]


class SpatialAverage(SubSample):
    """Mean over each group of regions of the sub-sampled variables of
    interest; spatial_mask gives each region's group, a contiguous set of
    indices from 0 (monitors.py:231-326).  (T, nvoi, groups)."""

    def __init__(self, period=None, variables_of_interest=None, spatial_mask=None):
        super().__init__(period, variables_of_interest)
        if spatial_mask is None:
            raise NotImplementedError('SpatialAverage on the device needs an explicit spatial_mask')
        self.spatial_mask = np.asarray(spatial_mask, dtype=int)

    def config_for_sim(self, sim):
        super().config_for_sim(sim)
        n = sim.number_of_nodes
        if self.spatial_mask.size != n:
            raise ValueError('spatial_mask must be a vector of length number_of_nodes.')
        areas = np.unique(self.spatial_mask)
        if not np.all(areas == np.arange(len(areas))):
            raise ValueError('Areas in the spatial_mask must be specified as a contiguous set of indices '
                             'starting from zero.')
        total = np.zeros((n, len(areas)))
        total[np.arange(n), self.spatial_mask] = 1
        total = total.T
        self.spatial_mean = total / total.sum(axis=1)[:, None]
        return self

    def reduce(self, y):
        # numpy.dot(spatial_mean, state[voi]) per sample, (groups, nvoi) -> (nvoi, groups)
        return np.einsum('gn,tvn->tvg', self.spatial_mean, y.astype(np.float64))


class AfferentCoupling(Monitor):
    """The coupling input of the model, node_coupling, recorded after every
    step: at step s the coupling that step s + 1 receives (simulator.py:
    314-320, 358-361; monitors.py:394-412).  variables_of_interest indexes
    the coupling variables (default: all of the model's cvar).  Data
    (T, nvoi, n), stamped step * dt."""
    default_period = 0.0

    def _config_vois(self, sim):
        vois = self.variables_of_interest
        self.voi = vois if vois is not None and vois.size else np.arange(len(sim.model.cvar))

    def _config_time(self, sim):
        self.dt = sim.integrator.dt
        self.period = sim.integrator.dt
        self.istep = 1

    def times(self, steps):
        return steps * self.dt


class AfferentCouplingTemporalAverage(AfferentCoupling):
    """AfferentCoupling averaged over each period and stamped at its middle, the
    TemporalAverage rule (monitors.py:415-433, 363-391)."""

    def _config_time(self, sim):
        Monitor._config_time(self, sim)
        if self.istep < 1:
            raise ValueError('AfferentCouplingTemporalAverage needs a period of at least one step (got %g)'
                             % self.period)

    def times(self, steps):
        return (steps - self.istep / 2.0) * self.dt

    def average(self, raw, s0, carry):
        """This monitor's samples from the every-step AfferentCoupling stream of
        steps s0 + 1 .. s0 + T, raw (T, ncvar, n) float32, when another
        AfferentCoupling monitor with a different period shares the run.
        carry is the float32 sum of the current period so far.  The sums run
        in step order in float32 and are divided by istep, the arithmetic the
        device does for a single period.  Returns (samples (S, ncvar, n),
        new carry)."""
        istep, T = self.istep, raw.shape[0]
        inv = np.float32(istep)
        acc = np.array(carry, dtype=np.float32, copy=True)
        out = []
        first = (s0 // istep + 1) * istep - s0       # steps up to and including the first sample step
        h = min(T, first)
        for k in range(h):
            acc = acc + raw[k]
        if first <= T:
            out.append(acc / inv)
            acc = np.zeros_like(acc)
        rest = raw[h:]
        W = rest.shape[0] // istep
        if W:
            R = rest[:W * istep].reshape((W, istep) + raw.shape[1:])
            w = np.zeros((W,) + raw.shape[1:], dtype=np.float32)
            for j in range(istep):
                w = w + R[:, j]
            out.extend(w / inv)
        for k in range(W * istep, rest.shape[0]):
            acc = acc + rest[k]
        samples = np.stack(out) if out else np.zeros((0,) + raw.shape[1:], dtype=np.float32)
        return samples, acc


MONITORS = {c.__name__: c for c in (Raw, RawVoi, ProgressLogger, TemporalAverage, Bold, SubSample, GlobalAverage,
                                    SpatialAverage, AfferentCoupling, AfferentCouplingTemporalAverage)}


def _array(obj, attr):
    """obj.<attr> for the reference's datatypes (and this package's), or obj itself for a plain array."""
    return np.asarray(getattr(obj, attr, obj))


class Projection(Monitor):
    """Lead-field monitors (monitors.py:436-643) for region simulations.

    The reference adds gain . observed state at every step and samples the
    sum over int(period / dt) steps divided by that count.  The gain is
    linear, so the device keeps the mean of the observed variables over each
    period (one float32 stream for all projection monitors of a run) and the
    sensor projection is a float64 GEMM on the device over all samples.
    Observation noise (sqrt(dt) times a normal draw of the monitor's own
    RandomState per sample, (sensors, nvoi) in order) is added on the host in
    sample order, so it is the reference's stream.

    sensors: object with labels / locations / usable (or the reference's
    Sensors); projection: object with projection_data (sensors, vertices) or
    an array; region_mapping: object with array_data (vertices,) or an array;
    obsnoise: 'default' (white, RandomState(42)), None, or an object with
    random_stream and ntau == 0.
    """
    default_period = 1e3 / 1024.0

    def __init__(self, period=None, variables_of_interest=None, sensors=None, projection=None, region_mapping=None,
                 obsnoise='default'):
        super().__init__(period, variables_of_interest)
        self.sensors = sensors
        self.projection = projection
        self.region_mapping = region_mapping
        if obsnoise == 'default':
            from .noise import Additive
            obsnoise = Additive()
        if obsnoise is not None and float(getattr(obsnoise, 'ntau', 0.0)) > 0.0:
            raise NotImplementedError('coloured observation noise is not supported')
        self.obsnoise = obsnoise
        self.gain = None

    def analytic(self, loc, ori):
        raise NotImplementedError('no general analytic lead field; give a projection matrix')

    def _config_time(self, sim):
        # the reference samples every int(period / dt) steps (monitors.py:600), not iround(period / dt)
        self.dt = sim.integrator.dt
        self.istep = int(self.period / self.dt)
        if self.istep < 1:
            raise ValueError('%s period %g is shorter than dt' % (type(self).__name__, self.period))

    def config_for_sim(self, sim):
        """The region lead field (monitors.py:492-600): vertex gains summed per
        region through the region mapping (cortical regions), the analytic
        lead field for non-cortical regions, unusable sensors and non-finite
        entries zeroed."""
        super().config_for_sim(sim)
        if self.sensors is None:
            raise ValueError('%s needs sensors' % type(self).__name__)
        if hasattr(self.sensors, 'configure'):
            self.sensors.configure()
        if self.obsnoise is not None and hasattr(self.obsnoise, 'configure_white'):
            self.obsnoise.configure_white(dt=self.dt)
        conn = sim.connectivity
        n = conn.number_of_regions
        cortical = np.asarray(getattr(conn, 'cortical', np.zeros(0)), dtype=bool)
        if cortical.size == 0:
            cortical = np.ones(n, dtype=bool)
        non_cortical, = np.where(~cortical)
        cortical_idx, = np.where(cortical)
        if self.region_mapping is None:
            raise ValueError('Please specify a region mapping on the EEG/MEG/iEEG monitor when performing a '
                             'region simulation.')
        if self.projection is None:
            raise ValueError('%s needs a projection matrix' % type(self).__name__)
        rmap = _array(self.region_mapping, 'array_data').astype(np.int64)
        gain = np.array(_array(self.projection, 'projection_data'), dtype=np.float64)
        cortical_rmap = rmap.copy()
        if rmap.max() + 1 != cortical.sum():
            drop = np.hstack([np.argwhere(rmap == i)[:, 0] for i in non_cortical])
            cortical_rmap = np.delete(cortical_rmap, drop)
        if gain.shape[1] == cortical_rmap.size:
            g = np.zeros((gain.shape[0], n))
            np.add.at(g.T, cortical_rmap, gain.T)
            gain = g
        if non_cortical.size:
            src = (np.asarray(conn.centres)[non_cortical], np.asarray(conn.orientations)[non_cortical])
            sub_gain = self.analytic(*src)
            if gain.shape[1] == cortical_idx.size + non_cortical.size:
                gain[:, non_cortical] = sub_gain
            else:
                full = np.zeros((gain.shape[0], gain.shape[1] + sub_gain.shape[1]))
                full[:, cortical_idx] = gain
                full[:, non_cortical] = sub_gain
                gain = full
        if gain.shape[1] != n:
            raise ValueError('lead field has %d sources for %d regions' % (gain.shape[1], n))
        usable = getattr(self.sensors, 'usable', None)
        if usable is not None and not np.asarray(usable).all():
            gain[~np.asarray(usable, dtype=bool)] = 0.0
        gain[~np.isfinite(gain)] = 0.0
        self.gain = gain
        return self

    def times(self, steps):
        return (steps - self.istep / 2.0) * self.dt

    def finish(self, y):
        """(T, nvoi, S) noise-free projections -> this monitor's samples: the
        observation noise of each sample in order, then post()."""
        y = np.array(y, dtype=np.float64)
        if self.obsnoise is not None:
            rs = self.obsnoise.random_stream
            for t in range(y.shape[0]):
                y[t] += (np.sqrt(self.dt) * rs.normal(size=(y.shape[2], y.shape[1]))).T
        return self.post(y)

    def post(self, y):
        return y


class EEG(Projection):
    """EEG (monitors.py:646-729): reference = None (reference-free), a sensor
    label, or 'average'.  The analytic lead field of non-cortical regions is
    the single-sphere formula of Sarvas (1987), Eq. 12."""

    def __init__(self, period=None, variables_of_interest=None, sensors=None, projection=None, region_mapping=None,
                 obsnoise='default', reference=None, sigma=1.0):
        super().__init__(period, variables_of_interest, sensors, projection, region_mapping, obsnoise)
        self.reference = reference
        self.sigma = float(sigma)

    def config_for_sim(self, sim):
        super().config_for_sim(sim)
        S = self.gain.shape[0]
        ref = np.zeros(S)
        if self.reference:
            if self.reference.lower() != 'average':
                ref[list(np.asarray(self.sensors.labels).tolist()).index(self.reference)] = 1.0
            else:
                ref[:] = 1.0 / S
        self._ref_mask = np.isfinite(self.gain).all(axis=1)
        self._ref_vec = ref[self._ref_mask]
        return self

    def analytic(self, loc, ori):
        """Potential of unit dipoles at loc with orientation ori on sensors
        projected to a sphere 1.05125 times the sources' radius around their
        centre: Q . a / |a|^3 / (4 pi sigma)."""
        centre = np.mean(loc, axis=0)[None]
        radius = 1.05125 * max(np.sqrt(np.sum((loc - centre) ** 2, axis=1)))
        sen = np.array(self.sensors.locations, dtype=np.float64)
        sen = sen / np.sqrt(np.sum(sen ** 2, axis=1))[:, None] * radius + centre
        out = np.zeros((sen.shape[0], loc.shape[0]))
        for k in range(sen.shape[0]):
            a = sen[k] - loc
            na = np.sqrt(np.sum(a ** 2, axis=1))[:, None]
            out[k] = np.sum(ori * (a / na ** 3), axis=1) / (4.0 * np.pi * self.sigma)
        return out

    def post(self, y):
        r = np.tensordot(y[:, :, self._ref_mask], self._ref_vec, axes=([2], [0]))   # (T, nvoi)
        return y - r[:, :, None]


class MEG(Projection):
    """MEG (monitors.py:732-790); non-cortical regions use the single-sphere
    magnetic lead field of Sarvas (1987), Eq. 25."""

    def analytic(self, loc, ori):
        """|B| of unit dipoles (loc, ori) at sensors projected to a sphere 1.01
        times the sources' radius around their centre, with
        B = mu0 / (4 pi F^2) (F Q x r0 - (Q x r0 . r) grad F)."""
        mu_0 = 1.25663706e-6
        r0, Q = loc, ori
        centre = np.mean(r0, axis=0)[None, :]
        radius = 1.01 * max(np.sqrt(np.sum((r0 - centre) ** 2, axis=1)))
        sen = np.array(self.sensors.locations, dtype=np.float64)
        sen = sen / np.sqrt(np.sum(sen ** 2, axis=1))[:, None] * radius + centre
        B = np.zeros((sen.shape[0], r0.shape[0], 3))
        for k in range(sen.shape[0]):
            r = sen[k][None, :]
            a = r - r0
            na = np.sqrt(np.sum(a ** 2, axis=1))[:, None]
            nr = np.sqrt(np.sum(r ** 2, axis=1))[:, None]
            F = a * (nr * a + nr ** 2 - np.sum(r0 * r, axis=1)[:, None])
            adotr = np.sum((a / na) * r, axis=1)[:, None]
            gradF = (na ** 2 / nr + adotr + 2.0 * na + 2.0 * nr) * r - (a + 2.0 * nr + adotr * r0)
            B[k] = (mu_0 / (4.0 * np.pi * F ** 2)) * (np.cross(F * Q, r0)
                                                       - np.sum(np.cross(Q, r0) * (r * gradF), axis=1)[:, None])
        return np.sqrt(np.sum(B ** 2, axis=2))


class iEEG(Projection):
    """Intracranial EEG (monitors.py:793-831); non-cortical regions use the
    point dipole in a homogeneous medium at the sensors' own positions,
    Q . a / |a|^3 / (4 pi sigma)."""

    def __init__(self, period=None, variables_of_interest=None, sensors=None, projection=None, region_mapping=None,
                 obsnoise='default', sigma=1.0):
        super().__init__(period, variables_of_interest, sensors, projection, region_mapping, obsnoise)
        self.sigma = float(sigma)

    def analytic(self, loc, ori):
        sen = np.array(self.sensors.locations, dtype=np.float64)
        out = np.zeros((sen.shape[0], loc.shape[0]))
        for k in range(sen.shape[0]):
            a = sen[k] - loc
            na = np.sqrt(np.sum(a ** 2, axis=1))[:, None]
            out[k] = np.sum(ori * (a / na ** 3), axis=1) / (4.0 * np.pi * self.sigma)
        return out


MONITORS.update({c.__name__: c for c in (EEG, MEG, iEEG)})
