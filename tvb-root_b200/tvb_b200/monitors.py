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


MONITORS = {c.__name__: c for c in (Raw, TemporalAverage, Bold, SubSample, GlobalAverage, SpatialAverage,
                                    AfferentCoupling, AfferentCouplingTemporalAverage)}
