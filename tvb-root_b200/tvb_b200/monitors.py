"""Raw, TemporalAverage and Bold monitors (tvb/simulator/monitors.py).

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


MONITORS = {cls.__name__: cls for cls in (Raw, TemporalAverage, Bold, SubSample, GlobalAverage, SpatialAverage)}
