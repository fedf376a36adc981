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


MONITORS = {cls.__name__: cls for cls in (Raw, TemporalAverage, Bold)}
