"""Balloon-Windkessel BOLD of a neural-activity time series on the device
(tvb_library/tvb/analyzers/fmri_balloon.py:72-364).

    bm = BalloonModel(time_series=ts)       # ts: .data (T, nvar, n, modes), .sample_period, .sample_period_unit
    bold = bm.evaluate()                    # .data (T', 1, n, modes) float64, .time in s, .sample_period in s

The input transformation (first variable, sum over variables, or the
absolute first difference), the optional mean subtraction and the derived
coefficients k1, k2, k3 are computed on the host exactly as the reference
does; the ODE integration (Heun, float64, one thread per series) and the BOLD
equation run in ``tvbk_balloon``.  A time series may also be a plain array
with ``sample_period`` (ms) given separately; several instances can be
integrated in one call by stacking them along the region axis.
"""
import ctypes

import numpy as np
import torch

from . import _lib


class Result:
    """TimeSeries-like result: data (T, 1, n, modes), time (s), sample_period (s)."""

    def __init__(self, data, time, sample_period):
        self.data = data
        self.time = time
        self.sample_period = sample_period
        self.sample_period_unit = 's'


class BalloonModel:
    _defaults = dict(tau_s=1.54, tau_f=1.44, tau_o=0.98, alpha=0.32, TE=0.04, V0=4.0, E0=0.4, epsilon=0.5,
                     nu_0=40.3, r_0=25.0, RBM=True, bold_model='nonlinear', neural_input_transformation='none',
                     normalize_neural_input=False)

    def __init__(self, time_series=None, sample_period=None, sample_period_unit='ms', time=None, **kwargs):
        for k, v in self._defaults.items():
            setattr(self, k, v)
        for k, v in kwargs.items():
            if k not in self._defaults:
                raise TypeError('BalloonModel has no parameter %r' % k)
            setattr(self, k, v)
        self.time_series = time_series
        self._sample_period = sample_period
        self._sample_period_unit = sample_period_unit
        self._time = time

    def _series(self):
        ts = self.time_series
        if not isinstance(ts, np.ndarray) and hasattr(ts, 'sample_period'):
            data = np.asarray(ts.data, dtype=np.float64)
            period, unit = float(ts.sample_period), getattr(ts, 'sample_period_unit', 'ms')
            time = getattr(ts, 'time', None)
        else:
            data = np.asarray(ts, dtype=np.float64)
            period, unit, time = float(self._sample_period), self._sample_period_unit, self._time
        if data.ndim != 4:
            raise ValueError('time series data must be (time, variables, regions, modes)')
        scale = {'s': 1.0, 'sec': 1.0, 'ms': 1e3, 'msec': 1e3, 'us': 1e6, 'usec': 1e6}[unit]
        rate = scale / period                                       # samples per second
        time = np.arange(data.shape[0]) * period if time is None else np.asarray(time, dtype=np.float64)
        return data, rate, rate * period, time

    def compute_derived_parameters(self):
        """k1, k2, k3 (fmri_balloon.py:285-308)."""
        eps = float(np.asarray(self.epsilon).reshape(-1)[0])
        if not self.RBM:
            return 7.0 * self.E0, 2.0 * self.E0, 1.0 - eps
        return 4.3 * self.nu_0 * self.E0 * self.TE, eps * self.r_0 * self.E0 * self.TE, 1 - eps

    def input_transformation(self, data, time, unit_factor):
        """fmri_balloon.py:310-337."""
        mode = getattr(self.neural_input_transformation, 'value', self.neural_input_transformation)
        if mode == 'none':
            return data[:, :1], time / unit_factor
        if mode == 'abs_diff':
            return np.abs(np.diff(data, axis=0)), (time[1:] - time[:-1]) / unit_factor
        if mode == 'sum':
            return np.sum(data, axis=1)[:, np.newaxis], time / unit_factor
        raise ValueError('Bad transformation mode %r' % mode)

    def evaluate(self, device=None):
        data, rate, unit_factor, time = self._series()
        x, t_int = self.input_transformation(data, time, unit_factor)
        if self.normalize_neural_input:
            x = x - x.mean(axis=0)[np.newaxis, :]
        T, _, n, m = x.shape
        k1, k2, k3 = self.compute_derived_parameters()
        dt = 1.0 / rate
        lib = _lib.load()
        dev = torch.device(device if device is not None else 'cuda')
        xd = torch.from_numpy(np.ascontiguousarray(x[:, 0].reshape(T, n * m))).to(dev)
        out = torch.empty_like(xd)
        params = np.array([self.tau_s, self.tau_f, self.tau_o, self.alpha, self.E0, self.V0, k1, k2, k3],
                          dtype=np.float64)
        model = getattr(self.bold_model, 'value', self.bold_model)
        st = torch.cuda.current_stream(dev)
        _lib.check(lib.tvbk_balloon(ctypes.c_void_p(xd.data_ptr()), T, n * m, dt, _lib.ptr(params),
                                    1 if model == 'nonlinear' else 0, ctypes.c_void_p(out.data_ptr()),
                                    ctypes.c_void_p(st.cuda_stream)))
        y = out.cpu().numpy().reshape(T, 1, n, m)
        return Result(y, t_int, dt)
