"""Equations of the stimulus patterns and the Bold monitor's haemodynamic
response kernel, with the reference's class names, parameter names and
defaults (tvb/datatypes/equations.py).  They are evaluated on the host in
float64 -- once per run, on the time grid or the region weights -- and the
device reads the resulting arrays.
"""
import numpy as np


class Equation:
    """Base: ``parameters`` starts from the class defaults and is updated from
    the constructor's dict; ``evaluate(var)`` is the equation of ``var``."""
    _defaults = {}

    def __init__(self, parameters=None):
        self.parameters = dict(self._defaults)
        if parameters:
            self.parameters.update(parameters)

    def _p(self, *names):
        return [self.parameters[k] for k in names]

    def evaluate(self, var):
        raise NotImplementedError

    def __repr__(self):
        return '%s(%r)' % (type(self).__name__, self.parameters)


class DiscreteEquation(Equation):
    """The value itself: each region is assigned its weight (equations.py:136-147)."""

    def evaluate(self, var):
        return np.asarray(var, dtype=np.float64)


class Linear(Equation):
    """a var + b (equations.py:150-164)."""
    _defaults = {'a': 1.0, 'b': 0.0}

    def evaluate(self, var):
        a, b = self._p('a', 'b')
        return a * var + b


class Gaussian(Equation):
    """amp exp(-(var - midpoint)^2 / (2 sigma^2)) + offset (equations.py:212-229)."""
    _defaults = {'amp': 1.0, 'sigma': 1.0, 'midpoint': 0.0, 'offset': 0.0}

    def evaluate(self, var):
        amp, sigma, mid, off = self._p('amp', 'sigma', 'midpoint', 'offset')
        return amp * np.exp(-((var - mid) ** 2 / (2.0 * sigma ** 2))) + off


class DoubleGaussian(Equation):
    """Difference of two Gaussians (equations.py:232-251)."""
    _defaults = {'amp_1': 0.5, 'sigma_1': 20.0, 'midpoint_1': 0.0,
                 'amp_2': 1.0, 'sigma_2': 10.0, 'midpoint_2': 0.0}

    def evaluate(self, var):
        a1, s1, m1, a2, s2, m2 = self._p('amp_1', 'sigma_1', 'midpoint_1', 'amp_2', 'sigma_2', 'midpoint_2')
        return a1 * np.exp(-((var - m1) ** 2 / (2.0 * s1 ** 2))) - a2 * np.exp(-((var - m2) ** 2 / (2.0 * s2 ** 2)))


# pi / sqrt(3): the logistic with this slope has the variance of a unit normal
_PI_OVER_SQRT3 = np.pi / np.sqrt(3.0)


class Sigmoid(Equation):
    """amp / (1 + exp(-pi/sqrt(3) (radius - var) / sigma)) + offset (equations.py:254-270)."""
    _defaults = {'amp': 1.0, 'radius': 5.0, 'sigma': 1.0, 'offset': 0.0}

    def evaluate(self, var):
        amp, radius, sigma, off = self._p('amp', 'radius', 'sigma', 'offset')
        return amp / (1.0 + np.exp(-_PI_OVER_SQRT3 * (radius - var) / sigma)) + off


class GeneralizedSigmoid(Equation):
    """low + (high - low) / (1 + exp(-pi/sqrt(3) (var - midpoint) / sigma)) (equations.py:273-287)."""
    _defaults = {'low': 0.0, 'high': 1.0, 'midpoint': 1.0, 'sigma': 0.3}

    def evaluate(self, var):
        low, high, mid, sigma = self._p('low', 'high', 'midpoint', 'sigma')
        return low + (high - low) / (1.0 + np.exp(-_PI_OVER_SQRT3 * (var - mid) / sigma))


class Sinusoid(Equation):
    """amp sin(2 pi frequency var) (equations.py:290-303)."""
    _defaults = {'amp': 1.0, 'frequency': 0.01}

    def evaluate(self, var):
        amp, f = self._p('amp', 'frequency')
        return amp * np.sin(2.0 * np.pi * f * var)


class Cosine(Equation):
    """amp cos(2 pi frequency var) (equations.py:306-319)."""
    _defaults = {'amp': 1.0, 'frequency': 0.01}

    def evaluate(self, var):
        amp, f = self._p('amp', 'frequency')
        return amp * np.cos(2.0 * np.pi * f * var)


class Alpha(Equation):
    """alpha beta / (beta - alpha) (exp(-alpha t) - exp(-beta t)) for t = var - onset > 0,
    else 0 (equations.py:322-337)."""
    _defaults = {'onset': 0.5, 'alpha': 13.0, 'beta': 42.0}

    def evaluate(self, var):
        onset, al, be = self._p('onset', 'alpha', 'beta')
        t = var - onset
        with np.errstate(over='ignore', invalid='ignore'):
            v = (al * be) / (be - al) * (np.exp(-al * t) - np.exp(-be * t))
        return np.where(t > 0, v, 0.0 * var)


class PulseTrain(Equation):
    """amp while var > onset and (var - onset) mod T < tau, else 0: pulses of width
    tau every T ms from onset (equations.py:340-364)."""
    _defaults = {'T': 42.0, 'tau': 13.0, 'amp': 1.0, 'onset': 30.0}

    def evaluate(self, var):
        T, tau, amp, onset = self._p('T', 'tau', 'amp', 'onset')
        var = np.asarray(var, dtype=np.float64)
        return np.where((var > onset) & (np.mod(var - onset, T) < tau), amp, 0)


class FirstOrderVolterra(Equation):
    """First Volterra kernel of the Balloon-Windkessel model
    (tvb/datatypes/equations.py:481-519), evaluated in float64:
    G(t) = 1/3 exp(-t / (2 tau_s)) sin(w t) / w, w = sqrt(1/tau_f - 1/(4 tau_s^2)), t in s."""
    _defaults = {'tau_s': 0.8, 'tau_f': 0.4, 'k_1': 5.6, 'V_0': 0.02}

    def evaluate(self, var):
        tau_s, tau_f = self.parameters['tau_s'], self.parameters['tau_f']
        om = np.sqrt(1. / tau_f - 1. / (4. * tau_s ** 2))
        return 1 / 3. * np.exp(-0.5 * (var / tau_s)) * (np.sin(om * var)) / om


EQUATIONS = {c.__name__: c for c in (DiscreteEquation, Linear, Gaussian, DoubleGaussian, Sigmoid,
                                     GeneralizedSigmoid, Sinusoid, Cosine, Alpha, PulseTrain, FirstOrderVolterra)}
