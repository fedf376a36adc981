"""Coupling functions with the reference's parameters (tvb/simulator/coupling.py).

The pre / weighted sum / post of each runs inside the simulation kernel;
``kernel_params`` gives the float32 parameters in the order it reads them.
"""
import numpy as np

from ._traits import HasParams


class Coupling(HasParams):
    def configure(self):
        return self

    def kernel_params(self):
        raise NotImplementedError


class Linear(Coupling):
    """a * gx + b, pre = x_j (coupling.py:170-200)."""
    _defaults = dict(a=0.00390625, b=0.0)

    def kernel_params(self):
        return [float(np.asarray(self.a).reshape(-1)[0]), float(np.asarray(self.b).reshape(-1)[0])]


class Difference(Coupling):
    """a * sum_j w_ij (x_j - x_i) (coupling.py:462-486)."""
    _defaults = dict(a=0.1)

    def kernel_params(self):
        return [float(np.asarray(self.a).reshape(-1)[0])]


class SigmoidalJansenRit(Coupling):
    """a * sum_j w_ij S(x_j0 - x_j1), S(v) = cmin + (cmax - cmin) / (1 + exp(r (midpoint - v)))
    (coupling.py:325-376)."""
    _defaults = dict(cmin=0.0, cmax=2.0 * 0.0025, midpoint=6.0, r=0.56, a=1.0)

    def kernel_params(self):
        return [float(np.asarray(getattr(self, k)).reshape(-1)[0]) for k in ('cmin', 'cmax', 'midpoint', 'r', 'a')]


def _f(v):
    return float(np.asarray(v).reshape(-1)[0])


class Scaling(Coupling):
    """a * gx, pre = x_j (coupling.py:203-224): run as Linear with b = 0."""
    _defaults = dict(a=0.00390625)
    kernel_id = 'Linear'

    def kernel_params(self):
        return [_f(self.a), 0.0]


class Sigmoidal(Coupling):
    """cmin + (cmax - cmin) / (1 + exp(-a ((gx - midpoint) / sigma))), pre = x_j
    (coupling.py:270-322)."""
    _defaults = dict(cmin=-1.0, cmax=1.0, midpoint=0.0, a=1.0, sigma=230.0)

    def kernel_params(self):
        return [_f(getattr(self, k)) for k in ('cmin', 'cmax', 'midpoint', 'a', 'sigma')]


class HyperbolicTangent(Coupling):
    """pre = a (1 + tanh((b x_j - midpoint) / sigma)), post = gx (coupling.py:227-267)."""
    _defaults = dict(a=1.0, b=1.0, midpoint=0.0, sigma=1.0)

    def kernel_params(self):
        return [_f(getattr(self, k)) for k in ('a', 'b', 'midpoint', 'sigma')]


class Kuramoto(Coupling):
    """pre = sin(x_j - x_i), post = a / ncvar * gx (coupling.py:489-508; the
    reference divides by gx.shape[0], the number of coupling variables)."""
    _defaults = dict(a=1.0)

    def kernel_params(self):
        return [_f(self.a)]


COUPLINGS = {cls.__name__: cls for cls in (Linear, Difference, SigmoidalJansenRit, Scaling, Sigmoidal,
                                           HyperbolicTangent, Kuramoto)}
