"""Integration schemes (tvb/simulator/integrators.py); the steps themselves run
in the simulation kernel."""
from .noise import Additive


class Integrator:
    stochastic = False

    def __init__(self, dt=0.01220703125, **kwargs):
        self.dt = float(dt)
        if kwargs:
            raise TypeError('%s has no parameters %s' % (type(self).__name__, sorted(kwargs)))

    def configure(self):
        return self


class IntegratorStochastic(Integrator):
    stochastic = True

    def __init__(self, dt=0.01220703125, noise=None):
        super().__init__(dt)
        self.noise = noise if noise is not None else Additive()

    def configure(self):
        self.noise.configure()
        return self


class HeunDeterministic(Integrator):
    """integrators.py:286-318."""


class HeunStochastic(IntegratorStochastic):
    """integrators.py:321-362; the same noise enters predictor and corrector."""


class EulerDeterministic(Integrator):
    """integrators.py:365-391."""


class EulerStochastic(IntegratorStochastic):
    """integrators.py:394-426."""


class Identity(Integrator):
    """integrators.py:483-507: x_{n+1} = f(x_n)."""


class RungeKutta4thOrderDeterministic(Integrator):
    """integrators.py:429-480: the classical four-stage Runge-Kutta step, the
    coupling held fixed over the step, bounds applied to each stage."""


INTEGRATORS = {cls.__name__: cls for cls in (HeunDeterministic, HeunStochastic, EulerDeterministic,
                                             EulerStochastic, Identity, RungeKutta4thOrderDeterministic)}
