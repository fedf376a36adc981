"""Neural mass models with the reference's parameter names, defaults, state
variables, coupling variables, ranges and observables.

The derivative functions run on the device (csrc/tvbk_models.cuh); these
classes carry the parameters, the initial-condition draw and the host-side
observer.  Parameter order of ``kernel_params`` is the order the kernel reads.
"""
import numpy as np

from ._traits import HasParams


class Model(HasParams):
    """Base of the device models (tvb/simulator/models/base.py:39-262)."""
    state_variables = ()
    cvar = None
    stvar = None  # state variables a stimulus drives; None: the coupling variables (models/base.py:91-92)
    state_variable_range = {}
    state_variable_boundaries = None
    variables_of_interest = ()
    observable_choices = ()
    kernel_param_names = ()
    number_of_modes = 1
    _defaults = {}

    @property
    def nvar(self):
        return len(self.state_variables)

    @property
    def nintvar(self):
        return len(self.state_variables)

    def configure(self):
        for name in self.variables_of_interest:
            if name not in self.observable_choices:
                raise ValueError('%s is not an observable of %s (choices %s)'
                                 % (name, type(self).__name__, self.observable_choices))
        if self.stvar is None:
            self.stvar = np.array(self.cvar, dtype=np.int32).copy()
        return self

    def initial(self, dt, history_shape, rng=np.random):
        """Uniform initial conditions in the state-variable ranges, drawn per
        state variable in order (tvb/simulator/models/base.py:138-149)."""
        nt, nvar, nnode, nmode = history_shape
        ic = np.empty(history_shape)
        for i in range(nvar):
            lo, hi = self.state_variable_range[self.state_variables[i]]
            ic[:, i] = rng.uniform(low=lo, high=hi, size=(nt, nnode, nmode))
        return ic

    def initial_for_simulator(self, integrator, shape):
        """RNG choice of tvb/simulator/models/base.py:151-155: the noise stream
        of a stochastic integrator, else the global numpy RNG."""
        noise = getattr(integrator, 'noise', None)
        rng = noise.random_stream if noise is not None else np.random
        return self.initial(integrator.dt, shape, rng)

    def voi_codes(self, names=None):
        names = self.variables_of_interest if names is None else names
        return [self.observable_choices.index(v) for v in names]

    def observe(self, state):
        """Observed variables of a (nvar, n, ...) state (models/base.py:56-71)."""
        env = dict(zip(self.state_variables, state))
        return np.array([eval(v, {}, env) for v in self.variables_of_interest])

    def kernel_params(self, n):
        """(nparam, n) float32 parameters, spatialised per region."""
        out = np.empty((len(self.kernel_param_names), n), dtype=np.float32)
        for k, name in enumerate(self.kernel_param_names):
            v = np.asarray(getattr(self, name), dtype=np.float64).reshape(-1)
            if v.size not in (1, n):
                raise ValueError('parameter %s has %d values for %d regions' % (name, v.size, n))
            out[k] = v if v.size == n else v[0]
        return out

    def bound(self, state):
        """Clamp to state_variable_boundaries in place (integrators.py:181-192)."""
        if not self.state_variable_boundaries:
            return state
        for sv, (lo, hi) in self.state_variable_boundaries.items():
            i = self.state_variables.index(sv)
            state[i] = np.clip(state[i], lo, hi)
        return state


class Generic2dOscillator(Model):
    """tvb/simulator/models/oscillator.py:39-395."""
    _defaults = dict(tau=1.0, I=0.0, a=-2.0, b=-10.0, c=0.0, d=0.02, e=3.0, f=1.0, g=0.0,
                     alpha=1.0, beta=1.0, gamma=1.0)
    state_variables = ('V', 'W')
    cvar = np.array([0], dtype=np.int32)
    state_variable_range = {'V': (-2.0, 4.0), 'W': (-6.0, 6.0)}
    observable_choices = ('V', 'W', 'V + W', 'V - W')
    variables_of_interest = ('V',)
    kernel_param_names = ('tau', 'I', 'a', 'b', 'c', 'd', 'e', 'f', 'g', 'alpha', 'beta', 'gamma')


class JansenRit(Model):
    """tvb/simulator/models/jansen_rit.py:38-289."""
    _defaults = dict(A=3.25, B=22.0, a=0.1, b=0.05, v0=5.52, nu_max=0.0025, r=0.56, J=135.0,
                     a_1=1.0, a_2=0.8, a_3=0.25, a_4=0.25, p_min=0.12, p_max=0.32, mu=0.22)
    state_variables = ('y0', 'y1', 'y2', 'y3', 'y4', 'y5')
    cvar = np.array([1, 2], dtype=np.int32)
    state_variable_range = {'y0': (-1.0, 1.0), 'y1': (-500.0, 500.0), 'y2': (-50.0, 50.0),
                            'y3': (-6.0, 6.0), 'y4': (-20.0, 20.0), 'y5': (-500.0, 500.0)}
    observable_choices = ('y0', 'y1', 'y2', 'y3', 'y4', 'y5')
    variables_of_interest = ('y0', 'y1', 'y2', 'y3')
    kernel_param_names = ('A', 'B', 'a', 'b', 'v0', 'nu_max', 'r', 'J', 'a_1', 'a_2', 'a_3', 'a_4', 'mu')


class ReducedWongWang(Model):
    """tvb/simulator/models/wong_wang.py:36-181."""
    _defaults = dict(a=0.270, b=0.108, d=154.0, gamma=0.641, tau_s=100.0, w=0.6, J_N=0.2609,
                     I_o=0.33, sigma_noise=1e-9)
    state_variables = ('S',)
    cvar = np.array([0], dtype=np.int32)
    state_variable_range = {'S': (0.0, 1.0)}
    state_variable_boundaries = {'S': (0.0, 1.0)}
    observable_choices = ('S',)
    variables_of_interest = ('S',)
    kernel_param_names = ('a', 'b', 'd', 'gamma', 'tau_s', 'w', 'J_N', 'I_o')


class Epileptor(Model):
    """tvb/simulator/models/epileptor.py:36-356."""
    _defaults = dict(a=1.0, b=3.0, c=1.0, d=5.0, r=0.00035, s=4.0, x0=-1.6, Iext=3.1, slope=0.0,
                     Iext2=0.45, tau=10.0, aa=6.0, bb=2.0, Kvf=0.0, Kf=0.0, Ks=0.0, tt=1.0,
                     modification=0.0)
    state_variables = ('x1', 'y1', 'z', 'x2', 'y2', 'g')
    cvar = np.array([0, 3], dtype=np.int32)
    state_variable_range = {'x1': (-2.0, 1.0), 'y1': (-20.0, 2.0), 'z': (2.0, 5.0),
                            'x2': (-2.0, 0.0), 'y2': (0.0, 2.0), 'g': (-1.0, 1.0)}
    observable_choices = ('x1', 'y1', 'z', 'x2', 'y2', 'g', 'x2 - x1')
    variables_of_interest = ('x2 - x1', 'z')
    kernel_param_names = ('a', 'b', 'c', 'd', 'r', 'x0', 'Iext', 'slope', 'Iext2', 'tau', 'aa', 'bb',
                          'Kvf', 'Kf', 'Ks', 'tt', 'modification')


class Sum(Model):
    """dx = x + c, the model of the reference's exact-propagation test
    (tvb/tests/library/simulator/history_test.py); use with Identity."""
    _defaults = {}
    state_variables = ('x',)
    cvar = np.array([0], dtype=np.int32)
    state_variable_range = {'x': (0.0, 100.0)}
    observable_choices = ('x',)
    variables_of_interest = ('x',)
    kernel_param_names = ()

    def kernel_params(self, n):
        return np.zeros((1, n), dtype=np.float32)


MODELS = {cls.__name__: cls for cls in (Generic2dOscillator, JansenRit, ReducedWongWang, Epileptor, Sum)}
