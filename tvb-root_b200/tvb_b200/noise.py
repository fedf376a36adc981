"""Additive white noise (tvb/simulator/noise.py:46-232).

``random_stream`` is a numpy RandomState seeded with ``noise_seed`` as in the
reference; it draws the initial history of stochastic simulations and, with
``Simulator(..., noise_source='reference')``, the integration noise itself
(the reference's exact stream, fed to the device).  Otherwise the device
draws from its counter-based Philox stream keyed by (noise_seed, instance).
"""
import numpy as np


class Additive:
    def __init__(self, nsig=(1.0,), noise_seed=42, random_stream=None, ntau=0.0):
        if ntau != 0.0:
            raise NotImplementedError('coloured noise (ntau > 0) is not supported on the device path')
        self.nsig = np.atleast_1d(np.asarray(nsig, dtype=np.float64)).copy()
        self.noise_seed = int(noise_seed)
        self.ntau = 0.0
        self.random_stream = random_stream if random_stream is not None else np.random.RandomState(self.noise_seed)
        self.dt = None

    def configure(self):
        return self

    def configure_white(self, dt, shape=None):
        self.dt = dt

    def reset_random_stream(self):
        self.random_stream = np.random.RandomState(self.noise_seed)

    def gfun(self, state_variables=None):
        """sqrt(2 nsig) (noise.py:223-232)."""
        return np.sqrt(2.0 * self.nsig)
