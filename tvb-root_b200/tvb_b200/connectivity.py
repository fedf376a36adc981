"""Region connectivity: weights, tract lengths and conduction speed
(tvb/datatypes/connectivity.py)."""
import numpy as np

from . import _lib


class Connectivity:
    def __init__(self, weights, tract_lengths, speed=None, region_labels=None, centres=None, orientations=None,
                 cortical=None):
        self.weights = np.asarray(weights, dtype=np.float64)
        self.tract_lengths = np.asarray(tract_lengths, dtype=np.float64)
        if self.weights.ndim != 2 or self.weights.shape[0] != self.weights.shape[1]:
            raise ValueError('weights must be a square matrix')
        if self.tract_lengths.shape != self.weights.shape:
            raise ValueError('tract_lengths must have the shape of weights')
        self.speed = None if speed is None else np.atleast_1d(np.asarray(speed, dtype=np.float64))
        self.region_labels = region_labels
        self.centres = None if centres is None else np.asarray(centres, dtype=np.float64)
        # source positions and unit orientations, and the cortical mask, used by the projection monitors
        self.orientations = None if orientations is None else np.asarray(orientations, dtype=np.float64)
        self.cortical = np.zeros(0, dtype=bool) if cortical is None else np.asarray(cortical, dtype=bool)
        self.delays = None
        self.idelays = None
        self._horizon = None

    @property
    def number_of_regions(self):
        return self.weights.shape[0]

    def configure(self):
        """delays = tract_lengths / speed (connectivity.py:266-275); speed
        defaults to 3.0 like the reference."""
        if self.speed is None:
            self.speed = np.array([3.0])
        self.delays = self.tract_lengths / self.speed
        return self

    def set_idelays(self, dt):
        """idelays = rint(delays / dt) and horizon = max + 1 (connectivity.py:308-326),
        computed by the library's bit-exact host routine."""
        if self.speed.size != 1:
            raise NotImplementedError('a single conduction speed is supported')
        self.idelays, self._horizon = _lib.idelays(self.tract_lengths, float(self.speed[0]), dt)
        self.has_delays = bool(self.idelays.any())
        return self.idelays

    @property
    def horizon(self):
        return self._horizon
