"""Region stimuli (tvb/datatypes/patterns.py:41-186): a temporal equation
evaluated on the simulation's time grid times a spatial pattern over the
regions.  The product is separable, so the device reads one value per step
and one weight per region instead of a (steps, regions) array.

    stim = StimuliRegion(temporal=PulseTrain({'onset': 50.0}), connectivity=conn,
                         weight=w)                      # w: (n_regions,)
    sim = Simulator(..., stimulus=stim).configure()
"""
import numpy as np

from .equations import DiscreteEquation, PulseTrain


class StimuliRegion:
    """Temporal profile of a stimulus and the scaling weight of each region.

    ``configure_space()`` sets ``spatial_pattern`` (n, 1) to the spatial
    equation of the weights summed over its trailing axis (the weights
    themselves for the default DiscreteEquation); ``configure_time(time)``
    sets ``temporal_pattern`` (1, T); ``stim(k)`` is the (n, 1) stimulus of
    time index k.
    """

    def __init__(self, temporal=None, connectivity=None, weight=None, spatial=None):
        self.temporal = temporal if temporal is not None else PulseTrain()
        self.spatial = spatial if spatial is not None else DiscreteEquation()
        self.connectivity = connectivity
        self.weight = weight
        self.space = None
        self.time = None
        self._spatial_pattern = None
        self._temporal_pattern = None

    @staticmethod
    def get_default_weights(number_of_regions):
        return np.array([0.0] * number_of_regions)

    @property
    def weight_array(self):
        return np.array(self.weight)[:, np.newaxis]

    @property
    def spatial_pattern(self):
        return self._spatial_pattern

    @property
    def temporal_pattern(self):
        return self._temporal_pattern

    def configure(self):
        return self

    def configure_space(self, region_mapping=None):
        if region_mapping is not None:
            raise NotImplementedError('surface stimuli are not supported on the device path')
        self.space = self.weight_array
        self._spatial_pattern = np.sum(self.spatial.evaluate(self.space), axis=1)[:, np.newaxis]

    def configure_time(self, time):
        self.time = time
        self._temporal_pattern = np.reshape(self.temporal.evaluate(self.time), (1, -1))

    def __call__(self, temporal_indices=None, spatial_indices=None):
        sp = self._spatial_pattern if spatial_indices is None else self._spatial_pattern[spatial_indices, 0]
        tp = self._temporal_pattern if temporal_indices is None else self._temporal_pattern[0, temporal_indices]
        return sp * tp
