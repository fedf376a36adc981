"""Sensors, lead-field (projection) matrices and region mappings for the
EEG / MEG / iEEG monitors, with the reference's attribute names
(tvb/datatypes/sensors.py, projections.py, region_mapping.py).  The monitors
read these by attribute, so the reference's own objects work as well."""
import numpy as np


class Sensors:
    """labels (S,), locations (S, 3), optional usable (S,) bool mask and
    orientations (S, 3)."""

    def __init__(self, labels, locations, usable=None, orientations=None):
        self.labels = np.asarray(labels, dtype='U128')
        self.locations = np.asarray(locations, dtype=np.float64)
        self.usable = None if usable is None else np.asarray(usable, dtype=bool)
        self.orientations = None if orientations is None else np.asarray(orientations, dtype=np.float64)
        self.number_of_sensors = int(self.labels.shape[0])

    def configure(self):
        self.number_of_sensors = int(self.labels.shape[0])
        return self


class SensorsEEG(Sensors):
    pass


class SensorsMEG(Sensors):
    pass


class SensorsInternal(Sensors):
    pass


class ProjectionMatrix:
    """projection_data (S, sources): the lead field from sources (surface
    vertices, or regions) to sensors."""

    def __init__(self, projection_data, sensors=None, sources=None):
        self.projection_data = np.asarray(projection_data, dtype=np.float64)
        self.sensors = sensors
        self.sources = sources


class ProjectionSurfaceEEG(ProjectionMatrix):
    pass


class ProjectionSurfaceMEG(ProjectionMatrix):
    pass


class ProjectionSurfaceSEEG(ProjectionMatrix):
    pass


class RegionMapping:
    """array_data (vertices,): the region of each source vertex."""

    def __init__(self, array_data, connectivity=None, surface=None):
        self.array_data = np.asarray(array_data, dtype=np.int64)
        self.connectivity = connectivity
        self.surface = surface
