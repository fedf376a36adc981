"""Minimal declarative-parameter base mirroring how the reference's traited
components are constructed: keyword arguments named after the reference's
attributes, numeric parameters stored as float64 arrays (NArray semantics,
tvb/basic/neotraits/_attr.py), unknown names rejected."""
import numpy as np


class HasParams:
    _defaults = {}
    _extra_attrs = ('variables_of_interest', 'state_variable_range', 'state_variable_boundaries')

    def __init__(self, **kwargs):
        for k, v in self._defaults.items():
            setattr(self, k, np.array([v], dtype=np.float64))
        for k, v in kwargs.items():
            if k in self._defaults:
                setattr(self, k, np.atleast_1d(np.asarray(v, dtype=np.float64)).copy())
            elif k in self._extra_attrs or hasattr(type(self), k):
                if k == 'variables_of_interest':
                    v = tuple(v)
                setattr(self, k, v)
            else:
                raise TypeError('%s has no parameter %r' % (type(self).__name__, k))

    @property
    def parameter_names(self):
        return list(self._defaults)

    def __repr__(self):
        parts = ['%s=%s' % (k, np.asarray(getattr(self, k)).tolist()) for k in self._defaults]
        return '%s(%s)' % (type(self).__name__, ', '.join(parts))
