"""Haemodynamic response kernel of the Bold monitor."""
import numpy as np


class FirstOrderVolterra:
    """First Volterra kernel of the Balloon-Windkessel model
    (tvb/datatypes/equations.py:481-519), evaluated in float64:
    G(t) = 1/3 exp(-t / (2 tau_s)) sin(w t) / w, w = sqrt(1/tau_f - 1/(4 tau_s^2)), t in s."""

    def __init__(self, parameters=None):
        self.parameters = {'tau_s': 0.8, 'tau_f': 0.4, 'k_1': 5.6, 'V_0': 0.02}
        if parameters:
            self.parameters.update(parameters)

    def evaluate(self, var):
        tau_s, tau_f = self.parameters['tau_s'], self.parameters['tau_f']
        om = np.sqrt(1. / tau_f - 1. / (4. * tau_s ** 2))
        return 1 / 3. * np.exp(-0.5 * (var / tau_s)) * (np.sin(om * var)) / om
