"""Loading the golden fixtures and regenerating the inputs they store as hashes.

Fixtures are written by tests/golden/make_golden.py from runs of the
reference.  Inputs larger than a few hundred KB are stored as SHA-256 digests
together with their recipe (synthetic connectome seed and shape, initial
history seed, noise seed); the functions here rebuild them and check the
digests, so every test runs on exactly the reference's inputs.
"""
import hashlib
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, 'golden')
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, 'tvb-root_b200'))

from oracle import tvb_oracle as O  # noqa: E402

_spec = importlib.util.spec_from_file_location('make_golden', os.path.join(GOLDEN, 'make_golden.py'))
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + '.npz'), allow_pickle=False))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def get(fx, key, regen):
    """fx[key], or regen() checked against the stored digest."""
    if key in fx:
        return fx[key]
    a = regen()
    want = str(fx[key + '_sha256'])
    if sha(a) != want:
        raise AssertionError('regenerated %s does not match the fixture digest' % key)
    return a


def connectome(fx):
    if 'weights' in fx and 'tract_lengths' in fx:
        return fx['weights'], fx['tract_lengths']
    n, dens, lo, hi, seed = fx['conn_recipe']
    w, L = make_golden.synthetic_connectome(int(n), float(dens), float(lo), float(hi), int(seed))
    return get(fx, 'weights', lambda: w), get(fx, 'tract_lengths', lambda: L)


def model_ranges(model):
    info = O.MODEL_INFO[model]
    return [info['ranges'][s] for s in info['svars']]


def initial_history(fx, model, n, seed=None, fp64=False, key='buffer0'):
    """Configured float32 ring (H, ncvar, n) of the reference: uniform initial
    history drawn from RandomState(seed) (the noise stream for stochastic
    runs, the seeded global RNG for deterministic ones), coupling variables
    only."""
    info = O.MODEL_INFO[model]
    H = int(fx['horizon'])

    def regen():
        hist = O.reference_initial_history(int(fx['ic_seed']) if seed is None else seed, model_ranges(model), H, n)
        for sv, (lo, hi) in info['bounds'].items():
            i = info['svars'].index(sv)
            hist[:, i] = np.clip(hist[:, i], lo, hi)
        b = hist[:, list(info['cvar'])]
        return b if fp64 else b.astype(np.float32)
    return get(fx, key, regen)


def reference_noise(fx, model, n_steps, n, seed=42):
    info = O.MODEL_INFO[model]
    return O.reference_noise(seed, model_ranges(model), int(fx['horizon']), n, len(info['svars']), n_steps)
