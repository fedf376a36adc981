"""CPU oracle for the TVB region simulation loop -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  It is a plain numpy restatement of the reference's classic numpy path
(the-virtual-brain/tvb-root, ``tvb_library/tvb/simulator``); each function
cites the reference file:line it follows.  Precision follows the reference:
the history ring and the connectome weights are float32 in the stock path
(``tvb/simulator/history.py:49-51,166-172``, coerced by
``tvb/simulator/descriptors.py:109-123``), everything else is float64;
``history_dtype=np.float64`` gives the all-FP64 variant.

Pinning: ``tests/test_oracle.py`` checks this restatement against golden
vectors produced by running the reference itself (``tests/golden/*.npz``,
generated by ``tests/golden/make_golden.py``) and against the reference's own
known-answer tests (exact delayed propagation, Difference coupling, model
fixed points, idelays at rounding ties).

The counter-based noise stream used by the device kernels
(Philox4x32-10, Salmon et al., SC'11, plus a Box-Muller transform) is also
restated here so that runs driven by device noise can be replayed on the CPU.
"""
import math

import numpy as np

# ----------------------------------------------------------------------------
# connectivity / history set-up


def conduction_delays(tract_lengths, speed):
    """``delays = tract_lengths / speed`` (tvb/datatypes/connectivity.py:275)."""
    return np.asarray(tract_lengths, dtype=np.float64) / np.asarray(speed, dtype=np.float64)


def integer_delays(tract_lengths, speed, dt):
    """``idelays = rint(delays / dt).astype(int32)`` and ``horizon = max + 1``
    over the full matrix, zero-weight pairs included
    (tvb/datatypes/connectivity.py:321-323)."""
    idelays = np.rint(conduction_delays(tract_lengths, speed) / dt).astype(np.int32)
    return idelays, int(idelays.max()) + 1


def sparse_layout(weights, idelays, hist_dtype=np.float32):
    """Row-major non-zero layout of SparseHistory (tvb/simulator/history.py:221-244)
    and the reduceat row starts of SparseCoupling._lri (tvb/simulator/coupling.py:140-147)."""
    weights = np.asarray(weights)
    mask = weights != 0.0
    row, col = np.argwhere(mask).T
    w = weights[mask].astype(hist_dtype)
    d = idelays.astype(np.float32)[mask].astype(np.int32)
    lri, = np.argwhere(np.diff(np.r_[-1, row])).T
    nzr = np.unique(row)
    return dict(mask=mask, row=row, col=col, w=w, d=d, lri=lri, nzr=nzr)


# ----------------------------------------------------------------------------
# models: derivative functions in the order of the numba gufuncs


MODEL_INFO = {
    # name: (state variables, cvar, state_variable_range order, VOI choices, default VOIs, boundaries)
    'Generic2dOscillator': dict(
        svars=('V', 'W'), cvar=(0,),
        ranges={'V': (-2.0, 4.0), 'W': (-6.0, 6.0)},
        choices=('V', 'W', 'V + W', 'V - W'), voi=('V',), bounds={}),
    'JansenRit': dict(
        svars=('y0', 'y1', 'y2', 'y3', 'y4', 'y5'), cvar=(1, 2),
        ranges={'y0': (-1.0, 1.0), 'y1': (-500.0, 500.0), 'y2': (-50.0, 50.0),
                'y3': (-6.0, 6.0), 'y4': (-20.0, 20.0), 'y5': (-500.0, 500.0)},
        choices=('y0', 'y1', 'y2', 'y3', 'y4', 'y5'), voi=('y0', 'y1', 'y2', 'y3'), bounds={}),
    'ReducedWongWang': dict(
        svars=('S',), cvar=(0,), ranges={'S': (0.0, 1.0)},
        choices=('S',), voi=('S',), bounds={'S': (0.0, 1.0)}),
    'Epileptor': dict(
        svars=('x1', 'y1', 'z', 'x2', 'y2', 'g'), cvar=(0, 3),
        ranges={'x1': (-2.0, 1.0), 'y1': (-20.0, 2.0), 'z': (2.0, 5.0),
                'x2': (-2.0, 0.0), 'y2': (0.0, 2.0), 'g': (-1.0, 1.0)},
        choices=('x1', 'y1', 'z', 'x2', 'y2', 'g', 'x2 - x1'), voi=('x2 - x1', 'z'), bounds={}),
}

MODEL_DEFAULTS = {
    # tvb/simulator/models/oscillator.py:225-305
    'Generic2dOscillator': dict(tau=1.0, I=0.0, a=-2.0, b=-10.0, c=0.0, d=0.02, e=3.0, f=1.0,
                                g=0.0, alpha=1.0, beta=1.0, gamma=1.0),
    # tvb/simulator/models/jansen_rit.py:74-170
    'JansenRit': dict(A=3.25, B=22.0, a=0.1, b=0.05, v0=5.52, nu_max=0.0025, r=0.56, J=135.0,
                      a_1=1.0, a_2=0.8, a_3=0.25, a_4=0.25, p_min=0.12, p_max=0.32, mu=0.22),
    # tvb/simulator/models/wong_wang.py:62-117
    'ReducedWongWang': dict(a=0.270, b=0.108, d=154.0, gamma=0.641, tau_s=100.0, w=0.6,
                            J_N=0.2609, I_o=0.33, sigma_noise=1e-9),
    # tvb/simulator/models/epileptor.py:76-178
    'Epileptor': dict(a=1.0, b=3.0, c=1.0, d=5.0, r=0.00035, s=4.0, x0=-1.6, Iext=3.1,
                      slope=0.0, Iext2=0.45, tau=10.0, aa=6.0, bb=2.0, Kvf=0.0, Kf=0.0,
                      Ks=0.0, tt=1.0, modification=0.0),
}


def dfun_g2d(X, c, p):
    """tvb/simulator/models/oscillator.py:387-395 (_numba_dfun_g2d)."""
    V, W = X[0], X[1]
    V2 = V * V
    dV = p['d'] * p['tau'] * (p['alpha'] * W - p['f'] * V2 * V + p['e'] * V2 + p['g'] * V
                              + p['gamma'] * p['I'] + p['gamma'] * c[0] + 0.0)
    dW = p['d'] * (p['a'] + p['b'] * V + p['c'] * V2 - p['beta'] * W) / p['tau']
    return np.array([dV, dW])


def dfun_jr(y, c, p):
    """tvb/simulator/models/jansen_rit.py:274-289 (_numba_dfun_jr)."""
    nu, r, v0 = p['nu_max'], p['r'], p['v0']
    s12 = 2.0 * nu / (1.0 + np.exp(r * (v0 - (y[1] - y[2]))))
    s01 = 2.0 * nu / (1.0 + np.exp(r * (v0 - (p['a_1'] * p['J'] * y[0]))))
    s03 = 2.0 * nu / (1.0 + np.exp(r * (v0 - (p['a_3'] * p['J'] * y[0]))))
    a, b, A, B, J = p['a'], p['b'], p['A'], p['B'], p['J']
    return np.array([
        y[3], y[4], y[5],
        A * a * s12 - 2.0 * a * y[3] - a ** 2 * y[0],
        A * a * (p['mu'] + p['a_2'] * J * s01 + c[0] + 0.0) - 2.0 * a * y[4] - a ** 2 * y[1],
        B * b * (p['a_4'] * J * s03) - 2.0 * b * y[5] - b ** 2 * y[2],
    ])


def dfun_rww(X, c, p):
    """tvb/simulator/models/wong_wang.py:36-42 (_numba_dfun)."""
    S = X[0]
    x = p['w'] * p['J_N'] * S + p['I_o'] + p['J_N'] * c[0]
    h = (p['a'] * x - p['b']) / (1 - np.exp(-p['d'] * (p['a'] * x - p['b'])))
    return np.array([-(S / p['tau_s']) + (1.0 - S) * h * p['gamma']])


def dfun_epileptor(y, c, p):
    """tvb/simulator/models/epileptor.py:36-71 (_numba_dfun)."""
    cp1, cp2 = c[0], c[1]
    tt = p['tt']
    f1 = np.where(y[0] < 0.0, -p['a'] * y[0] ** 2 + p['b'] * y[0],
                  p['slope'] - y[3] + 0.6 * (y[2] - 4.0) ** 2)
    d0 = tt * (y[1] - y[2] + p['Iext'] + p['Kvf'] * cp1 + f1 * y[0])
    d1 = tt * (p['c'] - p['d'] * y[0] ** 2 - y[1])
    z7 = np.where(y[2] < 0.0, -0.1 * y[2] ** 7, 0.0)
    if np.any(np.asarray(p['modification']) != 0):
        h = p['x0'] + 3 / (1 + np.exp(-(y[0] + 0.5) / 0.1))
    else:
        h = 4 * (y[0] - p['x0']) + z7
    d2 = tt * (p['r'] * (h - y[2] + p['Ks'] * cp1))
    d3 = tt * (-y[4] + y[3] - y[3] ** 3 + p['Iext2'] + p['bb'] * y[5] - 0.3 * (y[2] - 3.5) + p['Kf'] * cp2)
    f2 = np.where(y[3] < -0.25, 0.0, p['aa'] * (y[3] + 0.25))
    d4 = tt * ((-y[4] + f2) / p['tau'])
    d5 = tt * (-0.01 * (y[5] - 0.1 * y[0]))
    return np.array([d0, d1, d2, d3, d4, d5])


def dfun_sum(X, c, p):
    """Toy model of the reference's exact-propagation test: dx = x + c."""
    return X + c


DFUNS = {'Generic2dOscillator': dfun_g2d, 'JansenRit': dfun_jr,
         'ReducedWongWang': dfun_rww, 'Epileptor': dfun_epileptor, 'Sum': dfun_sum}


def observe(model, X, vois):
    """Model.observe built from the VOI expressions (tvb/simulator/models/base.py:56-71)."""
    info = MODEL_INFO[model]
    env = dict(zip(info['svars'], X))
    return np.array([eval(v, {}, env) for v in vois])


# ----------------------------------------------------------------------------
# coupling


def coupling_sparse(kind, buf, step, lay, params):
    """SparseHistory.query_sparse + SparseCoupling.__call__
    (tvb/simulator/history.py:251-256; tvb/simulator/coupling.py:149-167) with
    Linear.post (coupling.py:196-197) or Difference.pre/post (coupling.py:482-486)."""
    params = {k: np.atleast_1d(np.asarray(v, dtype=np.float64)) for k, v in params.items()}
    H = buf.shape[0]
    t_idx = (step - 1 - lay['d'] + H) % H
    x_j = buf[t_idx[None, :], np.arange(buf.shape[1])[:, None], lay['col'][None, :]]
    current = buf[(step - 1) % H]
    x_i = current[:, lay['row']]
    if kind in ('Linear', 'PassThrough', 'Scaling', 'Sigmoidal'):
        pre = x_j
    elif kind == 'Difference':
        pre = x_j - x_i
    elif kind == 'HyperbolicTangent':                          # coupling.py:259-260
        pre = params['a'] * (1 + np.tanh((params['b'] * x_j - params['midpoint']) / params['sigma']))
    elif kind == 'Kuramoto':                                   # coupling.py:504-505
        pre = np.sin(x_j - x_i)
    else:
        raise NotImplementedError(kind)
    out = np.zeros(current.shape, dtype=pre.dtype)
    out[:, lay['nzr']] = np.add.reduceat(lay['w'][None, :] * pre, lay['lri'], axis=1)
    if kind == 'Linear':
        return params['a'] * out + params['b']
    if kind in ('Difference', 'Scaling'):                      # coupling.py:220-221,485-486
        return params['a'] * out
    if kind == 'Sigmoidal':                                    # coupling.py:316-317
        return params['cmin'] + ((params['cmax'] - params['cmin']) /
                                 (1.0 + np.exp(-params['a'] * ((out - params['midpoint']) / params['sigma']))))
    if kind == 'Kuramoto':                                     # coupling.py:507-508 (a / gx.shape[0])
        return params['a'] / out.shape[0] * out
    return out


def coupling_sigmoidal_jr(buf, step, idelays, weights_h, params):
    """Dense Coupling.__call__ with SigmoidalJansenRit.pre/post
    (tvb/simulator/coupling.py:118-124,370-376; the dense delayed state of
    tvb/simulator/history.py:246-249 is zero where the weight is zero)."""
    H, ncv, n = buf.shape
    mask = weights_h != 0
    t_idx = (step - 1 - idelays + H) % H                      # (to, from)
    cols = np.broadcast_to(np.arange(n)[None, :], (n, n))
    xj = np.zeros((n, ncv, n), dtype=buf.dtype)               # (to, cvar, from)
    for cv in range(ncv):
        xj[:, cv, :][mask] = buf[t_idx[mask], cv, cols[mask]]
    diff = xj[:, 0] - xj[:, 1]
    pre = params['cmin'] + (params['cmax'] - params['cmin']) / (
        1.0 + np.exp(params['r'] * (params['midpoint'] - diff)))
    gx = (weights_h * pre).sum(axis=1)                        # (to,)
    return (params['a'] * gx)[None, :]


# ----------------------------------------------------------------------------
# noise


def reference_noise(seed, ic_ranges, horizon, n, nintvar, n_steps):
    """Standard normals the reference draws for integration noise, in order:
    the initial history is drawn first from the same RandomState
    (tvb/simulator/models/base.py:138-155), then one normal of shape
    (nintvar, n, 1) per step (tvb/simulator/noise.py:195-198).  Returns z of
    shape (n_steps, nintvar, n); the reference noise is sqrt(dt) * z."""
    rs = np.random.RandomState(seed)
    for lo, hi in ic_ranges:
        rs.uniform(low=lo, high=hi, size=(horizon, n, 1))
    return rs.normal(size=(n_steps, nintvar, n))


def reference_initial_history(seed_or_rs, ic_ranges, horizon, n):
    """Uniform initial history in the state-variable ranges (tvb/simulator/models/base.py:138-149)."""
    rs = seed_or_rs if isinstance(seed_or_rs, np.random.RandomState) else np.random.RandomState(seed_or_rs)
    hist = np.empty((horizon, len(ic_ranges), n))
    for i, (lo, hi) in enumerate(ic_ranges):
        hist[:, i] = rs.uniform(low=lo, high=hi, size=(horizon, n, 1))[..., 0]
    return hist


PHILOX_M0, PHILOX_M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
PHILOX_W0, PHILOX_W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32 with 10 rounds (Salmon, Moraes, Dror, Shaw, SC'11), vectorised over numpy uint32 arrays."""
    c = [np.asarray(x, dtype=np.uint32) for x in (c0, c1, c2, c3)]
    c = np.broadcast_arrays(*c)
    c = [x.astype(np.uint32) for x in c]
    k0 = np.broadcast_to(np.asarray(k0, dtype=np.uint32), c[0].shape).astype(np.uint32)
    k1 = np.broadcast_to(np.asarray(k1, dtype=np.uint32), c[0].shape).astype(np.uint32)
    mask = np.uint64(0xFFFFFFFF)
    with np.errstate(over='ignore'):
        for rnd in range(10):
            p0 = PHILOX_M0 * c[0].astype(np.uint64)
            p1 = PHILOX_M1 * c[2].astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & mask).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & mask).astype(np.uint32)
            c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
            if rnd < 9:
                k0 = (k0 + PHILOX_W0).astype(np.uint32)
                k1 = (k1 + PHILOX_W1).astype(np.uint32)
    return c


def uniform_open(x):
    """uint32 -> float32 uniform in (0, 1): ((x >> 9) + 0.5) * 2^-23, exact in float32."""
    return ((np.asarray(x, dtype=np.uint32) >> np.uint32(9)).astype(np.float32) + np.float32(0.5)) \
        * np.float32(2.0 ** -23)


def box_muller(u1, u2):
    """Box-Muller pair from two (0,1) uniforms: r = sqrt(-2 ln u1), (r cos 2 pi u2, r sin 2 pi u2)."""
    u1 = np.asarray(u1, dtype=np.float64)
    u2 = np.asarray(u2, dtype=np.float64)
    r = np.sqrt(-2.0 * np.log(u1))
    return r * np.cos(2.0 * np.pi * u2), r * np.sin(2.0 * np.pi * u2)


def philox_normals(seed, stream, steps, nintvar, n):
    """Standard normals of the device noise stream for the given absolute steps:
    block = Philox(key=(seed, stream), counter=((step - 1) >> 2, node, svar, 0));
    the pairs (x0, x1) and (x2, x3) give the normals of steps 4k+1..4k+2 and
    4k+3..4k+4.
    Returns (len(steps), nintvar, n) float64."""
    steps = np.asarray(steps, dtype=np.int64)
    blk = ((steps - 1) >> 2).astype(np.uint32)[:, None, None]
    node = np.arange(n, dtype=np.uint32)[None, None, :]
    sv = np.arange(nintvar, dtype=np.uint32)[None, :, None]
    x = philox4x32_10(blk, node, sv, np.uint32(0), np.uint32(seed & 0xFFFFFFFF), np.uint32(stream & 0xFFFFFFFF))
    za, zb = box_muller(uniform_open(x[0]), uniform_open(x[1]))
    zc, zd = box_muller(uniform_open(x[2]), uniform_open(x[3]))
    sel = ((steps - 1) & 3)[:, None, None]
    return np.where(sel == 0, za, np.where(sel == 1, zb, np.where(sel == 2, zc, zd)))


# ----------------------------------------------------------------------------
# Bold haemodynamic response


def first_order_volterra(t, tau_s=0.8, tau_f=0.4):
    """FirstOrderVolterra kernel (tvb/datatypes/equations.py:481-519), t in seconds."""
    om = np.sqrt(1. / tau_f - 1. / (4. * tau_s ** 2))
    return 1 / 3. * np.exp(-0.5 * (t / tau_s)) * (np.sin(om * t)) / om


def bold_hrf(hrf_length=20000.0):
    """Bold.compute_hrf (tvb/simulator/monitors.py:903-929): 4 ms stock samples,
    kernel reversed in time."""
    rate = 2.0 ** -2
    steps = int(np.ceil(rate * hrf_length))
    tmax = hrf_length / 1000.0
    t = np.arange(0.0, tmax, tmax / steps)
    return first_order_volterra(t)[::-1].copy(), steps


def iround(x):
    """ReferenceBackend.iround (tvb/simulator/backend/ref.py:103-121)."""
    y = round(x) - .5
    return int(y) + (y > 0)


# ----------------------------------------------------------------------------
# the loop


class Monitor:
    """kind, period, voi; SpatialAverage: spatial_mask; Projection (EEG / MEG /
    iEEG): gain (sensors, n), obs_z (one (sensors, nvoi) standard-normal draw
    per sample, or None) and ref_vec (sensors,) for the EEG reference."""

    def __init__(self, kind, period=None, voi=None, spatial_mask=None, gain=None, obs_z=None, ref_vec=None):
        self.kind, self.period, self.voi, self.spatial_mask = kind, period, voi, spatial_mask
        self.gain, self.obs_z, self.ref_vec = gain, obs_z, ref_vec


def simulate(model, model_params, weights, tract_lengths, speed, dt, coupling, coupling_params,
             integrator, n_steps, monitors, buffer0, state0, step0=0, nsig=None, noise_z=None,
             history_dtype=np.float32, voi=None, bounds=None, stimulus=None):
    """Run the region simulation loop of Simulator.__call__ (tvb/simulator/simulator.py:322-366).

    buffer0: (H, ncvar, n) initial history ring as configured by the reference
    (tvb/simulator/history.py:73-158); state0: (nsv, n) float64 current state;
    step0: current_step.  noise_z: (n_steps, nintvar, n) standard normals
    (the noise of step k is sqrt(dt) * noise_z[k]).  stimulus: (temporal,
    weight, stvar) -- step k of the run adds weight * temporal[k] to the state
    variables stvar through the scheme's stimulus term (simulator.py:290-306,
    patterns.py:116-134).  Returns a list, one entry per monitor, of
    (times, data[T, nvoi, n]).
    """
    info = MODEL_INFO.get(model)
    p = dict(MODEL_DEFAULTS.get(model, {}))
    p.update(model_params or {})
    p = {k: (np.asarray(v, dtype=np.float64) if np.ndim(v) == 0 else np.asarray(v, dtype=np.float64))
         for k, v in p.items()}
    dfun = DFUNS[model]
    cvar = np.array(info['cvar'] if info else (0,))
    if voi is None:
        voi = info['voi'] if info else ('x',)
    if bounds is None:
        bounds = info['bounds'] if info else {}
    svars = info['svars'] if info else ('x',)
    bidx = [(svars.index(k), lo, hi) for k, (lo, hi) in bounds.items()]

    idelays, H = integer_delays(tract_lengths, speed, dt)
    buf = np.array(buffer0, dtype=history_dtype).copy()
    assert buf.shape[0] == H
    X = np.array(state0, dtype=np.float64).copy()
    whist = np.asarray(weights).astype(history_dtype)
    lay = sparse_layout(weights, idelays, history_dtype)
    cp = {k: np.asarray(v, dtype=np.float64) for k, v in (coupling_params or {}).items()}
    if coupling == 'Linear':
        cp.setdefault('a', np.array(0.00390625))
        cp.setdefault('b', np.array(0.0))
    elif coupling == 'Difference':
        cp.setdefault('a', np.array(0.1))
    elif coupling == 'SigmoidalJansenRit':
        for k, v in dict(cmin=0.0, cmax=2.0 * 0.0025, midpoint=6.0, r=0.56, a=1.0).items():
            cp.setdefault(k, np.array(v))
    elif coupling == 'Scaling':
        cp.setdefault('a', np.array(0.00390625))
    elif coupling == 'HyperbolicTangent':
        for k, v in dict(a=1.0, b=1.0, midpoint=0.0, sigma=1.0).items():
            cp.setdefault(k, np.array(v))
    elif coupling == 'Sigmoidal':
        for k, v in dict(cmin=-1.0, cmax=1.0, midpoint=0.0, a=1.0, sigma=230.0).items():
            cp.setdefault(k, np.array(v))
    elif coupling == 'Kuramoto':
        cp.setdefault('a', np.array(1.0))

    def couple(step):
        if coupling == 'SigmoidalJansenRit':
            return coupling_sigmoidal_jr(buf, step, idelays, whist, cp)
        return coupling_sparse(coupling, buf, step, lay, cp)

    def bound(Z):
        for i, lo, hi in bidx:
            Z[i][Z[i] < lo] = lo
            Z[i][Z[i] > hi] = hi

    gfun = None
    if integrator in ('HeunStochastic', 'EulerStochastic'):
        nsig_arr = np.asarray(nsig, dtype=np.float64)
        if nsig_arr.ndim == 1 and nsig_arr.size == len(svars) and len(svars) > 1:
            nsig_arr = nsig_arr.reshape((-1, 1))
        gfun = np.sqrt(2.0 * nsig_arr)                      # Additive.gfun, noise.py:223-232

    # monitors
    hrf, stock_steps = bold_hrf()
    mstate = []
    afferent_rows = 1 if coupling == 'SigmoidalJansenRit' else len(cvar)
    for m in monitors:
        st = dict(m=m)
        if m.kind.startswith('AfferentCoupling'):                 # monitors.py:406-409: coupling rows
            mv = list(range(afferent_rows)) if m.voi is None else list(m.voi)
        else:
            mv = list(range(len(voi))) if m.voi is None else list(m.voi)
        st['voi'] = mv
        if m.kind in ('Raw', 'AfferentCoupling'):
            st['istep'] = 1
        elif m.kind in ('TemporalAverage', 'AfferentCouplingTemporalAverage'):
            st['istep'] = iround(m.period / dt)
            st['stock'] = np.zeros((st['istep'], len(mv), X.shape[1]))
        elif m.kind in ('SubSample', 'GlobalAverage', 'SpatialAverage'):
            st['istep'] = iround(m.period / dt)
            if m.kind == 'SpatialAverage':                # monitors.py:311-318
                nn = X.shape[1]
                total = np.zeros((nn, int(m.spatial_mask.max()) + 1))
                total[np.arange(nn), m.spatial_mask] = 1
                total = total.T
                st['mean'] = total / np.sum(total, axis=1)[:, np.newaxis]
        elif m.kind == 'Projection':                     # monitors.py:596-600
            st['istep'] = int(m.period / dt)
            st['state'] = np.zeros((m.gain.shape[0], len(mv)))
            st['k'] = 0
        elif m.kind == 'Bold':
            st['istep'] = iround(m.period / dt)
            st['ii'] = int(round((1.0 / 2.0 ** -2) / dt))
            st['interim'] = np.zeros((st['ii'], len(mv), X.shape[1]))
            st['stock'] = np.zeros((stock_steps, len(mv), X.shape[1]))
        st['t'], st['y'] = [], []
        mstate.append(st)

    start = step0 + 1
    c = couple(start)
    stim = 0.0
    if stimulus is not None:
        s_temporal, s_weight, s_vars = stimulus
        stim = np.zeros_like(X)
    for k, step in enumerate(range(start, start + n_steps)):
        if stimulus is not None:
            stim[np.asarray(s_vars)] = np.asarray(s_weight, dtype=np.float64) * s_temporal[k]
        if integrator == 'HeunDeterministic':          # integrators.py:296-318
            m0 = dfun(X, c, p)
            inter = X + dt * (m0 + stim)
            bound(inter)
            dX = (m0 + dfun(inter, c, p)) * dt / 2.0
            X = X + dX + dt * stim
        elif integrator == 'HeunStochastic':           # integrators.py:330-362
            noise = np.sqrt(dt) * noise_z[k]
            m0 = dfun(X, c, p)
            noise = noise * gfun
            inter = X + dt * m0 + noise + dt * stim
            bound(inter)
            dX = (m0 + dfun(inter, c, p)) * dt / 2.0
            X = X + dX + noise + dt * stim
        elif integrator == 'EulerDeterministic':       # integrators.py:376-391
            dX = dfun(X, c, p)
            X = X + dt * (dX + stim)
        elif integrator == 'EulerStochastic':          # integrators.py:405-426
            noise = np.sqrt(dt) * noise_z[k]
            dX = dfun(X, c, p) * dt
            X = X + dX + gfun * noise + dt * stim
        elif integrator == 'Identity':                 # integrators.py:494-507
            X = dfun(X, c, p) + stim
        elif integrator == 'RungeKutta4thOrderDeterministic':   # integrators.py:437-480
            dt2, dt6 = dt / 2.0, dt / 6.0
            k1 = dfun(X, c, p)
            i1 = X + dt2 * k1
            bound(i1)
            k2 = dfun(i1, c, p)
            i2 = X + dt2 * k2
            bound(i2)
            k3 = dfun(i2, c, p)
            i3 = X + dt * k3
            bound(i3)
            k4 = dfun(i3, c, p)
            X = X + dt6 * (k1 + 2.0 * k2 + 2.0 * k3 + k4) + dt * stim
        else:
            raise NotImplementedError(integrator)
        bound(X)
        buf[step % H] = X[cvar]                          # history.py:203-204
        c = couple(step + 1)                             # simulator.py:360
        obs = observe(model, X, voi) if info else X      # simulator.py:314-320
        for st in mstate:
            m = st['m']
            # AfferentCoupling monitors see node_coupling of step + 1 (simulator.py:314-320)
            o = (c if m.kind.startswith('AfferentCoupling') else obs)[st['voi']]
            if m.kind in ('Raw', 'AfferentCoupling'):    # monitors.py:188-190,411-412
                st['t'].append(step * dt)
                st['y'].append(o.copy())
            elif m.kind in ('TemporalAverage', 'AfferentCouplingTemporalAverage'):   # monitors.py:380-391
                st['stock'][(step % st['istep']) - 1] = o
                if step % st['istep'] == 0:
                    st['t'].append((step - st['istep'] / 2.0) * dt)
                    st['y'].append(np.mean(st['stock'], axis=0))
            elif m.kind in ('SubSample', 'GlobalAverage', 'SpatialAverage'):
                if step % st['istep'] == 0:
                    st['t'].append(step * dt)
                    if m.kind == 'SubSample':              # monitors.py:219-222
                        st['y'].append(o.copy())
                    elif m.kind == 'GlobalAverage':        # monitors.py:350-355
                        st['y'].append(np.mean(o, axis=1)[:, np.newaxis])
                    else:                                  # monitors.py:321-325 (o is (nvoi, n): no modes axis)
                        st['y'].append(np.dot(st['mean'], o.T).T)
            elif m.kind == 'Projection':                 # monitors.py:602-614, EEG 718-723
                st['state'] += m.gain.dot(o.T)
                if step % st['istep'] == 0:
                    sample = st['state'].copy() / st['istep']
                    if m.obs_z is not None:
                        sample += np.sqrt(dt) * m.obs_z[st['k']]
                    st['k'] += 1
                    st['state'][:] = 0.0
                    sample = sample.T
                    if m.ref_vec is not None:
                        sample = sample - m.ref_vec.dot(sample.T)[:, np.newaxis]
                    st['t'].append((step - st['istep'] / 2.0) * dt)
                    st['y'].append(sample)
            elif m.kind == 'Bold':                       # monitors.py:942-962
                ii = st['ii']
                st['interim'][(step % ii) - 1] = o
                if step % ii == 0:
                    st['stock'][(step // ii % stock_steps) - 1] = np.mean(st['interim'], axis=0)
                if step % st['istep'] == 0:
                    h = np.roll(hrf, (step // ii % stock_steps) - 1)
                    bold = (np.tensordot(h, st['stock'], axes=(0, 0)) - 1.0) * (5.6 * 0.02)
                    st['t'].append(step * dt)
                    st['y'].append(bold)
    out = []
    for st in mstate:
        out.append((np.array(st['t']), np.array(st['y'])))
    return out, dict(buffer=buf, state=X, step=start + n_steps - 1)


def functional_connectivity(bold):
    """Pearson FC over time as the framework analyzer computes it
    (tvb_framework/tvb/adapters/analyzers/cross_correlation_adapter.py:378):
    numpy.corrcoef(data.T) for data of shape (T, n)."""
    return np.corrcoef(np.asarray(bold, dtype=np.float64).T)


# ----------------------------------------------------------------------------
# Balloon-Windkessel BOLD (analyzer)


def balloon_bold(x, dt, tau_s=1.54, tau_f=1.44, tau_o=0.98, alpha=0.32, E0=0.4, V0=4.0, k=(None, None, None),
                 nonlinear=True):
    """BalloonModel.evaluate after its input transformation
    (tvb/analyzers/fmri_balloon.py:215-283,339-364): x (T, n) float64 neural
    input, dt in seconds, HeunDeterministic from s = 0, f = v = q = 1;
    returns the BOLD signal (T, n), step 0 included."""
    k1, k2, k3 = k
    T = x.shape[0]
    y = np.zeros((4, x.shape[1]))
    y[1:] = 1.0

    def dfun(y, xt):
        s, f, v, q = y
        return np.array([xt - (1. / tau_s) * s - (1. / tau_f) * (f - 1), s,
                         (1. / tau_o) * (f - v ** (1. / alpha)),
                         (1. / tau_o) * ((f * (1. - (1. - E0) ** (1. / f)) / E0) - (v ** (1. / alpha)) * (q / v))])

    def bold(y):
        v, q = y[2], y[3]
        if nonlinear:
            return V0 * (k1 * (1. - q) + k2 * (1. - q / v) + k3 * (1. - v))
        return V0 * ((k1 + k2) * (1. - q) + (k3 - k2) * (1. - v))

    out = np.zeros((T, x.shape[1]))
    out[0] = bold(y)
    for t in range(1, T):
        m0 = dfun(y, x[t])
        inter = y + dt * (m0 + 0.0)                          # integrators.py:310
        y = y + (m0 + dfun(inter, x[t])) * dt / 2.0          # integrators.py:313-315
        out[t] = bold(y)
    return out
