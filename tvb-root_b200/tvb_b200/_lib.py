"""ctypes binding of libtvbk.so (include/tvbk.h).

The struct mirrors below must match the C header field for field; the
library's ``tvbk_sizeof`` is checked at load time.  Loading fails loudly when
the shared library is missing: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, '_lib', 'libtvbk.so')

TVBK_OK = 0
TVBK_ERR_INVALID = -1
TVBK_ERR_UNSUPPORTED = -2
TVBK_ERR_CUDA = -3
TVBK_ERR_TOO_LARGE = -4
TVBK_STATUS_NONFINITE = 1
TVBK_STATUS_DEGREE = 2
TVBK_STATUS_UNSUPPORTED = 4
TVBK_STATUS_TIMEOUT = 8

MODEL_IDS = {'Generic2dOscillator': 0, 'JansenRit': 1, 'ReducedWongWang': 2, 'Epileptor': 3, 'Sum': 4}
CFUN_IDS = {'Linear': 0, 'Difference': 1, 'SigmoidalJansenRit': 2, 'Sigmoidal': 3, 'HyperbolicTangent': 4,
            'Kuramoto': 5}
# couplings whose kernel runs the row gather one step at a time with the pre / post chosen at run time
CFUN_GENERIC = (3, 4, 5)
SCHEME_IDS = {'EulerDeterministic': 0, 'EulerStochastic': 1, 'HeunDeterministic': 2,
              'HeunStochastic': 3, 'Identity': 4, 'RungeKutta4thOrderDeterministic': 5}
NOISE_NONE, NOISE_FED, NOISE_PHILOX = 0, 1, 2
MAX_REGIONS = 1024
MAX_VOI = 8
STATIC_SCRATCH_BYTES = 8 * 1024 * 1024
# mirrored slots past the end of a ring staged in shared memory with prefetch = 1 (TVBK_RING_GUARD)
RING_GUARD = 3


def group_sync_words(groups):
    """Words of launch.group_sync for `groups` groups (TVBK_GROUP_SYNC_WORDS)."""
    return 2 + 2 * groups


def ring_region_stride(ring_len, ncvar):
    """Slots per region of a region-major ring (TVBK_RING_REGION_STRIDE)."""
    spc = 8 // ncvar
    return -(-(ring_len + (14 if ncvar == 1 else 10)) // spc) * spc


class Edge(ctypes.Structure):
    _fields_ = [('off', ctypes.c_int32), ('weight', ctypes.c_float)]


class Inst(ctypes.Structure):
    _fields_ = [
        ('row_ptr', ctypes.c_void_p),
        ('edges', ctypes.c_void_p),
        ('slots', ctypes.c_void_p),
        ('ring', ctypes.c_void_p),
        ('pre_ring', ctypes.c_void_p),
        ('state', ctypes.c_void_p),
        ('params', ctypes.c_void_p),
        ('noise_sigma', ctypes.c_void_p),
        ('noise_fed', ctypes.c_void_p),
        ('stim', ctypes.c_void_p),
        ('stim_weight', ctypes.c_void_p),
        ('raw', ctypes.c_void_p),
        ('sub', ctypes.c_void_p),
        ('tavg', ctypes.c_void_p),
        ('aff', ctypes.c_void_p),
        ('aff_acc', ctypes.c_void_p),
        ('proj', ctypes.c_void_p),
        ('proj_acc', ctypes.c_void_p),
        ('tavg_acc', ctypes.c_void_p),
        ('bold', ctypes.c_void_p),
        ('bold_acc', ctypes.c_void_p),
        ('bold_stock', ctypes.c_void_p),
        ('hrf', ctypes.c_void_p),
        ('step', ctypes.c_int64),
        ('step_end', ctypes.c_int64),
        ('raw_base', ctypes.c_int64),
        ('fed_base', ctypes.c_int64),
        ('tavg_base', ctypes.c_int64),
        ('bold_base', ctypes.c_int64),
        ('sub_base', ctypes.c_int64),
        ('stim_base', ctypes.c_int64),
        ('aff_base', ctypes.c_int64),
        ('proj_base', ctypes.c_int64),
        ('n', ctypes.c_int32),
        ('nnz', ctypes.c_int32),
        ('horizon', ctypes.c_int32),
        ('ring_len', ctypes.c_int32),
        ('tavg_istep', ctypes.c_int32),
        ('bold_istep', ctypes.c_int32),
        ('bold_ii', ctypes.c_int32),
        ('stock_len', ctypes.c_int32),
        ('sub_istep', ctypes.c_int32),
        ('stim_vars', ctypes.c_uint32),
        ('aff_istep', ctypes.c_int32),
        ('proj_istep', ctypes.c_int32),
        ('slot_width', ctypes.c_int32),
        ('cfun', ctypes.c_float * 6),
        ('seed', ctypes.c_uint32),
        ('stream', ctypes.c_uint32),
        ('bold_k1v0', ctypes.c_double),
    ]


class Launch(ctypes.Structure):
    _fields_ = [
        ('insts', ctypes.c_void_p),
        ('status', ctypes.c_void_p),
        ('n_inst', ctypes.c_int32),
        ('model', ctypes.c_int32),
        ('cfun', ctypes.c_int32),
        ('scheme', ctypes.c_int32),
        ('noise', ctypes.c_int32),
        ('nvoi', ctypes.c_int32),
        ('voi', ctypes.c_int32 * MAX_VOI),
        ('max_n', ctypes.c_int32),
        ('max_ring_len', ctypes.c_int32),
        ('sync_every', ctypes.c_int32),
        ('ring_in_smem', ctypes.c_int32),
        ('max_degree', ctypes.c_int32),
        ('edges_per_thread', ctypes.c_int32),
        ('block_threads', ctypes.c_int32),
        ('prefetch', ctypes.c_int32),
        ('lanes', ctypes.c_int32),
        ('cluster', ctypes.c_int32),
        ('cluster_edges', ctypes.c_int32),
        ('ring_layout', ctypes.c_int32),
        ('block_steps', ctypes.c_int32),
        ('groups', ctypes.c_int32),
        ('group_sync', ctypes.c_void_p),
        ('extras', ctypes.c_int32),
        ('inst_order', ctypes.c_void_p),
        ('occupancy', ctypes.c_void_p),
        ('max_steps', ctypes.c_int64),
        ('dt', ctypes.c_float),
    ]


INST_DTYPE = np.dtype(Inst)

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

_SIGNATURES = {
    'tvbk_abi_version': (_I32, []),
    'tvbk_last_error': (ctypes.c_char_p, []),
    'tvbk_sizeof': (_I64, [_I32]),
    'tvbk_idelays': (_I32, [_P, _I64, _D, _D, _P, _P]),
    'tvbk_sparse_layout': (_I32, [_P, _P, _I32, _P, _P, _P, _P, _P, _P]),
    'tvbk_pack_edges': (_I32, [_P, _P, _P, _I32, _I32, _I32, _P]),
    'tvbk_ring_len': (_I32, [_I32, _I32]),
    'tvbk_ring_smem_bytes': (_I64, [_I32, _I32, _I32]),
    'tvbk_model_dims': (_I32, [_I32, _P, _P, _P, _P, _P]),
    'tvbk_sim_run': (_I32, [ctypes.POINTER(Launch), _P]),
    'tvbk_gather_delayed': (_I32, [ctypes.POINTER(Inst), _I32, _I64, _P, _P]),
    'tvbk_fc': (_I32, [_P, _I32, _I32, _I32, _P, _P]),
    'tvbk_project': (_I32, [_P, _I64, _I32, _I32, _P, _I32, _P, _I32, _P, _P]),
    'tvbk_balloon': (_I32, [_P, _I32, _I64, _D, _P, _I32, _P, _P]),
    'tvbk_sim_run_static': (_I32, [ctypes.POINTER(Launch), ctypes.POINTER(Inst), _P, _P]),
}

EXPORTED = tuple(_SIGNATURES)


class TvbkError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__('%s (status %d)' % (msg, code))
        self.code = code


_lib = None


def load():
    """Load libtvbk.so once; raise ImportError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError('libtvbk.so not built (%s); run tvb-root_b200/build.py' % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    sizes = [lib.tvbk_sizeof(k) for k in range(3)]
    want = [ctypes.sizeof(Inst), ctypes.sizeof(Launch), ctypes.sizeof(Edge)]
    if sizes != want:
        raise ImportError('libtvbk.so struct sizes %s do not match the binding %s' % (sizes, want))
    _lib = lib
    return lib


def check(code, what=''):
    if code != TVBK_OK:
        msg = load().tvbk_last_error().decode()
        raise TvbkError(code, msg or what)
    return code


def ptr(a):
    """Address of a numpy array's data as an int (None for None)."""
    if a is None:
        return None
    return a.ctypes.data


# ------------------------------------------------------------ host planning


def idelays(tract_lengths, speed, dt):
    """Integer delays and horizon via tvbk_idelays (rint((L / speed) / dt), half to even)."""
    L = np.ascontiguousarray(tract_lengths, dtype=np.float64)
    out = np.empty(L.shape, dtype=np.int32)
    hz = np.zeros(1, dtype=np.int32)
    check(load().tvbk_idelays(ptr(L), L.size, float(speed), float(dt), ptr(out), ptr(hz)))
    return out, int(hz[0])


def sparse_layout(weights, idel):
    """Row-major non-zero layout (row_ptr, col, idelay, weight f32, nnz, min_delay)."""
    W = np.ascontiguousarray(weights, dtype=np.float64)
    D = np.ascontiguousarray(idel, dtype=np.int32)
    n = W.shape[0]
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    col = np.zeros(n * n, dtype=np.int32)
    dly = np.zeros(n * n, dtype=np.int32)
    w = np.zeros(n * n, dtype=np.float32)
    nnz = np.zeros(1, dtype=np.int32)
    dmin = np.zeros(1, dtype=np.int32)
    check(load().tvbk_sparse_layout(ptr(W), ptr(D), n, ptr(row_ptr), ptr(col), ptr(dly), ptr(w),
                                     ptr(nnz), ptr(dmin)))
    k = int(nnz[0])
    return row_ptr, col[:k].copy(), dly[:k].copy(), w[:k].copy(), k, int(dmin[0])


def pack_edges(col, dly, w, n, ncvar):
    nnz = len(col)
    out = np.zeros(max(nnz, 1), dtype=np.dtype([('off', np.int32), ('weight', np.float32)]))
    col = np.ascontiguousarray(col, dtype=np.int32)
    dly = np.ascontiguousarray(dly, dtype=np.int32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    check(load().tvbk_pack_edges(ptr(col), ptr(dly), ptr(w), nnz, n, ncvar, ptr(out)))
    return out[:nnz] if nnz else out[:0]


def model_dims(model_id):
    v = [np.zeros(1, dtype=np.int32) for _ in range(5)]
    check(load().tvbk_model_dims(model_id, *[ptr(a) for a in v]))
    return tuple(int(a[0]) for a in v)  # ncvar, nsv, nintvar, nobs, nparam
