"""The C ABI of libtvbk.so without a GPU: the library loads, exports every
function include/tvbk.h declares, its struct sizes match the ctypes mirrors,
the host-side planning functions reproduce the reference's integer
arithmetic, and argument errors come back as status codes (no CUDA call is
made on those paths)."""
import ctypes
import os
import re

import numpy as np
import pytest

import golden_util as G
from oracle import tvb_oracle as O
from tvb_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'include', 'tvbk.h')


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', ' ', text, flags=re.S)
    names = re.findall(r'^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(tvbk_[a-z0-9_]+)\s*\(', text, flags=re.M)
    return sorted(set(names))


def test_every_declared_function_is_exported_and_bound():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(_lib.EXPORTED) == names


def test_struct_sizes_and_version():
    lib = _lib.load()
    assert lib.tvbk_abi_version() == 3
    assert lib.tvbk_sizeof(0) == ctypes.sizeof(_lib.Inst)
    assert lib.tvbk_sizeof(1) == ctypes.sizeof(_lib.Launch)
    assert lib.tvbk_sizeof(2) == 8
    assert lib.tvbk_sizeof(7) == -1


def test_idelays_match_reference_golden():
    fx = G.load('idelays')
    L = fx['tract_lengths']
    cases = [k[len('idelays_'):] for k in fx if k.startswith('idelays_')]
    assert len(cases) >= 8
    for case in cases:
        m = re.match(r's([0-9.]+)_dt([0-9.]+)$', case)
        idl, H = _lib.idelays(L, float(m.group(1)), float(m.group(2)))
        np.testing.assert_array_equal(idl, fx['idelays_' + case])
        assert H == int(fx['horizon_' + case])


def test_sparse_layout_and_packing_match_oracle():
    w, L = G.connectome(G.load('g2d_76'))
    idl, H = _lib.idelays(L, 3.0, 0.1)
    row_ptr, col, dly, wt, nnz, dmin = _lib.sparse_layout(w, idl)
    o_rows, o_cols = np.nonzero(w)  # row-major, as numpy.argwhere in SparseHistory
    assert nnz == o_rows.size
    np.testing.assert_array_equal(col, o_cols)
    np.testing.assert_array_equal(dly, idl[o_rows, o_cols])
    np.testing.assert_array_equal(wt, w[o_rows, o_cols].astype(np.float32))
    np.testing.assert_array_equal(np.diff(row_ptr), np.bincount(o_rows, minlength=w.shape[0]))
    assert dmin == int(idl[o_rows, o_cols].min())
    n = w.shape[0]
    for ncvar in (1, 2):
        e = _lib.pack_edges(col, dly, wt, n, ncvar)
        np.testing.assert_array_equal(e['off'], (dly.astype(np.int64) * n - col) * ncvar)
        np.testing.assert_array_equal(e['weight'], wt)
    ref_idl, ref_H = O.integer_delays(L, 3.0, 0.1)
    np.testing.assert_array_equal(idl, ref_idl)
    assert H == ref_H


def test_model_dims_and_ring_helpers():
    assert _lib.model_dims(_lib.MODEL_IDS['ReducedWongWang'])[:3] == (1, 1, 1)
    assert _lib.model_dims(_lib.MODEL_IDS['Epileptor'])[:2] == (2, 6)
    lib = _lib.load()
    assert lib.tvbk_ring_len(401, 21) == 422
    assert lib.tvbk_ring_len(0, 1) == -1
    assert lib.tvbk_ring_smem_bytes(68, 1, 422) == 422 * 68 * 4
    assert lib.tvbk_ring_smem_bytes(998, 2, 2001) == 0


def test_header_layout_macros_match_the_binding(tmp_path):
    """TVBK_RING_REGION_STRIDE / _GUARD and TVBK_GROUP_SYNC_WORDS, evaluated
    by a C compiler from include/tvbk.h, equal the Python mirrors; regions of
    region-major rings start on 32-byte boundaries."""
    import shutil
    import subprocess
    cc = shutil.which('gcc') or shutil.which('cc')
    if cc is None:
        pytest.skip('no C compiler')
    src = tmp_path / 'm.c'
    src.write_text('#include <stdio.h>\n#include "tvbk.h"\nint main(void) {\n'
                   '  for (int rl = 1; rl < 80; ++rl) for (int c = 1; c <= 2; ++c)\n'
                   '    printf("%d %d %d %d\\n", rl, c, TVBK_RING_REGION_STRIDE(rl, c), TVBK_RING_REGION_GUARD(c));\n'
                   '  printf("g %d\\n", TVBK_GROUP_SYNC_WORDS(9));\n  return 0;\n}\n')
    exe = tmp_path / 'm'
    subprocess.check_call([cc, '-std=c99', '-I', os.path.dirname(HEADER), str(src), '-o', str(exe)])
    lines = subprocess.check_output([str(exe)], text=True).split('\n')
    assert lines[-2] == 'g %d' % _lib.group_sync_words(9)
    for ln in lines[:-2]:
        rl, c, rs, guard = map(int, ln.split())
        assert rs == _lib.ring_region_stride(rl, c)
        assert rs >= rl + guard and (rs * c * 4) % 32 == 0


def test_argument_errors_are_status_codes():
    lib = _lib.load()
    assert lib.tvbk_sim_run(None, None) == _lib.TVBK_ERR_INVALID
    assert b'null launch' in lib.tvbk_last_error()
    L = _lib.Launch()
    L.model = 99
    assert lib.tvbk_sim_run(ctypes.byref(L), None) == _lib.TVBK_ERR_INVALID
    L.model = _lib.MODEL_IDS['ReducedWongWang']
    L.insts, L.status, L.n_inst = 16, 16, 1  # never dereferenced: max_n fails first
    L.max_n = 5000
    assert lib.tvbk_sim_run(ctypes.byref(L), None) == _lib.TVBK_ERR_TOO_LARGE
    with pytest.raises(_lib.TvbkError):
        _lib.idelays(np.full((2, 2), 10.0), -1.0, 0.1)
    assert lib.tvbk_fc(None, 1, 10, 4, None, None) == _lib.TVBK_ERR_INVALID


def test_group_launch_arguments_are_checked():
    """launch.groups (cooperative launch of groups of CTAs per instance) is
    refused without region-major rings or a 4-byte aligned group_sync, and
    allows up to 256 CTAs per instance; nothing is dereferenced or launched."""
    lib = _lib.load()
    L = _lib.Launch()
    L.model, L.cfun, L.scheme = _lib.MODEL_IDS['ReducedWongWang'], _lib.CFUN_IDS['Linear'], 0
    L.insts, L.status, L.n_inst = 16, 16, 1
    L.max_n, L.sync_every, L.max_steps, L.dt = 68, 4, 10, 0.1
    L.groups, L.cluster, L.ring_layout = 2, 2, 0
    L.group_sync = 64
    assert lib.tvbk_sim_run(ctypes.byref(L), None) == _lib.TVBK_ERR_INVALID
    assert b'groups' in lib.tvbk_last_error()
    L.ring_layout, L.group_sync = 1, None
    assert lib.tvbk_sim_run(ctypes.byref(L), None) == _lib.TVBK_ERR_INVALID
    assert b'group_sync' in lib.tvbk_last_error()
    L.group_sync = 66
    assert lib.tvbk_sim_run(ctypes.byref(L), None) == _lib.TVBK_ERR_INVALID
    assert b'aligned' in lib.tvbk_last_error()
    L.group_sync, L.cluster = 64, 300
    assert lib.tvbk_sim_run(ctypes.byref(L), None) == _lib.TVBK_ERR_INVALID
    assert b'0..256' in lib.tvbk_last_error()
    L.groups = 0
    L.cluster = 20
    assert lib.tvbk_sim_run(ctypes.byref(L), None) == _lib.TVBK_ERR_INVALID
    assert b'0..16' in lib.tvbk_last_error()

