"""Build libtvbk.so (the sm_100a kernels and their C ABI) in-tree.

    python tvb-root_b200/build.py [--force] [--verbose]

Each ``csrc/*.cu`` file is compiled separately (in parallel) with nvcc for
sm_100a and linked into ``tvb_b200/_lib/libtvbk.so``.  Objects are rebuilt
when a source or header is newer than them.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
INCLUDE = os.path.join(REPO, 'include')
OBJ = os.path.join(HERE, '_build')
LIBDIR = os.path.join(HERE, 'tvb_b200', '_lib')
LIB = os.path.join(LIBDIR, 'libtvbk.so')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC', '-Xcompiler', '-O3',
              '--expt-relaxed-constexpr', '-I', CSRC, '-I', INCLUDE]


def nvcc():
    path = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(path):
        raise RuntimeError('nvcc not found')
    return path


def _headers():
    return glob.glob(os.path.join(CSRC, '*.cuh')) + glob.glob(os.path.join(INCLUDE, '*.h'))


def _compile(src, force, verbose, extra):
    obj = os.path.join(OBJ, os.path.basename(src) + '.o')
    newest = max(os.path.getmtime(p) for p in [src] + _headers())
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ['-c', src, '-o', obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('nvcc failed for %s:\n%s\n%s' % (src, ' '.join(cmd), r.stderr))
    return obj, (r.stderr if verbose else None)


# Relative compile times of the simulation translation units (model x scheme), so that the longest start
# first and the parallel build does not end on one long unit.
_MODEL_COST = {'jr': 4, 'epileptor': 3, 'rww': 2, 'g2d': 2, 'sum': 1}
_SCHEME_COST = {'heun_stoch': 4, 'rk4': 4, 'heun_det': 3, 'euler_stoch': 2, 'euler_det': 1}


def _compile_cost(src):
    name = os.path.basename(src)[:-3]
    if not name.startswith('tvbk_sim_'):
        return (0, name)
    parts = name[len('tvbk_sim_'):]
    model = parts.split('_')[0]
    scheme = parts[len(model) + 1:]
    return (_MODEL_COST.get(model, 1) * _SCHEME_COST.get(scheme, 1), name)


def build(force=False, verbose=False, extra=()):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, '*.cu')), key=_compile_cost, reverse=True)
    with cf.ThreadPoolExecutor(max_workers=min(max(os.cpu_count() or 1, 1), 16, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose, list(extra)), srcs))
    objs = [o for o, _ in results]
    for _, log in results:
        if log:
            sys.stderr.write(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ['-shared', '-o', LIB] + objs + ['-lcudart']
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError('link failed:\n%s\n%s' % (' '.join(cmd), r.stderr))
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--verbose', action='store_true', help='print ptxas resource usage')
    args = ap.parse_args()
    extra = ['-Xptxas', '-v'] if args.verbose else []
    print(build(force=args.force or args.verbose, verbose=args.verbose, extra=extra))
