"""Autotuner for the batched simulation kernel.

The simulation kernel has several variants that compute the same loop with a
different mapping of the work onto the GPU:

* instances per CTA: one instance per CTA (``lanes=1``), groups of 8 / ncvar
  instances per CTA with interleaved rings (``lanes=8//ncvar``), or the other
  way round, a thread-block cluster of C CTAs per instance (``cluster=C``);
* history tiling: the ring staged in shared memory for the whole launch
  (``ring_in_smem=True``) or read in place from L2 / HBM;
* the coupling gather: one thread per row with the next step's gather issued
  ahead (``gather='row'``), the same with the gather on separate warps
  (``gather='split'``), or a balanced edge-parallel split (``gather='edge'``).

Which one is fastest depends on the instance count, the region count, the
horizon, the degree distribution and the model.  ``tune`` runs each variant
that applies on a short trial of the actual batch (same instances, same
connectomes, `trial_steps` steps, timed with CUDA events after a warm-up)
and returns the fastest.  Results are cached in a JSON file keyed by the GPU
name and the batch's shape, so later batches of the same shape skip the
trials.  Monitors are always fused into the simulation kernel (Raw,
TemporalAverage and Bold accumulate in registers and are written from the
kernel), so there is no separate monitor variant to tune.
"""
import json
import os

import numpy as np
import torch

from . import _lib

CACHE_ENV = 'TVB_B200_TUNE_CACHE'


def cache_path():
    p = os.environ.get(CACHE_ENV)
    if p:
        return p
    base = os.environ.get('XDG_CACHE_HOME', os.path.join(os.path.expanduser('~'), '.cache'))
    return os.path.join(base, 'tvb_b200', 'autotune.json')


def shape_key(model_id, cfun_id, scheme_id, noise_kind, dt, voi, specs, device):
    """Cache key: GPU, components, instance count and the connectome shapes."""
    name = torch.cuda.get_device_name(device) if torch.cuda.is_available() else 'cpu'
    c = specs[0].conn
    deg = np.diff(c.row_ptr)
    mons = (bool(specs[0].raw), specs[0].tavg_istep > 0, specs[0].bold is not None)
    same = all(s.conn is c for s in specs)
    return '|'.join(str(x) for x in (name, model_id, cfun_id, scheme_id, noise_kind, np.float32(dt), tuple(voi),
                                     len(specs), c.n, c.horizon, c.nnz, int(deg.max(initial=0)), c.min_delay,
                                     mons, same))


def candidates(ncvar, n, n_inst, shared_conn):
    """Variants to try (keyword arguments of ``Batch``)."""
    out = [dict(gather='row', lanes=1, ring_in_smem=None, cluster=0),
           dict(gather='split', lanes=1, ring_in_smem=True, cluster=0),
           dict(gather='row', lanes=1, ring_in_smem=False, cluster=0),
           dict(gather='edge', lanes=1, ring_in_smem=None, cluster=0)]
    if shared_conn and n_inst % (8 // ncvar) == 0:
        out.append(dict(gather='row', lanes=8 // ncvar, ring_in_smem=None, cluster=0))
    for C in (2, 4, 8, 16):
        if C <= max(2, -(-n // 32)):
            out.append(dict(gather='row', lanes=1, ring_in_smem=False, cluster=C))
    return out


def _load_cache(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save_cache(path, cache):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + '.tmp%d' % os.getpid()
        with open(tmp, 'w') as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def tune(make_batch, key, ncvar, n, n_inst, shared_conn, trial_steps=2000, use_cache=True, path=None):
    """Time the applicable variants and return (best kwargs, {variant: ms}).

    make_batch(**kwargs) builds and allocates a ``Batch`` of the instances
    with one variant (raising ValueError when the variant does not apply).
    """
    path = path or cache_path()
    cache = _load_cache(path) if use_cache else {}
    if use_cache and key in cache:
        return cache[key]['best'], cache[key]['ms']
    timings, best, best_ms = {}, None, None
    for cand in candidates(ncvar, n, n_inst, shared_conn):
        try:
            b = make_batch(**cand)
        except (ValueError, _lib.TvbkError):
            continue
        name = '%s/lanes%d/%s/cluster%d/prefetch%d' % (cand['gather'], b.lanes,
                                                        'smem' if b.ring_in_smem else 'inplace', b.cluster,
                                                        b.prefetch)
        if name in timings:
            continue
        try:
            b.snapshot()
            b.run(n_steps=max(1, trial_steps // 4))
            b.reset()
            st = torch.cuda.current_stream(b.device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            b.run(n_steps=trial_steps)
            e1.record(st)
            torch.cuda.synchronize(b.device)
            ms = e0.elapsed_time(e1)
        except _lib.TvbkError:
            continue
        finally:
            del b
        timings[name] = ms
        if best_ms is None or ms < best_ms:
            best, best_ms = cand, ms
    if best is None:
        raise RuntimeError('no kernel variant applies to this batch')
    if use_cache:
        cache = _load_cache(path)
        cache[key] = {'best': best, 'ms': timings}
        _save_cache(path, cache)
    return best, timings
