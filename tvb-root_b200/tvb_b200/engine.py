"""Device execution of a batch of simulation instances.

A ``Batch`` packs every per-instance array (ring, state, parameters, noise
scales, monitor accumulators and outputs) and the shared connectomes into
device arenas owned by torch, writes one ``tvbk_inst`` descriptor per
instance, and advances all instances with ``tvbk_sim_run`` in chunks.  All
instances of a batch share model, coupling, scheme, noise kind, dt and the
observed variables; they may differ in connectome, size, parameters,
length and monitors' presence.

Inputs travel in one host-to-device copy of a staging arena; accumulators and
outputs are zero-filled on the device.  Outputs come back in one
device-to-host copy.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib

ALIGN = 256


def _aligned(x):
    return (x + ALIGN - 1) // ALIGN * ALIGN


def _array_key(a):
    """Identity of an array's contents by its memory (views of one buffer with
    the same layout are the same input), else of the object."""
    if isinstance(a, np.ndarray):
        return ('np', a.__array_interface__['data'][0], a.shape, a.strides, a.dtype.str)
    if isinstance(a, torch.Tensor):
        return ('torch', a.data_ptr(), tuple(a.shape), tuple(a.stride()), str(a.dtype))
    return ('obj', id(a))


class _Arena:
    """Byte offsets of named regions in one allocation."""

    def __init__(self):
        self.size = 0
        self.regions = {}

    def add(self, key, nbytes):
        off = _aligned(self.size)
        self.regions[key] = (off, int(nbytes))
        self.size = off + int(nbytes)
        return off


def ring_from_reference(buffer, step, ring_len):
    """Reference history buffer (H, ncvar, n), time t in slot t % H for
    t in [step - H + 1, step], to the device ring (ring_len, n, ncvar) with
    time t in slot t % ring_len (tvb/simulator/history.py:197-204)."""
    buf = np.asarray(buffer)
    H, ncv, n = buf.shape
    ring = np.zeros((ring_len, n, ncv), dtype=np.float32)
    ts = np.arange(step - H + 1, step + 1)
    ring[ts % ring_len] = buf[ts % H].transpose(0, 2, 1)
    return ring


def ring_region_major(ring, ncvar):
    """Time-major ring (ring_len, n, ncvar) to the region-major layout of the
    cluster kernel's blocked runs: (n, stride, ncvar), the slots past ring_len
    mirroring slots 0, 1, ... (TVBK_RING_REGION_STRIDE / _GUARD)."""
    ring = np.asarray(ring)
    RL, n, ncv = ring.shape
    RS = _lib.ring_region_stride(RL, ncvar)
    out = np.zeros((n, RS, ncv), dtype=ring.dtype)
    out[:, :RL] = ring.transpose(1, 0, 2)
    g = RS - RL
    out[:, RL:RL + g] = out[:, :g]
    return out


def ring_time_major(rm, ring_len):
    """Inverse of ring_region_major."""
    return np.ascontiguousarray(np.asarray(rm)[:, :ring_len].transpose(1, 0, 2))


def ring_to_reference(ring, step, horizon):
    """Inverse of ring_from_reference for the times [step - horizon + 1, step]."""
    ring = np.asarray(ring)
    RL, n, ncv = ring.shape
    out = np.zeros((horizon, ncv, n), dtype=ring.dtype)
    ts = np.arange(step - horizon + 1, step + 1)
    out[ts % horizon] = ring[ts % RL].transpose(0, 2, 1)
    return out


class Connectome:
    """Host CSR + packed gather edges of one weight / delay matrix pair."""

    def __init__(self, weights, idelays, ncvar):
        self.row_ptr, self.col, self.idelay, self.weight, self.nnz, self.min_delay = \
            _lib.sparse_layout(weights, idelays)
        self.n = int(np.asarray(weights).shape[0])
        self.horizon = int(np.asarray(idelays).max()) + 1
        self.ncvar = ncvar
        self.edges = _lib.pack_edges(self.col, self.idelay, self.weight, self.n, ncvar)
        self._packed = {ncvar: self.edges}

    def packed(self, ncvar):
        """Gather edges for a ring with `ncvar` floats per (slot, region)."""
        if ncvar not in self._packed:
            self._packed[ncvar] = _lib.pack_edges(self.col, self.idelay, self.weight, self.n, ncvar)
        return self._packed[ncvar]

    def slot_table(self, width):
        """The row kernel's gather slots for a ring of one float per (slot,
        region) whose length times n is a multiple of 32: (n, width, 2) int32
        [offset, weight bits], or None when no bank-conflict-free order fits."""
        key = ('slots', width)
        if key not in self._packed:
            self._packed[key] = bank_slot_table(self.row_ptr, self.col, self.idelay, self.weight, self.n, width,
                                                self.min_delay)
        return self._packed[key]


def _colour_warp(lane_edges, width):
    """Edge colouring of the bipartite multigraph lanes x banks (one edge per
    gather edge, from its lane to its bank) with at most `width` colours: each
    colour is a slot in which the lanes read distinct banks.  A bipartite
    multigraph of largest degree D has a D-colouring (Koenig's edge colouring
    theorem); it is built edge by edge, and when the free colours a (at the
    lane) and b (at the bank) differ the a/b alternating path from the bank is
    swapped first.  Returns {edge: colour} or None when D > width."""
    lane_c = [dict() for _ in lane_edges]         # lane -> colour -> (bank, edge)
    bank_c = [dict() for _ in range(32)]          # bank -> colour -> (lane, edge)
    load = np.zeros(32, dtype=np.int64)
    for es in lane_edges:
        for b, _ in es:
            load[b] += 1
    if max(max((len(es) for es in lane_edges), default=0), int(load.max())) > width:
        return None
    tabs = {'lane': lane_c, 'bank': bank_c}
    for lane, es in enumerate(lane_edges):
        for b, e in es:
            a = next(c for c in range(width) if c not in lane_c[lane])
            if a in bank_c[b]:
                c2 = next(c for c in range(width) if c not in bank_c[b])
                path, node, side, col = [], b, 'bank', a
                while col in tabs[side][node]:
                    other, eid = tabs[side][node][col]
                    path.append((side, node, other, eid, col))
                    node, side = other, ('lane' if side == 'bank' else 'bank')
                    col = c2 if col == a else a
                for side, node, other, eid, col in path:
                    oside = 'lane' if side == 'bank' else 'bank'
                    del tabs[side][node][col]
                    del tabs[oside][other][col]
                for side, node, other, eid, col in path:
                    oside = 'lane' if side == 'bank' else 'bank'
                    nc = c2 if col == a else a
                    tabs[side][node][nc] = (other, eid)
                    tabs[oside][other][nc] = (node, eid)
            lane_c[lane][a] = (b, e)
            bank_c[b][a] = (lane, e)
    return {e: c for lc in lane_c for c, (_, e) in lc.items()}


def bank_slot_table(row_ptr, col, idelay, weight, n, width, dmin):
    """Slot table for the row kernel (one float per ring entry): row r's
    edges placed in slots 0..width-1 so that in every slot the 32 rows of a
    warp read 32 different shared-memory banks.  The address of edge e at
    step s is base(s) - off_e with off_e = d_e n - col_e; when the ring's
    float count is a multiple of 32 its bank is bank(base) + (col_e - d_e n)
    mod 32 whether or not it wraps, so a per-warp schedule holds at every
    step.  A slot without an edge reads, with weight 0, one word of a bank no
    edge of that slot uses (one address for all such lanes: a broadcast), at
    least dmin steps back, where no thread of the window writes."""
    off = idelay.astype(np.int64) * n - col.astype(np.int64)
    bank = (-off) % 32
    wbits = np.asarray(weight, dtype=np.float32).view(np.int32)
    table = np.zeros((n, width, 2), dtype=np.int32)
    for w0 in range(0, n, 32):
        rows = range(w0, min(n, w0 + 32))
        lane_edges = [[(int(bank[e]), e) for e in range(row_ptr[r], row_ptr[r + 1])] for r in rows]
        colour = _colour_warp(lane_edges, width)
        if colour is None:
            return None
        used = np.zeros((width, 32), dtype=bool)
        filled = np.zeros((len(rows), width), dtype=bool)
        for li, r in enumerate(rows):
            for b, e in lane_edges[li]:
                k = colour[e]
                assert not used[k, b] and not filled[li, k]
                used[k, b] = filled[li, k] = True
                table[r, k] = (off[e], wbits[e])
        for k in range(width):
            free = int(np.flatnonzero(~used[k])[0]) if not used[k].all() else 0
            for li, r in enumerate(rows):
                if not filled[li, k]:
                    table[r, k] = (dmin * n + (-free - dmin * n) % 32, 0)
    return table


class InstanceSpec:
    """One simulation instance.

    ring0: (H, ncvar, n) history as the reference lays it out, valid at step0;
    state0: (nsv, n); params: (nparam, n) float32; cfun: coupling parameters;
    sigma: (nintvar, n) sqrt(dt) sqrt(2 nsig) or None; n_steps: steps to run;
    raw: keep every step; tavg_istep / bold (dict istep, ii, hrf, k1v0): monitors.
    noise_fed: (n_steps, nintvar, n) standard normals or None.
    stim: region stimulus or None: dict with 'temporal' (the pattern of steps
    step0 + 1 ..., at least n_steps values), 'weight' (n,) spatial pattern and
    'vars' (indices of the state variables it drives, the model's stvar).
    """

    def __init__(self, conn, ring0, state0, params, cfun, n_steps, step0=0, sigma=None, noise_fed=None,
                 seed=42, stream=0, raw=False, tavg_istep=0, bold=None, sub_istep=0, stim=None, aff_istep=0,
                 proj_istep=0):
        self.conn = conn
        self.ring0 = ring0
        self.state0 = state0
        self.params = params
        self.cfun = cfun
        self.n_steps = int(n_steps)
        self.step0 = int(step0)
        self.sigma = sigma
        self.noise_fed = noise_fed
        self.seed = int(seed)
        self.stream = int(stream)
        self.raw = raw
        self.tavg_istep = int(tavg_istep)
        self.bold = bold
        self.sub_istep = int(sub_istep)  # SubSample / GlobalAverage / SpatialAverage period in steps (0: none)
        if stim is not None:
            t = np.asarray(stim['temporal'], dtype=np.float32).reshape(-1)
            if t.size < self.n_steps:
                raise IndexError('stimulus temporal pattern has %d samples for %d steps' % (t.size, self.n_steps))
            w = np.asarray(stim['weight'], dtype=np.float32).reshape(-1)
            if w.size != conn.n:
                raise ValueError('stimulus weight has %d values for %d regions' % (w.size, conn.n))
            mask = 0
            for v in np.asarray(stim['vars'], dtype=np.int64).reshape(-1):
                mask |= 1 << int(v)
            stim = dict(temporal=np.ascontiguousarray(t[:self.n_steps]), weight=np.ascontiguousarray(w), mask=mask)
        self.stim = stim
        self.aff_istep = int(aff_istep)  # AfferentCoupling period in steps (1: every step; 0: none)
        self.proj_istep = int(proj_istep)  # projection-monitor period in steps (0: none)
        # monitor accumulators carried over from a previous run of the same
        # simulation: dict with 'tavg_acc' (nvoi, n), 'bold_acc' (nvoi, n),
        # 'bold_stock' (stock_len, nvoi, n); None starts them at zero
        self.acc0 = None


class Batch:
    def __init__(self, model_id, cfun_id, scheme_id, noise_kind, dt, voi_codes, specs, device=None,
                 sync_every=None, ring_in_smem=None, gather='auto', lanes=1, allocate=True, cluster='auto',
                 region_rings=True, groups='auto', block_steps='auto'):
        self.lib = _lib.load()
        self.device = torch.device(device if device is not None else 'cuda')
        self.model_id, self.cfun_id, self.scheme_id, self.noise_kind = model_id, cfun_id, scheme_id, noise_kind
        self.dt = float(dt)
        self.voi = list(voi_codes)
        self.nvoi = len(self.voi)
        self.specs = list(specs)
        self.ncvar, self.nsv, self.nint, self.nobs, self.nparam = _lib.model_dims(model_id)
        if not self.specs:
            raise ValueError('empty batch')
        # barrier interval: no read of a time written inside a window (K <= d_min + 1)
        # the distinct connectomes (a sweep shares one): the planning below depends on them only
        self._uconns = list({id(s.conn): s.conn for s in self.specs}.values())
        dmin = min(c.min_delay for c in self._uconns)
        K = dmin + 1 if sync_every is None else int(sync_every)
        K = max(1, min(K, dmin + 1))
        self.max_n = max(c.n for c in self._uconns)
        self.max_degree = max(int(np.diff(c.row_ptr).max()) if c.nnz else 0 for c in self._uconns)
        if self.max_n > _lib.MAX_REGIONS:
            raise ValueError('%d regions exceed this build (%d)' % (self.max_n, _lib.MAX_REGIONS))
        hmax = max(c.horizon for c in self._uconns)
        # AfferentCoupling is written by the row kernel only
        self.afferent = any(s.aff_istep for s in self.specs)
        # launch.extras: without a stimulus or AfferentCoupling the row kernel runs its lean build
        self.extras = ((1 if any(s.stim is not None for s in self.specs) else 0) | (2 if self.afferent else 0)
                       | (4 if any(s.proj_istep for s in self.specs) else 0))
        self.lanes = self._choose_lanes(lanes, gather)
        V = self.lanes
        # SigmoidalJansenRit with the row / cluster kernels gathers from a ring of pre-applied sigmoid
        # values, one float per (slot, region)
        self.sigma = (self.cfun_id == _lib.CFUN_IDS['SigmoidalJansenRit'] and V == 1 and gather != 'edge')
        self.ncvar_gather = 1 if self.sigma else self.ncvar
        # stage rings in shared memory when the largest fits, shrinking K if that makes it fit
        smem_ok = self.max_n <= 256 and V == 1
        ncg = self.ncvar if gather == 'edge' else self.ncvar_gather
        self.generic = self.cfun_id in _lib.CFUN_GENERIC
        # the prefetching row kernel (below) stages RING_GUARD mirrored slots past each ring
        pipe = (gather not in ('edge', 'split') and V == 1 and dmin >= 1
                and self.cfun_id != _lib.CFUN_IDS['Difference'] and self.model_id != _lib.MODEL_IDS['Sum']
                and not self.generic)
        guard = _lib.RING_GUARD if pipe else 0
        if ring_in_smem is None:
            ring_in_smem = smem_ok
        if ring_in_smem:
            while K > 1 and self.lib.tvbk_ring_smem_bytes(self.max_n, ncg * V, hmax + K + guard) == 0:
                K -= 1
            if not smem_ok or self.lib.tvbk_ring_smem_bytes(self.max_n, ncg * V, hmax + K + guard) == 0:
                ring_in_smem = False
                K = dmin + 1 if sync_every is None else max(1, min(int(sync_every), dmin + 1))
        self.sync_every = K
        self.ring_in_smem = bool(ring_in_smem)
        self.edges_per_thread, self.block_threads = 0, 0
        self.prefetch = 0
        if gather not in ('auto', 'row', 'edge', 'split'):
            raise ValueError("gather must be 'auto', 'row', 'edge' or 'split'")
        if self.generic and (gather in ('edge', 'split') or V != 1):
            raise ValueError('Sigmoidal, HyperbolicTangent and Kuramoto run on the row gather, one instance '
                             'per CTA')
        if self.afferent and (gather in ('edge', 'split') or V != 1):
            raise ValueError('AfferentCoupling monitors run on the row gather, one instance per CTA')
        if gather != 'edge' and dmin >= 1 and self.cfun_id != _lib.CFUN_IDS['Difference'] \
                and self.model_id != _lib.MODEL_IDS['Sum'] and not self.generic:
            # row kernel with the next step's gather issued ahead: barrier interval K <= d_min
            self.prefetch = 1
            self.sync_every = min(self.sync_every, dmin)
        if gather == 'split':
            # separate gather and update warps (the prefetch overlap across warps)
            ring_b = -(-(hmax + self.sync_every) * self.max_n * self.ncvar_gather * 4 // 16) * 16
            if not (self.prefetch and self.ring_in_smem and V == 1 and self.max_degree <= 64
                    and ring_b + 2 * self.max_n * self.ncvar * 4 <= 227 * 1024):
                raise ValueError('the split gather needs rings in shared memory, delays >= 1, Linear or '
                                 'SigmoidalJansenRit coupling and row degrees <= 64')
            self.prefetch = 2
        if gather == 'edge' and V == 1:
            ep = self._choose_edge_parallel(dmin, hmax)
            if ep is not None:
                self.edges_per_thread, self.block_threads, self.sync_every = ep
            elif gather == 'edge':
                raise ValueError('the edge-parallel gather does not apply to this batch')
        # mirrored guard slots past a shared-memory ring (prefetch 1; the split kernel has none)
        self.guard = _lib.RING_GUARD if (self.prefetch == 1 and self.ring_in_smem and V == 1) else 0
        # an explicit cluster above 16 CTAs per instance needs cooperative groups
        self._cluster_max = 256 if (groups is not False and groups not in (0, None, 'off', 'auto')) else 16
        self.cluster, self.cluster_edges = self._choose_cluster(cluster)
        self.ring_layout = 0
        self.block_steps = 0
        if self.cluster:
            # edge runs for the cluster CTAs when they fit; with them Difference also prefetches
            runs = self._choose_cluster_runs(dmin)
            if runs:
                self.edges_per_thread = runs
                if dmin >= 1 and self.cfun_id == _lib.CFUN_IDS['Difference']:
                    self.prefetch = 1
                    self.sync_every = min(self.sync_every, dmin)
                # blocked runs on region-major rings: B = 4 or 8 steps per gather, K a multiple of B with
                # K <= d_min - B + 1 (d_min >= 2B - 1); eight-step blocks for the lean kernel only
                K0 = self.sync_every
                K4 = (min(K0, dmin - 3) // 4) * 4
                K8 = (min(K0, dmin - 7) // 8) * 8
                if (region_rings and self.prefetch == 1 and K4 >= 4 and self.ncvar <= 2
                        and self.cfun_id in (_lib.CFUN_IDS['Linear'], _lib.CFUN_IDS['Difference'],
                                             _lib.CFUN_IDS['SigmoidalJansenRit'])
                        and self._cluster_smem(blocks=4) <= self.CLUSTER_SMEM):
                    self.ring_layout = 1
                    self.block_steps, self.sync_every = 4, K4
                    if (block_steps in ('auto', 8) and K8 >= 8 and self.extras == 0
                            and self._cluster_smem(blocks=8) <= self.CLUSTER_SMEM):
                        self.block_steps, self.sync_every = 8, K8
                    elif block_steps == 8:
                        raise ValueError('eight-step blocks need a smallest delay of 15 steps, no stimulus, '
                                         'AfferentCoupling or projection stream, and the partials in shared memory')
        self.groups = 0
        if self.ring_layout == 1:
            self._choose_groups(groups, cluster, dmin)
            if self.groups and block_steps == 'auto' and self.block_steps == 8:
                # measured: eight-step blocks gain on thread-block clusters (+18 % on the large-network batch)
                # but not under the group launch (-2 %), whose barrier interval they shorten
                self.block_steps, self.sync_every = 4, K4
        if self.cluster > 16 and not self.groups:
            raise ValueError('%d CTAs per instance need cooperative groups, which need region-major rings '
                             '(Linear, Difference or SigmoidalJansenRit coupling, ncvar <= 2, smallest delay >= 7 steps)' % self.cluster)
        self.slot_width, self._ring_len = self._choose_slots()
        self._plan()
        self.allocated = False
        if allocate:
            self.allocate()

    def allocate(self):
        """Allocate the device arenas and upload the inputs (once)."""
        if not self.allocated:
            self._build()
            self.allocated = True
        return self

    @property
    def nbytes(self):
        """Device bytes of this batch's arenas (inputs, accumulators, outputs)."""
        return self.init.size + self.zero.size + self.out.size

    def _choose_lanes(self, lanes, gather):
        """Instance groups: G = 8 / ncvar consecutive instances that share the
        connectome object, start step and length (a parameter sweep) run
        together, one thread per (region, instance), rings interleaved."""
        if lanes in (None, 1, '1'):
            return 1
        G = 8 // self.ncvar
        if lanes not in ('auto', G):
            raise ValueError('instance groups have 8 / ncvar = %d lanes' % G)
        specs = self.specs
        same = all(s.conn is specs[0].conn and s.step0 == specs[0].step0 and s.n_steps == specs[0].n_steps
                   for s in specs)
        threads = -(-self.max_n * G // 32) * 32
        smem = -(-self.max_n * self.max_degree * 8 // 16) * 16 + 2 * self.max_degree * self.ncvar * threads * 4
        ok = (same and gather != 'edge' and self.model_id != _lib.MODEL_IDS['Sum'] and threads <= 1024
              and self.cfun_id not in _lib.CFUN_GENERIC and not self.afferent
              and smem <= 227 * 1024 and len(specs) % G == 0)
        if ok:
            return G
        if lanes != 'auto':
            raise ValueError('these instances cannot run as groups of %d' % G)
        return 1

    SM_SMEM = 228 * 1024       # shared memory of an SM
    CTA_RESERVED = 1024        # per-CTA shared memory the hardware reserves

    def _choose_slots(self):
        """Bank-conflict-free gather slots for the row kernel with rings in
        shared memory (one float per ring entry, 32..256 regions): the ring
        of each instance is lengthened to the next multiple of 32 / gcd(n, 32)
        slots (its float count then a multiple of 32), when that keeps the
        same number of CTAs per SM.  With guard slots (the prefetching row
        kernel) the barrier interval K may be lowered, down to 4, when a
        shorter padded ring plus its guard keeps more CTAs per SM resident.
        Returns (slot width or 0, ring length of a spec) and sets sync_every."""
        K0 = self.sync_every
        G = self.guard

        def plain(K):
            return lambda s: s.conn.horizon + K

        def padded(K):
            def f(s):
                m = 32 // math.gcd(s.conn.n, 32)
                return -(-(s.conn.horizon + K) // m) * m
            return f

        # ring lengths depend on a spec's horizon and size only: evaluate them once per distinct pair
        shapes = list({(s.conn.horizon, s.conn.n): s for s in self.specs}.values())

        def ctas(ring_len):
            b = (max(ring_len(s) for s in shapes) + G) * self.max_n * self.ncvar_gather * 4
            return 0 if b > 227 * 1024 else self.SM_SMEM // (b + self.CTA_RESERVED)

        if not (self.ring_in_smem and self.lanes == 1 and not self.edges_per_thread and self.prefetch != 2
                and self.ncvar_gather == 1 and not self.cluster and 0 < self.max_degree <= 64
                and all(s.conn.n >= 32 for s in self.specs)):
            return 0, plain(K0)
        width = 32 if self.max_degree <= 32 else 64
        cands = [K0] + (list(range(K0 - 1, 3, -1)) if G and K0 > 4 else [])
        (occ, K) = max((ctas(padded(K)), K) for K in cands)
        if occ == 0 or occ < ctas(plain(K0)):
            return 0, plain(K0)
        if any(c.slot_table(width) is None for c in self._uconns):
            return 0, plain(K0)
        self.sync_every = K
        return width, padded(K)

    CLUSTER_SMEM = 227 * 1024
    CLUSTER_MAX_ROWS = 480

    def _choose_cluster(self, cluster):
        """CTAs per instance (thread-block cluster) and the per-CTA edge
        allowance in shared memory.  'auto', for rings read in place and at
        least 64 regions: 16 CTAs per instance for up to 16 instances (their
        clusters run in waves when they outnumber the SMs, which also keeps
        each wave's rings closer to L2-sized), SMs // instances CTAs up to
        SMs / 2 instances, else one CTA per instance."""
        if cluster in (None, 0, 1, '0', '1'):
            return 0, 0
        able = (self.lanes == 1 and not self.ring_in_smem and not self.edges_per_thread
                and self.model_id != _lib.MODEL_IDS['Sum'] and not self.generic and not self.afferent)
        if cluster == 'auto':
            if not able or self.max_n < 64:
                return 0, 0
            sms = 148
            if self.device.type == 'cuda' and torch.cuda.is_available():
                sms = torch.cuda.get_device_properties(self.device).multi_processor_count
            ni = len(self.specs)
            C = 16 if ni <= 16 else sms // ni
            C = min(C, -(-self.max_n // 4))
            if C < 2:
                return 0, 0
        else:
            C = int(cluster)
            if not able or not 2 <= C <= self._cluster_max:
                raise ValueError('a cluster of 2..16 CTAs per instance (2..256 with groups=True) needs rings in '
                                 'place, the row gather and one instance per lane group')
        C = max(C, -(-self.max_n // self.CLUSTER_MAX_ROWS))
        R = -(-self.max_n // C)
        nacc = 1 if self.cfun_id == _lib.CFUN_IDS['SigmoidalJansenRit'] else self.ncvar
        head = -(-(R + 1) * 4 // 16) * 16 + -(-2 * R * nacc * 4 // 16) * 16
        emax = self._cluster_edges_for(C)
        return C, (emax if head + 8 * emax <= self.CLUSTER_SMEM else 0)

    CLUSTER_THREADS = 512
    CLUSTER_RUNS = (8, 16, 32)
    GROUP_SIZES = (8, 12, 16, 18, 20, 24, 32, 48, 64)

    def _sm_count(self):
        if self.device.type == 'cuda' and torch.cuda.is_available():
            return torch.cuda.get_device_properties(self.device).multi_processor_count
        return 148

    def _cluster_edges_for(self, C):
        """Largest edge count of one CTA's rows with C CTAs per instance."""
        R = -(-self.max_n // C)
        emax = 0
        for c in self._uconns:
            rp = c.row_ptr
            n = c.n
            for r in range(C):
                lo = min(n, r * R)
                hi = min(n, lo + R)
                emax = max(emax, int(rp[hi] - rp[lo]))
        return emax

    def _choose_groups(self, groups, cluster, dmin):
        """Cooperative groups (launch.groups) instead of thread-block clusters
        for blocked runs on region-major rings.  groups=True keeps the chosen
        CTAs per instance; 'auto' (with cluster='auto') picks C from
        GROUP_SIZES and G = min(SMs // C, instances) groups, minimising the
        longest-processing-time makespan of the instances' lengths on G groups
        times (1/C + 1/64): the gather of one step spreads over C CTAs, and a
        part of the step (the update warps, the barriers) does not shrink with
        C.  The device queue hands the instances out longest first, which is
        that schedule.  An int caps G.  False (or an explicit cluster with
        'auto') keeps thread-block clusters."""
        if groups is False or groups in (0, None, 'off') or (groups == 'auto' and cluster != 'auto'):
            return
        sms = self._sm_count()
        lengths = sorted((s.n_steps for s in self.specs), reverse=True)
        keep = (self.cluster, self.cluster_edges, self.edges_per_thread)

        def makespan(G):
            loads = [0] * G
            for L in lengths:
                i = loads.index(min(loads))
                loads[i] += L
            return max(loads)

        sizes = self.GROUP_SIZES if cluster == 'auto' else [self.cluster]
        cap = int(groups) if (isinstance(groups, int) and not isinstance(groups, bool)) else None
        best = None
        for C in sizes:
            G = min(sms // C, len(self.specs), cap or sms)
            if G < 1 or -(-self.max_n // C) > self.CLUSTER_MAX_ROWS:
                continue
            edges = self._cluster_edges_for(C)
            self.cluster, self.cluster_edges = C, edges
            runs = self._choose_cluster_runs(dmin)
            self.edges_per_thread = runs
            fits = runs and self._cluster_smem(blocks=self.block_steps) + 64 <= self.CLUSTER_SMEM
            self.cluster, self.cluster_edges, self.edges_per_thread = keep
            if not fits:
                continue
            est = makespan(G) * (1.0 / C + 1.0 / 64)
            if best is None or est < best[0] * (1 - 1e-9):
                best = (est, C, G, edges, runs)
        if best is None:
            return
        _, C, G, edges, runs = best
        self.cluster, self.cluster_edges, self.edges_per_thread, self.groups = C, edges, runs, G

    def _cluster_smem(self, blocks=0):
        """Shared memory of an edge-run cluster CTA: row pointers, the
        double-buffered partials (of a block of `blocks` steps for the blocked
        runs) and the CTA's edges with room for the interleaving."""
        R = -(-self.max_n // self.cluster)
        nacc = 1 if self.cfun_id == _lib.CFUN_IDS['SigmoidalJansenRit'] else self.ncvar
        parts = 2 * max(int(blocks), 1) * self.CLUSTER_THREADS * 2 * nacc * 4
        return -(-(R + 1) * 4 // 16) * 16 + -(-parts // 16) * 16 + 8 * (self.cluster_edges + max(self.CLUSTER_RUNS))

    def _choose_cluster_runs(self, dmin):
        """Edge-run length of the cluster kernel, or 0 for a warp per row: the
        smallest E of CLUSTER_RUNS whose runs cover every CTA's edges with the
        CTA's gather threads (512, less one update warp per 32 rows when the
        gather runs a step ahead) and that does not exceed the smallest
        non-zero row degree of any CTA (a run then holds at most two rows).
        Needs every CTA's edges in shared memory with the larger partials
        buffer of the run kernel."""
        if not self.cluster_edges:
            return 0
        C = self.cluster
        R = -(-self.max_n // C)
        if self._cluster_smem() > self.CLUSTER_SMEM:
            return 0
        ahead = dmin >= 1 and self.model_id != _lib.MODEL_IDS['Sum']
        need, cap = 1, 1 << 30
        for c in self._uconns:
            rp = np.asarray(c.row_ptr)
            deg = np.diff(rp)
            n = c.n
            for r in range(C):
                lo, hi = min(n, r * R), min(n, r * R + R)
                nr = hi - lo
                if nr == 0:
                    continue
                tg = self.CLUSTER_THREADS - (32 * -(-nr // 32) if ahead else 0)
                need = max(need, -(-int(rp[hi] - rp[lo]) // tg))
                d = deg[lo:hi]
                if (d > 0).any():
                    cap = min(cap, int(d[d > 0].min()))
        for E in self.CLUSTER_RUNS:
            if need <= E <= cap:
                return E
        return 0

    EP_SLOTS = (8, 12, 16, 24)

    def _choose_edge_parallel(self, dmin, hmax):
        """(edges per thread, CTA threads, barrier interval) of the edge-parallel
        gather, or None: needs rings in shared memory, a coupling whose pre()
        depends on the source only, and ceil(nnz / threads) <= the smallest
        non-zero row degree.  Picks the fewest padded edge slots, then the
        most threads."""
        if not self.ring_in_smem or self.cfun_id == _lib.CFUN_IDS['Difference']:
            return None
        K = 2 if dmin >= 1 else 1
        nacc = 1 if self.cfun_id == _lib.CFUN_IDS['SigmoidalJansenRit'] else self.ncvar
        need = []
        for c in self._uconns:
            if c.nnz == 0:
                return None
            deg = np.diff(c.row_ptr)
            need.append((c.nnz, int(deg[deg > 0].min())))
        best = None
        for T in range(((self.max_n + 31) // 32) * 32, 513, 32):
            ring = ((hmax + K) * self.max_n * self.ncvar + 3) // 4 * 4
            if (ring + 2 * T * 2 * nacc) * 4 > 227 * 1024:
                break
            for E in self.EP_SLOTS:
                if all(-(-nnz // T) <= min(E, mdeg) for nnz, mdeg in need):
                    key = (T * E, -T)
                    if best is None or key < best[0]:
                        best = (key, E, T)
                    break
        if best is None:
            return None
        return best[1], best[2], K

    # ------------------------------------------------------------------ build
    def _plan(self):
        """Arena layout and per-instance metadata (no device memory)."""
        specs, nvoi = self.specs, self.nvoi
        init, zero, outa = _Arena(), _Arena(), _Arena()
        # the rings first, one block: instances that start from the same history (a sweep) upload it once
        # and it is copied on the device
        self._ring_src = {}
        if self.lanes == 1:
            first = {}
            for k, s in enumerate(specs):
                RL = self._ring_len(s)
                slots = _lib.ring_region_stride(RL, self.ncvar) if self.ring_layout else RL
                init.add(('ring', k), slots * s.conn.n * self.ncvar * 4)
                key = (_array_key(s.ring0), s.step0, RL)
                self._ring_src[k] = first.setdefault(key, k)
        self._ring_block = init.size
        conns = {}
        for s in specs:
            if id(s.conn) not in conns:
                c = s.conn
                conns[id(s.conn)] = c
                init.add(('row_ptr', id(c)), c.row_ptr.nbytes)
                if self.slot_width:
                    init.add(('slots', id(c)), c.slot_table(self.slot_width).nbytes)
                init.add(('edges', id(c)), max(c.edges.nbytes, 8))
        hrfs = {}
        self.meta = []
        for k, s in enumerate(specs):
            n = s.conn.n
            RL = self._ring_len(s)
            m = dict(n=n, ring_len=RL)
            V = self.lanes
            if V > 1 and k % V == 0:
                init.add(('ring', k), V * RL * n * self.ncvar * 4)
            if self.sigma and not self.ring_in_smem:
                # region-major rings: the sigmoid ring too, one float per slot (filled by the kernel)
                zero.add(('pre_ring', k), (_lib.ring_region_stride(RL, 1) if self.ring_layout else RL) * n * 4)
            init.add(('state', k), self.nsv * n * 4)
            init.add(('params', k), max(self.nparam, 1) * n * 4)
            if s.stim is not None:
                init.add(('stim', k), max(s.n_steps, 1) * 4)
                init.add(('stim_w', k), n * 4)
            if s.sigma is not None:
                init.add(('sigma', k), self.nint * n * 4)
            acc_arena = init if s.acc0 is not None else zero
            if s.bold is not None:
                h = s.bold['hrf']
                if id(h) not in hrfs:
                    hrfs[id(h)] = h
                    init.add(('hrf', id(h)), h.nbytes)
                acc_arena.add(('bold_acc', k), nvoi * n * 8)
                acc_arena.add(('bold_stock', k), len(h) * nvoi * n * 8)
            if s.tavg_istep:
                acc_arena.add(('tavg_acc', k), nvoi * n * 4)
            if s.aff_istep:
                acc_arena.add(('aff_acc', k), self.ncvar * n * 4)
            if s.proj_istep:
                acc_arena.add(('proj_acc', k), nvoi * n * 4)
            # outputs
            s1 = s.step0 + s.n_steps
            if s.raw:
                m['raw_rows'] = s.n_steps
                outa.add(('raw', k), s.n_steps * nvoi * n * 4)
            if s.tavg_istep:
                m['tavg_rows'] = s1 // s.tavg_istep - s.step0 // s.tavg_istep
                outa.add(('tavg', k), max(m['tavg_rows'], 1) * nvoi * n * 4)
            if s.bold is not None:
                bi = s.bold['istep']
                m['bold_rows'] = s1 // bi - s.step0 // bi
                outa.add(('bold', k), max(m['bold_rows'], 1) * nvoi * n * 8)
            if s.sub_istep:
                m['sub_rows'] = s1 // s.sub_istep - s.step0 // s.sub_istep
                outa.add(('sub', k), max(m['sub_rows'], 1) * nvoi * n * 4)
            if s.aff_istep:
                m['aff_rows'] = s1 // s.aff_istep - s.step0 // s.aff_istep
                outa.add(('aff', k), max(m['aff_rows'], 1) * self.ncvar * n * 4)
            if s.proj_istep:
                m['proj_rows'] = s1 // s.proj_istep - s.step0 // s.proj_istep
                outa.add(('proj', k), max(m['proj_rows'], 1) * nvoi * n * 4)
            self.meta.append(m)
        init.add(('insts',), len(specs) * _lib.INST_DTYPE.itemsize)
        zero.add(('status',), len(specs) * 4)
        self.init, self.zero, self.out = init, zero, outa
        self._conns, self._hrfs = conns, hrfs

    def _build(self):
        specs = self.specs
        init, zero, outa = self.init, self.zero, self.out
        conns, hrfs = self._conns, self._hrfs
        dev = self.device
        self.init_buf = torch.empty(max(init.size, 1), dtype=torch.uint8, device=dev)
        self.zero_buf = torch.zeros(max(zero.size, 1), dtype=torch.uint8, device=dev)
        self.out_buf = torch.zeros(max(outa.size, 1), dtype=torch.uint8, device=dev)
        ib, zb, ob = self.init_buf.data_ptr(), self.zero_buf.data_ptr(), self.out_buf.data_ptr()

        # host staging of everything after the ring block; the rings themselves are uploaded once per
        # distinct history
        R0 = self._ring_block
        stage = np.zeros(max(init.size - R0, 1), dtype=np.uint8)
        ring_up = {}

        def put(key, arr):
            off, nb = init.regions[key]
            a = np.ascontiguousarray(arr).view(np.uint8).reshape(-1)
            if off < R0:
                ring_up[key] = a
            else:
                stage[off - R0:off - R0 + a.size] = a
            return ib + off

        def zaddr(key):
            if key in outa.regions:
                return ob + outa.regions[key][0]
            if key in zero.regions:
                return zb + zero.regions[key][0]
            if key in init.regions:
                return ib + init.regions[key][0]
            return 0

        cptr = {}
        for key, c in conns.items():
            cptr[key] = (put(('row_ptr', key), c.row_ptr), put(('edges', key), c.packed(self.ncvar_gather))
                         if c.nnz else ib + init.regions[('edges', key)][0])
        hptr = {key: put(('hrf', key), np.asarray(h, dtype=np.float64)) for key, h in hrfs.items()}
        sptr = {key: put(('slots', key), c.slot_table(self.slot_width)) for key, c in conns.items()} \
            if self.slot_width else {}

        # descriptor fields per instance as dicts, written into the structured array column by column
        recs = [dict() for _ in specs]
        self._fed = []
        for k, s in enumerate(specs):
            m = self.meta[k]
            n, RL = m['n'], m['ring_len']
            d = recs[k]
            d['row_ptr'], d['edges'] = cptr[id(s.conn)]
            if self.slot_width:
                d['slots'] = sptr[id(s.conn)]
                d['slot_width'] = self.slot_width
            V = self.lanes
            if V == 1:
                src = self._ring_src[k]
                if src == k:
                    r0 = ring_from_reference(s.ring0, s.step0, RL)
                    d['ring'] = put(('ring', k), ring_region_major(r0, self.ncvar) if self.ring_layout else r0)
                else:
                    d['ring'] = ib + init.regions[('ring', k)][0]
            elif k % V == 0:
                group = [ring_from_reference(specs[k + v].ring0, specs[k + v].step0, RL) for v in range(V)]
                d['ring'] = put(('ring', k), np.stack(group, axis=-1))  # [RL][n][ncvar][V]
            else:
                d['ring'] = recs[k - k % V]['ring']
            d['pre_ring'] = zaddr(('pre_ring', k))
            d['state'] = put(('state', k), np.asarray(s.state0, dtype=np.float32))
            params = np.asarray(s.params, dtype=np.float32)
            if params.size == 0:
                params = np.zeros((1, n), dtype=np.float32)
            d['params'] = put(('params', k), params)
            d['noise_sigma'] = put(('sigma', k), np.asarray(s.sigma, dtype=np.float32)) if s.sigma is not None else 0
            if s.noise_fed is not None:
                fed = s.noise_fed
                if not isinstance(fed, torch.Tensor):
                    fed = torch.from_numpy(np.ascontiguousarray(fed, dtype=np.float32))
                fed = fed.to(dev, dtype=torch.float32).contiguous()
                self._fed.append(fed)
                d['noise_fed'] = fed.data_ptr()
            if s.stim is not None:
                if s.stim['mask'] >> self.nsv:
                    raise ValueError('stimulus drives a state variable the model does not have')
                d['stim'] = put(('stim', k), s.stim['temporal'])
                d['stim_weight'] = put(('stim_w', k), s.stim['weight'])
                d['stim_vars'] = s.stim['mask']
                d['stim_base'] = s.step0
            if s.acc0 is not None:
                for key, dtype in (('tavg_acc', np.float32), ('bold_acc', np.float64), ('bold_stock', np.float64),
                                   ('aff_acc', np.float32), ('proj_acc', np.float32)):
                    if (key, k) in init.regions and s.acc0.get(key) is not None:
                        put((key, k), np.asarray(s.acc0[key], dtype=dtype))
            d['raw'] = zaddr(('raw', k))
            d['sub'] = zaddr(('sub', k))
            if s.aff_istep:
                d['aff'] = zaddr(('aff', k))
                d['aff_acc'] = zaddr(('aff_acc', k))
                d['aff_istep'] = s.aff_istep
                d['aff_base'] = s.step0 // s.aff_istep
            if s.proj_istep:
                d['proj'] = zaddr(('proj', k))
                d['proj_acc'] = zaddr(('proj_acc', k))
                d['proj_istep'] = s.proj_istep
                d['proj_base'] = s.step0 // s.proj_istep
            if s.sub_istep:
                d['sub_istep'] = s.sub_istep
                d['sub_base'] = s.step0 // s.sub_istep
            d['tavg'] = zaddr(('tavg', k))
            d['tavg_acc'] = zaddr(('tavg_acc', k))
            d['bold'] = zaddr(('bold', k))
            d['bold_acc'] = zaddr(('bold_acc', k))
            d['bold_stock'] = zaddr(('bold_stock', k))
            d['step'] = s.step0
            d['step_end'] = s.step0 + s.n_steps
            d['raw_base'] = s.step0
            d['fed_base'] = s.step0
            d['n'], d['nnz'], d['horizon'], d['ring_len'] = n, s.conn.nnz, s.conn.horizon, RL
            if s.tavg_istep:
                d['tavg_istep'] = s.tavg_istep
                d['tavg_base'] = s.step0 // s.tavg_istep
            if s.bold is not None:
                d['hrf'] = hptr[id(s.bold['hrf'])]
                d['bold_istep'] = s.bold['istep']
                d['bold_ii'] = s.bold['ii']
                d['stock_len'] = len(s.bold['hrf'])
                d['bold_base'] = s.step0 // s.bold['istep']
                d['bold_k1v0'] = s.bold['k1v0']
            cf = list(s.cfun) + [0.0] * (6 - len(s.cfun))
            d['cfun'] = cf
            d['seed'] = s.seed & 0xFFFFFFFF
            d['stream'] = s.stream & 0xFFFFFFFF
        insts = np.zeros(len(specs), dtype=_lib.INST_DTYPE)
        for name in _lib.INST_DTYPE.names:
            if any(name in r for r in recs):
                blank = np.zeros((), dtype=_lib.INST_DTYPE[name])
                insts[name] = [r.get(name, blank) for r in recs]
        self.insts_host = insts
        self.insts_ptr = put(('insts',), insts)
        self.status_ptr = zaddr(('status',))
        if init.size > R0:
            self.init_buf[R0:init.size].copy_(torch.from_numpy(stage[:init.size - R0]))
        self._upload_rings(ring_up)
        self.steps_done = 0
        self.max_total = max(s.n_steps for s in specs)
        self._longest_first = None
        lengths = np.array([s.n_steps for s in specs])
        if self.cluster and len(set(lengths.tolist())) > 1:
            order = np.argsort(-lengths, kind='stable').astype(np.int32)
            self._longest_first = torch.as_tensor(order, device=dev)
        # cooperative groups: queue head, abort flag, per-group barrier counters and claims (zeroed by the
        # library before each launch)
        self._group_sync = (torch.zeros(_lib.group_sync_words(self.groups), dtype=torch.int32, device=dev)
                            if self.groups else None)

    def _upload_rings(self, ring_up):
        """Host-to-device copy of each distinct initial ring, then device copies
        to the instances that share it (one broadcast copy when the regions
        are evenly spaced)."""
        self._h2d_ring_bytes = 0
        groups = {}
        for k, src in self._ring_src.items():
            groups.setdefault(src, []).append(k)
        if groups and len(groups) == len(self._ring_src):
            # every instance has its own history: one staged copy of the whole ring block
            R0 = self._ring_block
            stage = np.zeros(R0, dtype=np.uint8)
            for (_, k), a in ring_up.items():
                off = self.init.regions[('ring', k)][0]
                stage[off:off + a.size] = a
            self.init_buf[:R0].copy_(torch.from_numpy(stage))
            self._h2d_ring_bytes = R0
            return
        for src, ks in groups.items():
            off, nb = self.init.regions[('ring', src)]
            a = ring_up[('ring', src)]
            self.init_buf[off:off + nb].copy_(torch.from_numpy(a))
            self._h2d_ring_bytes += nb
            dst = [self.init.regions[('ring', k)][0] for k in ks if k != src]
            if not dst:
                continue
            steps = np.diff(dst)
            if len(dst) > 1 and (steps == steps[0]).all() and steps[0] >= nb:
                view = self.init_buf[dst[0]:dst[-1] + nb].as_strided((len(dst), nb), (int(steps[0]), 1))
                view.copy_(self.init_buf[off:off + nb].expand(len(dst), nb))
            else:
                for d in dst:
                    self.init_buf[d:d + nb].copy_(self.init_buf[off:off + nb])

    # ------------------------------------------------------------------ reset
    def snapshot(self):
        """Keep a device copy of the uploaded inputs so that reset() can restart
        the batch from its initial state without a host transfer."""
        self._pristine = self.init_buf.clone()

    def reset(self):
        """Restart every instance from its initial state (device-to-device)."""
        self.init_buf.copy_(self._pristine)
        self.zero_buf.zero_()
        self.out_buf.zero_()
        self.steps_done = 0

    @property
    def h2d_bytes(self):
        return (self.init.size - self._ring_block + getattr(self, '_h2d_ring_bytes', 0)
                + sum(int(f.numel()) * 4 for f in self._fed))

    @property
    def d2h_bytes(self):
        return self.out.size

    # -------------------------------------------------------------------- run
    def launch_struct(self, max_steps):
        L = _lib.Launch()
        L.insts = self.insts_ptr
        L.status = self.status_ptr
        L.n_inst = len(self.specs)
        L.model, L.cfun, L.scheme, L.noise = self.model_id, self.cfun_id, self.scheme_id, self.noise_kind
        L.nvoi = self.nvoi
        for v, code in enumerate(self.voi):
            L.voi[v] = code
        L.max_n = self.max_n
        L.max_ring_len = max(m['ring_len'] for m in self.meta)
        L.sync_every = self.sync_every
        L.ring_in_smem = 1 if self.ring_in_smem else 0
        L.max_degree = self.max_degree
        L.edges_per_thread = self.edges_per_thread
        L.block_threads = self.block_threads
        L.lanes = self.lanes
        L.cluster = self.cluster
        L.cluster_edges = self.cluster_edges
        L.ring_layout = self.ring_layout
        L.block_steps = self.block_steps
        L.groups = self.groups
        L.group_sync = self._group_sync.data_ptr() if self.groups else None
        L.extras = self.extras
        L.prefetch = self.prefetch
        L.max_steps = int(max_steps)
        L.dt = self.dt
        if self.cluster and getattr(self, "_longest_first", None) is not None:
            # clusters dispatch in launch order (groups take the queue in this order): the longest instances
            # start first, so that the batch's last steps do not run one long instance alone
            L.inst_order = self._longest_first.data_ptr()
        return L

    def occupancy(self):
        """Resident CTAs per SM of the row kernel variant this batch launches
        (0 for the other kernels)."""
        if self.lanes > 1 or self.cluster or self.edges_per_thread or self.prefetch == 2:
            return 0
        L = self.launch_struct(1)
        occ = ctypes.c_int32(0)
        L.occupancy = ctypes.addressof(occ)
        st = torch.cuda.current_stream(self.device)
        _lib.check(self.lib.tvbk_sim_run(ctypes.byref(L), ctypes.c_void_p(st.cuda_stream)))
        return int(occ.value)

    WAVE_MIN_CHUNK = 2000     # steps: a launch's ring stage-in / write-back stays negligible
    WAVE_MAX_CHUNKS = 64

    def _wave_plan(self, left):
        """Round-robin windows of exactly one wave of resident CTAs, for a batch
        of more instances than one wave that is not a whole number of waves
        (one launch would leave its last wave partly empty): each instance runs
        in C chunks and every launch takes the next R instances of the cyclic
        instance order, so all launches but possibly the last are full waves.
        Returns (R, C, chunk steps, launches) or None."""
        specs = self.specs
        if len({s.n_steps for s in specs}) != 1 or left <= 0 or self.device.type != 'cuda':
            return None
        key = ('wave_plan', left)
        if getattr(self, '_wave_key', None) == key:
            return self._wave_cached
        self._wave_key, self._wave_cached = key, self._make_wave_plan(left)
        return self._wave_cached

    def _make_wave_plan(self, left):
        specs = self.specs
        occ = self.occupancy()
        if occ <= 0:
            return None
        R = occ * torch.cuda.get_device_properties(self.device).multi_processor_count
        N = len(specs)
        if N <= R or N % R == 0:
            return None
        best = None
        for C in range(2, self.WAVE_MAX_CHUNKS + 1):
            chunk = -(-left // C)
            if chunk < self.WAVE_MIN_CHUNK:
                break
            launches = -(-N * C // R)
            eff = N * C / (launches * R)
            if best is None or eff > best[0] + 1e-9:
                best = (eff, C, chunk, launches)
            if eff >= 0.995:
                break
        one = N / (-(-N // R) * R)          # the fill of one launch over all instances
        if best is None or best[0] <= one:
            return None
        return R, best[1], best[2], best[3]

    def run(self, n_steps=None, chunk=None, stream=None, graph=False, waves=True):
        """Advance every instance by up to n_steps (default: to its end) in
        launches of at most `chunk` steps.

        graph=True: the chunk launches are recorded once into a CUDA graph of
        up to `graph_launches` launches (the kernel reads each instance's step
        from its device descriptor, so replaying the same launches continues
        the run) and the graph is replayed; a remainder runs eagerly.

        waves=True with no chunk given: a batch of more instances than fit at
        once, not a whole number of waves, runs as launches of exactly one wave
        each over a cyclic instance order (see _wave_plan); the same steps,
        without the last wave's idle SMs."""
        left = self.max_total - self.steps_done if n_steps is None else int(n_steps)
        st = torch.cuda.current_stream(self.device) if stream is None else stream
        plan = self._wave_plan(left) if (waves and chunk is None and not graph) else None
        if plan is not None:
            R, C, wchunk, launches = plan
            N = len(self.specs)
            if getattr(self, '_order_dev', None) is None:
                with torch.cuda.stream(st):
                    self._order_dev = torch.as_tensor(np.tile(np.arange(N, dtype=np.int32), 2), device=self.device)
            base = self._order_dev.data_ptr()
            for j in range(launches):
                start = (j * R) % N
                L = self.launch_struct(wchunk)
                L.inst_order = base + 4 * start
                L.n_inst = min(R, N * C - j * R)
                _lib.check(self.lib.tvbk_sim_run(ctypes.byref(L), ctypes.c_void_p(st.cuda_stream)))
            self.steps_done += left
            self.last_launches = launches
            return
        chunk = left if chunk is None else int(chunk)
        self.last_launches = 0
        if graph and chunk > 0 and left >= 2 * chunk:
            reps = left // chunk
            g = self._chunk_graph(chunk, min(reps, self.graph_launches), st)
            per = self._graph_launches
            with torch.cuda.stream(st):
                for _ in range(reps // per):
                    g.replay()
            done = (reps // per) * per * chunk
            left -= done
            self.steps_done += done
            self.last_launches += (reps // per) * per
        while left > 0:
            k = min(chunk, left)
            L = self.launch_struct(k)
            _lib.check(self.lib.tvbk_sim_run(ctypes.byref(L), ctypes.c_void_p(st.cuda_stream)))
            left -= k
            self.steps_done += k
            self.last_launches += 1

    graph_launches = 64

    def _chunk_graph(self, chunk, launches, st):
        """CUDA graph of `launches` chunk launches of `chunk` steps (cached)."""
        key = (chunk, launches)
        if getattr(self, '_graph_key', None) == key:
            return self._graph
        L = self.launch_struct(chunk)
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(device=self.device)
        cap.wait_stream(st)
        with torch.cuda.graph(g, stream=cap, capture_error_mode='relaxed'):
            for _ in range(launches):
                _lib.check(self.lib.tvbk_sim_run(ctypes.byref(L), ctypes.c_void_p(cap.cuda_stream)))
        st.wait_stream(cap)
        self._graph, self._graph_key, self._graph_launches = g, key, launches
        return g

    # ---------------------------------------------------------------- outputs
    def _zview(self, key, dtype, shape):
        off, nb = self.zero.regions[key]
        t = self.zero_buf[off:off + nb].view(dtype)
        return t[:int(np.prod(shape))].view(*shape)

    def _oview(self, key, dtype, shape):
        off, nb = self.out.regions[key]
        t = self.out_buf[off:off + nb].view(dtype)
        return t[:int(np.prod(shape))].view(*shape)

    def _iview(self, key, dtype, shape):
        off, nb = self.init.regions[key]
        t = self.init_buf[off:off + nb].view(dtype)
        return t[:int(np.prod(shape))].view(*shape)

    def outputs_device(self, k):
        """Device tensors of instance k's outputs: raw (T, nvoi, n) f32,
        tavg (T, nvoi, n) f32, bold (T, nvoi, n) f64."""
        m, nvoi = self.meta[k], self.nvoi
        out = {}
        if 'raw_rows' in m:
            out['raw'] = self._oview(('raw', k), torch.float32, (m['raw_rows'], nvoi, m['n']))
        if 'tavg_rows' in m:
            out['tavg'] = self._oview(('tavg', k), torch.float32, (m['tavg_rows'], nvoi, m['n']))
        if 'bold_rows' in m:
            out['bold'] = self._oview(('bold', k), torch.float64, (m['bold_rows'], nvoi, m['n']))
        if 'sub_rows' in m:
            out['sub'] = self._oview(('sub', k), torch.float32, (m['sub_rows'], nvoi, m['n']))
        if 'aff_rows' in m:
            out['aff'] = self._oview(('aff', k), torch.float32, (m['aff_rows'], self.ncvar, m['n']))
        if 'proj_rows' in m:
            out['proj'] = self._oview(('proj', k), torch.float32, (m['proj_rows'], nvoi, m['n']))
        return out

    def outputs_host(self):
        """All outputs of all instances as numpy arrays, from one device-to-host
        copy into pinned memory."""
        host = torch.empty(self.out_buf.numel(), dtype=torch.uint8, pin_memory=True)
        host.copy_(self.out_buf, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return self.outputs_from_bytes(host.numpy())

    def stacked_output(self, key, dtype=torch.float64):
        """Device view (I, T, nvoi, n) of one output of every instance without a
        copy when the instances' regions are evenly spaced and equally long,
        else a stacked copy."""
        rows = key + '_rows'
        metas = self.meta
        if not all(rows in m for m in metas) or len({m[rows] for m in metas}) != 1 \
                or len({m['n'] for m in metas}) != 1:
            return torch.stack([self.outputs_device(i)[key] for i in range(len(metas))])
        T, n = metas[0][rows], metas[0]['n']
        nv = self.ncvar if key == 'aff' else self.nvoi
        item = torch.empty((), dtype=dtype).element_size()
        offs = np.array([self.out.regions[(key, i)][0] for i in range(len(metas))])
        steps = np.diff(offs)
        if len(offs) > 1 and not ((steps == steps[0]).all() and steps[0] % item == 0 and offs[0] % item == 0):
            return torch.stack([self.outputs_device(i)[key] for i in range(len(metas))])
        stride = int(steps[0]) // item if len(offs) > 1 else T * nv * n
        base = self.out_buf[:self.out_buf.numel() // item * item].view(dtype)
        return base.as_strided((len(metas), T, nv, n), (stride, nv * n, n, 1), int(offs[0]) // item)

    def outputs_from_bytes(self, host):
        """Per-instance output arrays from a host copy (uint8 array) of the output arena."""
        res = []
        for k, m in enumerate(self.meta):
            o = {}
            nvoi, n = self.nvoi, m['n']
            for key, dt, rows in (('raw', np.float32, 'raw_rows'), ('tavg', np.float32, 'tavg_rows'),
                                  ('bold', np.float64, 'bold_rows'), ('sub', np.float32, 'sub_rows'),
                                  ('aff', np.float32, 'aff_rows'), ('proj', np.float32, 'proj_rows')):
                if rows in m:
                    off, nb = self.out.regions[(key, k)]
                    nv = self.ncvar if key == 'aff' else nvoi
                    cnt = m[rows] * nv * n
                    o[key] = host[off:off + nb].view(dt)[:cnt].reshape(m[rows], nv, n)
            res.append(o)
        return res

    def _region_view(self, key, dtype, shape):
        if key in self.zero.regions:
            return self._zview(key, dtype, shape)
        return self._iview(key, dtype, shape)

    def accumulators(self, k):
        """Monitor accumulators of instance k (to continue the simulation later)."""
        m, nvoi, s = self.meta[k], self.nvoi, self.specs[k]
        acc = {}
        if ('tavg_acc', k) in self.zero.regions or ('tavg_acc', k) in self.init.regions:
            acc['tavg_acc'] = self._region_view(('tavg_acc', k), torch.float32, (nvoi, m['n'])).cpu().numpy()
        if s.aff_istep:
            acc['aff_acc'] = self._region_view(('aff_acc', k), torch.float32, (self.ncvar, m['n'])).cpu().numpy()
        if s.proj_istep:
            acc['proj_acc'] = self._region_view(('proj_acc', k), torch.float32, (nvoi, m['n'])).cpu().numpy()
        if s.bold is not None:
            acc['bold_acc'] = self._region_view(('bold_acc', k), torch.float64, (nvoi, m['n'])).cpu().numpy()
            acc['bold_stock'] = self._region_view(('bold_stock', k), torch.float64,
                                                  (len(s.bold['hrf']), nvoi, m['n'])).cpu().numpy()
        return acc

    def status(self):
        return self._zview(('status',), torch.int32, (len(self.specs),)).cpu().numpy()

    def state(self, k):
        return self._iview(('state', k), torch.float32, (self.nsv, self.meta[k]['n'])).cpu().numpy()

    def ring(self, k):
        m = self.meta[k]
        V = self.lanes
        lead = k - k % V
        if self.ring_layout:
            RS = _lib.ring_region_stride(m['ring_len'], self.ncvar)
            rm = self._iview(('ring', k), torch.float32, (m['n'], RS, self.ncvar)).cpu().numpy()
            return ring_time_major(rm, m['ring_len'])
        r = self._iview(('ring', lead), torch.float32, (m['ring_len'], m['n'], self.ncvar, V)).cpu().numpy()
        return np.ascontiguousarray(r[..., k % V])

    def current_step(self, k):
        off, _ = self.init.regions[('insts',)]
        raw = self.init_buf[off:off + len(self.specs) * _lib.INST_DTYPE.itemsize].cpu().numpy()
        return int(raw.view(_lib.INST_DTYPE)[k]['step'])

    def gather_delayed(self, k, step):
        """Delayed values the coupling of `step` reads for every edge of instance k
        (read through the same address arithmetic as the kernel)."""
        if self.lanes != 1 or self.sigma or self.ring_layout:
            raise ValueError('gather_delayed reads single-instance time-major rings of raw coupling variables')
        m = self.meta[k]
        conn = self.specs[k].conn
        out = torch.empty(max(conn.nnz, 1) * self.ncvar, dtype=torch.float32, device=self.device)
        inst = _lib.Inst()
        d = self.insts_host[k]
        inst.edges = int(d['edges'])
        inst.ring = int(d['ring'])
        inst.n, inst.nnz, inst.horizon, inst.ring_len = m['n'], conn.nnz, conn.horizon, m['ring_len']
        st = torch.cuda.current_stream(self.device)
        _lib.check(self.lib.tvbk_gather_delayed(ctypes.byref(inst), self.ncvar, int(step),
                                                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st.cuda_stream)))
        return out[:conn.nnz * self.ncvar].view(conn.nnz, self.ncvar).cpu().numpy()


def functional_connectivity(series, stream=None):
    """Pearson FC per instance on the device: series (I, T, n) float64 tensor or
    array -> (I, n, n) float64 tensor (numpy.corrcoef over time)."""
    lib = _lib.load()
    x = series if isinstance(series, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(series))
    x = x.to('cuda', dtype=torch.float64).contiguous()
    if x.dim() == 2:
        x = x[None]
    I, T, n = x.shape
    fc = torch.empty((I, n, n), dtype=torch.float64, device=x.device)
    st = torch.cuda.current_stream(x.device) if stream is None else stream
    _lib.check(lib.tvbk_fc(ctypes.c_void_p(x.data_ptr()), I, T, n, ctypes.c_void_p(fc.data_ptr()),
                           ctypes.c_void_p(st.cuda_stream)))
    return fc
