"""Continuous-batching simulation service on one GPU.

Simulation requests -- each one what a user would run as
``Simulator(...).configure().run()`` -- arrive over time.  The server keeps
every admitted request resident on the device (history ring, state,
parameters, connectome, monitor accumulators and outputs) until it completes
and runs them concurrently:

* Admission by device footprint: a request is admitted, in arrival order,
  when the bytes of its arenas fit in the memory budget and its group has a
  free slot; otherwise it waits (requests behind it that fit are admitted).
* Groups: admitted requests with the same kernel configuration (model,
  coupling, scheme, noise kind, dt, observed variables, region count and the
  kernel variant chosen for them) share one slot table (a device array of
  ``tvbk_inst`` descriptors, allocated on the group's stream) and one CUDA
  stream; everything a group does on the device is ordered on that stream.  Each launch advances every occupied slot of a group by one chunk
  of steps (``tvbk_sim_run``); a slot whose request finished is inert.  Groups
  run on separate streams, so their launches overlap on the device.
* Continuous batching: between chunks, finished requests are retired (their
  outputs copied to pinned host memory on the group's stream, their
  descriptor cleared) and waiting requests are admitted into free slots.  A
  group keeps at most ``inflight`` chunks queued, so a new request starts
  within that many chunks of its admission.
* Completion is observed by polling CUDA events (``Event.query``), with a
  bounded wait in ``run``; the host never blocks on a device wait.

The noise of a request is keyed by (noise seed, request id) -- Philox
counter (step, region, state variable) -- and not by its slot, and the
kernel's arithmetic does not depend on the barrier interval or the chunking,
so a request's result is the same alone and in any mix.
"""
import collections
import ctypes
import time

import numpy as np
import torch

from . import _lib
from .engine import Batch

INST_BYTES = _lib.INST_DTYPE.itemsize


class _Request:
    def __init__(self, rid, sim, spec, noise_kind, key, plan, t_submit):
        self.rid = rid
        self.sim = sim
        self.spec = spec
        self.noise_kind = noise_kind
        self.key = key
        self.plan = plan                  # Batch of this request (arenas planned, allocated on admission)
        self.footprint = plan.nbytes
        self.t_submit = t_submit
        self.t_admit = None
        self.t_done = None
        self.slot = None
        self.step = spec.step0
        self.step_end = spec.step0 + spec.n_steps
        self.host_out = None
        self.host_status = None
        self.done_event = None
        self.result = None
        self.status = None


class _Group:
    def __init__(self, key, device, max_slots):
        self.key = key
        self.stream = torch.cuda.Stream(device=device)
        # allocated and zero-filled on the group's own stream: every later use of the slot table (descriptor
        # writes, launches) is on that stream, so no fill on another stream can land after a descriptor write
        with torch.cuda.stream(self.stream):
            self.desc = torch.zeros(max_slots * INST_BYTES, dtype=torch.uint8, device=device)
            self.status = torch.zeros(max_slots, dtype=torch.int32, device=device)
        self.slots = [None] * max_slots
        self.inflight = collections.deque()   # events of queued chunks
        self.launches = 0

    def free_slot(self):
        for j, r in enumerate(self.slots):
            if r is None:
                return j
        return None

    def active(self):
        return [r for r in self.slots if r is not None and r.step < r.step_end]


class SimulationServer:
    """Admits simulation requests by device footprint and advances the
    admitted ones together in chunks of `chunk_steps` steps.

    memory_budget: device bytes the requests' arenas may take (default: 80 %
    of the free device memory at construction).  max_slots: requests resident
    at once per group.  inflight: chunks a group may have queued.
    """

    def __init__(self, memory_budget=None, chunk_steps=2000, max_slots=1024, inflight=2, device=None):
        self.lib = _lib.load()
        self.device = torch.device(device if device is not None else 'cuda')
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            memory_budget = int(0.8 * free)
        self.budget = int(memory_budget)
        self.chunk_steps = int(chunk_steps)
        self.max_slots = int(max_slots)
        self.inflight = max(1, int(inflight))
        self.queue = collections.deque()
        self.groups = {}
        self.requests = {}
        self.draining = []
        self.used = 0
        self.peak_used = 0
        self.next_id = 0
        self.region_steps = 0
        self.mem_samples = []

    # -------------------------------------------------------------- requests
    def submit(self, sim, n_steps=None, t_submit=None):
        """Queue a configured ``Simulator`` for `n_steps` steps (default: its
        simulation_length).  Returns the request id.  Raises ValueError when
        the request can never fit the memory budget, NotImplementedError for
        fed noise (the server draws Philox noise keyed by the request)."""
        if not getattr(sim, '_configured', False):
            raise RuntimeError('submit a configured Simulator')
        if n_steps is None:
            n_steps = int(np.ceil(sim.simulation_length / sim.integrator.dt))
        rid = self.next_id
        self.next_id += 1
        spec, noise_kind = sim.instance_spec(int(n_steps), stream=rid)
        if noise_kind == _lib.NOISE_FED:
            raise NotImplementedError('the server draws device noise; use noise_source="philox"')
        plan = Batch(sim._model_id, sim._cfun_id, sim._scheme_id, noise_kind, sim.integrator.dt, sim._voi_codes,
                     [spec], device=self.device, gather='row', allocate=False, groups=False)
        # one kernel configuration per group: the components and the variant the plan chose (ring staging,
        # cluster, prefetch, sigmoid ring, ring layout), so every occupant of a launch has the buffers that
        # launch reads
        key = (sim._model_id, sim._cfun_id, sim._scheme_id, noise_kind, float(np.float32(sim.integrator.dt)),
               tuple(sim._voi_codes), sim.number_of_nodes, plan.ring_in_smem, plan.cluster, plan.prefetch,
               plan.sigma, plan.edges_per_thread if plan.cluster else 0, plan.ring_layout, plan.block_steps)
        req = _Request(rid, sim, spec, noise_kind, key, plan, time.perf_counter() if t_submit is None else t_submit)
        if req.footprint > self.budget:
            raise ValueError('request needs %d bytes, more than the budget of %d' % (req.footprint, self.budget))
        self.requests[rid] = req
        self.queue.append(req)
        return rid

    def result(self, rid):
        """Per-monitor (times, data[T, nvoi, n, 1]) of a completed request, as
        ``Simulator.run`` returns them; None while it runs."""
        return self.requests[rid].result

    def done(self, rid):
        return self.requests[rid].result is not None

    @property
    def idle(self):
        return not self.queue and not self.draining and all(
            all(r is None for r in g.slots) for g in self.groups.values())

    # ----------------------------------------------------------------- steps
    def _group(self, key):
        g = self.groups.get(key)
        if g is None:
            g = _Group(key, self.device, self.max_slots)
            self.groups[key] = g
        return g

    def _admit(self):
        waiting = collections.deque()
        while self.queue:
            req = self.queue.popleft()
            g = self._group(req.key)
            j = g.free_slot() if self.used + req.footprint <= self.budget else None
            if j is None:
                waiting.append(req)
                continue
            with torch.cuda.stream(g.stream):
                req.plan.allocate()
                d = req.plan.insts_host.copy()
                d[0]['step'] = req.step
                g.desc[j * INST_BYTES:(j + 1) * INST_BYTES].copy_(torch.from_numpy(d.view(np.uint8)))
                g.status[j:j + 1].zero_()
            g.slots[j] = req
            req.slot = j
            req.t_admit = time.perf_counter()
            self.used += req.footprint
        self.peak_used = max(self.peak_used, self.used)
        self.queue = waiting

    def _launch(self, g):
        occ = g.active()
        if not occ:
            return False
        plans = [r.plan for r in occ]
        hi = max(r.slot for r in occ) + 1
        p0 = plans[0]
        L = _lib.Launch()
        L.insts = g.desc.data_ptr()
        L.status = g.status.data_ptr()
        L.n_inst = hi
        L.model, L.cfun, L.scheme, L.noise = p0.model_id, p0.cfun_id, p0.scheme_id, p0.noise_kind
        L.nvoi = p0.nvoi
        for v, code in enumerate(p0.voi):
            L.voi[v] = code
        L.max_n = max(p.max_n for p in plans)
        L.max_ring_len = max(p.meta[0]['ring_len'] for p in plans)
        L.sync_every = min(p.sync_every for p in plans)
        L.ring_in_smem = 1 if all(p.ring_in_smem for p in plans) else 0
        L.max_degree = max(p.max_degree for p in plans)
        pf = {p.prefetch for p in plans}   # one value per group (the group key holds it)
        L.prefetch = pf.pop() if len(pf) == 1 else (1 if all(p.prefetch for p in plans) else 0)
        L.lanes = 1
        L.cluster = p0.cluster
        L.cluster_edges = max(p.cluster_edges for p in plans)
        L.edges_per_thread = p0.edges_per_thread if p0.cluster else 0   # edge runs (one value per group)
        # one value per group; region-major rings keep sync_every a multiple of the block length
        L.ring_layout, L.block_steps = p0.ring_layout, p0.block_steps
        L.extras = 0
        for p in plans:
            L.extras |= p.extras
        L.max_steps = self.chunk_steps
        L.dt = p0.dt
        st = g.stream
        _lib.check(self.lib.tvbk_sim_run(ctypes.byref(L), ctypes.c_void_p(st.cuda_stream)))
        g.launches += 1
        finished = []
        for r in occ:
            k = min(self.chunk_steps, r.step_end - r.step)
            r.step += k
            self.region_steps += k * r.spec.conn.n
            if r.step == r.step_end:
                finished.append(r)
        with torch.cuda.stream(st):
            for r in finished:
                # stream-ordered after the chunk: outputs and status to pinned host memory, slot cleared
                r.host_out = torch.empty(r.plan.out_buf.numel(), dtype=torch.uint8, pin_memory=True)
                r.host_out.copy_(r.plan.out_buf, non_blocking=True)
                r.host_status = torch.empty(1, dtype=torch.int32, pin_memory=True)
                r.host_status.copy_(g.status[r.slot:r.slot + 1], non_blocking=True)
                g.desc[r.slot * INST_BYTES:(r.slot + 1) * INST_BYTES].zero_()
                r.done_event = torch.cuda.Event()
                r.done_event.record(st)
                g.slots[r.slot] = None
                self.draining.append(r)
            ev = torch.cuda.Event()
            ev.record(st)
        g.inflight.append(ev)
        return True

    def _retire(self):
        keep = []
        for r in self.draining:
            if not r.done_event.query():
                keep.append(r)
                continue
            out = r.plan.outputs_from_bytes(r.host_out.numpy())[0]
            r.status = int(r.host_status[0])
            r.result = r.sim._collect(r.spec.step0, r.spec.n_steps, out)
            r.t_done = time.perf_counter()
            self.used -= r.footprint
            r.plan = None       # device arenas go back to the caching allocator
            r.host_out = None
        self.draining = keep

    def pump(self):
        """One scheduling round: retire finished requests, admit waiting ones,
        queue a chunk for every group with room.  Returns True if any chunk
        was queued."""
        self._retire()
        self._admit()
        launched = False
        for g in self.groups.values():
            while g.inflight and g.inflight[0].query():
                g.inflight.popleft()
            if len(g.inflight) < self.inflight:
                launched = self._launch(g) or launched
        self.mem_samples.append(self.used)
        return launched

    def run(self, arrivals=None, timeout=600.0, poll=2e-4):
        """Serve until every submitted request (and every arrival) is done.

        arrivals: optional list of (t_offset_seconds, callable) -- at
        t_offset after the start, the callable is called with this server
        (it submits requests).  Polls with a sleep of `poll` seconds when
        there is nothing to do; raises TimeoutError after `timeout` seconds.
        """
        pending = sorted(arrivals or [], key=lambda a: a[0])
        t0 = time.perf_counter()
        i = 0
        while True:
            now = time.perf_counter() - t0
            while i < len(pending) and pending[i][0] <= now:
                pending[i][1](self)
                i += 1
            launched = self.pump()
            if i == len(pending) and self.idle:
                break
            if time.perf_counter() - t0 > timeout:
                raise TimeoutError('serving did not finish within %g s' % timeout)
            if not launched:
                time.sleep(poll)
        return self

    # ----------------------------------------------------------------- stats
    def stats(self, rids=None):
        """Latency (submit to result on the host) percentiles, throughput and
        device-memory occupancy of the completed requests."""
        reqs = [self.requests[k] for k in (rids if rids is not None else self.requests)]
        reqs = [r for r in reqs if r.t_done is not None]
        if not reqs:
            return {}
        lat = np.array([r.t_done - r.t_submit for r in reqs])
        span = max(r.t_done for r in reqs) - min(r.t_submit for r in reqs)
        rs = sum(r.spec.n_steps * r.spec.conn.n for r in reqs)
        return {
            'completed': len(reqs),
            'latency_p50_s': float(np.percentile(lat, 50)),
            'latency_p99_s': float(np.percentile(lat, 99)),
            'latency_mean_s': float(lat.mean()),
            'latency_max_s': float(lat.max()),
            'sims_per_s': len(reqs) / span,
            'region_steps_per_s': rs / span,
            'span_s': span,
            'memory_budget_bytes': self.budget,
            'memory_peak_bytes': int(self.peak_used),
            'memory_mean_bytes': float(np.mean(self.mem_samples)) if self.mem_samples else 0.0,
            'groups': len(self.groups),
            'launches': int(sum(g.launches for g in self.groups.values())),
        }
