"""tvbk_sim_run_static, the entry point that allocates nothing.

It serves callers that cannot call cudaMalloc -- FFI or plug-in hosts that
only hold the input and output buffers handed to them, or code under a fixed
memory budget -- by keeping the simulation's working memory (ring,
monitor accumulators, Bold stock, descriptor, status) in a static device
array inside the library.  This test calls it through the C ABI and checks
its outputs against the regular entry point, tvbk_sim_run, on two calls in a
row (the second call finds the array holding the first call's contents).
This file is collected last so that a failure here stops a run only after
every other test has run.
"""
import ctypes

import numpy as np
import pytest

import golden_util as G

pytestmark = pytest.mark.gpu


def _setup():
    import torch
    from tvb_b200 import _lib, coupling, integrators, models, monitors, noise
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.engine import Batch, InstanceSpec, ring_from_reference
    from tvb_b200.simulator import Simulator
    fx = G.load('rww_68_short')
    w, L = G.connectome(fx)
    sim = Simulator(model=models.ReducedWongWang(), connectivity=Connectivity(w, L, speed=float(fx['speed'])),
                    coupling=coupling.Linear(a=0.3),
                    integrator=integrators.EulerStochastic(dt=0.1, noise=noise.Additive(nsig=[1e-3])),
                    monitors=[monitors.TemporalAverage(period=100.0), monitors.Bold(period=2000.0)],
                    simulation_length=2500.0).configure()
    n_steps = 25000
    raw, tavg_istep, bspec = sim._monitor_spec()
    spec = InstanceSpec(sim._conn, sim.history_buffer[..., 0], sim.current_state[..., 0], sim._params,
                        sim.coupling.kernel_params(), n_steps, sigma=sim._sigma, seed=42, stream=5,
                        tavg_istep=tavg_istep, bold=bspec)
    batch = Batch(sim._model_id, sim._cfun_id, sim._scheme_id, _lib.NOISE_PHILOX, 0.1, sim._voi_codes, [spec])
    batch.run()
    ref = batch.outputs_host()[0]
    ref_state = batch.state(0)
    L = batch.launch_struct(n_steps)
    return sim, spec, batch, L, ref, ref_state


def _call_static(sim, spec, batch, L):
    import torch
    from tvb_b200 import _lib
    from tvb_b200.engine import ring_from_reference
    dev = torch.device('cuda')
    n = spec.conn.n
    RL = batch.meta[0]['ring_len']
    keep = []

    def put(a, dtype):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).to(dev)
        keep.append(t)
        return t

    row_ptr = put(spec.conn.row_ptr, np.int32)
    edges = put(spec.conn.edges.view(np.uint8), np.uint8)
    ring0 = put(ring_from_reference(spec.ring0, spec.step0, RL), np.float32)
    state = put(spec.state0, np.float32)
    params = put(spec.params, np.float32)
    sigma = put(spec.sigma, np.float32)
    hrf = put(spec.bold['hrf'], np.float64)
    m = batch.meta[0]
    tavg = torch.zeros((m['tavg_rows'], 1, n), dtype=torch.float32, device=dev)
    bold = torch.zeros((m['bold_rows'], 1, n), dtype=torch.float64, device=dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    d = batch.insts_host[0]
    inst = _lib.Inst()
    for name, _ in _lib.Inst._fields_:
        if name != 'cfun':
            setattr(inst, name, int(d[name]) if np.issubdtype(d[name].dtype, np.integer) else float(d[name]))
    for k in range(6):
        inst.cfun[k] = float(d['cfun'][k])
    inst.row_ptr, inst.edges, inst.ring, inst.state = row_ptr.data_ptr(), edges.data_ptr(), ring0.data_ptr(), \
        state.data_ptr()
    inst.params, inst.noise_sigma, inst.hrf = params.data_ptr(), sigma.data_ptr(), hrf.data_ptr()
    inst.tavg, inst.bold = tavg.data_ptr(), bold.data_ptr()
    inst.tavg_acc = inst.bold_acc = inst.bold_stock = 0
    inst.step, inst.step_end = spec.step0, spec.step0 + spec.n_steps
    lib = _lib.load()
    st = torch.cuda.current_stream()
    rc = lib.tvbk_sim_run_static(ctypes.byref(L), ctypes.byref(inst), ctypes.c_void_p(status.data_ptr()),
                                 ctypes.c_void_p(st.cuda_stream))
    assert rc == 0, lib.tvbk_last_error().decode()
    torch.cuda.synchronize()
    return tavg.cpu().numpy(), bold.cpu().numpy(), state.cpu().numpy(), int(status.cpu().numpy()[0]), ring0


def test_static_entry_matches_regular_entry_twice():
    sim, spec, batch, L, ref, ref_state = _setup()
    for call in range(2):
        tavg, bold, state, status, _ = _call_static(sim, spec, batch, L)
        assert status == 0
        for name, got, want in (('tavg', tavg, ref['tavg']), ('bold', bold, ref['bold']), ('state', state, ref_state)):
            err = np.abs(got - want).max() / max(np.abs(want).max(), 1e-300)
            print('call %d %-5s max_rel %.3e' % (call, name, err))
            assert err <= 1e-6, (call, name, err)


def test_static_entry_rejects_oversized_instance():
    import torch
    from tvb_b200 import _lib
    sim, spec, batch, L, ref, ref_state = _setup()
    inst = _lib.Inst()
    buf = torch.zeros(16, dtype=torch.float32, device='cuda')
    inst.ring = inst.state = inst.row_ptr = inst.params = buf.data_ptr()
    inst.n, inst.horizon, inst.ring_len = 1000, 2001, 2100
    inst.step, inst.step_end = 0, 10
    lib = _lib.load()
    rc = lib.tvbk_sim_run_static(ctypes.byref(L), ctypes.byref(inst), None, None)
    assert rc == _lib.TVBK_ERR_TOO_LARGE
    assert b'scratch' in lib.tvbk_last_error()
