"""tvbk_sim_run_static, the entry point that allocates nothing.

It serves callers that cannot call cudaMalloc -- FFI or plug-in hosts that
only hold the input and output buffers handed to them, or code under a fixed
memory budget -- by keeping the simulation's working memory (ring, monitor
accumulators, Bold stock, sigmoid ring, descriptor, status) in a static
device array inside the library.  These tests call it through the C ABI and
check its outputs against the regular entry point, tvbk_sim_run, on two
calls in a row (the second call finds the array holding the first call's
contents), for every user of that array: the ring and the TemporalAverage /
Bold accumulators (ReducedWongWang), the AfferentCoupling and projection
period sums (Generic2dOscillator), and the pre-applied sigmoid ring of
SigmoidalJansenRit read in place (JansenRit).  The two entry points run the
same kernel on the same inputs, so the outputs must agree bit for bit, and
the device's free memory must not move across a call.

This file is collected last so that a failure here stops a run only after
every other test has run.
"""
import ctypes

import numpy as np
import pytest

import golden_util as G

pytestmark = pytest.mark.gpu


def _simulator(case):
    from tvb_b200 import coupling, integrators, models, monitors, noise
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.simulator import Simulator
    if case == 'rww_tavg_bold':
        fx = G.load('rww_68_short')
        w, L = G.connectome(fx)
        return Simulator(model=models.ReducedWongWang(), connectivity=Connectivity(w, L, speed=float(fx['speed'])),
                         coupling=coupling.Linear(a=0.3),
                         integrator=integrators.EulerStochastic(dt=0.1, noise=noise.Additive(nsig=[1e-3])),
                         monitors=[monitors.TemporalAverage(period=100.0), monitors.Bold(period=2000.0)],
                         simulation_length=2500.0).configure(), 25000, {}
    if case == 'g2d_afferent_projection':
        fx = G.load('projection_40')
        from tvb_b200 import sensors
        conn = Connectivity(fx['weights'], fx['tract_lengths'], speed=float(fx['speed']), centres=fx['centres'],
                            orientations=fx['orientations'])
        eeg = monitors.EEG(period=2.0, sensors=sensors.SensorsEEG(['e%d' % i for i in range(16)], fx['sensors_eeg']),
                           projection=sensors.ProjectionSurfaceEEG(fx['lead_eeg']),
                           region_mapping=sensors.RegionMapping(fx['rmap']), reference='average')
        np.random.seed(501)
        return Simulator(model=models.Generic2dOscillator(), connectivity=conn, coupling=coupling.Linear(a=0.0152),
                         integrator=integrators.HeunDeterministic(dt=0.1),
                         monitors=[monitors.AfferentCouplingTemporalAverage(period=1.0), eeg],
                         simulation_length=300.0).configure(), 3000, {}
    assert case == 'jr_sigmoidal_in_place'
    fx = G.load('afferent_40')
    conn = Connectivity(fx['weights'], fx['tract_lengths'], speed=float(fx['speed']))
    nsig = np.array([0.0, 0.0, 0.0, 0.0, 1e-5, 0.0])
    return Simulator(model=models.JansenRit(), connectivity=conn, coupling=coupling.SigmoidalJansenRit(),
                     integrator=integrators.HeunStochastic(dt=0.05, noise=noise.Additive(nsig=nsig, noise_seed=7)),
                     monitors=[monitors.TemporalAverage(period=1.0)],
                     simulation_length=200.0).configure(), 4000, dict(ring_in_smem=False)


CASES = ['rww_tavg_bold', 'g2d_afferent_projection', 'jr_sigmoidal_in_place']
OUTPUTS = ('raw', 'tavg', 'bold', 'sub', 'aff', 'proj')


def _regular_run(case):
    """One instance through tvbk_sim_run (Batch.run); returns the batch reset
    to its initial state, the reference outputs and final state."""
    from tvb_b200.engine import Batch
    sim, n_steps, kw = _simulator(case)
    spec, noise_kind = sim.instance_spec(n_steps)
    batch = Batch(sim._model_id, sim._cfun_id, sim._scheme_id, noise_kind, sim.integrator.dt, sim._voi_codes,
                  [spec], **kw)
    batch.snapshot()
    batch.run()
    assert int(batch.status()[0]) == 0
    ref = {k: v.copy() for k, v in batch.outputs_host()[0].items() if k in OUTPUTS}
    ref_state = batch.state(0).copy()
    batch.reset()
    return batch, n_steps, ref, ref_state


def _static_call(lib, batch, n_steps):
    """tvbk_sim_run_static on the batch's own (reset) inputs and output
    buffers; the descriptor's accumulator pointers are set to NULL, since the
    entry point keeps every accumulator in its own array."""
    import torch
    from tvb_b200 import _lib
    d = batch.insts_host[0]
    inst = _lib.Inst()
    for name, _ in _lib.Inst._fields_:
        if name != 'cfun':
            setattr(inst, name, int(d[name]) if np.issubdtype(d[name].dtype, np.integer) else float(d[name]))
    for k in range(6):
        inst.cfun[k] = float(d['cfun'][k])
    inst.tavg_acc = inst.bold_acc = inst.bold_stock = inst.aff_acc = inst.proj_acc = inst.pre_ring = 0
    L = batch.launch_struct(n_steps)
    status = torch.full((1,), -1, dtype=torch.int32, device=batch.device)
    st = torch.cuda.current_stream()
    rc = lib.tvbk_sim_run_static(ctypes.byref(L), ctypes.byref(inst), ctypes.c_void_p(status.data_ptr()),
                                 ctypes.c_void_p(st.cuda_stream))
    assert rc == 0, lib.tvbk_last_error().decode()
    torch.cuda.synchronize()
    return int(status.cpu()[0])


@pytest.mark.parametrize('case', CASES)
def test_static_entry_matches_regular_entry_twice(case):
    import torch
    from tvb_b200 import _lib
    lib = _lib.load()
    batch, n_steps, ref, ref_state = _regular_run(case)
    used = [k for k in OUTPUTS if k in ref]
    if case == 'g2d_afferent_projection':
        assert {'aff', 'proj'} <= set(used)
    for call in range(2):
        batch.reset()   # initial ring and state back in place, outputs zeroed
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        status = _static_call(lib, batch, n_steps)
        free1 = torch.cuda.mem_get_info()[0]
        assert status == 0
        got = batch.outputs_host()[0]
        for k in used:
            assert got[k].shape == ref[k].shape, (call, k)
            assert np.array_equal(got[k], ref[k]), (call, k, float(np.abs(got[k] - ref[k]).max()))
        assert np.array_equal(batch.state(0), ref_state), call
        if call:   # the first call may load the library's kernels; after it no call takes device memory
            assert free1 == free0, 'device free memory moved by %d bytes' % (free0 - free1)
        print('%s call %d: %s and final state bit-identical; free memory %+d bytes'
              % (case, call, '/'.join(used), free1 - free0))


def test_static_entry_rejects_oversized_instance():
    import torch
    from tvb_b200 import _lib
    batch, n_steps, _, _ = _regular_run('rww_tavg_bold')
    L = batch.launch_struct(n_steps)
    inst = _lib.Inst()
    buf = torch.zeros(16, dtype=torch.float32, device='cuda')
    inst.ring = inst.state = inst.row_ptr = inst.params = buf.data_ptr()
    inst.n, inst.horizon, inst.ring_len = 1000, 2001, 2100
    inst.step, inst.step_end = 0, 10
    lib = _lib.load()
    rc = lib.tvbk_sim_run_static(ctypes.byref(L), ctypes.byref(inst), None, None)
    assert rc == _lib.TVBK_ERR_TOO_LARGE
    assert b'scratch' in lib.tvbk_last_error()
