"""Host-side monitor logic (CPU): the AfferentCouplingTemporalAverage
reduction of an every-step coupling stream, used when AfferentCoupling
monitors of different periods share a run."""
import numpy as np


def _device_rule(raw, s0, istep, carry):
    """The device's arithmetic: float32 running sum from the carry, divided by
    istep at every step that is a multiple of istep."""
    acc = carry.copy()
    out = []
    for k in range(raw.shape[0]):
        acc = acc + raw[k]
        if (s0 + 1 + k) % istep == 0:
            out.append(acc / np.float32(istep))
            acc = np.zeros_like(acc)
    return (np.stack(out) if out else np.zeros((0,) + raw.shape[1:], np.float32)), acc


def test_afferent_average_matches_the_device_rule_across_chunks():
    from tvb_b200.monitors import AfferentCouplingTemporalAverage
    rng = np.random.default_rng(0)
    m = AfferentCouplingTemporalAverage(period=1.0)
    for istep in (1, 3, 10):
        m.istep = istep
        raw = rng.normal(size=(257, 2, 5)).astype(np.float32)
        for cuts in ([257], [7, 100, 150], [1, 1, 255], [13, 244]):
            carry_m = carry_d = np.zeros((2, 5), np.float32)
            s0 = 4
            got, want = [], []
            for a, b in zip(np.cumsum([0] + cuts[:-1]), np.cumsum(cuts)):
                y, carry_m = m.average(raw[a:b], s0 + a, carry_m)
                z, carry_d = _device_rule(raw[a:b], s0 + a, istep, carry_d)
                got.append(y)
                want.append(z)
            np.testing.assert_array_equal(np.concatenate(got), np.concatenate(want))
            np.testing.assert_array_equal(carry_m, carry_d)
