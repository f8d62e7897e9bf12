"""``pb_transport_score``: the whole exact pass (transport, then every CXR,
bremsstrahlung and characteristic scorer) in one C call gives the spectra and
tallies of the same entry points called one by one; its argument checks run
before anything is launched."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fused_pass_equals_separate_calls(cuda_device):
    import torch

    from pyrite_b200.configs import c2_si_50mev
    from pyrite_b200.pipeline import ScoringCase

    spec = c2_si_50mev(angular_shape=(2, 2), n_bins=512)
    out = []
    for fused in (True, False):
        case = ScoringCase(spec, precision="mixed", rng="philox", lut=True, batch_histories=2048)
        for b in range(2):
            if fused:
                case.run_batch(b * 2048, 2048)
            else:
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
                case.run_batch(b * 2048, 2048, events=ev)  # the per-entry-point path
        torch.cuda.synchronize()
        out.append(case.results())
        assert case.device_status() == 0
    a, b = out
    for k in ("cxr", "brem"):
        peak = float(np.max(np.abs(b[k])))
        assert peak > 0
        # the same work; only the order of the float shared-memory atomics differs
        assert float(np.max(np.abs(a[k] - b[k]))) <= 1e-6 * peak, k
    np.testing.assert_array_equal(a["fates"], b["fates"])


def test_fused_pass_checks_every_set_first(cuda_device):
    """A bad scorer set is refused before the transport is launched: the
    segment count stays untouched."""
    import torch

    from pyrite_b200 import _lib as L
    from pyrite_b200.configs import c2_si_50mev
    from pyrite_b200.pipeline import ScoringCase

    case = ScoringCase(c2_si_50mev(angular_shape=(1, 1), n_bins=256), precision="mixed", rng="philox", lut=True,
                       batch_histories=256)
    case.seg_count.fill_(12345)
    p = L.PbTransportScoreArgs()
    p.transport = case.targs
    p.transport.e_start, p.transport.n = 0, 256
    bad = L.PbCxrArgs.from_buffer_copy(case.cargs_all[0])
    bad.n_dir = 0
    arr = (L.PbCxrArgs * 1)(bad)
    p.n_cxr, p.cxr = 1, C.cast(arr, C.POINTER(L.PbCxrArgs))
    rc = L.load().pb_transport_score(C.byref(p), torch.cuda.current_stream().cuda_stream)
    assert rc == L.PB_ERR_INVALID
    torch.cuda.synchronize()
    assert int(case.seg_count.item()) == 12345
