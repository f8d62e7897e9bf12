"""``pb_cxr_score_noalloc``: the bin-mean PXR + CBS scorer without device allocation.

Some callers of this library cannot call cudaMalloc: code that runs inside an
allocator or memory-pool callback, an embedding runtime that owns every byte of
device memory, or a deployment that fixes all allocations when it loads. For
them this entry point keeps the far-field workspace in a fixed device array
built into the library instead of a caller-provided buffer.

The GPU test scores one segment list with the allocating entry point
(``pb_cxr_score``, workspace from the caller) and then twice in a row with the
no-allocation one, and requires the same spectra each time: the shared array
must come back cleared on every call. The CPU test checks that a request
larger than the fixed array is refused with a clear error.
"""

import ctypes as C

import numpy as np
import pytest


def _case(precision, cuda_device):
    from pyrite_b200 import configs
    from pyrite_b200.pipeline import ScoringCase

    return ScoringCase(configs.c2_si_50mev(seed=3), precision=precision, batch_histories=2048,
                       device=cuda_device)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_noalloc_matches_allocating_entry_point(precision, tol, cuda_device):
    import torch

    from pyrite_b200 import _lib as L

    case = _case(precision, cuda_device)
    lib = L.load()
    stream = torch.cuda.current_stream().cuda_stream
    case.seg_count.zero_()
    t = case.targs
    t.e_start, t.n = 0, 2048
    L.check(lib.pb_transport(C.byref(t), stream), "pb_transport")
    torch.cuda.synchronize()
    assert int(case.seg_count.item()) > 0
    assert case.cargs.exact_widths > 0 and case.cargs.far_pad >= 0  # far field in use

    def score(fn, name):
        case.spec_cxr.zero_()
        L.check(fn(C.byref(case.cargs), stream), name)
        torch.cuda.synchronize()
        return case.spec_cxr.cpu().numpy().copy()

    ref = score(lib.pb_cxr_score, "pb_cxr_score")
    first = score(lib.pb_cxr_score_noalloc, "pb_cxr_score_noalloc")
    second = score(lib.pb_cxr_score_noalloc, "pb_cxr_score_noalloc")
    peak = np.max(np.abs(ref))
    assert peak > 0
    # Same arithmetic; only the order of the atomic accumulations differs.
    assert np.max(np.abs(first - ref)) <= tol * peak
    assert np.max(np.abs(second - ref)) <= tol * peak


def test_noalloc_refuses_oversized_far_field():
    from pyrite_b200 import _lib as L

    lib = L.load()
    a = L.PbCxrArgs()
    a.quadrature = L.PB_QUAD_BINMEAN
    a.n_dir, a.n_E, a.n_seg = 64, 4096, 1
    a.exact_widths, a.far_pad = 64.0, 1024
    t = a.tables
    t.n_g, t.n_tab, t.n_mu = 1, 2, 1
    dummy = C.c_double(0.0)
    ptr = C.cast(C.pointer(dummy), C.c_void_p).value
    for name in ("G", "ES", "EP", "WM", "row_table", "E_tab", "chi_re", "chi_im", "u_re", "u_im",
                 "log_mu", "delta"):
        setattr(t, name, ptr)
    for name in ("n_hat", "r_mid", "v_hat", "L", "E_keV", "elec_id", "edges", "spec"):
        setattr(a, name, ptr)
    assert lib.pb_cxr_score_noalloc(C.byref(a), None) == 4  # PB_ERR_CAPACITY
    assert b"fixed workspace" in lib.pb_last_error()
    a.quadrature = L.PB_QUAD_NODE
    assert lib.pb_cxr_score_noalloc(C.byref(a), None) == 3  # PB_ERR_UNSUPPORTED
