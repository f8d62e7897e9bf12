"""Edge cases of the C-ABI scorers and the transport, on the GPU.

- empty segment lists (host size 0, and a device count of 0 behind a
  non-empty buffer) leave every spectrum untouched;
- ragged splits: scoring segments [0, n) equals scoring [0, k) plus [k, n)
  for k off every tile boundary (16-segment CXR tiles, 256-segment brem
  chunks), the size-independent additivity of the estimators;
- a direction count that is not a multiple of the brem kernel's 16;
- a line buffer too small for the kept lines reports the overflow and the
  true line count instead of writing past its end;
- the transport's step limit ends every history with the reference's
  "step-limited" exit code and sets the device status bit.
"""

import numpy as np
import pytest

import oracle
from conftest import golden

pytestmark = pytest.mark.gpu

SYM = {6.0: "C", 8.0: "O", 14.0: "Si", 74.0: "W"}


def _cxr_inputs(name="si50"):
    from pyrite_b200 import LineTables
    from pyrite_b200.tables import ReflectionRows

    d = golden(f"cxr_{name}")
    tr = golden(f"transport_{d['transport']}")
    seg = dict(v_hat=tr["v_hat"], E_repr_keV=tr["E_repr_keV"], L_ang=tr["L_ang"], r_mid=tr["r_mid"],
               elec_id=tr["elec_id"], Ne=int(d["Ne"]), thickness_ang=float(d["thickness"]))
    tables = LineTables(d["E_tab"], d["chi_re"], d["chi_im"], d["u_re"], d["u_im"], d["log_mu"], d["delta"])
    rows = ReflectionRows(d["G"], d["ES"][None], d["EP"][None], d["WM"], d["row_table"])
    return d, seg, tables, rows


def _sub(seg, lo, hi):
    out = dict(seg)
    for k in ("v_hat", "E_repr_keV", "L_ang", "r_mid", "elec_id", "E_keV"):
        if k in out:
            out[k] = np.ascontiguousarray(seg[k][lo:hi])
    return out


def _cxr(seg, d, tables, rows, device, **kw):
    from pyrite_b200 import mc_cxr_spectrum

    return mc_cxr_spectrum(seg, d["E_grid"], str(d["crystal"]), None, tables=tables, n_hat=d["n_hat"], rows=rows,
                           device=device, **kw)


def _brem(seg, d, device, n_hat=None, precision="fp64"):
    from pyrite_b200 import mc_brem_spectrum

    comp = [(SYM[float(z)], float(n)) for z, n in zip(d["Z"], d["n_ang3"])]
    return mc_brem_spectrum(seg, d["E_grid"], composition=comp, n_hat=d["n_hat"] if n_hat is None else n_hat,
                            mu=d["mu_grid"], precision=precision, device=device)


@pytest.mark.parametrize("quad", ["node", "bin-mean"])
def test_cxr_empty_and_ragged_split(quad, cuda_device):
    d, seg, tables, rows = _cxr_inputs()
    n = seg["L_ang"].size
    empty = _cxr(_sub(seg, 0, 0), d, tables, rows, cuda_device, line_quadrature=quad)
    assert not np.any(empty)
    whole = _cxr(seg, d, tables, rows, cuda_device, line_quadrature=quad)
    peak = np.max(np.abs(whole))
    assert peak > 0
    for k in (1, 17, n // 2 + 3, n - 5):
        parts = _cxr(_sub(seg, 0, k), d, tables, rows, cuda_device, line_quadrature=quad) + \
            _cxr(_sub(seg, k, n), d, tables, rows, cuda_device, line_quadrature=quad)
        assert np.max(np.abs(parts - whole)) <= 1e-12 * peak, k


def test_brem_empty_ragged_and_twenty_directions(cuda_device):
    d = golden("brem_c20")
    tr = golden(f"transport_{d['transport']}")
    seg = dict(v_hat=tr["v_hat"], E_repr_keV=tr["E_repr_keV"], L_ang=tr["L_ang"], r_mid=tr["r_mid"],
               elec_id=tr["elec_id"], Ne=int(d["Ne"]), thickness_ang=float(d["thickness"]))
    n = seg["L_ang"].size
    assert not np.any(_brem(_sub(seg, 0, 0), d, cuda_device))
    whole = _brem(seg, d, cuda_device)
    peak = np.max(whole)
    for k in (1, 255, 257, n - 3):
        parts = _brem(_sub(seg, 0, k), d, cuda_device) + _brem(_sub(seg, k, n), d, cuda_device)
        assert np.max(np.abs(parts - whole)) <= 1e-12 * peak, k
    # 20 directions: one full launch of 16 and a ragged one of 4, each
    # against the oracle's single-direction spectrum
    rng = np.random.default_rng(4)
    base = np.asarray(d["n_hat"], float)
    n_hats = base[None, :] + 0.05 * rng.normal(size=(20, 3))
    n_hats /= np.linalg.norm(n_hats, axis=1, keepdims=True)
    spec = _brem(seg, d, cuda_device, n_hat=n_hats)
    oseg = dict(v_hat=tr["v_hat"], E_keV=tr["E_repr_keV"], L_ang=tr["L_ang"], r_mid=tr["r_mid"], elec_id=tr["elec_id"])
    for i in (0, 15, 16, 19):
        ref = oracle.brem_spectrum(oseg, d["Z"], d["n_ang3"], d["thickness"], n_hats[i], d["E_grid"], d["mu_grid"],
                                   int(d["Ne"]))
        assert np.max(np.abs(spec[i] - ref)) <= 1e-11 * np.max(ref), i


def test_pipeline_batch_of_zero_histories(cuda_device):
    """A batch of no histories: the transport writes no segments and the
    scorers, reading the segment count on the device, do no work."""
    import torch

    from pyrite_b200.configs import c1_hopg_20mev
    from pyrite_b200.pipeline import ScoringCase

    case = ScoringCase(c1_hopg_20mev(), precision="mixed", batch_histories=256, device=cuda_device)
    case.run_batch(0, 0)
    torch.cuda.synchronize()
    assert case.device_status() == 0
    assert int(case.seg_count.item()) == 0
    assert not torch.any(case.spec_cxr) and not torch.any(case.spec_brem)
    assert int(case.fates.sum().item()) == 0


def test_line_buffer_overflow_is_reported(cuda_device):
    import torch

    from pyrite_b200 import _lib as L
    from pyrite_b200.configs import c2_si_50mev
    from pyrite_b200.surrogate import _cxr_lines, transported_segments

    spec = c2_si_50mev(angular_shape=(1, 1))
    seg, n = transported_segments(spec, 32, seed=3, device=cuda_device)
    lines, n_ok = _cxr_lines(spec, seg, n, spec.n_hats, cuda_device, cap_per_pair=64)
    assert n_ok > 10
    cap = 5
    with pytest.raises(L.PyriteB200Error) as err:
        _cxr_lines(spec, seg, n, spec.n_hats, cuda_device, cap_per_pair=(cap + 0.5) / (n * len(spec.n_hats)))
    msg = str(err.value)
    # PB_DEV_QUEUE_OVERFLOW, and the counter kept counting past the capacity
    assert "status 4" in msg and f"{n_ok} lines for capacity {cap}" in msg
    torch.cuda.synchronize()


@pytest.mark.parametrize("lut", [False, True])
def test_step_limit_ends_every_history(lut, cuda_device):
    from pyrite_b200 import simulate_trajectories

    out = simulate_trajectories(20000.0, 64, 1.0e6, element="C", n_atoms_per_ang3=0.1133, max_steps=3,
                                lut=lut, device=cuda_device)
    assert out["n_step_limited"] == 64
    assert out["device_status"] & 1  # PB_DEV_STEP_LIMIT
