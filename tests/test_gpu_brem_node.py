"""Depth-node form of the mixed bremsstrahlung scorer (pb_brem_node.cu).

The form scores the segments of the batch's top electron-energy window
through per-segment depth moments and one contraction per photon energy; the
segments outside the window, and every segment where a device-side check
turns the form off, take the per-(segment, energy) kernels. The tests compare
the mixed scorer with the FP64 per-pair scorer (the reference's expression)
on the same segments, check that the form engaged (or stood down) as the
inputs demand, and cover the left-out list and the fallbacks.
"""

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

SYM = {6.0: "C", 8.0: "O", 14.0: "Si", 74.0: "W"}


def _golden_segments(case):
    d = golden(f"brem_{case}")
    tr = golden(f"transport_{d['transport']}")
    seg = dict(v_hat=tr["v_hat"], E_repr_keV=tr["E_repr_keV"], L_ang=tr["L_ang"], r_mid=tr["r_mid"],
               elec_id=tr["elec_id"], Ne=int(d["Ne"]), thickness_ang=float(d["thickness"]))
    comp = [(SYM[float(z)], float(n)) for z, n in zip(d["Z"], d["n_ang3"])]
    return d, seg, comp


def _directions(kind):
    from pyrite_b200 import configs

    tiles = configs.c2_si_50mev().n_hats
    if kind == "tiles":
        return tiles
    if kind == "spread5pct":
        th = np.linspace(0.30, 0.55, 16)
        return np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], axis=1)
    n = tiles.copy()
    n[::2, 2] *= -1.0  # both exit faces
    return n


def _worst(a, b):
    worst = 0.0
    for i in range(a.shape[0]):
        peak = np.max(np.abs(b[i]))
        assert peak > 0
        worst = max(worst, float(np.max(np.abs(a[i] - b[i])) / peak))
    return worst


@pytest.mark.parametrize("kind", ["tiles", "spread5pct", "both_faces"])
def test_node_form_against_fp64(kind, cuda_device):
    """20 MeV electrons in carbon, every direction set the per-pair forms
    cover: the node form against the FP64 scorer within 1e-6 of each
    direction's peak (interpolation below 2e-9, float moment sums ~1e-7)."""
    from pyrite_b200 import mc_brem_spectrum

    d, seg, comp = _golden_segments("c20")
    n_hats = _directions(kind)
    kw = dict(composition=comp, n_hat=n_hats, mu=d["mu_grid"], device=cuda_device)
    ref = mc_brem_spectrum(seg, d["E_grid"], precision="fp64", **kw)
    node = mc_brem_spectrum(seg, d["E_grid"], precision="mixed", **kw)
    pair = mc_brem_spectrum(seg, d["E_grid"], precision="mixed", depth_nodes=False, **kw)
    assert _worst(node, ref) <= 1e-6
    assert _worst(pair, ref) <= 1e-4


def test_node_form_two_elements_against_fp64(cuda_device):
    """SiO2 at 300 keV: two elements in the shared accumulator; the segments
    below the window go to the per-pair kernels."""
    from pyrite_b200 import mc_brem_spectrum

    d, seg, comp = _golden_segments("sio2")
    kw = dict(composition=comp, n_hat=d["n_hat"], mu=d["mu_grid"], device=cuda_device)
    ref = mc_brem_spectrum(seg, d["E_grid"], precision="fp64", **kw)
    node = mc_brem_spectrum(seg, d["E_grid"], precision="mixed", **kw)
    peak = np.max(np.abs(ref))
    assert np.max(np.abs(node - ref)) <= 1e-6 * peak


def test_node_form_left_out_segments(cuda_device):
    """A third of the segments moved well below the window: they reach the
    per-pair kernels through the left-out list, the rest stay in the node
    form, and the sum matches FP64 at the per-pair form's tolerance."""
    from pyrite_b200 import mc_brem_spectrum

    d, seg, comp = _golden_segments("c20")
    seg = dict(seg)
    E = np.array(seg["E_repr_keV"], dtype=np.float64)
    E[::3] *= 0.6
    seg["E_repr_keV"] = E
    n_hats = _directions("tiles")
    kw = dict(composition=comp, n_hat=n_hats, mu=d["mu_grid"], device=cuda_device)
    ref = mc_brem_spectrum(seg, d["E_grid"], precision="fp64", **kw)
    node = mc_brem_spectrum(seg, d["E_grid"], precision="mixed", **kw)
    assert _worst(node, ref) <= 1e-4


def test_node_form_stands_down_for_grazing_directions(cuda_device):
    """A direction almost in the slab's plane needs more depth cells than
    the form holds: it stands down on the device and the per-pair kernels
    score every segment."""
    from pyrite_b200 import mc_brem_spectrum

    d, seg, comp = _golden_segments("c20")
    n_hats = _directions("tiles").copy()
    n_hats[0] = [np.sqrt(1.0 - 1e-8), 0.0, 1e-4]
    kw = dict(composition=comp, n_hat=n_hats, mu=d["mu_grid"], device=cuda_device)
    ref = mc_brem_spectrum(seg, d["E_grid"], precision="fp64", **kw)
    node = mc_brem_spectrum(seg, d["E_grid"], precision="mixed", **kw)
    assert _worst(node, ref) <= 1e-4


def test_node_form_engages_on_the_bench_scene(cuda_device):
    """The 50 MeV Si scene through the pipeline: the form scores the batch
    with (almost) every segment in its window, and its bremsstrahlung agrees
    with the FP64 scorer on the same segments within 1e-6 of each tile's
    peak."""
    import ctypes as C

    import torch

    from pyrite_b200 import _lib as L
    from pyrite_b200 import configs
    from pyrite_b200.pipeline import ScoringCase

    spec = configs.c2_si_50mev(seed=7)
    case = ScoringCase(spec, precision="mixed", batch_histories=1024, device=cuda_device)
    case.run_batch(0, 1024)
    torch.cuda.synchronize()
    mixed = case.spec_brem.cpu().numpy().copy()
    st = case.brem_node_state()
    n_seg = int(case.seg_count.item())
    assert len(st) == 1 and st[0]["ok"], st
    assert st[0]["left_out"] <= n_seg // 100, (st, n_seg)
    assert 1 <= st[0]["n_cells"] <= 64
    # the FP64 per-pair scorer on the same segment list
    b = L.PbBremArgs.from_buffer_copy(case.bargs)
    b.precision = L.PB_FP64
    b.work, b.work_bytes = None, 0
    ref = torch.zeros_like(case.spec_brem)
    b.spec = ref.data_ptr()
    lib = L.load()
    L.check(lib.pb_brem_score(C.byref(b), torch.cuda.current_stream().cuda_stream), "pb_brem_score")
    torch.cuda.synchronize()
    assert _worst(mixed, ref.cpu().numpy()) <= 1e-6
