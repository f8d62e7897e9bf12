"""Surrogate kernels against plain PyTorch FP32 references.

- ``pb_mlp_features``: the feature map, against the same formula in torch.
- ``pb_mlp_infer`` + ``pb_mlp_head``: the fused tcgen05 inference (bf16
  activations, FP32 accumulation, tanh-form SiLU) against an FP32 torch
  forward pass on the same bf16-rounded weights, activations rounded to bf16
  between layers like the kernel's.
- One training step's gradients (tcgen05 GEMMs with fused SiLU' epilogues)
  against torch autograd in FP32 on the same bf16 values.
- ``pb_cxr_bin_lines``: coarse per-pair line binning against the oracle's
  FP64 sinc^2 antiderivative.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _segments(n, device, seed=0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    E = 45000.0 + 5000.0 * torch.rand(n, generator=g, dtype=torch.float64)
    th = 0.01 * torch.randn(n, 2, generator=g, dtype=torch.float64)
    v = torch.stack([th[:, 0], th[:, 1], torch.ones(n, dtype=torch.float64)], 1)
    v = v / v.norm(dim=1, keepdim=True)
    r = torch.zeros(n, 3, dtype=torch.float64)
    r[:, 2] = 5.0e6 * torch.rand(n, generator=g, dtype=torch.float64)
    L = 1.0e5 * (0.2 + torch.rand(n, generator=g, dtype=torch.float64))
    seg = {"r": r, "v": v, "L": L, "E": E, "id": torch.zeros(n, dtype=torch.int64)}
    return {k: t.to(device) for k, t in seg.items()}


class _Spec:
    """Minimal case stand-in for the feature map (beam along +z, 500 um slab)."""

    class beam:
        beam_dir = np.array([0.0, 0.0, 1.0])

    class stack:
        thickness = 5.0e6


def _torch_features(seg, uv, spec):
    from pyrite_b200.surrogate import E_HI_MEV, E_LO_MEV, THETA_MAX_RAD, _beam_axes

    e_x, e_y = (torch.as_tensor(a, dtype=torch.float32, device=seg["v"].device) for a in _beam_axes(spec))
    v = seg["v"].float()
    n_dir, n = uv.shape[0], v.shape[0]
    x = torch.zeros(n_dir, n, 16, device=v.device)
    lnlo, lnhi = np.log(E_LO_MEV), np.log(E_HI_MEV)
    x[:, :, 0] = 2.0 * (torch.log(seg["E"].float() * 1e-3) - lnlo) / (lnhi - lnlo) - 1.0
    x[:, :, 1] = (v @ e_x) / THETA_MAX_RAD
    x[:, :, 2] = (v @ e_y) / THETA_MAX_RAD
    x[:, :, 3] = 2.0 * (seg["r"][:, 2].float() / spec.stack.thickness).clamp(0, 1) - 1.0
    x[:, :, 4] = uv[:, 0:1]
    x[:, :, 5] = uv[:, 1:2]
    return x


def test_features_match_torch(cuda_device):
    import ctypes as C

    from pyrite_b200 import _lib as L
    from pyrite_b200.surrogate import _feature_args

    seg = _segments(1000, cuda_device)
    uv = torch.tensor([[0.1, -0.2], [0.7, 0.4]], device=cuda_device)
    a = _feature_args(_Spec, seg, 1000, uv)
    X = torch.empty(2000, 16, device=cuda_device, dtype=torch.bfloat16)
    w = torch.empty(2000, device=cuda_device)
    L.check(L.load().pb_mlp_features(C.byref(a), X.data_ptr(), w.data_ptr(), None), "pb_mlp_features")
    torch.cuda.synchronize()
    ref = _torch_features(seg, uv, _Spec).reshape(2000, 16)
    assert float((X.float() - ref).abs().max()) <= 0.01 * float(ref.abs().max())
    assert torch.allclose(w, seg["L"].float().repeat(2))


def _torch_forward_hsum(model, X, Lw):
    """FP32 forward on bf16 weights, bf16 activations between layers; sum L h4."""
    h = X.to(torch.bfloat16).float()
    for W, b in (("W1", "b1"), ("W2", "b2"), ("W3", "b3"), ("W4", "b4")):
        z = h @ model.Wb[W].float().t() + model.p[b]
        h = 0.5 * z * (1.0 + torch.tanh(0.5 * z))
        if W != "W4":
            h = h.to(torch.bfloat16).float()
    return (Lw[:, None] * h).sum(0)


def test_infer_matches_torch(cuda_device):
    from pyrite_b200.surrogate import HIDDEN, Surrogate

    model = Surrogate(cuda_device, seed=3)
    with torch.no_grad():
        for k in ("b1", "b2", "b3", "b4", "b5"):
            model.p[k].normal_(0.0, 0.1)
    model.repack()
    n = 1000
    seg = _segments(n, cuda_device, seed=1)
    uv = torch.tensor([[0.1, -0.2], [0.7, 0.4], [-0.9, 0.9]], device=cuda_device)
    hsum = torch.zeros(3, HIDDEN, device=cuda_device, dtype=torch.float64)
    lsum = torch.zeros(3, device=cuda_device, dtype=torch.float64)
    status = torch.zeros(1, device=cuda_device, dtype=torch.int32)
    spec = torch.zeros(3, model.n_out, device=cuda_device, dtype=torch.float64)
    a = model.infer_args(_Spec, seg, n, uv, hsum, lsum, status=status)
    model.score(a, spec, hsum, lsum)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    X = _torch_features(seg, uv, _Spec)
    Lw = seg["L"].float()
    for d in range(3):
        ref = _torch_forward_hsum(model, X[d], Lw)
        err = float((hsum[d].float() - ref).abs().max())
        assert err <= 3e-2 * float(ref.abs().max()), (d, err, float(ref.abs().max()))
        assert abs(float(lsum[d]) - float(seg["L"].sum())) <= 1e-6 * float(seg["L"].sum())  # float block sums
        head = model.W5r @ hsum[d].float() + model.p["b5"] * float(lsum[d])
        assert torch.allclose(spec[d].float(), head, rtol=1e-4, atol=1e-4 * float(head.abs().max()))


def test_training_gradients_match_autograd(cuda_device):
    from pyrite_b200.surrogate import Surrogate

    model = Surrogate(cuda_device, seed=5)
    B = 1024
    g = torch.Generator(device=cuda_device).manual_seed(7)
    X = torch.zeros(B, 16, device=cuda_device)
    X[:, :6] = torch.rand(B, 6, device=cuda_device, generator=g) * 2 - 1
    Xb = X.to(torch.bfloat16)
    T = (0.5 * torch.randn(B, model.n_out, device=cuda_device, generator=g)).to(torch.bfloat16)
    ws = model._workspace(B)
    params_before = {k: v.clone() for k, v in model.p.items()}
    model.train_step(Xb, Xb.t().contiguous(), T, ws, lr=0.0)
    torch.cuda.synchronize()
    assert int(ws["status"].item()) == 0
    # autograd reference on the same bf16 weights, FP32 arithmetic
    P = {k: v.clone().requires_grad_(True) for k, v in params_before.items()}
    h = Xb.float()
    for W, b in (("W1", "b1"), ("W2", "b2"), ("W3", "b3"), ("W4", "b4")):
        h = torch.nn.functional.silu(h @ P[W].to(torch.bfloat16).float().t() + P[b])
    Y = h @ P["W5"].to(torch.bfloat16).float().t() + P["b5"]
    loss = ((Y - T.float()) ** 2).mean()
    loss.backward()
    for k in ("W5", "b5", "W4", "b4", "W2", "W1", "b1"):
        ref, got = P[k].grad, model.g[k]
        rel = float((got - ref).norm() / ref.norm().clamp_min(1e-30))
        assert rel < 5e-2, (k, rel)


def test_bin_lines_matches_oracle(cuda_device):
    import oracle
    from pyrite_b200 import _lib as L

    rng = np.random.default_rng(3)
    n = 4000
    E = rng.uniform(2000.0, 58000.0, n)
    a = 10.0 ** rng.uniform(-5.0, -1.5, n)
    w = rng.uniform(0.1, 1.0, n)
    dirs = rng.integers(0, 3, n).astype(np.int32)
    segs = rng.integers(0, 5, n).astype(np.int64)
    lo, width, n_bins = 985.6, 115.2, 512
    dev = cuda_device
    tE, ta, tw = (torch.as_tensor(x, dtype=torch.float64, device=dev) for x in (E, a, w))
    td = torch.as_tensor(dirs, dtype=torch.int32, device=dev)
    ts = torch.as_tensor(segs, dtype=torch.int64, device=dev)
    out = torch.zeros(15, n_bins, device=dev)
    L.check(L.load().pb_cxr_bin_lines(n, tE.data_ptr(), ta.data_ptr(), tw.data_ptr(), td.data_ptr(), ts.data_ptr(),
                                      0, 3, 5, lo, width, n_bins, out.data_ptr(), None), "pb_cxr_bin_lines")
    torch.cuda.synchronize()
    edges = lo + width * np.arange(n_bins + 1)
    ref = np.zeros((15, n_bins))
    for i in range(n):
        c = int(np.floor((E[i] - lo) / width))
        K = min(max(int(np.ceil(64.0 * np.pi / (a[i] * width))), 1), 64)
        b0, b1 = max(c - K, 0), min(c + K, n_bins - 1)
        if b1 < b0:
            continue
        x = a[i] * (edges[b0:b1 + 2] - E[i]) / np.pi
        R = np.array([oracle.sincsq_tail(float(v)) for v in x])
        m = R[1:] - R[:-1] + ((x[:-1] < 0) & (x[1:] >= 0))
        ref[dirs[i] * 5 + segs[i], b0:b1 + 1] += w[i] * np.pi / a[i] * m / width
    got = out.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 2e-4 * np.max(np.abs(ref))


def test_group_mse_grad_matches_torch(cuda_device):
    from pyrite_b200 import mlp

    B, S, C = 2048, 256, 512
    g = torch.Generator(device=cuda_device).manual_seed(11)
    Y = torch.randn(B, C, device=cuda_device, generator=g)
    T = torch.randn(B, C, device=cuda_device, generator=g).to(torch.bfloat16)
    w = torch.rand(B, device=cuda_device, generator=g)
    w = (w.view(-1, S) / w.view(-1, S).sum(1, keepdim=True)).reshape(-1).contiguous()
    dY = torch.empty(B, C, device=cuda_device, dtype=torch.bfloat16)
    dYt = torch.empty(C, B, device=cuda_device, dtype=torch.bfloat16)
    loss = torch.zeros(1, device=cuda_device)
    gs = 2.0 / ((B // S) * C)
    mlp.group_mse_grad(Y, T, w, S, 1.0, gs, dY, dYt, loss)
    torch.cuda.synchronize()
    A_hat = (w[:, None] * Y).view(-1, S, C).sum(1)
    A = (w[:, None] * T.float()).view(-1, S, C).sum(1)
    d = A_hat - A
    ref = gs * w[:, None] * d.repeat_interleave(S, dim=0)
    assert float((dY.float() - ref).abs().max()) <= 1e-2 * float(ref.abs().max())
    assert torch.equal(dYt, dY.t().contiguous())
    assert abs(float(loss) - float((d * d).sum())) <= 1e-3 * float((d * d).sum())


def test_control_variate_identity_and_accuracy(cuda_device):
    """With every history in the exact sub-sample the estimator is the exact
    coarse spectrum; with every 8th it stays within a few percent of it even
    for a barely trained surrogate (the estimator is unbiased)."""
    from pyrite_b200 import configs
    from pyrite_b200 import surrogate as S
    from pyrite_b200.pipeline import ScoringCase

    spec = configs.c2_si_50mev(seed=7)
    data = S.make_training_set(spec, n_seg=2048, n_dir=64, dir_chunk=64, seed=3, device=cuda_device)
    model = S.Surrogate(cuda_device, seed=0)
    model.train(data, epochs=2, batch=4096)
    H = 2048
    ce = ScoringCase(spec, precision="mixed", batch_histories=H, device=cuda_device)
    for i in range(2):
        ce.run_batch(i * H, H)
    out = {}
    for stride in (1, 8):
        cs = ScoringCase(spec, precision="mixed", batch_histories=H, device=cuda_device)
        cs.use_surrogate([model], exact_stride=stride)
        for i in range(2):
            cs.run_batch(i * H, H)
        out[stride] = cs.surrogate_spectrum()
        assert cs.device_status() == 0
    exact = (cs.coarse(ce.spec_cxr) / ce.histories).cpu().numpy()
    peak = np.max(np.abs(exact))
    assert peak > 0
    assert np.max(np.abs(out[1] - exact)) <= 1e-5 * peak
    assert np.max(np.abs(out[8].sum(0) - exact.sum(0))) <= 0.05 * np.max(exact.sum(0))


def test_single_tile_inference_variant_matches_torch(cuda_device):
    """The single-tile inference kernel (``PB_MLP_INFER=serial``, the
    reference point of the ping-pong kernel; the variant is read once per
    process) passes the same check against the torch forward pass."""
    import os
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, PB_MLP_INFER="serial")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider",
                        str(root / "tests" / "test_gpu_surrogate.py"), "-k", "test_infer_matches_torch"],
                       cwd=root, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "1 passed" in r.stdout


def test_error_gate_falls_back_to_the_exact_scorer(cuda_device):
    """A barely trained surrogate under a tolerance no control variate can
    meet (1e-6): after the probe batches every tile moves to the exact
    scorer, the batches already run are replayed for it, and the run's
    spectrum equals the exact mixed scorer's on the same histories, within
    1e-8 of the peak: the same kernel on the same segments, but the mixed
    scorer sums FP32 partials with shared-memory atomics and the transport
    appends segments in warp-atomic order, so the float sums group
    differently from run to run (measured 1e-9); the replay leaves the
    tallies counted once."""
    from pyrite_b200 import configs
    from pyrite_b200 import surrogate as S
    from pyrite_b200.pipeline import ScoringCase

    spec = configs.c2_si_50mev(seed=7)
    data = S.make_training_set(spec, n_seg=1024, n_dir=16, dir_chunk=16, seed=3, device=cuda_device)
    model = S.Surrogate(cuda_device, seed=0)
    model.train(data, epochs=1, batch=1024)
    H = 2048
    ce = ScoringCase(spec, precision="mixed", batch_histories=H, device=cuda_device)
    cs = ScoringCase(spec, precision="mixed", batch_histories=H, device=cuda_device)
    cs.use_surrogate([model], exact_stride=8, tol=1e-6, probe_batches=3)
    for i in range(5):
        ce.run_batch(i * H, H)
        cs.run_batch(i * H, H)
    rep = cs.surrogate_report()
    assert rep["checked"] and rep["fallback_tiles"] == list(range(cs.n_dir))
    assert all(e > 1e-6 for e in rep["estimate_per_tile"])
    got, ref = cs.results(), ce.results()
    peak = np.max(np.abs(ref["cxr"]))
    assert peak > 0
    assert np.max(np.abs(got["cxr"] - ref["cxr"])) <= 1e-8 * peak
    coarse_ref = ref["cxr"].reshape(cs.n_dir, model.n_out, -1).mean(-1)
    assert np.max(np.abs(cs.surrogate_spectrum() - coarse_ref)) <= 1e-8 * peak
    for k in ("fates", "exit_E", "exit_theta"):
        np.testing.assert_array_equal(got[k], ref[k])
    assert cs.device_status() == 0


def test_error_gate_keeps_a_trained_surrogate(cuda_device):
    """A briefly trained surrogate (2 epochs on 131k pairs) on 65,536
    histories under a 5 % tolerance: every tile's estimated error is below
    it, no tile falls back, and the estimate is calibrated against the actual
    worst-bin error of the control-variate spectrum against the exact scorer
    on the same histories: their ratio is 1 in the median (within a factor
    2) and within a factor 4 on every tile (four probe batches leave each
    bin's variance three degrees of freedom; measured ratios 0.7-3.2). The
    run's audit (surrogate alone on the sub-sample) is reported."""
    from pyrite_b200 import configs
    from pyrite_b200 import surrogate as S
    from pyrite_b200.pipeline import ScoringCase

    spec = configs.c2_si_50mev(seed=7)
    data = S.make_training_set(spec, n_seg=2048, n_dir=64, dir_chunk=64, seed=3, device=cuda_device)
    model = S.Surrogate(cuda_device, seed=0)
    model.train(data, epochs=2, batch=4096)
    H = 16384
    ce = ScoringCase(spec, precision="mixed", batch_histories=H, device=cuda_device)
    cs = ScoringCase(spec, precision="mixed", batch_histories=H, device=cuda_device)
    cs.use_surrogate([model], exact_stride=8, tol=0.05, probe_batches=4)
    for i in range(4):
        ce.run_batch(i * H, H)
        cs.run_batch(i * H, H)
    rep = cs.surrogate_report()
    est = np.array(rep["estimate_per_tile"])
    assert rep["checked"] and rep["fallback_tiles"] == [], est
    exact = ce.results()["cxr"].reshape(cs.n_dir, model.n_out, -1).mean(-1)
    actual = np.max(np.abs(cs.surrogate_spectrum() - exact), axis=1) / np.max(np.abs(exact), axis=1)
    ratio = actual / est
    assert 0.5 <= np.median(ratio) <= 2.0 and np.all((ratio > 0.25) & (ratio < 4.0)), (actual, est)
    audit = np.array(rep["audit_surrogate_alone_per_tile"])
    assert np.all((audit > 0) & (audit < 1)), audit


def test_tile_factored_form_heads_and_gradients(cuda_device):
    """The tile-factored surrogate (one 512-bin head per tile on shared
    segment features): one inference pass over the segments (direction
    features zero) and every tile's head on the one activation sum equals
    the torch forward of the same bf16 model per tile; its training step's
    output-layer gradient (N = tiles x 512) matches autograd."""
    from pyrite_b200.surrogate import HIDDEN, Surrogate

    n_tiles = 4
    model = Surrogate(cuda_device, seed=11, n_tiles=n_tiles)
    assert model.n_out == n_tiles * 512 and model.n_bins == 512
    with torch.no_grad():
        for k in ("b1", "b2", "b3", "b4", "b5"):
            model.p[k].normal_(0.0, 0.1)
    model.repack()
    n = 1000
    seg = _segments(n, cuda_device, seed=2)
    uv = torch.zeros(1, 2, device=cuda_device)
    hsum = torch.zeros(1, HIDDEN, device=cuda_device, dtype=torch.float64)
    lsum = torch.zeros(1, device=cuda_device, dtype=torch.float64)
    status = torch.zeros(1, device=cuda_device, dtype=torch.int32)
    spec = torch.zeros(1, model.n_out, device=cuda_device, dtype=torch.float64)
    a = model.infer_args(_Spec, seg, n, uv, hsum, lsum, status=status)
    model.score(a, spec, hsum, lsum)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ref_h = _torch_forward_hsum(model, _torch_features(seg, uv, _Spec)[0], seg["L"].float())
    assert float((hsum[0].float() - ref_h).abs().max()) <= 3e-2 * float(ref_h.abs().max())
    tiles = spec.view(n_tiles, 512).float()
    for t in range(n_tiles):
        W = model.W5r[t * 512:(t + 1) * 512]
        head = W @ hsum[0].float() + model.p["b5"][t * 512:(t + 1) * 512] * float(lsum[0])
        assert torch.allclose(tiles[t], head, rtol=1e-4, atol=1e-4 * float(head.abs().max()))
    # one training step: the output layer's gradient against autograd
    B = 1024
    g = torch.Generator(device=cuda_device).manual_seed(13)
    X = torch.zeros(B, 16, device=cuda_device)
    X[:, :4] = torch.rand(B, 4, device=cuda_device, generator=g) * 2 - 1
    Xb = X.to(torch.bfloat16)
    T = (0.5 * torch.randn(B, model.n_out, device=cuda_device, generator=g)).to(torch.bfloat16)
    ws = model._workspace(B)
    P = {k: v.clone().requires_grad_(True) for k, v in model.p.items()}
    model.train_step(Xb, Xb.t().contiguous(), T, ws, lr=0.0)
    torch.cuda.synchronize()
    assert int(ws["status"].item()) == 0
    h = Xb.float()
    for Wn, bn in (("W1", "b1"), ("W2", "b2"), ("W3", "b3"), ("W4", "b4")):
        h = torch.nn.functional.silu(h @ P[Wn].to(torch.bfloat16).float().t() + P[bn])
        h = h.to(torch.bfloat16).float()
    Y = h @ P["W5"].to(torch.bfloat16).float().t() + P["b5"]
    loss = ((Y - T.float()) ** 2).mean()
    loss.backward()
    gW5 = model.g["W5"]
    rel = float((gW5 - P["W5"].grad).norm() / P["W5"].grad.norm())
    assert rel < 2e-2, rel
