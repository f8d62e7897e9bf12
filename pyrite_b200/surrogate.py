"""BF16 MLP surrogate of the per-segment PXR+CBS spectrum, trained and run on tcgen05.

Model: 6 inputs -> 4 hidden layers of 256 SiLU units -> linear outputs,
bf16 weights and activations, FP32 accumulation (``pb_mlp_*`` kernels). The
inputs are the kernel's feature map (``pb_mlp_infer_args``): log energy, the
two transverse angles of the segment direction, depth, and a direction's
detector coordinates. The outputs are the segment's line spectrum per unit
path length on a coarse uniform grid of 512 bins spanning the case's bins
(each coarse bin = 4 fine bins of the 2048-bin grid), in units of the exact
scorer's spectrum times ``t_scale``. Two forms:

- pairwise (``Surrogate()``): one (segment, direction) pair per row, 512
  outputs; any direction of the detector plane;
- tile-factored (``Surrogate(n_tiles=T)``): the direction inputs are zero
  and the output layer holds one 512-bin head per tile of the case
  (T x 512 outputs); the network then runs once per segment and the heads
  apply to the one summed activation (``make_tile_training_set``).

Training pairs come from the exact FP64 reflection sum (``pb_cxr_score``
with its line buffer, ``pb_cxr_bin_lines``): segments of the case's own
transport (so the input distribution is the workload's) against uniformly
random detector points. Inference accumulates, per direction, the
length-weighted sum of the last hidden layer (``pb_mlp_infer``) and applies
the linear output layer once (``pb_mlp_head``): for a linear head the sum of
per-pair outputs is the head of the summed activations.

``audit`` compares the surrogate's aggregate spectrum with the exact sum on
held-out segments. In a run (``pipeline.ScoringCase.use_surrogate``) the
surrogate is paired with an exact control variate on a sub-sample of every
batch; ``control_variate_error`` estimates, per detector tile, the error of
that estimate from the batch-to-batch scatter of the sub-sample residuals,
and tiles whose estimate exceeds the tolerance (1 % of the tile's peak) fall
back to the exact scorer for the whole run.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from . import mlp
from .api import _fill_tables, _Holder, _ptr
from .detector import directions_at, tile_uv
from .tables import energy_bin_edges, line_keep_window, reflection_rows

E_LO_MEV, E_HI_MEV = 5.0, 100.0
THETA_MAX_RAD = 0.02
HIDDEN = 256
K_IN = 16          # 6 features, zero padded to one K=16 MMA
N_IN = 6


@dataclass(frozen=True)
class CoarseGrid:
    lo_eV: float
    width_eV: float
    n_bins: int

    @classmethod
    def of(cls, E_grid_eV, n_bins=512):
        edges = energy_bin_edges(np.asarray(E_grid_eV, dtype=float))
        return cls(float(edges[0]), float((edges[-1] - edges[0]) / n_bins), int(n_bins))


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _beam_axes(spec):
    """Transverse axes of the beam in the sample frame (the angle features)."""
    d = np.asarray(spec.beam.beam_dir, dtype=float)
    d = d / np.linalg.norm(d)
    ref = np.array([0.0, 1.0, 0.0]) if abs(d[1]) < 0.9 else np.array([1.0, 0.0, 0.0])
    e_x = np.cross(ref, d)
    e_x /= np.linalg.norm(e_x)
    e_y = np.cross(d, e_x)
    return e_x, e_y


class Surrogate:
    """Parameters, optimiser state and the packed weight copies of the MLP."""

    def __init__(self, device, n_out=512, seed=0, n_tiles=1):
        """``n_out`` coarse bins per output spectrum. ``n_tiles`` > 1 builds
        the tile-factored form: the hidden layers see the segment alone (the
        direction features are zero) and the output layer holds one linear
        head of ``n_out`` bins per detector tile, so a segment's hidden
        activations are computed once for all tiles."""
        self.device = torch.device(device)
        self.n_tiles = int(n_tiles)
        self.n_bins = int(n_out)
        self.n_out = self.n_bins * self.n_tiles
        shapes = [("W1", (HIDDEN, K_IN)), ("b1", (HIDDEN,)), ("W2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
                  ("W3", (HIDDEN, HIDDEN)), ("b3", (HIDDEN,)), ("W4", (HIDDEN, HIDDEN)), ("b4", (HIDDEN,)),
                  ("W5", (self.n_out, HIDDEN)), ("b5", (self.n_out,))]
        self.shapes = shapes
        n = sum(int(np.prod(s)) for _, s in shapes)
        self.flat = torch.zeros(n, device=self.device)
        self.grad = torch.zeros(n, device=self.device)
        self.m = torch.zeros(n, device=self.device)
        self.v = torch.zeros(n, device=self.device)
        self.p = self._views(self.flat)
        self.g = self._views(self.grad)
        gen = torch.Generator(device="cpu").manual_seed(seed)
        for name, shape in shapes:
            if name.startswith("W"):
                fan_in = N_IN if name == "W1" else shape[1]
                w = torch.randn(shape, generator=gen) * (1.0 / math.sqrt(fan_in))
                if name == "W1":
                    w[:, N_IN:] = 0.0
                if name == "W5":
                    w *= 0.1
                self.p[name].copy_(w)
        bf = torch.bfloat16
        dev = self.device
        self.Wb = {k: torch.zeros(self.p[k].shape, device=dev, dtype=bf) for k in ("W1", "W2", "W3", "W4", "W5")}
        self.Wt = {k: torch.zeros(self.p[k].shape[::-1], device=dev, dtype=bf) for k in ("W2", "W3", "W4", "W5")}
        self.w1p = torch.zeros(HIDDEN * 16 * 2, device=dev, dtype=torch.uint8)
        self.wp = [torch.zeros(HIDDEN * HIDDEN * 2, device=dev, dtype=torch.uint8) for _ in range(3)]
        self.t_scale = 1.0
        self.step = 0
        self.repack()

    def _views(self, flat):
        out, o = {}, 0
        for name, shape in self.shapes:
            n = int(np.prod(shape))
            out[name] = flat[o:o + n].view(shape)
            o += n
        return out

    def repack(self):
        """bf16 training copies (row-major and transposed) and the inference packing."""
        for k in ("W1", "W2", "W3", "W4", "W5"):
            mlp.pack(self.p[k], self.Wb[k], self.Wt.get(k), pad_cols=self.p[k].shape[1])
        # The output layer as trained: its bf16 rounding, in FP32 for the head.
        self.W5r = self.Wb["W5"].float()
        lib = L.load()
        s = _stream()
        L.check(lib.pb_mlp_pack_umma(K_IN, 16, self.p["W1"].data_ptr(), self.w1p.data_ptr(), s), "pb_mlp_pack_umma")
        for i, k in enumerate(("W2", "W3", "W4")):
            L.check(lib.pb_mlp_pack_umma(HIDDEN, 64, self.p[k].data_ptr(), self.wp[i].data_ptr(), s),
                    "pb_mlp_pack_umma")

    # ------------------------------------------------------------------
    # training
    # ------------------------------------------------------------------
    def _workspace(self, B):
        dev, f32, bf = self.device, torch.float32, torch.bfloat16
        ws = {"B": B}
        for i in range(1, 5):
            ws[f"Z{i}"] = torch.empty(B, HIDDEN, device=dev, dtype=f32)
            ws[f"H{i}"] = torch.empty(B, HIDDEN, device=dev, dtype=bf)
            ws[f"H{i}t"] = torch.empty(HIDDEN, B, device=dev, dtype=bf)
        ws["Y"] = torch.empty(B, self.n_out, device=dev, dtype=f32)
        ws["dY"] = torch.empty(B, self.n_out, device=dev, dtype=bf)
        ws["dYt"] = torch.empty(self.n_out, B, device=dev, dtype=bf)
        ws["dZ"] = torch.empty(B, HIDDEN, device=dev, dtype=f32)
        ws["dZb"] = [torch.empty(B, HIDDEN, device=dev, dtype=bf) for _ in range(2)]
        ws["dZt"] = torch.empty(HIDDEN, B, device=dev, dtype=bf)
        ws["loss"] = torch.zeros(1, device=dev, dtype=f32)
        ws["status"] = torch.zeros(1, device=dev, dtype=torch.int32)
        return ws

    def train_step(self, X, Xt, T, ws, lr, wd=0.0, b1=0.9, b2=0.999, eps=1e-8, group=None, grad_hook=None):
        """One Adam step on the batch X [B,16] bf16 (Xt its transpose view
        [16, B] with any row stride), T [B, n_out] bf16 scaled targets.

        ``group=(S, w)`` switches the loss from per-pair MSE to the MSE of
        group aggregates: rows in consecutive groups of S share a direction,
        w [B] are their normalised length weights."""
        B = ws["B"]
        p, g, st = self.p, self.g, ws["status"]
        self.grad.zero_()
        # forward
        prev = X
        for i, (W, b) in enumerate((("W1", "b1"), ("W2", "b2"), ("W3", "b3"), ("W4", "b4")), start=1):
            mlp.gemm(prev, self.Wb[W], bias=p[b], act=1, out_f32=ws[f"Z{i}"], out_bf16=ws[f"H{i}"],
                     out_bf16_t=ws[f"H{i}t"], status=st)
            prev = ws[f"H{i}"]
        mlp.gemm(prev, self.Wb["W5"], bias=p["b5"], out_f32=ws["Y"], status=st)
        # loss gradient: d/dY of mean (Y - T)^2 over B x n_out
        if group is None:
            mlp.mse_grad(ws["Y"], T, 1.0, 2.0 / (B * self.n_out), ws["dY"], ws["dYt"], ws["loss"])
        else:
            S, w = group
            mlp.group_mse_grad(ws["Y"], T, w, S, 1.0, 2.0 / ((B // S) * self.n_out), ws["dY"], ws["dYt"], ws["loss"])
        # backward
        mlp.gemm(ws["dYt"], ws["H4t"], out_f32=g["W5"], M=self.n_out, N=HIDDEN, K=B, status=st)
        dy32 = ws["Y"]  # reuse as FP32 dY for the bias gradient
        dy32.copy_(ws["dY"])
        mlp.colsum(dy32, g["b5"])
        up, up_t = ws["dY"], self.Wt["W5"]
        for i in range(4, 0, -1):
            dzb = ws["dZb"][i % 2]
            mlp.gemm(up, up_t, dsilu_z=ws[f"Z{i}"], out_f32=ws["dZ"], out_bf16=dzb, out_bf16_t=ws["dZt"], status=st)
            mlp.colsum(ws["dZ"], g[f"b{i}"])
            a_prev_t = ws[f"H{i - 1}t"] if i > 1 else Xt
            mlp.gemm(ws["dZt"], a_prev_t, out_f32=g[f"W{i}"], M=HIDDEN, N=K_IN if i == 1 else HIDDEN, K=B, status=st)
            if i > 1:
                up, up_t = dzb, self.Wt[f"W{i}"]
        if grad_hook is not None:
            grad_hook(self.grad)
        self.step += 1
        mlp.adam(self.flat, self.grad, self.m, self.v, lr, b1, b2, eps, wd, self.step)
        self.repack()

    def train(self, data, *, epochs=3, batch=8192, lr=2e-3, lr_final=1e-4, log=None, max_retries=3,
              process_group=None):
        """Adam over the pre-shuffled dataset ``data`` (``make_training_set``).

        An epoch whose loss is not finite (a divergent step) is undone: the
        parameters and Adam moments go back to the end of the previous epoch,
        the learning-rate schedule is halved, and the epoch runs again (at
        most ``max_retries`` times in all).

        ``process_group`` trains data-parallel: every rank holds its own
        shard of the data (same size on every rank) and the same initial
        parameters, the gradient is averaged over the group before each
        Adam step (``shard.average_gradients``), and the epoch loss is the
        group's, so every rank takes the same steps, retries included."""
        import torch.distributed as dist

        from .shard import average_gradients

        hook = None
        world = 1
        if process_group is not None:
            world = dist.get_world_size(process_group)
            hook = lambda g: average_gradients(g, process_group)  # noqa: E731
        X, Xt, T = data["X"], data["Xt"], data["T"]
        self.t_scale = float(data["t_scale"])
        N = X.shape[0] // batch * batch
        if world > 1:
            # the same number of steps on every rank; one target scale (rank 0's)
            nt = torch.tensor([N], device=self.device, dtype=torch.int64)
            dist.all_reduce(nt, op=dist.ReduceOp.MIN, group=process_group)
            N = int(nt.item())
        ws = self._workspace(batch)
        per_epoch = N // batch
        steps = epochs * per_epoch
        losses = []
        self.retries = 0
        scale = 1.0
        ep = 0
        while ep < epochs:
            snap = (self.flat.clone(), self.m.clone(), self.v.clone(), self.step)
            ws["loss"].zero_()
            k = ep * per_epoch
            for b0 in range(0, N, batch):
                frac = k / max(steps - 1, 1)
                lr_k = scale * lr * (lr_final / lr) ** frac
                self.train_step(X[b0:b0 + batch], Xt[:, b0:b0 + batch], T[b0:b0 + batch], ws, lr_k,
                                grad_hook=hook)
                k += 1
            torch.cuda.synchronize(self.device)
            if world > 1:
                red = torch.stack([ws["loss"].reshape(()).double(),
                                   (~torch.isfinite(self.flat)).any().double()])
                dist.all_reduce(red, group=process_group)
                loss = float(red[0].item()) / (world * N * self.n_out)
                finite = bool(np.isfinite(loss)) and float(red[1].item()) == 0.0
            else:
                loss = float(ws["loss"].item()) / (N * self.n_out)
                finite = bool(np.isfinite(loss)) and bool(torch.isfinite(self.flat).all().item())
            if not finite and self.retries < max_retries:
                self.flat.copy_(snap[0])
                self.m.copy_(snap[1])
                self.v.copy_(snap[2])
                self.step = snap[3]
                self.repack()
                self.retries += 1
                scale *= 0.5
                if log:
                    log(f"epoch {ep}: loss {loss} not finite; restarting it at {scale:g} x the learning rate")
                continue
            losses.append(loss)
            if log:
                log(f"epoch {ep}: mse {loss:.4e}")
            ep += 1
        if int(ws["status"].item()) != 0:
            raise L.PyriteB200Error(f"surrogate training: device status {int(ws['status'].item())}")
        return losses

    # ------------------------------------------------------------------
    # inference
    # ------------------------------------------------------------------
    def infer_args(self, spec, seg, n_seg, dir_uv, hsum, lsum, *, Ne=1 << 62, n_seg_device=None, status=None):
        a = L.PbMlpInferArgs()
        a.n_dir = int(dir_uv.shape[0])
        a.dir_uv = dir_uv.data_ptr()
        e_x, e_y = _beam_axes(spec)
        for i in range(3):
            a.e_x[i], a.e_y[i] = float(e_x[i]), float(e_y[i])
        a.theta_max, a.E_lo_MeV, a.E_hi_MeV = THETA_MAX_RAD, E_LO_MEV, E_HI_MEV
        a.thickness = float(spec.stack.thickness)
        a.Ne = int(Ne)
        a.n_seg = int(n_seg)
        a.r_mid, a.v_hat, a.L, a.E_keV, a.elec_id = (seg["r"].data_ptr(), seg["v"].data_ptr(), seg["L"].data_ptr(),
                                                     seg["E"].data_ptr(), seg["id"].data_ptr())
        a.n_seg_device = n_seg_device.data_ptr() if n_seg_device is not None else None
        a.w1_packed = self.w1p.data_ptr()
        for i in range(3):
            a.w_packed[i] = self.wp[i].data_ptr()
        for i, k in enumerate(("b1", "b2", "b3", "b4")):
            a.bias[i] = self.p[k].data_ptr()
        a.hsum, a.lsum = hsum.data_ptr(), lsum.data_ptr()
        a.status = status.data_ptr() if status is not None else None
        return a

    def score(self, a, spec_out, hsum, lsum, stream=None):
        """Accumulate the surrogate spectrum of the segments in ``a`` into
        spec_out [n_dir][n_out] (exact-scorer units, not normalised)."""
        lib = L.load()
        s = (stream or torch.cuda.current_stream()).cuda_stream
        hsum.zero_()
        lsum.zero_()
        L.check(lib.pb_mlp_infer(C.byref(a), s), "pb_mlp_infer")
        L.check(lib.pb_mlp_head(a.n_dir, self.n_out, self.W5r.data_ptr(), self.p["b5"].data_ptr(),
                                hsum.data_ptr(), lsum.data_ptr(), float(self.t_scale), spec_out.data_ptr(), s),
                "pb_mlp_head")


# ----------------------------------------------------------------------
# exact targets
# ----------------------------------------------------------------------
def transported_segments(spec, n_hist, seed, device, precision="mixed"):
    """Segments of ``n_hist`` histories of the case (compact device list)."""
    from .pipeline import ScoringCase

    from dataclasses import replace

    case = ScoringCase(replace(spec, seed=seed), precision=precision, batch_histories=n_hist, device=device)
    case.seg_count.zero_()
    t = case.targs
    t.e_start, t.n = 0, int(n_hist)
    L.check(case.lib.pb_transport(C.byref(t), _stream()), "pb_transport")
    torch.cuda.synchronize(device)
    n = int(case.seg_count.item())
    # The transport appends segments in a nondeterministic order; put them in
    # history order (decreasing energy along each track) so a seeded pick is
    # reproducible.
    E = case.seg_E[:n]
    order = torch.argsort(E, descending=True, stable=True)
    order = order[torch.argsort(case.seg_id[:n][order], stable=True)]
    seg = {"r": case.seg_r[:n][order].contiguous(), "v": case.seg_v[:n][order].contiguous(),
           "L": case.seg_L[:n][order].contiguous(), "E": E[order].contiguous(),
           "id": torch.zeros(n, dtype=torch.int64, device=device)}
    return seg, n


def _cxr_lines(spec, seg, n_seg, n_hats, device, cap_per_pair=64):
    """Exact FP64 lines (E, a, w, dir, seg) of every (segment, direction) pair."""
    h = _Holder(device)
    rows = reflection_rows(spec.crystal, spec.hkl_list, n_hats, surface_hkl=spec.surface_hkl,
                           mosaic_fwhm_rad=spec.mosaic_fwhm_rad, mosaic_nodes=spec.mosaic_nodes)
    lo_keep, hi_keep = line_keep_window(np.asarray(spec.E_grid, dtype=float))
    n_dir = n_hats.shape[0]
    a = L.PbCxrArgs()
    a.precision = L.PB_FP64
    a.quadrature = L.PB_QUAD_NODE
    a.n_dir = n_dir
    a.n_hat = _ptr(h.f64(n_hats))
    a.thickness = float(spec.stack.thickness)
    a.Ne = 1 << 62
    a.n_seg = int(n_seg)
    a.r_mid, a.v_hat, a.L, a.E_keV = (seg["r"].data_ptr(), seg["v"].data_ptr(), seg["L"].data_ptr(),
                                      seg["E"].data_ptr())
    a.elec_id = seg["id"].data_ptr()
    t = _fill_tables(h, rows, spec.line_tables, lo_keep, hi_keep)
    t.ES, t.EP = _ptr(h.f64(rows.ES)), _ptr(h.f64(rows.EP))
    a.tables = t
    a.n_E = 1
    a.E_grid = _ptr(h.f64([30000.0]))
    a.spec = None  # lines only, no node spectrum
    cap = int(int(n_seg) * n_dir * cap_per_pair)
    count = h.zeros(1, torch.int64)
    lines = {"E": h.empty(cap, torch.float64), "a": h.empty(cap, torch.float64), "w": h.empty(cap, torch.float64),
             "dir": h.zeros(cap, torch.int32), "seg": h.zeros(cap, torch.int64)}
    a.line_capacity = cap
    a.line_count = _ptr(count)
    a.line_E, a.line_a, a.line_w = _ptr(lines["E"]), _ptr(lines["a"]), _ptr(lines["w"])
    a.line_dir, a.line_seg = _ptr(lines["dir"]), _ptr(lines["seg"])
    status = h.zeros(1, torch.int32)
    a.status = _ptr(status)
    L.check(L.load().pb_cxr_score(C.byref(a), _stream()), "pb_cxr_score")
    torch.cuda.synchronize(device)
    n_lines = int(count.item())
    if int(status.item()) != 0 or n_lines > cap:
        raise L.PyriteB200Error(f"exact lines: status {int(status.item())}, {n_lines} lines for capacity {cap}")
    return lines, n_lines


def _bin(lines, n_lines, dir0, n_dir, n_seg, grid, out):
    L.check(L.load().pb_cxr_bin_lines(n_lines, lines["E"].data_ptr(), lines["a"].data_ptr(), lines["w"].data_ptr(),
                                      lines["dir"].data_ptr(), lines["seg"].data_ptr(), int(dir0), int(n_dir),
                                      int(n_seg), grid.lo_eV, grid.width_eV, grid.n_bins, out.data_ptr(), _stream()),
            "pb_cxr_bin_lines")


def uniform_segments(spec, n_seg, seed, device, L_pool, E_MeV=(E_LO_MEV, E_HI_MEV), half_angle=5e-3):
    """Synthetic segments spread over the surrogate's input domain: energy
    log-uniform over ``E_MeV``, direction uniform within +-``half_angle`` of
    the beam axis on both transverse axes, depth uniform through the slab,
    and lengths drawn from ``L_pool`` (a case's transported segment lengths:
    the line shape depends on the length, which is not an input)."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(E_MeV[0] * 1e3), np.log(E_MeV[1] * 1e3)
    E = np.exp(rng.uniform(lo, hi, n_seg))
    d0 = np.asarray(spec.beam.beam_dir, dtype=float)
    d0 = d0 / np.linalg.norm(d0)
    e_x, e_y = _beam_axes(spec)
    ax, ay = rng.uniform(-half_angle, half_angle, (2, n_seg))
    v = d0[None, :] + ax[:, None] * e_x[None, :] + ay[:, None] * e_y[None, :]
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    pool = np.asarray(L_pool, dtype=float)
    L = pool[rng.integers(0, pool.size, n_seg)]
    T = float(spec.stack.thickness)
    # keep the whole segment inside the slab
    half = 0.5 * L * np.abs(v[:, 2])
    z = rng.uniform(0.0, 1.0, n_seg) * np.maximum(T - 2.0 * half, 0.0) + half
    r = np.zeros((n_seg, 3))
    r[:, 2] = z
    t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=device)  # noqa: E731
    return {"r": t(r), "v": t(v), "L": t(L), "E": t(E), "id": torch.zeros(n_seg, dtype=torch.int64, device=device)}


def make_training_set(spec, *, n_seg=8192, n_dir=2048, dir_chunk=64, n_hist=None, seed=101, device=None,
                      grid=None, log=None, shuffle=True, process_group=None, domain="case"):
    """Exact per-(segment, direction) coarse spectra per unit length with their features.

    Returns a dict with X [N, 16] bf16, Xt [16, N] bf16, T [N, n_bins] bf16
    (targets / t_scale), t_scale, grid; rows shuffled. With ``process_group``
    (data-parallel training, each rank its own ``seed``) the ranks agree on
    one target scale: the RMS over the first direction chunk of every rank.

    ``domain="case"`` picks segments of the case's own transport (the
    workload's joint energy / angle / depth distribution); ``"uniform"``
    spreads them over the surrogate's whole input domain (``uniform_segments``:
    5-100 MeV log-uniform, +-5 mrad, every depth), with lengths from the
    case's transport.
    """
    device = torch.device(device or "cuda")
    grid = grid or CoarseGrid.of(spec.E_grid)
    # Many more histories than picked segments, so the segments sample the
    # workload's joint (energy, angle, depth) distribution, not a few tracks.
    n_hist = n_hist or max(4096, 4 * n_seg)
    all_seg, n_all = transported_segments(spec, n_hist, seed, device)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    # Targets are per unit length: segments of zero length carry no emission
    # and would divide by zero, so they are not candidates.
    cand = torch.nonzero(all_seg["L"] > 0.0).flatten().cpu()
    pick = cand[torch.randperm(cand.numel(), generator=gen)[:n_seg]].to(device)
    if domain == "uniform":
        seg = uniform_segments(spec, int(pick.numel()), seed, device, all_seg["L"][pick].cpu().numpy())
    elif domain == "case":
        seg = {k: v[pick].contiguous() for k, v in all_seg.items()}
    else:
        raise ValueError(f"unknown training domain {domain!r}")
    n_seg = int(pick.numel())
    rng = np.random.default_rng(seed)
    uv = rng.uniform(-1.0, 1.0, size=(n_dir, 2))
    n_hats = directions_at(spec.detector, uv, spec.beam.tilt_polar_rad)
    N = n_seg * n_dir
    X = torch.empty(N, K_IN, device=device, dtype=torch.bfloat16)
    T = torch.empty(N, grid.n_bins, device=device, dtype=torch.bfloat16)
    inv_L = (1.0 / seg["L"]).to(torch.float32)
    t_scale = None
    for d0 in range(0, n_dir, dir_chunk):
        nd = min(dir_chunk, n_dir - d0)
        lines, n_lines = _cxr_lines(spec, seg, n_seg, n_hats[d0:d0 + nd], device)
        tgt = torch.zeros(nd * n_seg, grid.n_bins, device=device, dtype=torch.float32)
        _bin(lines, n_lines, 0, nd, n_seg, grid, tgt)
        tgt.view(nd, n_seg, grid.n_bins).mul_(inv_L[None, :, None])
        if t_scale is None:
            ms = tgt.square().mean().double().reshape(1)
            if process_group is not None:
                import torch.distributed as dist

                dist.all_reduce(ms, group=process_group)
                ms /= dist.get_world_size(process_group)
            t_scale = float(ms.sqrt().item()) or 1.0
        T[d0 * n_seg:(d0 + nd) * n_seg] = (tgt / t_scale).to(torch.bfloat16)
        a = _feature_args(spec, seg, n_seg, torch.as_tensor(uv[d0:d0 + nd], dtype=torch.float32, device=device))
        L.check(L.load().pb_mlp_features(C.byref(a), X[d0 * n_seg:].data_ptr(), None, _stream()), "pb_mlp_features")
        del lines, tgt
        if log and (d0 // dir_chunk) % 8 == 0:
            log(f"targets: {d0 + nd}/{n_dir} directions")
    Lrow = seg["L"].to(torch.float32).repeat(n_dir)
    # A pair whose target or features are not finite (a degenerate line of
    # the exact scorer) is dropped rather than poisoning every step after it.
    good = torch.isfinite(T).all(dim=1) & torch.isfinite(X).all(dim=1)
    n_bad = int((~good).sum().item())
    if n_bad:
        # (a multiple of 64 rows keeps the transposed features' row stride
        # a multiple of 8, as the GEMMs want)
        keep = torch.nonzero(good).flatten()
        keep = keep[: keep.numel() // 64 * 64]
        X, T, Lrow = X[keep], T[keep], Lrow[keep]
        N = int(keep.numel())
        if log:
            log(f"targets: dropped {n_bad} pairs with non-finite values")
    if shuffle:
        perm = torch.randperm(N, generator=gen).to(device)
        X = X[perm].contiguous()
        T = T[perm].contiguous()
        Lrow = Lrow[perm].contiguous()
    return {"X": X, "Xt": X.t().contiguous(), "T": T, "L": Lrow, "t_scale": t_scale, "grid": grid,
            "n_seg": n_seg, "n_dir": n_dir, "nonfinite_pairs_dropped": n_bad}


def make_tile_training_set(spec, *, n_seg=65536, n_hist=None, seg_chunk=4096, seed=101, device=None, grid=None,
                           log=None, shuffle=True, process_group=None):
    """Training rows of the tile-factored surrogate: one row per segment of the
    case's own transport, its features without a direction (the tile
    features are zero), its targets the exact coarse spectra per unit length
    towards every one of the case's directions ``spec.n_hats``, concatenated
    tile after tile: T [n_seg, n_tiles * n_bins]. Returns the same dict as
    ``make_training_set`` (``n_dir`` = 1 feature direction, ``n_tiles``)."""
    device = torch.device(device or "cuda")
    grid = grid or CoarseGrid.of(spec.E_grid)
    n_hats = np.atleast_2d(np.asarray(spec.n_hats, dtype=float))
    n_tiles = n_hats.shape[0]
    n_hist = n_hist or max(4096, n_seg // 8)
    all_seg, _n_all = transported_segments(spec, n_hist, seed, device)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    cand = torch.nonzero(all_seg["L"] > 0.0).flatten().cpu()
    pick = cand[torch.randperm(cand.numel(), generator=gen)[:n_seg]].to(device)
    seg = {k: v[pick].contiguous() for k, v in all_seg.items()}
    n_seg = int(pick.numel())
    X = torch.empty(n_seg, K_IN, device=device, dtype=torch.bfloat16)
    T = torch.empty(n_seg, n_tiles * grid.n_bins, device=device, dtype=torch.bfloat16)
    t_scale = None
    for s0 in range(0, n_seg, seg_chunk):
        ns = min(seg_chunk, n_seg - s0)
        sub = {k: v[s0:s0 + ns] for k, v in seg.items()}
        lines, n_lines = _cxr_lines(spec, sub, ns, n_hats, device)
        tgt = torch.zeros(n_tiles * ns, grid.n_bins, device=device, dtype=torch.float32)
        _bin(lines, n_lines, 0, n_tiles, ns, grid, tgt)
        tgt = tgt.view(n_tiles, ns, grid.n_bins).permute(1, 0, 2).reshape(ns, n_tiles * grid.n_bins)
        tgt.mul_((1.0 / sub["L"]).to(torch.float32)[:, None])
        if t_scale is None:
            ms = tgt.square().mean().double().reshape(1)
            if process_group is not None:
                import torch.distributed as dist

                dist.all_reduce(ms, group=process_group)
                ms /= dist.get_world_size(process_group)
            t_scale = float(ms.sqrt().item()) or 1.0
        T[s0:s0 + ns] = (tgt / t_scale).to(torch.bfloat16)
        del lines, tgt
        if log and (s0 // seg_chunk) % 8 == 0:
            log(f"tile targets: {s0 + ns}/{n_seg} segments")
    a = _feature_args(spec, seg, n_seg, torch.zeros(1, 2, dtype=torch.float32, device=device))
    L.check(L.load().pb_mlp_features(C.byref(a), X.data_ptr(), None, _stream()), "pb_mlp_features")
    Lrow = seg["L"].to(torch.float32)
    good = torch.isfinite(T).all(dim=1) & torch.isfinite(X).all(dim=1)
    n_bad = int((~good).sum().item())
    # the GEMMs want the transposed features' row stride a multiple of 8:
    # keep a multiple of 64 rows
    keep = torch.nonzero(good).flatten()
    keep = keep[: keep.numel() // 64 * 64]
    if int(keep.numel()) != n_seg:
        X, T, Lrow = X[keep], T[keep], Lrow[keep]
        n_seg = int(keep.numel())
    if shuffle:
        perm = torch.randperm(n_seg, generator=gen).to(device)
        X, T, Lrow = X[perm].contiguous(), T[perm].contiguous(), Lrow[perm].contiguous()
    return {"X": X, "Xt": X.t().contiguous(), "T": T, "L": Lrow, "t_scale": t_scale, "grid": grid,
            "n_seg": n_seg, "n_dir": 1, "n_tiles": n_tiles, "nonfinite_pairs_dropped": n_bad}


def _feature_args(spec, seg, n_seg, dir_uv_t):
    a = L.PbMlpInferArgs()
    a.n_dir = int(dir_uv_t.shape[0])
    a.dir_uv = dir_uv_t.data_ptr()
    e_x, e_y = _beam_axes(spec)
    for i in range(3):
        a.e_x[i], a.e_y[i] = float(e_x[i]), float(e_y[i])
    a.theta_max, a.E_lo_MeV, a.E_hi_MeV = THETA_MAX_RAD, E_LO_MEV, E_HI_MEV
    a.thickness = float(spec.stack.thickness)
    a.Ne = 1 << 62
    a.n_seg = int(n_seg)
    a.r_mid, a.v_hat, a.L, a.E_keV, a.elec_id = (seg["r"].data_ptr(), seg["v"].data_ptr(), seg["L"].data_ptr(),
                                                 seg["E"].data_ptr(), seg["id"].data_ptr())
    a._keep = dir_uv_t  # the caller's tensor backs dir_uv
    return a


def exact_aggregate(spec, seg, n_seg, n_hats, grid, device, seg_chunk=4096):
    """Exact coarse spectrum per direction [n_dir, n_bins] (sum over segments)."""
    n_dir = n_hats.shape[0]
    out = torch.zeros(n_dir, grid.n_bins, device=device, dtype=torch.float32)
    for s0 in range(0, n_seg, seg_chunk):
        ns = min(seg_chunk, n_seg - s0)
        sub = {k: v[s0:s0 + ns] for k, v in seg.items()}
        lines, n_lines = _cxr_lines(spec, sub, ns, n_hats, device)
        lines["seg"].zero_()
        _bin(lines, n_lines, 0, n_dir, 1, grid, out)
    return out


def finetune_groups(model, data, *, S=512, epochs=3, batch=8192, lr=3e-4, lr_final=3e-6, log=None):
    """Fine-tune on group aggregates: batches of ``batch // S`` groups, each
    one detector direction with S segments (length-weighted), matching the
    per-direction sums that inference produces. ``data`` must come from
    ``make_training_set(..., shuffle=False)`` (rows d-major with segments in
    random order)."""
    X, Xt, T, Lw = data["X"], data["Xt"], data["T"], data["L"]
    n_seg = data["n_seg"]
    if n_seg % S or batch % S:
        raise ValueError("S must divide n_seg and the batch")
    N = X.shape[0] // batch * batch
    w = (Lw.view(-1, S) / Lw.view(-1, S).sum(1, keepdim=True)).reshape(-1).contiguous()
    ws = model._workspace(batch)
    total = epochs * (N // batch)
    gen = torch.Generator(device="cpu").manual_seed(17)
    k = 0
    losses = []
    for ep in range(epochs):
        ws["loss"].zero_()
        order = torch.randperm(N // batch, generator=gen).tolist()
        for bi in order:
            b0 = bi * batch
            lr_k = lr * (lr_final / lr) ** (k / max(total - 1, 1))
            model.train_step(X[b0:b0 + batch], Xt[:, b0:b0 + batch], T[b0:b0 + batch], ws, lr_k,
                             group=(S, w[b0:b0 + batch]))
            k += 1
        torch.cuda.synchronize(model.device)
        losses.append(float(ws["loss"].item()) / ((N // S) * model.n_out))
        if log:
            log(f"group epoch {ep}: mse {losses[-1]:.4e}")
    return losses


def train_streaming(spec, *, epochs=10, n_seg=16384, n_dir=1024, lr=2e-3, lr_final=2e-5, batch=8192, seed=101,
                    model_seed=0, device=None, log=None):
    """Train one surrogate on a fresh exact dataset every epoch (new transport
    histories and detector points each time), so no epoch sees a pair twice
    and the fit cannot specialise to one sample of segments."""
    device = torch.device(device or "cuda")
    model = Surrogate(device, seed=model_seed)
    n_batches = (n_seg * n_dir) // batch
    total = epochs * n_batches
    ws = model._workspace(batch)
    k = 0
    losses = []
    for ep in range(epochs):
        data = make_training_set(spec, n_seg=n_seg, n_dir=n_dir, dir_chunk=max(1, 2 ** 20 // n_seg),
                                 seed=seed + 7919 * ep, device=device)
        if ep == 0:
            model.t_scale = float(data["t_scale"])
        rescale = float(data["t_scale"]) / model.t_scale
        X, Xt, T = data["X"], data["Xt"], data["T"]
        if rescale != 1.0:
            T = (T.float() * rescale).to(torch.bfloat16)
        ws["loss"].zero_()
        for b0 in range(0, n_batches * batch, batch):
            lr_k = lr * (lr_final / lr) ** (k / max(total - 1, 1))
            model.train_step(X[b0:b0 + batch], Xt[:, b0:b0 + batch], T[b0:b0 + batch], ws, lr_k)
            k += 1
        torch.cuda.synchronize(device)
        losses.append(float(ws["loss"].item()) / (n_batches * batch * model.n_out))
        if log:
            log(f"epoch {ep}: mse {losses[-1]:.4e}")
        del data, X, Xt, T
    if int(ws["status"].item()) != 0:
        raise L.PyriteB200Error(f"surrogate training: device status {int(ws['status'].item())}")
    model.losses = losses
    return model


def train_ensemble(spec, *, k=4, n_seg=16384, n_dir=1024, epochs=10, lr=2e-3, seed=101, device=None, log=None):
    """Train ``k`` surrogates (different initialisations) on one exact dataset."""
    device = torch.device(device or "cuda")
    data = make_training_set(spec, n_seg=n_seg, n_dir=n_dir, dir_chunk=max(1, 2 ** 20 // n_seg), seed=seed,
                             device=device, log=log)
    models = []
    for i in range(k):
        m = Surrogate(device, seed=1000 + i)
        m.train(data, epochs=epochs, lr=lr, lr_final=lr / 100, log=log)
        models.append(m)
    del data
    return models


def control_variate_error(res_sum, res_sq, n_batches, stride, spectrum, n_sigma=3.0, window=9):
    """Estimated error of the control-variate spectrum per detector tile.

    The estimate is S = S_sur(all) + stride * sum_b r_b, with r_b the
    residual S_exact(sample_b) - S_sur(sample_b) of batch b's exact
    sub-sample ([n_tile, n_bin] each). Treating the batches' residuals as
    independent draws, the correction's variance per bin is
    stride^2 * B * var_b(r), var from the B batches' scatter (``res_sum`` =
    sum_b r_b, ``res_sq`` = sum_b r_b^2), pooled over ``window`` neighbouring
    bins (with only B - 1 degrees of freedom per bin, the worst of 512
    unpooled bins would overstate the error about 2.6-fold at B = 4). Returns
    n_sigma * (worst bin's standard error) / (tile's peak of ``spectrum``)
    per tile, ``spectrum`` in the same un-normalised units; three standard
    errors is about the largest deviation expected over a few hundred bins.
    None with fewer than two batches."""
    B = int(n_batches)
    if B < 2:
        return None
    res_sum = np.asarray(res_sum, dtype=np.float64)
    var = np.maximum((np.asarray(res_sq, dtype=np.float64) - res_sum * res_sum / B) / (B - 1), 0.0)
    if window > 1:
        k = np.ones(int(window))
        num = np.apply_along_axis(lambda v: np.convolve(v, k, mode="same"), 1, var)
        den = np.convolve(np.ones(var.shape[1]), k, mode="same")
        var = num / den[None, :]
    se = float(stride) * np.sqrt(B * var)
    peak = np.max(np.abs(np.asarray(spectrum, dtype=np.float64)), axis=1)
    out = n_sigma * np.max(se, axis=1) / np.where(peak > 0, peak, np.inf)
    return np.where(peak > 0, out, 0.0)


def audit_uniform(model, spec, *, n_seg=100_000, seed=303, device=None, grid=None, n_hist=4096):
    """Surrogate vs exact on held-out segments spread over the input domain
    (``uniform_segments``, lengths from ``n_hist`` transported histories of a
    seed of their own), aggregated per tile: the same error measures as
    ``audit``."""
    device = torch.device(device or "cuda")
    grid = grid or CoarseGrid.of(spec.E_grid)
    pool, n_pool = transported_segments(spec, n_hist, seed, device)
    Lp = pool["L"][:n_pool]
    seg = uniform_segments(spec, n_seg, seed, device, Lp[Lp > 0].cpu().numpy())
    return _audit_on(model, spec, seg, n_seg, device, grid)


def audit(model, spec, *, n_hist=4096, seed=202, device=None, grid=None):
    """Surrogate vs exact aggregate spectra on held-out histories at the case's tiles.

    ``model`` is one Surrogate or a list (their mean is the prediction).
    Returns dict(err_tile_max, err_total, exact, surrogate): errors are the
    max |difference| over bins relative to the peak, per tile (worst tile)
    and for the detector total (all tiles summed).
    """
    device = torch.device(device or "cuda")
    grid = grid or CoarseGrid.of(spec.E_grid)
    seg, n_seg = transported_segments(spec, n_hist, seed, device)
    return _audit_on(model, spec, seg, n_seg, device, grid)


def _audit_on(model, spec, seg, n_seg, device, grid):
    n_hats = np.atleast_2d(np.asarray(spec.n_hats, dtype=float))
    uv = tile_uv(spec.detector, spec.angular_shape)
    exact = exact_aggregate(spec, seg, n_seg, n_hats, grid, device).double()
    dir_uv = torch.as_tensor(uv, dtype=torch.float32, device=device)
    hsum = torch.zeros(n_hats.shape[0], HIDDEN, device=device, dtype=torch.float64)
    lsum = torch.zeros(n_hats.shape[0], device=device, dtype=torch.float64)
    status = torch.zeros(1, device=device, dtype=torch.int32)
    sur = torch.zeros(n_hats.shape[0], grid.n_bins, device=device, dtype=torch.float64)
    models = model if isinstance(model, (list, tuple)) else [model]
    for m in models:
        a = m.infer_args(spec, seg, n_seg, dir_uv, hsum, lsum, status=status)
        part = torch.zeros_like(sur)
        m.score(a, part, hsum, lsum)
        sur += part / len(models)
    torch.cuda.synchronize(device)
    ex, su = exact.cpu().numpy(), sur.cpu().numpy()
    per_tile = np.max(np.abs(su - ex), axis=1) / np.maximum(np.max(np.abs(ex), axis=1), 1e-300)
    tot_e, tot_s = ex.sum(0), su.sum(0)
    return {"err_tile_max": float(per_tile.max()), "err_total": float(np.max(np.abs(tot_s - tot_e)) / np.max(tot_e)),
            "exact": ex, "surrogate": su, "segments": n_seg, "status": int(status.item())}
