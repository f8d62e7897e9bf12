"""Host side of the BF16 MLP surrogate's tcgen05 kernels.

Thin wrappers over the C ABI (``pb_mlp_*``): tensors are torch CUDA tensors
used as device buffers; every product runs in the library's kernels.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L


def _p(t):
    return None if t is None else t.data_ptr()


def _s(stream):
    return (stream or torch.cuda.current_stream()).cuda_stream


def gemm(A, B, *, bias=None, act=0, dsilu_z=None, out_f32=None, beta=0.0, out_bf16=None, out_bf16_t=None,
         status=None, stream=None, M=None, N=None, K=None):
    """D = A . B^T on tcgen05 with the fused epilogue of ``pb_mlp_gemm``.

    ``A`` bf16 [M, K] and ``B`` bf16 [N, K] (row strides may exceed K);
    outputs are written in place. Returns nothing.
    """
    g = L.PbMlpGemmArgs()
    g.M = int(M if M is not None else A.shape[0])
    g.N = int(N if N is not None else B.shape[0])
    g.K = int(K if K is not None else A.shape[1])
    g.A, g.lda = _p(A), int(A.stride(0))
    g.B, g.ldb = _p(B), int(B.stride(0))
    g.bias = _p(bias)
    g.act = int(act)
    g.dsilu_z, g.ldz = _p(dsilu_z), int(dsilu_z.stride(0)) if dsilu_z is not None else 0
    g.out_f32, g.ldc = _p(out_f32), int(out_f32.stride(0)) if out_f32 is not None else 0
    g.beta = float(beta)
    g.out_bf16, g.ldh = _p(out_bf16), int(out_bf16.stride(0)) if out_bf16 is not None else 0
    g.out_bf16_t, g.ldt = _p(out_bf16_t), int(out_bf16_t.stride(0)) if out_bf16_t is not None else 0
    g.status = _p(status)
    L.check(L.load().pb_mlp_gemm(C.byref(g), _s(stream)), "pb_mlp_gemm")


def mse_grad(Y, T, t_scale, g_scale, dY, dYt, loss, stream=None):
    rows, cols = Y.shape
    L.check(L.load().pb_mlp_mse_grad(rows, cols, _p(Y), _p(T), int(T.stride(0)), float(t_scale), float(g_scale),
                                     _p(dY), _p(dYt), int(dYt.stride(0)), _p(loss), _s(stream)), "pb_mlp_mse_grad")


def group_mse_grad(Y, T, w, S, t_scale, g_scale, dY, dYt, loss, stream=None):
    rows, cols = Y.shape
    L.check(L.load().pb_mlp_group_mse_grad(rows // S, S, cols, _p(Y), _p(T), int(T.stride(0)), _p(w), float(t_scale),
                                           float(g_scale), _p(dY), _p(dYt), int(dYt.stride(0)), _p(loss), _s(stream)),
            "pb_mlp_group_mse_grad")


def colsum(X, out, stream=None):
    rows, cols = X.shape
    L.check(L.load().pb_mlp_colsum(rows, cols, _p(X), int(X.stride(0)), _p(out), _s(stream)), "pb_mlp_colsum")


def adam(p, g, m, v, lr, b1, b2, eps, wd, step, stream=None):
    bc1, bc2 = 1.0 - b1 ** step, 1.0 - b2 ** step
    L.check(L.load().pb_mlp_adam(p.numel(), _p(p), _p(g), _p(m), _p(v), lr, b1, b2, eps, wd, bc1, bc2, _s(stream)),
            "pb_mlp_adam")


def pack(W, Wb, Wt=None, pad_cols=None, stream=None):
    rows, cols = W.shape
    L.check(L.load().pb_mlp_pack(rows, cols, _p(W), _p(Wb), int(Wb.stride(0)), _p(Wt),
                                 int(Wt.stride(0)) if Wt is not None else 0,
                                 int(pad_cols if pad_cols is not None else Wb.shape[1]), _s(stream)), "pb_mlp_pack")
