"""History sharding over two gloo ranks on the CPU.

Each rank transports its own contiguous block of histories with the Philox
stream (keyed by history, so the block boundary changes nothing), scores its
segments into PXR+CBS bin-mean and Bethe-Heitler spectra and exit fates with
the oracle, and the ranks sum their results with
``pyrite_b200.shard.reduce_results``. The sum must equal one process running
all histories: fates exactly, spectra to FP64 summation order.
"""

import os
import socket
import tempfile

import numpy as np
import pytest

from conftest import golden

N_HIST = 24


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _score_block(start: int, count: int) -> dict:
    import oracle

    d = golden("transport_c20mev")
    c = golden("cxr_hopg20")
    b = golden("brem_c20")
    lt = oracle.LayerTables(d["z_top"], d["z_bot"], d["n_el"], d["Z"], d["J"], d["N"], d["E_cross"])
    pos = np.zeros((count, 3))
    direction = np.tile(np.asarray(d["beam_dir"], float), (count, 1))
    E = np.full(count, float(d["E0_keV"]))
    out = oracle.transport(lt, pos, direction, E, seed=7, E_cut=float(d["E_cut_keV"]), rng=oracle.RNG_PHILOX,
                           e_start=start, cap=512)
    seg = dict(v_hat=out["v_hat"], E_keV=0.5 * (out["E_start"] + out["E_end"]), L_ang=out["L"],
               r_mid=out["r_mid"], elec_id=out["elec_id"])
    E_grid = c["E_grid"]
    pad = 0.2 * (E_grid[-1] - E_grid[0])
    t = {k: c[k] for k in ("G", "ES", "EP", "WM", "row_table", "E_tab", "chi_re", "chi_im", "u_re", "u_im",
                            "log_mu", "delta")}
    t["lo_keep"], t["hi_keep"] = E_grid[0] - pad, E_grid[-1] + pad
    Er, a, w, good = oracle.cxr_lines(t, c["n_hat"], c["thickness"], seg, 1 << 40)
    spec_cxr = oracle.reduce_binmean(Er[good], a[good], w[good], oracle.energy_bin_edges(E_grid))
    spec_brem = oracle.brem_spectrum(seg, b["Z"], b["n_ang3"], float(b["thickness"]), b["n_hat"], b["E_grid"],
                                     b["mu_grid"], 1)
    fates = np.bincount(out["exit_code"].astype(np.int64), minlength=6)
    return dict(spec_cxr=spec_cxr, spec_brem=spec_brem, fates=fates)


def _rank_main(rank, world, port, out_path):
    import torch
    import torch.distributed as dist

    from pyrite_b200.shard import history_range, reduce_results

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        start, count = history_range(N_HIST, rank, world)
        res = _score_block(start, count)
        tens = {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in res.items()}
        reduce_results(tens)
        if rank == 0:
            np.savez(out_path, **{k: v.numpy() for k, v in tens.items()})
    finally:
        dist.destroy_process_group()


def test_history_range_partitions_exactly():
    from pyrite_b200.shard import batches, history_range

    for n in (0, 1, 7, 1000, 65536 + 3):
        for world in (1, 2, 3, 8):
            spans = [history_range(n, r, world) for r in range(world)]
            assert sum(c for _, c in spans) == n
            assert all(spans[r][0] + spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            assert max(c for _, c in spans) - min(c for _, c in spans) <= 1
    assert list(batches(10, 7, 3)) == [(10, 3), (13, 3), (16, 1)]
    with pytest.raises(ValueError):
        history_range(10, 2, 2)


def test_two_gloo_ranks_equal_one_process():
    import torch.multiprocessing as mp

    with tempfile.TemporaryDirectory() as tmp:
        out_path = os.path.join(tmp, "reduced.npz")
        mp.start_processes(_rank_main, args=(2, _free_port(), out_path), nprocs=2, join=True,
                           start_method="spawn")
        got = dict(np.load(out_path))
    ref = _score_block(0, N_HIST)
    np.testing.assert_array_equal(got["fates"], ref["fates"])
    for k in ("spec_cxr", "spec_brem"):
        peak = np.max(np.abs(ref[k]))
        assert peak > 0
        assert np.max(np.abs(got[k] - ref[k])) <= 1e-12 * peak


def _dp_data():
    rng = np.random.default_rng(5)
    X = rng.normal(size=(64, 6))
    t = X @ np.array([0.5, -1.0, 2.0, 0.0, 0.3, -0.7]) + 0.1 * rng.normal(size=64)
    return X, t


def _dp_steps(X, t, grad_fn, steps=20, lr=0.05):
    import torch

    w = torch.zeros(6, dtype=torch.float64)
    Xt, tt = torch.from_numpy(X), torch.from_numpy(t)
    for _ in range(steps):
        g = 2.0 * Xt.T @ (Xt @ w - tt) / Xt.shape[0]
        g = grad_fn(g)
        w -= lr * g
    return w.numpy()


def _dp_rank_main(rank, world, port, out_path):
    import torch.distributed as dist

    from pyrite_b200.shard import average_gradients, history_range

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        X, t = _dp_data()
        lo, n = history_range(X.shape[0], rank, world)  # equal shards (64 / 2)
        w = _dp_steps(X[lo:lo + n], t[lo:lo + n], lambda g: average_gradients(g))
        np.save(out_path + f".{rank}.npy", w)
    finally:
        dist.destroy_process_group()


def test_data_parallel_gradient_average_equals_full_batch():
    """Surrogate training on N ranks averages the flat gradient before every
    optimizer step (``shard.average_gradients``): with equal shards and equal
    initial parameters every rank follows the full-batch trajectory."""
    import torch.multiprocessing as mp

    X, t = _dp_data()
    ref = _dp_steps(X, t, lambda g: g)
    with tempfile.TemporaryDirectory() as tmp:
        out_path = os.path.join(tmp, "w")
        mp.start_processes(_dp_rank_main, args=(2, _free_port(), out_path), nprocs=2, join=True,
                           start_method="spawn")
        w0, w1 = np.load(out_path + ".0.npy"), np.load(out_path + ".1.npy")
    np.testing.assert_array_equal(w0, w1)
    np.testing.assert_allclose(w0, ref, rtol=1e-12, atol=1e-14)
