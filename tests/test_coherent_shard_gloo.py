"""Coherent reduction sharded by rows over two gloo ranks on the CPU.

Rows (reflection x mosaic orientation) add incoherently, so
``coherent.coherent_reduce_sharded`` gives each rank whole rows and sums the
FP64 spectra with one all-reduce. The per-rank reducer here is the oracle
(the device kernel needs a GPU); the sharded sum must equal the reference's
coherent spectrum of all rows.
"""

import os
import socket
import tempfile

import numpy as np

from conftest import GOLDEN


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_reduce(rec, cnt, w, E, dom, scale=1.0, sinc_cutoff=None):
    import torch

    from oracle import coherent as oc

    return torch.from_numpy(oc.coherent_spectrum(rec, cnt, w, E, dom) * scale)


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist

    from oracle import coherent as oc
    from pyrite_b200.coherent import coherent_reduce_sharded

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        rec, cnt, w, E, dom, Ne, _ = oc.load_golden(GOLDEN / "coherent_hopg20.npz")
        spec = coherent_reduce_sharded(rec, cnt, w, E, dom, scale=1.0 / Ne, reduce_fn=_oracle_reduce)
        np.save(out_path + f".{rank}.npy", spec.numpy())
    finally:
        dist.destroy_process_group()


def test_assign_rows_partitions_and_balances():
    from pyrite_b200.coherent import assign_rows

    rng = np.random.default_rng(4)
    for n_rows, world in ((144, 2), (126, 8), (5, 3), (1, 4)):
        counts = rng.integers(0, 900, n_rows)
        parts = assign_rows(counts, world)
        assert len(parts) == world
        assert np.array_equal(np.sort(np.concatenate(parts)), np.arange(n_rows))
        loads = [int(counts[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= int(counts.max())
        assert all(np.all(np.diff(p) > 0) for p in parts)


def test_two_gloo_ranks_equal_the_reference():
    import torch.multiprocessing as mp

    from oracle import coherent as oc

    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "spec")
        mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        got = [np.load(out + f".{r}.npy") for r in range(2)]
    *_, ref = oc.load_golden(GOLDEN / "coherent_hopg20.npz")
    assert np.array_equal(got[0], got[1])
    assert np.max(np.abs(got[0] - ref)) <= 1e-12 * np.max(ref)
