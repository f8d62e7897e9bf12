"""Host-side recovery, tested without a GPU fault: the step-budget retry
(runner/step_budget.py:33-53) and a rank that leaves a gloo group before the
final tally exchange (the survivor gets an error, not a hang)."""

import datetime
import os
import socket
import tempfile

import pytest


def test_step_budget_doubles_until_no_history_is_limited():
    from pyrite_b200.api import TransportStepLimitError, retry_step_budget

    calls = []

    def fake_simulate(E0, Ne, *, max_steps):
        calls.append(max_steps)
        need = 5000  # every history needs this many steps
        return {"n_step_limited": Ne if max_steps < need else 0, "max_steps": max_steps}

    out = retry_step_budget(fake_simulate, 1000.0, 8, initial_max_steps=1000)
    assert calls == [1000, 2000, 4000, 8000] and out["max_steps"] == 8000
    calls.clear()
    with pytest.raises(TransportStepLimitError):
        retry_step_budget(fake_simulate, 1000.0, 8, initial_max_steps=1000, ceiling=3000)
    assert calls == [1000, 2000, 3000]
    with pytest.raises(ValueError):
        retry_step_budget(fake_simulate, 1.0, 1, initial_max_steps=0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    from pyrite_b200.shard import reduce_results

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        os._exit(0)  # leaves between steps, before the exchange
    try:
        reduce_results({"spec": torch.ones(8, dtype=torch.float64)})
        msg = "completed"
    except Exception as e:  # noqa: BLE001 -- any collective error is the expected outcome
        msg = "error: " + type(e).__name__
    with open(os.path.join(out_dir, "rank0.txt"), "w") as f:
        f.write(msg)
    os._exit(0)


@pytest.mark.timeout(120)
def test_survivor_of_a_departed_rank_gets_an_error():
    import torch.multiprocessing as mp

    with tempfile.TemporaryDirectory() as tmp:
        ctx = mp.start_processes(_rank, args=(2, _free_port(), tmp), nprocs=2, join=False, start_method="spawn")
        for p in ctx.processes:
            p.join(90)
        alive = [p for p in ctx.processes if p.is_alive()]
        for p in alive:
            p.kill()
        assert not alive, "a rank hung"
        with open(os.path.join(tmp, "rank0.txt")) as f:
            assert f.read().startswith("error")
