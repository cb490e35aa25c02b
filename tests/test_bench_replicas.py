"""bench.py's multi-GPU form is replicas only: each rank solves its own
systems, the job time is the slowest rank's, and the value is the bodies all
ranks solved over it.  These run the aggregation on two gloo ranks on the CPU,
and check how `--gpus N` turns into a rank launch."""
import importlib.util
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    b = _bench()
    # rank r took (r + 1) seconds for its 1,000 bodies; tuned ncrit differs per rank
    tmax, value = b.replica_value(1.0 + rank, 1000, world, dist, device="cpu")
    ncrit = b.agree_ncrit(64 if rank == 0 else 128, world, dist, device="cpu")
    out[rank] = (tmax, value, ncrit)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_on_two_gloo_ranks():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, _port(), out), nprocs=world, join=True)
    for r in range(world):
        tmax, value, ncrit = out[r]
        assert tmax == 2.0                      # the slowest rank's time, on every rank
        assert value == pytest.approx(1000.0)   # 2 ranks x 1,000 bodies / 2 s
        assert ncrit == 64                      # rank 0's choice


def test_gpus_flag_launches_ranks_or_refuses_a_mismatch():
    b = _bench()
    assert b.check_world(1, env={}) == "run"
    assert b.check_world(4, env={}) == "spawn"
    assert b.check_world(4, env={"WORLD_SIZE": "4"}) == "run"
    with pytest.raises(SystemExit):
        b.check_world(8, env={"WORLD_SIZE": "1"})
    cmd = b.torchrun_command(["--gpus", "4", "--steps", "3"], 4, 29501)
    assert cmd[1:4] == ["-m", "torch.distributed.run", "--nnodes=1"]
    assert "--nproc-per-node=4" in cmd and "127.0.0.1" in cmd and cmd[-4:] == ["--gpus", "4", "--steps", "3"]
