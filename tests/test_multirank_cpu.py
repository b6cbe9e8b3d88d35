"""The multi-rank timing path of bench.py on world_size 2 with gloo on CPU: every rank gets the
maximum of the per-rank times, as the benchmark reports it."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    out[rank] = bench.max_over_ranks(10.0 * (rank + 1), "cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(out) == {0: 20.0, 1: 20.0}


def test_reference_arm_other_ranks_exit_quietly(capsys):
    import bench
    os.environ["RANK"] = "1"
    try:
        bench.run_reference(type("A", (), {"height": 1080, "width": 1920, "warmup": 3, "steps": 1,
                                           "gpus": 2})())
    finally:
        del os.environ["RANK"]
    assert capsys.readouterr().out == ""
