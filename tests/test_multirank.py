"""Multi-rank host logic of the benchmark on CPU: world-size-2 gloo ranks.

Rays are independent, so N GPUs shard the seeded workload into disjoint
consecutive ranges with no collective in the data path; the only collective is
the max-over-ranks reduction of the timed region."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from blackhorizon_b200.workloads import raw_throughput_inputs

        pos, d, spin = raw_throughput_inputs(n, offset=bench.shard_offset(rank, n))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), pos=pos, spin=spin)
        slowest = bench.max_over_ranks(1.5 + rank, world)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(repr(slowest))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_time(tmp_path):
    world, n = 2, 300
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    from blackhorizon_b200.workloads import raw_throughput_inputs

    full_pos, _, full_spin = raw_throughput_inputs(world * n)
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    np.testing.assert_array_equal(np.concatenate([p["pos"] for p in parts]), full_pos)
    np.testing.assert_array_equal(np.concatenate([p["spin"] for p in parts]), full_spin)
    for r in range(world):
        assert float((tmp_path / f"rank{r}.txt").read_text()) == 2.5
