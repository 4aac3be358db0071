"""Run by tests/test_dist_cpu.py under torch.distributed.run (two ranks,
gloo on CPU): the rank plumbing bench.py uses for --gpus N."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def main():
    ws, rank, local = bench.dist_env()
    assert ws == 2, ws
    bench.init_ranks(local)
    import torch.distributed as dist
    assert dist.get_backend() == "gloo"
    bench.barrier(ws)
    # the timed interval is the maximum over ranks
    got = bench.max_over_ranks(1.5 + rank, ws)
    assert got == 2.5, got
    bench.barrier(ws)
    if rank == 0:
        print("dist-ok", flush=True)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
