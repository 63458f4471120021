"""A rank of tests/test_multirank.py::test_bench_launcher_starts_the_ranks:
joins the process group from the environment a launcher gives it (gloo, no
GPU), all-reduces (rank + 1) and, on rank 0, writes what it saw to argv[1]."""
import json
import os
import sys

import torch
import torch.distributed as dist


def main():
    dist.init_process_group("gloo")
    t = torch.tensor([dist.get_rank() + 1], dtype=torch.int64)
    dist.all_reduce(t)
    if dist.get_rank() == 0:
        with open(sys.argv[1], "w") as f:
            json.dump({"world": dist.get_world_size(), "sum": int(t.item()),
                       "local_rank": int(os.environ["LOCAL_RANK"]),
                       "master": os.environ["MASTER_ADDR"]}, f)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
