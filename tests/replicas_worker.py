"""Rank process for test_replicas_gloo.py: launched by torch.distributed.run on CPU with the gloo
backend; writes what the replica helpers returned on this rank to <out_dir>/rank<r>.json."""
import datetime
import json
import sys
from pathlib import Path

import torch.distributed as dist

from bug_defense_b200 import replicas


def main(out_dir: str) -> None:
    rank, world, local = replicas.dist_env()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    share = replicas.rank_share(list(range(24)), rank, world)
    out = {"rank": rank, "world": world, "local": local, "share": share,
           "max": replicas.max_over_ranks(10.0 + 3.5 * rank),
           "total": replicas.sum_over_ranks(len(share)),
           "seed": replicas.replica_seed(7, rank)}
    dist.barrier()
    dist.destroy_process_group()
    Path(out_dir, f"rank{rank}.json").write_text(json.dumps(out))


if __name__ == "__main__":
    main(sys.argv[1])
