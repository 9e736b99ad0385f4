"""One rank of the two-rank CPU check of bench.py's multi-process path (run by
tests/test_multirank.py under torch.distributed.run with the gloo backend).

Each rank reports a different step time; every rank must see the slowest one, the job rate
must count the units of all ranks over that time, and a rank other than 0 of the
reference arm must return at once without work."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def main(out_dir: str) -> int:
    ws, rank, _ = bench._dist()
    pg = bench.init_ranks("gloo", timeout_s=30)
    local_s = 1.0 + 1.5 * rank                 # rank 0: 1.0 s, rank 1: 2.5 s
    slowest = bench.max_over_ranks(pg, local_s, "cpu")
    rate = bench.job_rate(ws, 1000.0, 4, slowest)
    pg.barrier()
    skipped = None
    if rank != 0:   # the reference arm runs on rank 0 only
        import argparse
        skipped = bench.run_reference(argparse.Namespace(steps=1, warmup=0, gpus=ws))
    pg.barrier()
    pg.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"ws": ws, "slowest": slowest, "rate": rate, "reference_rc": skipped}, f)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1]))
