"""bench.py's multi-rank path on CPU (gloo, world size 2): the job time is the slowest rank's and
the job value counts every replica; in the reference arm only rank 0 works and prints."""
import contextlib
import io
import json
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), OMP_NUM_THREADS="1")
    import torch.distributed as dist
    import bench
    w, r, _ = bench.dist_init(world)
    ms = bench.max_over_ranks(10.0 + 5.0 * r, w, "cpu")
    val = bench.job_value(w, 1000, 4, ms)
    args = bench.argparse.Namespace(gpus=world, steps=1, warmup=1, impl="reference", shape="12,10,8")
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        rc = bench.run_reference(args, w, r)
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, ms, val, rc, out.getvalue()))


def test_two_rank_timing_and_reference_arm():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, ms, val, rc, text in res:
        assert ms == 15.0                                  # the slower rank's time on both ranks
        assert abs(val - 2 * 1000 * 4 / 0.015 / 1e6) < 1e-9
        assert rc == 0
    assert res[1][4] == ""                                 # rank 1 does no reference work
    line = json.loads(res[0][4].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
