"""bench.py's multi-GPU path at world size 2, run as two CPU processes over gloo: every rank
reads its place from the launcher's environment, joins the replica process group, and the
job's timings are the maximum over ranks (the slowest replica); the reference arm does its
work on rank 0 only.  The replicas share no data-path collective, so nothing else crosses
ranks."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE="2")
    import bench

    ws, r, lr = bench.dist_env()
    dist = bench.init_replicas(ws, lr, backend="gloo")
    try:
        # each replica's own timings; the job's are the slowest replica's
        vals = bench.max_over_ranks(dist, [100.0 + 5 * rank, 7.0 - rank], device="cpu")
        skipped = bench.run_reference(None) == 0 if r == 1 else None  # rank 1: no reference work
        dist.barrier()
        out.put((r, ws, vals, skipped))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=180) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert res == [(0, 2, [105.0, 7.0], None), (1, 2, [105.0, 7.0], True)]
    assert all(p.exitcode == 0 for p in procs)


def test_single_process_needs_no_group():
    import bench

    assert bench.init_replicas(1, 0) is None
    assert bench.max_over_ranks(None, [3.0, 4.0]) == [3.0, 4.0]
