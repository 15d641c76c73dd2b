"""Multi-rank host logic of bench.py on CPU (gloo, world size 2).

On GPUs bench.py runs one process per GPU over NCCL, each rendering its own
image (weak scaling, no collective on the data path); the only collectives
are the barrier around the timed region and the max / sum over ranks of the
timings.  Here the same functions run as two gloo processes.
"""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "IPG_DIST_BACKEND": "gloo"})
    sys.path.insert(0, ROOT)
    try:
        import bench
        import torch.distributed as dist
        r, w, local = bench.dist_setup()
        out = {"rank": r, "world": w, "local": local}
        # every rank times its own image; the job's time is the slowest rank's
        ms = 100.0 * (r + 1)
        bench.barrier(w)
        out["ms_max"] = bench.max_over_ranks(ms, w)
        out["steps_sum"] = bench.sum_over_ranks(1000.0 * (r + 1), w)
        out["value"] = bench.images_per_s(w, 5, out["ms_max"])
        # the reference arm does its work on rank 0 only; other ranks leave at once
        if r != 0:

            class A:
                steps = warmup = 1
                gpus = w
                m_unit = bench.M_UNIT
            out["ref_rc"] = bench.run_reference_arm(A())
        bench.barrier(w)
        dist.destroy_process_group()
        q.put(out)
    except Exception as ex:  # reported to the parent
        q.put({"rank": rank, "error": repr(ex)})


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    outs.sort(key=lambda o: o["rank"])
    assert all("error" not in o for o in outs), outs
    for o in outs:
        assert o["world"] == 2 and o["local"] == o["rank"]
        assert o["ms_max"] == pytest.approx(200.0)
        assert o["steps_sum"] == pytest.approx(3000.0)
        assert o["value"] == pytest.approx(2 * 5 / 0.2)
    assert outs[1]["ref_rc"] == 0
