"""The multi-GPU plumbing of replica runs (one independent box per rank),
with the gloo backend on CPU: two ranks, each running the CPU oracle on its
own seeded box, reduce their step times (max) and particle counts (sum) the
way bench.py reports a run over N GPUs."""
import multiprocessing as mp
import os
import socket
import time

from cm_halofinder_b200.replicas import Replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from cm_halofinder_b200 import synth
    from oracle import cpu
    rep = Replicas("gloo", timeout_s=60)
    w = synth.config2(seed=500 + rank, scale=(3000 + 1000 * rank) / 256 ** 3)
    rep.barrier()
    t0 = time.perf_counter()
    res = cpu.run(w)
    dt = time.perf_counter() - t0
    t_max = rep.max(dt)
    n_all = rep.sum(w.n)
    nh_all = rep.sum(res["stats"]["nhalos"])
    out.put((rank, w.n, dt, t_max, n_all, res["stats"]["nhalos"], nh_all))
    rep.close()


def test_two_gloo_ranks_reduce_time_and_counts():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    rows = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, n0, dt0, tmax0, nall0, nh0, nhall0), (r1, n1, dt1, tmax1, nall1, nh1, nhall1) = rows
    assert (r0, r1) == (0, 1) and n0 != n1
    # every rank sees the slowest rank's time and the totals
    assert tmax0 == tmax1 == max(dt0, dt1)
    assert nall0 == nall1 == n0 + n1
    assert nhall0 == nhall1 == nh0 + nh1


def test_single_rank_needs_no_process_group():
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    rep = Replicas("gloo")
    assert (rep.rank, rep.world) == (0, 1) and rep.dist is None
    assert rep.max(2.5) == 2.5 and rep.sum(7) == 7.0
    rep.close()


def test_round_robin_share_covers_every_box_once():
    for world in (1, 2, 3, 8):
        got = sorted(b for r in range(world) for b in Replicas.share(64, r, world))
        assert got == list(range(64))
        sizes = [len(Replicas.share(64, r, world)) for r in range(world)]
        assert max(sizes) - min(sizes) <= 1
