"""Multi-rank host logic on CPU (gloo, world size 2): net sharding, the
max-over-ranks timing reduction, and failure detection of a rank that dies
between steps (heartbeat through the store, bounded waits only)."""
import datetime
import multiprocessing as mp
import os
import socket
import sys
import time

import numpy as np
import pytest

from mrcuda.dist import Heartbeat, RankFailure, max_over_ranks, shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_partitions_every_net():
    for n in (0, 1, 7, 256, 4096):
        for world in (1, 2, 3, 8):
            ranges = [shard(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [e - b for b, e in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _worker(rank, world, port, mode, q):
    try:
        import torch.distributed as dist

        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        sys.path.insert(0, os.path.join(root, "metal-route_b200"))
        from mrcuda.dist import Heartbeat, RankFailure, max_over_ranks, shard

        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
        if mode == "ok":
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=20))
            b, e = shard(257, rank, world)
            m = max_over_ranks(10.0 + rank)
            import torch

            sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
            dist.all_gather(sizes, torch.tensor([e - b]))
            dist.barrier()
            dist.destroy_process_group()
            q.put((rank, "ok", m, sum(int(s.item()) for s in sizes)))
        else:
            store = dist.TCPStore("127.0.0.1", port, world, is_master=rank == 0,
                                  timeout=datetime.timedelta(seconds=10))
            hb = Heartbeat(store, rank, world, timeout_s=2.0)
            for step in range(3):
                if rank == 1 and step == 2:
                    raise SystemExit(3)  # this rank dies between steps
                hb.beat(step)
                t0 = time.monotonic()
                try:
                    hb.check(step)
                except RankFailure as err:
                    q.put((rank, "detected", step, round(time.monotonic() - t0, 2)))
                    return
            q.put((rank, "finished", None, None))
    except SystemExit:
        q.put((rank, "died", None, None))
    except Exception as err:  # report instead of hanging the parent
        q.put((rank, "error", repr(err), None))


def _run(mode, world=2, timeout=60):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = []
    deadline = time.monotonic() + timeout
    while len(out) < world and time.monotonic() < deadline:
        try:
            out.append(q.get(timeout=1.0))
        except Exception:
            pass
    for p in ps:
        p.join(timeout=5)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_two_ranks_shard_and_reduce():
    out = _run("ok")
    assert [o[1] for o in out] == ["ok", "ok"], out
    assert all(o[2] == 11.0 for o in out)  # max over ranks
    assert all(o[3] == 257 for o in out)  # the shards cover every net


def test_a_dead_rank_is_detected_within_the_timeout():
    out = _run("fail")
    assert ("died" in [o[1] for o in out if o[0] == 1]), out
    r0 = [o for o in out if o[0] == 0][0]
    assert r0[1] == "detected" and r0[2] == 2 and r0[3] <= 5.0, out


def test_max_over_ranks_without_a_group():
    assert max_over_ranks(3.5) == 3.5


def _shard_worker(rank, world, port, q):
    try:
        import torch
        import torch.distributed as dist

        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        for p in (os.path.join(root, "metal-route_b200"), os.path.join(root, "oracle")):
            sys.path.insert(0, p)
        import oracle as orc
        from mrcuda import workloads as W
        from snapshot_oracle import SnapshotShard

        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        wl = W.snapshot_board(w=96, h=80, layers=2, n_nets=40, median=30)
        req = wl.request()
        owned = [i % world == rank for i in range(len(req.nets))]
        sh = SnapshotShard(orc.get(), req, owned)

        def exchange():
            t = torch.from_numpy(sh.local.astype(np.int64))
            dist.all_reduce(t)
            sh.glob = t.numpy().astype(np.uint32)

        over = []
        for _ in range(4):
            sh.ripup()
            exchange()
            sh.route()
            exchange()
            over.append(sh.settle())
        q.put((rank, [sh.paths[i] for i in range(len(req.nets)) if owned[i]], over, sh.history.sum().item()))
        dist.destroy_process_group()
    except Exception as err:
        q.put((rank, "error", repr(err), None))



def test_sharded_round_protocol_with_two_gloo_ranks(oracle):
    """The sharded round run by two gloo ranks (the oracle as each rank's
    router, occupancy all-reduced between the phases) equals one unsharded
    snapshot negotiation over all nets."""
    from mrcuda import workloads as W
    from snapshot_oracle import SnapshotNegotiation

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    deadline = time.monotonic() + 120
    while len(out) < 2 and time.monotonic() < deadline:
        try:
            r = q.get(timeout=1.0)
            out[r[0]] = r
        except Exception:
            pass
    for p in ps:
        p.join(timeout=5)
        if p.is_alive():
            p.kill()
    assert len(out) == 2 and all(v[1] != "error" for v in out.values()), out
    wl = W.snapshot_board(w=96, h=80, layers=2, n_nets=40, median=30)
    whole = SnapshotNegotiation(oracle, wl.request())
    over = [whole.round().get("overused_edges", 0) for _ in range(4)]
    assert out[0][2] == over and out[1][2] == over
    assert out[0][3] == out[1][3] == int(whole.history.sum())
    for rank in (0, 1):
        mine = [whole.paths[i] for i in range(40) if i % 2 == rank]
        assert out[rank][1] == mine
