"""Sharded negotiation rounds on one GPU: two shards (each routing half of the
nets, exchanging occupancy between the phases of every round) reproduce one
unsharded negotiation over all nets, round by round, bit for bit.  On several
GPUs the exchange is an all-reduce (mrcuda.dist.sharded_negotiation_round);
here the two shards live in one process and the exchange is a plain sum."""
import numpy as np
import pytest

import mrcuda
from mrcuda import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = mrcuda.Engine(0)
    yield e
    e.close()


def _exchange(shards):
    occ = [s.occupancy() for s in shards]
    total = occ[0][0].clone()
    for loc, _ in occ[1:]:
        total += loc
    for _, glob in occ:
        glob.copy_(total)


@pytest.mark.parametrize("split", ["halves", "interleaved"])
def test_two_shards_equal_one_negotiation(engine, split):
    wl = W.snapshot_board(w=192, h=160, layers=3, n_nets=96, median=60)
    req = wl.request()
    n = len(req.nets)
    owned_a = [i < n // 2 for i in range(n)] if split == "halves" else [i % 2 == 0 for i in range(n)]
    owned_b = [not x for x in owned_a]
    whole = engine.negotiation(req)
    shards = [engine.negotiation(req, owned=owned_a), engine.negotiation(req, owned=owned_b)]
    for r in range(6):
        ref = whole.round()
        for s in shards:
            s.ripup()
        _exchange(shards)
        for s in shards:
            s.route()
        _exchange(shards)
        st = [s.settle() for s in shards]
        assert sum(x["dirty"] for x in st) == ref["dirty"], r
        assert all(x["overused_edges"] == ref["overused_edges"] for x in st), r
        pa, pb = shards[0].paths(), shards[1].paths()
        merged = [pa[i] if owned_a[i] else pb[i] for i in range(n)]
        assert merged == whole.paths(), r
        pw, hw, _ = whole.read()
        la, ga = shards[0].occupancy()
        lb, _ = shards[1].occupancy()
        np.testing.assert_array_equal((la + lb).cpu().numpy().reshape(-1, 4), pw.astype(np.int32))
        np.testing.assert_array_equal(ga.cpu().numpy().reshape(-1, 4), pw.astype(np.int32))
        _, ha, _ = shards[0].read()
        np.testing.assert_array_equal(ha, hw)
        assert sorted(shards[0].dirty() + shards[1].dirty()) == whole.dirty(), r
    for s in shards + [whole]:
        s.close()


def test_shard_phases_are_ordered(engine):
    wl = W.snapshot_board(w=64, h=64, layers=2, n_nets=8, median=20)
    shard = engine.negotiation(wl.request(), owned=[True] * 8)
    with pytest.raises(mrcuda.InvalidArgument):
        shard.route()
    with pytest.raises(mrcuda.InvalidArgument):
        shard.round()  # a shard runs phase by phase
    shard.ripup()
    with pytest.raises(mrcuda.InvalidArgument):
        shard.ripup()
    shard.close()
