"""Many independent instances in one persistent launch, vs the CPU oracle.

Covers the uneven-instance batch: instances of different sizes and layer
counts routed together (mrc_route_instances), batches spanning several resident
boards (mrc_batch_create_multi), the per-instance full-board retry, and CUDA
graph replay of a staged batch (mrc_batch_capture_graph).  Every answer must
equal the oracle's for that instance alone, bit for bit.
"""
import numpy as np
import pytest

import mrcuda
from mrcuda import workloads as W
from mrcuda.types import COST_MAX, Dims, Grid, IsolatedRouteRequest, IsolatedRouteWindow, NetEndpoints

from test_gpu_parity import _assert_fields, _random_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[1, 2], ids=["cta-tiles", "warp-tiles"])
def engine(request):
    """Every test runs on both default schedules: a CTA per tile and a warp per tile."""
    e = mrcuda.Engine(0)
    e.set_schedule(request.param)
    yield e
    e.close()


def _oracle_each(oracle, reqs, retry=True, mode="astar"):
    return [oracle.isolated_batch(r, retry_full=retry, mode=mode) for r in reqs]


def test_uneven_instances_match_oracle(engine, oracle):
    """64 uneven instances (2-8 layers, sides 16-1024) solved in one launch."""
    s = W.uneven_instances(seed=11, n_instances=64)
    reqs = s.requests()
    got = engine.route_instances(reqs, keep_fields=True)
    exp = _oracle_each(oracle, reqs)
    for k, (g, e) in enumerate(zip(got, exp)):
        assert (g.paths, g.search_costs) == e, k
    assert all(p is not None for g in got for p in g.paths)
    for k in (0, 1, 17, 40, 63):
        _assert_fields(oracle, reqs[k], got[k])


def test_mixed_instances_with_every_feature(engine, oracle):
    """Adversarial instances (board bits, via masks, directed prices, own pads,
    windows that need the retry) mixed with plain ones; layer counts 1-12."""
    rng = np.random.default_rng(77)
    reqs = []
    for trial in range(40):
        r = _random_case(rng, trial, directed=trial % 3 == 0, max_side=70, max_layers=12 if trial % 5 == 0 else 4)
        if r is not None:
            reqs.append(r)
    for retry in (True, False):
        got = engine.route_instances(reqs, retry_full=retry, keep_fields=True)
        exp = _oracle_each(oracle, reqs, retry=retry, mode="field")
        for k, (g, e) in enumerate(zip(got, exp)):
            assert (g.paths, g.search_costs) == e, (retry, k)
            _assert_fields(oracle, reqs[k], g)


def test_instance_retry_uses_its_own_board(engine, oracle):
    """A window that cuts the only corridor fails; the retry runs on that
    instance's whole board, not on another instance's."""
    dims = Dims(12, 6, 2)
    cost = np.ones((2, 6, 12), np.uint32)
    cost[:, 0:5, 6] = COST_MAX  # wall with a gap at y = 5
    g = Grid(dims, cost.reshape(-1))
    net = NetEndpoints("r", dims.idx3(1, 1, 0), dims.idx3(10, 1, 0))
    narrow = IsolatedRouteWindow(0, 0, 11, 3)
    a = IsolatedRouteRequest(g, [net], [narrow], [16] * 11, [16] * 5, [30])
    b = W.plain_board(seed=4, n_nets=3).request()
    got = engine.route_instances([b, a, b])
    exp = _oracle_each(oracle, [b, a, b])
    assert [(x.paths, x.search_costs) for x in got] == exp
    assert got[1].paths[0] is not None
    assert engine.route_instances([a], retry_full=False)[0].paths == [None]


def test_empty_and_degenerate_instances(engine, oracle):
    one = IsolatedRouteRequest(Grid.filled(Dims(1, 1, 1), 1), [NetEndpoints("z", 0, 0)],
                               [IsolatedRouteWindow(0, 0, 0, 0)], [], [], [])
    empty = IsolatedRouteRequest(Grid.filled(Dims(4, 4, 2), 1), [], [], [1] * 3, [1] * 3, [10])
    assert engine.route_instances([]) == []
    got = engine.route_instances([empty, one, empty])
    assert got[0].paths == [] and got[1].paths == [[0]] and got[1].search_costs == [0] and got[2].paths == []
    bad = IsolatedRouteRequest(Grid.filled(Dims(4, 4, 2), 1), [NetEndpoints("x", 0, 99)],
                               [IsolatedRouteWindow(0, 0, 3, 3)], [1] * 3, [1] * 3, [10])
    with pytest.raises(mrcuda.InvalidEndpoint):
        engine.route_instances([one, bad])


def test_multi_board_batch_equals_single_board_batches(engine, oracle):
    """One staged batch over three resident boards (2, 4 and 6 layers; one with
    directed prices) gives each net the answer of its own board."""
    plain = W.plain_board(seed=9, n_nets=12)
    cong = W.scaled(W.congestion_board(w=160, h=140), 10)
    six = W.plain_board(seed=10, w=90, h=70, layers=6, n_nets=9)
    wls = [plain, cong, six]
    boards = [engine.board(w.grid, w.x, w.y, w.vias, w.directed) for w in wls]
    nets, wins, nb = [], [], []
    order = [(k, i) for k, w in enumerate(wls) for i in range(len(w.nets))]
    rng = np.random.default_rng(3)
    rng.shuffle(order)
    for k, i in order:
        nets.append(wls[k].nets[i])
        wins.append(wls[k].windows[i])
        nb.append(k)
    batch = mrcuda.Batch(boards, nets, wins, net_board=nb, keep_fields=True)
    batch.launch()
    got = batch.finish()
    exp = {k: oracle.isolated_batch(w.request(), mode="astar") for k, w in enumerate(wls)}
    for j, (k, i) in enumerate(order):
        assert got.paths[j] == exp[k][0][i], (k, i)
        assert got.search_costs[j] == exp[k][1][i], (k, i)
    with pytest.raises(mrcuda.InvalidArgument):
        mrcuda.Batch(boards, nets[:2], wins[:2], net_board=[0, 3])


def test_graph_replay_matches_stream_launch(engine, oracle):
    """A captured graph replays the whole launch sequence; results and the relax
    timing event survive replay, and a re-tune drops the stale graph."""
    s = W.uneven_instances(seed=12, n_instances=24)
    boards = [engine.board(w.grid, w.x, w.y, w.vias, w.directed) for w in s.instances]
    nets = [w.nets[0] for w in s.instances]
    wins = [w.windows[0] for w in s.instances]
    nb = list(range(len(boards)))
    batch = mrcuda.Batch(boards, nets, wins, net_board=nb, time_kernels=True)
    batch.launch()
    ref = batch.finish()
    exp = _oracle_each(oracle, s.requests())
    assert [([p], [c]) for p, c in zip(ref.paths, ref.search_costs)] == exp
    batch.capture_graph()
    for _ in range(3):
        batch.launch()
        got = batch.finish()
        assert got.paths == ref.paths and got.search_costs == ref.search_costs
        assert batch.relax_ms() > 0.0
    batch.set_config(8, 128)
    batch.launch()
    got = batch.finish()
    assert got.paths == ref.paths
    batch.capture_graph()
    batch.launch()
    assert batch.finish().paths == ref.paths


def _pinned_request(engine, r, shifts=(0, 0, 0)):
    """`r` with its cost, masks and directed prices copied into page-locked
    memory, each array starting `shifts` bytes past a 16-byte boundary (cost,
    masks, directed)."""
    def pin(a, dtype, shift):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dtype).reshape(-1)
        blk = engine.pinned_empty(a.nbytes + 32, np.uint8)
        v = blk[shift:shift + a.nbytes].view(dtype)
        v[:] = a
        return v
    g = r.grid
    grid = Grid(g.dims, pin(g.cost, np.uint32, shifts[0]), pin(g.board_constraint, np.uint8, shifts[1]),
                pin(g.via_forbidden, np.uint8, shifts[1]))
    assert grid.cost.ctypes.data % 16 == shifts[0]  # no copy was made
    d = pin(r.directed_in_costs, np.uint32, shifts[2])
    return IsolatedRouteRequest(grid, r.nets, r.windows, r.x_edge_costs, r.y_edge_costs, r.via_edge_costs, d)


def _big_bytes(reqs):
    b = 0
    for r in reqs:
        n = len(r.grid.dims)
        b += 4 * n + (n if r.grid.board_constraint is not None or r.grid.via_forbidden is not None else 0)
        b += 16 * n if r.directed_in_costs is not None else 0
    return b


@pytest.mark.parametrize("shifts", [(0, 0, 0), (4, 1, 8)], ids=["aligned", "unaligned"])
def test_page_locked_instances_are_read_in_place(engine, oracle, shifts):
    """Instances whose board arrays are page-locked are gathered straight from
    host memory by one launch (16-byte, word and byte paths; flag bytes built
    from both masks); the answers equal the staged upload's and the oracle's.
    A set that mixes page-locked and pageable instances takes the staged path."""
    rng = np.random.default_rng(78)
    reqs = []
    for trial in range(40):
        r = _random_case(rng, trial, directed=trial % 3 == 0, max_side=70, max_layers=12 if trial % 5 == 0 else 4)
        if r is not None:
            reqs.append(r)
    pinned = [_pinned_request(engine, r, shifts) for r in reqs]
    before = engine.upload_stats()
    got = engine.route_instances(pinned, keep_fields=True)
    after = engine.upload_stats()
    assert after["in_place_bytes"] - before["in_place_bytes"] == _big_bytes(reqs)
    assert after["staged_bytes"] == before["staged_bytes"]
    exp = _oracle_each(oracle, reqs, mode="field")
    staged = engine.route_instances(reqs, keep_fields=True)
    for k, (g, s, e) in enumerate(zip(got, staged, exp)):
        assert (g.paths, g.search_costs) == e, k
        assert all(np.array_equal(a, b) for a, b in zip(g.fields, s.fields)), k
    mixed = [p if k % 2 else r for k, (p, r) in enumerate(zip(pinned, reqs))]
    before = engine.upload_stats()
    got = engine.route_instances(mixed)
    assert engine.upload_stats()["in_place_bytes"] == before["in_place_bytes"]
    assert [(g.paths, g.search_costs) for g in got] == exp


def test_page_locked_uneven_instances_span_many_chunks(engine, oracle):
    """256 uneven instances (boards up to 1024x1024x8, spans of many 64 KiB
    gather chunks) read in place equal the staged upload and the oracle."""
    s = W.uneven_instances(seed=12, n_instances=256)
    reqs = s.requests()
    pinned = [_pinned_request(engine, r) for r in reqs]
    got = engine.route_instances(pinned)
    staged = engine.route_instances(reqs)
    assert [(g.paths, g.search_costs) for g in got] == [(g.paths, g.search_costs) for g in staged]
    for k in range(0, 256, 16):
        assert (got[k].paths, got[k].search_costs) == oracle.isolated_batch(reqs[k], retry_full=True, mode="astar"), k


def test_page_locked_single_board_upload(engine, oracle):
    """A single-board call with page-locked arrays copies them in place."""
    rng = np.random.default_rng(79)
    r = None
    trial = 0
    while r is None:
        r = _random_case(rng, trial, directed=True, max_side=60, max_layers=4)
        trial += 1
    p = _pinned_request(engine, r)
    before = engine.upload_stats()
    got = engine.route_isolated_batch(p)
    assert engine.upload_stats()["in_place_bytes"] - before["in_place_bytes"] == _big_bytes([r])
    assert (got.paths, got.search_costs) == oracle.isolated_batch(r, retry_full=True, mode="field")
