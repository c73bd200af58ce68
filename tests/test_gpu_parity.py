"""CUDA engine vs the CPU oracle, bit for bit (run on the B200 with -m gpu).

Paths, search costs and complete distance fields from libmr_cuda.so must equal
the oracle's on every golden case of the reference, on seeded adversarial
grids (zero costs, saturating prices, own pads, board node/edge/via masks,
static via masks with exemptions, restricted vias, directed prices) and on the
benchmark boards.
"""
import numpy as np
import pytest

from conftest import case_grid, case_nets, load_golden
import mrcuda
from mrcuda import workloads as W
from mrcuda.types import COST_MAX, Dims, Grid, IsolatedRouteRequest, IsolatedRouteWindow, NetEndpoints

pytestmark = pytest.mark.gpu
CASES = load_golden()


@pytest.fixture(scope="module", params=[1, 2], ids=["cta-tiles", "warp-tiles"])
def engine(request):
    """Every test runs on both default schedules: a CTA per tile and a warp per tile."""
    e = mrcuda.Engine(0)
    e.set_schedule(request.param)
    yield e
    e.close()


def _request(oracle, case):
    grid = case_grid(case)
    nets = case_nets(case)
    wins = case.get("windows")
    windows = ([IsolatedRouteWindow(*w) for w in wins] if wins is not None
               else [oracle.net_window(grid.dims, n) for n in nets])
    return IsolatedRouteRequest(grid, nets, windows, case["x"], case["y"], case["vias"])


def _window_slice(full: np.ndarray, dims: Dims, w: IsolatedRouteWindow) -> np.ndarray:
    f = full.reshape(dims.layers, dims.h, dims.w)
    return f[:, w.y0:w.y1 + 1, w.x0:w.x1 + 1].reshape(-1)


def _assert_fields(oracle, req, out, nets_idx=None):
    for i, net in enumerate(req.nets):
        if nets_idx is not None and i not in nets_idx:
            continue
        win = out.field_windows[i]
        dist, _ = oracle.isolated_field(req.grid, req.x_edge_costs, req.y_edge_costs, req.via_edge_costs, net, win,
                                        req.directed_in_costs)
        np.testing.assert_array_equal(out.fields[i], _window_slice(dist, req.grid.dims, win), err_msg=f"net {i}")


@pytest.mark.parametrize("case", [c for c in CASES if c["kind"] in ("isolated", "isolated_window")],
                         ids=lambda c: c["name"])
def test_golden_isolated_cases(engine, oracle, case):
    req = _request(oracle, case)
    retry = case["kind"] == "isolated"
    exp_paths, exp_costs = oracle.isolated_batch(req, retry_full=retry, mode="astar",
                                                 via_h_cost=case.get("via_h_cost"))
    got = engine.route_isolated_batch(req, retry_full=retry, keep_fields=True)
    assert got.paths == exp_paths
    assert got.search_costs == exp_costs
    exp = case.get("expect") or {}
    if "paths" in exp:
        assert got.paths == exp["paths"]
    if "search_costs" in exp:
        assert got.search_costs == exp["search_costs"]
    _assert_fields(oracle, req, got)
    # the plain form (one net per launch sequence) computes the same answers
    plain = engine.route_isolated_plain(req, retry_full=retry)
    assert plain.paths == exp_paths
    assert plain.search_costs == exp_costs


@pytest.mark.parametrize("case", [c for c in CASES if c["kind"] == "lee"], ids=lambda c: c["name"])
def test_golden_lee_cases(engine, oracle, case):
    grid = case_grid(case)
    nets = case_nets(case)
    board = engine.route_lee(grid, nets)
    exp = [oracle.lee_route_one(grid, n) for n in nets]
    assert [r.path for r in board.results] == [e[0] for e in exp if e is not None]
    assert [r.cost for r in board.results] == [e[1] for e in exp if e is not None]
    assert board.unrouted == [n.net for n, e in zip(nets, exp) if e is None]
    pins = case.get("expect") or {}
    if "path" in pins:
        assert board.results[0].path == pins["path"]
    if "cost" in pins:
        assert board.results[0].cost == pins["cost"]


@pytest.mark.parametrize("case", [c for c in CASES if c["kind"] in ("lee", "field")], ids=lambda c: c["name"])
def test_golden_distance_fields(engine, oracle, case):
    grid = case_grid(case)
    sources = list(range(len(grid.dims))) + [len(grid.dims) + 5]
    got = engine.distance_fields(grid, sources)
    for k, s in enumerate(sources):
        exp = oracle.bfs_distance_field(grid, s) if s < len(grid.dims) else np.full(len(grid.dims), COST_MAX)
        np.testing.assert_array_equal(got[k], exp, err_msg=f"source {s}")


def _random_case(rng, trial, directed=False, max_side=40, max_layers=4, min_layers=1):
    w, h = int(rng.integers(1, max_side)), int(rng.integers(1, max_side))
    layers = int(rng.integers(min_layers, max_layers + 1))
    dims = Dims(w, h, layers)
    n = len(dims)
    cost = rng.integers(0, 9, n).astype(np.uint32)
    if trial % 5 == 0:
        cost[rng.random(n) < 0.05] = COST_MAX - 1
    cost[rng.random(n) < 0.2] = COST_MAX
    board = None
    if trial % 3 == 0:
        board = (rng.integers(0, 64, n) * (rng.random(n) < 0.25)).astype(np.uint8)
    vf = (rng.random(n) < 0.3).astype(np.uint8) if trial % 4 == 1 else None
    grid = Grid(dims, cost, board, vf)
    big = trial % 7 == 3
    x = rng.integers(0, 0xFFFFFFFF if big else 40, max(w - 1, 0), dtype=np.uint64).astype(np.uint32)
    y = rng.integers(0, 40, max(h - 1, 0)).astype(np.uint32)
    vias = [None if rng.random() < 0.3 else int(rng.choice([0, 7, 30, 0xFFFFFFFF])) for _ in range(layers - 1)]
    d = None
    if directed:
        d = rng.integers(0, 60, (n, 4)).astype(np.uint32)
        d[rng.random((n, 4)) < 0.1] = COST_MAX
    nets = []
    legal = [c for c in range(n) if not (board is not None and board[c] & 1)]
    if not legal:
        return None
    for i in range(int(rng.integers(1, 12))):
        src, dst = int(rng.choice(legal)), int(rng.choice(legal))
        pads = sorted({c for c in (src, dst) if grid.is_obstacle(c)} |
                      {int(c) for c in rng.integers(0, n, int(rng.integers(0, 3)))})
        vpads = [c for c in pads if rng.random() < 0.5]
        nets.append(NetEndpoints(f"r{trial}-{i}", src, dst, pads, vpads))
    wins = []
    for i, nt in enumerate(nets):
        if i % 3 == 0:
            wins.append(IsolatedRouteWindow.full(dims))
        elif i % 3 == 1:
            wins.append(mrcuda.net_windows(dims, [nt])[0])
        else:
            x0, x1 = sorted(int(v) for v in rng.integers(0, w, 2))
            y0, y1 = sorted(int(v) for v in rng.integers(0, h, 2))
            wins.append(IsolatedRouteWindow(x0, y0, x1, y1))
    return IsolatedRouteRequest(grid, nets, wins, x, y, vias, d)


@pytest.mark.parametrize("directed", [False, True])
def test_seeded_adversarial_grids(engine, oracle, directed):
    rng = np.random.default_rng(2024 + directed)
    checked = 0
    for trial in range(120):
        req = _random_case(rng, trial, directed)
        if req is None:
            continue
        for retry in (True, False):
            exp = oracle.isolated_batch(req, retry_full=retry, mode="field")
            got = engine.route_isolated_batch(req, retry_full=retry, keep_fields=True)
            assert (got.paths, got.search_costs) == exp, (trial, retry)
            _assert_fields(oracle, req, got)
            checked += 1
    assert checked > 150


@pytest.mark.parametrize("layers", [1, 2, 3, 5, 8, 12])
def test_tile_shapes_and_multi_tile_windows(engine, oracle, layers):
    """Windows spanning many 32xTH tiles (TH shrinks with the layer count and
    with directed prices), serpentine walls that force repeated tile visits."""
    rng = np.random.default_rng(layers)
    w, h = 150, 70
    dims = Dims(w, h, layers)
    cost = rng.integers(1, 4, len(dims)).astype(np.uint32).reshape(layers, h, w)
    for k, x in enumerate(range(10, w - 5, 14)):
        if k % 2 == 0:
            cost[:, 0:h - 3, x] = COST_MAX
        else:
            cost[:, 3:h, x] = COST_MAX
    grid = Grid(dims, cost.reshape(-1))
    nets = [NetEndpoints("a", dims.idx3(1, 1, 0), dims.idx3(w - 2, h - 2, layers - 1)),
            NetEndpoints("b", dims.idx3(w - 1, 0, layers // 2), dims.idx3(0, h - 1, 0)),
            NetEndpoints("c", dims.idx3(70, 35, 0), dims.idx3(71, 35, 0))]
    wins = [IsolatedRouteWindow.full(dims)] * 3
    for directed in (None, rng.integers(1, 30, (len(dims), 4)).astype(np.uint32)):
        req = IsolatedRouteRequest(grid, nets, wins, rng.integers(1, 20, w - 1), rng.integers(1, 20, h - 1),
                                   [5] * (layers - 1), directed)
        exp = oracle.isolated_batch(req, mode="field")
        got = engine.route_isolated_batch(req, keep_fields=True)
        assert (got.paths, got.search_costs) == exp
        _assert_fields(oracle, req, got)


def test_plain_board_full_parity(engine, oracle):
    """128x128x2, 64 nets, complete fields + canonical paths, bit-exact."""
    wl = W.plain_board()
    req = wl.request()
    exp = oracle.isolated_batch(req, mode="astar")
    got = engine.route_isolated_batch(req, keep_fields=True)
    assert (got.paths, got.search_costs) == exp
    _assert_fields(oracle, req, got)
    assert all(p is not None for p in got.paths)


def test_congestion_board_parity(engine, oracle):
    """512x512x4 with an exact polygon outline and directed prices: every path
    and cost of all 256 nets, and complete fields of a sample of nets."""
    wl = W.congestion_board()
    req = wl.request()
    exp = oracle.isolated_batch(req, mode="astar")
    got = engine.route_isolated_batch(req, keep_fields=True)
    assert got.paths == exp[0]
    assert got.search_costs == exp[1]
    _assert_fields(oracle, req, got, nets_idx={0, 1, 2, 100, 255})
    for net, p in zip(req.nets, got.paths):
        if p is not None:
            assert oracle.provider_path_is_valid(req.grid, [True] * 3, net, p)


def test_deterministic_across_calls_and_batches(engine):
    wl = W.scaled(W.congestion_board(), 40)
    a = engine.route_isolated_batch(wl.request())
    b = engine.route_isolated_batch(wl.request())
    assert a.paths == b.paths and a.search_costs == b.search_costs
    board = engine.board(wl.grid, wl.x, wl.y, wl.vias, wl.directed)
    batch = mrcuda.Batch(board, wl.nets, wl.windows)
    for _ in range(3):
        batch.launch()
        c = batch.finish()
        assert c.paths == a.paths and c.search_costs == a.search_costs
    # relax, path offsets, path walk (+ the seed kernel of the queue schedules;
    # the price planes of the schedules that read them were computed by the
    # first launch of this layout and are not launched again)
    sched = batch.config()["schedule"]
    assert batch.kernel_launches == 3 + {0: 0, 1: 1, 2: 1, 3: 1}[sched]
    # every configuration the autotuner tries computes the same answer (on a
    # context of its own, so the tuned choice does not steer the other tests)
    e2 = mrcuda.Engine(0)
    board2 = e2.board(wl.grid, wl.x, wl.y, wl.vias, wl.directed)
    batch2 = mrcuda.Batch(board2, wl.nets, wl.windows)
    tuned = batch2.autotune()
    assert tuned["schedule"] in (0, 1, 2, 3)
    assert tuned["tile_h"] in (8, 16, 32, 64) and tuned["threads"] in (128, 256)
    batch2.launch()
    c = batch2.finish()
    assert c.paths == a.paths and c.search_costs == a.search_costs
    batch2.close()
    board2.close()
    e2.close()


def test_edge_cases_and_errors(engine):
    dims = Dims(5, 3)
    grid = Grid.filled(dims, 1)
    x, y = [16] * 4, [16] * 2
    # empty batch
    r = engine.route_isolated_batch(IsolatedRouteRequest(grid, [], [], x, y, []))
    assert r.paths == [] and r.search_costs == []
    # zero-length net and a window that excludes the source
    nets = [NetEndpoints("z", 7, 7), NetEndpoints("outside", 0, 14)]
    wins = [IsolatedRouteWindow.full(dims), IsolatedRouteWindow(2, 0, 4, 2)]
    r = engine.route_isolated_batch(IsolatedRouteRequest(grid, nets, wins, x, y, []), retry_full=False)
    assert r.paths == [[7], None] and r.search_costs[0] == 0
    r = engine.route_isolated_batch(IsolatedRouteRequest(grid, nets, wins, x, y, []), retry_full=True)
    assert r.paths[1] is not None and r.retried == 1
    # foreign obstacle endpoint, out-of-range pad, board-forbidden endpoint
    g2 = Grid.filled(dims, 1)
    g2.set(3, COST_MAX)
    with pytest.raises(mrcuda.InvalidEndpoint):
        engine.route_isolated_batch(IsolatedRouteRequest(g2, [NetEndpoints("f", 0, 3)], wins[:1], x, y, []))
    with pytest.raises(mrcuda.InvalidEndpoint):
        engine.route_isolated_batch(
            IsolatedRouteRequest(grid, [NetEndpoints("p", 0, 3, [99])], wins[:1], x, y, []))
    g3 = Grid(dims, np.ones(15, np.uint32), np.array([1] + [0] * 14, np.uint8))
    with pytest.raises(mrcuda.InvalidEndpoint):
        engine.route_isolated_batch(IsolatedRouteRequest(g3, [NetEndpoints("b", 0, 3)], wins[:1], x, y, []))
    # misaligned shapes: wrong edge vector length, bad window
    with pytest.raises(mrcuda.InvalidArgument):
        engine.route_isolated_batch(IsolatedRouteRequest(grid, [NetEndpoints("s", 0, 3)], wins[:1], [16] * 3, y, []))
    with pytest.raises(mrcuda.InvalidArgument):
        engine.route_isolated_batch(
            IsolatedRouteRequest(grid, [NetEndpoints("s", 0, 3)], [IsolatedRouteWindow(3, 0, 1, 2)], x, y, []))
    # the provider seam returns aligned Optional paths
    prov = mrcuda.CudaIsolatedProvider(engine)
    paths = prov.route_isolated_batch(IsolatedRouteRequest(grid, nets, wins, x, y, []))
    assert paths[0] == [7] and paths[1] is not None


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("tile_cfg", [(8, 128), (8, 256), (16, 128), (16, 256), (32, 128), (32, 256), (64, 128),
                                      (64, 256)])
def test_every_relax_configuration_is_bit_exact(engine, oracle, tile_cfg, schedule):
    """The autotuner may pick any tile height / CTA width / schedule (rounds or
    the asynchronous queue): each must reproduce the oracle."""
    rng = np.random.default_rng(sum(tile_cfg))
    for trial in range(6):
        req = _random_case(rng, trial, directed=trial % 2 == 1, max_side=90, max_layers=3)
        if req is None:
            continue
        exp = oracle.isolated_batch(req, retry_full=False, mode="field")
        board = engine.board(req.grid, req.x_edge_costs, req.y_edge_costs, req.via_edge_costs, req.directed_in_costs)
        batch = mrcuda.Batch(board, req.nets, req.windows, retry_full=False)
        batch.set_config(*tile_cfg)
        batch.set_schedule(schedule)
        batch.launch()
        got = batch.finish()
        assert (got.paths, got.search_costs) == exp, (tile_cfg, trial)
        batch.close()
        board.close()


@pytest.mark.parametrize("tile_cfg", [(8, 256), (16, 128)])
def test_queue_schedule_on_the_congestion_board(engine, oracle, tile_cfg):
    """The asynchronous queue (tiles relaxed by several CTAs at once, labels
    merged with atomicMin) on all 256 nets of the congestion board, three
    launches in a row: every path and cost equals the oracle's."""
    wl = W.congestion_board()
    req = wl.request()
    exp = oracle.isolated_batch(req, mode="astar")
    board = engine.board(wl.grid, wl.x, wl.y, wl.vias, wl.directed)
    batch = mrcuda.Batch(board, wl.nets, wl.windows, keep_fields=True)
    batch.set_config(*tile_cfg)
    batch.set_schedule(1)
    for _ in range(3):
        batch.launch()
        got = batch.finish()
        assert got.paths == exp[0] and got.search_costs == exp[1]
    _assert_fields(oracle, req, got, nets_idx={0, 7, 128, 255})
    assert batch.config()["schedule"] == 1
    batch.close()
    board.close()


@pytest.mark.parametrize("directed", [False, True], ids=["axis", "directed"])
@pytest.mark.parametrize("tile_cfg", [(8, 256), (16, 256), (32, 256)])
def test_tiled_walk_board_edges_and_long_paths(engine, oracle, tile_cfg, directed):
    """The queue form with price planes walks each path inside shared-memory
    windows placed ahead of the walk, which may start left of or above the
    board: nets between corners and along the edges of an open board, with
    full-board windows and no own pads (so every step off the endpoints' stacks
    reads the staged planes), must give the oracle's paths and costs."""
    rng = np.random.default_rng(7 + tile_cfg[0] + int(directed))
    w, h, layers = 150, 110, 3
    dims = Dims(w, h, layers)
    n = len(dims)
    grid = Grid(dims, rng.integers(1, 4, n).astype(np.uint32), None, None)
    x = rng.integers(1, 40, w - 1).astype(np.uint32)
    y = rng.integers(1, 40, h - 1).astype(np.uint32)
    vias = [7, 30]
    d = rng.integers(1, 60, (n, 4)).astype(np.uint32) if directed else None

    def cell(l, yy, xx):
        return (l * h + yy) * w + xx

    pairs = [(cell(0, 0, 0), cell(0, h - 1, w - 1)), (cell(0, h - 1, w - 1), cell(2, 0, 0)),
             (cell(1, 0, w - 1), cell(1, h - 1, 0)), (cell(2, h - 1, 0), cell(0, 0, w - 1)),
             (cell(0, 0, 3), cell(0, 0, w - 4)), (cell(1, 5, 0), cell(1, h - 6, 0)),
             (cell(2, h - 1, 10), cell(2, h - 1, w - 11)), (cell(0, 40, w - 1), cell(2, 70, w - 1))]
    nets = [NetEndpoints(f"edge{i}", s, t) for i, (s, t) in enumerate(pairs)]
    wins = [IsolatedRouteWindow.full(dims) for _ in nets]
    req = IsolatedRouteRequest(grid, nets, wins, x, y, vias, d)
    exp = oracle.isolated_batch(req, retry_full=False, mode="field")
    board = engine.board(grid, x, y, vias, d)
    batch = mrcuda.Batch(board, nets, wins, retry_full=False)
    batch.set_config(*tile_cfg)
    batch.set_schedule(1)
    batch.launch()
    got = batch.finish()
    assert (got.paths, got.search_costs) == exp, tile_cfg
    assert all(p is not None and len(p) > 30 for p in got.paths)  # the shortest, a stack change, has 39-51 cells
    assert batch.config()["schedule"] == 1
    batch.close()
    board.close()


@pytest.mark.parametrize("layers", [1, 2, 3, 4, 5, 6, 8, 9, 12, 16])
def test_warp_schedule_every_tile_geometry(engine, oracle, layers):
    """The warp schedule's tile width follows the layer count (4 * 32 /
    next_pow2(layers) cells): seeded adversarial boards of every geometry,
    ragged windows included, against the oracle's complete fields."""
    rng = np.random.default_rng(700 + layers)
    for trial in range(4):
        req = _random_case(rng, trial, directed=trial % 2 == 1, max_side=70, max_layers=layers,
                           min_layers=layers)
        if req is None:
            continue
        exp = oracle.isolated_batch(req, retry_full=False, mode="field")
        board = engine.board(req.grid, req.x_edge_costs, req.y_edge_costs, req.via_edge_costs, req.directed_in_costs)
        batch = mrcuda.Batch(board, req.nets, req.windows, retry_full=False, keep_fields=True)
        batch.set_schedule(2)
        batch.launch()
        got = batch.finish()
        assert (got.paths, got.search_costs) == exp, (layers, trial)
        _assert_fields(oracle, req, got)
        st = batch.stats()
        assert st["activations"] >= 1 or not any(p is not None for p in got.paths)
        batch.close()
        board.close()


def test_warp_schedule_refuses_more_than_16_layers(engine):
    dims = Dims(20, 10, 17)
    grid = Grid.filled(dims, 1)
    board = engine.board(grid, [1] * 19, [1] * 9, [3] * 16)
    batch = mrcuda.Batch(board, [NetEndpoints("a", 0, len(dims) - 1)], [IsolatedRouteWindow.full(dims)])
    with pytest.raises(mrcuda.LimitExceeded):
        batch.set_schedule(2)
    batch.close()
    board.close()


def test_warp_schedule_on_the_congestion_board(engine, oracle):
    """All 256 nets of the congestion board on the warp schedule, three
    launches in a row, plus complete fields of a sample of nets."""
    wl = W.congestion_board()
    req = wl.request()
    exp = oracle.isolated_batch(req, mode="astar")
    board = engine.board(wl.grid, wl.x, wl.y, wl.vias, wl.directed)
    batch = mrcuda.Batch(board, wl.nets, wl.windows, keep_fields=True)
    batch.set_schedule(2)
    assert batch.config()["schedule"] == 2
    for _ in range(3):
        batch.launch()
        got = batch.finish()
        assert got.paths == exp[0] and got.search_costs == exp[1]
    _assert_fields(oracle, req, got, nets_idx={0, 7, 128, 255})
    st = batch.stats()
    assert st["activations"] >= st["tiles"] // 4 and st["rows"] > 0
    batch.close()
    board.close()
