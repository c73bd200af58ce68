"""CPU-side checks of the C-ABI library: it loads, exports every entry point the
header declares, computes windows like the reference, and fails loudly (never
falls back) when no CUDA device exists."""
import os
import re

import pytest

from conftest import ROOT
import mrcuda
from mrcuda.types import Dims, IsolatedRouteWindow, NetEndpoints


def _declared_symbols():
    with open(os.path.join(ROOT, "include", "mr_cuda.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(mrc_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = mrcuda.load_library()
    declared = _declared_symbols()
    assert len(declared) >= 20
    missing = [name for name in declared if not hasattr(lib, name)]
    assert missing == []


def test_abi_version_matches_header():
    with open(os.path.join(ROOT, "include", "mr_cuda.h")) as f:
        m = re.search(r"#define MRC_ABI_VERSION (\d+)u", f.read())
    assert mrcuda.load_library().mrc_abi_version() == int(m.group(1))


def test_library_windows_match_oracle(oracle):
    import numpy as np

    rng = np.random.default_rng(11)
    for _ in range(50):
        dims = Dims(int(rng.integers(1, 300)), int(rng.integers(1, 300)), int(rng.integers(1, 5)))
        n = len(dims)
        pads = [int(p) for p in rng.integers(0, n, int(rng.integers(0, 4)))]
        net = NetEndpoints("w", int(rng.integers(0, n)), int(rng.integers(0, n)), pads)
        assert mrcuda.net_windows(dims, [net])[0] == oracle.net_window(dims, net)


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and os.path.exists("/dev/nvidia0"),
                    reason="a GPU is present; the no-device contract is checked on CPU-only hosts")
def test_no_device_is_an_error_not_a_fallback():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(mrcuda.BackendUnavailable):
        mrcuda.Engine(0)


def test_many_request_marshalling_matches_the_struct_path():
    """route_instances writes its C request array from numpy columns; every field
    (grid, edge vectors, via prices and masks, nets, pads, windows) must equal
    what the one-request struct path writes."""
    import ctypes as C

    import numpy as np

    from mrcuda import api
    from mrcuda import workloads as W
    from mrcuda.types import Dims, Grid, IsolatedRouteRequest, IsolatedRouteWindow, NetEndpoints

    reqs = W.uneven_instances(seed=21, n_instances=24).requests()
    dims = Dims(6, 4, 3)
    reqs.append(IsolatedRouteRequest(Grid.filled(dims, 2), [NetEndpoints("a", 1, 70, [5, 70], [70])],
                                     [IsolatedRouteWindow(0, 0, 5, 3)], [3] * 5, [4] * 3, [None, 9],
                                     np.arange(len(dims) * 4, dtype=np.uint32)))
    reqs.append(IsolatedRouteRequest(Grid.filled(Dims(1, 1, 1), 1), [], [], [], [], []))

    def dump(rq):
        g = rq.grid.contents
        e = rq.edges
        out = [g.w, g.h, g.layers, g.cost, g.board_constraint, g.via_forbidden, rq.n_nets, e.n_x_edge_costs,
               e.n_y_edge_costs, e.n_via_edge_costs, e.directed_in_costs]
        for ptr, cnt, typ in ((e.x_edge_costs, e.n_x_edge_costs, C.c_uint32), (e.y_edge_costs, e.n_y_edge_costs, C.c_uint32),
                              (e.via_edge_costs, e.n_via_edge_costs, C.c_uint32), (e.via_allowed, e.n_via_edge_costs, C.c_uint8)):
            p = C.cast(ptr, C.POINTER(typ))
            out.append(tuple(p[j] for j in range(cnt)))
        nets = C.cast(rq.nets, C.POINTER(api._Net))
        wins = C.cast(rq.windows, C.POINTER(api._Window))
        for i in range(rq.n_nets):
            nt = nets[i]
            pp = C.cast(nt.passable_pads, C.POINTER(C.c_uint32))
            vp = C.cast(nt.via_passable_pads, C.POINTER(C.c_uint32))
            out += [nt.src, nt.dst, tuple(pp[j] for j in range(nt.n_passable_pads)),
                    tuple(vp[j] for j in range(nt.n_via_passable_pads)), (wins[i].x0, wins[i].y0, wins[i].x1, wins[i].y1)]
        return out

    m = api._Marshal()
    fast = api._marshal_requests(m, reqs)
    m2 = api._Marshal()
    for k, r in enumerate(reqs):
        assert dump(fast[k]) == dump(api.Engine._request(None, m2, r)), k
