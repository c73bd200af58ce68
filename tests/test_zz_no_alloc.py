"""The no-allocation entry point, mrc_route_isolated_batch_noalloc.

Some callers cannot call cudaMalloc: a long-running router process whose own
allocator already holds nearly all of the GPU's memory, or a caller on a path
where cudaMalloc/cudaFree (which may synchronise the whole device) are not
allowed.  For them the library keeps one static device array and carves every
scratch buffer of a window solve from it.  These tests call that entry point
through the C ABI and require its paths and search costs to equal, bit for
bit, those of the allocating entry point (mrc_route_isolated_batch without the
full-board retry) and those of the CPU oracle on the same requests, on two
calls in a row, and require a request that does not fit the array to be
refused with a clear error.
"""
import ctypes as C

import numpy as np
import pytest

import mrcuda
from mrcuda import api
from mrcuda import workloads as W

pytestmark = pytest.mark.gpu


def _noalloc(lib, req):
    lib.mrc_route_isolated_batch_noalloc.restype = C.c_int
    lib.mrc_route_isolated_batch_noalloc.argtypes = [C.POINTER(api._Request), C.c_void_p, C.c_void_p, C.c_void_p,
                                                     C.c_void_p, C.c_uint64]
    m = api._Marshal()
    r = api._Request(C.pointer(m.grid(req.grid)), m.nets(req.nets), len(req.nets), m.windows(req.windows),
                     m.edges(req.x_edge_costs, req.y_edge_costs, req.via_edge_costs, req.directed_in_costs))
    n = len(req.nets)
    costs = np.zeros(max(n, 1), dtype=np.uint32)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    cap = sum(w.cells(req.grid.dims) for w in req.windows)
    cells = np.zeros(max(cap, 1), dtype=np.uint32)
    st = lib.mrc_route_isolated_batch_noalloc(C.byref(r), None, costs.ctypes.data, offsets.ctypes.data,
                                              cells.ctypes.data, cap)
    if st != 0:
        raise api._ERRORS.get(st, api.RouterError)(lib.mrc_last_error(None).decode())
    paths = [cells[offsets[i]:offsets[i + 1]].tolist() if offsets[i + 1] > offsets[i] else None for i in range(n)]
    return paths, [int(c) for c in costs[:n]]


def test_noalloc_entry_point_matches_the_allocating_one_on_two_calls_in_a_row(oracle):
    lib = mrcuda.load_library()
    eng = mrcuda.Engine(0)
    try:
        # two different boards back to back: the second call finds the first
        # call's contents in the shared array and must not be affected by them
        for wl in (W.plain_board(), W.scaled(W.congestion_board(), 8)):
            req = wl.request()
            ref = eng.route_isolated_batch(req, retry_full=False)
            got_paths, got_costs = _noalloc(lib, req)
            exp_paths, exp_costs = oracle.isolated_batch(req, retry_full=False, mode="astar")
            assert got_paths == ref.paths == exp_paths
            assert got_costs == ref.search_costs == exp_costs
            assert all(p is not None for p in got_paths)
    finally:
        eng.close()


def test_noalloc_entry_point_refuses_a_request_beyond_its_scratch():
    lib = mrcuda.load_library()
    req = W.congestion_board().request()  # 43 M window cells: far beyond 64 MiB of labels
    with pytest.raises(mrcuda.LimitExceeded, match="MRC_NOALLOC_SCRATCH_BYTES"):
        _noalloc(lib, req)
