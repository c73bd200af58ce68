"""ctypes wrapper around the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the oracle.  The product (the mr_cuda
library and its Python binding) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from typing import List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.join(os.path.dirname(_HERE), "metal-route_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from mrcuda.types import (  # noqa: E402
    COST_MAX,
    Grid,
    IsolatedRouteRequest,
    IsolatedRouteWindow,
    NetEndpoints,
)

LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build(force: bool = False) -> str:
    """Compile liboracle.so from oracle.c (gcc; a few seconds)."""
    src = os.path.join(_HERE, "oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
        os.path.getmtime(src), os.path.getmtime(os.path.join(_HERE, "oracle.h"))
    ):
        subprocess.check_call(["make", "-s", "-B", "liboracle.so"], cwd=_HERE)
    return LIB_PATH


class _Grid(C.Structure):
    _fields_ = [
        ("w", C.c_uint32),
        ("h", C.c_uint32),
        ("layers", C.c_uint32),
        ("cost", C.c_void_p),
        ("board", C.c_void_p),
        ("via_forbidden", C.c_void_p),
    ]


class _Edges(C.Structure):
    _fields_ = [
        ("x_edge", C.c_void_p),
        ("y_edge", C.c_void_p),
        ("via_edge", C.c_void_p),
        ("via_allowed", C.c_void_p),
        ("directed", C.c_void_p),
    ]


class _Net(C.Structure):
    _fields_ = [
        ("src", C.c_uint32),
        ("dst", C.c_uint32),
        ("pads", C.c_void_p),
        ("n_pads", C.c_uint32),
        ("via_pads", C.c_void_p),
        ("n_via_pads", C.c_uint32),
    ]


class _Window(C.Structure):
    _fields_ = [("x0", C.c_uint32), ("y0", C.c_uint32), ("x1", C.c_uint32), ("y1", C.c_uint32)]


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


class Oracle:
    def __init__(self):
        self.lib = C.CDLL(build())
        L = self.lib
        L.orc_edge_cost.restype = C.c_uint32
        L.orc_edge_cost.argtypes = [C.c_double]
        L.orc_axis_edge_costs.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
        L.orc_net_window.restype = _Window
        L.orc_net_window.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(_Net)]
        L.orc_isolated_astar.restype = C.c_uint32
        L.orc_isolated_astar.argtypes = [
            C.POINTER(_Grid), C.POINTER(_Edges), C.POINTER(_Net), _Window, C.c_int, C.c_uint32,
            C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]
        L.orc_isolated_field.argtypes = [
            C.POINTER(_Grid), C.POINTER(_Edges), C.POINTER(_Net), _Window, C.c_void_p, C.c_void_p]
        L.orc_isolated_path_from_labels.restype = C.c_uint32
        L.orc_isolated_path_from_labels.argtypes = [
            C.POINTER(_Grid), C.POINTER(_Edges), C.POINTER(_Net), _Window, C.c_void_p, C.c_void_p,
            C.c_void_p, C.c_uint32]
        L.orc_isolated_batch.restype = C.c_int
        L.orc_isolated_batch.argtypes = [
            C.POINTER(_Grid), C.POINTER(_Edges), C.c_void_p, C.c_uint32, C.c_void_p, C.c_int, C.c_int,
            C.c_int, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
        L.orc_lee_route_one.restype = C.c_uint32
        L.orc_lee_route_one.argtypes = [C.POINTER(_Grid), C.POINTER(_Net), C.c_void_p, C.c_uint32,
                                        C.POINTER(C.c_uint32)]
        L.orc_bfs_distance_field.argtypes = [C.POINTER(_Grid), C.c_uint32, C.c_void_p]
        L.orc_sweep_distance_field.argtypes = [C.POINTER(_Grid), C.c_uint32, C.c_void_p]
        L.orc_path_from_field.restype = C.c_uint32
        L.orc_path_from_field.argtypes = [C.POINTER(_Grid), C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                          C.c_uint32]
        L.orc_provider_path_is_valid.restype = C.c_int
        L.orc_provider_path_is_valid.argtypes = [C.POINTER(_Grid), C.c_void_p, C.POINTER(_Net), C.c_void_p,
                                                 C.c_uint32]

    # -- marshalling ---------------------------------------------------------
    @staticmethod
    def _grid(g: Grid):
        keep = [g.cost, g.board_constraint, g.via_forbidden]
        s = _Grid(g.dims.w, g.dims.h, g.dims.layers, _ptr(g.cost), _ptr(g.board_constraint),
                  _ptr(g.via_forbidden))
        return s, keep

    @staticmethod
    def _edges(x, y, vias, directed=None):
        xe = np.ascontiguousarray(np.asarray(x, dtype=np.uint32).reshape(-1))
        ye = np.ascontiguousarray(np.asarray(y, dtype=np.uint32).reshape(-1))
        ve = np.array([0 if v is None else int(v) for v in vias] or [0], dtype=np.uint32)
        va = np.array([0 if v is None else 1 for v in vias] or [0], dtype=np.uint8)
        d = None if directed is None else np.ascontiguousarray(directed, dtype=np.uint32).reshape(-1)
        keep = [xe, ye, ve, va, d]
        return _Edges(_ptr(xe) if xe.size else _ptr(ve), _ptr(ye) if ye.size else _ptr(ve), _ptr(ve), _ptr(va),
                      _ptr(d)), keep

    @staticmethod
    def _net(n: NetEndpoints):
        pads = np.array(list(n.passable_pads) or [0], dtype=np.uint32)
        vpads = np.array(list(n.via_passable_pads) or [0], dtype=np.uint32)
        s = _Net(n.src, n.dst, _ptr(pads), len(n.passable_pads), _ptr(vpads), len(n.via_passable_pads))
        return s, [pads, vpads]

    # -- API -----------------------------------------------------------------
    def edge_cost(self, length: float) -> int:
        return int(self.lib.orc_edge_cost(float(length)))

    def axis_edge_costs(self, lines: Sequence[float], count: int) -> List[int]:
        arr = np.array(list(lines) or [0.0], dtype=np.float64)
        out = np.zeros(max(count - 1, 1), dtype=np.uint32)
        self.lib.orc_axis_edge_costs(_ptr(arr), len(lines), count, _ptr(out))
        return [int(v) for v in out[: max(count - 1, 0)]]

    def net_window(self, dims, net: NetEndpoints) -> IsolatedRouteWindow:
        s, keep = self._net(net)
        w = self.lib.orc_net_window(dims.w, dims.h, dims.layers, C.byref(s))
        return IsolatedRouteWindow(w.x0, w.y0, w.x1, w.y1)

    def isolated_astar(self, grid: Grid, x, y, vias, net: NetEndpoints, window: IsolatedRouteWindow,
                       use_heuristic: bool = True, via_h_cost: Optional[int] = None, directed=None
                       ) -> Optional[Tuple[List[int], int]]:
        """One `route_legal_once` alone-path search (A*).  The heuristic is
        disabled automatically when the grid holds a zero cost, as the router
        does (negotiated.rs:1501)."""
        gs, k1 = self._grid(grid)
        es, k2 = self._edges(x, y, vias, directed)
        ns, k3 = self._net(net)
        if via_h_cost is None:
            allowed = [int(v) for v in vias if v is not None]
            via_h_cost = min(allowed) if allowed else 0
        use_h = bool(use_heuristic) and directed is None and not bool((grid.cost == 0).any())
        n = len(grid.dims)
        out = np.zeros(n + 1, dtype=np.uint32)
        cost = C.c_uint32(0)
        ln = self.lib.orc_isolated_astar(C.byref(gs), C.byref(es), C.byref(ns), _Window(*_win(window)),
                                         int(use_h), int(via_h_cost), _ptr(out), n + 1, C.byref(cost))
        if ln == 0:
            return None
        return [int(c) for c in out[:ln]], int(cost.value)

    def isolated_field(self, grid: Grid, x, y, vias, net: NetEndpoints, window: IsolatedRouteWindow,
                       directed=None) -> Tuple[np.ndarray, np.ndarray]:
        gs, k1 = self._grid(grid)
        es, k2 = self._edges(x, y, vias, directed)
        ns, k3 = self._net(net)
        n = len(grid.dims)
        dist = np.zeros(n, dtype=np.uint32)
        hops = np.zeros(n, dtype=np.uint32)
        self.lib.orc_isolated_field(C.byref(gs), C.byref(es), C.byref(ns), _Window(*_win(window)), _ptr(dist),
                                    _ptr(hops))
        return dist, hops

    def isolated_path_from_labels(self, grid: Grid, x, y, vias, net, window, dist, hops, directed=None):
        gs, k1 = self._grid(grid)
        es, k2 = self._edges(x, y, vias, directed)
        ns, k3 = self._net(net)
        n = len(grid.dims)
        out = np.zeros(n + 1, dtype=np.uint32)
        d = np.ascontiguousarray(dist, dtype=np.uint32)
        h = np.ascontiguousarray(hops, dtype=np.uint32)
        ln = self.lib.orc_isolated_path_from_labels(C.byref(gs), C.byref(es), C.byref(ns), _Window(*_win(window)),
                                                    _ptr(d), _ptr(h), _ptr(out), n + 1)
        return [int(c) for c in out[:ln]] if ln else None

    def isolated_batch(self, req: IsolatedRouteRequest, retry_full: bool = True, mode: str = "astar",
                       threads: int = 0, via_h_cost: Optional[int] = None):
        """Whole batch with the provider's window-then-full-retry rule.  Returns
        (paths, costs): paths[i] is None when unreachable after the retry."""
        grid = req.grid
        gs, k1 = self._grid(grid)
        es, k2 = self._edges(req.x_edge_costs, req.y_edge_costs, req.via_edge_costs, req.directed_in_costs)
        nets = (_Net * max(len(req.nets), 1))()
        keep = []
        for i, n in enumerate(req.nets):
            s, k = self._net(n)
            nets[i] = s
            keep.append(k)
        wins = (_Window * max(len(req.windows), 1))()
        for i, w in enumerate(req.windows):
            wins[i] = _Window(*_win(w))
        if via_h_cost is None:
            allowed = [int(v) for v in req.via_edge_costs if v is not None]
            via_h_cost = min(allowed) if allowed else 0
        use_h = req.directed_in_costs is None and not bool((grid.cost == 0).any())
        nn = len(req.nets)
        cap = sum(w.cells(grid.dims) for w in req.windows) + nn * len(grid.dims) + 1
        offsets = np.zeros(nn + 1, dtype=np.uint64)
        cells = np.zeros(cap, dtype=np.uint32)
        costs = np.zeros(max(nn, 1), dtype=np.uint32)
        rc = self.lib.orc_isolated_batch(C.byref(gs), C.byref(es), C.cast(nets, C.c_void_p), nn,
                                         C.cast(wins, C.c_void_p), int(retry_full), 0 if mode == "astar" else 1,
                                         int(use_h), int(via_h_cost), int(threads), _ptr(offsets), _ptr(cells),
                                         cap, _ptr(costs))
        assert rc == 0
        paths = []
        for i in range(nn):
            a, b = int(offsets[i]), int(offsets[i + 1])
            paths.append([int(c) for c in cells[a:b]] if b > a else None)
        return paths, [int(c) for c in costs[:nn]]

    def lee_route_one(self, grid: Grid, net: NetEndpoints):
        gs, k1 = self._grid(grid)
        ns, k2 = self._net(net)
        n = len(grid.dims)
        out = np.zeros(n + 1, dtype=np.uint32)
        cost = C.c_uint32(0)
        ln = self.lib.orc_lee_route_one(C.byref(gs), C.byref(ns), _ptr(out), n + 1, C.byref(cost))
        return ([int(c) for c in out[:ln]], int(cost.value)) if ln else None

    def bfs_distance_field(self, grid: Grid, src: int) -> np.ndarray:
        gs, k = self._grid(grid)
        out = np.zeros(max(len(grid.dims), 1), dtype=np.uint32)
        self.lib.orc_bfs_distance_field(C.byref(gs), src, _ptr(out))
        return out[: len(grid.dims)]

    def sweep_distance_field(self, grid: Grid, src: int) -> np.ndarray:
        gs, k = self._grid(grid)
        out = np.zeros(max(len(grid.dims), 1), dtype=np.uint32)
        self.lib.orc_sweep_distance_field(C.byref(gs), src, _ptr(out))
        return out[: len(grid.dims)]

    def path_from_field(self, grid: Grid, dist: np.ndarray, src: int, dst: int):
        gs, k = self._grid(grid)
        n = len(grid.dims)
        d = np.ascontiguousarray(dist, dtype=np.uint32)
        if d.size != n:
            return None
        out = np.zeros(n + 1, dtype=np.uint32)
        ln = self.lib.orc_path_from_field(C.byref(gs), _ptr(d), src, dst, _ptr(out), n + 1)
        return [int(c) for c in out[:ln]] if ln else None

    def provider_path_is_valid(self, grid: Grid, via_allowed: Sequence[bool], net: NetEndpoints,
                               path: Sequence[int]) -> bool:
        gs, k1 = self._grid(grid)
        ns, k2 = self._net(net)
        va = np.array([1 if v else 0 for v in via_allowed] or [0], dtype=np.uint8)
        p = np.array(list(path) or [0], dtype=np.uint32)
        return bool(self.lib.orc_provider_path_is_valid(C.byref(gs), _ptr(va), C.byref(ns), _ptr(p), len(path)))


def _win(w: IsolatedRouteWindow):
    return (w.x0, w.y0, w.x1, w.y1)


_INSTANCE: Optional[Oracle] = None


def get() -> Oracle:
    global _INSTANCE
    if _INSTANCE is None:
        _INSTANCE = Oracle()
    return _INSTANCE


__all__ = ["Oracle", "get", "build", "COST_MAX"]
