"""ctypes binding of libmr_cuda.so (include/mr_cuda.h).

This module mirrors the reference's provider seam so that callers read like
metalroute's own code:

* ``CudaIsolatedProvider.route_isolated_batch(request)`` — the
  ``IsolatedRouteProvider`` trait (crates/mr-cpu/src/negotiated.rs:554-560):
  aligned ``Optional[List[CellIdx]]`` per net, all-or-error.
* ``Engine.route_isolated_batch`` — ``metal_route_isolated_batch`` plus the
  adapter's full-board retry (crates/mr-metal/src/lib.rs:414-558,
  crates/mr-cli/src/lib.rs:549-607), returning paths and search costs.
* ``Engine.route_lee`` / ``Engine.distance_fields`` — the ``Router`` contract
  of LeeRouter/MetalRouter and the batched complete fields.

There is no CPU fallback anywhere in here: if the CUDA library or device is
unavailable every call raises ``BackendUnavailable`` and the caller decides.
"""
from __future__ import annotations

import array
import ctypes as C
import os
import threading
import weakref
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from .types import (
    COST_MAX,
    Grid,
    connection_group_ids,
    IsolatedRouteRequest,
    IsolatedRouteWindow,
    NetEndpoints,
)

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmr_cuda.so")

MRC_OK = 0
MRC_FLAG_RETRY_FULL = 0x1
MRC_FLAG_KEEP_FIELDS = 0x2
MRC_FLAG_NO_WAIT = 0x4
MRC_FLAG_TIME_KERNELS = 0x8
NO_PATH = 0xFFFFFFFF


class RouterError(Exception):
    """Base of the errors a routing call may raise (core/src/lib.rs:698-708)."""

    status = -1


class InvalidArgument(RouterError):
    status = 1


class MalformedGrid(RouterError):
    status = 2


class InvalidEndpoint(RouterError):
    status = 3


class BackendUnavailable(RouterError):
    status = 4


class Busy(BackendUnavailable):
    status = 5


class IterationLimit(BackendUnavailable):
    status = 6


class OutOfMemory(BackendUnavailable):
    status = 7


class LimitExceeded(BackendUnavailable):
    status = 8


_ERRORS = {c.status: c for c in (InvalidArgument, MalformedGrid, InvalidEndpoint, BackendUnavailable, Busy,
                                 IterationLimit, OutOfMemory, LimitExceeded)}


class _Grid(C.Structure):
    _fields_ = [("w", C.c_uint32), ("h", C.c_uint32), ("layers", C.c_uint32), ("cost", C.c_void_p),
                ("board_constraint", C.c_void_p), ("via_forbidden", C.c_void_p)]


class _Net(C.Structure):
    _fields_ = [("src", C.c_uint32), ("dst", C.c_uint32), ("passable_pads", C.c_void_p),
                ("n_passable_pads", C.c_uint32), ("via_passable_pads", C.c_void_p),
                ("n_via_passable_pads", C.c_uint32)]


class _Window(C.Structure):
    _fields_ = [("x0", C.c_uint32), ("y0", C.c_uint32), ("x1", C.c_uint32), ("y1", C.c_uint32)]


class _Edges(C.Structure):
    _fields_ = [("x_edge_costs", C.c_void_p), ("n_x_edge_costs", C.c_uint32), ("y_edge_costs", C.c_void_p),
                ("n_y_edge_costs", C.c_uint32), ("via_edge_costs", C.c_void_p), ("via_allowed", C.c_void_p),
                ("n_via_edge_costs", C.c_uint32), ("directed_in_costs", C.c_void_p)]


class _Request(C.Structure):
    _fields_ = [("grid", C.POINTER(_Grid)), ("nets", C.c_void_p), ("n_nets", C.c_uint32),
                ("windows", C.c_void_p), ("edges", _Edges)]


class _NegParams(C.Structure):
    _fields_ = [("present_weight", C.c_uint32), ("history_step", C.c_uint32)]


class _RoundStats(C.Structure):
    _fields_ = [("round", C.c_uint32), ("pfac", C.c_uint32), ("dirty", C.c_uint32), ("routed", C.c_uint32),
                ("retried", C.c_uint32), ("next_dirty", C.c_uint32), ("overused_edges", C.c_uint64),
                ("window_cells", C.c_uint64), ("path_cells", C.c_uint64), ("round_ms", C.c_float)]


class _ServerParams(C.Structure):
    _fields_ = [("hbm_fraction", C.c_float), ("slots", C.c_uint32), ("max_batch_requests", C.c_uint32),
                ("max_batch_cells", C.c_uint64), ("max_layers", C.c_uint32), ("merge_ratio", C.c_uint32)]


class _RequestInfo(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("run_ms", C.c_double), ("total_ms", C.c_double),
                ("batch_requests", C.c_uint32), ("status", C.c_uint32), ("batch_id", C.c_uint64)]


_lib = None
_lib_lock = threading.Lock()


def load_library(path: str = _LIB_PATH) -> C.CDLL:
    """Load libmr_cuda.so; raises BackendUnavailable when it is missing."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise BackendUnavailable(f"CUDA engine library not built: {path}")
        L = C.CDLL(path)
        vp, u32, u64p, u32p = C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)
        sig = {
            "mrc_abi_version": (u32, []),
            "mrc_last_error": (C.c_char_p, [vp]),
            "mrc_context_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
            "mrc_context_destroy": (None, [vp]),
            "mrc_host_alloc": (C.c_int, [vp, C.c_size_t, C.POINTER(vp)]),
            "mrc_host_free": (None, [vp]),
            "mrc_upload_stats": (C.c_int, [vp, u64p, u64p]),
            "mrc_route_isolated_batch": (C.c_int, [vp, C.POINTER(_Request), u32, C.POINTER(vp)]),
            "mrc_route_isolated_plain": (C.c_int, [vp, C.POINTER(_Request), u32, C.POINTER(vp)]),
            "mrc_route_lee": (C.c_int, [vp, C.POINTER(_Grid), vp, u32, C.POINTER(vp)]),
            "mrc_distance_fields": (C.c_int, [vp, C.POINTER(_Grid), vp, u32, vp]),
            "mrc_result_count": (u32, [vp]),
            "mrc_result_path_offsets": (u64p, [vp]),
            "mrc_result_path_cells": (u32p, [vp]),
            "mrc_result_search_costs": (u32p, [vp]),
            "mrc_result_field_offsets": (u64p, [vp]),
            "mrc_result_fields": (u32p, [vp]),
            "mrc_result_field_windows": (C.POINTER(_Window), [vp]),
            "mrc_result_retried": (u32, [vp]),
            "mrc_result_free": (None, [vp]),
            "mrc_board_create": (C.c_int, [vp, C.POINTER(_Grid), C.POINTER(_Edges), C.POINTER(vp)]),
            "mrc_board_destroy": (None, [vp]),
            "mrc_batch_create": (C.c_int, [vp, vp, vp, u32, vp, u32, C.POINTER(vp)]),
            "mrc_batch_launch": (C.c_int, [vp, vp, vp]),
            "mrc_batch_finish": (C.c_int, [vp, vp, C.POINTER(vp)]),
            "mrc_batch_kernel_launches": (u32, [vp]),
            "mrc_batch_window_cells": (C.c_uint64, [vp]),
            "mrc_batch_relax_ms": (C.c_float, [vp]),
            "mrc_batch_stats": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
            "mrc_batch_set_config": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32]),
            "mrc_batch_autotune": (C.c_int, [vp, vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_float)]),
            "mrc_batch_destroy": (None, [vp]),
            "mrc_batch_set_schedule": (C.c_int, [vp, vp, C.c_uint32]),
            "mrc_context_set_schedule": (C.c_int, [vp, C.c_uint32]),
            "mrc_batch_config": (C.c_int, [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                           C.POINTER(C.c_uint32)]),
            "mrc_net_windows": (C.c_int, [u32, u32, u32, vp, u32, vp]),
            "mrc_route_instances": (C.c_int, [vp, vp, u32, u32, C.POINTER(vp)]),
            "mrc_batch_create_multi": (C.c_int, [vp, vp, u32, vp, vp, u32, vp, u32, C.POINTER(vp)]),
            "mrc_batch_capture_graph": (C.c_int, [vp, vp]),
            "mrc_negotiation_create": (C.c_int, [vp, C.POINTER(_Request), C.POINTER(_NegParams), C.POINTER(vp)]),
            "mrc_negotiation_round": (C.c_int, [vp, vp, C.POINTER(_RoundStats)]),
            "mrc_negotiation_paths": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u64p), C.POINTER(u32p)]),
            "mrc_negotiation_read": (C.c_int, [vp, vp, vp, vp, vp]),
            "mrc_negotiation_dirty": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u32p)]),
            "mrc_negotiation_destroy": (None, [vp]),
            "mrc_negotiation_set_groups": (C.c_int, [vp, vp, vp]),
            "mrc_negotiation_set_clearance": (C.c_int, [vp, vp, u32, u32, u32]),
            "mrc_negotiation_read_halo": (C.c_int, [vp, vp, vp]),
            "mrc_negotiation_create_shard": (C.c_int, [vp, C.POINTER(_Request), C.POINTER(_NegParams), vp,
                                                       C.POINTER(vp)]),
            "mrc_negotiation_ripup": (C.c_int, [vp, vp]),
            "mrc_negotiation_route": (C.c_int, [vp, vp, C.POINTER(_RoundStats)]),
            "mrc_negotiation_settle": (C.c_int, [vp, vp, C.POINTER(_RoundStats)]),
            "mrc_negotiation_buffers": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(C.c_uint64)]),
            "mrc_server_create": (C.c_int, [vp, C.POINTER(_ServerParams), C.POINTER(vp)]),
            "mrc_server_submit": (C.c_int, [vp, C.POINTER(_Request), u32, C.POINTER(C.c_uint64)]),
            "mrc_server_submit_resident": (C.c_int, [vp, vp, vp, u32, vp, u32, C.POINTER(C.c_uint64)]),
            "mrc_server_wait": (C.c_int, [vp, C.c_uint64, u32, C.POINTER(vp), C.POINTER(_RequestInfo)]),
            "mrc_server_stats": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
            "mrc_server_destroy": (None, [vp]),
            "mrc_selftest_wait_timeout": (C.c_int, [vp, u32, C.POINTER(u32), C.POINTER(C.c_float)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
        return L


def exported_symbols() -> List[str]:
    """Names declared in include/mr_cuda.h that the binding resolves."""
    L = load_library()
    return [n for n in dir(L) if n.startswith("mrc_")]


def _u32(a) -> np.ndarray:
    if type(a) is np.ndarray and a.dtype == np.uint32 and a.ndim == 1 and a.flags.c_contiguous:
        return a
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32).reshape(-1))


_VIA_CACHE = {}


def _via_arrays(vias):
    """(prices u32, allowed u8) for an Option<u32> via vector, shared between
    requests with the same vector (arrays are never written)."""
    key = tuple(vias)
    hit = _VIA_CACHE.get(key)
    if hit is None:
        hit = (np.array([0 if v is None else int(v) for v in key], dtype=np.uint32),
               np.array([0 if v is None else 1 for v in key], dtype=np.uint8))
        if len(_VIA_CACHE) < 4096:
            _VIA_CACHE[key] = hit
    return hit


class _Marshal:
    """Keeps every numpy buffer alive for the duration of one C call."""

    def __init__(self):
        self.keep = []

    def arr(self, a: Optional[np.ndarray]):
        if a is None:
            return None
        self.keep.append(a)
        try:
            return C.addressof(C.c_char.from_buffer(a))
        except (TypeError, ValueError):  # read-only or empty buffer
            return a.ctypes.data

    def grid(self, g: Grid) -> _Grid:
        s = _Grid(g.dims.w, g.dims.h, g.dims.layers, self.arr(g.cost), self.arr(g.board_constraint),
                  self.arr(g.via_forbidden))
        self.keep.append(s)
        return s

    def nets(self, nets: Sequence[NetEndpoints]):
        arr = (_Net * max(len(nets), 1))()
        for i, n in enumerate(nets):
            pads = _u32(n.passable_pads) if len(n.passable_pads) else None
            vpads = _u32(n.via_passable_pads) if len(n.via_passable_pads) else None
            arr[i] = _Net(n.src, n.dst, self.arr(pads), len(n.passable_pads), self.arr(vpads),
                          len(n.via_passable_pads))
        self.keep.append(arr)
        return C.cast(arr, C.c_void_p)

    def windows(self, wins: Optional[Sequence[IsolatedRouteWindow]]):
        if wins is None:
            return None
        arr = (_Window * max(len(wins), 1))()
        for i, w in enumerate(wins):
            arr[i] = _Window(w.x0, w.y0, w.x1, w.y1)
        self.keep.append(arr)
        return C.cast(arr, C.c_void_p)

    def edges(self, x, y, vias, directed=None) -> _Edges:
        xe, ye = _u32(x), _u32(y)
        ve, va = _via_arrays(vias)
        d = None if directed is None else _u32(directed)
        e = _Edges(self.arr(xe) if xe.size else None, xe.size, self.arr(ye) if ye.size else None, ye.size,
                   self.arr(ve) if ve.size else None, self.arr(va) if va.size else None, ve.size, self.arr(d))
        self.keep.append(e)
        return e


def _addr(a: Optional[np.ndarray]) -> int:
    if a is None or a.size == 0:
        return 0
    try:
        return C.addressof(C.c_char.from_buffer(a))
    except (TypeError, ValueError):  # read-only buffer
        return a.__array_interface__["data"][0]


def _flat_u32(lists) -> np.ndarray:
    """Concatenation of many short integer sequences as one u32 array."""
    a = array.array("I")
    for p in lists:
        a.extend(p)
    return np.frombuffer(a, dtype=np.uint32) if len(a) else np.zeros(0, np.uint32)


def _marshal_requests(m: _Marshal, requests: Sequence[IsolatedRouteRequest]):
    """An array of C requests for many instances at once.  The structs are
    written as 64-bit words from numpy columns (the layouts of _Grid, _Net,
    _Window, _Edges and _Request on a 64-bit ABI), so the per-request Python work
    is collecting a few buffer addresses."""
    n = len(requests)
    nets_all = [nt for rq in requests for nt in rq.nets]
    nn = len(nets_all)
    reqs = (_Request * max(n, 1))()
    grids = np.zeros((max(n, 1), C.sizeof(_Grid) // 8), dtype=np.uint64)
    nets = np.zeros((max(nn, 1), C.sizeof(_Net) // 8), dtype=np.uint64)
    wins = np.zeros((max(nn, 1), 4), dtype=np.uint32)
    # pads of every net in one array
    pad_lists = [nt.passable_pads for nt in nets_all] + [nt.via_passable_pads for nt in nets_all]
    lens = np.fromiter(map(len, pad_lists), dtype=np.int64, count=len(pad_lists))
    pads = _flat_u32(pad_lists)
    starts = np.cumsum(lens) - lens
    # the caller's arrays stay referenced by the requests themselves
    m.keep += [requests, reqs, grids, nets, wins, pads]
    pbase = _addr(pads)
    if nn:
        nets[:, 0] = (np.fromiter((nt.src for nt in nets_all), np.uint64, nn)
                      | (np.fromiter((nt.dst for nt in nets_all), np.uint64, nn) << np.uint64(32)))
        lp, lv = lens[:nn], lens[nn:]
        nets[:, 1] = np.where(lp > 0, pbase + 4 * starts[:nn], 0).astype(np.uint64)
        nets[:, 2] = lp.astype(np.uint64)
        nets[:, 3] = np.where(lv > 0, pbase + 4 * starts[nn:], 0).astype(np.uint64)
        nets[:, 4] = lv.astype(np.uint64)
        wins.reshape(-1)[:] = np.fromiter((c for rq in requests for w in rq.windows for c in (w.x0, w.y0, w.x1, w.y1)),
                                          np.uint32, 4 * nn)
    if not n:
        return reqs
    if any(len(rq.windows) != len(rq.nets) for rq in requests):
        raise BackendUnavailable("isolated request windows are not net-aligned")
    rw = np.frombuffer(reqs, dtype=np.uint64).reshape(n, C.sizeof(_Request) // 8)
    gbase, nbase, wbase = _addr(grids), _addr(nets), _addr(wins)
    # the small edge vectors of every request in one array each
    xs = [_u32(rq.x_edge_costs) for rq in requests]
    ys = [_u32(rq.y_edge_costs) for rq in requests]
    vv = [_via_arrays(rq.via_edge_costs) for rq in requests]
    ds = [None if rq.directed_in_costs is None else _u32(rq.directed_in_costs) for rq in requests]
    xa, ya = np.concatenate(xs), np.concatenate(ys)
    vea, vaa = np.concatenate([v[0] for v in vv]), np.concatenate([v[1] for v in vv])
    m.keep += [xa, ya, vea, vaa, ds]
    kn = np.fromiter((len(rq.nets) for rq in requests), np.int64, n)
    nx = np.fromiter((a.size for a in xs), np.int64, n)
    ny = np.fromiter((a.size for a in ys), np.int64, n)
    nv = np.fromiter((v[0].size for v in vv), np.int64, n)
    first, xo, yo, vo = (np.cumsum(c) - c for c in (kn, nx, ny, nv))
    gl = [rq.grid for rq in requests]
    grids[:n, 0] = np.fromiter((g.dims.w | (g.dims.h << 32) for g in gl), np.uint64, n)
    grids[:n, 1] = np.fromiter((g.dims.layers for g in gl), np.uint64, n)
    grids[:n, 2] = np.fromiter((_addr(g.cost) for g in gl), np.uint64, n)
    grids[:n, 3] = np.fromiter((_addr(g.board_constraint) for g in gl), np.uint64, n)
    grids[:n, 4] = np.fromiter((_addr(g.via_forbidden) for g in gl), np.uint64, n)
    at = lambda cnt, base, off, size: np.where(cnt > 0, base + size * off, 0).astype(np.uint64)
    rw[:, 0] = gbase + C.sizeof(_Grid) * np.arange(n, dtype=np.uint64)
    rw[:, 1] = at(kn, nbase, first, C.sizeof(_Net))
    rw[:, 2] = kn
    rw[:, 3] = at(kn, wbase, first, 16)
    rw[:, 4] = at(nx, _addr(xa), xo, 4)
    rw[:, 5] = nx
    rw[:, 6] = at(ny, _addr(ya), yo, 4)
    rw[:, 7] = ny
    rw[:, 8] = at(nv, _addr(vea), vo, 4)
    rw[:, 9] = at(nv, _addr(vaa), vo, 1)
    rw[:, 10] = nv
    rw[:, 11] = np.fromiter((_addr(d) for d in ds), np.uint64, n)
    return reqs


class IsolatedBatchResult:
    """Per-net outputs, aligned with the request's nets.

    The library hands the paths back in CSR form, kept here as numpy arrays:
    ``offsets`` (n + 1 u64), ``cells`` (u32 global CellIdx) and ``costs`` (n u32,
    0xFFFFFFFF = unreachable); net i's path is cells[offsets[i]:offsets[i+1]],
    empty when the net has none.  ``paths`` (the provider's
    Vec<Option<Vec<CellIdx>>>) and ``search_costs`` are the same data as Python
    lists, built on first use, so callers that work on the arrays never pay
    for per-path list objects."""

    def __init__(self, paths: Optional[List[Optional[List[int]]]] = None, search_costs: Optional[List[int]] = None,
                 fields: Optional[List[np.ndarray]] = None, field_windows: Optional[List[IsolatedRouteWindow]] = None,
                 retried: int = 0, *, offsets: Optional[np.ndarray] = None, cells: Optional[np.ndarray] = None,
                 costs: Optional[np.ndarray] = None):
        if offsets is None:
            paths = [] if paths is None else list(paths)
            search_costs = [] if search_costs is None else list(search_costs)
            lens = [len(p) if p else 0 for p in paths]
            offsets = np.zeros(len(paths) + 1, np.uint64)
            offsets[1:] = np.cumsum(lens, dtype=np.uint64)
            cells = np.array([c for p in paths if p for c in p], dtype=np.uint32)
            costs = np.array(search_costs, dtype=np.uint32)
        self.offsets = offsets
        self.cells = cells
        self.costs = costs
        self._paths = paths
        self._search_costs = search_costs
        self.fields = fields
        self.field_windows = field_windows
        self.retried = retried

    def __len__(self) -> int:
        return len(self.offsets) - 1

    @property
    def paths(self) -> List[Optional[List[int]]]:
        if self._paths is None:
            cl, ol = self.cells.tolist(), self.offsets.tolist()
            self._paths = [cl[ol[i]:ol[i + 1]] if ol[i + 1] > ol[i] else None for i in range(len(ol) - 1)]
        return self._paths

    @property
    def search_costs(self) -> List[int]:
        if self._search_costs is None:
            self._search_costs = self.costs.tolist()
        return self._search_costs

    def path(self, i: int) -> Optional[np.ndarray]:
        """Net i's path as a u32 view of ``cells`` (None when unreachable)."""
        a, b = int(self.offsets[i]), int(self.offsets[i + 1])
        return self.cells[a:b] if b > a else None

    def routed(self) -> int:
        return int(np.count_nonzero(np.diff(self.offsets)))

    def slice(self, start: int, stop: int) -> "IsolatedBatchResult":
        """Nets [start, stop) as a result of their own (views, offsets rebased)."""
        off = self.offsets[start:stop + 1]
        a, b = int(off[0]), int(off[-1])
        return IsolatedBatchResult(fields=self.fields[start:stop] if self.fields is not None else None,
                                   field_windows=(self.field_windows[start:stop]
                                                  if self.field_windows is not None else None),
                                   offsets=off - np.uint64(a), cells=self.cells[a:b], costs=self.costs[start:stop])


def _take_result(L, res, n: int, fields: bool, layers: int = 1) -> IsolatedBatchResult:
    try:
        cnt = L.mrc_result_count(res)
        assert cnt == n, (cnt, n)
        off = np.ctypeslib.as_array(L.mrc_result_path_offsets(res), shape=(n + 1,)).copy()
        total = int(off[-1])
        cells = (np.ctypeslib.as_array(L.mrc_result_path_cells(res), shape=(total,)).copy()
                 if total else np.zeros(0, np.uint32))
        costs = (np.ctypeslib.as_array(L.mrc_result_search_costs(res), shape=(n,)).copy()
                 if n else np.zeros(0, np.uint32))
        out = IsolatedBatchResult(retried=int(L.mrc_result_retried(res)), offsets=off, cells=cells, costs=costs)
        wp = L.mrc_result_field_windows(res) if fields else None
        if n and wp:
            wa = np.ctypeslib.as_array(C.cast(wp, C.POINTER(C.c_uint32)), shape=(n * 4,)).tolist()
            out.field_windows = [IsolatedRouteWindow(*wa[4 * i:4 * i + 4]) for i in range(n)]
        if fields:
            fo = np.ctypeslib.as_array(L.mrc_result_field_offsets(res), shape=(n + 1,)).copy()
            ft = int(fo[-1])
            fa = (np.ctypeslib.as_array(L.mrc_result_fields(res), shape=(ft,)).copy() if ft
                  else np.zeros(0, np.uint32))
            out.fields = [fa[fo[i]:fo[i + 1]] for i in range(n)]
        return out
    finally:
        L.mrc_result_free(res)


class Board:
    """A board resident in HBM (cost, masks, edge prices)."""

    def __init__(self, engine: "Engine", grid: Grid, x, y, vias, directed=None):
        self.engine = engine
        self.grid = grid
        m = _Marshal()
        h = C.c_void_p()
        engine._check(engine.lib.mrc_board_create(engine.ctx, C.byref(m.grid(grid)),
                                                  C.byref(m.edges(x, y, vias, directed)), C.byref(h)))
        self.handle = h
        engine._adopt(self)

    def close(self):
        if self.handle:
            self.engine.lib.mrc_board_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """A validated batch of nets staged against one resident Board, or against
    several (``board`` a sequence and ``net_board[i]`` the board of net i)."""

    def __init__(self, board, nets: Sequence[NetEndpoints],
                 windows: Optional[Sequence[IsolatedRouteWindow]] = None, retry_full: bool = True,
                 keep_fields: bool = False, time_kernels: bool = False, net_board: Optional[Sequence[int]] = None):
        boards = list(board) if isinstance(board, (list, tuple)) else [board]
        self.board = board
        self.boards = boards
        self.engine = boards[0].engine
        self.n = len(nets)
        self.keep_fields = keep_fields
        flags = ((MRC_FLAG_RETRY_FULL if retry_full else 0) | (MRC_FLAG_KEEP_FIELDS if keep_fields else 0)
                 | (MRC_FLAG_TIME_KERNELS if time_kernels else 0))
        m = _Marshal()
        h = C.c_void_p()
        e = self.engine
        if net_board is None and len(boards) == 1:
            e._check(e.lib.mrc_batch_create(e.ctx, boards[0].handle, m.nets(nets), len(nets), m.windows(windows),
                                            flags, C.byref(h)))
        else:
            if net_board is None or len(net_board) != len(nets):
                raise InvalidArgument("net_board must give one board index per net")
            handles = (C.c_void_p * len(boards))(*[b.handle for b in boards])
            m.keep.append(handles)
            nb = _u32(net_board)
            e._check(e.lib.mrc_batch_create_multi(e.ctx, C.cast(handles, C.c_void_p), len(boards), m.nets(nets),
                                                  m.arr(nb) if nb.size else None, len(nets), m.windows(windows),
                                                  flags, C.byref(h)))
        self.handle = h
        e._adopt(self)

    def capture_graph(self) -> None:
        """Record the launch sequence as a CUDA graph; later launches replay it."""
        e = self.engine
        e._check(e.lib.mrc_batch_capture_graph(e.ctx, self.handle))

    def launch(self, stream: int = 0) -> None:
        """Enqueue the solve on a cudaStream_t (an integer handle, 0 = the engine's stream)."""
        e = self.engine
        e._check(e.lib.mrc_batch_launch(e.ctx, self.handle, C.c_void_p(stream) if stream else None))

    def finish(self) -> IsolatedBatchResult:
        e = self.engine
        res = C.c_void_p()
        e._check(e.lib.mrc_batch_finish(e.ctx, self.handle, C.byref(res)))
        return _take_result(e.lib, res, self.n, self.keep_fields)

    @property
    def kernel_launches(self) -> int:
        return int(self.engine.lib.mrc_batch_kernel_launches(self.handle))

    def set_config(self, tile_h: int, threads: int) -> None:
        """Force the relax kernel's tile height and CTA width for this batch."""
        e = self.engine
        e._check(e.lib.mrc_batch_set_config(e.ctx, self.handle, int(tile_h), int(threads)))

    def set_schedule(self, schedule: int) -> None:
        """0 = bulk-synchronous rounds, 1 = asynchronous work queue (a CTA per
        tile, prices from the TMA-loaded price planes), 2 = the queue with a warp
        per tile, 3 = the CTA queue with prices formed per tile."""
        e = self.engine
        e._check(e.lib.mrc_batch_set_schedule(e.ctx, self.handle, int(schedule)))

    def config(self) -> dict:
        th, nt, sc = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self.engine._check(self.engine.lib.mrc_batch_config(self.handle, C.byref(th), C.byref(nt), C.byref(sc)))
        return {"tile_h": int(th.value), "threads": int(nt.value), "schedule": int(sc.value)}

    def autotune(self) -> dict:
        """Time every relax configuration (tile height, CTA width, schedule) on
        this batch and keep the fastest."""
        th, nt, ms = C.c_uint32(), C.c_uint32(), C.c_float()
        e = self.engine
        e._check(e.lib.mrc_batch_autotune(e.ctx, self.handle, C.byref(th), C.byref(nt), C.byref(ms)))
        return dict(self.config(), ms=float(ms.value))

    def stats(self) -> dict:
        """Work counters of the last launch: tile activations, in-tile sweeps
        (passes), rounds (tile rows relaxed, warp schedule) and the batch's
        tile count."""
        out = (C.c_uint64 * 4)()
        self.engine._check(self.engine.lib.mrc_batch_stats(self.handle, out))
        d = {"activations": int(out[0]), "sweeps": int(out[1]), "rounds": int(out[2]), "tiles": int(out[3])}
        if self.config()["schedule"] == 2:
            d["rows"] = d.pop("rounds")
        return d

    def relax_ms(self) -> float:
        """Device time of the relax kernel in the last launch (needs time_kernels)."""
        return float(self.engine.lib.mrc_batch_relax_ms(self.handle))

    @property
    def window_cells(self) -> int:
        return int(self.engine.lib.mrc_batch_window_cells(self.handle))

    def close(self):
        if self.handle:
            self.engine.lib.mrc_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Negotiation:
    """Snapshot negotiation rounds on the device (mrc_negotiation_*): each
    round rips up the dirty nets, prices a frozen snapshot
    base + history + pfac * present_weight * present per directed planar edge
    slot, routes the dirty nets alone on it, merges them back and adds
    history_step to every edge two or more nets use.

    With a clearance (`clearance` cells around every path cell, `via_keepout`
    cells around every via) the rounds are the reference's clearance-active
    iteration: every net is routed every round, nothing is ripped up before
    pricing, the snapshot adds pfac * halo_weight * halo (the footprints of
    every net's path covering a cell) and each net is priced with its own path
    and footprint subtracted (mrc_negotiation_set_clearance)."""

    def __init__(self, engine: "Engine", req: IsolatedRouteRequest, present_weight: int = 16,
                 history_step: int = 1, owned: Optional[Sequence[bool]] = None, groups=None,
                 clearance: int = 0, via_keepout: int = 0, halo_weight: int = 16):
        """`groups`: None (every net its own group), "connections" (the
        reference's connection groups from the net names and shared endpoints),
        or one group id per net; with groups an edge is overused only when nets
        of two or more groups use it."""
        self.engine = engine
        self.n = len(req.nets)
        self.dims = req.grid.dims
        m = _Marshal()
        r = engine._request(m, req)
        h = C.c_void_p()
        prm = C.byref(_NegParams(present_weight, history_step))
        if owned is None:
            engine._check(engine.lib.mrc_negotiation_create(engine.ctx, C.byref(r), prm, C.byref(h)))
        else:
            mask = np.ascontiguousarray(np.asarray(owned, dtype=np.uint8))
            if mask.size != self.n:
                raise InvalidArgument("owned mask must have one entry per net")
            engine._check(engine.lib.mrc_negotiation_create_shard(engine.ctx, C.byref(r), prm, m.arr(mask),
                                                                  C.byref(h)))
        self.handle = h
        engine._adopt(self)
        try:
            self._set_groups(req, groups)
            if clearance or via_keepout:
                engine._check(engine.lib.mrc_negotiation_set_clearance(engine.ctx, self.handle, int(clearance),
                                                                       int(via_keepout), int(halo_weight)))
        except Exception:
            self.close()
            raise

    def _set_groups(self, req: IsolatedRouteRequest, groups) -> None:
        engine = self.engine
        if groups is not None:
            if isinstance(groups, str):
                if groups != "connections":
                    raise InvalidArgument("groups must be None, 'connections' or one id per net")
                groups = connection_group_ids(req.nets)
            g = np.ascontiguousarray(np.asarray(groups, dtype=np.uint32))
            if g.size != self.n:
                raise InvalidArgument("groups must have one entry per net")
            engine._check(engine.lib.mrc_negotiation_set_groups(engine.ctx, self.handle,
                                                                g.ctypes.data if g.size else None))

    @staticmethod
    def _stats(st) -> dict:
        return {f: getattr(st, f) for f, _ in _RoundStats._fields_}

    def round(self) -> dict:
        st = _RoundStats()
        e = self.engine
        e._check(e.lib.mrc_negotiation_round(e.ctx, self.handle, C.byref(st)))
        return self._stats(st)

    # -- the phases of a sharded round ----------------------------------------
    def ripup(self) -> None:
        self.engine._check(self.engine.lib.mrc_negotiation_ripup(self.engine.ctx, self.handle))

    def route(self) -> dict:
        st = _RoundStats()
        self.engine._check(self.engine.lib.mrc_negotiation_route(self.engine.ctx, self.handle, C.byref(st)))
        return self._stats(st)

    def settle(self) -> dict:
        st = _RoundStats()
        self.engine._check(self.engine.lib.mrc_negotiation_settle(self.engine.ctx, self.handle, C.byref(st)))
        return self._stats(st)

    def occupancy(self):
        """(local, global) occupancy as int32 CUDA tensors of 4 slots per cell,
        sharing the engine's device memory (for an all-reduce between phases)."""
        import torch

        loc, glo, nbytes = C.c_void_p(), C.c_void_p(), C.c_uint64()
        self.engine._check(self.engine.lib.mrc_negotiation_buffers(self.handle, C.byref(loc), C.byref(glo),
                                                                   C.byref(nbytes)))
        n = int(nbytes.value) // 4

        class _Dev:
            def __init__(self, ptr):
                self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False),
                                                 "version": 3}

        return (torch.as_tensor(_Dev(loc.value), device="cuda"), torch.as_tensor(_Dev(glo.value), device="cuda"))

    def paths(self) -> List[Optional[List[int]]]:
        n, off, cells = C.c_uint32(), C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
        self.engine._check(self.engine.lib.mrc_negotiation_paths(self.handle, C.byref(n), C.byref(off),
                                                                 C.byref(cells)))
        o = np.ctypeslib.as_array(off, shape=(n.value + 1,)).copy()
        total = int(o[-1])
        c = np.ctypeslib.as_array(cells, shape=(total,)).copy() if total else np.zeros(0, np.uint32)
        return [c[o[i]:o[i + 1]].tolist() if o[i + 1] > o[i] else None for i in range(n.value)]

    def read(self):
        """(present, history, snapshot) as uint32 arrays of shape (cells, 4)."""
        cells = len(self.dims)
        out = [np.zeros((cells, 4), np.uint32) for _ in range(3)]
        m = _Marshal()
        e = self.engine
        e._check(e.lib.mrc_negotiation_read(e.ctx, self.handle, m.arr(out[0]), m.arr(out[1]), m.arr(out[2])))
        return tuple(out)

    def read_halo(self) -> np.ndarray:
        """Footprint visits per cell (uint32, one per cell); needs a clearance."""
        out = np.zeros(len(self.dims), np.uint32)
        m = _Marshal()
        e = self.engine
        e._check(e.lib.mrc_negotiation_read_halo(e.ctx, self.handle, m.arr(out)))
        return out

    def dirty(self) -> List[int]:
        n, p = C.c_uint32(), C.POINTER(C.c_uint32)()
        self.engine._check(self.engine.lib.mrc_negotiation_dirty(self.handle, C.byref(n), C.byref(p)))
        return np.ctypeslib.as_array(p, shape=(n.value,)).tolist() if n.value else []

    def close(self):
        if self.handle:
            self.engine.lib.mrc_negotiation_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (mrc_server_*): submit from any thread,
    wait for each ticket; admitted requests are merged into shared launches
    under an HBM budget with `slots` launches in flight."""

    def __init__(self, engine: "Engine", hbm_fraction: float = 0.8, slots: int = 2, max_batch_requests: int = 64,
                 max_batch_cells: int = 0, max_layers: int = 8, merge_ratio: int = 8):
        """merge_ratio: requests merge into one launch only when their window
        cells are within this factor of each other (0 = regardless of size)."""
        self.engine = engine
        h = C.c_void_p()
        prm = _ServerParams(hbm_fraction, slots, max_batch_requests, max_batch_cells, max_layers, merge_ratio)
        engine._check(engine.lib.mrc_server_create(engine.ctx, C.byref(prm), C.byref(h)))
        self.handle = h
        engine._adopt(self)
        self._live = {}
        self._lock = threading.Lock()

    def submit(self, req: IsolatedRouteRequest, retry_full: bool = True, keep_fields: bool = False) -> int:
        m = _Marshal()
        r = self.engine._request(m, req)
        flags = (MRC_FLAG_RETRY_FULL if retry_full else 0) | (MRC_FLAG_KEEP_FIELDS if keep_fields else 0)
        t = C.c_uint64()
        self.engine._check(self.engine.lib.mrc_server_submit(self.handle, C.byref(r), flags, C.byref(t)))
        with self._lock:  # the request's arrays are borrowed until its wait returns
            self._live[t.value] = (m, len(req.nets), keep_fields)
        return t.value

    def submit_resident(self, board: Board, nets: Sequence[NetEndpoints],
                        windows: Optional[Sequence[IsolatedRouteWindow]] = None, retry_full: bool = True,
                        keep_fields: bool = False) -> int:
        """A request against a board already in HBM (no board upload)."""
        m = _Marshal()
        flags = (MRC_FLAG_RETRY_FULL if retry_full else 0) | (MRC_FLAG_KEEP_FIELDS if keep_fields else 0)
        t = C.c_uint64()
        self.engine._check(self.engine.lib.mrc_server_submit_resident(
            self.handle, board.handle, m.nets(nets), len(nets), m.windows(windows), flags, C.byref(t)))
        with self._lock:
            self._live[t.value] = (m, len(nets), keep_fields)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 0):
        """(IsolatedBatchResult, info) of a ticket; raises the request's error."""
        res = C.c_void_p()
        info = _RequestInfo()
        st = self.engine.lib.mrc_server_wait(self.handle, ticket, timeout_ms, C.byref(res), C.byref(info))
        if st == Busy.status:
            raise Busy("request still running")
        with self._lock:
            _, n, keep = self._live.pop(ticket, (None, 0, False))
        d = {f: getattr(info, f) for f, _ in _RequestInfo._fields_}
        if st != MRC_OK:
            msg = self.engine.lib.mrc_last_error(self.engine.ctx)
            raise _ERRORS.get(st, RouterError)(msg.decode() if msg else "")
        return _take_result(self.engine.lib, res, n, keep), d

    def stats(self) -> dict:
        out = (C.c_uint64 * 8)()
        self.engine._check(self.engine.lib.mrc_server_stats(self.handle, out))
        keys = ("submitted", "completed", "failed", "launches", "largest_launch", "peak_bytes", "budget_bytes",
                "queued")
        return dict(zip(keys, [int(v) for v in out]))

    def close(self):
        if self.handle:
            self.engine.lib.mrc_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _HostBlock:
    """Frees one mrc_host_alloc block when the buffer that owns it goes away."""

    def __init__(self, lib, ptr: int):
        self.lib, self.ptr = lib, ptr

    def __del__(self):
        if self.ptr:
            self.lib.mrc_host_free(C.c_void_p(self.ptr))
            self.ptr = 0


class Engine:
    """One CUDA context of the engine (one per process per device)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        ctx = C.c_void_p()
        self.ctx = None
        self._children = weakref.WeakSet()  # boards, batches, servers, negotiations made on this context
        self._check(self.lib.mrc_context_create(int(device), C.byref(ctx)))
        self.ctx = ctx

    def _adopt(self, obj) -> None:
        """Register an object whose handle lives in this context: it is closed
        before the context is, whatever order the garbage collector takes."""
        self._children.add(obj)

    def close(self):
        if self.ctx:
            for child in list(self._children):
                try:
                    child.close()
                except Exception:
                    pass
            self.lib.mrc_context_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_schedule(self, schedule: int) -> None:
        """Relax schedule of batches this engine builds without an autotuned
        configuration: 0, 1 (the default), 2 or 3, as Batch.set_schedule."""
        self._check(self.lib.mrc_context_set_schedule(self.ctx, int(schedule)))

    def _check(self, status: int) -> None:
        if status != MRC_OK:
            msg = self.lib.mrc_last_error(self.ctx)
            msg = msg.decode() if msg else ""
            raise _ERRORS.get(status, RouterError)(msg)

    # -- page-locked host arrays --------------------------------------------
    def pinned_empty(self, shape, dtype) -> np.ndarray:
        """An uninitialised numpy array in page-locked, device-mapped host
        memory (freed when the last view of it goes away).  Board arrays held
        here are read in place by route_instances and reach HBM at full link
        rate in the single-board calls."""
        dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape, dtype=np.int64)) * dtype.itemsize
        p = C.c_void_p()
        self._check(self.lib.mrc_host_alloc(self.ctx, max(nbytes, 1), C.byref(p)))
        buf = (C.c_char * max(nbytes, 1)).from_address(p.value)
        buf._block = _HostBlock(self.lib, p.value)
        return np.frombuffer(buf, dtype=dtype, count=nbytes // dtype.itemsize).reshape(shape)

    def upload_stats(self) -> dict:
        """Board bytes moved to HBM so far: staged, and read in place from
        page-locked arrays."""
        a, b = C.c_uint64(), C.c_uint64()
        self._check(self.lib.mrc_upload_stats(self.ctx, C.byref(a), C.byref(b)))
        return {"staged_bytes": a.value, "in_place_bytes": b.value}

    def pin(self, a):
        """A page-locked copy of `a` (None stays None)."""
        if a is None:
            return None
        a = np.asarray(a)
        out = self.pinned_empty(a.shape, a.dtype)
        out[...] = a
        return out

    # -- the provider seam ---------------------------------------------------
    def _request(self, m: _Marshal, req: IsolatedRouteRequest) -> _Request:
        """The C request for one board, written from numpy columns like the
        instances' (no per-net ctypes objects); `m` keeps every buffer alive."""
        if len(req.windows) != len(req.nets):
            raise BackendUnavailable("isolated request windows are not net-aligned")
        return _marshal_requests(m, [req])[0]

    def route_isolated_batch(self, req: IsolatedRouteRequest, retry_full: bool = True, keep_fields: bool = False,
                             no_wait: bool = False) -> IsolatedBatchResult:
        m = _Marshal()
        r = self._request(m, req)
        flags = ((MRC_FLAG_RETRY_FULL if retry_full else 0) | (MRC_FLAG_KEEP_FIELDS if keep_fields else 0)
                 | (MRC_FLAG_NO_WAIT if no_wait else 0))
        res = C.c_void_p()
        self._check(self.lib.mrc_route_isolated_batch(self.ctx, C.byref(r), flags, C.byref(res)))
        return _take_result(self.lib, res, len(req.nets), keep_fields)

    def route_instances(self, requests: Sequence[IsolatedRouteRequest], retry_full: bool = True,
                        keep_fields: bool = False, split: bool = True):
        """Solve many independent instances (own board, nets, windows) in one
        persistent launch; one result per instance, or with split=False one
        result over the instances' nets in order."""
        m = _Marshal()
        reqs = _marshal_requests(m, requests)
        flags = (MRC_FLAG_RETRY_FULL if retry_full else 0) | (MRC_FLAG_KEEP_FIELDS if keep_fields else 0)
        res = C.c_void_p()
        self._check(self.lib.mrc_route_instances(self.ctx, C.cast(reqs, C.c_void_p), len(requests), flags,
                                                 C.byref(res)))
        total = sum(len(rq.nets) for rq in requests)
        allr = _take_result(self.lib, res, total, keep_fields)
        if not split:
            return allr
        out, o = [], 0
        for rq in requests:
            n = len(rq.nets)
            out.append(allr.slice(o, o + n))
            o += n
        return out

    def route_isolated_plain(self, req: IsolatedRouteRequest, retry_full: bool = True,
                             keep_fields: bool = False) -> IsolatedBatchResult:
        m = _Marshal()
        r = self._request(m, req)
        flags = (MRC_FLAG_RETRY_FULL if retry_full else 0) | (MRC_FLAG_KEEP_FIELDS if keep_fields else 0)
        res = C.c_void_p()
        self._check(self.lib.mrc_route_isolated_plain(self.ctx, C.byref(r), flags, C.byref(res)))
        return _take_result(self.lib, res, len(req.nets), keep_fields)

    # -- Router contract and fields -------------------------------------------
    def route_lee(self, grid: Grid, nets: Sequence[NetEndpoints]) -> "BoardRoute":
        m = _Marshal()
        res = C.c_void_p()
        self._check(self.lib.mrc_route_lee(self.ctx, C.byref(m.grid(grid)), m.nets(nets), len(nets),
                                           C.byref(res)))
        out = _take_result(self.lib, res, len(nets), False)
        return BoardRoute.from_paths(grid, nets, out.paths, out.search_costs)

    def distance_fields(self, grid: Grid, sources: Sequence[int]) -> np.ndarray:
        m = _Marshal()
        src = _u32(sources)
        out = np.zeros((len(sources), len(grid.dims)), dtype=np.uint32)
        if len(sources):
            self._check(self.lib.mrc_distance_fields(self.ctx, C.byref(m.grid(grid)), m.arr(src), len(sources),
                                                     m.arr(out)))
        return out

    def board(self, grid: Grid, x, y, vias, directed=None) -> Board:
        return Board(self, grid, x, y, vias, directed)

    def selftest_wait_timeout(self, spin_limit: int = 1000) -> dict:
        """Runs the bounded-wait self-test kernel (a barrier wait that cannot
        complete) and returns its status bits and device time."""
        st, ms = C.c_uint32(), C.c_float()
        self._check(self.lib.mrc_selftest_wait_timeout(self.ctx, int(spin_limit), C.byref(st), C.byref(ms)))
        return {"status": int(st.value), "ms": float(ms.value)}

    def server(self, **kw) -> Server:
        return Server(self, **kw)

    def negotiation(self, req: IsolatedRouteRequest, present_weight: int = 16, history_step: int = 1,
                    owned: Optional[Sequence[bool]] = None, groups=None, clearance: int = 0,
                    via_keepout: int = 0, halo_weight: int = 16) -> Negotiation:
        """An unsharded negotiation, or (with `owned`) this GPU's shard of one;
        `groups` and the clearance radii as in Negotiation."""
        return Negotiation(self, req, present_weight, history_step, owned, groups, clearance, via_keepout,
                           halo_weight)


def net_windows(dims, nets: Sequence[NetEndpoints]) -> List[IsolatedRouteWindow]:
    """net_window (negotiated.rs:568-594), computed by the library."""
    L = load_library()
    m = _Marshal()
    out = (_Window * max(len(nets), 1))()
    st = L.mrc_net_windows(dims.w, dims.h, dims.layers, m.nets(nets), len(nets), C.cast(out, C.c_void_p))
    if st != MRC_OK:
        raise _ERRORS.get(st, RouterError)("net_windows failed")
    return [IsolatedRouteWindow(out[i].x0, out[i].y0, out[i].x1, out[i].y1) for i in range(len(nets))]


@dataclass
class RouteResult:
    net: str
    path: List[int]
    cost: int


@dataclass
class BoardRoute:
    """mr_core::BoardRoute (core/src/lib.rs:552-594)."""

    results: List[RouteResult]
    unrouted: List[str]
    congestion: np.ndarray

    @staticmethod
    def from_paths(grid: Grid, nets, paths, costs) -> "BoardRoute":
        results, unrouted = [], []
        cong = np.zeros(len(grid.dims), dtype=np.uint32)
        for n, p, c in zip(nets, paths, costs):
            if p is None:
                unrouted.append(n.net)
                continue
            results.append(RouteResult(n.net, p, c))
            cong[np.unique(np.asarray(p, dtype=np.int64))] += 1
        return BoardRoute(results, unrouted, cong)


class CudaIsolatedProvider:
    """IsolatedRouteProvider backed by the CUDA engine (negotiated.rs:554-560).

    Mirrors MetalIsolatedProvider (crates/mr-cli/src/lib.rs:612-625): a busy
    engine fails immediately (the router then takes its CPU path) instead of
    queueing behind another board's batch."""

    def __init__(self, engine: Optional[Engine] = None, device: int = 0):
        self.engine = engine or Engine(device)

    def route_isolated_batch(self, request: IsolatedRouteRequest) -> List[Optional[List[int]]]:
        out = self.engine.route_isolated_batch(request, retry_full=True, no_wait=True)
        if len(out.paths) != len(request.nets):
            raise BackendUnavailable("CUDA isolated result is not net-aligned")
        return out.paths


__all__ = [
    "Engine", "Board", "Batch", "Negotiation", "Server", "CudaIsolatedProvider", "IsolatedBatchResult", "BoardRoute", "RouteResult",
    "RouterError", "InvalidArgument", "MalformedGrid", "InvalidEndpoint", "BackendUnavailable", "Busy",
    "IterationLimit", "OutOfMemory", "LimitExceeded", "net_windows", "load_library", "exported_symbols",
    "COST_MAX", "NO_PATH",
]
