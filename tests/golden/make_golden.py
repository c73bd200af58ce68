#!/usr/bin/env python3
"""Generate tests/golden/reference_cases.json from the reference's own tests.

The reference (metal-route, Rust) cannot be built in this environment, so its
known answers are pinned by restating the INPUTS of its hot-path tests and the
OUTPUTS its assertions state (``expect``).  Every case names the test it comes
from (file:line relative to the metal-route project root).

Cases whose reference assertion is "GPU equals the CPU router" carry no pinned
answer; for those the oracle's answer is recorded under ``oracle_expect`` as a
regression fixture (the oracle itself is pinned by the known-answer cases).

Run:  python tests/golden/make_golden.py        (rewrites reference_cases.json)
"""
from __future__ import annotations

import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "metal-route_b200"))

MAX = 0xFFFFFFFF
SCALE = 16
TRACE_NODE, VIA_NODE, NEG_Y, NEG_X, POS_X, POS_Y = 1, 2, 4, 8, 16, 32


def fixed_edge(length: float) -> int:
    """edge_cost (crates/mr-cpu/src/dijkstra.rs:43-52): round-half-away(len*16)."""
    x = length * 16.0
    if not math.isfinite(x) or x <= 0.0:
        return 0
    r = math.floor(x)
    if x - r >= 0.5:
        r += 1
    if r <= 0:
        return 0
    return MAX if r >= MAX else int(r)


def axis_edges(lines, count):
    """axis_edge_costs (crates/mr-cpu/src/negotiated.rs:1197-1201,1268-1272)."""
    out = []
    for k in range(max(count - 1, 0)):
        a = lines[k] if k < len(lines) else float(k)
        b = lines[k + 1] if k + 1 < len(lines) else float(k + 1)
        out.append(fixed_edge(abs(b - a)))
    return out


def vias_of(layers, step_cost, allowed=None):
    """via_edge_costs (negotiated.rs:1423-1429) for ViaModel (core/src/lib.rs:329-372)."""
    out = []
    for k in range(max(layers - 1, 0)):
        ok = allowed is None or (k, k + 1) in allowed
        out.append(step_cost if ok else None)
    return out


class G:
    def __init__(self, w, h, layers=1, fill=1):
        self.w, self.h, self.layers = w, h, layers
        self.cost = [fill] * (w * h * layers)
        self.board = None
        self.via_forbidden = None

    def idx(self, x, y, l=0):
        return (l * self.h + y) * self.w + x

    def mark_rect(self, x0, y0, x1, y1, l=0):
        for y in range(y0, y1 + 1):
            for x in range(x0, x1 + 1):
                if x < self.w and y < self.h:
                    self.cost[self.idx(x, y, l)] = MAX

    def js(self):
        return {"dims": [self.w, self.h, self.layers], "cost": self.cost, "board": self.board,
                "via_forbidden": self.via_forbidden}


def net(src, dst, pads=(), via_pads=(), name="n0"):
    return {"name": name, "src": src, "dst": dst, "pads": list(pads), "via_pads": list(via_pads)}


def ascii_fixture(s):
    """parse_ascii (crates/mr-fixtures/src/lib.rs:41-79)."""
    rows = [r for r in s.split("\n") if r]
    h, w = len(rows), max(len(r) for r in rows)
    g = G(w, h)
    src = dst = None
    for y, row in enumerate(rows):
        for x, ch in enumerate(row):
            if ch == "#":
                g.cost[g.idx(x, y)] = MAX
            elif ch == "S":
                src = g.idx(x, y)
            elif ch == "T":
                dst = g.idx(x, y)
    return g, net(src, dst)


def xorshift(state):
    while True:
        state ^= (state << 13) & 0xFFFFFFFFFFFFFFFF
        state ^= state >> 7
        state ^= (state << 17) & 0xFFFFFFFFFFFFFFFF
        yield state


def cases():
    out = []

    def add(name, source, kind, g, nets, expect=None, **kw):
        c = {"name": name, "source": source, "kind": kind, **g.js(), "nets": nets, "expect": expect}
        c.update(kw)
        out.append(c)

    # ---- Lee / field battery (crates/mr-fixtures/src/lib.rs:87-139) ---------
    g = G(32, 32)
    g.mark_rect(15, 0, 15, 30)
    add("hand_32x32_wall", "crates/mr-fixtures/src/lib.rs:87-104; crates/mr-cpu/src/lee.rs:137-151",
        "lee", g, [net(g.idx(0, 0), g.idx(31, 0))], {"cost": 93, "path_len": 94, "field_at_dst": 93})
    g = G(2, 2)
    add("tie_break_2x2", "crates/mr-fixtures/src/lib.rs:109-125; crates/mr-cpu/src/lee.rs:153-161",
        "lee", g, [net(0, 3)], {"cost": 2, "path": [0, 1, 3]})
    battery = [("open_5x5", "S....\n.....\n.....\n.....\n....T", 8),
               ("notch", "S.#..\n..#..\n..#..\n..#..\n....T", 8),
               ("spiral", "S....\n####.\n...#.\n.#.#.\n.#..T", None),
               ("corridor", "S#...\n.#.#.\n.#.#.\n.#.#.\n...#T", None),
               ("blocked_gap", "S....\n.###.\n.#T#.\n.###.\n.....", "unrouted")]
    for name, art, exp in battery:
        g, n = ascii_fixture(art)
        e = {"cost": exp} if isinstance(exp, int) else ({"unrouted": True} if exp == "unrouted" else None)
        add(name, "crates/mr-fixtures/src/lib.rs:130-139; crates/mr-cpu/src/lee.rs:163-187", "lee", g, [n], e)

    # ---- shared router contracts (crates/mr-cpu/src/lib.rs:70-302) ----------
    g = G(2, 1)
    g.mark_rect(0, 0, 1, 0)
    add("own_pad_endpoints", "crates/mr-cpu/src/lib.rs:70-87", "lee", g, [net(0, 1, pads=[0, 1])],
        {"cost": 1, "path": [0, 1]})
    g = G(3, 2)
    g.cost[g.idx(1, 0)] = 100
    add("weighted_detour", "crates/mr-cpu/src/lib.rs:111-125", "lee", g, [net(0, 2)],
        {"cost": 4, "path": [0, 3, 4, 5, 2]})
    g = G(3, 2, fill=0)
    add("zero_cost_plateau", "crates/mr-cpu/src/lib.rs:127-143", "lee", g, [net(5, 3)],
        {"cost": 0, "path": [5, 4, 3]})
    g = G(3, 3)
    add("zero_length", "crates/mr-cpu/src/lib.rs:145-155", "lee", g, [net(4, 4)], {"cost": 0, "path": [4]})
    g = G(3, 2)
    g.board = [0] * 6
    g.board[0] |= POS_X
    g.board[1] |= NEG_X
    add("board_edge_barrier", "crates/mr-cpu/src/lib.rs:214-229", "lee", g, [net(0, 2)],
        {"path": [0, 3, 4, 1, 2]})
    g = G(5, 3)
    add("two_nets_cost_sum", "crates/mr-cpu/src/lib.rs:271-302", "lee", g,
        [net(g.idx(0, 0), g.idx(4, 0), name="a"), net(g.idx(0, 2), g.idx(4, 2), name="b")], {"total_cost": 8})
    # dijkstra.rs tests
    g = G(4, 1)
    add("generation_wrap_line", "crates/mr-cpu/src/dijkstra.rs:544-567", "lee", g, [net(0, 3)],
        {"cost": 3, "path": [0, 1, 2, 3]})
    g = G(3, 2)
    g.cost[1] = 0
    g.cost[2] = 0
    add("zero_cost_edges", "crates/mr-cpu/src/dijkstra.rs:569-588", "lee", g, [net(0, 2)],
        {"cost": 0, "path": [0, 1, 2]})
    g = G(3, 2)
    g.cost = [1, 1, 1, 1, 3, 1]
    add("lee_minimum_hops_weighted_tie", "crates/mr-metal/src/lib.rs:2565-2588", "lee", g, [net(3, 5)],
        {"cost": 4, "path": [3, 4, 5]})

    # ---- field routines (crates/mr-cpu/src/sweep.rs) -------------------------
    g = G(3, 2)
    g.board = [0] * 6
    g.board[g.idx(1, 0)] |= NEG_X
    g.board[g.idx(2, 1)] |= TRACE_NODE
    add("sweep_board_nodes_and_asymmetric_edges", "crates/mr-cpu/src/sweep.rs:350-370", "field", g,
        [net(0, 0)], {"field_values": {str(g.idx(1, 0)): 3, str(g.idx(2, 1)): MAX}})
    g = G(5, 4)
    for cell, cost in [(1, 7), (2, 0), (7, 3), (13, 11), (18, 0)]:
        g.cost[cell] = cost
    g.cost[8] = MAX
    add("sweep_weighted_and_zero", "crates/mr-cpu/src/sweep.rs:332-348", "field", g, [net(0, 0)], None)
    g = G(4, 3, 3)
    for (x, y, l) in [(1, 1, 0), (2, 0, 1), (0, 2, 2)]:
        g.cost[g.idx(x, y, l)] = MAX
    add("sweep_every_layer", "crates/mr-cpu/src/sweep.rs:280-299", "field", g, [net(0, 0)], None)

    # ---- isolated provider contract (crates/mr-metal/src/lib.rs tests) -------
    # isolated_batch_matches_cpu_minimum_hops_and_lower_predecessor_ties :1810-1879
    g = G(3, 2)
    g.cost = [1, 1, 1, 1, 3, 1]
    add("iso_minimum_hops", "crates/mr-metal/src/lib.rs:1810-1843", "isolated", g, [net(3, 5)],
        {"paths": [[3, 4, 5]]}, x=axis_edges([], 3), y=axis_edges([], 2), vias=[],
        windows=[[0, 0, 2, 1]])
    g = G(4, 3)
    g.cost[g.idx(2, 1)] = MAX
    add("iso_lower_predecessor", "crates/mr-metal/src/lib.rs:1845-1878", "isolated", g,
        [net(g.idx(0, 1), g.idx(3, 1))], {"paths": [[4, 0, 1, 2, 3, 7]]},
        x=axis_edges([], 4), y=axis_edges([], 3), vias=[], windows=[[0, 0, 3, 2]])
    # isolated_batch_is_deterministic_across_internal_chunk_boundary :2280-2318
    g = G(5, 5)
    nets = [net(g.idx(0, 0) if i % 2 == 0 else g.idx(0, 4), g.idx(4, 4) if i % 2 == 0 else g.idx(4, 0),
                name=f"chunk-{i:03}") for i in range(257)]
    add("iso_chunk_costs", "crates/mr-metal/src/lib.rs:2280-2318", "isolated", g, nets,
        {"search_costs": [8 * SCALE] * 257}, x=[SCALE] * 4, y=[SCALE] * 4, vias=[], windows=[[0, 0, 4, 4]] * 257)
    # isolated_batch_reports_window_failure_then_routes_full_retry :2236-2277
    g = G(5, 3)
    g.cost[g.idx(2, 1)] = MAX
    add("iso_window_failure", "crates/mr-metal/src/lib.rs:2236-2263", "isolated_window", g,
        [net(g.idx(0, 1), g.idx(4, 1), name="retry")], {"paths": [None]}, x=[SCALE] * 4, y=[SCALE] * 2,
        vias=[], windows=[[0, 1, 4, 1]])
    add("iso_window_then_full_retry", "crates/mr-metal/src/lib.rs:2265-2277", "isolated", g,
        [net(g.idx(0, 1), g.idx(4, 1), name="retry")], {"routed": [True]}, x=[SCALE] * 4, y=[SCALE] * 2,
        vias=[], windows=[[0, 1, 4, 1]])
    # isolated_batch_honours_cpu_window_before_full_retry :2192-2234
    g = G(50, 40)
    for y in range(4, 36):
        g.cost[g.idx(21, y)] = MAX
    dst = g.idx(22, 20)
    g.cost[dst] = MAX
    xl = [x * 0.17 for x in range(50)]
    yl = [y * 0.11 for y in range(40)]
    add("iso_windowed_pad", "crates/mr-metal/src/lib.rs:2192-2234", "isolated", g,
        [net(g.idx(20, 20), dst, pads=[dst], name="windowed-pad")], {"path_inside_window": True},
        x=axis_edges(xl, 50), y=axis_edges(yl, 40), vias=[], windows=None)
    # isolated_batch_matches_cpu_on_hanan_weights_zero_overflow_and_pads :1703-1755
    g = G(9, 7)
    g.cost[g.idx(2, 3)] = 0
    g.cost[g.idx(3, 3)] = 7
    g.cost[g.idx(1, 6)] = MAX - 1
    for (x, y) in [(0, 0), (8, 0), (3, 4), (5, 4), (4, 3), (4, 5)]:
        g.cost[g.idx(x, y)] = MAX
    nets = [net(g.idx(0, 3), g.idx(8, 3), name="weighted"),
            net(g.idx(0, 0), g.idx(8, 0), pads=[g.idx(0, 0), g.idx(8, 0)], name="own-obstacle-pads"),
            net(g.idx(0, 6), g.idx(1, 6), name="max-minus-one-enter"),
            net(g.idx(2, 3), g.idx(2, 3), name="zero-length"),
            net(g.idx(0, 4), g.idx(4, 4), name="enclosed")]
    add("iso_hanan_zero_overflow_pads", "crates/mr-metal/src/lib.rs:1703-1755", "isolated", g, nets,
        {"search_cost_of": {"max-minus-one-enter": None}},
        x=axis_edges([0.0, 0.2, 0.7, 1.9, 2.0, 4.5, 4.7, 8.0, 8.1], 9),
        y=axis_edges([0.0, 0.1, 1.0, 1.0, 2.7, 6.0, 6.2], 7), vias=[], windows=None, via_h_cost=160)
    # isolated_batch_matches_cpu_on_restricted_and_extreme_vias :1757-1807
    g = G(6, 5, 4)
    g.cost[g.idx(5, 4, 1)] = MAX
    xr = axis_edges([0.0, 0.25, 1.0, 2.75, 2.8, 7.0], 6)
    yr = axis_edges([0.0, 0.3, 1.2, 1.25, 4.0], 5)
    nets = [net(g.idx(0, 0, 0), g.idx(5, 4, 1), pads=[g.idx(5, 4, 1)], name="lower-span"),
            net(g.idx(5, 0, 2), g.idx(0, 4, 3), name="upper-span"),
            net(g.idx(2, 2, 0), g.idx(2, 2, 3), name="forbidden-middle-span")]
    add("iso_restricted_vias", "crates/mr-metal/src/lib.rs:1757-1790", "isolated", g, nets, None, x=xr, y=yr,
        vias=vias_of(4, 37, {(0, 1), (2, 3)}), windows=None, via_h_cost=37)
    g2 = G(6, 5, 4)
    g2.cost = list(g.cost)
    for layer in range(1, 4):
        g2.cost[g2.idx(3, 1, layer)] = 0
    add("iso_extreme_vias", "crates/mr-metal/src/lib.rs:1792-1806", "isolated", g2,
        [net(g2.idx(3, 1, 0), g2.idx(3, 1, 3), name="zero-weight-max-vias")], None, x=xr, y=yr,
        vias=vias_of(4, MAX, {(0, 1), (1, 2), (2, 3)}), windows=None, via_h_cost=MAX)
    # isolated_batch_deterministic_stress_matches_cpu_alone_paths :1881-1933
    for case in range(12):
        g = G(7, 5, 3)
        rng = xorshift(0xA0761D6478BD642F ^ case)
        for i in range(len(g.cost)):
            r = next(rng)
            g.cost[i] = MAX if r % 11 == 0 else (0 if r % 7 == 0 else 1 + r % 19)
        nets = []
        for i in range(8):
            src = next(rng) % len(g.cost)
            dst = next(rng) % len(g.cost)
            pads = []
            if g.cost[src] == MAX:
                pads.append(src)
            if g.cost[dst] == MAX and dst != src:
                pads.append(dst)
            nets.append(net(src, dst, pads=pads, name=f"case-{case}-net-{i}"))
        vias = vias_of(3, 23, {(0, 1), (1, 2)}) if case % 2 == 0 else vias_of(3, 0, {(1, 2)})
        add(f"iso_stress_{case:02}", "crates/mr-metal/src/lib.rs:1881-1933", "isolated", g, nets, None,
            x=axis_edges([0.0, 0.1, 0.8, 0.85, 2.5, 4.0, 4.2], 7), y=axis_edges([0.0, 0.4, 0.45, 3.0, 3.2], 5),
            vias=vias, windows=None, via_h_cost=23 if case % 2 == 0 else 0)
    # ragged_batch_matches_full_fields_on_adversarial_variable_windows :1935-2016 (no retry)
    xs = [(i * 17) % 41 for i in range(12)]
    ys = [(i * 23) % 37 for i in range(10)]
    patterns = [[0, MAX], [29, None], [None, 7]]
    for case in range(18):
        g = G(13, 11, 3)
        rng = xorshift(0xD1B54A32D192ED03 ^ ((case * 0x9E3779B9) & 0xFFFFFFFFFFFFFFFF))
        for i in range(len(g.cost)):
            r = next(rng)
            g.cost[i] = MAX if r % 13 == 0 else (0 if r % 7 == 0 else 1 + r % 31)
        nets, wins = [], []
        for ni in range(24):
            w = 2 + next(rng) % 12
            h = 2 + next(rng) % 10
            x0 = next(rng) % (13 - w + 1)
            y0 = next(rng) % (11 - h + 1)
            src = g.idx(x0 + next(rng) % w, y0 + next(rng) % h, next(rng) % 3)
            dst = g.idx(x0 + next(rng) % w, y0 + next(rng) % h, next(rng) % 3)
            pads = []
            if g.cost[src] == MAX:
                pads.append(src)
            if g.cost[dst] == MAX and dst != src:
                pads.append(dst)
            pad = g.idx(x0, y0, ni % 3)
            if g.cost[pad] == MAX and pad not in pads:
                pads.append(pad)
            nets.append(net(src, dst, pads=pads, name=f"ragged-{case:02}-{ni:02}"))
            wins.append([x0, y0, x0 + w - 1, y0 + h - 1])
        add(f"iso_ragged_{case:02}", "crates/mr-metal/src/lib.rs:1935-2016", "isolated_window", g, nets, None,
            x=xs, y=ys, vias=patterns[case % 3], windows=wins)
    # isolated_provider_matches_cpu_for_reachable_unreachable_and_zero_hop_nets
    # (crates/mr-cpu/src/negotiated.rs:4451-4480)
    g = G(5, 5)
    for (x, y) in [(2, 1), (1, 2), (3, 2), (2, 3)]:
        g.cost[g.idx(x, y)] = MAX
    add("provider_reachable_unreachable_zero", "crates/mr-cpu/src/negotiated.rs:4451-4467", "isolated", g,
        [net(g.idx(0, 4), g.idx(4, 4), name="open"), net(g.idx(0, 0), g.idx(2, 2), name="blocked"),
         net(g.idx(4, 0), g.idx(4, 0), name="zero")],
        {"routed": [True, False, True], "paths_of": {"zero": [g.idx(4, 0)]}},
        x=[SCALE] * 4, y=[SCALE] * 4, vias=[], windows=None)

    # ---- request edge vectors (negotiated.rs:4659-4705) ----------------------
    out.append({"name": "request_edge_vectors", "source": "crates/mr-cpu/src/negotiated.rs:4685-4705",
                "kind": "edge_vectors", "x_lines": [10.0], "y_lines": [], "dims": [4, 3, 3],
                "expect": {"x": [144, 16, 16], "y": [16, 16], "vias": [7, None]},
                "via_step_cost": 7, "allowed": [[0, 1]]})

    # ---- provider_path_is_valid (negotiated.rs:4519-4575) --------------------
    g = G(3, 2)
    g.cost[g.idx(1, 0)] = MAX
    add("valid_through_obstacle", "crates/mr-cpu/src/negotiated.rs:4523-4531", "path_valid", g,
        [net(0, 2)], {"valid": False}, path=[0, 1, 2], via_allowed=[])
    g = G(3, 2)
    add("valid_repeated_cell", "crates/mr-cpu/src/negotiated.rs:4532-4541", "path_valid", g, [net(0, 2)],
        {"valid": False}, path=[0, 3, 0, 2], via_allowed=[])
    g = G(1, 1, 2)
    add("valid_forbidden_via", "crates/mr-cpu/src/negotiated.rs:4543-4552", "path_valid", g, [net(0, 1)],
        {"valid": False}, path=[0, 1], via_allowed=[False])
    g = G(1, 1, 2)
    g.via_forbidden = [1, 1]
    add("valid_owned_via_exemptions", "crates/mr-cpu/src/negotiated.rs:4554-4567", "path_valid", g,
        [net(0, 1, pads=[1, 0], via_pads=[1, 0])], {"valid": True}, path=[0, 1], via_allowed=[True])
    add("valid_layer_local_exemption_only", "crates/mr-cpu/src/negotiated.rs:4568-4575", "path_valid", g,
        [net(0, 1, pads=[1, 0], via_pads=[0])], {"valid": False}, path=[0, 1], via_allowed=[True])
    return out


def main():
    import oracle as orc
    from mrcuda.types import Dims, Grid, IsolatedRouteRequest, IsolatedRouteWindow, NetEndpoints
    import numpy as np

    o = orc.get()
    cs = cases()
    for c in cs:
        if c["kind"] not in ("isolated", "isolated_window") or c.get("expect") is not None and "paths" in c["expect"]:
            continue
        dims = Dims(*c["dims"])
        grid = Grid(dims, np.array(c["cost"], dtype=np.uint32),
                    None if c["board"] is None else np.array(c["board"], dtype=np.uint8),
                    None if c["via_forbidden"] is None else np.array(c["via_forbidden"], dtype=np.uint8))
        nets = [NetEndpoints(n["name"], n["src"], n["dst"], n["pads"], n["via_pads"]) for n in c["nets"]]
        wins = ([IsolatedRouteWindow(*w) for w in c["windows"]] if c.get("windows") is not None
                else [o.net_window(dims, n) for n in nets])
        req = IsolatedRouteRequest(grid, nets, wins, c["x"], c["y"], c["vias"])
        paths, costs = o.isolated_batch(req, retry_full=c["kind"] == "isolated", mode="astar",
                                        via_h_cost=c.get("via_h_cost"))
        c["oracle_expect"] = {"paths": paths, "search_costs": costs}
    path = os.path.join(HERE, "reference_cases.json")
    with open(path, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cs}, f, separators=(",", ":"))
    print(f"wrote {len(cs)} cases to {path}")


if __name__ == "__main__":
    main()
