/*
 * oracle.h — CPU restatement of metalroute's canonical shortest-path semantics.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the test oracle of the CUDA engine in
 * metal-route_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it. Nothing in the product links, calls or falls back to it.
 *
 * Every function restates one routine of the reference (paths are relative to
 * the metal-route project root) and cites it. The reference is Rust and cannot
 * be compiled here (no cargo/rustc), so parity is pinned by the reference's own
 * known-answer tests, restated as golden fixtures under tests/golden/.
 *
 * Conventions (crates/mr-core/src/lib.rs:19-25, 83-164):
 *   Cost = uint32, OBSTACLE = 0xFFFFFFFF, CellIdx = uint32 with
 *   idx3(x, y, l) = (l*h + y)*w + x.  Neighbour order is ascending CellIdx:
 *   lower layer, -y, -x, +x, +y, upper layer.
 */
#ifndef MR_ORACLE_H
#define MR_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX 0xFFFFFFFFu

/* Grid::BOARD_* bits, crates/mr-core/src/lib.rs:411-416. */
#define ORC_BOARD_TRACE_NODE 0x01u
#define ORC_BOARD_VIA_NODE 0x02u
#define ORC_BOARD_EDGE_NEG_Y 0x04u
#define ORC_BOARD_EDGE_NEG_X 0x08u
#define ORC_BOARD_EDGE_POS_X 0x10u
#define ORC_BOARD_EDGE_POS_Y 0x20u

typedef struct {
    uint32_t w, h, layers;
    const uint32_t *cost;          /* w*h*layers enter weights */
    const uint8_t *board;          /* nullable: Grid::board_constraint */
    const uint8_t *via_forbidden;  /* nullable: Grid::via_forbidden (0/1) */
} orc_grid;

/* Already-rounded static edge prices, crates/mr-cpu/src/negotiated.rs:521-537.
 * `directed` (nullable) is the superset form: 4 base prices per destination cell
 * for the planar in-edges from its -y, -x, +x, +y neighbours (ascending source
 * CellIdx); 0xFFFFFFFF there marks a blocked edge. When `directed` is set it
 * replaces the per-axis gap price; the enter-weight product and cap still apply. */
typedef struct {
    const uint32_t *x_edge;       /* w-1 */
    const uint32_t *y_edge;       /* h-1 */
    const uint32_t *via_edge;     /* layers-1 */
    const uint8_t *via_allowed;   /* layers-1, 0 = Option::None */
    const uint32_t *directed;     /* nullable, 4*w*h*layers */
} orc_edges;

typedef struct {
    uint32_t src, dst;
    const uint32_t *pads;
    uint32_t n_pads;
    const uint32_t *via_pads;
    uint32_t n_via_pads;
} orc_net;

typedef struct {
    uint32_t x0, y0, x1, y1;
} orc_window;

/* --- small helpers exposed for tests --------------------------------------- */

/* edge_cost, crates/mr-cpu/src/dijkstra.rs:43-52: round(len*16), saturating. */
uint32_t orc_edge_cost(double length);
/* axis_edge_costs/axis_gap_cost, crates/mr-cpu/src/negotiated.rs:1197-1201,1268-1272. */
void orc_axis_edge_costs(const double *lines, uint32_t n_lines, uint32_t count, uint32_t *out);
/* net_window, crates/mr-cpu/src/negotiated.rs:568-594. */
orc_window orc_net_window(uint32_t w, uint32_t h, uint32_t layers, const orc_net *net);
/* Grid::is_board_planar_step_forbidden, crates/mr-core/src/lib.rs:466-496. */
int orc_board_planar_forbidden(const orc_grid *g, uint32_t u, uint32_t v);

/* --- isolated ("alone path") search, the provider contract --------------- */

/* astar_buf (crates/mr-cpu/src/dijkstra.rs:243-401) driven by the static cost
 * model of route_legal_once (crates/mr-cpu/src/negotiated.rs:2885-3052) with no
 * owners, no halo and an unoccupied via guard.  `via_h_cost` is the via model's
 * step_cost used by the heuristic (manhattan_scaled, negotiated.rs:1235-1251);
 * `use_heuristic` = 0 selects h = 0 (the has_zero_cost branch).
 * Returns the path length (0 = unreachable); writes up to `cap` cells. */
uint32_t orc_isolated_astar(const orc_grid *g, const orc_edges *e, const orc_net *net,
                            orc_window win, int use_heuristic, uint32_t via_h_cost,
                            uint32_t *path, uint32_t cap, uint32_t *cost_out);

/* Complete field of the same search: h = 0, every reached cell expanded
 * (dst included), labels (dist, hops) minimised lexicographically.  Writes
 * full-grid arrays (cells outside the window stay 0xFFFFFFFF). */
void orc_isolated_field(const orc_grid *g, const orc_edges *e, const orc_net *net,
                        orc_window win, uint32_t *dist, uint32_t *hops);

/* Canonical path from (dist, hops) labels: walk back from dst choosing the lowest
 * CellIdx predecessor p with dist[p] (+) step(p->cur) == dist[cur] and
 * hops[p] + 1 == hops[cur] (crates/mr-metal/src/lib.rs:308-396, with the board
 * edge legality of the CPU relax).  Returns length or 0. */
uint32_t orc_isolated_path_from_labels(const orc_grid *g, const orc_edges *e, const orc_net *net,
                                       orc_window win, const uint32_t *dist, const uint32_t *hops,
                                       uint32_t *path, uint32_t cap);

/* Provider semantics: window search, then a full-board retry only when the
 * window search is unreachable (crates/mr-cpu/src/negotiated.rs:2137-2174,
 * crates/mr-cli/src/lib.rs:549-607).  Batched over nets with `threads` OpenMP
 * threads (0 = all).  Outputs CSR: offsets[n+1], cells (capacity cells_cap),
 * cost[n] (0xFFFFFFFF = unreachable).  mode: 0 = A* (the CPU router's own
 * search), 1 = complete field + canonical walk.  Returns 0 or -1 on capacity. */
int orc_isolated_batch(const orc_grid *g, const orc_edges *e, const orc_net *nets, uint32_t n_nets,
                       const orc_window *windows, int retry_full, int mode, int use_heuristic,
                       uint32_t via_h_cost, int threads, uint64_t *offsets, uint32_t *cells,
                       uint64_t cells_cap, uint32_t *costs);

/* --- planar per-cell-cost routines (Lee / fields) ------------------------ */

/* LeeRouter::route_one_with_buf, crates/mr-cpu/src/lee.rs:39-65. */
uint32_t orc_lee_route_one(const orc_grid *g, const orc_net *net, uint32_t *path, uint32_t cap,
                           uint32_t *cost_out);
/* dijkstra (first-writer) field, crates/mr-cpu/src/dijkstra.rs:70-115, as used by
 * bfs_distance_field (crates/mr-cpu/src/sweep.rs:143-148). */
void orc_bfs_distance_field(const orc_grid *g, uint32_t src, uint32_t *dist);
/* sweep_distance_field, crates/mr-cpu/src/sweep.rs:64-139. */
void orc_sweep_distance_field(const orc_grid *g, uint32_t src, uint32_t *dist);
/* path_from_field, crates/mr-cpu/src/sweep.rs:158-235. */
uint32_t orc_path_from_field(const orc_grid *g, const uint32_t *dist, uint32_t src, uint32_t dst,
                             uint32_t *path, uint32_t cap);

/* --- boundary validation --------------------------------------------------- */

/* provider_path_is_valid, crates/mr-cpu/src/negotiated.rs:1284-1331, with the via
 * model given as the request's via_allowed vector. */
int orc_provider_path_is_valid(const orc_grid *g, const uint8_t *via_allowed, const orc_net *net,
                               const uint32_t *path, uint32_t len);

#ifdef __cplusplus
}
#endif
#endif
