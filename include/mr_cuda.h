/*
 * mr_cuda.h — C ABI of the B200 batched shortest-path engine for metalroute.
 *
 * Plain pointers and sizes only; no CUDA or torch types cross this boundary
 * (streams travel as `void *` holding a cudaStream_t).  Every entry point is
 * all-or-error: on a non-zero status no result object is produced and
 * mrc_last_error() describes the failure.  Nothing here ever falls back to a
 * CPU search; the caller (metalroute's NegotiatedRouter) owns that fallback,
 * exactly as with its Metal provider.
 *
 * Reference interfaces replaced (paths relative to the metal-route project):
 *   - IsolatedRouteProvider::route_isolated_batch
 *       crates/mr-cpu/src/negotiated.rs:554-560 (request :521-537, window :489-519)
 *     as adapted by MetalIsolatedProvider, crates/mr-cli/src/lib.rs:549-625
 *   - metal_route_isolated_batch / metal_route_isolated_batch_ragged
 *       crates/mr-metal/src/lib.rs:414-558, 695-984
 *   - metal_sweep_fields / metal_wavefront_field
 *       crates/mr-metal/src/lib.rs:128-204
 *   - MetalRouter::route (Router contract), crates/mr-metal/src/lib.rs:1143-1235,
 *     and LeeRouter::route, crates/mr-cpu/src/lee.rs:68-110
 *
 * Data contract (crates/mr-core/src/lib.rs): Cost = uint32, OBSTACLE =
 * 0xFFFFFFFF, CellIdx = uint32 with idx3(x, y, l) = (l*h + y)*w + x,
 * board_constraint bits = Grid::BOARD_* (lib.rs:411-416).
 * Canonical labels: (search cost, minimum hops, lowest predecessor CellIdx).
 */
#ifndef MR_CUDA_H
#define MR_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MRC_ABI_VERSION 1u
#define MRC_NO_PATH 0xFFFFFFFFu

/* Status codes.  RouterError (crates/mr-core/src/lib.rs:698-708) maps onto
 * MRC_ERR_MALFORMED_GRID, MRC_ERR_INVALID_ENDPOINT and, for everything the
 * Metal provider reports as BackendUnavailable, the remaining codes. */
typedef enum {
    MRC_OK = 0,
    MRC_ERR_INVALID_ARGUMENT = 1,    /* null pointer, shape mismatch, bad window */
    MRC_ERR_MALFORMED_GRID = 2,      /* cost/mask lengths do not match dims */
    MRC_ERR_INVALID_ENDPOINT = 3,    /* endpoint/pad out of bounds, foreign obstacle, board node */
    MRC_ERR_BACKEND_UNAVAILABLE = 4, /* no CUDA device, launch or copy failure */
    MRC_ERR_BUSY = 5,                /* context in use and MRC_FLAG_NO_WAIT given */
    MRC_ERR_ITERATION_LIMIT = 6,     /* a device loop hit its bound; nothing returned */
    MRC_ERR_OUT_OF_MEMORY = 7,       /* device or host allocation failed */
    MRC_ERR_LIMIT = 8                /* request exceeds a documented size limit */
} mrc_status;

/* Request flags. */
#define MRC_FLAG_RETRY_FULL 0x1u  /* unreachable-in-window nets are re-solved on the full board */
#define MRC_FLAG_KEEP_FIELDS 0x2u /* return each net's u32 distance field over its solved window */
#define MRC_FLAG_NO_WAIT 0x4u     /* fail with MRC_ERR_BUSY instead of waiting for the context */
#define MRC_FLAG_TIME_KERNELS 0x8u /* batches record CUDA events around their relax kernel */

typedef struct mrc_context mrc_context;
typedef struct mrc_result mrc_result;
typedef struct mrc_board mrc_board;
typedef struct mrc_batch mrc_batch;

/* Grid (crates/mr-core/src/lib.rs:393-408).  board_constraint and via_forbidden
 * may be NULL (the reference's empty vectors). via_forbidden holds 0/1 bytes. */
typedef struct {
    uint32_t w, h, layers;
    const uint32_t *cost;
    const uint8_t *board_constraint;
    const uint8_t *via_forbidden;
} mrc_grid;

/* NetEndpoints (crates/mr-core/src/lib.rs:519-537); the name stays with the caller. */
typedef struct {
    uint32_t src, dst;
    const uint32_t *passable_pads;
    uint32_t n_passable_pads;
    const uint32_t *via_passable_pads;
    uint32_t n_via_passable_pads;
} mrc_net;

/* IsolatedRouteWindow (crates/mr-cpu/src/negotiated.rs:494-500), inclusive. */
typedef struct {
    uint32_t x0, y0, x1, y1;
} mrc_window;

/* Already-rounded static edge prices (negotiated.rs:521-537).  The reference's
 * `via_edge_costs: &[Option<Cost>]` is split into via_edge_costs + via_allowed
 * (0 = None), as mr-metal does (crates/mr-metal/src/lib.rs:484-493).
 * directed_in_costs (nullable) is this engine's superset form: 4 base prices per
 * cell for the planar in-edges from its -y, -x, +x, +y neighbours, 0xFFFFFFFF =
 * blocked edge; when given it replaces the per-axis gap price.  A planar or via
 * step u->v costs min(base * enter(v), 0xFFFFFFFE) where enter(v) is 1 for an
 * obstacle that is one of the net's own passable pads and cost[v] otherwise. */
typedef struct {
    const uint32_t *x_edge_costs;   /* w-1 */
    uint32_t n_x_edge_costs;
    const uint32_t *y_edge_costs;   /* h-1 */
    uint32_t n_y_edge_costs;
    const uint32_t *via_edge_costs; /* layers-1 */
    const uint8_t *via_allowed;     /* layers-1 */
    uint32_t n_via_edge_costs;
    const uint32_t *directed_in_costs; /* nullable, 4*w*h*layers */
} mrc_edges;

/* IsolatedRouteRequest (negotiated.rs:529-537). */
typedef struct {
    const mrc_grid *grid;
    const mrc_net *nets;
    uint32_t n_nets;
    const mrc_window *windows; /* n_nets */
    mrc_edges edges;
} mrc_isolated_request;

/* ---- context -------------------------------------------------------------- */

/* One context per process per device; thread-safe (calls serialise on it).
 * Mirrors the process-global Metal context, crates/mr-metal/src/gpu.rs:865-878. */
mrc_status mrc_context_create(int device, mrc_context **out);
void mrc_context_destroy(mrc_context *ctx);
/* Last error message of the calling thread's most recent failed call on ctx. */
const char *mrc_last_error(const mrc_context *ctx);
uint32_t mrc_abi_version(void);

/* Page-locked host memory, mapped into every device's address space.  Board
 * arrays (cost, masks, directed prices) held here are read in place by one
 * gather launch in mrc_route_instances instead of being staged, and reach HBM
 * at full link rate in the single-board calls.  Ordinary (pageable) arrays
 * stay accepted everywhere. */
mrc_status mrc_host_alloc(mrc_context *ctx, size_t bytes, void **out);
void mrc_host_free(void *p);
/* Board bytes (cost, masks, directed prices) moved to HBM by this context so
 * far: through a staging copy, and read in place from page-locked arrays. */
mrc_status mrc_upload_stats(mrc_context *ctx, uint64_t *staged_bytes, uint64_t *in_place_bytes);

/* ---- the provider seam ------------------------------------------------------ */

/* Solve an isolated batch: per net, the canonical path inside its window and,
 * with MRC_FLAG_RETRY_FULL, a full-board re-solve of every net that was
 * unreachable in its window (IsolatedRouteProvider contract,
 * negotiated.rs:539-553; MetalIsolatedProvider retry, cli/src/lib.rs:574-607).
 * Without the flag this is metal_route_isolated_batch (metal/src/lib.rs:398-412).
 * Validation and its errors follow metal/src/lib.rs:433-467 and
 * negotiated.rs:1392-1407. */
mrc_status mrc_route_isolated_batch(mrc_context *ctx, const mrc_isolated_request *req, uint32_t flags,
                                    mrc_result **out);

/* ---- Router contract and plain fields (LeeRouter / MetalRouter / sweep fields) */

/* LeeRouter::route / MetalRouter::route: every net on the whole board, planar
 * moves only, step cost = enter cost of the destination (lee.rs:39-65), board
 * masks honoured.  Unreachable nets get search cost MRC_NO_PATH. */
mrc_status mrc_route_lee(mrc_context *ctx, const mrc_grid *grid, const mrc_net *nets, uint32_t n_nets,
                         mrc_result **out);

/* bfs_distance_field / metal_sweep_fields: one complete u32 field per source
 * (sweep.rs:143-148, metal/src/lib.rs:166-192) written to fields[i*n_cells ..].
 * An out-of-range, obstacle or board-forbidden source yields an all-0xFFFFFFFF
 * field (metal/src/lib.rs:1500-1520). */
mrc_status mrc_distance_fields(mrc_context *ctx, const mrc_grid *grid, const uint32_t *sources, uint32_t n_sources,
                               uint32_t *fields);

/* Many independent instances (each its own board, nets and windows; layer
 * counts may differ) solved in ONE persistent launch.  Results are concatenated
 * in instance order: the nets of instance k follow those of instance k-1.  The
 * retry, when flagged, re-solves a net on its own instance's full board. */
mrc_status mrc_route_instances(mrc_context *ctx, const mrc_isolated_request *instances, uint32_t n_instances,
                               uint32_t flags, mrc_result **out);

/* ---- results ---------------------------------------------------------------- */

uint32_t mrc_result_count(const mrc_result *r);
/* CSR paths: cells of net i are cells[offsets[i] .. offsets[i+1]) as global CellIdx. */
const uint64_t *mrc_result_path_offsets(const mrc_result *r);
const uint32_t *mrc_result_path_cells(const mrc_result *r);
/* Fixed-point search cost per net (MetalIsolatedRoute::search_cost), MRC_NO_PATH if none. */
const uint32_t *mrc_result_search_costs(const mrc_result *r);
/* With MRC_FLAG_KEEP_FIELDS: net i's field covers window windows[i] (the full
 * board when its retry ran), laid out (l, y-y0, x-x0) row-major, at
 * fields[field_offsets[i] ..].  NULL otherwise. */
const uint64_t *mrc_result_field_offsets(const mrc_result *r);
const uint32_t *mrc_result_fields(const mrc_result *r);
const mrc_window *mrc_result_field_windows(const mrc_result *r);
/* Number of nets that needed the full-board retry. */
uint32_t mrc_result_retried(const mrc_result *r);
void mrc_result_free(mrc_result *r);

/* ---- device-resident boards and prepared batches -------------------------- */

/* Upload a board once (cost, masks, edge prices) and keep it in HBM. */
mrc_status mrc_board_create(mrc_context *ctx, const mrc_grid *grid, const mrc_edges *edges, mrc_board **out);
void mrc_board_destroy(mrc_board *board);

/* Validate and stage a batch of nets against a resident board (descriptors,
 * pads and label storage in HBM).  Windows may be NULL: each net then gets
 * net_window (negotiated.rs:568-594). */
mrc_status mrc_batch_create(mrc_context *ctx, const mrc_board *board, const mrc_net *nets, uint32_t n_nets,
                            const mrc_window *windows, uint32_t flags, mrc_batch **out);
/* A batch over several resident boards: net i belongs to boards[net_board[i]]. */
mrc_status mrc_batch_create_multi(mrc_context *ctx, const mrc_board *const *boards, uint32_t n_boards,
                                  const mrc_net *nets, const uint32_t *net_board, uint32_t n_nets,
                                  const mrc_window *windows, uint32_t flags, mrc_batch **out);
/* Capture the batch's launch sequence (resets, relax, path kernels) into a CUDA
 * graph; later mrc_batch_launch calls replay it with one cudaGraphLaunch. */
mrc_status mrc_batch_capture_graph(mrc_context *ctx, mrc_batch *batch);
/* Enqueue the whole window solve (fields + canonical paths) on `stream`
 * (a cudaStream_t, NULL = the context's stream) without any host sync. */
mrc_status mrc_batch_launch(mrc_context *ctx, mrc_batch *batch, void *stream);
/* Wait for the batch, run the full-board retry if flagged, copy results out. */
mrc_status mrc_batch_finish(mrc_context *ctx, mrc_batch *batch, mrc_result **out);
/* Autotuner: time every relax configuration (tile height 8/16/32/64 cells,
 * 128 or 256 threads per CTA, and with them the CTAs per SM) on this batch,
 * keep the fastest for the batch, and cache it in the context for later batches
 * with the same layer count and price form.  Outputs may be NULL. */
mrc_status mrc_batch_autotune(mrc_context *ctx, mrc_batch *batch, uint32_t *tile_h, uint32_t *threads,
                              float *best_ms);
/* Force a relax configuration on a batch: tile height in {8, 16, 32, 64} cells
 * and 128 or 256 threads per CTA.  MRC_ERR_LIMIT when the tile does not fit. */
mrc_status mrc_batch_set_config(mrc_context *ctx, mrc_batch *batch, uint32_t tile_h, uint32_t threads);
/* The relax schedule: 0 = bulk-synchronous rounds over a shared tile list
 * (cooperative launch, grid barrier between rounds); 1 = one asynchronous
 * work queue (no rounds; a tile held by one CTA at a time), step prices brought
 * to each tile by one TMA load from per-board price planes computed once per
 * launch; 2 = the same queue with one warp per tile (tiles of 4 S x 8 cells
 * over every layer, S = 32 / next_pow2(layers), labels in shared memory;
 * boards of at most 16 layers, else MRC_ERR_LIMIT; a batch whose nets carry
 * negotiation price overrides runs 1 instead); 3 = the queue of 1 with step
 * prices formed per tile from the staged board words (no planes).  All give
 * the same labels and paths.  The autotuner tries every one.  These replace
 * the per-round dispatch loop of crates/mr-metal/src/gpu.rs:1630-2039. */
mrc_status mrc_batch_set_schedule(mrc_context *ctx, mrc_batch *batch, uint32_t schedule);
/* Schedule of batches built on this context while it holds no autotuned
 * configuration for their layer count and price form: 0, 1 (the default), 2
 * or 3 (see mrc_batch_set_schedule); with 2, batches with more than 16 layers
 * run 1. */
mrc_status mrc_context_set_schedule(mrc_context *ctx, uint32_t schedule);
/* The batch's current tile height, CTA width and schedule. */
mrc_status mrc_batch_config(const mrc_batch *batch, uint32_t *tile_h, uint32_t *threads, uint32_t *schedule);
/* Kernels launched by the last mrc_batch_launch (for launch accounting). */
uint32_t mrc_batch_kernel_launches(const mrc_batch *batch);
/* Device milliseconds of the relax kernel of the last launch, from CUDA events
 * recorded on the launching stream (batch created with MRC_FLAG_TIME_KERNELS;
 * call after the stream has been synchronised).  Negative when unavailable. */
float mrc_batch_relax_ms(const mrc_batch *batch);
/* Work counters of the last launch (after the stream has been synchronised):
 * out[0] = tile activations, out[1] = in-tile sweeps (passes of the warp
 * schedule), out[2] = rounds (tile rows relaxed, warp schedule),
 * out[3] = tiles in the batch.  Returns MRC_ERR_BACKEND_UNAVAILABLE if the
 * counters cannot be read. */
mrc_status mrc_batch_stats(const mrc_batch *batch, uint64_t out[4]);
/* Cells in all windows of the batch (the per-launch work unit). */
uint64_t mrc_batch_window_cells(const mrc_batch *batch);
void mrc_batch_destroy(mrc_batch *batch);

/* ---- the plain form (one net per launch sequence) --------------------------- */

/* The reference's plain GPU method restated on CUDA: per net, Jacobi relaxation
 * rounds of one thread per window cell, each round followed by a host read of
 * the changed flag (crates/mr-metal/src/gpu.rs:22-87,1242-1303 for the planar
 * wavefront, extended here to the isolated edge/via model).  Same results as
 * mrc_route_isolated_batch; kept as the baseline the batched engine is
 * measured against. */
mrc_status mrc_route_isolated_plain(mrc_context *ctx, const mrc_isolated_request *req, uint32_t flags,
                                    mrc_result **out);

/* ---- no device allocation --------------------------------------------------- */

/* Bytes of the one file-scope device array that backs every scratch buffer of
 * mrc_route_isolated_batch_noalloc.  Each GPU that loads the library holds this
 * much device memory until the process exits. */
#define MRC_NOALLOC_SCRATCH_BYTES (64u << 20)

/* Window solve of an isolated batch (the semantics of mrc_route_isolated_batch
 * without MRC_FLAG_RETRY_FULL) that never allocates device memory.  This entry
 * point has no counterpart in the reference.
 *
 * Who needs it: a caller that cannot call cudaMalloc — a long-running router
 * process that hands nearly all of HBM to its own allocator at start-up (a
 * PyTorch caching allocator, an arena shared by several engines) and has
 * nothing left for cudaMalloc, or a caller on a latency-critical path where
 * cudaMalloc/cudaFree, which can synchronise the whole device, are not allowed.
 * The caller passes the request and the host output buffers; all device
 * scratch (board copy, descriptors, labels, tile lists, outputs before their
 * download) is carved from MRC_NOALLOC_SCRATCH_BYTES of static device memory.
 *
 * - Runs on the calling thread's current device, on `stream` (a cudaStream_t;
 *   NULL = the legacy default stream), and returns after the results are on the
 *   host.
 * - The first call on a device looks the scratch array up (once per device);
 *   make that first call before any stream capture.
 * - A request whose scratch would exceed MRC_NOALLOC_SCRATCH_BYTES (8 B per
 *   window cell for labels plus 4 B per window cell for paths, the board copy,
 *   and per-tile state) fails with MRC_ERR_LIMIT and does no device work.
 * - The array is per process and per device, and all calls in a process share
 *   it and find the previous call's contents in it; the entry point clears what
 *   must start at zero.  Calls serialise on a process-wide lock, and every call
 *   (an error return included) waits for its own device work before it returns.
 *   Calls that overlapped on the GPU would race on the array; the lock and the
 *   wait are what keep them from overlapping.
 * - path_offsets[n+1] and search_costs[n] are always written on success; when
 *   the paths need more than path_cells_capacity cells the call returns
 *   MRC_ERR_LIMIT with the offsets filled so the caller can size the buffer. */
mrc_status mrc_route_isolated_batch_noalloc(const mrc_isolated_request *req, void *stream, uint32_t *search_costs,
                                            uint64_t *path_offsets, uint32_t *path_cells,
                                            uint64_t path_cells_capacity);

/* ---- snapshot negotiation rounds -------------------------------------------- */

/* One negotiation round on a frozen price snapshot, on the device: the Jacobi
 * iteration of NegotiatedRouter (crates/mr-cpu/src/negotiated.rs:1610-1991)
 * with occupancy and history kept per directed planar edge slot instead of per
 * cell.  Each round:
 *   1. dirty set: round 0 every net; later, every net that is unrouted or whose
 *      path uses a planar edge that two or more nets used after the previous
 *      round (the reference's prev_overused test, :1632-1642);
 *   2. rip-up: the dirty nets' old paths leave `present`;
 *   3. snapshot: price(slot) = base == 0xFFFFFFFF ? 0xFFFFFFFF
 *        : min(base + history + pfac * present_weight * present, 0xFFFFFFFE),
 *      pfac = 1 + round (priced_with_base :2768-2795, passable_search_cost);
 *   4. every dirty net is solved alone on the snapshot (the isolated batch:
 *      window, then full-board retry, canonical paths);
 *   5. merge: the new paths enter `present` (unrouted nets contribute nothing);
 *   6. history += history_step on every slot whose edge two or more nets use
 *      (:1929-1948), then the next dirty set is computed.
 * The snapshot is the request's directed in-price plane, so the cell enter
 * weight multiplies the whole price; with unit enter weights (the negotiation
 * boards) this is the reference's base*enter + congestion.  Slots of an
 * undirected edge {a, b}: b's slot "from a" and a's slot "from b", both counted.
 * This entry point has no single counterpart in the reference (its rounds run
 * on the CPU); the round semantics above are the reference's, on edges. */
typedef struct mrc_negotiation mrc_negotiation;

typedef struct {
    uint32_t present_weight; /* SCALE in the reference: 16 */
    uint32_t history_step;   /* added per overused edge and round */
} mrc_negotiation_params;

typedef struct {
    uint32_t round, pfac;
    uint32_t dirty;           /* nets routed this round */
    uint32_t routed;          /* of those, reached their target */
    uint32_t retried;         /* of those, needed the full-board retry */
    uint32_t next_dirty;      /* nets the next round will route */
    uint64_t overused_edges;  /* undirected planar edges used by >= 2 nets after the merge */
    uint64_t window_cells;    /* cells solved (windows + retries) */
    uint64_t path_cells;      /* cells on the current paths of all nets */
    float round_ms;           /* device-timeline time of the round on the engine stream */
} mrc_round_stats;

/* The request gives the board (grid, edges), the nets and their windows.  Base
 * planar prices come from edges.directed_in_costs or, when it is NULL, from the
 * per-axis prices (in-price from -x at x = x_edge_costs[x-1], and so on). */
mrc_status mrc_negotiation_create(mrc_context *ctx, const mrc_isolated_request *req,
                                  const mrc_negotiation_params *params, mrc_negotiation **out);
/* Runs the next round.  A round with no dirty net does nothing (converged). */
mrc_status mrc_negotiation_round(mrc_context *ctx, mrc_negotiation *neg, mrc_round_stats *stats);

/* Connection groups (the reference's connection_group_ids,
 * crates/mr-cpu/src/negotiated.rs:929-989, and its group-aware overuse scan,
 * :1923-1943): nets of one group may share edges.  With groups set, an edge is
 * overused when nets of two or more distinct groups use it; history, the
 * overused count and the next dirty set follow that test (occupancy prices are
 * unchanged: every net still pays for every other net's presence, as in
 * route_negotiated).  groups[i] is net i's group id (any value but 0xFFFFFFFF;
 * the reference's are dense first-appearance ids).  Called before the first
 * round; not on a shard, whose nets see only part of the paths.  Without this
 * call every net is its own group. */
mrc_status mrc_negotiation_set_groups(mrc_context *ctx, mrc_negotiation *neg, const uint32_t *groups);

/* Clearance-halo pricing: the reference's clearance-active snapshot iteration
 * (crates/mr-cpu/src/negotiated.rs:1565-1568 and :1610-1812 with
 * clearance_active, route_negotiated's pricing :2778-2797, footprints
 * for_each_halo_cell :3184-3271), on a uniform grid where a radius is a count of
 * cells.  The footprint of a path is the (2r+1)^2 box around every path cell on
 * its own layer (r = clearance_cells) and the box of radius
 * max(clearance_cells, via_keepout_cells) on both layers of every via, clipped
 * to the board, base obstacles skipped, counted with multiplicity; halo[c] is
 * the number of footprint visits of every net's current path on cell c.  With
 * a clearance set (either radius > 0) each round:
 *   - routes every net (until a round ends with no overused edge: then the
 *     dirty set is empty, the reference's convergence break);
 *   - rips nothing up before pricing: the snapshot holds every net's current
 *     path; the shared price is base + history + pfac * present_weight *
 *     present + pfac * halo_weight * halo[c] (capped at MAX - 1);
 *   - prices each net with its own contribution subtracted:
 *     base + history + pfac * present_weight * (present - own path slot)
 *     + pfac * halo_weight * (halo[c] - own footprint visits of c);
 *   - merges: every routed net's old path and footprint leave, its new ones
 *     enter (an unrouted net contributes nothing).
 * Overuse, history and groups are unchanged (copper only).  halo_weight is the
 * reference's CLEARANCE_NEG_WEIGHT (16).  Radii up to 255 cells; called before
 * the first round; not on a shard.  Both radii 0 turns it off. */
mrc_status mrc_negotiation_set_clearance(mrc_context *ctx, mrc_negotiation *neg, uint32_t clearance_cells,
                                         uint32_t via_keepout_cells, uint32_t halo_weight);
/* Copies halo[c] (one u32 per cell) to a host buffer (a clearance must be set). */
mrc_status mrc_negotiation_read_halo(mrc_context *ctx, mrc_negotiation *neg, uint32_t *halo);

/* Sharded rounds (one shard per GPU, each routing its own nets of the same
 * board).  A shard keeps the occupancy of its own paths ("local") and a global
 * occupancy that the caller sets to the sum of every shard's local one (an
 * all-reduce over NCCL, or a plain sum) between the phases of a round:
 *   ripup  -> global = sum(local) -> route -> global = sum(local) -> settle.
 * ripup takes this shard's dirty nets out of its local occupancy; route prices
 * the snapshot from the global occupancy and history, routes this shard's dirty
 * nets and merges them into the local occupancy; settle adds history on the
 * edges the global occupancy overuses (the same on every shard) and finds this
 * shard's next dirty nets.  The union of the shards' paths equals the paths of
 * one unsharded negotiation over all nets.  The unsharded object runs the same
 * three phases inside mrc_negotiation_round with its local occupancy as the
 * global one.  No counterpart in the reference (its rounds run on one host). */
mrc_status mrc_negotiation_create_shard(mrc_context *ctx, const mrc_isolated_request *req,
                                        const mrc_negotiation_params *params, const uint8_t *owned,
                                        mrc_negotiation **out);
mrc_status mrc_negotiation_ripup(mrc_context *ctx, mrc_negotiation *neg);
mrc_status mrc_negotiation_route(mrc_context *ctx, mrc_negotiation *neg, mrc_round_stats *stats);
mrc_status mrc_negotiation_settle(mrc_context *ctx, mrc_negotiation *neg, mrc_round_stats *stats);
/* Device addresses of the local and global occupancy (4 u32 per cell; the same
 * buffer for an unsharded object) and their size in bytes. */
mrc_status mrc_negotiation_buffers(mrc_negotiation *neg, void **local_present, void **global_present,
                                   uint64_t *bytes);
/* Current paths of every net (CSR, request order; an empty path = unrouted).
 * The pointers stay valid until the next round or destroy. */
mrc_status mrc_negotiation_paths(const mrc_negotiation *neg, uint32_t *n_nets, const uint64_t **offsets,
                                 const uint32_t **cells);
/* Copies 4 u32 per cell (slots -y, -x, +x, +y) of the occupancy, history and
 * the last snapshot's prices to host buffers; any of them may be NULL. */
mrc_status mrc_negotiation_read(mrc_context *ctx, mrc_negotiation *neg, uint32_t *present, uint32_t *history,
                                uint32_t *snapshot);
/* Nets the next round will route (ascending). */
mrc_status mrc_negotiation_dirty(const mrc_negotiation *neg, uint32_t *n, const uint32_t **nets);
void mrc_negotiation_destroy(mrc_negotiation *neg);

/* ---- serving: continuous batching behind the /solve seam --------------------- */

/* A request loop in front of the engine, for the reference's /solve route
 * (crates/mr-server/src/lib.rs:381-448, one synchronous solve per request on a
 * worker thread, no batching or admission).  Requests are submitted from any
 * thread and return at once with a ticket; one dispatcher thread
 *   - admits queued requests in arrival order while the device memory they
 *     need (boards, labels, paths, tile state) fits the HBM budget
 *     (hbm_fraction of the device's memory, minus what was in use at creation;
 *     the engine's own free cached blocks count as available),
 *   - merges every admitted request with the same flags, up to
 *     max_batch_requests / max_batch_cells, into ONE persistent launch over
 *     all of their boards (each request's board is uploaded into HBM and stays
 *     there while it is solved),
 *   - keeps up to `slots` such launches in flight on separate streams, each
 *     with 1/slots of the co-resident grid, so requests that arrive while
 *     others run are staged and launched beside them instead of queueing
 *     behind them,
 *   - reaps finished launches (with each request's full-board retry) and hands
 *     every request its own result.
 * A request's result is identical to mrc_route_isolated_batch on the same
 * request alone (bit for bit).  This entry point has no counterpart in the
 * reference. */
typedef struct mrc_server mrc_server;

typedef struct {
    float hbm_fraction;           /* admission budget, fraction of device memory (0.8) */
    uint32_t slots;               /* launches in flight at once (>= 1) */
    uint32_t max_batch_requests;  /* requests merged into one launch (>= 1) */
    uint64_t max_batch_cells;     /* window cells per launch (0 = no limit) */
    uint32_t max_layers;          /* largest layer count accepted (sizes the tile; <= 12) */
    uint32_t merge_ratio;         /* size-aware merging: a request joins a launch only when its window cells
                                   * are within this factor of the launch's first request, either way, so a
                                   * small request never waits in a launch that carries a much larger one
                                   * (0 = merge regardless of size) */
} mrc_server_params;

typedef struct {
    double queue_ms;              /* submit -> staged for launch */
    double run_ms;                /* launch -> results on the host */
    double total_ms;              /* submit -> results on the host */
    uint32_t batch_requests;      /* requests that shared its launch */
    uint32_t status;              /* mrc_status of this request */
    uint64_t batch_id;
} mrc_request_info;

mrc_status mrc_server_create(mrc_context *ctx, const mrc_server_params *params, mrc_server **out);
/* Validates the request and queues it.  The request's arrays (grid, edges,
 * nets, pads, windows) are BORROWED: they must stay valid and unchanged until
 * mrc_server_wait for this ticket has returned.  Flags: RETRY_FULL, KEEP_FIELDS. */
mrc_status mrc_server_submit(mrc_server *srv, const mrc_isolated_request *req, uint32_t flags, uint64_t *ticket);
/* The same against a board already resident in HBM (mrc_board_create): no
 * board upload.  The board, nets, pads and windows are borrowed until the
 * ticket's wait returns. */
mrc_status mrc_server_submit_resident(mrc_server *srv, const mrc_board *board, const mrc_net *nets, uint32_t n_nets,
                                      const mrc_window *windows, uint32_t flags, uint64_t *ticket);
/* Waits up to timeout_ms (0 = forever) for a ticket; on success hands over its
 * result (free with mrc_result_free).  MRC_ERR_BUSY = still running at the
 * timeout (the ticket stays valid); any other error is the request's own. */
mrc_status mrc_server_wait(mrc_server *srv, uint64_t ticket, uint32_t timeout_ms, mrc_result **out,
                           mrc_request_info *info);
/* out[0..7]: submitted, completed, failed, launches, largest launch (requests),
 * peak in-flight bytes, budget bytes, queued now. */
mrc_status mrc_server_stats(mrc_server *srv, uint64_t out[8]);
/* Finishes everything queued and in flight, then stops the dispatcher. */
void mrc_server_destroy(mrc_server *srv);

/* ---- self-test of the bounded device waits ---------------------------------- */

/* Launches one CTA that waits at the engine's grid barrier for a CTA that never
 * arrives.  The wait gives up after `spin_limit` polls and reports it; the call
 * returns MRC_OK with the kernel's status bits in *status (bit 4 = barrier wait
 * exceeded) and the device time in *elapsed_ms, and the context stays usable.
 * No counterpart in the reference (its Metal loop waits on the host). */
mrc_status mrc_selftest_wait_timeout(mrc_context *ctx, uint32_t spin_limit, uint32_t *status, float *elapsed_ms);

/* net_window (negotiated.rs:568-594) for a batch of nets. */
mrc_status mrc_net_windows(uint32_t w, uint32_t h, uint32_t layers, const mrc_net *nets, uint32_t n_nets,
                           mrc_window *out);

#ifdef __cplusplus
}
#endif
#endif
