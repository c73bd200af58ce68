// kernels.h — launch interface between the host runtime and relax.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "device.cuh"

namespace mrc {

constexpr int kRelaxThreads = 256;  // default CTA width of the relax kernel
constexpr uint64_t kTilesPerCta = 8;  // tiles per CTA at which a queue launch can use one more CTA
constexpr uint32_t kCountBatch = 64;    // activations a queue CTA counts locally before adding them to the launch's
constexpr uint32_t kContinueLimit = 4;  // activations of one held tile before it goes back to the queue

// Status bits reported through Ctl::status / PathArgs::status.
constexpr uint32_t kStatusActivationLimit = 1u << 0;
constexpr uint32_t kStatusRoundLimit = 1u << 1;
constexpr uint32_t kStatusPathBroken = 1u << 2;
constexpr uint32_t kStatusQueueOverflow = 1u << 3;
constexpr uint32_t kStatusBarrier = 1u << 4;

struct RelaxArgs {
    const DevBoard *boards;     // device array, indexed by DevField::board
    uint32_t max_layers;        // the largest layer count among the boards (sizes the tile)
    const DevField *fields;     // ascending lab_off
    uint32_t n_fields;
    const uint32_t *pads;       // sorted pad lists, indexed by DevField offsets
    u64 *lab;                   // label arena (dist << 32 | hops)
    uint32_t *tstamp;           // per tile: last round it was queued for, + 1 (zeroed)
    uint32_t *tvisit;           // per tile: labels valid (zeroed)
    const uint8_t *tover;       // nullable: per tile, 1 = its field has directed-price overrides inside it
    u64 *lists;                 // 3 rotating lists of (field << 32 | tile)
    uint32_t list_cap;          // total tiles of the batch
    Ctl *ctl;                   // zeroed before launch
    uint32_t tile_h;            // 32, 16 or 8
    uint32_t round_limit;       // guard on the number of rounds
    unsigned long long activation_limit;  // guard on tile activations (asynchronous form)
};

struct PathArgs {
    const DevBoard *boards;
    const DevField *fields;
    uint32_t n_fields;
    const uint32_t *pads;
    const u64 *lab;
    const uint32_t *tvisit;
    const uint8_t *tover;            // nullable: as RelaxArgs::tover
    uint32_t tile_h;
    uint32_t arena_filled;           // 1: the label arena was +inf-filled (queue schedule), tvisit not needed
    uint32_t walk_smem;              // > 0: the tile-staged walk (price planes + TMA maps, no overrides), its smem
    uint32_t *costs;                 // [n] by output slot
    uint32_t *lens;                  // [n] by output slot
    unsigned long long *offsets;     // [n+1] by output slot
    uint32_t *cells;                 // path arena
    uint32_t *status;
};

struct PlainArgs {
    DevBoard board;
    DevField field;
    const uint32_t *pads;
    const u64 *in;
    u64 *out;
    uint32_t *changed;
};

// Snapshot negotiation (negotiate.cu).  Occupancy / history / prices are
// uint4 per cell over the directed planar in-edge slots (-y, -x, +x, +y).
struct OccupancyArgs {
    const unsigned long long *offsets;  // path CSR of every net
    const uint32_t *cells;
    const uint32_t *list;               // nets to apply (nullable = nets 0..n_list-1)
    uint32_t n_list;
    uint32_t w, plane;
    uint32_t *present;                  // 4 per cell
    bool add;                           // add the paths (true) or rip them up (false)
};

struct SnapshotArgs {
    const uint4 *base, *present, *history;
    const uint32_t *halo;               // nullable: clearance footprints covering each cell
    uint4 *out;
    uint64_t n;                         // cells
    uint32_t pfac, weight, halo_weight;
};

// Clearance footprints (for_each_halo_cell, negotiated.rs:3184-3271, on a
// uniform grid): the (2r+1)^2 box around every path cell on its own layer and
// the box of radius vr = max(r, keepout) on both layers of every via, clipped
// to the board, base obstacles (cost == MAX) skipped, with multiplicity.
struct HaloArgs {
    const unsigned long long *offsets;  // path CSR of every net
    const uint32_t *cells;
    const uint32_t *list;               // nets to apply
    uint32_t n_list;
    uint32_t w, h, layers;
    const uint32_t *cost;               // base cell costs
    uint32_t r, vr;
    uint32_t *halo;                     // 1 per cell
    bool add;
};

// One entry per (listed net, visit): key = list index << 32 | cell, value = 1
// per footprint visit, or 1 << (24 + slot) for each in-edge slot of the cell
// that the net's own path uses.  A visit outside the board or onto an obstacle
// emits the key kNoKey.  The host lays the entries of list index j out from
// emit_off[j]: path cells x (2r+1)^2 boxes, then the path cells, then 2 boxes
// of (2vr+1)^2 per via (via_k: the path index k of each via step k -> k+1).
constexpr unsigned long long kNoKey = ~0ull;
constexpr uint32_t kOwnHaloMask = 0x00FFFFFFu;  // footprint visits of one net on one cell stay below 2^24
constexpr uint32_t kMaxClearanceCells = 255;      // ... for radii up to this many cells
struct EmitArgs {
    const unsigned long long *offsets;  // path CSR of every net
    const uint32_t *cells;
    const uint32_t *list;
    uint32_t n_list;
    const unsigned long long *emit_off; // n_list + 1
    const unsigned long long *via_off;  // n_list + 1, into via_k
    const uint32_t *via_k;
    uint32_t w, h, layers;
    const uint32_t *cost;
    uint32_t r, vr;
    unsigned long long *keys;
    uint32_t *vals;
};

// Overrides from the reduced (key, value) runs: for run i the net's own price
// of every slot of the cell, base == MAX ? MAX : min(base + history
// + pf * (present - own_slot) + hf * (halo - own_halo), MAX - 1), and the range
// of each list index (range[2 j], range[2 j + 1]; zeroed before).
struct OverrideArgs {
    const unsigned long long *keys;
    const uint32_t *vals;
    const uint32_t *n_runs;             // device count of runs
    uint64_t cap;                       // launch bound on runs
    const uint4 *base, *present, *history;
    const uint32_t *halo;
    uint64_t pf, hf;                    // pfac * present weight, pfac * halo weight
    uint32_t *out_cells;
    uint4 *out_price;
    uint32_t *range;
};

struct OveruseArgs {
    const uint4 *present;
    const uint8_t *over;                // nullable: group-aware overuse flags, 4 per cell
    uint4 *history;
    uint64_t n;
    uint32_t step;
    unsigned long long *count;          // overused slots (2 per undirected edge)
};

struct DirtyArgs {
    const unsigned long long *offsets;
    const uint32_t *cells;
    uint32_t n_nets;
    uint32_t w, plane;
    const uint32_t *present;
    const uint8_t *over;                // nullable: group-aware overuse flags (else present >= 2)
    uint8_t *flags;                     // 1 = route again next round
};

constexpr uint32_t kNoGroup = 0xFFFFFFFFu;

struct GroupArgs {
    const unsigned long long *offsets;  // path CSR of every net
    const uint32_t *cells;
    const uint32_t *group;              // connection group of every net
    uint32_t n_nets;
    uint32_t w, plane;
    uint32_t *first;                    // 4 per cell: first group seen, kNoGroup before any
    uint8_t *over;                      // 4 per cell: 1 = used by two or more groups
};

cudaError_t occupancy_launch(const OccupancyArgs &a, cudaStream_t st);
cudaError_t snapshot_launch(const SnapshotArgs &a, cudaStream_t st);
cudaError_t overuse_launch(const OveruseArgs &a, cudaStream_t st);
cudaError_t dirty_launch(const DirtyArgs &a, cudaStream_t st);
cudaError_t group_overuse_launch(const GroupArgs &a, cudaStream_t st);
cudaError_t halo_launch(const HaloArgs &a, cudaStream_t st);
cudaError_t emit_launch(const EmitArgs &a, cudaStream_t st);
// Sort (keys, vals) by key and sum the values of equal keys into (run_keys,
// run_vals, *n_runs); temp is resized as needed (bytes in *temp_bytes).
cudaError_t footprint_reduce(const unsigned long long *keys, const uint32_t *vals, unsigned long long *keys_sorted,
                             uint32_t *vals_sorted, unsigned long long *run_keys, uint32_t *run_vals,
                             uint32_t *n_runs, uint64_t n, int end_bit, void *temp, size_t *temp_bytes,
                             cudaStream_t st);
cudaError_t override_launch(const OverrideArgs &a, cudaStream_t st);

// Warp schedule (warp_relax.cu): one warp per tile of (4 S) x 8 cells over all
// layers, S = 32 / next_pow2(layers) segments per row; boards of up to 16 layers.
constexpr uint32_t kWarpLaneCells = 4;
constexpr uint32_t kWarpTileH = 8;
constexpr uint32_t kWarpMaxLayers = 16;
__host__ __device__ inline uint32_t warp_segments(uint32_t layers) {
    uint32_t lp = 1;
    while (lp < layers) lp <<= 1;
    return 32u / lp;
}
__host__ __device__ inline uint32_t warp_tile_w(uint32_t layers) { return kWarpLaneCells * warp_segments(layers); }
uint32_t warp_relax_threads();
cudaError_t warp_relax_occupancy(int *blocks_per_sm);
// seeds, then the persistent warp kernel (label arena +inf-filled, queue tags zeroed, as for the queue form)
cudaError_t warp_relax_launch(const RelaxArgs &a, uint32_t grid, cudaStream_t st);
// Step-price planes of every board of a batch (DevBoard::planes, 6 x cells u32
// each); chunk_start[k] = first chunk of board k (prefix sum of planes_chunks).
// Columns of the TMA box that brings one tile's price planes to shared memory:
// the tile's 32 columns plus the slack of rounding its first column down to a
// multiple of 4 (16 bytes, the TMA rule for the innermost coordinate).
constexpr uint32_t kPlaneTmaBoxW = 36;
// Tile-staged path walk: tiles of 32 x walk_tile_rows cells over all layers,
// their price planes brought by TMA loads of the relax kernel's box.
constexpr uint32_t kWalkRows = 16;          // walk tile rows (at least the relax tile height)
constexpr size_t kWalkSmemLimit = 200u << 10;  // larger tiles take the per-step walk
__host__ __device__ inline uint32_t walk_tile_rows(uint32_t tile_h) { return tile_h > kWalkRows ? tile_h : kWalkRows; }
__host__ __device__ inline size_t walk_smem_planes(uint32_t layers, uint32_t tile_h) {
    return (size_t)(walk_tile_rows(tile_h) / tile_h) * 6 * layers * tile_h * kPlaneTmaBoxW * 4;
}
__host__ __device__ inline size_t walk_smem_bytes(uint32_t layers, uint32_t tile_h) {
    return walk_smem_planes(layers, tile_h) + (size_t)layers * (walk_tile_rows(tile_h) + 2) * 34 * 8;
}
// Rows of a price plane are padded to a multiple of 4 cells (16 bytes), so a
// tensor map over the planes has 16-byte strides.
__host__ __device__ inline uint32_t planes_pitch(uint32_t w) { return (w + 3u) & ~3u; }
uint64_t planes_chunks(uint64_t cells);
cudaError_t planes_launch(const DevBoard *boards, const uint64_t *chunk_start, uint32_t n_boards, uint64_t n_chunks,
                          uint32_t sms, cudaStream_t st);

// Shared memory of one tile of 32 x tile_h cells over `layers` (tile_h in {8, 16, 32, 64}); `planes`: the
// queue form that stages the step prices from the boards' price planes by TMA (DevBoard::planes, ::tmap).
size_t relax_smem_bytes(uint32_t layers, uint32_t tile_h, bool directed, bool planes = false);
// The relax kernel is instantiated for threads in {128, 256} per CTA.
// `async` selects the queue-driven form (relax_async_kernel) over the
// bulk-synchronous rounds (relax_rounds_kernel); the async form needs the label
// arena filled with 0xFF and the queue tags (lists[cap, 2 cap)) zeroed.
// over: the fields carry directed-price overrides (DevField::n_over); those
// kernels exist for kOverTileH-row tiles and kOverThreads threads only.
constexpr uint32_t kOverTileH = 8, kOverThreads = 256;
cudaError_t relax_configure(uint32_t tile_h, uint32_t threads, size_t smem, bool async = false, bool planes = false,
                            bool over = false);
cudaError_t relax_occupancy(uint32_t tile_h, uint32_t threads, size_t smem, int *blocks_per_sm, bool async = false,
                            bool planes = false, bool over = false);
cudaError_t relax_launch(const RelaxArgs &a, uint32_t grid, uint32_t threads, size_t smem, cudaStream_t st,
                         bool async = false, bool planes = false, bool over = false);
// tover[f.tile_off + t] = 1 for every tile t of every field that holds one of
// the field's directed-price overrides (tover zeroed before).
cudaError_t mark_over_tiles_launch(const DevField *fields, uint32_t n_fields, const DevBoard *boards, uint32_t tile_h,
                                   uint8_t *tover, cudaStream_t st);
cudaError_t path_launch(const PathArgs &a, cudaStream_t st);
cudaError_t fields_launch(const PathArgs &a, uint32_t *out, uint64_t total, cudaStream_t st);
cudaError_t plain_round_launch(const PlainArgs &a, uint64_t wcells, cudaStream_t st);
cudaError_t wait_selftest_launch(Ctl *c, uint32_t spins, cudaStream_t st);
cudaError_t combine_flags_launch(uint8_t *flags, const uint8_t *via_forbidden, uint64_t n, cudaStream_t st);

// A span of page-locked host memory (device-mapped address) copied into HBM.
// kind 0: dst = src (src may be null: zeros); kind 1: flag bytes, dst[i] =
// src[i] | (src2[i] ? kStaticVia : 0), either source may be null.
struct HostSpan {
    const void *src;
    const void *src2;
    void *dst;
    uint64_t bytes;
    uint32_t kind;
};
// chunk_start[s] = the first chunk of span s (prefix sum of host_gather_chunks)
cudaError_t host_gather_launch(const HostSpan *spans, const uint64_t *chunk_start, uint32_t n_spans, uint64_t n_chunks,
                               uint32_t sms, cudaStream_t st);
uint64_t host_gather_chunks(uint64_t bytes);

}  // namespace mrc
