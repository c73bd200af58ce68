// device.cuh — data layout and label arithmetic shared by every kernel.
//
// Semantics follow the reference's isolated ("alone path") search exactly:
//   step(u->v) planar = min(base(u,v) * enter(v), 0xFFFFFFFE)
//       base  = per-axis Hanan gap price (negotiated.rs:2921-2932) or, in the
//               directed superset form, the per-edge in-price of v
//       enter = 1 for an obstacle that is one of the net's own pads, else cost[v]
//               (enter_weight, negotiated.rs:2914-2920)
//   step(u->v) via    = min(via_edge[k] * enter(v), 0xFFFFFFFE)   (negotiated.rs:3010-3043)
//   blocked(v)        = outside window | board trace node | foreign obstacle
//                       (blocked_fn, negotiated.rs:2933-2966)
// Labels (dist, hops) are minimised lexicographically and packed into one
// u64 = dist << 32 | hops, so a plain unsigned compare is the reference's
// (cost, hop count) order (dijkstra.rs:298-325).  A dist that reaches
// 0xFFFFFFFF is unreachable, as in every reference field.
#pragma once

#include <cstdint>

namespace mrc {

typedef unsigned long long u64;

constexpr uint32_t kMax = 0xFFFFFFFFu;      // OBSTACLE / unreachable / blocked step
constexpr uint32_t kCap = 0xFFFFFFFEu;      // passable_search_cost cap
constexpr u64 kInf = 0xFFFFFFFFFFFFFFFFull; // unreachable label

// Per-cell board flag byte (host combines Grid::board_constraint and
// Grid::via_forbidden into one array).
constexpr uint8_t kTraceNode = 1u << 0;   // Grid::BOARD_TRACE_NODE
constexpr uint8_t kViaNode = 1u << 1;     // Grid::BOARD_VIA_NODE
constexpr uint8_t kEdgeNegY = 1u << 2;    // Grid::BOARD_EDGE_NEG_Y
constexpr uint8_t kEdgeNegX = 1u << 3;    // Grid::BOARD_EDGE_NEG_X
constexpr uint8_t kEdgePosX = 1u << 4;    // Grid::BOARD_EDGE_POS_X
constexpr uint8_t kEdgePosY = 1u << 5;    // Grid::BOARD_EDGE_POS_Y
constexpr uint8_t kStaticVia = 1u << 6;   // Grid::via_forbidden (exemptible by via pads)
// In the per-tile shared copy bit 6 instead means "no via may touch this node"
// (board via node, or static via mask without the net's exemption).
constexpr uint8_t kViaBlocked = 1u << 6;

struct DevBoard {
    uint32_t w, h, layers;
    uint32_t via_mask;          // bit k: the k <-> k+1 transition is allowed
    const uint32_t *cost;       // w*h*layers
    const uint8_t *flags;       // nullable
    const uint32_t *x_edge;     // w-1 (at least one element)
    const uint32_t *y_edge;     // h-1
    const uint32_t *via_edge;   // layers-1
    const uint4 *directed;      // nullable: in-prices from -y, -x, +x, +y
    uint32_t *planes;           // nullable: 6 planes of step prices, rows padded (written by planes_kernel)
    const void *tmap;           // nullable: TMA tensor map (CUtensorMap, 64-byte aligned) over `planes`
    // nullable: per-field directed in-price overrides (the negotiation's prices
    // with each net's own path and clearance footprint subtracted), sorted by
    // cell inside each field's range DevField::over_off .. + n_over
    const uint32_t *over_cells;
    const uint4 *over_price;
};

// One field = one net solved inside one window.
struct DevField {
    uint32_t src, dst;          // global CellIdx
    uint32_t x0, y0, ww, wh;    // window origin and extent
    uint64_t lab_off;           // first cell of this field in the label arena
    uint32_t pad_off, n_pads;   // sorted own pads in the pad arena
    uint32_t vpad_off, n_vpads; // sorted via exemptions in the pad arena
    uint32_t out;               // output slot (the net's request index)
    uint32_t tile_off;          // first tile of this field in the tile-state arrays
    uint32_t board;             // index of this field's board in the batch's board array
    uint32_t n_over;            // directed-price overrides of this field (DevBoard::over_cells)
    uint32_t over_off;
    uint32_t pad_;
};

// Control block of one batch launch (device memory, zeroed before launch).
// The words that workers update atomically on every item (the list counts,
// the consumption cursors) and the words idle workers poll (status) sit on
// their own 128-byte lines, so polling never queues behind the atomics.
struct Ctl {
    uint32_t count[3];          // items in the three rotating tile lists (queue form: [0] tail, [1] in flight)
    uint32_t pad_count[29];
    uint32_t head[3];           // consumption cursors
    uint32_t pad_head[29];
    uint32_t bar_count, bar_gen;
    uint32_t pad_bar[30];
    uint32_t status;
    uint32_t rounds;
    uint32_t pad_status[30];
    unsigned long long activations;
    unsigned long long sweeps;
    unsigned long long rows;    // tile rows relaxed (warp schedule)
};

__device__ __forceinline__ uint32_t capmul(uint32_t e, uint32_t w) {
    u64 p = (u64)e * (u64)w;
    return p > (u64)kCap ? kCap : (uint32_t)p;
}

// Candidate label for v reached from a label `prev` over a step of `step`
// (kMax = blocked).  Saturation to 0xFFFFFFFF is unreachable.
__device__ __forceinline__ u64 extend(u64 prev, uint32_t step) {
    uint32_t d = (uint32_t)(prev >> 32);
    uint32_t nd = d + step;
    bool bad = (d == kMax) | (step == kMax) | (nd < d) | (nd == kMax);
    return bad ? kInf : (((u64)nd << 32) | (uint32_t)((uint32_t)prev + 1u));
}

__device__ __forceinline__ bool sorted_has(const uint32_t *a, uint32_t n, uint32_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t v = a[mid];
        if (v < key) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && a[lo] == key;
}

// First index of a sorted list whose entry is >= key.
__device__ __forceinline__ uint32_t over_lower_bound(const uint32_t *a, uint32_t n, uint32_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Directed in-price slot s (0 from -y, 1 from -x, 2 from +x, 3 from +y) of
// cell c as field f sees it: the field's own override at c when it has one,
// else the board's plane (which must be present).
__device__ __forceinline__ uint32_t field_directed(const DevBoard &b, const DevField &f, uint32_t c, int s) {
    if (f.n_over) {
        const uint32_t *oc = b.over_cells + f.over_off;
        const uint32_t lo = over_lower_bound(oc, f.n_over, c);
        if (lo < f.n_over && __ldg(oc + lo) == c)
            return __ldg(reinterpret_cast<const uint32_t *>(b.over_price + f.over_off + lo) + s);
    }
    return __ldg(reinterpret_cast<const uint32_t *>(b.directed + c) + s);
}

// enter weight of a cell inside the window, kMax when the node is blocked.
__device__ __forceinline__ uint32_t cell_enter(const DevBoard &b, const DevField &f, const uint32_t *pads,
                                               uint32_t gcell, uint8_t flags) {
    if (flags & kTraceNode) return kMax;
    uint32_t c = __ldg(b.cost + gcell);
    if (c != kMax) return c;
    // Own pads (and the endpoints, which validation guarantees are own pads
    // whenever they are obstacles) are entered at weight 1.
    if (gcell == f.src || gcell == f.dst || sorted_has(pads + f.pad_off, f.n_pads, gcell)) return 1;
    return kMax;
}

// Shared-tile flag byte: directed board edge bits plus kViaBlocked.
__device__ __forceinline__ uint8_t cell_tile_flags(const DevField &f, const uint32_t *pads, uint32_t gcell,
                                                   uint8_t flags) {
    uint8_t t = flags & (kEdgeNegY | kEdgeNegX | kEdgePosX | kEdgePosY);
    bool vb = (flags & kViaNode) != 0;
    if (!vb && (flags & kStaticVia)) vb = !sorted_has(pads + f.vpad_off, f.n_vpads, gcell);
    return t | (vb ? kViaBlocked : 0);
}

}  // namespace mrc
