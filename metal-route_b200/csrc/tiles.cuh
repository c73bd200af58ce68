// tiles.cuh — label arithmetic and the tile work queue shared by the relax kernels.
//
// Labels are u64 = dist << 32 | hops (device.cuh).  The queue is the
// asynchronous schedule's: a ticketed ring of (field, tile) items plus one
// state word per tile, so a tile is queued at most once and held by one worker
// (a CTA or a warp) at a time.
#pragma once

#include "device.cuh"
#include "kernels.h"

namespace mrc {

// Label extended by a run of `h` steps whose prices sum to `d` (kMax = blocked or
// saturated); a dist reaching 0xFFFFFFFF is unreachable.  With 32-bit wrapping
// addition, td or d equal to kMax always gives nd < td or nd == kMax, so those
// two tests cover the blocked operands too.
__device__ __forceinline__ u64 ext2(u64 t, uint32_t d, uint32_t h) {
    const uint32_t td = (uint32_t)(t >> 32);
    const uint32_t nd = td + d;
    const bool bad = (nd < td) | (nd == kMax);
    return bad ? kInf : (((u64)nd << 32) | (uint32_t)((uint32_t)t + h));
}

// Saturating sum of step prices; kMax absorbs (an operand equal to kMax gives
// s == kMax or s < a under wrapping addition).
__device__ __forceinline__ uint32_t dsum(uint32_t a, uint32_t b) {
    const uint32_t s = a + b;
    return s < a ? kMax : s;
}

__device__ __forceinline__ u64 umin64(u64 a, u64 b) { return a < b ? a : b; }

// Work queue of the asynchronous form.  count[0] = tickets handed to pushers
// (tail), head[0] = tickets handed to poppers, count[1] = items queued or in
// flight.  lists[0, cap) holds the items, lists[cap, 2 cap) their ticket tags
// (ticket + 1, zeroed before launch).  A tile is queued at most once at a time
// (its tstamp word is the queued flag), so cap = total tiles never overflows.
constexpr uint32_t kQueueSpinLimit = 1u << 24;  // polls of one wait (~16 s with the backoff below)

// Tile states in the tstamp word: 0 idle, 1 queued, 2 held by a worker,
// 3 held and improved again meanwhile (the holder continues it in place, or
// queues it once more, when it finishes, so improvements that arrive during a
// relaxation share one re-activation and no tile is ever relaxed by two
// workers at once).
constexpr uint32_t kTileIdle = 0, kTileQueued = 1, kTileHeld = 2, kTileHeldDirty = 3;

__device__ __forceinline__ void async_enqueue(const RelaxArgs &a, uint32_t fi, uint32_t u) {
    Ctl *c = a.ctl;
    atomicAdd(&c->count[1], 1u);  // in flight before it is visible
    const uint32_t h = atomicAdd(&c->count[0], 1u);
    const size_t slot = h % a.list_cap;
    a.lists[slot] = ((u64)fi << 32) | u;
    __threadfence();
    atomicExch(a.lists + a.list_cap + slot, (u64)h + 1u);
}

__device__ __forceinline__ void async_push(const RelaxArgs &a, uint32_t fi, uint32_t tile_off, uint32_t u) {
    uint32_t *st = a.tstamp + tile_off + u;
    for (int tries = 0; tries < 1024; ++tries) {
        const uint32_t old = atomicCAS(st, kTileIdle, kTileQueued);
        if (old == kTileIdle) {
            async_enqueue(a, fi, u);
            return;
        }
        if (old == kTileQueued || old == kTileHeldDirty) return;  // it will read our labels
        if (atomicCAS(st, kTileHeld, kTileHeldDirty) == kTileHeld) return;
        // the holder finished in between: try again from idle
    }
    atomicOr(&a.ctl->status, kStatusQueueOverflow);  // the state kept changing under us
}

// Called by the holder after its write-back and pushes: release the tile, or
// queue it again if a neighbour improved it while it was held.
__device__ __forceinline__ void async_release(const RelaxArgs &a, uint32_t fi, uint32_t tile_off, uint32_t t) {
    uint32_t *st = a.tstamp + tile_off + t;
    if (atomicCAS(st, kTileHeld, kTileIdle) == kTileHeldDirty) {
        atomicExch(st, kTileQueued);
        async_enqueue(a, fi, t);
    }
}

// An item is done: it leaves the in-flight count (after its own pushes were counted).
__device__ __forceinline__ void async_done(Ctl *c) { atomicSub(&c->count[1], 1u); }

// Next item for the calling worker (one thread), or kInf when no work is left.  The
// wait is bounded: kQueueSpinLimit polls, then kStatusBarrier and an exit.
__device__ __forceinline__ u64 async_pop(const RelaxArgs &a) {
    Ctl *c = a.ctl;
    const uint32_t h = atomicAdd(&c->head[0], 1u);
    const size_t slot = h % a.list_cap;
    const volatile u64 *tag = a.lists + a.list_cap + slot;
    // Each waiter polls its own slot tag; the shared in-flight count and status
    // words (which every worker updates) are read only every 16th poll, and the
    // sleep between polls doubles up to 1 us, so thousands of idle waiters do
    // not flood one L2 line while the busy workers update it.
    for (uint32_t spins = 0;; ++spins) {
        if (*tag == (u64)h + 1u) {
            __threadfence();
            return __ldcg(a.lists + slot);
        }
        if ((spins & 15u) == 15u) {
            if (*(volatile const uint32_t *)&c->count[1] == 0u) return kInf;  // nothing queued or running
            if (*(volatile const uint32_t *)&c->status) return kInf;
        }
        if (spins > kQueueSpinLimit) {
            atomicOr(&c->status, kStatusBarrier);
            return kInf;
        }
        __nanosleep(32u << min(spins >> 4, 5u));
    }
}

// Planes of step prices into a cell: from -x, +x, -y, +y, the layer below, the
// layer above (the order of the price planes and of a staged tile's planes).
enum { kInNegX = 0, kInPosX = 1, kInNegY = 2, kInPosY = 3, kInBelow = 4, kInAbove = 5 };

// Exact price of the step into cell c (at l, y, x) from direction `dir`, with
// the net's own pads, endpoints, via exemptions and directed-price overrides (the staging rules of the
// CTA-wide relax kernel without price planes, negotiated.rs:2914-2966 and :3010-3043).
static __device__ __noinline__ uint32_t exact_in_price(const DevBoard &b, const DevField &f, const uint32_t *pads, int dir, uint32_t c,
                                   uint32_t l, uint32_t y, uint32_t x) {
    const uint8_t fc = b.flags ? __ldg(b.flags + c) : 0;
    const uint32_t ec = cell_enter(b, f, pads, c, fc);
    if (ec == kMax) return kMax;
    const uint32_t plane = b.w * b.h;
    if (dir == kInBelow || dir == kInAbove) {
        const bool below = dir == kInBelow;
        if (below ? l == 0 : l + 1 >= b.layers) return kMax;
        const uint32_t k = below ? l - 1 : l;
        if (!((b.via_mask >> k) & 1u)) return kMax;
        const uint32_t p = below ? c - plane : c + plane;
        const uint8_t fp = b.flags ? __ldg(b.flags + p) : 0;
        if ((cell_tile_flags(f, pads, c, fc) | cell_tile_flags(f, pads, p, fp)) & kViaBlocked) return kMax;
        return capmul(__ldg(b.via_edge + k), ec);
    }
    uint32_t p, base;
    uint8_t out_bit, in_bit;
    if (dir == kInNegX) {
        if (x == 0) return kMax;
        p = c - 1;
        base = b.directed ? field_directed(b, f, c, 1) : __ldg(b.x_edge + x - 1);
        out_bit = kEdgePosX;
        in_bit = kEdgeNegX;
    } else if (dir == kInPosX) {
        if (x + 1 >= b.w) return kMax;
        p = c + 1;
        base = b.directed ? field_directed(b, f, c, 2) : __ldg(b.x_edge + x);
        out_bit = kEdgeNegX;
        in_bit = kEdgePosX;
    } else if (dir == kInNegY) {
        if (y == 0) return kMax;
        p = c - b.w;
        base = b.directed ? field_directed(b, f, c, 0) : __ldg(b.y_edge + y - 1);
        out_bit = kEdgePosY;
        in_bit = kEdgeNegY;
    } else {
        if (y + 1 >= b.h) return kMax;
        p = c + b.w;
        base = b.directed ? field_directed(b, f, c, 3) : __ldg(b.y_edge + y);
        out_bit = kEdgeNegY;
        in_bit = kEdgePosY;
    }
    const uint8_t fp = b.flags ? __ldg(b.flags + p) : 0;
    if ((fp & out_bit) | (fc & in_bit)) return kMax;
    if (b.directed && base == kMax) return kMax;
    return capmul(base, ec);
}

}  // namespace mrc
