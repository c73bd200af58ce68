// relax.cu — the batched field + canonical path kernels.
//
// relax_rounds_kernel: one cooperative persistent launch solves every field
// (net x window) of a batch.  Each field's labels live in HBM as u64
// (dist << 32 | hops), window-packed like the reference's ragged layout
// (metal/src/lib.rs:833-871).  Windows are cut into tiles of 32 x TH cells over
// every layer.  Work proceeds in bulk-synchronous rounds over a shared list of
// active (field, tile) items: a CTA stages a tile plus a one-cell halo ring in
// shared memory, relaxes it to local convergence with directional sweeps (the
// edge-aware row / column / layer-stack sweeps of gpu.rs:259-430, run on-chip
// instead of one dispatch per round), writes it back and queues each neighbour
// whose halo it now improves for the next round.  A field is final when no
// tile of it is queued; the launch ends when the whole list drains.
//
// Tiles of one field run concurrently in different CTAs.  That is safe because
// labels only decrease, every label is one aligned 64-bit word (a halo read is
// an old or a new label, never a torn mix), labels are read through L2
// (ld.global.cg) so no SM sees a stale L1 line, and a tile is processed by at
// most one CTA per round.  A neighbour read before it improves is re-queued by
// that neighbour's own push check, so no improvement is lost.
//
// path kernels: the path length is hops[dst] + 1 (every canonical predecessor
// has exactly one fewer hop), so offsets come from one device scan and one warp
// per net walks dst -> src choosing the lowest-CellIdx predecessor whose label
// and step reproduce the current label (metal/src/lib.rs:308-396).
#include <cuda_runtime.h>

#include <algorithm>

#include "device.cuh"
#include "kernels.h"
#include "tiles.cuh"

namespace mrc {

constexpr uint32_t kTW = 32;  // tile width (one warp across a row)
constexpr int kLaneCells = 4;  // cells per lane in the row / column passes
// Shared-memory row pitches of the staged tile: labels (u64) per 34-cell row
// (32 + halo), step prices (u32) per 32-cell row.  (Padding them to 35 / 33
// removes bank conflicts of the row passes but measured no faster, and the
// extra bytes cost a resident CTA per SM on 8-layer tiles.)
constexpr uint32_t kLabPitch = 34;
constexpr uint32_t kStPitch = 32;
constexpr uint32_t kFlPitch = 36;  // flag bytes per staged row (34 used)
constexpr int kStageUnroll = 4;    // cells whose loads one thread issues together
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kTmaSpinLimit = 1u << 22;

// ---- TMA and mbarrier primitives (sm_90+ PTX) ---------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// One tiled 4-D TMA load (coordinates innermost first) completing on `bar`.
__device__ __forceinline__ void tma_load_4d(void *dst, const void *tmap, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
constexpr uint32_t kBarrierSpinLimit = 1u << 25;  // ~ seconds with the backoff below

// Asynchronous 4-byte global -> shared copy (cp.async, L1-allocating) and its
// completion wait.
__device__ __forceinline__ void cp_async4(uint32_t *smem, const uint32_t *gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }


// Step-price planes of a staged tile: the move into cell c from its neighbour
// at -x, +x, -y, +y, the layer below and the layer above.
enum { kFromNegX = 0, kFromPosX = 1, kFromNegY = 2, kFromPosY = 3, kFromBelow = 4, kFromAbove = 5 };

template <int TH, bool FB>  // FB: fell marks as bytes (the price-plane kernels)
struct Tile {
    u64 *lab;        // [L][TH+2][34] labels with a one-cell halo ring
    uint32_t *st;    // [6][L][TH][sp] step prices into interior cells (column x at sp-offset xo + x)
    uint8_t *rowd;   // [L][TH] row needs a sweep
    uint8_t *cold;   // [L][32] column needs a sweep
    uint8_t *stackd; // [TH][32] layer stack needs a sweep
    uint32_t *fellw; // [L][TH] bit x: the label of (l, y, x) fell in this activation (staged prices), or
    uint8_t *fellb;  // [L][TH][32] 1 = it fell (price planes: plain byte stores, no shared atomics)
    uint8_t *fl;     // [L][TH+2][kFlPitch] board flag bytes of the tile and its halo (computed prices only)
    uint32_t L;
    uint32_t sp, xo; // price row pitch and column offset: 32, 0 computed; kPlaneTmaBoxW, tx0 & 3 from the planes
    __device__ __forceinline__ uint32_t li(uint32_t l, uint32_t sy, uint32_t sx) const {
        return (l * (TH + 2) + sy) * kLabPitch + sx;
    }
    __device__ __forceinline__ uint32_t si(uint32_t plane, uint32_t l, uint32_t y, uint32_t x) const {
        return ((plane * L + l) * TH + y) * sp + x + xo;
    }
    __device__ __forceinline__ void fell(uint32_t l, uint32_t y, uint32_t x) const {
        if constexpr (FB) fellb[(l * TH + y) * kTW + x] = 1;
        else atomicOr(&fellw[l * TH + y], 1u << x);
    }
    // a label of interior cell (l, y, x) fell: every other line through it must be swept again
    __device__ __forceinline__ void touched_by_row(uint32_t l, uint32_t y, uint32_t x) const {
        cold[l * 32 + x] = 1;
        stackd[y * 32 + x] = 1;
        fell(l, y, x);
    }
    __device__ __forceinline__ void touched_by_col(uint32_t l, uint32_t y, uint32_t x) const {
        rowd[l * TH + y] = 1;
        stackd[y * 32 + x] = 1;
        fell(l, y, x);
    }
    __device__ __forceinline__ void touched_by_stack(uint32_t l, uint32_t y, uint32_t x) const {
        rowd[l * TH + y] = 1;
        cold[l * 32 + x] = 1;
        fell(l, y, x);
    }
};

// Line passes over lines of K*S cells, S consecutive lanes per line (K cells
// each), skipping lines whose dirty flag is clear.  Each lane runs its
// segment's local chain, the S lanes combine their transfer functions
// f(t) = min(A, t (+) (D, H)) with a Kogge-Stone scan (H, the hop count, is the
// group's cell count), and every cell takes min(local, incoming (+) prefix).
// `halo(line, &before, &after)` gives the label indices outside both ends;
// `touch(line, pos)` marks the crossing lines of a cell whose label fell.
// Both directions of a line run in one pass: the forward scan, then, on its
// results still in registers, the backward scan (mirror image: shuffles down,
// the halo after the last cell).  A 1-D line is closed by one forward and one
// backward scan, so one load and one store of each label serve both.  `cell(line, pos, &lab,
// &step_fwd, &step_bwd)`: step_fwd prices the move into the cell from its
// predecessor in traversal order, step_bwd the move from its successor.
template <int K, int S, class CellFn, class HaloFn, class TouchFn>
__device__ __forceinline__ bool seg_pass(u64 *lab, const uint32_t *st, uint8_t *dirty, uint32_t nlines, CellFn cell,
                                          HaloFn halo, TouchFn touch) {
    bool changed = false;
    const uint32_t lanes_total = nlines * S;
    for (uint32_t base = 0; base < lanes_total; base += blockDim.x) {
        if (base + (threadIdx.x & ~31u) >= lanes_total) break;
        const uint32_t tl = base + threadIdx.x;
        const uint32_t line = tl / S, seg = tl % S;
        const bool mine = dirty[line] != 0;
        const uint32_t mask = __ballot_sync(0xFFFFFFFFu, mine);
        if (!mine) continue;
        if (seg == 0) dirty[line] = 0;
        u64 v[K], u[K];
        uint32_t spf[K], spb[K], P[K], li[K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            uint32_t sf, sb;
            cell(line, seg * K + i, &li[i], &sf, &sb);
            v[i] = lab[li[i]];
            spf[i] = st[sf];
            spb[i] = st[sb];
        }
        uint32_t hf, hb;
        halo(line, &hf, &hb);
        // forward
        u[0] = v[0];
        P[0] = spf[0];
#pragma unroll
        for (int i = 1; i < K; ++i) {
            u[i] = umin64(v[i], ext2(u[i - 1], spf[i], 1));
            P[i] = dsum(P[i - 1], spf[i]);
        }
        {
            u64 A = u[K - 1];
            uint32_t D = P[K - 1];
#pragma unroll
            for (int o = 1; o < S; o <<= 1) {
                const u64 Ap = __shfl_up_sync(mask, A, o, S);
                const uint32_t Dp = __shfl_up_sync(mask, D, o, S);
                if (seg >= (uint32_t)o) {
                    A = umin64(A, ext2(Ap, D, (uint32_t)(K * o)));
                    D = dsum(Dp, D);
                }
            }
            const u64 hl = lab[hf];
            u64 C = hl;
            if (S > 1) {
                const u64 Fa = __shfl_up_sync(mask, A, 1, S);
                const uint32_t Fd = __shfl_up_sync(mask, D, 1, S);
                if (seg > 0) C = umin64(Fa, ext2(hl, Fd, K * seg));
            }
            if (C != kInf) {
#pragma unroll
                for (int i = 0; i < K; ++i) u[i] = umin64(u[i], ext2(C, P[i], (uint32_t)i + 1u));
            }
        }
        // backward over the forward results; segment sb = S-1-seg counts from the far end
        {
            const uint32_t sbk = (uint32_t)(S - 1) - seg;
            P[K - 1] = spb[K - 1];
#pragma unroll
            for (int i = K - 2; i >= 0; --i) {
                u[i] = umin64(u[i], ext2(u[i + 1], spb[i], 1));
                P[i] = dsum(P[i + 1], spb[i]);
            }
            u64 A = u[0];
            uint32_t D = P[0];
#pragma unroll
            for (int o = 1; o < S; o <<= 1) {
                const u64 Ap = __shfl_down_sync(mask, A, o, S);
                const uint32_t Dp = __shfl_down_sync(mask, D, o, S);
                if (sbk >= (uint32_t)o) {
                    A = umin64(A, ext2(Ap, D, (uint32_t)(K * o)));
                    D = dsum(Dp, D);
                }
            }
            const u64 hr = lab[hb];
            u64 C = hr;
            if (S > 1) {
                const u64 Fa = __shfl_down_sync(mask, A, 1, S);
                const uint32_t Fd = __shfl_down_sync(mask, D, 1, S);
                if (sbk > 0) C = umin64(Fa, ext2(hr, Fd, K * sbk));
            }
            if (C != kInf) {
#pragma unroll
                for (int i = 0; i < K; ++i) u[i] = umin64(u[i], ext2(C, P[i], (uint32_t)(K - i)));
            }
        }
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (u[i] < v[i]) {
                lab[li[i]] = u[i];
                touch(line, seg * K + i);
                changed = true;
            }
        }
    }
    return changed;
}

// Grid-wide barrier for a cooperative launch.  The wait is bounded: after
// kBarrierSpinLimit polls it records kStatusBarrier and returns, and every CTA
// leaves the round loop once the status word is non-zero.
__device__ void grid_barrier(Ctl *c, uint32_t nblocks, uint32_t spin_limit = kBarrierSpinLimit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        volatile uint32_t *gen_p = &c->bar_gen;
        const uint32_t gen = *gen_p;
        const uint32_t arrived = atomicAdd(&c->bar_count, 1u) + 1u;
        if (arrived == nblocks) {
            atomicExch(&c->bar_count, 0u);
            __threadfence();
            atomicAdd(&c->bar_gen, 1u);
        } else {
            uint32_t spins = 0;
            while (*gen_p == gen) {
                if (++spins > spin_limit) {
                    atomicOr(&c->status, kStatusBarrier);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

__device__ __forceinline__ uint32_t ld_status(const Ctl *c) { return *(volatile const uint32_t *)&c->status; }

// Flags of a window cell as a via endpoint: blocked by the board via node bit or
// by the static via mask unless the net lists the cell as a via pad.
// Own-pad and via-exemption lookups against the shared-memory copy of the
// field's sorted lists when they fit (kPadCache / kVPadCache), else HBM.
constexpr uint32_t kPadCache = 128, kVPadCache = 32;
__device__ __forceinline__ bool own_pad(const uint32_t *s, uint32_t cap, const uint32_t *g, uint32_t n,
                                        uint32_t key) {
    return n <= cap ? sorted_has(s, n, key) : sorted_has(g, n, key);
}

__device__ __forceinline__ bool via_blocked(const DevField &f, const uint32_t *pads, uint32_t gcell, uint8_t gf) {
    return (cell_tile_flags(f, pads, gcell, gf) & kViaBlocked) != 0;
}

template <int TH, bool FB>
__device__ __forceinline__ bool stack_pass(const Tile<TH, FB> &t);

// With 8-row tiles and 4 cells per lane, the row lanes of a layer (8 rows x 8
// lanes) and its column lanes (32 columns x 2 lanes) fall on the same pair of
// warps (2p, 2p+1), in every iteration of a pass.  Between the row and column
// passes those 64 threads synchronise alone (named barrier 1 + p) instead of
// the whole CTA.
__device__ __forceinline__ void pair_barrier() {
    asm volatile("bar.sync %0, 64;" ::"r"(1u + (threadIdx.x >> 6)) : "memory");
}

// The row and the column pass of a sweep on their own (the reversed sweep's).
template <int TH, bool FB>
__device__ __forceinline__ bool row_pass(const Tile<TH, FB> &t) {
    constexpr int KC = kLaneCells, SR = 32 / KC;  // cells per lane, lanes per row
    return seg_pass<KC, SR>(
        t.lab, t.st, t.rowd, t.L * TH,
        [&](uint32_t line, uint32_t pos, uint32_t *li, uint32_t *sf, uint32_t *sb) {
            const uint32_t l = line / TH, y = line % TH;
            *li = t.li(l, y + 1, pos + 1);
            *sf = t.si(kFromNegX, l, y, pos);
            *sb = t.si(kFromPosX, l, y, pos);
        },
        [&](uint32_t line, uint32_t *hf, uint32_t *hb) {
            *hf = t.li(line / TH, line % TH + 1, 0);
            *hb = t.li(line / TH, line % TH + 1, 33);
        },
        [&](uint32_t line, uint32_t pos) { t.touched_by_row(line / TH, line % TH, pos); });
}

template <int TH, bool FB>
__device__ __forceinline__ bool col_pass(const Tile<TH, FB> &t) {
    constexpr int KC = kLaneCells, SC = TH / KC;  // cells per lane, lanes per column
    return seg_pass<KC, SC>(
        t.lab, t.st, t.cold, t.L * 32,
        [&](uint32_t line, uint32_t pos, uint32_t *li, uint32_t *sf, uint32_t *sb) {
            const uint32_t l = line / 32, x = line % 32;
            *li = t.li(l, pos + 1, x + 1);
            *sf = t.si(kFromNegY, l, pos, x);
            *sb = t.si(kFromPosY, l, pos, x);
        },
        [&](uint32_t line, uint32_t *hf, uint32_t *hb) {
            *hf = t.li(line / 32, 0, line % 32 + 1);
            *hb = t.li(line / 32, TH + 1, line % 32 + 1);
        },
        [&](uint32_t line, uint32_t pos) { t.touched_by_col(line / 32, pos, line % 32); });
}

// rows <-> columns: only the warps of the same layers exchange data
template <int TH>
__device__ __forceinline__ void plane_barrier() {
    if constexpr (TH == 8 && kLaneCells == 4) {
        pair_barrier();
    } else {
        __syncthreads();
    }
}

// One sweep of a staged tile: rows (8 lanes x 4 cells), columns (TH/4 lanes x
// 4 cells), layer stacks (one thread each), each forward then backward, only
// over lines whose dirty flag is set.
template <int TH, bool FB>
__device__ __forceinline__ bool relax_tile(const Tile<TH, FB> &t) {
    constexpr int KC = kLaneCells;          // cells per lane in a line pass
    constexpr int SR = 32 / KC, SC = TH / KC;  // lanes per row / per column
    const uint32_t L = t.L;
    bool ch = false;
    ch |= seg_pass<KC, SR>(
        t.lab, t.st, t.rowd, L * TH,
        [&](uint32_t line, uint32_t pos, uint32_t *li, uint32_t *sf, uint32_t *sb) {
            const uint32_t l = line / TH, y = line % TH;
            *li = t.li(l, y + 1, pos + 1);
            *sf = t.si(kFromNegX, l, y, pos);
            *sb = t.si(kFromPosX, l, y, pos);
        },
        [&](uint32_t line, uint32_t *hf, uint32_t *hb) {
            *hf = t.li(line / TH, line % TH + 1, 0);
            *hb = t.li(line / TH, line % TH + 1, 33);
        },
        [&](uint32_t line, uint32_t pos) { t.touched_by_row(line / TH, line % TH, pos); });
    // rows -> columns: only the warps of the same layers exchange data
    if constexpr (TH == 8 && kLaneCells == 4) {
        pair_barrier();
    } else {
        __syncthreads();
    }
    ch |= seg_pass<KC, SC>(
        t.lab, t.st, t.cold, L * 32,
        [&](uint32_t line, uint32_t pos, uint32_t *li, uint32_t *sf, uint32_t *sb) {
            const uint32_t l = line / 32, x = line % 32;
            *li = t.li(l, pos + 1, x + 1);
            *sf = t.si(kFromNegY, l, pos, x);
            *sb = t.si(kFromPosY, l, pos, x);
        },
        [&](uint32_t line, uint32_t *hf, uint32_t *hb) {
            *hf = t.li(line / 32, 0, line % 32 + 1);
            *hb = t.li(line / 32, TH + 1, line % 32 + 1);
        },
        [&](uint32_t line, uint32_t pos) { t.touched_by_col(line / 32, pos, line % 32); });
    if (L > 1) {
        __syncthreads();
        ch |= stack_pass<TH, FB>(t);
    }
    return ch;
}

// Columns first, then rows and stacks: the queue form's order (fewer sweeps per
// activation than rows first on its 32 x 8 tiles).
template <int TH, bool FB>
__device__ __forceinline__ bool relax_tile_cols_first(const Tile<TH, FB> &t) {
    bool ch = col_pass(t);
    plane_barrier<TH>();
    ch |= row_pass(t);
    if (t.L > 1) {
        __syncthreads();
        ch |= stack_pass<TH, FB>(t);
    }
    return ch;
}

// The same passes in the opposite order (stacks, columns, rows); the rounds
// form alternates the two orders between sweeps.
template <int TH, bool FB>
__device__ __forceinline__ bool relax_tile_rev(const Tile<TH, FB> &t) {
    bool ch = false;
    if (t.L > 1) {
        ch = stack_pass<TH, FB>(t);
        __syncthreads();
    }
    ch |= col_pass(t);
    plane_barrier<TH>();
    ch |= row_pass(t);
    return ch;
}

// Layer stacks: one thread per (y, x) column of the tile, upward then downward.
// Stacks of up to kStackRegs layers are held in registers between the two
// directions (one load and at most one store per label); taller ones run from
// shared memory.
constexpr uint32_t kStackRegs = 4;

template <int TH, bool FB>
__device__ __forceinline__ bool stack_pass(const Tile<TH, FB> &t) {
    const uint32_t L = t.L;
    bool ch = false;
    for (uint32_t r = threadIdx.x; r < TH * 32; r += blockDim.x) {
        if (!t.stackd[r]) continue;
        t.stackd[r] = 0;
        const uint32_t y = r / 32, x = r % 32;
        if (L <= kStackRegs) {
            u64 v[kStackRegs];
            uint32_t fell = 0;  // bit l: the label of layer l fell
#pragma unroll
            for (uint32_t l = 0; l < kStackRegs; ++l)
                if (l < L) v[l] = t.lab[t.li(l, y + 1, x + 1)];
            u64 prev = kInf;
#pragma unroll
            for (uint32_t l = 0; l < kStackRegs; ++l) {
                if (l < L) {
                    const u64 w = ext2(prev, l ? t.st[t.si(kFromBelow, l, y, x)] : kMax, 1);
                    if (w < v[l]) {
                        v[l] = w;
                        fell |= 1u << l;
                    }
                    prev = v[l];
                }
            }
            prev = kInf;
#pragma unroll
            for (int l = (int)kStackRegs - 1; l >= 0; --l) {
                if ((uint32_t)l < L) {
                    const u64 w = ext2(prev, (uint32_t)l + 1 < L ? t.st[t.si(kFromAbove, (uint32_t)l, y, x)] : kMax, 1);
                    if (w < v[l]) {
                        v[l] = w;
                        fell |= 1u << l;
                    }
                    prev = v[l];
                }
            }
#pragma unroll
            for (uint32_t l = 0; l < kStackRegs; ++l) {
                if ((fell >> l) & 1u) {
                    t.lab[t.li(l, y + 1, x + 1)] = v[l];
                    t.touched_by_stack(l, y, x);
                    ch = true;
                }
            }
            continue;
        }
        u64 prev = kInf;
        for (uint32_t l = 0; l < L; ++l) {
            const uint32_t c = t.li(l, y + 1, x + 1);
            const u64 cur = t.lab[c];
            const u64 w = umin64(cur, ext2(prev, l ? t.st[t.si(kFromBelow, l, y, x)] : kMax, 1));
            if (w < cur) {
                t.lab[c] = w;
                t.touched_by_stack(l, y, x);
                ch = true;
            }
            prev = w;
        }
        prev = kInf;
        for (int l = (int)L - 1; l >= 0; --l) {
            const uint32_t c = t.li((uint32_t)l, y + 1, x + 1);
            const u64 cur = t.lab[c];
            const u64 w =
                umin64(cur, ext2(prev, (uint32_t)l + 1 < L ? t.st[t.si(kFromAbove, (uint32_t)l, y, x)] : kMax, 1));
            if (w < cur) {
                t.lab[c] = w;
                t.touched_by_stack((uint32_t)l, y, x);
                ch = true;
            }
            prev = w;
        }
    }
    return ch;
}

// One (field, tile) item: stage the tile and its halo, relax it to local
// convergence, write it back and queue the neighbours it improves.
// Shared-memory layout of one staged tile (relax_smem_bytes sizes it the same way).
struct TileLayout {
    size_t st, rowd, fellw, fl, total;
};
__host__ __device__ inline TileLayout tile_layout(uint32_t L, uint32_t TH, bool planes) {
    TileLayout o;
    const size_t sp = planes ? kPlaneTmaBoxW : kStPitch;
    o.st = ((size_t)L * (TH + 2) * kLabPitch * 8 + 127) & ~(size_t)127;  // TMA destination: 128-byte aligned
    o.rowd = o.st + (size_t)6 * L * TH * sp * 4;
    // fell marks: bytes with the price planes (their tiles fit the same CTAs per SM
    // either way), bits otherwise
    o.fellw = (o.rowd + (size_t)L * TH + (size_t)L * kTW + (size_t)TH * kTW + 3) & ~(size_t)3;
    o.fl = o.fellw + (size_t)L * TH * (planes ? kTW : 4);
    o.total = o.fl + (planes ? 0 : (size_t)L * (TH + 2) * kFlPitch);
    return o;
}

// A field's directed-price overrides inside its tile (a negotiation net's own
// prices on its own footprint), into the shared planes laid out as Tile::si:
// the raw directed words before the step prices are formed (exact = false), or
// the four planar in-prices priced exactly (exact = true, over the price planes).
// Out of line: it runs only for overriding fields and keeps the staging's
// registers free.
static __device__ __noinline__ void stage_overrides(const DevBoard &b, const DevField &f, const uint32_t *pads,
                                                    uint32_t *st, uint32_t L, uint32_t TH, uint32_t sp, uint32_t xo,
                                                    int tx0, int ty0, uint32_t tw, uint32_t th, bool exact) {
    const uint32_t *oc = b.over_cells + f.over_off;
    auto si = [&](int p, uint32_t l, uint32_t y, uint32_t x) { return (((uint32_t)p * L + l) * TH + y) * sp + x + xo; };
    for (uint32_t j = threadIdx.x; j < L * th; j += blockDim.x) {
        const uint32_t l = j / th, y = j - l * th;
        const uint32_t lo_c = (l * b.h + (uint32_t)ty0 + y) * b.w + (uint32_t)tx0, hi_c = lo_c + tw;
        for (uint32_t k = over_lower_bound(oc, f.n_over, lo_c); k < f.n_over; ++k) {
            const uint32_t c = __ldg(oc + k);
            if (c >= hi_c) break;
            const uint32_t x = c - lo_c;
            if (exact) {
                for (int p = kInNegX; p <= kInPosY; ++p)
                    st[si(p, l, y, x)] = exact_in_price(b, f, pads, p, c, l, (uint32_t)ty0 + y, (uint32_t)tx0 + x);
            } else {
                const uint4 d = __ldg(b.over_price + f.over_off + k);
                st[si(kFromNegX, l, y, x)] = d.y;
                st[si(kFromPosX, l, y, x)] = d.z;
                st[si(kFromNegY, l, y, x)] = d.x;
                st[si(kFromPosY, l, y, x)] = d.w;
            }
        }
    }
}

// With PL the tile's six step-price planes come from the board's precomputed
// planes (planes_kernel) in one TMA load: box kPlaneTmaBoxW x TH x L x 6 at column
// tx0 rounded down to 4 (a TMA x coordinate times 4 bytes must be a multiple
// of 16; the tile's columns then start at xo = tx0 & 3 in the box).  Cells past
// the window and the stacks of the net's endpoints, own pads and via pads are
// then priced exactly (exact_in_price); the push checks read the planes.
// OV: the batch carries per-net directed-price overrides (negotiation with a
// clearance; always 8-row tiles, 256 threads); without it none of the override
// lookups is compiled in.
template <int TH, bool ASYNC, bool PL, bool OV>
__device__ __forceinline__ void process_item(const RelaxArgs &a, uint32_t fi, uint32_t t, uint32_t round,
                                             unsigned char *smem_raw, uint64_t *mbar, uint32_t &tma_phase,
                                             unsigned long long *s_cnt) {
    const uint32_t SW = kTW + 2, SH = TH + 2;
    Tile<TH, PL> tile;
    __shared__ uint32_t s_push[4];
    __shared__ uint32_t s_vis[5];  // self, left, right, top, bottom
    __shared__ uint32_t s_pads[kPadCache], s_vpads[kVPadCache];
    Ctl *ctl = a.ctl;
    const uint32_t tid = threadIdx.x;
    const uint32_t cap = a.list_cap;
    const DevField f = a.fields[fi];
    const DevBoard b = a.boards[f.board];
    const uint32_t L = b.layers;  // the shared tile is laid out for this board's layers
    const uint32_t nsm = L * SH * SW;  // staged cells (pitch kLabPitch in smem)
    const uint32_t ntx = (f.ww + kTW - 1) / kTW, nty = (f.wh + TH - 1) / TH;
    const uint32_t txi = t % ntx, tyi = t / ntx;
    const int tx0 = (int)(f.x0 + txi * kTW), ty0 = (int)(f.y0 + tyi * TH);
    const TileLayout lay = tile_layout(L, TH, PL);
    tile.lab = reinterpret_cast<u64 *>(smem_raw);
    tile.st = reinterpret_cast<uint32_t *>(smem_raw + lay.st);
    tile.rowd = smem_raw + lay.rowd;
    tile.cold = tile.rowd + L * TH;
    tile.stackd = tile.cold + L * kTW;
    tile.fellw = reinterpret_cast<uint32_t *>(smem_raw + lay.fellw);
    tile.fellb = PL ? smem_raw + lay.fellw : nullptr;
    const uint32_t fell_words = L * TH * (PL ? kTW / 4 : 1);  // words of fell marks to clear
    tile.fl = smem_raw + lay.fl;
    tile.L = L;
    tile.sp = PL ? kPlaneTmaBoxW : kStPitch;
    tile.xo = PL ? ((uint32_t)tx0 & 3u) : 0u;
    if constexpr (PL) {
        // every thread is past the previous item (the caller's barrier): the
        // planes of this tile go global -> shared while the labels are staged
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            mbar_expect_tx(mbar, 6u * L * TH * kPlaneTmaBoxW * 4u);
            tma_load_4d(tile.st, b.tmap, tx0 & ~3, ty0, 0, 0, mbar);
        }
    }
    const uint32_t tw = min(kTW, f.ww - txi * kTW), th = min(TH, f.wh - tyi * TH);
    const int wx0 = (int)f.x0, wy0 = (int)f.y0, wx1 = (int)(f.x0 + f.ww), wy1 = (int)(f.y0 + f.wh);
    const u64 *lab = a.lab + f.lab_off;
    if constexpr (ASYNC) {
        // hold the tile before reading any label: a neighbour that improves our
        // halo after this point marks it dirty, and we queue it again when done
        if (tid == 0) {
            atomicExch(a.tstamp + f.tile_off + t, kTileHeld);
            __threadfence();
        }
    } else if (tid < 5) {
        uint32_t u = kNone;
        if (tid == 0) u = t;
        else if (tid == 1 && txi > 0) u = t - 1;
        else if (tid == 2 && txi + 1 < ntx) u = t + 1;
        else if (tid == 3 && tyi > 0) u = t - ntx;
        else if (tid == 4 && tyi + 1 < nty) u = t + ntx;
        s_vis[tid] = u == kNone ? 0u : __ldcg(a.tvisit + f.tile_off + u);
    }
    if (tid < 4) s_push[tid] = 0;
    if (f.n_pads <= kPadCache)
        for (uint32_t i = tid; i < f.n_pads; i += blockDim.x) s_pads[i] = __ldg(a.pads + f.pad_off + i);
    if (f.n_vpads <= kVPadCache)
        for (uint32_t i = tid; i < f.n_vpads; i += blockDim.x) s_vpads[i] = __ldg(a.pads + f.vpad_off + i);
    const uint32_t *gpads = a.pads + f.pad_off, *gvpads = a.pads + f.vpad_off;
    auto is_own_pad = [&](uint32_t c) {
        return c == f.src || c == f.dst || own_pad(s_pads, kPadCache, gpads, f.n_pads, c);
    };
    auto via_blk = [&](uint32_t c, uint8_t gf) {
        if (gf & kViaNode) return true;
        return (gf & kStaticVia) != 0 && !own_pad(s_vpads, kVPadCache, gvpads, f.n_vpads, c);
    };
    // Dirty lines start clear; staging marks exactly the lines that hold a
    // finite label (in the tile, or at their ends in the halo ring): a line of
    // +inf labels with +inf ends cannot change until a crossing line lowers one
    // of its cells, and that pass marks it.
    for (uint32_t i = tid; i < L * TH + L * kTW + TH * kTW; i += blockDim.x) tile.rowd[i] = 0;
    for (uint32_t i = tid; i < fell_words; i += blockDim.x) tile.fellw[i] = 0;
    __syncthreads();

    // ---- step prices into every interior cell: phase 1 -----------------
    // Per interior cell its cost (parked in the below-plane) and its four
    // planar base prices go global -> shared with asynchronous copies issued
    // first, so they overlap the label and flag loads below.  The board is
    // read-only during the launch, so the L1-allocating cp.async is safe for it
    // (labels, which other CTAs write, keep their L2-only loads).
    if constexpr (!PL) {  // with the planes the prices arrive by TMA
        const uint32_t ncell = L * TH * kTW;
        for (uint32_t i = tid; i < ncell; i += blockDim.x) {
            const uint32_t x = i % kTW, r = i / kTW, y = r % TH, l = r / TH;
            const int gx = tx0 + (int)x, gy = ty0 + (int)y;
            uint32_t *d0 = &tile.st[tile.si(kFromNegX, l, y, x)], *d1 = &tile.st[tile.si(kFromPosX, l, y, x)];
            uint32_t *d2 = &tile.st[tile.si(kFromNegY, l, y, x)], *d3 = &tile.st[tile.si(kFromPosY, l, y, x)];
            uint32_t *dc = &tile.st[tile.si(kFromBelow, l, y, x)];
            if (gx < wx1 && gy < wy1) {
                const uint32_t gc = (l * b.h + (uint32_t)gy) * b.w + (uint32_t)gx;
                cp_async4(dc, b.cost + gc);
                if (b.directed) {
                    const uint32_t *dp = reinterpret_cast<const uint32_t *>(b.directed + gc);
                    cp_async4(d0, dp + 1);  // from -x
                    cp_async4(d1, dp + 2);  // from +x
                    cp_async4(d2, dp + 0);  // from -y
                    cp_async4(d3, dp + 3);  // from +y
                } else {
                    *d0 = gx > wx0 ? __ldg(b.x_edge + gx - 1) : kMax;
                    *d1 = gx + 1 < wx1 ? __ldg(b.x_edge + gx) : kMax;
                    *d2 = gy > wy0 ? __ldg(b.y_edge + gy - 1) : kMax;
                    *d3 = gy + 1 < wy1 ? __ldg(b.y_edge + gy) : kMax;
                }
            } else {
                *d0 = *d1 = *d2 = *d3 = *dc = kMax;
            }
        }
        cp_async_commit();
    }

    // ---- stage labels and flag bytes (tile + halo ring) ---------------
    // Every thread issues the loads of kStageUnroll cells before it
    // stores any of them, so several L2 requests per thread are in
    // flight (labels through L2 with ld.global.cg).
    const uint32_t plane = b.w * b.h;
    for (uint32_t i0 = tid; i0 < nsm; i0 += kStageUnroll * blockDim.x) {
        u64 lv[kStageUnroll];
        uint8_t fv[kStageUnroll];
#pragma unroll
        for (int k = 0; k < kStageUnroll; ++k) {
            const uint32_t i = i0 + k * blockDim.x;
            lv[k] = kInf;
            fv[k] = 0;
            if (i >= nsm) continue;
            const uint32_t sx = i % SW, r = i / SW, sy = r % SH, l = r / SH;
            const int gx = tx0 + (int)sx - 1, gy = ty0 + (int)sy - 1;
            if (gx >= wx0 && gx < wx1 && gy >= wy0 && gy < wy1) {
                const bool hx = sx == 0 || sx == SW - 1, hy = sy == 0 || sy == SH - 1;
                uint32_t owner;  // which tile's label this smem cell holds
                if (hx && hy) owner = 5;  // corner: never read
                else if (sx == 0) owner = 1;
                else if (sx == SW - 1) owner = 2;
                else if (sy == 0) owner = 3;
                else if (sy == SH - 1) owner = 4;
                else owner = 0;
                const uint32_t gcell = (l * b.h + (uint32_t)gy) * b.w + (uint32_t)gx;
                const uint64_t lc = ((uint64_t)l * f.wh + (uint32_t)(gy - wy0)) * f.ww + (uint32_t)(gx - wx0);
                if constexpr (ASYNC) {
                    if (owner < 5) lv[k] = __ldcg(lab + lc);  // the arena starts at +inf
                } else {
                    if (owner < 5 && s_vis[owner]) lv[k] = __ldcg(lab + lc);
                    else if (owner == 0 && gcell == f.src) lv[k] = 0;  // first visit of the source tile
                }
                if (!PL && b.flags) fv[k] = __ldg(b.flags + gcell);
            }
        }
#pragma unroll
        for (int k = 0; k < kStageUnroll; ++k) {
            const uint32_t i = i0 + k * blockDim.x;
            if (i >= nsm) continue;
            const uint32_t sx = i % SW, r = i / SW, sy = r % SH, l = r / SH;
            tile.lab[tile.li(l, sy, sx)] = lv[k];
            if (!PL) tile.fl[(l * SH + sy) * kFlPitch + sx] = fv[k];
            if (lv[k] != kInf) {
                const bool row_in = sy >= 1 && sy <= TH, col_in = sx >= 1 && sx <= kTW;
                if (row_in) tile.rowd[l * TH + sy - 1] = 1;
                if (col_in) tile.cold[l * kTW + sx - 1] = 1;
                if (row_in && col_in) tile.stackd[(sy - 1) * kTW + sx - 1] = 1;
            }
        }
    }
    if constexpr (PL) {
        // the planes: a bounded wait for the TMA load (a load that never lands
        // sets the status and the launch ends without results)
        for (uint32_t spins = 0; !mbar_try_wait(mbar, tma_phase & 1u); ++spins) {
            if (spins == kTmaSpinLimit) {
                if (tid == 0) atomicOr(&ctl->status, kStatusQueueOverflow);
            } else if (spins > 2 * kTmaSpinLimit) {
                break;
            }
        }
        ++tma_phase;
        // cells past the window: no step enters them
        if (tw < kTW || th < TH) {
            for (uint32_t i = tid; i < L * TH * kTW; i += blockDim.x) {
                const uint32_t x = i % kTW, r = i / kTW, y = r % TH, l = r / TH;
                if (x < tw && y < th) continue;
#pragma unroll
                for (int p = 0; p < 6; ++p) tile.st[tile.si(p, l, y, x)] = kMax;
            }
        }
        // stacks whose prices depend on this net: its endpoints, own pads and
        // via pads, priced exactly on every layer
        auto exact_stack = [&](uint32_t c) {
            const uint32_t r = c % (b.w * b.h), gy = r / b.w, gx = r - gy * b.w;
            if (gx < (uint32_t)tx0 || gx >= (uint32_t)tx0 + tw || gy < (uint32_t)ty0 || gy >= (uint32_t)ty0 + th)
                return;
            for (uint32_t l = 0; l < L; ++l) {
                const uint32_t cl = (l * b.h + gy) * b.w + gx;
                for (int p = 0; p < 6; ++p)
                    tile.st[tile.si(p, l, gy - ty0, gx - tx0)] = exact_in_price(b, f, a.pads, p, cl, l, gy, gx);
            }
        };
        if (tid == 0) exact_stack(f.src);
        if (tid == 1) exact_stack(f.dst);
        if (f.n_pads | f.n_vpads) {
            for (uint32_t j = tid; j < 2 * L * th; j += blockDim.x) {
                const uint32_t q = j & 1u, r = j >> 1, l = r / th, y = r - l * th;
                const uint32_t lo_c = (l * b.h + ty0 + y) * b.w + tx0, hi_c = lo_c + tw;
                const uint32_t *list = a.pads + (q ? f.vpad_off : f.pad_off);
                const uint32_t n = q ? f.n_vpads : f.n_pads;
                uint32_t lo = 0, hi = n;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (__ldg(list + mid) < lo_c) lo = mid + 1;
                    else hi = mid;
                }
                for (; lo < n; ++lo) {
                    const uint32_t c = __ldg(list + lo);
                    if (c >= hi_c) break;
                    exact_stack(c);
                }
            }
        }
        // cells where this net's own directed prices differ from the board's
        // (negotiation overrides): their four planar in-prices priced exactly
        // (the same values an overlapping exact stack writes)
        if (OV && f.n_over && a.tover[f.tile_off + t])
            stage_overrides(b, f, a.pads, tile.st, L, TH, tile.sp, tile.xo, tx0, ty0, tw, th, true);
    } else {
        cp_async_wait_all();  // the board words copied before the label loop
        __syncthreads();
        // this net's own directed prices (negotiation overrides) replace the
        // board's words before the step prices are formed
        if (OV && f.n_over && a.tover[f.tile_off + t]) {
            stage_overrides(b, f, a.pads, tile.st, L, TH, tile.sp, tile.xo, tx0, ty0, tw, th, false);
            __syncthreads();
        }
        // Phase 2: every step price from the staged bytes (own pads and via
        // exemptions are the only global reads left).
        for (uint32_t i = tid; i < L * TH * kTW; i += blockDim.x) {
            const uint32_t x = i % kTW, r = i / kTW, y = r % TH, l = r / TH;
            const int gx = tx0 + (int)x, gy = ty0 + (int)y;
            uint32_t s0 = kMax, s1 = kMax, s2 = kMax, s3 = kMax, s4 = kMax, s5 = kMax;
            if (gx < wx1 && gy < wy1) {
                const uint32_t gc = (l * b.h + (uint32_t)gy) * b.w + (uint32_t)gx;
                const uint8_t *flr = tile.fl + (l * SH + y + 1) * kFlPitch + x + 1;  // this cell
                const uint8_t fc = flr[0];
                const uint32_t cost = tile.st[tile.si(kFromBelow, l, y, x)];
                uint32_t ec;  // cell_enter on staged values
                if (fc & kTraceNode) ec = kMax;
                else if (cost != kMax) ec = cost;
                else ec = is_own_pad(gc) ? 1u : kMax;
                if (ec != kMax) {
                    const bool dir = b.directed != nullptr;
                    auto planar = [&](uint32_t base, uint8_t fp, uint8_t out_bit, uint8_t in_bit) -> uint32_t {
                        if (dir && base == kMax) return kMax;  // blocked directed edge
                        if ((fp & out_bit) | (fc & in_bit)) return kMax;
                        return capmul(base, ec);
                    };
                    if (gx > wx0) s0 = planar(tile.st[tile.si(kFromNegX, l, y, x)], flr[-1], kEdgePosX, kEdgeNegX);
                    if (gx + 1 < wx1) s1 = planar(tile.st[tile.si(kFromPosX, l, y, x)], flr[1], kEdgeNegX, kEdgePosX);
                    if (gy > wy0)
                        s2 = planar(tile.st[tile.si(kFromNegY, l, y, x)], flr[-(int)kFlPitch], kEdgePosY, kEdgeNegY);
                    if (gy + 1 < wy1)
                        s3 = planar(tile.st[tile.si(kFromPosY, l, y, x)], flr[kFlPitch], kEdgeNegY, kEdgePosY);
                    if (L > 1) {
                        const bool vc = via_blk(gc, fc);
                        if (l > 0 && ((b.via_mask >> (l - 1)) & 1u) && !vc) {
                            const uint8_t fq = flr[-(int)(SH * kFlPitch)];
                            if (!via_blk(gc - plane, fq)) s4 = capmul(__ldg(b.via_edge + l - 1), ec);
                        }
                        if (l + 1 < L && ((b.via_mask >> l) & 1u) && !vc) {
                            const uint8_t fq = flr[SH * kFlPitch];
                            if (!via_blk(gc + plane, fq)) s5 = capmul(__ldg(b.via_edge + l), ec);
                        }
                    }
                }
            }
            tile.st[tile.si(kFromNegX, l, y, x)] = s0;
            tile.st[tile.si(kFromPosX, l, y, x)] = s1;
            tile.st[tile.si(kFromNegY, l, y, x)] = s2;
            tile.st[tile.si(kFromPosY, l, y, x)] = s3;
            tile.st[tile.si(kFromBelow, l, y, x)] = s4;
            tile.st[tile.si(kFromAbove, l, y, x)] = s5;
        }
    }
    __syncthreads();

    // ---- relax to local convergence ---------------------------------
    // Queue form: a tile that a neighbour improved while this CTA held it is
    // continued here (up to kContinueLimit times): its halo ring is read again
    // and the sweeps resume on the staged tile, without a release, a queue
    // round trip and a full re-staging.  Each continuation counts as an
    // activation.
    const uint32_t sweep_limit = L * kTW * TH + 4;
    __shared__ uint32_t s_more;
    for (uint32_t cont = 0;; ++cont) {
        uint32_t sweep = 0;
        for (;;) {
            // the rounds form alternates the pass order between sweeps (fewer
            // sweeps on the one-activation tiles it runs); the queue form runs
            // columns first, where alternation costs sweeps
            bool ch;
            if constexpr (!ASYNC) ch = (sweep & 1) ? relax_tile_rev(tile) : relax_tile(tile);
            else ch = relax_tile_cols_first(tile);
            ++sweep;
            const int any = __syncthreads_or(ch ? 1 : 0);
            if (!any) break;
            if (sweep > sweep_limit) {
                if (tid == 0) atomicOr(&ctl->status, kStatusRoundLimit);
                break;
            }
        }

        // ---- write back and find neighbours this tile can improve -------
        u64 *labw = a.lab + f.lab_off;
        // the tile is held by this CTA alone (both schedules), so plain stores;
        // indices are split by the compile-time tile shape (cells past a ragged
        // window edge are skipped).  Only labels that fell are stored, unless the
        // arena holds nothing valid for this tile yet (first visit, rounds form).
        const bool all_labels = !ASYNC && !s_vis[0];
        for (uint32_t i = tid; i < L * TH * kTW; i += blockDim.x) {
            const uint32_t tx = i % kTW, r = i / kTW, ty = r % TH, l = r / TH;
            if (tx >= tw || ty >= th) continue;
            if (!all_labels && !(PL ? tile.fellb[(l * TH + ty) * kTW + tx] : (tile.fellw[l * TH + ty] >> tx) & 1u))
                continue;
            const uint64_t lc = ((uint64_t)l * f.wh + (uint32_t)(ty0 - wy0) + ty) * f.ww + (uint32_t)(tx0 - wx0) + tx;
            labw[lc] = tile.lab[tile.li(l, ty + 1, tx + 1)];
        }
        // borders: 0 = left (-x), 1 = right (+x), 2 = top (-y), 3 = bottom (+y)
        const uint32_t nb = 2 * L * TH + 2 * L * kTW;
        for (uint32_t i = tid; i < nb; i += blockDim.x) {
            uint32_t side, l, k;
            if (i < 2 * L * TH) {
                side = i >= L * TH;
                const uint32_t r = i - side * L * TH;
                l = r / TH;
                k = r % TH;
                if (k >= th) continue;
            } else {
                const uint32_t j = i - 2 * L * TH;
                const uint32_t hi = j >= L * kTW;
                side = 2 + hi;
                const uint32_t r = j - hi * L * kTW;
                l = r / kTW;
                k = r % kTW;
                if (k >= tw) continue;
            }
            bool exists;
            uint32_t bsx, bsy, nsx, nsy, dir;
            uint8_t out_bit, in_bit;
            if (side == 0) {
                exists = txi > 0;
                bsx = 1; bsy = k + 1; nsx = 0; nsy = bsy;
                dir = 2; out_bit = kEdgeNegX; in_bit = kEdgePosX;
            } else if (side == 1) {
                exists = txi + 1 < ntx;
                bsx = tw; bsy = k + 1; nsx = tw + 1; nsy = bsy;
                dir = 1; out_bit = kEdgePosX; in_bit = kEdgeNegX;
            } else if (side == 2) {
                exists = tyi > 0;
                bsx = k + 1; bsy = 1; nsx = bsx; nsy = 0;
                dir = 3; out_bit = kEdgeNegY; in_bit = kEdgePosY;
            } else {
                exists = tyi + 1 < nty;
                bsx = k + 1; bsy = th; nsx = bsx; nsy = th + 1;
                dir = 0; out_bit = kEdgePosY; in_bit = kEdgeNegY;
            }
            if (!exists || s_push[side]) continue;
            const u64 lb = tile.lab[tile.li(l, bsy, bsx)];
            if (lb == kInf) continue;
            // the neighbour tile holds cells this net prices with its own overrides
            bool nb_over = false;
            if constexpr (OV) {
                const uint32_t u = side == 0 ? t - 1 : side == 1 ? t + 1 : side == 2 ? t - ntx : t + ntx;
                nb_over = f.n_over && a.tover[f.tile_off + u];
            }
            if constexpr (PL) {
                // the planes hold the price into the neighbour cell; an own pad or
                // endpoint of this net there is priced exactly
                const uint32_t gx_n = (uint32_t)(tx0 + (int)nsx - 1), gy_n = (uint32_t)(ty0 + (int)nsy - 1);
                const int pin = side == 0 ? kInPosX : side == 1 ? kInNegX : side == 2 ? kInPosY : kInNegY;
                const uint32_t wp = planes_pitch(b.w);
                uint32_t step = __ldg(b.planes + (uint64_t)pin * wp * b.h * L + ((uint64_t)l * b.h + gy_n) * wp + gx_n);
                if (step == kMax || nb_over)
                    step = exact_in_price(b, f, a.pads, pin, (l * b.h + gy_n) * b.w + gx_n, l, gy_n, gx_n);
                if (ext2(lb, step, 1) < tile.lab[tile.li(l, nsy, nsx)]) s_push[side] = 1;
                continue;
            }
            const uint32_t gn = (l * b.h + (uint32_t)(ty0 + (int)nsy - 1)) * b.w + (uint32_t)(tx0 + (int)nsx - 1);
            const uint8_t fb = tile.fl[(l * SH + bsy) * kFlPitch + bsx];
            const uint8_t fn = tile.fl[(l * SH + nsy) * kFlPitch + nsx];
            // the neighbour's enter cost and in-price, both loaded before either is used
            const uint32_t gx_n = (uint32_t)(tx0 + (int)nsx - 1), gy_n = (uint32_t)(ty0 + (int)nsy - 1);
            const uint32_t cn = __ldg(b.cost + gn);
            uint32_t base;
            if (b.directed)
                base = nb_over ? field_directed(b, f, gn, (int)dir)
                               : __ldg(reinterpret_cast<const uint32_t *>(b.directed + gn) + dir);
            else if (side == 0) base = __ldg(b.x_edge + gx_n);
            else if (side == 1) base = __ldg(b.x_edge + gx_n - 1);
            else if (side == 2) base = __ldg(b.y_edge + gy_n);
            else base = __ldg(b.y_edge + gy_n - 1);
            uint32_t en = kMax;  // cell_enter of the neighbour
            if (!(fn & kTraceNode)) en = cn != kMax ? cn : (is_own_pad(gn) ? 1u : kMax);
            if (en == kMax) continue;
            uint32_t step = kMax;  // planar_step_g on the loaded values
            if (!((fb & out_bit) | (fn & in_bit)) && !(b.directed && base == kMax)) step = capmul(base, en);
            const u64 cand = ext2(lb, step, 1);
            if (cand < tile.lab[tile.li(l, nsy, nsx)]) s_push[side] = 1;
        }
        __syncthreads();
        if (tid < 5) {
            __threadfence();  // labels before the visited flag and the queue entries
            if (tid == 4) {
                if constexpr (ASYNC) {
                    // nothing reads the visited words during a queue launch: a plain
                    // store; the work counters are per CTA (s_cnt), added to the
                    // launch's every kCountBatch activations and when the CTA exits,
                    // so this thread makes no round trip to L2 here
                    a.tvisit[f.tile_off + t] = 1u;
                    s_cnt[1] += sweep;
                    if (++s_cnt[0] == kCountBatch) {
                        if (atomicAdd(&ctl->activations, (unsigned long long)kCountBatch) + kCountBatch >
                            a.activation_limit)
                            atomicOr(&ctl->status, kStatusActivationLimit);
                        atomicAdd(&ctl->sweeps, s_cnt[1]);
                        s_cnt[0] = s_cnt[1] = 0;
                    }
                } else {
                    if (!s_vis[0]) atomicExch(a.tvisit + f.tile_off + t, 1u);
                    atomicAdd(&ctl->activations, 1ull);
                    atomicAdd(&ctl->sweeps, (unsigned long long)sweep);
                }
            } else if (s_push[tid]) {
                const uint32_t u = tid == 0 ? t - 1 : tid == 1 ? t + 1 : tid == 2 ? t - ntx : t + ntx;
                if constexpr (ASYNC) {
                    async_push(a, fi, f.tile_off, u);
                } else {
                    const uint32_t want = round + 2;  // stamp s = queued for round s-1
                    if (atomicMax(a.tstamp + f.tile_off + u, want) < want) {
                        const uint32_t nxt = (round + 1) % 3;
                        const uint32_t idx = atomicAdd(&ctl->count[nxt], 1u);
                        if (idx < cap) {
                            a.lists[(size_t)nxt * cap + idx] = ((u64)fi << 32) | u;
                        } else {
                            atomicOr(&ctl->status, kStatusQueueOverflow);
                        }
                    }
                }
            }
        }
        __syncthreads();
        if constexpr (!ASYNC) {
            break;
        } else {
            if (tid == 0) {
                // its own pushes are counted (the barrier above): release the tile
                // with one atomic, or, if a neighbour improved it meanwhile, hold it
                // again and continue, or queue it once more past the limit
                __threadfence();
                uint32_t *stw = a.tstamp + f.tile_off + t;
                s_more = 0;
                if (atomicCAS(stw, kTileHeld, kTileIdle) != kTileHeld) {  // held and dirty
                    if (cont + 1 < kContinueLimit) {
                        atomicExch(stw, kTileHeld);
                        s_more = 1;
                    } else {
                        atomicExch(stw, kTileQueued);
                        async_enqueue(a, fi, t);
                    }
                }
                if (!s_more) async_done(ctl);  // this item leaves the in-flight count
            }
            __syncthreads();
            if (!s_more) break;
            __threadfence();  // the neighbours' labels were written before they marked this tile
            if (tid < 4) s_push[tid] = 0;
            for (uint32_t i = tid; i < fell_words; i += blockDim.x) tile.fellw[i] = 0;
            // the halo ring again: an improved cell marks the line that ends at it
            const uint32_t nr = 2 * L * TH + 2 * L * kTW;
            for (uint32_t i = tid; i < nr; i += blockDim.x) {
                uint32_t l, sx, sy;
                bool row;
                if (i < 2 * L * TH) {
                    const uint32_t side = i >= L * TH, r = i - side * L * TH;
                    l = r / TH;
                    sy = r % TH + 1;
                    if (sy > th || (side ? txi + 1 >= ntx : txi == 0)) continue;
                    sx = side ? tw + 1 : 0;
                    row = true;
                } else {
                    const uint32_t k = i - 2 * L * TH, side = k >= L * kTW, r = k - side * L * kTW;
                    l = r / kTW;
                    sx = r % kTW + 1;
                    if (sx > tw || (side ? tyi + 1 >= nty : tyi == 0)) continue;
                    sy = side ? th + 1 : 0;
                    row = false;
                }
                const int gx = tx0 + (int)sx - 1, gy = ty0 + (int)sy - 1;
                const u64 v = __ldcg(lab + ((uint64_t)l * f.wh + (uint32_t)(gy - wy0)) * f.ww + (uint32_t)(gx - wx0));
                u64 &cur = tile.lab[tile.li(l, sy, sx)];
                if (v < cur) {
                    cur = v;
                    if (row) tile.rowd[l * TH + sy - 1] = 1;
                    else tile.cold[l * kTW + sx - 1] = 1;
                }
            }
            __syncthreads();
        }
    }
    __syncthreads();  // (queue form: the tile was released, or queued again, inside the loop)
}

template <int TH, int NT, bool OV>
__global__ void __launch_bounds__(NT) relax_rounds_kernel(RelaxArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ u64 s_item;
    Ctl *ctl = a.ctl;
    const uint32_t tid = threadIdx.x;
    const uint32_t cap = a.list_cap;
    // ---- round 0: every field's source tile ---------------------------------
    for (uint32_t fi = blockIdx.x * blockDim.x + tid; fi < a.n_fields; fi += gridDim.x * blockDim.x) {
        const DevField f = a.fields[fi];
        const DevBoard b = a.boards[f.board];
        const uint32_t plane = b.w * b.h;
        const uint32_t sr = f.src % plane, sx = sr % b.w, sy = sr / b.w;
        const uint8_t sfl = b.flags ? b.flags[f.src] : 0;
        if (sx >= f.x0 && sx < f.x0 + f.ww && sy >= f.y0 && sy < f.y0 + f.wh &&
            cell_enter(b, f, a.pads, f.src, sfl) != kMax) {
            const uint32_t ntx = (f.ww + kTW - 1) / kTW;
            const uint32_t t = ((sy - f.y0) / TH) * ntx + (sx - f.x0) / kTW;
            a.tstamp[f.tile_off + t] = 1u;
            const uint32_t idx = atomicAdd(&ctl->count[0], 1u);
            a.lists[idx] = ((u64)fi << 32) | t;
        }
    }
    grid_barrier(ctl, gridDim.x);

    for (uint32_t round = 0;; ++round) {
        const uint32_t cur = round % 3, old = (round + 2) % 3;
        const uint32_t n = *(volatile uint32_t *)&ctl->count[cur];
        if (n == 0 || ld_status(ctl)) break;
        if (round >= a.round_limit) {
            if (blockIdx.x == 0 && tid == 0) atomicOr(&ctl->status, kStatusRoundLimit);
            break;
        }
        if (blockIdx.x == 0 && tid == 0) {
            ctl->count[old] = 0;
            ctl->head[old] = 0;
            ctl->rounds = round + 1;
        }
        for (;;) {
            if (tid == 0) {
                const uint32_t idx = atomicAdd(&ctl->head[cur], 1u);
                s_item = idx < n ? __ldcg(a.lists + (size_t)cur * cap + idx) : kInf;
            }
            __syncthreads();
            const u64 item = s_item;
            if (item == kInf) break;
            uint32_t no_phase = 0;
            process_item<TH, false, false, OV>(a, (uint32_t)(item >> 32), (uint32_t)item, round, smem_raw, nullptr,
                                               no_phase, nullptr);
        }
        grid_barrier(ctl, gridDim.x);
    }
}

// Asynchronous form: no rounds.  Every CTA pops items from one ticketed queue
// and pushes the neighbours it improves; the launch ends when no item is
// queued or in flight.  The label arena is +inf-initialised (every label is
// valid from the start), and a tile is held by one CTA at a time: improvements
// that reach a held tile mark it dirty and its holder queues it once more.
// 64 registers a thread: four 256-thread CTAs per SM
template <int TH, int NT, bool PL, bool OV>
__global__ void __launch_bounds__(NT, 65536 / (NT * 64)) relax_async_kernel(RelaxArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ u64 s_item;
    __shared__ __align__(8) uint64_t s_mbar;  // completion of the price-plane TMA loads (PL)
    __shared__ unsigned long long s_cnt[2];  // this CTA's activations and sweeps not yet added to the launch's
    uint32_t tma_phase = 0;
    if (threadIdx.x == 0) {
        s_cnt[0] = s_cnt[1] = 0;
        if (PL) {
            mbar_init(&s_mbar, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) s_item = async_pop(a);
        __syncthreads();
        const u64 item = s_item;
        if (item == kInf) break;
        process_item<TH, true, PL, OV>(a, (uint32_t)(item >> 32), (uint32_t)item, 0, smem_raw, &s_mbar, tma_phase,
                                       s_cnt);
    }
    if (threadIdx.x == 0) {
        if (s_cnt[0]) atomicAdd(&a.ctl->activations, s_cnt[0]);
        if (s_cnt[1]) atomicAdd(&a.ctl->sweeps, s_cnt[1]);
    }
}

// Seeds of the asynchronous form: the source label and the source tile of
// every field whose source is inside its window and enterable.
template <int TH>
__global__ void async_seed_kernel(RelaxArgs a) {
    for (uint32_t fi = blockIdx.x * blockDim.x + threadIdx.x; fi < a.n_fields; fi += gridDim.x * blockDim.x) {
        const DevField f = a.fields[fi];
        const DevBoard b = a.boards[f.board];
        const uint32_t plane = b.w * b.h;
        const uint32_t sl = f.src / plane, sr = f.src % plane, sx = sr % b.w, sy = sr / b.w;
        const uint8_t sfl = b.flags ? b.flags[f.src] : 0;
        if (sx >= f.x0 && sx < f.x0 + f.ww && sy >= f.y0 && sy < f.y0 + f.wh &&
            cell_enter(b, f, a.pads, f.src, sfl) != kMax) {
            a.lab[f.lab_off + ((uint64_t)sl * f.wh + (sy - f.y0)) * f.ww + (sx - f.x0)] = 0;
            const uint32_t ntx = (f.ww + kTW - 1) / kTW;
            const uint32_t t = ((sy - f.y0) / TH) * ntx + (sx - f.x0) / kTW;
            __threadfence();
            async_push(a, fi, f.tile_off, t);
        }
    }
}

// Label of a window cell after the relax launch (unvisited tiles are unreached).
__device__ __forceinline__ u64 field_label(const PathArgs &a, const DevField &f, uint32_t lx, uint32_t ly,
                                           uint32_t l) {
    if (!a.arena_filled) {
        const uint32_t ntx = (f.ww + kTW - 1) / kTW;
        const uint32_t t = (ly >> (__ffs((int)a.tile_h) - 1)) * ntx + lx / kTW;  // tile heights are powers of two
        if (!a.tvisit[f.tile_off + t]) return kInf;
    }
    return a.lab[f.lab_off + ((uint64_t)l * f.wh + ly) * f.ww + lx];
}

// Per field: search cost and path length (hops[dst] + 1), then an exclusive
// scan into path offsets.  Single CTA; loops over the fields in chunks.
__global__ void __launch_bounds__(1024) path_offsets_kernel(PathArgs a) {
    __shared__ unsigned long long warp_sums[32];
    __shared__ unsigned long long carry;
    // phase 1: cost and length of every field, stored at its output slot
    for (uint32_t i = threadIdx.x; i < a.n_fields; i += blockDim.x) {
        const DevField f = a.fields[i];
        const DevBoard b = a.boards[f.board];
        const uint32_t plane = b.w * b.h;
        const uint32_t dl = f.dst / plane, dr = f.dst % plane;
        const uint32_t dx = dr % b.w, dy = dr / b.w;
        uint32_t cost = kMax, len = 0;
        if (dx >= f.x0 && dx < f.x0 + f.ww && dy >= f.y0 && dy < f.y0 + f.wh) {
            const u64 v = field_label(a, f, dx - f.x0, dy - f.y0, dl);
            cost = (uint32_t)(v >> 32);
            if (cost != kMax) len = (uint32_t)v + 1u;
            // a simple path never has more cells than its window
            if ((uint64_t)len > (uint64_t)f.ww * f.wh * b.layers) {
                atomicOr(a.status, kStatusPathBroken);
                len = 0;
            }
        }
        a.costs[f.out] = cost;
        a.lens[f.out] = len;
    }
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    // phase 2: exclusive scan of the lengths in output order
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint32_t base = 0; base < a.n_fields; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const unsigned long long v = (i < a.n_fields) ? (unsigned long long)a.lens[i] : 0ull;
        unsigned long long x = v;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) warp_sums[wid] = x;
        __syncthreads();
        if (wid == 0) {
            unsigned long long w = lane < (blockDim.x >> 5) ? warp_sums[lane] : 0ull;
            for (int o = 1; o < 32; o <<= 1) {
                unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, w, o);
                if (lane >= (uint32_t)o) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const unsigned long long excl = carry + (wid ? warp_sums[wid - 1] : 0ull) + x - v;
        if (i < a.n_fields) a.offsets[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) a.offsets[a.n_fields] = carry;
}

// Step price of the move p -> cur for the walk and the plain form.
// kind: 0 = p is cur's lower layer, 1 = -y, 2 = -x, 3 = +x, 4 = +y, 5 = upper layer.
__device__ __forceinline__ uint32_t global_step(const DevBoard &b, const DevField &f, const uint32_t *pads,
                                                uint32_t p, uint32_t cur, int kind) {
    const uint8_t fc = b.flags ? b.flags[cur] : 0, fp = b.flags ? b.flags[p] : 0;
    const uint32_t ec = cell_enter(b, f, pads, cur, fc);
    if (ec == kMax) return kMax;
    const uint32_t plane = b.w * b.h;
    const uint32_t r = cur % plane, x = r % b.w, y = r / b.w, l = cur / plane;
    if (kind == 0 || kind == 5) {
        const uint32_t k = kind == 0 ? l - 1 : l;
        if (!((b.via_mask >> k) & 1u)) return kMax;
        const uint8_t tc = cell_tile_flags(f, pads, cur, fc), tp = cell_tile_flags(f, pads, p, fp);
        if ((tc | tp) & kViaBlocked) return kMax;
        return capmul(__ldg(b.via_edge + k), ec);
    }
    uint8_t out_bit, in_bit;
    uint32_t base;
    if (kind == 1) {  // p at -y: p moves +y
        out_bit = kEdgePosY;
        in_bit = kEdgeNegY;
        base = b.directed ? field_directed(b, f, cur, 0) : __ldg(b.y_edge + y - 1);
    } else if (kind == 2) {  // p at -x: p moves +x
        out_bit = kEdgePosX;
        in_bit = kEdgeNegX;
        base = b.directed ? field_directed(b, f, cur, 1) : __ldg(b.x_edge + x - 1);
    } else if (kind == 3) {  // p at +x: p moves -x
        out_bit = kEdgeNegX;
        in_bit = kEdgePosX;
        base = b.directed ? field_directed(b, f, cur, 2) : __ldg(b.x_edge + x);
    } else {  // p at +y: p moves -y
        out_bit = kEdgeNegY;
        in_bit = kEdgePosY;
        base = b.directed ? field_directed(b, f, cur, 3) : __ldg(b.y_edge + y);
    }
    if ((fp & out_bit) | (fc & in_bit)) return kMax;
    if (b.directed && base == kMax) return kMax;
    return capmul(base, ec);
}

// global_step for the path walk with every load issued before any is used
// (the flags of both cells, the enter cost and the base price), so a step costs
// one memory round trip instead of a chain of dependent ones.
// own: cur's tile holds directed-price overrides of this field.
__device__ __forceinline__ uint32_t walk_step(const DevBoard &b, const DevField &f, const uint32_t *pads,
                                              uint32_t p, uint32_t cur, uint32_t x, uint32_t y, uint32_t l, int kind,
                                              bool own) {
    const uint8_t fc = b.flags ? __ldg(b.flags + cur) : 0, fp = b.flags ? __ldg(b.flags + p) : 0;
    const uint32_t cc = __ldg(b.cost + cur);
    uint32_t base = 0;
    if (kind == 0) base = __ldg(b.via_edge + l - 1);
    else if (kind == 5) base = __ldg(b.via_edge + l);
    else if (b.directed) {
        const int slot = kind == 1 ? 0 : kind == 2 ? 1 : kind == 3 ? 2 : 3;
        base = own ? field_directed(b, f, cur, slot)
                   : __ldg(reinterpret_cast<const uint32_t *>(b.directed + cur) + slot);
    }
    else if (kind == 1) base = __ldg(b.y_edge + y - 1);
    else if (kind == 2) base = __ldg(b.x_edge + x - 1);
    else if (kind == 3) base = __ldg(b.x_edge + x);
    else base = __ldg(b.y_edge + y);
    // cell_enter on the loaded values
    uint32_t ec;
    if (fc & kTraceNode) ec = kMax;
    else if (cc != kMax) ec = cc;
    else ec = (cur == f.src || cur == f.dst || sorted_has(pads + f.pad_off, f.n_pads, cur)) ? 1u : kMax;
    if (ec == kMax) return kMax;
    if (kind == 0 || kind == 5) {
        const uint32_t k = kind == 0 ? l - 1 : l;
        if (!((b.via_mask >> k) & 1u)) return kMax;
        const uint8_t tc = cell_tile_flags(f, pads, cur, fc), tp = cell_tile_flags(f, pads, p, fp);
        if ((tc | tp) & kViaBlocked) return kMax;
        return capmul(base, ec);
    }
    uint8_t out_bit, in_bit;
    if (kind == 1) {
        out_bit = kEdgePosY;
        in_bit = kEdgeNegY;
    } else if (kind == 2) {
        out_bit = kEdgePosX;
        in_bit = kEdgeNegX;
    } else if (kind == 3) {
        out_bit = kEdgeNegX;
        in_bit = kEdgePosX;
    } else {
        out_bit = kEdgeNegY;
        in_bit = kEdgePosY;
    }
    if ((fp & out_bit) | (fc & in_bit)) return kMax;
    if (b.directed && base == kMax) return kMax;
    return capmul(base, ec);
}

// Neighbour `kind` of (x, y, l): 0 the layer below, 1 -y, 2 -x, 3 +x, 4 +y,
// 5 the layer above (ascending CellIdx); kind 5 - k is the opposite of k.
__device__ __forceinline__ void walk_offset(int kind, int &x, int &y, int &l) {
    if (kind == 0) l -= 1;
    else if (kind == 1) y -= 1;
    else if (kind == 2) x -= 1;
    else if (kind == 3) x += 1;
    else if (kind == 4) y += 1;
    else l += 1;
}

// Label of window cell (x, y, l) (absolute coordinates inside the window), or
// +inf when its tile was never visited.
__device__ __forceinline__ u64 walk_label(const PathArgs &a, const DevField &f, uint32_t ntx, uint32_t tile_shift,
                                          int x, int y, int l) {
    const uint32_t lx = (uint32_t)x - f.x0, ly = (uint32_t)y - f.y0;
    const u64 raw = a.lab[f.lab_off + ((uint64_t)(uint32_t)l * f.wh + ly) * f.ww + lx];
    if (a.arena_filled) return raw;
    return a.tvisit[f.tile_off + (ly >> tile_shift) * ntx + lx / kTW] ? raw : kInf;
}

__device__ __forceinline__ bool walk_inside(const DevField &f, const DevBoard &b, int x, int y, int l) {
    return l >= 0 && l < (int)b.layers && x >= (int)f.x0 && x < (int)(f.x0 + f.ww) && y >= (int)f.y0 &&
           y < (int)(f.y0 + f.wh);
}

// Is the neighbour `kind` of target t = (tx, ty, tl) a predecessor of t, i.e.
// its label extended by the step into t equals `need`?  Its cell and label are
// returned for the caller to carry forward.
// (px, py, pl) is that neighbour, computed by the caller.
__device__ __forceinline__ bool walk_try(const PathArgs &a, const DevField &f, const DevBoard &b, uint32_t ntx,
                                         uint32_t tile_shift, int tx, int ty, int tl, uint32_t t, u64 need, int kind,
                                         int px, int py, int pl, uint32_t *q, u64 *lq) {
    if (!walk_inside(f, b, px, py, pl)) return false;
    *q = ((uint32_t)pl * b.h + (uint32_t)py) * b.w + (uint32_t)px;
    *lq = walk_label(a, f, ntx, tile_shift, px, py, pl);
    bool own = false;
    if (a.tover && f.n_over)
        own = a.tover[f.tile_off + (((uint32_t)ty - f.y0) >> tile_shift) * ntx + ((uint32_t)tx - f.x0) / kTW] != 0;
    const uint32_t st = walk_step(b, f, a.pads, *q, t, (uint32_t)tx, (uint32_t)ty, (uint32_t)tl, kind, own);
    return *lq != kInf && extend(*lq, st) == need;
}

// One warp per field: lanes 0..5 test the six neighbours of the current cell
// (ascending CellIdx) and the lowest qualifying one is the canonical
// predecessor.  Each step issues all of its loads at once (the candidate's
// label and tile flag, and the step inputs) and carries the winner's label and
// coordinates forward, so no step divides a cell index.
__global__ void __launch_bounds__(256) path_walk_kernel(PathArgs a) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (warp >= a.n_fields) return;
    const DevField f = a.fields[warp];
    const uint32_t len = a.lens[f.out];
    if (len == 0) return;
    const DevBoard b = a.boards[f.board];
    const uint32_t plane = b.w * b.h;
    const uint32_t ntx = (f.ww + kTW - 1) / kTW;
    const uint32_t tile_shift = (uint32_t)(__ffs((int)a.tile_h) - 1);  // tile heights are powers of two
    uint32_t *out = a.cells + a.offsets[f.out];
    uint32_t cur = f.dst;
    int cx, cy, cl;
    {
        const uint32_t r = cur % plane;
        cx = (int)(r % b.w);
        cy = (int)(r / b.w);
        cl = (int)(cur / plane);
    }
    u64 need = walk_label(a, f, ntx, tile_shift, cx, cy, cl);
    int ox = 0, oy = 0, oz = 0;  // this lane's neighbour offset (lanes 0-5), a loop constant
    if (lane < 6) walk_offset((int)lane, ox, oy, oz);
    for (uint32_t pos = len - 1;; --pos) {
        if (lane == 0) out[pos] = cur;
        if (pos == 0) {
            if (lane == 0 && cur != f.src) atomicOr(a.status, kStatusPathBroken);
            return;
        }
        bool ok = false;
        uint32_t p = 0;
        u64 lp = kInf;
        const int px = cx + ox, py = cy + oy, pz = cl + oz;
        if (lane < 6) {
            ok = walk_try(a, f, b, ntx, tile_shift, cx, cy, cl, cur, need, (int)lane, px, py, pz, &p, &lp);
        }
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, ok);
        if (m == 0) {
            if (lane == 0) atomicOr(a.status, kStatusPathBroken);
            return;
        }
        const uint32_t win = __ffs(m) - 1;
        cur = __shfl_sync(0xFFFFFFFFu, p, win);
        need = __shfl_sync(0xFFFFFFFFu, lp, win);
        cx = __shfl_sync(0xFFFFFFFFu, px, win);
        cy = __shfl_sync(0xFFFFFFFFu, py, win);
        cl = __shfl_sync(0xFFFFFFFFu, pz, win);
    }
}

// Complete u32 distance field of every field (MRC_FLAG_KEEP_FIELDS).
// `fields_by_offset` lists the fields in ascending lab_off order.
__global__ void emit_fields_kernel(PathArgs a, uint32_t *out, uint64_t total) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = a.n_fields;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (a.fields[mid].lab_off <= i) lo = mid;
            else hi = mid;
        }
        const DevField f = a.fields[lo];
        // a window has at most 2^32 cells (the CellIdx domain): 32-bit index math
        const uint32_t li = (uint32_t)(i - f.lab_off);
        const uint32_t rr = li / f.ww, lx = li - rr * f.ww;
        const uint32_t l = rr / f.wh, ly = rr - l * f.wh;
        out[i] = (uint32_t)(field_label(a, f, lx, ly, l) >> 32);
    }
}

// ---- the plain form: one Jacobi round over one field ----------------------
__global__ void plain_round_kernel(PlainArgs a) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const DevField f = a.field;
    const DevBoard b = a.board;
    const uint64_t wcells = (uint64_t)f.ww * f.wh * b.layers;
    if (i >= wcells) return;
    const uint32_t lx = (uint32_t)(i % f.ww);
    const uint64_t r = i / f.ww;
    const uint32_t ly = (uint32_t)(r % f.wh), l = (uint32_t)(r / f.wh);
    const uint32_t x = f.x0 + lx, y = f.y0 + ly;
    const uint32_t cur = (l * b.h + y) * b.w + x;
    const u64 old = a.in[i];
    u64 best = old;
    if (!(cur == f.src && best == 0)) {
        const int64_t plane_l = (int64_t)f.ww * f.wh;
        const int64_t off[6] = {-plane_l, -(int64_t)f.ww, -1, 1, (int64_t)f.ww, plane_l};
        const bool has[6] = {l > 0, ly > 0, lx > 0, lx + 1 < f.ww, ly + 1 < f.wh, l + 1 < b.layers};
        const int64_t goff[6] = {-(int64_t)b.w * b.h, -(int64_t)b.w, -1, 1, (int64_t)b.w, (int64_t)b.w * b.h};
        for (int k = 0; k < 6; ++k) {
            if (!has[k]) continue;
            const uint64_t j = (uint64_t)((int64_t)i + off[k]);
            const u64 lp = a.in[j];
            if (lp == kInf) continue;
            const uint32_t p = (uint32_t)((int64_t)cur + goff[k]);
            const u64 cand = extend(lp, global_step(b, f, a.pads, p, cur, k));
            if (cand < best) best = cand;
        }
    }
    a.out[i] = best;
    if (best != old) *a.changed = 1u;
}

// OR Grid::via_forbidden into the flag byte as kStaticVia.
__global__ void combine_flags_kernel(uint8_t *flags, const uint8_t *via_forbidden, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (via_forbidden[i]) flags[i] |= kStaticVia;
}

// ---- gather of page-locked host buffers into HBM ---------------------------
// One launch moves many host spans of one instance set to their places in a
// device block: the SMs read the host memory through its device mapping (PCIe
// reads, 16 bytes a thread, several in flight), so thousands of small and large
// spans cost one launch instead of one copy call each.  The spans are cut into
// 64 KiB chunks and the blocks stride over the chunks.

constexpr uint64_t kGatherChunk = 64u << 10;

// 0x80 in each nonzero byte of w, 0 elsewhere
__device__ __forceinline__ uint32_t nonzero_bytes(uint32_t w) {
    return (((w & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | w) & 0x80808080u;
}
static_assert(kStaticVia == 0x40, "the via-mask bit is the nonzero mark shifted by one");

__device__ __forceinline__ uint32_t flag_word(uint32_t board, uint32_t via) { return board | (nonzero_bytes(via) >> 1); }

__global__ void __launch_bounds__(256) host_gather_kernel(const HostSpan *spans, const uint64_t *chunk_start,
                                                          uint32_t n_spans, uint64_t n_chunks) {
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        // the span holding chunk c: the last s with chunk_start[s] <= c
        uint32_t lo = 0, hi = n_spans - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (chunk_start[mid] <= c) lo = mid; else hi = mid - 1;
        }
        const HostSpan sp = spans[lo];
        const uint64_t off = (c - chunk_start[lo]) * kGatherChunk;
        const uint64_t len = min(kGatherChunk, sp.bytes - off);
        const unsigned char *src = static_cast<const unsigned char *>(sp.src) + off;
        const unsigned char *src2 = static_cast<const unsigned char *>(sp.src2) + off;
        unsigned char *dst = static_cast<unsigned char *>(sp.dst) + off;
        const bool have_src = sp.src != nullptr, have_src2 = sp.src2 != nullptr;
        const uintptr_t align = (uintptr_t)dst | (have_src ? (uintptr_t)src : 0) | (have_src2 ? (uintptr_t)src2 : 0);
        uint64_t done = 0;
        if ((align & 15) == 0) {
            const uint64_t n16 = len / 16;
            constexpr int U = 4;
            for (uint64_t i0 = 0; i0 < n16; i0 += (uint64_t)U * blockDim.x) {
                uint4 a[U], b[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t i = i0 + (uint64_t)u * blockDim.x + threadIdx.x;
                    a[u] = make_uint4(0, 0, 0, 0);
                    b[u] = make_uint4(0, 0, 0, 0);
                    if (i < n16) {
                        if (have_src) a[u] = reinterpret_cast<const uint4 *>(src)[i];
                        if (sp.kind == 1 && have_src2) b[u] = reinterpret_cast<const uint4 *>(src2)[i];
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t i = i0 + (uint64_t)u * blockDim.x + threadIdx.x;
                    if (i >= n16) continue;
                    if (sp.kind == 1)
                        a[u] = make_uint4(flag_word(a[u].x, b[u].x), flag_word(a[u].y, b[u].y), flag_word(a[u].z, b[u].z),
                                          flag_word(a[u].w, b[u].w));
                    reinterpret_cast<uint4 *>(dst)[i] = a[u];
                }
            }
            done = n16 * 16;
        } else if ((align & 3) == 0 && sp.kind == 0) {
            const uint64_t n4 = len / 4;
            constexpr int U = 8;
            for (uint64_t i0 = 0; i0 < n4; i0 += (uint64_t)U * blockDim.x) {
                uint32_t a[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t i = i0 + (uint64_t)u * blockDim.x + threadIdx.x;
                    a[u] = (i < n4 && have_src) ? reinterpret_cast<const uint32_t *>(src)[i] : 0u;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t i = i0 + (uint64_t)u * blockDim.x + threadIdx.x;
                    if (i < n4) reinterpret_cast<uint32_t *>(dst)[i] = a[u];
                }
            }
            done = n4 * 4;
        }
        for (uint64_t i = done + threadIdx.x; i < len; i += blockDim.x) {
            uint8_t v = have_src ? src[i] : 0;
            if (sp.kind == 1 && have_src2 && src2[i]) v |= kStaticVia;
            dst[i] = v;
        }
    }
}

// ---- host-side launch helpers ---------------------------------------------

cudaError_t host_gather_launch(const HostSpan *spans, const uint64_t *chunk_start, uint32_t n_spans, uint64_t n_chunks,
                               uint32_t sms, cudaStream_t st) {
    if (!n_spans || !n_chunks) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>(n_chunks, (uint64_t)sms * 8);
    host_gather_kernel<<<(uint32_t)blocks, 256, 0, st>>>(spans, chunk_start, n_spans, n_chunks);
    return cudaGetLastError();
}

uint64_t host_gather_chunks(uint64_t bytes) { return (bytes + kGatherChunk - 1) / kGatherChunk; }

cudaError_t combine_flags_launch(uint8_t *flags, const uint8_t *via_forbidden, uint64_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 4096);
    combine_flags_kernel<<<(uint32_t)blocks, 256, 0, st>>>(flags, via_forbidden, n);
    return cudaGetLastError();
}

size_t relax_smem_bytes(uint32_t layers, uint32_t tile_h, bool directed, bool planes) {
    (void)directed;  // directed prices are folded into the step planes
    return tile_layout(layers, tile_h, planes).total;
}

namespace {
template <int TH>
const void *relax_fn_th(bool wide, bool async, bool planes) {
    if (async && planes)
        return wide ? (const void *)relax_async_kernel<TH, 256, true, false>
                    : (const void *)relax_async_kernel<TH, 128, true, false>;
    if (async)
        return wide ? (const void *)relax_async_kernel<TH, 256, false, false>
                    : (const void *)relax_async_kernel<TH, 128, false, false>;
    return wide ? (const void *)relax_rounds_kernel<TH, 256, false> : (const void *)relax_rounds_kernel<TH, 128, false>;
}

const void *relax_fn(uint32_t tile_h, uint32_t threads, bool async, bool planes, bool over) {
    if (over) {  // the override variants exist for the 8 x 256 configuration only
        if (tile_h != kOverTileH || threads != kOverThreads) return nullptr;
        if (async && planes) return (const void *)relax_async_kernel<kOverTileH, kOverThreads, true, true>;
        if (async) return (const void *)relax_async_kernel<kOverTileH, kOverThreads, false, true>;
        return (const void *)relax_rounds_kernel<kOverTileH, kOverThreads, true>;
    }
    const bool wide = threads >= 256;
    switch (tile_h) {
        case 8: return relax_fn_th<8>(wide, async, planes);
        case 16: return relax_fn_th<16>(wide, async, planes);
        case 32: return relax_fn_th<32>(wide, async, planes);
        default: return relax_fn_th<64>(wide, async, planes);
    }
}

const void *seed_fn(uint32_t tile_h) {
    switch (tile_h) {
        case 8: return (const void *)async_seed_kernel<8>;
        case 16: return (const void *)async_seed_kernel<16>;
        case 32: return (const void *)async_seed_kernel<32>;
        default: return (const void *)async_seed_kernel<64>;
    }
}
}  // namespace

cudaError_t relax_configure(uint32_t tile_h, uint32_t threads, size_t smem, bool async, bool planes, bool over) {
    const void *fn = relax_fn(tile_h, threads, async, planes, over);
    if (!fn) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

cudaError_t relax_occupancy(uint32_t tile_h, uint32_t threads, size_t smem, int *blocks_per_sm, bool async,
                            bool planes, bool over) {
    const void *fn = relax_fn(tile_h, threads, async, planes, over);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, (int)threads, smem);
}

cudaError_t relax_launch(const RelaxArgs &a, uint32_t grid, uint32_t threads, size_t smem, cudaStream_t st,
                         bool async, bool planes, bool over) {
    const void *fn = relax_fn(a.tile_h, threads, async, planes, over);
    if (!fn) return cudaErrorInvalidValue;
    RelaxArgs copy = a;
    void *args[] = {&copy};
    if (async) {
        // seeds, then the queue-driven kernel (a plain launch: no grid barrier,
        // and a CTA only takes a ticket while it is resident)
        if (a.n_fields) {
            cudaError_t e = cudaLaunchKernel(seed_fn(a.tile_h), dim3((a.n_fields + 255) / 256), dim3(256), args, 0, st);
            if (e != cudaSuccess) return e;
        }
        return cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, smem, st);
    }
    // Cooperative (all CTAs co-resident, checked by the CUDA runtime against occupancy);
    // the attribute form is also what stream capture records as a graph node.
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

// Tile-staged walk, for batches whose boards carry price planes and a TMA map
// (the CTA queue form) and whose nets carry no price overrides.  One CTA per
// field stages a walk tile of 32 x WH cells over all layers — the labels with a
// one-cell ring by plain loads, the six price planes by WH / tile_h TMA loads of
// the relax kernel's box — and warp 0 walks inside it from shared memory,
// re-staging when the path leaves the tile.  A step then costs shared-memory
// reads instead of a round trip to L2 or HBM.  The step prices are the planes'
// except on the stacks of the net's endpoints, and for every step of a net with
// own or via pads, where walk_step prices exactly; the choice among the
// candidates is path_walk_kernel's.
//
// Origin of the walk tile along one axis of extent e for a walk at c heading in
// direction d (-1, 0, +1): a few cells behind c, so most of the tile lies ahead.
// A walk heading diagonally then leaves a tile through one side instead of two.
__device__ __forceinline__ int walk_origin(int c, int d, int e) {
    const int back = e / 8;
    return d > 0 ? c - back : d < 0 ? c - (e - 1 - back) : c - e / 2;
}

__device__ __forceinline__ int walk_dir(int from, int to) { return to > from ? 1 : to < from ? -1 : 0; }

// The exact step price, out of line: the tiled walk needs it only on the
// endpoints' stacks and for nets with own pads, so its loads and branches stay
// out of the common step's code.
// It reads the board and field records from global memory (L1-resident after
// the first call) so the caller's copies stay in registers.
__device__ __noinline__ uint32_t walk_step_exact(const DevBoard *b, const DevField *f, const uint32_t *pads,
                                                 uint32_t p, uint32_t cur, uint32_t x, uint32_t y, uint32_t l,
                                                 int kind) {
    return walk_step(*b, *f, pads, p, cur, x, y, l, kind, false);
}

__global__ void __launch_bounds__(256) path_walk_tiled_kernel(PathArgs a) {
    extern __shared__ __align__(128) unsigned char wsm[];
    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ int s_tile[2];   // walk tile origin (board x, y)
    __shared__ uint32_t s_done;
    const DevField f = a.fields[blockIdx.x];
    const uint32_t len = a.lens[f.out];
    if (len == 0) return;  // the same for the whole CTA
    const DevBoard b = a.boards[f.board];
    const uint32_t L = b.layers, TH = a.tile_h, WH = walk_tile_rows(TH), nload = WH / TH;
    const uint32_t plane = b.w * b.h;
    uint32_t *pl = reinterpret_cast<uint32_t *>(wsm);
    u64 *lab = reinterpret_cast<u64 *>(wsm + walk_smem_planes(L, TH));
    const uint32_t box_words = 6 * L * TH * kPlaneTmaBoxW;
    const bool exact_all = (f.n_pads | f.n_vpads) != 0;
    const uint32_t src_xy = f.src % plane, dst_xy = f.dst % plane;
    const int sx = (int)(src_xy % b.w), sy = (int)(src_xy / b.w);  // the walk heads for the source
    const int dstx = (int)(dst_xy % b.w), dsty = (int)(dst_xy / b.w);
    const int wx0 = (int)f.x0, wy0 = (int)f.y0, wx1 = (int)(f.x0 + f.ww), wy1 = (int)(f.y0 + f.wh);
    const uint32_t lane = threadIdx.x & 31;
    uint32_t *out = a.cells + a.offsets[f.out];
    // walk state (warp 0)
    uint32_t cur = f.dst, pos = len - 1;
    int cx = (int)((f.dst % plane) % b.w), cy = (int)((f.dst % plane) / b.w), cl = (int)(f.dst / plane);
    u64 need = a.lab[f.lab_off + ((uint64_t)(uint32_t)cl * f.wh + (uint32_t)(cy - wy0)) * f.ww + (uint32_t)(cx - wx0)];
    uint32_t phase = 0;
    // Per-lane constants of a step: the neighbour offset of kind `lane` (lanes 0-5),
    // the in-price plane of the move from it into the current cell, and the
    // relax tile height as a shift (tile heights are powers of two).
    int ox = 0, oy = 0, oz = 0;
    if (lane < 6) walk_offset((int)lane, ox, oy, oz);
    const uint32_t pin = lane == 0 ? kInBelow : lane == 1 ? kInNegY : lane == 2 ? kInNegX
                       : lane == 3 ? kInPosX : lane == 4 ? kInPosY : kInAbove;
    const uint32_t th_shift = (uint32_t)__ffs((int)TH) - 1u;
    if (threadIdx.x == 0) {
        mbar_init(&s_mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_tile[0] = walk_origin(cx, walk_dir(cx, sx), (int)kTW);
        s_tile[1] = walk_origin(cy, walk_dir(cy, sy), (int)WH);
        s_done = 0;
    }
    for (;;) {
        __syncthreads();
        const int tx0 = s_tile[0], ty0 = s_tile[1];
        const uint32_t xo = (uint32_t)tx0 & 3u;
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            mbar_expect_tx(&s_mbar, nload * box_words * 4u);
            for (uint32_t j = 0; j < nload; ++j)
                tma_load_4d(pl + j * box_words, b.tmap, tx0 & ~3, ty0 + (int)(j * TH), 0, 0, &s_mbar);
        }
        // labels of the tile and its ring (+inf outside the window), kStageBatch
        // loads in flight per thread before any is stored
        const uint32_t nl = L * (WH + 2) * 34;
        constexpr uint32_t kStageBatch = 8;
        for (uint32_t i0 = threadIdx.x; i0 < nl; i0 += kStageBatch * blockDim.x) {
            u64 v[kStageBatch];
#pragma unroll
            for (uint32_t k = 0; k < kStageBatch; ++k) {
                const uint32_t i = i0 + k * blockDim.x;
                const uint32_t sx = i % 34, r = i / 34, sy = r % (WH + 2), l = r / (WH + 2);
                const int gx = tx0 + (int)sx - 1, gy = ty0 + (int)sy - 1;
                v[k] = kInf;
                if (i < nl && gx >= wx0 && gx < wx1 && gy >= wy0 && gy < wy1)
                    v[k] = __ldcg(a.lab + f.lab_off + ((uint64_t)l * f.wh + (uint32_t)(gy - wy0)) * f.ww +
                                  (uint32_t)(gx - wx0));
            }
#pragma unroll
            for (uint32_t k = 0; k < kStageBatch; ++k)
                if (i0 + k * blockDim.x < nl) lab[i0 + k * blockDim.x] = v[k];
        }
        // bounded wait for the planes (a load that never lands breaks the path)
        for (uint32_t spins = 0; !mbar_try_wait(&s_mbar, phase & 1u); ++spins) {
            if (spins > kTmaSpinLimit) {
                if (threadIdx.x == 0) {
                    atomicOr(a.status, kStatusPathBroken);
                    s_done = 1;
                }
                break;
            }
        }
        ++phase;
        __syncthreads();
        if (s_done) return;
        if (threadIdx.x < 32) {
            for (;;) {
                if (lane == 0) out[pos] = cur;
                if (pos == 0) {
                    if (lane == 0) {
                        if (cur != f.src) atomicOr(a.status, kStatusPathBroken);
                        s_done = 1;
                    }
                    break;
                }
                bool ok = false;
                uint32_t p = 0;
                u64 lp = kInf;
                const int px = cx + ox, py = cy + oy, pz = cl + oz;
                if (lane < 6 && walk_inside(f, b, px, py, pz)) {
                    p = ((uint32_t)pz * b.h + (uint32_t)py) * b.w + (uint32_t)px;
                    lp = lab[((uint32_t)pz * (WH + 2) + (uint32_t)(py - ty0 + 1)) * 34 + (uint32_t)(px - tx0 + 1)];
                    uint32_t st;
                    if (exact_all || (cx == sx && cy == sy) || (cx == dstx && cy == dsty)) {
                        st = walk_step_exact(a.boards + f.board, a.fields + blockIdx.x, a.pads, p, cur, (uint32_t)cx,
                                             (uint32_t)cy, (uint32_t)cl, (int)lane);
                    } else {
                        // in-price plane `pin` at cur, from the TMA box of cur's relax-tile rows
                        const uint32_t yy = (uint32_t)(cy - ty0), j = yy >> th_shift;
                        st = pl[j * box_words + ((pin * L + (uint32_t)cl) * TH + (yy & (TH - 1u))) * kPlaneTmaBoxW +
                                (uint32_t)(cx - tx0) + xo];
                    }
                    ok = lp != kInf && extend(lp, st) == need;
                }
                const uint32_t m = __ballot_sync(0xFFFFFFFFu, ok);
                if (m == 0) {
                    if (lane == 0) {
                        atomicOr(a.status, kStatusPathBroken);
                        s_done = 1;
                    }
                    break;
                }
                const uint32_t win = __ffs(m) - 1;
                cur = __shfl_sync(0xFFFFFFFFu, p, win);
                need = __shfl_sync(0xFFFFFFFFu, lp, win);
                cx = __shfl_sync(0xFFFFFFFFu, px, win);
                cy = __shfl_sync(0xFFFFFFFFu, py, win);
                cl = __shfl_sync(0xFFFFFFFFu, pz, win);
                --pos;
                if (cx < tx0 || cx >= tx0 + (int)kTW || cy < ty0 || cy >= ty0 + (int)WH) {
                    if (lane == 0) {  // the path left the tile: stage one ahead of cur
                        const int dx = cx < tx0 ? -1 : cx >= tx0 + (int)kTW ? 1 : walk_dir(cx, sx);
                        const int dy = cy < ty0 ? -1 : cy >= ty0 + (int)WH ? 1 : walk_dir(cy, sy);
                        s_tile[0] = walk_origin(cx, dx, (int)kTW);
                        s_tile[1] = walk_origin(cy, dy, (int)WH);
                    }
                    break;
                }
            }
        }
        __syncthreads();
        if (s_done) return;
    }
}

namespace {
// One warp per field: every override cell inside the window flags its tile.
__global__ void mark_over_tiles_kernel(const DevField *fields, uint32_t n_fields, const DevBoard *boards,
                                       uint32_t tile_h, uint8_t *tover) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t fi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; fi < n_fields; fi += warps) {
        const DevField f = fields[fi];
        if (!f.n_over) continue;
        const DevBoard b = boards[f.board];
        const uint32_t plane = b.w * b.h, ntx = (f.ww + kTW - 1) / kTW;
        for (uint32_t k = lane; k < f.n_over; k += 32) {
            const uint32_t c = b.over_cells[f.over_off + k], r = c % plane, x = r % b.w, y = r / b.w;
            if (x < f.x0 || x >= f.x0 + f.ww || y < f.y0 || y >= f.y0 + f.wh) continue;
            tover[f.tile_off + ((y - f.y0) / tile_h) * ntx + (x - f.x0) / kTW] = 1;
        }
    }
}
}  // namespace

cudaError_t mark_over_tiles_launch(const DevField *fields, uint32_t n_fields, const DevBoard *boards, uint32_t tile_h,
                                   uint8_t *tover, cudaStream_t st) {
    if (!n_fields) return cudaSuccess;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>(((uint64_t)n_fields * 32 + 255) / 256, 148ull * 16);
    mark_over_tiles_kernel<<<blocks, 256, 0, st>>>(fields, n_fields, boards, tile_h, tover);
    return cudaGetLastError();
}

cudaError_t path_launch(const PathArgs &a, cudaStream_t st) {
    path_offsets_kernel<<<1, 1024, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.n_fields && a.walk_smem) {
        e = cudaFuncSetAttribute(path_walk_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)a.walk_smem);
        if (e != cudaSuccess) return e;
        path_walk_tiled_kernel<<<a.n_fields, 256, a.walk_smem, st>>>(a);
    } else if (a.n_fields) {
        const uint32_t warps_per_block = 8;
        path_walk_kernel<<<(a.n_fields + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, st>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t fields_launch(const PathArgs &a, uint32_t *out, uint64_t total, cudaStream_t st) {
    if (total == 0 || a.n_fields == 0) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>((total + 255) / 256, 8192);
    emit_fields_kernel<<<(uint32_t)blocks, 256, 0, st>>>(a, out, total);
    return cudaGetLastError();
}

cudaError_t plain_round_launch(const PlainArgs &a, uint64_t wcells, cudaStream_t st) {
    const uint32_t threads = 256;
    plain_round_kernel<<<(uint32_t)((wcells + threads - 1) / threads), threads, 0, st>>>(a);
    return cudaGetLastError();
}

// Self-test of the bounded wait: one CTA waits at the grid barrier for a CTA
// that does not exist, so the wait must give up after `spins` polls, record
// kStatusBarrier and return with the context intact.
__global__ void wait_selftest_kernel(Ctl *c, uint32_t spins) { grid_barrier(c, gridDim.x + 1, spins); }

cudaError_t wait_selftest_launch(Ctl *c, uint32_t spins, cudaStream_t st) {
    wait_selftest_kernel<<<1, 32, 0, st>>>(c, spins);
    return cudaGetLastError();
}

}  // namespace mrc
