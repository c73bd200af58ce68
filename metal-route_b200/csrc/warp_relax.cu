// warp_relax.cu — the warp-per-tile relax schedule and the step-price planes it reads.
//
// planes_kernel: per board, six u32 planes of N cells: the price of the step
// INTO cell c from its neighbour at -x, +x, -y, +y, the layer below and the
// layer above, under every rule that does not depend on the net (enter weight
// of cost[c], board trace-node / directed-edge / via-node bits, the static via
// mask, the via transitions, directed edge prices and the saturating product;
// negotiated.rs:2914-2966 and :3010-3043).  kMax = no such step.  The rules
// that do depend on the net — an obstacle that is one of its own pads (or an
// endpoint) is entered at weight 1, and its via pads are exempt from the static
// via mask — only touch the (y, x) stacks of those cells; the relax kernel
// recomputes every price of such a stack exactly (exact_in_price).
//
// relax_warp_kernel: one warp holds one tile of TW x 8 cells over all L layers
// of a field in registers.  Lane (l, seg) owns the 4 consecutive cells
// x = 4 seg .. 4 seg + 3 of every row y of layer l (S = 32 / next_pow2(L)
// segments per row, TW = 4 S).  A tile relaxes with three kinds of pass:
//   (+y)  rows top to bottom: each row first takes the step down from the row
//         above (registers, or the halo row), then is closed along x in both
//         directions at once (segmented min-plus scans across its S lanes);
//   (-y)  the mirror image, rows bottom to top;
//   stack the layer stacks of the changed rows, through a shared-memory row.
// A (+y) pass alone settles every path that runs down-monotone with any
// left/right moves, whatever its number of turns, so a tile converges in a few
// passes where alternating row and column sweeps need one sweep per turn.
// Per-row bookkeeping (rows not closed along x, rows whose neighbour row fell
// since their last vertical step, rows whose stacks changed) skips every row a
// pass cannot change; the tile is converged when no row is marked.  There are
// no CTA barriers: the warps of a CTA work on unrelated tiles of the same
// ticketed queue as the CTA-wide asynchronous schedule (tiles.cuh).
#include <cuda_runtime.h>

#include <algorithm>

#include "device.cuh"
#include "kernels.h"
#include "tiles.cuh"

namespace mrc {

namespace {

constexpr int K = kWarpLaneCells;  // cells per lane per row
constexpr int TH = kWarpTileH;     // rows per tile
constexpr int NW = 4;              // warps per CTA
constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint64_t kPlaneChunk = 8192;
constexpr uint32_t kMaxRounds = 8;  // relaxation rounds of one activation (see warp_item)

// ---- step-price planes ------------------------------------------------------

__device__ __forceinline__ bool via_blocked_board(uint8_t fl) { return (fl & (kViaNode | kStaticVia)) != 0; }

__global__ void __launch_bounds__(256) planes_kernel(const DevBoard *boards, const uint64_t *chunk_start,
                                                     uint32_t n_boards, uint64_t n_chunks) {
    for (uint64_t ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
        uint32_t lo = 0, hi = n_boards - 1;  // the last board whose first chunk is <= ch
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (chunk_start[mid] <= ch) lo = mid;
            else hi = mid - 1;
        }
        const DevBoard b = boards[lo];
        const uint32_t plane = b.w * b.h;
        const uint64_t N = (uint64_t)plane * b.layers;
        const uint32_t wp = planes_pitch(b.w);
        const uint64_t NP = (uint64_t)wp * b.h * b.layers;  // cells of one plane, rows padded
        const uint64_t c0 = (ch - chunk_start[lo]) * kPlaneChunk, c1 = min(c0 + kPlaneChunk, N);
        uint32_t *out = b.planes;
        for (uint64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
            const uint32_t c = (uint32_t)i;
            const uint32_t l = c / plane, r = c - l * plane, y = r / b.w, x = r - y * b.w;
            const uint8_t fc = b.flags ? __ldg(b.flags + c) : 0;
            const uint32_t cost = __ldg(b.cost + c);
            const uint32_t ec = (fc & kTraceNode) ? kMax : cost;  // obstacles stay kMax here
            uint32_t s[6] = {kMax, kMax, kMax, kMax, kMax, kMax};
            if (ec != kMax) {
                uint4 d = make_uint4(0, 0, 0, 0);
                if (b.directed) d = __ldg(b.directed + c);
                auto planar = [&](uint32_t base, uint32_t p, uint8_t out_bit, uint8_t in_bit) -> uint32_t {
                    const uint8_t fp = b.flags ? __ldg(b.flags + p) : 0;
                    if ((fp & out_bit) | (fc & in_bit)) return kMax;
                    if (b.directed && base == kMax) return kMax;
                    return capmul(base, ec);
                };
                if (x > 0) s[kInNegX] = planar(b.directed ? d.y : __ldg(b.x_edge + x - 1), c - 1, kEdgePosX, kEdgeNegX);
                if (x + 1 < b.w) s[kInPosX] = planar(b.directed ? d.z : __ldg(b.x_edge + x), c + 1, kEdgeNegX, kEdgePosX);
                if (y > 0) s[kInNegY] = planar(b.directed ? d.x : __ldg(b.y_edge + y - 1), c - b.w, kEdgePosY, kEdgeNegY);
                if (y + 1 < b.h) s[kInPosY] = planar(b.directed ? d.w : __ldg(b.y_edge + y), c + b.w, kEdgeNegY, kEdgePosY);
                if (b.layers > 1 && !via_blocked_board(fc)) {
                    if (l > 0 && ((b.via_mask >> (l - 1)) & 1u)) {
                        const uint8_t fq = b.flags ? __ldg(b.flags + c - plane) : 0;
                        if (!via_blocked_board(fq)) s[kInBelow] = capmul(__ldg(b.via_edge + l - 1), ec);
                    }
                    if (l + 1 < b.layers && ((b.via_mask >> l) & 1u)) {
                        const uint8_t fq = b.flags ? __ldg(b.flags + c + plane) : 0;
                        if (!via_blocked_board(fq)) s[kInAbove] = capmul(__ldg(b.via_edge + l), ec);
                    }
                }
            }
            const uint64_t o = ((uint64_t)l * b.h + y) * wp + x;
#pragma unroll
            for (int p = 0; p < 6; ++p) out[(uint64_t)p * NP + o] = s[p];
        }
    }
}

// ---- one tile held by one warp ---------------------------------------------

// Per-warp shared memory.  The tile's labels live here rather than in
// registers: the row loops then run with a runtime row index (one compact copy
// of the pass code instead of fully unrolled passes, which overflowed the
// instruction cache) and the stack pass works on the labels in place.
struct WarpSmem {
    u64 lab[TH][K][32];  // the tile: lane (l, seg) owns lab[y][0..K)[lane], x = 4 seg + i (i-major: no bank conflicts)
    u64 htb[2][128];     // halo rows above (0) and below (1) the tile, [l * TW + x]
    u64 hlr[2][128];     // halo columns left (0) and right (1), [l * TH + y]
    uint32_t spec[32];   // bit y * TW + x: the (y, x) stack holds an endpoint, own pad or via pad
    uint32_t fell[32];   // per lane: bits y * K + i of its cells that the stack pass lowered
};

struct WTile {
    const DevBoard *bp;           // the board and field (read again only for exact prices)
    const DevField *fp;
    const uint32_t *pads;
    const uint32_t *planes;
    uint64_t NP;                  // cells of one price plane (rows padded to wp)
    uint32_t w, h, wp;            // board plane extent, price-plane row pitch
    uint32_t L, S, TW, tw_shift;  // layers, segments per row, tile width (= 1 << tw_shift)
    uint32_t l, lc, seg, xb;      // this lane's layer (clamped copy for addresses), segment, first column
    uint32_t tx0, ty0, tw, th;    // tile origin (board coordinates) and valid extent
    uint32_t wx1, wy1;            // window end (exclusive)
    bool act;                     // lane holds cells (l < L)
};

__device__ __noinline__ uint32_t exact_price_t(const WTile &t, int dir, uint32_t c, uint32_t l, uint32_t y,
                                               uint32_t x) {
    const DevBoard b = *t.bp;
    const DevField f = *t.fp;
    return exact_in_price(b, f, t.pads, dir, c, l, y, x);
}

// Price plane p at (layer l, board row y, board column x).
__device__ __forceinline__ uint32_t plane_at(const WTile &t, int p, uint32_t l, uint32_t y, uint32_t x) {
    return __ldg(t.planes + (uint64_t)p * t.NP + ((uint64_t)l * t.h + y) * t.wp + x);
}

// Price into the tile cell (layer l, tile row y, tile column x).
__device__ __forceinline__ uint32_t tile_price(const WTile &t, const WarpSmem &sm, int p, uint32_t l, uint32_t y,
                                               uint32_t x) {
    const uint32_t gy = t.ty0 + y, gx = t.tx0 + x;
    const uint32_t c = (l * t.h + gy) * t.w + gx;
    const uint32_t bit = (y << t.tw_shift) + x;
    if ((sm.spec[bit >> 5] >> (bit & 31)) & 1u) return exact_price_t(t, p, c, l, gy, gx);
    return plane_at(t, p, l, gy, gx);
}

// Prices into this lane's K cells of tile row y: from -x, from +x and from the
// vertical direction `pv_dir`.  Cells past the window edge read a clamped
// (valid) address; their labels are forced to +inf anyway.
__device__ __forceinline__ void row_prices(const WTile &t, int y, int pv_dir, uint32_t spec_lane, uint32_t (&pnx)[K],
                                           uint32_t (&ppx)[K], uint32_t (&pv)[K]) {
    const uint32_t gy = min(t.ty0 + (uint32_t)y, t.wy1 - 1);
    const uint32_t rowc = (t.lc * t.h + gy) * t.w;
    const uint32_t *row = t.planes + ((uint64_t)t.lc * t.h + gy) * t.wp;
    uint32_t gx[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        gx[i] = min(t.tx0 + t.xb + i, t.wx1 - 1);
        pnx[i] = __ldg(row + gx[i]);
        ppx[i] = __ldg(row + t.NP + gx[i]);
        pv[i] = __ldg(row + (uint64_t)pv_dir * t.NP + gx[i]);
    }
    const uint32_t sb = (spec_lane >> (y * K)) & ((1u << K) - 1u);
    if (sb) {
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (!((sb >> i) & 1u)) continue;
            const uint32_t c = rowc + gx[i];
            pnx[i] = exact_price_t(t, kInNegX, c, t.lc, gy, gx[i]);
            ppx[i] = exact_price_t(t, kInPosX, c, t.lc, gy, gx[i]);
            pv[i] = exact_price_t(t, pv_dir, c, t.lc, gy, gx[i]);
        }
    }
}

// Close one row along x in both directions: each lane's K cells run their own
// chain, the S lanes of the row combine transfer functions
// f(t) = min(A, t (+) (D, hops)) with a Kogge-Stone scan (forward: shuffles up
// from the left halo `hl`; backward: shuffles down from the right halo `hr`,
// on the forward results), and every cell takes the best incoming label.
// pnx[i] prices the move into cell i from its left neighbour, ppx[i] from its
// right neighbour.
__device__ __forceinline__ void row_close(u64 (&u)[K], const uint32_t (&pnx)[K], const uint32_t (&ppx)[K], u64 hl,
                                          u64 hr, uint32_t S, uint32_t seg) {
    uint32_t P[K];
    // forward
    P[0] = pnx[0];
#pragma unroll
    for (int i = 1; i < K; ++i) {
        u[i] = umin64(u[i], ext2(u[i - 1], pnx[i], 1));
        P[i] = dsum(P[i - 1], pnx[i]);
    }
    {
        u64 A = u[K - 1];
        uint32_t D = P[K - 1];
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            if (o >= S) break;
            const u64 Ap = __shfl_up_sync(kFull, A, o, S);
            const uint32_t Dp = __shfl_up_sync(kFull, D, o, S);
            if (seg >= o) {
                A = umin64(A, ext2(Ap, D, K * o));
                D = dsum(Dp, D);
            }
        }
        u64 C = hl;
        if (S > 1) {
            const u64 Fa = __shfl_up_sync(kFull, A, 1, S);
            const uint32_t Fd = __shfl_up_sync(kFull, D, 1, S);
            if (seg > 0) C = umin64(Fa, ext2(hl, Fd, K * seg));
        }
        if (C != kInf) {
#pragma unroll
            for (int i = 0; i < K; ++i) u[i] = umin64(u[i], ext2(C, P[i], (uint32_t)i + 1u));
        }
    }
    // backward, on the forward results
    {
        const uint32_t sbk = S - 1 - seg;
        P[K - 1] = ppx[K - 1];
#pragma unroll
        for (int i = K - 2; i >= 0; --i) {
            u[i] = umin64(u[i], ext2(u[i + 1], ppx[i], 1));
            P[i] = dsum(P[i + 1], ppx[i]);
        }
        u64 A = u[0];
        uint32_t D = P[0];
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            if (o >= S) break;
            const u64 Ap = __shfl_down_sync(kFull, A, o, S);
            const uint32_t Dp = __shfl_down_sync(kFull, D, o, S);
            if (sbk >= o) {
                A = umin64(A, ext2(Ap, D, K * o));
                D = dsum(Dp, D);
            }
        }
        u64 C = hr;
        if (S > 1) {
            const u64 Fa = __shfl_down_sync(kFull, A, 1, S);
            const uint32_t Fd = __shfl_down_sync(kFull, D, 1, S);
            if (sbk > 0) C = umin64(Fa, ext2(hr, Fd, K * sbk));
        }
        if (C != kInf) {
#pragma unroll
            for (int i = 0; i < K; ++i) u[i] = umin64(u[i], ext2(C, P[i], (uint32_t)(K - i)));
        }
    }
}

// Row bookkeeping (warp-uniform bit masks over the tile rows):
//   H  rows not closed along x since they last changed outside a row pass
//   D  rows whose upper neighbour fell since their last step down from it
//   U  rows whose lower neighbour fell since their last step up from it
//   ST rows whose layer stacks changed since their last stack pass
struct RowMarks {
    uint32_t H, D, U, ST;
};

// A (+y) pass (down) or a (-y) pass over the marked rows.  One copy of the
// code serves both directions: only the neighbour row, its halo and the
// vertical price plane differ.
__device__ __forceinline__ void vert_pass(const WTile &t, WarpSmem &sm, bool down, RowMarks &m, uint32_t spec_lane,
                                       uint32_t valid, uint32_t &fell, uint32_t &rows, uint32_t lane) {
    const int pv_dir = down ? kInNegY : kInPosY;
    const int step = down ? -1 : 1;  // the neighbour row relaxed from
#pragma unroll 1
    for (int k = 0; k < TH; ++k) {
        const int y = down ? k : TH - 1 - k;
        const uint32_t rb = 1u << y;
        if (!((m.H | (down ? m.D : m.U)) & rb)) continue;
        if ((uint32_t)y >= t.th) {  // past the window: every label stays +inf
            m.H &= ~rb;
            m.D &= ~rb;
            m.U &= ~rb;
            continue;
        }
        ++rows;
        uint32_t pnx[K], ppx[K], pv[K];
        row_prices(t, y, pv_dir, spec_lane, pnx, ppx, pv);
        const int yn = y + step;
        const bool inner = yn >= 0 && yn < TH;
        const u64 *halo = &sm.htb[down ? 0 : 1][(t.lc << t.tw_shift) + t.xb];
        u64 cur[K], u[K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            cur[i] = sm.lab[y][i][lane];
            u[i] = umin64(cur[i], ext2(inner ? sm.lab[yn][i][lane] : halo[i], pv[i], 1));
        }
        row_close(u, pnx, ppx, sm.hlr[0][t.lc * TH + y], sm.hlr[1][t.lc * TH + y], t.S, t.seg);
        bool ch = false;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const uint32_t bit = 1u << (y * K + i);
            if (!(valid & bit)) u[i] = kInf;
            if (u[i] < cur[i]) {
                sm.lab[y][i][lane] = u[i];
                fell |= bit;
                ch = true;
            }
        }
        m.H &= ~rb;
        if (down) m.D &= ~rb;
        else m.U &= ~rb;
        if (__any_sync(kFull, ch)) {
            if (y + 1 < TH) m.D |= rb << 1;
            if (y > 0) m.U |= rb >> 1;
            m.ST |= rb;
        }
    }
}

// Layer stacks of the marked rows, in place in shared memory: lane j closes
// the stacks of columns j, j + 32, ... (upward, then downward); a lowered cell
// is flagged for its owner lane in sm.fell.
__device__ __forceinline__ void stack_pass(const WTile &t, WarpSmem &sm, RowMarks &m, uint32_t lane, uint32_t &rows) {
#pragma unroll 1
    for (int y = 0; y < TH; ++y) {
        const uint32_t rb = 1u << y;
        if (!(m.ST & rb)) continue;
        m.ST &= ~rb;
        if ((uint32_t)y >= t.th) continue;  // past the window: nothing to relax, and no board row to read
        ++rows;
        __syncwarp();  // the row passes' stores
        bool ch = false;
        for (uint32_t x = lane; x < t.tw; x += 32) {
            const uint32_t sg = x / K, xi = x % K;
            u64 prev = sm.lab[y][xi][sg];
            for (uint32_t l = 1; l < t.L; ++l) {
                u64 &cell = sm.lab[y][xi][l * t.S + sg];
                const u64 w = ext2(prev, tile_price(t, sm, kInBelow, l, y, x), 1);
                if (w < cell) {
                    cell = w;
                    atomicOr(&sm.fell[l * t.S + sg], 1u << (y * K + xi));
                    ch = true;
                }
                prev = cell;
            }
            prev = sm.lab[y][xi][(t.L - 1) * t.S + sg];
            for (int l = (int)t.L - 2; l >= 0; --l) {
                u64 &cell = sm.lab[y][xi][(uint32_t)l * t.S + sg];
                const u64 w = ext2(prev, tile_price(t, sm, kInAbove, (uint32_t)l, y, x), 1);
                if (w < cell) {
                    cell = w;
                    atomicOr(&sm.fell[(uint32_t)l * t.S + sg], 1u << (y * K + xi));
                    ch = true;
                }
                prev = cell;
            }
        }
        __syncwarp();  // the stack results, before any lane reads its row again
        if (__any_sync(kFull, ch)) {
            m.H |= rb;
            if (y + 1 < TH) m.D |= rb << 1;
            if (y > 0) m.U |= rb >> 1;
        }
    }
}

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *a, uint32_t n, uint32_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Price of the planar step from a border cell of this tile into the cell `c`
// of a neighbour tile, from direction `dir` as seen from c.
__device__ __forceinline__ uint32_t neighbour_price(const WTile &t, int dir, uint32_t c, uint32_t l, uint32_t gy,
                                                    uint32_t gx) {
    const uint32_t p = plane_at(t, dir, l, gy, gx);
    // only an own obstacle pad or endpoint can be priced differently for this net
    if (p == kMax) return exact_price_t(t, dir, c, l, gy, gx);
    return p;
}

// Work counters a warp accumulates and adds to the control block in batches.
struct WarpStats {
    uint32_t acts = 0, passes = 0, rows = 0;
};

__device__ __forceinline__ void flush_stats(const RelaxArgs &a, WarpStats &w) {
    if (!w.acts) return;
    if (atomicAdd(&a.ctl->activations, (unsigned long long)w.acts) + w.acts > a.activation_limit)
        atomicOr(&a.ctl->status, kStatusActivationLimit);
    atomicAdd(&a.ctl->sweeps, (unsigned long long)w.passes);
    atomicAdd(&a.ctl->rows, (unsigned long long)w.rows);
    w = WarpStats{};
}

__device__ void warp_item(const RelaxArgs &a, uint32_t fi, uint32_t tile, WarpSmem &sm, uint32_t lane,
                          WarpStats &ws) {
    WTile t;
    const DevField f = a.fields[fi];
    t.fp = a.fields + fi;
    t.bp = a.boards + f.board;
    t.pads = a.pads;
    t.planes = t.bp->planes;
    t.w = t.bp->w;
    t.h = t.bp->h;
    t.L = t.bp->layers;
    t.S = warp_segments(t.L);
    t.TW = K * t.S;
    t.tw_shift = (uint32_t)(__ffs((int)t.TW) - 1);
    t.wp = planes_pitch(t.w);
    t.NP = (uint64_t)t.wp * t.h * t.L;
    t.l = lane / t.S;
    t.seg = lane & (t.S - 1);
    t.act = t.l < t.L;
    t.lc = t.act ? t.l : t.L - 1;
    t.xb = t.seg * K;
    const uint32_t ntx = (f.ww + t.TW - 1) >> t.tw_shift, nty = (f.wh + TH - 1) / TH;
    const uint32_t txi = tile % ntx, tyi = tile / ntx;
    t.tx0 = f.x0 + (txi << t.tw_shift);
    t.ty0 = f.y0 + tyi * TH;
    t.tw = min(t.TW, f.ww - (txi << t.tw_shift));
    t.th = min((uint32_t)TH, f.wh - tyi * TH);
    t.wx1 = f.x0 + f.ww;
    t.wy1 = f.y0 + f.wh;
    const uint32_t plane = t.w * t.h;
    Ctl *ctl = a.ctl;

    // hold the tile before reading any label: a neighbour that improves our
    // halo after this point marks it dirty, and it is queued again when done
    if (lane == 0) {
        atomicExch(a.tstamp + f.tile_off + tile, kTileHeld);
        __threadfence();
    }
    __syncwarp();
    u64 *lab = a.lab + f.lab_off;
    auto lidx = [&](uint32_t l, uint32_t gy, uint32_t gx) -> uint64_t {
        return ((uint64_t)l * f.wh + (gy - f.y0)) * f.ww + (gx - f.x0);
    };

    // ---- stage: halo ring to shared memory, the tile into registers --------
    auto stage_halo = [&]() {
        for (uint32_t j = lane; j < (t.L << t.tw_shift); j += 32) {
            const uint32_t l = j >> t.tw_shift, x = j & (t.TW - 1);
            u64 top = kInf, bot = kInf;
            if (x < t.tw) {
                if (t.ty0 > f.y0) top = __ldcg(lab + lidx(l, t.ty0 - 1, t.tx0 + x));
                if (t.ty0 + t.th < t.wy1) bot = __ldcg(lab + lidx(l, t.ty0 + t.th, t.tx0 + x));
            }
            sm.htb[0][j] = top;
            sm.htb[1][j] = bot;
        }
        for (uint32_t j = lane; j < t.L * TH; j += 32) {
            const uint32_t l = j / TH, y = j % TH;
            u64 lft = kInf, rgt = kInf;
            if (y < t.th) {
                if (t.tx0 > f.x0) lft = __ldcg(lab + lidx(l, t.ty0 + y, t.tx0 - 1));
                if (t.tx0 + t.tw < t.wx1) rgt = __ldcg(lab + lidx(l, t.ty0 + y, t.tx0 + t.tw));
            }
            sm.hlr[0][j] = lft;
            sm.hlr[1][j] = rgt;
        }
    };
    stage_halo();
    sm.spec[lane] = 0;
    sm.fell[lane] = 0;
    uint32_t valid = 0;
#pragma unroll
    for (int y = 0; y < TH; ++y) {
        u64 v[K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const uint32_t x = t.xb + i;
            const bool ok = t.act && x < t.tw && (uint32_t)y < t.th;
            if (ok) valid |= 1u << (y * K + i);
            v[i] = ok ? __ldcg(lab + lidx(t.l, t.ty0 + y, t.tx0 + x)) : kInf;
        }
#pragma unroll
        for (int i = 0; i < K; ++i) sm.lab[y][i][lane] = v[i];
    }
    __syncwarp();
    // stacks whose prices depend on this net: endpoints, own pads, via pads
    auto mark = [&](uint32_t c) {
        const uint32_t r = c % plane, y = r / t.w, x = r - y * t.w;
        if (x >= t.tx0 && x < t.tx0 + t.tw && y >= t.ty0 && y < t.ty0 + t.th) {
            const uint32_t bit = ((y - t.ty0) << t.tw_shift) + (x - t.tx0);
            atomicOr(&sm.spec[bit >> 5], 1u << (bit & 31));
        }
    };
    if (lane == 0) mark(f.src);
    if (lane == 1) mark(f.dst);
    if (f.n_pads | f.n_vpads) {
        for (uint32_t j = lane; j < 2 * t.L * t.th; j += 32) {
            const uint32_t q = j & 1u, r = j >> 1, l = r / t.th, y = r - l * t.th;
            const uint32_t lo_c = (l * t.h + t.ty0 + y) * t.w + t.tx0, hi_c = lo_c + t.tw;
            const uint32_t *list = a.pads + (q ? f.vpad_off : f.pad_off);
            const uint32_t n = q ? f.n_vpads : f.n_pads;
            for (uint32_t k = lower_bound_u32(list, n, lo_c); k < n; ++k) {
                const uint32_t c = __ldg(list + k);
                if (c >= hi_c) break;
                mark(c);
            }
        }
    }
    __syncwarp();
    uint32_t spec_lane = 0;
    if (t.act) {
#pragma unroll
        for (int y = 0; y < TH; ++y) {
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const uint32_t bit = ((uint32_t)y << t.tw_shift) + t.xb + i;
                if ((sm.spec[bit >> 5] >> (bit & 31)) & 1u) spec_lane |= 1u << (y * K + i);
            }
        }
    }

    // ---- relax to local convergence ----------------------------------------
    // The labels are converged with respect to the halo of the previous
    // activation; new information enters through the halo: every row may be
    // open along x, row 0 to the step down from the upper halo, row TH-1 to the
    // step up from the lower one.  The source tile starts fully open.
    const uint32_t all = (1u << TH) - 1u;
    RowMarks m{all, 1u, 1u << (TH - 1), 0u};
    uint32_t fell = 0;
    {
        const uint32_t sl = f.src / plane, sr = f.src - sl * plane, sy = sr / t.w, sx = sr - sy * t.w;
        if (sx >= t.tx0 && sx < t.tx0 + t.tw && sy >= t.ty0 && sy < t.ty0 + t.th) {
            m = RowMarks{all, all, all, all};
            // The seeded source label never falls here, yet a neighbour tile
            // may be reachable only through its step across the border: it
            // counts as fallen, so the push checks see it.
            const uint32_t x = sx - t.tx0;
            if (t.act && t.l == sl && x >= t.xb && x < t.xb + K) fell |= 1u << ((sy - t.ty0) * K + (x - t.xb));
        }
    }
    // One activation may run several rounds: when a neighbour improved this
    // tile's halo while the warp held it (the state word says held-and-dirty),
    // the warp re-stages the halo only and relaxes again from the labels still
    // in shared memory, instead of releasing the tile to the queue and staging
    // all of it again later.  The number of such rounds is bounded; after the
    // last one a dirty tile is queued again as usual.
    for (uint32_t round = 0;; ++round) {
        // start with the vertical direction whose entry halo is closer to the source
        uint32_t dtop = kMax, dbot = kMax;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            dtop = min(dtop, (uint32_t)(sm.htb[0][(t.lc << t.tw_shift) + t.xb + i] >> 32));
            dbot = min(dbot, (uint32_t)(sm.htb[1][(t.lc << t.tw_shift) + t.xb + i] >> 32));
        }
        dtop = __reduce_min_sync(kFull, dtop);
        dbot = __reduce_min_sync(kFull, dbot);
        // passes cycle (first vertical direction, the other one, stacks)
        bool down = dtop <= dbot;
        uint32_t passes = 0, rows = 0;
        const uint32_t pass_limit = 12u * TH * t.TW * t.L + 48u;
        for (uint32_t step = 0;; ++step) {
            const uint32_t phase = step % 3;
            if (phase < 2) {
                vert_pass(t, sm, down, m, spec_lane, valid, fell, rows, lane);
                down = !down;
            } else if (t.L > 1) {
                stack_pass(t, sm, m, lane, rows);
            } else {
                m.ST = 0;
            }
            ++passes;
            if (!(m.H | m.D | m.U | m.ST)) break;
            if (passes > pass_limit) {
                if (lane == 0) atomicOr(&ctl->status, kStatusRoundLimit);
                break;
            }
        }

        // ---- write back the labels that fell; queue the neighbours they improve --
        __syncwarp();
        fell |= sm.fell[lane];  // cells lowered by the stack pass of another lane
        bool pl = false, pr = false, pt = false, pb = false;
        const auto v = sm.lab;  // the converged tile
        if (t.act && fell) {
#pragma unroll 1
            for (int y = 0; y < TH; ++y) {
#pragma unroll
                for (int i = 0; i < K; ++i)
                    if ((fell >> (y * K + i)) & 1u) lab[lidx(t.l, t.ty0 + y, t.tx0 + t.xb + i)] = v[y][i][lane];
            }
            // Only a border label that fell can improve a neighbour: an unchanged one
            // was checked when it was written.  Compare with the halo as staged.
            const uint32_t l = t.l;
            if (txi > 0 && t.seg == 0) {
#pragma unroll 1
                for (int y = 0; y < TH; ++y) {
                    if (!((fell >> (y * K)) & 1u)) continue;
                    const uint32_t gy = t.ty0 + y, gx = t.tx0 - 1, c = (l * t.h + gy) * t.w + gx;
                    const u64 cand = ext2(v[y][0][lane], neighbour_price(t, kInPosX, c, l, gy, gx), 1);
                    pl |= cand < sm.hlr[0][l * TH + y];
                }
            }
            if (txi + 1 < ntx && t.seg == t.S - 1) {  // not the last tile column: tw == TW
#pragma unroll 1
                for (int y = 0; y < TH; ++y) {
                    if (!((fell >> (y * K + K - 1)) & 1u)) continue;
                    const uint32_t gy = t.ty0 + y, gx = t.tx0 + t.TW, c = (l * t.h + gy) * t.w + gx;
                    const u64 cand = ext2(v[y][K - 1][lane], neighbour_price(t, kInNegX, c, l, gy, gx), 1);
                    pr |= cand < sm.hlr[1][l * TH + y];
                }
            }
            if (tyi > 0) {
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    if (!((fell >> i) & 1u)) continue;
                    const uint32_t gy = t.ty0 - 1, gx = t.tx0 + t.xb + i, c = (l * t.h + gy) * t.w + gx;
                    const u64 cand = ext2(v[0][i][lane], neighbour_price(t, kInPosY, c, l, gy, gx), 1);
                    pt |= cand < sm.htb[0][(l << t.tw_shift) + t.xb + i];
                }
            }
            if (tyi + 1 < nty) {  // not the last tile row: th == TH
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    if (!((fell >> ((TH - 1) * K + i)) & 1u)) continue;
                    const uint32_t gy = t.ty0 + TH, gx = t.tx0 + t.xb + i, c = (l * t.h + gy) * t.w + gx;
                    const u64 cand = ext2(v[TH - 1][i][lane], neighbour_price(t, kInNegY, c, l, gy, gx), 1);
                    pb |= cand < sm.htb[1][(l << t.tw_shift) + t.xb + i];
                }
            }
        }
        __threadfence();  // labels before the pushes and the release
        pl = __any_sync(kFull, pl);
        pr = __any_sync(kFull, pr);
        pt = __any_sync(kFull, pt);
        pb = __any_sync(kFull, pb);
        if (lane == 0) {
            ws.passes += passes;
            ws.rows += rows;
            if (pl) async_push(a, fi, f.tile_off, tile - 1);
            if (pr) async_push(a, fi, f.tile_off, tile + 1);
            if (pt) async_push(a, fi, f.tile_off, tile - ntx);
            if (pb) async_push(a, fi, f.tile_off, tile + ntx);
        }
        // improved while held?  take the new halo in place of a re-activation
        bool again = false;
        if (round + 1 < kMaxRounds && lane == 0)
            again = atomicCAS(a.tstamp + f.tile_off + tile, kTileHeldDirty, kTileHeld) == kTileHeldDirty;
        again = __shfl_sync(kFull, again, 0);
        if (!again) break;
        __threadfence();  // the neighbour's labels, written before it marked the tile
        stage_halo();
        sm.fell[lane] = 0;
        __syncwarp();
        m = RowMarks{all, 1u, 1u << (TH - 1), 0u};
        fell = 0;
    }  // rounds
    if (lane == 0) {
        ws.acts += 1;
        if (ws.acts == 32) flush_stats(a, ws);
        __threadfence();
        async_release(a, fi, f.tile_off, tile);  // this item is done: its own pushes are already counted
        atomicSub(&ctl->count[1], 1u);
    }
    __syncwarp();
}

__global__ void __launch_bounds__(NW * 32, 4) relax_warp_kernel(RelaxArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];  // NW x WarpSmem
    WarpSmem &sm = reinterpret_cast<WarpSmem *>(smem_raw)[threadIdx.x >> 5];
    const uint32_t lane = threadIdx.x & 31;
    WarpStats ws;
    for (;;) {
        u64 item = 0;
        if (lane == 0) item = async_pop(a);
        item = __shfl_sync(kFull, item, 0);
        if (item == kInf) break;
        warp_item(a, (uint32_t)(item >> 32), (uint32_t)item, sm, lane, ws);
    }
    if (lane == 0) flush_stats(a, ws);
}

// Seeds: the source label and the source tile (warp tile geometry) of every
// field whose source is inside its window and enterable.
__global__ void warp_seed_kernel(RelaxArgs a) {
    for (uint32_t fi = blockIdx.x * blockDim.x + threadIdx.x; fi < a.n_fields; fi += gridDim.x * blockDim.x) {
        const DevField f = a.fields[fi];
        const DevBoard b = a.boards[f.board];
        const uint32_t plane = b.w * b.h;
        const uint32_t sl = f.src / plane, sr = f.src % plane, sx = sr % b.w, sy = sr / b.w;
        const uint8_t sfl = b.flags ? b.flags[f.src] : 0;
        if (sx >= f.x0 && sx < f.x0 + f.ww && sy >= f.y0 && sy < f.y0 + f.wh &&
            cell_enter(b, f, a.pads, f.src, sfl) != kMax) {
            a.lab[f.lab_off + ((uint64_t)sl * f.wh + (sy - f.y0)) * f.ww + (sx - f.x0)] = 0;
            const uint32_t tw = warp_tile_w(b.layers);
            const uint32_t ntx = (f.ww + tw - 1) / tw;
            const uint32_t t = ((sy - f.y0) / TH) * ntx + (sx - f.x0) / tw;
            __threadfence();
            async_push(a, fi, f.tile_off, t);
        }
    }
}

}  // namespace

uint64_t planes_chunks(uint64_t cells) { return (cells + kPlaneChunk - 1) / kPlaneChunk; }

cudaError_t planes_launch(const DevBoard *boards, const uint64_t *chunk_start, uint32_t n_boards, uint64_t n_chunks,
                          uint32_t sms, cudaStream_t st) {
    if (!n_boards || !n_chunks) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>(n_chunks, (uint64_t)sms * 8);
    planes_kernel<<<(uint32_t)blocks, 256, 0, st>>>(boards, chunk_start, n_boards, n_chunks);
    return cudaGetLastError();
}

uint32_t warp_relax_threads() { return NW * 32; }

static constexpr size_t kWarpSmemBytes = NW * sizeof(WarpSmem);

cudaError_t warp_relax_occupancy(int *blocks_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(relax_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kWarpSmemBytes);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, relax_warp_kernel, NW * 32, kWarpSmemBytes);
}

cudaError_t warp_relax_launch(const RelaxArgs &a, uint32_t grid, cudaStream_t st) {
    if (!a.n_fields) return cudaSuccess;
    warp_seed_kernel<<<(a.n_fields + 255) / 256, 256, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    relax_warp_kernel<<<grid, NW * 32, kWarpSmemBytes, st>>>(a);
    return cudaGetLastError();
}

}  // namespace mrc
