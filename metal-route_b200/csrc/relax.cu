// relax.cu — the batched field + canonical path kernels.
//
// relax_tiles_kernel: a persistent CTA takes one field (net x window) at a
// time from a device work counter.  The field's labels live in HBM (u32 dist,
// u32 hops, window-packed like the reference's ragged layout,
// metal/src/lib.rs:833-871).  The window is cut into tiles of 32 x TH cells
// over every layer; an active tile is staged in shared memory with a one-cell
// halo ring, relaxed to local convergence by directional sweeps (rows, columns,
// layer stacks — the edge-aware sweep of gpu.rs:259-430 run on-chip instead of
// one dispatch per round), written back, and any neighbour whose halo it can
// now improve is queued.  The field is final when the tile queue drains.
//
// path kernels: the path length is hops[dst] + 1 (every canonical predecessor
// has exactly one fewer hop), so offsets come from one device scan and one warp
// per net walks dst -> src choosing the lowest-CellIdx predecessor whose label
// and step reproduce the current label (metal/src/lib.rs:308-396).
#include <cuda_runtime.h>

#include <algorithm>

#include "device.cuh"
#include "kernels.h"

namespace mrc {

// Status bits reported through the kernels' status word.
constexpr uint32_t kStatusActivationLimit = 1u << 0;
constexpr uint32_t kStatusRoundLimit = 1u << 1;
constexpr uint32_t kStatusPathBroken = 1u << 2;
constexpr uint32_t kStatusQueueOverflow = 1u << 3;

constexpr uint32_t kTW = 32;  // tile width (one warp across a row)

struct TileSmem {
    u64 *lab;
    uint32_t *ent;
    uint8_t *fl;
    uint4 *din;
};

// Price of the planar move p -> c between staged cells; kMax = not allowed.
// A kMax base price blocks only in the directed form: the reference's axis gap
// price may itself saturate and still yields the capped step.
template <bool DIRECTED>
__device__ __forceinline__ uint32_t planar_step(const TileSmem &s, uint32_t p, uint32_t c, uint32_t base,
                                                uint8_t out_bit, uint8_t in_bit) {
    uint32_t e = s.ent[c];
    if (e == kMax) return kMax;
    if ((s.fl[p] & out_bit) | (s.fl[c] & in_bit)) return kMax;
    if (DIRECTED && base == kMax) return kMax;
    return capmul(base, e);
}

template <bool DIRECTED>
__global__ void __launch_bounds__(kRelaxThreads) relax_tiles_kernel(RelaxArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const DevBoard b = a.board;
    const uint32_t L = b.layers;
    const uint32_t TH = a.tile_h;
    const uint32_t SW = kTW + 2, SH = TH + 2;
    const uint32_t nsm = L * SH * SW;
    TileSmem s;
    s.lab = reinterpret_cast<u64 *>(smem_raw);
    s.ent = reinterpret_cast<uint32_t *>(s.lab + nsm);
    s.fl = reinterpret_cast<uint8_t *>(s.ent + nsm);
    s.din = nullptr;
    if (DIRECTED) {
        size_t off = (size_t)nsm * 13;
        off = (off + 15) & ~(size_t)15;
        s.din = reinterpret_cast<uint4 *>(smem_raw + off);
    }
    __shared__ uint32_t xe_s[kTW + 2];
    __shared__ uint32_t ye_s[34];
    __shared__ uint32_t s_field, s_tile, s_qhead, s_qtail, s_act, s_abort;
    __shared__ uint32_t s_push[4];

    const uint32_t tid = threadIdx.x;
    uint32_t *queue = a.tile_scratch + (size_t)blockIdx.x * a.scratch_stride;
    uint32_t *inq = queue + a.max_tiles;

    for (;;) {
        if (tid == 0) s_field = atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const uint32_t fi = s_field;
        if (fi >= a.n_fields) break;
        const DevField f = a.fields[fi];
        const uint32_t ntx = (f.ww + kTW - 1) / kTW, nty = (f.wh + TH - 1) / TH;
        const uint32_t ntiles = ntx * nty;
        const uint64_t wcells = (uint64_t)f.ww * f.wh * L;
        uint32_t *dist = a.dist + f.lab_off;
        uint32_t *hops = a.hops + f.lab_off;

        for (uint64_t i = tid; i < wcells; i += blockDim.x) {
            dist[i] = kMax;
            hops[i] = kMax;
        }
        for (uint32_t i = tid; i < (ntiles + 31) / 32; i += blockDim.x) inq[i] = 0;
        __syncthreads();
        if (tid == 0) {
            s_qhead = 0;
            s_qtail = 0;
            s_act = 0;
            s_abort = 0;
            const uint32_t plane = b.w * b.h;
            const uint32_t sl = f.src / plane, sr = f.src % plane;
            const uint32_t sx = sr % b.w, sy = sr / b.w;
            const uint8_t sfl = b.flags ? b.flags[f.src] : 0;
            if (sx >= f.x0 && sx < f.x0 + f.ww && sy >= f.y0 && sy < f.y0 + f.wh &&
                cell_enter(b, f, a.pads, f.src, sfl) != kMax) {
                const uint64_t lc = ((uint64_t)sl * f.wh + (sy - f.y0)) * f.ww + (sx - f.x0);
                dist[lc] = 0;
                hops[lc] = 0;
                const uint32_t t = ((sy - f.y0) / TH) * ntx + (sx - f.x0) / kTW;
                queue[0] = t;
                s_qtail = 1;
                inq[t >> 5] |= 1u << (t & 31);
            }
        }
        __syncthreads();
        const uint32_t act_limit = a.activation_factor * ntiles + 65536u;

        for (;;) {
            if (tid == 0) {
                if (s_qhead == s_qtail || s_abort) {
                    s_tile = kMax;
                } else {
                    const uint32_t t = queue[s_qhead % a.max_tiles];
                    s_qhead++;
                    inq[t >> 5] &= ~(1u << (t & 31));
                    s_tile = t;
                    if (++s_act > act_limit) {
                        atomicOr(a.status, kStatusActivationLimit);
                        s_abort = 1;
                        s_tile = kMax;
                    }
                }
                s_push[0] = s_push[1] = s_push[2] = s_push[3] = 0;
            }
            __syncthreads();
            const uint32_t t = s_tile;
            if (t == kMax) break;
            const uint32_t txi = t % ntx, tyi = t / ntx;
            const int tx0 = (int)(f.x0 + txi * kTW), ty0 = (int)(f.y0 + tyi * TH);
            const uint32_t tw = min(kTW, f.ww - txi * kTW), th = min(TH, f.wh - tyi * TH);
            const int wx0 = (int)f.x0, wy0 = (int)f.y0, wx1 = (int)(f.x0 + f.ww), wy1 = (int)(f.y0 + f.wh);

            // ---- stage the tile and its halo ring ---------------------------
            for (uint32_t i = tid; i < nsm; i += blockDim.x) {
                const uint32_t sx = i % SW, r = i / SW, sy = r % SH, l = r / SH;
                const int gx = tx0 + (int)sx - 1, gy = ty0 + (int)sy - 1;
                u64 lab = kInf;
                uint32_t ent = kMax;
                uint8_t fl = 0;
                if (gx >= wx0 && gx < wx1 && gy >= wy0 && gy < wy1) {
                    const uint32_t gcell = (l * b.h + (uint32_t)gy) * b.w + (uint32_t)gx;
                    const uint64_t lc = ((uint64_t)l * f.wh + (uint32_t)(gy - wy0)) * f.ww + (uint32_t)(gx - wx0);
                    const uint32_t d = dist[lc];
                    lab = d == kMax ? kInf : (((u64)d << 32) | hops[lc]);
                    const uint8_t gf = b.flags ? __ldg(b.flags + gcell) : 0;
                    ent = cell_enter(b, f, a.pads, gcell, gf);
                    fl = cell_tile_flags(f, a.pads, gcell, gf);
                    if (DIRECTED && sx >= 1 && sx <= kTW && sy >= 1 && sy <= TH)
                        s.din[(l * TH + sy - 1) * kTW + sx - 1] = __ldg(b.directed + gcell);
                }
                s.lab[i] = lab;
                s.ent[i] = ent;
                s.fl[i] = fl;
            }
            // xe_s[sx] prices the gap between shared columns sx-1 and sx.
            for (uint32_t i = tid; i < SW; i += blockDim.x) {
                const int g = tx0 + (int)i - 2;
                xe_s[i] = (g >= 0 && g + 1 < (int)b.w) ? __ldg(b.x_edge + g) : kMax;
            }
            for (uint32_t i = tid; i < SH; i += blockDim.x) {
                const int g = ty0 + (int)i - 2;
                ye_s[i] = (g >= 0 && g + 1 < (int)b.h) ? __ldg(b.y_edge + g) : kMax;
            }
            __syncthreads();

            // ---- relax to local convergence ---------------------------------
            const uint32_t round_limit = L * kTW * TH + 4;
            uint32_t round = 0;
            for (;;) {
                bool ch = false;
                // rows: one thread per (layer, row)
                for (uint32_t r = tid; r < L * th; r += blockDim.x) {
                    const uint32_t l = r / th, ty = r % th;
                    const uint32_t base = (l * SH + ty + 1) * SW;
                    u64 prev = s.lab[base];
                    for (uint32_t sx = 1; sx <= tw; ++sx) {
                        const uint32_t c = base + sx;
                        u64 cur = s.lab[c];
                        const uint32_t bp = DIRECTED ? s.din[(l * TH + ty) * kTW + sx - 1].y : xe_s[sx];
                        const u64 cand = extend(prev, planar_step<DIRECTED>(s, c - 1, c, bp, kEdgePosX, kEdgeNegX));
                        if (cand < cur) {
                            cur = cand;
                            s.lab[c] = cur;
                            ch = true;
                        }
                        prev = cur;
                    }
                    prev = s.lab[base + tw + 1];
                    for (uint32_t sx = tw; sx >= 1; --sx) {
                        const uint32_t c = base + sx;
                        u64 cur = s.lab[c];
                        const uint32_t bp = DIRECTED ? s.din[(l * TH + ty) * kTW + sx - 1].z : xe_s[sx + 1];
                        const u64 cand = extend(prev, planar_step<DIRECTED>(s, c + 1, c, bp, kEdgeNegX, kEdgePosX));
                        if (cand < cur) {
                            cur = cand;
                            s.lab[c] = cur;
                            ch = true;
                        }
                        prev = cur;
                    }
                }
                __syncthreads();
                // columns: one thread per (layer, column)
                for (uint32_t r = tid; r < L * tw; r += blockDim.x) {
                    const uint32_t l = r / tw, tx = r % tw;
                    const uint32_t base = l * SH * SW + tx + 1;
                    u64 prev = s.lab[base];
                    for (uint32_t sy = 1; sy <= th; ++sy) {
                        const uint32_t c = base + sy * SW;
                        u64 cur = s.lab[c];
                        const uint32_t bp = DIRECTED ? s.din[(l * TH + sy - 1) * kTW + tx].x : ye_s[sy];
                        const u64 cand = extend(prev, planar_step<DIRECTED>(s, c - SW, c, bp, kEdgePosY, kEdgeNegY));
                        if (cand < cur) {
                            cur = cand;
                            s.lab[c] = cur;
                            ch = true;
                        }
                        prev = cur;
                    }
                    prev = s.lab[base + (th + 1) * SW];
                    for (uint32_t sy = th; sy >= 1; --sy) {
                        const uint32_t c = base + sy * SW;
                        u64 cur = s.lab[c];
                        const uint32_t bp = DIRECTED ? s.din[(l * TH + sy - 1) * kTW + tx].w : ye_s[sy + 1];
                        const u64 cand = extend(prev, planar_step<DIRECTED>(s, c + SW, c, bp, kEdgeNegY, kEdgePosY));
                        if (cand < cur) {
                            cur = cand;
                            s.lab[c] = cur;
                            ch = true;
                        }
                        prev = cur;
                    }
                }
                if (L > 1) {
                    __syncthreads();
                    // layer stacks: one thread per (x, y), up then down
                    for (uint32_t r = tid; r < th * tw; r += blockDim.x) {
                        const uint32_t ty = r / tw, tx = r % tw;
                        const uint32_t base = (ty + 1) * SW + tx + 1;
                        const uint32_t lstride = SH * SW;
                        u64 prev = s.lab[base];
                        for (uint32_t l = 1; l < L; ++l) {
                            const uint32_t c = base + l * lstride, p = c - lstride;
                            u64 cur = s.lab[c];
                            uint32_t st = kMax;
                            if (((b.via_mask >> (l - 1)) & 1u) && !((s.fl[p] | s.fl[c]) & kViaBlocked) &&
                                s.ent[c] != kMax)
                                st = capmul(__ldg(b.via_edge + l - 1), s.ent[c]);
                            const u64 cand = extend(prev, st);
                            if (cand < cur) {
                                cur = cand;
                                s.lab[c] = cur;
                                ch = true;
                            }
                            prev = cur;
                        }
                        for (int l = (int)L - 2; l >= 0; --l) {
                            const uint32_t c = base + (uint32_t)l * lstride, p = c + lstride;
                            u64 cur = s.lab[c];
                            uint32_t st = kMax;
                            if (((b.via_mask >> l) & 1u) && !((s.fl[p] | s.fl[c]) & kViaBlocked) &&
                                s.ent[c] != kMax)
                                st = capmul(__ldg(b.via_edge + l), s.ent[c]);
                            const u64 cand = extend(prev, st);
                            if (cand < cur) {
                                cur = cand;
                                s.lab[c] = cur;
                                ch = true;
                            }
                            prev = cur;
                        }
                    }
                }
                const int any = __syncthreads_or(ch ? 1 : 0);
                if (!any) break;
                if (++round > round_limit) {
                    if (tid == 0) {
                        atomicOr(a.status, kStatusRoundLimit);
                        s_abort = 1;
                    }
                    break;
                }
            }

            // ---- write back and find neighbours this tile can improve -------
            for (uint32_t i = tid; i < L * th * tw; i += blockDim.x) {
                const uint32_t tx = i % tw, r = i / tw, ty = r % th, l = r / th;
                const uint32_t c = (l * SH + ty + 1) * SW + tx + 1;
                const uint64_t lc = ((uint64_t)l * f.wh + (uint32_t)(ty0 - wy0) + ty) * f.ww + (uint32_t)(tx0 - wx0) + tx;
                const u64 v = s.lab[c];
                dist[lc] = (uint32_t)(v >> 32);
                hops[lc] = v == kInf ? kMax : (uint32_t)v;
            }
            // borders: 0 = left (-x), 1 = right (+x), 2 = top (-y), 3 = bottom (+y)
            const uint32_t nb = 2 * L * th + 2 * L * tw;
            for (uint32_t i = tid; i < nb; i += blockDim.x) {
                uint32_t side, l, k;
                if (i < 2 * L * th) {
                    side = i / (L * th);
                    const uint32_t r = i % (L * th);
                    l = r / th;
                    k = r % th;
                } else {
                    const uint32_t j = i - 2 * L * th;
                    side = 2 + j / (L * tw);
                    const uint32_t r = j % (L * tw);
                    l = r / tw;
                    k = r % tw;
                }
                bool exists;
                uint32_t bc, nc, dir;
                uint8_t out_bit, in_bit;
                uint32_t gap;
                if (side == 0) {
                    exists = txi > 0;
                    bc = (l * SH + k + 1) * SW + 1;
                    nc = bc - 1;
                    dir = 2;
                    out_bit = kEdgeNegX;
                    in_bit = kEdgePosX;
                    gap = xe_s[1];
                } else if (side == 1) {
                    exists = txi + 1 < ntx;
                    bc = (l * SH + k + 1) * SW + tw;
                    nc = bc + 1;
                    dir = 1;
                    out_bit = kEdgePosX;
                    in_bit = kEdgeNegX;
                    gap = xe_s[tw + 1];
                } else if (side == 2) {
                    exists = tyi > 0;
                    bc = (l * SH + 1) * SW + k + 1;
                    nc = bc - SW;
                    dir = 3;
                    out_bit = kEdgeNegY;
                    in_bit = kEdgePosY;
                    gap = ye_s[1];
                } else {
                    exists = tyi + 1 < nty;
                    bc = (l * SH + th) * SW + k + 1;
                    nc = bc + SW;
                    dir = 0;
                    out_bit = kEdgePosY;
                    in_bit = kEdgeNegY;
                    gap = ye_s[th + 1];
                }
                if (!exists || s_push[side]) continue;
                const u64 lb = s.lab[bc];
                if (lb == kInf || s.ent[nc] == kMax) continue;
                uint32_t base = gap;
                if (DIRECTED) {
                    // the neighbour's in-price is not staged; read it from HBM
                    const uint32_t nsx = nc % SW, nsy = (nc / SW) % SH;
                    const uint32_t gcell = (l * b.h + (uint32_t)(ty0 + (int)nsy - 1)) * b.w + (uint32_t)(tx0 + (int)nsx - 1);
                    const uint4 d4 = __ldg(b.directed + gcell);
                    base = dir == 0 ? d4.x : dir == 1 ? d4.y : dir == 2 ? d4.z : d4.w;
                }
                const u64 cand = extend(lb, planar_step<DIRECTED>(s, bc, nc, base, out_bit, in_bit));
                if (cand < s.lab[nc]) s_push[side] = 1;
            }
            __syncthreads();
            if (tid == 0) {
                const uint32_t nbr[4] = {t - 1, t + 1, t - ntx, t + ntx};
                for (int sdx = 0; sdx < 4; ++sdx) {
                    if (!s_push[sdx]) continue;
                    const uint32_t u = nbr[sdx];
                    if (inq[u >> 5] & (1u << (u & 31))) continue;
                    if (s_qtail - s_qhead >= a.max_tiles) {
                        atomicOr(a.status, kStatusQueueOverflow);
                        s_abort = 1;
                        break;
                    }
                    queue[s_qtail % a.max_tiles] = u;
                    s_qtail++;
                    inq[u >> 5] |= 1u << (u & 31);
                }
            }
            __syncthreads();
        }
        __syncthreads();
    }
}

// Per field: search cost and path length (hops[dst] + 1), then an exclusive
// scan into path offsets.  Single CTA; loops over the fields in chunks.
__global__ void __launch_bounds__(1024) path_offsets_kernel(PathArgs a) {
    __shared__ unsigned long long warp_sums[32];
    __shared__ unsigned long long carry;
    const uint32_t plane = a.board.w * a.board.h;
    // phase 1: cost and length of every field, stored at its output slot
    for (uint32_t i = threadIdx.x; i < a.n_fields; i += blockDim.x) {
        const DevField f = a.fields[i];
        const uint32_t dl = f.dst / plane, dr = f.dst % plane;
        const uint32_t dx = dr % a.board.w, dy = dr / a.board.w;
        uint32_t cost = kMax, len = 0;
        if (dx >= f.x0 && dx < f.x0 + f.ww && dy >= f.y0 && dy < f.y0 + f.wh) {
            const uint64_t lc = f.lab_off + ((uint64_t)dl * f.wh + (dy - f.y0)) * f.ww + (dx - f.x0);
            cost = a.dist[lc];
            if (cost != kMax) len = a.hops[lc] + 1u;
            // a simple path never has more cells than its window
            if ((uint64_t)len > (uint64_t)f.ww * f.wh * a.board.layers) {
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

// Shared by the path walk: is p a canonical predecessor candidate of cur?
// Returns the step price p->cur, kMax when the move is not allowed.
__device__ __forceinline__ uint32_t global_step(const DevBoard &b, const DevField &f, const uint32_t *pads,
                                                uint32_t p, uint32_t cur, int kind) {
    // kind: 0 = p is cur's lower layer, 1 = -y, 2 = -x, 3 = +x, 4 = +y, 5 = upper layer
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
        out_bit = kEdgePosY; in_bit = kEdgeNegY;
        base = b.directed ? __ldg(b.directed + cur).x : __ldg(b.y_edge + y - 1);
    } else if (kind == 2) {  // p at -x: p moves +x
        out_bit = kEdgePosX; in_bit = kEdgeNegX;
        base = b.directed ? __ldg(b.directed + cur).y : __ldg(b.x_edge + x - 1);
    } else if (kind == 3) {  // p at +x: p moves -x
        out_bit = kEdgeNegX; in_bit = kEdgePosX;
        base = b.directed ? __ldg(b.directed + cur).z : __ldg(b.x_edge + x);
    } else {  // p at +y: p moves -y
        out_bit = kEdgeNegY; in_bit = kEdgePosY;
        base = b.directed ? __ldg(b.directed + cur).w : __ldg(b.y_edge + y);
    }
    if ((fp & out_bit) | (fc & in_bit)) return kMax;
    if (b.directed && base == kMax) return kMax;
    return capmul(base, ec);
}

// One warp per field: lanes 0..5 test the six neighbours (ascending CellIdx)
// and the lowest qualifying one is the canonical predecessor.
__global__ void __launch_bounds__(256) path_walk_kernel(PathArgs a) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (warp >= a.n_fields) return;
    const DevField f = a.fields[warp];
    const uint32_t len = a.lens[f.out];
    if (len == 0) return;
    const DevBoard b = a.board;
    const uint32_t plane = b.w * b.h;
    uint32_t *out = a.cells + a.offsets[f.out];
    uint32_t cur = f.dst;
    for (uint32_t pos = len - 1;; --pos) {
        if (lane == 0) out[pos] = cur;
        if (pos == 0) {
            if (lane == 0 && cur != f.src) atomicOr(a.status, kStatusPathBroken);
            break;
        }
        const uint32_t r = cur % plane, x = r % b.w, y = r / b.w, l = cur / plane;
        const uint64_t lcur = f.lab_off + ((uint64_t)l * f.wh + (y - f.y0)) * f.ww + (x - f.x0);
        const uint32_t need_d = a.dist[lcur], need_h = a.hops[lcur];
        bool ok = false;
        uint32_t p = 0;
        if (lane < 6) {
            int px = (int)x, py = (int)y, pl = (int)l;
            if (lane == 0) pl -= 1;
            else if (lane == 1) py -= 1;
            else if (lane == 2) px -= 1;
            else if (lane == 3) px += 1;
            else if (lane == 4) py += 1;
            else pl += 1;
            if (pl >= 0 && pl < (int)b.layers && px >= (int)f.x0 && px < (int)(f.x0 + f.ww) && py >= (int)f.y0 &&
                py < (int)(f.y0 + f.wh)) {
                p = ((uint32_t)pl * b.h + (uint32_t)py) * b.w + (uint32_t)px;
                const uint64_t lp = f.lab_off + ((uint64_t)pl * f.wh + ((uint32_t)py - f.y0)) * f.ww + ((uint32_t)px - f.x0);
                const uint32_t dp = a.dist[lp], hp = a.hops[lp];
                if (dp != kMax && hp + 1u == need_h) {
                    const uint32_t st = global_step(b, f, a.pads, p, cur, (int)lane);
                    if (st != kMax) {
                        const uint32_t s = dp + st;
                        ok = s >= dp && s == need_d;
                    }
                }
            }
        }
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, ok);
        if (m == 0) {
            if (lane == 0) atomicOr(a.status, kStatusPathBroken);
            return;
        }
        const uint32_t win = __ffs(m) - 1;
        cur = __shfl_sync(0xFFFFFFFFu, p, win);
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
    const uint32_t *din = a.in_dist, *hin = a.in_hops;
    const uint32_t d0 = din[i];
    u64 best = d0 == kMax ? kInf : (((u64)d0 << 32) | hin[i]);
    if (!(cur == f.src && best == 0)) {
        const int64_t plane_l = (int64_t)f.ww * f.wh;
        const int64_t off[6] = {-plane_l, -(int64_t)f.ww, -1, 1, (int64_t)f.ww, plane_l};
        const bool has[6] = {l > 0, ly > 0, lx > 0, lx + 1 < f.ww, ly + 1 < f.wh, l + 1 < b.layers};
        const int64_t goff[6] = {-(int64_t)b.w * b.h, -(int64_t)b.w, -1, 1, (int64_t)b.w, (int64_t)b.w * b.h};
        for (int k = 0; k < 6; ++k) {
            if (!has[k]) continue;
            const uint64_t j = (uint64_t)((int64_t)i + off[k]);
            const uint32_t dp = din[j];
            if (dp == kMax) continue;
            const uint32_t p = (uint32_t)((int64_t)cur + goff[k]);
            const uint32_t st = global_step(b, f, a.pads, p, cur, k);
            const u64 cand = extend(((u64)dp << 32) | hin[j], st);
            if (cand < best) best = cand;
        }
    }
    a.out_dist[i] = (uint32_t)(best >> 32);
    a.out_hops[i] = best == kInf ? kMax : (uint32_t)best;
    if (best != (d0 == kMax ? kInf : (((u64)d0 << 32) | hin[i]))) *a.changed = 1u;
}

// OR Grid::via_forbidden into the flag byte as kStaticVia.
__global__ void combine_flags_kernel(uint8_t *flags, const uint8_t *via_forbidden, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (via_forbidden[i]) flags[i] |= kStaticVia;
}

// ---- host-side launch helpers ---------------------------------------------

cudaError_t combine_flags_launch(uint8_t *flags, const uint8_t *via_forbidden, uint64_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 4096);
    combine_flags_kernel<<<(uint32_t)blocks, 256, 0, st>>>(flags, via_forbidden, n);
    return cudaGetLastError();
}

size_t relax_smem_bytes(uint32_t layers, uint32_t tile_h, bool directed) {
    const size_t nsm = (size_t)layers * (tile_h + 2) * (kTW + 2);
    size_t bytes = nsm * 13;
    if (directed) {
        bytes = (bytes + 15) & ~(size_t)15;
        bytes += (size_t)layers * tile_h * kTW * 16;
    }
    return bytes;
}

cudaError_t relax_configure(bool directed, size_t smem) {
    if (directed)
        return cudaFuncSetAttribute(relax_tiles_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return cudaFuncSetAttribute(relax_tiles_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

cudaError_t relax_occupancy(bool directed, size_t smem, int *blocks_per_sm) {
    if (directed)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, relax_tiles_kernel<true>, kRelaxThreads, smem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, relax_tiles_kernel<false>, kRelaxThreads, smem);
}

cudaError_t relax_launch(const RelaxArgs &a, uint32_t grid, size_t smem, cudaStream_t st) {
    if (a.board.directed)
        relax_tiles_kernel<true><<<grid, kRelaxThreads, smem, st>>>(a);
    else
        relax_tiles_kernel<false><<<grid, kRelaxThreads, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t path_launch(const PathArgs &a, cudaStream_t st) {
    path_offsets_kernel<<<1, 1024, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.n_fields) {
        const uint32_t warps_per_block = 8;
        path_walk_kernel<<<(a.n_fields + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, st>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t plain_round_launch(const PlainArgs &a, uint64_t wcells, cudaStream_t st) {
    const uint32_t threads = 256;
    plain_round_kernel<<<(uint32_t)((wcells + threads - 1) / threads), threads, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace mrc
