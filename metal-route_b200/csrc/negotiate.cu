// negotiate.cu — device side of the snapshot negotiation round.
//
// Occupancy and history live on the directed planar in-edge slots of every
// cell, the layout of the directed price plane (uint4 per cell: in-edges from
// -y, -x, +x, +y).  An undirected planar edge {a, b} owns one slot at each end
// (b's slot "from a" and a's slot "from b"); both always carry the same count.
// The round follows the reference's Jacobi negotiation iteration
// (crates/mr-cpu/src/negotiated.rs:1610-1991) on edges instead of cells:
//   rip-up of the dirty nets' old paths, a frozen price snapshot
//   base + history + pfac * weight * present (priced_with_base, :2768-2795,
//   capped like passable_search_cost :1171-1173), the batched isolated solve,
//   merge of the new paths, then history += step on every edge used by two or
//   more nets (:1929-1948) and the next dirty set (:1632-1642).
//
// With a clearance the round is the reference's clearance-active iteration
// (:1565-1568, :1631-1634): nothing is ripped up before pricing, the snapshot
// adds pfac * halo_weight * halo[c] (the clearance footprints of every net's
// current path covering c), and each net is priced with its own path and
// footprint subtracted (priced_with_base :2778-2797).  Those per-net prices
// differ from the shared snapshot only on the net's own footprint, so they
// travel as sparse per-net overrides: emitted per footprint visit, sorted and
// summed by (net, cell), then priced from the snapshot's inputs.
#include <cuda_runtime.h>

#include <cstdint>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>

#include "kernels.h"

namespace mrc {
namespace {

// Slots of the planar edge a -> b: *sa at a (b seen from a), *sb at b.
// Returns false for a via step (different layers).
__device__ __forceinline__ bool planar_slots(uint32_t a, uint32_t b, uint32_t w, uint32_t plane, int *sa, int *sb) {
    if (a / plane != b / plane) return false;
    const uint32_t ax = (a % plane) % w;
    if (b == a + 1 && ax + 1 < w) {
        *sb = 1;  // b entered from -x
        *sa = 2;  // a entered from +x
        return true;
    }
    if (a == b + 1 && ax > 0) {
        *sb = 2;
        *sa = 1;
        return true;
    }
    if (b == a + w) {
        *sb = 0;  // from -y
        *sa = 3;  // from +y
        return true;
    }
    if (a == b + w) {
        *sb = 3;
        *sa = 0;
        return true;
    }
    return false;
}

__global__ void occupancy_kernel(OccupancyArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < a.n_list; item += warps) {
        const uint32_t net = a.list ? a.list[item] : item;
        const u64 p0 = a.offsets[net], p1 = a.offsets[net + 1];
        for (u64 k = p0 + lane; k + 1 < p1; k += 32) {
            const uint32_t u = a.cells[k], v = a.cells[k + 1];
            int su, sv;
            if (!planar_slots(u, v, a.w, a.plane, &su, &sv)) continue;
            if (a.add) {
                atomicAdd(a.present + 4ull * u + su, 1u);
                atomicAdd(a.present + 4ull * v + sv, 1u);
            } else {
                atomicSub(a.present + 4ull * u + su, 1u);
                atomicSub(a.present + 4ull * v + sv, 1u);
            }
        }
    }
}

// base + history + factor * present + extra, capped at MAX - 1 (every term
// below 2^32, every product below 2^64: no u64 overflow); a blocked edge stays blocked
__device__ __forceinline__ uint32_t snapshot_price(uint32_t base, uint32_t present, uint32_t history, u64 factor,
                                                   u64 extra = 0) {
    if (base == kMax) return kMax;
    const u64 c = factor * (u64)present + extra;
    const u64 p = (u64)base + (u64)history + c;
    return (p > (u64)kCap || c < extra) ? kCap : (uint32_t)p;
}

__global__ void snapshot_kernel(SnapshotArgs a) {
    const u64 factor = (u64)a.pfac * (u64)a.weight, hfac = (u64)a.pfac * (u64)a.halo_weight;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const uint4 b = __ldg(a.base + i), p = __ldg(a.present + i), h = __ldg(a.history + i);
        const u64 e = a.halo ? hfac * (u64)__ldg(a.halo + i) : 0;
        a.out[i] = make_uint4(snapshot_price(b.x, p.x, h.x, factor, e), snapshot_price(b.y, p.y, h.y, factor, e),
                              snapshot_price(b.z, p.z, h.z, factor, e), snapshot_price(b.w, p.w, h.w, factor, e));
    }
}

// Cell q of the (2r+1)^2 box around (x, y) on layer l, or kMax when it is off
// the board or a base obstacle (a footprint never claims an obstacle).
__device__ __forceinline__ uint32_t box_cell(uint32_t x, uint32_t y, uint32_t l, uint32_t r, uint32_t q, uint32_t w,
                                             uint32_t h, const uint32_t *cost) {
    const uint32_t side = 2 * r + 1;
    const int nx = (int)x + (int)(q % side) - (int)r, ny = (int)y + (int)(q / side) - (int)r;
    if (nx < 0 || ny < 0 || nx >= (int)w || ny >= (int)h) return kMax;
    const uint32_t c = (l * h + (uint32_t)ny) * w + (uint32_t)nx;
    return __ldg(cost + c) == kMax ? kMax : c;
}

__global__ void halo_kernel(HaloArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t plane = a.w * a.h;
    const uint32_t B = a.r ? (2 * a.r + 1) * (2 * a.r + 1) : 0, BV = a.vr ? (2 * a.vr + 1) * (2 * a.vr + 1) : 0;
    for (uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < a.n_list; item += warps) {
        const uint32_t net = a.list[item];
        const u64 p0 = a.offsets[net], p1 = a.offsets[net + 1];
        const u64 n = p1 - p0;
        // boxes around every path cell
        for (u64 t = lane; t < n * B; t += 32) {
            const uint32_t c = a.cells[p0 + t / B], r = c % plane;
            const uint32_t v = box_cell(r % a.w, r / a.w, c / plane, a.r, (uint32_t)(t % B), a.w, a.h, a.cost);
            if (v == kMax) continue;
            if (a.add) atomicAdd(a.halo + v, 1u);
            else atomicSub(a.halo + v, 1u);
        }
        // keepout boxes on both layers of every via step k -> k + 1
        if (BV && n > 1) {
            for (u64 t = lane; t < (n - 1) * 2 * BV; t += 32) {
                const u64 k = t / (2 * BV);
                const uint32_t c0 = a.cells[p0 + k], c1 = a.cells[p0 + k + 1];
                if (c0 % plane != c1 % plane) continue;  // not a via
                const uint32_t q = (uint32_t)(t % (2 * BV)), c = q < BV ? c0 : c1, r = c % plane;
                const uint32_t v = box_cell(r % a.w, r / a.w, c / plane, a.vr, q % BV, a.w, a.h, a.cost);
                if (v == kMax) continue;
                if (a.add) atomicAdd(a.halo + v, 1u);
                else atomicSub(a.halo + v, 1u);
            }
        }
    }
}

__global__ void emit_kernel(EmitArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t plane = a.w * a.h;
    const uint32_t B = a.r ? (2 * a.r + 1) * (2 * a.r + 1) : 0, BV = a.vr ? (2 * a.vr + 1) * (2 * a.vr + 1) : 0;
    for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < a.n_list; j += warps) {
        const uint32_t net = a.list[j];
        const u64 p0 = a.offsets[net], n = a.offsets[net + 1] - p0;
        const u64 hi = (u64)j << 32;
        unsigned long long *keys = a.keys + a.emit_off[j];
        uint32_t *vals = a.vals + a.emit_off[j];
        for (u64 t = lane; t < n * B; t += 32) {
            const uint32_t c = a.cells[p0 + t / B], r = c % plane;
            const uint32_t v = box_cell(r % a.w, r / a.w, c / plane, a.r, (uint32_t)(t % B), a.w, a.h, a.cost);
            keys[t] = v == kMax ? kNoKey : (hi | v);
            vals[t] = 1;
        }
        keys += n * B;
        vals += n * B;
        // the in-edge slots of every path cell that its own path uses
        for (u64 k = lane; k < n; k += 32) {
            const uint32_t c = a.cells[p0 + k];
            uint32_t bits = 0;
            int sa, sb;
            if (k > 0 && planar_slots(a.cells[p0 + k - 1], c, a.w, plane, &sa, &sb)) bits |= 1u << sb;
            if (k + 1 < n && planar_slots(c, a.cells[p0 + k + 1], a.w, plane, &sa, &sb)) bits |= 1u << sa;
            keys[k] = bits ? (hi | c) : kNoKey;
            vals[k] = bits << 24;
        }
        keys += n;
        vals += n;
        const u64 v0 = a.via_off[j], nv = a.via_off[j + 1] - v0;
        for (u64 t = lane; t < nv * 2 * BV; t += 32) {
            const u64 k = a.via_k[v0 + t / (2 * BV)];
            const uint32_t q = (uint32_t)(t % (2 * BV));
            const uint32_t c = a.cells[p0 + k + (q < BV ? 0 : 1)], r = c % plane;
            const uint32_t v = box_cell(r % a.w, r / a.w, c / plane, a.vr, q % BV, a.w, a.h, a.cost);
            keys[t] = v == kMax ? kNoKey : (hi | v);
            vals[t] = 1;
        }
    }
}

__device__ __forceinline__ uint32_t own_price(uint32_t base, uint32_t present, uint32_t history, uint32_t halo,
                                              uint32_t own_slot, uint32_t own_halo, u64 pf, u64 hf) {
    const uint32_t fp = present > own_slot ? present - own_slot : 0;  // saturating_sub
    const uint32_t fh = halo > own_halo ? halo - own_halo : 0;
    return snapshot_price(base, fp, history, pf, hf * (u64)fh);
}

__global__ void override_kernel(OverrideArgs a) {
    const u64 runs = *a.n_runs;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < runs && i < a.cap; i += stride) {
        const unsigned long long key = a.keys[i];
        if (key == kNoKey) continue;
        const uint32_t j = (uint32_t)(key >> 32), c = (uint32_t)key, v = a.vals[i];
        const uint32_t oh = v & kOwnHaloMask, os = v >> 24;
        const uint4 b = __ldg(a.base + c), p = __ldg(a.present + c), h = __ldg(a.history + c);
        const uint32_t hl = __ldg(a.halo + c);
        a.out_cells[i] = c;
        a.out_price[i] = make_uint4(own_price(b.x, p.x, h.x, hl, os & 1u, oh, a.pf, a.hf),
                                    own_price(b.y, p.y, h.y, hl, (os >> 1) & 1u, oh, a.pf, a.hf),
                                    own_price(b.z, p.z, h.z, hl, (os >> 2) & 1u, oh, a.pf, a.hf),
                                    own_price(b.w, p.w, h.w, hl, (os >> 3) & 1u, oh, a.pf, a.hf));
        if (i == 0 || (a.keys[i - 1] >> 32) != j) a.range[2 * j] = (uint32_t)i;
        if (i + 1 == runs || (a.keys[i + 1] >> 32) != j) a.range[2 * j + 1] = (uint32_t)(i + 1);
    }
}

// Group-aware overuse (the reference's scan, negotiated.rs:1923-1943, on edge
// slots): every planar step of every current path claims both of its slots for
// its net's connection group; a slot already claimed by another group is
// overused.  The outcome does not depend on the order of the claims: a slot is
// flagged exactly when two or more distinct groups use it.
__global__ void group_overuse_kernel(GroupArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t net = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; net < a.n_nets; net += warps) {
        const uint32_t g = a.group[net];
        const u64 p0 = a.offsets[net], p1 = a.offsets[net + 1];
        for (u64 k = p0 + lane; k + 1 < p1; k += 32) {
            const uint32_t u = a.cells[k], v = a.cells[k + 1];
            int su, sv;
            if (!planar_slots(u, v, a.w, a.plane, &su, &sv)) continue;
            const u64 iu = 4ull * u + su, iv = 4ull * v + sv;
            const uint32_t ou = atomicCAS(a.first + iu, kNoGroup, g);
            if (ou != kNoGroup && ou != g) a.over[iu] = 1;
            const uint32_t ov = atomicCAS(a.first + iv, kNoGroup, g);
            if (ov != kNoGroup && ov != g) a.over[iv] = 1;
        }
    }
}

__device__ __forceinline__ uint32_t bump(uint32_t h, bool over, uint32_t step, uint32_t *count) {
    if (!over) return h;
    ++*count;
    const uint32_t n = h + step;
    return n < h ? kMax : n;  // saturating_add
}

__global__ void overuse_kernel(OveruseArgs a) {
    uint32_t count = 0;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        bool ox, oy, oz, ow;
        if (a.over) {  // group-aware flags
            const uchar4 o = reinterpret_cast<const uchar4 *>(a.over)[i];
            ox = o.x, oy = o.y, oz = o.z, ow = o.w;
        } else {
            const uint4 p = a.present[i];
            ox = p.x >= 2, oy = p.y >= 2, oz = p.z >= 2, ow = p.w >= 2;
        }
        if (!(ox | oy | oz | ow)) continue;
        uint4 h = a.history[i];
        h.x = bump(h.x, ox, a.step, &count);
        h.y = bump(h.y, oy, a.step, &count);
        h.z = bump(h.z, oz, a.step, &count);
        h.w = bump(h.w, ow, a.step, &count);
        a.history[i] = h;
    }
    // every undirected edge owns two slots: the host halves the slot count
    for (int o = 16; o; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
    if ((threadIdx.x & 31) == 0 && count) atomicAdd(a.count, (unsigned long long)count);
}

__global__ void dirty_kernel(DirtyArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t net = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; net < a.n_nets; net += warps) {
        const u64 p0 = a.offsets[net], p1 = a.offsets[net + 1];
        bool hit = p0 == p1;  // unrouted: routed again next round
        for (u64 k = p0 + lane; !hit && k + 1 < p1; k += 32) {
            const uint32_t u = a.cells[k], v = a.cells[k + 1];
            int su, sv;
            if (planar_slots(u, v, a.w, a.plane, &su, &sv) &&
                (a.over ? __ldg(a.over + 4ull * v + sv) != 0 : __ldg(a.present + 4ull * v + sv) >= 2))
                hit = true;
        }
        hit = __any_sync(0xffffffffu, hit);
        if (lane == 0) a.flags[net] = hit ? 1 : 0;
    }
}

uint32_t grid_for(u64 work, uint32_t threads) {
    const u64 b = (work + threads - 1) / threads;
    return (uint32_t)(b < 1 ? 1 : (b > 148ull * 16 ? 148ull * 16 : b));
}

}  // namespace

cudaError_t occupancy_launch(const OccupancyArgs &a, cudaStream_t st) {
    if (!a.n_list) return cudaSuccess;
    occupancy_kernel<<<grid_for((u64)a.n_list * 32, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t snapshot_launch(const SnapshotArgs &a, cudaStream_t st) {
    if (!a.n) return cudaSuccess;
    snapshot_kernel<<<grid_for(a.n, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t overuse_launch(const OveruseArgs &a, cudaStream_t st) {
    if (!a.n) return cudaSuccess;
    overuse_kernel<<<grid_for(a.n, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t group_overuse_launch(const GroupArgs &a, cudaStream_t st) {
    if (!a.n_nets) return cudaSuccess;
    group_overuse_kernel<<<grid_for((u64)a.n_nets * 32, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t halo_launch(const HaloArgs &a, cudaStream_t st) {
    if (!a.n_list || !(a.r | a.vr)) return cudaSuccess;
    halo_kernel<<<grid_for((u64)a.n_list * 32, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t emit_launch(const EmitArgs &a, cudaStream_t st) {
    if (!a.n_list) return cudaSuccess;
    emit_kernel<<<grid_for((u64)a.n_list * 32, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t footprint_reduce(const unsigned long long *keys, const uint32_t *vals, unsigned long long *keys_sorted,
                             uint32_t *vals_sorted, unsigned long long *run_keys, uint32_t *run_vals,
                             uint32_t *n_runs, uint64_t n, int end_bit, void *temp, size_t *temp_bytes,
                             cudaStream_t st) {
    size_t need_sort = 0, need_reduce = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, need_sort, keys, keys_sorted, vals, vals_sorted, (int64_t)n,
                                                    0, end_bit, st);
    if (e != cudaSuccess) return e;
    e = cub::DeviceReduce::ReduceByKey(nullptr, need_reduce, keys_sorted, run_keys, vals_sorted, run_vals, n_runs,
                                       ::cuda::std::plus<uint32_t>(), (int64_t)n, st);
    if (e != cudaSuccess) return e;
    const size_t need = need_sort > need_reduce ? need_sort : need_reduce;
    if (!temp || *temp_bytes < need) {  // the caller grows the buffer and calls again
        *temp_bytes = need;
        return temp ? cudaErrorInvalidValue : cudaSuccess;
    }
    size_t bytes = *temp_bytes;
    e = cub::DeviceRadixSort::SortPairs(temp, bytes, keys, keys_sorted, vals, vals_sorted, (int64_t)n, 0, end_bit, st);
    if (e != cudaSuccess) return e;
    bytes = *temp_bytes;
    return cub::DeviceReduce::ReduceByKey(temp, bytes, keys_sorted, run_keys, vals_sorted, run_vals, n_runs,
                                          ::cuda::std::plus<uint32_t>(), (int64_t)n, st);
}

cudaError_t override_launch(const OverrideArgs &a, cudaStream_t st) {
    if (!a.cap) return cudaSuccess;
    override_kernel<<<grid_for(a.cap, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t dirty_launch(const DirtyArgs &a, cudaStream_t st) {
    if (!a.n_nets) return cudaSuccess;
    dirty_kernel<<<grid_for((u64)a.n_nets * 32, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace mrc
