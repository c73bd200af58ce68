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
#include <cuda_runtime.h>

#include <cstdint>

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

__device__ __forceinline__ uint32_t snapshot_price(uint32_t base, uint32_t present, uint32_t history, u64 factor) {
    if (base == kMax) return kMax;  // a blocked edge stays blocked
    const u64 p = (u64)base + (u64)history + factor * (u64)present;
    return p > (u64)kCap ? kCap : (uint32_t)p;
}

__global__ void snapshot_kernel(SnapshotArgs a) {
    const u64 factor = (u64)a.pfac * (u64)a.weight;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const uint4 b = __ldg(a.base + i), p = __ldg(a.present + i), h = __ldg(a.history + i);
        a.out[i] = make_uint4(snapshot_price(b.x, p.x, h.x, factor), snapshot_price(b.y, p.y, h.y, factor),
                              snapshot_price(b.z, p.z, h.z, factor), snapshot_price(b.w, p.w, h.w, factor));
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

cudaError_t dirty_launch(const DirtyArgs &a, cudaStream_t st) {
    if (!a.n_nets) return cudaSuccess;
    dirty_kernel<<<grid_for((u64)a.n_nets * 32, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace mrc
