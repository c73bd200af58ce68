// kernels.h — launch interface between the host runtime and relax.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "device.cuh"

namespace mrc {

constexpr int kRelaxThreads = 256;

struct RelaxArgs {
    DevBoard board;
    const DevField *fields;     // in processing order (largest windows first)
    uint32_t n_fields;
    const uint32_t *pads;       // sorted pad lists, indexed by DevField offsets
    uint32_t *dist, *hops;      // label arenas
    uint32_t *work_counter;     // zeroed before launch
    uint32_t *tile_scratch;     // per CTA: queue[max_tiles] + in-queue bitmap
    uint32_t scratch_stride;
    uint32_t max_tiles;
    uint32_t tile_h;            // 32, 16 or 8
    uint32_t activation_factor; // tile activations allowed per tile (guard)
    uint32_t *status;           // error bits (0 = fine)
};

struct PathArgs {
    DevBoard board;
    const DevField *fields;
    uint32_t n_fields;
    const uint32_t *pads;
    const uint32_t *dist, *hops;
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
    const uint32_t *in_dist, *in_hops;
    uint32_t *out_dist, *out_hops;
    uint32_t *changed;
};

size_t relax_smem_bytes(uint32_t layers, uint32_t tile_h, bool directed);
cudaError_t relax_configure(bool directed, size_t smem);
cudaError_t relax_occupancy(bool directed, size_t smem, int *blocks_per_sm);
cudaError_t relax_launch(const RelaxArgs &a, uint32_t grid, size_t smem, cudaStream_t st);
cudaError_t path_launch(const PathArgs &a, cudaStream_t st);
cudaError_t plain_round_launch(const PlainArgs &a, uint64_t wcells, cudaStream_t st);

}  // namespace mrc
