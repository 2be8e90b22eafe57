// Device workspace of a batch of monodomain simulations (built by
// tcb_batch_prepare, read by the batched ionic and CG kernels).
//
// The simulations keep their own arrays (MonoDev each).  A virtual slice
// space (the simulations' 32-row slices one after another) is split evenly
// over the CG blocks; a virtual tile space (128-node tiles) per ionic model
// drives the ionic kernels.
#pragma once
#include <stdint.h>

#include "mono.cuh"

namespace tcb {

constexpr int kBatchMaxSims = 1024;        // simulations per batch
constexpr int kBatchMaxPerBlock = 64;      // simulations overlapping one CG block's slice range
constexpr int kBatchTile = 128;            // nodes per ionic tile (n_pad is a multiple of it)
constexpr int kBatchGroups = 3;            // one per ionic model

struct BatchGroup {
    int32_t model;             // TCB_MODEL_*, 0 = unused
    int32_t count;             // simulations of this model
    int32_t shared_consts;     // 1 if all share one constant block (passed as a kernel argument)
    int32_t pad;
    const int32_t* idx;        // [count] simulation index
    const int64_t* tile_prefix;  // [count+1] first virtual tile of each
    const void* consts;        // [count] model constant blocks (M::C)
    const void* tables;        // [count] lookup-table views (M::Tables)
};

struct BatchWS {
    int32_t n, nb;             // simulations, CG blocks
    int32_t parts_stride;      // nb + n
    int32_t pad;
    int64_t total_slices;
    const MonoDev* dev;        // [n]
    const int64_t* slice_prefix;  // [n+1]
    const int32_t* blk_first;  // [nb] first simulation overlapping the block's slice range
    const int32_t* blk_count;  // [nb] simulations overlapping it
    const int32_t* blk_off;    // [nb] offset of the block's partials
    const int32_t* inst_b0;    // [n] first block overlapping the simulation
    const int32_t* inst_b1;    // [n] last block overlapping it
    double* parts;             // [2 parities][2 values][parts_stride]
    uint32_t* bar;             // [4] grid barrier words
    int32_t* err;              // [1] error word
    BatchGroup groups[kBatchGroups];
};

int launch_batch_ionic(const BatchWS* ws_dev, const BatchWS& ws_host_view, int g, int64_t total_tiles,
                       const void* shared_consts_host, cudaStream_t s);
int launch_batch_cg(const BatchWS* ws_dev, int nb, size_t smem, cudaStream_t s);
size_t batch_cg_smem(int n);
int batch_cg_max_blocks(size_t smem);

}  // namespace tcb
