// Device workspace of a batch of monodomain simulations (built by
// tcb_batch_prepare, read by the batched ionic and CG kernels).
//
// The simulations keep their own arrays (MonoDev each, plus a compact CgView
// of the fields the CG kernel reads).  The CG kernel splits the 32-row slices
// of the simulations that still iterate evenly over its blocks, again at every
// pass; a virtual tile space (128-node tiles) per ionic model drives the ionic
// kernels.
#pragma once
#include <stdint.h>

#include "mono.cuh"

namespace tcb {

constexpr int kBatchMaxSims = 1024;        // simulations per batch
constexpr int kBatchMaxPerBlock = 64;      // simulations staged at once by one CG block
constexpr int kBatchMaxBlocks = 1024;      // CG blocks of a batch
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

// what the batched CG kernel reads of one simulation
struct CgView {
    int64_t n, n_pad;
    const int64_t* slice_ptr;
    const int32_t* col;
    const int16_t* dcol;       // int16 column offsets from the row, or null
    const float *mv, *kv, *av, *dinv;
    float *x, *bp, *r, *p, *ap, *z, *p2;
    float cm;
    int32_t linear_guess, a_split, pad;
};

struct BatchWS {
    int32_t n, pad;            // simulations
    int64_t total_slices;
    const MonoDev* dev;        // [n]
    const CgView* cg;          // [n]
    const int32_t* slices;     // [n] 32-row slices of each simulation
    double* parts;             // [3 values][n][nb] per-simulation block partials
    uint32_t* bar;             // [4] grid barrier words
    int32_t* err;              // [1] error word
    cgk::WaitLimit wait;       // bounded-wait limits (grid barrier, bulk-copy mbarriers)
    BatchGroup groups[kBatchGroups];
};

constexpr int kBatchMaxTilesPerBlock = 64;   // tcb_batch_set_ionic's upper limit
int launch_batch_ionic_all(const BatchWS* ws_dev, int n_groups, const int32_t* models, const int64_t* tiles,
                           const int32_t* shared, const char (*consts)[1024], int tiles_per_block,
                           int blocks_per_sm, int staged, cudaStream_t s);
// register budgets of the batched ionic kernel (blocks of 128 threads per SM); 0 = default
inline bool batch_ionic_blocks_ok(int b, int staged) {
    return b == 0 || b == 4 || b == 6 || b == 8 || (b == 12 && !staged);
}
// batched CG variants: 1 / 2 = streaming, sized for 1 / 2 blocks per SM;
// 3 = ELL streams staged in shared memory by bulk copies, 1 block per SM
// flags: the (int16 columns 4, A rebuilt 2, linear guess 1) combination all the
// batch's simulations share, or -1 (the streaming variants specialise on it)
int launch_batch_cg(const BatchWS* ws_dev, int nb, size_t smem, int variant, int stage_bytes, int flags,
                    cudaStream_t s);
size_t batch_cg_smem(int n);
size_t batch_cg_smem_variant(int n, int variant);
int batch_cg_stage_bytes(int n);                    // 0 if the staged variant does not fit
int batch_cg_max_blocks(size_t smem, int variant, int flags);  // 0 if that variant cannot be resident

}  // namespace tcb
