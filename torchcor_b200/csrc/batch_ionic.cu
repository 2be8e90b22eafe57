// Batched ionic step: one launch covers every simulation of the batch, each
// block running the model of its group (the per-node work is the ionic_node the
// single-simulation kernel runs, with the same per-step arithmetic).
//
// Threads walk a virtual node space made of each simulation's 128-node tiles;
// a tile always lies in one simulation, so the simulation lookup (binary search
// over the tile prefix) is block-uniform.  Model constants are a kernel
// argument when every simulation of the group shares them (the common case:
// same parameters and dt), else read per simulation.
#include <cuda_runtime.h>
#include <string.h>

#include "batch.cuh"
#include "ionic_crn.cuh"
#include "ionic_ms.cuh"
#include "ionic_node.cuh"
#include "ionic_ttp.cuh"
#include "tcb_internal.h"

namespace tcb {
namespace {

constexpr int kThreads = kBatchTile;   // a block walks 128-node tiles
constexpr int kMaxTilesPerBlock = 8;   // consecutive tiles per block, at most
constexpr int kBlocksPerSmTarget = 16; // fewer tiles per block when the group is small

// A block walks tiles [blk * tpb, +tpb) of its group's virtual tile space
// (tpb = 1..8, so that small groups still fill the GPU); consecutive tiles
// mostly belong to one simulation, so its descriptor, table view and step view
// are set up once and again only when the walk crosses into the next
// simulation (the only points where the block syncs).
template <class M, bool SHARED>
__device__ __forceinline__ void ionic_tiles(const BatchWS* __restrict__ W, int g, int tpb, int64_t blk,
                                            const typename M::C& c0, MonoDev& sd, typename M::Tables& sT,
                                            int& s_lo) {
    const BatchGroup& G = W->groups[g];
    const int64_t total_tiles = G.tile_prefix[G.count];
    const int64_t t0 = blk * tpb;
    const int64_t t1 = t0 + tpb < total_tiles ? t0 + tpb : total_tiles;
    int lo = -1;
    int64_t first = 0, next = 0, step = 0;
    StepView sv = {};
    for (int64_t tile = t0; tile < t1; ++tile) {
        if (tile >= next) {   // block-uniform: entering a new simulation
            if (lo >= 0) __syncthreads();   // every thread is done with the staged view
            if (threadIdx.x == 0) {
                int l = lo < 0 ? 0 : lo + 1, h = G.count - 1;
                while (l < h) {
                    const int mid = (l + h + 1) >> 1;
                    if (G.tile_prefix[mid] <= tile) l = mid;
                    else h = mid - 1;
                }
                s_lo = l;
            }
            __syncthreads();
            lo = s_lo;
            const uint32_t* src = reinterpret_cast<const uint32_t*>(W->dev + G.idx[lo]);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
            for (int t = threadIdx.x; t < (int)(sizeof(MonoDev) / 4); t += blockDim.x) dst[t] = src[t];
            const uint32_t* ts = reinterpret_cast<const uint32_t*>(static_cast<const typename M::Tables*>(G.tables) + lo);
            uint32_t* td = reinterpret_cast<uint32_t*>(&sT);
            for (int t = threadIdx.x; t < (int)(sizeof(typename M::Tables) / 4); t += blockDim.x) td[t] = ts[t];
            first = G.tile_prefix[lo];
            next = G.tile_prefix[lo + 1];
            __syncthreads();
            step = sd.counter[0];
            if (step >= 1 && step <= sd.nt) sv = step_view(sd, step);
        }
        const int64_t node = (tile - first) * kBatchTile + threadIdx.x;
        if (step >= 1 && step <= sd.nt && node < sd.n) {
            const typename M::C& c = SHARED ? c0 : static_cast<const typename M::C*>(G.consts)[lo];
            ionic_node<M, QExact>(sd, c, sT, sv, node);
        }
    }
}

// Everything one launch needs for every model group of the batch.  A model
// appears in at most one group, so its shared constant block has a field of its
// own (read from the constant bank like any kernel argument).
struct IonicLaunch {
    const BatchWS* W;
    int32_t n_groups;
    int32_t group[kBatchGroups];          // launch order (heavier models first) -> group index
    int32_t tpb[kBatchGroups];
    int32_t shared[kBatchGroups];
    int64_t block_prefix[kBatchGroups + 1];
    MS::C ms;
    TTP::C ttp;
    CRN::C crn;
};

constexpr size_t kTablesBytes = sizeof(MS::Tables) > sizeof(TTP::Tables)
                                    ? (sizeof(MS::Tables) > sizeof(CRN::Tables) ? sizeof(MS::Tables) : sizeof(CRN::Tables))
                                    : (sizeof(TTP::Tables) > sizeof(CRN::Tables) ? sizeof(TTP::Tables) : sizeof(CRN::Tables));

template <class M>
__device__ __forceinline__ void run_group(const IonicLaunch& P, int k, int64_t blk, const typename M::C& c0,
                                          MonoDev& sd, unsigned char* tabs, int& s_lo) {
    auto& sT = *reinterpret_cast<typename M::Tables*>(tabs);
    if (P.shared[k]) ionic_tiles<M, true>(P.W, P.group[k], P.tpb[k], blk, c0, sd, sT, s_lo);
    else ionic_tiles<M, false>(P.W, P.group[k], P.tpb[k], blk, c0, sd, sT, s_lo);
}

// One launch for the ionic step of every simulation of the batch: blocks
// [block_prefix[k], block_prefix[k+1]) run the k-th group's model.  A batch with
// CRN groups runs an instance with every model, a batch without one without the
// CRN path; each is compiled for MINB = 4, 6, 8 or 12 blocks of 128 threads per SM
// (128, 80, 64 or 40 registers).  The defaults (no choice in the plan): 8 with
// CRN, where its state spills least, 12 without (measured on B200: 64 MS/TTP cubes
// 0.730 -> 0.714 ms a step at 12; a CRN-heavy batch 6 % slower at 12 than at 8);
// the batch tuner times the others.
template <bool WITH_CRN, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) batch_ionic_kernel(const IonicLaunch P) {
    __shared__ MonoDev sd;
    __shared__ __align__(16) unsigned char tabs[kTablesBytes];
    __shared__ int s_lo;
    int k = 0;
    while (k + 1 < P.n_groups && (int64_t)blockIdx.x >= P.block_prefix[k + 1]) ++k;
    const int64_t blk = (int64_t)blockIdx.x - P.block_prefix[k];
    switch (P.W->groups[P.group[k]].model) {
        case TCB_MODEL_MS: run_group<MS>(P, k, blk, P.ms, sd, tabs, s_lo); break;
        case TCB_MODEL_TTP: run_group<TTP>(P, k, blk, P.ttp, sd, tabs, s_lo); break;
        default:
            if constexpr (WITH_CRN) run_group<CRN>(P, k, blk, P.crn, sd, tabs, s_lo);
            break;
    }
}

}  // namespace

size_t model_consts_bytes(int model) {
    switch (model) {
        case TCB_MODEL_MS: return sizeof(MS::C);
        case TCB_MODEL_TTP: return sizeof(TTP::C);
        case TCB_MODEL_CRN: return sizeof(CRN::C);
    }
    return 0;
}

// Model constant block of a simulation (host), as the kernels read it.
int model_consts(int model, const double* params, void* out) {
    switch (model) {
        case TCB_MODEL_MS: {
            MS::C c = MS::derive(params);
            memcpy(out, &c, sizeof c);
            return TCB_OK;
        }
        case TCB_MODEL_TTP: {
            TTP::C c = TTP::derive(params);
            memcpy(out, &c, sizeof c);
            return TCB_OK;
        }
        case TCB_MODEL_CRN: {
            CRN::C c = CRN::derive(params);
            memcpy(out, &c, sizeof c);
            return TCB_OK;
        }
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}

size_t model_tables_bytes(int model) {
    switch (model) {
        case TCB_MODEL_MS: return sizeof(MS::Tables);
        case TCB_MODEL_TTP: return sizeof(TTP::Tables);
        case TCB_MODEL_CRN: return sizeof(CRN::Tables);
    }
    return 0;
}

// Lookup-table view (device pointers into the simulation's table array), host side.
int model_tables_view(int model, const float* tables, const double* params, void* out) {
    switch (model) {
        case TCB_MODEL_MS: {
            MS::Tables t = MS::tables(tables, params);
            memcpy(out, &t, sizeof t);
            return TCB_OK;
        }
        case TCB_MODEL_TTP: {
            TTP::Tables t = TTP::tables(tables, params);
            memcpy(out, &t, sizeof t);
            return TCB_OK;
        }
        case TCB_MODEL_CRN: {
            CRN::Tables t = CRN::tables(tables, params);
            memcpy(out, &t, sizeof t);
            return TCB_OK;
        }
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}

template <bool WITH_CRN>
int launch_ionic_instance(const IonicLaunch& P, unsigned blocks, int blocks_per_sm, cudaStream_t s) {
    switch (blocks_per_sm) {
        case 4: batch_ionic_kernel<WITH_CRN, 4><<<blocks, kThreads, 0, s>>>(P); break;
        case 6: batch_ionic_kernel<WITH_CRN, 6><<<blocks, kThreads, 0, s>>>(P); break;
        case 8: batch_ionic_kernel<WITH_CRN, 8><<<blocks, kThreads, 0, s>>>(P); break;
        case 12: batch_ionic_kernel<WITH_CRN, 12><<<blocks, kThreads, 0, s>>>(P); break;
        default: return fail(TCB_EINVAL, "batched ionic kernel: blocks per SM not 4, 6, 8 or 12");
    }
    TCB_CHECK_LAUNCH("batched ionic kernel");
    return TCB_OK;
}

int launch_batch_ionic_all(const BatchWS* ws_dev, int n_groups, const int32_t* models, const int64_t* tiles,
                           const int32_t* shared, const char (*consts)[1024], int tiles_per_block,
                           int blocks_per_sm, cudaStream_t s) {
    static_assert(sizeof(IonicLaunch) <= 4000, "kernel argument block");
    IonicLaunch P;
    memset(&P, 0, sizeof P);
    P.W = ws_dev;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // launch order: the heavier models first (TTP, CRN, then MS)
    int order[kBatchGroups], n = 0;
    for (int pass = 0; pass < 2; ++pass)
        for (int g = 0; g < n_groups; ++g)
            if ((models[g] == TCB_MODEL_MS) == (pass == 1) && tiles[g] > 0) order[n++] = g;
    P.n_groups = n;
    bool with_crn = false;
    int64_t blocks = 0;
    for (int k = 0; k < n; ++k) {
        const int g = order[k];
        // tiles per block: the plan's choice (a tuning knob), else sized from the group
        const int64_t per = (tiles[g] + (int64_t)sms * kBlocksPerSmTarget - 1) / ((int64_t)sms * kBlocksPerSmTarget);
        const int tpb = tiles_per_block > 0 ? tiles_per_block
                                            : (int)(per < 1 ? 1 : per > kMaxTilesPerBlock ? kMaxTilesPerBlock : per);
        P.group[k] = g;
        P.tpb[k] = tpb;
        P.shared[k] = shared[g];
        P.block_prefix[k] = blocks;
        blocks += (tiles[g] + tpb - 1) / tpb;
        with_crn |= models[g] == TCB_MODEL_CRN;
        if (shared[g]) {
            switch (models[g]) {
                case TCB_MODEL_MS: memcpy(&P.ms, consts[g], sizeof P.ms); break;
                case TCB_MODEL_TTP: memcpy(&P.ttp, consts[g], sizeof P.ttp); break;
                case TCB_MODEL_CRN: memcpy(&P.crn, consts[g], sizeof P.crn); break;
                default: return fail(TCB_EINVAL, "unknown ionic model in batch");
            }
        }
    }
    P.block_prefix[n] = blocks;
    if (blocks < 1) return TCB_OK;
    if (blocks > INT32_MAX) return fail(TCB_ERANGE, "batched ionic grid too large");
    if (with_crn) return launch_ionic_instance<true>(P, (unsigned)blocks, blocks_per_sm > 0 ? blocks_per_sm : 8, s);
    return launch_ionic_instance<false>(P, (unsigned)blocks, blocks_per_sm > 0 ? blocks_per_sm : 12, s);
}

}  // namespace tcb
