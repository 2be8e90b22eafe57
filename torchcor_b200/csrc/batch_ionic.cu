// Batched ionic step: one launch per ionic model covers every simulation of
// that model in the batch (compiled with -fmad=false, like ionic.cu; the
// per-node work is the same ionic_node the single-simulation kernel runs).
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

// resident blocks per SM the register budget is sized for (MS: 42 registers)
template <class M>
constexpr int min_blocks() { return M::kStates > 4 ? 8 : 12; }

// A block covers tiles [blockIdx.x * tpb, +tpb) of the group's virtual tile
// space (tpb = 1..8, so that small groups still fill the GPU);
// consecutive tiles mostly belong to one simulation, so its descriptor, table
// view and step view are set up once and again only when the walk crosses into
// the next simulation (the only points where the block syncs).
template <class M, bool SHARED>
__global__ void __launch_bounds__(kThreads, min_blocks<M>()) batch_ionic_kernel(const BatchWS* __restrict__ W,
                                                                                int g, int tpb,
                                                                                typename M::C c0) {
    __shared__ MonoDev sd;
    __shared__ typename M::Tables sT;
    __shared__ int s_lo;
    const BatchGroup& G = W->groups[g];
    const int64_t total_tiles = G.tile_prefix[G.count];
    const int64_t t0 = (int64_t)blockIdx.x * tpb;
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
            ionic_node<M>(sd, c, sT, sv, node);
        }
    }
}

template <class M>
int launch(const BatchWS* W, int g, int64_t total_tiles, const void* shared_consts, cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t per_block = (total_tiles + (int64_t)sms * kBlocksPerSmTarget - 1) / ((int64_t)sms * kBlocksPerSmTarget);
    const int tpb = (int)(per_block < 1 ? 1 : per_block > kMaxTilesPerBlock ? kMaxTilesPerBlock : per_block);
    const int64_t blocks = (total_tiles + tpb - 1) / tpb;
    if (blocks < 1) return TCB_OK;
    if (blocks > INT32_MAX) return fail(TCB_ERANGE, "batched ionic grid too large");
    typename M::C c;
    memset(&c, 0, sizeof c);
    if (shared_consts) {
        memcpy(&c, shared_consts, sizeof c);
        batch_ionic_kernel<M, true><<<(unsigned)blocks, kThreads, 0, s>>>(W, g, tpb, c);
    } else {
        batch_ionic_kernel<M, false><<<(unsigned)blocks, kThreads, 0, s>>>(W, g, tpb, c);
    }
    TCB_CHECK_LAUNCH("batched ionic kernel");
    return TCB_OK;
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

int launch_batch_ionic(const BatchWS* ws_dev, const BatchWS& host, int g, int64_t total_tiles,
                       const void* shared_consts, cudaStream_t s) {
    switch (host.groups[g].model) {
        case TCB_MODEL_MS: return launch<MS>(ws_dev, g, total_tiles, shared_consts, s);
        case TCB_MODEL_TTP: return launch<TTP>(ws_dev, g, total_tiles, shared_consts, s);
        case TCB_MODEL_CRN: return launch<CRN>(ws_dev, g, total_tiles, shared_consts, s);
    }
    return fail(TCB_EINVAL, "unknown ionic model in batch");
}

}  // namespace tcb
