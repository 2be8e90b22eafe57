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
#include "bulk.cuh"
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

// ---------------------------------------------------------------------------
// Staged form (the plan's ionic_staged): the state rows, u, AT/RT and stimulus
// bits of a block's next 128-node tile are copied into shared memory by bulk
// asynchronous copies (cp.async.bulk from this GPU's memory, no multicast,
// completion counted on an mbarrier, bounded waits) while the block computes the
// current tile from shared memory, as mono_ionic_staged_kernel does for one
// simulation.  A block walks a contiguous range of its group's tiles (the launch
// sizes the grid to the register budget's blocks per SM); the two-stage pipeline
// runs over each stretch of that range lying in one simulation and restarts at
// the next.  Padding nodes (n <= i < n_pad) are computed like the others, on
// memory that exists, and nothing reads their results; their u stays 0, so AT/RT
// are never set for them, and snapshots are written for real nodes only.  TTP and
// CRN take the division policy of the single-simulation default (QFast); the
// Mitchell-Schaeffer group of a staged launch runs the unstaged walk.
template <bool WITH_CRN>
struct BatchStage {
    static constexpr int kMaxStates = WITH_CRN ? (CRN::kStates > TTP::kStates ? CRN::kStates : TTP::kStates)
                                               : (TTP::kStates > MS::kStates ? TTP::kStates : MS::kStates);
    static constexpr int kRows = kMaxStates + 4;   // state rows, u, AT, RT, stimulus bits
    static constexpr size_t kBytes = 2ull * kRows * kBatchTile * sizeof(float);   // both stages
};

template <class M>
struct StagedPolicy {
    using Q = QFast;
};

// Walks tiles [blk*tpb, +tpb) of group g; false after a timed-out copy wait (the
// error word is set; the block returns).
template <class M, bool SHARED, int ROWS>
__device__ __forceinline__ bool staged_tiles(const BatchWS* __restrict__ W, int g, int tpb, int64_t blk,
                                             const typename M::C& c0, MonoDev& sd, typename M::Tables& sT,
                                             int& s_lo, float* stage, uint64_t* bar, uint32_t& phase,
                                             uint32_t& drop) {
    using Q = typename StagedPolicy<M>::Q;
    constexpr int S = M::kStates, T = kBatchTile;
    const BatchGroup& G = W->groups[g];
    const int64_t total_tiles = G.tile_prefix[G.count];
    const int64_t t0 = blk * tpb;
    const int64_t t1 = t0 + tpb < total_tiles ? t0 + tpb : total_tiles;
    const int tid = threadIdx.x;
    int lo = -1;
    int64_t tile = t0;
    while (tile < t1) {
        // enter the simulation of `tile` (block-uniform)
        if (lo >= 0) __syncthreads();   // every thread is done with the previous view
        if (tid == 0) {
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
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(W->dev + G.idx[lo]);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
            for (int t = tid; t < (int)(sizeof(MonoDev) / 4); t += blockDim.x) dst[t] = src[t];
            const uint32_t* ts = reinterpret_cast<const uint32_t*>(static_cast<const typename M::Tables*>(G.tables) + lo);
            uint32_t* td = reinterpret_cast<uint32_t*>(&sT);
            for (int t = tid; t < (int)(sizeof(typename M::Tables) / 4); t += blockDim.x) td[t] = ts[t];
        }
        const int64_t first = G.tile_prefix[lo];
        const int64_t end = G.tile_prefix[lo + 1] < t1 ? G.tile_prefix[lo + 1] : t1;
        __syncthreads();
        const int64_t step = sd.counter[0];
        if (step < 1 || step > sd.nt) {   // this simulation does not step now
            tile = end;
            continue;
        }
        const StepView sv = step_view(sd, step);
        const typename M::C& c = SHARED ? c0 : static_cast<const typename M::C*>(G.consts)[lo];
        // thread 0: copy tile t of this simulation into stage st
        auto issue = [&](int st, int64_t t) {
            const int64_t i0 = (t - first) * T;
            float* buf = stage + (size_t)st * ROWS * T;
            constexpr uint32_t bytes = T * sizeof(float);
            const uint32_t total = bytes * (S + 1) + (sv.do_atrt ? 2 * bytes : 0) + (sv.smask ? bytes : 0);
            fence_proxy_async_smem();
            mbar_arrive_tx(&bar[st], total);
            if (drop) {   // test hook: this issue's bytes never arrive, the wait runs out
                drop = 0;
                return;
            }
            for (int k = 0; k < S; ++k) bulk_load(buf + k * T, sd.state + k * sd.n_pad + i0, bytes, &bar[st]);
            bulk_load(buf + S * T, sv.u + i0, bytes, &bar[st]);
            if (sv.do_atrt) {
                bulk_load(buf + (S + 1) * T, sd.at + i0, bytes, &bar[st]);
                bulk_load(buf + (S + 2) * T, sd.rt + i0, bytes, &bar[st]);
            }
            if (sv.smask) bulk_load(buf + (S + 3) * T, sd.stim_bits + i0, bytes, &bar[st]);
        };
        if (tid == 0) {
            issue(0, tile);
            if (tile + 1 < end) issue(1, tile + 1);
        }
        int k = 0;
        for (int64_t t = tile; t < end; ++t, ++k) {
            const int st = k & 1;
            const bool ok = __syncthreads_and(mbar_wait_thread(&bar[st], (phase >> st) & 1u, W->wait.timeout_ns));
            if (!ok) {
                // a copy did not complete in time: record it, give the other stage's
                // copies (issued for the next tile) a bounded wait, and return
                if (tid == 0) atomicCAS(W->err, 0, TCB_ETIMEOUT);
                if (t + 1 < end) mbar_wait_thread(&bar[st ^ 1], (phase >> (st ^ 1)) & 1u, W->wait.timeout_ns);
                return false;
            }
            phase ^= 1u << st;
            const float* buf = stage + (size_t)st * ROWS * T;
            const int64_t i = (t - first) * T + tid;
            const float v = buf[S * T + tid];
            if (sv.do_atrt) {
                float a = buf[(S + 1) * T + tid];
                if (v > 0.0f && a == -1.0f) {   // padding nodes keep u = 0 and never pass
                    a = sv.t_prev;
                    sd.at[i] = a;
                }
                if (a > 0.0f && v < -70.0f && buf[(S + 2) * T + tid] == -1.0f) sd.rt[i] = sv.t_prev;
            }
            if (sv.snap && i < sd.n) sv.snap[i] = v;
            float s[S];
#pragma unroll
            for (int q = 0; q < S; ++q) s[q] = buf[q * T + tid];
            float b = v * sd.cm +
                      sd.dt * Q::div(M::template step<Q>(v, s, c, sT, M::node_g(c, sd.node_params, sd.n_pad, i)),
                                     100.0f);
#pragma unroll
            for (int q = 0; q < S; ++q) sd.state[q * sd.n_pad + i] = s[q];
            if (sv.smask) {
                const uint32_t on = reinterpret_cast<const uint32_t*>(buf + (S + 3) * T)[tid] & sv.smask;
                if (on) b = b + sd.dt * Q::div(stim_sum(sd, sv.smask, on), 100.0f);
            }
            sd.bp[i] = b;
            __syncthreads();   // every thread is done with this stage
            if (tid == 0 && t + 2 < end) issue(st, t + 2);
        }
        tile = end;
    }
    return true;
}

template <class M, int ROWS>
__device__ __forceinline__ bool run_group_staged(const IonicLaunch& P, int k, int64_t blk, const typename M::C& c0,
                                                 MonoDev& sd, unsigned char* tabs, int& s_lo, float* stage,
                                                 uint64_t* bar, uint32_t& phase, uint32_t& drop) {
    auto& sT = *reinterpret_cast<typename M::Tables*>(tabs);
    if (P.shared[k])
        return staged_tiles<M, true, ROWS>(P.W, P.group[k], P.tpb[k], blk, c0, sd, sT, s_lo, stage, bar, phase, drop);
    return staged_tiles<M, false, ROWS>(P.W, P.group[k], P.tpb[k], blk, c0, sd, sT, s_lo, stage, bar, phase, drop);
}

template <bool WITH_CRN, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) batch_ionic_staged_kernel(const IonicLaunch P) {
    constexpr int ROWS = BatchStage<WITH_CRN>::kRows;
    extern __shared__ __align__(128) float stage[];      // [2][ROWS][128]
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ MonoDev sd;
    __shared__ __align__(16) unsigned char tabs[kTablesBytes];
    __shared__ int s_lo;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0]);
        mbar_init(&bar[1]);
        mbar_init_fence();
    }
    __syncthreads();
    uint32_t phase = 0;
    // test hook (TCB_TEST_WAIT_STALL=copy): block 0's first copies are not made
    uint32_t drop = (P.W->wait.drop_first_copy && blockIdx.x == 0) ? 1u : 0u;
    int k = 0;
    while (k + 1 < P.n_groups && (int64_t)blockIdx.x >= P.block_prefix[k + 1]) ++k;
    const int64_t blk = (int64_t)blockIdx.x - P.block_prefix[k];
    switch (P.W->groups[P.group[k]].model) {
        // Mitchell-Schaeffer's one state and few operations leave nothing for the
        // stage to hide: its group takes the unstaged walk (short blocks)
        case TCB_MODEL_MS: run_group<MS>(P, k, blk, P.ms, sd, tabs, s_lo); break;
        case TCB_MODEL_TTP: run_group_staged<TTP, ROWS>(P, k, blk, P.ttp, sd, tabs, s_lo, stage, bar, phase, drop); break;
        default:
            if constexpr (WITH_CRN)
                run_group_staged<CRN, ROWS>(P, k, blk, P.crn, sd, tabs, s_lo, stage, bar, phase, drop);
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
int launch_ionic_staged(const IonicLaunch& P, unsigned blocks, int blocks_per_sm, cudaStream_t s) {
    constexpr size_t smem = BatchStage<WITH_CRN>::kBytes;
    switch (blocks_per_sm) {
        case 4: batch_ionic_staged_kernel<WITH_CRN, 4><<<blocks, kThreads, smem, s>>>(P); break;
        case 6: batch_ionic_staged_kernel<WITH_CRN, 6><<<blocks, kThreads, smem, s>>>(P); break;
        case 8: batch_ionic_staged_kernel<WITH_CRN, 8><<<blocks, kThreads, smem, s>>>(P); break;
        default: return fail(TCB_EINVAL, "staged batched ionic kernel: blocks per SM not 4, 6 or 8");
    }
    TCB_CHECK_LAUNCH("staged batched ionic kernel");
    return TCB_OK;
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
                           int blocks_per_sm, int staged, cudaStream_t s) {
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
    // the staged form's TTP and CRN groups walk contiguous tile ranges, each group
    // over as many blocks as the register budget keeps resident (the groups run
    // heavier first, so each fills the GPU in turn); Mitchell-Schaeffer takes the
    // unstaged walk's short blocks, which fill the slots as the others finish
    const int staged_bps = blocks_per_sm > 0 ? blocks_per_sm : 6;
    for (int k = 0; k < n; ++k) {
        const int g = order[k];
        int tpb;
        if (tiles_per_block > 0) {   // the plan's choice (a tuning knob)
            tpb = tiles_per_block;
        } else if (staged && models[g] != TCB_MODEL_MS) {
            const int64_t want = (int64_t)sms * staged_bps;
            const int64_t per = (tiles[g] + want - 1) / want;
            tpb = (int)(per < 1 ? 1 : per > kBatchMaxTilesPerBlock ? kBatchMaxTilesPerBlock : per);
        } else {                      // sized from the group
            const int64_t per =
                (tiles[g] + (int64_t)sms * kBlocksPerSmTarget - 1) / ((int64_t)sms * kBlocksPerSmTarget);
            tpb = (int)(per < 1 ? 1 : per > kMaxTilesPerBlock ? kMaxTilesPerBlock : per);
        }
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
    if (staged) {
        if (with_crn) return launch_ionic_staged<true>(P, (unsigned)blocks, staged_bps, s);
        return launch_ionic_staged<false>(P, (unsigned)blocks, staged_bps, s);
    }
    if (with_crn) return launch_ionic_instance<true>(P, (unsigned)blocks, blocks_per_sm > 0 ? blocks_per_sm : 8, s);
    return launch_ionic_instance<false>(P, (unsigned)blocks, blocks_per_sm > 0 ? blocks_per_sm : 12, s);
}

}  // namespace tcb
