// Host side of batched simulations: the workspace layout, the plan (block
// ranges, per-simulation reduction ranges, ionic model groups) and the step
// loop.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "batch.cuh"
#include "cg_common.cuh"
#include "tcb_internal.h"

namespace tcb {

size_t model_consts_bytes(int model);
int model_consts(int model, const double* params, void* out);
size_t model_tables_bytes(int model);
int model_tables_view(int model, const float* tables, const double* params, void* out);
int validate_mono(const tcb_mono* m);

namespace {

constexpr size_t kAlign = 256;
constexpr size_t kMaxConsts = 1024;   // bytes of one model constant block (checked below)
constexpr size_t kMaxTables = 256;    // bytes of one lookup-table view

size_t up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

struct Layout {
    size_t ws, dev, slice_prefix, blk_first, blk_count, blk_off, inst_b0, inst_b1, parts, bar, err;
    size_t g_idx[kBatchGroups], g_tiles[kBatchGroups], g_consts[kBatchGroups], g_tabs[kBatchGroups];
    size_t total;
};

Layout layout(int n, int nb) {
    Layout L;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        size_t at = o;
        o = up(o + bytes);
        return at;
    };
    L.ws = take(sizeof(BatchWS));
    L.dev = take(sizeof(MonoDev) * n);
    L.slice_prefix = take(sizeof(int64_t) * (n + 1));
    L.blk_first = take(sizeof(int32_t) * nb);
    L.blk_count = take(sizeof(int32_t) * nb);
    L.blk_off = take(sizeof(int32_t) * nb);
    L.inst_b0 = take(sizeof(int32_t) * n);
    L.inst_b1 = take(sizeof(int32_t) * n);
    L.parts = take(sizeof(double) * 4 * (size_t)(nb + n));
    L.bar = take(sizeof(uint32_t) * 4);
    L.err = take(sizeof(int32_t) * 4);
    for (int g = 0; g < kBatchGroups; ++g) {
        L.g_idx[g] = take(sizeof(int32_t) * n);
        L.g_tiles[g] = take(sizeof(int64_t) * (n + 1));
        L.g_consts[g] = take(kMaxConsts * n);
        L.g_tabs[g] = take(kMaxTables * n);
    }
    L.total = o;
    return L;
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int64_t tcb_batch_workspace_bytes(int32_t n_sims) {
    if (n_sims < 1 || n_sims > kBatchMaxSims) return -1;
    return (int64_t)layout(n_sims, cgk::kMaxBlocks).total;
}

extern "C" int tcb_batch_prepare(const tcb_mono* sims, int32_t n, void* workspace, int64_t bytes,
                                 tcb_batch_plan* plan) {
    if (!sims || !workspace || !plan || n < 1) return fail(TCB_EINVAL, "tcb_batch_prepare: bad arguments");
    if (n > kBatchMaxSims) return fail(TCB_ERANGE, "tcb_batch_prepare: more than 1024 simulations");
    static_assert(sizeof(MonoDev) < 4096, "MonoDev size");
    for (int m = TCB_MODEL_MS; m <= TCB_MODEL_CRN; ++m)
        if (model_consts_bytes(m) > kMaxConsts || model_tables_bytes(m) > kMaxTables)
            return fail(TCB_EINVAL, "model constants exceed the batch slot");
    std::vector<MonoDev> devs(n);
    std::vector<int64_t> sp(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        int st = validate_mono(&sims[i]);
        if (st) return st;
        if (sims[i].n_pad % kBatchTile != 0) return fail(TCB_EINVAL, "n_pad must be a multiple of 128");
        if (!sims[i].z || !sims[i].p2) return fail(TCB_EINVAL, "batched simulations need z and p2 buffers");
        devs[i] = make_dev(&sims[i]);
        sp[i + 1] = sp[i] + sims[i].n_slices;
    }
    const int64_t S = sp[n];
    const size_t smem = batch_cg_smem(n);
    int cap = batch_cg_max_blocks(smem);
    if (cap < 1) return fail(TCB_ECUDA, "batched CG kernel cannot be resident");
    int64_t want = ceil_div(S, cgk::kMinSlicesPerBlock);
    int nb = (int)std::max<int64_t>(1, std::min<int64_t>(want, cap));
    Layout L = layout(n, nb);
    if ((int64_t)L.total > bytes) return fail(TCB_ERANGE, "batch workspace too small");

    std::vector<char> host(L.total, 0);
    char* base = static_cast<char*>(workspace);
    auto hp = [&](size_t off) { return host.data() + off; };
    auto dp = [&](size_t off) { return base + off; };

    BatchWS ws;
    memset(&ws, 0, sizeof ws);
    ws.n = n;
    ws.nb = nb;
    ws.parts_stride = nb + n;
    ws.total_slices = S;
    ws.dev = reinterpret_cast<const MonoDev*>(dp(L.dev));
    ws.slice_prefix = reinterpret_cast<const int64_t*>(dp(L.slice_prefix));
    ws.blk_first = reinterpret_cast<const int32_t*>(dp(L.blk_first));
    ws.blk_count = reinterpret_cast<const int32_t*>(dp(L.blk_count));
    ws.blk_off = reinterpret_cast<const int32_t*>(dp(L.blk_off));
    ws.inst_b0 = reinterpret_cast<const int32_t*>(dp(L.inst_b0));
    ws.inst_b1 = reinterpret_cast<const int32_t*>(dp(L.inst_b1));
    ws.parts = reinterpret_cast<double*>(dp(L.parts));
    ws.bar = reinterpret_cast<uint32_t*>(dp(L.bar));
    ws.err = reinterpret_cast<int32_t*>(dp(L.err));
    memcpy(hp(L.dev), devs.data(), sizeof(MonoDev) * n);
    memcpy(hp(L.slice_prefix), sp.data(), sizeof(int64_t) * (n + 1));

    // block ranges over the virtual slice space and per-simulation block ranges
    int32_t* bf = reinterpret_cast<int32_t*>(hp(L.blk_first));
    int32_t* bc = reinterpret_cast<int32_t*>(hp(L.blk_count));
    int32_t* bo = reinterpret_cast<int32_t*>(hp(L.blk_off));
    int32_t* b0 = reinterpret_cast<int32_t*>(hp(L.inst_b0));
    int32_t* b1 = reinterpret_cast<int32_t*>(hp(L.inst_b1));
    for (int i = 0; i < n; ++i) {
        b0[i] = nb;
        b1[i] = -1;
    }
    int32_t acc = 0;
    int i = 0;
    for (int b = 0; b < nb; ++b) {
        const int64_t vb = (int64_t)b * S / nb, ve = (int64_t)(b + 1) * S / nb;
        while (i < n - 1 && sp[i + 1] <= vb) ++i;
        int last = i;
        while (last < n - 1 && sp[last + 1] < ve) ++last;
        if (ve <= vb) last = i - 1;   // empty range (only if S < nb)
        bf[b] = i;
        bc[b] = last - i + 1;
        bo[b] = acc;
        acc += std::max(0, bc[b]);
        if (bc[b] > kBatchMaxPerBlock)
            return fail(TCB_ERANGE, "more than 64 simulations overlap one CG block (too many tiny simulations)");
        for (int j = i; j <= last; ++j) {
            b0[j] = std::min(b0[j], b);
            b1[j] = std::max(b1[j], b);
        }
    }
    if (acc > nb + n) return fail(TCB_EINVAL, "batch partial layout overflow");
    for (int j = 0; j < n; ++j)
        if (b1[j] < b0[j]) return fail(TCB_EINVAL, "simulation with no slices in the batch");

    // ionic groups
    plan->n_groups = 0;
    int model_slot[4] = {-1, -1, -1, -1};
    for (int j = 0; j < n; ++j) {
        const int m = sims[j].model;
        if (m < TCB_MODEL_MS || m > TCB_MODEL_CRN) return fail(TCB_EINVAL, "unknown ionic model");
        if (model_slot[m] < 0) model_slot[m] = plan->n_groups++;
    }
    for (int g = 0; g < kBatchGroups; ++g) {
        plan->group_model[g] = 0;
        plan->group_tiles[g] = 0;
        plan->group_shared[g] = 0;
    }
    for (int m = TCB_MODEL_MS; m <= TCB_MODEL_CRN; ++m) {
        const int g = model_slot[m];
        if (g < 0) continue;
        const size_t cb = model_consts_bytes(m);
        int32_t* idx = reinterpret_cast<int32_t*>(hp(L.g_idx[g]));
        int64_t* tp = reinterpret_cast<int64_t*>(hp(L.g_tiles[g]));
        char* cs = hp(L.g_consts[g]);
        char* ts = hp(L.g_tabs[g]);
        const size_t tb = model_tables_bytes(m);
        int count = 0;
        tp[0] = 0;
        bool shared = true;
        for (int j = 0; j < n; ++j) {
            if (sims[j].model != m) continue;
            idx[count] = j;
            int st = model_consts(m, sims[j].params, cs + cb * count);
            if (st) return st;
            if (count > 0 && memcmp(cs, cs + cb * count, cb) != 0) shared = false;
            st = model_tables_view(m, sims[j].tables, sims[j].params, ts + tb * count);
            if (st) return st;
            tp[count + 1] = tp[count] + sims[j].n_pad / kBatchTile;
            ++count;
        }
        BatchGroup& G = ws.groups[g];
        G.model = m;
        G.count = count;
        G.shared_consts = shared;
        G.idx = reinterpret_cast<const int32_t*>(dp(L.g_idx[g]));
        G.tile_prefix = reinterpret_cast<const int64_t*>(dp(L.g_tiles[g]));
        G.consts = dp(L.g_consts[g]);
        G.tables = dp(L.g_tabs[g]);
        plan->group_model[g] = m;
        plan->group_tiles[g] = tp[count];
        plan->group_shared[g] = shared;
        if (shared) memcpy(plan->group_consts[g], cs, cb);
    }
    memcpy(hp(L.ws), &ws, sizeof ws);
    TCB_CHECK_CUDA(cudaMemcpy(workspace, host.data(), L.total, cudaMemcpyHostToDevice));
    plan->workspace = workspace;
    plan->n_sims = n;
    plan->cg_blocks = nb;
    plan->cg_smem = (int32_t)smem;
    plan->total_slices = S;
    return TCB_OK;
}

extern "C" int tcb_batch_run(const tcb_batch_plan* plan, int64_t steps, void* stream) {
    if (!plan || !plan->workspace || steps < 0) return fail(TCB_EINVAL, "tcb_batch_run: bad arguments");
    cudaStream_t s = as_stream(stream);
    const BatchWS* W = static_cast<const BatchWS*>(plan->workspace);
    BatchWS hv;
    memset(&hv, 0, sizeof hv);
    for (int g = 0; g < kBatchGroups; ++g) hv.groups[g].model = plan->group_model[g];
    for (int64_t k = 0; k < steps; ++k) {
        for (int g = 0; g < plan->n_groups; ++g) {
            int st = launch_batch_ionic(W, hv, g, plan->group_tiles[g],
                                        plan->group_shared[g] ? plan->group_consts[g] : nullptr, s);
            if (st) return st;
        }
        int st = launch_batch_cg(W, plan->cg_blocks, (size_t)plan->cg_smem, s);
        if (st) return st;
    }
    return TCB_OK;
}

extern "C" int tcb_batch_check(const tcb_batch_plan* plan, void* stream) {
    if (!plan || !plan->workspace) return fail(TCB_EINVAL, "tcb_batch_check: null plan");
    cudaStream_t s = as_stream(stream);
    BatchWS ws;
    TCB_CHECK_CUDA(cudaMemcpyAsync(&ws, plan->workspace, sizeof ws, cudaMemcpyDeviceToHost, s));
    TCB_CHECK_CUDA(cudaStreamSynchronize(s));
    int32_t err = 0;
    TCB_CHECK_CUDA(cudaMemcpy(&err, ws.err, sizeof err, cudaMemcpyDeviceToHost));
    if (err == TCB_ETIMEOUT) return fail(TCB_ETIMEOUT, "a grid barrier of the batched CG kernel timed out");
    if (err != 0) return fail(err, "batch device error word set");
    return TCB_OK;
}
