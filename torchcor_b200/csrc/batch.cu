// Host side of batched simulations: the workspace layout, the plan (CG grid,
// per-simulation CG views, ionic model groups) and the step loop.
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

constexpr int kDefaultVariant = 2;    // batched CG variant unless tuned

size_t up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// CG grid for S slices: at least kMinSlicesPerBlock slices a block, at most what is resident
int cg_grid(int64_t S, size_t smem, int variant, int flags) {
    const int cap = batch_cg_max_blocks(smem, variant, flags);
    if (cap < 1) return 0;
    const int64_t want = ceil_div(S, cgk::kMinSlicesPerBlock);
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, cap));
}

struct Layout {
    size_t ws, dev, cg, slices, parts, bar, err;
    size_t g_idx[kBatchGroups], g_tiles[kBatchGroups], g_consts[kBatchGroups], g_tabs[kBatchGroups];
    size_t total;
};

Layout layout(int n) {
    Layout L;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        size_t at = o;
        o = up(o + bytes);
        return at;
    };
    L.ws = take(sizeof(BatchWS));
    L.dev = take(sizeof(MonoDev) * n);
    L.cg = take(sizeof(CgView) * n);
    L.slices = take(sizeof(int32_t) * n);
    L.parts = take(sizeof(double) * 3 * (size_t)n * kBatchMaxBlocks);   // any grid of the plan
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
    return (int64_t)layout(n_sims).total;
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
    std::vector<CgView> views(n);
    std::vector<int32_t> slices(n);
    int64_t S = 0;
    for (int i = 0; i < n; ++i) {
        int st = validate_mono(&sims[i]);
        if (st) return st;
        if (sims[i].n_pad % kBatchTile != 0) return fail(TCB_EINVAL, "n_pad must be a multiple of 128");
        if (!sims[i].z || !sims[i].p2) return fail(TCB_EINVAL, "batched simulations need z and p2 buffers");
        if (sims[i].n_slices < 1 || sims[i].n_slices > INT32_MAX)
            return fail(TCB_EINVAL, "simulation slice count out of range");
        devs[i] = make_dev(&sims[i]);
        const MonoDev& d = devs[i];
        CgView& v = views[i];
        memset(&v, 0, sizeof v);
        v.n = d.n;
        v.n_pad = d.n_pad;
        v.slice_ptr = d.slice_ptr;
        v.col = d.col;
        v.dcol = d.dcol;
        v.mv = d.mv;
        v.kv = d.kv;
        v.av = d.av;
        v.dinv = d.dinv;
        v.x = d.x;
        v.bp = d.bp;
        v.r = d.r;
        v.p = d.p;
        v.ap = d.ap;
        v.z = d.z;
        v.p2 = d.p2;
        v.cm = d.cm;
        v.linear_guess = d.linear_guess;
        v.a_split = d.a_split;
        slices[i] = (int32_t)sims[i].n_slices;
        S += sims[i].n_slices;
    }
    // the combination of per-simulation code paths every simulation shares (or -1)
    int flags = -1;
    for (int i = 0; i < n; ++i) {
        const int f = (views[i].dcol ? 4 : 0) | (views[i].a_split ? 2 : 0) | (views[i].linear_guess ? 1 : 0);
        flags = i == 0 ? f : (f == flags ? flags : -1);
        if (flags < 0) break;
    }
    int variant = kDefaultVariant;
    size_t smem = batch_cg_smem_variant(n, variant);
    int nb = cg_grid(S, smem, variant, flags);
    if (nb < 1) {
        variant = 1;
        smem = batch_cg_smem_variant(n, variant);
        nb = cg_grid(S, smem, variant, flags);
    }
    if (nb < 1) return fail(TCB_ECUDA, "batched CG kernel cannot be resident");
    // bulk copies need 16-byte aligned sources (slices start at multiples of 32 entries)
    int stage_ok = batch_cg_stage_bytes(n) > 0;
    for (int i = 0; i < n && stage_ok; ++i) {
        const CgView& v = views[i];
        const void* ptrs[5] = {v.dcol ? (const void*)v.dcol : (const void*)v.col, v.mv, v.kv, v.av, nullptr};
        for (int k = 0; k < 4; ++k)
            if (reinterpret_cast<uintptr_t>(ptrs[k]) % 16 != 0) stage_ok = 0;
    }
    // the staged ionic form copies per-node rows (n_pad a multiple of 128 floats apart)
    int ionic_stage_ok = 1;
    for (int i = 0; i < n && ionic_stage_ok; ++i) {
        const MonoDev& d = devs[i];
        const void* ptrs[6] = {d.x, d.state, d.at, d.rt, d.stim_bits, d.bp};
        for (const void* q : ptrs)
            if (reinterpret_cast<uintptr_t>(q) % 16 != 0) ionic_stage_ok = 0;
    }
    Layout L = layout(n);
    if ((int64_t)L.total > bytes) return fail(TCB_ERANGE, "batch workspace too small");

    std::vector<char> host(L.total, 0);
    char* base = static_cast<char*>(workspace);
    auto hp = [&](size_t off) { return host.data() + off; };
    auto dp = [&](size_t off) { return base + off; };

    BatchWS ws;
    memset(&ws, 0, sizeof ws);
    ws.n = n;
    ws.total_slices = S;
    ws.dev = reinterpret_cast<const MonoDev*>(dp(L.dev));
    ws.cg = reinterpret_cast<const CgView*>(dp(L.cg));
    ws.slices = reinterpret_cast<const int32_t*>(dp(L.slices));
    ws.parts = reinterpret_cast<double*>(dp(L.parts));
    ws.bar = reinterpret_cast<uint32_t*>(dp(L.bar));
    ws.err = reinterpret_cast<int32_t*>(dp(L.err));
    ws.wait = wait_limit();
    memcpy(hp(L.dev), devs.data(), sizeof(MonoDev) * n);
    memcpy(hp(L.cg), views.data(), sizeof(CgView) * n);
    memcpy(hp(L.slices), slices.data(), sizeof(int32_t) * n);

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
    plan->cg_variant = variant;
    plan->cg_stage_bytes = 0;
    plan->cg_stage_ok = stage_ok;
    plan->cg_flags = flags;
    plan->cg_smem = (int32_t)smem;
    plan->total_slices = S;
    plan->ionic_tiles_per_block = 0;
    plan->ionic_blocks_per_sm = 0;
    plan->ionic_staged = 0;
    plan->ionic_stage_ok = ionic_stage_ok;
    return TCB_OK;
}

extern "C" int tcb_batch_set_cg(tcb_batch_plan* plan, int32_t variant) {
    if (!plan || !plan->workspace || variant < 1 || variant > 3)
        return fail(TCB_EINVAL, "tcb_batch_set_cg: bad arguments");
    if (variant == 3 && !plan->cg_stage_ok)
        return fail(TCB_ERANGE, "tcb_batch_set_cg: staged CG needs 16-byte aligned ELL arrays and shared memory");
    const size_t smem = batch_cg_smem_variant(plan->n_sims, variant);
    const int nb = cg_grid(plan->total_slices, smem, variant, plan->cg_flags);
    if (nb < 1) return fail(TCB_ERANGE, "tcb_batch_set_cg: that CG variant cannot be resident");
    plan->cg_variant = variant;
    plan->cg_stage_bytes = variant == 3 ? batch_cg_stage_bytes(plan->n_sims) : 0;
    plan->cg_smem = (int32_t)smem;
    plan->cg_blocks = nb;
    return TCB_OK;
}

extern "C" int tcb_batch_set_ionic(tcb_batch_plan* plan, int32_t tiles_per_block, int32_t blocks_per_sm,
                                   int32_t staged) {
    if (!plan || !plan->workspace || tiles_per_block < 0 || tiles_per_block > kBatchMaxTilesPerBlock)
        return fail(TCB_EINVAL, "tcb_batch_set_ionic: tiles per block outside 0..64");
    if (staged != 0 && staged != 1) return fail(TCB_EINVAL, "tcb_batch_set_ionic: staged not 0 or 1");
    if (!batch_ionic_blocks_ok(blocks_per_sm, staged))
        return fail(TCB_EINVAL, "tcb_batch_set_ionic: blocks per SM not 0, 4, 6, 8 or (unstaged) 12");
    if (staged && !plan->ionic_stage_ok)
        return fail(TCB_ERANGE, "tcb_batch_set_ionic: staged form needs 16-byte aligned per-node arrays");
    plan->ionic_tiles_per_block = tiles_per_block;
    plan->ionic_blocks_per_sm = blocks_per_sm;
    plan->ionic_staged = staged;
    return TCB_OK;
}

extern "C" int tcb_batch_run(const tcb_batch_plan* plan, int64_t steps, void* stream) {
    if (!plan || !plan->workspace || steps < 0) return fail(TCB_EINVAL, "tcb_batch_run: bad arguments");
    if (plan->cg_blocks < 1 || plan->cg_blocks > kBatchMaxBlocks || plan->cg_variant < 1 || plan->cg_variant > 3 ||
        (plan->cg_variant == 3 && (!plan->cg_stage_ok || plan->cg_stage_bytes < 2048)) || plan->cg_flags < -1 ||
        plan->cg_flags > 7)
        return fail(TCB_EINVAL, "tcb_batch_run: plan CG grid out of range");
    if (plan->ionic_tiles_per_block < 0 || plan->ionic_tiles_per_block > kBatchMaxTilesPerBlock ||
        plan->ionic_staged < 0 || plan->ionic_staged > 1 || (plan->ionic_staged && !plan->ionic_stage_ok) ||
        !batch_ionic_blocks_ok(plan->ionic_blocks_per_sm, plan->ionic_staged))
        return fail(TCB_EINVAL, "tcb_batch_run: plan ionic launch out of range");
    cudaStream_t s = as_stream(stream);
    const BatchWS* W = static_cast<const BatchWS*>(plan->workspace);
    for (int64_t k = 0; k < steps; ++k) {
        int st = launch_batch_ionic_all(W, plan->n_groups, plan->group_model, plan->group_tiles, plan->group_shared,
                                        plan->group_consts, plan->ionic_tiles_per_block,
                                        plan->ionic_blocks_per_sm, plan->ionic_staged, s);
        if (st) return st;
        st = launch_batch_cg(W, plan->cg_blocks, (size_t)plan->cg_smem, plan->cg_variant, plan->cg_stage_bytes,
                             plan->cg_flags, s);
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
    if (err == TCB_ETIMEOUT) return fail(TCB_ETIMEOUT, "a bounded wait (grid barrier or bulk-copy mbarrier) of the batched CG kernel timed out");
    if (err != 0) return fail(err, "batch device error word set");
    return TCB_OK;
}
