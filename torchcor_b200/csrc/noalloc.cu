// tcb_mono_run_noalloc: the monodomain time loop with the CG kernel's scratch
// (float64 reduction partials and grid-barrier words) in a file-scope device
// array instead of caller-provided buffers.
//
// Some callers cannot allocate device memory where they call the solver: host
// applications that own the device memory pool and forbid allocations after
// start-up, and latency-critical callers for whom cudaMalloc's implicit device
// synchronisation is unacceptable.  For them this entry point needs no scratch
// arguments and allocates nothing (no cudaMalloc/cudaFree, no allocating library
// call); the caller still passes every input and output in the tcb_mono struct
// (m->scratch and m->barrier are ignored and may be NULL).
//
// The array holds at most kNoAllocMaxBlocks CG blocks' partials (64 KiB) plus
// the barrier words; a launch that would need more blocks is rejected with
// TCB_ERANGE.  Every GPU that loads the library keeps one copy until the
// process exits.  All calls share it: calls whose kernels overlap on the GPU
// (different streams, or different threads without ordering) race and must be
// serialised by the caller.  The barrier words are cleared on every call; the
// partials are always written before they are read.
#include <cuda_runtime.h>

#include <mutex>

#include "cg_common.cuh"
#include "mono.cuh"
#include "tcb_internal.h"

namespace tcb {
int validate_mono(const tcb_mono* m);
namespace {

// Both CG kernels place their second partial buffer at scratch + 2 * cgk::kMaxBlocks
// whatever the block count, so the array is sized from that constant.
constexpr int kNoAllocMaxBlocks = cgk::kMaxBlocks;
constexpr int kPartials = 4 * kNoAllocMaxBlocks;   // doubles: two parity buffers x 2 values x blocks
static_assert(kPartials == 4 * cgk::kMaxBlocks, "static scratch must hold what tcb_mono_scratch_doubles() asks for");
constexpr int kBarrierWords = 4;

// Device scratch.  In host code `g_scratch` is only a stand-in symbol: its
// device address must be obtained with cudaGetSymbolAddress (done once per
// device below) before a kernel may be given it.
static __device__ __align__(256) double g_scratch[kPartials + kBarrierWords / 2];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device; looked up on the first
// call per device (so that first call should come before any stream capture).
int scratch_address(void** out) {
    int dev = 0;
    TCB_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(TCB_ERANGE, "tcb_mono_run_noalloc: device ordinal beyond 63");
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_scratch)");
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return TCB_OK;
}

}  // namespace

int cg_blocks(const MonoDev& d);

}  // namespace tcb

using namespace tcb;

extern "C" int tcb_mono_run_noalloc(const tcb_mono* m, int64_t step_begin, int64_t step_end, void* stream) {
    if (!m) return fail(TCB_EINVAL, "tcb_mono_run_noalloc: null tcb_mono");
    tcb_mono local = *m;
    void* base = nullptr;
    int st = scratch_address(&base);
    if (st) return st;
    local.scratch = static_cast<double*>(base);
    local.barrier = reinterpret_cast<uint32_t*>(static_cast<double*>(base) + kPartials);
    // the struct is checked before anything touches the shared array
    st = validate_mono(&local);
    if (st) return st;
    if (step_begin < 1 || step_end > local.nt + 1 || step_begin > step_end)
        return fail(TCB_EINVAL, "tcb_mono_run_noalloc: step range outside [1, nt]");
    if (step_begin == step_end) return TCB_OK;
    MonoDev d = make_dev(&local);
    if (cg_blocks(d) > kNoAllocMaxBlocks)
        return fail(TCB_ERANGE, "tcb_mono_run_noalloc: the CG launch needs more blocks than the static scratch holds");
    cudaStream_t s = as_stream(stream);
    TCB_CHECK_CUDA(cudaMemsetAsync(local.barrier, 0, kBarrierWords * sizeof(uint32_t), s));
    return tcb_mono_run(&local, step_begin, step_end, stream);
}
