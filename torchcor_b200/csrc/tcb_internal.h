// Internal helpers shared by the libtcb200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "tcb200.h"

namespace tcb {

// thread-local last error message (tcb_last_error)
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

#define TCB_CHECK_CUDA(call)                                    \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return ::tcb::cuda_fail(e_, #call); \
    } while (0)

#define TCB_CHECK_LAUNCH(what)                                  \
    do {                                                        \
        cudaError_t e_ = cudaGetLastError();                    \
        if (e_ != cudaSuccess) return ::tcb::cuda_fail(e_, what); \
    } while (0)

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

int num_sms();

}  // namespace tcb
