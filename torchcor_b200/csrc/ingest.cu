// Mesh ingest on the device: openCARP text tables parsed on the GPU and the CSR
// pattern + scatter map built on the GPU (the role of torchcor/core/mesh.py:26-63
// and of the COO construction + coalesce in torchcor/core/assemble.py:217-248).
//
// Text: the file's bytes are copied to the device once; the newline positions
// are found with a three-pass count / scan / write; one thread per row parses
// its whitespace-separated fields.  Decimal -> double is correctly rounded, so
// it is the double np.loadtxt reads: with a significand m <= 2^53 and
// |exponent| <= 22 both m and 10^|e| are exact doubles and one IEEE multiply or
// divide rounds once (Clinger 1990); larger significands (up to 19 digits) use
// exact integer arithmetic -- m * 10^e for e <= 19 (128-bit product), and
// m / 10^k = (m / 5^k) * 2^-k for k <= 54 (long division, round-half-even on the
// quotient with the remainder as sticky bit).  Rows outside these paths (more than 19 significant digits, other
// exponents, malformed fields) are counted in `bad`; the caller then parses the
// file on the host instead.
//
// Pattern: every element contribution (a, b, e) becomes the key
// (col << 32 | order), order = (a*k + b)*E + e its position in the reference's
// COO list, bucketed by row, sorted per row (bitonic, one warp per row in
// shared memory) and compacted: the unique columns are the CSR columns and, for
// each slot, its contributions in COO order -- the host builder's output, bit
// for bit.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tcb_internal.h"

namespace tcb {
namespace {

constexpr int kThreads = 256;
constexpr int kBytesPerThread = 32;
constexpr int kRowCap = 1024;          // entries one row may have in the device pattern build
constexpr int kSortWarps = 4;
constexpr int kScanThreads = 1024;

// ---------------------------------------------------------------- newlines
__device__ __forceinline__ int count_nl(const char* t, int64_t b, int64_t e) {
    int c = 0;
    for (int64_t i = b; i < e; ++i) c += t[i] == '\n';
    return c;
}

__global__ void nl_count_kernel(const char* __restrict__ t, int64_t n, int64_t* __restrict__ block_cnt) {
    __shared__ int sh[kThreads];
    const int64_t b = ((int64_t)blockIdx.x * kThreads + threadIdx.x) * kBytesPerThread;
    const int64_t e = b + kBytesPerThread < n ? b + kBytesPerThread : n;
    sh[threadIdx.x] = b < n ? count_nl(t, b, e) : 0;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_cnt[blockIdx.x] = sh[0];
}

// exclusive scan of n values in place (one block, sequential over chunks)
__global__ void scan_kernel(int64_t* __restrict__ v, int64_t n, int64_t* __restrict__ total) {
    __shared__ int64_t sh[kScanThreads];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < n; base += kScanThreads) {
        const int64_t i = base + threadIdx.x;
        const int64_t x = i < n ? v[i] : 0;
        sh[threadIdx.x] = x;
        __syncthreads();
        for (int o = 1; o < kScanThreads; o <<= 1) {
            const int64_t y = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += y;
            __syncthreads();
        }
        if (i < n) v[i] = carry + sh[threadIdx.x] - x;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry += sh[kScanThreads - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void nl_write_kernel(const char* __restrict__ t, int64_t n, const int64_t* __restrict__ block_off,
                                int64_t* __restrict__ pos) {
    __shared__ int sh[kThreads];
    const int64_t b = ((int64_t)blockIdx.x * kThreads + threadIdx.x) * kBytesPerThread;
    const int64_t e = b + kBytesPerThread < n ? b + kBytesPerThread : n;
    const int c = b < n ? count_nl(t, b, e) : 0;
    sh[threadIdx.x] = c;
    __syncthreads();
    for (int o = 1; o < kThreads; o <<= 1) {
        const int y = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += y;
        __syncthreads();
    }
    int64_t w = block_off[blockIdx.x] + sh[threadIdx.x] - c;
    for (int64_t i = b; i < e; ++i)
        if (t[i] == '\n') pos[w++] = i;
}

// ---------------------------------------------------------------- fields
__device__ __forceinline__ bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

__device__ const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                      1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

// Correctly rounded double of an unsigned 128-bit value times 2^scale (round
// half to even; `sticky` marks a nonzero remainder below the value's last bit).
__device__ double round_u128(unsigned __int128 v, int scale, bool sticky) {
    const uint64_t hi = (uint64_t)(v >> 64), lo = (uint64_t)v;
    const int len = hi ? 128 - __clzll((long long)hi) : 64 - __clzll((long long)lo);
    if (len <= 53) return ldexp((double)(uint64_t)v, scale);   // exact (sticky cannot occur: no bits dropped)
    const int sh = len - 53;
    uint64_t m = (uint64_t)(v >> sh);
    const unsigned __int128 rb = v & ((((unsigned __int128)1) << sh) - 1);
    const unsigned __int128 half = ((unsigned __int128)1) << (sh - 1);
    const bool up = rb > half || (rb == half && (sticky || (m & 1)));
    if (up) ++m;
    return ldexp((double)m, scale + sh);   // m <= 2^53: exact conversion, exact scaling
}

__device__ const uint64_t kPow10u[20] = {1ull, 10ull, 100ull, 1000ull, 10000ull, 100000ull, 1000000ull,
                                         10000000ull, 100000000ull, 1000000000ull, 10000000000ull,
                                         100000000000ull, 1000000000000ull, 10000000000000ull,
                                         100000000000000ull, 1000000000000000ull, 10000000000000000ull,
                                         100000000000000000ull, 1000000000000000000ull,
                                         10000000000000000000ull};

// parse one decimal field [p, e); false if malformed or outside the exact range
// (more than 19 significant digits, or an exponent the paths below do not cover)
__device__ bool parse_double(const char* p, const char* e, double* out) {
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
    uint64_t m = 0;
    int digits = 0, exp10 = 0;
    bool any = false, dropped = false;
    for (; p < e && *p >= '0' && *p <= '9'; ++p) {
        any = true;
        if (m == 0 && *p == '0') continue;
        if (digits < 19) {
            m = m * 10 + (uint64_t)(*p - '0');
            ++digits;
        } else {
            ++exp10;
            dropped |= *p != '0';
        }
    }
    if (p < e && *p == '.') {
        ++p;
        for (; p < e && *p >= '0' && *p <= '9'; ++p) {
            any = true;
            if (m == 0 && *p == '0') {
                --exp10;
                continue;
            }
            if (digits < 19) {
                m = m * 10 + (uint64_t)(*p - '0');
                ++digits;
                --exp10;
            } else {
                dropped |= *p != '0';
            }
        }
    }
    if (!any) return false;
    if (p < e && (*p == 'e' || *p == 'E')) {
        ++p;
        bool eneg = false;
        if (p < e && (*p == '+' || *p == '-')) eneg = *p++ == '-';
        int x = 0;
        bool ed = false;
        for (; p < e && *p >= '0' && *p <= '9'; ++p) {
            ed = true;
            if (x < 100000) x = x * 10 + (*p - '0');
        }
        if (!ed) return false;
        exp10 += eneg ? -x : x;
    }
    if (p != e || dropped) return false;
    double v;
    if (m == 0) {
        v = 0.0;
    } else if (m <= (1ull << 53) && exp10 >= -22 && exp10 <= 22) {
        // m and 10^|e| are exact doubles: one correctly rounded operation
        v = exp10 < 0 ? __ddiv_rn((double)m, kPow10[-exp10]) : __dmul_rn((double)m, kPow10[exp10]);
    } else if (exp10 >= 0 && exp10 <= 19) {
        v = round_u128((unsigned __int128)m * kPow10u[exp10], 0, false);   // < 2^128, exact product
    } else if (exp10 < 0 && exp10 >= -54) {
        // m / 10^k = (m / 5^k) * 2^-k: long division of m * 2^s by 5^k (< 2^126), s chosen
        // for a quotient of 56..57 bits, then one rounding with the remainder as sticky bit
        const int k = -exp10;
        unsigned __int128 p5 = 1;
        for (int i = 0; i < k; ++i) p5 *= 5;
        const uint64_t phi = (uint64_t)(p5 >> 64), plo = (uint64_t)p5;
        const int plen = phi ? 128 - __clzll((long long)phi) : 64 - __clzll((long long)plo);
        const int mlen = 64 - __clzll((long long)m);
        int sh = 56 + plen - mlen;
        if (sh < 0) sh = 0;
        const int len = mlen + sh;   // bits of m * 2^s (<= 182)
        unsigned __int128 r = 0;
        uint64_t q = 0;
        for (int i = len - 1; i >= 0; --i) {
            r = (r << 1) | (i >= sh ? (m >> (i - sh)) & 1ull : 0ull);   // r < 5^k < 2^127 before the shift
            q <<= 1;
            if (r >= p5) {
                r -= p5;
                q |= 1ull;
            }
        }
        v = round_u128(q, -sh - k, r != 0);
    } else {
        return false;
    }
    *out = neg ? -v : v;
    return true;
}

__device__ bool parse_int(const char* p, const char* e, int64_t* out) {
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
    if (p >= e) return false;
    int64_t v = 0;
    for (; p < e; ++p) {
        if (*p < '0' || *p > '9' || v > (INT64_MAX - 9) / 10) return false;
        v = v * 10 + (*p - '0');
    }
    *out = neg ? -v : v;
    return true;
}

__global__ void parse_kernel(const char* __restrict__ t, int64_t n, const int64_t* __restrict__ nl, int64_t n_nl,
                             int64_t first_line, int64_t rows, int skip, int cols, int as_int, void* __restrict__ out,
                             int64_t* __restrict__ bad) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int64_t line = first_line + r;
    if (line > n_nl) {   // no such line
        atomicAdd((unsigned long long*)bad, 1ull);
        return;
    }
    const int64_t lb = line == 0 ? 0 : nl[line - 1] + 1;
    const int64_t le = line < n_nl ? nl[line] : n;
    const char* p = t + lb;
    const char* end = t + le;
    int field = 0;
    bool ok = true;
    while (ok) {
        while (p < end && is_space(*p)) ++p;
        if (p >= end) break;
        const char* q = p;
        while (q < end && !is_space(*q)) ++q;
        if (field >= skip) {
            const int c = field - skip;
            if (c >= cols) {
                ok = false;
                break;
            }
            if (as_int) ok = parse_int(p, q, static_cast<int64_t*>(out) + r * cols + c);
            else ok = parse_double(p, q, static_cast<double*>(out) + r * cols + c);
        }
        ++field;
        p = q;
    }
    if (!ok || field != skip + cols) atomicAdd((unsigned long long*)bad, 1ull);
}

// ---------------------------------------------------------------- pattern
__global__ void pattern_count_kernel(const int32_t* __restrict__ el, int64_t E, int k, int64_t N,
                                     int32_t* __restrict__ row_cnt, int32_t* __restrict__ err) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    for (int a = 0; a < k; ++a) {
        const int32_t v = el[e * k + a];
        if (v < 0 || v >= N) {
            atomicExch(err, 1);
            return;
        }
        atomicAdd(row_cnt + v, k);
    }
}

__global__ void pattern_fill_kernel(const int32_t* __restrict__ el, int64_t E, int k, const int64_t* __restrict__ row_off,
                                    int32_t* __restrict__ fill, uint64_t* __restrict__ keys) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    for (int a = 0; a < k; ++a) {
        const int32_t row = el[e * k + a];
        const int64_t base = row_off[row] + atomicAdd(fill + row, k);
        for (int b = 0; b < k; ++b) {
            const uint64_t order = (uint64_t)(a * k + b) * (uint64_t)E + (uint64_t)e;
            keys[base + b] = ((uint64_t)(uint32_t)el[e * k + b] << 32) | order;
        }
    }
}

// one warp per row: bitonic sort of the row's keys in shared memory, then the
// number of distinct columns
__global__ void pattern_sort_kernel(const int64_t* __restrict__ row_off, int64_t N, uint64_t* __restrict__ keys,
                                    int32_t* __restrict__ uniq, int32_t* __restrict__ err) {
    __shared__ uint64_t sh[kSortWarps][kRowCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * kSortWarps + warp;
    if (row >= N) return;
    const int64_t b = row_off[row];
    const int cnt = (int)(row_off[row + 1] - b);
    if (cnt > kRowCap) {
        if (lane == 0) atomicExch(err, 2);
        return;
    }
    int p2 = 1;
    while (p2 < cnt) p2 <<= 1;
    uint64_t* s = sh[warp];
    for (int i = lane; i < p2; i += 32) s[i] = i < cnt ? keys[b + i] : ~0ull;
    __syncwarp();
    for (int size = 2; size <= p2; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = lane; i < p2; i += 32) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const uint64_t x = s[i], y = s[j];
                    if ((x > y) == up) {
                        s[i] = y;
                        s[j] = x;
                    }
                }
            }
            __syncwarp();
        }
    int u = 0;
    for (int i = lane; i < cnt; i += 32) {
        keys[b + i] = s[i];
        u += (i == 0 || (s[i] >> 32) != (s[i - 1] >> 32));
    }
    for (int o = 16; o > 0; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
    if (lane == 0) uniq[row] = u;
}

// one warp per row: CSR columns, slot boundaries, contributions (flat element-
// matrix index e*k*k + a*k + b) and the diagonal slot
__global__ void pattern_emit_kernel(const int64_t* __restrict__ row_off, const int64_t* __restrict__ rowptr64,
                                    int64_t N, int64_t E, int k, const uint64_t* __restrict__ keys,
                                    int32_t* __restrict__ rowptr, int32_t* __restrict__ col,
                                    int32_t* __restrict__ slot_ptr, int32_t* __restrict__ slot_src,
                                    int32_t* __restrict__ diag) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * kSortWarps + warp;
    if (row >= N) return;
    const int64_t b = row_off[row];
    const int cnt = (int)(row_off[row + 1] - b);
    int64_t w = rowptr64[row];
    if (lane == 0) rowptr[row] = (int32_t)w;
    for (int i0 = 0; i0 < cnt; i0 += 32) {
        const int i = i0 + lane;
        bool first = false;
        uint64_t key = 0;
        if (i < cnt) {
            key = keys[b + i];
            const uint64_t order = key & 0xffffffffull;
            const int64_t ab = (int64_t)(order / (uint64_t)E), e = (int64_t)(order % (uint64_t)E);
            slot_src[b + i] = (int32_t)(e * k * k + ab);
            first = i == 0 || (keys[b + i - 1] >> 32) != (key >> 32);
        }
        const unsigned m = __ballot_sync(0xffffffffu, first);
        if (first) {
            const int64_t j = w + __popc(m & ((1u << lane) - 1));
            const int32_t c = (int32_t)(key >> 32);
            col[j] = c;
            slot_ptr[j] = (int32_t)(b + i);
            if (c == row) diag[row] = (int32_t)j;
        }
        w += __popc(m);
    }
}

__global__ void widen_kernel(const int32_t* __restrict__ c, int64_t* __restrict__ o, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = c[i];
}

__global__ void pattern_tail_kernel(const int64_t* rp64, const int64_t* ro, int64_t n, int32_t* rp, int32_t* sp) {
    rp[n] = (int32_t)rp64[n];
    sp[rp64[n]] = (int32_t)ro[n];
}

inline unsigned blocks(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int64_t tcb_text_scratch(int64_t n_bytes) {
    if (n_bytes < 0) return -1;
    return (int64_t)blocks(n_bytes, kThreads * kBytesPerThread) + 1;
}

extern "C" int tcb_text_newlines(const char* text, int64_t n_bytes, int64_t* scratch, int64_t* pos, int64_t cap,
                                 int64_t* count, void* stream) {
    if (!text || !scratch || !count || n_bytes <= 0 || (pos && cap < 0))
        return fail(TCB_EINVAL, "tcb_text_newlines: bad arguments");
    cudaStream_t s = as_stream(stream);
    const unsigned nb = blocks(n_bytes, kThreads * kBytesPerThread);
    nl_count_kernel<<<nb, kThreads, 0, s>>>(text, n_bytes, scratch);
    TCB_CHECK_LAUNCH("newline count kernel");
    scan_kernel<<<1, kScanThreads, 0, s>>>(scratch, nb, scratch + nb);
    TCB_CHECK_LAUNCH("scan kernel");
    int64_t total = 0;
    TCB_CHECK_CUDA(cudaMemcpyAsync(&total, scratch + nb, sizeof total, cudaMemcpyDeviceToHost, s));
    TCB_CHECK_CUDA(cudaStreamSynchronize(s));
    *count = total;
    if (!pos) return TCB_OK;
    if (total > cap) return fail(TCB_ERANGE, "tcb_text_newlines: more newlines than capacity");
    nl_write_kernel<<<nb, kThreads, 0, s>>>(text, n_bytes, scratch, pos);
    TCB_CHECK_LAUNCH("newline write kernel");
    return TCB_OK;
}

extern "C" int tcb_text_parse(const char* text, int64_t n_bytes, const int64_t* nl, int64_t n_nl, int64_t first_line,
                              int64_t rows, int32_t skip, int32_t cols, int32_t as_int, void* out, int64_t* bad,
                              void* stream) {
    if (!text || !out || !bad || n_bytes <= 0 || (n_nl > 0 && !nl) || first_line < 0 || rows < 0 || skip < 0 ||
        cols < 1)
        return fail(TCB_EINVAL, "tcb_text_parse: bad arguments");
    if (rows == 0) return TCB_OK;
    cudaStream_t s = as_stream(stream);
    parse_kernel<<<blocks(rows, kThreads), kThreads, 0, s>>>(text, n_bytes, nl, n_nl, first_line, rows, skip, cols,
                                                             as_int, out, bad);
    TCB_CHECK_LAUNCH("parse kernel");
    return TCB_OK;
}

extern "C" int tcb_pattern_device(const int32_t* elems, int64_t E, int32_t k, int64_t N, int64_t* work,
                                  uint64_t* keys, int32_t* iwork, int64_t* nnz, void* stream) {
    if (!elems || !work || !keys || !iwork || !nnz || E <= 0 || N <= 0 || (k != 3 && k != 4))
        return fail(TCB_EINVAL, "tcb_pattern_device: bad arguments");
    if ((int64_t)k * k * E >= INT32_MAX) return fail(TCB_ERANGE, "too many element contributions for int32");
    cudaStream_t s = as_stream(stream);
    // work: row_off [N+1] | rowptr64 [N+1];  iwork: row counts / fill [N] | uniq [N] | err [1]
    int64_t* row_off = work;
    int64_t* rowptr64 = work + N + 1;
    int32_t* cnt = iwork;
    int32_t* uniq = iwork + N;
    int32_t* err = iwork + 2 * N;
    TCB_CHECK_CUDA(cudaMemsetAsync(iwork, 0, sizeof(int32_t) * (2 * N + 1), s));
    pattern_count_kernel<<<blocks(E, kThreads), kThreads, 0, s>>>(elems, E, k, N, cnt, err);
    TCB_CHECK_LAUNCH("pattern count kernel");
    // row_off = exclusive scan of the counts (widened to int64 on the way)
    widen_kernel<<<blocks(N, kThreads), kThreads, 0, s>>>(cnt, row_off, N);
    TCB_CHECK_LAUNCH("widen kernel");
    scan_kernel<<<1, kScanThreads, 0, s>>>(row_off, N, row_off + N);
    TCB_CHECK_LAUNCH("scan kernel");
    TCB_CHECK_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * N, s));
    pattern_fill_kernel<<<blocks(E, kThreads), kThreads, 0, s>>>(elems, E, k, row_off, cnt, keys);
    TCB_CHECK_LAUNCH("pattern fill kernel");
    pattern_sort_kernel<<<blocks(N, kSortWarps), kSortWarps * 32, 0, s>>>(row_off, N, keys, uniq, err);
    TCB_CHECK_LAUNCH("pattern sort kernel");
    widen_kernel<<<blocks(N, kThreads), kThreads, 0, s>>>(uniq, rowptr64, N);
    TCB_CHECK_LAUNCH("widen kernel");
    scan_kernel<<<1, kScanThreads, 0, s>>>(rowptr64, N, rowptr64 + N);
    TCB_CHECK_LAUNCH("scan kernel");
    int32_t h_err = 0;
    TCB_CHECK_CUDA(cudaMemcpyAsync(&h_err, err, sizeof h_err, cudaMemcpyDeviceToHost, s));
    TCB_CHECK_CUDA(cudaMemcpyAsync(nnz, rowptr64 + N, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    TCB_CHECK_CUDA(cudaStreamSynchronize(s));
    if (h_err == 1) return fail(TCB_EINVAL, "element node index out of range");
    if (h_err == 2) return fail(TCB_ERANGE, "a node has more than 1024 element contributions (device pattern)");
    if (*nnz >= INT32_MAX) return fail(TCB_ERANGE, "nnz beyond int32");
    return TCB_OK;
}

extern "C" int tcb_pattern_device_emit(const int64_t* work, const uint64_t* keys, int64_t E, int32_t k, int64_t N,
                                       int32_t* rowptr, int32_t* col, int32_t* slot_ptr, int32_t* slot_src,
                                       int32_t* diag, void* stream) {
    if (!work || !keys || !rowptr || !col || !slot_ptr || !slot_src || !diag || E <= 0 || N <= 0 ||
        (k != 3 && k != 4))
        return fail(TCB_EINVAL, "tcb_pattern_device_emit: bad arguments");
    cudaStream_t s = as_stream(stream);
    const int64_t* row_off = work;
    const int64_t* rowptr64 = work + N + 1;
    pattern_emit_kernel<<<blocks(N, kSortWarps), kSortWarps * 32, 0, s>>>(row_off, rowptr64, N, E, k, keys, rowptr,
                                                                          col, slot_ptr, slot_src, diag);
    TCB_CHECK_LAUNCH("pattern emit kernel");
    pattern_tail_kernel<<<1, 1, 0, s>>>(rowptr64, row_off, N, rowptr, slot_ptr);
    TCB_CHECK_LAUNCH("pattern tail kernel");
    return TCB_OK;
}
