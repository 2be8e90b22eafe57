// CSR pattern of the assembled P1 operator and the deterministic scatter map
// (host code).  The reference builds the COO lists entry (i, j)-major over
// all elements (torchcor/core/assemble.py:225-231) and coalesces them
// (:248); the coalesced pattern is the sorted set of (row, col) pairs that
// share an element, and each slot's value is the sum of its contributions in
// COO-list order.  Here the same pattern and order come from a node ->
// element incidence list, built once per mesh, without sorting 16*E keys.
#include <algorithm>
#include <cstring>
#include <vector>

#include "tcb_internal.h"

namespace {

struct Incidence {
    std::vector<int64_t> ptr;   // n_nodes + 1
    std::vector<int32_t> elem;  // element of each incidence, ascending per node
    std::vector<int8_t> local;  // local vertex index of the node in that element
};

int build_incidence(const int32_t* elems, int64_t E, int32_t k, int64_t N, Incidence& inc) {
    inc.ptr.assign(N + 1, 0);
    for (int64_t e = 0; e < E; ++e)
        for (int a = 0; a < k; ++a) {
            int32_t v = elems[e * k + a];
            if (v < 0 || v >= N) return tcb::fail(TCB_EINVAL, "element node index out of range");
            inc.ptr[v + 1]++;
        }
    for (int64_t i = 0; i < N; ++i) inc.ptr[i + 1] += inc.ptr[i];
    inc.elem.resize(inc.ptr[N]);
    inc.local.resize(inc.ptr[N]);
    std::vector<int64_t> cur(inc.ptr.begin(), inc.ptr.end() - 1);
    for (int64_t e = 0; e < E; ++e)  // ascending e: each node's list is sorted by element
        for (int a = 0; a < k; ++a) {
            int32_t v = elems[e * k + a];
            int64_t p = cur[v]++;
            inc.elem[p] = (int32_t)e;
            inc.local[p] = (int8_t)a;
        }
    return TCB_OK;
}

struct Entry {
    int32_t col;
    int64_t order;  // position in the reference COO list: (a*k+b)*E + e
    int32_t src;    // flat index e*k*k + a*k + b
};

// The row's (col, order, src) entries, sorted by (col, order).
void row_entries(const int32_t* elems, int64_t E, int32_t k, const Incidence& inc, int64_t row,
                 std::vector<Entry>& out) {
    out.clear();
    for (int64_t q = inc.ptr[row]; q < inc.ptr[row + 1]; ++q) {
        int32_t e = inc.elem[q];
        int a = inc.local[q];
        for (int b = 0; b < k; ++b) {
            Entry en;
            en.col = elems[(int64_t)e * k + b];
            en.order = (int64_t)(a * k + b) * E + e;
            en.src = (int32_t)((int64_t)e * k * k + a * k + b);
            out.push_back(en);
        }
    }
    std::sort(out.begin(), out.end(), [](const Entry& x, const Entry& y) {
        return x.col != y.col ? x.col < y.col : x.order < y.order;
    });
}

}  // namespace

extern "C" int tcb_pattern_size(const int32_t* elems, int64_t E, int32_t k, int64_t N, int64_t* nnz) {
    if (!elems || !nnz || E <= 0 || N <= 0 || (k != 3 && k != 4))
        return tcb::fail(TCB_EINVAL, "tcb_pattern_size: bad arguments");
    if ((int64_t)k * k * E >= INT32_MAX) return tcb::fail(TCB_ERANGE, "too many element contributions for int32");
    Incidence inc;
    int st = build_incidence(elems, E, k, N, inc);
    if (st) return st;
    int64_t total = 0;
#pragma omp parallel reduction(+ : total)
    {
        std::vector<Entry> ent;
#pragma omp for schedule(dynamic, 4096)
        for (int64_t i = 0; i < N; ++i) {
            row_entries(elems, E, k, inc, i, ent);
            int64_t c = 0;
            for (size_t j = 0; j < ent.size(); ++j)
                if (j == 0 || ent[j].col != ent[j - 1].col) ++c;
            total += c;
        }
    }
    if (total >= INT32_MAX) return tcb::fail(TCB_ERANGE, "nnz beyond int32");
    *nnz = total;
    return TCB_OK;
}

extern "C" int tcb_pattern_build(const int32_t* elems, int64_t E, int32_t k, int64_t N, int32_t* rowptr,
                                 int32_t* col, int32_t* slot_ptr, int32_t* slot_src, int32_t* diag) {
    if (!elems || !rowptr || !col || !slot_ptr || !slot_src || !diag || E <= 0 || N <= 0 || (k != 3 && k != 4))
        return tcb::fail(TCB_EINVAL, "tcb_pattern_build: bad arguments");
    Incidence inc;
    int st = build_incidence(elems, E, k, N, inc);
    if (st) return st;
    // pass 1: row lengths
    std::vector<int32_t> len(N);
#pragma omp parallel
    {
        std::vector<Entry> ent;
#pragma omp for schedule(dynamic, 4096)
        for (int64_t i = 0; i < N; ++i) {
            row_entries(elems, E, k, inc, i, ent);
            int32_t c = 0;
            for (size_t j = 0; j < ent.size(); ++j)
                if (j == 0 || ent[j].col != ent[j - 1].col) ++c;
            len[i] = c;
        }
    }
    rowptr[0] = 0;
    for (int64_t i = 0; i < N; ++i) rowptr[i + 1] = rowptr[i] + len[i];
    // contributions of row i start at k * (number of incidences before i)
    int status = TCB_OK;
#pragma omp parallel
    {
        std::vector<Entry> ent;
#pragma omp for schedule(dynamic, 4096)
        for (int64_t i = 0; i < N; ++i) {
            row_entries(elems, E, k, inc, i, ent);
            int64_t slot = rowptr[i] - 1;
            int64_t cpos = (int64_t)k * inc.ptr[i];
            bool has_diag = false;
            for (size_t j = 0; j < ent.size(); ++j) {
                if (j == 0 || ent[j].col != ent[j - 1].col) {
                    ++slot;
                    col[slot] = ent[j].col;
                    slot_ptr[slot] = (int32_t)cpos;
                    if (ent[j].col == i) {
                        diag[i] = (int32_t)slot;
                        has_diag = true;
                    }
                }
                slot_src[cpos++] = ent[j].src;
            }
            if (!has_diag) {
#pragma omp critical
                status = tcb::fail(TCB_EINVAL, "node without an element (empty matrix row)");
            }
        }
    }
    slot_ptr[rowptr[N]] = (int32_t)((int64_t)k * inc.ptr[N]);
    return status;
}

extern "C" int tcb_sell_layout(const int32_t* rowptr, int64_t n_rows, int64_t* slice_ptr, int64_t* n_entries) {
    if (!rowptr || !slice_ptr || !n_entries || n_rows <= 0) return tcb::fail(TCB_EINVAL, "tcb_sell_layout: bad arguments");
    int64_t ns = tcb::ceil_div(n_rows, TCB_SLICE);
    slice_ptr[0] = 0;
    for (int64_t s = 0; s < ns; ++s) {
        int32_t w = 0;
        for (int64_t r = s * TCB_SLICE; r < std::min<int64_t>(n_rows, (s + 1) * TCB_SLICE); ++r)
            w = std::max(w, rowptr[r + 1] - rowptr[r]);
        slice_ptr[s + 1] = slice_ptr[s] + (int64_t)w * TCB_SLICE;
    }
    *n_entries = slice_ptr[ns];
    return TCB_OK;
}
