// B200 PDHG iteration engine, host side: the replacement for the reference's
// CudaBackend (src/cuda.cu:565-950) behind the IterationBackend seam
// (src/internal.hpp:102-134), exported through the C ABI of include/nk_pdhg.h.
// The kernels are in nk_device.cuh.
//
// Engine order: the rows of A and the rows of A^T (the columns of A) are sorted
// by length, longest first (stable), and stored as SELL-32 (nk_sell.cuh).  Every
// vector lives on the device in that order; vectors are permuted on their way in
// and out, so callers only ever see their own order.
#include "nk_common.cuh"
#include "nk_device.cuh"
#include "nk_panel.cuh"
#include "nk_host.hpp"
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <algorithm>
#include <array>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <queue>
#include <utility>
#include <set>
#include <atomic>
#include <thread>
#include <vector>

#ifndef NK_SPLIT
#define NK_SPLIT 128 // rows with more entries are split into virtual rows of this length
#endif
#ifndef NK_SPLIT_MAX
#define NK_SPLIT_MAX 256 // longest segment of a row that spans several chunks
#endif
constexpr int64_t kSplitMax = NK_SPLIT_MAX;

namespace nk {

thread_local char g_last_error[2048] = {};
void set_last_error(const char *what) { std::snprintf(g_last_error, sizeof(g_last_error), "%s", what); }

inline int grid_for(int64_t n, int cap = 148 * 8) {
    int64_t g = (n + kThreads - 1) / kThreads;
    return int(std::max<int64_t>(1, std::min<int64_t>(g, cap)));
}

// ------------------------------------------------------------------ matrices
// A matrix in SELL-32 on the device (see nk_sell.cuh).
struct SellMatrix {
    int64_t rows = 0, cols = 0, nnz = 0, nv = 0, nsv = 0, nsr = 0, padded = 0;
    bool wide = false; // int64 column indices
    int vbits = 64;    // 64 (double) or 32 (float) values
    DevBuf<int64_t> cptr;
    DevBuf<int32_t> len;
    DevBuf<int32_t> idx32;
    DevBuf<int64_t> idx64;
    DevBuf<double> val64;
    DevBuf<float> val32;
    DevBuf<int4> seg;
    DevBuf<double> slots;
    DevBuf<unsigned> counters;
    int ncounters = 0;              // rows split across chunks
    std::vector<int32_t> chunk_len; // host: padded length of each chunk
    DevBuf<int64_t> coff, clist;    // the fused kernels' per-CTA chunk lists
    int max_cta_items = 0;          // longest of those lists

    // The view the fused trial kernels use: with the per-CTA chunk lists
    // (built for their persistent grid).
    template <class V, class I> Sell<V, I> fused_view() const {
        Sell<V, I> s = view<V, I>();
        s.coff = coff.p;
        s.clist = clist.p;
        return s;
    }

    template <class V, class I> Sell<V, I> view() const {
        Sell<V, I> s;
        s.cptr = cptr.p;
        s.len = len.p;
        if constexpr (sizeof(I) == 8)
            s.idx = reinterpret_cast<const I *>(idx64.p);
        else
            s.idx = reinterpret_cast<const I *>(idx32.p);
        if constexpr (sizeof(V) == 8)
            s.val = reinterpret_cast<const V *>(val64.p);
        else
            s.val = reinterpret_cast<const V *>(val32.p);
        s.nv = nv;
        s.nsv = nsv;
        s.nsr = nsr;
        s.seg = seg.p;
        s.slots = slots.p;
        s.counters = counters.p;
        return s;
    }
    size_t device_bytes() const {
        return cptr.bytes() + len.bytes() + idx32.bytes() + idx64.bytes() + val64.bytes() +
               val32.bytes() + seg.bytes() + slots.bytes() + counters.bytes() + coff.bytes() +
               clist.bytes();
    }
};

// Sparse Q in CSR, engine order on both sides.
struct QMatrix {
    int64_t n = 0, nnz = 0;
    bool wide = false;
    int vbits = 64;
    DevBuf<int64_t> ptr, idx64;
    DevBuf<int32_t> idx32;
    DevBuf<double> val64;
    DevBuf<float> val32;
    template <class V, class I> QCsr<V, I> view() const {
        QCsr<V, I> q;
        q.ptr = ptr.p;
        if constexpr (sizeof(I) == 8)
            q.idx = reinterpret_cast<const I *>(idx64.p);
        else
            q.idx = reinterpret_cast<const I *>(idx32.p);
        if constexpr (sizeof(V) == 8)
            q.val = reinterpret_cast<const V *>(val64.p);
        else
            q.val = reinterpret_cast<const V *>(val32.p);
        return q;
    }
    size_t device_bytes() const {
        return ptr.bytes() + idx64.bytes() + idx32.bytes() + val64.bytes() + val32.bytes();
    }
};

// A's long rows by column panel (nk_panel.cuh), for the dual kernel's A dx.
struct PanelMatrix {
    int64_t rows = 0, cols = 0, width = 0, entries = 0, padded = 0, nunits = 0, slots = 0;
    int npanels = 0, vbits = 64, grid = 0;
    size_t smem = 0; // dynamic shared memory of panel_kernel: one dx slice
    DevBuf<int64_t> cptr, uoff, roff; // roff: each long row's slots [roff[i], roff[i+1])
    std::vector<int64_t> hroff;       // roff on the host
    DevBuf<int4> units; // pieces: {panel, first chunk, end chunk, unit}
    DevBuf<uint16_t> lidx;
    DevBuf<double> val64, partial;
    DevBuf<float> val32;
    DevBuf<unsigned> claim;
    template <class V> PanelView<V> view() const {
        PanelView<V> P;
        P.rows = rows;
        P.cols = cols;
        P.width = width;
        P.nunits = nunits;
        P.units = units.p;
        P.uoff = uoff.p;
        P.cptr = cptr.p;
        P.lidx = lidx.p;
        if constexpr (sizeof(V) == 8)
            P.val = reinterpret_cast<const V *>(val64.p);
        else
            P.val = reinterpret_cast<const V *>(val32.p);
        P.partial = partial.p;
        P.slots = slots;
        P.claim = claim.p;
        return P;
    }
    size_t device_bytes() const {
        return cptr.bytes() + uoff.bytes() + roff.bytes() + units.bytes() + lidx.bytes() +
               val64.bytes() + partial.bytes() + val32.bytes() + claim.bytes();
    }
};

// Stable order of items by decreasing length (counting sort): result[k] is the
// item placed k-th.
std::vector<int64_t> order_by_length_desc(const std::vector<int64_t> &len) {
    int64_t top = 0;
    for (int64_t l : len)
        top = std::max(top, l);
    std::vector<int64_t> count(size_t(top + 2), 0);
    for (int64_t l : len)
        ++count[size_t(l)];
    std::vector<int64_t> start(size_t(top + 2), 0); // first slot of each length, longest first
    int64_t at = 0;
    for (int64_t l = top; l >= 0; --l) {
        start[size_t(l)] = at;
        at += count[size_t(l)];
    }
    std::vector<int64_t> order(len.size());
    for (size_t i = 0; i < len.size(); ++i)
        order[size_t(start[size_t(len[i])]++)] = int64_t(i);
    return order;
}

struct SellPlan {
    std::vector<int64_t> cptr, src;
    std::vector<int32_t> len;
    std::vector<int4> seg;
    int64_t nv = 0, nsv = 0, nsr = 0;
    int ncounters = 0; // split rows spanning more than one chunk
};

// Virtual rows and chunks for an engine-order CSR (rows sorted longest first):
// rows longer than `split` become consecutive segments, placed first in whole
// chunks -- a row of up to 32*kSplitMax entries as at most 32 equal segments
// inside one chunk, a longer row as segments of kSplitMax entries -- and chunks
// of 32 virtual rows are padded to their longest.
SellPlan plan_sell(const std::vector<int64_t> &ptr, int64_t rows, int64_t split) {
    SellPlan P;
    while (P.nsr < rows && ptr[size_t(P.nsr + 1)] - ptr[size_t(P.nsr)] > split)
        ++P.nsr;
    auto pad_to_chunk = [&]() {
        while (P.len.size() % 32) {
            P.len.push_back(0);
            P.src.push_back(0);
            P.seg.push_back(make_int4(-1, 0, 0, -1));
        }
    };
    int ncounters = 0;
    for (int64_t r = 0; r < P.nsr; ++r) {
        int64_t L = ptr[size_t(r + 1)] - ptr[size_t(r)];
        // rows of up to 32 * kSplitMax entries stay inside one chunk: at most 32
        // segments of equal length (combined by their warp); longer rows span
        // chunks in segments of kSplitMax (combined through slots)
        bool local = L <= 32 * kSplitMax;
        int64_t nseg = local ? std::min<int64_t>(32, (L + split - 1) / split)
                             : (L + kSplitMax - 1) / kSplitMax;
        int64_t seglen = (L + nseg - 1) / nseg;
        if (local && int64_t(P.len.size() % 32) + nseg > 32)
            pad_to_chunk(); // never straddle two chunks
        int first = int(P.len.size());
        int counter = local ? -1 : ncounters++;
        for (int64_t s = 0; s < nseg; ++s) {
            P.len.push_back(int32_t(std::min<int64_t>(seglen, L - s * seglen)));
            P.src.push_back(ptr[size_t(r)] + s * seglen);
            P.seg.push_back(make_int4(int(r), first, int(nseg), counter));
        }
    }
    pad_to_chunk(); // split segments fill whole chunks
    P.nsv = int64_t(P.len.size());
    P.ncounters = ncounters;
    for (int64_t r = P.nsr; r < rows; ++r) {
        P.len.push_back(int32_t(ptr[size_t(r + 1)] - ptr[size_t(r)]));
        P.src.push_back(ptr[size_t(r)]);
    }
    P.nv = int64_t(P.len.size());
    int64_t nchunks = (P.nv + 31) / 32;
    P.cptr.assign(size_t(nchunks + 1), 0);
    for (int64_t c = 0; c < nchunks; ++c) {
        int32_t top = 0;
        for (int64_t v = 32 * c; v < std::min(P.nv, 32 * c + 32); ++v)
            top = std::max(top, P.len[size_t(v)]);
        P.cptr[size_t(c + 1)] = P.cptr[size_t(c)] + 32 * int64_t(top);
    }
    return P;
}

template <class T> void upload_vector(DevBuf<T> &d, const std::vector<T> &h, cudaStream_t s) {
    d.alloc(std::max<size_t>(1, h.size()));
    if (!h.empty())
        cuda_check(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s),
                   "upload");
}

// SELL-32 from an engine-order CSR (host ptr, device int64 indices / double values).
void build_sell(SellMatrix &M, int64_t rows, int64_t cols, const std::vector<int64_t> &ptr,
                const int64_t *cidx, const double *cval, bool wide, int vbits, cudaStream_t s) {
    M.rows = rows;
    M.cols = cols;
    M.nnz = ptr[size_t(rows)];
    M.wide = wide;
    M.vbits = vbits;
    SellPlan P = plan_sell(ptr, rows, NK_SPLIT);
    M.nv = P.nv;
    M.nsv = P.nsv;
    M.nsr = P.nsr;
    M.ncounters = P.ncounters;
    M.padded = P.cptr.back();
    M.chunk_len.resize(P.cptr.size() - 1);
    for (size_t c = 0; c + 1 < P.cptr.size(); ++c)
        M.chunk_len[c] = int32_t((P.cptr[c + 1] - P.cptr[c]) / 32);
    upload_vector(M.cptr, P.cptr, s);
    upload_vector(M.len, P.len, s);
    upload_vector(M.seg, P.seg, s);
    DevBuf<int64_t> src;
    upload_vector(src, P.src, s);
    M.slots.alloc(size_t(std::max<int64_t>(1, P.nsv)));
    M.counters.alloc(size_t(std::max(1, P.ncounters)));
    cuda_check(cudaMemsetAsync(M.counters.p, 0, M.counters.bytes(), s), "split counters");
    size_t total = size_t(std::max<int64_t>(1, M.padded));
    if (wide) {
        M.idx64.alloc(total);
        cuda_check(cudaMemsetAsync(M.idx64.p, 0, M.idx64.bytes(), s), "sell idx");
    } else {
        M.idx32.alloc(total);
        cuda_check(cudaMemsetAsync(M.idx32.p, 0, M.idx32.bytes(), s), "sell idx");
    }
    if (vbits == 64) {
        M.val64.alloc(total);
        cuda_check(cudaMemsetAsync(M.val64.p, 0, M.val64.bytes(), s), "sell val");
    } else {
        M.val32.alloc(total);
        cuda_check(cudaMemsetAsync(M.val32.p, 0, M.val32.bytes(), s), "sell val");
    }
    if (M.nv) {
        int g = grid_for(M.nv, 148 * 32);
        if (wide && vbits == 64)
            fill_sell<double, int64_t><<<g, kThreads, 0, s>>>(M.nv, src.p, M.len.p, M.cptr.p, cidx,
                                                               cval, M.idx64.p, M.val64.p);
        else if (wide)
            fill_sell<float, int64_t><<<g, kThreads, 0, s>>>(M.nv, src.p, M.len.p, M.cptr.p, cidx,
                                                              cval, M.idx64.p, M.val32.p);
        else if (vbits == 64)
            fill_sell<double, int32_t><<<g, kThreads, 0, s>>>(M.nv, src.p, M.len.p, M.cptr.p, cidx,
                                                               cval, M.idx32.p, M.val64.p);
        else
            fill_sell<float, int32_t><<<g, kThreads, 0, s>>>(M.nv, src.p, M.len.p, M.cptr.p, cidx,
                                                              cval, M.idx32.p, M.val32.p);
        cuda_check(cudaGetLastError(), "sell fill");
    }
    cuda_check(cudaStreamSynchronize(s), "sell build");
}

// Build the explicit transpose on the device: a stable radix sort of the column
// indices carries every entry to its row of A^T in increasing row order, the
// order Sparse::transpose produces (src/model.cpp:39-58).
void device_transpose(int64_t rows, int64_t cols, int64_t nnz, const int64_t *dptr,
                      const int64_t *didx, const double *dval, DevBuf<int64_t> &tptr,
                      DevBuf<int64_t> &tidx, DevBuf<double> &tval, cudaStream_t stream) {
    tptr.alloc(size_t(cols + 1));
    tidx.alloc(std::max<int64_t>(1, nnz));
    tval.alloc(std::max<int64_t>(1, nnz));
    DevBuf<int64_t> counts(static_cast<size_t>(cols + 1));
    cuda_check(cudaMemsetAsync(counts.p, 0, size_t(cols + 1) * 8, stream), "counts");
    if (nnz) {
        int g = grid_for(nnz, 148 * 32);
        count_cols<<<g, kThreads, 0, stream>>>(nnz, didx, counts.p);
        DevBuf<int32_t> rowid(static_cast<size_t>(nnz));
        expand_rows<<<grid_for(rows, 148 * 32), kThreads, 0, stream>>>(rows, dptr, rowid.p);
        DevBuf<int64_t> keys_out(static_cast<size_t>(nnz)), perm_in(static_cast<size_t>(nnz)),
            perm_out(static_cast<size_t>(nnz));
        iota64<<<g, kThreads, 0, stream>>>(nnz, perm_in.p);
        int end_bit = 1;
        while (end_bit < 63 && (int64_t(1) << end_bit) < cols)
            ++end_bit;
        size_t temp = 0;
        cuda_check(cub::DeviceRadixSort::SortPairs(nullptr, temp, didx, keys_out.p, perm_in.p,
                                                   perm_out.p, nnz, 0, end_bit, stream),
                   "transpose sort size");
        DevBuf<char> work(temp);
        cuda_check(cub::DeviceRadixSort::SortPairs(work.p, temp, didx, keys_out.p, perm_in.p,
                                                   perm_out.p, nnz, 0, end_bit, stream),
                   "transpose sort");
        gather_transpose<<<g, kThreads, 0, stream>>>(nnz, perm_out.p, rowid.p, dval, tidx.p,
                                                    tval.p);
        cuda_check(cudaGetLastError(), "transpose gather");
        size_t t2 = 0;
        cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, t2, counts.p, tptr.p, cols + 1, stream),
                   "transpose scan size");
        DevBuf<char> w2(t2);
        cuda_check(cub::DeviceScan::ExclusiveSum(w2.p, t2, counts.p, tptr.p, cols + 1, stream),
                   "transpose scan");
        cuda_check(cudaStreamSynchronize(stream), "transpose");
    } else {
        cuda_check(cudaMemsetAsync(tptr.p, 0, size_t(cols + 1) * 8, stream), "empty transpose");
        cuda_check(cudaStreamSynchronize(stream), "transpose");
    }
}

// Engine-order CSR of a device CSR: rows in `perm` order, column indices through
// `inv`.  Returns the new host ptr; the device arrays land in (idx, val).
std::vector<int64_t> permute_device_csr(int64_t rows, const std::vector<int64_t> &src_ptr_h,
                                        const int64_t *src_ptr, const int64_t *src_idx,
                                        const double *src_val, const std::vector<int64_t> &perm,
                                        const int64_t *dperm, const int64_t *dinv,
                                        DevBuf<int64_t> &idx, DevBuf<double> &val,
                                        cudaStream_t s) {
    std::vector<int64_t> ptr(static_cast<size_t>(rows + 1), 0);
    for (int64_t i = 0; i < rows; ++i) {
        int64_t o = perm[size_t(i)];
        ptr[size_t(i + 1)] = ptr[size_t(i)] + (src_ptr_h[size_t(o + 1)] - src_ptr_h[size_t(o)]);
    }
    int64_t nnz = ptr[size_t(rows)];
    DevBuf<int64_t> dptr;
    upload_vector(dptr, ptr, s);
    idx.alloc(std::max<int64_t>(1, nnz));
    val.alloc(std::max<int64_t>(1, nnz));
    if (rows && nnz) {
        permute_csr<<<grid_for(rows * 32, 148 * 32), kThreads, 0, s>>>(
            rows, dperm, dinv, src_ptr, src_idx, src_val, dptr.p, idx.p, val.p);
        cuda_check(cudaGetLastError(), "csr permutation");
    }
    cuda_check(cudaStreamSynchronize(s), "csr permutation");
    return ptr;
}

void validate_csr(const nk_csr *M, int64_t rows, int64_t cols, const char *what) {
    if (!M || M->rows != rows || M->cols != cols || !M->ptr)
        throw Error(NK_ERR_INVALID, std::string("inconsistent ") + what + " dimensions");
    if (M->ptr[0] != 0)
        throw Error(NK_ERR_INVALID, std::string("invalid ") + what + " CSR storage");
    for (int64_t i = 0; i < rows; ++i)
        if (M->ptr[i + 1] < M->ptr[i])
            throw Error(NK_ERR_INVALID, std::string("invalid ") + what + " CSR offsets");
    if (M->ptr[rows] > 0 && (!M->index || !M->value))
        throw Error(NK_ERR_INVALID, std::string("missing ") + what + " entries");
}

// Upload a host CSR as int64/double device arrays and check its indices (and,
// for FP32 storage, that every coefficient survives the conversion).
void upload_raw(const nk_csr *H, int vbits, cudaStream_t stream, DevBuf<int64_t> &p,
                DevBuf<int64_t> &ix, DevBuf<double> &vv) {
    int64_t nnz = H->ptr[H->rows];
    p.alloc(static_cast<size_t>(H->rows + 1));
    ix.alloc(std::max<int64_t>(1, nnz));
    vv.alloc(std::max<int64_t>(1, nnz));
    cuda_check(cudaMemcpyAsync(p.p, H->ptr, size_t(H->rows + 1) * 8, cudaMemcpyHostToDevice, stream),
               "ptr upload");
    if (nnz) {
        cuda_check(cudaMemcpyAsync(ix.p, H->index, size_t(nnz) * 8, cudaMemcpyHostToDevice, stream),
                   "index upload");
        cuda_check(cudaMemcpyAsync(vv.p, H->value, size_t(nnz) * 8, cudaMemcpyHostToDevice, stream),
                   "value upload");
        DevBuf<int> bad(1);
        cuda_check(cudaMemsetAsync(bad.p, 0, sizeof(int), stream), "flag");
        check_indices<<<grid_for(nnz, 148 * 32), kThreads, 0, stream>>>(nnz, ix.p, vv.p, H->cols,
                                                                        bad.p);
        if (vbits == 32)
            fp32_flags<<<grid_for(nnz, 148 * 32), kThreads, 0, stream>>>(nnz, vv.p, bad.p);
        int hb = 0;
        cuda_check(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, stream), "flag");
        cuda_check(cudaStreamSynchronize(stream), "index check");
        if (hb)
            throw Error(NK_ERR_INVALID,
                        vbits == 32 ? "invalid coefficient/index, or FP32 matrix conversion would "
                                      "overflow or erase a coefficient; use fp64"
                                    : "Invalid matrix coefficient/index");
    }
    cuda_check(cudaStreamSynchronize(stream), "matrix upload");
}

// The primal kernel instance for a model: sparse Q or not, split rows of A^T
// or not (each leaves unused paths out of the build).
template <class V, class I> using PrimalFn = void (*)(Sell<V, I>, QCsr<V, I>, Vecs);
template <class Acc, class V, class I> PrimalFn<V, I> primal_kernel_for(bool sparse_q, bool split) {
    constexpr bool F = sizeof(Acc) == 4;
    if (sparse_q)
        return split ? primal_kernel<Acc, V, I, true, F, true>
                     : primal_kernel<Acc, V, I, true, F, false>;
    return split ? primal_kernel<Acc, V, I, false, F, true> : primal_kernel<Acc, V, I, false, F, false>;
}

// ------------------------------------------------------------------ engine
struct Engine {
    int64_t n = 0, m = 0;
    bool adaptive = false, halpern = false, residual_restarts = false, graphs = false;
    bool sparse_q = false, wide = false;
    bool diag_q = false; // some q_j != 0 (an LP has none: the primal kernel skips q)
    int precision = NK_PRECISION_FP64;
    double reflection = 0, a_norm = 0, q_norm = 0;
    cudaStream_t stream = nullptr;
    SellMatrix A, At;
    QMatrix Q;
    PanelMatrix pan; // A's long rows by column panel (the dual SpMV), when panels
    bool panels = false;
    DevBuf<double> c, q, lb, ub, rl, ru, x[2], y[2], ax[2], xa, ya, dx, anchor_x, anchor_y,
        anchor_ax, part_p, part_d, mon_ax, mon_aty, mon_qx, mon_part, mon_out;
    DevBuf<float> dx32, y32[2];
    DevBuf<Control> ctl;
    DevBuf<unsigned> mon_arrive;
    Control *host_ctl = nullptr; // pinned mirror
    int grid_p = 1, grid_d = 1, grid_s = 148;
    // rows split across chunks: each one's step-rule contributions (A^T: dx^2;
    // A: dy^2, dy * delta)
    DevBuf<double> split_p, split_d;
    int64_t accepted = 0, rejected = 0, trials = 0;
    int empty_chunks = 0;
    bool request_restart = false;
    cudaGraphExec_t graph_exec[8] = {};
    double cscale = 1;
    // engine order: engine column j is the caller's column col_perm[j], engine
    // row i the caller's row row_perm[i]
    DevBuf<int64_t> col_perm, row_perm;
    DevBuf<double> scratch_n, scratch_m;
    // per-kernel timing hooks: when set, events are recorded around the primal
    // and dual launches of each trial (profiling mode, no graphs)
    cudaEvent_t ev[4] = {};
    bool ev_in_graph = false; // profile(): the events are recorded inside a captured trial

    ~Engine() {
        if (stream)
            cudaStreamSynchronize(stream);
        for (auto &g : graph_exec)
            if (g)
                cudaGraphExecDestroy(g);
        if (host_ctl)
            cudaFreeHost(host_ctl);
        if (stream)
            cudaStreamDestroy(stream);
    }

    Vecs vecs() {
        Vecs v{};
        v.c = c.p;
        v.q = diag_q ? q.p : nullptr;
        v.lb = lb.p;
        v.ub = ub.p;
        v.rl = rl.p;
        v.ru = ru.p;
        v.x0 = x[0].p;
        v.x1 = x[1].p;
        v.y0 = y[0].p;
        v.y1 = y[1].p;
        v.ax0 = ax[0].p;
        v.ax1 = ax[1].p;
        v.xa = xa.p;
        v.ya = ya.p;
        v.dx = dx.p;
        v.dx32 = dx32.p;
        v.y32_0 = y32[0].p;
        v.y32_1 = y32[1].p;
        v.anchor_x = anchor_x.p;
        v.anchor_y = anchor_y.p;
        v.anchor_ax = anchor_ax.p;
        v.part_p = part_p.p;
        v.part_d = part_d.p;
        v.ctl = ctl.p;
        v.grid_p = grid_p;
        v.reflection = reflection;
        v.split_p = split_p.p;
        v.split_d = split_d.p;
        v.nsplit_p = At.ncounters;
        v.nsplit_d = panels ? 0 : A.ncounters; // with panels A's long rows never split
        v.panel_partial = pan.partial.p;
        v.panel_roff = pan.roff.p;
        v.panel_rows = panels ? pan.rows : 0;
        v.npanels = panels ? pan.npanels : 0;
        return v;
    }

    // -------------------------------------------------------------- launches
    // profiling event i after the preceding launch (inside a capture, as an
    // external node, so that replaying the graph records it)
    void mark(int i) {
        cuda_check(cudaEventRecordWithFlags(ev[i], stream,
                                            ev_in_graph ? cudaEventRecordExternal
                                                        : cudaEventRecordDefault),
                   "profile event");
    }
    template <class Acc, class V, class I> void launch_trial_t() {
        Vecs v = vecs();
        constexpr bool F32 = sizeof(Acc) == 4;
        auto at = At.fused_view<V, I>();
        auto a = A.fused_view<V, I>();
        auto qm = Q.view<V, I>();
        if (ev[0])
            mark(0);
        primal_kernel_for<Acc, V, I>(sparse_q, At.nsv > 0)<<<grid_p, kFusedThreads, smem_p(),
                                                              stream>>>(at, qm, v);
        if (ev[1])
            mark(1);
        if (panels) {
            using X = typename std::conditional<F32, float, double>::type;
            const X *dxp;
            if constexpr (F32)
                dxp = dx32.p;
            else
                dxp = dx.p;
            panel_kernel<Acc, V, X><<<pan.grid, kPanelThreads, pan.smem, stream>>>(
                pan.view<V>(), dxp, ctl.p);
            if (ev[3])
                mark(3);
            dual_kernel<Acc, V, I, F32, false, true><<<grid_d, kFusedThreads, smem_d(), stream>>>(a,
                                                                                                v);
        } else if (A.nsv > 0)
            dual_kernel<Acc, V, I, F32, true><<<grid_d, kFusedThreads, smem_d(), stream>>>(a, v);
        else
            dual_kernel<Acc, V, I, F32, false><<<grid_d, kFusedThreads, smem_d(), stream>>>(a, v);
        if (ev[2])
            mark(2);
        if (halpern)
            halpern_commit<<<grid_for(std::max(n, m)), kThreads, 0, stream>>>(n, m, v, F32);
    }
    // dynamic shared memory of the fused kernels: one slot per chunk of a CTA
    // (the primal kernel's dx^2, the dual kernel's dy^2 and dy * delta)
    size_t smem_p() const { return size_t(std::max(1, At.max_cta_items)) * sizeof(double); }
    size_t smem_d() const { return size_t(std::max(1, A.max_cta_items)) * 2 * sizeof(double); }

    void launch_trial() {
        if (precision == NK_PRECISION_FP64) {
            if (wide)
                launch_trial_t<double, double, int64_t>();
            else
                launch_trial_t<double, double, int32_t>();
        } else if (precision == NK_PRECISION_MIXED) {
            if (wide)
                launch_trial_t<double, float, int64_t>();
            else
                launch_trial_t<double, float, int32_t>();
        } else {
            if (wide)
                launch_trial_t<float, float, int64_t>();
            else
                launch_trial_t<float, float, int32_t>();
        }
    }

    template <class V, class I>
    void spmv_t(const SellMatrix &M, const double *xin, double *out) {
        if (M.nv == 0)
            return;
        int g = int(std::max<int64_t>(1, std::min<int64_t>((M.nv / 32 + kWarps) / kWarps, grid_s)));
        spmv_kernel<V, I><<<g, kThreads, 0, stream>>>(M.view<V, I>(), xin, out);
    }
    // out = M * xin with FP64 accumulation (activity rebasing, the monitor).
    void spmv(const SellMatrix &M, const double *xin, double *out) {
        if (M.vbits == 64) {
            if (M.wide)
                spmv_t<double, int64_t>(M, xin, out);
            else
                spmv_t<double, int32_t>(M, xin, out);
        } else {
            if (M.wide)
                spmv_t<float, int64_t>(M, xin, out);
            else
                spmv_t<float, int32_t>(M, xin, out);
        }
        cuda_check(cudaGetLastError(), "spmv launch");
    }
    void q_spmv(const double *xin, double *out) {
        int g = grid_for(n);
        if (Q.vbits == 64) {
            if (Q.wide)
                q_spmv_kernel<double, int64_t><<<g, kThreads, 0, stream>>>(n, Q.view<double, int64_t>(), xin, out);
            else
                q_spmv_kernel<double, int32_t><<<g, kThreads, 0, stream>>>(n, Q.view<double, int32_t>(), xin, out);
        } else {
            if (Q.wide)
                q_spmv_kernel<float, int64_t><<<g, kThreads, 0, stream>>>(n, Q.view<float, int64_t>(), xin, out);
            else
                q_spmv_kernel<float, int32_t><<<g, kThreads, 0, stream>>>(n, Q.view<float, int32_t>(), xin, out);
        }
        cuda_check(cudaGetLastError(), "Q spmv launch");
    }

    void sync_ctl() {
        cuda_check(cudaMemcpyAsync(host_ctl, ctl.p, sizeof(Control), cudaMemcpyDeviceToHost,
                                   stream),
                   "control download");
        cuda_check(cudaStreamSynchronize(stream), "control sync");
    }
    void push_ctl() {
        cuda_check(cudaMemcpyAsync(ctl.p, host_ctl, sizeof(Control), cudaMemcpyHostToDevice,
                                   stream),
                   "control upload");
    }
    void flush() {
        Vecs v = vecs();
        flush_average<<<grid_for(std::max(n, m)), kThreads, 0, stream>>>(n, m, v);
        clear_pending<<<1, 1, 0, stream>>>(ctl.p);
        cuda_check(cudaGetLastError(), "flush");
    }
    // Recompute the resident activity A*x of the current iterate.
    void refresh_activity(int cur) {
        if (m)
            spmv(A, x[cur].p, ax[cur].p);
    }
    void refresh_y32(int cur) {
        if (precision == NK_PRECISION_FP32 && m)
            to_float<<<grid_for(m), kThreads, 0, stream>>>(m, y[cur].p, y32[cur].p);
    }

    // Graph k holds 2^k trials; kernels read tau, sigma and the iterate index
    // from device memory, so graphs never need recapturing.
    cudaGraphExec_t graph_for(int k) {
        if (!graph_exec[k]) {
            cudaGraph_t g = nullptr;
            cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal),
                       "graph capture");
            try {
                for (int t = 0; t < (1 << k); ++t)
                    launch_trial();
            } catch (...) {
                cudaStreamEndCapture(stream, &g);
                if (g)
                    cudaGraphDestroy(g);
                throw;
            }
            cuda_check(cudaStreamEndCapture(stream, &g), "graph end capture");
            cudaError_t e = cudaGraphInstantiate(&graph_exec[k], g, 0);
            cudaGraphDestroy(g);
            cuda_check(e, "graph instantiate");
        }
        return graph_exec[k];
    }

    int advance(int count, double tau, double sigma) {
        if (count < 0)
            throw Error(NK_ERR_INVALID, "negative trial count");
        if (sparse_q) { // QP step safety, src/cpu.cpp:97-102 / src/cuda.cu:817-822
            double safety = std::sqrt(tau * sigma) * a_norm + tau * q_norm;
            double scale = safety > 0 ? std::min(1., .9 / safety) : 1.;
            tau *= scale;
            sigma *= scale;
        }
        sync_ctl();
        double before_rej = host_ctl->rejected;
        if (host_ctl->tau != tau || host_ctl->sigma != sigma) {
            host_ctl->tau = tau;
            host_ctl->sigma = sigma;
            push_ctl();
        }
        int left = count;
        if (graphs) {
            for (int k = 7; k >= 0 && left > 0; --k)
                while (left >= (1 << k)) {
                    cuda_check(cudaGraphLaunch(graph_for(k), stream), "graph launch");
                    left -= 1 << k;
                }
        } else {
            for (; left > 0; --left)
                launch_trial();
        }
        cuda_check(cudaGetLastError(), "trial launch");
        trials += count;
        sync_ctl();
        int64_t now = int64_t(host_ctl->accepted);
        int progress = int(now - accepted);
        accepted = now;
        rejected = int64_t(host_ctl->rejected);
        request_restart = host_ctl->restart != 0;
        empty_chunks = progress ? 0 : empty_chunks + 1;
        bool nonfinite_fixed = !adaptive && host_ctl->rejected != before_rej;
        if (empty_chunks >= 4 || nonfinite_fixed)
            throw Error(NK_ERR_STALLED,
                        "CUDA PDHG backtracking stalled or produced nonfinite steps");
        return progress;
    }

    void download(double *dst, const double *src, int64_t count) {
        if (count && dst)
            cuda_check(cudaMemcpyAsync(dst, src, size_t(count) * 8, cudaMemcpyDeviceToHost, stream),
                       "download");
    }
    void upload(double *dst, const double *src, int64_t count) {
        if (count)
            cuda_check(cudaMemcpyAsync(dst, src, size_t(count) * 8, cudaMemcpyHostToDevice, stream),
                       "upload");
    }
    // Vector transfers in the caller's order (columns: col_perm, rows: row_perm).
    // With sync = false the transfer is only enqueued: the caller synchronises
    // the stream before it reads (download) or reuses (upload) the host buffer.
    // Transfers through the same scratch stay ordered by the stream.
    void download_perm(double *host, const double *dev, int64_t len, const DevBuf<int64_t> &perm,
                       DevBuf<double> &scratch, bool sync = true) {
        if (!len || !host)
            return;
        scatter_vec<<<grid_for(len), kThreads, 0, stream>>>(len, perm.p, dev, scratch.p);
        cuda_check(cudaGetLastError(), "scatter");
        download(host, scratch.p, len);
        if (sync)
            cuda_check(cudaStreamSynchronize(stream), "download");
    }
    void upload_perm(double *dev, const double *host, int64_t len, const DevBuf<int64_t> &perm,
                     DevBuf<double> &scratch, bool sync = true) {
        if (!len)
            return;
        upload(scratch.p, host, len);
        gather_vec<<<grid_for(len), kThreads, 0, stream>>>(len, perm.p, scratch.p, dev);
        cuda_check(cudaGetLastError(), "gather");
        if (sync)
            cuda_check(cudaStreamSynchronize(stream), "upload");
    }
    void download_x(double *h, const double *d) { download_perm(h, d, n, col_perm, scratch_n); }
    void download_y(double *h, const double *d) { download_perm(h, d, m, row_perm, scratch_m); }
    void upload_x(double *d, const double *h) { upload_perm(d, h, n, col_perm, scratch_n); }
    void upload_y(double *d, const double *h) { upload_perm(d, h, m, row_perm, scratch_m); }

    void candidates(double *hx, double *hy, double *hxa, double *hya) {
        flush();
        sync_ctl();
        int cur = host_ctl->cur;
        // four stream-ordered transfers, one synchronisation
        download_perm(hx, x[cur].p, n, col_perm, scratch_n, false);
        download_perm(hy, y[cur].p, m, row_perm, scratch_m, false);
        download_perm(hxa, xa.p, n, col_perm, scratch_n, false);
        download_perm(hya, ya.p, m, row_perm, scratch_m, false);
        refresh_activity(cur); // rebase A*x like the reference (src/cuda.cu:874-891)
        cuda_check(cudaStreamSynchronize(stream), "candidates");
    }

    void zero_average() {
        if (n)
            cuda_check(cudaMemsetAsync(xa.p, 0, size_t(n) * 8, stream), "zero xa");
        if (m)
            cuda_check(cudaMemsetAsync(ya.p, 0, size_t(m) * 8, stream), "zero ya");
    }

    void restart_state(int cur) {
        // common tail of reset / reset_candidate (src/cuda.cu:911-930,941-948)
        if (halpern) {
            if (n)
                cuda_check(cudaMemcpyAsync(anchor_x.p, x[cur].p, size_t(n) * 8,
                                           cudaMemcpyDeviceToDevice, stream), "anchor x");
            if (m) {
                cuda_check(cudaMemcpyAsync(anchor_y.p, y[cur].p, size_t(m) * 8,
                                           cudaMemcpyDeviceToDevice, stream), "anchor y");
                cuda_check(cudaMemcpyAsync(anchor_ax.p, ax[cur].p, size_t(m) * 8,
                                           cudaMemcpyDeviceToDevice, stream), "anchor ax");
            }
        }
        zero_average();
        sync_ctl();
        host_ctl->cur = cur;
        host_ctl->pending = 0;
        host_ctl->mass = 0;
        if (halpern) {
            host_ctl->epoch = 0;
            host_ctl->init_res = INFINITY;
            host_ctl->prev_res = INFINITY;
            host_ctl->restart = 0;
            host_ctl->lambda = 0;
            request_restart = false;
        }
        push_ctl();
        cuda_check(cudaStreamSynchronize(stream), "restart");
    }

    void reset_candidate(bool average) {
        flush();
        sync_ctl();
        int cur = host_ctl->cur;
        if (average) {
            if (n)
                cuda_check(cudaMemcpyAsync(x[cur].p, xa.p, size_t(n) * 8, cudaMemcpyDeviceToDevice,
                                           stream), "restart x");
            if (m)
                cuda_check(cudaMemcpyAsync(y[cur].p, ya.p, size_t(m) * 8, cudaMemcpyDeviceToDevice,
                                           stream), "restart y");
        }
        refresh_y32(cur);
        refresh_activity(cur);
        restart_state(cur);
    }

    void reset(const double *hx, const double *hy) {
        sync_ctl();
        int cur = host_ctl->cur;
        upload_perm(x[cur].p, hx, n, col_perm, scratch_n, false);
        upload_perm(y[cur].p, hy, m, row_perm, scratch_m, false);
        refresh_y32(cur);
        refresh_activity(cur);
        restart_state(cur);
        cuda_check(cudaStreamSynchronize(stream), "reset"); // the caller may reuse hx, hy
    }

    double monitor() {
        if (!mon_ax.p) {
            mon_ax.alloc(std::max<int64_t>(1, m));
            mon_aty.alloc(std::max<int64_t>(1, n));
            mon_qx.alloc(std::max<int64_t>(1, n));
            mon_part.alloc(size_t(5 * 148 * 8));
            mon_out.alloc(1);
            mon_arrive.alloc(1);
            cuda_check(cudaMemsetAsync(mon_arrive.p, 0, sizeof(unsigned), stream), "monitor");
            std::vector<double> hc(static_cast<size_t>(n));
            if (n)
                cuda_check(cudaMemcpy(hc.data(), c.p, size_t(n) * 8, cudaMemcpyDeviceToHost), "c");
            cscale = 1;
            for (double v : hc)
                cscale = std::max(cscale, 1 + std::abs(v));
        }
        flush();
        sync_ctl();
        int cur = host_ctl->cur;
        double best = INFINITY;
        for (int which = 0; which < 2; ++which) {
            const double *px = which ? xa.p : x[cur].p;
            const double *py = which ? ya.p : y[cur].p;
            if (m)
                spmv(A, px, mon_ax.p);
            if (n)
                spmv(At, py, mon_aty.p);
            if (sparse_q)
                q_spmv(px, mon_qx.p);
            if (std::max(n, m) == 0)
                return 0;
            int g = grid_for(std::max(n, m));
            monitor_kernel<<<g, kThreads, 0, stream>>>(
                n, m, px, py, mon_ax.p, mon_aty.p, sparse_q ? mon_qx.p : nullptr, c.p, q.p, lb.p,
                ub.p, rl.p, ru.p, cscale, mon_part.p, mon_arrive.p, mon_out.p);
            cuda_check(cudaGetLastError(), "monitor");
            double r = 0;
            cuda_check(cudaMemcpyAsync(&r, mon_out.p, 8, cudaMemcpyDeviceToHost, stream),
                       "monitor result");
            cuda_check(cudaStreamSynchronize(stream), "monitor sync");
            best = std::min(best, r);
        }
        return best;
    }

    // snapshot parts: x, y, xa, ya, ax, anchor_x, anchor_y, anchor_ax, control(11),
    // counters {accepted, rejected, empty_chunks, request_restart}; vectors in
    // the caller's order
    std::vector<int64_t> layout() const {
        int64_t hn = halpern ? n : 0, hm = halpern ? m : 0;
        return {n, m, n, m, m, hn, hm, hm, 11, 4};
    }
    static bool column_part(int i) { return i == 0 || i == 2 || i == 5; }
    void snapshot(double *out) {
        flush();
        sync_ctl();
        int cur = host_ctl->cur;
        auto L = layout();
        int64_t at = 0;
        const double *src[8] = {x[cur].p, y[cur].p, xa.p, ya.p, ax[cur].p,
                                anchor_x.p, anchor_y.p, anchor_ax.p};
        for (int i = 0; i < 8; ++i) {
            if (L[size_t(i)]) {
                if (column_part(i))
                    download_x(out + at, src[i]);
                else
                    download_y(out + at, src[i]);
            }
            at += L[size_t(i)];
        }
        cuda_check(cudaStreamSynchronize(stream), "snapshot");
        const Control &s = *host_ctl;
        double st[11] = {s.factor, s.mass, s.accepted, s.rejected, s.accept, s.weight,
                         s.epoch, s.init_res, s.prev_res, s.restart, s.lambda};
        std::memcpy(out + at, st, sizeof(st));
        at += 11;
        double cnt[4] = {double(accepted), double(rejected), double(empty_chunks),
                         request_restart ? 1. : 0.};
        std::memcpy(out + at, cnt, sizeof(cnt));
    }
    void restore(const double *in, const int64_t *sizes, int parts) {
        auto L = layout();
        if (parts != int(L.size()))
            throw Error(NK_ERR_INVALID, "GPU checkpoint state count");
        for (int i = 0; i < parts; ++i)
            if (sizes[i] != L[size_t(i)])
                throw Error(NK_ERR_INVALID, "GPU checkpoint state dimensions");
        int64_t at = 0;
        for (int i = 0; i < 10; ++i)
            at += L[size_t(i)];
        const double *cnt = in + at - 4;
        for (int i = 0; i < 4; ++i)
            if (!std::isfinite(cnt[i]) || cnt[i] < 0)
                throw Error(NK_ERR_INVALID, "GPU checkpoint counters");
        const double *st = in + at - 15;
        if (!(st[0] > 0) || st[2] < 0 || st[3] < 0)
            throw Error(NK_ERR_INVALID, "GPU checkpoint counters");
        sync_ctl();
        int cur = 0;
        double *dst[8] = {x[cur].p, y[cur].p, xa.p, ya.p, ax[cur].p,
                          anchor_x.p, anchor_y.p, anchor_ax.p};
        at = 0;
        for (int i = 0; i < 8; ++i) {
            if (L[size_t(i)]) {
                if (column_part(i))
                    upload_x(dst[i], in + at);
                else
                    upload_y(dst[i], in + at);
            }
            at += L[size_t(i)];
        }
        refresh_y32(cur);
        Control &s = *host_ctl;
        s.factor = st[0];
        s.mass = st[1];
        s.accepted = st[2];
        s.rejected = st[3];
        s.accept = st[4];
        s.weight = st[5];
        s.epoch = st[6];
        s.init_res = st[7];
        s.prev_res = st[8];
        s.restart = st[9];
        s.lambda = st[10];
        s.cur = cur;
        s.pending = 0;
        accepted = int64_t(cnt[0]);
        rejected = int64_t(cnt[1]);
        empty_chunks = int(cnt[2]);
        request_restart = cnt[3] != 0;
        push_ctl();
        cuda_check(cudaStreamSynchronize(stream), "restore");
    }

    // Runs `count` trials one by one with events around each kernel; returns the
    // mean durations in milliseconds of the primal kernel, of the dual step (the
    // panel kernel, when A has panels, plus the dual kernel) and of the panel
    // kernel alone (0 without panels).  With graphs on, each trial is a replay
    // of one captured trial whose events are graph nodes, so the kernels run
    // back to back as in the graph path; without, launches are plain.
    void profile(int count, double tau, double sigma, double *ms_primal, double *ms_dual,
                 double *ms_panel = nullptr) {
        if (count <= 0)
            throw Error(NK_ERR_INVALID, "profile needs a positive trial count");
        sync_ctl();
        host_ctl->tau = tau;
        host_ctl->sigma = sigma;
        push_ctl();
        for (auto &e : ev)
            cuda_check(cudaEventCreate(&e), "event");
        double tp = 0, td = 0, tk = 0;
        cudaGraphExec_t one = nullptr;
        try {
            if (graphs) {
                // the trial as the graph path runs it: one captured trial with
                // the events as graph nodes, replayed `count` times
                cudaGraph_t g = nullptr;
                ev_in_graph = true;
                cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal),
                           "profile capture");
                try {
                    launch_trial();
                } catch (...) {
                    cudaStreamEndCapture(stream, &g);
                    if (g)
                        cudaGraphDestroy(g);
                    throw;
                }
                ev_in_graph = false;
                cuda_check(cudaStreamEndCapture(stream, &g), "profile capture");
                cudaError_t e = cudaGraphInstantiate(&one, g, 0);
                cudaGraphDestroy(g);
                cuda_check(e, "profile instantiate");
            }
            for (int t = 0; t < count; ++t) {
                if (one)
                    cuda_check(cudaGraphLaunch(one, stream), "profile launch");
                else
                    launch_trial();
                cuda_check(cudaEventSynchronize(ev[2]), "profile sync");
                float a = 0, b = 0, k = 0;
                cudaEventElapsedTime(&a, ev[0], ev[1]);
                cudaEventElapsedTime(&b, ev[1], ev[2]);
                if (panels)
                    cudaEventElapsedTime(&k, ev[1], ev[3]);
                tp += a;
                td += b;
                tk += k;
            }
        } catch (...) {
            ev_in_graph = false;
            if (one)
                cudaGraphExecDestroy(one);
            for (auto &e : ev) {
                cudaEventDestroy(e);
                e = nullptr;
            }
            throw;
        }
        if (one)
            cudaGraphExecDestroy(one);
        for (auto &e : ev) {
            cudaEventDestroy(e);
            e = nullptr;
        }
        trials += count;
        sync_ctl();
        accepted = int64_t(host_ctl->accepted);
        rejected = int64_t(host_ctl->rejected);
        *ms_primal = tp / count;
        *ms_dual = td / count;
        if (ms_panel)
            *ms_panel = tk / count;
    }

    // Mean duration (ms) of `reps` plain SpMVs with A (which = 0: A x into Ax) or
    // A^T (which = 1: A^T y into dx's buffer), timed with events on the stream.
    // Leaves the iterates untouched (the products go to scratch buffers).
    double time_spmv(int which, int reps) {
        if (reps <= 0)
            throw Error(NK_ERR_INVALID, "reps must be positive");
        if (!mon_ax.p) {
            mon_ax.alloc(std::max<int64_t>(1, m));
            mon_aty.alloc(std::max<int64_t>(1, n));
        }
        sync_ctl();
        int cur = host_ctl->cur;
        cudaEvent_t a, b;
        cuda_check(cudaEventCreate(&a), "event");
        cuda_check(cudaEventCreate(&b), "event");
        cudaEventRecord(a, stream);
        for (int r = 0; r < reps; ++r) {
            if (which == 0)
                spmv(A, x[cur].p, mon_ax.p);
            else
                spmv(At, y[cur].p, mon_aty.p);
        }
        cudaEventRecord(b, stream);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return double(ms) / reps;
    }

    size_t device_bytes() const {
        size_t b = A.device_bytes() + At.device_bytes() + Q.device_bytes() + pan.device_bytes();
        for (auto *d : {&c, &q, &lb, &ub, &rl, &ru, &x[0], &x[1], &y[0], &y[1], &ax[0], &ax[1],
                        &xa, &ya, &dx, &anchor_x, &anchor_y, &anchor_ax, &part_p, &part_d,
                        &scratch_n, &scratch_m})
            b += d->bytes();
        b += dx32.bytes() + y32[0].bytes() + y32[1].bytes() + col_perm.bytes() + row_perm.bytes();
        return b;
    }
};

// Schedule of the fused kernels over their persistent grid (one CTA per SM of
// 1024 threads; occupancy_grid never launches more than fit at once).
//
// The cost of a chunk of padded length L is its memory work, what an SM's load
// path spends on it: one scattered sector per gathered entry, the entries'
// index and value stream, and the row epilogue's vector traffic (about
// 44 L + 70 sectors).  The chunks go to the CTAs by longest-first list
// scheduling on that cost (the next chunk to the least-loaded CTA, ties to the
// lowest index); inside a CTA the warps claim them dynamically, costliest
// first, so a slow chunk does not leave the rest of its CTA idle.  Every SM
// holds the same number of CTAs, so balanced CTAs mean balanced SMs whatever
// the block scheduler's placement.  Rows are sorted by length, so plain
// round-robin would put the long split-row chunks on the lowest CTAs.  Which
// warp or CTA runs a chunk changes no row sum, and the step rule's sums are
// added in list order, so results stay deterministic.

// Longest-first list scheduling: items (by index into cost) go, costliest
// first, to the least-loaded machine (ties to the lowest index); owner[k] is
// item k's machine.  Returns the items in assignment order.
std::vector<int64_t> lpt_assign(const std::vector<int64_t> &items, const std::vector<int64_t> &cost,
                                int64_t machines, std::vector<int64_t> &owner) {
    using Slot = std::pair<int64_t, int64_t>; // (load so far, machine)
    std::vector<int64_t> order(items);
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t a, int64_t b) { return cost[size_t(a)] > cost[size_t(b)]; });
    std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> heap;
    for (int64_t k = 0; k < machines; ++k)
        heap.push({0, k});
    for (int64_t c : order) {
        Slot t = heap.top();
        heap.pop();
        owner[size_t(c)] = t.second;
        heap.push({t.first + cost[size_t(c)], t.second});
    }
    return order;
}

// The schedule of `ids` (item k is ids[k], with memory work work[k]) onto
// `ctas` persistent CTAs: longest-first list scheduling by memory work, then
// each CTA's items costliest first (its warps claim them in that order).
// Uploads the per-CTA lists (off, list); returns the longest list.
int schedule_items(const std::vector<int64_t> &ids, const std::vector<int64_t> &work,
                   int64_t ctas, DevBuf<int64_t> &off_d, DevBuf<int64_t> &list_d,
                   cudaStream_t s) {
    const int64_t nit = int64_t(ids.size());
    ctas = std::max<int64_t>(1, ctas);
    std::vector<int64_t> all(static_cast<size_t>(nit)), cta(static_cast<size_t>(nit));
    for (int64_t k = 0; k < nit; ++k)
        all[size_t(k)] = k;
    const std::vector<int64_t> order = lpt_assign(all, work, ctas, cta); // costliest first
    std::vector<int64_t> off(static_cast<size_t>(ctas + 1), 0);
    for (int64_t k = 0; k < nit; ++k)
        ++off[size_t(cta[size_t(k)] + 1)];
    int longest = 0;
    for (int64_t b = 0; b < ctas; ++b) {
        longest = std::max(longest, int(off[size_t(b + 1)]));
        off[size_t(b + 1)] += off[size_t(b)];
    }
    std::vector<int64_t> list(static_cast<size_t>(std::max<int64_t>(1, nit)), 0);
    {
        std::vector<int64_t> pos(off.begin(), off.end() - 1);
        for (int64_t k : order)
            list[size_t(pos[size_t(cta[size_t(k)])]++)] = ids[size_t(k)];
    }
    {   // every item exactly once
        std::vector<int64_t> got(list.begin(), list.begin() + nit), want(ids);
        std::sort(got.begin(), got.end());
        std::sort(want.begin(), want.end());
        if (got != want)
            throw Error(NK_ERR_INVALID, "internal: chunk schedule is not a permutation");
    }
    upload_vector(off_d, off, s);
    upload_vector(list_d, list, s);
    return longest;
}

// Memory work of a SELL chunk of padded length L (see above).
int64_t chunk_work(int64_t L, bool split) { return 44 * L + (split ? 100 : 70); }

void build_schedule(SellMatrix &M, int64_t ctas, cudaStream_t s) {
    const int64_t nch = int64_t(M.chunk_len.size());
    const int64_t split_chunks = M.nsv / 32;
    std::vector<int64_t> ids(static_cast<size_t>(nch)), work(ids.size());
    for (int64_t c = 0; c < nch; ++c) {
        ids[size_t(c)] = c;
        work[size_t(c)] = chunk_work(M.chunk_len[size_t(c)], c < split_chunks);
    }
    M.max_cta_items = schedule_items(ids, work, ctas, M.coff, M.clist, s);
}

// The dual kernel's schedule when A's long rows take the panel path: the
// chunks past the split region, plus one combine chunk per 32 long rows
// (encoded -k-1), whose lanes each read their row's run sums (roff: row i's
// slots [roff[i], roff[i+1]); the warp waits for its row with the most) and
// run the row epilogue.
void build_dual_panel_schedule(SellMatrix &M, int64_t long_rows, const std::vector<int64_t> &roff,
                               int64_t ctas, cudaStream_t s) {
    const int64_t nch = int64_t(M.chunk_len.size());
    const int64_t split_chunks = M.nsv / 32;
    const int64_t combine = (long_rows + 31) / 32;
    std::vector<int64_t> ids, work;
    for (int64_t k = 0; k < combine; ++k) {
        int64_t most = 0;
        for (int64_t i = 32 * k; i < std::min(long_rows, 32 * k + 32); ++i)
            most = std::max(most, roff[size_t(i + 1)] - roff[size_t(i)]);
        ids.push_back(-k - 1);
        work.push_back(8 * most + 70);
    }
    for (int64_t c = split_chunks; c < nch; ++c) {
        ids.push_back(c);
        work.push_back(chunk_work(M.chunk_len[size_t(c)], false));
    }
    M.max_cta_items = schedule_items(ids, work, ctas, M.coff, M.clist, s);
}

// Persistent grid: as many CTAs as fit on the device at once, at most one warp
// per SELL chunk.
int occupancy_grid(const void *kernel, int64_t chunks, int threads = kThreads, size_t dyn = 0) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, dyn),
               "occupancy");
    per = std::max(1, per);
    int64_t need = (chunks + threads / 32 - 1) / (threads / 32);
    return int(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(sms) * per)));
}

// Shared memory a CTA of `kernel` can use dynamically while the SM still holds
// ctas_per_sm of them: the SM's shared memory split between them, less the
// per-CTA reservation and the kernel's static arrays (for the primal kernel's
// staged y entries and the panel kernel's dx slice).
size_t smem_budget(const void *kernel, int ctas_per_sm) {
    int dev = 0, per_sm = 0, optin = 0, reserved = 0;
    cudaGetDevice(&dev);
    cuda_check(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev),
               "shared memory per SM");
    cuda_check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
               "shared memory per block");
    cuda_check(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev),
               "reserved shared memory");
    cudaFuncAttributes fa{};
    cuda_check(cudaFuncGetAttributes(&fa, kernel), "kernel attributes");
    int64_t b = int64_t(per_sm) / ctas_per_sm - reserved - int64_t(fa.sharedSizeBytes);
    b = std::min<int64_t>(b, int64_t(optin) - int64_t(fa.sharedSizeBytes));
    return size_t(std::max<int64_t>(0, b) & ~int64_t(15));
}

// The panel kernel instance of a precision, with its dynamic shared memory
// raised to `bytes`; returns the kernel and the budget it allows.
const void *panel_kernel_for(int precision) {
    if (precision == NK_PRECISION_FP64)
        return (const void *)panel_kernel<double, double, double>;
    if (precision == NK_PRECISION_MIXED)
        return (const void *)panel_kernel<double, float, double>;
    return (const void *)panel_kernel<float, float, float>;
}

// Panel layout (nk_panel.cuh) of the first `rows` rows of an engine-order CSR
// (host ptr; device int64 indices and double values), panels of `width`
// columns, work units sized for `grid` CTAs to claim.  Built on the host from
// one download of those rows' entries.
void build_panels(PanelMatrix &P, int64_t rows, int64_t cols, const std::vector<int64_t> &ptr,
                  const int64_t *didx, const double *dval, int64_t width, int vbits, int grid,
                  size_t xsize, cudaStream_t s) {
    P.rows = rows;
    P.cols = cols;
    P.width = width;
    P.vbits = vbits;
    P.grid = grid;
    const int64_t E = ptr[size_t(rows)];
    P.entries = E;
    const int64_t np = (cols + width - 1) / width;
    P.npanels = int(np);
    std::vector<int64_t> hidx(static_cast<size_t>(E));
    std::vector<double> hval(static_cast<size_t>(E));
    if (E) {
        cuda_check(cudaMemcpyAsync(hidx.data(), didx, size_t(E) * 8, cudaMemcpyDeviceToHost, s),
                   "panel index download");
        cuda_check(cudaMemcpyAsync(hval.data(), dval, size_t(E) * 8, cudaMemcpyDeviceToHost, s),
                   "panel value download");
        cuda_check(cudaStreamSynchronize(s), "panel download");
    }
    // entries of each (panel, row) segment
    std::vector<int64_t> cnt(size_t(np * rows), 0);
    for (int64_t r = 0; r < rows; ++r)
        for (int64_t k = ptr[size_t(r)]; k < ptr[size_t(r + 1)]; ++k)
            ++cnt[size_t((hidx[size_t(k)] / width) * rows + r)];
    // Runs: a segment longer than a quarter of a lane's expected stream is cut
    // into runs of about equal length, so that no lane carries much more than
    // its share; each run is closed by its own marker and sums into its own
    // slot.  Slots are numbered row by row, then by panel, then by run, so a
    // row's slots are contiguous and in the order the dual kernel adds them.
    const int64_t lanes_min = int64_t(kPanelThreads);
    int64_t grand0 = 0;
    for (int64_t v : cnt)
        grand0 += v > 0 ? v + 1 : 0;
    const int64_t units0 = std::max<int64_t>(1, std::min<int64_t>(grid, (grand0 + lanes_min - 1) / lanes_min));
    const int64_t lane_load = std::max<int64_t>(1, grand0 / (units0 * lanes_min));
    const int64_t run_max = std::max<int64_t>(NK_PANEL_MIN_SPLIT, (lane_load + 3) / 4);
    auto runs_of = [&](int64_t c) { return c > 0 ? (c + run_max - 1) / run_max : 0; };
    std::vector<int64_t> sbase(size_t(np * rows), -1), roff(size_t(rows + 1), 0);
    int64_t nslots = 0;
    for (int64_t r = 0; r < rows; ++r) {
        roff[size_t(r)] = nslots;
        for (int64_t p = 0; p < np; ++p) {
            const int64_t c = cnt[size_t(p * rows + r)];
            if (c > 0) {
                sbase[size_t(p * rows + r)] = nslots;
                nslots += runs_of(c);
            }
        }
    }
    roff[size_t(rows)] = nslots;
    P.slots = nslots;
    // length of run k of a segment of c entries in nr runs (the first c % nr runs
    // one longer), and its first entry's index within the segment
    auto run_len = [](int64_t c, int64_t nr, int64_t k) { return c / nr + (k < c % nr ? 1 : 0); };
    // units: one per CTA, each an equal share of all panels' entries (markers
    // included).  A unit holds one piece per panel it touches; a piece is one
    // chunk per warp, and the piece's runs go onto its kPanelThreads lanes
    // longest first onto the least-loaded lane, so every lane of a unit carries
    // nearly the same stream length.  A panel's runs (longest first) go to its
    // pieces by remaining quota.  A run's place is (lane, first step) in its
    // piece, then its first entry's offset.
    int64_t grand = 0;
    for (int64_t v : cnt)
        for (int64_t k = 0, nr = runs_of(v); k < nr; ++k)
            grand += run_len(v, nr, k) + 1;
    const int64_t nunits_target = std::max<int64_t>(1, std::min<int64_t>(
        grid, (grand + kPanelThreads - 1) / kPanelThreads)); // at least a run per lane
    const double share = double(grand) / double(nunits_target);
    std::vector<int64_t> place(size_t(std::max<int64_t>(1, nslots)), -1);
    std::vector<int64_t> cptr(1, 0);
    std::vector<int4> pieces;          // {panel, first chunk, end chunk, unit}
    std::vector<int64_t> items, isize, load, quota_left;
    using Slot = std::pair<int64_t, int64_t>; // (load, lane)
    double filled = 0;                 // entries placed in units before this panel
    for (int64_t p = 0; p < np; ++p) {
        items.clear();
        isize.clear();
        int64_t total = 0;
        for (int64_t r = 0; r < rows; ++r) {
            const int64_t c = cnt[size_t(p * rows + r)];
            for (int64_t k = 0, nr = runs_of(c); k < nr; ++k) {
                items.push_back(sbase[size_t(p * rows + r)] + k);
                isize.push_back(run_len(c, nr, k) + 1);
                total += isize.back();
            }
        }
        if (items.empty())
            continue;
        std::vector<int64_t> order(items.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](int64_t a, int64_t b) { return isize[size_t(a)] > isize[size_t(b)]; });
        // the units this panel's entries fall in, and each one's quota
        const int64_t u0 = std::min<int64_t>(nunits_target - 1, int64_t(filled / share));
        const int64_t u1 = std::min<int64_t>(nunits_target - 1,
                                             int64_t((filled + total - 1e-9) / share));
        quota_left.assign(size_t(u1 - u0 + 1), 0);
        for (int64_t u = u0; u <= u1; ++u) {
            const double lo = std::max(filled, double(u) * share);
            const double hi = u == nunits_target - 1 ? filled + total
                                                     : std::min(filled + total, (u + 1) * share);
            quota_left[size_t(u - u0)] = std::max<int64_t>(0, int64_t(hi - lo + 0.5));
        }
        filled += total;
        std::vector<std::vector<int64_t>> piece_items(quota_left.size());
        for (int64_t o : order) {
            size_t best = 0;
            for (size_t q = 1; q < quota_left.size(); ++q)
                if (quota_left[q] > quota_left[best])
                    best = q;
            piece_items[best].push_back(o);
            quota_left[best] -= isize[size_t(o)];
        }
        for (size_t q = 0; q < piece_items.size(); ++q) {
            if (piece_items[q].empty())
                continue;
            const int64_t c0 = int64_t(cptr.size()) - 1;
            load.assign(size_t(kPanelThreads), 0);
            std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> heap;
            for (int64_t l = 0; l < kPanelThreads; ++l)
                heap.push({0, l});
            for (int64_t o : piece_items[q]) {
                Slot t = heap.top();
                heap.pop();
                place[size_t(items[size_t(o)])] = t.second * (int64_t(1) << 20) + t.first;
                heap.push({t.first + isize[size_t(o)], t.second});
                load[size_t(t.second)] = t.first + isize[size_t(o)];
            }
            for (int64_t c = 0; c < kPanelWarps; ++c) {
                int64_t top = 0;
                for (int t = 0; t < 32; ++t)
                    top = std::max(top, load[size_t(c * 32 + t)]);
                cptr.push_back(cptr.back() + 32 * top);
            }
            for (int64_t o : piece_items[q]) { // (lane, step) -> offset of the first entry
                const int64_t sl = items[size_t(o)];
                const int64_t lane = place[size_t(sl)] >> 20,
                              step = place[size_t(sl)] & ((int64_t(1) << 20) - 1);
                place[size_t(sl)] = cptr[size_t(c0 + lane / 32)] + 32 * step + lane % 32;
            }
            pieces.push_back(make_int4(int(p), int(c0), int(c0 + kPanelWarps), int(u0 + q)));
        }
    }
    P.padded = cptr.back();
    std::vector<uint16_t> hl(static_cast<size_t>(std::max<int64_t>(1, P.padded)), 0);
    std::vector<double> hv64(vbits == 64 ? size_t(std::max<int64_t>(1, P.padded)) : 1, 0.);
    std::vector<float> hv32(vbits == 64 ? 1 : size_t(std::max<int64_t>(1, P.padded)), 0.f);
    auto put = [&](int64_t at, uint16_t j, double v, int64_t slot) {
        hl[size_t(at)] = j;
        if (j == kPanelMarker) {
            if (vbits == 64)
                std::memcpy(&hv64[size_t(at)], &slot, 8);
            else {
                const int32_t s32 = int32_t(slot);
                std::memcpy(&hv32[size_t(at)], &s32, 4);
            }
        } else if (vbits == 64)
            hv64[size_t(at)] = v;
        else
            hv32[size_t(at)] = float(v);
    };
    std::vector<int64_t> seen(size_t(np), 0); // entries of the current row placed per panel
    for (int64_t r = 0; r < rows; ++r) {
        std::fill(seen.begin(), seen.end(), 0);
        for (int64_t k = ptr[size_t(r)]; k < ptr[size_t(r + 1)]; ++k) {
            const int64_t j = hidx[size_t(k)], p = j / width;
            const int64_t c = cnt[size_t(p * rows + r)], nr = runs_of(c);
            // the run of the segment's seen-th entry: the first c % nr runs are one longer
            const int64_t e = seen[size_t(p)]++, big = c / nr + 1, nbig = c % nr;
            const int64_t run = e < nbig * big ? e / big : nbig + (e - nbig * big) / (c / nr);
            int64_t &at = place[size_t(sbase[size_t(p * rows + r)] + run)];
            put(at, uint16_t(j - p * width), hval[size_t(k)], 0);
            at += 32; // the lane's next step
        }
        for (int64_t p = 0; p < np; ++p) {
            const int64_t c = cnt[size_t(p * rows + r)];
            for (int64_t q = 0, nr = runs_of(c); q < nr; ++q) {
                const int64_t sl = sbase[size_t(p * rows + r)] + q;
                put(place[size_t(sl)], kPanelMarker, 0., sl);
            }
        }
    }
    // pieces in unit order; unit u runs pieces [uoff[u], uoff[u+1])
    std::stable_sort(pieces.begin(), pieces.end(),
                     [](const int4 &a, const int4 &b) { return a.w < b.w; });
    std::vector<int64_t> uoff(size_t(nunits_target + 1), 0);
    for (const int4 &pc : pieces)
        ++uoff[size_t(pc.w + 1)];
    for (int64_t u = 0; u < nunits_target; ++u)
        uoff[size_t(u + 1)] += uoff[size_t(u)];
    P.nunits = nunits_target;
    if (pieces.empty())
        pieces.push_back(make_int4(0, 0, 0, 0));
    upload_vector(P.units, pieces, s);
    upload_vector(P.uoff, uoff, s);
    upload_vector(P.roff, roff, s);
    P.hroff = roff;
    P.claim.alloc(2);
    cuda_check(cudaMemsetAsync(P.claim.p, 0, P.claim.bytes(), s), "panel claims");
    upload_vector(P.cptr, cptr, s);
    upload_vector(P.lidx, hl, s);
    if (vbits == 64)
        upload_vector(P.val64, hv64, s);
    else
        upload_vector(P.val32, hv32, s);
    P.partial.alloc(size_t(std::max<int64_t>(1, nslots)));
    cuda_check(cudaMemsetAsync(P.partial.p, 0, P.partial.bytes(), s), "panel partials");
    cuda_check(cudaStreamSynchronize(s), "panel build");
}

// Kernel instances and persistent grids of an engine.  The fused kernels'
// grids hold exactly the CTAs that fit on the device at once; their slot
// memory is sized after the schedules are built (attach_slots).
template <class Acc, class V, class I> void configure(Engine &E) {
    constexpr bool F32 = sizeof(Acc) == 4;
    const void *pk = (const void *)primal_kernel_for<Acc, V, I>(E.sparse_q, E.At.nsv > 0);
    const void *dk = E.panels           ? (const void *)dual_kernel<Acc, V, I, F32, false, true>
                     : E.A.nsv > 0 ? (const void *)dual_kernel<Acc, V, I, F32, true>
                                        : (const void *)dual_kernel<Acc, V, I, F32, false>;
    // the slot arrays stay far below the default 48 KB; the grids are sized
    // without them, which the occupancy check after the schedules confirms
    E.grid_p = occupancy_grid(pk, (E.At.nv + 31) / 32, kFusedThreads, 0);
    E.grid_d = occupancy_grid(dk, (E.A.nv + 31) / 32, kFusedThreads, 0);
    E.grid_s = occupancy_grid((const void *)spmv_kernel<V, I>, int64_t(1) << 40);
}
template <class Acc, class V, class I> void attach_slots(Engine &E) {
    constexpr bool F32 = sizeof(Acc) == 4;
    const void *pk = (const void *)primal_kernel_for<Acc, V, I>(E.sparse_q, E.At.nsv > 0);
    const void *dk = E.panels           ? (const void *)dual_kernel<Acc, V, I, F32, false, true>
                     : E.A.nsv > 0 ? (const void *)dual_kernel<Acc, V, I, F32, true>
                                        : (const void *)dual_kernel<Acc, V, I, F32, false>;
    for (auto [k, bytes, grid] : {std::tuple<const void *, size_t, int>{pk, E.smem_p(), E.grid_p},
                                  {dk, E.smem_d(), E.grid_d}}) {
        if (bytes > 48 * 1024)
            cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(bytes)),
                       "slot memory");
        int per = 0, dev = 0, sms = 148;
        cuda_check(cudaGetDevice(&dev), "device");
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, kFusedThreads, bytes),
                   "occupancy");
        if (int64_t(per) * sms < grid)
            throw Error(NK_ERR_UNSUPPORTED, "fused kernel grid does not fit the device");
    }
}

Engine *create_engine(const nk_csr *Ah, const nk_csr *Qh, const double *hc, const double *hq,
                      const double *hlb, const double *hub, const double *hrl, const double *hru,
                      const double *hx0, const double *hy0, const nk_pdhg_options *o) {
    if (!Ah || !hc || !hlb || !hub || !hrl || !hru || !hx0 || !hy0 || !o)
        throw Error(NK_ERR_INVALID, "null argument");
    int64_t m = Ah->rows, n = Ah->cols;
    if (m < 0 || n < 0)
        throw Error(NK_ERR_INVALID, "Negative matrix dimension");
    validate_csr(Ah, m, n, "A");
    bool sparse_q = Qh && Qh->rows > 0 && Qh->ptr && Qh->ptr[Qh->rows] > 0;
    if (sparse_q)
        validate_csr(Qh, n, n, "Q");
    if (o->halpern && o->adaptive)
        throw Error(NK_ERR_UNSUPPORTED, "Halpern requires a fixed PDHG operator");
    if (!std::isfinite(o->reflection) || o->reflection < 0 || o->reflection > 1)
        throw Error(NK_ERR_INVALID, "Invalid Halpern reflection");
    if (o->precision < 0 || o->precision > 2)
        throw Error(NK_ERR_INVALID, "unknown matrix precision");
    if (sparse_q && o->precision == NK_PRECISION_MIXED)
        throw Error(NK_ERR_UNSUPPORTED, "Sparse QP requires FP64 matrices");
    int64_t nnz = Ah->ptr[m], qnnz = sparse_q ? Qh->ptr[n] : 0;
    bool fits32 = m <= INT32_MAX && n <= INT32_MAX && nnz <= INT32_MAX && qnnz <= INT32_MAX;
    if (o->index_bits == 32 && !fits32)
        throw Error(NK_ERR_INVALID, "Model exceeds 32-bit CSR limits");
    if (m >= INT32_MAX || n >= INT32_MAX)
        throw Error(NK_ERR_UNSUPPORTED, "more than 2^31 rows or columns");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        throw Error(NK_ERR_NO_DEVICE, "no CUDA device");
    size_t freeb = 0, total = 0;
    cuda_check(cudaMemGetInfo(&freeb, &total), "cudaMemGetInfo");
    // the reference guard (src/cuda.cu:1292-1298)
    long double estimate = 48.L * (nnz + qnnz) + 240.L * (m + n + 2);
    if (estimate > .8L * freeb)
        throw Error(NK_ERR_MEMORY,
                    "Estimated GPU storage exceeds 80% of available memory; use --device cpu");
    auto E = std::make_unique<Engine>();
    E->n = n;
    E->m = m;
    E->adaptive = o->adaptive && !sparse_q;
    E->halpern = o->halpern;
    E->residual_restarts = o->residual_restarts;
    E->graphs = o->graphs;
    E->reflection = o->reflection;
    E->precision = o->precision;
    E->sparse_q = sparse_q;
    E->wide = !fits32 || o->index_bits == 64;
    cuda_check(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking), "stream");
    cudaStream_t s = E->stream;
    const int vbits = o->precision == NK_PRECISION_FP64 ? 64 : 32;

    // ---- A on the device, its transpose, and the engine orders
    DevBuf<int64_t> rp, ri, tp, ti;
    DevBuf<double> rv, tv;
    upload_raw(Ah, vbits, s, rp, ri, rv);
    device_transpose(m, n, nnz, rp.p, ri.p, rv.p, tp, ti, tv, s);
    std::vector<int64_t> aptr(Ah->ptr, Ah->ptr + m + 1), tptr(static_cast<size_t>(n + 1));
    cuda_check(cudaMemcpy(tptr.data(), tp.p, size_t(n + 1) * 8, cudaMemcpyDeviceToHost), "A^T ptr");
    std::vector<int64_t> rlen(static_cast<size_t>(m)), clen(static_cast<size_t>(n));
    for (int64_t i = 0; i < m; ++i)
        rlen[size_t(i)] = aptr[size_t(i + 1)] - aptr[size_t(i)];
    for (int64_t j = 0; j < n; ++j)
        clen[size_t(j)] = tptr[size_t(j + 1)] - tptr[size_t(j)];
    std::vector<int64_t> rperm = order_by_length_desc(rlen), cperm = order_by_length_desc(clen);
    std::vector<int64_t> rinv(static_cast<size_t>(m)), cinv(static_cast<size_t>(n));
    for (int64_t i = 0; i < m; ++i)
        rinv[size_t(rperm[size_t(i)])] = i;
    for (int64_t j = 0; j < n; ++j)
        cinv[size_t(cperm[size_t(j)])] = j;
    DevBuf<int64_t> d_rinv, d_cinv;
    upload_vector(E->row_perm, rperm, s);
    upload_vector(E->col_perm, cperm, s);
    upload_vector(d_rinv, rinv, s);
    upload_vector(d_cinv, cinv, s);
    {
        // rows of A in engine order, columns mapped to engine columns; entries
        // keep their CSR order (the CPU's summation order)
        DevBuf<int64_t> pi;
        DevBuf<double> pv;
        auto pptr = permute_device_csr(m, aptr, rp.p, ri.p, rv.p, rperm, E->row_perm.p, d_cinv.p,
                                       pi, pv, s);
        build_sell(E->A, m, n, pptr, pi.p, pv.p, E->wide, vbits, s);
        // A's long rows (the SELL's split rows) also by column panel, for the dual
        // kernel: panels as wide as one CTA's shared memory holds dx entries, at
        // most 65535 columns (16-bit offsets, one value kept for markers), a
        // multiple of 16
        if (NK_PANEL && E->A.nsr > 0 && n > 0) {
            const void *pk = panel_kernel_for(o->precision);
            const int64_t xsize = o->precision == NK_PRECISION_FP32 ? 4 : 8;
            int64_t width = std::min<int64_t>(kPanelMaxWidth,
                                              int64_t(smem_budget(pk, kPanelMinBlocks)) / xsize);
            width = std::min<int64_t>(width, (n + 15) / 16 * 16) / 16 * 16;
            const int64_t np = width > 0 ? (n + width - 1) / width : 0;
            // worth it only where the long rows' entries come in long runs per
            // panel: the stream then runs at memory speed, while a panel's
            // segments of a few entries each cost about what their gathers do
            int64_t long_entries = 0;
            for (int64_t i = 0; i < E->A.nsr; ++i)
                long_entries += pptr[size_t(i + 1)] - pptr[size_t(i)];
            const bool long_runs =
                width >= 16 && long_entries >= NK_PANEL_MIN_RUN * np * E->A.nsr;
            if (long_runs && np * E->A.nsr <= (int64_t(1) << 25)) {
                const size_t smem = size_t(width * xsize);
                cuda_check(cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                int(smem)),
                           "panel shared memory");
                int dev = 0, sms = 148, per = 0;
                cuda_check(cudaGetDevice(&dev), "device");
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, pk, kPanelThreads,
                                                                         smem),
                           "panel occupancy");
                if (per > 0) {
                    build_panels(E->pan, E->A.nsr, n, pptr, pi.p, pv.p, width, vbits, sms * per,
                                 size_t(xsize), s);
                    E->pan.smem = smem;
                    E->panels = true;
                }
            }
        }
    }
    {
        // rows of A^T (columns of A) in engine order; the transpose lists every
        // column's entries by increasing original row, the CPU's order
        DevBuf<int64_t> pi;
        DevBuf<double> pv;
        auto pptr = permute_device_csr(n, tptr, tp.p, ti.p, tv.p, cperm, E->col_perm.p, d_rinv.p,
                                       pi, pv, s);
        build_sell(E->At, n, m, pptr, pi.p, pv.p, E->wide, vbits, s);
    }
    rp.release(); ri.release(); rv.release(); tp.release(); ti.release(); tv.release();
    if (sparse_q) {
        DevBuf<int64_t> qp, qi, pi;
        DevBuf<double> qv, pv;
        upload_raw(Qh, vbits, s, qp, qi, qv);
        std::vector<int64_t> qptr_h(Qh->ptr, Qh->ptr + n + 1);
        auto pptr = permute_device_csr(n, qptr_h, qp.p, qi.p, qv.p, cperm, E->col_perm.p, d_cinv.p,
                                       pi, pv, s);
        E->Q.n = n;
        E->Q.nnz = qnnz;
        E->Q.wide = E->wide;
        E->Q.vbits = vbits;
        upload_vector(E->Q.ptr, pptr, s);
        E->Q.idx64.alloc(E->wide ? size_t(std::max<int64_t>(1, qnnz)) : 1);
        E->Q.idx32.alloc(E->wide ? 1 : size_t(std::max<int64_t>(1, qnnz)));
        E->Q.val64.alloc(vbits == 64 ? size_t(std::max<int64_t>(1, qnnz)) : 1);
        E->Q.val32.alloc(vbits == 64 ? 1 : size_t(std::max<int64_t>(1, qnnz)));
        int g = grid_for(qnnz, 148 * 32);
        if (E->wide && vbits == 64)
            convert_csr<double, int64_t><<<g, kThreads, 0, s>>>(qnnz, pi.p, pv.p, E->Q.idx64.p, E->Q.val64.p);
        else if (E->wide)
            convert_csr<float, int64_t><<<g, kThreads, 0, s>>>(qnnz, pi.p, pv.p, E->Q.idx64.p, E->Q.val32.p);
        else if (vbits == 64)
            convert_csr<double, int32_t><<<g, kThreads, 0, s>>>(qnnz, pi.p, pv.p, E->Q.idx32.p, E->Q.val64.p);
        else
            convert_csr<float, int32_t><<<g, kThreads, 0, s>>>(qnnz, pi.p, pv.p, E->Q.idx32.p, E->Q.val32.p);
        cuda_check(cudaGetLastError(), "Q convert");
        cuda_check(cudaStreamSynchronize(s), "Q build");
        // norms for the QP step safety (src/cpu.cpp:25-42, src/model.cpp:257-267)
        std::vector<double> cols(static_cast<size_t>(n), 0.0);
        double rowmax = 0;
        for (int64_t i = 0; i < m; ++i) {
            double sum = 0;
            for (int64_t k = Ah->ptr[i]; k < Ah->ptr[i + 1]; ++k) {
                sum += std::abs(Ah->value[k]);
                cols[size_t(Ah->index[k])] += std::abs(Ah->value[k]);
            }
            rowmax = std::max(rowmax, sum);
        }
        double colmax = 0;
        for (double v : cols)
            colmax = std::max(colmax, v);
        E->a_norm = std::sqrt(rowmax) * std::sqrt(colmax);
        long double largest = 0;
        for (int64_t i = 0; i < n; ++i) {
            long double sum = std::abs(hq ? hq[i] : 0.0);
            for (int64_t k = Qh->ptr[i]; k < Qh->ptr[i + 1]; ++k)
                sum += std::abs(Qh->value[k]);
            largest = std::max(largest, sum);
        }
        E->q_norm = std::nextafter(double(largest), INFINITY);
    }

    // ---- vectors, in engine order
    auto vec = [&](DevBuf<double> &d, const double *h, int64_t len, const std::vector<int64_t> &perm) {
        d.alloc(std::max<int64_t>(1, len));
        if (len && h) {
            std::vector<double> tmp(static_cast<size_t>(len));
            for (int64_t i = 0; i < len; ++i)
                tmp[size_t(i)] = h[perm[size_t(i)]];
            cuda_check(cudaMemcpyAsync(d.p, tmp.data(), size_t(len) * 8, cudaMemcpyHostToDevice, s),
                       "vector");
            cuda_check(cudaStreamSynchronize(s), "vector");
        } else if (len)
            cuda_check(cudaMemsetAsync(d.p, 0, size_t(len) * 8, s), "vector zero");
    };
    vec(E->c, hc, n, cperm);
    vec(E->q, hq, n, cperm);
    E->diag_q = hq && std::any_of(hq, hq + n, [](double v) { return v != 0.; });
    vec(E->lb, hlb, n, cperm);
    vec(E->ub, hub, n, cperm);
    vec(E->rl, hrl, m, rperm);
    vec(E->ru, hru, m, rperm);
    vec(E->x[0], hx0, n, cperm);
    vec(E->x[1], hx0, n, cperm);
    vec(E->y[0], hy0, m, rperm);
    vec(E->y[1], hy0, m, rperm);
    vec(E->xa, nullptr, n, cperm);
    vec(E->ya, nullptr, m, rperm);
    vec(E->ax[0], nullptr, m, rperm);
    vec(E->ax[1], nullptr, m, rperm);
    E->scratch_n.alloc(size_t(std::max<int64_t>(1, n)));
    E->scratch_m.alloc(size_t(std::max<int64_t>(1, m)));
    if (o->precision == NK_PRECISION_FP32) {
        E->dx32.alloc(std::max<int64_t>(1, n));
        E->y32[0].alloc(std::max<int64_t>(1, m));
        E->y32[1].alloc(std::max<int64_t>(1, m));
        E->dx.alloc(1);
    } else {
        vec(E->dx, nullptr, n, cperm);
        E->dx32.alloc(1);
        E->y32[0].alloc(1);
        E->y32[1].alloc(1);
    }
    if (E->halpern) {
        vec(E->anchor_x, hx0, n, cperm);
        vec(E->anchor_y, hy0, m, rperm);
        vec(E->anchor_ax, nullptr, m, rperm);
    } else {
        E->anchor_x.alloc(1);
        E->anchor_y.alloc(1);
        E->anchor_ax.alloc(1);
    }
    if (o->precision == NK_PRECISION_FP64)
        E->wide ? configure<double, double, int64_t>(*E) : configure<double, double, int32_t>(*E);
    else if (o->precision == NK_PRECISION_MIXED)
        E->wide ? configure<double, float, int64_t>(*E) : configure<double, float, int32_t>(*E);
    else
        E->wide ? configure<float, float, int64_t>(*E) : configure<float, float, int32_t>(*E);
    build_schedule(E->At, E->grid_p, s);
    if (E->panels)
        build_dual_panel_schedule(E->A, E->pan.rows, E->pan.hroff, E->grid_d, s);
    else
        build_schedule(E->A, E->grid_d, s);
    if (o->precision == NK_PRECISION_FP64)
        E->wide ? attach_slots<double, double, int64_t>(*E) : attach_slots<double, double, int32_t>(*E);
    else if (o->precision == NK_PRECISION_MIXED)
        E->wide ? attach_slots<double, float, int64_t>(*E) : attach_slots<double, float, int32_t>(*E);
    else
        E->wide ? attach_slots<float, float, int64_t>(*E) : attach_slots<float, float, int32_t>(*E);
    E->split_p.alloc(size_t(std::max(1, E->At.ncounters)));
    E->split_d.alloc(size_t(2 * std::max(1, E->A.ncounters)));
    cuda_check(cudaMemsetAsync(E->split_p.p, 0, E->split_p.bytes(), s), "split slots");
    cuda_check(cudaMemsetAsync(E->split_d.p, 0, E->split_d.bytes(), s), "split slots");
    E->part_p.alloc(size_t(E->grid_p));
    E->part_d.alloc(size_t(2 * E->grid_d));
    E->ctl.alloc(1);
    cuda_check(cudaMallocHost(reinterpret_cast<void **>(&E->host_ctl), sizeof(Control)), "pinned");
    Control init{};
    init.factor = 1;
    init.init_res = INFINITY;
    init.prev_res = INFINITY;
    init.flags = (E->adaptive ? 1 : 0) | (E->halpern ? 2 : 0) | (E->residual_restarts ? 4 : 0);
    *E->host_ctl = init;
    E->push_ctl();
    E->refresh_y32(0);
    E->refresh_activity(0);
    if (E->halpern && m)
        cuda_check(cudaMemcpyAsync(E->anchor_ax.p, E->ax[0].p, size_t(m) * 8,
                                   cudaMemcpyDeviceToDevice, s), "anchor activity");
    cuda_check(cudaStreamSynchronize(s), "engine init");
    return E.release();
}

} // namespace nk

#include "nk_solve.cuh"
#include "nk_batch.cuh"
#include "nk_presolve.cuh"
#include "nk_newton.cuh"

namespace nk {
// Copies a caller model (C ABI) into the host representation, with the checks
// of Model::validate for the continuous part (src/model.cpp:74-123).
HostModel host_model(const nk_model *model) {
    if (!model)
        throw Error(NK_ERR_INVALID, "null model");
    const int64_t m = model->A.rows, n = model->A.cols;
    if (m < 0 || n < 0 || !model->c || !model->lb || !model->ub || !model->rl || !model->ru)
        throw Error(NK_ERR_INVALID, "incomplete model");
    validate_csr(&model->A, m, n, "A");
    const bool has_q = model->Q.rows > 0 && model->Q.ptr && model->Q.ptr[model->Q.rows] > 0;
    if (has_q)
        validate_csr(&model->Q, n, n, "Q");
    HostModel hm;
    auto csr = [](const nk_csr &c, Csr &out) {
        out.rows = c.rows;
        out.cols = c.cols;
        out.ptr.assign(c.ptr, c.ptr + c.rows + 1);
        out.index.assign(c.index, c.index + c.ptr[c.rows]);
        out.value.assign(c.value, c.value + c.ptr[c.rows]);
    };
    csr(model->A, hm.A);
    if (has_q)
        csr(model->Q, hm.Q);
    else {
        hm.Q.rows = hm.Q.cols = n;
        hm.Q.ptr.assign(size_t(n + 1), 0);
    }
    hm.c.assign(model->c, model->c + n);
    hm.q = model->q ? std::vector<double>(model->q, model->q + n) : std::vector<double>(size_t(n), 0.0);
    hm.lb.assign(model->lb, model->lb + n);
    hm.ub.assign(model->ub, model->ub + n);
    hm.rl.assign(model->rl, model->rl + m);
    hm.ru.assign(model->ru, model->ru + m);
    hm.offset = model->offset;
    // the value checks of Model::validate (src/model.cpp:74-105)
    if (!std::isfinite(hm.offset))
        throw Error(NK_ERR_INVALID, "Invalid objective offset/sense");
    for (size_t j = 0; j < size_t(n); ++j) {
        if (!std::isfinite(hm.c[j]) || !std::isfinite(hm.q[j]))
            throw Error(NK_ERR_INVALID, "Nonfinite objective coefficient");
        const double l = hm.lb[j], u = hm.ub[j];
        if (std::isnan(l) || std::isnan(u) || l == kInf || u == -kInf || l > u)
            throw Error(NK_ERR_INVALID, "Invalid bounds for x" + std::to_string(j));
    }
    for (size_t i = 0; i < size_t(m); ++i) {
        const double l = hm.rl[i], u = hm.ru[i];
        if (std::isnan(l) || std::isnan(u) || l == kInf || u == -kInf || l > u)
            throw Error(NK_ERR_INVALID, "Invalid row bounds");
    }
    // coefficients and indices of A and Q; the reference's further convexity
    // certificate for a Q that is not diagonally dominant (a sparse LU above
    // 256 columns, a dense elimination below, src/model.cpp:143-252) is not
    // repeated: a non-convex Q is the caller's error
    validate_entries(hm);
    return hm;
}
} // namespace nk

using nk::guard;

namespace {
// A required pointer argument that is null is an argument error reported as
// NK_ERR_INVALID, never a host crash.
void need(const void *p, const char *what) {
    if (!p)
        throw nk::Error(NK_ERR_INVALID, std::string("null ") + what);
}
} // namespace

struct nk_pdhg {
    nk::Engine *e;
};

extern "C" {
unsigned nk_abi_version(void) { return 1; }
const char *nk_last_error(void) { return nk::g_last_error; }

nk_status nk_pdhg_create(const nk_csr *A, const nk_csr *Q, const double *c, const double *q,
                         const double *lb, const double *ub, const double *rl, const double *ru,
                         const double *x0, const double *y0, const nk_pdhg_options *opts,
                         nk_pdhg **out) {
    return guard([&] {
        if (!out)
            throw nk::Error(NK_ERR_INVALID, "null output handle");
        *out = nullptr;
        auto *e = nk::create_engine(A, Q, c, q, lb, ub, rl, ru, x0, y0, opts);
        *out = new nk_pdhg{e};
    });
}
void nk_pdhg_destroy(nk_pdhg *h) {
    if (h) {
        delete h->e;
        delete h;
    }
}
#define NK_HANDLE                                                                                  \
    if (!h || !h->e)                                                                               \
        throw nk::Error(NK_ERR_INVALID, "null engine handle");
nk_status nk_pdhg_advance(nk_pdhg *h, int count, double tau, double sigma, int *accepted) {
    return guard([&] {
        NK_HANDLE
        int r = h->e->advance(count, tau, sigma);
        if (accepted)
            *accepted = r;
    });
}
nk_status nk_pdhg_rejected_steps(nk_pdhg *h, int64_t *out) {
    return guard([&] {
        NK_HANDLE
        need(out, "output");
        *out = h->e->rejected;
    });
}
nk_status nk_pdhg_restart_requested(nk_pdhg *h, int *out) {
    return guard([&] {
        NK_HANDLE
        need(out, "output");
        *out = h->e->request_restart ? 1 : 0;
    });
}
nk_status nk_pdhg_monitor(nk_pdhg *h, double *out) {
    return guard([&] {
        NK_HANDLE
        need(out, "output");
        *out = h->e->monitor();
    });
}
// ---- KKT proxy on fixed library scratch (see nk_monitor_static in nk_pdhg.h).
// Callers that may not allocate device memory get the monitor kernel launched
// on this array instead of engine buffers: bytes [0, 256) hold the kernel's
// arrival counter, the rest five partial sums per block (room for one block
// per kThreads entries of NK_MONITOR_STATIC_MAX; a launch uses at most 1184).
namespace {
constexpr int64_t kStaticMonitorBlocks = NK_MONITOR_STATIC_MAX / nk::kThreads;
constexpr size_t kStaticMonitorBytes = 256 + size_t(kStaticMonitorBlocks) * 5 * sizeof(double);
static __device__ __align__(256) unsigned char g_monitor_scratch[kStaticMonitorBytes];

// Device address of g_monitor_scratch on the current device.  In host code the
// symbol is only a stand-in; its device address is looked up once per device.
unsigned char *static_monitor_scratch() {
    constexpr int kMaxDevices = 64;
    static std::mutex lock;
    static unsigned char *address[kMaxDevices] = {};
    int dev = 0;
    nk::cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices)
        throw nk::Error(NK_ERR_UNSUPPORTED, "device index beyond the static scratch table");
    std::lock_guard<std::mutex> hold(lock);
    if (!address[dev]) {
        void *p = nullptr;
        nk::cuda_check(cudaGetSymbolAddress(&p, g_monitor_scratch), "cudaGetSymbolAddress");
        address[dev] = static_cast<unsigned char *>(p);
    }
    return address[dev];
}
} // namespace

nk_status nk_monitor_static(int64_t n, int64_t m, const double *x, const double *y,
                            const double *ax, const double *aty, const double *qx,
                            const double *c, const double *q, const double *lb, const double *ub,
                            const double *rl, const double *ru, double cscale, double *result,
                            void *stream) {
    return guard([&] {
        if (n < 0 || m < 0)
            throw nk::Error(NK_ERR_INVALID, "negative vector length");
        if (n > NK_MONITOR_STATIC_MAX || m > NK_MONITOR_STATIC_MAX)
            throw nk::Error(NK_ERR_INVALID,
                            "nk_monitor_static: n and m must be at most NK_MONITOR_STATIC_MAX "
                            "(4194304 entries); its fixed scratch holds no more block partials");
        if (!result || (n && (!x || !aty || !c || !q || !lb || !ub)) ||
            (m && (!y || !ax || !rl || !ru)))
            throw nk::Error(NK_ERR_INVALID, "null vector");
        auto s = static_cast<cudaStream_t>(stream);
        unsigned char *base = static_monitor_scratch();
        auto *arrive = reinterpret_cast<unsigned *>(base);
        auto *partial = reinterpret_cast<double *>(base + 256);
        const int64_t top = std::max(n, m);
        if (top == 0) {
            nk::cuda_check(cudaMemsetAsync(result, 0, sizeof(double), s), "result");
            return;
        }
        // the grid of nk_pdhg_monitor (the kernel is grid-stride): at most
        // 1184 blocks, whose partials the last block adds serially
        const int blocks = nk::grid_for(top);
        // a call that ended early must not leave a stale count behind
        nk::cuda_check(cudaMemsetAsync(arrive, 0, sizeof(unsigned), s), "clear counter");
        nk::monitor_kernel<<<blocks, nk::kThreads, 0, s>>>(n, m, x, y, ax, aty, qx, c, q, lb, ub,
                                                           rl, ru, cscale, partial, arrive, result);
        nk::cuda_check(cudaGetLastError(), "monitor launch");
    });
}

nk_status nk_pdhg_candidates(nk_pdhg *h, double *x, double *y, double *xa, double *ya) {
    return guard([&] {
        NK_HANDLE
        h->e->candidates(x, y, xa, ya);
    });
}
nk_status nk_pdhg_reset_candidate(nk_pdhg *h, int average) {
    return guard([&] {
        NK_HANDLE
        h->e->reset_candidate(average != 0);
    });
}
nk_status nk_pdhg_reset(nk_pdhg *h, const double *x, const double *y) {
    return guard([&] {
        NK_HANDLE
        if (h->e->n)
            need(x, "x");
        if (h->e->m)
            need(y, "y");
        h->e->reset(x, y);
    });
}
nk_status nk_pdhg_snapshot_layout(nk_pdhg *h, int *parts, int64_t *sizes) {
    return guard([&] {
        NK_HANDLE
        need(parts, "part count");
        auto L = h->e->layout();
        *parts = int(L.size());
        if (sizes)
            for (size_t i = 0; i < L.size(); ++i)
                sizes[i] = L[i];
    });
}
nk_status nk_pdhg_snapshot(nk_pdhg *h, double *out) {
    return guard([&] {
        NK_HANDLE
        need(out, "snapshot buffer");
        h->e->snapshot(out);
    });
}
nk_status nk_pdhg_restore(nk_pdhg *h, const double *in, const int64_t *sizes, int parts) {
    return guard([&] {
        NK_HANDLE
        need(in, "snapshot");
        need(sizes, "part sizes");
        h->e->restore(in, sizes, parts);
    });
}
nk_status nk_pdhg_stats(nk_pdhg *h, int64_t *trials, int64_t *bytes) {
    return guard([&] {
        NK_HANDLE
        if (trials)
            *trials = h->e->trials;
        if (bytes)
            *bytes = int64_t(h->e->device_bytes());
    });
}
nk_status nk_pdhg_profile(nk_pdhg *h, int count, double tau, double sigma, double *ms_primal,
                          double *ms_dual) {
    return guard([&] {
        NK_HANDLE
        need(ms_primal, "output");
        need(ms_dual, "output");
        h->e->profile(count, tau, sigma, ms_primal, ms_dual);
    });
}
nk_status nk_pdhg_profile_kernels(nk_pdhg *h, int count, double tau, double sigma,
                                  double ms[3]) {
    return guard([&] {
        NK_HANDLE
        need(ms, "output");
        double p = 0, d = 0, k = 0;
        h->e->profile(count, tau, sigma, &p, &d, &k);
        ms[0] = p;
        ms[1] = k;
        ms[2] = d - k;
    });
}
nk_status nk_pdhg_layout_info(nk_pdhg *h, int64_t *long_rows, int64_t *panel_width,
                              int *panels, int64_t *runs, int *kernels_per_trial) {
    return guard([&] {
        NK_HANDLE
        const auto &e = *h->e;
        if (long_rows)
            *long_rows = e.panels ? e.pan.rows : 0;
        if (panel_width)
            *panel_width = e.panels ? e.pan.width : 0;
        if (panels)
            *panels = e.panels ? e.pan.npanels : 0;
        if (runs)
            *runs = e.panels ? e.pan.slots : 0;
        if (kernels_per_trial)
            *kernels_per_trial = 2 + (e.panels ? 1 : 0) + (e.halpern ? 1 : 0);
    });
}
nk_status nk_pdhg_time_spmv(nk_pdhg *h, int which, int reps, double *ms) {
    return guard([&] {
        NK_HANDLE
        if (which != 0 && which != 1)
            throw nk::Error(NK_ERR_INVALID, "which must be 0 (A) or 1 (A^T)");
        need(ms, "output");
        *ms = h->e->time_spmv(which, reps);
    });
}
nk_status nk_pdhg_stream(nk_pdhg *h, void **stream) {
    return guard([&] {
        NK_HANDLE
        need(stream, "output");
        *stream = reinterpret_cast<void *>(h->e->stream);
    });
}
nk_status nk_pdhg_schedule_info(nk_pdhg *h, int *a_width, int64_t *a_long, int *at_width,
                                int64_t *at_long, int *a_items, int *at_items) {
    return guard([&] {
        NK_HANDLE
        // SELL-32: one lane per row; reported: lanes per row, split length,
        // chunks.  Null outputs are skipped.
        auto put = [](auto *dst, auto v) {
            if (dst)
                *dst = v;
        };
        put(a_width, 1);
        put(a_long, int64_t(NK_SPLIT));
        put(at_width, 1);
        put(at_long, int64_t(NK_SPLIT));
        put(a_items, int((h->e->A.nv + 31) / 32));
        put(at_items, int((h->e->At.nv + 31) / 32));
    });
}
int nk_cuda_available(void) {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}
nk_status nk_cuda_description(char *buffer, int length) {
    return guard([&] {
        if (!buffer || length <= 0)
            throw nk::Error(NK_ERR_INVALID, "null buffer");
        if (!nk_cuda_available()) {
            std::snprintf(buffer, size_t(length), "No CUDA device");
            return;
        }
        cudaDeviceProp p{};
        nk::cuda_check(cudaGetDeviceProperties(&p, 0), "GPU properties");
        std::snprintf(buffer, size_t(length), "%s (%zu MiB)", p.name,
                      size_t(p.totalGlobalMem / (1024 * 1024)));
    });
}
nk_status nk_compact_csr(const nk_csr *matrix, int64_t rows, const int64_t *kept_rows,
                         const int64_t *column_map, int64_t output_columns, int64_t *out_ptr,
                         int64_t *out_index, double *out_value, int64_t capacity,
                         int64_t *out_nnz) {
    return guard([&] {
        if (!matrix || !out_ptr || !out_nnz || (rows > 0 && !kept_rows) ||
            (matrix->cols > 0 && !column_map) || rows < 0 || capacity < 0 || output_columns < 0)
            throw nk::Error(NK_ERR_INVALID, "invalid compaction arguments");
        nk::validate_csr(matrix, matrix->rows, matrix->cols, "compaction");
        const int64_t nnz = matrix->ptr[matrix->rows];
        for (int64_t k = 0; k < nnz; ++k)
            if (matrix->index[k] < 0 || matrix->index[k] >= matrix->cols)
                throw nk::Error(NK_ERR_INVALID, "compaction column index out of range");
        int64_t previous = -1;
        for (int64_t r = 0; r < rows; ++r) {
            if (kept_rows[r] <= previous || kept_rows[r] >= matrix->rows)
                throw nk::Error(NK_ERR_INVALID, "compaction row map");
            previous = kept_rows[r];
        }
        previous = -1;
        for (int64_t j = 0; j < matrix->cols; ++j) {
            const int64_t c = column_map[j];
            if (c < -1 || (c >= 0 && (c <= previous || c >= output_columns)))
                throw nk::Error(NK_ERR_INVALID, "compaction column map");
            if (c >= 0)
                previous = c;
        }
        if (capacity > 0 && (!out_index || !out_value))
            throw nk::Error(NK_ERR_INVALID, "null compaction output");
        if (!nk_cuda_available())
            throw nk::Error(NK_ERR_NO_DEVICE, "no CUDA device");
        *out_nnz = nk::compact_csr(*matrix, rows, kept_rows, column_map, out_ptr, out_index,
                                   out_value, capacity);
    });
}

nk_status nk_propagate_bounds(const nk_csr *A, const int *integer, const double *rl,
                              const double *ru, double *lb, double *ub, int passes,
                              int *feasible) {
    return guard([&] {
        if (!A || !feasible || !rl || !ru || (A->cols > 0 && (!integer || !lb || !ub)) ||
            passes < 0 || passes > 100)
            throw nk::Error(NK_ERR_INVALID, "invalid propagation arguments");
        nk::validate_csr(A, A->rows, A->cols, "propagation");
        const int64_t nnz = A->ptr[A->rows];
        for (int64_t k = 0; k < nnz; ++k)
            if (A->index[k] < 0 || A->index[k] >= A->cols)
                throw nk::Error(NK_ERR_INVALID, "propagation column index out of range");
        for (int64_t j = 0; j < A->cols; ++j)
            if (std::isnan(lb[j]) || std::isnan(ub[j]) || lb[j] > ub[j])
                throw nk::Error(NK_ERR_INVALID, "invalid propagation bounds");
        if (A->rows > 0 && passes > 0 && !nk_cuda_available())
            throw nk::Error(NK_ERR_NO_DEVICE, "no CUDA device");
        *feasible = nk::propagate_bounds(*A, integer, rl, ru, lb, ub, passes) ? 1 : 0;
    });
}

nk_status nk_linear_solve(const nk_csr *K, const double *rhs, int fp32_matrix, int precondition,
                          double time_limit, double *x, int *converged, int *timed_out) {
    return guard([&] {
        if (!K || !converged || !timed_out || K->rows != K->cols || K->rows < 0 ||
            (K->rows > 0 && (!rhs || !x)) || !(time_limit >= 0))
            throw nk::Error(NK_ERR_INVALID, "Newton matrix dimensions");
        nk::validate_csr(K, K->rows, K->cols, "Newton");
        const int64_t nnz = K->ptr[K->rows];
        for (int64_t k = 0; k < nnz; ++k)
            if (K->index[k] < 0 || K->index[k] >= K->cols)
                throw nk::Error(NK_ERR_INVALID, "Newton column index out of range");
        *converged = 1;
        *timed_out = 0;
        if (K->rows == 0)
            return;
        if (!nk_cuda_available())
            throw nk::Error(NK_ERR_NO_DEVICE, "no CUDA device");
        bool late = false;
        *converged = nk::newton_solve(*K, rhs, fp32_matrix != 0, precondition != 0, time_limit, x,
                                      &late) ? 1 : 0;
        *timed_out = late ? 1 : 0;
    });
}

nk_status nk_hardware_info(int *available, double *free_bytes, double *total_bytes) {
    return guard([&] {
        const int present = nk_cuda_available();
        size_t f = 0, t = 0;
        if (present && cudaMemGetInfo(&f, &t) != cudaSuccess)
            f = t = 0;
        if (available)
            *available = present;
        if (free_bytes)
            *free_bytes = double(f);
        if (total_bytes)
            *total_bytes = double(t);
    });
}

struct nk_prepared {
    nk::Prepared p;
};

nk_status nk_prepare(const nk_model *model, int presolve, int scaling_combined, int scaling_passes,
                     nk_prepared **out) {
    return guard([&] {
        if (!out)
            throw nk::Error(NK_ERR_INVALID, "null output handle");
        *out = nullptr;
        if (scaling_passes < 0)
            throw nk::Error(NK_ERR_INVALID, "negative scaling passes");
        nk::HostModel hm = nk::host_model(model);
        nk::PrepareOptions po;
        po.presolve = presolve != 0;
        po.scaling = scaling_combined ? "combined" : "ruiz";
        po.scaling_passes = scaling_passes;
        auto h = std::make_unique<nk_prepared>();
        h->p = nk::prepare(hm, po);
        *out = h.release();
    });
}
void nk_prepared_free(nk_prepared *p) { delete p; }
nk_status nk_prepared_dims(const nk_prepared *h, int64_t dims[5]) {
    return guard([&] {
        if (!h || !dims)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        const auto &m = h->p.model;
        dims[0] = int64_t(m.rl.size());
        dims[1] = int64_t(m.c.size());
        dims[2] = int64_t(m.A.value.size());
        dims[3] = int64_t(m.Q.value.size());
        dims[4] = h->p.failure.empty() ? 0 : 1;
    });
}
nk_status nk_prepared_get(const nk_prepared *h, int64_t *ptr, int64_t *index, double *value,
                          double *c, double *q, double *lb, double *ub, double *rl, double *ru,
                          int64_t *cols, int64_t *rows, int64_t *lower_rows, int64_t *upper_rows,
                          double *fixed, double *column_scale, double *row_scale, double *scalars,
                          int64_t *qptr, int64_t *qindex, double *qvalue) {
    return guard([&] {
        if (!h)
            throw nk::Error(NK_ERR_INVALID, "null handle");
        const auto &p = h->p;
        const auto &m = p.model;
        auto put = [](auto *dst, const auto &v) {
            if (dst && !v.empty())
                std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
        };
        put(ptr, m.A.ptr);
        put(index, m.A.index);
        put(value, m.A.value);
        put(c, m.c);
        put(q, m.q);
        put(lb, m.lb);
        put(ub, m.ub);
        put(rl, m.rl);
        put(ru, m.ru);
        put(cols, p.cols);
        put(rows, p.rows);
        put(lower_rows, p.lower_rows);
        put(upper_rows, p.upper_rows);
        put(fixed, p.fixed);
        put(column_scale, p.column_scale);
        put(row_scale, p.row_scale);
        if (scalars) {
            scalars[0] = p.objective_scale;
            scalars[1] = m.offset;
        }
        put(qptr, m.Q.ptr);
        put(qindex, m.Q.index);
        put(qvalue, m.Q.value);
    });
}
nk_status nk_verify(const nk_model *model, const double *x, const double *y, int safe_bound,
                    double accuracy[10]) {
    return guard([&] {
        if (!x || !y || !accuracy)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        nk::HostModel hm = nk::host_model(model);
        nk::Verifier v(hm);
        auto a = v.evaluate(std::vector<double>(x, x + hm.c.size()),
                            std::vector<double>(y, y + hm.rl.size()), safe_bound != 0);
        const double s[10] = {a.objective,       a.primal,          a.dual,   a.gap,
                              a.kkt,             a.primal_absolute, a.dual_absolute,
                              a.complementarity, a.lower_bound,     a.finite ? 1.0 : 0.0};
        std::memcpy(accuracy, s, sizeof(s));
    });
}
nk_status nk_infeasibility_bound(const nk_model *model, const double *y, double *bound) {
    return guard([&] {
        if (!y || !bound)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        nk::HostModel hm = nk::host_model(model);
        *bound = nk::Verifier(hm).infeasibility_bound(std::vector<double>(y, y + hm.rl.size()));
    });
}

void nk_solve_defaults(nk_solve_options *o) {
    if (!o)
        return;
    *o = nk_solve_options{};
    o->tol = 1e-6;
    o->time_limit = 60;
    o->iteration_limit = 100000;
    o->check_every = 100;
    o->presolve = 1;
    o->scaling_passes = 5;
    o->adaptive = 1;
    o->restart = 1;
    o->graphs = 1;
    o->precision = NK_PRECISION_FP64;
    o->refine = 1;
}

nk_status nk_solve(const nk_model *model, const nk_solve_options *o, nk_solve_result *result,
                   double *x, double *y) {
    return guard([&] {
        if (!o || !result)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        nk::HostModel hm = nk::host_model(model);
        const int64_t m = model->A.rows, n = model->A.cols;
        if (!(o->tol > 0) || o->check_every <= 0 || o->iteration_limit < 0 || !(o->time_limit >= 0) ||
            o->scaling_passes < 0 || o->precision < 0 || o->precision > 2)
            throw nk::Error(NK_ERR_INVALID, "invalid solve options");
        nk::SolveSettings S;
        S.driver.tol = o->tol;
        S.driver.time_limit = o->time_limit;
        S.driver.iteration_limit = o->iteration_limit;
        S.driver.check_every = o->check_every;
        S.driver.adaptive = o->adaptive != 0;
        S.driver.restart = o->restart != 0;
        S.driver.graphs = o->graphs != 0;
        S.driver.index_bits = o->index_bits;
        S.driver.verbose = o->verbose != 0;
        S.driver.cancel = o->cancel;
        S.prepare.presolve = o->presolve != 0;
        S.prepare.scaling = o->scaling_combined ? "combined" : "ruiz";
        S.prepare.scaling_passes = o->scaling_passes;
        S.precision = o->precision;
        S.refine = o->refine != 0;
        S.phase_tol = o->phase_tol;
        if (o->initial_x)
            S.initial_x.assign(o->initial_x, o->initial_x + n);
        if (o->initial_y)
            S.initial_y.assign(o->initial_y, o->initial_y + m);
        nk::SolveReport R = nk::solve(hm, S);
        nk_solve_result &r = *result;
        r = nk_solve_result{};
        r.status = R.status;
        r.iterations = R.iterations;
        r.restarts = R.restarts;
        r.rejected_steps = R.rejected;
        r.weight_updates = R.weight_updates;
        r.device_checks = R.device_checks;
        r.host_checks = R.host_checks;
        r.removed_rows = R.removed_rows;
        r.removed_columns = R.removed_columns;
        r.phase_iterations = R.mixed_iterations;
        r.refine_iterations = R.refine_iterations;
        r.seconds = R.seconds;
        r.preprocess_seconds = R.preprocess;
        r.transfer_seconds = R.transfer;
        r.iteration_seconds = R.iteration;
        r.verification_seconds = R.verification;
        r.phase_seconds = R.mixed_seconds;
        r.objective = R.accuracy.objective;
        r.kkt = R.accuracy.kkt;
        r.primal = R.accuracy.primal;
        r.dual = R.accuracy.dual;
        r.gap = R.accuracy.gap;
        r.lower_bound = R.accuracy.lower_bound;
        r.phase_objective = R.mixed.objective;
        r.phase_kkt = R.mixed.kkt;
        r.phase_primal = R.mixed.primal;
        r.phase_dual = R.mixed.dual;
        r.phase_gap = R.mixed.gap;
        for (int k = 0; k < 9; ++k)
            r.reached[k] = R.reached[k];
        if (x && R.x.size() == size_t(n))
            std::memcpy(x, R.x.data(), size_t(n) * 8);
        if (y && R.y.size() == size_t(m))
            std::memcpy(y, R.y.data(), size_t(m) * 8);
    });
}

// ------------------------------------------------------------------ batch
struct nk_batch {
    nk::Batch b;
    explicit nk_batch(const nk::BatchOptions &o) : b(o) {}
};
struct nk_batch_item {
    std::unique_ptr<nk::BatchItem> item;
};

void nk_batch_defaults(nk_batch_options *o) {
    if (!o)
        return;
    *o = nk_batch_options{};
    o->tol = 1e-6;
    o->time_limit = 60;
    o->iteration_limit = 100000;
    o->check_every = 100;
    o->presolve = 1;
    o->scaling_passes = 5;
    o->adaptive = 1;
    o->restart = 1;
    o->graphs = 1;
    o->autotune = 1;
    // FP64: on the 512-instance uneven LP/QP batch it certified more instances per second
    // than MIXED (318 against 310 OPTIMAL of 512 at the 100,000-iteration cap, in less time):
    // the reduced-precision phase and the refinement restarted after it cost iterations
    o->precision = NK_PRECISION_FP64;
    o->capacity = 4096;
}

static nk::BatchOptions batch_options(const nk_batch_options *o) {
    if (!o)
        throw nk::Error(NK_ERR_INVALID, "null batch options");
    if (!(o->tol > 0) || o->check_every <= 0 || o->iteration_limit < 0 || !(o->time_limit >= 0) ||
        o->scaling_passes < 0 || o->precision < 0 || o->precision > 2 || o->memory_budget < 0)
        throw nk::Error(NK_ERR_INVALID, "invalid batch options");
    nk::BatchOptions b;
    b.tol = o->tol;
    b.time_limit = o->time_limit;
    b.iteration_limit = o->iteration_limit;
    b.check_every = o->check_every;
    b.prepare.presolve = o->presolve != 0;
    b.prepare.scaling = o->scaling_combined ? "combined" : "ruiz";
    b.prepare.scaling_passes = o->scaling_passes;
    b.adaptive = o->adaptive != 0;
    b.restart = o->restart != 0;
    b.graphs = o->graphs != 0;
    b.autotune = o->autotune != 0;
    b.precision = o->precision;
    b.phase_tol = o->phase_tol;
    b.memory_budget = o->memory_budget;
    b.capacity = o->capacity;
    return b;
}

nk_status nk_batch_create(const nk_batch_options *o, nk_batch **out) {
    return guard([&] {
        if (!out)
            throw nk::Error(NK_ERR_INVALID, "null output handle");
        *out = nullptr;
        *out = new nk_batch(batch_options(o));
    });
}
void nk_batch_destroy(nk_batch *h) { delete h; }

nk_status nk_batch_estimate(const nk_model *model, double *bytes) {
    return guard([&] {
        if (!bytes)
            throw nk::Error(NK_ERR_INVALID, "null output");
        *bytes = nk::batch_estimate(nk::host_model(model));
    });
}

nk_status nk_batch_prepare(const nk_model *model, const nk_batch_options *o, nk_batch_item **out,
                           double *device_bytes) {
    return guard([&] {
        if (!out)
            throw nk::Error(NK_ERR_INVALID, "null output handle");
        *out = nullptr;
        auto opts = batch_options(o);
        auto item = std::make_unique<nk_batch_item>();
        // requests are prepared concurrently, one per host thread
        nk::HostSerialScope serial;
        item->item = nk::batch_prepare(nk::host_model(model), opts);
        if (device_bytes)
            *device_bytes = item->item->decided ? 0. : double(item->item->bytes);
        *out = item.release();
    });
}
nk_status nk_batch_prepare_from(const nk_model *model, const nk_batch_options *o,
                                const double *x0, const double *y0, nk_batch_item **out,
                                double *device_bytes) {
    return guard([&] {
        if (!out)
            throw nk::Error(NK_ERR_INVALID, "null output handle");
        *out = nullptr;
        auto opts = batch_options(o);
        // requests are prepared concurrently, one per host thread
        nk::HostSerialScope serial;
        auto host = nk::host_model(model);
        std::vector<double> x, y;
        if (x0)
            x.assign(x0, x0 + host.c.size());
        if (y0)
            y.assign(y0, y0 + host.rl.size());
        auto item = std::make_unique<nk_batch_item>();
        item->item = nk::batch_prepare(host, opts, x0 ? &x : nullptr, y0 ? &y : nullptr);
        if (device_bytes)
            *device_bytes = item->item->decided ? 0. : double(item->item->bytes);
        *out = item.release();
    });
}
void nk_batch_item_free(nk_batch_item *item) { delete item; }

nk_status nk_batch_admit(nk_batch *h, nk_batch_item *item, int64_t id, int *admitted) {
    return guard([&] {
        if (!h || !item || !item->item || !admitted)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        *admitted = h->b.admit(item->item, id) ? 1 : 0;
        if (*admitted)
            delete item;
    });
}

nk_status nk_batch_step(nk_batch *h, int checks, int64_t *finished, int capacity, int *count) {
    return guard([&] {
        if (!h || !count || checks < 0 || capacity < 0 || (capacity && !finished))
            throw nk::Error(NK_ERR_INVALID, "invalid argument");
        auto done = h->b.step(checks);
        if (int(done.size()) > capacity)
            throw nk::Error(NK_ERR_INVALID, "finished-id buffer too small");
        for (size_t k = 0; k < done.size(); ++k)
            finished[k] = done[k];
        *count = int(done.size());
    });
}

nk_status nk_batch_result(nk_batch *h, int64_t id, nk_solve_result *result, double *x, double *y) {
    return guard([&] {
        if (!h || !result)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        nk::SolveReport R = h->b.take(id);
        nk_solve_result &r = *result;
        r = nk_solve_result{};
        r.status = R.status;
        r.iterations = R.iterations;
        r.restarts = R.restarts;
        r.rejected_steps = R.rejected;
        r.weight_updates = R.weight_updates;
        r.device_checks = R.device_checks;
        r.host_checks = R.host_checks;
        r.removed_rows = R.removed_rows;
        r.removed_columns = R.removed_columns;
        r.preprocess_seconds = R.preprocess;
        r.transfer_seconds = R.transfer;
        r.iteration_seconds = R.iteration;
        r.verification_seconds = R.verification;
        r.seconds = R.preprocess + R.transfer + R.iteration + R.verification;
        r.objective = R.accuracy.objective;
        r.kkt = R.accuracy.kkt;
        r.primal = R.accuracy.primal;
        r.dual = R.accuracy.dual;
        r.gap = R.accuracy.gap;
        r.lower_bound = R.accuracy.lower_bound;
        r.phase_iterations = R.mixed_iterations;
        r.refine_iterations = R.refine_iterations;
        r.phase_objective = R.mixed.objective;
        r.phase_kkt = R.mixed.kkt;
        r.phase_primal = R.mixed.primal;
        r.phase_dual = R.mixed.dual;
        r.phase_gap = R.mixed.gap;
        for (int k = 0; k < 9; ++k)
            r.reached[k] = R.reached[k];
        if (x && !R.x.empty())
            std::memcpy(x, R.x.data(), R.x.size() * 8);
        if (y && !R.y.empty())
            std::memcpy(y, R.y.data(), R.y.size() * 8);
    });
}

nk_status nk_batch_info(nk_batch *h, int *active, double *used_bytes, double *budget_bytes,
                        int *variant_primal, int *variant_dual) {
    return guard([&] {
        if (!h)
            throw nk::Error(NK_ERR_INVALID, "null handle");
        if (active)
            *active = h->b.active();
        if (used_bytes)
            *used_bytes = h->b.used();
        if (budget_bytes)
            *budget_bytes = h->b.budget();
        if (variant_primal)
            *variant_primal = h->b.variant_primal();
        if (variant_dual)
            *variant_dual = h->b.variant_dual();
    });
}

nk_status nk_batch_progress(nk_batch *h, int64_t id, double progress[8]) {
    return guard([&] {
        if (!h || !progress)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        h->b.progress(id, progress);
    });
}
nk_status nk_batch_phase_seconds(nk_batch *h, double seconds[7]) {
    return guard([&] {
        if (!h || !seconds)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        std::memcpy(seconds, h->b.phase_seconds(), 7 * sizeof(double));
    });
}
nk_status nk_batch_kernel_times(nk_batch *h, double *primal_ms, double *dual_ms) {
    return guard([&] {
        if (!h || !primal_ms || !dual_ms)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        *primal_ms = h->b.tuned_ms_primal();
        *dual_ms = h->b.tuned_ms_dual();
    });
}
nk_status nk_batch_time_trials(nk_batch *h, int trials, double *ms, int64_t *bytes_per_trial) {
    return guard([&] {
        if (!h || !ms || trials < 0)
            throw nk::Error(NK_ERR_INVALID, "invalid argument");
        *ms = h->b.time_trials(trials);
        if (bytes_per_trial)
            *bytes_per_trial = h->b.matrix_bytes_per_trial();
    });
}
}
