// Device side of the reference's GPU presolve (--gpu-presolve):
//   compact_csr      cuda_compact_matrix (src/cuda.cu:953-1032): the CSR of the
//                    kept rows with their kept columns renumbered, entries in
//                    their original order (an exact, integer/byte operation).
//   propagate_bounds cuda_propagate_integer_bounds (src/cuda.cu:448-529,
//                    1033-1135): activity-based bound proposals with directed
//                    rounding, integer columns rounded inward.  Proposals only:
//                    the reference's host replays them with outward-rounded
//                    proofs before any is used.
// Included by nk_engine.cu.
#pragma once
#include "nk_common.cuh"
#include "nk_kernels.cuh"
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

namespace nk {

// One warp per output row: the number of the source row's entries whose column
// is kept (lane-strided over the row, coalesced; a fixed shuffle tree).
__global__ void compact_count(int64_t rows, const int64_t *__restrict__ kept,
                              const int64_t *__restrict__ ptr, const int64_t *__restrict__ index,
                              const int64_t *__restrict__ map, int64_t *__restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t stride = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t r = first; r < rows; r += stride) {
        const int64_t i = kept[r], b = ptr[i], e = ptr[i + 1];
        int64_t c = 0;
        for (int64_t k = b + lane; k < e; k += 32)
            c += map[index[k]] >= 0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            c += __shfl_xor_sync(0xffffffffu, c, off);
        if (lane == 0)
            counts[r] = c;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        counts[rows] = 0; // the exclusive scan over rows + 1 counts ends in the total
}

// One warp per output row: 32 entries at a time, the kept ones are written in
// order at the row's offset (ballot + prefix popcount), so reads and writes
// stay coalesced and the entry order is the source order.
__global__ void compact_scatter(int64_t rows, const int64_t *__restrict__ kept,
                                const int64_t *__restrict__ ptr,
                                const int64_t *__restrict__ index,
                                const double *__restrict__ value,
                                const int64_t *__restrict__ map,
                                const int64_t *__restrict__ out_ptr,
                                int64_t *__restrict__ out_index, double *__restrict__ out_value) {
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t stride = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t r = first; r < rows; r += stride) {
        const int64_t i = kept[r], b = ptr[i], e = ptr[i + 1];
        int64_t dest = out_ptr[r];
        for (int64_t k0 = b; k0 < e; k0 += 32) { // warp-uniform bounds
            const int64_t k = k0 + lane;
            int64_t col = -1;
            double v = 0;
            if (k < e) {
                col = map[index[k]];
                v = value[k];
            }
            const unsigned keep = __ballot_sync(0xffffffffu, col >= 0);
            if (col >= 0) {
                const int64_t at = dest + __popc(keep & below);
                out_index[at] = col;
                out_value[at] = v;
            }
            dest += __popc(keep);
        }
    }
}

// Host driver: uploads the source CSR and the maps, counts, scans, scatters and
// copies the result into the caller's arrays (out_ptr: rows + 1 entries;
// out_index / out_value: `capacity` entries).  Returns the kept entries.  The
// arguments are checked by the caller.
inline int64_t compact_csr(const nk_csr &M, int64_t rows, const int64_t *kept, const int64_t *map,
                           int64_t *out_ptr, int64_t *out_index, double *out_value,
                           int64_t capacity) {
    cudaStream_t s = nullptr;
    cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "compaction stream");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard_stream{s};
    const int64_t nnz = M.ptr[M.rows];
    DevBuf<int64_t> dptr(size_t(M.rows + 1)), didx(size_t(std::max<int64_t>(1, nnz))),
        dkept(size_t(std::max<int64_t>(1, rows))), dmap(size_t(std::max<int64_t>(1, M.cols))),
        counts(size_t(rows + 1)), optr(size_t(rows + 1));
    DevBuf<double> dval(size_t(std::max<int64_t>(1, nnz)));
    auto up = [&](void *d, const void *h, size_t bytes) {
        if (bytes)
            cuda_check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s), "compaction upload");
    };
    up(dptr.p, M.ptr, size_t(M.rows + 1) * 8);
    up(didx.p, M.index, size_t(nnz) * 8);
    up(dval.p, M.value, size_t(nnz) * 8);
    up(dkept.p, kept, size_t(rows) * 8);
    up(dmap.p, map, size_t(M.cols) * 8);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = int(std::max<int64_t>(1, std::min<int64_t>((rows + kWarps - 1) / kWarps,
                                                                int64_t(sms) * 8)));
    compact_count<<<grid, kThreads, 0, s>>>(rows, dkept.p, dptr.p, didx.p, dmap.p, counts.p);
    cuda_check(cudaGetLastError(), "compaction count");
    size_t temp = 0;
    cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, temp, counts.p, optr.p, rows + 1, s),
               "compaction scan size");
    DevBuf<unsigned char> work(std::max<size_t>(1, temp));
    cuda_check(cub::DeviceScan::ExclusiveSum(work.p, temp, counts.p, optr.p, rows + 1, s),
               "compaction scan");
    cuda_check(cudaMemcpyAsync(out_ptr, optr.p, size_t(rows + 1) * 8, cudaMemcpyDeviceToHost, s),
               "compaction offsets");
    cuda_check(cudaStreamSynchronize(s), "compaction offsets");
    const int64_t total = out_ptr[rows];
    if (total > capacity)
        throw Error(NK_ERR_INVALID, "compaction output capacity is too small");
    if (total) {
        DevBuf<int64_t> oidx(static_cast<size_t>(total));
        DevBuf<double> oval(static_cast<size_t>(total));
        compact_scatter<<<grid, kThreads, 0, s>>>(rows, dkept.p, dptr.p, didx.p, dval.p, dmap.p,
                                                  optr.p, oidx.p, oval.p);
        cuda_check(cudaGetLastError(), "compaction scatter");
        cuda_check(cudaMemcpyAsync(out_index, oidx.p, size_t(total) * 8, cudaMemcpyDeviceToHost, s),
                   "compaction indices");
        cuda_check(cudaMemcpyAsync(out_value, oval.p, size_t(total) * 8, cudaMemcpyDeviceToHost, s),
                   "compaction values");
        cuda_check(cudaStreamSynchronize(s), "compaction completion");
    }
    return total;
}

// ---------------------------------------------------------------- bound propagation
// new = max(new, v) / min(new, v) for doubles, by compare-and-swap: the result
// is the extreme proposal whatever the order the rows arrive in.
__device__ __forceinline__ void propose_lower(double *address, double value) {
    auto *bits = reinterpret_cast<unsigned long long *>(address);
    unsigned long long old = *reinterpret_cast<volatile unsigned long long *>(bits);
    while (value > __longlong_as_double((long long)old)) {
        const unsigned long long seen =
            atomicCAS(bits, old, (unsigned long long)__double_as_longlong(value));
        if (seen == old)
            break;
        old = seen;
    }
}
__device__ __forceinline__ void propose_upper(double *address, double value) {
    auto *bits = reinterpret_cast<unsigned long long *>(address);
    unsigned long long old = *reinterpret_cast<volatile unsigned long long *>(bits);
    while (value < __longlong_as_double((long long)old)) {
        const unsigned long long seen =
            atomicCAS(bits, old, (unsigned long long)__double_as_longlong(value));
        if (seen == old)
            break;
        old = seen;
    }
}

// One pass over the rows, one thread per row (a row's activity bounds are
// sums in the row's entry order with directed rounding, so they are not split
// across lanes).  Reads the bounds of the previous pass (lb, ub) and proposes
// into new_lb / new_ub; flags a row whose activity range misses [rl, ru].
__global__ void propagate_rows(int64_t rows, const int64_t *__restrict__ ptr,
                               const int64_t *__restrict__ index, const double *__restrict__ a,
                               const int *__restrict__ integer, const double *__restrict__ lb,
                               const double *__restrict__ ub, const double *__restrict__ rl,
                               const double *__restrict__ ru, double *new_lb, double *new_ub,
                               int *failed) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t row = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; row < rows; row += stride) {
        const int64_t b = ptr[row], e = ptr[row + 1];
        double low = 0, high = 0;
        int low_inf = 0, high_inf = 0;
        for (int64_t k = b; k < e; ++k) {
            const double v = a[k];
            if (v == 0)
                continue;
            const int64_t j = index[k];
            const double lo = __dmul_rd(v, v > 0 ? lb[j] : ub[j]);
            const double hi = __dmul_ru(v, v > 0 ? ub[j] : lb[j]);
            if (isinf(lo))
                ++low_inf;
            else
                low = __dadd_rd(low, lo);
            if (isinf(hi))
                ++high_inf;
            else
                high = __dadd_ru(high, hi);
        }
        const double rlo = rl[row], rhi = ru[row];
        if ((!low_inf && low > rhi) || (!high_inf && high < rlo))
            atomicExch(failed, 1);
        for (int64_t k = b; k < e; ++k) {
            const double v = a[k];
            if (v == 0)
                continue;
            const int64_t j = index[k];
            const double end_low = v > 0 ? lb[j] : ub[j], end_high = v > 0 ? ub[j] : lb[j];
            const double term_low = __dmul_rd(v, end_low), term_high = __dmul_ru(v, end_high);
            // the rest of the row: removing a term needs the opposite rounding
            const double rest_low = low_inf - int(isinf(term_low)) ? -INFINITY
                                    : isinf(term_low)              ? low
                                                : __dsub_rd(low, __dmul_ru(v, end_low));
            const double rest_high = high_inf - int(isinf(term_high)) ? INFINITY
                                     : isinf(term_high)               ? high
                                                : __dsub_ru(high, __dmul_rd(v, end_high));
            double l = -INFINITY, u = INFINITY;
            if (isfinite(rlo) && isfinite(rest_high)) {
                const double num = __dsub_rd(rlo, rest_high);
                if (v > 0)
                    l = __ddiv_rd(num, v);
                else
                    u = __ddiv_ru(num, v);
            }
            if (isfinite(rhi) && isfinite(rest_low)) {
                const double num = __dsub_ru(rhi, rest_low);
                if (v > 0)
                    u = __ddiv_ru(num, v);
                else
                    l = __ddiv_rd(num, v);
            }
            const bool whole = integer[j] != 0;
            if (isfinite(l) && (!whole || fabs(l) < 0x1p52))
                propose_lower(new_lb + j, whole ? ceil(l) : l);
            if (isfinite(u) && (!whole || fabs(u) < 0x1p52))
                propose_upper(new_ub + j, whole ? floor(u) : u);
        }
    }
}

// `passes` propagation passes over A (host arrays in, lb / ub updated in
// place).  Returns false when some row's activity range misses its bounds or a
// column's bounds cross.  The arguments are checked by the caller.
inline bool propagate_bounds(const nk_csr &A, const int *integer, const double *rl,
                             const double *ru, double *lb, double *ub, int passes) {
    const int64_t n = A.cols, m = A.rows, nnz = A.ptr[A.rows];
    if (m == 0 || passes == 0)
        return true;
    cudaStream_t s = nullptr;
    cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "propagation stream");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard_stream{s};
    const size_t nb = size_t(std::max<int64_t>(1, n));
    DevBuf<int64_t> dptr(size_t(m + 1)), didx(size_t(std::max<int64_t>(1, nnz)));
    DevBuf<double> dval(static_cast<size_t>(std::max<int64_t>(1, nnz))),
        drl(static_cast<size_t>(m)), dru(static_cast<size_t>(m));
    DevBuf<double> olb(nb), oub(nb), nlb(nb), nub(nb);
    DevBuf<int> dint(nb), dfail(1);
    auto up = [&](void *d, const void *h, size_t bytes) {
        if (bytes)
            cuda_check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s), "propagation upload");
    };
    up(dptr.p, A.ptr, size_t(m + 1) * 8);
    up(didx.p, A.index, size_t(nnz) * 8);
    up(dval.p, A.value, size_t(nnz) * 8);
    up(drl.p, rl, size_t(m) * 8);
    up(dru.p, ru, size_t(m) * 8);
    up(dint.p, integer, size_t(n) * sizeof(int));
    up(olb.p, lb, size_t(n) * 8);
    up(oub.p, ub, size_t(n) * 8);
    up(nlb.p, lb, size_t(n) * 8);
    up(nub.p, ub, size_t(n) * 8);
    cuda_check(cudaMemsetAsync(dfail.p, 0, sizeof(int), s), "propagation flag");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = int(std::max<int64_t>(1, std::min<int64_t>((m + kThreads - 1) / kThreads,
                                                                int64_t(sms) * 8)));
    for (int pass = 0; pass < passes; ++pass) {
        propagate_rows<<<grid, kThreads, 0, s>>>(m, dptr.p, didx.p, dval.p, dint.p, olb.p, oub.p,
                                                 drl.p, dru.p, nlb.p, nub.p, dfail.p);
        cuda_check(cudaGetLastError(), "propagation pass");
        cuda_check(cudaMemcpyAsync(olb.p, nlb.p, size_t(n) * 8, cudaMemcpyDeviceToDevice, s),
                   "propagation lower");
        cuda_check(cudaMemcpyAsync(oub.p, nub.p, size_t(n) * 8, cudaMemcpyDeviceToDevice, s),
                   "propagation upper");
    }
    int failed = 0;
    cuda_check(cudaMemcpyAsync(&failed, dfail.p, sizeof(int), cudaMemcpyDeviceToHost, s),
               "propagation flag");
    cuda_check(cudaMemcpyAsync(lb, nlb.p, size_t(n) * 8, cudaMemcpyDeviceToHost, s),
               "propagation lower");
    cuda_check(cudaMemcpyAsync(ub, nub.p, size_t(n) * 8, cudaMemcpyDeviceToHost, s),
               "propagation upper");
    cuda_check(cudaStreamSynchronize(s), "propagation completion");
    if (failed)
        return false;
    for (int64_t j = 0; j < n; ++j)
        if (lb[j] > ub[j])
            return false;
    return true;
}

} // namespace nk
