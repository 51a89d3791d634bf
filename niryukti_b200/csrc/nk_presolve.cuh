// Device side of the reference's GPU presolve (--gpu-presolve):
//   compact_csr      cuda_compact_matrix (src/cuda.cu:953-1032): the CSR of the
//                    kept rows with their kept columns renumbered, entries in
//                    their original order (an exact, integer/byte operation).
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

} // namespace nk
