// scan.cu -- exclusive prefix sum over int arrays (reduce, scan of block
// sums, downsweep), used to compact force tiles and contact cells.
#include "sfg_internal.h"

namespace sfg {

constexpr int SCAN_B = 1024;  // elements per block (256 threads x 4)

__device__ __forceinline__ int block_excl_scan(int v, int* sh) {
    // 256 threads: warp inclusive scans, then scan of warp totals
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        sh[lane] = t;
    }
    __syncthreads();
    const int base = wid > 0 ? sh[wid - 1] : 0;
    const int res = base + x - v;
    __syncthreads();
    return res;
}

__global__ void k_scan_reduce(const int* __restrict__ in, int n, int* __restrict__ sums) {
    __shared__ int sh[32];
    const int b0 = blockIdx.x * SCAN_B;
    int s = 0;
    for (int i = threadIdx.x; i < SCAN_B; i += blockDim.x) {
        const int g = b0 + i;
        if (g < n) s += in[g];
    }
    // block reduce
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        int t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = t;
    }
}

// Single block: exclusive scan of nb block sums in place; writes the total.
__global__ void k_scan_sums(int* __restrict__ sums, int nb, int* __restrict__ total) {
    __shared__ int sh[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? sums[i] : 0;
        const int ex = block_excl_scan(v, sh);
        if (i < nb) sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += ex + v;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void k_scan_down(const int* __restrict__ in, int n, const int* __restrict__ sums,
                            int* __restrict__ out) {
    __shared__ int sh[32];
    const int b0 = blockIdx.x * SCAN_B;
    // each thread owns 4 consecutive elements
    const int i0 = b0 + threadIdx.x * 4;
    int v[4], s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = (i0 + k < n) ? in[i0 + k] : 0;
        s += v[k];
    }
    int ex = block_excl_scan(s, sh) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (i0 + k < n) out[i0 + k] = ex;
        ex += v[k];
    }
}

size_t scan_tmp_ints(int n) { return (size_t)(n + SCAN_B - 1) / SCAN_B + 1; }

void scan_exclusive(const int* in, int* out, int n, int* tmp, int* total, cudaStream_t st) {
    if (n <= 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(int), st);
        return;
    }
    const int nb = (n + SCAN_B - 1) / SCAN_B;
    k_scan_reduce<<<nb, 256, 0, st>>>(in, n, tmp);
    k_scan_sums<<<1, 1024, 0, st>>>(tmp, nb, total);
    k_scan_down<<<nb, 256, 0, st>>>(in, n, tmp, out);
}

}  // namespace sfg
