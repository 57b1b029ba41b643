// Multi-block exclusive scan of int counts (start[n] = total), with the largest count.
// Header-only; every kernel has internal linkage in the including file.
#pragma once

#include <cuda_runtime.h>

namespace {

__global__ void __launch_bounds__(1024) k_cnt_blocksum(int n, const int *cnt, int *bsum, int *maxcnt)
{
    __shared__ int ws[32], wm[32];
    const int i = blockIdx.x * 1024 + threadIdx.x;
    const int v = i < n ? cnt[i] : 0;
    int s = v, m = v;
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    }
    if ((threadIdx.x & 31) == 0) {
        ws[threadIdx.x >> 5] = s;
        wm[threadIdx.x >> 5] = m;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        int t = ws[threadIdx.x], u = wm[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) {
            t += __shfl_down_sync(0xffffffffu, t, o);
            u = max(u, __shfl_down_sync(0xffffffffu, u, o));
        }
        if (threadIdx.x == 0) {
            bsum[blockIdx.x] = t;
            if (maxcnt) atomicMax(maxcnt, u);   // one atomic per CTA
        }
    }
}

// one CTA: exclusive scan of the block sums in chunks of 1024, total in off[m]
__global__ void __launch_bounds__(1024) k_cnt_scan_sums(int m, const int *bsum, int *off)
{
    __shared__ int ws[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < m; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < m ? bsum[i] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) ws[w] = incl;
        __syncthreads();
        if (w == 0) {
            const int a = ws[lane];
            int ai = a;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, ai, o);
                if (lane >= o) ai += t;
            }
            ws[lane] = ai - a;
        }
        __syncthreads();
        const int excl = carry + ws[w] + incl - v;
        if (i < m) off[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) off[m] = carry;
}

__global__ void __launch_bounds__(1024) k_cnt_apply(int n, const int *cnt, const int *boff, int nblk, int *start)
{
    __shared__ int ws[32];
    const int i = blockIdx.x * 1024 + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int v = i < n ? cnt[i] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) ws[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int a = ws[lane];
        int ai = a;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, ai, o);
            if (lane >= o) ai += t;
        }
        ws[lane] = ai - a;
    }
    __syncthreads();
    if (i < n) start[i] = boff[blockIdx.x] + ws[w] + incl - v;
    if (blockIdx.x == 0 && threadIdx.x == 0) start[n] = boff[nblk];
}

// start[0..n] = exclusive scan of cnt[0..n-1]; scratch holds 2 * (n / 1024 + 2) ints;
// maxcnt (optional) receives atomicMax of the counts.  Three launches on st.
inline cudaError_t dl_scan_counts(cudaStream_t st, const int *cnt, int *start, int n, int *scratch, int *maxcnt)
{
    const int nblk = (n + 1023) / 1024;
    int *bsum = scratch, *boff = scratch + (n / 1024 + 2);
    if (nblk == 0) return cudaMemsetAsync(start, 0, sizeof(int), st);
    k_cnt_blocksum<<<nblk, 1024, 0, st>>>(n, cnt, bsum, maxcnt);
    k_cnt_scan_sums<<<1, 1024, 0, st>>>(nblk, bsum, boff);
    k_cnt_apply<<<nblk, 1024, 0, st>>>(n, cnt, boff, nblk, start);
    return cudaGetLastError();
}

}  // namespace
