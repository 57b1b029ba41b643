// PERIODIC reorder permutation without any allocation (partlib.f90:866-1133, single rank).
//
// For callers that cannot allocate device memory during their time loop: host codes that
// hand the library a fixed device-memory budget they manage themselves (their own pool
// holds the field and droplet arrays), and loops where the implicit device synchronisation
// of cudaMalloc/cudaFree would stall the pipeline.  This entry point calls no cudaMalloc,
// cudaFree or allocating library routine: its scratch is a file-scope device array of fixed
// size, and the caller passes inputs and outputs.
//
// Limits: n <= DL_NOALLOC_MAX_N droplets and at most DL_NOALLOC_MAX_DEPART departing
// droplets per call.  Every call shares the scratch array, which keeps the last call's
// contents; calls that overlap on the GPU (different streams, different host threads)
// race on it and must be serialised by the caller.  The device address of the array is
// looked up once per device, by the first call on that device, and kept for the life of
// the process: that first call should come before any stream capture on the device, and a
// device reset (cudaDeviceReset) after it is not supported.
#include "dl_internal.cuh"

#include <mutex>

#define DL_NOALLOC_MAX_N (1 << 26)
#define DL_NOALLOC_MAX_DEPART (1 << 17)

namespace {

constexpr int kBlk = DL_NOALLOC_MAX_N / 1024;
// A departing droplet is carried as (neighbour code << 26) | index (index < 2^26, code 1..8).
constexpr int kIdxBits = 26;
constexpr int kIdxMask = (1 << kIdxBits) - 1;
// layout: [0] status, [1] departures, [2..10] departures per neighbour code 0..8, [11..15]
// unused, [16 .. 16+kBlk] block counts/offsets, then the departing droplets (ascending
// index), then the departures in the replay's examination order
constexpr int kOffCode = 2;
constexpr int kOffBlk = 16;
constexpr int kOffP = kOffBlk + kBlk + 16;
constexpr int kOffDep = kOffP + DL_NOALLOC_MAX_DEPART;
constexpr int kScratchInts = kOffDep + DL_NOALLOC_MAX_DEPART;

static __device__ __align__(256) int g_noalloc_scratch[kScratchInts];

__device__ __forceinline__ int depart_code(double y, double z, double pi2)
{
    const double lo = 0.0, hi = pi2;
    if (y > hi && z <= hi && z >= lo) return 1;
    if (y > hi && z > hi) return 2;
    if (y >= lo && y <= hi && z > hi) return 3;
    if (y < lo && z > hi) return 4;
    if (y < lo && z <= hi && z >= lo) return 5;
    if (y < lo && z < lo) return 6;
    if (z < lo && y <= hi && y >= lo) return 7;
    if (z < lo && y > hi) return 8;
    return 0;
}

__global__ void __launch_bounds__(1024) k_na_count(int n, const double *y, const double *z, double pi2, int *s,
                                                   int *new_of_old)
{
    const int i = blockIdx.x * 1024 + threadIdx.x;
    int f = 0;
    if (i < n) {
        new_of_old[i] = i;   // identity for the droplets PERIODIC leaves in place
        f = depart_code(y[i], z[i], pi2) != 0;
    }
    const int c = __syncthreads_count(f);
    if (threadIdx.x == 0) s[kOffBlk + blockIdx.x] = c;
}

// exclusive scan of the block counts in place (one CTA); total -> s[1]
__global__ void __launch_bounds__(1024) k_na_scan(int nblk, int *s)
{
    __shared__ int ws[32];
    __shared__ int carry;
    int *cnt = s + kOffBlk;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < nblk; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < nblk ? cnt[i] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) ws[w] = incl;
        __syncthreads();
        if (w == 0) {
            int a = ws[lane], ai = a;
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, ai, o);
                if (lane >= o) ai += t;
            }
            ws[lane] = ai - a;
        }
        __syncthreads();
        const int excl = carry + ws[w] + incl - v;
        if (i < nblk) cnt[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        s[1] = carry;
        if (carry > DL_NOALLOC_MAX_DEPART) s[0] = 1;   // too many departures: nothing is reordered
    }
}

// departing droplets in ascending index order, each with its neighbour code
__global__ void __launch_bounds__(1024) k_na_compact(int n, const double *y, const double *z, double pi2, int *s)
{
    __shared__ int wsum[32];
    if (s[0]) return;
    const int i = blockIdx.x * 1024 + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int code = i < n ? depart_code(y[i], z[i], pi2) : 0;
    const bool f = code != 0;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[w] = __popc(m);
    __syncthreads();
    if (w == 0) {
        int v = wsum[lane], incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        wsum[lane] = incl - v;
    }
    __syncthreads();
    if (f) s[kOffP + s[kOffBlk + blockIdx.x] + wsum[w] + __popc(m & ((1u << lane) - 1))] = (code << kIdxBits) | i;
}

// The swap-with-last loop of partlib.f90:866-1097 replayed over the departing droplets only
// (one thread: each step depends on the previous one): records the order in which the
// departures are examined and counts them per neighbour code.
__global__ void k_na_replay(int n, int *s, int *new_of_old)
{
    if (threadIdx.x != 0 || s[0]) return;
    const int k = s[1];
    const int *P = s + kOffP;
    int *dep = s + kOffDep;
    int cnt[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int lo = 0, hi = k - 1, sum = 0, nd = 0;
    while (lo <= hi) {
        const int h = (P[lo] & kIdxMask) + 1;
        if (h + sum > n) break;
        int pe = P[lo];
        lo++;
        for (int guard = 0; guard <= k; guard++) {
            dep[nd++] = pe;
            cnt[pe >> kIdxBits]++;
            sum++;
            const int t = n - sum + 1;
            if (t == h) break;
            if (hi >= lo && (P[hi] & kIdxMask) + 1 == t) { pe = P[hi]; hi--; continue; }
            new_of_old[t - 1] = h - 1;
            break;
        }
    }
    if (nd != k) { s[0] = 2; return; }
    for (int q = 0; q <= 8; q++) s[kOffCode + q] = cnt[q];
}

// The departures appended in neighbour order 1..8, each code's droplets in examination
// order (partlib.f90:1099-1133): a stable counting placement by one CTA.
__global__ void __launch_bounds__(1024) k_na_place(int n, const int *s, int *new_of_old)
{
    __shared__ int wcnt[32][9];   // per warp and code: count, then the warp's first slot
    __shared__ int base[9];       // next free slot of each code
    if (s[0]) return;
    const int k = s[1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        int b = n - k;
        base[0] = 0;
        for (int q = 1; q <= 8; q++) { base[q] = b; b += s[kOffCode + q]; }
    }
    const int *dep = s + kOffDep;
    for (int c0 = 0; c0 < k; c0 += 1024) {
        const int j = c0 + threadIdx.x;
        const int pe = j < k ? dep[j] : 0;
        const int q = pe >> kIdxBits;   // 0 past the end
        const unsigned peers = __match_any_sync(0xffffffffu, q);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (lane < 9) wcnt[w][lane] = 0;
        __syncwarp();
        if (rank == 0) wcnt[w][q] = __popc(peers);
        __syncthreads();
        if (threadIdx.x < 9) {
            const int c = threadIdx.x;
            int a = base[c];
            for (int v = 0; v < 32; v++) { const int t = wcnt[v][c]; wcnt[v][c] = a; a += t; }
            base[c] = a;
        }
        __syncthreads();
        if (q > 0) new_of_old[pe & kIdxMask] = wcnt[w][q] + rank;
        __syncthreads();
    }
}

std::mutex g_setup_mutex;
int *g_scratch_ptr[64];   // device address of g_noalloc_scratch per device ordinal

}  // namespace

// Returns 0 on success, DL_E_ARG for sizes beyond the limits or bad pointers, DL_E_CAPACITY
// when more than DL_NOALLOC_MAX_DEPART droplets depart, DL_E_CUDA on a CUDA error.
extern "C" int dl_periodic_order_noalloc(const double *y, const double *z, int n, int *new_of_old, void *stream)
{
    if (n < 0 || n > DL_NOALLOC_MAX_N || (n > 0 && (!y || !z || !new_of_old))) return DL_E_ARG;
    if (n == 0) return 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DL_E_CUDA;
    int *s = nullptr;
    {
        // set-up once per device (the first call on a device; it should precede any
        // stream capture on that device)
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DL_E_CUDA;
            g_scratch_ptr[dev] = (int *)p;
        }
        s = g_scratch_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const double pi2 = 4.0 * atan(1.0) * 2.0;
    const int nblk = (n + 1023) / 1024;
    if (cudaMemsetAsync(s, 0, 16 * sizeof(int), st) != cudaSuccess) return DL_E_CUDA;   // status, count
    k_na_count<<<nblk, 1024, 0, st>>>(n, y, z, pi2, s, new_of_old);
    k_na_scan<<<1, 1024, 0, st>>>(nblk, s);
    k_na_compact<<<nblk, 1024, 0, st>>>(n, y, z, pi2, s);
    k_na_replay<<<1, 32, 0, st>>>(n, s, new_of_old);
    k_na_place<<<1, 1024, 0, st>>>(n, s, new_of_old);
    if (cudaGetLastError() != cudaSuccess) return DL_E_CUDA;
    int status = 0;
    if (cudaMemcpyAsync(&status, s, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DL_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return DL_E_CUDA;
    if (status == 1) return DL_E_CAPACITY;
    if (status != 0) return DL_E_STATE;
    return 0;
}
