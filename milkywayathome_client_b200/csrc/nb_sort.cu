// LSD radix sort of 64-bit Morton keys with 32-bit body indices, and an int prefix sum.
//
// Replaces the lock-based concurrent insertion of the reference's OpenCL buildTree
// (nbody/kernels/nbody_kernels.cl:898-1159): bodies are ordered by octree path once and
// the tree is derived from the sorted order without locks or spin-waits.
//
// Each of the 8 passes sorts by one 8-bit digit: per-tile digit histograms, an exclusive
// scan of the (digit, tile) table (three coalesced phases), and a stable scatter that ranks
// keys inside a tile with warp match/ballot.  HBM-bound: a pass reads and writes
// 12 bytes per key.
#include "nb_common.cuh"

namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_ROUNDS = 8;                         // keys per thread per tile
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;      // 2048 keys per tile
constexpr int RS_WARPS = RS_THREADS / 32;

// digit of item i: 8 bits of its key, or (GROUPED) 8 bits of the group of its index
template <bool GROUPED>
__device__ __forceinline__ unsigned int rs_digit(unsigned long long key, unsigned int idx,
                                                 const int* group, int shift)
{
    if (GROUPED) return ((unsigned) group[idx] >> shift) & 255u;
    return (unsigned) (key >> shift) & 255u;
}

template <bool GROUPED>
__global__ void __launch_bounds__(RS_THREADS)
k_rs_hist(const unsigned long long* __restrict__ keys, const unsigned int* __restrict__ idx,
          const int* __restrict__ group, int n, int shift, unsigned int* __restrict__ hist,
          int nTiles)
{
    __shared__ unsigned int cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * RS_TILE;
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
        int i = base + r * RS_THREADS + threadIdx.x;
        if (i < n)
            atomicAdd(&cnt[rs_digit<GROUPED>(GROUPED ? 0ull : keys[i], GROUPED ? idx[i] : 0u,
                                             group, shift)], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nTiles + blockIdx.x] = cnt[threadIdx.x];
}

template <bool GROUPED>
__global__ void __launch_bounds__(RS_THREADS)
k_rs_scatter(const unsigned long long* __restrict__ keyIn, const unsigned int* __restrict__ idxIn,
             unsigned long long* __restrict__ keyOut, unsigned int* __restrict__ idxOut,
             const int* __restrict__ group, int n, int shift,
             const unsigned int* __restrict__ hist, int nTiles)
{
    __shared__ unsigned int gOff[256];             // global start of each digit for this tile
    __shared__ unsigned int dRun[256];             // keys of each digit already placed
    __shared__ unsigned int wHist[RS_WARPS][256];  // per-warp counts, then offsets
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    gOff[t] = hist[t * nTiles + blockIdx.x];
    dRun[t] = 0;
    const unsigned int ltMask = (1u << lane) - 1u;
    const int base = blockIdx.x * RS_TILE;
    for (int r = 0; r < RS_ROUNDS; ++r) {
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) wHist[w][t] = 0;
        __syncthreads();
        const int i = base + r * RS_THREADS + t;
        const bool valid = i < n;
        unsigned long long key = valid ? keyIn[i] : 0ull;
        unsigned int idx = valid ? idxIn[i] : 0u;
        const unsigned int d = valid ? rs_digit<GROUPED>(key, idx, group, shift) : 256u;
        const unsigned int peers = __match_any_sync(NB_FULL_MASK, d);
        const unsigned int rankInWarp = __popc(peers & ltMask);
        if (valid && rankInWarp == 0) wHist[warp][d] = __popc(peers);
        __syncthreads();
        {   // per digit: turn warp counts into offsets, in warp order (keeps the sort stable)
            unsigned int off = dRun[t];
#pragma unroll
            for (int w = 0; w < RS_WARPS; ++w) {
                unsigned int c = wHist[w][t];
                wHist[w][t] = off;
                off += c;
            }
            dRun[t] = off;
        }
        __syncthreads();
        if (valid) {
            unsigned int pos = gOff[d] + wHist[warp][d] + rankInWarp;
            keyOut[pos] = key;
            idxOut[pos] = idx;
        }
        __syncthreads();
    }
}

// ---- int inclusive scan (three phases) ----
constexpr int PS_THREADS = 1024;
constexpr int PS_ITEMS = 4;
constexpr int PS_TILE = PS_THREADS * PS_ITEMS;

__device__ __forceinline__ int block_inclusive_scan(int v, int* sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int u = __shfl_up_sync(NB_FULL_MASK, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(NB_FULL_MASK, w, o);
            if (lane >= o) w += u;
        }
        sh[lane] = w;
    }
    __syncthreads();
    int r = v + (warp > 0 ? sh[warp - 1] : 0);
    __syncthreads();
    return r;
}

template <bool EXCLUSIVE>
__global__ void __launch_bounds__(PS_THREADS)
k_ps_tile(int* __restrict__ data, int n, int* __restrict__ tileSums)
{
    __shared__ int sh[32];
    const int base = blockIdx.x * PS_TILE + threadIdx.x * PS_ITEMS;
    int v[PS_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < PS_ITEMS; ++k) {
        const int x = base + k < n ? data[base + k] : 0;
        v[k] = EXCLUSIVE ? s : s + x;
        s += x;
    }
    int incl = block_inclusive_scan(s, sh);
    int excl = incl - s;
#pragma unroll
    for (int k = 0; k < PS_ITEMS; ++k)
        if (base + k < n) data[base + k] = v[k] + excl;
    if (threadIdx.x == blockDim.x - 1) tileSums[blockIdx.x] = incl;
}

__global__ void __launch_bounds__(PS_THREADS)
k_ps_top(int* __restrict__ tileSums, int nTiles)
{
    __shared__ int sh[32];
    int carry = 0;
    for (int base = 0; base < nTiles; base += PS_THREADS) {
        int i = base + threadIdx.x;
        int v = i < nTiles ? tileSums[i] : 0;
        int incl = block_inclusive_scan(v, sh);
        if (i < nTiles) tileSums[i] = incl - v + carry;   // exclusive
        int total = __shfl_sync(NB_FULL_MASK, incl, 31);
        __shared__ int last;
        if (threadIdx.x == PS_THREADS - 1) last = incl;
        __syncthreads();
        carry += last;
        __syncthreads();
        (void) total;
    }
}

__global__ void __launch_bounds__(PS_THREADS)
k_ps_apply(int* __restrict__ data, int n, const int* __restrict__ tileSums)
{
    const int off = tileSums[blockIdx.x];
    const int base = blockIdx.x * PS_TILE + threadIdx.x * PS_ITEMS;
#pragma unroll
    for (int k = 0; k < PS_ITEMS; ++k)
        if (base + k < n) data[base + k] += off;
}

}  // namespace

static void rs_passes(NbSortBuffers& b, int n, const int* group, cudaStream_t s)
{
    if (n <= 0) return;
    const int nTiles = (n + RS_TILE - 1) / RS_TILE;
    unsigned long long* kin = b.keyA; unsigned long long* kout = b.keyB;
    unsigned int* iin = b.idxA; unsigned int* iout = b.idxB;
    const int passes = group ? 10 : 8;
    for (int pass = 0; pass < passes; ++pass) {
        const bool grouped = pass >= 8;
        const int shift = grouped ? (pass - 8) * 8 : pass * 8;
        if (grouped)
            k_rs_hist<true><<<nTiles, RS_THREADS, 0, s>>>(kin, iin, group, n, shift, b.hist, nTiles);
        else
            k_rs_hist<false><<<nTiles, RS_THREADS, 0, s>>>(kin, iin, nullptr, n, shift, b.hist, nTiles);
        // exclusive scan of the (digit, tile) table, three coalesced phases
        const int len = 256 * nTiles;
        const int scanTiles = (len + PS_TILE - 1) / PS_TILE;
        k_ps_tile<true><<<scanTiles, PS_THREADS, 0, s>>>((int*) b.hist, len, b.histTmp);
        k_ps_top<<<1, PS_THREADS, 0, s>>>(b.histTmp, scanTiles);
        k_ps_apply<<<scanTiles, PS_THREADS, 0, s>>>((int*) b.hist, len, b.histTmp);
        if (grouped)
            k_rs_scatter<true><<<nTiles, RS_THREADS, 0, s>>>(kin, iin, kout, iout, group, n, shift,
                                                             b.hist, nTiles);
        else
            k_rs_scatter<false><<<nTiles, RS_THREADS, 0, s>>>(kin, iin, kout, iout, nullptr, n,
                                                              shift, b.hist, nTiles);
        nb_count_launch(5);
        unsigned long long* tk = kin; kin = kout; kout = tk;
        unsigned int* ti = iin; iin = iout; iout = ti;
    }
    // an even number of passes: the result is back in keyA / idxA.
}

void nb_radix_sort(NbSortBuffers& b, int n, cudaStream_t s) { rs_passes(b, n, nullptr, s); }

void nb_radix_sort_grouped(NbSortBuffers& b, int n, const int* group, cudaStream_t s)
{
    rs_passes(b, n, group, s);
}

int nb_scan_tmp_ints(int n) { return (n + PS_TILE - 1) / PS_TILE + 1; }

void nb_inclusive_scan(int* data, int n, int* tmp, cudaStream_t s)
{
    if (n <= 0) return;
    const int nTiles = (n + PS_TILE - 1) / PS_TILE;
    k_ps_tile<false><<<nTiles, PS_THREADS, 0, s>>>(data, n, tmp);
    k_ps_top<<<1, PS_THREADS, 0, s>>>(tmp, nTiles);
    k_ps_apply<<<nTiles, PS_THREADS, 0, s>>>(data, n, tmp);
    nb_count_launch(3);
}
