// phx_merge.cuh : hit merging on the device — select records by flag mask, group them by
// (identity, time bucket) and reduce each group to one record with a summed hit count.
//
// Semantics follow SPM::merge_partial_select (sysrap/SPM.cu:110-200) with the record functors of
// sysrap/sphoton.h:292-320 (sphoton, 64 B) and sysrap/sphotonlite.h:68-97 (sphotonlite, 16 B):
//   select   (flagmask & mask) != 0, or every record when mask == 0xffffffff (already selected)
//   key      (uint64(identity) << 48) | unsigned(time / window)   (identity bits above 16 drop out)
//   order    groups ascending by key; within a group the input order decides ties
//   reduce   sphoton     : the earliest-time record (ties: first in input order), flagmask = OR,
//                          hitcount = sum (16 bits)
//            sphotonlite : the first record in input order, time = min, flagmask = OR,
//                          hitcount = sum (16 bits)
//   window 0 : selection only, records in input order
//
// The reference sorts with thrust::sort_by_key and folds with thrust::reduce_by_key.  Here:
//   1. ordered selection (ballot + tile offsets)           -> sel[m] input positions
//   2. keys (u64) and their bitwise OR                     -> passes only over non-zero key bytes
//   3. stable LSD radix sort, 8-bit digits: per-tile digit histograms (digit-major), one scan,
//      a scatter ranking equal digits by __match_any_sync so every pass is stable
//   4. group heads + scan -> group index; warp-segmented reductions (__reduce_*_sync over the
//      lanes of one group) with one atomic per (warp, group): min (time, position), min position,
//      OR flagmask, sum hitcount
//   5. one thread per group writes the representative record with the reduced fields
// Each reduction is associative and picks the record the left fold of reduce_op picks.  Included by
// phx_engine.cu after DevBuf and PHX_CU.
#pragma once
#include <stdint.h>

#define PHX_MERGE_TILE_ITEMS 8
#define PHX_MERGE_TILE (256 * PHX_MERGE_TILE_ITEMS)
#define PHX_MERGE_SCAN_TILE 1024

// word offsets of the fields a merge reads/writes, per record kind
template <int LITE> struct PhxRec;
template <> struct PhxRec<0> {       // sphoton (sysrap/sphoton.h:171-192)
    static constexpr int W = 16, TIME = 3, HC = 7, ID = 13, FLAG = 15;
    static constexpr uint32_t IDMASK = 0xffffffu;
};
template <> struct PhxRec<1> {       // sphotonlite (sysrap/sphotonlite.h:47-51)
    static constexpr int W = 4, TIME = 1, HC = 0, ID = 0, FLAG = 3;
    static constexpr uint32_t IDMASK = 0xffffu;
};

// monotone map of float bits to u32 order; NaN after +inf (fminf ignores NaN)
__device__ __forceinline__ uint32_t phx_time_order(uint32_t b)
{
    if ((b & 0x7fffffffu) > 0x7f800000u) return 0xffffffffu;
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ uint32_t phx_time_unorder(uint32_t o)
{
    if (o == 0xffffffffu) return 0x7fc00000u;
    return (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
}

// 1a. per-tile selected counts
template <int LITE>
__global__ void __launch_bounds__(256) k_merge_sel_count(const uint32_t* in, long long n, uint32_t mask, uint32_t* tcount)
{
    __shared__ uint32_t wsum[8];
    const long long tile = (long long)blockIdx.x * PHX_MERGE_TILE;
    uint32_t c = 0;
    for (int r = 0; r < PHX_MERGE_TILE_ITEMS; r++) {
        const long long i = tile + (long long)r * 256 + threadIdx.x;
        if (i < n) c += (in[i * PhxRec<LITE>::W + PhxRec<LITE>::FLAG] & mask) != 0u;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int k = 0; k < 8; k++) s += wsum[k];
        tcount[blockIdx.x] = s;
    }
}

// 1b. ordered write of selected positions (tile offsets already scanned)
template <int LITE>
__global__ void __launch_bounds__(256) k_merge_sel_write(const uint32_t* in, long long n, uint32_t mask, const uint32_t* toff,
                                                          uint32_t* sel)
{
    __shared__ uint32_t wsum[8];
    __shared__ uint32_t base;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) base = toff[blockIdx.x];
    __syncthreads();
    const long long tile = (long long)blockIdx.x * PHX_MERGE_TILE;
    for (int r = 0; r < PHX_MERGE_TILE_ITEMS; r++) {
        const long long i = tile + (long long)r * 256 + threadIdx.x;
        const bool s = i < n && (in[i * PhxRec<LITE>::W + PhxRec<LITE>::FLAG] & mask) != 0u;
        const uint32_t b = __ballot_sync(0xffffffffu, s);
        if (lane == 0) wsum[w] = __popc(b);
        __syncthreads();
        uint32_t before = base;
        for (int k = 0; k < w; k++) before += wsum[k];
        if (s) sel[before + __popc(b & ((1u << lane) - 1u))] = (uint32_t)i;
        __syncthreads();
        if (threadIdx.x == 0) { uint32_t t = 0; for (int k = 0; k < 8; k++) t += wsum[k]; base += t; }
        __syncthreads();
    }
}

// selection only (window 0): gather selected records in order
template <int LITE>
__global__ void k_merge_gather(const uint32_t* in, const uint32_t* sel, long long m, uint32_t* out)
{
    constexpr int W = PhxRec<LITE>::W;
    const long long total = m * W;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
        const long long j = k / W;
        const int w = (int)(k - j * W);
        const long long i = sel ? (long long)sel[j] : j;
        out[k] = in[i * W + w];
    }
}

// 2. keys of the selected records; OR of all keys
template <int LITE>
__global__ void k_merge_keys(const uint32_t* in, const uint32_t* sel, long long m, float tw, unsigned long long* key,
                             uint32_t* val, unsigned long long* key_or)
{
    unsigned long long acc = 0ull;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (long long)gridDim.x * blockDim.x) {
        const long long i = sel ? (long long)sel[j] : j;
        const uint32_t* r = in + i * PhxRec<LITE>::W;
        const uint32_t id = r[PhxRec<LITE>::ID] & PhxRec<LITE>::IDMASK;
        const unsigned bucket = static_cast<unsigned>(__uint_as_float(r[PhxRec<LITE>::TIME]) / tw);
        const unsigned long long k = ((unsigned long long)id << 48) | (unsigned long long)bucket;
        key[j] = k;
        val[j] = (uint32_t)j;
        acc |= k;
    }
    for (int o = 16; o > 0; o >>= 1) acc |= __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicOr(key_or, acc);
}

// 3a. digit histogram per tile, digit-major: hist[d * ntile + tile]
__global__ void __launch_bounds__(256) k_radix_hist(const unsigned long long* key, long long m, int shift, uint32_t* hist, int ntile)
{
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0u;
    __syncthreads();
    const long long tile = (long long)blockIdx.x * PHX_MERGE_TILE;
    for (int r = 0; r < PHX_MERGE_TILE_ITEMS; r++) {
        const long long j = tile + (long long)r * 256 + threadIdx.x;
        if (j < m) atomicAdd(&h[(uint32_t)(key[j] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * ntile + blockIdx.x] = h[threadIdx.x];
}

// 3b. stable scatter: equal digits ranked by (round, warp, lane), i.e. by position in the tile
__global__ void __launch_bounds__(256) k_radix_scatter(const unsigned long long* kin, const uint32_t* vin, unsigned long long* kout,
                                                       uint32_t* vout, long long m, int shift, const uint32_t* off, int ntile)
{
    __shared__ uint32_t base[256];
    __shared__ uint32_t wcnt[8][256];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    base[t] = off[(size_t)t * ntile + blockIdx.x];
    const long long tile = (long long)blockIdx.x * PHX_MERGE_TILE;
    for (int r = 0; r < PHX_MERGE_TILE_ITEMS; r++) {
        for (int q = 0; q < 8; q++) wcnt[q][t] = 0u;
        __syncthreads();
        const long long j = tile + (long long)r * 256 + t;
        const bool ok = j < m;
        const unsigned long long k = ok ? kin[j] : 0ull;
        const uint32_t v = ok ? vin[j] : 0u;
        const uint32_t d = ok ? ((uint32_t)(k >> shift) & 0xffu) : 0x100u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        if (ok && rank == 0u) wcnt[w][d] = __popc(peers);
        __syncthreads();
        {
            uint32_t run = base[t];
            for (int q = 0; q < 8; q++) { const uint32_t c = wcnt[q][t]; wcnt[q][t] = run; run += c; }
            base[t] = run;
        }
        __syncthreads();
        if (ok) {
            const uint32_t p = wcnt[w][d] + rank;
            kout[p] = k;
            vout[p] = v;
        }
        __syncthreads();
    }
}

// exclusive scan of u32 in tiles of 1024 (256 threads x 4): local scan + tile sums
__global__ void __launch_bounds__(256) k_scan_tile(uint32_t* x, long long n, uint32_t* tsum)
{
    __shared__ uint32_t wt[8];
    const long long b = (long long)blockIdx.x * PHX_MERGE_SCAN_TILE + (long long)threadIdx.x * 4;
    uint32_t v[4], s = 0;
    for (int k = 0; k < 4; k++) { v[k] = (b + k < n) ? x[b + k] : 0u; s += v[k]; }
    uint32_t inc = s;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) { const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o); if (lane >= o) inc += y; }
    if (lane == 31) wt[wid] = inc;
    __syncthreads();
    uint32_t before = 0;
    for (int k = 0; k < wid; k++) before += wt[k];
    uint32_t run = before + inc - s;
    for (int k = 0; k < 4; k++) { if (b + k < n) x[b + k] = run; run += v[k]; }
    if (threadIdx.x == 255) tsum[blockIdx.x] = before + inc;
}
__global__ void k_scan_add(uint32_t* x, long long n, const uint32_t* tsum)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += tsum[i / PHX_MERGE_SCAN_TILE];
}

// 4a. group heads
__global__ void k_merge_heads(const unsigned long long* key, long long m, uint32_t* head)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < m) head[j] = (j == 0 || key[j] != key[j - 1]) ? 1u : 0u;
}

// 4b. warp-segmented reduction per group, one atomic per (warp, group)
template <int LITE>
__global__ void k_merge_reduce(const uint32_t* in, const uint32_t* sel, const unsigned long long* key, const uint32_t* val,
                               const uint32_t* gexcl, long long m, unsigned long long* amin, uint32_t* pmin, uint32_t* gor,
                               uint32_t* gsum)
{
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < m; base += stride) {
        const long long j = base + lane;
        const bool ok = j < m;
        uint32_t g = 0xffffffffu, pos = 0xffffffffu, tb = 0xffffffffu, fl = 0u, hc = 0u;
        if (ok) {
            const uint32_t head = (j == 0 || key[j] != key[j - 1]) ? 1u : 0u;
            g = gexcl[j] + head - 1u;
            pos = val[j];
            const long long i = sel ? (long long)sel[pos] : (long long)pos;
            const uint32_t* r = in + i * PhxRec<LITE>::W;
            tb = phx_time_order(r[PhxRec<LITE>::TIME]);
            fl = r[PhxRec<LITE>::FLAG];
            hc = r[PhxRec<LITE>::HC] >> 16;
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, g);
        const uint32_t tmin = __reduce_min_sync(peers, tb);
        const uint32_t pfirst = __reduce_min_sync(peers, tb == tmin ? pos : 0xffffffffu);
        const uint32_t pm = __reduce_min_sync(peers, pos);
        const uint32_t fo = __reduce_or_sync(peers, fl);
        const uint32_t hs = __reduce_add_sync(peers, hc);
        if (ok && (__ffs(peers) - 1) == lane) {
            atomicMin(amin + g, ((unsigned long long)tmin << 32) | (unsigned long long)pfirst);
            atomicMin(pmin + g, pm);
            atomicOr(gor + g, fo);
            atomicAdd(gsum + g, hs);
        }
    }
}

// 5. representative record per group with the reduced fields
template <int LITE>
__global__ void k_merge_write(const uint32_t* in, const uint32_t* sel, long long ng, const unsigned long long* amin,
                              const uint32_t* pmin, const uint32_t* gor, const uint32_t* gsum, uint32_t* out)
{
    constexpr int W = PhxRec<LITE>::W;
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    const uint32_t pos = LITE ? pmin[g] : (uint32_t)(amin[g] & 0xffffffffull);
    const long long i = sel ? (long long)sel[pos] : (long long)pos;
    uint32_t r[W];
    for (int w = 0; w < W; w++) r[w] = in[i * W + w];
    if (LITE) r[PhxRec<LITE>::TIME] = phx_time_unorder((uint32_t)(amin[g] >> 32));
    r[PhxRec<LITE>::FLAG] = gor[g];
    r[PhxRec<LITE>::HC] = (r[PhxRec<LITE>::HC] & 0xffffu) | ((gsum[g] & 0xffffu) << 16);
    for (int w = 0; w < W; w++) out[g * W + w] = r[w];
}
