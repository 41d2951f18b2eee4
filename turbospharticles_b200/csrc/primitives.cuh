// primitives.cuh -- device-wide scan and stable LSD radix sort used by the neighbor build.
//
// Scan: reduce-then-scan over tiles of 1024 items with functors for the input and output,
// so the producers (run starts of the cell tables, SELL32 chunk sizes per format, CSR
// counts) never materialise an intermediate array. The grand total lands in device memory
// and stays there (no host round trip).
//
// Sort: stable LSD radix sort with 8-bit digits over (clamped cell key, particle index)
// pairs, the ordering rule of SortParticleOrderByCellId (source/simulation/CPU/backend/
// neighbor_search.cpp:415-564). Each pass: per-tile digit histograms -> per-digit
// cross-tile exclusive scan -> ranked scatter. Ranks are stable (tile index order) via
// __match_any_sync peers per warp and per-warp digit counters; each tile is staged in
// shared memory in digit order so the global writes are runs of consecutive addresses.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tsp {

// ------------------------------------------------------------------------------ scan
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

struct U64x2 {  // trivially constructible: usable in __shared__ arrays
    uint64_t a, b;
    __host__ __device__ U64x2 operator+(const U64x2& o) const { return U64x2{a + o.a, b + o.b}; }
};
__device__ __forceinline__ uint64_t ShflUp(uint64_t v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ U64x2 ShflUp(U64x2 v, int d) {
    return U64x2{__shfl_up_sync(0xffffffffu, v.a, d), __shfl_up_sync(0xffffffffu, v.b, d)};
}
__device__ __forceinline__ uint64_t ShflIdx(uint64_t v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ U64x2 ShflIdx(U64x2 v, int l) {
    return U64x2{__shfl_sync(0xffffffffu, v.a, l), __shfl_sync(0xffffffffu, v.b, l)};
}

// block-wide exclusive scan of one value per thread; returns the exclusive prefix and the total
template <typename T>
__device__ __forceinline__ T BlockExclusiveScan(T v, T& total) {
    __shared__ T warpSums[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T o = ShflUp(incl, d);
        if (lane >= d) incl = incl + o;
    }
    if (lane == 31) warpSums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T ws = (lane < SCAN_THREADS / 32) ? warpSums[lane] : T();
        T wi = ws;
#pragma unroll
        for (int d = 1; d < SCAN_THREADS / 32; d <<= 1) {
            const T o = ShflUp(wi, d);
            if (lane >= d) wi = wi + o;
        }
        if (lane < SCAN_THREADS / 32) warpSums[lane] = wi;  // inclusive warp prefixes
    }
    __syncthreads();
    total = warpSums[SCAN_THREADS / 32 - 1];
    const T warpPrefix = (warp > 0) ? warpSums[warp - 1] : T();
    const T prevIncl = ShflUp(incl, 1);  // inclusive value of the previous lane
    const T res = (lane > 0) ? (warpPrefix + prevIncl) : warpPrefix;
    __syncthreads();  // warpSums is reused by the next call
    return res;
}

template <typename T, typename In>
__global__ void __launch_bounds__(SCAN_THREADS) KScanReduce(In in, uint64_t n, T* blockSums) {
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    T s = T();
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
        if (base + k < n) s = s + in(base + k);
    T total;
    BlockExclusiveScan(s, total);
    if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

// exclusive scan of blockSums in place by one block (any length), grand total to *total
template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) KScanSingle(T* v, uint64_t n, T* total) {
    T carry = T();
    for (uint64_t start = 0; start < n; start += SCAN_TILE) {
        const uint64_t base = start + (uint64_t)threadIdx.x * SCAN_ITEMS;
        T loc[SCAN_ITEMS];
        T s = T();
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) {
            loc[k] = (base + k < n) ? v[base + k] : T();
            s = s + loc[k];
        }
        T tileTotal;
        T pre = BlockExclusiveScan(s, tileTotal) + carry;
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) {
            if (base + k < n) v[base + k] = pre;
            pre = pre + loc[k];
        }
        carry = carry + tileTotal;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <typename T, typename In, typename Out>
__global__ void __launch_bounds__(SCAN_THREADS) KScanDown(In in, Out out, uint64_t n, const T* blockOffsets) {
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    T loc[SCAN_ITEMS];
    T s = T();
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        loc[k] = (base + k < n) ? in(base + k) : T();
        s = s + loc[k];
    }
    T tileTotal;
    T pre = BlockExclusiveScan(s, tileTotal) + blockOffsets[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < n) out(base + k, pre, loc[k]);
        pre = pre + loc[k];
    }
}

// exclusive scan over n items; `scratch` must hold ceil(n / SCAN_TILE) values of T;
// the total is written to the device pointer `total`
template <typename T, typename In, typename Out>
void DeviceScan(In in, Out out, uint64_t n, T* scratch, T* total, cudaStream_t s) {
    if (n == 0) {
        cudaMemsetAsync(total, 0, sizeof(T), s);
        return;
    }
    const uint64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    KScanReduce<T, In><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, scratch);
    KScanSingle<T><<<1, SCAN_THREADS, 0, s>>>(scratch, nb, total);
    KScanDown<T, In, Out><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, scratch);
}
inline uint64_t ScanScratchItems(uint64_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

// ------------------------------------------------------------------------------ radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARPS = RS_THREADS / 32;

// Passes whose digit is the same in every key are the identity permutation. When the caller
// gives `orNot` = {OR of all keys, OR of all complemented keys} (computed while the keys are
// made), such a pass skips its histogram and scan and its scatter becomes a plain copy.
__device__ __forceinline__ bool RadixPassConstant(const uint64_t* orNot, uint32_t shift) {
    if (orNot == nullptr) return false;
    const uint64_t varying = orNot[0] & orNot[1];  // bits that are 1 in some key and 0 in another
    return ((varying >> shift) & 255u) == 0u;
}

template <typename K>
__global__ void __launch_bounds__(RS_THREADS) KRadixUpsweep(const K* __restrict__ keys, uint32_t n, uint32_t shift,
                                                          uint32_t* __restrict__ tileHist, uint32_t nTiles,
                                                          const uint64_t* __restrict__ orNot) {
    if (RadixPassConstant(orNot, shift)) return;
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * RS_TILE;
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        const uint32_t i = base + r * RS_THREADS + threadIdx.x;
        const uint32_t d = (i < n) ? (uint32_t)((keys[i] >> shift) & 255u) : 256u + lane;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (d < 256u && (__ffs(peers) - 1) == (int)lane) atomicAdd(&h[d], __popc(peers));
    }
    __syncthreads();
    tileHist[(uint64_t)threadIdx.x * nTiles + blockIdx.x] = h[threadIdx.x];
}

// one block per digit: exclusive scan of that digit's row across tiles, digit total out
static __global__ void __launch_bounds__(256) KRadixScanRows(uint32_t* __restrict__ tileHist, uint32_t nTiles,
                                                      uint32_t* __restrict__ digitTotals, uint32_t shift,
                                                      const uint64_t* __restrict__ orNot) {
    if (RadixPassConstant(orNot, shift)) return;
    __shared__ uint32_t ws[8];
    uint32_t* row = tileHist + (uint64_t)blockIdx.x * nTiles;
    uint32_t carry = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t start = 0; start < nTiles; start += 256) {
        const uint32_t i = start + threadIdx.x;
        const uint32_t v = (i < nTiles) ? row[i] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += o;
        }
        if (lane == 31) ws[warp] = incl;
        __syncthreads();
        uint32_t warpPre = 0, tot = 0;
        for (int w = 0; w < 8; w++) {
            if (w < warp) warpPre += ws[w];
            tot += ws[w];
        }
        if (i < nTiles) row[i] = carry + warpPre + incl - v;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) digitTotals[blockIdx.x] = carry;
}

template <typename K, typename V>
__global__ void __launch_bounds__(RS_THREADS) KRadixDownsweep(const K* __restrict__ kin, const V* __restrict__ vin,
                                                            K* __restrict__ kout, V* __restrict__ vout, uint32_t n,
                                                            uint32_t shift, const uint32_t* __restrict__ tileHist,
                                                            const uint32_t* __restrict__ digitTotals, uint32_t nTiles,
                                                            const uint64_t* __restrict__ orNot) {
    if (RadixPassConstant(orNot, shift)) {  // identity pass: copy the tile
        const uint32_t base = blockIdx.x * RS_TILE;
        for (uint32_t li = threadIdx.x; li < (uint32_t)RS_TILE && base + li < n; li += RS_THREADS) {
            kout[base + li] = kin[base + li];
            vout[base + li] = vin[base + li];
        }
        return;
    }
    __shared__ uint32_t digitBase[256];
    __shared__ uint32_t tileStart[256];
    __shared__ uint32_t cnt[256];
    __shared__ uint32_t warpCnt[RS_WARPS][256];
    __shared__ K skeys[RS_TILE];
    __shared__ V svals[RS_TILE];
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t base = blockIdx.x * RS_TILE;
    const uint32_t tileValid = (n - base < (uint32_t)RS_TILE) ? (n - base) : (uint32_t)RS_TILE;

    K key[RS_ITEMS];
    V val[RS_ITEMS];
    uint32_t dig[RS_ITEMS];
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        const uint32_t li = r * RS_THREADS + t;
        if (li < tileValid) {
            key[r] = kin[base + li];
            val[r] = vin[base + li];
            dig[r] = (uint32_t)((key[r] >> shift) & 255u);
        } else {
            dig[r] = 256u + lane;  // never matches a real digit
        }
    }
    // global digit bases: exclusive scan of the digit totals + this tile's cross-tile prefix
    {
        const uint32_t v = digitTotals[t];
        uint32_t incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += o;
        }
        cnt[t] = 0;
        if (lane == 31) warpCnt[0][warp] = incl;
        __syncthreads();
        uint32_t pre = 0;
        for (uint32_t w = 0; w < warp; w++) pre += warpCnt[0][w];
        digitBase[t] = pre + incl - v + tileHist[(uint64_t)t * nTiles + blockIdx.x];
        __syncthreads();
    }
    // this tile's digit histogram -> start of each digit run inside the tile
    for (int w = 0; w < RS_WARPS; w++) warpCnt[w][t] = 0;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        const uint32_t peers = __match_any_sync(0xffffffffu, dig[r]);
        if (dig[r] < 256u && (__ffs(peers) - 1) == (int)lane) atomicAdd(&cnt[dig[r]], __popc(peers));
    }
    __syncthreads();
    {
        const uint32_t v = cnt[t];
        uint32_t incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += o;
        }
        if (lane == 31) warpCnt[1][warp] = incl;
        __syncthreads();
        uint32_t pre = 0;
        for (uint32_t w = 0; w < warp; w++) pre += warpCnt[1][w];
        tileStart[t] = pre + incl - v;
        __syncthreads();
        cnt[t] = 0;
        for (int w = 0; w < RS_WARPS; w++) warpCnt[w][t] = 0;
        __syncthreads();
    }
    // stable ranks, round by round in tile index order
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        const uint32_t d = dig[r];
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rankInWarp = __popc(peers & ((1u << lane) - 1u));
        if (d < 256u && (__ffs(peers) - 1) == (int)lane) warpCnt[warp][d] = __popc(peers);
        __syncthreads();
        if (d < 256u) {
            uint32_t rank = cnt[d] + rankInWarp;
            for (uint32_t w = 0; w < warp; w++) rank += warpCnt[w][d];
            const uint32_t pos = tileStart[d] + rank;
            skeys[pos] = key[r];
            svals[pos] = val[r];
        }
        __syncthreads();
        uint32_t add = 0;
        for (int w = 0; w < RS_WARPS; w++) { add += warpCnt[w][t]; warpCnt[w][t] = 0; }
        cnt[t] += add;
        __syncthreads();
    }
    // runs of equal digits leave the tile as consecutive global addresses
    for (uint32_t k = t; k < tileValid; k += RS_THREADS) {
        const K kk = skeys[k];
        const uint32_t d = (uint32_t)((kk >> shift) & 255u);
        const uint32_t pos = digitBase[d] + (k - tileStart[d]);
        kout[pos] = kk;
        vout[pos] = svals[k];
    }
}

// sorts (keys, vals) stably by the low `bits` key bits; ping-pongs between the given buffers
// and returns true when the result ended up in the alternate buffers (kAlt, vAlt)
template <typename K, typename V>
bool RadixSortPairs(K* keys, V* vals, K* kAlt, V* vAlt, uint32_t n, uint32_t bits, uint32_t* tileHist,
                    uint32_t* digitTotals, cudaStream_t s, const uint64_t* orNot = nullptr) {
    if (n < 2) return false;
    const uint32_t nTiles = (n + RS_TILE - 1) / RS_TILE;
    K* ks = keys; V* vs = vals; K* kd = kAlt; V* vd = vAlt;
    bool alt = false;
    for (uint32_t shift = 0; shift < bits; shift += 8) {
        KRadixUpsweep<K><<<nTiles, RS_THREADS, 0, s>>>(ks, n, shift, tileHist, nTiles, orNot);
        KRadixScanRows<<<256, 256, 0, s>>>(tileHist, nTiles, digitTotals, shift, orNot);
        KRadixDownsweep<K, V><<<nTiles, RS_THREADS, 0, s>>>(ks, vs, kd, vd, n, shift, tileHist, digitTotals, nTiles,
                                                            orNot);
        K* tk = ks; ks = kd; kd = tk;
        V* tv = vs; vs = vd; vd = tv;
        alt = !alt;
    }
    return alt;
}
inline uint64_t RadixTileHistItems(uint32_t n) { return 256ull * ((n + RS_TILE - 1) / RS_TILE) + 256; }

}  // namespace tsp
