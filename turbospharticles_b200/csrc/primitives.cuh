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

template <typename K>
__global__ void __launch_bounds__(RS_THREADS) KRadixUpsweep(const K* __restrict__ keys, uint32_t n, uint32_t shift,
                                                          uint32_t* __restrict__ tileHist, uint32_t nTiles) {
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
                                                      uint32_t* __restrict__ digitTotals) {
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
                                                            const uint32_t* __restrict__ digitTotals, uint32_t nTiles) {
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
                    uint32_t* digitTotals, cudaStream_t s) {
    if (n < 2) return false;
    const uint32_t nTiles = (n + RS_TILE - 1) / RS_TILE;
    K* ks = keys; V* vs = vals; K* kd = kAlt; V* vd = vAlt;
    bool alt = false;
    for (uint32_t shift = 0; shift < bits; shift += 8) {
        KRadixUpsweep<K><<<nTiles, RS_THREADS, 0, s>>>(ks, n, shift, tileHist, nTiles);
        KRadixScanRows<<<256, 256, 0, s>>>(tileHist, nTiles, digitTotals);
        KRadixDownsweep<K, V><<<nTiles, RS_THREADS, 0, s>>>(ks, vs, kd, vd, n, shift, tileHist, digitTotals, nTiles);
        K* tk = ks; ks = kd; kd = tk;
        V* tv = vs; vs = vd; vd = tv;
        alt = !alt;
    }
    return alt;
}
inline uint64_t RadixTileHistItems(uint32_t n) { return 256ull * ((n + RS_TILE - 1) / RS_TILE) + 256; }

// ------------------------------------------------------------------------------ one-pass radix sort
// Stable LSD radix sort with one kernel per 8-bit digit pass (Merrill & Garland's "onesweep"):
// the key kernel also counts every pass's global digit histogram, and each pass kernel takes
// its tile in ticket order, ranks the tile's keys, publishes the tile's digit counts and finds
// the counts of all earlier tiles by a decoupled look-back (one status word per tile and digit:
// state in the two high bits, count in the low 30), then scatters. A tile publishes its own
// counts before it looks back, and earlier tiles hold earlier tickets, so every wait ends; the
// spin is bounded anyway (OS_SPIN_LIMIT, then an error bit). Same ordering rule, same
// permutation as RadixSortPairs: stable within a tile (tile index order via __match_any_sync
// ranks) and across tiles (ticket order = input order).
constexpr uint32_t OS_AGG = 1u << 30, OS_INC = 2u << 30, OS_VAL = (1u << 30) - 1u;
constexpr uint32_t OS_SPIN_LIMIT = 1u << 22;
constexpr uint32_t OS_MAX_PASSES = 8;

// layout of the sort's auxiliary words: [OS_MAX_PASSES][256] histogram, [OS_MAX_PASSES] tickets,
// padding, then [passes][nTiles][256] status words; all zero at the start of a sort
inline uint64_t OnesweepAuxWords(uint32_t n, uint32_t passes) {
    const uint64_t nTiles = (n + RS_TILE - 1) / RS_TILE;
    return 256ull * OS_MAX_PASSES + 64ull + (uint64_t)passes * nTiles * 256ull;
}
struct OnesweepAux {
    uint32_t* hist;
    uint32_t* tickets;
    uint32_t* status;
    uint32_t* err;     // error word (may be NULL)
    uint32_t errBit;
};
inline OnesweepAux OnesweepLayout(uint32_t* aux, uint32_t* err, uint32_t errBit) {
    return OnesweepAux{aux, aux + 256 * OS_MAX_PASSES, aux + 256 * OS_MAX_PASSES + 64, err, errBit};
}

// every pass's digit histogram of the given keys (warp-aggregated shared counters, one global
// atomic per non-zero bin and block); called by the key kernel for its own keys
__device__ __forceinline__ void OnesweepCountKey(uint64_t k, bool valid, uint32_t passes, uint32_t* sh) {
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t p = 0; p < passes; p++) {
        const uint32_t d = valid ? (uint32_t)((k >> (8u * p)) & 255u) : 256u + lane;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (d < 256u && (__ffs(peers) - 1) == (int)lane) atomicAdd(&sh[p * 256u + d], __popc(peers));
    }
}

template <typename K, typename V>
__global__ void __launch_bounds__(RS_THREADS) KOnesweepPass(const K* __restrict__ kin, const V* __restrict__ vin,
                                                          K* __restrict__ kout, V* __restrict__ vout, uint32_t n,
                                                          uint32_t pass, uint32_t nTiles, OnesweepAux a,
                                                          uint64_t* __restrict__ cidOut, uint64_t emptyKey) {
    __shared__ uint32_t sTile;
    __shared__ uint32_t digitBase[256];
    __shared__ uint32_t tileStart[256];
    __shared__ uint32_t cnt[256];
    __shared__ uint32_t warpCnt[RS_WARPS][256];
    __shared__ K skeys[RS_TILE];
    __shared__ V svals[RS_TILE];
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t shift = 8u * pass;
    if (t == 0) sTile = atomicAdd(&a.tickets[pass], 1u);
    // global exclusive digit bases of this pass; a pass whose digit is the same in every key
    // (one bin holds all n) is the identity permutation
    const uint32_t h = a.hist[pass * 256u + t];
    uint32_t gIncl = h;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, gIncl, d);
        if (lane >= d) gIncl += o;
    }
    if (lane == 31) warpCnt[0][warp] = gIncl;
    __syncthreads();
    uint32_t gPre = 0;
    for (uint32_t w = 0; w < warp; w++) gPre += warpCnt[0][w];
    const uint32_t gExcl = gPre + gIncl - h;
    const bool constant = __syncthreads_or(h == n) != 0;
    const uint32_t tile = sTile;
    const uint32_t base = tile * RS_TILE;
    const uint32_t tileValid = (n - base < (uint32_t)RS_TILE) ? (n - base) : (uint32_t)RS_TILE;
    if (constant) {
        for (uint32_t li = t; li < tileValid; li += RS_THREADS) {
            const K kk = kin[base + li];
            if (cidOut) cidOut[base + li] = ((uint64_t)kk == emptyKey) ? ~0ull : (uint64_t)kk;
            else kout[base + li] = kk;
            vout[base + li] = vin[base + li];
        }
        return;
    }
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
    cnt[t] = 0;
    for (int w = 0; w < RS_WARPS; w++) warpCnt[w][t] = 0;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        const uint32_t peers = __match_any_sync(0xffffffffu, dig[r]);
        if (dig[r] < 256u && (__ffs(peers) - 1) == (int)lane) atomicAdd(&cnt[dig[r]], __popc(peers));
    }
    __syncthreads();
    // publish this tile's count of digit t, then sum the counts of the earlier tiles
    const uint32_t mine = cnt[t];
    volatile uint32_t* st = a.status + (uint64_t)pass * nTiles * 256u;
    uint32_t prefix = 0;
    if (tile == 0) {
        st[t] = OS_INC | mine;
    } else {
        st[(uint64_t)tile * 256u + t] = OS_AGG | mine;
        for (uint32_t p = tile - 1;; p--) {
            uint32_t w = 0;
            for (uint32_t spins = 0; spins < OS_SPIN_LIMIT; spins++) {
                w = st[(uint64_t)p * 256u + t];
                if (w & ~OS_VAL) break;
            }
            if (!(w & ~OS_VAL)) {  // gave up: record it and stop (the result is then invalid)
                if (a.err) atomicOr(a.err, a.errBit);
                break;
            }
            prefix += w & OS_VAL;
            if ((w & ~OS_VAL) == OS_INC || p == 0) break;
        }
        st[(uint64_t)tile * 256u + t] = OS_INC | ((prefix + mine) & OS_VAL);
    }
    digitBase[t] = gExcl + prefix;
    // start of each digit's run inside the tile
    {
        uint32_t incl = mine;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += o;
        }
        __syncthreads();
        if (lane == 31) warpCnt[1][warp] = incl;
        __syncthreads();
        uint32_t pre = 0;
        for (uint32_t w = 0; w < warp; w++) pre += warpCnt[1][w];
        tileStart[t] = pre + incl - mine;
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
        if (pos >= n) continue;  // only after a look-back that gave up (error bit set)
        if (cidOut) cidOut[pos] = ((uint64_t)kk == emptyKey) ? ~0ull : (uint64_t)kk;
        else kout[pos] = kk;
        vout[pos] = svals[k];
    }
}

// the passes of a one-pass sort, keys and values ping-ponging between the given buffers (like
// RadixSortPairs); returns true when the result ended up in the alternate buffers
template <typename K, typename V>
bool OnesweepSortPairsPingPong(K* keys, V* vals, K* kAlt, V* vAlt, uint32_t n, uint32_t bits, const OnesweepAux& a,
                               cudaStream_t s) {
    const uint32_t nTiles = (n + RS_TILE - 1) / RS_TILE;
    const uint32_t passes = (bits + 7u) / 8u;
    K* ks = keys; V* vs = vals; K* kd = kAlt; V* vd = vAlt;
    bool alt = false;
    for (uint32_t p = 0; p < passes; p++) {
        KOnesweepPass<K, V><<<nTiles, RS_THREADS, 0, s>>>(ks, vs, kd, vd, n, p, nTiles, a, nullptr, 0ull);
        K* tk = ks; ks = kd; kd = tk;
        V* tv = vs; vs = vd; vd = tv;
        alt = !alt;
    }
    return alt;
}

// the passes of a one-pass sort over keys whose histograms the key kernel has counted into
// `a`; the last pass writes the sorted values to vFinal and the sorted keys, as cell IDs
// (emptyKey -> 0xFF..FF), to cidFinal. Keys and values ping-pong between the given buffers.
template <typename K, typename V>
void OnesweepSortPairs(K* keys, V* vals, K* kAlt, V* vAlt, uint32_t n, uint32_t bits, const OnesweepAux& a,
                       V* vFinal, uint64_t* cidFinal, uint64_t emptyKey, cudaStream_t s) {
    const uint32_t nTiles = (n + RS_TILE - 1) / RS_TILE;
    const uint32_t passes = (bits + 7u) / 8u;
    K* ks = keys; V* vs = vals; K* kd = kAlt; V* vd = vAlt;
    for (uint32_t p = 0; p < passes; p++) {
        const bool last = p + 1 == passes;
        KOnesweepPass<K, V><<<nTiles, RS_THREADS, 0, s>>>(ks, vs, last ? nullptr : kd, last ? vFinal : vd, n, p,
                                                          nTiles, a, last ? cidFinal : nullptr, emptyKey);
        K* tk = ks; ks = kd; kd = tk;
        V* tv = vs; vs = vd; vd = tv;
    }
}

}  // namespace tsp
