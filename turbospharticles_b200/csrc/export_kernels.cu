// export_kernels.cu -- export snapshot packing on the device (PackExportSnapshot,
// source/simulation/GPU/backend/gpu_backend.cpp:346-540 and CPU/backend/cpu_backend.cpp:829-975).
//
// The reference GPU backend copies every neighbor count, the whole compressed FF list, all
// positions and velocities to the host and classifies there. Here the classification and the
// compaction stay on the device and only the exported particles cross PCIe:
//   1. KSurfaceMark: a fluid particle is near-surface when it touches a boundary or rigid particle
//      or has fewer than `threshold` fluid neighbors (IsNearSurfaceFluidParticle,
//      core/backend_sim.h:109-117); it marks itself and every FF neighbor (plain byte stores of 1,
//      like the reference's relaxed atomic stores).
//   2. KSurfaceCount / KSurfaceScan / KSurfacePack: an ordered stream compaction of the marked
//      particles (the reference's sequential dst++ loop), writing x, y, z and
//      |v| = sqrt(vx*vx + vy*vy + vz*vz) (products and sums rounded separately, no contraction).
#include "kernels.h"

namespace tsp {

constexpr uint32_t EXP_THREADS = 256u;
constexpr uint32_t EXP_PER_THREAD = 4u;
constexpr uint32_t EXP_TILE = EXP_THREADS * EXP_PER_THREAD;

__global__ void __launch_bounds__(EXP_THREADS) KSurfaceMark(SellView ff, const uint16_t* __restrict__ cntFB,
                                                            const uint16_t* __restrict__ cntFR, uint32_t n,
                                                            uint32_t threshold, uint8_t* __restrict__ flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t cFF = ff.counts[i];
    const uint32_t cFB = cntFB ? cntFB[i] : 0u, cFR = cntFR ? cntFR[i] : 0u;
    if (!(cFB > 0u || cFR > 0u || cFF < threshold)) return;
    flags[i] = 1u;
    const uint32_t chunk = i / SELL_W, lane = i % SELL_W;
    const uint8_t fmt = ff.format[chunk];
    const uint32_t base = ff.base[chunk], base2 = ff.base2[chunk];
    const uint64_t off = ff.offset[chunk];
    for (uint32_t k = 0; k < cFF; k++) {
        const uint32_t j = SellNeighbor(fmt, base, base2, off, k, lane, ff.list16, ff.list32);
        if (j < n) flags[j] = 1u;
    }
}

// block-wide exclusive scan of one value per thread; returns the block total in `total`
__device__ __forceinline__ uint32_t BlockExclusiveScan(uint32_t v, uint32_t& total) {
    __shared__ uint32_t warpSums[EXP_THREADS / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = v;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= (uint32_t)d) incl += o;
    }
    if (lane == 31u) warpSums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < EXP_THREADS / 32 ? warpSums[lane] : 0u;
        uint32_t wi = w;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= (uint32_t)d) wi += o;
        }
        if (lane < EXP_THREADS / 32) warpSums[lane] = wi - w;
    }
    __syncthreads();
    const uint32_t before = warpSums[warp] + incl - v;
    // block total: last thread's inclusive value
    __shared__ uint32_t tot;
    if (threadIdx.x == EXP_THREADS - 1) tot = before + v;
    __syncthreads();
    total = tot;
    __syncthreads();
    return before;
}

__device__ __forceinline__ uint32_t TileFlags(const uint8_t* __restrict__ flags, uint32_t n, uint32_t first,
                                              uint32_t f[EXP_PER_THREAD]) {
    uint32_t c = 0;
    for (uint32_t q = 0; q < EXP_PER_THREAD; q++) {
        const uint32_t i = first + q;
        f[q] = (i < n) ? (uint32_t)(flags[i] != 0u) : 0u;
        c += f[q];
    }
    return c;
}

__global__ void __launch_bounds__(EXP_THREADS) KSurfaceCount(const uint8_t* __restrict__ flags, uint32_t n,
                                                             uint32_t* __restrict__ tileCounts) {
    uint32_t f[EXP_PER_THREAD];
    const uint32_t first = blockIdx.x * EXP_TILE + threadIdx.x * EXP_PER_THREAD;
    uint32_t total;
    BlockExclusiveScan(TileFlags(flags, n, first, f), total);
    if (threadIdx.x == 0) tileCounts[blockIdx.x] = total;
}

// one block: exclusive scan of the tile counts in place; out[0] = number of exported particles
__global__ void __launch_bounds__(EXP_THREADS) KSurfaceScan(uint32_t* __restrict__ tileCounts, uint32_t tiles,
                                                            uint32_t* __restrict__ out) {
    uint32_t carry = 0;
    for (uint32_t b = 0; b < tiles; b += EXP_THREADS) {
        const uint32_t t = b + threadIdx.x;
        const uint32_t v = t < tiles ? tileCounts[t] : 0u;
        uint32_t total;
        const uint32_t ex = BlockExclusiveScan(v, total);
        if (t < tiles) tileCounts[t] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) out[0] = carry;
}

__global__ void __launch_bounds__(EXP_THREADS) KSurfacePack(const uint8_t* __restrict__ flags, uint32_t n,
                                                            const uint32_t* __restrict__ tileOffsets,
                                                            const float4* __restrict__ posP,
                                                            const float4* __restrict__ velRho, uint64_t stride,
                                                            float* __restrict__ out) {
    uint32_t f[EXP_PER_THREAD];
    const uint32_t first = blockIdx.x * EXP_TILE + threadIdx.x * EXP_PER_THREAD;
    uint32_t total;
    uint32_t dst = tileOffsets[blockIdx.x] + BlockExclusiveScan(TileFlags(flags, n, first, f), total);
    for (uint32_t q = 0; q < EXP_PER_THREAD; q++) {
        if (!f[q]) continue;
        const uint32_t i = first + q;
        const float4 p = posP[i];
        const float4 v = velRho[i];
        const float vx2 = __fmul_rn(v.x, v.x), vy2 = __fmul_rn(v.y, v.y), vz2 = __fmul_rn(v.z, v.z);
        out[dst] = p.x;
        out[stride + dst] = p.y;
        out[2 * stride + dst] = p.z;
        out[3 * stride + dst] = __fsqrt_rn(__fadd_rn(__fadd_rn(vx2, vy2), vz2));
        dst++;
    }
}

__global__ void KMeshFlags(const uint64_t* __restrict__ idB, uint32_t n, uint64_t meshIdBegin,
                           uint8_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (uint8_t)(idB[i] >= meshIdBegin);
}

uint32_t ExportTiles(uint32_t n) { return (n + EXP_TILE - 1) / EXP_TILE; }

void LaunchExportSurface(const SellView& ff, const uint16_t* cntFB, const uint16_t* cntFR, uint32_t n,
                         uint32_t threshold, const float4* posP, const float4* velRho, uint8_t* flags,
                         uint32_t* tileCounts, uint32_t* nOut, float* out, uint64_t stride, cudaStream_t s) {
    const uint32_t tiles = ExportTiles(n);
    cudaMemsetAsync(flags, 0, n, s);
    KSurfaceMark<<<(n + EXP_THREADS - 1) / EXP_THREADS, EXP_THREADS, 0, s>>>(ff, cntFB, cntFR, n, threshold, flags);
    KSurfaceCount<<<tiles, EXP_THREADS, 0, s>>>(flags, n, tileCounts);
    KSurfaceScan<<<1, EXP_THREADS, 0, s>>>(tileCounts, tiles, nOut);
    KSurfacePack<<<tiles, EXP_THREADS, 0, s>>>(flags, n, tileCounts, posP, velRho, stride, out);
}

void LaunchMeshFlags(const uint64_t* idB, uint32_t n, uint64_t meshIdBegin, uint8_t* out, cudaStream_t s) {
    if (n) KMeshFlags<<<(n + 255) / 256, 256, 0, s>>>(idB, n, meshIdBegin, out);
}

}  // namespace tsp
