// stats_kernels.cu -- per-step statistics record (FillStatisticsRecord, source/simulation/GPU/
// backend/gpu_backend.cpp:1067-1203; metric list source/eval/stats/metrics.h:23-86).
//
// Neighbor counts of each relation: average from the totals the neighbor build already has,
// min / max / 99th percentile (index 99 (N - 1) / 100 of the sorted counts) from a 65,536-bin
// histogram of the u16 counts; blocks build shared-memory histograms of the low 2,048 values and
// send rarer values straight to the global histogram, then one block scans the histogram.
// Density errors and velocity magnitudes: per-block FP64 partial sums in a fixed order, folded
// by one block; min / max exact in FP32.
#include "kernels.h"

namespace tsp {

constexpr uint32_t STAT_BINS = 65536u;
constexpr uint32_t STAT_LOCAL_BINS = 2048u;
constexpr uint32_t STAT_THREADS = 256u;

__global__ void __launch_bounds__(STAT_THREADS) KStatHistogram(const uint16_t* __restrict__ counts, uint32_t n,
                                                               uint32_t* __restrict__ hist) {
    __shared__ uint32_t loc[STAT_LOCAL_BINS];
    for (uint32_t k = threadIdx.x; k < STAT_LOCAL_BINS; k += blockDim.x) loc[k] = 0u;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t v = counts[i];
        if (v < STAT_LOCAL_BINS) atomicAdd(&loc[v], 1u);
        else atomicAdd(&hist[v], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < STAT_LOCAL_BINS; k += blockDim.x)
        if (loc[k]) atomicAdd(&hist[k], loc[k]);
}

// one block of 1024 threads: thread t owns bins [64 t, 64 t + 64)
__global__ void __launch_bounds__(1024) KStatHistogramScan(const uint32_t* __restrict__ hist, uint32_t n,
                                                           uint32_t* __restrict__ out /* min, max, p99 */) {
    constexpr uint32_t PER = STAT_BINS / 1024u;
    const uint32_t t = threadIdx.x, b0 = t * PER;
    uint32_t sum = 0, first = EMPTY_32, last = 0;
    bool any = false;
    for (uint32_t k = 0; k < PER; k++) {
        const uint32_t c = hist[b0 + k];
        sum += c;
        if (c) { if (!any) first = b0 + k; last = b0 + k; any = true; }
    }
    // block exclusive scan of the per-thread sums (64-bit: up to 2^32 counts)
    __shared__ unsigned long long ws[32];
    unsigned long long incl = sum;
    const uint32_t lane = t & 31, warp = t >> 5;
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= (uint32_t)d) incl += o;
    }
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = ws[lane], wi = w;
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long o = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= (uint32_t)d) wi += o;
        }
        ws[lane] = wi - w;  // exclusive warp prefix
    }
    __syncthreads();
    const unsigned long long before = ws[warp] + incl - sum;
    __shared__ uint32_t mn, mx, p99;
    if (t == 0) { mn = EMPTY_32; mx = 0; p99 = 0; }
    __syncthreads();
    if (any) { atomicMin(&mn, first); atomicMax(&mx, last); }
    if (n > 0) {
        const unsigned long long i99 = (99ull * (unsigned long long)(n - 1u)) / 100ull;
        if (i99 >= before && i99 < before + sum) {
            unsigned long long acc = before;
            for (uint32_t k = 0; k < PER; k++) {
                acc += hist[b0 + k];
                if (i99 < acc) { p99 = b0 + k; break; }
            }
        }
    }
    __syncthreads();
    if (t == 0) {
        out[0] = (n > 0 && mn != EMPTY_32) ? mn : 0u;
        out[1] = n > 0 ? mx : 0u;
        out[2] = p99;
    }
}

// density (rho / rho0 - 1: raw, positive part, absolute) and velocity magnitude (sum, min, max)
__global__ void __launch_bounds__(STAT_THREADS) KStatFields(const float4* __restrict__ velRho, uint32_t n, float rho0,
                                                            double* __restrict__ partials, float* __restrict__ mm) {
    double s[4] = {0, 0, 0, 0};
    float vmin = 3.402823466e38f, vmax = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v = velRho[i];
        const float rel = (v.w / rho0) - 1.0f;
        s[0] += rel;
        s[1] += fmaxf(0.0f, rel);
        s[2] += fabsf(rel);
        const float mag = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
        s[3] += mag;
        vmin = fminf(vmin, mag);
        vmax = fmaxf(vmax, mag);
    }
    __shared__ double sm[4][STAT_THREADS / 32];
    __shared__ float smn[STAT_THREADS / 32], smx[STAT_THREADS / 32];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < 4; q++) {
        double v = s[q];
        for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        if (lane == 0) sm[q][warp] = v;
    }
    for (int d = 16; d > 0; d >>= 1) {
        vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, d));
        vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, d));
    }
    if (lane == 0) { smn[warp] = vmin; smx[warp] = vmax; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < 4; q++) {
            double t = 0.0;
            for (uint32_t w = 0; w < STAT_THREADS / 32; w++) t += sm[q][w];
            partials[4ull * blockIdx.x + q] = t;
        }
        float a = smn[0], b = smx[0];
        for (uint32_t w = 1; w < STAT_THREADS / 32; w++) { a = fminf(a, smn[w]); b = fmaxf(b, smx[w]); }
        mm[2ull * blockIdx.x] = a;
        mm[2ull * blockIdx.x + 1] = b;
    }
}
__global__ void KStatFieldsFold(const double* __restrict__ partials, const float* __restrict__ mm, uint32_t blocks,
                                double* __restrict__ out /* raw, pos, abs, velSum, velMin, velMax */) {
    if (threadIdx.x != 0) return;
    double s[4] = {0, 0, 0, 0};
    float a = 3.402823466e38f, b = 0.0f;
    for (uint32_t k = 0; k < blocks; k++) {
        for (int q = 0; q < 4; q++) s[q] += partials[4ull * k + q];
        a = fminf(a, mm[2ull * k]);
        b = fmaxf(b, mm[2ull * k + 1]);
    }
    for (int q = 0; q < 4; q++) out[q] = s[q];
    out[4] = blocks ? a : 0.0;
    out[5] = b;
}

uint32_t StatFieldBlocks(uint32_t n) { return std::max<uint32_t>(1u, std::min<uint32_t>((n + STAT_THREADS - 1) / STAT_THREADS, 148u * 8u)); }

void LaunchStatNeighborCounts(const uint16_t* counts, uint32_t n, uint32_t* hist, uint32_t* out, cudaStream_t s) {
    cudaMemsetAsync(hist, 0, STAT_BINS * sizeof(uint32_t), s);
    if (n) KStatHistogram<<<std::min<uint32_t>((n + STAT_THREADS - 1) / STAT_THREADS, 148u * 4u), STAT_THREADS, 0, s>>>(
        counts, n, hist);
    KStatHistogramScan<<<1, 1024, 0, s>>>(hist, n, out);
}
void LaunchStatFields(const float4* velRho, uint32_t n, float rho0, double* partials, float* mm, double* out,
                      cudaStream_t s) {
    const uint32_t blocks = StatFieldBlocks(n);
    KStatFields<<<blocks, STAT_THREADS, 0, s>>>(velRho, n, rho0, partials, mm);
    KStatFieldsFold<<<1, 32, 0, s>>>(partials, mm, blocks, out);
}

}  // namespace tsp
