// surface_kernels.cu -- mesh surface sampling on the GPU (Scene::SurfaceSampler,
// source/simulation/scene/geometry/surface_sampling.cpp), for mesh boundaries and mesh rigid
// bodies.
//
// Same decisions as the reference, step for step:
//   * candidates: seeded splitmix64 stream, area-proportional triangle (lower bound on the FP64
//     cumulative areas), uniform barycentric point (KCandidates), batched as the reference;
//   * per batch a stable radix sort by (cell phase group, z, y, x) and the per-cell candidate
//     ranges (KCellRanges); then, per candidate round and phase group (the order alternates per
//     batch), every cell's candidate is tested against the accepted samples in parallel
//     (KTestGroup: no sample closer than the minimum distance in the 3x3x3 cells) and the
//     accepted ones are appended in cell order and inserted into the sample hash
//     (KAppendGroup). Cells of one phase group cannot see each other, which is what makes the
//     reference's parallel group test exact;
//   * coverage: barycentric probe lattices per triangle, tested in batches of 10^6 against the
//     samples of the batch start (KProbeTest), uncovered probes compacted in probe order and
//     re-tested one after another by one warp, each still-uncovered probe becoming a sample
//     (KRepair) -- the reference's sequential repair loop.
// The sample hash: open addressing on packed cell coordinates (21 bits per axis) with a
// per-cell linked list of sample indices; every probe loop and list walk is bounded by the
// table / sample capacity and reports an error flag instead of running on.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "host_common.h"
#include "primitives.cuh"

namespace tsp {

namespace {

constexpr uint64_t EMPTY_KEY = ~0ull;
constexpr uint32_t NO_SAMPLE = 0xffffffffu;
constexpr int32_t HASH_OFF = 1 << 20;         // packed cell coordinate offset (21 bits per axis)
constexpr int32_t SORT_OFF = 1 << 19;         // candidate sort key offset (20 bits per axis)
constexpr uint32_t SURF_ERR_HASH = 1u, SURF_ERR_CAP = 2u, SURF_ERR_LIST = 4u;

__host__ __device__ __forceinline__ uint64_t Mix64(uint64_t h) {  // splitmix64 finalizer
    h = (h ^ (h >> 30)) * 0xbf58476d1ce4e5b9ull;
    h = (h ^ (h >> 27)) * 0x94d049bb133111ebull;
    return h ^ (h >> 31);
}
__device__ __forceinline__ double Random01(uint64_t seed, uint64_t streamIdx) {
    const uint64_t h = Mix64(seed + (streamIdx + 1ull) * 0x9e3779b97f4a7c15ull);
    return (double)(h >> 11) * 0x1.0p-53;
}
// floor(v * inv) of the exact product (two floats multiply exactly in FP64)
__device__ __forceinline__ int32_t CellAxis(float v, float inv) { return (int32_t)floor((double)v * (double)inv); }

struct Tris {
    const float4 *v0, *v1, *v2;
    const double* cum;
    const uint32_t* sub;
    const uint64_t* probeBegin;
    uint32_t n;
    double area;
};

// barycentric point v0 b.x + v1 b.y + v2 b.z, products and sums rounded separately (glm order)
__device__ __forceinline__ float3 SurfacePoint(const Tris& T, uint32_t t, float bx, float by, float bz) {
    const float4 a = T.v0[t], b = T.v1[t], c = T.v2[t];
    return make_float3(__fadd_rn(__fadd_rn(__fmul_rn(a.x, bx), __fmul_rn(b.x, by)), __fmul_rn(c.x, bz)),
                       __fadd_rn(__fadd_rn(__fmul_rn(a.y, bx), __fmul_rn(b.y, by)), __fmul_rn(c.y, bz)),
                       __fadd_rn(__fadd_rn(__fmul_rn(a.z, bx), __fmul_rn(b.z, by)), __fmul_rn(c.z, bz)));
}
// glm::distance: sqrt((dx*dx + dy*dy) + dz*dz)
__device__ __forceinline__ float Dist(float3 a, float4 b) {
    const float dx = __fsub_rn(b.x, a.x), dy = __fsub_rn(b.y, a.y), dz = __fsub_rn(b.z, a.z);
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}

struct Hash {
    uint64_t* keys;
    uint32_t* head;
    uint32_t* next;
    uint32_t mask;  // capacity - 1 (power of two)
    float inv;      // 1 / cell size
};
__device__ __forceinline__ uint64_t PackCell(int32_t x, int32_t y, int32_t z) {
    return ((uint64_t)(uint32_t)(x + HASH_OFF) & 0x1fffffull) | (((uint64_t)(uint32_t)(y + HASH_OFF) & 0x1fffffull) << 21) |
           (((uint64_t)(uint32_t)(z + HASH_OFF) & 0x1fffffull) << 42);
}
__device__ __forceinline__ uint32_t FindSlot(const Hash& h, uint64_t key, uint32_t* err) {
    uint32_t s = (uint32_t)Mix64(key) & h.mask;
    for (uint32_t probe = 0; probe <= h.mask; probe++) {
        const uint64_t k = h.keys[s];
        if (k == key) return s;
        if (k == EMPTY_KEY) return NO_SAMPLE;
        s = (s + 1u) & h.mask;
    }
    atomicOr(err, SURF_ERR_HASH);
    return NO_SAMPLE;
}
__device__ void HashInsert(const Hash& h, float3 p, uint32_t sample, uint32_t* err) {
    const uint64_t key = PackCell(CellAxis(p.x, h.inv), CellAxis(p.y, h.inv), CellAxis(p.z, h.inv));
    uint32_t s = (uint32_t)Mix64(key) & h.mask;
    for (uint32_t probe = 0; probe <= h.mask; probe++) {
        const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(h.keys + s),
                                                  (unsigned long long)EMPTY_KEY, (unsigned long long)key);
        if (prev == EMPTY_KEY || prev == key) {
            h.next[sample] = atomicExch(h.head + s, sample);
            return;
        }
        s = (s + 1u) & h.mask;
    }
    atomicOr(err, SURF_ERR_HASH);
}
// any sample within `radius` (strict: < radius, else <= radius) in the 3x3x3 cells around p
template <bool STRICT>
__device__ bool HashAny(const Hash& h, const float4* __restrict__ samples, uint32_t nSamples, float3 p, float radius,
                        uint32_t* err) {
    const int32_t cx = CellAxis(p.x, h.inv), cy = CellAxis(p.y, h.inv), cz = CellAxis(p.z, h.inv);
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const uint32_t slot = FindSlot(h, PackCell(cx + dx, cy + dy, cz + dz), err);
                if (slot == NO_SAMPLE) continue;
                uint32_t i = h.head[slot];
                for (uint32_t walk = 0; i != NO_SAMPLE; walk++) {
                    if (walk > nSamples || i >= nSamples) { atomicOr(err, SURF_ERR_LIST); return false; }
                    const float d = Dist(p, samples[i]);
                    if (STRICT ? (d < radius) : (d <= radius)) return true;
                    i = h.next[i];
                }
            }
    return false;
}

__global__ void KCandidates(Tris T, uint64_t seed, uint64_t first, uint32_t nb, float cellInv, float4* __restrict__ cand,
                            uint64_t* __restrict__ key, uint32_t* __restrict__ idx) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint64_t s = 3ull * (first + b);
    const double target = Random01(seed, s) * T.area;
    const float scale = __fsqrt_rn((float)Random01(seed, s + 1));
    const float off = (float)Random01(seed, s + 2);
    uint32_t lo = 0, hi = T.n;  // first triangle with cumulative area >= target
    while (lo < hi) {
        const uint32_t m = (lo + hi) >> 1;
        if (T.cum[m] < target) lo = m + 1; else hi = m;
    }
    const uint32_t t = lo == T.n ? T.n - 1 : lo;
    const float b1 = __fmul_rn(scale, __fsub_rn(1.0f, off));
    const float3 p = SurfacePoint(T, t, __fsub_rn(1.0f, scale), b1, __fsub_rn(scale, b1));
    cand[b] = make_float4(p.x, p.y, p.z, 0.0f);
    const int32_t x = CellAxis(p.x, cellInv), y = CellAxis(p.y, cellInv), z = CellAxis(p.z, cellInv);
    const uint64_t phase = (uint64_t)((x & 1) | ((y & 1) << 1) | ((z & 1) << 2));
    key[b] = (phase << 60) | ((uint64_t)(uint32_t)(z + SORT_OFF) << 40) | ((uint64_t)(uint32_t)(y + SORT_OFF) << 20) |
             (uint64_t)(uint32_t)(x + SORT_OFF);
    idx[b] = b;
}

// one block: cell run starts of the sorted keys, per phase group first cell, largest cell size.
// meta = {nCells, groupBegin[0..8], maxPerCell}
__global__ void __launch_bounds__(SCAN_THREADS) KCellRanges(const uint64_t* __restrict__ key, uint32_t nb,
                                                            uint32_t* __restrict__ cellBegin, uint32_t* __restrict__ meta) {
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nb; base += SCAN_THREADS) {
        const uint32_t k = base + threadIdx.x;
        const uint32_t start = (k < nb && (k == 0 || key[k] != key[k - 1])) ? 1u : 0u;
        uint32_t total;
        const uint32_t ex = BlockExclusiveScan<uint32_t>(start, total);
        if (start) cellBegin[carry + ex] = k;
        carry += total;
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x == 0) cellBegin[carry] = nb;
    __syncthreads();
    __shared__ uint32_t mx;
    if (threadIdx.x == 0) mx = 0;
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < carry; c += SCAN_THREADS) {
        atomicMax(&mx, cellBegin[c + 1] - cellBegin[c]);
        const uint32_t g = (uint32_t)(key[cellBegin[c]] >> 60);
        const uint32_t gPrev = c == 0 ? 0u : (uint32_t)(key[cellBegin[c - 1]] >> 60);
        // cells of groups gPrev+1 .. g (and group 0 for c == 0) begin at c
        for (uint32_t q = (c == 0 ? 0u : gPrev + 1); q <= g; q++) meta[1 + q] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t gLast = carry ? (uint32_t)(key[cellBegin[carry - 1]] >> 60) : 0u;
        for (uint32_t q = carry ? gLast + 1 : 0u; q <= 8; q++) meta[1 + q] = carry;
        meta[0] = carry;
        meta[10] = mx;
    }
}

__global__ void KTestGroup(const float4* __restrict__ cand, const uint32_t* __restrict__ idx,
                           const uint32_t* __restrict__ cellBegin, uint32_t cb, uint32_t ce, uint32_t round, Hash h,
                           const float4* __restrict__ samples, const uint32_t* __restrict__ nSamples, float minD,
                           uint8_t* __restrict__ accept, uint32_t* err) {
    const uint32_t c = cb + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ce) return;
    const uint32_t k = cellBegin[c] + round;
    uint8_t a = 0;
    if (k < cellBegin[c + 1]) {
        const float4 q = cand[idx[k]];
        a = HashAny<true>(h, samples, *nSamples, make_float3(q.x, q.y, q.z), minD, err) ? 0 : 1;
    }
    accept[c - cb] = a;
}

// one block: append the accepted candidates of cells [cb, ce) in cell order and insert them
__global__ void __launch_bounds__(SCAN_THREADS) KAppendGroup(const float4* __restrict__ cand, const uint32_t* __restrict__ idx,
                                                             const uint32_t* __restrict__ cellBegin, uint32_t cb, uint32_t ce,
                                                             uint32_t round, const uint8_t* __restrict__ accept, Hash h,
                                                             float4* __restrict__ samples, uint32_t* nSamples, uint32_t cap,
                                                             uint32_t* err) {
    const uint32_t n0 = *nSamples;
    uint32_t carry = 0;
    for (uint32_t base = cb; base < ce; base += SCAN_THREADS) {
        const uint32_t c = base + threadIdx.x;
        const uint32_t a = (c < ce && accept[c - cb]) ? 1u : 0u;
        uint32_t total;
        const uint32_t ex = BlockExclusiveScan<uint32_t>(a, total);
        if (a) {
            const uint32_t s = n0 + carry + ex;
            if (s < cap) {
                const float4 q = cand[idx[cellBegin[c] + round]];
                samples[s] = q;
                HashInsert(h, make_float3(q.x, q.y, q.z), s, err);
            } else {
                atomicOr(err, SURF_ERR_CAP);
            }
        }
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *nSamples = min(cap, n0 + carry);
}

__global__ void KInsertAll(Hash h, const float4* __restrict__ samples, uint32_t n, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 q = samples[i];
    HashInsert(h, make_float3(q.x, q.y, q.z), i, err);
}

// probe lattice point of a global probe index (locateProbe + MakeProbe, surface_sampling.cpp:857-877, 368-381)
__device__ float3 ProbePoint(const Tris& T, uint64_t probe) {
    uint32_t lo = 0, hi = T.n;  // last triangle whose first probe <= probe
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (T.probeBegin[m] <= probe) lo = m; else hi = m;
    }
    const uint32_t t = lo;
    const uint32_t n = T.sub[t];
    const uint64_t lattice = probe - T.probeBegin[t];
    uint32_t i = 0, rowHigh = n;
    while (i < rowHigh) {
        const uint32_t mid = i + (rowHigh - i + 1) / 2;
        if ((uint64_t)mid * (2ull * n + 3ull - mid) / 2ull <= lattice) i = mid; else rowHigh = mid - 1;
    }
    const uint32_t j = (uint32_t)(lattice - (uint64_t)i * (2ull * n + 3ull - i) / 2ull);
    const float ninv = __fdiv_rn(1.0f, (float)n);
    const uint32_t k = n - i - j;
    return SurfacePoint(T, t, __fmul_rn((float)i, ninv), __fmul_rn((float)j, ninv), __fmul_rn((float)k, ninv));
}

__global__ void KProbeTest(Tris T, uint64_t begin, uint32_t count, Hash h, const float4* __restrict__ samples,
                           const uint32_t* __restrict__ nSamples, float target, uint8_t* __restrict__ uncovered,
                           uint32_t* err) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const float3 p = ProbePoint(T, begin + k);
    uncovered[k] = HashAny<false>(h, samples, *nSamples, p, target, err) ? 0 : 1;
}

// one block: probe indices of the uncovered flags, in probe order; out[count] = their number
__global__ void __launch_bounds__(SCAN_THREADS) KCompactProbes(const uint8_t* __restrict__ uncovered, uint32_t count,
                                                               uint64_t begin, uint64_t* __restrict__ out,
                                                               uint32_t* __restrict__ nOut) {
    uint32_t carry = 0;
    for (uint32_t base = 0; base < count; base += SCAN_THREADS) {
        const uint32_t k = base + threadIdx.x;
        const uint32_t u = (k < count && uncovered[k]) ? 1u : 0u;
        uint32_t total;
        const uint32_t ex = BlockExclusiveScan<uint32_t>(u, total);
        if (u) out[carry + ex] = begin + k;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *nOut = carry;
}

// one warp: re-test each uncovered probe in probe order and turn the still-uncovered ones into
// samples (lanes 0..26 each walk one of the 27 cells; lane 0 appends and inserts)
__global__ void __launch_bounds__(32) KRepair(Tris T, const uint64_t* __restrict__ probes, const uint32_t* __restrict__ nProbes,
                                              Hash h, float4* __restrict__ samples, uint32_t* nSamples, uint32_t cap,
                                              float target, uint32_t* repairs, uint32_t* err) {
    const uint32_t lane = threadIdx.x;
    const uint32_t np = *nProbes;
    uint32_t n = *nSamples, rep = 0;
    for (uint32_t u = 0; u < np; u++) {
        const float3 p = ProbePoint(T, probes[u]);
        bool hit = false;
        if (lane < 27) {
            const int dx = (int)(lane % 3) - 1, dy = (int)((lane / 3) % 3) - 1, dz = (int)(lane / 9) - 1;
            const uint32_t slot = FindSlot(h, PackCell(CellAxis(p.x, h.inv) + dx, CellAxis(p.y, h.inv) + dy,
                                                       CellAxis(p.z, h.inv) + dz), err);
            if (slot != NO_SAMPLE) {
                uint32_t i = h.head[slot];
                for (uint32_t walk = 0; i != NO_SAMPLE && !hit; walk++) {
                    if (walk > n || i >= n) { atomicOr(err, SURF_ERR_LIST); break; }
                    hit = Dist(p, samples[i]) <= target;
                    i = h.next[i];
                }
            }
        }
        const bool covered = __any_sync(0xffffffffu, hit);
        if (!covered) {
            if (lane == 0) {
                if (n < cap) {
                    samples[n] = make_float4(p.x, p.y, p.z, 0.0f);
                    HashInsert(h, p, n, err);
                } else {
                    atomicOr(err, SURF_ERR_CAP);
                }
            }
            n = min(cap, n + 1);
            rep++;
        }
        __syncwarp();
    }
    if (lane == 0) { *nSamples = n; *repairs += rep; }
}

template <typename T>
struct Buf {  // device buffer owned by one sampling call
    T* p = nullptr;
    explicit Buf(size_t n) { CK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T))); }
    ~Buf() { if (p) cudaFree(p); }
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
};

float DistanceEpsilon(float d) {
    return 32.0f * std::numeric_limits<float>::epsilon() * std::max(std::fabs(d), std::numeric_limits<float>::min());
}
uint32_t NextPow2(uint64_t v) {
    uint64_t p = 1024;
    while (p < v) p <<= 1;
    if (p > (1ull << 31)) throw Error(TSP_ERR_UNSUPPORTED, "surface sample hash exceeds 2^31 cells");
    return (uint32_t)p;
}

}  // namespace

std::vector<float> SampleSurfaceGpu(int device, const float* vtx, uint32_t nV, const uint32_t* tri, uint32_t nT,
                                    const tsp_surface_sampling_params& p, tsp_surface_sampling_stats& st) {
    const float minD = p.minDistance, maxD = p.maxDistance, probeS = p.coverageProbeSpacing;
    auto invalid = [](const char* m) { return Error(TSP_ERR_INVALID, m); };
    // ---- PreprocessMesh (surface_sampling.cpp:455-578), host
    if (!vtx || !tri || nV == 0 || nT == 0) throw invalid("Cannot sample an empty triangle surface.");
    if (!std::isfinite(p.particleSizeF) || p.particleSizeF <= 0.0f)
        throw invalid("Surface sampling requires a finite positive fluid particle size.");
    if (maxD > p.particleSizeF + DistanceEpsilon(p.particleSizeF)) throw invalid("Surface sampling is coarser than the fluid spacing.");
    if (!std::isfinite(minD) || minD <= 0.0f) throw invalid("Surface sample minimum distance must be finite and positive.");
    if (!std::isfinite(maxD) || maxD < minD)
        throw invalid("Surface sample maximum distance must be finite and not smaller than the minimum distance.");
    if (!std::isfinite(probeS) || probeS <= 0.0f) throw invalid("Surface coverage probe spacing must be finite and positive.");
    if (maxD + DistanceEpsilon(maxD) < minD + probeS)
        throw invalid("Surface coverage maximum distance must be at least the minimum distance plus the probe spacing.");
    if (p.candidateMultiplier == 0) throw invalid("Surface sampling candidate multiplier must be positive.");
    for (uint64_t i = 0; i < 3ull * nV; i++)
        if (!std::isfinite(vtx[i])) throw invalid("Triangle surface contains a non-finite vertex.");
    for (uint64_t i = 0; i < 3ull * nT; i++)
        if (tri[i] >= nV) throw invalid("Triangle surface contains an invalid vertex index.");
    std::vector<float4> v0(nT), v1(nT), v2(nT);
    std::vector<double> cum(nT);
    std::vector<uint32_t> sub(nT);
    std::vector<uint64_t> pbeg(nT + 1ull, 0);
    double area = 0.0;
    float bmin[3] = {vtx[0], vtx[1], vtx[2]}, bmax[3] = {vtx[0], vtx[1], vtx[2]};
    for (uint64_t i = 0; i < nV; i++)
        for (int a = 0; a < 3; a++) { bmin[a] = std::min(bmin[a], vtx[3 * i + a]); bmax[a] = std::max(bmax[a], vtx[3 * i + a]); }
    auto len = [](float x, float y, float z) { return std::sqrt((x * x + y * y) + z * z); };
    for (uint32_t t = 0; t < nT; t++) {
        const float* a = vtx + 3ull * tri[3ull * t];
        const float* b = vtx + 3ull * tri[3ull * t + 1];
        const float* c = vtx + 3ull * tri[3ull * t + 2];
        const float ux = b[0] - a[0], uy = b[1] - a[1], uz = b[2] - a[2];
        const float wx = c[0] - a[0], wy = c[1] - a[1], wz = c[2] - a[2];
        const float cx = uy * wz - wy * uz, cy = uz * wx - wz * ux, cz = ux * wy - wx * uy;
        const float ar = 0.5f * len(cx, cy, cz);
        const float e = std::max(len(b[0] - a[0], b[1] - a[1], b[2] - a[2]),
                                 std::max(len(c[0] - b[0], c[1] - b[1], c[2] - b[2]), len(a[0] - c[0], a[1] - c[1], a[2] - c[2])));
        if (!std::isfinite(ar) || ar <= 0.0f) throw invalid("Triangle surface contains a degenerate triangle.");
        area += (double)ar;
        if (!std::isfinite(area) || area > std::numeric_limits<float>::max())
            throw invalid("Triangle surface area exceeds float limits.");
        v0[t] = make_float4(a[0], a[1], a[2], 0.f); v1[t] = make_float4(b[0], b[1], b[2], 0.f);
        v2[t] = make_float4(c[0], c[1], c[2], 0.f);
        cum[t] = area;
        const double d = std::ceil(e / probeS);
        if (!std::isfinite(d) || d >= (double)UINT32_MAX) throw invalid("Surface probe subdivision count exceeds uint32 loop limits.");
        sub[t] = std::max<uint32_t>(1u, (uint32_t)d);
        const uint64_t per = (sub[t] + 1ull) * (sub[t] + 2ull) / 2ull;
        if (per > UINT64_MAX - pbeg[t]) throw invalid("Surface coverage probe count exceeds uint64 limits.");
        pbeg[t + 1] = pbeg[t] + per;
    }
    st = tsp_surface_sampling_stats{};
    st.surfaceArea = (float)area;
    const double nEstD = std::ceil(area / ((double)minD * (double)minD));
    if (!std::isfinite(nEstD) || nEstD < 0.0 || nEstD > (double)UINT32_MAX)
        throw invalid("Surface estimated sample count exceeds uint32 limits.");
    const uint64_t nCand = std::max<uint64_t>(1, (uint64_t)nEstD * p.candidateMultiplier);
    const uint32_t nEst = std::max<uint32_t>(1, (uint32_t)nEstD);
    const uint32_t batchMax = (uint32_t)std::min<uint64_t>(nCand, std::min<uint32_t>(1000000u, std::max<uint32_t>(1u, nEst / 16)));
    const uint64_t nProbes = pbeg[nT];
    st.N_candidates = nCand;
    st.N_coverageProbes = nProbes;
    const float target = std::max(minD, maxD - probeS);
    // cell coordinates of every sample stay inside the sort-key and hash packing ranges
    for (float cs : {minD, target})
        for (int a = 0; a < 3; a++) {
            const double lo = std::floor((double)bmin[a] / (double)cs) - 4.0, hi = std::floor((double)bmax[a] / (double)cs) + 4.0;
            if (lo <= -(double)SORT_OFF || hi >= (double)SORT_OFF)
                throw Error(TSP_ERR_UNSUPPORTED, "mesh extent exceeds 2^19 sampling cells per axis");
        }
    const uint64_t capU = std::min<uint64_t>(nCand + nProbes, (uint64_t)INT32_MAX);
    const uint32_t cap = (uint32_t)capU;
    const uint32_t H = NextPow2(2ull * capU);
    // ---- device state (all validation above runs without touching the GPU)
    int nDev = 0;
    if (cudaGetDeviceCount(&nDev) != cudaSuccess || nDev == 0) throw Error(TSP_ERR_NO_DEVICE, "no CUDA device");
    if (device >= 0) CK(cudaSetDevice(device));
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); } } sg{s};
    Buf<float4> dv0(nT), dv1(nT), dv2(nT);
    Buf<double> dcum(nT);
    Buf<uint32_t> dsub(nT);
    Buf<uint64_t> dpb(nT + 1ull);
    CK(cudaMemcpyAsync(dv0.p, v0.data(), nT * sizeof(float4), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dv1.p, v1.data(), nT * sizeof(float4), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dv2.p, v2.data(), nT * sizeof(float4), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dcum.p, cum.data(), nT * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dsub.p, sub.data(), nT * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dpb.p, pbeg.data(), (nT + 1ull) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    const Tris T{dv0.p, dv1.p, dv2.p, dcum.p, dsub.p, dpb.p, nT, area};
    Buf<float4> samples(cap);
    Buf<uint64_t> hkeys(H);
    Buf<uint32_t> hhead(H), hnext(cap);
    Buf<uint32_t> ctr(4);  // nSamples, error flags, repairs, uncovered count
    CK(cudaMemsetAsync(ctr.p, 0, 4 * sizeof(uint32_t), s));
    auto resetHash = [&]() {
        CK(cudaMemsetAsync(hkeys.p, 0xff, (size_t)H * sizeof(uint64_t), s));
        CK(cudaMemsetAsync(hhead.p, 0xff, (size_t)H * sizeof(uint32_t), s));
    };
    Hash h{hkeys.p, hhead.p, hnext.p, H - 1u, 1.0f / minD};
    resetHash();
    uint32_t* nS = ctr.p;
    uint32_t* err = ctr.p + 1;
    // ---- SelectPoissonSamples (:580-813)
    {
        Buf<float4> cand(batchMax);
        Buf<uint64_t> key(batchMax), key2(batchMax);
        Buf<uint32_t> idx(batchMax), idx2(batchMax), cellBegin(batchMax + 1ull), meta(16);
        Buf<uint8_t> accept(batchMax);
        Buf<uint32_t> tileHist(RadixTileHistItems(batchMax)), digitTotals(256);
        const float cellInv = 1.0f / minD;
        for (uint64_t first = 0; first < nCand;) {
            const uint32_t nb = (uint32_t)std::min<uint64_t>(nCand - first, batchMax);
            KCandidates<<<(nb + 255) / 256, 256, 0, s>>>(T, p.seed, first, nb, cellInv, cand.p, key.p, idx.p);
            const bool alt = RadixSortPairs<uint64_t, uint32_t>(key.p, idx.p, key2.p, idx2.p, nb, 63, tileHist.p,
                                                                 digitTotals.p, s);
            const uint64_t* sk = alt ? key2.p : key.p;
            const uint32_t* si = alt ? idx2.p : idx.p;
            KCellRanges<<<1, SCAN_THREADS, 0, s>>>(sk, nb, cellBegin.p, meta.p);
            uint32_t m[11];
            CK(cudaMemcpyAsync(m, meta.p, sizeof(m), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            const bool reversed = (first / batchMax) % 2 == 1;
            for (uint32_t r = 0; r < m[10]; r++)
                for (uint32_t step = 0; step < 8; step++) {
                    const uint32_t g = reversed ? 7 - step : step;
                    const uint32_t cb = m[1 + g], ce = m[2 + g];
                    if (ce <= cb) continue;
                    KTestGroup<<<(ce - cb + 255) / 256, 256, 0, s>>>(cand.p, si, cellBegin.p, cb, ce, r, h, samples.p, nS,
                                                                      minD, accept.p, err);
                    KAppendGroup<<<1, SCAN_THREADS, 0, s>>>(cand.p, si, cellBegin.p, cb, ce, r, accept.p, h, samples.p, nS,
                                                            cap, err);
                }
            first += nb;
        }
        CK(cudaGetLastError());
    }
    uint32_t hc[4];
    CK(cudaMemcpyAsync(hc, ctr.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (hc[1]) throw Error(TSP_ERR_UNSUPPORTED, "surface sampling hash / capacity error");
    st.N_initialSamples = hc[0];
    // ---- RepairCoverage (:833-968)
    h.inv = 1.0f / target;
    resetHash();
    if (hc[0]) KInsertAll<<<(hc[0] + 255) / 256, 256, 0, s>>>(h, samples.p, hc[0], err);
    {
        const uint32_t batch = (uint32_t)std::min<uint64_t>(nProbes, 1000000ull);
        Buf<uint8_t> unc(batch);
        Buf<uint64_t> uncIdx(batch);
        for (uint64_t begin = 0; begin < nProbes;) {
            const uint32_t count = (uint32_t)std::min<uint64_t>(nProbes - begin, 1000000ull);
            KProbeTest<<<(count + 255) / 256, 256, 0, s>>>(T, begin, count, h, samples.p, nS, target, unc.p, err);
            KCompactProbes<<<1, SCAN_THREADS, 0, s>>>(unc.p, count, begin, uncIdx.p, ctr.p + 3);
            KRepair<<<1, 32, 0, s>>>(T, uncIdx.p, ctr.p + 3, h, samples.p, nS, cap, target, ctr.p + 2, err);
            begin += count;
        }
        CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(hc, ctr.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (hc[1]) throw Error(TSP_ERR_UNSUPPORTED, "surface sampling hash / capacity error");
    st.N_coverageRepairs = hc[2];
    const uint32_t n = hc[0];
    if (n == 0) throw invalid("Surface sampling produced no samples.");
    std::vector<float4> out4(n);
    CK(cudaMemcpyAsync(out4.data(), samples.p, n * sizeof(float4), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::vector<float> out(3ull * n);
    for (uint32_t i = 0; i < n; i++) {
        out[3ull * i] = out4[i].x; out[3ull * i + 1] = out4[i].y; out[3ull * i + 2] = out4[i].z;
        if (!std::isfinite(out4[i].x) || !std::isfinite(out4[i].y) || !std::isfinite(out4[i].z))
            throw invalid("Surface sampling produced a non-finite sample position.");
    }
    return out;
}

}  // namespace tsp
