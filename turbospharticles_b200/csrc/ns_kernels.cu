// ns_kernels.cu -- neighbor build of the B200 IISPH backend.
//
// Data layout (HBM): fluid posP[i] = (x, y, z, pressure), velRho[i] = (vx, vy, vz, density);
// boundary posB[i] = (x, y, z, psi); rigid posR[i] = (x, y, z, psi). All particle arrays are
// in Morton order after the reorder (rigid: storage order + a sorted index permutation).
//
// Pipeline of one build (reference: ReOrderParticleData + Construct + Query_Count +
// Finalize_Count + Query_Fill, source/simulation/CPU/backend/neighbor_search.cpp:613-1848):
//   KProbe          AABB of positions + "left the inner frame" flag -> host frame rule
//   KKeys           clamped Morton key per particle (min(cellId, emptyKey))
//   RadixSortPairs  stable LSD sort (primitives.cuh)
//   KReorder*       gather the SoA fields through the permutation, sorted cell IDs
//   cell table      run starts of the sorted cell IDs (device scan), count stays on device
//   KGridScatter    dense frame grid: linear cell coordinate -> compact cell index
//   KQueryFluid     one warp per SELL32 chunk (32 consecutive sorted fluid particles):
//                   stencil cells of the chunk staged in shared memory and sorted by
//                   Morton ID, so every lane's neighbors arrive in ascending index order;
//                   warp-uniform candidate sweep (broadcast loads), per-lane hit test
//   KQueryRigid     one thread per rigid particle, CSR rows (RF, RB, RR)
#include "kernels.h"
#include "primitives.cuh"

namespace tsp {

// ----------------------------------------------------------------------------- frame probe
__device__ __forceinline__ int OrderedInt(float f) {
    const int i = __float_as_int(f);
    return (i >= 0) ? i : (i ^ 0x7fffffff);
}
int OrderedIntHost(float f) {
    int i;
    memcpy(&i, &f, 4);
    return (i >= 0) ? i : (i ^ 0x7fffffff);
}
__host__ float OrderedIntToFloat(int k) {
    const int i = (k >= 0) ? k : (k ^ 0x7fffffff);
    float f;
    memcpy(&f, &i, 4);
    return f;
}

__global__ void __launch_bounds__(256) KProbe(const float4* __restrict__ pos, uint32_t n, Frame fr, int frameValid,
                                             DomainBox dom, ProbeResult* __restrict__ out) {
    float mn[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
    float mx[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    uint32_t exceeded = 0;
    const int m = (int)fr.reach;
    const int x0 = fr.ox + m, y0 = fr.oy + m, z0 = fr.oz + m;
    const int x1 = fr.ox + (int)fr.nx - 1 - m, y1 = fr.oy + (int)fr.ny - 1 - m, z1 = fr.oz + (int)fr.nz - 1 - m;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pos[i];
        mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
        mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
        if (frameValid) {
            const bool inside = !dom.bounded || (p.x >= dom.mn[0] && p.x <= dom.mx[0] && p.y >= dom.mn[1] &&
                                                 p.y <= dom.mx[1] && p.z >= dom.mn[2] && p.z <= dom.mx[2]);
            if (inside) {
                const int cx = FloorToInt(p.x * fr.cellSizeInv), cy = FloorToInt(p.y * fr.cellSizeInv),
                          cz = FloorToInt(p.z * fr.cellSizeInv);
                if (cx < x0 || cx > x1 || cy < y0 || cy > y1 || cz < z0 || cz > z1) exceeded = 1;
            }
        }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
        for (int a = 0; a < 3; a++) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], d));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], d));
        }
    exceeded = __any_sync(0xffffffffu, exceeded);
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; a++) {
            atomicMin(&out->mnKey[a], OrderedInt(mn[a]));
            atomicMax(&out->mxKey[a], OrderedInt(mx[a]));
        }
        if (exceeded) atomicOr(&out->exceeded, 1u);
    }
}

void LaunchProbe(const float4* pos, uint32_t n, const Frame& fr, bool frameValid, const DomainBox& dom,
                 ProbeResult* out, cudaStream_t s) {
    if (n == 0) return;
    const uint32_t blocks = std::min<uint32_t>((n + 255) / 256, 148u * 8u);
    KProbe<<<blocks, 256, 0, s>>>(pos, n, fr, frameValid ? 1 : 0, dom, out);
}

// ----------------------------------------------------------------------------- keys
template <typename K>
__global__ void __launch_bounds__(256) KKeys(const float4* __restrict__ pos, uint32_t n, Frame fr, uint64_t emptyKey,
                                            K* __restrict__ keys, uint32_t* __restrict__ idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    const uint64_t c = CellIdOf(p.x, p.y, p.z, fr);
    keys[i] = (K)(c < emptyKey ? c : emptyKey);
    idx[i] = i;
}

// (unclamped) cell IDs in storage order (rigid particles)
__global__ void KCellIds(const float4* __restrict__ pos, uint32_t n, Frame fr, uint64_t* __restrict__ cid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    cid[i] = CellIdOf(p.x, p.y, p.z, fr);
}

template <typename K>
__global__ void KKeysToCellIds(const K* __restrict__ keys, uint32_t n, uint64_t emptyKey, uint64_t* __restrict__ cid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t k = (uint64_t)keys[i];
    cid[i] = (k == emptyKey) ? EMPTY_64 : k;
}

// sorts `n` positions by cell key; perm[newIdx] = oldIdx and sorted cell IDs out
void SortByCell(const float4* pos, uint32_t n, const Frame& fr, SortScratch& sc, uint32_t* perm, uint64_t* cidSorted,
                cudaStream_t s) {
    if (n == 0) return;
    const uint64_t emptyKey = 1ull << (fr.keyBits - 1u);
    const uint32_t g = (n + 255) / 256;
    if (fr.keyBits <= 32) {
        uint32_t* k0 = reinterpret_cast<uint32_t*>(sc.keysA);
        uint32_t* k1 = reinterpret_cast<uint32_t*>(sc.keysB);
        KKeys<uint32_t><<<g, 256, 0, s>>>(pos, n, fr, emptyKey, k0, sc.valsA);
        const bool alt = RadixSortPairs<uint32_t, uint32_t>(k0, sc.valsA, k1, sc.valsB, n, fr.keyBits, sc.tileHist,
                                                            sc.digitTotals, s);
        KKeysToCellIds<uint32_t><<<g, 256, 0, s>>>(alt ? k1 : k0, n, emptyKey, cidSorted);
        cudaMemcpyAsync(perm, alt ? sc.valsB : sc.valsA, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    } else {
        KKeys<uint64_t><<<g, 256, 0, s>>>(pos, n, fr, emptyKey, sc.keysA, sc.valsA);
        const bool alt = RadixSortPairs<uint64_t, uint32_t>(sc.keysA, sc.valsA, sc.keysB, sc.valsB, n, fr.keyBits,
                                                            sc.tileHist, sc.digitTotals, s);
        KKeysToCellIds<uint64_t><<<g, 256, 0, s>>>(alt ? sc.keysB : sc.keysA, n, emptyKey, cidSorted);
        cudaMemcpyAsync(perm, alt ? sc.valsB : sc.valsA, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    }
}

void LaunchCellIds(const float4* pos, uint32_t n, const Frame& fr, uint64_t* cid, cudaStream_t s) {
    if (n) KCellIds<<<(n + 255) / 256, 256, 0, s>>>(pos, n, fr, cid);
}

// ----------------------------------------------------------------------------- reorders
template <typename T>
__global__ void KGather(const uint32_t* __restrict__ perm, const T* __restrict__ src, T* __restrict__ dst, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[perm[i]];
}
void GatherF4(const uint32_t* perm, const float4* src, float4* dst, uint32_t n, cudaStream_t s) {
    if (n) KGather<float4><<<(n + 255) / 256, 256, 0, s>>>(perm, src, dst, n);
}
void GatherF2(const uint32_t* perm, const float2* src, float2* dst, uint32_t n, cudaStream_t s) {
    if (n) KGather<float2><<<(n + 255) / 256, 256, 0, s>>>(perm, src, dst, n);
}
void GatherF1(const uint32_t* perm, const float* src, float* dst, uint32_t n, cudaStream_t s) {
    if (n) KGather<float><<<(n + 255) / 256, 256, 0, s>>>(perm, src, dst, n);
}
void GatherU64(const uint32_t* perm, const uint64_t* src, uint64_t* dst, uint32_t n, cudaStream_t s) {
    if (n) KGather<uint64_t><<<(n + 255) / 256, 256, 0, s>>>(perm, src, dst, n);
}

// fused gather of the solver-step fields: (pos, pressure), (vel, density) and IDs
__global__ void __launch_bounds__(256) KReorderFluidStep(const uint32_t* __restrict__ perm, const float4* __restrict__ posIn,
                                                        const float4* __restrict__ velIn, const uint64_t* __restrict__ idIn,
                                                        float4* __restrict__ posOut, float4* __restrict__ velOut,
                                                        uint64_t* __restrict__ idOut, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t src = perm[i];
    posOut[i] = posIn[src];
    velOut[i] = velIn[src];
    idOut[i] = idIn[src];
}
void LaunchReorderFluidStep(const uint32_t* perm, const float4* posIn, const float4* velIn, const uint64_t* idIn,
                            float4* posOut, float4* velOut, uint64_t* idOut, uint32_t n, cudaStream_t s) {
    if (n) KReorderFluidStep<<<(n + 255) / 256, 256, 0, s>>>(perm, posIn, velIn, idIn, posOut, velOut, idOut, n);
}

// ----------------------------------------------------------------------------- cell tables
struct RunFlagIn {
    const uint64_t* cid;
    __device__ uint64_t operator()(uint64_t i) const { return (i == 0 || cid[i] != cid[i - 1]) ? 1ull : 0ull; }
};
struct RunFlagOut {
    const uint64_t* cid;
    uint64_t* unique;
    uint32_t* start;
    uint64_t n;
    __device__ void operator()(uint64_t i, uint64_t pre, uint64_t v) const {
        if (v) { unique[pre] = cid[i]; start[pre] = (uint32_t)i; }
        if (i == n - 1) start[pre + v] = (uint32_t)n;  // sentinel = end of the last run
    }
};
void BuildCellTable(const uint64_t* cidSorted, uint32_t n, uint64_t* unique, uint32_t* start, uint64_t* nCellsDev,
                    uint64_t* scanScratch, cudaStream_t s) {
    DeviceScan<uint64_t>(RunFlagIn{cidSorted}, RunFlagOut{cidSorted, unique, start, n}, n, scanScratch, nCellsDev, s);
}

__global__ void KGridScatter(const uint64_t* __restrict__ unique, const uint64_t* __restrict__ nCellsDev, Frame fr,
                             uint32_t* __restrict__ grid, uint32_t nMax) {
    const uint64_t nCells = *nCellsDev;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nCells && c < nMax; c += gridDim.x * blockDim.x) {
        const uint64_t id = unique[c];
        if (id == EMPTY_64) continue;
        const uint32_t x = Compact21(id), y = Compact21(id >> 1), z = Compact21(id >> 2);
        grid[(uint64_t)x + (uint64_t)fr.nx * ((uint64_t)y + (uint64_t)fr.ny * z)] = c;
    }
}
void BuildGrid(const uint64_t* unique, const uint64_t* nCellsDev, uint32_t nMax, const Frame& fr, uint32_t* grid,
               uint64_t gridCells, cudaStream_t s) {
    cudaMemsetAsync(grid, 0xff, gridCells * sizeof(uint32_t), s);
    if (nMax) KGridScatter<<<std::min<uint32_t>((nMax + 255) / 256, 148u * 16u), 256, 0, s>>>(unique, nCellsDev, fr, grid, nMax);
}

// ----------------------------------------------------------------------------- fluid query
struct LaneRefs {
    uint32_t cnt, mn, mx, homeMin, farLoMax, farHiMin;
    __device__ void init() { cnt = 0; mn = 0xffffffffu; mx = 0; homeMin = 0xffffffffu; farLoMax = 0; farHiMin = 0xffffffffu; }
};

// CommitChunkCompressionMeta (GPU/backend/neighbor_search_kernels.cu:101-191) as a warp reduction
__device__ __forceinline__ void CommitChunkMeta(uint32_t chunk, bool owner, LaneRefs r, bool split, const SellMeta& m) {
    uint32_t pitch = r.cnt & 0xffffu, mn = r.mn, mx = r.mx, hm = r.homeMin, flm = r.farLoMax, fhm = r.farHiMin;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        pitch = max(pitch, __shfl_xor_sync(0xffffffffu, pitch, d));
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, d));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
        if (split) {
            hm = min(hm, __shfl_xor_sync(0xffffffffu, hm, d));
            flm = max(flm, __shfl_xor_sync(0xffffffffu, flm, d));
            fhm = min(fhm, __shfl_xor_sync(0xffffffffu, fhm, d));
        }
    }
    if (!owner) return;
    m.pitch[chunk] = (uint16_t)pitch;
    if (pitch == 0) {
        m.base[chunk] = 0; m.base2[chunk] = 0x8000u; m.format[chunk] = FMT_ABS32;
        return;
    }
    const uint32_t span = (mx >= mn) ? (mx - mn) : 0xffffffffu;
    if (mx >= mn && span <= 0xffffu) {
        m.base[chunk] = mn; m.base2[chunk] = mn + 0x8000u; m.format[chunk] = FMT_DELTA16X2;
        return;
    }
    if (split) {
        uint32_t lo, hi;
        HomeWindow(chunk, lo, hi);
        const bool hasLo = mn < lo, hasHi = mx > hi;
        const uint32_t farMin = hasLo ? mn : fhm;
        const uint32_t farMax = hasLo ? flm : mx;
        if (hasLo != hasHi && hm <= hi && farMax - farMin <= 0x7fffu) {
            m.base[chunk] = hm; m.base2[chunk] = farMin; m.format[chunk] = FMT_DELTA16X2;
            return;
        }
    }
    m.base[chunk] = mn; m.base2[chunk] = mn + 0x8000u; m.format[chunk] = FMT_ABS32;
}

struct LaneWriter {
    uint32_t wr, pitch, base, base2;
    uint64_t off;
    uint8_t fmt;
    __device__ void init(const SellMeta& m, uint32_t chunk) {
        wr = 0; pitch = m.pitch[chunk]; base = m.base[chunk]; base2 = m.base2[chunk]; off = m.offset[chunk];
        fmt = m.format[chunk];
    }
    // StoreNeighbor_CompressedSell32 (neighbor_search_kernels.cu:193-247)
    __device__ void store(const SellMeta& m, uint32_t lane, uint32_t j, uint32_t* err) {
        if (wr >= pitch) { atomicOr(err, ERR_FILL_OVERFLOW); return; }
        const uint64_t lin = off + (uint64_t)wr * SELL_W + lane;
        if (fmt == FMT_DELTA16X2) {
            const bool first = (j >= base) && (j - base <= 0x7fffu);
            if ((!first && (j < base2 || j - base2 > 0x7fffu)) || lin >= m.cap16) { atomicOr(err, ERR_DELTA_RANGE); return; }
            m.list16[lin] = first ? (uint16_t)(j - base) : (uint16_t)(0x8000u | (j - base2));
        } else {
            if (lin >= m.cap32) { atomicOr(err, ERR_FILL_OVERFLOW); return; }
            m.list32[lin] = j;
        }
        wr++;
    }
};

__device__ __forceinline__ void WarpBitonicSort(uint64_t* v, uint32_t S, uint32_t lane) {
    for (uint32_t k = 2; k <= S; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t t = lane; t < S; t += 32) {
                const uint32_t p = t ^ j;
                if (p > t) {
                    const uint64_t a = v[t], b = v[p];
                    const bool up = (t & k) == 0;
                    if ((a > b) == up) { v[t] = b; v[p] = a; }
                }
            }
            __syncwarp();
        }
    }
}

// per-warp record of the count pass: (candidate | species << 30, 32-lane hit mask) for every
// candidate that is a neighbor of at least one lane, in sweep order, staged 32 entries per
// coalesced 256 B store; the fill pass replays it instead of repeating the candidate sweep
struct DictRec {
    uint2* base;
    uint32_t n, cap;
    uint32_t pj, pm;
    bool ok;
    __device__ __forceinline__ void push(uint32_t tagged, uint32_t mask, uint32_t lane) {
        if (n < cap) {
            if (lane == (n & 31u)) { pj = tagged; pm = mask; }
            if ((n & 31u) == 31u) base[(n & ~31u) + lane] = make_uint2(pj, pm);
        }
        n++;
    }
    __device__ __forceinline__ void finish(uint32_t lane) {
        if (n <= cap && lane < (n & 31u)) base[(n & ~31u) + lane] = make_uint2(pj, pm);
    }
};

struct QueryLane {
    float4 pi;
    int lx, ly, lz;
    bool member;
    uint32_t homeLo, homeHi;
};

// candidate sweep of one species over the group's sorted candidate cells (warp-uniform loop)
template <int SP, bool FILL>
__device__ __forceinline__ void SweepSpecies(const QueryArgs& a, const uint64_t* cells, uint32_t vol, const QueryLane& q,
                                             uint32_t lane, LaneRefs& ref, LaneWriter& w, const SellMeta& m,
                                             DictRec& dict) {
    const uint32_t* grid = SP == 0 ? a.gridF : SP == 1 ? a.gridB : a.gridR;
    const uint32_t* start = SP == 0 ? a.startF : SP == 1 ? a.startB : a.startR;
    const float4* pos = SP == 0 ? a.posF : SP == 1 ? a.posB : a.posR;
    if (grid == nullptr) return;
    const int r = (int)a.fr.reach;
    for (uint32_t cb = 0; cb < vol; cb += 32) {
        const uint32_t t = cb + lane;
        uint32_t b = 0, e = 0;
        int cx = 0, cy = 0, cz = 0;
        if (t < vol) {
            const uint64_t mc = cells[t];
            cx = (int)Compact21(mc); cy = (int)Compact21(mc >> 1); cz = (int)Compact21(mc >> 2);
            const uint32_t c = grid[(uint64_t)cx + (uint64_t)a.fr.nx * ((uint64_t)cy + (uint64_t)a.fr.ny * cz)];
            if (c != EMPTY_32) { b = start[c]; e = start[c + 1]; }
        }
        uint32_t nonEmpty = __ballot_sync(0xffffffffu, b < e);
        while (nonEmpty) {
            const int l = __ffs(nonEmpty) - 1;
            nonEmpty &= nonEmpty - 1;
            const uint32_t cb_ = __shfl_sync(0xffffffffu, b, l), ce = __shfl_sync(0xffffffffu, e, l);
            const int ccx = __shfl_sync(0xffffffffu, cx, l), ccy = __shfl_sync(0xffffffffu, cy, l),
                      ccz = __shfl_sync(0xffffffffu, cz, l);
            // strict per-particle stencil (GatherCellQueryRanges, neighbor_search.cpp:917-947)
            const bool ok = q.member && abs(ccx - q.lx) <= r && abs(ccy - q.ly) <= r && abs(ccz - q.lz) <= r;
            if (!__any_sync(0xffffffffu, ok)) continue;
            for (uint32_t k = cb_; k < ce; k++) {
                const uint32_t j = (SP == 2) ? a.permR[k] : k;
                const float4 pj = pos[j];
                const bool hit = ok && IsNeighbor(q.pi.x, q.pi.y, q.pi.z, pj.x, pj.y, pj.z, a.r2);
                if (FILL) {
                    if (hit) w.store(m, lane, j, a.err);
                } else {
                    const uint32_t mask = __ballot_sync(0xffffffffu, hit);
                    if (mask) dict.push(j < (1u << 30) ? (j | ((uint32_t)SP << 30)) : 0xffffffffu, mask, lane);
                    if (j >= (1u << 30)) dict.ok = false;
                    if (hit) {
                        ref.cnt++;
                        ref.mn = min(ref.mn, j);
                        ref.mx = max(ref.mx, j);
                        if (SP == 0) {
                            if (j < q.homeLo) ref.farLoMax = max(ref.farLoMax, j);
                            else if (j > q.homeHi) ref.farHiMin = min(ref.farHiMin, j);
                            else ref.homeMin = min(ref.homeMin, j);
                        }
                    }
                }
            }
        }
    }
}

__device__ __forceinline__ void SortRowSell(const SellMeta& m, const LaneWriter& w, uint32_t lane) {
    // rigid candidates arrive in sorted-cell order; rows are kept in ascending index order
    // (the Delta16x2 / Abs32 codes of an FR chunk are monotonic in the index)
    for (uint32_t x = 1; x < w.wr; x++) {
        const uint64_t at = w.off + (uint64_t)x * SELL_W + lane;
        uint32_t y = x;
        if (w.fmt == FMT_DELTA16X2) {
            const uint16_t v = m.list16[at];
            while (y > 0 && m.list16[w.off + (uint64_t)(y - 1) * SELL_W + lane] > v) {
                m.list16[w.off + (uint64_t)y * SELL_W + lane] = m.list16[w.off + (uint64_t)(y - 1) * SELL_W + lane];
                y--;
            }
            m.list16[w.off + (uint64_t)y * SELL_W + lane] = v;
        } else {
            const uint32_t v = m.list32[at];
            while (y > 0 && m.list32[w.off + (uint64_t)(y - 1) * SELL_W + lane] > v) {
                m.list32[w.off + (uint64_t)y * SELL_W + lane] = m.list32[w.off + (uint64_t)(y - 1) * SELL_W + lane];
                y--;
            }
            m.list32[w.off + (uint64_t)y * SELL_W + lane] = v;
        }
    }
}

template <bool FILL>
__global__ void __launch_bounds__(QUERY_THREADS) KQueryFluid(QueryArgs a, SellMeta mFF, SellMeta mFB, SellMeta mFR) {
    extern __shared__ uint64_t qsmem[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t* cells = qsmem + (uint64_t)warp * a.cap;
    const uint32_t chunk = blockIdx.x * (QUERY_THREADS / 32) + warp;
    const uint32_t nChunks = (a.nF + SELL_W - 1) / SELL_W;
    if (chunk >= nChunks) return;  // uniform per warp
    const uint32_t i = chunk * SELL_W + lane;
    const bool inRange = i < a.nF;
    const uint64_t cid = inRange ? a.cidF[i] : EMPTY_64;
    const bool valid = cid != EMPTY_64;
    QueryLane q;
    q.pi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (inRange) q.pi = a.posF[i];
    q.lx = q.ly = q.lz = 0;
    if (valid) { q.lx = (int)Compact21(cid); q.ly = (int)Compact21(cid >> 1); q.lz = (int)Compact21(cid >> 2); }
    HomeWindow(chunk, q.homeLo, q.homeHi);
    const int r = (int)a.fr.reach;

    LaneRefs rFF, rFB, rFR;
    rFF.init(); rFB.init(); rFR.init();
    LaneWriter wFF, wFB, wFR;
    if (FILL) { wFF.init(mFF, chunk); wFB.init(mFB, chunk); wFR.init(mFR, chunk); }
    DictRec dict;
    dict.base = a.dict ? a.dict + (uint64_t)chunk * a.dictCap : nullptr;
    dict.n = 0; dict.cap = a.dict ? a.dictCap : 0u; dict.pj = 0; dict.pm = 0; dict.ok = a.dict != nullptr;

    if (FILL && a.dict) {
        // replay the count pass's hit masks (same order as the sweep)
        const uint32_t nd = a.dictCount[chunk];
        if (nd != EMPTY_32) {
            const uint2* d = a.dict + (uint64_t)chunk * a.dictCap;
            for (uint32_t b0 = 0; b0 < nd; b0 += 32) {
                const uint2 mine = (b0 + lane < nd) ? d[b0 + lane] : make_uint2(0u, 0u);
                const uint32_t cntHere = min(32u, nd - b0);
                for (uint32_t e = 0; e < cntHere; e++) {
                    const uint32_t tj = __shfl_sync(0xffffffffu, mine.x, e);
                    const uint32_t tm = __shfl_sync(0xffffffffu, mine.y, e);
                    if (!((tm >> lane) & 1u)) continue;
                    const uint32_t sp = tj >> 30, j = tj & 0x3fffffffu;
                    if (sp == 0) wFF.store(mFF, lane, j, a.err);
                    else if (sp == 1) wFB.store(mFB, lane, j, a.err);
                    else wFR.store(mFR, lane, j, a.err);
                }
            }
            if (inRange && wFR.wr > 1) SortRowSell(mFR, wFR, lane);
            return;
        }
    }

    const uint32_t validMask = __ballot_sync(0xffffffffu, valid);
    if (validMask) {
        int mnx = valid ? q.lx : 0x7fffffff, mny = valid ? q.ly : 0x7fffffff, mnz = valid ? q.lz : 0x7fffffff;
        int mxx = valid ? q.lx : -1, mxy = valid ? q.ly : -1, mxz = valid ? q.lz : -1;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            mnx = min(mnx, __shfl_xor_sync(0xffffffffu, mnx, d)); mxx = max(mxx, __shfl_xor_sync(0xffffffffu, mxx, d));
            mny = min(mny, __shfl_xor_sync(0xffffffffu, mny, d)); mxy = max(mxy, __shfl_xor_sync(0xffffffffu, mxy, d));
            mnz = min(mnz, __shfl_xor_sync(0xffffffffu, mnz, d)); mxz = max(mxz, __shfl_xor_sync(0xffffffffu, mxz, d));
        }
        const uint64_t prevCid = __shfl_up_sync(0xffffffffu, cid, 1);
        const bool isStart = valid && (lane == 0 || prevCid != cid);
        const uint32_t startMask = __ballot_sync(0xffffffffu, isStart);
        const uint32_t nDistinct = __popc(startMask);
        const int bx0 = max(mnx - r, 0), by0 = max(mny - r, 0), bz0 = max(mnz - r, 0);
        const int bx1 = min(mxx + r, (int)a.fr.nx - 1), by1 = min(mxy + r, (int)a.fr.ny - 1),
                  bz1 = min(mxz + r, (int)a.fr.nz - 1);
        const uint64_t boxVol = (uint64_t)(bx1 - bx0 + 1) * (uint64_t)(by1 - by0 + 1) * (uint64_t)(bz1 - bz0 + 1);
        const uint64_t stencilVol = (uint64_t)(2 * r + 1) * (2 * r + 1) * (2 * r + 1);
        // one box sweep when it is small (GatherChunkQueryRanges, neighbor_search.cpp:1008-1018),
        // else one stencil box per distinct cell of the chunk
        const bool boxMode = boxVol <= a.cap && boxVol <= (uint64_t)nDistinct * stencilVol;
        const uint32_t nGroups = boxMode ? 1u : nDistinct;
        uint32_t groupsLeft = startMask;
        for (uint32_t g = 0; g < nGroups; g++) {
            int gx0 = bx0, gy0 = by0, gz0 = bz0, gx1 = bx1, gy1 = by1, gz1 = bz1;
            q.member = valid;
            if (!boxMode) {
                const int L = __ffs(groupsLeft) - 1;
                groupsLeft &= groupsLeft - 1;
                const uint64_t gcid = __shfl_sync(0xffffffffu, cid, L);
                const int cx = __shfl_sync(0xffffffffu, q.lx, L), cy = __shfl_sync(0xffffffffu, q.ly, L),
                          cz = __shfl_sync(0xffffffffu, q.lz, L);
                q.member = valid && cid == gcid;
                gx0 = max(cx - r, 0); gy0 = max(cy - r, 0); gz0 = max(cz - r, 0);
                gx1 = min(cx + r, (int)a.fr.nx - 1); gy1 = min(cy + r, (int)a.fr.ny - 1); gz1 = min(cz + r, (int)a.fr.nz - 1);
            }
            const uint32_t ex = gx1 - gx0 + 1, ey = gy1 - gy0 + 1, ez = gz1 - gz0 + 1;
            const uint32_t vol = ex * ey * ez;
            if (vol > a.cap) {
                if (lane == 0) atomicOr(a.err, ERR_QUERY_CAP);
                continue;
            }
            uint32_t S = 32;
            while (S < vol) S <<= 1;
            for (uint32_t t = lane; t < S; t += 32) {
                uint64_t v = 0xffffffffffffffffull;
                if (t < vol) {
                    const uint32_t x = gx0 + t % ex, y = gy0 + (t / ex) % ey, z = gz0 + t / (ex * ey);
                    v = MortonLocal(x, y, z);
                }
                cells[t] = v;
            }
            __syncwarp();
            WarpBitonicSort(cells, S, lane);
            SweepSpecies<0, FILL>(a, cells, vol, q, lane, rFF, wFF, mFF, dict);
            SweepSpecies<1, FILL>(a, cells, vol, q, lane, rFB, wFB, mFB, dict);
            SweepSpecies<2, FILL>(a, cells, vol, q, lane, rFR, wFR, mFR, dict);
            __syncwarp();
        }
    }
    if (FILL) {
        if (inRange && wFR.wr > 1) SortRowSell(mFR, wFR, lane);
        return;
    }
    if (a.dict) {
        dict.finish(lane);
        if (lane == 0) a.dictCount[chunk] = (dict.ok && dict.n <= dict.cap) ? dict.n : EMPTY_32;
    }
    if (inRange) {
        if ((rFF.cnt | rFB.cnt | rFR.cnt) > 0xffffu) atomicOr(a.err, ERR_COUNT_U16);
        mFF.counts[i] = (uint16_t)rFF.cnt;
        mFB.counts[i] = (uint16_t)rFB.cnt;
        mFR.counts[i] = (uint16_t)rFR.cnt;
    }
    {
        uint32_t t0 = rFF.cnt & 0xffffu, t1 = rFB.cnt & 0xffffu, t2 = rFR.cnt & 0xffffu;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            t0 += __shfl_xor_sync(0xffffffffu, t0, d);
            t1 += __shfl_xor_sync(0xffffffffu, t1, d);
            t2 += __shfl_xor_sync(0xffffffffu, t2, d);
        }
        if (lane == 0 && a.nbrTotals) {
            atomicAdd(a.nbrTotals + 0, (unsigned long long)t0);
            atomicAdd(a.nbrTotals + 1, (unsigned long long)t1);
            atomicAdd(a.nbrTotals + 2, (unsigned long long)t2);
        }
    }
    const bool owner = lane == 0;
    CommitChunkMeta(chunk, owner, rFF, true, mFF);
    CommitChunkMeta(chunk, owner, rFB, false, mFB);
    CommitChunkMeta(chunk, owner, rFR, false, mFR);
}

uint32_t QueryCap(uint32_t reach) {
    const uint32_t stencil = (2 * reach + 1) * (2 * reach + 1) * (2 * reach + 1);
    uint32_t cap = 512;
    while (cap < stencil) cap <<= 1;
    return cap;
}

void LaunchQueryFluid(bool fill, const QueryArgs& a, const SellMeta& ff, const SellMeta& fb, const SellMeta& fr,
                      cudaStream_t s) {
    const uint32_t nChunks = (a.nF + SELL_W - 1) / SELL_W;
    if (nChunks == 0) return;
    const uint32_t warps = QUERY_THREADS / 32;
    const size_t smem = (size_t)a.cap * sizeof(uint64_t) * warps;
    const uint32_t blocks = (nChunks + warps - 1) / warps;
    if (fill) {
        cudaFuncSetAttribute(KQueryFluid<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        KQueryFluid<true><<<blocks, QUERY_THREADS, smem, s>>>(a, ff, fb, fr);
    } else {
        cudaFuncSetAttribute(KQueryFluid<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        KQueryFluid<false><<<blocks, QUERY_THREADS, smem, s>>>(a, ff, fb, fr);
    }
}

// ----------------------------------------------------------------------------- rigid query
__device__ __forceinline__ void SortRowU32(uint32_t* row, uint32_t n) {
    for (uint32_t x = 1; x < n; x++) {
        const uint32_t v = row[x];
        uint32_t y = x;
        while (y > 0 && row[y - 1] > v) { row[y] = row[y - 1]; y--; }
        row[y] = v;
    }
}

template <bool FILL>
__global__ void __launch_bounds__(128) KQueryRigid(QueryArgs a, RigidLists L) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nR) return;
    const float4 p = a.posR[i];
    const int cx = FloorToInt(p.x * a.fr.cellSizeInv) - a.fr.ox, cy = FloorToInt(p.y * a.fr.cellSizeInv) - a.fr.oy,
              cz = FloorToInt(p.z * a.fr.cellSizeInv) - a.fr.oz;
    uint32_t n[3] = {0, 0, 0};
    uint64_t off[3] = {0, 0, 0};
    if (FILL) { off[0] = L.offRF[i]; off[1] = L.offRB[i]; off[2] = L.offRR[i]; }
    const bool inFrame = cx >= 0 && cx < (int)a.fr.nx && cy >= 0 && cy < (int)a.fr.ny && cz >= 0 && cz < (int)a.fr.nz;
    if (inFrame) {
        const int r = (int)a.fr.reach;
        const uint32_t body = a.bodyR[i];
        for (int oz = max(cz - r, 0); oz <= min(cz + r, (int)a.fr.nz - 1); oz++)
            for (int oy = max(cy - r, 0); oy <= min(cy + r, (int)a.fr.ny - 1); oy++)
                for (int ox = max(cx - r, 0); ox <= min(cx + r, (int)a.fr.nx - 1); ox++) {
                    const uint64_t lin = (uint64_t)ox + (uint64_t)a.fr.nx * ((uint64_t)oy + (uint64_t)a.fr.ny * oz);
                    for (int sp = 0; sp < 3; sp++) {
                        const uint32_t* grid = sp == 0 ? a.gridF : sp == 1 ? a.gridB : a.gridR;
                        const uint32_t* start = sp == 0 ? a.startF : sp == 1 ? a.startB : a.startR;
                        const float4* pos = sp == 0 ? a.posF : sp == 1 ? a.posB : a.posR;
                        if (grid == nullptr) continue;
                        const uint32_t c = grid[lin];
                        if (c == EMPTY_32) continue;
                        for (uint32_t k = start[c]; k < start[c + 1]; k++) {
                            const uint32_t j = sp == 2 ? a.permR[k] : k;
                            if (sp == 2 && (j == i || a.bodyR[j] == body)) continue;
                            const float4 q = pos[j];
                            if (!IsNeighbor(p.x, p.y, p.z, q.x, q.y, q.z, a.r2)) continue;
                            if (FILL) {
                                uint32_t* list = sp == 0 ? L.listRF : sp == 1 ? L.listRB : L.listRR;
                                list[off[sp] + n[sp]] = j;
                            }
                            n[sp]++;
                        }
                    }
                }
    }
    if (FILL) {
        SortRowU32(L.listRF + off[0], n[0]);
        SortRowU32(L.listRB + off[1], n[1]);
        SortRowU32(L.listRR + off[2], n[2]);
    } else {
        if ((n[0] | n[1] | n[2]) > 0xffffu) atomicOr(a.err, ERR_COUNT_U16);
        L.cntRF[i] = (uint16_t)n[0]; L.cntRB[i] = (uint16_t)n[1]; L.cntRR[i] = (uint16_t)n[2];
    }
}
void LaunchQueryRigid(bool fill, const QueryArgs& a, const RigidLists& L, cudaStream_t s) {
    if (a.nR == 0) return;
    if (fill) KQueryRigid<true><<<(a.nR + 127) / 128, 128, 0, s>>>(a, L);
    else KQueryRigid<false><<<(a.nR + 127) / 128, 128, 0, s>>>(a, L);
}

// ----------------------------------------------------------------------------- finalize
struct SellSizeIn {
    const uint16_t* pitch;
    const uint8_t* format;
    __device__ U64x2 operator()(uint64_t c) const {
        const uint64_t sz = (uint64_t)pitch[c] * SELL_W;
        return format[c] == FMT_DELTA16X2 ? U64x2{sz, 0} : U64x2{0, sz};
    }
};
struct SellOffsetOut {
    const uint8_t* format;
    uint64_t* offset;
    __device__ void operator()(uint64_t c, U64x2 pre, U64x2) const {
        offset[c] = format[c] == FMT_DELTA16X2 ? pre.a : pre.b;
    }
};
// chunk offsets per format = exclusive prefix of pitch * 32 over chunks of that format
// (FinalizeNeighborLists_Count, neighbor_search.cu:392-425); totals (n16, n32) to device
void FinalizeSell(const SellMeta& m, uint32_t nChunks, U64x2* scratch, U64x2* totals, cudaStream_t s) {
    DeviceScan<U64x2>(SellSizeIn{m.pitch, m.format}, SellOffsetOut{m.format, m.offset}, nChunks, scratch, totals, s);
}

struct CountIn {
    const uint16_t* c;
    __device__ uint64_t operator()(uint64_t i) const { return c[i]; }
};
struct CsrOut {
    uint64_t* off;
    uint64_t n;
    __device__ void operator()(uint64_t i, uint64_t pre, uint64_t v) const {
        off[i] = pre;
        if (i == n - 1) off[n] = pre + v;
    }
};
void FinalizeCsr(const uint16_t* counts, uint64_t* off, uint32_t n, uint64_t* scratch, uint64_t* total, cudaStream_t s) {
    if (n == 0) {
        cudaMemsetAsync(off, 0, sizeof(uint64_t), s);
        cudaMemsetAsync(total, 0, sizeof(uint64_t), s);
        return;
    }
    DeviceScan<uint64_t>(CountIn{counts}, CsrOut{off, n}, n, scratch, total, s);
}

// ----------------------------------------------------------------------------- row decode
__global__ void KDecodeSellRows(SellMeta m, uint32_t nF, const uint64_t* __restrict__ rowOff, uint32_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nF) return;
    const uint32_t chunk = i / SELL_W, lane = i % SELL_W;
    const uint32_t cnt = m.counts[i];
    const uint8_t fmt = m.format[chunk];
    for (uint32_t k = 0; k < cnt; k++)
        out[rowOff[i] + k] = SellNeighbor(fmt, m.base[chunk], m.base2[chunk], m.offset[chunk], k, lane, m.list16, m.list32);
}
void LaunchDecodeSellRows(const SellMeta& m, uint32_t nF, const uint64_t* rowOff, uint32_t* out, cudaStream_t s) {
    if (nF) KDecodeSellRows<<<(nF + 255) / 256, 256, 0, s>>>(m, nF, rowOff, out);
}

}  // namespace tsp
