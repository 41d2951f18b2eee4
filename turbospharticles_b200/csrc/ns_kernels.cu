// ns_kernels.cu -- neighbor build of the B200 IISPH backend.
//
// Data layout (HBM): fluid posP[i] = (x, y, z, pressure), velRho[i] = (vx, vy, vz, density);
// boundary posB[i] = (x, y, z, psi); rigid posR[i] = (x, y, z, psi). All particle arrays are
// in Morton order after the reorder (rigid: storage order + a sorted index permutation).
//
// Pipeline of one build (reference: ReOrderParticleData + Construct + Query_Count +
// Finalize_Count + Query_Fill, source/simulation/CPU/backend/neighbor_search.cpp:613-1848):
//   KProbe          AABB of positions + "left the inner frame" flag -> host frame rule
//   KKeys           clamped Morton key per particle (min(cellId, emptyKey)) + the digit
//                   histograms of every sort pass
//   KOnesweepPass   stable LSD sort, one kernel per 8-bit digit (primitives.cuh); the last
//                   pass writes the permutation and the sorted cell IDs
//   KReorder*       gather the SoA fields through the permutation
//   KCellTableGrid  run starts of the sorted cell IDs (single-pass scan), each writing the
//                   compact cell table and the dense frame grid entry; count stays on device
//   KQueryFluid*    one warp per SELL32 chunk (32 consecutive sorted fluid particles):
//                   each lane walks only its own strict stencil, whose non-empty cell
//                   ranges are looked up once per distinct cell of the chunk and ranked by
//                   first index (= Morton order), so rows arrive in ascending index order.
//                   The count pass keeps each row in a [slot][lane] scratch; the fill pass
//                   encodes the scratch into the SELL32 slices (same layout, coalesced). A
//                   variant of the count pass first copies the block's neighboring cell
//                   blocks into shared memory (TMA bulk copies) and walks them there
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
    // block reduction first: one set of global atomics per block, not per warp (the atomics on
    // the seven shared words were the probe's cost)
    __shared__ float smn[3][8], smx[3][8];
    __shared__ uint32_t sex[8];
    const uint32_t warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; a++) { smn[a][warp] = mn[a]; smx[a][warp] = mx[a]; }
        sex[warp] = exceeded;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t w = 1; w < (blockDim.x >> 5); w++) {
            for (int a = 0; a < 3; a++) { mn[a] = fminf(mn[a], smn[a][w]); mx[a] = fmaxf(mx[a], smx[a][w]); }
            exceeded |= sex[w];
        }
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
    const uint32_t blocks = std::min<uint32_t>((n + 255) / 256, 148u * 4u);
    KProbe<<<blocks, 256, 0, s>>>(pos, n, fr, frameValid ? 1 : 0, dom, out);
}

// ----------------------------------------------------------------------------- keys
// clamped keys; with `hist`, also every sort pass's digit histogram (one-pass sort)
template <typename K>
__global__ void __launch_bounds__(256) KKeys(const float4* __restrict__ pos, uint32_t n, Frame fr, uint64_t emptyKey,
                                            K* __restrict__ keys, uint32_t* __restrict__ idx,
                                            uint32_t* __restrict__ hist, uint32_t passes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t k = 0;
    if (i < n) {
        const float4 p = pos[i];
        const uint64_t c = CellIdOf(p.x, p.y, p.z, fr);
        k = c < emptyKey ? c : emptyKey;
        keys[i] = (K)k;
        idx[i] = i;
    }
    if (hist == nullptr) return;
    __shared__ uint32_t sh[OS_MAX_PASSES * 256];
    for (uint32_t b = threadIdx.x; b < passes * 256u; b += blockDim.x) sh[b] = 0;
    __syncthreads();
    OnesweepCountKey(k, i < n, passes, sh);
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < passes * 256u; b += blockDim.x)
        if (sh[b]) atomicAdd(hist + b, sh[b]);
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
    const uint32_t passes = (fr.keyBits + 7u) / 8u;
    if (sc.osAux && n >= 2) {
        // one-pass sort: keys + all histograms in one launch, then one launch per pass; the last
        // pass writes the permutation and the sorted cell IDs directly
        cudaMemsetAsync(sc.osAux, 0, OnesweepAuxWords(n, passes) * sizeof(uint32_t), s);
        const OnesweepAux a = OnesweepLayout(sc.osAux, sc.err, ERR_SORT_LOOKBACK);
        if (fr.keyBits <= 32) {
            uint32_t* k0 = reinterpret_cast<uint32_t*>(sc.keysA);
            uint32_t* k1 = reinterpret_cast<uint32_t*>(sc.keysB);
            KKeys<uint32_t><<<g, 256, 0, s>>>(pos, n, fr, emptyKey, k0, sc.valsA, a.hist, passes);
            OnesweepSortPairs<uint32_t, uint32_t>(k0, sc.valsA, k1, sc.valsB, n, fr.keyBits, a, perm, cidSorted,
                                                  emptyKey, s);
        } else {
            KKeys<uint64_t><<<g, 256, 0, s>>>(pos, n, fr, emptyKey, sc.keysA, sc.valsA, a.hist, passes);
            OnesweepSortPairs<uint64_t, uint32_t>(sc.keysA, sc.valsA, sc.keysB, sc.valsB, n, fr.keyBits, a, perm,
                                                  cidSorted, emptyKey, s);
        }
        return;
    }
    if (fr.keyBits <= 32) {
        uint32_t* k0 = reinterpret_cast<uint32_t*>(sc.keysA);
        uint32_t* k1 = reinterpret_cast<uint32_t*>(sc.keysB);
        KKeys<uint32_t><<<g, 256, 0, s>>>(pos, n, fr, emptyKey, k0, sc.valsA, nullptr, 0);
        const bool alt = RadixSortPairs<uint32_t, uint32_t>(k0, sc.valsA, k1, sc.valsB, n, fr.keyBits, sc.tileHist,
                                                            sc.digitTotals, s);
        KKeysToCellIds<uint32_t><<<g, 256, 0, s>>>(alt ? k1 : k0, n, emptyKey, cidSorted);
        cudaMemcpyAsync(perm, alt ? sc.valsB : sc.valsA, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    } else {
        KKeys<uint64_t><<<g, 256, 0, s>>>(pos, n, fr, emptyKey, sc.keysA, sc.valsA, nullptr, 0);
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

// Cell table and dense grid in one pass: run starts of the sorted cell IDs by a single-pass
// scan (tiles of 1024 in ticket order, decoupled look-back on one status word per tile: state in
// the two high bits, count in the low 30), each run start writing its unique ID, its start and
// its dense-grid entry. Same tables as BuildCellTable + BuildGrid.
constexpr uint32_t CT_ITEMS = 4, CT_THREADS = 256, CT_TILE = CT_ITEMS * CT_THREADS;
inline uint64_t CellTableAuxWords(uint32_t n) { return (n + CT_TILE - 1) / CT_TILE + 64u; }
__global__ void __launch_bounds__(CT_THREADS) KCellTableGrid(const uint64_t* __restrict__ cid, uint32_t n,
                                                             uint64_t* __restrict__ unique, uint32_t* __restrict__ start,
                                                             uint64_t* __restrict__ nCells, uint32_t* __restrict__ grid,
                                                             Frame fr, uint32_t* __restrict__ aux, uint32_t* err) {
    __shared__ uint32_t sTile;
    __shared__ uint64_t sPrefix;
    if (threadIdx.x == 0) sTile = atomicAdd(aux, 1u);
    __syncthreads();
    const uint32_t tile = sTile;
    volatile uint32_t* status = aux + 64;
    const uint64_t base = (uint64_t)tile * CT_TILE + (uint64_t)threadIdx.x * CT_ITEMS;
    uint64_t c[CT_ITEMS];
    uint32_t f[CT_ITEMS];
    uint64_t own = 0;
    const uint64_t prevId = (base > 0 && base - 1 < n) ? cid[base - 1] : 0ull;
#pragma unroll
    for (uint32_t k = 0; k < CT_ITEMS; k++) {
        const uint64_t i = base + k;
        c[k] = i < n ? cid[i] : 0ull;
        const uint64_t before = k == 0 ? prevId : c[k - 1];
        f[k] = (i < n && (i == 0 || c[k] != before)) ? 1u : 0u;
        own += f[k];
    }
    uint64_t tileTotal;
    uint64_t pre = BlockExclusiveScan<uint64_t>(own, tileTotal);
    if (threadIdx.x == 0) {
        uint32_t prefix = 0;
        if (tile == 0) {
            status[0] = OS_INC | (uint32_t)tileTotal;
        } else {
            status[tile] = OS_AGG | (uint32_t)tileTotal;
            for (uint32_t p = tile - 1;; p--) {
                uint32_t w = 0;
                for (uint32_t spins = 0; spins < OS_SPIN_LIMIT; spins++) {
                    w = status[p];
                    if (w & ~OS_VAL) break;
                }
                if (!(w & ~OS_VAL)) {
                    if (err) atomicOr(err, ERR_SORT_LOOKBACK);
                    break;
                }
                prefix += w & OS_VAL;
                if ((w & ~OS_VAL) == OS_INC || p == 0) break;
            }
            status[tile] = OS_INC | ((prefix + (uint32_t)tileTotal) & OS_VAL);
        }
        sPrefix = prefix;
    }
    __syncthreads();
    uint64_t run = sPrefix + pre;
#pragma unroll
    for (uint32_t k = 0; k < CT_ITEMS; k++) {
        const uint64_t i = base + k;
        if (i >= n || run >= n) break;  // (run >= n only after a look-back that gave up)
        if (f[k]) {
            unique[run] = c[k];
            start[run] = (uint32_t)i;
            if (grid && c[k] != EMPTY_64) {
                const uint32_t x = Compact21(c[k]), y = Compact21(c[k] >> 1), z = Compact21(c[k] >> 2);
                grid[(uint64_t)x + (uint64_t)fr.nx * ((uint64_t)y + (uint64_t)fr.ny * z)] = (uint32_t)run;
            }
            run++;
        }
        if (i == n - 1) {  // sentinel = end of the last run, and the run count
            start[run] = n;
            *nCells = run;
        }
    }
}
// cell table of n sorted cell IDs and, when grid is set, the frame's dense grid (cleared here);
// `aux` holds CellTableAuxWords(n) words (zeroed here)
void BuildCellTableGrid(const uint64_t* cidSorted, uint32_t n, uint64_t* unique, uint32_t* start, uint64_t* nCellsDev,
                        uint32_t* grid, const Frame& fr, uint64_t gridCells, uint32_t* aux, uint32_t* err,
                        cudaStream_t s) {
    if (grid) cudaMemsetAsync(grid, 0xff, gridCells * sizeof(uint32_t), s);
    if (n == 0) {
        cudaMemsetAsync(nCellsDev, 0, sizeof(uint64_t), s);
        return;
    }
    cudaMemsetAsync(aux, 0, CellTableAuxWords(n) * sizeof(uint32_t), s);
    const uint32_t tiles = (n + CT_TILE - 1) / CT_TILE;
    KCellTableGrid<<<tiles, CT_THREADS, 0, s>>>(cidSorted, n, unique, start, nCellsDev, grid, fr, aux, err);
}
uint64_t CellTableGridAuxWords(uint32_t n) { return CellTableAuxWords(n); }

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

__device__ __forceinline__ void SortRowSell(const SellMeta& m, const LaneWriter& w, uint32_t lane) {
    // rigid candidates arrive in sorted-cell order through the rigid permutation; rows are kept
    // in ascending index order (the Delta16x2 / Abs32 codes of an FR chunk are monotonic in j)
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

// ---- per-lane stencil walk
//
// A chunk's lanes are grouped by their (sorted, hence contiguous) cell. For each group the
// non-empty cells of its strict (2*reach+1)^3 stencil (GatherCellQueryRanges,
// neighbor_search.cpp:917-947) are looked up once in the dense frame grid, and their particle
// ranges are ranked by first index -- ascending cell ranges are ascending Morton IDs, so each
// lane then walks exactly its own candidates in ascending index order. Groups are handled in
// batches that fit the per-warp range staging (QueryGroupsPerBatch).
struct QueryWarp {
    uint2* rng;      // [RCAP] (begin, end) per stencil slot, group-major
    uint2* srt;      // [RCAP] non-empty ranges of each group ranked by begin
    int* gc;         // [3][32] cell coordinates of each group
    uint32_t* nne;   // [32] non-empty ranges per group of the batch
};
__host__ __device__ __forceinline__ uint32_t StencilVolume(uint32_t reach) {
    const uint32_t d = 2u * reach + 1u;
    return d * d * d;
}
__host__ __device__ __forceinline__ uint32_t QueryGroupsPerBatch(uint32_t reach) {
    const uint32_t sv = StencilVolume(reach);
    return sv >= 256u ? 1u : 256u / sv;
}
__host__ __device__ __forceinline__ uint32_t QueryRangeCap(uint32_t reach) {
    return QueryGroupsPerBatch(reach) * StencilVolume(reach);
}
__host__ __device__ __forceinline__ size_t QueryWarpSmemBytes(uint32_t reach) {
    return (size_t)QueryRangeCap(reach) * 2u * sizeof(uint2) + 4u * 32u * sizeof(uint32_t);
}
__device__ __forceinline__ QueryWarp QueryWarpSmem(void* base, uint32_t warp, uint32_t reach) {
    const uint32_t rcap = QueryRangeCap(reach);
    char* p = (char*)base + (size_t)warp * QueryWarpSmemBytes(reach);
    QueryWarp w;
    w.rng = (uint2*)p;
    w.srt = w.rng + rcap;
    w.gc = (int*)(w.srt + rcap);
    w.nne = (uint32_t*)(w.gc + 96);
    return w;
}

// frame and grids the warp's chunk is queried against (its scene's, in a served batch)
struct QueryScene {
    Frame fr;
    const uint32_t *gridF, *gridB, *gridR;
};
__device__ __forceinline__ QueryScene ResolveScene(const QueryArgs& a, uint32_t chunk) {
    QueryScene sc;
    if (a.scenes) {
        const SceneGeom& g = a.scenes[a.chunkScene[chunk]];
        sc.fr = g.fr;
        sc.gridF = a.gridF ? a.gridF + g.gridOffF : nullptr;
        sc.gridB = a.gridB ? a.gridB + g.gridOffB : nullptr;
        sc.gridR = nullptr;
    } else {
        sc.fr = a.fr;
        sc.gridF = a.gridF; sc.gridB = a.gridB; sc.gridR = a.gridR;
    }
    return sc;
}

struct QueryLaneInfo {
    uint32_t i;
    bool inRange, valid;
    float4 pi;
    uint32_t g;        // group (distinct cell) of a valid lane, EMPTY_32 otherwise
    uint32_t nGroups;
};

__device__ __forceinline__ QueryLaneInfo QuerySetup(const QueryArgs& a, uint32_t chunk, uint32_t lane, const QueryWarp& w) {
    QueryLaneInfo q;
    q.i = chunk * SELL_W + lane;
    q.inRange = a.chunkLen ? lane < (uint32_t)a.chunkLen[chunk] : q.i < a.nF;
    const uint64_t cid = q.inRange ? a.cidF[q.i] : EMPTY_64;
    q.valid = cid != EMPTY_64;
    q.pi = q.inRange ? a.posF[q.i] : make_float4(0.f, 0.f, 0.f, 0.f);
    // out-of-frame particles (EMPTY cell ID) sort last, so valid lanes form a prefix of the chunk
    const uint64_t prevCid = __shfl_up_sync(0xffffffffu, cid, 1);
    const bool isStart = q.valid && (lane == 0 || prevCid != cid);
    const uint32_t startMask = __ballot_sync(0xffffffffu, isStart);
    q.nGroups = __popc(startMask);
    q.g = q.valid ? (uint32_t)__popc(startMask & (0xffffffffu >> (31u - lane))) - 1u : EMPTY_32;
    if (isStart) {
        w.gc[q.g] = (int)Compact21(cid);
        w.gc[32 + q.g] = (int)Compact21(cid >> 1);
        w.gc[64 + q.g] = (int)Compact21(cid >> 2);
    }
    __syncwarp();
    return q;
}

// stencil ranges of groups [g0, g0 + nb) of species SP, ranked by first index; RC is the
// frame's reach when known at compile time (1: cell size = kernel radius, the usual frame,
// where the stencil index arithmetic becomes constant multiplies), 0 to read it from the frame
template <int SP, int RC>
__device__ __forceinline__ void QueryRanges(const QueryArgs& a, const QueryScene& sc, const QueryWarp& w, uint32_t g0,
                                            uint32_t nb, uint32_t lane) {
    const uint32_t* grid = SP == 0 ? sc.gridF : SP == 1 ? sc.gridB : sc.gridR;
    const uint32_t* start = SP == 0 ? a.startF : SP == 1 ? a.startB : a.startR;
    const int r = RC ? RC : (int)sc.fr.reach, D = 2 * r + 1;
    const uint32_t sv = (uint32_t)(D * D * D), total = nb * sv;
    if (lane < nb) w.nne[lane] = 0;
    __syncwarp();
    for (uint32_t t = lane; t < total; t += 32) {
        const uint32_t gl = t / sv, s = t - gl * sv;
        const int x = w.gc[g0 + gl] + (int)(s % D) - r;
        const int y = w.gc[32 + g0 + gl] + (int)((s / D) % D) - r;
        const int z = w.gc[64 + g0 + gl] + (int)(s / (D * D)) - r;
        uint2 v = make_uint2(0u, 0u);
        if (x >= 0 && x < (int)sc.fr.nx && y >= 0 && y < (int)sc.fr.ny && z >= 0 && z < (int)sc.fr.nz) {
            const uint32_t c = grid[(uint64_t)x + (uint64_t)sc.fr.nx * ((uint64_t)y + (uint64_t)sc.fr.ny * z)];
            if (c != EMPTY_32) v = make_uint2(start[c], start[c + 1]);
        }
        w.rng[t] = v;
        if (v.x < v.y) atomicAdd(&w.nne[gl], 1u);
    }
    __syncwarp();
    for (uint32_t t = lane; t < total; t += 32) {
        const uint32_t gl = t / sv;
        const uint2 v = w.rng[t];
        if (v.x < v.y) {
            uint32_t rank = 0;
            const uint2* row = w.rng + gl * sv;
            for (uint32_t u = 0; u < sv; u++) {
                const uint2 o = row[u];
                rank += (o.x < o.y && o.x < v.x) ? 1u : 0u;
            }
            w.srt[gl * sv + rank] = v;
        }
    }
    __syncwarp();
}

enum WalkMode { WALK_COUNT = 0, WALK_STATS = 1, WALK_FILL = 2 };

// walk of each lane's own stencil candidates (ascending index order for F and B)
template <int SP, int MODE>
__device__ __forceinline__ void QueryWalk(const QueryArgs& a, const QueryScene& sc, const QueryWarp& w,
                                          const QueryLaneInfo& q, uint32_t g0, uint32_t nb, uint32_t lane,
                                          uint32_t homeLo, uint32_t homeHi, LaneRefs& ref, uint32_t* scr, uint32_t ks,
                                          LaneWriter& wr, const SellMeta& m) {
    const float4* pos = SP == 0 ? a.posF : SP == 1 ? a.posB : a.posR;
    const uint32_t sv = StencilVolume(sc.fr.reach);
    const bool mine = q.g != EMPTY_32 && q.g >= g0 && q.g < g0 + nb;
    const uint32_t gl = mine ? q.g - g0 : 0u;
    const uint32_t n = mine ? w.nne[gl] : 0u;
    const uint2* rows = w.srt + gl * sv;
    uint32_t k = 0, j = 0, e = 0;
    if (n > 0) { const uint2 v = rows[0]; j = v.x; e = v.y; }
    // count mode: rows go to the scratch through a running pointer (slot cnt of this lane);
    // min/max of F and B rows are their first/last entries (ascending), taken after the walk
    uint32_t* sp = scr + (uint64_t)ref.cnt * SELL_W;
    while (k < n) {
        const uint32_t jj = SP == 2 ? a.permR[j] : j;
        const float4 pj = pos[jj];
        const bool hit = IsNeighbor(q.pi.x, q.pi.y, q.pi.z, pj.x, pj.y, pj.z, a.r2);
        if (MODE == WALK_FILL) {
            if (hit) wr.store(m, lane, jj, a.err);
        } else if (MODE == WALK_COUNT) {
            if (hit && ref.cnt < ks) *sp = jj;
            if (hit) { sp += SELL_W; ref.cnt++; }
            if (SP == 2 && hit) { ref.mn = min(ref.mn, jj); ref.mx = max(ref.mx, jj); }
            if (SP != 2 && hit) ref.mx = jj;
        } else {
            if (hit) {
                ref.cnt++;
                ref.mn = min(ref.mn, jj);
                ref.mx = max(ref.mx, jj);
                if (jj < homeLo) ref.farLoMax = max(ref.farLoMax, jj);
                else if (jj > homeHi) ref.farHiMin = min(ref.farHiMin, jj);
                else ref.homeMin = min(ref.homeMin, jj);
            }
        }
        if (++j == e) {
            if (++k < n) { const uint2 v = rows[k]; j = v.x; e = v.y; }
        }
    }
}

// count walk of the fluid and boundary species, QUERY_WALK_U candidates of the current range per
// iteration (their loads in flight together, addressed from one pointer to the range's current
// candidate); same candidates, same order, same rows as QueryWalk. Hits are handled without
// branches: the row store is predicated, the slot count and the running maximum are selects.
#ifndef QUERY_WALK_U
#define QUERY_WALK_U 4
#endif
template <int SP>
__device__ __forceinline__ void QueryWalkCountU(const QueryArgs& a, const QueryScene& sc, const QueryWarp& w,
                                                const QueryLaneInfo& q, uint32_t g0, uint32_t nb, LaneRefs& ref,
                                                uint32_t* scr, uint32_t ks) {
    static_assert(SP != 2, "rigid candidates go through the permutation (QueryWalk)");
    constexpr uint32_t U = QUERY_WALK_U;
    const float4* pos = SP == 0 ? a.posF : a.posB;
    const uint32_t sv = StencilVolume(sc.fr.reach);
    const bool mine = q.g != EMPTY_32 && q.g >= g0 && q.g < g0 + nb;
    const uint32_t gl = mine ? q.g - g0 : 0u;
    const uint32_t n = mine ? w.nne[gl] : 0u;
    const uint2* rows = w.srt + gl * sv;
    const float xi = q.pi.x, yi = q.pi.y, zi = q.pi.z, r2 = a.r2;
    uint32_t k = 0, j = 0, e = 0;
    if (n > 0) { const uint2 v = rows[0]; j = v.x; e = v.y; }
    uint32_t cnt = ref.cnt, mx = ref.mx;
    while (k < n) {
        const uint32_t m = min(U, e - j);  // candidates of this iteration, all in the current range
        const float4* pp = pos + j;
        float4 p[U];
#pragma unroll
        for (uint32_t u = 0; u < U; u++) p[u] = (u < m) ? pp[u] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (uint32_t u = 0; u < U; u++) {
            const bool h = (u < m) && IsNeighbor(xi, yi, zi, p[u].x, p[u].y, p[u].z, r2);
            if (h && cnt < ks) scr[(size_t)cnt * SELL_W] = j + u;
            cnt += h ? 1u : 0u;
            mx = h ? j + u : mx;
        }
        j += m;
        if (j == e) {
            if (++k < n) { const uint2 v = rows[k]; j = v.x; e = v.y; }
        }
    }
    ref.cnt = cnt;
    ref.mx = mx;
}

// whole-chunk walk of one species in group batches
template <int SP, int MODE>
__device__ __forceinline__ void QuerySpecies(const QueryArgs& a, const QueryScene& sc, const QueryWarp& w,
                                             const QueryLaneInfo& q, uint32_t lane, uint32_t homeLo, uint32_t homeHi,
                                             LaneRefs& ref, uint32_t* scr, uint32_t ks, LaneWriter& wr,
                                             const SellMeta& m) {
    const uint32_t* grid = SP == 0 ? sc.gridF : SP == 1 ? sc.gridB : sc.gridR;
    if (grid == nullptr) return;
    const uint32_t gb = QueryGroupsPerBatch(sc.fr.reach);
    for (uint32_t g0 = 0; g0 < q.nGroups; g0 += gb) {
        const uint32_t nb = min(gb, q.nGroups - g0);
        if (sc.fr.reach == 1) QueryRanges<SP, 1>(a, sc, w, g0, nb, lane);
        else QueryRanges<SP, 0>(a, sc, w, g0, nb, lane);
        if constexpr (MODE == WALK_COUNT && SP != 2)
            QueryWalkCountU<SP>(a, sc, w, q, g0, nb, ref, scr, ks);
        else
            QueryWalk<SP, MODE>(a, sc, w, q, g0, nb, lane, homeLo, homeHi, ref, scr, ks, wr, m);
        __syncwarp();
    }
}

// home-window statistics of an FF row held in scratch (only needed when the chunk's index
// span exceeds 0xffff and the Delta16x2 home/far split is tried)
__device__ __forceinline__ void HomeStatsFromScratch(const uint32_t* scr, LaneRefs& ref, uint32_t homeLo,
                                                     uint32_t homeHi) {
    for (uint32_t k = 0; k < ref.cnt; k++) {
        const uint32_t j = scr[(uint64_t)k * SELL_W];
        if (j < homeLo) ref.farLoMax = max(ref.farLoMax, j);
        else if (j > homeHi) ref.farHiMin = min(ref.farHiMin, j);
        else ref.homeMin = min(ref.homeMin, j);
    }
}

// rest of the count pass after the FF walk (shared by both variants): FB and FR walks, the FF
// home-window statistics where needed, counts, neighbor totals and the chunk meta
__device__ __forceinline__ void QueryCountRest(const QueryArgs& a, const QueryScene& sc, const QueryWarp& w,
                                               const QueryLaneInfo& q, uint32_t chunk, uint32_t lane, LaneRefs& rFF,
                                               const uint32_t* sF, const SellMeta& mFF, const SellMeta& mFB,
                                               const SellMeta& mFR) {
    uint32_t homeLo, homeHi;
    HomeWindow(chunk, homeLo, homeHi);
    LaneRefs rFB, rFR;
    rFB.init(); rFR.init();
    LaneWriter none;
    uint32_t* sB = a.scrB + (uint64_t)chunk * a.ksB * SELL_W + lane;
    uint32_t* sR = a.scrR + (uint64_t)chunk * a.ksR * SELL_W + lane;
    QuerySpecies<1, WALK_COUNT>(a, sc, w, q, lane, homeLo, homeHi, rFB, sB, a.ksB, none, mFB);
    QuerySpecies<2, WALK_COUNT>(a, sc, w, q, lane, homeLo, homeHi, rFR, sR, a.ksR, none, mFR);
    // F and B rows are ascending: the minimum is the first stored entry
    if (rFF.cnt) rFF.mn = sF[0];
    if (rFB.cnt) rFB.mn = sB[0];
    const uint32_t over = (__any_sync(0xffffffffu, rFF.cnt > a.ksF) ? 1u : 0u) |
                          (__any_sync(0xffffffffu, rFB.cnt > a.ksB) ? 2u : 0u) |
                          (__any_sync(0xffffffffu, rFR.cnt > a.ksR) ? 4u : 0u);
    // the FF home/far split needs per-lane window statistics only when the span exceeds 16 bits
    uint32_t mn = rFF.mn, mx = rFF.mx;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, d));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
    }
    if (mx >= mn && mx - mn > 0xffffu) {
        if (!(over & 1u)) {
            HomeStatsFromScratch(sF, rFF, homeLo, homeHi);
        } else {
            LaneRefs s;
            s.init();
            QuerySpecies<0, WALK_STATS>(a, sc, w, q, lane, homeLo, homeHi, s, nullptr, 0, none, mFF);
            rFF.homeMin = s.homeMin; rFF.farLoMax = s.farLoMax; rFF.farHiMin = s.farHiMin;
        }
    }
    if (lane == 0) a.scrOver[chunk] = (uint8_t)over;
    if (q.inRange) {
        if ((rFF.cnt | rFB.cnt | rFR.cnt) > 0xffffu) atomicOr(a.err, ERR_COUNT_U16);
        mFF.counts[q.i] = (uint16_t)rFF.cnt;
        mFB.counts[q.i] = (uint16_t)rFB.cnt;
        mFR.counts[q.i] = (uint16_t)rFR.cnt;
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

// count pass: neighbor counts, chunk compression meta, rows into the per-chunk scratch.
// Instantiated per minimum resident blocks per SM (QUERY_COUNT_CANDIDATES: X plain, XS with the
// neighboring cell blocks staged in shared memory, below), chosen by the autotuner; an earlier
// hand sweep on the 1M dam (ms per count pass): 1 block (78 registers) 0.393, none given (64
// registers) 0.350, 9 (56) 0.332, 10 (48) 0.348, 12 (40, spills) 0.338
#define QUERY_COUNT_CANDIDATES(X, XS) X(6) X(8) X(9) X(10) X(12) XS(4) XS(5)
#define QUERY_FILL_CANDIDATES(X) X(8) X(10) X(12) X(16)
template <int MB>
__global__ void __launch_bounds__(QUERY_THREADS, MB) KQueryFluidCount(QueryArgs a, SellMeta mFF, SellMeta mFB, SellMeta mFR) {
    extern __shared__ uint2 qsm[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t chunk = blockIdx.x * (QUERY_THREADS / 32) + warp;
    const uint32_t nChunks = (a.nF + SELL_W - 1) / SELL_W;
    if (chunk >= nChunks) return;  // uniform per warp
    const QueryScene sc = ResolveScene(a, chunk);
    const QueryWarp w = QueryWarpSmem(qsm, warp, a.fr.reach);
    const QueryLaneInfo q = QuerySetup(a, chunk, lane, w);
    uint32_t homeLo, homeHi;
    HomeWindow(chunk, homeLo, homeHi);
    LaneRefs rFF;
    rFF.init();
    LaneWriter none;
    uint32_t* sF = a.scrF + (uint64_t)chunk * a.ksF * SELL_W + lane;
    QuerySpecies<0, WALK_COUNT>(a, sc, w, q, lane, homeLo, homeHi, rFF, sF, a.ksF, none, mFF);
    QueryCountRest(a, sc, w, q, chunk, lane, rFF, sF, mFF, mFB, mFR);
}

// ---- count pass with the neighboring cell blocks staged in shared memory
//
// A block's four chunks are 128 consecutive particles in Morton order, so their cells and the
// strict stencils of those cells lie in a small box of the frame (at 8 particles per cell about
// 6 x 4 x 4 cells). This variant looks up every cell of that box once (range from the dense grid
// and the cell table), copies the particles of each non-empty cell into shared memory with one
// TMA bulk copy per cell (cp.async.bulk global -> shared, completion counted in bytes on one
// mbarrier, wait bounded), takes the FF stencil ranges from the box table and walks candidate
// positions in shared memory instead of through L1. Same candidates in the same order, so the
// same rows. A block whose box exceeds STAGE_BOX_CAP cells or STAGE_CAP particles, or whose
// chunks belong to different scenes of a served batch, reads global memory like the plain
// variant. FB and FR walks are unchanged (boundary cells are mostly empty inside the fluid).
constexpr uint32_t STAGE_BOX_CAP = 256, STAGE_CAP = 1024;
constexpr uint32_t STAGE_WAIT_LIMIT = 1u << 20;

__device__ __forceinline__ uint32_t SmemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void MbarInit(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void MbarArriveExpectTx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool MbarTryWait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(SmemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}
// bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global memory
// into this CTA's shared memory, completion signalled on `bar`
__device__ __forceinline__ void BulkCopyG2S(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     SmemAddr(dst)),
                 "l"(src), "r"(bytes), "r"(SmemAddr(bar))
                 : "memory");
}

__host__ __device__ __forceinline__ size_t StageOffBytes(uint32_t reach) {
    return ((size_t)QueryRangeCap(reach) * 2u * sizeof(uint16_t) + 15u) & ~(size_t)15u;
}
__host__ __device__ __forceinline__ size_t QueryStagedSmemBytes(uint32_t reach) {
    return (QueryWarpSmemBytes(reach) + StageOffBytes(reach)) * (QUERY_THREADS / 32) + (size_t)STAGE_CAP * sizeof(float4) +
           (size_t)STAGE_BOX_CAP * 3u * sizeof(uint32_t);
}

struct StageBox {
    const float4* stage;                      // staged particles, cell after cell in box order
    const uint32_t *beg, *len, *off;          // per box cell: first particle, count, stage offset
    int x0, y0, z0;
    uint32_t bx, by, vol;
    uint16_t *offU, *offS;                    // this warp's stage offsets of its stencil slots
};

// FF stencil ranges of groups [g0, g0 + nb) from the box table, ranked by first index, with the
// stage offset of each ranked range (QueryRanges for staged particles)
__device__ __forceinline__ void QueryRangesStaged(const QueryArgs& a, const QueryScene& sc, const QueryWarp& w,
                                                  const StageBox& bx, uint32_t g0, uint32_t nb, uint32_t lane) {
    const int r = (int)sc.fr.reach, D = 2 * r + 1;
    const uint32_t sv = (uint32_t)(D * D * D), total = nb * sv;
    if (lane < nb) w.nne[lane] = 0;
    __syncwarp();
    for (uint32_t t = lane; t < total; t += 32) {
        const uint32_t gl = t / sv, s = t - gl * sv;
        const int x = w.gc[g0 + gl] + (int)(s % D) - r;
        const int y = w.gc[32 + g0 + gl] + (int)((s / D) % D) - r;
        const int z = w.gc[64 + g0 + gl] + (int)(s / (D * D)) - r;
        uint2 v = make_uint2(0u, 0u);
        uint32_t o = 0u;
        if (x >= 0 && x < (int)sc.fr.nx && y >= 0 && y < (int)sc.fr.ny && z >= 0 && z < (int)sc.fr.nz) {
            // inside the box by construction (box = the groups' cells widened by the reach)
            const uint32_t b = (uint32_t)(x - bx.x0) + bx.bx * ((uint32_t)(y - bx.y0) + bx.by * (uint32_t)(z - bx.z0));
            if (b < bx.vol) {
                v = make_uint2(bx.beg[b], bx.beg[b] + bx.len[b]);
                o = bx.off[b];
            } else {
                atomicOr(a.err, ERR_QUERY_CAP);
            }
        }
        w.rng[t] = v;
        bx.offU[t] = (uint16_t)o;
        if (v.x < v.y) atomicAdd(&w.nne[gl], 1u);
    }
    __syncwarp();
    for (uint32_t t = lane; t < total; t += 32) {
        const uint32_t gl = t / sv;
        const uint2 v = w.rng[t];
        if (v.x < v.y) {
            uint32_t rank = 0;
            const uint2* row = w.rng + gl * sv;
            for (uint32_t u = 0; u < sv; u++) {
                const uint2 o = row[u];
                rank += (o.x < o.y && o.x < v.x) ? 1u : 0u;
            }
            w.srt[gl * sv + rank] = v;
            bx.offS[gl * sv + rank] = bx.offU[t];
        }
    }
    __syncwarp();
}

// QueryWalkCountU over staged FF candidates: the position of candidate j of a ranked range
// (begin, end) with stage offset o is stage[o + (j - begin)]
__device__ __forceinline__ void QueryWalkCountStaged(const QueryArgs& a, const QueryScene& sc, const QueryWarp& w,
                                                     const StageBox& bx, const QueryLaneInfo& q, uint32_t g0,
                                                     uint32_t nb, LaneRefs& ref, uint32_t* scr, uint32_t ks) {
    constexpr uint32_t U = QUERY_WALK_U;
    const uint32_t sv = StencilVolume(sc.fr.reach);
    const bool mine = q.g != EMPTY_32 && q.g >= g0 && q.g < g0 + nb;
    const uint32_t gl = mine ? q.g - g0 : 0u;
    const uint32_t n = mine ? w.nne[gl] : 0u;
    const uint2* rows = w.srt + gl * sv;
    const uint16_t* offs = bx.offS + gl * sv;
    const float xi = q.pi.x, yi = q.pi.y, zi = q.pi.z, r2 = a.r2;
    uint32_t k = 0, j = 0, e = 0, so = 0;
    if (n > 0) { const uint2 v = rows[0]; j = v.x; e = v.y; so = offs[0]; }
    uint32_t cnt = ref.cnt, mx = ref.mx;
    while (k < n) {
        const uint32_t m = min(U, e - j);
        const float4* pp = bx.stage + so;
        float4 p[U];
#pragma unroll
        for (uint32_t u = 0; u < U; u++) p[u] = (u < m) ? pp[u] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (uint32_t u = 0; u < U; u++) {
            const bool h = (u < m) && IsNeighbor(xi, yi, zi, p[u].x, p[u].y, p[u].z, r2);
            if (h && cnt < ks) scr[(size_t)cnt * SELL_W] = j + u;
            cnt += h ? 1u : 0u;
            mx = h ? j + u : mx;
        }
        j += m;
        so += m;
        if (j == e) {
            if (++k < n) { const uint2 v = rows[k]; j = v.x; e = v.y; so = offs[k]; }
        }
    }
    ref.cnt = cnt;
    ref.mx = mx;
}

template <int MB>
__global__ void __launch_bounds__(QUERY_THREADS, MB)
    KQueryFluidCountStaged(QueryArgs a, SellMeta mFF, SellMeta mFB, SellMeta mFR) {
    extern __shared__ float4 qsmS[];
    constexpr uint32_t W = QUERY_THREADS / 32;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t chunk0 = blockIdx.x * W, chunk = chunk0 + warp;
    const uint32_t nChunks = (a.nF + SELL_W - 1) / SELL_W;
    const bool active = chunk < nChunks;  // chunk0 < nChunks for every launched block
    const uint32_t reach = a.fr.reach;
    char* base = reinterpret_cast<char*>(qsmS);
    const size_t wsz = QueryWarpSmemBytes(reach), osz = StageOffBytes(reach);
    const QueryWarp w = QueryWarpSmem(base, warp, reach);
    float4* stage = reinterpret_cast<float4*>(base + W * (wsz + osz));
    uint32_t* boxBeg = reinterpret_cast<uint32_t*>(stage + STAGE_CAP);
    uint32_t* boxLen = boxBeg + STAGE_BOX_CAP;
    uint32_t* boxOff = boxLen + STAGE_BOX_CAP;
    __shared__ int sLo[3], sHi[3];
    __shared__ uint32_t sScene[2], sWarpTot[W], sTot;
    __shared__ __align__(8) uint64_t sBar;
    if (tid < 3) { sLo[tid] = INT_MAX; sHi[tid] = INT_MIN; }
    if (tid == 0) {
        sScene[0] = 0xffffffffu; sScene[1] = 0u;
        MbarInit(&sBar, 1u);
    }
    __syncthreads();
    // the block's FF cell box: bounds of its chunks' cells (one entry per distinct cell)
    QueryLaneInfo q{};
    if (active) {
        q = QuerySetup(a, chunk, lane, w);
        if (lane < q.nGroups) {
            atomicMin(&sLo[0], w.gc[lane]); atomicMax(&sHi[0], w.gc[lane]);
            atomicMin(&sLo[1], w.gc[32 + lane]); atomicMax(&sHi[1], w.gc[32 + lane]);
            atomicMin(&sLo[2], w.gc[64 + lane]); atomicMax(&sHi[2], w.gc[64 + lane]);
        }
        if (lane == 0 && a.scenes) {
            atomicMin(&sScene[0], a.chunkScene[chunk]);
            atomicMax(&sScene[1], a.chunkScene[chunk]);
        }
    }
    __syncthreads();
    const QueryScene s0 = ResolveScene(a, chunk0);
    StageBox bx{};
    bx.offU = reinterpret_cast<uint16_t*>(base + W * wsz + warp * osz);
    bx.offS = bx.offU + QueryRangeCap(reach);
    bool ok = s0.gridF != nullptr && sLo[0] <= sHi[0] && (a.scenes == nullptr || sScene[0] == sScene[1]);
    if (ok) {
        const int r = (int)s0.fr.reach;
        bx.x0 = max(sLo[0] - r, 0); bx.y0 = max(sLo[1] - r, 0); bx.z0 = max(sLo[2] - r, 0);
        const int x1 = min(sHi[0] + r, (int)s0.fr.nx - 1), y1 = min(sHi[1] + r, (int)s0.fr.ny - 1),
                  z1 = min(sHi[2] + r, (int)s0.fr.nz - 1);
        const uint64_t vol = (uint64_t)(x1 - bx.x0 + 1) * (uint64_t)(y1 - bx.y0 + 1) * (uint64_t)(z1 - bx.z0 + 1);
        ok = x1 >= bx.x0 && y1 >= bx.y0 && z1 >= bx.z0 && vol <= STAGE_BOX_CAP;
        bx.bx = (uint32_t)(x1 - bx.x0 + 1); bx.by = (uint32_t)(y1 - bx.y0 + 1); bx.vol = ok ? (uint32_t)vol : 0u;
    }
    // ok is the same in every thread of the block (computed from shared values)
    if (ok) {
        for (uint32_t b = tid; b < bx.vol; b += QUERY_THREADS) {
            const uint32_t xx = b % bx.bx, yy = (b / bx.bx) % bx.by, zz = b / (bx.bx * bx.by);
            const uint32_t c = s0.gridF[(uint64_t)(bx.x0 + (int)xx) +
                                        (uint64_t)s0.fr.nx * ((uint64_t)(bx.y0 + (int)yy) +
                                                              (uint64_t)s0.fr.ny * (uint64_t)(bx.z0 + (int)zz))];
            uint32_t bg = 0u, ln = 0u;
            if (c != EMPTY_32) { bg = a.startF[c]; ln = a.startF[c + 1] - bg; }
            boxBeg[b] = bg;
            boxLen[b] = ln;
        }
        __syncthreads();
        // exclusive scan of the cell counts, two box cells per thread (STAGE_BOX_CAP = 2 x threads)
        const uint32_t b0 = 2u * tid;
        const uint32_t l0 = b0 < bx.vol ? boxLen[b0] : 0u, l1 = b0 + 1u < bx.vol ? boxLen[b0 + 1u] : 0u;
        uint32_t incl = l0 + l1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
            if ((int)lane >= d) incl += v;
        }
        if (lane == 31) sWarpTot[warp] = incl;
        __syncthreads();
        uint32_t pre = 0u;
        for (uint32_t v = 0; v < warp; v++) pre += sWarpTot[v];
        const uint32_t ex = pre + incl - (l0 + l1);
        if (b0 < bx.vol) boxOff[b0] = ex;
        if (b0 + 1u < bx.vol) boxOff[b0 + 1u] = ex + l0;
        if (tid == QUERY_THREADS - 1u) sTot = pre + incl;
    }
    __syncthreads();
    const uint32_t T = ok ? sTot : 0u;
    bool staged = ok && T <= STAGE_CAP;
    if (staged) {
        if (tid == 0) MbarArriveExpectTx(&sBar, T * (uint32_t)sizeof(float4));
        __syncthreads();  // the expected byte count is posted before any copy can complete
        for (uint32_t b = tid; b < bx.vol; b += QUERY_THREADS)
            if (boxLen[b]) BulkCopyG2S(stage + boxOff[b], a.posF + boxBeg[b], boxLen[b] * (uint32_t)sizeof(float4), &sBar);
        bool done = false;
        for (uint32_t spin = 0; spin < STAGE_WAIT_LIMIT && !done; spin++) done = MbarTryWait(&sBar, 0u);
        if (!done) atomicOr(a.err, ERR_STAGE_WAIT);
        staged = __syncthreads_and(done ? 1 : 0) != 0;
    }
    if (!active) return;  // no block-wide barrier below
    bx.stage = stage; bx.beg = boxBeg; bx.len = boxLen; bx.off = boxOff;
    const QueryScene sc = ResolveScene(a, chunk);
    uint32_t homeLo, homeHi;
    HomeWindow(chunk, homeLo, homeHi);
    LaneRefs rFF;
    rFF.init();
    LaneWriter none;
    uint32_t* sF = a.scrF + (uint64_t)chunk * a.ksF * SELL_W + lane;
    if (staged) {
        const uint32_t gb = QueryGroupsPerBatch(sc.fr.reach);
        for (uint32_t g0 = 0; g0 < q.nGroups; g0 += gb) {
            const uint32_t nb = min(gb, q.nGroups - g0);
            QueryRangesStaged(a, sc, w, bx, g0, nb, lane);
            QueryWalkCountStaged(a, sc, w, bx, q, g0, nb, rFF, sF, a.ksF);
            __syncwarp();
        }
    } else {
        QuerySpecies<0, WALK_COUNT>(a, sc, w, q, lane, homeLo, homeHi, rFF, sF, a.ksF, none, mFF);
    }
    QueryCountRest(a, sc, w, q, chunk, lane, rFF, sF, mFF, mFB, mFR);
}

// encode one species' scratch rows of a chunk into its SELL32 slice. The scratch and the slice
// share the [slot][lane] layout, so each thread takes four adjacent lanes of one slot: one
// 16-byte scratch load, four codes (StoreNeighbor_CompressedSell32,
// neighbor_search_kernels.cu:193-247), one 8-byte (Delta16x2) or 16-byte (Abs32) store; the
// warp's eight quarter-rows cover four slots per round. Slots past a lane's count (padding up
// to the chunk's pitch, never read by the sweeps) are written as zero. Every slot of the slice
// lies inside the scratch (pitch <= slots per lane when the chunk did not overflow), and the
// offsets of chunks are multiples of 32 entries, so the vector accesses are aligned.
__device__ __forceinline__ void EncodeFromScratch(const SellMeta& m, LaneWriter& wr, const uint32_t* scrChunk,
                                                  uint32_t cnt, uint32_t lane, uint32_t* err) {
    const uint32_t sub = lane & 7u, kFirst = lane >> 3;
    uint32_t c[4];
#pragma unroll
    for (uint32_t q = 0; q < 4; q++) c[q] = __shfl_sync(0xffffffffu, cnt, 4u * sub + q);
    const bool d16 = wr.fmt == FMT_DELTA16X2;
    const uint64_t cap = d16 ? m.cap16 : m.cap32;
    uint32_t errBits = 0u;
    constexpr uint32_t B = 4;  // rounds whose loads are in flight together
    for (uint32_t kb = kFirst; kb < wr.pitch; kb += 4u * B) {
        uint4 v[B];
#pragma unroll
        for (uint32_t b = 0; b < B; b++) {
            const uint32_t k = kb + 4u * b;
            v[b] = k < wr.pitch ? __ldcs(reinterpret_cast<const uint4*>(scrChunk + (size_t)k * SELL_W + 4u * sub))
                                : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (uint32_t b = 0; b < B; b++) {
            const uint32_t k = kb + 4u * b;
            if (k >= wr.pitch) break;
            const uint64_t lin = wr.off + (uint64_t)k * SELL_W + 4u * sub;
            if (lin + 4u > cap) { errBits |= ERR_FILL_OVERFLOW; continue; }
            const uint32_t j[4] = {v[b].x, v[b].y, v[b].z, v[b].w};
            uint32_t code[4];
#pragma unroll
            for (uint32_t q = 0; q < 4; q++) {
                const bool valid = k < c[q];
                if (d16) {
                    const bool first = j[q] >= wr.base && j[q] - wr.base <= 0x7fffu;
                    const bool second = j[q] >= wr.base2 && j[q] - wr.base2 <= 0x7fffu;
                    if (valid && !first && !second) errBits |= ERR_DELTA_RANGE;
                    code[q] = !valid ? 0u : first ? j[q] - wr.base : (0x8000u | (j[q] - wr.base2));
                } else {
                    code[q] = valid ? j[q] : 0u;
                }
            }
            if (d16)
                *reinterpret_cast<uint2*>(m.list16 + lin) = make_uint2(code[0] | (code[1] << 16), code[2] | (code[3] << 16));
            else
                *reinterpret_cast<uint4*>(m.list32 + lin) = make_uint4(code[0], code[1], code[2], code[3]);
        }
    }
    if (errBits) atomicOr(err, errBits);
    wr.wr = cnt;  // every slot below the lane's count is written
}

// fill pass: scratch rows -> SELL32 (a chunk whose scratch overflowed walks its stencil again);
// instantiated per minimum resident blocks per SM (QUERY_FILL_CANDIDATES), an earlier hand sweep
// on the 1M dam (ms per fill pass): none given 0.088, 8 0.086, 10 0.084, 12 0.095, 16 0.103
template <int MB>
__global__ void __launch_bounds__(QUERY_THREADS, MB) KQueryFluidFill(QueryArgs a, SellMeta mFF, SellMeta mFB, SellMeta mFR) {
    extern __shared__ uint2 qsm[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t chunk = blockIdx.x * (QUERY_THREADS / 32) + warp;
    const uint32_t nChunks = (a.nF + SELL_W - 1) / SELL_W;
    if (chunk >= nChunks) return;
    const uint32_t i = chunk * SELL_W + lane;
    const bool inRange = a.chunkLen ? lane < (uint32_t)a.chunkLen[chunk] : i < a.nF;
    const uint32_t over = a.scrOver[chunk];
    LaneWriter wFF, wFB, wFR;
    wFF.init(mFF, chunk); wFB.init(mFB, chunk); wFR.init(mFR, chunk);
    const uint32_t* sF = a.scrF + (uint64_t)chunk * a.ksF * SELL_W;
    const uint32_t* sB = a.scrB + (uint64_t)chunk * a.ksB * SELL_W;
    const uint32_t* sR = a.scrR + (uint64_t)chunk * a.ksR * SELL_W;
    if (!(over & 1u)) EncodeFromScratch(mFF, wFF, sF, inRange ? mFF.counts[i] : 0u, lane, a.err);
    if (!(over & 2u)) EncodeFromScratch(mFB, wFB, sB, inRange ? mFB.counts[i] : 0u, lane, a.err);
    if (!(over & 4u)) EncodeFromScratch(mFR, wFR, sR, inRange ? mFR.counts[i] : 0u, lane, a.err);
    if (over) {
        const QueryScene sc = ResolveScene(a, chunk);
        const QueryWarp w = QueryWarpSmem(qsm, warp, a.fr.reach);
        const QueryLaneInfo q = QuerySetup(a, chunk, lane, w);
        LaneRefs none;
        none.init();
        if (over & 1u) QuerySpecies<0, WALK_FILL>(a, sc, w, q, lane, 0u, 0u, none, nullptr, 0u, wFF, mFF);
        if (over & 2u) QuerySpecies<1, WALK_FILL>(a, sc, w, q, lane, 0u, 0u, none, nullptr, 0u, wFB, mFB);
        if (over & 4u) QuerySpecies<2, WALK_FILL>(a, sc, w, q, lane, 0u, 0u, none, nullptr, 0u, wFR, mFR);
    }
    if (inRange && wFR.wr > 1) SortRowSell(mFR, wFR, lane);
}

uint32_t QueryCap(uint32_t reach) { return QueryRangeCap(reach); }
size_t QuerySmemBytes(uint32_t reach) { return QueryWarpSmemBytes(reach) * (QUERY_THREADS / 32); }
size_t QueryScratchWords(uint32_t nChunks, uint32_t ks) { return (size_t)nChunks * ks * SELL_W; }

// `slots` of a count-pass candidate: 1 = neighboring cell blocks staged in shared memory
#define TSP_QC_ENTRY(mb) TuneCandidate{0, mb},
#define TSP_QS_ENTRY(mb) TuneCandidate{1, mb},
static const TuneCandidate kCountCandidates[] = {QUERY_COUNT_CANDIDATES(TSP_QC_ENTRY, TSP_QS_ENTRY)};
static const TuneCandidate kFillCandidates[] = {QUERY_FILL_CANDIDATES(TSP_QC_ENTRY)};
#undef TSP_QC_ENTRY
#undef TSP_QS_ENTRY
using QueryKernel = void (*)(QueryArgs, SellMeta, SellMeta, SellMeta);
#define TSP_QC_FN(mb) &KQueryFluidCount<mb>,
#define TSP_QS_FN(mb) &KQueryFluidCountStaged<mb>,
#define TSP_QF_FN(mb) &KQueryFluidFill<mb>,
static const QueryKernel kCountFns[] = {QUERY_COUNT_CANDIDATES(TSP_QC_FN, TSP_QS_FN)};
static const QueryKernel kFillFns[] = {QUERY_FILL_CANDIDATES(TSP_QF_FN)};
#undef TSP_QC_FN
#undef TSP_QS_FN
#undef TSP_QF_FN
const TuneCandidate* QueryCandidates(bool fill, int* n) {
    *n = fill ? (int)(sizeof(kFillCandidates) / sizeof(kFillCandidates[0]))
              : (int)(sizeof(kCountCandidates) / sizeof(kCountCandidates[0]));
    return fill ? kFillCandidates : kCountCandidates;
}

void LaunchQueryFluid(bool fill, const QueryArgs& a, const SellMeta& ff, const SellMeta& fb, const SellMeta& fr,
                      cudaStream_t s, int variant) {
    const uint32_t nChunks = (a.nF + SELL_W - 1) / SELL_W;
    if (nChunks == 0) return;
    const uint32_t warps = QUERY_THREADS / 32;
    const uint32_t blocks = (nChunks + warps - 1) / warps;
    int nc = 0;
    const TuneCandidate* cand = QueryCandidates(fill, &nc);
    const TuneKernel k = fill ? TUNE_QUERY_FILL : TUNE_QUERY_COUNT;
    int v = variant;
    if (v < 0 || v >= nc) {
        v = TuneChoice(k, a.nF);
        if (v < 0) v = TuneDefault(k);
    }
    bool staged = !fill && cand[v].slots == 1u;
    if (staged && QueryStagedSmemBytes(a.fr.reach) > 227u * 1024u) {  // large reach: plain variant
        v = TuneDefault(k);
        staged = false;
    }
    const size_t smem = staged ? QueryStagedSmemBytes(a.fr.reach) : QueryWarpSmemBytes(a.fr.reach) * warps;
    const QueryKernel fn = fill ? kFillFns[v] : kCountFns[v];
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    fn<<<blocks, QUERY_THREADS, smem, s>>>(a, ff, fb, fr);
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

// The same three scans (FF, FB, FR lists) in one launch: block b scans list b, each thread a
// contiguous run of chunks (local sums, block-wide exclusive scan of the thread sums, then the
// offsets of its run). Integer sums: the offsets and totals equal the three-kernel scan's.
constexpr uint32_t SELL3_THREADS = 1024;
constexpr uint32_t SELL3_MAX_CHUNKS = 64u * SELL3_THREADS;
__global__ void __launch_bounds__(SELL3_THREADS) KFinalizeSell3(SellMeta m0, SellMeta m1, SellMeta m2, uint32_t nChunks,
                                                               U64x2* __restrict__ totals) {
    __shared__ U64x2 warpSum[SELL3_THREADS / 32];
    const SellMeta& m = blockIdx.x == 0 ? m0 : (blockIdx.x == 1 ? m1 : m2);
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t seg = (nChunks + SELL3_THREADS - 1) / SELL3_THREADS;
    const uint32_t beg = min(t * seg, nChunks), end = min(beg + seg, nChunks);
    U64x2 own{0, 0};
#pragma unroll 8
    for (uint32_t c = beg; c < end; c++) {
        const uint64_t sz = (uint64_t)m.pitch[c] * SELL_W;
        if (m.format[c] == FMT_DELTA16X2) own.a += sz;
        else own.b += sz;
    }
    U64x2 incl = own;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const U64x2 o = ShflUp(incl, d);
        if ((int)lane >= d) incl = incl + o;
    }
    if (lane == 31) warpSum[warp] = incl;
    __syncthreads();
    U64x2 pre{0, 0}, tot{0, 0};
    for (uint32_t w = 0; w < SELL3_THREADS / 32; w++) {
        if (w < warp) pre = pre + warpSum[w];
        tot = tot + warpSum[w];
    }
    U64x2 run = pre + incl;
    run.a -= own.a;
    run.b -= own.b;
#pragma unroll 8
    for (uint32_t c = beg; c < end; c++) {
        const uint64_t sz = (uint64_t)m.pitch[c] * SELL_W;
        if (m.format[c] == FMT_DELTA16X2) { m.offset[c] = run.a; run.a += sz; }
        else { m.offset[c] = run.b; run.b += sz; }
    }
    if (t == 0) totals[blockIdx.x] = tot;
}
void FinalizeSell3(const SellMeta& m0, const SellMeta& m1, const SellMeta& m2, uint32_t nChunks, U64x2* scratch,
                   U64x2* totals, cudaStream_t s) {
    if (nChunks > 0 && nChunks <= SELL3_MAX_CHUNKS) {
        KFinalizeSell3<<<3, SELL3_THREADS, 0, s>>>(m0, m1, m2, nChunks, totals);
        return;
    }
    FinalizeSell(m0, nChunks, scratch, totals + 0, s);
    FinalizeSell(m1, nChunks, scratch, totals + 1, s);
    FinalizeSell(m2, nChunks, scratch, totals + 2, s);
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
