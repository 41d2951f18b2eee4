// batch.cu -- served batch: many independent scenes advanced together, one substep at a time,
// over one scene-offset fluid array.
//
// Layout. All admitted scenes' fluid particles live in one arena, scene after scene in rank
// order, each scene padded to whole SELL32 chunks (the padding lanes are never valid, never in
// a cell and never a neighbor). Per chunk the arena records its scene and its number of valid
// lanes, so every chunk-per-warp kernel of the one-scene path (query, density, non-pressure,
// source/diagonal, pressure acceleration, Jacobi, integration) runs over all scenes in one
// launch. Boundary particles of a scene occupy a range of a boundary arena, with its own cell
// table and dense grid, built once when the scene is admitted and again when its frame changes.
//
// Per substep: one probe over the arena (per-scene AABB + "left the inner frame" flags, one
// read-back for all scenes), host frame rule per scene, one radix sort of (scene rank, Morton
// key) composite keys -- a stable sort by scene then cell, so each scene's order is exactly the
// order it gets alone -- one reorder, one cell table and grid scatter, one query count, one
// size read-back, one fill, then the solver stages and a Jacobi loop (CUDA graph, conditional
// WHILE node) whose sweeps skip converged scenes and whose FP64 residuals are reduced per scene
// in a fixed order. A scene's results do not depend on which other scenes share the batch.
//
// Admission reserves an estimate of the scene's device memory against a fixed budget; a scene
// that does not fit is refused (the caller queues it). Admissions and retirements take effect
// at the next substep (one relayout of the fluid arena for all of them).
#include <cstdio>
#include <cstring>
#include <map>
#include <type_traits>
#include <memory>
#include <vector>

#include "../../include/tsp_b200.h"
#include "kernels.h"
#include "primitives.cuh"
#include "host_common.h"

namespace tsp {

// per scene (indexed by rank), device side
struct BatchSceneDev {
    Frame fr;
    DomainBox dom;
    uint64_t emptyKey;
    int frameValid;
    uint32_t chunkBegin, chunkEnd;  // chunks of the scene in the arena
    uint32_t nF;                    // real fluid particles (average-error denominator)
};
struct BatchSolverDev {
    double sums[3];
    float avg[3];
    uint32_t iters, itersTotal, done;
};

// ------------------------------------------------------------------------------ kernels
__device__ __forceinline__ int OrderedIntDev(float f) {
    const int i = __float_as_int(f);
    return (i >= 0) ? i : (i ^ 0x7fffffff);
}

__global__ void KBatchProbeReset(ProbeResult* out, uint32_t S, int lo, int hi) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    for (int a = 0; a < 3; a++) { out[s].mnKey[a] = lo; out[s].mxKey[a] = hi; }
    out[s].exceeded = 0;
    out[s].pad = 0;
}

// one warp per chunk (= one scene): AABB and inner-frame test (neighbor_search.cpp:1902-2006)
__global__ void __launch_bounds__(256) KBatchProbe(const float4* __restrict__ pos, uint32_t nChunks,
                                                  const uint8_t* __restrict__ chunkLen,
                                                  const uint32_t* __restrict__ chunkScene,
                                                  const BatchSceneDev* __restrict__ sc, ProbeResult* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t chunk = i >> 5, lane = i & 31, warp = threadIdx.x >> 5;
    const bool live = chunk < nChunks;  // whole warps
    const uint32_t s = live ? chunkScene[chunk] : EMPTY_32;
    const BatchSceneDev& d = sc[live ? s : 0u];
    const bool act = live && lane < (uint32_t)chunkLen[chunk];
    float mn[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
    float mx[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    uint32_t exceeded = 0;
    if (act) {
        const float4 p = pos[i];
        mn[0] = p.x; mn[1] = p.y; mn[2] = p.z;
        mx[0] = p.x; mx[1] = p.y; mx[2] = p.z;
        if (d.frameValid) {
            const DomainBox& dom = d.dom;
            const bool inside = !dom.bounded || (p.x >= dom.mn[0] && p.x <= dom.mx[0] && p.y >= dom.mn[1] &&
                                                 p.y <= dom.mx[1] && p.z >= dom.mn[2] && p.z <= dom.mx[2]);
            if (inside) {
                const Frame& fr = d.fr;
                const int m = (int)fr.reach;
                const int cx = FloorToInt(p.x * fr.cellSizeInv), cy = FloorToInt(p.y * fr.cellSizeInv),
                          cz = FloorToInt(p.z * fr.cellSizeInv);
                if (cx < fr.ox + m || cx > fr.ox + (int)fr.nx - 1 - m || cy < fr.oy + m ||
                    cy > fr.oy + (int)fr.ny - 1 - m || cz < fr.oz + m || cz > fr.oz + (int)fr.nz - 1 - m)
                    exceeded = 1;
            }
        }
    }
#pragma unroll
    for (int dd = 16; dd > 0; dd >>= 1)
        for (int a = 0; a < 3; a++) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], dd));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], dd));
        }
    exceeded = __any_sync(0xffffffffu, exceeded);
    // the block's warps merged per scene (a scene's chunks are contiguous, so a block mostly
    // holds one or two scenes), then one set of global atomics per scene run
    __shared__ float smn[3][8], smx[3][8];
    __shared__ uint32_t sex[8], ssc[8];
    if (lane == 0) {
        for (int a = 0; a < 3; a++) { smn[a][warp] = mn[a]; smx[a][warp] = mx[a]; }
        sex[warp] = exceeded;
        ssc[warp] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const uint32_t nw = blockDim.x >> 5;
    for (uint32_t w = 0; w < nw;) {
        const uint32_t cs = ssc[w];
        if (cs == EMPTY_32) break;
        float a0[3], a1[3];
        uint32_t ex = 0;
        for (int a = 0; a < 3; a++) { a0[a] = smn[a][w]; a1[a] = smx[a][w]; }
        for (; w < nw && ssc[w] == cs; w++) {
            for (int a = 0; a < 3; a++) { a0[a] = fminf(a0[a], smn[a][w]); a1[a] = fmaxf(a1[a], smx[a][w]); }
            ex |= sex[w];
        }
        for (int a = 0; a < 3; a++) {
            atomicMin(&out[cs].mnKey[a], OrderedIntDev(a0[a]));
            atomicMax(&out[cs].mxKey[a], OrderedIntDev(a1[a]));
        }
        if (ex) atomicOr(&out[cs].exceeded, 1u);
    }
}

// composite sort key (rank << shift) | min(cellId, emptyKey); padding lanes take the scene's
// empty key, so they stay behind the scene's particles (the sort is stable)
__global__ void KBatchKeys(const float4* __restrict__ pos, uint32_t n, const uint8_t* __restrict__ chunkLen,
                           const uint32_t* __restrict__ chunkScene, const BatchSceneDev* __restrict__ sc,
                           uint32_t shift, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx,
                           uint32_t* __restrict__ hist, uint32_t passes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t key = 0;
    if (i < n) {
        const uint32_t chunk = i >> 5, lane = i & 31;
        const uint32_t s = chunkScene[chunk];
        const BatchSceneDev& d = sc[s];
        uint64_t k = d.emptyKey;
        if (lane < (uint32_t)chunkLen[chunk]) {
            const float4 p = pos[i];
            const uint64_t c = CellIdOf(p.x, p.y, p.z, d.fr);
            k = c < d.emptyKey ? c : d.emptyKey;
        }
        key = ((uint64_t)s << shift) | k;
        keys[i] = key;
        idx[i] = i;
    }
    // every pass's digit histogram for the one-pass sort
    __shared__ uint32_t sh[OS_MAX_PASSES * 256];
    for (uint32_t b = threadIdx.x; b < passes * 256u; b += blockDim.x) sh[b] = 0;
    __syncthreads();
    OnesweepCountKey(key, i < n, passes, sh);
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < passes * 256u; b += blockDim.x)
        if (sh[b]) atomicAdd(hist + b, sh[b]);
}

__global__ void KBatchKeysToCellIds(const uint64_t* __restrict__ keys, uint32_t n, const BatchSceneDev* __restrict__ sc,
                                    uint32_t shift, uint64_t* __restrict__ cid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t k = keys[i];
    const uint64_t low = k & ((1ull << shift) - 1ull);
    cid[i] = (low == sc[k >> shift].emptyKey) ? EMPTY_64 : low;
}

// composite-key cell table -> each scene's dense fluid grid (global cell index)
__global__ void KBatchGridScatterF(const uint64_t* __restrict__ unique, const uint64_t* __restrict__ nCellsDev,
                                   const BatchSceneDev* __restrict__ sc, const SceneGeom* __restrict__ geom,
                                   uint32_t shift, uint32_t* __restrict__ grid, uint32_t nMax) {
    const uint64_t nCells = *nCellsDev;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nCells && c < nMax; c += gridDim.x * blockDim.x) {
        const uint64_t k = unique[c];
        const uint32_t s = (uint32_t)(k >> shift);
        const uint64_t low = k & ((1ull << shift) - 1ull);
        if (low == sc[s].emptyKey) continue;
        const Frame& fr = sc[s].fr;
        const uint32_t x = Compact21(low), y = Compact21(low >> 1), z = Compact21(low >> 2);
        grid[geom[s].gridOffF + (uint64_t)x + (uint64_t)fr.nx * ((uint64_t)y + (uint64_t)fr.ny * z)] = c;
    }
}

// one scene's boundary cell table (local starts) -> global starts and its grid (global cells)
__global__ void KBatchOffsetStarts(uint32_t* start, const uint64_t* nCellsDev, uint32_t nMax, uint32_t add) {
    const uint64_t nc = *nCellsDev;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c <= nc && c <= nMax; c += gridDim.x * blockDim.x)
        start[c] += add;
}
__global__ void KBatchGridScatterB(const uint64_t* __restrict__ unique, const uint64_t* __restrict__ nCellsDev, Frame fr,
                                   uint32_t cellBase, uint32_t* __restrict__ grid, uint32_t nMax) {
    const uint64_t nCells = *nCellsDev;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nCells && c < nMax; c += gridDim.x * blockDim.x) {
        const uint64_t id = unique[c];
        if (id == EMPTY_64) continue;
        const uint32_t x = Compact21(id), y = Compact21(id >> 1), z = Compact21(id >> 2);
        grid[(uint64_t)x + (uint64_t)fr.nx * ((uint64_t)y + (uint64_t)fr.ny * z)] = cellBase + c;
    }
}

// relayout: copy whole chunks of the fluid arena (src chunk per destination chunk)
template <typename T>
__global__ void KBatchMoveChunks(const T* __restrict__ src, T* __restrict__ dst, const uint32_t* __restrict__ srcChunk,
                                 uint32_t nDstChunks) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t c = i >> 5;
    if (c >= nDstChunks) return;
    const uint32_t sc = srcChunk[c];
    if (sc == EMPTY_32) return;
    dst[i] = src[(uint64_t)sc * SELL_W + (i & 31)];
}

__global__ void KBatchSolverReset(BatchSolverDev* st, uint32_t* active, const BatchSceneDev* __restrict__ sc,
                                  uint32_t S) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    st[s].iters = sc[s].nF > 0 ? 1u : 0u;
    st[s].avg[0] = st[s].avg[1] = st[s].avg[2] = 0.0f;
    st[s].sums[0] = st[s].sums[1] = st[s].sums[2] = 0.0;
    st[s].done = 0;
    active[s] = sc[s].nF > 0 ? 1u : 0u;
}

// one warp per active scene: fixed-order FP64 sum of its chunks' residual partials, then the
// loop bookkeeping of Step_IISPH (sph_solver.cpp:213-261) for that scene
__global__ void __launch_bounds__(128) KBatchSceneReduce(const double* __restrict__ partials,
                                                         const BatchSceneDev* __restrict__ sc, BatchSolverDev* st,
                                                         uint32_t* active, uint32_t* nActive, SolverControl ctl,
                                                         uint32_t S) {
    const uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (s >= S || active[s] == 0u) return;  // whole warp
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (uint32_t c = sc[s].chunkBegin + lane; c < sc[s].chunkEnd; c += 32) {
        s0 += partials[3ull * c + 0];
        s1 += partials[3ull * c + 1];
        s2 += partials[3ull * c + 2];
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, d);
        s1 += __shfl_xor_sync(0xffffffffu, s1, d);
        s2 += __shfl_xor_sync(0xffffffffu, s2, d);
    }
    if (lane != 0) return;
    BatchSolverDev& q = st[s];
    q.sums[0] = s0; q.sums[1] = s1; q.sums[2] = s2;
    const uint32_t iters = q.iters + 1;
    q.iters = iters;
    q.itersTotal += 1;
    SolverControl c = ctl;
    c.nF = sc[s].nF;
    float avg[3] = {q.avg[0], q.avg[1], q.avg[2]};
    const bool compute = iters >= c.minIters && (c.cond != 0 || Terminated(c, iters, avg));
    if (compute) {
        avg[0] = (float)s0 / (float)c.nF;
        avg[1] = (float)s1 / (float)c.nF;
        avg[2] = (float)s2 / (float)c.nF;
        q.avg[0] = avg[0]; q.avg[1] = avg[1]; q.avg[2] = avg[2];
    }
    const bool done = Terminated(c, iters, avg) || iters >= MAX_JACOBI_SWEEPS;
    q.done = done ? 1u : 0u;
    if (done) active[s] = 0u;
    else atomicAdd(nActive, 1u);
}

__global__ void KBatchLoopCond(uint32_t* nActive, cudaGraphConditionalHandle cond) {
    const uint32_t n = *nActive;
    *nActive = 0u;
    cudaGraphSetConditional(cond, n > 0u ? 1u : 0u);
}

// ------------------------------------------------------------------------------ host side
// first-fit allocator over [0, cap) in element units
class RangeAlloc {
public:
    uint64_t cap = 0;
    std::map<uint64_t, uint64_t> freeList;  // start -> length
    void reset(uint64_t c) { cap = c; freeList.clear(); if (c) freeList[0] = c; }
    void extend(uint64_t c) {  // [cap, c) becomes free (merged with a free tail)
        if (c <= cap) return;
        const uint64_t old = cap;
        cap = c;
        release(old, c - old);
    }
    bool alloc(uint64_t n, uint64_t& at) {
        if (n == 0) { at = 0; return true; }
        for (auto it = freeList.begin(); it != freeList.end(); ++it)
            if (it->second >= n) {
                at = it->first;
                const uint64_t rest = it->second - n;
                freeList.erase(it);
                if (rest) freeList[at + n] = rest;
                return true;
            }
        return false;
    }
    void release(uint64_t at, uint64_t n) {
        if (n == 0) return;
        auto it = freeList.emplace(at, n).first;
        auto nx = std::next(it);
        if (nx != freeList.end() && it->first + it->second == nx->first) { it->second += nx->second; freeList.erase(nx); }
        if (it != freeList.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) { pv->second += it->second; freeList.erase(it); }
        }
    }
};

// device bytes one admitted scene is charged (fluid arena + sort/query/list scratch per fluid
// particle, boundary arena + cell table per boundary particle, dense grids of its frame)
uint64_t BatchSceneBytes(uint64_t nFpad, uint64_t nB, uint64_t gridCells) {
    const uint64_t perF = 120 /* arena + reorder buffers */ + 48 /* keys, cell IDs, tables */ +
                          3 * 2 /* counts */ + 4 * 64 /* FF + FB + FR slices, grown by 1.5x (est.) */ +
                          4 * (64 + 48) /* query row scratch */ + 24 /* Jacobi partials, meta */;
    const uint64_t perB = 16 + 4 + 8 + 8 + 4 + 16 /* arena, table, sort scratch */;
    return nFpad * perF + nB * perB + gridCells * 8;
}

// list buffers of a batch grow faster than the one-scene backend's: admissions add whole
// scenes' lists at once while the batch fills up
constexpr double BATCH_LIST_GROWTH = 1.5;

class Batch {
public:
    struct Scene {
        bool live = false, admitted = false, retiring = false;
        uint32_t rank = 0;
        uint32_t nF = 0, nFpad = 0, nB = 0;
        uint64_t bStart = 0, cellOff = 0, gridOffB = 0, gridVolB = 0;
        uint64_t fStart = 0;
        Frame fr{};
        bool frameValid = false, bSorted = false;
        DomainBox dom{};
        float bMin[3] = {0, 0, 0}, bMax[3] = {0, 0, 0};
        uint64_t steps = 0;
        double time = 0.0;
        uint64_t bytes = 0;
        uint64_t frameRebuilds = 0;
        // admission payload, uploaded at the next relayout
        std::vector<float4> upPos, upVel;
        std::vector<uint64_t> upId;
        BatchSolverDev solver{};
    };

    int device = 0;
    cudaStream_t s = nullptr, capStream = nullptr;
    tsp_params prm{};
    uint64_t budget = 0, used = 0;
    std::vector<Scene> slots;       // by slot id
    std::vector<uint32_t> order;    // rank -> slot
    bool layoutDirty = false;
    std::string lastErr;
    uint64_t launches = 0;
    float lastSubstepMs = 0.f;

    // fluid arena (SELL32-chunk aligned scenes). Arrays are sized to a chunk capacity that only
    // grows, and scene-rank tables to a rank capacity plus one never-active rank that owns the
    // chunks past the live ones; the Jacobi-loop graph is captured over the capacities and reads
    // the live particle count from the device (dLiveN), so a relayout (admission / retirement)
    // neither allocates nor invalidates the captured graph.
    uint32_t nFtot = 0, nChunks = 0;
    uint32_t chunkCap = 0, sceneCap = 0;
    uint32_t hLiveN = 0;
    DBuf<uint32_t> dLiveN;
    DBuf<float4> posP, velRho, velPred, acc, posP2, velRho2, velPred2, acc2;
    DBuf<float2> srcDiag, srcDiag2;
    DBuf<uint64_t> idF, idF2;
    DBuf<uint8_t> chunkLen;
    DBuf<uint32_t> chunkScene, srcChunk;
    // boundary arena
    RangeAlloc allocB, allocCell, allocGridB;
    DBuf<float4> posB, posBtmp;
    DBuf<float> volB, volBtmp;
    DBuf<uint64_t> idB, idBtmp;
    DBuf<uint64_t> uniqB, cidBtmp;
    DBuf<uint32_t> startB, permBtmp;
    VBuf<uint32_t> gridB;  // grows in place: scenes keep their grid ranges when it grows
    DBuf<uint64_t> nCellsB;  // per slot
    // per-scene tables (by rank)
    std::vector<BatchSceneDev> hSc;
    std::vector<SceneGeom> hGeom;
    DBuf<BatchSceneDev> dSc;
    DBuf<SceneGeom> dGeom;
    DBuf<BatchSolverDev> dSolver;
    DBuf<uint32_t> dActive, dNActive;
    DBuf<ProbeResult> dProbe;
    BatchSolverDev* hSolver = nullptr;   // pinned read-back
    ProbeResult* hProbe = nullptr;       // pinned read-back
    size_t hCap = 0;
    // neighbor build
    DBuf<uint64_t> keysA, keysB, cidF, uniqF, nCellsDev;
    DBuf<uint32_t> valsA, valsB, tileHist, digitTotals, startF, err;
    VBuf<uint32_t> gridF;  // grows in place (no free / allocation in the middle of a stream)
    DBuf<uint32_t> osAux, cellAux;  // one-pass sort and single-pass cell table (look-back words)
    DBuf<uint64_t> scanScratch;
    DBuf<U64x2> scanScratch2, sellTot;
    DBuf<unsigned long long> nbrTot;
    struct Sell {
        DBuf<uint16_t> counts, pitch;
        DBuf<uint8_t> format;
        DBuf<uint32_t> base, base2;
        DBuf<uint64_t> offset;
        VBuf<uint16_t> l16;  // grow in place: list growth keeps the addresses
        VBuf<uint32_t> l32;
        uint64_t n16 = 0, n32 = 0;
    } sell[3];
    DBuf<uint32_t> scrF, scrB, scrR;
    DBuf<uint8_t> scrOver;
    DBuf<double> partials;
    uint64_t gridCellsF = 0;
    static constexpr uint32_t KS_F = 64, KS_B = 48;
    // solver loop graph
    struct LoopGraph {
        std::vector<uint64_t> key;
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ex = nullptr;
    };
    std::vector<LoopGraph> graphs;
    size_t graphNext = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t reach = 1;
    float cellSize = 0.f;

    Batch(const tsp_params& p, int dev, uint64_t budgetBytes) : device(dev), prm(p), budget(budgetBytes) {
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&capStream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&ev0));
        CK(cudaEventCreate(&ev1));
        err.ensure(1);
        CK(cudaMemset(err.p, 0, 4));
        nCellsDev.ensure(1);
        sellTot.ensure(3);
        nbrTot.ensure(3);
        dNActive.ensure(1);
        CK(cudaMemset(dNActive.p, 0, 4));
        dLiveN.ensure(1);
        CK(cudaMemset(dLiveN.p, 0, 4));
        // address reserves of the dense grids: admission charges 8 bytes per frame cell, so the
        // budget bounds their total; twice that leaves room for the boundary arena's fragmentation
        const uint64_t gridCells = std::max<uint64_t>(budget / 8, uint64_t(1) << 20);
        gridB.reserveAddress(2 * gridCells);
        gridF.reserveAddress(2 * gridCells);
        SetCellSize();
    }
    ~Batch() {
        cudaSetDevice(device);
        cudaStreamSynchronize(s);
        for (auto& g : graphs) {
            if (g.ex) cudaGraphExecDestroy(g.ex);
            if (g.g) cudaGraphDestroy(g.g);
        }
        if (hSolver) cudaFreeHost(hSolver);
        if (hProbe) cudaFreeHost(hProbe);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (s) cudaStreamDestroy(s);
        if (capStream) cudaStreamDestroy(capStream);
    }
    void Sync() { CK(cudaStreamSynchronize(s)); }

    void SetCellSize() {  // neighbor_search.cpp:1645-1659 (one cell size for the batch)
        const float cs = prm.kernelRadius * prm.gridCellSizeRatio;
        const bool zero = std::fabs(cs) <= 1e-7f;
        const float span = zero ? 0.0f : (prm.kernelRadius / cs);
        reach = zero ? 1u : std::max<uint32_t>(1u, (uint32_t)std::ceil(std::max(0.0f, span - 1e-6f)));
        if (QuerySmemBytes(reach) > 227u * 1024u)
            throw Error(TSP_ERR_UNSUPPORTED, "cell size ratio too small: query stencil exceeds shared memory");
        cellSize = cs;
    }
    Frame EmptyFrame() const {
        Frame f{};
        f.cellSizeInv = cellSize != 0.0f ? 1.0f / cellSize : 0.0f;
        f.reach = reach;
        return f;
    }

    // ------------------------------------------------------------------------ admission
    uint32_t Admit(const tsp_state_view& v, const float* dmin, const float* dmax) {
        if (v.N_R || v.N_RB) throw Error(TSP_ERR_UNSUPPORTED, "served batch scenes have no rigid bodies");
        if (v.N_F == 0) throw Error(TSP_ERR_INVALID, "a served scene needs fluid particles");
        if (!v.xPosF || !v.yPosF || !v.zPosF) throw Error(TSP_ERR_INVALID, "fluid positions missing");
        if (v.N_B && (!v.xPosB || !v.yPosB || !v.zPosB)) throw Error(TSP_ERR_INVALID, "boundary positions missing");
        Scene sc;
        sc.nF = v.N_F;
        sc.nFpad = (v.N_F + SELL_W - 1) / SELL_W * SELL_W;
        sc.nB = v.N_B;
        for (int a = 0; a < 3; a++) { sc.dom.mn[a] = dmin ? dmin[a] : 0.f; sc.dom.mx[a] = dmax ? dmax[a] : 0.f; }
        sc.dom.bounded = dmin && dmax && !(sc.dom.mx[0] <= sc.dom.mn[0] || sc.dom.mx[1] <= sc.dom.mn[1] ||
                                           sc.dom.mx[2] <= sc.dom.mn[2]);
        // budget: the scene's frame is at most its domain (+ margins) when bounded, else its bounds
        uint64_t cells = 0;
        {
            float lo[3], hi[3];
            for (int a = 0; a < 3; a++) { lo[a] = 3.4e38f; hi[a] = -3.4e38f; }
            auto acc = [&](const float* x, const float* y, const float* z, uint32_t n) {
                for (uint32_t i = 0; i < n; i++) {
                    lo[0] = std::min(lo[0], x[i]); hi[0] = std::max(hi[0], x[i]);
                    lo[1] = std::min(lo[1], y[i]); hi[1] = std::max(hi[1], y[i]);
                    lo[2] = std::min(lo[2], z[i]); hi[2] = std::max(hi[2], z[i]);
                }
            };
            acc(v.xPosF, v.yPosF, v.zPosF, v.N_F);
            if (v.N_B) acc(v.xPosB, v.yPosB, v.zPosB, v.N_B);
            cells = 1;
            for (int a = 0; a < 3; a++) {
                float l = lo[a], h = hi[a];
                if (sc.dom.bounded) { l = std::max(l, sc.dom.mn[a]); h = std::min(h, sc.dom.mx[a]); }
                if (sc.dom.bounded) { l = std::min(l, sc.dom.mn[a]); h = std::max(h, sc.dom.mx[a]); }
                const double ext = cellSize > 0 ? (double)(h - l) / cellSize : 0.0;
                cells *= (uint64_t)std::max(1.0, std::ceil(ext)) + 2ull * (reach + 8) + 1ull;
            }
        }
        sc.bytes = BatchSceneBytes(sc.nFpad, sc.nB, cells);
        if (used + sc.bytes > budget) throw Error(TSP_ERR_OVERFLOW, "scene does not fit the batch's memory budget");
        // stage fluid payload (padding lanes zero; they are never valid)
        sc.upPos.assign(sc.nFpad, make_float4(0.f, 0.f, 0.f, 0.f));
        sc.upVel.assign(sc.nFpad, make_float4(0.f, 0.f, 0.f, prm.restDensity));
        sc.upId.assign(sc.nFpad, ~0ull);
        for (uint32_t i = 0; i < v.N_F; i++) {
            sc.upPos[i] = make_float4(v.xPosF[i], v.yPosF[i], v.zPosF[i], v.pressureF ? v.pressureF[i] : 0.f);
            sc.upVel[i] = make_float4(v.xVelF ? v.xVelF[i] : 0.f, v.yVelF ? v.yVelF[i] : 0.f,
                                      v.zVelF ? v.zVelF[i] : 0.f, v.densityF ? v.densityF[i] : prm.restDensity);
            sc.upId[i] = v.idF ? v.idF[i] : (uint64_t)i;
        }
        // boundary: arena range now (boundary data never moves)
        if (!allocB.alloc(sc.nB, sc.bStart)) {
            GrowBoundary(sc.nB);
            if (!allocB.alloc(sc.nB, sc.bStart)) throw Error(TSP_ERR_OVERFLOW, "boundary arena allocation failed");
        }
        if (!allocCell.alloc(sc.nB + 1ull, sc.cellOff)) {
            GrowBoundary(sc.nB);
            if (!allocCell.alloc(sc.nB + 1ull, sc.cellOff)) {
                allocB.release(sc.bStart, sc.nB);
                throw Error(TSP_ERR_OVERFLOW, "boundary cell-table allocation failed");
            }
        }
        if (sc.nB) {
            std::vector<float4> pb(sc.nB);
            std::vector<float> vb(sc.nB);
            std::vector<uint64_t> ib(sc.nB);
            const float defPsi = prm.massB, defVol = prm.restDensity > 0.f ? prm.massB / prm.restDensity : 0.f;
            for (uint32_t i = 0; i < sc.nB; i++) {
                pb[i] = make_float4(v.xPosB[i], v.yPosB[i], v.zPosB[i], v.psiB ? v.psiB[i] : defPsi);
                vb[i] = v.volB ? v.volB[i] : defVol;
                ib[i] = v.idB ? v.idB[i] : (uint64_t)i;
                for (int a = 0; a < 3; a++) {
                    const float x = a == 0 ? pb[i].x : a == 1 ? pb[i].y : pb[i].z;
                    if (i == 0) { sc.bMin[a] = x; sc.bMax[a] = x; }
                    sc.bMin[a] = std::min(sc.bMin[a], x);
                    sc.bMax[a] = std::max(sc.bMax[a], x);
                }
            }
            CK(cudaMemcpyAsync(posB.p + sc.bStart, pb.data(), sc.nB * sizeof(float4), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(volB.p + sc.bStart, vb.data(), sc.nB * sizeof(float), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(idB.p + sc.bStart, ib.data(), sc.nB * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
            Sync();
        }
        sc.live = true;
        sc.admitted = false;
        sc.fr = EmptyFrame();
        used += sc.bytes;
        uint32_t slot = (uint32_t)slots.size();
        for (uint32_t k = 0; k < slots.size(); k++)
            if (!slots[k].live) { slot = k; break; }
        if (slot == slots.size()) slots.emplace_back();
        slots[slot] = std::move(sc);
        layoutDirty = true;
        return slot;
    }

    void GrowBoundary(uint64_t need) {
        // boundary data of admitted scenes is copied into larger arenas (offsets are kept)
        const uint64_t capB = std::max<uint64_t>(allocB.cap * 2, allocB.cap + need + 1024);
        const uint64_t capC = std::max<uint64_t>(allocCell.cap * 2, allocCell.cap + need + 1024 + 64);
        auto regrow = [&](auto& buf, uint64_t oldN, uint64_t newN) {
            using T = std::remove_reference_t<decltype(*buf.p)>;
            T* np = nullptr;
            CK(cudaMalloc(&np, newN * sizeof(T)));
            if (buf.p && oldN) CK(cudaMemcpyAsync(np, buf.p, oldN * sizeof(T), cudaMemcpyDeviceToDevice, s));
            Sync();
            buf.release();
            buf.p = np;
            buf.cap = newN;
        };
        regrow(posB, allocB.cap, capB);
        regrow(volB, allocB.cap, capB);
        regrow(idB, allocB.cap, capB);
        regrow(uniqB, allocCell.cap, capC);
        regrow(startB, allocCell.cap, capC);
        const uint64_t oldB = allocB.cap, oldC = allocCell.cap;
        allocB.cap = capB;
        allocB.release(oldB, capB - oldB);
        allocCell.cap = capC;
        allocCell.release(oldC, capC - oldC);
        posBtmp.ensure(capB); volBtmp.ensure(capB); idBtmp.ensure(capB); cidBtmp.ensure(capB);
        permBtmp.ensure(capB);
    }

    void Retire(uint32_t slot) {
        Scene& sc = At(slot);
        sc.retiring = true;
        layoutDirty = true;
    }
    Scene& At(uint32_t slot) {
        if (slot >= slots.size() || !slots[slot].live) throw Error(TSP_ERR_INVALID, "no such scene slot");
        return slots[slot];
    }

    // ------------------------------------------------------------------------ relayout
    void Relayout() {
        // retire: free boundary ranges and budget
        for (auto& sc : slots)
            if (sc.live && sc.retiring) {
                allocB.release(sc.bStart, sc.nB);
                allocCell.release(sc.cellOff, sc.nB + 1ull);
                allocGridB.release(sc.gridOffB, sc.gridVolB);
                used -= std::min(used, sc.bytes);
                sc = Scene();
            }
        // new rank order: surviving scenes in arena order, then new ones
        std::vector<uint32_t> newOrder;
        for (uint32_t slot : order)
            if (slots[slot].live && slots[slot].admitted) newOrder.push_back(slot);
        for (uint32_t k = 0; k < slots.size(); k++)
            if (slots[k].live && !slots[k].admitted) newOrder.push_back(k);
        uint64_t tot = 0;
        for (uint32_t slot : newOrder) tot += slots[slot].nFpad;
        if (tot > 0x7fffffe0ull) throw Error(TSP_ERR_OVERFLOW, "batch fluid arena exceeds 2^31 particles");
        const uint32_t nNew = (uint32_t)tot, chunksNew = nNew / SELL_W;
        if (chunksNew > chunkCap) {
            // the chunks the memory budget can hold, reserved at the first admission: a growth
            // frees and reallocates the arena and its multi-GB row scratch and re-captures the
            // loop graph, which took up to 0.7 s in the middle of a stream; the loop kernels
            // iterate over the live chunks only, so the reserve costs no launch time
            const uint64_t budgetChunks = budget / (BatchSceneBytes(SELL_W, 0, 0) * 1ull);
            const uint64_t want = std::max<uint64_t>(budgetChunks, chunksNew);
            chunkCap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(want, 64ull), 0x7fffffe0ull / SELL_W);
        }
        if (newOrder.size() > sceneCap) sceneCap = std::max<uint32_t>((uint32_t)newOrder.size(), std::max(2u * sceneCap, 16u));
        const uint32_t padRank = sceneCap;  // owner of the padding chunks, never active
        // chunk map: surviving scenes move whole chunks
        std::vector<uint32_t> srcMap(chunkCap, EMPTY_32);
        std::vector<uint8_t> len(chunkCap, 0);
        std::vector<uint32_t> scn(chunkCap, padRank);
        uint64_t at = 0;
        for (uint32_t r = 0; r < newOrder.size(); r++) {
            Scene& sc = slots[newOrder[r]];
            const uint32_t c0 = (uint32_t)(at / SELL_W), nc = sc.nFpad / SELL_W;
            for (uint32_t c = 0; c < nc; c++) {
                if (sc.admitted) srcMap[c0 + c] = (uint32_t)(sc.fStart / SELL_W) + c;
                const uint32_t valid = (uint32_t)std::min<uint64_t>(SELL_W, sc.nF > c * SELL_W ? sc.nF - c * SELL_W : 0);
                len[c0 + c] = (uint8_t)valid;
                scn[c0 + c] = r;
            }
            sc.fStart = at;
            sc.rank = r;
            at += sc.nFpad;
        }
        // move surviving chunks into the alternate arrays, then place the new scenes
        const size_t cap = (size_t)chunkCap * SELL_W;
        posP2.ensure(cap); velRho2.ensure(cap); velPred2.ensure(cap); acc2.ensure(cap); srcDiag2.ensure(cap);
        idF2.ensure(cap);
        if (nNew) {
            CK(cudaMemsetAsync(velPred2.p, 0, nNew * sizeof(float4), s));
            CK(cudaMemsetAsync(acc2.p, 0, nNew * sizeof(float4), s));
            CK(cudaMemsetAsync(srcDiag2.p, 0, nNew * sizeof(float2), s));
        }
        srcChunk.ensure(srcMap.size());
        CK(cudaMemcpyAsync(srcChunk.p, srcMap.data(), srcMap.size() * 4, cudaMemcpyHostToDevice, s));
        if (nFtot && chunksNew) {
            const unsigned g = (unsigned)((chunksNew * 32ull + 255) / 256);
            KBatchMoveChunks<float4><<<g, 256, 0, s>>>(posP.p, posP2.p, srcChunk.p, chunksNew);
            KBatchMoveChunks<float4><<<g, 256, 0, s>>>(velRho.p, velRho2.p, srcChunk.p, chunksNew);
            KBatchMoveChunks<float4><<<g, 256, 0, s>>>(velPred.p, velPred2.p, srcChunk.p, chunksNew);
            KBatchMoveChunks<float4><<<g, 256, 0, s>>>(acc.p, acc2.p, srcChunk.p, chunksNew);
            KBatchMoveChunks<float2><<<g, 256, 0, s>>>(srcDiag.p, srcDiag2.p, srcChunk.p, chunksNew);
            KBatchMoveChunks<uint64_t><<<g, 256, 0, s>>>(idF.p, idF2.p, srcChunk.p, chunksNew);
            launches += 6;
        }
        for (uint32_t slot : newOrder) {
            Scene& sc = slots[slot];
            if (sc.admitted) continue;
            CK(cudaMemcpyAsync(posP2.p + sc.fStart, sc.upPos.data(), sc.nFpad * sizeof(float4), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(velRho2.p + sc.fStart, sc.upVel.data(), sc.nFpad * sizeof(float4), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(idF2.p + sc.fStart, sc.upId.data(), sc.nFpad * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        }
        Sync();
        for (uint32_t slot : newOrder) {
            Scene& sc = slots[slot];
            if (sc.admitted) continue;
            sc.admitted = true;
            std::vector<float4>().swap(sc.upPos);
            std::vector<float4>().swap(sc.upVel);
            std::vector<uint64_t>().swap(sc.upId);
        }
        Swap(posP, posP2); Swap(velRho, velRho2); Swap(velPred, velPred2); Swap(acc, acc2); Swap(srcDiag, srcDiag2);
        Swap(idF, idF2);
        posP2.ensure(cap); velRho2.ensure(cap); idF2.ensure(cap);
        chunkLen.ensure(len.size());
        chunkScene.ensure(scn.size());
        CK(cudaMemcpyAsync(chunkLen.p, len.data(), len.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(chunkScene.p, scn.data(), scn.size() * 4, cudaMemcpyHostToDevice, s));
        order = newOrder;
        nFtot = nNew;
        nChunks = chunksNew;
        const size_t S = (size_t)sceneCap + 1;  // + the padding rank
        dSc.ensure(S); dGeom.ensure(S); dSolver.ensure(S); dActive.ensure(S); dProbe.ensure(S);
        CK(cudaMemsetAsync(dSc.p, 0, S * sizeof(BatchSceneDev), s));  // ranks >= order.size(): no fluid
        if (hCap < S) {
            if (hSolver) cudaFreeHost(hSolver);
            if (hProbe) cudaFreeHost(hProbe);
            hCap = std::max<size_t>(S, 2 * hCap);
            CK(cudaMallocHost(&hSolver, hCap * sizeof(BatchSolverDev)));
            CK(cudaMallocHost(&hProbe, hCap * sizeof(ProbeResult)));
        }
        EnsureScratch();
        hLiveN = nNew;
        CK(cudaMemcpyAsync(dLiveN.p, &hLiveN, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        Sync();
        layoutDirty = false;
    }

    // scratch sized to the arena capacity (and the largest boundary of a live scene, grown by
    // 1.25x), so a relayout allocates only when a capacity grows
    void EnsureScratch() {
        const uint32_t n = std::max<uint32_t>(chunkCap * SELL_W, 32), nc = std::max<uint32_t>(chunkCap, 1);
        uint32_t nSort = n;  // sort / scan scratch also serves the boundary sort of one scene
        for (const auto& sc : slots)
            if (sc.live) nSort = std::max(nSort, sc.nB);
        if (nSort > keysA.cap) nSort = (uint32_t)std::min<uint64_t>(nSort + nSort / 4ull, 0xffffffffull);
        keysA.ensure(nSort); keysB.ensure(nSort); valsA.ensure(nSort); valsB.ensure(nSort); cidF.ensure(n);
        uniqF.ensure(n); startF.ensure(n + 1ull);
        tileHist.ensure(RadixTileHistItems(nSort));
        digitTotals.ensure(256);
        osAux.ensure(OnesweepAuxWords(std::max<uint32_t>(nSort, 2), OS_MAX_PASSES));
        cellAux.ensure(CellTableGridAuxWords(std::max<uint32_t>(nSort, 1)));
        scanScratch.ensure(ScanScratchItems(nSort + 1ull));
        scanScratch2.ensure(ScanScratchItems(n + 1ull));
        for (auto& m : sell) {
            m.counts.ensure(n); m.pitch.ensure(nc); m.format.ensure(nc); m.base.ensure(nc); m.base2.ensure(nc);
            m.offset.ensure(nc);
            m.l16.ensure(std::max<size_t>(m.l16.cap, 16)); m.l32.ensure(std::max<size_t>(m.l32.cap, 16));
        }
        scrF.ensure(QueryScratchWords(nc, KS_F));
        scrB.ensure(QueryScratchWords(nc, KS_B));
        scrR.ensure(32);  // no rigid species: never read, one warp of lane offsets
        scrOver.ensure(nc);
        partials.ensure(3ull * nc);
        velPred.ensure(n); acc.ensure(n); srcDiag.ensure(n);
        velPred2.ensure(n); acc2.ensure(n); srcDiag2.ensure(n);
    }

    // ------------------------------------------------------------------------ frames
    // UpdateCellFrame (neighbor_search.cpp:1902-2006) of one scene from its probe
    bool UpdateFrame(Scene& sc, const ProbeResult& pr) {
        float mn[3], mx[3];
        for (int a = 0; a < 3; a++) { mn[a] = OrderedIntToFloat(pr.mnKey[a]); mx[a] = OrderedIntToFloat(pr.mxKey[a]); }
        bool rebuild = !sc.frameValid;
        if (!rebuild) {
            const int m = (int)reach;
            const Frame& f = sc.fr;
            const bool innerEmpty = f.ox + m > f.ox + (int)f.nx - 1 - m || f.oy + m > f.oy + (int)f.ny - 1 - m ||
                                    f.oz + m > f.oz + (int)f.nz - 1 - m;
            rebuild = innerEmpty || pr.exceeded != 0;
        }
        if (!rebuild) return false;
        if (sc.nB)
            for (int a = 0; a < 3; a++) { mn[a] = std::min(mn[a], sc.bMin[a]); mx[a] = std::max(mx[a], sc.bMax[a]); }
        if (sc.dom.bounded)
            for (int a = 0; a < 3; a++) {
                mn[a] = std::clamp(mn[a], sc.dom.mn[a], sc.dom.mx[a]);
                mx[a] = std::clamp(mx[a], sc.dom.mn[a], sc.dom.mx[a]);
            }
        Frame f = EmptyFrame();
        const int64_t margin = (int64_t)reach + 8;
        int64_t o[3], e[3];
        for (int a = 0; a < 3; a++) {
            o[a] = (int64_t)HostFloorToInt(mn[a] * f.cellSizeInv) - margin;
            e[a] = (int64_t)HostFloorToInt(mx[a] * f.cellSizeInv) + margin;
        }
        if (!TryBuildCellFrame(o, e, f.ox, f.oy, f.oz, f.nx, f.ny, f.nz))
            throw Error(TSP_ERR_FRAME, "Compact CLL cell frame exceeds the supported range.");
        f.keyBits = HostKeyBits(f.nx, f.ny, f.nz);
        if ((uint64_t)f.nx * f.ny * f.nz > (1ull << 28))
            throw Error(TSP_ERR_UNSUPPORTED, "cell frame volume exceeds the dense grid limit (2^28 cells)");
        sc.fr = f;
        sc.frameValid = true;
        sc.bSorted = false;
        sc.frameRebuilds++;
        return true;
    }

    // boundary grids of all scenes whose frame changed: grid ranges first (a full arena is
    // regrown and every scene's grid rebuilt), then sort + cell table + grid per scene
    void BuildBoundaries() {
        bool regrown = false;
        for (uint32_t slot : order) {
            Scene& sc = slots[slot];
            if (sc.bSorted) continue;
            const uint64_t vol = (uint64_t)sc.fr.nx * sc.fr.ny * sc.fr.nz;
            if (vol == sc.gridVolB) continue;
            allocGridB.release(sc.gridOffB, sc.gridVolB);
            sc.gridVolB = 0;
            sc.gridOffB = 0;
            if (!allocGridB.alloc(vol, sc.gridOffB)) {
                // grow the arena in place when its address reserve allows (other scenes keep
                // their ranges and sorts), else rebuild it below
                const uint64_t capNew = std::max<uint64_t>(allocGridB.cap * 2, allocGridB.cap + vol + 4096);
                if (capNew * sizeof(uint32_t) > gridB.reservedBytes) { regrown = true; break; }
                gridB.ensure(capNew);
                allocGridB.extend(gridB.cap);
                if (!allocGridB.alloc(vol, sc.gridOffB)) { regrown = true; break; }
            }
            sc.gridVolB = vol;
        }
        if (regrown) {
            uint64_t need = 0;
            for (uint32_t slot : order) {
                const Frame& f = slots[slot].fr;
                need += (uint64_t)f.nx * f.ny * f.nz;
            }
            const uint64_t capNew = std::max<uint64_t>(need + need / 4 + 4096, allocGridB.cap * 2);
            Sync();
            gridB.release();
            gridB.ensure(capNew);
            allocGridB.reset(capNew);
            for (uint32_t slot : order) {
                Scene& sc = slots[slot];
                const uint64_t vol = (uint64_t)sc.fr.nx * sc.fr.ny * sc.fr.nz;
                if (!allocGridB.alloc(vol, sc.gridOffB)) throw Error(TSP_ERR_OVERFLOW, "boundary grid arena");
                sc.gridVolB = vol;
                sc.bSorted = false;
            }
        }
        for (uint32_t slot : order)
            if (!slots[slot].bSorted) BuildBoundary(slots[slot], slot);
    }
    // boundary sort + cell table + grid of one scene under its (new) frame
    void BuildBoundary(Scene& sc, uint32_t slot) {
        const uint64_t vol = sc.gridVolB;
        CK(cudaMemsetAsync(gridB.p + sc.gridOffB, 0xff, vol * sizeof(uint32_t), s));
        if (sc.nB == 0) { sc.bSorted = true; return; }
        SortScratch ss{keysA.p, keysB.p, valsA.p, valsB.p, tileHist.p, digitTotals.p};
        const uint32_t n = sc.nB;
        float4* pb = posB.p + sc.bStart;
        SortByCell(pb, n, sc.fr, ss, permBtmp.p, cidBtmp.p, s);
        GatherF4(permBtmp.p, pb, posBtmp.p, n, s);
        GatherF1(permBtmp.p, volB.p + sc.bStart, volBtmp.p, n, s);
        GatherU64(permBtmp.p, idB.p + sc.bStart, idBtmp.p, n, s);
        CK(cudaMemcpyAsync(pb, posBtmp.p, n * sizeof(float4), cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(volB.p + sc.bStart, volBtmp.p, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(idB.p + sc.bStart, idBtmp.p, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        uint64_t* nc = nCellsB.p + slot;
        BuildCellTable(cidBtmp.p, n, uniqB.p + sc.cellOff, startB.p + sc.cellOff, nc, scanScratch.p, s);
        KBatchOffsetStarts<<<(n + 256) / 256, 256, 0, s>>>(startB.p + sc.cellOff, nc, n, (uint32_t)sc.bStart);
        KBatchGridScatterB<<<std::min<uint32_t>((n + 255) / 256, 148u * 16u), 256, 0, s>>>(
            uniqB.p + sc.cellOff, nc, sc.fr, (uint32_t)sc.cellOff, gridB.p + sc.gridOffB, n);
        launches += 12;
        sc.bSorted = true;
    }

    // ------------------------------------------------------------------------ one substep
    SellMeta Meta(int k) {
        Sell& m = sell[k];
        return SellMeta{m.counts.p, m.pitch.p, m.format.p, m.base.p, m.base2.p, m.offset.p, m.l16.p, m.l32.p,
                        (uint64_t)m.l16.cap, (uint64_t)m.l32.cap};
    }
    SellView View(int k) {
        Sell& m = sell[k];
        return SellView{m.counts.p, m.pitch.p, m.format.p, m.base.p, m.base2.p, m.offset.p, m.l16.p, m.l32.p};
    }
    // masked: the Jacobi-loop view (n = the arena capacity, the live count read on the device,
    // converged scenes masked out)
    FluidDev Fluid(bool masked) {
        FluidDev f{posP.p, velRho.p, velPred.p, acc.p, srcDiag.p, masked ? chunkCap * SELL_W : nFtot};
        f.chunkLen = chunkLen.p;
        f.chunkScene = chunkScene.p;
        f.sceneActive = masked ? dActive.p : nullptr;
        f.chunkPartials = masked ? partials.p : nullptr;
        f.liveN = masked ? dLiveN.p : nullptr;
        return f;
    }
    void CheckErrors() {
        uint32_t e = 0;
        CK(cudaMemcpy(&e, err.p, 4, cudaMemcpyDeviceToHost));
        if (!e) return;
        CK(cudaMemset(err.p, 0, 4));
        if (e & ERR_COUNT_U16) throw Error(TSP_ERR_OVERFLOW, "a neighbor count exceeds uint16 storage");
        if (e & ERR_SORT_LOOKBACK)
            throw Error(TSP_ERR_CUDA, "cell sort / cell table: a tile's look-back gave up waiting for its predecessors");
        if (e & ERR_STAGE_WAIT)
            throw Error(TSP_ERR_CUDA, "neighbor query: a block's staging copies did not complete");
        throw Error(TSP_ERR_NEIGHBOR_LIST, "SELL32 neighbor-list fill overflow / delta range error");
    }

    std::vector<uint64_t> LoopKey(const Consts& c, const SolverControl& ctl) {
        std::vector<uint64_t> k;
        auto P = [&](const void* q) { k.push_back((uint64_t)(uintptr_t)q); };
        const FluidDev f = Fluid(true);
        P(f.posP); P(f.velRho); P(f.velPred); P(f.acc); P(f.srcDiag); k.push_back(f.n);
        P(f.chunkLen); P(f.chunkScene); P(f.sceneActive); P(f.chunkPartials); P(f.liveN);
        P(posB.p); P(volB.p);
        for (int s2 = 0; s2 < 3; s2++) {
            const SellView v = View(s2);
            P(v.counts); P(v.pitch); P(v.format); P(v.base); P(v.base2); P(v.offset); P(v.list16); P(v.list32);
        }
        const uint32_t* cw = reinterpret_cast<const uint32_t*>(&c);
        for (size_t i = 0; i < sizeof(Consts) / 4; i++) k.push_back(cw[i]);
        k.push_back(ctl.minIters); k.push_back(ctl.maxIters); k.push_back(ctl.fixedIters); k.push_back(ctl.cond);
        uint32_t tb;
        std::memcpy(&tb, &ctl.target, 4);
        k.push_back(tb);
        P(dSc.p); P(dSolver.p); P(dActive.p); P(dNActive.p); k.push_back(sceneCap);
        k.push_back((uint64_t)(int64_t)TuneChoice(TUNE_PRESSURE_ACC, f.n));  // the launched instantiations
        k.push_back((uint64_t)(int64_t)TuneChoice(TUNE_JACOBI, f.n));
        return k;
    }
    cudaGraphExec_t LoopGraphFor(const Consts& c, const SolverControl& ctl) {
        std::vector<uint64_t> key = LoopKey(c, ctl);
        for (auto& g : graphs)
            if (g.ex && g.key == key) return g.ex;
        cudaGraph_t graph;
        CK(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle handle;
        CK(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(capStream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        const FluidDev f = Fluid(true);
        const BoundaryDev b{posB.p, volB.p, (uint32_t)allocB.cap};
        const RigidDev r{nullptr, nullptr, nullptr, 0};
        const NeighborView nv{View(0), View(1), View(2)};
        LaunchPressureAcc(c, f, b, r, nv, capStream);
        LaunchJacobi(c, f, b, r, nv, ctl, nullptr, nullptr, 0ull, false, capStream);
        const uint32_t S = sceneCap + 1;
        KBatchSceneReduce<<<(S * 32 + 127) / 128, 128, 0, capStream>>>(partials.p, dSc.p, dSolver.p, dActive.p,
                                                                      dNActive.p, ctl, S);
        KBatchLoopCond<<<1, 1, 0, capStream>>>(dNActive.p, handle);
        cudaGraph_t captured;
        CK(cudaStreamEndCapture(capStream, &captured));
        cudaGraphExec_t ex;
        CK(cudaGraphInstantiate(&ex, graph, 0));
        if (graphs.size() < 4) graphs.push_back({});
        LoopGraph& slot = graphs[graphNext % graphs.size()];
        graphNext++;
        if (slot.ex) cudaGraphExecDestroy(slot.ex);
        if (slot.g) cudaGraphDestroy(slot.g);
        slot.key = std::move(key); slot.g = graph; slot.ex = ex;
        return ex;
    }

    // the autotuner on the batch's live state, as the one-scene backend does it (tune.cu): kernels
    // that rewrite the positions' pressure run between a save into the reorder's alternate array
    // and a restore
    void EnsureTuned(TuneKernel k, uint32_t n, const std::function<void(int)>& launch, bool savePos = false) {
        if (n == 0 || !TuneEnabled() || TuneChoice(k, n) >= 0) return;
        if (savePos) CK(cudaMemcpyAsync(posP2.p, posP.p, (size_t)n * sizeof(float4), cudaMemcpyDeviceToDevice, s));
        TuneRun(k, n, launch, s);
        if (savePos) CK(cudaMemcpyAsync(posP.p, posP2.p, (size_t)n * sizeof(float4), cudaMemcpyDeviceToDevice, s));
        CheckErrors();
    }
    void Substep(const tsp_params& p) {
        CK(cudaSetDevice(device));
        if (p.kernelRadius != prm.kernelRadius || p.gridCellSizeRatio != prm.gridCellSizeRatio)
            throw Error(TSP_ERR_INVALID, "the batch's cell size is fixed at creation");
        if (p.solverTerminationCond > 3) throw Error(TSP_ERR_INVALID, "unknown solver termination condition");
        if (p.maxSolverIters > MAX_JACOBI_SWEEPS || p.minSolverIters > MAX_JACOBI_SWEEPS)
            throw Error(TSP_ERR_UNSUPPORTED, "solver iteration bounds above 100000");
        prm = p;
        // the substep's device time includes the relayout of admissions and retirements (chunk
        // moves, uploads of admitted scenes), batching work the one-scene path does not have
        CK(cudaEventRecord(ev0, s));
        if (layoutDirty) Relayout();
        const uint32_t S = (uint32_t)order.size();
        if (S == 0 || nFtot == 0) return;
        // ---- probe + host frame rule per scene
        hSc.resize(S);
        hGeom.resize(S);
        for (uint32_t r = 0; r < S; r++) {
            const Scene& sc = slots[order[r]];
            BatchSceneDev d{};
            d.fr = sc.fr; d.dom = sc.dom; d.frameValid = sc.frameValid ? 1 : 0;
            d.emptyKey = sc.frameValid ? (1ull << (sc.fr.keyBits - 1u)) : 0ull;
            d.chunkBegin = (uint32_t)(sc.fStart / SELL_W);
            d.chunkEnd = (uint32_t)((sc.fStart + sc.nFpad) / SELL_W);
            d.nF = sc.nF;
            hSc[r] = d;
        }
        CK(cudaMemcpyAsync(dSc.p, hSc.data(), S * sizeof(BatchSceneDev), cudaMemcpyHostToDevice, s));
        KBatchProbeReset<<<(S + 127) / 128, 128, 0, s>>>(dProbe.p, S, OrderedIntHost(3.402823466e38f),
                                                        OrderedIntHost(-3.402823466e38f));
        KBatchProbe<<<(unsigned)((nFtot + 255) / 256), 256, 0, s>>>(posP.p, nChunks, chunkLen.p, chunkScene.p, dSc.p,
                                                                    dProbe.p);
        CK(cudaMemcpyAsync(hProbe, dProbe.p, S * sizeof(ProbeResult), cudaMemcpyDeviceToHost, s));
        launches += 2;
        Sync();
        uint32_t keyBitsMax = 1;
        uint64_t gOff = 0;
        for (uint32_t r = 0; r < S; r++) {
            Scene& sc = slots[order[r]];
            UpdateFrame(sc, hProbe[r]);
            keyBitsMax = std::max(keyBitsMax, sc.fr.keyBits);
            BatchSceneDev& d = hSc[r];
            d.fr = sc.fr; d.frameValid = 1;
            d.emptyKey = 1ull << (sc.fr.keyBits - 1u);
            hGeom[r].fr = sc.fr;
            hGeom[r].gridOffF = gOff;
            gOff += (uint64_t)sc.fr.nx * sc.fr.ny * sc.fr.nz;
        }
        if (nCellsB.cap < slots.size()) nCellsB.ensure(std::max<size_t>(slots.size(), 2 * nCellsB.cap));
        BuildBoundaries();
        for (uint32_t r = 0; r < S; r++) hGeom[r].gridOffB = slots[order[r]].gridOffB;
        gridCellsF = gOff;
        gridF.grow(gridCellsF, 2.0);
        uint32_t rankBits = 1;
        while ((1u << rankBits) < S) rankBits++;
        const uint32_t shift = keyBitsMax;
        if (shift + rankBits > 64) throw Error(TSP_ERR_UNSUPPORTED, "batch sort key exceeds 64 bits");
        CK(cudaMemcpyAsync(dSc.p, hSc.data(), S * sizeof(BatchSceneDev), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dGeom.p, hGeom.data(), S * sizeof(SceneGeom), cudaMemcpyHostToDevice, s));
        // ---- fluid: composite keys, one stable sort, reorder, cell table, grids
        const uint32_t n = nFtot;
        const unsigned g = (unsigned)((n + 255) / 256);
        // one-pass sort of the composite keys (histograms counted by the key kernel)
        const uint32_t sortBits = shift + rankBits;
        const uint32_t passes = (sortBits + 7u) / 8u;
        CK(cudaMemsetAsync(osAux.p, 0, OnesweepAuxWords(n, passes) * sizeof(uint32_t), s));
        const OnesweepAux oa = OnesweepLayout(osAux.p, err.p, ERR_SORT_LOOKBACK);
        KBatchKeys<<<g, 256, 0, s>>>(posP.p, n, chunkLen.p, chunkScene.p, dSc.p, shift, keysA.p, valsA.p, oa.hist,
                                     passes);
        const bool alt = n >= 2 ? OnesweepSortPairsPingPong<uint64_t, uint32_t>(keysA.p, valsA.p, keysB.p, valsB.p, n,
                                                                                sortBits, oa, s)
                                : false;
        const uint64_t* sk = alt ? keysB.p : keysA.p;
        const uint32_t* perm = alt ? valsB.p : valsA.p;
        KBatchKeysToCellIds<<<g, 256, 0, s>>>(sk, n, dSc.p, shift, cidF.p);
        LaunchReorderFluidStep(perm, posP.p, velRho.p, idF.p, posP2.p, velRho2.p, idF2.p, n, s);
        Swap(posP, posP2); Swap(velRho, velRho2); Swap(idF, idF2);
        BuildCellTableGrid(sk, n, uniqF.p, startF.p, nCellsDev.p, nullptr, EmptyFrame(), 0, cellAux.p, err.p, s);
        CK(cudaMemsetAsync(gridF.p, 0xff, gridCellsF * sizeof(uint32_t), s));
        KBatchGridScatterF<<<std::min<uint32_t>(g, 148u * 16u), 256, 0, s>>>(uniqF.p, nCellsDev.p, dSc.p, dGeom.p, shift,
                                                                             gridF.p, n);
        launches += 4 + (n >= 2 ? passes : 0u) + 1 + 1;
        // ---- query count, sizes, fill
        QueryArgs qa{};
        qa.posF = posP.p; qa.cidF = cidF.p; qa.nF = n;
        qa.posB = posB.p; qa.nB = (uint32_t)allocB.cap;
        qa.startF = startF.p; qa.startB = startB.p;
        qa.gridF = gridF.p; qa.gridB = gridB.p; qa.gridR = nullptr;
        qa.fr = EmptyFrame(); qa.r2 = prm.kernelRadiusSqu; qa.err = err.p; qa.nbrTotals = nbrTot.p;
        qa.scrF = scrF.p; qa.scrB = scrB.p; qa.scrR = scrR.p; qa.ksF = KS_F; qa.ksB = KS_B; qa.ksR = 0;
        qa.scrOver = scrOver.p;
        qa.chunkLen = chunkLen.p; qa.chunkScene = chunkScene.p; qa.scenes = dGeom.p;
        EnsureTuned(TUNE_QUERY_COUNT, n, [&](int v) {
            QueryArgs t = qa;
            t.nbrTotals = nullptr;
            t.nF = std::min(n, TUNE_MAX_N);
            LaunchQueryFluid(false, t, Meta(0), Meta(1), Meta(2), s, v);
        });
        CK(cudaMemsetAsync(nbrTot.p, 0, 3 * sizeof(unsigned long long), s));
        LaunchQueryFluid(false, qa, Meta(0), Meta(1), Meta(2), s);
        FinalizeSell3(Meta(0), Meta(1), Meta(2), nChunks, scanScratch2.p, sellTot.p, s);
        U64x2 tot[3];
        CK(cudaMemcpyAsync(tot, sellTot.p, sizeof(tot), cudaMemcpyDeviceToHost, s));
        Sync();
        for (int k = 0; k < 3; k++) {
            sell[k].n16 = tot[k].a; sell[k].n32 = tot[k].b;
            sell[k].l16.grow(tot[k].a, BATCH_LIST_GROWTH); sell[k].l32.grow(tot[k].b, BATCH_LIST_GROWTH);
        }
        EnsureTuned(TUNE_QUERY_FILL, n, [&](int v) {
            QueryArgs t = qa;
            t.nF = std::min(n, TUNE_MAX_N);
            LaunchQueryFluid(true, t, Meta(0), Meta(1), Meta(2), s, v);
        });
        LaunchQueryFluid(true, qa, Meta(0), Meta(1), Meta(2), s);
        launches += 2 + FinalizeSell3Launches(nChunks);
        // ---- solver stages; the Jacobi loop skips converged scenes
        const Consts c = MakeConsts(prm);
        const FluidDev f = Fluid(false);
        const BoundaryDev b{posB.p, volB.p, (uint32_t)allocB.cap};
        const RigidDev rd{nullptr, nullptr, nullptr, 0};
        const NeighborView nv{View(0), View(1), View(2)};
        const FluidDev ft = TuneView(f, nFtot);
        EnsureTuned(TUNE_DENSITY, f.n, [&](int v) { LaunchDensity(c, ft, b, rd, nv, s, v); });
        LaunchDensity(c, f, b, rd, nv, s);
        EnsureTuned(TUNE_NON_PRESSURE, f.n, [&](int v) { LaunchNonPressure(c, ft, b, rd, nv, s, v); });
        LaunchNonPressure(c, f, b, rd, nv, s);
        EnsureTuned(TUNE_SOURCE_DIAG, f.n, [&](int v) { LaunchSourceDiagInit(c, ft, b, rd, nv, nullptr, s, v); }, true);
        LaunchSourceDiagInit(c, f, b, rd, nv, nullptr, s);
        KBatchSolverReset<<<(sceneCap + 1 + 127) / 128, 128, 0, s>>>(dSolver.p, dActive.p, dSc.p, sceneCap + 1);
        const SolverControl ctl{prm.minSolverIters, prm.maxSolverIters, prm.fixedIters, prm.solverTerminationCond,
                                prm.densityDevTarget, 0u};
        {
            // the loop's kernels are tuned as the loop graph launches them: masked view (live count
            // on the device, per-chunk FP64 partials, every scene active after the reset above)
            const FluidDev fm = Fluid(true);
            const FluidDev fmt = TuneView(fm, nFtot);  // live chunks only, per-chunk partials kept
            EnsureTuned(TUNE_PRESSURE_ACC, fm.n, [&](int v) { LaunchPressureAcc(c, fmt, b, rd, nv, s, v); });
            EnsureTuned(TUNE_JACOBI, fm.n, [&](int v) {
                LaunchJacobi(c, fmt, b, rd, nv, ctl, nullptr, nullptr, 0ull, false, s, v);
            }, true);
        }
        EnsureTuned(TUNE_PRESSURE_ACC, f.n, [&](int v) { LaunchPressureAcc(c, ft, b, rd, nv, s, v); });
        CK(cudaGraphLaunch(LoopGraphFor(c, ctl), s));
        LaunchPressureAcc(c, f, b, rd, nv, s);
        LaunchIntegration(c, f, s);
        CK(cudaMemcpyAsync(hSolver, dSolver.p, S * sizeof(BatchSolverDev), cudaMemcpyDeviceToHost, s));
        CK(cudaEventRecord(ev1, s));
        launches += 7;
        Sync();
        CheckErrors();
        cudaEventElapsedTime(&lastSubstepMs, ev0, ev1);
        for (uint32_t r = 0; r < S; r++) {
            Scene& sc = slots[order[r]];
            sc.solver = hSolver[r];
            sc.steps += 1;
            sc.time += (double)prm.timeStep;
            launches += 4ull * (hSolver[r].iters > 0 ? 0 : 0);
        }
        uint32_t maxIters = 0;
        for (uint32_t r = 0; r < S; r++) maxIters = std::max(maxIters, hSolver[r].iters);
        if (maxIters > 1) launches += 4ull * (maxIters - 1u);
    }

    // ------------------------------------------------------------------------ read-back
    void Push(uint32_t slot, tsp_state_view& v) {
        Scene& sc = At(slot);
        if (layoutDirty) Relayout();
        v.N_F = sc.nF; v.N_B = sc.nB; v.N_R = 0; v.N_RB = 0; v.step = sc.steps; v.time = sc.time;
        const uint32_t nf = sc.nF;
        std::vector<float4> p(nf), vr(nf), vp(nf), ac(nf);
        std::vector<float2> sd(nf);
        std::vector<uint64_t> id(nf);
        CK(cudaMemcpyAsync(p.data(), posP.p + sc.fStart, nf * sizeof(float4), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(vr.data(), velRho.p + sc.fStart, nf * sizeof(float4), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(vp.data(), velPred.p + sc.fStart, nf * sizeof(float4), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(ac.data(), acc.p + sc.fStart, nf * sizeof(float4), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(sd.data(), srcDiag.p + sc.fStart, nf * sizeof(float2), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(id.data(), idF.p + sc.fStart, nf * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        const uint32_t nb = sc.nB;
        std::vector<float4> pb(nb);
        std::vector<float> vb(nb);
        std::vector<uint64_t> ib(nb);
        if (nb) {
            CK(cudaMemcpyAsync(pb.data(), posB.p + sc.bStart, nb * sizeof(float4), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(vb.data(), volB.p + sc.bStart, nb * sizeof(float), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(ib.data(), idB.p + sc.bStart, nb * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        }
        Sync();
        auto put = [](float* a, uint32_t i, float x) { if (a) a[i] = x; };
        for (uint32_t i = 0; i < nf; i++) {
            if (v.idF) v.idF[i] = id[i];
            put(v.xPosF, i, p[i].x); put(v.yPosF, i, p[i].y); put(v.zPosF, i, p[i].z); put(v.pressureF, i, p[i].w);
            put(v.xVelF, i, vr[i].x); put(v.yVelF, i, vr[i].y); put(v.zVelF, i, vr[i].z); put(v.densityF, i, vr[i].w);
            put(v.xVelPredF, i, vp[i].x); put(v.yVelPredF, i, vp[i].y); put(v.zVelPredF, i, vp[i].z);
            put(v.xAccPressF, i, ac[i].x); put(v.yAccPressF, i, ac[i].y); put(v.zAccPressF, i, ac[i].z);
            put(v.sourceTermF, i, sd[i].x); put(v.diagElemF, i, sd[i].y);
        }
        for (uint32_t i = 0; i < nb; i++) {
            if (v.idB) v.idB[i] = ib[i];
            put(v.xPosB, i, pb[i].x); put(v.yPosB, i, pb[i].y); put(v.zPosB, i, pb[i].z); put(v.psiB, i, pb[i].w);
            put(v.volB, i, vb[i]);
        }
    }
    void Stats(uint32_t slot, tsp_step_stats& o) {
        Scene& sc = At(slot);
        o = tsp_step_stats{};
        o.step = sc.steps; o.time = sc.time;
        o.solverIters = sc.solver.iters;
        o.errSumRaw = sc.solver.sums[0]; o.errSumPos = sc.solver.sums[1]; o.errSumAbs = sc.solver.sums[2];
        o.avgRelDensityErrRaw = sc.solver.avg[0]; o.avgRelDensityErrPos = sc.solver.avg[1];
        o.avgRelDensityErrAbs = sc.solver.avg[2];
        o.frameRebuilds = (uint32_t)sc.frameRebuilds;
        o.cellOrig[0] = sc.fr.ox; o.cellOrig[1] = sc.fr.oy; o.cellOrig[2] = sc.fr.oz;
        o.cellDims[0] = sc.fr.nx; o.cellDims[1] = sc.fr.ny; o.cellDims[2] = sc.fr.nz;
        o.keyBits = sc.fr.keyBits;
        o.lastStepMs = lastSubstepMs;
    }
};

}  // namespace tsp

using tsp::Batch;
using tsp::Error;

struct tsp_batch {
    std::unique_ptr<Batch> b;
};

static thread_local std::string g_batchError;

#define TSPB_GUARD(h, body)                                   \
    try {                                                     \
        body;                                                 \
        return TSP_OK;                                        \
    } catch (const Error& e) {                                \
        if (h) (h)->b->lastErr = e.what();                    \
        g_batchError = e.what();                              \
        return e.code;                                        \
    } catch (const std::exception& e) {                       \
        if (h) (h)->b->lastErr = e.what();                    \
        g_batchError = e.what();                              \
        return TSP_ERR_INVALID;                               \
    }
#define TSPB_NEED(h)                          \
    if (!(h) || !(h)->b) {                    \
        g_batchError = "NULL batch handle";   \
        return TSP_ERR_INVALID;               \
    }

extern "C" {

int tsp_b200_batch_create(const tsp_params* params, int device, uint64_t hbm_budget_bytes, tsp_batch** out) {
    if (!params || !out) return TSP_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        g_batchError = "no CUDA device";
        return TSP_ERR_NO_DEVICE;
    }
    if (device < 0) cudaGetDevice(&device);
    tsp_batch* h = new tsp_batch();
    try {
        h->b = std::make_unique<Batch>(*params, device, hbm_budget_bytes);
    } catch (const Error& e) {
        g_batchError = e.what();
        delete h;
        return e.code;
    }
    *out = h;
    return TSP_OK;
}
int tsp_b200_batch_destroy(tsp_batch* h) {
    if (!h) return TSP_OK;
    delete h;
    return TSP_OK;
}
const char* tsp_b200_batch_last_error(const tsp_batch* h) {
    return (h && h->b) ? h->b->lastErr.c_str() : g_batchError.c_str();
}
int tsp_b200_admit(tsp_batch* h, const tsp_state_view* scene, const float dmin[3], const float dmax[3],
                   uint32_t* slot) {
    TSPB_NEED(h);
    if (!scene || !slot) return TSP_ERR_INVALID;
    TSPB_GUARD(h, *slot = h->b->Admit(*scene, dmin, dmax));
}
int tsp_b200_retire(tsp_batch* h, uint32_t slot, tsp_state_view* out) {
    TSPB_NEED(h);
    TSPB_GUARD(h, {
        if (out) h->b->Push(slot, *out);
        h->b->Retire(slot);
    });
}
int tsp_b200_substep_all(tsp_batch* h, const tsp_params* params, uint32_t n) {
    TSPB_NEED(h);
    if (!params) return TSP_ERR_INVALID;
    TSPB_GUARD(h, {
        for (uint32_t k = 0; k < n; k++) h->b->Substep(*params);
    });
}
int tsp_b200_batch_push(tsp_batch* h, uint32_t slot, tsp_state_view* out) {
    TSPB_NEED(h);
    if (!out) return TSP_ERR_INVALID;
    TSPB_GUARD(h, h->b->Push(slot, *out));
}
int tsp_b200_batch_stats(const tsp_batch* h, uint32_t slot, tsp_step_stats* out) {
    TSPB_NEED(h);
    if (!out) return TSP_ERR_INVALID;
    tsp_batch* hh = const_cast<tsp_batch*>(h);
    TSPB_GUARD(hh, hh->b->Stats(slot, *out));
}
int tsp_b200_batch_info(const tsp_batch* h, uint32_t* scenes, uint64_t* fluid_particles, uint64_t* bytes_used,
                        uint64_t* bytes_budget, float* last_substep_ms, uint64_t* launches) {
    TSPB_NEED(h);
    const Batch& b = *h->b;
    uint32_t live = 0;
    uint64_t nf = 0;
    for (const auto& sc : b.slots)
        if (sc.live && !sc.retiring) { live++; nf += sc.nF; }
    if (scenes) *scenes = live;
    if (fluid_particles) *fluid_particles = nf;
    if (bytes_used) *bytes_used = b.used;
    if (bytes_budget) *bytes_budget = b.budget;
    if (last_substep_ms) *last_substep_ms = b.lastSubstepMs;
    if (launches) *launches = b.launches;
    return TSP_OK;
}
uint64_t tsp_b200_batch_scene_bytes(uint32_t n_fluid, uint32_t n_boundary, uint64_t grid_cells) {
    const uint64_t pad = ((uint64_t)n_fluid + 31u) / 32u * 32u;
    return tsp::BatchSceneBytes(pad, n_boundary, grid_cells);
}

}  // extern "C"
