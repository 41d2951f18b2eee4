// kernels.h -- host-side launch interface of the CUDA kernels (one declaration per launcher).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <functional>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "common.cuh"
#include "../../include/tsp_b200.h"

namespace tsp {

struct U64x2;

// kernels with autotuned launch configurations (tune.cu) and one configuration of a candidate list
enum TuneKernel : int {
    TUNE_DENSITY, TUNE_NON_PRESSURE, TUNE_SOURCE_DIAG, TUNE_PRESSURE_ACC, TUNE_JACOBI, TUNE_QUERY_COUNT,
    TUNE_QUERY_FILL, TUNE_KERNELS
};
struct TuneCandidate {
    uint16_t slots;      // FF list slots per pipelined group (sweeps); count pass: 1 = cell blocks staged in shared memory
    uint16_t minBlocks;  // __launch_bounds__ minimum resident blocks per SM
};

constexpr uint32_t QUERY_THREADS = 128;  // 4 warps = 4 SELL32 chunks per block
constexpr uint32_t MAX_JACOBI_SWEEPS = 100000;  // hard bound of the device-driven Jacobi loop

// window of the Delta16x2 home group around a chunk (neighbor_search_kernels.cu:86-97)
__host__ __device__ __forceinline__ void HomeWindow(uint32_t chunk, uint32_t& lo, uint32_t& hi) {
    constexpr uint32_t reach = (0x8000u - SELL_W) / 2u;
    constexpr uint32_t hiOff = SELL_W - 1u + reach;
    const uint32_t b = chunk * SELL_W;
    lo = (b > reach) ? (b - reach) : 0u;
    hi = (b < 0xffffffffu - hiOff) ? (b + hiOff) : 0xffffffffu;
}

struct DomainBox {
    float mn[3], mx[3];
    int bounded;
};

struct ProbeResult {
    int mnKey[3], mxKey[3];   // order-preserving integer images of the float bounds
    uint32_t exceeded;
    uint32_t pad;
};
float OrderedIntToFloat(int k);
int OrderedIntHost(float f);

struct SortScratch {
    uint64_t* keysA;
    uint64_t* keysB;
    uint32_t* valsA;
    uint32_t* valsB;
    uint32_t* tileHist;
    uint32_t* digitTotals;
    // one-pass sort (OnesweepSortPairs) when set: its auxiliary words (OnesweepAuxWords; zeroed
    // by the sort) and the error word of its bounded look-back; NULL: the three-kernel passes
    uint32_t* osAux;
    uint32_t* err;
};

struct QueryArgs {
    const float4* posF;
    const uint64_t* cidF;
    uint32_t nF;
    const float4* posB;
    uint32_t nB;
    const float4* posR;
    const uint32_t* permR;
    const uint32_t* bodyR;
    uint32_t nR;
    const uint32_t *startF, *startB, *startR;
    const uint32_t *gridF, *gridB, *gridR;  // NULL when the species is absent
    Frame fr;
    float r2;
    uint32_t* err;
    unsigned long long* nbrTotals;  // FF, FB, FR neighbor totals (accumulated by the count pass)
    // count-pass rows per chunk in [slot][lane] layout, ks* slots per lane; a chunk with a
    // longer row sets its bit in scrOver (1 FF, 2 FB, 4 FR) and the fill walks it again
    uint32_t *scrF, *scrB, *scrR;
    uint32_t ksF, ksB, ksR;
    uint8_t* scrOver;
    // served batch only (NULL for one scene): valid lanes and scene of each chunk, and per
    // scene its frame and the offsets of its dense grids inside gridF / gridB
    const uint8_t* chunkLen;
    const uint32_t* chunkScene;
    const struct SceneGeom* scenes;
};
struct SceneGeom {
    Frame fr;
    uint64_t gridOffF, gridOffB;
};

struct RigidLists {
    uint16_t *cntRF, *cntRB, *cntRR;
    uint64_t *offRF, *offRB, *offRR;
    uint32_t *listRF, *listRB, *listRR;
};

// solver iteration state kept on the device across the Jacobi loop
struct SolverState {
    double partial[3];        // unused padding for alignment of sums
    double sums[3];           // FP64 raw / pos / abs of the last sweep
    uint32_t iters;           // N_solverIters_ (sph_solver.cpp:208)
    uint32_t done;
    float avg[3];             // avgRelDensityErrorF_{raw,pos,abs}
    uint32_t ticket;          // last-block-done counter of the reduction
    uint32_t itersTotal;      // sweeps since pull (statistics)
};

struct SolverControl {
    uint32_t minIters, maxIters, fixedIters, cond;
    float target;
    uint32_t nF;
};

// TerminationConditionSatisfied (source/simulation/CPU/backend/sph_solver.cpp:686-732)
__device__ __forceinline__ bool Terminated(const SolverControl& ctl, uint32_t iters, const float* avg) {
    if (iters < ctl.minIters) return false;
    if (iters >= ctl.maxIters) return true;
    switch (ctl.cond) {
        case 0: return iters >= ctl.fixedIters;
        case 1: return avg[0] <= ctl.target;
        case 2: return avg[1] <= ctl.target;
        case 3: return avg[2] <= ctl.target;
        default: return iters >= 3;
    }
}

// fluid SoA on the device (Morton order)
struct FluidDev {
    float4* posP;     // x, y, z, pressure
    float4* velRho;   // vx, vy, vz, density
    float4* velPred;  // vx*, vy*, vz*, -
    float4* acc;      // a^p x, y, z, -
    float2* srcDiag;  // source term, diagonal a_ii
    uint32_t n;
    // served batch only (all NULL for one scene): the particle array holds several scenes, each
    // padded to whole SELL32 chunks; chunkLen = valid lanes of a chunk, chunkScene = its scene,
    // sceneActive = scenes still iterating in the Jacobi loop (converged scenes are skipped),
    // chunkPartials = per-chunk FP64 residual sums (raw, pos, abs) of a Jacobi sweep
    const uint8_t* chunkLen;
    const uint32_t* chunkScene;
    const uint32_t* sceneActive;
    double* chunkPartials;
    // batch Jacobi loop only: the live particle count read on the device (n is then the arena
    // capacity, a graph-captured constant; the sweeps stop at the live chunks)
    const uint32_t* liveN;
};
__device__ __forceinline__ bool LaneActive(const FluidDev& f, uint32_t chunk, uint32_t lane, uint32_t i) {
    return f.chunkLen ? lane < (uint32_t)f.chunkLen[chunk] : i < f.n;
}
__device__ __forceinline__ uint32_t SweepCount(const FluidDev& f) { return f.liveN ? *f.liveN : f.n; }
__device__ __forceinline__ bool ChunkSkipped(const FluidDev& f, uint32_t chunk) {
    return f.sceneActive != nullptr && f.sceneActive[f.chunkScene[chunk]] == 0u;
}
struct BoundaryDev {
    const float4* pos;  // x, y, z, psi
    const float* vol;
    uint32_t n;
};
struct RigidDev {
    const float4* pos;      // world x, y, z, psi
    const float4* vel;      // vx, vy, vz, vol
    const float4* velPred;  // predicted particle velocities
    uint32_t n;
};
struct SellView {
    const uint16_t* counts;
    const uint16_t* pitch;
    const uint8_t* format;
    const uint32_t* base;
    const uint32_t* base2;
    const uint64_t* offset;
    const uint16_t* list16;
    const uint32_t* list32;
};
struct NeighborView {
    SellView ff, fb, fr;
};

// ---- ns_kernels.cu
void LaunchProbe(const float4* pos, uint32_t n, const Frame& fr, bool frameValid, const DomainBox& dom,
                 ProbeResult* out, cudaStream_t s);
void SortByCell(const float4* pos, uint32_t n, const Frame& fr, SortScratch& sc, uint32_t* perm, uint64_t* cidSorted,
                cudaStream_t s);
void LaunchCellIds(const float4* pos, uint32_t n, const Frame& fr, uint64_t* cid, cudaStream_t s);
void GatherF4(const uint32_t* perm, const float4* src, float4* dst, uint32_t n, cudaStream_t s);
void GatherF2(const uint32_t* perm, const float2* src, float2* dst, uint32_t n, cudaStream_t s);
void GatherF1(const uint32_t* perm, const float* src, float* dst, uint32_t n, cudaStream_t s);
void GatherU64(const uint32_t* perm, const uint64_t* src, uint64_t* dst, uint32_t n, cudaStream_t s);
void LaunchReorderFluidStep(const uint32_t* perm, const float4* posIn, const float4* velIn, const uint64_t* idIn,
                            float4* posOut, float4* velOut, uint64_t* idOut, uint32_t n, cudaStream_t s);
void BuildCellTable(const uint64_t* cidSorted, uint32_t n, uint64_t* unique, uint32_t* start, uint64_t* nCellsDev,
                    uint64_t* scanScratch, cudaStream_t s);
void BuildGrid(const uint64_t* unique, const uint64_t* nCellsDev, uint32_t nMax, const Frame& fr, uint32_t* grid,
               uint64_t gridCells, cudaStream_t s);
// the same table and grid by one single-pass kernel (decoupled look-back); aux: CellTableGridAuxWords(n)
uint64_t CellTableGridAuxWords(uint32_t n);
void BuildCellTableGrid(const uint64_t* cidSorted, uint32_t n, uint64_t* unique, uint32_t* start, uint64_t* nCellsDev,
                        uint32_t* grid, const Frame& fr, uint64_t gridCells, uint32_t* aux, uint32_t* err,
                        cudaStream_t s);
uint32_t QueryCap(uint32_t reach);
size_t QueryScratchWords(uint32_t nChunks, uint32_t ks);
size_t QuerySmemBytes(uint32_t reach);  // dynamic shared memory of one fluid-query block
const TuneCandidate* QueryCandidates(bool fill, int* n);
void LaunchQueryFluid(bool fill, const QueryArgs& a, const SellMeta& ff, const SellMeta& fb, const SellMeta& fr,
                      cudaStream_t s, int variant = -1);
void LaunchQueryRigid(bool fill, const QueryArgs& a, const RigidLists& L, cudaStream_t s);
void FinalizeSell(const SellMeta& m, uint32_t nChunks, U64x2* scratch, U64x2* totals, cudaStream_t s);
// the FF, FB and FR finalize scans in one launch (up to 65,536 chunks; three scans beyond)
void FinalizeSell3(const SellMeta& m0, const SellMeta& m1, const SellMeta& m2, uint32_t nChunks, U64x2* scratch,
                   U64x2* totals, cudaStream_t s);
inline uint32_t FinalizeSell3Launches(uint32_t nChunks) { return nChunks == 0 ? 0u : (nChunks <= 65536u ? 1u : 9u); }
void FinalizeCsr(const uint16_t* counts, uint64_t* off, uint32_t n, uint64_t* scratch, uint64_t* total, cudaStream_t s);
void LaunchDecodeSellRows(const SellMeta& m, uint32_t nF, const uint64_t* rowOff, uint32_t* out, cudaStream_t s);

// ---- tune.cu: autotuner of launch configurations (block residency, slots in flight)
const TuneCandidate* TuneCandidates(TuneKernel k, int* n);
const char* TuneKernelName(TuneKernel k);
int TuneDefault(TuneKernel k);                 // candidate used while untuned / with tuning off
int TuneChoice(TuneKernel k, uint32_t n);      // chosen candidate for the size class of n, -1 if none
bool TuneEnabled();
void SetTuneEnabled(bool on);
void TuneReset();
// times every candidate (one warm-up and three timed launches each, CUDA events on s) with
// `launch(i)` and records the fastest for the size class of n; returns the choice
int TuneRun(TuneKernel k, uint32_t n, const std::function<void(int)>& launch, cudaStream_t s);
std::string TuneReport();  // JSON object of every recorded choice on the current device
// records a given configuration as the choice of `kernel` (a TuneKernelName) for n's size class;
// false if the kernel or the configuration is not one of the candidates
bool TuneSet(const char* kernel, uint32_t n, uint32_t slots, uint32_t minBlocks);

// Tuning launches cover at most the first TUNE_MAX_N particles (a multiple of the SELL32 chunk):
// every size class at or above it shares one choice, timed on that many particles, so tuning a
// large scene or batch costs no more than tuning a 2^20-particle one.
constexpr uint32_t TUNE_MAX_N = 1u << 20;
// the view a tuning launch sweeps: the first min(live, TUNE_MAX_N) particles, all their chunks
__host__ __device__ inline FluidDev TuneView(FluidDev f, uint32_t live) {
    f.n = live < TUNE_MAX_N ? live : TUNE_MAX_N;
    f.liveN = nullptr;
    f.sceneActive = nullptr;
    return f;
}

// ---- sph_kernels.cu (variant < 0: the autotuner's choice for the size class, else that candidate)
const TuneCandidate* SweepCandidates(int* n);
void LaunchDensity(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r, const NeighborView& nv,
                   cudaStream_t s, int variant = -1);
void LaunchNonPressure(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r,
                       const NeighborView& nv, cudaStream_t s, int variant = -1);
void LaunchSourceDiagInit(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r,
                          const NeighborView& nv, SolverState* st, cudaStream_t s, int variant = -1);
void LaunchPressureAcc(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r,
                       const NeighborView& nv, cudaStream_t s, int variant = -1);
// one relaxed Jacobi sweep with the FP64 error reduction; the last block applies the
// termination rule and, when `cond` is non-zero, sets the graph's loop condition
void LaunchJacobi(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r, const NeighborView& nv,
                  const SolverControl& ctl, SolverState* st, double* partials, unsigned long long cond,
                  bool hasCond, cudaStream_t s, int variant = -1);
uint32_t JacobiBlocks(uint32_t nF);
void LaunchIntegration(const Consts& c, const FluidDev& f, cudaStream_t s);
void LaunchBoundaryVolumes(const Consts& c, const float4* posB, uint32_t nB, const uint32_t* startB,
                           const uint32_t* gridB, const Frame& fr, float defaultVol, float defaultPsi, float restDensity,
                           float* volOut, float* psiOut, cudaStream_t s);
void LaunchSolverReset(SolverState* st, uint32_t nF, cudaStream_t s);

// ---- rigid_kernels.cu
struct BodyDev {
    double* state;       // per body: 32 doubles (see rigid_kernels.cu)
    double* forceTorque; // per body: 6 doubles
    uint32_t n;
};
struct RigidParticlesDev {
    const uint32_t* body;
    const float4* rel;   // body-frame x, y, z, vol
    float4* pos;         // world x, y, z, psi
    float4* vel;         // x, y, z, vol
    float4* velPred;
    float4* force;       // x, y, z, -
    uint32_t n;
    const uint32_t* byBodyOff;
    const uint32_t* byBodyIdx;
};
void LaunchRigidUpdateParticles(const RigidParticlesDev& r, const BodyDev& b, bool predicted, uint32_t* err,
                                cudaStream_t s);

// ---- stats_kernels.cu: statistics record (gpu_backend.cpp:1067-1203)
uint32_t StatFieldBlocks(uint32_t n);
void LaunchStatNeighborCounts(const uint16_t* counts, uint32_t n, uint32_t* hist, uint32_t* out, cudaStream_t s);
void LaunchStatFields(const float4* velRho, uint32_t n, float rho0, double* partials, float* mm, double* out,
                      cudaStream_t s);

// ---- export_kernels.cu: export snapshot surface classification and compaction
//      (PackExportSnapshot, gpu_backend.cpp:346-540)
uint32_t ExportTiles(uint32_t n);
// writes x, y, z, |v| of the exported particles to out[0 .. ), out[stride ..), out[2 stride ..),
// out[3 stride ..) and their count to *nOut
void LaunchExportSurface(const SellView& ff, const uint16_t* cntFB, const uint16_t* cntFR, uint32_t n,
                         uint32_t threshold, const float4* posP, const float4* velRho, uint8_t* flags,
                         uint32_t* tileCounts, uint32_t* nOut, float* out, uint64_t stride, cudaStream_t s);
void LaunchMeshFlags(const uint64_t* idB, uint32_t n, uint64_t meshIdBegin, uint8_t* out, cudaStream_t s);

// ---- surface_kernels.cu: mesh surface sampling (SurfaceSampler, surface_sampling.cpp); throws
//      Error(TSP_ERR_INVALID) with the reference's message for invalid meshes / parameters
std::vector<float> SampleSurfaceGpu(int device, const float* vtx, uint32_t nV, const uint32_t* tri, uint32_t nT,
                                    const tsp_surface_sampling_params& p, tsp_surface_sampling_stats& st);

// ---- contact_kernels.cu: rigid contact solver (rigid_solver.cpp:90-799)
struct ContactState {
    double errSum;
    unsigned long long nContacts;  // N_contacts of RigidContactRelaxation
    uint32_t iters, maxIters, converged, doUpdate;
    float avgErr, target;
};
struct ContactDev {
    uint32_t nR, nRB;
    const uint32_t* nContactB;     // device count of contact boundary particles
    const uint64_t *offRR, *offRB;
    const uint32_t *listRR, *listRB;  // RR rows (rigid indices), RB rows (boundary indices)
    uint32_t* idxRB;               // RB rows as contact indices
    uint32_t* contactOfB;          // [nB] boundary -> contact index
    uint32_t* localB;              // contact -> boundary index
    uint64_t* offBR;
    uint32_t *idxBR, *curBR;
    const float4* posR;            // world x, y, z, psi
    const float4* relR;            // body-frame x, y, z, vol
    const uint32_t* bodyR;
    const uint32_t *byBodyOff, *byBodyIdx;
    const float4* posB;
    const float* volB;
    const double* bodyState;
    double* bodyFT;
    float4* relW;                  // world lever arms
    float* iw;                     // world inverse inertia, 9 per body
    float *densR, *diagR, *presR, *srcR, *errR, *omegaR;
    float4 *forceC, *velC;
    float *densB, *diagB, *presB, *srcB, *errB, *omegaB;
    double* ftC;                   // contact force / torque, 6 per body
    uint32_t* perBody;
    double* contrib;               // per-element error-sum contributions
    ContactState* st;
    uint32_t* err;
};
void LaunchContactSetup(const ContactDev& d, uint64_t nEntriesRB, uint32_t nB, uint64_t* scanScratch,
                        uint64_t* ncTotal, cudaStream_t s);
void LaunchContactLists(const ContactDev& d, uint64_t nEntriesRB, uint32_t nc, uint64_t* scanScratch,
                        uint64_t* totalScratch, cudaStream_t s);
void LaunchContactPrepare(const ContactDev& d, const Consts& c, uint32_t nc, float target, uint32_t maxIters,
                          cudaStream_t s);
void LaunchContactInitialError(const ContactDev& d, const Consts& c, uint32_t nc, const float4* velPredR,
                               cudaStream_t s);
void LaunchContactIteration(const ContactDev& d, const Consts& c, uint32_t ncCap, unsigned long long cond,
                            cudaStream_t s);
void LaunchContactAddLoads(const ContactDev& d, cudaStream_t s);
void LaunchRigidClearAddGravity(const BodyDev& b, float gx, float gy, float gz, cudaStream_t s);
void LaunchRigidViscousForces(const Consts& c, const RigidParticlesDev& r, const FluidDev& f, const uint64_t* offRF,
                              const uint32_t* listRF, cudaStream_t s);
void LaunchRigidPressureForces(const Consts& c, const RigidParticlesDev& r, const FluidDev& f, const uint64_t* offRF,
                               const uint32_t* listRF, cudaStream_t s);
void LaunchRigidReduce(const RigidParticlesDev& r, const BodyDev& b, cudaStream_t s);
void LaunchRigidPredict(const BodyDev& b, float dt, cudaStream_t s);
void LaunchRigidIntegrate(const BodyDev& b, float dt, uint32_t* err, cudaStream_t s);
void LaunchRigidVolumes(const Consts& c, const float4* rel, const uint32_t* byBodyOff, const uint32_t* byBodyIdx,
                        uint32_t nBodies, uint32_t nR, float defaultVol, float defaultPsi, float restDensity,
                        float* volOut, float* psiOut, cudaStream_t s);

}  // namespace tsp
