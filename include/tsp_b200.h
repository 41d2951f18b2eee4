/*
 * tsp_b200.h -- C ABI of the B200-native IISPH solver backend.
 *
 * One handle = one solver backend instance (one scene) resident on one GPU. The entry points
 * are the C-level replacement of the reference's solver-backend interface
 * `Sim::I_SimBackend` (source/simulation/core/backend_sim.h:194-261); each declaration below
 * cites the method it replaces. All functions return TSP_OK (0) or a negative status; no C++
 * exception crosses this boundary. `tsp_b200_last_error()` gives the message of the last
 * failure on that handle (thread-local message when the handle is NULL).
 *
 * Particle order: like the reference backends, the backend keeps its own (Morton-sorted)
 * particle order. Pushed fluid/boundary arrays come out in that order together with their
 * particle IDs; rigid particles keep their storage order (source/simulation/CPU/backend/
 * neighbor_search.cpp:747-774).
 *
 * Threading: a handle must be used by one host thread at a time (the reference calls its
 * backend from the single simulation-controller thread, source/simulation/core/simulation.h:150).
 */
#ifndef TSP_B200_H
#define TSP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------- */
#define TSP_OK                  0
#define TSP_ERR_INVALID        -1  /* bad argument / state (std::invalid_argument analogue)   */
#define TSP_ERR_CUDA           -2  /* CUDA runtime error (GPU::Check, gpu_utils.h:24-45)       */
#define TSP_ERR_OVERFLOW       -3  /* count/size overflow (particle_types.h:393-497)            */
#define TSP_ERR_FRAME          -4  /* cell frame exceeds 2^21 cells per axis (cell_frame.h:29)  */
#define TSP_ERR_NEIGHBOR_LIST  -5  /* SELL32 fill overflow / delta range (common.cuh:24-26)     */
#define TSP_ERR_RIGID          -6  /* degenerate rigid orientation (cpu_backend.cpp:46-58)      */
#define TSP_ERR_UNSUPPORTED    -7  /* configuration outside what this backend implements        */
#define TSP_ERR_NO_DEVICE      -8  /* no CUDA device / extension not usable                     */

/* Sim::SolverTerminationCond (source/base/enum_hub.h:212-218) */
#define TSP_TERM_FIXED_ITERS    0u
#define TSP_TERM_REL_ERR_RAW    1u
#define TSP_TERM_REL_ERR_POS    2u
#define TSP_TERM_REL_ERR_ABS    3u

/*
 * Subset of Sim::SimParams (source/simulation/core/parameters_sim.h:25-175) that the step
 * reads. Derived values follow the reference setters (parameters_sim.cpp:1478-1483):
 * massF = restDensity * h^3, kernelRadius = 2h, kernelRadiusSqu = kernelRadius^2.
 * `cubicSplineAlphaOverride` > 0 replaces alpha = 1/(4*pi*h^3) (solver_constants.h:20-36);
 * the reference's own kernel unit tests pass alpha directly (tests/unit/sph_pressure.cpp).
 */
typedef struct tsp_params {
    float timeStep;
    float particleSizeF;
    float particleSizeB;
    float kernelRadius;
    float kernelRadiusSqu;
    float restDensity;
    float massF;
    float massB;
    float viscosityF;
    float viscosityB;
    float gravity[3];
    float pressGamma;
    float jacobiOmega;
    float jacobiWarmStart;
    float densityDevTarget;
    uint32_t fixedIters;
    uint32_t minSolverIters;
    uint32_t maxSolverIters;
    uint32_t solverTerminationCond;   /* TSP_TERM_* */
    float gridCellSizeRatio;
    uint32_t boundaryLayers;
    float cubicSplineAlphaOverride;   /* <= 0: derive from particleSizeF */
    /* rigid contact solver (SolveRigidContacts, rigid_solver.cpp:602-799; parameters_sim.h:100-101);
     * both 0 selects the reference defaults 0.001 and 100 */
    float rigidContactDensityDevTarget;
    uint32_t rigidContactMaxSolverIters;
    /* export surface classification (parameters_sim.h:167-170): fewer fluid neighbors than this
     * marks a fluid particle near-surface; 0 selects the reference default 27 */
    uint32_t surfaceNbrCountThreshold;
    uint32_t reserved[1];
} tsp_params;

/*
 * Host view of Sync::UniversalSimState (source/simulation/sync/state_sim.h): plain SoA
 * pointers and counts. For pull, NULL optional fluid fields mean "zero" (density: rest density),
 * NULL boundary/rigid coefficients take the reference defaults psi = massB,
 * vol = massB / restDensity (state_sim.h:347-362, 461-475). For push, every non-NULL pointer
 * receives N_* values.
 */
typedef struct tsp_state_view {
    uint32_t N_F, N_B, N_R, N_RB;
    uint64_t step;
    double time;
    /* fluid */
    uint64_t* idF;
    float *xPosF, *yPosF, *zPosF;
    float *xVelF, *yVelF, *zVelF;
    float *xVelPredF, *yVelPredF, *zVelPredF;
    float *xAccPressF, *yAccPressF, *zAccPressF;
    float *sourceTermF, *diagElemF, *pressureF, *densityF;
    /* boundary */
    uint64_t* idB;
    float *xPosB, *yPosB, *zPosB;
    float *volB, *psiB;
    /* rigid particles (storage order is preserved) */
    uint64_t* idR;
    uint32_t* bodyIdR;
    float *xPosRelR, *yPosRelR, *zPosRelR;
    float *volR, *psiR;
    float *xPosR, *yPosR, *zPosR;         /* push only: world positions */
    /* rigid bodies */
    uint64_t* idRB;
    uint32_t* rigidParticleCountRB;
    float *xCM, *yCM, *zCM;
    float *xVelRB, *yVelRB, *zVelRB;
    float *xOmegaRB, *yOmegaRB, *zOmegaRB;
    float *xAngMomRB, *yAngMomRB, *zAngMomRB;
    float *a00, *a01, *a02, *a10, *a11, *a12, *a20, *a21, *a22;
    float *massRB, *massInvRB;
    float *iBodyInv00, *iBodyInv01, *iBodyInv02;
    float *iBodyInv10, *iBodyInv11, *iBodyInv12;
    float *iBodyInv20, *iBodyInv21, *iBodyInv22;
} tsp_state_view;

/* Sim::PressureSolveErrorSums (backend_sim.h:62-67) + solver iteration state of the last step */
typedef struct tsp_step_stats {
    uint64_t step;
    double time;
    uint32_t solverIters;          /* N_solverIters_ (sph_solver.cpp:208,229)            */
    uint32_t reserved0;
    double errSumRaw, errSumPos, errSumAbs;  /* FP64 sums of the last evaluated sweep    */
    float avgRelDensityErrRaw, avgRelDensityErrPos, avgRelDensityErrAbs;
    uint32_t frameRebuilds;        /* cell-frame rebuilds since pull                    */
    int32_t cellOrig[3];
    uint32_t cellDims[3];
    uint32_t keyBits;              /* CellIdKeyBits (neighbor_search.cpp:403-413)       */
    uint32_t nCellsF, nCellsB, nCellsR;
    uint64_t nNbrFF, nNbrFB, nNbrFR, nNbrRF, nNbrRB, nNbrRR;
    uint64_t sellPackedBytes;      /* FF+FB+FR Delta16x2 + Abs32 storage                */
    float lastStepMs;              /* device time of the last step (CUDA events)        */
    float lastNeighborMs;          /* of which neighbor search                          */
    float lastJacobiMs;            /* of which Jacobi loop                              */
    uint32_t reserved1;
} tsp_step_stats;

/* CPU::RigidContactReport (source/simulation/CPU/backend/rigid_solver.h:25-30) of the last
 * step's rigid contact solve, plus its contact counts (rigid particles with a contact after the
 * per-body relaxation count + boundary particles in contact; boundary particles referenced by
 * rigid neighbor rows) */
typedef struct tsp_contact_report {
    uint32_t solverIters;
    float avgDensityError;
    uint32_t converged;            /* 1 also when there was no contact */
    uint32_t reserved;
    uint64_t nContacts;
    uint64_t nContactBoundary;
} tsp_contact_report;

typedef struct tsp_backend tsp_backend;

/* ---- lifecycle: MakeSimBackend (backend_sim.cpp:18-38) -------------------------------- */
/* creates a backend on CUDA device `device` (current device when < 0) */
int tsp_b200_create(const tsp_params* params, int device, tsp_backend** out);
/* ~I_SimBackend (backend_sim.h:198) */
int tsp_b200_destroy(tsp_backend* h);
/* I_SimBackend::Name (backend_sim.h:200) */
const char* tsp_b200_name(const tsp_backend* h);
/* last error message of h (or of this thread when h is NULL) */
const char* tsp_b200_last_error(const tsp_backend* h);

/* ---- state boundary ------------------------------------------------------------------ */
/* I_SimBackend::SetSimDomainBounds (backend_sim.h:204); an empty extent leaves it unbounded */
int tsp_b200_set_domain(tsp_backend* h, const float min_xyz[3], const float max_xyz[3]);
/* I_SimBackend::PullFromUniversalSimState (backend_sim.h:207) */
int tsp_b200_pull_state(tsp_backend* h, const tsp_state_view* src, const tsp_params* params);
/* I_SimBackend::PushToUniversalSimState (backend_sim.h:211): copies into caller arrays */
int tsp_b200_push_state(tsp_backend* h, tsp_state_view* dst);
/* I_SimBackend::GetNumFluidParticles / Boundary / Rigid (backend_sim.h:258-260) */
int tsp_b200_get_counts(const tsp_backend* h, uint32_t* nF, uint32_t* nB, uint32_t* nR, uint32_t* nRB);

/* ---- hot path -------------------------------------------------------------------------- */
/* I_SimBackend::ExecuteNeighborSearch (backend_sim.h:249; CPU cpu_backend.cpp:1593-1624):
 * reorders ALL fluid fields, rebuilds cell tables and the SELL32 / CSR neighbor lists */
int tsp_b200_neighbor_search(tsp_backend* h, const tsp_params* params);
/* I_SimBackend::ExecuteFullSimStep (backend_sim.h:252; CPU Step_IISPH sph_solver.cpp:34-319):
 * runs n_steps IISPH steps (the step counters advance by n_steps) */
int tsp_b200_step(tsp_backend* h, const tsp_params* params, uint32_t n_steps);
/* solver statistics of the last step (FillStatisticsRecord analogue, backend_sim.h:243) */
int tsp_b200_get_stats(const tsp_backend* h, tsp_step_stats* out);

/* ---- inspection (test access, like the reference's NeighborSearchTestAccess) ----------- */
#define TSP_SPECIES_F 0u
#define TSP_SPECIES_B 1u
#define TSP_SPECIES_R 2u
/* per-particle cell IDs in current (sorted) order; rigid: in storage order */
int tsp_b200_read_cell_ids(const tsp_backend* h, uint32_t species, uint64_t* out, uint32_t n);
/* last sort permutation: oldIdx of newIdx (fluid, boundary); rigid: sorted-slot -> rigid idx */
int tsp_b200_read_permutation(const tsp_backend* h, uint32_t species, uint32_t* out, uint32_t n);
/* compact cell table: returns count in *n_cells; fills when buffers are non-NULL (capacity cap) */
int tsp_b200_read_cell_table(const tsp_backend* h, uint32_t species, uint64_t* unique_ids,
                             uint32_t* cell_start /* n_cells + 1 */, uint32_t cap, uint32_t* n_cells);

#define TSP_LIST_FF 0u
#define TSP_LIST_FB 1u
#define TSP_LIST_FR 2u
#define TSP_LIST_RF 3u
#define TSP_LIST_RB 4u
#define TSP_LIST_RR 5u
/* SELL32 meta of FF/FB/FR (GPU layout of the reference, neighbor_search_kernels.cu:86-250):
 * counts[N_F], chunk pitch/format/base/base2/offset [n_chunks]; sizes of the packed buffers */
int tsp_b200_read_sell32_meta(const tsp_backend* h, uint32_t list, uint16_t* counts,
                              uint16_t* chunk_pitch, uint8_t* chunk_format, uint32_t* chunk_base,
                              uint32_t* chunk_base2, uint64_t* chunk_offset, uint32_t n_chunks,
                              uint64_t* n_delta16, uint64_t* n_abs32);
int tsp_b200_read_sell32_words(const tsp_backend* h, uint32_t list, uint16_t* delta16, uint64_t n16,
                               uint32_t* abs32, uint64_t n32);
/* decoded neighbor rows as CSR: offsets[n_src+1], indices[total] (any list) */
int tsp_b200_read_rows(const tsp_backend* h, uint32_t list, uint64_t* offsets, uint32_t n_src,
                       uint32_t* indices, uint64_t cap, uint64_t* total);

/* ---- stage access (test access to single solver stages on the resident state) --------- */
#define TSP_STAGE_DENSITY            1u  /* Density_ChunkedSELL            sph_solver.cpp:734  */
#define TSP_STAGE_NON_PRESSURE       2u  /* NonPressureAcceleration        sph_solver.cpp:892  */
#define TSP_STAGE_SOURCE_DIAG_INIT   3u  /* SourceTermAndDiagonal...Init   sph_solver.cpp:1225 */
#define TSP_STAGE_PRESSURE_ACC       4u  /* PressureAcceleration           sph_solver.cpp:1507 */
#define TSP_STAGE_JACOBI_UPDATE      5u  /* PressureRelaxedJacobiSolver    sph_solver.cpp:1781 */
#define TSP_STAGE_INTEGRATION        6u  /* Integration                    sph_solver.cpp:2051 */
#define TSP_STAGE_BOUNDARY_VOLUMES   7u  /* ComputeParticleCoefficients    builder.cpp:174     */
/* runs one stage; for TSP_STAGE_JACOBI_UPDATE `err_sums` (3 doubles) receives the FP64 sums */
int tsp_b200_run_stage(tsp_backend* h, const tsp_params* params, uint32_t stage, double* err_sums);

#define TSP_FIELD_POS        0u  /* 3 floats per fluid particle */
#define TSP_FIELD_VEL        1u  /* 3 */
#define TSP_FIELD_VEL_PRED   2u  /* 3 */
#define TSP_FIELD_ACC_PRESS  3u  /* 3 */
#define TSP_FIELD_SOURCE     4u  /* 1 */
#define TSP_FIELD_DIAG       5u  /* 1 */
#define TSP_FIELD_PRESSURE   6u  /* 1 */
#define TSP_FIELD_DENSITY    7u  /* 1 */
#define TSP_FIELD_VOL_B      8u  /* 1 per boundary particle */
#define TSP_FIELD_PSI_B      9u  /* 1 per boundary particle */
#define TSP_FIELD_VOL_R     10u  /* 1 per rigid particle */
#define TSP_FIELD_PSI_R     11u  /* 1 per rigid particle */
#define TSP_FIELD_FORCE_R   12u  /* 3 per rigid particle */
#define TSP_FIELD_BODY_FT   13u  /* 6 doubles per body: force xyz, torque xyz (FP64) */
/* reads (write_field: overwrites) one field as an interleaved (n x comps) float array;
 * TSP_FIELD_BODY_FT uses double */
int tsp_b200_read_field(const tsp_backend* h, uint32_t field, void* out, uint32_t n);
int tsp_b200_write_field(tsp_backend* h, uint32_t field, const void* in, uint32_t n);

/* ---- measurement (the reference's BenchmarksTracker role, eval/bench/benchmarks.h) ------ */
/* launches `stage` `reps` times back to back on the backend's stream between two CUDA
 * events and returns the average device time per launch (the stage must be runnable, see
 * tsp_b200_run_stage; TSP_STAGE_JACOBI_UPDATE modifies the pressure field) */
int tsp_b200_time_stage(tsp_backend* h, const tsp_params* params, uint32_t stage, uint32_t reps,
                        float* ms_per_launch);
/* the cudaStream_t all work of this backend runs on (for events / ordering by the caller) */
int tsp_b200_get_stream(const tsp_backend* h, void** stream);
/* device time (ms, CUDA events) of the phases of the last step, in this order: frame update,
 * sort + reorder + cell tables + grids, query count, finalize + size read-back, query fill,
 * density, non-pressure (+ rigid viscous forces), source/diagonal/init, Jacobi loop, final
 * pressure acceleration (+ rigid pressure forces), integration (+ rigid integration), stats
 * read-back. *n = number written (0 before the first step). Analogue of the reference's
 * per-stage BenchOp timers (source/simulation/core/backend_sim.h:255, GetBenchOps). */
int tsp_b200_get_phase_times(const tsp_backend* h, float* ms, uint32_t cap, uint32_t* n);
/* Stats::StatMetric (source/eval/stats/metrics.h:23-86): index of each value in the record
 * tsp_b200_fill_statistics writes (same order and meaning as the reference's enum) */
#define TSP_STAT_NUM_F                       0
#define TSP_STAT_NUM_B                       1
#define TSP_STAT_NUM_R                       2
#define TSP_STAT_NUM_NBR_FF_AVG             3
#define TSP_STAT_NUM_NBR_FF_MIN             4
#define TSP_STAT_NUM_NBR_FF_MAX             5
#define TSP_STAT_NUM_NBR_FF_P99             6
#define TSP_STAT_NUM_NBR_FB_AVG             7
#define TSP_STAT_NUM_NBR_FB_MIN             8
#define TSP_STAT_NUM_NBR_FB_MAX             9
#define TSP_STAT_NUM_NBR_FB_P99             10
#define TSP_STAT_NUM_NBR_FR_AVG             11
#define TSP_STAT_NUM_NBR_FR_MIN             12
#define TSP_STAT_NUM_NBR_FR_MAX             13
#define TSP_STAT_NUM_NBR_FR_P99             14
#define TSP_STAT_NUM_NBR_RF_AVG             15
#define TSP_STAT_NUM_NBR_RF_MIN             16
#define TSP_STAT_NUM_NBR_RF_MAX             17
#define TSP_STAT_NUM_NBR_RF_P99             18
#define TSP_STAT_NUM_NBR_RB_AVG             19
#define TSP_STAT_NUM_NBR_RB_MIN             20
#define TSP_STAT_NUM_NBR_RB_MAX             21
#define TSP_STAT_NUM_NBR_RB_P99             22
#define TSP_STAT_NUM_NBR_RR_AVG             23
#define TSP_STAT_NUM_NBR_RR_MIN             24
#define TSP_STAT_NUM_NBR_RR_MAX             25
#define TSP_STAT_NUM_NBR_RR_P99             26
#define TSP_STAT_DENS_REL_ERROR_RAW_AVG      27
#define TSP_STAT_DENS_REL_ERROR_POS_AVG      28
#define TSP_STAT_DENS_REL_ERROR_ABS_AVG      29
#define TSP_STAT_NUM_SOLVER_ITERS            30
#define TSP_STAT_CFL_NUMBER                  31
#define TSP_STAT_VEL_MAG_AVG                 32
#define TSP_STAT_VEL_MAG_MIN                 33
#define TSP_STAT_VEL_MAG_MAX                 34
#define TSP_STAT_COUNT                       35
/* I_SimBackend::FillStatisticsRecord (backend_sim.h:243; GPU backend gpu_backend.cpp:1067-1203)
 * of the last step or neighbor search: particle counts, neighbor-count average / min / max /
 * 99th percentile per relation, average relative density errors, solver iterations, CFL
 * number and velocity magnitude average / min / max. `record` receives min(n, TSP_STAT_COUNT)
 * doubles. */
int tsp_b200_fill_statistics(const tsp_backend* h, const tsp_params* params, double* record, uint32_t n);
/* SimBackend_CPU::GetRigidContactReport (cpu_backend.h:132) */
int tsp_b200_get_contact_report(const tsp_backend* h, tsp_contact_report* out);
/* number of CUDA kernels this backend launched since creation (graph nodes included) */
int tsp_b200_get_launch_count(const tsp_backend* h, uint64_t* count);
/* device milliseconds of all steps this backend ran since creation (the sum of the per-step
 * times of tsp_step_stats.lastStepMs, GetBenchOps analogue, backend_sim.h:255) and their count */
int tsp_b200_get_step_time_total(const tsp_backend* h, double* ms, uint64_t* steps);
/* per-step record of the last 65,536 steps (GetBenchOps analogue, backend_sim.h:255): lets a
 * caller run many steps in one tsp_b200_step call and still read each step's time */
typedef struct tsp_step_record {
    uint64_t step;              /* simulation step counter after the step */
    float ms;                   /* device milliseconds of the step (as tsp_step_stats.lastStepMs) */
    uint32_t solverIters;       /* relaxed-Jacobi iterations of the step */
    double avgRelDensityErrPos; /* average positive density error at the end of its solve */
} tsp_step_record;
/* writes the records of the most recent min(cap, kept) steps, oldest first, and their number to
 * *n; with out NULL (cap ignored) *n receives the number of records kept */
int tsp_b200_get_step_history(const tsp_backend* h, tsp_step_record* out, uint32_t cap, uint32_t* n);

/*
 * Host view of Sync::ExportSnapshot (source/simulation/sync/snapshots.h:37-66): the particles
 * an export writes. Fluid: only the surface particles (near-surface particles and their fluid
 * neighbors), positions and velocity magnitudes, in the backend's particle order; boundary:
 * positions, volumes and mesh flags; rigid: world positions, volumes, body indices. Each
 * non-NULL array must hold the backend's full count of its population (tsp_b200_get_counts);
 * NULL arrays are skipped. The N_* fields receive the exported counts.
 */
typedef struct tsp_export_snapshot {
    uint64_t simStep;
    double simTime;
    uint32_t N_F, N_B, N_R, reserved;
    float *xPosF, *yPosF, *zPosF, *velMagF;
    float *xPosB, *yPosB, *zPosB, *volB;
    uint8_t* isMeshB;
    uint32_t* bodyIdR;
    float *xPosR, *yPosR, *zPosR, *volR;
} tsp_export_snapshot;
#define TSP_NO_MESH_ID UINT64_MAX
/* I_SimBackend::PackExportSnapshot (backend_sim.h:215; GPU backend gpu_backend.cpp:346-540):
 * classification and compaction run on the device, so only the exported particles are copied
 * to the host. `include_b` = 0 exports no boundary particles; boundary particles with an ID
 * >= `mesh_id_begin_b` are mesh particles (TSP_NO_MESH_ID: none). Before the first neighbor
 * search no neighbor counts exist and no fluid particle is exported (as SimBackend_CPU). */
int tsp_b200_pack_export_snapshot(tsp_backend* h, const tsp_params* params, int include_b,
                                  uint64_t mesh_id_begin_b, tsp_export_snapshot* snap);

/* ---- mesh surface sampling ---------------------------------------------------------------
 * Scene::SurfaceSampler (source/simulation/scene/geometry/surface_sampling.cpp): deterministic
 * Poisson sampling of a triangle surface (seeded candidates, area-proportional triangle choice,
 * acceptance in cell phase groups at a minimum spacing) followed by coverage repair (barycentric
 * probe lattices; a probe farther than max(minDistance, maxDistance - probeSpacing) from every
 * sample becomes a sample). Used for mesh boundaries and mesh rigid bodies
 * (boundary_mesh_helpers.h, rigid_mesh_helpers.h). Parameters: parameters_sim.h:122-139. */
typedef struct tsp_surface_sampling_params {
    float minDistance;             /* minimum accepted sample spacing */
    float maxDistance;             /* maximum surface-to-sample gap */
    float coverageProbeSpacing;    /* spacing of the coverage probes */
    float particleSizeF;           /* the sampling may not be coarser than the fluid spacing */
    uint32_t candidateMultiplier;  /* candidates = multiplier x estimated sample count */
    uint32_t reserved;
    uint64_t seed;
} tsp_surface_sampling_params;
/* SurfaceSamplingStats (surface_sampling.h:18-26) */
typedef struct tsp_surface_sampling_stats {
    uint64_t N_candidates;
    uint32_t N_initialSamples;
    uint32_t N_coverageRepairs;
    uint64_t N_coverageProbes;
    float surfaceArea;
    uint32_t reserved;
} tsp_surface_sampling_stats;
/* SurfaceSampler::Sample on the GPU `device` (-1: current): `vertices` 3*nV floats (x, y, z),
 * `triangles` 3*nT vertex indices. The samples (x, y, z) go to `out` (capacity `cap` samples) and
 * their count to *nOut; a too small `cap` returns TSP_ERR_OVERFLOW with *nOut = the count needed
 * (the result is deterministic, so a second call with that capacity returns it). Invalid meshes
 * or parameters return TSP_ERR_INVALID with the reference's message (tsp_b200_last_error(NULL)).
 * `stats` may be NULL. */
int tsp_b200_sample_surface(int device, const float* vertices, uint32_t nV, const uint32_t* triangles, uint32_t nT,
                            const tsp_surface_sampling_params* params, float* out, uint64_t cap, uint64_t* nOut,
                            tsp_surface_sampling_stats* stats);

/* ---- served batch ------------------------------------------------------------------------
 * No counterpart in the reference (its SimulationMgr runs one scene per backend). A batch keeps
 * many independent scenes of one physics setup resident on one GPU and advances all of them
 * per substep over one scene-offset fluid array: one sort, one neighbor build, one solver pass
 * for all scenes; the Jacobi loop drops each scene as it converges. A scene's results do not
 * depend on the other scenes in the batch. Scenes are fluid + boundary (no rigid bodies).
 * Admission charges an estimate of the scene's device memory (tsp_b200_batch_scene_bytes)
 * against the budget given at creation and fails with TSP_ERR_OVERFLOW when it does not fit;
 * admissions and retirements take effect at the next substep. */
typedef struct tsp_batch tsp_batch;
int tsp_b200_batch_create(const tsp_params* params, int device, uint64_t hbm_budget_bytes, tsp_batch** out);
int tsp_b200_batch_destroy(tsp_batch* b);
const char* tsp_b200_batch_last_error(const tsp_batch* b);
/* admits one scene (PullFromUniversalSimState analogue; boundary volumes/psi taken from the view,
 * defaults when NULL) with its sim domain; *slot identifies it until it is retired */
int tsp_b200_admit(tsp_batch* b, const tsp_state_view* scene, const float domain_min[3],
                   const float domain_max[3], uint32_t* slot);
/* retires a scene; when out != NULL its state is pushed first (PushToUniversalSimState) */
int tsp_b200_retire(tsp_batch* b, uint32_t slot, tsp_state_view* out);
/* advances every admitted scene by n steps (ExecuteFullSimStep of each, fused) */
int tsp_b200_substep_all(tsp_batch* b, const tsp_params* params, uint32_t n);
int tsp_b200_batch_push(tsp_batch* b, uint32_t slot, tsp_state_view* out);
int tsp_b200_batch_stats(const tsp_batch* b, uint32_t slot, tsp_step_stats* out);
int tsp_b200_batch_info(const tsp_batch* b, uint32_t* scenes, uint64_t* fluid_particles, uint64_t* bytes_used,
                        uint64_t* bytes_budget, float* last_substep_ms, uint64_t* launches);
/* device bytes a scene is charged at admission (host arithmetic, no GPU work) */
uint64_t tsp_b200_batch_scene_bytes(uint32_t n_fluid, uint32_t n_boundary, uint64_t grid_cells);

/* ---- autotuner (no counterpart in the reference: its CUDA kernels use one fixed block size,
 * source/simulation/GPU/backend/common.cuh:13-14) ---------------------------------------------
 * The neighbor sweeps and the fluid-query passes exist in several launch configurations (FF
 * slots per pipelined group, minimum resident blocks per SM; for KQueryFluidCount, slots = 1
 * selects the variant that stages the neighboring cell blocks in shared memory). The first step
 * of a backend times every configuration of each kernel on its live state (its first 2^20
 * particles at most), once per size class (particle count rounded to a power of two, all counts
 * from 2^20 up in one class) and device, and keeps the fastest for all later launches of that
 * class in the process; the served batch launches the same kernels with the same choices. The
 * configurations differ in registers, load grouping and staging only, never in the candidates
 * or the order of a sum, so results are identical whichever is chosen. tsp_b200_set_autotune(0) makes every launch use the untuned configuration;
 * tsp_b200_reset_tuning() forgets all choices; tsp_b200_get_tuning writes the choices of a device
 * as a JSON object ("kernel/nN": {slots, min_blocks, ms, untuned_ms, worst_ms, candidates}) and
 * its length (without the terminating zero) to *len; out may be NULL to query the length.
 * tsp_b200_set_tuning pins a configuration (one of the kernel's candidates, as the report names
 * them) for n's size class on a device, e.g. to replay a table saved from an earlier run;
 * TSP_ERR_INVALID if the kernel or configuration is unknown. */
int tsp_b200_set_autotune(int enabled);
int tsp_b200_reset_tuning(void);
int tsp_b200_set_tuning(int device, const char* kernel, uint32_t n, uint32_t slots, uint32_t min_blocks);
int tsp_b200_get_tuning(int device, char* out, uint32_t cap, uint32_t* len);

/* ---- host helpers (no GPU work) -------------------------------------------------------- */
/* Sim::TryBuildCellCoordFrame (source/simulation/core/cell_frame.h:32-66): inclusive signed
 * cell bounds -> frame origin and dimensions. Fails with TSP_ERR_FRAME, leaving origin/dims
 * untouched, if any axis has min > max, a bound outside int32, or more than 2^21 cells. The
 * neighbor search builds its frame with this rule (UpdateCellFrame, neighbor_search.cpp:1902). */
int tsp_b200_try_build_cell_frame(const int64_t cell_min[3], const int64_t cell_max[3], int32_t origin[3],
                                  uint32_t dims[3]);

/* ---- cell-table build without device allocation ---------------------------------------
 * No counterpart in the reference (its cell tables are built inside the backend's neighbor
 * search, source/simulation/CPU/backend/neighbor_search.cpp). For callers that own their
 * particle buffers and stream and must not allocate device memory on the way: a fixed-budget
 * embedding, or a time-critical loop where cudaMalloc / cudaFree (which synchronises the
 * device) would stall other work. The scan scratch is a fixed array inside this library
 * (one per device, 128 KiB); no cudaMalloc, cudaFree or allocating library call is made.
 *
 * Input: n Morton cell IDs sorted ascending (device memory; out-of-frame particles carry
 * 0xFFFFFFFFFFFFFFFF and sort last, as tsp_b200_read_cell_ids returns them). Output, all
 * device memory: d_unique_out[c] = cell ID of run c (room for n), d_start_out[c] = index of
 * the first particle of run c plus d_start_out[num_cells] = n (room for n + 1), and
 * *d_num_cells_out = num_cells. For n = 0 only *d_num_cells_out = 0 and, when d_start_out is
 * not NULL, d_start_out[0] = 0 are written. Outputs need not be zeroed, and nothing has to
 * start at zero.
 * Work is queued on `stream` (a cudaStream_t; NULL = legacy default stream); results are
 * ready when that stream reaches them.
 *
 * Setup: tsp_b200_noalloc_setup(), called once per device with that device current, looks up
 * the scratch's device address there (cudaGetSymbolAddress) and runs one tiny build on the
 * legacy default stream, waiting for it, so that this library's device code, scan kernels
 * included, is loaded on that device (under lazy module loading, the CUDA 12 default, code is
 * otherwise loaded at first use, which takes device memory). Call it during setup, before any
 * time-critical section; later calls then only queue kernels. A call on a device without
 * setup does the same set-up first.
 * Errors: an error that the caller's earlier work left pending is not reported (nor cleared)
 * by a call; a launch error of the call itself is reported as TSP_ERR_CUDA.
 * Limit: n <= TSP_NOALLOC_MAX_PARTICLES; larger n returns TSP_ERR_INVALID and queues nothing.
 * Races: all calls on one device share the scratch, so calls must not overlap in time on that
 * device (issue them on one stream, or order them with events).
 * Errors: TSP_ERR_INVALID / TSP_ERR_CUDA / TSP_ERR_NO_DEVICE; message from
 * tsp_b200_noalloc_last_error() (per host thread). */
#define TSP_NOALLOC_MAX_PARTICLES (1u << 24)
int tsp_b200_noalloc_setup(void);
int tsp_b200_build_cell_table_noalloc(const uint64_t* d_cell_ids_sorted, uint32_t n, uint64_t* d_unique_out,
                                      uint32_t* d_start_out, uint64_t* d_num_cells_out, void* stream);
const char* tsp_b200_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* TSP_B200_H */
