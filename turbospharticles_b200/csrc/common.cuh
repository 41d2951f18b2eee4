// common.cuh -- shared device types and math of the B200 IISPH backend.
//
// Everything here is compiled with -fmad=false: every fused multiply-add is an explicit
// fmaf(), so each per-pair term is computed with exactly the operation sequence of the
// reference CPU kernels (source/simulation/CPU/simd.h:279-435, sph_solver.cpp:734-2089).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tsp {

constexpr uint32_t EMPTY_32 = 0xffffffffu;
constexpr uint64_t EMPTY_64 = 0xffffffffffffffffull;
constexpr uint32_t SELL_W = 32u;           // SELL32 slice width = one warp (GPU/backend/common.cuh:11)
constexpr uint8_t FMT_DELTA16X2 = 0u;      // NbrChunkFormat (GPU/backend/common.cuh:17-21)
constexpr uint8_t FMT_ABS32 = 1u;

// error bits written by kernels (read by the host after a step)
constexpr uint32_t ERR_FILL_OVERFLOW = 1u << 0;    // NbrListError_FillOverflow (common.cuh:24)
constexpr uint32_t ERR_DELTA_RANGE = 1u << 2;      // NbrListError_DeltaRangeOverflow (common.cuh:26)
constexpr uint32_t ERR_COUNT_U16 = 1u << 3;        // a neighbor count above uint16 storage
constexpr uint32_t ERR_QUERY_CAP = 1u << 4;        // query stencil larger than the shared staging
constexpr uint32_t ERR_RIGID_ORIENT = 1u << 5;     // degenerate rigid orientation (cpu_backend.cpp:46-58)
constexpr uint32_t ERR_RIGID_ATTACH = 1u << 6;     // rigid particle attached to a missing body
constexpr uint32_t ERR_CONTACT_BODIES = 1u << 7;   // a contact element touches too many bodies
constexpr uint32_t ERR_CONTACT_INVALID = 1u << 8;  // invalid contact diagonal / non-finite error or pressure
                                                   // (rigid_solver.cpp:332-336, 567, 595)
constexpr uint32_t ERR_SORT_LOOKBACK = 1u << 9;    // a sort pass's look-back gave up waiting (bounded spin)
constexpr uint32_t ERR_STAGE_WAIT = 1u << 10;      // a staged query block's bulk copies did not complete (bounded wait)

// cell frame of the compact cell-linked list (source/simulation/core/cell_frame.h:18-26)
struct Frame {
    int32_t ox, oy, oz;
    uint32_t nx, ny, nz;
    float cellSizeInv;
    uint32_t reach;
    uint32_t keyBits;
};

// per-step solver constants, derived on the host exactly like the reference
// (solver_constants.h:287-303, simd.h:359-370, sph_solver.cpp:53-60,928-938,1261-1274,1537-1543)
struct Consts {
    float dt, dt2;
    float sizeInv, sizeSqu, radSqu, alpha;
    float kSize, kTwoSize, kInnerSlope, kInnerOffset, kOuterScale;   // KernelConstants_CubicSpline
    float massF, restDensity, restDensitySquInv, densInvSqu;
    float hEps;              // 0.01 * h^2
    float visFacF, visFacB;  // 10 * viscosity
    float gx, gy, gz;
    float cTermFacF, cTermFacB, diagBFac;
    float omega, warmStart;
    float accCoeffB;         // 2 * gamma / rho0^2 (pressure acceleration)
    int warm;
};

__device__ __forceinline__ int FloorToInt(float v) {  // neighbor_search.cpp:157-162
    const int i = static_cast<int>(v);
    return (v < static_cast<float>(i)) ? (i - 1) : i;
}

__host__ __device__ __forceinline__ uint64_t Spread21(uint32_t v) {  // neighbor_search.cpp:2057-2070
    uint64_t x = static_cast<uint64_t>(v & 0x1fffffu);
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}
__host__ __device__ __forceinline__ uint32_t Compact21(uint64_t x) {
    x &= 0x1249249249249249ULL;
    x = (x | (x >> 2)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x >> 4)) & 0x100f00f00f00f00fULL;
    x = (x | (x >> 8)) & 0x1f0000ff0000ffULL;
    x = (x | (x >> 16)) & 0x1f00000000ffffULL;
    x = (x | (x >> 32)) & 0x1fffffULL;
    return static_cast<uint32_t>(x);
}
__host__ __device__ __forceinline__ uint64_t MortonLocal(uint32_t lx, uint32_t ly, uint32_t lz) {
    return Spread21(lx) | (Spread21(ly) << 1) | (Spread21(lz) << 2);
}

// cell ID of a position under a frame; EMPTY_64 outside it (neighbor_search.cpp:2020-2055)
__device__ __forceinline__ uint64_t CellIdOf(float x, float y, float z, const Frame& f) {
    const int lx = FloorToInt(x * f.cellSizeInv) - f.ox;
    const int ly = FloorToInt(y * f.cellSizeInv) - f.oy;
    const int lz = FloorToInt(z * f.cellSizeInv) - f.oz;
    if (lx < 0 || lx >= (int)f.nx || ly < 0 || ly >= (int)f.ny || lz < 0 || lz >= (int)f.nz) return EMPTY_64;
    return MortonLocal((uint32_t)lx, (uint32_t)ly, (uint32_t)lz);
}

// neighbor test of the reference queries: inclusive cutoff with nested FMA
// (neighbor_search.cpp:1140-1145; GPU neighbor_search_kernels.cu:763-768)
__device__ __forceinline__ bool IsNeighbor(float xi, float yi, float zi, float xj, float yj, float zj, float r2) {
    const float dx = __fsub_rn(xi, xj), dy = __fsub_rn(yi, yj), dz = __fsub_rn(zi, zj);
    return fmaf(dx, dx, fmaf(dy, dy, __fmul_rn(dz, dz))) <= r2;
}

// Distance from its square as the reference's GPU kernels form it (sph_kernels.cu:88-97 of
// its CUDA backend): d2 * rsqrt(max(d2, FLT_MIN)), exactly zero at the self pair; rsqrtf is the
// hardware approximation (at most 2 ulp), not the IEEE square root of the CPU path
__device__ __forceinline__ float DistInv(float d2) { return rsqrtf(fmaxf(d2, 1.17549435e-38f)); }

// KernelWeight_CubicSpline_SIMD (simd.h:279-309): zero outside the strict support
__device__ __forceinline__ float KernelWeight(float dx, float dy, float dz, const Consts& c) {
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const float dist = d2 * DistInv(d2);
    const float q = dist * c.sizeInv;
    const float t1 = fmaxf(1.0f - q, 0.0f);
    const float t2 = fmaxf(2.0f - q, 0.0f);
    const float t1_2 = t1 * t1, t2_2 = t2 * t2;
    const float t1_3 = t1_2 * t1, t2_3 = t2_2 * t2;
    const float kw = c.alpha * fmaf(-4.0f, t1_3, t2_3);
    return (d2 < c.radSqu) ? kw : 0.0f;
}

// KernelGradientFactorNoMinDist_CubicSpline_SIMD (simd.h:374-388); gradient = factor * (dx,dy,dz);
// 1/dist and dist from one reciprocal square root, as the reference's GPU kernels do
// (sph_kernels.cu:99-114 of its CUDA backend)
__device__ __forceinline__ float GradFactor(float d2, const Consts& c) {
    const float distInv = DistInv(d2);
    const float dist = d2 * distInv;
    const float inner = fmaf(c.kInnerSlope, dist, c.kInnerOffset);
    const float t2 = fmaxf(c.kTwoSize - dist, 0.0f);
    const float outer = (t2 * t2) * (c.kOuterScale * distInv);
    return (dist < c.kSize) ? inner : outer;
}

// KernelGradient_CubicSpline_Scalar (simd.h:311-347), used by the rigid force accumulations
__device__ __forceinline__ void GradScalar(float dx, float dy, float dz, const Consts& c,
                                           float& gx, float& gy, float& gz) {
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if (d2 >= c.radSqu) { gx = gy = gz = 0.0f; return; }
    const float dist = sqrtf(d2);
    const float q = dist * c.sizeInv;
    float f;
    if (q < 1.0f) {
        f = c.alpha * c.sizeInv * c.sizeInv * fmaf(9.0f, q, -12.0f);
    } else {
        const float t2 = fmaxf(2.0f - q, 0.0f);
        f = c.alpha * (-3.0f * t2 * t2) * (c.sizeInv / dist);
    }
    gx = f * dx; gy = f * dy; gz = f * dz;
}

// builder.cpp:49-79: boundary-coefficient weight (self pair -> 4 alpha)
__device__ __forceinline__ float BoundaryWeight(float dx, float dy, float dz, const Consts& c) {
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if (d2 >= c.radSqu) return 0.0f;
    if (d2 < 1e-7f) return 4.0f * c.alpha;
    const float dist = sqrtf(d2);
    const float q = dist * c.sizeInv;
    const float t1 = fmaxf(1.0f - q, 0.0f), t2 = fmaxf(2.0f - q, 0.0f);
    const float t1_2 = t1 * t1, t2_2 = t2 * t2;
    const float t1_3 = t1_2 * t1, t2_3 = t2_2 * t2;
    return c.alpha * (t2_3 - 4.0f * t1_3);
}

// SELL32 chunk metadata of one neighbor category (FF, FB or FR)
struct SellMeta {
    uint16_t* counts;   // [N_F]
    uint16_t* pitch;    // [nChunks]
    uint8_t* format;    // [nChunks]
    uint32_t* base;     // [nChunks]
    uint32_t* base2;    // [nChunks]
    uint64_t* offset;   // [nChunks], index into list16 or list32 by format
    uint16_t* list16;
    uint32_t* list32;
    uint64_t cap16, cap32;
};

// neighbor j of (chunk meta, slot k, lane); decode of StoreNeighbor_CompressedSell32
// (neighbor_search_kernels.cu:193-247)
__device__ __forceinline__ uint32_t SellNeighbor(uint8_t fmt, uint32_t base, uint32_t base2, uint64_t off,
                                                 uint32_t k, uint32_t lane, const uint16_t* __restrict__ l16,
                                                 const uint32_t* __restrict__ l32) {
    const uint64_t lin = off + (uint64_t)k * SELL_W + lane;
    if (fmt == FMT_DELTA16X2) {
        const uint32_t e = __ldg(l16 + lin);
        return (e & 0x8000u) ? (base2 + (e & 0x7fffu)) : (base + e);
    }
    return __ldg(l32 + lin);
}

}  // namespace tsp
