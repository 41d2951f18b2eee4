// sph_kernels.cu -- IISPH solver kernels over SELL32 neighbor lists.
//
// One warp per SELL32 chunk, lane = fluid particle: slot k of all 32 lanes is one coalesced
// 64 B (Delta16x2) or 128 B (Abs32) load, the loop bound (chunk pitch) is warp-uniform and
// slots past a lane's own count are predicated off. Neighbor attributes are gathered as
// float4 (position + pressure, velocity + density), one 16 B load per neighbor.
//
// Arithmetic: compiled with -fmad=false; each per-pair term and each accumulation follows
// the operation order of the reference CPU kernels (source/simulation/CPU/backend/
// sph_solver.cpp:734-2089) with explicit fmaf where the reference uses fma, and the FF, FB
// and FR partial sums are kept apart and combined exactly as the reference combines them.

#include "kernels.h"

namespace tsp {

constexpr uint32_t SPH_THREADS = 256;
// 1: grid of resident blocks only (warps loop over chunks); 0: one warp per chunk
#ifndef TSP_SPH_PERSISTENT
#define TSP_SPH_PERSISTENT 1
#endif
// Each neighbor sweep is instantiated for every (FF slots per group U, minimum resident blocks
// per SM MB) pair of SWEEP_CANDIDATES; the autotuner (tune.cu) times them on the live state and
// picks one per size class. U and MB change register allocation and load grouping, never the
// order of a sum, so every candidate computes bit-identical results.
#define TSP_SWEEP_CANDIDATES(X) X(2, 4) X(3, 4) X(4, 4) X(2, 5) X(3, 5) X(4, 5) X(2, 6) X(3, 6) X(4, 6) X(2, 8) X(3, 8) X(4, 8)

struct ChunkCursor {
    uint32_t pitch, cnt, base, base2;
    uint64_t off;
    uint8_t fmt;
    __device__ __forceinline__ void load(const SellView& v, uint32_t chunk, uint32_t i, bool act) {
        pitch = v.pitch[chunk]; fmt = v.format[chunk]; base = v.base[chunk]; base2 = v.base2[chunk];
        off = v.offset[chunk];
        cnt = act ? v.counts[i] : 0u;
    }
    __device__ __forceinline__ uint32_t nbr(const SellView& v, uint32_t k, uint32_t lane) const {
        return SellNeighbor(fmt, base, base2, off, k, lane, v.list16, v.list32);
    }
};

// Visits the slots of a lane in order, U slots at a time, pipelined: the list entries of group
// g + 1 are loaded before the neighbor gathers of group g, so one group of stream loads is always
// in flight; then the U gathers (one or two float4 each) and the U pair terms in slot order (the
// sum order is that of one slot after the other). The chunk's format is resolved once per chunk
// (D16: Delta16x2, else Abs32). Slots past the lane's count are not branched around: their entry
// is not loaded, they gather a valid dummy (element 0 of the array) and the body receives
// ok = false and leaves its sums unchanged, so the whole warp runs one instruction stream.
// Addressing: one 64-bit pointer to the lane's column of the chunk's slice, slots at 32-entry
// strides from it; Delta16x2 decodes as j = base + e - (e >> 15) * (base + 0x8000 - base2)
// (= base + e below 0x8000, base2 + (e & 0x7fff) above: StoreNeighbor_CompressedSell32,
// neighbor_search_kernels.cu:193-247).
template <int U, bool TWO, bool D16, typename Body>
__device__ __forceinline__ void SweepFmtPipe(const ChunkCursor& cur, const SellView& v, uint32_t lane,
                                             const float4* A, const float4* B, Body&& body) {
    const uint16_t* p16 = v.list16 + cur.off + lane;
    const uint32_t* p32 = v.list32 + cur.off + lane;
    const uint32_t delta = cur.base + 0x8000u - cur.base2;
    uint32_t jn[U];
    auto fetch = [&](uint32_t k0) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint32_t k = k0 + u;
            const bool ok = k < cur.cnt;
            if constexpr (D16) {
                const uint32_t e = ok ? (uint32_t)__ldg(p16 + (size_t)k * SELL_W) : 0u;
                jn[u] = ok ? cur.base + e - (e >> 15) * delta : 0u;
            } else {
                jn[u] = ok ? __ldg(p32 + (size_t)k * SELL_W) : 0u;
            }
        }
    };
    fetch(0);
    for (uint32_t k0 = 0; k0 < cur.pitch; k0 += U) {
        uint32_t j[U];
#pragma unroll
        for (int u = 0; u < U; u++) j[u] = jn[u];
        fetch(k0 + U);
        float4 a[U], b[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            a[u] = A[j[u]];
            if constexpr (TWO) b[u] = B[j[u]];
            else b[u] = a[u];
        }
#pragma unroll
        for (int u = 0; u < U; u++) body(k0 + u < cur.cnt, j[u], a[u], b[u]);
    }
}
template <int U, bool TWO, typename Body>
__device__ __forceinline__ void SweepSlots(const ChunkCursor& cur, const SellView& v, uint32_t lane,
                                           const float4* A, const float4* B, Body&& body) {
    if (cur.fmt == FMT_DELTA16X2) SweepFmtPipe<U, TWO, true>(cur, v, lane, A, B, body);
    else SweepFmtPipe<U, TWO, false>(cur, v, lane, A, B, body);
}
// as SweepSlots, handing the body the pair's kernel-gradient factor, computed from the gathered
// position (A holds positions) with one reciprocal square root
template <int U, bool TWO, typename Body>
__device__ __forceinline__ void SweepSlotsGrad(const ChunkCursor& cur, const SellView& v, uint32_t lane,
                                               const float4& pi, const Consts& c, const float4* A, const float4* B,
                                               Body&& body) {
    SweepSlots<U, TWO>(cur, v, lane, A, B, [&](bool ok, uint32_t, const float4& a, const float4& b) {
        const float dx = pi.x - a.x, dy = pi.y - a.y, dz = pi.z - a.z;
        body(ok, GradFactor(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), c), a, b);
    });
}

// persistent warps: warp w of the grid handles chunks w, w + W, w + 2W, ...
#define FOR_EACH_CHUNK(n)                                                                  \
    const uint32_t lane = threadIdx.x & 31;                                                \
    const uint32_t nChunks_ = ((n) + SELL_W - 1) / SELL_W;                                 \
    const uint32_t warps_ = (gridDim.x * blockDim.x) >> 5;                                 \
    for (uint32_t chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; chunk < nChunks_; chunk += warps_)

// L2 prefetch of the SELL32 slices a warp sweeps next. A chunk's slice of each category is
// contiguous (pitch * 32 entries from its offset, a multiple of 32 entries, so the start is
// 64-byte aligned and the size a multiple of 64 bytes), so one bulk prefetch per slice pulls it
// into L2 while the warp still works on its current chunk. Lanes 0-2 each own one slice (FF,
// FB, FR list); the slice meta of chunk c + 2W is loaded while chunk c is processed and the
// prefetch of c + W is issued at the start of chunk c.
__device__ __forceinline__ void L2PrefetchBulk(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
struct SlicePrefetch {
    uint32_t pitch, fmt;
    uint64_t off;
    __device__ __forceinline__ const SellView& view(const NeighborView& nv, uint32_t lane) const {
        return lane == 0 ? nv.ff : (lane == 1 ? nv.fb : nv.fr);
    }
    __device__ __forceinline__ void load(const NeighborView& nv, uint32_t chunk, uint32_t nChunks, uint32_t lane) {
        pitch = 0; fmt = 0; off = 0;
        if (lane < 3 && chunk < nChunks) {
            const SellView& v = view(nv, lane);
            pitch = v.pitch[chunk]; fmt = v.format[chunk]; off = v.offset[chunk];
        }
    }
    __device__ __forceinline__ void issue(const NeighborView& nv, uint32_t lane) const {
        if (pitch == 0) return;
        const SellView& v = view(nv, lane);
        const uint32_t n = pitch * SELL_W;
        if (fmt == FMT_DELTA16X2) L2PrefetchBulk(v.list16 + off, n * 2u);
        else L2PrefetchBulk(v.list32 + off, n * 4u);
    }
};
#define FOR_EACH_CHUNK_PF(n, nv)                                                                \
    const uint32_t lane = threadIdx.x & 31;                                                     \
    const uint32_t nChunks_ = ((n) + SELL_W - 1) / SELL_W;                                      \
    const uint32_t warps_ = (gridDim.x * blockDim.x) >> 5;                                      \
    SlicePrefetch pf_;                                                                          \
    pf_.load(nv, ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) + warps_, nChunks_, lane);       \
    for (uint32_t chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; chunk < nChunks_;       \
         chunk += warps_)                                                                       \
        if (pf_.issue(nv, lane), pf_.load(nv, chunk + 2u * warps_, nChunks_, lane), true)

// ----------------------------------------------------------------------------- density
template <int U, int MB>
__global__ void __launch_bounds__(SPH_THREADS, MB) KDensity(Consts c, FluidDev f, BoundaryDev b, RigidDev r, NeighborView nv) {
    FOR_EACH_CHUNK_PF(f.n, nv) {
        const uint32_t i = chunk * SELL_W + lane;
        const bool act = LaneActive(f, chunk, lane, i);
        const float4 pi = act ? f.posP[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        float dF = 0.f, dB = 0.f, dR = 0.f;
        ChunkCursor cur;
        cur.load(nv.ff, chunk, i, act);
        SweepSlots<U, false>(cur, nv.ff, lane, f.posP, nullptr, [&](bool ok, uint32_t, const float4& pj, const float4&) {
            const float t = fmaf(c.massF, KernelWeight(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z, c), dF);
            dF = ok ? t : dF;
        });
        cur.load(nv.fb, chunk, i, act);
        SweepSlots<2, false>(cur, nv.fb, lane, b.pos, nullptr, [&](bool ok, uint32_t, const float4& pj, const float4&) {
            const float t = fmaf(pj.w, KernelWeight(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z, c), dB);
            dB = ok ? t : dB;
        });
        cur.load(nv.fr, chunk, i, act);
        SweepSlots<2, false>(cur, nv.fr, lane, r.pos, nullptr, [&](bool ok, uint32_t, const float4& pj, const float4&) {
            const float t = fmaf(pj.w, KernelWeight(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z, c), dR);
            dR = ok ? t : dR;
        });
        if (act) reinterpret_cast<float*>(f.velRho)[4ull * i + 3] = dF + dB + dR;
    }
}

// ----------------------------------------------------------------------------- non-pressure
template <int U, int MB>
__global__ void __launch_bounds__(SPH_THREADS, MB) KNonPressure(Consts c, FluidDev f, BoundaryDev b, RigidDev r,
                                                         NeighborView nv) {
    FOR_EACH_CHUNK_PF(f.n, nv) {
        const uint32_t i = chunk * SELL_W + lane;
        const bool act = LaneActive(f, chunk, lane, i);
        const float4 pi = act ? f.posP[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 vi = act ? f.velRho[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        float fx = 0.f, fy = 0.f, fz = 0.f, bx = 0.f, by = 0.f, bz = 0.f, rx = 0.f, ry = 0.f, rz = 0.f;
        ChunkCursor cur;
        cur.load(nv.ff, chunk, i, act);
        SweepSlots<U, true>(cur, nv.ff, lane, f.posP, f.velRho, [&](bool ok, uint32_t, const float4& pj, const float4& vj) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
            const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float kg = GradFactor(d2, c);
            const float dot = fmaf(dvx, dx, fmaf(dvy, dy, dvz * dz));
            const float rhoJ = fmaxf(vj.w, 1e-7f);
            // the quotient is formed in every lane (its denominator is positive) and the sums take
            // a select, so no branch around the division splits the warp at a lane's last slot
            const float a = (c.massF * dot) / (rhoJ * (d2 + c.hEps)) * kg;
            const float tx = fmaf(a, dx, fx), ty = fmaf(a, dy, fy), tz = fmaf(a, dz, fz);
            fx = ok ? tx : fx; fy = ok ? ty : fy; fz = ok ? tz : fz;
        });
        cur.load(nv.fb, chunk, i, act);
        SweepSlots<2, false>(cur, nv.fb, lane, b.pos, nullptr, [&](bool ok, uint32_t j, const float4& pj, const float4&) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float kg = GradFactor(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), c);
            const float gx = kg * dx, gy = kg * dy, gz = kg * dz;
            const float dvx = vi.x - 0.0f, dvy = vi.y - 0.0f, dvz = vi.z - 0.0f;
            const float dot = fmaf(dvx, dx, fmaf(dvy, dy, dvz * dz));
            const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float a = (b.vol[j] * dot) / (d2 + c.hEps);
            const float tx = fmaf(a, gx, bx), ty = fmaf(a, gy, by), tz = fmaf(a, gz, bz);
            bx = ok ? tx : bx; by = ok ? ty : by; bz = ok ? tz : bz;
        });
        cur.load(nv.fr, chunk, i, act);
        SweepSlots<2, true>(cur, nv.fr, lane, r.pos, r.vel, [&](bool ok, uint32_t, const float4& pj, const float4& vj) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float kg = GradFactor(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), c);
            const float gx = kg * dx, gy = kg * dy, gz = kg * dz;
            const float dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
            const float dot = fmaf(dvx, dx, fmaf(dvy, dy, dvz * dz));
            const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float a = (vj.w * dot) / (d2 + c.hEps);
            const float tx = fmaf(a, gx, rx), ty = fmaf(a, gy, ry), tz = fmaf(a, gz, rz);
            rx = ok ? tx : rx; ry = ok ? ty : ry; rz = ok ? tz : rz;
        });
        if (!act) continue;
        const float ax = fx * c.visFacF + (bx + rx) * c.visFacB + c.gx;
        const float ay = fy * c.visFacF + (by + ry) * c.visFacB + c.gy;
        const float az = fz * c.visFacF + (bz + rz) * c.visFacB + c.gz;
        f.velPred[i] = make_float4(fmaf(ax, c.dt, vi.x), fmaf(ay, c.dt, vi.y), fmaf(az, c.dt, vi.z), 0.0f);
    }
}

// ----------------------------------------------------------------------------- source / diagonal / init
template <int U, int MB>
__global__ void __launch_bounds__(SPH_THREADS, MB) KSourceDiagInit(Consts c, FluidDev f, BoundaryDev b, RigidDev r,
                                                            NeighborView nv) {
    FOR_EACH_CHUNK_PF(f.n, nv) {
        const uint32_t i = chunk * SELL_W + lane;
        const bool act = LaneActive(f, chunk, lane, i);
        const float4 pi = act ? f.posP[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 vi = act ? f.velPred[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        float sF = 0.f, sB = 0.f, sR = 0.f, cxF = 0.f, cyF = 0.f, czF = 0.f, g2 = 0.f;
        float cxB = 0.f, cyB = 0.f, czB = 0.f, cxR = 0.f, cyR = 0.f, czR = 0.f;
        ChunkCursor cur;
        cur.load(nv.ff, chunk, i, act);
        SweepSlots<U, true>(cur, nv.ff, lane, f.posP, f.velPred, [&](bool ok, uint32_t, const float4& pj, const float4& vj) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
            const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float kg = GradFactor(d2, c);
            const float st = fmaf(dvx, dx, fmaf(dvy, dy, dvz * dz));
            const float t0 = fmaf(kg, st, sF);
            const float t1 = fmaf(kg, dx, cxF), t2 = fmaf(kg, dy, cyF), t3 = fmaf(kg, dz, czF);
            const float t4 = fmaf(kg, kg * d2, g2);  // (kgFac * distSqu first keeps the self pair exactly zero)
            sF = ok ? t0 : sF; cxF = ok ? t1 : cxF; cyF = ok ? t2 : cyF; czF = ok ? t3 : czF; g2 = ok ? t4 : g2;
        });
        cur.load(nv.fb, chunk, i, act);
        SweepSlots<2, false>(cur, nv.fb, lane, b.pos, nullptr, [&](bool ok, uint32_t, const float4& pj, const float4&) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float kg = GradFactor(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), c);
            const float gx = kg * dx, gy = kg * dy, gz = kg * dz;
            const float dvx = vi.x - 0.0f, dvy = vi.y - 0.0f, dvz = vi.z - 0.0f;
            const float st = fmaf(dvx, gx, fmaf(dvy, gy, dvz * gz));
            const float t0 = fmaf(pj.w, st, sB);
            const float t1 = fmaf(pj.w, gx, cxB), t2 = fmaf(pj.w, gy, cyB), t3 = fmaf(pj.w, gz, czB);
            sB = ok ? t0 : sB; cxB = ok ? t1 : cxB; cyB = ok ? t2 : cyB; czB = ok ? t3 : czB;
        });
        cur.load(nv.fr, chunk, i, act);
        SweepSlots<2, true>(cur, nv.fr, lane, r.pos, r.velPred, [&](bool ok, uint32_t, const float4& pj, const float4& vj) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float kg = GradFactor(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), c);
            const float gx = kg * dx, gy = kg * dy, gz = kg * dz;
            const float dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
            const float st = fmaf(dvx, gx, fmaf(dvy, gy, dvz * gz));
            const float t0 = fmaf(pj.w, st, sR);
            const float t1 = fmaf(pj.w, gx, cxR), t2 = fmaf(pj.w, gy, cyR), t3 = fmaf(pj.w, gz, czR);
            sR = ok ? t0 : sR; cxR = ok ? t1 : cxR; cyR = ok ? t2 : cyR; czR = ok ? t3 : czR;
        });
        if (!act) continue;
        sF *= c.massF;
        const float rho = f.velRho[i].w;
        const float src = c.restDensity - rho - c.dt * (sF + sB + sR);
        const float cx = cxF * c.cTermFacF + (cxB + cxR) * c.cTermFacB;
        const float cy = cyF * c.cTermFacF + (cyB + cyR) * c.cTermFacB;
        const float cz = czF * c.cTermFacF + (czB + czR) * c.cTermFacB;
        const float dA = c.massF * fmaf(cx, cxF, fmaf(cy, cyF, cz * czF));
        const float dB = c.massF * c.diagBFac * g2;
        const float dC = fmaf(cx, cxB + cxR, fmaf(cy, cyB + cyR, cz * (czB + czR)));
        const float diag = c.dt2 * (dA + dB + dC);
        const bool valid = fabsf(diag) > 1e-7f;
        const float cold = c.omega * (src / diag);
        const float prev = c.warm ? pi.w : 0.0f;
        const float init = c.warm ? ((prev > 0.0f) ? c.warmStart * prev : cold) : cold;
        f.srcDiag[i] = make_float2(src, diag);
        reinterpret_cast<float*>(f.posP)[4ull * i + 3] = fmaxf(0.0f, valid ? init : 0.0f);
    }
}

// ----------------------------------------------------------------------------- pressure acceleration
template <int U, int MB>
__global__ void __launch_bounds__(SPH_THREADS, MB) KPressureAcc(Consts c, FluidDev f, BoundaryDev b, RigidDev r,
                                                         NeighborView nv) {
    FOR_EACH_CHUNK_PF(SweepCount(f), nv) {
        if (ChunkSkipped(f, chunk)) continue;  // converged scene of a batch
        const uint32_t i = chunk * SELL_W + lane;
        const bool act = LaneActive(f, chunk, lane, i);
        const float4 pi = act ? f.posP[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float fOuter = c.massF * pi.w * c.densInvSqu;
        float ax = 0.f, ay = 0.f, az = 0.f;
        ChunkCursor cur;
        cur.load(nv.ff, chunk, i, act);
        SweepSlotsGrad<U, false>(cur, nv.ff, lane, pi, c, f.posP, nullptr, [&](bool ok, float kg, const float4& pj, const float4&) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float a = (fOuter + c.massF * pj.w * c.densInvSqu) * kg;
            const float tx = fmaf(a, dx, ax), ty = fmaf(a, dy, ay), tz = fmaf(a, dz, az);
            ax = ok ? tx : ax; ay = ok ? ty : ay; az = ok ? tz : az;
        });
        cur.load(nv.fb, chunk, i, act);
        SweepSlotsGrad<2, false>(cur, nv.fb, lane, pi, c, b.pos, nullptr, [&](bool ok, float kg, const float4& pj, const float4&) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float gx = kg * dx, gy = kg * dy, gz = kg * dz;
            const float a = c.accCoeffB * pj.w * pi.w;
            const float tx = fmaf(a, gx, ax), ty = fmaf(a, gy, ay), tz = fmaf(a, gz, az);
            ax = ok ? tx : ax; ay = ok ? ty : ay; az = ok ? tz : az;
        });
        cur.load(nv.fr, chunk, i, act);
        SweepSlotsGrad<2, false>(cur, nv.fr, lane, pi, c, r.pos, nullptr, [&](bool ok, float kg, const float4& pj, const float4&) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float gx = kg * dx, gy = kg * dy, gz = kg * dz;
            const float a = c.accCoeffB * pj.w * pi.w;
            const float tx = fmaf(a, gx, ax), ty = fmaf(a, gy, ay), tz = fmaf(a, gz, az);
            ax = ok ? tx : ax; ay = ok ? ty : ay; az = ok ? tz : az;
        });
        if (act) f.acc[i] = make_float4(0.0f - ax, 0.0f - ay, 0.0f - az, 0.0f);
    }
}

// ----------------------------------------------------------------------------- relaxed Jacobi sweep

template <int U, int MB>
__global__ void __launch_bounds__(SPH_THREADS, MB) KJacobi(Consts c, FluidDev f, BoundaryDev b, RigidDev r, NeighborView nv,
                                                    SolverControl ctl, SolverState* st, double* partials,
                                                    cudaGraphConditionalHandle cond, int hasCond) {
    double eRaw = 0.0, ePos = 0.0, eAbs = 0.0;  // per-lane FP64 sums over the warp's chunks
    FOR_EACH_CHUNK_PF(SweepCount(f), nv) {
        if (ChunkSkipped(f, chunk)) continue;  // converged scene of a batch
        double cRaw = 0.0, cPos = 0.0, cAbs = 0.0;  // this chunk's contribution of the lane
        const uint32_t i = chunk * SELL_W + lane;
        const bool act = LaneActive(f, chunk, lane, i);
        const float4 pi = act ? f.posP[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 ai = act ? f.acc[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        float sF = 0.f, sB = 0.f;
        ChunkCursor cur;
        cur.load(nv.ff, chunk, i, act);
        SweepSlotsGrad<U, true>(cur, nv.ff, lane, pi, c, f.posP, f.acc, [&](bool ok, float kg, const float4& pj, const float4& aj) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float dax = ai.x - aj.x, day = ai.y - aj.y, daz = ai.z - aj.z;
            const float sv = fmaf(dax, dx, fmaf(day, dy, daz * dz));
            const float t = fmaf(kg, sv, sF);
            sF = ok ? t : sF;
        });
        sF *= c.massF;
        cur.load(nv.fb, chunk, i, act);
        SweepSlotsGrad<2, false>(cur, nv.fb, lane, pi, c, b.pos, nullptr, [&](bool ok, float kg, const float4& pj, const float4&) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float gx = kg * dx, gy = kg * dy, gz = kg * dz;
            const float sv = fmaf(ai.x, gx, fmaf(ai.y, gy, ai.z * gz));
            const float t = sB + pj.w * sv;
            sB = ok ? t : sB;
        });
        cur.load(nv.fr, chunk, i, act);
        SweepSlotsGrad<2, false>(cur, nv.fr, lane, pi, c, r.pos, nullptr, [&](bool ok, float kg, const float4& pj, const float4&) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float gx = kg * dx, gy = kg * dy, gz = kg * dz;
            const float sv = fmaf(ai.x, gx, fmaf(ai.y, gy, ai.z * gz));
            const float t = sB + pj.w * sv;
            sB = ok ? t : sB;
        });
        if (act) {
            const float2 sd = f.srcDiag[i];
            const float sys = c.dt2 * (sF + sB);
            const float resid = sd.x - sys;
            const float err = sys - sd.x;
            const bool valid = fabsf(sd.y) > 1e-7f;
            const float pn = fmaxf(0.0f, valid ? fmaf(c.omega, resid / sd.y, pi.w) : 0.0f);
            reinterpret_cast<float*>(f.posP)[4ull * i + 3] = pn;
            if (valid) {
                const double re = (double)(err / c.restDensity);
                cRaw = re;
                cPos = re > 0.0 ? re : 0.0;
                cAbs = fabs(re);
            }
        }
        if (f.chunkPartials) {
            // batch: fixed-order per-chunk sums, reduced per scene by a separate kernel
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                cRaw += __shfl_xor_sync(0xffffffffu, cRaw, d);
                cPos += __shfl_xor_sync(0xffffffffu, cPos, d);
                cAbs += __shfl_xor_sync(0xffffffffu, cAbs, d);
            }
            if (lane == 0) {
                f.chunkPartials[3ull * chunk + 0] = cRaw;
                f.chunkPartials[3ull * chunk + 1] = cPos;
                f.chunkPartials[3ull * chunk + 2] = cAbs;
            }
        } else {
            eRaw += cRaw;
            ePos += cPos;
            eAbs += cAbs;
        }
    }
    if (f.chunkPartials) return;
    // FP64 block reduction (fixed order), last block folds the partials in fixed order
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        eRaw += __shfl_xor_sync(0xffffffffu, eRaw, d);
        ePos += __shfl_xor_sync(0xffffffffu, ePos, d);
        eAbs += __shfl_xor_sync(0xffffffffu, eAbs, d);
    }
    __shared__ double ws[3][SPH_THREADS / 32];
    __shared__ bool amLast;
    const uint32_t warp = threadIdx.x >> 5;
    if (lane == 0) { ws[0][warp] = eRaw; ws[1][warp] = ePos; ws[2][warp] = eAbs; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int w = 0; w < SPH_THREADS / 32; w++) { s0 += ws[0][w]; s1 += ws[1][w]; s2 += ws[2][w]; }
        partials[3ull * blockIdx.x + 0] = s0;
        partials[3ull * blockIdx.x + 1] = s1;
        partials[3ull * blockIdx.x + 2] = s2;
        __threadfence();
        const uint32_t t = atomicAdd(&st->ticket, 1u);
        amLast = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!amLast) return;
    __threadfence();
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (uint32_t p = threadIdx.x; p < gridDim.x; p += SPH_THREADS) {
        s0 += __ldcg(partials + 3ull * p + 0);
        s1 += __ldcg(partials + 3ull * p + 1);
        s2 += __ldcg(partials + 3ull * p + 2);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, d);
        s1 += __shfl_xor_sync(0xffffffffu, s1, d);
        s2 += __shfl_xor_sync(0xffffffffu, s2, d);
    }
    __syncthreads();
    if (lane == 0) { ws[0][warp] = s0; ws[1][warp] = s1; ws[2][warp] = s2; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
    for (int w = 0; w < SPH_THREADS / 32; w++) { t0 += ws[0][w]; t1 += ws[1][w]; t2 += ws[2][w]; }
    st->sums[0] = t0; st->sums[1] = t1; st->sums[2] = t2;
    st->ticket = 0;
    // loop bookkeeping of Step_IISPH (sph_solver.cpp:213-261)
    const uint32_t iters = st->iters + 1;
    st->iters = iters;
    st->itersTotal += 1;
    float avg[3] = {st->avg[0], st->avg[1], st->avg[2]};
    const bool compute = iters >= ctl.minIters && (ctl.cond != 0 || Terminated(ctl, iters, avg));
    if (compute) {
        avg[0] = (float)t0 / (float)ctl.nF;
        avg[1] = (float)t1 / (float)ctl.nF;
        avg[2] = (float)t2 / (float)ctl.nF;
        st->avg[0] = avg[0]; st->avg[1] = avg[1]; st->avg[2] = avg[2];
    }
    // the loop always ends: maxIters is validated on the host, MAX_JACOBI_SWEEPS bounds it anyway
    const bool done = Terminated(ctl, iters, avg) || iters >= MAX_JACOBI_SWEEPS;
    st->done = done ? 1u : 0u;
    if (hasCond) cudaGraphSetConditional(cond, done ? 0u : 1u);
}

__global__ void KSolverReset(SolverState* st, uint32_t nF) {
    st->iters = nF > 0 ? 1u : 0u;
    st->avg[0] = st->avg[1] = st->avg[2] = 0.0f;
    st->sums[0] = st->sums[1] = st->sums[2] = 0.0;
    st->done = 0;
    st->ticket = 0;
}

// ----------------------------------------------------------------------------- integration
__global__ void __launch_bounds__(256) KIntegration(Consts c, FluidDev f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= f.n) return;
    if (f.chunkLen && (i & 31u) >= (uint32_t)f.chunkLen[i >> 5]) return;  // padding of a batched scene
    const float4 vp = f.velPred[i];
    const float4 a = f.acc[i];
    const float4 p = f.posP[i];
    const float4 v = f.velRho[i];
    const float vx = fmaf(c.dt, a.x, vp.x), vy = fmaf(c.dt, a.y, vp.y), vz = fmaf(c.dt, a.z, vp.z);
    f.velRho[i] = make_float4(vx, vy, vz, v.w);
    f.posP[i] = make_float4(fmaf(c.dt, vx, p.x), fmaf(c.dt, vy, p.y), fmaf(c.dt, vz, p.z), p.w);
}

// ----------------------------------------------------------------------------- boundary volumes
// ComputeParticleCoefficients (source/simulation/scene/builder.cpp:174-376): the reference
// walks, per particle, the (2 reach + 1)^2 rows of cells in z, y order with the cells of a
// row in ascending x and the particles of a cell in their (stable) order. The dense Morton
// grid visits exactly those cells in exactly that order, so the FP32 sums are the reference's.
__global__ void __launch_bounds__(256) KBoundaryVolumes(Consts c, const float4* __restrict__ pos, uint32_t n,
                                                      const uint32_t* __restrict__ start,
                                                      const uint32_t* __restrict__ grid, Frame fr, float defVol,
                                                      float defPsi, float rho0, float* __restrict__ vol,
                                                      float* __restrict__ psi) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    const int cx = FloorToInt(p.x * fr.cellSizeInv) - fr.ox, cy = FloorToInt(p.y * fr.cellSizeInv) - fr.oy,
              cz = FloorToInt(p.z * fr.cellSizeInv) - fr.oz;
    const int r = (int)fr.reach;
    float sum = 0.0f;
    for (int oz = cz - r; oz <= cz + r; oz++) {
        if (oz < 0 || oz >= (int)fr.nz) continue;
        for (int oy = cy - r; oy <= cy + r; oy++) {
            if (oy < 0 || oy >= (int)fr.ny) continue;
            for (int ox = cx - r; ox <= cx + r; ox++) {
                if (ox < 0 || ox >= (int)fr.nx) continue;
                const uint32_t cc = grid[(uint64_t)ox + (uint64_t)fr.nx * ((uint64_t)oy + (uint64_t)fr.ny * oz)];
                if (cc == EMPTY_32) continue;
                for (uint32_t j = start[cc]; j < start[cc + 1]; j++) {
                    const float4 q = pos[j];
                    sum += BoundaryWeight(p.x - q.x, p.y - q.y, p.z - q.z, c);
                }
            }
        }
    }
    if (sum > 0.0f && isfinite(sum)) {
        const float v = 1.0f / sum;
        vol[i] = v;
        psi[i] = rho0 * v;
    } else {
        vol[i] = defVol;
        psi[i] = defPsi;
    }
}

// ----------------------------------------------------------------------------- launchers
// persistent grids: at most (resident blocks per SM) x (SMs) blocks, never more than the chunks need
static uint32_t g_numSMs = 0;
template <typename K>
static uint32_t PersistentBlocks(K kernel, uint32_t n) {
    if (g_numSMs == 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g_numSMs = sms > 0 ? (uint32_t)sms : 148u;
    }
    int perSM = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, SPH_THREADS, 0);
    if (perSM <= 0) perSM = 1;
    const uint32_t need = (n + SPH_THREADS - 1) / SPH_THREADS;
    if (!TSP_SPH_PERSISTENT) return std::max(1u, need);
    return std::max(1u, std::min(need, (uint32_t)perSM * g_numSMs));
}
static inline uint32_t SphBlocks(uint32_t n) { return (n + SPH_THREADS - 1) / SPH_THREADS; }
uint32_t JacobiBlocks(uint32_t nF) { return SphBlocks(nF); }

// candidate tables, in TSP_SWEEP_CANDIDATES order
#define TSP_CAND_ENTRY(u, mb) TuneCandidate{u, mb},
static const TuneCandidate kSweepCandidates[] = {TSP_SWEEP_CANDIDATES(TSP_CAND_ENTRY)};
#undef TSP_CAND_ENTRY
constexpr int kSweepCandidateCount = (int)(sizeof(kSweepCandidates) / sizeof(kSweepCandidates[0]));
const TuneCandidate* SweepCandidates(int* n) {
    *n = kSweepCandidateCount;
    return kSweepCandidates;
}
using SweepKernel = void (*)(Consts, FluidDev, BoundaryDev, RigidDev, NeighborView);
using JacobiKernel = void (*)(Consts, FluidDev, BoundaryDev, RigidDev, NeighborView, SolverControl, SolverState*,
                              double*, cudaGraphConditionalHandle, int);
#define TSP_FN_ENTRY_DENSITY(u, mb) &KDensity<u, mb>,
#define TSP_FN_ENTRY_NP(u, mb) &KNonPressure<u, mb>,
#define TSP_FN_ENTRY_SD(u, mb) &KSourceDiagInit<u, mb>,
#define TSP_FN_ENTRY_PACC(u, mb) &KPressureAcc<u, mb>,
#define TSP_FN_ENTRY_JAC(u, mb) &KJacobi<u, mb>,
static const SweepKernel kDensityFns[] = {TSP_SWEEP_CANDIDATES(TSP_FN_ENTRY_DENSITY)};
static const SweepKernel kNonPressureFns[] = {TSP_SWEEP_CANDIDATES(TSP_FN_ENTRY_NP)};
static const SweepKernel kSourceDiagFns[] = {TSP_SWEEP_CANDIDATES(TSP_FN_ENTRY_SD)};
static const SweepKernel kPressureAccFns[] = {TSP_SWEEP_CANDIDATES(TSP_FN_ENTRY_PACC)};
static const JacobiKernel kJacobiFns[] = {TSP_SWEEP_CANDIDATES(TSP_FN_ENTRY_JAC)};
#undef TSP_FN_ENTRY_DENSITY
#undef TSP_FN_ENTRY_NP
#undef TSP_FN_ENTRY_SD
#undef TSP_FN_ENTRY_PACC
#undef TSP_FN_ENTRY_JAC

static int Pick(TuneKernel k, uint32_t n, int variant) {
    if (variant >= 0 && variant < kSweepCandidateCount) return variant;
    const int t = TuneChoice(k, n);
    return t >= 0 ? t : TuneDefault(k);
}
static void LaunchSweep(const SweepKernel* fns, TuneKernel k, int variant, const Consts& c, const FluidDev& f,
                        const BoundaryDev& b, const RigidDev& r, const NeighborView& nv, cudaStream_t s) {
    if (!f.n) return;
    const SweepKernel fn = fns[Pick(k, f.n, variant)];
    fn<<<PersistentBlocks(fn, f.n), SPH_THREADS, 0, s>>>(c, f, b, r, nv);
}

void LaunchDensity(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r, const NeighborView& nv,
                   cudaStream_t s, int variant) {
    LaunchSweep(kDensityFns, TUNE_DENSITY, variant, c, f, b, r, nv, s);
}
void LaunchNonPressure(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r,
                       const NeighborView& nv, cudaStream_t s, int variant) {
    LaunchSweep(kNonPressureFns, TUNE_NON_PRESSURE, variant, c, f, b, r, nv, s);
}
void LaunchSourceDiagInit(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r,
                          const NeighborView& nv, SolverState* st, cudaStream_t s, int variant) {
    LaunchSweep(kSourceDiagFns, TUNE_SOURCE_DIAG, variant, c, f, b, r, nv, s);
    if (st) KSolverReset<<<1, 1, 0, s>>>(st, f.n);
}
void LaunchSolverReset(SolverState* st, uint32_t nF, cudaStream_t s) { KSolverReset<<<1, 1, 0, s>>>(st, nF); }
void LaunchPressureAcc(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r,
                       const NeighborView& nv, cudaStream_t s, int variant) {
    LaunchSweep(kPressureAccFns, TUNE_PRESSURE_ACC, variant, c, f, b, r, nv, s);
}
void LaunchJacobi(const Consts& c, const FluidDev& f, const BoundaryDev& b, const RigidDev& r, const NeighborView& nv,
                  const SolverControl& ctl, SolverState* st, double* partials, unsigned long long cond, bool hasCond,
                  cudaStream_t s, int variant) {
    if (!f.n) return;
    const JacobiKernel fn = kJacobiFns[Pick(TUNE_JACOBI, f.n, variant)];
    fn<<<PersistentBlocks(fn, f.n), SPH_THREADS, 0, s>>>(c, f, b, r, nv, ctl, st, partials,
                                                         (cudaGraphConditionalHandle)cond, hasCond ? 1 : 0);
}
void LaunchIntegration(const Consts& c, const FluidDev& f, cudaStream_t s) {
    if (f.n) KIntegration<<<(f.n + 255) / 256, 256, 0, s>>>(c, f);
}
void LaunchBoundaryVolumes(const Consts& c, const float4* posB, uint32_t nB, const uint32_t* startB,
                           const uint32_t* gridB, const Frame& fr, float defaultVol, float defaultPsi, float restDensity,
                           float* volOut, float* psiOut, cudaStream_t s) {
    if (nB)
        KBoundaryVolumes<<<(nB + 255) / 256, 256, 0, s>>>(c, posB, nB, startB, gridB, fr, defaultVol, defaultPsi,
                                                          restDensity, volOut, psiOut);
}

}  // namespace tsp
