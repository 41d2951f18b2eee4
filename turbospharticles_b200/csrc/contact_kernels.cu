// contact_kernels.cu -- rigid contact solver: pressure-based relaxed Jacobi over rigid-rigid
// and rigid-boundary contact pairs (SolveRigidContacts, source/simulation/CPU/backend/
// rigid_solver.cpp:90-799), run after the fluid integration and before the rigid predictor /
// integrator of the step (sph_solver.cpp:310-316).
//
// Per-particle work is FP32 in the reference's operation order; the body reductions of the
// contact forces are FP64 (fixed-order block tree, as for the fluid forces), and the density
// error sum is FP64 in a fixed order (one value per element, one block folds them). Contact
// boundary particles are numbered in ascending boundary index (the reference numbers them in
// order of first reference; no per-particle result depends on that order). The iteration runs
// on the device in a CUDA graph with a conditional WHILE node; every kernel of the loop reads the
// contact count from device memory, so the captured graph does not depend on it.
#include <algorithm>

#include "kernels.h"
#include "primitives.cuh"

namespace tsp {

constexpr int BODY_STRIDE_C = 48;      // body state layout of rigid_kernels.cu
constexpr float CONTACT_VOL = 0.7f;    // RIGID_CONTACT_VOLUME_FACTOR (rigid_solver.h:23)
constexpr int CONTACT_MAX_BODIES = 8;  // distinct bodies one contact element may touch

// ContactKernel (rigid_solver.cpp:51-63): cubic-spline weight and scalar gradient
__device__ __forceinline__ float ContactKernel(float dx, float dy, float dz, const Consts& c, float& gx, float& gy,
                                               float& gz) {
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if (d2 >= c.radSqu) { gx = gy = gz = 0.0f; return 0.0f; }
    const float q = sqrtf(d2) * c.sizeInv;
    const float t1 = fmaxf(1.0f - q, 0.0f), t2 = fmaxf(2.0f - q, 0.0f);
    GradScalar(dx, dy, dz, c, gx, gy, gz);
    return c.alpha * (t2 * t2 * t2 - 4.0f * t1 * t1 * t1);
}

__device__ __forceinline__ float3 ContactPos(const ContactDev& d, bool boundary, uint32_t j) {
    if (boundary) {
        const float4 p = d.posB[d.localB[j]];
        return make_float3(p.x, p.y, p.z);
    }
    const float4 p = d.posR[j];
    return make_float3(p.x, p.y, p.z);
}
__device__ __forceinline__ float ContactVol(const ContactDev& d, bool boundary, uint32_t j) {
    return boundary ? d.volB[d.localB[j]] : d.relR[j].w;
}

// ForEachContactNeighbor (rigid_solver.cpp:22-48): BR row of a contact boundary particle; RR
// then RB (contact indices) row of a rigid particle
template <class Fn>
__device__ __forceinline__ void ForEachContact(const ContactDev& d, bool boundary, uint32_t i, Fn&& f) {
    if (boundary) {
        for (uint64_t k = d.offBR[i]; k < d.offBR[i + 1]; k++) f(d.idxBR[k], false);
        return;
    }
    for (uint64_t k = d.offRR[i]; k < d.offRR[i + 1]; k++) f(d.listRR[k], false);
    for (uint64_t k = d.offRB[i]; k < d.offRB[i + 1]; k++) f(d.idxRB[k], true);
}

// ---------------------------------------------------------------------------- contact set
__global__ void KCMark(ContactDev d, uint64_t nEntries) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nEntries) d.contactOfB[d.listRB[e]] = 1u;
}
struct CFlagIn {
    const uint32_t* f;
    __device__ uint64_t operator()(uint64_t b) const { return f[b] == 1u ? 1ull : 0ull; }
};
struct CFlagOut {
    uint32_t* contactOfB;
    uint32_t* localB;
    __device__ void operator()(uint64_t b, uint64_t pre, uint64_t v) const {
        if (v) localB[pre] = (uint32_t)b;
        contactOfB[b] = v ? (uint32_t)pre : EMPTY_32;
    }
};
__global__ void KCIdxRB(ContactDev d, uint64_t nEntries) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nEntries) return;
    const uint32_t c = d.contactOfB[d.listRB[e]];
    d.idxRB[e] = c;
    atomicAdd(&d.curBR[c], 1u);
}
struct CCountIn {
    const uint32_t* c;
    __device__ uint64_t operator()(uint64_t i) const { return c[i]; }
};
struct CCsrOut {
    uint64_t* off;
    uint32_t* cur;
    uint64_t n;
    __device__ void operator()(uint64_t i, uint64_t pre, uint64_t v) const {
        off[i] = pre;
        cur[i] = (uint32_t)pre;
        if (i == n - 1) off[n] = pre + v;
    }
};
__global__ void KCFillBR(ContactDev d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nR) return;
    for (uint64_t k = d.offRB[i]; k < d.offRB[i + 1]; k++) d.idxBR[atomicAdd(&d.curBR[d.idxRB[k]], 1u)] = i;
}
__global__ void KCSortBR(ContactDev d) {  // BR rows in ascending rigid index (the reference's build order)
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= *d.nContactB) return;
    uint32_t* row = d.idxBR + d.offBR[c];
    const uint32_t n = (uint32_t)(d.offBR[c + 1] - d.offBR[c]);
    for (uint32_t x = 1; x < n; x++) {
        const uint32_t v = row[x];
        uint32_t y = x;
        while (y > 0 && row[y - 1] > v) { row[y] = row[y - 1]; y--; }
        row[y] = v;
    }
}

// ---------------------------------------------------------------------------- geometry
// RigidContactGeometry (rigid_solver.cpp:151-227): world inverse inertia per body, world lever
// arm per rigid particle, FP32 from the FP32 images of the body state
__global__ void KCGeometry(ContactDev d) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < d.nRB) {
        const double* s = d.bodyState + (uint64_t)t * BODY_STRIDE_C;
        float A[9], B[9], T[9];
        for (int k = 0; k < 9; k++) { A[k] = (float)s[12 + k]; B[k] = (float)s[23 + k]; }
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++)
                T[r * 3 + c] = A[r * 3 + 0] * B[0 * 3 + c] + A[r * 3 + 1] * B[1 * 3 + c] + A[r * 3 + 2] * B[2 * 3 + c];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++)
                d.iw[9ull * t + r * 3 + c] = T[r * 3 + 0] * A[c * 3 + 0] + T[r * 3 + 1] * A[c * 3 + 1] +
                                             T[r * 3 + 2] * A[c * 3 + 2];
    }
    if (t < d.nR) {
        const uint32_t b = d.bodyR[t];
        const double* s = d.bodyState + (uint64_t)b * BODY_STRIDE_C;
        const float a00 = (float)s[12], a01 = (float)s[13], a02 = (float)s[14];
        const float a10 = (float)s[15], a11 = (float)s[16], a12 = (float)s[17];
        const float a20 = (float)s[18], a21 = (float)s[19], a22 = (float)s[20];
        const float4 l = d.relR[t];
        d.relW[t] = make_float4(fmaf(a00, l.x, fmaf(a01, l.y, a02 * l.z)), fmaf(a10, l.x, fmaf(a11, l.y, a12 * l.z)),
                                fmaf(a20, l.x, fmaf(a21, l.y, a22 * l.z)), 0.0f);
    }
}

// ---------------------------------------------------------------------------- density + diagonal
struct BodyGradC {
    uint32_t b;
    float x, y, z, tx, ty, tz;
};
__device__ __forceinline__ bool AddBodyGradC(BodyGradC* g, int& n, uint32_t b, float x, float y, float z, float rx,
                                             float ry, float rz) {
    int k = 0;
    while (k < n && g[k].b != b) k++;
    if (k == n) {
        if (n == CONTACT_MAX_BODIES) return false;
        g[n] = BodyGradC{b, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        n++;
    }
    g[k].x += x; g[k].y += y; g[k].z += z;
    g[k].tx += ry * z - rz * y;
    g[k].ty += rz * x - rx * z;
    g[k].tz += rx * y - ry * x;
    return true;
}
// RigidContactDensityAndDiagonal (rigid_solver.cpp:229-344); element t < nR is rigid particle t,
// t >= nR is contact boundary particle t - nR
__global__ void KCDensDiag(ContactDev d, Consts c) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nc = *d.nContactB;
    if (t >= d.nR + nc) return;
    const bool boundary = t >= d.nR;
    const uint32_t i = boundary ? t - d.nR : t;
    BodyGradC g[CONTACT_MAX_BODIES];
    int ng = 0;
    bool ok = true;
    const float volRest = CONTACT_VOL * ContactVol(d, boundary, i);
    float rho = CONTACT_VOL;
    bool has = false;
    const float3 p = ContactPos(d, boundary, i);
    ForEachContact(d, boundary, i, [&](uint32_t j, bool nb) {
        const float3 q = ContactPos(d, nb, j);
        float gx, gy, gz;
        const float w = ContactKernel(p.x - q.x, p.y - q.y, p.z - q.z, c, gx, gy, gz);
        if (!(w > 0.0f)) return;
        has = true;
        const float nv = CONTACT_VOL * ContactVol(d, nb, j);
        rho += nv * w;
        gx *= nv; gy *= nv; gz *= nv;
        if (!boundary) {
            const float4 r = d.relW[i];
            ok = AddBodyGradC(g, ng, d.bodyR[i], gx, gy, gz, r.x, r.y, r.z) && ok;
        }
        if (!nb) {
            const float4 r = d.relW[j];
            ok = AddBodyGradC(g, ng, d.bodyR[j], -gx, -gy, -gz, r.x, r.y, r.z) && ok;
        }
    });
    double diag = 0.0;
    for (int k = 0; k < ng; k++) {
        const uint32_t b = g[k].b;
        const float* I = d.iw + 9ull * b;
        const float wx = I[0] * g[k].tx + I[1] * g[k].ty + I[2] * g[k].tz;
        const float wy = I[3] * g[k].tx + I[4] * g[k].ty + I[5] * g[k].tz;
        const float wz = I[6] * g[k].tx + I[7] * g[k].ty + I[8] * g[k].tz;
        const float massInv = (float)d.bodyState[(uint64_t)b * BODY_STRIDE_C + 22];
        diag += (double)(massInv * (g[k].x * g[k].x + g[k].y * g[k].y + g[k].z * g[k].z) + g[k].tx * wx +
                         g[k].ty * wy + g[k].tz * wz);
    }
    const float dt = c.dt;
    const float dg = (float)((double)dt * (double)dt * (double)volRest / (double)(rho * rho) * diag);
    if (!ok) atomicOr(d.err, ERR_CONTACT_BODIES);
    if (!isfinite(dg) || dg < 0.0f) atomicOr(d.err, ERR_CONTACT_INVALID);
    float* dens = boundary ? d.densB : d.densR;
    float* dia = boundary ? d.diagB : d.diagR;
    float* pres = boundary ? d.presB : d.presR;
    float* src = boundary ? d.srcB : d.srcR;
    float* om = boundary ? d.omegaB : d.omegaR;
    dens[i] = rho; dia[i] = dg; pres[i] = 0.0f; src[i] = rho - 1.0f; om[i] = has ? 0.5f : 0.0f;
}

// ---------------------------------------------------------------------------- relaxation
// RigidContactRelaxation (rigid_solver.cpp:346-407). Rigid part: one block per body.
__global__ void __launch_bounds__(256) KCRelaxR(ContactDev d) {
    const uint32_t body = blockIdx.x;
    uint32_t cnt = 0;
    for (uint32_t w = d.byBodyOff[body] + threadIdx.x; w < d.byBodyOff[body + 1]; w += blockDim.x)
        cnt += d.omegaR[d.byBodyIdx[w]] > 0.0f ? 1u : 0u;
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    __shared__ uint32_t sm[8];
    __shared__ uint32_t total;
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < 8; k++) t += sm[k];
        total = t;
        if (t) atomicAdd((unsigned long long*)&d.st->nContacts, (unsigned long long)t);
    }
    __syncthreads();
    if (total == 0) return;
    for (uint32_t w = d.byBodyOff[body] + threadIdx.x; w < d.byBodyOff[body + 1]; w += blockDim.x) {
        const uint32_t i = d.byBodyIdx[w];
        d.omegaR[i] /= (float)total;
    }
}
// boundary part 1: each movable body counts the contact boundary particles it touches
__global__ void KCRelaxB1(ContactDev d) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= *d.nContactB) return;
    if (d.omegaB[c] <= 0.0f) return;
    atomicAdd((unsigned long long*)&d.st->nContacts, 1ull);
    if (d.diagB[c] <= 0.0f) return;
    const uint64_t b0 = d.offBR[c], b1 = d.offBR[c + 1];
    for (uint64_t k = b0; k < b1; k++) {
        const uint32_t body = d.bodyR[d.idxBR[k]];
        if (!(d.bodyState[(uint64_t)body * BODY_STRIDE_C + 22] > 0.0)) continue;
        bool seen = false;
        for (uint64_t q = b0; q < k && !seen; q++) seen = d.bodyR[d.idxBR[q]] == body;
        if (!seen) atomicAdd(&d.perBody[body], 1u);
    }
}
// boundary part 2: the largest count among the bodies a boundary particle touches
__global__ void KCRelaxB2(ContactDev d) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= *d.nContactB) return;
    if (d.omegaB[c] <= 0.0f || d.diagB[c] <= 0.0f) return;
    uint32_t mx = 0;
    for (uint64_t k = d.offBR[c]; k < d.offBR[c + 1]; k++) mx = max(mx, d.perBody[d.bodyR[d.idxBR[k]]]);
    if (mx > 0) d.omegaB[c] /= (float)mx;
}

// ---------------------------------------------------------------------------- density error
// RigidContactDensityError (rigid_solver.cpp:508-579): residual per element and its FP64
// contribution to the error sum (abs when pressurised, positive part otherwise)
__global__ void KCError(ContactDev d, Consts c, const float4* __restrict__ velR, const float* __restrict__ srcR,
                        const float* __restrict__ srcB, float* __restrict__ errR, float* __restrict__ errB) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nc = *d.nContactB;
    if (t >= d.nR + nc) return;
    const bool boundary = t >= d.nR;
    const uint32_t i = boundary ? t - d.nR : t;
    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (!boundary) { const float4 v = velR[i]; vx = v.x; vy = v.y; vz = v.z; }
    const float3 p = ContactPos(d, boundary, i);
    float res = boundary ? srcB[i] : srcR[i];
    const float dt = c.dt;
    ForEachContact(d, boundary, i, [&](uint32_t j, bool nb) {
        const float3 q = ContactPos(d, nb, j);
        float gx, gy, gz;
        const float w = ContactKernel(p.x - q.x, p.y - q.y, p.z - q.z, c, gx, gy, gz);
        if (!(w > 0.0f)) return;
        float jx = 0.f, jy = 0.f, jz = 0.f;
        if (!nb) { const float4 v = velR[j]; jx = v.x; jy = v.y; jz = v.z; }
        const float dvx = jx - vx, dvy = jy - vy, dvz = jz - vz;
        const float div = dt * (dvx * gx + dvy * gy + dvz * gz);
        res -= CONTACT_VOL * ContactVol(d, nb, j) * div;
    });
    if (!isfinite(res)) atomicOr(d.err, ERR_CONTACT_INVALID);
    (boundary ? errB : errR)[i] = res;
    const float pr = boundary ? d.presB[i] : d.presR[i];
    d.contrib[t] = pr > 0.0f ? fabs((double)res) : fmax((double)res, 0.0);
}

// fixed-order FP64 fold of the contributions by one block; in loop mode also the convergence
// decision of SolveRigidContacts (rigid_solver.cpp:772-790) and the loop condition
__global__ void __launch_bounds__(1024) KCErrorSum(ContactDev d, int loop, cudaGraphConditionalHandle cond) {
    const uint32_t n = d.nR + *d.nContactB;
    double s = 0.0;
    for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) s += d.contrib[t];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double sm[32];
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x != 0) return;
    double tot = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) tot += sm[k];
    ContactState& st = *d.st;
    st.errSum = tot;
    if (!loop) return;
    const uint64_t nct = st.nContacts;
    st.avgErr = nct > 0 ? (float)(tot / (double)nct) : 0.0f;
    st.converged = st.avgErr <= st.target ? 1u : 0u;
    const bool done = st.converged || st.iters >= st.maxIters;
    st.doUpdate = done ? 0u : 1u;
    if (!done) st.iters += 1u;
    cudaGraphSetConditional(cond, done ? 0u : 1u);
}

// ---------------------------------------------------------------------------- loop kernels
// RigidContactPressureForces (rigid_solver.cpp:409-460)
__global__ void KCForces(ContactDev d, Consts c) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nR) return;
    const float4 p = d.posR[i];
    const float pi = d.presR[i] / (d.densR[i] * d.densR[i]);
    const float vi = d.relR[i].w;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    ForEachContact(d, false, i, [&](uint32_t j, bool nb) {
        const float3 q = ContactPos(d, nb, j);
        float gx, gy, gz;
        const float w = ContactKernel(p.x - q.x, p.y - q.y, p.z - q.z, c, gx, gy, gz);
        if (!(w > 0.0f)) return;
        const float rho = nb ? d.densB[j] : d.densR[j];
        const float pj = (nb ? d.presB[j] : d.presR[j]) / (rho * rho);
        const float coef = -CONTACT_VOL * vi * CONTACT_VOL * ContactVol(d, nb, j) * (pi + pj);
        fx += coef * gx; fy += coef * gy; fz += coef * gz;
    });
    d.forceC[i] = make_float4(fx, fy, fz, 0.f);
}
// ReduceRigidParticleForcesToBody(Contact) (cpu_backend.cpp:2089-2172): FP64, one block per body
__global__ void __launch_bounds__(256) KCReduce(ContactDev d) {
    const uint32_t body = blockIdx.x;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t w = d.byBodyOff[body] + threadIdx.x; w < d.byBodyOff[body + 1]; w += blockDim.x) {
        const uint32_t i = d.byBodyIdx[w];
        const float4 r = d.relW[i];
        const float4 F = d.forceC[i];
        acc[0] += F.x; acc[1] += F.y; acc[2] += F.z;
        acc[3] += (double)r.y * F.z - (double)r.z * F.y;
        acc[4] += (double)r.z * F.x - (double)r.x * F.z;
        acc[5] += (double)r.x * F.y - (double)r.y * F.x;
    }
    __shared__ double sm[6][8];
    for (int q = 0; q < 6; q++) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) sm[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; q++) {
            double t = 0.0;
            for (int w = 0; w < 8; w++) t += sm[q][w];
            d.ftC[6ull * body + q] = t;
        }
}
// RigidContactParticleVelocities (rigid_solver.cpp:462-506)
__global__ void KCVelocities(ContactDev d, Consts c) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nR) return;
    const uint32_t b = d.bodyR[i];
    const double* ft = d.ftC + 6ull * b;
    const float tx = (float)ft[3], ty = (float)ft[4], tz = (float)ft[5];
    const float* I = d.iw + 9ull * b;
    const float wx = I[0] * tx + I[1] * ty + I[2] * tz;
    const float wy = I[3] * tx + I[4] * ty + I[5] * tz;
    const float wz = I[6] * tx + I[7] * ty + I[8] * tz;
    const float4 r = d.relW[i];
    const float mi = (float)d.bodyState[(uint64_t)b * BODY_STRIDE_C + 22];
    const float dt = c.dt;
    d.velC[i] = make_float4(dt * (mi * (float)ft[0] + wy * r.z - wz * r.y), dt * (mi * (float)ft[1] + wz * r.x - wx * r.z),
                            dt * (mi * (float)ft[2] + wx * r.y - wy * r.x), 0.f);
}
// RigidContactPressureRelaxedJacobi (rigid_solver.cpp:581-600), skipped once the loop is done
__global__ void KCJacobi(ContactDev d) {
    if (d.st->doUpdate == 0u) return;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nc = *d.nContactB;
    if (t >= d.nR + nc) return;
    const bool boundary = t >= d.nR;
    const uint32_t i = boundary ? t - d.nR : t;
    const float dg = boundary ? d.diagB[i] : d.diagR[i];
    if (!(dg > 0.0f)) return;
    float* pres = boundary ? d.presB : d.presR;
    const float e = boundary ? d.errB[i] : d.errR[i];
    const float om = boundary ? d.omegaB[i] : d.omegaR[i];
    const float p = pres[i] + om * e / dg;
    if (!isfinite(p)) atomicOr(d.err, ERR_CONTACT_INVALID);
    pres[i] = fmaxf(0.0f, p);
}
// add the final contact loads to the body loads once (rigid_solver.cpp:786-795)
__global__ void KCAddLoads(ContactDev d) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 6u * d.nRB) d.bodyFT[t] += d.ftC[t];
}
__global__ void KCResetState(ContactDev d, float target, uint32_t maxIters) {
    ContactState& st = *d.st;
    st.errSum = 0.0; st.nContacts = 0; st.iters = 0; st.maxIters = maxIters; st.converged = 1u; st.doUpdate = 0u;
    st.avgErr = 0.0f; st.target = target;
}

// ---------------------------------------------------------------------------- launchers
static inline unsigned Gc(uint64_t n) { return (unsigned)((n + 255) / 256); }

void LaunchContactSetup(const ContactDev& d, uint64_t nEntriesRB, uint32_t nB, uint64_t* scanScratch,
                        uint64_t* ncTotal, cudaStream_t s) {
    cudaMemsetAsync(d.contactOfB, 0, (size_t)nB * sizeof(uint32_t), s);
    if (nEntriesRB) KCMark<<<Gc(nEntriesRB), 256, 0, s>>>(d, nEntriesRB);
    DeviceScan<uint64_t>(CFlagIn{d.contactOfB}, CFlagOut{d.contactOfB, d.localB}, nB, scanScratch, ncTotal, s);
}
void LaunchContactLists(const ContactDev& d, uint64_t nEntriesRB, uint32_t nc, uint64_t* scanScratch,
                        uint64_t* totalScratch, cudaStream_t s) {
    cudaMemsetAsync(d.curBR, 0, (size_t)std::max<uint32_t>(nc, 1) * sizeof(uint32_t), s);
    if (nEntriesRB) KCIdxRB<<<Gc(nEntriesRB), 256, 0, s>>>(d, nEntriesRB);
    if (nc) {
        DeviceScan<uint64_t>(CCountIn{d.curBR}, CCsrOut{d.offBR, d.curBR, nc}, nc, scanScratch, totalScratch, s);
        KCFillBR<<<Gc(d.nR), 256, 0, s>>>(d);
        KCSortBR<<<Gc(nc), 256, 0, s>>>(d);
    } else {
        cudaMemsetAsync(d.offBR, 0, sizeof(uint64_t), s);
    }
}
void LaunchContactPrepare(const ContactDev& d, const Consts& c, uint32_t nc, float target, uint32_t maxIters,
                          cudaStream_t s) {
    KCResetState<<<1, 1, 0, s>>>(d, target, maxIters);
    KCGeometry<<<Gc(std::max(d.nR, d.nRB)), 256, 0, s>>>(d);
    KCDensDiag<<<Gc((uint64_t)d.nR + nc), 256, 0, s>>>(d, c);
    cudaMemsetAsync(d.perBody, 0, (size_t)std::max<uint32_t>(d.nRB, 1) * sizeof(uint32_t), s);
    if (d.nRB) KCRelaxR<<<d.nRB, 256, 0, s>>>(d);
    if (nc) {
        KCRelaxB1<<<Gc(nc), 256, 0, s>>>(d);
        KCRelaxB2<<<Gc(nc), 256, 0, s>>>(d);
    }
}
void LaunchContactInitialError(const ContactDev& d, const Consts& c, uint32_t nc, const float4* velPredR,
                               cudaStream_t s) {
    // the error of the predicted motion becomes the source term: written into the err arrays,
    // which the caller then uses as source arrays (the reference swaps the vectors)
    KCError<<<Gc((uint64_t)d.nR + nc), 256, 0, s>>>(d, c, velPredR, d.srcR, d.srcB, d.errR, d.errB);
    KCErrorSum<<<1, 1024, 0, s>>>(d, 0, 0ull);
}
void LaunchContactIteration(const ContactDev& d, const Consts& c, uint32_t ncCap, unsigned long long cond,
                            cudaStream_t s) {
    const unsigned ge = Gc((uint64_t)d.nR + ncCap);
    KCForces<<<Gc(d.nR), 256, 0, s>>>(d, c);
    if (d.nRB) KCReduce<<<d.nRB, 256, 0, s>>>(d);
    KCVelocities<<<Gc(d.nR), 256, 0, s>>>(d, c);
    KCError<<<ge, 256, 0, s>>>(d, c, d.velC, d.srcR, d.srcB, d.errR, d.errB);
    KCErrorSum<<<1, 1024, 0, s>>>(d, 1, (cudaGraphConditionalHandle)cond);
    KCJacobi<<<ge, 256, 0, s>>>(d);
}
void LaunchContactAddLoads(const ContactDev& d, cudaStream_t s) {
    if (d.nRB) KCAddLoads<<<Gc(6ull * d.nRB), 256, 0, s>>>(d);
}

}  // namespace tsp
