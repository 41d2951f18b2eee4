// rigid_kernels.cu -- two-way rigid coupling through rigid (boundary-like) particles.
//
// Per-particle work is FP32 with the reference's operation order
// (source/simulation/CPU/backend/cpu_backend.cpp:2009-2063, sph_solver.cpp:1151-1223,1717-1778).
// Per-body work is FP64: the force/torque reduction over a body's particles (one block per
// body, fixed-order tree) and the predictor / integrator with Gram-Schmidt
// re-orthonormalisation of the rotation matrix (cpu_backend.cpp:2089-2303). The body state
// stays FP64 on the device; FP32 copies feed the particle updates.
//
// Body state layout (doubles, BODY_STRIDE per body):
//   0 cm[3] | 3 v[3] | 6 omega[3] | 9 L[3] | 12 A[9] row-major | 21 mass | 22 massInv |
//   23 Ibinv[9] row-major | 32 vPred[3] | 35 omegaPred[3] | 38 LPred[3]
#include "kernels.h"

namespace tsp {

constexpr int BODY_STRIDE = 48;

__global__ void KRigidUpdateParticles(RigidParticlesDev r, BodyDev b, int predicted, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= r.n) return;
    const uint32_t body = r.body[i];
    if (body >= b.n) { atomicOr(err, ERR_RIGID_ATTACH); return; }
    const double* s = b.state + (uint64_t)body * BODY_STRIDE;
    const float a00 = (float)s[12], a01 = (float)s[13], a02 = (float)s[14];
    const float a10 = (float)s[15], a11 = (float)s[16], a12 = (float)s[17];
    const float a20 = (float)s[18], a21 = (float)s[19], a22 = (float)s[20];
    const float4 l = r.rel[i];
    const float rx = fmaf(a00, l.x, fmaf(a01, l.y, a02 * l.z));
    const float ry = fmaf(a10, l.x, fmaf(a11, l.y, a12 * l.z));
    const float rz = fmaf(a20, l.x, fmaf(a21, l.y, a22 * l.z));
    const int vo = predicted ? 32 : 3, wo = predicted ? 35 : 6;
    const float vx = (float)s[vo], vy = (float)s[vo + 1], vz = (float)s[vo + 2];
    const float wx = (float)s[wo], wy = (float)s[wo + 1], wz = (float)s[wo + 2];
    const float4 v = make_float4(vx + wy * rz - wz * ry, vy + wz * rx - wx * rz, vz + wx * ry - wy * rx, l.w);
    if (predicted) {
        r.velPred[i] = v;
    } else {
        const float psi = r.pos[i].w;
        r.pos[i] = make_float4((float)s[0] + rx, (float)s[1] + ry, (float)s[2] + rz, psi);
        r.vel[i] = v;
    }
}

__global__ void KRigidClearAddGravity(BodyDev b, float gx, float gy, float gz) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= b.n) return;
    const double* s = b.state + (uint64_t)k * BODY_STRIDE;
    double* ft = b.forceTorque + 6ull * k;
    for (int q = 0; q < 6; q++) ft[q] = 0.0;
    const double m = s[21], mi = s[22];
    if (m <= 0.0 || mi <= 0.0) return;
    ft[0] += m * (double)gx; ft[1] += m * (double)gy; ft[2] += m * (double)gz;
}

// RF viscosity reaction force per rigid particle (sph_solver.cpp:1151-1223)
__global__ void KRigidViscous(Consts c, RigidParticlesDev r, FluidDev f, const uint64_t* __restrict__ off,
                              const uint32_t* __restrict__ list) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= r.n) return;
    const float4 pi = r.pos[i];
    const float4 vi = r.vel[i];
    const float facB = c.visFacB;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    for (uint64_t e = off[i]; e < off[i + 1]; e++) {
        const uint32_t j = list[e];
        const float4 pj = f.posP[j];
        const float4 vj = f.velRho[j];
        const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
        const float dvx = vj.x - vi.x, dvy = vj.y - vi.y, dvz = vj.z - vi.z;
        float gx, gy, gz;
        GradScalar(dx, dy, dz, c, gx, gy, gz);
        const float dot = fmaf(dvx, dx, fmaf(dvy, dy, dvz * dz));
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float a = (vi.w * dot) / (d2 + c.hEps);
        const float fc = -c.massF * facB * a;
        fx = fmaf(fc, gx, fx); fy = fmaf(fc, gy, fy); fz = fmaf(fc, gz, fz);
    }
    r.force[i] = make_float4(fx, fy, fz, 0.f);
}

// RF pressure reaction force, added to the viscous one (sph_solver.cpp:1717-1778)
__global__ void KRigidPressure(Consts c, RigidParticlesDev r, FluidDev f, const uint64_t* __restrict__ off,
                               const uint32_t* __restrict__ list) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= r.n) return;
    const float4 pi = r.pos[i];
    float fx = 0.f, fy = 0.f, fz = 0.f;
    for (uint64_t e = off[i]; e < off[i + 1]; e++) {
        const uint32_t j = list[e];
        const float4 pj = f.posP[j];
        const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
        float gx, gy, gz;
        GradScalar(dx, dy, dz, c, gx, gy, gz);
        const float fc = c.massF * c.accCoeffB * pi.w * pj.w;
        fx = fmaf(fc, gx, fx); fy = fmaf(fc, gy, fy); fz = fmaf(fc, gz, fz);
    }
    const float4 old = r.force[i];
    r.force[i] = make_float4(old.x + fx, old.y + fy, old.z + fz, 0.f);
}

// body force and torque, FP64 fixed-order block reduction (one block per body)
__global__ void __launch_bounds__(256) KRigidReduce(RigidParticlesDev r, BodyDev b) {
    const uint32_t body = blockIdx.x;
    const double* s = b.state + (uint64_t)body * BODY_STRIDE;
    const float a00 = (float)s[12], a01 = (float)s[13], a02 = (float)s[14];
    const float a10 = (float)s[15], a11 = (float)s[16], a12 = (float)s[17];
    const float a20 = (float)s[18], a21 = (float)s[19], a22 = (float)s[20];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t w = r.byBodyOff[body] + threadIdx.x; w < r.byBodyOff[body + 1]; w += blockDim.x) {
        const uint32_t i = r.byBodyIdx[w];
        const float4 l = r.rel[i];
        const float4 F = r.force[i];
        const float rx = fmaf(a00, l.x, fmaf(a01, l.y, a02 * l.z));
        const float ry = fmaf(a10, l.x, fmaf(a11, l.y, a12 * l.z));
        const float rz = fmaf(a20, l.x, fmaf(a21, l.y, a22 * l.z));
        const double fx = F.x, fy = F.y, fz = F.z;
        acc[0] += fx; acc[1] += fy; acc[2] += fz;
        acc[3] += (double)ry * fz - (double)rz * fy;
        acc[4] += (double)rz * fx - (double)rx * fz;
        acc[5] += (double)rx * fy - (double)ry * fx;
    }
    __shared__ double sm[6][8];
    for (int q = 0; q < 6; q++) {
        double v = acc[q];
        for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        if ((threadIdx.x & 31) == 0) sm[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double* ft = b.forceTorque + 6ull * body;
        for (int q = 0; q < 6; q++) {
            double t = 0.0;
            for (int w = 0; w < 8; w++) t += sm[q][w];
            ft[q] += t;
        }
    }
}

// PredictRigidBodies (cpu_backend.cpp:2174-2235) in FP64
__global__ void KRigidPredict(BodyDev b, double dt) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= b.n) return;
    double* s = b.state + (uint64_t)k * BODY_STRIDE;
    const double* ft = b.forceTorque + 6ull * k;
    for (int a = 0; a < 3; a++) {
        s[32 + a] = s[3 + a] + dt * ft[a] * s[22];
        s[38 + a] = s[9 + a] + dt * ft[3 + a];
    }
    const double* A = s + 12;
    const double* B = s + 23;
    double t[9], I[9];
    for (int rr = 0; rr < 3; rr++)
        for (int cc = 0; cc < 3; cc++)
            t[rr * 3 + cc] = A[rr * 3 + 0] * B[0 * 3 + cc] + A[rr * 3 + 1] * B[1 * 3 + cc] + A[rr * 3 + 2] * B[2 * 3 + cc];
    for (int rr = 0; rr < 3; rr++)
        for (int cc = 0; cc < 3; cc++)
            I[rr * 3 + cc] = t[rr * 3 + 0] * A[cc * 3 + 0] + t[rr * 3 + 1] * A[cc * 3 + 1] + t[rr * 3 + 2] * A[cc * 3 + 2];
    const double lx = s[38], ly = s[39], lz = s[40];
    s[35] = fma(I[0], lx, fma(I[1], ly, I[2] * lz));
    s[36] = fma(I[3], lx, fma(I[4], ly, I[5] * lz));
    s[37] = fma(I[6], lx, fma(I[7], ly, I[8] * lz));
}

__device__ __forceinline__ double Dot3d(double ax, double ay, double az, double bx, double by, double bz) {
    return fma(ax, bx, fma(ay, by, az * bz));
}
__device__ __forceinline__ bool Norm3d(double& x, double& y, double& z) {
    const double len = sqrt(Dot3d(x, y, z, x, y, z));
    if (!(len > 1e-12) || !isfinite(len)) return false;
    const double inv = 1.0 / len;
    x *= inv; y *= inv; z *= inv;
    return true;
}

// IntegrateRigidBodies (cpu_backend.cpp:2237-2303) in FP64
__global__ void KRigidIntegrate(BodyDev b, double dt, uint32_t* err) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= b.n) return;
    double* s = b.state + (uint64_t)k * BODY_STRIDE;
    for (int a = 0; a < 3; a++) { s[3 + a] = s[32 + a]; s[9 + a] = s[38 + a]; }
    for (int a = 0; a < 3; a++) s[a] += dt * s[3 + a];
    const double ox = s[35], oy = s[36], oz = s[37];
    s[6] = ox; s[7] = oy; s[8] = oz;
    double* A = s + 12;
    const double a00 = A[0], a01 = A[1], a02 = A[2], a10 = A[3], a11 = A[4], a12 = A[5], a20 = A[6], a21 = A[7],
                 a22 = A[8];
    A[0] += dt * (-oz * a10 + oy * a20); A[1] += dt * (-oz * a11 + oy * a21); A[2] += dt * (-oz * a12 + oy * a22);
    A[3] += dt * (oz * a00 - ox * a20);  A[4] += dt * (oz * a01 - ox * a21);  A[5] += dt * (oz * a02 - ox * a22);
    A[6] += dt * (-oy * a00 + ox * a10); A[7] += dt * (-oy * a01 + ox * a11); A[8] += dt * (-oy * a02 + ox * a12);
    double b1x = A[0], b1y = A[3], b1z = A[6];
    bool ok = Norm3d(b1x, b1y, b1z);
    double b2x = A[1], b2y = A[4], b2z = A[7];
    const double d12 = Dot3d(b1x, b1y, b1z, b2x, b2y, b2z);
    b2x -= d12 * b1x; b2y -= d12 * b1y; b2z -= d12 * b1z;
    ok = Norm3d(b2x, b2y, b2z) && ok;
    double b3x = A[2], b3y = A[5], b3z = A[8];
    const double d13 = Dot3d(b1x, b1y, b1z, b3x, b3y, b3z), d23 = Dot3d(b2x, b2y, b2z, b3x, b3y, b3z);
    b3x -= d13 * b1x + d23 * b2x; b3y -= d13 * b1y + d23 * b2y; b3z -= d13 * b1z + d23 * b2z;
    ok = Norm3d(b3x, b3y, b3z) && ok;
    if (!ok) { atomicOr(err, ERR_RIGID_ORIENT); return; }
    A[0] = b1x; A[1] = b2x; A[2] = b3x; A[3] = b1y; A[4] = b2y; A[5] = b3y; A[6] = b1z; A[7] = b2z; A[8] = b3z;
}

// rigid volumes per body in the body frame (builder.cpp:174-376 via ComputeRigidCoefficients):
// the host supplies each body's particles sorted by (z, y, x) cell and index, plus their
// cells; a thread walks the (2 reach + 1)^2 rows of its cell exactly like the reference
struct RigidCellRow {
    int x, y, z;
};
__device__ __forceinline__ bool CellLess(const int4& a, int z, int y, int x) {
    if (a.z != z) return a.z < z;
    if (a.y != y) return a.y < y;
    return a.x < x;
}
__global__ void KRigidVolumes(Consts c, const float4* __restrict__ rel, const uint32_t* __restrict__ byBodyOff,
                              const uint32_t* __restrict__ sortedIdx, const int4* __restrict__ sortedCell,
                              const uint32_t* __restrict__ bodyOfSorted, uint32_t nR, int reach, float defVol,
                              float defPsi, float rho0, float* __restrict__ vol, float* __restrict__ psi) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nR) return;
    const uint32_t body = bodyOfSorted[s];
    const uint32_t lo = byBodyOff[body], hi = byBodyOff[body + 1];
    const uint32_t i = sortedIdx[s];
    const int4 base = sortedCell[s];
    const float4 p = rel[i];
    float sum = 0.0f;
    for (int dz = -reach; dz <= reach; dz++)
        for (int dy = -reach; dy <= reach; dy++) {
            // lower bound of (z, y, x - reach), upper bound of (z, y, x + reach)
            uint32_t a = lo, e = hi;
            while (a < e) { const uint32_t m = (a + e) >> 1; if (CellLess(sortedCell[m], base.z + dz, base.y + dy, base.x - reach)) a = m + 1; else e = m; }
            uint32_t b = a, e2 = hi;
            while (b < e2) {
                const uint32_t m = (b + e2) >> 1;
                const int4 cm = sortedCell[m];
                const bool le = !CellLess(make_int4(base.x + reach, base.y + dy, base.z + dz, 0), cm.z, cm.y, cm.x);
                if (le) b = m + 1; else e2 = m;
            }
            for (uint32_t q = a; q < b; q++) {
                const float4 o = rel[sortedIdx[q]];
                sum += BoundaryWeight(p.x - o.x, p.y - o.y, p.z - o.z, c);
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

void LaunchRigidUpdateParticles(const RigidParticlesDev& r, const BodyDev& b, bool predicted, uint32_t* err,
                                cudaStream_t s) {
    if (r.n) KRigidUpdateParticles<<<(r.n + 255) / 256, 256, 0, s>>>(r, b, predicted ? 1 : 0, err);
}
void LaunchRigidClearAddGravity(const BodyDev& b, float gx, float gy, float gz, cudaStream_t s) {
    if (b.n) KRigidClearAddGravity<<<(b.n + 63) / 64, 64, 0, s>>>(b, gx, gy, gz);
}
void LaunchRigidViscousForces(const Consts& c, const RigidParticlesDev& r, const FluidDev& f, const uint64_t* offRF,
                              const uint32_t* listRF, cudaStream_t s) {
    if (r.n) KRigidViscous<<<(r.n + 127) / 128, 128, 0, s>>>(c, r, f, offRF, listRF);
}
void LaunchRigidPressureForces(const Consts& c, const RigidParticlesDev& r, const FluidDev& f, const uint64_t* offRF,
                               const uint32_t* listRF, cudaStream_t s) {
    if (r.n) KRigidPressure<<<(r.n + 127) / 128, 128, 0, s>>>(c, r, f, offRF, listRF);
}
void LaunchRigidReduce(const RigidParticlesDev& r, const BodyDev& b, cudaStream_t s) {
    if (b.n) KRigidReduce<<<b.n, 256, 0, s>>>(r, b);
}
void LaunchRigidPredict(const BodyDev& b, float dt, cudaStream_t s) {
    if (b.n) KRigidPredict<<<(b.n + 63) / 64, 64, 0, s>>>(b, (double)dt);
}
void LaunchRigidIntegrate(const BodyDev& b, float dt, uint32_t* err, cudaStream_t s) {
    if (b.n) KRigidIntegrate<<<(b.n + 63) / 64, 64, 0, s>>>(b, (double)dt, err);
}
void LaunchRigidVolumesSorted(const Consts& c, const float4* rel, const uint32_t* byBodyOff, const uint32_t* sortedIdx,
                              const int4* sortedCell, const uint32_t* bodyOfSorted, uint32_t nR, int reach,
                              float defaultVol, float defaultPsi, float restDensity, float* volOut, float* psiOut,
                              cudaStream_t s) {
    if (nR)
        KRigidVolumes<<<(nR + 127) / 128, 128, 0, s>>>(c, rel, byBodyOff, sortedIdx, sortedCell, bodyOfSorted, nR,
                                                       reach, defaultVol, defaultPsi, restDensity, volOut, psiOut);
}

}  // namespace tsp
