// tsp_oracle.cpp -- CPU restatement of the reference IISPH step (TEST INFRASTRUCTURE ONLY).
//
// This file is the parity oracle of the B200 backend. It is never linked into, loaded by or
// called from the product library; only tests/ and __graft_entry__.smoke() use it, to check
// results, and bench.py's CPU-baseline leg, which times it beside the GPU.
//
// It restates, scalar per particle and templated on the real type (float = the reference's
// FP32 arithmetic, double = the "FP64 run" the reference does not have), the CPU path of
// TurboSPHarticles:
//   cell frame ............ source/simulation/CPU/backend/neighbor_search.cpp:1902-2006
//   Morton cell IDs ....... neighbor_search.cpp:157-162 (FloorToInt), 2020-2070
//   key bits / radix sort . neighbor_search.cpp:403-564 (stable; restated as std::stable_sort
//                            on the clamped key, which yields the identical permutation)
//   re-order .............. neighbor_search.cpp:1624-1848
//   cell tables ........... neighbor_search.cpp:296-393, Construct 613-815
//   queries ............... neighbor_search.cpp:1033-1612 (distance rule
//                            fma(dx,dx,fma(dy,dy,dz*dz)) <= r^2, FF includes self,
//                            RR excludes the own body)
//   SPH kernels ........... source/simulation/CPU/backend/sph_solver.cpp:686-2089 and the
//                            kernel math of source/simulation/CPU/simd.h:279-435
//   rigid helpers ......... source/simulation/CPU/backend/cpu_backend.cpp:2001-2303
//   boundary volumes ...... source/simulation/scene/builder.cpp:36-79, 174-376
//   SELL32 encoding ....... the reference GPU rule, GPU/backend/neighbor_search_kernels.cu:86-250
//                            and neighbor_search.cu:369-468 (offsets per format)
//
// Row order: the reference CPU emits each neighbor row in the scan order of its SIMD-chunk
// query boxes. The oracle emits rows in ascending neighbor index (the canonical order of the
// B200 backend); neighbor sets are identical, per-pair arithmetic is identical, and only the
// order of the per-particle sums differs from the reference binary. The reference's
// "dict chunk" path (sph_solver.cpp:789-811 etc.) is an algebraic rearrangement of the same
// sums and is not restated.
//
// Parity pins: tests/test_oracle_kats.py checks this oracle against the known answers of the
// reference's own unit tests (tests/unit/sph_pressure.cpp, sph_kernels.cpp, sph_density.cpp,
// sph_integration.cpp, neighbor_search.cpp). The reference CPU backend itself cannot be built
// here (it needs oneTBB, xsimd, glm and Boost, none of which is installed).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>
#include <unordered_map>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/tsp_b200.h"

namespace orc {

static constexpr uint32_t EMPTY_32 = 0xffffffffu;
static constexpr uint64_t EMPTY_64 = 0xffffffffffffffffull;
static constexpr uint32_t SELL_W = 32u;

template <typename T> static inline T fmaT(T a, T b, T c) { return std::fma(a, b, c); }

// neighbor_search.cpp:157-162
template <typename T> static inline int FloorToInt(T v) {
    int i = static_cast<int>(v);
    return (v < static_cast<T>(i)) ? (i - 1) : i;
}

// neighbor_search.cpp:2057-2070
static inline uint64_t Spread21(uint32_t v) {
    uint64_t x = static_cast<uint64_t>(v & 0x1fffffu);
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

struct Frame {
    int32_t ox = 0, oy = 0, oz = 0;
    uint32_t nx = 0, ny = 0, nz = 0;
};

static inline bool InFrame(const Frame& f, int cx, int cy, int cz) {
    const int lx = cx - f.ox, ly = cy - f.oy, lz = cz - f.oz;
    return lx >= 0 && lx < (int)f.nx && ly >= 0 && ly < (int)f.ny && lz >= 0 && lz < (int)f.nz;
}
static inline uint64_t Morton(const Frame& f, int cx, int cy, int cz) {
    return Spread21((uint32_t)(cx - f.ox)) | (Spread21((uint32_t)(cy - f.oy)) << 1) |
           (Spread21((uint32_t)(cz - f.oz)) << 2);
}
// neighbor_search.cpp:403-413
static inline uint32_t KeyBits(const Frame& f) {
    const uint32_t m = std::max(f.nx, std::max(f.ny, f.nz));
    uint32_t axisBits = 1;
    if (m >= 2) { axisBits = 32u - (uint32_t)__builtin_clz(m - 1u); }
    return 3u * axisBits + 1u;
}

// simd.h:279-309 (masked: strictly inside the support)
template <typename T>
static inline T KernelWeight(T dx, T dy, T dz, T sizeInv, T radSqu, T alpha) {
    const T distSqu = fmaT(dx, dx, fmaT(dy, dy, dz * dz));
    if (!(distSqu < radSqu)) return T(0);
    const T dist = std::sqrt(distSqu);
    const T q = dist * sizeInv;
    const T t1 = std::max(T(1) - q, T(0));
    const T t2 = std::max(T(2) - q, T(0));
    const T t1_2 = t1 * t1, t2_2 = t2 * t2;
    const T t1_3 = t1_2 * t1, t2_3 = t2_2 * t2;
    return alpha * fmaT(T(-4), t1_3, t2_3);
}

template <typename T> struct KConst {  // simd.h:350-370
    T size, twoSize, innerSlope, innerOffset, outerScale;
};
template <typename T> static KConst<T> MakeKConst(T sizeInv, T alpha) {
    KConst<T> k;
    k.size = T(1) / sizeInv;
    k.twoSize = T(2) / sizeInv;
    k.innerSlope = T(9) * alpha * sizeInv * sizeInv * sizeInv;
    k.innerOffset = T(-12) * alpha * sizeInv * sizeInv;
    k.outerScale = T(-3) * alpha * sizeInv * sizeInv * sizeInv;
    return k;
}
// simd.h:374-388
template <typename T> static inline T GradFac(T distSqu, const KConst<T>& k) {
    const T dist = std::sqrt(distSqu);
    const T inner = fmaT(k.innerSlope, dist, k.innerOffset);
    const T t2 = std::max(k.twoSize - dist, T(0));
    const T outer = (t2 * t2) * (k.outerScale / dist);
    return (dist < k.size) ? inner : outer;
}
// simd.h:311-347 (scalar gradient used by the rigid force accumulations)
template <typename T>
static inline void GradScalar(T dx, T dy, T dz, T sizeInv, T radSqu, T alpha, T& gx, T& gy, T& gz) {
    const T distSqu = fmaT(dx, dx, fmaT(dy, dy, dz * dz));
    if (distSqu >= radSqu) { gx = gy = gz = T(0); return; }
    const T dist = std::sqrt(distSqu);
    const T q = dist * sizeInv;
    T c;
    if (q < T(1)) c = alpha * sizeInv * sizeInv * fmaT(T(9), q, T(-12));
    else {
        const T t2 = std::max(T(2) - q, T(0));
        c = alpha * (T(-3) * t2 * t2) * (sizeInv / dist);
    }
    gx = c * dx; gy = c * dy; gz = c * dz;
}
// builder.cpp:49-79
template <typename T> static inline T BoundaryWeight(T dx, T dy, T dz, T sizeInv, T radSqu, T alpha) {
    const T distSqu = fmaT(dx, dx, fmaT(dy, dy, dz * dz));
    if (distSqu >= radSqu) return T(0);
    if (distSqu < T(1e-7f)) return T(4) * alpha;
    const T dist = std::sqrt(distSqu);
    const T q = dist * sizeInv;
    const T t1 = std::max(T(1) - q, T(0)), t2 = std::max(T(2) - q, T(0));
    const T t1_2 = t1 * t1, t2_2 = t2 * t2;
    const T t1_3 = t1_2 * t1, t2_3 = t2_2 * t2;
    return alpha * (t2_3 - T(4) * t1_3);
}

struct CSR {
    std::vector<uint64_t> off;
    std::vector<uint32_t> idx;
    uint64_t total() const { return off.empty() ? 0 : off.back(); }
};

struct Sell32 {
    std::vector<uint16_t> pitch;
    std::vector<uint8_t> format;  // 0 = Delta16x2, 1 = Abs32 (GPU/backend/common.cuh:17-21)
    std::vector<uint32_t> base, base2;
    std::vector<uint64_t> offset;
    std::vector<uint16_t> counts;
    std::vector<uint16_t> w16;
    std::vector<uint32_t> w32;
};

// GPU/backend/neighbor_search_kernels.cu:86-97
static inline void HomeWindow(uint32_t chunk, uint32_t& lo, uint32_t& hi) {
    constexpr uint32_t reach = (0x8000u - SELL_W) / 2u;
    constexpr uint32_t hiOff = SELL_W - 1u + reach;
    const uint32_t b = chunk * SELL_W;
    lo = (b > reach) ? (b - reach) : 0u;
    hi = (b < 0xffffffffu - hiOff) ? (b + hiOff) : 0xffffffffu;
}

// CommitChunkCompressionMeta (neighbor_search_kernels.cu:101-191) + offsets per format
// (neighbor_search.cu:392-425) + StoreNeighbor_CompressedSell32 (:193-247), applied to rows
static void EncodeSell32(const CSR& rows, uint32_t N, bool splitFar, Sell32& s) {
    const uint32_t nChunks = N == 0 ? 0 : (N - 1) / SELL_W + 1;
    s.pitch.assign(nChunks, 0); s.format.assign(nChunks, 1); s.base.assign(nChunks, 0);
    s.base2.assign(nChunks, 0); s.offset.assign(nChunks, 0); s.counts.assign(N, 0);
    for (uint32_t i = 0; i < N; i++) s.counts[i] = (uint16_t)(rows.off[i + 1] - rows.off[i]);
    for (uint32_t c = 0; c < nChunks; c++) {
        uint32_t pitch = 0, minRef = 0xffffffffu, maxRef = 0, homeMin = 0xffffffffu, farLoMax = 0,
                 farHiMin = 0xffffffffu, lo, hi;
        HomeWindow(c, lo, hi);
        for (uint32_t i = c * SELL_W; i < std::min(N, (c + 1) * SELL_W); i++) {
            pitch = std::max<uint32_t>(pitch, (uint16_t)(rows.off[i + 1] - rows.off[i]));
            for (uint64_t e = rows.off[i]; e < rows.off[i + 1]; e++) {
                const uint32_t j = rows.idx[e];
                minRef = std::min(minRef, j); maxRef = std::max(maxRef, j);
                if (j < lo) farLoMax = std::max(farLoMax, j);
                else if (j > hi) farHiMin = std::min(farHiMin, j);
                else homeMin = std::min(homeMin, j);
            }
        }
        s.pitch[c] = (uint16_t)pitch;
        if (pitch == 0) { s.base[c] = 0; s.format[c] = 1; continue; }
        const uint32_t span = (maxRef >= minRef) ? (maxRef - minRef) : 0xffffffffu;
        if (maxRef >= minRef && span <= 0xffffu) {
            s.base[c] = minRef; s.base2[c] = minRef + 0x8000u; s.format[c] = 0; continue;
        }
        if (splitFar) {
            const bool hasLo = minRef < lo, hasHi = maxRef > hi;
            const uint32_t farMin = hasLo ? minRef : farHiMin;
            const uint32_t farMax = hasLo ? farLoMax : maxRef;
            if (hasLo != hasHi && homeMin <= hi && farMax - farMin <= 0x7fffu) {
                s.base[c] = homeMin; s.base2[c] = farMin; s.format[c] = 0; continue;
            }
        }
        s.base[c] = minRef; s.format[c] = 1;
    }
    if (!splitFar)  // FB/FR: the second base sits 0x8000 above the first (:941-943)
        for (uint32_t c = 0; c < nChunks; c++) s.base2[c] = s.base[c] + 0x8000u;
    uint64_t tot[2] = {0, 0};
    for (uint32_t c = 0; c < nChunks; c++) {
        s.offset[c] = tot[s.format[c]];
        tot[s.format[c]] += (uint64_t)s.pitch[c] * SELL_W;
    }
    s.w16.assign(tot[0], 0); s.w32.assign(tot[1], 0);
    for (uint32_t i = 0; i < N; i++) {
        const uint32_t c = i / SELL_W, lane = i % SELL_W;
        uint32_t k = 0;
        for (uint64_t e = rows.off[i]; e < rows.off[i + 1]; e++, k++) {
            const uint32_t j = rows.idx[e];
            const uint64_t lin = s.offset[c] + (uint64_t)k * SELL_W + lane;
            if (s.format[c] == 0) {
                const bool first = (j >= s.base[c]) && (j - s.base[c] <= 0x7fffu);
                s.w16[lin] = first ? (uint16_t)(j - s.base[c]) : (uint16_t)(0x8000u | (j - s.base2[c]));
            } else {
                s.w32[lin] = j;
            }
        }
    }
}

template <typename T> struct Oracle {
    tsp_params prm{};
    float domMin[3] = {0, 0, 0}, domMax[3] = {0, 0, 0};
    uint32_t NF = 0, NB = 0, NR = 0, NRB = 0;
    uint64_t step = 0; double time = 0;
    // fluid
    std::vector<uint64_t> idF;
    std::vector<T> xF, yF, zF, vxF, vyF, vzF, vpxF, vpyF, vpzF, axF, ayF, azF, srcF, diagF, presF, densF;
    // boundary
    std::vector<uint64_t> idB;
    std::vector<T> xB, yB, zB, volB, psiB;
    // rigid particles
    std::vector<uint64_t> idR;
    std::vector<uint32_t> bodyR;
    std::vector<T> xRel, yRel, zRel, volR, psiR, xR, yR, zR, vxR, vyR, vzR, vpxR, vpyR, vpzR, fxR, fyR, fzR;
    // rigid bodies
    std::vector<uint64_t> idRB;
    std::vector<uint32_t> cntRB;
    std::vector<T> cmx, cmy, cmz, vx, vy, vz, wx, wy, wz, Lx, Ly, Lz, A[9], mass, massInv, Ib[9];
    std::vector<T> vpx, vpy, vpz, wpx, wpy, wpz, Lpx, Lpy, Lpz, Fx, Fy, Fz, Tx, Ty, Tz;
    std::vector<uint32_t> byBodyOff, byBodyIdx;
    // neighbor search state
    Frame frame; bool frameValid = false; uint32_t frameRebuilds = 0;
    T cellSize = 0, cellSizeInv = 0; uint32_t reach = 1;
    std::vector<uint64_t> cidF, cidB, cidR;  // F, B: sorted order; R: storage order
    std::vector<uint32_t> permF, permB, permR;
    std::vector<uint64_t> uniqF, uniqB, uniqR;
    std::vector<uint32_t> startF, startB, startR;
    CSR rows[6];
    // solver state
    uint32_t iters = 0; T avgRaw = 0, avgPos = 0, avgAbs = 0; double eRaw = 0, ePos = 0, eAbs = 0;
    // rigid contact solver state (rigid_solver.cpp)
    std::vector<uint32_t> cLocalB;                 // contact boundary particle -> boundary index
    std::vector<uint64_t> cOffRB, cOffBR;
    std::vector<uint32_t> cIdxRB, cIdxBR;          // RB: contact indices; BR: rigid indices
    std::vector<T> cRelWx, cRelWy, cRelWz, cIw[9];
    std::vector<T> cDensR, cDiagR, cPresR, cSrcR, cErrR, cOmegaR, cFxR, cFyR, cFzR, cVxR, cVyR, cVzR;
    std::vector<T> cDensB, cDiagB, cPresB, cSrcB, cErrB, cOmegaB;
    std::vector<T> cFx, cFy, cFz, cTx, cTy, cTz;   // per body contact force / torque
    uint32_t contactIters = 0; T contactAvgErr = 0; bool contactConverged = false; uint64_t contactCount = 0;

    T alpha() const {
        if (prm.cubicSplineAlphaOverride > 0.0f) return (T)prm.cubicSplineAlphaOverride;
        // solver_constants.h:287-303: FP64 derivation, FP32 result for the float instance
        const double h = (double)prm.particleSizeF, inv = 1.0 / h;
        const double a = inv * inv * inv / (4.0 * 3.14159265358979323846);
        return std::is_same<T, float>::value ? (T)(float)a : (T)a;
    }
    T sizeInv() const {
        const double inv = 1.0 / (double)prm.particleSizeF;
        return std::is_same<T, float>::value ? (T)(float)inv : (T)inv;
    }
    T sizeSqu() const {
        const double h = (double)prm.particleSizeF;
        return std::is_same<T, float>::value ? (T)(float)(h * h) : (T)(h * h);
    }
    T rhoSquInv() const {
        const double r = (double)prm.restDensity;
        return std::is_same<T, float>::value ? (T)(float)(1.0 / (r * r)) : (T)(1.0 / (r * r));
    }

    // ------------------------------------------------------------------ frame (1902-2006)
    bool InsideDomain(T x, T y, T z) const {
        if (domMax[0] <= domMin[0] || domMax[1] <= domMin[1] || domMax[2] <= domMin[2]) return true;
        return x >= domMin[0] && x <= domMax[0] && y >= domMin[1] && y <= domMax[1] && z >= domMin[2] &&
               z <= domMax[2];
    }
    void SetCellSize() {  // neighbor_search.cpp:1645-1659
        const float cs = prm.kernelRadius * prm.gridCellSizeRatio;
        const bool zero = std::fabs(cs) <= 1e-7f;  // Base::ApproxEqu (source/base/helpers.h:21-24)
        const float span = zero ? 0.0f : (prm.kernelRadius / cs);
        const uint32_t r = zero ? 1u : std::max<uint32_t>(1u, (uint32_t)std::ceil(std::max(0.0f, span - 1e-6f)));
        const bool changed = std::fabs((float)cellSize - cs) > 1e-7f || reach != r;
        cellSize = (T)cs;
        cellSizeInv = zero ? T(0) : (std::is_same<T, float>::value ? (T)(1.0f / cs) : T(1) / (T)cs);
        reach = r;
        if (changed) frameValid = false;
    }
    void UpdateFrame() {
        if (NF == 0 && NB == 0 && NR == 0) { frame = {}; frameValid = false; return; }
        bool rebuild = !frameValid;
        if (!rebuild) {
            const int m = (int)reach;
            const int x0 = frame.ox + m, y0 = frame.oy + m, z0 = frame.oz + m;
            const int x1 = frame.ox + (int)frame.nx - 1 - m, y1 = frame.oy + (int)frame.ny - 1 - m,
                      z1 = frame.oz + (int)frame.nz - 1 - m;
            auto exceeded = [&](const std::vector<T>& X, const std::vector<T>& Y, const std::vector<T>& Z, uint32_t N) {
                for (uint32_t i = 0; i < N; i++) {
                    if (!InsideDomain(X[i], Y[i], Z[i])) continue;
                    const int cx = FloorToInt(X[i] * cellSizeInv), cy = FloorToInt(Y[i] * cellSizeInv),
                              cz = FloorToInt(Z[i] * cellSizeInv);
                    if (cx < x0 || cx > x1 || cy < y0 || cy > y1 || cz < z0 || cz > z1) return true;
                }
                return false;
            };
            rebuild = x0 > x1 || y0 > y1 || z0 > z1 || exceeded(xF, yF, zF, NF) || exceeded(xB, yB, zB, NB) ||
                      exceeded(xR, yR, zR, NR);
        }
        if (!rebuild) return;
        T mn[3] = {std::numeric_limits<T>::max(), std::numeric_limits<T>::max(), std::numeric_limits<T>::max()};
        T mx[3] = {std::numeric_limits<T>::lowest(), std::numeric_limits<T>::lowest(), std::numeric_limits<T>::lowest()};
        auto acc = [&](const std::vector<T>& X, const std::vector<T>& Y, const std::vector<T>& Z, uint32_t N) {
            for (uint32_t i = 0; i < N; i++) {
                mn[0] = std::min(mn[0], X[i]); mn[1] = std::min(mn[1], Y[i]); mn[2] = std::min(mn[2], Z[i]);
                mx[0] = std::max(mx[0], X[i]); mx[1] = std::max(mx[1], Y[i]); mx[2] = std::max(mx[2], Z[i]);
            }
        };
        acc(xF, yF, zF, NF); acc(xB, yB, zB, NB); acc(xR, yR, zR, NR);
        if (!(domMax[0] <= domMin[0] || domMax[1] <= domMin[1] || domMax[2] <= domMin[2]))
            for (int a = 0; a < 3; a++) {
                mn[a] = std::clamp(mn[a], (T)domMin[a], (T)domMax[a]);
                mx[a] = std::clamp(mx[a], (T)domMin[a], (T)domMax[a]);
            }
        const int64_t margin = (int64_t)reach + 8;
        int64_t o[3], e[3];
        for (int a = 0; a < 3; a++) {
            o[a] = (int64_t)FloorToInt(mn[a] * cellSizeInv) - margin;
            e[a] = (int64_t)FloorToInt(mx[a] * cellSizeInv) + margin;
            if (o[a] > e[a] || o[a] < INT32_MIN || e[a] > INT32_MAX || e[a] - o[a] + 1 > (int64_t)(1u << 21))
                throw std::runtime_error("cell frame exceeds the supported range");
        }
        frame.ox = (int32_t)o[0]; frame.oy = (int32_t)o[1]; frame.oz = (int32_t)o[2];
        frame.nx = (uint32_t)(e[0] - o[0] + 1); frame.ny = (uint32_t)(e[1] - o[1] + 1); frame.nz = (uint32_t)(e[2] - o[2] + 1);
        frameValid = true;
        frameRebuilds++;
    }
    uint64_t CellId(T x, T y, T z) const {
        const int cx = FloorToInt(x * cellSizeInv), cy = FloorToInt(y * cellSizeInv), cz = FloorToInt(z * cellSizeInv);
        return InFrame(frame, cx, cy, cz) ? Morton(frame, cx, cy, cz) : EMPTY_64;
    }
    // SortParticleOrderByCellId (neighbor_search.cpp:419-564): stable on min(id, emptyKey)
    void StableSort(std::vector<uint64_t>& ids, std::vector<uint32_t>& perm) const {
        const uint64_t emptyKey = 1ull << (KeyBits(frame) - 1u);
        const uint32_t N = (uint32_t)ids.size();
        perm.resize(N);
        for (uint32_t i = 0; i < N; i++) perm[i] = i;
        std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) {
            return std::min(ids[a], emptyKey) < std::min(ids[b], emptyKey);
        });
        std::vector<uint64_t> s(N);
        for (uint32_t i = 0; i < N; i++) s[i] = ids[perm[i]];
        ids.swap(s);
    }
    template <typename V> static void Permute(V& v, const std::vector<uint32_t>& perm) {
        if (v.empty()) return;
        V s(v.size());
        for (size_t i = 0; i < perm.size(); i++) s[i] = v[perm[i]];
        v.swap(s);
    }
    static void CellTable(const std::vector<uint64_t>& ids, std::vector<uint64_t>& uniq, std::vector<uint32_t>& start) {
        uniq.clear(); start.clear();
        const uint32_t N = (uint32_t)ids.size();
        for (uint32_t i = 0; i < N; i++)
            if (i == 0 || ids[i] != ids[i - 1]) { uniq.push_back(ids[i]); start.push_back(i); }
        if (N > 0) start.push_back(N);
    }
    // ReOrderParticleData (neighbor_search.cpp:1624-1848) + Construct (613-815)
    void ReorderAndConstruct(bool permuteAll) {
        SetCellSize();
        UpdateFrame();
        // fluid: IDs, pos, vel always; pressure on warm start; everything for a standalone search
        cidF.resize(NF);
        for (uint32_t i = 0; i < NF; i++) cidF[i] = CellId(xF[i], yF[i], zF[i]);
        StableSort(cidF, permF);
        Permute(idF, permF);
        Permute(xF, permF); Permute(yF, permF); Permute(zF, permF);
        Permute(vxF, permF); Permute(vyF, permF); Permute(vzF, permF);
        if (permuteAll) {
            Permute(vpxF, permF); Permute(vpyF, permF); Permute(vpzF, permF);
            Permute(axF, permF); Permute(ayF, permF); Permute(azF, permF);
            Permute(srcF, permF); Permute(diagF, permF); Permute(presF, permF); Permute(densF, permF);
        } else if (prm.jacobiWarmStart > 0.0f) {
            Permute(presF, permF);
        }
        // boundary: sorted only when its cell IDs are not already non-decreasing
        cidB.resize(NB);
        for (uint32_t i = 0; i < NB; i++) cidB[i] = CellId(xB[i], yB[i], zB[i]);
        bool sorted = true;
        for (uint32_t i = 1; i < NB && sorted; i++) sorted = cidB[i - 1] <= cidB[i];
        if (!sorted) {
            StableSort(cidB, permB);
            Permute(idB, permB); Permute(xB, permB); Permute(yB, permB); Permute(zB, permB);
            Permute(volB, permB); Permute(psiB, permB);
        } else {
            permB.resize(NB);
            for (uint32_t i = 0; i < NB; i++) permB[i] = i;
        }
        // rigid: an index permutation only, rigid storage order is preserved (747-774)
        cidR.resize(NR);
        for (uint32_t i = 0; i < NR; i++) cidR[i] = CellId(xR[i], yR[i], zR[i]);
        std::vector<uint64_t> sortedR = cidR;
        StableSort(sortedR, permR);
        CellTable(cidF, uniqF, startF);
        CellTable(cidB, uniqB, startB);
        CellTable(sortedR, uniqR, startR);
    }
    static uint32_t FindCell(const std::vector<uint64_t>& uniq, uint64_t id) {
        auto it = std::lower_bound(uniq.begin(), uniq.end(), id);
        if (it == uniq.end() || *it != id) return EMPTY_32;
        return (uint32_t)(it - uniq.begin());
    }
    // stencil cells of a particle in ascending cell ID (= ascending particle index)
    void Stencil(T x, T y, T z, std::vector<uint64_t>& cells) const {
        cells.clear();
        const int cx = FloorToInt(x * cellSizeInv), cy = FloorToInt(y * cellSizeInv), cz = FloorToInt(z * cellSizeInv);
        if (!InFrame(frame, cx, cy, cz)) return;
        const int r = (int)reach;
        for (int oz = cz - r; oz <= cz + r; oz++)
            for (int oy = cy - r; oy <= cy + r; oy++)
                for (int ox = cx - r; ox <= cx + r; ox++)
                    if (InFrame(frame, ox, oy, oz)) cells.push_back(Morton(frame, ox, oy, oz));
        std::sort(cells.begin(), cells.end());
    }
    // Query_Count + Query_Fill (neighbor_search.cpp:1033-1612), rows in ascending index
    void Query() {
        const T r2 = (T)prm.kernelRadiusSqu;
        for (int l = 0; l < 6; l++) { rows[l].off.assign(1, 0); rows[l].idx.clear(); }
        std::vector<std::vector<uint32_t>> rF[3], rR[3];
        for (int l = 0; l < 3; l++) { rF[l].assign(NF, {}); rR[l].assign(NR, {}); }
        auto hit = [&](T xi, T yi, T zi, T xj, T yj, T zj) {
            const T dx = xi - xj, dy = yi - yj, dz = zi - zj;
            return fmaT(dx, dx, fmaT(dy, dy, dz * dz)) <= r2;
        };
#pragma omp parallel
        {
            std::vector<uint64_t> cells;
#pragma omp for schedule(dynamic, 256)
            for (int64_t ii = 0; ii < (int64_t)NF; ii++) {
                const uint32_t i = (uint32_t)ii;
                if (cidF[i] == EMPTY_64) continue;  // left the frame: queries no cells
                Stencil(xF[i], yF[i], zF[i], cells);
                for (uint64_t c : cells) {
                    uint32_t k = FindCell(uniqF, c);
                    if (k != EMPTY_32)
                        for (uint32_t j = startF[k]; j < startF[k + 1]; j++)
                            if (hit(xF[i], yF[i], zF[i], xF[j], yF[j], zF[j])) rF[0][i].push_back(j);
                    k = FindCell(uniqB, c);
                    if (k != EMPTY_32)
                        for (uint32_t j = startB[k]; j < startB[k + 1]; j++)
                            if (hit(xF[i], yF[i], zF[i], xB[j], yB[j], zB[j])) rF[1][i].push_back(j);
                    k = FindCell(uniqR, c);
                    if (k != EMPTY_32)
                        for (uint32_t s = startR[k]; s < startR[k + 1]; s++) {
                            const uint32_t j = permR[s];
                            if (hit(xF[i], yF[i], zF[i], xR[j], yR[j], zR[j])) rF[2][i].push_back(j);
                        }
                }
                std::sort(rF[2][i].begin(), rF[2][i].end());
            }
#pragma omp for schedule(dynamic, 64)
            for (int64_t ii = 0; ii < (int64_t)NR; ii++) {
                const uint32_t i = (uint32_t)ii;
                Stencil(xR[i], yR[i], zR[i], cells);
                for (uint64_t c : cells) {
                    uint32_t k = FindCell(uniqF, c);
                    if (k != EMPTY_32)
                        for (uint32_t j = startF[k]; j < startF[k + 1]; j++)
                            if (hit(xR[i], yR[i], zR[i], xF[j], yF[j], zF[j])) rR[0][i].push_back(j);
                    k = FindCell(uniqB, c);
                    if (k != EMPTY_32)
                        for (uint32_t j = startB[k]; j < startB[k + 1]; j++)
                            if (hit(xR[i], yR[i], zR[i], xB[j], yB[j], zB[j])) rR[1][i].push_back(j);
                    k = FindCell(uniqR, c);
                    if (k != EMPTY_32)
                        for (uint32_t s = startR[k]; s < startR[k + 1]; s++) {
                            const uint32_t j = permR[s];
                            if (j == i || bodyR[j] == bodyR[i]) continue;
                            if (hit(xR[i], yR[i], zR[i], xR[j], yR[j], zR[j])) rR[2][i].push_back(j);
                        }
                }
                std::sort(rR[2][i].begin(), rR[2][i].end());
            }
        }
        for (int l = 0; l < 3; l++) {
            for (uint32_t i = 0; i < NF; i++) {
                if (rF[l][i].size() > 0xffffu) throw std::runtime_error("neighbor count exceeds uint16");
                rows[l].idx.insert(rows[l].idx.end(), rF[l][i].begin(), rF[l][i].end());
                rows[l].off.push_back(rows[l].idx.size());
            }
            for (uint32_t i = 0; i < NR; i++) {
                rows[3 + l].idx.insert(rows[3 + l].idx.end(), rR[l][i].begin(), rR[l][i].end());
                rows[3 + l].off.push_back(rows[3 + l].idx.size());
            }
        }
    }

    // ------------------------------------------------------------------ SPH stages
    void Density() {  // sph_solver.cpp:734-890
        const T sInv = sizeInv(), r2 = (T)prm.kernelRadiusSqu, a = alpha(), m = (T)prm.massF;
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)NF; ii++) {
            const uint32_t i = (uint32_t)ii;
            T dF = 0, dB = 0, dR = 0;
            for (uint64_t e = rows[0].off[i]; e < rows[0].off[i + 1]; e++) {
                const uint32_t j = rows[0].idx[e];
                dF = fmaT(m, KernelWeight(xF[i] - xF[j], yF[i] - yF[j], zF[i] - zF[j], sInv, r2, a), dF);
            }
            for (uint64_t e = rows[1].off[i]; e < rows[1].off[i + 1]; e++) {
                const uint32_t j = rows[1].idx[e];
                dB = fmaT(psiB[j], KernelWeight(xF[i] - xB[j], yF[i] - yB[j], zF[i] - zB[j], sInv, r2, a), dB);
            }
            for (uint64_t e = rows[2].off[i]; e < rows[2].off[i + 1]; e++) {
                const uint32_t j = rows[2].idx[e];
                dR = fmaT(psiR[j], KernelWeight(xF[i] - xR[j], yF[i] - yR[j], zF[i] - zR[j], sInv, r2, a), dR);
            }
            densF[i] = dF + dB + dR;
        }
    }
    void NonPressure() {  // sph_solver.cpp:892-1149
        const T sInv = sizeInv(), a = alpha(), m = (T)prm.massF, dt = (T)prm.timeStep;
        const KConst<T> k = MakeKConst(sInv, a);
        const T eps = T(1e-7f), hEps = T(0.01f) * sizeSqu();
        const T visF = T(10.0f) * (T)prm.viscosityF, visB = T(10.0f) * (T)prm.viscosityB;
        const T g[3] = {(T)prm.gravity[0], (T)prm.gravity[1], (T)prm.gravity[2]};
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)NF; ii++) {
            const uint32_t i = (uint32_t)ii;
            const T xi = xF[i], yi = yF[i], zi = zF[i], vxi = vxF[i], vyi = vyF[i], vzi = vzF[i];
            T fx = 0, fy = 0, fz = 0, bx = 0, by = 0, bz = 0, rx = 0, ry = 0, rz = 0;
            for (uint64_t e = rows[0].off[i]; e < rows[0].off[i + 1]; e++) {
                const uint32_t j = rows[0].idx[e];
                const T dx = xi - xF[j], dy = yi - yF[j], dz = zi - zF[j];
                const T dvx = vxi - vxF[j], dvy = vyi - vyF[j], dvz = vzi - vzF[j];
                const T d2 = fmaT(dx, dx, fmaT(dy, dy, dz * dz));
                const T kg = GradFac(d2, k);
                const T dot = fmaT(dvx, dx, fmaT(dvy, dy, dvz * dz));
                const T rhoJ = std::max(densF[j], eps);
                const T c = (m * dot) / (rhoJ * (d2 + hEps)) * kg;
                fx = fmaT(c, dx, fx); fy = fmaT(c, dy, fy); fz = fmaT(c, dz, fz);
            }
            for (uint64_t e = rows[1].off[i]; e < rows[1].off[i + 1]; e++) {
                const uint32_t j = rows[1].idx[e];
                const T dx = xi - xB[j], dy = yi - yB[j], dz = zi - zB[j];
                const T kg = GradFac(fmaT(dx, dx, fmaT(dy, dy, dz * dz)), k);
                const T gx = kg * dx, gy = kg * dy, gz = kg * dz;
                const T dvx = vxi - T(0), dvy = vyi - T(0), dvz = vzi - T(0);
                const T dot = fmaT(dvx, dx, fmaT(dvy, dy, dvz * dz));
                const T d2 = fmaT(dx, dx, fmaT(dy, dy, dz * dz));
                const T c = (volB[j] * dot) / (d2 + hEps);
                bx = fmaT(c, gx, bx); by = fmaT(c, gy, by); bz = fmaT(c, gz, bz);
            }
            for (uint64_t e = rows[2].off[i]; e < rows[2].off[i + 1]; e++) {
                const uint32_t j = rows[2].idx[e];
                const T dx = xi - xR[j], dy = yi - yR[j], dz = zi - zR[j];
                const T kg = GradFac(fmaT(dx, dx, fmaT(dy, dy, dz * dz)), k);
                const T gx = kg * dx, gy = kg * dy, gz = kg * dz;
                const T dvx = vxi - vxR[j], dvy = vyi - vyR[j], dvz = vzi - vzR[j];
                const T dot = fmaT(dvx, dx, fmaT(dvy, dy, dvz * dz));
                const T d2 = fmaT(dx, dx, fmaT(dy, dy, dz * dz));
                const T c = (volR[j] * dot) / (d2 + hEps);
                rx = fmaT(c, gx, rx); ry = fmaT(c, gy, ry); rz = fmaT(c, gz, rz);
            }
            const T ax = fx * visF + (bx + rx) * visB + g[0];
            const T ay = fy * visF + (by + ry) * visB + g[1];
            const T az = fz * visF + (bz + rz) * visB + g[2];
            vpxF[i] = fmaT(ax, dt, vxi); vpyF[i] = fmaT(ay, dt, vyi); vpzF[i] = fmaT(az, dt, vzi);
        }
    }
    void SourceDiagInit() {  // sph_solver.cpp:1225-1504
        const T sInv = sizeInv(), a = alpha(), m = (T)prm.massF, dt = (T)prm.timeStep;
        const KConst<T> k = MakeKConst(sInv, a);
        const T rhoSI = rhoSquInv();
        const T cF = -m * rhoSI, cB = T(-2.0f) * (T)prm.pressGamma * rhoSI, diagB = -m * rhoSI;
        const T om = (T)prm.jacobiOmega, ws = (T)prm.jacobiWarmStart, eps = T(1e-7f), rho0 = (T)prm.restDensity;
        const bool warm = prm.jacobiWarmStart > 0.0f;
        const T dt2 = dt * dt;
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)NF; ii++) {
            const uint32_t i = (uint32_t)ii;
            const T xi = xF[i], yi = yF[i], zi = zF[i], vx = vpxF[i], vy = vpyF[i], vz = vpzF[i];
            T sF = 0, sB = 0, sR = 0, cxF = 0, cyF = 0, czF = 0, g2 = 0, cxB = 0, cyB = 0, czB = 0, cxR = 0, cyR = 0, czR = 0;
            for (uint64_t e = rows[0].off[i]; e < rows[0].off[i + 1]; e++) {
                const uint32_t j = rows[0].idx[e];
                const T dx = xi - xF[j], dy = yi - yF[j], dz = zi - zF[j];
                const T dvx = vx - vpxF[j], dvy = vy - vpyF[j], dvz = vz - vpzF[j];
                const T d2 = fmaT(dx, dx, fmaT(dy, dy, dz * dz));
                const T kg = GradFac(d2, k);
                const T st = fmaT(dvx, dx, fmaT(dvy, dy, dvz * dz));
                sF = fmaT(kg, st, sF);
                cxF = fmaT(kg, dx, cxF); cyF = fmaT(kg, dy, cyF); czF = fmaT(kg, dz, czF);
                g2 = fmaT(kg, kg * d2, g2);
            }
            for (uint64_t e = rows[1].off[i]; e < rows[1].off[i + 1]; e++) {
                const uint32_t j = rows[1].idx[e];
                const T dx = xi - xB[j], dy = yi - yB[j], dz = zi - zB[j];
                const T kg = GradFac(fmaT(dx, dx, fmaT(dy, dy, dz * dz)), k);
                const T gx = kg * dx, gy = kg * dy, gz = kg * dz;
                const T dvx = vx - T(0), dvy = vy - T(0), dvz = vz - T(0);
                const T st = fmaT(dvx, gx, fmaT(dvy, gy, dvz * gz));
                const T p = psiB[j];
                sB = fmaT(p, st, sB);
                cxB = fmaT(p, gx, cxB); cyB = fmaT(p, gy, cyB); czB = fmaT(p, gz, czB);
            }
            for (uint64_t e = rows[2].off[i]; e < rows[2].off[i + 1]; e++) {
                const uint32_t j = rows[2].idx[e];
                const T dx = xi - xR[j], dy = yi - yR[j], dz = zi - zR[j];
                const T kg = GradFac(fmaT(dx, dx, fmaT(dy, dy, dz * dz)), k);
                const T gx = kg * dx, gy = kg * dy, gz = kg * dz;
                const T dvx = vx - vpxR[j], dvy = vy - vpyR[j], dvz = vz - vpzR[j];
                const T st = fmaT(dvx, gx, fmaT(dvy, gy, dvz * gz));
                const T p = psiR[j];
                sR = fmaT(p, st, sR);
                cxR = fmaT(p, gx, cxR); cyR = fmaT(p, gy, cyR); czR = fmaT(p, gz, czR);
            }
            sF *= m;
            const T src = rho0 - densF[i] - dt * (sF + sB + sR);
            const T cx = cxF * cF + (cxB + cxR) * cB;
            const T cy = cyF * cF + (cyB + cyR) * cB;
            const T cz = czF * cF + (czB + czR) * cB;
            const T dA = m * fmaT(cx, cxF, fmaT(cy, cyF, cz * czF));
            const T dB_ = m * diagB * g2;
            const T dC = fmaT(cx, cxB + cxR, fmaT(cy, cyB + cyR, cz * (czB + czR)));
            const T diag = dt2 * (dA + dB_ + dC);
            const bool valid = std::fabs(diag) > eps;
            const T cold = om * (src / diag);
            const T prev = warm ? presF[i] : T(0);
            const T init = warm ? ((prev > T(0)) ? ws * prev : cold) : cold;
            srcF[i] = src; diagF[i] = diag;
            presF[i] = std::max(T(0), valid ? init : T(0));
        }
    }
    void PressureAcc() {  // sph_solver.cpp:1507-1715
        const T sInv = sizeInv(), a = alpha(), m = (T)prm.massF;
        const KConst<T> k = MakeKConst(sInv, a);
        const T rho0 = (T)prm.restDensity;
        const T dInv2 = T(1) / (rho0 * rho0);
        const T bOuter = T(2.0f) * (T)prm.pressGamma * dInv2;
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)NF; ii++) {
            const uint32_t i = (uint32_t)ii;
            const T xi = xF[i], yi = yF[i], zi = zF[i], pi = presF[i];
            const T fOuter = m * pi * dInv2;
            T ax = 0, ay = 0, az = 0;
            for (uint64_t e = rows[0].off[i]; e < rows[0].off[i + 1]; e++) {
                const uint32_t j = rows[0].idx[e];
                const T dx = xi - xF[j], dy = yi - yF[j], dz = zi - zF[j];
                const T kg = GradFac(fmaT(dx, dx, fmaT(dy, dy, dz * dz)), k);
                const T c = (fOuter + m * presF[j] * dInv2) * kg;
                ax = fmaT(c, dx, ax); ay = fmaT(c, dy, ay); az = fmaT(c, dz, az);
            }
            for (int cat = 1; cat <= 2; cat++) {
                const std::vector<T>& X = cat == 1 ? xB : xR;
                const std::vector<T>& Y = cat == 1 ? yB : yR;
                const std::vector<T>& Z = cat == 1 ? zB : zR;
                const std::vector<T>& P = cat == 1 ? psiB : psiR;
                for (uint64_t e = rows[cat].off[i]; e < rows[cat].off[i + 1]; e++) {
                    const uint32_t j = rows[cat].idx[e];
                    const T dx = xi - X[j], dy = yi - Y[j], dz = zi - Z[j];
                    const T kg = GradFac(fmaT(dx, dx, fmaT(dy, dy, dz * dz)), k);
                    const T gx = kg * dx, gy = kg * dy, gz = kg * dz;
                    const T c = bOuter * P[j] * pi;
                    ax = fmaT(c, gx, ax); ay = fmaT(c, gy, ay); az = fmaT(c, gz, az);
                }
            }
            axF[i] = T(0) - ax; ayF[i] = T(0) - ay; azF[i] = T(0) - az;
        }
    }
    void JacobiUpdate() {  // sph_solver.cpp:1781-2049
        const T sInv = sizeInv(), a = alpha(), m = (T)prm.massF, dt = (T)prm.timeStep;
        const KConst<T> k = MakeKConst(sInv, a);
        const T dt2 = dt * dt, rho0 = (T)prm.restDensity, om = (T)prm.jacobiOmega, eps = T(1e-7f);
        std::vector<T> pNew(NF);
        std::vector<double> eR(NF, 0.0), eP(NF, 0.0), eA(NF, 0.0);
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)NF; ii++) {
            const uint32_t i = (uint32_t)ii;
            const T xi = xF[i], yi = yF[i], zi = zF[i], axi = axF[i], ayi = ayF[i], azi = azF[i];
            T sF = 0, sB = 0;
            for (uint64_t e = rows[0].off[i]; e < rows[0].off[i + 1]; e++) {
                const uint32_t j = rows[0].idx[e];
                const T dx = xi - xF[j], dy = yi - yF[j], dz = zi - zF[j];
                const T kg = GradFac(fmaT(dx, dx, fmaT(dy, dy, dz * dz)), k);
                const T dax = axi - axF[j], day = ayi - ayF[j], daz = azi - azF[j];
                const T sv = fmaT(dax, dx, fmaT(day, dy, daz * dz));
                sF = fmaT(kg, sv, sF);
            }
            sF *= m;
            for (int cat = 1; cat <= 2; cat++) {
                const std::vector<T>& X = cat == 1 ? xB : xR;
                const std::vector<T>& Y = cat == 1 ? yB : yR;
                const std::vector<T>& Z = cat == 1 ? zB : zR;
                const std::vector<T>& P = cat == 1 ? psiB : psiR;
                for (uint64_t e = rows[cat].off[i]; e < rows[cat].off[i + 1]; e++) {
                    const uint32_t j = rows[cat].idx[e];
                    const T dx = xi - X[j], dy = yi - Y[j], dz = zi - Z[j];
                    const T kg = GradFac(fmaT(dx, dx, fmaT(dy, dy, dz * dz)), k);
                    const T gx = kg * dx, gy = kg * dy, gz = kg * dz;
                    const T sv = fmaT(axi, gx, fmaT(ayi, gy, azi * gz));
                    sB += P[j] * sv;
                }
            }
            const T sys = dt2 * (sF + sB);
            const T resid = srcF[i] - sys;
            const T err = sys - srcF[i];
            const bool valid = std::fabs(diagF[i]) > eps;
            pNew[i] = std::max(T(0), valid ? fmaT(om, resid / diagF[i], presF[i]) : T(0));
            if (valid) {
                const double re = (double)(err / rho0);
                eR[i] = re; eP[i] = std::max(0.0, re); eA[i] = std::fabs(re);
            }
        }
        presF.swap(pNew);
        eRaw = ePos = eAbs = 0.0;
        for (uint32_t i = 0; i < NF; i++) { eRaw += eR[i]; ePos += eP[i]; eAbs += eA[i]; }
    }
    void Integration() {  // sph_solver.cpp:2051-2089
        const T dt = (T)prm.timeStep;
        for (uint32_t i = 0; i < NF; i++) {
            vxF[i] = fmaT(dt, axF[i], vpxF[i]); vyF[i] = fmaT(dt, ayF[i], vpyF[i]); vzF[i] = fmaT(dt, azF[i], vpzF[i]);
            xF[i] = fmaT(dt, vxF[i], xF[i]); yF[i] = fmaT(dt, vyF[i], yF[i]); zF[i] = fmaT(dt, vzF[i], zF[i]);
        }
    }
    bool Terminated() const {  // sph_solver.cpp:686-732
        if (iters < prm.minSolverIters) return false;
        if (iters >= prm.maxSolverIters) return true;
        const T tgt = (T)prm.densityDevTarget;
        switch (prm.solverTerminationCond) {
            case TSP_TERM_FIXED_ITERS: return iters >= prm.fixedIters;
            case TSP_TERM_REL_ERR_RAW: return avgRaw <= tgt;
            case TSP_TERM_REL_ERR_POS: return avgPos <= tgt;
            case TSP_TERM_REL_ERR_ABS: return avgAbs <= tgt;
            default: return iters >= 3;
        }
    }

    // ------------------------------------------------------------------ rigid (cpu_backend.cpp)
    void BuildByBody() {
        byBodyOff.assign(NRB + 1, 0);
        for (uint32_t i = 0; i < NR; i++) byBodyOff[bodyR[i] + 1]++;
        for (uint32_t b = 0; b < NRB; b++) byBodyOff[b + 1] += byBodyOff[b];
        byBodyIdx.assign(NR, 0);
        std::vector<uint32_t> cur(byBodyOff.begin(), byBodyOff.end() - 1);
        for (uint32_t i = 0; i < NR; i++) byBodyIdx[cur[bodyR[i]]++] = i;
    }
    void UpdateRigidParticles(bool predicted) {  // 2009-2063
        for (uint32_t i = 0; i < NR; i++) {
            const uint32_t b = bodyR[i];
            if (b >= NRB) throw std::runtime_error("Invalid rigid particle attachment.");
            const T lx = xRel[i], ly = yRel[i], lz = zRel[i];
            const T rx = fmaT(A[0][b], lx, fmaT(A[1][b], ly, A[2][b] * lz));
            const T ry = fmaT(A[3][b], lx, fmaT(A[4][b], ly, A[5][b] * lz));
            const T rz = fmaT(A[6][b], lx, fmaT(A[7][b], ly, A[8][b] * lz));
            if (!predicted) { xR[i] = cmx[b] + rx; yR[i] = cmy[b] + ry; zR[i] = cmz[b] + rz; }
            const T ox = predicted ? wpx[b] : wx[b], oy = predicted ? wpy[b] : wy[b], oz = predicted ? wpz[b] : wz[b];
            const T bx = predicted ? vpx[b] : vx[b], by = predicted ? vpy[b] : vy[b], bz = predicted ? vpz[b] : vz[b];
            (predicted ? vpxR : vxR)[i] = bx + oy * rz - oz * ry;
            (predicted ? vpyR : vyR)[i] = by + oz * rx - ox * rz;
            (predicted ? vpzR : vzR)[i] = bz + ox * ry - oy * rx;
        }
    }
    void ClearForcesAddGravity() {  // 2065-2087
        for (uint32_t b = 0; b < NRB; b++) {
            Fx[b] = Fy[b] = Fz[b] = Tx[b] = Ty[b] = Tz[b] = 0;
            if (mass[b] <= T(0) || massInv[b] <= T(0)) continue;
            Fx[b] += mass[b] * (T)prm.gravity[0]; Fy[b] += mass[b] * (T)prm.gravity[1]; Fz[b] += mass[b] * (T)prm.gravity[2];
        }
    }
    void ReduceForces() {  // 2089-2172 (sequential order of the per-body index list)
        for (uint32_t b = 0; b < NRB; b++) {
            T fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
            for (uint32_t w = byBodyOff[b]; w < byBodyOff[b + 1]; w++) {
                const uint32_t i = byBodyIdx[w];
                const T lx = xRel[i], ly = yRel[i], lz = zRel[i];
                const T rx = fmaT(A[0][b], lx, fmaT(A[1][b], ly, A[2][b] * lz));
                const T ry = fmaT(A[3][b], lx, fmaT(A[4][b], ly, A[5][b] * lz));
                const T rz = fmaT(A[6][b], lx, fmaT(A[7][b], ly, A[8][b] * lz));
                fx += fxR[i]; fy += fyR[i]; fz += fzR[i];
                tx += ry * fzR[i] - rz * fyR[i]; ty += rz * fxR[i] - rx * fzR[i]; tz += rx * fyR[i] - ry * fxR[i];
            }
            Fx[b] += fx; Fy[b] += fy; Fz[b] += fz; Tx[b] += tx; Ty[b] += ty; Tz[b] += tz;
        }
    }
    void PredictBodies() {  // 2174-2235
        const T dt = (T)prm.timeStep;
        for (uint32_t b = 0; b < NRB; b++) {
            vpx[b] = vx[b] + dt * Fx[b] * massInv[b]; vpy[b] = vy[b] + dt * Fy[b] * massInv[b];
            vpz[b] = vz[b] + dt * Fz[b] * massInv[b];
            Lpx[b] = Lx[b] + dt * Tx[b]; Lpy[b] = Ly[b] + dt * Ty[b]; Lpz[b] = Lz[b] + dt * Tz[b];
            T t[9], I[9];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++)
                    t[r * 3 + c] = A[r * 3 + 0][b] * Ib[0 * 3 + c][b] + A[r * 3 + 1][b] * Ib[1 * 3 + c][b] +
                                   A[r * 3 + 2][b] * Ib[2 * 3 + c][b];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++)
                    I[r * 3 + c] = t[r * 3 + 0] * A[c * 3 + 0][b] + t[r * 3 + 1] * A[c * 3 + 1][b] + t[r * 3 + 2] * A[c * 3 + 2][b];
            wpx[b] = fmaT(I[0], Lpx[b], fmaT(I[1], Lpy[b], I[2] * Lpz[b]));
            wpy[b] = fmaT(I[3], Lpx[b], fmaT(I[4], Lpy[b], I[5] * Lpz[b]));
            wpz[b] = fmaT(I[6], Lpx[b], fmaT(I[7], Lpy[b], I[8] * Lpz[b]));
        }
    }
    static T Dot3(T ax, T ay, T az, T bx, T by, T bz) { return fmaT(ax, bx, fmaT(ay, by, az * bz)); }
    static void Norm3(T& x, T& y, T& z) {
        const T len = std::sqrt(Dot3(x, y, z, x, y, z));
        if (len <= T(1e-12f) || !std::isfinite((double)len)) throw std::runtime_error("Degenerate rigid body orientation.");
        const T inv = T(1) / len;
        x *= inv; y *= inv; z *= inv;
    }
    void IntegrateBodies() {  // 2237-2303
        const T dt = (T)prm.timeStep;
        for (uint32_t b = 0; b < NRB; b++) {
            vx[b] = vpx[b]; vy[b] = vpy[b]; vz[b] = vpz[b]; Lx[b] = Lpx[b]; Ly[b] = Lpy[b]; Lz[b] = Lpz[b];
            cmx[b] += dt * vx[b]; cmy[b] += dt * vy[b]; cmz[b] += dt * vz[b];
            const T ox = wpx[b], oy = wpy[b], oz = wpz[b];
            wx[b] = ox; wy[b] = oy; wz[b] = oz;
            const T a00 = A[0][b], a01 = A[1][b], a02 = A[2][b], a10 = A[3][b], a11 = A[4][b], a12 = A[5][b],
                    a20 = A[6][b], a21 = A[7][b], a22 = A[8][b];
            A[0][b] += dt * (-oz * a10 + oy * a20); A[1][b] += dt * (-oz * a11 + oy * a21); A[2][b] += dt * (-oz * a12 + oy * a22);
            A[3][b] += dt * (oz * a00 - ox * a20); A[4][b] += dt * (oz * a01 - ox * a21); A[5][b] += dt * (oz * a02 - ox * a22);
            A[6][b] += dt * (-oy * a00 + ox * a10); A[7][b] += dt * (-oy * a01 + ox * a11); A[8][b] += dt * (-oy * a02 + ox * a12);
            T b1x = A[0][b], b1y = A[3][b], b1z = A[6][b];
            Norm3(b1x, b1y, b1z);
            T b2x = A[1][b], b2y = A[4][b], b2z = A[7][b];
            const T d12 = Dot3(b1x, b1y, b1z, b2x, b2y, b2z);
            b2x -= d12 * b1x; b2y -= d12 * b1y; b2z -= d12 * b1z;
            Norm3(b2x, b2y, b2z);
            T b3x = A[2][b], b3y = A[5][b], b3z = A[8][b];
            const T d13 = Dot3(b1x, b1y, b1z, b3x, b3y, b3z), d23 = Dot3(b2x, b2y, b2z, b3x, b3y, b3z);
            b3x -= d13 * b1x + d23 * b2x; b3y -= d13 * b1y + d23 * b2y; b3z -= d13 * b1z + d23 * b2z;
            Norm3(b3x, b3y, b3z);
            A[0][b] = b1x; A[1][b] = b2x; A[2][b] = b3x; A[3][b] = b1y; A[4][b] = b2y; A[5][b] = b3y;
            A[6][b] = b1z; A[7][b] = b2z; A[8][b] = b3z;
        }
    }
    void RigidViscousForces() {  // sph_solver.cpp:1151-1223
        const T sInv = sizeInv(), a = alpha(), r2 = (T)prm.kernelRadiusSqu, m = (T)prm.massF;
        const T hEps = T(0.01f) * sizeSqu(), visB = T(10.0f) * (T)prm.viscosityB;
        for (uint32_t i = 0; i < NR; i++) {
            T fx = 0, fy = 0, fz = 0;
            for (uint64_t e = rows[3].off[i]; e < rows[3].off[i + 1]; e++) {
                const uint32_t j = rows[3].idx[e];
                const T dx = xF[j] - xR[i], dy = yF[j] - yR[i], dz = zF[j] - zR[i];
                const T dvx = vxF[j] - vxR[i], dvy = vyF[j] - vyR[i], dvz = vzF[j] - vzR[i];
                T gx, gy, gz;
                GradScalar(dx, dy, dz, sInv, r2, a, gx, gy, gz);
                const T dot = fmaT(dvx, dx, fmaT(dvy, dy, dvz * dz));
                const T d2 = fmaT(dx, dx, fmaT(dy, dy, dz * dz));
                const T c = (volR[i] * dot) / (d2 + hEps);
                const T fc = -m * visB * c;
                fx = fmaT(fc, gx, fx); fy = fmaT(fc, gy, fy); fz = fmaT(fc, gz, fz);
            }
            fxR[i] = fx; fyR[i] = fy; fzR[i] = fz;
        }
    }
    void RigidPressureForces() {  // sph_solver.cpp:1717-1778
        const T sInv = sizeInv(), a = alpha(), r2 = (T)prm.kernelRadiusSqu, m = (T)prm.massF;
        const T rho0 = (T)prm.restDensity;
        const T dInv2 = T(1) / (rho0 * rho0), bOuter = T(2.0f) * (T)prm.pressGamma * dInv2;
        for (uint32_t i = 0; i < NR; i++) {
            T fx = 0, fy = 0, fz = 0;
            for (uint64_t e = rows[3].off[i]; e < rows[3].off[i + 1]; e++) {
                const uint32_t j = rows[3].idx[e];
                const T dx = xF[j] - xR[i], dy = yF[j] - yR[i], dz = zF[j] - zR[i];
                T gx, gy, gz;
                GradScalar(dx, dy, dz, sInv, r2, a, gx, gy, gz);
                const T fc = m * bOuter * psiR[i] * presF[j];
                fx = fmaT(fc, gx, fx); fy = fmaT(fc, gy, fy); fz = fmaT(fc, gz, fz);
            }
            fxR[i] += fx; fyR[i] += fy; fzR[i] += fz;
        }
    }

    // ------------------------------------------------------------------ rigid contacts
    // RIGID_CONTACT_VOLUME_FACTOR (rigid_solver.h:23)
    static constexpr float kContactVol = 0.7f;
    // ContactKernel (rigid_solver.cpp:51-63): cubic-spline weight and scalar gradient
    T ContactKernel(T dx, T dy, T dz, T& gx, T& gy, T& gz) const {
        const T sInv = sizeInv(), r2 = (T)prm.kernelRadiusSqu, a = alpha();
        const T d2 = fmaT(dx, dx, fmaT(dy, dy, dz * dz));
        if (d2 >= r2) { gx = gy = gz = T(0); return T(0); }
        const T q = std::sqrt(d2) * sInv;
        const T t1 = std::max(T(1) - q, T(0)), t2 = std::max(T(2) - q, T(0));
        GradScalar(dx, dy, dz, sInv, r2, a, gx, gy, gz);
        return a * (t2 * t2 * t2 - T(4) * t1 * t1 * t1);
    }
    // BuildRigidBoundaryNeighbors (rigid_solver.cpp:90-149): contact boundary particles in order
    // of first reference by the rigid particles' RB rows, RB rows as contact indices, BR rows
    bool BuildContactNeighbors() {
        cLocalB.clear(); cOffRB.clear(); cIdxRB.clear(); cOffBR.clear(); cIdxBR.clear();
        std::unordered_map<uint32_t, uint32_t> toContact;
        bool any = false;
        const CSR& RB = rows[4];
        const CSR& RR = rows[5];
        for (uint32_t i = 0; i < NR; i++) {
            const uint64_t b0 = RB.off[i], b1 = RB.off[i + 1];
            if (cOffRB.empty()) {
                if (b0 == b1) { any = any || RR.off[i + 1] > RR.off[i]; continue; }
                cOffRB.assign((size_t)NR + 1, 0);
                cOffBR.push_back(0);
            }
            for (uint64_t k = b0; k < b1; k++) {
                const uint32_t b = RB.idx[k];
                auto ins = toContact.emplace(b, (uint32_t)cLocalB.size());
                if (ins.second) { cLocalB.push_back(b); cOffBR.push_back(0); }
                const uint32_t c = ins.first->second;
                cIdxRB.push_back(c);
                cOffBR[c + 1]++;
            }
            cOffRB[i + 1] = cIdxRB.size();
        }
        if (cOffRB.empty()) return any;
        const uint32_t nc = (uint32_t)cLocalB.size();
        for (uint32_t c = 0; c < nc; c++) cOffBR[c + 1] += cOffBR[c];
        cIdxBR.assign(cOffBR.back(), 0);
        std::vector<uint64_t> w(cOffBR.begin(), cOffBR.end() - 1);
        for (uint32_t i = 0; i < NR; i++)
            for (uint64_t k = cOffRB[i]; k < cOffRB[i + 1]; k++) cIdxBR[w[cIdxRB[k]]++] = i;
        return true;
    }
    // ForEachContactNeighbor (rigid_solver.cpp:22-48): BR row of a boundary contact; RR then RB
    // row of a rigid particle. f(j, neighborIsBoundary) with j a rigid or contact index.
    template <class Fn> void ForEachContact(bool boundary, uint32_t i, const Fn& f) const {
        if (boundary) {
            for (uint64_t k = cOffBR[i]; k < cOffBR[i + 1]; k++) f(cIdxBR[k], false);
            return;
        }
        const CSR& RR = rows[5];
        for (uint64_t k = RR.off[i]; k < RR.off[i + 1]; k++) f(RR.idx[k], false);
        if (!cOffRB.empty())
            for (uint64_t k = cOffRB[i]; k < cOffRB[i + 1]; k++) f(cIdxRB[k], true);
    }
    T CPosX(bool boundary, uint32_t j) const { return boundary ? xB[cLocalB[j]] : xR[j]; }
    T CPosY(bool boundary, uint32_t j) const { return boundary ? yB[cLocalB[j]] : yR[j]; }
    T CPosZ(bool boundary, uint32_t j) const { return boundary ? zB[cLocalB[j]] : zR[j]; }
    T CVol(bool boundary, uint32_t j) const { return boundary ? volB[cLocalB[j]] : volR[j]; }
    // RigidContactGeometry (rigid_solver.cpp:151-227)
    void ContactGeometry() {
        for (int k = 0; k < 9; k++) cIw[k].assign(NRB, T(0));
        for (uint32_t b = 0; b < NRB; b++) {
            T t[9];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++)
                    t[r * 3 + c] = A[r * 3 + 0][b] * Ib[0 * 3 + c][b] + A[r * 3 + 1][b] * Ib[1 * 3 + c][b] +
                                   A[r * 3 + 2][b] * Ib[2 * 3 + c][b];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++)
                    cIw[r * 3 + c][b] = t[r * 3 + 0] * A[c * 3 + 0][b] + t[r * 3 + 1] * A[c * 3 + 1][b] +
                                        t[r * 3 + 2] * A[c * 3 + 2][b];
        }
        cRelWx.assign(NR, T(0)); cRelWy.assign(NR, T(0)); cRelWz.assign(NR, T(0));
        for (uint32_t i = 0; i < NR; i++) {
            const uint32_t b = bodyR[i];
            const T lx = xRel[i], ly = yRel[i], lz = zRel[i];
            cRelWx[i] = fmaT(A[0][b], lx, fmaT(A[1][b], ly, A[2][b] * lz));
            cRelWy[i] = fmaT(A[3][b], lx, fmaT(A[4][b], ly, A[5][b] * lz));
            cRelWz[i] = fmaT(A[6][b], lx, fmaT(A[7][b], ly, A[8][b] * lz));
        }
    }
    struct BodyGrad { uint32_t b; T x, y, z, tx, ty, tz; };
    static void AddBodyGrad(std::vector<BodyGrad>& g, uint32_t b, T x, T y, T z, T rx, T ry, T rz) {
        auto it = std::find_if(g.begin(), g.end(), [&](const BodyGrad& e) { return e.b == b; });
        if (it == g.end()) { g.push_back({b, T(0), T(0), T(0), T(0), T(0), T(0)}); it = g.end() - 1; }
        it->x += x; it->y += y; it->z += z;
        it->tx += ry * z - rz * y;
        it->ty += rz * x - rx * z;
        it->tz += rx * y - ry * x;
    }
    // RigidContactDensityAndDiagonal (rigid_solver.cpp:229-344)
    void ContactDensityAndDiagonal(bool boundary) {
        const uint32_t N = boundary ? (uint32_t)cLocalB.size() : NR;
        auto& dens = boundary ? cDensB : cDensR;
        auto& diag = boundary ? cDiagB : cDiagR;
        auto& pres = boundary ? cPresB : cPresR;
        auto& src = boundary ? cSrcB : cSrcR;
        auto& omg = boundary ? cOmegaB : cOmegaR;
        dens.assign(N, T(0)); diag.assign(N, T(0)); pres.assign(N, T(0)); src.assign(N, T(0)); omg.assign(N, T(0));
        const T dt = (T)prm.timeStep;
        std::vector<BodyGrad> g;
        for (uint32_t i = 0; i < N; i++) {
            g.clear();
            const T volRest = T(kContactVol) * CVol(boundary, i);
            T rho = T(kContactVol);
            bool has = false;
            const T px = CPosX(boundary, i), py = CPosY(boundary, i), pz = CPosZ(boundary, i);
            ForEachContact(boundary, i, [&](uint32_t j, bool nb) {
                T gx, gy, gz;
                const T w = ContactKernel(px - CPosX(nb, j), py - CPosY(nb, j), pz - CPosZ(nb, j), gx, gy, gz);
                if (!(w > T(0))) return;
                has = true;
                const T nv = T(kContactVol) * CVol(nb, j);
                rho += nv * w;
                gx *= nv; gy *= nv; gz *= nv;
                if (!boundary) AddBodyGrad(g, bodyR[i], gx, gy, gz, cRelWx[i], cRelWy[i], cRelWz[i]);
                if (!nb) AddBodyGrad(g, bodyR[j], -gx, -gy, -gz, cRelWx[j], cRelWy[j], cRelWz[j]);
            });
            double d = 0.0;
            for (const BodyGrad& e : g) {
                const uint32_t b = e.b;
                const T wx = cIw[0][b] * e.tx + cIw[1][b] * e.ty + cIw[2][b] * e.tz;
                const T wy = cIw[3][b] * e.tx + cIw[4][b] * e.ty + cIw[5][b] * e.tz;
                const T wz = cIw[6][b] * e.tx + cIw[7][b] * e.ty + cIw[8][b] * e.tz;
                d += (double)(massInv[b] * (e.x * e.x + e.y * e.y + e.z * e.z) + e.tx * wx + e.ty * wy + e.tz * wz);
            }
            const double dv = (double)dt * (double)dt * (double)volRest / (double)(rho * rho) * d;
            diag[i] = (T)dv;
            if (!std::isfinite((double)diag[i]) || diag[i] < T(0))
                throw std::runtime_error("Invalid rigid contact diagonal.");
            dens[i] = rho; pres[i] = T(0); src[i] = rho - T(1); omg[i] = has ? T(0.5f) : T(0);
        }
    }
    // RigidContactRelaxation (rigid_solver.cpp:346-407)
    uint64_t ContactRelaxation() {
        uint64_t n = 0;
        for (uint32_t b = 0; b < NRB; b++) {
            uint32_t count = 0;
            for (uint32_t w = byBodyOff[b]; w < byBodyOff[b + 1]; w++) count += cOmegaR[byBodyIdx[w]] > T(0);
            if (count == 0) continue;
            for (uint32_t w = byBodyOff[b]; w < byBodyOff[b + 1]; w++) cOmegaR[byBodyIdx[w]] /= (T)count;
            n += count;
        }
        const uint32_t NC = (uint32_t)cLocalB.size();
        if (NC == 0) return n;
        std::vector<uint32_t> perBody(NRB, 0), last(NRB, NC);
        for (uint32_t c = 0; c < NC; c++) {
            if (cOmegaB[c] <= T(0)) continue;
            n++;
            if (cDiagB[c] <= T(0)) continue;
            for (uint64_t k = cOffBR[c]; k < cOffBR[c + 1]; k++) {
                const uint32_t b = bodyR[cIdxBR[k]];
                if (massInv[b] <= T(0) || last[b] == c) continue;
                last[b] = c;
                perBody[b]++;
            }
        }
        for (uint32_t c = 0; c < NC; c++) {
            if (cOmegaB[c] <= T(0) || cDiagB[c] <= T(0)) continue;
            uint32_t mx = 0;
            for (uint64_t k = cOffBR[c]; k < cOffBR[c + 1]; k++) mx = std::max(mx, perBody[bodyR[cIdxBR[k]]]);
            if (mx > 0) cOmegaB[c] /= (T)mx;
        }
        return n;
    }
    // RigidContactPressureForces (rigid_solver.cpp:409-460)
    void ContactPressureForces() {
        cFxR.assign(NR, T(0)); cFyR.assign(NR, T(0)); cFzR.assign(NR, T(0));
        for (uint32_t i = 0; i < NR; i++) {
            T fx = 0, fy = 0, fz = 0;
            const T pi = cPresR[i] / (cDensR[i] * cDensR[i]);
            ForEachContact(false, i, [&](uint32_t j, bool nb) {
                T gx, gy, gz;
                const T w = ContactKernel(xR[i] - CPosX(nb, j), yR[i] - CPosY(nb, j), zR[i] - CPosZ(nb, j), gx, gy, gz);
                if (!(w > T(0))) return;
                const T rho = nb ? cDensB[j] : cDensR[j];
                const T pj = (nb ? cPresB[j] : cPresR[j]) / (rho * rho);
                const T c = -T(kContactVol) * volR[i] * T(kContactVol) * CVol(nb, j) * (pi + pj);
                fx += c * gx; fy += c * gy; fz += c * gz;
            });
            cFxR[i] = fx; cFyR[i] = fy; cFzR[i] = fz;
        }
    }
    // ReduceRigidParticleForcesToBody(Contact) (cpu_backend.cpp:2089-2172)
    void ReduceContactForces() {
        cFx.assign(NRB, T(0)); cFy.assign(NRB, T(0)); cFz.assign(NRB, T(0));
        cTx.assign(NRB, T(0)); cTy.assign(NRB, T(0)); cTz.assign(NRB, T(0));
        for (uint32_t b = 0; b < NRB; b++) {
            T fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
            for (uint32_t w = byBodyOff[b]; w < byBodyOff[b + 1]; w++) {
                const uint32_t i = byBodyIdx[w];
                const T lx = xRel[i], ly = yRel[i], lz = zRel[i];
                const T rx = fmaT(A[0][b], lx, fmaT(A[1][b], ly, A[2][b] * lz));
                const T ry = fmaT(A[3][b], lx, fmaT(A[4][b], ly, A[5][b] * lz));
                const T rz = fmaT(A[6][b], lx, fmaT(A[7][b], ly, A[8][b] * lz));
                fx += cFxR[i]; fy += cFyR[i]; fz += cFzR[i];
                tx += ry * cFzR[i] - rz * cFyR[i]; ty += rz * cFxR[i] - rx * cFzR[i]; tz += rx * cFyR[i] - ry * cFxR[i];
            }
            cFx[b] += fx; cFy[b] += fy; cFz[b] += fz; cTx[b] += tx; cTy[b] += ty; cTz[b] += tz;
        }
    }
    // RigidContactParticleVelocities (rigid_solver.cpp:462-506)
    void ContactParticleVelocities() {
        const T dt = (T)prm.timeStep;
        cVxR.assign(NR, T(0)); cVyR.assign(NR, T(0)); cVzR.assign(NR, T(0));
        for (uint32_t i = 0; i < NR; i++) {
            const uint32_t b = bodyR[i];
            const T tx = cTx[b], ty = cTy[b], tz = cTz[b];
            const T wx = cIw[0][b] * tx + cIw[1][b] * ty + cIw[2][b] * tz;
            const T wy = cIw[3][b] * tx + cIw[4][b] * ty + cIw[5][b] * tz;
            const T wz = cIw[6][b] * tx + cIw[7][b] * ty + cIw[8][b] * tz;
            const T rx = cRelWx[i], ry = cRelWy[i], rz = cRelWz[i];
            cVxR[i] = dt * (massInv[b] * cFx[b] + wy * rz - wz * ry);
            cVyR[i] = dt * (massInv[b] * cFy[b] + wz * rx - wx * rz);
            cVzR[i] = dt * (massInv[b] * cFz[b] + wx * ry - wy * rx);
        }
    }
    // RigidContactDensityError (rigid_solver.cpp:508-579), velocities of rigid particles given
    double ContactDensityError(const std::vector<T>& vxr, const std::vector<T>& vyr, const std::vector<T>& vzr) {
        const T dt = (T)prm.timeStep;
        double sum = 0.0;
        for (int pass = 0; pass < 2; pass++) {
            const bool boundary = pass == 1;
            const uint32_t N = boundary ? (uint32_t)cLocalB.size() : NR;
            const auto& src = boundary ? cSrcB : cSrcR;
            const auto& pres = boundary ? cPresB : cPresR;
            auto& err = boundary ? cErrB : cErrR;
            err.assign(N, T(0));
            for (uint32_t i = 0; i < N; i++) {
                const T vx = boundary ? T(0) : vxr[i], vy = boundary ? T(0) : vyr[i], vz = boundary ? T(0) : vzr[i];
                const T px = CPosX(boundary, i), py = CPosY(boundary, i), pz = CPosZ(boundary, i);
                T res = src[i];
                ForEachContact(boundary, i, [&](uint32_t j, bool nb) {
                    T gx, gy, gz;
                    const T w = ContactKernel(px - CPosX(nb, j), py - CPosY(nb, j), pz - CPosZ(nb, j), gx, gy, gz);
                    if (!(w > T(0))) return;
                    const T dvx = (nb ? T(0) : vxr[j]) - vx, dvy = (nb ? T(0) : vyr[j]) - vy, dvz = (nb ? T(0) : vzr[j]) - vz;
                    const T div = dt * (dvx * gx + dvy * gy + dvz * gz);
                    res -= T(kContactVol) * CVol(nb, j) * div;
                });
                if (!std::isfinite((double)res)) throw std::runtime_error("Non-finite rigid contact density error.");
                err[i] = res;
                sum += pres[i] > T(0) ? std::abs((double)res) : std::max((double)res, 0.0);
            }
        }
        return sum;
    }
    // RigidContactPressureRelaxedJacobi (rigid_solver.cpp:581-600)
    static void ContactJacobi(const std::vector<T>& err, const std::vector<T>& diag, const std::vector<T>& omg,
                              std::vector<T>& pres) {
        for (size_t i = 0; i < pres.size(); i++) {
            if (!(diag[i] > T(0))) continue;
            const T p = pres[i] + omg[i] * err[i] / diag[i];
            if (!std::isfinite((double)p)) throw std::runtime_error("Non-finite rigid contact pressure.");
            pres[i] = std::max(T(0), p);
        }
    }
    T ContactTarget() const {
        return (prm.rigidContactDensityDevTarget == 0.0f && prm.rigidContactMaxSolverIters == 0)
                   ? T(0.001f) : (T)prm.rigidContactDensityDevTarget;
    }
    uint32_t ContactMaxIters() const {
        return (prm.rigidContactDensityDevTarget == 0.0f && prm.rigidContactMaxSolverIters == 0)
                   ? 100u : prm.rigidContactMaxSolverIters;
    }
    // SolveRigidContacts (rigid_solver.cpp:602-799)
    void SolveRigidContacts() {
        const T target = ContactTarget();
        const uint32_t maxIters = ContactMaxIters();
        if (!std::isfinite((double)target) || target <= T(0) || maxIters == 0)
            throw std::runtime_error("Invalid rigid contact solver tolerance or iteration limit.");
        contactIters = 0; contactAvgErr = T(0); contactConverged = true; contactCount = 0;
        const bool has = BuildContactNeighbors();
        const uint32_t NC = (uint32_t)cLocalB.size();
        cDensB.assign(NC, T(0)); cDiagB.assign(NC, T(0)); cPresB.assign(NC, T(0)); cSrcB.assign(NC, T(0));
        cErrB.assign(NC, T(0)); cOmegaB.assign(NC, T(0));
        if (!has) return;
        ContactGeometry();
        ContactDensityAndDiagonal(false);
        ContactDensityAndDiagonal(true);
        contactCount = ContactRelaxation();
        // source motion: external and fluid forces, no contact forces
        PredictBodies();
        UpdateRigidParticles(true);
        (void)ContactDensityError(vpxR, vpyR, vpzR);
        cSrcR.swap(cErrR);
        cSrcB.swap(cErrB);
        for (;;) {
            ContactPressureForces();
            ReduceContactForces();
            ContactParticleVelocities();
            const double e = ContactDensityError(cVxR, cVyR, cVzR);
            contactAvgErr = contactCount > 0 ? (T)(float)(e / (double)contactCount) : T(0);
            contactConverged = contactAvgErr <= target;
            if (contactConverged || contactIters == maxIters) break;
            ContactJacobi(cErrR, cDiagR, cOmegaR, cPresR);
            ContactJacobi(cErrB, cDiagB, cOmegaB, cPresB);
            contactIters++;
        }
        for (uint32_t b = 0; b < NRB; b++) {
            Fx[b] += cFx[b]; Fy[b] += cFy[b]; Fz[b] += cFz[b];
            Tx[b] += cTx[b]; Ty[b] += cTy[b]; Tz[b] += cTz[b];
        }
    }

    // ------------------------------------------------------------------ drivers
    void NeighborSearch() {  // cpu_backend.cpp:1593-1624
        ReorderAndConstruct(true);
        Query();
    }
    void Step() {  // sph_solver.cpp:34-319 (serial)
        if (NF == 0 && NRB == 0) { return; }
        ReorderAndConstruct(false);
        Query();
        Density();
        if (NRB > 0) ClearForcesAddGravity();
        NonPressure();
        if (NRB > 0) {
            RigidViscousForces();
            ReduceForces();
            PredictBodies();
            UpdateRigidParticles(true);
        }
        SourceDiagInit();
        iters = NF > 0 ? 1 : 0;
        avgRaw = avgPos = avgAbs = 0;
        while (NF > 0) {
            PressureAcc();
            iters++;
            const bool compute = iters >= prm.minSolverIters &&
                                 (prm.solverTerminationCond != TSP_TERM_FIXED_ITERS || Terminated());
            JacobiUpdate();
            if (compute) {
                avgRaw = (T)((float)eRaw / (float)NF);
                avgPos = (T)((float)ePos / (float)NF);
                avgAbs = (T)((float)eAbs / (float)NF);
            }
            if (Terminated()) break;
        }
        PressureAcc();
        if (NRB > 0) {
            RigidPressureForces();
            ClearForcesAddGravity();
            ReduceForces();
        }
        Integration();
        if (NRB > 0) {
            SolveRigidContacts();
            PredictBodies();
            IntegrateBodies();
            UpdateRigidParticles(false);
        }
    }
    // ComputeParticleCoefficients (builder.cpp:174-376): sums over z-y-x sorted cells
    static void Coefficients(const std::vector<T>& X, const std::vector<T>& Y, const std::vector<T>& Z,
                             uint32_t begin, uint32_t end, const tsp_params& p, T sInv, T alpha,
                             std::vector<T>& vol, std::vector<T>& psi) {
        const float cs = p.kernelRadius * p.gridCellSizeRatio;
        const float span = p.kernelRadius / cs;
        const int reach = std::max(1, (int)std::ceil(std::max(0.0f, span - 1e-6f)));
        const float csInv = 1.0f / cs;
        const uint32_t n = end - begin;
        struct CC { int x, y, z; };
        std::vector<CC> cc(n);
        std::vector<uint32_t> srt(n);
        for (uint32_t l = 0; l < n; l++) {
            const uint32_t i = begin + l;
            cc[l] = {(int)std::floor((float)X[i] * csInv), (int)std::floor((float)Y[i] * csInv), (int)std::floor((float)Z[i] * csInv)};
            srt[l] = l;
        }
        auto less = [&](const CC& a, const CC& b) {
            if (a.z != b.z) return a.z < b.z;
            if (a.y != b.y) return a.y < b.y;
            return a.x < b.x;
        };
        std::sort(srt.begin(), srt.end(), [&](uint32_t a, uint32_t b) {
            if (less(cc[a], cc[b])) return true;
            if (less(cc[b], cc[a])) return false;
            return a < b;
        });
        const T r2 = (T)p.kernelRadiusSqu;
        const T defPsi = (T)p.massB, defVol = p.restDensity > 0.0f ? (T)(p.massB / p.restDensity) : T(0);
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t ss = 0; ss < (int64_t)n; ss++) {
            const uint32_t i = begin + srt[ss];
            const CC base = cc[srt[ss]];
            T sum = 0;
            for (int dz = -reach; dz <= reach; dz++)
                for (int dy = -reach; dy <= reach; dy++) {
                    const CC lo{base.x - reach, base.y + dy, base.z + dz}, hi{base.x + reach, base.y + dy, base.z + dz};
                    auto f = std::lower_bound(srt.begin(), srt.end(), lo, [&](uint32_t l, const CC& t) { return less(cc[l], t); });
                    auto e = std::upper_bound(f, srt.end(), hi, [&](const CC& t, uint32_t l) { return less(t, cc[l]); });
                    for (auto it = f; it != e; ++it) {
                        const uint32_t j = begin + *it;
                        sum += BoundaryWeight(X[i] - X[j], Y[i] - Y[j], Z[i] - Z[j], sInv, r2, alpha);
                    }
                }
            if (sum > T(0) && std::isfinite((double)sum)) {
                vol[i] = T(1) / sum;
                psi[i] = (T)p.restDensity * vol[i];
            } else {
                vol[i] = defVol; psi[i] = defPsi;
            }
        }
    }
};

}  // namespace orc

// ====================================================================== C API (test infra)
using namespace orc;

struct orc_handle {
    int fp64 = 0;
    Oracle<float>* f = nullptr;
    Oracle<double>* d = nullptr;
    std::string err;
};

#define ORC_DISPATCH(h, expr)              \
    do {                                   \
        if ((h)->fp64) { auto& O = *(h)->d; expr; } \
        else { auto& O = *(h)->f; expr; }  \
    } while (0)

#define ORC_TRY(h, body)                                     \
    try { body; return 0; }                                  \
    catch (const std::exception& e) { (h)->err = e.what(); return -1; }

template <typename T, typename S>
static void Load(std::vector<T>& dst, const S* src, uint32_t n, T def) {
    dst.resize(n);
    for (uint32_t i = 0; i < n; i++) dst[i] = src ? (T)src[i] : def;
}
template <typename T, typename S>
static void Store(const std::vector<T>& src, S* dst, uint32_t n) {
    if (!dst) return;
    for (uint32_t i = 0; i < n && i < src.size(); i++) dst[i] = (S)src[i];
}

template <typename T> static void Pull(Oracle<T>& O, const tsp_state_view& s, const tsp_params& p) {
    O.prm = p;
    O.NF = s.N_F; O.NB = s.N_B; O.NR = s.N_R; O.NRB = s.N_RB; O.step = s.step; O.time = s.time;
    O.idF.resize(O.NF);
    for (uint32_t i = 0; i < O.NF; i++) O.idF[i] = s.idF ? s.idF[i] : i;
    Load(O.xF, s.xPosF, O.NF, T(0)); Load(O.yF, s.yPosF, O.NF, T(0)); Load(O.zF, s.zPosF, O.NF, T(0));
    Load(O.vxF, s.xVelF, O.NF, T(0)); Load(O.vyF, s.yVelF, O.NF, T(0)); Load(O.vzF, s.zVelF, O.NF, T(0));
    Load(O.vpxF, s.xVelPredF, O.NF, T(0)); Load(O.vpyF, s.yVelPredF, O.NF, T(0)); Load(O.vpzF, s.zVelPredF, O.NF, T(0));
    Load(O.axF, s.xAccPressF, O.NF, T(0)); Load(O.ayF, s.yAccPressF, O.NF, T(0)); Load(O.azF, s.zAccPressF, O.NF, T(0));
    Load(O.srcF, s.sourceTermF, O.NF, T(0)); Load(O.diagF, s.diagElemF, O.NF, T(0));
    Load(O.presF, s.pressureF, O.NF, T(0)); Load(O.densF, s.densityF, O.NF, (T)p.restDensity);
    const T defPsi = (T)p.massB, defVol = p.restDensity > 0.0f ? (T)(p.massB / p.restDensity) : T(0);
    O.idB.resize(O.NB);
    for (uint32_t i = 0; i < O.NB; i++) O.idB[i] = s.idB ? s.idB[i] : i;
    Load(O.xB, s.xPosB, O.NB, T(0)); Load(O.yB, s.yPosB, O.NB, T(0)); Load(O.zB, s.zPosB, O.NB, T(0));
    Load(O.volB, s.volB, O.NB, defVol); Load(O.psiB, s.psiB, O.NB, defPsi);
    O.idR.resize(O.NR); O.bodyR.resize(O.NR);
    for (uint32_t i = 0; i < O.NR; i++) { O.idR[i] = s.idR ? s.idR[i] : i; O.bodyR[i] = s.bodyIdR ? s.bodyIdR[i] : 0; }
    Load(O.xRel, s.xPosRelR, O.NR, T(0)); Load(O.yRel, s.yPosRelR, O.NR, T(0)); Load(O.zRel, s.zPosRelR, O.NR, T(0));
    Load(O.volR, s.volR, O.NR, defVol); Load(O.psiR, s.psiR, O.NR, defPsi);
    for (auto* v : {&O.xR, &O.yR, &O.zR, &O.vxR, &O.vyR, &O.vzR, &O.vpxR, &O.vpyR, &O.vpzR, &O.fxR, &O.fyR, &O.fzR})
        v->assign(O.NR, T(0));
    O.idRB.resize(O.NRB); O.cntRB.resize(O.NRB);
    for (uint32_t b = 0; b < O.NRB; b++) {
        O.idRB[b] = s.idRB ? s.idRB[b] : b;
        O.cntRB[b] = s.rigidParticleCountRB ? s.rigidParticleCountRB[b] : 0;
    }
    Load(O.cmx, s.xCM, O.NRB, T(0)); Load(O.cmy, s.yCM, O.NRB, T(0)); Load(O.cmz, s.zCM, O.NRB, T(0));
    Load(O.vx, s.xVelRB, O.NRB, T(0)); Load(O.vy, s.yVelRB, O.NRB, T(0)); Load(O.vz, s.zVelRB, O.NRB, T(0));
    Load(O.wx, s.xOmegaRB, O.NRB, T(0)); Load(O.wy, s.yOmegaRB, O.NRB, T(0)); Load(O.wz, s.zOmegaRB, O.NRB, T(0));
    Load(O.Lx, s.xAngMomRB, O.NRB, T(0)); Load(O.Ly, s.yAngMomRB, O.NRB, T(0)); Load(O.Lz, s.zAngMomRB, O.NRB, T(0));
    float* const aa[9] = {s.a00, s.a01, s.a02, s.a10, s.a11, s.a12, s.a20, s.a21, s.a22};
    float* const ib[9] = {s.iBodyInv00, s.iBodyInv01, s.iBodyInv02, s.iBodyInv10, s.iBodyInv11,
                          s.iBodyInv12, s.iBodyInv20, s.iBodyInv21, s.iBodyInv22};
    for (int k = 0; k < 9; k++) {
        Load(O.A[k], aa[k], O.NRB, (k % 4 == 0) ? T(1) : T(0));
        Load(O.Ib[k], ib[k], O.NRB, T(0));
    }
    Load(O.mass, s.massRB, O.NRB, T(0)); Load(O.massInv, s.massInvRB, O.NRB, T(0));
    for (auto* v : {&O.vpx, &O.vpy, &O.vpz, &O.wpx, &O.wpy, &O.wpz, &O.Lpx, &O.Lpy, &O.Lpz, &O.Fx, &O.Fy, &O.Fz,
                    &O.Tx, &O.Ty, &O.Tz})
        v->assign(O.NRB, T(0));
    O.frameValid = false; O.frameRebuilds = 0; O.cellSize = 0; O.reach = 1;
    O.BuildByBody();
    O.UpdateRigidParticles(false);
}

template <typename T> static void Push(Oracle<T>& O, tsp_state_view& s) {
    s.N_F = O.NF; s.N_B = O.NB; s.N_R = O.NR; s.N_RB = O.NRB; s.step = O.step; s.time = O.time;
    if (s.idF) std::memcpy(s.idF, O.idF.data(), O.NF * 8ull);
    Store(O.xF, s.xPosF, O.NF); Store(O.yF, s.yPosF, O.NF); Store(O.zF, s.zPosF, O.NF);
    Store(O.vxF, s.xVelF, O.NF); Store(O.vyF, s.yVelF, O.NF); Store(O.vzF, s.zVelF, O.NF);
    Store(O.vpxF, s.xVelPredF, O.NF); Store(O.vpyF, s.yVelPredF, O.NF); Store(O.vpzF, s.zVelPredF, O.NF);
    Store(O.axF, s.xAccPressF, O.NF); Store(O.ayF, s.yAccPressF, O.NF); Store(O.azF, s.zAccPressF, O.NF);
    Store(O.srcF, s.sourceTermF, O.NF); Store(O.diagF, s.diagElemF, O.NF);
    Store(O.presF, s.pressureF, O.NF); Store(O.densF, s.densityF, O.NF);
    if (s.idB) std::memcpy(s.idB, O.idB.data(), O.NB * 8ull);
    Store(O.xB, s.xPosB, O.NB); Store(O.yB, s.yPosB, O.NB); Store(O.zB, s.zPosB, O.NB);
    Store(O.volB, s.volB, O.NB); Store(O.psiB, s.psiB, O.NB);
    if (s.idR) std::memcpy(s.idR, O.idR.data(), O.NR * 8ull);
    if (s.bodyIdR) std::memcpy(s.bodyIdR, O.bodyR.data(), O.NR * 4ull);
    Store(O.xRel, s.xPosRelR, O.NR); Store(O.yRel, s.yPosRelR, O.NR); Store(O.zRel, s.zPosRelR, O.NR);
    Store(O.volR, s.volR, O.NR); Store(O.psiR, s.psiR, O.NR);
    Store(O.xR, s.xPosR, O.NR); Store(O.yR, s.yPosR, O.NR); Store(O.zR, s.zPosR, O.NR);
    if (s.idRB) std::memcpy(s.idRB, O.idRB.data(), O.NRB * 8ull);
    if (s.rigidParticleCountRB) std::memcpy(s.rigidParticleCountRB, O.cntRB.data(), O.NRB * 4ull);
    Store(O.cmx, s.xCM, O.NRB); Store(O.cmy, s.yCM, O.NRB); Store(O.cmz, s.zCM, O.NRB);
    Store(O.vx, s.xVelRB, O.NRB); Store(O.vy, s.yVelRB, O.NRB); Store(O.vz, s.zVelRB, O.NRB);
    Store(O.wx, s.xOmegaRB, O.NRB); Store(O.wy, s.yOmegaRB, O.NRB); Store(O.wz, s.zOmegaRB, O.NRB);
    Store(O.Lx, s.xAngMomRB, O.NRB); Store(O.Ly, s.yAngMomRB, O.NRB); Store(O.Lz, s.zAngMomRB, O.NRB);
    float* const aa[9] = {s.a00, s.a01, s.a02, s.a10, s.a11, s.a12, s.a20, s.a21, s.a22};
    float* const ib[9] = {s.iBodyInv00, s.iBodyInv01, s.iBodyInv02, s.iBodyInv10, s.iBodyInv11,
                          s.iBodyInv12, s.iBodyInv20, s.iBodyInv21, s.iBodyInv22};
    for (int k = 0; k < 9; k++) { Store(O.A[k], aa[k], O.NRB); Store(O.Ib[k], ib[k], O.NRB); }
    Store(O.mass, s.massRB, O.NRB); Store(O.massInv, s.massInvRB, O.NRB);
}

namespace orc {
// FillStatisticsRecord (gpu_backend.cpp:1067-1203): same record layout as tsp_b200_fill_statistics
template <typename T> static void FillStats(const Oracle<T>& O, const tsp_params& p, double* r) {
    std::memset(r, 0, sizeof(double) * TSP_STAT_COUNT);
    r[TSP_STAT_NUM_F] = O.NF; r[TSP_STAT_NUM_B] = O.NB; r[TSP_STAT_NUM_R] = O.NR;
    for (int k = 0; k < 6; k++) {
        const CSR& c = O.rows[k];
        const uint32_t n = k < 3 ? O.NF : O.NR;
        if (n == 0 || c.off.size() != (size_t)n + 1) continue;
        std::vector<uint32_t> cnt(n);
        for (uint32_t i = 0; i < n; i++) cnt[i] = (uint32_t)(c.off[i + 1] - c.off[i]);
        std::vector<uint32_t> srt = cnt;
        std::sort(srt.begin(), srt.end());
        r[TSP_STAT_NUM_NBR_FF_AVG + 4 * k] = (double)c.total() / (double)n;
        r[TSP_STAT_NUM_NBR_FF_MIN + 4 * k] = srt.front();
        r[TSP_STAT_NUM_NBR_FF_MAX + 4 * k] = srt.back();
        r[TSP_STAT_NUM_NBR_FF_P99 + 4 * k] = srt[(99ull * (uint64_t)(n - 1)) / 100ull];
    }
    double raw = 0, pos = 0, ab = 0, vs = 0;
    float vmin = 3.402823466e38f, vmax = 0.0f;
    for (uint32_t i = 0; i < O.NF; i++) {
        const float rel = ((float)O.densF[i] / p.restDensity) - 1.0f;
        raw += rel; pos += std::max(0.0f, rel); ab += std::fabs(rel);
        const float vx = (float)O.vxF[i], vy = (float)O.vyF[i], vz = (float)O.vzF[i];
        const float mag = std::sqrt(vx * vx + vy * vy + vz * vz);
        vs += mag; vmin = std::min(vmin, mag); vmax = std::max(vmax, mag);
    }
    const double inv = O.NF ? 1.0 / (double)O.NF : 0.0;
    r[TSP_STAT_DENS_REL_ERROR_RAW_AVG] = raw * inv;
    r[TSP_STAT_DENS_REL_ERROR_POS_AVG] = pos * inv;
    r[TSP_STAT_DENS_REL_ERROR_ABS_AVG] = ab * inv;
    r[TSP_STAT_NUM_SOLVER_ITERS] = O.iters;
    r[TSP_STAT_CFL_NUMBER] = (O.NF ? vmax : 0.0f) * p.timeStep / p.particleSizeF;
    r[TSP_STAT_VEL_MAG_AVG] = vs * inv;
    r[TSP_STAT_VEL_MAG_MIN] = O.NF ? vmin : 0.0f;
    r[TSP_STAT_VEL_MAG_MAX] = O.NF ? vmax : 0.0f;
}
// PackExportSnapshot (cpu_backend.cpp:829-975): FillFluidParticleNearSurfaceFlags +
// ClassifyExportSurfaceParticles + the ordered copy of the marked fluid particles
template <typename T> static void PackExport(const Oracle<T>& O, const tsp_params& p, bool includeB,
                                             uint64_t meshBegin, tsp_export_snapshot& o) {
    o.simStep = O.step;
    o.simTime = O.time;
    o.N_B = includeB ? O.NB : 0u;
    for (uint32_t i = 0; i < o.N_B; i++) {
        if (o.xPosB) o.xPosB[i] = (float)O.xB[i];
        if (o.yPosB) o.yPosB[i] = (float)O.yB[i];
        if (o.zPosB) o.zPosB[i] = (float)O.zB[i];
        if (o.volB) o.volB[i] = (float)O.volB[i];
        if (o.isMeshB) o.isMeshB[i] = (uint8_t)(O.idB[i] >= meshBegin);
    }
    o.N_R = O.NR;
    for (uint32_t i = 0; i < O.NR; i++) {
        if (o.bodyIdR) o.bodyIdR[i] = O.bodyR[i];
        if (o.xPosR) o.xPosR[i] = (float)O.xR[i];
        if (o.yPosR) o.yPosR[i] = (float)O.yR[i];
        if (o.zPosR) o.zPosR[i] = (float)O.zR[i];
        if (o.volR) o.volR[i] = (float)O.volR[i];
    }
    o.N_F = 0;
    const CSR& ff = O.rows[0];
    if (O.NF == 0 || ff.off.size() != (size_t)O.NF + 1) return;
    const uint32_t threshold = p.surfaceNbrCountThreshold ? p.surfaceNbrCountThreshold : 27u;
    auto count = [&](int k, uint32_t i) -> uint64_t {
        const CSR& c = O.rows[k];
        return c.off.size() == (size_t)O.NF + 1 ? c.off[i + 1] - c.off[i] : 0u;
    };
    std::vector<uint8_t> flag(O.NF, 0);
    for (uint32_t i = 0; i < O.NF; i++) {
        const uint64_t cFF = count(0, i), cFB = count(1, i), cFR = count(2, i);
        if (!(cFB > 0 || cFR > 0 || cFF < threshold)) continue;  // IsNearSurfaceFluidParticle
        flag[i] = 1;
        for (uint64_t k = ff.off[i]; k < ff.off[i + 1]; k++) flag[ff.idx[k]] = 1;
    }
    uint32_t dst = 0;
    for (uint32_t i = 0; i < O.NF; i++) {
        if (!flag[i]) continue;
        const float vx = (float)O.vxF[i], vy = (float)O.vyF[i], vz = (float)O.vzF[i];
        if (o.xPosF) o.xPosF[dst] = (float)O.xF[i];
        if (o.yPosF) o.yPosF[dst] = (float)O.yF[i];
        if (o.zPosF) o.zPosF[dst] = (float)O.zF[i];
        if (o.velMagF) o.velMagF[dst] = std::sqrt(vx * vx + vy * vy + vz * vz);
        dst++;
    }
    o.N_F = dst;
}
}  // namespace orc

extern "C" {

orc_handle* orc_create(const tsp_params* p, int fp64) {
    orc_handle* h = new orc_handle();
    h->fp64 = fp64;
    if (fp64) { h->d = new Oracle<double>(); h->d->prm = *p; }
    else { h->f = new Oracle<float>(); h->f->prm = *p; }
    return h;
}
void orc_destroy(orc_handle* h) { if (!h) return; delete h->f; delete h->d; delete h; }
const char* orc_last_error(orc_handle* h) { return h->err.c_str(); }
int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}

int orc_set_domain(orc_handle* h, const float* mn, const float* mx) {
    ORC_TRY(h, ORC_DISPATCH(h, { for (int a = 0; a < 3; a++) { O.domMin[a] = mn[a]; O.domMax[a] = mx[a]; } }))
}
int orc_pull_state(orc_handle* h, const tsp_state_view* s, const tsp_params* p) {
    ORC_TRY(h, ORC_DISPATCH(h, Pull(O, *s, *p)))
}
int orc_push_state(orc_handle* h, tsp_state_view* s) { ORC_TRY(h, ORC_DISPATCH(h, Push(O, *s))) }
int orc_neighbor_search(orc_handle* h, const tsp_params* p) {
    ORC_TRY(h, ORC_DISPATCH(h, { O.prm = *p; O.NeighborSearch(); }))
}
int orc_step(orc_handle* h, const tsp_params* p, uint32_t n) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        O.prm = *p;
        for (uint32_t s = 0; s < n; s++) { O.Step(); O.step += 1; O.time += (double)p->timeStep; }
    }))
}
int orc_fill_statistics(orc_handle* h, const tsp_params* p, double* r) {
    ORC_TRY(h, ORC_DISPATCH(h, orc::FillStats(O, *p, r)))
}
int orc_pack_export_snapshot(orc_handle* h, const tsp_params* p, int includeB, uint64_t meshBegin,
                             tsp_export_snapshot* o) {
    ORC_TRY(h, ORC_DISPATCH(h, orc::PackExport(O, *p, includeB != 0, meshBegin, *o)))
}
int orc_get_contact_report(orc_handle* h, tsp_contact_report* r) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        std::memset(r, 0, sizeof(*r));
        r->solverIters = O.contactIters;
        r->avgDensityError = (float)O.contactAvgErr;
        r->converged = O.contactConverged ? 1u : 0u;
        r->nContacts = O.contactCount;
        r->nContactBoundary = O.cLocalB.size();
    }))
}
int orc_get_stats(orc_handle* h, tsp_step_stats* st) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        std::memset(st, 0, sizeof(*st));
        st->step = O.step; st->time = O.time; st->solverIters = O.iters;
        st->errSumRaw = O.eRaw; st->errSumPos = O.ePos; st->errSumAbs = O.eAbs;
        st->avgRelDensityErrRaw = (float)O.avgRaw; st->avgRelDensityErrPos = (float)O.avgPos;
        st->avgRelDensityErrAbs = (float)O.avgAbs; st->frameRebuilds = O.frameRebuilds;
        st->cellOrig[0] = O.frame.ox; st->cellOrig[1] = O.frame.oy; st->cellOrig[2] = O.frame.oz;
        st->cellDims[0] = O.frame.nx; st->cellDims[1] = O.frame.ny; st->cellDims[2] = O.frame.nz;
        st->keyBits = KeyBits(O.frame);
        st->nCellsF = (uint32_t)O.uniqF.size(); st->nCellsB = (uint32_t)O.uniqB.size(); st->nCellsR = (uint32_t)O.uniqR.size();
        st->nNbrFF = O.rows[0].total(); st->nNbrFB = O.rows[1].total(); st->nNbrFR = O.rows[2].total();
        st->nNbrRF = O.rows[3].total(); st->nNbrRB = O.rows[4].total(); st->nNbrRR = O.rows[5].total();
    }))
}
int orc_read_cell_ids(orc_handle* h, uint32_t species, uint64_t* out, uint32_t n) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        const auto& v = species == 0 ? O.cidF : species == 1 ? O.cidB : O.cidR;
        if (n != v.size()) throw std::runtime_error("size mismatch");
        std::memcpy(out, v.data(), n * 8ull);
    }))
}
int orc_read_permutation(orc_handle* h, uint32_t species, uint32_t* out, uint32_t n) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        const auto& v = species == 0 ? O.permF : species == 1 ? O.permB : O.permR;
        if (n != v.size()) throw std::runtime_error("size mismatch");
        std::memcpy(out, v.data(), n * 4ull);
    }))
}
int orc_read_cell_table(orc_handle* h, uint32_t species, uint64_t* uniq, uint32_t* start, uint32_t cap, uint32_t* nc) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        const auto& u = species == 0 ? O.uniqF : species == 1 ? O.uniqB : O.uniqR;
        const auto& s = species == 0 ? O.startF : species == 1 ? O.startB : O.startR;
        *nc = (uint32_t)u.size();
        if (uniq && start) {
            if (cap < u.size()) throw std::runtime_error("capacity");
            std::memcpy(uniq, u.data(), u.size() * 8ull);
            std::memcpy(start, s.data(), s.size() * 4ull);
        }
    }))
}
int orc_read_rows(orc_handle* h, uint32_t list, uint64_t* off, uint32_t nsrc, uint32_t* idx, uint64_t cap, uint64_t* total) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        const CSR& r = O.rows[list];
        *total = r.total();
        if (off) {
            if (nsrc + 1 != r.off.size()) throw std::runtime_error("size mismatch");
            std::memcpy(off, r.off.data(), r.off.size() * 8ull);
        }
        if (idx) {
            if (cap < r.idx.size()) throw std::runtime_error("capacity");
            std::memcpy(idx, r.idx.data(), r.idx.size() * 4ull);
        }
    }))
}
// SELL32 encoding of the oracle rows (reference GPU rule)
int orc_encode_sell32(orc_handle* h, uint32_t list, uint16_t* counts, uint16_t* pitch, uint8_t* fmt,
                      uint32_t* base, uint32_t* base2, uint64_t* offs, uint32_t nchunks,
                      uint16_t* w16, uint64_t n16cap, uint32_t* w32, uint64_t n32cap, uint64_t* n16, uint64_t* n32) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        Sell32 s;
        EncodeSell32(O.rows[list], O.NF, list == 0, s);
        *n16 = s.w16.size(); *n32 = s.w32.size();
        if (counts) {
            if (nchunks != s.pitch.size()) throw std::runtime_error("chunk count mismatch");
            std::memcpy(counts, s.counts.data(), s.counts.size() * 2ull);
            std::memcpy(pitch, s.pitch.data(), nchunks * 2ull);
            std::memcpy(fmt, s.format.data(), nchunks);
            std::memcpy(base, s.base.data(), nchunks * 4ull);
            std::memcpy(base2, s.base2.data(), nchunks * 4ull);
            std::memcpy(offs, s.offset.data(), nchunks * 8ull);
        }
        if (w16 && n16cap >= s.w16.size()) std::memcpy(w16, s.w16.data(), s.w16.size() * 2ull);
        if (w32 && n32cap >= s.w32.size()) std::memcpy(w32, s.w32.data(), s.w32.size() * 4ull);
    }))
}
// stage access mirroring tsp_b200_run_stage
int orc_run_stage(orc_handle* h, const tsp_params* p, uint32_t stage, double* err) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        O.prm = *p;
        switch (stage) {
            case TSP_STAGE_DENSITY: O.Density(); break;
            case TSP_STAGE_NON_PRESSURE: O.NonPressure(); break;
            case TSP_STAGE_SOURCE_DIAG_INIT: O.SourceDiagInit(); break;
            case TSP_STAGE_PRESSURE_ACC: O.PressureAcc(); break;
            case TSP_STAGE_JACOBI_UPDATE:
                O.JacobiUpdate();
                if (err) { err[0] = O.eRaw; err[1] = O.ePos; err[2] = O.eAbs; }
                break;
            case TSP_STAGE_INTEGRATION: O.Integration(); break;
            case TSP_STAGE_BOUNDARY_VOLUMES:
                decltype(O.volB)* vb = &O.volB;
                O.Coefficients(O.xB, O.yB, O.zB, 0, O.NB, O.prm, O.sizeInv(), O.alpha(), *vb, O.psiB);
                for (uint32_t b = 0; b < O.NRB; b++)
                    O.Coefficients(O.xRel, O.yRel, O.zRel, O.byBodyOff[b], O.byBodyOff[b + 1], O.prm, O.sizeInv(),
                                   O.alpha(), O.volR, O.psiR);
                break;
        }
    }))
}
// interleaved field access (doubles), mirroring tsp_b200_read_field / write_field
int orc_read_field(orc_handle* h, uint32_t field, double* out, uint32_t n) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        auto put3 = [&](const auto& X, const auto& Y, const auto& Z) {
            for (uint32_t i = 0; i < n; i++) { out[3 * i] = X[i]; out[3 * i + 1] = Y[i]; out[3 * i + 2] = Z[i]; }
        };
        auto put1 = [&](const auto& X) { for (uint32_t i = 0; i < n; i++) out[i] = X[i]; };
        switch (field) {
            case TSP_FIELD_POS: put3(O.xF, O.yF, O.zF); break;
            case TSP_FIELD_VEL: put3(O.vxF, O.vyF, O.vzF); break;
            case TSP_FIELD_VEL_PRED: put3(O.vpxF, O.vpyF, O.vpzF); break;
            case TSP_FIELD_ACC_PRESS: put3(O.axF, O.ayF, O.azF); break;
            case TSP_FIELD_SOURCE: put1(O.srcF); break;
            case TSP_FIELD_DIAG: put1(O.diagF); break;
            case TSP_FIELD_PRESSURE: put1(O.presF); break;
            case TSP_FIELD_DENSITY: put1(O.densF); break;
            case TSP_FIELD_VOL_B: put1(O.volB); break;
            case TSP_FIELD_PSI_B: put1(O.psiB); break;
            case TSP_FIELD_VOL_R: put1(O.volR); break;
            case TSP_FIELD_PSI_R: put1(O.psiR); break;
            case TSP_FIELD_FORCE_R: put3(O.fxR, O.fyR, O.fzR); break;
            case TSP_FIELD_BODY_FT:
                for (uint32_t b = 0; b < n; b++) {
                    out[6 * b] = O.Fx[b]; out[6 * b + 1] = O.Fy[b]; out[6 * b + 2] = O.Fz[b];
                    out[6 * b + 3] = O.Tx[b]; out[6 * b + 4] = O.Ty[b]; out[6 * b + 5] = O.Tz[b];
                }
                break;
            default: throw std::runtime_error("unknown field");
        }
    }))
}
int orc_write_field(orc_handle* h, uint32_t field, const double* in, uint32_t n) {
    ORC_TRY(h, ORC_DISPATCH(h, {
        using TT = std::remove_reference_t<decltype(O.xF[0])>;
        auto get3 = [&](auto& X, auto& Y, auto& Z) {
            for (uint32_t i = 0; i < n; i++) { X[i] = (TT)in[3 * i]; Y[i] = (TT)in[3 * i + 1]; Z[i] = (TT)in[3 * i + 2]; }
        };
        auto get1 = [&](auto& X) { for (uint32_t i = 0; i < n; i++) X[i] = (TT)in[i]; };
        switch (field) {
            case TSP_FIELD_POS: get3(O.xF, O.yF, O.zF); break;
            case TSP_FIELD_VEL: get3(O.vxF, O.vyF, O.vzF); break;
            case TSP_FIELD_VEL_PRED: get3(O.vpxF, O.vpyF, O.vpzF); break;
            case TSP_FIELD_ACC_PRESS: get3(O.axF, O.ayF, O.azF); break;
            case TSP_FIELD_SOURCE: get1(O.srcF); break;
            case TSP_FIELD_DIAG: get1(O.diagF); break;
            case TSP_FIELD_PRESSURE: get1(O.presF); break;
            case TSP_FIELD_DENSITY: get1(O.densF); break;
            case TSP_FIELD_VOL_B: get1(O.volB); break;
            case TSP_FIELD_PSI_B: get1(O.psiB); break;
            case TSP_FIELD_VOL_R: get1(O.volR); break;
            case TSP_FIELD_PSI_R: get1(O.psiR); break;
            default: throw std::runtime_error("field is not writable");
        }
    }))
}
// closed-form kernel values (the reference's tests/unit/sph_kernels.cpp checks these)
void orc_kernel_eval(float dx, float dy, float dz, float sizeInv, float radSqu, float alpha, float* out5) {
    out5[0] = KernelWeight<float>(dx, dy, dz, sizeInv, radSqu, alpha);
    const KConst<float> k = MakeKConst<float>(sizeInv, alpha);
    const float d2 = std::fma(dx, dx, std::fma(dy, dy, dz * dz));
    out5[1] = GradFac<float>(d2, k);
    float gx, gy, gz;
    GradScalar<float>(dx, dy, dz, sizeInv, radSqu, alpha, gx, gy, gz);
    out5[2] = gx; out5[3] = gy; out5[4] = gz;
}

}  // extern "C"
