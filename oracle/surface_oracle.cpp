// surface_oracle.cpp -- TEST INFRASTRUCTURE ONLY: sequential CPU restatement of the reference's
// mesh surface sampler (Scene::SurfaceSampler, source/simulation/scene/geometry/
// surface_sampling.cpp), the oracle of tsp_b200_sample_surface. Compiled with
// -ffp-contract=off: every product and sum is rounded as written.
//
// The reference tests one cell phase group of a candidate round in parallel against the sample
// set of the group's start and then inserts the accepted candidates in cell order
// (surface_sampling.cpp:744-800); two cells of one phase group are never within each other's
// 3x3x3 query, so testing the group's cells one after another against the growing set gives
// the same decisions -- this file does that. Coverage probes are tested per batch of 10^6
// against the set of the batch start and repaired in probe order (:889-960), as the reference.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../include/tsp_b200.h"

namespace {

struct V3 { float x, y, z; };
inline V3 Sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 Scale(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 Add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline float Dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }  // glm::dot order
inline float Length(V3 a) { return std::sqrt(Dot(a, a)); }
inline V3 Cross(V3 a, V3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }

struct Tri { V3 v0, v1, v2; float area; double cum; float longestEdge; };

inline uint64_t Mix(uint64_t h) {  // splitmix64 finalizer (surface_sampling.cpp:54-59)
    h = (h ^ (h >> 30)) * 0xbf58476d1ce4e5b9ull;
    h = (h ^ (h >> 27)) * 0x94d049bb133111ebull;
    return h ^ (h >> 31);
}
inline double Random01(uint64_t seed, uint64_t streamIdx) {
    const uint64_t h = Mix(seed + (streamIdx + 1ull) * 0x9e3779b97f4a7c15ull);
    return (double)(h >> 11) * 0x1.0p-53;
}
inline float DistanceEpsilon(float d) {
    return 32.0f * std::numeric_limits<float>::epsilon() * std::max(std::fabs(d), std::numeric_limits<float>::min());
}
struct Cell { int32_t x, y, z; };
inline int32_t Axis(float v, float inv) {
    const double s = std::floor((double)v * (double)inv);  // exact product of two floats
    if (!std::isfinite(s) || s < (double)INT32_MIN || s > (double)INT32_MAX)
        throw std::runtime_error("Surface sample grid coordinate exceeds int32 limits.");
    return (int32_t)s;
}
inline Cell CellOf(V3 p, float inv) { return {Axis(p.x, inv), Axis(p.y, inv), Axis(p.z, inv)}; }
inline uint64_t CellKey(Cell c) {
    return ((uint64_t)(uint32_t)c.x * 0x9E3779B97F4A7C15ull) ^ Mix((uint64_t)(uint32_t)c.y) ^
           (Mix((uint64_t)(uint32_t)c.z ^ 0x5bd1e995ull) << 1);
}
inline V3 Point(const Tri& t, V3 b) { return Add(Add(Scale(t.v0, b.x), Scale(t.v1, b.y)), Scale(t.v2, b.z)); }

struct Hash {  // cell -> sample indices, 3x3x3 queries
    float inv;
    const std::vector<V3>& samples;
    std::unordered_map<uint64_t, std::vector<std::pair<Cell, uint32_t>>> cells;
    Hash(float cellSize, const std::vector<V3>& s) : inv(1.0f / cellSize), samples(s) {}
    void Insert(uint32_t i) {
        const Cell c = CellOf(samples[i], inv);
        cells[CellKey(c)].push_back({c, i});
    }
    template <class F> bool Any(V3 p, F&& f) const {
        const Cell c = CellOf(p, inv);
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const Cell q{c.x + dx, c.y + dy, c.z + dz};
                    auto it = cells.find(CellKey(q));
                    if (it == cells.end()) continue;
                    for (const auto& e : it->second)
                        if (e.first.x == q.x && e.first.y == q.y && e.first.z == q.z && f(e.second)) return true;
                }
        return false;
    }
};

inline uint32_t Phase(Cell c) { return (uint32_t)((c.x & 1) | ((c.y & 1) << 1) | ((c.z & 1) << 2)); }

std::vector<V3> Sample(const float* vtx, uint32_t nV, const uint32_t* tri, uint32_t nT,
                       const tsp_surface_sampling_params& p, tsp_surface_sampling_stats& st) {
    const float minD = p.minDistance, maxD = p.maxDistance, probeS = p.coverageProbeSpacing;
    // PreprocessMesh (surface_sampling.cpp:455-578)
    if (nV == 0 || nT == 0) throw std::runtime_error("Cannot sample an empty triangle surface.");
    if (!std::isfinite(p.particleSizeF) || p.particleSizeF <= 0.0f)
        throw std::runtime_error("Surface sampling requires a finite positive fluid particle size.");
    if (maxD > p.particleSizeF + DistanceEpsilon(p.particleSizeF))
        throw std::runtime_error("Surface sampling is coarser than the fluid spacing.");
    if (!std::isfinite(minD) || minD <= 0.0f) throw std::runtime_error("Surface sample minimum distance must be finite and positive.");
    if (!std::isfinite(maxD) || maxD < minD)
        throw std::runtime_error("Surface sample maximum distance must be finite and not smaller than the minimum distance.");
    if (!std::isfinite(probeS) || probeS <= 0.0f) throw std::runtime_error("Surface coverage probe spacing must be finite and positive.");
    if (maxD + DistanceEpsilon(maxD) < minD + probeS)
        throw std::runtime_error("Surface coverage maximum distance must be at least the minimum distance plus the probe spacing.");
    if (p.candidateMultiplier == 0) throw std::runtime_error("Surface sampling candidate multiplier must be positive.");
    for (uint32_t i = 0; i < 3 * nV; i++)
        if (!std::isfinite(vtx[i])) throw std::runtime_error("Triangle surface contains a non-finite vertex.");
    for (uint32_t i = 0; i < 3 * nT; i++)
        if (tri[i] >= nV) throw std::runtime_error("Triangle surface contains an invalid vertex index.");
    std::vector<Tri> T(nT);
    double area = 0.0;
    for (uint32_t t = 0; t < nT; t++) {
        auto V = [&](uint32_t k) { return V3{vtx[3 * k], vtx[3 * k + 1], vtx[3 * k + 2]}; };
        const V3 v0 = V(tri[3 * t]), v1 = V(tri[3 * t + 1]), v2 = V(tri[3 * t + 2]);
        const float a = 0.5f * Length(Cross(Sub(v1, v0), Sub(v2, v0)));
        T[t] = {v0, v1, v2, a, 0.0,
                std::max(Length(Sub(v1, v0)), std::max(Length(Sub(v2, v1)), Length(Sub(v0, v2))))};
        if (!std::isfinite(a) || a <= 0.0f) throw std::runtime_error("Triangle surface contains a degenerate triangle.");
        area += (double)a;
        if (!std::isfinite(area) || area > std::numeric_limits<float>::max())
            throw std::runtime_error("Triangle surface area exceeds float limits.");
        T[t].cum = area;
    }
    st = tsp_surface_sampling_stats{};
    st.surfaceArea = (float)area;
    // SelectPoissonSamples (:580-813)
    const double nEstD = std::ceil(area / ((double)minD * (double)minD));
    if (!std::isfinite(nEstD) || nEstD < 0.0 || nEstD > (double)UINT32_MAX)
        throw std::runtime_error("Surface estimated sample count exceeds uint32 limits.");
    const uint64_t nCand = std::max<uint64_t>(1, (uint64_t)nEstD * p.candidateMultiplier);
    st.N_candidates = nCand;
    const uint32_t nEst = std::max<uint32_t>(1, (uint32_t)nEstD);
    const uint32_t batchMax = (uint32_t)std::min<uint64_t>(nCand, std::min<uint32_t>(1000000u, std::max<uint32_t>(1, nEst / 16)));
    const float inv = 1.0f / minD;
    std::vector<V3> acc;
    Hash hash(minD, acc);
    std::vector<V3> cand;
    std::vector<Cell> cc;
    std::vector<uint32_t> order;
    for (uint64_t begin = 0; begin < nCand;) {
        const uint32_t nb = (uint32_t)std::min<uint64_t>(nCand - begin, batchMax);
        cand.resize(nb); cc.resize(nb); order.resize(nb);
        for (uint32_t b = 0; b < nb; b++) {
            const uint64_t s = 3ull * (begin + b);
            const double target = Random01(p.seed, s) * area;
            const float scale = std::sqrt((float)Random01(p.seed, s + 1));
            const float off = (float)Random01(p.seed, s + 2);
            uint32_t lo = 0, hi = nT;  // lower_bound: first cum >= target
            while (lo < hi) { const uint32_t m = (lo + hi) / 2; if (T[m].cum < target) lo = m + 1; else hi = m; }
            const uint32_t t = lo == nT ? nT - 1 : lo;
            const float b1 = scale * (1.0f - off);
            cand[b] = Point(T[t], V3{1.0f - scale, b1, scale - b1});
            cc[b] = CellOf(cand[b], inv);
            order[b] = b;
        }
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
            const Cell A = cc[a], B = cc[b];
            if (Phase(A) != Phase(B)) return Phase(A) < Phase(B);
            if (A.z != B.z) return A.z < B.z;
            if (A.y != B.y) return A.y < B.y;
            return A.x < B.x;
        });
        std::vector<uint32_t> cellBegin;
        for (uint32_t k = 0; k < nb; k++) {
            const Cell a = cc[order[k]];
            if (k == 0) { cellBegin.push_back(0); continue; }
            const Cell b = cc[order[k - 1]];
            if (a.x != b.x || a.y != b.y || a.z != b.z) cellBegin.push_back(k);
        }
        const uint32_t nCells = (uint32_t)cellBegin.size();
        cellBegin.push_back(nb);
        uint32_t groupBegin[9];
        for (uint32_t g = 0; g <= 8; g++) {
            uint32_t c = 0;
            while (c < nCells && Phase(cc[order[cellBegin[c]]]) < g) c++;
            groupBegin[g] = c;
        }
        uint32_t maxPer = 0;
        for (uint32_t c = 0; c < nCells; c++) maxPer = std::max(maxPer, cellBegin[c + 1] - cellBegin[c]);
        const bool reversed = (begin / batchMax) % 2 == 1;
        for (uint32_t r = 0; r < maxPer; r++)
            for (uint32_t step = 0; step < 8; step++) {
                const uint32_t g = reversed ? 7 - step : step;
                for (uint32_t c = groupBegin[g]; c < groupBegin[g + 1]; c++) {
                    const uint32_t k = cellBegin[c] + r;
                    if (k >= cellBegin[c + 1]) continue;
                    const V3 q = cand[order[k]];
                    const bool conflict = hash.Any(q, [&](uint32_t i) { return Length(Sub(acc[i], q)) < minD; });
                    if (conflict) continue;
                    if (acc.size() >= (size_t)INT32_MAX) throw std::runtime_error("Surface sample count exceeds the local particle limit.");
                    acc.push_back(q);
                    hash.Insert((uint32_t)acc.size() - 1);
                }
            }
        begin += nb;
    }
    st.N_initialSamples = (uint32_t)acc.size();
    // RepairCoverage (:833-968)
    std::vector<uint32_t> sub(nT);
    std::vector<uint64_t> pb(nT + 1, 0);
    for (uint32_t t = 0; t < nT; t++) {
        const double d = std::ceil(T[t].longestEdge / probeS);
        if (!std::isfinite(d) || d >= (double)UINT32_MAX) throw std::runtime_error("Surface probe subdivision count exceeds uint32 loop limits.");
        sub[t] = std::max<uint32_t>(1, (uint32_t)d);
        pb[t + 1] = pb[t] + (uint64_t)(sub[t] + 1ull) * (sub[t] + 2ull) / 2ull;
    }
    const uint64_t nProbes = pb[nT];
    st.N_coverageProbes = nProbes;
    const float target = std::max(minD, maxD - probeS);
    Hash cover(target, acc);
    for (uint32_t i = 0; i < (uint32_t)acc.size(); i++) cover.Insert(i);
    auto probeAt = [&](uint32_t t, uint32_t i, uint32_t j) {
        const uint32_t n = sub[t];
        const float ninv = 1.0f / (float)n;
        const uint32_t k = n - i - j;
        return Point(T[t], V3{(float)i * ninv, (float)j * ninv, (float)k * ninv});
    };
    auto covered = [&](V3 q) { return cover.Any(q, [&](uint32_t s) { return Length(Sub(acc[s], q)) <= target; }); };
    uint32_t repairs = 0;
    uint32_t t = 0, i = 0, j = 0;
    std::vector<std::array<uint32_t, 3>> unc;
    for (uint64_t begin = 0; begin < nProbes;) {
        const uint64_t end = begin + std::min<uint64_t>(nProbes - begin, 1000000ull);
        unc.clear();
        for (uint64_t q = begin; q < end; q++) {
            if (!covered(probeAt(t, i, j))) unc.push_back({t, i, j});
            if (++j <= sub[t] - i) continue;
            j = 0;
            if (++i <= sub[t]) continue;
            i = 0;
            ++t;
        }
        for (const auto& u : unc) {
            const V3 q = probeAt(u[0], u[1], u[2]);
            if (covered(q)) continue;
            if (acc.size() >= (size_t)INT32_MAX) throw std::runtime_error("Repaired surface sample count exceeds the local particle limit.");
            acc.push_back(q);
            cover.Insert((uint32_t)acc.size() - 1);
            repairs++;
        }
        begin = end;
    }
    st.N_coverageRepairs = repairs;
    if (acc.empty()) throw std::runtime_error("Surface sampling produced no samples.");
    return acc;
}

thread_local std::string g_err;

}  // namespace

extern "C" {

const char* orc_surface_last_error() { return g_err.c_str(); }

int orc_sample_surface(const float* vtx, uint32_t nV, const uint32_t* tri, uint32_t nT,
                       const tsp_surface_sampling_params* p, float* out, uint64_t cap, uint64_t* nOut,
                       tsp_surface_sampling_stats* stats) {
    try {
        tsp_surface_sampling_stats st{};
        const std::vector<V3> s = Sample(vtx, nV, tri, nT, *p, st);
        if (stats) *stats = st;
        *nOut = s.size();
        if (s.size() > cap) return TSP_ERR_OVERFLOW;
        for (size_t k = 0; k < s.size(); k++) { out[3 * k] = s[k].x; out[3 * k + 1] = s[k].y; out[3 * k + 2] = s[k].z; }
        return TSP_OK;
    } catch (const std::exception& e) {
        g_err = e.what();
        return TSP_ERR_INVALID;
    }
}

}  // extern "C"
