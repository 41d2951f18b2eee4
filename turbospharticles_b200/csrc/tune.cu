// tune.cu -- autotuner of the launch configurations of the hot kernels.
//
// The neighbor sweeps (density, non-pressure, source/diagonal, pressure acceleration, Jacobi)
// and the two fluid-query passes are compiled in several configurations each: FF list slots per
// pipelined group (the sweeps' loads in flight) and the minimum resident blocks per SM of
// __launch_bounds__ (which sets the register budget and so the occupancy). Which one is fastest
// depends on the scene (neighbor counts, list formats) and the GPU, so it is measured, not set:
// the first time a kernel runs for a size class (particle count rounded to a power of two, all
// counts from 2^20 up in one class) on a device, the caller hands TuneRun a launcher and every
// candidate is timed on the live state (its first 2^20 particles at most) --
// one warm-up launch, then three launches between CUDA events on the caller's stream -- and the
// fastest is kept for that class. Candidates change register allocation and load grouping, never
// the order of a sum, so the choice does not change any result bit.
//
// The reference has no counterpart (its CUDA kernels use one fixed block size,
// source/simulation/GPU/backend/common.cuh:13-14).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.h"

namespace tsp {
namespace {

constexpr int kClasses = 33;  // size class = bit length of n

struct TuneEntry {
    int choice = -1;
    float bestMs = 0.f, defaultMs = 0.f, worstMs = 0.f;
    uint32_t n = 0;
};
struct DeviceTable {
    TuneEntry e[TUNE_KERNELS][kClasses];
};

std::mutex g_mutex;
std::map<int, DeviceTable> g_tables;
bool g_enabled = true;

int CurrentDevice() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}
int SizeClass(uint32_t n) {  // bit length of n, sizes from TUNE_MAX_N up share one class
    if (n > TUNE_MAX_N) n = TUNE_MAX_N;
    int b = 0;
    while (n) { b++; n >>= 1; }
    return b;
}

const char* kNames[TUNE_KERNELS] = {"KDensity", "KNonPressure", "KSourceDiagInit", "KPressureAcc", "KJacobi",
                                    "KQueryFluidCount", "KQueryFluidFill"};

}  // namespace

const TuneCandidate* TuneCandidates(TuneKernel k, int* n) {
    if (k == TUNE_QUERY_COUNT) return QueryCandidates(false, n);
    if (k == TUNE_QUERY_FILL) return QueryCandidates(true, n);
    return SweepCandidates(n);
}
const char* TuneKernelName(TuneKernel k) { return (k >= 0 && k < TUNE_KERNELS) ? kNames[k] : "?"; }
int TuneDefault(TuneKernel) { return 0; }

int TuneChoice(TuneKernel k, uint32_t n) {
    std::lock_guard<std::mutex> lock(g_mutex);
    auto it = g_tables.find(CurrentDevice());
    if (it == g_tables.end()) return -1;
    return it->second.e[k][SizeClass(n)].choice;
}
bool TuneEnabled() {
    std::lock_guard<std::mutex> lock(g_mutex);
    return g_enabled;
}
void SetTuneEnabled(bool on) {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_enabled = on;
}
void TuneReset() {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_tables.clear();
}

int TuneRun(TuneKernel k, uint32_t n, const std::function<void(int)>& launch, cudaStream_t s) {
    int nc = 0;
    const TuneCandidate* cand = TuneCandidates(k, &nc);
    (void)cand;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return TuneDefault(k);
    if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return TuneDefault(k); }
    constexpr int kReps = 3;
    std::vector<float> ms(nc, INFINITY);
    for (int i = 0; i < nc; i++) {
        launch(i);  // warm-up (module load, caches)
        cudaEventRecord(e0, s);
        for (int r = 0; r < kReps; r++) launch(i);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) continue;
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms[i] = t / kReps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int best = TuneDefault(k);
    for (int i = 0; i < nc; i++)
        if (ms[i] < ms[best]) best = i;
    float worst = 0.f;
    for (int i = 0; i < nc; i++)
        if (std::isfinite(ms[i])) worst = std::max(worst, ms[i]);
    std::lock_guard<std::mutex> lock(g_mutex);
    TuneEntry& e = g_tables[CurrentDevice()].e[k][SizeClass(n)];
    e.choice = best;
    e.bestMs = ms[best];
    e.defaultMs = ms[TuneDefault(k)];
    e.worstMs = worst;
    e.n = n;
    return best;
}

bool TuneSet(const char* kernel, uint32_t n, uint32_t slots, uint32_t minBlocks) {
    for (int k = 0; k < TUNE_KERNELS; k++) {
        if (std::string(kNames[k]) != kernel) continue;
        int nc = 0;
        const TuneCandidate* cand = TuneCandidates((TuneKernel)k, &nc);
        for (int c = 0; c < nc; c++) {
            if (cand[c].slots != slots || cand[c].minBlocks != minBlocks) continue;
            std::lock_guard<std::mutex> lock(g_mutex);
            TuneEntry& e = g_tables[CurrentDevice()].e[k][SizeClass(n)];
            e = TuneEntry{};
            e.choice = c;
            e.n = n;
            return true;
        }
    }
    return false;
}

std::string TuneReport() {
    std::lock_guard<std::mutex> lock(g_mutex);
    std::string out = "{";
    auto it = g_tables.find(CurrentDevice());
    bool first = true;
    if (it != g_tables.end()) {
        for (int k = 0; k < TUNE_KERNELS; k++) {
            int nc = 0;
            const TuneCandidate* cand = TuneCandidates((TuneKernel)k, &nc);
            for (int c = 0; c < kClasses; c++) {
                const TuneEntry& e = it->second.e[k][c];
                if (e.choice < 0) continue;
                char buf[320];
                std::snprintf(buf, sizeof(buf),
                              "%s\"%s/n%u\": {\"slots\": %u, \"min_blocks\": %u, \"ms\": %.4f, \"untuned_ms\": %.4f, "
                              "\"worst_ms\": %.4f, \"candidates\": %d}",
                              first ? "" : ", ", kNames[k], e.n, cand[e.choice].slots, cand[e.choice].minBlocks,
                              e.bestMs, e.defaultMs, e.worstMs, nc);
                out += buf;
                first = false;
            }
        }
    }
    out += "}";
    return out;
}

}  // namespace tsp
