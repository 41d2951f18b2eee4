// noalloc.cu -- cell-table build that allocates no device memory.
//
// Who needs it: a caller that owns the particle buffers and drives its own stream but must
// not allocate on the way -- a fixed-budget embedding that sizes every buffer up front, or a
// time-critical loop where a cudaMalloc / cudaFree (cudaFree synchronises the whole device)
// would stall the other work on the GPU. The handle-based entry points keep grow-only pools
// inside their backend object; this one has no handle, so the scan's scratch is a fixed-size
// array in the library's own device memory (`g_cellTableScratch` below) instead.
//
// The computation is the compact cell table of the neighbor build, the same kernels that
// tsp_b200_neighbor_search runs: run starts of the sorted Morton cell IDs by a device-wide
// exclusive scan of the "new cell" flags (source/simulation/CPU/backend/neighbor_search.cpp
// builds the same table sequentially from the sorted cell IDs).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/tsp_b200.h"
#include "kernels.h"
#include "primitives.cuh"

namespace tsp {
namespace {

// Largest particle count one call accepts, and the scan scratch that count needs: one
// uint64 partial per 1024-item tile plus one (16,385 words = 128 KiB for 2^24 particles).
constexpr uint32_t kNoAllocMaxParticles = TSP_NOALLOC_MAX_PARTICLES;
constexpr uint64_t kNoAllocScratchItems = (kNoAllocMaxParticles + SCAN_TILE - 1) / SCAN_TILE + 1;
static_assert(kNoAllocScratchItems >= 12, "scratch holds the setup build's partial, input and outputs");

// One scratch per device (each device that loads this library has its own copy of a
// __device__ variable). Nothing in it has to start at zero: each call writes every word it
// reads before reading it. Two calls in flight at the same time on one device (different
// streams or host threads without ordering between them) share it and race.
static __device__ __align__(256) uint64_t g_cellTableScratch[kNoAllocScratchItems];

constexpr int kMaxDevices = 64;
std::atomic<uint64_t*> g_scratchAddr[kMaxDevices];
std::mutex g_setupMutex;
thread_local std::string g_noAllocError;

int Fail(int code, const std::string& msg) {
    g_noAllocError = msg;
    return code;
}

// Device address of the scratch on the current device, looked up once per device, followed by
// one small build that loads the scan kernels on that device. Both may load device code (and
// so take device memory for it), which is why they belong in setup, before any time-critical
// section. The setup build runs on the legacy default stream and waits for it.
int ScratchForCurrentDevice(uint64_t** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return Fail(TSP_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return Fail(TSP_ERR_UNSUPPORTED, "device ordinal above 63");
    uint64_t* p = g_scratchAddr[dev].load(std::memory_order_acquire);
    if (!p) {
        std::lock_guard<std::mutex> lock(g_setupMutex);
        p = g_scratchAddr[dev].load(std::memory_order_relaxed);
        if (!p) {
            void* addr = nullptr;
            e = cudaGetSymbolAddress(&addr, g_cellTableScratch);
            if (e != cudaSuccess || !addr)
                return Fail(TSP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            p = static_cast<uint64_t*>(addr);
            // One n = 1 build on this device, its input and outputs carved out of the scratch
            // beyond the one tile partial it needs: with lazy module loading (the CUDA 12
            // default) this loads the scan kernels now, so no later call loads device code.
            uint64_t* cid = p + 8;
            uint32_t* start = reinterpret_cast<uint32_t*>(p + 10);
            e = cudaMemsetAsync(cid, 0, sizeof(uint64_t), 0);
            if (e == cudaSuccess) {
                BuildCellTable(cid, 1u, p + 9, start, p + 11, p, 0);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(0);
            if (e != cudaSuccess)
                return Fail(TSP_ERR_CUDA, std::string("noalloc setup build: ") + cudaGetErrorString(e));
            g_scratchAddr[dev].store(p, std::memory_order_release);
        }
    }
    *out = p;
    return TSP_OK;
}

}  // namespace
}  // namespace tsp

extern "C" {

int tsp_b200_noalloc_setup(void) {
    uint64_t* p = nullptr;
    return tsp::ScratchForCurrentDevice(&p);
}

int tsp_b200_build_cell_table_noalloc(const uint64_t* d_cell_ids_sorted, uint32_t n, uint64_t* d_unique_out,
                                      uint32_t* d_start_out, uint64_t* d_num_cells_out, void* stream) {
    using namespace tsp;
    if (n > kNoAllocMaxParticles)
        return Fail(TSP_ERR_INVALID, "tsp_b200_build_cell_table_noalloc: n = " + std::to_string(n) +
                                         " exceeds TSP_NOALLOC_MAX_PARTICLES = " +
                                         std::to_string(kNoAllocMaxParticles));
    if (!d_num_cells_out || (n > 0 && (!d_cell_ids_sorted || !d_unique_out || !d_start_out)))
        return Fail(TSP_ERR_INVALID, "tsp_b200_build_cell_table_noalloc: NULL device pointer");
    uint64_t* scratch = nullptr;
    const int rc = ScratchForCurrentDevice(&scratch);
    if (rc != TSP_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // an error left pending by the caller's earlier work is neither reported nor cleared here;
    // only an error that appears with this call's launches is
    const cudaError_t before = cudaPeekAtLastError();
    if (n == 0 && d_start_out) cudaMemsetAsync(d_start_out, 0, sizeof(uint32_t), s);  // start[0] = n = 0
    BuildCellTable(d_cell_ids_sorted, n, d_unique_out, d_start_out, d_num_cells_out, scratch, s);
    const cudaError_t after = cudaPeekAtLastError();
    if (before == cudaSuccess && after != cudaSuccess) {
        cudaGetLastError();
        return Fail(TSP_ERR_CUDA, std::string("tsp_b200_build_cell_table_noalloc: ") + cudaGetErrorString(after));
    }
    return TSP_OK;
}

const char* tsp_b200_noalloc_last_error(void) { return tsp::g_noAllocError.c_str(); }

}  // extern "C"
