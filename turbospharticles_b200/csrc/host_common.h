// host_common.h -- host-side helpers shared by the one-scene backend and the served batch:
// status-carrying exception, device buffers, the cell-frame rule and the solver constants.
#pragma once

#include <algorithm>
#include <climits>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#include <cuda.h>  // types of the driver's virtual-memory calls (resolved at run time, no libcuda link)
#include <cuda_runtime.h>

#include "../../include/tsp_b200.h"
#include "kernels.h"

namespace tsp {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
#define CK(x)                                                                                       \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess) throw Error(TSP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t cap = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    void ensure(size_t n) {  // contents are not preserved
        if (n <= cap && (p || n == 0)) return;
        release();
        if (n == 0) return;
        CK(cudaMalloc(&p, n * sizeof(T)));
        cap = n;
    }
    void grow(size_t n, double slack) {
        if (n <= cap && p) return;
        ensure((size_t)((double)n * slack) + 16);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    ~DBuf() { release(); }
};
template <typename T> inline void Swap(DBuf<T>& a, DBuf<T>& b) { std::swap(a.p, b.p); std::swap(a.cap, b.cap); }

// The driver's virtual-memory entry points, looked up once through the runtime.
struct VmmApi {
    decltype(&cuMemAddressReserve) reserve = nullptr;
    decltype(&cuMemAddressFree) addressFree = nullptr;
    decltype(&cuMemCreate) create = nullptr;
    decltype(&cuMemRelease) release = nullptr;
    decltype(&cuMemMap) map = nullptr;
    decltype(&cuMemUnmap) unmap = nullptr;
    decltype(&cuMemSetAccess) setAccess = nullptr;
    decltype(&cuMemGetAllocationGranularity) granularity = nullptr;
    static const VmmApi& Get() {
        static const VmmApi api = [] {
            VmmApi a;
            auto get = [](const char* name, void** fn) {
                cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
                CK(cudaGetDriverEntryPointByVersion(name, fn, 12000, cudaEnableDefault, &q));
                if (q != cudaDriverEntryPointSuccess || !*fn)
                    throw Error(TSP_ERR_CUDA, std::string("driver entry point not found: ") + name);
            };
            get("cuMemAddressReserve", reinterpret_cast<void**>(&a.reserve));
            get("cuMemAddressFree", reinterpret_cast<void**>(&a.addressFree));
            get("cuMemCreate", reinterpret_cast<void**>(&a.create));
            get("cuMemRelease", reinterpret_cast<void**>(&a.release));
            get("cuMemMap", reinterpret_cast<void**>(&a.map));
            get("cuMemUnmap", reinterpret_cast<void**>(&a.unmap));
            get("cuMemSetAccess", reinterpret_cast<void**>(&a.setAccess));
            get("cuMemGetAllocationGranularity", reinterpret_cast<void**>(&a.granularity));
            return a;
        }();
        return api;
    }
};
#define CKD(x)                                                                                      \
    do {                                                                                            \
        CUresult e_ = (x);                                                                          \
        if (e_ != CUDA_SUCCESS) throw Error(TSP_ERR_CUDA, std::string(#x) + ": driver error " + std::to_string((int)e_)); \
    } while (0)

// Device buffer that grows in place: a virtual address range (8x the first request, at least
// 64 MB) is reserved once and physical memory (at least 32 MB) is mapped onto the end of the
// used part as the buffer grows. The address does not change (graphs captured with it stay valid) and a growth costs
// neither a copy, a free nor a device-wide synchronisation; only a request beyond the
// reservation re-reserves (new address, contents not kept, like DBuf::ensure).
template <typename T>
struct VBuf {
    T* p = nullptr;
    size_t cap = 0;  // elements backed by physical memory
    size_t reservedBytes = 0, mappedBytes = 0;
    std::vector<std::pair<CUmemGenericAllocationHandle, size_t>> maps;  // in address order
    VBuf() = default;
    VBuf(const VBuf&) = delete;
    VBuf& operator=(const VBuf&) = delete;
    static CUmemAllocationProp Prop() {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CUmemAllocationProp prop{};
        prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
        prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
        prop.location.id = dev;
        return prop;
    }
    void ensure(size_t n) {  // contents of the backed part are kept unless re-reserved
        const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
        if (p && bytes <= mappedBytes) return;
        const VmmApi& api = VmmApi::Get();
        const CUmemAllocationProp prop = Prop();
        size_t gran = 0;
        CKD(api.granularity(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_RECOMMENDED));
        // at least 32 MB backed: small lists (boundary, 32-bit entries) then never grow in a run
        const size_t need = (std::max<size_t>(bytes, size_t(32) << 20) + gran - 1) / gran * gran;
        if (!p || need > reservedBytes) {
            release();
            const size_t want = std::max<size_t>(need * 8, size_t(64) << 20);
            reservedBytes = (want + gran - 1) / gran * gran;
            CUdeviceptr va = 0;
            CKD(api.reserve(&va, reservedBytes, gran, 0, 0));
            p = reinterpret_cast<T*>(va);
        }
        const size_t add = need - mappedBytes;
        CUmemGenericAllocationHandle h = 0;
        CKD(api.create(&h, add, &prop, 0));
        const CUdeviceptr at = reinterpret_cast<CUdeviceptr>(p) + mappedBytes;
        if (api.map(at, add, 0, h, 0) != CUDA_SUCCESS) {
            api.release(h);
            throw Error(TSP_ERR_CUDA, "cuMemMap of a growing neighbor-list buffer failed");
        }
        maps.emplace_back(h, add);
        CUmemAccessDesc acc{};
        acc.location = prop.location;
        acc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
        CKD(api.setAccess(at, add, &acc, 1));
        mappedBytes = need;
        cap = mappedBytes / sizeof(T);
    }
    void grow(size_t n, double slack) {
        if (n <= cap && p) return;
        ensure((size_t)((double)n * slack) + 16);
    }
    // reserves the virtual range for up to `elems` elements before anything is mapped, so that
    // growth up to that size maps in place (addresses and contents kept); no physical memory
    void reserveAddress(size_t elems) {
        if (p) return;
        const VmmApi& api = VmmApi::Get();
        const CUmemAllocationProp prop = Prop();
        size_t gran = 0;
        CKD(api.granularity(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_RECOMMENDED));
        const size_t want = std::max<size_t>(elems * sizeof(T), size_t(64) << 20);
        reservedBytes = (want + gran - 1) / gran * gran;
        CUdeviceptr va = 0;
        CKD(api.reserve(&va, reservedBytes, gran, 0, 0));
        p = reinterpret_cast<T*>(va);
    }
    void release() {
        if (!p) return;
        cudaDeviceSynchronize();  // no kernel may still use the range (destruction / re-reservation only)
        const VmmApi& api = VmmApi::Get();
        CUdeviceptr at = reinterpret_cast<CUdeviceptr>(p);
        for (auto& m : maps) {
            api.unmap(at, m.second);
            api.release(m.first);
            at += m.second;
        }
        maps.clear();
        api.addressFree(reinterpret_cast<CUdeviceptr>(p), reservedBytes);
        p = nullptr;
        cap = 0;
        reservedBytes = mappedBytes = 0;
    }
    ~VBuf() { release(); }
};

inline unsigned G(uint32_t n) { return (n + 255) / 256; }

// Growth factor of the neighbor-list buffers (VBuf: grown in place, addresses kept). A flow that
// compresses or spreads grows its lists by a few percent per hundred steps; each growth maps
// physical memory (a few driver calls, 0.3-0.6 ms measured, but steps with a growth have also
// shown 5-10 ms outliers), so the buffers grow in 50 % steps and never shrink.
constexpr double LIST_GROWTH = 1.5;

// ------------------------------------------------------------------------------ helpers
inline int HostFloorToInt(float v) {
    const int i = (int)v;
    return (v < (float)i) ? (i - 1) : i;
}
// TryBuildCellCoordFrame (source/simulation/core/cell_frame.h:32-66): inclusive signed cell
// bounds -> origin + dimensions; every axis must have min <= max, both within int32, and at
// most 2^21 cells. On failure the frame is left unchanged.
inline bool TryBuildCellFrame(const int64_t lo[3], const int64_t hi[3], int32_t& ox, int32_t& oy, int32_t& oz,
                              uint32_t& nx, uint32_t& ny, uint32_t& nz) {
    for (int a = 0; a < 3; a++)
        if (lo[a] > hi[a] || lo[a] < (int64_t)INT32_MIN || hi[a] > (int64_t)INT32_MAX ||
            hi[a] - lo[a] + 1 > (int64_t)(1u << 21))
            return false;
    ox = (int32_t)lo[0]; oy = (int32_t)lo[1]; oz = (int32_t)lo[2];
    nx = (uint32_t)(hi[0] - lo[0] + 1); ny = (uint32_t)(hi[1] - lo[1] + 1); nz = (uint32_t)(hi[2] - lo[2] + 1);
    return true;
}
inline uint32_t HostKeyBits(uint32_t nx, uint32_t ny, uint32_t nz) {  // neighbor_search.cpp:403-413
    const uint32_t m = std::max(nx, std::max(ny, nz));
    uint32_t axisBits = 1;
    if (m >= 2) axisBits = 32u - (uint32_t)__builtin_clz(m - 1u);
    return 3u * axisBits + 1u;
}

// solver constants exactly as the reference derives them (see common.cuh: Consts)
inline Consts MakeConsts(const tsp_params& p) {
    Consts c{};
    const double h = (double)p.particleSizeF, hInv = 1.0 / h, rho = (double)p.restDensity;
    c.sizeInv = (float)hInv;
    c.sizeSqu = (float)(h * h);
    c.alpha = p.cubicSplineAlphaOverride > 0.0f ? p.cubicSplineAlphaOverride
                                                : (float)(hInv * hInv * hInv / (4.0 * 3.14159265358979323846));
    c.restDensitySquInv = (float)(1.0 / (rho * rho));
    c.radSqu = p.kernelRadiusSqu;
    c.dt = p.timeStep;
    c.dt2 = p.timeStep * p.timeStep;
    c.kSize = 1.0f / c.sizeInv;
    c.kTwoSize = 2.0f / c.sizeInv;
    c.kInnerSlope = 9.0f * c.alpha * c.sizeInv * c.sizeInv * c.sizeInv;
    c.kInnerOffset = -12.0f * c.alpha * c.sizeInv * c.sizeInv;
    c.kOuterScale = -3.0f * c.alpha * c.sizeInv * c.sizeInv * c.sizeInv;
    c.massF = p.massF;
    c.restDensity = p.restDensity;
    c.densInvSqu = 1.0f / (p.restDensity * p.restDensity);
    c.hEps = 0.01f * c.sizeSqu;
    c.visFacF = 10.0f * p.viscosityF;
    c.visFacB = 10.0f * p.viscosityB;
    c.gx = p.gravity[0]; c.gy = p.gravity[1]; c.gz = p.gravity[2];
    c.cTermFacF = -p.massF * c.restDensitySquInv;
    c.cTermFacB = -2.0f * p.pressGamma * c.restDensitySquInv;
    c.diagBFac = -p.massF * c.restDensitySquInv;
    c.omega = p.jacobiOmega;
    c.warmStart = p.jacobiWarmStart;
    c.warm = p.jacobiWarmStart > 0.0f ? 1 : 0;
    c.accCoeffB = 2.0f * p.pressGamma * c.densInvSqu;
    return c;
}


// pack / unpack kernels of the state boundary (defined in backend.cu)
void LaunchPack4(const float* a, const float* b, const float* c, const float* d, float dDefault, float4* out,
                 uint32_t n, cudaStream_t s);
void LaunchUnpack4(const float4* in, float* a, float* b, float* c, float* d, uint32_t n, cudaStream_t s);
void LaunchPack2(const float* a, const float* b, float2* out, uint32_t n, cudaStream_t s);
void LaunchUnpack2(const float2* in, float* a, float* b, uint32_t n, cudaStream_t s);

}  // namespace tsp
