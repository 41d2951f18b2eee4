// backend.cu -- host driver of the B200 IISPH backend and its C ABI (include/tsp_b200.h).
//
// One `Backend` = one scene resident on one GPU, one CUDA stream. A solver step mirrors
// SimBackend_CPU::Step_IISPH (source/simulation/CPU/backend/sph_solver.cpp:34-319):
//   neighbor build (frame rule, sort, reorder, cell tables, SELL32 count -> offsets -> fill)
//   density -> [rigid clear+gravity] -> non-pressure -> [rigid viscous forces, reduce,
//   predict] -> source/diagonal/init -> relaxed Jacobi loop -> pressure acceleration ->
//   [rigid pressure forces, reduce] -> integration -> [rigid predict, integrate, update]
// Host round trips per step: the frame probe (6 floats + a flag, needed by the reference's
// hysteresis frame rule) and the neighbor-list totals (buffer capacities). The Jacobi loop
// runs entirely on the device inside a CUDA graph whose conditional WHILE node is driven
// by the last block of each sweep (no host synchronisation per iteration, unlike
// gpu_backend.cpp:1432-1496 of the reference GPU backend).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <algorithm>

#include "../../include/tsp_b200.h"
#include "kernels.h"
#include "primitives.cuh"
#include "host_common.h"

namespace tsp {

void LaunchRigidVolumesSorted(const Consts& c, const float4* rel, const uint32_t* byBodyOff, const uint32_t* sortedIdx,
                              const int4* sortedCell, const uint32_t* bodyOfSorted, uint32_t nR, int reach,
                              float defaultVol, float defaultPsi, float restDensity, float* volOut, float* psiOut,
                              cudaStream_t s);

// ------------------------------------------------------------------------------ small kernels
__global__ void KPack4(const float* a, const float* b, const float* c, const float* d, float dDefault, float4* out,
                       uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_float4(a ? a[i] : 0.f, b ? b[i] : 0.f, c ? c[i] : 0.f, d ? d[i] : dDefault);
}
__global__ void KUnpack4(const float4* in, float* a, float* b, float* c, float* d, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = in[i];
    if (a) a[i] = v.x;
    if (b) b[i] = v.y;
    if (c) c[i] = v.z;
    if (d) d[i] = v.w;
}
__global__ void KPack2(const float* a, const float* b, float2* out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_float2(a ? a[i] : 0.f, b ? b[i] : 0.f);
}
__global__ void KUnpack2(const float2* in, float* a, float* b, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (a) a[i] = in[i].x;
    if (b) b[i] = in[i].y;
}
__global__ void KSetW(float4* v, const float* w, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i].w = w[i];
}
// bitwise equality of two boundary uploads (positions + psi, volumes, IDs); any difference sets *diff
__global__ void KBoundaryDiff(const float4* __restrict__ a, const float* __restrict__ va, const uint64_t* __restrict__ ia,
                              const float4* __restrict__ b, const float* __restrict__ vb, const uint64_t* __restrict__ ib,
                              uint32_t n, uint32_t* diff) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 x = *reinterpret_cast<const uint4*>(a + i), y = *reinterpret_cast<const uint4*>(b + i);
    const bool d = x.x != y.x || x.y != y.y || x.z != y.z || x.w != y.w || __float_as_uint(va[i]) != __float_as_uint(vb[i]) ||
                   ia[i] != ib[i];
    if (d) *diff = 1u;
}
void LaunchPack4(const float* a, const float* b, const float* c, const float* d, float dDefault, float4* out,
                 uint32_t n, cudaStream_t s) {
    if (n) KPack4<<<G(n), 256, 0, s>>>(a, b, c, d, dDefault, out, n);
}
void LaunchUnpack4(const float4* in, float* a, float* b, float* c, float* d, uint32_t n, cudaStream_t s) {
    if (n) KUnpack4<<<G(n), 256, 0, s>>>(in, a, b, c, d, n);
}
void LaunchPack2(const float* a, const float* b, float2* out, uint32_t n, cudaStream_t s) {
    if (n) KPack2<<<G(n), 256, 0, s>>>(a, b, out, n);
}
void LaunchUnpack2(const float2* in, float* a, float* b, uint32_t n, cudaStream_t s) {
    if (n) KUnpack2<<<G(n), 256, 0, s>>>(in, a, b, n);
}

// neighbor-build totals the host reads before the fill (written into mapped pinned memory)
struct NsTotals {
    unsigned long long nbrTot[3];
    U64x2 sellTot[3];
    uint64_t csrTot[3];
    uint64_t nCells[3];
};
__global__ void KGatherNsTotals(const U64x2* sell, const uint64_t* csr, const uint64_t* nCells,
                                const unsigned long long* nbr, int hasRigid, NsTotals* out) {
    const uint32_t k = threadIdx.x;
    if (k >= 3) return;
    out->nbrTot[k] = nbr[k];
    out->sellTot[k] = sell[k];
    out->csrTot[k] = hasRigid ? csr[k] : 0ull;
    out->nCells[k] = nCells[k];
}
// end-of-step read-back, written by one thread straight into mapped pinned host memory: solver
// state, the frame probe of the new positions (the accumulator is reset for the next probe by
// the same kernel) and the error flags
struct StepEnd {
    SolverState st;
    ProbeResult probe;
    uint32_t err;
    uint32_t pad;
};
__global__ void KStepEnd(const SolverState* st, ProbeResult* probe, int takeProbe, const uint32_t* err,
                         StepEnd* out, ProbeResult init) {
    if (threadIdx.x != 0) return;
    if (st) out->st = *st;
    if (takeProbe) {
        out->probe = *probe;
        *probe = init;
    }
    out->err = *err;
}
struct HostMirror {
    StepEnd se;
    NsTotals ns;
    ProbeResult probe;
    SolverState st;
    uint32_t err;
    ContactState contact;
    uint64_t contactTot[2];
    uint32_t exportCount;
    uint32_t bDiff;
    ProbeResult probeInit;  // identity bounds of an empty class, the probe accumulator's reset
};

class Backend {
public:
    int device = 0;
    cudaStream_t s = nullptr, capStream = nullptr;
    tsp_params prm{};
    DomainBox dom{};
    uint32_t nF = 0, nB = 0, nR = 0, nRB = 0;
    uint64_t stepCount = 0;
    double simTime = 0.0;
    // fluid
    DBuf<float4> posP, posP2, velRho, velRho2, velPred, velPred2, acc, acc2;
    DBuf<float2> srcDiag, srcDiag2;
    DBuf<uint64_t> idF, idF2;
    // boundary
    DBuf<float4> posB, posB2;
    DBuf<float> volB, volB2, psiTmpB;
    DBuf<uint64_t> idB, idB2;
    // rigid particles and bodies
    DBuf<uint32_t> bodyR, byBodyOff, byBodyIdx;
    DBuf<float4> relR, posR, velR, velPredR, forceR;
    DBuf<uint64_t> idR;
    DBuf<float> volR, psiR;
    std::vector<float> hRelX, hRelY, hRelZ;
    std::vector<uint32_t> hBodyR, hByBodyOff, hByBodyIdx;
    std::vector<uint64_t> hIdRB;
    std::vector<uint32_t> hCntRB;
    DBuf<double> bodyState, bodyFT;
    // neighbor search
    Frame fr{};
    bool frameValid = false;
    // the probe (bounds + frame-exit flag) of the current positions under the current frame and
    // domain was taken at the end of the last step, with its read-back: the next frame rule uses
    // it without a launch and a round trip of its own
    bool probeFresh = false;
    float cellSize = 0.0f;
    uint32_t reach = 1;
    uint32_t frameRebuilds = 0;
    // Boundary arrays: posB/volB/idB hold the last pull's boundary in its raw (uploaded) order
    // (B_RAW), the stable cell sort of that order under bSortFr (B_SORTED_FROM_RAW), or another
    // order / other values (B_OTHER: sorted again after a frame change, volumes rewritten).
    // rawPosB/rawVolB/rawIdB keep the raw upload, so a pull of the same boundary keeps a sort of
    // it, and the first step after that pull sorts nothing when its fresh frame equals bSortFr
    // (the reference re-sorts the raw order under the fresh frame: the same arrays).
    enum { B_RAW = 0, B_SORTED_FROM_RAW = 1, B_OTHER = 2 };
    int bState = B_OTHER;
    bool bSortedValid = false;  // posB sorted, cell table and grid built, under bSortFr
    Frame bSortFr{};
    bool rawBValid = false;
    uint32_t rawNB = 0;
    bool bKeptAtPull = false;   // the last pull kept a sort of the same raw boundary (B_SORTED_FROM_RAW)
    DBuf<uint32_t> rawPermB;    // permutation of the sort of the raw order under bSortFr
    DBuf<float4> rawPosB;
    DBuf<float> rawVolB;
    DBuf<uint64_t> rawIdB;
    DBuf<uint32_t> bDiff;
    bool bAabbValid = false;
    float bMin[3] = {0, 0, 0}, bMax[3] = {0, 0, 0};
    DBuf<uint64_t> keysA, keysB;
    DBuf<uint32_t> valsA, valsB, tileHist, digitTotals;
    DBuf<uint32_t> osAux;     // one-pass sort: histograms, tickets, look-back status
    DBuf<uint32_t> cellAux;   // single-pass cell table: ticket and look-back status
    DBuf<uint32_t> permF, permB, permR;
    bool permBIdentity = false;  // the last build's boundary permutation is the identity (not written)
    DBuf<uint64_t> cidF, cidB, cidR, cidRs;
    DBuf<uint64_t> uniqF, uniqB, uniqR;
    DBuf<uint32_t> startF, startB, startR;
    DBuf<uint64_t> nCellsDev;
    DBuf<uint32_t> gridF, gridB, gridR;
    uint64_t gridCells = 0;
    DBuf<uint64_t> scanScratch;
    DBuf<U64x2> scanScratch2;
    struct Sell {
        DBuf<uint16_t> counts, pitch;
        DBuf<uint8_t> format;
        DBuf<uint32_t> base, base2;
        DBuf<uint64_t> offset;
        VBuf<uint16_t> l16;  // grow in place: list growth keeps the addresses
        VBuf<uint32_t> l32;
        uint64_t n16 = 0, n32 = 0;
    } sell[3];
    DBuf<U64x2> sellTot;
    DBuf<unsigned long long> nbrTot;
    StepEnd* seDev = nullptr;   // device view of hm->se (mapped pinned memory)
    NsTotals* nsDev = nullptr;  // device view of hm->ns
    // count-pass rows of the fluid query ([chunk][slot][lane]); rows longer than KS_* slots make
    // the fill walk that chunk's stencil again
    static constexpr uint32_t KS_F = 64, KS_B = 48, KS_R = 16;
    DBuf<uint32_t> scrF, scrB, scrR;
    DBuf<uint8_t> scrOver;
    uint64_t nNbr[3] = {0, 0, 0};
    DBuf<float4> tunePos;           // posP kept aside while kernels that rewrite it are tuned
    DBuf<SolverState> tuneSt;
    DBuf<uint16_t> cntR[3];
    DBuf<uint64_t> offR[3];
    VBuf<uint32_t> listR[3];
    DBuf<uint64_t> csrTot;
    uint64_t csrN[3] = {0, 0, 0};
    bool listsValid = false;
    // solver
    DBuf<SolverState> st;
    DBuf<double> partials;
    DBuf<uint32_t> err;
    DBuf<ProbeResult> probe;
    HostMirror* hm = nullptr;
    struct JacobiGraph {
        std::vector<uint64_t> key;
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ex = nullptr;
    };
    std::vector<JacobiGraph> graphs;
    // rigid contact solver (rigid_solver.cpp): per rigid particle, per contact boundary particle
    // (capacity contactCap, grow-only), per body; the contact loop runs in its own WHILE graph
    DBuf<uint32_t> cOfB, cLocalB, cIdxRB, cIdxBR, cCurBR, cPerBody;
    DBuf<uint64_t> cOffBR, cTot;
    DBuf<float4> cRelW, cForce, cVel;
    DBuf<float> cIw, cDensR, cDiagR, cPresR, cSrcR, cErrR, cOmegaR;
    DBuf<float> cDensB, cDiagB, cPresB, cSrcB, cErrB, cOmegaB;
    DBuf<double> cFT, cContrib;
    DBuf<ContactState> cState;
    uint32_t contactCap = 0, lastContactB = 0;
    bool contactRan = false;
    std::vector<JacobiGraph> cgraphs;
    size_t cgraphNext = 0;
    DBuf<float> stage;  // device staging of the SoA <-> packed conversions at the state boundary (grow-only)
    size_t graphNext = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // phase boundaries of the last step: 0 start, 1 frame, 2 sort/reorder/cell tables/grids,
    // 3 query count, 4 finalize + size read-back, 5 query fill (= neighbor build end),
    // 6 density, 7 non-pressure (+ rigid viscous forces), 8 source/diagonal/init,
    // 9 Jacobi loop, 10 final pressure acceleration (+ rigid pressure forces), 11 integration
    // (+ rigid integration), 12 end
    static constexpr int N_PHASE_EVENTS = 13;
    cudaEvent_t pev[N_PHASE_EVENTS] = {};
    // copy stream of the state boundary: the host <-> device copies of pull / push run on xs
    // while the pack / unpack kernels run on s, ordered by events in both directions
    cudaStream_t xs = nullptr;
    cudaEvent_t xev[8] = {};
    uint32_t xevNext = 0;
    cudaEvent_t NextXev() { return xev[xevNext++ % 8]; }
    void CopiesAfterCompute() {  // xs waits for everything queued on s so far
        cudaEvent_t e = NextXev();
        CK(cudaEventRecord(e, s));
        CK(cudaStreamWaitEvent(xs, e, 0));
    }
    void ComputeAfterCopies() {  // s waits for everything queued on xs so far
        cudaEvent_t e = NextXev();
        CK(cudaEventRecord(e, xs));
        CK(cudaStreamWaitEvent(s, e, 0));
    }
    bool phaseValid = false;
    float lastStepMs = 0.f, lastNbrMs = 0.f, lastJacMs = 0.f;
    double stepMsTotal = 0.0;   // device milliseconds of all steps since creation
    uint64_t stepsTimed = 0;
    // records of the last HIST_CAP steps (a ring, allocated at the first step)
    static constexpr uint32_t HIST_CAP = 1u << 16;
    std::vector<tsp_step_record> hist;
    uint64_t histCount = 0;
    std::string lastErr;
    uint64_t launches = 0;  // kernels launched by this backend (graph nodes included)
    // one-pass sort: the key kernel (with the histograms) and one kernel per 8-bit pass
    static uint32_t SortLaunches(uint32_t n, uint32_t bits) { return n < 2 ? 3u : 1u + (bits + 7u) / 8u; }

    explicit Backend(int dev) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw Error(TSP_ERR_NO_DEVICE, "no CUDA device");
        if (dev < 0) CK(cudaGetDevice(&dev));
        device = dev;
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&capStream, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&xs, cudaStreamNonBlocking));
        for (auto& e : xev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CK(cudaHostAlloc((void**)&hm, sizeof(HostMirror), cudaHostAllocMapped | cudaHostAllocPortable));
        std::memset(hm, 0, sizeof(HostMirror));
        for (int a = 0; a < 3; a++) {  // (neighbor_search.cpp:205-213)
            hm->probeInit.mnKey[a] = OrderedIntHost(3.402823466e38f);
            hm->probeInit.mxKey[a] = OrderedIntHost(-3.402823466e38f);
        }
        // the step-end and neighbor-total gathers write straight into this pinned host memory
        CK(cudaHostGetDevicePointer((void**)&seDev, &hm->se, 0));
        CK(cudaHostGetDevicePointer((void**)&nsDev, &hm->ns, 0));
        st.ensure(1);
        err.ensure(1);
        probe.ensure(1);
        nCellsDev.ensure(3);
        sellTot.ensure(3);
        nbrTot.ensure(3);
        csrTot.ensure(3);
        CK(cudaMemset(st.p, 0, sizeof(SolverState)));
        CK(cudaMemset(err.p, 0, sizeof(uint32_t)));
        // the probe accumulator holds the empty bounds whenever no probe is in flight
        CK(cudaMemcpy(probe.p, &hm->probeInit, sizeof(ProbeResult), cudaMemcpyHostToDevice));
        for (auto& e : ev) CK(cudaEventCreate(&e));
        for (auto& e : pev) CK(cudaEventCreate(&e));
    }
    ~Backend() {
        cudaSetDevice(device);
        if (s) cudaStreamSynchronize(s);
        for (auto* gs : {&graphs, &cgraphs})
            for (auto& g : *gs) {
                if (g.ex) cudaGraphExecDestroy(g.ex);
                if (g.g) cudaGraphDestroy(g.g);
            }
        for (auto& e : ev) if (e) cudaEventDestroy(e);
        for (auto& e : pev) if (e) cudaEventDestroy(e);
        if (xs) cudaStreamSynchronize(xs);
        for (auto& e : xev) if (e) cudaEventDestroy(e);
        if (xs) cudaStreamDestroy(xs);
        if (hm) cudaFreeHost(hm);
        if (capStream) cudaStreamDestroy(capStream);
        if (s) cudaStreamDestroy(s);
    }
    void Sync() { CK(cudaStreamSynchronize(s)); }
    void CheckErrors() {
        CK(cudaMemcpyAsync(&hm->err, err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        Sync();
        RaiseErrors(hm->err);
    }
    void RaiseErrors(uint32_t e) {
        CK(cudaGetLastError());
        if (!e) return;
        CK(cudaMemsetAsync(err.p, 0, sizeof(uint32_t), s));
        if (e & (ERR_RIGID_ORIENT | ERR_RIGID_ATTACH))
            throw Error(TSP_ERR_RIGID, (e & ERR_RIGID_ORIENT) ? "Degenerate rigid body orientation."
                                                               : "Invalid rigid particle attachment.");
        if (e & ERR_CONTACT_INVALID)
            throw Error(TSP_ERR_RIGID, "Invalid rigid contact diagonal, density error or pressure.");
        if (e & ERR_CONTACT_BODIES)
            throw Error(TSP_ERR_UNSUPPORTED, "a rigid contact particle touches more than 8 bodies");
        if (e & ERR_QUERY_CAP) throw Error(TSP_ERR_UNSUPPORTED, "query stencil exceeds the shared-memory staging");
        if (e & ERR_COUNT_U16) throw Error(TSP_ERR_OVERFLOW, "a neighbor count exceeds uint16 storage");
        if (e & ERR_SORT_LOOKBACK)
            throw Error(TSP_ERR_CUDA, "cell sort / cell table: a tile's look-back gave up waiting for its predecessors");
        if (e & ERR_STAGE_WAIT)
            throw Error(TSP_ERR_CUDA, "neighbor query: a block's staging copies did not complete");
        throw Error(TSP_ERR_NEIGHBOR_LIST, "SELL32 neighbor-list fill overflow / delta range error");
    }

    // -------------------------------------------------------------------------- state boundary
    void SetDomain(const float* mn, const float* mx) {
        probeFresh = false;
        for (int a = 0; a < 3; a++) { dom.mn[a] = mn[a]; dom.mx[a] = mx[a]; }
        dom.bounded = !(mx[0] <= mn[0] || mx[1] <= mn[1] || mx[2] <= mn[2]);
    }

    template <typename T>
    void Upload(DBuf<T>& d, const T* h, size_t n) {
        d.ensure(std::max<size_t>(n, 1));
        if (n && h) CK(cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    // Pack4 with the host columns copied on the copy stream into stg[0, 4n) (the caller's own
    // staging region) and the pack kernel on s once they have arrived
    void Pack4X(DBuf<float4>& out, uint32_t n, const float* a, const float* b, const float* c, const float* d,
                float dDefault, float* stg) {
        out.ensure(std::max<uint32_t>(n, 1));
        if (n == 0) return;
        const float* src[4] = {a, b, c, d};
        float* dst[4] = {nullptr, nullptr, nullptr, nullptr};
        for (int k = 0; k < 4; k++)
            if (src[k]) {
                dst[k] = stg + (uint64_t)k * n;
                CK(cudaMemcpyAsync(dst[k], src[k], n * sizeof(float), cudaMemcpyHostToDevice, xs));
            }
        ComputeAfterCopies();
        KPack4<<<G(n), 256, 0, s>>>(dst[0], dst[1], dst[2], dst[3], dDefault, out.p, n);
    }
    template <typename T>
    void UploadX(DBuf<T>& d, const T* h, size_t n) {
        d.ensure(std::max<size_t>(n, 1));
        if (n && h) CK(cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, xs));
    }
    void Pack4(DBuf<float4>& out, uint32_t n, const float* a, const float* b, const float* c, const float* d,
               float dDefault, DBuf<float>& tmp) {
        out.ensure(std::max<uint32_t>(n, 1));
        if (n == 0) return;
        tmp.ensure(4ull * n);
        const float* src[4] = {a, b, c, d};
        float* dst[4] = {nullptr, nullptr, nullptr, nullptr};
        for (int k = 0; k < 4; k++)
            if (src[k]) {
                dst[k] = tmp.p + (uint64_t)k * n;
                CK(cudaMemcpyAsync(dst[k], src[k], n * sizeof(float), cudaMemcpyHostToDevice, s));
            }
        KPack4<<<G(n), 256, 0, s>>>(dst[0], dst[1], dst[2], dst[3], dDefault, out.p, n);
    }
    void Unpack4(const float4* in, uint32_t n, float* a, float* b, float* c, float* d, DBuf<float>& tmp) {
        if (n == 0) return;
        tmp.ensure(4ull * n);
        UnpackTo(in, n, a, b, c, d, tmp.p);
    }
    // unpack into the 4 * n floats at dev (only the columns a host array asks for) and queue
    // their device-to-host copies; dev must stay untouched until the stream passes the copies
    // cs: the stream of the device-to-host copies (s, or the copy stream xs ordered after the
    // unpack kernel)
    void UnpackTo(const float4* in, uint32_t n, float* a, float* b, float* c, float* d, float* dev0,
                  cudaStream_t cs = nullptr) {
        if (n == 0) return;
        float* host[4] = {a, b, c, d};
        float* dev[4];
        for (int k = 0; k < 4; k++) dev[k] = host[k] ? dev0 + (uint64_t)k * n : nullptr;
        if (!host[0] && !host[1] && !host[2] && !host[3]) return;
        KUnpack4<<<G(n), 256, 0, s>>>(in, dev[0], dev[1], dev[2], dev[3], n);
        if (!cs) cs = s;
        else CopiesAfterCompute();
        for (int k = 0; k < 4; k++)
            if (host[k]) CK(cudaMemcpyAsync(host[k], dev[k], n * sizeof(float), cudaMemcpyDeviceToHost, cs));
    }

    void Pull(const tsp_state_view& v, const tsp_params& p) {
        CK(cudaSetDevice(device));
        DBuf<float>& tmp = stage;
        prm = p;
        nF = v.N_F; nB = v.N_B; nR = v.N_R; nRB = v.N_RB;
        if (nF > 0x7fffffffu || nB > 0x7fffffffu || nR > 0x7fffffffu)
            throw Error(TSP_ERR_OVERFLOW, "particle count exceeds the local particle limit");
        stepCount = v.step; simTime = v.time;
        // every column group has its own staging region, so the copies (on xs) run back to back
        // while the pack kernels (on s) follow each group as it arrives
        const uint64_t F = nF, B = nB, R = nR;
        tmp.ensure(std::max<uint64_t>(18 * F + 4 * B + 8 * R, 1));
        float* stg = tmp.p;
        CopiesAfterCompute();  // no copy may overwrite staging that queued work still reads
        // fluid
        std::vector<uint64_t> ids;
        if (!v.idF) { ids.resize(nF); for (uint32_t i = 0; i < nF; i++) ids[i] = i; }
        UploadX(idF, v.idF ? v.idF : ids.data(), nF);
        Pack4X(posP, nF, v.xPosF, v.yPosF, v.zPosF, v.pressureF, 0.0f, stg);
        Pack4X(velRho, nF, v.xVelF, v.yVelF, v.zVelF, v.densityF, p.restDensity, stg + 4 * F);
        Pack4X(velPred, nF, v.xVelPredF, v.yVelPredF, v.zVelPredF, nullptr, 0.0f, stg + 8 * F);
        Pack4X(acc, nF, v.xAccPressF, v.yAccPressF, v.zAccPressF, nullptr, 0.0f, stg + 12 * F);
        srcDiag.ensure(std::max<uint32_t>(nF, 1));
        if (nF) {
            const float* sh[2] = {v.sourceTermF, v.diagElemF};
            float* sd[2] = {nullptr, nullptr};
            for (int k = 0; k < 2; k++)
                if (sh[k]) {
                    sd[k] = stg + 16 * F + (uint64_t)k * nF;
                    CK(cudaMemcpyAsync(sd[k], sh[k], nF * sizeof(float), cudaMemcpyHostToDevice, xs));
                }
            ComputeAfterCopies();
            KPack2<<<G(nF), 256, 0, s>>>(sd[0], sd[1], srcDiag.p, nF);
        }
        posP2.ensure(std::max<uint32_t>(nF, 1)); velRho2.ensure(std::max<uint32_t>(nF, 1));
        idF2.ensure(std::max<uint32_t>(nF, 1));
        // boundary: defaults psi = massB, vol = massB / rho0 (state_sim.h:347-362)
        const float defPsi = p.massB, defVol = p.restDensity > 0.0f ? p.massB / p.restDensity : 0.0f;
        // the upload lands in posB2/volB2/idB2 and is compared with the raw copy of the last
        // boundary upload (decided after the pull's synchronisation, PullBoundaryCommit)
        std::vector<uint64_t> idsB;
        if (!v.idB) { idsB.resize(nB); for (uint32_t i = 0; i < nB; i++) idsB[i] = i; }
        UploadX(idB2, v.idB ? v.idB : idsB.data(), nB);
        volB2.ensure(std::max<uint32_t>(nB, 1));
        std::vector<float> defVolB;
        if (nB) {
            if (!v.volB) defVolB.assign(nB, defVol);
            CK(cudaMemcpyAsync(volB2.p, v.volB ? v.volB : defVolB.data(), nB * sizeof(float), cudaMemcpyHostToDevice,
                               xs));
        }
        Pack4X(posB2, nB, v.xPosB, v.yPosB, v.zPosB, v.psiB, defPsi, stg + 18 * F);
        hm->bDiff = 1u;
        const bool compare = nB && rawBValid && rawNB == nB;
        if (compare) {
            bDiff.ensure(1);
            CK(cudaMemsetAsync(bDiff.p, 0, sizeof(uint32_t), s));
            KBoundaryDiff<<<G(nB), 256, 0, s>>>(posB2.p, volB2.p, idB2.p, rawPosB.p, rawVolB.p, rawIdB.p, nB, bDiff.p);
            CK(cudaMemcpyAsync(&hm->bDiff, bDiff.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        }
        // rigid particles (storage order preserved)
        ids.clear();
        if (!v.idR) { ids.resize(nR); for (uint32_t i = 0; i < nR; i++) ids[i] = i; }
        Upload(idR, v.idR ? v.idR : ids.data(), nR);
        hBodyR.assign(nR, 0);
        for (uint32_t i = 0; i < nR; i++) hBodyR[i] = v.bodyIdR ? v.bodyIdR[i] : 0u;
        for (uint32_t i = 0; i < nR; i++)
            if (hBodyR[i] >= nRB) throw Error(TSP_ERR_RIGID, "Invalid rigid particle attachment.");
        Upload(bodyR, hBodyR.data(), nR);
        hRelX.assign(nR, 0.f); hRelY.assign(nR, 0.f); hRelZ.assign(nR, 0.f);
        for (uint32_t i = 0; i < nR; i++) {
            hRelX[i] = v.xPosRelR ? v.xPosRelR[i] : 0.f;
            hRelY[i] = v.yPosRelR ? v.yPosRelR[i] : 0.f;
            hRelZ[i] = v.zPosRelR ? v.zPosRelR[i] : 0.f;
        }
        Pack4X(relR, nR, v.xPosRelR, v.yPosRelR, v.zPosRelR, v.volR, defVol, stg + 18 * F + 4 * B);
        Pack4X(posR, nR, nullptr, nullptr, nullptr, v.psiR, defPsi, stg + 18 * F + 4 * B + 4 * R);
        velR.ensure(std::max<uint32_t>(nR, 1)); velPredR.ensure(std::max<uint32_t>(nR, 1));
        forceR.ensure(std::max<uint32_t>(nR, 1));
        if (nR) CK(cudaMemsetAsync(forceR.p, 0, nR * sizeof(float4), s));
        volR.ensure(std::max<uint32_t>(nR, 1)); psiR.ensure(std::max<uint32_t>(nR, 1));
        hByBodyOff.assign(nRB + 1, 0);
        for (uint32_t i = 0; i < nR; i++) hByBodyOff[hBodyR[i] + 1]++;
        for (uint32_t b = 0; b < nRB; b++) hByBodyOff[b + 1] += hByBodyOff[b];
        hByBodyIdx.assign(nR, 0);
        {
            std::vector<uint32_t> cur(hByBodyOff.begin(), hByBodyOff.end() - 1);
            for (uint32_t i = 0; i < nR; i++) hByBodyIdx[cur[hBodyR[i]]++] = i;
        }
        Upload(byBodyOff, hByBodyOff.data(), hByBodyOff.size());
        Upload(byBodyIdx, hByBodyIdx.data(), nR);
        // bodies (FP64 state)
        hIdRB.assign(nRB, 0); hCntRB.assign(nRB, 0);
        std::vector<double> bs((size_t)nRB * 48, 0.0);
        auto g = [](const float* a, uint32_t b, float d) { return a ? (double)a[b] : (double)d; };
        for (uint32_t b = 0; b < nRB; b++) {
            hIdRB[b] = v.idRB ? v.idRB[b] : b;
            hCntRB[b] = v.rigidParticleCountRB ? v.rigidParticleCountRB[b] : 0u;
            double* q = &bs[(size_t)b * 48];
            q[0] = g(v.xCM, b, 0); q[1] = g(v.yCM, b, 0); q[2] = g(v.zCM, b, 0);
            q[3] = g(v.xVelRB, b, 0); q[4] = g(v.yVelRB, b, 0); q[5] = g(v.zVelRB, b, 0);
            q[6] = g(v.xOmegaRB, b, 0); q[7] = g(v.yOmegaRB, b, 0); q[8] = g(v.zOmegaRB, b, 0);
            q[9] = g(v.xAngMomRB, b, 0); q[10] = g(v.yAngMomRB, b, 0); q[11] = g(v.zAngMomRB, b, 0);
            const float* A[9] = {v.a00, v.a01, v.a02, v.a10, v.a11, v.a12, v.a20, v.a21, v.a22};
            const float* I[9] = {v.iBodyInv00, v.iBodyInv01, v.iBodyInv02, v.iBodyInv10, v.iBodyInv11,
                                 v.iBodyInv12, v.iBodyInv20, v.iBodyInv21, v.iBodyInv22};
            for (int k = 0; k < 9; k++) { q[12 + k] = g(A[k], b, (k % 4 == 0) ? 1.f : 0.f); q[23 + k] = g(I[k], b, 0.f); }
            q[21] = g(v.massRB, b, 0); q[22] = g(v.massInvRB, b, 0);
        }
        Upload(bodyState, bs.data(), bs.size());
        bodyFT.ensure(std::max<size_t>((size_t)nRB * 6, 1));
        CK(cudaMemsetAsync(bodyFT.p, 0, bodyFT.cap * sizeof(double), s));
        // neighbor-search state is rebuilt from scratch
        frameValid = false; frameRebuilds = 0; cellSize = 0.0f; reach = 1; listsValid = false; probeFresh = false;
        CK(cudaMemsetAsync(st.p, 0, sizeof(SolverState), s));
        // UpdateRigidParticles() at import (cpu_backend.cpp:326)
        if (nR) LaunchRigidUpdateParticles(RigidView(), BodyView(), false, err.p, s);
        ComputeAfterCopies();
        CheckErrors();
        PullBoundaryCommit(compare && hm->bDiff == 0u);
    }
    // same: the pulled boundary equals the raw copy bit for bit
    void PullBoundaryCommit(bool same) {
        if (same && bState != B_OTHER) {  // raw order or a sort of it: kept as is
            bKeptAtPull = bState == B_SORTED_FROM_RAW;
            return;
        }
        bKeptAtPull = false;
        if (same) {  // other order / values: back to the raw order
            CK(cudaMemcpyAsync(posB.p, rawPosB.p, nB * sizeof(float4), cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(volB.p, rawVolB.p, nB * sizeof(float), cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(idB.p, rawIdB.p, nB * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        } else {
            Swap(posB, posB2); Swap(volB, volB2); Swap(idB, idB2);
            rawPosB.ensure(std::max<uint32_t>(nB, 1)); rawVolB.ensure(std::max<uint32_t>(nB, 1));
            rawIdB.ensure(std::max<uint32_t>(nB, 1));
            if (nB) {
                CK(cudaMemcpyAsync(rawPosB.p, posB.p, nB * sizeof(float4), cudaMemcpyDeviceToDevice, s));
                CK(cudaMemcpyAsync(rawVolB.p, volB.p, nB * sizeof(float), cudaMemcpyDeviceToDevice, s));
                CK(cudaMemcpyAsync(rawIdB.p, idB.p, nB * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
            }
            rawBValid = true;
            rawNB = nB;
            bAabbValid = false;
        }
        posB2.ensure(std::max<uint32_t>(nB, 1)); volB2.ensure(std::max<uint32_t>(nB, 1));
        idB2.ensure(std::max<uint32_t>(nB, 1));
        bState = B_RAW;
        bSortedValid = false;
    }
    static bool SameFrame(const Frame& a, const Frame& b) {
        return a.ox == b.ox && a.oy == b.oy && a.oz == b.oz && a.nx == b.nx && a.ny == b.ny && a.nz == b.nz &&
               a.cellSizeInv == b.cellSizeInv && a.reach == b.reach && a.keyBits == b.keyBits;
    }
    // Boundary sorted by cell, with its cell table and grid, under the current frame. A stable
    // sort of sorted cell IDs is the identity, so the reference's "sort only when not
    // non-decreasing" (neighbor_search.cpp:1779-1810) is the same result. After a pull that kept
    // a sort of the raw boundary, the reference sorts the raw order under the fresh frame: the
    // kept arrays when the frame is the same, else the raw order is restored and sorted.
    enum { B_SORTED_NOW = 0, B_KEPT_FROM_PULL = 1, B_ALREADY_SORTED = 2 };
    int EnsureBoundarySorted(SortScratch& sc) {
        const bool kept = bKeptAtPull;
        bKeptAtPull = false;
        if (bSortedValid && SameFrame(bSortFr, fr)) return kept ? B_KEPT_FROM_PULL : B_ALREADY_SORTED;
        if (kept && nB) {
            CK(cudaMemcpyAsync(posB.p, rawPosB.p, nB * sizeof(float4), cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(volB.p, rawVolB.p, nB * sizeof(float), cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(idB.p, rawIdB.p, nB * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
            bState = B_RAW;
        }
        if (nB) {
            SortByCell(posB.p, nB, fr, sc, permB.p, cidB.p, s);
            GatherF4(permB.p, posB.p, posB2.p, nB, s); Swap(posB, posB2);
            GatherF1(permB.p, volB.p, volB2.p, nB, s); Swap(volB, volB2);
            GatherU64(permB.p, idB.p, idB2.p, nB, s); Swap(idB, idB2);
            BuildCellTableGrid(cidB.p, nB, uniqB.p, startB.p, nCellsDev.p + 1, gridB.p, fr, gridCells, cellAux.p, err.p, s);
            launches += SortLaunches(nB, fr.keyBits) + 3 + 1;
        }
        if (bState == B_RAW && nB) {
            rawPermB.ensure(nB);
            CK(cudaMemcpyAsync(rawPermB.p, permB.p, nB * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        }
        bState = bState == B_RAW ? B_SORTED_FROM_RAW : B_OTHER;
        bSortFr = fr;
        bSortedValid = true;
        return B_SORTED_NOW;
    }

    void Push(tsp_state_view& v) {
        CK(cudaSetDevice(device));
        v.N_F = nF; v.N_B = nB; v.N_R = nR; v.N_RB = nRB; v.step = stepCount; v.time = simTime;
        // every field gets its own staging columns: the unpack kernels run on s and the copies
        // on the copy stream xs, each group's copies after its kernel, one synchronisation at the end
        const uint64_t F = nF, B = nB, R = nR;
        stage.ensure(std::max<uint64_t>(18 * F + 4 * B + 8 * R, 1));
        float* st0 = stage.p;
        CopiesAfterCompute();  // the state the copies read is final
        if (v.idF && nF) CK(cudaMemcpyAsync(v.idF, idF.p, nF * 8ull, cudaMemcpyDeviceToHost, xs));
        UnpackTo(posP.p, nF, v.xPosF, v.yPosF, v.zPosF, v.pressureF, st0, xs);
        UnpackTo(velRho.p, nF, v.xVelF, v.yVelF, v.zVelF, v.densityF, st0 + 4 * F, xs);
        UnpackTo(velPred.p, nF, v.xVelPredF, v.yVelPredF, v.zVelPredF, nullptr, st0 + 8 * F, xs);
        UnpackTo(acc.p, nF, v.xAccPressF, v.yAccPressF, v.zAccPressF, nullptr, st0 + 12 * F, xs);
        if (nF && (v.sourceTermF || v.diagElemF)) {
            float* sd = st0 + 16 * F;
            KUnpack2<<<G(nF), 256, 0, s>>>(srcDiag.p, sd, sd + F, nF);
            CopiesAfterCompute();
            if (v.sourceTermF) CK(cudaMemcpyAsync(v.sourceTermF, sd, nF * 4ull, cudaMemcpyDeviceToHost, xs));
            if (v.diagElemF) CK(cudaMemcpyAsync(v.diagElemF, sd + F, nF * 4ull, cudaMemcpyDeviceToHost, xs));
        }
        if (v.idB && nB) CK(cudaMemcpyAsync(v.idB, idB.p, nB * 8ull, cudaMemcpyDeviceToHost, xs));
        UnpackTo(posB.p, nB, v.xPosB, v.yPosB, v.zPosB, v.psiB, st0 + 18 * F, xs);
        if (v.volB && nB) CK(cudaMemcpyAsync(v.volB, volB.p, nB * 4ull, cudaMemcpyDeviceToHost, xs));
        if (v.idR && nR) CK(cudaMemcpyAsync(v.idR, idR.p, nR * 8ull, cudaMemcpyDeviceToHost, xs));
        if (v.bodyIdR && nR) CK(cudaMemcpyAsync(v.bodyIdR, bodyR.p, nR * 4ull, cudaMemcpyDeviceToHost, xs));
        UnpackTo(relR.p, nR, v.xPosRelR, v.yPosRelR, v.zPosRelR, v.volR, st0 + 18 * F + 4 * B, xs);
        UnpackTo(posR.p, nR, v.xPosR, v.yPosR, v.zPosR, v.psiR, st0 + 18 * F + 4 * B + 4 * R, xs);
        CK(cudaStreamSynchronize(xs));
        ComputeAfterCopies();  // later work on s may reuse the staging the copies read
        if (nRB) {
            std::vector<double> bs((size_t)nRB * 48);
            CK(cudaMemcpyAsync(bs.data(), bodyState.p, bs.size() * 8, cudaMemcpyDeviceToHost, s));
            Sync();
            for (uint32_t b = 0; b < nRB; b++) {
                const double* q = &bs[(size_t)b * 48];
                auto put = [&](float* a, double x) { if (a) a[b] = (float)x; };
                if (v.idRB) v.idRB[b] = hIdRB[b];
                if (v.rigidParticleCountRB) v.rigidParticleCountRB[b] = hCntRB[b];
                put(v.xCM, q[0]); put(v.yCM, q[1]); put(v.zCM, q[2]);
                put(v.xVelRB, q[3]); put(v.yVelRB, q[4]); put(v.zVelRB, q[5]);
                put(v.xOmegaRB, q[6]); put(v.yOmegaRB, q[7]); put(v.zOmegaRB, q[8]);
                put(v.xAngMomRB, q[9]); put(v.yAngMomRB, q[10]); put(v.zAngMomRB, q[11]);
                float* A[9] = {v.a00, v.a01, v.a02, v.a10, v.a11, v.a12, v.a20, v.a21, v.a22};
                float* I[9] = {v.iBodyInv00, v.iBodyInv01, v.iBodyInv02, v.iBodyInv10, v.iBodyInv11,
                               v.iBodyInv12, v.iBodyInv20, v.iBodyInv21, v.iBodyInv22};
                for (int k = 0; k < 9; k++) { put(A[k], q[12 + k]); put(I[k], q[23 + k]); }
                put(v.massRB, q[21]); put(v.massInvRB, q[22]);
            }
        }
        Sync();
    }

    // -------------------------------------------------------------------------- views
    FluidDev FluidView() { return FluidDev{posP.p, velRho.p, velPred.p, acc.p, srcDiag.p, nF}; }
    BoundaryDev BoundaryView() { return BoundaryDev{posB.p, volB.p, nB}; }
    RigidDev RigidDevView() { return RigidDev{posR.p, velR.p, velPredR.p, nR}; }
    RigidParticlesDev RigidView() {
        return RigidParticlesDev{bodyR.p, relR.p, posR.p, velR.p, velPredR.p, forceR.p, nR, byBodyOff.p, byBodyIdx.p};
    }
    BodyDev BodyView() { return BodyDev{bodyState.p, bodyFT.p, nRB}; }
    SellMeta Meta(int k) {
        Sell& m = sell[k];
        return SellMeta{m.counts.p, m.pitch.p, m.format.p, m.base.p, m.base2.p, m.offset.p, m.l16.p, m.l32.p,
                        (uint64_t)m.l16.cap, (uint64_t)m.l32.cap};
    }
    NeighborView NView() {
        auto sv = [&](int k) {
            Sell& m = sell[k];
            return SellView{m.counts.p, m.pitch.p, m.format.p, m.base.p, m.base2.p, m.offset.p, m.l16.p, m.l32.p};
        };
        return NeighborView{sv(0), sv(1), sv(2)};
    }
    SolverControl Control() const {
        return SolverControl{prm.minSolverIters, prm.maxSolverIters, prm.fixedIters, prm.solverTerminationCond,
                             prm.densityDevTarget, nF};
    }

    // -------------------------------------------------------------------------- neighbor build
    void SetCellSize() {  // neighbor_search.cpp:1645-1659
        const float cs = prm.kernelRadius * prm.gridCellSizeRatio;
        const bool zero = std::fabs(cs) <= 1e-7f;
        const float span = zero ? 0.0f : (prm.kernelRadius / cs);
        const uint32_t r = zero ? 1u : std::max<uint32_t>(1u, (uint32_t)std::ceil(std::max(0.0f, span - 1e-6f)));
        // (a sort under another cell size is caught by the frame comparison of the boundary sort)
        if (std::fabs(cellSize - cs) > 1e-7f || reach != r) frameValid = false;
        if (QuerySmemBytes(r) > 227u * 1024u)
            throw Error(TSP_ERR_UNSUPPORTED, "cell size ratio too small: query stencil exceeds shared memory");
        cellSize = cs;
        reach = r;
        fr.cellSizeInv = zero ? 0.0f : 1.0f / cs;
        fr.reach = r;
    }
    // UpdateCellFrame (neighbor_search.cpp:1902-2006); returns true when the frame changed
    bool UpdateFrame() {
        if (nF == 0 && nB == 0 && nR == 0) { frameValid = false; return false; }
        if (!probeFresh) {
            QueueProbe();
            QueueStepEnd(false, true);
            Sync();
            hm->probe = hm->se.probe;
        }
        probeFresh = false;
        ProbeResult pr = hm->probe;
        float mn[3], mx[3];
        for (int a = 0; a < 3; a++) { mn[a] = OrderedIntToFloat(pr.mnKey[a]); mx[a] = OrderedIntToFloat(pr.mxKey[a]); }
        if (nB && !bAabbValid) {
            // boundary particles never move: their bounds are probed once per import
            LaunchProbe(posB.p, nB, fr, false, dom, probe.p, s);
            QueueStepEnd(false, true);
            Sync();
            const ProbeResult& bp = hm->se.probe;
            for (int a = 0; a < 3; a++) { bMin[a] = OrderedIntToFloat(bp.mnKey[a]); bMax[a] = OrderedIntToFloat(bp.mxKey[a]); }
            bAabbValid = true;
        }
        bool rebuild = !frameValid;
        if (!rebuild) {
            const int m = (int)reach;
            const bool innerEmpty = fr.ox + m > fr.ox + (int)fr.nx - 1 - m || fr.oy + m > fr.oy + (int)fr.ny - 1 - m ||
                                    fr.oz + m > fr.oz + (int)fr.nz - 1 - m;
            rebuild = innerEmpty || pr.exceeded != 0;
        }
        if (!rebuild) return false;
        if (nB)
            for (int a = 0; a < 3; a++) { mn[a] = std::min(mn[a], bMin[a]); mx[a] = std::max(mx[a], bMax[a]); }
        if (dom.bounded)
            for (int a = 0; a < 3; a++) {
                mn[a] = std::clamp(mn[a], dom.mn[a], dom.mx[a]);
                mx[a] = std::clamp(mx[a], dom.mn[a], dom.mx[a]);
            }
        const int64_t margin = (int64_t)reach + 8;
        int64_t o[3], e[3];
        for (int a = 0; a < 3; a++) {
            o[a] = (int64_t)HostFloorToInt(mn[a] * fr.cellSizeInv) - margin;
            e[a] = (int64_t)HostFloorToInt(mx[a] * fr.cellSizeInv) + margin;
        }
        if (!TryBuildCellFrame(o, e, fr.ox, fr.oy, fr.oz, fr.nx, fr.ny, fr.nz))
            throw Error(TSP_ERR_FRAME, "Compact CLL cell frame exceeds the supported range.");
        fr.keyBits = HostKeyBits(fr.nx, fr.ny, fr.nz);
        frameValid = true;
        frameRebuilds++;
        const uint64_t cells = (uint64_t)fr.nx * fr.ny * fr.nz;
        if (cells > (1ull << 28))
            throw Error(TSP_ERR_UNSUPPORTED, "cell frame volume exceeds the dense grid limit (2^28 cells)");
        gridCells = cells;
        return true;
    }
    // queue the read-back of the solver state (when st), the accumulated probe (reset for the
    // next probe) and the error flags into hm->se, one copy
    void QueueStepEnd(bool withState, bool withProbe) {
        KStepEnd<<<1, 32, 0, s>>>(withState ? st.p : nullptr, probe.p, withProbe ? 1 : 0, err.p, seDev, hm->probeInit);
        launches += 1;
    }
    // probe of the fluid and rigid positions, read back into hm->se.probe
    void QueueProbe() {
        LaunchProbe(posP.p, nF, fr, frameValid, dom, probe.p, s);
        LaunchProbe(posR.p, nR, fr, frameValid, dom, probe.p, s);
        launches += (nF ? 1 : 0) + (nR ? 1 : 0);
    }
    void EnsureNsScratch() {
        const uint32_t nMax = std::max(nF, std::max(nB, nR));
        keysA.ensure(std::max<uint32_t>(nMax, 1)); keysB.ensure(std::max<uint32_t>(nMax, 1));
        valsA.ensure(std::max<uint32_t>(nMax, 1)); valsB.ensure(std::max<uint32_t>(nMax, 1));
        tileHist.ensure(RadixTileHistItems(std::max<uint32_t>(nMax, 1)));
        digitTotals.ensure(256);
        osAux.ensure(OnesweepAuxWords(std::max<uint32_t>(nMax, 2), OS_MAX_PASSES));
        cellAux.ensure(CellTableGridAuxWords(std::max<uint32_t>(nMax, 1)));
        scanScratch.ensure(ScanScratchItems(std::max<uint32_t>(nMax, 1) + 1));
        scanScratch2.ensure(ScanScratchItems(std::max<uint32_t>(nMax, 1) + 1));
        permF.ensure(std::max<uint32_t>(nF, 1)); permB.ensure(std::max<uint32_t>(nB, 1));
        permR.ensure(std::max<uint32_t>(nR, 1));
        cidF.ensure(std::max<uint32_t>(nF, 1)); cidB.ensure(std::max<uint32_t>(nB, 1));
        cidR.ensure(std::max<uint32_t>(nR, 1)); cidRs.ensure(std::max<uint32_t>(nR, 1));
        uniqF.ensure(std::max<uint32_t>(nF, 1)); uniqB.ensure(std::max<uint32_t>(nB, 1));
        uniqR.ensure(std::max<uint32_t>(nR, 1));
        startF.ensure(nF + 1ull); startB.ensure(nB + 1ull); startR.ensure(nR + 1ull);
        const uint32_t nChunks = (nF + SELL_W - 1) / SELL_W;
        for (int k = 0; k < 3; k++) {
            Sell& m = sell[k];
            m.counts.ensure(std::max<uint32_t>(nF, 1));
            m.pitch.ensure(std::max<uint32_t>(nChunks, 1)); m.format.ensure(std::max<uint32_t>(nChunks, 1));
            m.base.ensure(std::max<uint32_t>(nChunks, 1)); m.base2.ensure(std::max<uint32_t>(nChunks, 1));
            m.offset.ensure(std::max<uint32_t>(nChunks, 1));
            m.l16.ensure(std::max<size_t>(m.l16.cap, 16)); m.l32.ensure(std::max<size_t>(m.l32.cap, 16));
            cntR[k].ensure(std::max<uint32_t>(nR, 1)); offR[k].ensure(nR + 1ull);
            listR[k].ensure(std::max<size_t>(listR[k].cap, 16));
        }
        velPred2.ensure(std::max<uint32_t>(nF, 1)); acc2.ensure(std::max<uint32_t>(nF, 1));
        srcDiag2.ensure(std::max<uint32_t>(nF, 1));
        scrF.ensure(std::max<size_t>(QueryScratchWords(nChunks, KS_F), 1));
        scrB.ensure(std::max<size_t>(QueryScratchWords(nChunks, KS_B), 1));
        scrR.ensure(std::max<size_t>(QueryScratchWords(nChunks, nR ? KS_R : 0), 1));
        scrOver.ensure(std::max<uint32_t>(nChunks, 1));
    }
    // ReOrderParticleData + Construct + Query_Count + Finalize_Count + Query_Fill
    void NeighborBuild(bool permuteAll) {
        SetCellSize();
        CK(cudaEventRecord(pev[0], s));
        UpdateFrame();  // a changed frame invalidates the boundary sort through bSortFr
        CK(cudaEventRecord(pev[1], s));
        if (!frameValid) { listsValid = false; return; }
        EnsureNsScratch();
        SortScratch sc{keysA.p, keysB.p, valsA.p, valsB.p, tileHist.p, digitTotals.p, osAux.p, err.p};
        // boundary: sorted under this frame unless it already is (then its permutation this
        // step is the identity, or, on the first build after a pull that kept a sort of the same
        // raw boundary, that sort's permutation)
        if (gridCells > gridB.cap) bSortedValid = false;
        gridF.ensure(gridCells); gridB.ensure(gridCells); gridR.ensure(gridCells);
        const int bs = EnsureBoundarySorted(sc);
        // an already sorted boundary's permutation is the identity: nothing reads it on the
        // device, so it is only materialised when read (tsp_b200_read_permutation)
        permBIdentity = nB && bs == B_ALREADY_SORTED;
        if (nB && bs == B_KEPT_FROM_PULL)
            CK(cudaMemcpyAsync(permB.p, rawPermB.p, nB * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        // fluid: IDs, pos (+pressure), vel (+density) always; all fields for a standalone search
        if (nF) {
            SortByCell(posP.p, nF, fr, sc, permF.p, cidF.p, s);
            LaunchReorderFluidStep(permF.p, posP.p, velRho.p, idF.p, posP2.p, velRho2.p, idF2.p, nF, s);
            Swap(posP, posP2); Swap(velRho, velRho2); Swap(idF, idF2);
            if (permuteAll) {
                GatherF4(permF.p, velPred.p, velPred2.p, nF, s); Swap(velPred, velPred2);
                GatherF4(permF.p, acc.p, acc2.p, nF, s); Swap(acc, acc2);
                GatherF2(permF.p, srcDiag.p, srcDiag2.p, nF, s); Swap(srcDiag, srcDiag2);
            }
            BuildCellTableGrid(cidF.p, nF, uniqF.p, startF.p, nCellsDev.p + 0, gridF.p, fr, gridCells, cellAux.p, err.p, s);
            launches += SortLaunches(nF, fr.keyBits) + 1 + (permuteAll ? 3 : 0) + 1;
        }
        // rigid: cell IDs in storage order, sorted index permutation (747-774)
        if (nR) {
            LaunchCellIds(posR.p, nR, fr, cidR.p, s);
            SortByCell(posR.p, nR, fr, sc, permR.p, cidRs.p, s);
            BuildCellTableGrid(cidRs.p, nR, uniqR.p, startR.p, nCellsDev.p + 2, gridR.p, fr, gridCells, cellAux.p, err.p, s);
            launches += 1 + SortLaunches(nR, fr.keyBits) + 1;
        }
        QueryArgs qa = MakeQueryArgs();
        SellMeta m0 = Meta(0), m1 = Meta(1), m2 = Meta(2);
        RigidLists rl = RLists();
        CK(cudaEventRecord(pev[2], s));
        EnsureTuned(TUNE_QUERY_COUNT, nF, [&](int v) {
            QueryArgs t = qa;
            t.nbrTotals = nullptr;  // tuning runs leave the neighbor totals alone
            t.nF = std::min(nF, TUNE_MAX_N);
            LaunchQueryFluid(false, t, m0, m1, m2, s, v);
        });
        CK(cudaMemsetAsync(nbrTot.p, 0, 3 * sizeof(unsigned long long), s));
        LaunchQueryFluid(false, qa, m0, m1, m2, s);
        LaunchQueryRigid(false, qa, rl, s);
        CK(cudaEventRecord(pev[3], s));
        const uint32_t nChunks = (nF + SELL_W - 1) / SELL_W;
        FinalizeSell3(Meta(0), Meta(1), Meta(2), nChunks, scanScratch2.p, sellTot.p, s);
        if (nR)
            for (int k = 0; k < 3; k++) FinalizeCsr(cntR[k].p, offR[k].p, nR, scanScratch.p, csrTot.p + k, s);
        KGatherNsTotals<<<1, 32, 0, s>>>(sellTot.p, csrTot.p, nCellsDev.p, nbrTot.p, nR ? 1 : 0, nsDev);
        CK(cudaEventRecord(pev[4], s));
        Sync();
        for (int k = 0; k < 3; k++) {
            nNbr[k] = nF ? hm->ns.nbrTot[k] : 0;
            sell[k].n16 = hm->ns.sellTot[k].a;
            sell[k].n32 = hm->ns.sellTot[k].b;
            sell[k].l16.grow(sell[k].n16, LIST_GROWTH);
            sell[k].l32.grow(sell[k].n32, LIST_GROWTH);
            csrN[k] = hm->ns.csrTot[k];
            listR[k].grow(csrN[k], LIST_GROWTH);
        }
        m0 = Meta(0); m1 = Meta(1); m2 = Meta(2);
        rl = RLists();
        EnsureTuned(TUNE_QUERY_FILL, nF, [&](int v) {
            QueryArgs t = qa;
            t.nF = std::min(nF, TUNE_MAX_N);
            LaunchQueryFluid(true, t, m0, m1, m2, s, v);
        });
        LaunchQueryFluid(true, qa, m0, m1, m2, s);
        LaunchQueryRigid(true, qa, rl, s);
        CK(cudaEventRecord(pev[5], s));
        launches += 2u * ((nF ? 1u : 0u) + (nR ? 1u : 0u)) + FinalizeSell3Launches(nChunks) + (nR ? 9u : 0u) + 1u;
        listsValid = true;
    }
    // first run of a kernel for this size class on this device: time its candidates on the live
    // state (the autotuner, tune.cu); kernels that rewrite their own inputs run between a save and
    // a restore of those inputs (positions with pressure, solver state)
    void EnsureTuned(TuneKernel k, uint32_t n, const std::function<void(int)>& launch, bool savePos = false,
                     bool saveSolver = false) {
        if (n == 0 || !TuneEnabled() || TuneChoice(k, n) >= 0) return;
        if (savePos) {
            tunePos.ensure(nF);
            CK(cudaMemcpyAsync(tunePos.p, posP.p, nF * sizeof(float4), cudaMemcpyDeviceToDevice, s));
        }
        if (saveSolver) {
            tuneSt.ensure(1);
            CK(cudaMemcpyAsync(tuneSt.p, st.p, sizeof(SolverState), cudaMemcpyDeviceToDevice, s));
        }
        TuneRun(k, n, launch, s);
        if (savePos) CK(cudaMemcpyAsync(posP.p, tunePos.p, nF * sizeof(float4), cudaMemcpyDeviceToDevice, s));
        if (saveSolver) CK(cudaMemcpyAsync(st.p, tuneSt.p, sizeof(SolverState), cudaMemcpyDeviceToDevice, s));
        CheckErrors();
    }
    QueryArgs MakeQueryArgs() {
        QueryArgs qa{};
        qa.posF = posP.p; qa.cidF = cidF.p; qa.nF = nF;
        qa.posB = posB.p; qa.nB = nB;
        qa.posR = posR.p; qa.permR = permR.p; qa.bodyR = bodyR.p; qa.nR = nR;
        qa.startF = startF.p; qa.startB = startB.p; qa.startR = startR.p;
        qa.gridF = nF ? gridF.p : nullptr; qa.gridB = nB ? gridB.p : nullptr; qa.gridR = nR ? gridR.p : nullptr;
        qa.fr = fr; qa.r2 = prm.kernelRadiusSqu; qa.err = err.p;
        qa.nbrTotals = nbrTot.p;
        qa.scrF = scrF.p; qa.scrB = scrB.p; qa.scrR = scrR.p;
        qa.ksF = KS_F; qa.ksB = KS_B; qa.ksR = nR ? KS_R : 0u;
        qa.scrOver = scrOver.p;
        return qa;
    }
    RigidLists RLists() {
        return RigidLists{cntR[0].p, cntR[1].p, cntR[2].p, offR[0].p, offR[1].p, offR[2].p,
                          listR[0].p, listR[1].p, listR[2].p};
    }

    // -------------------------------------------------------------------------- Jacobi loop graph
    // Exact key of a captured Jacobi graph: every pointer, size and constant its kernels were
    // captured with, field by field (struct padding never enters the key).
    std::vector<uint64_t> GraphKey(const Consts& c, const SolverControl& ctl) {
        std::vector<uint64_t> k;
        auto P = [&](const void* q) { k.push_back((uint64_t)(uintptr_t)q); };
        const FluidDev f = FluidView(); const BoundaryDev b = BoundaryView(); const RigidDev r = RigidDevView();
        const NeighborView nv = NView();
        P(f.posP); P(f.velRho); P(f.velPred); P(f.acc); P(f.srcDiag); k.push_back(f.n);
        P(b.pos); P(b.vol); k.push_back(b.n);
        P(r.pos); P(r.vel); P(r.velPred); k.push_back(r.n);
        for (const SellView* v : {&nv.ff, &nv.fb, &nv.fr}) {
            P(v->counts); P(v->pitch); P(v->format); P(v->base); P(v->base2); P(v->offset);
            P(v->list16); P(v->list32);
        }
        static_assert(sizeof(Consts) % 4 == 0, "Consts holds 4-byte fields only");
        const uint32_t* cw = reinterpret_cast<const uint32_t*>(&c);
        for (size_t i = 0; i < sizeof(Consts) / 4; i++) k.push_back(cw[i]);
        k.push_back(ctl.minIters); k.push_back(ctl.maxIters); k.push_back(ctl.fixedIters); k.push_back(ctl.cond);
        uint32_t tb;
        std::memcpy(&tb, &ctl.target, 4);
        k.push_back(tb); k.push_back(ctl.nF);
        P(st.p); P(partials.p);
        k.push_back((uint64_t)(int64_t)TuneChoice(TUNE_PRESSURE_ACC, f.n));  // the launched instantiations
        k.push_back((uint64_t)(int64_t)TuneChoice(TUNE_JACOBI, f.n));
        return k;
    }
    cudaGraphExec_t JacobiGraphFor(const Consts& c, const SolverControl& ctl) {
        std::vector<uint64_t> key = GraphKey(c, ctl);
        for (auto& g : graphs)
            if (g.ex && g.key == key) return g.ex;
        // build: while (cond) { pressure acceleration; Jacobi sweep (sets cond) }
        cudaGraph_t graph;
        CK(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle handle;
        CK(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(capStream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        FluidDev f = FluidView(); BoundaryDev b = BoundaryView(); RigidDev r = RigidDevView(); NeighborView nv = NView();
        LaunchPressureAcc(c, f, b, r, nv, capStream);
        LaunchJacobi(c, f, b, r, nv, ctl, st.p, partials.p, (unsigned long long)handle, true, capStream);
        cudaGraph_t captured;
        CK(cudaStreamEndCapture(capStream, &captured));
        cudaGraphExec_t ex;
        CK(cudaGraphInstantiate(&ex, graph, 0));
        const size_t maxGraphs = 4;
        if (graphs.size() < maxGraphs) graphs.push_back({});
        JacobiGraph& slot = graphs[graphNext % graphs.size()];
        graphNext++;
        if (slot.ex) cudaGraphExecDestroy(slot.ex);
        if (slot.g) cudaGraphDestroy(slot.g);
        slot.key = std::move(key); slot.g = graph; slot.ex = ex;
        return ex;
    }

    // -------------------------------------------------------------------------- rigid contacts
    ContactDev ContactView() {
        ContactDev d{};
        d.nR = nR; d.nRB = nRB;
        d.nContactB = reinterpret_cast<const uint32_t*>(cTot.p);  // low word of the scan total
        d.offRR = offR[2].p; d.listRR = listR[2].p; d.offRB = offR[1].p; d.listRB = listR[1].p;
        d.idxRB = cIdxRB.p; d.contactOfB = cOfB.p; d.localB = cLocalB.p;
        d.offBR = cOffBR.p; d.idxBR = cIdxBR.p; d.curBR = cCurBR.p;
        d.posR = posR.p; d.relR = relR.p; d.bodyR = bodyR.p; d.byBodyOff = byBodyOff.p; d.byBodyIdx = byBodyIdx.p;
        d.posB = posB.p; d.volB = volB.p; d.bodyState = bodyState.p; d.bodyFT = bodyFT.p;
        d.relW = cRelW.p; d.iw = cIw.p;
        d.densR = cDensR.p; d.diagR = cDiagR.p; d.presR = cPresR.p; d.srcR = cSrcR.p; d.errR = cErrR.p;
        d.omegaR = cOmegaR.p; d.forceC = cForce.p; d.velC = cVel.p;
        d.densB = cDensB.p; d.diagB = cDiagB.p; d.presB = cPresB.p; d.srcB = cSrcB.p; d.errB = cErrB.p;
        d.omegaB = cOmegaB.p;
        d.ftC = cFT.p; d.perBody = cPerBody.p; d.contrib = cContrib.p; d.st = cState.p; d.err = err.p;
        return d;
    }
    std::vector<uint64_t> ContactKey(const Consts& c) {
        std::vector<uint64_t> k;
        const ContactDev d = ContactView();
        const uint64_t* w = reinterpret_cast<const uint64_t*>(&d);
        static_assert(sizeof(ContactDev) % 8 == 0, "ContactDev holds 8-byte fields only after its two counts");
        for (size_t i = 0; i < sizeof(ContactDev) / 8; i++) k.push_back(w[i]);
        const uint32_t* cw = reinterpret_cast<const uint32_t*>(&c);
        for (size_t i = 0; i < sizeof(Consts) / 4; i++) k.push_back(cw[i]);
        k.push_back(contactCap);
        return k;
    }
    cudaGraphExec_t ContactGraphFor(const Consts& c) {
        std::vector<uint64_t> key = ContactKey(c);
        for (auto& g : cgraphs)
            if (g.ex && g.key == key) return g.ex;
        cudaGraph_t graph;
        CK(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle handle;
        CK(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(capStream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        LaunchContactIteration(ContactView(), c, contactCap, (unsigned long long)handle, capStream);
        cudaGraph_t captured;
        CK(cudaStreamEndCapture(capStream, &captured));
        cudaGraphExec_t ex;
        CK(cudaGraphInstantiate(&ex, graph, 0));
        if (cgraphs.size() < 2) cgraphs.push_back({});
        JacobiGraph& slot = cgraphs[cgraphNext % cgraphs.size()];
        cgraphNext++;
        if (slot.ex) cudaGraphExecDestroy(slot.ex);
        if (slot.g) cudaGraphDestroy(slot.g);
        slot.key = std::move(key); slot.g = graph; slot.ex = ex;
        return ex;
    }
    // SolveRigidContacts (rigid_solver.cpp:602-799), between the fluid integration and the rigid
    // predictor/integrator of the step
    void SolveRigidContacts(const Consts& c, const RigidParticlesDev& rp, const BodyDev& bd) {
        const bool defaults = prm.rigidContactDensityDevTarget == 0.0f && prm.rigidContactMaxSolverIters == 0;
        const float target = defaults ? 0.001f : prm.rigidContactDensityDevTarget;
        const uint32_t maxIters = defaults ? 100u : prm.rigidContactMaxSolverIters;
        if (!std::isfinite(target) || target <= 0.0f || maxIters == 0)
            throw Error(TSP_ERR_INVALID, "Invalid rigid contact solver tolerance or iteration limit.");
        if (maxIters > MAX_JACOBI_SWEEPS) throw Error(TSP_ERR_UNSUPPORTED, "contact iteration limit above 100000");
        contactRan = false;
        lastContactB = 0;
        std::memset(&hm->contact, 0, sizeof(ContactState));
        hm->contact.converged = 1u;
        const uint64_t nRBe = csrN[1], nRRe = csrN[2];
        if (nRBe == 0 && nRRe == 0) return;  // BuildRigidBoundaryNeighbors found no contact
        // contact set: boundary particles referenced by rigid RB rows, ascending
        cOfB.ensure(std::max<uint32_t>(nB, 1)); cLocalB.ensure(std::max<uint32_t>(nB, 1));
        cIdxRB.ensure(std::max<uint64_t>(nRBe, 1)); cIdxBR.ensure(std::max<uint64_t>(nRBe, 1));
        cTot.ensure(2);
        CK(cudaMemsetAsync(cTot.p, 0, 2 * sizeof(uint64_t), s));
        ContactDev d0 = ContactView();
        if (nB) LaunchContactSetup(d0, nRBe, nB, scanScratch.p, cTot.p, s);
        CK(cudaMemcpyAsync(hm->contactTot, cTot.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        Sync();
        const uint32_t nc = (uint32_t)hm->contactTot[0];
        if (nc > contactCap || !cDensB.p) {
            contactCap = std::max<uint32_t>(nc + nc / 2 + 64, contactCap);
            for (auto* b : {&cDensB, &cDiagB, &cPresB, &cSrcB, &cErrB, &cOmegaB}) b->ensure(contactCap);
            cCurBR.ensure(contactCap); cOffBR.ensure(contactCap + 1ull);
        }
        const uint32_t nr1 = std::max<uint32_t>(nR, 1), nb1 = std::max<uint32_t>(nRB, 1);
        cRelW.ensure(nr1); cForce.ensure(nr1); cVel.ensure(nr1);
        for (auto* b : {&cDensR, &cDiagR, &cPresR, &cSrcR, &cErrR, &cOmegaR}) b->ensure(nr1);
        cIw.ensure(9ull * nb1); cFT.ensure(6ull * nb1); cPerBody.ensure(nb1);
        cContrib.ensure((uint64_t)nR + contactCap);
        cState.ensure(1);
        ContactDev d = ContactView();
        LaunchContactLists(d, nRBe, nc, scanScratch.p, cTot.p + 1, s);
        LaunchContactPrepare(d, c, nc, target, maxIters, s);
        // predicted motion from external and fluid loads, no contact loads
        LaunchRigidPredict(bd, prm.timeStep, s);
        LaunchRigidUpdateParticles(rp, bd, true, err.p, s);
        LaunchContactInitialError(d, c, nc, velPredR.p, s);
        // the predicted-motion error becomes the source term (the reference swaps the vectors)
        Swap(cSrcR, cErrR);
        Swap(cSrcB, cErrB);
        CK(cudaGraphLaunch(ContactGraphFor(c), s));
        LaunchContactAddLoads(ContactView(), s);
        CK(cudaMemcpyAsync(&hm->contact, cState.p, sizeof(ContactState), cudaMemcpyDeviceToHost, s));
        contactRan = true;
        lastContactB = nc;
        launches += 16;
    }
    // PackExportSnapshot (gpu_backend.cpp:346-540; classification as cpu_backend.cpp:829-975)
    DBuf<uint8_t> expFlags, expMesh;
    DBuf<uint32_t> expTiles, expCount;
    void PackExport(const tsp_params& p, bool includeB, uint64_t meshBegin, tsp_export_snapshot& o) {
        CK(cudaSetDevice(device));
        o.simStep = stepCount;
        o.simTime = simTime;
        DBuf<float>& tmp = stage;
        o.N_B = includeB ? nB : 0u;
        if (o.N_B) {
            Unpack4(posB.p, nB, o.xPosB, o.yPosB, o.zPosB, nullptr, tmp);
            if (o.volB) CK(cudaMemcpyAsync(o.volB, volB.p, nB * 4ull, cudaMemcpyDeviceToHost, s));
            if (o.isMeshB) {
                expMesh.ensure(nB);
                LaunchMeshFlags(idB.p, nB, meshBegin, expMesh.p, s);
                CK(cudaMemcpyAsync(o.isMeshB, expMesh.p, nB, cudaMemcpyDeviceToHost, s));
                launches += 1;
            }
            launches += 1;
            Sync();
        }
        o.N_R = nR;
        if (nR) {
            if (o.bodyIdR) CK(cudaMemcpyAsync(o.bodyIdR, bodyR.p, nR * 4ull, cudaMemcpyDeviceToHost, s));
            Unpack4(posR.p, nR, o.xPosR, o.yPosR, o.zPosR, nullptr, tmp);
            Sync();
            Unpack4(relR.p, nR, nullptr, nullptr, nullptr, o.volR, tmp);
            launches += 2;
            Sync();
        }
        o.N_F = 0;
        if (nF == 0 || !listsValid) return;
        const uint32_t threshold = p.surfaceNbrCountThreshold ? p.surfaceNbrCountThreshold : 27u;
        expFlags.ensure(nF);
        expTiles.ensure(ExportTiles(nF));
        expCount.ensure(1);
        tmp.ensure(4ull * nF);
        const NeighborView nv = NView();
        LaunchExportSurface(nv.ff, nv.fb.counts, nv.fr.counts, nF, threshold, posP.p, velRho.p, expFlags.p,
                            expTiles.p, expCount.p, tmp.p, nF, s);
        launches += 4;
        CK(cudaMemcpyAsync(&hm->exportCount, expCount.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        Sync();
        const uint32_t nS = hm->exportCount;
        if (nS > nF) throw Error(TSP_ERR_INVALID, "export surface count exceeds the fluid count");
        o.N_F = nS;
        float* dst[4] = {o.xPosF, o.yPosF, o.zPosF, o.velMagF};
        for (int k = 0; k < 4; k++)
            if (dst[k] && nS) CK(cudaMemcpyAsync(dst[k], tmp.p + (uint64_t)k * nF, nS * 4ull, cudaMemcpyDeviceToHost, s));
        Sync();
    }
    // FillStatisticsRecord (gpu_backend.cpp:1067-1203) of the last step / neighbor search
    DBuf<uint32_t> statHist, statOut;
    DBuf<double> statPart, statF;
    DBuf<float> statMM;
    void Statistics(const tsp_params& p, double* rec, uint32_t n) {
        CK(cudaSetDevice(device));
        double r[TSP_STAT_COUNT] = {};
        r[TSP_STAT_NUM_F] = nF; r[TSP_STAT_NUM_B] = nB; r[TSP_STAT_NUM_R] = nR;
        statHist.ensure(65536); statOut.ensure(18); statF.ensure(6);
        const uint32_t blocks = StatFieldBlocks(nF);
        statPart.ensure(4ull * blocks); statMM.ensure(2ull * blocks);
        uint32_t cnt[18] = {};
        double fld[6] = {};
        if (listsValid) {
            const uint16_t* counts[6] = {sell[0].counts.p, sell[1].counts.p, sell[2].counts.p,
                                         cntR[0].p, cntR[1].p, cntR[2].p};
            const uint32_t srcN[6] = {nF, nF, nF, nR, nR, nR};
            for (int k = 0; k < 6; k++)
                LaunchStatNeighborCounts(srcN[k] ? counts[k] : nullptr, srcN[k], statHist.p, statOut.p + 3 * k, s);
            CK(cudaMemcpyAsync(cnt, statOut.p, sizeof(cnt), cudaMemcpyDeviceToHost, s));
        }
        if (nF) {
            LaunchStatFields(velRho.p, nF, p.restDensity, statPart.p, statMM.p, statF.p, s);
            CK(cudaMemcpyAsync(fld, statF.p, sizeof(fld), cudaMemcpyDeviceToHost, s));
        }
        Sync();
        const double invNF = nF ? 1.0 / (double)nF : 0.0, invNR = nR ? 1.0 / (double)nR : 0.0;
        const uint64_t tot[6] = {nNbr[0], nNbr[1], nNbr[2], csrN[0], csrN[1], csrN[2]};
        for (int k = 0; k < 6 && listsValid; k++) {
            const double inv = k < 3 ? invNF : invNR;
            r[TSP_STAT_NUM_NBR_FF_AVG + 4 * k] = (double)tot[k] * inv;
            r[TSP_STAT_NUM_NBR_FF_MIN + 4 * k] = cnt[3 * k];
            r[TSP_STAT_NUM_NBR_FF_MAX + 4 * k] = cnt[3 * k + 1];
            r[TSP_STAT_NUM_NBR_FF_P99 + 4 * k] = cnt[3 * k + 2];
        }
        r[TSP_STAT_DENS_REL_ERROR_RAW_AVG] = fld[0] * invNF;
        r[TSP_STAT_DENS_REL_ERROR_POS_AVG] = fld[1] * invNF;
        r[TSP_STAT_DENS_REL_ERROR_ABS_AVG] = fld[2] * invNF;
        r[TSP_STAT_NUM_SOLVER_ITERS] = hm->st.iters;
        const float vmax = nF ? (float)fld[5] : 0.0f;
        r[TSP_STAT_CFL_NUMBER] = vmax * p.timeStep / p.particleSizeF;
        r[TSP_STAT_VEL_MAG_AVG] = fld[3] * invNF;
        r[TSP_STAT_VEL_MAG_MIN] = nF ? fld[4] : 0.0;
        r[TSP_STAT_VEL_MAG_MAX] = vmax;
        for (uint32_t k = 0; k < n && k < (uint32_t)TSP_STAT_COUNT; k++) rec[k] = r[k];
    }
    void ContactReport(tsp_contact_report& o) {
        Sync();
        o = tsp_contact_report{};
        o.solverIters = hm->contact.iters;
        o.avgDensityError = hm->contact.avgErr;
        o.converged = contactRan ? hm->contact.converged : 1u;
        o.nContacts = hm->contact.nContacts;
        o.nContactBoundary = lastContactB;
    }

    // -------------------------------------------------------------------------- step
    void Step(const tsp_params& p) {  // Step_IISPH (sph_solver.cpp:34-319) without the contact solve
        CK(cudaSetDevice(device));
        prm = p;
        if (p.solverTerminationCond > 3) throw Error(TSP_ERR_INVALID, "unknown solver termination condition");
        if (p.maxSolverIters > MAX_JACOBI_SWEEPS || p.minSolverIters > MAX_JACOBI_SWEEPS)
            throw Error(TSP_ERR_UNSUPPORTED, "solver iteration bounds above 100000");
        if (!(p.timeStep >= 0.0f) || !(p.particleSizeF > 0.0f) || !(p.kernelRadiusSqu > 0.0f))
            throw Error(TSP_ERR_INVALID, "time step, particle size and kernel radius must be positive");
        if (nF == 0 && nRB == 0) return;  // empty serial sim (cpu_backend.cpp:2309-2315)
        const Consts c = MakeConsts(prm);
        phaseValid = false;
        CK(cudaEventRecord(ev[0], s));
        NeighborBuild(false);
        CK(cudaEventRecord(ev[1], s));
        FluidDev f = FluidView(); BoundaryDev b = BoundaryView(); RigidDev r = RigidDevView(); NeighborView nv = NView();
        RigidParticlesDev rp = RigidView(); BodyDev bd = BodyView();
        const FluidDev ft = TuneView(f, nF);
        EnsureTuned(TUNE_DENSITY, nF, [&](int v) { LaunchDensity(c, ft, b, r, nv, s, v); });
        LaunchDensity(c, f, b, r, nv, s);
        if (nRB) LaunchRigidClearAddGravity(bd, prm.gravity[0], prm.gravity[1], prm.gravity[2], s);
        CK(cudaEventRecord(pev[6], s));
        EnsureTuned(TUNE_NON_PRESSURE, nF, [&](int v) { LaunchNonPressure(c, ft, b, r, nv, s, v); });
        LaunchNonPressure(c, f, b, r, nv, s);
        if (nRB) {
            LaunchRigidViscousForces(c, rp, f, offR[0].p, listR[0].p, s);
            LaunchRigidReduce(rp, bd, s);
            LaunchRigidPredict(bd, prm.timeStep, s);
            LaunchRigidUpdateParticles(rp, bd, true, err.p, s);
        }
        CK(cudaEventRecord(pev[7], s));
        EnsureTuned(TUNE_SOURCE_DIAG, nF, [&](int v) { LaunchSourceDiagInit(c, ft, b, r, nv, nullptr, s, v); }, true);
        LaunchSourceDiagInit(c, f, b, r, nv, st.p, s);
        CK(cudaEventRecord(ev[2], s));
        CK(cudaEventRecord(pev[8], s));
        if (nF) {
            partials.ensure(3ull * JacobiBlocks(nF) + 3);
            const SolverControl ctl = Control();
            EnsureTuned(TUNE_PRESSURE_ACC, nF, [&](int v) { LaunchPressureAcc(c, ft, b, r, nv, s, v); });
            EnsureTuned(TUNE_JACOBI, nF, [&](int v) {
                LaunchJacobi(c, ft, b, r, nv, ctl, st.p, partials.p, 0ull, false, s, v);
            }, true, true);
            cudaGraphExec_t ex = JacobiGraphFor(c, ctl);
            CK(cudaGraphLaunch(ex, s));
        }
        CK(cudaEventRecord(ev[3], s));
        CK(cudaEventRecord(pev[9], s));
        LaunchPressureAcc(c, f, b, r, nv, s);
        if (nRB) {
            LaunchRigidPressureForces(c, rp, f, offR[0].p, listR[0].p, s);
            LaunchRigidClearAddGravity(bd, prm.gravity[0], prm.gravity[1], prm.gravity[2], s);
            LaunchRigidReduce(rp, bd, s);
        }
        CK(cudaEventRecord(pev[10], s));
        LaunchIntegration(c, f, s);
        if (nRB) {
            SolveRigidContacts(c, rp, bd);
            LaunchRigidPredict(bd, prm.timeStep, s);
            LaunchRigidIntegrate(bd, prm.timeStep, err.p, s);
            LaunchRigidUpdateParticles(rp, bd, false, err.p, s);
        }
        CK(cudaEventRecord(pev[11], s));
        probeFresh = false;
        const bool probeNext = frameValid;  // the next step's frame rule reads it with this read-back
        if (probeNext) QueueProbe();
        QueueStepEnd(true, probeNext);
        launches += (nF ? 6u : 0u) + (nRB ? 13u : 0u);
        CK(cudaEventRecord(pev[12], s));
        Sync();
        hm->st = hm->se.st;
        if (probeNext) hm->probe = hm->se.probe;
        RaiseErrors(hm->se.err);
        probeFresh = probeNext;
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[0], pev[12]); lastStepMs = t;
        stepMsTotal += t;
        stepsTimed += 1;
        cudaEventElapsedTime(&t, ev[0], ev[1]); lastNbrMs = t;
        cudaEventElapsedTime(&t, ev[2], ev[3]); lastJacMs = t;
        phaseValid = listsValid;
        if (nF && hm->st.iters > 0) launches += 2ull * (hm->st.iters - 1u);
    }

    void RecordStep() {
        if (hist.empty()) hist.resize(HIST_CAP);
        tsp_step_record& r = hist[histCount % HIST_CAP];
        r.step = stepCount;
        r.ms = lastStepMs;
        r.solverIters = hm->st.iters;
        r.avgRelDensityErrPos = hm->st.avg[1];
        histCount++;
    }
    uint32_t History(tsp_step_record* out, uint32_t cap) const {
        const uint64_t kept = std::min<uint64_t>(histCount, HIST_CAP);
        const uint64_t m = std::min<uint64_t>(kept, cap);
        for (uint64_t k = 0; k < m; k++) out[k] = hist[(histCount - m + k) % HIST_CAP];
        return (uint32_t)m;
    }

    // device milliseconds between consecutive phase events of the last completed step
    uint32_t PhaseTimes(float* ms, uint32_t cap) {
        if (!phaseValid) return 0;
        const uint32_t n = std::min<uint32_t>(cap, N_PHASE_EVENTS - 1);
        for (uint32_t k = 0; k < n; k++) {
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, pev[k], pev[k + 1]));
            ms[k] = t;
        }
        return n;
    }

    void NeighborSearchStandalone(const tsp_params& p) {  // ExecuteNeighborSearch (cpu_backend.cpp:1593-1624)
        CK(cudaSetDevice(device));
        prm = p;
        NeighborBuild(true);
        CheckErrors();
    }

    void RunStage(const tsp_params& p, uint32_t stage, double* errSums) {
        CK(cudaSetDevice(device));
        prm = p;
        const Consts c = MakeConsts(prm);
        FluidDev f = FluidView(); BoundaryDev b = BoundaryView(); RigidDev r = RigidDevView(); NeighborView nv = NView();
        if (stage != TSP_STAGE_BOUNDARY_VOLUMES && stage != TSP_STAGE_INTEGRATION && !listsValid)
            throw Error(TSP_ERR_INVALID, "run the neighbor search before a solver stage");
        switch (stage) {
            case TSP_STAGE_DENSITY: LaunchDensity(c, f, b, r, nv, s); break;
            case TSP_STAGE_NON_PRESSURE: LaunchNonPressure(c, f, b, r, nv, s); break;
            case TSP_STAGE_SOURCE_DIAG_INIT: LaunchSourceDiagInit(c, f, b, r, nv, st.p, s); break;
            case TSP_STAGE_PRESSURE_ACC: LaunchPressureAcc(c, f, b, r, nv, s); break;
            case TSP_STAGE_JACOBI_UPDATE: {
                partials.ensure(3ull * JacobiBlocks(nF) + 3);
                LaunchJacobi(c, f, b, r, nv, Control(), st.p, partials.p, 0ull, false, s);
                CK(cudaMemcpyAsync(&hm->st, st.p, sizeof(SolverState), cudaMemcpyDeviceToHost, s));
                Sync();
                if (errSums) for (int k = 0; k < 3; k++) errSums[k] = hm->st.sums[k];
                break;
            }
            case TSP_STAGE_INTEGRATION: LaunchIntegration(c, f, s); probeFresh = false; break;
            case TSP_STAGE_BOUNDARY_VOLUMES: BoundaryVolumes(c); break;
            default: throw Error(TSP_ERR_INVALID, "unknown stage");
        }
        CheckErrors();
    }

    // device time per launch of one solver stage (CUDA events on the backend stream)
    float TimeStage(const tsp_params& p, uint32_t stage, uint32_t reps) {
        CK(cudaSetDevice(device));
        prm = p;
        if (!listsValid) throw Error(TSP_ERR_INVALID, "run the neighbor search before timing a stage");
        if (reps == 0) reps = 1;
        const Consts c = MakeConsts(prm);
        FluidDev f = FluidView(); BoundaryDev b = BoundaryView(); RigidDev r = RigidDevView(); NeighborView nv = NView();
        partials.ensure(3ull * JacobiBlocks(nF) + 3);
        const SolverControl ctl = Control();
        Sync();
        CK(cudaEventRecord(ev[0], s));
        for (uint32_t k = 0; k < reps; k++) {
            switch (stage) {
                case TSP_STAGE_DENSITY: LaunchDensity(c, f, b, r, nv, s); break;
                case TSP_STAGE_NON_PRESSURE: LaunchNonPressure(c, f, b, r, nv, s); break;
                case TSP_STAGE_SOURCE_DIAG_INIT: LaunchSourceDiagInit(c, f, b, r, nv, st.p, s); break;
                case TSP_STAGE_PRESSURE_ACC: LaunchPressureAcc(c, f, b, r, nv, s); break;
                case TSP_STAGE_JACOBI_UPDATE: LaunchJacobi(c, f, b, r, nv, ctl, st.p, partials.p, 0ull, false, s); break;
                case TSP_STAGE_INTEGRATION: LaunchIntegration(c, f, s); probeFresh = false; break;
                default: throw Error(TSP_ERR_INVALID, "stage cannot be timed");
            }
            launches += 1;
        }
        CK(cudaEventRecord(ev[1], s));
        CheckErrors();
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        return ms / (float)reps;
    }

    // ComputeBoundaryCoefficients / ComputeRigidCoefficients (builder.cpp:150-376)
    void BoundaryVolumes(const Consts& c) {
        const float defPsi = prm.massB, defVol = prm.restDensity > 0.0f ? prm.massB / prm.restDensity : 0.0f;
        const float cs = prm.kernelRadius * prm.gridCellSizeRatio;
        if (!(prm.particleSizeF > 0.f && prm.kernelRadius > 0.f && prm.kernelRadiusSqu > 0.f &&
              prm.gridCellSizeRatio > 0.f && prm.restDensity > 0.f && cs > 0.f)) {
            std::vector<float> dv(std::max(nB, nR), defVol), dp(std::max(nB, nR), defPsi);
            if (nB) {
                CK(cudaMemcpy(volB.p, dv.data(), nB * 4ull, cudaMemcpyHostToDevice));
                psiTmpB.ensure(nB);
                CK(cudaMemcpy(psiTmpB.p, dp.data(), nB * 4ull, cudaMemcpyHostToDevice));
                KSetW<<<G(nB), 256, 0, s>>>(posB.p, psiTmpB.p, nB);
                bState = B_OTHER;
            }
            if (nR) {
                CK(cudaMemcpy(volR.p, dv.data(), nR * 4ull, cudaMemcpyHostToDevice));
                CK(cudaMemcpy(psiR.p, dp.data(), nR * 4ull, cudaMemcpyHostToDevice));
                KSetW<<<G(nR), 256, 0, s>>>(relR.p, volR.p, nR);
                KSetW<<<G(nR), 256, 0, s>>>(posR.p, psiR.p, nR);
            }
            return;
        }
        if (nB) {
            // the boundary must be sorted and gridded under the current frame
            SetCellSize();
            UpdateFrame();
            EnsureNsScratch();
            if (gridCells > gridB.cap) bSortedValid = false;
            gridF.ensure(gridCells); gridB.ensure(gridCells); gridR.ensure(gridCells);
            SortScratch sc{keysA.p, keysB.p, valsA.p, valsB.p, tileHist.p, digitTotals.p, osAux.p, err.p};
            EnsureBoundarySorted(sc);
            psiTmpB.ensure(nB);
            LaunchBoundaryVolumes(c, posB.p, nB, startB.p, gridB.p, fr, defVol, defPsi, prm.restDensity, volB.p,
                                  psiTmpB.p, s);
            KSetW<<<G(nB), 256, 0, s>>>(posB.p, psiTmpB.p, nB);
            bState = B_OTHER;  // volumes and psi no longer those of the raw upload
        }
        if (nR) {
            // per body, in the body frame, over the body's own particles, sorted by (z, y, x) cell
            const float csInv = 1.0f / cs;
            const float span = prm.kernelRadius / cs;
            const int rr = std::max(1, (int)std::ceil(std::max(0.0f, span - 1e-6f)));
            std::vector<uint32_t> sortedIdx(nR), bodyOf(nR);
            std::vector<int4> cells(nR);
            for (uint32_t b = 0; b < nRB; b++) {
                const uint32_t lo = hByBodyOff[b], hi = hByBodyOff[b + 1];
                std::vector<uint32_t> loc(hByBodyIdx.begin() + lo, hByBodyIdx.begin() + hi);
                std::sort(loc.begin(), loc.end());
                auto cellOf = [&](uint32_t i) {
                    return int4{(int)std::floor(hRelX[i] * csInv), (int)std::floor(hRelY[i] * csInv),
                                (int)std::floor(hRelZ[i] * csInv), 0};
                };
                std::stable_sort(loc.begin(), loc.end(), [&](uint32_t a, uint32_t bb) {
                    const int4 ca = cellOf(a), cb = cellOf(bb);
                    if (ca.z != cb.z) return ca.z < cb.z;
                    if (ca.y != cb.y) return ca.y < cb.y;
                    return ca.x < cb.x;
                });
                for (uint32_t k = 0; k < hi - lo; k++) {
                    sortedIdx[lo + k] = loc[k];
                    cells[lo + k] = cellOf(loc[k]);
                    bodyOf[lo + k] = b;
                }
            }
            DBuf<uint32_t> dIdx, dBody;
            DBuf<int4> dCells;
            Upload(dIdx, sortedIdx.data(), nR);
            Upload(dBody, bodyOf.data(), nR);
            Upload(dCells, cells.data(), nR);
            LaunchRigidVolumesSorted(c, relR.p, byBodyOff.p, dIdx.p, dCells.p, dBody.p, nR, rr, defVol, defPsi,
                                     prm.restDensity, volR.p, psiR.p, s);
            KSetW<<<G(nR), 256, 0, s>>>(relR.p, volR.p, nR);
            KSetW<<<G(nR), 256, 0, s>>>(posR.p, psiR.p, nR);
            LaunchRigidUpdateParticles(RigidView(), BodyView(), false, err.p, s);
            Sync();
        }
    }

    // -------------------------------------------------------------------------- inspection
    void ReadField(uint32_t field, void* out, uint32_t n) {
        DBuf<float>& tmp = stage;
        float* o = (float*)out;
        auto un3 = [&](const float4* src, uint32_t cnt) {
            if (n != cnt) throw Error(TSP_ERR_INVALID, "field size mismatch");
            std::vector<float> a(cnt), b(cnt), c(cnt);
            Unpack4(src, cnt, a.data(), b.data(), c.data(), nullptr, tmp);
            Sync();
            for (uint32_t i = 0; i < cnt; i++) { o[3 * i] = a[i]; o[3 * i + 1] = b[i]; o[3 * i + 2] = c[i]; }
        };
        auto unW = [&](const float4* src, uint32_t cnt) {
            if (n != cnt) throw Error(TSP_ERR_INVALID, "field size mismatch");
            Unpack4(src, cnt, nullptr, nullptr, nullptr, o, tmp);
            Sync();
        };
        auto un1 = [&](const float* src, uint32_t cnt) {
            if (n != cnt) throw Error(TSP_ERR_INVALID, "field size mismatch");
            if (cnt) CK(cudaMemcpy(o, src, cnt * 4ull, cudaMemcpyDeviceToHost));
        };
        CK(cudaStreamSynchronize(s));
        switch (field) {
            case TSP_FIELD_POS: un3(posP.p, nF); break;
            case TSP_FIELD_VEL: un3(velRho.p, nF); break;
            case TSP_FIELD_VEL_PRED: un3(velPred.p, nF); break;
            case TSP_FIELD_ACC_PRESS: un3(acc.p, nF); break;
            case TSP_FIELD_PRESSURE: unW(posP.p, nF); break;
            case TSP_FIELD_DENSITY: unW(velRho.p, nF); break;
            case TSP_FIELD_SOURCE:
            case TSP_FIELD_DIAG: {
                if (n != nF) throw Error(TSP_ERR_INVALID, "field size mismatch");
                std::vector<float2> v(nF);
                if (nF) CK(cudaMemcpy(v.data(), srcDiag.p, nF * 8ull, cudaMemcpyDeviceToHost));
                for (uint32_t i = 0; i < nF; i++) o[i] = field == TSP_FIELD_SOURCE ? v[i].x : v[i].y;
                break;
            }
            case TSP_FIELD_VOL_B: un1(volB.p, nB); break;
            case TSP_FIELD_PSI_B: unW(posB.p, nB); break;
            case TSP_FIELD_VOL_R: unW(relR.p, nR); break;
            case TSP_FIELD_PSI_R: unW(posR.p, nR); break;
            case TSP_FIELD_FORCE_R: un3(forceR.p, nR); break;
            case TSP_FIELD_BODY_FT:
                if (n != nRB) throw Error(TSP_ERR_INVALID, "field size mismatch");
                if (nRB) CK(cudaMemcpy(out, bodyFT.p, nRB * 6ull * 8ull, cudaMemcpyDeviceToHost));
                break;
            default: throw Error(TSP_ERR_INVALID, "unknown field");
        }
    }
    void WriteField(uint32_t field, const void* in, uint32_t n) {
        const float* x = (const float*)in;
        CK(cudaStreamSynchronize(s));
        auto setW = [&](DBuf<float4>& dst, uint32_t cnt) {
            if (n != cnt) throw Error(TSP_ERR_INVALID, "field size mismatch");
            DBuf<float> t;
            t.ensure(std::max<uint32_t>(cnt, 1));
            if (cnt) CK(cudaMemcpy(t.p, x, cnt * 4ull, cudaMemcpyHostToDevice));
            KSetW<<<G(cnt), 256, 0, s>>>(dst.p, t.p, cnt);
            Sync();
        };
        auto set3 = [&](DBuf<float4>& dst, uint32_t cnt) {
            if (n != cnt) throw Error(TSP_ERR_INVALID, "field size mismatch");
            std::vector<float4> h(cnt);
            if (cnt) CK(cudaMemcpy(h.data(), dst.p, cnt * 16ull, cudaMemcpyDeviceToHost));
            for (uint32_t i = 0; i < cnt; i++) { h[i].x = x[3 * i]; h[i].y = x[3 * i + 1]; h[i].z = x[3 * i + 2]; }
            if (cnt) CK(cudaMemcpy(dst.p, h.data(), cnt * 16ull, cudaMemcpyHostToDevice));
        };
        switch (field) {
            case TSP_FIELD_POS: set3(posP, nF); probeFresh = false; break;
            case TSP_FIELD_VEL: set3(velRho, nF); break;
            case TSP_FIELD_VEL_PRED: set3(velPred, nF); break;
            case TSP_FIELD_ACC_PRESS: set3(acc, nF); break;
            case TSP_FIELD_PRESSURE: setW(posP, nF); break;
            case TSP_FIELD_DENSITY: setW(velRho, nF); break;
            case TSP_FIELD_SOURCE:
            case TSP_FIELD_DIAG: {
                if (n != nF) throw Error(TSP_ERR_INVALID, "field size mismatch");
                std::vector<float2> v(nF);
                if (nF) CK(cudaMemcpy(v.data(), srcDiag.p, nF * 8ull, cudaMemcpyDeviceToHost));
                for (uint32_t i = 0; i < nF; i++) (field == TSP_FIELD_SOURCE ? v[i].x : v[i].y) = x[i];
                if (nF) CK(cudaMemcpy(srcDiag.p, v.data(), nF * 8ull, cudaMemcpyHostToDevice));
                break;
            }
            case TSP_FIELD_VOL_B:
                if (n != nB) throw Error(TSP_ERR_INVALID, "field size mismatch");
                if (nB) CK(cudaMemcpy(volB.p, x, nB * 4ull, cudaMemcpyHostToDevice));
                bState = B_OTHER;
                break;
            case TSP_FIELD_PSI_B: setW(posB, nB); bState = B_OTHER; break;
            default: throw Error(TSP_ERR_INVALID, "field is not writable");
        }
    }
    void Stats(tsp_step_stats& o) {
        Sync();
        std::memset(&o, 0, sizeof(o));
        o.step = stepCount; o.time = simTime;
        o.solverIters = hm->st.iters;
        o.errSumRaw = hm->st.sums[0]; o.errSumPos = hm->st.sums[1]; o.errSumAbs = hm->st.sums[2];
        o.avgRelDensityErrRaw = hm->st.avg[0]; o.avgRelDensityErrPos = hm->st.avg[1]; o.avgRelDensityErrAbs = hm->st.avg[2];
        o.frameRebuilds = frameRebuilds;
        o.cellOrig[0] = fr.ox; o.cellOrig[1] = fr.oy; o.cellOrig[2] = fr.oz;
        o.cellDims[0] = fr.nx; o.cellDims[1] = fr.ny; o.cellDims[2] = fr.nz;
        o.keyBits = fr.keyBits;
        o.nCellsF = nF ? (uint32_t)hm->ns.nCells[0] : 0; o.nCellsB = nB ? (uint32_t)hm->ns.nCells[1] : 0;
        o.nCellsR = nR ? (uint32_t)hm->ns.nCells[2] : 0;
        const bool lv = listsValid && nF;
        o.nNbrFF = lv ? nNbr[0] : 0; o.nNbrFB = lv ? nNbr[1] : 0; o.nNbrFR = lv ? nNbr[2] : 0;
        o.nNbrRF = csrN[0]; o.nNbrRB = csrN[1]; o.nNbrRR = csrN[2];
        for (int k = 0; k < 3; k++) o.sellPackedBytes += sell[k].n16 * 2 + sell[k].n32 * 4;
        o.lastStepMs = lastStepMs; o.lastNeighborMs = lastNbrMs; o.lastJacobiMs = lastJacMs;
    }
};

}  // namespace tsp

// ================================================================================ C ABI
using tsp::Backend;
using tsp::Error;

struct tsp_backend {
    Backend* b;
};

static thread_local std::string g_lastError;

#define TSP_GUARD(h, body)                                                 \
    try {                                                                  \
        body;                                                              \
        return TSP_OK;                                                     \
    } catch (const Error& e) {                                             \
        if (h) (h)->b->lastErr = e.what();                                 \
        g_lastError = e.what();                                            \
        return e.code;                                                     \
    } catch (const std::exception& e) {                                    \
        if (h) (h)->b->lastErr = e.what();                                 \
        g_lastError = e.what();                                            \
        return TSP_ERR_INVALID;                                            \
    }

#define TSP_NEED(h)                                                        \
    if (!(h) || !(h)->b) {                                                 \
        g_lastError = "NULL backend handle";                               \
        return TSP_ERR_INVALID;                                            \
    }

extern "C" {

int tsp_b200_create(const tsp_params* params, int device, tsp_backend** out) {
    if (!params || !out) { g_lastError = "NULL argument"; return TSP_ERR_INVALID; }
    tsp_backend* h = nullptr;
    try {
        h = new tsp_backend{new Backend(device)};
        h->b->prm = *params;
        *out = h;
        return TSP_OK;
    } catch (const Error& e) {
        g_lastError = e.what();
        if (h) { delete h->b; delete h; }
        return e.code;
    } catch (const std::exception& e) {
        g_lastError = e.what();
        return TSP_ERR_INVALID;
    }
}
int tsp_b200_destroy(tsp_backend* h) {
    if (!h) return TSP_OK;
    delete h->b;
    delete h;
    return TSP_OK;
}
const char* tsp_b200_name(const tsp_backend*) { return "B200 (sm_100a) IISPH"; }
int tsp_b200_set_autotune(int enabled) {
    tsp::SetTuneEnabled(enabled != 0);
    return TSP_OK;
}
int tsp_b200_set_tuning(int device, const char* kernel, uint32_t n, uint32_t slots, uint32_t min_blocks) {
    if (!kernel) { g_lastError = "NULL argument"; return TSP_ERR_INVALID; }
    int prev = 0;
    cudaGetDevice(&prev);
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) { g_lastError = "no such device"; return TSP_ERR_NO_DEVICE; }
    const bool ok = tsp::TuneSet(kernel, n, slots, min_blocks);
    if (device >= 0) cudaSetDevice(prev);
    if (!ok) { g_lastError = "not a tuned kernel or not one of its configurations"; return TSP_ERR_INVALID; }
    return TSP_OK;
}
int tsp_b200_reset_tuning(void) {
    tsp::TuneReset();
    return TSP_OK;
}
int tsp_b200_get_tuning(int device, char* out, uint32_t cap, uint32_t* len) {
    if (!len) { g_lastError = "NULL argument"; return TSP_ERR_INVALID; }
    int prev = 0;
    cudaGetDevice(&prev);
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) { g_lastError = "no such device"; return TSP_ERR_NO_DEVICE; }
    const std::string r = tsp::TuneReport();
    if (device >= 0) cudaSetDevice(prev);
    *len = (uint32_t)r.size();
    if (out && cap) {
        const size_t n = std::min<size_t>(r.size(), cap - 1);
        std::memcpy(out, r.data(), n);
        out[n] = 0;
    }
    return TSP_OK;
}
int tsp_b200_try_build_cell_frame(const int64_t cell_min[3], const int64_t cell_max[3], int32_t origin[3],
                                  uint32_t dims[3]) {
    if (!cell_min || !cell_max || !origin || !dims) return TSP_ERR_INVALID;
    int32_t o[3] = {origin[0], origin[1], origin[2]};
    uint32_t d[3] = {dims[0], dims[1], dims[2]};
    if (!tsp::TryBuildCellFrame(cell_min, cell_max, o[0], o[1], o[2], d[0], d[1], d[2])) {
        g_lastError = "Compact CLL cell frame exceeds the supported range.";
        return TSP_ERR_FRAME;
    }
    for (int a = 0; a < 3; a++) { origin[a] = o[a]; dims[a] = d[a]; }
    return TSP_OK;
}
const char* tsp_b200_last_error(const tsp_backend* h) {
    return (h && h->b) ? h->b->lastErr.c_str() : g_lastError.c_str();
}
int tsp_b200_set_domain(tsp_backend* h, const float* mn, const float* mx) {
    TSP_NEED(h);
    if (!mn || !mx) return TSP_ERR_INVALID;
    TSP_GUARD(h, h->b->SetDomain(mn, mx));
}
int tsp_b200_pull_state(tsp_backend* h, const tsp_state_view* src, const tsp_params* p) {
    TSP_NEED(h);
    if (!src || !p) return TSP_ERR_INVALID;
    TSP_GUARD(h, h->b->Pull(*src, *p));
}
int tsp_b200_push_state(tsp_backend* h, tsp_state_view* dst) {
    TSP_NEED(h);
    if (!dst) return TSP_ERR_INVALID;
    TSP_GUARD(h, h->b->Push(*dst));
}
int tsp_b200_get_counts(const tsp_backend* h, uint32_t* nF, uint32_t* nB, uint32_t* nR, uint32_t* nRB) {
    TSP_NEED(h);
    if (nF) *nF = h->b->nF;
    if (nB) *nB = h->b->nB;
    if (nR) *nR = h->b->nR;
    if (nRB) *nRB = h->b->nRB;
    return TSP_OK;
}
int tsp_b200_neighbor_search(tsp_backend* h, const tsp_params* p) {
    TSP_NEED(h);
    if (!p) return TSP_ERR_INVALID;
    TSP_GUARD(h, h->b->NeighborSearchStandalone(*p));
}
int tsp_b200_step(tsp_backend* h, const tsp_params* p, uint32_t n) {
    TSP_NEED(h);
    if (!p) return TSP_ERR_INVALID;
    TSP_GUARD(h, {
        for (uint32_t k = 0; k < n; k++) {
            const uint64_t timed = h->b->stepsTimed;
            h->b->Step(*p);
            h->b->stepCount += 1;
            h->b->simTime += (double)p->timeStep;
            if (h->b->stepsTimed != timed) h->b->RecordStep();
        }
    });
}
int tsp_b200_get_stats(const tsp_backend* h, tsp_step_stats* out) {
    TSP_NEED(h);
    if (!out) return TSP_ERR_INVALID;
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, hh->b->Stats(*out));
}
int tsp_b200_read_cell_ids(const tsp_backend* h, uint32_t species, uint64_t* out, uint32_t n) {
    TSP_NEED(h);
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, {
        Backend& b = *hh->b;
        b.Sync();
        const uint32_t cnt = species == 0 ? b.nF : species == 1 ? b.nB : b.nR;
        if (n != cnt || !out) throw Error(TSP_ERR_INVALID, "size mismatch");
        const uint64_t* src = species == 0 ? b.cidF.p : species == 1 ? b.cidB.p : b.cidR.p;
        if (cnt) CK(cudaMemcpy(out, src, cnt * 8ull, cudaMemcpyDeviceToHost));
    });
}
int tsp_b200_read_permutation(const tsp_backend* h, uint32_t species, uint32_t* out, uint32_t n) {
    TSP_NEED(h);
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, {
        Backend& b = *hh->b;
        b.Sync();
        const uint32_t cnt = species == 0 ? b.nF : species == 1 ? b.nB : b.nR;
        if (n != cnt || !out) throw Error(TSP_ERR_INVALID, "size mismatch");
        const uint32_t* src = species == 0 ? b.permF.p : species == 1 ? b.permB.p : b.permR.p;
        if (species == 1 && b.permBIdentity) {
            for (uint32_t i = 0; i < cnt; i++) out[i] = i;
        } else if (cnt) {
            CK(cudaMemcpy(out, src, cnt * 4ull, cudaMemcpyDeviceToHost));
        }
    });
}
int tsp_b200_read_cell_table(const tsp_backend* h, uint32_t species, uint64_t* uniq, uint32_t* start, uint32_t cap,
                             uint32_t* nCells) {
    TSP_NEED(h);
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, {
        Backend& b = *hh->b;
        b.Sync();
        const uint32_t cnt = species == 0 ? b.nF : species == 1 ? b.nB : b.nR;
        uint64_t nc = 0;
        if (cnt) CK(cudaMemcpy(&nc, b.nCellsDev.p + species, 8, cudaMemcpyDeviceToHost));
        if (nCells) *nCells = (uint32_t)nc;
        if (uniq && start) {
            if (cap < nc) throw Error(TSP_ERR_INVALID, "capacity");
            const uint64_t* u = species == 0 ? b.uniqF.p : species == 1 ? b.uniqB.p : b.uniqR.p;
            const uint32_t* s = species == 0 ? b.startF.p : species == 1 ? b.startB.p : b.startR.p;
            if (nc) {
                CK(cudaMemcpy(uniq, u, nc * 8ull, cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(start, s, (nc + 1) * 4ull, cudaMemcpyDeviceToHost));
            }
        }
    });
}
int tsp_b200_read_sell32_meta(const tsp_backend* h, uint32_t list, uint16_t* counts, uint16_t* pitch, uint8_t* fmt,
                              uint32_t* base, uint32_t* base2, uint64_t* offs, uint32_t nChunks, uint64_t* n16,
                              uint64_t* n32) {
    TSP_NEED(h);
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, {
        Backend& b = *hh->b;
        b.Sync();
        if (list > 2) throw Error(TSP_ERR_INVALID, "not a SELL32 list");
        Backend::Sell& m = b.sell[list];
        if (n16) *n16 = m.n16;
        if (n32) *n32 = m.n32;
        const uint32_t nc = (b.nF + 31) / 32;
        if (counts) {
            if (nChunks != nc) throw Error(TSP_ERR_INVALID, "chunk count mismatch");
            if (b.nF) CK(cudaMemcpy(counts, m.counts.p, b.nF * 2ull, cudaMemcpyDeviceToHost));
            if (nc) {
                CK(cudaMemcpy(pitch, m.pitch.p, nc * 2ull, cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(fmt, m.format.p, nc, cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(base, m.base.p, nc * 4ull, cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(base2, m.base2.p, nc * 4ull, cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(offs, m.offset.p, nc * 8ull, cudaMemcpyDeviceToHost));
            }
        }
    });
}
int tsp_b200_read_sell32_words(const tsp_backend* h, uint32_t list, uint16_t* w16, uint64_t n16, uint32_t* w32,
                               uint64_t n32) {
    TSP_NEED(h);
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, {
        Backend& b = *hh->b;
        b.Sync();
        if (list > 2) throw Error(TSP_ERR_INVALID, "not a SELL32 list");
        Backend::Sell& m = b.sell[list];
        if (n16 != m.n16 || n32 != m.n32) throw Error(TSP_ERR_INVALID, "size mismatch");
        if (n16) CK(cudaMemcpy(w16, m.l16.p, n16 * 2ull, cudaMemcpyDeviceToHost));
        if (n32) CK(cudaMemcpy(w32, m.l32.p, n32 * 4ull, cudaMemcpyDeviceToHost));
    });
}
int tsp_b200_read_rows(const tsp_backend* h, uint32_t list, uint64_t* offsets, uint32_t nSrc, uint32_t* indices,
                       uint64_t cap, uint64_t* total) {
    TSP_NEED(h);
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, {
        Backend& b = *hh->b;
        b.Sync();
        if (list > 5) throw Error(TSP_ERR_INVALID, "unknown list");
        if (list >= 3) {
            const int k = (int)list - 3;
            if (b.nR == 0 || !b.listsValid) {  // nothing built: every row is empty
                if (total) *total = 0;
                if (offsets) {
                    if (nSrc != b.nR) throw Error(TSP_ERR_INVALID, "size mismatch");
                    std::memset(offsets, 0, (b.nR + 1ull) * 8ull);
                }
                return TSP_OK;
            }
            if (total) *total = b.csrN[k];
            if (offsets) {
                if (nSrc != b.nR) throw Error(TSP_ERR_INVALID, "size mismatch");
                CK(cudaMemcpy(offsets, b.offR[k].p, (b.nR + 1ull) * 8ull, cudaMemcpyDeviceToHost));
            }
            if (indices && b.csrN[k]) {
                if (cap < b.csrN[k]) throw Error(TSP_ERR_INVALID, "capacity");
                CK(cudaMemcpy(indices, b.listR[k].p, b.csrN[k] * 4ull, cudaMemcpyDeviceToHost));
            }
            return TSP_OK;
        }
        std::vector<uint16_t> cnt(b.nF, 0);
        if (b.nF && b.listsValid) CK(cudaMemcpy(cnt.data(), b.sell[list].counts.p, b.nF * 2ull, cudaMemcpyDeviceToHost));
        std::vector<uint64_t> off(b.nF + 1ull, 0);
        for (uint32_t i = 0; i < b.nF; i++) off[i + 1] = off[i] + cnt[i];
        if (total) *total = off[b.nF];
        if (offsets) {
            if (nSrc != b.nF) throw Error(TSP_ERR_INVALID, "size mismatch");
            std::memcpy(offsets, off.data(), off.size() * 8);
        }
        if (indices && off[b.nF] && b.listsValid) {
            if (cap < off[b.nF]) throw Error(TSP_ERR_INVALID, "capacity");
            tsp::DBuf<uint64_t> dOff;
            tsp::DBuf<uint32_t> dOut;
            dOff.ensure(b.nF + 1ull);
            dOut.ensure(off[b.nF]);
            CK(cudaMemcpy(dOff.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice));
            tsp::LaunchDecodeSellRows(b.Meta((int)list), b.nF, dOff.p, dOut.p, b.s);
            b.Sync();
            CK(cudaMemcpy(indices, dOut.p, off[b.nF] * 4ull, cudaMemcpyDeviceToHost));
        }
    });
}
int tsp_b200_run_stage(tsp_backend* h, const tsp_params* p, uint32_t stage, double* errSums) {
    TSP_NEED(h);
    if (!p) return TSP_ERR_INVALID;
    TSP_GUARD(h, h->b->RunStage(*p, stage, errSums));
}
int tsp_b200_read_field(const tsp_backend* h, uint32_t field, void* out, uint32_t n) {
    TSP_NEED(h);
    if (!out && n) return TSP_ERR_INVALID;
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, hh->b->ReadField(field, out, n));
}
int tsp_b200_write_field(tsp_backend* h, uint32_t field, const void* in, uint32_t n) {
    TSP_NEED(h);
    if (!in && n) return TSP_ERR_INVALID;
    TSP_GUARD(h, h->b->WriteField(field, in, n));
}

int tsp_b200_time_stage(tsp_backend* h, const tsp_params* p, uint32_t stage, uint32_t reps, float* ms) {
    TSP_NEED(h);
    if (!p || !ms) return TSP_ERR_INVALID;
    TSP_GUARD(h, *ms = h->b->TimeStage(*p, stage, reps));
}
int tsp_b200_get_stream(const tsp_backend* h, void** stream) {
    TSP_NEED(h);
    if (!stream) return TSP_ERR_INVALID;
    *stream = (void*)h->b->s;
    return TSP_OK;
}
int tsp_b200_fill_statistics(const tsp_backend* h, const tsp_params* p, double* record, uint32_t n) {
    TSP_NEED(h);
    if (!p || (n && !record)) return TSP_ERR_INVALID;
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, hh->b->Statistics(*p, record, n));
}
int tsp_b200_get_contact_report(const tsp_backend* h, tsp_contact_report* out) {
    TSP_NEED(h);
    if (!out) return TSP_ERR_INVALID;
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, hh->b->ContactReport(*out));
}
int tsp_b200_pack_export_snapshot(tsp_backend* h, const tsp_params* params, int include_b,
                                  uint64_t mesh_id_begin_b, tsp_export_snapshot* snap) {
    TSP_NEED(h);
    if (!params || !snap) return TSP_ERR_INVALID;
    TSP_GUARD(h, h->b->PackExport(*params, include_b != 0, mesh_id_begin_b, *snap));
}
int tsp_b200_sample_surface(int device, const float* vertices, uint32_t nV, const uint32_t* triangles, uint32_t nT,
                            const tsp_surface_sampling_params* params, float* out, uint64_t cap, uint64_t* nOut,
                            tsp_surface_sampling_stats* stats) {
    if (!params || !nOut) { g_lastError = "NULL argument"; return TSP_ERR_INVALID; }
    try {
        tsp_surface_sampling_stats st{};
        const std::vector<float> smp = tsp::SampleSurfaceGpu(device, vertices, nV, triangles, nT, *params, st);
        if (stats) *stats = st;
        *nOut = smp.size() / 3;
        if (*nOut > cap || !out) {
            g_lastError = "surface sample buffer too small";
            return TSP_ERR_OVERFLOW;
        }
        std::memcpy(out, smp.data(), smp.size() * sizeof(float));
        return TSP_OK;
    } catch (const Error& e) {
        g_lastError = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_lastError = e.what();
        return TSP_ERR_INVALID;
    }
}
int tsp_b200_get_phase_times(const tsp_backend* h, float* ms, uint32_t cap, uint32_t* n) {
    TSP_NEED(h);
    if (!n || (cap && !ms)) return TSP_ERR_INVALID;
    tsp_backend* hh = const_cast<tsp_backend*>(h);
    TSP_GUARD(hh, *n = hh->b->PhaseTimes(ms, cap));
}
int tsp_b200_get_launch_count(const tsp_backend* h, uint64_t* count) {
    TSP_NEED(h);
    if (!count) return TSP_ERR_INVALID;
    *count = h->b->launches;
    return TSP_OK;
}
int tsp_b200_get_step_time_total(const tsp_backend* h, double* ms, uint64_t* steps) {
    TSP_NEED(h);
    if (!ms || !steps) return TSP_ERR_INVALID;
    *ms = h->b->stepMsTotal;
    *steps = h->b->stepsTimed;
    return TSP_OK;
}
int tsp_b200_get_step_history(const tsp_backend* h, tsp_step_record* out, uint32_t cap, uint32_t* n) {
    TSP_NEED(h);
    if (!n) return TSP_ERR_INVALID;
    *n = out ? h->b->History(out, cap) : (uint32_t)std::min<uint64_t>(h->b->histCount, Backend::HIST_CAP);
    return TSP_OK;
}

}  // extern "C"
