// tsp_b200_backend.hpp -- C++ host adapter of the B200 IISPH backend over the C ABI.
//
// `SimBackendB200` has the shape of the reference's `Sim::I_SimBackend`
// (source/simulation/core/backend_sim.h:194-261): the same method names, the same argument
// meaning (a parameter struct by const reference per call, the universal SoA state for
// pull/push) and the same error behaviour (failures throw std::runtime_error, like
// GPU::Check in source/simulation/GPU/gpu_utils.h:24-45). It depends only on tsp_b200.h;
// deriving a class from both `Sim::I_SimBackend` and this one, with each interface method
// forwarding to the method of the same name, makes it a backend of the reference tree.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>

#include "tsp_b200.h"

namespace tsp {

class SimBackendB200 {
public:
    explicit SimBackendB200(const tsp_params& params, int device = -1) {
        Check(tsp_b200_create(&params, device, &h_), nullptr);
    }
    ~SimBackendB200() { tsp_b200_destroy(h_); }
    SimBackendB200(const SimBackendB200&) = delete;
    SimBackendB200& operator=(const SimBackendB200&) = delete;
    SimBackendB200(SimBackendB200&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}

    const char* Name() const { return tsp_b200_name(h_); }

    void SetSimDomainBounds(const float min[3], const float max[3]) { Check(tsp_b200_set_domain(h_, min, max)); }

    void PullFromUniversalSimState(const tsp_state_view& src, const tsp_params& params) {
        Check(tsp_b200_pull_state(h_, &src, &params));
    }
    void PushToUniversalSimState(tsp_state_view& dst) { Check(tsp_b200_push_state(h_, &dst)); }

    void ExecuteNeighborSearch(const tsp_params& params, bool /*bench*/ = false) {
        Check(tsp_b200_neighbor_search(h_, &params));
    }
    void ExecuteFullSimStep(const tsp_params& params, uint32_t N_steps = 1) {
        Check(tsp_b200_step(h_, &params, N_steps));
    }

    uint32_t GetNumFluidParticles() const { return Count(0); }
    uint32_t GetNumBoundaryParticles() const { return Count(1); }
    uint32_t GetNumRigidParticles() const { return Count(2); }

    tsp_step_stats Stats() const {
        tsp_step_stats s{};
        Check(tsp_b200_get_stats(h_, &s));
        return s;
    }
    // I_SimBackend::FillStatisticsRecord (backend_sim.h:243): record[k] is Stats::StatMetric k
    void FillStatisticsRecord(const tsp_params& params, double (&record)[TSP_STAT_COUNT]) const {
        Check(tsp_b200_fill_statistics(h_, &params, record, TSP_STAT_COUNT));
    }
    // SimBackend_CPU::GetRigidContactReport (source/simulation/CPU/backend/cpu_backend.h:132)
    tsp_contact_report GetRigidContactReport() const {
        tsp_contact_report r{};
        Check(tsp_b200_get_contact_report(h_, &r));
        return r;
    }
    // I_SimBackend::PackExportSnapshot (backend_sim.h:215); the snapshot's non-NULL arrays must
    // hold the backend's full population counts, its N_* fields receive the exported counts
    void PackExportSnapshot(tsp_export_snapshot& snap, const tsp_params& params, bool includeB,
                            uint64_t meshIdBeginB = TSP_NO_MESH_ID) {
        Check(tsp_b200_pack_export_snapshot(h_, &params, includeB ? 1 : 0, meshIdBeginB, &snap));
    }
    tsp_backend* Handle() const { return h_; }

private:
    tsp_backend* h_ = nullptr;

    uint32_t Count(int which) const {
        uint32_t n[4] = {0, 0, 0, 0};
        Check(tsp_b200_get_counts(h_, &n[0], &n[1], &n[2], &n[3]));
        return n[which];
    }
    void Check(int rc) const { Check(rc, h_); }
    static void Check(int rc, const tsp_backend* h) {
        if (rc != TSP_OK) throw std::runtime_error(std::string("tsp_b200: ") + tsp_b200_last_error(h));
    }
};

}  // namespace tsp
