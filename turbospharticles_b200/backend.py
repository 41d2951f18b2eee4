"""SimBackendB200: Python mirror of the reference's `Sim::I_SimBackend`
(source/simulation/core/backend_sim.h:194-261) over the C ABI of include/tsp_b200.h.

Method names follow the reference interface (Name, SetSimDomainBounds,
PullFromUniversalSimState, PushToUniversalSimState, ExecuteNeighborSearch,
ExecuteFullSimStep, GetNum*Particles); failures raise `TspError` like the reference's
std::runtime_error. The snake_case methods below them are the test-access surface
(neighbor structures, single solver stages, field reads).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .abi import TspError, TspStepStats, FIELD_COMPONENTS, FIELD_BODY_FT
from .params import SimParams
from .state import ExportSnapshot, UniversalSimState


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class SimBackendB200:
    def __init__(self, params: SimParams | None = None, device: int = -1):
        self.L = abi.load_library()
        self.params = params or SimParams()
        self._cp = self.params.to_c()
        h = C.c_void_p()
        rc = self.L.tsp_b200_create(C.byref(self._cp), device, C.byref(h))
        if rc != 0:
            raise TspError(rc, self.L.tsp_b200_last_error(None).decode())
        self.h = h
        self.counts = (0, 0, 0, 0)

    def close(self):
        if getattr(self, "h", None):
            self.L.tsp_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise TspError(rc, self.L.tsp_b200_last_error(self.h).decode())

    def _cparams(self, params):
        if params is not None:
            self.params = params
        self._cp = self.params.to_c()
        return C.byref(self._cp)

    # ------------------------------------------------------------ I_SimBackend surface
    def Name(self) -> str:
        return self.L.tsp_b200_name(self.h).decode()

    def SetSimDomainBounds(self, mn, mx):
        a = np.ascontiguousarray(mn, np.float32)
        b = np.ascontiguousarray(mx, np.float32)
        self._chk(self.L.tsp_b200_set_domain(self.h, a.ctypes.data_as(C.POINTER(C.c_float)),
                                             b.ctypes.data_as(C.POINTER(C.c_float))))

    def PullFromUniversalSimState(self, state: UniversalSimState, params: SimParams | None = None):
        v = state.view()
        self._chk(self.L.tsp_b200_pull_state(self.h, C.byref(v), self._cparams(params)))
        self.counts = (state.N_F, state.N_B, state.N_R, state.N_RB)

    def PushToUniversalSimState(self, dst: UniversalSimState | None = None) -> UniversalSimState:
        st = dst if dst is not None else UniversalSimState(*self.counts)
        v = st.view()
        self._chk(self.L.tsp_b200_push_state(self.h, C.byref(v)))
        st.step, st.time = int(v.step), float(v.time)
        return st

    def ExecuteNeighborSearch(self, params: SimParams | None = None, bench: bool = False):
        self._chk(self.L.tsp_b200_neighbor_search(self.h, self._cparams(params)))

    def ExecuteFullSimStep(self, params: SimParams | None = None, N_steps: int = 1):
        self._chk(self.L.tsp_b200_step(self.h, self._cparams(params), N_steps))

    def GetNumFluidParticles(self):
        return self.counts[0]

    def GetNumBoundaryParticles(self):
        return self.counts[1]

    def GetNumRigidParticles(self):
        return self.counts[2]

    # ------------------------------------------------------------ shared test surface
    set_sim_domain_bounds = SetSimDomainBounds
    pull = PullFromUniversalSimState
    push = PushToUniversalSimState
    neighbor_search = ExecuteNeighborSearch

    def step(self, params=None, n_steps=1):
        self.ExecuteFullSimStep(params, n_steps)

    def stats(self) -> TspStepStats:
        s = TspStepStats()
        self._chk(self.L.tsp_b200_get_stats(self.h, C.byref(s)))
        return s

    def cell_ids(self, species):
        n = self.counts[species]
        out = np.zeros(n, np.uint64)
        self._chk(self.L.tsp_b200_read_cell_ids(self.h, species, out.ctypes.data_as(C.POINTER(C.c_uint64)), n))
        return out

    def permutation(self, species):
        n = self.counts[species]
        out = np.zeros(n, np.uint32)
        self._chk(self.L.tsp_b200_read_permutation(self.h, species, out.ctypes.data_as(C.POINTER(C.c_uint32)), n))
        return out

    def cell_table(self, species):
        nc = C.c_uint32()
        self._chk(self.L.tsp_b200_read_cell_table(self.h, species, None, None, 0, C.byref(nc)))
        u = np.zeros(nc.value, np.uint64)
        s = np.zeros(nc.value + 1, np.uint32)
        self._chk(self.L.tsp_b200_read_cell_table(self.h, species, u.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                  s.ctypes.data_as(C.POINTER(C.c_uint32)), nc.value, C.byref(nc)))
        return u, (s if nc.value else np.zeros(0, np.uint32))

    def rows(self, lst):
        nsrc = self.counts[0] if lst < 3 else self.counts[2]
        tot = C.c_uint64()
        self._chk(self.L.tsp_b200_read_rows(self.h, lst, None, nsrc, None, 0, C.byref(tot)))
        off = np.zeros(nsrc + 1, np.uint64)
        idx = np.zeros(max(tot.value, 1), np.uint32)
        self._chk(self.L.tsp_b200_read_rows(self.h, lst, off.ctypes.data_as(C.POINTER(C.c_uint64)), nsrc,
                                            idx.ctypes.data_as(C.POINTER(C.c_uint32)), tot.value, C.byref(tot)))
        return off, idx[:tot.value]

    def sell32(self, lst):
        nF = self.counts[0]
        nch = (nF + 31) // 32
        n16, n32 = C.c_uint64(), C.c_uint64()
        m = dict(counts=np.zeros(nF, np.uint16), pitch=np.zeros(nch, np.uint16),
                 format=np.zeros(nch, np.uint8), base=np.zeros(nch, np.uint32),
                 base2=np.zeros(nch, np.uint32), offset=np.zeros(nch, np.uint64))
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
        self._chk(self.L.tsp_b200_read_sell32_meta(
            self.h, lst, P(m["counts"], C.c_uint16), P(m["pitch"], C.c_uint16), P(m["format"], C.c_uint8),
            P(m["base"], C.c_uint32), P(m["base2"], C.c_uint32), P(m["offset"], C.c_uint64), nch,
            C.byref(n16), C.byref(n32)))
        m["w16"] = np.zeros(n16.value, np.uint16)
        m["w32"] = np.zeros(n32.value, np.uint32)
        self._chk(self.L.tsp_b200_read_sell32_words(self.h, lst, P(m["w16"], C.c_uint16), n16.value,
                                                    P(m["w32"], C.c_uint32), n32.value))
        return m

    def run_stage(self, stage, params=None):
        err = (C.c_double * 3)()
        self._chk(self.L.tsp_b200_run_stage(self.h, self._cparams(params), stage, err))
        return tuple(err)

    def _field_n(self, field):
        if field == FIELD_BODY_FT:
            return self.counts[3]
        if field in (abi.FIELD_VOL_B, abi.FIELD_PSI_B):
            return self.counts[1]
        if field in (abi.FIELD_VOL_R, abi.FIELD_PSI_R, abi.FIELD_FORCE_R):
            return self.counts[2]
        return self.counts[0]

    def read_field(self, field):
        n = self._field_n(field)
        k = FIELD_COMPONENTS[field]
        out = np.zeros(n * k, np.float64 if field == FIELD_BODY_FT else np.float32)
        self._chk(self.L.tsp_b200_read_field(self.h, field, _p(out), n))
        return out.reshape(n, k) if k > 1 else out

    def time_stage(self, stage, reps=20, params=None) -> float:
        """Average device milliseconds per launch of one solver stage (CUDA events)."""
        ms = C.c_float()
        self._chk(self.L.tsp_b200_time_stage(self.h, self._cparams(params), stage, reps, C.byref(ms)))
        return ms.value

    def FillStatisticsRecord(self, params: SimParams | None = None) -> dict:
        """Statistics of the last step (I_SimBackend::FillStatisticsRecord, backend_sim.h:243),
        keyed by the reference's Stats::StatMetric names."""
        buf = (C.c_double * len(abi.STAT_NAMES))()
        self._chk(self.L.tsp_b200_fill_statistics(self.h, self._cparams(params), buf, len(abi.STAT_NAMES)))
        return dict(zip(abi.STAT_NAMES, list(buf)))

    statistics = FillStatisticsRecord

    def PackExportSnapshot(self, params: SimParams | None = None, include_b: bool = True,
                           mesh_id_begin_b: int | None = None) -> ExportSnapshot:
        """I_SimBackend::PackExportSnapshot (backend_sim.h:215): surface fluid particles,
        boundary (when `include_b`) and rigid particles of the current state; boundary particles
        with ID >= `mesh_id_begin_b` are flagged as mesh particles (None: no mesh)."""
        cp = self.params.to_c() if params is None else params.to_c()
        return ExportSnapshot.pack(lambda *a: self._chk(self.L.tsp_b200_pack_export_snapshot(self.h, *a)),
                                   self.counts[:3], cp, include_b, mesh_id_begin_b)

    pack_export_snapshot = PackExportSnapshot

    def contact_report(self):
        """Rigid contact solve of the last step (GetRigidContactReport, cpu_backend.h:132)."""
        r = abi.TspContactReport()
        self._chk(self.L.tsp_b200_get_contact_report(self.h, C.byref(r)))
        return r

    def phase_times(self) -> dict:
        """Device milliseconds of the phases of the last step (empty before the first step)."""
        buf = (C.c_float * len(abi.PHASE_NAMES))()
        n = C.c_uint32()
        self._chk(self.L.tsp_b200_get_phase_times(self.h, buf, len(abi.PHASE_NAMES), C.byref(n)))
        return {abi.PHASE_NAMES[k]: float(buf[k]) for k in range(n.value)}

    def launch_count(self) -> int:
        n = C.c_uint64()
        self._chk(self.L.tsp_b200_get_launch_count(self.h, C.byref(n)))
        return n.value

    def step_time_total(self) -> tuple:
        """(device milliseconds, steps) of all steps since creation."""
        ms, n = C.c_double(), C.c_uint64()
        self._chk(self.L.tsp_b200_get_step_time_total(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def step_history(self, last: int | None = None) -> list:
        """Records of the most recent `last` steps (all kept ones if None), oldest first: dicts of
        step, ms (device milliseconds), solverIters, avgRelDensityErrPos."""
        n = C.c_uint32()
        self._chk(self.L.tsp_b200_get_step_history(self.h, None, 0, C.byref(n)))
        k = n.value if last is None else min(int(last), n.value)
        buf = (abi.TspStepRecord * max(k, 1))()
        self._chk(self.L.tsp_b200_get_step_history(self.h, buf, k, C.byref(n)))
        return [{"step": r.step, "ms": r.ms, "solverIters": r.solverIters,
                 "avgRelDensityErrPos": r.avgRelDensityErrPos} for r in buf[:n.value]]

    def stream_handle(self) -> int:
        s = C.c_void_p()
        self._chk(self.L.tsp_b200_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def write_field(self, field, values):
        v = np.ascontiguousarray(values, np.float32).ravel()
        k = FIELD_COMPONENTS[field]
        self._chk(self.L.tsp_b200_write_field(self.h, field, _p(v), v.size // k))


class ServedBatchB200:
    """Served batch over the C ABI (`tsp_b200_batch_*`): independent fluid + boundary scenes of
    one physics setup, resident on one GPU and advanced together per substep. `admit` returns a
    slot (raises TspError with TSP_ERR_OVERFLOW when the scene does not fit the memory budget);
    admissions and retirements take effect at the next `substep`."""

    def __init__(self, params: SimParams, budget_bytes: int, device: int = -1):
        self.L = abi.load_library()
        self.params = params
        self._cp = params.to_c()
        h = C.c_void_p()
        rc = self.L.tsp_b200_batch_create(C.byref(self._cp), device, int(budget_bytes), C.byref(h))
        if rc != 0:
            raise TspError(rc, self.L.tsp_b200_batch_last_error(None).decode())
        self.h = h
        self.counts = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.tsp_b200_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise TspError(rc, self.L.tsp_b200_batch_last_error(self.h).decode())

    def admit(self, state: UniversalSimState, dmin, dmax) -> int:
        v = state.view()
        a = np.ascontiguousarray(dmin, np.float32)
        b = np.ascontiguousarray(dmax, np.float32)
        slot = C.c_uint32()
        self._chk(self.L.tsp_b200_admit(self.h, C.byref(v), a.ctypes.data_as(C.POINTER(C.c_float)),
                                        b.ctypes.data_as(C.POINTER(C.c_float)), C.byref(slot)))
        self.counts[slot.value] = (state.N_F, state.N_B)
        return slot.value

    def retire(self, slot: int, push: bool = False):
        st = None
        if push:
            st = UniversalSimState(self.counts[slot][0], self.counts[slot][1], 0, 0)
            v = st.view()
            self._chk(self.L.tsp_b200_retire(self.h, slot, C.byref(v)))
            st.step, st.time = int(v.step), float(v.time)
        else:
            self._chk(self.L.tsp_b200_retire(self.h, slot, None))
        self.counts.pop(slot, None)
        return st

    def substep(self, n: int = 1, params: SimParams | None = None):
        if params is not None:
            self.params = params
            self._cp = params.to_c()
        self._chk(self.L.tsp_b200_substep_all(self.h, C.byref(self._cp), n))

    def push(self, slot: int) -> UniversalSimState:
        st = UniversalSimState(self.counts[slot][0], self.counts[slot][1], 0, 0)
        v = st.view()
        self._chk(self.L.tsp_b200_batch_push(self.h, slot, C.byref(v)))
        st.step, st.time = int(v.step), float(v.time)
        return st

    def stats(self, slot: int) -> TspStepStats:
        s = TspStepStats()
        self._chk(self.L.tsp_b200_batch_stats(self.h, slot, C.byref(s)))
        return s

    def info(self) -> dict:
        sc, nf, used, budget, launches = C.c_uint32(), C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        ms = C.c_float()
        self._chk(self.L.tsp_b200_batch_info(self.h, C.byref(sc), C.byref(nf), C.byref(used), C.byref(budget),
                                             C.byref(ms), C.byref(launches)))
        return {"scenes": sc.value, "fluid_particles": nf.value, "bytes_used": used.value,
                "bytes_budget": budget.value, "last_substep_ms": ms.value, "launches": launches.value}


def batch_scene_bytes(n_fluid: int, n_boundary: int, grid_cells: int) -> int:
    """Device bytes a served scene is charged at admission (host arithmetic)."""
    return int(abi.load_library().tsp_b200_batch_scene_bytes(n_fluid, n_boundary, grid_cells))
