"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/ and __graft_entry__.smoke() import this module, to check results, and bench.py's
CPU-baseline leg, which times it beside the GPU. It exposes the same method names as the product backend
(turbospharticles_b200.backend.SimBackendB200) so parity tests drive both identically.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from turbospharticles_b200.abi import (TspParams, TspStateView, TspStepStats, TspContactReport, TspExportSnapshot,
                                       FIELD_COMPONENTS, FIELD_BODY_FT)
from turbospharticles_b200.state import ExportSnapshot, UniversalSimState

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(ORACLE_DIR, "_build", "libtsp_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-C", ORACLE_DIR], check=True, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        sig = {
            "orc_create": (vp, [C.POINTER(TspParams), C.c_int]),
            "orc_destroy": (None, [vp]),
            "orc_last_error": (C.c_char_p, [vp]),
            "orc_set_threads": (C.c_int, [C.c_int]),
            "orc_set_domain": (C.c_int, [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
            "orc_pull_state": (C.c_int, [vp, C.POINTER(TspStateView), C.POINTER(TspParams)]),
            "orc_push_state": (C.c_int, [vp, C.POINTER(TspStateView)]),
            "orc_neighbor_search": (C.c_int, [vp, C.POINTER(TspParams)]),
            "orc_step": (C.c_int, [vp, C.POINTER(TspParams), C.c_uint32]),
            "orc_get_stats": (C.c_int, [vp, C.POINTER(TspStepStats)]),
            "orc_get_contact_report": (C.c_int, [vp, C.POINTER(TspContactReport)]),
            "orc_fill_statistics": (C.c_int, [vp, C.POINTER(TspParams), C.POINTER(C.c_double)]),
            "orc_pack_export_snapshot": (C.c_int, [vp, C.POINTER(TspParams), C.c_int, C.c_uint64,
                                                   C.POINTER(TspExportSnapshot)]),
            "orc_read_cell_ids": (C.c_int, [vp, C.c_uint32, vp, C.c_uint32]),
            "orc_read_permutation": (C.c_int, [vp, C.c_uint32, vp, C.c_uint32]),
            "orc_read_cell_table": (C.c_int, [vp, C.c_uint32, vp, vp, C.c_uint32, C.POINTER(C.c_uint32)]),
            "orc_read_rows": (C.c_int, [vp, C.c_uint32, vp, C.c_uint32, vp, C.c_uint64, C.POINTER(C.c_uint64)]),
            "orc_encode_sell32": (C.c_int, [vp, C.c_uint32, vp, vp, vp, vp, vp, vp, C.c_uint32, vp,
                                            C.c_uint64, vp, C.c_uint64, C.POINTER(C.c_uint64),
                                            C.POINTER(C.c_uint64)]),
            "orc_run_stage": (C.c_int, [vp, C.POINTER(TspParams), C.c_uint32, C.POINTER(C.c_double)]),
            "orc_read_field": (C.c_int, [vp, C.c_uint32, vp, C.c_uint32]),
            "orc_write_field": (C.c_int, [vp, C.c_uint32, vp, C.c_uint32]),
            "orc_kernel_eval": (None, [C.c_float] * 6 + [C.POINTER(C.c_float)]),
            "orc_surface_last_error": (C.c_char_p, []),
            "orc_sample_surface": (C.c_int, [C.POINTER(C.c_float), C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32,
                                             vp, C.POINTER(C.c_float), C.c_uint64, C.POINTER(C.c_uint64), vp]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def sample_surface(mesh, sp):
    """Sequential CPU restatement of SurfaceSampler::Sample (surface_oracle.cpp): the oracle of
    turbospharticles_b200.mesh.sample_surface."""
    from turbospharticles_b200.mesh import _sample_with
    L = lib()
    return _sample_with(lambda v, nv, t, nt, p, o, cap, n, st: L.orc_sample_surface(
        v, nv, t, nt, C.cast(p, C.c_void_p), o, cap, n, C.cast(st, C.c_void_p)), mesh, sp,
        lambda: L.orc_surface_last_error().decode())


class OracleBackend:
    """CPU restatement of the reference step; `fp64=True` gives the FP64 run."""

    def __init__(self, params, fp64=False, threads=0):
        self.L = lib()
        if threads:
            self.L.orc_set_threads(threads)
        self.params = params
        self._cp = params.to_c()
        self.h = self.L.orc_create(C.byref(self._cp), 1 if fp64 else 0)
        self.counts = (0, 0, 0, 0)

    def __del__(self):
        try:
            self.L.orc_destroy(self.h)
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError(self.L.orc_last_error(self.h).decode())

    def _cparams(self, params):
        if params is not None:
            self.params = params
        self._cp = self.params.to_c()
        return C.byref(self._cp)

    def set_sim_domain_bounds(self, mn, mx):
        a = np.asarray(mn, np.float32); b = np.asarray(mx, np.float32)
        self._chk(self.L.orc_set_domain(self.h, a.ctypes.data_as(C.POINTER(C.c_float)),
                                        b.ctypes.data_as(C.POINTER(C.c_float))))

    def pull(self, state: UniversalSimState, params=None):
        v = state.view()
        self._chk(self.L.orc_pull_state(self.h, C.byref(v), self._cparams(params)))
        self.counts = (state.N_F, state.N_B, state.N_R, state.N_RB)

    def push(self) -> UniversalSimState:
        st = UniversalSimState(*self.counts)
        v = st.view()
        self._chk(self.L.orc_push_state(self.h, C.byref(v)))
        st.step, st.time = int(v.step), float(v.time)
        return st

    def neighbor_search(self, params=None):
        self._chk(self.L.orc_neighbor_search(self.h, self._cparams(params)))

    def step(self, params=None, n_steps=1):
        self._chk(self.L.orc_step(self.h, self._cparams(params), n_steps))

    def stats(self) -> TspStepStats:
        s = TspStepStats()
        self._chk(self.L.orc_get_stats(self.h, C.byref(s)))
        return s

    def statistics(self, params=None) -> dict:
        """FillStatisticsRecord of the last step (names of Stats::StatMetric)."""
        from turbospharticles_b200.abi import STAT_NAMES
        buf = (C.c_double * len(STAT_NAMES))()
        cp = (params or self.params).to_c()
        self._chk(self.L.orc_fill_statistics(self.h, C.byref(cp), buf))
        return dict(zip(STAT_NAMES, list(buf)))

    def pack_export_snapshot(self, params=None, include_b=True, mesh_id_begin_b=None) -> ExportSnapshot:
        """PackExportSnapshot (cpu_backend.cpp:829-975)."""
        cp = (params or self.params).to_c()
        return ExportSnapshot.pack(lambda *a: self._chk(self.L.orc_pack_export_snapshot(self.h, *a)),
                                   (self.counts[0], self.counts[1], self.counts[2]), cp, include_b,
                                   mesh_id_begin_b)

    def contact_report(self) -> TspContactReport:
        r = TspContactReport()
        self._chk(self.L.orc_get_contact_report(self.h, C.byref(r)))
        return r

    def cell_ids(self, species):
        n = self.counts[species]
        out = np.zeros(n, np.uint64)
        self._chk(self.L.orc_read_cell_ids(self.h, species, _p(out), n))
        return out

    def permutation(self, species):
        n = self.counts[species]
        out = np.zeros(n, np.uint32)
        self._chk(self.L.orc_read_permutation(self.h, species, _p(out), n))
        return out

    def cell_table(self, species):
        nc = C.c_uint32()
        self._chk(self.L.orc_read_cell_table(self.h, species, None, None, 0, C.byref(nc)))
        u = np.zeros(nc.value, np.uint64)
        s = np.zeros(nc.value + 1, np.uint32)
        self._chk(self.L.orc_read_cell_table(self.h, species, _p(u), _p(s), nc.value, C.byref(nc)))
        return u, (s if nc.value else np.zeros(0, np.uint32))

    def rows(self, lst):
        nsrc = self.counts[0] if lst < 3 else self.counts[2]
        tot = C.c_uint64()
        self._chk(self.L.orc_read_rows(self.h, lst, None, nsrc, None, 0, C.byref(tot)))
        off = np.zeros(nsrc + 1, np.uint64)
        idx = np.zeros(tot.value, np.uint32)
        self._chk(self.L.orc_read_rows(self.h, lst, _p(off), nsrc, _p(idx), tot.value, C.byref(tot)))
        return off, idx

    def sell32(self, lst):
        nF = self.counts[0]
        nch = (nF + 31) // 32
        n16, n32 = C.c_uint64(), C.c_uint64()
        self._chk(self.L.orc_encode_sell32(self.h, lst, None, None, None, None, None, None, 0,
                                           None, 0, None, 0, C.byref(n16), C.byref(n32)))
        m = dict(counts=np.zeros(nF, np.uint16), pitch=np.zeros(nch, np.uint16),
                 format=np.zeros(nch, np.uint8), base=np.zeros(nch, np.uint32),
                 base2=np.zeros(nch, np.uint32), offset=np.zeros(nch, np.uint64),
                 w16=np.zeros(n16.value, np.uint16), w32=np.zeros(n32.value, np.uint32))
        self._chk(self.L.orc_encode_sell32(
            self.h, lst, _p(m["counts"]), _p(m["pitch"]), _p(m["format"]), _p(m["base"]),
            _p(m["base2"]), _p(m["offset"]), nch, _p(m["w16"]), n16.value, _p(m["w32"]), n32.value,
            C.byref(n16), C.byref(n32)))
        return m

    def run_stage(self, stage, params=None):
        err = (C.c_double * 3)()
        self._chk(self.L.orc_run_stage(self.h, self._cparams(params), stage, err))
        return tuple(err)

    def read_field(self, field):
        n = self.counts[3] if field == FIELD_BODY_FT else (
            self.counts[1] if field in (8, 9) else self.counts[2] if field in (10, 11, 12) else self.counts[0])
        k = FIELD_COMPONENTS[field]
        out = np.zeros(n * k, np.float64)
        self._chk(self.L.orc_read_field(self.h, field, _p(out), n))
        return out.reshape(n, k) if k > 1 else out

    def write_field(self, field, values):
        v = np.ascontiguousarray(values, np.float64).ravel()
        k = FIELD_COMPONENTS[field]
        self._chk(self.L.orc_write_field(self.h, field, _p(v), v.size // k))


def kernel_eval(dx, dy, dz, size_inv, rad_squ, alpha):
    out = (C.c_float * 5)()
    lib().orc_kernel_eval(dx, dy, dz, size_inv, rad_squ, alpha, out)
    return tuple(out)
