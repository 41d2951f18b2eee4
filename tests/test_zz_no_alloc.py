"""tsp_b200_build_cell_table_noalloc: the cell-table build whose scan scratch is a fixed
array inside the library (no device allocation by the call), checked against the cell
table the backend's own neighbor search built, on two consecutive calls.

Device buffers for inputs and outputs come from torch (the caller owns them); the entry
point itself is called through the C ABI with raw device pointers and a stream handle.
"""
import ctypes as C

import numpy as np
import pytest

from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import SimBackendB200

pytestmark = pytest.mark.gpu


def _noalloc_table(lib, torch, cid_sorted, stream):
    n = int(cid_sorted.size)
    dev = torch.device("cuda", 0)
    d_cid = torch.from_numpy(cid_sorted.view(np.int64).copy()).to(dev)
    d_uniq = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    d_start = torch.empty(n + 1, dtype=torch.int32, device=dev)
    d_nc = torch.empty(1, dtype=torch.int64, device=dev)
    torch.cuda.synchronize(dev)
    rc = lib.tsp_b200_build_cell_table_noalloc(d_cid.data_ptr(), n, d_uniq.data_ptr(), d_start.data_ptr(),
                                               d_nc.data_ptr(), stream.cuda_stream)
    assert rc == 0, lib.tsp_b200_noalloc_last_error()
    stream.synchronize()
    nc = int(d_nc.cpu()[0])
    uniq = d_uniq[:nc].cpu().numpy().view(np.uint64)
    start = d_start[:nc + 1].cpu().numpy().view(np.uint32) if nc else np.zeros(0, np.uint32)
    return uniq, start


@pytest.mark.parametrize("which", ["uniform_fluid", "dam_boundary"])
def test_noalloc_cell_table_matches_neighbor_search(which):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    if which == "uniform_fluid":
        st, dmin, dmax, p = S.neighbor_search_scene(200_000, "uniform", seed=3)
        species = abi.SPECIES_F
    else:
        st, dmin, dmax, p = S.dam_32k()
        species = abi.SPECIES_B
    g = SimBackendB200(p)
    g.set_sim_domain_bounds(dmin, dmax)
    g.pull(st, p)
    g.neighbor_search(p)
    cid = g.cell_ids(species)
    want_u, want_s = g.cell_table(species)
    assert want_u.size > 1000

    lib = abi.load_library()
    torch.cuda.set_device(0)
    assert lib.tsp_b200_noalloc_setup() == 0, lib.tsp_b200_noalloc_last_error()
    stream = torch.cuda.Stream(device=0)
    for _ in range(2):  # two consecutive calls on the same scratch
        u, s = _noalloc_table(lib, torch, cid, stream)
        assert np.array_equal(u, want_u)
        assert np.array_equal(s, want_s)


def test_noalloc_calls_leave_free_device_memory_unchanged():
    """The property the entry point exists for: after setup, calls take no device memory.
    Buffers are allocated first; free memory (cudaMemGetInfo) is read before and after a
    series of calls."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    st, dmin, dmax, p = S.neighbor_search_scene(100_000, "uniform", seed=5)
    g = SimBackendB200(p)
    g.set_sim_domain_bounds(dmin, dmax)
    g.pull(st, p)
    g.neighbor_search(p)
    cid = g.cell_ids(abi.SPECIES_F)
    want_u, _ = g.cell_table(abi.SPECIES_F)
    lib = abi.load_library()
    torch.cuda.set_device(0)
    assert lib.tsp_b200_noalloc_setup() == 0, lib.tsp_b200_noalloc_last_error()
    n = int(cid.size)
    dev = torch.device("cuda", 0)
    d_cid = torch.from_numpy(cid.view(np.int64).copy()).to(dev)
    d_uniq = torch.empty(n, dtype=torch.int64, device=dev)
    d_start = torch.empty(n + 1, dtype=torch.int32, device=dev)
    d_nc = torch.empty(1, dtype=torch.int64, device=dev)
    stream = torch.cuda.Stream(device=0)
    torch.cuda.synchronize(dev)
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(5):
        rc = lib.tsp_b200_build_cell_table_noalloc(d_cid.data_ptr(), n, d_uniq.data_ptr(), d_start.data_ptr(),
                                                   d_nc.data_ptr(), stream.cuda_stream)
        assert rc == 0, lib.tsp_b200_noalloc_last_error()
    stream.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    assert int(d_nc.cpu()[0]) == want_u.size


_LAZY_CHILD = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from turbospharticles_b200 import abi
cu = ctypes.CDLL("libcudart.so.12")
def free():
    f, t = ctypes.c_size_t(), ctypes.c_size_t()
    assert cu.cudaMemGetInfo(ctypes.byref(f), ctypes.byref(t)) == 0
    return f.value
lib = abi.load_library()
assert cu.cudaSetDevice(0) == 0
assert lib.tsp_b200_noalloc_setup() == 0, lib.tsp_b200_noalloc_last_error()
n = 4096
cid = np.repeat(np.arange(n // 4, dtype=np.uint64), 4)
bufs = []
for nbytes in (8 * n, 8 * n, 4 * (n + 1), 8):
    p = ctypes.c_void_p()
    assert cu.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(nbytes)) == 0
    bufs.append(p)
assert cu.cudaMemcpy(bufs[0], cid.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(8 * n), 1) == 0
assert cu.cudaDeviceSynchronize() == 0
f0 = free()
rc = lib.tsp_b200_build_cell_table_noalloc(bufs[0], n, bufs[1], bufs[2], bufs[3], None)
assert rc == 0, lib.tsp_b200_noalloc_last_error()
assert cu.cudaDeviceSynchronize() == 0
f1 = free()
nc = np.zeros(1, np.uint64)
assert cu.cudaMemcpy(nc.ctypes.data_as(ctypes.c_void_p), bufs[3], ctypes.c_size_t(8), 2) == 0
assert int(nc[0]) == n // 4, nc
assert f1 == f0, (f0, f1)
print("lazy ok")
"""


def test_noalloc_first_call_after_setup_loads_nothing_under_lazy_loading():
    """Fresh process with CUDA_MODULE_LOADING=LAZY: the first call after setup takes no device
    memory (setup has loaded the scan kernels already)."""
    import os
    import subprocess
    import sys
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY")
    r = subprocess.run([sys.executable, "-c", _LAZY_CHILD, root], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "lazy ok" in r.stdout, r.stdout + r.stderr


def test_noalloc_rejects_sizes_beyond_the_scratch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    lib = abi.load_library()
    n = abi.NOALLOC_MAX_PARTICLES + 1
    # rejected on the host before any pointer is touched or any work is queued
    rc = lib.tsp_b200_build_cell_table_noalloc(None, n, None, None, None, None)
    assert rc == -1
    assert b"TSP_NOALLOC_MAX_PARTICLES" in lib.tsp_b200_noalloc_last_error()


def test_noalloc_empty_input():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    lib = abi.load_library()
    torch.cuda.set_device(0)
    d_nc = torch.full((1,), 7, dtype=torch.int64, device="cuda:0")
    stream = torch.cuda.Stream(device=0)
    torch.cuda.synchronize()
    assert lib.tsp_b200_build_cell_table_noalloc(None, 0, None, None, d_nc.data_ptr(), stream.cuda_stream) == 0
    stream.synchronize()
    assert int(d_nc.cpu()[0]) == 0
    # with a start array, n = 0 writes start[0] = 0 (the end of the empty table)
    d_start = torch.full((1,), 7, dtype=torch.int32, device="cuda:0")
    d_nc.fill_(7)
    torch.cuda.synchronize()
    assert lib.tsp_b200_build_cell_table_noalloc(None, 0, None, d_start.data_ptr(), d_nc.data_ptr(),
                                                 stream.cuda_stream) == 0
    stream.synchronize()
    assert int(d_nc.cpu()[0]) == 0 and int(d_start.cpu()[0]) == 0
