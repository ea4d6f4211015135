"""The F_s reduction for callers that cannot allocate device memory
when they sample: real-time loops that forbid allocation after start-up, and
programs whose device memory is reserved up front by another allocator.
bd_fself_isotropic_noalloc keeps its scratch in a fixed device array, so the
GPU test checks it against the allocating entry point bd_fself_isotropic on
two calls in a row (the second call finds the first call's partial sums in the
shared scratch), that calls after the first leave the driver's free-memory
figure unchanged, and that oversized inputs are refused.  Called through the C
ABI with ctypes.  A CPU test checks that the compiled entry point references
no allocation routine.  This file sorts last so a failure here comes after
every other test has run."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from bd_aging_b200 import build as BLD
from bd_aging_b200 import lib as B


def _abi():
    L = B.lib()
    f = L.bd_fself_isotropic_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_void_p]
    f.restype = C.c_int
    g = L.bd_fself_isotropic
    g.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_void_p]
    g.restype = C.c_int
    return f, g


def _inputs(rng, n):
    import torch
    r0 = rng.uniform(0, 30, size=(n, 3)).astype(np.float32)
    raw = (r0 + rng.normal(0, 0.4, size=(n, 3))).astype(np.float32)
    return torch.from_numpy(raw).cuda(), torch.from_numpy(r0).cuda()


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    noalloc, alloc = _abi()
    rng = np.random.default_rng(42)
    for call, n in enumerate((70001, 1234)):
        d_raw, d_r0 = _inputs(rng, n)
        torch.cuda.synchronize()
        out_a = np.zeros(3, np.float32)
        out_b = np.zeros(3, np.float32)
        assert noalloc(d_raw.data_ptr(), d_r0.data_ptr(), n, out_a.ctypes.data, 1, 6.19, None) == 0
        assert alloc(d_raw.data_ptr(), d_r0.data_ptr(), n, out_b.ctypes.data, 1, 6.19, None) == 0
        np.testing.assert_allclose(out_a, out_b, rtol=2e-6, atol=2e-7, err_msg="call %d" % call)
        assert out_a[0] == 0.0 and out_a[2] == 0.0


@pytest.mark.gpu
def test_noalloc_calls_leave_device_memory_unchanged():
    import torch
    noalloc, _ = _abi()
    rng = np.random.default_rng(7)
    inputs = [_inputs(rng, n) for n in (4096 * 256, 5000, 1)]  # the largest accepted size included
    torch.cuda.synchronize()
    out = np.zeros(1, np.float32)
    d_raw, d_r0 = inputs[1]
    assert noalloc(d_raw.data_ptr(), d_r0.data_ptr(), 5000, out.ctypes.data, 0, 6.19, None) == 0  # set-up call
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        for d_raw, d_r0 in inputs:
            assert noalloc(d_raw.data_ptr(), d_r0.data_ptr(), d_raw.shape[0], out.ctypes.data, 0, 6.19, None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert np.isfinite(out[0])


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_its_scratch():
    noalloc, _ = _abi()
    out = np.zeros(1, np.float32)
    # rejected on the host before any device access: the pointers are never used
    rc = noalloc(C.c_void_p(16), C.c_void_p(16), 4096 * 256 + 1, out.ctypes.data, 0, 6.19, None)
    assert rc == 1
    assert out[0] == 0.0


ALLOCATORS = ("cudaMalloc", "cudaFree", "cudaMallocAsync", "cudaFreeAsync", "cudaMallocManaged", "cudaMallocHost",
              "cudaHostAlloc", "cudaMallocPitch", "cudaMalloc3D", "cudaMallocArray", "cuMemAlloc", "cuMemCreate",
              "cudaMemPoolCreate", "malloc", "_Znwm", "_Znam")


def test_noalloc_object_references_no_allocation_routine(tmp_path):
    """The object file of the entry point (built here from csrc/noalloc.cu)
    imports none of the CUDA or C++ allocation routines (nm -u)."""
    if not shutil.which("nm"):
        pytest.skip("nm not available")
    obj = os.path.join(BLD.BUILD, "noalloc.o")
    src = os.path.join(BLD.CSRC, "noalloc.cu")
    if not os.path.exists(obj) or os.path.getmtime(obj) < os.path.getmtime(src):
        obj = str(tmp_path / "noalloc.o")
        subprocess.run([BLD.nvcc()] + BLD.NVCC_FLAGS + ["-c", src, "-o", obj], check=True, capture_output=True)
    syms = subprocess.run(["nm", "-u", obj], capture_output=True, text=True, check=True).stdout.split()
    used = sorted(s for s in syms if s in ALLOCATORS or s.startswith(("cudaMalloc", "cuMemAlloc")))
    assert not used, used
