"""bd_fself_isotropic_noalloc: the F_s reduction for callers that cannot
allocate device memory when they sample (code running inside a stream
capture in global capture mode, real-time loops, hosts whose device memory
belongs to another allocator).  Its scratch is a fixed device array, so the
test checks it against the allocating entry point bd_fself_isotropic on two
calls in a row (the second call finds the first call's partial sums in the
shared scratch) and that oversized inputs are refused.  Called through the C
ABI with ctypes.  This file sorts last so a failure here comes after every
other test has run."""
import ctypes as C

import numpy as np
import pytest

from bd_aging_b200 import lib as B

pytestmark = pytest.mark.gpu


def _abi():
    L = B.lib()
    f = L.bd_fself_isotropic_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_void_p]
    f.restype = C.c_int
    g = L.bd_fself_isotropic
    g.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_void_p]
    g.restype = C.c_int
    return f, g


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    noalloc, alloc = _abi()
    rng = np.random.default_rng(42)
    for call, n in enumerate((70001, 1234)):
        r0 = rng.uniform(0, 30, size=(n, 3)).astype(np.float32)
        raw = (r0 + rng.normal(0, 0.4, size=(n, 3))).astype(np.float32)
        d_raw = torch.from_numpy(raw).cuda()
        d_r0 = torch.from_numpy(r0).cuda()
        out_a = np.zeros(3, np.float32)
        out_b = np.zeros(3, np.float32)
        assert noalloc(d_raw.data_ptr(), d_r0.data_ptr(), n, out_a.ctypes.data, 1, 6.19, None) == 0
        assert alloc(d_raw.data_ptr(), d_r0.data_ptr(), n, out_b.ctypes.data, 1, 6.19, None) == 0
        np.testing.assert_allclose(out_a, out_b, rtol=2e-6, atol=2e-7, err_msg="call %d" % call)
        assert out_a[0] == 0.0 and out_a[2] == 0.0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    noalloc, _ = _abi()
    out = np.zeros(1, np.float32)
    # rejected on the host before any device access: the pointers are never used
    rc = noalloc(C.c_void_p(16), C.c_void_p(16), 4096 * 256 + 1, out.ctypes.data, 0, 6.19, None)
    assert rc == 1
    assert out[0] == 0.0
