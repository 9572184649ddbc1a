"""The allocation-free Schur operator, qexstag_stagD2ee_noalloc.

It exists for callers that cannot let a library call cudaMalloc (a host
whose pool allocator already holds the device memory, or one that cannot
take cudaMalloc's device-wide synchronisation mid-pipeline).  Called through
the C ABI it must give what qexstag_stagD2ee gives for device fields, on two
calls in a row (the calls share one static temporary), without lowering the
device's free memory, and must reject lattices beyond its static limit.  Both
entry points run the same FP64 half-sweep kernel on every site, so their
results are compared bit for bit; the oracle is the CPU reference, within
the Dslash tolerance.
This file is collected last so that a failure here does not hide the others.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import _lib as L
from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu
TOL = 1e-13  # the Dslash parity tolerance used throughout the tests


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("dims,naik", [((8, 8, 8, 8), True), ((16, 16, 16, 16), False)])
def test_noalloc_schur_matches_stagD2ee(cuda, dims, naik):
    torch = cuda
    V = F.volume(dims)
    h = V // 2
    g = F.fat_naik_links(dims, 7) if naik else F.naive_links(dims, 0.3, 7)
    s = S.Staggered(S.Layout(dims), S.to_device_links(g))
    x = S.to_device_vector(F.gaussian_vector(V, 11))
    m2 = 0.05 ** 2
    ref = torch.zeros_like(x)
    s.stagD2ee(ref, x, m2)  # the existing entry point, device fields
    outs = [torch.zeros_like(x) for _ in range(2)]
    lib = L.load()
    # first call: may do the once-per-device set-up (the static array's
    # address; in a fresh process CUDA's lazy loading commits the array then)
    rc = lib.qexstag_stagD2ee_noalloc(s.handle, _ptr(outs[0]), _ptr(x), m2)
    assert rc == L.OK, lib.qexstag_last_error().decode()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    # second call in a row: must not take any device memory
    rc = lib.qexstag_stagD2ee_noalloc(s.handle, _ptr(outs[1]), _ptr(x), m2)
    assert rc == L.OK, lib.qexstag_last_error().decode()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    want = S.to_host_vector(ref)[:h]
    xo = S.to_host_vector(x)
    xo[h:] = 0
    o = O.Oracle(dims, g)
    ro = o.vec()
    o.stagD2ee(ro, xo, m2)
    scale = np.abs(ro[:h]).max()
    for r in outs:
        got = S.to_host_vector(r)
        assert np.array_equal(got[:h], want)  # same kernel, same sites: bit-identical
        assert np.abs(got[:h] - ro[:h]).max() / scale < TOL
        assert not np.any(got[h:])  # odd sites untouched


def test_noalloc_rejects_lattices_beyond_its_limit(cuda):
    torch = cuda
    dims = (32, 32, 32, 8)  # 131072 even sites > 65536
    V = F.volume(dims)
    s = S.Staggered(S.Layout(dims), S.to_device_links(F.naive_links(dims, 0.3, 3)))
    x = torch.zeros((3, V), dtype=torch.complex128, device="cuda")
    r = torch.zeros_like(x)
    lib = L.load()
    rc = lib.qexstag_stagD2ee_noalloc(s.handle, _ptr(r), _ptr(x), 0.01)
    assert rc == L.ERR_ARG
    assert "65536" in lib.qexstag_last_error().decode()


def test_noalloc_after_finalize(cuda):
    """qexstag_finalize forgets the array's address; the next call looks it
    up again and still matches stagD2ee bit for bit."""
    torch = cuda
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = F.naive_links(dims, 0.3, 9)
    s = S.Staggered(S.Layout(dims), S.to_device_links(g))
    x = S.to_device_vector(F.gaussian_vector(V, 12))
    ref = torch.zeros_like(x)
    s.stagD2ee(ref, x, 0.04)
    lib = L.load()
    r = torch.zeros_like(x)
    assert lib.qexstag_stagD2ee_noalloc(s.handle, _ptr(r), _ptr(x), 0.04) == L.OK
    torch.cuda.synchronize()
    assert lib.qexstag_finalize() == L.OK
    r2 = torch.zeros_like(x)
    rc = lib.qexstag_stagD2ee_noalloc(s.handle, _ptr(r2), _ptr(x), 0.04)
    assert rc == L.OK, lib.qexstag_last_error().decode()
    torch.cuda.synchronize()
    assert torch.equal(r2, ref) and torch.equal(r, ref)
