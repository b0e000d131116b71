"""umag_demag_exec_noalloc: the demag field for callers that cannot allocate
device memory at the time of the call (an external allocator owns the
device pool, or the host runtime forbids allocation after start-up).

The entry point keeps all of its working memory in one fixed __device__
array inside the library, so it is checked here, through the C-ABI, against
the allocating plan path (umag_demag_exec) on two calls in a row -- the
second call must not see anything left over from the first.  Tolerance:
|dB| <= 1e-5 max|B|, the field tolerance of the other demag tests.  This
file is collected last so a failure here never hides another test.
"""
import ctypes

import numpy as np
import pytest

from tests import golden_pins as G

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL_FIELD = 1e-5


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def libs():
    from umagnus_b200 import _lib, opencl
    opencl.Init(0)
    return _lib.load(), opencl


def _noalloc(L, N, K, m, B, Ms):
    kp = (ctypes.c_void_p * 6)(*[None if k is None else k.data_ptr() for k in K])
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.umag_demag_exec_noalloc(N[0], N[1], N[2], kp, _ptr(B[0]), _ptr(B[1]), _ptr(B[2]), _ptr(m[0]),
                                   _ptr(m[1]), _ptr(m[2]), None, None, float(Ms), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return rc


@pytest.mark.parametrize("N,cell", [((64, 64, 1), (4e-9, 4e-9, 3e-9)), ((128, 128, 16), (2e-9, 2e-9, 1e-9))])
def test_noalloc_matches_plan_exec_twice(libs, N, cell):
    L, cl = libs
    plan = cl.NewNewellDemag(N, (0, 0, 0), cell)
    spec = plan.spectrum()
    K = [torch.as_tensor(spec[c]).cuda() for c in range(6)]
    if N[2] == 1:
        K[3] = K[4] = None
    Ms = 8e5
    for call, seed in enumerate((11, 12)):
        m = torch.as_tensor(G.random_unit(N, seed)).cuda()
        want = torch.zeros_like(m)
        plan.Exec(want, m, None, Ms)
        got = torch.full_like(m, 7.0)  # overwritten, like the plan path
        rc = _noalloc(L, N, K, m, got, Ms)
        assert rc == 0, L.umag_last_error().decode()
        w = want.cpu().numpy().astype(np.float64)
        g = got.cpu().numpy().astype(np.float64)
        assert np.abs(g - w).max() <= TOL_FIELD * np.abs(w).max(), f"call {call}"
    plan.Free()


def test_noalloc_rejects_meshes_beyond_its_scratch(libs):
    L, _ = libs
    N = (256, 256, 16)  # the spectrum alone needs 51 MB, beyond the 16 MiB scratch
    dummy = torch.zeros(1, device="cuda")
    K = [dummy] * 6
    B = [dummy] * 3
    kp = (ctypes.c_void_p * 6)(*[k.data_ptr() for k in K])
    rc = L.umag_demag_exec_noalloc(N[0], N[1], N[2], kp, _ptr(B[0]), _ptr(B[1]), _ptr(B[2]), _ptr(B[0]),
                                   _ptr(B[1]), _ptr(B[2]), None, None, 8e5, None)
    assert rc == 3  # UMAG_E_UNSUPPORTED
    assert b"scratch" in L.umag_last_error()
