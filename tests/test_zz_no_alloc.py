"""umag_demag_exec_noalloc: the demag field for callers that cannot allocate
device memory at the time of the call (an external allocator owns the
device pool, or the host runtime forbids allocation after start-up).

The entry point keeps all of its working memory in one fixed __device__
array inside the library, so it is checked here, through the C-ABI, against
the allocating plan path (umag_demag_exec) and against the oracle's FP64
field on two calls in a row -- the second call must not see anything left
over from the first -- and the device's free memory must not move across a
call.  Tolerance: |dB| <= 1e-5 max|B|, the field tolerance of the other
demag tests.  One case runs in a fresh process that calls the entry point
before umag_init, as its header allows.  This file is collected last so a
failure here never hides another test.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_pins as G
from tests.conftest import ROOT

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL_FIELD = 1e-5
UMAG_E_UNSUPPORTED = 3


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


def _oracle_field(N, cell, m, Ms):
    Kf, _ = O.kernel_spectrum(O.newell_kernel(N, cell))
    return O.demag_field(Kf, O.pad_size(N), m.astype(np.float64), Ms, dtype=np.float64)


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
        mh = G.random_unit(N, seed)
        m = torch.as_tensor(mh).cuda()
        want = torch.zeros_like(m)
        plan.Exec(want, m, None, Ms)
        got = torch.full_like(m, 7.0)  # overwritten, like the plan path
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        rc = _noalloc(L, N, K, m, got, Ms)
        free1, _ = torch.cuda.mem_get_info()
        assert rc == 0, L.umag_last_error().decode()
        if call == 1:  # everything is loaded by now: the call itself takes no device memory
            assert free1 == free0, (free0, free1)
        w = want.cpu().numpy().astype(np.float64)
        g = got.cpu().numpy().astype(np.float64)
        assert np.abs(g - w).max() <= TOL_FIELD * np.abs(w).max(), f"call {call}"
        o = _oracle_field(N, cell, mh, Ms)
        assert np.abs(g - o).max() <= TOL_FIELD * np.abs(o).max(), f"call {call} vs oracle"
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
    assert rc == UMAG_E_UNSUPPORTED
    assert b"scratch" in L.umag_last_error()


@pytest.mark.parametrize("N", [(40, 40, 1), (64, 64, 2), (64, 64, 5)])
def test_noalloc_rejects_meshes_without_a_compile_time_plan(libs, N):
    """Nx = 40 has no compile-time x transform; Nz = 2..5 pad to an odd
    Pz = 2Nz - 1, which only the allocating plan path transforms."""
    L, _ = libs
    dummy = torch.zeros(1, device="cuda")
    kp = (ctypes.c_void_p * 6)(*([dummy.data_ptr()] * 6))
    B = [dummy] * 3
    rc = L.umag_demag_exec_noalloc(N[0], N[1], N[2], kp, _ptr(B[0]), _ptr(B[1]), _ptr(B[2]), _ptr(B[0]),
                                   _ptr(B[1]), _ptr(B[2]), None, None, 8e5, None)
    assert rc == UMAG_E_UNSUPPORTED
    assert b"no compile-time FFT plan" in L.umag_last_error()


_FRESH = r"""
import ctypes, sys
import numpy as np, torch
sys.path.insert(0, ROOT)
from oracle import oracle as O
from tests import golden_pins as G
from umagnus_b200 import _lib
L = _lib.load()
N, cell, Ms = (64, 64, 1), (4e-9, 4e-9, 3e-9), 8e5
Kf, _ = O.kernel_spectrum(O.newell_kernel(N, cell))
K = [torch.as_tensor(np.ascontiguousarray(Kf[c], np.float32)).cuda() for c in range(6)]
kp = (ctypes.c_void_p * 6)(K[0].data_ptr(), K[1].data_ptr(), K[2].data_ptr(), None, None, K[5].data_ptr())
outs = []
for seed in (21, 22):
    m = torch.as_tensor(G.random_unit(N, seed)).cuda()
    B = torch.full_like(m, 7.0)
    rc = L.umag_demag_exec_noalloc(N[0], N[1], N[2], kp, *[ctypes.c_void_p(B[c].data_ptr()) for c in range(3)],
                                   *[ctypes.c_void_p(m[c].data_ptr()) for c in range(3)], None, None, Ms, None)
    torch.cuda.synchronize()
    assert rc == 0, L.umag_last_error()
    outs.append((m, B))
assert _lib._initialised is None  # no umag_init so far in this process
from umagnus_b200 import opencl as cl
cl.Init(0)
plan = cl.NewNewellDemag(N, (0, 0, 0), cell)
for m, B in outs:
    want = torch.zeros_like(m)
    plan.Exec(want, m, None, Ms)
    w = want.double()
    err = float((B.double() - w).abs().max() / w.abs().max())
    assert err <= 1e-5, err
plan.Free()
print("fresh ok")
"""


def test_noalloc_first_call_before_init_in_a_fresh_process():
    code = "ROOT = %r\n" % ROOT + _FRESH
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ))
    assert r.returncode == 0 and "fresh ok" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]
