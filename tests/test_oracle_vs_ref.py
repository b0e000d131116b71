"""Pins the oracle's C restatement against the reference's own kernel code.

oracle/_ref/libclref.so holds the reference's OpenCL C kernels compiled
unchanged as C++ (oracle/build_ref.py).  Per-cell kernels must agree bit for
bit in float32 and float64; the demag glue (pad + Ms scaling, kernel
multiply with mirror symmetry, crop) is checked with numpy's FP64 FFT in
place of VkFFT.
"""
import numpy as np
import pytest

from oracle import clref
from oracle import oracle as O
from tests import golden_pins as G

pytestmark = pytest.mark.skipif(not clref.available(), reason="oracle/_ref/libclref.so not built")

DT = [np.float32, np.float64]


def _setup(N, dtype, seed=3, nreg=3):
    rng = np.random.default_rng(seed)
    m = G.random_unit(N, seed, dtype)
    # a few empty cells exercise the "missing neighbour" branches
    m[:, rng.random(m.shape[1:]) < 0.05] = 0
    regions = rng.integers(0, nreg, size=m.shape[1:]).astype(np.uint8)
    aex = np.zeros(256, dtype)
    aex[:nreg] = np.array([1.3e-11, 0.8e-11, 2.1e-11])[:nreg]
    dind = np.zeros(256, dtype)
    dind[:nreg] = np.array([3e-3, -1e-3, 2e-3])[:nreg]
    return m, regions, O.exch_lut(aex, dtype=dtype), O.exch_lut(dind, dtype=dtype)


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("N,pbc", [((13, 9, 4), 0), ((16, 16, 1), 0), ((7, 5, 3), 7), ((8, 6, 1), 3)])
def test_exchange_bitexact(dtype, N, pbc):
    m, regions, alut, _ = _setup(N, dtype)
    cell = (2e-9, 3e-9, 1.5e-9)
    Ms = dtype(8e5) + np.arange(m[0].size, dtype=dtype).reshape(m[0].shape)
    B1 = np.random.default_rng(0).standard_normal(m.shape).astype(dtype)
    B2 = B1.copy()
    O.add_exchange(B1, m, alut, regions, cell, Ms, pbc=pbc)
    w = [float(dtype(2.0 / (c * c))) for c in cell]
    clref.call("addexchange", dtype, B2[0], B2[1], B2[2], m[0], m[1], m[2], Ms, 1.0, alut, regions,
               w[0], w[1], w[2], N[0], N[1], N[2], pbc)
    assert np.array_equal(B1, B2)


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("N,pbc,openbc", [((13, 9, 4), 0, 0), ((16, 16, 1), 0, 1), ((7, 5, 3), 3, 0)])
def test_dmi_bitexact(dtype, N, pbc, openbc):
    m, regions, alut, dlut = _setup(N, dtype)
    cell = (2e-9, 2e-9, 1e-9)
    B1 = np.zeros(m.shape, dtype)
    B2 = B1.copy()
    O.add_dmi(B1, m, alut, dlut, regions, cell, 1.1e6, pbc=pbc, openbc=openbc)
    clref.call("adddmi", dtype, B2[0], B2[1], B2[2], m[0], m[1], m[2], None, 1.1e6, alut, dlut, regions,
               float(dtype(cell[0])), float(dtype(cell[1])), float(dtype(cell[2])), N[0], N[1], N[2], pbc, openbc)
    assert np.array_equal(B1, B2, equal_nan=True)


@pytest.mark.parametrize("dtype", DT)
def test_uniaxial_bitexact(dtype):
    N = (11, 7, 3)
    m, _, _, _ = _setup(N, dtype)
    rng = np.random.default_rng(5)
    u = rng.standard_normal((3,) + m.shape[1:]).astype(dtype)
    K1 = (rng.random(m.shape[1:]) * 5e5).astype(dtype)
    B1 = np.zeros(m.shape, dtype)
    B2 = B1.copy()
    O.add_uniaxial(B1, m, 1.1e6, K1, 1e4, u)
    n = m[0].size
    clref.call("adduniaxialanisotropy2", dtype, B2[0], B2[1], B2[2], m[0], m[1], m[2], None, 1.1e6,
               K1, 1.0, None, 1e4, u[0], 1.0, u[1], 1.0, u[2], 1.0, n)
    assert np.array_equal(B1, B2)


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("N,pbc,openbc", [((13, 9, 4), 0, 0), ((16, 16, 1), 0, 1), ((7, 5, 3), 5, 0),
                                          ((6, 7, 4), 0, 1)])
def test_dmibulk_bitexact(dtype, N, pbc, openbc):
    m, regions, alut, dlut = _setup(N, dtype)
    cell = (2e-9, 3e-9, 1e-9)
    Ms = dtype(8e5) + np.arange(m[0].size, dtype=dtype).reshape(m[0].shape)
    B1 = np.random.default_rng(1).standard_normal(m.shape).astype(dtype)
    B2 = B1.copy()
    O.add_dmibulk(B1, m, alut, dlut, regions, cell, Ms, pbc=pbc, openbc=openbc)
    clref.call("adddmibulk", dtype, B2[0], B2[1], B2[2], m[0], m[1], m[2], Ms, 1.0, alut, dlut, regions,
               float(dtype(cell[0])), float(dtype(cell[1])), float(dtype(cell[2])), N[0], N[1], N[2], pbc, openbc)
    assert np.array_equal(B1, B2, equal_nan=True)


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("per_cell", [False, True])
def test_cubic_bitexact(dtype, per_cell):
    N = (11, 7, 3)
    m, _, _, _ = _setup(N, dtype)
    rng = np.random.default_rng(6)
    if per_cell:
        c1 = rng.standard_normal((3,) + m.shape[1:]).astype(dtype)
        c2 = rng.standard_normal((3,) + m.shape[1:]).astype(dtype)
        K1 = (rng.random(m.shape[1:]) * 5e5).astype(dtype)
    else:
        c1 = np.array([1.0, 0.2, 0.1])
        c2 = np.array([-0.1, 1.0, 0.3])
        K1 = 4.5e4
    B1 = rng.standard_normal(m.shape).astype(dtype)
    B2 = B1.copy()
    O.add_cubic(B1, m, 1.1e6, K1, -2e4, 7e3, c1, c2)
    n = m[0].size
    if per_cell:
        cargs = [c1[0], 1.0, c1[1], 1.0, c1[2], 1.0, c2[0], 1.0, c2[1], 1.0, c2[2], 1.0]
        kargs = [K1, 1.0]
    else:
        cargs = [None, float(c1[0]), None, float(c1[1]), None, float(c1[2]),
                 None, float(c2[0]), None, float(c2[1]), None, float(c2[2])]
        kargs = [None, 4.5e4]
    clref.call("addcubicanisotropy2", dtype, B2[0], B2[1], B2[2], m[0], m[1], m[2], None, 1.1e6, *kargs,
               None, -2e4, None, 7e3, *cargs, n)
    assert np.array_equal(B1, B2)


@pytest.mark.parametrize("dtype", DT)
def test_set_temperature_bitexact(dtype):
    rng = np.random.default_rng(8)
    n = 3001
    noise = rng.standard_normal(n).astype(dtype)
    Ms = (rng.random(n) * 1e6 + 1e5).astype(dtype)
    Ms[::17] = 0
    temp = (rng.random(n) * 400).astype(dtype)
    k2 = float(dtype(2 * 1.380650424e-23 / (1.7595e11 * 1e-24 * 2e-13)))
    B1 = np.zeros(n, dtype)
    B2 = np.zeros(n, dtype)
    O.set_temperature(B1, noise, k2, Ms, temp, 0.05)
    clref.call("settemperature2", dtype, B2, noise, k2, Ms, 1.0, temp, 1.0, None, 0.05, n)
    assert np.array_equal(B1, B2)


@pytest.mark.parametrize("dtype", DT)
def test_torque_zeeman_madd_normalize_bitexact(dtype):
    N = (9, 8, 2)
    n = N[0] * N[1] * N[2]
    m, regions, _, _ = _setup(N, dtype)
    rng = np.random.default_rng(9)
    H = rng.standard_normal(m.shape).astype(dtype)
    alpha = rng.random(m.shape[1:]).astype(dtype)
    t1 = O.lltorque(m, H, alpha)
    t2 = np.zeros_like(m)
    clref.call("lltorque2", dtype, t2[0], t2[1], t2[2], m[0], m[1], m[2], H[0], H[1], H[2], alpha, 1.0, n)
    assert np.array_equal(t1, t2)
    t1 = O.llnoprecess(m, H)
    clref.call("llnoprecess", dtype, t2[0], t2[1], t2[2], m[0], m[1], m[2], H[0], H[1], H[2], n)
    assert np.array_equal(t1, t2)
    lut = rng.standard_normal((3, 256)).astype(dtype)
    B1 = H.copy()
    B2 = H.copy()
    O.region_addv(B1, lut, regions)
    clref.call("regionaddv", dtype, B2[0], B2[1], B2[2], lut[0], lut[1], lut[2], regions, n)
    assert np.array_equal(B1, B2)
    srcs = [rng.standard_normal(n).astype(dtype) for _ in range(7)]
    facs = [float(dtype(f)) for f in rng.standard_normal(7)]
    for k in range(2, 8):
        d1 = O.madd(srcs[:k], facs[:k], dtype)
        d2 = np.zeros(n, dtype)
        args = []
        for j in range(k):
            args += [srcs[j], facs[j]]
        clref.call(f"madd{k}", dtype, d2, *args, n)
        assert np.array_equal(d1, d2), k
    v1 = H.copy()
    v2 = H.copy()
    vol = rng.random(m.shape[1:]).astype(dtype)
    vol[0, 0, :3] = 0
    O.normalize(v1, vol)
    clref.call("normalize2", dtype, v2[0], v2[1], v2[2], vol, n)
    assert np.array_equal(v1, v2)


@pytest.mark.parametrize("N", [(6, 5, 3), (8, 6, 1), (5, 4, 7)])
def test_demag_glue_matches_reference(N):
    """copypadmul2 -> FFT -> kernmulRSymm* -> IFFT -> copyunpad with the
    reference's kernels and numpy's FFT equals the oracle's convolution."""
    dtype = np.float64
    cell = (2e-9, 3e-9, 2.5e-9)
    K = O.newell_kernel(N, cell)
    Kf, _ = O.kernel_spectrum(K)
    P = O.pad_size(N)
    m = G.random_unit(N, 11, dtype)
    Ms = (6e5 + 3e5 * np.random.default_rng(2).random(m.shape[1:]))
    want = O.demag_field(Kf, P, m, Ms, dtype=dtype)
    spec = []
    for c in range(3):
        pad = np.zeros((P[2], P[1], P[0]), dtype)
        clref.call("copypadmul2", dtype, pad, P[0], P[1], P[2], np.ascontiguousarray(m[c]), N[0], N[1], N[2],
                   Ms, 1.0, None)
        spec.append(np.ascontiguousarray(np.fft.rfftn(pad).view(np.float64)))  # (Pz, Py, Px/2+1) complex
    Kfc = [np.ascontiguousarray(Kf[c]) for c in range(6)]
    hx = P[0] // 2 + 1
    if P[2] == 1:
        clref.call("kernmulRSymm2Dz", dtype, spec[2], Kfc[2], hx, P[1])
        clref.call("kernmulRSymm2Dxy", dtype, spec[0], spec[1], Kfc[0], Kfc[1], Kfc[5], hx, P[1])
    else:
        clref.call("kernmulRSymm3D", dtype, spec[0], spec[1], spec[2], *Kfc, hx, P[1], P[2])
    got = np.zeros_like(m)
    for c in range(3):
        full = np.fft.irfftn(spec[c].view(np.complex128), s=(P[2], P[1], P[0]), axes=(0, 1, 2)) * (P[0] * P[1] * P[2])
        full = np.ascontiguousarray(full)
        out = np.zeros((N[2], N[1], N[0]), dtype)
        clref.call("copyunpad", dtype, out, N[0], N[1], N[2], full, P[0], P[1], P[2])
        got[c] = out
    scale = np.abs(want).max()
    assert np.max(np.abs(got - want)) <= 1e-13 * scale
