"""Device-op layer (opencl package mirror) against the oracle, through the C-ABI.

Per-cell kernels must be bit-identical to the oracle's float32 restatement
(which is itself bit-identical to the reference's kernels); reductions are
exact maxima / compensated sums.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_pins as G

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def cu(a, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def cl():
    from umagnus_b200 import opencl
    opencl.Init(0)
    return opencl


def _setup(N, seed=3, nreg=3):
    rng = np.random.default_rng(seed)
    m = G.random_unit(N, seed)
    m[:, rng.random(m.shape[1:]) < 0.05] = 0
    regions = rng.integers(0, nreg, size=m.shape[1:]).astype(np.uint8)
    aex = np.zeros(256, np.float32)
    aex[:nreg] = [1.3e-11, 0.8e-11, 2.1e-11][:nreg]
    dind = np.zeros(256, np.float32)
    dind[:nreg] = [3e-3, -1e-3, 2e-3][:nreg]
    return m, regions, O.exch_lut(aex), O.exch_lut(dind)


@pytest.mark.parametrize("N,pbc", [((13, 9, 4), 0), ((64, 64, 1), 0), ((40, 33, 7), 5)])
def test_exchange_bitexact(cl, N, pbc):
    m, regions, alut, _ = _setup(N)
    cell = (2e-9, 3e-9, 1.5e-9)
    Ms = (6e5 + 3e5 * np.random.default_rng(1).random(m.shape[1:])).astype(np.float32)
    B0 = np.random.default_rng(0).standard_normal(m.shape).astype(np.float32)
    want = B0.copy()
    O.add_exchange(want, m, alut, regions, cell, Ms, pbc=pbc)
    B = cu(B0)
    mesh = cl.Mesh(N, cell, ((pbc & 1), (pbc & 2) >> 1, (pbc & 4) >> 2))
    cl.AddExchange(B, cu(m), cu(alut), cl.MSlice(cu(Ms), 1.0), cu(regions), mesh)
    assert np.array_equal(B.cpu().numpy(), want)


@pytest.mark.parametrize("N,openbc", [((13, 9, 4), 0), ((32, 32, 1), 1), ((17, 20, 3), 0)])
def test_dmi_bitexact(cl, N, openbc):
    m, regions, alut, dlut = _setup(N)
    cell = (2e-9, 2e-9, 1e-9)
    want = np.zeros(m.shape, np.float32)
    O.add_dmi(want, m, alut, dlut, regions, cell, 1.1e6, openbc=openbc)
    B = cu(np.zeros(m.shape, np.float32))
    cl.AddDMI(B, cu(m), cu(alut), cu(dlut), 1.1e6, cu(regions), cl.Mesh(N, cell), OpenBC=openbc)
    assert np.array_equal(B.cpu().numpy(), want, equal_nan=True)


def test_uniaxial_zeeman_torque_bitexact(cl):
    N = (31, 17, 5)
    m, regions, _, _ = _setup(N)
    rng = np.random.default_rng(5)
    u = rng.standard_normal((3,) + m.shape[1:]).astype(np.float32)
    K1 = (rng.random(m.shape[1:]) * 5e5).astype(np.float32)
    want = np.zeros(m.shape, np.float32)
    O.add_uniaxial(want, m, 1.1e6, K1, 1e4, u)
    B = cu(np.zeros(m.shape, np.float32))
    cl.AddUniaxialAnisotropy2(B, cu(m), 1.1e6, cl.MSlice(cu(K1)), 1e4, cu(u))
    assert np.array_equal(B.cpu().numpy(), want)
    lut = rng.standard_normal((3, 256)).astype(np.float32)
    O.region_addv(want, lut, regions)
    cl.RegionAddV(B, cu(lut), cu(regions))
    assert np.array_equal(B.cpu().numpy(), want)
    alpha = rng.random(m.shape[1:]).astype(np.float32)
    t_want = O.lltorque(m, want, alpha)
    t = cu(np.zeros(m.shape, np.float32))
    cl.LLTorque(t, cu(m), B, cl.MSlice(cu(alpha)))
    assert np.array_equal(t.cpu().numpy(), t_want)
    cl.LLTorque(B, cu(m), B, 0.3)  # in place over B, engine/torque.go:140
    assert np.array_equal(B.cpu().numpy(), O.lltorque(m, want, 0.3))
    t2 = cu(np.zeros(m.shape, np.float32))
    cl.LLNoPrecess(t2, cu(m), cu(want))
    assert np.array_equal(t2.cpu().numpy(), O.llnoprecess(m, want))


@pytest.mark.parametrize("N,pbc,openbc", [((13, 9, 4), 0, 0), ((16, 16, 1), 0, 1), ((7, 5, 3), 5, 0)])
def test_dmibulk_bitexact(cl, N, pbc, openbc):
    """opencl/dmibulk.go AddDMIBulk (dmibulk.cl) against the oracle (itself
    bit-identical to the reference kernel)."""
    m, regions, aex, dind = _setup(N)
    cell = (2e-9, 3e-9, 1e-9)
    Ms = (np.float32(8e5) + np.arange(m[0].size, dtype=np.float32)).reshape(m[0].shape)
    want = np.random.default_rng(1).standard_normal(m.shape).astype(np.float32)
    B = cu(want.copy())
    O.add_dmibulk(want, m, aex, dind, regions, cell, Ms, pbc=pbc, openbc=openbc)
    mesh = cl.Mesh(N, cell, (pbc & 1, (pbc >> 1) & 1, (pbc >> 2) & 1))
    cl.AddDMIBulk(B, cu(m), cu(aex), cu(dind), cl.MSlice(cu(Ms)), cu(regions), mesh, OpenBC=bool(openbc))
    assert np.array_equal(B.cpu().numpy(), want)


@pytest.mark.parametrize("per_cell", [False, True])
def test_cubic_bitexact(cl, per_cell):
    """opencl/anisotropy.go AddCubicAnisotropy2 (cubicanisotropy2.cl)."""
    N = (31, 17, 5)
    m, _, _, _ = _setup(N)
    rng = np.random.default_rng(6)
    if per_cell:
        c1 = rng.standard_normal((3,) + m.shape[1:]).astype(np.float32)
        c2 = rng.standard_normal((3,) + m.shape[1:]).astype(np.float32)
        K1 = (rng.random(m.shape[1:]) * 5e5).astype(np.float32)
        gc1, gc2, gK1 = cu(c1), cu(c2), cl.MSlice(cu(K1))
    else:
        c1, c2, K1 = (1.0, 0.2, 0.1), (-0.1, 1.0, 0.3), 4.5e4
        gc1, gc2, gK1 = c1, c2, K1
    want = rng.standard_normal(m.shape).astype(np.float32)
    B = cu(want.copy())
    O.add_cubic(want, m, 1.1e6, K1, -2e4, 7e3, np.asarray(c1), np.asarray(c2))
    cl.AddCubicAnisotropy2(B, cu(m), 1.1e6, gK1, -2e4, 7e3, gc1, gc2)
    assert np.array_equal(B.cpu().numpy(), want)


def test_zero_mask(cl):
    """opencl/zeromask.go:12 ZeroMask: zero where the region's LUT entry is non-zero."""
    N = (19, 11, 3)
    m, regions, _, _ = _setup(N)
    lut = np.zeros(256, np.float32)
    lut[np.unique(regions)[::2]] = 1.0
    want = m.copy()
    want[:, lut[regions] != 0] = 0.0
    d = cu(m)
    cl.ZeroMask(d, cu(lut), cu(regions))
    assert np.array_equal(d.cpu().numpy(), want)


def test_madd_normalize_bitexact(cl):
    rng = np.random.default_rng(9)
    n = 5000
    srcs = [rng.standard_normal((3, 1, 1, n)).astype(np.float32) for _ in range(7)]
    facs = [float(np.float32(f)) for f in rng.standard_normal(7)]
    for k in range(2, 8):
        want = np.stack([O.madd([s[c].ravel() for s in srcs[:k]], facs[:k]) for c in range(3)]).reshape(3, 1, 1, n)
        d = cu(np.zeros((3, 1, 1, n), np.float32))
        cl.Madd(d, [cu(s) for s in srcs[:k]], facs[:k])
        assert np.array_equal(d.cpu().numpy(), want), k
    v = rng.standard_normal((3, 1, 1, n)).astype(np.float32)
    vol = rng.random((1, 1, n)).astype(np.float32)
    vol[0, 0, :7] = 0
    want = v.copy()
    O.normalize(want, vol)
    vt = cu(v)
    cl.Normalize(vt, cu(vol))
    assert np.array_equal(vt.cpu().numpy(), want)


def test_reductions_known_answers(cl):
    # opencl/reduce_test.go:46-120
    a = cu(np.arange(1000, dtype=np.float32))
    assert cl.Sum(a) == G.REDUCE_SUM_0_999
    x, y, want = G.REDUCE_DOT_1
    assert cl.Dot(cu(np.array(x, np.float32)), cu(np.array(y, np.float32))) == want
    c = cu(np.stack([np.full((1, 1, 32), v, np.float32) for v in (1, 2, 3)]))
    d = cu(np.stack([np.full((1, 1, 32), v, np.float32) for v in (4, 5, 6)]))
    assert cl.Dot(c, d) == 32 * (4 + 10 + 18)
    assert cl.MaxAbs(a) == 999
    assert cl.MaxVecDiff(c, d) == np.sqrt(27.0)
    assert cl.MaxVecNorm(d) == np.sqrt(77.0)


def test_reductions_match_oracle(cl):
    rng = np.random.default_rng(4)
    for n in (1, 255, 256, 257, 100003, 2 ** 20 + 7):
        v = rng.standard_normal((3, 1, 1, n)).astype(np.float32)
        w = rng.standard_normal((3, 1, 1, n)).astype(np.float32)
        assert cl.MaxVecNorm(cu(v)) == O.max_vec_norm(v)
        assert cl.MaxVecDiff(cu(v), cu(w)) == O.max_vec_diff(v, w)
        assert cl.MaxAbs(cu(v[0])) == O.max_abs(v[0])
        s_ref = O.rsum(v[0])
        assert abs(cl.Sum(cu(v[0])) - s_ref) <= 1e-12 * np.abs(v[0]).astype(np.float64).sum() + 1e-30
        d_ref = O.rdot(v[0], w[0])
        assert abs(cl.Dot(cu(v[0]), cu(w[0])) - d_ref) <= 1e-12 * np.abs(v[0] * w[0]).astype(np.float64).sum() + 1e-30


def test_empty_and_bad_arguments(cl):
    a = cu(np.zeros(0, np.float32))
    assert cl.MaxAbs(a) == 0.0
    with pytest.raises(cl.UmagError):
        cl.Madd(cu(np.zeros((1, 1, 4), np.float32)), [cu(np.zeros((1, 1, 4), np.float32))], [1.0])
