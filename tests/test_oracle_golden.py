"""Pins the CPU oracle against known answers before it is trusted as checker.

Sources: the reference's own test scripts and Go unit tests (values quoted in
tests/golden_pins.py), and the closed-form demag factor of a prism.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_pins as G


def _avg_demag(N, cell, comp, Ms=1 / G.MU0, dtype=np.float64):
    K = O.newell_kernel(N, cell)
    Kf, maximg = O.kernel_spectrum(K)
    assert maximg < 1e-6  # opencl/conv_common.go:43-53 FFT_IMAG_TOLERANCE
    P = O.pad_size(N)
    m = np.zeros((3, N[2], N[1], N[0]), dtype)
    m[comp] = 1
    B = O.demag_field(Kf, P, m, Ms, dtype=dtype)
    return B.reshape(3, -1).mean(axis=1)


@pytest.mark.parametrize("pin", [G.DEMAG_CUBE, G.DEMAG_SMALL, G.DEMAG_SMALL3D])
def test_newell_matches_prism_formula(pin):
    """The Newell tensor summed over all cell pairs is the exact prism demag
    factor; uMagNUS64 rounds the Ms multiplier to float32 (amul.clh), so the
    comparison is done with an Ms that is exact in float32."""
    Ms = float(np.float32(1 / G.MU0))
    exact = G.prism_factors(pin["N"], pin["cell"])
    for c in range(3):
        b = _avg_demag(pin["N"], pin["cell"], c, Ms=Ms)
        assert abs(b[c] / (G.MU0 * Ms) + exact[c]) < 1e-12
        others = [b[(c + 1) % 3], b[(c + 2) % 3]]
        assert max(abs(o) for o in others) < 1e-14


@pytest.mark.parametrize("pin", [G.DEMAG_CUBE, G.DEMAG_SMALL, G.DEMAG_SMALL3D])
def test_demag_scripts_within_bruteforce_error(pin):
    """test/demag*.mx3 values (brute-force kernel) agree with Newell to the
    brute-force kernel's own discretisation error (<2e-3 relative)."""
    for c in range(3):
        b = _avg_demag(pin["N"], pin["cell"], c, dtype=np.float32)
        assert abs(b[c] - pin["want"][c]) <= max(2e-3 * abs(pin["want"][c]), pin.get("tol", 0))


def test_newell_kernel_symmetry():
    N, cell = (8, 6, 3), (2e-9, 3e-9, 1.5e-9)
    K = O.newell_kernel(N, cell)
    P = O.pad_size(N)
    assert K.shape == (6, P[2], P[1], P[0])
    # mirror in x: xx,yy,zz,yz even; xz,xy odd
    for c, s in zip(range(6), (1, 1, 1, 1, -1, -1)):
        a = K[c][:, :, 1:]
        assert np.array_equal(a, s * a[:, :, ::-1])
    # Nyquist planes of an even padded size are never computed (zero)
    assert np.all(K[:, :, :, P[0] // 2] == 0)
    # trace of the self term = -1
    assert abs(K[0, 0, 0, 0] + K[1, 0, 0, 0] + K[2, 0, 0, 0] + 1) < 1e-14


def test_newell_far_field_continuity():
    """Near (27-point) and far (asymptotic) formulas agree where both are
    accurate: at 9-16 cells the expansion error (~R^-8) and the near-field
    cancellation error (~eps R^6) are both near 1e-9; at 33-40 cells the
    near-field cancellation has grown to ~1e-6 (which is why the reference
    switches to the expansion beyond 32 cells)."""
    N, cell = (48, 48, 1), (1e-9, 1e-9, 1e-9)
    Knear = O.newell_kernel(N, cell, asymptotic_radius=1000)
    Kfar = O.newell_kernel(N, cell, asymptotic_radius=4)
    for pts, tol in (([(12, 0), (9, 8), (11, 4), (16, 0)], 1e-8), ([(33, 0), (30, 15), (25, 25), (40, 3)], 1e-5)):
        for x, y in pts:
            for c in (0, 1, 2, 5):
                a, b = Knear[c, 0, y, x], Kfar[c, 0, y, x]
                if c == 5 and (x == 0 or y == 0):
                    continue
                assert abs(a - b) <= tol * abs(a), (x, y, c, a, b)


def test_pad_size():
    # mag/demagkernel.go:404-420
    assert O.pad_size((256, 256, 16)) == (512, 512, 32)
    assert O.pad_size((64, 64, 1)) == (128, 128, 1)
    assert O.pad_size((3, 4, 2)) == (6, 8, 3)
    assert O.pad_size((10, 10, 5)) == (20, 20, 9)
    assert O.pad_size((10, 10, 6)) == (20, 20, 12)
    assert O.pad_size((10, 12, 4), (1, 0, 0)) == (10, 24, 7)


def test_fft_matches_numpy():
    rng = np.random.default_rng(1)
    for n in (1, 2, 3, 5, 7, 12, 96, 192, 512, 11, 13 * 4):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert np.allclose(O.fft(x), np.fft.fft(x), rtol=1e-12, atol=1e-12 * n)
        assert np.allclose(O.fft(x, +1), np.fft.ifft(x) * n, rtol=1e-12, atol=1e-12 * n)


def test_reduce_known_answers():
    # opencl/reduce_test.go:46-120
    a = np.arange(1000, dtype=np.float32)
    assert O.rsum(a) == G.REDUCE_SUM_0_999
    x, y, want = G.REDUCE_DOT_1
    assert O.rdot(np.array(x, np.float32), np.array(y, np.float32)) == want
    c = np.stack([np.full(32, v, np.float32) for v in (1, 2, 3)])
    d = np.stack([np.full(32, v, np.float32) for v in (4, 5, 6)])
    assert sum(O.rdot(c[i], d[i]) for i in range(3)) == 32 * (4 + 10 + 18)
    assert O.max_abs(a) == 999
    in2 = a.copy()
    in2[500] = np.float32(999.99)
    assert O.max_abs(in2) == np.float32(999.99)
    assert O.max_vec_diff(c, d) == pytest.approx(np.sqrt(27.0))
    assert O.max_vec_norm(d) == pytest.approx(np.sqrt(16 + 25 + 36.0))


def test_exchange_mx3_region_averages():
    """test/exchange.mx3: two-domain state, two regions, no demag."""
    p = G.EXCHANGE_MX3
    N, cell = p["N"], p["cell"]
    m = G.twodomain(N, cell, *p["twodomain"])
    O.normalize(m)
    X, _, _ = G.cell_coords(N, cell)
    regions = np.where(X < 0, 0, 1).astype(np.uint8)
    lut = O.exch_lut(np.full(256, p["Aex"], np.float32))
    B = np.zeros_like(m)
    O.add_exchange(B, m, lut, regions, cell, p["Ms"])
    tol = p["tol"]
    for r, want in ((0, p["region0"]), (1, p["region1"])):
        sel = regions == r
        got = [B[c][sel].astype(np.float64).mean() for c in range(3)]
        assert np.max(np.abs(np.array(got) - want)) < tol, (r, got, want)
    avg = [B[c].astype(np.float64).mean() for c in range(3)]
    assert np.max(np.abs(avg)) < tol


def test_exch_lut_harmonic_mean():
    # engine/exchange.go:193-201
    ex = np.zeros(256, np.float32)
    ex[0], ex[1], ex[2] = 1e-11, 2e-11, -1e-11
    lut = O.exch_lut(ex)
    assert lut[O.symidx(1, 0)] == np.float32(2) / (np.float32(1) / np.float32(1e-11) + np.float32(1) / np.float32(2e-11))
    assert lut[O.symidx(0, 0)] == np.float32(1e-11)
    v = lut[O.symidx(2, 0)]  # opposite signs: signed geometric-arithmetic mean -> 0 here
    assert v == 0.0
    assert lut[O.symidx(5, 5)] == 0.0
