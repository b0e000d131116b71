"""Demag path on the GPU against the oracle, through the C-ABI.

Tolerances: the FP64 Newell tensor built on the GPU agrees with the oracle's
FP64 restatement to 1e-10 relative (different libm ulps, amplified by the
near-field cancellation); the float32 kernel spectrum to 1e-6 of its largest
entry; the float32 demag field to 1e-5 relative per cell (|dB| <= 1e-5 *
max|B|), the accuracy the hot path promises against uMagNUS float32.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_pins as G

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL_FIELD = 1e-5


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def cl():
    from umagnus_b200 import opencl
    opencl.Init(0)
    return opencl


CASES = [
    ((12, 10, 6), (2e-9, 3e-9, 1.5e-9)),
    ((16, 12, 1), (4e-9, 4e-9, 3e-9)),
    ((7, 5, 3), (2e-9, 2e-9, 2e-9)),     # odd sizes: radix 7 in x, Pz = 5
    ((9, 6, 4), (1e-9, 2e-9, 1e-9)),     # Pz = 7
    ((24, 48, 2), (3e-9, 3e-9, 3e-9)),   # Pz = 3, radix 3 in y (96)
    ((64, 64, 1), (4e-9, 4e-9, 3e-9)),   # thin film
]


@pytest.mark.parametrize("N,cell", CASES)
def test_newell_kernel_fp64_matches_oracle(cl, N, cell):
    d = cl.NewNewellDemag(N, (0, 0, 0), cell)
    Kg = d.kernel()
    Ko = O.newell_kernel(N, cell)
    scale = np.abs(Ko).max()
    assert np.max(np.abs(Kg - Ko)) <= 1e-10 * scale
    d.Free()


@pytest.mark.parametrize("N,cell", CASES)
def test_kernel_spectrum_matches_oracle(cl, N, cell):
    d = cl.NewNewellDemag(N, (0, 0, 0), cell)
    S = d.spectrum()
    Kf, _ = O.kernel_spectrum(O.newell_kernel(N, cell))
    comps = [0, 1, 2, 5] if N[2] == 1 else range(6)
    for c in comps:
        assert np.max(np.abs(S[c] - Kf[c])) <= 1e-6 * np.abs(Kf[c]).max() + 1e-12, c
    d.Free()


def _check_field(cl, N, cell, Ms, vol=None, seed=7):
    m = G.random_unit(N, seed)
    d = cl.NewNewellDemag(N, (0, 0, 0), cell)
    Kf, _ = O.kernel_spectrum(O.newell_kernel(N, cell))
    want = O.demag_field(Kf, O.pad_size(N), m.astype(np.float64),
                         Ms if np.isscalar(Ms) else Ms.astype(np.float64),
                         vol=None if vol is None else vol.astype(np.float64), dtype=np.float64)
    B = cu(np.full(m.shape, 123.0, np.float32))  # overwritten (demag is the first term)
    ms = Ms if np.isscalar(Ms) else cl.MSlice(cu(Ms.astype(np.float32)))
    d.Exec(B, cu(m), None if vol is None else cu(vol.astype(np.float32)), ms)
    got = B.cpu().numpy().astype(np.float64)
    err = np.abs(got - want).max() / np.abs(want).max()
    d.Free()
    return err


@pytest.mark.parametrize("N,cell", CASES)
def test_demag_field_matches_oracle(cl, N, cell):
    assert _check_field(cl, N, cell, 8e5) <= TOL_FIELD


def test_demag_field_per_cell_ms_and_geometry(cl):
    N, cell = (20, 14, 5), (2e-9, 2e-9, 2e-9)
    rng = np.random.default_rng(3)
    Ms = (6e5 + 3e5 * rng.random((N[2], N[1], N[0])))
    vol = rng.random((N[2], N[1], N[0]))
    vol[0, 0, :4] = 0
    assert _check_field(cl, N, cell, Ms, vol) <= TOL_FIELD


def test_demag_field_3d_multilayer_subsize(cl):
    """128x128x16 cells of 2x2x1 nm (a quarter of the 256x256x16 multilayer)."""
    assert _check_field(cl, (128, 128, 16), (2e-9, 2e-9, 1e-9), 1.1e6) <= TOL_FIELD


@pytest.mark.parametrize("pin", [G.DEMAG_CUBE, G.DEMAG_SMALL, G.DEMAG_SMALL3D])
def test_uniform_prism_average_matches_closed_form(cl, pin):
    N, cell = pin["N"], pin["cell"]
    d = cl.NewNewellDemag(N, (0, 0, 0), cell)
    exact = G.prism_factors(N, cell)
    Ms = float(np.float32(1 / G.MU0))
    for comp in range(3):
        m = np.zeros((3, N[2], N[1], N[0]), np.float32)
        m[comp] = 1
        B = cu(np.zeros_like(m))
        d.Exec(B, cu(m), None, Ms)
        avg = B.cpu().numpy().reshape(3, -1).astype(np.float64).mean(axis=1)
        assert abs(avg[comp] / (G.MU0 * Ms) + exact[comp]) < 2e-6
    d.Free()


def test_unsupported_sizes_raise(cl):
    with pytest.raises(cl.UmagError):
        cl.NewNewellDemag((7, 8, 8), (1, 0, 0), (1e-9, 1e-9, 1e-9))   # periodic x needs an even Nx
    with pytest.raises(cl.UmagError):
        cl.NewNewellDemag((17, 8, 2), (0, 0, 0), (1e-9, 1e-9, 1e-9))  # 17 is a prime factor > 13


PBC_CASES = [
    ((16, 12, 1), (4e-9, 4e-9, 3e-9), (2, 3, 0)),   # film periodic in-plane
    ((12, 10, 6), (2e-9, 3e-9, 1.5e-9), (0, 0, 2)),  # periodic along z only
    ((8, 9, 4), (2e-9, 2e-9, 2e-9), (1, 2, 1)),     # every axis, odd Ny
]


@pytest.mark.parametrize("N,cell,pbc", PBC_CASES)
def test_pbc_kernel_and_field_match_oracle(cl, N, cell, pbc):
    """mag/demagkernel.go:339-355: no padding along periodic axes and the
    tensor summed over the periodic images (reference loop order)."""
    d = cl.NewNewellDemag(N, pbc, cell)
    assert d.padded_size() == O.pad_size(N, pbc)
    Kg = d.kernel()
    Ko = O.newell_kernel(N, cell, pbc)
    assert np.max(np.abs(Kg - Ko)) <= 1e-10 * np.abs(Ko).max()
    m = G.random_unit(N, 3)
    Kf, _ = O.kernel_spectrum(Ko)
    want = O.demag_field(Kf, O.pad_size(N, pbc), m.astype(np.float64), 8e5, dtype=np.float64)
    B = cu(np.zeros(m.shape, np.float32))
    d.Exec(B, cu(m), None, 8e5)
    got = B.cpu().numpy().astype(np.float64)
    assert np.abs(got - want).max() <= TOL_FIELD * np.abs(want).max()
    d.Free()


def test_pbc_film_of_uniform_m_is_thin_film_limit(cl):
    """A film periodic in-plane over many repetitions, magnetised along z,
    approaches the infinite-film demag field -mu0 Ms (N_zz -> 1)."""
    N, cell = (8, 8, 1), (2e-9, 2e-9, 2e-9)
    d = cl.NewNewellDemag(N, (32, 32, 0), cell)
    m = np.zeros((3, 1, 8, 8), np.float32)
    m[2] = 1
    B = cu(np.zeros(m.shape, np.float32))
    d.Exec(B, cu(m), None, 8e5)
    bz = float(B[2].mean()) / (G.MU0 * 8e5)
    assert abs(bz + 1.0) < 0.02, bz
    d.Free()
