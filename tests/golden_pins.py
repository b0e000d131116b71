"""Known answers for the hot path, with their sources.

Values quoted from the reference's own tests (read as text) and from the
published closed-form demag factor of a rectangular prism.
"""
import numpy as np

MU0 = 4 * np.pi * 1e-7

# test/demagcube.mx3: 2x2x2 cubes -> -1/3 each (tol 5e-4)
DEMAG_CUBE = dict(N=(2, 2, 2), cell=(1e-9, 1e-9, 1e-9), want=(-1 / 3, -1 / 3, -1 / 3), tol=5e-4)
# test/demagSmall.mx3:15-27 and test/demagSmall3D.mx3:15-27.  These numbers come
# from the reference's default brute-force kernel (mag/demagkernel.go); the
# Newell kernel is exact, so it agrees with them only to the brute-force error.
DEMAG_SMALL = dict(N=(3, 4, 1), cell=(1e-9, 2e-9, 0.5e-9),
                   want=(-0.15768295526, -0.05676037073, -0.78447151184))
DEMAG_SMALL3D = dict(N=(3, 4, 2), cell=(1e-9, 2e-9, 3e-9),
                     want=(-0.52710835138, -0.20121671756, -0.27112555503))

# test/exchange.mx3:6-21: region-averaged exchange field of a two-domain state
EXCHANGE_MX3 = dict(
    N=(300, 200, 4), cell=(2e-9, 3e-9, 4e-9), Ms=800e3, Aex=13e-12, tol=1.2e-8,
    twodomain=((1, 2, 3), (-1, -3, 5), (3, -1, 2)),
    avg=(0.0, 0.0, 0.0),
    region0=(0.00118888104756673, -0.00164631487528483, -0.00074591267903645),
    region1=(-0.00118888041178385, 0.00164631512959798, 0.00074591242472330),
)

# opencl/reduce_test.go:46-120
REDUCE_SUM_0_999 = 499500.0
REDUCE_DOT_1 = ([1, 2, 3, 4, 5], [5, 4, 3, -1, 2], 5 + 8 + 9 - 4 + 10)


def aharoni_nzz(a, b, c):
    """Demag factor N_zz of a uniformly magnetised prism with half-sides a, b, c
    along x, y, z: A. Aharoni, J. Appl. Phys. 83, 3432 (1998), eq. (1)."""
    r = np.sqrt(a * a + b * b + c * c)
    ab, bc, ac = np.sqrt(a * a + b * b), np.sqrt(b * b + c * c), np.sqrt(a * a + c * c)
    t = ((b * b - c * c) / (2 * b * c)) * np.log((r - a) / (r + a))
    t += ((a * a - c * c) / (2 * a * c)) * np.log((r - b) / (r + b))
    t += (b / (2 * c)) * np.log((ab + a) / (ab - a)) + (a / (2 * c)) * np.log((ab + b) / (ab - b))
    t += (c / (2 * a)) * np.log((bc - b) / (bc + b)) + (c / (2 * b)) * np.log((ac - a) / (ac + a))
    t += 2 * np.arctan(a * b / (c * r)) + (a ** 3 + b ** 3 - 2 * c ** 3) / (3 * a * b * c)
    t += ((a * a + b * b - 2 * c * c) / (3 * a * b * c)) * r + (c / (a * b)) * (ac + bc)
    t -= (ab ** 3 + bc ** 3 + ac ** 3) / (3 * a * b * c)
    return t / np.pi


def prism_factors(N, cell):
    """(Nxx, Nyy, Nzz) of the whole N-cell box."""
    L = [N[i] * cell[i] / 2 for i in range(3)]
    return (aharoni_nzz(L[1], L[2], L[0]), aharoni_nzz(L[2], L[0], L[1]), aharoni_nzz(L[0], L[1], L[2]))


def cell_coords(N, cell):
    """engine/util.go:132-140 Index2Coord, arrays shaped (Nz, Ny, Nx)."""
    ix = np.arange(N[0]); iy = np.arange(N[1]); iz = np.arange(N[2])
    x = cell[0] * (ix - 0.5 * (N[0] - 1))
    y = cell[1] * (iy - 0.5 * (N[1] - 1))
    z = cell[2] * (iz - 0.5 * (N[2] - 1))
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return X, Y, Z


def twodomain(N, cell, m1, mw, m2):
    """engine/config.go:144-158 TwoDomain, evaluated in float64, stored float32
    (engine/magnetization.go:89-114)."""
    X, _, _ = cell_coords(N, cell)
    ww = 2 * cell[0]
    g = np.exp(-((X / ww) ** 2))
    m = np.empty((3,) + X.shape)
    for c in range(3):
        base = np.where(X < 0, m1[c], m2[c])
        m[c] = (1 - g) * base + g * mw[c]
    return m.astype(np.float32)


def random_unit(N, seed, dtype=np.float32):
    """Seeded i.i.d. uniform directions on the sphere (normalised 3D Gaussian),
    shape (3, Nz, Ny, Nx)."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((3, N[2], N[1], N[0]))
    v /= np.sqrt((v * v).sum(axis=0))
    return v.astype(dtype)
