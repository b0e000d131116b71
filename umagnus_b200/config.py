"""Initial magnetisation and geometry on the mesh, evaluated at cell centres
as the reference does (engine/util.go:132 Index2Coord, engine/magnetization.go:89
SetInShape): the mesh is centred on the origin.

Configurations follow engine/config.go, shapes engine/shape.go.  They are
host-side helpers producing arrays for Simulation.set_m / Simulation(geom=...).
"""
import numpy as np


def coords(N, cell):
    """(x, y, z) of every cell centre, each an array of shape (Nz, Ny, Nx)."""
    Nx, Ny, Nz = N
    cx, cy, cz = cell
    x = cx * (np.arange(Nx) - 0.5 * (Nx - 1))
    y = cy * (np.arange(Ny) - 0.5 * (Ny - 1))
    z = cz * (np.arange(Nz) - 0.5 * (Nz - 1))
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return X, Y, Z


def uniform(N, mx, my, mz):
    """engine/config.go:55 Uniform."""
    shape = (3, N[2], N[1], N[0])
    m = np.empty(shape, np.float32)
    m[0], m[1], m[2] = mx, my, mz
    return m


def vortex(N, cell, circ, pol):
    """engine/config.go:63-73 Vortex: in-plane curl with circulation circ and a
    core of polarisation pol smoothed over 2*cellsize_x^2."""
    X, Y, _ = coords(N, cell)
    diam2 = 2.0 * cell[0] ** 2
    r2 = X * X + Y * Y
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.sqrt(r2)
        mx = -Y * circ / r
        my = X * circ / r
    mz = 1.5 * pol * np.exp(-r2 / diam2)
    bad = np.isnan(mx) | np.isnan(my) | np.isnan(mz)  # engine/config.go:128-134 noNaN
    mx = np.where(bad, 0.0, mx)
    my = np.where(bad, 0.0, my)
    mz = np.where(bad, float(pol), mz)
    return np.stack([mx, my, mz]).astype(np.float32)


def ellipsoid(N, cell, dx, dy, dz=np.inf):
    """engine/shape.go:39-47 Ellipsoid / Ellipse: 1 inside, 0 outside (cell centre test)."""
    X, Y, Z = coords(N, cell)
    zt = 0.0 if np.isinf(dz) else (Z / dz) ** 2
    return ((X / dx) ** 2 + (Y / dy) ** 2 + zt <= 0.25).astype(np.float32)


def ellipse(N, cell, dx, dy):
    return ellipsoid(N, cell, dx, dy)


def two_domain_fn(cell, m1, mwall, m2):
    """engine/config.go:144-159 TwoDomain as a function of the cell-centre
    coordinates (X, Y, Z): m1 for x < 0, m2 for x >= 0, a Gaussian wall of
    width 2*cellsize_x blending in mwall.  Returns (3, ...) float64."""
    ww = 2 * cell[0]

    def f(X, Y, Z):
        gauss = np.exp(-((X / ww) ** 2))
        return np.stack([(1 - gauss) * np.where(X < 0, m1[c], m2[c]) + gauss * mwall[c] for c in range(3)])
    return f


def rot_z(f, theta):
    """engine/config.go:207-218 Config.RotZ: the configuration f rotated by
    theta about z (coordinates rotated back, the vectors forward)."""
    cs, sn = np.cos(theta), np.sin(theta)

    def g(X, Y, Z):
        m = f(X * cs + Y * sn, -X * sn + Y * cs, Z)
        return np.stack([m[0] * cs - m[1] * sn, m[0] * sn + m[1] * cs, m[2]])
    return g


def sample(N, cell, f):
    """A configuration function evaluated at every cell centre, as float32 (3, Nz, Ny, Nx)."""
    return np.asarray(f(*coords(N, cell)), np.float64).astype(np.float32)


def two_domain(N, cell, m1, mwall, m2):
    """engine/config.go TwoDomain: m1 for x < 0, m2 for x >= 0, a Gaussian
    wall of width 2*cellsize_x blending in mwall."""
    return sample(N, cell, two_domain_fn(cell, m1, mwall, m2))


def _fmod(a, b):
    """engine/shape.go:222-231 fmod: a folded into (-b/2, b/2]; b = 0 or inf: no folding."""
    if b == 0 or np.isinf(b):
        return a
    folded = np.sign(a) * (np.mod(np.abs(a + b / 2), b) - b / 2)
    return np.where(np.abs(a) > b / 2, folded, a)


def rect(N, cell, sidex, sidey, repeat=(0.0, 0.0, 0.0), transl=(0.0, 0.0, 0.0)):
    """engine/shape.go:77-82 Rect(sidex, sidey) (strict inequalities), then
    .Repeat(*repeat) (:216-220) and .Transl(*transl) (:208-212) in that
    order, as `rect(...).repeat(...).transl(...)` in a script: 1 inside, 0 outside."""
    X, Y, Z = coords(N, cell)
    x, y, z = X - transl[0], Y - transl[1], Z - transl[2]
    x, y, z = _fmod(x, repeat[0]), _fmod(y, repeat[1]), _fmod(z, repeat[2])
    rx, ry = sidex / 2, sidey / 2
    return ((x < rx) & (x > -rx) & (y < ry) & (y > -ry)).astype(np.float32)
