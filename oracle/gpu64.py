"""FP64 instantiation of the oracle on the GPU (torch float64 + cuFFT), for
meshes the CPU oracle cannot step in reasonable time.

TEST INFRASTRUCTURE ONLY: bench.py's precision report and tests/ use it as
the FP64 reference (the uMagNUS64 semantics); the product never imports it.
It restates the FP64 variant of orc_sim.inc (engine64/effectivefield.go,
torque.go, rk45dp.go, stepcontroller.go, run.go:150-188) operation by
operation, in FP64 throughout, and is checked against the CPU oracle on
small meshes by tests/test_gpu_fp64_oracle.py.  Fields are (3, Nz, Ny, Nx)
float64 tensors on the device.
"""
import math

import numpy as np
import torch

MU0 = 4 * math.pi * 1e-7  # kernels_src/clh/constants.clh:5
NREGION = 256


def symidx(i, j):
    """kernels_src/clh/exchange.clh:5"""
    hi = torch.maximum(i, j)
    lo = torch.minimum(i, j)
    return hi * (hi + 1) // 2 + lo


class System64:
    """Effective field and LL torque in FP64 (engine64/effectivefield.go:14-24
    order: demag sets B, exchange, uniaxial anisotropy, Zeeman add).

    kernel: real-space demag kernel (6, Pz, Py, Px) float64 (xx yy zz yz xz
    xy) or None for no demag; Ms, Ku1: (Nz, Ny, Nx) arrays or scalars; aLUT:
    32896 float64 exchange LUT with `regions` (uint8 map); anisU: 3-vector or
    (3, Nz, Ny, Nx); B_ext: 3-vector or None; alpha scalar; dLUT: 32896
    float64 interfacial-DMI LUT (None: exchange only), which switches the
    exchange term to dmi.cl's exchange + DMI as engine/exchange.go:49-66
    does; openbc: dmi.cl's OpenBC (no boundary extrapolation).  Open
    boundaries only (no PBC)."""

    def __init__(self, N, cell, Ms, aLUT, regions, alpha, kernel=None, Ku1=0.0, anisU=(0.0, 0.0, 1.0), B_ext=None,
                 device="cuda", dLUT=None, openbc=False):
        self.dev = torch.device(device)
        self.N = tuple(int(n) for n in N)
        Nx, Ny, Nz = self.N
        self.shape = (Nz, Ny, Nx)
        f64 = torch.float64

        def field(v):
            t = torch.as_tensor(np.asarray(v, np.float64), device=self.dev)
            return t.expand(self.shape).contiguous() if t.dim() == 0 else t.reshape(self.shape)

        # a uniform parameter passes through amul's float multiplier
        # (clh/amul.clh:5, declared float in uMagNUS64 too): float32-rounded
        def uniform(v):
            return float(np.float32(v)) if np.isscalar(v) else v

        Ms, Ku1, alpha = uniform(Ms), uniform(Ku1), uniform(alpha)
        self.Ms = field(Ms)
        self.inv_ms = torch.where(self.Ms == 0, torch.zeros_like(self.Ms), 1.0 / self.Ms)
        self.alpha = float(alpha)
        self.gilb = -1.0 / (1.0 + self.alpha * self.alpha)  # lltorque2.cl:18
        # exchange coefficients per direction: w_d * aLUT[symidx(r, r_neighbour)]
        # (exchange.cl with opencl/exchange.go:17-20 weights 2/c^2)
        reg = torch.as_tensor(np.asarray(regions, np.uint8).reshape(self.shape), device=self.dev).long()
        lut = torch.as_tensor(np.asarray(aLUT, np.float64), device=self.dev)
        w = [2.0 / (c * c) for c in cell]
        self.cell = tuple(float(c) for c in cell)
        self.reg, self.aLUT = reg, lut
        self.dLUT = None if dLUT is None else torch.as_tensor(np.asarray(dLUT, np.float64), device=self.dev)
        self.openbc = bool(openbc)
        self.dirs = []  # (axis, side, coefficient tensor)
        for axis, wd in ((2, w[0]), (1, w[1]), (0, w[2])):
            if axis == 0 and Nz == 1:
                continue
            for side in (-1, 1):
                rn = self._shift(reg, axis, side)
                self.dirs.append((axis, side, wd * lut[symidx(reg, rn)]))
        self.K1 = field(Ku1)
        self.anis = bool((self.K1 != 0).any())
        u = np.asarray(anisU, np.float64)
        if u.ndim == 1:
            u = u.astype(np.float32).astype(np.float64)
            ut = torch.as_tensor(u, device=self.dev)[:, None, None, None].expand((3,) + self.shape)
        else:
            ut = torch.as_tensor(u.reshape((3,) + self.shape), device=self.dev)
        ln = torch.sqrt((ut * ut).sum(0))
        self.u = ut * torch.where(ln != 0, 1.0 / ln, torch.zeros_like(ln))  # uniaxialanisotropy2.cl:20-22
        self.B_ext = None if B_ext is None else torch.as_tensor(np.asarray(B_ext, np.float64),
                                                                device=self.dev)[:, None, None, None]
        self.demag = kernel is not None
        if self.demag:
            K = torch.as_tensor(np.asarray(kernel, np.float64), device=self.dev)
            self.P = tuple(K.shape[1:])  # (Pz, Py, Px)
            # the FP64 kernel spectrum (real for the even/odd-symmetric tensor)
            self.Kf = torch.stack([torch.fft.rfftn(K[c]).real for c in range(6)])
            del K
        self.f64 = f64

    @staticmethod
    def _shift(x, axis, side):
        """x at the clamped neighbour (index + side along axis; stencil.clh)."""
        n = x.shape[axis]
        idx = torch.arange(n, device=x.device) + side
        idx = idx.clamp(0, n - 1)
        return torch.index_select(x, axis, idx)

    def demag_field(self, m):
        Nz, Ny, Nx = self.shape
        Pz, Py, Px = self.P
        V = torch.zeros((3, Pz, Py, Px), dtype=self.f64, device=self.dev)
        V[:, :Nz, :Ny, :Nx] = (MU0 * self.Ms) * m  # copypadmul2.cl: MU0*Ms in FP64
        F = torch.fft.rfftn(V, dim=(1, 2, 3))
        del V
        xx, yy, zz, yz, xz, xy = self.Kf
        B = torch.empty((3, Nz, Ny, Nx), dtype=self.f64, device=self.dev)
        for c, (a, b, d) in enumerate(((xx, xy, xz), (xy, yy, yz), (xz, yz, zz))):
            Bc = torch.fft.irfftn(a * F[0] + b * F[1] + d * F[2], s=(Pz, Py, Px), dim=(0, 1, 2))
            B[c] = Bc[:Nz, :Ny, :Nx]
        return B

    def exchange_field(self, m):
        """exchange.cl: sum_d coef (m_nb - m0), m_nb = m0 where m_nb is zero;
        times 1/Ms; nothing where m0 is zero."""
        m0zero = (m * m).sum(0) == 0
        e = torch.zeros_like(m)
        for axis, side, coef in self.dirs:
            mn = self._shift(m, axis + 1, side)
            nz = (mn * mn).sum(0) == 0
            mn = torch.where(nz[None], m, mn)
            e += coef[None] * (mn - m)
        e = e * self.inv_ms[None]
        return torch.where(m0zero[None], torch.zeros_like(e), e)

    def dmi_field(self, m):
        """dmi.cl:8-148 (exchange + interfacial DMI) in FP64.  In-plane
        neighbours outside the mesh or empty (m = 0) take the Neumann
        extrapolation of dmi.cl:46-50, 67-71, 89-93, 110-114 (nothing with
        OpenBC); the pair coefficients A, D come from the LUTs at (r0, rn) with
        rn = r0 for a missing neighbour; z neighbours carry exchange only
        (clamped, an empty one counts as m0); the sum is times 1/Ms and zero
        where m0 is zero."""
        m0zero = (m * m).sum(0) == 0
        h = torch.zeros_like(m)
        reg = self.reg
        for axis, c in ((2, self.cell[0]), (1, self.cell[1])):  # x, y: tensor axes of (Nz, Ny, Nx)
            n = m.shape[axis + 1]
            for side in (-1, 1):
                idx = torch.arange(n, device=m.device) + side
                inside = (idx >= 0) & (idx < n)
                mn = torch.index_select(m, axis + 1, idx.clamp(0, n - 1))
                shape = [1, 1, 1]
                shape[axis] = n
                mn = mn * inside.to(m.dtype).reshape([1] + shape)
                nz = (mn * mn).sum(0) == 0
                rn = torch.where(nz, reg, self._shift(reg, axis, side))
                k = symidx(reg, rn)
                A = self.aLUT[k]
                D = self.dLUT[k]
                sc = -c if side < 0 else c
                q = sc * (0.5 * D / A)
                mx, my, mz = m[0], m[1], m[2]
                if axis == 2:
                    ext = torch.stack([mx - q * mz, my, mz + q * mx])
                else:
                    ext = torch.stack([mx, my - q * mz, mz + q * my])
                mn = torch.where(nz[None], ext, mn)
                act = (~nz) if self.openbc else torch.ones_like(nz)
                act = act.to(m.dtype)
                s = 2.0 * A / (c * c)
                h += (act * s)[None] * (mn - m)
                Dc = act * D / c
                tz = -mn[2] if side < 0 else mn[2]
                tp = -mn[0 if axis == 2 else 1] if side < 0 else mn[0 if axis == 2 else 1]
                h[0 if axis == 2 else 1] += Dc * tz
                h[2] -= Dc * tp
        if self.shape[0] != 1:
            cz = self.cell[2]
            for side in (-1, 1):
                mn = self._shift(m, 1, side)
                nz = (mn * mn).sum(0) == 0
                mn = torch.where(nz[None], m, mn)
                A = self.aLUT[symidx(reg, self._shift(reg, 0, side))]
                h += (2.0 * A / (cz * cz))[None] * (mn - m)
        h = h * self.inv_ms[None]
        return torch.where(m0zero[None], torch.zeros_like(h), h)

    def field_terms(self, m):
        """(demag, exchange or exchange + DMI, anisotropy, zeeman) fields of m."""
        Bd = self.demag_field(m) if self.demag else torch.zeros_like(m)
        Be = self.exchange_field(m) if self.dLUT is None else self.dmi_field(m)
        if self.anis:
            mu = (m * self.u).sum(0)
            Ba = (2.0 * self.K1 * self.inv_ms * mu)[None] * self.u
        else:
            Ba = torch.zeros_like(m)
        Bz = torch.zeros_like(m) if self.B_ext is None else self.B_ext.expand_as(m)
        return Bd, Be, Ba, Bz

    def beff(self, m):
        Bd, Be, Ba, Bz = self.field_terms(m)
        return ((Bd + Be) + Ba) + Bz

    def torque(self, m, B=None):
        if B is None:
            B = self.beff(m)
        mxB = torch.linalg.cross(m, B, dim=0)
        return self.gilb * (mxB + self.alpha * torch.linalg.cross(m, mxB, dim=0))

    def energy_density(self, m):
        """engine64/energy.go SetTotalEdens: -1/2 M.(B_anis + B_demag + B_exch) - M.B_ext."""
        Bd, Be, Ba, Bz = self.field_terms(m)
        Mf = self.Ms[None] * m
        d = lambda B: (Mf * B).sum(0)  # noqa: E731
        return ((-0.5 * d(Ba) + -0.5 * d(Bd)) + -0.5 * d(Be)) + -1.0 * d(Bz)


def normalize(v):
    """normalize2.cl in FP64: v / |v|, zero for a zero vector."""
    n = torch.sqrt((v * v).sum(0))
    return v * torch.where(n > 0, 1.0 / n, torch.zeros_like(n))[None]


class RK45DP64:
    """engine64/rk45dp.go:12-98 with engine64/stepcontroller.go:35-97 and
    run.go:150-188 (adaptDt), FP64.  Knobs as the engine's solver."""

    A = [(1. / 5.,), (3. / 40., 9. / 40.), (44. / 45., -56. / 15., 32. / 9.),
         (19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729.),
         (9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656.)]
    C = (1. / 5., 3. / 10., 4. / 5., 8. / 9., 1.)
    B5 = (35. / 384., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84.)   # k1, k3, k4, k5, k6
    E = (71. / 57600., -71. / 16695., 71. / 1920., -17253. / 339200., 22. / 525., -1. / 40.)  # k1 k3 k4 k5 k6 k7

    def __init__(self, system, m0, dt=1e-15, max_err=1e-5, rel_err=1e-4, min_slope=1e8, min_dt=0.0, max_dt=0.0,
                 headroom=0.8, gamma_ll=1.7595e11):
        self.s = system
        self.m = normalize(torch.as_tensor(np.asarray(m0, np.float64), device=system.dev).reshape(
            (3,) + system.shape))
        self.dt, self.max_err, self.rel_err, self.min_slope = dt, max_err, rel_err, min_slope
        self.min_dt, self.max_dt, self.headroom, self.gamma = min_dt, max_dt, headroom, gamma_ll
        self.time = 0.0
        self.k1 = None
        self.nsteps = self.nundone = self.nevals = 0
        self.last_err = self.peak_err = 0.0

    def _eval(self, m):
        self.nevals += 1
        return self.s.torque(m)

    @staticmethod
    def _corr(num, den, p):
        return math.inf if den == 0 else (num / den) ** p

    def _adapt(self, corr):
        if math.isnan(corr):
            corr = 1.0
        if corr == 0:
            raise RuntimeError("time step correction 0")
        corr *= self.headroom
        corr = min(max(corr, 0.5), 2.0)
        self.dt *= corr
        if self.min_dt != 0 and self.dt < self.min_dt:
            self.dt = self.min_dt
        if self.max_dt != 0 and self.dt > self.max_dt:
            self.dt = self.max_dt

    def step(self):
        """One step attempt; returns True if accepted."""
        if self.k1 is None:
            self.k1 = self._eval(self.m)
        m0, k1 = self.m, self.k1
        h = self.dt * self.gamma
        ks = [k1]
        for i, row in enumerate(self.A):
            acc = m0
            for a, k in zip(row, ks):
                acc = acc + (a * h) * k
            ks.append(self._eval(normalize(acc)))
        k2, k3, k4, k5, k6 = ks[1:]
        acc = m0
        for b, k in zip(self.B5, (k1, k3, k4, k5, k6)):
            acc = acc + (b * h) * k
        m = normalize(acc)
        k7 = self._eval(m)
        Err = sum(e * k for e, k in zip(self.E, (k1, k3, k4, k5, k6, k7)))
        err = float(torch.sqrt((Err * Err).sum(0)).max()) * h
        if err < self.max_err or self.dt <= self.min_dt:
            en = torch.sqrt((Err * Err).sum(0))
            dn = torch.sqrt((k7 * k7).sum(0))
            maxdm = float(dn.max())
            fail = False
            rlerr = 0.0
            if not (maxdm < self.min_slope):
                rlerr = float(torch.where(dn == 0, torch.zeros_like(en), en / dn).abs().max())
                fail = True
            if not fail or self.rel_err <= 0 or rlerr < self.rel_err or self.dt <= self.min_dt:
                self.last_err = err
                self.peak_err = max(self.peak_err, err)
                self.nsteps += 1
                self.time += self.dt
                self._adapt(self._corr(self.max_err, err, 1. / 5.) if not fail else
                            self._corr(self.rel_err, rlerr, 1. / 5.))
                self.m, self.k1 = m, k7
                return True
            self.nundone += 1
            self._adapt(self._corr(self.rel_err, rlerr, 1. / 6.))
            return False
        self.nundone += 1
        self._adapt(self._corr(self.max_err, err, 1. / 6.))
        return False

    def average_m(self):
        return self.m.reshape(3, -1).mean(1).cpu().numpy()
