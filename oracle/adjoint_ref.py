"""FP64 CPU restatement of the differentiable fixed-step simulation (RK4 or
Heun) and its adjoint.

TEST INFRASTRUCTURE ONLY: tests/ and bench.py import this module to check
the GPU adjoint (umag_adj_*); the product never does.

The model is the engine's effective field and LL torque for uniform region
0 (engine/effectivefield.go:14-24, engine/demag.go, engine/exchange.go,
engine/anisotropy.go, engine/zeeman.go, engine/torque.go:135-144) with a
per-cell Ms map, exchange or (Dind != 0) exchange + interfacial DMI
(kernels_src/cl/dmi.cl:8-148 with its Neumann extrapolation of missing
in-plane neighbours, uniform A and D), stepped by fixed-step RK4 (engine/rk4.go:35-61, every stage
normalised, opencl normalize2.cl) or Heun (engine/heun.go:27-43: the
predictor m + h k0 is not normalised, the result is).  The reference has no gradients; this
module gives the FP64 gradient two ways: a hand-written reverse pass (the
same vector-Jacobian products as the GPU adjoint, in FP64) and central
finite differences of the FP64 forward, so that the two can pin each other.

Arrays are (3, Nz, Ny, Nx) for vectors and (Nz, Ny, Nx) for Ms.
"""
import numpy as np

from . import oracle

MU0 = 4 * np.pi * 1e-7  # kernels_src/clh/constants.clh:5
GAMMA_LL = 1.7595e11    # engine/torque.go:27


class _Numpy:
    """Array operations of the restatement in numpy (FP64, host)."""

    def asarray(self, x):
        return np.asarray(x, np.float64)

    def zeros(self, shape):
        return np.zeros(shape)

    def zeros_like(self, x):
        return np.zeros_like(x)

    def cross(self, a, b):
        return np.cross(a, b, axis=0)

    def rfftn(self, x):
        return np.fft.rfftn(x, axes=(1, 2, 3))

    def irfftn(self, x, s):
        return np.fft.irfftn(x, s=s, axes=(1, 2, 3))

    def stack(self, xs):
        return np.stack(xs)

    def take(self, v, idx, axis):
        return np.take(v, idx, axis=axis)

    def index(self, idx):
        return idx

    def col(self, u):  # a 3-vector as a (3, 1, 1, 1) field
        return np.asarray(u, np.float64)[:, None, None, None]

    def scalar(self, x):
        return float(x)

    def host(self, x):
        return x

    def sqrt(self, x):
        return np.sqrt(x)

    def numel(self, x):
        return x.size


class _Torch:
    """The same operations in torch float64 on a device (CUDA for the
    benchmark's FP64 gradient check: thousands of steps in seconds)."""

    def __init__(self, device):
        import torch
        self.t = torch
        self.dev = torch.device(device)

    def asarray(self, x):
        return self.t.as_tensor(np.asarray(x, np.float64) if not isinstance(x, self.t.Tensor) else x,
                                dtype=self.t.float64, device=self.dev)

    def zeros(self, shape):
        return self.t.zeros(shape, dtype=self.t.float64, device=self.dev)

    def zeros_like(self, x):
        return self.t.zeros_like(x)

    def cross(self, a, b):
        return self.t.linalg.cross(a, b, dim=0)

    def rfftn(self, x):
        return self.t.fft.rfftn(x, dim=(1, 2, 3))

    def irfftn(self, x, s):
        return self.t.fft.irfftn(x, s=tuple(s), dim=(1, 2, 3))

    def stack(self, xs):
        return self.t.stack(xs)

    def take(self, v, idx, axis):
        return self.t.index_select(v, axis, idx)

    def index(self, idx):
        return self.t.as_tensor(idx, device=self.dev)

    def col(self, u):
        return self.asarray(u).reshape(3, 1, 1, 1)

    def scalar(self, x):
        return float(x)

    def host(self, x):
        return x.cpu().numpy() if isinstance(x, self.t.Tensor) else x

    def sqrt(self, x):
        return self.t.sqrt(x)

    def numel(self, x):
        return x.numel()


class Problem:
    """Static part of the problem: mesh, demag kernel, stepper, loss."""

    def __init__(self, N, cell, alpha, anisU, dt, nsteps, probe, avg_from, w_probe=1.0, w_target=1.0,
                 target=(0.0, 0.0, 1.0), demag=True, gamma_ll=GAMMA_LL, solver=4, backend="numpy", device="cuda",
                 Dind=0.0, pbc=(0, 0, 0), geom=None, regions=None):
        """backend: "numpy" (host) or "torch" (float64 on `device`), the same
        operations in the same order.  Dind: uniform interfacial DMI (J/m^2),
        a fixed (not differentiated) parameter.  pbc: periodic repetitions
        per axis (data/mesh.go): the demag kernel sums the images
        (mag/demagkernel.go) and the stencils wrap (stencil.clh:13-29).
        geom: cell volume fractions (Nz, Ny, Nx) or None (engine/geom.go):
        m is zero where geom is 0 (normalize2.cl), the demag source is
        Ms * geom * m (copypadmul2.cl), and a neighbour outside the geometry
        is a missing neighbour of the stencils (exchange.cl, dmi.cl: a zero
        m).  regions: a region map (Nz, Ny, Nx) of small integers or None;
        with it the parameters A, K1 are per-region arrays and B a
        (regions, 3) array, the exchange coefficient of a cell pair is the
        harmonic mean of its regions' A (engine/exchange.go:153-167), and
        the gradients come per region (no interfacial DMI with regions)."""
        if solver not in (2, 4):
            raise ValueError("solver must be 4 (RK4) or 2 (Heun)")
        self.xp = _Numpy() if backend == "numpy" else _Torch(device)
        self.solver = int(solver)
        self.N = tuple(int(n) for n in N)
        self.cell = tuple(float(c) for c in cell)
        self.alpha = float(alpha)
        u = np.asarray(anisU, np.float64)
        u = u / np.linalg.norm(u) if np.linalg.norm(u) > 0 else u
        self.u = u
        self.ucol = self.xp.col(u)
        self.h = dt * gamma_ll
        self.nsteps = int(nsteps)
        self.probe = tuple(int(p) for p in probe)
        self.avg_from = int(avg_from)
        self.w_probe, self.w_target = float(w_probe), float(w_target)
        self.target = self.xp.asarray(target)
        self.gilb = -1.0 / (1.0 + self.alpha ** 2)
        self.w = [2.0 / (c * c) for c in self.cell]
        self.D = float(Dind)
        self.pbc = tuple(int(p) for p in pbc)
        shape = (self.N[2], self.N[1], self.N[0])
        if regions is None:
            self.reg = None
        else:
            if float(Dind) != 0:
                raise ValueError("region maps with interfacial DMI are not supported here")
            self.reg = np.asarray(regions).astype(np.int64).reshape(shape)
            self.nreg = int(self.reg.max()) + 1
        if geom is None:
            self.vol, self.inside = None, None
        else:
            g = np.asarray(geom, np.float64).reshape(shape)
            self.vol = self.xp.asarray(g)
            self.inside = self.xp.asarray((g != 0).astype(np.float64))  # cells of the geometry
        # periodic flag per array axis of (3, Nz, Ny, Nx) fields
        self.per = {3: self.pbc[0] > 0, 2: self.pbc[1] > 0, 1: self.pbc[2] > 0}
        if self.D != 0:
            # in-plane neighbour masks (1 where the neighbour exists) along x and y
            Nx, Ny, Nz = self.N
            self.ins = {}
            for ax, n in ((3, Nx), (2, Ny)):
                for sd in (-1, 1):
                    idx = np.arange(n) + sd
                    shape = [1, 1, 1, 1]
                    shape[ax] = n
                    has = np.ones(n, bool) if self.per[ax] else (idx >= 0) & (idx < n)
                    self.ins[(ax, sd)] = self.xp.asarray(has.astype(np.float64).reshape(shape))
                    if self.inside is not None:  # and the neighbour is in the geometry
                        nbin = self.xp.take(self.inside[None], self.xp.index(self._nb(ax, n, sd)), ax)
                        self.ins[(ax, sd)] = self.ins[(ax, sd)] * nbin
        self.demag = demag
        if demag:
            K = oracle.newell_kernel(self.N, self.cell, pbc=self.pbc)  # (6, Pz, Py, Px): xx yy zz yz xz xy
            self.P = K.shape[1:]
            self.Kf = self.xp.rfftn(self.xp.asarray(K))

    # ------------------------------------------------------------ field
    def demag_field(self, v):
        """mu0 * K * v (v already scaled by Ms and the geometry), zero-padded
        convolution."""
        Nx, Ny, Nz = self.N
        Pz, Py, Px = self.P
        xp = self.xp
        V = xp.zeros((3, Pz, Py, Px))
        V[:, :Nz, :Ny, :Nx] = v
        F = xp.rfftn(V)
        xx, yy, zz, yz, xz, xy = self.Kf
        Bf = xp.stack([xx * F[0] + xy * F[1] + xz * F[2],
                       xy * F[0] + yy * F[1] + yz * F[2],
                       xz * F[0] + yz * F[1] + zz * F[2]])
        B = xp.irfftn(Bf, (Pz, Py, Px))
        return MU0 * B[:, :Nz, :Ny, :Nx]

    def _nb(self, ax, n, sd):
        """neighbour index along array axis ax: clamped (stencil.clh hclamp /
        lclamp) or wrapped on a periodic axis"""
        idx = np.arange(n) + sd
        return idx % n if self.per[ax] else np.clip(idx, 0, n - 1)

    def _present(self, ax, n, sd):
        """1 where the neighbour along array axis ax is in the geometry (a
        neighbour outside it has m = 0, which the stencils treat as missing:
        its term vanishes), or None without a geometry"""
        if self.inside is None:
            return None
        return self.xp.take(self.inside[None], self.xp.index(self._nb(ax, n, sd)), ax)

    def stencil(self, v):
        """sum_d w_d (v_neighbour - v) with clamped or wrapped neighbours
        (exchange.cl), over the neighbours in the geometry and zero at cells
        outside it; symmetric."""
        xp = self.xp
        out = xp.zeros_like(v)
        Nz = v.shape[1]
        axes = [(3, self.w[0]), (2, self.w[1])] + ([(1, self.w[2])] if Nz > 1 else [])
        for ax, w in axes:
            n = v.shape[ax]
            for sd in (-1, 1):
                nb = xp.take(v, xp.index(self._nb(ax, n, sd)), ax)
                pr = self._present(ax, n, sd)
                out += w * (nb - v) if pr is None else w * pr * (nb - v)
        return out if self.inside is None else self.inside[None] * out

    def _zstencil(self, v):
        """sum over z neighbours of (v_nb - v), clamped or wrapped, over the
        neighbours in the geometry (exchange.cl z terms)."""
        xp = self.xp
        out = xp.zeros_like(v)
        n = v.shape[1]
        if n > 1:
            for sd in (-1, 1):
                nb = xp.take(v, xp.index(self._nb(1, n, sd)), 1)
                pr = self._present(1, n, sd)
                out += (nb - v) if pr is None else pr * (nb - v)
        return out

    def dmi(self, m, A):
        """dmi.cl:8-148 (exchange + interfacial DMI, uniform A and D, no
        holes, not OpenBC) in FP64, the reference's operations: for each
        in-plane side a neighbour outside the mesh is extrapolated from m0
        (dmi.cl:46-50, 67-71, 89-93, 110-114), then 2A/c^2 (mn - m0) and the
        D/c terms; z neighbours add exchange only.  Linear in m, and (with a
        geometry-based rather than value-based test for missing neighbours)
        its own transpose, which the reverse pass uses."""
        xp = self.xp
        D = self.D
        h = xp.zeros_like(m)
        for ax, c, d in ((3, self.cell[0], 0), (2, self.cell[1], 1)):
            n = m.shape[ax]
            for sd in (-1, 1):
                mn = xp.take(m, xp.index(self._nb(ax, n, sd)), ax)
                ins = self.ins[(ax, sd)]
                q = sd * c * (0.5 * D / A)
                if d == 0:
                    ext = xp.stack([m[0] - q * m[2], m[1], m[2] + q * m[0]])
                else:
                    ext = xp.stack([m[0], m[1] - q * m[2], m[2] + q * m[1]])
                mn = ins * mn + (1.0 - ins) * ext
                h += (2.0 * A / (c * c)) * (mn - m)
                Dc = D / c
                h[d] += Dc * sd * mn[2]
                h[2] -= Dc * sd * mn[d]
        h = h + (2.0 * A / (self.cell[2] ** 2)) * self._zstencil(m)
        return h if self.inside is None else self.inside[None] * h

    def dmi_dA(self, m, A):
        """d dmi(m, A) / dA: the exchange terms over A, and -D^2/(2A^2) times
        the boundary cells' (m0x, 0, m0z) (x sides) / (0, m0y, m0z) (y sides),
        which is what the extrapolated neighbour contributes (D^2/(2A) m0)."""
        xp = self.xp
        D = self.D
        g = xp.zeros_like(m)
        for ax, c, d in ((3, self.cell[0], 0), (2, self.cell[1], 1)):
            n = m.shape[ax]
            for sd in (-1, 1):
                mn = xp.take(m, xp.index(self._nb(ax, n, sd)), ax)
                ins = self.ins[(ax, sd)]
                g += (2.0 / (c * c)) * ins * (mn - m)
                bd = (1.0 - ins) * (-(D * D) / (2.0 * A * A))
                g[d] += bd[0] * m[d]
                g[2] += bd[0] * m[2]
        g = g + (2.0 / (self.cell[2] ** 2)) * self._zstencil(m)
        return g if self.inside is None else self.inside[None] * g

    # ------------------------------------------------------------ regions
    def _pair(self, A, ax, n, sd):
        """exchange coefficient of each cell with its neighbour along array
        axis ax: the harmonic mean of the two regions' A, and its derivative
        with respect to the cell's own region's A (A_i^2 / ... = a^2/(2 A_i^2))"""
        A = np.asarray(A, np.float64)
        ri = self.reg
        rj = np.take(self.reg[None], self._nb(ax, n, sd), ax)[0]
        Ai, Aj = A[ri], A[rj]
        a = 2.0 / (1.0 / Ai + 1.0 / Aj)
        return self.xp.asarray(a), self.xp.asarray(a * a / (2.0 * Ai * Ai))

    def _stencil_r(self, v, A, dA=False):
        """the exchange stencil with per-pair coefficients (sum_d w_d a_ij
        (v_j - v_i)); dA: with the derivatives w.r.t. the cell's region's A
        instead of the coefficients"""
        xp = self.xp
        out = xp.zeros_like(v)
        Nz = v.shape[1]
        axes = [(3, self.w[0]), (2, self.w[1])] + ([(1, self.w[2])] if Nz > 1 else [])
        for ax, w in axes:
            n = v.shape[ax]
            for sd in (-1, 1):
                nb = xp.take(v, xp.index(self._nb(ax, n, sd)), ax)
                a, da = self._pair(A, ax, n, sd)
                c = (da if dA else a)[None]
                pr = self._present(ax, n, sd)
                out += w * c * (nb - v) if pr is None else w * c * pr * (nb - v)
        return out if self.inside is None else self.inside[None] * out

    def _pair_grad(self, m, x, A):
        """dL/dA per region: at each cell i, sum over its neighbours j of
        (c_ij + c_ji) da_ij/dA_i, c_ij = w_d x_i.(m_j - m_i) (the field
        cotangent over Ms); every pair is seen from both cells, so each side
        takes the derivative with respect to its own region's A"""
        xp = self.xp
        g = xp.zeros_like(m[0])
        Nz = m.shape[1]
        axes = [(3, self.w[0]), (2, self.w[1])] + ([(1, self.w[2])] if Nz > 1 else [])
        for ax, w in axes:
            n = m.shape[ax]
            for sd in (-1, 1):
                idx = xp.index(self._nb(ax, n, sd))
                mj, xj = xp.take(m, idx, ax), xp.take(x, idx, ax)
                _, da = self._pair(A, ax, n, sd)
                c = (x * (mj - m)).sum(0) + (xj * (m - mj)).sum(0)
                pr = self._present(ax, n, sd)
                g += w * da * c if pr is None else w * da * pr[0] * c
        if self.inside is not None:
            g = g * self.inside
        return self._bin(g)

    def _rmap(self, vals):
        """a per-region value (or 3-vector) as a field"""
        v = np.asarray(vals, np.float64)
        return self.xp.asarray(v[self.reg] if v.ndim == 1 else np.moveaxis(v[self.reg], -1, 0))

    def field(self, m, th):
        Ms, A, K1, Bext = th["Ms"], th["A"], th["K1"], th["B"]
        src = Ms * m if self.vol is None else Ms * self.vol * m
        B = self.demag_field(src) if self.demag else self.xp.zeros_like(m)
        if self.reg is not None:
            B = B + self._stencil_r(m, A) / Ms
            mu = (m * self.ucol).sum(0)
            B = B + (2 * self._rmap(K1) / Ms * mu)[None] * self.ucol
            return B + self._rmap(Bext)
        B = B + (self.dmi(m, A) if self.D != 0 else A * self.stencil(m)) / Ms
        if K1 != 0:
            mu = (m * self.ucol).sum(0)
            B = B + (2 * K1 / Ms * mu)[None] * self.ucol
        return B + self.xp.col(Bext)

    def torque(self, m, B):
        mxB = self.xp.cross(m, B)
        return self.gilb * (mxB + self.alpha * self.xp.cross(m, mxB))

    def normalize(self, v):
        if self.inside is None:
            return v / self.xp.sqrt((v * v).sum(0))[None]
        ln = self.xp.sqrt((v * v).sum(0))
        ln = ln + (1.0 - self.inside)  # no division by zero outside the geometry
        return self.inside[None] * v / ln[None]

    def step(self, m, th, keep=False):
        h = self.h
        if self.solver == 2:  # engine/heun.go:30-43 with FixDt
            B0 = self.field(m, th)
            k0 = self.torque(m, B0)
            y1 = m + h * k0
            B1 = self.field(y1, th)
            k1 = self.torque(y1, B1)
            out = self.normalize(y1 + 0.5 * h * k1 - 0.5 * h * k0)
            return (out, [m, y1], [B0, B1], [k0, k1]) if keep else out
        ms, Bs, ks = [m], [], []
        for q in range(4):
            B = self.field(ms[q], th)
            k = self.torque(ms[q], B)
            Bs.append(B)
            ks.append(k)
            if q < 3:
                c = (0.5, 0.5, 1.0)[q]
                ms.append(self.normalize(m + c * h * k))
        out = self.normalize(m + h / 6 * ks[0] + h / 3 * ks[1] + h / 3 * ks[2] + h / 6 * ks[3])
        return (out, ms, Bs, ks) if keep else out

    # ------------------------------------------------------------ loss
    def probe_mean(self, m):
        x0, y0, w, h = self.probe
        return m[2, 0, y0:y0 + h, x0:x0 + w].mean()

    def forward(self, m0, th, keep=False):
        th = self._params(th)
        m = self.normalize(self.xp.asarray(m0))
        states = [m]
        acc = 0.0
        for n in range(1, self.nsteps + 1):
            m = self.step(m, th)
            if keep:
                states.append(m)
            if n >= self.avg_from:
                acc += self.probe_mean(m)
        navg = self.nsteps - self.avg_from + 1
        avg = m.reshape(3, -1).mean(1)
        loss = self.xp.scalar(self.w_probe * acc / navg + self.w_target * ((avg - self.target) ** 2).sum())
        return (loss, states) if keep else loss

    def _params(self, th):
        """th on this backend (Ms a field, B a 3-vector, A and K1 floats)."""
        xp = self.xp
        if self.reg is not None:  # per-region arrays (host)
            return {"Ms": xp.asarray(th["Ms"]), "A": np.asarray(th["A"], np.float64),
                    "K1": np.asarray(th["K1"], np.float64), "B": np.asarray(th["B"], np.float64)}
        return {"Ms": xp.asarray(th["Ms"]), "A": float(th["A"]), "K1": float(th["K1"]), "B": xp.asarray(th["B"])}

    # ------------------------------------------------------------ adjoint
    def _loss_grad(self, m, with_probe, with_avg):
        g = self.xp.zeros_like(m)
        x0, y0, w, h = self.probe
        navg = self.nsteps - self.avg_from + 1
        if with_probe:
            g[2, 0, y0:y0 + h, x0:x0 + w] += self.w_probe / (navg * w * h)
        if with_avg:
            avg = m.reshape(3, -1).mean(1)
            g += (2 * self.w_target * (avg - self.target) / self.xp.numel(m[0]))[:, None, None, None]
        return g

    def _norm_vjp(self, u, w):
        ln = self.xp.sqrt((u * u).sum(0))[None]
        if self.inside is not None:
            ln = ln + (1.0 - self.inside[None])
        n = u / ln
        g = (w - n * (n * w).sum(0)[None]) / ln
        return g if self.inside is None else self.inside[None] * g

    def _bin(self, f):
        """sum of a per-cell field over each region (host)"""
        return np.bincount(self.reg.ravel(), weights=self.xp.host(f).ravel(), minlength=self.nreg)

    def _field_vjp(self, m, wB, th, grads):
        Ms, A, K1 = th["Ms"], th["A"], th["K1"]
        gm = self.xp.zeros_like(m)
        if self.demag:
            dw = self.demag_field(wB)
            if self.vol is not None:
                dw = self.vol[None] * dw
            gm += Ms * dw
            grads["Ms"] += (m * dw).sum(0)
        if self.reg is not None:
            # exchange: the per-pair operator is symmetric; dL/dA_r collects,
            # at each cell of region r, (c_ij + c_ji) da_ij/dA_i over its
            # neighbours, c_ij = w_d (wB_i/Ms_i).(m_j - m_i)
            x = wB / Ms
            e = self._stencil_r(m, A)
            gm += self._stencil_r(x, A)
            grads["Ms"] -= (wB * e).sum(0) / Ms ** 2
            grads["A"] += self._pair_grad(m, x, A)
            mu = (m * self.ucol).sum(0)
            wu = (wB * self.ucol).sum(0)
            K1c = self._rmap(K1)
            gm += (2 * K1c / Ms * wu)[None] * self.ucol
            grads["Ms"] -= 2 * K1c * mu * wu / Ms ** 2
            grads["K1"] += self._bin(2 * mu * wu / Ms)
            grads["B"] += np.stack([self._bin(wB[c]) for c in range(3)], axis=1)
            return gm
        if self.D != 0:
            h = self.dmi(m, A)
            gm += self.dmi(wB / Ms, A)  # the operator is symmetric
            grads["Ms"] -= (wB * h).sum(0) / Ms ** 2
            grads["A"] += ((wB * self.dmi_dA(m, A)).sum(0) / Ms).sum()
        else:
            e = self.stencil(m)
            gm += A * self.stencil(wB / Ms)
            we = (wB * e).sum(0)
            grads["Ms"] -= A * we / Ms ** 2
            grads["A"] += (we / Ms).sum()
        if K1 != 0:
            mu = (m * self.ucol).sum(0)
            wu = (wB * self.ucol).sum(0)
            gm += (2 * K1 / Ms * wu)[None] * self.ucol
            grads["Ms"] -= 2 * K1 * mu * wu / Ms ** 2
            grads["K1"] += (2 * mu * wu / Ms).sum()
        grads["B"] += wB.reshape(3, -1).sum(1)
        return gm

    def _torque_vjp(self, m, B, w):
        g = self.gilb
        a = self.alpha
        cross = self.xp.cross
        mxB = cross(m, B)
        wxm = cross(w, m)
        gm = g * (cross(B, w) + a * (cross(mxB, w) + cross(B, wxm)))
        wB = g * (wxm + a * cross(wxm, m))
        return gm, wB

    def _heun_step_vjp(self, m, ms, Bs, ks, lam, th, grads):
        """dL/dm of one Heun step out = normalize(y1 + h/2 k1 - h/2 k0), y1 =
        m + h k0, k_q = torque(state_q, field(state_q)), given dL/dout."""
        h = self.h
        y1 = ms[1]
        gz = self._norm_vjp(y1 + 0.5 * h * ks[1] - 0.5 * h * ks[0], lam)
        gk0 = -0.5 * h * gz
        gm1, wB = self._torque_vjp(y1, Bs[1], 0.5 * h * gz)
        ly1 = gz + gm1 + self._field_vjp(y1, wB, th, grads)  # dL/dy1
        gk0 = gk0 + h * ly1
        gm0, wB = self._torque_vjp(m, Bs[0], gk0)
        return ly1 + gm0 + self._field_vjp(m, wB, th, grads)

    def backward(self, m0, th):
        """Gradient of forward(m0, th) by the reverse pass (all states kept)."""
        th = self._params(th)
        loss, states = self.forward(m0, th, keep=True)
        xp = self.xp
        if self.reg is not None:
            grads = {"Ms": xp.zeros_like(th["Ms"]), "A": np.zeros(self.nreg), "K1": np.zeros(self.nreg),
                     "B": np.zeros((self.nreg, 3))}
        else:
            grads = {"Ms": xp.zeros_like(th["Ms"]), "A": 0.0, "K1": 0.0, "B": xp.zeros((3,))}
        h = self.h
        lam = self._loss_grad(states[-1], self.nsteps >= self.avg_from, True)
        fin = (h / 6, h / 3, h / 3, h / 6)
        stc = (0.5 * h, 0.5 * h, 1.0 * h)
        for n in range(self.nsteps, 0, -1):
            m = states[n - 1]
            _, ms, Bs, ks = self.step(m, th, keep=True)
            if self.solver == 2:
                lam = self._heun_step_vjp(m, ms, Bs, ks, lam, th, grads)
                if n - 1 >= self.avg_from:
                    lam = lam + self._loss_grad(states[n - 1], True, False)
                continue
            u = m + sum(f * k for f, k in zip(fin, ks))
            gu = self._norm_vjp(u, lam)
            lam2 = gu + 0.0
            gk = [f * gu for f in fin]
            for q in range(3, -1, -1):
                gmq, wB = self._torque_vjp(ms[q], Bs[q], gk[q])
                gmq = gmq + self._field_vjp(ms[q], wB, th, grads)
                if q > 0:
                    gu = self._norm_vjp(m + stc[q - 1] * ks[q - 1], gmq)
                    lam2 += gu
                    gk[q - 1] = gk[q - 1] + stc[q - 1] * gu
                else:
                    lam2 += gmq
            lam = lam2
            if n - 1 >= self.avg_from:
                lam = lam + self._loss_grad(states[n - 1], True, False)
        grads["m0"] = self._norm_vjp(xp.asarray(m0), lam)
        if self.reg is not None:
            grads = {k: (v if isinstance(v, np.ndarray) else xp.host(v)) for k, v in grads.items()}
        else:
            grads = {k: (float(v) if k in ("A", "K1") else xp.host(v)) for k, v in grads.items()}
        return loss, grads


def params(Ms, A, K1, B):
    """the parameter record: scalars A, K1 and a 3-vector B, or per-region
    arrays (A[r], K1[r], B[r, c]) for a problem with a region map"""
    def sc(v):
        return float(v) if np.ndim(v) == 0 else np.asarray(v, np.float64)
    return {"Ms": np.asarray(Ms, np.float64), "A": sc(A), "K1": sc(K1), "B": np.asarray(B, np.float64)}


def fd_gradient(prob, m0, th, which, rel=1e-4):
    """Central finite differences of the FP64 loss with relative step rel.

    which: ("Ms", (z, y, x)), ("A", None), ("K1", None) or ("B", c), or
    with a region map ("A", r), ("K1", r), ("B", (r, c)); for a
    zero-valued parameter the step is rel (absolute)."""
    name, idx = which

    def with_value(v):
        t = {k: (np.array(x, copy=True) if isinstance(x, np.ndarray) else x) for k, x in th.items()}
        if idx is None:
            t[name] = v
        else:
            t[name][idx] = v
        return t

    x0 = th[name] if idx is None else th[name][idx]
    d = rel * abs(x0) if x0 != 0 else rel
    return (prob.forward(m0, with_value(x0 + d)) - prob.forward(m0, with_value(x0 - d))) / (2 * d)
