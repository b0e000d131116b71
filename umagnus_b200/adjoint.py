"""Differentiable fixed-step RK4 or Heun simulation on the device (umag_adj_*).

No counterpart in the reference, which has no gradients.  The forward pass
is the engine's effective field (demag, exchange, uniaxial anisotropy,
Zeeman; engine/effectivefield.go:14-24) and LL torque (engine/torque.go)
for a per-cell Ms map and uniform Aex, Ku1, B_ext and alpha (and a fixed
uniform interfacial DMI, Dind), on an open or periodic mesh (pbc) with an
optional geometry (geom: cell volume fractions), stepped
by fixed-step RK4 (engine/rk4.go with FixDt) or Heun (engine/heun.go,
solver=2), m checkpointed every K steps.
The loss is

    w_probe * mean over states avg_from..nsteps of the mean m_z in the probe
    window (layer 0) + w_target * |<m>(final) - target|^2

and `backward` returns its gradient with respect to the Ms map, Aex, Ku1,
B_ext and m0 by hand-written vector-Jacobian products (CUDA kernels),
recomputing each K-step segment from its checkpoint.

`AdjointRK4.loss` wraps the pair as a torch.autograd.Function so that the
simulation can sit inside a torch optimisation loop.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import AdjParams, check

GAMMA_LL = 1.7595e11  # engine/torque.go:27


class AdjointRK4:
    def __init__(self, N, cell, alpha, anisU, dt, nsteps, K, probe, avg_from, w_probe=1.0, w_target=1.0,
                 target=(0.0, 0.0, 1.0), demag=True, demag_kernel="newell", demag_accuracy=6.0, gamma_ll=GAMMA_LL,
                 use_graph=True, device=0, solver=4, Dind=0.0, pbc=(0, 0, 0), geom=None, regions=None):
        self.L = _lib.init(device)
        p = AdjParams()
        p.N[:] = [int(n) for n in N]
        p.cell[:] = [float(c) for c in cell]
        p.alpha = float(alpha)
        p.anisU[:] = [float(u) for u in anisU]
        p.enable_demag = int(bool(demag))
        p.demag_kernel = {"newell": 0, "brute": 1}[demag_kernel]
        p.demag_accuracy = float(demag_accuracy)
        p.dt, p.gamma_ll = float(dt), float(gamma_ll)
        p.nsteps, p.K = int(nsteps), int(K)
        p.probe[:] = [int(v) for v in probe]
        p.avg_from = int(avg_from)
        p.w_probe, p.w_target = float(w_probe), float(w_target)
        p.target[:] = [float(t) for t in target]
        p.no_graph = 0 if use_graph else 1
        p.solver = int(solver)  # 4 RK4, 2 Heun
        p.Dind = float(Dind)    # interfacial DMI (fixed parameter)
        p.pbc[:] = [int(v) for v in pbc]  # periodic repetitions per axis (engine/mesh.go SetPBC)
        self._vol = None
        if geom is not None:  # cell volume fractions (engine/geom.go), kept on the device
            g = torch.as_tensor(np.asarray(geom, np.float32)).reshape(-1)
            self._vol = g.to(torch.device("cuda", device)).contiguous()
            torch.cuda.synchronize()
            p.vol = self._vol.data_ptr()
        # a region map: Aex, Ku1 and B_ext become per-region arrays in
        # forward() and backward() (regions 0 .. max of the map)
        self._reg, self.nregions = None, 0
        if regions is not None:
            r = np.asarray(regions).astype(np.uint8).reshape(-1)
            self.nregions = int(r.max()) + 1
            self._reg = torch.as_tensor(r).to(torch.device("cuda", device)).contiguous()
            torch.cuda.synchronize()
            p.regions = self._reg.data_ptr()
            p.nregions = self.nregions
        self.N = tuple(int(n) for n in N)
        self.ncell = self.N[0] * self.N[1] * self.N[2]
        h = ctypes.c_void_p()
        check(self.L.umag_adj_new(ctypes.byref(p), ctypes.byref(h)))
        self._h = h.value
        self.device = torch.device("cuda", device)

    def _dev(self, x, n):
        t = torch.as_tensor(x, dtype=torch.float32, device=self.device).contiguous()
        if t.numel() != n:
            raise ValueError(f"expected {n} values, got {t.numel()}")
        return t

    def forward(self, m0, Ms, Aex, Ku1, B_ext):
        """Run the forward pass; returns the loss (float).  m0 (3, Nz, Ny, Nx)
        and Ms (Nz, Ny, Nx) as arrays or tensors; with a region map Aex and
        Ku1 are per-region sequences and B_ext is (regions, 3)."""
        self._m0 = self._dev(m0, 3 * self.ncell)
        self._Ms = self._dev(Ms, self.ncell)
        loss = ctypes.c_double()
        torch.cuda.synchronize(self.device)
        if self._reg is not None:
            nr = self.nregions
            A = np.asarray(Aex, np.float32).reshape(nr)
            K = np.asarray(Ku1, np.float32).reshape(nr)
            B = np.ascontiguousarray(np.asarray(B_ext, np.float32).reshape(nr, 3))
            fp = ctypes.POINTER(ctypes.c_float)
            check(self.L.umag_adj_forward_regions(self._h, self._m0.data_ptr(), self._Ms.data_ptr(),
                                                  A.ctypes.data_as(fp), K.ctypes.data_as(fp), B.ctypes.data_as(fp),
                                                  ctypes.byref(loss)))
            return loss.value
        b = (ctypes.c_float * 3)(*[float(v) for v in B_ext])
        check(self.L.umag_adj_forward(self._h, self._m0.data_ptr(), self._Ms.data_ptr(), float(Aex), float(Ku1), b,
                                      ctypes.byref(loss)))
        return loss.value

    def final_m(self):
        out = torch.empty((3,) + self.N[::-1], dtype=torch.float32, device=self.device)
        check(self.L.umag_adj_final_m(self._h, out.data_ptr()))
        return out

    def backward(self, want_m0=True):
        """Gradients of the last forward's loss: dict with Ms (tensor),
        Aex, Ku1 (floats), B_ext (3 floats) and m0 (tensor, if asked)."""
        gMs = torch.empty(self.N[::-1], dtype=torch.float32, device=self.device)
        gm0 = torch.empty((3,) + self.N[::-1], dtype=torch.float32, device=self.device) if want_m0 else None
        if self._reg is not None:  # per-region arrays
            nr = self.nregions
            gA, gK, gB = np.zeros(nr), np.zeros(nr), np.zeros((nr, 3))
            dp = ctypes.POINTER(ctypes.c_double)
            check(self.L.umag_adj_backward_regions(self._h, gMs.data_ptr(), gm0.data_ptr() if want_m0 else None,
                                                   gA.ctypes.data_as(dp), gK.ctypes.data_as(dp),
                                                   gB.ctypes.data_as(dp)))
            out = {"Ms": gMs, "Aex": gA, "Ku1": gK, "B_ext": gB}
            if want_m0:
                out["m0"] = gm0
            return out
        gA, gK = ctypes.c_double(), ctypes.c_double()
        gB = (ctypes.c_double * 3)()
        check(self.L.umag_adj_backward(self._h, gMs.data_ptr(), gm0.data_ptr() if want_m0 else None,
                                       ctypes.byref(gA), ctypes.byref(gK), gB))
        out = {"Ms": gMs, "Aex": gA.value, "Ku1": gK.value, "B_ext": list(gB)}
        if want_m0:
            out["m0"] = gm0
        return out

    def loss(self, m0, Ms, Aex, Ku1, B_ext):
        """The loss as a differentiable torch scalar (float64) of tensors m0,
        Ms, Aex, Ku1, B_ext."""
        return _AdjFn.apply(self, m0, Ms, Aex, Ku1, B_ext)

    def free(self):
        if getattr(self, "_h", None):
            check(self.L.umag_adj_free(self._h))
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class AdjointHeun(AdjointRK4):
    """The same differentiable simulation stepped by fixed-step Heun
    (engine/heun.go: predictor m + h k0 unnormalised, result normalised)."""

    def __init__(self, *args, **kw):
        kw["solver"] = 2
        super().__init__(*args, **kw)


class _AdjFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sim, m0, Ms, Aex, Ku1, B_ext):
        ctx.sim = sim
        ctx.shapes = (m0.shape, Ms.shape)
        ctx.devs = (m0.device, Ms.device, torch.as_tensor(Aex).device, torch.as_tensor(Ku1).device,
                    torch.as_tensor(B_ext).device)
        if sim.nregions:  # per-region parameters
            host = lambda t: torch.as_tensor(t).detach().cpu().numpy()
            loss = sim.forward(m0.detach(), Ms.detach(), host(Aex), host(Ku1), host(B_ext))
        else:
            loss = sim.forward(m0.detach(), Ms.detach(), float(Aex), float(Ku1),
                               [float(v) for v in torch.as_tensor(B_ext).detach().cpu()])
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gl):
        g = ctx.sim.backward(want_m0=ctx.needs_input_grad[1])
        s = float(gl)
        d = ctx.devs
        gm0 = (g["m0"] * s).reshape(ctx.shapes[0]).to(d[0]) if ctx.needs_input_grad[1] else None
        gMs = (g["Ms"] * s).reshape(ctx.shapes[1]).to(d[1])
        gA = torch.tensor(np.asarray(g["Aex"]) * s, dtype=torch.float64, device=d[2])
        gK = torch.tensor(np.asarray(g["Ku1"]) * s, dtype=torch.float64, device=d[3])
        gB = torch.tensor(np.asarray(g["B_ext"]) * s, dtype=torch.float64, device=d[4])
        return None, gm0, gMs, gA, gK, gB
