"""The reference's field + RK45DP path executed on host cores (TEST / BENCH
INFRASTRUCTURE ONLY: the CPU arm that the CUDA path is compared against).

Every per-cell operation is the reference's own OpenCL C kernel compiled for
the host (oracle/_ref/libclref.so, spread over host threads):
copypadmul2 -> FFT -> kernmulRSymm3D -> inverse FFT -> copyunpad
(mag/demag convolution, opencl/conv_*.go), adddmi, adduniaxialanisotropy2,
regionaddv, lltorque2, madd2..madd7 and normalize2.  The reference runs its
FFTs with the vendored VkFFT library on the OpenCL device
(cl/fft_interface.h, opencl/fft3dr2c.go); here scipy.fft's multi-threaded
pocketfft stands in for it.  The stepper restates engine/rk45dp.go:12-98 and
the integral controller of engine/stepcontroller.go:35-97 (the same
restatement as oracle/orc_sim.inc, in numpy).
"""
import os

import numpy as np

from . import clref
from . import oracle as O


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class RefRK45:
    """RK45DP on the multilayer-type system: uniform Ms/alpha/Ku1, region 0
    everywhere, interfacial DMI, uniaxial anisotropy, uniform B_ext, Newell
    demag (kernel from the oracle's FP64 restatement)."""

    def __init__(self, N, cell, Ms, Aex, alpha, Dind, Ku1, anisU, B_ext, threads=None, Kf=None):
        import scipy.fft  # noqa: F401  (fail early when absent)

        if not clref.available():
            raise RuntimeError("oracle/_ref/libclref.so is not built")
        self.threads = threads or host_threads()
        clref.set_threads(self.threads)
        self.N = tuple(N)
        self.cell = [float(np.float32(c)) for c in cell]
        self.cell_f64 = [float(c) for c in cell]
        self.Dind = float(Dind)
        self.alarm = None  # engine/run.go:181-184: a step does not cross the alarm time
        self.n = N[0] * N[1] * N[2]
        self.P = O.pad_size(N)
        if Kf is None:
            Kf, _ = O.kernel_spectrum(O.newell_kernel(N, cell))
        self.Kf = [np.ascontiguousarray(Kf[c], dtype=np.float32) for c in range(6)]
        self.Ms, self.alpha, self.Ku1 = float(Ms), float(alpha), float(Ku1)
        self.anisU = [float(u) for u in anisU]
        self.alut = O.exch_lut(np.full(256, Aex, np.float32))
        self.dlut = O.exch_lut(np.full(256, Dind, np.float32))
        self.regions = np.zeros(self.n, np.uint8)
        self.lut = np.zeros((3, 256), np.float32)
        self.lut[:] = np.asarray(B_ext, np.float32)[:, None]
        shape = (3, N[2], N[1], N[0])
        self.m = np.zeros(shape, np.float32)
        self.k = [np.zeros(shape, np.float32) for _ in range(7)]
        self.m0 = np.zeros(shape, np.float32)
        self.err = np.zeros(shape, np.float32)
        self.pad = np.zeros((self.P[2], self.P[1], self.P[0]), np.float32)
        self.tmp = np.zeros(self.n, np.float32)
        self.tmp2 = np.zeros(self.n, np.float32)
        # solver state (engine/run.go defaults)
        self.dt, self.time = 1e-15, 0.0
        self.max_err, self.rel_err, self.min_slope, self.headroom = 1e-5, 1e-4, 1e8, 0.8
        self.gamma_ll = 1.7595e11
        self.have_k1 = False
        self.nsteps = self.nundone = 0

    def set_m(self, m):
        self.m[:] = m
        self.have_k1 = False

    # ---------------------------------------------------------------- field
    def torque(self, out, m):
        import scipy.fft as F

        N, P = self.N, self.P
        spec = []
        for c in range(3):
            self.pad[:] = 0
            clref.call("copypadmul2", np.float32, self.pad, P[0], P[1], P[2], m[c], N[0], N[1], N[2], None,
                       self.Ms, None)
            spec.append(np.ascontiguousarray(F.rfftn(self.pad, workers=self.threads)))
        sv = [s.view(np.float32) for s in spec]
        clref.call("kernmulRSymm3D", np.float32, sv[0], sv[1], sv[2], *self.Kf, P[0] // 2 + 1, P[1], P[2])
        scale = float(P[0] * P[1] * P[2])
        for c in range(3):
            full = F.irfftn(spec[c], s=(P[2], P[1], P[0]), axes=(0, 1, 2), workers=self.threads)
            full = np.ascontiguousarray(full * np.float32(scale), dtype=np.float32)
            clref.call("copyunpad", np.float32, out[c], N[0], N[1], N[2], full, P[0], P[1], P[2])
        c = self.cell
        if self.Dind != 0:  # engine/exchange.go:49-66: exchange + DMI, or exchange alone
            clref.call("adddmi", np.float32, out[0], out[1], out[2], m[0], m[1], m[2], None, self.Ms, self.alut,
                       self.dlut, self.regions, c[0], c[1], c[2], N[0], N[1], N[2], 0, 0)
        else:
            w = [float(np.float32(2.0 / (x * x))) for x in self.cell_f64]
            clref.call("addexchange", np.float32, out[0], out[1], out[2], m[0], m[1], m[2], None, self.Ms,
                       self.alut, self.regions, w[0], w[1], w[2], N[0], N[1], N[2], 0)
        u = self.anisU
        if self.Ku1 != 0:  # engine/anisotropy.go:40: only with a non-zero constant
            clref.call("adduniaxialanisotropy2", np.float32, out[0], out[1], out[2], m[0], m[1], m[2], None,
                       self.Ms, None, self.Ku1, None, 0.0, None, u[0], None, u[1], None, u[2], self.n)
        clref.call("regionaddv", np.float32, out[0], out[1], out[2], self.lut[0], self.lut[1], self.lut[2],
                   self.regions, self.n)
        clref.call("lltorque2", np.float32, out[0], out[1], out[2], m[0], m[1], m[2], out[0], out[1], out[2],
                   None, self.alpha, self.n)

    # ---------------------------------------------------------------- stepper
    def _madd(self, dst, srcs, fs):
        for c in range(3):
            args = []
            for s, f in zip(srcs, fs):
                args += [s[c], float(np.float32(f))]
            clref.call(f"madd{len(srcs)}", np.float32, dst[c], *args, self.n)

    def _normalize(self, v):
        clref.call("normalize2", np.float32, v[0], v[1], v[2], None, self.n)

    def _maxnorm(self, v):
        clref.call("vecnorm", np.float32, self.tmp, v[0].ravel(), v[1].ravel(), v[2].ravel(), self.n)
        return float(self.tmp.max())

    def _adapt(self, corr):
        if np.isnan(corr):
            corr = 1.0
        corr = min(max(corr * self.headroom, 0.5), 2.0)
        self.dt *= corr
        if self.alarm is not None and self.time < self.alarm and self.time + self.dt > self.alarm:
            self.dt = self.alarm - self.time

    def step(self):
        """One RK45DP attempt (engine/rk45dp.go:12-98); returns True if accepted."""
        m, k, m0 = self.m, self.k, self.m0
        if not self.have_k1:
            self.torque(k[0], m)
            self.have_k1 = True
        t0 = self.time
        m0[:] = m
        h = np.float32(self.dt * self.gamma_ll)
        ch = lambda c: np.float32(c) * h  # noqa: E731
        tab = [
            ([m, k[0]], [1, ch(1 / 5)]),
            ([m0, k[0], k[1]], [1, ch(3 / 40), ch(9 / 40)]),
            ([m0, k[0], k[1], k[2]], [1, ch(44 / 45), ch(-56 / 15), ch(32 / 9)]),
            ([m0, k[0], k[1], k[2], k[3]], [1, ch(19372 / 6561), ch(-25360 / 2187), ch(64448 / 6561),
                                            ch(-212 / 729)]),
            ([m0, k[0], k[1], k[2], k[3], k[4]], [1, ch(9017 / 3168), ch(-355 / 33), ch(46732 / 5247),
                                                  ch(49 / 176), ch(-5103 / 18656)]),
            ([m0, k[0], k[2], k[3], k[4], k[5]], [1, ch(35 / 384), ch(500 / 1113), ch(125 / 192),
                                                  ch(-2187 / 6784), ch(11 / 84)]),
        ]
        outs = [k[1], k[2], k[3], k[4], k[5], k[6]]
        for (srcs, fs), kout in zip(tab, outs):
            self._madd(m, srcs, fs)
            self._normalize(m)
            self.torque(kout, m)
        self._madd(self.err, [k[0], k[2], k[3], k[4], k[5], k[6]],
                   [71 / 57600, -71 / 16695, 71 / 1920, -17253 / 339200, 22 / 525, -1 / 40])
        err = self._maxnorm(self.err) * float(h)
        if err < self.max_err:
            maxdm = self._maxnorm(k[6])
            ok, corr = True, (self.max_err / err) ** (1 / 5) if err > 0 else 2.0
            if not (maxdm < self.min_slope):
                clref.call("vecnorm", np.float32, self.tmp2, k[6][0].ravel(), k[6][1].ravel(), k[6][2].ravel(),
                           self.n)
                clref.call("vecnorm", np.float32, self.tmp, self.err[0].ravel(), self.err[1].ravel(),
                           self.err[2].ravel(), self.n)
                clref.call("pointwise_div", np.float32, self.tmp, self.tmp, self.tmp2, self.n)
                rlerr = float(np.abs(self.tmp).max())
                ok = rlerr < self.rel_err
                corr = (self.rel_err / rlerr) ** (1 / (5 if ok else 6)) if rlerr > 0 else 2.0
            if ok:
                self.nsteps += 1
                self.time = t0 + self.dt
                self._adapt(corr)
                k[0], k[6] = k[6], k[0]  # FSAL
                return True
        else:
            corr = (self.max_err / err) ** (1 / 6)
        self.time = t0
        m[:] = m0
        self.nundone += 1
        self._adapt(corr)
        return False
