"""Engine-level API: one simulation whose effective field, torque and time
stepping run on the device (libumagnus_b200.so, umag_sim_*).

Mirrors the reference's engine globals and functions used on the hot path:
SetEffectiveField / SetTorque (engine/effectivefield.go, engine/torque.go),
the Stepper interface and SetSolver (engine/run.go:69-125), Run / Steps
(engine/run.go:190-200), m.average() (engine/average.go) and the solver
knobs MaxErr, RelErr, MinDt, MaxDt, FixDt, Headroom (engine/run.go:14-43).
Parameters follow engine/parameter.go: a scalar is a uniform value, a
tensor a per-cell map; exchange and DMI are per-region values expanded into
the symmetric inter-region LUT exactly as engine/exchange.go:153-201 does.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import EnsInstance, SimParams, SolverParams, SolverState, Tuning, UmagError, check

NREGION = 256  # engine/regions.go:11
GAMMA_LL = 1.7595e11  # engine/torque.go:27
EULER, HEUN, BOGAKISHAMPINE, RUNGEKUTTA, DORMANDPRINCE = 1, 2, 3, 4, 5  # engine/run.go:83-95


def symmidx(i, j):
    """engine/exchange.go:181-187"""
    return i * (i + 1) // 2 + j if j <= i else j * (j + 1) // 2 + i


def exch_average(exi, exj):
    """engine/exchange.go:193-201 (float32 arithmetic)."""
    exi, exj = np.float32(exi), np.float32(exj)
    if exi * exj >= 0:
        with np.errstate(divide="ignore"):
            return np.float32(2) / (np.float32(1) / exi + np.float32(1) / exj)
    a, b = float(exi), float(exj)
    sign = np.copysign(1.0, a + b)
    return np.float32(sign * np.sqrt(np.sqrt(-a * b) * abs(a + b) / 2))


def exchange_lut(values, scale=None, inter=None):
    """engine/exchange.go:153-167: lut[symidx(i,j)] = scale*avg(ex_i, ex_j) + inter."""
    ex = np.zeros(NREGION, np.float32)
    v = np.asarray(values, np.float32).ravel()
    ex[: v.size] = v
    if v.size == 1:
        ex[:] = v[0]
    lut = np.zeros(NREGION * (NREGION + 1) // 2, np.float32)
    a = ex[:, None]
    b = ex[None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        same = (a * b) >= 0
        harm = np.float32(2) / (np.float32(1) / a + np.float32(1) / b)
    I, J = np.tril_indices(NREGION)
    vals = np.where(same[I, J], harm[I, J], 0).astype(np.float32)
    for k in np.nonzero(~same[I, J])[0]:
        vals[k] = exch_average(ex[I[k]], ex[J[k]])
    idx = I * (I + 1) // 2 + J
    sc = np.ones(lut.size, np.float32) if scale is None else np.asarray(scale, np.float32)
    it = np.zeros(lut.size, np.float32) if inter is None else np.asarray(inter, np.float32)
    lut[idx] = sc[idx] * vals + it[idx]
    return lut


def pair_tables(scale=None, inter=None):
    """The scale and inter tables of an inter-region LUT (engine/exchange.go:
    136-148): {(i, j): s} as ScaleExchange / ScaleDind (scale s, inter 0) and
    {(i, j): v} as InterExchange / InterDind (scale 0, inter v); defaults 1
    and 0.  Returns (scale, inter) arrays indexed by symmidx, or (None, None)."""
    if not scale and not inter:
        return None, None
    n = NREGION * (NREGION + 1) // 2
    sc, it = np.ones(n, np.float32), np.zeros(n, np.float32)
    for (i, j), v in (scale or {}).items():
        sc[symmidx(i, j)], it[symmidx(i, j)] = np.float32(v), 0
    for (i, j), v in (inter or {}).items():
        sc[symmidx(i, j)], it[symmidx(i, j)] = 0, np.float32(v)
    return sc, it


def _dev(x, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype).cuda()


def sim_params(keepalive, N, cell, Msat, Aex, alpha, Dind=0.0, Ku1=0.0, Ku2=0.0, anisU=(0.0, 0.0, 1.0), B_ext=None,
               regions=None, geom=None, demag=True, open_bc=False, precess=True, asymptotic_radius=32,
               demag_kernel="newell", demag_accuracy=6.0, FrozenSpins=None, Kc1=0.0, Kc2=0.0, Kc3=0.0,
               anisC1=(1.0, 0.0, 0.0), anisC2=(0.0, 1.0, 0.0), Dbulk=0.0, Temp=0.0, ThermSeed=0, pbc=(0, 0, 0),
               NoDemagSpins=None, exchange_scale=None, exchange_inter=None, dmi_scale=None, dmi_inter=None):
    """The umag_sim_params record of a simulation (the arguments of
    Simulation, which documents them), with its device maps and LUTs
    appended to `keepalive` (they must outlive the simulation).  Returns
    (params, luts): luts names the device LUTs built here (aLUT, dLUT,
    dbLUT, bext, frozen, nodemag) that exist."""
    N = tuple(int(n) for n in N)
    shape = (N[2], N[1], N[0])
    luts = {}
    p = SimParams()
    p.N[:] = N
    p.cell[:] = [float(c) for c in cell]
    p.pbc[:] = tuple(int(x) for x in pbc)  # data/mesh.go PBC repetitions (SetPBC)

    def keep(t):
        keepalive.append(t)
        return t.data_ptr()

    if regions is not None:
        p.regions = keep(_dev(np.asarray(regions, np.uint8).reshape(shape), torch.uint8))
    if geom is not None:
        p.vol = keep(_dev(np.asarray(geom, np.float32).reshape(shape)))

    def param(v):
        if np.isscalar(v):
            return None, float(np.float32(v))
        return keep(_dev(np.asarray(v, np.float32).reshape(shape))), 1.0

    p.Ms, p.Ms_mul = param(Msat)
    p.alpha, p.alpha_mul = param(alpha)
    p.Ku1, p.Ku1_mul = param(Ku1)
    p.Ku2, p.Ku2_mul = param(Ku2)
    u = np.asarray(anisU, np.float64)
    for c in range(3):
        if u.ndim == 1:
            p.anisU[c], p.anisU_mul[c] = None, float(np.float32(u[c]))
        else:
            p.anisU[c], p.anisU_mul[c] = param(u[c])
    # cubic anisotropy (engine/anisotropy.go:14-19)
    p.Kc1, p.Kc1_mul = param(Kc1)
    p.Kc2, p.Kc2_mul = param(Kc2)
    p.Kc3, p.Kc3_mul = param(Kc3)
    for name, val in (("anisC1", anisC1), ("anisC2", anisC2)):
        v = np.asarray(val, np.float64)
        ptrs, muls = getattr(p, name), getattr(p, name + "_mul")
        for c in range(3):
            if v.ndim == 1:
                ptrs[c], muls[c] = None, float(np.float32(v[c]))
            else:
                ptrs[c], muls[c] = param(v[c])
    luts["aLUT"] = _dev(exchange_lut(Aex, *pair_tables(exchange_scale, exchange_inter)))
    p.aLUT = keep(luts["aLUT"])
    if np.any(np.asarray(Dind) != 0) or dmi_inter:
        luts["dLUT"] = _dev(exchange_lut(Dind, *pair_tables(dmi_scale, dmi_inter)))
        p.dLUT = keep(luts["dLUT"])
    if np.any(np.asarray(Dbulk) != 0):  # engine/exchange.go:60-61 AddDMIBulk
        luts["dbLUT"] = _dev(exchange_lut(Dbulk))
        p.dbulkLUT = keep(luts["dbLUT"])
    if B_ext is not None:
        b = np.asarray(B_ext, np.float32)
        lut = np.tile(b, (NREGION, 1)) if b.ndim == 1 else b
        luts["bext"] = _dev(np.ascontiguousarray(lut.T))
        keep(luts["bext"])
        for c in range(3):
            p.bextLUT[c] = luts["bext"][c].data_ptr()
    p.enable_demag = int(bool(demag))
    p.openbc = int(bool(open_bc))
    p.precess = int(bool(precess))
    p.asymptotic_radius = int(asymptotic_radius)
    # engine/demag.go:21-27: EnableDemag (brute force, the reference default) or EnableNewellDemag
    if demag_kernel not in ("newell", "brute"):
        raise ValueError("demag_kernel must be 'newell' or 'brute'")
    p.demag_kernel = 1 if demag_kernel == "brute" else 0
    p.demag_accuracy = float(demag_accuracy)
    # engine/temperature.go: Temp (K), scalar or per-cell; ThermSeed seeds the noise
    p.temp, p.temp_mul = param(Temp)
    p.therm_seed = int(ThermSeed) & ((1 << 64) - 1)

    def region_lut(val):  # a scalar or up to 256 per-region values
        lut = np.zeros(NREGION, np.float32)
        v = np.asarray(val, np.float32).ravel()
        lut[: v.size] = v
        if v.size == 1:
            lut[:] = v[0]
        return _dev(lut)

    if FrozenSpins is not None:  # engine/torque.go:348-352
        luts["frozen"] = region_lut(FrozenSpins)
        p.frozen_lut = keep(luts["frozen"])
    if NoDemagSpins is not None:  # engine/demag.go:22, :67-98
        luts["nodemag"] = region_lut(NoDemagSpins)
        p.nodemag_lut = keep(luts["nodemag"])
    return p, luts


class Simulation:
    """A micromagnetic simulation on one GPU.

    N: (Nx, Ny, Nz); cell: cell size in m; Msat, alpha, Ku1, Ku2: scalar or
    per-cell (Nz, Ny, Nx) array; Aex, Dind: scalar or 256 per-region values;
    anisU: 3-vector or (3, Nz, Ny, Nx); B_ext: 3-vector (T) or (256, 3)
    per-region; regions: uint8 (Nz, Ny, Nx) map; geom: cell volume fraction;
    demag_kernel: "newell" (EnableNewellDemag) or "brute" (EnableDemag, the
    reference default, with DemagAccuracy = demag_accuracy); FrozenSpins: a
    scalar or 256 per-region values, the torque is zero where non-zero;
    Kc1, Kc2, Kc3, anisC1, anisC2: cubic anisotropy (scalars / 3-vectors or
    per-cell maps); Dbulk: bulk DMI (scalar or 256 per-region values; not
    together with Dind); Temp (K, scalar or per-cell map) with ThermSeed: the
    thermal field, new noise every accepted step; pbc: periodic repetitions
    per axis (engine/mesh.go SetPBC), 0 = open; NoDemagSpins: a scalar or 256
    per-region values, cells of non-zero regions neither make nor feel demag
    field; exchange_scale / exchange_inter ({(i, j): value}): ext_ScaleExchange /
    ext_InterExchange between regions i and j, dmi_scale / dmi_inter the same
    for Dind (engine/exchange.go:84-102).
    """

    def __init__(self, N, cell, Msat, Aex, alpha, Dind=0.0, Ku1=0.0, Ku2=0.0, anisU=(0.0, 0.0, 1.0), B_ext=None,
                 regions=None, geom=None, demag=True, open_bc=False, precess=True, solver=DORMANDPRINCE,
                 dt=1e-15, MaxErr=1e-5, RelErr=1e-4, MinDt=0.0, MaxDt=0.0, FixDt=0.0, Headroom=0.8,
                 device=0, asymptotic_radius=32, demag_kernel="newell", demag_accuracy=6.0, FrozenSpins=None,
                 Kc1=0.0, Kc2=0.0, Kc3=0.0, anisC1=(1.0, 0.0, 0.0), anisC2=(0.0, 1.0, 0.0), Dbulk=0.0,
                 Temp=0.0, ThermSeed=0, pbc=(0, 0, 0), NoDemagSpins=None, exchange_scale=None,
                 exchange_inter=None, dmi_scale=None, dmi_inter=None):
        self.L = _lib.init(device)
        self.N = tuple(int(n) for n in N)
        self.ncell = self.N[0] * self.N[1] * self.N[2]
        self.shape = (self.N[2], self.N[1], self.N[0])
        self._keep = []
        p, luts = sim_params(self._keep, N, cell, Msat, Aex, alpha, Dind=Dind, Ku1=Ku1, Ku2=Ku2, anisU=anisU,
                             B_ext=B_ext, regions=regions, geom=geom, demag=demag, open_bc=open_bc, precess=precess,
                             asymptotic_radius=asymptotic_radius, demag_kernel=demag_kernel,
                             demag_accuracy=demag_accuracy, FrozenSpins=FrozenSpins, Kc1=Kc1, Kc2=Kc2, Kc3=Kc3,
                             anisC1=anisC1, anisC2=anisC2, Dbulk=Dbulk, Temp=Temp, ThermSeed=ThermSeed, pbc=pbc,
                             NoDemagSpins=NoDemagSpins, exchange_scale=exchange_scale,
                             exchange_inter=exchange_inter, dmi_scale=dmi_scale, dmi_inter=dmi_inter)
        for k, v in luts.items():
            setattr(self, k, v)
        sp = SolverParams()
        self.L.umag_solver_defaults(ctypes.byref(sp))
        sp.solver = int(solver)
        sp.dt, sp.max_err, sp.rel_err, sp.min_dt, sp.max_dt = dt, MaxErr, RelErr, MinDt, MaxDt
        sp.fix_dt, sp.headroom, sp.gamma_ll = FixDt, Headroom, GAMMA_LL
        self.params, self.solver = p, sp
        h = ctypes.c_void_p()
        torch.cuda.synchronize()
        check(self.L.umag_sim_new(ctypes.byref(p), ctypes.byref(sp), ctypes.byref(h)))
        self._h = h.value

    # ---------------------------------------------------------------- state
    def set_m(self, m):
        """m = array (3, Nz, Ny, Nx); normalised on the device (engine/magnetization.go:55)."""
        t = _dev(np.asarray(m, np.float32).reshape((3,) + self.shape)) if not torch.is_tensor(m) else m.contiguous()
        torch.cuda.synchronize()
        check(self.L.umag_sim_set_m(self._h, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr()))
        check(self.L.umag_sync())

    def restore_m(self, m):
        """Put back a state read by get_m, without normalising it again
        (checkpoint resume: the trajectory continues bit for bit)."""
        t = m.contiguous()
        torch.cuda.synchronize()
        check(self.L.umag_sim_restore_m(self._h, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr()))

    def m_ptrs(self):
        ptrs = (ctypes.c_void_p * 3)()
        check(self.L.umag_sim_m_ptrs(self._h, ptrs))
        return [ptrs[i] for i in range(3)]

    def get_m(self, out=None):
        """Copy of the current m as a (3, Nz, Ny, Nx) CUDA tensor."""
        if out is None:
            out = torch.empty((3,) + self.shape, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        check(self.L.umag_sim_get_m(self._h, out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr()))
        return out

    def torque(self, beff=False):
        """engine/torque.go:124 SetTorque of the current m (and B_eff if asked)."""
        t = torch.empty((3,) + self.shape, dtype=torch.float32, device="cuda")
        b = torch.empty_like(t) if beff else None
        torch.cuda.synchronize()
        bp = (b[0].data_ptr(), b[1].data_ptr(), b[2].data_ptr()) if beff else (None, None, None)
        check(self.L.umag_sim_torque(self._h, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), *bp))
        return (t, b) if beff else t

    # ---------------------------------------------------------------- stepping
    def steps(self, n):
        """engine/run.go:197 Steps(n) without host synchronisation."""
        check(self.L.umag_sim_steps(self._h, int(n)))

    def run(self, seconds, chunk=64, max_steps=10 ** 12):
        """engine/run.go:190 Run(seconds)."""
        check(self.L.umag_sim_run(self._h, float(seconds), int(chunk), int(max_steps)))

    def sync(self):
        check(self.L.umag_sync())

    def state(self):
        st = SolverState()
        check(self.L.umag_sim_get_state(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in SolverState._fields_}

    def set_time(self, t, dt=0.0):
        check(self.L.umag_sim_set_time(self._h, float(t), float(dt)))

    def average_m(self):
        """engine/average.go:29 (compensated sums)."""
        out = (ctypes.c_double * 3)()
        check(self.L.umag_sim_average_m(self._h, out))
        return [out[0], out[1], out[2]]

    def set_B_ext(self, B_ext):
        """Change the applied field (engine/zeeman.go B_ext = ...): a 3-vector (T)
        or (256, 3) per-region values.  The simulation must have been created
        with a B_ext (possibly zero); the device table is overwritten in place,
        so captured step graphs see the new value."""
        if getattr(self, "bext", None) is None:
            raise UmagError("set_B_ext needs a Simulation created with B_ext")
        b = np.asarray(B_ext, np.float32)
        lut = np.tile(b, (NREGION, 1)) if b.ndim == 1 else b
        torch.cuda.synchronize()
        self.sync()
        self.bext.copy_(torch.from_numpy(np.ascontiguousarray(lut.T)))
        torch.cuda.synchronize()

    _SOLVER_KNOBS = {"FixDt": "fix_dt", "MaxErr": "max_err", "RelErr": "rel_err", "MinDt": "min_dt",
                     "MaxDt": "max_dt", "Headroom": "headroom", "MinSlope": "min_slope", "GammaLL": "gamma_ll"}
    _PARAMS = {"Msat": 0, "alpha": 1, "Ku1": 2, "Ku2": 3, "Temp": 4, "Kc1": 8, "Kc2": 9, "Kc3": 10}
    _VECTORS = {"anisU": 5, "anisC1": 11, "anisC2": 14}

    def set_solver(self, solver=None, **knobs):
        """Script assignments between runs: SetSolver(solver) and FixDt, MaxErr,
        RelErr, MinDt, MaxDt, Headroom, MinSlope, GammaLL (engine/run.go:14-43,
        :92-125).  Time and dt are kept."""
        sp = self.solver
        if solver is not None:
            sp.solver = int(solver)
        for k, v in knobs.items():
            if k not in self._SOLVER_KNOBS:
                raise ValueError(f"unknown solver setting {k!r}")
            setattr(sp, self._SOLVER_KNOBS[k], float(v))
        torch.cuda.synchronize()
        check(self.L.umag_sim_set_solver(self._h, ctypes.byref(sp)))

    def set_param(self, name, value):
        """Reassign a parameter between runs, as `alpha = 0.02` does in a
        script: Msat, alpha, Ku1, Ku2, Temp, Kc1, Kc2, Kc3 (a scalar or a
        (Nz, Ny, Nx) map) or anisU, anisC1, anisC2 (a 3-vector or (3, Nz, Ny, Nx))."""
        if name in self._VECTORS:
            v = value if not np.isscalar(value) else None
            if v is None or len(v) != 3:
                raise ValueError(f"{name} needs 3 components")
            for c in range(3):
                self._set_one(self._VECTORS[name] + c, v[c])
            return
        if name not in self._PARAMS:
            raise ValueError(f"parameter must be one of {sorted(self._PARAMS) + sorted(self._VECTORS)}")
        self._set_one(self._PARAMS[name], value)

    def _set_one(self, which, value):
        if np.isscalar(value):
            t, ptr, mul = None, None, float(np.float32(value))
        else:
            t = _dev(np.asarray(value, np.float32).reshape(self.shape))
            ptr, mul = t.data_ptr(), 1.0
        torch.cuda.synchronize()
        check(self.L.umag_sim_set_param(self._h, which, ptr, mul))
        if t is not None:
            self._keep.append(t)  # the device map stays alive while the simulation may use it

    def energies(self):
        """engine/energy.go:27 GetTotalEnergy and its terms (J) for the current m:
        dict with total, demag, exchange (incl. DMI), anisotropy, zeeman."""
        out = (ctypes.c_double * 5)()
        check(self.L.umag_sim_energies(self._h, out))
        return dict(zip(("total", "demag", "exchange", "anisotropy", "zeeman"), list(out)))

    def energy_density(self, out=None):
        """engine/energy.go:36 SetTotalEdens (Edens_total, J/m^3) for the
        current m, as a (Nz, Ny, Nx) float32 tensor on the device."""
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        check(self.L.umag_sim_energy_density(self._h, out.data_ptr()))
        return out

    def relax(self, torque_threshold=-1.0):
        """engine/relax.go:23 Relax() (RelaxTorqueThreshold = torque_threshold)."""
        check(self.L.umag_sim_relax(self._h, float(torque_threshold)))

    def use_graph(self, enable=True, steps_per_graph=16):
        check(self.L.umag_sim_use_graph(self._h, int(bool(enable)), int(steps_per_graph)))

    def torque_evals(self, n):
        """Enqueue n field + torque evaluations of the current m (timing aid)."""
        check(self.L.umag_sim_torque_evals(self._h, int(n)))

    def set_stream(self, stream):
        """Queue all library work on a torch.cuda.Stream (None = library stream)."""
        check(self.L.umag_set_stream(None if stream is None else stream.cuda_stream))
        self.stream = stream

    def get_tuning(self):
        """Launch shapes of the per-cell kernels (umag_tuning) as a dict."""
        t = Tuning()
        check(self.L.umag_sim_get_tuning(self._h, ctypes.byref(t)))
        return {"torque_block": [t.torque_block[0], t.torque_block[1]], "stage_threads": t.stage_threads,
                "stage_waves": t.stage_waves, "err_waves": t.err_waves, "torque_tma": t.torque_tma}

    def set_tuning(self, tuning):
        """Apply launch shapes (a dict like get_tuning's); results are unchanged."""
        t = Tuning()
        t.torque_block[0], t.torque_block[1] = (int(v) for v in tuning["torque_block"])
        t.stage_threads, t.stage_waves, t.err_waves = (int(tuning[k]) for k in ("stage_threads", "stage_waves",
                                                                                "err_waves"))
        t.torque_tma = int(tuning.get("torque_tma", 1))
        torch.cuda.synchronize()
        check(self.L.umag_sim_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, cache_path=None, use_cache=True):
        """Choose the fastest launch shapes for this mesh on this GPU
        (umagnus_b200.autotune.tune); returns (tuning, timings or None)."""
        from . import autotune
        return autotune.tune(self, cache_path=cache_path, use_cache=use_cache)

    def launches_per_step(self):
        n = ctypes.c_int()
        check(self.L.umag_sim_launches_per_step(self._h, ctypes.byref(n)))
        return n.value

    def free(self):
        if getattr(self, "_h", None):
            self.L.umag_sim_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Ensemble:
    """Many independent simulations advanced together on one GPU (no
    counterpart in the reference, which runs one simulation per process).

    instances: list of dicts with N, cell, Msat, Aex, alpha and optional
    Dind, Ku1, Ku2, anisU, B_ext.  Each instance keeps its own time, dt and
    step controller; the solver knobs are shared.  Instances with uniform
    values of those parameters and the same mesh run as one batch of
    launches, and one CUDA graph steps all of them.  An instance whose dict
    holds anything else -- region maps, per-cell or per-region parameter
    arrays, geom, pbc, Temp, FrozenSpins, any other Simulation argument -- or
    "general": True is a general instance: the simulation Simulation(**dict)
    would be, stepped by the single-simulation kernels in a graph of its own,
    concurrently with the batches, with the same trajectory bit for bit
    (umag_ens_new_general).
    """

    UNIFORM_KEYS = {"N", "cell", "Msat", "Aex", "alpha", "Dind", "Ku1", "Ku2", "anisU", "B_ext"}

    @classmethod
    def is_general(cls, d):
        if d.get("general", False) or set(d) - cls.UNIFORM_KEYS - {"general"}:
            return True
        scal = ("Msat", "Aex", "alpha", "Dind", "Ku1", "Ku2")
        if any(np.ndim(d[k]) != 0 for k in scal if k in d):
            return True
        return any(np.ndim(d[k]) > 1 for k in ("anisU", "B_ext") if k in d)

    def __init__(self, instances, demag=True, solver=DORMANDPRINCE, dt=1e-15, MaxErr=1e-5, RelErr=1e-4,
                 MinDt=0.0, MaxDt=0.0, FixDt=0.0, Headroom=0.8, device=0):
        self.L = _lib.init(device)
        arr = (EnsInstance * len(instances))()
        gen = (ctypes.c_void_p * len(instances))()
        self._keep = []
        self._gen_params = []
        self.shapes = []
        for k, d in enumerate(instances):
            if self.is_general(d):
                kw = {key: v for key, v in d.items() if key != "general"}
                kw.setdefault("demag", demag)
                p, _ = sim_params(self._keep, **kw)
                self._gen_params.append(p)
                gen[k] = ctypes.addressof(p)
                N = tuple(int(n) for n in d["N"])
                self.shapes.append((3, N[2], N[1], N[0]))
                continue
            r = arr[k]
            N = tuple(int(n) for n in d["N"])
            r.N[:] = N
            r.cell[:] = [float(c) for c in d["cell"]]
            r.Ms, r.Aex, r.alpha = float(d["Msat"]), float(d["Aex"]), float(d["alpha"])
            r.Dind, r.Ku1, r.Ku2 = float(d.get("Dind", 0.0)), float(d.get("Ku1", 0.0)), float(d.get("Ku2", 0.0))
            r.anisU[:] = [float(u) for u in d.get("anisU", (0.0, 0.0, 1.0))]
            r.B_ext[:] = [float(b) for b in d.get("B_ext", (0.0, 0.0, 0.0))]
            self.shapes.append((3, N[2], N[1], N[0]))
        sp = SolverParams()
        self.L.umag_solver_defaults(ctypes.byref(sp))
        sp.solver = int(solver)
        sp.dt, sp.max_err, sp.rel_err, sp.min_dt, sp.max_dt = dt, MaxErr, RelErr, MinDt, MaxDt
        sp.fix_dt, sp.headroom, sp.gamma_ll = FixDt, Headroom, GAMMA_LL
        h = ctypes.c_void_p()
        torch.cuda.synchronize()  # the general instances' device maps are in place
        check(self.L.umag_ens_new_general(len(instances), arr, gen, ctypes.byref(sp), int(bool(demag)),
                                          ctypes.byref(h)))
        self._h = h.value

    def __len__(self):
        return len(self.shapes)

    def classes(self):
        n, c = ctypes.c_int(), ctypes.c_int()
        check(self.L.umag_ens_count(self._h, ctypes.byref(n), ctypes.byref(c)))
        return c.value

    def class_info(self, cls):
        """(mesh N, number of instances) of class `cls` (classes numbered in
        the order their first instance appears)."""
        N = (ctypes.c_int * 3)()
        n = ctypes.c_int()
        check(self.L.umag_ens_class_info(self._h, int(cls), N, ctypes.byref(n)))
        return tuple(N), n.value

    def class_general(self, cls):
        """True when class `cls` is a general instance (one simulation with
        the single-simulation kernels)."""
        g = ctypes.c_int()
        check(self.L.umag_ens_class_general(self._h, int(cls), ctypes.byref(g)))
        return bool(g.value)

    def get_tuning(self, cls):
        """Launch shapes of class `cls`'s batched per-cell kernels (a dict)."""
        t = Tuning()
        check(self.L.umag_ens_get_tuning(self._h, int(cls), ctypes.byref(t)))
        return {"torque_block": [t.torque_block[0], t.torque_block[1]], "stage_threads": t.stage_threads,
                "stage_waves": t.stage_waves, "err_waves": t.err_waves, "torque_tma": t.torque_tma}

    def set_tuning(self, cls, tuning):
        """Apply launch shapes to class `cls` (speed only; results unchanged)."""
        t = Tuning()
        t.torque_block[0], t.torque_block[1] = (int(v) for v in tuning["torque_block"])
        t.stage_threads, t.stage_waves, t.err_waves = (int(tuning[k]) for k in ("stage_threads", "stage_waves",
                                                                                "err_waves"))
        t.torque_tma = int(tuning.get("torque_tma", 0))
        torch.cuda.synchronize()
        check(self.L.umag_ens_set_tuning(self._h, int(cls), ctypes.byref(t)))

    def autotune(self, instances, cache_path=None, use_cache=True):
        """Launch shapes of every class from umagnus_b200.autotune.tune_ensemble
        (`instances`: the list this ensemble was made from)."""
        from . import autotune
        return autotune.tune_ensemble(self, instances, cache_path=cache_path, use_cache=use_cache)

    def set_m(self, i, m):
        a = np.ascontiguousarray(np.asarray(m, np.float32).reshape(self.shapes[i]))
        check(self.L.umag_ens_set_m(self._h, int(i), a.ctypes.data))

    def get_m(self, i):
        a = np.empty(self.shapes[i], np.float32)
        check(self.L.umag_ens_get_m(self._h, int(i), a.ctypes.data))
        return a

    def state(self, i):
        st = SolverState()
        check(self.L.umag_ens_get_state(self._h, int(i), ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in SolverState._fields_}

    def run(self, seconds, chunk=8, max_replays=10 ** 12):
        """engine/run.go:190 Run(seconds) for every instance."""
        check(self.L.umag_ens_run(self._h, float(seconds), int(chunk), int(max_replays)))

    def free(self):
        if getattr(self, "_h", None):
            self.L.umag_ens_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
