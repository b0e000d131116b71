"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  The oracle is a plain-C restatement of the uMagNUS
hot path (see umag_oracle.h for the file:line citations).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference leg import this
module; the product (umagnus_b200) never does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

f32p = ctypes.POINTER(ctypes.c_float)
f64p = ctypes.POINTER(ctypes.c_double)
u8p = ctypes.POINTER(ctypes.c_uint8)
ip = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile liboracle.so from the C sources in this directory."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class OrcSystem(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int * 3), ("pbc", ctypes.c_int * 3), ("cell", ctypes.c_double * 3),
        ("Ms", ctypes.c_void_p), ("alpha", ctypes.c_void_p), ("Ku1", ctypes.c_void_p),
        ("Ku2", ctypes.c_void_p), ("u", ctypes.c_void_p * 3), ("vol", ctypes.c_void_p),
        ("Ms_mul", ctypes.c_double), ("alpha_mul", ctypes.c_double), ("Ku1_mul", ctypes.c_double),
        ("Ku2_mul", ctypes.c_double), ("u_mul", ctypes.c_double * 3),
        ("aLUT", ctypes.c_void_p), ("dLUT", ctypes.c_void_p), ("regions", u8p),
        ("bext_lut", ctypes.c_void_p * 3),
        ("enable_demag", ctypes.c_int), ("dmi", ctypes.c_int), ("openbc", ctypes.c_int),
        ("precess", ctypes.c_int), ("anis", ctypes.c_int),
        ("Kf", f64p * 6), ("P", ctypes.c_int * 3),
        ("Kc1", ctypes.c_void_p), ("Kc2", ctypes.c_void_p), ("Kc3", ctypes.c_void_p),
        ("c1", ctypes.c_void_p * 3), ("c2", ctypes.c_void_p * 3),
        ("Kc1_mul", ctypes.c_double), ("Kc2_mul", ctypes.c_double), ("Kc3_mul", ctypes.c_double),
        ("c1_mul", ctypes.c_double * 3), ("c2_mul", ctypes.c_double * 3),
        ("cubic", ctypes.c_int), ("dbLUT", ctypes.c_void_p),
        ("nodemag", ctypes.c_void_p), ("frozen", ctypes.c_void_p),
    ]


class OrcSolver(ctypes.Structure):
    _fields_ = [
        ("time", ctypes.c_double), ("dt", ctypes.c_double), ("alarm", ctypes.c_double),
        ("max_err", ctypes.c_double), ("rel_err", ctypes.c_double), ("min_dt", ctypes.c_double),
        ("max_dt", ctypes.c_double), ("fix_dt", ctypes.c_double), ("headroom", ctypes.c_double),
        ("min_slope", ctypes.c_double), ("gamma_ll", ctypes.c_double),
        ("last_err", ctypes.c_double), ("peak_err", ctypes.c_double), ("last_torque", ctypes.c_double),
        ("nsteps", ctypes.c_long), ("nundone", ctypes.c_long), ("nevals", ctypes.c_long),
        ("solver", ctypes.c_int), ("have_k1", ctypes.c_int), ("status", ctypes.c_int),
    ]


def _declare(L):
    L.orc_pad_size.argtypes = [ip, ip, ip]
    L.orc_newell_kernel.argtypes = [ip, ip, f64p, ctypes.c_int, ctypes.c_int, f64p * 6]
    L.orc_brute_kernel.argtypes = [ip, ip, f64p, ctypes.c_double, ctypes.POINTER(ctypes.c_float) * 6]
    L.orc_newell_f.restype = ctypes.c_double
    L.orc_newell_g.restype = ctypes.c_double
    L.orc_self_demag_nx.restype = ctypes.c_double
    for f in (L.orc_newell_f, L.orc_newell_g, L.orc_self_demag_nx):
        f.argtypes = [ctypes.c_double] * 3
    L.orc_kernel_spectrum.argtypes = [ip, f64p * 6, ctypes.c_int, f64p * 6]
    L.orc_kernel_spectrum.restype = ctypes.c_double
    L.orc_fft_line.argtypes = [f64p, ctypes.c_int, ctypes.c_int]
    L.orc_solver_defaults.argtypes = [ctypes.POINTER(OrcSolver)]
    for s in ("f32", "f64"):
        for name in ("orc_max_vec_norm", "orc_max_vec_diff", "orc_max_abs", "orc_sum", "orc_dot"):
            getattr(L, f"{name}_{s}").restype = ctypes.c_double
        getattr(L, f"orc_step_{s}").restype = ctypes.c_int


def _ptr(a):
    if a is None:
        return None
    if a.dtype == np.float32:
        return a.ctypes.data_as(f32p)
    if a.dtype == np.float64:
        return a.ctypes.data_as(f64p)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(u8p)
    raise TypeError(a.dtype)


def _vp(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _arr3(arrs):
    """Three component arrays -> C array of 3 pointers."""
    t = arrs[0].dtype
    P = f32p if t == np.float32 else f64p
    return (P * 3)(*[_ptr(a) for a in arrs])


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


# ---------------------------------------------------------------- geometry
def pad_size(size, pbc=(0, 0, 0)):
    out = (ctypes.c_int * 3)()
    lib().orc_pad_size((ctypes.c_int * 3)(*size), (ctypes.c_int * 3)(*pbc), out)
    return tuple(out)


def newell_kernel(size, cellsize, pbc=(0, 0, 0), asymptotic_radius=32, zero_self_demag=0):
    """Real-space Newell tensor, components (xx, yy, zz, yz, xz, xy), shape (6, Pz, Py, Px)."""
    P = pad_size(size, pbc)
    K = np.zeros((6, P[2], P[1], P[0]), dtype=np.float64)
    ptrs = (f64p * 6)(*[K[c].ctypes.data_as(f64p) for c in range(6)])
    lib().orc_newell_kernel((ctypes.c_int * 3)(*size), (ctypes.c_int * 3)(*pbc),
                            (ctypes.c_double * 3)(*cellsize), asymptotic_radius, zero_self_demag, ptrs)
    return K


def brute_kernel(size, cellsize, pbc=(0, 0, 0), accuracy=6.0):
    """mag/demagkernel.go:113 CalcDemagKernel (engine/demag.go:25 DemagAccuracy = 6):
    float32 real-space kernel (xx, yy, zz, yz, xz, xy), shape (6, Pz, Py, Px)."""
    P = pad_size(size, pbc)
    K = np.zeros((6, P[2], P[1], P[0]), dtype=np.float32)
    f32p = ctypes.POINTER(ctypes.c_float)
    ptrs = (f32p * 6)(*[K[c].ctypes.data_as(f32p) for c in range(6)])
    lib().orc_brute_kernel((ctypes.c_int * 3)(*size), (ctypes.c_int * 3)(*pbc), (ctypes.c_double * 3)(*cellsize),
                           float(accuracy), ptrs)
    return K


def kernel_spectrum(K, round_f32=False):
    """(6, Pz/2+1, Py/2+1, Px/2+1) real spectrum scaled by 1/(PxPyPz); also returns max imag."""
    _, Pz, Py, Px = K.shape
    K = np.ascontiguousarray(K, dtype=np.float64)
    Kf = np.zeros((6, Pz // 2 + 1, Py // 2 + 1, Px // 2 + 1), dtype=np.float64)
    kin = (f64p * 6)(*[K[c].ctypes.data_as(f64p) for c in range(6)])
    kout = (f64p * 6)(*[Kf[c].ctypes.data_as(f64p) for c in range(6)])
    mi = lib().orc_kernel_spectrum((ctypes.c_int * 3)(Px, Py, Pz), kin, 1 if round_f32 else 0, kout)
    return Kf, mi


def newell_f(x, y, z):
    return lib().orc_newell_f(x, y, z)


def newell_g(x, y, z):
    return lib().orc_newell_g(x, y, z)


def self_demag_nx(x, y, z):
    return lib().orc_self_demag_nx(x, y, z)


def fft(x, sign=-1):
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().orc_fft_line(a.ctypes.data_as(f64p), a.size, sign)
    return a


# ---------------------------------------------------------------- per-cell kernels
def _sfx(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def demag_field(Kf, P, m, Ms, vol=None, dtype=np.float32):
    """Demag field of m (shape (3, Nz, Ny, Nx)); Ms scalar or per-cell array."""
    m = _c(m, dtype)
    N = (m.shape[3], m.shape[2], m.shape[1])
    B = np.zeros_like(m)
    Kf = np.ascontiguousarray(Kf)
    kp = (f64p * 6)(*[Kf[c].ctypes.data_as(f64p) for c in range(6)])
    ms_arr, ms_mul = (None, float(Ms)) if np.isscalar(Ms) else (_c(Ms, dtype), 1.0)
    vol = None if vol is None else _c(vol, dtype)
    fn = getattr(lib(), f"orc_demag_{_sfx(dtype)}")
    scal = ctypes.c_float if np.dtype(dtype) == np.float32 else ctypes.c_double
    fn((ctypes.c_int * 3)(*N), (ctypes.c_int * 3)(*P), kp, _arr3(list(B)), _arr3(list(m)),
       _ptr(vol), _ptr(ms_arr), scal(ms_mul))
    return B


def _scal(dtype):
    return ctypes.c_float if np.dtype(dtype) == np.float32 else ctypes.c_double


def add_exchange(B, m, aLUT, regions, cell, Ms, pbc=0):
    dt = B.dtype
    S = _scal(dt)
    Nz, Ny, Nx = m.shape[1:]
    ms_arr, ms_mul = (None, float(Ms)) if np.isscalar(Ms) else (_c(Ms, dt), 1.0)
    w = [dt.type(2.0 / (c * c)) for c in cell]
    getattr(lib(), f"orc_add_exchange_{_sfx(dt)}")(
        _arr3(list(B)), _arr3(list(m)), _ptr(ms_arr), S(ms_mul), _ptr(_c(aLUT, dt)), _ptr(_c(regions, np.uint8)),
        S(w[0]), S(w[1]), S(w[2]), Nx, Ny, Nz, pbc)


def add_dmi(B, m, aLUT, dLUT, regions, cell, Ms, pbc=0, openbc=0):
    dt = B.dtype
    S = _scal(dt)
    Nz, Ny, Nx = m.shape[1:]
    ms_arr, ms_mul = (None, float(Ms)) if np.isscalar(Ms) else (_c(Ms, dt), 1.0)
    getattr(lib(), f"orc_add_dmi_{_sfx(dt)}")(
        _arr3(list(B)), _arr3(list(m)), _ptr(ms_arr), S(ms_mul), _ptr(_c(aLUT, dt)), _ptr(_c(dLUT, dt)),
        _ptr(_c(regions, np.uint8)), S(cell[0]), S(cell[1]), S(cell[2]), Nx, Ny, Nz, pbc, openbc)


def add_uniaxial(B, m, Ms, K1, K2, u):
    """Ms/K1/K2 scalar or per-cell arrays; u a 3-vector or (3, ...) array."""
    dt = B.dtype
    S = _scal(dt)
    n = m[0].size

    def ms(v):
        return (None, float(v)) if np.isscalar(v) else (_c(v, dt).ravel(), 1.0)

    Msa, Msm = ms(Ms)
    K1a, K1m = ms(K1)
    K2a, K2m = ms(K2)
    if np.asarray(u).ndim == 1:
        ua = [None, None, None]
        um = [float(x) for x in u]
    else:
        ua = [_c(u[c], dt).ravel() for c in range(3)]
        um = [1.0, 1.0, 1.0]
    P = f32p if dt == np.float32 else f64p
    uarr = (P * 3)(*[_ptr(a) for a in ua])
    umul = (S * 3)(*um)
    getattr(lib(), f"orc_add_uniaxial2_{_sfx(dt)}")(
        _arr3(list(B)), _arr3(list(m)), _ptr(Msa), S(Msm), _ptr(K1a), S(K1m), _ptr(K2a), S(K2m),
        uarr, umul, n)


def add_cubic(B, m, Ms, K1, K2, K3, c1, c2):
    """kernels_src/cl/cubicanisotropy2.cl; Ms/K1/K2/K3 scalar or per-cell
    arrays, c1/c2 3-vectors or (3, ...) arrays."""
    dt = B.dtype
    S = _scal(dt)
    n = m[0].size
    P = f32p if dt == np.float32 else f64p

    def ms(v):
        return (None, float(v)) if np.isscalar(v) else (_c(v, dt).ravel(), 1.0)

    def vec(u):
        if np.asarray(u).ndim == 1:
            return (P * 3)(None, None, None), (S * 3)(*[float(x) for x in u]), []
        arrs = [_c(u[c], dt).ravel() for c in range(3)]
        return (P * 3)(*[_ptr(a) for a in arrs]), (S * 3)(1.0, 1.0, 1.0), arrs

    Msa, Msm = ms(Ms)
    K1a, K1m = ms(K1)
    K2a, K2m = ms(K2)
    K3a, K3m = ms(K3)
    c1p, c1m, keep1 = vec(c1)
    c2p, c2m, keep2 = vec(c2)
    getattr(lib(), f"orc_add_cubic2_{_sfx(dt)}")(
        _arr3(list(B)), _arr3(list(m)), _ptr(Msa), S(Msm), _ptr(K1a), S(K1m), _ptr(K2a), S(K2m), _ptr(K3a), S(K3m),
        c1p, c1m, c2p, c2m, n)


def add_dmibulk(B, m, aLUT, dLUT, regions, cell, Ms, pbc=0, openbc=0):
    """kernels_src/cl/dmibulk.cl: exchange + bulk DMI."""
    dt = B.dtype
    S = _scal(dt)
    Nz, Ny, Nx = m.shape[1:]
    ms_arr, ms_mul = (None, float(Ms)) if np.isscalar(Ms) else (_c(Ms, dt), 1.0)
    getattr(lib(), f"orc_add_dmibulk_{_sfx(dt)}")(
        _arr3(list(B)), _arr3(list(m)), _ptr(ms_arr), S(ms_mul), _ptr(_c(aLUT, dt)), _ptr(_c(dLUT, dt)),
        _ptr(_c(regions, np.uint8)), S(cell[0]), S(cell[1]), S(cell[2]), Nx, Ny, Nz, pbc, openbc)


def set_temperature(B, noise, k2, Ms, temp, alpha):
    """kernels_src/cl/temperature2.cl (one component); Ms/temp/alpha scalar or arrays."""
    dt = B.dtype
    S = _scal(dt)

    def ms(v):
        return (None, float(v)) if np.isscalar(v) else (_c(v, dt).ravel(), 1.0)

    Msa, Msm = ms(Ms)
    ta, tm = ms(temp)
    aa, am = ms(alpha)
    getattr(lib(), f"orc_set_temperature_{_sfx(dt)}")(
        _ptr(B), _ptr(_c(noise, dt)), S(k2), _ptr(Msa), S(Msm), _ptr(ta), S(tm), _ptr(aa), S(am), B.size)


M0_PHILOX, M1_PHILOX = 0xD2511F53, 0xCD9E8D57
W0_PHILOX, W1_PHILOX = 0x9E3779B9, 0xBB67AE85


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 (Salmon et al., SC'11) on uint64 arrays holding 32-bit words."""
    m32 = np.uint64(0xFFFFFFFF)
    c = [np.asarray(x, np.uint64) & m32 for x in (c0, c1, c2, c3)]
    k0, k1 = int(k0) & 0xFFFFFFFF, int(k1) & 0xFFFFFFFF
    for r in range(10):
        if r:
            k0 = (k0 + W0_PHILOX) & 0xFFFFFFFF
            k1 = (k1 + W1_PHILOX) & 0xFFFFFFFF
        p0 = np.uint64(M0_PHILOX) * c[0]
        p1 = np.uint64(M1_PHILOX) * c[2]
        c = [(p1 >> np.uint64(32)) ^ c[1] ^ np.uint64(k0), p1 & m32, (p0 >> np.uint64(32)) ^ c[3] ^ np.uint64(k1),
             p0 & m32]
    return c


def thermal_normals(seed, step, n):
    """The three standard normals per cell of the device's thermal noise
    (umag_thermal_noise): Philox4x32-10 of (cell, step lo, step hi, 0) under
    the 64-bit seed, Box-Muller on 24-bit uniforms.  Shape (3, n), float32;
    the transcendental functions are evaluated in FP64 and rounded."""
    cell = np.arange(n, dtype=np.uint64)
    step = int(step) & ((1 << 64) - 1)
    r = philox4x32_10(cell, step & 0xFFFFFFFF, step >> 32, 0, seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    u = [((x >> np.uint64(8)).astype(np.float64) + 0.5) / 16777216.0 for x in r]
    a = np.sqrt(-2.0 * np.log(u[0]))
    b = np.sqrt(-2.0 * np.log(u[2]))
    return np.stack([a * np.cos(2 * np.pi * u[1]), a * np.sin(2 * np.pi * u[1]),
                     b * np.cos(2 * np.pi * u[3])]).astype(np.float32)


def region_addv(B, lut, regions):
    dt = B.dtype
    getattr(lib(), f"orc_region_addv_{_sfx(dt)}")(
        _arr3(list(B)), _arr3([_c(l, dt) for l in lut]), _ptr(_c(regions, np.uint8)), B[0].size)


def lltorque(m, H, alpha):
    dt = m.dtype
    t = np.zeros_like(m)
    aa, am = (None, float(alpha)) if np.isscalar(alpha) else (_c(alpha, dt), 1.0)
    getattr(lib(), f"orc_lltorque_{_sfx(dt)}")(_arr3(list(t)), _arr3(list(m)), _arr3(list(H)),
                                               _ptr(aa), _scal(dt)(am), m[0].size)
    return t


def llnoprecess(m, H):
    dt = m.dtype
    t = np.zeros_like(m)
    getattr(lib(), f"orc_llnoprecess_{_sfx(dt)}")(_arr3(list(t)), _arr3(list(m)), _arr3(list(H)), m[0].size)
    return t


def madd(srcs, facs, dtype=np.float32):
    srcs = [_c(s, dtype) for s in srcs]
    dst = np.zeros_like(srcs[0])
    P = f32p if np.dtype(dtype) == np.float32 else f64p
    S = _scal(dtype)
    getattr(lib(), f"orc_madd_{_sfx(dtype)}")(_ptr(dst), len(srcs), (P * len(srcs))(*[_ptr(s) for s in srcs]),
                                              (S * len(facs))(*facs), dst.size)
    return dst


def normalize(v, vol=None):
    dt = v.dtype
    vol = None if vol is None else _c(vol, dt)
    getattr(lib(), f"orc_normalize_{_sfx(dt)}")(_arr3(list(v)), _ptr(vol), v[0].size)


def max_vec_norm(v):
    return getattr(lib(), f"orc_max_vec_norm_{_sfx(v.dtype)}")(_arr3(list(v)), v[0].size)


def max_vec_diff(a, b):
    return getattr(lib(), f"orc_max_vec_diff_{_sfx(a.dtype)}")(_arr3(list(a)), _arr3(list(b)), a[0].size)


def max_abs(v):
    v = np.ascontiguousarray(v)
    return getattr(lib(), f"orc_max_abs_{_sfx(v.dtype)}")(_ptr(v), v.size)


def rsum(v):
    v = np.ascontiguousarray(v)
    return getattr(lib(), f"orc_sum_{_sfx(v.dtype)}")(_ptr(v), v.size)


def rdot(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b, dtype=a.dtype)
    return getattr(lib(), f"orc_dot_{_sfx(a.dtype)}")(_ptr(a), _ptr(b), a.size)


def symidx(i, j):
    """kernels_src/clh/exchange.clh:5"""
    return (i * (i + 1)) // 2 + j if j <= i else (j * (j + 1)) // 2 + i


def exch_lut(ex, scale=None, inter=None, dtype=np.float32):
    ex = _c(ex, dtype)
    lut = np.zeros(32896, dtype=dtype)
    sc = None if scale is None else _c(scale, dtype)
    it = None if inter is None else _c(inter, dtype)
    getattr(lib(), f"orc_exch_lut_{_sfx(dtype)}")(_ptr(ex), _ptr(sc), _ptr(it), _ptr(lut))
    return lut


# ---------------------------------------------------------------- whole simulation
class Simulation:
    """Engine restatement (SetEffectiveField -> LLTorque -> Stepper.Step) on the CPU.

    Parameters follow the reference's conventions: uniform values as scalars,
    per-cell maps as arrays (regiondecode'd values), exchange/DMI as per-region
    values expanded into the 256x256 symmetric LUT.
    """

    def __init__(self, N, cell, Ms, Aex, alpha, dtype=np.float32, pbc=(0, 0, 0), Dind=0.0,
                 Ku1=0.0, Ku2=0.0, anisU=(0.0, 0.0, 1.0), B_ext=None, regions=None, vol=None,
                 Aex_regions=None, Dind_regions=None, Bext_regions=None, demag=True, openbc=False,
                 precess=True, solver=5, kernel=None, round_kernel_f32=False, Kc1=0.0, Kc2=0.0, Kc3=0.0,
                 anisC1=(1.0, 0.0, 0.0), anisC2=(0.0, 1.0, 0.0), Dbulk=0.0, Dbulk_regions=None,
                 NoDemagSpins=None, FrozenSpins=None):
        self.dtype = np.dtype(dtype)
        self.N = tuple(N)
        self.ncell = N[0] * N[1] * N[2]
        self._keep = []
        # the material as given, for the energy restatement (energies())
        self.cfg = dict(cell=tuple(cell), Ms=Ms, Aex=Aex, Dind=Dind, Ku1=Ku1, Ku2=Ku2, anisU=anisU, B_ext=B_ext,
                        vol=vol, Aex_regions=Aex_regions, Dind_regions=Dind_regions, Bext_regions=Bext_regions,
                        demag=demag, openbc=openbc, Kc1=Kc1, Kc2=Kc2, Kc3=Kc3, anisC1=anisC1, anisC2=anisC2,
                        Dbulk=Dbulk, Dbulk_regions=Dbulk_regions)
        s = OrcSystem()
        s.N[:] = N
        s.pbc[:] = pbc
        s.cell[:] = cell
        self.regions = np.zeros(self.ncell, np.uint8) if regions is None else _c(regions, np.uint8).ravel()
        s.regions = self.regions.ctypes.data_as(u8p)

        def param(v):
            if np.isscalar(v):
                return None, float(v)
            a = _c(v, self.dtype).ravel()
            self._keep.append(a)
            return _vp(a), 1.0

        s.Ms, s.Ms_mul = param(Ms)
        s.alpha, s.alpha_mul = param(alpha)
        s.Ku1, s.Ku1_mul = param(Ku1)
        s.Ku2, s.Ku2_mul = param(Ku2)
        if np.asarray(anisU).ndim == 1:
            for c in range(3):
                s.u[c] = None
                s.u_mul[c] = float(anisU[c])
        else:
            for c in range(3):
                s.u[c], s.u_mul[c] = param(anisU[c])
        s.anis = int(not (np.all(np.asarray(Ku1) == 0) and np.all(np.asarray(Ku2) == 0)))
        s.Kc1, s.Kc1_mul = param(Kc1)
        s.Kc2, s.Kc2_mul = param(Kc2)
        s.Kc3, s.Kc3_mul = param(Kc3)
        for name, val in (("c1", anisC1), ("c2", anisC2)):
            ptrs, muls = getattr(s, name), getattr(s, name + "_mul")
            if np.asarray(val).ndim == 1:
                for c in range(3):
                    ptrs[c], muls[c] = None, float(val[c])
            else:
                for c in range(3):
                    ptrs[c], muls[c] = param(val[c])
        s.cubic = int(not all(np.all(np.asarray(k) == 0) for k in (Kc1, Kc2, Kc3)))
        self.vol = None
        if vol is not None:
            self.vol = _c(vol, self.dtype).ravel()
            s.vol = _vp(self.vol)
        # exchange LUTs (engine/exchange.go:153-167)
        aex = np.full(256, Aex, dtype=self.dtype) if Aex_regions is None else _c(Aex_regions, self.dtype)
        self.aLUT = exch_lut(aex, dtype=self.dtype)
        s.aLUT = _vp(self.aLUT)
        dmi_on = (Dind != 0.0) or (Dind_regions is not None and np.any(np.asarray(Dind_regions) != 0))
        s.dmi = int(dmi_on)
        din = np.full(256, Dind, dtype=self.dtype) if Dind_regions is None else _c(Dind_regions, self.dtype)
        self.dLUT = exch_lut(din, dtype=self.dtype)
        s.dLUT = _vp(self.dLUT)
        dbk = np.full(256, Dbulk, dtype=self.dtype) if Dbulk_regions is None else _c(Dbulk_regions, self.dtype)
        if np.any(dbk != 0):
            self.dbLUT = exch_lut(dbk, dtype=self.dtype)
            s.dbLUT = _vp(self.dbLUT)
        s.openbc = int(openbc)
        s.precess = int(precess)
        # per-region switches (a scalar or 256 values): engine/demag.go:22, engine/torque.go:348
        for name, val in (("nodemag", NoDemagSpins), ("frozen", FrozenSpins)):
            if val is not None:
                lut = np.zeros(256, self.dtype)
                v = np.asarray(val, self.dtype).ravel()
                lut[: v.size] = v
                if v.size == 1:
                    lut[:] = v[0]
                setattr(self, name + "_lut", lut)
                setattr(s, name, _vp(lut))
        # Zeeman LUT (engine/excitation.go:41-53)
        if Bext_regions is not None or B_ext is not None:
            if Bext_regions is None:
                Bext_regions = np.tile(np.asarray(B_ext, dtype=np.float64), (256, 1))
            lut = _c(np.asarray(Bext_regions).T, self.dtype)
            self.bext = [np.ascontiguousarray(lut[c]) for c in range(3)]
            for c in range(3):
                s.bext_lut[c] = _vp(self.bext[c])
        s.enable_demag = int(demag)
        self.P = pad_size(N, pbc)
        s.P[:] = self.P
        if demag:
            if kernel is None:
                K = newell_kernel(N, cell, pbc)
                kernel, _ = kernel_spectrum(K, round_f32=round_kernel_f32)
            self.Kf = np.ascontiguousarray(kernel)
            for c in range(6):
                s.Kf[c] = self.Kf[c].ctypes.data_as(f64p)
        self.sys = s
        self.solver = OrcSolver()
        lib().orc_solver_defaults(ctypes.byref(self.solver))
        self.solver.solver = solver
        self.m = np.zeros((3,) + tuple(reversed(N)), dtype=self.dtype)
        self.k1 = np.zeros_like(self.m)

    def set_m(self, m):
        self.m[...] = np.asarray(m, dtype=self.dtype).reshape(self.m.shape)
        normalize(self.m, self.vol)
        self.solver.have_k1 = 0

    def torque(self, m=None, beff=False):
        m = self.m if m is None else _c(m, self.dtype)
        tau = np.zeros_like(m)
        B = np.zeros_like(m) if beff else None
        fn = getattr(lib(), f"orc_torque_{_sfx(self.dtype)}")
        P = f32p if self.dtype == np.float32 else f64p
        fn(ctypes.byref(self.sys), _ptr(tau), _ptr(m), None if B is None else _ptr(B))
        return (tau, B) if beff else tau

    def step(self):
        fn = getattr(lib(), f"orc_step_{_sfx(self.dtype)}")
        ok = fn(ctypes.byref(self.sys), ctypes.byref(self.solver), _ptr(self.m), _ptr(self.k1))
        if self.solver.status:
            raise RuntimeError(f"oracle solver failure status {self.solver.status}")
        return bool(ok)

    def run(self, seconds, max_steps=10 ** 9, on_step=None):
        """engine/run.go:190-195 Run(): step until Time >= start + seconds."""
        stop = self.solver.time + seconds
        self.solver.alarm = stop
        self.solver.have_k1 = 0  # RunWhile frees the stepper (engine/run.go:207)
        n = 0
        while self.solver.time < stop and n < max_steps:
            ok = self.step()
            n += 1
            if on_step is not None:
                on_step(self, ok)
        return n


# ---------------------------------------------------------------- energies / relax
def energies(sim, m=None):
    """engine/energy.go:27-35 GetTotalEnergy and its terms, in FP64, for an
    oracle Simulation: E_demag = -1/2 V sum M_full.B_demag (engine/demag.go:146),
    E_exch = -1/2 V sum M_full.B_exch incl. DMI (engine/exchange.go:79),
    E_anis = V sum(-1/2 M_full.B_K1 - 1/4 M_full.B_K2) (engine/anisotropy.go:164-216),
    E_Zeeman = -V sum M_full.B_ext (engine/zeeman.go:15); M_full = Ms m (vol)
    (engine/demag.go:101-121).  Total in the terms' registration order."""
    c = sim.cfg
    f8 = np.float64
    m = np.asarray(sim.m if m is None else m, f8).reshape((3,) + tuple(reversed(sim.N)))
    cell = c["cell"]
    V = cell[0] * cell[1] * cell[2]
    shape = m.shape[1:]
    regions = sim.regions.reshape(shape)
    vol = None if c["vol"] is None else np.asarray(c["vol"], f8).reshape(shape)
    Ms = c["Ms"]
    Ms_arr = np.full(shape, float(Ms)) if np.isscalar(Ms) else np.asarray(Ms, f8).reshape(shape)
    Mf = m * Ms_arr
    if vol is not None:
        Mf = Mf * vol
    E = {}
    Bd = demag_field(sim.Kf, sim.P, m, Ms, vol=vol, dtype=f8) if c["demag"] else np.zeros_like(m)
    E["demag"] = -0.5 * V * float(np.sum(Mf * Bd))
    aex = np.full(256, c["Aex"], f8) if c["Aex_regions"] is None else np.asarray(c["Aex_regions"], f8)
    alut = exch_lut(aex, dtype=f8)
    Be = np.zeros_like(m)
    din = np.full(256, c["Dind"], f8) if c["Dind_regions"] is None else np.asarray(c["Dind_regions"], f8)
    dbk = np.full(256, c["Dbulk"], f8) if c["Dbulk_regions"] is None else np.asarray(c["Dbulk_regions"], f8)
    if np.any(dbk != 0):
        add_dmibulk(Be, m, alut, exch_lut(dbk, dtype=f8), regions, cell, Ms, 0, int(c["openbc"]))
    elif np.any(din != 0):
        add_dmi(Be, m, alut, exch_lut(din, dtype=f8), regions, cell, Ms, 0, int(c["openbc"]))
    else:
        add_exchange(Be, m, alut, regions, cell, Ms)
    E["exchange"] = -0.5 * V * float(np.sum(Mf * Be))
    Ea = 0.0
    if not (np.all(np.asarray(c["Ku1"]) == 0) and np.all(np.asarray(c["Ku2"]) == 0)):
        B1 = np.zeros_like(m)
        add_uniaxial(B1, m, Ms, c["Ku1"], 0.0, c["anisU"])
        B2 = np.zeros_like(m)
        add_uniaxial(B2, m, Ms, 0.0, c["Ku2"], c["anisU"])
        Ea = V * float(np.sum(-0.5 * np.sum(Mf * B1, axis=0) - 0.25 * np.sum(Mf * B2, axis=0)))
    if not all(np.all(np.asarray(c[k]) == 0) for k in ("Kc1", "Kc2", "Kc3")):
        # engine/anisotropy.go:191-206: -1/4, -1/6, -1/8 of M_full.B of each constant alone
        for k, pre in (("Kc1", -0.25), ("Kc2", -1.0 / 6.0), ("Kc3", -0.125)):
            Ks = [c[k] if j == k else 0.0 for j in ("Kc1", "Kc2", "Kc3")]
            Bc = np.zeros_like(m)
            add_cubic(Bc, m, Ms, Ks[0], Ks[1], Ks[2], np.asarray(c["anisC1"], f8), np.asarray(c["anisC2"], f8))
            Ea += V * pre * float(np.sum(Mf * Bc))
    E["anisotropy"] = Ea
    Ez = 0.0
    if c["Bext_regions"] is not None or c["B_ext"] is not None:
        lut = c["Bext_regions"]
        if lut is None:
            lut = np.tile(np.asarray(c["B_ext"], f8), (256, 1))
        lut = np.ascontiguousarray(np.asarray(lut, f8).T)
        Bz = np.zeros_like(m)
        region_addv(Bz, lut, regions)
        Ez = -1.0 * V * float(np.sum(Mf * Bz))
    E["zeeman"] = Ez
    E["total"] = ((E["anisotropy"] + E["demag"]) + E["exchange"]) + E["zeeman"]
    return E


def relax(sim, torque_threshold=-1.0, max_relax_steps=10 ** 6):
    """engine/relax.go:23-112 Relax() on an oracle Simulation: RK23 without
    precession; 3-step chunks while the total energy decreases, then the
    torque phase (max |k1| against the threshold, or the mean squared torque
    while MaxErr is lowered by sqrt(2) down to 1e-9).  Time is restored after
    every chunk (relax.go:134-141); solver settings are restored at the end."""
    s = sim.solver
    prev = (s.solver, s.max_err, s.fix_dt, sim.sys.precess)
    s.solver, s.fix_dt, sim.sys.precess = 3, 0.0, 0
    s.have_k1 = 0
    budget = [max_relax_steps]

    def steps(n):
        t0 = s.time
        target = s.nsteps + n
        s.have_k1 = 0  # runWhile frees the stepper
        while s.nsteps < target:
            sim.step()
            budget[0] -= 1
            if budget[0] < 0:
                raise RuntimeError("relax: step budget exhausted")
        s.time = t0

    def etot():
        return energies(sim)["total"]

    def k1():
        return sim.k1.reshape(3, -1)

    try:
        n = 3
        steps(n)
        E0 = etot()
        steps(n)
        E1 = etot()
        while E1 < E0:
            steps(n)
            E0, E1 = E1, etot()
        if torque_threshold > 0:
            while True:
                while max_vec_norm(k1()) > torque_threshold:
                    steps(n)
                s.max_err /= np.sqrt(2)
                if s.max_err < 1e-9:
                    break
        else:
            T1 = np.float32(rdot(k1(), k1()))
            while s.max_err > 1e-9:
                s.max_err /= np.sqrt(2)
                steps(n)
                T0, T1 = T1, np.float32(rdot(k1(), k1()))
                while T1 < T0:
                    steps(n)
                    T0, T1 = T1, np.float32(rdot(k1(), k1()))
    finally:
        s.solver, s.max_err, s.fix_dt, sim.sys.precess = prev
        s.have_k1 = 0
