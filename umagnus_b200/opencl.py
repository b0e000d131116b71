"""Python mirror of the hot-path subset of the reference's Go package `opencl`
(the device-op layer), backed by libumagnus_b200.so.

Names, argument meaning and order follow the Go functions they replace
(file:line in the uMagNUS tree); slices are torch CUDA float32 tensors of
shape (ncomp, Nz, Ny, Nx), x fastest (data/slice.go:53-100).  Errors raise
UmagError, the Python counterpart of the reference's util.Fatal.
"""
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import UmagError, check

__all__ = ["Init", "ReleaseAndClean", "NewSlice", "Zero", "Memset", "Mesh", "MSlice", "AddExchange", "AddDMI",
           "AddUniaxialAnisotropy2", "RegionAddV", "RegionDecode", "LLTorque", "LLNoPrecess", "Madd", "Madd2",
           "Madd3", "Madd4", "Madd5", "Madd6", "Madd7", "Normalize", "VecNorm", "Div", "AddDotProduct", "MaxVecNorm",
           "MaxVecDiff", "MaxAbs", "Sum", "Dot", "DemagConvolution", "NewNewellDemag", "NewBruteDemag", "NewDemag", "UmagError",
           "Sync"]


def _L():
    return _lib.init(_device())


def _device():
    return torch.cuda.current_device() if torch.cuda.is_available() else 0


def _in():
    """Make the library stream see work queued by torch."""
    torch.cuda.current_stream().synchronize()


def Sync():
    check(_L().umag_sync())


def _p(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise UmagError("device arrays must be CUDA tensors")
    if not t.is_contiguous():
        raise UmagError("device arrays must be contiguous")
    return t.data_ptr()


def _f32(t, name):
    if t.dtype != torch.float32:
        raise UmagError(f"{name} must be float32")
    return t


@dataclass
class Mesh:
    """data/mesh.go: grid size (Nx, Ny, Nz), cell size (m), PBC repetitions."""
    size: tuple
    cellsize: tuple
    pbc: tuple = (0, 0, 0)

    def PBC_code(self):
        return (1 if self.pbc[0] else 0) | (2 if self.pbc[1] else 0) | (4 if self.pbc[2] else 0)

    def NCell(self):
        return self.size[0] * self.size[1] * self.size[2]


@dataclass
class MSlice:
    """opencl/mslice.go:11: a per-cell array times a multiplier; arr None = uniform mul."""
    arr: object = None
    mul: float = 1.0

    def ptr(self):
        return _p(self.arr) if self.arr is not None else None


def _ms(x):
    if isinstance(x, MSlice):
        return x
    if torch.is_tensor(x):
        return MSlice(x, 1.0)
    return MSlice(None, float(x))


def Init(gpu=0):
    """opencl/init.go:48"""
    _lib.init(gpu)


def ReleaseAndClean():
    """opencl/init.go:287"""
    check(_lib.load().umag_release())
    _lib._initialised = None


def NewSlice(ncomp, size):
    """opencl/slice.go:14 (size = (Nx, Ny, Nz))"""
    _L()
    return torch.zeros((ncomp, size[2], size[1], size[0]), dtype=torch.float32, device="cuda")


def Zero(s):
    """opencl/slice.go:156"""
    L = _L()
    _in()
    check(L.umag_memset_f32(_p(s), 0.0, s.numel()))
    Sync()


def Memset(s, *vals):
    """opencl/slice.go:170"""
    L = _L()
    _in()
    for c, v in enumerate(vals):
        check(L.umag_memset_f32(_p(s[c]), float(v), s[c].numel()))
    Sync()


def _comps(s):
    return [_p(s[c]) for c in range(s.shape[0])]


def AddExchange(B, m, Aex_red, Msat, regions, mesh):
    """opencl/exchange.go:16"""
    L = _L()
    _in()
    ms = _ms(Msat)
    c = mesh.cellsize
    check(L.umag_add_exchange(*_comps(B), *_comps(m), ms.ptr(), ms.mul, _p(Aex_red), _p(regions), *mesh.size,
                              c[0], c[1], c[2], mesh.PBC_code()))
    Sync()


def AddDMI(Beff, m, Aex_red, Dex_red, Msat, regions, mesh, OpenBC=False):
    """opencl/dmi.go:15"""
    L = _L()
    _in()
    ms = _ms(Msat)
    c = mesh.cellsize
    check(L.umag_add_dmi(*_comps(Beff), *_comps(m), ms.ptr(), ms.mul, _p(Aex_red), _p(Dex_red), _p(regions),
                         *mesh.size, c[0], c[1], c[2], mesh.PBC_code(), int(bool(OpenBC))))
    Sync()


def AddUniaxialAnisotropy2(Beff, m, Msat, k1, k2, u):
    """opencl/anisotropy.go:153.  u: 3 MSlices (or a 3-vector, or a (3,...) tensor)."""
    L = _L()
    _in()
    ms, K1, K2 = _ms(Msat), _ms(k1), _ms(k2)
    if torch.is_tensor(u):
        us = [MSlice(u[i], 1.0) for i in range(3)]
    else:
        us = [_ms(x) for x in u]
    n = m[0].numel()
    check(L.umag_add_uniaxial_anisotropy2(*_comps(Beff), *_comps(m), ms.ptr(), ms.mul, K1.ptr(), K1.mul, K2.ptr(),
                                          K2.mul, us[0].ptr(), us[0].mul, us[1].ptr(), us[1].mul, us[2].ptr(),
                                          us[2].mul, n))
    Sync()


def AddDMIBulk(Beff, m, Aex_red, D_red, Msat, regions, mesh, OpenBC=False):
    """opencl/dmibulk.go:14"""
    L = _L()
    _in()
    ms = _ms(Msat)
    c = mesh.cellsize
    check(L.umag_add_dmi_bulk(*_comps(Beff), *_comps(m), ms.ptr(), ms.mul, _p(Aex_red), _p(D_red), _p(regions),
                              *mesh.size, c[0], c[1], c[2], mesh.PBC_code(), int(bool(OpenBC))))
    Sync()


def AddCubicAnisotropy2(Beff, m, Msat, k1, k2, k3, c1, c2):
    """opencl/anisotropy.go:12.  c1, c2: 3 MSlices each (or 3-vectors, or (3,...) tensors)."""
    import ctypes
    L = _L()
    _in()
    ms, K1, K2, K3 = _ms(Msat), _ms(k1), _ms(k2), _ms(k3)

    def axes(u):
        us = [MSlice(u[i], 1.0) for i in range(3)] if torch.is_tensor(u) else [_ms(x) for x in u]
        return (ctypes.c_void_p * 3)(*[x.ptr() for x in us]), (ctypes.c_float * 3)(*[x.mul for x in us])

    p1, m1 = axes(c1)
    p2, m2 = axes(c2)
    check(L.umag_add_cubic_anisotropy2(*_comps(Beff), *_comps(m), ms.ptr(), ms.mul, K1.ptr(), K1.mul, K2.ptr(),
                                       K2.mul, K3.ptr(), K3.mul, p1, m1, p2, m2, m[0].numel()))
    Sync()


def RegionAddV(dst, lut, regions):
    """opencl/region.go:13; lut: (3, 256) float32 CUDA tensor"""
    L = _L()
    _in()
    check(L.umag_region_addv(*_comps(dst), _p(lut[0]), _p(lut[1]), _p(lut[2]), _p(regions), dst[0].numel()))
    Sync()


def RegionDecode(dst, lut, regions):
    """opencl/region.go:108"""
    L = _L()
    _in()
    check(L.umag_region_decode(_p(dst), _p(lut), _p(regions), dst.numel()))
    Sync()


def LLTorque(torque, m, B, alpha):
    """opencl/lltorque.go:16 (torque may be B)"""
    L = _L()
    _in()
    a = _ms(alpha)
    check(L.umag_lltorque(*_comps(torque), *_comps(m), *_comps(B), a.ptr(), a.mul, m[0].numel()))
    Sync()


def SetTemperature(Bth, noise, k2mu0_Mu0VgammaDt, Msat, Temp, Alpha):
    """opencl/temperature.go:14 (temperature2.cl): Bth = noise * sqrt(k2 alpha T / Ms); one component."""
    L = _L()
    _in()
    ms, t, a = _ms(Msat), _ms(Temp), _ms(Alpha)
    check(L.umag_set_temperature(_p(Bth), _p(noise), float(k2mu0_Mu0VgammaDt), ms.ptr(), ms.mul, t.ptr(), t.mul,
                                 a.ptr(), a.mul, Bth.numel()))
    Sync()


def ThermalNoise(noise, seed, step):
    """Standard normal noise (3, ...) of accepted step `step` under `seed`
    (the stand-in for the reference's device-dependent Threefry stream)."""
    L = _L()
    _in()
    check(L.umag_thermal_noise(*_comps(noise), noise[0].numel(), int(seed) & ((1 << 64) - 1), int(step)))
    Sync()


def ZeroMask(dst, mask, regions):
    """opencl/zeromask.go:12: dst = 0 where mask[regions] != 0 (mask: 256-entry LUT)."""
    L = _L()
    _in()
    check(L.umag_zero_mask(*_comps(dst), _p(_f32(mask, "mask")), _p(regions), dst[0].numel()))
    Sync()


def LLNoPrecess(torque, m, B):
    """opencl/lltorque.go:97"""
    L = _L()
    _in()
    check(L.umag_llnoprecess(*_comps(torque), *_comps(m), *_comps(B), m[0].numel()))
    Sync()


def Madd(dst, srcs, facs):
    """opencl/madd.go:111-413: dst = sum_j facs[j]*srcs[j] (all components)."""
    import ctypes
    L = _L()
    _in()
    ncomp = dst.shape[0] if dst.dim() == 4 else 1
    d = dst if dst.dim() == 4 else dst.unsqueeze(0)
    ss = [s if s.dim() == 4 else s.unsqueeze(0) for s in srcs]
    dptr = (ctypes.c_void_p * ncomp)(*[d[c].data_ptr() for c in range(ncomp)])
    sptr = (ctypes.c_void_p * (ncomp * len(ss)))(*[s[c].data_ptr() for s in ss for c in range(ncomp)])
    f = (ctypes.c_float * len(facs))(*[float(x) for x in facs])
    check(L.umag_madd(ncomp, dptr, len(ss), sptr, f, d[0].numel()))
    Sync()


def Madd2(dst, src1, src2, fac1, fac2):
    Madd(dst, [src1, src2], [fac1, fac2])


def Madd3(dst, s1, s2, s3, f1, f2, f3):
    Madd(dst, [s1, s2, s3], [f1, f2, f3])


def Madd4(dst, s1, s2, s3, s4, f1, f2, f3, f4):
    Madd(dst, [s1, s2, s3, s4], [f1, f2, f3, f4])


def Madd5(dst, s1, s2, s3, s4, s5, f1, f2, f3, f4, f5):
    Madd(dst, [s1, s2, s3, s4, s5], [f1, f2, f3, f4, f5])


def Madd6(dst, s1, s2, s3, s4, s5, s6, f1, f2, f3, f4, f5, f6):
    Madd(dst, [s1, s2, s3, s4, s5, s6], [f1, f2, f3, f4, f5, f6])


def Madd7(dst, s1, s2, s3, s4, s5, s6, s7, f1, f2, f3, f4, f5, f6, f7):
    Madd(dst, [s1, s2, s3, s4, s5, s6, s7], [f1, f2, f3, f4, f5, f6, f7])


def Normalize(vec, vol=None):
    """opencl/normalize.go:13"""
    L = _L()
    _in()
    check(L.umag_normalize(*_comps(vec), _p(vol), vec[0].numel()))
    Sync()


def VecNorm(dst, a):
    """opencl/vecnorm.go:12"""
    L = _L()
    _in()
    check(L.umag_vecnorm(_p(dst), *_comps(a), dst.numel()))
    Sync()


def Div(dst, a, b):
    """opencl/madd.go:60"""
    L = _L()
    _in()
    check(L.umag_div(_p(dst), _p(a), _p(b), dst.numel()))
    Sync()


def AddDotProduct(dst, prefactor, a, b):
    """opencl/dotproduct.go"""
    L = _L()
    _in()
    check(L.umag_add_dot_product(_p(dst), float(prefactor), *_comps(a), *_comps(b), dst.numel()))
    Sync()


def _dbl():
    import ctypes
    return ctypes.c_double()


def MaxVecNorm(v):
    """opencl/reduce.go:180"""
    import ctypes
    L = _L()
    _in()
    out = _dbl()
    check(L.umag_max_vec_norm(*_comps(v), v[0].numel(), ctypes.byref(out)))
    return out.value


def MaxVecDiff(x, y):
    """opencl/reduce.go:214"""
    import ctypes
    L = _L()
    _in()
    out = _dbl()
    check(L.umag_max_vec_diff(*_comps(x), *_comps(y), x[0].numel(), ctypes.byref(out)))
    return out.value


def MaxAbs(v):
    """opencl/reduce.go:105"""
    import ctypes
    L = _L()
    _in()
    out = _dbl()
    check(L.umag_max_abs(_p(v), v.numel(), ctypes.byref(out)))
    return out.value


def Sum(v):
    """opencl/reduce.go:26 (compensated)"""
    import ctypes
    L = _L()
    _in()
    out = _dbl()
    check(L.umag_sum(_p(v), v.numel(), ctypes.byref(out)))
    return out.value


def Dot(a, b):
    """opencl/reduce.go:54 (compensated; all components)"""
    import ctypes
    L = _L()
    _in()
    tot = 0.0
    aa = a if a.dim() == 4 else a.unsqueeze(0)
    bb = b if b.dim() == 4 else b.unsqueeze(0)
    for c in range(aa.shape[0]):
        out = _dbl()
        check(L.umag_dot(_p(aa[c]), _p(bb[c]), aa[c].numel(), ctypes.byref(out)))
        tot += out.value
    return tot


class DemagConvolution:
    """opencl/conv_demag.go:14 -- FFT demag convolution with a symmetric kernel."""

    def __init__(self, handle, size):
        self._h = handle
        self.size = tuple(size)

    def Exec(self, B, m, vol, Msat):
        """opencl/conv_demag.go:43: B = demag field of m*vol*Msat (B overwritten)."""
        L = _L()
        _in()
        ms = _ms(Msat)
        check(L.umag_demag_exec(self._h, *_comps(B), *_comps(m), _p(vol), ms.ptr(), ms.mul))
        Sync()

    def ExecPass(self, p, B, m, vol, Msat):
        """One pass (0: x/z forward, 1: y + kernel multiply, 2: inverse z/x) of
        Exec, queued without a synchronize (for timing the passes one by one)."""
        L = _L()
        _in()
        ms = _ms(Msat)
        check(L.umag_demag_exec_pass(self._h, int(p), *_comps(B), *_comps(m), _p(vol), ms.ptr(), ms.mul))

    def padded_size(self):
        import ctypes
        P = (ctypes.c_int * 3)()
        check(_L().umag_demag_padded_size(self._h, P))
        return tuple(P)

    def spectrum(self):
        """float32 kernel spectrum, 6 arrays (xx yy zz yz xz xy) of shape (Pz/2+1, Py/2+1, Px/2+1)."""
        import ctypes
        Px, Py, Pz = self.padded_size()
        shape = (Pz // 2 + 1, Py // 2 + 1, Px // 2 + 1)
        out = [np.zeros(shape, np.float32) for _ in range(6)]
        ptrs = (ctypes.c_void_p * 6)(*[o.ctypes.data for o in out])
        check(_L().umag_demag_get_spectrum(self._h, ptrs))
        return np.stack(out)

    def kernel(self):
        """FP64 real-space Newell tensor, (6, Pz, Py, Px)."""
        import ctypes
        Px, Py, Pz = self.padded_size()
        out = [np.zeros((Pz, Py, Px), np.float64) for _ in range(6)]
        ptrs = (ctypes.c_void_p * 6)(*[o.ctypes.data for o in out])
        check(_L().umag_demag_get_kernel(self._h, ptrs))
        return np.stack(out)

    def Free(self):
        if self._h:
            _L().umag_demag_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Free()
        except Exception:
            pass


def NewNewellDemag(inputSize, PBC, cellsize, asymptotic_radius=32, zero_self_demag=0):
    """engine/demag.go:135-143 newellDemagConv: Newell tensor (FP64, on the GPU) + plan."""
    import ctypes
    L = _L()
    h = ctypes.c_void_p()
    pbc = (ctypes.c_int * 3)(*PBC)
    check(L.umag_demag_new_newell(inputSize[0], inputSize[1], inputSize[2], pbc, cellsize[0], cellsize[1],
                                  cellsize[2], asymptotic_radius, zero_self_demag, ctypes.byref(h)))
    return DemagConvolution(h.value, inputSize)


def NewBruteDemag(inputSize, PBC, cellsize, accuracy=6.0):
    """engine/demag.go:124-133 demagConv with EnableDemag: mag/demagkernel.go:113
    CalcDemagKernel (brute force, built on the GPU) + plan."""
    import ctypes
    L = _L()
    h = ctypes.c_void_p()
    pbc = (ctypes.c_int * 3)(*PBC)
    check(L.umag_demag_new_brute(inputSize[0], inputSize[1], inputSize[2], pbc, cellsize[0], cellsize[1],
                                 cellsize[2], float(accuracy), ctypes.byref(h)))
    return DemagConvolution(h.value, inputSize)


def NewDemag(inputSize, kernel):
    """opencl/conv_demag.go:27 with a real-space kernel (6, Pz, Py, Px) float64 (xx yy zz yz xz xy)."""
    import ctypes
    L = _L()
    k = [np.ascontiguousarray(kernel[c], dtype=np.float64) for c in range(6)]
    ptrs = (ctypes.c_void_p * 6)(*[a.ctypes.data for a in k])
    h = ctypes.c_void_p()
    check(L.umag_demag_new_from_kernel(inputSize[0], inputSize[1], inputSize[2], ptrs, ctypes.byref(h)))
    return DemagConvolution(h.value, inputSize)
