"""Build oracle/_ref/libclref.so: the reference's own OpenCL C hot-path kernels
compiled unchanged as C++ for the host (TEST INFRASTRUCTURE ONLY).

The kernel sources are #included from the read-only reference tree
(kernels_src/cl, kernels_src/clh) at build time; nothing is copied into this
repository.  Outputs go to oracle/_ref/ only (git-ignored).  The library is
used by tests to pin the oracle's C restatement (oracle/orc_cells.inc)
against the reference's kernel code, and by bench.py --impl reference as the
CPU baseline ("reference kernel source executed as C++ on host cores").

Kernels with work-group barriers (the reductions) are not built: their
semantics are a plain max / sum, restated directly in the oracle.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# Where the reference checkout lives: $UMAG_REFERENCE, else the build
# machine's read-only checkout.  This recipe is the one place that names the
# default; tests and fixture scripts ask reference_root().
DEFAULT_REFERENCE = "/root/reference"


def reference_root():
    """The reference checkout ($UMAG_REFERENCE, else the default location), or
    None when neither exists (the GPU box has no reference tree)."""
    env = os.environ.get("UMAG_REFERENCE")
    if env:
        if not os.path.isdir(env):
            raise FileNotFoundError(f"UMAG_REFERENCE={env} is not a directory")
        return env
    return DEFAULT_REFERENCE if os.path.isdir(DEFAULT_REFERENCE) else None


def _kernels_src():
    ref = reference_root()
    if ref is None:
        raise FileNotFoundError("reference checkout not found: set UMAG_REFERENCE to its root")
    return os.path.join(ref, "kernels_src")

HEADERS = ["typedefs.clh", "constants.clh", "stencil.clh", "float3.clh", "exchange.clh", "amul.clh"]
KERNELS = ["copypadmul2", "copyunpad", "kernmulrsymm3d", "kernmulrsymm2dxy", "kernmulrsymm2dz",
           "exchange", "dmi", "dmibulk", "uniaxialanisotropy2", "cubicanisotropy2", "regionaddv", "regiondecode", "lltorque2",
           "llnoprecess", "madd2", "madd3", "madd4", "madd5", "madd6", "madd7", "normalize2",
           "vecnorm", "div", "dotproduct", "temperature2"]

# extern "C" wrappers: (name, C parameter list, kernel call, launch kind)
#   kind "3d:<x>,<y>,<z>"  -> make3DConf (opencl/util.go:35-45): local 16x16x1
#   kind "1d:<n>"          -> one work-item per element (grid-stride kernels)
R = "R"
WRAPPERS = [
    ("addexchange", f"R* Bx, R* By, R* Bz, R* mx, R* my, R* mz, R* Ms, R Ms_mul, R* aLUT, uint8_t* regions,"
                    f" R wx, R wy, R wz, int Nx, int Ny, int Nz, int pbc",
     "addexchange(Bx, By, Bz, mx, my, mz, Ms, Ms_mul, aLUT, regions, wx, wy, wz, Nx, Ny, Nz, (uint8_t)pbc)",
     "3d:Nx,Ny,Nz"),
    ("adddmi", f"R* Hx, R* Hy, R* Hz, R* mx, R* my, R* mz, R* Ms, R Ms_mul, R* aLUT, R* dLUT, uint8_t* regions,"
               f" R cx, R cy, R cz, int Nx, int Ny, int Nz, int pbc, int openbc",
     "adddmi(Hx, Hy, Hz, mx, my, mz, Ms, Ms_mul, aLUT, dLUT, regions, cx, cy, cz, Nx, Ny, Nz,"
     " (uint8_t)pbc, (uint8_t)openbc)", "3d:Nx,Ny,Nz"),
    ("adduniaxialanisotropy2", "R* Bx, R* By, R* Bz, R* mx, R* my, R* mz, R* Ms, R Ms_mul, R* K1, R K1_mul,"
                               " R* K2, R K2_mul, R* ux, R ux_mul, R* uy, R uy_mul, R* uz, R uz_mul, int N",
     "adduniaxialanisotropy2(Bx, By, Bz, mx, my, mz, Ms, Ms_mul, K1, K1_mul, K2, K2_mul, ux, ux_mul,"
     " uy, uy_mul, uz, uz_mul, N)", "1d:N"),
    ("adddmibulk", f"R* Hx, R* Hy, R* Hz, R* mx, R* my, R* mz, R* Ms, R Ms_mul, R* aLUT, R* dLUT, uint8_t* regions,"
                   f" R cx, R cy, R cz, int Nx, int Ny, int Nz, int pbc, int openbc",
     "adddmibulk(Hx, Hy, Hz, mx, my, mz, Ms, Ms_mul, aLUT, dLUT, regions, cx, cy, cz, Nx, Ny, Nz,"
     " (uint8_t)pbc, (uint8_t)openbc)", "3d:Nx,Ny,Nz"),
    ("addcubicanisotropy2", "R* Bx, R* By, R* Bz, R* mx, R* my, R* mz, R* Ms, R Ms_mul, R* K1, R K1_mul,"
                            " R* K2, R K2_mul, R* K3, R K3_mul, R* c1x, R c1x_mul, R* c1y, R c1y_mul, R* c1z,"
                            " R c1z_mul, R* c2x, R c2x_mul, R* c2y, R c2y_mul, R* c2z, R c2z_mul, int N",
     "addcubicanisotropy2(Bx, By, Bz, mx, my, mz, Ms, Ms_mul, K1, K1_mul, K2, K2_mul, K3, K3_mul, c1x, c1x_mul,"
     " c1y, c1y_mul, c1z, c1z_mul, c2x, c2x_mul, c2y, c2y_mul, c2z, c2z_mul, N)", "1d:N"),
    ("settemperature2", "R* B, R* noise, R k2, R* Ms, R Ms_mul, R* temp, R temp_mul, R* alpha, R alpha_mul, int N",
     "settemperature2(B, noise, k2, Ms, Ms_mul, temp, temp_mul, alpha, alpha_mul, N)", "1d:N"),
    ("regionaddv", "R* dx, R* dy, R* dz, R* lx, R* ly, R* lz, uint8_t* regions, int N",
     "regionaddv(dx, dy, dz, lx, ly, lz, regions, N)", "1d:N"),
    ("regiondecode", "R* dst, R* lut, uint8_t* regions, int N", "regiondecode(dst, lut, regions, N)", "1d:N"),
    ("lltorque2", "R* tx, R* ty, R* tz, R* mx, R* my, R* mz, R* hx, R* hy, R* hz, R* alpha, R alpha_mul, int N",
     "lltorque2(tx, ty, tz, mx, my, mz, hx, hy, hz, alpha, alpha_mul, N)", "1d:N"),
    ("llnoprecess", "R* tx, R* ty, R* tz, R* mx, R* my, R* mz, R* hx, R* hy, R* hz, int N",
     "llnoprecess(tx, ty, tz, mx, my, mz, hx, hy, hz, N)", "1d:N"),
    ("normalize2", "R* vx, R* vy, R* vz, R* vol, int N", "normalize2(vx, vy, vz, vol, N)", "1d:N"),
    ("vecnorm", "R* dst, R* ax, R* ay, R* az, int N", "vecnorm(dst, ax, ay, az, N)", "1d:N"),
    ("pointwise_div", "R* dst, R* a, R* b, int N", "pointwise_div(dst, a, b, N)", "1d:N"),
    ("dotproduct", "R* dst, R pre, R* ax, R* ay, R* az, R* bx, R* by, R* bz, int N",
     "dotproduct(dst, pre, ax, ay, az, bx, by, bz, N)", "1d:N"),
    ("copypadmul2", "R* dst, int Dx, int Dy, int Dz, R* src, int Sx, int Sy, int Sz, R* Ms, R Ms_mul, R* vol",
     "copypadmul2(dst, Dx, Dy, Dz, src, Sx, Sy, Sz, Ms, Ms_mul, vol)", "3d:Sx,Sy,Sz"),
    ("copyunpad", "R* dst, int Dx, int Dy, int Dz, R* src, int Sx, int Sy, int Sz",
     "copyunpad(dst, Dx, Dy, Dz, src, Sx, Sy, Sz)", "3d:Dx,Dy,Dz"),
    ("kernmulRSymm3D", "R* Mx, R* My, R* Mz, R* Kxx, R* Kyy, R* Kzz, R* Kyz, R* Kxz, R* Kxy, int Nx, int Ny, int Nz",
     "kernmulRSymm3D(Mx, My, Mz, Kxx, Kyy, Kzz, Kyz, Kxz, Kxy, Nx, Ny, Nz)", "3d:Nx,Ny,Nz"),
    ("kernmulRSymm2Dxy", "R* Mx, R* My, R* Kxx, R* Kyy, R* Kxy, int Nx, int Ny",
     "kernmulRSymm2Dxy(Mx, My, Kxx, Kyy, Kxy, Nx, Ny)", "3d:Nx,Ny,1"),
    ("kernmulRSymm2Dz", "R* Mz, R* Kzz, int Nx, int Ny", "kernmulRSymm2Dz(Mz, Kzz, Nx, Ny)", "3d:Nx,Ny,1"),
]
MADD = {n: ", ".join(["R* dst"] + [f"R* s{i}, R f{i}" for i in range(1, n + 1)] + ["int N"]) for n in range(2, 8)}


def gen_tu(real, sfx):
    KS = _kernels_src()
    lines = ["// generated by oracle/build_ref.py -- do not edit", '#include "../clshim.hpp"']
    if real == "double":
        lines += ["#define __REAL_IS_DOUBLE__ 1", "#define cl_khr_fp64 1"]
    lines.append(f"namespace ref_{sfx} {{")
    lines.append("#pragma GCC diagnostic push")
    lines.append('#pragma GCC diagnostic ignored "-Wunknown-pragmas"')
    for h in HEADERS:
        lines.append(f'#include "{os.path.join(KS, "clh", h)}"')
    for k in KERNELS:
        lines.append(f'#include "{os.path.join(KS, "cl", k + ".cl")}"')
    lines.append("#pragma GCC diagnostic pop")
    lines.append("}")
    lines.append(f"using R = {real};")
    lines.append("thread_local clshim_item clshim_cur;\nint clshim_nthreads = 1;" if sfx == "f32" else "")
    lines.append('extern "C" {')
    if sfx == "f32":
        lines.append("void clref_set_threads(int n) { clshim_nthreads = n > 0 ? n : 1; }")

    def launch(kind, call):
        if kind.startswith("1d:"):
            n = kind[3:]
            return (f"  size_t g[3] = {{(size_t)({n} > 0 ? {n} : 1), 1, 1}}, l[3] = {{1, 1, 1}};\n"
                    f"  clshim_ndrange(g, l, [&] {{ ref_{sfx}::{call}; }});")
        x, y, z = kind[3:].split(",")
        return (f"  size_t g[3] = {{(size_t)((({x}) + 15) / 16 * 16), (size_t)((({y}) + 15) / 16 * 16), (size_t)({z})}};\n"
                f"  size_t l[3] = {{16, 16, 1}};\n"
                f"  clshim_ndrange(g, l, [&] {{ ref_{sfx}::{call}; }});")

    for name, params, call, kind in WRAPPERS:
        lines.append(f"void clref_{name}_{sfx}({params}) {{\n{launch(kind, call)}\n}}")
    for n, params in MADD.items():
        args = ", ".join(["dst"] + [f"s{i}, f{i}" for i in range(1, n + 1)] + ["N"])
        lines.append(f"void clref_madd{n}_{sfx}({params}) {{\n{launch('1d:N', f'madd{n}({args})')}\n}}")
    lines.append("}")
    return "\n".join(lines) + "\n"


def build(verbose=False):
    KS = _kernels_src()
    if not os.path.isdir(KS):
        raise FileNotFoundError(f"reference kernels not found at {KS}")
    os.makedirs(OUT, exist_ok=True)
    srcs = []
    for real, sfx in (("float", "f32"), ("double", "f64")):
        p = os.path.join(OUT, f"clref_{sfx}.cpp")
        with open(p, "w") as f:
            f.write(gen_tu(real, sfx))
        srcs.append(p)
    lib = os.path.join(OUT, "libclref.so")
    cmd = ["g++", "-std=gnu++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
           "-pthread", "-w", "-o", lib] + srcs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
