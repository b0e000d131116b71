/*
 * umag_oracle.h -- CPU oracle for the uMagNUS effective-field + LLG hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain-C restatement of the
 * reference algorithms (uMagNUS 2.3.0) used as the checker for the CUDA
 * implementation in umagnus_b200/.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / --impl reference leg may load it.  The product
 * path never links, calls or falls back to it.
 *
 * Every function cites the reference file:line it restates.  Two numeric
 * variants exist for the per-cell kernels: *_f32 follows the reference's
 * float32 evaluation order (compile with -ffp-contract=off, like the OpenCL
 * program that is built without -cl-mad-enable, opencl/init.go:175) and
 * *_f64 is the uMagNUS64 (FP64) oracle.  The FFT is always FP64: the
 * reference's float32 FFT library rounding is not reproducible, so demag
 * results are compared within a stated tolerance, not bit for bit.
 */
#ifndef UMAG_ORACLE_H
#define UMAG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- geometry ----------------------------------------------------------- */
/* mag/demagkernel.go:404-420 padSize (SMALL_N = 5 only for z). */
void orc_pad_size(const int size[3], const int pbc[3], int padded[3]);

/* ---- Newell demag tensor (FP64) ---------------------------------------- */
/* mag/newellDemagKernel.go:1108-1324 CalcNewellDemagKernel.  Writes the six
 * real-space components (order xx, yy, zz, yz, xz, xy) on the padded grid
 * P = padSize(size, pbc); each array holds Px*Py*Pz doubles, x fastest.
 * For a 2D padded grid (Pz == 1) xz and yz are written as zeros. */
int orc_newell_kernel(const int size[3], const int pbc[3], const double cellsize[3],
                      int asymptotic_radius, int zero_self_demag, double* K[6]);

/* mag/demagkernel.go:113-336 CalcDemagKernel: brute-force kernel (FP64
 * integration, float32 result as the reference stores it), six arrays
 * (xx yy zz yz xz xy) of the padded grid. */
int orc_brute_kernel(const int size[3], const int pbc[3], const double cellsize[3], double accuracy,
                     float* const K[6]);

/* Individual Newell pieces, exported for the golden tests. */
double orc_newell_f(double x, double y, double z);
double orc_newell_g(double x, double y, double z);
double orc_self_demag_nx(double x, double y, double z);

/* opencl/conv_demag.go:155-201 + opencl/conv_common.go:27-53: real parts of
 * the R2C FFT of each kernel component, non-redundant y/z half only,
 * scaled by 1/(Px*Py*Pz).  Output per component: (Px/2+1)*(Py/2+1)*(Pz/2+1)
 * doubles, x fastest.  round_f32 != 0 first rounds the real-space kernel to
 * float32 like the reference's float32 kernel slices.  Returns the max
 * |imag|*sqrt(scale) (the reference's FFT_IMAG_TOLERANCE check). */
double orc_kernel_spectrum(const int P[3], double* const K[6], int round_f32, double* Kf[6]);

/* ---- demag convolution -------------------------------------------------- */
/* opencl/conv_demag.go:43-129 + copypadmul2.cl + kernmulrsymm*.cl + copyunpad.cl.
 * B is OVERWRITTEN (demag is the first term of SetEffectiveField).  Kf as
 * produced by orc_kernel_spectrum; vol may be NULL; Ms NULL -> Ms_mul. */
void orc_demag_f32(const int N[3], const int P[3], double* const Kf[6],
                   float* B[3], float* const m[3], const float* vol,
                   const float* Ms, float Ms_mul);
void orc_demag_f64(const int N[3], const int P[3], double* const Kf[6],
                   double* B[3], double* const m[3], const double* vol,
                   const double* Ms, double Ms_mul);

/* In-place complex FFT (FP64) over a strided line; sign -1 forward. */
void orc_fft_line(double* re_im, int n, int sign);

/* ---- per-cell kernels (float32 and float64) ----------------------------- */
#define ORC_DECL(R, S)                                                                        \
void orc_add_exchange_##S(R* B[3], R* const m[3], const R* Ms, R Ms_mul, const R* aLUT2d,     \
                          const uint8_t* regions, R wx, R wy, R wz, int Nx, int Ny, int Nz,   \
                          int pbc);                                                           \
void orc_add_dmi_##S(R* H[3], R* const m[3], const R* Ms, R Ms_mul, const R* aLUT2d,          \
                     const R* dLUT2d, const uint8_t* regions, R cx, R cy, R cz, int Nx,       \
                     int Ny, int Nz, int pbc, int openbc);                                    \
void orc_add_uniaxial2_##S(R* B[3], R* const m[3], const R* Ms, R Ms_mul, const R* K1,        \
                           R K1_mul, const R* K2, R K2_mul, R* const u[3],                    \
                           const R u_mul[3], int N);                                          \
void orc_add_cubic2_##S(R* B[3], R* const m[3], const R* Ms, R Ms_mul, const R* K1, R K1_mul,  \
                        const R* K2, R K2_mul, const R* K3, R K3_mul, R* const c1[3],          \
                        const R c1_mul[3], R* const c2[3], const R c2_mul[3], int N);          \
void orc_add_dmibulk_##S(R* H[3], R* const m[3], const R* Ms, R Ms_mul, const R* aLUT2d,      \
                         const R* dLUT2d, const uint8_t* regions, R cx, R cy, R cz, int Nx,   \
                         int Ny, int Nz, int pbc, int openbc);                                \
void orc_set_temperature_##S(R* B, const R* noise, R k2, const R* Ms, R Ms_mul, const R* temp,  \
                             R temp_mul, const R* alpha, R alpha_mul, int N);                 \
void orc_region_addv_##S(R* dst[3], R* const lut[3], const uint8_t* regions, int N);          \
void orc_region_decode_##S(R* dst, const R* lut, const uint8_t* regions, int N);              \
void orc_lltorque_##S(R* t[3], R* const m[3], R* const h[3], const R* alpha, R alpha_mul,     \
                      int N);                                                                 \
void orc_llnoprecess_##S(R* t[3], R* const m[3], R* const h[3], int N);                       \
void orc_madd_##S(R* dst, int nsrc, R* const src[], const R fac[], int N);                    \
void orc_normalize_##S(R* v[3], const R* vol, int N);                                         \
void orc_vecnorm_##S(R* dst, R* const a[3], int N);                                           \
void orc_div_##S(R* dst, const R* a, const R* b, int N);                                      \
void orc_add_dot_product_##S(R* dst, R prefactor, R* const a[3], R* const b[3], int N);       \
double orc_max_vec_norm_##S(R* const v[3], int N);                                            \
double orc_max_vec_diff_##S(R* const a[3], R* const b[3], int N);                             \
double orc_max_abs_##S(const R* v, int N);                                                    \
double orc_sum_##S(const R* v, int N);                                                        \
double orc_dot_##S(const R* a, const R* b, int N);

ORC_DECL(float, f32)
ORC_DECL(double, f64)
#undef ORC_DECL

/* engine/exchange.go:153-201: inter-region LUT from per-region values. */
void orc_exch_lut_f32(const float ex[256], const float scale[32896], const float inter[32896],
                      float lut[32896]);
void orc_exch_lut_f64(const double ex[256], const double scale[32896], const double inter[32896],
                      double lut[32896]);

/* ---- whole simulation (engine restated) ----------------------------- */
typedef struct {
    int N[3], pbc[3];
    double cell[3];
    /* material (uniform value in *_mul when the pointer is NULL) */
    const void *Ms, *alpha, *Ku1, *Ku2, *u[3], *vol;
    double Ms_mul, alpha_mul, Ku1_mul, Ku2_mul, u_mul[3];
    const void *aLUT, *dLUT;      /* 32896-entry symmetric LUTs (A and D) */
    const uint8_t* regions;       /* N cells, never NULL */
    const void* bext_lut[3];      /* 256 entries each, NULL = no Zeeman */
    int enable_demag, dmi, openbc, precess, anis;
    double* Kf[6];                /* kernel spectrum (orc_kernel_spectrum) */
    int P[3];
    /* cubic anisotropy (engine/anisotropy.go:54-74) and bulk DMI (engine/exchange.go:60-61) */
    const void *Kc1, *Kc2, *Kc3, *c1[3], *c2[3];
    double Kc1_mul, Kc2_mul, Kc3_mul, c1_mul[3], c2_mul[3];
    int cubic;
    const void* dbLUT;            /* 32896-entry bulk DMI LUT or NULL */
    /* per-region LUTs (256 entries) or NULL: NoDemagSpins (engine/demag.go:67-98)
     * and FrozenSpins (engine/torque.go:348-352) */
    const void *nodemag, *frozen;
} orc_system;

typedef struct {
    double time, dt, alarm;
    double max_err, rel_err, min_dt, max_dt, fix_dt, headroom, min_slope, gamma_ll;
    double last_err, peak_err, last_torque;
    long nsteps, nundone, nevals;
    int solver;                   /* 2 heun, 3 rk23, 4 rk4, 5 rk45dp (engine/run.go:83-95) */
    int have_k1;                  /* FSAL k1 valid */
    int status;                   /* 0 ok, nonzero = failure (dt underflow) */
} orc_solver;

void orc_solver_defaults(orc_solver* s);
/* engine/torque.go:124-144 + engine/effectivefield.go:14-24, float32 / float64.
 * m and tau are 3*N arrays (SoA). */
void orc_torque_f32(const orc_system* sys, float* tau, const float* m, float* beff_out);
void orc_torque_f64(const orc_system* sys, double* tau, const double* m, double* beff_out);
/* One Stepper.Step() (engine/rk45dp.go, rk23.go, heun.go, rk4.go).  k1 is the
 * caller-held FSAL buffer (3N).  Returns 1 if accepted. */
int orc_step_f32(const orc_system* sys, orc_solver* s, float* m, float* k1);
int orc_step_f64(const orc_system* sys, orc_solver* s, double* m, double* k1);

#ifdef __cplusplus
}
#endif
#endif
