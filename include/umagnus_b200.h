/*
 * umagnus_b200.h -- C-ABI of the B200 (sm_100a) effective-field + LLG hot path.
 *
 * Drop-in replacement for the hot-path subset of the uMagNUS Go package
 * `opencl` (device-op layer) plus the engine-level stepper loop.  Every
 * entry point cites the reference function it replaces (path:line in the
 * uMagNUS source tree).  All arithmetic is float32 unless stated; device
 * arrays are structure-of-arrays, one float32 array per vector component,
 * x fastest (data/slice.go:53-100, data/slice.go:413 Index).
 *
 * Conventions kept from the reference:
 *   - a NULL parameter array means "uniform value = mul" (kernels_src/clh/amul.clh:5-7);
 *   - region maps are uint8 (NREGION = 256, engine/regions.go:11);
 *   - per-region LUTs hold 256 floats, symmetric inter-region LUTs hold
 *     256*257/2 = 32896 floats indexed by symidx (kernels_src/clh/exchange.clh:5);
 *   - the library never frees caller memory; plans/contexts are opaque
 *     handles with explicit free.
 * Every function returns 0 on success or a nonzero UMAG_E* status (the Go
 * shim maps nonzero to util.Fatal, keeping the reference's abort-on-error
 * behaviour); umag_last_error() describes the last failure.
 * All calls are stream-ordered on the library stream (umag_set_stream) and
 * must come from one host thread, like the reference's single command queue
 * (opencl/init.go:60,145).
 */
#ifndef UMAGNUS_B200_H
#define UMAGNUS_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define UMAG_OK 0
#define UMAG_E_CUDA 1        /* CUDA runtime error */
#define UMAG_E_ARG 2         /* invalid argument */
#define UMAG_E_UNSUPPORTED 3 /* size/feature outside what this build handles */
#define UMAG_E_NOMEM 4
#define UMAG_E_NOT_INIT 5
#define UMAG_E_SOLVER 6      /* time step underflow / NaN in the solver */
#define UMAG_E_TIMEOUT 7     /* a kernel gave up waiting for a bulk copy (bounded wait) */

/* ---- device bring-up (opencl/init.go) ------------------------------------ */
/* opencl/init.go:48 Init(gpu): select the device, create the stream. */
int umag_init(int device);
/* opencl/init.go:287 ReleaseAndClean. */
int umag_release(void);
const char* umag_last_error(void);
/* Run subsequent calls on a caller-owned cudaStream_t (NULL = library stream). */
int umag_set_stream(void* cuda_stream);
/* Wait for all work queued by the library (ClCmdQueue.Finish, opencl/init.go). */
int umag_sync(void);
/* Build/version string. */
const char* umag_version(void);

/* ---- memory (opencl/slice.go:14-193, opencl/buffer.go:25-106) ------------ */
int umag_malloc(void** ptr, size_t bytes);       /* opencl/slice.go:14 NewSlice / MemAlloc */
int umag_free(void* ptr);                        /* data/slice.go Free */
int umag_memcpy_htod(void* dst, const void* src, size_t bytes); /* opencl/init.go:275 data.Copy hooks */
int umag_memcpy_dtoh(void* dst, const void* src, size_t bytes);
int umag_memcpy_dtod(void* dst, const void* src, size_t bytes);
int umag_memset_f32(float* dst, float value, size_t n); /* opencl/slice.go:156-193 Memset / Zero */

/* ---- local field terms --------------------------------------------------- */
/* opencl/exchange.go:16 AddExchange (kernel kernels_src/cl/exchange.cl).
 * Weights 2/c^2 are formed in FP64 and rounded to float32 as the reference
 * does (opencl/exchange.go:18-20).  pbc = PBC_code bits (1:x, 2:y, 4:z). */
int umag_add_exchange(float* Bx, float* By, float* Bz, const float* mx, const float* my,
                      const float* mz, const float* Ms, float Ms_mul, const float* aLUT2d,
                      const uint8_t* regions, int Nx, int Ny, int Nz, double cx, double cy,
                      double cz, int pbc);
/* opencl/dmi.go:15 AddDMI (kernels_src/cl/dmi.cl): exchange + interfacial DMI. */
int umag_add_dmi(float* Hx, float* Hy, float* Hz, const float* mx, const float* my,
                 const float* mz, const float* Ms, float Ms_mul, const float* aLUT2d,
                 const float* dLUT2d, const uint8_t* regions, int Nx, int Ny, int Nz, double cx,
                 double cy, double cz, int pbc, int openbc);
/* opencl/anisotropy.go:153 AddUniaxialAnisotropy2 (uniaxialanisotropy2.cl). */
int umag_add_uniaxial_anisotropy2(float* Bx, float* By, float* Bz, const float* mx,
                                  const float* my, const float* mz, const float* Ms, float Ms_mul,
                                  const float* K1, float K1_mul, const float* K2, float K2_mul,
                                  const float* ux, float ux_mul, const float* uy, float uy_mul,
                                  const float* uz, float uz_mul, int N);
/* opencl/dmibulk.go AddDMIBulk (dmibulk.cl): exchange + bulk DMI, boundary
 * extrapolation of missing neighbours in x, y and z. */
int umag_add_dmi_bulk(float* Hx, float* Hy, float* Hz, const float* mx, const float* my,
                      const float* mz, const float* Ms, float Ms_mul, const float* aLUT2d,
                      const float* dLUT2d, const uint8_t* regions, int Nx, int Ny, int Nz, double cx,
                      double cy, double cz, int pbc, int openbc);
/* opencl/anisotropy.go AddCubicAnisotropy2 (cubicanisotropy2.cl): Kc1, Kc2,
 * Kc3 with axes c1, c2 (c3 = c1 x c2), each as (array or NULL, multiplier). */
int umag_add_cubic_anisotropy2(float* Bx, float* By, float* Bz, const float* mx, const float* my,
                               const float* mz, const float* Ms, float Ms_mul, const float* K1,
                               float K1_mul, const float* K2, float K2_mul, const float* K3, float K3_mul,
                               const float* const c1[3], const float c1_mul[3],
                               const float* const c2[3], const float c2_mul[3], int N);
/* opencl/region.go:13 RegionAddV (regionaddv.cl): dst += LUT[region]. */
int umag_region_addv(float* dx, float* dy, float* dz, const float* lutx, const float* luty,
                     const float* lutz, const uint8_t* regions, int N);
/* opencl/region.go:108 RegionDecode (regiondecode.cl). */
int umag_region_decode(float* dst, const float* lut, const uint8_t* regions, int N);

/* ---- thermal field --------------------------------------------------------
 * opencl/temperature.go:14 SetTemperature (temperature2.cl): B = noise *
 * sqrt(k2 * alpha * T / Ms), k2 = 2 kB / (GammaLL V dt) as float32. */
int umag_set_temperature(float* B, const float* noise, float k2, const float* Ms, float Ms_mul,
                         const float* temp, float temp_mul, const float* alpha, float alpha_mul, int N);
/* Standard normal noise for N cells (three components) of accepted step
 * `step` under `seed`: Philox4x32-10 of (cell, step) + Box-Muller.  Stands in
 * for the reference's device-dependent Threefry stream (opencl/rng.go,
 * engine/temperature.go:117-120): same distribution, reproducible on any
 * device. */
int umag_thermal_noise(float* nx, float* ny, float* nz, int N, unsigned long long seed, long long step);

/* ---- torque -------------------------------------------------------------- */
/* opencl/zeromask.go:12 ZeroMask (zeromask.cl): dst_c[i] = 0 where
 * maskLUT[regions[i]] != 0, for the three components. */
int umag_zero_mask(float* dx, float* dy, float* dz, const float* maskLUT, const uint8_t* regions, int N);
/* opencl/lltorque.go:16 LLTorque (lltorque2.cl); t may alias h. */
int umag_lltorque(float* tx, float* ty, float* tz, const float* mx, const float* my,
                  const float* mz, const float* hx, const float* hy, const float* hz,
                  const float* alpha, float alpha_mul, int N);
/* opencl/lltorque.go:97 LLNoPrecess (llnoprecess.cl). */
int umag_llnoprecess(float* tx, float* ty, float* tz, const float* mx, const float* my,
                     const float* mz, const float* hx, const float* hy, const float* hz, int N);

/* ---- linear combinations and normalisation ------------------------------- */
/* opencl/madd.go:111-413 Madd2..Madd7 on ncomp components at once:
 * dst[c] = sum_j fac[j] * src[j*ncomp + c], 2 <= nsrc <= 7, same rounding
 * order as madd<n>.cl.  dst may alias a source. */
int umag_madd(int ncomp, float* const* dst, int nsrc, const float* const* src, const float* fac,
              int N);
/* opencl/normalize.go:13 Normalize (normalize2.cl). vol may be NULL. */
int umag_normalize(float* vx, float* vy, float* vz, const float* vol, int N);
/* opencl/vecnorm.go:12 VecNorm, opencl/madd.go:60 Div, opencl/dotproduct.go AddDotProduct. */
int umag_vecnorm(float* dst, const float* ax, const float* ay, const float* az, int N);
int umag_div(float* dst, const float* a, const float* b, int N);
int umag_add_dot_product(float* dst, float prefactor, const float* ax, const float* ay,
                         const float* az, const float* bx, const float* by, const float* bz,
                         int N);

/* ---- reductions (opencl/reduce.go), results on the host ------------------ */
/* reduce.go:180 MaxVecNorm: max_i |v_i| (float32 max, FP64 sqrt). */
int umag_max_vec_norm(const float* x, const float* y, const float* z, int N, double* out);
/* reduce.go:214 MaxVecDiff: max_i |a_i - b_i|. */
int umag_max_vec_diff(const float* ax, const float* ay, const float* az, const float* bx,
                      const float* by, const float* bz, int N, double* out);
/* reduce.go:105 MaxAbs: max_i |v_i|. */
int umag_max_abs(const float* v, int N, double* out);
/* reduce.go:26 Sum / :54 Dot with compensated accumulation (float32 inputs,
 * Neumaier-compensated float32 per thread, two-sum tree, FP64 final). */
int umag_sum(const float* v, int N, double* out);
int umag_dot(const float* a, const float* b, int N, double* out);

/* ---- demag convolution (opencl/conv_demag.go) ---------------------------- */
typedef struct umag_demag umag_demag;
/* engine/demag.go:135-143 newellDemagConv: builds the Newell tensor in FP64
 * on the GPU (mag/newellDemagKernel.go:1108-1324), FFTs it in FP64 and
 * keeps the real, non-redundant spectrum in float32 (opencl/conv_demag.go:131-202).
 * pbc[3] must be zero in this build (no periodic images). */
int umag_demag_new_newell(int Nx, int Ny, int Nz, const int pbc[3], double cx, double cy,
                          double cz, int asymptotic_radius, int zero_self_demag,
                          umag_demag** out);
/* engine/demag.go:124-133 demagConv with EnableDemag (the reference's
 * default): mag/demagkernel.go:113-336 CalcDemagKernel, the brute-force
 * kernel (face charges integrated over the cells, point counts set by
 * `accuracy`, DemagAccuracy = 6 by default), built in FP64 on the GPU and
 * rounded to float32 like the reference's kernel slices. */
int umag_demag_new_brute(int Nx, int Ny, int Nz, const int pbc[3], double cx, double cy, double cz,
                         double accuracy, umag_demag** out);
/* opencl/conv_demag.go:27 NewDemag with a caller-supplied real-space kernel:
 * six host arrays (xx, yy, zz, yz, xz, xy) on the padded grid, doubles. */
int umag_demag_new_from_kernel(int Nx, int Ny, int Nz, const double* const kern[6],
                               umag_demag** out);
/* opencl/conv_demag.go:43 (*DemagConvolution).Exec: B = demag field of
 * MU0*Ms*vol*m (B is overwritten).  vol and Ms may be NULL.  Returns after
 * the field is complete (the reference's Exec waits for its kernels too);
 * UMAG_E_TIMEOUT if a pass gave up waiting for one of its bulk copies (the
 * count stays set, like a sticky CUDA error, until umag_debug_plant_fault
 * clears it). */
int umag_demag_exec(umag_demag* d, float* Bx, float* By, float* Bz, const float* mx,
                    const float* my, const float* mz, const float* vol, const float* Ms,
                    float Ms_mul);
/* One of the three passes of umag_demag_exec, for timing them one by one:
 * 0 = x/z forward transforms of MU0*Ms*vol*m into the plan's spectrum,
 * 1 = y transform, kernel multiply and inverse y transform in place,
 * 2 = inverse z/x transforms of the spectrum into B.  Running 0, 1, 2 in
 * order equals umag_demag_exec.  No counterpart in the reference. */
int umag_demag_exec_pass(umag_demag* d, int pass, float* Bx, float* By, float* Bz,
                         const float* mx, const float* my, const float* mz, const float* vol,
                         const float* Ms, float Ms_mul);
/* Copies the stored float32 kernel spectrum (6 arrays of (Px/2+1)(Py/2+1)(Pz/2+1),
 * reference layout kernmulrsymm3d.cl) to host arrays; for tests. */
int umag_demag_get_spectrum(umag_demag* d, float* const host[6]);
/* Copies the FP64 real-space Newell tensor (6 x Px*Py*Pz) to host; for tests. */
int umag_demag_get_kernel(umag_demag* d, double* const host[6]);
int umag_demag_padded_size(umag_demag* d, int P[3]);
int umag_demag_free(umag_demag* d);
/* Demag field for callers that cannot allocate device memory when they need
 * it (an external pool that owns the device, a runtime that forbids
 * allocation after start-up).  No counterpart in the reference.  It needs
 * neither umag_init nor a plan: K holds the six float32 kernel-spectrum
 * arrays (the layout umag_demag_get_spectrum returns, yz/xz may be NULL for
 * Nz == 1) on the device, and all working memory lives in one 16 MiB
 * __device__ array that every GPU loading this library keeps until the
 * process exits.  The driver reserves that array when the library's module
 * is loaded on a device: umag_init does this for its device, otherwise the
 * first call of this function does (and looks up the array's address) --
 * make one of the two on each device before an external pool claims the
 * device's memory and before any stream capture.  Meshes whose spectrum
 * and twiddles exceed 16 MiB, or without a compile-time FFT plan, return
 * UMAG_E_UNSUPPORTED.  Work is queued on `stream` (a cudaStream_t, NULL =
 * legacy default stream); every call shares the array, so calls that
 * overlap on the GPU (other streams, other host threads) race.  Calls no
 * cudaMalloc, cudaFree or other allocating routine. */
int umag_demag_exec_noalloc(int Nx, int Ny, int Nz, const float* const K[6], float* Bx, float* By, float* Bz,
                            const float* mx, const float* my, const float* mz, const float* vol, const float* Ms,
                            float Ms_mul, void* stream);

/* Test hook for the error paths of bounded device waits (no counterpart in
 * the reference): with sim == NULL, sets the device counter of timed-out
 * demag bulk copies that umag_demag_exec reports (0 clears it); with a
 * simulation, writes `code` into its device-side solver status, as a
 * device kernel does when a wait gives up (status 7).  Nothing on the GPU
 * faults or waits: the planted value is what the host-side checks read. */
typedef struct umag_sim umag_sim;
int umag_debug_plant_fault(umag_sim* sim, unsigned code);

/* ---- engine: a whole simulation on the device ---------------------------- */
/* Material and mesh description.  Uniform parameters use the *_mul value
 * with a NULL map; per-cell maps are device pointers owned by the caller
 * (regiondecode'd values, engine/parameter.go:37-45). */
typedef struct {
    int N[3];
    double cell[3];
    int pbc[3];
    const uint8_t* regions;        /* device, N cells; NULL = all region 0 */
    const float* vol;              /* device geometry mask or NULL */
    const float* Ms; float Ms_mul; /* saturation magnetisation A/m */
    const float* alpha; float alpha_mul;
    const float* Ku1; float Ku1_mul;
    const float* Ku2; float Ku2_mul;
    const float* anisU[3]; float anisU_mul[3];
    const float* aLUT;             /* device, 32896 floats (Aex inter-region LUT) */
    const float* dLUT;             /* device, 32896 floats (Dind LUT) or NULL */
    const float* bextLUT[3];       /* device, 256 floats each, or NULL (no Zeeman) */
    int enable_demag;              /* Newell demag (engine/demag.go EnableNewellDemag) */
    int openbc;                    /* engine/exchange.go OpenBC */
    int precess;                   /* engine/torque.go Precess */
    int asymptotic_radius;         /* engine/demag.go:27, default 32 */
    int demag_kernel;              /* 0 Newell (EnableNewellDemag), 1 brute force (EnableDemag) */
    double demag_accuracy;         /* brute force: DemagAccuracy (engine/demag.go:25); <= 0 -> 6 */
    const float* frozen_lut;       /* FrozenSpins per region (256 floats, device) or NULL
                                      (engine/torque.go:348-352: torque zeroed where != 0) */
    /* cubic anisotropy (engine/anisotropy.go:14-19, :54-74): Kc1..Kc3 and the
     * axes anisC1, anisC2, each (array or NULL, multiplier); off when all
     * three constants are zero */
    const float* Kc1; float Kc1_mul;
    const float* Kc2; float Kc2_mul;
    const float* Kc3; float Kc3_mul;
    const float* anisC1[3]; float anisC1_mul[3];
    const float* anisC2[3]; float anisC2_mul[3];
    const float* dbulkLUT;         /* bulk DMI LUT (engine/exchange.go:49-66 Dbulk) or NULL;
                                      exclusive with dLUT */
    /* thermal field (engine/temperature.go): Temp (array or NULL, multiplier);
     * off when zero; noise from umag_thermal_noise's generator under therm_seed
     * (ThermSeed), drawn anew for every accepted step */
    const float* temp; float temp_mul;
    unsigned long long therm_seed;
    /* NoDemagSpins per region (256 floats, device) or NULL (engine/demag.go:67-98):
     * cells of regions with a non-zero value neither make nor feel demag field */
    const float* nodemag_lut;
} umag_sim_params;

/* Solver knobs, engine/run.go:14-43 (defaults by umag_solver_defaults). */
typedef struct {
    int solver;      /* 1 Euler, 2 Heun, 3 RK23, 4 RK4, 5 RK45DP (engine/run.go:83-95) */
    double dt, min_dt, max_dt, fix_dt, max_err, rel_err, min_slope, headroom, gamma_ll;
} umag_solver_params;

/* Snapshot of the solver state (engine/run.go globals). */
typedef struct {
    double time, dt, last_err, peak_err, last_torque;
    long long nsteps, nundone, nevals;
    int status;      /* 0 ok; nonzero: UMAG_E_SOLVER cause code */
} umag_solver_state;

void umag_solver_defaults(umag_solver_params* p);
int umag_sim_new(const umag_sim_params* p, const umag_solver_params* s, umag_sim** out);
int umag_sim_free(umag_sim* s);
/* engine/magnetization.go:55 SetArray: copy m (device, 3 arrays) and normalise. */
int umag_sim_set_m(umag_sim* s, const float* mx, const float* my, const float* mz);
int umag_sim_get_m(umag_sim* s, float* mx, float* my, float* mz);   /* device destinations */
/* Checkpoint resume: copy a state saved by umag_sim_get_m back without
 * normalising it again (so the trajectory continues bit for bit). */
int umag_sim_restore_m(umag_sim* s, const float* mx, const float* my, const float* mz);
/* Device pointers of the current magnetisation (valid until the next step). */
int umag_sim_m_ptrs(umag_sim* s, float** m3);
/* engine/torque.go:124 SetTorque / engine/effectivefield.go:14 SetEffectiveField
 * for the current m: writes torque (and B_eff if non-NULL) to device arrays. */
int umag_sim_torque(umag_sim* s, float* tx, float* ty, float* tz, float* bx, float* by, float* bz);
/* engine/run.go:238 step(): n calls of Stepper.Step() without host
 * synchronisation (device-side step controller). */
int umag_sim_steps(umag_sim* s, int n);
/* engine/run.go:190 Run(seconds): steps until the simulated time reaches
 * t+seconds (alarm honoured by adaptDt, engine/run.go:181-184), checking
 * the device time every `chunk` steps; max_steps bounds the loop. */
int umag_sim_run(umag_sim* s, double seconds, int chunk, long long max_steps);
int umag_sim_get_state(umag_sim* s, umag_solver_state* st);
int umag_sim_set_time(umag_sim* s, double time, double dt);
/* Average m over the magnet (engine/average.go:29-40), compensated sum. */
int umag_sim_average_m(umag_sim* s, double avg[3]);
/* Capture `steps_per_graph` steps into a CUDA graph and replay it (1 = on,
 * 0 = plain stream launches).  Default on. */
int umag_sim_use_graph(umag_sim* s, int enable, int steps_per_graph);
/* Number of kernel launches one step issues (for launch accounting). */
int umag_sim_launches_per_step(umag_sim* s, int* n);
/* Enqueue n effective-field + torque evaluations of the current m into the
 * FSAL slot (the value it already holds), without host synchronisation; for
 * timing the field evaluation alone.  No reference counterpart. */
int umag_sim_torque_evals(umag_sim* s, int n);
/* engine/energy.go:27-35 GetTotalEnergy and its terms for the current m, in
 * joules: E[0] total, E[1] demag (engine/demag.go:146 GetDemagEnergy),
 * E[2] exchange including DMI (engine/exchange.go:79), E[3] uniaxial
 * anisotropy (engine/anisotropy.go:210), E[4] Zeeman (engine/zeeman.go:15).
 * Each term is -k V sum(M_full . B_term) with float32 dot products per cell
 * and FP64 accumulation. */
int umag_sim_energies(umag_sim* s, double E[5]);
/* engine/energy.go:36-42 SetTotalEdens (Edens_total) for the current m:
 * per-cell total energy density in J/m^3 into dst (device, N floats), each
 * term added in float32 as opencl.AddDotProduct does, in the terms'
 * registration order. */
int umag_sim_energy_density(umag_sim* s, float* dst);
/* engine/relax.go:23-112 Relax(): RK23 without precession; steps while the
 * total energy decreases (checked every 3 steps), then while the mean
 * squared torque decreases, lowering MaxErr by sqrt(2) down to 1e-9 --
 * or, with torque_threshold > 0 (RelaxTorqueThreshold), while the maximum
 * torque exceeds it.  The time is left unchanged; solver, MaxErr, FixDt and
 * precession are restored afterwards. */
int umag_sim_relax(umag_sim* s, double torque_threshold);
/* Between runs, the script assignments SetSolver(n) / FixDt / MaxErr / RelErr /
 * MinDt / MaxDt / Headroom / MinSlope / GammaLL (engine/run.go:14-43, :92-125):
 * the stepper restarts, time and dt are kept (sp->dt is ignored), so FixDt = 0
 * resumes adaptive stepping from the last dt. */
int umag_sim_set_solver(umag_sim* s, const umag_solver_params* sp);
/* Between runs, reassign one material parameter or vector component (Msat = ..., alpha = ...;
 * engine/parameter.go SetValue / setRegion): `values` a device map of N
 * floats owned by the caller, or NULL for the uniform value `mul`.  The next
 * step recomputes the FSAL torque and recaptures its graphs. */
#define UMAG_PARAM_MSAT 0
#define UMAG_PARAM_ALPHA 1
#define UMAG_PARAM_KU1 2
#define UMAG_PARAM_KU2 3
#define UMAG_PARAM_TEMP 4
#define UMAG_PARAM_ANISU_X 5   /* AnisU components: _X + 0, 1, 2 */
#define UMAG_PARAM_KC1 8
#define UMAG_PARAM_KC2 9
#define UMAG_PARAM_KC3 10
#define UMAG_PARAM_ANISC1_X 11  /* AnisC1 components: _X + 0, 1, 2 */
#define UMAG_PARAM_ANISC2_X 14  /* AnisC2 components: _X + 0, 1, 2 */
int umag_sim_set_param(umag_sim* s, int which, const float* values, float mul);
/* Launch shapes of the per-cell kernels (no reference counterpart; chosen by
 * the autotuner, umagnus_b200/autotune.py).  Results do not depend on them:
 * every cell's arithmetic is the same and the reductions are maxima.
 * torque_block: CTA shape (x multiple of 32, x*y <= 256) of the field +
 * torque kernel; stage_threads (64, 128 or 256) and stage_waves (CTAs per SM
 * cap, 1..64) of the stage sums; err_waves of the error norms; torque_tma
 * (1 = default) feeds the torque kernel's stencils from TMA-loaded tiles with
 * a halo where the mesh allows it (non-periodic, Nx a multiple of 4, no
 * region map, no bulk DMI, block width <= 248), 0 = plain global loads. */
typedef struct {
    int torque_block[2];
    int stage_threads, stage_waves, err_waves;
    int torque_tma;
} umag_tuning;
int umag_sim_get_tuning(umag_sim* s, umag_tuning* t);
int umag_sim_set_tuning(umag_sim* s, const umag_tuning* t);

/* ---- ensembles: many independent simulations at once --------------------
 * No counterpart in the reference, which runs one simulation per process.
 * Each instance has its own mesh (instances with the same mesh and cell
 * size are batched into one set of launches), its own uniform material and
 * applied field, its own time, dt and step controller (the solver knobs of
 * `sp` are shared); Newell demag when enable_demag.  Region maps, per-cell
 * maps, geometry masks and PBC: general instances (umag_ens_new_general). */
typedef struct {
    int N[3];
    double cell[3];
    float Ms, Aex, alpha, Dind, Ku1, Ku2;
    float anisU[3];
    float B_ext[3];   /* T */
} umag_ens_instance;
typedef struct umag_ens umag_ens;
int umag_ens_new(int n, const umag_ens_instance* instances, const umag_solver_params* sp, int enable_demag,
                 umag_ens** out);
/* As umag_ens_new, with general instances: where general[i] is not NULL,
 * instance i is the simulation umag_sim_new would make from *general[i]
 * (region maps and LUTs, per-cell parameters, geometry, PBC, thermal field,
 * every term; enable_demag taken from it) and `instances[i]` is not read
 * (`instances` may be NULL when every instance is general).  A general
 * instance is a class of its own, stepped by the single-simulation kernels
 * in its own CUDA graph on its own stream, concurrently with the other
 * classes; its trajectory equals the lone simulation's bit for bit.  The
 * device arrays *general[i] points to must stay valid until umag_ens_free.
 * No counterpart in the reference (one simulation per process there). */
int umag_ens_new_general(int n, const umag_ens_instance* instances, const umag_sim_params* const* general,
                         const umag_solver_params* sp, int enable_demag, umag_ens** out);
int umag_ens_free(umag_ens* e);
/* host arrays of 3*N floats (SoA); set_m normalises (engine/magnetization.go:34;
 * a general instance within its geometry) */
int umag_ens_set_m(umag_ens* e, int i, const float* host_m);
int umag_ens_get_m(umag_ens* e, int i, float* host_m);
int umag_ens_get_state(umag_ens* e, int i, umag_solver_state* st);
/* engine/run.go:190 Run(seconds) for every instance from its own current
 * time.  Each class (instances of one mesh) replays its own CUDA graph of 16
 * steps on its own stream, fed and checked by the host every `chunk`
 * replays independently of the other classes (at most max_replays replays
 * per class); finished instances leave their class's batch (compaction) and
 * return at the next run.  No counterpart in the reference. */
int umag_ens_run(umag_ens* e, double seconds, int chunk, long long max_replays);
int umag_ens_count(umag_ens* e, int* n_instances, int* n_classes);
/* Classes (instances of one mesh and cell size, numbered in the order their
 * first instance appears): the mesh and the number of instances of class
 * `cls`.  No counterpart in the reference. */
int umag_ens_class_info(umag_ens* e, int cls, int N[3], int* n_instances);
/* 1 when class `cls` is a general instance (umag_ens_new_general), else 0. */
int umag_ens_class_general(umag_ens* e, int cls, int* general);
/* Launch shapes of class `cls`'s batched per-cell kernels (the fields of
 * umag_tuning; the torque kernel of a batch reads global memory, so
 * torque_tma is ignored).  Speed only: every instance's arithmetic is the
 * same under every shape.  No counterpart in the reference. */
int umag_ens_get_tuning(umag_ens* e, int cls, umag_tuning* t);
int umag_ens_set_tuning(umag_ens* e, int cls, const umag_tuning* t);

/* ---- differentiable simulation: forward RK4 and its adjoint --------------
 * No counterpart in the reference (which has no gradients).  A thin film or
 * block (open or periodic, optionally with a geometry) with a per-cell Ms
 * map, uniform exchange Aex, uniaxial Ku1 along anisU, Zeeman field B_ext,
 * an optional fixed interfacial DMI and damping alpha, integrated by fixed-step RK4
 * (engine/rk4.go with FixDt) or Heun (engine/heun.go) for nsteps steps; m is checkpointed every K
 * steps.  Loss = w_probe * (mean over states avg_from..nsteps of the mean
 * m_z over the probe window of layer 0) + w_target * |<m>(final) - target|^2.
 * umag_adj_backward returns dLoss/dMs (per cell), dLoss/dAex, dLoss/dKu1,
 * dLoss/dB_ext and, if gm0 is not NULL, dLoss/dm0, by hand-written
 * vector-Jacobian products through the steps, recomputing each segment of
 * K steps from its checkpoint. */
typedef struct {
    int N[3];
    double cell[3];
    float alpha;
    float anisU[3];
    int enable_demag;
    int demag_kernel;       /* 0 Newell, 1 brute force (engine/demag.go) */
    double demag_accuracy;  /* brute force; <= 0: 6 */
    double dt, gamma_ll;    /* gamma_ll <= 0: 1.7595e11 */
    int nsteps, K;
    int probe[4];           /* x0, y0, width, height (cells, layer 0) */
    int avg_from;           /* 1 <= avg_from <= nsteps */
    double w_probe, w_target;
    double target[3];
    int no_graph;           /* 1: plain stream launches instead of CUDA graphs */
    int solver;             /* 4 (or 0) RK4, 2 Heun (engine/heun.go with FixDt) */
    float Dind;             /* uniform interfacial DMI (J/m^2; 0 = exchange only): dmi.cl's
                               exchange + DMI stencil, a fixed (not differentiated) parameter */
    int pbc[3];             /* periodic repetitions per axis (engine/mesh.go SetPBC; 0 = open):
                               the demag kernel's images and wrapped stencils, as umag_sim_params */
    const float* vol;       /* device geometry (cell volume fractions, N floats) or NULL, as
                               umag_sim_params.vol: m = 0 where it is 0, demag source Ms*vol*m;
                               it must stay valid while the handle is used */
    const uint8_t* regions; /* device region map (N bytes, values < nregions) or NULL; with it
                               Aex, Ku1 and B_ext are per region (the _regions entry points), the
                               exchange of a cell pair the engine's harmonic-mean LUT
                               (engine/exchange.go:153-167); not with Dind */
    int nregions;           /* 1..256 with a region map */
} umag_adj_params;
typedef struct umag_adj umag_adj;
int umag_adj_new(const umag_adj_params* p, umag_adj** out);
int umag_adj_free(umag_adj* a);
/* device arrays: m0 3N floats (normalised first), Ms N floats */
int umag_adj_forward(umag_adj* a, const float* m0, const float* Ms, float Aex, float Ku1, const float B_ext[3],
                     double* loss);
/* final m of the last forward (device, 3N floats) */
int umag_adj_final_m(umag_adj* a, float* m);
/* gradients of the last forward's loss: gMs device N floats, gm0 device 3N
 * floats or NULL; the scalars on the host */
int umag_adj_backward(umag_adj* a, float* gMs, float* gm0, double* gAex, double* gKu1, double gB_ext[3]);
/* With a region map: Aex, Ku1 host arrays of nregions values, B_ext host
 * [nregions][3] (T); the gradients per region in host arrays of the same
 * shapes (gMs device N floats, gm0 device 3N floats or NULL).  No
 * counterpart in the reference. */
int umag_adj_forward_regions(umag_adj* a, const float* m0, const float* Ms, const float* Aex, const float* Ku1,
                             const float* B_ext, double* loss);
int umag_adj_backward_regions(umag_adj* a, float* gMs, float* gm0, double* gAex, double* gKu1, double* gB_ext);

/* ---- field files (oommf/*.go, dump/*.go) ----------------------------------
 * Host arrays of float32, structure of arrays [c][z][y][x] (x fastest), the
 * layout of data.Slice.Tensors(); numbers in headers and text data are
 * written as the reference's Go fmt %v writes them. */
typedef struct {
    int N[3];          /* xnodes, ynodes, znodes */
    int ncomp;         /* valuedim */
    double cell[3];    /* x/y/z stepsize (m) */
    double time;       /* total simulation time (s) */
    char title[64];
    char unit[32];
} umag_field_info;
/* oommf/oommf.go:16-46 Read / ReadFile and dump/read.go:17 Read: OVF 1.0
 * (text, binary 4, binary 8, big-endian), OVF 2.0 (text, binary 4,
 * binary 8) or the "#dump002" format (CRC-64 checked), detected from the
 * file's first bytes.  _info reads the header only. */
int umag_field_read_info(const char* path, umag_field_info* info);
int umag_field_read(const char* path, float* dst, size_t capacity, umag_field_info* info);
/* oommf/ovf2.go:13 WriteOVF2 (version 2) and oommf/ovf1.go:14 WriteOVF1
 * (version 1, 3 components only); format "text" or "binary 4". */
int umag_ovf_write(const char* path, const float* src, const umag_field_info* info, const char* format,
                   int version);
/* dump/write.go:17 Write: the legacy "#dump002" format with its CRC-64. */
int umag_dump_write(const char* path, const float* src, const umag_field_info* info);
/* A number as Go's fmt %v prints it (bits 64: float64, 32: float32), as
 * the table writer (engine/table.go:112-133) needs. */
int umag_format_float(double v, int bits, char* buf, int cap);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
