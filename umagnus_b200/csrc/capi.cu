// capi.cu -- extern "C" entry points declared in include/umagnus_b200.h.
#include <cstring>

#include "common.cuh"
#include "demag.cuh"
#include "engine.cuh"
#include "ops.cuh"

using namespace umag;

extern "C" {

int umag_init(int device) { return init_device(device); }
int umag_release(void) { return release_device(); }
const char* umag_last_error(void) { return last_error(); }
const char* umag_version(void) { return "umagnus_b200 1.0 (sm_100a)"; }

int umag_debug_plant_fault(umag_sim* sim, unsigned code) {
    UMAG_TRY(ensure_init());
    if (sim == nullptr) return demag_set_slab_timeouts(code);
    return sim_plant_status(sim, (int)code);
}

int umag_set_stream(void* s) {
    UMAG_TRY(ensure_init());
    ctx().stream = s ? (cudaStream_t)s : ctx().own_stream;
    return UMAG_OK;
}

int umag_sync(void) {
    UMAG_TRY(ensure_init());
    UMAG_CUDA(cudaStreamSynchronize(ctx().stream));
    return UMAG_OK;
}

int umag_malloc(void** p, size_t bytes) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(p != nullptr, "NULL pointer");
    if (cudaMalloc(p, bytes ? bytes : 1) != cudaSuccess) return set_error(UMAG_E_NOMEM, "cudaMalloc(%zu)", bytes);
    return UMAG_OK;
}
int umag_free(void* p) {
    UMAG_TRY(ensure_init());
    UMAG_CUDA(cudaFree(p));
    return UMAG_OK;
}
int umag_memcpy_htod(void* dst, const void* src, size_t bytes) {
    UMAG_TRY(ensure_init());
    UMAG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx().stream));
    UMAG_CUDA(cudaStreamSynchronize(ctx().stream));
    return UMAG_OK;
}
int umag_memcpy_dtoh(void* dst, const void* src, size_t bytes) {
    UMAG_TRY(ensure_init());
    UMAG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx().stream));
    UMAG_CUDA(cudaStreamSynchronize(ctx().stream));
    return UMAG_OK;
}
int umag_memcpy_dtod(void* dst, const void* src, size_t bytes) {
    UMAG_TRY(ensure_init());
    UMAG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx().stream));
    return UMAG_OK;
}
int umag_memset_f32(float* dst, float v, size_t n) { return memset_f32(dst, v, n); }

int umag_add_exchange(float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
                      const float* Ms, float Ms_mul, const float* aLUT2d, const uint8_t* regions, int Nx, int Ny,
                      int Nz, double cx, double cy, double cz, int pbc) {
    return add_exchange(Bx, By, Bz, mx, my, mz, Ms, Ms_mul, aLUT2d, regions, Nx, Ny, Nz, cx, cy, cz, pbc);
}
int umag_add_dmi(float* Hx, float* Hy, float* Hz, const float* mx, const float* my, const float* mz, const float* Ms,
                 float Ms_mul, const float* aLUT2d, const float* dLUT2d, const uint8_t* regions, int Nx, int Ny,
                 int Nz, double cx, double cy, double cz, int pbc, int openbc) {
    return add_dmi(Hx, Hy, Hz, mx, my, mz, Ms, Ms_mul, aLUT2d, dLUT2d, regions, Nx, Ny, Nz, cx, cy, cz, pbc, openbc);
}
int umag_add_uniaxial_anisotropy2(float* Bx, float* By, float* Bz, const float* mx, const float* my,
                                  const float* mz, const float* Ms, float Ms_mul, const float* K1, float K1_mul,
                                  const float* K2, float K2_mul, const float* ux, float ux_mul, const float* uy,
                                  float uy_mul, const float* uz, float uz_mul, int N) {
    UniaxParams p{Ms, K1, K2, ux, uy, uz, Ms_mul, K1_mul, K2_mul, ux_mul, uy_mul, uz_mul};
    return add_uniaxial(Bx, By, Bz, mx, my, mz, p, N);
}
int umag_add_dmi_bulk(float* Hx, float* Hy, float* Hz, const float* mx, const float* my, const float* mz,
                      const float* Ms, float Ms_mul, const float* aLUT2d, const float* dLUT2d, const uint8_t* regions,
                      int Nx, int Ny, int Nz, double cx, double cy, double cz, int pbc, int openbc) {
    return add_dmibulk(Hx, Hy, Hz, mx, my, mz, Ms, Ms_mul, aLUT2d, dLUT2d, regions, Nx, Ny, Nz, cx, cy, cz, pbc,
                       openbc);
}
int umag_add_cubic_anisotropy2(float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
                               const float* Ms, float Ms_mul, const float* K1, float K1_mul, const float* K2,
                               float K2_mul, const float* K3, float K3_mul, const float* const c1[3],
                               const float c1_mul[3], const float* const c2[3], const float c2_mul[3], int N) {
    UMAG_REQUIRE(c1 && c1_mul && c2 && c2_mul, "NULL axis arguments");
    CubicParams p{Ms, K1, K2, K3, {c1[0], c1[1], c1[2]}, {c2[0], c2[1], c2[2]}, Ms_mul, K1_mul, K2_mul, K3_mul,
                  {c1_mul[0], c1_mul[1], c1_mul[2]}, {c2_mul[0], c2_mul[1], c2_mul[2]}};
    return add_cubic(Bx, By, Bz, mx, my, mz, p, N);
}
int umag_region_addv(float* dx, float* dy, float* dz, const float* lx, const float* ly, const float* lz,
                     const uint8_t* regions, int N) {
    return region_addv(dx, dy, dz, lx, ly, lz, regions, N);
}
int umag_region_decode(float* dst, const float* lut, const uint8_t* regions, int N) {
    return region_decode(dst, lut, regions, N);
}
int umag_thermal_noise(float* nx, float* ny, float* nz, int N, unsigned long long seed, long long step) {
    return thermal_noise(nx, ny, nz, N, (uint64_t)seed, step);
}
int umag_set_temperature(float* B, const float* noise, float k2, const float* Ms, float Ms_mul, const float* temp,
                         float temp_mul, const float* alpha, float alpha_mul, int N) {
    return set_temperature(B, noise, k2, Ms, Ms_mul, temp, temp_mul, alpha, alpha_mul, N);
}
int umag_zero_mask(float* dx, float* dy, float* dz, const float* maskLUT, const uint8_t* regions, int N) {
    return zero_mask(dx, dy, dz, maskLUT, regions, N);
}
int umag_lltorque(float* tx, float* ty, float* tz, const float* mx, const float* my, const float* mz,
                  const float* hx, const float* hy, const float* hz, const float* alpha, float alpha_mul, int N) {
    return torque(tx, ty, tz, mx, my, mz, hx, hy, hz, alpha, alpha_mul, N, 1);
}
int umag_llnoprecess(float* tx, float* ty, float* tz, const float* mx, const float* my, const float* mz,
                     const float* hx, const float* hy, const float* hz, int N) {
    return torque(tx, ty, tz, mx, my, mz, hx, hy, hz, nullptr, 0.f, N, 0);
}
int umag_madd(int ncomp, float* const* dst, int nsrc, const float* const* src, const float* fac, int N) {
    return madd(ncomp, dst, nsrc, src, fac, N);
}
int umag_normalize(float* vx, float* vy, float* vz, const float* vol, int N) { return normalize(vx, vy, vz, vol, N); }
int umag_vecnorm(float* dst, const float* ax, const float* ay, const float* az, int N) {
    return vecnorm(dst, ax, ay, az, N);
}
int umag_div(float* dst, const float* a, const float* b, int N) { return umag::div(dst, a, b, N); }
int umag_add_dot_product(float* dst, float pre, const float* ax, const float* ay, const float* az, const float* bx,
                         const float* by, const float* bz, int N) {
    return add_dot(dst, pre, ax, ay, az, bx, by, bz, N);
}
int umag_max_vec_norm(const float* x, const float* y, const float* z, int N, double* out) {
    return max_vec_norm(x, y, z, N, out);
}
int umag_max_vec_diff(const float* ax, const float* ay, const float* az, const float* bx, const float* by,
                      const float* bz, int N, double* out) {
    return max_vec_diff(ax, ay, az, bx, by, bz, N, out);
}
int umag_max_abs(const float* v, int N, double* out) { return max_abs(v, N, out); }
int umag_sum(const float* v, int N, double* out) { return sum_dot(v, nullptr, N, out); }
int umag_dot(const float* a, const float* b, int N, double* out) {
    UMAG_REQUIRE(b != nullptr, "NULL argument");
    return sum_dot(a, b, N, out);
}

int umag_demag_new_newell(int Nx, int Ny, int Nz, const int pbc[3], double cx, double cy, double cz,
                          int asymptotic_radius, int zero_self_demag, umag_demag** out) {
    return demag_new_newell(Nx, Ny, Nz, pbc, cx, cy, cz, asymptotic_radius, zero_self_demag, out);
}
int umag_demag_new_brute(int Nx, int Ny, int Nz, const int pbc[3], double cx, double cy, double cz, double accuracy,
                         umag_demag** out) {
    return demag_new_brute(Nx, Ny, Nz, pbc, cx, cy, cz, accuracy, out);
}
int umag_demag_new_from_kernel(int Nx, int Ny, int Nz, const double* const kern[6], umag_demag** out) {
    return demag_new_from_kernel(Nx, Ny, Nz, kern, out);
}
int umag_demag_exec(umag_demag* d, float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
                    const float* vol, const float* Ms, float Ms_mul) {
    UMAG_TRY(ensure_init());
    return demag_exec(d, Bx, By, Bz, mx, my, mz, vol, Ms, Ms_mul);
}
int umag_demag_exec_pass(umag_demag* d, int pass, float* Bx, float* By, float* Bz, const float* mx, const float* my,
                         const float* mz, const float* vol, const float* Ms, float Ms_mul) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(pass >= 0 && pass <= 2, "pass must be 0, 1 or 2");
    return demag_exec(d, Bx, By, Bz, mx, my, mz, vol, Ms, Ms_mul, pass);
}
int umag_demag_get_spectrum(umag_demag* d, float* const host[6]) { return demag_get_spectrum(d, host); }
int umag_demag_get_kernel(umag_demag* d, double* const host[6]) { return demag_get_kernel(d, host); }
int umag_demag_padded_size(umag_demag* d, int P[3]) {
    UMAG_REQUIRE(d && P, "NULL argument");
    for (int i = 0; i < 3; i++) P[i] = d->P[i];
    return UMAG_OK;
}
int umag_demag_free(umag_demag* d) {
    if (d) {
        cudaStreamSynchronize(ctx().stream);
        demag_free(d);
    }
    return UMAG_OK;
}

// engine/run.go:14-43 defaults, engine/torque.go:27 GammaLL
void umag_solver_defaults(umag_solver_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->solver = 5;
    p->dt = 1e-15;
    p->max_err = 1e-5;
    p->rel_err = 1e-4;
    p->min_slope = 1e8;
    p->headroom = 0.8;
    p->gamma_ll = 1.7595e11;
}
int umag_sim_new(const umag_sim_params* p, const umag_solver_params* s, umag_sim** out) { return sim_new(p, s, out); }
int umag_sim_free(umag_sim* s) { return sim_free(s); }
int umag_sim_set_m(umag_sim* s, const float* mx, const float* my, const float* mz) {
    return sim_set_m(s, mx, my, mz, 1);
}
int umag_sim_restore_m(umag_sim* s, const float* mx, const float* my, const float* mz) {
    return sim_set_m(s, mx, my, mz, 0);
}
int umag_sim_get_m(umag_sim* s, float* mx, float* my, float* mz) { return sim_get_m(s, mx, my, mz); }
int umag_sim_m_ptrs(umag_sim* s, float** m3) { return sim_m_ptrs(s, m3); }
int umag_sim_torque(umag_sim* s, float* tx, float* ty, float* tz, float* bx, float* by, float* bz) {
    return sim_torque(s, tx, ty, tz, bx, by, bz);
}
int umag_sim_steps(umag_sim* s, int n) { return sim_steps(s, n); }
int umag_sim_run(umag_sim* s, double seconds, int chunk, long long max_steps) {
    return sim_run(s, seconds, chunk, max_steps);
}
int umag_sim_get_state(umag_sim* s, umag_solver_state* st) { return sim_get_state(s, st); }
int umag_sim_set_time(umag_sim* s, double t, double dt) { return sim_set_time(s, t, dt); }
int umag_sim_average_m(umag_sim* s, double avg[3]) { return sim_average_m(s, avg); }
int umag_sim_use_graph(umag_sim* s, int enable, int steps) { return sim_use_graph(s, enable, steps); }
int umag_sim_launches_per_step(umag_sim* s, int* n) { return sim_launches_per_step(s, n); }
int umag_sim_torque_evals(umag_sim* s, int n) { return sim_torque_evals(s, n); }
int umag_sim_energies(umag_sim* s, double E[5]) { return sim_energies(s, E); }
int umag_sim_energy_density(umag_sim* s, float* dst) { return sim_energy_density(s, dst); }
int umag_sim_relax(umag_sim* s, double torque_threshold) { return sim_relax(s, torque_threshold); }
int umag_sim_set_solver(umag_sim* s, const umag_solver_params* sp) { return sim_set_solver(s, sp); }
int umag_sim_set_param(umag_sim* s, int which, const float* values, float mul) {
    return sim_set_param(s, which, values, mul);
}
int umag_sim_get_tuning(umag_sim* s, umag_tuning* t) { return sim_get_tuning(s, t); }
int umag_sim_set_tuning(umag_sim* s, const umag_tuning* t) { return sim_set_tuning(s, t); }
int umag_ens_new(int n, const umag_ens_instance* in, const umag_solver_params* sp, int enable_demag, umag_ens** out) {
    return ens_new(n, in, sp, enable_demag, out);
}
int umag_ens_new_general(int n, const umag_ens_instance* in, const umag_sim_params* const* general,
                         const umag_solver_params* sp, int enable_demag, umag_ens** out) {
    return ens_new_general(n, in, general, sp, enable_demag, out);
}
int umag_ens_free(umag_ens* e) { return ens_free(e); }
int umag_ens_set_m(umag_ens* e, int i, const float* host_m) { return ens_set_m(e, i, host_m); }
int umag_ens_get_m(umag_ens* e, int i, float* host_m) { return ens_get_m(e, i, host_m); }
int umag_ens_get_state(umag_ens* e, int i, umag_solver_state* st) { return ens_get_state(e, i, st); }
int umag_ens_run(umag_ens* e, double seconds, int chunk, long long max_replays) {
    return ens_run(e, seconds, chunk, max_replays);
}
int umag_ens_count(umag_ens* e, int* n_instances, int* n_classes) { return ens_count(e, n_instances, n_classes); }
int umag_ens_class_info(umag_ens* e, int cls, int N[3], int* n_instances) {
    return ens_class_info(e, cls, N, n_instances);
}
int umag_ens_class_general(umag_ens* e, int cls, int* general) { return ens_class_general(e, cls, general); }
int umag_ens_get_tuning(umag_ens* e, int cls, umag_tuning* t) { return ens_get_tuning(e, cls, t); }
int umag_ens_set_tuning(umag_ens* e, int cls, const umag_tuning* t) { return ens_set_tuning(e, cls, t); }
int umag_adj_new(const umag_adj_params* p, umag_adj** out) { return adj_new(p, out); }
int umag_adj_free(umag_adj* a) { return adj_free(a); }
int umag_adj_forward(umag_adj* a, const float* m0, const float* Ms, float Aex, float Ku1, const float B_ext[3],
                     double* loss) {
    return adj_forward(a, m0, Ms, Aex, Ku1, B_ext, loss);
}
int umag_adj_final_m(umag_adj* a, float* m) { return adj_final_m(a, m); }
int umag_adj_backward(umag_adj* a, float* gMs, float* gm0, double* gAex, double* gKu1, double gB_ext[3]) {
    return adj_backward(a, gMs, gm0, gAex, gKu1, gB_ext);
}
int umag_adj_forward_regions(umag_adj* a, const float* m0, const float* Ms, const float* Aex, const float* Ku1,
                             const float* B_ext, double* loss) {
    return adj_forward_regions(a, m0, Ms, Aex, Ku1, B_ext, loss);
}
int umag_adj_backward_regions(umag_adj* a, float* gMs, float* gm0, double* gAex, double* gKu1, double* gB_ext) {
    return adj_backward_regions(a, gMs, gm0, gAex, gKu1, gB_ext);
}

}  // extern "C"
