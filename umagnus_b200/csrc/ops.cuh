// ops.cuh -- device-op layer entry points (C++ side of the C-ABI).
#pragma once
#include <cstdint>

#include "cellmath.cuh"

namespace umag {
int init_device(int device);
int release_device();
const char* last_error();
int add_exchange(float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
                 const float* Ms, float Ms_mul, const float* aLUT, const uint8_t* regions, int Nx, int Ny, int Nz,
                 double cx, double cy, double cz, int pbc);
int add_dmi(float* Hx, float* Hy, float* Hz, const float* mx, const float* my, const float* mz, const float* Ms,
            float Ms_mul, const float* aLUT, const float* dLUT, const uint8_t* regions, int Nx, int Ny, int Nz,
            double cx, double cy, double cz, int pbc, int openbc);
int add_uniaxial(float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
                 const UniaxParams& p, int N);
int add_dmibulk(float* Hx, float* Hy, float* Hz, const float* mx, const float* my, const float* mz,
                const float* Ms, float Ms_mul, const float* aLUT, const float* dLUT, const uint8_t* regions, int Nx,
                int Ny, int Nz, double cx, double cy, double cz, int pbc, int openbc);
int add_cubic(float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
              const CubicParams& p, int N);
int region_addv(float* dx, float* dy, float* dz, const float* lx, const float* ly, const float* lz,
                const uint8_t* regions, int N);
int region_decode(float* dst, const float* lut, const uint8_t* regions, int N);
int torque(float* tx, float* ty, float* tz, const float* mx, const float* my, const float* mz, const float* hx,
           const float* hy, const float* hz, const float* alpha, float alpha_mul, int N, int precess);
int zero_mask(float* dx, float* dy, float* dz, const float* lut, const uint8_t* regions, int N);
int thermal_noise(float* nx, float* ny, float* nz, int N, uint64_t seed, long long step);
int set_temperature(float* B, const float* noise, float k2, const float* Ms, float Ms_mul, const float* temp,
                    float temp_mul, const float* alpha, float alpha_mul, int N);
int madd(int ncomp, float* const* dst, int nsrc, const float* const* src, const float* fac, int N);
int normalize(float* vx, float* vy, float* vz, const float* vol, int N);
int vecnorm(float* dst, const float* ax, const float* ay, const float* az, int N);
int div(float* dst, const float* a, const float* b, int N);
int add_dot(float* dst, float pre, const float* ax, const float* ay, const float* az, const float* bx,
            const float* by, const float* bz, int N);
int memset_f32(float* p, float v, size_t n);
int max_vec_norm(const float* x, const float* y, const float* z, int N, double* out);
int max_vec_diff(const float* ax, const float* ay, const float* az, const float* bx, const float* by,
                 const float* bz, int N, double* out);
int max_abs(const float* v, int N, double* out);
int sum_dot(const float* a, const float* b, int N, double* out);
}  // namespace umag
