// ops.cu -- library context and the device-op layer (opencl package subset).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "cellmath.cuh"
#include <cstdlib>

#include "common.cuh"
#include "demag.cuh"
#include "ops.cuh"

namespace umag {

static Context g_ctx;
static thread_local char g_err[1024] = "";

Context& ctx() { return g_ctx; }

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int ensure_init() {
    if (!g_ctx.initialised) return set_error(UMAG_E_NOT_INIT, "umag_init has not been called");
    return UMAG_OK;
}

static constexpr int kRedBlocks = 1024;

int init_device(int device) {
    if (g_ctx.initialised) {
        if (device == g_ctx.device) return UMAG_OK;
        return set_error(UMAG_E_ARG, "already initialised on device %d", g_ctx.device);
    }
    int n = 0;
    UMAG_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return set_error(UMAG_E_ARG, "device %d out of range (%d devices)", device, n);
    UMAG_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    UMAG_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return set_error(UMAG_E_UNSUPPORTED, "device %d (%s, sm_%d%d) is not sm_100", device, prop.name, prop.major,
                         prop.minor);
    g_ctx.sm_count = prop.multiProcessorCount;
    UMAG_CUDA(cudaStreamCreateWithFlags(&g_ctx.own_stream, cudaStreamNonBlocking));
    g_ctx.stream = g_ctx.own_stream;
    g_ctx.red_bytes = sizeof(double) * 4 * kRedBlocks + 64;
    UMAG_CUDA(cudaMalloc(&g_ctx.red_dev, g_ctx.red_bytes));
    UMAG_CUDA(cudaMallocHost(&g_ctx.red_host, sizeof(double) * 8));
    // load the no-alloc entry point's module now, so that its fixed scratch
    // array is reserved before a caller's pool claims the device
    UMAG_TRY(noalloc_preload());
    g_ctx.device = device;
    g_ctx.initialised = true;
    return UMAG_OK;
}

int release_device() {
    if (!g_ctx.initialised) return UMAG_OK;
    cudaStreamSynchronize(g_ctx.stream);
    cudaFree(g_ctx.red_dev);
    cudaFreeHost(g_ctx.red_host);
    cudaStreamDestroy(g_ctx.own_stream);
    g_ctx = Context();
    return UMAG_OK;
}

const char* last_error() { return g_err; }

// =================================================================== kernels
__global__ void k_memset_f32(float* p, float v, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_add_exchange(float* __restrict__ Bx, float* __restrict__ By, float* __restrict__ Bz,
                               const float* __restrict__ mx, const float* __restrict__ my,
                               const float* __restrict__ mz, const float* __restrict__ Ms, float Ms_mul,
                               const float* __restrict__ aLUT, const uint8_t* __restrict__ regions, float wx,
                               float wy, float wz, Mesh3 g) {
    int ix = blockIdx.x * blockDim.x + threadIdx.x;
    int iy = blockIdx.y * blockDim.y + threadIdx.y;
    int iz = blockIdx.z;
    if (ix >= g.Nx || iy >= g.Ny) return;
    int I = (iz * g.Ny + iy) * g.Nx + ix;
    f3 m0 = ld3(mx, my, mz, I);
    if (is0(m0)) return;
    f3 b = exchange_sum(mx, my, mz, aLUT, regions, wx, wy, wz, g, ix, iy, iz, m0, __ldg(regions + I));
    float inv = inv_msat(Ms, Ms_mul, I);
    Bx[I] = fa(Bx[I], fm(b.x, inv));
    By[I] = fa(By[I], fm(b.y, inv));
    Bz[I] = fa(Bz[I], fm(b.z, inv));
}

__global__ void k_add_dmi(float* __restrict__ Hx, float* __restrict__ Hy, float* __restrict__ Hz,
                          const float* __restrict__ mx, const float* __restrict__ my, const float* __restrict__ mz,
                          const float* __restrict__ Ms, float Ms_mul, const float* __restrict__ aLUT,
                          const float* __restrict__ dLUT, const uint8_t* __restrict__ regions, float cx, float cy,
                          float cz, Mesh3 g, int openbc) {
    int ix = blockIdx.x * blockDim.x + threadIdx.x;
    int iy = blockIdx.y * blockDim.y + threadIdx.y;
    int iz = blockIdx.z;
    if (ix >= g.Nx || iy >= g.Ny) return;
    int I = (iz * g.Ny + iy) * g.Nx + ix;
    f3 m0 = ld3(mx, my, mz, I);
    if (is0(m0)) return;
    f3 h = dmi_sum(mx, my, mz, aLUT, dLUT, regions, cx, cy, cz, g, openbc != 0, ix, iy, iz, m0, __ldg(regions + I));
    float inv = inv_msat(Ms, Ms_mul, I);
    Hx[I] = fa(Hx[I], fm(h.x, inv));
    Hy[I] = fa(Hy[I], fm(h.y, inv));
    Hz[I] = fa(Hz[I], fm(h.z, inv));
}

__global__ void k_add_dmibulk(float* __restrict__ Hx, float* __restrict__ Hy, float* __restrict__ Hz,
                              const float* __restrict__ mx, const float* __restrict__ my,
                              const float* __restrict__ mz, const float* __restrict__ Ms, float Ms_mul,
                              const float* __restrict__ aLUT, const float* __restrict__ dLUT,
                              const uint8_t* __restrict__ regions, float cx, float cy, float cz, Mesh3 g,
                              int openbc) {
    int ix = blockIdx.x * blockDim.x + threadIdx.x;
    int iy = blockIdx.y * blockDim.y + threadIdx.y;
    int iz = blockIdx.z;
    if (ix >= g.Nx || iy >= g.Ny) return;
    int I = (iz * g.Ny + iy) * g.Nx + ix;
    f3 m0 = ld3(mx, my, mz, I);
    if (is0(m0)) return;
    f3 h = dmibulk_sum(mx, my, mz, aLUT, dLUT, regions, cx, cy, cz, g, openbc != 0, ix, iy, iz, m0,
                       __ldg(regions + I));
    float inv = inv_msat(Ms, Ms_mul, I);
    Hx[I] = fa(Hx[I], fm(h.x, inv));
    Hy[I] = fa(Hy[I], fm(h.y, inv));
    Hz[I] = fa(Hz[I], fm(h.z, inv));
}

__global__ void k_add_cubic(float* __restrict__ Bx, float* __restrict__ By, float* __restrict__ Bz,
                            const float* __restrict__ mx, const float* __restrict__ my,
                            const float* __restrict__ mz, CubicParams p, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        f3 B{Bx[i], By[i], Bz[i]};
        add_cubic(B, p, ld3(mx, my, mz, i), i);
        Bx[i] = B.x; By[i] = B.y; Bz[i] = B.z;
    }
}

__global__ void k_add_uniaxial(float* __restrict__ Bx, float* __restrict__ By, float* __restrict__ Bz,
                               const float* __restrict__ mx, const float* __restrict__ my,
                               const float* __restrict__ mz, UniaxParams p, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        f3 B{Bx[i], By[i], Bz[i]};
        add_uniaxial(B, p, ld3(mx, my, mz, i), i);
        Bx[i] = B.x; By[i] = B.y; Bz[i] = B.z;
    }
}

__global__ void k_region_addv(float* __restrict__ dx, float* __restrict__ dy, float* __restrict__ dz,
                              const float* __restrict__ lx, const float* __restrict__ ly,
                              const float* __restrict__ lz, const uint8_t* __restrict__ regions, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        int r = __ldg(regions + i);
        dx[i] = fa(dx[i], __ldg(lx + r));
        dy[i] = fa(dy[i], __ldg(ly + r));
        dz[i] = fa(dz[i], __ldg(lz + r));
    }
}

__global__ void k_region_decode(float* __restrict__ dst, const float* __restrict__ lut,
                                const uint8_t* __restrict__ regions, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        dst[i] = __ldg(lut + __ldg(regions + i));
}

// t may alias h: each element is read before it is written by the same thread
__global__ void k_lltorque(float* tx, float* ty, float* tz, const float* __restrict__ mx,
                           const float* __restrict__ my, const float* __restrict__ mz, const float* hx,
                           const float* hy, const float* hz, const float* __restrict__ alpha, float alpha_mul,
                           int N, int precess) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        f3 m = ld3(mx, my, mz, i);
        f3 H{hx[i], hy[i], hz[i]};
        f3 t = precess ? lltorque(m, H, amul(alpha, alpha_mul, i)) : llnoprecess(m, H);
        tx[i] = t.x; ty[i] = t.y; tz[i] = t.z;
    }
}

struct MaddArgs {
    float* dst[3];
    const float* src[7][3];
    float fac[7];
};
template <int NS>
__global__ void k_madd(MaddArgs a, int ncomp, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        for (int c = 0; c < ncomp; c++) {
            float acc;
            if (NS == 3) {
                acc = fa(fm(a.fac[0], a.src[0][c][i]), fa(fm(a.fac[1], a.src[1][c][i]), fm(a.fac[2], a.src[2][c][i])));
            } else {
                acc = fm(a.fac[0], a.src[0][c][i]);
#pragma unroll
                for (int j = 1; j < NS; j++) acc = fa(acc, fm(a.fac[j], a.src[j][c][i]));
            }
            a.dst[c][i] = acc;
        }
    }
}

__global__ void k_normalize(float* vx, float* vy, float* vz, const float* __restrict__ vol, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float w = vol == nullptr ? 1.0f : vol[i];
        f3 r = normalize_vol(f3{vx[i], vy[i], vz[i]}, w);
        vx[i] = r.x; vy[i] = r.y; vz[i] = r.z;
    }
}

__global__ void k_vecnorm(float* dst, const float* __restrict__ ax, const float* __restrict__ ay,
                          const float* __restrict__ az, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        f3 a = ld3(ax, ay, az, i);
        dst[i] = __fsqrt_rn(dot3(a, a));
    }
}

__global__ void k_div(float* dst, const float* a, const float* b, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float bb = b[i];
        dst[i] = bb == 0.0f ? 0.0f : fd(a[i], bb);
    }
}

__global__ void k_add_dot(float* dst, float pre, const float* __restrict__ ax, const float* __restrict__ ay,
                          const float* __restrict__ az, const float* __restrict__ bx, const float* __restrict__ by,
                          const float* __restrict__ bz, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        dst[i] = fa(dst[i], fm(pre, dot3(ld3(ax, ay, az, i), ld3(bx, by, bz, i))));
}

// thermal noise of (seed, step) for N cells, three components
__global__ void k_thermal_noise(float* nx, float* ny, float* nz, int N, uint64_t seed, long long step) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const f3 n = therm_normals(seed, step, i);
        nx[i] = n.x;
        ny[i] = n.y;
        nz[i] = n.z;
    }
}

// temperature2.cl:3-19 settemperature2
__global__ void k_set_temperature(float* B, const float* __restrict__ noise, float k2, const float* __restrict__ Ms,
                                  float Ms_mul, const float* __restrict__ temp, float temp_mul,
                                  const float* __restrict__ alpha, float alpha_mul, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float invMs = inv_msat(Ms, Ms_mul, i);
        B[i] = fm(noise[i], therm_scale(k2, amul(alpha, alpha_mul, i), amul(temp, temp_mul, i), invMs));
    }
}

int thermal_noise(float* nx, float* ny, float* nz, int N, uint64_t seed, long long step) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(nx && ny && nz, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_thermal_noise<<<grid_for(N, 256), 256, 0, ctx().stream>>>(nx, ny, nz, N, seed, step);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int set_temperature(float* B, const float* noise, float k2, const float* Ms, float Ms_mul, const float* temp,
                    float temp_mul, const float* alpha, float alpha_mul, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(B && noise, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_set_temperature<<<grid_for(N, 256), 256, 0, ctx().stream>>>(B, noise, k2, Ms, Ms_mul, temp, temp_mul, alpha,
                                                                   alpha_mul, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

// zeromask.cl
__global__ void k_zero_mask(float* dx, float* dy, float* dz, const float* __restrict__ lut,
                            const uint8_t* __restrict__ regions, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        if (lut[regions[i]] != 0.0f) {
            dx[i] = 0.0f;
            dy[i] = 0.0f;
            dz[i] = 0.0f;
        }
}

int zero_mask(float* dx, float* dy, float* dz, const float* lut, const uint8_t* regions, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(dx && dy && dz && lut && regions, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_zero_mask<<<grid_for(N, 256), 256, 0, ctx().stream>>>(dx, dy, dz, lut, regions, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

// ---- reductions ------------------------------------------------------------
// kind 0: max |v|^2 of a vector field; 1: max |a-b|^2; 2: max |v| of a scalar
template <int KIND>
__global__ void k_reduce_max(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                             const float* __restrict__ x2, const float* __restrict__ y2,
                             const float* __restrict__ z2, int N, unsigned int* out) {
    __shared__ float sh[32];
    float mx = 0.0f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float v;
        if (KIND == 0) {
            f3 a = ld3(x, y, z, i);
            v = dot3(a, a);
        } else if (KIND == 1) {
            f3 d{fs(__ldg(x + i), __ldg(x2 + i)), fs(__ldg(y + i), __ldg(y2 + i)), fs(__ldg(z + i), __ldg(z2 + i))};
            v = dot3(d, d);
        } else {
            v = fabsf(__ldg(x + i));
        }
        mx = fmaxf(mx, v);
    }
    mx = block_max<256>(mx, sh);
    if (threadIdx.x == 0) atomic_max_nonneg(out, mx);
}

// Compensated sum: Neumaier per thread in float32, two-sum tree per block,
// block partials (hi, lo) combined in FP64 by a single block.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = fa(a, b);
    float bb = fs(s, a);
    e = fa(fs(a, fs(s, bb)), fs(b, bb));
}
template <bool DOT>
__global__ void k_sum_partials(const float* __restrict__ a, const float* __restrict__ b, int N, double* part) {
    __shared__ float sh_s[256], sh_c[256];
    float s = 0.0f, c = 0.0f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float v, pe = 0.0f;
        if (DOT) {
            float x = __ldg(a + i), y = __ldg(b + i);
            v = __fmul_rn(x, y);
            pe = __fmaf_rn(x, y, -v);  // exact rounding error of the product
        } else {
            v = __ldg(a + i);
        }
        float t, e;
        two_sum(s, v, t, e);
        s = t;
        c = fa(c, fa(e, pe));
    }
    sh_s[threadIdx.x] = s;
    sh_c[threadIdx.x] = c;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            float t, e;
            two_sum(sh_s[threadIdx.x], sh_s[threadIdx.x + o], t, e);
            sh_s[threadIdx.x] = t;
            sh_c[threadIdx.x] = fa(fa(sh_c[threadIdx.x], sh_c[threadIdx.x + o]), e);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = (double)sh_s[0] + (double)sh_c[0];
}
__global__ void k_sum_final(const double* part, int n, double* out) {
    __shared__ double sh[256];
    double s = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {  // fixed order per thread (deterministic)
        double y = part[i] - c;
        double t = s + y;
        c = (t - s) - y;
        s = t;
    }
    sh[threadIdx.x] = s - c;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0, cc = 0.0;
        for (int i = 0; i < blockDim.x; i++) {
            double y = sh[i] - cc;
            double t = tot + y;
            cc = (t - tot) - y;
            tot = t;
        }
        *out = tot;
    }
}

// =================================================================== host API
static dim3 block3d() { return dim3(32, 8, 1); }
static dim3 grid3d(int Nx, int Ny, int Nz) { return dim3((Nx + 31) / 32, (Ny + 7) / 8, Nz); }

int add_exchange(float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
                 const float* Ms, float Ms_mul, const float* aLUT, const uint8_t* regions, int Nx, int Ny, int Nz,
                 double cx, double cy, double cz, int pbc) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(Bx && By && Bz && mx && my && mz && aLUT && regions, "NULL argument");
    UMAG_REQUIRE(Nx > 0 && Ny > 0 && Nz > 0, "bad mesh size");
    // opencl/exchange.go:17-20: FP64 weights rounded to float32
    float wx = (float)(2 / (cx * cx)), wy = (float)(2 / (cy * cy)), wz = (float)(2 / (cz * cz));
    k_add_exchange<<<grid3d(Nx, Ny, Nz), block3d(), 0, ctx().stream>>>(Bx, By, Bz, mx, my, mz, Ms, Ms_mul, aLUT,
                                                                       regions, wx, wy, wz, Mesh3{Nx, Ny, Nz, pbc});
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int add_dmi(float* Hx, float* Hy, float* Hz, const float* mx, const float* my, const float* mz, const float* Ms,
            float Ms_mul, const float* aLUT, const float* dLUT, const uint8_t* regions, int Nx, int Ny, int Nz,
            double cx, double cy, double cz, int pbc, int openbc) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(Hx && Hy && Hz && mx && my && mz && aLUT && dLUT && regions, "NULL argument");
    UMAG_REQUIRE(Nx > 0 && Ny > 0 && Nz > 0, "bad mesh size");
    // opencl/dmi.go:61: cell sizes passed as float32
    k_add_dmi<<<grid3d(Nx, Ny, Nz), block3d(), 0, ctx().stream>>>(Hx, Hy, Hz, mx, my, mz, Ms, Ms_mul, aLUT, dLUT,
                                                                  regions, (float)cx, (float)cy, (float)cz,
                                                                  Mesh3{Nx, Ny, Nz, pbc}, openbc);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int add_dmibulk(float* Hx, float* Hy, float* Hz, const float* mx, const float* my, const float* mz,
                const float* Ms, float Ms_mul, const float* aLUT, const float* dLUT, const uint8_t* regions, int Nx,
                int Ny, int Nz, double cx, double cy, double cz, int pbc, int openbc) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(Hx && Hy && Hz && mx && my && mz && aLUT && dLUT && regions, "NULL argument");
    UMAG_REQUIRE(Nx > 0 && Ny > 0 && Nz > 0, "bad mesh size");
    // opencl/dmibulk.go: cell sizes passed as float32
    k_add_dmibulk<<<grid3d(Nx, Ny, Nz), block3d(), 0, ctx().stream>>>(Hx, Hy, Hz, mx, my, mz, Ms, Ms_mul, aLUT,
                                                                      dLUT, regions, (float)cx, (float)cy,
                                                                      (float)cz, Mesh3{Nx, Ny, Nz, pbc}, openbc);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int add_cubic(float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
              const CubicParams& p, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(Bx && By && Bz && mx && my && mz, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_add_cubic<<<grid_for(N, 256), 256, 0, ctx().stream>>>(Bx, By, Bz, mx, my, mz, p, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int add_uniaxial(float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
                 const UniaxParams& p, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(Bx && By && Bz && mx && my && mz, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_add_uniaxial<<<grid_for(N, 256), 256, 0, ctx().stream>>>(Bx, By, Bz, mx, my, mz, p, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int region_addv(float* dx, float* dy, float* dz, const float* lx, const float* ly, const float* lz,
                const uint8_t* regions, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(dx && dy && dz && lx && ly && lz && regions, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_region_addv<<<grid_for(N, 256), 256, 0, ctx().stream>>>(dx, dy, dz, lx, ly, lz, regions, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int region_decode(float* dst, const float* lut, const uint8_t* regions, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(dst && lut && regions, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_region_decode<<<grid_for(N, 256), 256, 0, ctx().stream>>>(dst, lut, regions, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int torque(float* tx, float* ty, float* tz, const float* mx, const float* my, const float* mz, const float* hx,
           const float* hy, const float* hz, const float* alpha, float alpha_mul, int N, int precess) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(tx && ty && tz && mx && my && mz && hx && hy && hz, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_lltorque<<<grid_for(N, 256), 256, 0, ctx().stream>>>(tx, ty, tz, mx, my, mz, hx, hy, hz, alpha, alpha_mul, N,
                                                            precess);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int madd(int ncomp, float* const* dst, int nsrc, const float* const* src, const float* fac, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(ncomp >= 1 && ncomp <= 3, "ncomp must be 1..3");
    UMAG_REQUIRE(nsrc >= 2 && nsrc <= 7, "nsrc must be 2..7 (Madd2..Madd7)");
    UMAG_REQUIRE(dst && src && fac, "NULL argument");
    if (N <= 0) return UMAG_OK;
    MaddArgs a{};
    for (int c = 0; c < ncomp; c++) {
        UMAG_REQUIRE(dst[c] != nullptr, "NULL destination");
        a.dst[c] = dst[c];
    }
    for (int j = 0; j < nsrc; j++) {
        a.fac[j] = fac[j];
        for (int c = 0; c < ncomp; c++) {
            UMAG_REQUIRE(src[j * ncomp + c] != nullptr, "NULL source");
            a.src[j][c] = src[j * ncomp + c];
        }
    }
    int g = grid_for(N, 256);
    cudaStream_t s = ctx().stream;
    switch (nsrc) {
    case 2: k_madd<2><<<g, 256, 0, s>>>(a, ncomp, N); break;
    case 3: k_madd<3><<<g, 256, 0, s>>>(a, ncomp, N); break;
    case 4: k_madd<4><<<g, 256, 0, s>>>(a, ncomp, N); break;
    case 5: k_madd<5><<<g, 256, 0, s>>>(a, ncomp, N); break;
    case 6: k_madd<6><<<g, 256, 0, s>>>(a, ncomp, N); break;
    default: k_madd<7><<<g, 256, 0, s>>>(a, ncomp, N); break;
    }
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int normalize(float* vx, float* vy, float* vz, const float* vol, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(vx && vy && vz, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_normalize<<<grid_for(N, 256), 256, 0, ctx().stream>>>(vx, vy, vz, vol, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int vecnorm(float* dst, const float* ax, const float* ay, const float* az, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(dst && ax && ay && az, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_vecnorm<<<grid_for(N, 256), 256, 0, ctx().stream>>>(dst, ax, ay, az, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int div(float* dst, const float* a, const float* b, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(dst && a && b, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_div<<<grid_for(N, 256), 256, 0, ctx().stream>>>(dst, a, b, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int add_dot(float* dst, float pre, const float* ax, const float* ay, const float* az, const float* bx,
            const float* by, const float* bz, int N) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(dst && ax && ay && az && bx && by && bz, "NULL argument");
    if (N <= 0) return UMAG_OK;
    k_add_dot<<<grid_for(N, 256), 256, 0, ctx().stream>>>(dst, pre, ax, ay, az, bx, by, bz, N);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int memset_f32(float* p, float v, size_t n) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(p != nullptr || n == 0, "NULL pointer");
    if (n == 0) return UMAG_OK;
    k_memset_f32<<<grid_for((long long)n, 256), 256, 0, ctx().stream>>>(p, v, (long)n);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

// reductions: result to host (blocking, like the reference's copyback)
static int reduce_max(int kind, const float* x, const float* y, const float* z, const float* x2, const float* y2,
                      const float* z2, int N, double* out, bool sq) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(out != nullptr, "NULL output");
    if (N <= 0) { *out = 0.0; return UMAG_OK; }
    cudaStream_t s = ctx().stream;
    unsigned int* d = (unsigned int*)ctx().red_dev;
    UMAG_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned int), s));
    int g = grid_for(N, 256, 4);
    if (kind == 0) k_reduce_max<0><<<g, 256, 0, s>>>(x, y, z, nullptr, nullptr, nullptr, N, d);
    else if (kind == 1) k_reduce_max<1><<<g, 256, 0, s>>>(x, y, z, x2, y2, z2, N, d);
    else k_reduce_max<2><<<g, 256, 0, s>>>(x, nullptr, nullptr, nullptr, nullptr, nullptr, N, d);
    UMAG_LAUNCH_CHECK();
    unsigned int bits = 0;
    UMAG_CUDA(cudaMemcpyAsync(ctx().red_host, d, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    UMAG_CUDA(cudaStreamSynchronize(s));
    memcpy(&bits, ctx().red_host, sizeof(bits));
    float f;
    memcpy(&f, &bits, sizeof(f));
    *out = sq ? sqrt((double)f) : (double)f;
    return UMAG_OK;
}

int max_vec_norm(const float* x, const float* y, const float* z, int N, double* out) {
    UMAG_REQUIRE((x && y && z) || N <= 0, "NULL argument");
    return reduce_max(0, x, y, z, nullptr, nullptr, nullptr, N, out, true);
}
int max_vec_diff(const float* ax, const float* ay, const float* az, const float* bx, const float* by,
                 const float* bz, int N, double* out) {
    UMAG_REQUIRE((ax && ay && az && bx && by && bz) || N <= 0, "NULL argument");
    return reduce_max(1, ax, ay, az, bx, by, bz, N, out, true);
}
int max_abs(const float* v, int N, double* out) {
    UMAG_REQUIRE(v || N <= 0, "NULL argument");
    return reduce_max(2, v, nullptr, nullptr, nullptr, nullptr, nullptr, N, out, false);
}

int sum_dot(const float* a, const float* b, int N, double* out) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(out != nullptr, "NULL output");
    if (N <= 0) { *out = 0.0; return UMAG_OK; }
    UMAG_REQUIRE(a != nullptr, "NULL argument");
    cudaStream_t s = ctx().stream;
    double* part = (double*)ctx().red_dev + 8;
    int g = grid_for(N, 256, 4);
    if (g > kRedBlocks) g = kRedBlocks;
    if (b) k_sum_partials<true><<<g, 256, 0, s>>>(a, b, N, part);
    else k_sum_partials<false><<<g, 256, 0, s>>>(a, nullptr, N, part);
    k_sum_final<<<1, 256, 0, s>>>(part, g, (double*)ctx().red_dev);
    UMAG_LAUNCH_CHECK();
    UMAG_CUDA(cudaMemcpyAsync(ctx().red_host, ctx().red_dev, sizeof(double), cudaMemcpyDeviceToHost, s));
    UMAG_CUDA(cudaStreamSynchronize(s));
    *out = ctx().red_host[0];
    return UMAG_OK;
}

}  // namespace umag
