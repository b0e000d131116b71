// noalloc.cu -- a demag convolution entry point that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they need a
// field: code running under an external memory manager that owns the whole
// device pool, a host runtime that forbids allocation after start-up, or a
// caller that has reserved every byte for its own arrays.  For them
// umag_demag_exec_noalloc() computes the demag field with all of its
// working memory in one file-scope __device__ array (kNoallocScratchBytes,
// 16 MiB), which every GPU that loads this library holds until the process
// exits.  The caller passes the kernel spectrum, m, the output B and a
// stream; nothing is allocated or freed, neither by this file nor by any
// library routine it calls.
//
// With lazy module loading (the CUDA default since 12.2) the driver reserves
// the array when this file's module is first loaded on a device, i.e. on the
// first look-up of its address.  umag_init does that look-up for its device
// (noalloc_preload), so a caller that initialises the library before an
// external pool claims the device's memory never sees that reservation fail
// later; a caller that skips umag_init gets it on its first no-alloc call.
#include <atomic>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "demag.cuh"
#include "fft.cuh"

namespace umag {

constexpr size_t kNoallocScratchBytes = (size_t)16 << 20;

// Working memory of umag_demag_exec_noalloc: the 3-component half spectrum
// followed by the twiddle tables.  Shared by every call on this device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// Device address of g_noalloc_scratch, looked up once per device (the host
// symbol is only a stand-in and must never be handed to a kernel).  Atomic:
// two host threads may look it up at once (both store the same address).
static std::atomic<void*> g_noalloc_ptr[64];

static int noalloc_scratch(void** out) {
    int dev = 0;
    UMAG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(UMAG_E_ARG, "device %d out of range", dev);
    void* p = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!p) {
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return set_error(UMAG_E_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
        g_noalloc_ptr[dev].store(p, std::memory_order_release);
    }
    *out = p;
    return UMAG_OK;
}

// Loads this module on the current device (reserving the scratch array) and
// caches the array's address; called by umag_init.
int noalloc_preload() {
    void* p = nullptr;
    return noalloc_scratch(&p);
}

// twiddles exp(-2 pi i j / L) of the four tables, evaluated in FP64 on the device
__global__ void k_noalloc_twiddles(float2* tw, int M, int Py, int Pz, int Px) {
    const int n = M + Py + Pz + M;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        int j = e, L = M;
        if (j >= M) {
            j -= M; L = Py;
            if (j >= Py) {
                j -= Py; L = Pz;
                if (j >= Pz) { j -= Pz; L = Px; }
            }
        }
        double s, c;
        sincospi(-2.0 * (double)j / (double)L, &s, &c);
        tw[e] = make_float2((float)c, (float)s);
    }
}

}  // namespace umag

using namespace umag;

extern "C" __attribute__((visibility("default"))) int umag_demag_exec_noalloc(
    int Nx, int Ny, int Nz, const float* const K[6], float* Bx, float* By, float* Bz, const float* mx,
    const float* my, const float* mz, const float* vol, const float* Ms, float Ms_mul, void* stream) {
    UMAG_REQUIRE(K && K[0] && K[1] && K[2] && K[5], "NULL kernel spectrum");
    UMAG_REQUIRE(Bx && By && Bz && mx && my && mz, "NULL field or magnetisation pointer");
    UMAG_REQUIRE(Nx > 0 && Ny > 0 && Nz > 0, "bad mesh size");
    // plan description on the stack (no plan object, no device allocation)
    umag_demag d;
    d.N[0] = Nx; d.N[1] = Ny; d.N[2] = Nz;
    d.P[0] = 2 * Nx;
    d.P[1] = 2 * Ny;
    d.P[2] = Nz > 5 ? 2 * Nz : 2 * Nz - 1;  // mag/demagkernel.go:404-420
    d.M = Nx;
    d.Hx = d.M + 1;
    d.HxP = d.M + 1;
    d.Lx = (d.Hx + 3) / 4 * 4;
    d.is2d = Nz == 1;
    if (Nz > 1) UMAG_REQUIRE(K[3] && K[4], "NULL yz/xz kernel spectrum for a 3D mesh");
    UMAG_TRY(demag_fast_setup());
    if (!demag_fast_select(d.M, d.P[1], d.P[2], d.fast))
        return set_error(UMAG_E_UNSUPPORTED, "mesh %dx%dx%d has no compile-time FFT plan (no-alloc path)", Nx, Ny, Nz);
    int dev = 0, sms = 0;
    UMAG_CUDA(cudaGetDevice(&dev));
    UMAG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    UMAG_TRY(demag_fast_grid(d.fast, d.M, d.P[2], sms));
    d.use_fast = true;
    d.WB = d.fast.wb;
    // scratch layout: spectrum | tw(M) | tw(Py) | tw(Pz) | exp(-2 pi i k/Px), k < M
    const size_t spec = (size_t)3 * d.P[2] * Ny * d.Lx;
    const size_t ntw = (size_t)d.M + d.P[1] + d.P[2] + d.M;
    const size_t need = sizeof(float2) * (spec + ntw);
    if (need > kNoallocScratchBytes)
        return set_error(UMAG_E_UNSUPPORTED, "mesh %dx%dx%d needs %zu bytes of scratch, the no-alloc limit is %zu",
                         Nx, Ny, Nz, need, kNoallocScratchBytes);
    void* base = nullptr;
    UMAG_TRY(noalloc_scratch(&base));
    float2* sp = reinterpret_cast<float2*>(base);
    float2* tw = sp + spec;
    cudaStream_t st = (cudaStream_t)stream;
    k_noalloc_twiddles<<<(unsigned)((ntw + 255) / 256), 256, 0, st>>>(tw, d.M, d.P[1], d.P[2], d.P[0]);
    UMAG_LAUNCH_CHECK();
    FftLine<float> fx{}, fy{}, fz{};
    fx.L = d.M; fx.nst = fft_factor(d.M, fx.R); fx.tw = tw;
    fy.L = d.P[1]; fy.nst = fft_factor(d.P[1], fy.R); fy.tw = tw + d.M;
    fz.L = d.P[2]; fz.nst = d.P[2] > 1 ? fft_factor(d.P[2], fz.R) : 0; fz.tw = tw + d.M + d.P[1];
    PassArgs a{};
    a.Nx = Nx; a.Ny = Ny; a.Nz = Nz;
    a.Px = d.P[0]; a.Py = d.P[1]; a.Pz = d.P[2];
    a.M = d.M; a.Hx = d.Hx; a.HxP = d.HxP; a.Lx = d.Lx; a.WB = d.WB;
    a.fx = fx; a.fy = fy; a.fz = fz;
    a.twr = tw + d.M + d.P[1] + d.P[2];
    a.spec = sp;
    for (int c = 0; c < 6; c++) a.K[c] = K[c];
    a.Kp = d.Hx;  // caller's spectrum: reference layout, rows of Px/2+1 floats
    a.Kblocked = 0;
    a.blocked = d.fast.blocked ? 1 : 0;
    if (d.is2d) a.K[3] = a.K[4] = nullptr;
    a.m[0] = mx; a.m[1] = my; a.m[2] = mz;
    a.B[0] = Bx; a.B[1] = By; a.B[2] = Bz;
    a.vol = vol; a.Ms = Ms; a.Ms_mul = Ms_mul;
    return demag_launch(&d, a, st);
}
