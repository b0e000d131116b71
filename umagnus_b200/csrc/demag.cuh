// demag.cuh -- demag plan shared by the device-op API and the engine.
#pragma once
#include <vector>

#include <cuda.h>

#include "common.cuh"
#include "fft.cuh"

constexpr int kPassThreads = 256;   // passes A and C
constexpr int kPassBThreads = 512;  // pass B
constexpr int kChunkW = 32;         // kx columns per z-transform block in passes A/C

namespace umag {
struct PassArgs;
// compile-time-planned pass kernels for one mesh size (demag_fast.cu)
struct FastPasses {
    void (*a)(PassArgs) = nullptr;
    void (*b)(PassArgs) = nullptr;
    void (*c)(PassArgs) = nullptr;
    // batched variants (grid.y extended by the instance count; demag_batch_fix)
    void (*ab)(PassArgs) = nullptr;
    void (*bb)(PassArgs) = nullptr;
    void (*cb)(PassArgs) = nullptr;
    size_t smem_ac = 0, smem_b = 0;
    int wb = 0;
    int nt_b = 512;   // threads per pass-B CTA
    int nt_ac = 256;  // threads per pass-A/C CTA
    bool ac_reg = false, b_reg = false;  // register-FFT kernels (k_reg_a/c, k_reg_b)
    // spectrum stored in blocks of 4 columns, [c][kz][kx/4][y][kx%4], so that
    // pass B's column reads and writes are contiguous (set when ac_reg && b_reg)
    bool blocked = false;
    unsigned gbx = 0, gby = 0;  // pass-B grid (demag_fast_grid)
    // narrower pass-B CTAs (fewer columns each) for single meshes whose
    // default pass-B grid has fewer CTAs than the GPU has SMs
    void (*b_n)(PassArgs) = nullptr;
    size_t smem_b_n = 0;
    int wb_n = 0, nt_b_n = 0;
    unsigned gbx_n = 0;
    bool use_narrow = false;
    // bytes of pass C's x/z scratch (Xs and the exchange lines), which its
    // z phase can borrow for a TMA-loaded spectrum slab (register passes)
    size_t ac_scratch = 0;
    bool slab_ok = false;  // pass C can take its z input as one slab
};
}  // namespace umag

struct umag_demag {
    umag::FastPasses fast;
    bool use_fast = false;
    int N[3], P[3];
    int pbc[3] = {0, 0, 0};  // PBC repetitions per axis (mag/demagkernel.go:339-355); padded size = N there
    double cell[3];
    int arad, zero_self;
    int kind = 0;           // real-space kernel: 0 Newell, 1 brute force, 2 caller-supplied
    double accuracy = 6.0;  // brute force: DemagAccuracy (engine/demag.go:25)
    int M, Hx, HxP, Lx, WB;
    bool is2d;
    umag::FftLine<float> fx, fy, fz;  // x: length Px/2 (packed real), y: Py, z: Pz
    std::vector<float2*> tw_dev;
    float2* twr = nullptr;            // exp(-2 pi i k / Px), k in [0, Px/2)
    float2* spec = nullptr;           // 3 * Pz * Ny * Lx
    float* K[6] = {};                 // xx yy zz yz xz xy (yz, xz NULL in 2D)
    size_t Kn = 0;  // floats per kernel array (Kp * (Py/2+1) * (Pz/2+1))
    int Kp = 0;     // row pitch: Px/2+1 rounded up to 4 floats (16-byte rows)
    CUtensorMap* slab_map = nullptr;  // device copy: pass C's (y, component) slabs of spec
};

namespace umag {

struct PassArgs {
    int Nx, Ny, Nz, Px, Py, Pz, M, Hx, HxP, Lx, WB;
    FftLine<float> fx, fy, fz;
    const float2* twr;
    float2* spec;
    const float* K[6];
    int Kp;  // row pitch (floats) of the kernel arrays: Hx padded to 4 in plans, Hx for caller-owned spectra
    // layouts: blocked = spectrum in 4-column blocks [c][kz][kx/4][y][kx%4]
    // (else rows [c][kz][y][kx]); Kblocked = kernel arrays in 4-column blocks
    // [kz][kx/4][ky][kx%4] (else rows [kz][ky][kx] of pitch Kp)
    int blocked, Kblocked;
    // batched launches: per-instance strides of the spectrum scratch (float2),
    // of the field output (floats) and of the controller structs holding
    // m_ind / m_ind_w / active (bytes); per-instance Ms (NULL: Ms_mul for all)
    long spec_stride, b_stride, ctl_stride;
    const float* ms_mul_b;
    const float* m[3];
    // engine use: magnetisation read through a device-side slot
    // (m_sel ? *m_ind_w : *m_ind) + c*ncell, and a device flag that turns a
    // skipped step into no-ops.  NULL for the plain device-op API.
    float* const* m_ind;
    float* const* m_ind_w;
    int m_sel;
    int ncell;
    const int* active;
    const float* vol;
    const float* Ms;
    float Ms_mul;
    float* B[3];
    // tensor map (device memory) of the blocked spectrum viewed as
    // (8 floats, y, kx/4, kz, component): pass C loads the slab of one
    // (y, component) with one bulk tensor copy; NULL: plain loads
    const CUtensorMap* slab_map;
    // engine use: the controller's status word (instance ib at fault +
    // ib * ctl_stride bytes), set to 7 when a pass gives up waiting for a
    // bulk copy; NULL for the plain device-op API, which counts such
    // timeouts in g_slab_timeouts instead
    int* fault;
};

int demag_new_newell(int Nx, int Ny, int Nz, const int pbc[3], double cx, double cy, double cz, int arad,
                     int zero_self, umag_demag** out);
int demag_new_from_kernel(int Nx, int Ny, int Nz, const double* const kern[6], umag_demag** out);
int demag_new_brute(int Nx, int Ny, int Nz, const int pbc[3], double cx, double cy, double cz, double accuracy,
                    umag_demag** out);
// brute-force real-space kernel (brute.cu) into six device arrays of the padded grid
int build_brute(const umag_demag* d, double accuracy, double* Kr[6], cudaStream_t st);
int demag_exec(umag_demag* d, float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
               const float* vol, const float* Ms, float Ms_mul, int pass = -1);
int demag_get_kernel(umag_demag* d, double* const host[6]);
int demag_get_spectrum(umag_demag* d, float* const host[6]);
void demag_free(umag_demag* d);
void fill_pass_args(const umag_demag* d, PassArgs& a);
int demag_launch(const umag_demag* d, const PassArgs& a, cudaStream_t st);
int demag_launch_batch(const umag_demag* d, const PassArgs& a, int nb, cudaStream_t st);
bool demag_fast_select(int M, int Py, int Pz, FastPasses& f);
// pass-B launch grid for a selected plan (after demag_fast_setup; current
// device); sm_count <= 0: the library context's SM count
int demag_fast_grid(FastPasses& f, int M, int Pz, int sm_count = 0);
// opt-in shared memory of the compile-time-planned passes, once per device
// (the attributes are per device context); thread-safe
int demag_fast_setup();
// no-alloc entry point: load its module on the current device (umag_init)
int noalloc_preload();
// bulk-copy waits that gave up in pass C since the counter was last cleared
// (demag_fast.cu); demag_exec reports them as an error
int demag_slab_timeouts(unsigned* out, cudaStream_t st);
int demag_set_slab_timeouts(unsigned v);

}  // namespace umag
