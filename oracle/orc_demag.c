/*
 * orc_demag.c -- FP64 FFT, demag kernel spectrum and demag convolution.
 * TEST INFRASTRUCTURE ONLY (see umag_oracle.h).
 *
 * The reference performs these FFTs with the third-party VkFFT v1.2.21
 * (cl/vkFFT.h, called from opencl/fft3dr2c.go / fft3dc2r.go).  The oracle
 * uses its own exact-math mixed-radix FFT in FP64, so the f32 demag oracle
 * rounds like the reference everywhere except inside the FFT.
 */
#include "umag_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.1415926535897932384626433
#define ORC_MU0 (4 * ORC_PI * 1e-7) /* kernels_src/clh/constants.clh:5 */

typedef struct { double re, im; } cpx;

/* ---- mixed-radix FFT ----------------------------------------------------- */
typedef struct {
    int n, nf, f[40];
    cpx* tw; /* tw[j] = exp(-2 pi i j / n) */
} fft_plan;

static fft_plan g_plans[64];
static int g_nplans = 0;

static const fft_plan* get_plan(int n) {
    const fft_plan* found = NULL;
#pragma omp critical(orc_fft_plan)
    {
        for (int i = 0; i < g_nplans; i++)
            if (g_plans[i].n == n) found = &g_plans[i];
        if (!found && g_nplans < 64) {
            fft_plan* p = &g_plans[g_nplans];
            p->n = n;
            p->nf = 0;
            int m = n;
            static const int pref[] = {4, 2, 3, 5, 7};
            for (int k = 0; k < 5 && m > 1; k++)
                while (m % pref[k] == 0) { p->f[p->nf++] = pref[k]; m /= pref[k]; }
            for (int q = 11; m > 1; q += 2)
                while (m % q == 0) { p->f[p->nf++] = q; m /= q; }
            p->tw = (cpx*)malloc(sizeof(cpx) * n);
            for (int j = 0; j < n; j++) {
                double a = -2.0 * ORC_PI * (double)j / (double)n;
                p->tw[j].re = cos(a);
                p->tw[j].im = sin(a);
            }
            g_nplans++;
            found = p;
        }
    }
    return found;
}

/* out[0..n) = DFT of in[0], in[s], in[2s], ... ; recursive decimation in time */
static void fft_rec(const cpx* in, long s, cpx* out, int n, const int* f, const fft_plan* P,
                    long step, int sign) {
    if (n == 1) { out[0] = in[0]; return; }
    int p = f[0], m = n / p;
    for (int r = 0; r < p; r++) fft_rec(in + r * s, s * p, out + (long)r * m, m, f + 1, P, step * p, sign);
    cpx t[64];
    cpx* tt = p <= 64 ? t : (cpx*)malloc(sizeof(cpx) * p);
    long N0 = P->n;
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++) {
            cpx y = out[(long)r * m + k];
            long e = ((long)r * k * step) % N0;
            cpx w = P->tw[e];
            if (sign > 0) w.im = -w.im;
            tt[r].re = y.re * w.re - y.im * w.im;
            tt[r].im = y.re * w.im + y.im * w.re;
        }
        for (int q = 0; q < p; q++) {
            double sr = 0, si = 0;
            for (int r = 0; r < p; r++) {
                long e = ((long)r * q * m * step) % N0;
                cpx w = P->tw[e];
                if (sign > 0) w.im = -w.im;
                sr += tt[r].re * w.re - tt[r].im * w.im;
                si += tt[r].re * w.im + tt[r].im * w.re;
            }
            out[k + (long)q * m].re = sr;
            out[k + (long)q * m].im = si;
        }
    }
    if (tt != t) free(tt);
}

static void fft_strided(cpx* a, int n, long stride, int sign, cpx* tmp_in, cpx* tmp_out) {
    if (n == 1) return;
    const fft_plan* P = get_plan(n);
    for (int i = 0; i < n; i++) tmp_in[i] = a[i * stride];
    fft_rec(tmp_in, 1, tmp_out, n, P->f, P, 1, sign);
    for (int i = 0; i < n; i++) a[i * stride] = tmp_out[i];
}

void orc_fft_line(double* re_im, int n, int sign) {
    cpx* ti = (cpx*)malloc(sizeof(cpx) * n);
    cpx* to = (cpx*)malloc(sizeof(cpx) * n);
    fft_strided((cpx*)re_im, n, 1, sign, ti, to);
    free(ti);
    free(to);
}

/* unnormalised 3D complex FFT, x fastest */
static void fft3d(cpx* a, const int P[3], int sign) {
    get_plan(P[0]); get_plan(P[1]); get_plan(P[2]);
    int nmax = P[0] > P[1] ? P[0] : P[1];
    if (P[2] > nmax) nmax = P[2];
    long nx = P[0], ny = P[1], nz = P[2];
#pragma omp parallel
    {
        cpx* ti = (cpx*)malloc(sizeof(cpx) * nmax);
        cpx* to = (cpx*)malloc(sizeof(cpx) * nmax);
#pragma omp for
        for (long l = 0; l < ny * nz; l++) fft_strided(a + l * nx, (int)nx, 1, sign, ti, to);
#pragma omp for
        for (long l = 0; l < nx * nz; l++) {
            long x = l % nx, z = l / nx;
            fft_strided(a + z * nx * ny + x, (int)ny, nx, sign, ti, to);
        }
#pragma omp for
        for (long l = 0; l < nx * ny; l++) fft_strided(a + l, (int)nz, nx * ny, sign, ti, to);
        free(ti);
        free(to);
    }
}

/* ---- kernel spectrum (opencl/conv_demag.go:155-201, conv_common.go:27-53) */
double orc_kernel_spectrum(const int P[3], double* const K[6], int round_f32, double* Kf[6]) {
    long n = (long)P[0] * P[1] * P[2];
    int hx = P[0] / 2 + 1, hy = P[1] / 2 + 1, hz = P[2] / 2 + 1;
    double scale = 1.0 / (double)n;
    double maximg = 0.0;
    cpx* a = (cpx*)malloc(sizeof(cpx) * n);
    for (int c = 0; c < 6; c++) {
        for (long i = 0; i < n; i++) {
            double v = K[c][i];
            if (round_f32) v = (double)(float)v;
            a[i].re = v;
            a[i].im = 0.0;
        }
        fft3d(a, P, -1);
        for (int z = 0; z < hz; z++)
            for (int y = 0; y < hy; y++)
                for (int x = 0; x < hx; x++) {
                    cpx v = a[((long)z * P[1] + y) * P[0] + x];
                    Kf[c][((long)z * hy + y) * hx + x] = v.re * scale;
                    if (fabs(v.im) > maximg) maximg = fabs(v.im);
                }
    }
    free(a);
    return maximg * sqrt(scale);
}

/* kernel lookup with the mirror rules of kernmulrsymm3d.cl:62-82, extended
 * to kx > Px/2 (the full complex spectrum used here) with the x-odd signs */
static void kern_at(double* const Kf[6], const int P[3], int kx, int ky, int kz, int round_f32,
                    double k[6]) {
    double sx = 1, sy = 1, sz = 1;
    if (kx > P[0] / 2) { kx = P[0] - kx; sx = -1; }
    if (ky > P[1] / 2) { ky = P[1] - ky; sy = -1; }
    if (kz > P[2] / 2) { kz = P[2] - kz; sz = -1; }
    int hx = P[0] / 2 + 1, hy = P[1] / 2 + 1;
    long I = ((long)kz * hy + ky) * hx + kx;
    for (int c = 0; c < 6; c++) {
        double v = Kf[c][I];
        k[c] = round_f32 ? (double)(float)v : v;
    }
    k[3] *= sy * sz; /* yz */
    k[4] *= sx * sz; /* xz */
    k[5] *= sx * sy; /* xy */
}

static void demag_core(const int N[3], const int P[3], double* const Kf[6], cpx* buf[3],
                       int round_f32) {
    long n = (long)P[0] * P[1] * P[2];
    for (int c = 0; c < 3; c++) fft3d(buf[c], P, -1);
#pragma omp parallel for
    for (long I = 0; I < n; I++) {
        int kx = (int)(I % P[0]), ky = (int)((I / P[0]) % P[1]), kz = (int)(I / ((long)P[0] * P[1]));
        double k[6];
        kern_at(Kf, P, kx, ky, kz, round_f32, k);
        cpx mx = buf[0][I], my = buf[1][I], mz = buf[2][I];
        /* kernmulrsymm3d.cl:85-90 (K order xx yy zz yz xz xy) */
        buf[0][I].re = mx.re * k[0] + my.re * k[5] + mz.re * k[4];
        buf[0][I].im = mx.im * k[0] + my.im * k[5] + mz.im * k[4];
        buf[1][I].re = mx.re * k[5] + my.re * k[1] + mz.re * k[3];
        buf[1][I].im = mx.im * k[5] + my.im * k[1] + mz.im * k[3];
        buf[2][I].re = mx.re * k[4] + my.re * k[3] + mz.re * k[2];
        buf[2][I].im = mx.im * k[4] + my.im * k[3] + mz.im * k[2];
    }
    for (int c = 0; c < 3; c++) fft3d(buf[c], P, +1);
    (void)N;
}

/* opencl/conv_demag.go:52-129 with copypadmul2.cl:3-21 and copyunpad.cl:2-13 */
void orc_demag_f32(const int N[3], const int P[3], double* const Kf[6], float* B[3],
                   float* const m[3], const float* vol, const float* Ms, float Ms_mul) {
    long n = (long)P[0] * P[1] * P[2];
    cpx* buf[3];
    for (int c = 0; c < 3; c++) {
        buf[c] = (cpx*)calloc(n, sizeof(cpx));
        for (int z = 0; z < N[2]; z++)
            for (int y = 0; y < N[1]; y++)
                for (int x = 0; x < N[0]; x++) {
                    int s = (z * N[1] + y) * N[0] + x;
                    float fac = Ms == NULL ? Ms_mul : Ms_mul * Ms[s];
                    float bsat = (float)(ORC_MU0 * (double)fac);
                    float v = vol == NULL ? 1.0f : 1.0f * vol[s];
                    float val = bsat * v * m[c][s];
                    buf[c][((long)z * P[1] + y) * P[0] + x].re = val;
                }
    }
    demag_core(N, P, Kf, buf, 1);
    for (int c = 0; c < 3; c++) {
        for (int z = 0; z < N[2]; z++)
            for (int y = 0; y < N[1]; y++)
                for (int x = 0; x < N[0]; x++)
                    B[c][(z * N[1] + y) * N[0] + x] = (float)buf[c][((long)z * P[1] + y) * P[0] + x].re;
        free(buf[c]);
    }
}

void orc_demag_f64(const int N[3], const int P[3], double* const Kf[6], double* B[3],
                   double* const m[3], const double* vol, const double* Ms, double Ms_mul) {
    long n = (long)P[0] * P[1] * P[2];
    cpx* buf[3];
    double mul = (double)(float)Ms_mul; /* amul.clh: float multiplier */
    for (int c = 0; c < 3; c++) {
        buf[c] = (cpx*)calloc(n, sizeof(cpx));
        for (int z = 0; z < N[2]; z++)
            for (int y = 0; y < N[1]; y++)
                for (int x = 0; x < N[0]; x++) {
                    int s = (z * N[1] + y) * N[0] + x;
                    double fac = Ms == NULL ? mul : mul * Ms[s];
                    double bsat = ORC_MU0 * fac;
                    double v = vol == NULL ? 1.0 : vol[s];
                    buf[c][((long)z * P[1] + y) * P[0] + x].re = bsat * v * m[c][s];
                }
    }
    demag_core(N, P, Kf, buf, 0);
    for (int c = 0; c < 3; c++) {
        for (int z = 0; z < N[2]; z++)
            for (int y = 0; y < N[1]; y++)
                for (int x = 0; x < N[0]; x++)
                    B[c][(z * N[1] + y) * N[0] + x] = buf[c][((long)z * P[1] + y) * P[0] + x].re;
        free(buf[c]);
    }
}
