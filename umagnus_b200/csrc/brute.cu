// brute.cu -- the brute-force demag kernel on the GPU (mag/demagkernel.go:113-336).
//
// The reference's default demag kernel (engine/demag.go:21,124-133,
// DemagAccuracy = 6): the field of the two charged faces of a source cell,
// each face a staggered nv x nw grid of point charges, averaged over an
// nx x ny x nz grid of points in the destination cell, the point counts set
// by the distance between the cells.  One thread per (source direction s,
// destination cell of the computed octant), FP64 in the reference's
// operation order -- this file is compiled with -fmad=false so that no
// multiply-add is fused, as Go does not fuse them on amd64 -- and each
// result rounded to float32 as the reference stores its kernel.  The other
// octants follow from the mirror signs of demagkernel.go:270-318.
#include <cmath>

#include "common.cuh"
#include "demag.cuh"

namespace umag {

struct BruteArgs {
    int P[3], r1[3], r2[3], ext[3];
    double c[3];
    double accuracy, L;
};

__device__ __forceinline__ double brute_delta(int d) {  // demagkernel.go:360-369
    if (d < 0) d = -d;
    if (d > 0) d -= 1;
    return (double)d;
}
__device__ __forceinline__ int brute_wrap(int n, int max) {  // demagkernel.go:372-381
    while (n < 0) n += max;
    while (n >= max) n -= max;
    return n;
}

// the field of source direction s at destination displacement (x, y, z)
// cells (demagkernel.go:200-268): FP64 in the reference's operation order
__device__ void brute_point(const BruteArgs& a, int s, int x, int y, int z, double B[3]) {
    const int u = s, v = (s + 1) % 3, w = (s + 2) % 3;
    const double* c = a.c;
    double R[3] = {(double)x * c[0], (double)y * c[1], (double)z * c[2]};
    const double dx = brute_delta(x) * c[0], dy = brute_delta(y) * c[1], dz = brute_delta(z) * c[2];
    double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (d == 0) d = a.L;
    const double maxSize = d / a.accuracy;
    int nv = (int)(fmax(c[v] / maxSize, 1.0) + 0.5);
    int nw = (int)(fmax(c[w] / maxSize, 1.0) + 0.5);
    const int nx = (int)(fmax(c[0] / maxSize, 1.0) + 0.5);
    const int ny = (int)(fmax(c[1] / maxSize, 1.0) + 0.5);
    const int nz = (int)(fmax(c[2] / maxSize, 1.0) + 0.5);
    nv *= 2;  // staggered source and destination grids
    nw *= 2;
    const double scale = 1 / (double)(nv * nw * nx * ny * nz);
    const double surface = c[v] * c[w];
    const double charge = surface * scale;
    const double pu1 = c[u] / 2.;
    const double pu2 = -pu1;
    const double fourpi = 4 * M_PI;
    double pole[3], R2[3];
    B[0] = B[1] = B[2] = 0;
    for (int i = 0; i < nv; i++) {
        pole[v] = -(c[v] / 2.) + c[v] / (double)(2 * nv) + (double)i * (c[v] / (double)nv);
        for (int j = 0; j < nw; j++) {
            pole[w] = -(c[w] / 2.) + c[w] / (double)(2 * nw) + (double)j * (c[w] / (double)nw);
            for (int al = 0; al < nx; al++) {
                const double rx = R[0] - c[0] / 2 + c[0] / (double)(2 * nx) + (c[0] / (double)nx) * (double)al;
                for (int be = 0; be < ny; be++) {
                    const double ry = R[1] - c[1] / 2 + c[1] / (double)(2 * ny) + (c[1] / (double)ny) * (double)be;
                    for (int ga = 0; ga < nz; ga++) {
                        const double rz =
                            R[2] - c[2] / 2 + c[2] / (double)(2 * nz) + (c[2] / (double)nz) * (double)ga;
                        pole[u] = pu1;
                        R2[0] = rx - pole[0]; R2[1] = ry - pole[1]; R2[2] = rz - pole[2];
                        double r = sqrt(R2[0] * R2[0] + R2[1] * R2[1] + R2[2] * R2[2]);
                        double qr = charge / (fourpi * r * r * r);
                        const double bx = R2[0] * qr, by = R2[1] * qr, bz = R2[2] * qr;
                        pole[u] = pu2;
                        R2[0] = rx - pole[0]; R2[1] = ry - pole[1]; R2[2] = rz - pole[2];
                        r = sqrt(R2[0] * R2[0] + R2[1] * R2[1] + R2[2] * R2[2]);
                        qr = -charge / (fourpi * r * r * r);
                        B[0] += (bx + R2[0] * qr);  // addition ordered for accuracy (as the reference)
                        B[1] += (by + R2[1] * qr);
                        B[2] += (bz + R2[2] * qr);
                    }
                }
            }
        }
    }
}

// first and last image index k with w + k P in [r1, r2]
__device__ __forceinline__ void brute_images(int w, int P, int r1, int r2, int& k0, int& k1) {
    k0 = (int)floor((double)(r1 - w) / P);
    if (w + k0 * P < r1) k0++;
    k1 = (int)floor((double)(r2 - w) / P);
}

// One thread per (source direction s, octant point in [0, P/2]): the field
// of every periodic image inside the kernel ranges (demagkernel.go:189-268),
// each rounded to float32 and summed in float32 in the reference's loop
// order (z, y, x ascending), as the reference accumulates into its float32
// kernel.  Without PBC the only image is the point itself.
__global__ void k_brute_octant(double* K0, double* K1, double* K2, double* K3, double* K4, double* K5, BruteArgs a) {
    const long npt = (long)a.ext[0] * a.ext[1] * a.ext[2];
    double* K[6] = {K0, K1, K2, K3, K4, K5};
    const int comp[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};  // array[s][d] -> xx yy zz yz xz xy
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < 3 * npt; e += (long)gridDim.x * blockDim.x) {
        const int s = (int)(e / npt);
        const long q = e - s * npt;
        const int xw = (int)(q % a.ext[0]);
        const int yw = (int)((q / a.ext[0]) % a.ext[1]);
        const int zw = (int)(q / ((long)a.ext[0] * a.ext[1]));
        int kx0, kx1, ky0, ky1, kz0, kz1;
        brute_images(xw, a.P[0], a.r1[0], a.r2[0], kx0, kx1);
        brute_images(yw, a.P[1], a.r1[1], a.r2[1], ky0, ky1);
        brute_images(zw, a.P[2], a.r1[2], a.r2[2], kz0, kz1);
        float acc[3] = {0.f, 0.f, 0.f};
        for (int kz = kz0; kz <= kz1; kz++)
            for (int ky = ky0; ky <= ky1; ky++)
                for (int kx = kx0; kx <= kx1; kx++) {
                    double B[3];
                    brute_point(a, s, xw + kx * a.P[0], yw + ky * a.P[1], zw + kz * a.P[2], B);
                    for (int dd = s; dd < 3; dd++) acc[dd] += (float)B[dd];
                }
        const long I = ((long)zw * a.P[1] + yw) * a.P[0] + xw;
        for (int dd = s; dd < 3; dd++) K[comp[s][dd]][I] = (double)acc[dd];  // float32 kernel slices
    }
}

// the seven other octants (mirror signs of demagkernel.go:270-318)
__global__ void k_brute_mirror(double* K0, double* K1, double* K2, double* K3, double* K4, double* K5, int Px, int Py,
                               int Pz) {
    const long n = (long)Px * Py * Pz;
    double* K[6] = {K0, K1, K2, K3, K4, K5};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % Px), y = (int)((i / Px) % Py), z = (int)(i / ((long)Px * Py));
        const bool fx = x > Px / 2, fy = y > Py / 2, fz = z > Pz / 2;
        if (!fx && !fy && !fz) continue;
        const long S = ((long)(fz ? Pz - z : z) * Py + (fy ? Py - y : y)) * Px + (fx ? Px - x : x);
        const double gx = fx ? -1.0 : 1.0, gy = fy ? -1.0 : 1.0, gz = fz ? -1.0 : 1.0;
        const double sgn[6] = {1.0, 1.0, 1.0, gy * gz, gx * gz, gx * gy};
#pragma unroll
        for (int c = 0; c < 6; c++) K[c][i] = sgn[c] * K[c][S];
    }
}

int build_brute(const umag_demag* d, double accuracy, double* Kr[6], cudaStream_t st) {
    UMAG_REQUIRE(accuracy > 0, "demag accuracy must be positive");
    const double* c = d->cell;
    // demagkernel.go:384-398 sanityCheck: cell aspect ratio within 1/100 .. 100
    const double a3 = c[0] / c[1], a2 = c[1] / c[2], a1 = c[2] / c[0];
    const double amax = fmax(a1, fmax(a2, a3)), amin = fmin(a1, fmin(a2, a3));
    if (amax > 100.0 || amin < 1. / 100.) return set_error(UMAG_E_ARG, "unrealistic cell aspect ratio");
    BruteArgs a{};
    for (int i = 0; i < 3; i++) {
        a.P[i] = d->P[i];
        // kernelRanges (demagkernel.go:338-351)
        if (d->pbc[i] == 0) { a.r1[i] = -(d->P[i] - 1) / 2; a.r2[i] = (d->P[i] - 1) / 2; }
        else { a.r1[i] = -(d->P[i] * d->pbc[i] - 1); a.r2[i] = d->P[i] * d->pbc[i] - 1; }
        a.c[i] = c[i];
        a.ext[i] = d->P[i] / 2 + 1;  // the octant [0, P/2]
    }
    if (d->P[2] == 1 && d->pbc[2] == 0) a.r2[2] = 0;
    a.accuracy = accuracy;
    a.L = fmin(c[0], fmin(c[1], c[2]));
    const long n = (long)d->P[0] * d->P[1] * d->P[2];
    for (int k = 0; k < 6; k++) UMAG_CUDA(cudaMemsetAsync(Kr[k], 0, sizeof(double) * n, st));
    const long npt = 3L * a.ext[0] * a.ext[1] * a.ext[2];
    k_brute_octant<<<grid_for(npt, 128, 32), 128, 0, st>>>(Kr[0], Kr[1], Kr[2], Kr[3], Kr[4], Kr[5], a);
    UMAG_LAUNCH_CHECK();
    k_brute_mirror<<<grid_for(n, 256), 256, 0, st>>>(Kr[0], Kr[1], Kr[2], Kr[3], Kr[4], Kr[5], d->P[0], d->P[1],
                                                      d->P[2]);
    UMAG_LAUNCH_CHECK();
    if (d->P[2] == 1) {  // 2D: xz and yz vanish (demagkernel.go:320-324)
        UMAG_CUDA(cudaMemsetAsync(Kr[3], 0, sizeof(double) * n, st));
        UMAG_CUDA(cudaMemsetAsync(Kr[4], 0, sizeof(double) * n, st));
    }
    UMAG_CUDA(cudaStreamSynchronize(st));
    return UMAG_OK;
}

}  // namespace umag
