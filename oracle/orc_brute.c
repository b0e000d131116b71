/* orc_brute.c -- brute-force demag kernel (TEST INFRASTRUCTURE ONLY).
 *
 * Restates mag/demagkernel.go:113-336 CalcDemagKernel: for every destination
 * cell of one octant of the padded grid and every source direction s, the
 * field of the two charged faces of the source cell (point charges on a
 * staggered nv x nw grid) averaged over an nx x ny x nz grid of destination
 * points, the point counts growing near the source (accuracy); FP64
 * arithmetic in the reference's operation order (compiled without
 * contraction), stored as float32 like the reference's kernel slices, the
 * other octants filled by the mirror signs of demagkernel.go:270-318.
 * Output: six arrays (xx yy zz yz xz xy) of size Px*Py*Pz, x fastest.
 */
#include <math.h>
#include <string.h>

#include "umag_oracle.h"

/* demagkernel.go:360-369: closest distance between cells at index distance d */
static double delta_(int d) {
    if (d < 0) d = -d;
    if (d > 0) d -= 1;
    return (double)d;
}
/* demagkernel.go:372-381 */
static int wrap_(int n, int max) {
    while (n < 0) n += max;
    while (n >= max) n -= max;
    return n;
}

int orc_brute_kernel(const int size[3], const int pbc[3], const double cellsize[3], double accuracy,
                     float* const K[6]) {
    int P[3];
    orc_pad_size(size, pbc, P);
    const long n = (long)P[0] * P[1] * P[2];
    /* array[s][d], s <= d: index of the 6-array order xx yy zz yz xz xy */
    static const int comp[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};
    for (int c = 0; c < 6; c++) memset(K[c], 0, sizeof(float) * n);
    int r1[3], r2[3];
    for (int c = 0; c < 3; c++) { /* demagkernel.go:338-351 kernelRanges */
        if (pbc[c] == 0) { r1[c] = -(P[c] - 1) / 2; r2[c] = (P[c] - 1) / 2; }
        else { r1[c] = -(P[c] * pbc[c] - 1); r2[c] = P[c] * pbc[c] - 1; }
    }
    if (P[2] == 1 && pbc[2] == 0) r2[2] = 0;
    double L = cellsize[0];
    if (cellsize[1] < L) L = cellsize[1];
    if (cellsize[2] < L) L = cellsize[2];
    for (int s = 0; s < 3; s++) {
        const int u = s, v = (s + 1) % 3, w = (s + 2) % 3;
        double R[3], R2[3], pole[3];
        for (int z = r1[2]; z <= r2[2]; z++) {
            const int zw = wrap_(z, P[2]);
            if (zw > P[2] / 2) continue;
            R[2] = (double)z * cellsize[2];
            for (int y = r1[1]; y <= r2[1]; y++) {
                const int yw = wrap_(y, P[1]);
                if (yw > P[1] / 2) continue;
                R[1] = (double)y * cellsize[1];
                for (int x = r1[0]; x <= r2[0]; x++) {
                    const int xw = wrap_(x, P[0]);
                    if (xw > P[0] / 2) continue;
                    R[0] = (double)x * cellsize[0];
                    const double dx = delta_(x) * cellsize[0], dy = delta_(y) * cellsize[1], dz = delta_(z) * cellsize[2];
                    double d = sqrt(dx * dx + dy * dy + dz * dz);
                    if (d == 0) d = L;
                    const double maxSize = d / accuracy;
                    int nv = (int)(fmax(cellsize[v] / maxSize, 1) + 0.5);
                    int nw = (int)(fmax(cellsize[w] / maxSize, 1) + 0.5);
                    const int nx = (int)(fmax(cellsize[0] / maxSize, 1) + 0.5);
                    const int ny = (int)(fmax(cellsize[1] / maxSize, 1) + 0.5);
                    const int nz = (int)(fmax(cellsize[2] / maxSize, 1) + 0.5);
                    nv *= 2;
                    nw *= 2;
                    const double scale = 1 / (double)(nv * nw * nx * ny * nz);
                    const double surface = cellsize[v] * cellsize[w];
                    const double charge = surface * scale;
                    const double pu1 = cellsize[u] / 2.;
                    const double pu2 = -pu1;
                    double B[3] = {0, 0, 0};
                    for (int i = 0; i < nv; i++) {
                        const double pv = -(cellsize[v] / 2.) + cellsize[v] / (double)(2 * nv) +
                                          (double)i * (cellsize[v] / (double)nv);
                        pole[v] = pv;
                        for (int j = 0; j < nw; j++) {
                            const double pw = -(cellsize[w] / 2.) + cellsize[w] / (double)(2 * nw) +
                                              (double)j * (cellsize[w] / (double)nw);
                            pole[w] = pw;
                            for (int a = 0; a < nx; a++) {
                                const double rx = R[0] - cellsize[0] / 2 + cellsize[0] / (double)(2 * nx) +
                                                  (cellsize[0] / (double)nx) * (double)a;
                                for (int b = 0; b < ny; b++) {
                                    const double ry = R[1] - cellsize[1] / 2 + cellsize[1] / (double)(2 * ny) +
                                                      (cellsize[1] / (double)ny) * (double)b;
                                    for (int g = 0; g < nz; g++) {
                                        const double rz = R[2] - cellsize[2] / 2 + cellsize[2] / (double)(2 * nz) +
                                                          (cellsize[2] / (double)nz) * (double)g;
                                        pole[u] = pu1;
                                        R2[0] = rx - pole[0]; R2[1] = ry - pole[1]; R2[2] = rz - pole[2];
                                        double r = sqrt(R2[0] * R2[0] + R2[1] * R2[1] + R2[2] * R2[2]);
                                        double qr = charge / (4 * M_PI * r * r * r);
                                        const double bx = R2[0] * qr, by = R2[1] * qr, bz = R2[2] * qr;
                                        pole[u] = pu2;
                                        R2[0] = rx - pole[0]; R2[1] = ry - pole[1]; R2[2] = rz - pole[2];
                                        r = sqrt(R2[0] * R2[0] + R2[1] * R2[1] + R2[2] * R2[2]);
                                        qr = -charge / (4 * M_PI * r * r * r);
                                        B[0] += (bx + R2[0] * qr);
                                        B[1] += (by + R2[1] * qr);
                                        B[2] += (bz + R2[2] * qr);
                                    }
                                }
                            }
                        }
                    }
                    const long I = ((long)zw * P[1] + yw) * P[0] + xw;
                    for (int dd = s; dd < 3; dd++) K[comp[s][dd]][I] += (float)B[dd];
                }
            }
        }
    }
    /* demagkernel.go:270-318: mirror signs (x: xy, xz flip; y: xy, yz; z: xz, yz) */
    for (int z = 0; z < P[2]; z++)
        for (int y = 0; y < P[1]; y++)
            for (int x = P[0] / 2 + 1; x < P[0]; x++) {
                const long I = ((long)z * P[1] + y) * P[0] + x, S = ((long)z * P[1] + y) * P[0] + (P[0] - x);
                K[0][I] = K[0][S]; K[5][I] = -K[5][S]; K[4][I] = -K[4][S];
                K[1][I] = K[1][S]; K[3][I] = K[3][S]; K[2][I] = K[2][S];
            }
    for (int z = 0; z < P[2]; z++)
        for (int y = P[1] / 2 + 1; y < P[1]; y++)
            for (int x = 0; x < P[0]; x++) {
                const long I = ((long)z * P[1] + y) * P[0] + x, S = ((long)z * P[1] + (P[1] - y)) * P[0] + x;
                K[0][I] = K[0][S]; K[5][I] = -K[5][S]; K[4][I] = K[4][S];
                K[1][I] = K[1][S]; K[3][I] = -K[3][S]; K[2][I] = K[2][S];
            }
    for (int z = P[2] / 2 + 1; z < P[2]; z++)
        for (int y = 0; y < P[1]; y++)
            for (int x = 0; x < P[0]; x++) {
                const long I = ((long)z * P[1] + y) * P[0] + x, S = ((long)(P[2] - z) * P[1] + y) * P[0] + x;
                K[0][I] = K[0][S]; K[5][I] = K[5][S]; K[4][I] = -K[4][S];
                K[1][I] = K[1][S]; K[3][I] = -K[3][S]; K[2][I] = K[2][S];
            }
    if (P[2] == 1) { /* 2D: yz and xz vanish (demagkernel.go:320-324) */
        memset(K[3], 0, sizeof(float) * n);
        memset(K[4], 0, sizeof(float) * n);
    }
    return 0;
}
