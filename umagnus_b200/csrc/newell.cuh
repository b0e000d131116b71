// newell.cuh -- FP64 Newell demag tensor for one octant of the padded grid.
//
// Restates mag/newellDemagKernel.go (a port of OOMMF's demagcoef):
//   near field: 27-point second differences of Newell's f and g
//     (:613-835) with a magnitude-sorted compensated sum (:506-527);
//   far field (R > asymptotic radius): the 1/R^3..1/R^9 expansion with
//     sub-cell refinement to aspect ratio <= 1.5 (:15-500);
//   self demag (:838-903).
// The expansion coefficients are the published OOMMF values, held as
// monomial tables (NXX_*/NXY_* below, one row per coefficient).
#pragma once
#include <cmath>

namespace umag {
namespace newell {

// ---- magnitude-sorted compensated sum ----------------------------------
__host__ __device__ inline double sorted_sum(double* v, int n) {
    for (int i = 1; i < n; i++) {
        double key = v[i];
        int j = i - 1;
        while (j >= 0 && fabs(v[j]) > fabs(key)) { v[j + 1] = v[j]; j--; }
        v[j + 1] = key;
    }
    double s = v[n - 1], c = 0.0;
    for (int i = n - 2; i >= 0; i--) {
        double a = v[i];
        double y = c + a;
        double lo1 = a - (y - c);
        double t = y + s;
        double lo2 = y - (t - s);
        double e = lo1 + lo2;
        s = t + e;
        c = e - (s - t);
    }
    return s;
}

__host__ __device__ inline double f_fn(double x, double y, double z) {
    x = fabs(x); y = fabs(y); z = fabs(z);
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double R2 = x2 + y2 + z2;
    if (R2 <= 0.0) return 0.0;
    double R = sqrt(R2);
    double p[4];
    int n = 0;
    if (z > 0.0) {
        p[n++] = 2.0 * (2.0 * x2 - y2 - z2) * R;
        double xyz = x * y * z;
        if (xyz > 0.0) p[n++] = -12.0 * xyz * atan2(y * z, x * R);
        double sxz = x2 + z2;
        if (y > 0.0 && sxz > 0.0) p[n++] = 3.0 * y * (z2 - x2) * log(((y + R) * (y + R)) / sxz);
        double sxy = x2 + y2;
        if (sxy > 0.0) p[n++] = 3.0 * z * (y2 - x2) * log(((z + R) * (z + R)) / sxy);
    } else if (x == y) {
        const double K = 2.0 * sqrt(2.0) - 6.0 * log(1.0 + sqrt(2.0));
        p[n++] = K * x2 * x;
    } else {
        p[n++] = 2.0 * (2.0 * x2 - y2) * R;
        if (y > 0.0 && x > 0.0) p[n++] = -6.0 * y * x2 * log((y + R) / x);
    }
    return sorted_sum(p, n) / 12.0;
}

__host__ __device__ inline double g_fn(double x, double y, double z) {
    double sgn = 1.0;
    if (x < 0.0) sgn = -sgn;
    if (y < 0.0) sgn = -sgn;
    x = fabs(x); y = fabs(y); z = fabs(z);
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double R2 = x2 + y2 + z2;
    if (R2 <= 0.0) return 0.0;
    double R = sqrt(R2);
    double p[7];
    int n = 0;
    p[n++] = -2.0 * x * y * R;
    if (z > 0.0) {
        p[n++] = -z * z2 * atan2(x * y, z * R);
        p[n++] = -3.0 * z * y2 * atan2(x * z, y * R);
        p[n++] = -3.0 * z * x2 * atan2(y * z, x * R);
        double sxy = x2 + y2, syz = y2 + z2, sxz = x2 + z2;
        if (sxy > 0.0) p[n++] = 3.0 * x * y * z * log((z + R) * (z + R) / sxy);
        if (syz > 0.0) p[n++] = 0.5 * y * (3.0 * z2 - y2) * log((x + R) * (x + R) / syz);
        if (sxz > 0.0) p[n++] = 0.5 * x * (3.0 * z2 - x2) * log((y + R) * (y + R) / sxz);
    } else {
        if (y > 0.0) p[n++] = -y * y2 * log((x + R) / y);
        if (x > 0.0) p[n++] = -x * x2 * log((y + R) / x);
    }
    return sgn * sorted_sum(p, n) / 6.0;
}

__host__ __device__ inline double logterm(double cx, double q, double num, double den, double div) {
    return q > -0.5 ? cx * log1p(q) / div : cx * log(num / den) / div;
}

// Self demag factor of an x*y*z cell along x (mag/newellDemagKernel.go:838-903)
__host__ __device__ inline double self_nx(double x, double y, double z) {
    if (x <= 0.0 || y <= 0.0 || z <= 0.0) return 0.0;
    if (x == y && y == z) return 1.0 / 3.0;
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double R = sqrt(x2 + y2 + z2);
    double Rxy = sqrt(x2 + y2), Rxz = sqrt(x2 + z2), Ryz = sqrt(y2 + z2);
    double p[8];
    p[0] = 2.0 * x * y * z *
           ((x / (x + Rxy) + (2 * x2 + y2 + z2) / (R * Rxy + x * Rxz)) / (x + Rxz) +
            (x / (x + Rxz) + (2 * x2 + y2 + z2) / (R * Rxz + x * Rxy)) / (x + Rxy)) /
           ((x + R) * (Rxy + Rxz + R));
    p[1] = -1.0 * x * y * z *
           ((y / (y + Rxy) + (2 * y2 + x2 + z2) / (R * Rxy + y * Ryz)) / (y + Ryz) +
            (y / (y + Ryz) + (2 * y2 + x2 + z2) / (R * Ryz + y * Rxy)) / (y + Rxy)) /
           ((y + R) * (Rxy + Ryz + R));
    p[2] = -1.0 * x * y * z *
           ((z / (z + Rxz) + (2 * z2 + x2 + y2) / (R * Rxz + z * Ryz)) / (z + Ryz) +
            (z / (z + Ryz) + (2 * z2 + x2 + y2) / (R * Ryz + z * Rxz)) / (z + Rxz)) /
           ((z + R) * (Rxz + Ryz + R));
    p[3] = 6.0 * atan(y * z / (x * R));
    double q4 = -1.0 * y * z * z * (1.0 / (x + Rxz) + y / (Rxy * Rxz + x * R)) / (Rxz * (y + Rxy));
    p[4] = logterm(3.0 * x, q4, x * (y + R), Rxz * (y + Rxy), z);
    double q5 = -1.0 * y * y * z * (1.0 / (x + Rxy) + z / (Rxy * Rxz + x * R)) / (Rxy * (z + Rxz));
    p[5] = logterm(3.0 * x, q5, x * (z + R), Rxy * (z + Rxz), y);
    double q6 = -1.0 * x2 * z * (1 / (y + Rxy) + z / (Rxy * Ryz + y * R)) / (Rxy * (z + Ryz));
    p[6] = logterm(-3.0 * y, q6, y * (z + R), Rxy * (z + Ryz), x);
    double q7 = -1.0 * x2 * y * (1 / (z + Rxz) + y / (Rxz * Ryz + z * R)) / (Rxz * (y + Ryz));
    p[7] = logterm(-3.0 * z, q7, z * (y + R), Rxz * (y + Ryz), x);
    return sorted_sum(p, 8) / (3.0 * M_PI);
}

// -(D2x D2y D2z) fn on the 3x3x3 offsets: corners -1, edges 2, faces -4, centre 8
template <bool G>
__host__ __device__ inline double stencil27(double x, double y, double z, double dx, double dy, double dz) {
    double v[27];
    int n = 0;
    for (int i = -1; i <= 1; i++)
        for (int j = -1; j <= 1; j++)
            for (int k = -1; k <= 1; k++) {
                int zeros = (i == 0) + (j == 0) + (k == 0);
                double w = zeros == 0 ? -1.0 : zeros == 1 ? 2.0 : zeros == 2 ? -4.0 : 8.0;
                double a = x + i * dx, b = y + j * dy, c = z + k * dz;
                v[n++] = w * (G ? g_fn(a, b, c) : f_fn(a, b, c));
            }
    return sorted_sum(v, 27);
}
__host__ __device__ inline double sda00(double x, double y, double z, double dx, double dy, double dz) {
    if (x == 0.0 && y == 0.0 && z == 0.0) return self_nx(dx, dy, dz) * (4.0 * M_PI * dx * dy * dz);
    return stencil27<false>(x, y, z, dx, dy, dz);
}
__host__ __device__ inline double sda01(double x, double y, double z, double dx, double dy, double dz) {
    if (x == 0.0 || y == 0.0) return 0.0;
    return stencil27<true>(x, y, z, dx, dy, dz);
}

// ---- far field -----------------------------------------------------------
struct Refine {
    double rdx, rdy, rdz, scale;
    int nx, ny, nz;
};
// Coefficients of one expansion (Nxx-type: 6/10/15 terms, Nxy-type: 3/6/10)
struct Expansion {
    int is_xy, cube;
    double lead, self_demag;
    double a[6], b[10], c[15];
    Refine r;
};

// monomials: order 2 {dx2,dy2,dz2}; order 4 {dx4,dx2dy2,dx2dz2,dy4,dy2dz2,dz4};
// order 6 {dx6,dx4dy2,dx4dz2,dx2dy4,dx2dy2dz2,dx2dz4,dy6,dy4dz2,dy2dz4,dz6}
static const double kXxA[6][3] = {{8, -4, -4}, {-24, 27, -3}, {-24, -3, 27}, {3, -4, 1}, {6, -3, -3}, {3, 1, -4}};
static const double kXxB[10][6] = {
    {32, -40, -40, 12, 10, 12},        {-240, 580, 20, -202, -75, 22}, {-240, 20, 580, 22, -75, -202},
    {180, -505, 55, 232, -75, 8},      {360, -450, -450, -180, 900, -180}, {180, 55, -505, 8, -75, 232},
    {-10, 30, -5, -16, 10, -2},        {-30, 55, 20, 8, -75, 22},      {-30, 20, 55, 22, -75, 8},
    {-10, -5, 30, -2, 10, -16}};
static const double kXxC[15][10] = {
    {384, -896, -896, 672, 560, 672, -120, -112, -112, -120},
    {-5376, 22624, 2464, -19488, -7840, 672, 3705, 2198, 938, -345},
    {-5376, 2464, 22624, 672, -7840, -19488, -345, 938, 2198, 3705},
    {10080, -48720, 1680, 49770, -2625, -630, -10440, -1050, 2100, -315},
    {20160, -47040, -47040, -6300, 133350, -6300, 7065, -26670, -26670, 7065},
    {10080, 1680, -48720, -630, -2625, 49770, -315, 2100, -1050, -10440},
    {-3360, 17290, -1610, -19488, 5495, -588, 4848, -3136, 938, -75},
    {-10080, 32970, 14070, -6300, -66675, 12600, -10080, 53340, -26670, 3015},
    {-10080, 14070, 32970, 12600, -66675, -6300, 3015, -26670, 53340, -10080},
    {-3360, -1610, 17290, -588, 5495, -19488, -75, 938, -3136, 4848},
    {105, -560, 70, 672, -280, 42, -192, 224, -112, 15},
    {420, -1610, -350, 672, 2345, -588, 528, -3136, 2198, -345},
    {630, -1470, -1470, -630, 5250, -630, 360, -1050, -1050, 360},
    {420, -350, -1610, -588, 2345, 672, -345, 2198, -3136, 528},
    {105, 70, -560, 42, -280, 672, 15, -112, 224, -192}};
static const double kXyA[3][3] = {{4, -3, -1}, {-3, 4, -1}, {-3, -3, 6}};
static const double kXyB[6][6] = {{16, -30, -10, 10, 5, 2},  {-40, 105, -5, -40, -5, 4},   {-40, -15, 115, 20, -35, -32},
                                  {10, -30, 5, 16, -10, 2},  {20, -15, -35, -40, 115, -32}, {10, 15, -40, 10, -40, 32}};
static const double kXyC[10][10] = {
    {576, -2016, -672, 1680, 840, 336, -315, -210, -126, -45},
    {-3024, 13664, 448, -12670, -2485, 546, 2520, 910, 84, -135},
    {-3024, 1344, 12768, 2730, -10185, -8694, -945, 1680, 2394, 1350},
    {2520, -12670, 910, 13664, -2485, 84, -3024, 448, 546, -135},
    {5040, -9940, -13580, -9940, 49700, -6300, 5040, -13580, -6300, 2700},
    {2520, 2730, -14490, 420, -7875, 17640, -945, 3990, -840, -3600},
    {-315, 1680, -210, -2016, 840, -126, 576, -672, 336, -45},
    {-945, 2730, 1680, 1344, -10185, 2394, -3024, 12768, -8694, 1350},
    {-945, 420, 3990, 2730, -7875, -840, 2520, -14490, 17640, -3600},
    {-315, -630, 2100, -630, 3150, -3360, -315, 2100, -3360, 1440}};

inline double mono2(const double* c, double x2, double y2, double z2) { return c[0] * x2 + c[1] * y2 + c[2] * z2; }
inline double mono4(const double* c, double x2, double y2, double z2) {
    return c[0] * x2 * x2 + c[1] * x2 * y2 + c[2] * x2 * z2 + c[3] * y2 * y2 + c[4] * y2 * z2 + c[5] * z2 * z2;
}
inline double mono6(const double* c, double x2, double y2, double z2) {
    double x4 = x2 * x2, y4 = y2 * y2, z4 = z2 * z2;
    return c[0] * x4 * x2 + c[1] * x4 * y2 + c[2] * x4 * z2 + c[3] * x2 * y4 + c[4] * x2 * y2 * z2 + c[5] * x2 * z4 +
           c[6] * y4 * y2 + c[7] * y4 * z2 + c[8] * y2 * z4 + c[9] * z4 * z2;
}

// Host-side set-up of one expansion for cell (dx, dy, dz) (:98-134, :136-226, :314-386)
inline Expansion make_expansion(int is_xy, double dx, double dy, double dz) {
    Expansion e{};
    e.is_xy = is_xy;
    Refine& r = e.r;
    const double maxratio = 1.5;
    if (dz <= dx && dz <= dy) {
        double xr = ceil(dx / (maxratio * dz)), yr = ceil(dy / (maxratio * dz));
        r.nx = (int)xr; r.rdx = dx / xr; r.ny = (int)yr; r.rdy = dy / yr; r.nz = 1; r.rdz = dz;
    } else if (dy <= dx && dy <= dz) {
        double xr = ceil(dx / (maxratio * dy)), zr = ceil(dz / (maxratio * dy));
        r.nx = (int)xr; r.rdx = dx / xr; r.nz = (int)zr; r.rdz = dz / zr; r.ny = 1; r.rdy = dy;
    } else {
        double yr = ceil(dy / (maxratio * dx)), zr = ceil(dz / (maxratio * dx));
        r.ny = (int)yr; r.rdy = dy / yr; r.nz = (int)zr; r.rdz = dz / zr; r.nx = 1; r.rdx = dx;
    }
    r.scale = 1.0 / ((double)r.nx * (double)r.ny * (double)r.nz);
    double x = r.rdx, y = r.rdy, z = r.rdz;
    double x2 = x * x, y2 = y * y, z2 = z * z;
    e.cube = !((x2 != y2) || (x2 != z2) || (y2 != z2));
    if (!is_xy) {
        e.self_demag = self_nx(x, y, z);
        e.lead = (-1.0 * x * y * z) / (4.0 * M_PI);
        for (int i = 0; i < 6; i++) e.a[i] = e.cube ? 0.0 : (e.lead / 4.0) * mono2(kXxA[i], x2, y2, z2);
        for (int i = 0; i < 10; i++) e.b[i] = (e.lead / 16.0) * mono4(kXxB[i], x2, y2, z2);
        for (int i = 0; i < 15; i++) e.c[i] = (e.lead / 192.0) * mono6(kXxC[i], x2, y2, z2);
    } else {
        e.lead = (-x * y * z / (4 * M_PI));
        for (int i = 0; i < 3; i++) e.a[i] = e.cube ? 0.0 : ((e.lead * 5.0) / 4.0) * mono2(kXyA[i], x2, y2, z2);
        for (int i = 0; i < 6; i++) e.b[i] = ((e.lead * 7.0) / 16.0) * mono4(kXyB[i], x2, y2, z2);
        for (int i = 0; i < 10; i++) e.c[i] = (e.lead / 64.0) * mono6(kXyC[i], x2, y2, z2);
    }
    return e;
}

__host__ __device__ inline double expansion_point(const Expansion& e, double x, double y, double z) {
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double R2 = x2 + y2 + z2;
    if (R2 <= 0.0) return e.is_xy ? 0.0 : e.self_demag;
    double R4 = R2 * R2;
    double R = sqrt(R2);
    double tx2 = x2 / R4, ty2 = y2 / R4, tz2 = z2 / R4;
    double iR2 = 1.0 / R2, iR = 1.0 / R;
    double tz4 = tz2 * tz2;
    const double *a = e.a, *b = e.b, *c = e.c;
    if (!e.is_xy) {
        double tz6 = tz4 * tz2;
        double t3 = (2 * tx2 - ty2 - tz2) * e.lead;
        double t5 = 0.0, t7;
        if (e.cube) {
            double ty4 = ty2 * ty2;
            t7 = ((b[0] * tx2 + (b[1] * ty2 + b[2] * tz2)) * tx2 + (b[3] * ty4 + b[5] * tz4)) * tx2 +
                 b[6] * ty4 * ty2 + b[9] * tz6;
        } else {
            t5 = (a[0] * tx2 + (a[1] * ty2 + a[2] * tz2)) * tx2 + (a[3] * ty2 + a[4] * tz2) * ty2 + a[5] * tz4;
            t7 = ((b[0] * tx2 + (b[1] * ty2 + b[2] * tz2)) * tx2 + ((b[3] * ty2 + b[4] * tz2) * ty2 + b[5] * tz4)) * tx2 +
                 ((b[6] * ty2 + b[7] * tz2) * ty2 + b[8] * tz4) * ty2 + b[9] * tz6;
        }
        double t9 = (((c[0] * tx2 + (c[1] * ty2 + c[2] * tz2)) * tx2 + ((c[3] * ty2 + c[4] * tz2) * ty2 + c[5] * tz4)) * tx2 +
                     (((c[6] * ty2 + c[7] * tz2) * ty2 + c[8] * tz4) * ty2 + c[9] * tz6)) * tx2 +
                    (((c[10] * ty2 + c[11] * tz2) * ty2 + c[12] * tz4) * ty2 + c[13] * tz6) * ty2 + c[14] * tz4 * tz4;
        return (t9 + t7 + t5 + t3) * iR;
    }
    double t3 = 3.0 * e.lead;
    double t5 = e.cube ? 0.0 : a[0] * tx2 + a[1] * ty2 + a[2] * tz2;
    double t7 = (b[0] * tx2 + (b[1] * ty2 + b[2] * tz2)) * tx2 + (b[3] * ty2 + b[4] * tz2) * ty2 + b[5] * tz4;
    double t9 = ((c[0] * tx2 + (c[1] * ty2 + c[2] * tz2)) * tx2 + ((c[3] * ty2 + c[4] * tz2) * ty2 + c[5] * tz4)) * tx2 +
                ((c[6] * ty2 + c[7] * tz2) * ty2 + c[8] * tz4) * ty2 + c[9] * tz4 * tz2;
    double iR5 = iR2 * iR2 * iR;
    return (t9 + t7 + t5 + t3) * iR5 * x * y;
}

// weighted sum over sub-cell offsets, weight (nx-|i|)(ny-|j|)(nz-|k|)
__host__ __device__ inline double expansion_eval(const Expansion& e, double x, double y, double z) {
    const Refine& r = e.r;
    double zsum = 0.0;
    for (int k = 1 - r.nz; k < r.nz; k++) {
        double zo = z + k * r.rdz;
        double ysum = 0.0;
        for (int j = 1 - r.ny; j < r.ny; j++) {
            double yo = y + j * r.rdy;
            double xsum = (double)r.nx * expansion_point(e, x, yo, zo);
            for (int i = 1; i < r.nx; i++)
                xsum += (double)(r.nx - i) * (expansion_point(e, x + i * r.rdx, yo, zo) +
                                              expansion_point(e, x - i * r.rdx, yo, zo));
            ysum += (double)(r.ny - (j < 0 ? -j : j)) * xsum;
        }
        zsum += (double)(r.nz - (k < 0 ? -k : k)) * ysum;
    }
    return zsum * r.scale;
}

// ---- rational cell-size reduction (:905-989) -------------------------------
inline double gcd_f(double m, double n) {
    m = floor(fabs(m)); n = floor(fabs(n));
    if (m == 0.0 || n == 0.0) return 0.0;
    double t = m - floor(m / n) * n;
    while (t > 0.0) { m = n; n = t; t = m - floor(m / n) * n; }
    return n;
}
inline bool rat_approx(double x, double y, double relerr, double maxq, double* p, double* q) {
    if (x < 0.0) x = -x;
    if (y < 0.0) y = -y;
    bool swap = false;
    if (x < y) { double t = x; x = y; y = t; swap = true; }
    double x0 = x, y0 = y, p0 = 0.0, p1 = 1.0, q0 = 1.0, q1 = 0.0;
    double m = floor(x / y), r = x - m * y;
    double p2 = m * p1 + p0, q2 = m * q1 + q0;
    while (q2 < maxq && fabs(x0 * q2 - p2 * y0) > relerr * x0 * q2) {
        x = y; y = r; m = floor(x / y); r = x - m * y;
        p0 = p1; p1 = p2; p2 = m * p1 + p0;
        q0 = q1; q1 = q2; q2 = m * q1 + q0;
    }
    if (!swap) { *p = p2; *q = q2; } else { *p = q2; *q = p2; }
    return fabs(x0 * q2 - p2 * y0) <= relerr * x0 * q2;
}
// Cell sizes reduced to small integers when their ratios are rational
// (mag/newellDemagKernel.go:1141-1159), else scaled by the largest edge.
inline void reduce_cell(double& dx, double& dy, double& dz) {
    double p1, p2, q1, q2;
    if (rat_approx(dx, dy, 1e-12, 1000, &p1, &q1) && rat_approx(dz, dy, 1e-12, 1000, &p2, &q2)) {
        double g = gcd_f(q1, q2);
        dx = p1 * q2 / g; dy = q1 * q2 / g; dz = p2 * q1 / g;
    } else {
        double mx = dx > dy ? dx : dy;
        mx = dz > mx ? dz : mx;
        dx /= mx; dy /= mx; dz /= mx;
    }
}

}  // namespace newell
}  // namespace umag
