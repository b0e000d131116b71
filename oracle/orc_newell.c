/*
 * orc_newell.c -- FP64 Newell demag tensor, restated from the reference.
 *
 * TEST INFRASTRUCTURE ONLY (see umag_oracle.h).
 *
 * Follows mag/newellDemagKernel.go (itself a port of OOMMF's demagcoef):
 *   - near field: 27-point second differences of Newell's f and g
 *     (mag/newellDemagKernel.go:613-835) summed with a magnitude-sorted
 *     compensated sum (:506-527);
 *   - far field (R > asymptotic_radius cells): the 1/R^3..1/R^9 asymptotic
 *     expansion with cell refinement to aspect ratio <= 1.5 (:15-500);
 *   - self demag (:838-903), rational cell-size reduction (:936-989),
 *     octant computation + mirror symmetry (:1108-1324).
 * The expansion coefficients are the published OOMMF values; they are kept
 * as monomial tables (one row per coefficient) rather than as the
 * reference's unrolled statements.
 */
#include "umag_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- magnitude-sorted compensated sum (mag/newellDemagKernel.go:506-527) -- */
static double sorted_comp_sum(double* v, int n) {
    if (n <= 0) return 0.0;
    /* ascending |v| (insertion sort, n <= 27) */
    for (int i = 1; i < n; i++) {
        double key = v[i];
        int j = i - 1;
        while (j >= 0 && fabs(v[j]) > fabs(key)) { v[j + 1] = v[j]; j--; }
        v[j + 1] = key;
    }
    /* add from the largest down, carrying a running correction */
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

/* ---- Newell f and g (mag/newellDemagKernel.go:713-835) ------------------- */
double orc_newell_f(double x, double y, double z) {
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
    return sorted_comp_sum(p, n) / 12.0;
}

double orc_newell_g(double x, double y, double z) {
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
    return sgn * sorted_comp_sum(p, n) / 6.0;
}

/* ---- self demag (mag/newellDemagKernel.go:838-903) ----------------------- */
static double log_piece(double coef_x, double piece, double fallback_num, double fallback_den,
                        double div) {
    /* log1p branch when the argument is well conditioned, plain log otherwise */
    if (piece > -0.5) return coef_x * log1p(piece) / div;
    return coef_x * log(fallback_num / fallback_den) / div;
}

double orc_self_demag_nx(double x, double y, double z) {
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
    p[4] = log_piece(3.0 * x, q4, x * (y + R), Rxz * (y + Rxy), z);
    double q5 = -1.0 * y * y * z * (1.0 / (x + Rxy) + z / (Rxy * Rxz + x * R)) / (Rxy * (z + Rxz));
    p[5] = log_piece(3.0 * x, q5, x * (z + R), Rxy * (z + Rxz), y);
    double q6 = -1.0 * x2 * z * (1 / (y + Rxy) + z / (Rxy * Ryz + y * R)) / (Rxy * (z + Ryz));
    p[6] = log_piece(-3.0 * y, q6, y * (z + R), Rxy * (z + Ryz), x);
    double q7 = -1.0 * x2 * y * (1 / (z + Rxz) + y / (Rxz * Ryz + z * R)) / (Rxz * (y + Ryz));
    p[7] = log_piece(-3.0 * z, q7, z * (y + R), Rxz * (y + Ryz), x);
    return sorted_comp_sum(p, 8) / (3.0 * M_PI);
}

/* ---- 27-point stencils (mag/newellDemagKernel.go:613-710) --------------- */
/* Weights of -(D2x D2y D2z) on the 3x3x3 offsets: corners -1, edges +2,
 * faces -4, centre +8. */
static double stencil27(double (*fn)(double, double, double), double x, double y, double z,
                        double dx, double dy, double dz) {
    double v[27];
    int n = 0;
    for (int i = -1; i <= 1; i++)
        for (int j = -1; j <= 1; j++)
            for (int k = -1; k <= 1; k++) {
                int zeros = (i == 0) + (j == 0) + (k == 0);
                double w = (zeros == 0) ? -1.0 : (zeros == 1) ? 2.0 : (zeros == 2) ? -4.0 : 8.0;
                v[n++] = w * fn(x + i * dx, y + j * dy, z + k * dz);
            }
    return sorted_comp_sum(v, 27);
}

static double sda00(double x, double y, double z, double dx, double dy, double dz) {
    if (x == 0.0 && y == 0.0 && z == 0.0)
        return orc_self_demag_nx(dx, dy, dz) * (4.0 * M_PI * dx * dy * dz);
    return stencil27(orc_newell_f, x, y, z, dx, dy, dz);
}
static double sda01(double x, double y, double z, double dx, double dy, double dz) {
    if (x == 0.0 || y == 0.0) return 0.0;
    return stencil27(orc_newell_g, x, y, z, dx, dy, dz);
}

/* ---- far-field asymptotics (mag/newellDemagKernel.go:15-500) ------------- */
typedef struct {
    double x, y, z, tx2, ty2, tz2, R, iR, R2, iR2;
} nab_pt;

static void nab_set(nab_pt* p, double x, double y, double z) {
    p->x = x; p->y = y; p->z = z;
    double x2 = x * x, y2 = y * y, z2 = z * z;
    p->R2 = x2 + y2 + z2;
    double R4 = p->R2 * p->R2;
    p->R = sqrt(p->R2);
    if (p->R2 != 0.0) {
        p->tx2 = x2 / R4; p->ty2 = y2 / R4; p->tz2 = z2 / R4;
        p->iR2 = 1.0 / p->R2; p->iR = 1.0 / p->R;
    } else {
        p->tx2 = p->ty2 = p->tz2 = 0.0;
        p->iR2 = p->R = p->iR = 0.0;
    }
}

typedef struct {
    double rdx, rdy, rdz, scale;
    int nx, ny, nz;
} refine_t;

/* mag/newellDemagKernel.go:98-134: split the cell so no sub-cell edge
 * exceeds maxratio times the shortest edge. */
static void refine_init(refine_t* r, double dx, double dy, double dz, double maxratio) {
    if (dz <= dx && dz <= dy) {
        double xr = ceil(dx / (maxratio * dz)), yr = ceil(dy / (maxratio * dz));
        r->nx = (int)xr; r->rdx = dx / xr;
        r->ny = (int)yr; r->rdy = dy / yr;
        r->nz = 1; r->rdz = dz;
    } else if (dy <= dx && dy <= dz) {
        double xr = ceil(dx / (maxratio * dy)), zr = ceil(dz / (maxratio * dy));
        r->nx = (int)xr; r->rdx = dx / xr;
        r->nz = (int)zr; r->rdz = dz / zr;
        r->ny = 1; r->rdy = dy;
    } else {
        double yr = ceil(dy / (maxratio * dx)), zr = ceil(dz / (maxratio * dx));
        r->ny = (int)yr; r->rdy = dy / yr;
        r->nz = (int)zr; r->rdz = dz / zr;
        r->nx = 1; r->rdx = dx;
    }
    r->scale = 1.0 / ((double)r->nx * (double)r->ny * (double)r->nz);
}

/* Monomial order of the coefficient tables:
 *   order 2: dx2 dy2 dz2
 *   order 4: dx4 dx2dy2 dx2dz2 dy4 dy2dz2 dz4
 *   order 6: dx6 dx4dy2 dx4dz2 dx2dy4 dx2dy2dz2 dx2dz4 dy6 dy4dz2 dy2dz4 dz6 */
static const double NXX_A[6][3] = {
    {8, -4, -4}, {-24, 27, -3}, {-24, -3, 27}, {3, -4, 1}, {6, -3, -3}, {3, 1, -4}};
static const double NXX_B[10][6] = {
    {32, -40, -40, 12, 10, 12},       {-240, 580, 20, -202, -75, 22},
    {-240, 20, 580, 22, -75, -202},   {180, -505, 55, 232, -75, 8},
    {360, -450, -450, -180, 900, -180}, {180, 55, -505, 8, -75, 232},
    {-10, 30, -5, -16, 10, -2},       {-30, 55, 20, 8, -75, 22},
    {-30, 20, 55, 22, -75, 8},        {-10, -5, 30, -2, 10, -16}};
static const double NXX_C[15][10] = {
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
static const double NXY_A[3][3] = {{4, -3, -1}, {-3, 4, -1}, {-3, -3, 6}};
static const double NXY_B[6][6] = {
    {16, -30, -10, 10, 5, 2},   {-40, 105, -5, -40, -5, 4},   {-40, -15, 115, 20, -35, -32},
    {10, -30, 5, 16, -10, 2},   {20, -15, -35, -40, 115, -32}, {10, 15, -40, 10, -40, 32}};
static const double NXY_C[10][10] = {
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

static double mono2(const double* c, double dx2, double dy2, double dz2) {
    return c[0] * dx2 + c[1] * dy2 + c[2] * dz2;
}
static double mono4(const double* c, double dx2, double dy2, double dz2) {
    return c[0] * dx2 * dx2 + c[1] * dx2 * dy2 + c[2] * dx2 * dz2 + c[3] * dy2 * dy2 +
           c[4] * dy2 * dz2 + c[5] * dz2 * dz2;
}
static double mono6(const double* c, double dx2, double dy2, double dz2) {
    double dx4 = dx2 * dx2, dy4 = dy2 * dy2, dz4 = dz2 * dz2;
    return c[0] * dx4 * dx2 + c[1] * dx4 * dy2 + c[2] * dx4 * dz2 + c[3] * dx2 * dy4 +
           c[4] * dx2 * dy2 * dz2 + c[5] * dx2 * dz4 + c[6] * dy4 * dy2 + c[7] * dy4 * dz2 +
           c[8] * dy2 * dz4 + c[9] * dz4 * dz2;
}

typedef struct {
    int cube;
    double self_demag, lead;
    double a[6], b[10], c[15];
} asym_xx;
typedef struct {
    int cube;
    double lead;
    double a[3], b[6], c[10];
} asym_xy;

static void asym_xx_init(asym_xx* s, const refine_t* r) {
    double dx = r->rdx, dy = r->rdy, dz = r->rdz;
    double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
    s->self_demag = orc_self_demag_nx(dx, dy, dz);
    s->lead = (-1.0 * dx * dy * dz) / (4.0 * M_PI);
    s->cube = !((dx2 != dy2) || (dx2 != dz2) || (dy2 != dz2));
    for (int i = 0; i < 6; i++) s->a[i] = s->cube ? 0.0 : (s->lead / 4.0) * mono2(NXX_A[i], dx2, dy2, dz2);
    for (int i = 0; i < 10; i++) s->b[i] = (s->lead / 16.0) * mono4(NXX_B[i], dx2, dy2, dz2);
    for (int i = 0; i < 15; i++) s->c[i] = (s->lead / 192.0) * mono6(NXX_C[i], dx2, dy2, dz2);
}

static double asym_xx_eval(const asym_xx* s, const nab_pt* p) {
    if (p->iR2 <= 0.0) return s->self_demag;
    double tx2 = p->tx2, ty2 = p->ty2, tz2 = p->tz2;
    double tz4 = tz2 * tz2, tz6 = tz4 * tz2;
    const double *a = s->a, *b = s->b, *c = s->c;
    double t3 = (2 * tx2 - ty2 - tz2) * s->lead;
    double t5 = 0.0, t7;
    if (s->cube) {
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
                (((c[10] * ty2 + c[11] * tz2) * ty2 + c[12] * tz4) * ty2 + c[13] * tz6) * ty2 +
                c[14] * tz4 * tz4;
    return (t9 + t7 + t5 + t3) * p->iR;
}

static void asym_xy_init(asym_xy* s, const refine_t* r) {
    double dx = r->rdx, dy = r->rdy, dz = r->rdz;
    double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
    s->lead = (-dx * dy * dz / (4 * M_PI));
    s->cube = !(dx2 != dy2 || dx2 != dz2 || dy2 != dz2);
    for (int i = 0; i < 3; i++)
        s->a[i] = s->cube ? 0.0 : ((s->lead * 5.0) / 4.0) * mono2(NXY_A[i], dx2, dy2, dz2);
    for (int i = 0; i < 6; i++) s->b[i] = ((s->lead * 7.0) / 16.0) * mono4(NXY_B[i], dx2, dy2, dz2);
    for (int i = 0; i < 10; i++) s->c[i] = (s->lead / 64.0) * mono6(NXY_C[i], dx2, dy2, dz2);
}

static double asym_xy_eval(const asym_xy* s, const nab_pt* p) {
    if (p->R2 <= 0.0) return 0.0;
    double tx2 = p->tx2, ty2 = p->ty2, tz2 = p->tz2;
    const double *a = s->a, *b = s->b, *c = s->c;
    double t3 = 3.0 * s->lead;
    double t5 = s->cube ? 0.0 : a[0] * tx2 + a[1] * ty2 + a[2] * tz2;
    double tz4 = tz2 * tz2;
    double t7 = (b[0] * tx2 + (b[1] * ty2 + b[2] * tz2)) * tx2 + (b[3] * ty2 + b[4] * tz2) * ty2 + b[5] * tz4;
    double t9 = ((c[0] * tx2 + (c[1] * ty2 + c[2] * tz2)) * tx2 + ((c[3] * ty2 + c[4] * tz2) * ty2 + c[5] * tz4)) * tx2 +
                ((c[6] * ty2 + c[7] * tz2) * ty2 + c[8] * tz4) * ty2 + c[9] * tz4 * tz2;
    double iR5 = p->iR2 * p->iR2 * p->iR;
    return (t9 + t7 + t5 + t3) * iR5 * p->x * p->y;
}

/* A far-field evaluator: refinement + one of the two base expansions. */
typedef struct {
    refine_t r;
    int is_xy;
    asym_xx xx;
    asym_xy xy;
} asym_t;

static void asym_init(asym_t* s, int is_xy, double dx, double dy, double dz) {
    refine_init(&s->r, dx, dy, dz, 1.5 /* DEMAG_ASYMPTOTIC_DEFAULT_REFINE_RATIO */);
    s->is_xy = is_xy;
    if (is_xy) asym_xy_init(&s->xy, &s->r);
    else asym_xx_init(&s->xx, &s->r);
}

static double asym_base(const asym_t* s, double x, double y, double z) {
    nab_pt p;
    nab_set(&p, x, y, z);
    return s->is_xy ? asym_xy_eval(&s->xy, &p) : asym_xx_eval(&s->xx, &p);
}

/* mag/newellDemagKernel.go:278-312 / 424-467: weighted sum over sub-cell
 * offsets, weight (nx-|i|)(ny-|j|)(nz-|k|). */
static double asym_eval(const asym_t* s, double x, double y, double z) {
    const refine_t* r = &s->r;
    double zsum = 0.0;
    for (int k = 1 - r->nz; k < r->nz; k++) {
        double zo = z + k * r->rdz;
        double ysum = 0.0;
        for (int j = 1 - r->ny; j < r->ny; j++) {
            double yo = y + j * r->rdy;
            double xsum = (double)r->nx * asym_base(s, x, yo, zo);
            for (int i = 1; i < r->nx; i++) {
                double a = asym_base(s, x + i * r->rdx, yo, zo);
                double b = asym_base(s, x - i * r->rdx, yo, zo);
                xsum += (double)(r->nx - i) * (a + b);
            }
            ysum += (double)(r->ny - abs(j)) * xsum;
        }
        zsum += (double)(r->nz - abs(k)) * ysum;
    }
    return zsum * r->scale;
}

/* ---- rational cell-size reduction (mag/newellDemagKernel.go:905-989) ---- */
static double gcd_f(double m, double n) {
    m = floor(fabs(m)); n = floor(fabs(n));
    if (m == 0.0 || n == 0.0) return 0.0;
    double t = m - floor(m / n) * n;
    while (t > 0.0) { m = n; n = t; t = m - floor(m / n) * n; }
    return n;
}

static int rat_approx(double x, double y, double relerr, double maxq, double* p, double* q) {
    if (x < 0.0) x = -x;
    if (y < 0.0) y = -y;
    int swap = 0;
    if (x < y) { double t = x; x = y; y = t; swap = 1; }
    double x0 = x, y0 = y;
    double p0 = 0.0, p1 = 1.0, q0 = 1.0, q1 = 0.0;
    double m = floor(x / y), r = x - m * y;
    double p2 = m * p1 + p0, q2 = m * q1 + q0;
    while (q2 < maxq && fabs(x0 * q2 - p2 * y0) > relerr * x0 * q2) {
        x = y; y = r;
        m = floor(x / y); r = x - m * y;
        p0 = p1; p1 = p2; p2 = m * p1 + p0;
        q0 = q1; q1 = q2; q2 = m * q1 + q0;
    }
    if (!swap) { *p = p2; *q = q2; } else { *p = q2; *q = p2; }
    return fabs(x0 * q2 - p2 * y0) <= relerr * x0 * q2;
}

/* ---- padding and ranges (mag/demagkernel.go:339-352, 404-420) ----------- */
void orc_pad_size(const int size[3], const int pbc[3], int padded[3]) {
    for (int i = 0; i < 3; i++) {
        if (pbc[i] != 0) padded[i] = size[i];
        else if (i != 2 || size[i] > 5) padded[i] = size[i] * 2;
        else padded[i] = size[i] * 2 - 1;
    }
}

static int wrap_idx(int n, int max) {
    while (n < 0) n += max;
    while (n >= max) n -= max;
    return n;
}

int orc_newell_kernel(const int size_in[3], const int pbc[3], const double cellsize[3],
                      int asymptotic_radius, int zero_self_demag, double* K[6]) {
    int P[3];
    orc_pad_size(size_in, pbc, P);
    int r1[3], r2[3];
    for (int c = 0; c < 3; c++) {
        if (pbc[c] == 0) { r1[c] = -(P[c] - 1) / 2; r2[c] = (P[c] - 1) / 2; }
        else { r1[c] = -(P[c] * pbc[c] - 1); r2[c] = P[c] * pbc[c] - 1; }
    }
    if (P[2] == 1 && pbc[2] == 0) r2[2] = 0;
    size_t n = (size_t)P[0] * P[1] * P[2];
    for (int c = 0; c < 6; c++) memset(K[c], 0, n * sizeof(double));

    double dx = cellsize[0], dy = cellsize[1], dz = cellsize[2];
    double p1, p2, q1, q2;
    if (rat_approx(dx, dy, 1e-12, 1000, &p1, &q1) && rat_approx(dz, dy, 1e-12, 1000, &p2, &q2)) {
        double g = gcd_f(q1, q2);
        dx = p1 * q2 / g; dy = q1 * q2 / g; dz = p2 * q1 / g;
    } else {
        double mx = dx;
        if (dy > mx) mx = dy;
        if (dz > mx) mx = dz;
        dx /= mx; dy /= mx; dz /= mx;
    }
    double scale = -1.0 / (4.0 * M_PI * dx * dy * dz);
    double arad = (double)asymptotic_radius * pow(dx * dy * dz, 1.0 / 3.0);
    double arad2 = arad * arad;

    /* component order: 0 xx, 1 yy, 2 zz, 3 yz, 4 xz, 5 xy */
    asym_t Axx, Axy, Axz, Ayy, Ayz, Azz;
    asym_init(&Axx, 0, dx, dy, dz);
    asym_init(&Axy, 1, dx, dy, dz);
    asym_init(&Axz, 1, dx, dz, dy);
    asym_init(&Ayy, 0, dy, dx, dz);
    asym_init(&Ayz, 1, dy, dz, dx);
    asym_init(&Azz, 0, dz, dy, dx);

    int nz = r2[2] - r1[2] + 1;
#pragma omp parallel for schedule(dynamic)
    for (int iz = 0; iz < nz; iz++) {
        int z = r1[2] + iz;
        int zw = wrap_idx(z, P[2]);
        if (zw > P[2] / 2) continue;
        double Rz = z * dz;
        for (int y = r1[1]; y <= r2[1]; y++) {
            int yw = wrap_idx(y, P[1]);
            if (yw > P[1] / 2) continue;
            double Ry = y * dy;
            for (int x = r1[0]; x <= r2[0]; x++) {
                int xw = wrap_idx(x, P[0]);
                if (xw > P[0] / 2) continue;
                double Rx = x * dx;
                size_t I = ((size_t)zw * P[1] + yw) * P[0] + xw;
                double v[6];
                if (arad >= 0.0 && Rx * Rx > arad2 - Rz * Rz - Ry * Ry) {
                    v[0] = -asym_eval(&Axx, Rx, Ry, Rz);
                    v[5] = -asym_eval(&Axy, Rx, Ry, Rz);
                    v[4] = -asym_eval(&Axz, Rx, Rz, Ry);
                    v[1] = -asym_eval(&Ayy, Ry, Rx, Rz);
                    v[3] = -asym_eval(&Ayz, Ry, Rz, Rx);
                    v[2] = -asym_eval(&Azz, Rz, Ry, Rx);
                } else {
                    v[0] = sda00(Rx, Ry, Rz, dx, dy, dz) * scale;
                    v[5] = sda01(Rx, Ry, Rz, dx, dy, dz) * scale;
                    v[4] = sda01(Rx, Rz, Ry, dx, dz, dy) * scale;
                    v[1] = sda00(Ry, Rx, Rz, dy, dx, dz) * scale;
                    v[3] = sda01(Ry, Rz, Rx, dy, dz, dx) * scale;
                    v[2] = sda00(Rz, Ry, Rx, dz, dy, dx) * scale;
                }
                for (int c = 0; c < 6; c++) K[c][I] += v[c];
            }
        }
    }

    /* mirror symmetry: sign of xy flips with x and y, xz with x and z, yz with y and z */
    static const double sx[6] = {1, 1, 1, 1, -1, -1};
    static const double sy[6] = {1, 1, 1, -1, 1, -1};
    static const double sz[6] = {1, 1, 1, -1, -1, 1};
    for (int z = 0; z < P[2]; z++)
        for (int y = 0; y < P[1]; y++)
            for (int x = P[0] / 2 + 1; x < P[0]; x++) {
                size_t d = ((size_t)z * P[1] + y) * P[0] + x, s = ((size_t)z * P[1] + y) * P[0] + (P[0] - x);
                for (int c = 0; c < 6; c++) K[c][d] = sx[c] * K[c][s];
            }
    for (int z = 0; z < P[2]; z++)
        for (int y = P[1] / 2 + 1; y < P[1]; y++)
            for (int x = 0; x < P[0]; x++) {
                size_t d = ((size_t)z * P[1] + y) * P[0] + x, s = ((size_t)z * P[1] + (P[1] - y)) * P[0] + x;
                for (int c = 0; c < 6; c++) K[c][d] = sy[c] * K[c][s];
            }
    for (int z = P[2] / 2 + 1; z < P[2]; z++)
        for (int y = 0; y < P[1]; y++)
            for (int x = 0; x < P[0]; x++) {
                size_t d = ((size_t)z * P[1] + y) * P[0] + x, s = ((size_t)(P[2] - z) * P[1] + y) * P[0] + x;
                for (int c = 0; c < 6; c++) K[c][d] = sz[c] * K[c][s];
            }

    K[0][0] = -orc_self_demag_nx(dx, dy, dz);
    K[1][0] = -orc_self_demag_nx(dy, dz, dx);
    K[2][0] = -orc_self_demag_nx(dz, dx, dy);
    if (zero_self_demag != 0) {
        K[0][0] += 1.0 / 3.0; K[1][0] += 1.0 / 3.0; K[2][0] += 1.0 / 3.0;
    }
    K[3][0] = K[4][0] = K[5][0] = 0.0;
    if (P[2] == 1) {
        memset(K[3], 0, n * sizeof(double));
        memset(K[4], 0, n * sizeof(double));
    }
    return 0;
}
