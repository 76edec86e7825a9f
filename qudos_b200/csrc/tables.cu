// Coefficient tables of the solve path, built on the GPU:
//   shape Fourier transforms chi_s(G)      characteristic_function_fourier.c:58-1411
//   strain eps_ij(G) (strain cell)         strain_region_reciprocal_space.c:24-140,
//                                          strain_fourier_coefficient.c:23-173
//   piezoelectric potential phi(G)         piezo_region_reciprocal_space.c:23-787,
//                                          piezo_fourier_coefficient.c:24-132
//   strain cell -> electronic cell         strain_reciprocal_space.c:23-230,
//                                          piezo_reciprocal_space.c:23-186
//   chi (*) eps convolutions               convolutions.c:24-411
//   fused per-difference coefficients      (feeds the assembly kernel)
//
// Grids are (N_xT, N_yT, N_zT) with flat index iz + N_zT (iy + N_yT ix).  The
// reference's zero-padded FFT convolutions are done on padded grids of at
// least 2 N_T - 1 points per axis, rounded up to sizes with factors 2, 3, 5, 7,
// with the batched mixed-radix FFT kernels below.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#include "qd_complex.cuh"
#include "qd_internal.h"

#define CK(x)                                                                                 \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess)                                                                \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)

typedef struct supercell_geometry geo_t;
typedef struct material_params mat_t;

// --------------------------------------------------------------------------
// Gauss-Legendre rule on [0, 1] for the lens integral I_J0 (96 points)
// --------------------------------------------------------------------------
#define QD_GL_N 96
__constant__ double c_gl_x[QD_GL_N];
__constant__ double c_gl_w[QD_GL_N];

static void gauss_legendre01(int n, double *x, double *w) {
    for (int i = 0; i < n; i++) {
        double z = cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0;
        for (int it = 0; it < 100; it++) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 0; j < n; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j + 1.0) * z * p2 - j * p3) / (j + 1);
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) < 1e-16) break;
        }
        x[i] = 0.5 * (1.0 - z);
        w[i] = 1.0 / ((1.0 - z * z) * pp * pp);  // 2/((1-z^2)pp^2) scaled by 1/2
    }
}

// I_J0(alpha, beta) = int_0^1 x cos(alpha sqrt(1-x^2)) J0(beta x) dx
// (characteristic_function_fourier_integrals.c:107-153).  The integrand is
// entire (cos of alpha*sqrt(1-x^2) is a series in 1-x^2), so the reference's
// adaptive Gauss-Kronrod 61 pass and this 96-point Gauss-Legendre rule agree to
// rounding over the argument range of these grids.
__device__ double i_j0(double alpha, double beta) {
    double s = 0.0;
    for (int i = 0; i < QD_GL_N; i++) {
        double x = c_gl_x[i];
        s += c_gl_w[i] * x * cos(alpha * sqrt(1.0 - x * x)) * j0(beta * x);
    }
    return s;
}

// int_lo^hi x^p J0(a x) exp(i b x) dx, p = 1 or 2: the one-dimensional integrals
// of the cones (I_2, I_2_Gz, I_2_TC, I_2_TC_Gz, I_2_ETC, I_2_ETC_Gz,
// characteristic_function_fourier_integrals.c:217-861), which the reference
// evaluates with GSL's adaptive 61-point Gauss-Kronrod rule to 1e-4.  The
// integrands are entire; a composite 96-point Gauss-Legendre rule with one
// panel per 40 radians of |a| + |b| over the interval reproduces the exact
// integral to rounding, and so the adaptive rule's value wherever it meets its
// tolerance (the oracle restates the adaptive rule).
__device__ zc bessel_moment(double lo, double hi, double a, double b, int p) {
    const double span = hi - lo;
    const int panels = 1 + (int)((fabs(a) + fabs(b)) * fabs(span) / 40.0);
    const double h = span / panels;
    double re = 0.0, im = 0.0;
    for (int k = 0; k < panels; k++) {
        for (int i = 0; i < QD_GL_N; i++) {
            const double x = lo + h * (k + c_gl_x[i]);
            double f = c_gl_w[i] * j0(a * x) * (p == 2 ? x * x : x);
            double sn, cs;
            sincos(b * x, &sn, &cs);
            re += f * cs;
            im += f * sn;
        }
    }
    return zc(h * re, h * im);
}

__device__ inline double sinc_pi(double x) {  // gsl_sf_sinc: sin(pi x)/(pi x)
    if (fabs(x) < 1e-8) return 1.0 - (M_PI * M_PI) * x * x / 6.0;
    return sinpi(x) / (M_PI * x);
}

__device__ zc i_e0(double a, double G) {  // characteristic_function_fourier_integrals.c:28-47
    if (fabs(G) < QD_EPS) return zc(a);
    zc e = cexpi(G * a) - zc(1.0);
    return zc(e.im / G, -e.re / G);  // (e^{iGa}-1)/(iG)
}

// characteristic_function_fourier.c:1112-1296
__device__ zc pyramid_segment(double Gx0, double Gy0, double Gz0, int idx_side, int N_side, double L1,
                              double L2, double L3) {
    double alpha, x0, y0, h;
    if (N_side == 0) alpha = (idx_side == 0 || idx_side == 2) ? atan(L2 / L1) : atan(L1 / L2);
    else alpha = M_PI / (double)N_side;
    if (N_side == 0 && (idx_side == 0 || idx_side == 2)) { x0 = L1; y0 = L2; }
    else if (N_side == 0) { x0 = L2; y0 = L1; }
    else { x0 = L1; y0 = tan(alpha) * L1; }
    h = (N_side == 0) ? L3 : L2;
    double ang = 2.0 * alpha * (double)idx_side;
    double sa, ca;
    sincos(ang, &sa, &ca);
    double Gx = ca * Gx0 + sa * Gy0;
    double Gy = -1.0 * sa * Gx0 + ca * Gy0;
    double Gz = Gz0;
    double G_mag = sqrt(Gx * Gx + Gy * Gy + Gz * Gz);
    const zc I(0.0, 1.0);
    if (fabs(G_mag) < QD_EPS) return zc((x0 * y0 * h) / 3.0);
    if (fabs(Gx) < QD_EPS && fabs(Gy) < QD_EPS) {
        zc t = (zc(1.0) - I * (Gz * h) - cexpi(-Gz * h)) / (Gz * Gz * h * h) - zc(0.5);
        return zc(0.0, 2.0 * y0 * x0 / Gz) * t;
    }
    if (fabs(Gx) < QD_EPS && fabs(Gz) < QD_EPS)
        return zc(((2.0 * h * x0) / (Gy * Gy * y0)) * (1.0 - sin(Gy * y0) / (Gy * y0)));
    if (fabs(Gy) < QD_EPS && fabs(Gz) < QD_EPS) {
        zc e = cexpi(-Gx * x0);
        zc t = zc(-1.0) - e - zc(0.0, 2.0 / (Gx * x0)) + I * e * (2.0 / (Gx * x0));
        return ((2.0 * h * y0) / (Gx * Gx * x0)) * t;
    }
    if (fabs(Gx) < QD_EPS) {
        zc pre(0.0, -x0 / (Gz * Gy));
        double c = 2.0 * (cos(Gy * y0) - 1.0) / (Gy * y0);
        zc ez = cexpi(-Gz * h);
        double ap = Gy * y0 + Gz * h, am = Gy * y0 - Gz * h;
        if (fabs(am) < QD_EPS) return pre * (ez * (zc(0.0, -1.0) + (cexpi(ap) - zc(1.0)) / ap) - zc(c));
        if (fabs(ap) < QD_EPS) return pre * (ez * ((cexpi(-am) - zc(1.0)) / am + I) - zc(c));
        return pre * (ez * ((cexpi(-am) - zc(1.0)) / am + (cexpi(ap) - zc(1.0)) / ap) - zc(c));
    }
    if (fabs(Gy) < QD_EPS) {
        zc pre(0.0, 2.0 * y0 / (Gz * x0));
        zc t2 = (cexpi(-Gx * x0) * zc(1.0, Gx * x0) - zc(1.0)) / (Gx * Gx);
        double q = Gx - (Gz * h) / x0;
        if (fabs(q) < QD_EPS) return pre * (0.5 * x0 * x0 * cexpi(-Gz * h) - t2);
        double r = Gx * x0 - Gz * h;
        return pre * (cexpi(-Gz * h) * (cexpi(-r) * zc(1.0, r) - zc(1.0)) / (q * q) - t2);
    }
    if (fabs(Gz) < QD_EPS) {
        double ap = Gx + (Gy * y0) / x0, am = Gx - (Gy * y0) / x0;
        if (fabs(am) < QD_EPS)
            return (h / Gy) * (zc(1.0 / ap) - zc(0.0, 1.0 / (x0 * ap * ap)) * (cexpi(-x0 * ap) - zc(1.0)) -
                               zc(0.0, 0.5 * x0));
        if (fabs(ap) < QD_EPS)
            return (h / Gy) * (zc(-1.0 / am) + zc(0.0, 1.0 / (x0 * am * am)) * (cexpi(-x0 * am) - zc(1.0)) +
                               zc(0.0, 0.5 * x0));
        return (h / Gy) * (zc(1.0 / ap - 1.0 / am) -
                           zc(0.0, 1.0 / (x0 * ap * ap)) * (cexpi(-x0 * ap) - zc(1.0)) +
                           zc(0.0, 1.0 / (x0 * am * am)) * (cexpi(-x0 * am) - zc(1.0)));
    }
    zc e = cexpi(-Gz * h);
    zc r = i_e0(x0, -Gx - (Gy * y0) / x0 + (Gz * h) / x0) * e - i_e0(x0, -Gx + (Gy * y0) / x0 + (Gz * h) / x0) * e -
           i_e0(x0, -Gx - (Gy * y0) / x0) + i_e0(x0, -Gx + (Gy * y0) / x0);
    return (-1.0 / (Gy * Gz)) * r;
}

// characteristic_function_fourier.c:1298-1411
__device__ zc prism_segment(double Gx0, double Gy0, double Gz0, int idx_side, int N_side, double x0, double h) {
    double alpha = M_PI / (double)N_side;
    double ang = (2.0 * M_PI * (double)idx_side) / N_side;
    double sa, ca;
    sincos(ang, &sa, &ca);
    double Gx = ca * Gx0 + sa * Gy0;
    double Gy = -1.0 * sa * Gx0 + ca * Gy0;
    double Gz = Gz0;
    double G_mag = sqrt(Gx * Gx + Gy * Gy + Gz * Gz);
    double ta = tan(alpha);
    const zc I(0.0, 1.0);
    if (fabs(G_mag) < QD_EPS) return zc(x0 * x0 * h * ta);
    if (fabs(Gx) < QD_EPS && fabs(Gy) < QD_EPS) return zc(2.0 * x0 * x0 * ta * sin(0.5 * Gz * h) / Gz);
    if (fabs(Gx) < QD_EPS && fabs(Gz) < QD_EPS) return zc((2.0 * h / (Gy * Gy * ta)) * (1.0 - cos(Gy * x0 * ta)));
    zc ex = cexpi(-Gx * x0);
    zc bx = I * (x0 * ex) + (1.0 / Gx) * (ex - zc(1.0));
    if (fabs(Gy) < QD_EPS && fabs(Gz) < QD_EPS) return (2.0 * h * ta / Gx) * bx;
    if (fabs(Gx) < QD_EPS) return zc((4.0 * sin(0.5 * Gz * h) / (Gy * Gy * Gz * ta)) * (1.0 - cos(Gy * x0 * ta)));
    if (fabs(Gy) < QD_EPS) return (4.0 * sin(0.5 * Gz * h) * ta / (Gz * Gx)) * bx;
    double pre = (fabs(Gz) < QD_EPS) ? h / Gy : (2.0 / (Gy * Gz)) * sin(0.5 * Gz * h);
    double p = Gy * ta + Gx, m = -Gy * ta + Gx;
    zc tp = zc(1.0) - cexpi(-Gy * x0 * ta - Gx * x0);
    zc tm = zc(1.0) - cexpi(Gy * x0 * ta - Gx * x0);
    if (fabs(p) < QD_EPS) return pre * (zc(0.0, x0) - (1.0 / m) * tm);
    if (fabs(m) < QD_EPS) return pre * ((1.0 / p) * tp - zc(0.0, x0));
    return pre * ((1.0 / p) * tp - (1.0 / m) * tm);
}

// Cylinder of radius R and height H centred in z (characteristic_function_fourier.c:532-578).
__device__ zc cylinder_factor(double Gx, double Gy, double Gz, double R, double H) {
    const double G_mag = sqrt(Gx * Gx + Gy * Gy + Gz * Gz), G_par = sqrt(Gx * Gx + Gy * Gy);
    if (fabs(G_mag) < QD_EPS) return zc(M_PI * R * R * H);
    if (fabs(G_par) < QD_EPS && fabs(Gz) > QD_EPS) return zc(2.0 * M_PI * R * R * sin(0.5 * Gz * H) / Gz);
    if (fabs(Gz) < QD_EPS && fabs(G_par) > QD_EPS) return zc((2.0 * M_PI * R * H * j1(G_par * R)) / G_par);
    return zc((4.0 * M_PI * R * sin(0.5 * Gz * H) * j1(G_par * R)) / (G_par * Gz));
}

// Truncated cone, base radius R1 on z = 0, top radius R2 at z = H
// (characteristic_function_fourier.c:671-723).
__device__ zc truncated_cone_factor(double Gx, double Gy, double Gz, double R1, double R2, double H) {
    const double G_mag = sqrt(Gx * Gx + Gy * Gy + Gz * Gz), G_par = sqrt(Gx * Gx + Gy * Gy);
    const zc I(0.0, 1.0);
    if (fabs(G_mag) < QD_EPS) return zc((M_PI * H * (R1 * R1 + R1 * R2 + R2 * R2)) / 3.0);
    const double d = R1 - R2;
    if (fabs(G_par) < QD_EPS) {
        const zc e = cexpi(-Gz * H);
        const zc t = 0.5 * R2 * R2 * (e - zc(1.0)) +
                     (d * d / ((Gz * H) * (Gz * H))) *
                         (e * (I * ((Gz * R2 * H) / d) - zc(1.0)) + (zc(1.0) - I * ((R1 * Gz * H) / d))) -
                     zc(0.5 * (R1 * R1 - R2 * R2));
        return zc(0.0, 2.0 * M_PI / Gz) * t;
    }
    if (fabs(Gz) < QD_EPS) {
        const zc i2 = bessel_moment(R2 / d, R1 / d, d * G_par, 0.0, 2);
        return (2.0 * M_PI * H) * (zc(R2 * j1(G_par * R2) / G_par) - (d * d) * i2 +
                                   zc((R1 / d) * (R1 * j1(G_par * R1) - R2 * j1(G_par * R2)) / G_par));
    }
    const zc i2 = bessel_moment(R2 / d, R1 / d, d * G_par, Gz * H, 1);
    const zc t = (R2 * j1(G_par * R2) / G_par) * (cexpi(-Gz * H) - zc(1.0)) +
                 (d * d) * cexpi((-Gz * H * R1) / d) * i2 - zc((R1 * j1(G_par * R1) - R2 * j1(G_par * R2)) / G_par);
    return zc(0.0, 2.0 * M_PI / Gz) * t;
}

// characteristic_function_fourier.c:58-1110 for one wave vector.  cell: 0
// electronic cell, 1/2 strain cell, 3 Coulomb cell (volume normalisation).
__device__ zc chi_point(double Gx0, double Gy0, double Gz0, const geo_t *geo, int s, int cell, int softening,
                        double sigma) {
    const geo_t &g = geo[s];
    const geo_t &g0 = geo[0];
    double vol;
    if (cell == 3) vol = g0.CL1 * g0.CL2 * g0.CL3;
    else if (cell == 0 || s == 0) vol = g0.L1 * g0.L2 * g0.L3;
    else vol = g0.SL1 * g0.SL2 * g0.SL3;
    zc r = cexpi(-(Gx0 * g.Ox + Gy0 * g.Oy + Gz0 * g.Oz)) / vol;
    double sa = sin(M_PI * g.alpha / 180), ca = cos(M_PI * g.alpha / 180);
    double sb = sin(M_PI * g.beta / 180), cb = cos(M_PI * g.beta / 180);
    double sg = sin(M_PI * g.gamma / 180), cg = cos(M_PI * g.gamma / 180);
    double Gx = ((cb * ca * cg) - (sa * sg)) * Gx0 + ((cg * cb * sa) + (sg * ca)) * Gy0 + (-sb * cg) * Gz0;
    double Gy = ((cb * -ca * sg) - (sa * cg)) * Gx0 + ((-sg * cb * sa) + (cg * ca)) * Gy0 + (sb * sg) * Gz0;
    double Gz = (sb * ca) * Gx0 + (sa * sb) * Gy0 + (cb)*Gz0;
    if (softening != 0) r *= exp(-0.5 * sigma * sigma * (Gx * Gx + Gy * Gy + Gz * Gz));
    switch (g.shape) {
        case 0:
            r *= g.L1 * sinc_pi((0.5 * Gx * g.L1) / M_PI) * g.L2 * sinc_pi((0.5 * Gy * g.L2) / M_PI) * g.L3 *
                 sinc_pi((0.5 * Gz * g.L3) / M_PI);
            break;
        case 4: {
            double a = Gx * g.L1, b = Gy * g.L2, c = Gz * g.L3;
            double G_mag = sqrt(a * a + b * b + c * c), G_par = sqrt(a * a + b * b);
            if (fabs(G_mag) < QD_EPS) {
                r *= (2.0 * M_PI * g.L1 * g.L2 * g.L3) / 3.0;
            } else {
                double sph = (2.0 * M_PI * g.L1 * g.L2 * g.L3 * (sin(G_mag) - G_mag * cos(G_mag))) /
                             (G_mag * G_mag * G_mag);
                double pre = 2.0 * M_PI * g.L1 * g.L2 / Gz;
                if (fabs(G_par) < QD_EPS) {
                    double t = 0.5 - (cos(Gz * g.L3) + Gz * g.L3 * sin(g.L3 * Gz) - 1.0) / ((Gz * g.L3) * (Gz * g.L3));
                    r *= zc(sph, -pre * t);
                } else if (fabs(Gz) < QD_EPS) {
                    r *= sph;
                } else {
                    double t = j1(G_par) / G_par - i_j0(Gz * g.L3, G_par);
                    r *= zc(sph, -pre * t);
                }
            }
            break;
        }
        case 5: {
            zc seg;
            for (int k = 0; k < 4; k++) seg += pyramid_segment(Gx, Gy, Gz, k, 0, g.L1, g.L2, g.L3);
            r *= seg;
            break;
        }
        case 6: {
            zc seg;
            double h1 = (g.L4 * g.L1) / (g.L1 - g.L3);
            for (int k = 0; k < 4; k++) seg += pyramid_segment(Gx, Gy, Gz, k, 0, g.L1, g.L2, h1);
            double L1b = g.L3, L2b = (g.L2 * g.L3) / g.L1, h2 = (g.L4 * g.L3) / (g.L1 - g.L3);
            zc ez = cexpi(-Gz * g.L4);
            for (int k = 0; k < 4; k++) seg -= ez * pyramid_segment(Gx, Gy, Gz, k, 0, L1b, L2b, h2);
            r *= seg;
            break;
        }
        case 1: {  // sphere, radius L1
            const double G = sqrt(Gx * Gx + Gy * Gy + Gz * Gz);
            if (fabs(G) < QD_EPS) r *= (4.0 * M_PI * g.L1 * g.L1 * g.L1) / 3.0;
            else r *= (4.0 * M_PI * (sin(G * g.L1) - G * g.L1 * cos(G * g.L1))) / (G * G * G);
            break;
        }
        case 2: {  // ellipsoid, semi-axes L1, L2, L3
            const double a = Gx * g.L1, b = Gy * g.L2, c = Gz * g.L3, G = sqrt(a * a + b * b + c * c);
            if (fabs(G) < QD_EPS) r *= (4.0 * M_PI * g.L1 * g.L2 * g.L3) / 3.0;
            else r *= (4.0 * M_PI * g.L1 * g.L2 * g.L3 * (sin(G) - G * cos(G))) / (G * G * G);
            break;
        }
        case 3: {  // hemisphere, radius L1, base at the centre
            const double R = g.L1, G = sqrt(Gx * Gx + Gy * Gy + Gz * Gz), Gp = sqrt(Gx * Gx + Gy * Gy);
            if (fabs(G) < QD_EPS) {
                r *= (2.0 * M_PI * R * R * R) / 3.0;
            } else {
                const double sph = (2.0 * M_PI * (sin(G * R) - G * R * cos(G * R))) / (G * G * G);
                if (fabs(Gp) < QD_EPS && fabs(Gz) > QD_EPS) {
                    const double t = 0.5 - (R * Gz * sin(R * Gz) + cos(R * Gz) - 1.0) / ((Gz * R) * (Gz * R));
                    r *= zc(sph, -(2.0 * M_PI * R * R / Gz) * t);
                } else if (fabs(Gz) < QD_EPS && fabs(Gp) > QD_EPS) {
                    r *= sph;
                } else {
                    const double t = -(2.0 * M_PI * R * j1(Gp * R)) / (Gp * Gz) +
                                     (2.0 * M_PI * R * R * i_j0(Gz * R, Gp * R)) / Gz;
                    r *= zc(sph, t);
                }
            }
            break;
        }
        case 7: {  // N-sided pyramid, N = lround(L3 / 10), inradius L1, height L2
            const int n = (int)lround(0.1 * g.L3);
            zc seg;
            for (int k = 0; k < n; k++) seg += pyramid_segment(Gx, Gy, Gz, k, n, g.L1, g.L2, g.L3);
            r *= seg;
            break;
        }
        case 8: {  // truncated N-sided pyramid, N = lround(L4 / 10): inradii L1 (base), L2 (top), height L3
            const int n = (int)lround(0.1 * g.L4);
            zc seg;
            const double h1 = (g.L1 * g.L3) / (g.L1 - g.L2), h2 = (g.L3 * g.L2) / (g.L1 - g.L2);
            for (int k = 0; k < n; k++) seg += pyramid_segment(Gx, Gy, Gz, k, n, g.L1, h1, g.L3);
            const zc ez = cexpi(-Gz * g.L3);
            for (int k = 0; k < n; k++) seg -= ez * pyramid_segment(Gx, Gy, Gz, k, n, g.L2, h2, g.L3);
            r *= seg;
            break;
        }
        case 9:  // cylinder, radius L1, height L2
            r *= cylinder_factor(Gx, Gy, Gz, g.L1, g.L2);
            break;
        case 10:  // cylindrical ring, radii L1 > L2, height L3
            r *= cylinder_factor(Gx, Gy, Gz, g.L1, g.L3) - cylinder_factor(Gx, Gy, Gz, g.L2, g.L3);
            break;
        case 11: {  // cone, base radius L1, height L2
            const double R = g.L1, H = g.L2, G = sqrt(Gx * Gx + Gy * Gy + Gz * Gz), Gp = sqrt(Gx * Gx + Gy * Gy);
            const zc I(0.0, 1.0);
            if (fabs(G) < QD_EPS) {
                r *= (M_PI * R * R * H) / 3.0;
            } else if (fabs(Gp) < QD_EPS) {
                const zc t = (zc(1.0) - I * (Gz * H) - cexpi(-Gz * H)) / ((Gz * H) * (Gz * H)) - zc(0.5);
                r *= zc(0.0, 2.0 * M_PI * R * R / Gz) * t;
            } else if (fabs(Gz) < QD_EPS) {
                r *= (2.0 * M_PI * R * R * H) * (zc(j1(Gp * R) / (Gp * R)) - bessel_moment(0.0, 1.0, Gp * R, 0.0, 2));
            } else {
                r *= zc(0.0, 2.0 * M_PI * R * R / Gz) * cexpi(-Gz * H) * bessel_moment(0.0, 1.0, Gp * R, Gz * H, 1) -
                     zc(0.0, (2.0 * M_PI * R * j1(Gp * R)) / (Gp * Gz));
            }
            break;
        }
        case 12:  // truncated cone, base radius L1, top radius L2, height L3
            r *= truncated_cone_factor(Gx, Gy, Gz, g.L1, g.L2, g.L3);
            break;
        case 13:  // truncated conic ring: truncated cone (L1, L2, height L4) less a cylinder of radius L3
            r *= truncated_cone_factor(Gx, Gy, Gz, g.L1, g.L2, g.L4) -
                 cexpi(-0.5 * Gz * g.L4) * cylinder_factor(Gx, Gy, Gz, g.L3, g.L4);
            break;
        case 14: {  // elliptical cone, semi-axes L1, L2, height L3
            const double A = g.L1 * g.L2, H = g.L3, G = sqrt(Gx * Gx + Gy * Gy + Gz * Gz);
            const double Gp = sqrt((Gx * g.L1) * (Gx * g.L1) + (Gy * g.L2) * (Gy * g.L2));
            const zc I(0.0, 1.0);
            if (fabs(G) < QD_EPS) {
                r *= (M_PI * A * H) / 3.0;
            } else if (fabs(Gp) < QD_EPS) {
                const zc t = (zc(1.0) - I * (Gz * H) - cexpi(-Gz * H)) / ((Gz * H) * (Gz * H)) - zc(0.5);
                r *= zc(0.0, 2.0 * M_PI * A / Gz) * t;
            } else if (fabs(Gz) < QD_EPS) {
                r *= (2.0 * M_PI * A * H) * (zc(j1(Gp) / Gp) - bessel_moment(0.0, 1.0, Gp, 0.0, 2));
            } else {
                r *= zc(0.0, 2.0 * M_PI * A / Gz) * cexpi(-Gz * H) * bessel_moment(0.0, 1.0, Gp, Gz * H, 1) -
                     zc(0.0, (2.0 * M_PI * A * j1(Gp)) / (Gp * Gz));
            }
            break;
        }
        case 15: {  // truncated elliptical cone: semi-axes L1, L2, top ratio f = L3 / L1, height L4
            const double A = g.L1 * g.L2, H = g.L4, f = g.L3 / g.L1, G = sqrt(Gx * Gx + Gy * Gy + Gz * Gz);
            const double Gp = sqrt((Gx * g.L1) * (Gx * g.L1) + (Gy * g.L2) * (Gy * g.L2));
            const zc I(0.0, 1.0);
            if (fabs(G) < QD_EPS) {
                r *= (M_PI * A * H * (1.0 + f + f * f)) / 3.0;
            } else if (fabs(Gp) < QD_EPS) {
                const zc e = cexpi(-Gz * H);
                const zc t = 0.5 * f * f * (e - zc(1.0)) +
                             ((f - 1.0) / (Gz * Gz * H * H)) *
                                 (e * zc(-f + 1.0, -Gz * H * f) + zc(f - 1.0, Gz * H)) -
                             zc(0.5 * (1.0 - f * f));
                r *= zc(0.0, 2.0 * M_PI * A / Gz) * t;
            } else if (fabs(Gz) < QD_EPS) {
                r *= (2.0 * M_PI * A * H) * (zc(f * j1(f * Gp) / Gp) - bessel_moment(f, 1.0, Gp, 0.0, 2) / (1.0 - f) +
                                             zc((j1(Gp) - f * j1(f * Gp)) / ((1.0 - f) * Gp)));
            } else {
                const zc t = (f * j1(f * Gp) / Gp) * (cexpi(-Gz * H) - zc(1.0)) +
                             cexpi(-Gz * H / (1.0 - f)) * bessel_moment(f, 1.0, Gp, Gz * H / (1.0 - f), 1) -
                             zc((j1(Gp) - f * j1(f * Gp)) / Gp);
                r *= zc(0.0, 2.0 * M_PI * A / Gz) * t;
            }
            break;
        }
        case 18: {  // quantum wire along axis lround(L1 / 10), cross-section L2 x L3
            const int d = (int)lround(0.1 * g.L1);
            double c[3];
            if (cell == 0) { c[0] = g0.L1; c[1] = g0.L2; c[2] = g0.L3; }
            else { c[0] = g0.SL1; c[1] = g0.SL2; c[2] = g0.SL3; }
            double l[3];
            if (d == 0) { l[0] = c[0]; l[1] = g.L2; l[2] = g.L3; }
            else if (d == 1) { l[0] = g.L2; l[1] = c[1]; l[2] = g.L3; }
            else if (d == 2) { l[0] = g.L2; l[1] = g.L3; l[2] = c[2]; }
            else break;  // another axis index leaves the prefactor alone, as in the reference
            r *= l[0] * sinc_pi((0.5 * Gx * l[0]) / M_PI) * l[1] * sinc_pi((0.5 * Gy * l[1]) / M_PI) * l[2] *
                 sinc_pi((0.5 * Gz * l[2]) / M_PI);
            break;
        }
        case 16: {
            int n = (int)lround(0.1 * g.L3);
            zc seg;
            for (int k = 0; k < n; k++) seg += prism_segment(Gx, Gy, Gz, k, n, g.L1, g.L2);
            r *= seg;
            break;
        }
        case 17: {
            int d = (int)lround(0.1 * g.L1);
            double l[3];
            if (cell == 0) { l[0] = g0.L1; l[1] = g0.L2; l[2] = g0.L3; }
            else { l[0] = g0.SL1; l[1] = g0.SL2; l[2] = g0.SL3; }
            if (d < 0 || d > 2) break;  // another axis index leaves the prefactor alone, as in the reference
            l[d] = g.L2;
            r *= l[0] * sinc_pi((0.5 * Gx * l[0]) / M_PI) * l[1] * sinc_pi((0.5 * Gy * l[1]) / M_PI) * l[2] *
                 sinc_pi((0.5 * Gz * l[2]) / M_PI);
            break;
        }
        default:
            r = zc(0.0);
    }
    return r;
}

// One thread per grid point (ix, iy, iz) and shape s0 + blockIdx.y.  Launched
// with 64-thread blocks: the transforms are FP64-latency bound and a small
// grid (21^3 points) then still spreads over every SM.
__global__ void chi_kernel(const geo_t *geo, int s0, int s1, const double *Gx, const double *Gy,
                           const double *Gz, int nx, int ny, int nz, int cell, int softening, double sigma,
                           double2 *out) {
    int64_t n = (int64_t)nx * ny * nz;
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int s = s0 + blockIdx.y;
    if (t >= n || s >= s1) return;
    int ix = (int)(t / ((int64_t)ny * nz)), iy = (int)((t / nz) % ny), iz = (int)(t % nz);
    out[(int64_t)s * n + t] = chi_point(Gx[ix], Gy[iy], Gz[iz], geo, s, cell, softening, sigma).d2();
}

// y += t x over n complex values
__global__ void axpy_kernel(double2 *y, const double2 *x, double t, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = make_double2(y[i].x + t * x[i].x, y[i].y + t * x[i].y);
}

// Fourth-order central difference of shape s's transform along a geometry
// parameter: geo4 holds four copies of the shapes with that parameter at
// +2h, +h, -h, -2h; out = (-chi(+2h) + 8 chi(+h) - 8 chi(-h) + chi(-2h)) / 12,
// which is h dchi/dp to O(h^5).  Block (32, 4): threadIdx.y picks the stencil
// point, so the four evaluations of one grid point run on four warps and a
// small grid still spreads over every SM; the sum keeps the order k = 0..3.
__global__ void __launch_bounds__(128) chi_direction_kernel(const geo_t *geo4, int ns, int s, const double *Gx,
                                                            const double *Gy, const double *Gz, int nx, int ny, int nz,
                                                            int cell, int softening, double sigma, double2 *out) {
    __shared__ double2 part[4][32];
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t t = blockIdx.x * (int64_t)32 + threadIdx.x;
    const int k = threadIdx.y;
    const double w[4] = {-1.0 / 12.0, 8.0 / 12.0, -8.0 / 12.0, 1.0 / 12.0};
    if (t < n) {
        const int ix = (int)(t / ((int64_t)ny * nz)), iy = (int)((t / nz) % ny), iz = (int)(t % nz);
        part[k][threadIdx.x] = (w[k] * chi_point(Gx[ix], Gy[iy], Gz[iz], geo4 + k * ns, s, cell, softening, sigma)).d2();
    }
    __syncthreads();
    if (k == 0 && t < n) {
        zc acc(0.0);
        for (int j = 0; j < 4; j++) acc += zc(part[j][threadIdx.x].x, part[j][threadIdx.x].y);
        out[t] = acc.d2();
    }
}

// --------------------------------------------------------------------------
// Strain (strain_fourier_coefficient.c:108-173), position-independent elastic constants
// --------------------------------------------------------------------------
__device__ double strain_factor(int comp, double Gx, double Gy, double Gz, const mat_t &p0, int isotropic) {
    const int ii[6] = {0, 1, 2, 1, 0, 0}, jj[6] = {0, 1, 2, 2, 2, 1};
    double G3[3] = {Gx, Gy, Gz};
    double Gi = G3[ii[comp]], Gj = G3[jj[comp]];
    double dij = ii[comp] == jj[comp] ? 1.0 : 0.0;
    double G = sqrt(Gx * Gx + Gy * Gy + Gz * Gz);
    double C11 = p0.C11, C12 = p0.C12, C44 = p0.C44;
    if (fabs(G) < QD_EPS) {
        if (isotropic == 1) return dij * (1.0 - (3.0 * C12 + 2.0 * C44) / (3.0 * C12 + 6.0 * C44));
        double D = C11 - C12 - 2.0 * C44;
        double s0 = 1.0 / (C44 + D / 3.0);
        return dij * (1.0 - (0.5 * (C11 + 2.0 * C12) / 3.0) * (2.0 / (C44 + D / 3.0)) / (1.0 + (C12 + C44) * s0));
    }
    if (isotropic == 1) return dij - (((3.0 * C12 + 2.0 * C44) * Gi * Gj) / ((C12 + 2.0 * C44) * G * G));
    double D = C11 - C12 - 2.0 * C44;
    double s = (Gx * Gx) / (C44 * G * G + D * Gx * Gx) + (Gy * Gy) / (C44 * G * G + D * Gy * Gy) +
               (Gz * Gz) / (C44 * G * G + D * Gz * Gz);
    return dij - (0.5 * (C11 + 2.0 * C12) * (2.0 * C44 * G * G + D * (Gi * Gi + Gj * Gj)) * Gi * Gj) /
                     ((1.0 + (C12 + C44) * s) * (C44 * G * G + D * Gi * Gi) * (C44 * G * G + D * Gj * Gj));
}

// eps_c(G) = sum_{s>=1} eps0_s chi_s(G) f_c(G)  (strain_region_reciprocal_space.c:62-140)
__global__ void strain_kernel(const geo_t *geo, const mat_t *mat, int n_shape, const double *Gx,
                              const double *Gy, const double *Gz, int nx, int ny, int nz, int isotropic,
                              const double2 *chi, double2 *eps) {
    int64_t n = (int64_t)nx * ny * nz;
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    int ix = (int)(t / ((int64_t)ny * nz)), iy = (int)((t / nz) % ny), iz = (int)(t % nz);
    double gx = Gx[ix], gy = Gy[iy], gz = Gz[iz];
    double f[6];
    for (int c = 0; c < 6; c++) f[c] = strain_factor(c, gx, gy, gz, mat[0], isotropic);
    zc acc[6];
    for (int s = 1; s < n_shape; s++) {
        double eps0 = (mat[geo[s].embedded].a - mat[s].a) / mat[0].a;
        zc ch(chi[(int64_t)s * n + t]);
        zc e0 = eps0 * ch;
        for (int c = 0; c < 6; c++) acc[c] += e0 * f[c];
    }
    for (int c = 0; c < 6; c++) eps[(int64_t)c * n + t] = acc[c].d2();
}

// --------------------------------------------------------------------------
// Position-dependent elastic constants (Elastic_const 1,
// strain_region_reciprocal_space.c:141-418, strain_fourier_coefficient.c:
// 177-470): per shape s the initial term eps0 chi_s delta_ij, a zeroth-order
// term with the shape's own constants, and `order` corrections, each
// chi_s (*) (previous correction) times a factor of the constant differences
// and the matrix's elastic Green tensor.
// --------------------------------------------------------------------------
__device__ double green_tensor(int comp, double Gx, double Gy, double Gz, double G, double ssum, const mat_t &p0) {
    const int ii[6] = {0, 1, 2, 1, 0, 0}, jj[6] = {0, 1, 2, 2, 2, 1};
    const double G3[3] = {Gx, Gy, Gz};
    const double Gi = G3[ii[comp]], Gj = G3[jj[comp]];
    const double D = p0.C11 - p0.C12 - 2.0 * p0.C44;
    const double dij = ii[comp] == jj[comp] ? 1.0 : 0.0;
    return (dij / (p0.C44 * G * G + D * Gi * Gi)) -
           ((p0.C12 + p0.C44) * Gi * Gj /
            ((1.0 + (p0.C12 + p0.C44) * ssum) * (p0.C44 * G * G + D * Gi * Gi) * (p0.C44 * G * G + D * Gj * Gj)));
}

__device__ double pd_order0_factor(int comp, double Gx, double Gy, double Gz, const mat_t &p0, const mat_t &ps,
                                   int isotropic) {
    const int ii[6] = {0, 1, 2, 1, 0, 0}, jj[6] = {0, 1, 2, 2, 2, 1};
    const double G3[3] = {Gx, Gy, Gz};
    const double Gi = G3[ii[comp]], Gj = G3[jj[comp]];
    const double dij = ii[comp] == jj[comp] ? 1.0 : 0.0;
    const double G = sqrt(Gx * Gx + Gy * Gy + Gz * Gz);
    const double C11 = p0.C11, C12 = p0.C12, C44 = p0.C44, D = C11 - C12 - 2.0 * C44;
    if (fabs(G) < QD_EPS) {
        if (isotropic == 1) return dij * (-1 * (3.0 * ps.C12 + 2.0 * ps.C44) / (3.0 * C12 + 6.0 * C44));
        const double s0 = 1.0 / (C44 + D / 3.0);
        return dij * ((-0.5 * (ps.C11 + 2.0 * ps.C12) / 3.0) * (2.0 / (C44 + D / 3.0)) / (1.0 + (C12 + C44) * s0));
    }
    if (isotropic == 1) return -((3.0 * ps.C12 + 2.0 * ps.C44) * Gi * Gj) / ((C12 + 2.0 * C44) * G * G);
    const double ssum = (Gx * Gx) / (C44 * G * G + D * Gx * Gx) + (Gy * Gy) / (C44 * G * G + D * Gy * Gy) +
                        (Gz * Gz) / (C44 * G * G + D * Gz * Gz);
    return -(0.5 * (ps.C11 + 2.0 * ps.C12) * (2.0 * C44 * G * G + D * (Gi * Gi + Gj * Gj)) * Gi * Gj) /
           ((1.0 + (C12 + C44) * ssum) * (C44 * G * G + D * Gi * Gi) * (C44 * G * G + D * Gj * Gj));
}

__device__ double pd_correction_factor(int comp, double Gx, double Gy, double Gz, const mat_t &p0, const mat_t &ps,
                                       int isotropic) {
    const double G = sqrt(Gx * Gx + Gy * Gy + Gz * Gz);
    const double C11 = p0.C11, C12 = p0.C12, C44 = p0.C44, D = C11 - C12 - 2.0 * C44;
    const double dC11 = ps.C11 - C11, dC12 = ps.C12 - C12, dC44 = ps.C44 - C44;
    if (fabs(G) < QD_EPS) {
        if (comp > 2) return 0.0;
        if (isotropic == 1) return -(1.0 / (3.0 * C44)) * (ps.C11 - C11 + 2.0 * ps.C12 - 2.0 * C12);
        const double s0 = 1.0 / (C44 + D / 3.0);
        return -(s0 / 3.0) * (ps.C11 - C11 + 2.0 * ps.C12 - 2.0 * C12);
    }
    const double ssum = (Gx * Gx) / (C44 * G * G + D * Gx * Gx) + (Gy * Gy) / (C44 * G * G + D * Gy * Gy) +
                        (Gz * Gz) / (C44 * G * G + D * Gz * Gz);
    double g[6];
    for (int c = 0; c < 6; c++) g[c] = green_tensor(c, Gx, Gy, Gz, G, ssum, p0);  // xx yy zz yz xz xy
    switch (comp) {
        case 0: return -1.0 * (Gx * ((dC11 * Gx * g[0]) + (dC12 * Gy * g[5]) + (dC12 * Gz * g[4])));
        case 1: return -1.0 * (Gy * ((dC12 * Gx * g[5]) + (dC11 * Gy * g[1]) + (dC12 * Gz * g[3])));
        case 2: return -1.0 * (Gz * ((dC12 * Gx * g[4]) + (dC12 * Gy * g[3]) + (dC11 * Gz * g[2])));
        case 3: return -0.5 * dC44 * (Gy * ((Gz * g[3]) + (Gy * g[2])) + Gz * ((Gz * g[1]) + (Gy * g[3])));
        case 4: return -0.5 * dC44 * (Gx * ((Gz * g[4]) + (Gx * g[2])) + Gz * ((Gz * g[0]) + (Gx * g[4])));
        default: return -0.5 * dC44 * (Gx * ((Gy * g[5]) + (Gx * g[1])) + Gy * ((Gy * g[0]) + (Gx * g[5])));
    }
}

// Initial and zeroth-order terms of shape s: eps += eps0 chi (delta + f0), corr = eps0 chi f0.
__global__ void strain_pd_init_kernel(const geo_t *geo, const mat_t *mat, int s, const double *Gx, const double *Gy,
                                      const double *Gz, int nx, int ny, int nz, int isotropic, const double2 *chi,
                                      double2 *eps, double2 *corr) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int ix = (int)(t / ((int64_t)ny * nz)), iy = (int)((t / nz) % ny), iz = (int)(t % nz);
    const double eps0 = (mat[geo[s].embedded].a - mat[s].a) / mat[0].a;
    const zc e0 = eps0 * zc(chi[t]);
    for (int c = 0; c < 6; c++) {
        const zc v = e0 * pd_order0_factor(c, Gx[ix], Gy[iy], Gz[iz], mat[0], mat[s], isotropic);
        zc acc(eps[(int64_t)c * n + t]);
        acc += v;
        if (c < 3) acc += e0;
        eps[(int64_t)c * n + t] = acc.d2();
        corr[(int64_t)c * n + t] = v.d2();
    }
}

// One correction order of shape s from conv = chi_s (*) corr: corr = conv f_k, eps += corr.
__global__ void strain_pd_corr_kernel(const mat_t *mat, int s, const double *Gx, const double *Gy, const double *Gz,
                                      int nx, int ny, int nz, int isotropic, const double2 *conv, double2 *eps,
                                      double2 *corr) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int ix = (int)(t / ((int64_t)ny * nz)), iy = (int)((t / nz) % ny), iz = (int)(t % nz);
    for (int c = 0; c < 6; c++) {
        const zc v = zc(conv[(int64_t)c * n + t]) * pd_correction_factor(c, Gx[ix], Gy[iy], Gz[iz], mat[0], mat[s],
                                                                           isotropic);
        zc acc(eps[(int64_t)c * n + t]);
        acc += v;
        eps[(int64_t)c * n + t] = acc.d2();
        corr[(int64_t)c * n + t] = v.d2();
    }
}

// --------------------------------------------------------------------------
// Zero-padded linear convolution machinery on the (2 N_T - 1)^3 grid
// --------------------------------------------------------------------------
struct Grid3 {
    int n[3];
    int64_t size() const { return (int64_t)n[0] * n[1] * n[2]; }
};

// in: nb arrays of N_T^3 (stride_in), out: nb padded arrays (stride_out), placed at [0, N_T)
__global__ void pad_kernel(const double2 *in, int64_t stride_in, double2 *out, int64_t stride_out, int tx, int ty,
                           int tz, int px, int py, int pz) {
    int64_t np = (int64_t)px * py * pz;
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int b = blockIdx.y;
    if (t >= np) return;
    int ix = (int)(t / ((int64_t)py * pz)), iy = (int)((t / pz) % py), iz = (int)(t % pz);
    double2 v = make_double2(0.0, 0.0);
    if (ix < tx && iy < ty && iz < tz) v = in[b * stride_in + ((int64_t)ix * ty + iy) * tz + iz];
    out[b * stride_out + t] = v;
}

// Central N_T^3 block of a padded array times scale (crop after inverse DFT).
__global__ void crop_kernel(const double2 *in, int64_t stride_in, double2 *out, int64_t stride_out, int tx, int ty,
                            int tz, int px, int py, int pz, double scale) {
    int64_t nt = (int64_t)tx * ty * tz;
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int b = blockIdx.y;
    if (t >= nt) return;
    int ix = (int)(t / ((int64_t)ty * tz)), iy = (int)((t / tz) % ty), iz = (int)(t % tz);
    int64_t src = ((int64_t)(ix + tx / 2) * py + (iy + ty / 2)) * pz + (iz + tz / 2);
    double2 v = in[b * stride_in + src];
    out[b * stride_out + t] = make_double2(v.x * scale, v.y * scale);
}

// out[b] = a[ia(b)] * c[ic(b)] elementwise; ia = b*sa + oa, ic = b*sc + oc (strides in arrays)
__global__ void mul_kernel(const double2 *a, int64_t sa, const double2 *c, int64_t sc, double2 *out, int64_t so,
                           int64_t n) {
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int b = blockIdx.y;
    if (t >= n) return;
    zc x(a[b * sa + t]), y(c[b * sc + t]);
    out[b * so + t] = (x * y).d2();
}

// Batched 1-D FFTs along one axis of nb three-dimensional arrays: mixed-radix
// Stockham (self-sorting) transforms in shared memory, LPB lines per block.
// A stage of radix R over a line of n points with Ns = product of the radices
// already applied takes, for every j < n / R, the inputs x[j + r n / R],
// multiplies them by w^(r k) with k = j mod Ns and w = exp(sign 2 pi i /
// (Ns R)), applies the R-point DFT and writes the results to
// (j / Ns) Ns R + k + q Ns (q < R).  Radices 4, 2, 3, 5, 7 come first, any other
// prime factor is one stage of an R-point DFT.  Every twiddle is a power of
// exp(sign 2 pi i / n), tabulated once per block with sincospi.
constexpr int FFT_MAX_STAGES = 16;
struct FftAxis {
    int n, nst;
    int radix[FFT_MAX_STAGES];
};

__global__ void __launch_bounds__(128) fft_axis_kernel(double2 *data, int64_t stride_b, int n0, int n1, int n2,
                                                       int axis, int sign, FftAxis fa, int lpb, int64_t lines) {
    extern __shared__ double2 sm[];
    const int n = fa.n;
    double2 *buf0 = sm, *buf1 = sm + lpb * n, *tw = sm + 2 * lpb * n;
    const int64_t L0 = (int64_t)blockIdx.x * lpb;
    const int nl = (int)min((int64_t)lpb, lines - L0);
    double2 *p = data + (int64_t)blockIdx.y * stride_b;
    // line L starts at base(L) and advances by step
    int64_t step;
    if (axis == 2) step = 1;
    else if (axis == 1) step = n2;
    else step = (int64_t)n1 * n2;
    auto base = [&](int64_t L) -> int64_t {
        if (axis == 2) return L * n2;
        if (axis == 1) return (L / n2) * (int64_t)n1 * n2 + (L % n2);
        return L;
    };
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double s, c;
        sincospi((2.0 * j) / n, &s, &c);
        tw[j] = make_double2(c, sign * s);
    }
    // coalesced loads: along the line for axis 2, across neighbouring lines otherwise
    for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
        int l, e;
        if (axis == 2) { l = idx / n; e = idx % n; }
        else { e = idx / nl; l = idx % nl; }
        buf0[l * n + e] = p[base(L0 + l) + e * step];
    }
    __syncthreads();
    double2 *src = buf0, *dst = buf1;
    int Ns = 1;
    for (int st = 0; st < fa.nst; st++) {
        const int R = fa.radix[st], nR = n / R, tstep = n / (Ns * R), dstep = nR;  // w_n^(tstep) = w_(Ns R)
        for (int idx = threadIdx.x; idx < nl * nR; idx += blockDim.x) {
            const int l = idx / nR, j = idx % nR, k = j % Ns;
            const double2 *x = src + l * n;
            double2 *y = dst + l * n + (j / Ns) * Ns * R + k;
            for (int q = 0; q < R; q++) {
                // twiddle w_(Ns R)^(r k) times the DFT factor w_R^(r q) is w_n^(r inc), inc = k tstep + q dstep
                const int inc = (int)(((int64_t)k * tstep + (int64_t)q * dstep) % n);
                double re = 0.0, im = 0.0;
                int e = 0;
                for (int r = 0; r < R; r++) {
                    const double2 v = x[j + r * nR], w = tw[e];
                    re += v.x * w.x - v.y * w.y;
                    im += v.x * w.y + v.y * w.x;
                    e += inc;
                    if (e >= n) e -= n;
                }
                y[q * Ns] = make_double2(re, im);
            }
        }
        __syncthreads();
        double2 *t = src;
        src = dst;
        dst = t;
        Ns *= R;
    }
    for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
        int l, e;
        if (axis == 2) { l = idx / n; e = idx % n; }
        else { e = idx / nl; l = idx % nl; }
        p[base(L0 + l) + e * step] = src[l * n + e];
    }
}

// Smallest size >= n whose prime factors are 2, 3, 5 and 7.
static int smooth_size(int n) {
    for (int p = n > 1 ? n : 1;; p++) {
        int m = p;
        for (int f : {2, 3, 5, 7})
            while (m % f == 0) m /= f;
        if (m == 1) return p;
    }
}

static FftAxis fft_plan(int n) {
    FftAxis f;
    f.n = n;
    f.nst = 0;
    int m = n;
    const int small[5] = {4, 2, 3, 5, 7};
    for (int i = 0; i < 5; i++)
        while (m % small[i] == 0 && f.nst < FFT_MAX_STAGES - 1) {
            f.radix[f.nst++] = small[i];
            m /= small[i];
        }
    for (int pf = 11; m > 1 && f.nst < FFT_MAX_STAGES; pf += 2)
        while (m % pf == 0) {
            f.radix[f.nst++] = pf;
            m /= pf;
        }
    if (m > 1) f.radix[f.nst++] = m;  // not reached for n < 11^16
    return f;
}

static int dft3(double2 *d, int64_t stride_b, int nb, const Grid3 &g, int sign, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        CK(cudaFuncSetAttribute(fft_axis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        configured = true;
    }
    for (int axis = 2; axis >= 0; axis--) {
        const int n = g.n[axis];
        if (n == 1) continue;
        if (3 * (size_t)n * sizeof(double2) > 200 * 1024)
            return qd_set_error(QD_ERR_UNSUPPORTED, "FFT length %d exceeds the shared-memory line buffer", n);
        const FftAxis fa = fft_plan(n);
        int lpb = 512 / n;
        lpb = lpb < 1 ? 1 : lpb > 16 ? 16 : lpb;
        while (lpb > 1 && (size_t)(2 * lpb + 1) * n * sizeof(double2) > 48 * 1024) lpb--;
        const int64_t lines = g.size() / n;
        const size_t smem = (size_t)(2 * lpb + 1) * n * sizeof(double2);
        for (int b0 = 0; b0 < nb; b0 += 65535) {
            const int bn = nb - b0 < 65535 ? nb - b0 : 65535;
            dim3 grid((unsigned)((lines + lpb - 1) / lpb), (unsigned)bn);
            qd_count_launch(1);
            fft_axis_kernel<<<grid, 128, smem, st>>>(d + (int64_t)b0 * stride_b, stride_b, g.n[0], g.n[1], g.n[2],
                                                     axis, sign, fa, lpb, lines);
        }
    }
    CK(cudaGetLastError());
    return QD_OK;
}

static inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// Batched 3-D DFT (sign -1 forward, +1 inverse without scaling) of nb arrays
// of n[0] x n[1] x n[2] points, stride_b elements apart; shared with the
// Coulomb stage.
extern "C" int qd_dft3_batched(double2 *d, int64_t stride_b, int nb, const int n[3], int sign, void *stream) {
    Grid3 g = {{n[0], n[1], n[2]}};
    int rc = dft3(d, stride_b, nb, g, sign, (cudaStream_t)stream);
    if (rc) return rc;
    CK(cudaGetLastError());
    return QD_OK;
}

// --------------------------------------------------------------------------
// Piezoelectric potential (piezo_fourier_coefficient.c:24-132)
// --------------------------------------------------------------------------
// order 1: t = 6 tables (xx yy zz yz xz xy; only yz xz xy are read), coefficient e
// order 2: t = 12 product tables (xx_yz yy_yz zz_yz xy_xz yy_xz xx_xz zz_xz xy_yz zz_xy xx_xy yy_xy xz_yz)
__global__ void piezo_add_kernel(double2 *phi, const double2 *t, int64_t stride, int order, double e, double B114,
                                 double B124, double B156, double nr0, const double *Gx, const double *Gy,
                                 const double *Gz, int nx, int ny, int nz) {
    int64_t n = (int64_t)nx * ny * nz;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int ix = (int)(i / ((int64_t)ny * nz)), iy = (int)((i / nz) % ny), iz = (int)(i % nz);
    double gx = Gx[ix], gy = Gy[iy], gz = Gz[iz];
    double G = sqrt(gx * gx + gy * gy + gz * gz);
    if (!(G > QD_EPS)) return;
    zc Px, Py, Pz;
    auto T = [&](int k) { return zc(t[(int64_t)k * stride + i]); };
    if (order == 1) {
        Px = 2.0 * e * T(3);
        Py = 2.0 * e * T(4);
        Pz = 2.0 * e * T(5);
    } else {
        Px = 2.0 * B114 * T(0) + 2.0 * B124 * T(1) + 2.0 * B124 * T(2) + 4.0 * B156 * T(3);
        Py = 2.0 * B114 * T(4) + 2.0 * B124 * T(5) + 2.0 * B124 * T(6) + 4.0 * B156 * T(7);
        Pz = 2.0 * B114 * T(8) + 2.0 * B124 * T(9) + 2.0 * B124 * T(10) + 4.0 * B156 * T(11);
    }
    zc dot = gx * Px + gy * Py + gz * Pz;
    zc r = zc(100.0 * dot.im, -100.0 * dot.re) / (8.854188 * nr0 * nr0 * G * G);  // -100 i (G.P)/(...)
    zc acc(phi[i]);
    phi[i] = (acc + r).d2();
}

// --------------------------------------------------------------------------
// Downsampling strain cell -> electronic cell, free lengths
// (strain_reciprocal_space.c:88-165): T_es(G) = (1/V) sum_GS T_s(GS) prod_a I0_a
// --------------------------------------------------------------------------
__global__ void downsample_kernel(const double2 *in, int64_t sin_, double2 *out, int64_t sout, int nb,
                                  const double *Gx, const double *Gy, const double *Gz, int ex, int ey, int ez,
                                  const double *Sx, const double *Sy, const double *Sz, int sx, int sy, int sz,
                                  double L1, double L2, double L3, int same_x, int same_y, int same_z) {
    int64_t n = (int64_t)ex * ey * ez;
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int b = blockIdx.y;
    if (t >= n || b >= nb) return;
    int ix = (int)(t / ((int64_t)ey * ez)), iy = (int)((t / ez) % ey), iz = (int)(t % ez);
    double inv_v = 1.0 / (L1 * L2 * L3);
    zc acc;
    int ax0 = same_x ? ix : 0, ax1 = same_x ? ix + 1 : sx;
    int ay0 = same_y ? iy : 0, ay1 = same_y ? iy + 1 : sy;
    int az0 = same_z ? iz : 0, az1 = same_z ? iz + 1 : sz;
    for (int a = ax0; a < ax1; a++) {
        double dx = Sx[a] - Gx[ix];
        double I0x = fabs(dx) < QD_EPS ? L1 : 2 * sin(dx * L1 / 2) / dx;
        for (int c = ay0; c < ay1; c++) {
            double dy = Sy[c] - Gy[iy];
            double I0y = fabs(dy) < QD_EPS ? L2 : 2 * sin(dy * L2 / 2) / dy;
            for (int d = az0; d < az1; d++) {
                double dz = Sz[d] - Gz[iz];
                double I0z = fabs(dz) < QD_EPS ? L3 : 2 * sin(dz * L3 / 2) / dz;
                zc v(in[b * sin_ + ((int64_t)a * sy + c) * sz + d]);
                acc += ((inv_v * v) * I0x) * I0y * I0z;
            }
        }
    }
    out[b * sout + t] = acc.d2();
}

// Commensurate strain cells, SL = RL L (strain_reciprocal_space_fft.c:23-362,
// piezo_reciprocal_space_fft.c): the reference convolves the strain-cell table
// with chi_0, the electronic cell's cuboid (shape record 0) on the strain grid,
// by zero-padded FFTs and keeps every RL-th point about the centre.  chi_0 is a
// product over axes (L sinc(G L / 2), softened like every shape, times
// 1/(L1 L2 L3)), so the same linear convolution is the separable sum
//   T_es(e) = 1/(L1 L2 L3) sum_s prod_a w_a(e_a, s_a) T_s(s),
//   w_a(e, s) = L_a sinc(GS_a[q] L_a / 2) exp(-sigma^2 GS_a[q]^2 / 2),
//   q = RL_a (e - h_a) - (s - hs_a) + hs_a  (h, hs: centre indices),
// with w = 0 where q leaves the strain grid (the support of the padded chi_0).
// Weights of one axis, row-major n_e x n_s.
__global__ void comm_weights_kernel(const double *GS, int ns, int ne, int RL, double L, int softening, double sigma,
                                    double *W) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ne * ns) return;
    const int e = t / ns, s = t % ns, hs = ns / 2, h = ne / 2;
    const int q = RL * (e - h) - (s - hs) + hs;
    double v = 0.0;
    if (q >= 0 && q < ns) {
        const double g = GS[q];
        v = L * sinc_pi((0.5 * g * L) / M_PI);
        if (softening != 0) v *= exp(-0.5 * sigma * sigma * g * g);
    }
    W[t] = v;
}

// One axis of a separable linear map on nb complex arrays [x][y][z] of extents
// (d0, d1, d2): along `axis` its d[axis] points become n_out points,
// out = scale * W in, W row-major (n_out x d[axis]).
__global__ void sep_axis_kernel(const double2 *in, int64_t sin_, int d0, int d1, int d2, int axis, int n_out,
                                const double *W, double scale, int nb, double2 *out, int64_t sout) {
    const int n_in = axis == 0 ? d0 : axis == 1 ? d1 : d2;
    const int o0 = axis == 0 ? n_out : d0, o1 = axis == 1 ? n_out : d1, o2 = axis == 2 ? n_out : d2;
    const int64_t n = (int64_t)o0 * o1 * o2;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (t >= n || b >= nb) return;
    int i0 = (int)(t / ((int64_t)o1 * o2)), i1 = (int)((t / o2) % o1), i2 = (int)(t % o2);
    int e;
    int64_t stride;
    if (axis == 0) {
        e = i0; i0 = 0; stride = (int64_t)d1 * d2;
    } else if (axis == 1) {
        e = i1; i1 = 0; stride = d2;
    } else {
        e = i2; i2 = 0; stride = 1;
    }
    const double2 *src = in + b * sin_ + ((int64_t)i0 * d1 + i1) * d2 + i2;
    const double *w = W + (int64_t)e * n_in;
    double re = 0.0, im = 0.0;
    for (int k = 0; k < n_in; k++) {
        const double wk = w[k];
        if (wk != 0.0) {
            const double2 v = src[k * stride];
            re += wk * v.x;
            im += wk * v.y;
        }
    }
    out[b * sout + t] = make_double2(scale * re, scale * im);
}

// hydrostatic / biaxial combinations of the six chi (*) eps tables (convolutions.c:313-314)
__global__ void hydro_biax_kernel(double2 *conv8, int64_t n) {
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    zc xx(conv8[t]), yy(conv8[n + t]), zz(conv8[2 * n + t]);
    conv8[6 * n + t] = (xx + yy + zz).d2();
    conv8[7 * n + t] = (xx + yy - 2.0 * zz).d2();
}

// --------------------------------------------------------------------------
// Fused per-difference coefficients (assembly input)
// --------------------------------------------------------------------------
// Field index list of the coefficient table:
//  0 Ecb 1 sc 2 Ehh 3 g1+g2 4 g1-2g2 5 Elh 6 g1-g2 7 g1+2g2 8 Eso 9 g1 10 g2 11 g3 12 P
// 13 CB-edge strain+phi+field 14 HH-edge 15 LH-edge 16 SO-edge 17 Q strain 18 R (b part)
// 19 R (d part) 20 S xz 21 S yz 22..27 T_xx T_xy T_yy T_xz T_yz T_zz (P-weighted strain)
__device__ inline double mparam(const mat_t &m, int k) {
    switch (k) {
        case 0: return m.E_cb;
        case 1: return m.sc;
        case 2: return m.E_hh;
        case 3: return m.g1 + m.g2;
        case 4: return m.g1 - 2.0 * m.g2;
        case 5: return m.E_lh;
        case 6: return m.g1 - m.g2;
        case 7: return m.g1 + 2.0 * m.g2;
        case 8: return m.E_so;
        case 9: return m.g1;
        case 10: return m.g2;
        case 11: return m.g3;
        default: return m.P;
    }
}

__global__ void fused_coef_kernel(const geo_t *geo, const mat_t *mat, int n_shape, int nx, int ny, int nz,
                                  double dgx, double dgy, double dgz, double Fx, double Fy, double Fz, int strain_on,
                                  int piezo_on, const double2 *chi, const double2 *eps, const double2 *phi,
                                  const double2 *conv, double2 *coef) {
    int64_t n = (int64_t)nx * ny * nz;
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    int ix = (int)(t / ((int64_t)ny * nz)), iy = (int)((t / nz) % ny), iz = (int)(t % nz);
    int dx = ix - nx / 2, dy = iy - ny / 2, dz = iz - nz / 2;
    bool d0 = dx == 0 && dy == 0 && dz == 0;
    // parameter_matrix_element.c:23-48
    for (int k = 0; k < 13; k++) {
        zc acc(d0 ? mparam(mat[0], k) : 0.0);
        for (int s = 1; s < n_shape; s++) {
            double dp = mparam(mat[s], k) - mparam(mat[geo[s].embedded], k);
            acc += dp * zc(chi[(int64_t)s * n + t]);
        }
        coef[k * n + t] = acc.d2();
    }
    // field_fourier_coefficient.c:23-55: i F (-1)^(d+1) / (G2 - G1), G2 - G1 = -d * 2 pi / L
    zc field;
    if (dx != 0 && dy == 0 && dz == 0) field = zc(0.0, Fx * ((dx + 1) % 2 == 0 ? 1.0 : -1.0) / (-dx * dgx));
    if (dy != 0 && dx == 0 && dz == 0) field = zc(0.0, Fy * ((dy + 1) % 2 == 0 ? 1.0 : -1.0) / (-dy * dgy));
    if (dz != 0 && dx == 0 && dy == 0) field = zc(0.0, Fz * ((dz + 1) % 2 == 0 ? 1.0 : -1.0) / (-dz * dgz));
    zc cb = field, hh = field, lh = field, so = field, Q, Rb, Rd, Sxz, Syz, Txx, Txy, Tyy, Txz, Tyz, Tzz;
    if (strain_on) {
        const mat_t &p0 = mat[0];
        zc xx(eps[t]), yy(eps[n + t]), zz(eps[2 * n + t]), yz(eps[3 * n + t]), xz(eps[4 * n + t]), xy(eps[5 * n + t]);
        zc tr = xx + yy + zz, bi = xx + yy - 2.0 * zz;
        zc scb = p0.ac * tr, shh = p0.av * tr + 0.5 * p0.b * bi, slh = p0.av * tr - 0.5 * p0.b * bi,
           sso = p0.av * tr;
        Q = sqrt(0.5) * p0.b * bi;
        Rb = p0.b * (xx - yy);
        Rd = p0.d * xy;
        Sxz = p0.d * xz;
        Syz = p0.d * yz;
        Txx = p0.P * xx; Txy = p0.P * xy; Tyy = p0.P * yy; Txz = p0.P * xz; Tyz = p0.P * yz; Tzz = p0.P * zz;
        for (int s = 1; s < n_shape; s++) {
            const mat_t &ps = mat[s], &pe = mat[geo[s].embedded];
            const double2 *cv = conv + (int64_t)s * 8 * n;
            zc cxx(cv[t]), cyy(cv[n + t]), czz(cv[2 * n + t]), cyz(cv[3 * n + t]), cxz(cv[4 * n + t]),
                cxy(cv[5 * n + t]), hyd(cv[6 * n + t]), bia(cv[7 * n + t]);
            double dac = ps.ac - pe.ac, dav = ps.av - pe.av, db = ps.b - pe.b, dd = ps.d - pe.d, dP = ps.P - pe.P;
            scb += dac * hyd;
            shh += dav * hyd + 0.5 * db * bia;
            slh += dav * hyd - 0.5 * db * bia;
            sso += dav * hyd;
            Q += sqrt(0.5) * db * bia;
            Rb += db * (cxx - cyy);
            Rd += dd * cxy;
            Sxz += dd * cxz;
            Syz += dd * cyz;
            Txx += dP * cxx; Txy += dP * cxy; Tyy += dP * cyy; Txz += dP * cxz; Tyz += dP * cyz; Tzz += dP * czz;
        }
        if (piezo_on) {
            zc ph(phi[t]);
            scb += ph; shh += ph; slh += ph; sso += ph;
        }
        cb += scb; hh += shh; lh += slh; so += sso;
        Rb = -0.5 * sqrt(3.0) * Rb;
    }
    zc f[15] = {cb, hh, lh, so, Q, Rb, Rd, Sxz, Syz, Txx, Txy, Tyy, Txz, Tyz, Tzz};
    for (int k = 0; k < 15; k++) coef[(13 + k) * n + t] = f[k].d2();
}

// --------------------------------------------------------------------------
// Orchestration
// --------------------------------------------------------------------------
static int upload_gl_rule() {
    static int done = 0;
    if (done) return QD_OK;
    double x[QD_GL_N], w[QD_GL_N];
    gauss_legendre01(QD_GL_N, x, w);
    CK(cudaMemcpyToSymbol(c_gl_x, x, sizeof(x)));
    CK(cudaMemcpyToSymbol(c_gl_w, w, sizeof(w)));
    done = 1;
    return QD_OK;
}

template <class T>
static int dalloc(T **p, size_t bytes) {
    // stream-ordered pool (per-thread default stream): unlike cudaMalloc / cudaFree it does not
    // synchronise the device, so table builds of concurrent solves do not stall each other
    if (qd_pool_alloc((void **)p, bytes, 0) != 0) return qd_set_error(QD_ERR_NOMEM, "device allocation of %zu bytes", bytes);
    return QD_OK;
}

#define RC(x)                      \
    do {                           \
        int rc_ = (x);             \
        if (rc_ != QD_OK) return rc_; \
    } while (0)

// Convolve every array of `a_hat` (nb arrays, padded grid, transformed) with the
// single transformed array `x_hat`, crop into `out` (nb arrays of N_T^3).
static int conv_batch(const double2 *x_hat, const double2 *a_hat, int nb, const Grid3 &pg, const int nt[3],
                      double2 *tmp, double2 *out, cudaStream_t st) {
    int64_t np = pg.size();
    int64_t ntt = (int64_t)nt[0] * nt[1] * nt[2];
    mul_kernel<<<dim3(nblk(np, 256), nb), 256, 0, st>>>(x_hat, 0, a_hat, np, tmp, np, np);
    RC(dft3(tmp, np, nb, pg, +1, st));
    crop_kernel<<<dim3(nblk(ntt, 256), nb), 256, 0, st>>>(tmp, np, out, ntt, nt[0], nt[1], nt[2], pg.n[0], pg.n[1],
                                                          pg.n[2], 1.0 / (double)np);
    CK(cudaGetLastError());
    return QD_OK;
}

// pairs (a, b) of the second-order products, component order xx yy zz yz xz xy
static const int prod_pairs[12][2] = {{0, 3}, {1, 3}, {2, 3}, {5, 4}, {1, 4}, {0, 4},
                                      {2, 4}, {5, 3}, {2, 5}, {0, 5}, {1, 5}, {4, 3}};

extern "C" int qd_tables_build_dev(struct qd_problem *pr) {
    const qd_params &P = pr->p;
    int ns = P.n_shape;
    cudaStream_t st = 0;
    RC(upload_gl_rule());
    for (int s = 1; s < ns; s++) {
        int sh = pr->geo[s].shape;
        if (sh < 0 || sh > 18) return qd_set_error(QD_ERR_INPUT, "unknown shape %d (shape index %d)", sh, s);
    }
    if (P.strain && P.elastic_const != 0 && P.elastic_order < 0)
        return qd_set_error(QD_ERR_INPUT, "Elastic_const_order must be >= 0");
    if (P.strain && pr->p.strain_type == 1) {
        // 8_band_main.c:159-192: the strain grid must resolve every RL-th wave vector
        const int rl[3] = {pr->geo[0].RL1, pr->geo[0].RL2, pr->geo[0].RL3};
        for (int a = 0; a < 3; a++) {
            if (rl[a] < 1) return qd_set_error(QD_ERR_INPUT, "relative strain length %d must be >= 1", a + 1);
            const int n2 = P.N[a] / 2;
            if (P.NS[a] / 2 < n2 * rl[a] / 2 + (n2 % 2) * (rl[a] % 2))
                return qd_set_error(QD_ERR_INPUT, "M_S_G%c is too small for the relative strain length %d",
                                    "xyz"[a], rl[a]);
        }
    }
    int64_t nT = pr->nT, nTS = pr->nTS;
    // device copies of geometry, materials, grids
    RC(dalloc(&pr->d_geo, sizeof(geo_t) * ns));
    RC(dalloc(&pr->d_mat, sizeof(mat_t) * ns));
    CK(cudaMemcpy(pr->d_geo, pr->geo, sizeof(geo_t) * ns, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(pr->d_mat, pr->mat, sizeof(mat_t) * ns, cudaMemcpyHostToDevice));
    for (int a = 0; a < 3; a++) {
        RC(dalloc(&pr->d_G[a], sizeof(double) * pr->NT[a]));
        CK(cudaMemcpy(pr->d_G[a], pr->G[a], sizeof(double) * pr->NT[a], cudaMemcpyHostToDevice));
        if (P.strain) {
            RC(dalloc(&pr->d_GS[a], sizeof(double) * pr->NTS[a]));
            CK(cudaMemcpy(pr->d_GS[a], pr->GS[a], sizeof(double) * pr->NTS[a], cudaMemcpyHostToDevice));
        }
    }
    const geo_t *dg = (const geo_t *)pr->d_geo;
    const mat_t *dm = (const mat_t *)pr->d_mat;
    double2 *chi, *eps = NULL, *phi = NULL, *conv = NULL;
    RC(dalloc(&chi, sizeof(double2) * nT * ns));
    CK(cudaMemset(chi, 0, sizeof(double2) * nT * ns));
    pr->d_chi = chi;
    if (P.strain) {
        double2 *chi_s, *eps_s, *phi_s;
        RC(dalloc(&chi_s, sizeof(double2) * nTS * ns));
        CK(cudaMemset(chi_s, 0, sizeof(double2) * nTS * ns));
        RC(dalloc(&eps_s, sizeof(double2) * nTS * 6));
        RC(dalloc(&phi_s, sizeof(double2) * nTS));
        CK(cudaMemset(phi_s, 0, sizeof(double2) * nTS));
        pr->d_chi_s = chi_s; pr->d_eps_s = eps_s; pr->d_phi_s = phi_s;
        if (ns > 1) {
            chi_kernel<<<dim3(nblk(nTS, 64), ns - 1), 64, 0, st>>>(dg, 1, ns, pr->d_GS[0], pr->d_GS[1], pr->d_GS[2],
                                                                      pr->NTS[0], pr->NTS[1], pr->NTS[2], 1,
                                                                      P.softening, P.sigma, chi_s);
            CK(cudaGetLastError());
            if (pr->chi_dir_t != 0.0 && pr->d_chi_dir_s)
                axpy_kernel<<<nblk(nTS, 256), 256, 0, st>>>(chi_s + (int64_t)pr->chi_dir_shape * nTS,
                                                            (const double2 *)pr->d_chi_dir_s, pr->chi_dir_t, nTS);
        }
        // isotropic approximation (strain_region_reciprocal_space.c:28-40) mutates C44 of every shape
        if (P.isotropic != 0) {
            for (int s = 0; s < ns; s++) pr->mat[s].C44 = 0.5 * (pr->mat[s].C11 - pr->mat[s].C12);
            CK(cudaMemcpy(pr->d_mat, pr->mat, sizeof(mat_t) * ns, cudaMemcpyHostToDevice));
        }
        if (P.elastic_const == 0) {
            strain_kernel<<<nblk(nTS, 128), 128, 0, st>>>(dg, dm, ns, pr->d_GS[0], pr->d_GS[1], pr->d_GS[2],
                                                          pr->NTS[0], pr->NTS[1], pr->NTS[2], P.isotropic, chi_s,
                                                          eps_s);
            CK(cudaGetLastError());
        } else {
            CK(cudaMemsetAsync(eps_s, 0, sizeof(double2) * nTS * 6, st));
            // any size >= 2 N_TS - 1 keeps the linear convolutions free of wrap-around (the crop reads
            // the central block); the next size with factors 2, 3, 5, 7 keeps the FFTs to small radices
            Grid3 pg = {{smooth_size(2 * pr->NTS[0] - 1), smooth_size(2 * pr->NTS[1] - 1),
                         smooth_size(2 * pr->NTS[2] - 1)}};
            const int64_t np = pg.size();
            double2 *corr, *conv, *work;
            RC(dalloc(&corr, sizeof(double2) * nTS * 6));
            RC(dalloc(&conv, sizeof(double2) * nTS * 6));
            RC(dalloc(&work, sizeof(double2) * np * 13));  // X, 6 transformed corrections, 6 products
            double2 *X = work, *Ch = X + np, *tmp = Ch + 6 * np;
            for (int s = 1; s < ns; s++) {
                strain_pd_init_kernel<<<nblk(nTS, 128), 128, 0, st>>>(
                    dg, dm, s, pr->d_GS[0], pr->d_GS[1], pr->d_GS[2], pr->NTS[0], pr->NTS[1], pr->NTS[2],
                    P.isotropic, chi_s + (int64_t)s * nTS, eps_s, corr);
                if (P.elastic_order > 0) {
                    pad_kernel<<<dim3(nblk(np, 256), 1), 256, 0, st>>>(chi_s + (int64_t)s * nTS, 0, X, 0, pr->NTS[0],
                                                                       pr->NTS[1], pr->NTS[2], pg.n[0], pg.n[1],
                                                                       pg.n[2]);
                    RC(dft3(X, 0, 1, pg, -1, st));
                }
                for (int k = 1; k <= P.elastic_order; k++) {
                    pad_kernel<<<dim3(nblk(np, 256), 6), 256, 0, st>>>(corr, nTS, Ch, np, pr->NTS[0], pr->NTS[1],
                                                                       pr->NTS[2], pg.n[0], pg.n[1], pg.n[2]);
                    RC(dft3(Ch, np, 6, pg, -1, st));
                    RC(conv_batch(X, Ch, 6, pg, pr->NTS, tmp, conv, st));
                    strain_pd_corr_kernel<<<nblk(nTS, 128), 128, 0, st>>>(
                        dm, s, pr->d_GS[0], pr->d_GS[1], pr->d_GS[2], pr->NTS[0], pr->NTS[1], pr->NTS[2], P.isotropic,
                        conv, eps_s, corr);
                }
            }
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(st));
            qd_pool_free(corr, 0);
            qd_pool_free(conv, 0);
            qd_pool_free(work, 0);
        }
        if (P.piezo != 0) {
            Grid3 pg = {{smooth_size(2 * pr->NTS[0] - 1), smooth_size(2 * pr->NTS[1] - 1),
                         smooth_size(2 * pr->NTS[2] - 1)}};
            int64_t np = pg.size();
            int second = (P.piezo == 2 || P.piezo == 3);
            int nbuf = 6 + (second ? 12 : 0) + 1 + 12;
            double2 *work;
            RC(dalloc(&work, sizeof(double2) * np * nbuf));
            double2 *E = work, *F = E + 6 * np, *X = F + (second ? 12 : 0) * np,
                    *tmp = X + np;  // tmp holds 12 padded arrays
            double2 *prod = NULL, *ctab = NULL;
            RC(dalloc(&ctab, sizeof(double2) * nTS * 12));
            pad_kernel<<<dim3(nblk(np, 256), 6), 256, 0, st>>>(eps_s, nTS, E, np, pr->NTS[0], pr->NTS[1], pr->NTS[2],
                                                               pg.n[0], pg.n[1], pg.n[2]);
            RC(dft3(E, np, 6, pg, -1, st));
            const mat_t &m0 = pr->mat[0];
            piezo_add_kernel<<<nblk(nTS, 256), 256, 0, st>>>(phi_s, eps_s, nTS, 1, m0.e14, 0, 0, 0, m0.nr, pr->d_GS[0],
                                                             pr->d_GS[1], pr->d_GS[2], pr->NTS[0], pr->NTS[1],
                                                             pr->NTS[2]);
            if (second) {
                RC(dalloc(&prod, sizeof(double2) * nTS * 12));
                for (int k = 0; k < 12; k++) {
                    mul_kernel<<<dim3(nblk(np, 256), 1), 256, 0, st>>>(E + prod_pairs[k][0] * np, 0,
                                                                       E + prod_pairs[k][1] * np, 0, tmp + k * np, 0,
                                                                       np);
                }
                RC(dft3(tmp, np, 12, pg, +1, st));
                crop_kernel<<<dim3(nblk(nTS, 256), 12), 256, 0, st>>>(tmp, np, prod, nTS, pr->NTS[0], pr->NTS[1],
                                                                      pr->NTS[2], pg.n[0], pg.n[1], pg.n[2],
                                                                      1.0 / (double)np);
                piezo_add_kernel<<<nblk(nTS, 256), 256, 0, st>>>(phi_s, prod, nTS, 2, 0, m0.B114, m0.B124, m0.B156,
                                                                 m0.nr, pr->d_GS[0], pr->d_GS[1], pr->d_GS[2],
                                                                 pr->NTS[0], pr->NTS[1], pr->NTS[2]);
                pad_kernel<<<dim3(nblk(np, 256), 12), 256, 0, st>>>(prod, nTS, F, np, pr->NTS[0], pr->NTS[1],
                                                                    pr->NTS[2], pg.n[0], pg.n[1], pg.n[2]);
                RC(dft3(F, np, 12, pg, -1, st));
            }
            for (int s = 1; s < ns; s++) {
                pad_kernel<<<dim3(nblk(np, 256), 1), 256, 0, st>>>(chi_s + s * nTS, 0, X, 0, pr->NTS[0], pr->NTS[1],
                                                                   pr->NTS[2], pg.n[0], pg.n[1], pg.n[2]);
                RC(dft3(X, 0, 1, pg, -1, st));
                const mat_t &ps = pr->mat[s], &pe = pr->mat[pr->geo[s].embedded];
                RC(conv_batch(X, E, 6, pg, pr->NTS, tmp, ctab, st));
                piezo_add_kernel<<<nblk(nTS, 256), 256, 0, st>>>(phi_s, ctab, nTS, 1, ps.e14 - pe.e14, 0, 0, 0, m0.nr,
                                                                 pr->d_GS[0], pr->d_GS[1], pr->d_GS[2], pr->NTS[0],
                                                                 pr->NTS[1], pr->NTS[2]);
                if (second) {
                    RC(conv_batch(X, F, 12, pg, pr->NTS, tmp, ctab, st));
                    piezo_add_kernel<<<nblk(nTS, 256), 256, 0, st>>>(
                        phi_s, ctab, nTS, 2, 0, ps.B114 - pe.B114, ps.B124 - pe.B124, ps.B156 - pe.B156, m0.nr,
                        pr->d_GS[0], pr->d_GS[1], pr->d_GS[2], pr->NTS[0], pr->NTS[1], pr->NTS[2]);
                }
            }
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(st));
            qd_pool_free(work, 0);
            qd_pool_free(ctab, 0);
            if (prod) qd_pool_free(prod, 0);
        }
        // electronic-cell chi: copy when the cells coincide (8_band_main.c:425-442)
        if (pr->same_cells) {
            CK(cudaMemcpy(chi, chi_s, sizeof(double2) * nT * ns, cudaMemcpyDeviceToDevice));
        } else if (ns > 1) {
            chi_kernel<<<dim3(nblk(nT, 64), ns - 1), 64, 0, st>>>(dg, 1, ns, pr->d_G[0], pr->d_G[1], pr->d_G[2],
                                                                     pr->NT[0], pr->NT[1], pr->NT[2], 0, P.softening,
                                                                     P.sigma, chi);
            CK(cudaGetLastError());
            if (pr->chi_dir_t != 0.0 && pr->d_chi_dir)
                axpy_kernel<<<nblk(nT, 256), 256, 0, st>>>(chi + (int64_t)pr->chi_dir_shape * nT,
                                                           (const double2 *)pr->d_chi_dir, pr->chi_dir_t, nT);
        }
        // downsample strain and phi (free lengths, identity when the cells coincide; or commensurate lengths)
        RC(dalloc(&eps, sizeof(double2) * nT * 6));
        RC(dalloc(&phi, sizeof(double2) * nT));
        CK(cudaMemset(phi, 0, sizeof(double2) * nT));
        const geo_t &g0 = pr->geo[0];
        if (P.strain_type == 1) {
            // commensurate cells: three separable passes (z, y, x) with the weights above
            const int *NTS = pr->NTS, *NT = pr->NT;
            const int rl[3] = {g0.RL1, g0.RL2, g0.RL3};
            const double Ls[3] = {g0.L1, g0.L2, g0.L3};
            double *W;
            double2 *t0, *t1;
            const int64_t woff[3] = {0, (int64_t)NT[0] * NTS[0], (int64_t)NT[0] * NTS[0] + (int64_t)NT[1] * NTS[1]};
            const int64_t n0 = (int64_t)NTS[0] * NTS[1] * NT[2], n1 = (int64_t)NTS[0] * NT[1] * NT[2];
            RC(dalloc(&W, sizeof(double) * (woff[2] + (int64_t)NT[2] * NTS[2])));
            RC(dalloc(&t0, sizeof(double2) * n0 * 6));
            RC(dalloc(&t1, sizeof(double2) * n1 * 6));
            for (int a = 0; a < 3; a++)
                comm_weights_kernel<<<nblk((int64_t)NT[a] * NTS[a], 128), 128, 0, st>>>(
                    pr->d_GS[a], NTS[a], NT[a], rl[a], Ls[a], P.softening, P.sigma, W + woff[a]);
            const double inv_v = 1.0 / (g0.L1 * g0.L2 * g0.L3);
            for (int pass = 0; pass < 2; pass++) {
                const int nb = pass == 0 ? 6 : 1;
                if (pass == 1 && P.piezo == 0) break;
                const double2 *src = pass == 0 ? eps_s : phi_s;
                double2 *dst = pass == 0 ? eps : phi;
                sep_axis_kernel<<<dim3(nblk(n0, 128), nb), 128, 0, st>>>(src, nTS, NTS[0], NTS[1], NTS[2], 2, NT[2],
                                                                         W + woff[2], 1.0, nb, t0, n0);
                sep_axis_kernel<<<dim3(nblk(n1, 128), nb), 128, 0, st>>>(t0, n0, NTS[0], NTS[1], NT[2], 1, NT[1],
                                                                         W + woff[1], 1.0, nb, t1, n1);
                sep_axis_kernel<<<dim3(nblk(nT, 128), nb), 128, 0, st>>>(t1, n1, NTS[0], NT[1], NT[2], 0, NT[0],
                                                                         W + woff[0], inv_v, nb, dst, nT);
            }
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(st));
            qd_pool_free(W, 0);
            qd_pool_free(t0, 0);
            qd_pool_free(t1, 0);
        } else {
            int same[3];
            for (int a = 0; a < 3; a++) {
                double L = a == 0 ? g0.L1 : a == 1 ? g0.L2 : g0.L3, SL = a == 0 ? g0.SL1 : a == 1 ? g0.SL2 : g0.SL3;
                same[a] = P.N[a] == P.NS[a] && L == SL;
            }
            downsample_kernel<<<dim3(nblk(nT, 128), 6), 128, 0, st>>>(
                eps_s, nTS, eps, nT, 6, pr->d_G[0], pr->d_G[1], pr->d_G[2], pr->NT[0], pr->NT[1], pr->NT[2],
                pr->d_GS[0], pr->d_GS[1], pr->d_GS[2], pr->NTS[0], pr->NTS[1], pr->NTS[2], g0.L1, g0.L2, g0.L3,
                same[0], same[1], same[2]);
            if (P.piezo != 0)
                downsample_kernel<<<dim3(nblk(nT, 128), 1), 128, 0, st>>>(
                    phi_s, nTS, phi, nT, 1, pr->d_G[0], pr->d_G[1], pr->d_G[2], pr->NT[0], pr->NT[1], pr->NT[2],
                    pr->d_GS[0], pr->d_GS[1], pr->d_GS[2], pr->NTS[0], pr->NTS[1], pr->NTS[2], g0.L1, g0.L2, g0.L3,
                    same[0], same[1], same[2]);
            CK(cudaGetLastError());
        }
        pr->d_eps = eps; pr->d_phi = phi;
        // convolutions chi_s (*) eps_ij (convolutions.c)
        Grid3 pg = {{smooth_size(2 * pr->NT[0] - 1), smooth_size(2 * pr->NT[1] - 1), smooth_size(2 * pr->NT[2] - 1)}};
        int64_t np = pg.size();
        RC(dalloc(&conv, sizeof(double2) * nT * 8 * ns));
        CK(cudaMemset(conv, 0, sizeof(double2) * nT * 8 * ns));
        pr->d_conv = conv;
        double2 *work;
        RC(dalloc(&work, sizeof(double2) * np * 13));
        double2 *E = work, *X = E + 6 * np, *tmp = X + np;
        pad_kernel<<<dim3(nblk(np, 256), 6), 256, 0, st>>>(eps, nT, E, np, pr->NT[0], pr->NT[1], pr->NT[2], pg.n[0],
                                                           pg.n[1], pg.n[2]);
        RC(dft3(E, np, 6, pg, -1, st));
        for (int s = 1; s < ns; s++) {
            pad_kernel<<<dim3(nblk(np, 256), 1), 256, 0, st>>>(chi + s * nT, 0, X, 0, pr->NT[0], pr->NT[1], pr->NT[2],
                                                               pg.n[0], pg.n[1], pg.n[2]);
            RC(dft3(X, 0, 1, pg, -1, st));
            RC(conv_batch(X, E, 6, pg, pr->NT, tmp, conv + (int64_t)s * 8 * nT, st));
            hydro_biax_kernel<<<nblk(nT, 256), 256, 0, st>>>(conv + (int64_t)s * 8 * nT, nT);
        }
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        qd_pool_free(work, 0);
    } else if (ns > 1) {
        chi_kernel<<<dim3(nblk(nT, 64), ns - 1), 64, 0, st>>>(dg, 1, ns, pr->d_G[0], pr->d_G[1], pr->d_G[2],
                                                                 pr->NT[0], pr->NT[1], pr->NT[2], 0, P.softening,
                                                                 P.sigma, chi);
        CK(cudaGetLastError());
        if (pr->chi_dir_t != 0.0 && pr->d_chi_dir)
            axpy_kernel<<<nblk(nT, 256), 256, 0, st>>>(chi + (int64_t)pr->chi_dir_shape * nT,
                                                       (const double2 *)pr->d_chi_dir, pr->chi_dir_t, nT);
    }
    // fused per-difference coefficients
    double2 *coef;
    RC(dalloc(&coef, sizeof(double2) * nT * QD_N_COEF));
    pr->d_coef = coef;
    const geo_t &g0 = pr->geo[0];
    fused_coef_kernel<<<nblk(nT, 128), 128, 0, st>>>(
        dg, dm, ns, pr->NT[0], pr->NT[1], pr->NT[2], 2.0 * M_PI / g0.L1, 2.0 * M_PI / g0.L2, 2.0 * M_PI / g0.L3,
        P.F[0], P.F[1], P.F[2], P.strain != 0, P.strain != 0 && P.piezo != 0, chi, eps, phi, conv, coef);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    pr->tables_ready = 1;
    return QD_OK;
}

// Derivative of the fused coefficient table along a direction in which the
// shape functions, the strain and the piezoelectric potential stay fixed and
// only the material parameters (dmat, one entry per shape) and the field (dF)
// move.  The table is linear in both, so the derivative is the same fused sum
// evaluated with dmat and dF in place of the parameters and field, without the
// piezoelectric potential (it depends on neither).  Exact: Ep and gamma_1
// scales and the field components use it.  dcoef: QD_N_COEF x nT, device.
extern "C" int qd_tables_tangent_dev(struct qd_problem *pr, const struct material_params *dmat, const double dF[3],
                                     void *dcoef) {
    if (!pr->tables_ready) return qd_set_error(QD_ERR_ARG, "qd_tables_tangent_dev: tables not built");
    const qd_params &P = pr->p;
    const int ns = P.n_shape;
    mat_t *dm = nullptr;
    RC(dalloc(&dm, sizeof(mat_t) * ns));
    cudaError_t e = cudaMemcpy(dm, dmat, sizeof(mat_t) * ns, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const geo_t &g0 = pr->geo[0];
        qd_count_launch(1);
        fused_coef_kernel<<<nblk(pr->nT, 128), 128>>>(
            (const geo_t *)pr->d_geo, dm, ns, pr->NT[0], pr->NT[1], pr->NT[2], 2.0 * M_PI / g0.L1,
            2.0 * M_PI / g0.L2, 2.0 * M_PI / g0.L3, dF[0], dF[1], dF[2], P.strain != 0, 0,
            (const double2 *)pr->d_chi, (const double2 *)pr->d_eps, nullptr, (const double2 *)pr->d_conv,
            (double2 *)dcoef);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    }
    qd_pool_free(dm, 0);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "tangent table: %s", cudaGetErrorString(e));
    return QD_OK;
}

// Direction arrays for a derivative along one geometry parameter of shape s:
// geo4 holds four host copies of the problem's shapes with that parameter at
// +2h, +h, -h, -2h.  Allocates *dir_s (strain cell, when strain is on) and
// *dir (electronic cell) = h dchi_s/dp to O(h^5); free with qd_pool_free.
extern "C" int qd_chi_direction(struct qd_problem *pr, int s, const struct supercell_geometry *geo4, void **dir_s,
                                void **dir) {
    if (!pr->tables_ready) return qd_set_error(QD_ERR_ARG, "qd_chi_direction: tables not built");
    const qd_params &P = pr->p;
    const int ns = P.n_shape;
    if (s < 1 || s >= ns) return qd_set_error(QD_ERR_ARG, "qd_chi_direction: shape %d", s);
    cudaStream_t st = 0;
    geo_t *dg4 = nullptr;
    double2 *ds = nullptr, *de = nullptr;
    RC(dalloc(&dg4, sizeof(geo_t) * 4 * ns));
    CK(cudaMemcpy(dg4, geo4, sizeof(geo_t) * 4 * ns, cudaMemcpyHostToDevice));
    if (P.strain) {
        RC(dalloc(&ds, sizeof(double2) * pr->nTS));
        chi_direction_kernel<<<nblk(pr->nTS, 32), dim3(32, 4), 0, st>>>(dg4, ns, s, pr->d_GS[0], pr->d_GS[1], pr->d_GS[2],
                                                                 pr->NTS[0], pr->NTS[1], pr->NTS[2], 1, P.softening,
                                                                 P.sigma, ds);
    }
    RC(dalloc(&de, sizeof(double2) * pr->nT));
    chi_direction_kernel<<<nblk(pr->nT, 32), dim3(32, 4), 0, st>>>(dg4, ns, s, pr->d_G[0], pr->d_G[1], pr->d_G[2], pr->NT[0],
                                                            pr->NT[1], pr->NT[2], 0, P.softening, P.sigma, de);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    qd_pool_free(dg4, 0);
    *dir_s = ds;
    *dir = de;
    return QD_OK;
}

// Drop-in path: the reference's host tables (global arrays) are uploaded and
// fused on the device.
extern "C" int qd_coef_from_host_tables(int n_shape, const int N[3], const double *Gx, const double *Gy,
                                        const double *Gz, double Kx, double Ky, double Kz, const double F[3],
                                        const struct supercell_geometry *geo, const struct material_params *mat,
                                        int strain_on, int piezo_on, const qd_complex128 *const *chi_h,
                                        const qd_complex128 *const *eps_h, const qd_complex128 *phi_h,
                                        const qd_complex128 *const *conv8_h, void **d_coef_out, double **d_G_out) {
    (void)Kx; (void)Ky; (void)Kz;
    int NT[3] = {2 * N[0] - 1, 2 * N[1] - 1, 2 * N[2] - 1};
    int64_t nT = (int64_t)NT[0] * NT[1] * NT[2];
    geo_t *dg;
    mat_t *dm;
    double2 *chi, *eps = NULL, *phi = NULL, *conv = NULL, *coef;
    RC(dalloc(&dg, sizeof(geo_t) * n_shape));
    RC(dalloc(&dm, sizeof(mat_t) * n_shape));
    CK(cudaMemcpy(dg, geo, sizeof(geo_t) * n_shape, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dm, mat, sizeof(mat_t) * n_shape, cudaMemcpyHostToDevice));
    RC(dalloc(&chi, sizeof(double2) * nT * n_shape));
    CK(cudaMemset(chi, 0, sizeof(double2) * nT * n_shape));
    for (int s = 1; s < n_shape; s++)
        CK(cudaMemcpy(chi + s * nT, chi_h[s], sizeof(double2) * nT, cudaMemcpyHostToDevice));
    if (strain_on) {
        RC(dalloc(&eps, sizeof(double2) * nT * 6));
        for (int c = 0; c < 6; c++) CK(cudaMemcpy(eps + c * nT, eps_h[c], sizeof(double2) * nT, cudaMemcpyHostToDevice));
        RC(dalloc(&conv, sizeof(double2) * nT * 8 * n_shape));
        CK(cudaMemset(conv, 0, sizeof(double2) * nT * 8 * n_shape));
        for (int s = 1; s < n_shape; s++)
            for (int c = 0; c < 8; c++)
                CK(cudaMemcpy(conv + ((int64_t)s * 8 + c) * nT, conv8_h[s * 8 + c], sizeof(double2) * nT,
                              cudaMemcpyHostToDevice));
        if (piezo_on) {
            RC(dalloc(&phi, sizeof(double2) * nT));
            CK(cudaMemcpy(phi, phi_h, sizeof(double2) * nT, cudaMemcpyHostToDevice));
        }
    }
    RC(dalloc(&coef, sizeof(double2) * nT * QD_N_COEF));
    // grid spacing 2 pi / L of the reference's basis arrays (only used where the
    // plane-wave index along that axis differs, i.e. N_T > 1)
    double dgx = NT[0] > 1 ? Gx[1] - Gx[0] : 1.0, dgy = NT[1] > 1 ? Gy[1] - Gy[0] : 1.0,
           dgz = NT[2] > 1 ? Gz[1] - Gz[0] : 1.0;
    fused_coef_kernel<<<nblk(nT, 128), 128>>>(dg, dm, n_shape, NT[0], NT[1], NT[2], dgx, dgy, dgz, F[0], F[1], F[2],
                                              strain_on, strain_on && piezo_on, chi, eps, phi, conv, coef);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    double *dG;
    RC(dalloc(&dG, sizeof(double) * (NT[0] + NT[1] + NT[2])));
    CK(cudaMemcpy(dG, Gx, sizeof(double) * NT[0], cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dG + NT[0], Gy, sizeof(double) * NT[1], cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dG + NT[0] + NT[1], Gz, sizeof(double) * NT[2], cudaMemcpyHostToDevice));
    qd_pool_free(dg, 0); qd_pool_free(dm, 0); qd_pool_free(chi, 0);
    if (eps) qd_pool_free(eps, 0);
    if (phi) qd_pool_free(phi, 0);
    if (conv) qd_pool_free(conv, 0);
    *d_coef_out = coef;
    *d_G_out = dG;
    return QD_OK;
}
