// Minimal double/float complex arithmetic for device code (layout: {re, im}).
#pragma once
#include <cuda_runtime.h>

struct zc {
    double re, im;
    __host__ __device__ zc() : re(0), im(0) {}
    __host__ __device__ zc(double r) : re(r), im(0) {}
    __host__ __device__ zc(double r, double i) : re(r), im(i) {}
    __host__ __device__ explicit zc(double2 v) : re(v.x), im(v.y) {}
    __host__ __device__ double2 d2() const { return make_double2(re, im); }
};
__host__ __device__ inline zc operator+(zc a, zc b) { return zc(a.re + b.re, a.im + b.im); }
__host__ __device__ inline zc operator-(zc a, zc b) { return zc(a.re - b.re, a.im - b.im); }
__host__ __device__ inline zc operator-(zc a) { return zc(-a.re, -a.im); }
__host__ __device__ inline zc operator*(zc a, zc b) {
    return zc(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__host__ __device__ inline zc operator*(double s, zc a) { return zc(s * a.re, s * a.im); }
__host__ __device__ inline zc operator*(zc a, double s) { return zc(s * a.re, s * a.im); }
__host__ __device__ inline zc operator/(zc a, double s) { return zc(a.re / s, a.im / s); }
__host__ __device__ inline zc operator/(zc a, zc b) {
    // Smith's algorithm
    if (fabs(b.re) >= fabs(b.im)) {
        double r = b.im / b.re, den = b.re + b.im * r;
        return zc((a.re + a.im * r) / den, (a.im - a.re * r) / den);
    }
    double r = b.re / b.im, den = b.im + b.re * r;
    return zc((a.re * r + a.im) / den, (a.im * r - a.re) / den);
}
__host__ __device__ inline zc operator/(double a, zc b) { return zc(a) / b; }
__host__ __device__ inline zc& operator+=(zc& a, zc b) { a.re += b.re; a.im += b.im; return a; }
__host__ __device__ inline zc& operator-=(zc& a, zc b) { a.re -= b.re; a.im -= b.im; return a; }
__host__ __device__ inline zc& operator*=(zc& a, zc b) { a = a * b; return a; }
__host__ __device__ inline zc& operator*=(zc& a, double s) { a.re *= s; a.im *= s; return a; }
__host__ __device__ inline zc conj(zc a) { return zc(a.re, -a.im); }
__host__ __device__ inline double norm2(zc a) { return a.re * a.re + a.im * a.im; }
__device__ inline zc cexpi(double t) {  // exp(i t)
    double s, c;
    sincos(t, &s, &c);
    return zc(c, s);
}
__device__ inline zc cexpz(zc z) {  // exp(z)
    double e = exp(z.re), s, c;
    sincos(z.im, &s, &c);
    return zc(e * c, e * s);
}
__host__ __device__ inline zc I_times(zc a) { return zc(-a.im, a.re); }
