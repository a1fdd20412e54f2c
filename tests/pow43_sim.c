/*
 * Test harness (host only): the device's two-phase x^(4./3) (pow43_fast_or_exact in
 * dg-rain_b200/csrc/dgr_device.cuh) restated with host stand-ins for the device
 * intrinsics, so that its error analysis can be stressed on the CPU: the float seed
 * x^(-1/3) and the float log2 of the mantissa are pushed to the ends of their documented
 * error bounds (rcbrtf 1 ulp, __log2f 2^-21.5 absolute on [1, 2)).  Every fast value kept
 * by the rounding test must equal the exact path's; the count of arguments that fall
 * back is reported.
 *
 *   usage: pow43_sim N   -> "perturbation k: N values, D differ, F fall back" x 3, exit 1 if D > 0
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* the exact phase, as dgr_device.cuh evaluates it (pow43_exact) */
static double pow43_exact(double x)
{
    if (!(x >= 1e-200 && x <= 1e200)) return pow(x, 4. / 3);
    const double c0 = cbrt(x);
    const double a_h = c0 * c0;
    const double a_l = fma(c0, c0, -a_h);
    const double b_h = a_h * c0;
    const double b_l = fma(a_h, c0, -b_h);
    const double r = ((b_h - x) + b_l) + a_l * c0;
    const double d = r / (3.0 * a_h);
    const double p_h = x * c0;
    const double p_l = fma(x, c0, -p_h);
    const double eta = log(x) * -7.401486830834377e-17;
    const double lo = (p_l - x * d) + p_h * eta;
    return p_h + lo;
}

static long n_fallback;

/* the fast phase; seed_rel and log_abs move the two float intrinsics within their bounds */
static double pow43_fast(double x, float seed_rel, float log_abs)
{
    if (!(x >= 0x1p-120 && x < 0x1p120)) return pow43_exact(x);
    float rf = 1.0f / cbrtf((float)x);
    rf *= 1.0f + seed_rel;
    const double r0 = (double)rf;
    const double q = r0 * r0;
    const double t = fma(-x, q * r0, 1.0);
    const double r1 = fma(r0 * t, 0x1.5555555555555p-2, r0);
    const double c0 = (x * r1) * r1;
    const double a_h = c0 * c0;
    const double a_l = fma(c0, c0, -a_h);
    const double b_h = a_h * c0;
    const double b_l = fma(a_h, c0, -b_h);
    const double res = ((b_h - x) + b_l) + a_l * c0;
    const double d = res * ((r1 * r1) * 0x1.5555555555555p-2);
    const double p_h = x * c0;
    const double p_l = fma(x, c0, -p_h);
    uint64_t u;
    memcpy(&u, &x, 8);
    const int e = (int)((u >> 52) & 0x7ff) - 1023;
    const uint64_t mu = (u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double m;
    memcpy(&m, &mu, 8);
    const double lg2 = (double)e + (double)(log2f((float)m) + log_abs);
    const double eta = lg2 * -0x1.d9303fea2f7eap-55;
    const double lo = (p_l - x * d) + p_h * eta;
    const double err = p_h * 0x1p-70;
    const double y_lo = p_h + (lo - err);
    const double y_hi = p_h + (lo + err);
    if (y_lo == y_hi) return y_lo;
    ++n_fallback;
    return pow43_exact(x);
}

int main(int argc, char **argv)
{
    const long n = argc > 1 ? atol(argv[1]) : 1000000;
    const float seed[3] = {0.0f, 0x1p-22f, -0x1p-22f};
    const float lg[3] = {0.0f, 3.3719e-7f, -3.3719e-7f}; /* 2^-21.5 */
    long bad = 0;
    for (int k = 0; k < 3; ++k) {
        srand48(7 + k);
        long diff = 0;
        n_fallback = 0;
        for (long i = 0; i < n; ++i) {
            double x;
            switch (i % 4) {
            case 0: x = exp(log(1e-6) + drand48() * (log(1e3) - log(1e-6))); break; /* depths */
            case 1: x = 1e-3 + (drand48() - 0.5) * 4e-5; break;                     /* near H0 */
            case 2: x = exp((drand48() - 0.5) * 164.0); break;                      /* the fast domain */
            default: x = 0.5 + drand48() * 20.0;
            }
            if (pow43_fast(x, seed[k], lg[k]) != pow43_exact(x)) ++diff;
        }
        printf("perturbation %d: %ld values, %ld differ, %ld fall back\n", k, n, diff, n_fallback);
        bad += diff;
    }
    return bad ? 1 : 0;
}
