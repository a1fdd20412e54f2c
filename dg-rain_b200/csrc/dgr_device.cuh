/*
 * Device arithmetic of the DG-RAIN 2D step.
 *
 * Every function here evaluates the reference's expressions in the reference's order and
 * parenthesisation, and the library is compiled with --fmad=false, so each multiply, add,
 * divide and square root is one IEEE operation exactly as in the reference's C.  The one
 * transcendental on the path, pow(H, 4/3) in the Manning term, is evaluated correctly
 * rounded by pow43() below, which agrees with glibc's pow wherever glibc's is correctly
 * rounded (all but ~0.1% of arguments).
 */
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#ifndef __CUDACC__
/* plain C++ compilers (the host test harness of the derivative cores): the library's
 * overloads in the global namespace, as CUDA provides them */
using std::isnan;
#endif

#define DGR_DEV __device__ __forceinline__
/* arithmetic shared by the kernels and by the host-compiled test harness of the
 * differentiation cores */
#define DGR_HD __host__ __device__ __forceinline__

namespace dgr {

/* sign() of 2DCode/mathfunctions.c:4-12 */
template <class T>
DGR_HD int sgn(const T &a)
{
    if (a < 0) return -1;
    if (a == 0) return 0;
    return 1;
}
/* max()/min() macros of 2DCode/mathfunctions.h:8-14 (not fmax/fmin: NaN order matters) */
template <class T>
DGR_HD T rmax(const T &a, const T &b) { return (a > b) ? a : b; }
template <class T>
DGR_HD T rmin(const T &a, const T &b) { return (a < b) ? a : b; }

/* value of a scalar (decisions are taken on values; the dual-number overload lives with
 * the dual type) */
DGR_HD double val(double x) { return x; }

/* Which operand fmax(a, b) passes on, for derivatives: b when b > a or a is NaN.  At a
 * tie the values agree and a is taken. */
DGR_HD bool fmax_takes_b(double a, double b) { return (b > a) || isnan(a); }

/* fmax as the reference build evaluates it.  glibc's x86-64 fmax(x, y) returns
 * x > y ? x : y, a NaN operand giving the other one, so a tie returns y (which decides
 * the sign of a zero result); and gcc passes a call's operands in whichever order it
 * chooses, fmax being commutative up to that sign.  The reference step as compiled
 * (gcc -O2 -ffp-contract=off, x86-64) keeps the written order at the limiter's clamp
 * (2DCode/SlopeLimiter2D.c:244-246) and swaps it in RoeFlux's entropy fix
 * (2DCode/numericalFlux2D.c:74-84).  fmax_b(a, b) is the call as written (a tie returns
 * b), fmax_a(a, b) the swapped call (a tie returns a).  CUDA's fmax is not used there: its
 * result for zeros of opposite sign is not the reference's. */
DGR_HD double fmax_b(double a, double b) { return (a > b || isnan(b)) ? a : b; }
DGR_HD double fmax_a(double a, double b) { return (b > a || isnan(a)) ? b : a; }

/* Dense 3x3 times vector, summed from +0 in column order (2DCode/mathfunctions.c:24-35). */
template <class T>
DGR_HD void matvec3(const T m[3][3], const T v[3], T out[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        T s = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j) s += m[i][j] * v[j];
        out[i] = s;
    }
}

/* biased exponent field of a double */
DGR_HD unsigned exponent_bits(double a)
{
#ifdef __CUDA_ARCH__
    return ((unsigned)__double2hiint(a) >> 20) & 0x7ffu;
#else
    uint64_t u;
    memcpy(&u, &a, 8);
    return (unsigned)(u >> 52) & 0x7ffu;
#endif
}

/*
 * a / b rounded to nearest exactly as the IEEE division, from y = 1/b (itself an IEEE
 * division, shared by every quotient with the same divisor): Markstein's correction
 * (P. Markstein, "Computation of elementary functions on the IBM RISC System/6000
 * processor", IBM J. Res. Develop. 34(1), 1990), taken twice.  q0 = a y is within two
 * ulps of a/b; q1 = q0 + (a - b q0) y is within one ulp; with the residual a - b q1 then
 * exact (a fused multiply-add), q2 = q1 + (a - b q1) y is a/b rounded to nearest.  That
 * needs every quantity clear of underflow and overflow: the caller keeps b within
 * [2^-100, 2^100], and `ok` is cleared when a is outside [2^-900, 2^900] (zero aside:
 * a zero a gives a y, the IEEE signed zero), so that the caller can redo the work with
 * plain divisions.  The library's tests compare it with the IEEE division bit for bit.
 */
DGR_HD double div_rcp(double a, double b, double y, bool &ok)
{
    const double q0 = a * y;
    const double r0 = fma(-b, q0, a);
    const double q1 = fma(r0, y, q0);
    const double r1 = fma(-b, q1, a);
    const double q2 = fma(r1, y, q1);
    const unsigned e = exponent_bits(a);
    ok = ok && ((e >= 1023u - 900u && e <= 1023u + 900u) || a == 0.0);
    return a == 0.0 ? q0 : q2;
}

/* whether b may serve as div_rcp's divisor: |b| within [2^-100, 2^100] */
DGR_HD bool rcp_divisor_ok(double b)
{
    const unsigned e = exponent_bits(b);
    return e >= 1023u - 100u && e <= 1023u + 100u;
}

/* rt0_fit below with its three divisions by dM taken through div_rcp (y = 1/dM) */
DGR_HD void rt0_fit_rcp(double R1, double R2, double R3, double M11, double M12, double M13, double M21,
                         double M22, double M23, double M31, double M32, double M33, double dM, double y, double &a,
                         double &b, double &c, bool &ok)
{
    a = div_rcp(R3 * M13 * M22 - R3 * M12 * M23 - R2 * M13 * M32 + R1 * M23 * M32 + R2 * M12 * M33 - R1 * M22 * M33,
                dM, y, ok);
    b = -div_rcp(R3 * M13 * M21 - R3 * M11 * M23 - R2 * M13 * M31 + R1 * M23 * M31 + R2 * M11 * M33 - R1 * M21 * M33,
                 dM, y, ok);
    c = div_rcp(R3 * M12 * M21 - R3 * M11 * M22 - R2 * M12 * M31 + R1 * M22 * M31 + R2 * M11 * M32 - R1 * M21 * M32,
                dM, y, ok);
}

/* Division policies of the flux arithmetic.  PlainDiv: every quotient an IEEE division.
 * RcpDiv (doubles): one reciprocal per divisor, shared by that divisor's quotients
 * (div_rcp: the same bits); ok records whether every divisor and dividend was in the
 * range where that holds, and the caller redoes the work with PlainDiv where not. */
struct PlainDiv {
    template <class B>
    struct By {
        B b;
    };
    template <class B>
    DGR_HD By<B> by(const B &b) const { return {b}; }
    template <class A, class B>
    DGR_HD auto div(const A &a, const By<B> &d) const { return a / d.b; }
};
struct RcpDiv {
    bool ok = true;
    struct By {
        double b, y;
    };
    DGR_HD By by(double b)
    {
        ok = ok && rcp_divisor_ok(b);
        return {b, 1.0 / b};
    }
    DGR_HD double div(double a, const By &d) { return div_rcp(a, d.b, d.y, ok); }
};

/* Roe flux with entropy fix, 2DCode/numericalFlux2D.c:6-108.  Returns max |lambda| of the
 * two traces.  local_g scales the pressure term only; g sets the eigen-structure. */
template <class T, class Div>
DGR_HD T roe_flux_div(Div &dv, T fh[3], T zeta_in, T zeta_ex, T qx_in, T qx_ex, T qy_in, T qy_ex, T z_edge,
                      double nx, double ny, double local_g, double g)
{
    const T h_in = zeta_in + z_edge;
    const T h_ex = zeta_ex + z_edge;
    const auto by_h_in = dv.by(h_in), by_h_ex = dv.by(h_ex);
    const T u_in = dv.div(qx_in, by_h_in), u_ex = dv.div(qx_ex, by_h_ex);
    const T v_in = dv.div(qy_in, by_h_in), v_ex = dv.div(qy_ex, by_h_ex);
    const T jump[3] = {zeta_in - zeta_ex, qx_in - qx_ex, qy_in - qy_ex};

    const T p_in = 0.5 * local_g * (h_in * h_in - z_edge * z_edge);
    const T p_ex = 0.5 * local_g * (h_ex * h_ex - z_edge * z_edge);
    const T huv_in = h_in * u_in * v_in, huv_ex = h_ex * u_ex * v_ex;
    const T fn_in[3] = {h_in * u_in * nx + h_in * v_in * ny, (h_in * u_in * u_in + p_in) * nx + huv_in * ny,
                        huv_in * nx + (h_in * v_in * v_in + p_in) * ny};
    const T fn_ex[3] = {h_ex * u_ex * nx + h_ex * v_ex * ny, (h_ex * u_ex * u_ex + p_ex) * nx + huv_ex * ny,
                        huv_ex * nx + (h_ex * v_ex * v_ex + p_ex) * ny};

    const T s_in = sqrt(h_in), s_ex = sqrt(h_ex);
    const T h_hat = 0.5 * (h_in + h_ex);
    const auto by_s = dv.by(s_in + s_ex);
    const T u_hat = dv.div(u_in * s_in + u_ex * s_ex, by_s);
    const T v_hat = dv.div(v_in * s_in + v_ex * s_ex, by_s);
    const T c = sqrt(g * h_hat);

    const T r[3][3] = {{1, 0, 1}, {u_hat - c * nx, -ny, u_hat + c * nx}, {v_hat - c * ny, nx, v_hat + c * ny}};
    const T den = -2 * c;
    const auto by_den = dv.by(den);
    /* (-nx)/den is exactly -(nx/den): IEEE division is symmetric in sign, so the third
     * row reuses the first row's quotients. */
    const T nx_den = dv.div(nx, by_den), ny_den = dv.div(ny, by_den);
    const T ri[3][3] = {{dv.div(-c - nx * u_hat - ny * v_hat, by_den), nx_den, ny_den},
                        {dv.div(-2 * c * ny * u_hat + 2 * c * nx * v_hat, by_den), dv.div(2 * c * ny, by_den),
                         dv.div(-2 * c * nx, by_den)},
                        {dv.div(-c + nx * u_hat + ny * v_hat, by_den), -nx_den, -ny_den}};

    const T un_in = u_in * nx + v_in * ny, un_ex = u_ex * nx + v_ex * ny;
    const T c_in = sqrt(g * h_in), c_ex = sqrt(g * h_ex);
    const T l1_in = un_in - c_in, l2_in = un_in, l3_in = un_in + c_in;
    const T l1_ex = un_ex - c_ex, l2_ex = un_ex, l3_ex = un_ex + c_ex;
    const T un_hat = u_hat * nx + v_hat * ny;
    T lh1 = un_hat - c, lh2 = un_hat, lh3 = un_hat + c;

    T e1 = fmax_a(0.0, (lh1 - l1_in));
    e1 = fmax_a(e1, (l1_ex - lh1));
    lh1 = fmax_a(e1, fabs(lh1));
    T e2 = fmax_a(0.0, (lh2 - l2_in));
    e2 = fmax_a(e2, (l2_ex - lh2));
    lh2 = fmax_a(e2, fabs(lh2));
    T e3 = fmax_a(0.0, (lh3 - l3_in));
    e3 = fmax_a(e3, (l3_ex - lh3));
    lh3 = fmax_a(e3, fabs(lh3));

    const T lam[3][3] = {{lh1, 0, 0}, {0, lh2, 0}, {0, 0, lh3}};
    T p1[3], p2[3], p3[3];
    matvec3(ri, jump, p1);
    matvec3(lam, p1, p2);
    matvec3(r, p2, p3);
#pragma unroll
    for (int k = 0; k < 3; ++k) fh[k] = 0.5 * (fn_in[k] + fn_ex[k]) + 0.5 * p3[k];

    T m = rmax(fabs(l1_in), fabs(l1_ex));
    m = rmax(m, fabs(l2_in));
    m = rmax(m, fabs(l2_ex));
    m = rmax(m, fabs(l3_in));
    m = rmax(m, fabs(l3_ex));
    return m;
}

template <class T>
DGR_HD T roe_flux(T fh[3], T zeta_in, T zeta_ex, T qx_in, T qx_ex, T qy_in, T qy_ex, T z_edge, double nx,
                  double ny, double local_g, double g)
{
    PlainDiv dv;
    return roe_flux_div<T>(dv, fh, zeta_in, zeta_ex, qx_in, qx_ex, qy_in, qy_ex, z_edge, nx, ny, local_g, g);
}

/* Local Lax-Friedrichs flux (DG-SWEM src/numerical_flux.F:887-1141, LLF_FLUX, in its
 * nonlinear Cartesian form): the mean of the two traces' normal fluxes (the normal-flux
 * expressions of roe_flux) minus half the largest wave speed of either trace, |u.n| + c
 * over both, times the jump ex - in.  Returns that speed, the max |lambda| of roe_flux, in
 * the same order.  local_g scales the pressure term only; g sets the wave speeds.  An
 * extension: 2DCode has the Roe flux only (dgr_params.flux = 1 selects this one). */
template <class T>
DGR_HD T llf_flux(T fh[3], T zeta_in, T zeta_ex, T qx_in, T qx_ex, T qy_in, T qy_ex, T z_edge, double nx,
                  double ny, double local_g, double g)
{
    const T h_in = zeta_in + z_edge;
    const T h_ex = zeta_ex + z_edge;
    const T u_in = qx_in / h_in, u_ex = qx_ex / h_ex;
    const T v_in = qy_in / h_in, v_ex = qy_ex / h_ex;
    const T p_in = 0.5 * local_g * (h_in * h_in - z_edge * z_edge);
    const T p_ex = 0.5 * local_g * (h_ex * h_ex - z_edge * z_edge);
    const T huv_in = h_in * u_in * v_in, huv_ex = h_ex * u_ex * v_ex;
    const T fn_in[3] = {h_in * u_in * nx + h_in * v_in * ny, (h_in * u_in * u_in + p_in) * nx + huv_in * ny,
                        huv_in * nx + (h_in * v_in * v_in + p_in) * ny};
    const T fn_ex[3] = {h_ex * u_ex * nx + h_ex * v_ex * ny, (h_ex * u_ex * u_ex + p_ex) * nx + huv_ex * ny,
                        huv_ex * nx + (h_ex * v_ex * v_ex + p_ex) * ny};
    const T un_in = u_in * nx + v_in * ny, un_ex = u_ex * nx + v_ex * ny;
    const T c_in = sqrt(g * h_in), c_ex = sqrt(g * h_ex);
    T m = rmax(fabs(un_in - c_in), fabs(un_ex - c_ex));
    m = rmax(m, fabs(un_in));
    m = rmax(m, fabs(un_ex));
    m = rmax(m, fabs(un_in + c_in));
    m = rmax(m, fabs(un_ex + c_ex));
    const T jump[3] = {zeta_ex - zeta_in, qx_ex - qx_in, qy_ex - qy_in};
#pragma unroll
    for (int k = 0; k < 3; ++k) fh[k] = 0.5 * (fn_in[k] + fn_ex[k]) - 0.5 * m * jump[k];
    return m;
}

/* HLLC flux (DG-SWEM src/numerical_flux.F:1154-1400, HLLC_FLUX, nonlinear Cartesian
 * form): wave speeds S_in = un_in - c_in l_in, S_ex = un_ex + c_ex l_ex with the
 * shock/rarefaction factors l = sqrt((h* h* + h* h) / (2 h h)) when h* > h (else 1),
 * h* = (0.5 (c_in + c_ex) + 0.25 (un_in - un_ex))^2 / g, the contact speed S*, and the
 * four branches: the in trace's normal flux for S_in >= 0, the in star state for
 * S_in <= 0 <= S*, the ex star state for S* <= 0 <= S_ex, the ex trace's flux otherwise;
 * star-state corrections S (Q* - Q) in normal/tangential components rotated back.  The
 * normal fluxes are roe_flux's expressions (local_g in the pressure); returns max |lambda|
 * of the two traces as roe_flux does (for the CFL dt).  An extension (flux = 2). */
template <class T>
DGR_HD T hllc_flux(T fh[3], T zeta_in, T zeta_ex, T qx_in, T qx_ex, T qy_in, T qy_ex, T z_edge, double nx,
                   double ny, double local_g, double g)
{
    const T h_in = zeta_in + z_edge;
    const T h_ex = zeta_ex + z_edge;
    const T u_in = qx_in / h_in, u_ex = qx_ex / h_ex;
    const T v_in = qy_in / h_in, v_ex = qy_ex / h_ex;
    const T un_in = u_in * nx + v_in * ny, un_ex = u_ex * nx + v_ex * ny;
    const T ut_in = -u_in * ny + v_in * nx, ut_ex = -u_ex * ny + v_ex * nx;
    const T c_in = sqrt(g * h_in), c_ex = sqrt(g * h_ex);
    const T P = 0.5 * (c_in + c_ex) + 0.25 * (un_in - un_ex);
    const T hs = 1.0 / g * P * P;
    T l_in = 1.0, l_ex = 1.0;
    if (hs > h_ex) l_ex = sqrt((hs * hs + hs * h_ex) / (2.0 * h_ex * h_ex));
    if (hs > h_in) l_in = sqrt((hs * hs + hs * h_in) / (2.0 * h_in * h_in));
    const T s_in = un_in - c_in * l_in;
    const T s_ex = un_ex + c_ex * l_ex;
    const T A = un_ex - s_ex, B = un_in - s_in;
    const T s_st = (s_in * h_ex * A - s_ex * h_in * B) / (h_ex * A - h_in * B);
    /* DG-SWEM's branch order: S_in >= 0; S* >= 0; S_ex >= 0; otherwise */
    const int branch = s_in >= 0.0 ? 0 : (s_st >= 0.0 ? 1 : (s_ex >= 0.0 ? 2 : 3));
    const bool use_in = branch <= 1;
    const T h = use_in ? h_in : h_ex, u = use_in ? u_in : u_ex, v = use_in ? v_in : v_ex;
    const T p = 0.5 * local_g * (h * h - z_edge * z_edge);
    const T huv = h * u * v;
    fh[0] = h * u * nx + h * v * ny;
    fh[1] = (h * u * u + p) * nx + huv * ny;
    fh[2] = huv * nx + (h * v * v + p) * ny;
    if (branch == 1 || branch == 2) { /* a star state */
        const T S = use_in ? s_in : s_ex, un = use_in ? un_in : un_ex, ut = use_in ? ut_in : ut_ex;
        const T qx = use_in ? qx_in : qx_ex, qy = use_in ? qy_in : qy_ex;
        const T q1 = h * ((S - un) / (S - s_st));
        const T d1 = q1 - h;
        const T d2 = q1 * s_st - (qx * nx + qy * ny);
        const T d3 = q1 * ut - (-qx * ny + qy * nx);
        fh[0] = fh[0] + S * d1;
        fh[1] = fh[1] + S * (d2 * nx - d3 * ny);
        fh[2] = fh[2] + S * (d2 * ny + d3 * nx);
    }
    T m = rmax(fabs(un_in - c_in), fabs(un_ex - c_ex));
    m = rmax(m, fabs(un_in));
    m = rmax(m, fabs(un_ex));
    m = rmax(m, fabs(un_in + c_in));
    m = rmax(m, fabs(un_ex + c_ex));
    return m;
}

/* numerical flux of kind `type` (0: Roe, 2DCode; 1: local Lax-Friedrichs, 2: HLLC, DG-SWEM) */
template <class T, class Div = PlainDiv>
DGR_HD T numerical_flux(int type, T fh[3], T zeta_in, T zeta_ex, T qx_in, T qx_ex, T qy_in, T qy_ex, T z_edge,
                        double nx, double ny, double local_g, double g, Div *dv = nullptr)
{
    if (type == 1) return llf_flux<T>(fh, zeta_in, zeta_ex, qx_in, qx_ex, qy_in, qy_ex, z_edge, nx, ny, local_g, g);
    if (type == 2) return hllc_flux<T>(fh, zeta_in, zeta_ex, qx_in, qx_ex, qy_in, qy_ex, z_edge, nx, ny, local_g, g);
    if (dv) return roe_flux_div<T>(*dv, fh, zeta_in, zeta_ex, qx_in, qx_ex, qy_in, qy_ex, z_edge, nx, ny, local_g, g);
    return roe_flux<T>(fh, zeta_in, zeta_ex, qx_in, qx_ex, qy_in, qy_ex, z_edge, nx, ny, local_g, g);
}

/*
 * x^p for p = 4./3 (the double nearest 4/3, used by the Manning term
 * pow(H[e], 4./3) of 2DCode/2DInnerProducts.c:318), correctly rounded.
 *
 * Method.  p = 4/3 - 1/(3*2^52) exactly, so x^p = x * cbrt(x) * exp(eta) with
 * eta = -ln(x)/(3*2^52), |eta| < 1e-15 for the depths that occur.
 *   1. c0 = cbrt(x) (CUDA, <= 1 ulp), refined by one Newton step c = c0 - (c0^3 - x)/(3 c0^2)
 *      whose residual is formed without rounding loss by FMA-based exact products
 *      (Dekker's product; Sterbenz makes c0^3 - x exact): c is within ~2^-100 of cbrt(x).
 *   2. x*c0 split exactly into hi + lo by FMA; exp(eta) = 1 + eta to 1e-30, where the
 *      double log(x) gives eta far more accurately than needed.
 *   3. y = hi + ((lo - x*d) + hi*eta) is within a few 2^-100 relative of x^p, so its final
 *      rounding is the correctly rounded result unless x^p lies within that distance of a
 *      rounding midpoint.
 * glibc's pow is correctly rounded for all but ~0.1% of arguments, CUDA's pow for far
 * fewer; this keeps the device friction term on the reference's bits.
 * Zero, negative, non-finite and extreme arguments go to pow(), whose special-case
 * results are the C standard's on both sides.
 */
DGR_HD double fma_exact(double a, double b, double c)
{
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

DGR_HD double pow43_exact(double x)
{
    if (!(x >= 1e-200 && x <= 1e200)) return pow(x, 4. / 3);
    const double c0 = cbrt(x);
    const double a_h = c0 * c0;
    const double a_l = fma_exact(c0, c0, -a_h);
    const double b_h = a_h * c0;
    const double b_l = fma_exact(a_h, c0, -b_h);
    const double r = ((b_h - x) + b_l) + a_l * c0; /* c0^3 - x */
    const double d = r / (3.0 * a_h);
    const double p_h = x * c0;
    const double p_l = fma_exact(x, c0, -p_h);
    const double eta = log(x) * -7.401486830834377e-17;
    const double lo = (p_l - x * d) + p_h * eta;
    return p_h + lo;
}

/*
 * pow43 on the device: the same correctly rounded value in two phases (Ziv's strategy).
 *   Fast phase, for 2^-120 <= x < 2^120 (every float conversion below stays normal):
 *     1. r0 = rcbrtf(x) (float, 1 ulp), one Newton step in double for x^(-1/3):
 *        r1 = r0 + r0 (1 - x r0^3)/3, relative error 2 e0^2 ~ 2^-44;
 *     2. c0 = x r1^2 ~ cbrt(x) to 2^-43, corrected by c = c0 - (c0^3 - x)/(3 c0^2) with the
 *        residual formed exactly as in pow43_exact and 1/(3 c0^2) taken as r1^2/3: the
 *        error left is ~2^-84 relative;
 *     3. eta = -ln(x)/(3*2^52) from the exponent and a float log2 of the mantissa
 *        (absolute error of log2 below 2^-21.5 on [1, 2)): eta is off by < 2^-75 relative.
 *   The result y = RN(x c e^eta) is then within 2^-74 of x^p, so when both ends of the
 *   interval +-2^-70 |y| round to the same double, that double is the correctly rounded
 *   x^p.  Otherwise (x^p within 2^-70 of a rounding midpoint, about 1 argument in 10^5)
 *   pow43_exact, whose error is a few 2^-100, decides.  The host keeps pow43_exact.
 */
#ifdef __CUDA_ARCH__
/* the rare slow phase stays out of line: one copy per kernel instead of one per call site */
__device__ __noinline__ double pow43_slow(double x) { return pow43_exact(x); }

DGR_DEV double pow43_fast_or_exact(double x)
{
    if (!(x >= 0x1p-120 && x < 0x1p120)) return pow43_slow(x);
    const double r0 = (double)rcbrtf(__double2float_rn(x));
    const double q = r0 * r0; /* exact: 24-bit significands */
    const double t = __fma_rn(-x, q * r0, 1.0);
    const double r1 = __fma_rn(r0 * t, 0x1.5555555555555p-2, r0);
    const double c0 = (x * r1) * r1;
    const double a_h = c0 * c0;
    const double a_l = __fma_rn(c0, c0, -a_h);
    const double b_h = a_h * c0;
    const double b_l = __fma_rn(a_h, c0, -b_h);
    const double res = ((b_h - x) + b_l) + a_l * c0; /* c0^3 - x */
    const double d = res * ((r1 * r1) * 0x1.5555555555555p-2);
    const double p_h = x * c0;
    const double p_l = __fma_rn(x, c0, -p_h);
    /* x = 2^e m, m in [1, 2) */
    const int hi = __double2hiint(x);
    const int e = ((hi >> 20) & 0x7ff) - 1023;
    const double m = __hiloint2double((hi & 0x000fffff) | 0x3ff00000, __double2loint(x));
    const double lg2 = (double)e + (double)__log2f(__double2float_rn(m));
    const double eta = lg2 * -0x1.d9303fea2f7eap-55; /* -ln(2)/(3*2^52) */
    const double lo = (p_l - x * d) + p_h * eta;
    const double err = p_h * 0x1p-70;
    const double y_lo = p_h + (lo - err);
    const double y_hi = p_h + (lo + err);
    if (y_lo == y_hi) return y_lo;
    return pow43_slow(x);
}
#endif

DGR_HD double pow43(double x)
{
#ifdef __CUDA_ARCH__
    return pow43_fast_or_exact(x);
#else
    return pow43_exact(x);
#endif
}

/* x / d for the limiter's redistribution count d in {1, 2, 3} (as a double).  Division
 * by 1 and by 2 are exact (x and x*0.5 are the correctly rounded x/d); only d = 3 needs
 * the full IEEE division. */
template <class T>
DGR_HD T div_by_count(const T &x, double d)
{
    if (d == 1.0) return x;
    if (d == 2.0) return x * 0.5;
    return x / d;
}

/* RT0 fit F = (a + b x, c + b y) through three normal-flux values (Cramer's rule of
 * 2DCode/2DInnerProducts.c:134-146 and :507-519). */
template <class T>
DGR_HD void rt0_fit(const T &R1, const T &R2, const T &R3, double M11, double M12, double M13, double M21,
                    double M22, double M23, double M31, double M32, double M33, double dM, T &a, T &b, T &c)
{
    a = (R3 * M13 * M22 - R3 * M12 * M23 - R2 * M13 * M32 + R1 * M23 * M32 + R2 * M12 * M33 - R1 * M22 * M33) / dM;
    b = -(R3 * M13 * M21 - R3 * M11 * M23 - R2 * M13 * M31 + R1 * M23 * M31 + R2 * M11 * M33 - R1 * M21 * M33) / dM;
    c = (R3 * M12 * M21 - R3 * M11 * M22 - R2 * M12 * M31 + R1 * M22 * M31 + R2 * M11 * M32 - R1 * M21 * M32) / dM;
}

/* Status key: earlier step, then earlier phase, then lower index wins under atomicMin,
 * which is the failure the sequential reference would have stopped at. */
DGR_HD unsigned long long err_key(int step, int phase, int code, int index)
{
    return ((unsigned long long)(unsigned)step << 40) | ((unsigned long long)(phase & 15) << 36) |
           ((unsigned long long)(code & 15) << 32) | (unsigned long long)(unsigned)index;
}

}  // namespace dgr
