/*
 * Boundary forcing shared by the host C code and the CUDA kernels.
 *
 * The reference fills two per-edge arrays before every step
 * (2DCode/boundary_conditions.c:9-82, called at 2DCode/time_evolution.c:252 and :319):
 *
 *   type 1 (first inflow list)  zeta_b = -1000,  qn = -0.042/0.914   (:134-135)
 *   type 2 (outflow list)       zeta_b = 0.296,  qn = 1e6            (:168-169)
 *   type 3 (second inflow list) zeta_b = -10000, qn = -0.1275/0.914  (:182-183)
 *   type 0 (land)               zeta_b and qn unused: reflective wall (2DCode/compute2DL.c:175-190)
 *
 * zeta_b < 0 and qn > 1000 are sentinels that the edge flux replaces by the interior
 * value (2DCode/compute2DL.c:151-156).
 *
 * The tide is an extension: the reference has no time-dependent forcing.  When it is on,
 * the type-2 elevation becomes A*sin(2*pi*t/T), evaluated at the same point of the time
 * loop where the reference calls boundary_conditions().  The sentinel rule still applies,
 * so a negative tide value means "use the interior elevation", exactly as the reference
 * edge flux would treat it.
 *
 * dgr_sin_turns() is written out as plain IEEE multiplies and adds so that the host
 * (gcc, -ffp-contract=off) and the device (nvcc --fmad=false) produce the same bits.
 * Method: reduce p to its fractional part, fold it into the first quarter wave by the
 * symmetries sin(pi+x) = -sin(x) and sin(pi-x) = sin(x), then sum the Taylor series of
 * sin to the theta^23 term (truncation error < 1e-20 on [0, pi/2]) by Horner's rule.
 */
#ifndef DGR_FORCING_H
#define DGR_FORCING_H

#include <math.h>

#if defined(__CUDACC__)
#define DGR_HD __host__ __device__ __forceinline__
#else
#define DGR_HD static inline
#endif

/* Reference constants of 2DCode/boundary_conditions.c, in type order 1, 2, 3. */
#define DGR_BC1_ZETA (-1000.0)
#define DGR_BC1_QN (-0.042 / 0.914)
#define DGR_BC2_ZETA (0.296)
#define DGR_BC2_QN (1000000.0)
#define DGR_BC3_ZETA (-10000.0)
#define DGR_BC3_QN (-0.1275 / 0.914)

/* sin(2*pi*p) for p >= 0. */
DGR_HD double dgr_sin_turns(double p)
{
    double f = p - floor(p);
    double sgn = 1.0;
    if (f >= 0.5) {
        f = f - 0.5;
        sgn = -1.0;
    }
    if (f > 0.25) f = 0.5 - f;
    const double th = f * 6.283185307179586;
    const double t2 = th * th;
    double s = -3.868170170630684e-23;
    s = s * t2 + 1.9572941063391263e-20;
    s = s * t2 + -8.22063524662433e-18;
    s = s * t2 + 2.8114572543455206e-15;
    s = s * t2 + -7.647163731819816e-13;
    s = s * t2 + 1.6059043836821613e-10;
    s = s * t2 + -2.505210838544172e-08;
    s = s * t2 + 2.7557319223985893e-06;
    s = s * t2 + -0.0001984126984126984;
    s = s * t2 + 0.008333333333333333;
    s = s * t2 + -0.16666666666666666;
    s = s * t2;
    return sgn * (th + th * s);
}

/* Type-2 boundary elevation at time t: the tide when tide_on is set, else the reference
 * constant 0.296. */
DGR_HD double dgr_outflow_zeta(double t, int tide_on, double amp, double period)
{
    if (!tide_on) return DGR_BC2_ZETA;
    return amp * dgr_sin_turns(t / period);
}

#endif
