/*
 * Forward-mode dual numbers for the tangent-linear model (TLM) of the 2D step.
 *
 * A Dual carries a value v and one directional derivative d.  The value part of every
 * operation is the same single IEEE operation the double code performs (so a TLM run
 * reproduces the forward trajectory bit for bit), and every branch of the scheme is taken
 * on values: the derivative is that of the discrete scheme with its decisions (wet/dry
 * flags, limiter clamps, entropy-fix selections, PDop branches) frozen at the primal's.
 *
 * Conventions at the kinks, shared with the hand-written reverse in dgr_reverse.cuh:
 *   fmax(a, b)  takes b when b > a (or a is NaN), else a
 *   fabs(a)     derivative -d for a < 0, +d otherwise
 *   sqrt(a)     derivative 0 at a == 0 (the only zero argument on the path is the speed
 *               |u| of the Manning term, whose product with the discharge has derivative 0)
 *
 * The type lives in its own namespace so that unqualified calls on plain doubles inside
 * namespace dgr never see these overloads; calls on Duals find them by argument lookup.
 */
#pragma once

#include <cmath>

#include "dgr_device.cuh"

namespace dgr {
namespace ad {

struct Dual {
    double v, d;
    DGR_HD Dual() : v(0.0), d(0.0) {}
    DGR_HD Dual(double x) : v(x), d(0.0) {}
    DGR_HD Dual(double x, double dx) : v(x), d(dx) {}
};

DGR_HD Dual operator-(const Dual &a) { return Dual(-a.v, -a.d); }
DGR_HD Dual operator+(const Dual &a, const Dual &b) { return Dual(a.v + b.v, a.d + b.d); }
DGR_HD Dual operator+(const Dual &a, double b) { return Dual(a.v + b, a.d); }
DGR_HD Dual operator+(double a, const Dual &b) { return Dual(a + b.v, b.d); }
DGR_HD Dual operator-(const Dual &a, const Dual &b) { return Dual(a.v - b.v, a.d - b.d); }
DGR_HD Dual operator-(const Dual &a, double b) { return Dual(a.v - b, a.d); }
DGR_HD Dual operator-(double a, const Dual &b) { return Dual(a - b.v, -b.d); }
DGR_HD Dual operator*(const Dual &a, const Dual &b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
DGR_HD Dual operator*(const Dual &a, double b) { return Dual(a.v * b, a.d * b); }
DGR_HD Dual operator*(double a, const Dual &b) { return Dual(a * b.v, a * b.d); }
DGR_HD Dual operator/(const Dual &a, const Dual &b)
{
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
DGR_HD Dual operator/(const Dual &a, double b) { return Dual(a.v / b, a.d / b); }
DGR_HD Dual operator/(double a, const Dual &b)
{
    const double q = a / b.v;
    return Dual(q, -q * b.d / b.v);
}
DGR_HD Dual &operator+=(Dual &a, const Dual &b) { return a = a + b; }
DGR_HD Dual &operator-=(Dual &a, const Dual &b) { return a = a - b; }

DGR_HD bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
DGR_HD bool operator<(const Dual &a, double b) { return a.v < b; }
DGR_HD bool operator<(double a, const Dual &b) { return a < b.v; }
DGR_HD bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
DGR_HD bool operator>(const Dual &a, double b) { return a.v > b; }
DGR_HD bool operator>(double a, const Dual &b) { return a > b.v; }
DGR_HD bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
DGR_HD bool operator<=(const Dual &a, double b) { return a.v <= b; }
DGR_HD bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }
DGR_HD bool operator>=(const Dual &a, double b) { return a.v >= b; }
DGR_HD bool operator==(const Dual &a, double b) { return a.v == b; }

DGR_HD bool isnan(const Dual &a) { return ::isnan(a.v); }

DGR_HD Dual sqrt(const Dual &a)
{
    const double s = ::sqrt(a.v);
    return Dual(s, a.v == 0.0 ? 0.0 : a.d / (2.0 * s));
}

DGR_HD Dual fabs(const Dual &a) { return a.v < 0 ? -a : a; }

DGR_HD Dual fmax(const Dual &a, const Dual &b)
{
    const double v = ::fmax(a.v, b.v);
    const bool take_b = (b.v > a.v) || ::isnan(a.v);
    return Dual(v, take_b ? b.d : a.d);
}
DGR_HD Dual fmax(double a, const Dual &b) { return fmax(Dual(a), b); }
DGR_HD Dual fmax(const Dual &a, double b) { return fmax(a, Dual(b)); }

/* x^(4/3) with the correctly rounded value of the double path; d/dx = (4/3) x^(1/3) */
DGR_HD Dual pow43(const Dual &a)
{
    const double p = dgr::pow43(a.v);
    return Dual(p, a.d * (4.0 / 3.0) * (p / a.v));
}

}  // namespace ad

/* value of a scalar of either kind (decisions are taken on values) */
DGR_HD double val(double x) { return x; }
DGR_HD double val(const ad::Dual &x) { return x.v; }

}  // namespace dgr
