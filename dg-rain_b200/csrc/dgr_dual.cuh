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
 *   fmax(a, b)  takes b when b > a (or a is NaN), else a; so do fmax_a and fmax_b (the
 *               reference build's two operand orders), whose values differ from fmax's
 *               only in the sign of a zero
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
/* the reference build's two orders of fmax (dgr_device.cuh): values as the double
 * functions, derivatives by the same convention as fmax */
DGR_HD Dual fmax_a(const Dual &a, const Dual &b) { return ((b.v > a.v) || ::isnan(a.v)) ? b : a; }
DGR_HD Dual fmax_a(double a, const Dual &b) { return fmax_a(Dual(a), b); }
DGR_HD Dual fmax_a(const Dual &a, double b) { return fmax_a(a, Dual(b)); }
DGR_HD Dual fmax_b(const Dual &a, const Dual &b)
{
    return Dual(dgr::fmax_b(a.v, b.v), ((b.v > a.v) || ::isnan(a.v)) ? b.d : a.d);
}
DGR_HD Dual fmax_b(double a, const Dual &b) { return fmax_b(Dual(a), b); }
DGR_HD Dual fmax_b(const Dual &a, double b) { return fmax_b(a, Dual(b)); }

/* x^(4/3) with the correctly rounded value of the double path; d/dx = (4/3) x^(1/3) */
DGR_HD Dual pow43(const Dual &a)
{
    const double p = dgr::pow43(a.v);
    return Dual(p, a.d * (4.0 / 3.0) * (p / a.v));
}

/* value part (the double overload is in dgr_device.cuh) */
DGR_HD double val(const Dual &x) { return x.v; }

/*
 * A base value v and a perturbed value p evaluated side by side, every decision taken on
 * v: running the scheme in Pert arithmetic from (u, u + h du) gives the scheme at the
 * perturbed point with the base run's decisions frozen (finite differences "with frozen
 * masks").  Each operation applies the double operation to both lanes; fabs and fmax
 * choose by the base lane (the same kink conventions as Dual).
 */
struct Pert {
    double v, p;
    DGR_HD Pert() : v(0.0), p(0.0) {}
    DGR_HD Pert(double x) : v(x), p(x) {}
    DGR_HD Pert(double x, double xp) : v(x), p(xp) {}
};

DGR_HD Pert operator-(const Pert &a) { return Pert(-a.v, -a.p); }
DGR_HD Pert operator+(const Pert &a, const Pert &b) { return Pert(a.v + b.v, a.p + b.p); }
DGR_HD Pert operator+(const Pert &a, double b) { return Pert(a.v + b, a.p + b); }
DGR_HD Pert operator+(double a, const Pert &b) { return Pert(a + b.v, a + b.p); }
DGR_HD Pert operator-(const Pert &a, const Pert &b) { return Pert(a.v - b.v, a.p - b.p); }
DGR_HD Pert operator-(const Pert &a, double b) { return Pert(a.v - b, a.p - b); }
DGR_HD Pert operator-(double a, const Pert &b) { return Pert(a - b.v, a - b.p); }
DGR_HD Pert operator*(const Pert &a, const Pert &b) { return Pert(a.v * b.v, a.p * b.p); }
DGR_HD Pert operator*(const Pert &a, double b) { return Pert(a.v * b, a.p * b); }
DGR_HD Pert operator*(double a, const Pert &b) { return Pert(a * b.v, a * b.p); }
DGR_HD Pert operator/(const Pert &a, const Pert &b) { return Pert(a.v / b.v, a.p / b.p); }
DGR_HD Pert operator/(const Pert &a, double b) { return Pert(a.v / b, a.p / b); }
DGR_HD Pert operator/(double a, const Pert &b) { return Pert(a / b.v, a / b.p); }
DGR_HD Pert &operator+=(Pert &a, const Pert &b) { return a = a + b; }
DGR_HD Pert &operator-=(Pert &a, const Pert &b) { return a = a - b; }

DGR_HD bool operator<(const Pert &a, const Pert &b) { return a.v < b.v; }
DGR_HD bool operator<(const Pert &a, double b) { return a.v < b; }
DGR_HD bool operator<(double a, const Pert &b) { return a < b.v; }
DGR_HD bool operator>(const Pert &a, const Pert &b) { return a.v > b.v; }
DGR_HD bool operator>(const Pert &a, double b) { return a.v > b; }
DGR_HD bool operator>(double a, const Pert &b) { return a > b.v; }
DGR_HD bool operator<=(const Pert &a, const Pert &b) { return a.v <= b.v; }
DGR_HD bool operator<=(const Pert &a, double b) { return a.v <= b; }
DGR_HD bool operator>=(const Pert &a, const Pert &b) { return a.v >= b.v; }
DGR_HD bool operator>=(const Pert &a, double b) { return a.v >= b; }
DGR_HD bool operator==(const Pert &a, double b) { return a.v == b; }

DGR_HD bool isnan(const Pert &a) { return ::isnan(a.v); }
DGR_HD Pert sqrt(const Pert &a) { return Pert(::sqrt(a.v), ::sqrt(a.p)); }
DGR_HD Pert fabs(const Pert &a) { return a.v < 0 ? -a : a; }
DGR_HD Pert fmax(const Pert &a, const Pert &b)
{
    const bool take_b = (b.v > a.v) || ::isnan(a.v);
    return Pert(::fmax(a.v, b.v), take_b ? b.p : a.p);
}
DGR_HD Pert fmax(double a, const Pert &b) { return fmax(Pert(a), b); }
DGR_HD Pert fmax(const Pert &a, double b) { return fmax(a, Pert(b)); }
DGR_HD Pert fmax_a(const Pert &a, const Pert &b) { return ((b.v > a.v) || ::isnan(a.v)) ? b : a; }
DGR_HD Pert fmax_a(double a, const Pert &b) { return fmax_a(Pert(a), b); }
DGR_HD Pert fmax_a(const Pert &a, double b) { return fmax_a(a, Pert(b)); }
DGR_HD Pert fmax_b(const Pert &a, const Pert &b)
{
    return Pert(dgr::fmax_b(a.v, b.v), ((b.v > a.v) || ::isnan(a.v)) ? b.p : a.p);
}
DGR_HD Pert fmax_b(double a, const Pert &b) { return fmax_b(Pert(a), b); }
DGR_HD Pert fmax_b(const Pert &a, double b) { return fmax_b(a, Pert(b)); }
DGR_HD Pert pow43(const Pert &a) { return Pert(dgr::pow43(a.v), dgr::pow43(a.p)); }
DGR_HD double val(const Pert &x) { return x.v; }

/* lanes of the two types: a value with its tangent (Dual) or its perturbed value (Pert) */
DGR_HD Dual lane(const Dual *, double v, double x) { return Dual(v, x); }
DGR_HD Pert lane(const Pert *, double v, double x) { return Pert(v, x); }
DGR_HD double second(const Dual &a) { return a.d; }
DGR_HD double second(const Pert &a) { return a.p; }

/* g n^2 of the Manning term: tangent 2 g n dn, or the value at the perturbed n (the
 * expression of the element set-up, (g n) n) */
DGR_HD Dual gnn_lane(const Dual *, double gnn, double g, double n, double x) { return Dual(gnn, 2.0 * g * n * x); }
DGR_HD Pert gnn_lane(const Pert *, double gnn, double g, double n, double x) { return Pert(gnn, g * x * x); }

}  // namespace ad
}  // namespace dgr
