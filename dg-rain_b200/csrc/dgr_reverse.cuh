/*
 * Hand-written reverse (adjoint) of the per-edge and per-element arithmetic in
 * dgr_scheme.cuh, FP64.  Each function recomputes the forward values it needs from the
 * same inputs (same expressions, so the same decisions: entropy-fix selections, clamps,
 * redistribution path, PDop branches) and then propagates adjoints backwards through them.
 * Decisions are frozen at the primal's, with the kink conventions of dgr_dual.cuh, so each
 * function is the exact transpose of the tangent-linear model of its forward counterpart.
 *
 * Adjoint outputs are ACCUMULATED (+=) into the caller's variables.
 */
#pragma once

#include "dgr_scheme.cuh"

namespace dgr {

/* adjoints of the Roe flux inputs */
struct RoeBar {
    double zin, zex, qxin, qxex, qyin, qyex, zed;
};

/* adjoints of one edge's traces: interior side, exterior side, mid-edge depth */
struct EdgeBar {
    double zi, qxi, qyi, ze, qxe, qye, zed;
};

/* T3: midpoint values -> vertex values (v0 = m0 - m1 + m2, ...), and its transpose */
DGR_HD void t3_transpose(const double y[3], double x[3])
{
    x[0] = y[0] + y[1] - y[2];
    x[1] = -y[0] + y[1] + y[2];
    x[2] = y[0] - y[1] + y[2];
}

/* normal-flux vector of one trace (the fn_in / fn_ex rows of roe_flux), reversed */
DGR_HD void normal_flux_rev(const double fb[3], double h, double u, double v, double z_edge, double nx, double ny,
                            double local_g, double &hb, double &ub, double &vb, double &zb)
{
    hb += fb[0] * (u * nx + v * ny);
    ub += fb[0] * h * nx;
    vb += fb[0] * h * ny;
    const double t1 = fb[1] * nx, t2 = fb[2] * ny;
    hb += t1 * u * u + t2 * v * v;
    ub += t1 * 2.0 * h * u;
    vb += t2 * 2.0 * h * v;
    const double pb = t1 + t2;
    const double huvb = fb[1] * ny + fb[2] * nx;
    hb += huvb * u * v;
    ub += huvb * h * v;
    vb += huvb * h * u;
    hb += pb * local_g * h;
    zb -= pb * local_g * z_edge;
}

/* Reverse of roe_flux (2DCode/numericalFlux2D.c:6-108): fhb = adjoint of Fhat.n. */
DGR_HD void roe_flux_rev(const double fhb[3], double zeta_in, double zeta_ex, double qx_in, double qx_ex, double qy_in,
                         double qy_ex, double z_edge, double nx, double ny, double local_g, double g, RoeBar &b)
{
    /* forward values, same expressions as roe_flux (the entropy fix's selections depend
     * on them): the quotients through one reciprocal per divisor, corrected to the IEEE
     * bits (div_rcp), and plain divisions where that is not valid */
    const double h_in = zeta_in + z_edge, h_ex = zeta_ex + z_edge;
    const double jump[3] = {zeta_in - zeta_ex, qx_in - qx_ex, qy_in - qy_ex};
    const double s_in = sqrt(h_in), s_ex = sqrt(h_ex);
    const double h_hat = 0.5 * (h_in + h_ex);
    const double D = s_in + s_ex;
    double u_in, u_ex, v_in, v_ex, u_hat, v_hat;
    {
        RcpDiv dv;
        const auto bi = dv.by(h_in), be = dv.by(h_ex);
        u_in = dv.div(qx_in, bi);
        u_ex = dv.div(qx_ex, be);
        v_in = dv.div(qy_in, bi);
        v_ex = dv.div(qy_ex, be);
        const auto bd = dv.by(D);
        u_hat = dv.div(u_in * s_in + u_ex * s_ex, bd);
        v_hat = dv.div(v_in * s_in + v_ex * s_ex, bd);
        if (!dv.ok) {
            u_in = qx_in / h_in;
            u_ex = qx_ex / h_ex;
            v_in = qy_in / h_in;
            v_ex = qy_ex / h_ex;
            u_hat = (u_in * s_in + u_ex * s_ex) / D;
            v_hat = (v_in * s_in + v_ex * s_ex) / D;
        }
    }
    const double c = sqrt(g * h_hat);
    const double un_in = u_in * nx + v_in * ny, un_ex = u_ex * nx + v_ex * ny;
    const double c_in = sqrt(g * h_in), c_ex = sqrt(g * h_ex);
    const double un_hat = u_hat * nx + v_hat * ny;
    const double raw[3] = {un_hat - c, un_hat, un_hat + c};
    const double lin[3] = {un_in - c_in, un_in, un_in + c_in};
    const double lex[3] = {un_ex - c_ex, un_ex, un_ex + c_ex};
    double lh[3];
    int sel[3]; /* entropy fix: 0 zero, 1 raw - l_in, 2 l_ex - raw, 3 |raw| */
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double ea = raw[i] - lin[i];
        int s = fmax_takes_b(0.0, ea) ? 1 : 0;
        double e = fmax_a(0.0, ea);
        const double eb = lex[i] - raw[i];
        if (fmax_takes_b(e, eb)) s = 2;
        e = fmax_a(e, eb);
        const double al = fabs(raw[i]);
        if (fmax_takes_b(e, al)) s = 3;
        lh[i] = fmax_a(e, al);
        sel[i] = s;
    }
    /* p1 = R^-1 jump in closed form (the forward's matrix entries simplified):
     * p1_0 = j0/2 + A, p1_2 = j0/2 - A, A = (un' j0 - nx j1 - ny j2)/(2c),
     * p1_1 = (ny u_hat - nx v_hat) j0 - ny j1 + nx j2.  These values only scale
     * derivatives, so their last-bit rounding does not matter. */
    const double ic2 = 1.0 / (2.0 * c);
    const double unp = nx * u_hat + ny * v_hat;
    const double A = (unp * jump[0] - nx * jump[1] - ny * jump[2]) * ic2;
    const double p1[3] = {0.5 * jump[0] + A, (ny * u_hat - nx * v_hat) * jump[0] - ny * jump[1] + nx * jump[2],
                          0.5 * jump[0] - A};
    const double p2[3] = {lh[0] * p1[0], lh[1] * p1[1], lh[2] * p1[2]};

    /* fh = 0.5 (fn_in + fn_ex) + 0.5 r p2 */
    const double p3b[3] = {0.5 * fhb[0], 0.5 * fhb[1], 0.5 * fhb[2]};
    const double p2b[3] = {p3b[0] + (u_hat - c * nx) * p3b[1] + (v_hat - c * ny) * p3b[2],
                           -ny * p3b[1] + nx * p3b[2],
                           p3b[0] + (u_hat + c * nx) * p3b[1] + (v_hat + c * ny) * p3b[2]};
    double uhb = p3b[1] * (p2[0] + p2[2]);
    double vhb = p3b[2] * (p2[0] + p2[2]);
    double cb = (p2[2] - p2[0]) * (nx * p3b[1] + ny * p3b[2]);
    const double lhb[3] = {p2b[0] * p1[0], p2b[1] * p1[1], p2b[2] * p1[2]};
    const double p1b[3] = {lh[0] * p2b[0], lh[1] * p2b[1], lh[2] * p2b[2]};

    /* p1 = R^-1 jump */
    const double Ab = p1b[0] - p1b[2];
    const double j0b = 0.5 * (p1b[0] + p1b[2]) + Ab * unp * ic2 + p1b[1] * (ny * u_hat - nx * v_hat);
    const double j1b = -Ab * nx * ic2 - ny * p1b[1];
    const double j2b = -Ab * ny * ic2 + nx * p1b[1];
    const double unpb = Ab * jump[0] * ic2;
    uhb += nx * unpb + p1b[1] * ny * jump[0];
    vhb += ny * unpb - p1b[1] * nx * jump[0];
    cb -= 2.0 * Ab * A * ic2;

    /* entropy fix */
    double rawb[3] = {0, 0, 0}, linb[3] = {0, 0, 0}, lexb[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double gb = lhb[i];
        if (sel[i] == 3) {
            rawb[i] += raw[i] < 0 ? -gb : gb;
        } else if (sel[i] == 2) {
            lexb[i] += gb;
            rawb[i] -= gb;
        } else if (sel[i] == 1) {
            rawb[i] += gb;
            linb[i] -= gb;
        }
    }
    const double unhb = rawb[0] + rawb[1] + rawb[2];
    cb += rawb[2] - rawb[0];
    const double un_in_b = linb[0] + linb[1] + linb[2], c_in_b = linb[2] - linb[0];
    const double un_ex_b = lexb[0] + lexb[1] + lexb[2], c_ex_b = lexb[2] - lexb[0];
    uhb += nx * unhb;
    vhb += ny * unhb;
    double uib = nx * un_in_b, vib = ny * un_in_b, ueb = nx * un_ex_b, veb = ny * un_ex_b;
    double hib = c_in == 0.0 ? 0.0 : c_in_b * g / (2.0 * c_in);
    double heb = c_ex == 0.0 ? 0.0 : c_ex_b * g / (2.0 * c_ex);

    /* c = sqrt(g h_hat), h_hat = (h_in + h_ex)/2 */
    const double hhb = c == 0.0 ? 0.0 : cb * g * ic2;
    hib += 0.5 * hhb;
    heb += 0.5 * hhb;

    /* Roe averages */
    const double iD = 1.0 / D;
    const double Nub = uhb * iD, Nvb = vhb * iD;
    const double Db = -(uhb * u_hat + vhb * v_hat) * iD;
    uib += Nub * s_in;
    ueb += Nub * s_ex;
    vib += Nvb * s_in;
    veb += Nvb * s_ex;
    const double sib = Nub * u_in + Nvb * v_in + Db, seb = Nub * u_ex + Nvb * v_ex + Db;
    hib += s_in == 0.0 ? 0.0 : sib / (2.0 * s_in);
    heb += s_ex == 0.0 ? 0.0 : seb / (2.0 * s_ex);

    /* physical normal fluxes */
    double zb = 0.0;
    normal_flux_rev(p3b, h_in, u_in, v_in, z_edge, nx, ny, local_g, hib, uib, vib, zb);
    normal_flux_rev(p3b, h_ex, u_ex, v_ex, z_edge, nx, ny, local_g, heb, ueb, veb, zb);

    /* velocities */
    const double ihi = 1.0 / h_in, ihe = 1.0 / h_ex;
    b.qxin += uib * ihi;
    b.qyin += vib * ihi;
    hib -= (uib * u_in + vib * v_in) * ihi;
    b.qxex += ueb * ihe;
    b.qyex += veb * ihe;
    heb -= (ueb * u_ex + veb * v_ex) * ihe;

    /* jump and depths */
    b.zin += j0b + hib;
    b.zex += heb - j0b;
    b.qxin += j1b;
    b.qxex -= j1b;
    b.qyin += j2b;
    b.qyex -= j2b;
    b.zed += zb + hib + heb;
}

/* Reverse of llf_flux: fhb = adjoint of Fhat.n.  The selected wave speed is the one the
 * forward's rmax chain keeps (ties to the later operand), |x| differentiated with the sign
 * of x (+ at 0), sqrt with derivative 0 at 0. */
DGR_HD void llf_flux_rev(const double fhb[3], double zeta_in, double zeta_ex, double qx_in, double qx_ex, double qy_in,
                         double qy_ex, double z_edge, double nx, double ny, double local_g, double g, RoeBar &b)
{
    const double h_in = zeta_in + z_edge, h_ex = zeta_ex + z_edge;
    const double u_in = qx_in / h_in, u_ex = qx_ex / h_ex;
    const double v_in = qy_in / h_in, v_ex = qy_ex / h_ex;
    const double un_in = u_in * nx + v_in * ny, un_ex = u_ex * nx + v_ex * ny;
    const double c_in = sqrt(g * h_in), c_ex = sqrt(g * h_ex);
    const double x[6] = {un_in - c_in, un_ex - c_ex, un_in, un_ex, un_in + c_in, un_ex + c_ex};
    int s = 0;
    double m = fabs(x[0]);
#pragma unroll
    for (int i = 1; i < 6; ++i) {
        const double a = fabs(x[i]);
        if (!(m > a)) {
            m = a;
            s = i;
        }
    }
    const double jump[3] = {zeta_ex - zeta_in, qx_ex - qx_in, qy_ex - qy_in};
    /* fh = 0.5 (fn_in + fn_ex) - 0.5 m jump */
    const double fnb[3] = {0.5 * fhb[0], 0.5 * fhb[1], 0.5 * fhb[2]};
    const double mb = -0.5 * (fhb[0] * jump[0] + fhb[1] * jump[1] + fhb[2] * jump[2]);
    const double jb[3] = {-0.5 * m * fhb[0], -0.5 * m * fhb[1], -0.5 * m * fhb[2]};
    const double xb = x[s] < 0 ? -mb : mb;
    double un_in_b = 0, un_ex_b = 0, c_in_b = 0, c_ex_b = 0;
    if (s == 0 || s == 2 || s == 4) un_in_b = xb;
    else un_ex_b = xb;
    if (s == 0) c_in_b = -xb;
    else if (s == 4) c_in_b = xb;
    else if (s == 1) c_ex_b = -xb;
    else if (s == 5) c_ex_b = xb;
    double uib = nx * un_in_b, vib = ny * un_in_b, ueb = nx * un_ex_b, veb = ny * un_ex_b;
    double hib = c_in == 0.0 ? 0.0 : c_in_b * g / (2.0 * c_in);
    double heb = c_ex == 0.0 ? 0.0 : c_ex_b * g / (2.0 * c_ex);
    double zb = 0.0;
    normal_flux_rev(fnb, h_in, u_in, v_in, z_edge, nx, ny, local_g, hib, uib, vib, zb);
    normal_flux_rev(fnb, h_ex, u_ex, v_ex, z_edge, nx, ny, local_g, heb, ueb, veb, zb);
    const double ihi = 1.0 / h_in, ihe = 1.0 / h_ex;
    b.qxin += uib * ihi;
    b.qyin += vib * ihi;
    hib -= (uib * u_in + vib * v_in) * ihi;
    b.qxex += ueb * ihe;
    b.qyex += veb * ihe;
    heb -= (ueb * u_ex + veb * v_ex) * ihe;
    b.zin += hib - jb[0];
    b.zex += heb + jb[0];
    b.qxin -= jb[1];
    b.qxex += jb[1];
    b.qyin -= jb[2];
    b.qyex += jb[2];
    b.zed += zb + hib + heb;
}

/* Reverse of hllc_flux with its branch and shock factors frozen at the forward's (the
 * branch by the forward's comparisons; sqrt with derivative 0 at 0). */
DGR_HD void hllc_flux_rev(const double fhb[3], double zeta_in, double zeta_ex, double qx_in, double qx_ex,
                          double qy_in, double qy_ex, double z_edge, double nx, double ny, double local_g, double g,
                          RoeBar &b)
{
    /* forward values, hllc_flux's expressions */
    const double h_in = zeta_in + z_edge, h_ex = zeta_ex + z_edge;
    const double u_in = qx_in / h_in, u_ex = qx_ex / h_ex;
    const double v_in = qy_in / h_in, v_ex = qy_ex / h_ex;
    const double un_in = u_in * nx + v_in * ny, un_ex = u_ex * nx + v_ex * ny;
    const double ut_in = -u_in * ny + v_in * nx, ut_ex = -u_ex * ny + v_ex * nx;
    const double c_in = sqrt(g * h_in), c_ex = sqrt(g * h_ex);
    const double P = 0.5 * (c_in + c_ex) + 0.25 * (un_in - un_ex);
    const double hs = 1.0 / g * P * P;
    const bool sh_ex = hs > h_ex, sh_in = hs > h_in;
    const double l_ex = sh_ex ? sqrt((hs * hs + hs * h_ex) / (2.0 * h_ex * h_ex)) : 1.0;
    const double l_in = sh_in ? sqrt((hs * hs + hs * h_in) / (2.0 * h_in * h_in)) : 1.0;
    const double s_in = un_in - c_in * l_in;
    const double s_ex = un_ex + c_ex * l_ex;
    const double A = un_ex - s_ex, B = un_in - s_in;
    const double N = s_in * h_ex * A - s_ex * h_in * B, D = h_ex * A - h_in * B;
    const double s_st = N / D;
    const int branch = s_in >= 0.0 ? 0 : (s_st >= 0.0 ? 1 : (s_ex >= 0.0 ? 2 : 3));
    const bool use_in = branch <= 1;
    const double h = use_in ? h_in : h_ex, u = use_in ? u_in : u_ex, v = use_in ? v_in : v_ex;

    /* adjoints of the chosen trace (h, u, v, un, ut, qx, qy) and of the speeds */
    double hb = 0, ub = 0, vb = 0, unb = 0, utb = 0, qxb = 0, qyb = 0;
    double s_inb = 0, s_exb = 0, s_stb = 0, zb = 0;
    normal_flux_rev(fhb, h, u, v, z_edge, nx, ny, local_g, hb, ub, vb, zb);
    if (branch == 1 || branch == 2) {
        const double S = use_in ? s_in : s_ex, un = use_in ? un_in : un_ex, ut = use_in ? ut_in : ut_ex;
        const double qx = use_in ? qx_in : qx_ex, qy = use_in ? qy_in : qy_ex;
        const double R = (S - un) / (S - s_st);
        const double q1 = h * R;
        const double d1 = q1 - h;
        const double d2 = q1 * s_st - (qx * nx + qy * ny);
        const double d3 = q1 * ut - (-qx * ny + qy * nx);
        const double Sb = fhb[0] * d1 + fhb[1] * (d2 * nx - d3 * ny) + fhb[2] * (d2 * ny + d3 * nx);
        const double d1b = S * fhb[0];
        const double d2b = S * (fhb[1] * nx + fhb[2] * ny);
        const double d3b = S * (-fhb[1] * ny + fhb[2] * nx);
        const double q1b = d1b + d2b * s_st + d3b * ut;
        s_stb += d2b * q1;
        utb += d3b * q1;
        hb -= d1b;
        qxb -= d2b * nx - d3b * ny;
        qyb -= d2b * ny + d3b * nx;
        hb += q1b * R;
        const double Rb = q1b * h;
        const double numb = Rb / (S - s_st);
        const double denb = -Rb * R / (S - s_st);
        const double Sbt = Sb + numb + denb;
        unb -= numb;
        s_stb -= denb;
        if (use_in)
            s_inb += Sbt;
        else
            s_exb += Sbt;
    }
    /* per-side adjoints */
    double h_inb = 0, h_exb = 0, un_inb = 0, un_exb = 0, ut_inb = 0, ut_exb = 0, c_inb = 0, c_exb = 0;
    double u_inb = 0, v_inb = 0, u_exb = 0, v_exb = 0;
    if (use_in) {
        h_inb += hb;
        u_inb += ub;
        v_inb += vb;
        un_inb += unb;
        ut_inb += utb;
        b.qxin += qxb;
        b.qyin += qyb;
    } else {
        h_exb += hb;
        u_exb += ub;
        v_exb += vb;
        un_exb += unb;
        ut_exb += utb;
        b.qxex += qxb;
        b.qyex += qyb;
    }
    /* s* = N / D */
    if (s_stb != 0.0) {
        const double Nb = s_stb / D, Db = -s_stb * s_st / D;
        double Ab = Nb * s_in * h_ex + Db * h_ex;
        double Bb = -Nb * s_ex * h_in - Db * h_in;
        s_inb += Nb * h_ex * A;
        h_exb += Nb * s_in * A + Db * A;
        s_exb -= Nb * h_in * B;
        h_inb -= Nb * s_ex * B + Db * B;
        un_exb += Ab;
        s_exb -= Ab;
        un_inb += Bb;
        s_inb -= Bb;
    }
    /* s_in = un_in - c_in l_in, s_ex = un_ex + c_ex l_ex */
    un_inb += s_inb;
    c_inb -= s_inb * l_in;
    const double l_inb = -s_inb * c_in;
    un_exb += s_exb;
    c_exb += s_exb * l_ex;
    const double l_exb = s_exb * c_ex;
    /* l = sqrt(W), W = (hs hs + hs h) / (2 h h) */
    double hsb = 0;
    if (sh_in && l_inb != 0.0) {
        const double Wb = l_inb / (2.0 * l_in);
        hsb += Wb * (2.0 * hs + h_in) / (2.0 * h_in * h_in);
        h_inb += Wb * (hs / (2.0 * h_in * h_in) - (hs * hs + hs * h_in) / (h_in * h_in * h_in));
    }
    if (sh_ex && l_exb != 0.0) {
        const double Wb = l_exb / (2.0 * l_ex);
        hsb += Wb * (2.0 * hs + h_ex) / (2.0 * h_ex * h_ex);
        h_exb += Wb * (hs / (2.0 * h_ex * h_ex) - (hs * hs + hs * h_ex) / (h_ex * h_ex * h_ex));
    }
    /* hs = P P / g */
    const double Pb = hsb * 2.0 * P / g;
    c_inb += 0.5 * Pb;
    c_exb += 0.5 * Pb;
    un_inb += 0.25 * Pb;
    un_exb -= 0.25 * Pb;
    /* c = sqrt(g h) */
    h_inb += c_in == 0.0 ? 0.0 : c_inb * g / (2.0 * c_in);
    h_exb += c_ex == 0.0 ? 0.0 : c_exb * g / (2.0 * c_ex);
    /* un = u nx + v ny, ut = -u ny + v nx */
    u_inb += un_inb * nx - ut_inb * ny;
    v_inb += un_inb * ny + ut_inb * nx;
    u_exb += un_exb * nx - ut_exb * ny;
    v_exb += un_exb * ny + ut_exb * nx;
    /* u = qx / h, v = qy / h */
    b.qxin += u_inb / h_in;
    b.qyin += v_inb / h_in;
    h_inb -= (u_inb * u_in + v_inb * v_in) / h_in;
    b.qxex += u_exb / h_ex;
    b.qyex += v_exb / h_ex;
    h_exb -= (u_exb * u_ex + v_exb * v_ex) / h_ex;
    b.zin += h_inb;
    b.zex += h_exb;
    b.zed += zb + h_inb + h_exb;
}

/* reverse of numerical_flux */
DGR_HD void numerical_flux_rev(int type, const double fhb[3], double zeta_in, double zeta_ex, double qx_in,
                               double qx_ex, double qy_in, double qy_ex, double z_edge, double nx, double ny,
                               double local_g, double g, RoeBar &b)
{
    if (type == 1)
        llf_flux_rev(fhb, zeta_in, zeta_ex, qx_in, qx_ex, qy_in, qy_ex, z_edge, nx, ny, local_g, g, b);
    else if (type == 2)
        hllc_flux_rev(fhb, zeta_in, zeta_ex, qx_in, qx_ex, qy_in, qy_ex, z_edge, nx, ny, local_g, g, b);
    else
        roe_flux_rev(fhb, zeta_in, zeta_ex, qx_in, qx_ex, qy_in, qy_ex, z_edge, nx, ny, local_g, g, b);
}

/* Reverse of the reflection (qx, qy) -> ghost discharge with the normal part negated and
 * the tangential part kept (2DCode/compute2DL.c:175-191). */
DGR_HD void reflect_rev(double nx, double ny, double oxb, double oyb, double &qxb, double &qyb)
{
    const double tx = -ny, ty = nx;
    const double d = 1. / (nx * ty - ny * tx);
    const double qnb = -(ty * oxb - tx * oyb) * d;
    const double qtb = (-ny * oxb + nx * oyb) * d;
    qxb += qnb * nx + qtb * tx;
    qyb += qnb * ny + qtb * ty;
}

/* Reverse of ghost_state: adjoints of the ghost (ze, qxe, qye) go to the interior trace.
 * For a land edge the exterior elevation is read from the interior trace's own slot, so
 * its adjoint lands in zib as well. */
DGR_HD void ghost_state_rev(int bd, double nx, double ny, double bz, double bq, double zeb, double qxeb, double qyeb,
                            double &zib, double &qxib, double &qyib)
{
    const double tx = -ny, ty = nx;
    const double d = 1. / (nx * ty - ny * tx);
    const double qnb = (ty * qxeb - tx * qyeb) * d;
    const double qtb = (-ny * qxeb + nx * qyeb) * d;
    qxib += qtb * tx;
    qyib += qtb * ty;
    if (bd) {
        if (bq > 1000) {
            qxib += qnb * nx;
            qyib += qnb * ny;
        }
        if (bz < 0) zib += zeb;
    } else {
        qxib -= qnb * nx;
        qyib -= qnb * ny;
        zib += zeb;
    }
}

/* Reverse of flux_core: finb/fexb = adjoints of the stored Fhat.n of the two sides. */
template <bool WD>
DGR_HD void flux_core_rev(double zi, double qxi, double qyi, double ze, double qxe, double qye, double z_edge, double nx,
                          double ny, int wdi, int wde, double g, const double finb[3], const double fexb[3], EdgeBar &b,
                          int ftype = 0)
{
    const double tx = -ny, ty = nx;
    if (WD && wdi == 0 && wde == 0) {
        const double d = 1. / (nx * ty - ny * tx);
        double qn_in = qxi * nx + qyi * ny;
        double qt_in = qxi * tx + qyi * ty;
        double qn_ex = -qn_in, qt_ex = qt_in;
        const double qxe_ref = (ty * qn_ex - ny * qt_ex) * d;
        const double qye_ref = (-tx * qn_ex + nx * qt_ex) * d;
        RoeBar r = {0, 0, 0, 0, 0, 0, 0};
        numerical_flux_rev(ftype, finb, zi, zi, qxi, qxe_ref, qyi, qye_ref, z_edge, nx, ny, 0.0, g, r);
        b.zi += r.zin + r.zex;
        b.qxi += r.qxin;
        b.qyi += r.qyin;
        b.zed += r.zed;
        reflect_rev(nx, ny, r.qxex, r.qyex, b.qxi, b.qyi);
        qn_ex = qxe * nx + qye * ny;
        qt_ex = qxe * tx + qye * ty;
        qn_in = -qn_ex;
        qt_in = qt_ex;
        const double qxi_ref = (ty * qn_in - ny * qt_in) * d;
        const double qyi_ref = (-tx * qn_in + nx * qt_ex) * d;
        RoeBar s = {0, 0, 0, 0, 0, 0, 0};
        numerical_flux_rev(ftype, fexb, ze, ze, qxi_ref, qxe, qyi_ref, qye, z_edge, nx, ny, 0.0, g, s);
        b.ze += s.zin + s.zex;
        b.qxe += s.qxex;
        b.qye += s.qyex;
        b.zed += s.zed;
        reflect_rev(nx, ny, s.qxin, s.qyin, b.qxe, b.qye);
        return;
    }
    const bool in_shared = !WD || wdi == 1, ex_shared = !WD || wde == 1;
    RoeBar r = {0, 0, 0, 0, 0, 0, 0};
    if (in_shared || ex_shared) {
        double fhb[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (in_shared) fhb[k] += finb[k];
            if (ex_shared) fhb[k] += fexb[k];
        }
        numerical_flux_rev(ftype, fhb, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, g, g, r);
    }
    if (!in_shared) numerical_flux_rev(ftype, finb, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, 0.0, g, r);
    if (!ex_shared) numerical_flux_rev(ftype, fexb, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, 0.0, g, r);
    b.zi += r.zin;
    b.ze += r.zex;
    b.qxi += r.qxin;
    b.qxe += r.qxex;
    b.qyi += r.qyin;
    b.qye += r.qyex;
    b.zed += r.zed;
}

/* Reverse of the RT0 fit (Cramer's rule): adjoints of (a, b, c) -> adjoints of R1..R3 (idM = 1/dM). */
DGR_HD void rt0_fit_rev(double ab, double bb, double cb, double M11, double M12, double M13, double M21, double M22,
                        double M23, double M31, double M32, double M33, double idM, double &R1b, double &R2b,
                        double &R3b)
{
    R1b += (ab * (M23 * M32 - M22 * M33) - bb * (M23 * M31 - M21 * M33) + cb * (M22 * M31 - M21 * M32)) * idM;
    R2b += (ab * (M12 * M33 - M13 * M32) - bb * (M11 * M33 - M13 * M31) + cb * (M11 * M32 - M12 * M31)) * idM;
    R3b += (ab * (M13 * M22 - M12 * M23) - bb * (M13 * M21 - M11 * M23) + cb * (M12 * M21 - M11 * M22)) * idM;
}

/*
 * Reverse of element_core.  wb = adjoint of its output w (of the RHS for MODE_RHS).
 * Accumulates: Fb[v][k] (adjoint of the gathered, outward F), Sb[v][k] (stage input; v = 0
 * elevation, 1 Qx, 2 Qy), midzb, gnnb, gradzb (depth and Manning factors).  The adjoint of
 * the step input u^n (cu wb, stage_coefficients) is left to the caller.
 */
template <int MODE, class Geo, class ZGeoV>
DGR_HD void element_core_rev(const double wb[3][3], const double zr[3], const double qxr[3], const double qyr[3],
                             const Geo &geo, const ZGeoV &zg, double local_g, double dt, double Fb[3][3],
                             double Sb[3][3], double midzb[3], double gnnb[3], double gradzb[2])
{
    const double nx[3] = {geo(G_NX), geo(G_NX + 1), geo(G_NX + 2)};
    const double ny[3] = {geo(G_NY), geo(G_NY + 1), geo(G_NY + 2)};
    const double M12 = geo(G_M12), M22 = geo(G_M12 + 1), M32 = geo(G_M12 + 2), dM = geo(G_DM);
    const double M11 = nx[0], M13 = ny[0], M21 = nx[1], M23 = ny[1], M31 = nx[2], M33 = ny[2];
    const double aj = geo(G_AJ), ajw = geo(G_AJW);
    const double weight = 1.0 / 6;
    const double m11 = geo(G_M11);
    /* The quotients below only scale derivatives (no decision of the forward depends on
     * them), so they are taken as products with one reciprocal per divisor: their last bit
     * does not matter, their count does (this kernel is latency-bound). */
    const double idM = 1.0 / dM;

    /* RK combination w = cu u + cs s + cr dt rhs, and the diagonal mass inverse */
    double Xb[3][3];
    double cu, sk, cr;
    stage_coefficients(MODE, cu, sk, cr);
    const double rk = MODE == MODE_RHS ? 1.0 : cr * dt;
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Sb[v][k] += sk * wb[v][k];
            Xb[v][k] = m11 * (wb[v][k] * rk);
        }

    /* volume terms: forward values */
    double H[3], iH[3], u[3], v[3], sp[3], iP[3], tau[3], midz[3], gnn[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        midz[e] = zg.midz(e);
        gnn[e] = zg.gnn(e);
        H[e] = zr[e] + midz[e];
        iH[e] = 1.0 / H[e];
        u[e] = qxr[e] * iH[e];
        v[e] = qyr[e] * iH[e];
        sp[e] = sqrt(u[e] * u[e] + v[e] * v[e]);
        iP[e] = 1.0 / pow43(H[e]);
        tau[e] = gnn[e] * sp[e] * iP[e];
    }
    const double bedx = local_g * aj * zg.gradz(0) * weight;
    const double bedy = local_g * aj * zg.gradz(1) * weight;

    /* X = -SI + DV + bed slope - friction */
    double zrb[3] = {0, 0, 0}, qxrb[3] = {0, 0, 0}, qyrb[3] = {0, 0, 0}, taub[3];
    double bedxb = 0, bedyb = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        bedxb += Xb[1][j] * zr[j];
        bedyb += Xb[2][j] * zr[j];
        zrb[j] += bedx * Xb[1][j] + bedy * Xb[2][j];
        taub[j] = -ajw * (Xb[1][j] * qxr[j] + Xb[2][j] * qyr[j]);
        qxrb[j] -= ajw * tau[j] * Xb[1][j];
        qyrb[j] -= ajw * tau[j] * Xb[2][j];
    }
    gradzb[0] += local_g * aj * weight * bedxb;
    gradzb[1] += local_g * aj * weight * bedyb;

    /* DV[v][bf] = aj (a/2 gp_bf,x + c/2 gp_bf,y + b w P_bf), (a, b, c) = RT0 fit of R[v] */
    double Rb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
    for (int vv = 0; vv < 3; ++vv) {
        double ab = 0, bb = 0, cb = 0;
#pragma unroll
        for (int bf = 0; bf < 3; ++bf) {
            ab += Xb[vv][bf] * geo(G_GP + 2 * bf);
            cb += Xb[vv][bf] * geo(G_GP + 2 * bf + 1);
            bb += Xb[vv][bf] * geo(G_P + bf);
        }
        rt0_fit_rev(aj * 0.5 * ab, aj * weight * bb, aj * 0.5 * cb, M11, M12, M13, M21, M22, M23, M31, M32, M33, idM,
                    Rb[vv][0], Rb[vv][1], Rb[vv][2]);
    }

    /* R[.][e] and tau[e] from the midpoint state */
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        double Hb = 0, qxb = 0, qyb = 0;
        qxb += Rb[0][e] * nx[e];
        qyb += Rb[0][e] * ny[e];
        const double prb = Rb[1][e] * nx[e] + Rb[2][e] * ny[e];
        const double qxyb = Rb[1][e] * ny[e] + Rb[2][e] * nx[e];
        const double a1 = Rb[1][e] * nx[e], a2 = Rb[2][e] * ny[e];
        qxb += a1 * 2.0 * u[e];
        Hb -= a1 * u[e] * u[e];
        qyb += a2 * 2.0 * v[e];
        Hb -= a2 * v[e] * v[e];
        qxb += qxyb * v[e];
        qyb += qxyb * u[e];
        Hb -= qxyb * u[e] * v[e];
        Hb += prb * local_g * H[e];
        midzb[e] -= prb * local_g * midz[e];
        const double tb = taub[e];
        gnnb[e] += tb * sp[e] * iP[e];
        Hb -= tb * tau[e] * (4.0 / 3.0) * iH[e];
        if (sp[e] != 0.0) {
            const double spb = tb * gnn[e] * iP[e];
            const double isp = 1.0 / sp[e];
            const double ub = spb * u[e] * isp, vb = spb * v[e] * isp;
            qxb += ub * iH[e];
            qyb += vb * iH[e];
            Hb -= (ub * u[e] + vb * v[e]) * iH[e];
        }
        zrb[e] += Hb;
        midzb[e] += Hb;
        qxrb[e] += qxb;
        qyrb[e] += qyb;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        Sb[0][k] += zrb[k];
        Sb[1][k] += qxrb[k];
        Sb[2][k] += qyrb[k];
    }

    /* surface integrals: SI[3v+bf] = sum_e ej_e sum_n fd[e][n] psi_bf(e, n) */
    const double ej[3] = {geo(G_EJ), geo(G_EJ + 1), geo(G_EJ + 2)};
#pragma unroll
    for (int vv = 0; vv < 3; ++vv) {
        double ab = 0, bb = 0, cb = 0;
#pragma unroll
        for (int e = 0; e < 3; ++e)
#pragma unroll
            for (int n = 0; n < 2; ++n) {
                double fdb = 0;
#pragma unroll
                for (int bf = 0; bf < 3; ++bf) fdb += -Xb[vv][bf] * geo(G_PSI + 6 * bf + 2 * e + n);
                fdb *= ej[e];
                ab += fdb * nx[e];
                bb += fdb * (geo(G_XE + 2 * e + n) * nx[e] + geo(G_YE + 2 * e + n) * ny[e]);
                cb += fdb * ny[e];
            }
        rt0_fit_rev(ab, bb, cb, M11, M12, M13, M21, M22, M23, M31, M32, M33, idM, Fb[vv][0], Fb[vv][1], Fb[vv][2]);
    }
}

/*
 * Reverse of limit_core (limiter then PDop) for one element.
 *   w         limiter input (the element stage output before limiting), values
 *   bnd       node max/min values as in limit_core
 *   wb        in: adjoint of limit_core's output; out: adjoint of its input
 *   bmaxb, bminb  accumulate the adjoints of bnd(v, k, 0) and bnd(v, k, 1) as [v][k]
 *   znb       accumulates the adjoint of the vertex depths
 * Returns the forward decisions.
 */
template <bool LIMIT, bool PDOP, class Bnd>
DGR_HD LimitDecisions limit_core_rev(const double w[3][3], const Bnd &bnd, const double zn[3], double h0, double velzero,
                                     double wb[3][3], double bmaxb[3][3], double bminb[3][3], double znb[3])
{
    /* forward: limited values and decisions */
    double wl[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) wl[v][k] = w[v][k];
    LimitDecisions dec;
    LimitTrace trace;
    limit_core<LIMIT, false, double, Bnd, true>(wl, bnd, zn, h0, velzero, dec, &trace);
    const int modify = dec.modify;

    if (PDOP) {
        /* forward PDop on wl, keeping what the reverse needs */
        const double midz[3] = {0.5 * (zn[0] + zn[1]), 0.5 * (zn[1] + zn[2]), 0.5 * (zn[2] + zn[0])};
        const double mh[3] = {wl[0][0] + midz[0], wl[0][1] + midz[1], wl[0][2] + midz[2]};
        const double ht[3] = {mh[0] - mh[1] + mh[2], mh[0] + mh[1] - mh[2], -mh[0] + mh[1] + mh[2]};
        const double avg_h = (ht[0] + ht[1] + ht[2]) / 3;
        double htp[3] = {ht[0], ht[1], ht[2]};
        int mass = 0, imin = 0, inext = 1, irem = 2, takes_x = 0;
        double hmin = 0, hnext = 0;
        if (ht[0] <= h0 || ht[1] <= h0 || ht[2] <= h0) {
            if (avg_h <= h0) {
                mass = 1;
                htp[0] = htp[1] = htp[2] = avg_h;
            } else {
                mass = 2;
                hmin = ht[0];
                if (ht[1] < hmin) { imin = 1; hmin = ht[1]; }
                if (ht[2] < hmin) { imin = 2; hmin = ht[2]; }
                hnext = ht[1];
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (ht[i] < hnext && i != imin) { inext = i; hnext = ht[i]; }
                if (0 != imin && 0 != inext) irem = 0;
                else if (1 != imin && 1 != inext) irem = 1;
                double hh[3] = {ht[0], ht[1], ht[2]};
                hh[imin] = h0;
                const double X = hnext - 0.5 * (hh[imin] - hmin);
                takes_x = fmax_takes_b(h0, X);
                hh[inext] = fmax(h0, X);
                hh[irem] = hh[irem] - (hh[imin] - hmin) - (hh[inext] - hnext);
                htp[0] = hh[0];
                htp[1] = hh[1];
                htp[2] = hh[2];
            }
        }
        const int wet[3] = {htp[0] > h0, htp[1] > h0, htp[2] > h0};
        int mom = 0;
        if (wet[0] == 0 && wet[1] == 0 && wet[2] == 0) mom = 1;
        else if (wet[0] == 0 || wet[1] == 0 || wet[2] == 0) mom = 2;

        /* reverse: momentum */
        double htpb[3] = {0, 0, 0};
        double w1b[3], w2b[3];
        if (mom == 1) {
            w1b[0] = w1b[1] = w1b[2] = 0;
            w2b[0] = w2b[1] = w2b[2] = 0;
        } else if (mom == 2) {
            const double q[2][3] = {{wl[1][0], wl[1][1], wl[1][2]}, {wl[2][0], wl[2][1], wl[2][2]}};
            int npos = wet[0] + wet[1] + wet[2];
            double qbar_v[2][3];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const double qe[3] = {q[c][0] - q[c][1] + q[c][2], q[c][0] + q[c][1] - q[c][2],
                                      -q[c][0] + q[c][1] + q[c][2]};
                double uu[3], up[3];
                int mask[3];
                double del = 0;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    uu[i] = qe[i] / htp[i];
                    mask[i] = (1 - wet[i]) && (fabs(qe[i]) > velzero);
                    del += uu[i] * (double)(1 - wet[i]) * (double)(fabs(qe[i]) > velzero);
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) up[i] = (double)wet[i] * (uu[i] + del / (double)npos);
                const double *ob = wb[1 + c];
                double qepb[3], ub[3], delb = 0;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    qepb[i] = 0.5 * (ob[i] + ob[(i + 2) % 3]);
                    htpb[i] += qepb[i] * up[i];
                    const double upb = qepb[i] * htp[i];
                    ub[i] = wet[i] ? upb : 0.0;
                    if (wet[i]) delb += upb / (double)npos;
                }
                double qeb[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    if (mask[i]) ub[i] += delb;
                    qeb[i] = 0.0;
                    if (ub[i] != 0.0) {
                        qeb[i] = ub[i] / htp[i];
                        htpb[i] -= ub[i] * uu[i] / htp[i];
                    }
                }
                t3_transpose(qeb, qbar_v[c]);
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                w1b[i] = qbar_v[0][i];
                w2b[i] = qbar_v[1][i];
            }
        } else {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                w1b[i] = wb[1][i];
                w2b[i] = wb[2][i];
            }
        }

        /* reverse: mass */
        double midzb[3] = {0, 0, 0}, w0b[3];
        if (mass) {
            double mhpb[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                mhpb[k] = wb[0][k];
                midzb[k] -= wb[0][k];
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) htpb[i] += 0.5 * (mhpb[i] + mhpb[(i + 2) % 3]);
            double htb[3] = {0, 0, 0};
            if (mass == 1) {
                const double ab = htpb[0] + htpb[1] + htpb[2];
#pragma unroll
                for (int i = 0; i < 3; ++i) htb[i] = ab / 3;
            } else {
                /* the assignments of :127-139 in reverse, with index aliasing handled by
                 * accumulation (the reference's next-smallest search may return imin) */
                double hhb[3] = {htpb[0], htpb[1], htpb[2]};
                double hminb = 0, hnextb = 0;
                const double t = hhb[irem];
                hhb[irem] = 0;
                hhb[irem] += t;
                hhb[imin] -= t;
                hhb[inext] -= t;
                hminb += t;
                hnextb += t;
                const double cbar = hhb[inext];
                hhb[inext] = 0;
                if (takes_x) {
                    hnextb += cbar;
                    hhb[imin] -= 0.5 * cbar;
                    hminb += 0.5 * cbar;
                }
                hhb[imin] = 0;
#pragma unroll
                for (int i = 0; i < 3; ++i) htb[i] = hhb[i];
                htb[imin] += hminb;
                htb[inext] += hnextb;
            }
            double mhb[3];
            t3_transpose(htb, mhb);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                w0b[k] = mhb[k];
                midzb[k] += mhb[k];
            }
        } else {
            double mhb[3];
            t3_transpose(htpb, mhb);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                w0b[k] = wb[0][k] + mhb[k];
                midzb[k] += mhb[k];
            }
        }
        znb[0] += 0.5 * (midzb[0] + midzb[2]);
        znb[1] += 0.5 * (midzb[0] + midzb[1]);
        znb[2] += 0.5 * (midzb[1] + midzb[2]);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            wb[0][k] = w0b[k];
            wb[1][k] = w1b[k];
            wb[2][k] = w2b[k];
        }
        dec.mass_branch = mass;
        dec.mom_branch = mom;
    }

    if (LIMIT && modify) {
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const unsigned long long tb = trace.bits[v];
            double vxb[3] = {0.5 * (wb[v][0] + wb[v][2]), 0.5 * (wb[v][0] + wb[v][1]), 0.5 * (wb[v][1] + wb[v][2])};
            double avgb = 0;
#pragma unroll
            for (int ll = 2; ll >= 0; --ll) {
                const int sd = (int)((tb >> (6 + 2 * ll)) & 3) - 1;
                const double sdd = (double)sd;
                double sumdiffb = 0;
#pragma unroll
                for (int k = 2; k >= 0; --k) {
                    const int bits = (int)((tb >> (12 + 4 * (3 * ll + k))) & 15);
                    const double rfb = -sdd * (sumdiffb + vxb[k]);
                    if (bits & 2) {
                        if (sd > 0) {
                            vxb[k] += rfb;
                            bminb[v][k] -= rfb;
                        } else {
                            bmaxb[v][k] += rfb;
                            vxb[k] -= rfb;
                        }
                    } else if (bits & 1) {
                        sumdiffb += rfb * sdd / (double)(bits >> 2);
                    }
                }
                vxb[0] += sumdiffb;
                vxb[1] += sumdiffb;
                vxb[2] += sumdiffb;
                avgb -= 3.0 * sumdiffb;
            }
            double rawb[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int clamp = (int)((tb >> (2 * k)) & 3);
                rawb[k] = 0;
                if (clamp == 2) bminb[v][k] += vxb[k];
                else if (clamp == 1) bmaxb[v][k] += vxb[k];
                else rawb[k] = vxb[k];
            }
            double inb[3];
            t3_transpose(rawb, inb);
#pragma unroll
            for (int k = 0; k < 3; ++k) wb[v][k] = inb[k] + avgb / 3;
        }
    }
    return dec;
}

}  // namespace dgr
