// Point exchange-correlation functionals (FP64), host+device.
//
// Restated from the published functionals in the form LIO evaluates them:
//   LDA:  Slater exchange + Gunnarsson-Lundqvist (iexch 2) / VWN (iexch 3)
//         correlation, g2g/pointxc/calc_ldaCS.h:33-102;
//   PBE closed shell (iexch 9): g2g/pointxc/calc_ggaCS.h:127-149 and
//         g2g/pointxc/pbeCS.h:30-185 with the PW92 G-function of gcorc.h:22-33;
//   PBE open shell: g2g/pointxc/calc_ggaOS.h:11-109, pbeOS_main.h:29-205,
//         pbeOS_exch.h:42-75, pbeOS_corr.h:63-251, gcorc.h (three parameter sets).
// The potential is LIO's scalar "Laplacian" form: for GGA y2a depends on rho,
// |grad rho|, grad rho . grad|grad rho| and the Laplacian, so the Kohn-Sham
// update needs only the basis values.
//
// Constant values must equal the reference's to the last bit, since a change of
// 1e-8 relative in a parameter moves E_xc by more than the 1e-6 Ha tolerance on
// large systems. Several reference constants are float literals converted to
// double (e.g. 0.804f, the PW92 parameters, 4.0f/3.0f evaluated in float); they
// are written here as F(x) = (double)(float)x and F43 = (double)(4.0f/3.0f).
#pragma once
#include <cfloat>
#include <cmath>

#ifndef __CUDACC__
#define LIO_HD
#else
#define LIO_HD __host__ __device__
#endif

namespace lio {
namespace xc {

#define LIO_F(x) ((double)(float)(x))

// ---------------------------------------------------------------- LDA (calc_ldaCS.h)
struct LdaOut {
  double ex, ec, v;
};

LIO_HD inline LdaOut lda_closed(double dens, int iexch) {
  LdaOut o{0.0, 0.0, 0.0};
  if (dens == 0) return o;  // only exact zero is guarded (calc_ldaCS.h:38-43)
  const double y = cbrt(dens);
  const double v0 = -0.984745021842697 * y;  // -4/3 (3/pi)^(1/3) rho^(1/3)
  o.ex = -0.738558766382022447 * y;          // -(3/pi)^(1/3) rho^(1/3)
  if (iexch == 1) {
    o.ec = 0;
    o.v = v0;
  } else if (iexch == 2) {  // Gunnarsson-Lundqvist
    const double rs = 0.620350490899400087 / y;
    const double x1 = rs / 11.4;
    double vc;
    if (x1 > 1.0) {
      o.ec = -0.0333 * (0.5 * x1 - 0.33333333333333);
      vc = 0.0111 * x1 * 0.5;
    } else {
      const double t1 = 1.0 + x1 * x1 * x1;
      const double t2 = log(1.0 + 1.0 / x1);
      const double t3 = x1 * x1;
      o.ec = -0.0333 * (t1 * t2 - t3 + 0.5 * x1 - 0.33333333333333);
      vc = 0.0111 * x1 * (3.0 * t3 * t2 - t1 / (x1 * (x1 + 1.0)) - 2.0 * x1 + 0.5);
    }
    o.v = v0 + o.ec + vc;
  } else {  // iexch 3: Vosko-Wilk-Nusair
    const double A1 = 0.03109205, B1 = 3.72744, X0 = -0.10498, Q = 6.15199066246304849;
    const double A16 = 0.005182008333, T4 = -0.0311676086789438, C1x2 = 25.8704;
    const double B1x2_Q = 1.21178337371132, B2X0_Q = 1.14352579286644, B1x4 = 14.90976;
    const double QSQ = 37.8469891110325, B1X0 = 1.0329232240928, C1 = 12.9352;
    const double rs = 0.620350490899400087 / y;
    const double x1 = sqrt(rs);
    const double Xx = rs + B1 * x1 + C1;
    const double t1 = 2.0 * x1 + B1;
    const double t2 = log(Xx);
    const double t3 = atan(Q / t1);
    const double t5 = (B1 * x1 + C1x2) / x1;
    o.ec = (2.0 * log(x1) - t2 + B1x2_Q * t3 - T4 * (2.0 * log(x1 - X0) - t2 + B2X0_Q * t3)) * A1;
    const double vc =
        o.ec - A16 * x1 * (t5 / Xx - B1x4 / (t1 * t1 + QSQ) * B1X0 - T4 * (2.0 / (x1 - X0) - t1 / Xx));
    o.v = v0 + vc;
  }
  return o;
}

// ------------------------------------------------ PW92 G-function (gcorc.h)
struct PW92Set {
  double a0, a1, b1, b2, b3, b4;
};
LIO_HD inline PW92Set pw92_set(int which) {
  if (which == 1)
    return {LIO_F(0.0310907f), LIO_F(0.21370f), LIO_F(7.5957f), LIO_F(3.5876f), LIO_F(1.6382f),
            LIO_F(0.49294f)};
  if (which == 2)
    return {LIO_F(0.01554535f), LIO_F(0.20548f), LIO_F(14.1189f), LIO_F(6.1977f), LIO_F(3.3662f),
            LIO_F(0.62517f)};
  return {LIO_F(0.0168869f), LIO_F(0.11125f), LIO_F(10.357f), LIO_F(3.6231f), LIO_F(0.88026f),
          LIO_F(0.49671f)};
}

// G(rs) and dG/drs for the interpolation of J. P. Perdew, Y. Wang, PRB 45, 13244 (1992)
LIO_HD inline void pw92_g(const PW92Set& s, double rtrs, double& g, double& dgdrs) {
  const double q0 = -2.0 * s.a0 * (1.0 + s.a1 * rtrs * rtrs);
  const double q1 = 2.0 * s.a0 * rtrs * (s.b1 + rtrs * (s.b2 + rtrs * (s.b3 + s.b4 * rtrs)));
  const double q2 = log(1.0 + 1.0 / q1);
  g = q0 * q2;
  const double q3 = s.a0 * (s.b1 / rtrs + 2.0 * s.b2 + rtrs * (3.0 * s.b3 + 4.0 * s.b4 * rtrs));
  dgdrs = -2.0 * s.a0 * s.a1 * q2 - q0 * q3 / (q1 * (1.0 + q1));
}

// float-evaluated constant expressions of the reference
#define LIO_F43 ((double)(4.0f / 3.0f))
#define LIO_F13 ((double)(1.0f / 3.0f))
#define LIO_FM16 ((double)(-1.0f / 6.0f))
// pow(2.0, 4.0 / 3.0) - 2.0 as the C library evaluates it (pbeOS_corr.h)
#define LIO_GAM 0x1.0a28be635ca2cp-1

// ---------------------------------------------------- PBE closed shell (pbeCS.h)
struct GgaOut {
  double ex, ec, v;
};

LIO_HD inline void pbe_closed_core(double rho, double agrad, double delgrad, double rlap, double& expbe,
                                   double& vxpbe, double& ecpbe, double& vcpbe) {
  const double MIN_RHO = 1e-18;
  const double PI32 = LIO_F(29.608813203268075856503472999628f);  // 3 pi^2
  const double AX = LIO_F(-0.738558766382022405884230032680836f);
  const double UM = LIO_F(0.2195149727645171f), UK = LIO_F(0.804f), UL = LIO_F(0.273028573090195f);
  const double GAMMAINV = LIO_F(32.1639684429148f), BETA = LIO_F(0.06672455060314922f);
  const double DELTA = LIO_F(2.14612633996736f);

  const double rho2 = rho * rho;
  const double rho13 = cbrt(rho);
  const double fk = cbrt(PI32) * rho13;
  if (rho2 > MIN_RHO) {
    const double twofk = 2.0 * fk, twofk2 = twofk * twofk, twofk3 = twofk * twofk2;
    const double s = agrad / (twofk * rho);
    const double s2 = s * s, s3 = s * s2;
    const double exlda = AX * rho13;
    const double p0 = 1.0 + UL * s2;
    const double fxpbe = 1.0 + UK - UK / p0;
    expbe = exlda * fxpbe;
    const double v = rlap / (twofk2 * rho);
    const double u = delgrad / (twofk3 * rho2);
    const double Fs = 2.0 * UM / (p0 * p0);
    const double Fss = (-4.0 * UL * s * Fs) / p0;
    vxpbe = exlda * (LIO_F43 * fxpbe - (u - LIO_F43 * s3) * Fss - v * Fs);
  } else {
    expbe = 0.0;
    vxpbe = 0.0;
  }
  if (rho < MIN_RHO * 1e6) {  // correlation dropped below 1e-12 (pbeCS.h:118-122)
    ecpbe = 0.0;
    vcpbe = 0.0;
    return;
  }
  const double pirho = 4.0 * M_PI * rho;
  const double rs = cbrt(3.0 / pirho);
  const double rtrs = sqrt(rs);
  const double sk = sqrt(4.0 * fk / M_PI);
  const double twoks = 2.0 * sk, twoks2 = twoks * twoks, twoks3 = twoks2 * twoks;
  const double t = agrad / (twoks * rho);
  const double t2 = t * t;
  const double UU = delgrad / (rho2 * twoks3);
  const double VV = rlap / (rho * twoks2);
  double ec, ecrs;
  pw92_g(pw92_set(1), rtrs, ec, ecrs);
  const double vclda = ec - rs * LIO_F13 * ecrs;
  const double PON = -ec * GAMMAINV;
  const double B = DELTA / (exp(PON) - 1.0);
  const double B2 = B * B;
  const double T4 = t2 * t2;
  const double Q4 = 1.0 + B * t2;
  const double Q5 = 1.0 + B * t2 + B2 * T4;
  const double H = (BETA / DELTA) * log(1.0 + DELTA * Q4 * t2 / Q5);
  ecpbe = ec + H;
  const double T6 = T4 * t2;
  const double RSTHRD = rs / 3.0;
  const double FAC = DELTA / B + 1.0;
  const double BEC = B2 * FAC / BETA;
  const double Q8 = (Q5 + DELTA * Q4 * t2) * Q5;
  const double Q9 = 1.0 + 2.0 * B * t2;
  const double hB = -BETA * B * (T6 / Q8) * (2.0 + B * t2);
  const double hRS = -RSTHRD * hB * BEC * ecrs;
  const double FACT0 = 2.0 * DELTA - 6.0 * B;
  const double FACT1 = Q5 * Q9 + Q4 * Q9 * Q9;
  const double hBT = 2.0 * BETA * T4 * ((Q4 * Q5 * FACT0 - DELTA * FACT1) / Q8) / Q8;
  const double hRST = RSTHRD * t2 * hBT * BEC * ecrs;
  const double hT = 2.0 * BETA * (Q9 / Q8);
  const double FACT2 = Q4 * Q5 + B * t2 * (Q4 * Q9 + Q5);
  const double FACT3 = 2.0 * B * Q5 * Q9 + DELTA * FACT2;
  const double hTT = 4.0 * BETA * t * (2.0 * B / Q8 - ((Q9 / Q8) * FACT3) / Q8);
  double COMM = H + hRS + hRST + t2 * hT / 6.0 + 7.0 * t2 * t * hTT / 6.0;
  COMM = COMM - UU * hTT - VV * hT;
  vcpbe = vclda + COMM;
}

// calc_ggaCS.h:36-57,127-149: rho, grad, (xx,yy,zz), (xy,xz,yz) -> ex, ec, y2a
LIO_HD inline GgaOut pbe_closed(double dens, const double g[3], const double h1[3], const double h2[3]) {
  GgaOut o{0.0, 0.0, 0.0};
  if (dens < 1e-18) return o;
  double grad2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
  if (grad2 < DBL_MIN) grad2 = DBL_MIN;
  const double dgrad = sqrt(grad2);
  const double d1 = g[0] * g[0] * h1[0], d2 = g[1] * g[1] * h1[1], d3 = g[2] * g[2] * h1[2];
  const double d4 = g[0] * g[1] * h2[0], d5 = g[0] * g[2] * h2[1], d6 = g[1] * g[2] * h2[2];
  const double delgrad = (d1 + d2 + d3 + 2 * (d4 + d5 + d6)) / dgrad;
  const double rlap = h1[0] + h1[1] + h1[2];
  double expbe, vxpbe, ecpbe, vcpbe;
  pbe_closed_core(dens, dgrad, delgrad, rlap, expbe, vxpbe, ecpbe, vcpbe);
  o.ex = expbe;
  o.ec = ecpbe;
  o.v = vxpbe + vcpbe;
  return o;
}

// ------------------------------------- other closed-shell GGAs (calc_ggaCS.h)
// iexch 4: Perdew 86 exchange + Perdew 86 correlation; 5: Becke 88 exchange +
// Perdew 86; 6: Becke 88 + the VWN-form local correlation alone; 7: Becke 88 +
// Lee-Yang-Parr; 8: Perdew 86 exchange + LYP (g2g/pointxc/calc_ggaCS.h:36-262).
// The reference's constants, including its float literals (LIO_F), and its
// operation order are kept; rho, grad, (xx, yy, zz), (xy, xz, yz) -> ex, ec, y2a.
LIO_HD inline GgaOut gga_closed_other(double dens, const double g[3], const double h1[3], const double h2[3],
                                      int iexch) {
  GgaOut o{0.0, 0.0, 0.0};
  if (dens < 1e-18) return o;
  const double ALPHA = -0.738558766382022447, GL = 0.620350490899400087;
  const double VA1 = 0.03109205, VB1 = 3.72744, VC1 = 12.9352, VX0 = -0.10498, VQ = 6.15199066246304849;
  const double VA16 = 0.005182008333, VQ2 = 4.7309269;
  const double ALYP = 0.04918, BLYP = 0.132, CLYP = 0.2533, CLYP3 = 0.0844333333, DLYP = 0.349,
               DLYP3 = 0.116333333, CF = 2.87123400018819;
  const double B88 = 0.0042, ALF = 0.023266, BET = 7.389, GAM = 8.723, DEL = 0.472;
  const double y = cbrt(dens);
  double grad2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
  if (grad2 < DBL_MIN) grad2 = DBL_MIN;
  const double dgrad = sqrt(grad2);
  const double lap = h1[0] + h1[1] + h1[2];
  const double u0 = ((g[0] * g[0]) * h1[0] + 2.0 * g[0] * g[1] * h2[0] + 2.0 * g[1] * g[2] * h2[2] +
                     2.0 * g[0] * g[2] * h2[1] + (g[1] * g[1]) * h1[1] + (g[2] * g[2]) * h1[2]) /
                    dgrad;
  double v = 0.0;
  if (iexch == 4 || iexch == 8) {  // exchange: Perdew, PRB 33, 8800 (1986)
    const double dens2 = dens * dens;
    const double ckf = 3.0936677 * y;
    const double s = dgrad / (2.0 * ckf * dens);
    const double fx = 1.0 / 15.0;
    const double s2 = s * s, s3 = s * s * s, s4 = pow(s, 4);
    const double g0 = 1.0 + 1.296 * s2 + 14.0 * s4 + 0.2 * pow(s, 6);
    const double F = pow(g0, fx);
    o.ex = ALPHA * F * y;
    const double t = lap / (dens * 4.0 * (ckf * ckf));
    const double u = u0 / (pow(2.0 * ckf, 3) * dens2);
    const double g2 = 2.592 * s + 56.0 * s3 + 1.2 * pow(s, 5);
    const double g3 = 2.592 + 56.0 * s2 + 1.2 * s4;
    const double g4 = 112.0 * s + 4.8 * s3;
    const double dF = fx * F / g0 * g2;
    const double dsF = fx * F / g0 * (-14.0 * fx * g3 * g2 / g0 + g4);
    v = ALPHA * y * (1.33333333333 * F - t / s * dF - (u - 1.3333333333 * s3) * dsF);
  } else {  // exchange: Becke, PRA 38, 3098 (1988)
    const double e0 = ALPHA * y;
    const double half = dens / 2.0;
    const double r13 = cbrt(half);
    const double r43 = cbrt(pow(half, 4));
    const double xs = dgrad / (2.0 * r43);
    const double ash = asinh(xs);
    const double dn = 1.0 + 6.0 * B88 * xs * ash;
    o.ex = e0 + (-2.0 * B88 * r43 * xs * xs / (dn * dens));
    const double v0 = 1.33333333333333 * e0;
    const double fb = 1.0 / dn;
    const double xa1 = xs / sqrt(1.0 + xs * xs);
    const double dn1 = 1.0 + fb * (1.0 - 6.0 * B88 * xs * xa1);
    const double dn2 = 1.0 / (1.0 + xs * xs) + 2.0 * fb * (2.0 - 6.0 * B88 * xs * xa1);
    const double dn3 = ash * (1.0 + 2.0 * fb) + xa1 * dn2;
    const double d02 = lap / 2.0;
    const double de1 = 1.33333333333333 / (cbrt(pow(dens, 7)));
    const double c2 = cbrt(2.0);
    // d|grad|/da along each axis and the gradient of x_sigma
    const double dgx = (g[0] * h1[0] + g[1] * h2[0] + g[2] * h2[1]) / dgrad;
    const double gxx = c2 * (1.0 / (dens * y) * dgx - de1 * g[0] * dgrad);
    const double dgy = (g[0] * h2[0] + g[1] * h1[1] + g[2] * h2[2]) / dgrad;
    const double gxy = c2 * (1.0 / (dens * y) * dgy - de1 * g[1] * dgrad);
    const double dgz = (g[0] * h2[1] + g[1] * h2[2] + g[2] * h1[2]) / dgrad;
    const double gxz = c2 * (1.0 / (dens * y) * dgz - de1 * g[2] * dgrad);
    const double dn4 = 6.0 * B88 * fb * (g[0] / 2.0 * gxx + g[1] / 2.0 * gxy + g[2] / 2.0 * gxz);
    const double dn5 = 1.33333333333333 * r43 * r13 * xs * xs;
    const double tot2 = dn5 - d02 * dn1 + dn4 * dn3;
    v = v0 + (-B88 * fb / r43 * tot2);
  }
  if (iexch >= 4 && iexch <= 6) {  // correlation: VWN-form local part (+ Perdew, PRB 33, 8822 (1986))
    const double dens2 = dens * dens;
    const double rs = GL / y;
    const double x1 = sqrt(rs);
    const double Xx = rs + VB1 * x1 + VC1;
    const double Xxo = (VX0 * VX0) + VB1 * VX0 + VC1;
    const double t1 = 2.0 * x1 + VB1;
    const double t2 = log(Xx);
    const double t3 = atan(VQ / t1);
    const double t4 = VB1 * VX0 / Xxo;
    double ec = VA1 * (2.0 * log(x1) - t2 + 2.0 * VB1 / VQ * t3 -
                       t4 * (2.0 * log(x1 - VX0) - t2 + 2.0 * (VB1 + 2.0 * VX0) / VQ * t3));
    const double t5 = (VB1 * x1 + 2.0 * VC1) / x1;
    const double t6 = VX0 / Xxo;
    double vc = ec - VA16 * x1 *
                         (t5 / Xx - 4.0 * VB1 / ((t1 * t1) + (VQ * VQ2)) * (1.0 - t6 * (VB1 - 2.0 * VX0)) -
                          t4 * (2.0 / (x1 - VX0) - t1 / Xx));
    if (iexch != 6) {
      const double rs2 = rs * rs;
      const double cx1 = LIO_F(0.002568f) + ALF * rs + BET * rs2;
      const double cx2 = 1.0 + GAM * rs + DEL * rs2 + 1.0e4 * BET * (rs * rs * rs);
      const double C = 0.001667 + cx1 / cx2;
      const double cx3 = ALF + 2.0 * BET * rs;
      const double cx4 = GAM + 2.0 * DEL * rs + 3.0e4 * BET * rs2;
      double dC = cx3 / cx2 - cx1 / (cx2 * cx2) * cx4;
      dC = LIO_F(-0.333333333333333f) * dC * GL / (y * dens);
      const double phi = LIO_F(0.0008129082f) / C * dgrad / pow(dens, (double)(7.0f / 6.0f));
      const double ex_ = exp(-phi);
      const double ex0 = ex_ * C;
      ec = ec + ex0 * grad2 / (y * dens2);
      const double D1 = (2.0 - phi) * lap / dens;
      const double phi2 = phi * phi;
      double D2 = LIO_F(1.33333333333333333f) - LIO_F(3.666666666666666666f) * phi + LIO_F(1.166666666666666f) * phi2;
      D2 = D2 * grad2 / dens2;
      const double D3 = phi * (phi - 3.0) * u0 / (dens * dgrad);
      const double D4 = ex_ * grad2 / (y * dens) * (phi2 - phi - 1.0) * dC;
      vc = vc - 1.0 * (ex0 / y * (D1 - D2 + D3) - D4);
    }
    o.ec = ec;
    v = v + vc;
  } else {  // correlation: Lee, Yang, Parr, PRB 37, 785 (1988)
    const double rom13 = 1 / cbrt(dens);
    const double rom53 = cbrt(pow(dens, 5));
    const double ecro = exp(-CLYP * rom13);
    const double f1 = 1.0 / (1.0 + DLYP * rom13);
    const double tw = 0.125 * (grad2 / dens - lap);
    double term = (tw / 9.0 + lap / 18.0) - 2.0 * tw + CF * rom53;
    term = dens + BLYP * (rom13 * rom13) * ecro * term;
    o.ec = -ALYP * f1 * term / dens;
    const double hh1 = ecro / rom53;
    const double gg1 = f1 * hh1;
    const double tm1 = DLYP3 * (rom13 / dens);
    const double fp1 = tm1 * (f1 * f1);
    const double tm2 = LIO_F(-1.666666666f) + CLYP3 * rom13;
    const double hp1 = hh1 * tm2 / dens;
    const double gp1 = fp1 * hh1 + hp1 * f1;
    const double fp2 = tm1 * 2.0 * f1 * (fp1 - LIO_F(0.6666666666f) * f1 / dens);
    const double tm3 = LIO_F(1.6666666666f) - CLYP3 * LIO_F(1.3333333333f) * rom13;
    const double hp2 = hp1 * tm2 / dens + hh1 * tm3 / (dens * dens);
    const double gp2 = fp2 * hh1 + 2.0 * fp1 * hp1 + hp2 * f1;
    const double term3 = -ALYP * (fp1 * dens + f1) - ALYP * BLYP * CF * (gp1 * dens + (double)(8.0f / 3.0f) * gg1) * rom53;
    const double term4 = (gp2 * dens * grad2 + gp1 * (3.0 * grad2 + 2.0 * dens * lap) + 4.0 * gg1 * lap) * ALYP * BLYP / 4.0;
    const double term5 =
        (3.0 * gp2 * dens * grad2 + gp1 * (5.0 * grad2 + 6.0 * dens * lap) + 4.0 * gg1 * lap) * ALYP * BLYP / 72.0;
    v = v + (term3 - term4 - term5);
  }
  o.v = v;
  return o;
}

// ----------------------------------------------------- PBE open shell (pbeOS_*.h)
// rho13 = cbrt(rho) of the spin-doubled density (pbeOS_exch.h:42-75 takes rho)
LIO_HD inline void pbe_exchange_spin(double rho13, double s, double u, double v, double& ex, double& vx) {
  const double AX = LIO_F(-0.738558766382022405884230032680836f);
  const double UM = LIO_F(0.2195149727645171f), UK = LIO_F(0.804f), UL = LIO_F(0.273028573090195f);
  const double exunif = AX * rho13;
  const double s2 = s * s, s3 = s * s2;
  const double p0 = 1.0 + UL * s2;
  const double fxpbe = 1.0 + UK - UK / p0;
  ex = exunif * fxpbe;
  const double Fs = 2.0 * UM / (p0 * p0);
  const double Fss = (-4.0 * UL * s * Fs) / p0;
  vx = exunif * (LIO_F43 * fxpbe - (u - LIO_F43 * s3) * Fss - v * Fs);
}

// cp, cm = cbrt(1 + zet), cbrt(1 - zet); every (1 +- zet)^(k/3) of the
// reference's pbeOS_corr.h is formed from them by products.
LIO_HD inline void pbe_correlation_spin(double rs, double zet, double cp, double cm, double t, double uu, double vv,
                                        double ww, double& ec, double& vc_a, double& vc_b, double& h,
                                        double& dvc_a, double& dvc_b) {
  const double GAMMA = LIO_F(0.03109069086965489503494086371273f);
  const double BETA = LIO_F(0.06672455060314922f);
  const double DELTA = BETA / GAMMA;
  const double ETA = LIO_F(0.000000000001f);
  const double rtrs = sqrt(rs);
  double EU, EURS, EP, EPRS, ALFM, ALFRSM;
  pw92_g(pw92_set(1), rtrs, EU, EURS);
  pw92_g(pw92_set(2), rtrs, EP, EPRS);
  pw92_g(pw92_set(3), rtrs, ALFM, ALFRSM);
  const double Z2 = zet * zet, Z4 = Z2 * Z2;
  const double zp = 1.0 + zet, zm = 1.0 - zet, zp2 = zp * zp, zm2 = zm * zm;
  const double ZET1 = zp * cp, ZET2 = zm * cm;  // (1 +- zet)^(4/3)
  const double GAM = LIO_GAM;
  const double F = (ZET1 + ZET2 - 2.0) / GAM;
  const double FZZ = 8.0 / (9.0 * GAM);
  ec = EU * (1.0 - F * Z4) + EP * F * Z4 - ALFM * F * (1.0 - Z4) / FZZ;
  const double ECRS = EURS * (1.0 - F * Z4) + EPRS * F * Z4 - ALFRSM * F * (1.0 - Z4) / FZZ;
  const double ZET3 = cp, ZET4 = cm;
  const double FZ = LIO_F43 * (ZET3 - ZET4) / GAM;
  const double ECZET = 4.0 * (Z2 * zet) * F * (EP - EU + ALFM / FZZ) + FZ * (Z4 * EP - Z4 * EU - (1.0 - Z4) * ALFM / FZZ);
  double COMM = ec - rs * ECRS / 3.0 - zet * ECZET;
  vc_a = COMM + ECZET;
  vc_b = COMM - ECZET;
  const double G = (cp * cp + cm * cm) / 2.0;  // ((1+zet)^(2/3) + (1-zet)^(2/3)) / 2
  const double G3 = G * G * G;
  const double PON = -ec / (G3 * GAMMA);
  const double B = DELTA / (exp(PON) - 1.0);
  const double B2 = B * B;
  const double T2 = t * t, T4 = T2 * T2;
  const double Q4 = 1.0 + B * T2;
  const double Q5 = 1.0 + B * T2 + B2 * T4;
  h = G3 * (BETA / DELTA) * log(1.0 + DELTA * Q4 * T2 / Q5);
  const double G4 = G3 * G;
  const double T6 = T4 * T2;
  const double rsthrd = rs / 3.0;
  const double GZ1 = pow(zp2 + ETA, LIO_FM16);
  const double GZ2 = pow(zm2 + ETA, LIO_FM16);
  const double GZ = (GZ1 - GZ2) / 3.0;
  const double FAC = DELTA / B + 1.0;
  const double BG = -3.0 * B2 * ec * FAC / (BETA * G4);
  const double BEC = B2 * FAC / (BETA * G3);
  const double Q8 = Q5 * Q5 + DELTA * Q4 * Q5 * T2;
  const double Q9 = 1.0 + 2.0 * B * T2;
  const double hB = -BETA * G3 * B * (T6 / Q8) * (2.0 + B * T2);
  const double hRS = -rsthrd * hB * BEC * ECRS;
  const double FACT0 = 2.0 * DELTA - 6.0 * B;
  const double FACT1 = Q5 * Q9 + Q4 * Q9 * Q9;
  const double hBT = 2.0 * BETA * G3 * T4 * ((Q4 * Q5 * FACT0 - DELTA * FACT1) / Q8) / Q8;
  const double hRST = rsthrd * T2 * hBT * BEC * ECRS;
  const double hz = 3.0 * GZ * h / G + hB * (BG * GZ + BEC * ECZET);
  const double hT = 2.0 * BETA * G3 * Q9 / Q8;
  const double hZT = 3.0 * GZ * hT / G + hBT * (BG * GZ + BEC * ECZET);
  const double FACT2 = Q4 * Q5 + B * T2 * (Q4 * Q9 + Q5);
  const double FACT3 = 2.0 * B * Q5 * Q9 + DELTA * FACT2;
  const double hTT = 4.0 * BETA * G3 * t * (2.0 * B / Q8 - ((Q9 / Q8) * FACT3) / Q8);
  COMM = h + hRS + hRST + T2 * hT / 6.0 + 7.0 * T2 * t * hTT / 6.0;
  const double PREF = hz - GZ * T2 * hT / G;
  const double FACT5 = GZ * (2.0 * hT + t * hTT) / G;
  COMM = COMM - PREF * zet - uu * hTT - vv * hT - ww * (hZT - FACT5);
  dvc_a = COMM + PREF;
  dvc_b = COMM - PREF;
}

struct GgaOpenOut {
  double ex, ec, va, vb;
};

LIO_HD inline void spin_scalars(const double g[3], const double h1[3], const double h2[3], double& dgrad,
                                double& delgrad, double& rlap) {
  const double gx2 = g[0] * g[0], gy2 = g[1] * g[1], gz2 = g[2] * g[2];
  const double grad2 = gx2 + gy2 + gz2;
  dgrad = sqrt(grad2);
  delgrad = (gx2 * h1[0] + 2.0 * g[0] * g[1] * h2[0] + 2.0 * g[1] * g[2] * h2[2] + 2.0 * g[0] * g[2] * h2[1] +
             gy2 * h1[1] + gz2 * h1[2]) /
            dgrad;
  rlap = h1[0] + h1[1] + h1[2];
}

// calc_ggaOS.h + pbeOS_main.h: alpha/beta densities -> ex, ec, v_alpha, v_beta
LIO_HD inline GgaOpenOut pbe_open(double da, double db, const double ga[3], const double gb[3],
                                  const double h1a[3], const double h1b[3], const double h2a[3],
                                  const double h2b[3]) {
  GgaOpenOut o{0.0, 0.0, 0.0, 0.0};
  const double MIN_RHO = 1e-18;
  if (!((da > MIN_RHO) || (db > MIN_RHO))) return o;
  const double PI_F = LIO_F(3.141592653589793238462643383279f);
  // cbrt(PI32) and cbrt(9 PI_F / 4) with PI32 = (double)(float)(3 pi^2) and
  // PI_F = (double)(float)pi, the values the C library's cbrt gives
  const double CBRT_PI32 = 0x1.8bfd4d9560ebcp+1, CBRT_ALPHA = 0x1.eb4df5835af6bp+0;
  double dgrad_a, delgrad_a, rlap_a, dgrad_b, delgrad_b, rlap_b;
  spin_scalars(ga, h1a, h2a, dgrad_a, delgrad_a, rlap_a);
  spin_scalars(gb, h1b, h2b, dgrad_b, delgrad_b, rlap_b);
  const double g[3] = {ga[0] + gb[0], ga[1] + gb[1], ga[2] + gb[2]};
  const double h1[3] = {h1a[0] + h1b[0], h1a[1] + h1b[1], h1a[2] + h1b[2]};
  const double h2[3] = {h2a[0] + h2b[0], h2a[1] + h2b[1], h2a[2] + h2b[2]};
  const double gx2 = g[0] * g[0], gy2 = g[1] * g[1], gz2 = g[2] * g[2];
  const double grad2 = gx2 + gy2 + gz2;
  const double dgrad = sqrt(grad2);
  const double delgrad = (gx2 * h1[0] + gy2 * h1[1] + gz2 * h1[2] +
                          2.0 * g[0] * g[1] * h2[0] + 2.0 * g[1] * g[2] * h2[2] + 2.0 * g[0] * g[2] * h2[1]) /
                         dgrad;
  // exchange by exact spin scaling: Ex[a,b] = (Ex[2a] + Ex[2b]) / 2
  double ex_a = 0.0, vx_a = 0.0, ex_b = 0.0, vx_b = 0.0;
  const double dens[2] = {da, db};
  const double dg[2] = {dgrad_a, dgrad_b}, dl[2] = {delgrad_a, delgrad_b}, lp[2] = {rlap_a, rlap_b};
  for (int sp = 0; sp < 2; sp++) {
    const double twodens = 2.0 * dens[sp];
    if (twodens > MIN_RHO) {
      const double twodens2 = twodens * twodens;
      const double td13 = cbrt(twodens);
      const double fk = CBRT_PI32 * td13;
      const double twofk = 2.0 * fk, twofk2 = twofk * twofk, twofk3 = twofk * twofk2;
      const double s = (2.0 * dg[sp]) / (twodens * twofk);
      const double v = (2.0 * lp[sp]) / (twodens * twofk2);
      const double u = (4.0 * dl[sp]) / (twodens2 * twofk3);
      if (sp == 0)
        pbe_exchange_spin(td13, s, u, v, ex_a, vx_a);
      else
        pbe_exchange_spin(td13, s, u, v, ex_b, vx_b);
    }
  }
  const double rho = da + db;
  o.ex = ex_a * (da / rho) + ex_b * (db / rho);
  o.va = vx_a;
  o.vb = vx_b;
  if (rho < (MIN_RHO * 1e5)) return o;
  const double zet = (da - db) / rho;
  const double cp = cbrt(1.0 + zet), cm = cbrt(1.0 - zet);
  const double gphi = (cp * cp + cm * cm) / 2.0;
  const double fk = CBRT_PI32 * cbrt(rho);
  const double rs = CBRT_ALPHA / fk;
  const double sk = sqrt(4.0 * fk / PI_F);
  const double twoksg = 2.0 * sk * gphi;
  const double t = dgrad / (twoksg * rho);
  const double uu = delgrad / (rho * rho * twoksg * twoksg * twoksg);
  const double vv = (rlap_a + rlap_b) / (rho * twoksg * twoksg);
  const double num = (dgrad_a * dgrad_a) - (dgrad_b * dgrad_b) - (zet * dgrad * dgrad);
  const double den = (rho * rho) * (twoksg * twoksg);
  const double ww = num / den;
  double ec, vc_a, vc_b, h, dvc_a, dvc_b;
  pbe_correlation_spin(rs, zet, cp, cm, t, uu, vv, ww, ec, vc_a, vc_b, h, dvc_a, dvc_b);
  o.ec = ec + h;
  o.va = vx_a + vc_a + dvc_a;
  o.vb = vx_b + vc_b + dvc_b;
  return o;
}

#undef LIO_F43
#undef LIO_F13
#undef LIO_FM16
#undef LIO_GAM
#undef LIO_F

}  // namespace xc
}  // namespace lio
