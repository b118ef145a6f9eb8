// physics.cuh -- per-face device arithmetic of the fully-coupled step:
// limiters, the seven convective flux schemes and the Roe flux Jacobian.
//
// Each function restates one reference routine (cited) in scalar per-face
// form; the surface-field algebra of the reference evaluates every term on
// every face, so the formulas below keep its branch-free masks (cf_*) and
// its operation order where that order is observable.
#pragma once

#include <math.h>

namespace rdst {

constexpr double D_SMALL = 1.0e-15;    // foam SMALL
constexpr double D_VSMALL = 1.0e-300;  // foam VSMALL

// DST::pos/pos0/neg/neg0 (libraries/rhoDST/DST/DST.C:323-341)
__device__ __forceinline__ double dpos(double s) { return s > 0 ? 1.0 : 0.0; }
__device__ __forceinline__ double dpos0(double s) { return s >= 0 ? 1.0 : 0.0; }
__device__ __forceinline__ double dneg(double s) { return s < 0 ? 1.0 : 0.0; }
__device__ __forceinline__ double dneg0(double s) { return s <= 0 ? 1.0 : 0.0; }
__device__ __forceinline__ double fsgn(double s) { return s >= 0 ? 1.0 : -1.0; }   // foam sign
__device__ __forceinline__ double sq(double x) { return x * x; }

struct V3 { double x, y, z; };
__device__ __forceinline__ V3 mk(double a, double b, double c) { V3 r; r.x = a; r.y = b; r.z = c; return r; }
__device__ __forceinline__ double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double magSqr3(V3 a) { return dot3(a, a); }
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 scl3(double s, V3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ V3 div3(V3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }

enum { L_LINEAR = 0, L_UPWIND, L_OSPRE, L_VANLEER, L_MINMOD, L_VANALBADA, L_SUPERBEE, L_MUSCL, L_VENKAT };
enum { F_KURGANOV = 0, F_HLL, F_HLLC, F_HLLCP, F_AUSMPLUS, F_AUSMPLUSUP, F_AUSM };

// TVD limiters of foam's limitedSchemes, smooth ones clipped at 0 for r<0
__device__ __forceinline__ double tvd_lim(int L, double r) {
    switch (L) {
        case L_OSPRE: { double rr = r * (r + 1); return fmax(1.5 * rr / (rr + 1), 0.0); }
        case L_VANLEER: return (r + fabs(r)) / (1 + fabs(r));
        case L_MINMOD: return fmax(fmin(fmin(r, 1.0), 2.0), 0.0);
        case L_VANALBADA: return fmax(r * (r + 1) / (r * r + 1), 0.0);
        case L_SUPERBEE: return fmax(fmax(fmin(2 * r, 1.0), fmin(r, 2.0)), 0.0);
        case L_MUSCL: return fmax(fmin(fmin(2 * r, 0.5 * r + 0.5), 2.0), 0.0);
        default: return 1.0;
    }
}

// NVDTVD::r with the 1000x guard (r = 2 gradcf/gradf - 1)
__device__ __forceinline__ double nvd_r(double gradcf, double gradf) {
    if (fabs(gradcf) >= 1000 * fabs(gradf)) return 2 * 1000 * fsgn(gradcf) * fsgn(gradf) - 1;
    return 2 * (gradcf / gradf) - 1;
}

// weights = lim*w + (1-lim)*pos(faceFlux), faceFlux = +1 (owner side) / -1
__device__ __forceinline__ double side_w(int L, bool ownerSide, double w, double r) {
    if (L == L_LINEAR) return w;
    if (L == L_UPWIND) return ownerSide ? 1.0 : 0.0;
    double lim = tvd_lim(L, r);
    return lim * w + (1 - lim) * (ownerSide ? 1.0 : 0.0);
}

struct SideState { double rho; V3 rhoU; double rPsi, e, s; };
struct FFlux { double phi; V3 phiUp; double phiEp; V3 Up; };

// KurganovDST::computeFluxDST (KurganovDST.C:93-167)
__device__ __forceinline__ FFlux flux_kurganov(const SideState& o, const SideState& n, V3 Sf, double magSf) {
    V3 U_own = div3(o.rhoU, o.rho), U_nei = div3(n.rhoU, n.rho);
    double rhoE_own = o.rho * (o.e + 0.5 * magSqr3(U_own));
    double rhoE_nei = n.rho * (n.e + 0.5 * magSqr3(U_nei));
    double p_own = o.rho * o.rPsi, p_nei = n.rho * n.rPsi;
    double phiv_own = dot3(U_own, Sf), phiv_nei = dot3(U_nei, Sf);
    double cSf_own = o.s * magSf, cSf_nei = n.s * magSf;
    double ap = fmax(fmax(phiv_own + cSf_own, phiv_nei + cSf_nei), 0.0);
    double am = fmin(fmin(phiv_own - cSf_own, phiv_nei - cSf_nei), 0.0);
    double a_own = ap / (ap - am);
    double aSf = am * a_own;
    double a_nei = 1.0 - a_own;
    phiv_own *= a_own;
    phiv_nei *= a_nei;
    double aphiv_own = phiv_own - aSf, aphiv_nei = phiv_nei + aSf;
    FFlux F;
    F.phi = aphiv_own * o.rho + aphiv_nei * n.rho;
    F.phiUp = add3(add3(scl3(aphiv_own, o.rhoU), scl3(aphiv_nei, n.rhoU)), scl3(a_own * p_own + a_nei * p_nei, Sf));
    F.phiEp = aphiv_own * (rhoE_own + p_own) + aphiv_nei * (rhoE_nei + p_nei) + aSf * p_own - aSf * p_nei;
    F.Up = add3(scl3(a_own, U_own), scl3(a_nei, U_nei));
    return F;
}

struct HLLQ {
    V3 U_own, U_nei, normal, UTilde;
    double E_own, E_nei, p_own, p_nei, H_own, H_nei, coefR, aTilde;
    double Uv_own, Uv_nei, S_own, S_nei;
};

// Roe-averaged wave speeds shared by HLL/HLLC/HLLCP (HLLDST.C:93-160)
__device__ __forceinline__ HLLQ hll_pro(const SideState& o, const SideState& n, V3 Sf, double magSf, double g) {
    HLLQ q;
    q.U_own = div3(o.rhoU, o.rho);
    q.U_nei = div3(n.rhoU, n.rho);
    q.E_own = o.e + 0.5 * magSqr3(q.U_own);
    q.E_nei = n.e + 0.5 * magSqr3(q.U_nei);
    q.p_own = o.rho * o.rPsi;
    q.p_nei = n.rho * n.rPsi;
    q.H_own = q.E_own + q.p_own / o.rho;
    q.H_nei = q.E_nei + q.p_nei / n.rho;
    q.coefR = sqrt(fmax(D_VSMALL, n.rho) / fmax(D_VSMALL, o.rho));
    double HTilde = (q.coefR * q.H_nei + q.H_own) / (q.coefR + 1.0);
    q.UTilde = div3(add3(scl3(q.coefR, q.U_nei), q.U_own), q.coefR + 1.0);
    q.aTilde = sqrt((g - 1.0) * (HTilde - 0.5 * magSqr3(q.UTilde)));
    q.normal = div3(Sf, magSf);
    q.Uv_own = dot3(q.U_own, q.normal);
    q.Uv_nei = dot3(q.U_nei, q.normal);
    double UvTilde = dot3(q.UTilde, q.normal);
    q.S_own = fmin(q.Uv_own - o.s, UvTilde - q.aTilde);
    q.S_nei = fmax(q.Uv_nei + n.s, UvTilde + q.aTilde);
    return q;
}

// HLLDST::computeFluxDST (HLLDST.C:160-200)
__device__ __forceinline__ FFlux flux_hll(const SideState& o, const SideState& n, V3 Sf, double magSf, double g) {
    HLLQ q = hll_pro(o, n, Sf, magSf, g);
    double cf_own = dpos0(q.S_own);
    double cf_m = dneg(q.S_own) * dpos0(q.S_nei);
    double cf_nei = dneg(q.S_nei) * dneg(q.S_own);
    V3 rhoUPhi_own = add3(scl3(o.rho * q.Uv_own, q.U_own), scl3(q.p_own, q.normal));
    V3 rhoUPhi_nei = add3(scl3(n.rho * q.Uv_nei, q.U_nei), scl3(q.p_nei, q.normal));
    double dS = q.S_nei - q.S_own;
    FFlux F;
    F.phi = (cf_own * o.rho * q.Uv_own +
             cf_m * (q.S_nei * o.rho * q.Uv_own - q.S_own * n.rho * q.Uv_nei + q.S_own * q.S_nei * (n.rho - o.rho)) / dS +
             cf_nei * n.rho * q.Uv_nei) * magSf;
    V3 mid = scl3(1.0 / dS, add3(sub3(scl3(q.S_nei, rhoUPhi_own), scl3(q.S_own, rhoUPhi_nei)),
                                 scl3(q.S_own * q.S_nei, sub3(scl3(n.rho, q.U_nei), scl3(o.rho, q.U_own)))));
    F.phiUp = scl3(magSf, add3(add3(scl3(cf_own, rhoUPhi_own), scl3(cf_m, mid)), scl3(cf_nei, rhoUPhi_nei)));
    F.phiEp = (cf_own * o.rho * q.Uv_own * q.H_own +
               cf_m * (q.S_nei * o.rho * q.Uv_own * q.H_own - q.S_own * n.rho * q.Uv_nei * q.H_nei +
                       q.S_own * q.S_nei * (n.rho * q.E_nei - o.rho * q.E_own)) / dS +
               cf_nei * n.rho * q.Uv_nei * q.H_nei) * magSf;
    V3 Um = scl3(1.0 / dS, sub3(add3(sub3(scl3(q.S_nei, q.U_own), scl3(q.S_own, q.U_nei)), scl3(q.Uv_own, q.U_own)),
                              scl3(q.Uv_nei, q.U_nei)));
    F.Up = add3(add3(scl3(cf_own, q.U_own), scl3(cf_m, Um)), scl3(cf_nei, q.U_nei));
    return F;
}

// HLLCDST::computeFluxDST (HLLCDST.C:217-266); with pressure_sensor the
// HLLCP variant (HLLCPDST.C:228-311) with face sensor f.
__device__ __forceinline__ FFlux flux_hllc(const SideState& o, const SideState& n, V3 Sf, double magSf, double g,
                                           bool pressure_sensor, double f) {
    HLLQ q = hll_pro(o, n, Sf, magSf, g);
    const double S_own = q.S_own, S_nei = q.S_nei, Uv_own = q.Uv_own, Uv_nei = q.Uv_nei;
    double S_star = (q.p_nei - q.p_own + o.rho * Uv_own * (S_own - Uv_own) - n.rho * Uv_nei * (S_nei - Uv_nei)) /
                    (o.rho * (S_own - Uv_own) - n.rho * (S_nei - Uv_nei));
    double cf_own = dpos(S_own);
    double cf_m1 = dneg0(S_own) * dpos(S_star);
    double cf_m2 = dneg0(S_own) * dneg0(S_star) * dpos0(S_nei);
    double cf_nei = dneg0(S_own) * dneg0(S_star) * dneg(S_nei);
    double rhoE_own = o.rho * q.E_own, rhoE_nei = n.rho * q.E_nei;
    V3 rhoUPhi_own = add3(scl3(Uv_own, o.rhoU), scl3(q.p_own, q.normal));
    V3 rhoUPhi_nei = add3(scl3(Uv_nei, n.rhoU), scl3(q.p_nei, q.normal));
    double rhoEPhi_own = (rhoE_own + q.p_own) * Uv_own;
    double rhoEPhi_nei = (rhoE_nei + q.p_nei) * Uv_nei;
    double d1 = S_own - S_star, d2 = S_nei - S_star;
    FFlux F;
    if (!pressure_sensor) {
        double pstar_own = q.p_own + o.rho * (S_own - Uv_own) * (S_star - Uv_own);
        double pstar_nei = q.p_nei + n.rho * (S_nei - Uv_nei) * (S_star - Uv_nei);
        F.phi = (cf_own * o.rho * Uv_own + cf_m1 * S_star * o.rho * (S_own - Uv_own) / d1 +
                 cf_m2 * S_star * n.rho * (S_nei - Uv_nei) / d2 + cf_nei * n.rho * Uv_nei) * magSf;
        V3 m1 = scl3(1.0 / d1, add3(scl3(S_star, sub3(scl3(S_own, o.rhoU), rhoUPhi_own)), scl3(S_own * pstar_own, q.normal)));
        V3 m2 = scl3(1.0 / d2, add3(scl3(S_star, sub3(scl3(S_nei, n.rhoU), rhoUPhi_nei)), scl3(S_nei * pstar_nei, q.normal)));
        F.phiUp = scl3(magSf, add3(add3(add3(scl3(cf_own, rhoUPhi_own), scl3(cf_m1, m1)), scl3(cf_m2, m2)),
                                   scl3(cf_nei, rhoUPhi_nei)));
        F.phiEp = (cf_own * rhoEPhi_own + cf_m1 * S_star * (S_own * rhoE_own - rhoEPhi_own + S_own * pstar_own) / d1 +
                   cf_m2 * S_star * (S_nei * rhoE_nei - rhoEPhi_nei + S_nei * pstar_nei) / d2 +
                   cf_nei * rhoEPhi_nei) * magSf;
    } else {
        double Ma_own = Uv_own / o.s, Ma_nei = Uv_nei / n.s;
        double MaTilde = (q.coefR * Ma_nei + Ma_own) / (q.coefR + 1.0);
        double c_own = o.rho * (S_own - Uv_own), c_nei = n.rho * (S_nei - Uv_nei);
        double p_star = (c_nei * q.p_own - c_own * q.p_nei - c_own * c_nei * (Uv_own - Uv_nei)) / (c_nei - c_own);
        double theta = fmin(fmax(fabs(Ma_own), fabs(Ma_nei)), 1.0);
        double p_av = 0.5 * (q.p_own + q.p_nei);
        double p_ss = p_star * theta + (1.0 - theta) * p_av;
        double p_sss = f * p_ss + (1.0 - f) * p_star;
        double phip = (f - 1.0) * S_own * S_nei / (S_nei - S_own) / (1.0 + fabs(MaTilde)) * (q.p_nei - q.p_own) /
                      sq(q.aTilde);
        F.phi = (cf_own * o.rho * Uv_own + cf_m1 * (S_star * o.rho * (S_own - Uv_own) / d1 + phip) +
                 cf_m2 * (S_star * n.rho * (S_nei - Uv_nei) / d2 + phip) + cf_nei * n.rho * Uv_nei) * magSf;
        V3 m1 = add3(scl3(1.0 / d1, add3(scl3(S_star, sub3(scl3(S_own, o.rhoU), rhoUPhi_own)), scl3(S_own * p_sss, q.normal))),
                     scl3(phip, q.UTilde));
        V3 m2 = add3(scl3(1.0 / d2, add3(scl3(S_star, sub3(scl3(S_nei, n.rhoU), rhoUPhi_nei)), scl3(S_nei * p_sss, q.normal))),
                     scl3(phip, q.UTilde));
        F.phiUp = scl3(magSf, add3(add3(add3(scl3(cf_own, rhoUPhi_own), scl3(cf_m1, m1)), scl3(cf_m2, m2)),
                                   scl3(cf_nei, rhoUPhi_nei)));
        double kin = 0.5 * phip * magSqr3(q.UTilde);
        F.phiEp = (cf_own * rhoEPhi_own + cf_m1 * (S_star * (S_own * rhoE_own - rhoEPhi_own + S_own * p_star) / d1 + kin) +
                   cf_m2 * (S_star * (S_nei * rhoE_nei - rhoEPhi_nei + S_nei * p_star) / d2 + kin) +
                   cf_nei * rhoEPhi_nei) * magSf;
    }
    F.Up = add3(add3(add3(scl3(cf_own, q.U_own), scl3(cf_m1 * ((S_own - Uv_own) / d1), q.U_own)),
                     scl3(cf_m2 * ((S_nei - Uv_nei) / d2), q.U_nei)), scl3(cf_nei, q.U_nei));
    return F;
}

// AUSMPLDST (AUSMPLDST.C:127-217) and AUSMPLUPDST (AUSMPLUPDST.C:209-320)
__device__ __forceinline__ FFlux flux_ausm_plus(const SideState& o, const SideState& n, V3 Sf, double magSf, bool up,
                                                bool lowMach, double Mainf) {
    const double beta = 0.125, Kp = 0.25, Ku = 0.75, sigma = 1.0;
    V3 U_own = div3(o.rhoU, o.rho), U_nei = div3(n.rhoU, n.rho);
    V3 nrm = div3(Sf, magSf);
    double Uv_own = dot3(U_own, nrm), Uv_nei = dot3(U_nei, nrm);
    double rhoE_own = o.rho * (o.e + 0.5 * magSqr3(U_own));
    double rhoE_nei = n.rho * (n.e + 0.5 * magSqr3(U_nei));
    double p_own = o.rho * o.rPsi, p_nei = n.rho * n.rPsi;
    double a_own = o.s, a_nei = n.s, a12;
    double alpha = up ? 0.0 : 3.0 / 16.0;
    if (up) {
        a_own = sq(a_own) / fmax(a_own, Uv_own);
        a_nei = sq(a_nei) / fmax(a_nei, -Uv_nei);
        a12 = fmin(a_own, a_nei);
    } else {
        a12 = 0.5 * (a_own + a_nei);
    }
    double Ma_own = Uv_own / a12, Ma_nei = Uv_nei / a12;
    double Mmean2 = 0, fa = 0;
    if (up && lowMach) {
        Mmean2 = 0.5 * (sq(Uv_own) + sq(Uv_nei)) / sq(a12);
        double M0 = sqrt(fmin(1.0, fmax(Mmean2, sq(Mainf))));
        fa = M0 * (2.0 - M0);
        alpha = 3.0 / 16.0 * (-4.0 + 5.0 * sq(fa));
    }
    double in_o = dpos0(1.0 - fabs(Ma_own)), out_o = dpos0(-1.0 + fabs(Ma_own));
    double in_n = dpos0(1.0 - fabs(Ma_nei)), out_n = dpos0(-1.0 + fabs(Ma_nei));
    double Ma4_own = in_o * (0.25 * sq(Ma_own + 1.0)) * (1.0 - 16.0 * beta * (-0.25) * sq(Ma_own - 1.0)) +
                     out_o * fmax(Ma_own, 0.0);
    double P5_own = in_o * 0.25 * sq(Ma_own + 1.0) * (2.0 - Ma_own - 16.0 * alpha * Ma_own * (-0.25) * sq(Ma_own - 1.0)) +
                    out_o * dpos(Ma_own);
    double Ma4_nei = in_n * (-0.25) * sq(Ma_nei - 1.0) * (1.0 + 16.0 * beta * 0.25 * sq(Ma_nei + 1.0)) +
                     out_n * fmin(Ma_nei, 0.0);
    double P5_nei = in_n * (-0.25) * sq(Ma_nei - 1.0) * (-2.0 - Ma_nei + 16.0 * alpha * Ma_nei * 0.25 * sq(Ma_nei + 1.0)) +
                    out_n * dneg(Ma_nei);
    double Ma12 = Ma4_own + Ma4_nei;
    double P12 = P5_own * p_own + P5_nei * p_nei;
    if (up && lowMach) {
        double Mp = -Kp / fa * fmax(1.0 - sigma * Mmean2, 0.0) * (p_nei - p_own) / (0.5 * (o.rho + n.rho)) / sq(a12);
        double pu = -Ku * P5_own * P5_nei * (o.rho + n.rho) * a12 * fa * (Uv_own - Uv_nei);
        Ma12 += Mp;
        P12 += pu;
    }
    FFlux F;
    F.Up = add3(scl3(dpos(Ma12), U_own), scl3(dneg0(Ma12), U_nei));
    F.phi = Ma12 * a12 * (dpos(Ma12) * o.rho + dneg0(Ma12) * n.rho) * magSf;
    F.phiUp = add3(scl3(F.phi, F.Up), scl3(P12, Sf));
    double H_own = (rhoE_own + p_own) / o.rho, H_nei = (rhoE_nei + p_nei) / n.rho;
    F.phiEp = F.phi * (dpos(Ma12) * H_own + dneg0(Ma12) * H_nei);
    return F;
}

// Liou-Steffen AUSM (1993), not implemented in the reference
__device__ __forceinline__ FFlux flux_ausm(const SideState& o, const SideState& n, V3 Sf, double magSf) {
    V3 U_own = div3(o.rhoU, o.rho), U_nei = div3(n.rhoU, n.rho);
    V3 nrm = div3(Sf, magSf);
    double Uv_own = dot3(U_own, nrm), Uv_nei = dot3(U_nei, nrm);
    double p_own = o.rho * o.rPsi, p_nei = n.rho * n.rPsi;
    double rhoE_own = o.rho * (o.e + 0.5 * magSqr3(U_own));
    double rhoE_nei = n.rho * (n.e + 0.5 * magSqr3(U_nei));
    double M_o = Uv_own / o.s, M_n = Uv_nei / n.s;
    double Mp = fabs(M_o) <= 1 ? 0.25 * sq(M_o + 1) : 0.5 * (M_o + fabs(M_o));
    double Mm = fabs(M_n) <= 1 ? -0.25 * sq(M_n - 1) : 0.5 * (M_n - fabs(M_n));
    double Pp = fabs(M_o) <= 1 ? 0.25 * sq(M_o + 1) * (2 - M_o) : 0.5 * (1 + fsgn(M_o));
    double Pm = fabs(M_n) <= 1 ? 0.25 * sq(M_n - 1) * (2 + M_n) : 0.5 * (1 - fsgn(M_n));
    double M12 = Mp + Mm;
    double upw = dpos0(M12);
    FFlux F;
    double mdot = M12 * (upw * o.rho * o.s + (1 - upw) * n.rho * n.s) * magSf;
    F.phi = mdot;
    F.Up = add3(scl3(upw, U_own), scl3(1 - upw, U_nei));
    F.phiUp = add3(scl3(mdot, F.Up), scl3(Pp * p_own + Pm * p_nei, Sf));
    double H_own = (rhoE_own + p_own) / o.rho, H_nei = (rhoE_nei + p_nei) / n.rho;
    F.phiEp = mdot * (upw * H_own + (1 - upw) * H_nei);
    return F;
}

__device__ __forceinline__ FFlux face_flux(int scheme, const SideState& o, const SideState& n, V3 Sf, double magSf,
                                           double g, double fsens, bool lowMach, double Mainf) {
    switch (scheme) {
        case F_KURGANOV: return flux_kurganov(o, n, Sf, magSf);
        case F_HLL: return flux_hll(o, n, Sf, magSf, g);
        case F_HLLC: return flux_hllc(o, n, Sf, magSf, g, false, 1.0);
        case F_HLLCP: return flux_hllc(o, n, Sf, magSf, g, true, fsens);
        case F_AUSMPLUS: return flux_ausm_plus(o, n, Sf, magSf, false, false, 0.0);
        case F_AUSMPLUSUP: return flux_ausm_plus(o, n, Sf, magSf, true, lowMach, Mainf);
        default: return flux_ausm(o, n, Sf, magSf);
    }
}

// Roe<tensor5>::calcJ (Roe.C:247-272): Blazek (2001) A.7 flux Jacobian A(W).n
__device__ __forceinline__ void calcJ(V3 Uf, double gammaf, double phiJf, double a1f, V3 n, double J[25]) {
    const double U[3] = {Uf.x, Uf.y, Uf.z};
    const double N[3] = {n.x, n.y, n.z};
    double Un = dot3(Uf, n);
    J[0] = 0.0;
    for (int k = 0; k < 3; ++k) J[1 + k] = N[k];
    J[4] = 0.0;
    for (int k = 0; k < 3; ++k) {
        J[(1 + k) * 5 + 0] = phiJf * N[k] - U[k] * Un;
        for (int l = 0; l < 3; ++l) J[(1 + k) * 5 + 1 + l] = U[k] * N[l] + (k == l ? Un : 0.0) - (gammaf - 1) * (N[k] * U[l]);
        J[(1 + k) * 5 + 4] = (gammaf - 1) * N[k];
    }
    J[20] = Un * (phiJf - a1f);
    for (int l = 0; l < 3; ++l) J[21 + l] = a1f * N[l] - Un * (gammaf - 1) * U[l];
    J[24] = gammaf * Un;
}

}  // namespace rdst
