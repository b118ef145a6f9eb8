// physics.cuh -- per-face device arithmetic of the fully-coupled step:
// limiters, the seven convective flux schemes and the Roe flux Jacobian.
//
// Each function restates one reference routine (cited) in scalar per-face
// form; the surface-field algebra of the reference evaluates every term on
// every face, so the formulas below keep its branch-free masks (cf_*) and
// its operation order where that order is observable.  The flux schemes,
// limiters and vector helpers are templated on the scalar type: the step
// evaluates them in double, the discrete adjoint on forward-mode dual
// numbers (dual.cuh) to obtain their exact local Jacobians.
#pragma once

#include <math.h>

#include "dual.cuh"

namespace rdst {

constexpr double D_SMALL = 1.0e-15;    // foam SMALL
constexpr double D_VSMALL = 1.0e-300;  // foam VSMALL

// DST::pos/pos0/neg/neg0 (libraries/rhoDST/DST/DST.C:323-341)
template <typename T> __device__ __forceinline__ double dpos(const T& s) { return val(s) > 0 ? 1.0 : 0.0; }
template <typename T> __device__ __forceinline__ double dpos0(const T& s) { return val(s) >= 0 ? 1.0 : 0.0; }
template <typename T> __device__ __forceinline__ double dneg(const T& s) { return val(s) < 0 ? 1.0 : 0.0; }
template <typename T> __device__ __forceinline__ double dneg0(const T& s) { return val(s) <= 0 ? 1.0 : 0.0; }
template <typename T> __device__ __forceinline__ double fsgn(const T& s) { return val(s) >= 0 ? 1.0 : -1.0; }   // foam sign
template <typename T> __device__ __forceinline__ T sq(const T& x) { return x * x; }

template <typename T> struct Vec3 { T x, y, z; };
using V3 = Vec3<double>;
__device__ __forceinline__ V3 mk(double a, double b, double c) { V3 r; r.x = a; r.y = b; r.z = c; return r; }
template <typename T> __device__ __forceinline__ Vec3<T> mkv(const T& a, const T& b, const T& c) {
    Vec3<T> r; r.x = a; r.y = b; r.z = c; return r;
}
template <typename A, typename B>
__device__ __forceinline__ auto dot3(const Vec3<A>& a, const Vec3<B>& b) -> decltype(a.x * b.x) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename A> __device__ __forceinline__ A magSqr3(const Vec3<A>& a) { return dot3(a, a); }
template <typename A, typename B>
__device__ __forceinline__ auto add3(const Vec3<A>& a, const Vec3<B>& b) -> Vec3<decltype(a.x + b.x)> {
    return mkv(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <typename A, typename B>
__device__ __forceinline__ auto sub3(const Vec3<A>& a, const Vec3<B>& b) -> Vec3<decltype(a.x - b.x)> {
    return mkv(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename S, typename A>
__device__ __forceinline__ auto scl3(const S& s, const Vec3<A>& a) -> Vec3<decltype(s * a.x)> {
    return mkv(s * a.x, s * a.y, s * a.z);
}
template <typename A, typename S>
__device__ __forceinline__ auto div3(const Vec3<A>& a, const S& s) -> Vec3<decltype(a.x / s)> {
    return mkv(a.x / s, a.y / s, a.z / s);
}

enum { L_LINEAR = 0, L_UPWIND, L_OSPRE, L_VANLEER, L_MINMOD, L_VANALBADA, L_SUPERBEE, L_MUSCL, L_VENKAT };
enum { F_KURGANOV = 0, F_HLL, F_HLLC, F_HLLCP, F_AUSMPLUS, F_AUSMPLUSUP, F_AUSM };

// TVD limiters of foam's limitedSchemes, smooth ones clipped at 0 for r<0
template <typename T>
__device__ __forceinline__ T tvd_lim(int L, const T& r) {
    switch (L) {
        case L_OSPRE: { T rr = r * (r + 1.0); return fmax(1.5 * rr / (rr + 1.0), 0.0); }
        case L_VANLEER: return (r + fabs(r)) / (1.0 + fabs(r));
        case L_MINMOD: return fmax(fmin(fmin(r, 1.0), 2.0), 0.0);
        case L_VANALBADA: return fmax(r * (r + 1.0) / (r * r + 1.0), 0.0);
        case L_SUPERBEE: return fmax(fmax(fmin(2.0 * r, 1.0), fmin(r, 2.0)), 0.0);
        case L_MUSCL: return fmax(fmin(fmin(2.0 * r, 0.5 * r + 0.5), 2.0), 0.0);
        default: return T(1.0);
    }
}

// NVDTVD::r with the 1000x guard (r = 2 gradcf/gradf - 1)
template <typename T>
__device__ __forceinline__ T nvd_r(const T& gradcf, const T& gradf) {
    if (val(fabs(gradcf)) >= 1000 * val(fabs(gradf))) return T(2 * 1000 * fsgn(gradcf) * fsgn(gradf) - 1);
    return 2.0 * (gradcf / gradf) - 1.0;
}

// weights = lim*w + (1-lim)*pos(faceFlux), faceFlux = +1 (owner side) / -1
template <typename T>
__device__ __forceinline__ T side_w(int L, bool ownerSide, double w, const T& r) {
    if (L == L_LINEAR) return T(w);
    if (L == L_UPWIND) return T(ownerSide ? 1.0 : 0.0);
    T lim = tvd_lim(L, r);
    return lim * w + (1.0 - lim) * (ownerSide ? 1.0 : 0.0);
}

template <typename T> struct SideStateT { T rho; Vec3<T> rhoU; T rPsi, e, s; };
template <typename T> struct FFluxT { T phi; Vec3<T> phiUp; T phiEp; Vec3<T> Up; };
using SideState = SideStateT<double>;
using FFlux = FFluxT<double>;

// KurganovDST::computeFluxDST (KurganovDST.C:93-167)
template <typename T>
__device__ __forceinline__ FFluxT<T> flux_kurganov(const SideStateT<T>& o, const SideStateT<T>& n, V3 Sf, double magSf) {
    Vec3<T> U_own = div3(o.rhoU, o.rho), U_nei = div3(n.rhoU, n.rho);
    T rhoE_own = o.rho * (o.e + 0.5 * magSqr3(U_own));
    T rhoE_nei = n.rho * (n.e + 0.5 * magSqr3(U_nei));
    T p_own = o.rho * o.rPsi, p_nei = n.rho * n.rPsi;
    T phiv_own = dot3(U_own, Sf), phiv_nei = dot3(U_nei, Sf);
    T cSf_own = o.s * magSf, cSf_nei = n.s * magSf;
    T ap = fmax(fmax(phiv_own + cSf_own, phiv_nei + cSf_nei), 0.0);
    T am = fmin(fmin(phiv_own - cSf_own, phiv_nei - cSf_nei), 0.0);
    T a_own = ap / (ap - am);
    T aSf = am * a_own;
    T a_nei = 1.0 - a_own;
    phiv_own *= a_own;
    phiv_nei *= a_nei;
    T aphiv_own = phiv_own - aSf, aphiv_nei = phiv_nei + aSf;
    FFluxT<T> F;
    F.phi = aphiv_own * o.rho + aphiv_nei * n.rho;
    F.phiUp = add3(add3(scl3(aphiv_own, o.rhoU), scl3(aphiv_nei, n.rhoU)), scl3(a_own * p_own + a_nei * p_nei, Sf));
    F.phiEp = aphiv_own * (rhoE_own + p_own) + aphiv_nei * (rhoE_nei + p_nei) + aSf * p_own - aSf * p_nei;
    F.Up = add3(scl3(a_own, U_own), scl3(a_nei, U_nei));
    return F;
}

template <typename T>
struct HLLQ {
    Vec3<T> U_own, U_nei, UTilde;
    V3 normal;
    T E_own, E_nei, p_own, p_nei, H_own, H_nei, coefR, aTilde;
    T Uv_own, Uv_nei, S_own, S_nei;
};

// Roe-averaged wave speeds shared by HLL/HLLC/HLLCP (HLLDST.C:93-160)
template <typename T>
__device__ __forceinline__ HLLQ<T> hll_pro(const SideStateT<T>& o, const SideStateT<T>& n, V3 Sf, double magSf, double g) {
    HLLQ<T> q;
    q.U_own = div3(o.rhoU, o.rho);
    q.U_nei = div3(n.rhoU, n.rho);
    q.E_own = o.e + 0.5 * magSqr3(q.U_own);
    q.E_nei = n.e + 0.5 * magSqr3(q.U_nei);
    q.p_own = o.rho * o.rPsi;
    q.p_nei = n.rho * n.rPsi;
    q.H_own = q.E_own + q.p_own / o.rho;
    q.H_nei = q.E_nei + q.p_nei / n.rho;
    q.coefR = sqrt(fmax(D_VSMALL, n.rho) / fmax(D_VSMALL, o.rho));
    T HTilde = (q.coefR * q.H_nei + q.H_own) / (q.coefR + 1.0);
    q.UTilde = div3(add3(scl3(q.coefR, q.U_nei), q.U_own), q.coefR + 1.0);
    q.aTilde = sqrt((g - 1.0) * (HTilde - 0.5 * magSqr3(q.UTilde)));
    q.normal = div3(Sf, magSf);
    q.Uv_own = dot3(q.U_own, q.normal);
    q.Uv_nei = dot3(q.U_nei, q.normal);
    T UvTilde = dot3(q.UTilde, q.normal);
    q.S_own = fmin(q.Uv_own - o.s, UvTilde - q.aTilde);
    q.S_nei = fmax(q.Uv_nei + n.s, UvTilde + q.aTilde);
    return q;
}

// HLLDST::computeFluxDST (HLLDST.C:160-200)
template <typename T>
__device__ __forceinline__ FFluxT<T> flux_hll(const SideStateT<T>& o, const SideStateT<T>& n, V3 Sf, double magSf, double g) {
    HLLQ<T> q = hll_pro(o, n, Sf, magSf, g);
    double cf_own = dpos0(q.S_own);
    double cf_m = dneg(q.S_own) * dpos0(q.S_nei);
    double cf_nei = dneg(q.S_nei) * dneg(q.S_own);
    Vec3<T> rhoUPhi_own = add3(scl3(o.rho * q.Uv_own, q.U_own), scl3(q.p_own, q.normal));
    Vec3<T> rhoUPhi_nei = add3(scl3(n.rho * q.Uv_nei, q.U_nei), scl3(q.p_nei, q.normal));
    T dS = q.S_nei - q.S_own;
    FFluxT<T> F;
    F.phi = (cf_own * o.rho * q.Uv_own +
             cf_m * (q.S_nei * o.rho * q.Uv_own - q.S_own * n.rho * q.Uv_nei + q.S_own * q.S_nei * (n.rho - o.rho)) / dS +
             cf_nei * n.rho * q.Uv_nei) * magSf;
    Vec3<T> mid = scl3(1.0 / dS, add3(sub3(scl3(q.S_nei, rhoUPhi_own), scl3(q.S_own, rhoUPhi_nei)),
                                 scl3(q.S_own * q.S_nei, sub3(scl3(n.rho, q.U_nei), scl3(o.rho, q.U_own)))));
    F.phiUp = scl3(magSf, add3(add3(scl3(cf_own, rhoUPhi_own), scl3(cf_m, mid)), scl3(cf_nei, rhoUPhi_nei)));
    F.phiEp = (cf_own * o.rho * q.Uv_own * q.H_own +
               cf_m * (q.S_nei * o.rho * q.Uv_own * q.H_own - q.S_own * n.rho * q.Uv_nei * q.H_nei +
                       q.S_own * q.S_nei * (n.rho * q.E_nei - o.rho * q.E_own)) / dS +
               cf_nei * n.rho * q.Uv_nei * q.H_nei) * magSf;
    Vec3<T> Um = scl3(1.0 / dS, sub3(add3(sub3(scl3(q.S_nei, q.U_own), scl3(q.S_own, q.U_nei)), scl3(q.Uv_own, q.U_own)),
                              scl3(q.Uv_nei, q.U_nei)));
    F.Up = add3(add3(scl3(cf_own, q.U_own), scl3(cf_m, Um)), scl3(cf_nei, q.U_nei));
    return F;
}

// HLLCDST::computeFluxDST (HLLCDST.C:217-266); with pressure_sensor the
// HLLCP variant (HLLCPDST.C:228-311) with face sensor f.
template <typename T>
__device__ __forceinline__ FFluxT<T> flux_hllc(const SideStateT<T>& o, const SideStateT<T>& n, V3 Sf, double magSf, double g,
                                              bool pressure_sensor, const T& f) {
    HLLQ<T> q = hll_pro(o, n, Sf, magSf, g);
    const T S_own = q.S_own, S_nei = q.S_nei, Uv_own = q.Uv_own, Uv_nei = q.Uv_nei;
    T S_star = (q.p_nei - q.p_own + o.rho * Uv_own * (S_own - Uv_own) - n.rho * Uv_nei * (S_nei - Uv_nei)) /
                    (o.rho * (S_own - Uv_own) - n.rho * (S_nei - Uv_nei));
    double cf_own = dpos(S_own);
    double cf_m1 = dneg0(S_own) * dpos(S_star);
    double cf_m2 = dneg0(S_own) * dneg0(S_star) * dpos0(S_nei);
    double cf_nei = dneg0(S_own) * dneg0(S_star) * dneg(S_nei);
    T rhoE_own = o.rho * q.E_own, rhoE_nei = n.rho * q.E_nei;
    Vec3<T> rhoUPhi_own = add3(scl3(Uv_own, o.rhoU), scl3(q.p_own, q.normal));
    Vec3<T> rhoUPhi_nei = add3(scl3(Uv_nei, n.rhoU), scl3(q.p_nei, q.normal));
    T rhoEPhi_own = (rhoE_own + q.p_own) * Uv_own;
    T rhoEPhi_nei = (rhoE_nei + q.p_nei) * Uv_nei;
    T d1 = S_own - S_star, d2 = S_nei - S_star;
    FFluxT<T> F;
    if (!pressure_sensor) {
        T pstar_own = q.p_own + o.rho * (S_own - Uv_own) * (S_star - Uv_own);
        T pstar_nei = q.p_nei + n.rho * (S_nei - Uv_nei) * (S_star - Uv_nei);
        F.phi = (cf_own * o.rho * Uv_own + cf_m1 * S_star * o.rho * (S_own - Uv_own) / d1 +
                 cf_m2 * S_star * n.rho * (S_nei - Uv_nei) / d2 + cf_nei * n.rho * Uv_nei) * magSf;
        Vec3<T> m1 = scl3(1.0 / d1, add3(scl3(S_star, sub3(scl3(S_own, o.rhoU), rhoUPhi_own)), scl3(S_own * pstar_own, q.normal)));
        Vec3<T> m2 = scl3(1.0 / d2, add3(scl3(S_star, sub3(scl3(S_nei, n.rhoU), rhoUPhi_nei)), scl3(S_nei * pstar_nei, q.normal)));
        F.phiUp = scl3(magSf, add3(add3(add3(scl3(cf_own, rhoUPhi_own), scl3(cf_m1, m1)), scl3(cf_m2, m2)),
                                   scl3(cf_nei, rhoUPhi_nei)));
        F.phiEp = (cf_own * rhoEPhi_own + cf_m1 * S_star * (S_own * rhoE_own - rhoEPhi_own + S_own * pstar_own) / d1 +
                   cf_m2 * S_star * (S_nei * rhoE_nei - rhoEPhi_nei + S_nei * pstar_nei) / d2 +
                   cf_nei * rhoEPhi_nei) * magSf;
    } else {
        T Ma_own = Uv_own / o.s, Ma_nei = Uv_nei / n.s;
        T MaTilde = (q.coefR * Ma_nei + Ma_own) / (q.coefR + 1.0);
        T c_own = o.rho * (S_own - Uv_own), c_nei = n.rho * (S_nei - Uv_nei);
        T p_star = (c_nei * q.p_own - c_own * q.p_nei - c_own * c_nei * (Uv_own - Uv_nei)) / (c_nei - c_own);
        T theta = fmin(fmax(fabs(Ma_own), fabs(Ma_nei)), 1.0);
        T p_av = 0.5 * (q.p_own + q.p_nei);
        T p_ss = p_star * theta + (1.0 - theta) * p_av;
        T p_sss = f * p_ss + (1.0 - f) * p_star;
        T phip = (f - 1.0) * S_own * S_nei / (S_nei - S_own) / (1.0 + fabs(MaTilde)) * (q.p_nei - q.p_own) /
                      sq(q.aTilde);
        F.phi = (cf_own * o.rho * Uv_own + cf_m1 * (S_star * o.rho * (S_own - Uv_own) / d1 + phip) +
                 cf_m2 * (S_star * n.rho * (S_nei - Uv_nei) / d2 + phip) + cf_nei * n.rho * Uv_nei) * magSf;
        Vec3<T> m1 = add3(scl3(1.0 / d1, add3(scl3(S_star, sub3(scl3(S_own, o.rhoU), rhoUPhi_own)), scl3(S_own * p_sss, q.normal))),
                     scl3(phip, q.UTilde));
        Vec3<T> m2 = add3(scl3(1.0 / d2, add3(scl3(S_star, sub3(scl3(S_nei, n.rhoU), rhoUPhi_nei)), scl3(S_nei * p_sss, q.normal))),
                     scl3(phip, q.UTilde));
        F.phiUp = scl3(magSf, add3(add3(add3(scl3(cf_own, rhoUPhi_own), scl3(cf_m1, m1)), scl3(cf_m2, m2)),
                                   scl3(cf_nei, rhoUPhi_nei)));
        T kin = 0.5 * phip * magSqr3(q.UTilde);
        F.phiEp = (cf_own * rhoEPhi_own + cf_m1 * (S_star * (S_own * rhoE_own - rhoEPhi_own + S_own * p_star) / d1 + kin) +
                   cf_m2 * (S_star * (S_nei * rhoE_nei - rhoEPhi_nei + S_nei * p_star) / d2 + kin) +
                   cf_nei * rhoEPhi_nei) * magSf;
    }
    F.Up = add3(add3(add3(scl3(cf_own, q.U_own), scl3(cf_m1 * ((S_own - Uv_own) / d1), q.U_own)),
                     scl3(cf_m2 * ((S_nei - Uv_nei) / d2), q.U_nei)), scl3(cf_nei, q.U_nei));
    return F;
}

// AUSMPLDST (AUSMPLDST.C:127-217) and AUSMPLUPDST (AUSMPLUPDST.C:209-320)
template <typename T>
__device__ __forceinline__ FFluxT<T> flux_ausm_plus(const SideStateT<T>& o, const SideStateT<T>& n, V3 Sf, double magSf,
                                                   bool up, bool lowMach, double Mainf) {
    const double beta = 0.125, Kp = 0.25, Ku = 0.75, sigma = 1.0;
    Vec3<T> U_own = div3(o.rhoU, o.rho), U_nei = div3(n.rhoU, n.rho);
    V3 nrm = div3(Sf, magSf);
    T Uv_own = dot3(U_own, nrm), Uv_nei = dot3(U_nei, nrm);
    T rhoE_own = o.rho * (o.e + 0.5 * magSqr3(U_own));
    T rhoE_nei = n.rho * (n.e + 0.5 * magSqr3(U_nei));
    T p_own = o.rho * o.rPsi, p_nei = n.rho * n.rPsi;
    T a_own = o.s, a_nei = n.s, a12;
    T alpha = T(up ? 0.0 : 3.0 / 16.0);
    if (up) {
        a_own = sq(a_own) / fmax(a_own, Uv_own);
        a_nei = sq(a_nei) / fmax(a_nei, -Uv_nei);
        a12 = fmin(a_own, a_nei);
    } else {
        a12 = 0.5 * (a_own + a_nei);
    }
    T Ma_own = Uv_own / a12, Ma_nei = Uv_nei / a12;
    T Mmean2 = T(0.0), fa = T(0.0);
    if (up && lowMach) {
        Mmean2 = 0.5 * (sq(Uv_own) + sq(Uv_nei)) / sq(a12);
        T M0 = sqrt(fmin(1.0, fmax(Mmean2, sq(Mainf))));
        fa = M0 * (2.0 - M0);
        alpha = 3.0 / 16.0 * (-4.0 + 5.0 * sq(fa));
    }
    double in_o = dpos0(1.0 - fabs(Ma_own)), out_o = dpos0(-1.0 + fabs(Ma_own));
    double in_n = dpos0(1.0 - fabs(Ma_nei)), out_n = dpos0(-1.0 + fabs(Ma_nei));
    T Ma4_own = in_o * (0.25 * sq(Ma_own + 1.0)) * (1.0 - 16.0 * beta * (-0.25) * sq(Ma_own - 1.0)) +
                     out_o * fmax(Ma_own, 0.0);
    T P5_own = in_o * 0.25 * sq(Ma_own + 1.0) * (2.0 - Ma_own - 16.0 * alpha * Ma_own * (-0.25) * sq(Ma_own - 1.0)) +
                    out_o * dpos(Ma_own);
    T Ma4_nei = in_n * (-0.25) * sq(Ma_nei - 1.0) * (1.0 + 16.0 * beta * 0.25 * sq(Ma_nei + 1.0)) +
                     out_n * fmin(Ma_nei, 0.0);
    T P5_nei = in_n * (-0.25) * sq(Ma_nei - 1.0) * (-2.0 - Ma_nei + 16.0 * alpha * Ma_nei * 0.25 * sq(Ma_nei + 1.0)) +
                    out_n * dneg(Ma_nei);
    T Ma12 = Ma4_own + Ma4_nei;
    T P12 = P5_own * p_own + P5_nei * p_nei;
    if (up && lowMach) {
        T Mp = -Kp / fa * fmax(1.0 - sigma * Mmean2, 0.0) * (p_nei - p_own) / (0.5 * (o.rho + n.rho)) / sq(a12);
        T pu = -Ku * P5_own * P5_nei * (o.rho + n.rho) * a12 * fa * (Uv_own - Uv_nei);
        Ma12 += Mp;
        P12 += pu;
    }
    FFluxT<T> F;
    F.Up = add3(scl3(dpos(Ma12), U_own), scl3(dneg0(Ma12), U_nei));
    F.phi = Ma12 * a12 * (dpos(Ma12) * o.rho + dneg0(Ma12) * n.rho) * magSf;
    F.phiUp = add3(scl3(F.phi, F.Up), scl3(P12, Sf));
    T H_own = (rhoE_own + p_own) / o.rho, H_nei = (rhoE_nei + p_nei) / n.rho;
    F.phiEp = F.phi * (dpos(Ma12) * H_own + dneg0(Ma12) * H_nei);
    return F;
}

// Liou-Steffen AUSM (1993), not implemented in the reference
template <typename T>
__device__ __forceinline__ FFluxT<T> flux_ausm(const SideStateT<T>& o, const SideStateT<T>& n, V3 Sf, double magSf) {
    Vec3<T> U_own = div3(o.rhoU, o.rho), U_nei = div3(n.rhoU, n.rho);
    V3 nrm = div3(Sf, magSf);
    T Uv_own = dot3(U_own, nrm), Uv_nei = dot3(U_nei, nrm);
    T p_own = o.rho * o.rPsi, p_nei = n.rho * n.rPsi;
    T rhoE_own = o.rho * (o.e + 0.5 * magSqr3(U_own));
    T rhoE_nei = n.rho * (n.e + 0.5 * magSqr3(U_nei));
    T M_o = Uv_own / o.s, M_n = Uv_nei / n.s;
    T Mp = val(fabs(M_o)) <= 1 ? T(0.25 * sq(M_o + 1.0)) : T(0.5 * (M_o + fabs(M_o)));
    T Mm = val(fabs(M_n)) <= 1 ? T(-0.25 * sq(M_n - 1.0)) : T(0.5 * (M_n - fabs(M_n)));
    T Pp = val(fabs(M_o)) <= 1 ? T(0.25 * sq(M_o + 1.0) * (2.0 - M_o)) : T(0.5 * (1 + fsgn(M_o)));
    T Pm = val(fabs(M_n)) <= 1 ? T(0.25 * sq(M_n - 1.0) * (2.0 + M_n)) : T(0.5 * (1 - fsgn(M_n)));
    T M12 = Mp + Mm;
    double upw = dpos0(M12);
    FFluxT<T> F;
    T mdot = M12 * (upw * o.rho * o.s + (1 - upw) * n.rho * n.s) * magSf;
    F.phi = mdot;
    F.Up = add3(scl3(upw, U_own), scl3(1 - upw, U_nei));
    F.phiUp = add3(scl3(mdot, F.Up), scl3(Pp * p_own + Pm * p_nei, Sf));
    T H_own = (rhoE_own + p_own) / o.rho, H_nei = (rhoE_nei + p_nei) / n.rho;
    F.phiEp = mdot * (upw * H_own + (1 - upw) * H_nei);
    return F;
}

template <typename T>
__device__ __forceinline__ FFluxT<T> face_flux(int scheme, const SideStateT<T>& o, const SideStateT<T>& n, V3 Sf,
                                              double magSf, double g, const T& fsens, bool lowMach, double Mainf) {
    switch (scheme) {
        case F_KURGANOV: return flux_kurganov(o, n, Sf, magSf);
        case F_HLL: return flux_hll(o, n, Sf, magSf, g);
        case F_HLLC: return flux_hllc(o, n, Sf, magSf, g, false, T(1.0));
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
