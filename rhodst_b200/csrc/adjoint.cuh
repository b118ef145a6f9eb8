// adjoint.cuh -- discrete adjoint of the steady residual (convective terms
// and, with transport options set, the viscous terms of calcFields at frozen
// turbulent viscosity).
//
// u = (dR/dW)^T v for the per-unit-volume residual R(W) of the step
// (reconstruction, Gauss gradients, Venkatakrishnan/TVD limiters, the seven
// convective flux schemes, all boundary conditions), matrix-free: nothing
// from the primal is stored but the cell records (W, prim, q, gradients,
// limiter values, boundary states).  The pass runs in reverse order of the
// residual:
//   k_adj_faces   per internal face: face states recomputed, flux VJP by
//                 forward-mode dual numbers (dF/d(owner side), dF/d(neighbour
//                 side)) applied to lambda_o - lambda_n, lambda = v / V;
//   k_adj_bfaces  per boundary face: VJP of the boundary flux;
//   k_adj_cells   per cell, gathering over its faces: reconstruction VJP
//                 (recomputed from the cell records), Venkatakrishnan and
//                 HLLCP-sensor VJP with records for the neighbour that holds
//                 the extremum;
//   k_adj_gather  per cell: Gauss-gradient transpose, neighbour records,
//                 VJP of the recon record q(W) -> W;
//   k_adj_bc      per boundary face: VJP of the boundary state (frozen
//                 in/outflow and sub/supersonic branches) -> the adjacent
//                 cell's W and the patch velocity values;
//   k_adj_finish  per cell: boundary contributions gathered.
// With the viscous terms, k_adj_visc_faces / k_adj_visc_bfaces run first (VJP
// of the face terms wrt the cell velocities, velocity gradients, muEff and
// the convective face velocity Up, whose bar feeds k_adj_faces/k_adj_bfaces),
// k_adj_visc_cells gathers the per-cell bars, and k_adj_gather transposes the
// Gauss gradient of U as well (muEff = mu(T) + frozen mu_t).
// Every kernel writes only its own face or cell: no atomics, deterministic.
// The adjoint of the reference's step has no counterpart in the reference.
#pragma once

#include "kernels.cuh"

namespace rdst {

constexpr int ADJ_FB = 16;   // per internal face: xbar owner side [7], neighbour side [7], fs bar
constexpr int ADJ_QB = 8;    // per cell: q bar [7], p bar
constexpr int ADJ_VF = 32;   // per internal face, viscous input bars: UP[3], UQ[3], gP[9], gQ[9], muP, muQ, Up[3]
constexpr int ADJ_VBF = 20;  // per boundary face, viscous input bars: Ub[3], UP[3], gP[9], mub, Up[3]

// prim (p, T, h, U) and rho of a cell from W, as the field update computes them
template <typename T>
__device__ __forceinline__ void adj_prim(const Thermo& th, const Bounds& bd, const T (&W)[5], T& rho, T& p, T& Tt,
                                         T& h, Vec3<T>& U) {
    rho = fmin(fmax(W[0], bd.rho_min), bd.rho_max);
    U = div3(mkv(W[1], W[2], W[3]), rho);
    T hh = (th.Cp / th.Cv) * (W[4] / rho - 0.5 * magSqr3(U));
    h = fmin(fmax(hh, th.Cp * bd.T_min), th.Cp * bd.T_max);
    Tt = h / th.Cp;
    p = fmin(fmax(rho * th.R * Tt, bd.p_min), bd.p_max);
}

// recon record (rho, rhoU, rPsi, e, s) from conserved and thermodynamic values
template <typename T>
__device__ __forceinline__ void adj_qrec(const Thermo& th, int use_c, const T& rho, const Vec3<T>& rhoU, const T& rhoE,
                                         const T& p, const T& Tt, const T& h, T (&q)[7]) {
    const double g = th.gamma;
    T rPsi = th.R * Tt;
    T s;
    if (use_c) s = sqrt(g * rPsi);
    else {
        T H = fmax(rhoE / rho, D_SMALL) + fmax(p / rho, D_SMALL);
        s = sqrt(2.0 * (g - 1.0) / (g + 1.0) * H);
    }
    q[0] = rho; q[1] = rhoU.x; q[2] = rhoU.y; q[3] = rhoU.z;
    q[4] = rPsi; q[5] = h - p / rho; q[6] = s;
}

template <int K>
__device__ __forceinline__ SideStateT<Dual<K>> adj_side(const SideState& s, int k0) {
    SideStateT<Dual<K>> r;
    r.rho = Dual<K>::seed(s.rho, k0);
    r.rhoU = mkv(Dual<K>::seed(s.rhoU.x, k0 + 1), Dual<K>::seed(s.rhoU.y, k0 + 2), Dual<K>::seed(s.rhoU.z, k0 + 3));
    r.rPsi = Dual<K>::seed(s.rPsi, k0 + 4);
    r.e = Dual<K>::seed(s.e, k0 + 5);
    r.s = Dual<K>::seed(s.s, k0 + 6);
    return r;
}

// sum_k Fbar_k dF_k
template <int K>
__device__ __forceinline__ double adj_fdot(const FFluxT<Dual<K>>& F, const double (&Fb)[5], int k) {
    return Fb[0] * F.phi.d[k] + Fb[1] * F.phiUp.x.d[k] + Fb[2] * F.phiUp.y.d[k] + Fb[3] * F.phiUp.z.d[k] +
           Fb[4] * F.phiEp.d[k];
}

// sum_j Upbar_j dUp_j (the viscous energy term's use of the face velocity)
template <int K>
__device__ __forceinline__ double adj_updot(const FFluxT<Dual<K>>& F, const double* Upb, int k) {
    return Upb ? Upb[0] * F.Up.x.d[k] + Upb[1] * F.Up.y.d[k] + Upb[2] * F.Up.z.d[k] : 0.0;
}

// ---------------------------------------------------------------- viscous
// VJP of visc_face per internal face: bars of its 29 inputs for the output
// bar of R_P -= (lap + tauS, sig) / V_P, R_Q += (...) / V_Q; forward mode in
// chunks of 8 inputs.
__global__ void __launch_bounds__(128) k_adj_visc_faces(DevMesh m, const double* __restrict__ q,
                                                        const double* __restrict__ prim, const double* __restrict__ gU,
                                                        const double* __restrict__ up, const double* __restrict__ v,
                                                        double* __restrict__ vfbar) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.Fi) return;
    const int P = m.own[f], Q = m.nei[f];
    const double w = m.w[f], dc = m.dc[f], magS = m.magSf[f];
    const V3 S = ldv3(m.Sf, m.Fi, f);
    const V3 kc = sub3(div3(S, magS), scl3(dc, ldv3(m.d, m.Fi, f)));
    const double VP = m.V[P], VQ = m.V[Q];
    double bo[7];
#pragma unroll
    for (int j = 0; j < 3; ++j) bo[j] = bo[3 + j] = v[5 * Q + 1 + j] / VQ - v[5 * P + 1 + j] / VP;
    bo[6] = v[5 * Q + 4] / VQ - v[5 * P + 4] / VP;
    double in[29];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        in[j] = prim[PW * P + 3 + j]; in[3 + j] = prim[PW * Q + 3 + j]; in[26 + j] = up[3 * f + j];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) { in[6 + k] = gU[9 * P + k]; in[15 + k] = gU[9 * Q + k]; }
    in[24] = q[QW * P + 7]; in[25] = q[QW * Q + 7];
    double* out = vfbar + ADJ_VF * f;
    using D = Dual<8>;
    for (int k0 = 0; k0 < 29; k0 += 8) {
        D UP[3], UQ[3], gP[9], gQ[9], Up[3], o[7];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            UP[j] = D::seed(in[j], j - k0); UQ[j] = D::seed(in[3 + j], 3 + j - k0);
            Up[j] = D::seed(in[26 + j], 26 + j - k0);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) { gP[k] = D::seed(in[6 + k], 6 + k - k0); gQ[k] = D::seed(in[15 + k], 15 + k - k0); }
        const D muP = D::seed(in[24], 24 - k0), muQ = D::seed(in[25], 25 - k0);
        visc_face(S, magS, w, dc, kc, UP, UQ, gP, gQ, muP, muQ, Up, o);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k0 + k >= 29) break;
            double a = 0.0;
#pragma unroll
            for (int t = 0; t < 7; ++t) a += bo[t] * o[t].d[k];
            out[k0 + k] = a;
        }
    }
    out[29] = out[30] = out[31] = 0.0;
}

// VJP of visc_bface per boundary face (19 inputs)
__global__ void k_adj_visc_bfaces(DevMesh m, const double* __restrict__ qb, const double* __restrict__ prim,
                                  const double* __restrict__ gU, const double* __restrict__ bs,
                                  const double* __restrict__ bup, const double* __restrict__ v,
                                  double* __restrict__ vbbar) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const int P = m.bcell[b];
    const double* B = bs + BW * b;
    const double VP = m.V[P];
    double bo[7];
#pragma unroll
    for (int j = 0; j < 3; ++j) bo[j] = bo[3 + j] = -v[5 * P + 1 + j] / VP;
    bo[6] = -v[5 * P + 4] / VP;
    double in[19];
#pragma unroll
    for (int j = 0; j < 3; ++j) { in[j] = B[12 + j]; in[3 + j] = prim[PW * P + 3 + j]; in[16 + j] = bup[3 * b + j]; }
#pragma unroll
    for (int k = 0; k < 9; ++k) in[6 + k] = gU[9 * P + k];
    in[15] = qb[QW * b + 7];
    const V3 S = ldv3(m.bSf, m.NB, b);
    const double magS = m.bmagSf[b], dc = m.bdc[b];
    double* out = vbbar + ADJ_VBF * b;
    using D = Dual<8>;
    for (int k0 = 0; k0 < 19; k0 += 8) {
        D Ub[3], UP[3], gP[9], Up[3], o[7];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Ub[j] = D::seed(in[j], j - k0); UP[j] = D::seed(in[3 + j], 3 + j - k0); Up[j] = D::seed(in[16 + j], 16 + j - k0);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) gP[k] = D::seed(in[6 + k], 6 + k - k0);
        const D mub = D::seed(in[15], 15 - k0);
        visc_bface(S, magS, dc, Ub, UP, gP, mub, Up, o);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k0 + k >= 19) break;
            double a = 0.0;
#pragma unroll
            for (int t = 0; t < 7; ++t) a += bo[t] * o[t].d[k];
            out[k0 + k] = a;
        }
    }
    out[19] = 0.0;
}

// Per cell: the viscous input bars of its faces gathered -- velocity
// gradient bar gUbar (9) and the direct bars of its velocity and muEff
// (ucbar: U[3], mu).
__global__ void k_adj_visc_cells(DevMesh m, const double* __restrict__ vfbar, const double* __restrict__ vbbar,
                                 double* __restrict__ gUbar, double* __restrict__ ucbar) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m.N) return;
    double gb[9], ub[4] = {0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 9; ++k) gb[k] = 0.0;
    for (int kk = m.cf_start[j]; kk < m.cf_start[j + 1]; ++kk) {
        const int code = m.cf_list[kk];
        if (code < m.Fi) {
            const double* r = vfbar + ADJ_VF * code;
            const bool own = m.own[code] == j;
            const int u0 = own ? 0 : 3, g0 = own ? 6 : 15;
#pragma unroll
            for (int t = 0; t < 3; ++t) ub[t] += r[u0 + t];
#pragma unroll
            for (int k = 0; k < 9; ++k) gb[k] += r[g0 + k];
            ub[3] += r[own ? 24 : 25];
        } else {
            const double* r = vbbar + ADJ_VBF * (code - m.Fi);
#pragma unroll
            for (int t = 0; t < 3; ++t) ub[t] += r[3 + t];
#pragma unroll
            for (int k = 0; k < 9; ++k) gb[k] += r[6 + k];
        }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) gUbar[9 * j + k] = gb[k];
#pragma unroll
    for (int t = 0; t < 4; ++t) ucbar[4 * j + t] = ub[t];
}

// ---------------------------------------------------------------- faces
__global__ void __launch_bounds__(128) k_adj_faces(DevMesh m, Thermo th, int scheme, int lr, int lu, int lt,
                                                   int lowMach, double Mainf, const double* __restrict__ q,
                                                   const double* __restrict__ g, const double* __restrict__ psi,
                                                   const double* __restrict__ fcell, const double* __restrict__ v,
                                                   const double* __restrict__ vfbar, double* __restrict__ fbar) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.Fi) return;
    const double* Upb = vfbar ? vfbar + ADJ_VF * f + 26 : nullptr;
    const int o = m.own[f], n = m.nei[f];
    const double wf = m.w[f];
    const V3 S = ldv3(m.Sf, m.Fi, f);
    const double magS = m.magSf[f];
    SideState so, sn;
    face_recon(m, f, lr, lu, lt, q, g, psi, so, sn);
    double Fb[5];
    const double Vo = m.V[o], Vn = m.V[n];
#pragma unroll
    for (int k = 0; k < 5; ++k) Fb[k] = v[5 * o + k] / Vo - v[5 * n + k] / Vn;
    double fs = 1.0;
    if (scheme == F_HLLCP) fs = wf * pow(fcell[o], 3.0) + (1 - wf) * pow(fcell[n], 3.0);
    double* out = fbar + ADJ_FB * f;
    {   // owner side and the HLLCP sensor
        using D = Dual<8>;
        const SideStateT<D> a = adj_side<8>(so, 0);
        SideStateT<D> b;
        b.rho = D(sn.rho); b.rhoU = mkv(D(sn.rhoU.x), D(sn.rhoU.y), D(sn.rhoU.z));
        b.rPsi = D(sn.rPsi); b.e = D(sn.e); b.s = D(sn.s);
        const FFluxT<D> F = face_flux(scheme, a, b, S, magS, th.gamma, D::seed(fs, 7), lowMach != 0, Mainf);
#pragma unroll
        for (int k = 0; k < 7; ++k) out[k] = adj_fdot(F, Fb, k) + adj_updot(F, Upb, k);
        out[14] = adj_fdot(F, Fb, 7) + adj_updot(F, Upb, 7);
    }
    {   // neighbour side
        using D = Dual<7>;
        SideStateT<D> a;
        a.rho = D(so.rho); a.rhoU = mkv(D(so.rhoU.x), D(so.rhoU.y), D(so.rhoU.z));
        a.rPsi = D(so.rPsi); a.e = D(so.e); a.s = D(so.s);
        const SideStateT<D> b = adj_side<7>(sn, 0);
        const FFluxT<D> F = face_flux(scheme, a, b, S, magS, th.gamma, D(fs), lowMach != 0, Mainf);
#pragma unroll
        for (int k = 0; k < 7; ++k) out[7 + k] = adj_fdot(F, Fb, k) + adj_updot(F, Upb, k);
    }
    out[15] = 0.0;
}

// boundary faces: F(qb, qb), both sides carry the boundary record
__global__ void k_adj_bfaces(DevMesh m, Thermo th, int scheme, int lowMach, double Mainf,
                             const double* __restrict__ qb, const double* __restrict__ v,
                             const double* __restrict__ vbbar, double* __restrict__ qbbar) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const double* Upb = vbbar ? vbbar + ADJ_VBF * b + 16 : nullptr;
    using D = Dual<7>;
    const double* qq = qb + QW * b;
    SideState s;
    s.rho = qq[0]; s.rhoU = mk(qq[1], qq[2], qq[3]); s.rPsi = qq[4]; s.e = qq[5]; s.s = qq[6];
    const SideStateT<D> a = adj_side<7>(s, 0);
    const FFluxT<D> F = face_flux(scheme, a, a, ldv3(m.bSf, m.NB, b), m.bmagSf[b], th.gamma, D(1.0), lowMach != 0, Mainf);
    const int c = m.bcell[b];
    double Fb[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) Fb[k] = v[5 * c + k] / m.V[c];
    double* out = qbbar + ADJ_QB * b;
#pragma unroll
    for (int k = 0; k < 7; ++k) out[k] = adj_fdot(F, Fb, k) + adj_updot(F, Upb, k);
    out[7] = 0.0;
}

// ---------------------------------------------------------------- cells
// Scalar limited reconstruction with the projected gradients aP = d.gP,
// aN = d.gN as inputs (same arithmetic as recon_scalar).
template <typename T>
__device__ __forceinline__ void adj_recon_scalar(int L, const T& xP, const T& xN, const T& aP, const T& aN, double w,
                                                 T& xo, T& xn) {
    T ro = T(0.0), rn = T(0.0);
    if (L != L_LINEAR && L != L_UPWIND) {
        T gradf = xN - xP;
        ro = nvd_r(aP, gradf);
        rn = nvd_r(aN, gradf);
    }
    T wo = side_w(L, true, w, ro), wn = side_w(L, false, w, rn);
    xo = wo * xP + (1.0 - wo) * xN;
    xn = wn * xP + (1.0 - wn) * xN;
}

// Venkatakrishnan phi(dm, d2) of k_grad
template <typename T>
__device__ __forceinline__ T adj_venkat_phi(const T& dm, const T& d2, double eps2) {
    return ((dm * dm + eps2) * d2 + 2.0 * d2 * d2 * dm) / (dm * dm + 2.0 * d2 * d2 + dm * d2 + eps2) / d2;
}

// Per cell i: reconstruction VJP of its faces (cell i's share), then the
// Venkatakrishnan and HLLCP-sensor VJP.  Outputs qbar (q bar, p bar),
// gbar (gradient bar, 21), and records of the contributions that belong to
// a neighbour (the cell or boundary face that holds the max/min):
// vrec_idx (>= 0 cell, <= -2 boundary face -2-b, -1 none) / vrec_val per
// field, hrec_idx / hrec_val for the HLLCP pressure ratio.
__global__ void __launch_bounds__(128) k_adj_cells(DevMesh m, int scheme, int lr, int lu, int lt, int venkat_mask,
                                                   double venkat_K, const double* __restrict__ q,
                                                   const double* __restrict__ qb, const double* __restrict__ g,
                                                   const double* __restrict__ psi, const double* __restrict__ fcell,
                                                   const double* __restrict__ prim, const double* __restrict__ fbar,
                                                   double* __restrict__ qbar, double* __restrict__ gbar,
                                                   int* __restrict__ vrec_idx, double* __restrict__ vrec_val,
                                                   int* __restrict__ hrec_idx, double* __restrict__ hrec_val) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    double qa[7] = {0, 0, 0, 0, 0, 0, 0}, ga[21], pa[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 21; ++k) ga[k] = 0.0;
    double fca = 0.0;   // fcell bar
    const int Ls[7] = {lr, lu, lu, lu, lt, lt, lt};
    const bool venk = lr == L_VENKAT || lu == L_VENKAT || lt == L_VENKAT;
    const bool lim = (lr > L_UPWIND) || (lu > L_UPWIND) || (lt > L_UPWIND);
    const int k0 = m.cf_start[i], k1 = m.cf_start[i + 1];
    for (int kk = k0; kk < k1; ++kk) {
        const int code = m.cf_list[kk];
        if (code >= m.Fi) continue;
        const int f = code, o = m.own[f], n = m.nei[f];
        const bool own = (o == i);
        const double wf = m.w[f];
        const double* xb = fbar + ADJ_FB * f;   // [0,7) owner side, [7,14) neighbour side, 14 fs
        const double* qo = q + QW * o;
        const double* qn = q + QW * n;
        if (venk) {
            const V3 Cf = ldv3(m.Cf, m.Fi, f);
            const V3 dI = sub3(Cf, ldv3(m.C, m.N, i));
            for (int j = 0; j < 7; ++j) {
                if (Ls[j] == L_VENKAT) {
                    // x_side = q_i + psi_i (d_i . g_i): only cell i's own side
                    const double xbj = own ? xb[j] : xb[7 + j];
                    const double* gi = g + GW * i + 3 * j;
                    const double pj = psi[QW * i + j];
                    qa[j] += xbj;
                    pa[j] += xbj * (dI.x * gi[0] + dI.y * gi[1] + dI.z * gi[2]);
                    ga[3 * j] += xbj * pj * dI.x; ga[3 * j + 1] += xbj * pj * dI.y; ga[3 * j + 2] += xbj * pj * dI.z;
                } else {
                    // linear / upwind: constant side weights
                    const double wo = side_w(Ls[j], true, wf, 0.0), wn = side_w(Ls[j], false, wf, 0.0);
                    qa[j] += own ? (xb[j] * wo + xb[7 + j] * wn) : (xb[j] * (1 - wo) + xb[7 + j] * (1 - wn));
                }
            }
        } else {
            const V3 d = ldv3(m.d, m.Fi, f);
            const double* gP = g + GW * o;
            const double* gN = g + GW * n;
            // scalar fields 0, 4, 5, 6
            const int sf[4] = {0, 4, 5, 6};
            for (int t = 0; t < 4; ++t) {
                const int j = sf[t];
                using D = Dual<4>;
                const double aP = lim ? dot3(d, mk(gP[3 * j], gP[3 * j + 1], gP[3 * j + 2])) : 0.0;
                const double aN = lim ? dot3(d, mk(gN[3 * j], gN[3 * j + 1], gN[3 * j + 2])) : 0.0;
                D xo, xn;
                adj_recon_scalar(Ls[j], D::seed(qo[j], 0), D::seed(qn[j], 1), D::seed(aP, 2), D::seed(aN, 3), wf, xo, xn);
                const double bo = xb[j], bn = xb[7 + j];
                if (own) {
                    qa[j] += bo * xo.d[0] + bn * xn.d[0];
                    const double ab = bo * xo.d[2] + bn * xn.d[2];
                    if (lim) { ga[3 * j] += ab * d.x; ga[3 * j + 1] += ab * d.y; ga[3 * j + 2] += ab * d.z; }
                } else {
                    qa[j] += bo * xo.d[1] + bn * xn.d[1];
                    const double ab = bo * xo.d[3] + bn * xn.d[3];
                    if (lim) { ga[3 * j] += ab * d.x; ga[3 * j + 1] += ab * d.y; ga[3 * j + 2] += ab * d.z; }
                }
            }
            // rhoU with the vector limiter
            {
                using D = Dual<12>;
                const int base = own ? 0 : 3;   // xP / xN seeds
                Vec3<D> xP = mkv(D::seed(qo[1], 0), D::seed(qo[2], 1), D::seed(qo[3], 2));
                Vec3<D> xN = mkv(D::seed(qn[1], 3), D::seed(qn[2], 4), D::seed(qn[3], 5));
                D ro = D(0.0), rn = D(0.0);
                if (lu > L_UPWIND) {
                    Vec3<D> gradfV = sub3(xN, xP);
                    D gradf = dot3(gradfV, gradfV);
                    Vec3<D> dgP = mkv(D::seed(d.x * gP[3] + d.y * gP[4] + d.z * gP[5], 6),
                                      D::seed(d.x * gP[6] + d.y * gP[7] + d.z * gP[8], 7),
                                      D::seed(d.x * gP[9] + d.y * gP[10] + d.z * gP[11], 8));
                    Vec3<D> dgN = mkv(D::seed(d.x * gN[3] + d.y * gN[4] + d.z * gN[5], 9),
                                      D::seed(d.x * gN[6] + d.y * gN[7] + d.z * gN[8], 10),
                                      D::seed(d.x * gN[9] + d.y * gN[10] + d.z * gN[11], 11));
                    ro = nvd_r(dot3(gradfV, dgP), gradf);
                    rn = nvd_r(dot3(gradfV, dgN), gradf);
                }
                D wo = side_w(lu, true, wf, ro), wn = side_w(lu, false, wf, rn);
                Vec3<D> xo = add3(scl3(wo, xP), scl3(1.0 - wo, xN));
                Vec3<D> xn = add3(scl3(wn, xP), scl3(1.0 - wn, xN));
                const double bo[3] = {xb[1], xb[2], xb[3]}, bn[3] = {xb[8], xb[9], xb[10]};
                auto vjp = [&](int k) {
                    return bo[0] * xo.x.d[k] + bo[1] * xo.y.d[k] + bo[2] * xo.z.d[k] + bn[0] * xn.x.d[k] +
                           bn[1] * xn.y.d[k] + bn[2] * xn.z.d[k];
                };
                for (int c = 0; c < 3; ++c) qa[1 + c] += vjp(base + c);
                if (lu > L_UPWIND) {
                    const int gb = own ? 6 : 9;
                    for (int c = 0; c < 3; ++c) {
                        const double ab = vjp(gb + c);
                        ga[3 * (1 + c)] += ab * d.x; ga[3 * (1 + c) + 1] += ab * d.y; ga[3 * (1 + c) + 2] += ab * d.z;
                    }
                }
            }
        }
        if (scheme == F_HLLCP) {
            // fs = w fo^3 + (1-w) fn^3
            const double fi = fcell[i];
            fca += xb[14] * (own ? wf : 1 - wf) * 3.0 * fi * fi;
        }
    }
    // ---- Venkatakrishnan: psi_i = min_f phi(dmax|dmin, g_i . (Cf - C_i)), start 1
    for (int j = 0; j < 7; ++j) {
        vrec_idx[7 * i + j] = -1;
        vrec_val[7 * i + j] = 0.0;
    }
    if (venkat_mask) {
        const double Vi = m.V[i];
        const double eps2 = pow(venkat_K * cbrt(Vi), 3.0);
        const V3 Ci = ldv3(m.C, m.N, i);
        const double* qi = q + QW * i;
        for (int j = 0; j < 7; ++j) {
            if (!((venkat_mask >> j) & 1) || pa[j] == 0.0) continue;
            const double x = qi[j];
            double mx = x, mn = x;
            int imx = -1, imn = -1;
            for (int kk = k0; kk < k1; ++kk) {
                const int code = m.cf_list[kk];
                double xo;
                int id;
                if (code < m.Fi) { const int o = m.own[code]; id = (o == i ? m.nei[code] : o); xo = q[QW * id + j]; }
                else { id = -2 - (code - m.Fi); xo = qb[QW * (code - m.Fi) + j]; }
                if (xo > mx) { mx = xo; imx = id; }
                if (xo < mn) { mn = xo; imn = id; }
            }
            const double dmax = mx - x, dmin = mn - x;
            const V3 gj = mk(g[GW * i + 3 * j], g[GW * i + 3 * j + 1], g[GW * i + 3 * j + 2]);
            double p = 1.0;
            int kbest = -1;
            for (int kk = k0; kk < k1; ++kk) {
                const int code = m.cf_list[kk];
                const V3 Cf = code < m.Fi ? ldv3(m.Cf, m.Fi, code) : ldv3(m.bCf, m.NB, code - m.Fi);
                const double d2 = dot3(gj, sub3(Cf, Ci));
                double ph;
                if (d2 > 0) ph = adj_venkat_phi(dmax, d2, eps2);
                else if (d2 < 0) ph = adj_venkat_phi(dmin, d2, eps2);
                else ph = 1.0;
                if (ph < p) { p = ph; kbest = kk; }
            }
            if (kbest < 0) continue;
            const int code = m.cf_list[kbest];
            const V3 Cf = code < m.Fi ? ldv3(m.Cf, m.Fi, code) : ldv3(m.bCf, m.NB, code - m.Fi);
            const V3 dC = sub3(Cf, Ci);
            const double d2 = dot3(gj, dC);
            if (d2 == 0.0) continue;
            const bool up = d2 > 0;
            using D = Dual<2>;
            const D ph = adj_venkat_phi(D::seed(up ? dmax : dmin, 0), D::seed(d2, 1), eps2);
            const double pb = pa[j];
            const double b_dm = pb * ph.d[0], b_d2 = pb * ph.d[1];
            ga[3 * j] += b_d2 * dC.x; ga[3 * j + 1] += b_d2 * dC.y; ga[3 * j + 2] += b_d2 * dC.z;
            const int ext = up ? imx : imn;
            if (ext != -1) {
                // dm = q_ext - q_i
                qa[j] -= b_dm;
                vrec_idx[7 * i + j] = ext;
                vrec_val[7 * i + j] = b_dm;
            }
        }
    }
    // ---- HLLCP sensor: fcell_i = min(1, min_k min(p_i/p_k, p_k/p_i))
    double pbar = 0.0;
    hrec_idx[i] = -1;
    hrec_val[i] = 0.0;
    if (scheme == F_HLLCP && fca != 0.0) {
        const double pi = prim[PW * i];
        double best = 1.0;
        int kb = -1, which = 0;
        for (int kk = k0; kk < k1; ++kk) {
            const int code = m.cf_list[kk];
            if (code >= m.Fi) continue;
            const int o = m.own[code];
            const int k = (o == i ? m.nei[code] : o);
            const double pk = prim[PW * k];
            const double a = pi / pk, b = pk / pi;
            const double r = fmin(a, b);
            if (r < best) { best = r; kb = k; which = (a <= b) ? 0 : 1; }
        }
        if (kb >= 0) {
            const double pk = prim[PW * kb];
            double dpi, dpk;
            if (which == 0) { dpi = 1.0 / pk; dpk = -pi / (pk * pk); }
            else { dpi = -pk / (pi * pi); dpk = 1.0 / pi; }
            pbar += fca * dpi;
            hrec_idx[i] = kb;
            hrec_val[i] = fca * dpk;
        }
    }
    double* qo = qbar + ADJ_QB * i;
#pragma unroll
    for (int j = 0; j < 7; ++j) qo[j] = qa[j];
    qo[7] = pbar;
    double* go = gbar + GW * i;
#pragma unroll
    for (int k = 0; k < 21; ++k) go[k] = ga[k];
}

// Per cell j: Gauss-gradient transpose over its faces, neighbour records,
// then the VJP of the recon record q(W_j) (and of p) to W_j.  Boundary faces
// of j receive their gradient and record shares in qbbar (only cell j
// writes them).
__global__ void __launch_bounds__(128) k_adj_gather(DevMesh m, Thermo th, Bounds bd, Transport tr, int use_c,
                                                    const double* __restrict__ W, const double* __restrict__ gbar,
                                                    const double* __restrict__ qbar, const int* __restrict__ vrec_idx,
                                                    const double* __restrict__ vrec_val,
                                                    const int* __restrict__ hrec_idx,
                                                    const double* __restrict__ hrec_val,
                                                    const double* __restrict__ gUbar, const double* __restrict__ ucbar,
                                                    double* __restrict__ vbbar, double* __restrict__ qbbar,
                                                    double* __restrict__ wbar) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m.N) return;
    double qa[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) qa[k] = qbar[ADJ_QB * j + k];
    double ua[4] = {0, 0, 0, 0};      // viscous: velocity bar [3], muEff bar
    if (gUbar) {
#pragma unroll
        for (int t = 0; t < 4; ++t) ua[t] = ucbar[4 * j + t];
    }
    const double Vj = m.V[j];
    const int k0 = m.cf_start[j], k1 = m.cf_start[j + 1];
    for (int kk = k0; kk < k1; ++kk) {
        const int code = m.cf_list[kk];
        if (code < m.Fi) {
            const int f = code, o = m.own[f], n = m.nei[f];
            const int k = (o == j) ? n : o;
            const double coef = (o == j) ? m.w[f] : 1.0 - m.w[f];
            const V3 S = ldv3(m.Sf, m.Fi, f);
            const double* go = gbar + GW * o;
            const double* gn = gbar + GW * n;
            const double Vo = m.V[o], Vn = m.V[n];
#pragma unroll
            for (int fld = 0; fld < 7; ++fld) {
                const double xf = (S.x * go[3 * fld] + S.y * go[3 * fld + 1] + S.z * go[3 * fld + 2]) / Vo -
                                  (S.x * gn[3 * fld] + S.y * gn[3 * fld + 1] + S.z * gn[3 * fld + 2]) / Vn;
                qa[fld] += coef * xf;
            }
            if (gUbar) {    // Gauss gradient of U: (grad U)_dj += S_d U_f,j / V, U_f = w U_o + (1 - w) U_n
                const double* uo = gUbar + 9 * o;
                const double* un = gUbar + 9 * n;
#pragma unroll
                for (int jc = 0; jc < 3; ++jc) {
                    const double xf = (S.x * uo[jc] + S.y * uo[3 + jc] + S.z * uo[6 + jc]) / Vo -
                                      (S.x * un[jc] + S.y * un[3 + jc] + S.z * un[6 + jc]) / Vn;
                    ua[jc] += coef * xf;
                }
            }
            // a neighbour's records count once, also when several faces
            // join the pair
            bool first = true;
            for (int k2 = k0; k2 < kk && first; ++k2) {
                const int c2 = m.cf_list[k2];
                if (c2 < m.Fi && (m.own[c2] == k || m.nei[c2] == k)) first = false;
            }
            if (first) {
#pragma unroll
                for (int fld = 0; fld < 7; ++fld)
                    if (vrec_idx[7 * k + fld] == j) qa[fld] += vrec_val[7 * k + fld];
                if (hrec_idx[k] == j) qa[7] += hrec_val[k];
            }
        } else {
            const int b = code - m.Fi;
            const V3 S = ldv3(m.bSf, m.NB, b);
            const double* gj = gbar + GW * j;
            double* qbb = qbbar + ADJ_QB * b;
#pragma unroll
            for (int fld = 0; fld < 7; ++fld) {
                double add = (S.x * gj[3 * fld] + S.y * gj[3 * fld + 1] + S.z * gj[3 * fld + 2]) / Vj;
                if (vrec_idx[7 * j + fld] == -2 - b) add += vrec_val[7 * j + fld];
                qbb[fld] += add;
            }
            if (gUbar) {    // the boundary velocity's share of j's velocity gradient
                const double* uj = gUbar + 9 * j;
                double* vb = vbbar + ADJ_VBF * b;
#pragma unroll
                for (int jc = 0; jc < 3; ++jc) vb[jc] += (S.x * uj[jc] + S.y * uj[3 + jc] + S.z * uj[6 + jc]) / Vj;
            }
        }
    }
    // q(W_j), p(W_j) VJP
    using D = Dual<5>;
    D Wd[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) Wd[k] = D::seed(W[5 * j + k], k);
    D rho, p, Tt, h;
    Vec3<D> U;
    adj_prim(th, bd, Wd, rho, p, Tt, h, U);
    D qd[7];
    adj_qrec(th, use_c, Wd[0], mkv(Wd[1], Wd[2], Wd[3]), Wd[4], p, Tt, h, qd);
    const D mu = gUbar ? tr.mu_of(Tt) : D(0.0);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double s = qa[7] * p.d[k];
#pragma unroll
        for (int fld = 0; fld < 7; ++fld) s += qa[fld] * qd[fld].d[k];
        if (gUbar) s += ua[0] * U.x.d[k] + ua[1] * U.y.d[k] + ua[2] * U.z.d[k] + ua[3] * mu.d[k];
        wbar[5 * j + k] = s;
    }
}

// Per boundary face: VJP of qb(bs(W_c, U_patch)) with qbbar (and, for the
// objective, of the face pressure with pbar) -> W_c share (wbarb) and the
// patch-velocity share (ubarb), with the branches recorded in bs.
__global__ void k_adj_bc(DevMesh m, Thermo th, Bounds bd, Transport tr, int use_c, const double* __restrict__ W,
                         const double* __restrict__ bs, const double* __restrict__ qbbar,
                         const double* __restrict__ pbar, const double* __restrict__ vbbar,
                         double* __restrict__ wbarb, double* __restrict__ ubarb) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const DevPatch P = m.patches[m.bpatch[b]];
    const int c = m.bcell[b];
    const V3 S = ldv3(m.bSf, m.NB, b);
    const double magS = m.bmagSf[b];
    const V3 n = div3(S, magS);
    const double* B = bs + BW * b;
    using D = Dual<8>;
    D Wd[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) Wd[k] = D::seed(W[5 * c + k], k);
    // the patch velocity values of the free stream: walls' values are their
    // own motion and are held
    const int sU = (P.type == RDST_PATCH_WALL) ? -1 : 5;
    const Vec3<D> Ud = mkv(D::seed(P.U_value[0], sU), D::seed(P.U_value[1], sU < 0 ? -1 : 6),
                           D::seed(P.U_value[2], sU < 0 ? -1 : 7));
    D rho, p, Tt, h;
    Vec3<D> U;
    adj_prim(th, bd, Wd, rho, p, Tt, h, U);
    const BcOut<D> o = bc_state<D>(P, th, bd, n, magS, Wd[0], p, Tt, U, Ud, B[11], B[15]);
    // boundary record as k_boundary + k_recon build it
    const D hb = th.Cp * o.Tb;
    const Vec3<D> rhoU = scl3(o.rho, o.U);
    const D rhoE = o.rho * (hb + 0.5 * magSqr3(o.U)) - o.p;
    D qd[7];
    adj_qrec(th, use_c, o.rho, rhoU, rhoE, o.p, o.Tb, hb, qd);
    const double* qbb = qbbar ? qbbar + ADJ_QB * b : nullptr;
    const double pb = pbar ? pbar[b] : 0.0;
    double acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        double s = pb * o.p.d[k];
        if (qbb) {
#pragma unroll
            for (int fld = 0; fld < 7; ++fld) s += qbb[fld] * qd[fld].d[k];
        }
        acc[k] = s;
    }
    if (vbbar) {    // viscous: boundary velocity and muEff_b = mu(T_b) + mu_t,b
        const double* vb = vbbar + ADJ_VBF * b;
        const D mub = tr.mu_of(o.Tb);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += vb[0] * o.U.x.d[k] + vb[1] * o.U.y.d[k] + vb[2] * o.U.z.d[k] + vb[15] * mub.d[k];
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) wbarb[5 * b + k] = acc[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) ubarb[3 * b + k] = acc[5 + k];
}

// u_j = wbar_j + sum over j's boundary faces of wbarb
__global__ void k_adj_finish(DevMesh m, const double* __restrict__ wbar, const double* __restrict__ wbarb,
                             double* __restrict__ u) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m.N) return;
    double a[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) a[k] = wbar ? wbar[5 * j + k] : 0.0;
    for (int kk = m.cf_start[j]; kk < m.cf_start[j + 1]; ++kk) {
        const int code = m.cf_list[kk];
        if (code < m.Fi) continue;
        const int b = code - m.Fi;
#pragma unroll
        for (int k = 0; k < 5; ++k) a[k] += wbarb[5 * b + k];
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) u[5 * j + k] = a[k];
}

// Objective: J = scale sum_{b in patch} (p_b - p_ref) S_b . d.  pbar_b =
// dJ/dp_b; partials of J and of the force scale sum (p_b - p_ref) S_b.
__global__ void k_adj_objective(DevMesh m, int patch, V3 dir, double p_ref, double scale,
                                const double* __restrict__ bs, double* __restrict__ pbar,
                                double* __restrict__ partial) {
    double acc[4] = {0, 0, 0, 0};
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < m.NB; b += gridDim.x * blockDim.x) {
        double pb = 0.0;
        if (m.bpatch[b] == patch) {
            const V3 S = ldv3(m.bSf, m.NB, b);
            const double dp = bs[BW * b + 5] - p_ref;
            pb = scale * dot3(S, dir);
            acc[0] += dp * pb;
            acc[1] += scale * dp * S.x; acc[2] += scale * dp * S.y; acc[3] += scale * dp * S.z;
        }
        pbar[b] = pb;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double v = block_sum(acc[k]);
        if (threadIdx.x == 0) partial[4 * blockIdx.x + k] = v;
    }
}

// sum over boundary faces of ubarb (3), blockwise
__global__ void k_adj_usum(int NB, const double* __restrict__ ubarb, double* __restrict__ partial) {
    double a[3] = {0, 0, 0};
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < NB; b += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < 3; ++k) a[k] += ubarb[3 * b + k];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double v = block_sum(a[k]);
        if (threadIdx.x == 0) partial[3 * blockIdx.x + k] = v;
    }
}

// out[k] = sum_b partial[b * nv + k], fixed order
__global__ void k_adj_psum(const double* __restrict__ partial, int nb, int nv, double* __restrict__ out) {
    for (int k = 0; k < nv; ++k) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[b * nv + k];
        s = block_sum(s);
        if (threadIdx.x == 0) out[k] = s;
    }
}

// A^T blocks: row r, slot k with column c takes the transpose of block
// (c, r) of A (the pattern is symmetric)
template <typename MT>
__global__ void k_transpose_blocks(SellMat<MT> A, MT* __restrict__ AT) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.N) return;
    const int s = r >> 5, lane = r & 31;
    const int base = A.slice_off[s], width = A.slice_w[s];
    for (int k = 0; k < width; ++k) {
        const size_t slot = (size_t)(base + k);
        const int c = A.col[slot * 32 + lane];
        if (c < 0) continue;
        const int sc = c >> 5, lc = c & 31;
        const int bc = A.slice_off[sc], wc = A.slice_w[sc];
        size_t src = (size_t)-1;
        for (int k2 = 0; k2 < wc; ++k2)
            if (A.col[(size_t)(bc + k2) * 32 + lc] == r) { src = (size_t)(bc + k2); break; }
        MT* dst = AT + slot * (32 * 25) + lane;
        if (src == (size_t)-1) {
#pragma unroll
            for (int e = 0; e < 25; ++e) dst[e * 32] = mt_zero<MT>();
            continue;
        }
        const MT* sv = A.val + src * (32 * 25) + lc;
#pragma unroll
        for (int i = 0; i < 5; ++i)
#pragma unroll
            for (int jj = 0; jj < 5; ++jj) dst[(5 * i + jj) * 32] = sv[(5 * jj + i) * 32];
    }
}

__global__ void k_adj_axpy(long n, double a, const double* __restrict__ x, double* __restrict__ y) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}
__global__ void k_adj_sub(long n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ y) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = a[i] - b[i];
}
// y_i = V_i x_i (5 per cell)
__global__ void k_adj_scale_V(int N, const double* __restrict__ V, const double* __restrict__ x, double* __restrict__ y) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 5L * N) y[i] = V[i / 5] * x[i];
}

}  // namespace rdst

namespace rdst {

// ---------------------------------------------------------------- tangent
// Forward-mode linearization Ju = (dR/dW) u of the same residual, every
// record carried as value + derivative (Dual<1>), with the branches of the
// primal evaluation.  It is the exact counterpart the transposed product is
// checked against (v . Ju = (J^T v) . u to rounding), and a tangent
// sensitivity in its own right.  Records: value and derivative arrays side
// by side (x[0..n) values, x[n..2n) derivatives).
using Tn = Dual<1>;

__device__ __forceinline__ Tn tn_ld(const double* v, const double* d, long i) { Tn r(v[i]); r.d[0] = d[i]; return r; }
__device__ __forceinline__ void tn_st(double* v, double* d, long i, const Tn& x) { v[i] = x.v; d[i] = x.d[0]; }

// cells: q record of W + eps u
// (viscous: also the velocity and muEff = mu(T) + mu_t per cell, 4 each)
__global__ void k_tan_q(int N, Thermo th, Bounds bd, Transport tr, int use_c, const double* __restrict__ W,
                        const double* __restrict__ u, const double* __restrict__ mut, double* __restrict__ qv,
                        double* __restrict__ qd, double* __restrict__ pv, double* __restrict__ pd,
                        double* __restrict__ uv, double* __restrict__ ud) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    Tn Wd[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) { Wd[k] = Tn(W[5 * i + k]); Wd[k].d[0] = u[5 * i + k]; }
    Tn rho, p, Tt, h;
    Vec3<Tn> U;
    adj_prim(th, bd, Wd, rho, p, Tt, h, U);
    Tn q[7];
    adj_qrec(th, use_c, Wd[0], mkv(Wd[1], Wd[2], Wd[3]), Wd[4], p, Tt, h, q);
#pragma unroll
    for (int k = 0; k < 7; ++k) tn_st(qv, qd, (long)QW * i + k, q[k]);
    tn_st(pv, pd, i, p);
    if (uv) {
        tn_st(uv, ud, 4L * i, U.x); tn_st(uv, ud, 4L * i + 1, U.y); tn_st(uv, ud, 4L * i + 2, U.z);
        tn_st(uv, ud, 4L * i + 3, tr.mu_of(Tt) + mut[i]);
    }
}

// boundary faces: boundary record of the perturbed state
// (viscous: also the boundary velocity and muEff_b, 4 per face)
__global__ void k_tan_qb(DevMesh m, Thermo th, Bounds bd, Transport tr, int use_c, const double* __restrict__ W,
                         const double* __restrict__ u, const double* __restrict__ bs, const double* __restrict__ mut_b,
                         double* __restrict__ qbv, double* __restrict__ qbd, double* __restrict__ ubv,
                         double* __restrict__ ubd) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const DevPatch P = m.patches[m.bpatch[b]];
    const int c = m.bcell[b];
    const V3 S = ldv3(m.bSf, m.NB, b);
    const double magS = m.bmagSf[b];
    const double* B = bs + BW * b;
    Tn Wd[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) { Wd[k] = Tn(W[5 * c + k]); Wd[k].d[0] = u[5 * c + k]; }
    Tn rho, p, Tt, h;
    Vec3<Tn> U;
    adj_prim(th, bd, Wd, rho, p, Tt, h, U);
    const Vec3<Tn> Ui = mkv(Tn(P.U_value[0]), Tn(P.U_value[1]), Tn(P.U_value[2]));
    const BcOut<Tn> o = bc_state<Tn>(P, th, bd, div3(S, magS), magS, Wd[0], p, Tt, U, Ui, B[11], B[15]);
    const Tn hb = th.Cp * o.Tb;
    const Tn rhoE = o.rho * (hb + 0.5 * magSqr3(o.U)) - o.p;
    Tn q[7];
    adj_qrec(th, use_c, o.rho, scl3(o.rho, o.U), rhoE, o.p, o.Tb, hb, q);
#pragma unroll
    for (int k = 0; k < 7; ++k) tn_st(qbv, qbd, (long)QW * b + k, q[k]);
    if (ubv) {
        tn_st(ubv, ubd, 4L * b, o.U.x); tn_st(ubv, ubd, 4L * b + 1, o.U.y); tn_st(ubv, ubd, 4L * b + 2, o.U.z);
        tn_st(ubv, ubd, 4L * b + 3, tr.mu_of(o.Tb) + mut_b[b]);
    }
}

// cells: Gauss gradient of U (k_grad's aU) from the velocity records
__global__ void k_tan_gradU(DevMesh m, const double* __restrict__ uv, const double* __restrict__ ud,
                            const double* __restrict__ ubv, const double* __restrict__ ubd,
                            double* __restrict__ gUv, double* __restrict__ gUd) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    Tn a[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = Tn(0.0);
    for (int kk = m.cf_start[i]; kk < m.cf_start[i + 1]; ++kk) {
        const int code = m.cf_list[kk];
        if (code < m.Fi) {
            const int o = m.own[code], n = m.nei[code];
            const double wf = m.w[code];
            const V3 S = ldv3(m.Sf, m.Fi, code);
            const double sg = (o == i) ? 1.0 : -1.0;
            const double Sv[3] = {sg * S.x, sg * S.y, sg * S.z};
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const Tn xf = wf * tn_ld(uv, ud, 4L * o + j) + (1 - wf) * tn_ld(uv, ud, 4L * n + j);
#pragma unroll
                for (int d = 0; d < 3; ++d) a[3 * d + j] += Sv[d] * xf;
            }
        } else {
            const int b = code - m.Fi;
            const V3 S = ldv3(m.bSf, m.NB, b);
            const double Sv[3] = {S.x, S.y, S.z};
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int d = 0; d < 3; ++d) a[3 * d + j] += Sv[d] * tn_ld(ubv, ubd, 4L * b + j);
        }
    }
    const double Vi = m.V[i];
#pragma unroll
    for (int k = 0; k < 9; ++k) tn_st(gUv, gUd, 9L * i + k, a[k] / Vi);
}

// internal faces: derivative of the viscous terms (8 per face)
__global__ void k_tan_visc_faces(DevMesh m, const double* __restrict__ uv, const double* __restrict__ ud,
                                 const double* __restrict__ gUv, const double* __restrict__ gUd,
                                 const double* __restrict__ upv, const double* __restrict__ upd,
                                 double* __restrict__ vfd) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.Fi) return;
    const int P = m.own[f], Q = m.nei[f];
    const double dc = m.dc[f], magS = m.magSf[f];
    const V3 S = ldv3(m.Sf, m.Fi, f);
    const V3 kc = sub3(div3(S, magS), scl3(dc, ldv3(m.d, m.Fi, f)));
    Tn UP[3], UQ[3], gP[9], gQ[9], Up[3], o[7];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        UP[j] = tn_ld(uv, ud, 4L * P + j); UQ[j] = tn_ld(uv, ud, 4L * Q + j); Up[j] = tn_ld(upv, upd, 3L * f + j);
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) { gP[k] = tn_ld(gUv, gUd, 9L * P + k); gQ[k] = tn_ld(gUv, gUd, 9L * Q + k); }
    visc_face(S, magS, m.w[f], dc, kc, UP, UQ, gP, gQ, tn_ld(uv, ud, 4L * P + 3), tn_ld(uv, ud, 4L * Q + 3), Up, o);
#pragma unroll
    for (int k = 0; k < 7; ++k) vfd[8L * f + k] = o[k].d[0];
}

__global__ void k_tan_visc_bfaces(DevMesh m, const double* __restrict__ uv, const double* __restrict__ ud,
                                  const double* __restrict__ gUv, const double* __restrict__ gUd,
                                  const double* __restrict__ ubv, const double* __restrict__ ubd,
                                  const double* __restrict__ bupv, const double* __restrict__ bupd,
                                  double* __restrict__ bvfd) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const int P = m.bcell[b];
    Tn Ub[3], UP[3], gP[9], Up[3], o[7];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        Ub[j] = tn_ld(ubv, ubd, 4L * b + j); UP[j] = tn_ld(uv, ud, 4L * P + j); Up[j] = tn_ld(bupv, bupd, 3L * b + j);
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) gP[k] = tn_ld(gUv, gUd, 9L * P + k);
    visc_bface(ldv3(m.bSf, m.NB, b), m.bmagSf[b], m.bdc[b], Ub, UP, gP, tn_ld(ubv, ubd, 4L * b + 3), Up, o);
#pragma unroll
    for (int k = 0; k < 7; ++k) bvfd[8L * b + k] = o[k].d[0];
}

// cells: Gauss gradient, Venkatakrishnan limiter and HLLCP sensor (k_grad)
__global__ void k_tan_grad(DevMesh m, int venkat_mask, double venkat_K, int hllcp, const double* __restrict__ qv,
                           const double* __restrict__ qd, const double* __restrict__ qbv,
                           const double* __restrict__ qbd, const double* __restrict__ pv,
                           const double* __restrict__ pd, double* __restrict__ gv, double* __restrict__ gd,
                           double* __restrict__ psv, double* __restrict__ psd, double* __restrict__ fcv,
                           double* __restrict__ fcd) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    Tn acc[21];
#pragma unroll
    for (int k = 0; k < 21; ++k) acc[k] = Tn(0.0);
    const int k0 = m.cf_start[i], k1 = m.cf_start[i + 1];
    Tn fmin_c = Tn(1.0);
    const Tn pi = tn_ld(pv, pd, i);
    for (int kk = k0; kk < k1; ++kk) {
        const int code = m.cf_list[kk];
        if (code < m.Fi) {
            const int f = code, o = m.own[f], n = m.nei[f];
            const double wf = m.w[f];
            const V3 S = ldv3(m.Sf, m.Fi, f);
            const double sg = (o == i) ? 1.0 : -1.0;
            for (int j = 0; j < 7; ++j) {
                const Tn xf = wf * tn_ld(qv, qd, (long)QW * o + j) + (1 - wf) * tn_ld(qv, qd, (long)QW * n + j);
                acc[3 * j] += sg * (xf * S.x); acc[3 * j + 1] += sg * (xf * S.y); acc[3 * j + 2] += sg * (xf * S.z);
            }
            if (hllcp) {
                const Tn pk = tn_ld(pv, pd, o == i ? n : o);
                fmin_c = fmin(fmin_c, fmin(pi / pk, pk / pi));
            }
        } else {
            const int b = code - m.Fi;
            const V3 S = ldv3(m.bSf, m.NB, b);
            for (int j = 0; j < 7; ++j) {
                const Tn xf = tn_ld(qbv, qbd, (long)QW * b + j);
                acc[3 * j] += xf * S.x; acc[3 * j + 1] += xf * S.y; acc[3 * j + 2] += xf * S.z;
            }
        }
    }
    const double Vi = m.V[i];
#pragma unroll
    for (int k = 0; k < 21; ++k) { acc[k] = acc[k] / Vi; tn_st(gv, gd, (long)GW * i + k, acc[k]); }
    if (hllcp) tn_st(fcv, fcd, i, fmin_c);
    if (venkat_mask) {
        const double eps2 = pow(venkat_K * cbrt(Vi), 3.0);
        const V3 Ci = ldv3(m.C, m.N, i);
        for (int j = 0; j < 7; ++j) {
            if (!((venkat_mask >> j) & 1)) { tn_st(psv, psd, (long)QW * i + j, Tn(1.0)); continue; }
            const Tn x = tn_ld(qv, qd, (long)QW * i + j);
            Tn mx = x, mn = x;
            for (int kk = k0; kk < k1; ++kk) {
                const int code = m.cf_list[kk];
                Tn xo;
                if (code < m.Fi) { const int o = m.own[code]; xo = tn_ld(qv, qd, (long)QW * (o == i ? m.nei[code] : o) + j); }
                else xo = tn_ld(qbv, qbd, (long)QW * (code - m.Fi) + j);
                if (xo.v > mx.v) mx = xo;
                if (xo.v < mn.v) mn = xo;
            }
            const Tn dmax = mx - x, dmin = mn - x;
            Tn p = Tn(1.0);
            const Vec3<Tn> gj = mkv(acc[3 * j], acc[3 * j + 1], acc[3 * j + 2]);
            for (int kk = k0; kk < k1; ++kk) {
                const int code = m.cf_list[kk];
                const V3 Cf = code < m.Fi ? ldv3(m.Cf, m.Fi, code) : ldv3(m.bCf, m.NB, code - m.Fi);
                const Tn d2 = dot3(gj, sub3(Cf, Ci));
                Tn ph;
                if (d2.v > 0) ph = adj_venkat_phi(dmax, d2, eps2);
                else if (d2.v < 0) ph = adj_venkat_phi(dmin, d2, eps2);
                else ph = Tn(1.0);
                if (ph.v < p.v) p = ph;
            }
            tn_st(psv, psd, (long)QW * i + j, p);
        }
    }
}

// internal faces: reconstruction + flux of the perturbed records; fl gets
// the flux derivative (5 per face)
__global__ void __launch_bounds__(128) k_tan_faces(DevMesh m, Thermo th, int scheme, int lr, int lu, int lt,
                                                   int lowMach, double Mainf, const double* __restrict__ qv,
                                                   const double* __restrict__ qd, const double* __restrict__ gv,
                                                   const double* __restrict__ gd, const double* __restrict__ psv,
                                                   const double* __restrict__ psd, const double* __restrict__ fcv,
                                                   const double* __restrict__ fcd, double* __restrict__ fld,
                                                   double* __restrict__ upv, double* __restrict__ upd) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.Fi) return;
    const int o = m.own[f], n = m.nei[f];
    const double wf = m.w[f];
    const V3 S = ldv3(m.Sf, m.Fi, f);
    const double magS = m.magSf[f];
    const int Ls[7] = {lr, lu, lu, lu, lt, lt, lt};
    Tn xo[7], xn[7];
    if (lr == L_VENKAT || lu == L_VENKAT || lt == L_VENKAT) {
        const V3 Cf = ldv3(m.Cf, m.Fi, f);
        const V3 dP = sub3(Cf, ldv3(m.C, m.N, o)), dN = sub3(Cf, ldv3(m.C, m.N, n));
        for (int j = 0; j < 7; ++j) {
            const Tn qo = tn_ld(qv, qd, (long)QW * o + j), qn = tn_ld(qv, qd, (long)QW * n + j);
            if (Ls[j] == L_VENKAT) {
                const long go = (long)GW * o + 3 * j, gn = (long)GW * n + 3 * j;
                xo[j] = qo + tn_ld(psv, psd, (long)QW * o + j) *
                                 (dP.x * tn_ld(gv, gd, go) + dP.y * tn_ld(gv, gd, go + 1) + dP.z * tn_ld(gv, gd, go + 2));
                xn[j] = qn + tn_ld(psv, psd, (long)QW * n + j) *
                                 (dN.x * tn_ld(gv, gd, gn) + dN.y * tn_ld(gv, gd, gn + 1) + dN.z * tn_ld(gv, gd, gn + 2));
            } else {
                adj_recon_scalar(Ls[j], qo, qn, Tn(0.0), Tn(0.0), wf, xo[j], xn[j]);
            }
        }
    } else {
        const V3 d = ldv3(m.d, m.Fi, f);
        const bool lim = (lr > L_UPWIND) || (lu > L_UPWIND) || (lt > L_UPWIND);
        auto proj = [&](int c, int j) {
            if (!lim) return Tn(0.0);
            const long g0 = (long)GW * c + 3 * j;
            return d.x * tn_ld(gv, gd, g0) + d.y * tn_ld(gv, gd, g0 + 1) + d.z * tn_ld(gv, gd, g0 + 2);
        };
        const int sf[4] = {0, 4, 5, 6};
        for (int t = 0; t < 4; ++t) {
            const int j = sf[t];
            adj_recon_scalar(Ls[j], tn_ld(qv, qd, (long)QW * o + j), tn_ld(qv, qd, (long)QW * n + j), proj(o, j),
                             proj(n, j), wf, xo[j], xn[j]);
        }
        const Vec3<Tn> xP = mkv(tn_ld(qv, qd, (long)QW * o + 1), tn_ld(qv, qd, (long)QW * o + 2), tn_ld(qv, qd, (long)QW * o + 3));
        const Vec3<Tn> xN = mkv(tn_ld(qv, qd, (long)QW * n + 1), tn_ld(qv, qd, (long)QW * n + 2), tn_ld(qv, qd, (long)QW * n + 3));
        Tn ro = Tn(0.0), rn = Tn(0.0);
        if (lu > L_UPWIND) {
            const Vec3<Tn> gradfV = sub3(xN, xP);
            const Tn gradf = dot3(gradfV, gradfV);
            const Vec3<Tn> dgP = mkv(proj(o, 1), proj(o, 2), proj(o, 3));
            const Vec3<Tn> dgN = mkv(proj(n, 1), proj(n, 2), proj(n, 3));
            ro = nvd_r(dot3(gradfV, dgP), gradf);
            rn = nvd_r(dot3(gradfV, dgN), gradf);
        }
        const Tn wo = side_w(lu, true, wf, ro), wn = side_w(lu, false, wf, rn);
        const Vec3<Tn> so = add3(scl3(wo, xP), scl3(1.0 - wo, xN));
        const Vec3<Tn> sn = add3(scl3(wn, xP), scl3(1.0 - wn, xN));
        xo[1] = so.x; xo[2] = so.y; xo[3] = so.z;
        xn[1] = sn.x; xn[2] = sn.y; xn[3] = sn.z;
    }
    SideStateT<Tn> a, b;
    a.rho = xo[0]; a.rhoU = mkv(xo[1], xo[2], xo[3]); a.rPsi = xo[4]; a.e = xo[5]; a.s = xo[6];
    b.rho = xn[0]; b.rhoU = mkv(xn[1], xn[2], xn[3]); b.rPsi = xn[4]; b.e = xn[5]; b.s = xn[6];
    Tn fs = Tn(1.0);
    if (scheme == F_HLLCP) fs = wf * pow(tn_ld(fcv, fcd, o), 3.0) + (1 - wf) * pow(tn_ld(fcv, fcd, n), 3.0);
    const FFluxT<Tn> F = face_flux(scheme, a, b, S, magS, th.gamma, fs, lowMach != 0, Mainf);
    double* out = fld + 5 * f;
    out[0] = F.phi.d[0]; out[1] = F.phiUp.x.d[0]; out[2] = F.phiUp.y.d[0]; out[3] = F.phiUp.z.d[0]; out[4] = F.phiEp.d[0];
    if (upv) { tn_st(upv, upd, 3L * f, F.Up.x); tn_st(upv, upd, 3L * f + 1, F.Up.y); tn_st(upv, upd, 3L * f + 2, F.Up.z); }
}

__global__ void k_tan_bfaces(DevMesh m, Thermo th, int scheme, int lowMach, double Mainf,
                             const double* __restrict__ qbv, const double* __restrict__ qbd,
                             double* __restrict__ bfld, double* __restrict__ bupv, double* __restrict__ bupd) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    SideStateT<Tn> s;
    const long i0 = (long)QW * b;
    s.rho = tn_ld(qbv, qbd, i0);
    s.rhoU = mkv(tn_ld(qbv, qbd, i0 + 1), tn_ld(qbv, qbd, i0 + 2), tn_ld(qbv, qbd, i0 + 3));
    s.rPsi = tn_ld(qbv, qbd, i0 + 4); s.e = tn_ld(qbv, qbd, i0 + 5); s.s = tn_ld(qbv, qbd, i0 + 6);
    const FFluxT<Tn> F = face_flux(scheme, s, s, ldv3(m.bSf, m.NB, b), m.bmagSf[b], th.gamma, Tn(1.0), lowMach != 0, Mainf);
    double* out = bfld + 5 * b;
    out[0] = F.phi.d[0]; out[1] = F.phiUp.x.d[0]; out[2] = F.phiUp.y.d[0]; out[3] = F.phiUp.z.d[0]; out[4] = F.phiEp.d[0];
    if (bupv) {
        tn_st(bupv, bupd, 3L * b, F.Up.x); tn_st(bupv, bupd, 3L * b + 1, F.Up.y); tn_st(bupv, bupd, 3L * b + 2, F.Up.z);
    }
}

// cells: Ju_i = (sum_f +-dF_f + sum_b dF_b) / V_i, less the viscous terms'
// derivatives when given
__global__ void k_tan_residual(DevMesh m, const double* __restrict__ fld, const double* __restrict__ bfld,
                               const double* __restrict__ vfd, const double* __restrict__ bvfd,
                               double* __restrict__ Ju) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    double a[5] = {0, 0, 0, 0, 0};
    for (int kk = m.cf_start[i]; kk < m.cf_start[i + 1]; ++kk) {
        const int code = m.cf_list[kk];
        if (code < m.Fi) {
            const double sg = m.own[code] == i ? 1.0 : -1.0;
#pragma unroll
            for (int k = 0; k < 5; ++k) a[k] += sg * fld[5 * code + k];
            if (vfd) {
                const double* t = vfd + 8L * code;
#pragma unroll
                for (int k = 0; k < 3; ++k) a[1 + k] -= sg * (t[k] + t[3 + k]);
                a[4] -= sg * t[6];
            }
        } else {
#pragma unroll
            for (int k = 0; k < 5; ++k) a[k] += bfld[5 * (code - m.Fi) + k];
            if (bvfd) {
                const double* t = bvfd + 8L * (code - m.Fi);
#pragma unroll
                for (int k = 0; k < 3; ++k) a[1 + k] -= t[k] + t[3 + k];
                a[4] -= t[6];
            }
        }
    }
    const double Vi = m.V[i];
#pragma unroll
    for (int k = 0; k < 5; ++k) Ju[5 * i + k] = a[k] / Vi;
}

}  // namespace rdst
