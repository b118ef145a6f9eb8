// turbulence.cuh -- Spalart-Allmaras transport of nuTilda on the device,
// segregated after the coupled update (turbulence_.correct(),
// Single.C:101): SAneg (SAneg.C:490-605, negative nuTilda and the modified
// Stilda), SARC1 (SARC1.C:125-180, 619-697: the Spalart-Shur
// rotation/curvature multiplier with the material derivative of the strain
// rate) and SARC2 (SARC2.C:121-155, 425-488).  The scalar system is
// built per face (upwind convection with the step's mass flux, Gauss linear
// corrected diffusion) and per cell (ddt, Cb2 term, production /
// destruction with implicit Sp parts), relaxed as fvMatrix::relax and
// solved by point-Jacobi sweeps (gathers, deterministic).
#pragma once

#include "kernels.cuh"

namespace rdst {

struct SAConst {
    double sigmaNut = 0.66666, kappa = 0.41, Cb1 = 0.1355, Cb2 = 0.622, Cw2 = 0.3, Cw3 = 2.0, Cv1 = 7.1, Cv2 = 5.0;
    double Cn1 = 16.0, Cn2 = 0.7, Cn3 = 0.9, Ct3 = 1.2, Ct4 = 0.5, Cr1 = 1.0, Cr2 = 2.0, Cr3 = 1.0;
    double Cr2_SARC1 = 12.0;     // SARC1.C:310-317
    __device__ double Cw1() const { return Cb1 / (kappa * kappa) + (1.0 + Cb2) / sigmaNut; }
};

__device__ __forceinline__ double fpos(double s) { return s >= 0 ? 1.0 : 0.0; }   // foam pos(): pos(0) = 1
__device__ __forceinline__ double fneg(double s) { return s < 0 ? 1.0 : 0.0; }

struct SAFields {
    double* nut;      // [N]
    double* nut_b;    // [NB]
    double* mut;      // [N]
    double* mut_b;    // [NB]
    const double* y;  // [N] wall distance
    double* D;        // [N] DnuTildaEff
    double* fv1;      // [N] fv1 before the solve
    double* diag;     // [N]
    double* b;        // [N]
    double* x2;       // [N] Jacobi ping-pong
    double* gn;       // [3N] grad nuTilda
    double* fup;      // [Fi] row-owner coefficient of nu_N
    double* flo;      // [Fi] row-neighbour coefficient of nu_P
    double* fdP;      // [Fi] diagonal contribution to the owner
    double* fdQ;      // [Fi] diagonal contribution to the neighbour
    double* fcorr;    // [Fi] explicit non-orthogonal correction
    double* bd;       // [NB] boundary diagonal contribution
    double* bb;       // [NB] boundary source contribution
    double* S_old;    // [6N] SARC1: strain rate of the last update (old time)
    double* rho0;     // [N]  SARC1: rho before the coupled update (rho.oldTime())
    int* S_old_valid; // [1]  SARC1: 0 until the first update after a new state
    // SARC1 under dual-time stepping (S_o null: the single-step form):
    // dual2ndDST::fvcDdt(rho, S) = d_rdt (d_c rho S - d_c0 rho_o S_o + d_c00 rho_oo S_oo)
    double* S_o;        // [6N] S.oldTime(): S of the last update of the previous physical step
    double* S_oo;       // [6N] S.oldTime().oldTime()
    const double* W_o;  // [5N] W of the previous physical step (rho.oldTime() = W_o[5i])
    const double* W_oo; // [5N] W two physical steps back
    double d_rdt, d_c, d_c0, d_c00;
    int o_new, oo_new;  // S_o (S_oo) created in this update as a copy of S (of S_o)
};

// symmetric-tensor slot of (a, q): xx xy xz yy yz zz
__device__ __forceinline__ int sym6(int a, int q) { return a <= q ? (a == 0 ? q : a + q + 1) : (q == 0 ? a : a + q + 1); }

// S = symm(grad U) (6), g_ij = dU_j/dx_i
__device__ __forceinline__ void strain6(const double* g, double S[6]) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int q = a; q < 3; ++q) S[sym6(a, q)] = 0.5 * (g[3 * a + q] + g[3 * q + a]);
}

// nuTilda boundary value: fixedValue, inletOutlet on phi, else zeroGradient
__device__ __forceinline__ double nut_vf(const DevPatch& P, double phi) {
    if (P.bc_nut == 0) return 1.0;
    if (P.bc_nut == 2) return phi >= 0 ? 0.0 : 1.0;
    return 0.0;
}

__global__ void k_sa_bc(DevMesh m, const double* __restrict__ bs, SAFields F) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const DevPatch P = m.patches[m.bpatch[b]];
    const double f = nut_vf(P, bs[BW * b + 7]);
    F.nut_b[b] = f * P.nut_value + (1 - f) * F.nut[m.bcell[b]];
}

// grad U and grad nuTilda (Gauss linear, face gather in foam order)
__global__ void __launch_bounds__(128) k_sa_grad(DevMesh m, const double* __restrict__ prim, const double* __restrict__ bs,
                                                 SAFields F, double* __restrict__ gU) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    double aU[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, an[3] = {0, 0, 0};
    for (int k = m.cf_start[i]; k < m.cf_start[i + 1]; ++k) {
        int code = m.cf_list[k];
        double Sv[3], Uf[3], nf;
        if (code < m.Fi) {
            int o = m.own[code], n = m.nei[code];
            double w = m.w[code], sg = (o == i) ? 1.0 : -1.0;
            V3 S = ldv3(m.Sf, m.Fi, code);
            Sv[0] = sg * S.x; Sv[1] = sg * S.y; Sv[2] = sg * S.z;
#pragma unroll
            for (int j = 0; j < 3; ++j) Uf[j] = w * prim[PW * o + 3 + j] + (1 - w) * prim[PW * n + 3 + j];
            nf = w * F.nut[o] + (1 - w) * F.nut[n];
        } else {
            int b = code - m.Fi;
            V3 S = ldv3(m.bSf, m.NB, b);
            Sv[0] = S.x; Sv[1] = S.y; Sv[2] = S.z;
#pragma unroll
            for (int j = 0; j < 3; ++j) Uf[j] = bs[BW * b + 12 + j];
            nf = F.nut_b[b];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
#pragma unroll
            for (int j = 0; j < 3; ++j) aU[3 * d + j] += Sv[d] * Uf[j];
            an[d] += Sv[d] * nf;
        }
    }
    const double Vi = m.V[i];
#pragma unroll
    for (int k = 0; k < 9; ++k) gU[9 * i + k] = aU[k] / Vi;
#pragma unroll
    for (int d = 0; d < 3; ++d) F.gn[3 * i + d] = an[d] / Vi;
}

// per cell: ddt, Cb2 term, sources with implicit parts, DnuTildaEff, fv1
// sarc1: 0 SARC2 multiplier, 1 SARC1 multiplier, 2 none (SpalartAllmaras)
__global__ void k_sa_cell(DevMesh m, Transport tr, int neg_sa, int sarc1, int steady, const double* __restrict__ W,
                          const double* __restrict__ prim, const double* __restrict__ gU,
                          const double* __restrict__ rdtc, const Scalars* __restrict__ sc,
                          const double* __restrict__ fl, const double* __restrict__ bs, SAFields F) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    const SAConst K;
    const double rho = W[5 * i], nt = F.nut[i], V = m.V[i], yy = F.y[i];
    const double mu = tr.mu_of_T(prim[PW * i + 1]);
    const double chi = rho * nt / mu, chi3 = chi * chi * chi;
    const double fv1 = chi3 / (chi3 + K.Cv1 * K.Cv1 * K.Cv1);
    double g[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = gU[9 * i + k];
    double W2 = 0, S2 = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            double w = 0.5 * (g[3 * a + q] - g[3 * q + a]), s = 0.5 * (g[3 * a + q] + g[3 * q + a]);
            W2 += w * w; S2 += s * s;
        }
    const double Omega = sqrt(2.0) * sqrt(W2);
    const double fv2 = 1.0 / pow(1.0 + chi / K.Cv2, 3.0);
    const double kd2 = (K.kappa * yy) * (K.kappa * yy);
    double Stilda;
    if (neg_sa) {
        double Sbar = fv2 * nt / kd2;
        Stilda = Omega + fpos(K.Cn2 * Omega + Sbar) * Sbar +
                 fneg(K.Cn2 * Omega + Sbar) * (Omega * (K.Cn2 * K.Cn2 * Omega + K.Cn3 * Sbar)) /
                     fmax((K.Cn3 - 2.0 * K.Cn2) * Omega - Sbar, D_SMALL);
    } else {
        double cb = chi / K.Cv2;
        double fv3 = (1.0 + chi * fv1) * (1.0 / K.Cv2) * (3 * (1.0 + cb) + cb * cb) / pow(1.0 + cb, 3.0);
        Stilda = fv3 * sqrt(2.0) * sqrt(W2) + fv2 * nt / kd2;
    }
    const double r = fmin(nt / (fmax(Stilda, D_SMALL) * kd2), 10.0);
    const double gg = r + K.Cw2 * (pow(r, 6.0) - r);
    const double fw = gg * pow((1.0 + pow(K.Cw3, 6.0)) / (pow(gg, 6.0) + pow(K.Cw3, 6.0)), 1.0 / 6.0);
    const double rdt = steady ? rdtc[i] : 1.0 / sc->deltaT;
    double diag = rdt * rho * V;
    double b = rdt * rho * nt * V;
    const double gn2 = F.gn[3 * i] * F.gn[3 * i] + F.gn[3 * i + 1] * F.gn[3 * i + 1] + F.gn[3 * i + 2] * F.gn[3 * i + 2];
    b += K.Cb2 / K.sigmaNut * rho * gn2 * V;
    if (neg_sa) {
        const double ft2 = K.Ct3 * exp(-K.Ct4 * chi * chi);
        const double pp = fpos(nt), nn = fneg(nt);
        b += pp * K.Cb1 * (1.0 - ft2) * rho * Stilda * nt * V;
        diag += pp * (K.Cw1() * fw - K.Cb1 / (K.kappa * K.kappa) * ft2) * nt * rho / (yy * yy) * V;
        b += nn * K.Cb1 * (1.0 - K.Ct3) * rho * Omega * nt * V;
        diag -= nn * K.Cw1() * nt * rho / (yy * yy) * V;
        const double fn = fpos(chi) + fneg(chi) * (K.Cn1 + chi3) / (K.Cn1 - chi3);
        F.D[i] = (rho * nt * fn + mu) / K.sigmaNut;
    } else {
        const double sqrS = 2.0 * S2, sqrW = 2.0 * W2;
        const double rStar = sqrt(sqrS / fmax(sqrW, D_SMALL));
        double fr1;
        if (sarc1 == 2) {
            fr1 = 1.0;                      // SpalartAllmaras: no rotation/curvature multiplier
        } else if (sarc1) {
            // DS/Dt = ddt(rho, S) + div(phi, S): the flow's ddt scheme with
            // the last update's S as old time (the current S at the first
            // update), Gauss upwind on the step's mass flux, zeroGradient S_b
            double Si[6], So[6], Soo[6], dv[6] = {0, 0, 0, 0, 0, 0};
            strain6(g, Si);
            if (F.S_o) {
                // dual-time: the old times of the physical step, created
                // from the current S (S_o) and from S_o (S_oo) at first use
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    So[k] = F.o_new ? Si[k] : F.S_o[6 * i + k];
                    Soo[k] = F.oo_new ? So[k] : F.S_oo[6 * i + k];
                }
                if (F.o_new)
#pragma unroll
                    for (int k = 0; k < 6; ++k) F.S_o[6 * i + k] = So[k];
                if (F.oo_new)
#pragma unroll
                    for (int k = 0; k < 6; ++k) F.S_oo[6 * i + k] = Soo[k];
            } else {
                const int valid = *F.S_old_valid;
#pragma unroll
                for (int k = 0; k < 6; ++k) So[k] = valid ? F.S_old[6 * i + k] : Si[k];
            }
            for (int kk = m.cf_start[i]; kk < m.cf_start[i + 1]; ++kk) {
                const int code = m.cf_list[kk];
                if (code < m.Fi) {
                    const double ph = fl[5 * code];
                    const int up = ph >= 0 ? m.own[code] : m.nei[code];      // upwind, pos(0) = 1
                    const double sg = (m.own[code] == i) ? 1.0 : -1.0;
                    double Su[6];
                    strain6(gU + 9 * up, Su);
#pragma unroll
                    for (int k = 0; k < 6; ++k) dv[k] += sg * ph * Su[k];
                } else {
                    const double ph = bs[BW * (code - m.Fi) + 7];
#pragma unroll
                    for (int k = 0; k < 6; ++k) dv[k] += ph * Si[k];
                }
            }
            double DS[6];
            if (F.S_o) {
                const double ro = F.W_o[5 * i], roo = F.W_oo[5 * i];
#pragma unroll
                for (int k = 0; k < 6; ++k)
                    DS[k] = F.d_rdt * (F.d_c * rho * Si[k] - F.d_c0 * ro * So[k] + F.d_c00 * roo * Soo[k]) + dv[k] / V;
            } else {
                const double rdt0 = steady ? rdtc[i] : 1.0 / sc->deltaT;
#pragma unroll
                for (int k = 0; k < 6; ++k) DS[k] = rdt0 * (rho * Si[k] - F.rho0[i] * So[k]) + dv[k] / V;
            }
            // rTilda = 2/(rho max(D^2, SMALL)^2) sum_aq (sum_k W_ak S_qk) DS_aq/Dt
            const double sqrD = 0.5 * (sqrS + sqrW);
            double acc = 0;
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    double ws = 0;
#pragma unroll
                    for (int k = 0; k < 3; ++k) ws += 0.5 * (g[3 * a + k] - g[3 * k + a]) * Si[sym6(q, k)];
                    acc += ws * DS[sym6(a, q)];
                }
            const double mD = fmax(sqrD, D_SMALL);
            const double rTilda = 2.0 / (rho * (mD * mD)) * acc;
            fr1 = (1 + K.Cr1) * 2.0 * rStar / (1.0 + rStar) * (1.0 - K.Cr3 * atan(K.Cr2_SARC1 * rTilda)) - K.Cr1;
            // this update's S is the next one's old time (only cell i reads slot i)
#pragma unroll
            for (int k = 0; k < 6; ++k) F.S_old[6 * i + k] = Si[k];
        } else {
            const double rrStar = sqrt(sqrW / fmax(sqrS, D_SMALL));
            const double rTilda = rrStar * (rrStar - 1.0);
            fr1 = (1 + K.Cr1) * 2.0 * rStar / (1.0 + rStar) * (1.0 - K.Cr3 * atan(K.Cr2 * rTilda)) - K.Cr1;
        }
        b += K.Cb1 * rho * Stilda * nt * fr1 * V;
        diag += K.Cw1() * fw * nt * rho / (yy * yy) * V;
        F.D[i] = rho * nt / K.sigmaNut + mu;
    }
    F.diag[i] = diag;
    F.b[i] = b;
    F.fv1[i] = fv1;
}

// SARC1 bookkeeping: rho before the coupled update; old-time S now valid
__global__ void k_sarc1_rho0(int N, const double* __restrict__ W, double* __restrict__ rho0) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) rho0[i] = W[5 * i];
}
__global__ void k_sarc1_valid(int* __restrict__ flag) { *flag = 1; }

// per internal face: upwind convection + corrected diffusion coefficients
__global__ void k_sa_faces(DevMesh m, const double* __restrict__ fl, SAFields F, int lin_upwind) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.Fi) return;
    const int P = m.own[f], Q = m.nei[f];
    const double w = m.w[f], ph = fl[5 * f], magS = m.magSf[f], dc = m.dc[f];
    const double wu = fpos(ph);
    const double Df = w * F.D[P] + (1 - w) * F.D[Q];
    const double dcoef = Df * magS * dc;
    F.fdP[f] = wu * ph + dcoef;
    F.fdQ[f] = -(1 - wu) * ph + dcoef;
    F.fup[f] = (1 - wu) * ph - dcoef;
    F.flo[f] = -wu * ph - dcoef;
    const V3 S = ldv3(m.Sf, m.Fi, f);
    const V3 n = div3(S, magS);
    const V3 kc = sub3(n, scl3(dc, ldv3(m.d, m.Fi, f)));
    const V3 gf = add3(scl3(w, mk(F.gn[3 * P], F.gn[3 * P + 1], F.gn[3 * P + 2])),
                       scl3(1 - w, mk(F.gn[3 * Q], F.gn[3 * Q + 1], F.gn[3 * Q + 2])));
    double corr = Df * magS * dot3(kc, gf);
    if (lin_upwind) {
        // linearUpwind grad(nuTilda): explicit part phi (Cf - C) . grad nuTilda_C
        // of the upwind cell C, moved to the source
        const int C = ph >= 0 ? P : Q;
        const V3 dC = sub3(ldv3(m.Cf, m.Fi, f), ldv3(m.C, m.N, C));
        corr -= ph * dot3(dC, mk(F.gn[3 * C], F.gn[3 * C + 1], F.gn[3 * C + 2]));
    }
    F.fcorr[f] = corr;
}

// per boundary face: convection through f ref + (1-f) nu_P, diffusion with
// DnuTildaEff of the boundary values
__global__ void k_sa_bfaces(DevMesh m, Transport tr, int neg_sa, const double* __restrict__ bs, SAFields F) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const SAConst K;
    const DevPatch P = m.patches[m.bpatch[b]];
    const double* B = bs + BW * b;
    const double ph = B[7];
    const double fv = nut_vf(P, ph), ref = P.nut_value;
    const double mub = tr.mu_of_T(B[6]);
    const double nb = F.nut_b[b], rhob = B[0];
    double Db;
    if (neg_sa) {
        const double chib = rhob * nb / mub, chib3 = chib * chib * chib;
        const double fnb = fpos(chib) + fneg(chib) * (K.Cn1 + chib3) / (K.Cn1 - chib3);
        Db = (rhob * nb * fnb + mub) / K.sigmaNut;
    } else {
        Db = rhob * nb / K.sigmaNut + mub;
    }
    const double dcoef = Db * m.bmagSf[b] * m.bdc[b] * fv;
    F.bd[b] = ph * (1 - fv) + dcoef;
    F.bb[b] = -ph * fv * ref + dcoef * ref;
}

// per cell: gather the face parts, fvMatrix::relax (diagonal dominance,
// divide by alpha, source += (D - D0) psi)
__global__ void k_sa_assemble(DevMesh m, double alpha, SAFields F) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    double diag = F.diag[i], b = F.b[i], off = 0.0;
    for (int k = m.cf_start[i]; k < m.cf_start[i + 1]; ++k) {
        int code = m.cf_list[k];
        if (code < m.Fi) {
            if (m.own[code] == i) { diag += F.fdP[code]; b += F.fcorr[code]; off += fabs(F.fup[code]); }
            else { diag += F.fdQ[code]; b -= F.fcorr[code]; off += fabs(F.flo[code]); }
        } else {
            int bb = code - m.Fi;
            diag += F.bd[bb];
            b += F.bb[bb];
        }
    }
    const double Dn = fmax(diag, off) / alpha;
    F.b[i] = b + (Dn - diag) * F.nut[i];
    F.diag[i] = Dn;
}

// dual2ndDST::fvmDdt(rho, nuTilda) (dual2ndDST.C:456-488) on top of the
// pseudo-time part rDeltaTau rho V of k_sa_cell: diag += a rho V, source
// -= V (b rho^n nuTilda^n + c rho^n-1 nuTilda^n-1)
__global__ void k_sa_dual(int N, const double* __restrict__ V, const double* __restrict__ W,
                          const double* __restrict__ Wn, const double* __restrict__ Wnm1,
                          const double* __restrict__ nutN, const double* __restrict__ nutNm1, double a, double b,
                          double c, SAFields F) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double Vi = V[i];
    F.diag[i] += a * W[5L * i] * Vi;
    F.b[i] -= Vi * (b * Wn[5L * i] * nutN[i] + c * Wnm1[5L * i] * nutNm1[i]);
}

// one point-Jacobi sweep x_out = (b - offdiag x_in) / D
__global__ void k_sa_jacobi(DevMesh m, SAFields F, const double* __restrict__ xin, double* __restrict__ xout) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    if (m.rmask && m.rmask[i]) { xout[i] = xin[i]; return; }      // held cell keeps its nuTilda
    double s = F.b[i];
    for (int k = m.cf_start[i]; k < m.cf_start[i + 1]; ++k) {
        int code = m.cf_list[k];
        if (code >= m.Fi) continue;
        if (m.own[code] == i) s -= F.fup[code] * xin[m.nei[code]];
        else s -= F.flo[code] * xin[m.own[code]];
    }
    xout[i] = s / F.diag[i];
}

// bound (SARC2: nuTilda >= 0), copy the solution, mut = |fv1| nuTilda rho
__global__ void k_sa_finish(int N, int neg_sa, const double* __restrict__ W, const double* __restrict__ x, SAFields F) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double nt = x[i];
    if (!neg_sa) nt = fmax(nt, 0.0);
    F.nut[i] = nt;
    double mm = (neg_sa ? fabs(F.fv1[i]) : F.fv1[i]) * nt * W[5 * i];
    F.mut[i] = neg_sa ? fmax(mm, 0.0) : mm;
}

// boundary mut: 0 on walls, fv1(chi_b) nuTilda_b rho_b elsewhere
__global__ void k_sa_mutb(DevMesh m, Transport tr, const double* __restrict__ bs, SAFields F) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const SAConst K;
    if (m.patches[m.bpatch[b]].type == 1) { F.mut_b[b] = 0.0; return; }
    const double* B = bs + BW * b;
    const double chi = B[0] * F.nut_b[b] / tr.mu_of_T(B[6]), chi3 = chi * chi * chi;
    const double fv1 = chi3 / (chi3 + K.Cv1 * K.Cv1 * K.Cv1);
    F.mut_b[b] = fmax(fv1 * F.nut_b[b] * B[0], 0.0);
}

// mut from an initial nuTilda (set_primitive)
__global__ void k_sa_init_mut(int N, Transport tr, const double* __restrict__ W, const double* __restrict__ prim, SAFields F) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const SAConst K;
    const double chi = W[5 * i] * F.nut[i] / tr.mu_of_T(prim[PW * i + 1]), chi3 = chi * chi * chi;
    F.fv1[i] = chi3 / (chi3 + K.Cv1 * K.Cv1 * K.Cv1);
}

}  // namespace rdst
