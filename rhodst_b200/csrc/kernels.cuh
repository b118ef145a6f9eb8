// kernels.cuh -- sm_100a kernels of the fully-coupled density-based step.
//
// Every kernel is a gather (one thread per cell / face / matrix row) with a
// fixed, face-ordered accumulation order: no floating-point atomics, so
// results are bitwise reproducible run to run.  The path is HBM/L2 bound
// (no dense contraction), so none of it uses tensor cores; the levers are
// coalesced SoA/entry-interleaved layouts, fused per-face arithmetic and
// single-pass reductions.
#pragma once

#include "physics.cuh"
#include "rdst_internal.h"

namespace rdst {

constexpr int TPB = 256;

__device__ __forceinline__ V3 ldv3(const double* a, int n, int i) { return mk(a[i], a[n + i], a[2 * n + i]); }

// ------------------------------------------------------------------ reductions
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
// block-wide sum in a fixed order; result valid in thread 0
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
    if (wid == 0) v = warp_sum(v);
    return v;
}
__device__ __forceinline__ double block_min(double v) {
    __shared__ double sh[32];
    v = warp_min(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : 1e300;
    if (wid == 0) v = warp_min(v);
    return v;
}
__device__ __forceinline__ double block_max(double v) {
    __shared__ double sh[32];
    v = warp_max(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : -1e300;
    if (wid == 0) v = warp_max(v);
    return v;
}

// ------------------------------------------------------------------ state / BCs
struct Bounds { double rho_min, rho_max, p_min, p_max, T_min, T_max; };

// constTransport mu / Prandtl, or Sutherland mu = As sqrt(T)/(1 + Ts/T)
struct Transport {
    double mu, As, Ts, Pr, Prt;
    int viscous;
    __device__ __forceinline__ double mu_of_T(double T) const {
        return As > 0 ? As * sqrt(T) / (1.0 + Ts / T) : mu;
    }
    // the same law on any scalar type (the adjoint's dual numbers)
    template <typename T>
    __device__ __forceinline__ T mu_of(const T& Tt) const {
        if (As > 0) return As * sqrt(Tt) / (1.0 + Ts / Tt);
        return T(mu);
    }
};

// initial state from primitives (createFields.H:21-72)
__global__ void k_init_state(int N, Thermo th, const double* __restrict__ prim, double* __restrict__ W) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double* P = prim + PW * i;
    double p = P[0], T = P[1], h = P[2];
    V3 U = mk(P[3], P[4], P[5]);
    double rho = p / (th.R * T);
    W[5 * i + 0] = rho;
    W[5 * i + 1] = rho * U.x;
    W[5 * i + 2] = rho * U.y;
    W[5 * i + 3] = rho * U.z;
    W[5 * i + 4] = rho * (h * th.Cv / th.Cp + 0.5 * magSqr3(U));
}

// Conservative fields in the caller's cell order (rho[N], rhoU[3N],
// rhoE[N], staged on the device) -> W and the primitive record in the
// internal order (perm[r] = caller's index of internal row r).  The
// arithmetic is written with explicit roundings so that it matches a plain
// host evaluation of the same formulas bit for bit.
__global__ void k_set_conservative(int N, Thermo th, const int* __restrict__ perm, const double* __restrict__ rho,
                                   const double* __restrict__ rhoU, const double* __restrict__ rhoE,
                                   double* __restrict__ W, double* __restrict__ prim) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    const int i = perm[r];
    const double rh = rho[i], mx = rhoU[3 * i], my = rhoU[3 * i + 1], mz = rhoU[3 * i + 2], E = rhoE[i];
    W[5 * r] = rh; W[5 * r + 1] = mx; W[5 * r + 2] = my; W[5 * r + 3] = mz; W[5 * r + 4] = E;
    const double Ux = __ddiv_rn(mx, rh), Uy = __ddiv_rn(my, rh), Uz = __ddiv_rn(mz, rh);
    const double k2 = __dadd_rn(__dadd_rn(__dmul_rn(Ux, Ux), __dmul_rn(Uy, Uy)), __dmul_rn(Uz, Uz));
    const double e = __dsub_rn(__ddiv_rn(E, rh), __dmul_rn(0.5, k2));
    const double T = __ddiv_rn(e, th.Cv);
    double* P = prim + PW * r;
    P[0] = __dmul_rn(__dmul_rn(rh, th.R), T); P[1] = T; P[2] = __dmul_rn(th.Cp, T);
    P[3] = Ux; P[4] = Uy; P[5] = Uz;
}

// the states of a list of cells (internal rows): rho, rhoU, rhoE, nuTilda
// (0 without a turbulence model), six values per cell
__global__ void k_get_cells(int n, const int* __restrict__ rows, const double* __restrict__ W,
                            const double* __restrict__ nut, double* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int r = rows[j];
#pragma unroll
    for (int k = 0; k < 5; ++k) out[6L * j + k] = W[5L * r + k];
    out[6L * j + 5] = nut ? nut[r] : 0.0;
}

// the same six values into a list of cells; W and the primitive record as
// k_set_conservative makes them (same operations, so the same bits)
__global__ void k_set_cells(int n, Thermo th, const int* __restrict__ rows, const double* __restrict__ in,
                            double* __restrict__ W, double* __restrict__ prim, double* __restrict__ nut) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int r = rows[j];
    const double* v = in + 6L * j;
    const double rh = v[0], mx = v[1], my = v[2], mz = v[3], E = v[4];
    W[5 * r] = rh; W[5 * r + 1] = mx; W[5 * r + 2] = my; W[5 * r + 3] = mz; W[5 * r + 4] = E;
    const double Ux = __ddiv_rn(mx, rh), Uy = __ddiv_rn(my, rh), Uz = __ddiv_rn(mz, rh);
    const double k2 = __dadd_rn(__dadd_rn(__dmul_rn(Ux, Ux), __dmul_rn(Uy, Uy)), __dmul_rn(Uz, Uz));
    const double e = __dsub_rn(__ddiv_rn(E, rh), __dmul_rn(0.5, k2));
    const double T = __ddiv_rn(e, th.Cv);
    double* P = prim + PW * r;
    P[0] = __dmul_rn(__dmul_rn(rh, th.R), T); P[1] = T; P[2] = __dmul_rn(th.Cp, T);
    P[3] = Ux; P[4] = Uy; P[5] = Uz;
    if (nut) nut[r] = v[5];
}

// W (internal order) -> rho, rhoU, rhoE in the caller's cell order
__global__ void k_get_conservative(int N, const int* __restrict__ perm, const double* __restrict__ W,
                                   double* __restrict__ rho, double* __restrict__ rhoU, double* __restrict__ rhoE) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    const int i = perm[r];
    rho[i] = W[5 * r];
    rhoU[3 * i] = W[5 * r + 1]; rhoU[3 * i + 1] = W[5 * r + 2]; rhoU[3 * i + 2] = W[5 * r + 3];
    rhoE[i] = W[5 * r + 4];
}

// boundary state before the first BC evaluation: internal values and the
// mass flux (rho U)_owner . Sf
__global__ void k_init_phib(DevMesh m, const double* __restrict__ W, const double* __restrict__ prim,
                            double* __restrict__ bs) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    int c = m.bcell[b];
    V3 S = ldv3(m.bSf, m.NB, b);
    double* B = bs + BW * b;
    B[7] = dot3(mk(W[5 * c + 1], W[5 * c + 2], W[5 * c + 3]), S);
    B[0] = W[5 * c];
    B[5] = prim[PW * c];
    B[6] = prim[PW * c + 1];
}

// Boundary values of p, U, T from the internal field (fixedValue,
// zeroGradient, inletOutlet, symmetryPlane/slip, characteristic far field
// of farField*DSTFvPatch*Field.C:144-221) and rho/rhoU/rhoE rebuilt as
// updateFields.H:84-93.  The valueFractions are stored for the boundary
// Jacobian (valueInternalCoeffs = 1 - valueFraction).
// Boundary state of one face from the adjacent cell's rho, p, T, U and the
// patch values (UInf the patch velocity value): the patch-field updates of
// fixedValue, zeroGradient, inletOutlet, symmetryPlane/slip and the
// characteristic far field (farField*DST::updateCoeffs, *.C:144-221).
// phi_prev (the face's previous mass flux) and mach (the far-field face
// Mach number from the previous boundary density, temperature and mass
// flux) only choose branches (in/outflow, sub/supersonic); k_boundary keeps
// both in the boundary record, so the adjoint differentiates the branches
// the current states were built with.  Templated so that the adjoint
// differentiates the same arithmetic.
template <typename T>
struct BcOut {
    T rho, p, Tb;
    Vec3<T> U;
    double fp, fU, fT;
};

__device__ __forceinline__ bool bc_farfield(const DevPatch& P) { return P.bc_p == 5 || P.bc_U == 5 || P.bc_T == 5; }

template <typename T>
__device__ __forceinline__ BcOut<T> bc_state(const DevPatch& P, const Thermo& th, const Bounds& bd, V3 n, double magS,
                                             const T& rhoI, const T& pI, const T& TI, const Vec3<T>& Ui,
                                             const Vec3<T>& UInf, double phi_prev, double mach) {
    const bool outflow = phi_prev >= 0.0;
    double supIn = 0, supOut = 0, subIn = 0, subOut = 0;
    T rho0c0 = T(0.0), cI = T(0.0), pbU = T(0.0);
    if (bc_farfield(P)) {
        cI = sqrt(th.gamma * th.R * TI);
        supIn = dneg0(mach + 1);
        supOut = dpos0(mach - 1);
        subIn = dneg(mach) - supIn;
        subOut = dpos0(mach) - supOut;
        rho0c0 = rhoI * cI;
        pbU = 0.5 * (P.p_value + pI - rho0c0 * dot3(n, sub3(UInf, Ui)));
    }
    BcOut<T> o;
    o.fp = 0; o.fU = 0; o.fT = 0;
    T pb, Tb;
    Vec3<T> Ub;
    switch (P.bc_p) {
        case 0: pb = T(P.p_value); o.fp = 1; break;
        case 2: o.fp = outflow ? 0.0 : 1.0; pb = outflow ? pI : T(P.p_value); break;
        case 5: {
            T pbp = P.p_value - rho0c0 * dot3(n, sub3(UInf, Ui));
            T ref = supIn * P.p_value + subIn * pbp + subOut * P.p_value;
            o.fp = 1 - supOut - 0.5 * subIn;
            pb = o.fp * ref + (1 - o.fp) * pI;
            break;
        }
        default: pb = pI; break;
    }
    switch (P.bc_T) {
        case 0: Tb = T(P.T_value); o.fT = 1; break;
        case 2: o.fT = outflow ? 0.0 : 1.0; Tb = outflow ? TI : T(P.T_value); break;
        case 5: {
            T RI = pI / rhoI / TI;
            T rhoa = P.p_value / P.T_value / RI;
            T subsInValue = pbU / (rhoa + (pbU - P.p_value) / sq(cI)) / RI;
            T sOVF = pbU / (pI + RI * TI * (pbU - pI) / sq(cI));
            T ref = supIn * P.T_value + subIn * subsInValue;
            T fT = 1.0 - supOut - sOVF * subOut;
            o.fT = val(fT);
            Tb = fT * ref + (1.0 - fT) * TI;
            break;
        }
        default: Tb = TI; break;
    }
    switch (P.bc_U) {
        case 0: Ub = UInf; o.fU = 1; break;
        case 2: o.fU = outflow ? 0.0 : 1.0; Ub = outflow ? Ui : UInf; break;
        case 3:
        case 4: Ub = sub3(Ui, scl3(dot3(n, Ui), n)); break;
        case 5: {
            Vec3<T> subsIn = sub3(UInf, scl3((P.p_value - pbU) / rho0c0, n));
            Vec3<T> subsOut = scl3((pI - pbU) / rho0c0, n);
            Vec3<T> ref = add3(add3(scl3(supIn, UInf), scl3(subIn, subsIn)), scl3(subOut, subsOut));
            o.fU = 1 - supOut - subOut;
            Ub = add3(scl3(o.fU, ref), scl3(1 - o.fU, Ui));
            break;
        }
        default: Ub = Ui; break;
    }
    o.p = fmin(fmax(pb, bd.p_min), bd.p_max);
    o.Tb = Tb;
    o.U = Ub;
    o.rho = o.p * (1.0 / (th.R * Tb));
    return o;
}

__global__ void k_boundary(DevMesh m, Thermo th, Bounds bd, const double* __restrict__ W,
                           const double* __restrict__ prim, double* __restrict__ bs) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const DevPatch P = m.patches[m.bpatch[b]];
    const int ci = m.bcell[b];
    V3 S = ldv3(m.bSf, m.NB, b);
    double magS = m.bmagSf[b];
    V3 n = div3(S, magS);
    const double* Pi = prim + PW * ci;
    double* B = bs + BW * b;
    // branch inputs from the previous record (kept: B[11] mass flux, B[15] Mach)
    const double phi_prev = B[7];
    const double mach = bc_farfield(P) ? B[7] / B[0] / magS / sqrt(th.gamma * th.R * B[6]) : 0.0;
    const BcOut<double> o = bc_state<double>(P, th, bd, n, magS, W[5 * ci], Pi[0], Pi[1], mk(Pi[3], Pi[4], Pi[5]),
                                             mk(P.U_value[0], P.U_value[1], P.U_value[2]), phi_prev, mach);
    B[11] = phi_prev;
    B[15] = mach;
    const double hb = th.Cp * o.Tb;
    const double rhob = o.rho;
    B[0] = rhob;
    B[1] = rhob * o.U.x;
    B[2] = rhob * o.U.y;
    B[3] = rhob * o.U.z;
    B[4] = rhob * (hb + 0.5 * magSqr3(o.U)) - o.p;
    B[5] = o.p;
    B[6] = o.Tb;
    B[8] = o.fp;
    B[9] = o.fU;
    B[10] = o.fT;
    B[12] = o.U.x;
    B[13] = o.U.y;
    B[14] = o.U.z;
}

// ------------------------------------------------------------------ residual
// Reconstruction record per cell (and per boundary face):
// q = (rho, rhoU xyz, rPsi = RT, e = h - p/rho, s) with s = c = sqrt(gamma RT)
// (Kurganov, AUSM) or the critical speed sqrt(2(g-1)/(g+1) H) (HLL family,
// AUSM+, AUSM+up; HLLDST.C:130-137).
__global__ void k_recon(DevMesh m, Thermo th, Transport tr, int use_c, const double* __restrict__ W,
                        const double* __restrict__ prim, const double* __restrict__ bs, const double* __restrict__ mut,
                        const double* __restrict__ mut_b, double* __restrict__ q, double* __restrict__ qb) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double g = th.gamma;
    if (i < m.N) {
        const double* w5 = W + 5 * i;
        const double* P = prim + PW * i;
        double rho = w5[0], rhoE = w5[4], p = P[0], T = P[1], h = P[2];
        double rPsi = th.R * T;
        double s;
        if (use_c) s = sqrt(g * rPsi);
        else {
            double H = fmax(rhoE / rho, D_SMALL) + fmax(p / rho, D_SMALL);
            s = sqrt(2.0 * (g - 1.0) / (g + 1.0) * H);
        }
        double* o = q + QW * i;
        o[0] = rho; o[1] = w5[1]; o[2] = w5[2]; o[3] = w5[3];
        o[4] = rPsi; o[5] = h - p / rho; o[6] = s;
        o[7] = tr.viscous ? tr.mu_of_T(T) + mut[i] : 0.0;     // muEff
    } else if (i < m.N + m.NB) {
        int b = i - m.N;
        const double* B = bs + BW * b;
        double rho = B[0], rhoE = B[4], p = B[5], T = B[6];
        double h = th.Cp * T;
        double rPsi = th.R * T;
        double s;
        if (use_c) s = sqrt(g * rPsi);
        else {
            double H = fmax(rhoE / rho, D_SMALL) + fmax(p / rho, D_SMALL);
            s = sqrt(2.0 * (g - 1.0) / (g + 1.0) * H);
        }
        double* o = qb + QW * b;
        o[0] = rho; o[1] = B[1]; o[2] = B[2]; o[3] = B[3];
        o[4] = rPsi; o[5] = h - p / rho; o[6] = s;
        o[7] = tr.viscous ? tr.mu_of_T(T) + mut_b[b] : 0.0;
    }
}

// Gauss linear gradient of the 7 recon fields (cell gather over the faces
// in foam order), plus optionally the Venkatakrishnan limiter per field and
// the HLLCP pressure-ratio sensor fCells (HLLCPDST.C:131-164).
__global__ void __launch_bounds__(128) k_grad(DevMesh m, int venkat_mask, double venkat_K, const double* __restrict__ q,
                                              const double* __restrict__ qb, const double* __restrict__ prim,
                                              double* __restrict__ g, double* __restrict__ psi,
                                              double* __restrict__ fcell, int hllcp, const double* __restrict__ bs,
                                              double* __restrict__ gU) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    double acc[21];
#pragma unroll
    for (int k = 0; k < 21; ++k) acc[k] = 0.0;
    const int k0 = m.cf_start[i], k1 = m.cf_start[i + 1];
    double fmin_c = 1.0;
    const double pi = prim[PW * i];
    double aU[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};    // (grad U)_ij = dU_j/dx_i
    for (int k = k0; k < k1; ++k) {
        int code = m.cf_list[k];
        if (code < m.Fi) {
            int f = code, o = m.own[f], n = m.nei[f];
            double wf = m.w[f];
            V3 S = ldv3(m.Sf, m.Fi, f);
            const double* qo = q + QW * o;
            const double* qn = q + QW * n;
            if (gU) {
                const double sg = (o == i) ? 1.0 : -1.0;
                const double Sv[3] = {sg * S.x, sg * S.y, sg * S.z};
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    double xf = wf * prim[PW * o + 3 + j] + (1 - wf) * prim[PW * n + 3 + j];
#pragma unroll
                    for (int d = 0; d < 3; ++d) aU[3 * d + j] += Sv[d] * xf;
                }
            }
            if (o == i) {
#pragma unroll
                for (int j = 0; j < 7; ++j) {
                    double xf = wf * qo[j] + (1 - wf) * qn[j];
                    acc[3 * j] += xf * S.x; acc[3 * j + 1] += xf * S.y; acc[3 * j + 2] += xf * S.z;
                }
            } else {
#pragma unroll
                for (int j = 0; j < 7; ++j) {
                    double xf = wf * qo[j] + (1 - wf) * qn[j];
                    acc[3 * j] -= xf * S.x; acc[3 * j + 1] -= xf * S.y; acc[3 * j + 2] -= xf * S.z;
                }
            }
            if (hllcp) {
                double pk = prim[PW * (o == i ? n : o)];
                fmin_c = fmin(fmin_c, fmin(pi / pk, pk / pi));
            }
        } else {
            int b = code - m.Fi;
            V3 S = ldv3(m.bSf, m.NB, b);
            const double* qq = qb + QW * b;
#pragma unroll
            for (int j = 0; j < 7; ++j) {
                double xf = qq[j];
                acc[3 * j] += xf * S.x; acc[3 * j + 1] += xf * S.y; acc[3 * j + 2] += xf * S.z;
            }
            if (gU) {
                const double Sv[3] = {S.x, S.y, S.z};
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int d = 0; d < 3; ++d) aU[3 * d + j] += Sv[d] * bs[BW * b + 12 + j];
            }
        }
    }
    const double Vi = m.V[i];
    if (gU) {
#pragma unroll
        for (int k = 0; k < 9; ++k) gU[9 * i + k] = aU[k] / Vi;
    }
    double* go = g + GW * i;
#pragma unroll
    for (int k = 0; k < 21; ++k) { acc[k] /= Vi; go[k] = acc[k]; }
    if (hllcp) fcell[i] = fmin_c;
    if (venkat_mask) {
        // Venkatakrishnan (1995): psi = min_f phi(dmax|dmin, d2), eps^2 = (K h)^3
        const double* qi = q + QW * i;
        double eps2 = pow(venkat_K * cbrt(Vi), 3.0);
        V3 Ci = ldv3(m.C, m.N, i);
        // unrolled: acc stays in registers (indexed by constants only)
#pragma unroll
        for (int j = 0; j < 7; ++j) {
            if (!((venkat_mask >> j) & 1)) { psi[QW * i + j] = 1.0; continue; }
            double x = qi[j], mx = x, mn = x;
            for (int k = k0; k < k1; ++k) {
                int code = m.cf_list[k];
                double xo;
                if (code < m.Fi) { int o = m.own[code]; xo = q[QW * (o == i ? m.nei[code] : o) + j]; }
                else xo = qb[QW * (code - m.Fi) + j];
                mx = fmax(mx, xo); mn = fmin(mn, xo);
            }
            double dmax = mx - x, dmin = mn - x, p = 1.0;
            V3 gj = mk(acc[3 * j], acc[3 * j + 1], acc[3 * j + 2]);
            for (int k = k0; k < k1; ++k) {
                int code = m.cf_list[k];
                V3 Cf = code < m.Fi ? ldv3(m.Cf, m.Fi, code) : ldv3(m.bCf, m.NB, code - m.Fi);
                double d2 = dot3(gj, sub3(Cf, Ci));
                double ph;
                if (d2 > 0) ph = ((dmax * dmax + eps2) * d2 + 2 * d2 * d2 * dmax) / (dmax * dmax + 2 * d2 * d2 + dmax * d2 + eps2) / d2;
                else if (d2 < 0) ph = ((dmin * dmin + eps2) * d2 + 2 * d2 * d2 * dmin) / (dmin * dmin + 2 * d2 * d2 + dmin * d2 + eps2) / d2;
                else ph = 1.0;
                p = fmin(p, ph);
            }
            psi[QW * i + j] = p;
        }
    }
}

// cellLimited Gauss linear k for grad(U) (foam-extend cellLimitedGrad of a
// vector field): per velocity component j, the spread maxD/minD of U_j over
// the cell's face neighbours and boundary values (widened by
// (1/k - 1)(maxD - minD) for k < 1), the limiter min over the cell's faces
// of maxD/d (d > maxD + VSMALL) or minD/d (d < minD - VSMALL) with
// d = (Cf - C) . grad U_j, and grad U_j scaled by it, in place (each thread
// reads its neighbours' velocities, not their gradients).
__global__ void __launch_bounds__(128) k_limit_gradU(DevMesh m, double k_lim, const double* __restrict__ prim,
                                                     const double* __restrict__ bs, double* __restrict__ gU) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    const int k0 = m.cf_start[i], k1 = m.cf_start[i + 1];
    double Ui[3], mx[3], mn[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) { Ui[j] = prim[PW * i + 3 + j]; mx[j] = Ui[j]; mn[j] = Ui[j]; }
    for (int k = k0; k < k1; ++k) {
        const int code = m.cf_list[k];
        const double* xo;
        if (code < m.Fi) { const int o = m.own[code]; xo = prim + PW * (o == i ? m.nei[code] : o) + 3; }
        else xo = bs + BW * (code - m.Fi) + 12;
#pragma unroll
        for (int j = 0; j < 3; ++j) { mx[j] = fmax(mx[j], xo[j]); mn[j] = fmin(mn[j], xo[j]); }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        mx[j] -= Ui[j];
        mn[j] -= Ui[j];
        if (k_lim < 1.0) {
            const double w = (1.0 / k_lim - 1.0) * (mx[j] - mn[j]);
            mx[j] += w;
            mn[j] -= w;
        }
    }
    double g[9], lim[3] = {1.0, 1.0, 1.0};
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = gU[9 * i + k];
    const V3 Ci = ldv3(m.C, m.N, i);
    for (int k = k0; k < k1; ++k) {
        const int code = m.cf_list[k];
        const V3 Cf = code < m.Fi ? ldv3(m.Cf, m.Fi, code) : ldv3(m.bCf, m.NB, code - m.Fi);
        const V3 d = sub3(Cf, Ci);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double e = d.x * g[j] + d.y * g[3 + j] + d.z * g[6 + j];
            if (e > mx[j] + D_VSMALL) lim[j] = fmin(lim[j], mx[j] / e);
            else if (e < mn[j] - D_VSMALL) lim[j] = fmin(lim[j], mn[j] / e);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int j = 0; j < 3; ++j) gU[9 * i + 3 * a + j] = g[3 * a + j] * lim[j];
}

// scalar limited reconstruction to the owner (xo) and neighbour (xn) sides
__device__ __forceinline__ void recon_scalar(int L, double xP, double xN, V3 gP, V3 gN, V3 d, double w,
                                             double& xo, double& xn) {
    double ro = 0, rn = 0;
    if (L != L_LINEAR && L != L_UPWIND) {
        double gradf = xN - xP;
        ro = nvd_r(dot3(d, gP), gradf);
        rn = nvd_r(dot3(d, gN), gradf);
    }
    double wo = side_w(L, true, w, ro), wn = side_w(L, false, w, rn);
    xo = wo * xP + (1 - wo) * xN;
    xn = wn * xP + (1 - wn) * xN;
}

// Limited reconstruction of the seven recon fields to the owner (so) and
// neighbour (sn) sides of internal face f (foam limitedSurfaceInterpolation
// with NVDTVD r, V-limiters for rhoU, or Venkatakrishnan).
__device__ __forceinline__ void face_recon(const DevMesh& m, int f, int lr, int lu, int lt,
                                           const double* __restrict__ q, const double* __restrict__ g,
                                           const double* __restrict__ psi, SideState& so, SideState& sn) {
    const int o = m.own[f], n = m.nei[f];
    const double wf = m.w[f];
    const double* qo = q + QW * o;
    const double* qn = q + QW * n;
    const int Ls[7] = {lr, lu, lu, lu, lt, lt, lt};
    if (lr == L_VENKAT || lu == L_VENKAT || lt == L_VENKAT) {
        // all fields Venkatakrishnan-limited or linear/upwind (parse enforces a
        // single family per case)
        V3 Cf = ldv3(m.Cf, m.Fi, f);
        V3 dP = sub3(Cf, ldv3(m.C, m.N, o)), dN = sub3(Cf, ldv3(m.C, m.N, n));
        double xo[7], xn[7];
        for (int j = 0; j < 7; ++j) {
            if (Ls[j] == L_VENKAT) {
                const double* gP = g + GW * o + 3 * j;
                const double* gN = g + GW * n + 3 * j;
                xo[j] = qo[j] + psi[QW * o + j] * (dP.x * gP[0] + dP.y * gP[1] + dP.z * gP[2]);
                xn[j] = qn[j] + psi[QW * n + j] * (dN.x * gN[0] + dN.y * gN[1] + dN.z * gN[2]);
            } else {
                recon_scalar(Ls[j], qo[j], qn[j], mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0), wf, xo[j], xn[j]);
            }
        }
        so.rho = xo[0]; so.rhoU = mk(xo[1], xo[2], xo[3]); so.rPsi = xo[4]; so.e = xo[5]; so.s = xo[6];
        sn.rho = xn[0]; sn.rhoU = mk(xn[1], xn[2], xn[3]); sn.rPsi = xn[4]; sn.e = xn[5]; sn.s = xn[6];
    } else {
        const V3 d = ldv3(m.d, m.Fi, f);
        const bool lim = (lr > L_UPWIND) || (lu > L_UPWIND) || (lt > L_UPWIND);
        const double* gP = g + GW * o;
        const double* gN = g + GW * n;
        auto GV = [&](const double* gg, int j) { return lim ? mk(gg[3 * j], gg[3 * j + 1], gg[3 * j + 2]) : mk(0, 0, 0); };
        recon_scalar(lr, qo[0], qn[0], GV(gP, 0), GV(gN, 0), d, wf, so.rho, sn.rho);
        recon_scalar(lt, qo[4], qn[4], GV(gP, 4), GV(gN, 4), d, wf, so.rPsi, sn.rPsi);
        recon_scalar(lt, qo[5], qn[5], GV(gP, 5), GV(gN, 5), d, wf, so.e, sn.e);
        recon_scalar(lt, qo[6], qn[6], GV(gP, 6), GV(gN, 6), d, wf, so.s, sn.s);
        // rhoU with the vector (V) limiter: r from the projection on phi_N - phi_P
        double ro = 0, rn = 0;
        V3 xP = mk(qo[1], qo[2], qo[3]), xN = mk(qn[1], qn[2], qn[3]);
        if (lu > L_UPWIND) {
            V3 gradfV = sub3(xN, xP);
            double gradf = dot3(gradfV, gradfV);
            // (d . grad U)_j = sum_i d_i dU_j/dx_i ; field j = 1+comp, direction i
            V3 dgP = mk(d.x * gP[3] + d.y * gP[4] + d.z * gP[5], d.x * gP[6] + d.y * gP[7] + d.z * gP[8],
                        d.x * gP[9] + d.y * gP[10] + d.z * gP[11]);
            V3 dgN = mk(d.x * gN[3] + d.y * gN[4] + d.z * gN[5], d.x * gN[6] + d.y * gN[7] + d.z * gN[8],
                        d.x * gN[9] + d.y * gN[10] + d.z * gN[11]);
            ro = nvd_r(dot3(gradfV, dgP), gradf);
            rn = nvd_r(dot3(gradfV, dgN), gradf);
        }
        double wo = side_w(lu, true, wf, ro), wn = side_w(lu, false, wf, rn);
        so.rhoU = add3(scl3(wo, xP), scl3(1 - wo, xN));
        sn.rhoU = add3(scl3(wn, xP), scl3(1 - wn, xN));
    }
}

// Face fluxes of all internal faces (reconstruction + scheme), AoS output.
__global__ void __launch_bounds__(128, 4) k_face_flux(DevMesh m, Thermo th, int scheme, int lr, int lu, int lt,
                                                   int lowMach, double Mainf, const double* __restrict__ q,
                                                   const double* __restrict__ g, const double* __restrict__ psi,
                                                   const double* __restrict__ fcell, double* __restrict__ fl,
                                                   double* __restrict__ up) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.Fi) return;
    const int o = m.own[f], n = m.nei[f];
    const double wf = m.w[f];
    const V3 S = ldv3(m.Sf, m.Fi, f);
    const double magS = m.magSf[f];
    SideState so, sn;
    face_recon(m, f, lr, lu, lt, q, g, psi, so, sn);
    double fs = 1.0;
    if (scheme == F_HLLCP) fs = wf * pow(fcell[o], 3.0) + (1 - wf) * pow(fcell[n], 3.0);
    FFlux F = face_flux(scheme, so, sn, S, magS, th.gamma, fs, lowMach != 0, Mainf);
    double* out = fl + 5 * f;
    out[0] = F.phi; out[1] = F.phiUp.x; out[2] = F.phiUp.y; out[3] = F.phiUp.z; out[4] = F.phiEp;
    if (up) { up[3 * f] = F.Up.x; up[3 * f + 1] = F.Up.y; up[3 * f + 2] = F.Up.z; }
}

// Boundary face fluxes: both sides carry the boundary value (foam
// interpolate() returns the patch value on non-coupled patches).
__global__ void k_bface_flux(DevMesh m, Thermo th, int scheme, int lowMach, double Mainf, const double* __restrict__ qb,
                             double* __restrict__ bfl, double* __restrict__ bs, double* __restrict__ bup) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const double* qq = qb + QW * b;
    SideState s;
    s.rho = qq[0]; s.rhoU = mk(qq[1], qq[2], qq[3]); s.rPsi = qq[4]; s.e = qq[5]; s.s = qq[6];
    FFlux F = face_flux(scheme, s, s, ldv3(m.bSf, m.NB, b), m.bmagSf[b], th.gamma, 1.0, lowMach != 0, Mainf);
    double* out = bfl + 5 * b;
    out[0] = F.phi; out[1] = F.phiUp.x; out[2] = F.phiUp.y; out[3] = F.phiUp.z; out[4] = F.phiEp;
    bs[BW * b + 7] = F.phi;
    if (bup) { bup[3 * b] = F.Up.x; bup[3 * b + 1] = F.Up.y; bup[3 * b + 2] = F.Up.z; }
}

// tau = muEff dev2(T(grad U)): t(i,j) = mu (g(j,i) - 2/3 tr(g) d_ij)
template <typename T>
__device__ __forceinline__ void tau_of(const T (&g)[9], const T& mu, T (&t)[9]) {
    const T tr = g[0] + g[4] + g[8];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T a = g[3 * j + i];
            if (i == j) a = a - (2.0 / 3.0) * tr;
            t[3 * i + j] = mu * a;
        }
}

// Viscous terms of one internal face (baseFluxDST.C:229-250): lap = muEff_f
// |Sf| snGrad(U) (corrected: dc (U_N - U_P) + (n - d dc) . (grad U)_f),
// tauS = Sf . (tau)_f, sig = (lap + tauS) . Up; out = (lap[3], tauS[3], sig).
// Inputs: cell velocities, velocity gradients (g_ij = dU_j/dx_i), muEff of
// both cells and the face velocity Up of the convective flux.
template <typename T>
__device__ __forceinline__ void visc_face(const V3& S, double magS, double w, double dc, const V3& kc, const T (&UP)[3],
                                          const T (&UQ)[3], const T (&gP)[9], const T (&gQ)[9], const T& muP,
                                          const T& muQ, const T (&Up)[3], T (&out)[7]) {
    const T muf = w * muP + (1 - w) * muQ;
    T tP[9], tQ[9];
    tau_of(gP, muP, tP);
    tau_of(gQ, muQ, tQ);
    const double kv[3] = {kc.x, kc.y, kc.z}, Sv[3] = {S.x, S.y, S.z};
    T lap[3], ts[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        T corr(0.0), a(0.0);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            corr += kv[i] * (w * gP[3 * i + j] + (1 - w) * gQ[3 * i + j]);
            a += Sv[i] * (w * tP[3 * i + j] + (1 - w) * tQ[3 * i + j]);
        }
        const T sn = dc * (UQ[j] - UP[j]) + corr;
        lap[j] = (muf * magS) * sn;
        ts[j] = a;
    }
    out[6] = (lap[0] + ts[0]) * Up[0] + (lap[1] + ts[1]) * Up[1] + (lap[2] + ts[2]) * Up[2];
#pragma unroll
    for (int j = 0; j < 3; ++j) { out[j] = lap[j]; out[3 + j] = ts[j]; }
}

// Viscous terms of one boundary face: snGrad = (U_b - U_P) dc_b, the cell
// gradient corrected to the patch snGrad (gaussGrad::correctBoundaryConditions),
// tau_b from muEff_b.  Same outputs as visc_face.
template <typename T>
__device__ __forceinline__ void visc_bface(const V3& S, double magS, double dc, const T (&Ub)[3], const T (&UP)[3],
                                           const T (&gP)[9], const T& mub, const T (&Up)[3], T (&out)[7]) {
    const double n[3] = {S.x / magS, S.y / magS, S.z / magS}, Sv[3] = {S.x, S.y, S.z};
    T snb[3], g[9], t[9];
#pragma unroll
    for (int j = 0; j < 3; ++j) snb[j] = dc * (Ub[j] - UP[j]);
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = gP[k];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const T ng = n[0] * g[j] + n[1] * g[3 + j] + n[2] * g[6 + j];
#pragma unroll
        for (int i = 0; i < 3; ++i) g[3 * i + j] += n[i] * (snb[j] - ng);
    }
    tau_of(g, mub, t);
    T lap[3], ts[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        ts[j] = Sv[0] * t[j] + Sv[1] * t[3 + j] + Sv[2] * t[6 + j];
        lap[j] = (mub * magS) * snb[j];
    }
    out[6] = (lap[0] + ts[0]) * Up[0] + (lap[1] + ts[1]) * Up[1] + (lap[2] + ts[2]) * Up[2];
#pragma unroll
    for (int j = 0; j < 3; ++j) { out[j] = lap[j]; out[3 + j] = ts[j]; }
}

// Viscous face terms per internal face (visc_face on the cell records).
__global__ void __launch_bounds__(128) k_visc_faces(DevMesh m, const double* __restrict__ q, const double* __restrict__ prim,
                                                    const double* __restrict__ gU, const double* __restrict__ up,
                                                    double* __restrict__ vf) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.Fi) return;
    const int P = m.own[f], Q = m.nei[f];
    const double dc = m.dc[f], magS = m.magSf[f];
    const V3 S = ldv3(m.Sf, m.Fi, f);
    const V3 kc = sub3(div3(S, magS), scl3(dc, ldv3(m.d, m.Fi, f)));
    double UP[3], UQ[3], gP[9], gQ[9], Up[3], out[7];
#pragma unroll
    for (int j = 0; j < 3; ++j) { UP[j] = prim[PW * P + 3 + j]; UQ[j] = prim[PW * Q + 3 + j]; Up[j] = up[3 * f + j]; }
#pragma unroll
    for (int k = 0; k < 9; ++k) { gP[k] = gU[9 * P + k]; gQ[k] = gU[9 * Q + k]; }
    visc_face(S, magS, m.w[f], dc, kc, UP, UQ, gP, gQ, q[QW * P + 7], q[QW * Q + 7], Up, out);
    double* o = vf + 8 * f;
#pragma unroll
    for (int k = 0; k < 7; ++k) o[k] = out[k];
}

// boundary faces (visc_bface on the boundary record and the cell's records)
__global__ void k_visc_bfaces(DevMesh m, const double* __restrict__ qb, const double* __restrict__ prim,
                              const double* __restrict__ gU, const double* __restrict__ bs,
                              const double* __restrict__ bup, double* __restrict__ bvf) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const int P = m.bcell[b];
    const double* B = bs + BW * b;
    double Ub[3], UP[3], gP[9], Up[3], out[7];
#pragma unroll
    for (int j = 0; j < 3; ++j) { Ub[j] = B[12 + j]; UP[j] = prim[PW * P + 3 + j]; Up[j] = bup[3 * b + j]; }
#pragma unroll
    for (int k = 0; k < 9; ++k) gP[k] = gU[9 * P + k];
    visc_bface(ldv3(m.bSf, m.NB, b), m.bmagSf[b], m.bdc[b], Ub, UP, gP, qb[QW * b + 7], Up, out);
    double* o = bvf + 8 * b;
#pragma unroll
    for (int k = 0; k < 7; ++k) o[k] = out[k];
}

// calcFields (baseFluxDST.C:223-255): R = div(face fluxes) per unit volume,
// gathered per cell in foam face order; rhs = -R V (fluxDST.C:124); fused
// partial sums for |R|^2 (timeDST.C:330) and (R V)^2 per component.
__global__ void k_residual(DevMesh m, const double* __restrict__ fl, const double* __restrict__ bfl,
                           const double* __restrict__ vf, const double* __restrict__ bvf,
                           double* __restrict__ R, double* __restrict__ rhs, double* __restrict__ partial) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double r[5] = {0, 0, 0, 0, 0};
    double vs[7] = {0, 0, 0, 0, 0, 0, 0};
    double sq_mag = 0, sq_c[5] = {0, 0, 0, 0, 0};
    if (i < m.N) {
        for (int k = m.cf_start[i]; k < m.cf_start[i + 1]; ++k) {
            int code = m.cf_list[k];
            const double* F;
            const double* Fv = nullptr;
            double sg = 1.0;
            if (code < m.Fi) {
                F = fl + 5 * code;
                sg = (m.own[code] == i) ? 1.0 : -1.0;
                if (vf) Fv = vf + 8 * code;
            } else {
                F = bfl + 5 * (code - m.Fi);
                if (bvf) Fv = bvf + 8 * (code - m.Fi);
            }
#pragma unroll
            for (int c = 0; c < 5; ++c) r[c] += sg * F[c];
            if (Fv) {
#pragma unroll
                for (int c = 0; c < 7; ++c) vs[c] += sg * Fv[c];
            }
        }
        double Vi = m.V[i];
        double Rv[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) Rv[c] = r[c] / Vi;
        if (vf) {
            // R_U -= laplacian(muEff,U) + div(tauMC); R_E -= div(sigmaDotU)
#pragma unroll
            for (int k = 0; k < 3; ++k) Rv[1 + k] -= vs[k] / Vi + vs[3 + k] / Vi;
            Rv[4] -= vs[6] / Vi;
        }
        if (m.rmask && m.rmask[i]) {
#pragma unroll
            for (int c = 0; c < 5; ++c) Rv[c] = 0.0;
        }
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            double Rc = Rv[c];
            R[5 * i + c] = Rc;
            double rv = Rc * Vi;
            rhs[5 * i + c] = 0.0 - rv;
            sq_mag += Rc * Rc;
            sq_c[c] = rv * rv;
        }
    }
    double v = block_sum(sq_mag);
    if (threadIdx.x == 0) partial[blockIdx.x * 6] = v;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        v = block_sum(sq_c[c]);
        if (threadIdx.x == 0) partial[blockIdx.x * 6 + 1 + c] = v;
    }
}

// one block: each thread sums a fixed stride of the partials, then a
// fixed-order block reduction (deterministic)
__global__ void k_residual_finalize(const double* __restrict__ partial, int nb, Scalars* sc) {
    for (int c = 0; c < 6; ++c) {
        double s = 0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[b * 6 + c];
        s = block_sum(s);
        if (threadIdx.x == 0) {
            if (c == 0) sc->res_mag = sqrt(s);
            else sc->res_l2[c - 1] = sqrt(s);
        }
    }
}

// ------------------------------------------------------------------ assembly
__device__ __forceinline__ size_t sidx(const int* slice_off, int r, int k, int e) {
    size_t slot = (size_t)slice_off[r >> 5] + k;
    return slot * (32 * 25) + (size_t)e * 32 + (r & 31);
}

// Entry e of the convective flux Jacobian calcJ (physics.cuh) with the same
// operations, for a loop that needs one entry at a time (e a constant after
// unrolling): no 25-entry array stays live.
__device__ __forceinline__ double calcJ_entry(int e, const V3& Uf, double gammaf, double phiJf, double a1f,
                                              const V3& n, double Un) {
    const double U[3] = {Uf.x, Uf.y, Uf.z};
    const double N[3] = {n.x, n.y, n.z};
    const int i = e / 5, c = e % 5;
    if (i == 0) return (c >= 1 && c <= 3) ? N[c - 1] : 0.0;
    if (i == 4) {
        if (c == 0) return Un * (phiJf - a1f);
        if (c == 4) return gammaf * Un;
        return a1f * N[c - 1] - Un * (gammaf - 1) * U[c - 1];
    }
    const int k = i - 1;
    if (c == 0) return phiJf * N[k] - U[k] * Un;
    if (c == 4) return (gammaf - 1) * N[k];
    const int l = c - 1;
    return U[k] * N[l] + (k == l ? Un : 0.0) - (gammaf - 1) * (N[k] * U[l]);
}

// Roe::computeBoundaryJacobians (Roe.C:274-379), one thread per active
// boundary face: the block (dR/dX) diag(valueInternalCoeffs) (dX/dW) that
// k_assemble adds to the diagonal of the face's cell.
__global__ void k_bjac(DevMesh m, Thermo th, const double* __restrict__ W, const double* __restrict__ prim,
                       const double* __restrict__ bs, double* __restrict__ bjac) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.NB) return;
    const int r = m.bcell[b];
    const DevPatch P = m.patches[m.bpatch[b]];
    const double* B = bs + BW * b;
    const V3 pSf = ldv3(m.bSf, m.NB, b);
    const V3 nrm = div3(pSf, m.bmagSf[b]);
    V3 UB = div3(mk(B[1], B[2], B[3]), B[0]);
    double pB = B[5], TB = B[6], rhoB = B[0], EB = B[4] / B[0];
    double rRT = rhoB / pB;
    double UBS = dot3(UB, pSf);
    const double Sv[3] = {pSf.x, pSf.y, pSf.z}, Uv[3] = {UB.x, UB.y, UB.z};
    double dR[25];
    dR[0] = UBS * rRT;
    for (int k2 = 0; k2 < 3; ++k2) dR[1 + k2] = rhoB * Sv[k2];
    dR[4] = -rhoB / TB * UBS;
    for (int k2 = 0; k2 < 3; ++k2) {
        dR[(1 + k2) * 5 + 0] = rRT * UBS * Uv[k2] + Sv[k2];
        for (int l = 0; l < 3; ++l) dR[(1 + k2) * 5 + 1 + l] = rhoB * Uv[k2] * Sv[l] + (k2 == l ? rhoB * UBS : 0.0);
        dR[(1 + k2) * 5 + 4] = -rhoB / TB * UBS * Uv[k2];
    }
    dR[20] = (EB * rRT + 1) * UBS;
    for (int l = 0; l < 3; ++l) dR[21 + l] = rhoB * UBS * Uv[l] + Sv[l] * (rhoB * EB + pB);
    dR[24] = rhoB * th.Cv * UBS;
    // dX/dW at the internal cell
    const double* w5 = W + 5 * r;
    const V3 UI = div3(mk(w5[1], w5[2], w5[3]), w5[0]);
    const double UIv[3] = {UI.x, UI.y, UI.z};
    double rhoEI = w5[4], pI = prim[PW * r], rRho = 1.0 / w5[0];
    double rRhoCv = rRho / th.Cv;
    double e = rhoEI * rRho - 0.5 * magSqr3(UI);
    double RT = pI * rRho;
    double RCv = RT / e;
    double dX[25];
#pragma unroll
    for (int q2 = 0; q2 < 25; ++q2) dX[q2] = 0.0;
    dX[0] = RT - RCv * (e - 0.5 * magSqr3(UI));
    for (int l = 0; l < 3; ++l) dX[1 + l] = -RCv * UIv[l];
    dX[4] = RCv;
    for (int k2 = 0; k2 < 3; ++k2) { dX[(1 + k2) * 5] = -rRho * UIv[k2]; dX[(1 + k2) * 5 + 1 + k2] = rRho; }
    dX[20] = rRhoCv * (0.5 * magSqr3(UI) - e);
    for (int l = 0; l < 3; ++l) dX[21 + l] = -rRhoCv * UIv[l];
    dX[24] = rRhoCv;
    // valueInternalCoeffs: 1 - valueFraction (mixed types), basicSymmetry
    double cdiag[5];
    cdiag[0] = 1.0 - B[8];
    cdiag[4] = 1.0 - B[10];
    if (P.bc_U == 3 || P.bc_U == 4) {
        cdiag[1] = 1 - fabs(nrm.x); cdiag[2] = 1 - fabs(nrm.y); cdiag[3] = 1 - fabs(nrm.z);
    } else { cdiag[1] = cdiag[2] = cdiag[3] = 1.0 - B[9]; }
    // pic = (dR . diag(cdiag)) . dX
    for (int a = 0; a < 5; ++a) {
        double t1[5];
        for (int c2 = 0; c2 < 5; ++c2) {
            double acc2 = 0;
            for (int k2 = 0; k2 < 5; ++k2) acc2 += dR[5 * a + k2] * (k2 == c2 ? cdiag[k2] : 0.0);
            t1[c2] = acc2;
        }
        for (int c2 = 0; c2 < 5; ++c2) {
            double acc2 = 0;
            for (int k2 = 0; k2 < 5; ++k2) acc2 += t1[k2] * dX[5 * k2 + c2];
            bjac[25 * (size_t)b + 5 * a + c2] = acc2;
        }
    }
}

// Roe Jacobian blocks (Roe.C:152-214) assembled straight into the SELL
// matrix, one row (cell) per thread: off-diagonal (row, column) blocks from
// the face's upper (row = owner) / lower (row = neighbour) coefficient,
// the diagonal as ddt + negSumDiag + boundary Jacobians (fluxDST.C:98-112,
// the latter from k_bjac), accumulated in foam face order.  The flux
// Jacobians of the two cells are formed entry by entry inside the block
// loop, which keeps a thread's registers to about the diagonal block.
template <typename MT>
__global__ void __launch_bounds__(128, 4) k_assemble(DevMesh m, Thermo th, Transport tr, SellMat<MT> A,
                                                     const int* __restrict__ cf_slot,
                                                     const double* __restrict__ W, const double* __restrict__ prim,
                                                     const double* __restrict__ bjac, const double* __restrict__ rdtc,
                                                     const double* __restrict__ mut,
                                                     const Scalars* __restrict__ sc, int steady, double beta,
                                                     double dual_a) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m.N) return;
    const double g = th.gamma;
    double D[25];
    {
        // local pseudo-time (steady, dual: + a of dual2ndDST, dual2ndDST.C:397)
        // or the global physical step
        double dg = (steady ? rdtc[r] + dual_a : 1.0 / sc->deltaT) * m.V[r];
#pragma unroll
        for (int e = 0; e < 25; ++e) D[e] = (e % 6 == 0) ? dg : 0.0;
    }
    auto cellJ = [&](int c, V3& U, double& phiJ, double& a1, double& cs) {
        const double* w5 = W + 5 * c;
        U = div3(mk(w5[1], w5[2], w5[3]), w5[0]);
        phiJ = 0.5 * (g - 1) * magSqr3(U);
        a1 = g * w5[4] / w5[0] - phiJ;
        cs = sqrt(g * th.R * prim[PW * c + 1]);
    };
    V3 Ur;
    double phiJr, a1r, cr;
    cellJ(r, Ur, phiJr, a1r, cr);
    for (int k = m.cf_start[r]; k < m.cf_start[r + 1]; ++k) {
        int code = m.cf_list[k];
        if (code < m.Fi) {
            const int f = code, o = m.own[f], n = m.nei[f];
            const bool isOwner = (o == r);
            const int oc_ = isOwner ? n : o;
            V3 Uc;
            double phiJc, a1c, cc;
            cellJ(oc_, Uc, phiJc, a1c, cc);
            const double wf = m.w[f];
            const V3 S = ldv3(m.Sf, m.Fi, f);
            const double magS = m.magSf[f];
            const V3 nn = div3(S, magS);
            V3 Uo = isOwner ? Ur : Uc, Un = isOwner ? Uc : Ur;
            double co = isOwner ? cr : cc, cn = isOwner ? cc : cr;
            V3 Uf = add3(scl3(wf, Uo), scl3(1 - wf, Un));
            double cf = wf * co + (1 - wf) * cn;
            double amaxSf = fabs(dot3(Uf, S)) + magS * cf;
            double lambda;
            if (tr.viscous) {
                // + |Sf| (muEff_f + alphaEff_f)/rho_f deltaCoeffs (Roe.C:187-199)
                const int Po = isOwner ? r : oc_, Qn = isOwner ? oc_ : r;
                double TP = prim[PW * Po + 1], TQ = prim[PW * Qn + 1];
                double mP = tr.mu_of_T(TP), mQ = tr.mu_of_T(TQ);
                double muEf = wf * (mP + mut[Po]) + (1 - wf) * (mQ + mut[Qn]);
                double alEf = wf * (mP / tr.Pr + mut[Po] / tr.Prt) + (1 - wf) * (mQ / tr.Pr + mut[Qn] / tr.Prt);
                double rhof = wf * prim[PW * Po] / (th.R * TP) + (1 - wf) * prim[PW * Qn] / (th.R * TQ);
                lambda = 0.5 * (amaxSf + magS * (muEf + alEf) / rhof * m.dc[f]);
            } else {
                lambda = 0.5 * amaxSf;
            }
            const double Unr = dot3(Ur, nn), Unc = dot3(Uc, nn);
            const int cs = cf_slot[k];
            const bool accum = cs < 0;          // further face of an already written cell pair
            const int slot = accum ? -cs - 1 : cs;
            MT* p0 = &A.val[sidx(A.slice_off, r, slot, 0)];
            // owner row: D -= lower(J_r), A_rc = upper(J_c); neighbour row:
            // D -= upper(J_r), A_rc = lower(J_c)
            const double wr = isOwner ? wf : 1 - wf, wc = isOwner ? 1 - wf : wf;
#pragma unroll
            for (int e = 0; e < 25; ++e) {
                const double I = (e % 6 == 0) ? 1.0 : 0.0;
                const double J = calcJ_entry(e, Ur, g, phiJr, a1r, nn, Unr);
                const double Jc = calcJ_entry(e, Uc, g, phiJc, a1c, nn, Unc);
                double dsub, offd;
                if (isOwner) {
                    dsub = -beta * ((J * wr) * magS + I * lambda);
                    offd = beta * ((Jc * wc) * magS - I * lambda);
                } else {
                    dsub = beta * ((J * wr) * magS - I * lambda);
                    offd = -beta * ((Jc * wc) * magS + I * lambda);
                }
                D[e] -= dsub;
                MT* p = p0 + e * 32;
                st(p, accum ? ld(p) + offd : offd);
            }
        } else {
            const double* pj = bjac + 25 * (size_t)(code - m.Fi);
#pragma unroll
            for (int e = 0; e < 25; ++e) D[e] += beta * pj[e];
        }
    }
#pragma unroll
    for (int e = 0; e < 25; ++e) st(&A.val[sidx(A.slice_off, r, 0, e)], D[e]);
}

// ------------------------------------------------------------------ update
// updateFields.H:40-94: W += dW, bound rho/h/p, U = rhoU/rho,
// h = Cp/Cv (rhoE/rho - |U|^2/2), T = h/Cp, p = rho R T.
__global__ void k_update(int N, Thermo th, Bounds bd, const double* __restrict__ dx, double* __restrict__ W,
                         double* __restrict__ prim, Scalars* sc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int flag = 0;
    if (i < N) {
        double* w5 = W + 5 * i;
        double rho = w5[0] + dx[5 * i + 0];
        double rUx = w5[1] + dx[5 * i + 1], rUy = w5[2] + dx[5 * i + 2], rUz = w5[3] + dx[5 * i + 3];
        double rhoE = w5[4] + dx[5 * i + 4];
        if (rho < bd.rho_min) { rho = bd.rho_min; flag = 1; }
        if (rho > bd.rho_max) { rho = bd.rho_max; flag = 1; }
        V3 U = div3(mk(rUx, rUy, rUz), rho);
        double hh = th.Cp / th.Cv * (rhoE / rho - 0.5 * magSqr3(U));
        double h = hh;
        if (h < th.Cp * bd.T_min) { h = th.Cp * bd.T_min; flag = 1; }
        if (h > th.Cp * bd.T_max) { h = th.Cp * bd.T_max; flag = 1; }
        double T = h / th.Cp;
        double p = rho * th.R * T;
        if (p < bd.p_min) { p = bd.p_min; flag = 1; }
        if (p > bd.p_max) { p = bd.p_max; flag = 1; }
        if (!(rho > 0) || !(p > 0) || !isfinite(rhoE) || !isfinite(rho)) flag |= 2;
        w5[0] = rho; w5[1] = rUx; w5[2] = rUy; w5[3] = rUz; w5[4] = rhoE;
        double* P = prim + PW * i;
        P[0] = p; P[1] = T; P[2] = h; P[3] = U.x; P[4] = U.y; P[5] = U.z;
    }
    unsigned b = __ballot_sync(0xffffffffu, flag & 1), d = __ballot_sync(0xffffffffu, flag & 2);
    if ((threadIdx.x & 31) == 0 && (b | d)) atomicOr(&sc->flags, (b ? 1 : 0) | (d ? 2 : 0));
}

// ------------------------------------------------------------------ time control
// timeDST::setTransientDeltaT (timeDST.C:275-314): per-face (neighbouring)
// or per-cell (Blazek) stable step, reduced with min.
__global__ void k_dt_transient(DevMesh m, Thermo th, int neighbouring, const double* __restrict__ prim,
                               const double* __restrict__ dS, const Scalars* sc, double* partial) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double g = th.gamma, courant = sc->courant;
    double v = 1e300;
    if (neighbouring) {
        if (i < m.Fi) {
            int P = m.own[i], Q = m.nei[i];
            double wf = m.w[i];
            V3 UP = mk(prim[PW * P + 3], prim[PW * P + 4], prim[PW * P + 5]);
            V3 UQ = mk(prim[PW * Q + 3], prim[PW * Q + 4], prim[PW * Q + 5]);
            V3 Uf = add3(scl3(wf, UP), scl3(1 - wf, UQ));
            double cf = wf * sqrt(g * th.R * prim[PW * P + 1]) + (1 - wf) * sqrt(g * th.R * prim[PW * Q + 1]);
            V3 S = ldv3(m.Sf, m.Fi, i);
            double amaxSf = fabs(dot3(Uf, S)) + m.magSf[i] * cf;
            double dtSf = m.magSf[i] / (amaxSf * m.dc[i]);
            v = dtSf * courant;
        }
    } else if (i < m.N) {
        double cs = sqrt(g * th.R * prim[PW * i + 1]);
        double lambdaC = (fabs(prim[PW * i + 3]) + cs) * dS[3 * i] + (fabs(prim[PW * i + 4]) + cs) * dS[3 * i + 1] +
                         (fabs(prim[PW * i + 5]) + cs) * dS[3 * i + 2];
        v = courant * m.V[i] / lambdaC;
    }
    v = block_min(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
}

__global__ void k_dt_finalize(const double* partial, int nb, Scalars* sc) {
    double v = 1e300;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v = fmin(v, partial[b]);
    v = block_min(v);
    if (threadIdx.x == 0) sc->deltaT = v;
}

// setSteadyStateDeltaT (timeDST.C:218-273): local 1/dtau per cell
__global__ void k_dt_steady(DevMesh m, Thermo th, int neighbouring, const double* __restrict__ prim,
                            const double* __restrict__ dS, const double* __restrict__ courantF,
                            const Scalars* __restrict__ sc, double* __restrict__ rdt, double* partial) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double g = th.gamma;
    double v = 0;
    double lo = 1e300, hi = -1e300;
    if (i < m.N) {
        if (!neighbouring) {
            double cs = sqrt(g * th.R * prim[PW * i + 1]);
            double lambdaC = (fabs(prim[PW * i + 3]) + cs) * dS[3 * i] + (fabs(prim[PW * i + 4]) + cs) * dS[3 * i + 1] +
                             (fabs(prim[PW * i + 5]) + cs) * dS[3 * i + 2];
            // the scalar courant (timeDST.C:221-227), not the ramped per-cell field
            v = lambdaC / (sc->courant * m.V[i]);
        } else {
            for (int k = m.cf_start[i]; k < m.cf_start[i + 1]; ++k) {
                int code = m.cf_list[k];
                if (code < m.Fi) {
                    int P = m.own[code], Q = m.nei[code];
                    double wf = m.w[code];
                    V3 UP = mk(prim[PW * P + 3], prim[PW * P + 4], prim[PW * P + 5]);
                    V3 UQ = mk(prim[PW * Q + 3], prim[PW * Q + 4], prim[PW * Q + 5]);
                    V3 Uf = add3(scl3(wf, UP), scl3(1 - wf, UQ));
                    double cf = wf * sqrt(g * th.R * prim[PW * P + 1]) + (1 - wf) * sqrt(g * th.R * prim[PW * Q + 1]);
                    v = fmax(v, (sqrt(magSqr3(Uf)) + cf) * m.dc[code]);
                } else {
                    int b = code - m.Fi;
                    if (m.patches[m.bpatch[b]].type != 1) continue;
                    double pl = 0.5 * m.bdc[b] * sqrt(g * th.R * prim[PW * i + 1]) +
                                sqrt(magSqr3(mk(prim[PW * i + 3], prim[PW * i + 4], prim[PW * i + 5])));
                    v = fmax(v, pl);
                }
            }
            v /= courantF[i];
        }
        rdt[i] = v;
        lo = hi = v;
    }
    lo = block_min(lo);
    if (threadIdx.x == 0) partial[2 * blockIdx.x] = lo;
    hi = block_max(hi);
    if (threadIdx.x == 0) partial[2 * blockIdx.x + 1] = hi;
}

__global__ void k_rdt_finalize(const double* partial, int nb, Scalars* sc) {
    double lo = 1e300, hi = -1e300;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) { lo = fmin(lo, partial[2 * b]); hi = fmax(hi, partial[2 * b + 1]); }
    lo = block_min(lo);
    hi = block_max(hi);
    if (threadIdx.x == 0) { sc->rdt_min = lo; sc->rdt_max = hi; }
}

// setCourantDST (timeDST.C:316-443) scalar part: residual-ratio CFL ramp
__global__ void k_courant_scalar(Scalars* sc, int transient_adjust, double min_co, double max_co) {
    if (threadIdx.x != 0) return;
    double residualR = sc->res_mag;
    if (sc->residual != -1) sc->residualRatio = fmin(fmax(sc->residual / residualR, 0.1), 2.0);
    sc->residual = residualR;
    if (transient_adjust) sc->courant = fmin(fmax(sc->courant * sc->residualRatio, min_co), max_co);
}

// steady branch: per-cell CFL cut on rho / e drops (HiSA rule) and ramp
__global__ void k_courant_cells(DevMesh m, const double* __restrict__ W, double* __restrict__ rhoOld,
                                double* __restrict__ eOld, double* __restrict__ courantF, const Scalars* sc,
                                double min_co, double max_co, double* __restrict__ eNewBuf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    auto eN = [&](int c) {
        const double* w5 = W + 5 * c;
        V3 U = div3(mk(w5[1], w5[2], w5[3]), w5[0]);
        return w5[4] / w5[0] - 0.5 * magSqr3(U);
    };
    auto drop = [&](int c) {
        double e = eN(c);
        return W[5 * c] < 0.95 * rhoOld[c] || e < 0.95 * eOld[c] || e < D_SMALL;
    };
    double factor = 1.0;
    bool di = drop(i);
    for (int k = m.cf_start[i]; k < m.cf_start[i + 1]; ++k) {
        int code = m.cf_list[k];
        if (code >= m.Fi) continue;
        int o = m.own[code], other = (o == i) ? m.nei[code] : o;
        if (di) factor = fmin(factor, 0.5);
        if (drop(other)) factor = fmin(factor, 0.75);
    }
    eNewBuf[i] = eN(i);
    courantF[i] = fmin(fmax(courantF[i] * sc->residualRatio * factor, min_co), max_co);
}

__global__ void k_store_old(int N, const double* __restrict__ W, const double* __restrict__ eNewBuf,
                            double* __restrict__ rhoOld, double* __restrict__ eOld) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    rhoOld[i] = W[5 * i];
    eOld[i] = eNewBuf[i];
}

// dual2ndDST source less diag W per component (dual2ndDST.C:399-405,
// fvmDST.C:98-125), added to rhs = -R V
__global__ void k_dual_source(int N, const double* __restrict__ V, const double* __restrict__ W,
                              const double* __restrict__ rdtc, const double* __restrict__ Wn,
                              const double* __restrict__ Wnm1, double a, double b, double c,
                              double* __restrict__ rhs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double rdt = rdtc[i], Vi = V[i];
    const double dg = (rdt + a) * Vi;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const double w = W[5 * i + k];
        const double s = Vi * (rdt * w - b * Wn[5 * i + k] - c * Wnm1[5 * i + k]) - dg * w;
        rhs[5 * i + k] = s + rhs[5 * i + k];
    }
}

// setCourantDST's residual ratio with a given residualR (|initialResidual| of
// a dual-time inner solve), and the scalar courant when adjusting
__global__ void k_courant_scalar_r(Scalars* sc, double residualR, int transient_adjust, double min_co, double max_co) {
    if (threadIdx.x != 0) return;
    if (sc->residual != -1) sc->residualRatio = fmin(fmax(sc->residual / residualR, 0.1), 2.0);
    sc->residual = residualR;
    if (transient_adjust) sc->courant = fmin(fmax(sc->courant * sc->residualRatio, min_co), max_co);
}

__global__ void k_time_advance(Scalars* sc) {
    if (threadIdx.x == 0) {
        sc->time += sc->deltaT;
        sc->flags &= ~1;       // bounding flag per step; bit1 (non-physical) stays set
    }
}

}  // namespace rdst
