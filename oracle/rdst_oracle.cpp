// rdst_oracle.cpp -- CPU FP64 restatement of rhoDST's fully-coupled step.
//
// TEST INFRASTRUCTURE ONLY.  This is the parity oracle and the timed CPU
// baseline for the B200 library; nothing in the product links or calls it.
// Parity is UNPINNED against the reference itself: rhoDST needs foam-extend
// 4.1, which cannot be built here, and the reference ships no tests, golden
// data or published outputs.  The oracle is pinned instead by known-answer
// tests (tests/test_oracle_*.py): free-stream preservation, flux
// consistency, Jacobian vs. finite differences, exact ILU(0) and Krylov
// solves vs. dense linear algebra.
//
// Each routine cites the reference file:line it restates (paths relative to
// the rhoDST source tree).  foam-extend library arithmetic the reference
// calls (limitedSurfaceInterpolationScheme, Gauss gradients, block
// GMRES/BiCGStab/ILUC0/diagonal, Euler ddt, boundMinMax) is restated from
// its published definitions; see the comments at each routine.
//
// Exposes the C ABI of include/rdst.h with an `rdsto_` prefix so both
// libraries can be loaded side by side.
#include "../include/rdst.h"
#include "../rhodst_b200/csrc/rdst_options.h"
#include "../rhodst_b200/csrc/rdst_amg.h"
#include "../rhodst_b200/csrc/rdst_order.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <complex>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#define OMP_FOR_DYN _Pragma("omp parallel for schedule(dynamic, 1)")
#define OMP_FOR_REDUCE_OR_ANY _Pragma("omp parallel for schedule(static) reduction(|:any)")
#else
#define OMP_FOR_REDUCE_OR_ANY
#define OMP_FOR
#define OMP_FOR_DYN
#endif

#define ORACLE_API extern "C" __attribute__((visibility("default")))

namespace {

using namespace rdst;
typedef std::array<double, 3> v3;
typedef std::array<double, 25> t5;   // 5x5 block, row-major
typedef std::array<double, 5> v5;

inline double dot(const v3& a, const v3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double magSqr(const v3& a) { return dot(a, a); }
inline double mag(const v3& a) { return std::sqrt(magSqr(a)); }
inline v3 operator+(const v3& a, const v3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline v3 operator-(const v3& a, const v3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline v3 operator*(double s, const v3& a) { return {s * a[0], s * a[1], s * a[2]}; }
inline v3 operator/(const v3& a, double s) { return {a[0] / s, a[1] / s, a[2] / s}; }

// DST::pos/pos0/neg/neg0 (libraries/rhoDST/DST/DST.C:323-341)
inline double pos(double s) { return s > 0 ? 1.0 : 0.0; }
inline double pos0(double s) { return s >= 0 ? 1.0 : 0.0; }
inline double neg(double s) { return s < 0 ? 1.0 : 0.0; }
inline double neg0(double s) { return s <= 0 ? 1.0 : 0.0; }
// foam sign(): sign(0) = +1
inline double fsign(double s) { return s >= 0 ? 1.0 : -1.0; }
inline double sqr(double x) { return x * x; }

// Threading.  Cell loops run in parallel; face loops that scatter into
// cells are written as per-cell gathers over the cell's faces in ascending
// order, the order in which a serial face loop adds them, so fields are the
// same bit for bit for any thread count.  Sums over all cells use fixed
// blocks of 2048 summed in order: one value for any thread count.
template <class F>
double det_sum(int n, F&& term) {
    const int B = 2048, nb = (n + B - 1) / B;
    std::vector<double> part(nb, 0.0);
    OMP_FOR
    for (int k = 0; k < nb; ++k) {
        double s = 0;
        const int e = std::min(n, (k + 1) * B);
        for (int i = k * B; i < e; ++i) s += term(i);
        part[k] = s;
    }
    double s = 0;
    for (double v : part) s += v;
    return s;
}

struct Patch {
    int start, size, type, bc_p, bc_U, bc_T, bc_nut;
    double p_value, T_value, nut_value;
    v3 U_value;
};

struct Report {
    double res_l2[5] = {0, 0, 0, 0, 0}, res_mag = 0;
    double lin_initial[5] = {0, 0, 0, 0, 0}, lin_final[5] = {0, 0, 0, 0, 0};
    int lin_iterations = 0, flags = 0;
    double t[5] = {0, 0, 0, 0, 0};
};

// ----------------------------------------------------------------------
// Block system in foam's LDU layout (BlockLduMatrix<vector5>, square coeffs)
// ----------------------------------------------------------------------
struct LDU {
    std::vector<t5> d, u, l;     // diag [N], upper [Fi] (row owner), lower [Fi] (row neighbour)
    std::vector<v5> s;           // source [N]
};

inline v5 mv(const t5& A, const v5& x) {
    v5 y;
    for (int i = 0; i < 5; ++i) {
        double a = 0;
        for (int j = 0; j < 5; ++j) a += A[5 * i + j] * x[j];
        y[i] = a;
    }
    return y;
}
inline t5 mm(const t5& A, const t5& B) {
    t5 C;
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) {
            double a = 0;
            for (int k = 0; k < 5; ++k) a += A[5 * i + k] * B[5 * k + j];
            C[5 * i + j] = a;
        }
    return C;
}
// Inverse of a 5x5 block by Gauss-Jordan elimination with partial pivoting.
inline t5 inv5(const t5& A) {
    double a[5][10];
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) { a[i][j] = A[5 * i + j]; a[i][j + 5] = (i == j) ? 1.0 : 0.0; }
    for (int c = 0; c < 5; ++c) {
        int p = c;
        for (int r = c + 1; r < 5; ++r) if (std::fabs(a[r][c]) > std::fabs(a[p][c])) p = r;
        if (p != c) for (int j = 0; j < 10; ++j) std::swap(a[p][j], a[c][j]);
        double piv = 1.0 / a[c][c];
        for (int j = 0; j < 10; ++j) a[c][j] *= piv;
        for (int r = 0; r < 5; ++r) {
            if (r == c) continue;
            double f = a[r][c];
            if (f != 0.0) for (int j = 0; j < 10; ++j) a[r][j] -= f * a[c][j];
        }
    }
    t5 X;
    for (int i = 0; i < 5; ++i) for (int j = 0; j < 5; ++j) X[5 * i + j] = a[i][j + 5];
    return X;
}

struct Ctx {
    Options o;
    std::string err;
    // mesh
    int N = 0, Fi = 0, F = 0, NB = 0;
    std::vector<int> own, nei;
    std::vector<v3> Sf, Cf, C;
    std::vector<double> magSf, w, dc, V, y;
    std::vector<Patch> patches;
    std::vector<int> bpatch;          // patch of boundary face (f - Fi)
    std::vector<char> active;         // boundary face carries flux (not empty)
    std::vector<std::vector<int>> cellFaces;   // all non-empty faces of each cell
    std::vector<std::vector<int>> cellCells;   // internal-face neighbours
    std::vector<int> part;            // ILU partition (empty: one part)
    // breadth-first factorisation ranks of the partition they were made for
    mutable std::vector<int> bfs_rank, bfs_part;
    // thermo
    double R, Cp, Cv, gamma;
    // state: conservative + thermo fields (createFields.H / updateFields.H)
    std::vector<double> rho, rhoE, p, T, h;
    std::vector<v3> rhoU, U;
    // boundary values (indexed by boundary face b = f - Fi)
    std::vector<double> rho_b, rhoE_b, p_b, T_b, h_b, phi_b;
    std::vector<v3> rhoU_b, U_b;
    // valueFraction of the mixed-type BCs at their last evaluation
    // (used by valueInternalCoeffs in the boundary Jacobian)
    std::vector<double> fp_b, fU_b, fT_b;
    // turbulence: mut (cells, boundary faces), nuTilda; viscous switch
    std::vector<double> mut, mut_b, nut, nut_b;
    bool viscous = false;
    // residual R_ (baseFluxDST R_, per unit volume) and face fluxes
    std::vector<v5> Rv;
    std::vector<unsigned char> rmask;  // held cells: zero residual, identity rows (empty: none)
    std::vector<double> phi, phiEp;
    std::vector<v3> phiUp, Up;
    // time control (timeDST)
    double time = 0, deltaT = 1, courant = 1, residual = -1, residualRatio = 1;
    std::vector<double> courantField, rDeltaT, rhoOld, eOld;
    std::vector<v3> dS;
    bool bounded = false;
    // SARC1: the strain-rate tensor of the last turbulence update (its
    // old-time value; 6 components, symmetric) and rho before the update
    std::vector<std::array<double, 6>> S_old;
    bool S_old_valid = false;
    bool state_set = false;           // a state has been set (later sets keep the time-control history)
    std::vector<double> nutN, nutNm1;  // nuTilda old time levels of dual-time stepping
    std::vector<double> rho0;
    // dual-time stepping: W at the two previous time levels, foam Time's
    // deltaTSave (deltaT0 of the next step), the step's BDF2 coefficients
    std::vector<std::array<double, 5>> Wn, Wnm1;
    bool dual_started = false;
    double dt_save = 1.0, dual_a = 0, dual_b = 0, dual_c = 0;
    // SARC1 under dual-time stepping: S.oldTime() and its oldTime(), the
    // time indices foam gives S and each of them (-1: not created), the
    // physical step's index, deltaT and deltaT0
    std::vector<std::array<double, 6>> S_o, S_oo;
    int S_idx = -1, S_o_idx = -1, S_oo_idx = -1, dual_tidx = 0;
    double dual_dt = 1.0, dual_dt0 = 1.0;
};

// ----------------------------------------------------------------------
// Boundary conditions.  Values of p, U, T on each boundary face from the
// internal field (fvPatchField::evaluate of fixedValue, zeroGradient,
// inletOutlet, symmetryPlane/slip), then rho/rhoU/rhoE boundary values as
// updateFields.H:84-93 rebuilds them: rho_b = p_b psi_b,
// rhoU_b = rho_b U_b, rhoE_b = rho_b (h_b + |U_b|^2/2) - p_b.
// inletOutlet switches on the boundary mass flux phi (valueFraction =
// 1 - pos(phi), foam pos(0) = 1).
// ----------------------------------------------------------------------
void eval_boundary(Ctx& c) {
    OMP_FOR
    for (int b = 0; b < c.NB; ++b) {
        if (!c.active[b]) continue;
        const int f = c.Fi + b;
        const Patch& P = c.patches[c.bpatch[b]];
        const int ci = c.own[f];
        const v3 n = c.Sf[f] / c.magSf[f];
        const bool outflow = c.phi_b[b] >= 0.0;
        const v3& Ui = c.U[ci];
        double fp = 0, fU = 0, fT = 0;
        // characteristic far field (farField*DSTFvPatch*Field.C:144-221):
        // boundary Mach from the last boundary mass flux, rho_b and c_b
        double supIn = 0, supOut = 0, subIn = 0, subOut = 0, rho0c0 = 0, cI = 0, pbU = 0;
        if (P.bc_p == RDST_BC_FARFIELD || P.bc_U == RDST_BC_FARFIELD || P.bc_T == RDST_BC_FARFIELD) {
            double cb = std::sqrt(c.gamma * c.R * c.T_b[b]);
            cI = std::sqrt(c.gamma * c.R * c.T[ci]);
            double mach = c.phi_b[b] / c.rho_b[b] / c.magSf[f] / cb;
            supIn = neg0(mach + 1);
            supOut = pos0(mach - 1);
            subIn = neg(mach) - supIn;
            subOut = pos0(mach) - supOut;
            rho0c0 = c.rho[ci] * cI;
            pbU = 0.5 * (P.p_value + c.p[ci] - rho0c0 * dot(n, P.U_value - Ui));
        }
        // p
        switch (P.bc_p) {
            case RDST_BC_FIXED_VALUE: c.p_b[b] = P.p_value; fp = 1; break;
            case RDST_BC_INLET_OUTLET: fp = outflow ? 0.0 : 1.0; c.p_b[b] = outflow ? c.p[ci] : P.p_value; break;
            case RDST_BC_FARFIELD: {
                double pb = P.p_value - rho0c0 * dot(n, P.U_value - Ui);
                double ref = supIn * P.p_value + subIn * pb + subOut * P.p_value;
                fp = 1 - supOut - 0.5 * subIn;
                c.p_b[b] = fp * ref + (1 - fp) * c.p[ci];
                break;
            }
            default: c.p_b[b] = c.p[ci]; break;
        }
        // T
        switch (P.bc_T) {
            case RDST_BC_FIXED_VALUE: c.T_b[b] = P.T_value; fT = 1; break;
            case RDST_BC_INLET_OUTLET: fT = outflow ? 0.0 : 1.0; c.T_b[b] = outflow ? c.T[ci] : P.T_value; break;
            case RDST_BC_FARFIELD: {
                double TI = c.T[ci], pI = c.p[ci], rhoI = c.rho[ci];
                double RI = pI / rhoI / TI;
                double rhoa = P.p_value / P.T_value / RI;
                double subsInValue = pbU / (rhoa + (pbU - P.p_value) / sqr(cI)) / RI;
                double sOVF = pbU / (pI + RI * TI * (pbU - pI) / sqr(cI));
                double ref = supIn * P.T_value + subIn * subsInValue;
                fT = 1 - supOut - sOVF * subOut;
                c.T_b[b] = fT * ref + (1 - fT) * TI;
                break;
            }
            default: c.T_b[b] = c.T[ci]; break;
        }
        // U
        switch (P.bc_U) {
            case RDST_BC_FIXED_VALUE: c.U_b[b] = P.U_value; fU = 1; break;
            case RDST_BC_INLET_OUTLET: fU = outflow ? 0.0 : 1.0; c.U_b[b] = outflow ? Ui : P.U_value; break;
            case RDST_BC_SYMMETRY:
            case RDST_BC_SLIP: c.U_b[b] = Ui - dot(n, Ui) * n; break;
            case RDST_BC_FARFIELD: {
                v3 subsIn = P.U_value - ((P.p_value - pbU) / rho0c0) * n;
                v3 subsOut = ((c.p[ci] - pbU) / rho0c0) * n;
                v3 ref = supIn * P.U_value + subIn * subsIn + subOut * subsOut;
                fU = 1 - supOut - subOut;
                c.U_b[b] = fU * ref + (1 - fU) * Ui;
                break;
            }
            default: c.U_b[b] = Ui; break;
        }
        c.fp_b[b] = fp; c.fU_b[b] = fU; c.fT_b[b] = fT;
        // bounding of the boundary pressure (boundMinMax acts on the patch values too)
        c.p_b[b] = std::min(std::max(c.p_b[b], c.o.p_min), c.o.p_max);
        c.h_b[b] = c.Cp * c.T_b[b];
        const double psi_b = 1.0 / (c.R * c.T_b[b]);
        c.rho_b[b] = c.p_b[b] * psi_b;
        c.rhoU_b[b] = c.rho_b[b] * c.U_b[b];
        c.rhoE_b[b] = c.rho_b[b] * (c.h_b[b] + 0.5 * magSqr(c.U_b[b])) - c.p_b[b];
    }
}

// valueInternalCoeffs(weights) of each BC (used by Roe.C:363-365): mixed
// types (fixedValue f=1, zeroGradient f=0, inletOutlet, far field) give
// 1 - valueFraction from their last evaluation; symmetry/slip vectors
// 1 - |n_i| per component (basicSymmetry), scalars 1.
void internal_coeffs(const Ctx& c, int b, double& cp, v3& cu, double& cT) {
    const int f = c.Fi + b;
    const Patch& P = c.patches[c.bpatch[b]];
    const v3 n = c.Sf[f] / c.magSf[f];
    cp = 1.0 - c.fp_b[b];
    cT = 1.0 - c.fT_b[b];
    if (P.bc_U == RDST_BC_SYMMETRY || P.bc_U == RDST_BC_SLIP)
        cu = {1 - std::fabs(n[0]), 1 - std::fabs(n[1]), 1 - std::fabs(n[2])};
    else {
        double u = 1.0 - c.fU_b[b];
        cu = {u, u, u};
    }
}

// ----------------------------------------------------------------------
// Gauss linear gradient (foam gaussGrad with linear interpolation):
// grad(phi)_c = 1/V_c sum_f S_f phi_f, phi_f = w phi_P + (1-w) phi_N on
// internal faces, the boundary value on boundary faces (empty: none).
// ----------------------------------------------------------------------
void grad_scalar(const Ctx& c, const std::vector<double>& x, const std::vector<double>& xb,
                 std::vector<v3>& g) {
    g.assign(c.N, v3{0, 0, 0});
    OMP_FOR
    for (int i = 0; i < c.N; ++i) {
        v3 a{0, 0, 0};
        for (int f : c.cellFaces[i]) {
            if (f < c.Fi) {
                double xf = c.w[f] * x[c.own[f]] + (1 - c.w[f]) * x[c.nei[f]];
                v3 s = xf * c.Sf[f];
                a = (c.own[f] == i) ? a + s : a - s;
            } else {
                a = a + xb[f - c.Fi] * c.Sf[f];
            }
        }
        g[i] = a / c.V[i];
    }
}

// tensor gradient (grad U)_{ij} = d U_j / d x_i, stored row-major [9]
void grad_vector(const Ctx& c, const std::vector<v3>& x, const std::vector<v3>& xb,
                 std::vector<std::array<double, 9>>& g) {
    g.assign(c.N, std::array<double, 9>{});
    OMP_FOR
    for (int cell = 0; cell < c.N; ++cell) {
        std::array<double, 9> a{};
        auto add = [&](const v3& S, const v3& xf, double sgn) {
            for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) a[3 * i + j] += sgn * S[i] * xf[j];
        };
        for (int f : c.cellFaces[cell]) {
            if (f < c.Fi) {
                v3 xf = c.w[f] * x[c.own[f]] + (1 - c.w[f]) * x[c.nei[f]];
                add(c.Sf[f], xf, c.own[f] == cell ? 1.0 : -1.0);
            } else {
                add(c.Sf[f], xb[f - c.Fi], 1.0);
            }
        }
        for (int k = 0; k < 9; ++k) a[k] /= c.V[cell];
        g[cell] = a;
    }
}

// cellLimited Gauss linear k for grad(U) (foam-extend cellLimitedGrad for a
// vector field, as the RAE2822 tutorial selects it): per velocity component
// j the spread maxD/minD of U_j over the face neighbours and boundary values
// (widened by (1/k - 1)(maxD - minD) for k < 1); the limiter is the minimum
// over the cell's faces of maxD/d (d > maxD + VSMALL) or minD/d
// (d < minD - VSMALL), d = (Cf - C) . grad U_j; grad U_j is scaled by it.
void limit_grad_U(const Ctx& c, std::vector<std::array<double, 9>>& g) {
    const double k = c.o.grad_U_limit;
    if (!(k > 0)) return;
    OMP_FOR
    for (int i = 0; i < c.N; ++i) {
        v3 mx = c.U[i], mn = c.U[i];
        for (int f : c.cellFaces[i]) {
            if (f < c.Fi) {
                const v3& o = c.U[c.own[f] == i ? c.nei[f] : c.own[f]];
                for (int j = 0; j < 3; ++j) { mx[j] = std::max(mx[j], o[j]); mn[j] = std::min(mn[j], o[j]); }
            } else if (c.active[f - c.Fi]) {
                const v3& o = c.U_b[f - c.Fi];
                for (int j = 0; j < 3; ++j) { mx[j] = std::max(mx[j], o[j]); mn[j] = std::min(mn[j], o[j]); }
            }
        }
        for (int j = 0; j < 3; ++j) {
            mx[j] -= c.U[i][j];
            mn[j] -= c.U[i][j];
            if (k < 1.0) {
                const double w = (1.0 / k - 1.0) * (mx[j] - mn[j]);
                mx[j] += w;
                mn[j] -= w;
            }
        }
        v3 lim{1.0, 1.0, 1.0};
        for (int f : c.cellFaces[i]) {
            if (f >= c.Fi && !c.active[f - c.Fi]) continue;
            const v3 d = c.Cf[f] - c.C[i];
            for (int j = 0; j < 3; ++j) {
                const double e = d[0] * g[i][j] + d[1] * g[i][3 + j] + d[2] * g[i][6 + j];
                if (e > mx[j] + VSMALL) lim[j] = std::min(lim[j], mx[j] / e);
                else if (e < mn[j] - VSMALL) lim[j] = std::min(lim[j], mn[j] / e);
            }
        }
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 3; ++j) g[i][3 * a + j] *= lim[j];
    }
}

// ----------------------------------------------------------------------
// Limited reconstruction (foam-extend limitedSurfaceInterpolationScheme with
// a TVD limiter, as selected by "reconstruct(X)" and called with the +-1
// face-flux fields own_/nei_ of baseFluxDST.C:144-171):
//   weights = lim*w + (1 - lim)*pos(faceFlux)      (foam pos(0) = 1)
//   phi_f   = weights*phi_P + (1 - weights)*phi_N
// with lim = limiter(r) and r from NVDTVD::r / NVDVTVDV::r:
//   r = 2 (d . grad phi_C)/(phi_N - phi_P) - 1, C the upwind cell,
//   |d.grad| >= 1000|phi_N - phi_P|  ->  r = 2000 sign(.)sign(.) - 1.
// The smooth limiters (OSPRE, vanAlbada) are clipped at 0 for r < 0 (TVD
// region).  Unpinned: foam-extend's limiter sources are not vendored.
// ----------------------------------------------------------------------
double tvd_limiter(Limiter L, double r) {
    switch (L) {
        case LIM_OSPRE: { double rr = r * (r + 1); return std::max(1.5 * rr / (rr + 1), 0.0); }
        case LIM_VANLEER: return (r + std::fabs(r)) / (1 + std::fabs(r));
        case LIM_MINMOD: return std::max(std::min(std::min(r, 1.0), 2.0), 0.0);
        case LIM_VANALBADA: return std::max(r * (r + 1) / (r * r + 1), 0.0);
        case LIM_SUPERBEE: return std::max(std::max(std::min(2 * r, 1.0), std::min(r, 2.0)), 0.0);
        case LIM_MUSCL: return std::max(std::min(std::min(2 * r, 0.5 * r + 0.5), 2.0), 0.0);
        default: return 1.0;
    }
}

double nvd_r(double gradcf, double gradf) {
    if (std::fabs(gradcf) >= 1000 * std::fabs(gradf)) return 2 * 1000 * fsign(gradcf) * fsign(gradf) - 1;
    return 2 * (gradcf / gradf) - 1;
}

// Face weight on the owner value for one side (faceFlux = +1 owner side, -1 neighbour side)
double side_weight(Limiter L, double faceFlux, double w, double r) {
    if (L == LIM_LINEAR) return w;
    if (L == LIM_UPWIND) return faceFlux >= 0 ? 1.0 : 0.0;
    double lim = tvd_limiter(L, r);
    return lim * w + (1 - lim) * (faceFlux >= 0 ? 1.0 : 0.0);
}

// Venkatakrishnan (1995) cell limiter psi_c (new option, not in the
// reference): psi = min over faces of phi_V(dmax/dmin, d2 = grad.(Cf - C)),
// eps^2 = (K h)^3 with h = V^(1/3); reconstruction phi_f = phi_C + psi grad.(Cf-C).
void venkat_psi(const Ctx& c, const std::vector<double>& x, const std::vector<double>& xb,
                const std::vector<v3>& g, std::vector<double>& psi) {
    psi.assign(c.N, 1.0);
    OMP_FOR
    for (int i = 0; i < c.N; ++i) {
        double mxi = x[i], mni = x[i];         // max/min over the face neighbours (order-free)
        for (int f : c.cellFaces[i]) {
            double xo = f < c.Fi ? x[c.own[f] == i ? c.nei[f] : c.own[f]] : xb[f - c.Fi];
            mxi = std::max(mxi, xo); mni = std::min(mni, xo);
        }
        double hh = std::cbrt(c.V[i]);
        double eps2 = std::pow(c.o.venkat_K * hh, 3);
        double dmax = mxi - x[i], dmin = mni - x[i];
        double p = 1.0;
        for (int f : c.cellFaces[i]) {
            double d2 = dot(g[i], c.Cf[f] - c.C[i]);
            double phi;
            if (d2 > 0) phi = ((dmax * dmax + eps2) * d2 + 2 * d2 * d2 * dmax) / (dmax * dmax + 2 * d2 * d2 + dmax * d2 + eps2) / d2;
            else if (d2 < 0) phi = ((dmin * dmin + eps2) * d2 + 2 * d2 * d2 * dmin) / (dmin * dmin + 2 * d2 * d2 + dmin * d2 + eps2) / d2;
            else phi = 1.0;
            p = std::min(p, phi);
        }
        psi[i] = p;
    }
}

// Reconstruct one scalar cell field to owner/neighbour face values.
void reconstruct_scalar(const Ctx& c, Limiter L, const std::vector<double>& x,
                        const std::vector<double>& xb, std::vector<double>& xo,
                        std::vector<double>& xn) {
    xo.assign(c.F, 0.0);
    xn.assign(c.F, 0.0);
    std::vector<v3> g;
    if (L != LIM_LINEAR && L != LIM_UPWIND) grad_scalar(c, x, xb, g);
    std::vector<double> psi;
    if (L == LIM_VENKATAKRISHNAN) venkat_psi(c, x, xb, g, psi);
    OMP_FOR
    for (int f = 0; f < c.Fi; ++f) {
        int P = c.own[f], Nn = c.nei[f];
        if (L == LIM_VENKATAKRISHNAN) {
            xo[f] = x[P] + psi[P] * dot(g[P], c.Cf[f] - c.C[P]);
            xn[f] = x[Nn] + psi[Nn] * dot(g[Nn], c.Cf[f] - c.C[Nn]);
            continue;
        }
        double ro = 0, rn = 0;
        if (L != LIM_LINEAR && L != LIM_UPWIND) {
            v3 d = c.C[Nn] - c.C[P];
            double gradf = x[Nn] - x[P];
            ro = nvd_r(dot(d, g[P]), gradf);
            rn = nvd_r(dot(d, g[Nn]), gradf);
        }
        double wo = side_weight(L, +1, c.w[f], ro);
        double wn = side_weight(L, -1, c.w[f], rn);
        xo[f] = wo * x[P] + (1 - wo) * x[Nn];
        xn[f] = wn * x[P] + (1 - wn) * x[Nn];
    }
    for (int b = 0; b < c.NB; ++b) { xo[c.Fi + b] = xb[b]; xn[c.Fi + b] = xb[b]; }
}

void reconstruct_vector(const Ctx& c, Limiter L, const std::vector<v3>& x, const std::vector<v3>& xb,
                        std::vector<v3>& xo, std::vector<v3>& xn) {
    xo.assign(c.F, v3{0, 0, 0});
    xn.assign(c.F, v3{0, 0, 0});
    std::vector<std::array<double, 9>> g;
    if (L != LIM_LINEAR && L != LIM_UPWIND) grad_vector(c, x, xb, g);
    std::vector<double> psi[3];
    if (L == LIM_VENKATAKRISHNAN) {
        for (int k = 0; k < 3; ++k) {
            std::vector<double> xk(c.N), xbk(c.NB);
            std::vector<v3> gk(c.N);
            OMP_FOR
            for (int i = 0; i < c.N; ++i) { xk[i] = x[i][k]; gk[i] = {g[i][k], g[i][3 + k], g[i][6 + k]}; }
            for (int b = 0; b < c.NB; ++b) xbk[b] = xb[b][k];
            venkat_psi(c, xk, xbk, gk, psi[k]);
        }
    }
    OMP_FOR
    for (int f = 0; f < c.Fi; ++f) {
        int P = c.own[f], Nn = c.nei[f];
        if (L == LIM_VENKATAKRISHNAN) {
            v3 dP = c.Cf[f] - c.C[P], dN = c.Cf[f] - c.C[Nn];
            for (int k = 0; k < 3; ++k) {
                double gP = dP[0] * g[P][k] + dP[1] * g[P][3 + k] + dP[2] * g[P][6 + k];
                double gN = dN[0] * g[Nn][k] + dN[1] * g[Nn][3 + k] + dN[2] * g[Nn][6 + k];
                xo[f][k] = x[P][k] + psi[k][P] * gP;
                xn[f][k] = x[Nn][k] + psi[k][Nn] * gN;
            }
            continue;
        }
        double ro = 0, rn = 0;
        if (L != LIM_LINEAR && L != LIM_UPWIND) {
            v3 d = c.C[Nn] - c.C[P];
            v3 gradfV = x[Nn] - x[P];
            double gradf = dot(gradfV, gradfV);
            v3 dgP, dgN;
            for (int j = 0; j < 3; ++j) {
                dgP[j] = d[0] * g[P][j] + d[1] * g[P][3 + j] + d[2] * g[P][6 + j];
                dgN[j] = d[0] * g[Nn][j] + d[1] * g[Nn][3 + j] + d[2] * g[Nn][6 + j];
            }
            ro = nvd_r(dot(gradfV, dgP), gradf);
            rn = nvd_r(dot(gradfV, dgN), gradf);
        }
        double wo = side_weight(L, +1, c.w[f], ro);
        double wn = side_weight(L, -1, c.w[f], rn);
        xo[f] = wo * x[P] + (1 - wo) * x[Nn];
        xn[f] = wn * x[P] + (1 - wn) * x[Nn];
    }
    for (int b = 0; b < c.NB; ++b) { xo[c.Fi + b] = xb[b]; xn[c.Fi + b] = xb[b]; }
}

// ----------------------------------------------------------------------
// Convective flux schemes, one face at a time.  Inputs are the owner- and
// neighbour-side reconstructed rho, rhoU, rPsi = 1/psi, e = h - p/rho and
// the scheme's speed field s (Kurganov, AUSM: c = sqrt(gamma rPsi);
// HLL family and AUSM+/AUSM+up: critical speed a = sqrt(2(g-1)/(g+1) H)).
// Outputs phi, phiUp, phiEp (integrated over the face) and Up.
// ----------------------------------------------------------------------
struct Side { double rho; v3 rhoU; double rPsi, e, s; };
struct FaceFlux { double phi; v3 phiUp; double phiEp; v3 Up; };

// KurganovDST::computeFluxDST (KurganovDST.C:93-167)
FaceFlux flux_kurganov(const Side& o, const Side& n, const v3& Sf, double magSf) {
    v3 U_own = o.rhoU / o.rho, U_nei = n.rhoU / n.rho;
    double rhoE_own = o.rho * (o.e + 0.5 * magSqr(U_own));
    double rhoE_nei = n.rho * (n.e + 0.5 * magSqr(U_nei));
    double p_own = o.rho * o.rPsi, p_nei = n.rho * n.rPsi;
    double phiv_own = dot(U_own, Sf), phiv_nei = dot(U_nei, Sf);
    double cSf_own = o.s * magSf, cSf_nei = n.s * magSf;
    double ap = std::max(std::max(phiv_own + cSf_own, phiv_nei + cSf_nei), 0.0);
    double am = std::min(std::min(phiv_own - cSf_own, phiv_nei - cSf_nei), 0.0);
    double a_own = ap / (ap - am);
    double aSf = am * a_own;
    double a_nei = 1.0 - a_own;
    phiv_own *= a_own;
    phiv_nei *= a_nei;
    double aphiv_own = phiv_own - aSf, aphiv_nei = phiv_nei + aSf;
    FaceFlux F;
    F.phi = aphiv_own * o.rho + aphiv_nei * n.rho;
    F.phiUp = (aphiv_own * o.rhoU + aphiv_nei * n.rhoU) + (a_own * p_own + a_nei * p_nei) * Sf;
    F.phiEp = aphiv_own * (rhoE_own + p_own) + aphiv_nei * (rhoE_nei + p_nei) + aSf * p_own - aSf * p_nei;
    F.Up = a_own * U_own + a_nei * U_nei;
    return F;
}

// Common HLL-family prologue: Roe-averaged wave-speed estimates
// (HLLDST.C:93-160, HLLCDST.C:137-195, HLLCPDST.C:168-224)
struct HLLPro {
    v3 U_own, U_nei, normal, UTilde;
    double E_own, E_nei, p_own, p_nei, H_own, H_nei, coefR, HTilde, aTilde;
    double Uv_own, Uv_nei, UvTilde, S_own, S_nei;
};
HLLPro hll_prologue(const Side& o, const Side& n, const v3& Sf, double magSf, double gamma) {
    HLLPro q;
    q.U_own = o.rhoU / o.rho;
    q.U_nei = n.rhoU / n.rho;
    q.E_own = o.e + 0.5 * magSqr(q.U_own);
    q.E_nei = n.e + 0.5 * magSqr(q.U_nei);
    q.p_own = o.rho * o.rPsi;
    q.p_nei = n.rho * n.rPsi;
    q.H_own = q.E_own + q.p_own / o.rho;
    q.H_nei = q.E_nei + q.p_nei / n.rho;
    q.coefR = std::sqrt(std::max(VSMALL, n.rho) / std::max(VSMALL, o.rho));
    q.HTilde = (q.coefR * q.H_nei + q.H_own) / (q.coefR + 1.0);
    q.UTilde = (q.coefR * q.U_nei + q.U_own) / (q.coefR + 1.0);
    q.aTilde = std::sqrt((gamma - 1.0) * (q.HTilde - 0.5 * magSqr(q.UTilde)));
    q.normal = Sf / magSf;
    q.Uv_own = dot(q.U_own, q.normal);
    q.Uv_nei = dot(q.U_nei, q.normal);
    q.UvTilde = dot(q.UTilde, q.normal);
    q.S_own = std::min(q.Uv_own - o.s, q.UvTilde - q.aTilde);
    q.S_nei = std::max(q.Uv_nei + n.s, q.UvTilde + q.aTilde);
    return q;
}

// HLLDST::computeFluxDST (HLLDST.C:91-204)
FaceFlux flux_hll(const Side& o, const Side& n, const v3& Sf, double magSf, double gamma) {
    HLLPro q = hll_prologue(o, n, Sf, magSf, gamma);
    double cf_own = pos0(q.S_own);
    double cf_m = neg(q.S_own) * pos0(q.S_nei);
    double cf_nei = neg(q.S_nei) * neg(q.S_own);
    v3 rhoUPhi_own = (o.rho * q.Uv_own) * q.U_own + q.p_own * q.normal;
    v3 rhoUPhi_nei = (n.rho * q.Uv_nei) * q.U_nei + q.p_nei * q.normal;
    double dS = q.S_nei - q.S_own;
    FaceFlux F;
    F.phi = (cf_own * o.rho * q.Uv_own +
             cf_m * (q.S_nei * o.rho * q.Uv_own - q.S_own * n.rho * q.Uv_nei + q.S_own * q.S_nei * (n.rho - o.rho)) / dS +
             cf_nei * n.rho * q.Uv_nei) * magSf;
    v3 mid = (1.0 / dS) * (q.S_nei * rhoUPhi_own - q.S_own * rhoUPhi_nei +
                           (q.S_own * q.S_nei) * (n.rho * q.U_nei - o.rho * q.U_own));
    F.phiUp = magSf * (cf_own * rhoUPhi_own + cf_m * mid + cf_nei * rhoUPhi_nei);
    F.phiEp = (cf_own * o.rho * q.Uv_own * q.H_own +
               cf_m * (q.S_nei * o.rho * q.Uv_own * q.H_own - q.S_own * n.rho * q.Uv_nei * q.H_nei +
                       q.S_own * q.S_nei * (n.rho * q.E_nei - o.rho * q.E_own)) / dS +
               cf_nei * n.rho * q.Uv_nei * q.H_nei) * magSf;
    v3 Um = (1.0 / dS) * (q.S_nei * q.U_own - q.S_own * q.U_nei + q.Uv_own * q.U_own - q.Uv_nei * q.U_nei);
    F.Up = cf_own * q.U_own + cf_m * Um + cf_nei * q.U_nei;
    return F;
}

// HLLCDST::computeFluxDST (HLLCDST.C:135-272) and HLLCPDST (HLLCPDST.C:166-317)
FaceFlux flux_hllc(const Side& o, const Side& n, const v3& Sf, double magSf, double gamma,
                   bool pressure_sensor, double f) {
    HLLPro q = hll_prologue(o, n, Sf, magSf, gamma);
    const double S_own = q.S_own, S_nei = q.S_nei, Uv_own = q.Uv_own, Uv_nei = q.Uv_nei;
    double S_star = (q.p_nei - q.p_own + o.rho * Uv_own * (S_own - Uv_own) - n.rho * Uv_nei * (S_nei - Uv_nei)) /
                    (o.rho * (S_own - Uv_own) - n.rho * (S_nei - Uv_nei));
    double pstar_own = q.p_own + o.rho * (S_own - Uv_own) * (S_star - Uv_own);
    double pstar_nei = q.p_nei + n.rho * (S_nei - Uv_nei) * (S_star - Uv_nei);
    double cf_own = pos(S_own);
    double cf_m1 = neg0(S_own) * pos(S_star);
    double cf_m2 = neg0(S_own) * neg0(S_star) * pos0(S_nei);
    double cf_nei = neg0(S_own) * neg0(S_star) * neg(S_nei);
    double rhoE_own = o.rho * q.E_own, rhoE_nei = n.rho * q.E_nei;
    v3 rhoUPhi_own = Uv_own * o.rhoU + q.p_own * q.normal;
    v3 rhoUPhi_nei = Uv_nei * n.rhoU + q.p_nei * q.normal;
    double rhoEPhi_own = (rhoE_own + q.p_own) * Uv_own;
    double rhoEPhi_nei = (rhoE_nei + q.p_nei) * Uv_nei;
    double d1 = S_own - S_star, d2 = S_nei - S_star;
    FaceFlux F;
    if (!pressure_sensor) {
        F.phi = (cf_own * o.rho * Uv_own + cf_m1 * S_star * o.rho * (S_own - Uv_own) / d1 +
                 cf_m2 * S_star * n.rho * (S_nei - Uv_nei) / d2 + cf_nei * n.rho * Uv_nei) * magSf;
        v3 m1 = (1.0 / d1) * (S_star * (S_own * o.rhoU - rhoUPhi_own) + (S_own * pstar_own) * q.normal);
        v3 m2 = (1.0 / d2) * (S_star * (S_nei * n.rhoU - rhoUPhi_nei) + (S_nei * pstar_nei) * q.normal);
        F.phiUp = magSf * (cf_own * rhoUPhi_own + cf_m1 * m1 + cf_m2 * m2 + cf_nei * rhoUPhi_nei);
        F.phiEp = (cf_own * rhoEPhi_own + cf_m1 * S_star * (S_own * rhoE_own - rhoEPhi_own + S_own * pstar_own) / d1 +
                   cf_m2 * S_star * (S_nei * rhoE_nei - rhoEPhi_nei + S_nei * pstar_nei) / d2 +
                   cf_nei * rhoEPhi_nei) * magSf;
    } else {
        // HLLCPDST.C:228-303 (pressure sensor f, p** / p*** blends, anti-dissipation phip)
        double Ma_own = Uv_own / o.s, Ma_nei = Uv_nei / n.s;
        double MaTilde = (q.coefR * Ma_nei + Ma_own) / (q.coefR + 1.0);
        double c_own = o.rho * (S_own - Uv_own), c_nei = n.rho * (S_nei - Uv_nei);
        double p_star = (c_nei * q.p_own - c_own * q.p_nei - c_own * c_nei * (Uv_own - Uv_nei)) / (c_nei - c_own);
        double theta = std::min(std::max(std::fabs(Ma_own), std::fabs(Ma_nei)), 1.0);
        double p_av = 0.5 * (q.p_own + q.p_nei);
        double p_ss = p_star * theta + (1.0 - theta) * p_av;
        double p_sss = f * p_ss + (1.0 - f) * p_star;
        double phip = (f - 1.0) * S_own * S_nei / (S_nei - S_own) / (1.0 + std::fabs(MaTilde)) *
                      (q.p_nei - q.p_own) / sqr(q.aTilde);
        F.phi = (cf_own * o.rho * Uv_own + cf_m1 * (S_star * o.rho * (S_own - Uv_own) / d1 + phip) +
                 cf_m2 * (S_star * n.rho * (S_nei - Uv_nei) / d2 + phip) + cf_nei * n.rho * Uv_nei) * magSf;
        v3 m1 = (1.0 / d1) * (S_star * (S_own * o.rhoU - rhoUPhi_own) + (S_own * p_sss) * q.normal) + phip * q.UTilde;
        v3 m2 = (1.0 / d2) * (S_star * (S_nei * n.rhoU - rhoUPhi_nei) + (S_nei * p_sss) * q.normal) + phip * q.UTilde;
        F.phiUp = magSf * (cf_own * rhoUPhi_own + cf_m1 * m1 + cf_m2 * m2 + cf_nei * rhoUPhi_nei);
        double kin = 0.5 * phip * magSqr(q.UTilde);
        F.phiEp = (cf_own * rhoEPhi_own + cf_m1 * (S_star * (S_own * rhoE_own - rhoEPhi_own + S_own * p_star) / d1 + kin) +
                   cf_m2 * (S_star * (S_nei * rhoE_nei - rhoEPhi_nei + S_nei * p_star) / d2 + kin) +
                   cf_nei * rhoEPhi_nei) * magSf;
    }
    F.Up = cf_own * q.U_own + cf_m1 * ((S_own - Uv_own) / d1) * q.U_own +
           cf_m2 * ((S_nei - Uv_nei) / d2) * q.U_nei + cf_nei * q.U_nei;
    return F;
}

// AUSMPLDST::computeFluxDST (AUSMPLDST.C:127-217, alpha=3/16, beta=1/8 at
// AUSMPLDST.H:78-79) and AUSMPLUPDST::computeFluxDST (AUSMPLUPDST.C:209-320,
// Kp=0.25, Ku=0.75, sigma=1, beta=1/8 at AUSMPLUPDST.H:84-87; alpha stays 0
// unless lowMach, AUSMPLUPDST.C:118-131).  0.5(sign(x)+|sign(x)|) = pos0(x).
FaceFlux flux_ausm_plus(const Side& o, const Side& n, const v3& Sf, double magSf, bool up,
                        bool lowMach, double Mainf) {
    const double beta = 0.125, Kp = 0.25, Ku = 0.75, sigma = 1.0;
    v3 U_own = o.rhoU / o.rho, U_nei = n.rhoU / n.rho;
    v3 nrm = Sf / magSf;
    double Uv_own = dot(U_own, nrm), Uv_nei = dot(U_nei, nrm);
    double rhoE_own = o.rho * (o.e + 0.5 * magSqr(U_own));
    double rhoE_nei = n.rho * (n.e + 0.5 * magSqr(U_nei));
    double p_own = o.rho * o.rPsi, p_nei = n.rho * n.rPsi;
    double a_own = o.s, a_nei = n.s, a12;
    double alpha = up ? 0.0 : 3.0 / 16.0;
    if (up) {
        a_own = sqr(a_own) / std::max(a_own, Uv_own);
        a_nei = sqr(a_nei) / std::max(a_nei, -Uv_nei);
        a12 = std::min(a_own, a_nei);
    } else {
        a12 = 0.5 * (a_own + a_nei);
    }
    double Ma_own = Uv_own / a12, Ma_nei = Uv_nei / a12;
    double Mmean2 = 0, fa = 0;
    if (up && lowMach) {
        Mmean2 = 0.5 * (sqr(Uv_own) + sqr(Uv_nei)) / sqr(a12);
        double M0 = std::sqrt(std::min(1.0, std::max(Mmean2, sqr(Mainf))));
        fa = M0 * (2.0 - M0);
        alpha = 3.0 / 16.0 * (-4.0 + 5.0 * sqr(fa));
    }
    double in_o = pos0(1.0 - std::fabs(Ma_own)), out_o = pos0(-1.0 + std::fabs(Ma_own));
    double in_n = pos0(1.0 - std::fabs(Ma_nei)), out_n = pos0(-1.0 + std::fabs(Ma_nei));
    double Ma4_own = in_o * (0.25 * sqr(Ma_own + 1.0)) * (1.0 - 16.0 * beta * (-0.25) * sqr(Ma_own - 1.0)) +
                     out_o * std::max(Ma_own, 0.0);
    double P5_own = in_o * 0.25 * sqr(Ma_own + 1.0) * (2.0 - Ma_own - 16.0 * alpha * Ma_own * (-0.25) * sqr(Ma_own - 1.0)) +
                    out_o * pos(Ma_own);
    double Ma4_nei = in_n * (-0.25) * sqr(Ma_nei - 1.0) * (1.0 + 16.0 * beta * 0.25 * sqr(Ma_nei + 1.0)) +
                     out_n * std::min(Ma_nei, 0.0);
    double P5_nei = in_n * (-0.25) * sqr(Ma_nei - 1.0) * (-2.0 - Ma_nei + 16.0 * alpha * Ma_nei * 0.25 * sqr(Ma_nei + 1.0)) +
                    out_n * neg(Ma_nei);
    double Ma12 = Ma4_own + Ma4_nei;
    double P12 = P5_own * p_own + P5_nei * p_nei;
    if (up && lowMach) {
        double Mp = -Kp / fa * std::max(1.0 - sigma * Mmean2, 0.0) * (p_nei - p_own) / (0.5 * (o.rho + n.rho)) / sqr(a12);
        double pu = -Ku * P5_own * P5_nei * (o.rho + n.rho) * a12 * fa * (Uv_own - Uv_nei);
        Ma12 += Mp;
        P12 += pu;
    }
    FaceFlux F;
    F.Up = pos(Ma12) * U_own + neg0(Ma12) * U_nei;
    F.phi = Ma12 * a12 * (pos(Ma12) * o.rho + neg0(Ma12) * n.rho) * magSf;
    F.phiUp = F.phi * F.Up + P12 * Sf;
    double H_own = (rhoE_own + p_own) / o.rho, H_nei = (rhoE_nei + p_nei) / n.rho;
    F.phiEp = F.phi * (pos(Ma12) * H_own + neg0(Ma12) * H_nei);
    return F;
}

// Plain AUSM (Liou & Steffen 1993; listed in the reference README but not
// implemented there): split Mach M+-(M) = +-(M+-1)^2/4 for |M|<=1 else
// (M+-|M|)/2, split pressure P+-(M) = (M+-1)^2 (2-+M)/4 for |M|<=1 else
// (1+-sign M)/2, Mach from each side's own speed of sound.
FaceFlux flux_ausm(const Side& o, const Side& n, const v3& Sf, double magSf) {
    v3 U_own = o.rhoU / o.rho, U_nei = n.rhoU / n.rho;
    v3 nrm = Sf / magSf;
    double Uv_own = dot(U_own, nrm), Uv_nei = dot(U_nei, nrm);
    double p_own = o.rho * o.rPsi, p_nei = n.rho * n.rPsi;
    double rhoE_own = o.rho * (o.e + 0.5 * magSqr(U_own));
    double rhoE_nei = n.rho * (n.e + 0.5 * magSqr(U_nei));
    double M_o = Uv_own / o.s, M_n = Uv_nei / n.s;
    double Mp = std::fabs(M_o) <= 1 ? 0.25 * sqr(M_o + 1) : 0.5 * (M_o + std::fabs(M_o));
    double Mm = std::fabs(M_n) <= 1 ? -0.25 * sqr(M_n - 1) : 0.5 * (M_n - std::fabs(M_n));
    double Pp = std::fabs(M_o) <= 1 ? 0.25 * sqr(M_o + 1) * (2 - M_o) : 0.5 * (1 + fsign(M_o));
    double Pm = std::fabs(M_n) <= 1 ? 0.25 * sqr(M_n - 1) * (2 + M_n) : 0.5 * (1 - fsign(M_n));
    double M12 = Mp + Mm;
    double up = pos0(M12);
    FaceFlux F;
    double mdot = M12 * (up * o.rho * o.s + (1 - up) * n.rho * n.s) * magSf;
    F.phi = mdot;
    F.Up = up * U_own + (1 - up) * U_nei;
    F.phiUp = mdot * F.Up + (Pp * p_own + Pm * p_nei) * Sf;
    double H_own = (rhoE_own + p_own) / o.rho, H_nei = (rhoE_nei + p_nei) / n.rho;
    F.phiEp = mdot * (up * H_own + (1 - up) * H_nei);
    return F;
}

// ----------------------------------------------------------------------
// Residual: reconstruction + face fluxes + calcFields (baseFluxDST.C:223-255)
// ----------------------------------------------------------------------
void viscous_terms(Ctx& c);
double mu_of_T(const Ctx& c, double T);
void compute_flux(Ctx& c) {
    const double g = c.gamma;
    const bool kt = (c.o.flux == FLUX_KURGANOV || c.o.flux == FLUX_AUSM);
    // cell fields reconstructed by every scheme (KurganovDST.C:95-132 etc.)
    std::vector<double> rPsi(c.N), e(c.N), s(c.N), rPsi_b(c.NB, 0), e_b(c.NB, 0), s_b(c.NB, 0);
    OMP_FOR
    for (int i = 0; i < c.N; ++i) {
        rPsi[i] = c.R * c.T[i];                 // 1/psi, psi = 1/(R T)
        e[i] = c.h[i] - c.p[i] / c.rho[i];
        if (kt) s[i] = std::sqrt(g * rPsi[i]);
        else {
            double H = std::max(c.rhoE[i] / c.rho[i], SMALL) + std::max(c.p[i] / c.rho[i], SMALL);
            s[i] = std::sqrt(2.0 * (g - 1.0) / (g + 1.0) * H);
        }
    }
    for (int b = 0; b < c.NB; ++b) {
        if (!c.active[b]) continue;
        rPsi_b[b] = c.R * c.T_b[b];
        e_b[b] = c.h_b[b] - c.p_b[b] / c.rho_b[b];
        if (kt) s_b[b] = std::sqrt(g * rPsi_b[b]);
        else {
            double H = std::max(c.rhoE_b[b] / c.rho_b[b], SMALL) + std::max(c.p_b[b] / c.rho_b[b], SMALL);
            s_b[b] = std::sqrt(2.0 * (g - 1.0) / (g + 1.0) * H);
        }
    }
    std::vector<double> rho_o, rho_n, rPsi_o, rPsi_n, e_o, e_n, s_o, s_n;
    std::vector<v3> rhoU_o, rhoU_n;
    reconstruct_scalar(c, c.o.lim_rho, c.rho, c.rho_b, rho_o, rho_n);
    reconstruct_vector(c, c.o.lim_U, c.rhoU, c.rhoU_b, rhoU_o, rhoU_n);
    reconstruct_scalar(c, c.o.lim_T, rPsi, rPsi_b, rPsi_o, rPsi_n);
    reconstruct_scalar(c, c.o.lim_T, e, e_b, e_o, e_n);
    reconstruct_scalar(c, c.o.lim_T, s, s_b, s_o, s_n);
    // HLLCP pressure sensor (HLLCPDST.C:131-164): f = interpolate(fCells^3), boundary 1
    std::vector<double> fface(c.F, 1.0);
    if (c.o.flux == FLUX_HLLCP) {
        std::vector<double> fc(c.N, 1.0);
        OMP_FOR
        for (int i = 0; i < c.N; ++i)
            for (int k : c.cellCells[i]) fc[i] = std::min(fc[i], std::min(c.p[i] / c.p[k], c.p[k] / c.p[i]));
        OMP_FOR
        for (int f = 0; f < c.Fi; ++f)
            fface[f] = c.w[f] * std::pow(fc[c.own[f]], 3) + (1 - c.w[f]) * std::pow(fc[c.nei[f]], 3);
    }
    c.phi.assign(c.F, 0.0);
    c.phiEp.assign(c.F, 0.0);
    c.phiUp.assign(c.F, v3{0, 0, 0});
    c.Up.assign(c.F, v3{0, 0, 0});
    OMP_FOR
    for (int f = 0; f < c.F; ++f) {
        if (f >= c.Fi && !c.active[f - c.Fi]) continue;
        Side so{rho_o[f], rhoU_o[f], rPsi_o[f], e_o[f], s_o[f]};
        Side sn{rho_n[f], rhoU_n[f], rPsi_n[f], e_n[f], s_n[f]};
        FaceFlux F;
        switch (c.o.flux) {
            case FLUX_KURGANOV: F = flux_kurganov(so, sn, c.Sf[f], c.magSf[f]); break;
            case FLUX_HLL: F = flux_hll(so, sn, c.Sf[f], c.magSf[f], g); break;
            case FLUX_HLLC: F = flux_hllc(so, sn, c.Sf[f], c.magSf[f], g, false, 1.0); break;
            case FLUX_HLLCP: F = flux_hllc(so, sn, c.Sf[f], c.magSf[f], g, true, fface[f]); break;
            case FLUX_AUSMPLUS: F = flux_ausm_plus(so, sn, c.Sf[f], c.magSf[f], false, false, 0); break;
            case FLUX_AUSMPLUSUP: F = flux_ausm_plus(so, sn, c.Sf[f], c.magSf[f], true, c.o.low_mach, c.o.mainf); break;
            default: F = flux_ausm(so, sn, c.Sf[f], c.magSf[f]); break;
        }
        c.phi[f] = F.phi; c.phiUp[f] = F.phiUp; c.phiEp[f] = F.phiEp; c.Up[f] = F.Up;
        if (f >= c.Fi) c.phi_b[f - c.Fi] = F.phi;
    }
    // calcFields: R = [div(phi), div(phiUp), div(phiEp)] (fvc::div = surface sum / V)
    c.Rv.assign(c.N, v5{0, 0, 0, 0, 0});
    auto div = [&](int i, auto&& val) {
        double r = 0;
        for (int f : c.cellFaces[i]) r += ((c.own[f] == i) ? 1.0 : -1.0) * val(f);
        return r / c.V[i];
    };
    OMP_FOR
    for (int i = 0; i < c.N; ++i) {
        c.Rv[i][0] = div(i, [&](int f) { return c.phi[f]; });
        for (int k = 0; k < 3; ++k) c.Rv[i][1 + k] = div(i, [&](int f) { return c.phiUp[f][k]; });
        c.Rv[i][4] = div(i, [&](int f) { return c.phiEp[f]; });
    }
    if (c.viscous) viscous_terms(c);
    if (!c.rmask.empty())
        for (int i = 0; i < c.N; ++i)
            if (c.rmask[i]) c.Rv[i] = v5{0, 0, 0, 0, 0};
}

// Laminar viscosity: constTransport mu, or Sutherland As sqrt(T)/(1 + Ts/T)
double mu_of_T(const Ctx& c, double T) {
    if (c.o.As > 0) return c.o.As * std::sqrt(T) / (1.0 + c.o.Ts / T);
    return c.o.mu;
}

// Viscous part of baseFluxDST::calcFields (baseFluxDST.C:229-250):
//   tauMC     = muEff dev2(T(grad U))
//   sigmaDotU = (interpolate(muEff)|Sf| snGrad(U) + Sf . interpolate(tauMC)) . Up
//   R_U      -= laplacian(muEff, U) + div(tauMC),  R_E -= div(sigmaDotU)
// Gauss linear gradient; corrected snGrad  dc (U_N - U_P) + k . (grad U)_f
// with k = n - d dc (foam-extend nonOrthCorrectionVectors); boundary
// snGrad = (U_b - U_P) dc_b and boundary gradient
// grad U_P + n (snGrad_b - n . grad U_P) (gaussGrad::correctBoundaryConditions).
// No heat-conduction term in the energy equation (as in the reference).
void viscous_terms(Ctx& c) {
    typedef std::array<double, 9> t3;
    std::vector<t3> gU;
    grad_vector(c, c.U, c.U_b, gU);
    limit_grad_U(c, gU);
    std::vector<double> muE(c.N), muE_b(c.NB, 0.0);
    OMP_FOR
    for (int i = 0; i < c.N; ++i) muE[i] = mu_of_T(c, c.T[i]) + c.mut[i];
    for (int b = 0; b < c.NB; ++b) if (c.active[b]) muE_b[b] = mu_of_T(c, c.T_b[b]) + c.mut_b[b];
    auto tau_of = [&](const t3& g, double m) {
        // dev2(T(g)) with T(g)(i,j) = g(j,i): t(i,j) = m (g(j,i) - 2/3 tr(g) d_ij)
        double tr = g[0] + g[4] + g[8];
        t3 t;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) t[3 * i + j] = m * (g[3 * j + i] - (i == j ? (2.0 / 3.0) * tr : 0.0));
        return t;
    };
    std::vector<t3> tau(c.N);
    OMP_FOR
    for (int i = 0; i < c.N; ++i) tau[i] = tau_of(gU[i], muE[i]);
    std::vector<v3> lap(c.F, v3{0, 0, 0}), tauS(c.F, v3{0, 0, 0});
    std::vector<double> sig(c.F, 0.0);
    OMP_FOR
    for (int f = 0; f < c.Fi; ++f) {
        int P = c.own[f], Q = c.nei[f];
        double w = c.w[f];
        v3 n = c.Sf[f] / c.magSf[f];
        v3 d = c.C[Q] - c.C[P];
        v3 kc = n - c.dc[f] * d;
        double muf = w * muE[P] + (1 - w) * muE[Q];
        v3 sn;
        for (int j = 0; j < 3; ++j) {
            double corr = 0;
            for (int i = 0; i < 3; ++i) corr += kc[i] * (w * gU[P][3 * i + j] + (1 - w) * gU[Q][3 * i + j]);
            sn[j] = c.dc[f] * (c.U[Q][j] - c.U[P][j]) + corr;
        }
        v3 ts;
        for (int j = 0; j < 3; ++j) {
            double a = 0;
            for (int i = 0; i < 3; ++i) a += c.Sf[f][i] * (w * tau[P][3 * i + j] + (1 - w) * tau[Q][3 * i + j]);
            ts[j] = a;
        }
        lap[f] = (muf * c.magSf[f]) * sn;
        tauS[f] = ts;
        sig[f] = dot(lap[f] + tauS[f], c.Up[f]);
    }
    for (int b = 0; b < c.NB; ++b) {
        if (!c.active[b]) continue;
        int f = c.Fi + b, P = c.own[f];
        v3 n = c.Sf[f] / c.magSf[f];
        v3 snb = c.dc[f] * (c.U_b[b] - c.U[P]);
        t3 gb = gU[P];
        for (int j = 0; j < 3; ++j) {
            double ng = n[0] * gb[j] + n[1] * gb[3 + j] + n[2] * gb[6 + j];
            for (int i = 0; i < 3; ++i) gb[3 * i + j] += n[i] * (snb[j] - ng);
        }
        t3 tb = tau_of(gb, muE_b[b]);
        v3 ts;
        for (int j = 0; j < 3; ++j) ts[j] = c.Sf[f][0] * tb[j] + c.Sf[f][1] * tb[3 + j] + c.Sf[f][2] * tb[6 + j];
        lap[f] = (muE_b[b] * c.magSf[f]) * snb;
        tauS[f] = ts;
        sig[f] = dot(lap[f] + tauS[f], c.Up[f]);
    }
    auto div = [&](int i, auto&& val) {
        double r = 0;
        for (int f : c.cellFaces[i]) r += ((c.own[f] == i) ? 1.0 : -1.0) * val(f);
        return r / c.V[i];
    };
    OMP_FOR
    for (int i = 0; i < c.N; ++i) {
        for (int k = 0; k < 3; ++k) {
            double l = div(i, [&](int f) { return lap[f][k]; });
            double t = div(i, [&](int f) { return tauS[f][k]; });
            c.Rv[i][1 + k] -= l + t;
        }
        c.Rv[i][4] -= div(i, [&](int f) { return sig[f]; });
    }
}

// ----------------------------------------------------------------------
// Roe Jacobian (Roe.C:152-379) + assembly (fluxDST.C:73-127) + ddt
// (fvmDST.C:77-143; Euler: diag = V/dt; steadyStateDST.C:173-198: V rDeltaT)
// ----------------------------------------------------------------------

// Roe<tensor5>::calcJ (Roe.C:247-272): Blazek A.7 flux Jacobian A(W).n
t5 calcJ(const v3& Uf, double gammaf, double phiJf, double a1f, const v3& n) {
    t5 J{};
    double Un = dot(Uf, n);
    for (int k = 0; k < 3; ++k) J[0 * 5 + 1 + k] = n[k];
    for (int k = 0; k < 3; ++k) J[(1 + k) * 5 + 0] = phiJf * n[k] - Uf[k] * Un;
    for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l)
            J[(1 + k) * 5 + 1 + l] = Uf[k] * n[l] + (k == l ? Un : 0.0) - (gammaf - 1) * (n[k] * Uf[l]);
    for (int k = 0; k < 3; ++k) J[(1 + k) * 5 + 4] = (gammaf - 1) * n[k];
    J[4 * 5 + 0] = Un * (phiJf - a1f);
    for (int l = 0; l < 3; ++l) J[4 * 5 + 1 + l] = a1f * n[l] - Un * (gammaf - 1) * Uf[l];
    J[4 * 5 + 4] = gammaf * Un;
    return J;
}

void assemble(Ctx& c, LDU& A) {
    const int N = c.N, Fi = c.Fi;
    const double g = c.gamma, beta = c.o.beta;
    A.d.assign(N, t5{});
    A.u.assign(Fi, t5{});
    A.l.assign(Fi, t5{});
    A.s.assign(N, v5{0, 0, 0, 0, 0});
    // fvmDST::ddt: d = I * ddt diag; s = ddt source - diag*psi (zero within Single)
    // dual2ndDST::fvmDdt (dual2ndDST.C:375-412): diag (rDeltaTau + a) V,
    // source V (rDeltaTau W - b W^n - c W^n-1) less diag W (fvmDST.C:98-125)
    const bool dual = c.o.ddt == DDT_DUAL2ND;
    OMP_FOR
    for (int i = 0; i < N; ++i) {
        double rdt = (c.o.ddt == DDT_EULER) ? 1.0 / c.deltaT : c.rDeltaT[i];
        double dg = dual ? (rdt + c.dual_a) * c.V[i] : rdt * c.V[i];
        for (int k = 0; k < 5; ++k) A.d[i][6 * k] = dg;
        if (dual) {
            const double Wi[5] = {c.rho[i], c.rhoU[i][0], c.rhoU[i][1], c.rhoU[i][2], c.rhoE[i]};
            for (int k = 0; k < 5; ++k)
                A.s[i][k] = c.V[i] * (rdt * Wi[k] - c.dual_b * c.Wn[i][k] - c.dual_c * c.Wnm1[i][k]) - dg * Wi[k];
        }
    }
    // Roe::computeJacobianDST
    std::vector<v3> Uc(N);
    std::vector<double> phiJ(N), a1(N), cc(N);
    OMP_FOR
    for (int i = 0; i < N; ++i) {
        Uc[i] = c.rhoU[i] / c.rho[i];
        phiJ[i] = 0.5 * (g - 1) * magSqr(Uc[i]);
        a1[i] = g * c.rhoE[i] / c.rho[i] - phiJ[i];
        cc[i] = std::sqrt(g * c.R * c.T[i]);   // sqrt(Cp/Cv/psi)
    }
    std::vector<double> lambda(Fi);
    OMP_FOR
    for (int f = 0; f < Fi; ++f) {
        int P = c.own[f], Q = c.nei[f];
        v3 n = c.Sf[f] / c.magSf[f];
        t5 Jo = calcJ(Uc[P], g, phiJ[P], a1[P], n);
        t5 Jn = calcJ(Uc[Q], g, phiJ[Q], a1[Q], n);
        // amaxSf = |interpolate(U).Sf| + |Sf| interpolate(c)  (Roe.C:181-185)
        v3 Uf = c.w[f] * Uc[P] + (1 - c.w[f]) * Uc[Q];
        double cf = c.w[f] * cc[P] + (1 - c.w[f]) * cc[Q];
        double amaxSf = std::fabs(dot(Uf, c.Sf[f])) + c.magSf[f] * cf;
        if (c.viscous) {
            // + |Sf| (muEff_f + alphaEff_f)/rho_f deltaCoeffs (Roe.C:187-199),
            // alpha = mu/Pr, alphat = mut/Prt, rho_f = interpolate(p psi)
            double mP = mu_of_T(c, c.T[P]), mQ = mu_of_T(c, c.T[Q]);
            double muEf = c.w[f] * (mP + c.mut[P]) + (1 - c.w[f]) * (mQ + c.mut[Q]);
            double alEf = c.w[f] * (mP / c.o.Pr + c.mut[P] / c.o.Prt) + (1 - c.w[f]) * (mQ / c.o.Pr + c.mut[Q] / c.o.Prt);
            double rhof = c.w[f] * c.p[P] / (c.R * c.T[P]) + (1 - c.w[f]) * c.p[Q] / (c.R * c.T[Q]);
            lambda[f] = 0.5 * (amaxSf + c.magSf[f] * (muEf + alEf) / rhof * c.dc[f]);
        } else {
            lambda[f] = 0.5 * amaxSf;
        }
        for (int k = 0; k < 25; ++k) {
            double oc = Jo[k] * c.w[f];          // ownerCoeffs *= weights
            double nc = Jn[k] * (1 - c.w[f]);    // neighbourCoeffs *= (1 - weights)
            double I = (k % 6 == 0) ? 1.0 : 0.0;
            A.l[f][k] = -beta * (oc * c.magSf[f] + I * lambda[f]);
            A.u[f][k] = beta * (nc * c.magSf[f] - I * lambda[f]);
        }
    }
    // negSumDiag: d[owner] -= lower, d[neighbour] -= upper
    OMP_FOR
    for (int i = 0; i < N; ++i)
        for (int f : c.cellFaces[i]) {
            if (f >= Fi) break;
            const t5& M = (c.own[f] == i) ? A.l[f] : A.u[f];
            for (int k = 0; k < 25; ++k) A.d[i][k] -= M[k];
        }
    // Boundary Jacobians (Roe::computeBoundaryJacobians, Roe.C:274-379),
    // computed per face in parallel and added in face order
    const double Cv = c.Cv;
    std::vector<t5> pics(c.NB);
    OMP_FOR
    for (int b = 0; b < c.NB; ++b) {
        if (!c.active[b]) continue;
        const int f = Fi + b, ci = c.own[f];
        const v3& pSf = c.Sf[f];
        v3 UB = c.rhoU_b[b] / c.rho_b[b];
        double pB = c.p_b[b], TB = c.T_b[b], rhoB = c.rho_b[b];
        double EB = c.rhoE_b[b] / c.rho_b[b];
        double rRT = rhoB / pB;
        double UBS = dot(UB, pSf);
        t5 dRdXb{};
        dRdXb[0] = UBS * rRT;
        for (int k = 0; k < 3; ++k) dRdXb[1 + k] = rhoB * pSf[k];
        dRdXb[4] = -rhoB / TB * UBS;
        for (int k = 0; k < 3; ++k) {
            dRdXb[(1 + k) * 5 + 0] = rRT * UBS * UB[k] + pSf[k];
            for (int l = 0; l < 3; ++l) dRdXb[(1 + k) * 5 + 1 + l] = rhoB * UB[k] * pSf[l] + (k == l ? rhoB * UBS : 0.0);
            dRdXb[(1 + k) * 5 + 4] = -rhoB / TB * UBS * UB[k];
        }
        dRdXb[20] = (EB * rRT + 1) * UBS;
        for (int l = 0; l < 3; ++l) dRdXb[21 + l] = rhoB * UBS * UB[l] + pSf[l] * (rhoB * EB + pB);
        dRdXb[24] = rhoB * Cv * UBS;
        // dX/dW at the internal cell
        v3 UI = Uc[ci];
        double rhoEI = c.rhoE[ci], pI = c.p[ci], rRho = 1.0 / c.rho[ci];
        double rRhoCv = rRho / Cv;
        double e = rhoEI * rRho - 0.5 * magSqr(UI);
        double RT = pI * rRho;
        double RCv = RT / e;
        t5 dXidWi{};
        dXidWi[0] = RT - RCv * (e - 0.5 * magSqr(UI));
        for (int l = 0; l < 3; ++l) dXidWi[1 + l] = -RCv * UI[l];
        dXidWi[4] = RCv;
        for (int k = 0; k < 3; ++k) {
            dXidWi[(1 + k) * 5 + 0] = -rRho * UI[k];
            dXidWi[(1 + k) * 5 + 1 + k] = rRho;
        }
        dXidWi[20] = rRhoCv * (0.5 * magSqr(UI) - e);
        for (int l = 0; l < 3; ++l) dXidWi[21 + l] = -rRhoCv * UI[l];
        dXidWi[24] = rRhoCv;
        // dX_b/dX_i = diag(valueInternalCoeffs)
        double cp, cT;
        v3 cu;
        internal_coeffs(c, b, cp, cu, cT);
        t5 dXbdXi{};
        dXbdXi[0] = cp; dXbdXi[6] = cu[0]; dXbdXi[12] = cu[1]; dXbdXi[18] = cu[2]; dXbdXi[24] = cT;
        pics[b] = mm(mm(dRdXb, dXbdXi), dXidWi);
    }
    for (int b = 0; b < c.NB; ++b) {
        if (!c.active[b]) continue;
        const int ci = c.own[Fi + b];
        for (int k = 0; k < 25; ++k) A.d[ci][k] += beta * pics[b][k];
    }
    // source -= R V (fluxDST.C:124)
    OMP_FOR
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < 5; ++k) A.s[i][k] -= c.Rv[i][k] * c.V[i];
    // held (halo) cells: identity rows, no source, so their update is zero
    if (!c.rmask.empty()) {
        for (int i = 0; i < N; ++i) {
            if (!c.rmask[i]) continue;
            A.d[i] = t5{};
            for (int k = 0; k < 5; ++k) A.d[i][6 * k] = 1.0;
            A.s[i] = v5{0, 0, 0, 0, 0};
        }
        for (int f = 0; f < Fi; ++f) {
            if (c.rmask[c.own[f]]) A.u[f] = t5{};      // row owner, column neighbour
            if (c.rmask[c.nei[f]]) A.l[f] = t5{};      // row neighbour, column owner
        }
    }
}

// ----------------------------------------------------------------------
// Block linear algebra: Amul, preconditioners, GMRES, BiCGStab and the
// stationary solvers (foam-extend BlockLduMatrix::Amul, BlockDiagonalPrecon,
// BlockILUC0Precon, BlockCholeskyPrecon, BlockGaussSeidelPrecon,
// BlockILUCpPrecon, BlockGMRESSolver, BlockBiCGStabSolver,
// BlockGaussSeidelSolver, BlockILUSolver as instantiated at
// libraries/vector5/Vector5typedefs/Vector5typedefs.C:1602-1708; restated
// from the published algorithms, foam-extend 4.1 is not vendored)
// ----------------------------------------------------------------------
typedef std::vector<v5> Vec;

void Amul(const Ctx& c, const LDU& A, const Vec& x, Vec& y) {
    y.resize(c.N);
    OMP_FOR
    for (int i = 0; i < c.N; ++i) {
        v5 yi = mv(A.d[i], x[i]);
        for (int f : c.cellFaces[i]) {
            if (f >= c.Fi) break;
            v5 a = (c.own[f] == i) ? mv(A.u[f], x[c.nei[f]]) : mv(A.l[f], x[c.own[f]]);
            for (int k = 0; k < 5; ++k) yi[k] += a[k];
        }
        y[i] = yi;
    }
}

double sumProd(const Vec& a, const Vec& b) {
    return det_sum((int)a.size(), [&](int i) {
        double s = 0;
        for (int k = 0; k < 5; ++k) s += a[i][k] * b[i][k];
        return s;
    });
}

// y = x (parallel copy of a block vector)
void vcopy(Vec& y, const Vec& x) {
    y.resize(x.size());
    OMP_FOR
    for (int i = 0; i < (int)x.size(); ++i) y[i] = x[i];
}

// one coarse level of the AMG hierarchy: block CSR (rows ascending, columns
// ascending, the diagonal among them), its diagonal inverses, and the map of
// the finer level's nodes onto it
struct AmgLevel {
    int n = 0;
    std::vector<int> start, col, dslot;
    std::vector<t5> val, dinv;
    std::vector<int> agg;                 // finer node -> node of this level
};

struct PreconData {
    int kind = PRECON_NONE;
    std::vector<AmgLevel> amg;            // levels 1.. (level 0 is the matrix itself)
    int sweeps = 1;                       // Gauss-Seidel sweeps per application
    const LDU* A = nullptr;               // the matrix (Gauss-Seidel residual sweeps)
    std::vector<t5> Dinv;                 // diagonal: inv(D); factored: inv(pivot)
    // factors in CSR per row; rows factorised in the order of key(i): the
    // cell number (mesh order) or the breadth-first rank of rdst_order.h
    std::vector<int> rowStart, col;       // off-diagonal columns per row, by key
    std::vector<t5> val;                  // L D~^-1 (key k < key i) or U (key k > key i) block
    std::vector<std::vector<int>> prow;   // rows of each partition part, by key (independent)
    std::vector<int> rank;                // breadth-first ranks (empty: mesh order)
    int key(int i) const { return rank.empty() ? i : rank[i]; }
};

// rows of each part in ascending order (one part: all rows)
std::vector<std::vector<int>> part_rows(const Ctx& c) {
    if (c.part.empty()) {
        std::vector<std::vector<int>> r(1, std::vector<int>(c.N));
        for (int i = 0; i < c.N; ++i) r[0][i] = i;
        return r;
    }
    int np = 0;
    for (int i = 0; i < c.N; ++i) np = std::max(np, c.part[i] + 1);
    std::vector<std::vector<int>> r(np);
    for (int i = 0; i < c.N; ++i) r[c.part[i]].push_back(i);
    return r;
}

// AMG set-up: the aggregation plan of the cell graph, then per coarse
// level the Galerkin blocks (sums of the finer blocks between two
// aggregates, finer rows ascending, then the finer row's blocks in column
// order) and their diagonal inverses
void build_amg(const Ctx& c, const LDU& A, PreconData& M) {
    const int N = c.N;
    M.A = &A;
    M.Dinv.resize(N);
    for (int i = 0; i < N; ++i) M.Dinv[i] = inv5(A.d[i]);
    std::vector<std::vector<int>> adj(N);
    for (int f = 0; f < c.Fi; ++f) { adj[c.own[f]].push_back(c.nei[f]); adj[c.nei[f]].push_back(c.own[f]); }
    const AmgPlan P = amg_plan(adj, c.o.amg_min_coarse, c.o.amg_max_levels);
    M.amg.clear();
    // finer level as row lists of (column, block); level 0 from the LDU faces
    std::vector<std::vector<std::pair<int, t5>>> rows(N);
    for (int i = 0; i < N; ++i) {
        rows[i].push_back({i, A.d[i]});
        for (int f : c.cellFaces[i]) {
            if (f >= c.Fi) break;
            if (c.own[f] == i) rows[i].push_back({c.nei[f], A.u[f]});
            else rows[i].push_back({c.own[f], A.l[f]});
        }
        std::stable_sort(rows[i].begin(), rows[i].end(), [](auto& a, auto& b) { return a.first < b.first; });
    }
    for (size_t l = 0; l < P.agg.size(); ++l) {
        AmgLevel L;
        L.n = P.n[l + 1];
        L.agg = P.agg[l];
        const auto& cadj = P.adj[l + 1];
        L.start.assign(L.n + 1, 0);
        for (int I = 0; I < L.n; ++I) L.start[I + 1] = L.start[I] + (int)cadj[I].size() + 1;
        L.col.resize(L.start[L.n]);
        L.dslot.resize(L.n);
        for (int I = 0; I < L.n; ++I) {
            std::vector<int> cols(cadj[I]);
            cols.push_back(I);
            std::sort(cols.begin(), cols.end());
            for (size_t q = 0; q < cols.size(); ++q) {
                L.col[L.start[I] + q] = cols[q];
                if (cols[q] == I) L.dslot[I] = L.start[I] + (int)q;
            }
        }
        L.val.assign(L.col.size(), t5{});
        for (int i = 0; i < (int)rows.size(); ++i) {
            const int I = L.agg[i];
            for (auto& e : rows[i]) {
                const int J = L.agg[e.first];
                auto b = L.col.begin() + L.start[I], en = L.col.begin() + L.start[I + 1];
                const int slot = (int)(std::lower_bound(b, en, J) - L.col.begin());
                for (int k = 0; k < 25; ++k) L.val[slot][k] += e.second[k];
            }
        }
        L.dinv.resize(L.n);
        for (int I = 0; I < L.n; ++I) L.dinv[I] = inv5(L.val[L.dslot[I]]);
        std::vector<std::vector<std::pair<int, t5>>> next(L.n);
        for (int I = 0; I < L.n; ++I)
            for (int q = L.start[I]; q < L.start[I + 1]; ++q) next[I].push_back({L.col[q], L.val[q]});
        rows.swap(next);
        M.amg.push_back(std::move(L));
    }
}

void build_precon(const Ctx& c, const LDU& A, PreconData& M) {
    M.kind = c.o.precon;
    const int N = c.N;
    if (M.kind == PRECON_DIAGONAL) {
        M.Dinv.resize(N);
        OMP_FOR
        for (int i = 0; i < N; ++i) M.Dinv[i] = inv5(A.d[i]);
        return;
    }
    if (M.kind == PRECON_AMG) {
        build_amg(c, A, M);
        return;
    }
    if (!lu_factored((Precon)M.kind)) return;
    M.A = &A;
    M.sweeps = c.o.n_sweeps;
    // factorisation order inside the parts: mesh order, or breadth first
    // (rdst_order.h; the default with more than one part)
    {
        int np = 1;
        for (int i = 0; i < (int)c.part.size(); ++i) np = std::max(np, c.part[i] + 1);
        M.rank.clear();
        if (c.o.ilu_order == 1 || (c.o.ilu_order < 0 && np > 1)) {
            std::vector<int> part = c.part.empty() ? std::vector<int>(N, 0) : c.part;
            if (c.bfs_rank.empty() || c.bfs_part != part) {      // once per partition
                std::vector<std::vector<int>> adj(N);
                for (int f = 0; f < c.Fi; ++f) { adj[c.own[f]].push_back(c.nei[f]); adj[c.nei[f]].push_back(c.own[f]); }
                c.bfs_rank = subdomain_bfs_rank(adj, part);
                c.bfs_part = part;
            }
            M.rank = c.bfs_rank;
        }
    }
    // Incomplete block LU in factorisation order (IKJ form; order = key(i),
    // the cell number, or the breadth-first rank inside the parts): for row
    // i, for each k before i in the pattern: L_ik = A_ik inv(U_kk);
    // A_ij -= L_ik U_kj for j after k in the pattern of row i (j == i: the
    // pivot).  ILUC0 keeps every update on
    // the matrix pattern; ILUCp on the pattern extended to the cells within
    // fillInLevel + 1 faces (foam-extend extendedLduAddressing: neighbours
    // of neighbours, level by level); Cholesky keeps only the pivot updates
    // (the diagonal-based factorisation (D~ + L) D~^-1 (D~ + U)); Gauss-Seidel
    // keeps none (pivots = diagonal blocks).  Couplings between cells of
    // different partition parts are dropped (block-Jacobi across parts, as
    // foam-extend's preconditioners treat processor interfaces).
    std::vector<std::vector<std::pair<int, t5>>> rows(N);
    auto same = [&](int a, int b) { return c.part.empty() || c.part[a] == c.part[b]; };
    // row entries in face order (owner row: upper, neighbour row: lower)
    OMP_FOR
    for (int i = 0; i < N; ++i)
        for (int f : c.cellFaces[i]) {
            if (f >= c.Fi) break;
            int P = c.own[f], Q = c.nei[f];
            if (!same(P, Q)) continue;
            if (P == i) rows[i].push_back({Q, A.u[f]});
            else rows[i].push_back({P, A.l[f]});
        }
    if (M.kind == PRECON_ILUCP && c.o.fill_in > 0) {
        // cells within fill_in + 1 faces (inside the part), zero blocks
        std::vector<std::vector<int>> adj(N);
        for (int i = 0; i < N; ++i)
            for (auto& e : rows[i]) adj[i].push_back(e.first);
        const t5 zero{};
        OMP_FOR
        for (int i = 0; i < N; ++i) {
            std::vector<int> front = adj[i], seen = adj[i];
            seen.push_back(i);
            for (int lev = 0; lev < c.o.fill_in; ++lev) {
                std::vector<int> next;
                for (int a : front)
                    for (int b2 : adj[a])
                        if (std::find(seen.begin(), seen.end(), b2) == seen.end()) {
                            seen.push_back(b2);
                            next.push_back(b2);
                        }
                for (int b2 : next) rows[i].push_back({b2, zero});
                front.swap(next);
            }
        }
    }
    const bool upd_off = M.kind == PRECON_ILU0 || M.kind == PRECON_ILUCP;
    const bool upd_diag = upd_off || M.kind == PRECON_CHOLESKY;
    // one block per cell pair: faces joining the same pair are summed
    OMP_FOR
    for (int ii = 0; ii < N; ++ii) {
        auto& r = rows[ii];
        std::sort(r.begin(), r.end(), [](auto& a, auto& b) { return a.first < b.first; });
        std::vector<std::pair<int, t5>> m;
        for (auto& e : r) {
            if (!m.empty() && m.back().first == e.first)
                for (int k = 0; k < 25; ++k) m.back().second[k] += e.second[k];
            else m.push_back(e);
        }
        if (!M.rank.empty())
            std::sort(m.begin(), m.end(), [&](auto& a, auto& b) { return M.rank[a.first] < M.rank[b.first]; });
        r.swap(m);
    }
    M.rowStart.assign(N + 1, 0);
    for (int i = 0; i < N; ++i) M.rowStart[i + 1] = M.rowStart[i] + (int)rows[i].size();
    M.col.resize(M.rowStart[N]);
    M.val.resize(M.rowStart[N]);
    OMP_FOR
    for (int i = 0; i < N; ++i)
        for (size_t k = 0; k < rows[i].size(); ++k) {
            M.col[M.rowStart[i] + k] = rows[i][k].first;
            M.val[M.rowStart[i] + k] = rows[i][k].second;
        }
    std::vector<t5> D(A.d.begin(), A.d.end());
    M.Dinv.resize(N);
    // parts are independent (no couplings between them): one part per task,
    // rows of a part in ascending order
    M.prow = part_rows(c);
    if (!M.rank.empty())
        for (auto& rows_p : M.prow)
            std::sort(rows_p.begin(), rows_p.end(), [&](int a, int b) { return M.rank[a] < M.rank[b]; });
    OMP_FOR_DYN
    for (int pp = 0; pp < (int)M.prow.size(); ++pp)
    for (int i : M.prow[pp]) {
        for (int q = M.rowStart[i]; q < M.rowStart[i + 1]; ++q) {
            int k = M.col[q];
            if (M.key(k) >= M.key(i)) break;
            M.val[q] = mm(M.val[q], M.Dinv[k]);          // L_ik
            // for j after k in row k's upper part and in row i's pattern (or j = i)
            for (int r = M.rowStart[k]; r < M.rowStart[k + 1]; ++r) {
                int j = M.col[r];
                if (M.key(j) <= M.key(k)) continue;
                if (j == i) {
                    if (!upd_diag) continue;
                    t5 t = mm(M.val[q], M.val[r]);
                    for (int e = 0; e < 25; ++e) D[i][e] -= t[e];
                } else {
                    if (!upd_off) continue;
                    for (int s = M.rowStart[i]; s < M.rowStart[i + 1]; ++s)
                        if (M.col[s] == j) {
                            t5 t = mm(M.val[q], M.val[r]);
                            for (int e = 0; e < 25; ++e) M.val[s][e] -= t[e];
                            break;
                        }
                }
            }
        }
        M.Dinv[i] = inv5(D[i]);
    }
}

void lu_apply(const Ctx& c, const PreconData& M, Vec& x, const Vec& b, bool upper);

// r = b - A x on AMG level l (0: the step's matrix)
void amg_residual(const Ctx& c, const PreconData& M, int l, const Vec& x, const Vec& b, Vec& r) {
    if (l == 0) {
        Vec t;
        Amul(c, *M.A, x, t);
        r.resize(b.size());
        for (size_t i = 0; i < b.size(); ++i) for (int k = 0; k < 5; ++k) r[i][k] = b[i][k] - t[i][k];
        return;
    }
    const AmgLevel& L = M.amg[l - 1];
    r.resize(L.n);
    for (int I = 0; I < L.n; ++I) {
        v5 a = b[I];
        for (int q = L.start[I]; q < L.start[I + 1]; ++q) {
            v5 t = mv(L.val[q], x[L.col[q]]);
            for (int k = 0; k < 5; ++k) a[k] -= t[k];
        }
        r[I] = a;
    }
}

// damped block-Jacobi sweep x += omega D^-1 (b - A x); from x = 0 when `zero`
void amg_smooth(const Ctx& c, const PreconData& M, int l, Vec& x, const Vec& b, bool zero) {
    const std::vector<t5>& Di = l == 0 ? M.Dinv : M.amg[l - 1].dinv;
    const double w = c.o.amg_omega;
    if (zero) {
        x.resize(b.size());
        for (size_t i = 0; i < b.size(); ++i) {
            v5 t = mv(Di[i], b[i]);
            for (int k = 0; k < 5; ++k) x[i][k] = w * t[k];
        }
        return;
    }
    Vec r;
    amg_residual(c, M, l, x, b, r);
    for (size_t i = 0; i < b.size(); ++i) {
        v5 t = mv(Di[i], r[i]);
        for (int k = 0; k < 5; ++k) x[i][k] += w * t[k];
    }
}

// x = V-cycle on level l from x = 0: nPreSweeps sweeps, the residual
// summed over the aggregates, the coarse correction injected back, then
// nPostSweeps sweeps; the coarsest level takes amg.coarsestSweeps sweeps
void amg_vcycle(const Ctx& c, const PreconData& M, int l, Vec& x, const Vec& b) {
    const int nl = (int)M.amg.size() + 1;
    if (l == nl - 1) {
        amg_smooth(c, M, l, x, b, true);
        for (int s = 1; s < c.o.amg_coarsest_sweeps; ++s) amg_smooth(c, M, l, x, b, false);
        return;
    }
    bool zero = true;
    for (int s = 0; s < c.o.amg_pre; ++s) { amg_smooth(c, M, l, x, b, zero); zero = false; }
    if (zero) x.assign(b.size(), v5{0, 0, 0, 0, 0});
    Vec r;
    amg_residual(c, M, l, x, b, r);
    const AmgLevel& L = M.amg[l];
    Vec bc(L.n, v5{0, 0, 0, 0, 0}), xc;
    for (size_t i = 0; i < r.size(); ++i) for (int k = 0; k < 5; ++k) bc[L.agg[i]][k] += r[i][k];
    amg_vcycle(c, M, l + 1, xc, bc);
    for (size_t i = 0; i < x.size(); ++i) for (int k = 0; k < 5; ++k) x[i][k] += xc[L.agg[i]][k];
    for (int s = 0; s < c.o.amg_post; ++s) amg_smooth(c, M, l, x, b, false);
}

void precondition(const Ctx& c, const PreconData& M, Vec& x, const Vec& b) {
    const int N = c.N;
    x.resize(N);
    if (M.kind == PRECON_NONE) { x = b; return; }
    if (M.kind == PRECON_DIAGONAL) {
        OMP_FOR
        for (int i = 0; i < N; ++i) x[i] = mv(M.Dinv[i], b[i]);
        return;
    }
    if (M.kind == PRECON_AMG) {
        amg_vcycle(c, M, 0, x, b);
        return;
    }
    if (M.kind == PRECON_GAUSS_SEIDEL) {
        // forward sweeps x += (D + L)^-1 (b - A x) from x = 0, L the
        // same-part strict lower blocks (BlockGaussSeidelPrecon)
        Vec r, z, t;
        lu_apply(c, M, x, b, false);
        for (int sw = 1; sw < M.sweeps; ++sw) {
            Amul(c, *M.A, x, t);
            r.resize(N);
            OMP_FOR
            for (int i = 0; i < N; ++i) for (int k = 0; k < 5; ++k) r[i][k] = b[i][k] - t[i][k];
            lu_apply(c, M, z, r, false);
            OMP_FOR
            for (int i = 0; i < N; ++i) for (int k = 0; k < 5; ++k) x[i][k] += z[i][k];
        }
        return;
    }
    lu_apply(c, M, x, b, true);
}

// x = (L U)^-1 b with the stored factors, per part (independent): forward
// y_i = b_i - sum_{k<i} L_ik y_k, then backward x_i = inv(U_ii) (y_i -
// sum_{j>i} U_ij x_j) (without the U terms when `upper` is false)
void lu_apply(const Ctx& c, const PreconData& M, Vec& x, const Vec& b, bool upper) {
    x.resize(c.N);
    OMP_FOR_DYN
    for (int pp = 0; pp < (int)M.prow.size(); ++pp) {
        const std::vector<int>& rows = M.prow[pp];
        for (int i : rows) {
            v5 y = b[i];
            for (int q = M.rowStart[i]; q < M.rowStart[i + 1]; ++q) {
                int k = M.col[q];
                if (M.key(k) >= M.key(i)) break;
                v5 t = mv(M.val[q], x[k]);
                for (int e = 0; e < 5; ++e) y[e] -= t[e];
            }
            x[i] = y;
        }
        for (int r = (int)rows.size() - 1; r >= 0; --r) {
            const int i = rows[r];
            v5 y = x[i];
            for (int q = M.rowStart[i]; q < M.rowStart[i + 1] && upper; ++q) {
                int j = M.col[q];
                if (M.key(j) <= M.key(i)) continue;
                v5 t = mv(M.val[q], x[j]);
                for (int e = 0; e < 5; ++e) y[e] -= t[e];
            }
            x[i] = mv(M.Dinv[i], y);
        }
    }
}

// foam normFactor: sum(|A x - A xRef| + |b - A xRef|) + small, xRef = average(x)
double norm_factor(const Ctx& c, const LDU& A, const Vec& x, const Vec& b, const Vec& Ax) {
    v5 xr{0, 0, 0, 0, 0};
    for (int k = 0; k < 5; ++k) xr[k] = det_sum(c.N, [&](int i) { return x[i][k]; }) / c.N;
    Vec xref(c.N, xr), pA;
    Amul(c, A, xref, pA);
    double s = det_sum(c.N, [&](int i) {
        double a = 0, bb = 0;
        for (int k = 0; k < 5; ++k) { a += sqr(Ax[i][k] - pA[i][k]); bb += sqr(b[i][k] - pA[i][k]); }
        return std::sqrt(a) + std::sqrt(bb);
    });
    return s + SOLVER_SMALL;
}

void cmpt_residual(const Vec& r, double nf, double* out) {
    for (int k = 0; k < 5; ++k) out[k] = det_sum((int)r.size(), [&](int i) { return std::fabs(r[i][k]); }) / nf;
}

// the solver performance's converged(): every component below the
// tolerance or below relTol x initial (maxIter aside)
bool tolerances_reached(const Options& o, const double* ini, const double* fin) {
    bool tol = true, rel = o.rel_tol > 0;
    for (int k = 0; k < 5; ++k) {
        if (!(fin[k] < o.tolerance)) tol = false;
        if (!(fin[k] < o.rel_tol * ini[k])) rel = false;
    }
    return tol || rel;
}

bool converged(const Options& o, const double* ini, const double* fin, int it) {
    if (it < o.min_iter) return false;
    bool tol = true, rel = o.rel_tol > 0;
    for (int k = 0; k < 5; ++k) {
        if (!(fin[k] < o.tolerance)) tol = false;
        if (!(fin[k] < o.rel_tol * ini[k])) rel = false;
    }
    return tol || rel || it >= o.max_iter;
}

// Solve A dx = s (dependentVariable deltaW form; the W form's residual
// normalisation is kept by evaluating normFactor on x = W, b = A W + s).
void linear_solve(Ctx& c, const LDU& A, const PreconData& M, Vec& dx, Report& rep) {
    const int N = c.N;
    const Options& o = c.o;
    Vec x0(N), Ax0, b(N);
    OMP_FOR
    for (int i = 0; i < N; ++i) x0[i] = {c.rho[i], c.rhoU[i][0], c.rhoU[i][1], c.rhoU[i][2], c.rhoE[i]};
    double nf;
    if (o.dependent_W) {
        Amul(c, A, x0, Ax0);
        OMP_FOR
        for (int i = 0; i < N; ++i) for (int k = 0; k < 5; ++k) b[i][k] = Ax0[i][k] + A.s[i][k];
        nf = norm_factor(c, A, x0, b, Ax0);
    } else {
        Vec z(N, v5{0, 0, 0, 0, 0}), Az(N, v5{0, 0, 0, 0, 0});
        nf = norm_factor(c, A, z, A.s, Az);
    }
    dx.assign(N, v5{0, 0, 0, 0, 0});
    Vec r = A.s;                          // b - A*0
    cmpt_residual(r, nf, rep.lin_initial);
    std::copy(rep.lin_initial, rep.lin_initial + 5, rep.lin_final);
    int it = 0;
    if (o.solver == SOLVER_GMRES) {
        const int m = o.n_directions;
        std::vector<Vec> Vk(m + 1);
        std::vector<double> H((m + 1) * m), bh(m + 1), yh(m), cs(m), sn(m);
        Vec w, t;
        while (!converged(o, rep.lin_initial, rep.lin_final, it)) {
            precondition(c, M, w, r);
            double beta = std::sqrt(sumProd(w, w));
            std::fill(bh.begin(), bh.end(), 0.0);
            std::fill(H.begin(), H.end(), 0.0);
            bh[0] = beta;
            int used = 0;
            for (int i = 0; i < m; ++i) {
                if (beta == 0.0) break;          // lucky breakdown
                Vk[i].resize(N);
                {
                    Vec& Vi = Vk[i];
                    OMP_FOR
                    for (int q = 0; q < N; ++q) for (int k = 0; k < 5; ++k) Vi[q][k] = w[q][k] / beta;
                }
                Amul(c, A, Vk[i], t);
                precondition(c, M, w, t);
                for (int j = 0; j <= i; ++j) {   // modified Gram-Schmidt
                    double hji = sumProd(w, Vk[j]);
                    H[j * m + i] = hji;
                    const Vec& Vj = Vk[j];
                    OMP_FOR
                    for (int q = 0; q < N; ++q) for (int k = 0; k < 5; ++k) w[q][k] -= hji * Vj[q][k];
                }
                beta = std::sqrt(sumProd(w, w));
                for (int j = 0; j < i; ++j) {   // previous Givens rotations
                    double Hji = H[j * m + i];
                    H[j * m + i] = cs[j] * Hji - sn[j] * H[(j + 1) * m + i];
                    H[(j + 1) * m + i] = sn[j] * Hji + cs[j] * H[(j + 1) * m + i];
                }
                double hh = H[i * m + i];        // givensRotation(H[i][i], beta, c, s)
                if (beta == 0.0) { cs[i] = 1; sn[i] = 0; }
                else if (std::fabs(beta) > std::fabs(hh)) {
                    double tau = -hh / beta; sn[i] = 1.0 / std::sqrt(1.0 + tau * tau); cs[i] = sn[i] * tau;
                } else {
                    double tau = -beta / hh; cs[i] = 1.0 / std::sqrt(1.0 + tau * tau); sn[i] = cs[i] * tau;
                }
                double bhi = bh[i];
                bh[i] = cs[i] * bhi - sn[i] * bh[i + 1];
                bh[i + 1] = sn[i] * bhi + cs[i] * bh[i + 1];
                H[i * m + i] = cs[i] * H[i * m + i] - sn[i] * beta;
                used = i + 1;
            }
            for (int i = used - 1; i >= 0; --i) {
                double sum = bh[i];
                for (int j = i + 1; j < used; ++j) sum -= H[i * m + j] * yh[j];
                yh[i] = sum / H[i * m + i];
            }
            OMP_FOR
            for (int q = 0; q < N; ++q)
                for (int i = 0; i < used; ++i) for (int k = 0; k < 5; ++k) dx[q][k] += yh[i] * Vk[i][q][k];
            Amul(c, A, dx, t);
            OMP_FOR
            for (int q = 0; q < N; ++q) for (int k = 0; k < 5; ++k) r[q][k] = A.s[q][k] - t[q][k];
            cmpt_residual(r, nf, rep.lin_final);
            ++it;
        }
    } else if (o.solver == SOLVER_GAUSS_SEIDEL || o.solver == SOLVER_ILU || o.solver == SOLVER_AMG) {
        // stationary iteration dx += M^-1 (b - A dx) with Gauss-Seidel sweeps
        // or the Cholesky-type factorisation (BlockGaussSeidelSolver,
        // BlockILUSolver), the residual checked after every application
        Vec z, t;
        while (!converged(o, rep.lin_initial, rep.lin_final, it)) {
            precondition(c, M, z, r);
            OMP_FOR
            for (int q = 0; q < N; ++q) for (int k = 0; k < 5; ++k) dx[q][k] += z[q][k];
            Amul(c, A, dx, t);
            OMP_FOR
            for (int q = 0; q < N; ++q) for (int k = 0; k < 5; ++k) r[q][k] = A.s[q][k] - t[q][k];
            cmpt_residual(r, nf, rep.lin_final);
            ++it;
        }
    } else {
        // BiCGStab (van der Vorst), right preconditioned
        double rho = 1e300, rhoOld, alpha = 0, omega = 1e300, beta;
        Vec p(N, v5{0, 0, 0, 0, 0}), v(N, v5{0, 0, 0, 0, 0}), ph, s(N), sh, t2, rw = r;
        while (!converged(o, rep.lin_initial, rep.lin_final, it)) {
            rhoOld = rho;
            rho = sumProd(rw, r);
            beta = rho / rhoOld * (alpha / omega);
            OMP_FOR
            for (int q = 0; q < N; ++q) for (int k = 0; k < 5; ++k) p[q][k] = r[q][k] + beta * (p[q][k] - omega * v[q][k]);
            precondition(c, M, ph, p);
            Amul(c, A, ph, v);
            alpha = rho / sumProd(rw, v);
            OMP_FOR
            for (int q = 0; q < N; ++q) for (int k = 0; k < 5; ++k) s[q][k] = r[q][k] - alpha * v[q][k];
            precondition(c, M, sh, s);
            Amul(c, A, sh, t2);
            double tt = sumProd(t2, t2);
            omega = tt > 0 ? sumProd(t2, s) / tt : 0.0;
            OMP_FOR
            for (int q = 0; q < N; ++q)
                for (int k = 0; k < 5; ++k) {
                    dx[q][k] += alpha * ph[q][k] + omega * sh[q][k];
                    r[q][k] = s[q][k] - omega * t2[q][k];
                }
            cmpt_residual(r, nf, rep.lin_final);
            ++it;
        }
    }
    rep.lin_iterations = it;
}

// ----------------------------------------------------------------------
// updateFields.H:40-94 (W -> rho, U, h, T, p with min/max bounding; the
// bounding is a clamp to [min, max], a simplification of foam's boundMinMax
// that only differs when a bound is active)
// ----------------------------------------------------------------------
void update_fields(Ctx& c, const Vec& dx) {
    int any = 0;
    OMP_FOR_REDUCE_OR_ANY
    for (int i = 0; i < c.N; ++i) {
        bool bnd = false;
        auto clampv = [&](double v, double lo, double hi) {
            if (v < lo) { bnd = true; return lo; }
            if (v > hi) { bnd = true; return hi; }
            return v;
        };
        c.rho[i] += dx[i][0];
        for (int k = 0; k < 3; ++k) c.rhoU[i][k] += dx[i][1 + k];
        c.rhoE[i] += dx[i][4];
        c.rho[i] = clampv(c.rho[i], c.o.rho_min, c.o.rho_max);
        c.U[i] = c.rhoU[i] / c.rho[i];
        double hh = c.Cp / c.Cv * (c.rhoE[i] / c.rho[i] - 0.5 * magSqr(c.U[i]));
        c.h[i] = clampv(hh, c.Cp * c.o.T_min, c.Cp * c.o.T_max);
        c.T[i] = c.h[i] / c.Cp;                       // thermo.correct(): hConstThermo
        c.p[i] = clampv(c.rho[i] * c.R * c.T[i], c.o.p_min, c.o.p_max);   // p = rho/psi
        if (bnd) any = 1;
    }
    c.bounded = any != 0;
    eval_boundary(c);
}

// ----------------------------------------------------------------------
// Time control (timeDST.C:67-443)
// ----------------------------------------------------------------------
void set_steady_dt(Ctx& c) {           // setSteadyStateDeltaT (timeDST.C:218-273)
    const double g = c.gamma;
    c.rDeltaT.assign(c.N, 0.0);
    if (!c.o.neighbouring) {
        // the cell-centre definition divides by the scalar courant
        // (timeDST.C:221-227), not the per-cell field that setCourantDST
        // ramps: with neighbouring false a steady run keeps initialCo
        OMP_FOR
        for (int i = 0; i < c.N; ++i) {
            double cs = std::sqrt(g * c.R * c.T[i]);
            double lambdaC = (std::fabs(c.U[i][0]) + cs) * c.dS[i][0] + (std::fabs(c.U[i][1]) + cs) * c.dS[i][1] +
                             (std::fabs(c.U[i][2]) + cs) * c.dS[i][2];
            c.rDeltaT[i] = lambdaC / (c.courant * c.V[i]);
        }
        return;
    }
    OMP_FOR
    for (int i = 0; i < c.N; ++i)               // max over the cell's faces (order-free)
        for (int f : c.cellFaces[i]) {
            if (f >= c.Fi) break;
            int P = c.own[f], Q = c.nei[f];
            v3 Uf = c.w[f] * c.U[P] + (1 - c.w[f]) * c.U[Q];
            double cf = c.w[f] * std::sqrt(g * c.R * c.T[P]) + (1 - c.w[f]) * std::sqrt(g * c.R * c.T[Q]);
            double dtSf = (mag(Uf) + cf) * c.dc[f];
            c.rDeltaT[i] = std::max(c.rDeltaT[i], dtSf);
        }
    for (int b = 0; b < c.NB; ++b) {
        if (!c.active[b]) continue;
        if (c.patches[c.bpatch[b]].type != RDST_PATCH_WALL) continue;
        int f = c.Fi + b, ci = c.own[f];
        double pLambda = 0.5 * c.dc[f] * std::sqrt(g * c.R * c.T[ci]) + mag(c.U[ci]);
        c.rDeltaT[ci] = std::max(c.rDeltaT[ci], pLambda);
    }
    for (int i = 0; i < c.N; ++i) c.rDeltaT[i] /= c.courantField[i];
}

void set_transient_dt(Ctx& c) {        // setTransientDeltaT (timeDST.C:275-314)
    const double g = c.gamma;
    double m = 1e300;
    if (!c.o.neighbouring) {
        for (int i = 0; i < c.N; ++i) {
            double cs = std::sqrt(g * c.R * c.T[i]);
            double lambdaC = (std::fabs(c.U[i][0]) + cs) * c.dS[i][0] + (std::fabs(c.U[i][1]) + cs) * c.dS[i][1] +
                             (std::fabs(c.U[i][2]) + cs) * c.dS[i][2];
            m = std::min(m, c.courant * c.V[i] / lambdaC);
        }
    } else {
        for (int f = 0; f < c.Fi; ++f) {
            int P = c.own[f], Q = c.nei[f];
            v3 Uf = c.w[f] * c.U[P] + (1 - c.w[f]) * c.U[Q];
            double cf = c.w[f] * std::sqrt(g * c.R * c.T[P]) + (1 - c.w[f]) * std::sqrt(g * c.R * c.T[Q]);
            double amaxSf = std::fabs(dot(Uf, c.Sf[f])) + c.magSf[f] * cf;
            double dtSf = c.magSf[f] / (amaxSf * c.dc[f]);
            m = std::min(m, dtSf * c.courant);
        }
    }
    c.deltaT = m;
}

void courant_update(Ctx& c, double residualR, bool pseudo);

void set_courant(Ctx& c, Report& rep) {   // setCourantDST (timeDST.C:316-443), no solverPerf
    double ss = det_sum(c.N, [&](int i) {     // gSumSqr(mag(R))
        double m2 = 0;
        for (int k = 0; k < 5; ++k) m2 += sqr(c.Rv[i][k]);
        return m2;
    });
    double residualR = std::sqrt(ss);
    rep.res_mag = residualR;
    courant_update(c, residualR, c.o.ddt == DDT_STEADY);
}

// setCourantDST after residualR is known: the residual ratio, then the
// per-cell ramp and local time step (steady state, or a dual-time inner
// iteration before its convergence) or the scalar courant and the global
// time step (adjustTimeStep)
void courant_update(Ctx& c, double residualR, bool pseudo) {
    if (c.residual != -1) c.residualRatio = std::min(std::max(c.residual / residualR, 0.1), 2.0);
    c.residual = residualR;
    if (pseudo) {
        std::vector<double> factor(c.N, 1.0), eNew(c.N);
        OMP_FOR
        for (int i = 0; i < c.N; ++i) eNew[i] = c.rhoE[i] / c.rho[i] - 0.5 * magSqr(c.rhoU[i] / c.rho[i]);
        auto drop = [&](int k) { return c.rho[k] < 0.95 * c.rhoOld[k] || eNew[k] < 0.95 * c.eOld[k] || eNew[k] < SMALL; };
        OMP_FOR
        for (int i = 0; i < c.N; ++i)               // min over the cell's faces (order-free)
            for (int f : c.cellFaces[i]) {
                if (f >= c.Fi) break;
                const int k = c.own[f] == i ? c.nei[f] : c.own[f];
                if (drop(i)) factor[i] = std::min(factor[i], 0.5);
                if (drop(k)) factor[i] = std::min(factor[i], 0.75);
            }
        c.rhoOld = c.rho;
        c.eOld = eNew;
        OMP_FOR
        for (int i = 0; i < c.N; ++i)
            c.courantField[i] = std::min(std::max(c.courantField[i] * c.residualRatio * factor[i], c.o.min_co), c.o.max_co);
        set_steady_dt(c);
    } else if (c.o.adjust_time_step) {
        c.courant = std::min(std::max(c.courant * c.residualRatio, c.o.min_co), c.o.max_co);
        set_transient_dt(c);
    }
}

void initialize_time(Ctx& c) {           // timeDST::initialize (timeDST.C:67-208)
    c.rhoOld.resize(c.N);
    c.eOld.resize(c.N);
    for (int i = 0; i < c.N; ++i) {
        c.rhoOld[i] = c.p[i] / (c.R * c.T[i]);     // thermo rho = p psi
        c.eOld[i] = c.h[i] * c.Cv / c.Cp;
    }
    c.dS.assign(c.N, v3{0, 0, 0});
    if (!c.o.neighbouring) {
        for (int f = 0; f < c.F; ++f) {
            if (f >= c.Fi && !c.active[f - c.Fi]) continue;
            v3 a{std::fabs(c.Sf[f][0]), std::fabs(c.Sf[f][1]), std::fabs(c.Sf[f][2])};
            c.dS[c.own[f]] = c.dS[c.own[f]] + a;
            if (f < c.Fi) c.dS[c.nei[f]] = c.dS[c.nei[f]] + a;
        }
        for (auto& d : c.dS) d = 0.5 * d;
    }
    c.residual = -1;
    c.residualRatio = 1;
    c.courant = c.o.initial_co;
    c.courantField.assign(c.N, c.courant);
    c.deltaT = c.o.delta_t;
    if (c.o.ddt == DDT_STEADY) set_steady_dt(c);
    else {
        set_transient_dt(c);          // unconditional in timeDST::initialize (timeDST.C:196-205)
        set_steady_dt(c);
    }
}

// ----------------------------------------------------------------------
// Spalart-Allmaras, segregated nuTilda equation after the coupled update
// (turbulence_.correct(), Single.C:101): SAneg (SAneg.C:490-605, negative
// nuTilda and the modified Stilda of Allmaras et al. 2012), SARC1
// (SARC1.C:125-180, 619-697) and SARC2 (SARC2.C:121-155, 425-488).
// Discretisation of the foam-extend fvMatrix
// (restated, not vendored): ddt with the flow's ddt scheme; upwind
// convection with the flow's face mass flux phi; Gauss linear corrected
// diffusion; explicit Cb2 |grad nuTilda|^2; implicit Sp parts of the
// destruction terms; fvMatrix::relax (diagonal made dominant, divided by
// alpha); solved by a fixed number of point-Jacobi sweeps.
// ----------------------------------------------------------------------
struct SACoeffs {
    double sigmaNut = 0.66666, kappa = 0.41, Cb1 = 0.1355, Cb2 = 0.622, Cw2 = 0.3, Cw3 = 2.0, Cv1 = 7.1, Cv2 = 5.0;
    double Cn1 = 16.0, Cn2 = 0.7, Cn3 = 0.9, Ct3 = 1.2, Ct4 = 0.5, Cr1 = 1.0, Cr2 = 2.0, Cr3 = 1.0;
    double Cr2_SARC1 = 12.0;                 // SARC1.C:310-317
    double Cw1() const { return Cb1 / (kappa * kappa) + (1.0 + Cb2) / sigmaNut; }
};
inline double fpos(double s) { return s >= 0 ? 1.0 : 0.0; }   // foam pos(): pos(0) = 1
inline double fneg(double s) { return s < 0 ? 1.0 : 0.0; }

// nuTilda boundary values: fixedValue, inletOutlet on phi, else zeroGradient
void eval_nut_boundary(Ctx& c) {
    for (int b = 0; b < c.NB; ++b) {
        if (!c.active[b]) continue;
        const Patch& P = c.patches[c.bpatch[b]];
        int ci = c.own[c.Fi + b];
        switch (P.bc_nut) {
            case RDST_BC_FIXED_VALUE: c.nut_b[b] = P.nut_value; break;
            case RDST_BC_INLET_OUTLET: c.nut_b[b] = c.phi_b[b] >= 0 ? c.nut[ci] : P.nut_value; break;
            default: c.nut_b[b] = c.nut[ci]; break;
        }
    }
}

// nuTilda valueFraction (for the implicit boundary coefficients)
double nut_vf(const Ctx& c, int b) {
    const Patch& P = c.patches[c.bpatch[b]];
    if (P.bc_nut == RDST_BC_FIXED_VALUE) return 1.0;
    if (P.bc_nut == RDST_BC_INLET_OUTLET) return c.phi_b[b] >= 0 ? 0.0 : 1.0;
    return 0.0;
}

void update_mut(Ctx& c, const std::vector<double>& fv1c) {
    const SACoeffs K;
    const bool neg_sa = c.o.turbulence == TURB_SANEG;
    for (int i = 0; i < c.N; ++i) {
        double m = (neg_sa ? std::fabs(fv1c[i]) : fv1c[i]) * c.nut[i] * c.rho[i];
        c.mut[i] = neg_sa ? std::max(m, 0.0) : m;
    }
    for (int b = 0; b < c.NB; ++b) {
        if (!c.active[b]) continue;
        if (c.patches[c.bpatch[b]].type == RDST_PATCH_WALL) { c.mut_b[b] = 0.0; continue; }
        double chi = c.rho_b[b] * c.nut_b[b] / mu_of_T(c, c.T_b[b]);
        double chi3 = chi * chi * chi;
        double fv1 = chi3 / (chi3 + std::pow(K.Cv1, 3));
        c.mut_b[b] = std::max(fv1 * c.nut_b[b] * c.rho_b[b], 0.0);
    }
}

// symmetric-tensor slot of (a, q): xx xy xz yy yz zz
inline int sym6(int a, int q) {
    static const int T[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    return T[3 * a + q];
}

void sa_correct(Ctx& c) {
    const SACoeffs K;
    const int N = c.N;
    const bool neg_sa = c.o.turbulence == TURB_SANEG;
    const bool sarc1 = c.o.turbulence == TURB_SARC1;
    typedef std::array<double, 9> t3;
    std::vector<t3> gU;
    grad_vector(c, c.U, c.U_b, gU);
    limit_grad_U(c, gU);
    std::vector<v3> gn;
    grad_scalar(c, c.nut, c.nut_b, gn);
    // SARC1 (SARC1.C:125-180, 655-669): S = symm(grad U) per cell; the
    // material derivative ddt(rho, S_ij) + div(phi, S_ij) with the flow's
    // ddt scheme (old time: the last update's S; at the first update the
    // current S, as foam creates an old-time field from the current one),
    // div by Gauss upwind on the step's mass flux, zeroGradient boundary
    // values of S_ij
    std::vector<std::array<double, 6>> Sc;
    std::vector<std::array<double, 6>> DSDt;
    if (sarc1) {
        Sc.resize(N);
        DSDt.resize(N);
        for (int i = 0; i < N; ++i) {
            const t3& g = gU[i];
            for (int a = 0; a < 3; ++a)
                for (int q = a; q < 3; ++q) Sc[i][sym6(a, q)] = 0.5 * (g[3 * a + q] + g[3 * q + a]);
        }
        // under dual-time stepping, dual2ndDST::fvcDdt(rho, S)
        // (dual2ndDST.C:231-372) with the physical step's old times
        const bool dual_ddt = c.o.dual && c.dual_a != 0.0;
        double d_c = 0, d_c0 = 0, d_c00 = 0;
        if (dual_ddt) {
            // Sxx_ = S.component(..) (SARC1.C:655-669) at a new time index
            // stores the old times first (GeometricField::storeOldTimes):
            // S.oo <- S.o, S.o <- S (the last update's S)
            if (c.S_o_idx >= 0 && c.S_idx != c.dual_tidx) {
                if (c.S_oo_idx >= 0) {
                    c.S_oo = c.S_o;
                    c.S_oo_idx = c.S_o_idx;
                }
                c.S_o = c.S_old;
                c.S_o_idx = c.S_idx;
            }
            c.S_idx = c.dual_tidx;
            // fvc::ddt creates S.oldTime() from S, and its oldTime() from
            // that, at first use (with their time indices)
            if (c.S_o_idx < 0) {
                c.S_o = Sc;
                c.S_o_idx = c.S_idx;
            }
            if (c.S_oo_idx < 0) {
                c.S_oo = c.S_o;
                c.S_oo_idx = c.S_o_idx;
            }
            // deltaT0_(vf) (dual2ndDST.C:76-90): GREAT while both old times
            // carry one time index
            const double dt = c.dual_dt, dt0 = (c.S_o_idx == c.S_oo_idx) ? 1.0e15 : c.dual_dt0;
            d_c = 1 + dt / (dt + dt0);
            d_c00 = dt * dt / (dt0 * (dt + dt0));
            d_c0 = d_c + d_c00;
        } else if (!c.S_old_valid) {
            c.S_old = Sc;
        }
        for (int i = 0; i < N; ++i) {
            double rdt = (c.o.ddt == DDT_EULER) ? 1.0 / c.deltaT : c.rDeltaT[i];
            std::array<double, 6> dv{};
            for (int f : c.cellFaces[i]) {
                if (f < c.Fi) {
                    const double ph = c.phi[f];
                    const int up = ph >= 0 ? c.own[f] : c.nei[f];        // upwind, pos(0) = 1
                    const double sg = (c.own[f] == i) ? 1.0 : -1.0;
                    for (int k = 0; k < 6; ++k) dv[k] += sg * ph * Sc[up][k];
                } else {
                    const double ph = c.phi_b[f - c.Fi];
                    for (int k = 0; k < 6; ++k) dv[k] += ph * Sc[i][k];
                }
            }
            if (dual_ddt) {
                const double rdtp = 1.0 / c.dual_dt, ro = c.Wn[i][0], roo = c.Wnm1[i][0];
                for (int k = 0; k < 6; ++k)
                    DSDt[i][k] = rdtp * (d_c * c.rho[i] * Sc[i][k] - d_c0 * ro * c.S_o[i][k] +
                                         d_c00 * roo * c.S_oo[i][k]) + dv[k] / c.V[i];
            } else {
                for (int k = 0; k < 6; ++k)
                    DSDt[i][k] = rdt * (c.rho[i] * Sc[i][k] - c.rho0[i] * c.S_old[i][k]) + dv[k] / c.V[i];
            }
        }
    }
    std::vector<double> mu(N), chi(N), fv1(N), D(N), diag(N), b(N, 0.0);
    for (int i = 0; i < N; ++i) {
        mu[i] = mu_of_T(c, c.T[i]);
        chi[i] = c.rho[i] * c.nut[i] / mu[i];
        double chi3 = chi[i] * chi[i] * chi[i];
        fv1[i] = chi3 / (chi3 + std::pow(K.Cv1, 3));
        const t3& g = gU[i];
        double W2 = 0;                       // |skew(gradU)|^2
        for (int a = 0; a < 3; ++a)
            for (int q = 0; q < 3; ++q) { double w = 0.5 * (g[3 * a + q] - g[3 * q + a]); W2 += w * w; }
        double Omega = std::sqrt(2.0) * std::sqrt(W2);
        double fv2 = 1.0 / std::pow(1.0 + chi[i] / K.Cv2, 3);
        double kd2 = sqr(K.kappa * c.y[i]);
        double Stilda;
        if (neg_sa) {
            double Sbar = fv2 * c.nut[i] / kd2;
            Stilda = Omega + fpos(K.Cn2 * Omega + Sbar) * Sbar +
                     fneg(K.Cn2 * Omega + Sbar) * (Omega * (sqr(K.Cn2) * Omega + K.Cn3 * Sbar)) /
                         std::max((K.Cn3 - 2.0 * K.Cn2) * Omega - Sbar, SMALL);
        } else {
            double cb = chi[i] / K.Cv2;
            double fv3 = (1.0 + chi[i] * fv1[i]) * (1.0 / K.Cv2) * (3 * (1.0 + cb) + sqr(cb)) / std::pow(1.0 + cb, 3);
            Stilda = fv3 * std::sqrt(2.0) * std::sqrt(W2) + fv2 * c.nut[i] / kd2;
        }
        double r = std::min(c.nut[i] / (std::max(Stilda, SMALL) * kd2), 10.0);
        double gg = r + K.Cw2 * (std::pow(r, 6) - r);
        double fw = gg * std::pow((1.0 + std::pow(K.Cw3, 6)) / (std::pow(gg, 6) + std::pow(K.Cw3, 6)), 1.0 / 6.0);
        double V = c.V[i], rho = c.rho[i], nt = c.nut[i];
        double rdt = (c.o.ddt == DDT_EULER) ? 1.0 / c.deltaT : c.rDeltaT[i];
        // fvm::ddt(rho, nuTilda): diag rdt rho V, source rdt rho nuTilda_old V
        diag[i] = rdt * rho * V;
        b[i] = rdt * rho * nt * V;
        if (c.dual_a != 0.0) {
            // dual2ndDST::fvmDdt(rho, vf) (dual2ndDST.C:456-488): diag
            // (rDeltaTau + a) rho V, source V (rDeltaTau rho nuTilda
            // - b rho^n nuTilda^n - c rho^n-1 nuTilda^n-1)
            diag[i] += c.dual_a * rho * V;
            b[i] -= V * (c.dual_b * c.Wn[i][0] * c.nutN[i] + c.dual_c * c.Wnm1[i][0] * c.nutNm1[i]);
        }
        // + Cb2/sigma rho |grad nuTilda|^2 (explicit, moved to the right)
        b[i] += K.Cb2 / K.sigmaNut * rho * magSqr(gn[i]) * V;
        if (neg_sa) {
            double ft2 = K.Ct3 * std::exp(-K.Ct4 * sqr(chi[i]));
            double pp = fpos(nt), nn = fneg(nt);
            b[i] += pp * K.Cb1 * (1.0 - ft2) * rho * Stilda * nt * V;
            diag[i] += pp * (K.Cw1() * fw - K.Cb1 / sqr(K.kappa) * ft2) * nt * rho / sqr(c.y[i]) * V;
            b[i] += nn * K.Cb1 * (1.0 - K.Ct3) * rho * Omega * nt * V;
            diag[i] -= nn * K.Cw1() * nt * rho / sqr(c.y[i]) * V;
            double chi3 = chi[i] * chi[i] * chi[i];
            double fn = fpos(chi[i]) + fneg(chi[i]) * (K.Cn1 + chi3) / (K.Cn1 - chi3);
            D[i] = (rho * nt * fn + mu[i]) / K.sigmaNut;
        } else {
            // SARC2 fr1 (SARC2.C:121-155): rotation/curvature multiplier
            double S2 = 0, W2b = 0;
            for (int a = 0; a < 3; ++a)
                for (int q = 0; q < 3; ++q) {
                    double sy = 0.5 * (g[3 * a + q] + g[3 * q + a]), sk = 0.5 * (g[3 * a + q] - g[3 * q + a]);
                    S2 += sy * sy; W2b += sk * sk;
                }
            double sqrS = 2.0 * S2, sqrW = 2.0 * W2b;
            double rStar = std::sqrt(sqrS / std::max(sqrW, SMALL));
            double fr1;
            if (c.o.turbulence == TURB_SA) {
                fr1 = 1.0;                  // no rotation/curvature multiplier
            } else if (sarc1) {
                // rTilda = 2/(rho max(D^2, SMALL)^2) sum_aq (sum_k W_ak S_qk) DS_aq/Dt, D^2 = (S^2 + W^2)/2
                double sqrD = 0.5 * (sqrS + sqrW);
                double acc = 0;
                for (int a = 0; a < 3; ++a)
                    for (int q = 0; q < 3; ++q) {
                        double ws = 0;
                        for (int k = 0; k < 3; ++k)
                            ws += 0.5 * (g[3 * a + k] - g[3 * k + a]) * Sc[i][sym6(q, k)];
                        acc += ws * DSDt[i][sym6(a, q)];
                    }
                double rTilda = 2.0 / (rho * sqr(std::max(sqrD, SMALL))) * acc;
                fr1 = (1 + K.Cr1) * 2.0 * rStar / (1.0 + rStar) * (1.0 - K.Cr3 * std::atan(K.Cr2_SARC1 * rTilda)) - K.Cr1;
            } else {
                double rrStar = std::sqrt(sqrW / std::max(sqrS, SMALL));
                double rTilda = rrStar * (rrStar - 1.0);
                fr1 = (1 + K.Cr1) * 2.0 * rStar / (1.0 + rStar) * (1.0 - K.Cr3 * std::atan(K.Cr2 * rTilda)) - K.Cr1;
            }
            b[i] += K.Cb1 * rho * Stilda * nt * fr1 * V;
            diag[i] += K.Cw1() * fw * nt * rho / sqr(c.y[i]) * V;
            D[i] = rho * nt / K.sigmaNut + mu[i];
        }
    }
    // face coefficients: upwind convection with phi, corrected diffusion
    std::vector<double> up(c.Fi), lo(c.Fi);
    for (int f = 0; f < c.Fi; ++f) {
        int P = c.own[f], Q = c.nei[f];
        double w = c.w[f], ph = c.phi[f];
        double wu = fpos(ph);
        double Df = w * D[P] + (1 - w) * D[Q];
        double dcoef = Df * c.magSf[f] * c.dc[f];
        // convection: row P: diag += wu phi, upper += (1-wu) phi;
        //             row Q: diag -= (1-wu) phi, lower += -wu phi
        diag[P] += wu * ph;
        diag[Q] -= (1 - wu) * ph;
        up[f] = (1 - wu) * ph - dcoef;
        lo[f] = -wu * ph - dcoef;
        diag[P] += dcoef;
        diag[Q] += dcoef;
        // explicit non-orthogonal correction Df |Sf| k . (grad nuTilda)_f
        v3 n = c.Sf[f] / c.magSf[f];
        v3 kc = n - c.dc[f] * (c.C[Q] - c.C[P]);
        double corr = Df * c.magSf[f] * dot(kc, c.w[f] * gn[P] + (1 - c.w[f]) * gn[Q]);
        // linearUpwind grad(nuTilda): the explicit part of the face value
        // nuTilda_C + (Cf - C) . grad nuTilda_C of the upwind cell C
        // (fvm::div's faceFluxCorrection phi * correction, moved to the source)
        if (c.o.nut_linear_upwind) {
            const int C = ph >= 0 ? P : Q;
            corr -= ph * dot(c.Cf[f] - c.C[C], gn[C]);
        }
        b[P] += corr;
        b[Q] -= corr;
    }
    for (int bb = 0; bb < c.NB; ++bb) {
        if (!c.active[bb]) continue;
        int f = c.Fi + bb, P = c.own[f];
        const Patch& Pt = c.patches[c.bpatch[bb]];
        double fvf = nut_vf(c, bb);
        double ref = Pt.nut_value;
        double ph = c.phi_b[bb];
        // convection through the boundary value f ref + (1-f) nu_P
        diag[P] += ph * (1 - fvf);
        b[P] -= ph * fvf * ref;
        // diffusion: snGrad = f (ref - nu_P) dc
        // DnuTildaEff evaluated on the boundary values
        double mub = mu_of_T(c, c.T_b[bb]);
        double Db;
        if (neg_sa) {
            double chib = c.rho_b[bb] * c.nut_b[bb] / mub, chib3 = chib * chib * chib;
            double fnb = fpos(chib) + fneg(chib) * (K.Cn1 + chib3) / (K.Cn1 - chib3);
            Db = (c.rho_b[bb] * c.nut_b[bb] * fnb + mub) / K.sigmaNut;
        } else {
            Db = c.rho_b[bb] * c.nut_b[bb] / K.sigmaNut + mub;
        }
        double dcoef = Db * c.magSf[f] * c.dc[f] * fvf;
        diag[P] += dcoef;
        b[P] += dcoef * ref;
    }
    // fvMatrix::relax: D0 -> max(D0, sum|offdiag|)/alpha, source += (D - D0) psi
    std::vector<double> sumOff(N, 0.0);
    for (int f = 0; f < c.Fi; ++f) { sumOff[c.own[f]] += std::fabs(up[f]); sumOff[c.nei[f]] += std::fabs(lo[f]); }
    for (int i = 0; i < N; ++i) {
        double D0 = diag[i];
        double Dn = std::max(D0, sumOff[i]) / c.o.nut_relax;
        b[i] += (Dn - D0) * c.nut[i];
        diag[i] = Dn;
    }
    // point-Jacobi sweeps from the current nuTilda
    std::vector<double> x(c.nut), xn(N);
    for (int it = 0; it < c.o.nut_sweeps; ++it) {
        for (int i = 0; i < N; ++i) xn[i] = b[i];
        for (int f = 0; f < c.Fi; ++f) { xn[c.own[f]] -= up[f] * x[c.nei[f]]; xn[c.nei[f]] -= lo[f] * x[c.own[f]]; }
        for (int i = 0; i < N; ++i)
            if (c.rmask.empty() || !c.rmask[i]) x[i] = xn[i] / diag[i];   // held cells keep their nuTilda
    }
    c.nut = x;
    if (!neg_sa) for (auto& v : c.nut) v = std::max(v, 0.0);
    eval_nut_boundary(c);
    update_mut(c, fv1);
    if (sarc1) {                // this update's S is the next one's old time
        c.S_old = Sc;
        c.S_old_valid = true;
    }
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Single::iterate (Single.C:80-104)
void single_iterate(Ctx& c, Report& rep) {
    auto t0 = std::chrono::steady_clock::now();
    compute_flux(c);
    rep.t[0] = seconds_since(t0) * 1e3;
    for (int k = 0; k < 5; ++k) rep.res_l2[k] = std::sqrt(det_sum(c.N, [&](int i) { return sqr(c.Rv[i][k] * c.V[i]); }));
    t0 = std::chrono::steady_clock::now();
    LDU A;
    assemble(c, A);
    rep.t[1] = seconds_since(t0) * 1e3;
    t0 = std::chrono::steady_clock::now();
    PreconData M;
    build_precon(c, A, M);
    rep.t[2] = seconds_since(t0) * 1e3;
    t0 = std::chrono::steady_clock::now();
    Vec dx;
    linear_solve(c, A, M, dx, rep);
    rep.t[3] = seconds_since(t0) * 1e3;
    t0 = std::chrono::steady_clock::now();
    if (c.o.turbulence == TURB_SARC1) c.rho0 = c.rho;     // rho.oldTime() of the turbulence update
    update_fields(c, dx);
    rep.flags = (c.bounded ? 1 : 0) | (tolerances_reached(c.o, rep.lin_initial, rep.lin_final) ? 0 : 8);
    if (c.o.turbulence != TURB_LAMINAR && !c.o.frozen_turbulence) sa_correct(c);   // turbulence_.correct()
    set_courant(c, rep);
    rep.t[4] = seconds_since(t0) * 1e3;
}

// residualControls + steadyCheck (residualControls.C:70-82,
// steadyCheck.C:69-98): the mean of the five normalised initial residuals of
// each inner solve, converged after maxInnerIter iterations, below
// minResudual, or when the scaled slope of log(residual) over the last 20 %
// of the history falls under magConvergedSlope (from iterationStart on)
struct SteadyCheck {
    std::vector<double> residuals;
    int count = 0;
    double residual = 1, slope = 1;
    const Options& o;
    explicit SteadyCheck(const Options& opt) : o(opt) {}
    void add(const double ir[5]) {
        double mean = 0;
        for (int k = 0; k < 5; ++k) mean += ir[k];
        mean /= 5;
        ++count;
        residual = mean;
        residuals.push_back(mean);
    }
    bool converged_now() const {
        return count > o.max_inner_iter || residual < o.min_residual || slope < o.mag_converged_slope;
    }
    bool converged() {
        if (count >= o.iteration_start) {
            double sumXi = 0, sumYi = 0, sumXiSqr = 0, sumYiXi = 0;
            const int N = (int)(0.2 * residuals.size());
            const double maxY = std::log(*std::max_element(residuals.begin(), residuals.end()));
            const double minY = std::log(*std::min_element(residuals.begin(), residuals.end()));
            const double deltaY = maxY - minY;
            for (int i = 0; i < N; ++i) {
                const int xi = (int)residuals.size() - 1 - i;
                const double yi = std::log(residuals[xi]);
                sumXi += xi;
                sumXiSqr += std::pow(xi, 2);
                sumYi += yi;
                sumYiXi += yi * xi;
            }
            slope = (residuals.size() - 1) / deltaY *
                    std::fabs((sumYiXi - sumXi * sumYi / N) / (sumXiSqr - std::pow(sumXi, 2) / N));
        }
        return converged_now();
    }
};

// Dual::iterate (Dual.C:80-124) for one physical time step: inner
// pseudo-time iterations of the coupled system with the dual2ndDST ddt until
// the steadyCheck converges, then the physical time-step control
void dual_iterate(Ctx& c, Report& rep, double dt, double dt0) {
    // old time levels (foam creates them from the current field at first use)
    if (!c.dual_started) {
        c.Wn.resize(c.N);
        for (int i = 0; i < c.N; ++i) c.Wn[i] = {c.rho[i], c.rhoU[i][0], c.rhoU[i][1], c.rhoU[i][2], c.rhoE[i]};
        c.Wnm1 = c.Wn;
        c.nutN = c.nut;
        c.nutNm1 = c.nut;
        c.dual_started = true;
        c.S_idx = c.S_o_idx = c.S_oo_idx = -1;   // SARC1's S history restarts too
    } else {
        c.Wnm1.swap(c.Wn);
        for (int i = 0; i < c.N; ++i) c.Wn[i] = {c.rho[i], c.rhoU[i][0], c.rhoU[i][1], c.rhoU[i][2], c.rhoE[i]};
        c.nutNm1.swap(c.nutN);
        c.nutN = c.nut;
    }
    c.dual_dt = dt;
    c.dual_dt0 = dt0;
    ++c.dual_tidx;
    const bool turb = c.o.turbulence != TURB_LAMINAR;
    // dual2ndDST::fvmDdt coefficients (dual2ndDST.C:391-395)
    c.dual_a = 1.0 / dt + 1.0 / (dt + dt0);
    c.dual_c = dt / (dt0 * (dt + dt0));
    c.dual_b = -(c.dual_a + c.dual_c);
    SteadyCheck rc(c.o);
    int inner = 0;
    do {
        compute_flux(c);
        for (int k = 0; k < 5; ++k) rep.res_l2[k] = std::sqrt(det_sum(c.N, [&](int i) { return sqr(c.Rv[i][k] * c.V[i]); }));
        LDU A;
        assemble(c, A);
        PreconData M;
        build_precon(c, A, M);
        Vec dx;
        linear_solve(c, A, M, dx, rep);
        update_fields(c, dx);
        // turbulence inside the loop when innerCorrectTurbulence
        // (timeDST::correctTurbulence, timeDST.C:460-463; Dual.C:111-112)
        if (turb && c.o.inner_correct_turbulence && !c.o.frozen_turbulence) sa_correct(c);
        rc.add(rep.lin_initial);
        // setCourantDST(&solverPerf): |initialResidual|, pseudo-time branch
        // while the steadyCheck (its last slope) is not converged
        double ir2 = 0;
        for (int k = 0; k < 5; ++k) ir2 += sqr(rep.lin_initial[k]);
        courant_update(c, std::sqrt(ir2), !rc.converged_now());
        ++inner;
    } while (!rc.converged());
    // and once after it otherwise (Dual.C:120-121)
    if (turb && !c.o.inner_correct_turbulence && !c.o.frozen_turbulence) sa_correct(c);
    set_courant(c, rep);             // setCourantDST(): residual of R_, converged: physical time step
    rep.flags = (c.bounded ? 1 : 0) | (tolerances_reached(c.o, rep.lin_initial, rep.lin_final) ? 0 : 8);
    rep.lin_iterations = inner;
    c.dual_a = c.dual_b = c.dual_c = 0;
}

}  // namespace

struct rdst_ctx { Ctx c; };

static rdst_status fail(rdst_ctx* ctx, rdst_status s, const std::string& m) {
    if (ctx) ctx->c.err = m;
    return s;
}

ORACLE_API const char* rdsto_version(void) { return "rdst-oracle fp64 cpu"; }

ORACLE_API rdst_status rdsto_create(const rdst_mesh* m, int32_t n_opts, const char* const* keys,
                                    const char* const* values, rdst_ctx** out) {
    if (!m || !out) return RDST_ERR_ARG;
    *out = nullptr;
    std::unique_ptr<rdst_ctx> h(new rdst_ctx);
    Ctx& c = h->c;
    try {
        c.o = parse_options(n_opts, keys, values);
    } catch (const ConfigError& e) {
        return e.unsupported ? RDST_ERR_UNSUPPORTED : RDST_ERR_CONFIG;
    }
    if (c.o.turbulence != TURB_LAMINAR && !m->wall_distance) return RDST_ERR_MESH;
    c.N = m->n_cells; c.Fi = m->n_internal_faces; c.F = m->n_faces; c.NB = c.F - c.Fi;
    if (c.N <= 0 || c.Fi < 0 || c.F < c.Fi) return RDST_ERR_MESH;
    c.own.assign(m->owner, m->owner + c.F);
    c.nei.assign(m->neighbour, m->neighbour + c.Fi);
    c.Sf.resize(c.F); c.Cf.resize(c.F); c.C.resize(c.N);
    for (int f = 0; f < c.F; ++f)
        for (int k = 0; k < 3; ++k) { c.Sf[f][k] = m->Sf[3 * f + k]; c.Cf[f][k] = m->Cf[3 * f + k]; }
    for (int i = 0; i < c.N; ++i) for (int k = 0; k < 3; ++k) c.C[i][k] = m->C[3 * i + k];
    c.magSf.assign(m->magSf, m->magSf + c.F);
    c.w.assign(m->weights, m->weights + c.F);
    c.dc.assign(m->deltaCoeffs, m->deltaCoeffs + c.F);
    c.V.assign(m->V, m->V + c.N);
    if (m->wall_distance) c.y.assign(m->wall_distance, m->wall_distance + c.N);
    c.bpatch.assign(c.NB, -1);
    c.active.assign(c.NB, 0);
    for (int p = 0; p < m->n_patches; ++p) {
        const rdst_patch& P = m->patches[p];
        Patch q{P.start, P.size, P.type, P.bc_p, P.bc_U, P.bc_T, P.bc_nuTilda, P.p_value, P.T_value,
                P.nuTilda_value, {P.U_value[0], P.U_value[1], P.U_value[2]}};
        c.patches.push_back(q);
        for (int f = P.start; f < P.start + P.size; ++f) {
            if (f < c.Fi || f >= c.F) return RDST_ERR_MESH;
            c.bpatch[f - c.Fi] = p;
            c.active[f - c.Fi] = (P.type != RDST_PATCH_EMPTY);
        }
    }
    for (int b = 0; b < c.NB; ++b) if (c.bpatch[b] < 0) return RDST_ERR_MESH;
    c.cellFaces.assign(c.N, {});
    c.cellCells.assign(c.N, {});
    for (int f = 0; f < c.F; ++f) {
        if (f >= c.Fi && !c.active[f - c.Fi]) continue;
        c.cellFaces[c.own[f]].push_back(f);
        if (f < c.Fi) {
            c.cellFaces[c.nei[f]].push_back(f);
            c.cellCells[c.own[f]].push_back(c.nei[f]);
            c.cellCells[c.nei[f]].push_back(c.own[f]);
        }
    }
    c.R = c.o.R; c.Cp = c.o.Cp; c.Cv = c.o.Cv(); c.gamma = c.o.gamma();
    c.time = c.o.start_time;
    int Nn = c.N, NB = c.NB;
    c.rho.assign(Nn, 1); c.rhoE.assign(Nn, 1); c.p.assign(Nn, 1); c.T.assign(Nn, 1); c.h.assign(Nn, 1);
    c.rhoU.assign(Nn, v3{0, 0, 0}); c.U.assign(Nn, v3{0, 0, 0});
    c.rho_b.assign(NB, 0); c.rhoE_b.assign(NB, 0); c.p_b.assign(NB, 0); c.T_b.assign(NB, 0);
    c.h_b.assign(NB, 0); c.phi_b.assign(NB, 0); c.rhoU_b.assign(NB, v3{0, 0, 0}); c.U_b.assign(NB, v3{0, 0, 0});
    c.fp_b.assign(NB, 0); c.fU_b.assign(NB, 0); c.fT_b.assign(NB, 0);
    c.mut.assign(Nn, 0.0); c.mut_b.assign(NB, 0.0); c.nut.assign(Nn, 0.0); c.nut_b.assign(NB, 0.0);
    c.viscous = (c.o.mu > 0 || c.o.As > 0 || c.o.turbulence != TURB_LAMINAR);
    *out = h.release();
    return RDST_OK;
}

// Threads of the oracle's parallel loops (n <= 0: the OpenMP default).
ORACLE_API int32_t rdsto_set_threads(int32_t n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

// Recursive coordinate bisection of the cells into n_parts parts (longest
// extent, split at the proportional rank; ties by index) and the ILU(0)
// partition set to it: the subdomains of a run on n_parts processors, whose
// ILU factors drop the couplings between processors.
static void rcb_split(const Ctx& c, std::vector<int>& idx, int lo, int hi, int p0, int np, std::vector<int>& part) {
    if (np <= 1 || hi - lo <= 1) {
        for (int i = lo; i < hi; ++i) part[idx[i]] = p0;
        return;
    }
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int i = lo; i < hi; ++i)
        for (int k = 0; k < 3; ++k) { mn[k] = std::min(mn[k], c.C[idx[i]][k]); mx[k] = std::max(mx[k], c.C[idx[i]][k]); }
    int ax = 0;
    for (int k = 1; k < 3; ++k) if (mx[k] - mn[k] > mx[ax] - mn[ax]) ax = k;
    const int nl = np / 2;
    const int mid = lo + (int)((long)(hi - lo) * nl / np);
    std::nth_element(idx.begin() + lo, idx.begin() + mid, idx.begin() + hi, [&](int a, int b) {
        return c.C[a][ax] < c.C[b][ax] || (c.C[a][ax] == c.C[b][ax] && a < b);
    });
    rcb_split(c, idx, lo, mid, p0, nl, part);
    rcb_split(c, idx, mid, hi, p0 + nl, np - nl, part);
}

ORACLE_API rdst_status rdsto_partition_rcb(rdst_ctx* ctx, int32_t n_parts) {
    if (!ctx || n_parts < 1) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    if (n_parts == 1) { c.part.clear(); return RDST_OK; }
    std::vector<int> idx(c.N);
    for (int i = 0; i < c.N; ++i) idx[i] = i;
    c.part.assign(c.N, 0);
    rcb_split(c, idx, 0, c.N, 0, n_parts, c.part);
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_get_partition(rdst_ctx* ctx, int32_t* part) {
    if (!ctx || !part) return RDST_ERR_ARG;
    const Ctx& c = ctx->c;
    for (int i = 0; i < c.N; ++i) part[i] = c.part.empty() ? 0 : c.part[i];
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_set_partition(rdst_ctx* ctx, const int32_t* part) {
    if (!ctx) return RDST_ERR_ARG;
    if (part) ctx->c.part.assign(part, part + ctx->c.N);
    else ctx->c.part.clear();
    return RDST_OK;
}

static void init_from_primitive(Ctx& c) {
    c.S_old_valid = false;          // a new state: SARC1's old-time S restarts from the current one
    c.dual_started = false;         // and the time levels of dual-time stepping from it
    c.dt_save = c.o.delta_t;        // foam Time: deltaT0 of the first step = controlDict deltaT
    for (int i = 0; i < c.N; ++i) {
        c.h[i] = c.Cp * c.T[i];
        c.rho[i] = c.p[i] / (c.R * c.T[i]);
        c.rhoU[i] = c.rho[i] * c.U[i];
        c.rhoE[i] = c.rho[i] * (c.h[i] * c.Cv / c.Cp + 0.5 * magSqr(c.U[i]));
    }
    // initial boundary state (before the first BC evaluation): internal
    // values and mass flux (rho U)_owner . Sf
    for (int b = 0; b < c.NB; ++b) {
        int f = c.Fi + b, ci = c.own[f];
        c.phi_b[b] = dot(c.rhoU[ci], c.Sf[f]);
        c.rho_b[b] = c.rho[ci]; c.T_b[b] = c.T[ci]; c.p_b[b] = c.p[ci]; c.U_b[b] = c.U[ci];
    }
    eval_boundary(c);
    initialize_time(c);
    c.state_set = true;
}

ORACLE_API rdst_status rdsto_set_primitive(rdst_ctx* ctx, const double* p, const double* U, const double* T,
                                           const double* nut) {
    if (!ctx || !p || !U || !T) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    for (int i = 0; i < c.N; ++i) {
        c.p[i] = p[i]; c.T[i] = T[i];
        c.U[i] = {U[3 * i], U[3 * i + 1], U[3 * i + 2]};
        c.nut[i] = nut ? nut[i] : 0.0;
    }
    init_from_primitive(c);
    if (c.o.turbulence != TURB_LAMINAR) {
        eval_nut_boundary(c);
        std::vector<double> fv1(c.N);
        for (int i = 0; i < c.N; ++i) {
            double chi = c.rho[i] * c.nut[i] / mu_of_T(c, c.T[i]);
            fv1[i] = chi * chi * chi / (chi * chi * chi + std::pow(7.1, 3));
        }
        update_mut(c, fv1);
    }
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_set_nu_tilda(rdst_ctx* ctx, const double* nut) {
    if (!ctx || !nut) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    if (c.o.turbulence == TURB_LAMINAR || !c.state_set) return RDST_ERR_ARG;
    for (int i = 0; i < c.N; ++i) c.nut[i] = nut[i];
    eval_nut_boundary(c);
    std::vector<double> fv1(c.N);
    for (int i = 0; i < c.N; ++i) {
        double chi = c.rho[i] * c.nut[i] / mu_of_T(c, c.T[i]);
        fv1[i] = chi * chi * chi / (chi * chi * chi + std::pow(7.1, 3));
    }
    update_mut(c, fv1);
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_get_cells(rdst_ctx* ctx, int32_t n, const int32_t* cells, double* out) {
    if (!ctx || n < 0 || (n > 0 && (!cells || !out))) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    for (int j = 0; j < n; ++j) {
        const int i = cells[j];
        if (i < 0 || i >= c.N) return RDST_ERR_ARG;
        double* o = out + 6L * j;
        o[0] = c.rho[i]; o[1] = c.rhoU[i][0]; o[2] = c.rhoU[i][1]; o[3] = c.rhoU[i][2]; o[4] = c.rhoE[i];
        o[5] = c.o.turbulence != TURB_LAMINAR ? c.nut[i] : 0.0;
    }
    return RDST_OK;
}

// the listed cells' states between steps, as set_conservative after a first
// state (boundary values from the new internal field, time control kept)
// with mu_t from nuTilda
ORACLE_API rdst_status rdsto_set_cells(rdst_ctx* ctx, int32_t n, const int32_t* cells, const double* in) {
    if (!ctx || n < 0 || (n > 0 && (!cells || !in))) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    if (!c.state_set) return RDST_ERR_ARG;
    const bool turb = c.o.turbulence != TURB_LAMINAR;
    for (int j = 0; j < n; ++j) {
        const int i = cells[j];
        if (i < 0 || i >= c.N) return RDST_ERR_ARG;
        const double* v = in + 6L * j;
        c.rho[i] = v[0];
        c.rhoU[i] = {v[1], v[2], v[3]};
        c.rhoE[i] = v[4];
        c.U[i] = c.rhoU[i] / c.rho[i];
        double e = c.rhoE[i] / c.rho[i] - 0.5 * magSqr(c.U[i]);
        c.T[i] = e / c.Cv;
        c.p[i] = c.rho[i] * c.R * c.T[i];
        c.h[i] = c.Cp * c.T[i];
        if (turb) c.nut[i] = v[5];
    }
    c.S_old_valid = false;
    c.dual_started = false;
    c.dt_save = c.o.delta_t;
    eval_boundary(c);
    if (turb) {
        eval_nut_boundary(c);
        std::vector<double> fv1(c.N);
        for (int i = 0; i < c.N; ++i) {
            double chi = c.rho[i] * c.nut[i] / mu_of_T(c, c.T[i]);
            fv1[i] = chi * chi * chi / (chi * chi * chi + std::pow(7.1, 3));
        }
        update_mut(c, fv1);
    }
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_set_held_cells(rdst_ctx* ctx, const uint8_t* mask) {
    if (!ctx) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    if (!mask) c.rmask.clear();
    else c.rmask.assign(mask, mask + c.N);
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_set_conservative(rdst_ctx* ctx, const double* rho, const double* rhoU,
                                              const double* rhoE) {
    if (!ctx || !rho || !rhoU || !rhoE) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    for (int i = 0; i < c.N; ++i) {
        c.U[i] = v3{rhoU[3 * i], rhoU[3 * i + 1], rhoU[3 * i + 2]} / rho[i];
        double e = rhoE[i] / rho[i] - 0.5 * magSqr(c.U[i]);
        c.T[i] = e / c.Cv;
        c.p[i] = rho[i] * c.R * c.T[i];
    }
    if (c.state_set) {
        // fields replaced between steps: boundary values from the new
        // internal field (with the boundary branches of the last
        // evaluation), time-control history kept
        c.S_old_valid = false;
        c.dual_started = false;
        c.dt_save = c.o.delta_t;
        for (int i = 0; i < c.N; ++i) {
            c.h[i] = c.Cp * c.T[i];
            c.rho[i] = rho[i];
            c.rhoU[i] = {rhoU[3 * i], rhoU[3 * i + 1], rhoU[3 * i + 2]};
            c.rhoE[i] = rhoE[i];
        }
        eval_boundary(c);
        return RDST_OK;
    }
    init_from_primitive(c);
    for (int i = 0; i < c.N; ++i) {           // keep the given W exactly
        c.rho[i] = rho[i];
        c.rhoU[i] = {rhoU[3 * i], rhoU[3 * i + 1], rhoU[3 * i + 2]};
        c.rhoE[i] = rhoE[i];
    }
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_get_conservative(rdst_ctx* ctx, double* rho, double* rhoU, double* rhoE) {
    if (!ctx) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    for (int i = 0; i < c.N; ++i) {
        if (rho) rho[i] = c.rho[i];
        if (rhoE) rhoE[i] = c.rhoE[i];
        if (rhoU) for (int k = 0; k < 3; ++k) rhoU[3 * i + k] = c.rhoU[i][k];
    }
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_get_primitive(rdst_ctx* ctx, double* p, double* U, double* T, double* nut) {
    if (!ctx) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    for (int i = 0; i < c.N; ++i) {
        if (p) p[i] = c.p[i];
        if (T) T[i] = c.T[i];
        if (U) for (int k = 0; k < 3; ++k) U[3 * i + k] = c.U[i][k];
        if (nut) nut[i] = c.nut[i];
    }
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_step(rdst_ctx* ctx, int32_t n, rdst_step_report* reps) {
    if (!ctx || n < 0) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    for (int s = 0; s < n; ++s) {
        double dt = c.deltaT;
        const double dt0 = c.dt_save;       // Time::operator++: deltaT0 = deltaTSave, deltaTSave = deltaT
        c.dt_save = dt;
        c.time += dt;                       // runTime++ (rhoDST.C:73)
        Report rep;
        if (c.o.dual) dual_iterate(c, rep, dt, dt0);
        else single_iterate(c, rep);
        for (int i = 0; i < c.N; ++i)
            if (!(c.rho[i] > 0) || !(c.p[i] > 0) || !std::isfinite(c.rhoE[i]))
                return fail(ctx, RDST_ERR_DIVERGED, "non-physical state after step");
        if (reps) {
            rdst_step_report& r = reps[s];
            std::memset(&r, 0, sizeof(r));
            r.time = c.time; r.deltaT = dt;
            if (c.o.ddt == DDT_STEADY) {
                double sc = 0;
                for (double v : c.courantField) sc += v;
                r.courant = sc / c.N;
            } else r.courant = c.courant;
            for (int k = 0; k < 5; ++k) {
                r.res_l2[k] = rep.res_l2[k]; r.lin_initial[k] = rep.lin_initial[k]; r.lin_final[k] = rep.lin_final[k];
            }
            r.res_mag = rep.res_mag;
            r.lin_iterations = rep.lin_iterations;
            r.flags = rep.flags;
            r.rdt_min = *std::min_element(c.rDeltaT.begin(), c.rDeltaT.end());
            r.rdt_max = *std::max_element(c.rDeltaT.begin(), c.rDeltaT.end());
            r.t_flux_ms = rep.t[0]; r.t_jacobian_ms = rep.t[1]; r.t_precond_ms = rep.t[2];
            r.t_krylov_ms = rep.t[3]; r.t_update_ms = rep.t[4];
        }
    }
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_residual(rdst_ctx* ctx, double* out) {
    if (!ctx || !out) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    compute_flux(c);
    for (int i = 0; i < c.N; ++i) for (int k = 0; k < 5; ++k) out[5 * i + k] = c.Rv[i][k];
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_assemble(rdst_ctx* ctx, double* d, double* u, double* l, double* s) {
    if (!ctx) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    compute_flux(c);
    LDU A;
    assemble(c, A);
    for (int i = 0; i < c.N; ++i) {
        if (d) std::memcpy(d + 25 * i, A.d[i].data(), 25 * sizeof(double));
        if (s) std::memcpy(s + 5 * i, A.s[i].data(), 5 * sizeof(double));
    }
    for (int f = 0; f < c.Fi; ++f) {
        if (u) std::memcpy(u + 25 * f, A.u[f].data(), 25 * sizeof(double));
        if (l) std::memcpy(l + 25 * f, A.l[f].data(), 25 * sizeof(double));
    }
    return RDST_OK;
}

// Preconditioner application on a given vector (test hook: exact ILU(0)
// and block-Jacobi checks against dense algebra).
ORACLE_API rdst_status rdsto_precondition(rdst_ctx* ctx, const double* b, double* x) {
    if (!ctx || !b || !x) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    compute_flux(c);
    LDU A;
    assemble(c, A);
    PreconData M;
    build_precon(c, A, M);
    Vec bb(c.N), xx;
    for (int i = 0; i < c.N; ++i) for (int k = 0; k < 5; ++k) bb[i][k] = b[5 * i + k];
    precondition(c, M, xx, bb);
    for (int i = 0; i < c.N; ++i) for (int k = 0; k < 5; ++k) x[5 * i + k] = xx[i][k];
    return RDST_OK;
}

// grad(U) at the current state as the viscous terms use it (test hook:
// Gauss linear, cellLimited when selected), row-major d U_j / d x_i, N x 9.
ORACLE_API rdst_status rdsto_grad_U(rdst_ctx* ctx, double* out) {
    if (!ctx || !out) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    compute_flux(c);
    std::vector<std::array<double, 9>> g;
    grad_vector(c, c.U, c.U_b, g);
    limit_grad_U(c, g);
    for (int i = 0; i < c.N; ++i) for (int k = 0; k < 9; ++k) out[9 * i + k] = g[i][k];
    return RDST_OK;
}

// One linear solve of the current system (test hook): dx[N*5] and the report.
ORACLE_API rdst_status rdsto_linear_solve(rdst_ctx* ctx, double* dx, rdst_step_report* rep) {
    if (!ctx || !dx) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    compute_flux(c);
    LDU A;
    assemble(c, A);
    PreconData M;
    build_precon(c, A, M);
    Vec x;
    Report r;
    linear_solve(c, A, M, x, r);
    for (int i = 0; i < c.N; ++i) for (int k = 0; k < 5; ++k) dx[5 * i + k] = x[i][k];
    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        for (int k = 0; k < 5; ++k) { rep->lin_initial[k] = r.lin_initial[k]; rep->lin_final[k] = r.lin_final[k]; }
        rep->lin_iterations = r.lin_iterations;
    }
    return RDST_OK;
}

ORACLE_API rdst_status rdsto_forces(rdst_ctx* ctx, int32_t patch, const double lift[3], const double drag[3],
                                    const double cofr[3], const double axis[3], double p_ref, double qA,
                                    double l_ref, double out[3]) {
    if (!ctx || !lift || !drag || !out || !cofr || !axis) return RDST_ERR_ARG;
    Ctx& c = ctx->c;
    if (patch < 0 || patch >= (int)c.patches.size()) return fail(ctx, RDST_ERR_ARG, "bad patch");
    const Patch& P = c.patches[patch];
    double Fl = 0, Fd = 0, Mm = 0;
    for (int f = P.start; f < P.start + P.size; ++f) {
        int b = f - c.Fi;
        v3 dF = (c.p_b[b] - p_ref) * c.Sf[f];
        Fl += dF[0] * lift[0] + dF[1] * lift[1] + dF[2] * lift[2];
        Fd += dF[0] * drag[0] + dF[1] * drag[1] + dF[2] * drag[2];
        v3 r = c.Cf[f] - v3{cofr[0], cofr[1], cofr[2]};
        v3 mo{r[1] * dF[2] - r[2] * dF[1], r[2] * dF[0] - r[0] * dF[2], r[0] * dF[1] - r[1] * dF[0]};
        Mm += mo[0] * axis[0] + mo[1] * axis[1] + mo[2] * axis[2];
    }
    out[0] = Fl / qA;
    out[1] = Fd / qA;
    out[2] = Mm / (qA * l_ref);
    return RDST_OK;
}

ORACLE_API const char* rdsto_last_error(const rdst_ctx* ctx) { return ctx ? ctx->c.err.c_str() : ""; }

ORACLE_API void rdsto_destroy(rdst_ctx* ctx) { delete ctx; }

// ---------------------------------------------------------------------
// Unit-test hooks on single faces (known-answer tests of the restatement).
// side arrays: (rho, rhoU x, y, z, rPsi, e, s)
// out: (phi, phiUp x, y, z, phiEp, Up x, y, z)
ORACLE_API void rdsto_face_flux(int32_t scheme, const double* so, const double* sn, const double* Sf,
                                double gamma, double fsens, int32_t lowMach, double Mainf, double* out) {
    Side o{so[0], {so[1], so[2], so[3]}, so[4], so[5], so[6]};
    Side n{sn[0], {sn[1], sn[2], sn[3]}, sn[4], sn[5], sn[6]};
    v3 S{Sf[0], Sf[1], Sf[2]};
    double mS = mag(S);
    FaceFlux F;
    switch (scheme) {
        case FLUX_KURGANOV: F = flux_kurganov(o, n, S, mS); break;
        case FLUX_HLL: F = flux_hll(o, n, S, mS, gamma); break;
        case FLUX_HLLC: F = flux_hllc(o, n, S, mS, gamma, false, 1.0); break;
        case FLUX_HLLCP: F = flux_hllc(o, n, S, mS, gamma, true, fsens); break;
        case FLUX_AUSMPLUS: F = flux_ausm_plus(o, n, S, mS, false, false, 0); break;
        case FLUX_AUSMPLUSUP: F = flux_ausm_plus(o, n, S, mS, true, lowMach != 0, Mainf); break;
        default: F = flux_ausm(o, n, S, mS); break;
    }
    out[0] = F.phi; out[1] = F.phiUp[0]; out[2] = F.phiUp[1]; out[3] = F.phiUp[2]; out[4] = F.phiEp;
    out[5] = F.Up[0]; out[6] = F.Up[1]; out[7] = F.Up[2];
}

// Roe calcJ on a conservative state W = (rho, rhoU, rhoE) and unit normal n
ORACLE_API void rdsto_flux_jacobian(const double* W, const double* n, double gamma, double* out) {
    v3 U{W[1] / W[0], W[2] / W[0], W[3] / W[0]};
    double phiJ = 0.5 * (gamma - 1) * magSqr(U);
    double a1 = gamma * W[4] / W[0] - phiJ;
    t5 J = calcJ(U, gamma, phiJ, a1, v3{n[0], n[1], n[2]});
    for (int k = 0; k < 25; ++k) out[k] = J[k];
}

// limiter function value (for the limiter unit tests)
ORACLE_API double rdsto_limiter(int32_t L, double r) { return tvd_limiter((Limiter)L, r); }

// complex-step residual (test reference for the adjoint)
#include "rdst_cs.inc"
