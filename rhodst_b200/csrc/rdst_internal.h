// rdst_internal.h -- device data layout and kernel launchers of the B200
// fully-coupled step.  Not part of the public ABI (include/rdst.h).
//
// HBM layout (one context, FP64 unless noted):
//   cells      : internal numbering (ILU subdomain-major, wavefront level
//                within a subdomain); state W[N][5] AoS, prim[N][8] AoS
//                (p, T, h, Ux, Uy, Uz, -, -), recon record q[N][8] and its
//                Gauss gradient g[N][24] (7 fields x xyz, padded)
//   faces      : internal faces in foam order, geometry SoA
//                (Sf xyz, |Sf|, w, deltaCoeffs, C_N - C_P xyz, Cf xyz)
//   bfaces     : active (non-empty) boundary faces, compact, SoA geometry,
//                boundary state bs[NB][8] (rho, rhoU xyz, rhoE, p, T, phi)
//   cell->face : CSR of face codes in ascending foam face order
//                (code < Fi: internal face, else Fi + bface)
//   matrix     : SELL-32 block matrix (slices of 32 rows, slot 0 = diagonal,
//                then off-diagonals by column), values entry-interleaved:
//                val[(slot_base)*25 + e*32 + lane], MT = double|float|bf16
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace rdst {

constexpr int QW = 8;     // recon record stride (7 used)
constexpr int GW = 24;    // gradient record stride (21 used)
constexpr int PW = 8;     // prim record stride
constexpr int BW = 8;     // boundary state stride
constexpr int SELL_C = 32;

struct DevPatch {
    int type, bc_p, bc_U, bc_T;
    double p_value, T_value, nut_value;
    double U_value[3];
};

struct DevMesh {
    int N, Fi, NB, n_patches;
    // internal faces (foam order)
    const int* own;
    const int* nei;
    const double* Sf;      // [3][Fi]
    const double* magSf;
    const double* w;
    const double* dc;
    const double* d;       // [3][Fi]  C_N - C_P
    const double* Cf;      // [3][Fi]
    // active boundary faces
    const int* bcell;
    const int* bpatch;
    const int* bface;      // foam face index
    const double* bSf;     // [3][NB]
    const double* bmagSf;
    const double* bdc;
    const double* bCf;     // [3][NB]
    // cells
    const double* V;
    const double* C;       // [3][N]
    const int* cf_start;   // [N+1]
    const int* cf_list;    // face codes
    const int* cc_start;   // [N+1] cell->cell (internal faces), for HLLCP
    const int* cc_list;
    const DevPatch* patches;
};

struct Thermo {
    double R, Cp, Cv, gamma;
};

// Device-resident scalars of one context (time control, solver state).
struct Scalars {
    double time, deltaT, courant, residual, residualRatio;
    double res_mag, res_l2[5];
    double nf;                 // linear solver normFactor
    double lin_initial[5], lin_final[5];
    int lin_iterations;
    int flags;                 // bit0 bounding active, bit1 non-physical state
    int converged;
    double rdt_min, rdt_max, dt_face_min;
    // GMRES
    double beta;
    int gm_active, gm_used;
    double H[64 * 65], bh[65], cs[64], sn[64], yh[64], hcol[2][65];
    // BiCGStab
    double bi_rho, bi_rhoOld, bi_alpha, bi_omega, bi_beta, bi_tt, bi_ts, bi_rwv;
};

// SELL-32 block matrix
template <typename MT>
struct SellMat {
    int N, n_slices;
    const int* slice_off;  // [n_slices+1] slot offsets (slot = 32 lanes)
    const int* slice_w;    // [n_slices] width (blocks per row)
    const int* col;        // [slots*32], -1 padding
    MT* val;               // [slots*32*25]
};

struct IluPlan {
    int n_parts;
    const int* part_row0;     // [n_parts+1] first row of each part (rows contiguous)
    const int* lvl_off;       // [total_levels+1] row offsets (global rows)
    const int* part_lvl0;     // [n_parts+1] first level of each part
    int max_level_rows;
    // factorization update triples: for each off-diagonal lower slot q of row r
    // (in slot order), triples [tr_start[q], tr_start[q+1]) of (slot_kj, slot_rj)
    // with slot_rj = -1 meaning the diagonal
    const int* low_start;     // [N+1] per row: range of lower slots in `low_slot`
    const int* low_slot;      // global SELL flat slot index of L_rk
    const int* low_kdiag;     // row k of each lower slot
    const int* tr_start;      // [n_low+1]
    const int* tr_kj;         // flat slot of U_kj
    const int* tr_rj;         // flat slot of A_rj, or -1 for diag
};

// ---------------------------------------------------------------- helpers
__host__ __device__ inline size_t sell_index(int slot_base_lane, int e) {
    // slot_base_lane = slice_off*32 + k*32 + lane ; entries interleaved by 32
    return (size_t)(slot_base_lane - (slot_base_lane & 31)) * 25 + (size_t)e * 32 + (slot_base_lane & 31);
}

template <typename T> __device__ __forceinline__ double ld(const T* p) { return (double)(*p); }
template <> __device__ __forceinline__ double ld<__nv_bfloat16>(const __nv_bfloat16* p) { return (double)__bfloat162float(*p); }
template <typename T> __device__ __forceinline__ void st(T* p, double v) { *p = (T)v; }
template <> __device__ __forceinline__ void st<__nv_bfloat16>(__nv_bfloat16* p, double v) { *p = __float2bfloat16_rn((float)v); }

// ---------------------------------------------------------------- launchers
// flux / residual (kernels_flux.cu)
void launch_recon(const DevMesh& m, const Thermo& th, int flux, const double* W, const double* prim,
                  const double* bs, double* q, double* qb, cudaStream_t s);
void launch_grad(const DevMesh& m, int limiter_mask, int venkat_mask, double venkat_K, const double* q,
                 const double* qb, double* g, double* psi, const double* prim, double* fcell, bool hllcp,
                 cudaStream_t s);
void launch_face_flux(const DevMesh& m, const Thermo& th, int flux, int lim_rho, int lim_U, int lim_T,
                      bool low_mach, double mainf, const double* q, const double* g, const double* psi,
                      const double* qb, const double* fcell, double* fl, double* bfl, double* bs, cudaStream_t s);
void launch_residual(const DevMesh& m, const double* fl, const double* bfl, double* R, double* rhs,
                     double* partial, cudaStream_t s);
int residual_blocks(int N);

// Jacobian + assembly (kernels_jac.cu)
template <typename MT>
void launch_assemble(const DevMesh& m, const Thermo& th, const SellMat<MT>& A, const int* slot_face,
                     const double* W, const double* prim, const double* bs, const double* rdt_cell,
                     const Scalars* sc, int ddt_steady, double beta, cudaStream_t s);

// linear algebra (kernels_linalg.cu)
template <typename MT>
void launch_spmv(const SellMat<MT>& A, const double* x, double* y, const double* b, cudaStream_t s);
template <typename MT>
void launch_spmv_const(const SellMat<MT>& A, const double* xbar, double* y, cudaStream_t s);
template <typename MT>
void launch_dinv(const SellMat<MT>& A, MT* dinv, cudaStream_t s);
template <typename MT>
void launch_jacobi(int N, const MT* dinv, const double* x, double* y, cudaStream_t s);
template <typename MT>
void launch_ilu_factor(const SellMat<MT>& A, MT* L, MT* dinv, const IluPlan& P, cudaStream_t s);
template <typename MT>
void launch_ilu_apply(const SellMat<MT>& LU, const MT* dinv, const IluPlan& P, const double* b, double* x,
                      cudaStream_t s);

int reduce_blocks(int n);
void launch_dot(int n, const double* a, const double* b, double* partial, cudaStream_t s);
void launch_finalize_sum(const double* partial, int nb, double* out, int take_sqrt, cudaStream_t s);
void launch_multidot(int n, int nv, const double* V, size_t ldv, const double* w, double* partial,
                     const int* active, cudaStream_t s);
void launch_finalize_multi(const double* partial, int nb, int nv, double* out, const int* active,
                           cudaStream_t s);

}  // namespace rdst
