// rdst_internal.h -- device data layout of the B200
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
//                boundary state bs[NB][16] (rho, rhoU xyz, rhoE, p, T, phi,
//                valueFractions of p, U, T, pad, U_b xyz, pad)
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

constexpr int QW = 8;     // recon record stride (7 recon fields + muEff)
constexpr int GW = 24;    // gradient record stride (21 used)
constexpr int PW = 8;     // prim record stride
constexpr int BW = 16;    // boundary state stride (rho, rhoU, rhoE, p, T, phi, f_p, f_U, f_T, -, phi_prev, U_b xyz, mach_prev)
constexpr int SELL_C = 32;

struct DevPatch {
    int type, bc_p, bc_U, bc_T, bc_nut;
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
    const unsigned char* rmask = nullptr;   // cells whose residual is held at zero (halo cells), or none
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
    int step_idx;              // report slot of the current step
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

// ---------------------------------------------------------------- helpers
template <typename T> __device__ __forceinline__ double ld(const T* p) { return (double)(*p); }
template <> __device__ __forceinline__ double ld<__nv_bfloat16>(const __nv_bfloat16* p) { return (double)__bfloat162float(*p); }
template <typename T> __device__ __forceinline__ void st(T* p, double v) { *p = (T)v; }
template <> __device__ __forceinline__ void st<__nv_bfloat16>(__nv_bfloat16* p, double v) { *p = __float2bfloat16_rn((float)v); }
// register value -> double, and the storage type's zero
__device__ __forceinline__ double tod(double v) { return v; }
__device__ __forceinline__ double tod(float v) { return (double)v; }
__device__ __forceinline__ double tod(__nv_bfloat16 v) { return (double)__bfloat162float(v); }
template <typename T> __device__ __forceinline__ T mt_zero() { return T(0); }
// storage type <-> the compute type of the block factorisations (FP64
// storage: double; FP32 and BF16 storage: float), without a detour
// through double
__device__ __forceinline__ double ct_ld(const double* p) { return *p; }
__device__ __forceinline__ float ct_ld(const float* p) { return *p; }
__device__ __forceinline__ float ct_ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ void ct_st(double* p, double v) { *p = v; }
__device__ __forceinline__ void ct_st(float* p, float v) { *p = v; }
__device__ __forceinline__ void ct_st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 mt_zero<__nv_bfloat16>() { return __float2bfloat16_rn(0.0f); }

}  // namespace rdst
