// amg.cuh -- device kernels of the block AMG preconditioner: Galerkin coarse
// blocks gathered from the finer level's storage (the step's SELL matrix,
// or a coarser level's block CSR) in a fixed order, block-diagonal
// inverses, damped block-Jacobi sweeps, restriction (sum over an
// aggregate) and piecewise-constant prolongation.  The coarsening plan is
// built on the host (rdst_amg.h); coarse levels are FP64 block CSR.  Every
// kernel of the V-cycle returns at once when *active is 0 (a GMRES cycle
// that has already broken down).
#pragma once

#include "linalg.cuh"

namespace rdst {

// coarse level blocks from the step's matrix: val[25 s + e] = sum over the
// gathered SELL slots, one thread per (slot, entry)
template <typename MT>
__global__ void k_amg_gather_sell(SellMat<MT> A, const int* __restrict__ gstart, const int* __restrict__ gsrc,
                                  double* __restrict__ val, int nnz) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nnz * 25) return;
    const int s = (int)(t / 25), e = (int)(t - 25L * (t / 25));
    double a = 0.0;
    for (int q = gstart[s]; q < gstart[s + 1]; ++q) a += ld(A.val + flat_e(gsrc[q], e));
    val[t] = a;
}

// coarse level blocks from the next finer coarse level's block CSR
__global__ void k_amg_gather_csr(const double* __restrict__ fval, const int* __restrict__ gstart,
                                 const int* __restrict__ gsrc, double* __restrict__ val, int nnz) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nnz * 25) return;
    const int s = (int)(t / 25), e = (int)(t - 25L * (t / 25));
    double a = 0.0;
    for (int q = gstart[s]; q < gstart[s + 1]; ++q) a += fval[25L * gsrc[q] + e];
    val[t] = a;
}

// dinv[25 i + e] = inv(diagonal block of row i)
__global__ void k_amg_dinv(int n, const int* __restrict__ dslot, const double* __restrict__ val,
                           double* __restrict__ dinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double D[25], X[25];
    const double* v = val + 25L * dslot[i];
#pragma unroll
    for (int e = 0; e < 25; ++e) D[e] = v[e];
    inv5(D, X);
#pragma unroll
    for (int e = 0; e < 25; ++e) dinv[25L * i + e] = X[e];
}

// r = b - A x on a block CSR level, one row per thread
__global__ void k_amg_resid(int n, const int* __restrict__ start, const int* __restrict__ col,
                            const double* __restrict__ val, const double* __restrict__ x,
                            const double* __restrict__ b, double* __restrict__ r, const int* __restrict__ active) {
    if (active && !*active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double y[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) y[k] = b[5L * i + k];
    for (int q = start[i]; q < start[i + 1]; ++q) {
        const double* a = val + 25L * q;
        const double* xj = x + 5L * col[q];
        double xv[5];
#pragma unroll
        for (int j = 0; j < 5; ++j) xv[j] = xj[j];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 5; ++j) s += a[5 * k + j] * xv[j];
            y[k] -= s;
        }
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) r[5L * i + k] = y[k];
}

// x += omega D^-1 r (zero: x = omega D^-1 r) on a block CSR level
__global__ void k_amg_jacobi(int n, const double* __restrict__ dinv, const double* __restrict__ r,
                             double* __restrict__ x, double omega, int zero, const int* __restrict__ active) {
    if (active && !*active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double rv[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) rv[j] = r[5L * i + j];
    const double* d = dinv + 25L * i;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 5; ++j) s += d[5 * k + j] * rv[j];
        x[5L * i + k] = zero ? omega * s : x[5L * i + k] + omega * s;
    }
}

// the same on the step's matrix level (pivot inverses in the sliced store)
template <typename MT>
__global__ void k_amg_jacobi0(int N, const MT* __restrict__ dinv, const double* __restrict__ r, double* __restrict__ x,
                              double omega, int zero, const int* __restrict__ active) {
    if (active && !*active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double rv[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) rv[j] = r[5L * i + j];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 5; ++j) s += ld(&dinv[flat_e(i, 5 * k + j)]) * rv[j];
        x[5L * i + k] = zero ? omega * s : x[5L * i + k] + omega * s;
    }
}

// bc[I] = sum of r over the members of aggregate I (ascending)
__global__ void k_amg_restrict(int n, const int* __restrict__ mstart, const int* __restrict__ mem,
                               const double* __restrict__ r, double* __restrict__ bc, const int* __restrict__ active) {
    if (active && !*active) return;
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n) return;
    double a[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int q = mstart[I]; q < mstart[I + 1]; ++q) {
        const double* ri = r + 5L * mem[q];
#pragma unroll
        for (int k = 0; k < 5; ++k) a[k] += ri[k];
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) bc[5L * I + k] = a[k];
}

// x[i] += xc[agg[i]]
__global__ void k_amg_prolong(int n, const int* __restrict__ agg, const double* __restrict__ xc,
                              double* __restrict__ x, const int* __restrict__ active) {
    if (active && !*active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* c = xc + 5L * agg[i];
#pragma unroll
    for (int k = 0; k < 5; ++k) x[5L * i + k] += c[k];
}

__global__ void k_amg_zero(long n, double* __restrict__ x, const int* __restrict__ active) {
    if (active && !*active) return;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = 0.0;
}

}  // namespace rdst
