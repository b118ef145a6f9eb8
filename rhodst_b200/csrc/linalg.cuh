// linalg.cuh -- block Krylov kernels of the fully-coupled step: SELL-32
// block SpMV, block-Jacobi and subdomain ILU(0) preconditioners, and the
// vector/reduction pieces of block GMRES (CGS2 orthogonalisation, Givens
// least squares on the device) and BiCGStab.  Matrix storage MT may be
// double, float or bf16; vectors, dot products, Hessenberg and norms are FP64.
#pragma once

#include <climits>

#include "kernels.cuh"

namespace rdst {

// entry e of 5x5 block `flat` in a slice-interleaved store: 32 blocks per
// 800-entry chunk, entries interleaved by lane (SELL slots, ILU factors,
// block-Jacobi / pivot inverses with flat = row)
__device__ __forceinline__ size_t flat_e(int flat, int e) {
    return (size_t)(flat >> 5) * (32 * 25) + (size_t)e * 32 + (flat & 31);
}

// compute type of the block factorisations for storage type MT: FP64
// storage in double, FP32 and BF16 storage in float
template <typename MT> struct IluCT { using T = float; };
template <> struct IluCT<double> { using T = double; };

// inverse of a 5x5 block (Gauss-Jordan, partial pivoting: the first row
// with the largest |a[r][c]| below the diagonal), fully unrolled so that the
// row swaps are selects on registers, not indexed local memory
template <typename T>
__device__ __forceinline__ void inv5(const T A[25], T X[25]) {
    T a[5][10];
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
        for (int j = 0; j < 5; ++j) { a[i][j] = A[5 * i + j]; a[i][j + 5] = (i == j) ? T(1) : T(0); }
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        int p = c;
        T best = fabs(a[c][c]);
#pragma unroll
        for (int r = c + 1; r < 5; ++r) {
            const T v = fabs(a[r][c]);
            if (v > best) { best = v; p = r; }
        }
#pragma unroll
        for (int r = c + 1; r < 5; ++r) {
            const bool sw = r == p;
#pragma unroll
            for (int j = 0; j < 10; ++j) {
                const T t = a[r][j], u = a[c][j];
                a[r][j] = sw ? u : t;
                a[c][j] = sw ? t : u;
            }
        }
        const T piv = T(1) / a[c][c];
#pragma unroll
        for (int j = 0; j < 10; ++j) a[c][j] *= piv;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            if (r == c) continue;
            const T f = a[r][c];
            if (f != T(0)) {
#pragma unroll
                for (int j = 0; j < 10; ++j) a[r][j] -= f * a[c][j];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
        for (int j = 0; j < 5; ++j) X[5 * i + j] = a[i][j + 5];
}

// y = A x  (or y = b - A x when b != nullptr); one row per thread; x in
// FP64 or (a Krylov basis vector) FP32, products and y in FP64
template <typename MT, typename XT = double>
__global__ void __launch_bounds__(256) k_spmv(SellMat<MT> A, const XT* __restrict__ x, double* __restrict__ y,
                                              const double* __restrict__ b, const int* __restrict__ active) {
    if (active && !*active) return;
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.N) return;
    const int s = r >> 5, lane = r & 31;
    const int base = A.slice_off[s], width = A.slice_w[s];
    double acc[5] = {0, 0, 0, 0, 0};
    for (int k = 0; k < width; ++k) {
        size_t slot = (size_t)(base + k);
        int c = A.col[slot * 32 + lane];
        if (c < 0) continue;
        const XT* xc = x + 5 * c;
        double xv[5] = {tod(xc[0]), tod(xc[1]), tod(xc[2]), tod(xc[3]), tod(xc[4])};
        const MT* v = A.val + slot * (32 * 25) + lane;
#pragma unroll
        for (int i = 0; i < 5; ++i)
#pragma unroll
            for (int j = 0; j < 5; ++j) acc[i] += ld(v + (5 * i + j) * 32) * xv[j];
    }
    double* yr = y + 5 * r;
    if (b) {
#pragma unroll
        for (int i = 0; i < 5; ++i) yr[i] = b[5 * r + i] - acc[i];
    } else {
#pragma unroll
        for (int i = 0; i < 5; ++i) yr[i] = acc[i];
    }
}

// y = A xbar for a constant 5-vector xbar (normFactor reference field)
template <typename MT>
__global__ void k_spmv_const(SellMat<MT> A, const double* __restrict__ xbar, double* __restrict__ y) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.N) return;
    const int s = r >> 5, lane = r & 31;
    const int base = A.slice_off[s], width = A.slice_w[s];
    double acc[5] = {0, 0, 0, 0, 0};
    double xv[5] = {xbar[0], xbar[1], xbar[2], xbar[3], xbar[4]};
    for (int k = 0; k < width; ++k) {
        size_t slot = (size_t)(base + k);
        if (A.col[slot * 32 + lane] < 0) continue;
        const MT* v = A.val + slot * (32 * 25) + lane;
        for (int i = 0; i < 5; ++i)
            for (int j = 0; j < 5; ++j) acc[i] += ld(v + (5 * i + j) * 32) * xv[j];
    }
    for (int i = 0; i < 5; ++i) y[5 * r + i] = acc[i];
}

// block-Jacobi: dinv = inv(diagonal block), entry-major [25][N]
template <typename MT>
__global__ void k_dinv(SellMat<MT> A, MT* __restrict__ dinv) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.N) return;
    const MT* v = A.val + (size_t)A.slice_off[r >> 5] * (32 * 25) + (r & 31);
    double D[25], X[25];
#pragma unroll
    for (int e = 0; e < 25; ++e) D[e] = ld(v + e * 32);
    inv5(D, X);
#pragma unroll
    for (int e = 0; e < 25; ++e) st(&dinv[flat_e(r, e)], X[e]);
}

template <typename MT>
__global__ void k_jacobi(int N, const MT* __restrict__ dinv, const double* __restrict__ x, double* __restrict__ y,
                         const int* __restrict__ active) {
    if (active && !*active) return;
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    double xv[5] = {x[5 * r], x[5 * r + 1], x[5 * r + 2], x[5 * r + 3], x[5 * r + 4]};
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        double a = 0;
#pragma unroll
        for (int j = 0; j < 5; ++j) a += ld(&dinv[flat_e(r, 5 * i + j)]) * xv[j];
        y[5 * r + i] = a;
    }
}

// held cells' rows of the block matrix -> identity (their update is zero;
// the right-hand side of those rows is zero through the residual mask)
template <typename MT>
__global__ void k_hold_rows(SellMat<MT> A, const unsigned char* __restrict__ mask) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.N || !mask[r]) return;
    const int sl = r >> 5, w = A.slice_w[sl];
    for (int k = 0; k < w; ++k) {
        const int fid = (A.slice_off[sl] + k) * 32 + (r & 31);
#pragma unroll
        for (int e = 0; e < 25; ++e) st(A.val + flat_e(fid, e), (k == 0 && e % 6 == 0) ? 1.0 : 0.0);
    }
}

// y += x (skipped when *active is 0)
__global__ void k_vadd(long n, const double* __restrict__ x, double* __restrict__ y, const int* __restrict__ active) {
    if (active && !*active) return;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
}

template <typename MT>
__global__ void k_copy_identity(int n, const double* __restrict__ x, double* __restrict__ y, const int* __restrict__ active) {
    if (active && !*active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = x[i];
}

// ---------------------------------------------------------------- ILU(0)
// One CTA per subdomain.  Rows of a subdomain are contiguous and sorted by
// wavefront level, so each level is a contiguous row range processed in
// parallel with a CTA barrier between levels (exact ILU(0) within the
// subdomain, block-Jacobi between subdomains).  The factors are stored in
// a fixed-width sliced layout of their own: factor slot s (L_q: s = q < ml,
// U_q: s = ml + q) of row r has id fid = ((r/32)*(ml+mu) + s)*32 + r%32 and
// its entries at flat_e(fid, e); the Jacobian keeps its SELL layout.
struct IluDev {
    int n_parts;
    const int* part_lvl0;   // [n_parts+1] level index range of each part
    const int* lvl_off;     // [n_levels+1] row range of each level
    const int* nlu;         // [N] nl | nu << 8
    const int* low_start;   // [N+1] prefix of nl (first triple range of the row)
    const int* tr_start;    // [n_low+1]
    const int* tr_kj;       // factor id of U_kj
    const int* tr_rj;       // factor id of A_rj (-1: diagonal)
    int ml, mu;             // factor slots per row
    int mu_use;             // U slots the backward sweep applies (0: (D + L)^-1 of Gauss-Seidel)
    const int* lu_col;      // [fid] column of each factor slot (-1: empty)
    const int* lu_src;      // [fid] SELL flat slot of the same block in A
    // task records of the bulk apply (null: not kept).  Each sweep's tasks
    // (24 rows of one level, in the order the sweep takes them) are laid
    // out one after the other in rec_f (forward) / rec_b (backward): a
    // 96-byte header of 24 words (byte offset of the row's record from the
    // task start | slot count << 24), then the row records: the columns of
    // the row's L (U) slots, padded to 16 bytes, the blocks (entry 5i+j),
    // and backward the pivot inverse, each record padded to 16 bytes.
    // task_f/task_b: (offset in 16-byte units, bytes) per task; part_tf /
    // part_tb: first task of each part.  The headers and columns are set
    // once; k_ilu_pack writes the blocks at val_f/val_b (16-byte units) of
    // every row after each factorisation.
    unsigned char* rec_f;
    unsigned char* rec_b;
    const uint2* task_f;
    const uint2* task_b;
    const int* part_tf;
    const int* part_tb;
    const unsigned* val_f;
    const unsigned* val_b;
    // the direct factorisation's addressing (null: gather + factor
    // instead).  Per update triple (tr_start ranges):
    // fr_trk: where U_kj is read, the flat SELL slot of A_kj (>= 0), factor
    // id fid of the sliced store as -fid - 1 (row k takes updates of its
    // own), or INT_MIN (a fill block of a row without updates: zero);
    // fr_trt: -1 the diagonal, else the slot of row r that takes it.
    // fr_desc[low_start[r] + q]: (column k of L_q, flat SELL slot of A_rk or
    // -2 for a fill, fr_trk of the slot's first triple, its fr_trt + 2 or 0
    // for none, | 1 << 20 when more triples follow).
    // nlu bit 16: the row updates one of its own off-diagonal slots.
    const int* fr_trk;
    const int* fr_trt;
    const int4* fr_desc;
};

__device__ __forceinline__ int lu_fid(int r, int s, int ms) { return ((r >> 5) * ms + s) * 32 + (r & 31); }

constexpr int ILU_TPB = 128;

// same-subdomain blocks of A -> factor storage (fully parallel, before the
// level-scheduled factorisation); fill slots outside the matrix pattern
// (lu_src -2) restart from zero, empty slots (-1) stay zero
template <typename MT>
__global__ void k_ilu_gather(SellMat<MT> A, MT* __restrict__ lu, const int* __restrict__ lu_src, int n_fid) {
    const int fid = blockIdx.x * blockDim.x + threadIdx.x;
    if (fid >= n_fid) return;
    const int src = lu_src[fid];
    if (src == -1) return;
    if (src < 0) {
#pragma unroll
        for (int e = 0; e < 25; ++e) lu[flat_e(fid, e)] = mt_zero<MT>();
        return;
    }
#pragma unroll
    for (int e = 0; e < 25; ++e) lu[flat_e(fid, e)] = A.val[flat_e(src, e)];
}

// Level-scheduled subdomain factorisation into the factor store: one CTA
// per subdomain, a thread per row of the current level, in the compute
// type of the storage (IluCT).
template <typename MT>
__global__ void __launch_bounds__(ILU_TPB) k_ilu_factor(SellMat<MT> A, MT* __restrict__ lu, MT* __restrict__ dinv,
                                                        IluDev P) {
    using CT = typename IluCT<MT>::T;
    const int part = blockIdx.x;
    const int ms = P.ml + P.mu;
    for (int l = P.part_lvl0[part]; l < P.part_lvl0[part + 1]; ++l) {
        for (int r = P.lvl_off[l] + threadIdx.x; r < P.lvl_off[l + 1]; r += blockDim.x) {
            const int nl = P.nlu[r] & 255;
            const MT* dv = A.val + (size_t)A.slice_off[r >> 5] * (32 * 25) + (r & 31);
            CT D[25];
#pragma unroll
            for (int e = 0; e < 25; ++e) D[e] = ct_ld(dv + e * 32);
            const int q0 = P.low_start[r];
            for (int q = 0; q < nl; ++q) {
                const int fq = lu_fid(r, q, ms);
                const int k = P.lu_col[fq];
                CT Ark[25], Dk[25], Lrk[25];
#pragma unroll
                for (int e = 0; e < 25; ++e) {
                    Ark[e] = ct_ld(lu + flat_e(fq, e));
                    Dk[e] = ct_ld(dinv + flat_e(k, e));
                }
#pragma unroll
                for (int i = 0; i < 5; ++i)
#pragma unroll
                    for (int j = 0; j < 5; ++j) {
                        CT a = 0;
#pragma unroll
                        for (int t = 0; t < 5; ++t) a += Ark[5 * i + t] * Dk[5 * t + j];
                        Lrk[5 * i + j] = a;
                    }
#pragma unroll
                for (int e = 0; e < 25; ++e) ct_st(lu + flat_e(fq, e), Lrk[e]);
                for (int t = P.tr_start[q0 + q]; t < P.tr_start[q0 + q + 1]; ++t) {
                    const int kj = P.tr_kj[t], rj = P.tr_rj[t];
                    CT U[25];
#pragma unroll
                    for (int e = 0; e < 25; ++e) U[e] = ct_ld(lu + flat_e(kj, e));
                    if (rj < 0) {
#pragma unroll
                        for (int i = 0; i < 5; ++i)
#pragma unroll
                            for (int j = 0; j < 5; ++j) {
                                CT a = 0;
#pragma unroll
                                for (int t2 = 0; t2 < 5; ++t2) a += Lrk[5 * i + t2] * U[5 * t2 + j];
                                D[5 * i + j] -= a;
                            }
                    } else {
#pragma unroll
                        for (int i = 0; i < 5; ++i)
#pragma unroll
                            for (int j = 0; j < 5; ++j) {
                                CT a = 0;
#pragma unroll
                                for (int t2 = 0; t2 < 5; ++t2) a += Lrk[5 * i + t2] * U[5 * t2 + j];
                                MT* p = lu + flat_e(rj, 5 * i + j);
                                ct_st(p, ct_ld(p) - a);
                            }
                    }
                }
            }
            CT X[25];
            inv5(D, X);
#pragma unroll
            for (int e = 0; e < 25; ++e) ct_st(dinv + flat_e(r, e), X[e]);
        }
        __syncthreads();
    }
}

constexpr int ILU_APPLY_TPB = 128;
constexpr int ILU_APPLY_MINB = 4;      // resident CTAs per SM the register budget is sized for
constexpr int ILU_MAX_LV = 1023;       // level offsets staged in shared memory up to this many
constexpr int ILU_LB_MAX = 1024;       // widest level the bulk apply's level buffers hold (2 x 40 KB)

// One row task of a sweep: the factor row's columns, this lane's entries
// of each slot, its pivot-inverse row (backward sweep) and the starting
// value of y.  Tasks are loaded one ahead of use, so their global loads
// are in flight across the previous task and its barrier; only the loads
// of x (rows finished in earlier levels) stay on the level-to-level chain.
template <typename MT, int NB>
struct IluTask {
    int cq[NB];
    MT v[NB][5];
    MT di[5];
    double y0;
};

template <typename MT, int NB, bool BACK>
__device__ __forceinline__ void ilu_load_task(IluTask<MT, NB>& t, const MT* __restrict__ lu,
                                              const MT* __restrict__ dinv, const int* __restrict__ lu_col,
                                              const double* y_src, int r, bool act, int comp, int s0, int ns,
                                              int ms) {
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const bool ok = act && q < ns;
        const int fid = ok ? lu_fid(r, s0 + q, ms) : 0;
        t.cq[q] = ok ? lu_col[fid] : -1;
        // empty factor slots hold zeros: the value loads do not wait for the column
#pragma unroll
        for (int j = 0; j < 5; ++j) t.v[q][j] = ok ? lu[flat_e(fid, 5 * comp + j)] : mt_zero<MT>();
    }
    if (BACK) {
#pragma unroll
        for (int j = 0; j < 5; ++j) t.di[j] = act ? dinv[flat_e(r, 5 * comp + j)] : mt_zero<MT>();
    }
    t.y0 = act ? y_src[5 * r + comp] : 0.0;
}

// Tasks of one sweep in order: level by level (forward ascending, backward
// descending), rpp rows per task.  The cursor is uniform over the CTA.
struct IluCursor {
    int l, base;
};

// x = (LU)^-1 b on each subdomain: one CTA per part walks the part's
// wavefront levels forward (x = L^-1 b, unit diagonal) and backward
// (x = U^-1 x with the stored pivot inverses), a barrier between levels.
// Five lanes per row (one per component), six rows per warp.  PF tasks
// are loaded ahead of the one being computed (two with 4- or 2-byte
// factors, one with 8-byte ones: the register budget of four CTAs per SM).
template <typename MT, int NB>
__global__ void __launch_bounds__(ILU_APPLY_TPB, ILU_APPLY_MINB)
    k_ilu_apply(int N, const MT* __restrict__ lu, const MT* __restrict__ dinv, IluDev P,
                const double* __restrict__ b, double* x, const int* __restrict__ active) {
    constexpr int PF = sizeof(MT) < 8 ? 2 : 1;
    if (active && !*active) return;
    __shared__ int s_off[ILU_MAX_LV + 1];
    const int part = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rsub = lane / 5, comp = lane - 5 * (lane / 5);
    const bool lane_ok = lane < 30;
    const int rpp = (blockDim.x >> 5) * 6;
    const int l0 = P.part_lvl0[part], l1 = P.part_lvl0[part + 1];
    const int ml = P.ml, mu = P.mu, ms = ml + mu;
    const bool staged = l1 - l0 <= ILU_MAX_LV;
    if (staged)
        for (int i = threadIdx.x; i <= l1 - l0; i += blockDim.x) s_off[i] = P.lvl_off[l0 + i];
    __syncthreads();
    auto off = [&](int l) { return staged ? s_off[l - l0] : P.lvl_off[l]; };

#pragma unroll 1
    for (int sweep = 0; sweep < 2; ++sweep) {
        const bool back = sweep == 1;
        const int dir = back ? -1 : 1;
        const int s0 = back ? ml : 0, ns = back ? P.mu_use : ml;
        const double* ysrc = back ? x : b;
        IluCursor cur{back ? l1 - 1 : l0, 0};
        auto in_range = [&](int l) { return back ? l >= l0 : l < l1; };
        // task queue: slot 0 is computed, slots 1..PF are in flight
        IluTask<MT, NB> q[PF + 1];
        int rq[PF + 1];
        bool aq[PF + 1], eq[PF + 1], vq[PF + 1];
        auto next = [&](int d) {
            vq[d] = in_range(cur.l);
            rq[d] = 0; aq[d] = false; eq[d] = false;
            if (vq[d]) {
                const int r0 = off(cur.l), n = off(cur.l + 1) - r0;
                rq[d] = r0 + cur.base + warp * 6 + rsub;
                aq[d] = lane_ok && cur.base + warp * 6 + rsub < n;
                cur.base += rpp;
                eq[d] = cur.base >= n;
                if (eq[d]) { cur.l += dir; cur.base = 0; }
            }
            if (back) ilu_load_task<MT, NB, true>(q[d], lu, dinv, P.lu_col, ysrc, rq[d], aq[d], comp, s0, ns, ms);
            else ilu_load_task<MT, NB, false>(q[d], lu, dinv, P.lu_col, ysrc, rq[d], aq[d], comp, s0, ns, ms);
        };
#pragma unroll
        for (int d = 0; d < PF; ++d) next(d);
        while (vq[0]) {
            next(PF);
            double y = q[0].y0;
            if (aq[0]) {
#pragma unroll
                for (int k = 0; k < NB; ++k) {
                    if (q[0].cq[k] >= 0) {
                        const double* xk = x + 5 * q[0].cq[k];
#pragma unroll
                        for (int j = 0; j < 5; ++j) y -= tod(q[0].v[k][j]) * xk[j];
                    }
                }
            }
            if (back) {
                // x_r = inv(U_rr) y: gather the row's five components by
                // shuffle (all lanes take part)
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < 5; ++j) {
                    const double yj = __shfl_sync(0xffffffffu, y, (lane_ok ? 5 * rsub : 0) + j);
                    a += tod(q[0].di[j]) * yj;
                }
                y = a;
            }
            if (aq[0]) x[5 * rq[0] + comp] = y;
            if (eq[0]) __syncthreads();
#pragma unroll
            for (int d = 0; d < PF; ++d) {
                q[d] = q[d + 1]; rq[d] = rq[d + 1]; aq[d] = aq[d + 1]; eq[d] = eq[d + 1]; vq[d] = vq[d + 1];
            }
        }
    }
}

// ---- ILU apply with the factor rows of each task brought in by bulk copies
//
// Same subdomains, levels and tasks as k_ilu_apply.  What differs is how a
// task's data reaches the lanes, and the arithmetic (below): the task records
// (IluDev::rec_f / rec_b, one contiguous byte range per task) are brought
// in by a single cp.async.bulk (TMA) copy, issued by one thread, into a
// shared-memory stage whose mbarrier counts the bytes; NS stages keep
// NS - 1 tasks in flight ahead of the one being computed.  The copies run
// in the async proxy (no register of the lanes waits on them), the lanes
// read 16-byte-aligned records from shared memory, and the memory system
// sees large contiguous requests.  The starting values y0 (b forward, the
// forward result backward) come by per-lane cp.async.  With LB, the x
// values of each level also go to one of two shared-memory level buffers
// (level l to buffer l & 1, row r at r - first row of l, padded to 16
// bytes for vector loads): the dependencies
// of a row in the level the sweep took just before are read from there,
// older ones from global memory.  In breadth-first order (rdst_order.h)
// nearly all couplings join consecutive levels.
//
// A stage is refilled only after the barrier that ends the task that read
// it.  Each mbarrier wait is bounded (2 s of globaltimer): on expiry the
// CTA raises bit 2 of *flags (reported as a timeout by the host), waits,
// again bounded, for its copies in flight and returns.
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// global -> shared bulk copy completing on an mbarrier (no multicast)
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}
// true once the phase of parity `parity` has completed; false after 2 s
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
    unsigned long long t0 = 0;
    for (unsigned it = 0;; ++it) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok) return true;
        if ((it & 63) == 0) {
            const unsigned long long now = globaltimer_ns();
            if (it == 0) t0 = now;
            else if (now - t0 > 2000000000ull) return false;
        }
    }
}
__device__ __forceinline__ void cpa8(unsigned dst, const void* src, bool ok) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(ok ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Four warps a subdomain, five lanes a row (one per component), six rows a
// warp: a task is up to 24 rows of one level.  The lanes multiply in CT,
// the arithmetic of the factors' storage type: double for 8-byte factors,
// float for 4- and 2-byte ones (the reduced-precision preconditioner
// applies its FP32/BF16 factors in FP32; its input b and output x stay
// FP64 vectors).  Each factor block's product with x_k is summed first
// (the block-times-vector of the oracle's apply), then subtracted from y,
// block by block in column order.
constexpr int ILU_BULK_TPB = 128;
constexpr int ILU_BULK_RPT = (ILU_BULK_TPB / 32) * 6;   // rows per task (24)
constexpr int ILU_BULK_HDR = ILU_BULK_RPT * 4;           // task header bytes (96)

__device__ __forceinline__ double to_ct(double v, double) { return v; }
__device__ __forceinline__ float to_ct(float v, float) { return v; }
__device__ __forceinline__ float to_ct(__nv_bfloat16 v, float) { return __bfloat162float(v); }
__device__ __forceinline__ float to_ct(double v, float) { return (float)v; }
// level-buffer row: five values padded to 16 bytes (6 doubles / 8 floats)
template <typename CT> constexpr int lb_row() { return sizeof(CT) == 8 ? 6 : 8; }
__device__ __forceinline__ void lb_load(const double* p, double (&o)[5]) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a0 = q[0], a1 = q[1], a2 = q[2];
    o[0] = a0.x; o[1] = a0.y; o[2] = a1.x; o[3] = a1.y; o[4] = a2.x;
}
__device__ __forceinline__ void lb_load(const float* p, float (&o)[5]) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a0 = q[0], a1 = q[1];
    o[0] = a0.x; o[1] = a0.y; o[2] = a0.z; o[3] = a0.w; o[4] = a1.x;
}

// stages the bulk apply keeps (NS - 1 tasks in flight)
template <typename MT>
constexpr int ilu_bulk_stages() { return 3; }
constexpr int ILU_FR_MAXQ = 8;      // lower slots per row the direct factorisation takes

// factor blocks -> task records (after each factorisation): one CTA per 32
// rows.  The blocks the chunk's rows use are staged through shared memory
// (loads of the sliced stores contiguous over the rows): the L blocks of the
// factor store, the U blocks of A (of the factor store for rows whose own
// blocks take updates), the pivot inverses; then the rows' value areas are
// written as whole 16-byte chunks, the threads on consecutive chunks of
// consecutive rows.
template <typename MT>
__host__ __device__ constexpr int ilu_pack_tile() { return 25 * 33; }

template <typename MT>
__global__ void __launch_bounds__(256) k_ilu_pack(int N, SellMat<MT> A, const MT* __restrict__ lu,
                                                  const MT* __restrict__ dinv, IluDev P) {
    extern __shared__ __align__(16) unsigned char s_pack[];
    MT* tiles = reinterpret_cast<MT*>(s_pack);        // [slots][25][33]
    __shared__ int s_n[2][32], s_pre[33], s_max[2], s_upd[32];
    __shared__ int s_src[ILU_FR_MAXQ * 2][32];
    constexpr int TL = ilu_pack_tile<MT>();
    constexpr int EPC = 16 / (int)sizeof(MT);
    const int chunk = blockIdx.x, r0 = chunk * 32;
    const int ms = P.ml + P.mu;
    if (threadIdx.x < 32) {
        const int r = r0 + threadIdx.x;
        const int nlu = r < N ? P.nlu[r] : 0;
        int nl = nlu & 255, nu = P.mu_use ? (nlu >> 8) & 255 : 0;
        s_n[0][threadIdx.x] = r < N ? nl : -1;
        s_n[1][threadIdx.x] = r < N ? nu : -1;
        s_upd[threadIdx.x] = (nlu >> 16) & 1;
        for (int o = 16; o > 0; o >>= 1) {
            nl = max(nl, __shfl_xor_sync(0xffffffffu, nl, o));
            nu = max(nu, __shfl_xor_sync(0xffffffffu, nu, o));
        }
        if (threadIdx.x == 0) { s_max[0] = nl; s_max[1] = nu; }
    }
    __syncthreads();
    // sources of the U blocks: flat SELL slot of A, -1 - fid of the factor
    // store (rows whose own blocks take updates), or -2 (zero)
    for (int i = threadIdx.x; i < s_max[1] * 32; i += blockDim.x) {
        const int u = i >> 5, j = i & 31;
        const int f = (chunk * ms + P.ml + u) * 32 + j;
        const int src = r0 + j < N ? P.lu_src[f] : -2;
        s_src[u][j] = s_upd[j] ? -1 - f : (src >= 0 ? src : -2);     // -2: empty slot or fill, zero
    }
    for (int side = 0; side < 2; ++side) {
        const int nmax = s_max[side];
        const int ntile = side == 0 ? nmax : nmax + 1;     // backward: U slots, then the pivot inverses
        __syncthreads();
        for (int t = 0; t < ntile; ++t) {
            for (int i = threadIdx.x; i < 800; i += blockDim.x) {
                const int e = i >> 5, j = i & 31;
                MT v;
                if (side == 0) v = lu[(size_t)(chunk * ms + t) * 800 + i];
                else if (t == nmax) v = dinv[(size_t)chunk * 800 + i];
                else {
                    const int src = s_src[t][j];
                    v = src >= 0 ? A.val[flat_e(src, e)] : (src == -2 ? mt_zero<MT>() : lu[flat_e(-1 - src, e)]);
                }
                tiles[t * TL + e * 33 + j] = v;
            }
        }
        // chunks per row, prefix
        if (threadIdx.x < 32) {
            const int n = s_n[side][threadIdx.x];
            const int nel = n < 0 ? 0 : 25 * (side == 0 ? n : n + 1);
            int c = (nel + EPC - 1) / EPC, x = c;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if ((int)threadIdx.x >= o) x += y;
            }
            s_pre[threadIdx.x + 1] = x;
            if (threadIdx.x == 0) s_pre[0] = 0;
        }
        __syncthreads();
        const int total = s_pre[32];
        for (int g = threadIdx.x; g < total; g += blockDim.x) {
            int j = 0;
#pragma unroll
            for (int st = 16; st > 0; st >>= 1)
                if (s_pre[j + st] <= g) j += st;
            const int ch = g - s_pre[j];
            const int n = s_n[side][j];
            const int nel = 25 * (side == 0 ? n : n + 1);
            alignas(16) MT v[EPC];
#pragma unroll
            for (int k = 0; k < EPC; ++k) {
                const int e = ch * EPC + k;
                const int q = e / 25, ee = e - 25 * q;
                const int t = (side == 1 && q == n) ? nmax : q;
                v[k] = e < nel ? tiles[t * TL + ee * 33 + j] : mt_zero<MT>();
            }
            uint4* dst = reinterpret_cast<uint4*>(side == 0 ? P.rec_f + (size_t)P.val_f[r0 + j] * 16
                                                            : P.rec_b + (size_t)P.val_b[r0 + j] * 16);
            dst[ch] = *reinterpret_cast<const uint4*>(v);
        }
    }
}

// one IKJ update triple of row r: U_kj read from A (us >= 0), the sliced
// factor store (fid -us - 1) or zero (INT_MIN); L_rk U_kj taken from the
// diagonal (tgt < 0) or from slot tgt of the row in the factor store
template <typename MT, typename CT>
__device__ __forceinline__ void ilu_fr_update(const SellMat<MT>& A, MT* __restrict__ lu, int r, int ms,
                                              const CT (&Lrk)[25], CT (&D)[25], int us, int tgt) {
    CT U[25];
    if (us >= 0) {
#pragma unroll
        for (int e = 0; e < 25; ++e) U[e] = ct_ld(A.val + flat_e(us, e));
    } else if (us != INT_MIN) {
#pragma unroll
        for (int e = 0; e < 25; ++e) U[e] = ct_ld(lu + flat_e(-us - 1, e));
    } else {
#pragma unroll
        for (int e = 0; e < 25; ++e) U[e] = CT(0);
    }
    if (tgt < 0) {
#pragma unroll
        for (int i = 0; i < 5; ++i)
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                CT a = 0;
#pragma unroll
                for (int t2 = 0; t2 < 5; ++t2) a += Lrk[5 * i + t2] * U[5 * t2 + j];
                D[5 * i + j] -= a;
            }
    } else {
        const int ft = lu_fid(r, tgt, ms);
#pragma unroll
        for (int i = 0; i < 5; ++i)
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                CT a = 0;
#pragma unroll
                for (int t2 = 0; t2 < 5; ++t2) a += Lrk[5 * i + t2] * U[5 * t2 + j];
                MT* pe = lu + flat_e(ft, 5 * i + j);
                ct_st(pe, ct_ld(pe) - a);
            }
    }
}

// The subdomain factorisations with the blocks of A read where they lie
// (no gather; the bulk apply's records are written by k_ilu_pack after it):
// one CTA (one warp) per subdomain, a thread per row of the current
// wavefront level, in the compute type of the storage (IluCT: FP32 for FP32
// and BF16 factors).  Row r forms L_rk = A_rk D_k^-1 and the IKJ updates
// from its blocks of A and, of earlier rows, the pivot inverses (dinv) and
// U blocks (A itself, or the factor store for rows whose own blocks take
// updates: those rows first copy their blocks of A there), and stores L and
// its pivot inverse in the sliced factor store, lanes side by side.  The
// addressing of each lower slot is one 16-byte descriptor (fr_desc), all
// read at the row's start.  Same operations, order and roundings as
// k_ilu_gather + k_ilu_factor.
template <typename MT>
__global__ void __launch_bounds__(32) k_ilu_factor_direct(SellMat<MT> A, MT* __restrict__ lu,
                                                          MT* __restrict__ dinv, IluDev P) {
    using CT = typename IluCT<MT>::T;
    __shared__ int s_off[ILU_MAX_LV + 1];
    const int ln = threadIdx.x;
    const int ms = P.ml + P.mu;
    const int part = blockIdx.x;
    const int l0 = P.part_lvl0[part], l1 = P.part_lvl0[part + 1];
    const bool staged = l1 - l0 <= ILU_MAX_LV;
    if (staged)
        for (int i = ln; i <= l1 - l0; i += 32) s_off[i] = P.lvl_off[l0 + i];
    __syncwarp();
    auto off = [&](int l) { return staged ? s_off[l - l0] : P.lvl_off[l]; };
    for (int l = l0; l < l1; ++l) {
        const int end = off(l + 1);
        for (int base = off(l); base < end; base += 32) {
            const int r = base + ln;
            if (r < end) {
                const int nlu = P.nlu[r];
                const int q0 = P.low_start[r];
                const int nl = nlu & 255;
                const int nu = P.mu_use ? (nlu >> 8) & 255 : 0;
                const bool upd = (nlu >> 16) & 1;
                int4 dsc[ILU_FR_MAXQ];
#pragma unroll
                for (int q = 0; q < ILU_FR_MAXQ; ++q)
                    if (q < nl) dsc[q] = P.fr_desc[q0 + q];
                const MT* dv = A.val + (size_t)A.slice_off[r >> 5] * (32 * 25) + (r & 31);
                CT D[25];
#pragma unroll
                for (int e = 0; e < 25; ++e) D[e] = ct_ld(dv + e * 32);
                // a row that updates its own blocks takes them from A into
                // the factor store first (zero where ILU(p) fills)
                if (upd) {
                    for (int sl = 0; sl < nl + nu; ++sl) {
                        const int f = lu_fid(r, sl < nl ? sl : P.ml + sl - nl, ms);
                        const int src = P.lu_src[f];
#pragma unroll
                        for (int e = 0; e < 25; ++e) lu[flat_e(f, e)] = src >= 0 ? A.val[flat_e(src, e)] : mt_zero<MT>();
                    }
                }
#pragma unroll
                for (int q = 0; q < ILU_FR_MAXQ; ++q) {
                    if (q < nl) {
                        const int k = dsc[q].x, sl = dsc[q].y, us0 = dsc[q].z, tw = dsc[q].w;
                        const int fq = lu_fid(r, q, ms);
                        CT Ark[25], Dk[25], Lrk[25];
                        if (upd) {
#pragma unroll
                            for (int e = 0; e < 25; ++e) Ark[e] = ct_ld(lu + flat_e(fq, e));
                        } else {
#pragma unroll
                            for (int e = 0; e < 25; ++e) Ark[e] = sl >= 0 ? ct_ld(A.val + flat_e(sl, e)) : CT(0);
                        }
#pragma unroll
                        for (int e = 0; e < 25; ++e) Dk[e] = ct_ld(dinv + flat_e(k, e));
#pragma unroll
                        for (int i = 0; i < 5; ++i)
#pragma unroll
                            for (int j = 0; j < 5; ++j) {
                                CT a = 0;
#pragma unroll
                                for (int t = 0; t < 5; ++t) a += Ark[5 * i + t] * Dk[5 * t + j];
                                Lrk[5 * i + j] = a;
                            }
#pragma unroll
                        for (int e = 0; e < 25; ++e) ct_st(lu + flat_e(fq, e), Lrk[e]);
                        // update triples: the first rides in the descriptor (w:
                        // its target slot + 2, 0 none; bit 20: more follow)
                        const int tfirst = (tw & 0xfffff) - 2;
                        if (tfirst >= -1) ilu_fr_update(A, lu, r, ms, Lrk, D, us0, tfirst);
                        if (tw >> 20) {
                            for (int t = P.tr_start[q0 + q] + 1; t < P.tr_start[q0 + q + 1]; ++t)
                                ilu_fr_update(A, lu, r, ms, Lrk, D, P.fr_trk[t], P.fr_trt[t]);
                        }
                    }
                }
                CT X[25];
                inv5(D, X);
#pragma unroll
                for (int e = 0; e < 25; ++e) ct_st(dinv + flat_e(r, e), X[e]);
            }
            __syncwarp();
        }
    }
}

// The apply is specialised by warp: warps 0-3 compute (five lanes a row,
// six rows a warp), a fifth warp produces.  For each task the producer
// walks the cursor, publishes the task's rows and level buffers in s_q,
// starts the bulk copy of its record into a stage and the copies of its y0
// into the y0 slot, and waits for the latter before the barrier that ends
// the task being computed; the compute warps only wait for the stage,
// multiply and store.  All 160 threads take the same barriers.
constexpr int ILU_BULK_THREADS = ILU_BULK_TPB + 32;

template <typename MT, int NS, bool LB>
__global__ void __launch_bounds__(ILU_BULK_THREADS, 6)
    k_ilu_apply_bulk(IluDev P, const double* __restrict__ b, double* x, const int* __restrict__ active,
                     int lb_rows, int stage_bytes, int off_slots, int task_slots, int* flags) {
    using CT = typename IluCT<MT>::T;
    constexpr int T = ILU_BULK_TPB;
    constexpr int RPT = ILU_BULK_RPT;
    constexpr int LR = lb_row<CT>();
    if (active && !*active) return;
    __shared__ __align__(8) unsigned long long s_bar[NS];
    __shared__ int s_abort;
    // per stage: valid, first row, rows, the level's first row, its buffer,
    // the previous level's first row and width
    __shared__ int s_q[NS][8];
    extern __shared__ __align__(128) unsigned char s_dyn[];
    unsigned char* s_stage = s_dyn;                                                   // [NS][stage_bytes]
    double* s_y0 = reinterpret_cast<double*>(s_dyn + (size_t)NS * stage_bytes);       // [NS][T]
    CT* s_lvx = reinterpret_cast<CT*>(s_y0 + NS * T);                                 // [2][lb_rows][LR]
    uint2* s_task = reinterpret_cast<uint2*>(s_lvx + 2 * LR * lb_rows);               // [task_slots] f then b
    int* s_off = reinterpret_cast<int*>(s_task + task_slots);                         // [off_slots]
    const int part = blockIdx.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = warp == T / 32;
    const int rsub = lane / 5, comp = lane - 5 * (lane / 5);
    const bool lane_ok = !producer && lane < 30;
    const int i_row = warp * 6 + rsub;
    const int l0 = P.part_lvl0[part], l1 = P.part_lvl0[part + 1];
    const bool staged = l1 - l0 < off_slots;
    if (staged)
        for (int i = tid; i <= l1 - l0; i += ILU_BULK_THREADS) s_off[i] = P.lvl_off[l0 + i];
    const int tf0 = P.part_tf[part], ntf = P.part_tf[part + 1] - tf0;
    const int tb0 = P.part_tb[part], ntb = P.part_tb[part + 1] - tb0;
    const bool tstaged = ntf + ntb <= task_slots;
    if (tstaged) {
        for (int i = tid; i < ntf; i += ILU_BULK_THREADS) s_task[i] = P.task_f[tf0 + i];
        for (int i = tid; i < ntb; i += ILU_BULK_THREADS) s_task[ntf + i] = P.task_b[tb0 + i];
    }
    const unsigned bar0 = (unsigned)__cvta_generic_to_shared(&s_bar[0]);
    const unsigned stage0 = (unsigned)__cvta_generic_to_shared(s_stage);
    const unsigned y0s = (unsigned)__cvta_generic_to_shared(s_y0);
    if (tid == 0) {
        for (int k = 0; k < NS; ++k) mbar_init(bar0 + 8 * k, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto off = [&](int l) { return staged ? s_off[l - l0] : P.lvl_off[l]; };
    unsigned par = 0;          // compute warps: bit k, parity of stage k's next completion
    unsigned ipar = 0;         // producer: bit k, parity of the next copy issued into stage k
    unsigned lastp = 0;        // producer: bit k, parity of the last copy issued into stage k
    unsigned issued = 0;       // producer: bit k, stage k has taken a copy

#pragma unroll 1
    for (int sweep = 0; sweep < 2; ++sweep) {
        const bool back = sweep == 1;
        const int dir = back ? -1 : 1;
        const unsigned char* rec = back ? P.rec_b : P.rec_f;
        const double* ysrc = back ? x : b;
        IluCursor cur{back ? l1 - 1 : l0, 0};
        int tcount = 0;        // tasks of this sweep issued so far (producer)
        auto in_range = [&](int l) { return back ? l >= l0 : l < l1; };
        // producer: the next task into stage d (cursor, s_q, record copy,
        // y0 copies of the compute lanes: thread 32k + lane, row 6k + lane/5)
        auto prepare = [&](int d) {
            const bool v = in_range(cur.l);
            int r0q = 0, nq = 0, aq = 0, bufq = 0, paq = 0, pwq = 0;
            if (v) {
                const int r0 = off(cur.l), r1 = off(cur.l + 1), n = r1 - r0;
                r0q = r0 + cur.base;
                nq = min(RPT, n - cur.base);
                if (LB) {
                    aq = r0;
                    bufq = (cur.l & 1) * lb_rows * LR;
                    const int lp = cur.l - dir;          // the level taken just before
                    if (in_range(lp)) { paq = off(lp); pwq = off(lp + 1) - paq; }
                }
                cur.base += RPT;
                if (cur.base >= n) { cur.l += dir; cur.base = 0; }
                if (lane == 0) {
                    const uint2 tk = tstaged ? s_task[(back ? ntf : 0) + tcount]
                                             : (back ? P.task_b[tb0 + tcount] : P.task_f[tf0 + tcount]);
                    mbar_expect_tx(bar0 + 8 * d, tk.y);
                    bulk_g2s(stage0 + (unsigned)(d * stage_bytes), rec + (size_t)tk.x * 16, tk.y, bar0 + 8 * d);
                }
                ++tcount;
                lastp = (lastp & ~(1u << d)) | (ipar & (1u << d));
                ipar ^= 1u << d;
                issued |= 1u << d;
            }
            if (lane == 0) {
                s_q[d][0] = v; s_q[d][1] = r0q; s_q[d][2] = nq; s_q[d][3] = aq;
                s_q[d][4] = bufq; s_q[d][5] = paq; s_q[d][6] = pwq;
            }
#pragma unroll
            for (int k = 0; k < T / 32; ++k) {
                const int row = 6 * k + rsub;
                const bool ok = v && lane < 30 && row < nq;
                cpa8(y0s + (unsigned)((d * T + 32 * k + lane) * 8), ysrc + (ok ? 5 * (size_t)(r0q + row) + comp : 0),
                     ok);
            }
            cpa_commit();
        };
        // compute warps: task d, after its stage has landed: y = y0 -
        // sum_k (L_rk x_k) (backward x_r = inv(U_rr) y)
        auto run = [&](int d) {
            if (!mbar_wait(bar0 + 8 * d, (par >> d) & 1u)) {
                atomicOr(flags, 4);
                s_abort = 1;
            }
            par ^= 1u << d;
            const int qr0 = s_q[d][1], qn = s_q[d][2], qa = s_q[d][3], qbuf = s_q[d][4];
            const int qpa = s_q[d][5], qpw = s_q[d][6];
            const bool act = lane_ok && i_row < qn && !s_abort;
            const int r = qr0 + i_row;
            const unsigned char* st0 = s_stage + (size_t)d * stage_bytes;
            const unsigned hdr = act ? reinterpret_cast<const unsigned*>(st0)[i_row] : 0u;
            const int cnt = (int)(hdr >> 24);
            const int* cols = reinterpret_cast<const int*>(st0 + (hdr & 0xffffffu));
            const MT* vals = reinterpret_cast<const MT*>(st0 + (hdr & 0xffffffu) + 16 * ((cnt + 3) >> 2));
            CT y = to_ct(s_y0[d * T + tid], CT());
            if (act) {
                // the first four blocks side by side (their products are
                // independent), then subtracted in column order; a block
                // past the row's count loads nothing and contributes 0
                const CT* pbuf = s_lvx + (lb_rows * LR - qbuf);   // the other level buffer
                CT part4[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    CT t = CT(0);
                    if (k < cnt) {
                        const int ck = cols[k];
                        const unsigned rel = (unsigned)(ck - qpa);
                        CT xk[5];
                        if (LB && rel < (unsigned)qpw) {
                            lb_load(pbuf + LR * rel, xk);
                        } else {
#pragma unroll
                            for (int j = 0; j < 5; ++j) xk[j] = to_ct(x[5 * ck + j], CT());
                        }
                        t = to_ct(vals[25 * k + 5 * comp], CT()) * xk[0];
#pragma unroll
                        for (int j = 1; j < 5; ++j) t += to_ct(vals[25 * k + 5 * comp + j], CT()) * xk[j];
                    }
                    part4[k] = t;
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) y -= part4[k];
                for (int k = 4; k < cnt; ++k) {
                    const int ck = cols[k];
                    const unsigned rel = (unsigned)(ck - qpa);
                    CT xk[5];
                    if (LB && rel < (unsigned)qpw) {
                        lb_load(pbuf + LR * rel, xk);
                    } else {
#pragma unroll
                        for (int j = 0; j < 5; ++j) xk[j] = to_ct(x[5 * ck + j], CT());
                    }
                    CT t = to_ct(vals[25 * k + 5 * comp], CT()) * xk[0];
#pragma unroll
                    for (int j = 1; j < 5; ++j) t += to_ct(vals[25 * k + 5 * comp + j], CT()) * xk[j];
                    y -= t;
                }
            }
            if (back) {
                CT a = CT(0);
#pragma unroll
                for (int j = 0; j < 5; ++j) {
                    const CT yj = __shfl_sync(0xffffffffu, y, (lane_ok ? 5 * rsub : 0) + j);
                    a += (act ? to_ct(vals[25 * cnt + 5 * comp + j], CT()) : CT(0)) * yj;
                }
                y = a;
            }
            if (act) {
                x[5 * (size_t)r + comp] = (double)y;
                if (LB) s_lvx[qbuf + LR * (r - qa) + comp] = y;
            }
        };
        if (producer) {
#pragma unroll
            for (int d = 0; d < NS - 1; ++d) prepare(d);
            cpa_wait<0>();
        }
        __syncthreads();
        bool go = s_q[0][0] != 0;
        while (go) {
            // stage slots rotate with compile-time indices (the body is
            // unrolled NS times), so the queue stays in registers
#pragma unroll
            for (int u = 0; u < NS; ++u) {
                if (go) {
                    if (producer) {
                        prepare((u + NS - 1) % NS);
                        cpa_wait<0>();
                    } else {
                        run(u);
                    }
                    __syncthreads();
                    go = s_q[(u + 1) % NS][0] != 0 && !s_abort;
                }
            }
        }
        if (s_abort) {
            // copies still in flight land before the CTA's shared memory goes
            if (producer && lane == 0)
                for (int d = 0; d < NS; ++d)
                    if ((issued >> d) & 1u) mbar_wait(bar0 + 8 * d, (lastp >> d) & 1u);
            return;
        }
        // the next sweep prepares its first tasks into stages 0..NS-2 again:
        // the rotation restarts, parities carry on
        __syncthreads();
    }
}

// ---------------------------------------------------------------- vectors
// deterministic two-stage reductions: fixed grid -> partials -> one block
constexpr int RED_TPB = 256;
inline int red_blocks(long n) {
    long b = (n + RED_TPB * 4 - 1) / (RED_TPB * 4);
    if (b < 1) b = 1;
    if (b > 592) b = 592;           // 4 x 148 SMs
    return (int)b;
}

// partial[blk * nv + j] = sum_i V_j[i] * w[i], j < nv (nv <= 8 per launch)
__global__ void __launch_bounds__(RED_TPB) k_multidot(long n, int nv, const double* __restrict__ V, long ldv,
                                                      const double* __restrict__ w, double* __restrict__ partial,
                                                      int pstride, const int* __restrict__ active) {
    if (active && !*active) return;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double wi = w[i];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j < nv) acc[j] += V[j * ldv + i] * wi;
    }
    for (int j = 0; j < nv; ++j) {
        double v = block_sum(acc[j]);
        if (threadIdx.x == 0) partial[(long)blockIdx.x * pstride + j] = v;
    }
}

// Deterministic block reduction of NV per-thread values: warp shuffles,
// then one fixed-order sum over the warps; result -> partial[blk*pstride+j].
template <int NV>
__device__ __forceinline__ void block_multi_sum(double (&acc)[NV], int nv, double* __restrict__ partial, int pstride) {
    __shared__ double sh[RED_TPB / 32][NV];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        if (j < nv) {
            double v = warp_sum(acc[j]);
            if (lane == 0) sh[wid][j] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double v = 0;
        for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) v += sh[w2][threadIdx.x];
        partial[(long)blockIdx.x * pstride + threadIdx.x] = v;
    }
}

// partial[blk][j] = sum_i V_j[i] w[i] for j < nv <= NV (one pass over w)
// Four consecutive entries of a vector as doubles (16-byte loads; the
// caller guarantees 4-entry alignment of p), or fewer at the vector's end.
__device__ __forceinline__ void load4(const double* __restrict__ p, double (&o)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void load4(const float* __restrict__ p, double (&o)[4]) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
}
template <typename T>
__device__ __forceinline__ void load4_tail(const T* __restrict__ p, long rem, double (&o)[4]) {
#pragma unroll
    for (int e = 0; e < 4; ++e) o[e] = e < rem ? tod(p[e]) : 0.0;
}
template <typename T>
__device__ __forceinline__ void load4_any(const T* __restrict__ p, long i0, long n, double (&o)[4]) {
    if (i0 + 4 <= n) load4(p + i0, o);
    else load4_tail(p + i0, n - i0, o);
}

// partial[blk * pstride + j] = sum_i V_j[i] w[i], j < nv: four entries per
// thread and 16-byte loads; V (fp64 or fp32) has a row stride ldv that is
// a multiple of 4 entries.  Full chunks take a branch-free path so that
// the loads of all nv vectors are in flight together.
template <int NV, typename VT = double>
__global__ void __launch_bounds__(RED_TPB, 2) k_vmultidot(long n, int nv, const VT* __restrict__ V, long ldv,
                                                       const double* __restrict__ w, double* __restrict__ partial,
                                                       int pstride, const int* __restrict__ active) {
    if (active && !*active) return;
    double acc[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] = 0.0;
    const long nc = (n + 3) / 4, nfull = n / 4;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (long)gridDim.x * blockDim.x) {
        const long i0 = 4 * c;
        double wv[4];
        if (c < nfull) {
            load4(w + i0, wv);
#pragma unroll
            for (int j = 0; j < NV; ++j)
                if (j < nv) {
                    double v[4];
                    load4(V + j * ldv + i0, v);
                    acc[j] += v[0] * wv[0] + v[1] * wv[1] + v[2] * wv[2] + v[3] * wv[3];
                }
        } else {
            load4_tail(w + i0, n - i0, wv);
            for (int j = 0; j < nv && j < NV; ++j) {
                double v[4];
                load4_tail(V + j * ldv + i0, n - i0, v);
                acc[j] += v[0] * wv[0] + v[1] * wv[1] + v[2] * wv[2] + v[3] * wv[3];
            }
        }
    }
    block_multi_sum<NV>(acc, nv, partial, pstride);
}

// w -= sum_j coef[j] V_j (j < nv), then in the same pass either the dots
// V_j . w_new (mode 0: the second CGS2 pass) or w_new . w_new (mode 1);
// four entries per thread as in k_vmultidot
template <int NV, typename VT = double>
__global__ void __launch_bounds__(RED_TPB, 2) k_maxpy_dot(long n, int nv, const VT* __restrict__ V, long ldv,
                                                       const double* __restrict__ coef, double* __restrict__ w,
                                                       double* __restrict__ partial, int pstride, int mode,
                                                       const int* __restrict__ active) {
    if (active && !*active) return;
    __shared__ double cs[NV];
    if (threadIdx.x < NV) cs[threadIdx.x] = threadIdx.x < nv ? coef[threadIdx.x] : 0.0;
    __syncthreads();
    double acc[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] = 0.0;
    const long nc = (n + 3) / 4, nfull = n / 4;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (long)gridDim.x * blockDim.x) {
        const long i0 = 4 * c;
        double a[4];
        if (c < nfull) {
            load4(w + i0, a);
#pragma unroll
            for (int j = 0; j < NV; ++j)
                if (j < nv) {
                    double v[4];
                    load4(V + j * ldv + i0, v);
#pragma unroll
                    for (int e = 0; e < 4; ++e) a[e] -= cs[j] * v[e];
                }
            reinterpret_cast<double2*>(w + i0)[0] = make_double2(a[0], a[1]);
            reinterpret_cast<double2*>(w + i0)[1] = make_double2(a[2], a[3]);
            if (mode == 0) {
                // second read of V_j: the lines were just fetched (L1 hit)
#pragma unroll
                for (int j = 0; j < NV; ++j)
                    if (j < nv) {
                        double v[4];
                        load4(V + j * ldv + i0, v);
                        acc[j] += v[0] * a[0] + v[1] * a[1] + v[2] * a[2] + v[3] * a[3];
                    }
            }
        } else {
            load4_tail(w + i0, n - i0, a);
            for (int j = 0; j < nv && j < NV; ++j) {
                double v[4];
                load4_tail(V + j * ldv + i0, n - i0, v);
                for (int e = 0; e < 4; ++e) a[e] -= cs[j] * v[e];
            }
            for (int e = 0; e < 4; ++e)
                if (i0 + e < n) w[i0 + e] = a[e];
            if (mode == 0) {
                for (int j = 0; j < nv && j < NV; ++j) {
                    double v[4];
                    load4_tail(V + j * ldv + i0, n - i0, v);
                    acc[j] += v[0] * a[0] + v[1] * a[1] + v[2] * a[2] + v[3] * a[3];
                }
            }
        }
        if (mode != 0) acc[0] += a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
    }
    block_multi_sum<NV>(acc, mode == 0 ? nv : 1, partial, pstride);
}

// out[j] = sum_b partial[b * pstride + j] (fixed order); optional sqrt
__global__ void k_finalize(const double* __restrict__ partial, int nb, int nv, int pstride, double* __restrict__ out,
                           int take_sqrt, const int* __restrict__ active) {
    if (active && !*active) return;
    int j = blockIdx.x;
    if (j >= nv) return;
    double s = 0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(long)b * pstride + j];
    s = block_sum(s);
    if (threadIdx.x == 0) out[j] = take_sqrt ? sqrt(s) : s;
}

// w -= sum_j coef[j] V_j (j < nv); coef on the device
template <typename VT = double>
__global__ void k_maxpy(long n, int nv, const VT* __restrict__ V, long ldv, const double* __restrict__ coef,
                        double* __restrict__ w, double sign, const int* __restrict__ active) {
    if (active && !*active) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = w[i];
    for (int j = 0; j < nv; ++j) a -= sign * coef[j] * tod(V[j * ldv + i]);
    w[i] = a;
}

// x /= *s
__global__ void k_scale_inv(long n, double* __restrict__ x, const double* __restrict__ s, const int* __restrict__ active) {
    if (active && !*active) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = x[i] / *s;
}

// v = w / *s stored as a (FP32) basis vector
template <typename VT>
__global__ void k_scale_store(long n, const double* __restrict__ w, VT* __restrict__ v, const double* __restrict__ s,
                              const int* __restrict__ active) {
    if (active && !*active) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (VT)(w[i] / *s);
}

// per-component sum |r_c| and the foam normFactor pieces
__global__ void __launch_bounds__(RED_TPB) k_abs5(int N, const double* __restrict__ r, double* __restrict__ partial) {
    double a[5] = {0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int c = 0; c < 5; ++c) a[c] += fabs(r[5 * i + c]);
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        double v = block_sum(a[c]);
        if (threadIdx.x == 0) partial[blockIdx.x * 5 + c] = v;
    }
}

// sum over cells of the 5 components (for the average x)
__global__ void __launch_bounds__(RED_TPB) k_sum5(int N, const double* __restrict__ x, double* __restrict__ partial) {
    double a[5] = {0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int c = 0; c < 5; ++c) a[c] += x[5 * i + c];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        double v = block_sum(a[c]);
        if (threadIdx.x == 0) partial[blockIdx.x * 5 + c] = v;
    }
}

// sum_i |Ax_i - pA_i| + |Ax_i + s_i - pA_i| (normFactor, x = W, b = A W + s)
__global__ void __launch_bounds__(RED_TPB) k_normfactor(int N, const double* __restrict__ Ax, const double* __restrict__ s,
                                                        const double* __restrict__ pA, int dependentW,
                                                        double* __restrict__ partial) {
    double a = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        double s1 = 0, s2 = 0;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            double ax = dependentW ? Ax[5 * i + c] : 0.0;
            double pa = dependentW ? pA[5 * i + c] : 0.0;
            double b = ax + s[5 * i + c];
            s1 += (ax - pa) * (ax - pa);
            s2 += (b - pa) * (b - pa);
        }
        a += sqrt(s1) + sqrt(s2);
    }
    a = block_sum(a);
    if (threadIdx.x == 0) partial[blockIdx.x] = a;
}

__global__ void k_nf_finalize(const double* __restrict__ partial, int nb, Scalars* sc) {
    double s = 0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[b];
    s = block_sum(s);
    if (threadIdx.x == 0) sc->nf = s + 1.0e-20;
}

__global__ void k_mean5_finalize(const double* __restrict__ partial, int nb, int N, double* __restrict__ xbar) {
    for (int c = 0; c < 5; ++c) {
        double s = 0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[b * 5 + c];
        s = block_sum(s);
        if (threadIdx.x == 0) xbar[c] = s / N;
    }
}

// linear residual per component / normFactor -> initial or final
__global__ void k_linres_finalize(const double* __restrict__ partial, int nb, Scalars* sc, int initial) {
    for (int c = 0; c < 5; ++c) {
        double s = 0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[b * 5 + c];
        s = block_sum(s);
        if (threadIdx.x == 0) {
            const double v = s / sc->nf;
            if (initial) { sc->lin_initial[c] = v; sc->lin_final[c] = v; }
            else sc->lin_final[c] = v;
        }
    }
}

// BlockSolverPerformance check: converged if every component below the
// tolerance, or below relTol x initial, or maxIter reached (after minIter).
// A solve that stops on maxIter alone raises bit 3 of the step flags (the
// solver performance's converged() is false); one that stops on the
// tolerances clears it.
__global__ void k_check(Scalars* sc, double tol, double relTol, int minIter, int maxIter, int count) {
    if (threadIdx.x != 0) return;
    if (count) sc->lin_iterations += 1;
    int it = sc->lin_iterations;
    bool t = true, r = relTol > 0;
    for (int c = 0; c < 5; ++c) {
        if (!(sc->lin_final[c] < tol)) t = false;
        if (!(sc->lin_final[c] < relTol * sc->lin_initial[c])) r = false;
    }
    sc->converged = (it >= minIter) && (t || r || it >= maxIter);
    if (sc->converged) sc->flags = (t || r) ? (sc->flags & ~8) : (sc->flags | 8);
}

// ---------------------------------------------------------------- GMRES
__global__ void k_gm_start(Scalars* sc) {
    if (threadIdx.x != 0) return;
    for (int i = 0; i < 65; ++i) sc->bh[i] = 0.0;
    for (int i = 0; i < 64 * 65; ++i) sc->H[i] = 0.0;
    sc->bh[0] = sc->beta;
    sc->gm_active = (sc->beta != 0.0);
    sc->gm_used = 0;
}

// H[:,i] = h1 + h2 (CGS2), Givens rotations (foam givensRotation), bh
__global__ void k_gm_givens(Scalars* sc, int i, int m) {
    if (threadIdx.x != 0 || !sc->gm_active) return;
    double* H = sc->H;
    for (int j = 0; j <= i; ++j) H[j * m + i] = sc->hcol[0][j] + sc->hcol[1][j];
    double beta = sc->beta;
    for (int j = 0; j < i; ++j) {
        double Hji = H[j * m + i];
        H[j * m + i] = sc->cs[j] * Hji - sc->sn[j] * H[(j + 1) * m + i];
        H[(j + 1) * m + i] = sc->sn[j] * Hji + sc->cs[j] * H[(j + 1) * m + i];
    }
    double hh = H[i * m + i], c, s;
    if (beta == 0.0) { c = 1; s = 0; }
    else if (fabs(beta) > fabs(hh)) { double tau = -hh / beta; s = 1.0 / sqrt(1.0 + tau * tau); c = s * tau; }
    else { double tau = -beta / hh; c = 1.0 / sqrt(1.0 + tau * tau); s = c * tau; }
    sc->cs[i] = c;
    sc->sn[i] = s;
    double bhi = sc->bh[i];
    sc->bh[i] = c * bhi - s * sc->bh[i + 1];
    sc->bh[i + 1] = s * bhi + c * sc->bh[i + 1];
    H[i * m + i] = c * H[i * m + i] - s * beta;
    sc->gm_used = i + 1;
    if (beta == 0.0) sc->gm_active = 0;
}

__global__ void k_gm_backsub(Scalars* sc, int m) {
    if (threadIdx.x != 0) return;
    int used = sc->gm_used;
    for (int i = used - 1; i >= 0; --i) {
        double sum = sc->bh[i];
        for (int j = i + 1; j < used; ++j) sum -= sc->H[i * m + j] * sc->yh[j];
        sc->yh[i] = sum / sc->H[i * m + i];
    }
    for (int i = used; i < m; ++i) sc->yh[i] = 0.0;
}

// ---------------------------------------------------------------- BiCGStab
// p = r + beta (p - omega v)
__global__ void k_bi_p(long n, const double* __restrict__ r, const double* __restrict__ v, double* __restrict__ p,
                       const Scalars* sc) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = r[i] + sc->bi_beta * (p[i] - sc->bi_omega * v[i]);
}
__global__ void k_bi_scal_rho(Scalars* sc) {       // rho, beta from rw.r
    if (threadIdx.x != 0) return;
    sc->bi_rhoOld = sc->bi_rho;
    sc->bi_rho = sc->hcol[0][0];
    sc->bi_beta = sc->bi_rho / sc->bi_rhoOld * (sc->bi_alpha / sc->bi_omega);
}
__global__ void k_bi_scal_alpha(Scalars* sc) {
    if (threadIdx.x != 0) return;
    sc->bi_alpha = sc->bi_rho / sc->hcol[0][0];
}
__global__ void k_bi_s(long n, const double* __restrict__ r, const double* __restrict__ v, double* __restrict__ s,
                       const Scalars* sc) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) s[i] = r[i] - sc->bi_alpha * v[i];
}
__global__ void k_bi_scal_omega(Scalars* sc) {     // omega = (t.s)/(t.t)
    if (threadIdx.x != 0) return;
    double tt = sc->hcol[0][0], ts = sc->hcol[0][1];
    sc->bi_omega = tt > 0 ? ts / tt : 0.0;
}
__global__ void k_bi_update(long n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ ph,
                            const double* __restrict__ sh, const double* __restrict__ s, const double* __restrict__ t,
                            const Scalars* sc) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] += sc->bi_alpha * ph[i] + sc->bi_omega * sh[i];
    r[i] = s[i] - sc->bi_omega * t[i];
}
__global__ void k_bi_init(Scalars* sc) {
    if (threadIdx.x != 0) return;
    sc->bi_rho = 1e300;
    sc->bi_alpha = 0.0;
    sc->bi_omega = 1e300;
}

}  // namespace rdst
