// rdst_api.cu -- host side of the B200 fully-coupled step: context set-up
// (mesh upload, subdomain partition, wavefront levels, SELL-32 block matrix
// structure, ILU(0) plan), the step driver that replaces
// Single::iterate (libraries/finiteVolume/iteration/Single/Single.C:80-104)
// and the C ABI of include/rdst.h.
#include "../../include/rdst.h"
#include "rdst_options.h"
#include "rdst_internal.h"
#include "linalg.cuh"
#include "turbulence.cuh"
#include "adjoint.cuh"
#include "amg.cuh"
#include "rdst_amg.h"
#include "rdst_order.h"

#include <algorithm>
#include <cmath>
#include <array>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <unordered_map>
#include <type_traits>
#include <vector>

#define RDST_API extern "C" __attribute__((visibility("default")))

using namespace rdst;

namespace {

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& m) : std::runtime_error(m) {}
};
// a bounded device wait gave up (a kernel raised bit 2 of the step flags)
struct TimeoutError : std::runtime_error {
    using std::runtime_error::runtime_error;
};


inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}
// kernels launched by the calling thread's current context (CKL follows
// every launch)
thread_local long* g_launch_counter = nullptr;
inline void count_launch() { if (g_launch_counter) ++*g_launch_counter; }
#define CK(x) ck((x), #x)
#define RDST_STR2(x) #x
#define RDST_STR(x) RDST_STR2(x)
// the launch's source line goes into the message
#define CKL() (count_launch(), ck(cudaGetLastError(), "kernel launch at rdst_api.cu:" RDST_STR(__LINE__)))

enum { KS_SPMV = 0, KS_PRECOND, KS_FLUX, KS_ASSEMBLE, KS_FACTOR, KS_ORTH, KS_UPDATE, KS_N };
const char* const KS_NAMES[KS_N] = {"spmv", "precond", "flux", "assemble", "factor", "orth", "update"};

template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        free_();
        n = count;
        if (count) CK(cudaMalloc((void**)&p, count * sizeof(T)));
    }
    void upload(const std::vector<T>& v, cudaStream_t s) {
        alloc(v.size());
        if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    // copy into the existing allocation: device pointers (and graphs that hold them) stay valid
    void overwrite(const std::vector<T>& v, cudaStream_t s) {
        if (v.size() != n) throw std::invalid_argument("buffer size changed");
        if (n) CK(cudaMemcpyAsync(p, v.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void zero(cudaStream_t s) { if (n) CK(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    void free_() { if (p) cudaFree(p); p = nullptr; n = 0; }
    ~DBuf() { free_(); }
};

inline int nblk(long n, int tpb) { return (int)std::max<long>(1, (n + tpb - 1) / tpb); }

// recursive coordinate bisection (deterministic: ties broken by index)
void rcb(const double* C, std::vector<int>& idx, int lo, int hi, int part0, int nparts, int32_t* out) {
    if (nparts <= 1 || hi - lo <= 1) {
        for (int i = lo; i < hi; ++i) out[idx[i]] = part0;
        return;
    }
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int i = lo; i < hi; ++i)
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], C[3 * idx[i] + k]);
            mx[k] = std::max(mx[k], C[3 * idx[i] + k]);
        }
    int ax = 0;
    for (int k = 1; k < 3; ++k) if (mx[k] - mn[k] > mx[ax] - mn[ax]) ax = k;
    int n1 = nparts / 2;
    int mid = lo + (int)((long)(hi - lo) * n1 / nparts);
    std::nth_element(idx.begin() + lo, idx.begin() + mid, idx.begin() + hi, [&](int a, int b) {
        double ca = C[3 * a + ax], cb = C[3 * b + ax];
        return ca < cb || (ca == cb && a < b);
    });
    rcb(C, idx, lo, mid, part0, n1, out);
    rcb(C, idx, mid, hi, part0 + n1, nparts - n1, out);
}

// Recursive graph bisection of the cell graph (internal faces): each set is
// ordered by breadth-first distance from a pseudo-peripheral cell (the cell
// farthest from the set's first cell; ties by position), then by cell
// index, and cut at the proportional rank; cells the search does not reach
// (another component) go last.  Subdomains cut this way are graph slabs,
// whose wavefront level chains are shorter than those of coordinate boxes
// on stretched body-fitted meshes.
struct CellGraph {
    std::vector<int> start, adj;            // CSR, neighbours ascending
    CellGraph(int N, int Fi, const int32_t* own, const int32_t* nei) : start(N + 1, 0) {
        for (int f = 0; f < Fi; ++f) { ++start[own[f] + 1]; ++start[nei[f] + 1]; }
        for (int i = 0; i < N; ++i) start[i + 1] += start[i];
        adj.resize(start[N]);
        std::vector<int> pos(start.begin(), start.end() - 1);
        for (int f = 0; f < Fi; ++f) { adj[pos[own[f]]++] = nei[f]; adj[pos[nei[f]]++] = own[f]; }
        for (int i = 0; i < N; ++i) std::sort(adj.begin() + start[i], adj.begin() + start[i + 1]);
    }
};

void graph_bisect(const CellGraph& g, std::vector<int>& idx, int lo, int hi, int part0, int nparts, int32_t* out,
                  std::vector<int>& dist, std::vector<int>& stamp, int& tick) {
    if (nparts <= 1 || hi - lo <= 1) {
        for (int i = lo; i < hi; ++i) out[idx[i]] = part0;
        return;
    }
    // distances inside the set idx[lo, hi): -1 = not reached
    auto bfs = [&](int src) {
        ++tick;
        for (int i = lo; i < hi; ++i) { stamp[idx[i]] = tick; dist[idx[i]] = -1; }
        std::vector<int> q;
        q.reserve(hi - lo);
        q.push_back(src);
        dist[src] = 0;
        for (size_t h = 0; h < q.size(); ++h) {
            const int v = q[h];
            for (int k = g.start[v]; k < g.start[v + 1]; ++k) {
                const int w = g.adj[k];
                if (stamp[w] == tick && dist[w] < 0) { dist[w] = dist[v] + 1; q.push_back(w); }
            }
        }
        int far = idx[lo];
        for (int i = lo; i < hi; ++i)
            if (dist[idx[i]] > dist[far]) far = idx[i];
        return far;
    };
    bfs(bfs(idx[lo]));
    int dmax = 0;
    for (int i = lo; i < hi; ++i) dmax = std::max(dmax, dist[idx[i]]);
    for (int i = lo; i < hi; ++i)
        if (dist[idx[i]] < 0) dist[idx[i]] = dmax + 1;
    std::sort(idx.begin() + lo, idx.begin() + hi, [&](int a, int b) {
        return dist[a] < dist[b] || (dist[a] == dist[b] && a < b);
    });
    const int n1 = nparts / 2;
    const int mid = lo + (int)((long)(hi - lo) * n1 / nparts);
    graph_bisect(g, idx, lo, mid, part0, n1, out, dist, stamp, tick);
    graph_bisect(g, idx, mid, hi, part0 + n1, nparts - n1, out, dist, stamp, tick);
}

void graph_partition(int N, int Fi, const int32_t* own, const int32_t* nei, int nparts, int32_t* out) {
    CellGraph g(N, Fi, own, nei);
    std::vector<int> idx(N), dist(N, -1), stamp(N, 0);
    std::iota(idx.begin(), idx.end(), 0);
    int tick = 0;
    graph_bisect(g, idx, 0, N, 0, nparts, out, dist, stamp, tick);
}

struct Report5 { rdst_step_report r; };

// report of the current step into reps[sc->step_idx]; advances the slot
__global__ void k_report(Scalars* sc, rdst_step_report* reps, int cap) {
    if (threadIdx.x != 0) return;
    int idx = sc->step_idx;
    if (idx >= cap) return;
    rdst_step_report& r = reps[idx];
    r.time = sc->time;
    r.courant = sc->courant;
    for (int c = 0; c < 5; ++c) {
        r.res_l2[c] = sc->res_l2[c];
        r.lin_initial[c] = sc->lin_initial[c];
        r.lin_final[c] = sc->lin_final[c];
    }
    r.res_mag = sc->res_mag;
    r.lin_iterations = sc->lin_iterations;
    r.flags = sc->flags;
    r.rdt_min = sc->rdt_min;
    r.rdt_max = sc->rdt_max;
    r.t_flux_ms = r.t_jacobian_ms = r.t_precond_ms = r.t_krylov_ms = r.t_update_ms = 0.0;
    sc->step_idx = idx + 1;
}

__global__ void k_report_dt(const Scalars* sc, rdst_step_report* reps, int cap) {
    if (threadIdx.x == 0 && sc->step_idx < cap) reps[sc->step_idx].deltaT = sc->deltaT;
}

// mean of the per-cell Courant numbers: block partials, then one block
__global__ void k_mean_courant_partial(const double* __restrict__ cf, int N, double* __restrict__ partial) {
    double s = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) s += cf[i];
    s = block_sum(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}
__global__ void k_mean_courant(const double* __restrict__ partial, int nb, int N, const Scalars* sc,
                               rdst_step_report* reps, int cap) {
    double s = 0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[b];
    s = block_sum(s);
    if (threadIdx.x == 0 && sc->step_idx < cap) reps[sc->step_idx].courant = s / N;
}


}  // namespace

// ============================================================================
struct rdst_ctx {
    Options o;
    std::string err;
    cudaStream_t s = nullptr;
    int dev = -1;                   // the context's GPU (set at creation)
    // sizes
    int N = 0, Fi = 0, F = 0, NBall = 0, NB = 0, n_patches = 0;
    Thermo th{};
    Bounds bd{};
    // numbering
    std::vector<int> perm, iperm;       // perm[internal] = original
    DBuf<int> perm_d;                   // perm on the device
    DBuf<double> stage;                 // conservative fields in the caller's order (5N)
    std::vector<int> bface_orig;        // active bface -> foam face
    std::vector<double> hV, hC;         // original numbering, for forces
    std::vector<int> hown, hnei;        // foam owner/neighbour lists (topology check of a new geometry)
    std::vector<int> hpatch_start, hpatch_size;
    std::vector<int> bface_of_face;     // foam boundary face -> active bface (or -1)
    // device mesh
    DBuf<int> own, nei, bcell, bpatch, bfaceD, cf_start, cf_list, cf_slot, cc_start, cc_list;
    DBuf<double> Sf, magSf, w, dc, d, Cf, bSf, bmagSf, bdc, bCf, V, C, dS;
    DBuf<DevPatch> patches;
    DevMesh m{};
    // fields
    DBuf<double> W, prim, bs, q, qb, g, psi, fcell, fl, bfl, R, rhs, partial;
    DBuf<double> bjac;             // boundary Jacobian blocks of the active boundary faces
    DBuf<double> rdt, courantF, rhoOld, eOld, eNew;
    // viscous: grad U, face Up, viscous face terms, turbulent viscosity
    DBuf<double> gU, up, bup, vf, bvf, mut, mut_b;
    Transport tr{};
    // Spalart-Allmaras
    DBuf<double> nut, nut_b, ywall, saD, safv1, sadiag, sab, sax2, sagn, safup, saflo, safdP, safdQ, safcorr, sabd, sabb;
    DBuf<double> saSold, saRho0;        // SARC1: old-time strain rate, pre-update rho
    DBuf<int> saSoldValid;
    SAFields sa{};
    bool turb = false;
    DBuf<Scalars> sc;
    DBuf<rdst_step_report> reps;
    // matrix
    int n_slices = 0, n_slots = 0;
    DBuf<int> slice_off, slice_w, col;
    void* Aval = nullptr;
    void* LUval = nullptr;
    void* dinv = nullptr;
    size_t mt_size = 8;
    // ILU plan
    int n_parts = 1;
    DBuf<int> part_lvl0, lvl_off, low_start, nlu, tr_start, tr_kj, tr_rj, lu_col, lu_src;
    int lu_slots = 0;
    int ilu_ml = 0, ilu_mu = 0, ilu_mu_use = 0;
    // task records of the bulk ILU apply (empty: the register apply runs)
    DBuf<unsigned char> rec_f, rec_b;
    DBuf<uint2> task_f, task_b;
    DBuf<int> part_tf, part_tb;
    DBuf<unsigned> val_f, val_b;
    // addressing of the factorisation that reads A directly (else gather +
    // factor), both followed by the record pack
    DBuf<int> fr_trk, fr_trt;
    DBuf<int4> fr_desc;
    bool ilu_direct = false;
    int ilu_stage_bytes = 0;         // largest task record, rounded to 128 bytes
    int ilu_stages = 0;              // stages of the bulk apply (2 or 3)
    int ilu_lb_rows = 0;             // rows of each level buffer (0: none)
    int ilu_off_slots = 0;           // level offsets staged in shared memory (max levels + 1, even)
    int ilu_task_slots = 0;          // task table entries staged (max forward + backward tasks, even)
    // Krylov
    DBuf<double> dx, r, t, Vb, s2, sh, ph, pv, xbar, Ax, pA;
    DBuf<double> gs_r, gs_z;        // residual and correction of Gauss-Seidel sweeps after the first
    // block AMG: coarse levels 1.. (level 0 is the step's matrix)
    struct AmgDev {
        int n = 0, nnz = 0;
        DBuf<int> start, col, dslot;   // block CSR, columns ascending
        DBuf<int> gstart, gsrc;        // Galerkin gather: coarse slot -> finer slots
        DBuf<int> mstart, mem;         // members (finer nodes) of each node, ascending
        DBuf<int> agg;                 // finer node -> node of this level
        DBuf<double> val, dinv;        // 25 nnz, 25 n
        DBuf<double> x, b, r;          // 5 n
    };
    std::vector<std::unique_ptr<AmgDev>> amg;
    DBuf<double> amg_r0;            // level-0 residual
    DBuf<unsigned char> rmask;      // held cells (internal order): zero residual, identity rows; empty: none
    DBuf<float> Vf;                 // GMRES basis when it is kept in FP32
    long ldv = 0;                   // stride between basis vectors (entries)
    DBuf<double> wv;                // FP64 Arnoldi vector that is orthogonalised before it is stored in Vf
    // discrete adjoint (allocated on first use)
    DBuf<double> a_fbar, a_qbbar, a_qbar, a_gbar, a_vval, a_hval, a_wbar, a_wbarb, a_ubarb, a_pbar;
    DBuf<double> a_r, a_z, a_t, a_psi, a_rhs, a_V, a_tmp, a_u3;
    DBuf<int> a_vidx, a_hidx;
    DBuf<double> a_Z;               // flexible-GMRES preconditioned directions
    DBuf<double> a_vfbar, a_vbbar, a_gUbar, a_ucbar;   // viscous input bars (faces, boundary faces, cells)
    // dual-time stepping: W at the previous two time levels, foam Time's
    // deltaTSave, the step's a of dual2ndDST (0 outside a dual step)
    DBuf<double> dWn, dWnm1;
    DBuf<double> nutN, nutNm1;      // nuTilda old time levels of dual-time stepping
    bool dual_started = false;
    double dt_save = 1.0, dual_a = 0.0, dual_b = 0.0, dual_c = 0.0;
    // SARC1 under dual-time stepping: S.oldTime() and its oldTime(), the
    // time indices foam gives S and each of them (-1: not created), the
    // physical step's index and its deltaT / deltaT0
    DBuf<double> saSo, saSoo;
    int sa_S_idx = -1, sa_o_idx = -1, sa_oo_idx = -1, dual_tidx = 0;
    double dual_dt = 1.0, dual_dt0 = 1.0;
    DBuf<Scalars> a_sc;             // Hessenberg and rotations of the adjoint's outer solve
    void* a_AT = nullptr;           // transposed Jacobian (storage type of A)
    DBuf<double> t_buf;             // tangent records (value, derivative)
    int a_m = 0;
    int limiter_need_grad = 1, venkat_mask = 0;
    bool steady = false;
    bool state_set = false;
    // graphs: whole step (fixed iteration count) or pre / one iteration / post
    struct EvRec { cudaEvent_t a, b; int kind; };
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        long launches = 0;
        std::vector<EvRec> events;   // external event records inside the graph
    };
    Graph g_step, g_pre, g_cycle, g_post;
    bool capturing = false;
    std::vector<EvRec>* capture_events = nullptr;
    static constexpr int REP_CAP = 1024;
    // instrumentation
    long launches = 0;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<EvRec> ev_pending;
    long ks_launches[KS_N] = {0, 0, 0, 0, 0, 0, 0};
    double ks_ms[KS_N] = {0, 0, 0, 0, 0, 0, 0};
    cudaEvent_t step_ev[2] = {nullptr, nullptr};
    double last_step_ms = 0.0;
    cudaEvent_t get_event() {
        if (!ev_pool.empty()) { cudaEvent_t e = ev_pool.back(); ev_pool.pop_back(); return e; }
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        return e;
    }
    void collect_graph_events(const Graph& g) {
        for (auto& r : g.events) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, r.a, r.b));
            ks_ms[r.kind] += ms;
            ks_launches[r.kind] += 1;
        }
    }
    void collect_events() {
        for (auto& r : ev_pending) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, r.a, r.b));
            ks_ms[r.kind] += ms;
            ks_launches[r.kind] += 1;
            ev_pool.push_back(r.a);
            ev_pool.push_back(r.b);
        }
        ev_pending.clear();
    }

    // drop the captured step graphs (recaptured by the next step)
    void reset_graphs() {
        for (Graph* g : {&g_step, &g_pre, &g_cycle, &g_post}) {
            if (g->exec) cudaGraphExecDestroy(g->exec);
            for (auto& r : g->events) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
            *g = Graph{};
        }
    }

    ~rdst_ctx() {
        for (auto e : ev_pool) cudaEventDestroy(e);
        for (auto e : step_ev) if (e) cudaEventDestroy(e);
        for (auto& r : ev_pending) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
        for (Graph* g : {&g_step, &g_pre, &g_cycle, &g_post}) {
            if (g->exec) cudaGraphExecDestroy(g->exec);
            for (auto& r : g->events) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
        }
        if (Aval) cudaFree(Aval);
        if (LUval) cudaFree(LUval);
        if (dinv) cudaFree(dinv);
        if (a_AT) cudaFree(a_AT);
        if (s) cudaStreamDestroy(s);
    }

    template <typename MT>
    SellMat<MT> mat(void* val) const {
        SellMat<MT> A;
        A.N = N; A.n_slices = n_slices; A.slice_off = slice_off.p; A.slice_w = slice_w.p; A.col = col.p;
        A.val = (MT*)val;
        return A;
    }
    IluDev ilu() const {
        IluDev P;
        P.n_parts = n_parts; P.part_lvl0 = part_lvl0.p; P.lvl_off = lvl_off.p;
        P.nlu = nlu.p; P.low_start = low_start.p; P.ml = ilu_ml; P.mu = ilu_mu; P.mu_use = ilu_mu_use; P.lu_col = lu_col.p; P.lu_src = lu_src.p;
        P.tr_start = tr_start.p; P.tr_kj = tr_kj.p; P.tr_rj = tr_rj.p;
        P.rec_f = rec_f.p; P.rec_b = rec_b.p; P.task_f = task_f.p; P.task_b = task_b.p;
        P.part_tf = part_tf.p; P.part_tb = part_tb.p; P.val_f = val_f.p; P.val_b = val_b.p;
        P.fr_trk = fr_trk.p; P.fr_trt = fr_trt.p; P.fr_desc = fr_desc.p;
        return P;
    }
    long nvec() const { return 5L * N; }
};

namespace {

// event pair around one kernel launch when the context profiles
struct Timed {
    rdst_ctx& c;
    int kind;
    cudaEvent_t a = nullptr;
    Timed(rdst_ctx& c_, int k) : c(c_), kind(k) {
        if (!c.o.profile) return;
        if (c.capturing) {
            CK(cudaEventCreate(&a));
            CK(cudaEventRecordWithFlags(a, c.s, cudaEventRecordExternal));
        } else {
            a = c.get_event();
            CK(cudaEventRecord(a, c.s));
        }
    }
    ~Timed() {
        if (!a) return;
        if (c.capturing) {
            cudaEvent_t b;
            cudaEventCreate(&b);
            cudaEventRecordWithFlags(b, c.s, cudaEventRecordExternal);
            c.capture_events->push_back({a, b, kind});
        } else {
            cudaEvent_t b = c.get_event();
            cudaEventRecord(b, c.s);
            c.ev_pending.push_back({a, b, kind});
        }
    }
};

struct CounterScope {
    long* prev;
    explicit CounterScope(rdst_ctx& c) : prev(g_launch_counter) { g_launch_counter = &c.launches; }
    ~CounterScope() { g_launch_counter = prev; }
};

int flux_code(FluxScheme f) { return (int)f; }
int lim_code(Limiter l) { return (int)l; }

// Default number of ILU(0) subdomains: about 1536 rows each.  The apply
// runs one CTA per subdomain and its time is set by the level-to-level
// chain of each CTA, so once there are more subdomains than CTAs the GPU
// holds at once the count is rounded to a whole number of such waves (a
// partial last wave costs a whole extra chain: measured on the 1.2 M-cell
// wing with the register apply, 784 parts took 23% longer than 592 or
// 1184).  The bulk apply holds eight CTAs an SM (64 registers a thread, its
// shared memory sized for that), the register apply four.
int auto_ilu_parts(int N, Precision prec, bool bulk) {
    int dev = 0, sms = 0, per_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // a small mesh still gets one subdomain per SM, down to 128 rows each:
    // with a few large subdomains the apply is one long level chain on a few
    // SMs (257x65 C-mesh: 10 subdomains 259 us per apply, 130 subdomains
    // 104 us, and 280 steps to a 1e-10 drop instead of 284)
    const int p0 = std::max({1, N / 1536, std::min(sms, N / 128)});
    // the four-slot instance bounds the register use of the ones hex meshes need
    if (bulk)
        per_sm = 8;
    else if (prec == PREC_FP64)
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ilu_apply<double, 4>, ILU_APPLY_TPB, 0));
    else if (prec == PREC_FP32)
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ilu_apply<float, 4>, ILU_APPLY_TPB, 0));
    else
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ilu_apply<__nv_bfloat16, 4>, ILU_APPLY_TPB, 0));
    const long wave = std::max(1L, (long)sms * per_sm);
    if (p0 <= wave) return std::min(p0, N);
    const long waves = std::max(1L, std::lround((double)p0 / (double)wave));
    return (int)std::min<long>(waves * wave, N);
}

// ---------------------------------------------------------------- set-up
// Mesh metrics in the internal row order: face area vectors, centres,
// interpolation weights and delta coefficients, owner-to-neighbour vectors,
// cell volumes and centres, the componentwise half face-area sums of the
// local time step (timeDST.C:117-153) and the wall distance.  With
// `in_place` the values are copied into the buffers of an existing context
// whose topology is unchanged, so every device pointer (and the CUDA graphs
// that hold them) stays valid.
void load_geometry(rdst_ctx& c, const rdst_mesh* mh, bool in_place) {
    cudaStream_t s = c.s;
    const int N = c.N, Fi = c.Fi, F = c.F, NB = c.NB;
    std::vector<double> Sf(3 * (size_t)Fi), magSf(Fi), w(Fi), dc(Fi), d(3 * (size_t)Fi), Cf(3 * (size_t)Fi);
    for (int f = 0; f < Fi; ++f) {
        for (int k = 0; k < 3; ++k) {
            Sf[k * (size_t)Fi + f] = mh->Sf[3 * f + k];
            Cf[k * (size_t)Fi + f] = mh->Cf[3 * f + k];
            d[k * (size_t)Fi + f] = mh->C[3 * mh->neighbour[f] + k] - mh->C[3 * mh->owner[f] + k];
        }
        magSf[f] = mh->magSf[f]; w[f] = mh->weights[f]; dc[f] = mh->deltaCoeffs[f];
    }
    std::vector<double> bSf(3 * (size_t)NB), bmagSf(NB), bdc(NB), bCf(3 * (size_t)NB);
    for (int b = 0; b < NB; ++b) {
        int f = c.bface_orig[b];
        for (int k = 0; k < 3; ++k) {
            bSf[k * (size_t)NB + b] = mh->Sf[3 * f + k];
            bCf[k * (size_t)NB + b] = mh->Cf[3 * f + k];
        }
        bmagSf[b] = mh->magSf[f]; bdc[b] = mh->deltaCoeffs[f];
    }
    std::vector<double> V(N), C(3 * (size_t)N), dS(3 * (size_t)N, 0.0);
    c.hV.assign(mh->V, mh->V + N);
    c.hC.assign(mh->C, mh->C + 3 * (size_t)N);
    for (int r = 0; r < N; ++r) {
        int i = c.perm[r];
        V[r] = mh->V[i];
        for (int k = 0; k < 3; ++k) C[k * (size_t)N + r] = mh->C[3 * i + k];
    }
    // dS = 1/2 sum |Sf| componentwise (timeDST.C:117-153), non-empty faces
    for (int f = 0; f < F; ++f) {
        if (f >= Fi && c.bface_of_face[f - Fi] < 0) continue;
        int ro = c.iperm[mh->owner[f]];
        for (int k = 0; k < 3; ++k) dS[3 * ro + k] += std::fabs(mh->Sf[3 * f + k]);
        if (f < Fi) {
            int rn = c.iperm[mh->neighbour[f]];
            for (int k = 0; k < 3; ++k) dS[3 * rn + k] += std::fabs(mh->Sf[3 * f + k]);
        }
    }
    for (auto& x : dS) x *= 0.5;
    std::vector<double> yv;
    if (c.turb) {
        yv.resize(N);
        for (int r = 0; r < N; ++r) yv[r] = mh->wall_distance[c.perm[r]];
    }
    auto put = [&](DBuf<double>& b, const std::vector<double>& v) {
        if (in_place) b.overwrite(v, s); else b.upload(v, s);
    };
    put(c.Sf, Sf); put(c.magSf, magSf); put(c.w, w); put(c.dc, dc); put(c.d, d); put(c.Cf, Cf);
    put(c.bSf, bSf); put(c.bmagSf, bmagSf); put(c.bdc, bdc); put(c.bCf, bCf);
    put(c.V, V); put(c.C, C); put(c.dS, dS);
    if (c.turb) put(c.ywall, yv);
    CK(cudaStreamSynchronize(s));
}

// The bulk apply's task records (IluDev::rec_f / rec_b): the tasks of each
// part in the order the apply's cursor takes them (forward: levels
// ascending; backward: levels descending; 24-row chunks of a level in
// ascending rows), their headers and columns written here, the blocks by
// k_ilu_pack after each factorisation.  Three stages when the CTAs every
// subdomain needs at once (up to eight an SM) still fit with them, else
// two; a task too large for one CTA's shared memory leaves the register
// apply in place.
void build_task_records(rdst_ctx& c, const Options& o, int nparts, const std::vector<int>& part_lvl0,
                        const std::vector<int>& lvl_off, const std::vector<int>& lu_col,
                        const std::vector<int>& lu_src, const std::vector<int>& nlu,
                        const std::vector<int>& low_start, const std::vector<int>& tr_start,
                        const std::vector<int>& tr_kj, const std::vector<int>& tr_rj, const std::vector<int>& nl,
                        const std::vector<int>& nu, int ML, int MS) {
    const int N = c.N;
    const size_t S = o.precision == PREC_FP64 ? 8 : (o.precision == PREC_FP32 ? 4 : 2);
    auto lfid = [&](int r, int sl) { return ((r >> 5) * MS + sl) * 32 + (r & 31); };
    auto r16 = [](size_t v) { return (v + 15) / 16 * 16; };
    auto cnt_of = [&](int r, bool back) { return back ? (c.ilu_mu_use ? nu[r] : 0) : nl[r]; };
    auto rec_bytes = [&](int r, bool back) {
        const int n = cnt_of(r, back);
        return r16(16 * (size_t)((n + 3) / 4) + (size_t)(n + (back ? 1 : 0)) * 25 * S);
    };
    struct Tk { int r0, n; };
    std::vector<Tk> tf, tb;
    std::vector<int> ptf(nparts + 1, 0), ptb(nparts + 1, 0);
    int maxw = 0, maxlv = 0, maxtasks = 0;
    for (int p = 0; p < nparts; ++p) {
        ptf[p] = (int)tf.size();
        ptb[p] = (int)tb.size();
        const int a = part_lvl0[p], e = part_lvl0[p + 1];
        maxlv = std::max(maxlv, e - a);
        for (int li = a; li < e; ++li) {
            const int r0 = lvl_off[li], n = lvl_off[li + 1] - r0;
            maxw = std::max(maxw, n);
            for (int b = 0; b < n; b += ILU_BULK_RPT) tf.push_back({r0 + b, std::min(ILU_BULK_RPT, n - b)});
        }
        for (int li = e - 1; li >= a; --li) {
            const int r0 = lvl_off[li], n = lvl_off[li + 1] - r0;
            for (int b = 0; b < n; b += ILU_BULK_RPT) tb.push_back({r0 + b, std::min(ILU_BULK_RPT, n - b)});
        }
        maxtasks = std::max(maxtasks, (int)(tf.size() - ptf[p] + tb.size() - ptb[p]));
    }
    ptf[nparts] = (int)tf.size();
    ptb[nparts] = (int)tb.size();
    size_t max_task = 0;
    auto layout = [&](const std::vector<Tk>& tasks, bool back, std::vector<uint2>& tab) {
        tab.resize(tasks.size());
        size_t pos = 0;
        for (size_t t = 0; t < tasks.size(); ++t) {
            size_t bytes = ILU_BULK_HDR;
            for (int i = 0; i < tasks[t].n; ++i) bytes += rec_bytes(tasks[t].r0 + i, back);
            tab[t] = make_uint2((unsigned)(pos / 16), (unsigned)bytes);
            pos += bytes;
            max_task = std::max(max_task, bytes);
        }
        return pos;
    };
    std::vector<uint2> tabf, tabb;
    const size_t totf = layout(tf, false, tabf), totb = layout(tb, true, tabb);
    // shared memory: stages, y0 slots, level buffers, task table, level offsets
    const int stage = (int)((max_task + 127) / 128 * 128);
    const int lb = maxw <= ILU_LB_MAX ? maxw : 0;
    const int task_slots = (maxtasks + 1) / 2 * 2;
    const int off_slots = (maxlv + 2) / 2 * 2;
    auto smem = [&](int ns) {
        return (size_t)ns * stage + (size_t)ns * ILU_BULK_TPB * 8 + (size_t)lb * (S == 8 ? 96 : 64) +
               (size_t)task_slots * 8 + (size_t)off_slots * 4 + 64;
    };
    int dev = 0, per_sm = 0, per_block = 0, reserved = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    CK(cudaDeviceGetAttribute(&per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    CK(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    // CTAs an SM must hold for all subdomains to run at once (up to 8)
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t want = (size_t)std::min(8, std::max(1, (nparts + sms - 1) / std::max(sms, 1)));
    int ns = 3;
    if ((smem(3) + reserved) * want > (size_t)per_sm) ns = 2;
    if (smem(ns) > (size_t)per_block) return;
    if ((size_t)(std::max(ML, MS - ML) + 1) * 25 * 33 * S > (size_t)per_block) return;   // the pack's tiles
    std::vector<unsigned char> bf(totf, 0), bb(totb, 0);
    std::vector<unsigned> vf(N, 0), vb(N, 0);
    auto fill = [&](const std::vector<Tk>& tasks, const std::vector<uint2>& tab, bool back,
                    std::vector<unsigned char>& buf, std::vector<unsigned>& val) {
        for (size_t t = 0; t < tasks.size(); ++t) {
            const size_t start = (size_t)tab[t].x * 16;
            unsigned* hdr = reinterpret_cast<unsigned*>(buf.data() + start);
            size_t pos = start + ILU_BULK_HDR;
            for (int i = 0; i < tasks[t].n; ++i) {
                const int r = tasks[t].r0 + i, n = cnt_of(r, back);
                hdr[i] = (unsigned)(pos - start) | ((unsigned)n << 24);
                int* cols = reinterpret_cast<int*>(buf.data() + pos);
                const int ncol = 4 * ((n + 3) / 4);
                for (int q = 0; q < ncol; ++q) cols[q] = q < n ? lu_col[lfid(r, back ? ML + q : q)] : -1;
                val[r] = (unsigned)((pos + 16 * (size_t)((n + 3) / 4)) / 16);
                pos += rec_bytes(r, back);
            }
        }
    };
    fill(tf, tabf, false, bf, vf);
    fill(tb, tabb, true, bb, vb);
    cudaStream_t s = c.s;
    c.rec_f.upload(bf, s); c.rec_b.upload(bb, s);
    c.task_f.upload(tabf, s); c.task_b.upload(tabb, s);
    c.part_tf.upload(ptf, s); c.part_tb.upload(ptb, s);
    c.val_f.upload(vf, s); c.val_b.upload(vb, s);
    // the factorisation reading A directly: where each update triple reads
    // U_kj and which slot of row r takes it, and one descriptor per L slot
    {
        std::vector<int> trk(tr_kj.size()), trt(tr_rj.size());
        for (size_t t = 0; t < tr_kj.size(); ++t) {
            const int kj = tr_kj[t];
            const int k = ((kj >> 5) / MS) * 32 + (kj & 31);
            trk[t] = (nlu[k] >> 16) & 1 ? -kj - 1 : (lu_src[kj] >= 0 ? lu_src[kj] : INT_MIN);
            trt[t] = tr_rj[t] < 0 ? -1 : (tr_rj[t] >> 5) % MS;
        }
        std::vector<int4> desc(low_start[N]);
        for (int r = 0; r < N; ++r)
            for (int q = 0; q < nl[r]; ++q) {
                const int i = low_start[r] + q, t0 = tr_start[i], t1 = tr_start[i + 1];
                int4 d;
                d.x = lu_col[lfid(r, q)];
                d.y = lu_src[lfid(r, q)];
                d.z = t1 > t0 ? trk[t0] : 0;
                d.w = (t1 > t0 ? trt[t0] + 2 : 0) | (t1 - t0 > 1 ? 1 << 20 : 0);
                desc[i] = d;
            }
        if (ML <= ILU_FR_MAXQ) {
            c.fr_trk.upload(trk, s);
            c.fr_trt.upload(trt, s);
            c.fr_desc.upload(desc, s);
            c.ilu_direct = true;
        }
    }
    c.ilu_stage_bytes = stage;
    c.ilu_stages = ns;
    c.ilu_lb_rows = lb;
    c.ilu_task_slots = task_slots;
    c.ilu_off_slots = off_slots;
    CK(cudaStreamSynchronize(s));
}

template <typename MT>
static void ilu_bulk_attr(rdst_ctx& c);

void build(rdst_ctx& c, const rdst_mesh* mh) {
    cudaStream_t s = c.s;
    const int N = mh->n_cells, Fi = mh->n_internal_faces, F = mh->n_faces;
    c.N = N; c.Fi = Fi; c.F = F; c.NBall = F - Fi; c.n_patches = mh->n_patches;
    const Options& o = c.o;
    c.th.R = o.R; c.th.Cp = o.Cp; c.th.Cv = o.Cv(); c.th.gamma = o.gamma();
    c.bd = Bounds{o.rho_min, o.rho_max, o.p_min, o.p_max, o.T_min, o.T_max};
    c.tr = Transport{o.mu, o.As, o.Ts, o.Pr, o.Prt, (o.mu > 0 || o.As > 0 || o.turbulence != TURB_LAMINAR) ? 1 : 0};
    c.steady = (o.ddt == DDT_STEADY);
    // active boundary faces
    std::vector<int> fpatch(c.NBall, -1);
    std::vector<DevPatch> dp(mh->n_patches);
    for (int p = 0; p < mh->n_patches; ++p) {
        const rdst_patch& P = mh->patches[p];
        if (P.start < Fi || P.start + P.size > F || P.size < 0) throw std::invalid_argument("patch range outside the boundary faces");
        for (int f = P.start; f < P.start + P.size; ++f) fpatch[f - Fi] = p;
        DevPatch& d = dp[p];
        d.type = P.type; d.bc_p = P.bc_p; d.bc_U = P.bc_U; d.bc_T = P.bc_T; d.bc_nut = P.bc_nuTilda;
        d.p_value = P.p_value; d.T_value = P.T_value; d.nut_value = P.nuTilda_value;
        for (int k = 0; k < 3; ++k) d.U_value[k] = P.U_value[k];
        c.hpatch_start.push_back(P.start);
        c.hpatch_size.push_back(P.size);
    }
    c.bface_of_face.assign(c.NBall, -1);
    for (int b = 0; b < c.NBall; ++b) {
        if (fpatch[b] < 0) throw std::invalid_argument("boundary face not covered by a patch");
        if (mh->patches[fpatch[b]].type != RDST_PATCH_EMPTY) {
            c.bface_of_face[b] = (int)c.bface_orig.size();
            c.bface_orig.push_back(Fi + b);
        }
    }
    const int NB = (int)c.bface_orig.size();
    c.NB = NB;
    for (int f = 0; f < F; ++f)
        if (mh->owner[f] < 0 || mh->owner[f] >= N) throw std::invalid_argument("owner index out of range");
    for (int f = 0; f < Fi; ++f)
        if (mh->neighbour[f] < 0 || mh->neighbour[f] >= N || mh->neighbour[f] == mh->owner[f])
            throw std::invalid_argument("neighbour index out of range");
    // cell adjacency (original numbering), faces ascending
    std::vector<std::vector<int>> cfaces(N);
    for (int f = 0; f < Fi; ++f) { cfaces[mh->owner[f]].push_back(f); cfaces[mh->neighbour[f]].push_back(f); }
    for (int b = 0; b < NB; ++b) cfaces[mh->owner[c.bface_orig[b]]].push_back(Fi + b);
    for (auto& v : cfaces) std::sort(v.begin(), v.end());
    // partition + wavefront levels for the subdomain factorisations.  The
    // factor pattern of a row (original numbering) is its same-part face
    // neighbours, or for ILUCp the same-part cells within fill_in + 1 faces
    // (neighbours of neighbours, level by level, as foam-extend's
    // extendedLduAddressing builds them).
    std::vector<int> part(N, 0), level(N, 0), rank;
    bool bfs_order = false;
    std::vector<std::vector<int>> lupat;
    int nparts = 1;
    const bool factored = lu_factored(o.precon);
    if (factored) {
        nparts = o.ilu_parts > 0 ? o.ilu_parts : auto_ilu_parts(N, o.precision, o.ilu_bulk);
        nparts = std::min(nparts, N);
        if (o.ilu_graph) {
            graph_partition(N, Fi, mh->owner, mh->neighbour, nparts, part.data());
        } else {
            std::vector<int> idx(N);
            std::iota(idx.begin(), idx.end(), 0);
            rcb(mh->C, idx, 0, N, 0, nparts, part.data());
        }
        lupat.resize(N);
        for (int i = 0; i < N; ++i)
            for (int f : cfaces[i]) {
                if (f >= Fi) continue;
                int k = mh->owner[f] == i ? mh->neighbour[f] : mh->owner[f];
                if (part[k] == part[i]) lupat[i].push_back(k);
            }
        for (auto& v : lupat) { std::sort(v.begin(), v.end()); v.erase(std::unique(v.begin(), v.end()), v.end()); }
        if (o.precon == PRECON_ILUCP && o.fill_in > 0) {
            std::vector<std::vector<int>> ext(N);
            std::vector<int> mark(N, -1);
            for (int i = 0; i < N; ++i) {
                std::vector<int> front = lupat[i], seen = lupat[i];
                mark[i] = i;
                for (int k : front) mark[k] = i;
                for (int lev = 0; lev < o.fill_in; ++lev) {
                    std::vector<int> next;
                    for (int a : front)
                        for (int b2 : lupat[a])
                            if (mark[b2] != i) { mark[b2] = i; next.push_back(b2); seen.push_back(b2); }
                    front.swap(next);
                }
                std::sort(seen.begin(), seen.end());
                ext[i].swap(seen);
            }
            lupat.swap(ext);
        }
        // factorisation order of each subdomain: mesh order, or breadth
        // first (rdst_order.h); a row's wavefront level is one past the
        // deepest of its pattern cells that come before it
        bfs_order = o.ilu_order == 1 || (o.ilu_order < 0 && nparts > 1);
        rank.resize(N);
        if (bfs_order) {
            std::vector<std::vector<int>> adj(N);
            for (int f = 0; f < Fi; ++f) { adj[mh->owner[f]].push_back(mh->neighbour[f]); adj[mh->neighbour[f]].push_back(mh->owner[f]); }
            rank = subdomain_bfs_rank(adj, part);
        } else {
            std::iota(rank.begin(), rank.end(), 0);
        }
        std::vector<int> byrank(N);
        std::iota(byrank.begin(), byrank.end(), 0);
        if (bfs_order)
            std::sort(byrank.begin(), byrank.end(), [&](int a, int b) {
                return part[a] != part[b] ? part[a] < part[b] : rank[a] < rank[b];
            });
        for (int i : byrank) {
            int lv = 0;
            for (int k : lupat[i])
                if (rank[k] < rank[i]) lv = std::max(lv, level[k] + 1);
            level[i] = lv;
        }
    }
    c.n_parts = nparts;
    c.perm.resize(N);
    std::iota(c.perm.begin(), c.perm.end(), 0);
    if (factored)
        std::stable_sort(c.perm.begin(), c.perm.end(), [&](int a, int b) {
            if (part[a] != part[b]) return part[a] < part[b];
            if (level[a] != level[b]) return level[a] < level[b];
            return rank[a] < rank[b];
        });
    c.iperm.resize(N);
    for (int r = 0; r < N; ++r) c.iperm[c.perm[r]] = r;
    // ---- device mesh
    std::vector<int> own(Fi), nei(Fi);
    for (int f = 0; f < Fi; ++f) {
        own[f] = c.iperm[mh->owner[f]];
        nei[f] = c.iperm[mh->neighbour[f]];
    }
    std::vector<int> bcell(NB), bpatch(NB);
    for (int b = 0; b < NB; ++b) {
        int f = c.bface_orig[b];
        bcell[b] = c.iperm[mh->owner[f]];
        bpatch[b] = fpatch[f - Fi];
    }
    c.hown.assign(mh->owner, mh->owner + F);
    c.hnei.assign(mh->neighbour, mh->neighbour + Fi);
    // cell -> face CSR in internal row order (codes: f < Fi internal, Fi+b boundary)
    std::vector<int> cf_start(N + 1, 0), cf_list, cc_start(N + 1, 0), cc_list;
    for (int r = 0; r < N; ++r) {
        for (int fc : cfaces[c.perm[r]]) cf_list.push_back(fc);
        cf_start[r + 1] = (int)cf_list.size();
    }
    // SELL-32 structure for the Jacobian: slot 0 the diagonal, then the
    // neighbours by internal column (several faces may join one cell pair,
    // allowed by foam's polyMesh: one block per pair, the faces accumulate).
    std::vector<int> ipart(N, 0);
    for (int r = 0; r < N; ++r) ipart[r] = part[c.perm[r]];
    c.n_slices = (N + 31) / 32;
    std::vector<int> slice_off(c.n_slices + 1, 0), slice_w(c.n_slices, 1);
    std::vector<std::vector<int>> rowcols(N);
    for (int r = 0; r < N; ++r) {
        for (int k = cf_start[r]; k < cf_start[r + 1]; ++k) {
            int fc = cf_list[k];
            if (fc >= Fi) continue;
            int other = own[fc] == r ? nei[fc] : own[fc];
            rowcols[r].push_back(other);
            cc_list.push_back(other);
        }
        cc_start[r + 1] = (int)cc_list.size();
        std::sort(rowcols[r].begin(), rowcols[r].end());
        rowcols[r].erase(std::unique(rowcols[r].begin(), rowcols[r].end()), rowcols[r].end());
    }
    auto pos_of = [&](int r, int cc) {
        auto it = std::lower_bound(rowcols[r].begin(), rowcols[r].end(), cc);
        return (it != rowcols[r].end() && *it == cc) ? (int)(it - rowcols[r].begin()) : -1;
    };
    for (int sl = 0; sl < c.n_slices; ++sl) {
        int wmax = 1;
        for (int r = sl * 32; r < std::min(N, sl * 32 + 32); ++r) wmax = std::max(wmax, 1 + (int)rowcols[r].size());
        slice_w[sl] = wmax;
        slice_off[sl + 1] = slice_off[sl] + wmax;
    }
    c.n_slots = slice_off[c.n_slices];
    std::vector<int> col((size_t)c.n_slots * 32, -1);
    auto flat = [&](int r, int k) { return (slice_off[r >> 5] + k) * 32 + (r & 31); };
    for (int r = 0; r < N; ++r) {
        col[flat(r, 0)] = r;
        for (size_t k = 0; k < rowcols[r].size(); ++k) col[flat(r, 1 + (int)k)] = rowcols[r][k];
    }
    // slot of each cell-face entry: k >= 0 stores the block into slot k, a
    // negative entry -(k+1) adds it (second and later faces of a cell pair)
    std::vector<int> cf_slot(cf_list.size(), 0);
    for (int r = 0; r < N; ++r) {
        std::vector<char> seen(rowcols[r].size(), 0);
        for (int k = cf_start[r]; k < cf_start[r + 1]; ++k) {
            int fc = cf_list[k];
            if (fc >= Fi) continue;
            int other = own[fc] == r ? nei[fc] : own[fc];
            int pos = pos_of(r, other);
            int slot = 1 + pos;
            cf_slot[k] = seen[pos] ? -(1 + slot) : slot;
            seen[pos] = 1;
        }
    }
    // ---- factorisation plan.  The factors live in their own ELL layout,
    // factor slot s x cell: L_q (same-subdomain lower, by column) at
    // s = q < ML, U_q at s = ML + q; entries interleaved by cell,
    // lu_val[(s*25 + e)*N + r].  Wavefront levels are contiguous row ranges
    // per subdomain.  Slots outside the matrix pattern (ILUCp fill) start
    // from zero blocks.
    if (factored) {
        std::vector<std::vector<int>> lurows(N);     // factor pattern in row order, ascending
        for (int r = 0; r < N; ++r) {
            for (int k : lupat[c.perm[r]]) lurows[r].push_back(c.iperm[k]);
            std::sort(lurows[r].begin(), lurows[r].end());
        }
        std::vector<int> nl(N, 0), nu(N, 0);
        for (int r = 0; r < N; ++r)
            for (int cc : lurows[r]) { if (cc < r) ++nl[r]; else ++nu[r]; }
        const int ML = *std::max_element(nl.begin(), nl.end());
        const int MU = *std::max_element(nu.begin(), nu.end());
        // the mesh's own pattern: up to 8 lower/upper neighbours; ILUCp fill
        // up to 16 (the wider apply keeps its factor rows partly in local
        // memory)
        if (ML > 8 || MU > 8) {
            if (!(o.precon == PRECON_ILUCP && o.fill_in > 0))
                throw std::invalid_argument("a cell has more than 8 lower/upper neighbours");
            if (ML > 16 || MU > 16)
                throw ConfigError("ILUCp fillInLevel " + std::to_string(o.fill_in) +
                                  " gives a cell more than 16 lower/upper factor blocks on this mesh", true);
        }
        c.ilu_ml = ML;
        c.ilu_mu = MU;
        // Gauss-Seidel applies (D + L)^-1: the backward sweep uses no U blocks
        c.ilu_mu_use = o.precon == PRECON_GAUSS_SEIDEL ? 0 : MU;
        const int MS = std::max(ML + MU, 1);
        // factor id of slot s of row r: slices of 32 rows, MS slots each,
        // entries interleaved by lane (the SELL addressing with width MS)
        auto lfid = [&](int r, int sl) { return ((r >> 5) * MS + sl) * 32 + (r & 31); };
        std::vector<int> lu_col((size_t)c.n_slices * MS * 32, -1), lu_src((size_t)c.n_slices * MS * 32, -1);
        auto fid_of = [&](int r, int cc) {     // factor id of coupling (r, cc), or -1
            auto it = std::lower_bound(lurows[r].begin(), lurows[r].end(), cc);
            if (it == lurows[r].end() || *it != cc) return -1;
            const int k = (int)(it - lurows[r].begin());
            return cc < r ? lfid(r, k) : lfid(r, ML + k - nl[r]);
        };
        for (int r = 0; r < N; ++r) {
            int ql = 0, qu = 0;
            for (int cc : lurows[r]) {
                int sidx = cc < r ? ql++ : ML + qu++;
                lu_col[lfid(r, sidx)] = cc;
                const int pos = pos_of(r, cc);
                lu_src[lfid(r, sidx)] = pos >= 0 ? flat(r, 1 + pos) : -2;   // -2: fill, zeroed per factorisation
            }
        }
        std::vector<int> lvl_off, part_lvl0(nparts + 1, 0);
        for (int r = 0; r < N; ++r) {
            if (r == 0 || ipart[r] != ipart[r - 1] || level[c.perm[r]] != level[c.perm[r - 1]]) lvl_off.push_back(r);
        }
        lvl_off.push_back(N);
        {
            int li = 0;
            for (int p = 0; p < nparts; ++p) {
                part_lvl0[p] = li;
                while (li < (int)lvl_off.size() - 1 && ipart[lvl_off[li]] == p) ++li;
            }
            part_lvl0[nparts] = (int)lvl_off.size() - 1;
        }
        // IKJ update triples: for each L_rk (row order, then q), the pairs
        // (U_kj, A_rj) with j > k in row k's upper factor and in row r's
        // pattern (j == r: the diagonal, encoded -1).  Cholesky keeps only
        // the diagonal ones, Gauss-Seidel none.
        const bool upd_off = o.precon == PRECON_ILU0 || o.precon == PRECON_ILUCP;
        const bool upd_diag = upd_off || o.precon == PRECON_CHOLESKY;
        std::vector<int> nlu(N), low_start(N + 1, 0), tr_start(1, 0), tr_kj, tr_rj;
        for (int r = 0; r < N; ++r) {
            nlu[r] = nl[r] | (nu[r] << 8);
            low_start[r + 1] = low_start[r] + nl[r];
        }
        for (int r = 0; r < N; ++r) {
            for (int q = 0; q < nl[r]; ++q) {
                int k = lu_col[lfid(r, q)];
                for (int u = 0; u < nu[k]; ++u) {
                    int j = lu_col[lfid(k, ML + u)];
                    int kj = lfid(k, ML + u);
                    if (j == r) {
                        if (upd_diag) { tr_kj.push_back(kj); tr_rj.push_back(-1); }
                        continue;
                    }
                    if (!upd_off || ipart[j] != ipart[r]) continue;
                    int rj = fid_of(r, j);
                    if (rj >= 0) { tr_kj.push_back(kj); tr_rj.push_back(rj); nlu[r] |= 1 << 16; }
                }
                tr_start.push_back((int)tr_kj.size());
            }
        }
        c.part_lvl0.upload(part_lvl0, s); c.lvl_off.upload(lvl_off, s);
        c.low_start.upload(low_start, s); c.nlu.upload(nlu, s);
        c.tr_start.upload(tr_start, s); c.tr_kj.upload(tr_kj, s); c.tr_rj.upload(tr_rj, s);
        c.lu_col.upload(lu_col, s); c.lu_src.upload(lu_src, s);
        c.lu_slots = MS;
        if (o.ilu_bulk)
            build_task_records(c, o, nparts, part_lvl0, lvl_off, lu_col, lu_src, nlu, low_start, tr_start, tr_kj, tr_rj,
                               nl, nu, ML, MS);
    }
    // ---- AMG hierarchy: plan on the cell graph (original numbering), level
    // 0 in the internal row order; the Galerkin gather lists sum the finer
    // blocks in finer-row order, then by slot
    if (o.precon == PRECON_AMG) {
        std::vector<std::vector<int>> adj0(N);
        for (int f = 0; f < Fi; ++f) { adj0[mh->owner[f]].push_back(mh->neighbour[f]); adj0[mh->neighbour[f]].push_back(mh->owner[f]); }
        const AmgPlan P = amg_plan(adj0, o.amg_min_coarse, o.amg_max_levels);
        // finer-level slots per row: (column, slot id) with slot ids of the
        // SELL store on level 0, CSR positions on coarse levels
        std::vector<std::vector<std::pair<int, int>>> fine(N);
        for (int r = 0; r < N; ++r) {
            fine[r].push_back({r, flat(r, 0)});
            for (size_t k = 0; k < rowcols[r].size(); ++k) fine[r].push_back({rowcols[r][k], flat(r, 1 + (int)k)});
        }
        // level-0 node ids are internal rows; the plan's are original cells
        std::vector<int> node_of_row(c.perm);
        for (size_t l = 0; l < P.agg.size(); ++l) {
            auto L = std::make_unique<rdst_ctx::AmgDev>();
            const int nf = (int)fine.size(), nc = P.n[l + 1];
            const std::vector<int>& aggp = P.agg[l];          // plan node of level l -> level l+1
            std::vector<int> agg(nf);                         // this context's finer ids -> coarse
            for (int i = 0; i < nf; ++i) agg[i] = aggp[l == 0 ? node_of_row[i] : i];
            const auto& cadj = P.adj[l + 1];
            std::vector<int> start(nc + 1, 0), col, dslot(nc);
            for (int I = 0; I < nc; ++I) {
                std::vector<int> cols(cadj[I]);
                cols.push_back(I);
                std::sort(cols.begin(), cols.end());
                for (int cc : cols) {
                    if (cc == I) dslot[I] = (int)col.size();
                    col.push_back(cc);
                }
                start[I + 1] = (int)col.size();
            }
            const int nnz = (int)col.size();
            std::vector<std::vector<int>> lists(nnz);
            // finer rows in plan order (original cell order on level 0)
            std::vector<int> order(nf);
            for (int i = 0; i < nf; ++i) order[i] = i;
            if (l == 0) for (int i = 0; i < nf; ++i) order[i] = c.iperm[i];
            for (int i : order)
                for (auto& e : fine[i]) {
                    const int I = agg[i], J = agg[e.first];
                    const int sl = (int)(std::lower_bound(col.begin() + start[I], col.begin() + start[I + 1], J) -
                                         col.begin());
                    lists[sl].push_back(e.second);
                }
            std::vector<int> gstart(nnz + 1, 0), gsrc;
            for (int q = 0; q < nnz; ++q) {
                gsrc.insert(gsrc.end(), lists[q].begin(), lists[q].end());
                gstart[q + 1] = (int)gsrc.size();
            }
            std::vector<std::vector<int>> members(nc);
            for (int i : order) members[agg[i]].push_back(i);
            std::vector<int> mstart(nc + 1, 0), mem;
            for (int I = 0; I < nc; ++I) {
                mem.insert(mem.end(), members[I].begin(), members[I].end());
                mstart[I + 1] = (int)mem.size();
            }
            L->n = nc; L->nnz = nnz;
            L->start.upload(start, s); L->col.upload(col, s); L->dslot.upload(dslot, s);
            L->gstart.upload(gstart, s); L->gsrc.upload(gsrc, s);
            L->mstart.upload(mstart, s); L->mem.upload(mem, s); L->agg.upload(agg, s);
            L->val.alloc(25L * nnz); L->dinv.alloc(25L * nc);
            L->x.alloc(5L * nc); L->b.alloc(5L * nc); L->r.alloc(5L * nc);
            L->x.zero(s);
            c.amg.push_back(std::move(L));
            // this level's rows for the next: (column, CSR position)
            std::vector<std::vector<std::pair<int, int>>> next(nc);
            for (int I = 0; I < nc; ++I)
                for (int q = start[I]; q < start[I + 1]; ++q) next[I].push_back({col[q], q});
            fine.swap(next);
            CK(cudaStreamSynchronize(s));     // the host vectors of this level go out of scope
        }
        c.amg_r0.alloc(5L * N);
    }
    // ---- upload
    c.own.upload(own, s); c.nei.upload(nei, s);
    c.bcell.upload(bcell, s); c.bpatch.upload(bpatch, s);
    std::vector<int> bfo(c.bface_orig);
    c.bfaceD.upload(bfo, s);
    c.turb = (o.turbulence != TURB_LAMINAR);
    if (c.turb && !mh->wall_distance) throw std::invalid_argument("Spalart-Allmaras needs the wall distance field");
    load_geometry(c, mh, false);
    c.cf_start.upload(cf_start, s); c.cf_list.upload(cf_list, s); c.cf_slot.upload(cf_slot, s);
    c.cc_start.upload(cc_start, s); c.cc_list.upload(cc_list, s);
    c.patches.upload(dp, s);
    c.slice_off.upload(slice_off, s); c.slice_w.upload(slice_w, s); c.col.upload(col, s);
    DevMesh& m = c.m;
    m.N = N; m.Fi = Fi; m.NB = NB; m.n_patches = mh->n_patches;
    m.own = c.own.p; m.nei = c.nei.p; m.Sf = c.Sf.p; m.magSf = c.magSf.p; m.w = c.w.p; m.dc = c.dc.p;
    m.d = c.d.p; m.Cf = c.Cf.p;
    m.bcell = c.bcell.p; m.bpatch = c.bpatch.p; m.bface = c.bfaceD.p; m.bSf = c.bSf.p; m.bmagSf = c.bmagSf.p;
    m.bdc = c.bdc.p; m.bCf = c.bCf.p; m.V = c.V.p; m.C = c.C.p;
    m.cf_start = c.cf_start.p; m.cf_list = c.cf_list.p; m.cc_start = c.cc_start.p; m.cc_list = c.cc_list.p;
    m.patches = c.patches.p;
    // ---- fields
    c.perm_d.upload(c.perm, s); c.stage.alloc(5L * N);
    c.W.alloc(5L * N); c.prim.alloc((size_t)PW * N); c.bs.alloc((size_t)BW * std::max(NB, 1));
    c.bjac.alloc((size_t)25 * std::max(NB, 1));
    c.q.alloc((size_t)QW * N); c.qb.alloc((size_t)QW * std::max(NB, 1)); c.g.alloc((size_t)GW * N);
    c.psi.alloc((size_t)QW * N); c.fcell.alloc(N); c.fl.alloc(5L * std::max(Fi, 1)); c.bfl.alloc(5L * std::max(NB, 1));
    c.R.alloc(5L * N); c.rhs.alloc(5L * N);
    c.mut.alloc(N); c.mut.zero(s); c.mut_b.alloc(std::max(NB, 1)); c.mut_b.zero(s);
    if (c.turb) {
        const size_t nb1 = std::max(NB, 1), fi1 = std::max(Fi, 1);
        c.nut.alloc(N); c.nut.zero(s); c.nut_b.alloc(nb1); c.nut_b.zero(s);
        c.saD.alloc(N); c.safv1.alloc(N); c.sadiag.alloc(N); c.sab.alloc(N); c.sax2.alloc(N); c.sagn.alloc(3L * N);
        c.safup.alloc(fi1); c.saflo.alloc(fi1); c.safdP.alloc(fi1); c.safdQ.alloc(fi1); c.safcorr.alloc(fi1);
        c.sabd.alloc(nb1); c.sabb.alloc(nb1);
        c.saSold.alloc(6L * N); c.saSold.zero(s); c.saRho0.alloc(N); c.saRho0.zero(s);
        c.saSoldValid.alloc(1); c.saSoldValid.zero(s);
        SAFields& F = c.sa;
        F.nut = c.nut.p; F.nut_b = c.nut_b.p; F.mut = c.mut.p; F.mut_b = c.mut_b.p; F.y = c.ywall.p;
        F.D = c.saD.p; F.fv1 = c.safv1.p; F.diag = c.sadiag.p; F.b = c.sab.p; F.x2 = c.sax2.p; F.gn = c.sagn.p;
        F.fup = c.safup.p; F.flo = c.saflo.p; F.fdP = c.safdP.p; F.fdQ = c.safdQ.p; F.fcorr = c.safcorr.p;
        F.bd = c.sabd.p; F.bb = c.sabb.p;
        F.S_old = c.saSold.p; F.rho0 = c.saRho0.p; F.S_old_valid = c.saSoldValid.p;
    }
    if (c.tr.viscous) {
        c.gU.alloc(9L * N); c.up.alloc(3L * std::max(Fi, 1)); c.bup.alloc(3L * std::max(NB, 1));
        c.vf.alloc(8L * std::max(Fi, 1)); c.bvf.alloc(8L * std::max(NB, 1));
    }
    c.rdt.alloc(N); c.courantF.alloc(N); c.rhoOld.alloc(N); c.eOld.alloc(N); c.eNew.alloc(N);
    c.sc.alloc(1); c.sc.zero(s);
    c.reps.alloc(rdst_ctx::REP_CAP);
    int nbmax = std::max(nblk(std::max(N, Fi), TPB), red_blocks(5L * N));
    c.partial.alloc((size_t)std::max(nbmax, 1) * 72);
    c.bs.zero(s); c.W.zero(s); c.prim.zero(s); c.psi.zero(s); c.fcell.zero(s);
    // ---- matrix storage
    c.mt_size = o.precision == PREC_FP64 ? 8 : (o.precision == PREC_FP32 ? 4 : 2);
    size_t mbytes = (size_t)c.n_slots * 32 * 25 * c.mt_size;
    CK(cudaMalloc(&c.Aval, mbytes));
    CK(cudaMemsetAsync(c.Aval, 0, mbytes, s));
    if (factored) {
        size_t lbytes = (size_t)c.n_slices * c.lu_slots * 32 * 25 * c.mt_size;
        CK(cudaMalloc(&c.LUval, lbytes));
        CK(cudaMemsetAsync(c.LUval, 0, lbytes, s));
    }
    if (o.precon != PRECON_NONE) CK(cudaMalloc(&c.dinv, (size_t)c.n_slices * 32 * 25 * c.mt_size));
    if (c.rec_f.p) {
        if (o.precision == PREC_FP64) ilu_bulk_attr<double>(c);
        else if (o.precision == PREC_FP32) ilu_bulk_attr<float>(c);
        else ilu_bulk_attr<__nv_bfloat16>(c);
    }
    if (o.precon == PRECON_GAUSS_SEIDEL && o.n_sweeps > 1) { c.gs_r.alloc(5L * N); c.gs_z.alloc(5L * N); }
    // ---- Krylov
    const long n5 = 5L * N;
    c.dx.alloc(n5); c.r.alloc(n5); c.t.alloc(n5); c.Ax.alloc(n5); c.pA.alloc(n5); c.xbar.alloc(8);
    // basis vectors 64-entry aligned (the orthogonalisation reads 4 entries per 16-byte load)
    c.ldv = (n5 + 63) / 64 * 64;
    if (o.solver == SOLVER_GMRES && o.basis32) { c.Vf.alloc((size_t)(o.n_directions + 1) * c.ldv); c.wv.alloc(n5); }
    else if (o.solver == SOLVER_GMRES) c.Vb.alloc((size_t)(o.n_directions + 1) * c.ldv);
    else { c.s2.alloc(n5); c.sh.alloc(n5); c.ph.alloc(n5); c.pv.alloc(n5); c.Vb.alloc(2 * n5); }
    // limiter needs
    auto vk = [](Limiter l) { return l == LIM_VENKATAKRISHNAN; };
    c.venkat_mask = (vk(o.lim_rho) ? 1 : 0) | (vk(o.lim_U) ? 0xE : 0) | (vk(o.lim_T) ? 0x70 : 0);
    CK(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------- step pieces
// The bulk-copy apply (factor rows as records, one TMA copy per task):
// its dynamic shared memory is the stages, the lanes' y0 slots and the x
// ring when the context has one.
// the pack's shared memory: the widest side's slots (L, or U + pivot inverse)
template <typename MT>
static size_t ilu_pack_smem(const rdst_ctx& c) {
    return (size_t)(std::max(c.ilu_ml, c.ilu_mu) + 1) * ilu_pack_tile<MT>() * sizeof(MT);
}
template <typename MT>
static size_t ilu_bulk_smem(const rdst_ctx& c) {
    return (size_t)c.ilu_stages * c.ilu_stage_bytes + (size_t)c.ilu_stages * ILU_BULK_TPB * 8 +
           (size_t)c.ilu_lb_rows * (sizeof(MT) == 8 ? 96 : 64) + (size_t)c.ilu_task_slots * 8 +
           (size_t)c.ilu_off_slots * 4;
}
// A kernel's dynamic shared memory limit is a property of the function on
// the device, shared by every context of the process: it is raised to the
// device's per-block maximum less the kernel's static shared memory (never
// lowered to one context's need, which would fail the launches of a context
// built earlier with larger tasks).
template <typename K>
static void set_max_dyn_smem(K* kernel) {
    int dev = 0, per_block = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, kernel));
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, per_block - (int)fa.sharedSizeBytes));
}
template <typename MT, int NS, bool LB>
static void ilu_bulk_launch(rdst_ctx& c, bool attr_only, const IluDev& P, const double* in, double* out,
                            const int* active) {
    const size_t sm = ilu_bulk_smem<MT>(c);
    if (attr_only) {
        set_max_dyn_smem(k_ilu_apply_bulk<MT, NS, LB>);
        return;
    }
    k_ilu_apply_bulk<MT, NS, LB><<<c.n_parts, ILU_BULK_THREADS, sm, c.s>>>(P, in, out, active, c.ilu_lb_rows,
                                                                        c.ilu_stage_bytes, c.ilu_off_slots,
                                                                        c.ilu_task_slots, &c.sc.p->flags);
}
template <typename MT>
static void ilu_bulk_dispatch(rdst_ctx& c, bool attr_only, const IluDev& P, const double* in, double* out,
                              const int* active) {
    const bool lb = c.ilu_lb_rows > 0;
    if (c.ilu_stages == 3) {
        if (lb) ilu_bulk_launch<MT, 3, true>(c, attr_only, P, in, out, active);
        else ilu_bulk_launch<MT, 3, false>(c, attr_only, P, in, out, active);
    } else {
        if (lb) ilu_bulk_launch<MT, 2, true>(c, attr_only, P, in, out, active);
        else ilu_bulk_launch<MT, 2, false>(c, attr_only, P, in, out, active);
    }
}
// dynamic shared memory above the default 48 KB: set when a context is
// built (not while a step is being captured)
template <typename MT>
static void ilu_bulk_attr(rdst_ctx& c) {
    ilu_bulk_dispatch<MT>(c, true, c.ilu(), nullptr, nullptr, nullptr);
    set_max_dyn_smem(k_ilu_pack<MT>);
}
template <typename MT>
static void ilu_apply_bulk(rdst_ctx& c, const IluDev& P, const double* in, double* out, const int* active) {
    ilu_bulk_dispatch<MT>(c, false, P, in, out, active);
}
// blocks of the fresh factors -> the task records
template <typename MT>
static void ilu_pack(rdst_ctx& c, void* val) {
    if (!c.rec_f.p) return;
    k_ilu_pack<MT><<<c.n_slices, 256, ilu_pack_smem<MT>(c), c.s>>>(c.N, c.mat<MT>(val), (const MT*)c.LUval,
                                                                   (const MT*)c.dinv, c.ilu());
    CKL();
}

// block ILU factorisation of the matrix at val into the factor store:
// reading A directly when the descriptors were built, else gather + factor;
// then packed into the bulk apply's records when there are records
template <typename MT>
static void ilu_factorise(rdst_ctx& c, void* val) {
    if (c.ilu_direct) {
        k_ilu_factor_direct<MT><<<c.n_parts, 32, 0, c.s>>>(c.mat<MT>(val), (MT*)c.LUval, (MT*)c.dinv, c.ilu());
        CKL();
    } else {
        const int n_fid = c.n_slices * c.lu_slots * 32;
        k_ilu_gather<MT><<<nblk(n_fid, TPB), TPB, 0, c.s>>>(c.mat<MT>(val), (MT*)c.LUval, c.lu_src.p, n_fid);
        CKL();
        k_ilu_factor<MT><<<c.n_parts, c.o.ilu_factor_threads, 0, c.s>>>(c.mat<MT>(val), (MT*)c.LUval,
                                                                       (MT*)c.dinv, c.ilu());
        CKL();
    }
    ilu_pack<MT>(c, val);
}

template <typename MT>
struct Ops {
    static void flux(rdst_ctx& c) {
        const Options& o = c.o;
        cudaStream_t s = c.s;
        const DevMesh& m = c.m;
        int use_c = (o.flux == FLUX_KURGANOV || o.flux == FLUX_AUSM);
        const bool visc = c.tr.viscous != 0;
        k_recon<<<nblk(m.N + m.NB, TPB), TPB, 0, s>>>(m, c.th, c.tr, use_c, c.W.p, c.prim.p, c.bs.p, c.mut.p, c.mut_b.p,
                                                     c.q.p, c.qb.p);
        CKL();
        k_grad<<<nblk(m.N, 128), 128, 0, s>>>(m, c.venkat_mask, o.venkat_K, c.q.p, c.qb.p, c.prim.p, c.g.p, c.psi.p,
                                             c.fcell.p, o.flux == FLUX_HLLCP, c.bs.p, visc ? c.gU.p : nullptr);
        CKL();
        if (visc && o.grad_U_limit > 0) {
            k_limit_gradU<<<nblk(m.N, 128), 128, 0, s>>>(m, o.grad_U_limit, c.prim.p, c.bs.p, c.gU.p);
            CKL();
        }
        if (m.Fi > 0) {
            Timed tm(c, KS_FLUX);
            k_face_flux<<<nblk(m.Fi, 128), 128, 0, s>>>(m, c.th, flux_code(o.flux), lim_code(o.lim_rho), lim_code(o.lim_U),
                                                       lim_code(o.lim_T), o.low_mach, o.mainf, c.q.p, c.g.p, c.psi.p,
                                                       c.fcell.p, c.fl.p, visc ? c.up.p : nullptr);
            CKL();
        }
        if (m.NB > 0) {
            k_bface_flux<<<nblk(m.NB, 128), 128, 0, s>>>(m, c.th, flux_code(o.flux), o.low_mach, o.mainf, c.qb.p, c.bfl.p,
                                                        c.bs.p, visc ? c.bup.p : nullptr);
            CKL();
        }
        if (visc) {
            if (m.Fi > 0) {
                k_visc_faces<<<nblk(m.Fi, 128), 128, 0, s>>>(m, c.q.p, c.prim.p, c.gU.p, c.up.p, c.vf.p);
                CKL();
            }
            if (m.NB > 0) {
                k_visc_bfaces<<<nblk(m.NB, 128), 128, 0, s>>>(m, c.qb.p, c.prim.p, c.gU.p, c.bs.p, c.bup.p, c.bvf.p);
                CKL();
            }
        }
        int nb = nblk(m.N, TPB);
        k_residual<<<nb, TPB, 0, s>>>(m, c.fl.p, c.bfl.p, visc ? c.vf.p : nullptr, visc ? c.bvf.p : nullptr, c.R.p,
                                      c.rhs.p, c.partial.p);
        CKL();
        k_residual_finalize<<<1, RED_TPB, 0, s>>>(c.partial.p, nb, c.sc.p);
        CKL();
    }
    static void assemble(rdst_ctx& c) {
        SellMat<MT> A = c.mat<MT>(c.Aval);
        Timed tm(c, KS_ASSEMBLE);
        if (c.m.NB > 0) {
            k_bjac<<<nblk(c.m.NB, 128), 128, 0, c.s>>>(c.m, c.th, c.W.p, c.prim.p, c.bs.p, c.bjac.p);
            CKL();
        }
        k_assemble<MT><<<nblk(c.N, 128), 128, 0, c.s>>>(c.m, c.th, c.tr, A, c.cf_slot.p, c.W.p, c.prim.p, c.bjac.p,
                                                        c.rdt.p, c.mut.p, c.sc.p, (c.steady || c.o.dual) ? 1 : 0,
                                                        c.o.beta, c.dual_a);
        CKL();
        if (c.m.rmask) {
            k_hold_rows<MT><<<nblk(c.N, 128), 128, 0, c.s>>>(A, c.m.rmask);
            CKL();
        }
    }
    // AMG coarse levels of the matrix in Aval (the step's A, or A^T for the adjoint)
    static void amg_setup(rdst_ctx& c) {
        k_dinv<MT><<<nblk(c.N, 128), 128, 0, c.s>>>(c.mat<MT>(c.Aval), (MT*)c.dinv);
        CKL();
        for (size_t l = 0; l < c.amg.size(); ++l) {
            auto& L = *c.amg[l];
            const long t = 25L * L.nnz;
            if (l == 0)
                k_amg_gather_sell<MT><<<nblk(t, TPB), TPB, 0, c.s>>>(c.mat<MT>(c.Aval), L.gstart.p, L.gsrc.p, L.val.p,
                                                                     L.nnz);
            else
                k_amg_gather_csr<<<nblk(t, TPB), TPB, 0, c.s>>>(c.amg[l - 1]->val.p, L.gstart.p, L.gsrc.p, L.val.p,
                                                                L.nnz);
            CKL();
            k_amg_dinv<<<nblk(L.n, 128), 128, 0, c.s>>>(L.n, L.dslot.p, L.val.p, L.dinv.p);
            CKL();
        }
    }
    // r = b - A x and the damped block-Jacobi update on level l
    static void amg_resid(rdst_ctx& c, int l, const double* x, const double* b, double* r, const int* act) {
        if (l == 0) {
            k_spmv<MT, double><<<nblk(c.N, 256), 256, 0, c.s>>>(c.mat<MT>(c.Aval), x, r, b, act);
        } else {
            auto& L = *c.amg[l - 1];
            k_amg_resid<<<nblk(L.n, 128), 128, 0, c.s>>>(L.n, L.start.p, L.col.p, L.val.p, x, b, r, act);
        }
        CKL();
    }
    static void amg_jacobi(rdst_ctx& c, int l, const double* r, double* x, int zero, const int* act) {
        if (l == 0)
            k_amg_jacobi0<MT><<<nblk(c.N, 128), 128, 0, c.s>>>(c.N, (const MT*)c.dinv, r, x, c.o.amg_omega, zero, act);
        else {
            auto& L = *c.amg[l - 1];
            k_amg_jacobi<<<nblk(L.n, 128), 128, 0, c.s>>>(L.n, L.dinv.p, r, x, c.o.amg_omega, zero, act);
        }
        CKL();
    }
    // x = one V-cycle on level l from x = 0 (level 0: b = in, x = out)
    static void amg_vcycle(rdst_ctx& c, int l, const double* b, double* x, const int* act) {
        const int nl = (int)c.amg.size() + 1;
        const long n = l == 0 ? c.N : c.amg[l - 1]->n;
        double* r = l == 0 ? c.amg_r0.p : c.amg[l - 1]->r.p;
        if (l == nl - 1) {
            amg_jacobi(c, l, b, x, 1, act);
            for (int sw = 1; sw < c.o.amg_coarsest_sweeps; ++sw) {
                amg_resid(c, l, x, b, r, act);
                amg_jacobi(c, l, r, x, 0, act);
            }
            return;
        }
        bool zero = true;
        for (int sw = 0; sw < c.o.amg_pre; ++sw) {
            if (zero) amg_jacobi(c, l, b, x, 1, act);
            else { amg_resid(c, l, x, b, r, act); amg_jacobi(c, l, r, x, 0, act); }
            zero = false;
        }
        if (zero) { k_amg_zero<<<nblk(5 * n, TPB), TPB, 0, c.s>>>(5 * n, x, act); CKL(); }
        amg_resid(c, l, x, b, r, act);
        auto& C = *c.amg[l];
        k_amg_restrict<<<nblk(C.n, 128), 128, 0, c.s>>>(C.n, C.mstart.p, C.mem.p, r, C.b.p, act);
        CKL();
        amg_vcycle(c, l + 1, C.b.p, C.x.p, act);
        k_amg_prolong<<<nblk(n, 128), 128, 0, c.s>>>((int)n, C.agg.p, C.x.p, x, act);
        CKL();
        for (int sw = 0; sw < c.o.amg_post; ++sw) {
            amg_resid(c, l, x, b, r, act);
            amg_jacobi(c, l, r, x, 0, act);
        }
    }
    static void precond_setup(rdst_ctx& c) {
        if (c.o.precon == PRECON_DIAGONAL) {
            k_dinv<MT><<<nblk(c.N, 128), 128, 0, c.s>>>(c.mat<MT>(c.Aval), (MT*)c.dinv);
            CKL();
        } else if (c.o.precon == PRECON_AMG) {
            Timed tm(c, KS_FACTOR);
            amg_setup(c);
        } else if (lu_factored(c.o.precon)) {
            Timed tm(c, KS_FACTOR);
            ilu_factorise<MT>(c, c.Aval);
        }
    }
    // out = (L U)^-1 in with the stored factors
    static void lu_apply(rdst_ctx& c, const double* in, double* out, const int* active) {
        const int nb = std::max(c.ilu_ml, c.ilu_mu);
        const MT* LU = (const MT*)c.LUval;
        auto P = c.ilu();
        const MT* di = (const MT*)c.dinv;
        const int N = c.N;
        if (c.rec_f.p) {
            ilu_apply_bulk<MT>(c, P, in, out, active);
        } else {
            if (nb <= 2) k_ilu_apply<MT, 2><<<c.n_parts, ILU_APPLY_TPB, 0, c.s>>>(N, LU, di, P, in, out, active);
            else if (nb <= 3) k_ilu_apply<MT, 3><<<c.n_parts, ILU_APPLY_TPB, 0, c.s>>>(N, LU, di, P, in, out, active);
            else if (nb <= 4) k_ilu_apply<MT, 4><<<c.n_parts, ILU_APPLY_TPB, 0, c.s>>>(N, LU, di, P, in, out, active);
            else if (nb <= 6) k_ilu_apply<MT, 6><<<c.n_parts, ILU_APPLY_TPB, 0, c.s>>>(N, LU, di, P, in, out, active);
            else if (nb <= 8) k_ilu_apply<MT, 8><<<c.n_parts, ILU_APPLY_TPB, 0, c.s>>>(N, LU, di, P, in, out, active);
            else k_ilu_apply<MT, 16><<<c.n_parts, ILU_APPLY_TPB, 0, c.s>>>(N, LU, di, P, in, out, active);
        }
        CKL();
    }
    static void precond(rdst_ctx& c, const double* in, double* out, const int* active) {
        Timed tm(c, KS_PRECOND);
        if (c.o.precon == PRECON_DIAGONAL) {
            k_jacobi<MT><<<nblk(c.N, 128), 128, 0, c.s>>>(c.N, (const MT*)c.dinv, in, out, active);
            CKL();
        } else if (c.o.precon == PRECON_AMG) {
            amg_vcycle(c, 0, in, out, active);
        } else if (lu_factored(c.o.precon)) {
            lu_apply(c, in, out, active);
            // further Gauss-Seidel sweeps: out += (D + L)^-1 (in - A out)
            for (int sw = 1; c.o.precon == PRECON_GAUSS_SEIDEL && sw < c.o.n_sweeps; ++sw) {
                k_spmv<MT, double><<<nblk(c.N, 256), 256, 0, c.s>>>(c.mat<MT>(c.Aval), out, c.gs_r.p, in, active);
                CKL();
                lu_apply(c, c.gs_r.p, c.gs_z.p, active);
                k_vadd<<<nblk(c.nvec(), TPB), TPB, 0, c.s>>>(c.nvec(), c.gs_z.p, out, active);
                CKL();
            }
        } else {
            k_copy_identity<MT><<<nblk(c.nvec(), TPB), TPB, 0, c.s>>>((int)c.nvec(), in, out, active);
            CKL();
        }
    }
    template <typename XT>
    static void spmv(rdst_ctx& c, const XT* x, double* y, const double* b, const int* active) {
        Timed tm(c, KS_SPMV);
        k_spmv<MT, XT><<<nblk(c.N, 256), 256, 0, c.s>>>(c.mat<MT>(c.Aval), x, y, b, active);
        CKL();
    }
    // normFactor + initial residual (dx = 0 -> r = rhs)
    static void solve_init(rdst_ctx& c) {
        cudaStream_t s = c.s;
        const int N = c.N;
        int nb = red_blocks(N);
        if (c.o.dependent_W) {
            spmv(c, c.W.p, c.Ax.p, nullptr, nullptr);
            k_sum5<<<nb, RED_TPB, 0, s>>>(N, c.W.p, c.partial.p); CKL();
            k_mean5_finalize<<<1, RED_TPB, 0, s>>>(c.partial.p, nb, N, c.xbar.p); CKL();
            k_spmv_const<MT><<<nblk(N, 256), 256, 0, s>>>(c.mat<MT>(c.Aval), c.xbar.p, c.pA.p); CKL();
        }
        k_normfactor<<<nb, RED_TPB, 0, s>>>(N, c.Ax.p, c.rhs.p, c.pA.p, c.o.dependent_W ? 1 : 0, c.partial.p); CKL();
        k_nf_finalize<<<1, RED_TPB, 0, s>>>(c.partial.p, nb, c.sc.p); CKL();
        k_abs5<<<nb, RED_TPB, 0, s>>>(N, c.rhs.p, c.partial.p); CKL();
        k_linres_finalize<<<1, RED_TPB, 0, s>>>(c.partial.p, nb, c.sc.p, 1); CKL();
        CK(cudaMemsetAsync(c.dx.p, 0, sizeof(double) * c.nvec(), s));
        CK(cudaMemsetAsync(&c.sc.p->lin_iterations, 0, sizeof(int), s));
        k_check<<<1, 1, 0, s>>>(c.sc.p, c.o.tolerance, c.o.rel_tol, c.o.min_iter, c.o.max_iter, 0); CKL();
        if (c.o.solver == SOLVER_BICGSTAB) {
            CK(cudaMemcpyAsync(c.r.p, c.rhs.p, sizeof(double) * c.nvec(), cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(c.Vb.p, c.rhs.p, sizeof(double) * c.nvec(), cudaMemcpyDeviceToDevice, s));  // rw
            c.pv.zero(s);
            CK(cudaMemsetAsync(c.ph.p, 0, sizeof(double) * c.nvec(), s));
            k_bi_init<<<1, 1, 0, s>>>(c.sc.p); CKL();
        } else if (c.o.solver != SOLVER_GMRES) {
            CK(cudaMemcpyAsync(c.r.p, c.rhs.p, sizeof(double) * c.nvec(), cudaMemcpyDeviceToDevice, s));
        }
    }
    static void dot(rdst_ctx& c, const double* a, const double* b, double* out, int sq, const int* active) {
        long n = c.nvec();
        int nb = red_blocks(n);
        k_multidot<<<nb, RED_TPB, 0, c.s>>>(n, 1, a, 0, b, c.partial.p, 8, active); CKL();
        k_finalize<<<1, RED_TPB, 0, c.s>>>(c.partial.p, nb, 1, 8, out, sq, active); CKL();
    }
    // V^T w (one pass over w) into out[0..nv)
    template <int NV, typename VT>
    static void vmultidot(rdst_ctx& c, const VT* V, int nv, const double* w, double* out, const int* active) {
        long n = c.nvec();
        int nb = red_blocks(n);
        k_vmultidot<NV, VT><<<nb, RED_TPB, 0, c.s>>>(n, nv, V, c.ldv, w, c.partial.p, 64, active); CKL();
        k_finalize<<<nv, RED_TPB, 0, c.s>>>(c.partial.p, nb, nv, 64, out, 0, active); CKL();
    }
    // w -= V coef, fused with the next dots (mode 0) or the norm (mode 1)
    template <int NV, typename VT>
    static void maxpy_dot(rdst_ctx& c, const VT* V, int nv, const double* coef, double* w, double* out, int mode,
                          const int* active) {
        long n = c.nvec();
        int nb = red_blocks(n);
        k_maxpy_dot<NV, VT><<<nb, RED_TPB, 0, c.s>>>(n, nv, V, c.ldv, coef, w, c.partial.p, 64, mode, active); CKL();
        if (mode == 0) { k_finalize<<<nv, RED_TPB, 0, c.s>>>(c.partial.p, nb, nv, 64, out, 0, active); CKL(); }
        else { k_finalize<<<1, RED_TPB, 0, c.s>>>(c.partial.p, nb, 1, 64, out, 1, active); CKL(); }
    }
    // CGS2 orthogonalisation of w against V_0..V_i: H[:,i] pieces, beta = |w|
    template <int NV, typename VT>
    static void orth(rdst_ctx& c, const VT* V, int nv, double* w, const int* act) {
        Scalars* sc = c.sc.p;
        vmultidot<NV, VT>(c, V, nv, w, sc->hcol[0], act);
        maxpy_dot<NV, VT>(c, V, nv, sc->hcol[0], w, sc->hcol[1], 0, act);
        maxpy_dot<NV, VT>(c, V, nv, sc->hcol[1], w, &sc->beta, 1, act);
    }
    // One restart cycle of left-preconditioned GMRES(m) with CGS2.  With an
    // FP64 basis each Arnoldi vector is built in place in its basis slot;
    // with an FP32 basis it is built and orthogonalised in the FP64 vector
    // wv (dots, Hessenberg and Givens stay FP64) and stored normalised.
    template <typename VT>
    static void gmres_cycle_t(rdst_ctx& c, VT* Vb) {
        constexpr bool in_place = std::is_same<VT, double>::value;
        cudaStream_t s = c.s;
        const long n = c.nvec();
        const int m = c.o.n_directions;
        Scalars* sc = c.sc.p;
        int* act = &sc->gm_active;
        double* w0 = in_place ? (double*)Vb : c.wv.p;
        spmv(c, c.dx.p, c.r.p, c.rhs.p, nullptr);            // r = rhs - A dx
        precond(c, c.r.p, w0, nullptr);                      // w = M^-1 r
        dot(c, w0, w0, &sc->beta, 1, nullptr);
        k_gm_start<<<1, 1, 0, s>>>(sc); CKL();
        if (in_place) { k_scale_inv<<<nblk(n, TPB), TPB, 0, s>>>(n, w0, &sc->beta, act); CKL(); }
        else { k_scale_store<VT><<<nblk(n, TPB), TPB, 0, s>>>(n, w0, Vb, &sc->beta, act); CKL(); }
        for (int i = 0; i < m; ++i) {
            const VT* Vi = Vb + i * c.ldv;
            double* w = in_place ? (double*)(Vb + (i + 1) * c.ldv) : c.wv.p;
            spmv(c, Vi, c.t.p, nullptr, act);
            precond(c, c.t.p, w, act);
            {
                Timed tm(c, KS_ORTH);
                const int nv = i + 1;
                if (nv <= 8) orth<8, VT>(c, Vb, nv, w, act);
                else if (nv <= 16) orth<16, VT>(c, Vb, nv, w, act);
                else if (nv <= 32) orth<32, VT>(c, Vb, nv, w, act);
                else orth<64, VT>(c, Vb, nv, w, act);
            }
            k_gm_givens<<<1, 1, 0, s>>>(sc, i, m); CKL();
            if (i < m - 1) {
                if (in_place) { k_scale_inv<<<nblk(n, TPB), TPB, 0, s>>>(n, w, &sc->beta, act); CKL(); }
                else { k_scale_store<VT><<<nblk(n, TPB), TPB, 0, s>>>(n, w, Vb + (i + 1) * c.ldv, &sc->beta, act); CKL(); }
            }
        }
        k_gm_backsub<<<1, 1, 0, s>>>(sc, m); CKL();
        k_maxpy<VT><<<nblk(n, TPB), TPB, 0, s>>>(n, m, Vb, c.ldv, sc->yh, c.dx.p, -1.0, nullptr); CKL();
        finish_iteration(c);
    }
    static void gmres_cycle(rdst_ctx& c) {
        if (c.o.basis32) gmres_cycle_t<float>(c, c.Vf.p);
        else gmres_cycle_t<double>(c, c.Vb.p);
    }
    static void finish_iteration(rdst_ctx& c) {
        spmv(c, c.dx.p, c.r.p, c.rhs.p, nullptr);
        int nb = red_blocks(c.N);
        k_abs5<<<nb, RED_TPB, 0, c.s>>>(c.N, c.r.p, c.partial.p); CKL();
        k_linres_finalize<<<1, RED_TPB, 0, c.s>>>(c.partial.p, nb, c.sc.p, 0); CKL();
        k_check<<<1, 1, 0, c.s>>>(c.sc.p, c.o.tolerance, c.o.rel_tol, c.o.min_iter, c.o.max_iter, 1); CKL();
    }
    // one BiCGStab iteration (van der Vorst, right preconditioned)
    static void bicgstab_iter(rdst_ctx& c) {
        cudaStream_t s = c.s;
        const long n = c.nvec();
        Scalars* sc = c.sc.p;
        double* rw = c.Vb.p;
        double* t2 = c.Vb.p + n;
        dot(c, rw, c.r.p, &sc->hcol[0][0], 0, nullptr);
        k_bi_scal_rho<<<1, 1, 0, s>>>(sc); CKL();
        k_bi_p<<<nblk(n, TPB), TPB, 0, s>>>(n, c.r.p, c.pv.p, c.t.p, sc); CKL();      // t holds p
        precond(c, c.t.p, c.ph.p, nullptr);
        spmv(c, c.ph.p, c.pv.p, nullptr, nullptr);                                  // v = A ph
        dot(c, rw, c.pv.p, &sc->hcol[0][0], 0, nullptr);
        k_bi_scal_alpha<<<1, 1, 0, s>>>(sc); CKL();
        k_bi_s<<<nblk(n, TPB), TPB, 0, s>>>(n, c.r.p, c.pv.p, c.s2.p, sc); CKL();
        precond(c, c.s2.p, c.sh.p, nullptr);
        spmv(c, c.sh.p, t2, nullptr, nullptr);
        dot(c, t2, t2, &sc->hcol[0][0], 0, nullptr);
        dot(c, t2, c.s2.p, &sc->hcol[0][1], 0, nullptr);
        k_bi_scal_omega<<<1, 1, 0, s>>>(sc); CKL();
        k_bi_update<<<nblk(n, TPB), TPB, 0, s>>>(n, c.dx.p, c.r.p, c.ph.p, c.sh.p, c.s2.p, t2, sc); CKL();
        int nb = red_blocks(c.N);
        k_abs5<<<nb, RED_TPB, 0, s>>>(c.N, c.r.p, c.partial.p); CKL();
        k_linres_finalize<<<1, RED_TPB, 0, s>>>(c.partial.p, nb, sc, 0); CKL();
        k_check<<<1, 1, 0, s>>>(sc, c.o.tolerance, c.o.rel_tol, c.o.min_iter, c.o.max_iter, 1); CKL();
    }
    // one stationary iteration dx += M^-1 (rhs - A dx) (Gauss-Seidel sweeps
    // or the Cholesky-type factorisation), then the residual check
    static void stationary_iter(rdst_ctx& c) {
        precond(c, c.r.p, c.t.p, nullptr);
        k_vadd<<<nblk(c.nvec(), TPB), TPB, 0, c.s>>>(c.nvec(), c.t.p, c.dx.p, nullptr);
        CKL();
        finish_iteration(c);
    }
    static void iteration(rdst_ctx& c) {
        if (c.o.solver == SOLVER_GMRES) gmres_cycle(c);
        else if (c.o.solver == SOLVER_BICGSTAB) bicgstab_iter(c);
        else stationary_iter(c);
    }
};

void set_steady_dt(rdst_ctx& c) {
    int nb = nblk(c.N, TPB);
    k_dt_steady<<<nb, TPB, 0, c.s>>>(c.m, c.th, c.o.neighbouring, c.prim.p, c.dS.p, c.courantF.p, c.sc.p, c.rdt.p,
                                     c.partial.p);
    CKL();
    k_rdt_finalize<<<1, RED_TPB, 0, c.s>>>(c.partial.p, nb, c.sc.p);
    CKL();
}

void set_transient_dt(rdst_ctx& c) {
    long n = c.o.neighbouring ? c.Fi : c.N;
    int nb = nblk(n, TPB);
    k_dt_transient<<<nb, TPB, 0, c.s>>>(c.m, c.th, c.o.neighbouring, c.prim.p, c.dS.p, c.sc.p, c.partial.p);
    CKL();
    k_dt_finalize<<<1, RED_TPB, 0, c.s>>>(c.partial.p, nb, c.sc.p);
    CKL();
}

// Spalart-Allmaras transport (SAneg / SARC1 / SARC2), segregated
void sa_correct(rdst_ctx& c) {
    cudaStream_t s = c.s;
    const DevMesh& m = c.m;
    const int neg_sa = c.o.turbulence == TURB_SANEG;
    SAFields F = c.sa;
    k_sa_grad<<<nblk(c.N, 128), 128, 0, s>>>(m, c.prim.p, c.bs.p, F, c.gU.p); CKL();
    if (c.o.grad_U_limit > 0) {
        k_limit_gradU<<<nblk(c.N, 128), 128, 0, s>>>(m, c.o.grad_U_limit, c.prim.p, c.bs.p, c.gU.p); CKL();
    }
    const int sarc1 = c.o.turbulence == TURB_SARC1 ? 1 : (c.o.turbulence == TURB_SA ? 2 : 0);
    F.S_o = nullptr;
    if (sarc1 == 1 && c.o.dual && c.dual_a != 0.0) {
        // Sxx_ = S.component(..) (SARC1.C:655-669) at a new time index stores
        // the old times first (GeometricField::storeOldTimes): S_oo <- S_o,
        // S_o <- S (the last update's S, in saSold)
        const size_t n6 = 6 * (size_t)c.N * sizeof(double);
        if (!c.saSo.p) { c.saSo.alloc(6L * c.N); c.saSoo.alloc(6L * c.N); }
        if (c.sa_o_idx >= 0 && c.sa_S_idx != c.dual_tidx) {
            if (c.sa_oo_idx >= 0) {
                CK(cudaMemcpyAsync(c.saSoo.p, c.saSo.p, n6, cudaMemcpyDeviceToDevice, s));
                c.sa_oo_idx = c.sa_o_idx;
            }
            CK(cudaMemcpyAsync(c.saSo.p, c.saSold.p, n6, cudaMemcpyDeviceToDevice, s));
            c.sa_o_idx = c.sa_S_idx;
        }
        c.sa_S_idx = c.dual_tidx;
        // fvc::ddt creates S.oldTime() from S and its oldTime() from that at first use
        F.o_new = c.sa_o_idx < 0;
        if (F.o_new) c.sa_o_idx = c.sa_S_idx;
        F.oo_new = c.sa_oo_idx < 0;
        if (F.oo_new) c.sa_oo_idx = c.sa_o_idx;
        // dual2ndDST::fvcDdt(rho, vf) (dual2ndDST.C:231-372); deltaT0_(vf)
        // (:76-90) is GREAT while both old times carry one time index
        const double dt = c.dual_dt, dt0 = (c.sa_o_idx == c.sa_oo_idx) ? 1.0e15 : c.dual_dt0;
        F.d_rdt = 1.0 / dt;
        F.d_c = 1 + dt / (dt + dt0);
        F.d_c00 = dt * dt / (dt0 * (dt + dt0));
        F.d_c0 = F.d_c + F.d_c00;
        F.S_o = c.saSo.p;
        F.S_oo = c.saSoo.p;
        F.W_o = c.dWn.p;
        F.W_oo = c.dWnm1.p;
    }
    k_sa_cell<<<nblk(c.N, 128), 128, 0, s>>>(m, c.tr, neg_sa, sarc1, (c.steady || c.o.dual) ? 1 : 0, c.W.p, c.prim.p,
                                            c.gU.p, c.rdt.p, c.sc.p, c.fl.p, c.bs.p, F); CKL();
    if (c.o.dual && c.dual_a != 0.0) {
        k_sa_dual<<<nblk(c.N, TPB), TPB, 0, s>>>(c.N, c.V.p, c.W.p, c.dWn.p, c.dWnm1.p, c.nutN.p, c.nutNm1.p,
                                                 c.dual_a, c.dual_b, c.dual_c, F); CKL();
    }
    if (sarc1 == 1) { k_sarc1_valid<<<1, 1, 0, s>>>(F.S_old_valid); CKL(); }
    if (m.Fi > 0) { k_sa_faces<<<nblk(m.Fi, TPB), TPB, 0, s>>>(m, c.fl.p, F, c.o.nut_linear_upwind ? 1 : 0); CKL(); }
    if (m.NB > 0) { k_sa_bfaces<<<nblk(m.NB, TPB), TPB, 0, s>>>(m, c.tr, neg_sa, c.bs.p, F); CKL(); }
    k_sa_assemble<<<nblk(c.N, TPB), TPB, 0, s>>>(m, c.o.nut_relax, F); CKL();
    // Jacobi sweeps from the current nuTilda, ping-pong nut <-> x2
    double* xin = c.nut.p;
    double* xout = c.sax2.p;
    for (int it = 0; it < c.o.nut_sweeps; ++it) {
        k_sa_jacobi<<<nblk(c.N, TPB), TPB, 0, s>>>(m, F, xin, xout); CKL();
        std::swap(xin, xout);
    }
    k_sa_finish<<<nblk(c.N, TPB), TPB, 0, s>>>(c.N, neg_sa, c.W.p, xin, F); CKL();
    if (m.NB > 0) {
        k_sa_bc<<<nblk(m.NB, TPB), TPB, 0, s>>>(m, c.bs.p, F); CKL();
        k_sa_mutb<<<nblk(m.NB, TPB), TPB, 0, s>>>(m, c.tr, c.bs.p, F); CKL();
    }
}

// updateFields.H + turbulence + setCourantDST
void post_update(rdst_ctx& c) {
    cudaStream_t s = c.s;
    {
        Timed tm(c, KS_UPDATE);
        if (c.turb && c.o.turbulence == TURB_SARC1) {      // rho.oldTime() of the turbulence update
            k_sarc1_rho0<<<nblk(c.N, TPB), TPB, 0, s>>>(c.N, c.W.p, c.saRho0.p); CKL();
        }
        k_update<<<nblk(c.N, TPB), TPB, 0, s>>>(c.N, c.th, c.bd, c.dx.p, c.W.p, c.prim.p, c.sc.p); CKL();
    }
    k_boundary<<<nblk(c.NB, TPB), TPB, 0, s>>>(c.m, c.th, c.bd, c.W.p, c.prim.p, c.bs.p); CKL();
    if (c.turb && !c.o.frozen_turbulence) sa_correct(c);   // turbulence_.correct(); frozen: mu_t held
    k_courant_scalar<<<1, 1, 0, s>>>(c.sc.p, (!c.steady && c.o.adjust_time_step) ? 1 : 0, c.o.min_co, c.o.max_co); CKL();
    if (c.steady) {
        k_courant_cells<<<nblk(c.N, TPB), TPB, 0, s>>>(c.m, c.W.p, c.rhoOld.p, c.eOld.p, c.courantF.p, c.sc.p,
                                                      c.o.min_co, c.o.max_co, c.eNew.p); CKL();
        k_store_old<<<nblk(c.N, TPB), TPB, 0, s>>>(c.N, c.W.p, c.eNew.p, c.rhoOld.p, c.eOld.p); CKL();
        set_steady_dt(c);
    } else if (c.o.adjust_time_step) {
        set_transient_dt(c);
    }
}

__global__ void k_init_time(int N, const double* __restrict__ prim, Thermo th, double* __restrict__ rhoOld,
                            double* __restrict__ eOld, double* __restrict__ courantF, double co) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    rhoOld[i] = prim[PW * i] / (th.R * prim[PW * i + 1]);
    eOld[i] = prim[PW * i + 2] * th.Cv / th.Cp;
    courantF[i] = co;
}

__global__ void k_init_scalars(Scalars* sc, double time, double dt, double co) {
    if (threadIdx.x != 0) return;
    sc->time = time;
    sc->deltaT = dt;
    sc->courant = co;
    sc->residual = -1;
    sc->residualRatio = 1;
    sc->flags = 0;
}

// timeDST::initialize (timeDST.C:67-208) on the freshly set state
void initialize_time(rdst_ctx& c) {
    k_init_time<<<nblk(c.N, TPB), TPB, 0, c.s>>>(c.N, c.prim.p, c.th, c.rhoOld.p, c.eOld.p, c.courantF.p, c.o.initial_co);
    CKL();
    k_init_scalars<<<1, 1, 0, c.s>>>(c.sc.p, c.o.start_time, c.o.delta_t, c.o.initial_co);
    CKL();
    if (c.steady) set_steady_dt(c);
    else {
        set_transient_dt(c);          // unconditional in timeDST::initialize (timeDST.C:196-205)
        set_steady_dt(c);
    }
}

template <typename MT>
void pre_solve(rdst_ctx& c) {
    k_time_advance<<<1, 1, 0, c.s>>>(c.sc.p);
    CKL();
    Ops<MT>::flux(c);
    Ops<MT>::assemble(c);
    Ops<MT>::precond_setup(c);
    Ops<MT>::solve_init(c);
}

template <typename MT>
void iterations_direct(rdst_ctx& c) {
    const Options& o = c.o;
    int conv = 0;
    const bool fixed = (o.min_iter >= o.max_iter);
    if (!fixed && o.min_iter == 0) {
        CK(cudaMemcpyAsync(&conv, &c.sc.p->converged, sizeof(int), cudaMemcpyDeviceToHost, c.s));
        CK(cudaStreamSynchronize(c.s));
    }
    for (int it = 1; !conv && it <= o.max_iter; ++it) {
        Ops<MT>::iteration(c);
        if (it >= o.max_iter) break;
        if (it >= o.min_iter) {
            CK(cudaMemcpyAsync(&conv, &c.sc.p->converged, sizeof(int), cudaMemcpyDeviceToHost, c.s));
            CK(cudaStreamSynchronize(c.s));
        }
    }
}

template <typename MT>
void step_head(rdst_ctx& c) {
    k_report_dt<<<1, 1, 0, c.s>>>(c.sc.p, c.reps.p, rdst_ctx::REP_CAP);
    CKL();
    pre_solve<MT>(c);
}

void step_tail(rdst_ctx& c) {
    post_update(c);
    if (c.steady) {
        const int nb = red_blocks(c.N);
        k_mean_courant_partial<<<nb, RED_TPB, 0, c.s>>>(c.courantF.p, c.N, c.partial.p); CKL();
        k_mean_courant<<<1, RED_TPB, 0, c.s>>>(c.partial.p, nb, c.N, c.sc.p, c.reps.p, rdst_ctx::REP_CAP); CKL();
    }
    k_report<<<1, 1, 0, c.s>>>(c.sc.p, c.reps.p, rdst_ctx::REP_CAP);
    CKL();
}

template <typename Fn>
void capture(rdst_ctx& c, rdst_ctx::Graph& g, Fn&& body) {
    cudaGraph_t graph = nullptr;
    long l0 = c.launches;
    c.capturing = true;
    c.capture_events = &g.events;
    CK(cudaStreamBeginCapture(c.s, cudaStreamCaptureModeThreadLocal));
    try {
        body();
    } catch (...) {
        cudaStreamEndCapture(c.s, &graph);
        if (graph) cudaGraphDestroy(graph);
        c.capturing = false;
        throw;
    }
    CK(cudaStreamEndCapture(c.s, &graph));
    c.capturing = false;
    CK(cudaGraphInstantiate(&g.exec, graph, 0));
    CK(cudaGraphDestroy(graph));
    g.launches = c.launches - l0;
    c.launches = l0;
}

void launch_graph(rdst_ctx& c, rdst_ctx::Graph& g) {
    CK(cudaGraphLaunch(g.exec, c.s));
    c.launches += g.launches;
}

template <typename MT>
void run_steps(rdst_ctx& c, int n, rdst_step_report* host_reps) {
    cudaStream_t s = c.s;
    const Options& o = c.o;
    const bool fixed = (o.min_iter >= o.max_iter);
    if (!c.step_ev[0]) { CK(cudaEventCreate(&c.step_ev[0])); CK(cudaEventCreate(&c.step_ev[1])); }
    if (o.graphs) {
        if (fixed && !c.g_step.exec)
            capture(c, c.g_step, [&] {
                step_head<MT>(c);
                for (int it = 1; it <= o.max_iter; ++it) Ops<MT>::iteration(c);
                step_tail(c);
            });
        if (!fixed && !c.g_pre.exec) {
            capture(c, c.g_pre, [&] { step_head<MT>(c); });
            capture(c, c.g_cycle, [&] { Ops<MT>::iteration(c); });
            capture(c, c.g_post, [&] { step_tail(c); });
        }
    }
    int done = 0;
    double total_ms = 0;
    while (done < n) {
        const int chunk = std::min(n - done, rdst_ctx::REP_CAP);
        CK(cudaMemsetAsync(&c.sc.p->step_idx, 0, sizeof(int), s));
        CK(cudaEventRecord(c.step_ev[0], s));
        for (int st = 0; st < chunk; ++st) {
            if (!o.graphs) {
                step_head<MT>(c);
                iterations_direct<MT>(c);
                step_tail(c);
            } else if (fixed) {
                launch_graph(c, c.g_step);
                if (o.profile) { CK(cudaStreamSynchronize(s)); c.collect_graph_events(c.g_step); }
            } else {
                launch_graph(c, c.g_pre);
                if (o.profile) { CK(cudaStreamSynchronize(s)); c.collect_graph_events(c.g_pre); }
                int conv = 0;
                if (o.min_iter == 0) {
                    CK(cudaMemcpyAsync(&conv, &c.sc.p->converged, sizeof(int), cudaMemcpyDeviceToHost, s));
                    CK(cudaStreamSynchronize(s));
                }
                for (int it = 1; !conv && it <= o.max_iter; ++it) {
                    launch_graph(c, c.g_cycle);
                    if (o.profile) { CK(cudaStreamSynchronize(s)); c.collect_graph_events(c.g_cycle); }
                    if (it >= o.max_iter) break;
                    if (it >= o.min_iter) {
                        CK(cudaMemcpyAsync(&conv, &c.sc.p->converged, sizeof(int), cudaMemcpyDeviceToHost, s));
                        CK(cudaStreamSynchronize(s));
                    }
                }
                launch_graph(c, c.g_post);
                if (o.profile) { CK(cudaStreamSynchronize(s)); c.collect_graph_events(c.g_post); }
            }
        }
        CK(cudaEventRecord(c.step_ev[1], s));
        if (host_reps)
            CK(cudaMemcpyAsync(host_reps + done, c.reps.p, sizeof(rdst_step_report) * chunk, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, c.step_ev[0], c.step_ev[1]));
        total_ms += ms;
        done += chunk;
    }
    c.last_step_ms = total_ms;
    int flags = 0;
    CK(cudaMemcpyAsync(&flags, &c.sc.p->flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    c.collect_events();
    if (flags & 4) throw TimeoutError("a bounded wait of the ILU apply expired (bulk copy not completed)");
    if (flags & 2) throw std::domain_error("non-physical state (NaN or non-positive rho/p) after the update");
}

// residualControls + steadyCheck (residualControls.C:70-82,
// steadyCheck.C:69-98): mean of the five normalised initial residuals of
// each inner solve; converged after maxInnerIter iterations, below
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

// Dual::iterate (Dual.C:80-124), one physical time step per report: inner
// pseudo-time iterations of the coupled system with the dual2ndDST ddt until
// the steadyCheck converges, then the physical time-step control.  The
// inner-loop decisions are the host's, so the launches are direct.
template <typename MT>
void run_dual_steps(rdst_ctx& c, int n, rdst_step_report* host_reps) {
    cudaStream_t s = c.s;
    const Options& o = c.o;
    const long n5 = 5L * c.N;
    if (!c.dWn.p) { c.dWn.alloc(n5); c.dWnm1.alloc(n5); }
    if (c.turb && !c.nutN.p) { c.nutN.alloc(c.N); c.nutNm1.alloc(c.N); }
    if (!c.step_ev[0]) { CK(cudaEventCreate(&c.step_ev[0])); CK(cudaEventCreate(&c.step_ev[1])); }
    std::vector<int> inner_counts;
    int done = 0;
    double total_ms = 0;
    while (done < n) {
        const int chunk = std::min(n - done, rdst_ctx::REP_CAP);
        CK(cudaMemsetAsync(&c.sc.p->step_idx, 0, sizeof(int), s));
        CK(cudaEventRecord(c.step_ev[0], s));
        for (int st = 0; st < chunk; ++st) {
            // runTime++: deltaT0 = deltaTSave, deltaTSave = deltaT
            double dt = 0;
            CK(cudaMemcpyAsync(&dt, &c.sc.p->deltaT, sizeof(double), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            const double dt0 = c.dt_save;
            c.dt_save = dt;
            c.dual_dt = dt;
            c.dual_dt0 = dt0;
            ++c.dual_tidx;
            // old time levels (created from the current field at first use)
            if (!c.dual_started) {
                CK(cudaMemcpyAsync(c.dWn.p, c.W.p, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
                CK(cudaMemcpyAsync(c.dWnm1.p, c.W.p, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
                if (c.turb) {
                    CK(cudaMemcpyAsync(c.nutN.p, c.nut.p, c.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
                    CK(cudaMemcpyAsync(c.nutNm1.p, c.nut.p, c.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
                }
                c.sa_S_idx = c.sa_o_idx = c.sa_oo_idx = -1;   // SARC1's S history restarts too
                c.dual_started = true;
            } else {
                std::swap(c.dWn.p, c.dWnm1.p);
                CK(cudaMemcpyAsync(c.dWn.p, c.W.p, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
                if (c.turb) {
                    std::swap(c.nutN.p, c.nutNm1.p);
                    CK(cudaMemcpyAsync(c.nutN.p, c.nut.p, c.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
                }
            }
            // dual2ndDST::fvmDdt coefficients (dual2ndDST.C:391-395)
            const double a = 1.0 / dt + 1.0 / (dt + dt0);
            const double cc = dt / (dt0 * (dt + dt0));
            const double b = -(a + cc);
            c.dual_a = a;
            c.dual_b = b;
            c.dual_c = cc;
            const bool sa = c.turb && !o.frozen_turbulence;
            k_report_dt<<<1, 1, 0, s>>>(c.sc.p, c.reps.p, rdst_ctx::REP_CAP); CKL();
            k_time_advance<<<1, 1, 0, s>>>(c.sc.p); CKL();
            SteadyCheck rc(o);
            int inner = 0;
            do {
                Ops<MT>::flux(c);
                Ops<MT>::assemble(c);
                k_dual_source<<<nblk(c.N, TPB), TPB, 0, s>>>(c.N, c.V.p, c.W.p, c.rdt.p, c.dWn.p, c.dWnm1.p, a, b, cc,
                                                             c.rhs.p);
                CKL();
                Ops<MT>::precond_setup(c);
                Ops<MT>::solve_init(c);
                iterations_direct<MT>(c);
                {
                    Timed tm(c, KS_UPDATE);
                    k_update<<<nblk(c.N, TPB), TPB, 0, s>>>(c.N, c.th, c.bd, c.dx.p, c.W.p, c.prim.p, c.sc.p); CKL();
                }
                k_boundary<<<nblk(c.NB, TPB), TPB, 0, s>>>(c.m, c.th, c.bd, c.W.p, c.prim.p, c.bs.p); CKL();
                // turbulence inside the loop when innerCorrectTurbulence
                // (timeDST::correctTurbulence, timeDST.C:460-463; Dual.C:111-112)
                if (sa && o.inner_correct_turbulence) sa_correct(c);
                double ir[5];
                CK(cudaMemcpyAsync(ir, c.sc.p->lin_initial, sizeof(ir), cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
                rc.add(ir);
                // setCourantDST(&solverPerf): |initialResidual|; the pseudo-time
                // branch while the steadyCheck (its last slope) is not converged
                double ir2 = 0;
                for (int k = 0; k < 5; ++k) ir2 += ir[k] * ir[k];
                const bool pseudo = !rc.converged_now();
                k_courant_scalar_r<<<1, 1, 0, s>>>(c.sc.p, std::sqrt(ir2), (!pseudo && o.adjust_time_step) ? 1 : 0,
                                                   o.min_co, o.max_co);
                CKL();
                if (pseudo) {
                    k_courant_cells<<<nblk(c.N, TPB), TPB, 0, s>>>(c.m, c.W.p, c.rhoOld.p, c.eOld.p, c.courantF.p,
                                                                  c.sc.p, o.min_co, o.max_co, c.eNew.p);
                    CKL();
                    k_store_old<<<nblk(c.N, TPB), TPB, 0, s>>>(c.N, c.W.p, c.eNew.p, c.rhoOld.p, c.eOld.p); CKL();
                    set_steady_dt(c);
                } else if (o.adjust_time_step) {
                    set_transient_dt(c);
                }
                ++inner;
            } while (!rc.converged());
            // and once after it otherwise (Dual.C:120-121)
            if (sa && !o.inner_correct_turbulence) sa_correct(c);
            // setCourantDST(): residual of R, the converged branch
            k_courant_scalar<<<1, 1, 0, s>>>(c.sc.p, o.adjust_time_step ? 1 : 0, o.min_co, o.max_co); CKL();
            if (o.adjust_time_step) set_transient_dt(c);
            k_report<<<1, 1, 0, s>>>(c.sc.p, c.reps.p, rdst_ctx::REP_CAP); CKL();
            c.dual_a = c.dual_b = c.dual_c = 0.0;
            inner_counts.push_back(inner);
        }
        CK(cudaEventRecord(c.step_ev[1], s));
        if (host_reps)
            CK(cudaMemcpyAsync(host_reps + done, c.reps.p, sizeof(rdst_step_report) * chunk, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, c.step_ev[0], c.step_ev[1]));
        total_ms += ms;
        done += chunk;
    }
    // the report's iteration count of a dual step: its inner iterations
    if (host_reps)
        for (int k = 0; k < n; ++k) host_reps[k].lin_iterations = inner_counts[k];
    c.last_step_ms = total_ms;
    int flags = 0;
    CK(cudaMemcpyAsync(&flags, &c.sc.p->flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    c.collect_events();
    if (flags & 4) throw TimeoutError("a bounded wait of the ILU apply expired (bulk copy not completed)");
    if (flags & 2) throw std::domain_error("non-physical state (NaN or non-positive rho/p) after the update");
}

template <typename F>
rdst_status guarded(rdst_ctx* c, F&& fn) {
    if (!c) return RDST_ERR_ARG;
    CounterScope cs(*c);
    try {
        c->err.clear();
        // this library's CUDA runtime keeps its own current device: every
        // call runs on the context's GPU, whatever the caller's runtime set
        if (c->dev >= 0) CK(cudaSetDevice(c->dev));
        fn();
        return RDST_OK;
    } catch (const ConfigError& e) {
        c->err = e.what();
        return e.unsupported ? RDST_ERR_UNSUPPORTED : RDST_ERR_CONFIG;
    } catch (const CudaError& e) {
        c->err = e.what();
        return RDST_ERR_CUDA;
    } catch (const TimeoutError& e) {
        c->err = e.what();
        return RDST_ERR_TIMEOUT;
    } catch (const std::invalid_argument& e) {
        c->err = e.what();
        return RDST_ERR_MESH;
    } catch (const std::domain_error& e) {
        c->err = e.what();
        return RDST_ERR_DIVERGED;
    } catch (const std::exception& e) {
        c->err = e.what();
        return RDST_ERR_ARG;
    }
}

template <typename Fn>
void dispatch(rdst_ctx& c, Fn&& fn) {
    switch (c.o.precision) {
        case PREC_FP64: fn((double*)nullptr); break;
        case PREC_FP32: fn((float*)nullptr); break;
        default: fn((__nv_bfloat16*)nullptr); break;
    }
}

void after_state_set(rdst_ctx& c) {
    k_init_phib<<<nblk(c.NB, TPB), TPB, 0, c.s>>>(c.m, c.W.p, c.prim.p, c.bs.p);
    CKL();
    k_boundary<<<nblk(c.NB, TPB), TPB, 0, c.s>>>(c.m, c.th, c.bd, c.W.p, c.prim.p, c.bs.p);
    CKL();
    initialize_time(c);
    CK(cudaStreamSynchronize(c.s));
    c.state_set = true;
}

// ---------------------------------------------------------------- adjoint
// Buffers of the adjoint pass and of its GMRES(m) (FP64 basis).
void adj_alloc(rdst_ctx& c, int m) {
    const long n5 = 5L * c.N;
    if (!c.a_fbar.p) {
        c.a_fbar.alloc((size_t)ADJ_FB * std::max(c.Fi, 1));
        c.a_qbbar.alloc((size_t)ADJ_QB * std::max(c.NB, 1));
        c.a_qbar.alloc((size_t)ADJ_QB * c.N);
        c.a_gbar.alloc((size_t)GW * c.N);
        c.a_vval.alloc(7L * c.N); c.a_vidx.alloc(7L * c.N);
        c.a_hval.alloc(c.N); c.a_hidx.alloc(c.N);
        c.a_wbar.alloc(n5);
        c.a_wbarb.alloc(5L * std::max(c.NB, 1)); c.a_ubarb.alloc(3L * std::max(c.NB, 1));
        c.a_pbar.alloc(std::max(c.NB, 1));
        c.a_r.alloc(n5); c.a_z.alloc(n5); c.a_t.alloc(n5); c.a_psi.alloc(n5); c.a_rhs.alloc(n5);
        c.a_tmp.alloc(n5); c.a_u3.alloc(16);
        c.a_fbar.zero(c.s); c.a_qbbar.zero(c.s);
        if (c.tr.viscous) {
            c.a_vfbar.alloc((size_t)ADJ_VF * std::max(c.Fi, 1)); c.a_vbbar.alloc((size_t)ADJ_VBF * std::max(c.NB, 1));
            c.a_gUbar.alloc(9L * c.N); c.a_ucbar.alloc(4L * c.N);
            c.a_vfbar.zero(c.s); c.a_vbbar.zero(c.s);
        }
    }
    if (m > 0 && c.a_m != m) {
        c.a_V.alloc((size_t)(m + 1) * c.ldv);
        c.a_Z.alloc((size_t)(m + 1) * c.ldv);
        c.a_m = m;
    }
    if (!c.a_sc.p) { c.a_sc.alloc(1); c.a_sc.zero(c.s); }
}

int adj_use_c(const rdst_ctx& c) { return (c.o.flux == FLUX_KURGANOV || c.o.flux == FLUX_AUSM) ? 1 : 0; }

// u = (dR/dW)^T v (internal order, device); usum (device, 3) = sum of the
// patch-velocity shares when given
void adj_product(rdst_ctx& c, const double* v, double* u, double* usum) {
    const DevMesh& m = c.m;
    const Options& o = c.o;
    cudaStream_t s = c.s;
    const int use_c = adj_use_c(c);
    const bool visc = c.tr.viscous != 0;
    double* vfbar = visc ? c.a_vfbar.p : nullptr;
    double* vbbar = visc ? c.a_vbbar.p : nullptr;
    if (visc) {     // viscous face terms first: their face-velocity bars feed the convective VJP
        if (m.Fi > 0) {
            k_adj_visc_faces<<<nblk(m.Fi, 128), 128, 0, s>>>(m, c.q.p, c.prim.p, c.gU.p, c.up.p, v, vfbar);
            CKL();
        }
        if (m.NB > 0) {
            k_adj_visc_bfaces<<<nblk(m.NB, 128), 128, 0, s>>>(m, c.qb.p, c.prim.p, c.gU.p, c.bs.p, c.bup.p, v, vbbar);
            CKL();
        }
    }
    if (m.Fi > 0) {
        k_adj_faces<<<nblk(m.Fi, 128), 128, 0, s>>>(m, c.th, flux_code(o.flux), lim_code(o.lim_rho), lim_code(o.lim_U),
                                                   lim_code(o.lim_T), o.low_mach, o.mainf, c.q.p, c.g.p, c.psi.p,
                                                   c.fcell.p, v, vfbar, c.a_fbar.p);
        CKL();
    }
    if (m.NB > 0) {
        k_adj_bfaces<<<nblk(m.NB, 128), 128, 0, s>>>(m, c.th, flux_code(o.flux), o.low_mach, o.mainf, c.qb.p, v,
                                                     vbbar, c.a_qbbar.p);
        CKL();
    }
    k_adj_cells<<<nblk(m.N, 128), 128, 0, s>>>(m, flux_code(o.flux), lim_code(o.lim_rho), lim_code(o.lim_U),
                                               lim_code(o.lim_T), c.venkat_mask, o.venkat_K, c.q.p, c.qb.p, c.g.p,
                                               c.psi.p, c.fcell.p, c.prim.p, c.a_fbar.p, c.a_qbar.p, c.a_gbar.p,
                                               c.a_vidx.p, c.a_vval.p, c.a_hidx.p, c.a_hval.p);
    CKL();
    if (visc) {
        k_adj_visc_cells<<<nblk(m.N, 128), 128, 0, s>>>(m, vfbar, vbbar, c.a_gUbar.p, c.a_ucbar.p);
        CKL();
    }
    k_adj_gather<<<nblk(m.N, 128), 128, 0, s>>>(m, c.th, c.bd, c.tr, use_c, c.W.p, c.a_gbar.p, c.a_qbar.p, c.a_vidx.p,
                                                c.a_vval.p, c.a_hidx.p, c.a_hval.p, visc ? c.a_gUbar.p : nullptr,
                                                visc ? c.a_ucbar.p : nullptr, vbbar, c.a_qbbar.p, c.a_wbar.p);
    CKL();
    if (m.NB > 0) {
        k_adj_bc<<<nblk(m.NB, 128), 128, 0, s>>>(m, c.th, c.bd, c.tr, use_c, c.W.p, c.bs.p, c.a_qbbar.p, nullptr, vbbar,
                                                 c.a_wbarb.p, c.a_ubarb.p);
        CKL();
    }
    k_adj_finish<<<nblk(m.N, TPB), TPB, 0, s>>>(m, c.a_wbar.p, c.a_wbarb.p, u);
    CKL();
    if (usum) {
        if (m.NB > 0) {
            const int nb = red_blocks(m.NB);
            k_adj_usum<<<nb, RED_TPB, 0, s>>>(m.NB, c.a_ubarb.p, c.partial.p); CKL();
            k_adj_psum<<<1, RED_TPB, 0, s>>>(c.partial.p, nb, 3, usum); CKL();
        } else {
            CK(cudaMemsetAsync(usum, 0, 3 * sizeof(double), s));
        }
    }
}

// dJ/dW (device, internal order) of J = scale sum_patch (p - p_ref) S.d;
// host out: J, force[3], dJ/dU_patch explicit part [3]
void adj_objective(rdst_ctx& c, const rdst_objective& ob, double* dJdW, double out[7]) {
    const DevMesh& m = c.m;
    cudaStream_t s = c.s;
    const int nb = red_blocks(std::max(m.NB, 1));
    V3 dir;
    dir.x = ob.direction[0]; dir.y = ob.direction[1]; dir.z = ob.direction[2];
    k_adj_objective<<<nb, RED_TPB, 0, s>>>(m, ob.patch, dir, ob.p_ref,
                                           ob.scale, c.bs.p, c.a_pbar.p, c.partial.p);
    CKL();
    k_adj_psum<<<1, RED_TPB, 0, s>>>(c.partial.p, nb, 4, c.a_u3.p); CKL();
    if (m.NB > 0) {
        k_adj_bc<<<nblk(m.NB, 128), 128, 0, s>>>(m, c.th, c.bd, c.tr, adj_use_c(c), c.W.p, c.bs.p, nullptr, c.a_pbar.p,
                                                 nullptr, c.a_wbarb.p, c.a_ubarb.p);
        CKL();
        const int nbu = red_blocks(m.NB);
        k_adj_usum<<<nbu, RED_TPB, 0, s>>>(m.NB, c.a_ubarb.p, c.partial.p); CKL();
        k_adj_psum<<<1, RED_TPB, 0, s>>>(c.partial.p, nbu, 3, c.a_u3.p + 4); CKL();
    }
    k_adj_finish<<<nblk(m.N, TPB), TPB, 0, s>>>(m, nullptr, c.a_wbarb.p, dJdW);
    CKL();
    CK(cudaMemcpyAsync(out, c.a_u3.p, 7 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
}

// Preconditioner of the transposed system: A is the step's approximate
// Jacobian (Roe blocks + pseudo-time diagonal, A ~ V dR/dW + V/dtau); the
// adjoint is right-preconditioned with M^-1 y = V (A^T)^-1 y, (A^T)^-1 by
// block ILU(0) (or block Jacobi) of the transposed matrix.
template <typename MT>
void adj_precond_setup(rdst_ctx& c) {
    Ops<MT>::assemble(c);
    const size_t bytes = (size_t)c.n_slots * 32 * 25 * sizeof(MT);
    if (!c.a_AT) CK(cudaMalloc(&c.a_AT, bytes));
    k_transpose_blocks<MT><<<nblk(c.N, 128), 128, 0, c.s>>>(c.mat<MT>(c.Aval), (MT*)c.a_AT);
    CKL();
    if (c.o.precon == PRECON_DIAGONAL) {
        k_dinv<MT><<<nblk(c.N, 128), 128, 0, c.s>>>(c.mat<MT>(c.a_AT), (MT*)c.dinv);
        CKL();
    } else if (c.o.precon == PRECON_AMG) {
        std::swap(c.Aval, c.a_AT);
        Ops<MT>::amg_setup(c);
        std::swap(c.Aval, c.a_AT);
    } else if (lu_factored(c.o.precon)) {
        ilu_factorise<MT>(c, c.a_AT);
    }
}

template <typename MT>
void adj_precond(rdst_ctx& c, const double* in, double* out) {
    // Gauss-Seidel sweeps after the first take their residual with A^T
    std::swap(c.Aval, c.a_AT);
    Ops<MT>::precond(c, in, c.a_tmp.p, nullptr);
    std::swap(c.Aval, c.a_AT);
    k_adj_scale_V<<<nblk(5L * c.N, TPB), TPB, 0, c.s>>>(c.N, c.m.V, c.a_tmp.p, out);
    CKL();
}

// One application of the adjoint's preconditioner: out ~ V (A^T)^-1 in.
// With the GMRES step solver it is one restart cycle of that same solver
// (its directions, basis precision and block ILU(0)/Jacobi) run on A^T, the
// linear solve the step itself performs on A; otherwise the block
// preconditioner of A^T alone.
template <typename MT>
void adj_prec(rdst_ctx& c, const double* in, double* out) {
    if (c.o.solver != SOLVER_GMRES) {
        adj_precond<MT>(c, in, out);
        return;
    }
    const long n = c.nvec();
    std::swap(c.Aval, c.a_AT);
    CK(cudaMemcpyAsync(c.rhs.p, in, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.s));
    CK(cudaMemsetAsync(c.dx.p, 0, sizeof(double) * n, c.s));
    Ops<MT>::gmres_cycle(c);
    std::swap(c.Aval, c.a_AT);
    k_adj_scale_V<<<nblk(n, TPB), TPB, 0, c.s>>>(c.N, c.m.V, c.dx.p, out);
    CKL();
}

// Flexible GMRES(m), right preconditioned by adj_prec, for
// (dR/dW)^T psi = rhs; its Hessenberg lives in its own Scalars (the inner
// cycles use the step's).  Returns the number of outer iterations; res0 /
// res are the true residual norms at the start and at exit.
template <typename MT>
int adj_solve(rdst_ctx& c, const double* rhs, double* psi, double rel_tol, int max_cycles, int m, double& res0,
              double& res, int& cycles) {
    cudaStream_t s = c.s;
    const long n = c.nvec();
    Scalars* sc = c.a_sc.p;
    int* act = &sc->gm_active;
    double* Vb = c.a_V.p;
    double* Zb = c.a_Z.p;
    CK(cudaMemsetAsync(psi, 0, sizeof(double) * n, s));
    int iters = 0;
    res0 = 0.0;
    res = 0.0;
    cycles = 0;
    for (int cyc = 0; cyc < max_cycles; ++cyc) {
        // r = rhs - J^T psi (into V_0)
        adj_product(c, psi, c.a_t.p, nullptr);
        k_adj_sub<<<nblk(n, TPB), TPB, 0, s>>>(n, rhs, c.a_t.p, Vb); CKL();
        Ops<MT>::dot(c, Vb, Vb, &sc->beta, 1, nullptr);
        double beta = 0.0;
        CK(cudaMemcpyAsync(&beta, &sc->beta, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        res = beta;
        if (cyc == 0) res0 = res;
        if (res <= rel_tol * res0 || res == 0.0) break;
        ++cycles;
        k_gm_start<<<1, 1, 0, s>>>(sc); CKL();
        k_scale_inv<<<nblk(n, TPB), TPB, 0, s>>>(n, Vb, &sc->beta, act); CKL();
        for (int i = 0; i < m; ++i) {
            const double* Vi = Vb + i * c.ldv;
            double* Zi = Zb + i * c.ldv;
            double* w = Vb + (i + 1) * c.ldv;
            adj_prec<MT>(c, Vi, Zi);
            adj_product(c, Zi, w, nullptr);
            const int nv = i + 1;
            // CGS2 against V_0..V_i into this solve's own Hessenberg column
            auto orth = [&](auto nvtag) {
                constexpr int NV = decltype(nvtag)::value;
                Ops<MT>::template vmultidot<NV, double>(c, Vb, nv, w, sc->hcol[0], act);
                Ops<MT>::template maxpy_dot<NV, double>(c, Vb, nv, sc->hcol[0], w, sc->hcol[1], 0, act);
                Ops<MT>::template maxpy_dot<NV, double>(c, Vb, nv, sc->hcol[1], w, &sc->beta, 1, act);
            };
            if (nv <= 8) orth(std::integral_constant<int, 8>());
            else if (nv <= 16) orth(std::integral_constant<int, 16>());
            else if (nv <= 32) orth(std::integral_constant<int, 32>());
            else orth(std::integral_constant<int, 64>());
            k_gm_givens<<<1, 1, 0, s>>>(sc, i, m); CKL();
            if (i < m - 1) { k_scale_inv<<<nblk(n, TPB), TPB, 0, s>>>(n, w, &sc->beta, act); CKL(); }
            ++iters;
        }
        k_gm_backsub<<<1, 1, 0, s>>>(sc, m); CKL();
        // psi += Z y
        k_maxpy<double><<<nblk(n, TPB), TPB, 0, s>>>(n, m, Zb, c.ldv, sc->yh, psi, -1.0, nullptr); CKL();
    }
    return iters;
}

// the cell records (q, gradients, limiters; the boundary states and their
// branches are those of the last boundary evaluation) at the current W
template <typename MT>
void adj_forward(rdst_ctx& c) {
    if (c.tr.viscous && c.o.grad_U_limit > 0)
        throw ConfigError("the linearization of cellLimited grad(U) is not on this path", true);
    Ops<MT>::flux(c);
}


// Ju = (dR/dW) u by the forward-mode (tangent) pass (internal order, device)
void tan_product(rdst_ctx& c, const double* u, double* Ju) {
    const DevMesh& m = c.m;
    const Options& o = c.o;
    cudaStream_t s = c.s;
    const long N = c.N, NB = std::max(c.NB, 1), Fi = std::max(c.Fi, 1);
    const bool visc = c.tr.viscous != 0;
    // viscous records: velocity + muEff (4) per cell and boundary face, grad U
    // (9) per cell, face velocity (3) per face, viscous terms (8) per face
    const size_t nvisc = visc ? 2 * (4 * N + 4 * NB + 9 * N + 3 * Fi + 3 * NB) + 8 * Fi + 8 * NB : 0;
    const size_t need = 2 * (N * QW + N + NB * QW + N * GW + N * QW + N) + 5 * Fi + 5 * NB + nvisc;
    if (c.t_buf.n < need) c.t_buf.alloc(need);
    double* p0 = c.t_buf.p;
    double* qv = p0;            double* qd = qv + N * QW;
    double* pv = qd + N * QW;   double* pd = pv + N;
    double* qbv = pd + N;       double* qbd = qbv + NB * QW;
    double* gv = qbd + NB * QW; double* gd = gv + N * GW;
    double* psv = gd + N * GW;  double* psd = psv + N * QW;
    double* fcv = psd + N * QW; double* fcd = fcv + N;
    double* fld = fcd + N;      double* bfld = fld + 5 * Fi;
    double *uv = nullptr, *ud = nullptr, *ubv = nullptr, *ubd = nullptr, *gUv = nullptr, *gUd = nullptr;
    double *upv = nullptr, *upd = nullptr, *bupv = nullptr, *bupd = nullptr, *vfd = nullptr, *bvfd = nullptr;
    if (visc) {
        uv = bfld + 5 * NB;  ud = uv + 4 * N;
        ubv = ud + 4 * N;    ubd = ubv + 4 * NB;
        gUv = ubd + 4 * NB;  gUd = gUv + 9 * N;
        upv = gUd + 9 * N;   upd = upv + 3 * Fi;
        bupv = upd + 3 * Fi; bupd = bupv + 3 * NB;
        vfd = bupd + 3 * NB; bvfd = vfd + 8 * Fi;
    }
    const int use_c = adj_use_c(c);
    k_tan_q<<<nblk(N, TPB), TPB, 0, s>>>(c.N, c.th, c.bd, c.tr, use_c, c.W.p, u, c.mut.p, qv, qd, pv, pd, uv, ud); CKL();
    if (m.NB > 0) {
        k_tan_qb<<<nblk(m.NB, 128), 128, 0, s>>>(m, c.th, c.bd, c.tr, use_c, c.W.p, u, c.bs.p, c.mut_b.p, qbv, qbd,
                                                 ubv, ubd);
        CKL();
    }
    k_tan_grad<<<nblk(N, 128), 128, 0, s>>>(m, c.venkat_mask, o.venkat_K, o.flux == FLUX_HLLCP, qv, qd, qbv, qbd, pv, pd,
                                           gv, gd, psv, psd, fcv, fcd);
    CKL();
    if (m.Fi > 0) {
        k_tan_faces<<<nblk(m.Fi, 128), 128, 0, s>>>(m, c.th, flux_code(o.flux), lim_code(o.lim_rho), lim_code(o.lim_U),
                                                   lim_code(o.lim_T), o.low_mach, o.mainf, qv, qd, gv, gd, psv, psd,
                                                   fcv, fcd, fld, upv, upd);
        CKL();
    }
    if (m.NB > 0) {
        k_tan_bfaces<<<nblk(m.NB, 128), 128, 0, s>>>(m, c.th, flux_code(o.flux), o.low_mach, o.mainf, qbv, qbd, bfld,
                                                     bupv, bupd);
        CKL();
    }
    if (visc) {
        k_tan_gradU<<<nblk(N, 128), 128, 0, s>>>(m, uv, ud, ubv, ubd, gUv, gUd); CKL();
        if (m.Fi > 0) { k_tan_visc_faces<<<nblk(m.Fi, 128), 128, 0, s>>>(m, uv, ud, gUv, gUd, upv, upd, vfd); CKL(); }
        if (m.NB > 0) {
            k_tan_visc_bfaces<<<nblk(m.NB, 128), 128, 0, s>>>(m, uv, ud, gUv, gUd, ubv, ubd, bupv, bupd, bvfd);
            CKL();
        }
    }
    k_tan_residual<<<nblk(N, TPB), TPB, 0, s>>>(m, fld, bfld, vfd, bvfd, Ju);
    CKL();
}

// internal <-> caller order for N x 5 fields
void adj_to_internal(rdst_ctx& c, const double* host, double* dev) {
    std::vector<double> t(5L * c.N);
    for (int r = 0; r < c.N; ++r)
        for (int k = 0; k < 5; ++k) t[5L * r + k] = host[5L * c.perm[r] + k];
    CK(cudaMemcpyAsync(dev, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice, c.s));
    CK(cudaStreamSynchronize(c.s));
}
void adj_to_caller(rdst_ctx& c, const double* dev, double* host) {
    std::vector<double> t(5L * c.N);
    CK(cudaMemcpyAsync(t.data(), dev, t.size() * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    for (int r = 0; r < c.N; ++r)
        for (int k = 0; k < 5; ++k) host[5L * c.perm[r] + k] = t[5L * r + k];
}

}  // namespace

// ============================================================================ ABI
RDST_API const char* rdst_version(void) { return "rdst-b200 sm_100a"; }

RDST_API rdst_status rdst_create(const rdst_mesh* mesh, int32_t n_options, const char* const* keys,
                                 const char* const* values, rdst_ctx** out) {
    if (!mesh || !out || (n_options > 0 && (!keys || !values))) return RDST_ERR_ARG;
    *out = nullptr;
    if (mesh->n_cells <= 0 || mesh->n_internal_faces < 0 || mesh->n_faces < mesh->n_internal_faces ||
        !mesh->owner || (mesh->n_internal_faces > 0 && !mesh->neighbour) || !mesh->Sf || !mesh->Cf ||
        !mesh->magSf || !mesh->weights || !mesh->deltaCoeffs || !mesh->C || !mesh->V ||
        (mesh->n_patches > 0 && !mesh->patches))
        return RDST_ERR_MESH;
    std::unique_ptr<rdst_ctx> c(new rdst_ctx);
    try {
        c->o = parse_options(n_options, keys, values);
    } catch (const ConfigError& e) {
        return e.unsupported ? RDST_ERR_UNSUPPORTED : RDST_ERR_CONFIG;
    }
    if (c->o.turbulence != TURB_LAMINAR && !mesh->wall_distance) return RDST_ERR_MESH;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return RDST_ERR_CUDA;
    rdst_status st = guarded(c.get(), [&] {
        if (c->o.device >= 0) {
            if (c->o.device >= ndev) throw ConfigError("option device: no such GPU");
            CK(cudaSetDevice(c->o.device));
        }
        CK(cudaGetDevice(&c->dev));
        CK(cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking));
        build(*c, mesh);
    });
    if (st != RDST_OK) {
        fprintf(stderr, "rdst_create: %s\n", c->err.c_str());
        return st;
    }
    *out = c.release();
    return RDST_OK;
}

RDST_API rdst_status rdst_set_geometry(rdst_ctx* c, const rdst_mesh* mesh) {
    if (!c || !mesh) return RDST_ERR_ARG;
    if (!mesh->owner || (c->Fi > 0 && !mesh->neighbour) || !mesh->Sf || !mesh->Cf || !mesh->magSf ||
        !mesh->weights || !mesh->deltaCoeffs || !mesh->C || !mesh->V || (c->turb && !mesh->wall_distance))
        return RDST_ERR_MESH;
    return guarded(c, [&] {
        if (mesh->n_cells != c->N || mesh->n_internal_faces != c->Fi || mesh->n_faces != c->F ||
            mesh->n_patches != c->n_patches)
            throw std::invalid_argument("mesh sizes differ from the context's");
        if (!std::equal(c->hown.begin(), c->hown.end(), mesh->owner) ||
            !std::equal(c->hnei.begin(), c->hnei.end(), mesh->neighbour))
            throw std::invalid_argument("owner/neighbour lists differ from the context's");
        for (int p = 0; p < c->n_patches; ++p)
            if (mesh->patches[p].start != c->hpatch_start[p] || mesh->patches[p].size != c->hpatch_size[p])
                throw std::invalid_argument("patch ranges differ from the context's");
        load_geometry(*c, mesh, true);
    });
}

RDST_API rdst_status rdst_set_primitive(rdst_ctx* c, const double* p, const double* U, const double* T,
                                        const double* nut) {
    if (!c || !p || !U || !T) return RDST_ERR_ARG;
    if (c->turb && !nut) { c->err = "Spalart-Allmaras needs an initial nuTilda"; return RDST_ERR_ARG; }
    return guarded(c, [&] {
        std::vector<double> prim((size_t)PW * c->N, 0.0);
        for (int r = 0; r < c->N; ++r) {
            int i = c->perm[r];
            double* P = &prim[(size_t)PW * r];
            P[0] = p[i]; P[1] = T[i]; P[2] = c->o.Cp * T[i];
            P[3] = U[3 * i]; P[4] = U[3 * i + 1]; P[5] = U[3 * i + 2];
        }
        CK(cudaMemcpyAsync(c->prim.p, prim.data(), prim.size() * sizeof(double), cudaMemcpyHostToDevice, c->s));
        k_init_state<<<nblk(c->N, TPB), TPB, 0, c->s>>>(c->N, c->th, c->prim.p, c->W.p);
        CKL();
        CK(cudaStreamSynchronize(c->s));
        after_state_set(*c);
        // a new state: SARC1's old-time strain rate and the dual-time levels
        // restart from the current one; deltaT0 of the first step is
        // controlDict's deltaT (foam Time)
        if (c->saSoldValid.p) CK(cudaMemsetAsync(c->saSoldValid.p, 0, sizeof(int), c->s));
        c->dual_started = false;
        c->dt_save = c->o.delta_t;
        if (c->turb) {
            std::vector<double> nv(c->N);
            for (int r = 0; r < c->N; ++r) nv[r] = nut[c->perm[r]];
            CK(cudaMemcpyAsync(c->nut.p, nv.data(), nv.size() * sizeof(double), cudaMemcpyHostToDevice, c->s));
            const DevMesh& m = c->m;
            if (m.NB > 0) { k_sa_bc<<<nblk(m.NB, TPB), TPB, 0, c->s>>>(m, c->bs.p, c->sa); CKL(); }
            k_sa_init_mut<<<nblk(c->N, TPB), TPB, 0, c->s>>>(c->N, c->tr, c->W.p, c->prim.p, c->sa); CKL();
            k_sa_finish<<<nblk(c->N, TPB), TPB, 0, c->s>>>(c->N, c->o.turbulence == TURB_SANEG, c->W.p, c->nut.p, c->sa);
            CKL();
            if (m.NB > 0) { k_sa_mutb<<<nblk(m.NB, TPB), TPB, 0, c->s>>>(m, c->tr, c->bs.p, c->sa); CKL(); }
            CK(cudaStreamSynchronize(c->s));
        }
    });
}

RDST_API rdst_status rdst_set_nu_tilda(rdst_ctx* c, const double* nut) {
    if (!c || !nut) return RDST_ERR_ARG;
    if (!c->turb || !c->state_set) { c->err = "set_nu_tilda needs a turbulence model and a state"; return RDST_ERR_ARG; }
    return guarded(c, [&] {
        // nuTilda replaced between steps: boundary values and mu_t from it,
        // with the mean flow and the time-control history kept
        std::vector<double> nv(c->N);
        for (int r = 0; r < c->N; ++r) nv[r] = nut[c->perm[r]];
        CK(cudaMemcpyAsync(c->nut.p, nv.data(), nv.size() * sizeof(double), cudaMemcpyHostToDevice, c->s));
        const DevMesh& m = c->m;
        if (m.NB > 0) { k_sa_bc<<<nblk(m.NB, TPB), TPB, 0, c->s>>>(m, c->bs.p, c->sa); CKL(); }
        k_sa_init_mut<<<nblk(c->N, TPB), TPB, 0, c->s>>>(c->N, c->tr, c->W.p, c->prim.p, c->sa); CKL();
        k_sa_finish<<<nblk(c->N, TPB), TPB, 0, c->s>>>(c->N, c->o.turbulence == TURB_SANEG, c->W.p, c->nut.p, c->sa);
        CKL();
        if (m.NB > 0) { k_sa_mutb<<<nblk(m.NB, TPB), TPB, 0, c->s>>>(m, c->tr, c->bs.p, c->sa); CKL(); }
        CK(cudaStreamSynchronize(c->s));
    });
}

// cell ids (original numbering) -> internal rows on the device
static void upload_rows(rdst_ctx& c, int32_t n, const int32_t* cells, DBuf<int>& rows) {
    std::vector<int> r(n);
    for (int j = 0; j < n; ++j) {
        if (cells[j] < 0 || cells[j] >= c.N) throw std::invalid_argument("cell id out of range");
        r[j] = c.iperm[cells[j]];
    }
    rows.upload(r, c.s);
}

RDST_API rdst_status rdst_get_cells(rdst_ctx* c, int32_t n, const int32_t* cells, double* out) {
    if (!c || n < 0 || (n > 0 && (!cells || !out))) return RDST_ERR_ARG;
    if (n == 0) return RDST_OK;
    return guarded(c, [&] {
        DBuf<int> rows;
        DBuf<double> buf;
        upload_rows(*c, n, cells, rows);
        buf.alloc(6L * n);
        k_get_cells<<<nblk(n, TPB), TPB, 0, c->s>>>(n, rows.p, c->W.p, c->turb ? c->nut.p : nullptr, buf.p);
        CKL();
        CK(cudaMemcpyAsync(out, buf.p, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, c->s));
        CK(cudaStreamSynchronize(c->s));
    });
}

RDST_API rdst_status rdst_set_cells(rdst_ctx* c, int32_t n, const int32_t* cells, const double* in) {
    if (!c || n < 0 || (n > 0 && (!cells || !in))) return RDST_ERR_ARG;
    if (!c->state_set) { c->err = "set_cells needs a state"; return RDST_ERR_ARG; }
    return guarded(c, [&] {
        DBuf<int> rows;
        DBuf<double> buf;
        if (n > 0) {
            upload_rows(*c, n, cells, rows);
            std::vector<double> v(in, in + 6L * n);
            buf.upload(v, c->s);
            k_set_cells<<<nblk(n, TPB), TPB, 0, c->s>>>(n, c->th, rows.p, buf.p, c->W.p, c->prim.p,
                                                        c->turb ? c->nut.p : nullptr);
            CKL();
        }
        // as rdst_set_conservative between steps: boundary values from the
        // new internal field, time-control history kept; and mu_t from nuTilda
        if (c->saSoldValid.p) CK(cudaMemsetAsync(c->saSoldValid.p, 0, sizeof(int), c->s));
        c->dual_started = false;
        c->dt_save = c->o.delta_t;
        const DevMesh& m = c->m;
        k_boundary<<<nblk(c->NB, TPB), TPB, 0, c->s>>>(m, c->th, c->bd, c->W.p, c->prim.p, c->bs.p);
        CKL();
        if (c->turb) {
            if (m.NB > 0) { k_sa_bc<<<nblk(m.NB, TPB), TPB, 0, c->s>>>(m, c->bs.p, c->sa); CKL(); }
            k_sa_init_mut<<<nblk(c->N, TPB), TPB, 0, c->s>>>(c->N, c->tr, c->W.p, c->prim.p, c->sa); CKL();
            k_sa_finish<<<nblk(c->N, TPB), TPB, 0, c->s>>>(c->N, c->o.turbulence == TURB_SANEG, c->W.p, c->nut.p,
                                                           c->sa);
            CKL();
            if (m.NB > 0) { k_sa_mutb<<<nblk(m.NB, TPB), TPB, 0, c->s>>>(m, c->tr, c->bs.p, c->sa); CKL(); }
        }
        CK(cudaStreamSynchronize(c->s));
    });
}

// the same gather into a DEVICE buffer of the context's GPU (6 doubles per
// cell), for a halo handed to NCCL without a host copy; returns once the
// values are in the buffer
RDST_API rdst_status rdst_get_cells_device(rdst_ctx* c, int32_t n, const int32_t* cells, double* out_dev) {
    if (!c || n < 0 || (n > 0 && (!cells || !out_dev))) return RDST_ERR_ARG;
    if (n == 0) return RDST_OK;
    return guarded(c, [&] {
        DBuf<int> rows;
        upload_rows(*c, n, cells, rows);
        k_get_cells<<<nblk(n, TPB), TPB, 0, c->s>>>(n, rows.p, c->W.p, c->turb ? c->nut.p : nullptr, out_dev);
        CKL();
        CK(cudaStreamSynchronize(c->s));
    });
}

// rdst_set_cells from a DEVICE buffer of the context's GPU (6 doubles per
// cell, ready when the call is made)
RDST_API rdst_status rdst_set_cells_device(rdst_ctx* c, int32_t n, const int32_t* cells, const double* in_dev) {
    if (!c || n < 0 || (n > 0 && (!cells || !in_dev))) return RDST_ERR_ARG;
    if (!c->state_set) { c->err = "set_cells needs a state"; return RDST_ERR_ARG; }
    return guarded(c, [&] {
        DBuf<int> rows;
        if (n > 0) {
            upload_rows(*c, n, cells, rows);
            k_set_cells<<<nblk(n, TPB), TPB, 0, c->s>>>(n, c->th, rows.p, in_dev, c->W.p, c->prim.p,
                                                        c->turb ? c->nut.p : nullptr);
            CKL();
        }
        // as rdst_set_conservative between steps: boundary values from the
        // new internal field, time-control history kept; and mu_t from nuTilda
        if (c->saSoldValid.p) CK(cudaMemsetAsync(c->saSoldValid.p, 0, sizeof(int), c->s));
        c->dual_started = false;
        c->dt_save = c->o.delta_t;
        const DevMesh& m = c->m;
        k_boundary<<<nblk(c->NB, TPB), TPB, 0, c->s>>>(m, c->th, c->bd, c->W.p, c->prim.p, c->bs.p);
        CKL();
        if (c->turb) {
            if (m.NB > 0) { k_sa_bc<<<nblk(m.NB, TPB), TPB, 0, c->s>>>(m, c->bs.p, c->sa); CKL(); }
            k_sa_init_mut<<<nblk(c->N, TPB), TPB, 0, c->s>>>(c->N, c->tr, c->W.p, c->prim.p, c->sa); CKL();
            k_sa_finish<<<nblk(c->N, TPB), TPB, 0, c->s>>>(c->N, c->o.turbulence == TURB_SANEG, c->W.p, c->nut.p,
                                                           c->sa);
            CKL();
            if (m.NB > 0) { k_sa_mutb<<<nblk(m.NB, TPB), TPB, 0, c->s>>>(m, c->tr, c->bs.p, c->sa); CKL(); }
        }
        CK(cudaStreamSynchronize(c->s));
    });
}

RDST_API rdst_status rdst_set_held_cells(rdst_ctx* c, const uint8_t* mask) {
    if (!c) return RDST_ERR_ARG;
    return guarded(c, [&] {
        if (!mask) {
            c->rmask.free_();
            c->m.rmask = nullptr;
        } else {
            std::vector<unsigned char> mk(c->N);
            for (int r = 0; r < c->N; ++r) mk[r] = mask[c->perm[r]] ? 1 : 0;
            c->rmask.upload(mk, c->s);
            c->m.rmask = c->rmask.p;
            CK(cudaStreamSynchronize(c->s));
        }
        // the captured step graphs hold the mesh record: capture them again
        c->reset_graphs();
    });
}

RDST_API rdst_status rdst_set_conservative(rdst_ctx* c, const double* rho, const double* rhoU, const double* rhoE) {
    if (!c || !rho || !rhoU || !rhoE) return RDST_ERR_ARG;
    return guarded(c, [&] {
        const int N = c->N;
        double* d_rho = c->stage.p;
        double* d_rhoU = d_rho + N;
        double* d_rhoE = d_rhoU + 3L * N;
        CK(cudaMemcpyAsync(d_rho, rho, sizeof(double) * N, cudaMemcpyHostToDevice, c->s));
        CK(cudaMemcpyAsync(d_rhoU, rhoU, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, c->s));
        CK(cudaMemcpyAsync(d_rhoE, rhoE, sizeof(double) * N, cudaMemcpyHostToDevice, c->s));
        k_set_conservative<<<nblk(N, TPB), TPB, 0, c->s>>>(N, c->th, c->perm_d.p, d_rho, d_rhoU, d_rhoE, c->W.p,
                                                           c->prim.p);
        CKL();
        if (c->saSoldValid.p) CK(cudaMemsetAsync(c->saSoldValid.p, 0, sizeof(int), c->s));
        c->dual_started = false;
        c->dt_save = c->o.delta_t;
        if (c->state_set) {
            // fields replaced between steps: boundary values from the new
            // internal field, time-control history kept
            k_boundary<<<nblk(c->NB, TPB), TPB, 0, c->s>>>(c->m, c->th, c->bd, c->W.p, c->prim.p, c->bs.p);
            CKL();
            CK(cudaStreamSynchronize(c->s));
            return;
        }
        CK(cudaStreamSynchronize(c->s));
        after_state_set(*c);
    });
}

RDST_API rdst_status rdst_get_conservative(rdst_ctx* c, double* rho, double* rhoU, double* rhoE) {
    if (!c) return RDST_ERR_ARG;
    return guarded(c, [&] {
        const int N = c->N;
        double* d_rho = c->stage.p;
        double* d_rhoU = d_rho + N;
        double* d_rhoE = d_rhoU + 3L * N;
        k_get_conservative<<<nblk(N, TPB), TPB, 0, c->s>>>(N, c->perm_d.p, c->W.p, d_rho, d_rhoU, d_rhoE);
        CKL();
        if (rho) CK(cudaMemcpyAsync(rho, d_rho, sizeof(double) * N, cudaMemcpyDeviceToHost, c->s));
        if (rhoU) CK(cudaMemcpyAsync(rhoU, d_rhoU, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, c->s));
        if (rhoE) CK(cudaMemcpyAsync(rhoE, d_rhoE, sizeof(double) * N, cudaMemcpyDeviceToHost, c->s));
        CK(cudaStreamSynchronize(c->s));
    });
}

RDST_API rdst_status rdst_get_primitive(rdst_ctx* c, double* p, double* U, double* T, double* nut) {
    if (!c) return RDST_ERR_ARG;
    return guarded(c, [&] {
        std::vector<double> P((size_t)PW * c->N), nv(c->turb ? c->N : 0);
        CK(cudaMemcpyAsync(P.data(), c->prim.p, P.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        if (c->turb) CK(cudaMemcpyAsync(nv.data(), c->nut.p, nv.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        CK(cudaStreamSynchronize(c->s));
        for (int r = 0; r < c->N; ++r) {
            int i = c->perm[r];
            const double* q = &P[(size_t)PW * r];
            if (p) p[i] = q[0];
            if (T) T[i] = q[1];
            if (U) for (int k = 0; k < 3; ++k) U[3 * i + k] = q[3 + k];
            if (nut) nut[i] = c->turb ? nv[r] : 0.0;
        }
    });
}

RDST_API rdst_status rdst_step(rdst_ctx* c, int32_t n, rdst_step_report* reps) {
    if (!c || n < 0) return RDST_ERR_ARG;
    if (!c->state_set) { c->err = "rdst_step before the state was set"; return RDST_ERR_ARG; }
    return guarded(c, [&] {
        if (n == 0) return;
        dispatch(*c, [&](auto* tag) {
            using MT = std::remove_pointer_t<decltype(tag)>;
            if (c->o.dual) run_dual_steps<MT>(*c, n, reps);
            else run_steps<MT>(*c, n, reps);
        });
    });
}

RDST_API rdst_status rdst_residual(rdst_ctx* c, double* out) {
    if (!c || !out) return RDST_ERR_ARG;
    if (!c->state_set) return RDST_ERR_ARG;
    return guarded(c, [&] {
        dispatch(*c, [&](auto* tag) {
            using MT = std::remove_pointer_t<decltype(tag)>;
            Ops<MT>::flux(*c);
        });
        std::vector<double> R(5L * c->N);
        CK(cudaMemcpyAsync(R.data(), c->R.p, R.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        CK(cudaStreamSynchronize(c->s));
        for (int r = 0; r < c->N; ++r)
            for (int k = 0; k < 5; ++k) out[5 * c->perm[r] + k] = R[5 * r + k];
    });
}

RDST_API rdst_status rdst_assemble(rdst_ctx* c, double* diag, double* upper, double* lower, double* source) {
    if (!c || !c->state_set) return RDST_ERR_ARG;
    return guarded(c, [&] {
        size_t ms = c->mt_size;
        std::vector<unsigned char> raw((size_t)c->n_slots * 32 * 25 * ms);
        dispatch(*c, [&](auto* tag) {
            using MT = std::remove_pointer_t<decltype(tag)>;
            Ops<MT>::flux(*c);
            Ops<MT>::assemble(*c);
        });
        CK(cudaMemcpyAsync(raw.data(), c->Aval, raw.size(), cudaMemcpyDeviceToHost, c->s));
        std::vector<double> rhs(5L * c->N);
        CK(cudaMemcpyAsync(rhs.data(), c->rhs.p, rhs.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        std::vector<int> slice_off(c->n_slices + 1), col((size_t)c->n_slots * 32);
        CK(cudaMemcpyAsync(slice_off.data(), c->slice_off.p, slice_off.size() * sizeof(int), cudaMemcpyDeviceToHost, c->s));
        CK(cudaMemcpyAsync(col.data(), c->col.p, col.size() * sizeof(int), cudaMemcpyDeviceToHost, c->s));
        std::vector<int> own(c->Fi), nei(c->Fi);
        CK(cudaMemcpyAsync(own.data(), c->own.p, own.size() * sizeof(int), cudaMemcpyDeviceToHost, c->s));
        CK(cudaMemcpyAsync(nei.data(), c->nei.p, nei.size() * sizeof(int), cudaMemcpyDeviceToHost, c->s));
        CK(cudaStreamSynchronize(c->s));
        auto val = [&](size_t idx) -> double {
            if (ms == 8) return ((const double*)raw.data())[idx];
            if (ms == 4) return ((const float*)raw.data())[idx];
            uint16_t b = ((const uint16_t*)raw.data())[idx];
            uint32_t u = (uint32_t)b << 16;
            float f;
            std::memcpy(&f, &u, 4);
            return f;
        };
        auto block_of = [&](int r, int cc, double* out25) {
            int s0 = slice_off[r >> 5], wdt = slice_off[(r >> 5) + 1] - s0;
            for (int k = 0; k < wdt; ++k) {
                size_t slot = (size_t)(s0 + k);
                if (col[slot * 32 + (r & 31)] == cc) {
                    for (int e = 0; e < 25; ++e) out25[e] = val(slot * 800 + (size_t)e * 32 + (r & 31));
                    return;
                }
            }
            throw std::runtime_error("matrix slot missing");
        };
        for (int r = 0; r < c->N; ++r) {
            int i = c->perm[r];
            if (diag) block_of(r, r, diag + 25L * i);
            if (source) for (int k = 0; k < 5; ++k) source[5L * i + k] = rhs[5L * r + k];
        }
        // a cell pair joined by several faces holds one summed block: it is
        // reported on the pair's first face, the others get zero blocks
        std::unordered_map<long long, int> first_face;
        for (int f = 0; f < c->Fi; ++f) {
            long long key = (long long)own[f] * c->N + nei[f];
            bool dup = !first_face.emplace(key, f).second;
            if (dup) {
                if (upper) std::fill(upper + 25L * f, upper + 25L * f + 25, 0.0);
                if (lower) std::fill(lower + 25L * f, lower + 25L * f + 25, 0.0);
                continue;
            }
            if (upper) block_of(own[f], nei[f], upper + 25L * f);
            if (lower) block_of(nei[f], own[f], lower + 25L * f);
        }
    });
}

RDST_API rdst_status rdst_forces(rdst_ctx* c, int32_t patch, const double lift[3], const double drag[3],
                                 const double cofr[3], const double axis[3], double p_ref, double qA, double l_ref,
                                 double out[3]) {
    if (!c || !lift || !drag || !cofr || !axis || !out) return RDST_ERR_ARG;
    if (patch < 0 || patch >= c->n_patches) { c->err = "bad patch index"; return RDST_ERR_ARG; }
    return guarded(c, [&] {
        std::vector<double> bs((size_t)BW * std::max(c->NB, 1)), Sf(3L * std::max(c->NB, 1)), Cf(3L * std::max(c->NB, 1));
        CK(cudaMemcpyAsync(bs.data(), c->bs.p, bs.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        CK(cudaMemcpyAsync(Sf.data(), c->bSf.p, Sf.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        CK(cudaMemcpyAsync(Cf.data(), c->bCf.p, Cf.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        CK(cudaStreamSynchronize(c->s));
        double Fl = 0, Fd = 0, Mm = 0;
        const int NB = c->NB;
        for (int f = c->hpatch_start[patch]; f < c->hpatch_start[patch] + c->hpatch_size[patch]; ++f) {
            int b = c->bface_of_face[f - c->Fi];
            if (b < 0) continue;
            double pb = bs[(size_t)BW * b + 5] - p_ref;
            double dF[3] = {pb * Sf[b], pb * Sf[NB + b], pb * Sf[2L * NB + b]};
            Fl += dF[0] * lift[0] + dF[1] * lift[1] + dF[2] * lift[2];
            Fd += dF[0] * drag[0] + dF[1] * drag[1] + dF[2] * drag[2];
            double rr[3] = {Cf[b] - cofr[0], Cf[NB + b] - cofr[1], Cf[2L * NB + b] - cofr[2]};
            double mo[3] = {rr[1] * dF[2] - rr[2] * dF[1], rr[2] * dF[0] - rr[0] * dF[2], rr[0] * dF[1] - rr[1] * dF[0]};
            Mm += mo[0] * axis[0] + mo[1] * axis[1] + mo[2] * axis[2];
        }
        out[0] = Fl / qA;
        out[1] = Fd / qA;
        out[2] = Mm / (qA * l_ref);
    });
}

const char* rdst_noalloc_error_message();   // rdst_noalloc.cu

RDST_API const char* rdst_last_error(const rdst_ctx* c) { return c ? c->err.c_str() : rdst_noalloc_error_message(); }

RDST_API void* rdst_stream(rdst_ctx* c) { return c ? (void*)c->s : nullptr; }

RDST_API int64_t rdst_launch_count(const rdst_ctx* c) { return c ? (int64_t)c->launches : 0; }

RDST_API double rdst_last_step_ms(const rdst_ctx* c) { return c ? c->last_step_ms : 0.0; }

RDST_API rdst_status rdst_kernel_stats(rdst_ctx* c, const char* kernel, int64_t* launches, double* total_ms) {
    if (!c || !kernel || !launches || !total_ms) return RDST_ERR_ARG;
    for (int k = 0; k < KS_N; ++k)
        if (std::strcmp(kernel, KS_NAMES[k]) == 0) {
            *launches = c->ks_launches[k];
            *total_ms = c->ks_ms[k];
            return RDST_OK;
        }
    c->err = std::string("unknown kernel class ") + kernel;
    return RDST_ERR_ARG;
}

RDST_API rdst_status rdst_set_profile(rdst_ctx* c, int32_t on) {
    if (!c) return RDST_ERR_ARG;
    try {
        CK(cudaStreamSynchronize(c->s));
        c->collect_events();
        if (c->o.profile != (on != 0)) {
            c->o.profile = on != 0;
            c->reset_graphs();
        }
        return RDST_OK;
    } catch (const std::exception& e) {
        c->err = e.what();
        return RDST_ERR_CUDA;
    }
}

RDST_API rdst_status rdst_objective_gradient(rdst_ctx* c, const rdst_objective* ob, double* J, double force[3],
                                             double* dJdW, double dJdU[3]) {
    if (!c || !ob || !c->state_set) return RDST_ERR_ARG;
    if (ob->patch < 0 || ob->patch >= c->n_patches) { c->err = "bad patch index"; return RDST_ERR_ARG; }
    return guarded(c, [&] {
        dispatch(*c, [&](auto* tag) {
            using MT = std::remove_pointer_t<decltype(tag)>;
            adj_forward<MT>(*c);
        });
        adj_alloc(*c, 0);
        double out[7];
        adj_objective(*c, *ob, c->a_rhs.p, out);
        if (J) *J = out[0];
        if (force) for (int k = 0; k < 3; ++k) force[k] = out[1 + k];
        if (dJdU) for (int k = 0; k < 3; ++k) dJdU[k] = out[4 + k];
        if (dJdW) adj_to_caller(*c, c->a_rhs.p, dJdW);
    });
}

RDST_API rdst_status rdst_boundary_branches(rdst_ctx* c, double* phi_prev, double* mach) {
    if (!c || !phi_prev || !mach || !c->state_set) return RDST_ERR_ARG;
    return guarded(c, [&] {
        const int nball = c->NBall;
        std::fill(phi_prev, phi_prev + nball, 0.0);
        std::fill(mach, mach + nball, 0.0);
        if (c->NB == 0) return;
        std::vector<double> bs((size_t)BW * c->NB);
        CK(cudaMemcpyAsync(bs.data(), c->bs.p, bs.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        CK(cudaStreamSynchronize(c->s));
        for (int b = 0; b < c->NB; ++b) {
            const int k = c->bface_orig[b] - c->Fi;
            phi_prev[k] = bs[(size_t)BW * b + 11];
            mach[k] = bs[(size_t)BW * b + 15];
        }
    });
}

RDST_API rdst_status rdst_tangent_product(rdst_ctx* c, const double* u, double* Ju) {
    if (!c || !u || !Ju || !c->state_set) return RDST_ERR_ARG;
    return guarded(c, [&] {
        dispatch(*c, [&](auto* tag) {
            using MT = std::remove_pointer_t<decltype(tag)>;
            adj_forward<MT>(*c);
        });
        adj_alloc(*c, 0);
        adj_to_internal(*c, u, c->a_z.p);
        tan_product(*c, c->a_z.p, c->a_t.p);
        adj_to_caller(*c, c->a_t.p, Ju);
    });
}

RDST_API rdst_status rdst_adjoint_product(rdst_ctx* c, const double* v, double* u, double dU[3]) {
    if (!c || !v || !u || !c->state_set) return RDST_ERR_ARG;
    return guarded(c, [&] {
        dispatch(*c, [&](auto* tag) {
            using MT = std::remove_pointer_t<decltype(tag)>;
            adj_forward<MT>(*c);
        });
        adj_alloc(*c, 0);
        adj_to_internal(*c, v, c->a_z.p);
        adj_product(*c, c->a_z.p, c->a_t.p, c->a_u3.p + 8);
        adj_to_caller(*c, c->a_t.p, u);
        if (dU) {
            CK(cudaMemcpyAsync(dU, c->a_u3.p + 8, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->s));
            CK(cudaStreamSynchronize(c->s));
        }
    });
}

RDST_API rdst_status rdst_adjoint(rdst_ctx* c, const rdst_objective* ob, double rel_tol, int32_t max_cycles,
                                  int32_t n_directions, double* psi, rdst_adjoint_report* rep) {
    if (!c || !ob || !c->state_set || max_cycles < 1 || n_directions < 1 || n_directions > 64 || !(rel_tol > 0))
        return RDST_ERR_ARG;
    if (ob->patch < 0 || ob->patch >= c->n_patches) { c->err = "bad patch index"; return RDST_ERR_ARG; }
    return guarded(c, [&] {
        cudaEvent_t e0 = c->get_event(), e1 = c->get_event();
        CK(cudaEventRecord(e0, c->s));
        double out[7], usum[3];
        double res0 = 0, res = 0;
        int iters = 0, cycles = 0;
        dispatch(*c, [&](auto* tag) {
            using MT = std::remove_pointer_t<decltype(tag)>;
            adj_forward<MT>(*c);
            adj_alloc(*c, n_directions);
            adj_objective(*c, *ob, c->a_rhs.p, out);
            adj_precond_setup<MT>(*c);
            iters = adj_solve<MT>(*c, c->a_rhs.p, c->a_psi.p, rel_tol, max_cycles, n_directions, res0, res, cycles);
            adj_product(*c, c->a_psi.p, c->a_t.p, c->a_u3.p + 8);
        });
        CK(cudaMemcpyAsync(usum, c->a_u3.p + 8, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        CK(cudaEventRecord(e1, c->s));
        CK(cudaStreamSynchronize(c->s));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        c->ev_pool.push_back(e0);
        c->ev_pool.push_back(e1);
        if (psi) adj_to_caller(*c, c->a_psi.p, psi);
        if (rep) {
            rep->J = out[0];
            for (int k = 0; k < 3; ++k) { rep->force[k] = out[1 + k]; rep->dJ_dU[k] = out[4 + k] - usum[k]; }
            rep->residual0 = res0;
            rep->residual = res;
            rep->iterations = iters;
            rep->cycles = cycles;
            rep->t_ms = ms;
        }
    });
}

RDST_API void rdst_destroy(rdst_ctx* c) { delete c; }

RDST_API rdst_status rdst_partition_cells(int32_t n_cells, const double* C, int32_t n_parts, int32_t* out) {
    if (n_cells <= 0 || !C || !out || n_parts <= 0) return RDST_ERR_ARG;
    std::vector<int> idx(n_cells);
    std::iota(idx.begin(), idx.end(), 0);
    rcb(C, idx, 0, n_cells, 0, std::min(n_parts, n_cells), out);
    return RDST_OK;
}

RDST_API rdst_status rdst_partition_graph(int32_t n_cells, int32_t n_internal_faces, const int32_t* owner,
                                          const int32_t* neighbour, int32_t n_parts, int32_t* out) {
    if (n_cells <= 0 || n_internal_faces < 0 || !out || n_parts <= 0 ||
        (n_internal_faces > 0 && (!owner || !neighbour)))
        return RDST_ERR_ARG;
    for (int f = 0; f < n_internal_faces; ++f)
        if (owner[f] < 0 || owner[f] >= n_cells || neighbour[f] < 0 || neighbour[f] >= n_cells ||
            owner[f] == neighbour[f])
            return RDST_ERR_MESH;
    graph_partition(n_cells, n_internal_faces, owner, neighbour, std::min(n_parts, n_cells), out);
    return RDST_OK;
}
