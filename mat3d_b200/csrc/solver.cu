// solver.cu -- host runtime and C ABI of libmat3d_b200.so.
//
// A solver handle owns one CUDA stream, the device buffers of its batch and
// the per-phase constant tables.  A run launches chunks of sweeps (five pass
// kernels + a finalize kernel each); every kernel reads the device-side done
// flag of its batch entry, so the host only synchronises once per chunk to
// read the control blocks.  Chunks of the steady iteration are captured once
// into CUDA graphs and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <set>
#include <string>
#include <vector>

#include "../../include/mat3d_b200.h"
#include "physics.cuh"
#include "inelastic.cuh"
#include "passes_fast.cuh"
#include "passes_slab.cuh"
#include "fft_plan.hpp"

#include <cudaTypedefs.h>

using namespace m3d;

namespace {

thread_local std::string g_last_error;

int fail(int st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

#define M3D_CUDA(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            return fail(e_ == cudaErrorMemoryAllocation ? M3D_ERR_OOM : M3D_ERR_CUDA,                 \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                           \
        }                                                                                              \
    } while (0)

// ---- small dense algebra (host, double) ------------------------------------
typedef std::vector<double> Mat;  // row-major n x n

Mat mat_inv(const Mat& A, int n) {
    Mat a = A, inv(n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(a[r * n + c]) > std::fabs(a[piv * n + c])) piv = r;
        if (piv != c)
            for (int j = 0; j < n; ++j) {
                std::swap(a[c * n + j], a[piv * n + j]);
                std::swap(inv[c * n + j], inv[piv * n + j]);
            }
        const double p = a[c * n + c];
        for (int j = 0; j < n; ++j) { a[c * n + j] /= p; inv[c * n + j] /= p; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = a[r * n + c];
            if (f == 0.0) continue;
            for (int j = 0; j < n; ++j) { a[r * n + j] -= f * a[c * n + j]; inv[r * n + j] -= f * inv[c * n + j]; }
        }
    }
    return inv;
}
Mat mat_mul(const Mat& A, const Mat& B, int n) {
    Mat o(n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j) o[i * n + j] += A[i * n + k] * B[k * n + j];
    return o;
}
Mat mat_add(const Mat& A, const Mat& B, double s = 1.0) {
    Mat o(A.size());
    for (size_t i = 0; i < A.size(); ++i) o[i] = A[i] + s * B[i];
    return o;
}
Mat mat_scale(const Mat& A, double s) {
    Mat o(A);
    for (auto& v : o) v *= s;
    return o;
}
Mat iso_stiffness(double la, double mu) {
    // src/3d/FFT_analysis3D.cpp:457-462 (Voigt, tensor shear)
    Mat C(36, 0.0);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[i * 6 + j] = la;
    for (int i = 0; i < 3; ++i) C[i * 6 + i] = la + 2 * mu;
    for (int i = 3; i < 6; ++i) C[i * 6 + i] = 2 * mu;
    return C;
}
Mat diag(int n, double v) {
    Mat o(n * n, 0.0);
    for (int i = 0; i < n; ++i) o[i * n + i] = v;
    return o;
}


// Let a kernel use all dynamic shared memory left next to its static arrays
// (227 KB per block on sm_100 in total).
// Done once per kernel and device; safe to call from several host threads.
std::mutex g_attr_mu;
std::set<std::pair<int, const void*>> g_attr_done;
template <class K>
void allow_smem(K kernel) {
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(g_attr_mu);
        if (!g_attr_done.insert(std::make_pair(dev, (const void*)kernel)).second) return;
    }
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, kernel) == cudaSuccess) {
        const int maxdyn = 227 * 1024 - (int)a.sharedSizeBytes;
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, maxdyn);
    }
    (void)cudaGetLastError();  // an unsupported request must not surface at the next launch check
}

int even_up(int v) { return (v + 1) & ~1; }

}  // namespace

// ============================================================================
struct m3d_solver {
    // configuration
    int kind = 0, behav = 0, prec = 0, B = 1, C = 6;
    int Nx = 0, Ny = 0, Nz = 0;
    GridDims g{};
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    bool material_set = false;
    bool load_set = false;
    bool run_done = false;

    // model (host)
    int nph = 0;
    int scheme = 0;                // 1 primal (strain/gradient), 2 dual (stress/flux)
    std::vector<double> mat;       // nph x 7
    std::vector<long long> counts; // voxels per phase
    std::vector<double> vol;
    double la0 = 0, mu0 = 0, k0 = 0, km = 0, ki = 0;
    Mat Cp[kMaxPhases], Sp[kMaxPhases];
    Mat C0, S0;
    std::vector<double> hP, hA, hO, hOsum, hQ;  // per phase, C x C (hOsum: C)
    double den_ref = 0;   // reference stop rule denominator (without V*sum(E))
    std::vector<double> E;   // B x C
    std::vector<double> X0;  // B x 6

    // RVEs of the batch: entry b solves RVE b / (B / nrve) (nrve == 1: one RVE
    // shared by every entry).  Each RVE has its own phase map (V bytes at
    // r * V in d_phase), its own table block (mstride doubles at r * mstride
    // in d_mats) and its own reference medium, whose Green-operator constants
    // travel in the entries' control blocks.
    struct RveHost {
        bool set = false;
        int nph = 0, scheme = 0;
        double den_ref = 0;
        std::vector<long long> counts;
        std::vector<double> hOsum;
        int gkind = 0, gnyq = 0, gxw = 0;
        double gp1 = 0, gp2 = 0;
        bool diag = false;  // P and A diagonal in the components for every phase (slab pass usable)
    };
    int nrve = 1;
    std::vector<RveHost> rv;
    long long mstride = 0;  // doubles per RVE table block (kMaxPhases phase slots)
    int entries_per_rve() const { return B / nrve; }
    int rve_of(int b) const { return b / entries_per_rve(); }
    void set_green(Ctl& c, int r) const {
        const RveHost& m = rv[r];
        c.gkind = m.gkind; c.gnyq = m.gnyq; c.gxw = m.gxw; c.gp1 = m.gp1; c.gp2 = m.gp2;
    }
    // per-RVE table and phase-map addressing of a pointwise operator
    template <class Op> Op tab(Op o) const {
        o.lc = entries_per_rve();
        o.mstride = mstride;
        return o;
    }
    void snapshot_rve(int r);
    bool all_rves_set() const {
        for (const RveHost& m : rv) if (!m.set) return false;
        return true;
    }
    int nph_max() const {
        int n = 1;
        for (const RveHost& m : rv) n = std::max(n, m.nph);
        return n;
    }

    // device
    uint8_t* d_phase = nullptr;
    void* d_x = nullptr;       // state: T (FP32/FP64) or double (refine)
    float* d_delta = nullptr;  // refine correction
    float* d_r32 = nullptr;    // refine defect
    void* d_spec = nullptr;    // half spectrum (double2 or float2); refine: double2, aliased as float2
    double* d_part = nullptr;
    size_t part_cap = 0;
    Ctl* d_ctl = nullptr;
    Ctl* d_ctl_in = nullptr;
    Ctl* h_ctl = nullptr;  // pinned, B entries
    double* d_mats = nullptr;  // per RVE: [P | A | O | Osum | Q] blocks
    size_t off_P = 0, off_A = 0, off_O = 0, off_Os = 0, off_Q = 0;
    void* d_tw64 = nullptr;  // double2: Nx | Ny | Nz
    void* d_tw32 = nullptr;  // float2
    LinePlan px{}, py{}, pz{};
    double* d_out = nullptr;  // export scratch (C*V doubles)
    // asynchronous export: copy stream, export-written and copy-done events
    cudaStream_t xstream = nullptr;
    cudaEvent_t ev_exp = nullptr, ev_d2h = nullptr;
    bool d2h_pending = false;
    size_t alloc_B = 0;

    // inelastic state (J2 / damage)
    InelasticState in{};

    // stats
    m3d_stats st{};
    std::vector<double> prop;  // nInc x 9

    // launch geometry
    int G64 = 2, G32 = 2, TZy64 = 8, TZy32 = 16, TZx64 = 4, TZx32 = 8;

    // per-sweep event timing (m3d_set_profiling)
    static constexpr int kChunk = 8;
    bool prof = false;
    cudaEvent_t pev[kChunk + 1] = {};
    cudaEvent_t ppev[kChunk][6] = {};  // around each of the 5 passes of a sweep (launch_sweep)
    bool pass_rec[kChunk] = {};
    int prof_k = 0;
    m3d_profile pr{};
    void prof_mark(int k) {
        if (!prof) return;
        cudaEventRecord(pev[k], stream);
        prof_k = k;
        if (k < kChunk) pass_rec[k] = false;
    }
    void prof_pass(int p) {
        if (!prof || prof_k >= kChunk) return;
        cudaEventRecord(ppev[prof_k][p], stream);
        if (p == 5) pass_rec[prof_k] = true;
    }
    // add the first `executed` sweep intervals of the last chunk (host has synced)
    void prof_collect(int executed, bool fp64) {
        if (!prof) return;
        for (int k = 0; k < executed && k < kChunk; ++k) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, pev[k], pev[k + 1]) != cudaSuccess) continue;
            if (fp64) { pr.ms_fp64 += ms; pr.n_fp64 += 1; } else { pr.ms_fp32 += ms; pr.n_fp32 += 1; }
            if (!pass_rec[k]) continue;
            for (int p = 0; p < 5; ++p) {
                float mp = 0;
                if (cudaEventElapsedTime(&mp, ppev[k][p], ppev[k][p + 1]) != cudaSuccess) continue;
                (fp64 ? pr.pass_ms_fp64 : pr.pass_ms_fp32)[p] += mp;
            }
        }
        (void)cudaGetLastError();
    }
    int max_iters() const {
        int m = 0;
        for (int b = 0; b < B; ++b) m = std::max(m, h_ctl[b].iters);
        return m;
    }

    ~m3d_solver();
    int alloc(int batch);
    void free_all();
    template <typename T> int G() const { return sizeof(T) == 8 ? G64 : G32; }
    template <typename T> int TZy() const { return sizeof(T) == 8 ? TZy64 : TZy32; }
    template <typename T> int TZx() const { return sizeof(T) == 8 ? TZx64 : TZx32; }
    template <typename T> typename Cx<T>::t* tw(int axis) const {
        typedef typename Cx<T>::t C2;
        C2* base = (C2*)(sizeof(T) == 8 ? d_tw64 : d_tw32);
        return axis == 0 ? base : (axis == 1 ? base + Nx : base + Nx + Ny);
    }
    const double* dm(size_t off) const { return d_mats + off; }

    // sweeps
    template <typename T, int CC, class Pro, class Spec, class Epi>
    int launch_sweep(Pro pro, Spec spec, Epi epi, Ctl* ctl, typename Cx<T>::t* sp, int policy, const Ctl* outer);
    template <typename T, int CC>
    int launch_check(Ctl* ctl, const void* x, typename Cx<T>::t* sp);
    template <typename T, int CC> size_t op_smem() const;
    template <typename T, int CC, class Pro> void pass_zfwd(Pro pro, Ctl* ctl, typename Cx<T>::t* sp);
    template <typename T> void pass_y(int sign, int CC, Ctl* ctl, typename Cx<T>::t* sp);
    template <typename T, int CC, class Spec> int pass_x(Spec op, Ctl* ctl, typename Cx<T>::t* sp);
    template <typename T, int CC, class Epi, class Fin> int pass_zinv(Epi epi, Ctl* ctl, typename Cx<T>::t* sp, Fin fin);
    int* d_counter = nullptr;  // completion counters of the fused finalize, one per batch entry
    // TMA-staged y pass: tensor maps of the half spectrum viewed as rows of
    // 2*Hzp FP32 / FP64 scalars (built for the current buffer and batch)
    bool use_tma_y = false;
    CUtensorMap ymap32{}, ymap64{};
    const void* ymap_base = nullptr;
    int ymap_B = -1;
    int* d_err = nullptr;  // device-side error word (bounded waits that expired)
    bool ensure_ymaps(int CC);
    // TMA-staged rank-one x turnaround (thermal, FP32): a 3-D map of the half
    // spectrum, boxes of cpw columns x 1 row x Nx points (M3D_XTURN_TMA=0
    // keeps the plain rank-one kernel)
    bool use_xr1_tma = true;
    CUtensorMap xmap32{};
    const void* xmap_base = nullptr;
    int xmap_B = -1, xmap_cpw = -1;
    bool ensure_xmap(int cpw);
    bool use_fast = true;
    // two-pass sweeps (x turnaround + y-z slab pass) where the operators are
    // per-component and the slab fits two CTAs per SM; M3D_NO_SLAB=1 keeps
    // the five-pass sweep
    bool use_slab = true;
    int slab_nt = 256;  // M3D_SLAB_NT=512: one 512-thread slab CTA per SM at FP32 128^2 (measured slower)
    // thermal FP32 x turnaround with the three components in registers
    // (M3D_XTURN_STAGED=1 keeps the shared-memory-staged kernel)
    bool use_xreg = true;
    // thermal x turnaround in rank-one form (M3D_XTURN_R1=0 turns it off)
    bool use_xr1 = true;
    // x turnaround with a warp per component where no rank form applies
    // (M3D_XTURN_CP=0: the staged kernel, all components of its columns in
    // each warp)
    bool use_xcp = true;
    template <typename T> bool slab_ok() const;
    template <typename T, int CC, bool MIX, class Fin>
    int pass_slab(Ctl* ctl, T* x, const float* r, typename Cx<T>::t* sp, Fin fin);
    template <typename T, int CC>
    int launch_em_slab(Ctl* ctl, T* x, const float* r, typename Cx<T>::t* sp, int zero_k0, int policy,
                       const Ctl* outer);
    template <typename T, int CC> int tune_time(int sweeps, float* ms);
    int autotune(int sweeps, m3d_tune* out);
    template <typename T, int CC>
    int run_linear(double tol_field, double tol_eq, int criterion, int max_iter);
    template <int CC>
    int run_refine(double tol_field, int max_iter);
    // Graph-captured solves: the whole iteration runs as one CUDA graph launch,
    // its loops as conditional while nodes that a one-block kernel re-arms
    // after each sweep (no host round trip until the batch is done).
    bool use_graph = true;
    // Compacted sweeps (multi-entry graph solves, residual rule): the loop
    // runs as a chain of while nodes over shrinking launch grids (B, B/2,
    // B/4, ... entries), each sweep's CTAs mapped to the entries still
    // iterating through a live list that the loop control rebuilds after
    // every sweep, so converged entries stop costing CTAs.  Opt-in
    // (M3D_COMPACT=1): on the batch workload's grid-size groups (65-76% of
    // entry-sweeps live) it measured 0-2% slower than one loop over all B
    // entries, whose converged entries cost only early-exiting CTAs.
    bool use_compact = false;
    int* d_live = nullptr;  // [0] entries still iterating, [1..] their ids
    int Bl = 0;             // entries per launch grid while a compacted level is captured (0: B)
    int gridB() const { return Bl > 0 ? Bl : B; }
    std::vector<int> compact_levels() const {
        std::vector<int> lv;
        if (!use_compact || B < 4) return lv;
        lv.push_back(B);
        while (lv.back() > 2) lv.push_back((lv.back() + 1) / 2);
        return lv;
    }
    cudaError_t add_compacted_loop(const std::vector<int>& lv, const Ctl* ctl, int slot,
                                   std::vector<cudaGraph_t>& bodies, std::vector<cudaGraphConditionalHandle>& hs,
                                   cudaGraph_t owner);
    struct GraphSlot {
        cudaGraphExec_t exec = nullptr;
        long long key = -1;
    };
    GraphSlot gslot[3];  // 0: linear residual rule, 1: linear reference rule, 2: refinement
    int* d_trips = nullptr;  // [0] loop trips this run, [1] outer trips total, [2] inner trips this round, [3] inner total
    unsigned long long* d_pstat = nullptr;  // phase-map statistics: [0, 16) counts per id, [16] id sum, [17] first bad voxel
    int load_phase(int r, const int32_t* phase, int nph, std::vector<long long>& counts, long long& idsum,
                   long long& bad);
    void drop_graphs() {
        for (GraphSlot& s : gslot) {
            if (s.exec) cudaGraphExecDestroy(s.exec);
            s.exec = nullptr;
            s.key = -1;
        }
    }
    long long graph_key(int type) const {
        return (((((long long)type * 8192 + B) * 32 + nph_max()) * 2 + (use_fast ? 1 : 0)) * 4 + prec) * 2 +
               (use_slab ? 1 : 0);
    }
    template <typename T, int CC>
    int run_linear_graph(double tol_field, double tol_eq, int criterion, int max_iter);
    template <int CC>
    int run_refine_graph(double tol_field, int max_iter);
    template <typename T, int CC>
    int launch_em(Ctl* ctl, T* x, const float* r, typename Cx<T>::t* sp, int zero_k0, int policy, const Ctl* outer);
    int init_ctl(Ctl* dctl, double tol_field, double tol_eq, int max_iter, bool inner);
    int sync_ctl(Ctl* dctl);
    int dispatch_run(double tol_field, double tol_eq, int nInc, int criterion, int max_iter);
    int dispatch_core(double tol_field, double tol_eq, int nInc, int criterion, int max_iter);
    SpecGreen<double, 6> green_params_d6(int zero_k0) const;
    template <typename T, int CC> SpecGreen<T, CC> green(int zero_k0) const;
    template <typename T, int CC> int run_inelastic(double tol_field, double tol_eq, int nInc, int criterion, int max_iter);
};

m3d_solver::~m3d_solver() { free_all(); }

void m3d_solver::free_all() {
    drop_graphs();
    cudaFree(d_trips); d_trips = nullptr;
    cudaFree(d_err); d_err = nullptr;
    cudaFree(d_live); d_live = nullptr;
    cudaFree(d_pstat); d_pstat = nullptr;
    cudaFree(d_phase); d_phase = nullptr;
    cudaFree(d_x); d_x = nullptr;
    cudaFree(d_delta); d_delta = nullptr;
    cudaFree(d_r32); d_r32 = nullptr;
    cudaFree(d_spec); d_spec = nullptr;
    cudaFree(d_part); d_part = nullptr;
    cudaFree(d_ctl); d_ctl = nullptr;
    cudaFree(d_ctl_in); d_ctl_in = nullptr;
    cudaFree(d_counter); d_counter = nullptr;
    if (h_ctl) cudaFreeHost(h_ctl);
    h_ctl = nullptr;
    cudaFree(d_mats); d_mats = nullptr;
    cudaFree(d_tw64); d_tw64 = nullptr;
    cudaFree(d_tw32); d_tw32 = nullptr;
    cudaFree(d_out); d_out = nullptr;
    in.free_all();
}

int m3d_solver::alloc(int batch) {
    // (Re)allocate batch-sized buffers.  Phase map, tables and twiddles are
    // batch independent and allocated once.
    const long long V = g.V;
    const size_t specN = (size_t)batch * C * g.NL * g.Hzp;
    drop_graphs();  // captured launches hold the old buffers
    if (!d_trips) M3D_CUDA(cudaMalloc(&d_trips, 8 * sizeof(int)));
    if (!d_err) {
        M3D_CUDA(cudaMalloc(&d_err, sizeof(int)));
        M3D_CUDA(cudaMemset(d_err, 0, sizeof(int)));
    }
    ymap_base = nullptr;  // tensor maps name the old spectrum
    xmap_base = nullptr;
    cudaFree(d_x); cudaFree(d_delta); cudaFree(d_r32); cudaFree(d_spec); cudaFree(d_part);
    cudaFree(d_ctl); cudaFree(d_ctl_in);
    if (h_ctl) cudaFreeHost(h_ctl);
    d_x = nullptr; d_delta = nullptr; d_r32 = nullptr; d_spec = nullptr; d_part = nullptr;
    d_ctl = nullptr; d_ctl_in = nullptr; h_ctl = nullptr;
    const size_t xw = (prec == M3D_PREC_FP32) ? 4 : 8;
    M3D_CUDA(cudaMalloc(&d_x, (size_t)batch * C * V * xw));
    const size_t sw = (prec == M3D_PREC_FP32) ? 8 : 16;
    M3D_CUDA(cudaMalloc(&d_spec, specN * sw));
    M3D_CUDA(cudaMemsetAsync(d_spec, 0, specN * sw, stream));
    if (prec == M3D_PREC_FP32_REFINE) {
        M3D_CUDA(cudaMalloc(&d_delta, (size_t)batch * C * V * 4));
        M3D_CUDA(cudaMalloc(&d_r32, (size_t)batch * C * V * 4));
    }
    // partials: max over kernels of blocks x sums x batch
    const int Gmin = std::min(G32, G64);
    const size_t zblk = (size_t)((g.NL + Gmin - 1) / Gmin);
    const int TZmin = std::min(TZx32, TZx64);
    const size_t xblk = (size_t)Ny * ((g.Hzp + TZmin - 1) / TZmin);
    // (the pointwise kernels launch up to 592 blocks with up to 13 sums each;
    // the fast z passes use at least 2 lines per block, the x passes at least
    // one column per block)
    (void)zblk; (void)xblk;
    const size_t blk_max = std::max(std::max((size_t)(g.NL / 2 + 1), (size_t)Ny * g.Hzp), (size_t)1024);
    part_cap = blk_max * (size_t)batch * 16;
    M3D_CUDA(cudaMalloc(&d_part, part_cap * sizeof(double)));
    M3D_CUDA(cudaMalloc(&d_ctl, batch * sizeof(Ctl)));
    M3D_CUDA(cudaMalloc(&d_ctl_in, batch * sizeof(Ctl)));
    cudaFree(d_counter);
    d_counter = nullptr;
    M3D_CUDA(cudaMalloc(&d_counter, batch * sizeof(int)));
    M3D_CUDA(cudaMemsetAsync(d_counter, 0, batch * sizeof(int), stream));
    M3D_CUDA(cudaMemsetAsync(d_ctl, 0, batch * sizeof(Ctl), stream));
    M3D_CUDA(cudaMemsetAsync(d_ctl_in, 0, batch * sizeof(Ctl), stream));
    M3D_CUDA(cudaMallocHost(&h_ctl, batch * sizeof(Ctl)));
    cudaFree(d_live);
    d_live = nullptr;
    M3D_CUDA(cudaMalloc(&d_live, (size_t)(batch + 1) * sizeof(int)));
    alloc_B = batch;
    B = batch;
    E.assign((size_t)B * C, 0.0);
    X0.assign((size_t)B * 6, 0.0);
    return M3D_OK;
}

int m3d_solver::init_ctl(Ctl* dctl, double tol_field, double tol_eq, int max_iter, bool inner) {
    for (int b = 0; b < B; ++b) {
        const RveHost& m = rv[rve_of(b)];
        Ctl c;
        std::memset(&c, 0, sizeof(c));
        set_green(c, rve_of(b));
        c.max_iter = max_iter;
        c.tol_field = tol_field;
        c.tol_eq = tol_eq;
        double es = 0, en = 0;
        for (int i = 0; i < C; ++i) {
            const double e = E[b * C + i];
            c.E[i] = e;
            c.kzero[i] = e * (double)g.V;
            es += e;
            en += ((C == 6 && i >= 3) ? 2.0 : 1.0) * e * e;
        }
        c.enorm = std::sqrt(en);
        if (c.enorm == 0) c.enorm = 1;
        c.den = (double)g.V * m.den_ref * es;
        // sum of the "other" field at the initial uniform state (sum_field_old of the first sweep)
        double s0 = 0;
        for (int p = 0; p < m.nph; ++p) {
            double o = 0;
            for (int i = 0; i < C; ++i) o += m.hOsum[p * C + i] * E[b * C + i];
            s0 += (double)m.counts[p] * o;
        }
        c.sum_prev = s0;
        c.inner_tol = inner ? 1e-3 : 0;
        h_ctl[b] = c;
    }
    M3D_CUDA(cudaMemcpyAsync(dctl, h_ctl, B * sizeof(Ctl), cudaMemcpyHostToDevice, stream));
    return M3D_OK;
}

int m3d_solver::sync_ctl(Ctl* dctl) {
    M3D_CUDA(cudaMemcpyAsync(h_ctl, dctl, B * sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
    M3D_CUDA(cudaStreamSynchronize(stream));
    return M3D_OK;
}

// Green-operator constants of the current reference medium, kept per RVE
// (the kernels read them from each entry's control block).
void m3d_solver::snapshot_rve(int r) {
    RveHost& m = rv[r];
    m.set = true;
    m.diag = hP.size() >= (size_t)nph * C * C && hA.size() >= (size_t)nph * C * C;
    for (int p = 0; m.diag && p < nph; ++p)
        for (int i = 0; i < C; ++i)
            for (int j = 0; j < C; ++j)
                if (i != j && (hP[((size_t)p * C + i) * C + j] != 0.0 || hA[((size_t)p * C + i) * C + j] != 0.0))
                    m.diag = false;
    m.nph = nph;
    m.scheme = scheme;
    m.den_ref = den_ref;
    m.counts = counts;
    m.hOsum = hOsum;
    m.gxw = Nx;
    m.gnyq = 0;
    m.gp2 = 0;
    if (kind == M3D_KIND_MECH) {
        if (scheme == 1) {
            m.gkind = GREEN_STRAIN;
            m.gp1 = 1.0 / (2.0 * mu0);                      // 2*d1, d1 = 1/(4 mu0)   (src/3d/FFT_analysis3D.cpp:162)
            m.gp2 = (la0 + mu0) / (mu0 * (la0 + 2 * mu0));  // d2                     (:163)
        } else {
            m.gkind = GREEN_STRESS;
            const double c1 = 2 * mu0 * (3 * la0 + 2 * mu0) / (la0 + 2 * mu0), c2 = 2 * mu0;  // (:157-160)
            m.gp1 = (c1 - c2) / 2.0;
            m.gp2 = 2.0 * (c2 / 2.0);
        }
    } else {
        if (scheme == 1) {
            m.gkind = GREEN_TGRAD;
            m.gnyq = 1;  // src/3dTherm/FFT_thermal3D.cpp:113-120
            m.gp1 = 1.0 / k0;
        } else {
            m.gkind = GREEN_TFLUX;
            m.gxw = Ny;  // :151 wraps x with Ny
            m.gp1 = k0;
        }
    }
}

// The operator object; its kind and constants are taken from the control
// block of each entry (SpecGreen::prepare).
template <typename T, int CC>
SpecGreen<T, CC> m3d_solver::green(int zero_k0) const {
    SpecGreen<T, CC> s;
    s.g = g;
    s.zero_k0 = zero_k0;
    s.kind = rv[0].gkind;
    s.pos_nyq = rv[0].gnyq;
    s.xwrap = rv[0].gxw;
    s.p1 = (T)rv[0].gp1;
    s.p2 = (T)rv[0].gp2;
    return s;
}

template <int NN> struct IntC { static constexpr int value = NN; };
// Calls f(IntC<n>) when n has a compile-time specialised FFT.
template <class F> bool with_fast_n(int n, F&& f) {
    switch (n) {
        case 32: f(IntC<32>{}); return true;
        case 48: f(IntC<48>{}); return true;
        case 64: f(IntC<64>{}); return true;
        case 96: f(IntC<96>{}); return true;
        case 128: f(IntC<128>{}); return true;
        case 256: f(IntC<256>{}); return true;
        default: return false;
    }
}

template <typename T, int CC>
size_t m3d_solver::op_smem() const {
    return (size_t)nph_max() * std::max(sizeof(PhaseMech), (size_t)(CC * CC + CC) * sizeof(double)) + 64;
}

template <typename T, int CC, class Pro>
void m3d_solver::pass_zfwd(Pro pro, Ctl* ctl, typename Cx<T>::t* sp) {
    typedef typename Cx<T>::t C2;
    const size_t extra = op_smem<T, CC>();
    const bool done = use_fast && with_fast_n(Nz, [&](auto nc) {
        constexpr int NN = decltype(nc)::value;
        typedef ZTile<T, NN, CC> Z;
        allow_smem(k_zfwd_fast<T, NN, CC, Pro>);
        const int blk = (int)((g.NL + Z::G - 1) / Z::G);
        k_zfwd_fast<T, NN, CC, Pro><<<dim3(blk, gridB()), kFastThreads, z_fast_smem<T, NN, CC>(extra), stream>>>(
            g, tw<T>(2), sp, pro, ctl);
    });
    if (!done) {
        const int Gl = G<T>();
        const int zblk = (int)((g.NL + Gl - 1) / Gl);
        const size_t zsmem = (size_t)Nz * sizeof(C2) + 2 * (size_t)(Gl / 2) * CC * Nz * sizeof(C2) + 16 + 32 * 32 * 8 + extra;
        allow_smem(k_zfwd<T, CC, Pro>);
        k_zfwd<T, CC, Pro><<<dim3(zblk, gridB()), 256, zsmem, stream>>>(g, pz, tw<T>(2), sp, pro, ctl, Gl, d_part);
    }
    st.kernel_launches += 1;
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        (void)cudaGetLastError();
    });
    return fn;
}

// Tensor maps of the half spectrum for the TMA y pass: 2-D, rows of 2*Hzp
// scalars (one (batch, comp, x, y) line each), boxes 128 bytes wide and Ny rows
// high with the 128-byte swizzle.  False if TMA cannot be used for this shape.
bool m3d_solver::ensure_ymaps(int CC) {
    if (ymap_base == d_spec && ymap_B == B) return true;
    auto enc = tensor_map_encoder();
    const long long R = (long long)B * CC * Nx * Ny;
    if (!enc || R >= (1LL << 31) || Ny > 256 || !d_err) return false;
    for (int w = 0; w < 2; ++w) {
        const int sz = w ? 8 : 4;
        const cuuint64_t dims[2] = {(cuuint64_t)2 * g.Hzp, (cuuint64_t)R};
        const cuuint64_t strides[1] = {(cuuint64_t)g.Hzp * 2 * sz};
        const cuuint32_t box[2] = {(cuuint32_t)(128 / sz), (cuuint32_t)Ny};
        const cuuint32_t estr[2] = {1, 1};
        const CUresult r = enc(w ? &ymap64 : &ymap32, w ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                               d_spec, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
    }
    ymap_base = d_spec;
    ymap_B = B;
    return true;
}

// Tensor map of the FP32 half spectrum for the TMA-staged rank-one x
// turnaround: 3-D, (2*Hzp scalars, Ny rows, B*3*Nx lines), boxes of cpw
// complex columns x 1 row x Nx lines (one component of one work item).
bool m3d_solver::ensure_xmap(int cpw) {
    if (xmap_base == d_spec && xmap_B == B && xmap_cpw == cpw) return true;
    auto enc = tensor_map_encoder();
    const long long L = (long long)B * 3 * Nx;
    if (!enc || L >= (1LL << 31) || Nx > 256 || !d_err) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)2 * g.Hzp, (cuuint64_t)Ny, (cuuint64_t)L};
    const cuuint64_t strides[2] = {(cuuint64_t)g.Hzp * 8, (cuuint64_t)Ny * g.Hzp * 8};
    const cuuint32_t box[3] = {(cuuint32_t)(2 * cpw), 1, (cuuint32_t)Nx};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(&xmap32, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, d_spec, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    xmap_base = d_spec;
    xmap_B = B;
    xmap_cpw = cpw;
    return true;
}

template <typename T>
void m3d_solver::pass_y(int sign, int CC, Ctl* ctl, typename Cx<T>::t* sp) {
    typedef typename Cx<T>::t C2;
    const bool done = use_fast && with_fast_n(Ny, [&](auto nc) {
        constexpr int NN = decltype(nc)::value;
        constexpr int CPW = 32 / LineSplit<T, NN>::Tl;
        const int ntz = (g.Hzp + 4 * CPW - 1) / (4 * CPW);
        if (use_tma_y && ensure_ymaps(CC)) {
            typedef YTma<T, NN> Y;
            const int ntiles = CC * gridB() * Nx * ntz;
            auto kern = sign < 0 ? k_ypass_tma<T, NN, -1> : k_ypass_tma<T, NN, +1>;
            allow_smem(kern);
            int per_sm = 1, dev = 0, nsm = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFastThreads, Y::smem());
            const int grid = std::max(1, std::min(ntiles, nsm * std::max(per_sm, 1)));
            kern<<<grid, kFastThreads, Y::smem(), stream>>>(sizeof(T) == 8 ? ymap64 : ymap32, g, tw<T>(1), CC, ntiles,
                                                             ctl, d_err);
            return;
        }
        const dim3 grid(Nx * ntz, CC * gridB());
        const size_t sm = ypass_fast_smem<T, NN>();
        allow_smem(k_ypass_fast<T, NN, -1>);
        allow_smem(k_ypass_fast<T, NN, +1>);
        if (sign < 0) k_ypass_fast<T, NN, -1><<<grid, kFastThreads, sm, stream>>>(g, tw<T>(1), sp, CC, ctl);
        else k_ypass_fast<T, NN, +1><<<grid, kFastThreads, sm, stream>>>(g, tw<T>(1), sp, CC, ctl);
    });
    if (!done) {
        const int tzy = TZy<T>();
        const size_t ysmem = (size_t)Ny * sizeof(C2) + 2 * (size_t)Ny * tzy * sizeof(C2);
        const int ntzy = (g.Hzp + tzy - 1) / tzy;
        allow_smem(k_ypass<T>);
        k_ypass<T><<<dim3(Nx * ntzy, CC * gridB()), 256, ysmem, stream>>>(g, py, tw<T>(1), sp, tzy, CC, sign, ctl);
    }
    st.kernel_launches += 1;
}

template <typename T, int CC, class Spec>
int m3d_solver::pass_x(Spec op, Ctl* ctl, typename Cx<T>::t* sp) {
    typedef typename Cx<T>::t C2;
    int nblk = 0;
    const bool done = use_fast && with_fast_n(Nx, [&](auto nc) {
        constexpr int NN = decltype(nc)::value;
        constexpr int CPW = 32 / LineSplit<T, NN>::Tl;
        // (not FP64 at N = 96: its 24 points per lane spill at any register cap)
        if constexpr (CC == 3 && NN <= 128 && (sizeof(T) == 4 || NN != 96) &&
                      std::is_same<Spec, SpecGreen<T, 3>>::value) {
            if (use_xr1) {  // thermal Green operators in rank-one form; warp-granular (y, column group) items
                const int ngrp = (g.Hzp + CPW - 1) / CPW;
                if constexpr (sizeof(T) == 4) {
                    if (use_xr1_tma && (void*)sp == d_spec && ensure_xmap(CPW)) {  // column loads staged by TMA
                        typedef XR1Tma<T, NN> X;
                        auto kern = k_xturn_r1_tma<T, NN>;
                        allow_smem(kern);
                        static const int slots = [kern] {  // resident CTAs per SM x SMs
                            int per_sm = 1, dev = 0, nsm = 148;
                            cudaGetDevice(&dev);
                            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
                            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kXRegWarps * 32, X::smem());
                            (void)cudaGetLastError();
                            return std::max(1, per_sm) * nsm;
                        }();
                        const int nitems = gridB() * Ny * ngrp;
                        nblk = std::max(1, std::min((nitems + kXRegWarps - 1) / kXRegWarps, slots));
                        kern<<<nblk, kXRegWarps * 32, X::smem(), stream>>>(xmap32, g, tw<T>(0), sp, op, ctl, nitems, d_err);
                        return;
                    }
                }
                nblk = (Ny * ngrp + kXRegWarps - 1) / kXRegWarps;
                const size_t sm = (size_t)NN * sizeof(typename Cx<T>::t) +
                                  (size_t)kXRegWarps * CPW * RowLen<T, NN, true>::value * sizeof(typename Cx<T>::t);
                allow_smem(k_xturn_r1<T, NN>);
                k_xturn_r1<T, NN><<<dim3(nblk, gridB()), kXRegWarps * 32, sm, stream>>>(g, tw<T>(0), sp, op, ctl);
                return;
            }
        }
        if constexpr (CC == 3 && sizeof(T) == 4 && NN <= 64) {
            if (use_xreg) {  // the three components in registers (fits them without spilling up to N = 64)
                const int ntz = (g.Hzp + kXRegWarps * CPW - 1) / (kXRegWarps * CPW);
                nblk = Ny * ntz;
                allow_smem(k_xturn_reg<T, NN, Spec>);
                k_xturn_reg<T, NN, Spec><<<dim3(nblk, gridB()), kXRegWarps * 32, xturn_reg_smem<T, NN, Spec::NSUM>(), stream>>>(
                    g, tw<T>(0), sp, op, ctl, d_part);
                return;
            }
        }
        if constexpr (CC == 6 || CC == 3) {
            if (use_xcp) {  // one CTA of CC warps per column group, a warp per component
                const int ngrp = (g.Hzp + CPW - 1) / CPW;
                nblk = Ny * ngrp;
                allow_smem(k_xturn_cp<T, NN, CC, Spec>);
                k_xturn_cp<T, NN, CC, Spec><<<dim3(nblk, gridB()), 32 * CC, xturn_cp_smem<T, NN, CC, Spec::NSUM>(),
                                              stream>>>(g, tw<T>(0), sp, op, ctl, d_part);
                return;
            }
        }
        constexpr int WPC = XWarps<T, NN, CC>::value;
        const int ntz = (g.Hzp + WPC * CPW - 1) / (WPC * CPW);
        nblk = Ny * ntz;
        allow_smem(k_xturn_fast<T, NN, CC, Spec>);
        k_xturn_fast<T, NN, CC, Spec><<<dim3(nblk, gridB()), WPC * 32, xturn_fast_smem<T, NN, CC, Spec::NSUM>(), stream>>>(
            g, tw<T>(0), sp, op, ctl, d_part);
    });
    if (!done) {
        const int tzx = TZx<T>();
        const size_t xsmem = (size_t)Nx * sizeof(C2) + 2 * (size_t)CC * Nx * tzx * sizeof(C2) + 16 + 32 * 32 * 8;
        const int ntzx = (g.Hzp + tzx - 1) / tzx;
        nblk = Ny * ntzx;
        allow_smem(k_xturn<T, CC, Spec>);
        k_xturn<T, CC, Spec><<<dim3(nblk, gridB()), 256, xsmem, stream>>>(g, px, tw<T>(0), sp, tzx, op, ctl, d_part);
    }
    st.kernel_launches += 1;
    return nblk;
}

template <typename T, int CC, class Epi, class Fin>
int m3d_solver::pass_zinv(Epi epi, Ctl* ctl, typename Cx<T>::t* sp, Fin fin) {
    typedef typename Cx<T>::t C2;
    const size_t extra = op_smem<T, CC>();
    int nblk = 0;
    const bool done = use_fast && with_fast_n(Nz, [&](auto nc) {
        constexpr int NN = decltype(nc)::value;
        typedef ZTile<T, NN, CC> Z;
        nblk = (int)((g.NL + Z::G - 1) / Z::G);
        allow_smem(k_zinv_fast<T, NN, CC, Epi, Fin>);
        k_zinv_fast<T, NN, CC, Epi, Fin><<<dim3(nblk, gridB()), kFastThreads, zinv_fast_smem<T, NN, CC>(extra), stream>>>(
            g, tw<T>(2), sp, epi, ctl, d_part, fin);
    });
    if (!done) {
        const int Gl = G<T>();
        nblk = (int)((g.NL + Gl - 1) / Gl);
        const size_t zsmem = (size_t)Nz * sizeof(C2) + 2 * (size_t)(Gl / 2) * CC * Nz * sizeof(C2) + 16 + 32 * 32 * 8 + extra;
        allow_smem(k_zinv<T, CC, Epi, Fin>);
        k_zinv<T, CC, Epi, Fin><<<dim3(nblk, gridB()), 256, zsmem, stream>>>(g, pz, tw<T>(2), sp, epi, ctl, Gl, d_part, fin);
    }
    st.kernel_launches += 1;
    return nblk;
}

// One sweep; the finalize (sum of partials + stop rule) runs in the last
// block of the z-inverse pass.
template <typename T, int CC, class Pro, class Spec, class Epi>
int m3d_solver::launch_sweep(Pro pro, Spec spec, Epi epi, Ctl* ctl, typename Cx<T>::t* sp, int policy,
                             const Ctl* outer) {
    prof_pass(0);
    pass_zfwd<T, CC>(pro, ctl, sp);
    prof_pass(1);
    pass_y<T>(-1, CC, ctl, sp);
    prof_pass(2);
    pass_x<T, CC>(spec, ctl, sp);
    prof_pass(3);
    pass_y<T>(+1, CC, ctl, sp);
    prof_pass(4);
    pass_zinv<T, CC>(epi, ctl, sp, FinLinear{policy, (double)g.V, outer, d_counter});
    prof_pass(5);
    M3D_CUDA(cudaGetLastError());
    return M3D_OK;
}

// Reference stop rule: forward transform of the stress (heat flux) and the
// convergenceCheck reductions (src/3d/FFT_analysis3D.cpp:351-416).
template <typename T, int CC>
int m3d_solver::launch_check(Ctl* ctl, const void* x, typename Cx<T>::t* sp) {
    ProMat<T, CC> pro = tab(ProMat<T, CC>{d_phase, (const T*)x, g.V, dm(off_Q), nph_max(), nullptr});
    SpecEqVar<T, CC> sv{g};
    pass_zfwd<T, CC>(pro, ctl, sp);
    pass_y<T>(-1, CC, ctl, sp);
    const int xblk = pass_x<T, CC>(sv, ctl, sp);
    k_finalize<<<B, 256, 0, stream>>>(ctl, d_part, 2, xblk, POL_REF_CHECK, (double)g.V, nullptr);
    st.kernel_launches += 1;
    M3D_CUDA(cudaGetLastError());
    return M3D_OK;
}

template <typename T, int CC>
int m3d_solver::launch_em(Ctl* ctl, T* x, const float* r, typename Cx<T>::t* sp, int zero_k0, int policy,
                          const Ctl* outer) {
    ProMat<T, CC> pro = tab(ProMat<T, CC>{d_phase, x, g.V, dm(off_P), nph_max(), nullptr});
    EpiEM<T, CC> epi = tab(EpiEM<T, CC>{d_phase, x, r, g.V, dm(off_A), dm(off_Os), nph_max(), nullptr});
    return launch_sweep<T, CC>(pro, green<T, CC>(zero_k0), epi, ctl, sp, policy, outer);
}

// ---- two-pass sweeps: x turnaround + y-z slab pass (passes_slab.cuh) --------
// A slab instantiation is used where its shared memory leaves room for two
// CTAs per SM.
// CTA width of the slab pass: two 256-thread CTAs per SM (measured 56 us vs
// 60 us per launch at FP32 128^2 against one 512-thread CTA, which
// M3D_SLAB_NT=512 selects there)
template <typename T, int NN> constexpr int slab_nt_wide() { return (sizeof(T) == 4 && NN == 128) ? 512 : 256; }
template <typename T, int NN>
constexpr bool slab_fits() {
    return SlabGeom<T, NN, slab_nt_wide<T, NN>()>::fits();
}

template <typename T>
bool m3d_solver::slab_ok() const {
    if (!use_fast || !use_slab || Ny != Nz) return false;
    for (const RveHost& m : rv)
        if (!m.diag) return false;
    bool ok = false;
    with_fast_n(Nz, [&](auto nc) { ok = slab_fits<T, decltype(nc)::value>(); });
    return ok;
}

template <typename T, int CC, bool MIX, class Fin>
int m3d_solver::pass_slab(Ctl* ctl, T* x, const float* r, typename Cx<T>::t* sp, Fin fin) {
    SlabOps<T> ops{CC, d_phase, x, r, dm(off_P), dm(off_A), dm(off_Os), nph_max(), entries_per_rve(), mstride};
    bool done = false;
    with_fast_n(Nz, [&](auto nc) {
        constexpr int NN = decltype(nc)::value;
        if constexpr (slab_fits<T, NN>()) {
            constexpr int NTW = slab_nt_wide<T, NN>();
            if (NTW == 512 && slab_nt == 256 && SlabGeom<T, NN, 256>::fits()) {
                auto kern = k_slab<T, NN, 256, MIX, Fin>;
                allow_smem(kern);
                kern<<<dim3(CC * Nx, gridB()), 256, SlabGeom<T, NN, 256>::smem(), stream>>>(g, tw<T>(2), sp, ops, ctl, d_part,
                                                                                    fin);
            } else {
                auto kern = k_slab<T, NN, NTW, MIX, Fin>;
                allow_smem(kern);
                kern<<<dim3(CC * Nx, gridB()), NTW, SlabGeom<T, NN, NTW>::smem(), stream>>>(g, tw<T>(2), sp, ops, ctl, d_part,
                                                                                    fin);
            }
            done = true;
        }
    });
    if (!done) return fail(M3D_ERR_STATE, "slab pass requested for a grid without a slab kernel");
    st.kernel_launches += 1;
    M3D_CUDA(cudaGetLastError());
    return M3D_OK;
}

// One two-pass sweep; the finalize runs in the last CTA of the slab pass.
// Profiling slots: 2 = x turnaround, 4 = slab pass.
template <typename T, int CC>
int m3d_solver::launch_em_slab(Ctl* ctl, T* x, const float* r, typename Cx<T>::t* sp, int zero_k0, int policy,
                               const Ctl* outer) {
    prof_pass(0);
    prof_pass(1);
    prof_pass(2);
    pass_x<T, CC>(green<T, CC>(zero_k0), ctl, sp);
    prof_pass(3);
    prof_pass(4);
    const int rc = pass_slab<T, CC, true>(ctl, x, r, sp, FinLinear{policy, (double)g.V, outer, d_counter});
    prof_pass(5);
    return rc;
}

// Fill the state with the uniform load (setLoad, src/3d/FFT_analysis3D.cpp:551-564).
template <typename T>
__global__ void k_fill_load(T* x, const Ctl* ctl, int C, long long V) {
    const int cb = blockIdx.y;
    const int b = cb / C, c = cb % C;
    const T e = (T)ctl[b].E[c];
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x)
        x[(long long)cb * V + v] = e;
}

template <typename T, int CC>
int m3d_solver::run_linear(double tol_field, double tol_eq, int criterion, int max_iter) {
    typedef typename Cx<T>::t C2;
    int rc = init_ctl(d_ctl, tol_field, tol_eq, max_iter, false);
    if (rc) return rc;
    T* x = (T*)d_x;
    k_fill_load<T><<<dim3(256, B * CC), 256, 0, stream>>>(x, d_ctl, CC, g.V);
    st.kernel_launches += 1;
    C2* sp = (C2*)d_spec;
    const int chunk = kChunk;
    int before = 0;
    const bool slab = criterion == M3D_CRIT_RESIDUAL && slab_ok<T>();
    st.passes_per_sweep = slab ? 2 : 5;
    if (slab) {
        rc = pass_slab<T, CC, false>(d_ctl, x, nullptr, sp, FinNone{});
        if (rc) return rc;
    }
    for (;;) {
        for (int k = 0; k < chunk; ++k) {
            prof_mark(k);
            if (slab) {
                rc = launch_em_slab<T, CC>(d_ctl, x, nullptr, sp, 0, POL_RESIDUAL, nullptr);
            } else if (criterion == M3D_CRIT_RESIDUAL) {
                rc = launch_em<T, CC>(d_ctl, x, nullptr, sp, 0, POL_RESIDUAL, nullptr);
            } else {
                rc = launch_em<T, CC>(d_ctl, x, nullptr, sp, 0, POL_REF_SWEEP, nullptr);
                if (!rc) rc = launch_check<T, CC>(d_ctl, x, sp);
            }
            if (rc) return rc;
        }
        prof_mark(chunk);
        rc = sync_ctl(d_ctl);
        if (rc) return rc;
        prof_collect(max_iters() - before, sizeof(T) == 8);
        before = max_iters();
        bool all = true;
        for (int b = 0; b < B; ++b) all = all && h_ctl[b].done;
        if (all) break;
    }
    long long sw = 0;
    int status = M3D_OK;
    for (int b = 0; b < B; ++b) {
        sw += h_ctl[b].iters;
        if (h_ctl[b].status == 1 && status == M3D_OK) status = M3D_NOT_CONVERGED;
        if (h_ctl[b].status == 2) status = M3D_ERR_NAN;
    }
    st.sweeps = sw;
    if (sizeof(T) == 8) st.sweeps_fp64 = sw; else st.sweeps_fp32 = sw;
    st.iters = h_ctl[0].iters;
    st.residual = h_ctl[0].residual;
    st.eqvar = h_ctl[0].eqvar;
    st.diff_sum = h_ctl[0].diff_sum;
    st.diff_eq = h_ctl[0].diff_eq;
    return status;
}

// FP32 sweeps with FP64 defect correction (iterative refinement of the affine
// fixed point x = x_c(x)): each outer step evaluates r = x_c(x) - x in FP64,
// then solves delta = r + L(delta) by FP32 accelerated sweeps (k = 0 mode
// fixed to 0), and the next FP64 pass folds x += delta into its prologue.
template <int CC>
int m3d_solver::run_refine(double tol_field, int max_iter) {
    int rc = init_ctl(d_ctl, tol_field, 0, max_iter, false);
    if (rc) return rc;
    double* x = (double*)d_x;
    k_fill_load<double><<<dim3(256, B * CC), 256, 0, stream>>>(x, d_ctl, CC, g.V);
    st.kernel_launches += 1;
    double2* sp64 = (double2*)d_spec;
    float2* sp32 = (float2*)d_spec;
    long long n64 = 0, n32 = 0;
    bool first = true;
    const int chunk = 8;
    const bool slab = slab_ok<float>();
    st.passes_per_sweep = slab ? 2 : 5;
    std::vector<long long> in32((size_t)B, 0);  // FP32 sweeps per entry
    for (;;) {
        ProRefine64<CC> pro = tab(ProRefine64<CC>{d_phase, x, first ? nullptr : d_delta, g.V, dm(off_P), nph_max(), nullptr});
        EpiDefect<CC> epi = tab(EpiDefect<CC>{d_phase, x, d_r32, g.V, dm(off_Os), nph_max(), nullptr});
        prof_mark(0);
        rc = launch_sweep<double, CC>(pro, green<double, CC>(0), epi, d_ctl, sp64, POL_REFINE_OUTER, nullptr);
        if (rc) return rc;
        prof_mark(1);
        first = false;
        rc = sync_ctl(d_ctl);
        if (rc) return rc;
        prof_collect(1, true);
        bool all = true;
        for (int b = 0; b < B; ++b) all = all && h_ctl[b].done;
        if (all) break;
        // inner FP32 correction solve; entries already converged stay done
        std::vector<Ctl> outer(h_ctl, h_ctl + B);
        for (int b = 0; b < B; ++b) {
            Ctl c;
            std::memset(&c, 0, sizeof(c));
            set_green(c, rve_of(b));
            c.done = outer[b].done;
            c.max_iter = max_iter;
            c.inner_tol = refine_inner_tol(outer[b].tol_field, outer[b].residual);
            h_ctl[b] = c;
        }
        M3D_CUDA(cudaMemcpyAsync(d_ctl_in, h_ctl, B * sizeof(Ctl), cudaMemcpyHostToDevice, stream));
        M3D_CUDA(cudaMemsetAsync(d_delta, 0, (size_t)B * CC * g.V * sizeof(float), stream));
        // two-pass sweeps carry the forward spectrum from sweep to sweep; the
        // correction starts at 0, whose spectrum is 0
        if (slab) M3D_CUDA(cudaMemsetAsync(sp32, 0, (size_t)B * CC * g.NL * g.Hzp * sizeof(float2), stream));
        int before = 0;
        for (;;) {
            for (int k = 0; k < chunk; ++k) {
                prof_mark(k);
                if (slab) rc = launch_em_slab<float, CC>(d_ctl_in, d_delta, d_r32, sp32, 1, POL_REFINE_INNER, d_ctl);
                else rc = launch_em<float, CC>(d_ctl_in, d_delta, d_r32, sp32, 1, POL_REFINE_INNER, d_ctl);
                if (rc) return rc;
            }
            prof_mark(chunk);
            rc = sync_ctl(d_ctl_in);
            if (rc) return rc;
            prof_collect(max_iters() - before, false);
            before = max_iters();
            bool alli = true;
            for (int b = 0; b < B; ++b) alli = alli && h_ctl[b].done;
            if (alli) break;
        }
        for (int b = 0; b < B; ++b) {
            n32 += h_ctl[b].iters;
            in32[b] += h_ctl[b].iters;
        }
    }
    for (int b = 0; b < B; ++b) {
        n64 += h_ctl[b].iters;
        h_ctl[b].aux[1] = (double)in32[b];  // as the graph-captured loop counts them (m3d_get_entry_stats)
    }
    int status = M3D_OK;
    for (int b = 0; b < B; ++b) {
        if (h_ctl[b].status == 1 && status == M3D_OK) status = M3D_NOT_CONVERGED;
        if (h_ctl[b].status == 2) status = M3D_ERR_NAN;
    }
    st.sweeps = n64 + n32;
    st.sweeps_fp64 = n64;
    st.sweeps_fp32 = n32;
    st.iters = h_ctl[0].iters;
    st.residual = h_ctl[0].residual;
    return status;
}

// ---- graph-captured solves -------------------------------------------------------
// Loop control of a captured while node: continue while any entry of the batch
// is not done.  Every entry stops by its own rule or at its iteration cap; the
// trip count is a second cap on the loop itself.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, const Ctl* __restrict__ ctl, int B, int* trips, int slot) {
    int any = 0;
    for (int b = threadIdx.x; b < B; b += blockDim.x) any |= (ctl[b].done == 0);
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        const int t = ++trips[slot];
        ++trips[slot + 1];
        cudaGraphSetConditional(h, (any && t <= ctl[0].max_iter + 2) ? 1u : 0u);
    }
}

// One block rebuilds the live list from the control blocks: live[0] = the
// number of entries not done, live[1..] their ids in increasing order.
__device__ void build_live(const Ctl* __restrict__ ctl, int B, int* live) {
    __shared__ int wsum[32];
    __shared__ int base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (int c0 = 0; c0 < B; c0 += blockDim.x) {
        const int b = c0 + threadIdx.x;
        const bool f = b < B && !ctl[b].done;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) wsum[warp] = __popc(m);
        __syncthreads();
        int off = base;
        for (int w = 0; w < warp; ++w) off += wsum[w];
        if (f) live[1 + off + __popc(m & ((1u << lane) - 1u))] = b;
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int w = 0; w < nw; ++w) tot += wsum[w];
            base += tot;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) live[0] = base;
}

// Entry into a level of a compacted loop: rebuild the live list and run the
// level while more entries iterate than the next level's grid holds (thr).
__global__ void k_live_arm(cudaGraphConditionalHandle h, const Ctl* __restrict__ ctl, int B, int* live, int thr,
                           const int* trips, int slot) {
    build_live(ctl, B, live);
    __syncthreads();
    if (threadIdx.x == 0)
        cudaGraphSetConditional(h, (live[0] > thr && trips[slot] <= ctl[0].max_iter + 2) ? 1u : 0u);
}

// Loop control of a level of a compacted loop: count the sweep, rebuild the
// live list for the next one, and stay on this level while more than thr
// entries iterate.
__global__ void k_loop_cond_live(cudaGraphConditionalHandle h, const Ctl* __restrict__ ctl, int B, int* live,
                                 int thr, int* trips, int slot) {
    build_live(ctl, B, live);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int t = ++trips[slot];
        ++trips[slot + 1];
        cudaGraphSetConditional(h, (live[0] > thr && t <= ctl[0].max_iter + 2) ? 1u : 0u);
    }
}

// Between the FP64 defect sweep and the FP32 correction solve of the
// refinement: count the inner sweeps of the previous round (aux[1]), give
// every entry a fresh inner control block (the entries already converged stay
// done) and arm both loops.
__global__ void k_refine_mid(cudaGraphConditionalHandle h_outer, cudaGraphConditionalHandle h_inner, Ctl* ctl,
                             Ctl* ctl_in, int B, int* trips) {
    int any = 0;
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        Ctl& o = ctl[b];
        o.aux[1] += (double)ctl_in[b].iters;
        Ctl c;
        memset(&c, 0, sizeof(c));
        c.gkind = o.gkind; c.gnyq = o.gnyq; c.gxw = o.gxw; c.gp1 = o.gp1; c.gp2 = o.gp2;
        c.done = o.done;
        c.max_iter = o.max_iter;
        c.inner_tol = refine_inner_tol(o.tol_field, o.residual);
        ctl_in[b] = c;
        any |= (o.done == 0);
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        const int t = ++trips[0];
        ++trips[1];
        trips[2] = 0;
        const unsigned go = (any && t <= ctl[0].max_iter + 2) ? 1u : 0u;
        cudaGraphSetConditional(h_outer, go);
        cudaGraphSetConditional(h_inner, go);
    }
}

// A while node appended to `graph` after `deps`; returns its body graph.
static cudaError_t add_while(cudaGraph_t graph, const cudaGraphNode_t* deps, size_t ndeps,
                             cudaGraphConditionalHandle h, cudaGraphNode_t* node, cudaGraph_t* body) {
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};  // the remaining members are zero
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(node, graph, deps, ndeps, &p);
    if (e == cudaSuccess) *body = p.conditional.phGraph_out[0];
    return e;
}

// Appends to the graph being captured on the solver's stream the levels of a
// compacted loop: per level k, a kernel that rebuilds the live list and arms
// the level's while node (handle created on `owner`, the graph holding the
// nodes), then the node.  The level bodies are returned for capture once the
// enclosing capture has ended.
cudaError_t m3d_solver::add_compacted_loop(const std::vector<int>& lv, const Ctl* ctl, int slot,
                                           std::vector<cudaGraph_t>& bodies,
                                           std::vector<cudaGraphConditionalHandle>& hs, cudaGraph_t owner) {
    for (size_t k = 0; k < lv.size(); ++k) {
        cudaGraphConditionalHandle h;
        cudaError_t e = cudaGraphConditionalHandleCreate(&h, owner, 0, 0);
        if (e != cudaSuccess) return e;
        const int thr = k + 1 < lv.size() ? lv[k + 1] : 0;
        k_live_arm<<<1, 256, 0, stream>>>(h, ctl, B, d_live, thr, d_trips, slot);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        cudaStreamCaptureStatus cs;
        cudaGraph_t capg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        e = cudaStreamGetCaptureInfo(stream, &cs, nullptr, &capg, &deps, &nd);
        if (e != cudaSuccess) return e;
        cudaGraphNode_t node;
        cudaGraph_t body = nullptr;
        e = add_while(capg, deps, nd, h, &node, &body);
        if (e != cudaSuccess) return e;
        e = cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies);
        if (e != cudaSuccess) return e;
        bodies.push_back(body);
        hs.push_back(h);
    }
    return cudaSuccess;
}

// Launch grids over the live list while a compacted level is captured.
struct CompactScope {
    m3d_solver* s;
    CompactScope(m3d_solver* s_, int entries) : s(s_) {
        s->Bl = entries;
        s->g.live = s->d_live;
    }
    ~CompactScope() {
        s->Bl = 0;
        s->g.live = nullptr;
    }
};

#define M3D_CAP(call)                                                         \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) {                                              \
            cudaGraph_t junk_ = nullptr;                                      \
            cudaStreamEndCapture(stream, &junk_);                             \
            if (junk_) cudaGraphDestroy(junk_);                               \
            cudaGraphDestroy(top);                                            \
            (void)cudaGetLastError();                                         \
            return fail(M3D_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e_)); \
        }                                                                     \
    } while (0)

template <typename T, int CC>
int m3d_solver::run_linear_graph(double tol_field, double tol_eq, int criterion, int max_iter) {
    typedef typename Cx<T>::t C2;
    int rc = init_ctl(d_ctl, tol_field, tol_eq, max_iter, false);
    if (rc) return rc;
    T* x = (T*)d_x;
    C2* sp = (C2*)d_spec;
    k_fill_load<T><<<dim3(256, B * CC), 256, 0, stream>>>(x, d_ctl, CC, g.V);
    M3D_CUDA(cudaMemsetAsync(d_trips, 0, 8 * sizeof(int), stream));
    const bool resid = (criterion == M3D_CRIT_RESIDUAL);
    const bool slab = resid && slab_ok<T>();
    st.passes_per_sweep = slab ? 2 : 5;
    if (slab) {
        rc = pass_slab<T, CC, false>(d_ctl, x, nullptr, sp, FinNone{});
        if (rc) return rc;
    }
    GraphSlot& gs = gslot[resid ? 0 : 1];
    const long long key = graph_key(resid ? 0 : 1);
    const std::vector<int> lv = resid ? compact_levels() : std::vector<int>();
    if (gs.key != key) {
        drop_graphs();
        cudaGraph_t top = nullptr;
        M3D_CUDA(cudaGraphCreate(&top, 0));
        const long long kl = st.kernel_launches;  // captured launches are counted per executed trip below
        cudaGraph_t got = nullptr;
        if (!lv.empty()) {
            // compacted: one while node per launch-grid level
            std::vector<cudaGraph_t> bodies;
            std::vector<cudaGraphConditionalHandle> hs;
            M3D_CAP(cudaStreamBeginCaptureToGraph(stream, top, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            M3D_CAP(add_compacted_loop(lv, d_ctl, 0, bodies, hs, top));
            M3D_CAP(cudaStreamEndCapture(stream, &got));
            for (size_t k = 0; k < lv.size(); ++k) {
                M3D_CAP(cudaStreamBeginCaptureToGraph(stream, bodies[k], nullptr, nullptr, 0,
                                                      cudaStreamCaptureModeRelaxed));
                {
                    CompactScope scope(this, lv[k]);
                    rc = slab ? launch_em_slab<T, CC>(d_ctl, x, nullptr, sp, 0, POL_RESIDUAL, nullptr)
                              : launch_em<T, CC>(d_ctl, x, nullptr, sp, 0, POL_RESIDUAL, nullptr);
                }
                if (rc) M3D_CAP(cudaErrorUnknown);
                k_loop_cond_live<<<1, 256, 0, stream>>>(hs[k], d_ctl, B, d_live, k + 1 < lv.size() ? lv[k + 1] : 0,
                                                        d_trips, 0);
                M3D_CAP(cudaGetLastError());
                M3D_CAP(cudaStreamEndCapture(stream, &got));
            }
        } else {
            cudaGraphConditionalHandle h;
            cudaGraphNode_t node;
            cudaGraph_t body = nullptr;
            M3D_CAP(cudaGraphConditionalHandleCreate(&h, top, 1, cudaGraphCondAssignDefault));
            M3D_CAP(add_while(top, nullptr, 0, h, &node, &body));
            M3D_CAP(cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            if (slab) {
                rc = launch_em_slab<T, CC>(d_ctl, x, nullptr, sp, 0, POL_RESIDUAL, nullptr);
            } else if (resid) {
                rc = launch_em<T, CC>(d_ctl, x, nullptr, sp, 0, POL_RESIDUAL, nullptr);
            } else {
                rc = launch_em<T, CC>(d_ctl, x, nullptr, sp, 0, POL_REF_SWEEP, nullptr);
                if (!rc) rc = launch_check<T, CC>(d_ctl, x, sp);
            }
            if (rc) M3D_CAP(cudaErrorUnknown);
            k_loop_cond<<<1, 256, 0, stream>>>(h, d_ctl, B, d_trips, 0);
            M3D_CAP(cudaGetLastError());
            M3D_CAP(cudaStreamEndCapture(stream, &got));
        }
        st.kernel_launches = kl;
        cudaError_t e = cudaGraphInstantiate(&gs.exec, top, 0);
        cudaGraphDestroy(top);
        if (e != cudaSuccess) { gs.exec = nullptr; return fail(M3D_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); }
        gs.key = key;
    }
    M3D_CUDA(cudaGraphLaunch(gs.exec, stream));
    rc = sync_ctl(d_ctl);
    if (rc) return rc;
    int trips[8];
    M3D_CUDA(cudaMemcpy(trips, d_trips, sizeof(trips), cudaMemcpyDeviceToHost));
    st.kernel_launches += 1 + (long long)lv.size() + (long long)trips[0] * (slab ? 3 : (resid ? 6 : 10));
    long long sw = 0;
    int status = M3D_OK;
    for (int b = 0; b < B; ++b) {
        sw += h_ctl[b].iters;
        if (h_ctl[b].status == 1 && status == M3D_OK) status = M3D_NOT_CONVERGED;
        if (h_ctl[b].status == 2) status = M3D_ERR_NAN;
    }
    st.sweeps = sw;
    if (sizeof(T) == 8) { st.sweeps_fp64 = sw; st.sweeps_fp32 = 0; } else { st.sweeps_fp32 = sw; st.sweeps_fp64 = 0; }
    st.iters = h_ctl[0].iters;
    st.residual = h_ctl[0].residual;
    st.eqvar = h_ctl[0].eqvar;
    st.diff_sum = h_ctl[0].diff_sum;
    st.diff_eq = h_ctl[0].diff_eq;
    return status;
}

template <int CC>
int m3d_solver::run_refine_graph(double tol_field, int max_iter) {
    int rc = init_ctl(d_ctl, tol_field, 0, max_iter, false);
    if (rc) return rc;
    double* x = (double*)d_x;
    double2* sp64 = (double2*)d_spec;
    float2* sp32 = (float2*)d_spec;
    const size_t dbytes = (size_t)B * CC * g.V * sizeof(float);
    k_fill_load<double><<<dim3(256, B * CC), 256, 0, stream>>>(x, d_ctl, CC, g.V);
    M3D_CUDA(cudaMemsetAsync(d_delta, 0, dbytes, stream));
    M3D_CUDA(cudaMemsetAsync(d_ctl_in, 0, (size_t)B * sizeof(Ctl), stream));
    M3D_CUDA(cudaMemsetAsync(d_trips, 0, 8 * sizeof(int), stream));
    const bool slab = slab_ok<float>();
    st.passes_per_sweep = slab ? 2 : 5;
    const size_t sbytes32 = (size_t)B * CC * g.NL * g.Hzp * sizeof(float2);
    GraphSlot& gs = gslot[2];
    const long long key = graph_key(2);
    const std::vector<int> lv = compact_levels();  // levels of the compacted inner loop (none: one loop)
    if (gs.key != key) {
        drop_graphs();
        cudaGraph_t top = nullptr;
        M3D_CUDA(cudaGraphCreate(&top, 0));
        cudaGraphConditionalHandle h_out, h_in;
        cudaGraphNode_t n_out, n_in;
        cudaGraph_t b_out = nullptr, b_in = nullptr;
        M3D_CAP(cudaGraphConditionalHandleCreate(&h_out, top, 1, cudaGraphCondAssignDefault));
        M3D_CAP(add_while(top, nullptr, 0, h_out, &n_out, &b_out));
        // one inner loop: its handle, armed with the outer one; compacted: the
        // levels arm their own handles (the outer one stands in here)
        if (lv.empty()) M3D_CAP(cudaGraphConditionalHandleCreate(&h_in, b_out, 0, 0));
        else h_in = h_out;
        const long long kl = st.kernel_launches;  // captured launches are counted per executed trip below
        // outer body: FP64 defect sweep (folds in the previous correction),
        // loop control, cleared correction, then the inner while node(s)
        M3D_CAP(cudaStreamBeginCaptureToGraph(stream, b_out, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        ProRefine64<CC> pro = tab(ProRefine64<CC>{d_phase, x, d_delta, g.V, dm(off_P), nph_max(), nullptr});
        EpiDefect<CC> epi = tab(EpiDefect<CC>{d_phase, x, d_r32, g.V, dm(off_Os), nph_max(), nullptr});
        rc = launch_sweep<double, CC>(pro, green<double, CC>(0), epi, d_ctl, sp64, POL_REFINE_OUTER, nullptr);
        if (rc) M3D_CAP(cudaErrorUnknown);
        k_refine_mid<<<1, 256, 0, stream>>>(h_out, h_in, d_ctl, d_ctl_in, B, d_trips);
        M3D_CAP(cudaGetLastError());
        M3D_CAP(cudaMemsetAsync(d_delta, 0, dbytes, stream));
        // two-pass sweeps: the correction starts at 0, whose spectrum is 0
        if (slab) M3D_CAP(cudaMemsetAsync(sp32, 0, sbytes32, stream));
        std::vector<cudaGraph_t> bodies;
        std::vector<cudaGraphConditionalHandle> hs;
        if (!lv.empty()) {
            M3D_CAP(add_compacted_loop(lv, d_ctl_in, 2, bodies, hs, b_out));
        } else {
            cudaStreamCaptureStatus cs;
            cudaGraph_t capg = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            M3D_CAP(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &capg, &deps, &nd));
            M3D_CAP(add_while(capg, deps, nd, h_in, &n_in, &b_in));
            M3D_CAP(cudaStreamUpdateCaptureDependencies(stream, &n_in, 1, cudaStreamSetCaptureDependencies));
            bodies.push_back(b_in);
            hs.push_back(h_in);
        }
        cudaGraph_t got = nullptr;
        M3D_CAP(cudaStreamEndCapture(stream, &got));
        // inner bodies: FP32 correction sweep + loop control (one per level)
        for (size_t k = 0; k < bodies.size(); ++k) {
            M3D_CAP(cudaStreamBeginCaptureToGraph(stream, bodies[k], nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeRelaxed));
            if (!lv.empty()) {
                {
                    CompactScope scope(this, lv[k]);
                    rc = slab ? launch_em_slab<float, CC>(d_ctl_in, d_delta, d_r32, sp32, 1, POL_REFINE_INNER, d_ctl)
                              : launch_em<float, CC>(d_ctl_in, d_delta, d_r32, sp32, 1, POL_REFINE_INNER, d_ctl);
                }
                if (rc) M3D_CAP(cudaErrorUnknown);
                k_loop_cond_live<<<1, 256, 0, stream>>>(hs[k], d_ctl_in, B, d_live,
                                                        k + 1 < lv.size() ? lv[k + 1] : 0, d_trips, 2);
            } else {
                rc = slab ? launch_em_slab<float, CC>(d_ctl_in, d_delta, d_r32, sp32, 1, POL_REFINE_INNER, d_ctl)
                          : launch_em<float, CC>(d_ctl_in, d_delta, d_r32, sp32, 1, POL_REFINE_INNER, d_ctl);
                if (rc) M3D_CAP(cudaErrorUnknown);
                k_loop_cond<<<1, 256, 0, stream>>>(hs[k], d_ctl_in, B, d_trips, 2);
            }
            M3D_CAP(cudaGetLastError());
            M3D_CAP(cudaStreamEndCapture(stream, &got));
        }
        st.kernel_launches = kl;
        cudaError_t e = cudaGraphInstantiate(&gs.exec, top, 0);
        cudaGraphDestroy(top);
        if (e != cudaSuccess) { gs.exec = nullptr; return fail(M3D_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); }
        gs.key = key;
    }
    M3D_CUDA(cudaGraphLaunch(gs.exec, stream));
    rc = sync_ctl(d_ctl);
    if (rc) return rc;
    int trips[8];
    M3D_CUDA(cudaMemcpy(trips, d_trips, sizeof(trips), cudaMemcpyDeviceToHost));
    st.kernel_launches += 1 + (long long)trips[1] * (6 + (long long)lv.size()) + (long long)trips[3] * (slab ? 3 : 6);
    long long n64 = 0, n32 = 0;
    int status = M3D_OK;
    for (int b = 0; b < B; ++b) {
        n64 += h_ctl[b].iters;
        n32 += (long long)h_ctl[b].aux[1];
        if (h_ctl[b].status == 1 && status == M3D_OK) status = M3D_NOT_CONVERGED;
        if (h_ctl[b].status == 2) status = M3D_ERR_NAN;
    }
    st.sweeps = n64 + n32;
    st.sweeps_fp64 = n64;
    st.sweeps_fp32 = n32;
    st.iters = h_ctl[0].iters;
    st.residual = h_ctl[0].residual;
    return status;
}
#undef M3D_CAP

int m3d_solver::dispatch_run(double tol_field, double tol_eq, int nInc, int criterion, int max_iter) {
    int rc = dispatch_core(tol_field, tol_eq, nInc, criterion, max_iter);
    if (d_err) {  // the TMA-staged passes' bounded waits
        int e = 0;
        if (cudaMemcpy(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && e) {
            cudaMemset(d_err, 0, sizeof(int));
            return fail(M3D_ERR_TIMEOUT, "a TMA pipeline wait expired on the device; results are invalid");
        }
    }
    return rc;
}

int m3d_solver::dispatch_core(double tol_field, double tol_eq, int nInc, int criterion, int max_iter) {
    if (max_iter <= 0) max_iter = (kind == M3D_KIND_MECH) ? 2000 : 500;
    st.passes_per_sweep = 5;
    if (kind == M3D_KIND_MECH && behav != M3D_BEHAV_ELASTIC) {
        if (prec == M3D_PREC_FP32_REFINE)
            return fail(M3D_ERR_UNSUPPORTED, "FP32 refinement applies to the linear (elastic/thermal) solves; use FP32 or FP64 for ep/ed");
        if (prec == M3D_PREC_FP64) return run_inelastic<double, 6>(tol_field, tol_eq, nInc, criterion, max_iter);
        return run_inelastic<float, 6>(tol_field, tol_eq, nInc, criterion, max_iter);
    }
    const bool graph = use_graph && !prof;  // per-sweep event timing needs the host-driven loop
    if (prec == M3D_PREC_FP32_REFINE) {
        if (criterion != M3D_CRIT_RESIDUAL)
            return fail(M3D_ERR_UNSUPPORTED, "FP32 refinement stops on the residual criterion only");
        if (graph) return C == 6 ? run_refine_graph<6>(tol_field, max_iter) : run_refine_graph<3>(tol_field, max_iter);
        return C == 6 ? run_refine<6>(tol_field, max_iter) : run_refine<3>(tol_field, max_iter);
    }
    if (graph) {
        if (prec == M3D_PREC_FP64)
            return C == 6 ? run_linear_graph<double, 6>(tol_field, tol_eq, criterion, max_iter)
                          : run_linear_graph<double, 3>(tol_field, tol_eq, criterion, max_iter);
        return C == 6 ? run_linear_graph<float, 6>(tol_field, tol_eq, criterion, max_iter)
                      : run_linear_graph<float, 3>(tol_field, tol_eq, criterion, max_iter);
    }
    if (prec == M3D_PREC_FP64)
        return C == 6 ? run_linear<double, 6>(tol_field, tol_eq, criterion, max_iter)
                      : run_linear<double, 3>(tol_field, tol_eq, criterion, max_iter);
    return C == 6 ? run_linear<float, 6>(tol_field, tol_eq, criterion, max_iter)
                  : run_linear<float, 3>(tol_field, tol_eq, criterion, max_iter);
}

// ---- exports ----------------------------------------------------------------
// out[v*C + c] = (M[ph] x)_c  (M = identity when mats == nullptr)
template <typename TX, int CC>
__global__ void k_export(const TX* __restrict__ x, const uint8_t* __restrict__ phase, const double* __restrict__ mats,
                         int b, long long V, double* __restrict__ out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        double xv[CC];
#pragma unroll
        for (int c = 0; c < CC; ++c) xv[c] = (double)x[((long long)b * CC + c) * V + v];
        if (mats) {
            const double* M = mats + phase[v] * CC * CC;
#pragma unroll
            for (int i = 0; i < CC; ++i) {
                double s = 0;
#pragma unroll
                for (int j = 0; j < CC; ++j) s += M[i * CC + j] * xv[j];
                out[v * CC + i] = s;
            }
        } else {
#pragma unroll
            for (int c = 0; c < CC; ++c) out[v * CC + c] = xv[c];
        }
    }
}

template <typename TX, int CC>
static int export_field(m3d_solver* h, const void* x, const double* mats, int b, double* host_out,
                        bool async = false) {
    const long long V = h->g.V;
    if (!h->d_out) {
        cudaError_t e = cudaMalloc(&h->d_out, (size_t)6 * V * sizeof(double));
        if (e != cudaSuccess) return fail(M3D_ERR_OOM, "export buffer allocation failed");
    }
    if (h->d2h_pending) M3D_CUDA(cudaStreamWaitEvent(h->stream, h->ev_d2h, 0));  // the pending copy reads d_out
    const int r = h->rve_of(b);
    const double* M = mats ? mats + (size_t)r * h->mstride : nullptr;
    k_export<TX, CC><<<592, 256, 0, h->stream>>>((const TX*)x, h->d_phase + (size_t)r * V, M, b, V, h->d_out);
    h->st.kernel_launches += 1;
    M3D_CUDA(cudaGetLastError());
    const size_t bytes = (size_t)CC * V * sizeof(double);
    if (!async) {
        M3D_CUDA(cudaMemcpyAsync(host_out, h->d_out, bytes, cudaMemcpyDeviceToHost, h->stream));
        M3D_CUDA(cudaStreamSynchronize(h->stream));
        h->d2h_pending = false;
        return M3D_OK;
    }
    if (!h->xstream) {
        M3D_CUDA(cudaStreamCreateWithFlags(&h->xstream, cudaStreamNonBlocking));
        M3D_CUDA(cudaEventCreateWithFlags(&h->ev_exp, cudaEventDisableTiming));
        M3D_CUDA(cudaEventCreateWithFlags(&h->ev_d2h, cudaEventDisableTiming));
    }
    M3D_CUDA(cudaEventRecord(h->ev_exp, h->stream));
    M3D_CUDA(cudaStreamWaitEvent(h->xstream, h->ev_exp, 0));
    M3D_CUDA(cudaMemcpyAsync(host_out, h->d_out, bytes, cudaMemcpyDeviceToHost, h->xstream));
    M3D_CUDA(cudaEventRecord(h->ev_d2h, h->xstream));
    h->d2h_pending = true;
    return M3D_OK;
}

#include "solver_inelastic.inl"

// Lets the allocation-free entry point (noalloc.cu) report through m3d_last_error().
void m3d_internal_set_error(const std::string& msg) { g_last_error = msg; }

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

int m3d_abi_version(void) { return M3D_ABI_VERSION; }

const char* m3d_last_error(void) { return g_last_error.c_str(); }

const char* m3d_status_string(int s) {
    switch (s) {
        case M3D_OK: return "ok";
        case M3D_ERR_ARG: return "invalid argument";
        case M3D_ERR_CUDA: return "CUDA error";
        case M3D_ERR_OOM: return "device out of memory";
        case M3D_NOT_CONVERGED: return "not converged (iteration cap)";
        case M3D_ERR_NAN: return "non-finite residual";
        case M3D_ERR_STATE: return "call order violated";
        case M3D_ERR_UNSUPPORTED: return "unsupported";
        case M3D_ERR_TIMEOUT: return "device wait timed out";
        case M3D_PENDING: return "pending";
        default: return "unknown status";
    }
}

static void table_layout(m3d_solver* h);

static int create_impl(int kind, int Nx, int Ny, int Nz, int behav, int precision, int nrve, int batch,
                       m3d_solver** out) {
    if (!out) return fail(M3D_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (kind != M3D_KIND_MECH && kind != M3D_KIND_THERMAL) return fail(M3D_ERR_ARG, "kind must be MECH or THERMAL");
    if (Nx < 2 || Ny < 2 || Nz < 2 || Nx > 1024 || Ny > 1024 || Nz > 1024)
        return fail(M3D_ERR_ARG, "grid sizes must be in [2, 1024]");
    if (behav < 0 || behav > 2 || (kind == M3D_KIND_THERMAL && behav != 0)) return fail(M3D_ERR_ARG, "invalid behaviour");
    if (precision < 0 || precision > 2) return fail(M3D_ERR_ARG, "invalid precision");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(M3D_ERR_CUDA, "no CUDA device");
    m3d_solver* h = new m3d_solver();
    h->nrve = nrve;
    h->rv.assign(nrve, m3d_solver::RveHost{});
    h->kind = kind;
    h->behav = behav;
    h->prec = precision;
    h->C = (kind == M3D_KIND_MECH) ? 6 : 3;
    h->Nx = Nx; h->Ny = Ny; h->Nz = Nz;
    h->g.Nx = Nx; h->g.Ny = Ny; h->g.Nz = Nz;
    h->g.Hz = Nz / 2 + 1;
    h->g.Hzp = even_up(Nz / 2 + 1);
    h->g.V = (long long)Nx * Ny * Nz;
    h->g.NL = (long long)Nx * Ny;
    // M3D_FFT_SCHEDULE=<0..3>: the generic line FFTs' radix-stage order (make_plan)
    const char* esch = std::getenv("M3D_FFT_SCHEDULE");
    const int sched = esch ? std::max(0, std::min(kPlanOrders - 1, std::atoi(esch))) : 0;
    if (!make_plan(Nx, h->px, false, sched) || !make_plan(Ny, h->py, false, sched) || !make_plan(Nz, h->pz, false, sched)) {
        delete h;
        return fail(M3D_ERR_UNSUPPORTED, "grid sizes need prime factors <= 32");
    }
    // launch geometry: z passes hold G lines x C components (ping-pong) in ~48 KB,
    // y tiles TZ columns of 128 B rows, x tiles all C components in ~64 KB
    auto pick_G = [&](size_t csz) {
        int Gv = (int)(48 * 1024 / ((size_t)h->C * Nz * csz));
        Gv = std::max(2, std::min(16, Gv)) & ~1;
        return Gv;
    };
    h->G64 = pick_G(16);
    h->G32 = pick_G(8);
    auto pick_tz = [&](size_t csz, int ncomp, int n, int maxtz) {
        int tz = maxtz;
        while (tz > 1 && 2 * (size_t)ncomp * n * tz * csz > 64 * 1024) tz >>= 1;
        return tz;
    };
    h->TZy64 = pick_tz(16, 1, Ny, 8);
    h->TZy32 = pick_tz(8, 1, Ny, 16);
    h->TZx64 = pick_tz(16, h->C, Nx, 8);
    h->TZx32 = pick_tz(8, h->C, Nx, 16);
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete h; return fail(M3D_ERR_CUDA, cudaGetErrorString(e)); }
    h->own_stream = h->stream;
    {
        const char* e2 = std::getenv("M3D_GENERIC_FFT");
        h->use_fast = !(e2 && e2[0] == '1');
        const char* e3 = std::getenv("M3D_NO_GRAPH");
        h->use_graph = !(e3 && e3[0] == '1');
        const char* e10 = std::getenv("M3D_COMPACT");
        h->use_compact = e10 && e10[0] == '1';
        const char* e4 = std::getenv("M3D_TMA_Y");
        h->use_tma_y = (e4 && e4[0] == '1');
        const char* e5 = std::getenv("M3D_NO_SLAB");
        h->use_slab = !(e5 && e5[0] == '1');
        const char* e7 = std::getenv("M3D_SLAB_NT");
        h->slab_nt = (e7 && std::atoi(e7) == 512) ? 512 : 256;
        const char* e8 = std::getenv("M3D_XTURN_R1");
        h->use_xr1 = !(e8 && e8[0] == '0');
        const char* e9 = std::getenv("M3D_XTURN_TMA");
        h->use_xr1_tma = !(e9 && e9[0] == '0');
        const char* e11 = std::getenv("M3D_XTURN_CP");
        h->use_xcp = !(e11 && e11[0] == '0');
        const char* e6 = std::getenv("M3D_XTURN_STAGED");
        h->use_xreg = !(e6 && e6[0] == '1');
    }
    int rc = h->alloc(batch);
    if (rc) { cudaStreamDestroy(h->stream); delete h; return rc; }
    // twiddles
    {
        std::vector<double2> t64;
        std::vector<float2> t32;
        for (int n : {Nx, Ny, Nz}) {
            auto a = twiddles<double>(n);
            auto b2 = twiddles<float>(n);
            t64.insert(t64.end(), a.begin(), a.end());
            t32.insert(t32.end(), b2.begin(), b2.end());
        }
        if (cudaMalloc(&h->d_tw64, t64.size() * sizeof(double2)) != cudaSuccess ||
            cudaMalloc(&h->d_tw32, t32.size() * sizeof(float2)) != cudaSuccess) {
            cudaStreamDestroy(h->stream); delete h;
            return fail(M3D_ERR_OOM, "twiddle allocation failed");
        }
        cudaMemcpy(h->d_tw64, t64.data(), t64.size() * sizeof(double2), cudaMemcpyHostToDevice);
        cudaMemcpy(h->d_tw32, t32.data(), t32.size() * sizeof(float2), cudaMemcpyHostToDevice);
    }
    table_layout(h);
    if (cudaMalloc(&h->d_phase, (size_t)nrve * h->g.V) != cudaSuccess ||
        cudaMalloc(&h->d_mats, (size_t)nrve * h->mstride * sizeof(double)) != cudaSuccess ||
        cudaMemset(h->d_phase, 0, (size_t)nrve * h->g.V) != cudaSuccess ||
        cudaMemset(h->d_mats, 0, (size_t)nrve * h->mstride * sizeof(double)) != cudaSuccess) {
        cudaStreamDestroy(h->stream); delete h;
        return fail(M3D_ERR_OOM, "phase map / table allocation failed");
    }
    *out = h;
    return M3D_OK;
}

int m3d_create(int kind, int Nx, int Ny, int Nz, int behav, int precision, int batch, m3d_solver** out) {
    if (batch < 1 || batch > 64) return fail(M3D_ERR_ARG, "batch must be in [1, 64]");
    return create_impl(kind, Nx, Ny, Nz, behav, precision, 1, batch, out);
}

long long m3d_footprint_bytes(int kind, int Nx, int Ny, int Nz, int behav, int precision, int nrve, int batch) {
    if (Nx < 2 || Ny < 2 || Nz < 2 || nrve < 1 || batch < nrve || precision < 0 || precision > 2) return -1;
    const long long C = (kind == M3D_KIND_MECH) ? 6 : 3;
    const long long V = (long long)Nx * Ny * Nz, NL = (long long)Nx * Ny, Hzp = even_up(Nz / 2 + 1);
    const long long B = batch;
    const long long xw = (precision == M3D_PREC_FP32) ? 4 : 8, sw = (precision == M3D_PREC_FP32) ? 8 : 16;
    long long b = nrve * V                                          // phase maps
                  + nrve * (4 * kMaxPhases * C * C + kMaxPhases * C) * 8  // table blocks
                  + (long long)(Nx + Ny + Nz) * 24                 // twiddles
                  + B * C * V * xw + B * C * NL * Hzp * sw          // state, half spectrum
                  + std::max(std::max(NL / 2 + 1, (long long)Ny * Hzp), 1024LL) * B * 16 * 8  // partials
                  + B * (2 * (long long)sizeof(Ctl) + 4) + 64;
    if (precision == M3D_PREC_FP32_REFINE) b += 2 * B * C * V * 4;  // correction + defect
    if (kind == M3D_KIND_MECH && behav != M3D_BEHAV_ELASTIC)  // FP64 eps, sig, eps_old (+ sig_old, ep | d)
        b += B * V * 8 * (18 + (behav == M3D_BEHAV_J2 ? 7 : 1));
    return b;
}

int m3d_create_multi(int kind, int Nx, int Ny, int Nz, int precision, int nrve, int nload, m3d_solver** out) {
    if (nrve < 1 || nrve > 4096) return fail(M3D_ERR_ARG, "nrve must be in [1, 4096]");
    if (nload < 1 || nload > 6) return fail(M3D_ERR_ARG, "nload must be in [1, 6]");
    if ((long long)nrve * nload > 8192) return fail(M3D_ERR_ARG, "nrve * nload must be <= 8192");
    return create_impl(kind, Nx, Ny, Nz, M3D_BEHAV_ELASTIC, precision, nrve, nrve * nload, out);
}

int m3d_destroy(m3d_solver* h) {
    if (!h) return M3D_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->xstream) {
        cudaStreamSynchronize(h->xstream);
        cudaStreamDestroy(h->xstream);
        cudaEventDestroy(h->ev_exp);
        cudaEventDestroy(h->ev_d2h);
    }
    for (int k = 0; k <= m3d_solver::kChunk; ++k)
        if (h->pev[k]) cudaEventDestroy(h->pev[k]);
    for (int k = 0; k < m3d_solver::kChunk; ++k)
        for (int p = 0; p < 6; ++p)
            if (h->ppev[k][p]) cudaEventDestroy(h->ppev[k][p]);
    h->free_all();
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
    return M3D_OK;
}

// Table block of RVE r: P, A, O (C x C per phase slot), Osum (C per slot), Q
// (C x C per slot), kMaxPhases slots each, at r * mstride in d_mats.
static void table_layout(m3d_solver* h) {
    const size_t C = h->C, S = kMaxPhases;
    h->off_P = 0;
    h->off_A = S * C * C;
    h->off_O = 2 * S * C * C;
    h->off_Os = 3 * S * C * C;
    h->off_Q = 3 * S * C * C + S * C;
    h->mstride = (long long)(4 * S * C * C + S * C);
}

// The caller's int32 phase ids of one RVE -> the uint8 map the sweeps read,
// with the statistics the material set-up needs: per id below nph its
// voxel count, the sum of the raw ids, and the first voxel whose id is
// outside [0, nph).  nph = 0 (thermal): any id, mapped to id != 0 and counted
// as 0 / 1.  st: [0, 16) counts, [16] id sum (two's complement), [17] first
// bad voxel (initialised to all ones).
__global__ void k_phase_in(const int32_t* __restrict__ ids, uint8_t* __restrict__ out, long long V, int nph,
                           unsigned long long* st) {
    __shared__ unsigned long long hist[kMaxPhases];
    if (threadIdx.x < kMaxPhases) hist[threadIdx.x] = 0;
    __syncthreads();
    long long sum = 0;
    unsigned long long bad = ~0ull;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        const int id = ids[v];
        sum += id;
        if (nph == 0) {
            const int p = id != 0 ? 1 : 0;
            out[v] = (uint8_t)p;
            atomicAdd(&hist[p], 1ull);
        } else if (id >= 0 && id < nph) {
            out[v] = (uint8_t)id;
            atomicAdd(&hist[id], 1ull);
        } else if ((unsigned long long)v < bad) {
            bad = (unsigned long long)v;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        const unsigned long long ob = __shfl_down_sync(0xffffffffu, bad, o);
        bad = ob < bad ? ob : bad;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&st[kMaxPhases], (unsigned long long)sum);
        if (bad != ~0ull) atomicMin(&st[kMaxPhases + 1], bad);
    }
    __syncthreads();
    if (threadIdx.x < kMaxPhases && hist[threadIdx.x]) atomicAdd(&st[threadIdx.x], hist[threadIdx.x]);
}

// RVE r's phase map from the caller's int32 ids, converted on the device: the
// ids are copied into the spectrum buffer, which holds nothing between solves
// (every solve writes it before reading it) and always has room for them
// (>= 12 bytes per voxel), then k_phase_in writes the map and the statistics.
int m3d_solver::load_phase(int r, const int32_t* phase, int nph, std::vector<long long>& counts, long long& idsum,
                           long long& bad) {
    const long long V = g.V;
    if (!d_pstat) M3D_CUDA(cudaMalloc(&d_pstat, (kMaxPhases + 2) * sizeof(unsigned long long)));
    M3D_CUDA(cudaMemsetAsync(d_pstat, 0, (kMaxPhases + 1) * sizeof(unsigned long long), stream));
    M3D_CUDA(cudaMemsetAsync(d_pstat + kMaxPhases + 1, 0xff, sizeof(unsigned long long), stream));
    int32_t* ids = (int32_t*)d_spec;
    M3D_CUDA(cudaMemcpyAsync(ids, phase, (size_t)V * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
    const int nblk = (int)std::min<long long>((V + 255) / 256, 148 * 8);
    k_phase_in<<<nblk, 256, 0, stream>>>(ids, d_phase + (size_t)r * V, V, nph, d_pstat);
    M3D_CUDA(cudaGetLastError());
    unsigned long long hs[kMaxPhases + 2];
    M3D_CUDA(cudaMemcpyAsync(hs, d_pstat, sizeof(hs), cudaMemcpyDeviceToHost, stream));
    M3D_CUDA(cudaStreamSynchronize(stream));
    const int np = nph == 0 ? 2 : nph;
    counts.assign(np, 0);
    for (int i = 0; i < np; ++i) counts[i] = (long long)hs[i];
    idsum = (long long)hs[kMaxPhases];
    bad = hs[kMaxPhases + 1] == ~0ull ? -1 : (long long)hs[kMaxPhases + 1];
    return M3D_OK;
}

static int upload_tables(m3d_solver* h, int r) {
    std::vector<double> blk((size_t)h->mstride, 0.0);
    std::copy(h->hP.begin(), h->hP.end(), blk.begin() + h->off_P);
    std::copy(h->hA.begin(), h->hA.end(), blk.begin() + h->off_A);
    std::copy(h->hO.begin(), h->hO.end(), blk.begin() + h->off_O);
    std::copy(h->hOsum.begin(), h->hOsum.end(), blk.begin() + h->off_Os);
    std::copy(h->hQ.begin(), h->hQ.end(), blk.begin() + h->off_Q);
    M3D_CUDA(cudaMemcpy(h->d_mats + (size_t)r * h->mstride, blk.data(), blk.size() * sizeof(double),
                        cudaMemcpyHostToDevice));
    return M3D_OK;
}

static void push_mat(std::vector<double>& dst, const Mat& m) { dst.insert(dst.end(), m.begin(), m.end()); }

int m3d_set_material_mech(m3d_solver* h, const double* mat, int nph, const int32_t* phase, int scheme) {
    return m3d_set_material_mech_rve(h, 0, mat, nph, phase, scheme);
}

int m3d_set_material_mech_rve(m3d_solver* h, int r, const double* mat, int nph, const int32_t* phase, int scheme) {
    if (!h || !mat || !phase) return fail(M3D_ERR_ARG, "NULL argument");
    if (r < 0 || r >= h->nrve) return fail(M3D_ERR_ARG, "RVE index out of range");
    if (h->kind != M3D_KIND_MECH) return fail(M3D_ERR_ARG, "not a mechanical solver");
    if (nph < 1 || nph > kMaxPhases) return fail(M3D_ERR_ARG, "nph must be in [1, 16]");
    if (scheme < 0 || scheme > 2) return fail(M3D_ERR_ARG, "invalid scheme");
    const long long V = h->g.V;
    long long idsum = 0, bad = -1;
    int prc = h->load_phase(r, phase, nph, h->counts, idsum, bad);
    if (prc) return prc;
    if (bad >= 0) {  // RVE r's device map is now incomplete: the RVE counts as not set
        h->rv[r].set = false;
        h->material_set = false;
        return fail(M3D_ERR_ARG, "phase id out of range at voxel " + std::to_string(bad));
    }
    h->nph = nph;
    h->mat.assign(mat, mat + nph * 7);
    // material(), src/3d/FFT_analysis3D.cpp:441-546
    std::vector<double> mu(nph), la(nph), K(nph);
    h->vol.assign(nph, 0.0);
    for (int i = 0; i < nph; ++i) {
        const double El = mat[i * 7 + 0], v = mat[i * 7 + 1];
        if (!(El > 0) || !(v > -1.0 && v < 0.5)) return fail(M3D_ERR_ARG, "phase " + std::to_string(i) + ": need E > 0 and -1 < nu < 0.5");
        mu[i] = El / (1 + v) / 2.;
        la[i] = v * El / (1 + v) / (1 - 2 * v);
        K[i] = la[i] + (2. / 3.) * mu[i];
        h->Cp[i] = iso_stiffness(la[i], mu[i]);
        h->Sp[i] = mat_inv(h->Cp[i], 6);
        h->vol[i] = (double)h->counts[i] / (double)V;
    }
    int imu = 0;
    for (int i = 1; i < nph; ++i) if (mu[i] > mu[imu]) imu = i;  // first strict maximum (:5-23)
    const double mu_max = *std::max_element(mu.begin(), mu.end()), mu_min = *std::min_element(mu.begin(), mu.end());
    const double la_max = *std::max_element(la.begin(), la.end()), la_min = *std::min_element(la.begin(), la.end());
    const double K_max = *std::max_element(K.begin(), K.end()), K_min = *std::min_element(K.begin(), K.end());
    const double vol_max = *std::max_element(h->vol.begin(), h->vol.end());
    if (h->behav == M3D_BEHAV_ELASTIC) {
        const double K0 = std::sqrt(K_min * K_max);
        h->mu0 = std::sqrt(mu_min * mu_max);
        h->la0 = K0 - h->mu0 * 2. / 3.;
        h->scheme = (h->vol[imu] == vol_max) ? 1 : 2;  // (:503-512)
    } else {
        h->scheme = 1;  // (:515-522)
        h->mu0 = (mu_min + mu_max) / 2;
        h->la0 = (la_min + la_max) / 2;
    }
    if (scheme != M3D_SCHEME_AUTO) {
        if (h->behav != M3D_BEHAV_ELASTIC && scheme == M3D_SCHEME_DUAL)
            return fail(M3D_ERR_ARG, "the ep/ed path is strain-based only");
        h->scheme = scheme;
    }
    h->C0 = iso_stiffness(h->la0, h->mu0);
    h->S0 = mat_inv(h->C0, 6);
    h->hP.clear(); h->hA.clear(); h->hO.clear(); h->hOsum.clear(); h->hQ.clear();
    for (int i = 0; i < nph; ++i) {
        if (h->scheme == 1) {
            push_mat(h->hP, mat_add(h->Cp[i], h->C0, -1.0));
            push_mat(h->hA, mat_mul(mat_scale(mat_inv(mat_add(h->Cp[i], h->C0), 6), 2.0), h->C0, 6));
            push_mat(h->hO, h->Cp[i]);
            push_mat(h->hQ, h->Cp[i]);
        } else {
            push_mat(h->hP, mat_add(h->Sp[i], h->S0, -1.0));
            push_mat(h->hA, mat_mul(mat_scale(mat_inv(mat_add(h->Sp[i], h->S0), 6), 2.0), h->S0, 6));
            push_mat(h->hO, h->Sp[i]);
            push_mat(h->hQ, diag(6, 1.0));
        }
        const Mat& O = (h->scheme == 1) ? h->Cp[i] : h->Sp[i];
        for (int c = 0; c < 6; ++c) {
            double s = 0;
            for (int r = 0; r < 6; ++r) s += O[r * 6 + c];
            h->hOsum.push_back(s);
        }
    }
    const int p1 = nph > 1 ? 1 : 0;  // the reference reads phases 0 and 1 (:399, :408)
    h->den_ref = (h->scheme == 1) ? 0.5 * h->Cp[0][0] + 0.5 * h->Cp[p1][0] : 0.5 * h->Sp[0][0] + 0.5 * h->Sp[p1][0];
    int rc = upload_tables(h, r);
    if (rc) return rc;
    M3D_CUDA(cudaStreamSynchronize(h->stream));
    h->snapshot_rve(r);
    h->material_set = h->all_rves_set();
    h->st.scheme = h->scheme;
    h->st.la0 = h->la0;
    h->st.mu0 = h->mu0;
    for (int i = 0; i < 16; ++i) h->st.vol_fraction[i] = i < nph ? h->vol[i] : 0.0;
    if (h->behav != M3D_BEHAV_ELASTIC) {
        rc = h->in.setup(h);
        if (rc) return rc;
    }
    return M3D_OK;
}

int m3d_set_material_thermal(m3d_solver* h, double km, double ki, const int32_t* phase, int scheme) {
    return m3d_set_material_thermal_rve(h, 0, km, ki, phase, scheme);
}

int m3d_set_material_thermal_rve(m3d_solver* h, int r, double km, double ki, const int32_t* phase, int scheme) {
    if (!h || !phase) return fail(M3D_ERR_ARG, "NULL argument");
    if (r < 0 || r >= h->nrve) return fail(M3D_ERR_ARG, "RVE index out of range");
    if (h->kind != M3D_KIND_THERMAL) return fail(M3D_ERR_ARG, "not a thermal solver");
    if (!(km > 0) || !(ki > 0)) return fail(M3D_ERR_ARG, "conductivities must be positive");
    if (scheme < 0 || scheme > 2) return fail(M3D_ERR_ARG, "invalid scheme");
    const long long V = h->g.V;
    // multipKx()/strainUpdate() test `if (RVE(i))` (src/3dTherm/FFT_thermal3D.cpp:186,249): map id != 0 to 1
    long long idsum = 0, bad = -1;
    int prc = h->load_phase(r, phase, 0, h->counts, idsum, bad);
    if (prc) return prc;
    h->nph = 2;
    h->km = km;
    h->ki = ki;
    // vol_1 = RVE.sum()/xyz is an integer division in the reference (:399)
    const long long vol_1 = idsum / V;
    h->scheme = ((vol_1 >= 1 && km > ki) || (vol_1 < 1 && km < ki)) ? 1 : 2;  // (:401-410)
    if (scheme != M3D_SCHEME_AUTO) h->scheme = scheme;
    h->k0 = std::sqrt(ki * km);  // (:415)
    const double kk[2] = {ki, km};
    h->hP.clear(); h->hA.clear(); h->hO.clear(); h->hOsum.clear(); h->hQ.clear();
    h->vol.assign(2, 0.0);
    for (int p = 0; p < 2; ++p) {
        const double k = kk[p], k0 = h->k0;
        h->vol[p] = (double)h->counts[p] / (double)V;
        if (h->scheme == 1) {
            push_mat(h->hP, diag(3, k - k0));
            push_mat(h->hA, diag(3, 2 * k0 / (k + k0)));
            push_mat(h->hO, diag(3, k));
            push_mat(h->hQ, diag(3, k));
            for (int c = 0; c < 3; ++c) h->hOsum.push_back(k);
        } else {
            const double r = 1.0 / k, r0 = 1.0 / k0;
            push_mat(h->hP, diag(3, r - r0));
            push_mat(h->hA, diag(3, 2 * r0 / (r + r0)));
            push_mat(h->hO, diag(3, r));
            push_mat(h->hQ, diag(3, 1.0));
            for (int c = 0; c < 3; ++c) h->hOsum.push_back(r);
        }
    }
    h->den_ref = (h->scheme == 1) ? 0.5 * ki + 0.5 * km : 0.5 / ki + 0.5 / km;  // (:346, :356)
    int rc = upload_tables(h, r);
    if (rc) return rc;
    M3D_CUDA(cudaStreamSynchronize(h->stream));
    h->snapshot_rve(r);
    h->material_set = h->all_rves_set();
    h->st.scheme = h->scheme;
    h->st.k0 = h->k0;
    h->st.vol_fraction[0] = h->vol[0];
    h->st.vol_fraction[1] = h->vol[1];
    return M3D_OK;
}

int m3d_set_load(m3d_solver* h, int b, const double* E, const double* X0) {
    if (!h || !E) return fail(M3D_ERR_ARG, "NULL argument");
    if (b < -1 || b >= h->B) return fail(M3D_ERR_ARG, "batch index out of range");
    for (int i = 0; i < h->C; ++i)
        if (!std::isfinite(E[i])) return fail(M3D_ERR_ARG, "non-finite load");
    const int lo = b < 0 ? 0 : b, hi = b < 0 ? h->B : b + 1;
    for (int k = lo; k < hi; ++k) {
        for (int i = 0; i < h->C; ++i) h->E[k * h->C + i] = E[i];
        for (int i = 0; i < 6; ++i) h->X0[k * 6 + i] = X0 ? X0[i] : 0.0;
    }
    h->load_set = true;
    return M3D_OK;
}

int m3d_run(m3d_solver* h, double tol_field, double tol_eq, int nInc, int criterion, int max_iter) {
    if (!h) return fail(M3D_ERR_ARG, "NULL handle");
    if (!h->material_set) return fail(M3D_ERR_STATE, "material not set");
    if (!h->load_set) return fail(M3D_ERR_STATE, "load not set");
    if (criterion != M3D_CRIT_REFERENCE && criterion != M3D_CRIT_RESIDUAL) return fail(M3D_ERR_ARG, "invalid criterion");
    if (!(tol_field > 0) || !(tol_eq >= 0)) return fail(M3D_ERR_ARG, "tolerances must be positive");
    if (h->behav != M3D_BEHAV_ELASTIC && nInc < 1) return fail(M3D_ERR_ARG, "nInc must be >= 1");
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = h->dispatch_run(tol_field, tol_eq, nInc, criterion, max_iter);
    cudaStreamSynchronize(h->stream);
    h->st.solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    h->st.status = rc;
    h->run_done = (rc == M3D_OK || rc == M3D_NOT_CONVERGED);
    return rc;
}

}  // extern "C"

static int assemble_rve(m3d_solver* h, int r, double* Ceff, double* Seff, double* ep_means, double* sig_means);

// means of the strain-like and stress-like fields of entry b
template <typename TX, int CC>
__global__ void k_means(const TX* __restrict__ x, const uint8_t* __restrict__ phase, const double* __restrict__ mats,
                        int b, long long V, double* __restrict__ part) {
    double acc[2 * CC] = {};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        double xv[CC];
#pragma unroll
        for (int c = 0; c < CC; ++c) xv[c] = (double)x[((long long)b * CC + c) * V + v];
        const double* M = mats + phase[v] * CC * CC;
#pragma unroll
        for (int i = 0; i < CC; ++i) {
            acc[i] += xv[i];
            double s = 0;
#pragma unroll
            for (int j = 0; j < CC; ++j) s += M[i * CC + j] * xv[j];
            acc[CC + i] += s;
        }
    }
    __shared__ double red[32 * 2 * CC];
    block_reduce_store<2 * CC>(acc, red, part, 0, gridDim.x, blockIdx.x);
}

extern "C" {

int m3d_get_means(m3d_solver* h, int b, double* strain_mean, double* stress_mean) {
    if (!h) return fail(M3D_ERR_ARG, "NULL handle");
    if (!h->run_done) return fail(M3D_ERR_STATE, "no finished run");
    if (b < 0 || b >= h->B) return fail(M3D_ERR_ARG, "batch index out of range");
    const int C = h->C;
    if (h->kind == M3D_KIND_MECH && h->behav != M3D_BEHAV_ELASTIC)
        return h->in.means(h, b, strain_mean, stress_mean);
    const int nblk = 296;
    double* part = h->d_part;
    if (h->part_cap < (size_t)nblk * 2 * C) return fail(M3D_ERR_STATE, "partials buffer too small");
    const int r = h->rve_of(b);
    const double* O = h->d_mats + (size_t)r * h->mstride + h->off_O;
    const uint8_t* ph = h->d_phase + (size_t)r * h->g.V;
    if (C == 6) {
        if (h->prec == M3D_PREC_FP32) k_means<float, 6><<<nblk, 256, 0, h->stream>>>((const float*)h->d_x, ph, O, b, h->g.V, part);
        else k_means<double, 6><<<nblk, 256, 0, h->stream>>>((const double*)h->d_x, ph, O, b, h->g.V, part);
    } else {
        if (h->prec == M3D_PREC_FP32) k_means<float, 3><<<nblk, 256, 0, h->stream>>>((const float*)h->d_x, ph, O, b, h->g.V, part);
        else k_means<double, 3><<<nblk, 256, 0, h->stream>>>((const double*)h->d_x, ph, O, b, h->g.V, part);
    }
    h->st.kernel_launches += 1;
    M3D_CUDA(cudaGetLastError());
    std::vector<double> hp((size_t)nblk * 2 * C);
    M3D_CUDA(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    M3D_CUDA(cudaStreamSynchronize(h->stream));
    double s[12] = {};
    for (int k = 0; k < 2 * C; ++k)
        for (int i = 0; i < nblk; ++i) s[k] += hp[(size_t)k * nblk + i];
    const double V = (double)h->g.V;
    // state = strain-like in the primal scheme, stress-like in the dual scheme
    const bool primal = h->rv[r].scheme == 1;
    double* prim = primal ? strain_mean : stress_mean;
    double* dual = primal ? stress_mean : strain_mean;
    for (int c = 0; c < C; ++c) {
        if (prim) prim[c] = s[c] / V;
        if (dual) dual[c] = s[C + c] / V;
    }
    return M3D_OK;
}

int m3d_homogenize(m3d_solver* h, double tol_field, double tol_eq, int criterion, int max_iter, double* Ceff,
                   double* Seff, double* ep_means, double* sig_means) {
    if (!h) return fail(M3D_ERR_ARG, "NULL handle");
    if (!h->material_set) return fail(M3D_ERR_STATE, "material not set");
    if (h->kind == M3D_KIND_MECH && h->behav != M3D_BEHAV_ELASTIC)
        return fail(M3D_ERR_ARG, "homogenization runs the elastic solver; create the solver with behaviour ELASTIC");
    const int C = h->C, R = h->nrve;
    if (h->B != C * R) {
        int rc = h->alloc(C * R);
        if (rc) return rc;
    }
    // load cases (src/3d/FFT_analysis3D.cpp:866-877; src/3dTherm/FFT_thermal3D.cpp:501-507, 544-549);
    // entry r * C + w is load case w of RVE r
    for (int r = 0; r < R; ++r)
        for (int w = 0; w < C; ++w) {
            double E[6] = {0, 0, 0, 0, 0, 0};
            if (h->kind == M3D_KIND_MECH) E[w] = (h->rv[r].scheme == 1) ? 0.0005 : 1.e6;
            else E[w] = 1.0;
            int rc = m3d_set_load(h, r * C + w, E, h->kind == M3D_KIND_MECH ? E : nullptr);
            if (rc) return rc;
        }
    const auto t0 = std::chrono::steady_clock::now();
    int rc = h->dispatch_run(tol_field, tol_eq, 1, criterion, max_iter);
    if (rc != M3D_OK && rc != M3D_NOT_CONVERGED) return rc;
    const int status = rc;
    h->run_done = true;
    for (int r = 0; r < R; ++r) {
        rc = assemble_rve(h, r, Ceff ? Ceff + (size_t)r * C * C : nullptr, Seff ? Seff + (size_t)r * C * C : nullptr,
                          ep_means ? ep_means + (size_t)r * C * C : nullptr,
                          sig_means ? sig_means + (size_t)r * C * C : nullptr);
        if (rc) return rc;
    }
    h->st.solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    h->st.status = status;
    return status;
}

}  // extern "C"

// Effective tensor of RVE r from the means of its C load-case entries.
static int assemble_rve(m3d_solver* h, int r, double* Ceff, double* Seff, double* ep_means, double* sig_means) {
    const int C = h->C;
    int rc;
    // strain-like means g[w][c], stress-like q[w][c] per load case w
    std::vector<double> gm(C * C), qm(C * C);
    for (int w = 0; w < C; ++w) {
        rc = m3d_get_means(h, r * C + w, &gm[w * C], &qm[w * C]);
        if (rc) return rc;
    }
    // Assembly exactly as the reference: one matrix stores the means with one
    // ROW per load case, the other with one COLUMN per load case, and the
    // result is X = first^-1 * second.
    //  mech strain-based  (src/3d/FFT_analysis3D.cpp:880-895): epHomo(t,w) = <eps_t>_w (columns),
    //      sigHomo(w,t) = <sig_t>_w (rows), CHomo = epHomo^-1 sigHomo
    //  mech stress-based  (:897-901): SHomo = sigHomo^-1 epHomo
    //  thermal gradient   (src/3dTherm/FFT_thermal3D.cpp:525-536): tempGradHomo(w,j) (rows),
    //      heatFluxHomo(j,w) (columns), KHomo = tempGradHomo^-1 heatFluxHomo
    //  thermal flux       (:567-578): heatFluxHomo(w,j) (rows), tempGradHomo(j,w) (columns),
    //      RHomo = heatFluxHomo^-1 tempGradHomo
    const bool primal = (h->rv[r].scheme == 1);
    Mat rows_g(C * C), cols_g(C * C), rows_q(C * C), cols_q(C * C);
    for (int w = 0; w < C; ++w)
        for (int t = 0; t < C; ++t) {
            rows_g[w * C + t] = gm[w * C + t];
            cols_g[t * C + w] = gm[w * C + t];
            rows_q[w * C + t] = qm[w * C + t];
            cols_q[t * C + w] = qm[w * C + t];
        }
    Mat first, second, strain_store, stress_store;
    if (h->kind == M3D_KIND_MECH) {
        strain_store = cols_g;  // epHomo
        stress_store = rows_q;  // sigHomo
        if (primal) { first = cols_g; second = rows_q; } else { first = rows_q; second = cols_g; }
    } else {
        if (primal) { first = rows_g; second = cols_q; strain_store = rows_g; stress_store = cols_q; }
        else { first = rows_q; second = cols_g; strain_store = cols_g; stress_store = rows_q; }
    }
    const Mat X = mat_mul(mat_inv(first, C), second, C);
    const Mat Xi = mat_inv(X, C);
    // primal: X is the stiffness (conductivity); dual: X is the compliance (resistivity)
    const Mat& Cm = primal ? X : Xi;
    const Mat& Sm = primal ? Xi : X;
    if (Ceff) std::memcpy(Ceff, Cm.data(), C * C * sizeof(double));
    if (Seff) std::memcpy(Seff, Sm.data(), C * C * sizeof(double));
    if (ep_means) std::memcpy(ep_means, strain_store.data(), C * C * sizeof(double));
    if (sig_means) std::memcpy(sig_means, stress_store.data(), C * C * sizeof(double));
    return M3D_OK;
}

static int get_field_impl(m3d_solver* h, int which, int b, double* out, bool async);

extern "C" {

int m3d_get_field(m3d_solver* h, int which, int b, double* out) { return get_field_impl(h, which, b, out, false); }

int m3d_get_field_async(m3d_solver* h, int which, int b, double* out) {
    return get_field_impl(h, which, b, out, true);
}

int m3d_wait_field(m3d_solver* h) {
    if (!h) return fail(M3D_ERR_ARG, "NULL handle");
    if (h->d2h_pending) {
        M3D_CUDA(cudaEventSynchronize(h->ev_d2h));
        h->d2h_pending = false;
    }
    return M3D_OK;
}

}  // extern "C"

static int get_field_impl(m3d_solver* h, int which, int b, double* out, bool async) {
    if (!h || !out) return fail(M3D_ERR_ARG, "NULL argument");
    if (!h->run_done) return fail(M3D_ERR_STATE, "no finished run");
    if (b < 0 || b >= h->B) return fail(M3D_ERR_ARG, "batch index out of range");
    if (h->kind == M3D_KIND_MECH && h->behav != M3D_BEHAV_ELASTIC) {  // synchronous, after any pending copy
        if (h->d2h_pending) {
            M3D_CUDA(cudaEventSynchronize(h->ev_d2h));
            h->d2h_pending = false;
        }
        return h->in.get_field(h, which, b, out);
    }
    if (which != M3D_FIELD_STRAIN && which != M3D_FIELD_STRESS)
        return fail(M3D_ERR_ARG, "field not available for this behaviour");
    const bool state = (which == M3D_FIELD_STRAIN) == (h->rv[h->rve_of(b)].scheme == 1);
    const double* M = state ? nullptr : h->d_mats + h->off_O;
    if (h->C == 6)
        return h->prec == M3D_PREC_FP32 ? export_field<float, 6>(h, h->d_x, M, b, out, async)
                                        : export_field<double, 6>(h, h->d_x, M, b, out, async);
    return h->prec == M3D_PREC_FP32 ? export_field<float, 3>(h, h->d_x, M, b, out, async)
                                    : export_field<double, 3>(h, h->d_x, M, b, out, async);
}

// ---- autotuner ----------------------------------------------------------------
// Launch schedules that give identical arithmetic per line but run at
// different speeds: the compile-time warp-split kernels or the generic
// shared-memory Stockham kernels, the TMA-staged or the register-staged y pass,
// and the generic kernels' tile sizes (G z lines per CTA, TZ columns per y / x
// tile).  Each candidate is timed with CUDA events over a few full sweeps of
// the handle's own batch (stop rule disabled); the fastest is kept, and
// remembered per shape and precision for later handles (m3d_autotune with
// sweeps = 0).
namespace {
struct TuneKey {
    int kind, Nx, Ny, Nz, prec;
    bool operator<(const TuneKey& o) const {
        return std::tie(kind, Nx, Ny, Nz, prec) < std::tie(o.kind, o.Nx, o.Ny, o.Nz, o.prec);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, m3d_tune> g_tune;
}  // namespace

template <typename T, int CC>
int m3d_solver::tune_time(int sweeps, float* ms) {
    typedef typename Cx<T>::t C2;
    drop_graphs();
    int rc = init_ctl(d_ctl, 0.0, 0.0, 1 << 30, false);  // tolerance 0: no entry stops
    if (rc) return rc;
    // time a few entries only (the others skip every pass), so tuning a large batch stays cheap
    for (int b = 6; b < B; ++b) h_ctl[b].done = 1;
    M3D_CUDA(cudaMemcpyAsync(d_ctl, h_ctl, B * sizeof(Ctl), cudaMemcpyHostToDevice, stream));
    T* x = (prec == M3D_PREC_FP32_REFINE) ? (T*)(void*)d_delta : (T*)d_x;
    const float* r = (prec == M3D_PREC_FP32_REFINE) ? d_r32 : nullptr;
    k_fill_load<T><<<dim3(256, B * CC), 256, 0, stream>>>(x, d_ctl, CC, g.V);
    C2* sp = (C2*)d_spec;
    cudaEvent_t e0, e1;
    M3D_CUDA(cudaEventCreate(&e0));
    M3D_CUDA(cudaEventCreate(&e1));
    const bool slab = slab_ok<T>();
    auto sweep = [&]() {
        return slab ? launch_em_slab<T, CC>(d_ctl, x, r, sp, 0, POL_RESIDUAL, nullptr)
                    : launch_em<T, CC>(d_ctl, x, r, sp, 0, POL_RESIDUAL, nullptr);
    };
    if (slab) rc = pass_slab<T, CC, false>(d_ctl, x, nullptr, sp, FinNone{});
    if (!rc) rc = sweep();  // warm-up (attributes, tensor maps)
    cudaEventRecord(e0, stream);
    for (int k = 0; k < sweeps && !rc; ++k) rc = sweep();
    cudaEventRecord(e1, stream);
    cudaError_t e = cudaEventSynchronize(e1);
    if (!rc && e == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!rc && e != cudaSuccess) return fail(M3D_ERR_CUDA, cudaGetErrorString(e));
    return rc;
}

int m3d_solver::autotune(int sweeps, m3d_tune* out) {
    const bool fp64 = (prec == M3D_PREC_FP64);
    const size_t csz = fp64 ? 16 : 8;
    std::vector<m3d_tune> cand;
    const bool fast_ok = fast_size(Nx) && fast_size(Ny) && fast_size(Nz);
    const int G0 = fp64 ? G64 : G32, Y0 = fp64 ? TZy64 : TZy32, X0 = fp64 ? TZx64 : TZx32;  // heuristic tiles
    const size_t lim = 200 * 1024;
    if (fast_ok) {
        // compile-time kernels with either y pass, the two-pass sweep where the
        // operators allow it, and the generic kernels with their default tiles
        cand.push_back(m3d_tune{1, 0, G0, Y0, X0, 0, 0, 0, 0});
        cand.push_back(m3d_tune{1, 1, G0, Y0, X0, 0, 0, 0, 0});
        const bool f1 = use_fast, s1 = use_slab;
        use_fast = use_slab = true;
        const bool slab_possible = fp64 ? slab_ok<double>() : slab_ok<float>();
        use_fast = f1;
        use_slab = s1;
        if (slab_possible) cand.push_back(m3d_tune{1, 0, G0, Y0, X0, 0, 0, 1, 0});
        cand.push_back(m3d_tune{0, 0, G0, Y0, X0, 0, 0, 0, 0});
    } else {
        // generic kernels: every tile size whose shared memory fits comfortably,
        // and (with the heuristic tiles) every distinct order of the radix stages
        for (int Gv : {2, 4, 8, 16}) {
            if ((size_t)Nz * csz * (1 + (size_t)Gv * C) + 32 * 32 * 8 + op_smem<double, 6>() > lim) continue;
            for (int tz : {2, 4, 8, 16}) {
                if (2 * (size_t)C * Nx * tz * csz + (size_t)Nx * csz > lim || 2 * (size_t)Ny * tz * csz > lim) continue;
                cand.push_back(m3d_tune{0, 0, Gv, tz, tz, 0, 0, 0, 0});
            }
        }
        auto same = [](const LinePlan& a, const LinePlan& b) {
            if (a.nstages != b.nstages) return false;
            for (int i = 0; i < a.nstages; ++i)
                if (a.radix[i] != b.radix[i]) return false;
            return true;
        };
        for (int o = 1; o < kPlanOrders; ++o) {
            LinePlan qx{}, qy{}, qz{}, rx{}, ry{}, rz{};
            if (!make_plan(Nx, qx, false, o) || !make_plan(Ny, qy, false, o) || !make_plan(Nz, qz, false, o)) continue;
            bool dup = false;
            for (int o2 = 0; o2 < o && !dup; ++o2)
                if (make_plan(Nx, rx, false, o2) && make_plan(Ny, ry, false, o2) && make_plan(Nz, rz, false, o2))
                    dup = same(qx, rx) && same(qy, ry) && same(qz, rz);
            if (!dup) cand.push_back(m3d_tune{0, 0, G0, Y0, X0, 0, 0, 0, o});
        }
    }
    const bool f0 = use_fast, t0 = use_tma_y, sl0 = use_slab;
    const int g32 = G32, g64 = G64, y32 = TZy32, y64 = TZy64, x32 = TZx32, x64 = TZx64;
    const LinePlan px0 = px, py0 = py, pz0 = pz;
    int best = -1;
    for (size_t i = 0; i < cand.size(); ++i) {
        m3d_tune& c = cand[i];
        use_fast = c.fast != 0;
        use_tma_y = c.tma_y != 0;
        use_slab = c.slab != 0;
        make_plan(Nx, px, false, c.schedule);
        make_plan(Ny, py, false, c.schedule);
        make_plan(Nz, pz, false, c.schedule);
        (fp64 ? G64 : G32) = c.G;
        (fp64 ? TZy64 : TZy32) = c.tzy;
        (fp64 ? TZx64 : TZx32) = c.tzx;
        float ms = 0;
        int rc = fp64 ? (C == 6 ? tune_time<double, 6>(sweeps, &ms) : tune_time<double, 3>(sweeps, &ms))
                      : (C == 6 ? tune_time<float, 6>(sweeps, &ms) : tune_time<float, 3>(sweeps, &ms));
        if (rc) {
            (void)cudaGetLastError();
            continue;
        }
        c.sweep_us = 1000.0 * ms / sweeps;
        if (best < 0 || c.sweep_us < cand[best].sweep_us) best = (int)i;
    }
    use_fast = f0; use_tma_y = t0; use_slab = sl0;
    px = px0; py = py0; pz = pz0;
    G32 = g32; G64 = g64; TZy32 = y32; TZy64 = y64; TZx32 = x32; TZx64 = x64;
    drop_graphs();
    if (best < 0) return fail(M3D_ERR_CUDA, "autotune: no candidate ran");
    m3d_tune t = cand[best];
    t.candidates = (int)cand.size();
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[TuneKey{kind, Nx, Ny, Nz, prec}] = t;
    }
    if (out) *out = t;
    return M3D_OK;
}

extern "C" {

int m3d_autotune(m3d_solver* h, int sweeps, m3d_tune* out) {
    if (!h) return fail(M3D_ERR_ARG, "NULL handle");
    if (h->kind == M3D_KIND_MECH && h->behav != M3D_BEHAV_ELASTIC)
        return fail(M3D_ERR_UNSUPPORTED, "the autotuner times the linear sweeps (elastic or thermal solvers)");
    if (sweeps < 0 || sweeps > 1000) return fail(M3D_ERR_ARG, "sweeps must be in [0, 1000]");
    m3d_tune t{};
    if (sweeps > 0) {
        if (!h->material_set) return fail(M3D_ERR_STATE, "material not set");
        const int rc = h->autotune(sweeps, &t);
        if (rc) return rc;
    } else {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(TuneKey{h->kind, h->Nx, h->Ny, h->Nz, h->prec});
        if (it == g_tune.end()) return fail(M3D_ERR_STATE, "no tuned schedule for this shape yet");
        t = it->second;
    }
    // apply
    const bool fp64 = (h->prec == M3D_PREC_FP64);
    h->use_fast = t.fast != 0;
    h->use_tma_y = t.tma_y != 0;
    h->use_slab = t.slab != 0;
    make_plan(h->Nx, h->px, false, t.schedule);
    make_plan(h->Ny, h->py, false, t.schedule);
    make_plan(h->Nz, h->pz, false, t.schedule);
    (fp64 ? h->G64 : h->G32) = t.G;
    (fp64 ? h->TZy64 : h->TZy32) = t.tzy;
    (fp64 ? h->TZx64 : h->TZx32) = t.tzx;
    if (h->prec == M3D_PREC_FP32_REFINE) {  // its FP64 defect sweeps keep the fast/TMA choice, generic sizes of FP32
        h->G64 = std::max(2, t.G / 2) & ~1;
    }
    h->drop_graphs();
    if (out) *out = t;
    return M3D_OK;
}

int m3d_set_profiling(m3d_solver* h, int enable) {
    if (!h) return fail(M3D_ERR_ARG, "NULL handle");
    if (enable && !h->pev[0]) {
        for (int k = 0; k <= m3d_solver::kChunk; ++k) M3D_CUDA(cudaEventCreate(&h->pev[k]));
        for (int k = 0; k < m3d_solver::kChunk; ++k)
            for (int p = 0; p < 6; ++p) M3D_CUDA(cudaEventCreate(&h->ppev[k][p]));
    }
    h->prof = enable != 0;
    std::memset(&h->pr, 0, sizeof(h->pr));
    return M3D_OK;
}

int m3d_get_profile(const m3d_solver* h, m3d_profile* out) {
    if (!h || !out) return fail(M3D_ERR_ARG, "NULL argument");
    *out = h->pr;
    return M3D_OK;
}

void* m3d_get_stream(const m3d_solver* h) { return h ? (void*)h->stream : nullptr; }

int m3d_set_stream(m3d_solver* h, void* s) {
    if (!h) return fail(M3D_ERR_ARG, "NULL handle");
    M3D_CUDA(cudaStreamSynchronize(h->stream));
    h->stream = s ? (cudaStream_t)s : h->own_stream;
    return M3D_OK;
}

int m3d_get_stats(const m3d_solver* h, m3d_stats* out) {
    if (!h || !out) return fail(M3D_ERR_ARG, "NULL argument");
    *out = h->st;
    return M3D_OK;
}

int m3d_get_entry_stats(const m3d_solver* h, int b, int* iters, long long* sweeps, double* residual, int* status) {
    if (!h) return fail(M3D_ERR_ARG, "NULL handle");
    if (b < 0 || b >= h->B || !h->h_ctl) return fail(M3D_ERR_ARG, "batch entry out of range");
    const Ctl& c = h->h_ctl[b];
    if (iters) *iters = c.iters;
    // the refinement's control block counts its FP64 sweeps, its inner FP32 sweeps in aux[1]
    if (sweeps) *sweeps = (long long)c.iters + (h->prec == M3D_PREC_FP32_REFINE ? (long long)c.aux[1] : 0);
    if (residual) *residual = c.residual;
    if (status) *status = c.status == 2 ? M3D_ERR_NAN : (c.status == 1 ? M3D_NOT_CONVERGED : M3D_OK);
    return M3D_OK;
}

int m3d_get_increments(const m3d_solver* h, double* out, int max_rows) {
    if (!h || !out) return fail(M3D_ERR_ARG, "NULL argument");
    const int rows = std::min<int>(max_rows, (int)(h->prop.size() / 9));
    std::memcpy(out, h->prop.data(), (size_t)rows * 9 * sizeof(double));
    return rows;
}

}  // extern "C"
