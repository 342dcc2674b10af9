// inelastic.cuh -- J2 elasto-plasticity and scalar damage (mater_behav "ep" /
// "ed"), basic scheme with mixed load control, on the same FFT passes.
//
// Reference: runAnalysis ep/ed branch, src/3d/FFT_analysis3D.cpp:796-853.
// Per iteration the reference does FFT(sig), FFT(eps), updateE, t3 = eps^ -
// Gamma0 sig^ (k=0 <- E V), IFFT -> eps, constitutive, and one more FFT(sig)
// for convergenceCheck.  Here, by linearity of the c2r transform,
//     eps_new = eps + IFFT(-Gamma0 sig^),  mode k=0 set to (E - <eps>) V,
// so FFT(eps) is not needed, and the convergenceCheck spectrum of sig_k is the
// forward spectrum the NEXT sweep computes anyway: its reductions are taken
// in the x turnaround before Gamma0 is applied, and a finalize step between
// the turnaround and the inverse passes stops the entry, leaving
// (eps_k, sig_k) in place.  One sweep = one forward + one inverse transform.
#pragma once
#include "physics.cuh"

struct m3d_solver;

namespace m3d {

enum { BEHAV_J2 = 1, BEHAV_DAMAGE = 2 };

// per-phase constants for the constitutive update (double)
struct PhaseMech {
    double C[36];
    double mu, Sy, H, n, P, Y0;
};

// von Mises stress and deviator (sigma_eff_calculator, :597-606)
__device__ __forceinline__ double vonmises(const double (&s)[6], double (&sd)[6]) {
    const double sm = (s[0] + s[1] + s[2]) / 3.;
#pragma unroll
    for (int c = 0; c < 6; ++c) sd[c] = s[c];
    sd[0] -= sm; sd[1] -= sm; sd[2] -= sm;
    return sqrt(3. / 2.) * sqrt(sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2] + 2 * sd[3] * sd[3] + 2 * sd[4] * sd[4] +
                                2 * sd[5] * sd[5]);
}

// x^n of the hardening law H ep^n: linear hardening (n = 1, and n - 1 = 0
// in the Newton derivative) needs no pow call, which in FP64 costs more than
// the rest of the update.
__device__ __forceinline__ double hpow(double x, double n) { return n == 1.0 ? x : (n == 0.0 ? 1.0 : pow(x, n)); }

// J2 return map (elastoPlastic, :640-691).  Returns dp (0 when elastic), sets
// sig, phi.  NR on the plastic multiplier from 0 with the reference's absolute
// tolerance 1e-5 on the yield function, capped at 200 steps (*nr_fail set).
__device__ __forceinline__ double j2_update(const PhaseMech& P, const double (&eps)[6], const double (&eps_old)[6],
                                            const double (&sig_old)[6], double ep, double (&sig)[6], double& phi,
                                            int* nr_fail) {
    double de[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) de[c] = eps[c] - eps_old[c];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < 6; ++j) s += P.C[i * 6 + j] * de[j];
        sig[i] = sig_old[i] + s;
    }
    double sd[6];
    const double seff = vonmises(sig, sd);
    phi = seff - P.Sy - P.H * hpow(ep, P.n);
    if (!(phi > 0)) return 0.0;
    double x = 0, xo = 0;
    int it = 0;
    for (;;) {
        x = xo - (seff - 3 * P.mu * xo - P.Sy - P.H * hpow(ep + xo, P.n)) /
                     (-3 * P.mu - P.H * P.n * hpow(ep + xo, P.n - 1));
        xo = x;
        const double res = seff - 3 * P.mu * x - P.Sy - P.H * hpow(ep + x, P.n);
        if (!(x == x)) { *nr_fail = 1; break; }
        if (fabs(res) < 1e-5) break;
        if (++it >= 200) { *nr_fail = 1; break; }
    }
    // sig -= (1.5 x / seff) C sd
    const double f = 1.5 * x / seff;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < 6; ++j) s += P.C[i * 6 + j] * sd[j];
        sig[i] -= f * s;
    }
    return x;
}

// Damage update (elastoDamage, :619-638): d_old = d; Y = sqrt(eps.C.eps) with
// doubled shear; if Y > Y0, d = max(1 - exp(-P (Y - Y0)), d_old); sig = (1-d) C eps
__device__ __forceinline__ void damage_update(const PhaseMech& P, const double (&eps)[6], double& d, double (&sig)[6]) {
    double ce[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < 6; ++j) s += P.C[i * 6 + j] * eps[j];
        ce[i] = s;
    }
    const double Y = sqrt(ce[0] * eps[0] + ce[1] * eps[1] + ce[2] * eps[2] + 2 * ce[3] * eps[3] + 2 * ce[4] * eps[4] +
                          2 * ce[5] * eps[5]);
    const double dold = d;
    if (Y > P.Y0) d = fmax(1 - exp(-P.P * (Y - P.Y0)), dold);
#pragma unroll
    for (int i = 0; i < 6; ++i) sig[i] = (1 - d) * ce[i];
}

template <typename T>
struct InelasticPtrs {
    const uint8_t* phase;
    T* eps;
    T* sig;
    const T* eps_old;
    const T* sig_old;
    const T* ep;   // equivalent plastic strain (J2)
    T* dmg;        // damage (ed)
    long long V;
    const PhaseMech* ph;
    int nph;
    int behav;
    int* nr_fail;
};

// constitutive from the current eps; sums (NSUM=13): sig (6), eps (6), 0.
// The state is FP64 in both precisions; T is the transforms' type (the
// strain increment xc arrives in it).
template <typename T>
struct EpiConstitutive {
    static constexpr int NSUM = 13;
    InelasticPtrs<double> p;
    PhaseMech* sm;
    // entry-bound base pointers (bind)
    double *eb = nullptr, *sb = nullptr, *db = nullptr;
    const double *eob = nullptr, *sob = nullptr, *epb = nullptr;
    __device__ __forceinline__ void bind(int b) {
        const long long o6 = (long long)b * 6 * p.V, o1 = (long long)b * p.V;
        eb = p.eps + o6;
        sb = p.sig + o6;
        eob = p.eps_old ? p.eps_old + o6 : nullptr;
        sob = p.sig_old ? p.sig_old + o6 : nullptr;
        epb = p.ep ? p.ep + o1 : nullptr;
        db = p.dmg ? p.dmg + o1 : nullptr;
    }
    __device__ __forceinline__ void load_smem(char* s, int = 0) {
        sm = (PhaseMech*)s;
        const double* src = (const double*)p.ph;
        double* dst = (double*)s;
        const int n = p.nph * (int)(sizeof(PhaseMech) / sizeof(double));
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    }
    // a voxel's inputs: phase, state, and (J2) the last increment's strain,
    // stress and equivalent plastic strain, or (damage) the damage variable
    struct In {
        int k;
        double e[6], eo[6], so[6], ep;
    };
    __device__ __forceinline__ In load(long long v) const {
        In q;
        q.k = p.phase[v];
        const long long V = p.V;
#pragma unroll
        for (int c = 0; c < 6; ++c) q.e[c] = eb[c * V + v];
        if (p.behav == BEHAV_J2) {
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                q.eo[c] = eob[c * V + v];
                q.so[c] = sob[c * V + v];
            }
            q.ep = epb[v];
        } else {
            q.ep = db[v];
        }
        return q;
    }
    // xc: increment from the inverse transform (zero for the standalone update)
    __device__ __forceinline__ void apply(int b, long long v, const T (&xc)[6], double* acc) const {
        apply_in(load(v), v, xc, acc);
    }
    __device__ __forceinline__ void apply_in(const In& q, long long v, const T (&xc)[6], double* acc) const {
        const PhaseMech& P = sm[q.k];
        const long long V = p.V;
        double e[6], sg[6];
        double dd = 0;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double inc = (double)xc[c];
            e[c] = q.e[c] + inc;
            dd += ((c >= 3) ? 2.0 : 1.0) * inc * inc;
        }
        if (p.behav == BEHAV_J2) {
            double phi;
            j2_update(P, e, q.eo, q.so, q.ep, sg, phi, p.nr_fail);
        } else {
            double d = q.ep;
            damage_update(P, e, d, sg);
            db[v] = d;
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            eb[c * V + v] = e[c];
            sb[c * V + v] = sg[c];
            acc[c] += sg[c];
            acc[6 + c] += e[c];
        }
        acc[12] += dd;
    }
};

// prologue: the stress field (FP64 state) in the transforms' type, or, with
// sig_old set, the stress increment of the load step sig - sig_old.  The
// increment form (FP32 transforms under the residual stop rule): sig_old is
// the previous step's equilibrated stress, so -Gamma0 (sig - sig_old)^ is the
// same strain update up to that step's residual, while the FP32 rounding of
// the transform scales with the increment instead of the total stress (which
// grows with every load step).
template <typename T>
struct ProStress {
    static constexpr int NSUM = 0;
    static constexpr int kW = 1;  // scalar loads only
    const double* sig;
    long long V;
    const double* sig_old = nullptr;
    const double* sb = nullptr;
    const double* sob = nullptr;
    struct Pre {
        double s[6];
    };
    __device__ __forceinline__ void bind(int b) {
        sb = sig + (long long)b * 6 * V;
        sob = sig_old ? sig_old + (long long)b * 6 * V : nullptr;
    }
    __device__ __forceinline__ void load_smem(char*, int = 0) {}
    __device__ __forceinline__ Pre load(int, long long v) const {
        Pre q;
#pragma unroll
        for (int c = 0; c < 6; ++c) q.s[c] = sob ? sb[c * V + v] - sob[c * V + v] : sb[c * V + v];
        return q;
    }
    __device__ __forceinline__ void eval_pre(const Pre& q, int, long long, T (&out)[6]) const {
#pragma unroll
        for (int c = 0; c < 6; ++c) out[c] = (T)q.s[c];
    }
    __device__ __forceinline__ void eval(int b, long long v, T (&out)[6], double*) const { eval_pre(load(b, v), b, v, out); }
};

// spectral op of the basic scheme: reductions of sig^ for the reference stop
// rule (cc, dd^2), then -Gamma0 sig^ with k = 0 from ctl
template <typename T>
struct SpecBasic {
    static constexpr bool kInverse = true;
    static constexpr int NSUM = 2;
    SpecGreen<T, 6> green;
    SpecEqVar<T, 6> eq;
    __device__ __forceinline__ void prepare(const Ctl* ctl, int b) { green.prepare(ctl, b); }
    __device__ __forceinline__ void apply(int b, int x, int y, int kz, typename Cx<T>::t (&v)[6], double* acc,
                                          const Ctl* ctl) const {
        eq.apply(b, x, y, kz, v, acc, ctl);
        green.apply(b, x, y, kz, v, acc, ctl);
    }
};

// The z-inverse epilogue wrapper: increment = xc (already scaled by 1/V).
template <typename T>
struct EpiBasic {
    static constexpr bool kJ2 = true;  // the inelastic update (its z inverse's CTAs per SM: M3D_J2_MINB)
    static constexpr int NSUM = 13;
    // 19 values per voxel.  FP64 transforms: one voxel's inputs prefetched
    // before the transform, then each next voxel's while the current one is
    // updated (j2_256 in FP64: 9.81 -> 9.28 s per solve).  FP32 transforms:
    // loaded at use (the rolling prefetch measured 19% slower there: 2.26 ->
    // 2.69 ms per 256^3 z inverse, at 240 instead of 180 registers).
    static constexpr bool kPrefetch = sizeof(T) == 8;
    static constexpr bool kRolling = sizeof(T) == 8;
    static constexpr int kW = 1;
    EpiConstitutive<T> c;
    typedef typename EpiConstitutive<T>::In Pre;
    __device__ __forceinline__ void bind(int b) { c.bind(b); }
    __device__ __forceinline__ Pre load(int, long long v) const { return c.load(v); }
    __device__ __forceinline__ void apply_pre(const Pre& q, int, long long v, T (&xc)[6], double* acc) const {
        c.apply_in(q, v, xc, acc);
    }
    __device__ __forceinline__ void load_smem(char* s, int b = 0) { c.load_smem(s, b); }
    __device__ __forceinline__ void apply(int b, long long v, T (&xc)[6], double* acc) const { c.apply(b, v, xc, acc); }
};

// standalone constitutive pass (increment start), same sums
template <typename T>
__global__ void k_constitutive(EpiConstitutive<T> epi, const Ctl* ctl, double* partials) {
    const int b = blockIdx.y;
    if (ctl[b].done) return;
    extern __shared__ __align__(16) char smem_raw[];
    double* red = (double*)smem_raw;
    epi.bind(b);
    epi.load_smem(smem_raw + 32 * 32 * sizeof(double));
    __syncthreads();
    double acc[13] = {};
    const T zero[6] = {0, 0, 0, 0, 0, 0};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < epi.p.V;
         v += (long long)gridDim.x * blockDim.x)
        epi.apply(b, v, zero, acc);
    block_reduce_store<13>(acc, red, partials, b, gridDim.x, blockIdx.x);
}

// Increment commit (export_homogen_var :722-746 then update_old_Variable
// :693-719): sums of eps_t, sig (6), sig_eff (J2) or d (ed), eps_p; then
// eps_p += dp where phi > 0, sig_old = sig, eps extrapolation.
__global__ void k_commit(InelasticPtrs<double> p, double* eps_old_w, double* sig_old_w, double* ep_w, int t_comp,
                         double* partials) {
    extern __shared__ __align__(16) char smem_raw[];
    double* red = (double*)smem_raw;
    PhaseMech* sm = (PhaseMech*)(smem_raw + 32 * 32 * sizeof(double));
    {
        const double* src = (const double*)p.ph;
        double* dst = (double*)sm;
        const int n = p.nph * (int)(sizeof(PhaseMech) / sizeof(double));
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const int b = blockIdx.y;
    double acc[9] = {};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < p.V; v += (long long)gridDim.x * blockDim.x) {
        const PhaseMech& P = sm[p.phase[v]];
        double e[6], s[6], sd[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const long long idx = ((long long)b * 6 + c) * p.V + v;
            e[c] = (double)p.eps[idx];
            s[c] = (double)p.sig[idx];
        }
        acc[0] += e[t_comp];
#pragma unroll
        for (int c = 0; c < 6; ++c) acc[1 + c] += s[c];
        if (p.behav == BEHAV_J2) {
            const double ep = (double)p.ep[(long long)b * p.V + v];
            acc[7] += vonmises(s, sd);
            acc[8] += ep;
            // recompute the last return map to get dp and phi (same inputs as the
            // last constitutive call, so the same values)
            double eo[6], so[6], st[6], phi;
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const long long idx = ((long long)b * 6 + c) * p.V + v;
                eo[c] = (double)p.eps_old[idx];
                so[c] = (double)p.sig_old[idx];
            }
            const double dp = j2_update(P, e, eo, so, ep, st, phi, p.nr_fail);
            if (phi > 0) ep_w[(long long)b * p.V + v] = ep + dp;
#pragma unroll
            for (int c = 0; c < 6; ++c) sig_old_w[((long long)b * 6 + c) * p.V + v] = s[c];
        } else {
            acc[7] += (double)p.dmg[(long long)b * p.V + v];
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const long long idx = ((long long)b * 6 + c) * p.V + v;
            const double eo = (double)p.eps_old[idx];
            eps_old_w[idx] = e[c];
            p.eps[idx] = e[c] + (e[c] - eo);
        }
    }
    block_reduce_store<9>(acc, red, partials, b, gridDim.x, blockIdx.x);
}

enum PolicyJ2 {
    POLJ2_START = 0,  // after the increment-start constitutive: sum_prev, updateE
    POLJ2_CHECK = 1,  // after the turnaround: reference stop rule for the previous sweep
    POLJ2_SWEEP = 2,  // after the inverse pass: count, record sums, residual, updateE
};

// ctl.aux layout for the inelastic path
enum {
    AUX_SUMSIG = 0,     // sum of all sig components of the current state
    AUX_ESUM_USED = 1,  // sum(E) used by the current state's sweep
    AUX_MEANS = 2,      // 12: <sig_c>, <eps_c>
    AUX_S0 = 14,        // 6: S0 X0
    AUX_DESUM = 20,     // sum(dE) * incNo
    AUX_PXY = 21,       // prod(S0 X0, X0)
    AUX_X0 = 22,        // 6: X0
};

__device__ __forceinline__ double prodv(const double* a, const double* b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + 2 * a[3] * b[3] + 2 * a[4] * b[4] + 2 * a[5] * b[5];
}

// updateE (:583-594): x = S0 <sig> - <eps>; k = (sum(dE) incNo + prod(x,X0)) / prod(S0 X0, X0);
// E = k S0 X0 - S0 <sig> + <eps>.  S0 is isotropic: passed as its 6x6 in aux2.
__device__ __forceinline__ void policy_j2(Ctl& c, const double* tot, int policy, double V, const double* S0m);

__global__ void k_finalize_j2(Ctl* ctl, const double* __restrict__ partials, int NS, int nblk, int policy, double V,
                              const double* __restrict__ S0m) {
    const int b = blockIdx.x;
    if (ctl[b].done) return;
    __shared__ double red[256];
    __shared__ double tot[16];
    sum_partials(partials, NS, nblk, b, red, tot);
    if (threadIdx.x == 0) policy_j2(ctl[b], tot, policy, V, S0m);
}

struct FinJ2 {
    int policy;
    double V;
    const double* S0m;
    int* counter;
    __device__ __forceinline__ void run(Ctl* ctl, const double* partials, int NS, int nblk, int b, double* red,
                                        double* tot) const {
        sum_partials(partials, NS, nblk, b, red, tot);
        if (threadIdx.x == 0) policy_j2(ctl[b], tot, policy, V, S0m);
    }
};

__device__ __forceinline__ void policy_j2(Ctl& c, const double* tot, int policy, double V, const double* S0m) {
    if (policy == POLJ2_CHECK) {
        // convergenceCheck of the state produced by the previous sweep (itNo = iters)
        if (c.iters < 1) return;
        const double eq = tot[0] / sqrt(tot[1]) / V;
        c.eqvar = eq;
        c.diff_sum = fabs((c.aux[AUX_SUMSIG] - c.sum_prev) / (V * c.den * c.aux[AUX_ESUM_USED]));
        c.diff_eq = fabs(eq - c.eq_old);
        c.eq_old = eq;
        if (c.iters > 1 && c.diff_eq < c.tol_eq && c.diff_sum < c.tol_field) c.done = 1;
        else if (c.iters > c.max_iter) { c.status = 1; c.done = 1; }
        return;
    }
    // START / SWEEP: tot = [sig sums 6, eps sums 6, |d eps|^2]
    double ms[6], me[6];
    double sumsig = 0;
    for (int i = 0; i < 6; ++i) {
        ms[i] = tot[i] / V;
        me[i] = tot[6 + i] / V;
        sumsig += tot[i];
    }
    if (policy == POLJ2_SWEEP) {
        c.iters += 1;
        double es = 0;
        for (int i = 0; i < 6; ++i) es += c.E[i];
        c.aux[AUX_ESUM_USED] = es;
        c.sum_prev = c.aux[AUX_SUMSIG];  // sum_field_old of this sweep = previous state's sum
        c.residual = sqrt(tot[12] / V) / c.enorm;
        if (!(c.residual == c.residual)) { c.status = 2; c.done = 1; }
    }
    c.aux[AUX_SUMSIG] = sumsig;
    for (int i = 0; i < 6; ++i) { c.aux[AUX_MEANS + i] = ms[i]; c.aux[AUX_MEANS + 6 + i] = me[i]; }
    // updateE for the next sweep
    double xv[6];
    for (int i = 0; i < 6; ++i) {
        double s = 0;
        for (int j = 0; j < 6; ++j) s += S0m[i * 6 + j] * ms[j];
        xv[i] = s - me[i];
    }
    const double* X0 = &c.aux[AUX_X0];
    const double* y = &c.aux[AUX_S0];
    const double kf = (c.aux[AUX_DESUM] + prodv(xv, X0)) / c.aux[AUX_PXY];
    for (int i = 0; i < 6; ++i) {
        c.E[i] = kf * y[i] - (xv[i] + me[i]) + me[i];
        c.kzero[i] = (c.E[i] - me[i]) * V;
    }
    if (policy == POLJ2_SWEEP && c.crit_residual && c.done == 0) {
        if (c.residual < c.tol_field) c.done = 1;
        else if (c.iters >= c.max_iter) { c.status = 1; c.done = 1; }
    }
}

}  // namespace m3d

// Host-side state of the inelastic path (buffers owned by the solver handle).
struct InelasticState {
    void* eps = nullptr;
    void* sig = nullptr;
    void* eps_old = nullptr;
    void* sig_old = nullptr;
    void* ep = nullptr;
    void* dmg = nullptr;
    m3d::PhaseMech* d_ph = nullptr;
    double* d_S0 = nullptr;
    int* d_nrfail = nullptr;
    size_t batch = 0;
    void free_all();
    int setup(m3d_solver* h);
    int means(m3d_solver* h, int b, double* strain_mean, double* stress_mean);
    int get_field(m3d_solver* h, int which, int b, double* out);
};
