// physics.cuh -- the pointwise and spectral physics fused into the FFT passes.
//
// One linear accelerated (Eyre-Milton) sweep in unified form, for every
// elastic and thermal scheme of the reference:
//     pol   = P[ph] x                        (prologue of the z-forward pass)
//     x_c^  = -G(xi) pol^ ,  x_c^(0) = E V    (spectral op in the x turnaround)
//     x    += A[ph] (x_c - x)                (epilogue of the z-inverse pass)
// with, per scheme (reference file:line):
//   elastic strain-based: x = eps, P = C - C0, G = Gamma0, A = 2(C+C0)^-1 C0
//       (src/3d/FFT_analysis3D.cpp:759-760, 223-224, 283-288, 539-546)
//   elastic stress-based: x = sig, P = S - S0, G = Delta0, A = 2(S+S0)^-1 S0
//       (:765-766, 226-228, 290-293)
//   thermal gradient-based: x = grad T, P = (k - k0) I, G = xi xi^T/(k0|xi|^2),
//       A = 2k0/(k+k0)   (src/3dTherm/FFT_thermal3D.cpp:451-454, 126-136, 242-253)
//   thermal flux-based: x = q, P = (1/k - 1/k0) I, G = k0 (I - n n^T),
//       A = 2r0/(r+r0)   (:456-459, 161-169, 255-266)
// The reference forms K0 g - q and R0 q - g (opposite sign) and applies +G;
// the products are identical.  Elastic contractions count each shear term
// twice (tensor shear in Voigt slots 3..5, :315-319), which the closed forms
// below do by working on the full symmetric tensor.
#pragma once
#include "passes.cuh"

namespace m3d {

constexpr int kMaxPhases = 16;

enum GreenKind { GREEN_STRAIN = 0, GREEN_STRESS = 1, GREEN_TGRAD = 2, GREEN_TFLUX = 3 };

// Signed frequency of FFT index i: i <= lim -> i, else i - wrap.
__device__ __forceinline__ int sfreq(int i, int lim, int wrap) { return i <= lim ? i : i - wrap; }

template <typename T>
__device__ __forceinline__ void green_elastic_strain(T x0, T x1, T x2, T p1, T p2, const T (&t)[6], T (&o)[6]) {
    // q = tau xi ; s = xi . tau . xi ; out_ij = -[ p1 (xi_j q_i + xi_i q_j)/|xi|^2 - p2 s xi_i xi_j/|xi|^4 ]
    const T q0 = t[0] * x0 + t[5] * x1 + t[4] * x2;
    const T q1 = t[5] * x0 + t[1] * x1 + t[3] * x2;
    const T q2 = t[4] * x0 + t[3] * x1 + t[2] * x2;
    const T s = x0 * q0 + x1 * q1 + x2 * q2;
    const T inv = (T)1 / (x0 * x0 + x1 * x1 + x2 * x2);
    const T a = p1 * inv;
    const T bb = p2 * s * inv * inv;
    o[0] = -((T)2 * a * x0 * q0 - bb * x0 * x0);
    o[1] = -((T)2 * a * x1 * q1 - bb * x1 * x1);
    o[2] = -((T)2 * a * x2 * q2 - bb * x2 * x2);
    o[3] = -(a * (x2 * q1 + x1 * q2) - bb * x1 * x2);
    o[4] = -(a * (x2 * q0 + x0 * q2) - bb * x0 * x2);
    o[5] = -(a * (x1 * q0 + x0 * q1) - bb * x0 * x1);
}

template <typename T>
__device__ __forceinline__ void green_elastic_stress(T x0, T x1, T x2, T c3, T c4x2, const T (&t)[6], T (&o)[6]) {
    // P = I - n n^T ; out_ij = -[ c3 P_ij (P:tau) + 2 c4 (P tau P)_ij ]
    const T inv = (T)1 / sqrt(x0 * x0 + x1 * x1 + x2 * x2);
    const T n0 = x0 * inv, n1 = x1 * inv, n2 = x2 * inv;
    const T u0 = t[0] * n0 + t[5] * n1 + t[4] * n2;
    const T u1 = t[5] * n0 + t[1] * n1 + t[3] * n2;
    const T u2 = t[4] * n0 + t[3] * n1 + t[2] * n2;
    const T s = n0 * u0 + n1 * u1 + n2 * u2;
    const T ptr = (t[0] + t[1] + t[2]) - s;
    auto ptp = [&](T tij, T ni, T nj, T ui, T uj) { return tij - ni * uj - ui * nj + s * ni * nj; };
    o[0] = -(c3 * ((T)1 - n0 * n0) * ptr + c4x2 * ptp(t[0], n0, n0, u0, u0));
    o[1] = -(c3 * ((T)1 - n1 * n1) * ptr + c4x2 * ptp(t[1], n1, n1, u1, u1));
    o[2] = -(c3 * ((T)1 - n2 * n2) * ptr + c4x2 * ptp(t[2], n2, n2, u2, u2));
    o[3] = -(c3 * (-n1 * n2) * ptr + c4x2 * ptp(t[3], n1, n2, u1, u2));
    o[4] = -(c3 * (-n0 * n2) * ptr + c4x2 * ptp(t[4], n0, n2, u0, u2));
    o[5] = -(c3 * (-n0 * n1) * ptr + c4x2 * ptp(t[5], n0, n1, u0, u1));
}

// ----------------------------------------------------------------------------
// Spectral op: apply -G(xi) at every mode except k = 0, which is set from ctl.
// ----------------------------------------------------------------------------
template <typename T, int C>
struct SpecGreen {
    static constexpr bool kInverse = true;
    static constexpr int NSUM = 0;
    GridDims g;
    int kind;        // GreenKind
    int pos_nyq;     // 1: index <= N/2 is positive (thermal gradient-based)
    int xwrap;       // wrap length of the x index (Ny for the flux-based thermal quirk)
    int zero_k0;     // 1: k = 0 mode set to 0 (correction solves), else ctl.kzero
    T p1, p2;
    // take the operator of batch entry b's RVE from its control block
    __device__ __forceinline__ void prepare(const Ctl* ctl, int b) {
        kind = ctl[b].gkind;
        pos_nyq = ctl[b].gnyq;
        xwrap = ctl[b].gxw;
        p1 = (T)ctl[b].gp1;
        p2 = (T)ctl[b].gp2;
    }
    __device__ __forceinline__ void apply(int b, int x, int y, int kz, typename Cx<T>::t (&v)[C], double*,
                                          const Ctl* ctl) const {
        typedef typename Cx<T>::t C2;
        if (x == 0 && y == 0 && kz == 0) {
#pragma unroll
            for (int c = 0; c < C; ++c) v[c] = mk<C2>(zero_k0 ? (T)0 : (T)ctl[b].kzero[c], (T)0);
            return;
        }
        const T x0 = (T)sfreq(kz, pos_nyq ? g.Nz / 2 : (g.Nz - 1) / 2, g.Nz);
        const T x1 = (T)sfreq(y, pos_nyq ? g.Ny / 2 : (g.Ny - 1) / 2, g.Ny);
        const T x2 = (T)sfreq(x, pos_nyq ? g.Nx / 2 : (g.Nx - 1) / 2, xwrap);
        if constexpr (C == 6) {
            T tr[6], ti[6], orr[6], oi[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) { tr[c] = v[c].x; ti[c] = v[c].y; }
            if (kind == GREEN_STRAIN) {
                green_elastic_strain(x0, x1, x2, p1, p2, tr, orr);
                green_elastic_strain(x0, x1, x2, p1, p2, ti, oi);
            } else {
                green_elastic_stress(x0, x1, x2, p1, p2, tr, orr);
                green_elastic_stress(x0, x1, x2, p1, p2, ti, oi);
            }
#pragma unroll
            for (int c = 0; c < 6; ++c) v[c] = mk<C2>(orr[c], oi[c]);
        } else {
            const T n2 = x0 * x0 + x1 * x1 + x2 * x2;
            const C2 d = mk<C2>(x0 * v[0].x + x1 * v[1].x + x2 * v[2].x, x0 * v[0].y + x1 * v[1].y + x2 * v[2].y);
            const T xs[3] = {x0, x1, x2};
            if (kind == GREEN_TGRAD) {
                const T f = -p1 / n2;  // p1 = 1/k0
#pragma unroll
                for (int c = 0; c < 3; ++c) v[c] = mk<C2>(f * xs[c] * d.x, f * xs[c] * d.y);
            } else {
                const T f = (T)1 / n2;  // p1 = k0
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    v[c] = mk<C2>(-p1 * (v[c].x - f * xs[c] * d.x), -p1 * (v[c].y - f * xs[c] * d.y));
            }
        }
    }
};

template <typename T> using SpecGreenT = SpecGreen<T, 3>;

// ----------------------------------------------------------------------------
// Reference stop rule (convergenceCheck): forward spectrum of the stress (heat
// flux) reduced to cc = sum sqrt|...| and dd^2 = |stress^(0)|^2
// (src/3d/FFT_analysis3D.cpp:357-392, src/3dTherm/FFT_thermal3D.cpp:309-338).
// ----------------------------------------------------------------------------
template <typename T, int C>
struct SpecEqVar {
    static constexpr bool kInverse = false;
    static constexpr int NSUM = 2;
    GridDims g;
    __device__ __forceinline__ void prepare(const Ctl*, int) {}
    __device__ __forceinline__ void apply(int, int x, int y, int kz, typename Cx<T>::t (&v)[C], double* acc,
                                          const Ctl*) const {
        if (x == 0 && y == 0 && kz == 0) {
            double dd = 0;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const double w = (C == 6 && c >= 3) ? 2.0 : 1.0;
                dd += w * ((double)v[c].x * v[c].x + (double)v[c].y * v[c].y);
            }
            acc[1] += dd;
        }
        if constexpr (C == 6) {
            if (kz < 1) return;  // elastic sum starts at z = 1 (:368)
            const double z0 = sfreq(kz, (g.Nz - 1) / 2, g.Nz), z1 = sfreq(y, (g.Ny - 1) / 2, g.Ny),
                         z2 = sfreq(x, (g.Nx - 1) / 2, g.Nx);
            double p[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) p[c] = (double)v[c].x * v[c].x + (double)v[c].y * v[c].y;
            const double s = p[0] * z0 * z0 + p[1] * z1 * z1 + p[2] * z2 * z2 + p[3] * ((z1 + z1) + (z2 + z2)) +
                             p[4] * ((z0 + z0) + (z2 + z2)) + p[5] * ((z0 + z0) + (z1 + z1));
            acc[0] += sqrt(fabs(s));
        } else {
            const double z0 = sfreq(kz, g.Nz / 2, g.Nz), z1 = sfreq(y, g.Ny / 2, g.Ny), z2 = sfreq(x, g.Nx / 2, g.Nx);
            double p[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) p[c] = (double)v[c].x * v[c].x + (double)v[c].y * v[c].y;
            acc[0] += sqrt(p[0] * z0 * z0 + p[1] * z1 * z1 + p[2] * z2 * z2);
        }
    }
};

// ----------------------------------------------------------------------------
// Prologues
// ----------------------------------------------------------------------------
// Every prologue/epilogue splits into load() -- the global reads of one voxel
// -- and a compute step, so a pass can issue the loads of all its voxels
// before the first compute and keep them in flight together.  Operators with
// kW = 4 also offer loadw()/..._prew(): four consecutive voxels per call with
// 16-byte loads and stores of each component (the fast z passes use them;
// voxel offsets are multiples of 4 there).
// ----------------------------------------------------------------------------
__device__ __forceinline__ void ld4(const float* p, float (&o)[4]) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&o)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void ld4(const uint8_t* p, int (&o)[4]) {
    const uchar4 v = *reinterpret_cast<const uchar4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void st4(float* p, const float (&o)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&o)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(o[0], o[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(o[2], o[3]);
}
// out = M[ph] x  (M: per phase CxC, row-major, double in global -> T in smem)
template <typename T, int C, typename TX = T>
struct ProMat {
    static constexpr int NSUM = 0;
    const uint8_t* phase;
    const TX* x;
    long long V;
    const double* mats;
    int nph;
    T* sm;
    int lc = 0;             // batch entries per RVE (0: one RVE shared by all entries)
    long long mstride = 0;  // stride of an RVE's table block in `mats`
    const uint8_t* phb = nullptr;  // phase map and state of the bound entry (bind)
    const TX* xb = nullptr;
    struct Pre {
        int p;
        T xv[C];
    };
    // per-block: address the entry's RVE and state once, so per-voxel loads
    // are plain offsets
    __device__ __forceinline__ void bind(int b) {
        phb = phase + (lc ? (long long)(b / lc) * V : 0);
        xb = x + (long long)b * C * V;
    }
    __device__ __forceinline__ void load_smem(char* s, int b) {
        sm = (T*)s;
        const double* m = mats + (lc ? (long long)(b / lc) * mstride : 0);
        for (int i = threadIdx.x; i < nph * C * C; i += blockDim.x) sm[i] = (T)m[i];
    }
    __device__ __forceinline__ Pre load(int, long long v) const {
        Pre q;
        q.p = phb[v];
#pragma unroll
        for (int c = 0; c < C; ++c) q.xv[c] = (T)xb[c * V + v];
        return q;
    }
    __device__ __forceinline__ void eval_pre(const Pre& q, int, long long, T (&out)[C]) const {
        const T* M = sm + q.p * C * C;
#pragma unroll
        for (int i = 0; i < C; ++i) {
            T s = 0;
#pragma unroll
            for (int j = 0; j < C; ++j) s += M[i * C + j] * q.xv[j];
            out[i] = s;
        }
    }
    __device__ __forceinline__ void eval(int b, long long v, T (&out)[C], double*) const { eval_pre(load(b, v), b, v, out); }
    static constexpr int kW = 4;
    struct PreW {
        int p[4];
        T xv[4][C];
    };
    __device__ __forceinline__ PreW loadw(long long v) const {
        PreW q;
        ld4(phb + v, q.p);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            TX t[4];
            ld4(xb + c * V + v, t);
#pragma unroll
            for (int w = 0; w < 4; ++w) q.xv[w][c] = (T)t[w];
        }
        return q;
    }
    __device__ __forceinline__ void eval_prew(const PreW& q, int w, T (&out)[C]) const {
        const T* M = sm + q.p[w] * C * C;
#pragma unroll
        for (int i = 0; i < C; ++i) {
            T s = 0;
#pragma unroll
            for (int j = 0; j < C; ++j) s += M[i * C + j] * q.xv[w][j];
            out[i] = s;
        }
    }
};

// FP64 defect pass of the refinement: x += delta (FP32 correction of the
// previous inner solve, if any), then out = P[ph] x.
template <int C>
struct ProRefine64 {
    static constexpr int NSUM = 0;
    const uint8_t* phase;
    double* x;
    const float* delta;  // may be null
    long long V;
    const double* mats;
    int nph;
    double* sm;
    int lc = 0;
    long long mstride = 0;
    const uint8_t* phb = nullptr;
    double* xb = nullptr;
    const float* db = nullptr;
    struct Pre {
        int p;
        double xv[C];
    };
    __device__ __forceinline__ void bind(int b) {
        phb = phase + (lc ? (long long)(b / lc) * V : 0);
        xb = x + (long long)b * C * V;
        db = delta ? delta + (long long)b * C * V : nullptr;
    }
    __device__ __forceinline__ void load_smem(char* s, int b) {
        sm = (double*)s;
        const double* m = mats + (lc ? (long long)(b / lc) * mstride : 0);
        for (int i = threadIdx.x; i < nph * C * C; i += blockDim.x) sm[i] = m[i];
    }
    __device__ __forceinline__ Pre load(int, long long v) const {
        Pre q;
        q.p = phb[v];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            q.xv[c] = xb[c * V + v];
            if (db) q.xv[c] += (double)db[c * V + v];
        }
        return q;
    }
    __device__ __forceinline__ void eval_pre(const Pre& q, int, long long v, double (&out)[C]) const {
        const double* M = sm + q.p * C * C;
        if (db) {
#pragma unroll
            for (int c = 0; c < C; ++c) xb[c * V + v] = q.xv[c];
        }
#pragma unroll
        for (int i = 0; i < C; ++i) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < C; ++j) s += M[i * C + j] * q.xv[j];
            out[i] = s;
        }
    }
    __device__ __forceinline__ void eval(int b, long long v, double (&out)[C], double*) const {
        eval_pre(load(b, v), b, v, out);
    }
    static constexpr int kW = 4;
    struct PreW {
        int p[4];
        double xv[4][C];
    };
    // the folded state x + delta is written back at load time (each voxel
    // belongs to one thread and nothing else in the pass reads x)
    __device__ __forceinline__ PreW loadw(long long v) const {
        PreW q;
        ld4(phb + v, q.p);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            double t[4];
            ld4(xb + c * V + v, t);
            if (db) {
                float d[4];
                ld4(db + c * V + v, d);
#pragma unroll
                for (int w = 0; w < 4; ++w) t[w] += (double)d[w];
                st4(xb + c * V + v, t);
            }
#pragma unroll
            for (int w = 0; w < 4; ++w) q.xv[w][c] = t[w];
        }
        return q;
    }
    __device__ __forceinline__ void eval_prew(const PreW& q, int w, double (&out)[C]) const {
        const double* M = sm + q.p[w] * C * C;
#pragma unroll
        for (int i = 0; i < C; ++i) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < C; ++j) s += M[i * C + j] * q.xv[w][j];
            out[i] = s;
        }
    }
};

// ----------------------------------------------------------------------------
// Epilogues
// ----------------------------------------------------------------------------
// EM update: d = x_c (+ r) - x ; x += A[ph] d ; sums: [0] sum w d^2, [1] sum_c (O x_new)_c
template <typename T, int C>
struct EpiEM {
    static constexpr int NSUM = 2;
    static constexpr bool kPrefetch = true;
    const uint8_t* phase;
    T* x;
    const float* r;  // defect forcing of the correction solve, may be null
    long long V;
    const double* amats;  // [nph][C][C]
    const double* osum;   // [nph][C]: column sums of the "other field" matrix
    int nph;
    T* sm;
    int lc = 0;
    long long mstride = 0;
    const uint8_t* phb = nullptr;
    T* xb = nullptr;
    const float* rb = nullptr;
    struct Pre {
        int p;
        T xv[C];
        T rv[C];
    };
    __device__ __forceinline__ void bind(int b) {
        phb = phase + (lc ? (long long)(b / lc) * V : 0);
        xb = x + (long long)b * C * V;
        rb = r ? r + (long long)b * C * V : nullptr;
    }
    __device__ __forceinline__ void load_smem(char* s, int b) {
        sm = (T*)s;
        const long long o = lc ? (long long)(b / lc) * mstride : 0;
        for (int i = threadIdx.x; i < nph * C * C; i += blockDim.x) sm[i] = (T)amats[o + i];
        for (int i = threadIdx.x; i < nph * C; i += blockDim.x) sm[nph * C * C + i] = (T)osum[o + i];
    }
    __device__ __forceinline__ Pre load(int, long long v) const {
        Pre q;
        q.p = phb[v];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            q.xv[c] = xb[c * V + v];
            q.rv[c] = rb ? (T)rb[c * V + v] : (T)0;
        }
        return q;
    }
    __device__ __forceinline__ void apply_pre(const Pre& q, int, long long v, T (&xc)[C], double* acc) const {
        const T* Am = sm + q.p * C * C;
        const T* os = sm + nph * C * C + q.p * C;
        T d[C], xn[C];
#pragma unroll
        for (int c = 0; c < C; ++c) d[c] = (xc[c] + q.rv[c]) - q.xv[c];
        double rs = 0, ot = 0;
#pragma unroll
        for (int i = 0; i < C; ++i) {
            const double w = (C == 6 && i >= 3) ? 2.0 : 1.0;
            rs += w * (double)d[i] * (double)d[i];
            T s = 0;
#pragma unroll
            for (int j = 0; j < C; ++j) s += Am[i * C + j] * d[j];
            xn[i] = q.xv[i] + s;
            xb[i * V + v] = xn[i];
        }
#pragma unroll
        for (int c = 0; c < C; ++c) ot += (double)os[c] * (double)xn[c];
        acc[0] += rs;
        acc[1] += ot;
    }
    __device__ __forceinline__ void apply(int b, long long v, T (&xc)[C], double* acc) const {
        apply_pre(load(b, v), b, v, xc, acc);
    }
    static constexpr int kW = 4;
    struct PreW {
        int p[4];
        T xv[4][C];
        T rv[4][C];
    };
    __device__ __forceinline__ PreW loadw(long long v) const {
        PreW q;
        ld4(phb + v, q.p);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            T t[4];
            ld4(xb + c * V + v, t);
            float u[4] = {0.f, 0.f, 0.f, 0.f};
            if (rb) ld4(rb + c * V + v, u);
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                q.xv[w][c] = t[w];
                q.rv[w][c] = (T)u[w];
            }
        }
        return q;
    }
    __device__ __forceinline__ void apply_prew(const PreW& q, long long v, T (&xc)[4][C], double* acc) const {
        T xn[C][4];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const T* Am = sm + q.p[w] * C * C;
            const T* os = sm + nph * C * C + q.p[w] * C;
            T d[C];
#pragma unroll
            for (int c = 0; c < C; ++c) d[c] = (xc[w][c] + q.rv[w][c]) - q.xv[w][c];
            double rs = 0, ot = 0;
#pragma unroll
            for (int i = 0; i < C; ++i) {
                const double wt = (C == 6 && i >= 3) ? 2.0 : 1.0;
                rs += wt * (double)d[i] * (double)d[i];
                T s = 0;
#pragma unroll
                for (int j = 0; j < C; ++j) s += Am[i * C + j] * d[j];
                xn[i][w] = q.xv[w][i] + s;
            }
#pragma unroll
            for (int c = 0; c < C; ++c) ot += (double)os[c] * (double)xn[c][w];
            acc[0] += rs;
            acc[1] += ot;
        }
#pragma unroll
        for (int c = 0; c < C; ++c) st4(xb + c * V + v, xn[c]);
    }
};

// FP64 defect of the refinement: r = x_c - x (stored FP32), x unchanged.
// sums: [0] sum w r^2, [1] sum_c (O x)_c
template <int C>
struct EpiDefect {
    static constexpr int NSUM = 2;
    static constexpr bool kPrefetch = true;
    const uint8_t* phase;
    const double* x;
    float* r;
    long long V;
    const double* osum;
    int nph;
    double* sm;
    int lc = 0;
    long long mstride = 0;
    const uint8_t* phb = nullptr;
    const double* xb = nullptr;
    float* rb = nullptr;
    struct Pre {
        int p;
        double xv[C];
    };
    __device__ __forceinline__ void bind(int b) {
        phb = phase + (lc ? (long long)(b / lc) * V : 0);
        xb = x + (long long)b * C * V;
        rb = r + (long long)b * C * V;
    }
    __device__ __forceinline__ void load_smem(char* s, int b) {
        sm = (double*)s;
        const double* m = osum + (lc ? (long long)(b / lc) * mstride : 0);
        for (int i = threadIdx.x; i < nph * C; i += blockDim.x) sm[i] = m[i];
    }
    __device__ __forceinline__ Pre load(int, long long v) const {
        Pre q;
        q.p = phb[v];
#pragma unroll
        for (int c = 0; c < C; ++c) q.xv[c] = xb[c * V + v];
        return q;
    }
    __device__ __forceinline__ void apply_pre(const Pre& q, int, long long v, double (&xc)[C], double* acc) const {
        double rs = 0, ot = 0;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const double d = xc[c] - q.xv[c];
            rb[c * V + v] = (float)d;
            const double w = (C == 6 && c >= 3) ? 2.0 : 1.0;
            rs += w * d * d;
            ot += sm[q.p * C + c] * q.xv[c];
        }
        acc[0] += rs;
        acc[1] += ot;
    }
    __device__ __forceinline__ void apply(int b, long long v, double (&xc)[C], double* acc) const {
        apply_pre(load(b, v), b, v, xc, acc);
    }
    static constexpr int kW = 4;
    struct PreW {
        int p[4];
        double xv[4][C];
    };
    __device__ __forceinline__ PreW loadw(long long v) const {
        PreW q;
        ld4(phb + v, q.p);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            double t[4];
            ld4(xb + c * V + v, t);
#pragma unroll
            for (int w = 0; w < 4; ++w) q.xv[w][c] = t[w];
        }
        return q;
    }
    __device__ __forceinline__ void apply_prew(const PreW& q, long long v, double (&xc)[4][C], double* acc) const {
        float rr[C][4];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            double rs = 0, ot = 0;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const double d = xc[w][c] - q.xv[w][c];
                rr[c][w] = (float)d;
                const double wt = (C == 6 && c >= 3) ? 2.0 : 1.0;
                rs += wt * d * d;
                ot += sm[q.p[w] * C + c] * q.xv[w][c];
            }
            acc[0] += rs;
            acc[1] += ot;
        }
#pragma unroll
        for (int c = 0; c < C; ++c) st4(rb + c * V + v, rr[c]);
    }
};

// ----------------------------------------------------------------------------
// Finalize: deterministic sum of per-block partials, then a policy step.
// ----------------------------------------------------------------------------
enum Policy {
    POL_RESIDUAL = 0,     // linear sweep, product stop rule on rms |x_c - x| / |E|
    POL_REF_SWEEP = 1,    // linear sweep, reference rule: record sum, count sweep
    POL_REF_CHECK = 2,    // reference rule: eqVar from the check pass, decide
    POL_REFINE_OUTER = 3, // FP64 defect pass
    POL_REFINE_INNER = 4, // FP32 correction sweep
};

// tot[s] = sum over the nblk block partials of sum s, in a fixed order (every
// thread strides the same blocks, then a fixed tree) -> bit-reproducible.
// Called by all threads of a block whose size is a power of two; the first
// min(blockDim.x, 256) threads take part (red holds 256 doubles).
__device__ __forceinline__ void sum_partials(const double* partials, int NS, int nblk, int b, double* red,
                                             double* tot) {
    const int nt = blockDim.x < 256 ? (int)blockDim.x : 256;
    for (int s = 0; s < NS; ++s) {
        const double* p = partials + ((long long)b * NS + s) * nblk;
        if (threadIdx.x < nt) {
            double t = 0;
            for (int i = threadIdx.x; i < nblk; i += nt) t += __ldcg(p + i);
            red[threadIdx.x] = t;
        }
        __syncthreads();
        for (int o = nt / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) tot[s] = red[0];
        __syncthreads();
    }
}

__device__ __forceinline__ void policy_linear(Ctl& c, const double* tot, int policy, double V, const Ctl* outer,
                                              int b);

// Stop ratio of the FP32 correction solve of the refinement (its defect norm
// relative to the FP64 defect it started from): the correction only has to
// shrink the defect by the factor still missing to reach the tolerance (with
// a 0.3 margin), but never asks for less than 2e-5, what FP32 sweeps reach
// reliably, nor more than 0.1.  Same arithmetic on host and device.
__host__ __device__ inline double refine_inner_tol(double tol, double res) {
    const double need = res > 0 ? 0.3 * tol / res : 0.1;
    return fmin(0.1, fmax(2e-5, need));
}

static __global__ void k_finalize(Ctl* ctl, const double* __restrict__ partials, int NS, int nblk, int policy, double V,
                                  const Ctl* outer) {
    const int b = blockIdx.x;
    if (ctl[b].done) return;
    __shared__ double red[256];
    __shared__ double tot[16];
    sum_partials(partials, NS, nblk, b, red, tot);
    if (threadIdx.x == 0) policy_linear(ctl[b], tot, policy, V, outer, b);
}

// Finalize run by the last block of the pass that produced the partials.
struct FinLinear {
    int policy;
    double V;
    const Ctl* outer;
    int* counter;
    __device__ __forceinline__ void run(Ctl* ctl, const double* partials, int NS, int nblk, int b, double* red,
                                        double* tot) const {
        sum_partials(partials, NS, nblk, b, red, tot);
        if (threadIdx.x == 0) policy_linear(ctl[b], tot, policy, V, outer, b);
    }
};

__device__ __forceinline__ void policy_linear(Ctl& c, const double* tot, int policy, double V, const Ctl* outer,
                                              int b) {
    switch (policy) {
        case POL_RESIDUAL: {
            c.iters += 1;
            const double res = sqrt(tot[0] / V) / c.enorm;
            c.residual = res;
            c.aux[0] = tot[1];
            if (!(res == res) || isinf(res)) { c.status = 2; c.done = 1; }
            else if (res < c.tol_field) c.done = 1;
            else if (c.iters >= c.max_iter) { c.status = 1; c.done = 1; }
            break;
        }
        case POL_REF_SWEEP: {
            c.iters += 1;
            c.residual = sqrt(tot[0] / V) / c.enorm;
            c.aux[0] = tot[1];
            break;
        }
        case POL_REF_CHECK: {
            const double eq = tot[0] / sqrt(tot[1]) / V;
            c.eqvar = eq;
            c.diff_sum = fabs((c.aux[0] - c.sum_prev) / c.den);
            c.diff_eq = fabs(eq - c.eq_old);
            c.eq_old = eq;
            c.sum_prev = c.aux[0];
            if (!(c.residual == c.residual)) { c.status = 2; c.done = 1; }
            else if (c.iters > 1 && c.diff_eq < c.tol_eq && c.diff_sum < c.tol_field) c.done = 1;
            else if (c.iters > c.max_iter) { c.status = 1; c.done = 1; }
            break;
        }
        case POL_REFINE_OUTER: {
            c.iters += 1;
            const double res = sqrt(tot[0] / V) / c.enorm;
            c.residual = res;
            c.rnorm = sqrt(tot[0]);
            c.aux[0] = tot[1];
            if (!(res == res) || isinf(res)) { c.status = 2; c.done = 1; }
            else if (res < c.tol_field) c.done = 1;
            else if (c.iters >= c.max_iter) { c.status = 1; c.done = 1; }
            break;
        }
        case POL_REFINE_INNER: {
            c.iters += 1;
            const double r = sqrt(tot[0]);
            c.residual = r;
            const double target = c.inner_tol * outer[b].rnorm;
            if (!(r == r)) { c.status = 2; c.done = 1; }
            else if (r < target) c.done = 1;
            else if (c.iters >= c.max_iter) c.done = 1;
            break;
        }
        default: break;
    }
}

}  // namespace m3d
