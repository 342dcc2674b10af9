// passes.cuh -- the five FFT passes of one Lippmann-Schwinger sweep, with the
// pointwise physics fused into the first and last pass.
//
// Device data layout (all buffers component-major, "SoA"):
//   real field   f[(b*C + c)*V + v],          v = z + Nz*(y + Ny*x)
//   phase map    phase[v]                     (uint8, shared by the batch)
//   half spectrum s[((b*C + c)*Nx*Ny + x*Ny + y)*Hzp + kz],  kz < Hz = Nz/2+1
// Hzp = Hz rounded up to even (16-byte aligned rows for FP32 complex).
// This is the reference's FFTW layout (src/3d/FFT_analysis3D.cpp:115-150:
// z fastest, R2C halving along z) with the component axis moved outermost.
//
// Sweep:  zfwd (prologue -> R2C along z) -> y fwd -> x turnaround
//         (x fwd, spectral op per mode, x inv) -> y inv -> zinv (C2R along z
//         -> epilogue).  Each kernel first reads ctl[b].done and returns when
//         that batch entry has converged, so a captured chain of sweeps costs
//         almost nothing once it is finished.
#pragma once
#include "fft_smem.cuh"

namespace m3d {

struct GridDims {
    int Nx, Ny, Nz, Hz, Hzp;
    long long V;   // Nx*Ny*Nz
    long long NL;  // Nx*Ny (z lines)
    // compacted launches: live[0] = number of entries still iterating,
    // live[1..] their ids in order; the launch's entry slots (blockIdx.y)
    // index this list.  Null: slot = entry.
    const int* live = nullptr;
};

// Batch entry of launch slot s; -1 for a slot past the live list.
__device__ __forceinline__ int entry_of(const GridDims& g, int s) {
    if (!g.live) return s;
    return s < g.live[0] ? g.live[1 + s] : -1;
}

// Per batch entry control block (device memory).
struct Ctl {
    int done;       // 1: skip all work for this entry
    int iters;      // sweeps performed
    int status;     // 0 ok, 1 iteration cap, 2 non-finite residual
    int max_iter;
    int crit_residual;    // 1: residual stop rule, 0: the reference's rule
    int gkind;            // Green operator of this entry's RVE (GreenKind)
    int gnyq;             // 1: index <= N/2 is a positive frequency
    int gxw;              // wrap length of the x index
    double gp1, gp2;      // Green operator constants (see SpecGreen)
    double kzero[6];      // value of the k = 0 mode after the spectral op (already times V)
    double residual;      // last residual (criterion dependent)
    double tol_field, tol_eq;
    double enorm;         // |E| for the residual normalisation
    double sum_prev;      // reference criterion: previous sum of the "other" field
    double den;           // reference criterion: V * (0.5 M0 + 0.5 M1) * sum(E)
    double eq_old, eqvar, diff_sum, diff_eq;
    double rnorm;         // refinement: |defect| of the outer FP64 pass
    double inner_tol;     // refinement: inner stop ratio
    double E[6];          // macroscopic load (mixed control updates it)
    double aux[32];       // policy scratch (means etc.)
};

constexpr int kMaxC = 6;

// ---- block reduction of NS doubles -> partials[(b*NS + s)*nblk + blk] -------
template <int NS>
__device__ __forceinline__ void block_reduce_store(double (&acc)[NS], double* red_smem, double* partials, int b,
                                                   int nblk, int blk) {
    if constexpr (NS == 0) {
        return;
    } else {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            double v = acc[s];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red_smem[s * 32 + warp] = v;
        }
        __syncthreads();
        if (threadIdx.x < NS) {
            double t = 0.0;
            for (int w = 0; w < nw; ++w) t += red_smem[threadIdx.x * 32 + w];
            partials[((long long)b * NS + threadIdx.x) * nblk + blk] = t;
        }
    }
}

// No fused finalize.
struct FinNone {
    int* counter = nullptr;
    __device__ __forceinline__ void run(Ctl*, const double*, int, int, int, double*, double*) const {}
};

// completion-counter increment with acquire-release semantics at GPU scope:
// the block's earlier writes (ordered before it by the preceding barrier) are
// released with it, and the last arriver acquires every other block's
__device__ __forceinline__ int atomic_add_acq_rel_gpu(int* p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;\n" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// The last block of a pass (per batch entry) to finish runs the finalize on
// all blocks' partials: barrier + one acquire-release completion counter
// (rather than a fence in every thread), the counter reset by that block for
// the next launch.  All threads of the block must call it.
template <class Fin>
__device__ __forceinline__ void fused_finalize(const Fin& fin, Ctl* ctl, const double* partials, int NS, int b) {
    if (fin.counter == nullptr) return;
    __shared__ int last;
    __shared__ double red[256];
    __shared__ double tot[16];
    __syncthreads();
    if (threadIdx.x == 0) last = (atomic_add_acq_rel_gpu(&fin.counter[b], 1) == (int)gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    fin.run(ctl, partials, NS, gridDim.x, b, red, tot);
    if (threadIdx.x == 0) fin.counter[b] = 0;
}

// ---- shared-memory carve-up helper -----------------------------------------
__device__ __forceinline__ char* align_up(char* p, int a) {
    return (char*)(((uintptr_t)p + (a - 1)) & ~(uintptr_t)(a - 1));
}

// ============================================================================
// z forward: prologue (per voxel: C input values) -> pairs of real lines packed
// as one complex line -> FFT along z -> split into two half spectra.
// ============================================================================
template <typename T, int C, class Pro>
__global__ void __launch_bounds__(256) k_zfwd(GridDims g, LinePlan pz, const typename Cx<T>::t* __restrict__ twz,
                                              typename Cx<T>::t* __restrict__ spec, Pro pro, const Ctl* __restrict__ ctl,
                                              int G, double* partials) {
    typedef typename Cx<T>::t C2;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
    extern __shared__ __align__(16) char smem_raw[];
    const int Nz = g.Nz;
    const int npairs = G / 2;
    const int nl = npairs * C;
    C2* tw = (C2*)smem_raw;
    C2* A = tw + Nz;
    C2* B = A + (size_t)nl * Nz;
    char* extra = align_up((char*)(B + (size_t)nl * Nz), 16);
    double* red = (double*)extra;
    extra += 32 * 32 * sizeof(double);
    for (int i = threadIdx.x; i < Nz; i += blockDim.x) tw[i] = twz[i];
    pro.bind(b);
    pro.load_smem(extra, b);
    __syncthreads();

    const long long l0 = (long long)blockIdx.x * G;
    double acc[Pro::NSUM > 0 ? Pro::NSUM : 1] = {};
    for (int i = threadIdx.x; i < G * Nz; i += blockDim.x) {
        const int gi = i / Nz, z = i - gi * Nz;
        const long long l = l0 + gi;
        T val[C];
        if (l < g.NL) {
            pro.eval(b, l * Nz + z, val, acc);
        } else {
#pragma unroll
            for (int c = 0; c < C; ++c) val[c] = (T)0;
        }
        const int p = gi >> 1;
        T* dstf = (T*)A;
#pragma unroll
        for (int c = 0; c < C; ++c) dstf[2 * ((size_t)(p * C + c) * Nz + z) + (gi & 1)] = val[c];
    }
    __syncthreads();
    LineLayout L{nl, 1, 0, Nz, 1, false};
    C2* R = fft_lines<C2>(A, B, tw, pz, L, -1);

    const int Hz = g.Hz, Hzp = g.Hzp;
    for (int i = threadIdx.x; i < nl * Hzp; i += blockDim.x) {
        const int k = i % Hzp, pc = i / Hzp;
        const int p = pc / C, c = pc - p * C;
        const long long la = l0 + 2 * p, lb = la + 1;
        C2 Av = mk<C2>(0, 0), Bv = mk<C2>(0, 0);
        if (k < Hz) {
            const C2 Z = R[(size_t)pc * Nz + k];
            const C2 Zm = R[(size_t)pc * Nz + (k == 0 ? 0 : Nz - k)];
            Av = mk<C2>((T)0.5 * (Z.x + Zm.x), (T)0.5 * (Z.y - Zm.y));
            Bv = mk<C2>((T)0.5 * (Z.y + Zm.y), (T)-0.5 * (Z.x - Zm.x));
        }
        const long long rowbase = ((long long)b * C + c) * g.NL;
        if (la < g.NL) spec[(rowbase + la) * Hzp + k] = Av;
        if (lb < g.NL) spec[(rowbase + lb) * Hzp + k] = Bv;
    }
    if constexpr (Pro::NSUM > 0) {
        block_reduce_store<Pro::NSUM>(acc, red, partials, b, gridDim.x, blockIdx.x);
    }
}

// ============================================================================
// y pass (forward sign -1 or inverse +1), in place on the half spectrum.
// CTA = one x, TZ consecutive kz columns, one (batch, component).
// ============================================================================
template <typename T>
__global__ void __launch_bounds__(256) k_ypass(GridDims g, LinePlan py, const typename Cx<T>::t* __restrict__ twy,
                                               typename Cx<T>::t* __restrict__ spec, int TZ, int C, int sign,
                                               const Ctl* __restrict__ ctl) {
    typedef typename Cx<T>::t C2;
    const int b = entry_of(g, blockIdx.y / C);
    if (b < 0 || ctl[b].done) return;
    const int cb = b * C + blockIdx.y % C;
    extern __shared__ __align__(16) char smem_raw[];
    const int Ny = g.Ny, Hzp = g.Hzp;
    C2* tw = (C2*)smem_raw;
    C2* A = tw + Ny;
    C2* B = A + (size_t)Ny * TZ;
    for (int i = threadIdx.x; i < Ny; i += blockDim.x) tw[i] = twy[i];
    const int ntz = (Hzp + TZ - 1) / TZ;
    const int x = blockIdx.x / ntz, kz0 = (blockIdx.x - x * ntz) * TZ;
    C2* base = spec + ((long long)cb * g.NL + (long long)x * Ny) * Hzp + kz0;
    for (int i = threadIdx.x; i < Ny * TZ; i += blockDim.x) {
        const int y = i / TZ, col = i - y * TZ;
        A[i] = (kz0 + col < Hzp) ? base[(long long)y * Hzp + col] : mk<C2>(0, 0);
    }
    __syncthreads();
    LineLayout L{TZ, TZ, 1, 0, TZ, true};
    C2* R = fft_lines<C2>(A, B, tw, py, L, sign);
    for (int i = threadIdx.x; i < Ny * TZ; i += blockDim.x) {
        const int y = i / TZ, col = i - y * TZ;
        if (kz0 + col < Hzp) base[(long long)y * Hzp + col] = R[i];
    }
}

// ============================================================================
// x turnaround: for one y and TZ kz columns, all C components:
//   forward FFT along x -> spectral op per mode (Green operator, k=0 value,
//   optional reductions) -> inverse FFT along x (when Spec::kInverse).
// ============================================================================
template <typename T, int C, class Spec>
__global__ void __launch_bounds__(256) k_xturn(GridDims g, LinePlan px, const typename Cx<T>::t* __restrict__ twx,
                                               typename Cx<T>::t* __restrict__ spec, int TZ, Spec op,
                                               const Ctl* __restrict__ ctl, double* partials) {
    typedef typename Cx<T>::t C2;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
    op.prepare(ctl, b);
    extern __shared__ __align__(16) char smem_raw[];
    const int Nx = g.Nx, Ny = g.Ny, Hzp = g.Hzp;
    C2* tw = (C2*)smem_raw;
    C2* A = tw + Nx;
    C2* B = A + (size_t)C * Nx * TZ;
    double* red = (double*)align_up((char*)(B + (size_t)C * Nx * TZ), 16);
    for (int i = threadIdx.x; i < Nx; i += blockDim.x) tw[i] = twx[i];
    const int ntz = (Hzp + TZ - 1) / TZ;
    const int y = blockIdx.x / ntz, kz0 = (blockIdx.x - y * ntz) * TZ;
    for (int i = threadIdx.x; i < C * Nx * TZ; i += blockDim.x) {
        const int col = i % TZ, r = i / TZ;
        const int x = r % Nx, c = r / Nx;
        A[i] = (kz0 + col < Hzp)
                   ? spec[(((long long)b * C + c) * g.NL + (long long)x * Ny + y) * Hzp + kz0 + col]
                   : mk<C2>(0, 0);
    }
    __syncthreads();
    LineLayout L{C * TZ, TZ, 1, Nx * TZ, TZ, true};
    C2* R = fft_lines<C2>(A, B, tw, px, L, -1);
    C2* S = (R == A) ? B : A;

    double acc[Spec::NSUM > 0 ? Spec::NSUM : 1] = {};
    for (int i = threadIdx.x; i < Nx * TZ; i += blockDim.x) {
        const int col = i % TZ, x = i / TZ;
        const int kz = kz0 + col;
        if (kz >= g.Hz) continue;
        C2 v[C];
#pragma unroll
        for (int c = 0; c < C; ++c) v[c] = R[(size_t)(c * Nx + x) * TZ + col];
        op.apply(b, x, y, kz, v, acc, ctl);
        if constexpr (Spec::kInverse) {
#pragma unroll
            for (int c = 0; c < C; ++c) R[(size_t)(c * Nx + x) * TZ + col] = v[c];
        }
    }
    if constexpr (Spec::NSUM > 0) {
        block_reduce_store<Spec::NSUM>(acc, red, partials, b, gridDim.x, blockIdx.x);
    }
    if constexpr (Spec::kInverse) {
        __syncthreads();
        C2* Q = fft_lines<C2>(R, S, tw, px, L, +1);
        for (int i = threadIdx.x; i < C * Nx * TZ; i += blockDim.x) {
            const int col = i % TZ, r = i / TZ;
            const int x = r % Nx, c = r / Nx;
            if (kz0 + col < Hzp)
                spec[(((long long)b * C + c) * g.NL + (long long)x * Ny + y) * Hzp + kz0 + col] = Q[i];
        }
    }
}

// ============================================================================
// z inverse: two half spectra -> one complex line (Hermitian extension, DC and
// Nyquist imaginary parts dropped, which is FFTW's c2r rule) -> inverse FFT ->
// real parts / imaginary parts are the two real lines -> epilogue per voxel.
// ============================================================================
template <typename T, int C, class Epi, class Fin>
__global__ void __launch_bounds__(256) k_zinv(GridDims g, LinePlan pz, const typename Cx<T>::t* __restrict__ twz,
                                              const typename Cx<T>::t* __restrict__ spec, Epi epi, Ctl* ctl, int G,
                                              double* partials, Fin fin) {
    typedef typename Cx<T>::t C2;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
    extern __shared__ __align__(16) char smem_raw[];
    const int Nz = g.Nz, Hz = g.Hz, Hzp = g.Hzp;
    const int npairs = G / 2;
    const int nl = npairs * C;
    C2* tw = (C2*)smem_raw;
    C2* A = tw + Nz;
    C2* B = A + (size_t)nl * Nz;
    char* extra = align_up((char*)(B + (size_t)nl * Nz), 16);
    double* red = (double*)extra;
    extra += 32 * 32 * sizeof(double);
    for (int i = threadIdx.x; i < Nz; i += blockDim.x) tw[i] = twz[i];
    epi.bind(b);
    epi.load_smem(extra, b);
    const long long l0 = (long long)blockIdx.x * G;
    for (int i = threadIdx.x; i < nl * Hz; i += blockDim.x) {
        const int k = i % Hz, pc = i / Hz;
        const int p = pc / C, c = pc - p * C;
        const long long la = l0 + 2 * p, lb = la + 1;
        const long long rowbase = ((long long)b * C + c) * g.NL;
        C2 a = (la < g.NL) ? spec[(rowbase + la) * Hzp + k] : mk<C2>(0, 0);
        C2 bb = (lb < g.NL) ? spec[(rowbase + lb) * Hzp + k] : mk<C2>(0, 0);
        C2* line = A + (size_t)pc * Nz;
        const bool self = (k == 0) || (2 * k == Nz);
        if (self) {
            line[k] = mk<C2>(a.x, bb.x);
        } else {
            line[k] = mk<C2>(a.x - bb.y, a.y + bb.x);
            line[Nz - k] = mk<C2>(a.x + bb.y, bb.x - a.y);
        }
    }
    __syncthreads();
    LineLayout L{nl, 1, 0, Nz, 1, false};
    C2* R = fft_lines<C2>(A, B, tw, pz, L, +1);

    const T invV = (T)(1.0 / (double)g.V);
    double acc[Epi::NSUM > 0 ? Epi::NSUM : 1] = {};
    for (int i = threadIdx.x; i < G * Nz; i += blockDim.x) {
        const int gi = i / Nz, z = i - gi * Nz;
        const long long l = l0 + gi;
        if (l >= g.NL) continue;
        const int p = gi >> 1;
        const T* srcf = (const T*)R;
        T xc[C];
#pragma unroll
        for (int c = 0; c < C; ++c) xc[c] = srcf[2 * ((size_t)(p * C + c) * Nz + z) + (gi & 1)] * invV;
        epi.apply(b, l * Nz + z, xc, acc);
    }
    if constexpr (Epi::NSUM > 0) {
        block_reduce_store<Epi::NSUM>(acc, red, partials, b, gridDim.x, blockIdx.x);
        fused_finalize(fin, ctl, partials, Epi::NSUM, b);
    }
}

}  // namespace m3d
