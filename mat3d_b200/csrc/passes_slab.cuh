// passes_slab.cuh -- the y-z slab pass: four of a sweep's five passes in one
// kernel, for operators that act on each component separately.
//
// The z forward, y forward, y inverse and z inverse passes of a sweep couple
// voxels only inside one x slab of one component: for a fixed (entry b,
// component c, x) the half spectrum block s[((b*C + c)*Nx + x)*Ny*Hzp ...] is
// Ny rows of Hzp modes, contiguous in global memory, and the real field and
// phase map of the slab are Ny*Nz contiguous values.  When the prologue
// (pol = P[ph] x) and the epilogue (x += A[ph] (x_c - x)) are diagonal in the
// components -- every thermal scheme (P = p I, A = a I,
// src/3dTherm/FFT_thermal3D.cpp:242-266) -- one CTA can keep the whole slab's
// half spectrum in shared memory and carry it from the x turnaround of sweep k
// to the x turnaround of sweep k+1:
//
//   MIX:  load slab -> y inverse (columns) -> z inverse (C2R, two rows packed
//         per complex line) -> EM update of x and the residual partials ->
//         polarization of the new x -> z forward (R2C, two rows per line) ->
//         y forward -> store slab            (+ fused finalize of the sweep)
//   FWD:  polarization of x -> z forward -> y forward -> store slab
//         (the first sweep of a solve)
//
// so a sweep is two launches (x turnaround + MIX) instead of five, and the
// spectrum crosses L2/HBM twice per sweep instead of six times.  The forward
// half of MIX is speculative: when the finalize stops the entry, the spectrum
// it wrote is simply never read.  The arithmetic per line is the one of the
// five-pass kernels (same warp-split line FFTs, twiddles and Hermitian
// conventions: the imaginary parts of the kz = 0 and kz = N/2 modes are
// dropped in the C2R, as FFTW's c2r does); only the pairing of real lines into
// complex lines differs (rows y, y+1 of one component instead of components
// c, c+1 of one line), so results agree to rounding.
//
// Shared memory: the slab S (Ny rows, row stride SP = Hzp padded so that the
// column FFT's 8-lane row groups hit distinct banks), a work area W used as
// the column FFTs' exchange rows and then as the z lines' tile rows, the line
// twiddles (Ny == Nz share one table) and the per-phase coefficients of the
// slab's component.  FP32 at N = 128: 69.6 + 37.9 KB, two CTAs per SM.
#pragma once
#include "passes_fast.cuh"

namespace m3d {

constexpr int kSlabThreads = 256;

template <typename T, int N>
struct SlabGeom {
    typedef typename Cx<T>::t C2;
    static constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl;
    static constexpr int CPW = 32 / TL;  // columns (y FFTs) or packed lines (z FFTs) per warp
    static constexpr int NW = kSlabThreads / 32;
    static constexpr int Hz = N / 2 + 1, Hzp = HzOf<N>::Hzp;
    static constexpr int BMOD = sizeof(T) == 4 ? 16 : 8;  // complex elements per bank cycle
    static constexpr int SP = Hzp + ((4 - Hzp % BMOD) + BMOD) % BMOD;  // slab row stride, = 4 mod BMOD
    static constexpr int XS = RowLen<T, N, true>::value, XSW = RowLen<T, N, true>::sw;    // column exchange rows
    static constexpr int ROW = RowLen<T, N, false>::value, RSW = RowLen<T, N, false>::sw;  // z tile rows
    static constexpr int LPC = NW * CPW;  // packed z lines per chunk
    static constexpr int NPL = N / 2;     // packed lines per slab (rows 2m, 2m+1)
    static constexpr int NG = (Hz + CPW - 1) / CPW;  // column groups (live columns kz < Hz)
    static constexpr size_t s_bytes = (size_t)N * SP * sizeof(C2);
    static constexpr size_t xch_bytes = (size_t)NW * CPW * XS * sizeof(C2);
    static constexpr size_t tile_bytes = (size_t)LPC * ROW * sizeof(C2);
    static constexpr size_t w_bytes = xch_bytes > tile_bytes ? xch_bytes : tile_bytes;
    static constexpr size_t smem() {
        return (size_t)N * sizeof(C2) + s_bytes + w_bytes + 64 * sizeof(double) + 3 * kMaxPhases * sizeof(T) + 16;
    }
    static_assert(SP % 2 == 0, "16-byte aligned slab rows");
    static_assert((Hzp * sizeof(C2)) % 16 == 0, "whole 16-byte copies per row");
};

// Per-component operators of the slab pass, addressed per batch entry like
// ProMat / EpiEM: tables P, A ([phase][C][C]) and Osum ([phase][C]) of the
// entry's RVE block; only the diagonal entries (c, c) are used.
template <typename T>
struct SlabOps {
    int C;
    const uint8_t* phase;
    T* x;                  // state (FP32 correction or FP32/FP64 field)
    const float* r;        // defect forcing of a correction solve, may be null
    const double* P;
    const double* A;
    const double* Os;
    int nph;
    int lc;                // batch entries per RVE (0: one RVE shared by all entries)
    long long mstride;     // doubles per RVE table block
};

__device__ __forceinline__ void ld4x(const float* p, float (&o)[4]) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void ld4x(const double* p, double (&o)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}

// Column FFTs of the slab (all live kz columns, in place, natural order in
// and out; SIGN < 0 forward, > 0 inverse).
template <typename T, int N, int SIGN>
__device__ __forceinline__ void slab_columns(typename Cx<T>::t* S, typename Cx<T>::t* W, const typename Cx<T>::t* tw) {
    typedef typename Cx<T>::t C2;
    typedef SlabGeom<T, N> G;
    constexpr int E = G::E, TL = G::TL, CPW = G::CPW;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % CPW, t = lane / CPW;
    C2* xl = W + (warp * CPW + col) * G::XS;
    const int sw = G::XSW ? (col & 1) : 0;
#pragma unroll 1
    for (int gi = warp; gi < G::NG; gi += G::NW) {
        const int kz = gi * CPW + col;
        const bool ok = kz < G::Hz;
        C2* base = S + (ok ? kz : 0);
        C2 v[E];
        if constexpr (SIGN < 0) {
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = ok ? base[(t + TL * j) * G::SP] : mk<C2>(0, 0);
            line_fwd<C2, E, TL>(v, t, xl, tw, sw);
            if (ok) {
#pragma unroll
                for (int r = 0; r < E; ++r) base[spec_mode<E, TL>(t, r) * G::SP] = v[r];
            }
        } else {
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = ok ? base[spec_mode<E, TL>(t, r) * G::SP] : mk<C2>(0, 0);
            line_inv<C2, E, TL>(v, t, xl, tw, sw);
            if (ok) {
#pragma unroll
                for (int j = 0; j < E; ++j) base[(t + TL * j) * G::SP] = v[j];
            }
        }
    }
}

template <typename T, int N, bool MIX, class Fin>
__global__ void __launch_bounds__(kSlabThreads, 2)
    k_slab(GridDims g, const typename Cx<T>::t* __restrict__ twz, typename Cx<T>::t* __restrict__ spec, SlabOps<T> ops,
           Ctl* ctl, double* partials, Fin fin) {
    typedef typename Cx<T>::t C2;
    typedef SlabGeom<T, N> G;
    constexpr int E = G::E, TL = G::TL, CPW = G::CPW, SP = G::SP, ROW = G::ROW;
    const int b = blockIdx.y;
    if (ctl[b].done) return;
    const int C = ops.C;
    const int c = blockIdx.x / g.Nx, x = blockIdx.x - c * g.Nx;
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* S = tw + N;
    C2* W = (C2*)((char*)S + G::s_bytes);
    double* red = (double*)((char*)W + G::w_bytes);
    T* cp = (T*)(red + 64);  // P diagonal of component c per phase slot
    T* ca = cp + kMaxPhases; // A diagonal
    T* co = ca + kMaxPhases; // Osum entry

    const long long entry = (long long)b * C + c;
    C2* gs = spec + (entry * g.Nx + x) * (long long)N * G::Hzp;
    const long long vox0 = (long long)x * N * N;
    T* xs = ops.x + entry * g.V + vox0;
    const float* rs = ops.r ? ops.r + entry * g.V + vox0 : nullptr;
    const uint8_t* ph = ops.phase + (ops.lc ? (long long)(b / ops.lc) * g.V : 0) + vox0;
    {
        const long long mo = ops.lc ? (long long)(b / ops.lc) * ops.mstride : 0;
        for (int i = threadIdx.x; i < ops.nph; i += blockDim.x) {
            cp[i] = (T)ops.P[mo + ((long long)i * C + c) * C + c];
            if (MIX) {
                ca[i] = (T)ops.A[mo + ((long long)i * C + c) * C + c];
                co[i] = (T)ops.Os[mo + (long long)i * C + c];
            }
        }
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twz[i];
    constexpr int CPR = (int)(G::Hzp * sizeof(C2) / 16);  // 16-byte copies per slab row
    if constexpr (MIX) {
        for (int i = threadIdx.x; i < N * CPR; i += kSlabThreads) {
            const int row = i / CPR, q = i - row * CPR;
            cp_async((char*)(S + row * SP) + q * 16, (const char*)(gs + (long long)row * G::Hzp) + q * 16, 16, 16);
        }
        cp_async_wait_all();
    }
    __syncthreads();
    if constexpr (MIX) {
        slab_columns<T, N, +1>(S, W, tw);
        __syncthreads();
    }

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = lane % TL, lw = lane / TL;
    const T invV = (T)(1.0 / (double)g.V);
    const double wt = (C == 6 && c >= 3) ? 2.0 : 1.0;
    double acc[2] = {0.0, 0.0};
#pragma unroll 1
    for (int m0 = 0; m0 < G::NPL; m0 += G::LPC) {
        const int li = warp * CPW + lw;  // this lane's packed line within the chunk
        const int m = m0 + li;
        const bool live = m < G::NPL;
        C2* row = W + li * ROW;
        const int sw = (li & 1) * G::RSW;
        if constexpr (MIX) {
            // z inverse: the line's spectrum (rows 2m + i 2m+1) assembled from the
            // two stored half spectra as the lanes load it (Hermitian extension)
            const C2* ra = S + (live ? 2 * m : 0) * SP;
            const C2* rb = ra + SP;
            C2 v[E];
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int k = spec_mode<E, TL>(t, r);
                const bool lo = 2 * k <= N;
                const int kk = lo ? k : N - k;
                const C2 a = live ? ra[kk] : mk<C2>(0, 0);
                const C2 q = live ? rb[kk] : mk<C2>(0, 0);
                if (kk == 0 || 2 * kk == N) v[r] = mk<C2>(a.x, q.x);
                else if (lo) v[r] = mk<C2>(a.x - q.y, a.y + q.x);
                else v[r] = mk<C2>(a.x + q.y, q.x - a.y);
            }
            line_inv<C2, E, TL>(v, t, row, tw, sw);
#pragma unroll
            for (int j = 0; j < E; ++j) row[(t + TL * j) ^ sw] = v[j];
        }
        __syncthreads();
        // pointwise: (MIX) EM update x += A (x_c + r - x) with the residual
        // partials, then the polarization P x of the (new) state into the tile
        {
            const int rows = min(2 * G::LPC, N - 2 * m0);
            const int nq = rows * N / 4;
#pragma unroll 1
            for (int i4 = threadIdx.x; i4 < nq; i4 += kSlabThreads) {
                const int i = i4 * 4;
                const int yl = i / N, z0 = i - yl * N;
                const long long vo = (long long)(2 * m0 + yl) * N + z0;
                const int lt = yl >> 1, odd = yl & 1;
                C2* tr = W + lt * ROW;
                const int tsw = (lt & 1) * G::RSW;
                T xv[4];
                ld4x(xs + vo, xv);
                const uchar4 p4 = *reinterpret_cast<const uchar4*>(ph + vo);
                const int pp[4] = {p4.x, p4.y, p4.z, p4.w};
                if constexpr (MIX) {
                    float rv[4] = {0.f, 0.f, 0.f, 0.f};
                    if (rs) ld4x(rs + vo, rv);
                    T xn[4];
#pragma unroll
                    for (int w = 0; w < 4; ++w) {
                        const C2 u = tr[(z0 + w) ^ tsw];
                        const T xc = (odd ? u.y : u.x) * invV;
                        const T d = (xc + (T)rv[w]) - xv[w];
                        acc[0] += wt * (double)d * (double)d;
                        xn[w] = xv[w] + ca[pp[w]] * d;
                        acc[1] += (double)co[pp[w]] * (double)xn[w];
                    }
                    if constexpr (sizeof(T) == 4) {
                        *reinterpret_cast<float4*>(xs + vo) = make_float4(xn[0], xn[1], xn[2], xn[3]);
                    } else {
                        reinterpret_cast<double2*>(xs + vo)[0] = make_double2(xn[0], xn[1]);
                        reinterpret_cast<double2*>(xs + vo)[1] = make_double2(xn[2], xn[3]);
                    }
#pragma unroll
                    for (int w = 0; w < 4; ++w) xv[w] = xn[w];
                }
#pragma unroll
                for (int w = 0; w < 4; ++w) reinterpret_cast<T*>(&tr[(z0 + w) ^ tsw])[odd] = cp[pp[w]] * xv[w];
            }
        }
        __syncthreads();
        // z forward of the packed lines; each row is split into the two rows'
        // half spectra (Z[k] and Z[N-k] sit in the same tile row) into S
        {
            C2 v[E];
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = row[(t + TL * j) ^ sw];
            __syncwarp();
            line_fwd<C2, E, TL>(v, t, row, tw, sw);
#pragma unroll
            for (int r = 0; r < E; ++r) row[spec_mode<E, TL>(t, r) ^ sw] = v[r];
            __syncwarp();
            if (live) {
                C2* oa = S + (2 * m) * SP;
                C2* ob = oa + SP;
#pragma unroll 1
                for (int k = t; k < G::Hzp; k += TL) {
                    C2 ea = mk<C2>(0, 0), eb = mk<C2>(0, 0);
                    if (k < G::Hz) {
                        const C2 Zk = row[k ^ sw];
                        const C2 Zm = row[(k == 0 ? 0 : N - k) ^ sw];
                        ea = mk<C2>((T)0.5 * (Zk.x + Zm.x), (T)0.5 * (Zk.y - Zm.y));
                        eb = mk<C2>((T)0.5 * (Zk.y + Zm.y), (T)-0.5 * (Zk.x - Zm.x));
                    }
                    oa[k] = ea;
                    ob[k] = eb;
                }
            }
        }
        __syncthreads();
    }
    slab_columns<T, N, -1>(S, W, tw);
    __syncthreads();
    for (int i = threadIdx.x; i < N * CPR; i += kSlabThreads) {
        const int row = i / CPR, q = i - row * CPR;
        *reinterpret_cast<float4*>((char*)(gs + (long long)row * G::Hzp) + q * 16) =
            *reinterpret_cast<const float4*>((const char*)(S + row * SP) + q * 16);
    }
    if constexpr (MIX) {
        block_reduce_store<2>(acc, red, partials, b, gridDim.x, blockIdx.x);
        fused_finalize(fin, ctl, partials, 2, b);
    }
}

}  // namespace m3d
