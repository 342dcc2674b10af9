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

// NT threads per CTA: 256 (8 warps, two CTAs per SM) or 512 (16 warps, one
// CTA per SM: the FP32 128^2 slab with all its z lines in one chunk)
template <typename T, int N, int NT_ = 256>
struct SlabGeom {
    typedef typename Cx<T>::t C2;
    static constexpr int NT = NT_;
    static constexpr int MINB = NT == 512 ? 1 : 2;
    static constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl;
    static constexpr int CPW = 32 / TL;  // columns (y FFTs) or packed lines (z FFTs) per warp
    static constexpr int NW = NT / 32;
    static constexpr int Hz = N / 2 + 1, Hzp = HzOf<N>::Hzp;
    static constexpr int BMOD = sizeof(T) == 4 ? 16 : 8;  // complex elements per bank cycle
    static constexpr int SP = Hzp + ((4 - Hzp % BMOD) + BMOD) % BMOD;  // slab row stride, = 4 mod BMOD
    static constexpr int XS = RowLen<T, N, true>::value, XSW = RowLen<T, N, true>::sw;    // column exchange rows
    static constexpr int ROW = RowLen<T, N, false>::value, RSW = RowLen<T, N, false>::sw;  // z tile rows
    static constexpr int LPC = NW * CPW;  // packed z lines per chunk
    static constexpr int NPL = N / 2;     // packed lines per slab (rows 2m, 2m+1)
    // column groups: kz = 0 .. N/2-1, column 0 carrying the DC (kz = 0) and
    // Nyquist (kz = N/2) columns packed into one complex FFT
    static constexpr int NG = (N / 2) / CPW;
    static_assert((N / 2) % CPW == 0, "whole column groups");
    static constexpr size_t s_bytes = (size_t)N * SP * sizeof(C2);
    static constexpr size_t xch_bytes = (size_t)NW * CPW * XS * sizeof(C2);
    static constexpr size_t tile_bytes = (size_t)LPC * ROW * sizeof(C2);
    static constexpr size_t w_bytes = xch_bytes > tile_bytes ? xch_bytes : tile_bytes;
    static constexpr size_t smem() {
        return (size_t)N * sizeof(C2) + s_bytes + w_bytes + 64 * sizeof(double) + 3 * kMaxPhases * sizeof(T) + 16;
    }
    // fits the CTAs per SM it is launched for (227 KB per SM, static shared
    // memory of the finalize included)
    static constexpr bool fits() { return smem() <= (MINB == 1 ? (size_t)220 * 1024 : (size_t)110 * 1024); }
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

// One pointwise item of a chunk: voxels z0, z0+1 of rows 2m and 2m+1, i.e.
// one 16-byte (FP32) pair of complex tile entries of packed line m.  A warp's
// items are consecutive pairs of one line, so its tile accesses are
// contiguous (conflict-free) and its global loads are 256-byte runs.
template <typename T>
struct SlabItem {
    T x[4];       // row 2m: z0, z0+1; row 2m+1: z0, z0+1
    float r[4];
    uint32_t p;   // the four phase ids, one byte each
};
__device__ __forceinline__ void ld2(const float* p, float& a, float& b) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    a = v.x; b = v.y;
}
__device__ __forceinline__ void ld2(const double* p, double& a, double& b) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    a = v.x; b = v.y;
}
__device__ __forceinline__ void st2(float* p, float a, float b) { *reinterpret_cast<float2*>(p) = make_float2(a, b); }
__device__ __forceinline__ void st2(double* p, double a, double b) {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
}
// tile pair at z0 (even) of a tile row, its two logical entries (z0, z0+1)
// in order whatever the row's swizzle (XOR 1)
__device__ __forceinline__ void tile_get2(const float2* tr, int z0, int sw, float2& a, float2& b) {
    const float4 v = *reinterpret_cast<const float4*>(tr + z0);
    a = make_float2(sw ? v.z : v.x, sw ? v.w : v.y);
    b = make_float2(sw ? v.x : v.z, sw ? v.y : v.w);
}
__device__ __forceinline__ void tile_put2(float2* tr, int z0, int sw, float2 a, float2 b) {
    *reinterpret_cast<float4*>(tr + z0) = sw ? make_float4(b.x, b.y, a.x, a.y) : make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void tile_get2(const double2* tr, int z0, int sw, double2& a, double2& b) {
    a = tr[z0 ^ sw];
    b = tr[(z0 + 1) ^ sw];
}
__device__ __forceinline__ void tile_put2(double2* tr, int z0, int sw, double2 a, double2 b) {
    tr[z0 ^ sw] = a;
    tr[(z0 + 1) ^ sw] = b;
}

// Column FFTs of the slab (in place, natural order in and out; SIGN < 0
// forward, > 0 inverse) over kz = 0 .. N/2, the DC and Nyquist columns
// sharing one complex FFT (column 0):
//   forward: both columns are real after the z R2C (their imaginary parts are
//     exact zeros), so P = S0 + i S_N/2 is transformed and split by Hermitian
//     symmetry, F0[k] = (F[k] + conj F[-k]) / 2, F_N/2[k] = (F[k] - conj F[-k]) / 2i;
//   inverse: the z C2R keeps only the real parts of these two columns (FFTW's
//     c2r semantics), and Re IFFT(S) = IFFT((S[k] + conj S[-k]) / 2), so the
//     Hermitian parts H0 + i H_N/2 are transformed together and the real and
//     imaginary parts of the result are the two columns' real parts.
// The pre- and post-steps are done by the warp that owns column group 0.
template <typename T, int N, int NT, int SIGN>
__device__ __forceinline__ void slab_columns(typename Cx<T>::t* S, typename Cx<T>::t* W, const typename Cx<T>::t* tw) {
    typedef typename Cx<T>::t C2;
    typedef SlabGeom<T, N, NT> G;
    constexpr int E = G::E, TL = G::TL, CPW = G::CPW, SP = G::SP, H = N / 2;
    constexpr int KPL = (N + 31) / 32;  // column entries per lane in the pack / split steps
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % CPW, t = lane / CPW;
    C2* xl = W + (warp * CPW + col) * G::XS;
    const int sw = G::XSW ? (col & 1) : 0;
#pragma unroll 1
    for (int gi = warp; gi < G::NG; gi += G::NW) {
        if (gi == 0) {  // pack the DC and Nyquist columns into column 0
            if constexpr (SIGN < 0) {
#pragma unroll
                for (int q = 0; q < KPL; ++q) {
                    const int y = lane + 32 * q;
                    if (y < N) S[y * SP] = mk<C2>(S[y * SP].x, S[y * SP + H].x);
                }
            } else {
                C2 pk[KPL];
#pragma unroll
                for (int q = 0; q < KPL; ++q) {
                    const int k = min(lane + 32 * q, N - 1), km = (N - k) % N;
                    const C2 a = S[k * SP], a2 = S[km * SP], b = S[k * SP + H], b2 = S[km * SP + H];
                    const C2 h0 = mk<C2>((T)0.5 * (a.x + a2.x), (T)0.5 * (a.y - a2.y));
                    const C2 hn = mk<C2>((T)0.5 * (b.x + b2.x), (T)0.5 * (b.y - b2.y));
                    pk[q] = mk<C2>(h0.x - hn.y, h0.y + hn.x);
                }
                __syncwarp();
#pragma unroll
                for (int q = 0; q < KPL; ++q)
                    if (lane + 32 * q < N) S[(lane + 32 * q) * SP] = pk[q];
            }
            __syncwarp();
        }
        C2* base = S + gi * CPW + col;
        C2 v[E];
        if constexpr (SIGN < 0) {
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = base[(t + TL * j) * SP];
            line_fwd<C2, E, TL>(v, t, xl, tw, sw);
#pragma unroll
            for (int r = 0; r < E; ++r) base[spec_mode<E, TL>(t, r) * SP] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = base[spec_mode<E, TL>(t, r) * SP];
            line_inv<C2, E, TL>(v, t, xl, tw, sw);
#pragma unroll
            for (int j = 0; j < E; ++j) base[(t + TL * j) * SP] = v[j];
        }
        if (gi == 0) {  // unpack column 0 into the DC and Nyquist columns
            __syncwarp();
            if constexpr (SIGN < 0) {
                C2 f0[KPL], fn[KPL];
#pragma unroll
                for (int q = 0; q < KPL; ++q) {
                    const int k = min(lane + 32 * q, N - 1), km = (N - k) % N;
                    const C2 F = S[k * SP], Fm = S[km * SP];
                    f0[q] = mk<C2>((T)0.5 * (F.x + Fm.x), (T)0.5 * (F.y - Fm.y));
                    fn[q] = mk<C2>((T)0.5 * (F.y + Fm.y), (T)-0.5 * (F.x - Fm.x));
                }
                __syncwarp();
#pragma unroll
                for (int q = 0; q < KPL; ++q) {
                    const int k = lane + 32 * q;
                    if (k < N) {
                        S[k * SP] = f0[q];
                        S[k * SP + H] = fn[q];
                    }
                }
            } else {
#pragma unroll
                for (int q = 0; q < KPL; ++q) {
                    const int y = lane + 32 * q;
                    if (y < N) {
                        const C2 pv = S[y * SP];
                        S[y * SP] = mk<C2>(pv.x, (T)0);
                        S[y * SP + H] = mk<C2>(pv.y, (T)0);
                    }
                }
            }
            __syncwarp();
        }
    }
}

template <typename T, int N, int NT, bool MIX, class Fin>
__global__ void __launch_bounds__(NT, SlabGeom<T, N, NT>::MINB)
    k_slab(GridDims g, const typename Cx<T>::t* __restrict__ twz, typename Cx<T>::t* __restrict__ spec, SlabOps<T> ops,
           Ctl* ctl, double* partials, Fin fin) {
    typedef typename Cx<T>::t C2;
    typedef SlabGeom<T, N, NT> G;
    constexpr int E = G::E, TL = G::TL, CPW = G::CPW, SP = G::SP, ROW = G::ROW;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
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
        for (int i = threadIdx.x; i < N * CPR; i += G::NT) {
            const int row = i / CPR, q = i - row * CPR;
            cp_async((char*)(S + row * SP) + q * 16, (const char*)(gs + (long long)row * G::Hzp) + q * 16, 16, 16);
        }
        cp_async_wait_all();
    }
    __syncthreads();
    if constexpr (MIX) {
        slab_columns<T, N, NT, +1>(S, W, tw);
        __syncthreads();
    }

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = lane % TL, lw = lane / TL;
    const T invV = (T)(1.0 / (double)g.V);
    const double wt = (C == 6 && c >= 3) ? 2.0 : 1.0;
    // per-thread partial sums in the field's type (a thread sums a few dozen
    // voxels), widened to FP64 once for the block reduction
    T racc = 0, oacc = 0;
    // pointwise items of a chunk per thread; the first PRE are loaded before
    // the chunk's z inverse (their latency hidden by it), the rest after it
    constexpr int HP = N / 2;  // z pairs per line
    constexpr int IPT = (G::LPC * HP + G::NT - 1) / G::NT;
    constexpr int PRE = MIX ? ((sizeof(T) == 4 && E < 16) ? IPT / 2 : IPT / 4) : 0;
    auto load_item = [&](int it, int m0, SlabItem<T>& q) {
        const int i = threadIdx.x + it * G::NT;
        const int li = i / HP, z0 = 2 * (i - li * HP);
        if (li >= G::LPC || m0 + li >= G::NPL) return;
        const long long vo = (long long)(2 * (m0 + li)) * N + z0;
        ld2(xs + vo, q.x[0], q.x[1]);
        ld2(xs + vo + N, q.x[2], q.x[3]);
        const uint32_t pa = *reinterpret_cast<const uint16_t*>(ph + vo);
        const uint32_t pb = *reinterpret_cast<const uint16_t*>(ph + vo + N);
        q.p = pa | (pb << 16);
        if (MIX) {
            if (rs) {
                ld2(rs + vo, q.r[0], q.r[1]);
                ld2(rs + vo + N, q.r[2], q.r[3]);
            } else {
                q.r[0] = q.r[1] = q.r[2] = q.r[3] = 0.f;
            }
        }
    };
    // (MIX) EM update x += A (x_c + r - x) with the residual partials; then
    // the polarization P x of the (new) state, written into the tile
    auto point_item = [&](int it, int m0, const SlabItem<T>& q) {
        const int i = threadIdx.x + it * G::NT;
        const int li = i / HP, z0 = 2 * (i - li * HP);
        if (li >= G::LPC || m0 + li >= G::NPL) return;
        C2* tr = W + li * ROW;
        const int tsw = (li & 1) * G::RSW;
        T v[4];
#pragma unroll
        for (int w = 0; w < 4; ++w) v[w] = q.x[w];
        if constexpr (MIX) {
            C2 a, bq;
            tile_get2(tr, z0, tsw, a, bq);
            const T xc[4] = {a.x, bq.x, a.y, bq.y};
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const int pw = (q.p >> (8 * w)) & 0xff;
                const T d = (xc[w] * invV + (T)q.r[w]) - q.x[w];
                racc += d * d;
                v[w] = q.x[w] + ca[pw] * d;
                oacc += co[pw] * v[w];
            }
            const long long vo = (long long)(2 * (m0 + li)) * N + z0;
            st2(xs + vo, v[0], v[1]);
            st2(xs + vo + N, v[2], v[3]);
        }
        T pol[4];
#pragma unroll
        for (int w = 0; w < 4; ++w) pol[w] = cp[(q.p >> (8 * w)) & 0xff] * v[w];
        tile_put2(tr, z0, tsw, mk<C2>(pol[0], pol[2]), mk<C2>(pol[1], pol[3]));
    };
#pragma unroll 1
    for (int m0 = 0; m0 < G::NPL; m0 += G::LPC) {
        const int li = warp * CPW + lw;  // this lane's packed line within the chunk
        const int m = m0 + li;
        const bool live = m < G::NPL;
        C2* row = W + li * ROW;
        const int sw = (li & 1) * G::RSW;
        SlabItem<T> pre[PRE > 0 ? PRE : 1];
        if constexpr (MIX) {
#pragma unroll
            for (int it = 0; it < PRE; ++it) load_item(it, m0, pre[it]);
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
        {
            SlabItem<T> rest[IPT - PRE > 0 ? IPT - PRE : 1];
#pragma unroll
            for (int it = PRE; it < IPT; ++it) load_item(it, m0, rest[it - PRE]);
#pragma unroll
            for (int it = 0; it < PRE; ++it) point_item(it, m0, pre[it]);
#pragma unroll
            for (int it = PRE; it < IPT; ++it) point_item(it, m0, rest[it - PRE]);
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
    slab_columns<T, N, NT, -1>(S, W, tw);
    __syncthreads();
    for (int i = threadIdx.x; i < N * CPR; i += G::NT) {
        const int row = i / CPR, q = i - row * CPR;
        *reinterpret_cast<float4*>((char*)(gs + (long long)row * G::Hzp) + q * 16) =
            *reinterpret_cast<const float4*>((const char*)(S + row * SP) + q * 16);
    }
    if constexpr (MIX) {
        double acc[2] = {wt * (double)racc, (double)oacc};
        block_reduce_store<2>(acc, red, partials, b, gridDim.x, blockIdx.x);
        fused_finalize(fin, ctl, partials, 2, b);
    }
}

}  // namespace m3d
