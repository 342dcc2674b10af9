// passes_fast.cuh -- the five sweep passes for compile-time line lengths
// (16, 32, 48, 64, 96, 128, 256), built on the warp-split line FFT of
// fft_reg.cuh.  Same data layout, operators and reductions as the generic
// kernels in passes.cuh, which remain the path for any other length.
//
// Column passes (y, x): lane = col + CPW*t with CPW = 32/T columns per warp,
// so one load instruction touches CPW consecutive complex words of T rows
// (whole 32-byte sectors); data goes from global memory straight into
// registers, one warp-local exchange per transform, and back.
// z passes: a tile of G voxel lines is staged in shared memory (the
// prologue/epilogue need all components of a voxel); components are packed
// two per complex line (c0 + i c1, ...), transformed by warps in registers and
// split into half spectra.
#pragma once
#include "fft_reg.cuh"
#include "passes.cuh"

namespace m3d {

constexpr int kFastThreads = 128;

// ---------------------------------------------------------------------------
// y pass: CTA = 4 warps = 4*CPW consecutive kz columns of one (batch*comp, x)
// ---------------------------------------------------------------------------
template <typename T, int N, int SIGN>
__global__ void __launch_bounds__(kFastThreads) k_ypass_fast(GridDims g, const typename Cx<T>::t* __restrict__ twy,
                                                            typename Cx<T>::t* __restrict__ spec, int C,
                                                            const Ctl* __restrict__ ctl) {
    typedef typename Cx<T>::t C2;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    constexpr int XS = Xch<E, TL>::size;
    const int cb = blockIdx.y;
    if (ctl[cb / C].done) return;
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* xch = tw + N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twy[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % CPW, t = lane / CPW;
    const int ncol_cta = 4 * CPW;
    const int ntz = (g.Hzp + ncol_cta - 1) / ncol_cta;
    const int x = blockIdx.x / ntz;
    const int kz = (blockIdx.x - x * ntz) * ncol_cta + warp * CPW + col;
    const bool ok = kz < g.Hzp;
    C2* base = spec + ((long long)cb * g.NL + (long long)x * g.Ny) * g.Hzp + (ok ? kz : 0);
    C2* xl = xch + (warp * CPW + col) * XS;
    C2 v[E];
    if constexpr (SIGN < 0) {
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = ok ? base[(long long)(t + TL * j) * g.Hzp] : mk<C2>(0, 0);
        line_fwd<C2, E, TL>(v, t, xl, tw);
        if (ok) {
#pragma unroll
            for (int r = 0; r < E; ++r) base[(long long)spec_mode<E, TL>(t, r) * g.Hzp] = v[r];
        }
    } else {
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = ok ? base[(long long)spec_mode<E, TL>(t, r) * g.Hzp] : mk<C2>(0, 0);
        line_inv<C2, E, TL>(v, t, xl, tw);
        if (ok) {
#pragma unroll
            for (int j = 0; j < E; ++j) base[(long long)(t + TL * j) * g.Hzp] = v[j];
        }
    }
}

// ---------------------------------------------------------------------------
// x turnaround: CTA = 4 warps = 4*CPW kz columns of one (batch, y); each lane
// transforms all C components of its column, staging the spectra in shared
// memory so the spectral op sees all components of a mode.
// ---------------------------------------------------------------------------
template <typename T, int N>
constexpr size_t ypass_fast_smem() {
    typedef typename Cx<T>::t C2;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    return (size_t)N * sizeof(C2) + (size_t)4 * CPW * Xch<E, TL>::size * sizeof(C2);
}

// warps per CTA of the x turnaround: as many as keep the staging <= 64 KB
template <typename T, int N, int C>
struct XWarps {
    static constexpr size_t per_warp = (size_t)C * N * (32 / LineSplit<T, N>::Tl) * sizeof(typename Cx<T>::t);
    static constexpr int value = (4 * per_warp <= 64 * 1024) ? 4 : ((2 * per_warp <= 64 * 1024) ? 2 : 1);
};

template <typename T, int N, int C, class Spec>
__global__ void __launch_bounds__(kFastThreads) k_xturn_fast(GridDims g, const typename Cx<T>::t* __restrict__ twx,
                                                            typename Cx<T>::t* __restrict__ spec, Spec op,
                                                            const Ctl* __restrict__ ctl, double* partials) {
    typedef typename Cx<T>::t C2;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    constexpr int XS = Xch<E, TL>::size;
    constexpr int WPC = XWarps<T, N, C>::value;
    const int b = blockIdx.y;
    if (ctl[b].done) return;
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* xch = tw + N;
    C2* stage = xch + WPC * CPW * XS;                    // [warp][c][r][lane]
    double* red = (double*)align_up((char*)(stage + WPC * C * E * 32), 16);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twx[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % CPW, t = lane / CPW;
    const int ncol_cta = WPC * CPW;
    const int ntz = (g.Hzp + ncol_cta - 1) / ncol_cta;
    const int y = blockIdx.x / ntz;
    const int kz = (blockIdx.x - y * ntz) * ncol_cta + warp * CPW + col;
    const bool ok = kz < g.Hzp;
    const long long cstride = g.NL * g.Hzp;  // component stride
    C2* base = spec + ((long long)b * C * g.NL + y) * g.Hzp + (ok ? kz : 0);
    const long long xstride = (long long)g.Ny * g.Hzp;
    C2* xl = xch + (warp * CPW + col) * XS;
    C2* st = stage + warp * C * E * 32;
#pragma unroll 1
    for (int c = 0; c < C; ++c) {
        C2 v[E];
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = ok ? base[c * cstride + (t + TL * j) * xstride] : mk<C2>(0, 0);
        line_fwd<C2, E, TL>(v, t, xl, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) st[(c * E + r) * 32 + lane] = v[r];
    }
    double acc[Spec::NSUM > 0 ? Spec::NSUM : 1] = {};
    const bool live = ok && kz < g.Hz;
#pragma unroll 1
    for (int r = 0; r < E; ++r) {
        C2 m[C];
#pragma unroll
        for (int c = 0; c < C; ++c) m[c] = st[(c * E + r) * 32 + lane];
        if (live) op.apply(b, spec_mode<E, TL>(t, r), y, kz, m, acc, ctl);
        if constexpr (Spec::kInverse) {
#pragma unroll
            for (int c = 0; c < C; ++c) st[(c * E + r) * 32 + lane] = m[c];
        }
    }
    if constexpr (Spec::NSUM > 0) {
        block_reduce_store<Spec::NSUM>(acc, red, partials, b, gridDim.x, blockIdx.x);
    }
    if constexpr (Spec::kInverse) {
#pragma unroll 1
        for (int c = 0; c < C; ++c) {
            C2 v[E];
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = st[(c * E + r) * 32 + lane];
            line_inv<C2, E, TL>(v, t, xl, tw);
            if (ok) {
#pragma unroll
                for (int j = 0; j < E; ++j) base[c * cstride + (t + TL * j) * xstride] = v[j];
            }
        }
    }
}

template <typename T, int N, int C>
constexpr size_t xturn_fast_smem() {
    typedef typename Cx<T>::t C2;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    constexpr int WPC = XWarps<T, N, C>::value;
    return (size_t)N * sizeof(C2) + (size_t)WPC * CPW * Xch<E, TL>::size * sizeof(C2) +
           (size_t)WPC * C * E * 32 * sizeof(C2) + 16 + 32 * 32 * sizeof(double);
}

// ---------------------------------------------------------------------------
// z passes.  Tile of G voxel lines x NCL complex lines (NCL = ceil(C/2)).
// ---------------------------------------------------------------------------
template <int C> struct NclOf { static constexpr int value = (C + 1) / 2; };

// G: voxel lines per CTA; chosen so that G * NCL lines keep 4 warps busy
template <typename T, int N, int C>
struct ZTile {
    static constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, LPW = 32 / TL;
    static constexpr int NCL = NclOf<C>::value;
    static constexpr int G = (4 * LPW) / NCL > 0 ? (4 * LPW) / NCL : 1;  // voxel lines per CTA
    static constexpr int LINES = G * NCL;
    // padded tile row: consecutive lines start 16 banks apart
    static constexpr int ROW = N + (sizeof(T) == 4 ? 8 : 4);
};

template <typename T, int N, int C>
constexpr size_t z_fast_smem(size_t extra) {
    typedef typename Cx<T>::t C2;
    typedef ZTile<T, N, C> Z;
    return (size_t)N * sizeof(C2) + (size_t)Z::LINES * Z::ROW * sizeof(C2) +
           (size_t)4 * Z::LPW * Xch<Z::E, Z::TL>::size * sizeof(C2) + 16 + 32 * 32 * sizeof(double) + extra;
}

// transform the tile's complex lines in place: fwd (natural -> natural order
// spectrum) or inv
template <typename C2, int N, int E, int TL, int LINES, int ROW, bool FWD>
__device__ __forceinline__ void z_tile_fft(C2* tile, C2* xch, const C2* tw) {
    constexpr int LPW = 32 / TL;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = lane % TL, lw = lane / TL;
    C2* xl = xch + (warp * LPW + lw) * Xch<E, TL>::size;
    const int nw = blockDim.x >> 5;
#pragma unroll 1
    for (int l0 = warp * LPW; l0 < LINES; l0 += nw * LPW) {
        const int line = l0 + lw;
        const bool ok = line < LINES;
        C2* row = tile + (ok ? line : 0) * ROW;
        C2 v[E];
        if constexpr (FWD) {
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = row[t + TL * j];
            line_fwd<C2, E, TL>(v, t, xl, tw);
            if (ok) {
#pragma unroll
                for (int r = 0; r < E; ++r) row[spec_mode<E, TL>(t, r)] = v[r];
            }
        } else {
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = row[spec_mode<E, TL>(t, r)];
            line_inv<C2, E, TL>(v, t, xl, tw);
            if (ok) {
#pragma unroll
                for (int j = 0; j < E; ++j) row[t + TL * j] = v[j];
            }
        }
    }
}

template <typename T, int N, int C, class Pro>
__global__ void __launch_bounds__(kFastThreads) k_zfwd_fast(GridDims g, const typename Cx<T>::t* __restrict__ twz,
                                                           typename Cx<T>::t* __restrict__ spec, Pro pro,
                                                           const Ctl* __restrict__ ctl) {
    typedef typename Cx<T>::t C2;
    typedef ZTile<T, N, C> Z;
    const int b = blockIdx.y;
    if (ctl[b].done) return;
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* tile = tw + N;
    C2* xch = tile + Z::LINES * Z::ROW;
    char* extra = align_up((char*)(xch + 4 * Z::LPW * Xch<Z::E, Z::TL>::size), 16) + 32 * 32 * sizeof(double);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twz[i];
    pro.load_smem(extra);
    __syncthreads();
    const long long l0 = (long long)blockIdx.x * Z::G;
    double dummy[1];
    for (int i = threadIdx.x; i < Z::G * N; i += blockDim.x) {
        const int gi = i / N, z = i - gi * N;
        const long long l = l0 + gi;
        T val[C];
        if (l < g.NL) {
            pro.eval(b, l * N + z, val, dummy);
        } else {
#pragma unroll
            for (int c = 0; c < C; ++c) val[c] = (T)0;
        }
#pragma unroll
        for (int cl = 0; cl < Z::NCL; ++cl)
            tile[(gi * Z::NCL + cl) * Z::ROW + z] = mk<C2>(val[2 * cl], (2 * cl + 1 < C) ? val[2 * cl + 1] : (T)0);
    }
    __syncthreads();
    z_tile_fft<C2, N, Z::E, Z::TL, Z::LINES, Z::ROW, true>(tile, xch, tw);
    __syncthreads();
    const int Hz = g.Hz, Hzp = g.Hzp;
    for (int i = threadIdx.x; i < Z::G * C * Hzp; i += blockDim.x) {
        const int k = i % Hzp, gc = i / Hzp;
        const int gi = gc / C, c = gc - gi * C;
        const long long l = l0 + gi;
        if (l >= g.NL) continue;
        C2 out = mk<C2>(0, 0);
        if (k < Hz) {
            const C2* row = tile + (gi * Z::NCL + c / 2) * Z::ROW;
            const C2 Zk = row[k];
            const C2 Zm = row[k == 0 ? 0 : N - k];
            out = (c & 1) ? mk<C2>((T)0.5 * (Zk.y + Zm.y), (T)-0.5 * (Zk.x - Zm.x))
                          : mk<C2>((T)0.5 * (Zk.x + Zm.x), (T)0.5 * (Zk.y - Zm.y));
        }
        spec[(((long long)b * C + c) * g.NL + l) * Hzp + k] = out;
    }
}

template <typename T, int N, int C, class Epi>
__global__ void __launch_bounds__(kFastThreads) k_zinv_fast(GridDims g, const typename Cx<T>::t* __restrict__ twz,
                                                           const typename Cx<T>::t* __restrict__ spec, Epi epi,
                                                           const Ctl* __restrict__ ctl, double* partials) {
    typedef typename Cx<T>::t C2;
    typedef ZTile<T, N, C> Z;
    const int b = blockIdx.y;
    if (ctl[b].done) return;
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* tile = tw + N;
    C2* xch = tile + Z::LINES * Z::ROW;
    double* red = (double*)align_up((char*)(xch + 4 * Z::LPW * Xch<Z::E, Z::TL>::size), 16);
    char* extra = (char*)red + 32 * 32 * sizeof(double);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twz[i];
    epi.load_smem(extra);
    const long long l0 = (long long)blockIdx.x * Z::G;
    const int Hz = g.Hz, Hzp = g.Hzp;
    for (int i = threadIdx.x; i < Z::G * Z::NCL * Hz; i += blockDim.x) {
        const int k = i % Hz, gl = i / Hz;
        const int gi = gl / Z::NCL, cl = gl - gi * Z::NCL;
        const long long l = l0 + gi;
        C2 a = mk<C2>(0, 0), bb = mk<C2>(0, 0);
        if (l < g.NL) {
            a = spec[(((long long)b * C + 2 * cl) * g.NL + l) * Hzp + k];
            if (2 * cl + 1 < C) bb = spec[(((long long)b * C + 2 * cl + 1) * g.NL + l) * Hzp + k];
        }
        C2* row = tile + gl * Z::ROW;
        if (k == 0 || 2 * k == N) {
            row[k] = mk<C2>(a.x, bb.x);
        } else {
            row[k] = mk<C2>(a.x - bb.y, a.y + bb.x);
            row[N - k] = mk<C2>(a.x + bb.y, bb.x - a.y);
        }
    }
    __syncthreads();
    z_tile_fft<C2, N, Z::E, Z::TL, Z::LINES, Z::ROW, false>(tile, xch, tw);
    __syncthreads();
    const T invV = (T)(1.0 / (double)g.V);
    double acc[Epi::NSUM > 0 ? Epi::NSUM : 1] = {};
    for (int i = threadIdx.x; i < Z::G * N; i += blockDim.x) {
        const int gi = i / N, z = i - gi * N;
        const long long l = l0 + gi;
        if (l >= g.NL) continue;
        T xc[C];
#pragma unroll
        for (int cl = 0; cl < Z::NCL; ++cl) {
            const C2 w = tile[(gi * Z::NCL + cl) * Z::ROW + z];
            xc[2 * cl] = w.x * invV;
            if (2 * cl + 1 < C) xc[2 * cl + 1] = w.y * invV;
        }
        epi.apply(b, l * N + z, xc, acc);
    }
    if constexpr (Epi::NSUM > 0) {
        block_reduce_store<Epi::NSUM>(acc, red, partials, b, gridDim.x, blockIdx.x);
    }
}

}  // namespace m3d
