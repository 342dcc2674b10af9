// passes_fast.cuh -- the five sweep passes for compile-time line lengths
// (32, 48, 64, 96, 128, 256), built on the warp-split line FFT of
// fft_reg.cuh.  Same data layout, operators and reductions as the generic
// kernels in passes.cuh, which remain the path for any other length.
//
// Column passes (y, x): lane = col + CPW*t with CPW = 32/T columns per warp,
// so one load instruction touches CPW consecutive complex words of T rows
// (whole 32-byte sectors).  The y pass goes global -> registers -> one
// warp-local exchange -> global.  The x turnaround first issues cp.async
// copies of all C components of its columns into a per-warp staging area
// (all loads in flight together), transforms each component there (the
// staging rows double as the exchange buffer), applies the spectral op to
// every mode with all components at hand, and transforms back.
// z passes: a tile of G voxel lines is staged in shared memory (the
// prologue/epilogue need all components of a voxel); components are packed
// two per complex line (c0 + i c1, ...) and each line is transformed by T
// lanes in registers, exchanging through its own padded tile row.  The
// epilogue's global loads are issued before the tile FFT so their latency
// overlaps it.
#pragma once
#include <type_traits>

#include "fft_reg.cuh"
#include "passes.cuh"
#include "physics.cuh"
#include "tma.cuh"

namespace m3d {

constexpr int kFastThreads = 128;

// CTAs per SM the FP64 z kernels of long lines (N >= 96) with up to three
// components are compiled for: their register cap is 65536 / (128 x value)
// per thread.  Uncapped, the 128-point thermal z inverse takes 244 registers
// (two 4-warp CTAs per SM); at three CTAs it fits 168 with a small spill.
// Six- and nine-component kernels keep no cap (a 168 cap spills ~1 KB).
#ifndef M3D_FP64_MINB
#define M3D_FP64_MINB 3
#endif
template <typename T, int N, int C>
struct FastMinB {
    static constexpr int value = (sizeof(T) == 8 && N >= 96 && C <= 3) ? M3D_FP64_MINB : 1;
};

// Shared-memory bank layout of a line's row (which is also its exchange
// buffer).  Rows hold at least max(N, E*(T+1)) complex elements, padded so
// that row length == `tgt` modulo the number of complex elements per
// wavefront slot cycle (16 for 8-byte FP32 complex, 8 for 16-byte FP64), and
// lines with odd index XOR-swizzle bit 0 when `sw`.  The (tgt, sw) pairs are
// the conflict-free choices for the four access patterns of a warp
// (natural, spectral, exchange write, exchange read), found by enumerating
// all paddings and both swizzles under half-warp (8-byte) / quarter-warp
// (16-byte) servicing, separately for the column layout of the x/y passes
// (lane = col + CPW*t) and the line layout of the z tiles (lane = t + T*line).
constexpr int bank_tgt(bool fp32, int E, int T, bool col) {
    if (fp32) {
        if (col) return (E == 16 && T == 8) ? 4 : (E == 8 && T == 8) ? 4 : (E == 32) ? 3 : (T == 4) ? 2 : 8;
        return (T == 4) ? 4 : 8;
    }
    if (col) return (T == 16) ? 4 : (T == 8) ? 2 : 1;
    return (T == 4) ? 4 : 0;
}
constexpr int bank_sw(bool fp32, int E, int T, bool col) {
    if (fp32) {
        if (col) return (E == 16 && T == 8) || (E == 8 && T == 4) || (E == 24 && T == 4);
        return (E == 16 && T == 8) || (E == 32) || (E == 8 && T == 4) || (E == 24 && T == 4);
    }
    if (col) return (E == 16 && T == 8);
    return (E == 8 && T == 4) || (E == 24 && T == 4);
}

template <typename T, int N, bool COL>
struct RowLen {
    static constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl;
    static constexpr bool fp32 = sizeof(T) == 4;
    static constexpr int base = (N > E * (TL + 1)) ? N : E * (TL + 1);
    static constexpr int mod = fp32 ? 16 : 8, tgt = bank_tgt(fp32, E, TL, COL);
    static constexpr int value = base + ((tgt - base % mod) + mod) % mod;
    static constexpr int sw = bank_sw(fp32, E, TL, COL);
};

// ---------------------------------------------------------------------------
// y pass: CTA = 4 warps = 4*CPW consecutive kz columns of one (batch*comp, x)
// ---------------------------------------------------------------------------
template <typename T, int N>
constexpr size_t ypass_fast_smem() {
    typedef typename Cx<T>::t C2;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    (void)E;
    return (size_t)N * sizeof(C2) + (size_t)4 * CPW * RowLen<T, N, true>::value * sizeof(C2);
}

template <typename T, int N, int SIGN>
__global__ void __launch_bounds__(kFastThreads) k_ypass_fast(GridDims g, const typename Cx<T>::t* __restrict__ twy,
                                                            typename Cx<T>::t* __restrict__ spec, int C,
                                                            const Ctl* __restrict__ ctl) {
    typedef typename Cx<T>::t C2;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    constexpr int XS = RowLen<T, N, true>::value;
    const int b = entry_of(g, blockIdx.y / C);
    if (b < 0 || ctl[b].done) return;
    const int cb = b * C + blockIdx.y % C;
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
    const int sw = RowLen<T, N, true>::sw ? (col & 1) : 0;
    C2 v[E];
    if constexpr (SIGN < 0) {
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = ok ? base[(long long)(t + TL * j) * g.Hzp] : mk<C2>(0, 0);
        line_fwd<C2, E, TL>(v, t, xl, tw, sw);
        if (ok) {
#pragma unroll
            for (int r = 0; r < E; ++r) base[(long long)spec_mode<E, TL>(t, r) * g.Hzp] = v[r];
        }
    } else {
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = ok ? base[(long long)spec_mode<E, TL>(t, r) * g.Hzp] : mk<C2>(0, 0);
        line_inv<C2, E, TL>(v, t, xl, tw, sw);
        if (ok) {
#pragma unroll
            for (int j = 0; j < E; ++j) base[(long long)(t + TL * j) * g.Hzp] = v[j];
        }
    }
}

// ---------------------------------------------------------------------------
// x turnaround
// ---------------------------------------------------------------------------
// 8- or 16-byte asynchronous global->shared copy; src_bytes = 0 writes zeros
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gmem_src, int bytes, int src_bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gmem_src), "r"(src_bytes));
    else
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gmem_src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
}

// warps per CTA of the x turnaround: as many as keep the staging <= 24 KB
// (small CTAs: many resident per SM and a fine-grained tail)
template <typename T, int N, int C>
struct XWarps {
    static constexpr size_t per_warp =
        (size_t)C * (32 / LineSplit<T, N>::Tl) * RowLen<T, N, true>::value * sizeof(typename Cx<T>::t);
    static constexpr int value = (4 * per_warp <= 24 * 1024) ? 4 : ((2 * per_warp <= 24 * 1024) ? 2 : 1);
};

template <typename T, int N, int C, int NSUM>
constexpr size_t xturn_fast_smem() {
    typedef typename Cx<T>::t C2;
    return (size_t)N * sizeof(C2) + (size_t)XWarps<T, N, C>::value * XWarps<T, N, C>::per_warp + 16 +
           (size_t)32 * NSUM * sizeof(double);
}

template <typename T, int N, int C, class Spec>
__global__ void __launch_bounds__(kFastThreads) k_xturn_fast(GridDims g, const typename Cx<T>::t* __restrict__ twx,
                                                            typename Cx<T>::t* __restrict__ spec, Spec op,
                                                            const Ctl* __restrict__ ctl, double* partials) {
    typedef typename Cx<T>::t C2;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    constexpr int WPC = XWarps<T, N, C>::value;
    constexpr int RL = RowLen<T, N, true>::value;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
    op.prepare(ctl, b);
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* stage = tw + N;  // [warp][c][col][RL]
    double* red = (double*)align_up((char*)(stage + WPC * C * CPW * RL), 16);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % CPW, t = lane / CPW;
    const int ncol_cta = WPC * CPW;
    const int ntz = (g.Hzp + ncol_cta - 1) / ncol_cta;
    const int y = blockIdx.x / ntz;
    const int kz = (blockIdx.x - y * ntz) * ncol_cta + warp * CPW + col;
    const bool ok = kz < g.Hzp;
    const long long cstride = g.NL * g.Hzp;            // component stride
    const long long xstride = (long long)g.Ny * g.Hzp;  // x stride
    const C2* base = spec + ((long long)b * C * g.NL + y) * g.Hzp + (ok ? kz : 0);
    C2* wst = stage + warp * C * CPW * RL;
    const int sw = RowLen<T, N, true>::sw ? (col & 1) : 0;  // bank swizzle of this column's rows
    // issue every load of the warp's columns (all components) at once
#pragma unroll 1
    for (int c = 0; c < C; ++c) {
        C2* row = wst + (c * CPW + col) * RL;
#pragma unroll
        for (int j = 0; j < E; ++j)
            cp_async(row + ((t + TL * j) ^ sw), base + c * cstride + (long long)(t + TL * j) * xstride,
                     (int)sizeof(C2), ok ? (int)sizeof(C2) : 0);
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twx[i];
    cp_async_wait_all();
    __syncthreads();
#pragma unroll 1
    for (int c = 0; c < C; ++c) {
        C2* row = wst + (c * CPW + col) * RL;
        C2 v[E];
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = row[(t + TL * j) ^ sw];
        __syncwarp();
        line_fwd<C2, E, TL>(v, t, row, tw, sw);
#pragma unroll
        for (int r = 0; r < E; ++r) row[spec_mode<E, TL>(t, r) ^ sw] = v[r];
    }
    double acc[Spec::NSUM > 0 ? Spec::NSUM : 1] = {};
    const bool live = ok && kz < g.Hz;
#pragma unroll 1
    for (int r = 0; r < E; ++r) {
        const int mode = spec_mode<E, TL>(t, r);
        C2 m[C];
#pragma unroll
        for (int c = 0; c < C; ++c) m[c] = wst[(c * CPW + col) * RL + (mode ^ sw)];
        if (live) op.apply(b, mode, y, kz, m, acc, ctl);
        if constexpr (Spec::kInverse) {
#pragma unroll
            for (int c = 0; c < C; ++c) wst[(c * CPW + col) * RL + (mode ^ sw)] = m[c];
        }
    }
    if constexpr (Spec::NSUM > 0) {
        block_reduce_store<Spec::NSUM>(acc, red, partials, b, gridDim.x, blockIdx.x);
    }
    if constexpr (Spec::kInverse) {
        C2* out = spec + ((long long)b * C * g.NL + y) * g.Hzp + (ok ? kz : 0);
#pragma unroll 1
        for (int c = 0; c < C; ++c) {
            C2* row = wst + (c * CPW + col) * RL;
            C2 v[E];
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = row[spec_mode<E, TL>(t, r) ^ sw];
            __syncwarp();
            line_inv<C2, E, TL>(v, t, row, tw, sw);
            if (ok) {
#pragma unroll
                for (int j = 0; j < E; ++j) out[c * cstride + (long long)(t + TL * j) * xstride] = v[j];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// x turnaround, component-parallel: one CTA of C warps per group of CPW kz
// columns, warp c transforming component c of the group's columns.  The
// staged kernel above gives each warp all C components of its own columns,
// so one warp owns C x CPW staged rows (six FP32 96-point components: 50 KB,
// four warps per SM); here the same rows are shared by C warps (six: 24 warps
// per SM at 96^3).  Phases, with a block barrier between them: (1) warp c
// copies and forward-transforms component c of every column; (2) all threads
// apply the spectral operator, one (mode, column) point at a time, to the C
// components of the point; (3) warp c inverse-transforms and stores
// component c.  Per line and per mode the arithmetic is the staged kernel's
// (equal bits where the operator keeps no sums; sums of the reference stop
// rule are added in another order).
// ---------------------------------------------------------------------------
template <typename T, int N, int C, int NSUM>
constexpr size_t xturn_cp_smem() {
    typedef typename Cx<T>::t C2;
    constexpr int CPW = 32 / LineSplit<T, N>::Tl;
    return (size_t)N * sizeof(C2) + (size_t)C * CPW * RowLen<T, N, true>::value * sizeof(C2) + 16 +
           (size_t)32 * (NSUM > 0 ? NSUM : 1) * sizeof(double);
}

// CTAs per SM of the six-component FP32 kernel at N = 96: three (a cap of
// 112 registers instead of 152, 140 bytes of spill; the batch workload's
// 96^3 group's x turnaround 157 -> 142 ms on one box, bitwise the same).  At
// 64^3 the same cap timed equal; FP64 and N = 256 spill up to 1 KB under it.
#ifndef M3D_XCP_MINB
#define M3D_XCP_MINB 3
#endif
template <typename T, int N, int C, class Spec>
__global__ void __launch_bounds__(32 * C, (C == 6 && sizeof(T) == 4 && N == 96) ? M3D_XCP_MINB : 1) k_xturn_cp(GridDims g, const typename Cx<T>::t* __restrict__ twx,
                                                     typename Cx<T>::t* __restrict__ spec, Spec op,
                                                     const Ctl* __restrict__ ctl, double* partials) {
    typedef typename Cx<T>::t C2;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    constexpr int RL = RowLen<T, N, true>::value;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
    op.prepare(ctl, b);
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* stage = tw + N;  // [c][col][RL]
    double* red = (double*)align_up((char*)(stage + C * CPW * RL), 16);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % CPW, t = lane / CPW;
    const int ngrp = (g.Hzp + CPW - 1) / CPW;
    const int y = blockIdx.x / ngrp;
    const int kz0 = (blockIdx.x - y * ngrp) * CPW;
    const int kz = kz0 + col;
    const bool ok = kz < g.Hzp;
    const long long cstride = g.NL * g.Hzp;            // component stride
    const long long xstride = (long long)g.Ny * g.Hzp;  // x stride
    C2* cbase = spec + ((long long)b * C * g.NL + y) * g.Hzp + warp * cstride + (ok ? kz : 0);  // component `warp`
    const int sw = RowLen<T, N, true>::sw ? (col & 1) : 0;
    C2* row = stage + (warp * CPW + col) * RL;
#pragma unroll
    for (int j = 0; j < E; ++j)
        cp_async(row + ((t + TL * j) ^ sw), cbase + (long long)(t + TL * j) * xstride, (int)sizeof(C2),
                 ok ? (int)sizeof(C2) : 0);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twx[i];
    cp_async_wait_all();
    __syncthreads();
    {
        C2 v[E];
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = row[(t + TL * j) ^ sw];
        __syncwarp();
        line_fwd<C2, E, TL>(v, t, row, tw, sw);
#pragma unroll
        for (int r = 0; r < E; ++r) row[spec_mode<E, TL>(t, r) ^ sw] = v[r];
    }
    __syncthreads();
    double acc[Spec::NSUM > 0 ? Spec::NSUM : 1] = {};
    for (int p = threadIdx.x; p < CPW * N; p += blockDim.x) {
        const int pc = p % CPW, mode = p / CPW;
        const int pkz = kz0 + pc;
        if (pkz >= g.Hz) continue;  // past the half spectrum (padding or beyond Hzp)
        const int psw = RowLen<T, N, true>::sw ? (pc & 1) : 0;
        C2 m[C];
#pragma unroll
        for (int c = 0; c < C; ++c) m[c] = stage[(c * CPW + pc) * RL + (mode ^ psw)];
        op.apply(b, mode, y, pkz, m, acc, ctl);
        if constexpr (Spec::kInverse) {
#pragma unroll
            for (int c = 0; c < C; ++c) stage[(c * CPW + pc) * RL + (mode ^ psw)] = m[c];
        }
    }
    if constexpr (Spec::NSUM > 0) {
        block_reduce_store<Spec::NSUM>(acc, red, partials, b, gridDim.x, blockIdx.x);
    }
    if constexpr (Spec::kInverse) {
        __syncthreads();
        C2 v[E];
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = row[spec_mode<E, TL>(t, r) ^ sw];
        __syncwarp();
        line_inv<C2, E, TL>(v, t, row, tw, sw);
        if (ok) {
#pragma unroll
            for (int j = 0; j < E; ++j) cbase[(long long)(t + TL * j) * xstride] = v[j];
        }
    }
}

// ---------------------------------------------------------------------------
// x turnaround with the three components of a column in registers (thermal
// fields in FP32): each lane loads its E points of all three components
// straight from global memory (every load of a warp covers CPW consecutive
// columns of TL rows), transforms them with only the column's exchange row in
// shared memory, applies the spectral operator to the three components of
// each of its modes from registers, and transforms back.  Compared with the
// staged kernel above, no component is staged or round-tripped through shared
// memory for the operator: about 200 fewer shared-memory instructions per
// lane, the same per-line arithmetic (results are bitwise equal).  Used up to
// N = 64, where the 3 x E points per lane fit the registers without spilling.
// ---------------------------------------------------------------------------
constexpr int kXRegWarps = 4;

template <typename T, int N, int NSUM>
constexpr size_t xturn_reg_smem() {
    typedef typename Cx<T>::t C2;
    constexpr int CPW = 32 / LineSplit<T, N>::Tl;
    return (size_t)N * sizeof(C2) + (size_t)kXRegWarps * CPW * RowLen<T, N, true>::value * sizeof(C2) + 16 +
           (size_t)32 * (NSUM > 0 ? NSUM : 1) * sizeof(double);
}

template <typename T, int N, class Spec>
__global__ void __launch_bounds__(32 * kXRegWarps) k_xturn_reg(GridDims g, const typename Cx<T>::t* __restrict__ twx,
                                                              typename Cx<T>::t* __restrict__ spec, Spec op,
                                                              const Ctl* __restrict__ ctl, double* partials) {
    typedef typename Cx<T>::t C2;
    constexpr int C = 3;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    constexpr int RL = RowLen<T, N, true>::value;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
    op.prepare(ctl, b);
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* xch = tw + N;  // [warp][col][RL]
    double* red = (double*)align_up((char*)(xch + kXRegWarps * CPW * RL), 16);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % CPW, t = lane / CPW;
    constexpr int ncol_cta = kXRegWarps * CPW;
    const int ntz = (g.Hzp + ncol_cta - 1) / ncol_cta;
    const int y = blockIdx.x / ntz;
    const int kz = (blockIdx.x - y * ntz) * ncol_cta + warp * CPW + col;
    const bool ok = kz < g.Hzp;
    const long long cstride = g.NL * g.Hzp;            // component stride
    const long long xstride = (long long)g.Ny * g.Hzp;  // x stride
    C2* base = spec + ((long long)b * C * g.NL + y) * g.Hzp + (ok ? kz : 0);
    C2* xl = xch + (warp * CPW + col) * RL;
    const int sw = RowLen<T, N, true>::sw ? (col & 1) : 0;
    C2 v[C][E];
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
        for (int j = 0; j < E; ++j) v[c][j] = ok ? base[c * cstride + (long long)(t + TL * j) * xstride] : mk<C2>(0, 0);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twx[i];
    __syncthreads();
#pragma unroll
    for (int c = 0; c < C; ++c) line_fwd<C2, E, TL>(v[c], t, xl, tw, sw);
    double acc[Spec::NSUM > 0 ? Spec::NSUM : 1] = {};
    const bool live = ok && kz < g.Hz;
#pragma unroll
    for (int r = 0; r < E; ++r) {
        C2 m[C] = {v[0][r], v[1][r], v[2][r]};
        if (live) op.apply(b, spec_mode<E, TL>(t, r), y, kz, m, acc, ctl);
#pragma unroll
        for (int c = 0; c < C; ++c) v[c][r] = m[c];
    }
    if constexpr (Spec::NSUM > 0) {
        block_reduce_store<Spec::NSUM>(acc, red, partials, b, gridDim.x, blockIdx.x);
    }
    if constexpr (Spec::kInverse) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
            line_inv<C2, E, TL>(v[c], t, xl, tw, sw);
            if (ok) {
#pragma unroll
                for (int j = 0; j < E; ++j) base[c * cstride + (long long)(t + TL * j) * xstride] = v[c][j];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// x turnaround of the thermal Green operators in rank-one form.  Both act on
// a mode through d = xi . v only (physics.cuh, SpecGreen):
//   gradient-based  v_c' = xi_c D,                 D = -p1 d / |xi|^2
//   flux-based      v_c' = -p1 (v_c - xi_c D),    D = d / |xi|^2
// and along an x column xi_z and xi_y are constant, so the inverse transforms
// of the three outputs need only IFFT(D) and IFFT(xi_x D):
//   gradient  out_z = xi_z IFFT(D), out_y = xi_y IFFT(D), out_x = IFFT(xi_x D)
//   flux      out_c = -p1 N v_c + p1 (same terms),  N v_c = IFFT(FFT(v_c))
// (unnormalised transforms; v_c is re-read from global memory, where it still
// lies).  d is accumulated while each component is transformed, so a column
// costs three forward and two inverse line transforms instead of six, and no
// component is staged in shared memory.  The k = 0 mode, whose value is set
// rather than computed (the load or 0), is handled in the one column holding
// it: D(0) = 0 and the missing constant is added to every x.  Arithmetic is
// the same to rounding (FP32 and FP64); the wave vectors follow SpecGreen's sign and
// wrap rules exactly.
// ---------------------------------------------------------------------------
// CTAs per SM the rank-one x turnaround is compiled for (bounds its registers;
// an FP64 lane holds twice the registers per point)
template <typename T, int N> struct XR1MinB {
    static constexpr int value = sizeof(T) == 4 ? (N == 128 ? 3 : (N == 96 ? 2 : 4)) : (N == 128 ? 2 : 3);
};

template <typename T, int N>
__global__ void __launch_bounds__(32 * kXRegWarps, XR1MinB<T, N>::value) k_xturn_r1(GridDims g, const typename Cx<T>::t* __restrict__ twx,
                                                             typename Cx<T>::t* __restrict__ spec, SpecGreenT<T> op,
                                                             const Ctl* __restrict__ ctl) {
    typedef typename Cx<T>::t C2;
    constexpr int C = 3;
    constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    constexpr int RL = RowLen<T, N, true>::value;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
    op.prepare(ctl, b);
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* xch = tw + N;  // [warp][col][RL]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % CPW, t = lane / CPW;
    // warp-granular work items: item = (y, group of CPW kz columns), kXRegWarps
    // consecutive items per CTA, so the short last group of a y row (Hzp is
    // not a multiple of CPW) costs one warp, not a whole CTA
    const int ngrp = (g.Hzp + CPW - 1) / CPW;
    const int item = blockIdx.x * kXRegWarps + warp;
    const bool have = item < g.Ny * ngrp;
    const int y = have ? item / ngrp : 0;
    const int kz = (item - y * ngrp) * CPW + col;
    const bool ok = have && kz < g.Hzp;
    const long long cstride = g.NL * g.Hzp;            // component stride
    const long long xstride = (long long)g.Ny * g.Hzp;  // x stride
    C2* base = spec + ((long long)b * C * g.NL + y) * g.Hzp + (ok ? kz : 0);
    C2* xl = xch + (warp * CPW + col) * RL;
    const int sw = RowLen<T, N, true>::sw ? (col & 1) : 0;
    const bool grad = op.kind == GREEN_TGRAD;
    const T fz = (T)sfreq(kz, op.pos_nyq ? g.Nz / 2 : (g.Nz - 1) / 2, g.Nz);
    const T fy = (T)sfreq(y, op.pos_nyq ? g.Ny / 2 : (g.Ny - 1) / 2, g.Ny);
    const bool origin = ok && y == 0 && kz == 0;  // the column holding the k = 0 mode
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twx[i];
    __syncthreads();
    if (!have) return;  // no block barrier follows
    C2 v[E], d[E];
    T fx[E];   // x frequency of each of this lane's modes
    C2 k0[C];  // mode 0 of each component (origin column)
#pragma unroll
    for (int r = 0; r < E; ++r) {
        fx[r] = (T)sfreq(spec_mode<E, TL>(t, r), op.pos_nyq ? g.Nx / 2 : (g.Nx - 1) / 2, op.xwrap);
        d[r] = mk<C2>(0, 0);
    }
    // one component per trip (its loads are not hoisted over the others'
    // transforms: the registers hold one component and d)
#pragma unroll 1
    for (int c = 0; c < C; ++c) {
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = ok ? base[c * cstride + (long long)(t + TL * j) * xstride] : mk<C2>(0, 0);
        line_fwd<C2, E, TL>(v, t, xl, tw, sw);
        const C2 m0 = mk<C2>(__shfl_sync(0xffffffffu, v[0].x, col), __shfl_sync(0xffffffffu, v[0].y, col));  // t = 0: mode 0
        if (c == 0) k0[0] = m0;
        else if (c == 1) k0[1] = m0;
        else k0[2] = m0;
        const T fcol = c == 0 ? fz : fy;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const T fc = c == 2 ? fx[r] : fcol;
            d[r] = mk<C2>(d[r].x + fc * v[r].x, d[r].y + fc * v[r].y);
        }
    }
    // D = coef d per mode; the x-frequency weighted copy for the x component
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const int mode = spec_mode<E, TL>(t, r);
        const T n2 = fz * fz + fy * fy + fx[r] * fx[r];
        const T coef = (origin && mode == 0) ? (T)0 : (grad ? -op.p1 : (T)1) / n2;
        d[r] = mk<C2>(coef * d[r].x, coef * d[r].y);
        v[r] = mk<C2>(fx[r] * d[r].x, fx[r] * d[r].y);
    }
    // the k = 0 mode's value (the load, or 0 in a correction solve) minus what
    // the rank-one terms give there (0, and -p1 N mean for the flux form)
    C2 add[C] = {mk<C2>(0, 0), mk<C2>(0, 0), mk<C2>(0, 0)};
    if (origin) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const T kc = op.zero_k0 ? (T)0 : (T)ctl[b].kzero[c];
            add[c] = grad ? mk<C2>(kc, 0) : mk<C2>(kc + op.p1 * k0[c].x, op.p1 * k0[c].y);
        }
    }
    const T sc = grad ? (T)1 : op.p1;  // scale of the rank-one terms
    // out_c = sc * (column term) [- p1 N v_c] + add_c, written over v_c
    auto emit = [&](int c, const C2 (&u)[E], T f) {
#pragma unroll
        for (int j = 0; j < E; ++j) {
            C2* p = base + c * cstride + (long long)(t + TL * j) * xstride;
            C2 o = mk<C2>(sc * f * u[j].x, sc * f * u[j].y);
            if (!grad) {
                const C2 in = *p;
                o = mk<C2>(o.x - op.p1 * (T)N * in.x, o.y - op.p1 * (T)N * in.y);
            }
            *p = mk<C2>(o.x + add[c].x, o.y + add[c].y);
        }
    };
    line_inv<C2, E, TL>(d, t, xl, tw, sw);  // IFFT(D), natural order
    if (ok) {
        emit(0, d, fz);
        emit(1, d, fy);
    }
    line_inv<C2, E, TL>(v, t, xl, tw, sw);  // IFFT(xi_x D)
    if (ok) emit(2, v, (T)1);
}

// ---------------------------------------------------------------------------
// The rank-one x turnaround with its column loads staged by TMA.  A warp walks
// work items (entry, y, group of CPW kz columns) persistently; each component
// of an item is one 3-D box (CPW columns x 1 row x N points along x) copied
// into one of the warp's two slots.  The copies of a warp form one sequence
// (item k, component c) = copy 3k + c, slot (3k + c) mod 2, and copy m + 2 is
// requested as soon as copy m has been read and transformed: a copy is in
// flight while the previous one is transformed, across item boundaries, so
// the loads' latency is hidden by the transforms.  Columns past Hzp (the short last group) are
// zero-filled by the copy, as the plain kernel zero-fills them.  The
// arithmetic is k_xturn_r1's, operation for operation, so the two give equal
// bits.  Every barrier wait is bounded: on expiry the error word is set, the
// warp waits (bounded) for the copies it still has in flight and stops.
// ---------------------------------------------------------------------------
template <typename T, int N>
struct XR1Tma {
    typedef typename Cx<T>::t C2;
    static constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL;
    static constexpr int RL = RowLen<T, N, true>::value;
    static constexpr int SLOT = N * CPW;  // complex elements per slot: [x][column]
    static constexpr uint32_t slot_bytes = (uint32_t)(SLOT * sizeof(C2));
    static_assert(slot_bytes % 128 == 0, "slots stay 128-byte aligned");
    static constexpr size_t smem() {
        return 128 + (size_t)kXRegWarps * 2 * slot_bytes + (size_t)N * sizeof(C2) +
               (size_t)kXRegWarps * CPW * RL * sizeof(C2) + 16 + (size_t)kXRegWarps * 2 * sizeof(uint64_t);
    }
};

// CTAs per SM: those of the plain kernel (at FP32 N = 128 three, 168
// registers; a 128-register cap for four CTAs -- every 128^3 work item in one
// round -- spills and measured the same, 25.2 us per launch)
#ifndef M3D_XR1TMA_MINB
#define M3D_XR1TMA_MINB 0
#endif
template <typename T, int N> struct XR1TmaMinB {
    static constexpr int value = M3D_XR1TMA_MINB > 0 ? M3D_XR1TMA_MINB : XR1MinB<T, N>::value;
};

template <typename T, int N>
__global__ void __launch_bounds__(32 * kXRegWarps, XR1TmaMinB<T, N>::value)
    k_xturn_r1_tma(const __grid_constant__ CUtensorMap map, GridDims g, const typename Cx<T>::t* __restrict__ twx,
                   typename Cx<T>::t* __restrict__ spec, SpecGreenT<T> op, const Ctl* __restrict__ ctl, int nitems,
                   int* err) {
    typedef typename Cx<T>::t C2;
    typedef XR1Tma<T, N> X;
    constexpr int C = 3;
    constexpr int E = X::E, TL = X::TL, CPW = X::CPW, RL = X::RL;
    extern __shared__ __align__(16) char smem_raw[];
    C2* stage = (C2*)align_up(smem_raw, 128);
    C2* tw = stage + kXRegWarps * 2 * X::SLOT;
    C2* xch = tw + N;
    uint64_t* bars = (uint64_t*)align_up((char*)(xch + kXRegWarps * CPW * RL), 16);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % CPW, t = lane / CPW;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twx[i];
    if (threadIdx.x == 0) {
        for (int s = 0; s < kXRegWarps * 2; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();  // the only block barrier
    C2* st = stage + warp * 2 * X::SLOT;
    uint64_t* bar = bars + warp * 2;
    C2* xl = xch + (warp * CPW + col) * RL;
    const int sw = RowLen<T, N, true>::sw ? (col & 1) : 0;
    const int ngrp = (g.Hzp + CPW - 1) / CPW;
    const int per_entry = g.Ny * ngrp;
    const int wstride = gridDim.x * kXRegWarps;
    const long long cstride = g.NL * g.Hzp;            // component stride
    const long long xstride = (long long)g.Ny * g.Hzp;  // x stride
    // this warp's next item (from `it` on) whose entry is still iterating
    // (items are numbered over the launch's entry slots)
    auto next = [&](int it) {
        for (; it < nitems; it += wstride) {
            const int b = entry_of(g, it / per_entry);
            if (b >= 0 && !ctl[b].done) return it;
        }
        return -1;
    };
    auto issue = [&](int m, int it) {  // lane 0: copy m (component m % 3 of item `it`) into slot m % 2
        const int s = it / per_entry, rem = it - s * per_entry, b = entry_of(g, s);
        const int y = rem / ngrp, grp = rem - y * ngrp;
        mbar_expect_tx(&bar[m & 1], X::slot_bytes);
        tma_load_3d(st + (m & 1) * X::SLOT, &map, 2 * grp * CPW, y, (b * C + m % 3) * g.Nx, &bar[m & 1]);
    };
    int it = next(blockIdx.x * kXRegWarps + warp);
    int issued = 0;  // copies requested so far (warp-uniform)
    if (it >= 0) {
        if (lane == 0) {
            issue(0, it);
            issue(1, it);
        }
        issued = 2;
    }
    int m = 0;  // the next copy to consume
    while (it >= 0) {
        const int nx = next(it + wstride);
        const int s = it / per_entry, rem = it - s * per_entry, b = entry_of(g, s);
        const int y = rem / ngrp;
        const int kz = (rem - y * ngrp) * CPW + col;
        const bool ok = kz < g.Hzp;
        op.prepare(ctl, b);
        C2* base = spec + ((long long)b * C * g.NL + y) * g.Hzp + (ok ? kz : 0);
        const bool grad = op.kind == GREEN_TGRAD;
        const T fz = (T)sfreq(kz, op.pos_nyq ? g.Nz / 2 : (g.Nz - 1) / 2, g.Nz);
        const T fy = (T)sfreq(y, op.pos_nyq ? g.Ny / 2 : (g.Ny - 1) / 2, g.Ny);
        const bool origin = ok && y == 0 && kz == 0;
        C2 v[E], d[E];
        T fx[E];  // x frequency of each of this lane's modes
        C2 k0[C];
#pragma unroll
        for (int r = 0; r < E; ++r) {
            fx[r] = (T)sfreq(spec_mode<E, TL>(t, r), op.pos_nyq ? g.Nx / 2 : (g.Nx - 1) / 2, op.xwrap);
            d[r] = mk<C2>(0, 0);
        }
        bool failed = false;
#pragma unroll 1
        for (int c = 0; c < C; ++c, ++m) {
            const bool arrived = mbar_wait(&bar[m & 1], (uint32_t)((m >> 1) & 1), err);
            if (__any_sync(0xffffffffu, !arrived)) { failed = true; break; }
            const C2* sl = st + (m & 1) * X::SLOT;
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = sl[(t + TL * j) * CPW + col];
            line_fwd<C2, E, TL>(v, t, xl, tw, sw);
            // the slot is refilled only after every lane's reads of it have
            // returned (the transform consumed them; line_fwd ends with a warp
            // barrier) and a proxy fence orders them before the copy's writes
            const int it2 = c == 0 ? it : nx;  // copy m + 2: this item's component 2, or the next item's 0 and 1
            if (it2 >= 0) {
                if (lane == 0) {
                    fence_proxy_async();
                    issue(m + 2, it2);
                }
                issued = m + 3;
            }
            const C2 m0 = mk<C2>(__shfl_sync(0xffffffffu, v[0].x, col), __shfl_sync(0xffffffffu, v[0].y, col));
            if (c == 0) k0[0] = m0;
            else if (c == 1) k0[1] = m0;
            else k0[2] = m0;
            const T fcol = c == 0 ? fz : fy;
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const T fc = c == 2 ? fx[r] : fcol;
                d[r] = mk<C2>(d[r].x + fc * v[r].x, d[r].y + fc * v[r].y);
            }
        }
        if (failed) {
            // wait (bounded, no further error) for the copies still in flight: m .. issued - 1
            for (int q = m; q < issued; ++q) mbar_wait(&bar[q & 1], (uint32_t)((q >> 1) & 1), nullptr, 1 << 16);
            return;
        }
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int mode = spec_mode<E, TL>(t, r);
            const T n2 = fz * fz + fy * fy + fx[r] * fx[r];
            const T coef = (origin && mode == 0) ? (T)0 : (grad ? -op.p1 : (T)1) / n2;
            d[r] = mk<C2>(coef * d[r].x, coef * d[r].y);
            v[r] = mk<C2>(fx[r] * d[r].x, fx[r] * d[r].y);
        }
        C2 add[C] = {mk<C2>(0, 0), mk<C2>(0, 0), mk<C2>(0, 0)};
        if (origin) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const T kc = op.zero_k0 ? (T)0 : (T)ctl[b].kzero[c];
                add[c] = grad ? mk<C2>(kc, 0) : mk<C2>(kc + op.p1 * k0[c].x, op.p1 * k0[c].y);
            }
        }
        const T sc = grad ? (T)1 : op.p1;
        auto emit = [&](int c, const C2 (&u)[E], T f) {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                C2* p = base + c * cstride + (long long)(t + TL * j) * xstride;
                C2 o = mk<C2>(sc * f * u[j].x, sc * f * u[j].y);
                if (!grad) {
                    const C2 in = *p;
                    o = mk<C2>(o.x - op.p1 * (T)N * in.x, o.y - op.p1 * (T)N * in.y);
                }
                *p = mk<C2>(o.x + add[c].x, o.y + add[c].y);
            }
        };
        line_inv<C2, E, TL>(d, t, xl, tw, sw);
        if (ok) {
            emit(0, d, fz);
            emit(1, d, fy);
        }
        line_inv<C2, E, TL>(v, t, xl, tw, sw);
        if (ok) emit(2, v, (T)1);
        it = nx;
    }
}

// ---------------------------------------------------------------------------
// z passes.  Tile of G voxel lines x NCL complex lines (NCL = ceil(C/2)).
// ---------------------------------------------------------------------------
template <int C> struct NclOf { static constexpr int value = (C + 1) / 2; };

// per-thread prefetch record of an operator: four voxels (kW = 4) or one
template <class Op, bool V = (Op::kW > 1)> struct PreOf { typedef typename Op::Pre type; };
template <class Op> struct PreOf<Op, true> { typedef typename Op::PreW type; };

template <typename T, int N, int C>
struct ZTile {
    static constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, LPW = 32 / TL;
    static constexpr int NCL = NclOf<C>::value;
    static constexpr int G = (4 * LPW) / NCL > 0 ? (4 * LPW) / NCL : 1;  // voxel lines per CTA
    static constexpr int LINES = G * NCL;
    static constexpr int SLOTS = ((LINES + 4 * LPW - 1) / (4 * LPW)) * 4 * LPW;  // rows incl. idle-lane rows
    static constexpr int ROW = RowLen<T, N, false>::value;
    static constexpr int SW = RowLen<T, N, false>::sw;
    static constexpr int TOT = G * N;  // voxels per CTA
    static constexpr int PER = (TOT + kFastThreads - 1) / kFastThreads;
};

template <typename T, int N, int C>
constexpr size_t z_fast_smem(size_t extra) {
    typedef typename Cx<T>::t C2;
    typedef ZTile<T, N, C> Z;
    return (size_t)N * sizeof(C2) + (size_t)Z::SLOTS * Z::ROW * sizeof(C2) + 16 + 32 * 16 * sizeof(double) + extra;
}

// half-spectrum row length as stored: N/2 + 1 modes rounded up to even (the
// grid's Hzp for Nz = N), so pairs of modes are 16-byte (FP32) aligned
template <int N> struct HzOf {
    static constexpr int Hz = N / 2 + 1, Hzp = (Hz + 1) & ~1, P2 = Hzp / 2;
};

template <typename T, int N, int C>
constexpr size_t zinv_fast_smem(size_t extra) {
    return z_fast_smem<T, N, C>(extra) + 16 + (size_t)ZTile<T, N, C>::G * C * HzOf<N>::Hzp * sizeof(typename Cx<T>::t);
}

// two consecutive modes to global memory (one 16-byte store for FP32)
__device__ __forceinline__ void store_pair(float2* p, float2 a, float2 b) {
    *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void store_pair(double2* p, double2 a, double2 b) {
    p[0] = a;
    p[1] = b;
}
// asynchronous copy of two consecutive modes (zero-filled when !ok)
__device__ __forceinline__ void cp_async_pair(float2* dst, const float2* src, bool ok) {
    cp_async(dst, src, 16, ok ? 16 : 0);
}
__device__ __forceinline__ void cp_async_pair(double2* dst, const double2* src, bool ok) {
    cp_async(dst, src, 16, ok ? 16 : 0);
    cp_async(dst + 1, src + 1, 16, ok ? 16 : 0);
}

// transform the tile's complex lines in place (FWD: natural order in,
// natural-order spectrum out; !FWD: the inverse), each line's row doubling as
// its exchange buffer
template <typename C2, int N, int E, int TL, int SLOTS, int ROW, int SW, bool FWD>
__device__ __forceinline__ void z_tile_fft(C2* tile, const C2* tw) {
    constexpr int LPW = 32 / TL;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = lane % TL, lw = lane / TL;
    constexpr int NW = kFastThreads / 32;
#pragma unroll 1
    for (int l0 = warp * LPW; l0 < SLOTS; l0 += NW * LPW) {
        C2* row = tile + (l0 + lw) * ROW;
        const int sw = ((l0 + lw) & 1) * SW;  // odd tile rows are swizzled when SW
        C2 v[E];
        if constexpr (FWD) {
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = row[(t + TL * j) ^ sw];
            __syncwarp();
            line_fwd<C2, E, TL>(v, t, row, tw, sw);
#pragma unroll
            for (int r = 0; r < E; ++r) row[spec_mode<E, TL>(t, r) ^ sw] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = row[spec_mode<E, TL>(t, r) ^ sw];
            __syncwarp();
            line_inv<C2, E, TL>(v, t, row, tw, sw);
#pragma unroll
            for (int j = 0; j < E; ++j) row[(t + TL * j) ^ sw] = v[j];
        }
    }
}

template <typename T, int N, int C, class Pro>
__global__ void __launch_bounds__(kFastThreads, FastMinB<T, N, C>::value) k_zfwd_fast(GridDims g, const typename Cx<T>::t* __restrict__ twz,
                                                           typename Cx<T>::t* __restrict__ spec, Pro pro,
                                                           const Ctl* __restrict__ ctl) {
    typedef typename Cx<T>::t C2;
    typedef ZTile<T, N, C> Z;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
    pro.bind(b);
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* tile = tw + N;
    char* extra = align_up((char*)(tile + Z::SLOTS * Z::ROW), 16) + 32 * 16 * sizeof(double);
    const long long l0 = (long long)blockIdx.x * Z::G;
    // all prologue loads first: W consecutive voxels per load (kW of the operator)
    constexpr int W = Pro::kW;
    constexpr int NV = Z::TOT / W, PERW = (NV + kFastThreads - 1) / kFastThreads;
    typename PreOf<Pro>::type pre[PERW];
#pragma unroll
    for (int k = 0; k < PERW; ++k) {
        const int i = (threadIdx.x + k * kFastThreads) * W;
        const int gi = i / N, z = i - gi * N;
        if (i < Z::TOT && l0 + gi < g.NL) {
            if constexpr (W > 1) pre[k] = pro.loadw((l0 + gi) * N + z);
            else pre[k] = pro.load(b, (l0 + gi) * N + z);
        }
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twz[i];
    pro.load_smem(extra, b);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PERW; ++k) {
        const int i = (threadIdx.x + k * kFastThreads) * W;
        if (i >= Z::TOT) break;
        const int gi = i / N, z0 = i - gi * N;
        const long long l = l0 + gi;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const int z = z0 + w;
            T val[C];
            if (l < g.NL) {
                if constexpr (W > 1) pro.eval_prew(pre[k], w, val);
                else pro.eval_pre(pre[k], b, l * N + z, val);
            } else {
#pragma unroll
                for (int c = 0; c < C; ++c) val[c] = (T)0;
            }
#pragma unroll
            for (int cl = 0; cl < Z::NCL; ++cl) {
                const int rw = gi * Z::NCL + cl;
                tile[rw * Z::ROW + (z ^ ((rw & 1) * Z::SW))] =
                    mk<C2>(val[2 * cl], (2 * cl + 1 < C) ? val[2 * cl + 1] : (T)0);
            }
        }
    }
    __syncthreads();
    // Each warp transforms its tile rows (complex lines c0 + i c1 of voxel line
    // gi) and, without a block barrier, splits each row into the two
    // components' half spectra (Z[k] and Z[N-k] are in the same row) and
    // stores them, two modes per store.
    {
        constexpr int E = Z::E, TL = Z::TL, LPW = 32 / TL, NW = kFastThreads / 32;
        constexpr int Hz = HzOf<N>::Hz, Hzp = HzOf<N>::Hzp, P2 = HzOf<N>::P2;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int t = lane % TL, lw = lane / TL;
        C2* ob = spec + ((long long)b * C * g.NL + l0) * Hzp;
        const long long cst = g.NL * (long long)Hzp;
#pragma unroll 1
        for (int r0 = warp * LPW; r0 < Z::SLOTS; r0 += NW * LPW) {
            const int gl = r0 + lw;
            C2* row = tile + gl * Z::ROW;
            const int sw = (gl & 1) * Z::SW;
            C2 v[E];
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = row[(t + TL * j) ^ sw];
            __syncwarp();
            line_fwd<C2, E, TL>(v, t, row, tw, sw);
#pragma unroll
            for (int r = 0; r < E; ++r) row[spec_mode<E, TL>(t, r) ^ sw] = v[r];
            __syncwarp();
            const int gi = gl / Z::NCL, cl = gl - gi * Z::NCL;
            if (gl >= Z::G * Z::NCL || l0 + gi >= g.NL) continue;
            const bool two = 2 * cl + 1 < C;
            C2* oa = ob + (2 * cl) * cst + gi * Hzp;
#pragma unroll 1
            for (int k2 = t; k2 < P2; k2 += TL) {
                C2 ea[2], eb[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = 2 * k2 + h;
                    ea[h] = mk<C2>(0, 0);
                    eb[h] = mk<C2>(0, 0);
                    if (k < Hz) {
                        const C2 Zk = row[k ^ sw];
                        const C2 Zm = row[(k == 0 ? 0 : N - k) ^ sw];
                        ea[h] = mk<C2>((T)0.5 * (Zk.x + Zm.x), (T)0.5 * (Zk.y - Zm.y));
                        eb[h] = mk<C2>((T)0.5 * (Zk.y + Zm.y), (T)-0.5 * (Zk.x - Zm.x));
                    }
                }
                store_pair(oa + 2 * k2, ea[0], ea[1]);
                if (two) store_pair(oa + cst + 2 * k2, eb[0], eb[1]);
            }
        }
    }
}

// Epilogue items per thread loaded before the z inverse's transform (the
// rest after it).  The six-component EM update: one (a 96-point FP32 tile
// holds two per thread), so that the kernel fits the 168 registers of three
// CTAs per SM.
#ifndef M3D_ZINV_PF6
#define M3D_ZINV_PF6 1
#endif
#ifndef M3D_ZINV_PF6_64
#define M3D_ZINV_PF6_64 1
#endif
template <class Epi, class = void> struct EpiIsJ2 { static constexpr bool value = false; };
template <class Epi> struct EpiIsJ2<Epi, decltype((void)Epi::kJ2, void())> { static constexpr bool value = true; };
// epilogues that load each next item while the current one is processed
template <class Epi, class = void> struct EpiRolling { static constexpr bool value = false; };
template <class Epi> struct EpiRolling<Epi, decltype((void)Epi::kRolling, void())> {
    static constexpr bool value = Epi::kRolling;
};
template <typename T, int C, class Epi> struct ZinvPrefetch {
    static constexpr int value =
        std::is_same<Epi, EpiEM<T, 6>>::value ? (sizeof(T) == 4 ? M3D_ZINV_PF6 : M3D_ZINV_PF6_64)
                                              : (EpiIsJ2<Epi>::value ? 1 : 64);
};

// CTAs per SM of the z inverse: FastMinB, and three for the six-component
// EM update of the elastic sweeps (uncapped it takes 250-255 registers, two
// CTAs per SM; capped at 168 it spills 0-16 bytes, and the batch workload's
// z inverse runs 20-28% faster; FP64 only up to N = 64, where the cap does
// not spill more than 16 bytes).
#ifndef M3D_F32C6_MINB
#define M3D_F32C6_MINB 3
#endif
#ifndef M3D_F64C6_MINB
#define M3D_F64C6_MINB 3
#endif
// CTAs per SM of the inelastic update's z inverse in FP32 (1: uncapped, 180
// registers; a 168-register cap for three CTAs timed 2202-2458 us per 256^3
// launch against 2256-2274 us uncapped, no reliable gain).  FP64 keeps its
// 240 registers for the rolling prefetch (a 168 cap spills 2.4 KB).
#ifndef M3D_J2_MINB
#define M3D_J2_MINB 1
#endif
template <typename T, int N, int C, class Epi> struct ZinvMinB {
    static constexpr int value = std::is_same<Epi, EpiEM<T, 6>>::value
                                     ? (sizeof(T) == 4 ? M3D_F32C6_MINB : (N <= 64 ? M3D_F64C6_MINB : 1))
                                     : (EpiIsJ2<Epi>::value ? (sizeof(T) == 4 ? M3D_J2_MINB : 1)
                                                            : FastMinB<T, N, C>::value);
};

template <typename T, int N, int C, class Epi, class Fin>
__global__ void __launch_bounds__(kFastThreads, ZinvMinB<T, N, C, Epi>::value) k_zinv_fast(GridDims g, const typename Cx<T>::t* __restrict__ twz,
                                                           const typename Cx<T>::t* __restrict__ spec, Epi epi,
                                                           Ctl* ctl, double* partials, Fin fin) {
    typedef typename Cx<T>::t C2;
    typedef ZTile<T, N, C> Z;
    const int b = entry_of(g, blockIdx.y);
    if (b < 0 || ctl[b].done) return;
    epi.bind(b);
    extern __shared__ __align__(16) char smem_raw[];
    C2* tw = (C2*)smem_raw;
    C2* tile = tw + N;
    constexpr int Hzp = HzOf<N>::Hzp, P2 = HzOf<N>::P2;
    C2* raw = (C2*)align_up((char*)(tile + Z::SLOTS * Z::ROW), 16);  // [gi][c][Hzp] half spectra as stored
    double* red = (double*)align_up((char*)(raw + Z::G * C * Hzp), 16);
    char* extra = (char*)red + 32 * 16 * sizeof(double);
    const long long l0 = (long long)blockIdx.x * Z::G;
    // asynchronous copies of the G x C half-spectrum rows, two modes per copy
    {
        const C2* ib = spec + ((long long)b * C * g.NL + l0) * Hzp;
        const long long cst = g.NL * (long long)Hzp;
        for (int i = threadIdx.x; i < Z::G * C * P2; i += kFastThreads) {
            const int k2 = i % P2, gc = i / P2;
            const int gi = gc / C, c = gc - gi * C;
            const bool okl = l0 + gi < g.NL;
            cp_async_pair(raw + gc * Hzp + 2 * k2, okl ? ib + c * cst + gi * Hzp + 2 * k2 : ib, okl);
        }
    }
    // epilogue loads do not depend on the transform: issue the first PF of
    // them meanwhile, the rest after it
    constexpr int W = Epi::kW;
    constexpr int NV = Z::TOT / W, PERW = (NV + kFastThreads - 1) / kFastThreads;
    constexpr int PF = Epi::kPrefetch ? (ZinvPrefetch<T, C, Epi>::value < PERW ? ZinvPrefetch<T, C, Epi>::value : PERW) : 0;
    typename PreOf<Epi>::type pre[PF > 0 ? PF : 1];
    if constexpr (PF > 0) {
#pragma unroll
        for (int k = 0; k < PF; ++k) {
            const int i = (threadIdx.x + k * kFastThreads) * W;
            const int gi = i / N, z = i - gi * N;
            if (i < Z::TOT && l0 + gi < g.NL) {
                if constexpr (W > 1) pre[k] = epi.loadw((l0 + gi) * N + z);
                else pre[k] = epi.load(b, (l0 + gi) * N + z);
            }
        }
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twz[i];
    epi.load_smem(extra, b);
    cp_async_wait_all();
    __syncthreads();
    // Inverse transform of each complex line (components 2cl + i (2cl+1) of
    // voxel line gi); its spectrum is assembled from the two stored half
    // spectra as the lanes load it (Hermitian extension; the imaginary parts of
    // the k = 0 and k = N/2 modes are dropped, as FFTW's c2r does).  The line's
    // tile row is the exchange buffer and receives the natural-order result.
    {
        constexpr int E = Z::E, TL = Z::TL, LPW = 32 / TL, NW = kFastThreads / 32;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int t = lane % TL, lw = lane / TL;
#pragma unroll 1
        for (int r0 = warp * LPW; r0 < Z::SLOTS; r0 += NW * LPW) {
            const int gl = r0 + lw;
            C2* row = tile + gl * Z::ROW;
            const int sw = (gl & 1) * Z::SW;
            const bool live = gl < Z::G * Z::NCL;
            const int gi = gl / Z::NCL, cl = gl - gi * Z::NCL;
            const bool hasb = live && (2 * cl + 1 < C);
            const C2* ra = raw + (live ? (gi * C + 2 * cl) * Hzp : 0);
            const C2* rb = raw + (hasb ? (gi * C + 2 * cl + 1) * Hzp : 0);
            C2 v[E];
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int k = spec_mode<E, TL>(t, r);
                const bool lo = 2 * k <= N;
                const int kk = lo ? k : N - k;
                const C2 a = live ? ra[kk] : mk<C2>(0, 0);
                const C2 q = hasb ? rb[kk] : mk<C2>(0, 0);
                if (kk == 0 || 2 * kk == N) v[r] = mk<C2>(a.x, q.x);
                else if (lo) v[r] = mk<C2>(a.x - q.y, a.y + q.x);
                else v[r] = mk<C2>(a.x + q.y, q.x - a.y);
            }
            line_inv<C2, E, TL>(v, t, row, tw, sw);
#pragma unroll
            for (int j = 0; j < E; ++j) row[(t + TL * j) ^ sw] = v[j];
        }
    }
    __syncthreads();
    const T invV = (T)(1.0 / (double)g.V);
    double acc[Epi::NSUM > 0 ? Epi::NSUM : 1] = {};
    constexpr bool ROLL = W == 1 && Epi::kPrefetch && EpiRolling<Epi>::value && PF < PERW;
    typename PreOf<Epi>::type roll;  // rolling epilogues: the next item's inputs
    if constexpr (ROLL) {
        const int i = (threadIdx.x + PF * kFastThreads) * W;
        const int gi = i / N;
        if (i < Z::TOT && l0 + gi < g.NL) roll = epi.load(b, (l0 + gi) * N + (i - gi * N));
    }
#pragma unroll
    for (int k = 0; k < PERW; ++k) {
        const int i = (threadIdx.x + k * kFastThreads) * W;
        if (i >= Z::TOT) break;
        const int gi = i / N, z0 = i - gi * N;
        const long long l = l0 + gi;
        typename PreOf<Epi>::type cur;
        if constexpr (ROLL) {
            if (k >= PF) {
                cur = roll;
                const int i1 = i + kFastThreads * W;
                const int g1 = i1 / N;
                if (k + 1 < PERW && i1 < Z::TOT && l0 + g1 < g.NL) roll = epi.load(b, (l0 + g1) * N + (i1 - g1 * N));
            }
        }
        if (l >= g.NL) continue;
        T xc[W][C];
#pragma unroll
        for (int w = 0; w < W; ++w) {
#pragma unroll
            for (int cl = 0; cl < Z::NCL; ++cl) {
                const int rw = gi * Z::NCL + cl;
                const C2 u = tile[rw * Z::ROW + ((z0 + w) ^ ((rw & 1) * Z::SW))];
                xc[w][2 * cl] = u.x * invV;
                if (2 * cl + 1 < C) xc[w][2 * cl + 1] = u.y * invV;
            }
        }
        if constexpr (W > 1) {
            if (k < PF) epi.apply_prew(pre[k < PF ? k : 0], l * N + z0, xc, acc);
            else epi.apply_prew(epi.loadw(l * N + z0), l * N + z0, xc, acc);
        } else if constexpr (Epi::kPrefetch) {
            if (k < PF) epi.apply_pre(pre[k < PF ? k : 0], b, l * N + z0, xc[0], acc);
            else if constexpr (ROLL) epi.apply_pre(cur, b, l * N + z0, xc[0], acc);
            else epi.apply_pre(epi.load(b, l * N + z0), b, l * N + z0, xc[0], acc);
        } else {
            epi.apply(b, l * N + z0, xc[0], acc);
        }
    }
    if constexpr (Epi::NSUM > 0) {
        block_reduce_store<Epi::NSUM>(acc, red, partials, b, gridDim.x, blockIdx.x);
        fused_finalize(fin, ctl, partials, Epi::NSUM, b);
    }
}


// ---------------------------------------------------------------------------
// TMA-staged y pass.  A tile is KC = 4*CPW consecutive kz columns of all Ny
// rows of one (batch*comp, x) plane: TMA copies it into shared memory as
// 128-byte-wide boxes with the 128-byte swizzle (16-byte chunk index XOR
// row mod 8, which makes the column reads of the line FFT conflict-free),
// the warps transform the columns in place, and TMA stores the tile back.
// Persistent CTAs walk the tiles with kYStages tiles in flight, so the copies
// of the next tiles overlap the transforms of the current one.
// ---------------------------------------------------------------------------
constexpr int kYStages = 2;

template <typename T, int N>
struct YTma {
    typedef typename Cx<T>::t C2;
    static constexpr int E = LineSplit<T, N>::E, TL = LineSplit<T, N>::Tl, CPW = 32 / TL, KC = 4 * CPW;
    static constexpr int CPB = 128 / (int)sizeof(C2);  // columns per 128-byte box row
    static constexpr int NB = KC / CPB;                // boxes per tile
    static constexpr int BOXE = 128 / (int)sizeof(T);  // box width in scalars
    static constexpr int STAGE = NB * N * 128;         // bytes per tile
    static constexpr int XS = RowLen<T, N, false>::value, SWX = RowLen<T, N, false>::sw;
    static_assert(KC % CPB == 0, "a tile is a whole number of boxes");
    static constexpr size_t smem() {
        return 1024 + (size_t)kYStages * STAGE + (size_t)N * sizeof(C2) + (size_t)KC * XS * sizeof(C2) + 8 +
               kYStages * sizeof(uint64_t);
    }
    // byte offset of (column, row) in a tile
    static __device__ __forceinline__ int off(int col, int y) {
        const int box = col / CPB, cib = col - box * CPB;
        if constexpr (sizeof(C2) == 8)
            return box * N * 128 + y * 128 + ((((cib >> 1) ^ (y & 7)) << 4) | ((cib & 1) << 3));
        else
            return box * N * 128 + y * 128 + ((cib ^ (y & 7)) << 4);
    }
};

template <typename T, int N, int SIGN>
__global__ void __launch_bounds__(kFastThreads) k_ypass_tma(const __grid_constant__ CUtensorMap map, GridDims g,
                                                           const typename Cx<T>::t* __restrict__ twy, int C, int ntiles,
                                                           const Ctl* __restrict__ ctl, int* err) {
    typedef typename Cx<T>::t C2;
    typedef YTma<T, N> Y;
    constexpr int E = Y::E, TL = Y::TL, CPW = Y::CPW, S = kYStages;
    extern __shared__ __align__(16) char smem_raw[];
    char* stage = align_up(smem_raw, 1024);
    C2* tw = (C2*)(stage + S * Y::STAGE);
    C2* xch = tw + N;
    uint64_t* full = (uint64_t*)align_up((char*)(xch + Y::KC * Y::XS), 8);
    const int ntz = (g.Hzp + Y::KC - 1) / Y::KC;
    const int per_cb = g.Nx * ntz;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twy[i];
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // the tiles of this CTA whose entry is still iterating, in order
    auto next = [&](int id) {
        for (; id < ntiles; id += gridDim.x) {
            const int b = entry_of(g, (id / per_cb) / C);
            if (b >= 0 && !ctl[b].done) return id;
        }
        return -1;
    };
    auto coords = [&](int id, int& c0, int& r0) {
        const int scb = id / per_cb, rem = id - scb * per_cb;  // (entry slot, component), then (x, kz tile)
        const int cb = entry_of(g, scb / C) * C + scb % C;
        const int x = rem / ntz, kzt = rem - x * ntz;
        r0 = (cb * g.Nx + x) * N;
        c0 = 2 * kzt * Y::KC;
    };
    auto issue = [&](int id, int s) {
        int c0, r0;
        coords(id, c0, r0);
        mbar_expect_tx(&full[s], Y::STAGE);
#pragma unroll
        for (int nb = 0; nb < Y::NB; ++nb) tma_load_2d(stage + s * Y::STAGE + nb * N * 128, &map, c0 + nb * Y::BOXE, r0, &full[s]);
    };
    int pid = -1;
    if (threadIdx.x == 0) {
        pid = next(blockIdx.x);
        for (int s = 0; s < S && pid >= 0; ++s) {
            issue(pid, s);
            pid = next(pid + gridDim.x);
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = lane % TL, col = warp * CPW + lane / TL;
    C2* xl = xch + col * Y::XS;
    const int sw = (col & 1) * Y::SWX;
    int it = 0;
    for (int id = next(blockIdx.x); id >= 0; id = next(id + gridDim.x), ++it) {
        const int s = it % S;
        const bool ok = mbar_wait(&full[s], (uint32_t)((it / S) & 1), err);
        if (__syncthreads_or(!ok)) break;
        char* tile = stage + s * Y::STAGE;
        C2 v[E];
        if constexpr (SIGN < 0) {
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = *(const C2*)(tile + Y::off(col, t + TL * j));
            line_fwd<C2, E, TL>(v, t, xl, tw, sw);
#pragma unroll
            for (int r = 0; r < E; ++r) *(C2*)(tile + Y::off(col, spec_mode<E, TL>(t, r))) = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = *(const C2*)(tile + Y::off(col, spec_mode<E, TL>(t, r)));
            line_inv<C2, E, TL>(v, t, xl, tw, sw);
#pragma unroll
            for (int j = 0; j < E; ++j) *(C2*)(tile + Y::off(col, t + TL * j)) = v[j];
        }
        fence_proxy_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            int c0, r0;
            coords(id, c0, r0);
#pragma unroll
            for (int nb = 0; nb < Y::NB; ++nb) tma_store_2d(&map, c0 + nb * Y::BOXE, r0, tile + nb * N * 128);
            bulk_commit();
            bulk_wait_read0();  // the stage may be refilled once the store has read it
            if (pid >= 0) {
                issue(pid, s);
                pid = next(pid + gridDim.x);
            }
        }
    }
    if (threadIdx.x == 0) bulk_wait0();
    (void)CPW;
}

}  // namespace m3d
