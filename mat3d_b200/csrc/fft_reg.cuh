// fft_reg.cuh -- compile-time-sized FFT of one line spread over T lanes of a warp.
//
// A line of N = E*T points is transformed by the four-step split
//     X[k1 + E k2] = sum_t w_T^(t k2) w_N^(t k1) sum_j w_E^(j k1) x[t + T j]
// Lane t of the line holds E points in registers:
//   natural distribution : v[j]          = x[t + T j],            j < E
//   spectral distribution: v[q*T + k2]   = X[(t*Q + q) + E k2],   q < Q = E/T, k2 < T
// line_fwd maps natural -> spectral: a radix-E DFT in registers, the w_N
// twiddles, one exchange through shared memory among the T lanes of the line
// (warp-synchronous, no block barrier), and Q radix-T DFTs in registers.
// line_inv is the transposed algorithm and maps spectral -> natural, so a
// forward + pointwise + inverse sequence needs no reordering at all.
// The in-register DFTs are mixed-radix (2, 3, 4, 5, 8) decimation in time
// with every index a compile-time constant; twiddles are read from the
// per-line table tw[m] = exp(-2 pi i m / N) held in shared memory.
#pragma once
#include "fft_smem.cuh"

namespace m3d {

// DFT of compile-time length L in registers; w_L^m = tw[m * (NL/L)].
template <typename C2, int L, int NL>
__device__ __forceinline__ void dft_reg(C2 (&v)[L], const C2* tw, int sign) {
    static_assert(NL % L == 0, "sub-DFT length must divide the table length");
    if constexpr (L == 1) {
        return;
    } else if constexpr (L == 2 || L == 3 || L == 4 || L == 5 || L == 8) {
        dft_small<C2, L>(v, tw, NL, sign);
    } else {
        constexpr int P = (L % 4 == 0) ? 4 : ((L % 2 == 0) ? 2 : ((L % 3 == 0) ? 3 : 5));
        constexpr int Q = L / P;
        constexpr int st = NL / L;
        C2 sub[P][Q];
#pragma unroll
        for (int p = 0; p < P; ++p)
#pragma unroll
            for (int m = 0; m < Q; ++m) sub[p][m] = v[P * m + p];
#pragma unroll
        for (int p = 0; p < P; ++p) dft_reg<C2, Q, NL>(sub[p], tw, sign);
#pragma unroll
        for (int p = 1; p < P; ++p)
#pragma unroll
            for (int k1 = 1; k1 < Q; ++k1) sub[p][k1] = cmul(sub[p][k1], twid(tw, p * k1 * st, sign));
#pragma unroll
        for (int k1 = 0; k1 < Q; ++k1) {
            C2 t[P];
#pragma unroll
            for (int p = 0; p < P; ++p) t[p] = sub[p][k1];
            dft_small<C2, P>(t, tw, NL, sign);
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) v[k1 + Q * k2] = t[k2];
        }
    }
}

// Line split for each supported length and element type: N = E * T, T | E,
// T lanes per line (so 32/T lines per warp).
template <typename T, int N> struct LineSplit;
#define M3D_SPLIT(TY, NN, EE, TT) \
    template <> struct LineSplit<TY, NN> { static constexpr int E = EE, Tl = TT; };
M3D_SPLIT(float, 16, 4, 4)
M3D_SPLIT(float, 32, 8, 4)
M3D_SPLIT(float, 48, 12, 4)
M3D_SPLIT(float, 64, 8, 8)
M3D_SPLIT(float, 96, 24, 4)
M3D_SPLIT(float, 128, 16, 8)
M3D_SPLIT(float, 256, 32, 8)
M3D_SPLIT(double, 16, 4, 4)
M3D_SPLIT(double, 32, 8, 4)
M3D_SPLIT(double, 48, 12, 4)
M3D_SPLIT(double, 64, 8, 8)
M3D_SPLIT(double, 96, 24, 4)
M3D_SPLIT(double, 128, 16, 8)
M3D_SPLIT(double, 256, 16, 16)
#undef M3D_SPLIT

constexpr bool fast_size(int n) {
    return n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 256;
}

// exchange buffer of one line: element (k1, t) at k1*(T+1) + t
template <int E, int T> struct Xch { static constexpr int size = E * (T + 1) + 1; };

// Exchange element (k1, t) lives at k1*(T+1) + (t ^ sw); `sw` (0 or 1) is a
// per-line bank swizzle chosen with the row padding (BankCfg in
// passes_fast.cuh) so that the natural, spectral and both exchange access
// patterns of a warp are conflict-free.
template <typename C2, int E, int T>
__device__ __forceinline__ void line_fwd(C2 (&v)[E], int t, C2* xch, const C2* tw, int sw = 0) {
    constexpr int N = E * T, Q = E / T;
    dft_reg<C2, E, N>(v, tw, -1);
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) v[k1] = cmul(v[k1], twid(tw, t * k1, -1));
    const int ts = t ^ sw;
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) xch[k1 * (T + 1) + ts] = v[k1];
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        C2 u[T];
#pragma unroll
        for (int t2 = 0; t2 < T; ++t2) u[t2] = xch[(t * Q + q) * (T + 1) + (t2 ^ sw)];
        dft_reg<C2, T, N>(u, tw, -1);
#pragma unroll
        for (int k2 = 0; k2 < T; ++k2) v[q * T + k2] = u[k2];
    }
    __syncwarp();
}

template <typename C2, int E, int T>
__device__ __forceinline__ void line_inv(C2 (&v)[E], int t, C2* xch, const C2* tw, int sw = 0) {
    constexpr int N = E * T, Q = E / T;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        C2 u[T];
#pragma unroll
        for (int k2 = 0; k2 < T; ++k2) u[k2] = v[q * T + k2];
        dft_reg<C2, T, N>(u, tw, +1);
        const int k1 = t * Q + q;
#pragma unroll
        for (int t2 = 0; t2 < T; ++t2) {
            const C2 w = (t2 == 0) ? u[t2] : cmul(u[t2], twid(tw, t2 * k1, +1));
            xch[k1 * (T + 1) + (t2 ^ sw)] = w;
        }
    }
    __syncwarp();
    const int ts = t ^ sw;
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) v[k1] = xch[k1 * (T + 1) + ts];
    __syncwarp();
    dft_reg<C2, E, N>(v, tw, +1);
}

// mode index held in v[r] (spectral distribution) by lane t
template <int E, int T>
__device__ __forceinline__ int spec_mode(int t, int r) {
    constexpr int Q = E / T;
    return (t * Q + r / T) + E * (r % T);
}

}  // namespace m3d
