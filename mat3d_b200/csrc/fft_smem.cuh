// fft_smem.cuh -- mixed-radix Stockham FFT stages on lines held in shared memory.
//
// A CTA holds a set of complex lines in shared memory and transforms all of
// them cooperatively: in each stage every thread loops over (line, butterfly)
// work items, reads R inputs from buffer `a`, applies the stage twiddles, does
// an R-point DFT in registers and writes R outputs to buffer `b` (autosort, so
// the result is in natural order without a bit-reversal pass).  Stage s with
// radix R and Ns = product of the previous radices:
//     v[r]  = a[j + r*(n/R)]                    r = 0..R-1, j = 0..n/R-1
//     v[r] *= w_n^( (j mod Ns) * r * n/(Ns*R) )
//     v     = DFT_R(v)
//     b[(j/Ns)*Ns*R + (j mod Ns) + r*Ns] = v[r]
// Twiddles come from a per-length table tw[m] = exp(-2 pi i m / n) in shared
// memory (computed on the host in long double); the inverse uses conj().
// Radices 2, 3, 4, 5 and 8 have dedicated butterflies; any other factor
// (e.g. 13 for n = 65) uses a direct O(R^2) DFT through the table.
//
// Line addressing is two-level so one routine serves every pass layout:
//     element e of line L lives at  (L / lpg) * gstride + (L % lpg) * lstride + e * estride
// and `lines_fast` chooses whether consecutive threads walk lines (column
// tiles: consecutive columns are consecutive words, no bank conflicts) or
// butterflies (contiguous lines).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace m3d {

constexpr int kMaxStages = 12;

struct LinePlan {
    int n;
    int nstages;
    int radix[kMaxStages];
};

template <typename T> struct Cx;
template <> struct Cx<float> { typedef float2 t; };
template <> struct Cx<double> { typedef double2 t; };

template <typename C2> __device__ __forceinline__ C2 mk(decltype(C2().x) re, decltype(C2().x) im) {
    C2 r; r.x = re; r.y = im; return r;
}
template <typename C2> __device__ __forceinline__ C2 cadd(C2 a, C2 b) { return mk<C2>(a.x + b.x, a.y + b.y); }
template <typename C2> __device__ __forceinline__ C2 csub(C2 a, C2 b) { return mk<C2>(a.x - b.x, a.y - b.y); }
template <typename C2> __device__ __forceinline__ C2 cmul(C2 a, C2 b) {
    return mk<C2>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by -i (sign < 0) or +i (sign > 0)
template <typename C2> __device__ __forceinline__ C2 crot(C2 a, int sign) {
    return sign < 0 ? mk<C2>(a.y, -a.x) : mk<C2>(-a.y, a.x);
}
template <typename C2> __device__ __forceinline__ C2 twid(const C2* tw, int m, int sign) {
    C2 w = tw[m];
    if (sign > 0) w.y = -w.y;
    return w;
}

// x / d for 0 <= x, 1 <= d with x * d < 2^32 (always true for indices of a
// shared-memory tile): round-up reciprocal m = ceil(2^32 / d), q = hi32(x m).
// The error of x m / 2^32 against x / d is below x / 2^32 < 1 / d, too small
// to carry the quotient past the next integer.
struct FastDiv {
    unsigned m;
    int d;
    __device__ __forceinline__ void init(int dd) {
        d = dd;
        m = dd > 1 ? 0xFFFFFFFFu / (unsigned)dd + 1u : 0u;
    }
    __device__ __forceinline__ int div(int x) const { return d == 1 ? x : (int)__umulhi((unsigned)x, m); }
};

// per-stage constants shared by every butterfly of a Stockham stage
struct StageIdx {
    int nb;    // n / R: butterflies per line, and the input stride
    int Ns;    // product of the earlier radices
    int step;  // n / (Ns R): twiddle index step
};

template <typename C2, int R>
__device__ __forceinline__ void dft_small(C2 (&v)[R], const C2* tw, int n, int sign) {
    typedef decltype(C2().x) T;
    if constexpr (R == 2) {
        C2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        C2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        C2 b0 = cadd(v[1], v[3]), b1 = crot(csub(v[1], v[3]), sign);
        v[0] = cadd(a0, b0);
        v[1] = cadd(a1, b1);
        v[2] = csub(a0, b0);
        v[3] = csub(a1, b1);
    } else if constexpr (R == 8) {
        const T h = (T)0.70710678118654752440084436210484903928483593768847L;
        // radix-2 across halves, then two radix-4 on even/odd outputs
        C2 e[4], o[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            e[r] = cadd(v[r], v[r + 4]);
            o[r] = csub(v[r], v[r + 4]);
        }
        // o[r] *= w^r with w = exp(sign * i pi / 4) = (h, sg*h)
        const T sg = (T)sign;
        {
            const T x = o[1].x, y = o[1].y;
            o[1] = mk<C2>(h * (x - sg * y), h * (y + sg * x));
        }
        o[2] = crot(o[2], sign);
        {
            // w^3 = (-h, sg*h)
            const T x = o[3].x, y = o[3].y;
            o[3] = mk<C2>(h * (-x - sg * y), h * (sg * x - y));
        }
        // radix-4 on e -> outputs 0,2,4,6 ; on o -> outputs 1,3,5,7
        C2 a0 = cadd(e[0], e[2]), a1 = csub(e[0], e[2]);
        C2 b0 = cadd(e[1], e[3]), b1 = crot(csub(e[1], e[3]), sign);
        C2 c0 = cadd(o[0], o[2]), c1 = csub(o[0], o[2]);
        C2 d0 = cadd(o[1], o[3]), d1 = crot(csub(o[1], o[3]), sign);
        v[0] = cadd(a0, b0);
        v[4] = csub(a0, b0);
        v[2] = cadd(a1, b1);
        v[6] = csub(a1, b1);
        v[1] = cadd(c0, d0);
        v[5] = csub(c0, d0);
        v[3] = cadd(c1, d1);
        v[7] = csub(c1, d1);
    } else if constexpr (R == 3) {
        const T c = (T)-0.5L;
        const T s = (T)0.86602540378443864676372317075293618347140262690519L * (T)(sign < 0 ? -1 : 1);
        C2 a = v[0], b = v[1], d = v[2];
        C2 t1 = cadd(b, d);
        C2 t2 = mk<C2>(a.x + c * t1.x, a.y + c * t1.y);
        C2 t3 = csub(b, d);  // times i*s
        C2 t3r = mk<C2>(-s * t3.y, s * t3.x);
        v[0] = cadd(a, t1);
        v[1] = cadd(t2, t3r);
        v[2] = csub(t2, t3r);
    } else {
        // direct DFT through the table: w_R^m = tw[m * (n/R)]
        C2 in[R];
#pragma unroll
        for (int q = 0; q < R; ++q) in[q] = v[q];
        const int st = n / R;
#pragma unroll
        for (int s = 0; s < R; ++s) {
            C2 acc = in[0];
#pragma unroll
            for (int q = 1; q < R; ++q) acc = cadd(acc, cmul(in[q], twid(tw, ((q * s) % R) * st, sign)));
            v[s] = acc;
        }
    }
}

// butterfly j of a stage: inputs j + r nb, twiddles w^(k r step) with
// j = g Ns + k, outputs g Ns R + k + r Ns
template <typename C2, int R>
__device__ __forceinline__ void butterfly(const C2* __restrict__ src, C2* __restrict__ dst, int j, int g, int k,
                                          const StageIdx& S, int es, const C2* tw, int sign) {
    C2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * S.nb) * es];
    if (S.Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid(tw, k * r * S.step, sign));
    }
    dft_small<C2, R>(v, tw, S.nb * R, sign);
    const int idx = g * S.Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(idx + r * S.Ns) * es] = v[r];
}

// Odd radix R >= 5, compile time: inputs j and R-j are paired
// (a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j}) so outputs k and R-k share one set
// of products:
//   y_k, y_{R-k} = x_0 + sum_j a_j cos(2 pi jk/R) +- i sign sum_j b_j sin(2 pi jk/R)
// -- (R-1)^2 real multiply-adds per butterfly instead of the 4 R^2 of a direct
// DFT.  Outputs go straight to `dst`, so only a, b and the h = (R-1)/2 cosines
// and sines (from the table: tw[m n/R] = (cos, -sin) of 2 pi m/R) live in
// registers.
template <typename C2, int R>
__device__ __forceinline__ void butterfly_odd(const C2* __restrict__ src, C2* __restrict__ dst, int j, int g, int k0,
                                              const StageIdx& S, int es, const C2* tw, int sign) {
    typedef decltype(C2().x) T;
    constexpr int h = (R - 1) / 2;
    const int nb = S.nb, Ns = S.Ns, step = S.step;
    const C2 x0 = src[j * es];
    C2 a[h], b[h];
#pragma unroll
    for (int q = 1; q <= h; ++q) {
        C2 u = src[(j + q * nb) * es], w = src[(j + (R - q) * nb) * es];
        if (Ns > 1) {
            u = cmul(u, twid(tw, k0 * q * step, sign));
            w = cmul(w, twid(tw, k0 * (R - q) * step, sign));
        }
        a[q - 1] = cadd(u, w);
        b[q - 1] = csub(u, w);
    }
    T c[h], sn[h];
#pragma unroll
    for (int m = 1; m <= h; ++m) {
        const C2 w = tw[m * nb];
        c[m - 1] = w.x;
        sn[m - 1] = sign < 0 ? w.y : -w.y;  // sign * sin(2 pi m / R)
    }
    const int idx = g * Ns * R + k0;
    C2 y0 = x0;
#pragma unroll
    for (int q = 0; q < h; ++q) y0 = cadd(y0, a[q]);
    dst[idx * es] = y0;
#pragma unroll
    for (int k = 1; k <= h; ++k) {
        T px = x0.x, py = x0.y, qx = 0, qy = 0;
#pragma unroll
        for (int q = 1; q <= h; ++q) {
            const int m = (q * k) % R;  // 0 only for a composite R (e.g. 3 * 3 for R = 9)
            const T cc = m == 0 ? (T)1 : (m <= h ? c[m - 1] : c[R - m - 1]);
            const T ss = m == 0 ? (T)0 : (m <= h ? sn[m - 1] : -sn[R - m - 1]);
            px += a[q - 1].x * cc;
            py += a[q - 1].y * cc;
            qx += b[q - 1].x * ss;
            qy += b[q - 1].y * ss;
        }
        dst[(idx + k * Ns) * es] = mk<C2>(px - qy, py + qx);
        dst[(idx + (R - k) * Ns) * es] = mk<C2>(px + qy, py - qx);
    }
}

// generic-radix butterfly (any R up to kMaxGenericRadix), run-time R
constexpr int kMaxGenericRadix = 32;
template <typename C2>
__device__ __noinline__ void butterfly_generic(const C2* __restrict__ src, C2* __restrict__ dst, int R, int j, int g,
                                               int k, StageIdx S, int es, const C2* tw, int sign) {
    typedef decltype(C2().x) T;
    const int nb = S.nb, Ns = S.Ns, step = S.step;
    C2 v[kMaxGenericRadix];
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * es];
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid(tw, k * r * step, sign));
    const int st = nb;
    const int idx = g * Ns * R + k;
    for (int s = 0; s < R; ++s) {
        C2 acc = v[0];
        for (int q = 1; q < R; ++q) acc = cadd(acc, cmul(v[q], twid(tw, ((q * s) % R) * st, sign)));
        dst[(idx + s * Ns) * es] = acc;
    }
    (void)sizeof(T);
}

struct LineLayout {
    int nlines;   // number of lines
    int lpg;      // lines per group
    int lstride;  // stride between lines inside a group
    int gstride;  // stride between groups
    int estride;  // stride between elements of a line
    bool lines_fast;
};

// Transforms every line; returns the buffer (a or b) that holds the result.
// Must be called by all threads of the CTA; ends with __syncthreads().
// Radices 2, 3, 4, 5, 8 are compile-time butterflies; odd radices 7..MaxR
// (the primes and 9) are compile-time too when MaxR reaches them (each adds registers to the
// kernel, so callers pick the smallest MaxR their lengths need); any other
// radix runs the run-time generic butterfly.
// one Stockham stage of radix R over every line of the tile (R fixed at
// compile time, so the loop body is one straight-line butterfly); KIND 0 =
// butterfly (2, 3, 4, 8), 1 = butterfly_odd, 2 = run-time generic
template <typename C2, int R, int KIND>
__device__ __forceinline__ void run_stage(const C2* a, C2* b, const C2* tw, const StageIdx& S, int Rrt,
                                          const LineLayout& L, const FastDiv& dl, const FastDiv& dg, int sign) {
    FastDiv dnb, dns;
    dnb.init(S.nb);
    dns.init(S.Ns);
    const int total = S.nb * L.nlines;
    const int es = L.estride;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        int line, j;
        if (L.lines_fast) { j = dl.div(w); line = w - j * L.nlines; }
        else { line = dnb.div(w); j = w - line * S.nb; }
        const int grp = dg.div(line);
        const int base = grp * L.gstride + (line - grp * L.lpg) * L.lstride;
        const int g = dns.div(j), k = j - g * S.Ns;
        if constexpr (KIND == 0) butterfly<C2, R>(a + base, b + base, j, g, k, S, es, tw, sign);
        else if constexpr (KIND == 1) butterfly_odd<C2, R>(a + base, b + base, j, g, k, S, es, tw, sign);
        else butterfly_generic<C2>(a + base, b + base, Rrt, j, g, k, S, es, tw, sign);
    }
}

template <typename C2, int MaxR = 5>
__device__ C2* fft_lines(C2* a, C2* b, const C2* tw, const LinePlan& p, const LineLayout& L, int sign) {
    const int n = p.n;
    FastDiv dl, dg;  // by the lines of the tile, by the lines of a group
    dl.init(L.nlines);
    dg.init(L.lpg);
    int Ns = 1;
    for (int s = 0; s < p.nstages; ++s) {
        const int R = p.radix[s];
        StageIdx S;
        S.nb = n / R;
        S.Ns = Ns;
        S.step = S.nb / Ns;
        switch (R) {
            case 2: run_stage<C2, 2, 0>(a, b, tw, S, R, L, dl, dg, sign); break;
            case 3: run_stage<C2, 3, 0>(a, b, tw, S, R, L, dl, dg, sign); break;
            case 4: run_stage<C2, 4, 0>(a, b, tw, S, R, L, dl, dg, sign); break;
            case 5: run_stage<C2, 5, 1>(a, b, tw, S, R, L, dl, dg, sign); break;
            case 8: run_stage<C2, 8, 0>(a, b, tw, S, R, L, dl, dg, sign); break;
            default:
                if constexpr (MaxR >= 7) if (R == 7) { run_stage<C2, 7, 1>(a, b, tw, S, R, L, dl, dg, sign); break; }
                if constexpr (MaxR >= 9) if (R == 9) { run_stage<C2, 9, 1>(a, b, tw, S, R, L, dl, dg, sign); break; }
                if constexpr (MaxR >= 11) if (R == 11) { run_stage<C2, 11, 1>(a, b, tw, S, R, L, dl, dg, sign); break; }
                if constexpr (MaxR >= 13) if (R == 13) { run_stage<C2, 13, 1>(a, b, tw, S, R, L, dl, dg, sign); break; }
                if constexpr (MaxR >= 17) if (R == 17) { run_stage<C2, 17, 1>(a, b, tw, S, R, L, dl, dg, sign); break; }
                if constexpr (MaxR >= 19) if (R == 19) { run_stage<C2, 19, 1>(a, b, tw, S, R, L, dl, dg, sign); break; }
                if constexpr (MaxR >= 23) if (R == 23) { run_stage<C2, 23, 1>(a, b, tw, S, R, L, dl, dg, sign); break; }
                if constexpr (MaxR >= 29) if (R == 29) { run_stage<C2, 29, 1>(a, b, tw, S, R, L, dl, dg, sign); break; }
                if constexpr (MaxR >= 31) if (R == 31) { run_stage<C2, 31, 1>(a, b, tw, S, R, L, dl, dg, sign); break; }
                run_stage<C2, 1, 2>(a, b, tw, S, R, L, dl, dg, sign);
                break;
        }
        __syncthreads();
        C2* t = a; a = b; b = t;
        Ns *= R;
    }
    return a;
}

}  // namespace m3d
