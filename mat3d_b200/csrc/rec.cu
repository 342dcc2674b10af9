// rec.cu -- microstructure reconstruction by phase retrieval (recon::recPlan,
// src/rec/reconstruction.cpp) on the GPU.
//
// Given the modulus |M(k)| = normC = sqrt(|TPCF| * xyz) of the 3-D Fourier
// transform of a two-phase field, runRec(n, beta) looks for a field m in
// [0, 1] with that modulus (:283-400):
//     m = (U + 1) / 2                                   (U uniform in [-1, 1))
//     loop: M = FFT(m); err = mean | |M| - normC |; stop if err < 0.1 or i >= n
//           ang = arg M   (every 150th pass: 0.3 arg FFT(U') + 0.7 arg M)
//           (on other passes normC e^{i ang} is formed as M normC / |M|)
//           m' = IFFT(normC e^{i ang}) / xyz
//           j < 100:  hybrid input-output  m' < 0 -> m - beta m' ; m' > 1 -> m - beta (m' - 1) ; m' > 1 -> 1
//           j >= 100: box projection       m' < 0 -> 0 ; m' > 1 -> 1 ; j > 200 -> j = 0
//           (the imaginary part is zeroed only where a projection fired)
//     threshold m at 0.5 - x, moving x by 0.001 until the phase-1 fraction is
//     within 1e-4 of normC[0] / xyz (at most 202 tries).
//
// Layout: complex FP64 fields in the reference's voxel order v = z + Nz (y + Ny x).
// One pass of the loop = 5 launches over the work buffer A:
//   zfwd  (m -> A, z lines)  yfwd (y lines)  xturn (x FFT, error partials,
//   modulus replacement, inverse x FFT; its last CTA reduces the error in a
//   fixed order and advances the loop state)  yinv  zinv (z lines, 1/xyz,
//   projection -> m).
// A restart pass adds three launches before them that transform U' (drawn in
// the z-pass load, never stored) and keep 0.3 arg FFT(U') in R.  Those three
// return at once on other passes.  Everything the loop decides (i, j, the
// draw counter, convergence) lives in a device control block, so the whole
// loop is one CUDA graph with a conditional while node; the threshold walk is
// a second while node (an integer count per try, so it is exact).
//
// Random draws: the reference calls Eigen's setRandom (std::rand underneath,
// implementation defined).  Here draw number `call` (0 = the initial field,
// then one per restart) of voxel v is 2 u - 1 with
//   u = (mix(mix(seed * 0x100000001B3 + call) + v) >> 11) * 2^-53,
// mix = the SplitMix64 finaliser: the CPU restatement and the stand-in Eigen
// the reference is built against for testing use the same formula.
//
// Arithmetic that the reference writes as separate operations is kept
// separate (__dmul_rn / __dadd_rn / __dsub_rn) so no fused multiply-add
// changes its rounding; the transforms themselves round differently from any
// CPU FFT, and the iteration amplifies such differences (about threefold per
// pass), so long runs agree with the CPU statistically, not bit for bit.
#include <cuda_runtime.h>

#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/mat3d_b200.h"
#include "fft_plan.hpp"
#include "fft_smem.cuh"

using namespace m3d;

void m3d_internal_set_error(const std::string& msg);

namespace {

int failr(int code, const std::string& msg) {
    m3d_internal_set_error(msg);
    return code;
}

#define MR_CUDA(call)                                                                             \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return failr(M3D_ERR_CUDA, std::string(cudaGetErrorString(e_)) + " (" #call ")"); \
    } while (0)

constexpr int kThreads = 128;

// The dynamic shared-memory limit is an attribute of the kernel, shared by
// every handle: raise it once to the device maximum (227 KB less the static
// shared memory) rather than to one handle's need, which would lower it under
// a larger handle made earlier.
template <class K>
void allow_smem(K kernel) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, kernel) == cudaSuccess)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024 - (int)a.sharedSizeBytes);
    (void)cudaGetLastError();
}
constexpr int kRestartPeriod = 150;  // remainder(i + 1, 150) == 0 (:320)

struct RecCtl {
    int i, j, n, done;      // loop counters (:287-288), stop bound, 1 = converged
    int hio, trips, ctr, thr_done;
    unsigned int ticket, pad0;
    unsigned long long seed, call;  // generator seed, draws taken so far
    unsigned long long count_lt;    // threshold: voxels below the cut
    double beta, x, cut;            // HIO beta; threshold offset and the cut last applied
    double normC0;                  // normC[0]
    long long xyz;
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__device__ __forceinline__ unsigned long long draw_base(unsigned long long seed, unsigned long long call) {
    return mix64(seed * 0x100000001B3ULL + call);
}
// 2 u - 1: both steps are exact in double (u has 53 bits, 2 u is a scaling)
__device__ __forceinline__ double draw_pm1(unsigned long long base, unsigned long long v) {
    const double u = (double)(mix64(base + v) >> 11) * (1.0 / 9007199254740992.0);
    return __dsub_rn(__dmul_rn(2.0, u), 1.0);
}

__device__ __forceinline__ bool restart_pass(const RecCtl* c) { return !c->done && (c->i + 1) % kRestartPeriod == 0; }

// initial field (:289-291): m = (U + 1) * 0.5 from draw 0
__global__ void krec_init(double2* __restrict__ m, RecCtl* ctl, long long xyz) {
    const unsigned long long base = draw_base(ctl->seed, 0);
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < xyz; v += (long long)gridDim.x * blockDim.x)
        m[v] = make_double2(__dmul_rn(__dadd_rn(draw_pm1(base, (unsigned long long)v), 1.0), 0.5), 0.0);
}

// 16-byte global -> shared copies that complete asynchronously (zero-filled
// when !valid; the source is then not read)
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_group1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

enum ZMode { Z_FWD = 0, Z_RAND = 1, Z_INV = 2, Z_BWD = 3 };

// z lines (contiguous): tiles of G lines of length Nz, walked by persistent
// CTAs with three shared buffers (the next tile streams in by cp.async while
// the current one is transformed).
//   Z_FWD : A = FFT_z(m)
//   Z_RAND: A = FFT_z(U') on restart passes (U' = draw `call`, real)
//   Z_INV : m = projection(IFFT_z(A) / xyz, m) unless the pass converged
//   Z_BWD : A = unnormalised inverse FFT_z(m) (plain transforms)
template <int MODE, int MaxR>
__global__ void __launch_bounds__(kThreads) krec_z(double2* __restrict__ A, double2* __restrict__ m,
                                                    const double2* __restrict__ twz, LinePlan pz, int G,
                                                    long long nlines, int ntiles, const RecCtl* __restrict__ ctl) {
    if (MODE == Z_RAND && !restart_pass(ctl)) return;
    if (MODE == Z_INV && ctl->done) return;
    extern __shared__ __align__(16) char smem_raw[];
    const int Nz = pz.n;
    const int tsz = G * Nz;
    double2* tw = (double2*)smem_raw;
    double2* B[3];
    B[0] = tw + Nz;
    B[1] = B[0] + tsz;
    B[2] = B[1] + tsz;
    double* MB = (double*)(B[2] + tsz);  // Z_INV: the old field's real part of the current tile
    const long long xyz = ctl->xyz;
    unsigned long long base = 0;
    if (MODE == Z_RAND) base = draw_base(ctl->seed, ctl->call);
    const double2* src = (MODE == Z_FWD || MODE == Z_BWD) ? m : A;
    // a tile's G lines are one contiguous run of voxels: v0 = tile G Nz ..
    auto valid_of = [&](int tile) { return (int)(min((long long)G, nlines - (long long)tile * G) * Nz); };
    auto fetch = [&](double2* S, int tile) {
        const long long v0 = (long long)tile * tsz;
        const int valid = valid_of(tile);
#pragma unroll 4
        for (int t = threadIdx.x; t < tsz; t += blockDim.x) {
            if (MODE == Z_RAND) S[t] = t < valid ? make_double2(draw_pm1(base, (unsigned long long)(v0 + t)), 0.0)
                                                 : make_double2(0, 0);
            else cp_async16(S + t, t < valid ? src + v0 + t : src, t < valid);
        }
    };
    int tile = blockIdx.x;
    if (tile < ntiles) fetch(B[0], tile);
    cp_async_commit();
    for (int t = threadIdx.x; t < Nz; t += blockDim.x) tw[t] = twz[t];
    const LineLayout L{G, G, Nz, 0, 1, false};
    const double dxyz = (double)xyz;
    const double beta = MODE == Z_INV ? ctl->beta : 0.0;
    const bool hio = MODE == Z_INV && ctl->hio != 0;
    int d = 0;
    for (; tile < ntiles; tile += gridDim.x) {
        cp_async_wait_all();
        __syncthreads();
        const int f = d == 0 ? 2 : d - 1;
        if (MODE == Z_INV) {
            // this tile's old field (the projection needs it only after the
            // transform, so the copy completes behind it): its own group
            const long long v0 = (long long)tile * tsz;
            const int valid = valid_of(tile);
#pragma unroll 4
            for (int t = threadIdx.x; t < valid; t += blockDim.x) cp_async8(MB + t, &m[v0 + t].x, true);
            cp_async_commit();
        }
        const int nxt = tile + gridDim.x;
        if (nxt < ntiles) fetch(B[f], nxt);
        cp_async_commit();
        double2* r = fft_lines<double2, MaxR>(B[d], B[d == 2 ? 0 : d + 1], tw, pz, L,
                                              (MODE == Z_INV || MODE == Z_BWD) ? +1 : -1);
        if (MODE == Z_INV) {
            cp_async_wait_group1();  // the old field landed (the next tile may still be in flight)
            __syncthreads();
        }
        const double* old = MB;
        const long long v0 = (long long)tile * tsz;
        const int valid = valid_of(tile);
        if (MODE != Z_INV) {
#pragma unroll 4
            for (int t = threadIdx.x; t < valid; t += blockDim.x) A[v0 + t] = r[t];
        } else {
            // temp = temp / xyz, then the projections (:345-364) against the
            // old field (prefetched with the tile)
#pragma unroll 2
            for (int t = threadIdx.x; t < valid; t += blockDim.x) {
                const long long v = v0 + t;
                const double2 w = r[t];
                double re = w.x / dxyz, im = w.y / dxyz;
                if (hio) {
                    if (re < 0) { re = __dsub_rn(old[t], __dmul_rn(beta, re)); im = 0; }
                    if (re > 1) { re = __dsub_rn(old[t], __dmul_rn(beta, __dsub_rn(re, 1.0))); im = 0; }
                    if (re > 1) { re = 1; im = 0; }
                } else {
                    if (re < 0) { re = 0; im = 0; }
                    if (re > 1) { re = 1; im = 0; }
                }
                m[v] = make_double2(re, im);
            }
        }
        d = f;
    }
    cp_async_wait_all();
}

// column passes (y or x lines): TZ consecutive z columns of one plane, N
// elements each at `stride`; smem element e of column t at e * TZ + t.
struct ColTile {
    long long base;  // offset of element 0 of column 0
    long long stride;
    int nz;          // columns present in this tile
};

__device__ __forceinline__ void col_store(double2* __restrict__ A, const double2* S, const ColTile& c, int N, int TZ,
                                          const FastDiv& dz) {
#pragma unroll 4
    for (int t = threadIdx.x; t < N * TZ; t += blockDim.x) {
        const int e = dz.div(t), tz = t - e * TZ;
        if (tz < c.nz) A[c.base + e * c.stride + tz] = S[t];
    }
}

__device__ __forceinline__ void col_fetch(double2* S, const double2* __restrict__ A, const ColTile& c, int N, int TZ,
                                          const FastDiv& dz) {
#pragma unroll 4
    for (int t = threadIdx.x; t < N * TZ; t += blockDim.x) {
        const int e = dz.div(t), tz = t - e * TZ;
        const bool ok = tz < c.nz;
        cp_async16(S + t, ok ? A + c.base + e * c.stride + tz : A, ok);
    }
}

enum YMode { Y_FWD = 0, Y_RAND = 1, Y_INV = 2 };

// y lines, in place on A: tiles (x, z range of TZ columns).  Persistent CTAs
// walk the tiles with three shared buffers: while one tile is transformed in
// two of them, the next tile streams into the third (cp.async), so the load
// of a tile overlaps the arithmetic of the one before.
template <int MODE, int MaxR>
__global__ void __launch_bounds__(kThreads) krec_y(double2* __restrict__ A, const double2* __restrict__ twy,
                                                    LinePlan py, int Nz, int TZ, int ntz, int ntiles,
                                                    const RecCtl* __restrict__ ctl) {
    if (MODE == Y_RAND && !restart_pass(ctl)) return;
    if (MODE == Y_INV && ctl->done) return;
    extern __shared__ __align__(16) char smem_raw[];
    const int Ny = py.n;
    double2* tw = (double2*)smem_raw;
    double2* B[3];
    B[0] = tw + Ny;
    B[1] = B[0] + (size_t)Ny * TZ;
    B[2] = B[1] + (size_t)Ny * TZ;
    FastDiv dz, dt;
    dz.init(TZ);
    dt.init(ntz);
    auto tile_of = [&](int tile) {
        const int x = dt.div(tile), z0 = (tile - x * ntz) * TZ;
        return ColTile{(long long)x * Ny * Nz + z0, Nz, min(TZ, Nz - z0)};
    };
    int tile = blockIdx.x;
    if (tile < ntiles) col_fetch(B[0], A, tile_of(tile), Ny, TZ, dz);
    cp_async_commit();
    for (int t = threadIdx.x; t < Ny; t += blockDim.x) tw[t] = twy[t];
    const LineLayout L{TZ, TZ, 1, 0, TZ, true};
    int d = 0;
    for (; tile < ntiles; tile += gridDim.x) {
        cp_async_wait_all();
        __syncthreads();  // tile data landed; the previous tile's stores are done with its buffers
        const int f = d == 0 ? 2 : d - 1;  // the buffer this tile does not use
        const int nxt = tile + gridDim.x;
        if (nxt < ntiles) col_fetch(B[f], A, tile_of(nxt), Ny, TZ, dz);
        cp_async_commit();
        const double2* r = fft_lines<double2, MaxR>(B[d], B[d == 2 ? 0 : d + 1], tw, py, L, MODE == Y_INV ? +1 : -1);
        col_store(A, r, tile_of(tile), Ny, TZ, dz);
        d = f;
    }
    cp_async_wait_all();
}

// x lines with an element-wise output, persistent CTAs as the y passes:
//   XO_ANGLE: restart passes only, R = 0.3 arg FFT(U') (:326-327)
//   XO_COPY : A = the transform (plain transforms, sign as given)
//   XO_NORM : R = sqrt(sqrt(re^2 + im^2)) of the transform (estimateNormFFT_RVE :276-277)
enum XOut { XO_ANGLE = 0, XO_COPY = 1, XO_NORM = 2 };
template <int OUT, int MaxR>
__global__ void __launch_bounds__(kThreads) krec_xout(double2* __restrict__ A, double* __restrict__ R,
                                                       const double2* __restrict__ twx, LinePlan px, int Ny, int Nz,
                                                       int TZ, int ntz, int ntiles, int sign,
                                                       const RecCtl* __restrict__ ctl) {
    if (OUT == XO_ANGLE && !restart_pass(ctl)) return;
    extern __shared__ __align__(16) char smem_raw[];
    const int Nx = px.n;
    double2* tw = (double2*)smem_raw;
    double2* B[3];
    B[0] = tw + Nx;
    B[1] = B[0] + (size_t)Nx * TZ;
    B[2] = B[1] + (size_t)Nx * TZ;
    FastDiv dz, dt;
    dz.init(TZ);
    dt.init(ntz);
    auto tile_of = [&](int tile) {
        const int y = dt.div(tile), z0 = (tile - y * ntz) * TZ;
        return ColTile{(long long)y * Nz + z0, (long long)Ny * Nz, min(TZ, Nz - z0)};
    };
    int tile = blockIdx.x;
    if (tile < ntiles) col_fetch(B[0], A, tile_of(tile), Nx, TZ, dz);
    cp_async_commit();
    for (int t = threadIdx.x; t < Nx; t += blockDim.x) tw[t] = twx[t];
    const LineLayout L{TZ, TZ, 1, 0, TZ, true};
    int d = 0;
    for (; tile < ntiles; tile += gridDim.x) {
        cp_async_wait_all();
        __syncthreads();
        const int f = d == 0 ? 2 : d - 1;
        const int nxt = tile + gridDim.x;
        if (nxt < ntiles) col_fetch(B[f], A, tile_of(nxt), Nx, TZ, dz);
        cp_async_commit();
        const double2* r = fft_lines<double2, MaxR>(B[d], B[d == 2 ? 0 : d + 1], tw, px, L, sign);
        const ColTile c = tile_of(tile);
        if (OUT == XO_COPY) {
            col_store(A, r, c, Nx, TZ, dz);
        } else {
            for (int t = threadIdx.x; t < Nx * TZ; t += blockDim.x) {
                const int e = dz.div(t), tz = t - e * TZ;
                if (tz >= c.nz) continue;
                const double2 w = r[t];
                R[c.base + e * c.stride + tz] =
                    OUT == XO_ANGLE ? __dmul_rn(atan2(w.y, w.x), 0.3)
                                    : sqrt(sqrt(__dadd_rn(__dmul_rn(w.x, w.x), __dmul_rn(w.y, w.y))));
            }
        }
        d = f;
    }
    cp_async_wait_all();
}

// x turnaround: forward x FFT (M = FFT(m) complete), error partials
// (funcNormC, include/reconstruction.hpp:37-44), modulus replacement
// (:317-336), inverse x FFT.  Persistent CTAs with three field buffers and
// two normC buffers (the next tile's field and modulus stream in while the
// current tile is worked on).  Each CTA sums its error terms in a fixed
// order; the last CTA to finish reduces the partials in a fixed order,
// records err[i] and advances the loop state (:300-314, :360-365).
template <int MaxR>
__global__ void __launch_bounds__(kThreads) krec_xturn(double2* __restrict__ A, const double* __restrict__ normC,
                                                        const double* __restrict__ R, const double2* __restrict__ twx,
                                                        LinePlan px, int Ny, int Nz, int TZ, int ntz, int ntiles,
                                                        double* __restrict__ part, double* __restrict__ errs,
                                                        RecCtl* ctl) {
    extern __shared__ __align__(16) char smem_raw[];
    __shared__ double red[kThreads / 32];
    __shared__ bool last;
    const int Nx = px.n;
    const int tsz = Nx * TZ;
    double2* tw = (double2*)smem_raw;
    double2* B[3];
    B[0] = tw + Nx;
    B[1] = B[0] + tsz;
    B[2] = B[1] + tsz;
    double* NB[2];
    NB[0] = (double*)(B[2] + tsz);
    NB[1] = NB[0] + tsz;
    FastDiv dz, dt;
    dz.init(TZ);
    dt.init(ntz);
    auto tile_of = [&](int tile) {
        const int y = dt.div(tile), z0 = (tile - y * ntz) * TZ;
        return ColTile{(long long)y * Nz + z0, (long long)Ny * Nz, min(TZ, Nz - z0)};
    };
    auto fetch = [&](double2* S, double* NS, int tile) {
        const ColTile c = tile_of(tile);
        col_fetch(S, A, c, Nx, TZ, dz);
#pragma unroll 4
        for (int t = threadIdx.x; t < tsz; t += blockDim.x) {
            const int e = dz.div(t), tz = t - e * TZ;
            const bool ok = tz < c.nz;
            cp_async8(NS + t, ok ? normC + c.base + e * c.stride + tz : normC, ok);
        }
    };
    const bool restart = restart_pass(ctl);
    int tile = blockIdx.x;
    if (tile < ntiles) fetch(B[0], NB[0], tile);
    cp_async_commit();
    for (int t = threadIdx.x; t < Nx; t += blockDim.x) tw[t] = twx[t];
    const LineLayout L{TZ, TZ, 1, 0, TZ, true};
    double acc = 0;
    int d = 0, nbi = 0;
    for (; tile < ntiles; tile += gridDim.x) {
        cp_async_wait_all();
        __syncthreads();
        const int f = d == 0 ? 2 : d - 1;
        const int nxt = tile + gridDim.x;
        if (nxt < ntiles) fetch(B[f], NB[nbi ^ 1], nxt);
        cp_async_commit();
        double2* r = fft_lines<double2, MaxR>(B[d], B[d == 2 ? 0 : d + 1], tw, px, L, -1);
        double2* o = (r == B[d]) ? B[d == 2 ? 0 : d + 1] : B[d];
        const ColTile c = tile_of(tile);
        const double* nct = NB[nbi];
#pragma unroll 2
        for (int t = threadIdx.x; t < tsz; t += blockDim.x) {
            const int e = dz.div(t), tz = t - e * TZ;
            if (tz >= c.nz) continue;  // padding columns stay zero through the inverse transform
            const double2 w = r[t];
            const double nc = nct[t];
            const double mod = sqrt(__dadd_rn(__dmul_rn(w.x, w.x), __dmul_rn(w.y, w.y)));
            acc += fabs(__dsub_rn(mod, nc));
            if (restart) {
                const double ang = __dadd_rn(R[c.base + e * c.stride + tz], __dmul_rn(atan2(w.y, w.x), 0.7));
                double sn, co;
                sincos(ang, &sn, &co);
                r[t] = make_double2(__dmul_rn(nc, co), __dmul_rn(nc, sn));
            } else if (mod > 0) {
                // normC e^{i arg M} = M normC / |M|: the same quantity as
                // normC (cos(atan2), sin(atan2)) without the three transcendentals
                const double fct = nc / mod;
                r[t] = make_double2(w.x * fct, w.y * fct);
            } else {
                r[t] = make_double2(nc, 0.0);  // arg 0 = 0
            }
        }
        __syncthreads();
        const double2* q = fft_lines<double2, MaxR>(r, o, tw, px, L, +1);
        col_store(A, q, c, Nx, TZ, dz);
        d = f;
        nbi ^= 1;
    }
    cp_async_wait_all();
    // CTA partial in a fixed order: warp shuffle tree, then the warps in order
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0;
        for (int w = 0; w < kThreads / 32; ++w) b += red[w];
        part[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(&ctl->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x >= 32) return;
    __threadfence();
    double s = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += 32) s += __ldcg(part + k);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x != 0) return;
    const int i = ctl->i;
    int j = ctl->j + 1;  // j += 1 at the top of the pass (:296)
    const double err = s / (double)ctl->xyz;
    errs[i] = err;
    if (err < 0.1) {  // converged: the field stays as it is (:310-314)
        ctl->done = 1;
    } else {
        if (restart) ctl->call += 1;
        ctl->hio = j < 100;
        if (j >= 100 && j > 200) j = 0;
        ctl->i = i + 1;
    }
    ctl->j = j;
    ctl->ticket = 0;
}

// loop condition: another pass while not converged, i < n, and (bound) at most n + 2 trips
__global__ void krec_cond(cudaGraphConditionalHandle h, RecCtl* ctl) {
    const int t = ++ctl->trips;
    cudaGraphSetConditional(h, (!ctl->done && ctl->i < ctl->n && t <= ctl->n + 2) ? 1u : 0u);
}

// threshold walk (:370-395).  The real parts are first copied to a
// contiguous array (40 MB at 171^3, so it stays in L2 across the tries); one
// try = one launch that counts the voxels below 0.5 - x (integer counts, so
// the order does not matter) and whose last CTA steps x exactly as the
// reference does and sets the loop condition.
__global__ void krec_thr_prep(const double2* __restrict__ m, double* __restrict__ re, long long xyz) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < xyz; v += (long long)gridDim.x * blockDim.x)
        re[v] = m[v].x;
}

__global__ void krec_thr_try(const double* __restrict__ re, RecCtl* ctl, long long xyz,
                             cudaGraphConditionalHandle h, int use_cond) {
    __shared__ unsigned int red[kThreads / 32];
    __shared__ bool last;
    const double cut = __dsub_rn(0.5, ctl->x);
    unsigned int cnt = 0;
    // two values per 16-byte load (the copy is 256-byte aligned), the odd tail by one thread
    const double2* re2 = reinterpret_cast<const double2*>(re);
    const long long n2 = xyz / 2;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
#pragma unroll 4
    for (long long v = tid; v < n2; v += (long long)gridDim.x * blockDim.x) {
        const double2 q = re2[v];
        cnt += (q.x < cut ? 1u : 0u) + (q.y < cut ? 1u : 0u);
    }
    if ((xyz & 1) && tid == 0) cnt += re[xyz - 1] < cut ? 1u : 0u;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long b = 0;
        for (int w = 0; w < kThreads / 32; ++w) b += red[w];
        if (b) atomicAdd(&ctl->count_lt, b);
        __threadfence();
        last = atomicAdd(&ctl->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    const unsigned long long below = atomicAdd(&ctl->count_lt, 0ull);
    const double ones = (double)(xyz - (long long)below);  // ang.sum() of the 0/1 field
    const double vol_dif = __dsub_rn(ones / (1.0 * xyz), ctl->normC0 / (1.0 * xyz));
    ctl->cut = cut;
    if (vol_dif > 0) ctl->x = __dsub_rn(ctl->x, 0.001);
    else ctl->x = __dadd_rn(ctl->x, 0.001);
    const bool stop = fabs(vol_dif) < 0.0001 || ctl->ctr > 200;
    if (!stop) ctl->ctr += 1;
    ctl->thr_done = stop;
    ctl->count_lt = 0;
    ctl->ticket = 0;
    const int t = ++ctl->trips;
    if (use_cond) cudaGraphSetConditional(h, (!stop && t <= 203) ? 1u : 0u);
}

// the field after the walk: real part 0 / 1 at the last cut, imaginary part kept (:397)
__global__ void krec_thr_apply(double2* __restrict__ m, const RecCtl* __restrict__ ctl, long long xyz) {
    const double cut = ctl->cut;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < xyz; v += (long long)gridDim.x * blockDim.x)
        m[v].x = m[v].x < cut ? 0.0 : 1.0;
}

__global__ void krec_real(const double2* __restrict__ m, double* __restrict__ out, long long xyz) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < xyz; v += (long long)gridDim.x * blockDim.x)
        out[v] = m[v].x;
}

cudaError_t add_while(cudaGraph_t graph, const cudaGraphNode_t* deps, size_t ndeps, cudaGraphConditionalHandle h,
                      cudaGraphNode_t* node, cudaGraph_t* body) {
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};  // the remaining members are zero
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(node, graph, deps, ndeps, &p);
    if (e == cudaSuccess) *body = p.conditional.phGraph_out[0];
    return e;
}

}  // namespace

struct m3d_rec {
    int Nx = 0, Ny = 0, Nz = 0;
    long long xyz = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    double2 *m = nullptr, *A = nullptr, *twx = nullptr, *twy = nullptr, *twz = nullptr;
    double *R = nullptr, *normC = nullptr, *part = nullptr, *errs = nullptr, *real = nullptr;
    int err_cap = 0;
    RecCtl* d_ctl = nullptr;
    RecCtl* h_ctl = nullptr;  // pinned mirror
    LinePlan px{}, py{}, pz{};
    int G = 1, TZ = 1, ntz = 1;
    long long zlines = 0;
    int nb_y = 0, nb_x = 0;
    int TZX = 1, ntzx = 1;  // column tile of the x passes (they also stage normC)
    int grid_y = 1, grid_z = 1, grid_zi = 1, grid_x = 1, grid_xr = 1;  // persistent CTAs per pass
    double normC0 = 0;
    unsigned long long seed = 1;
    bool started = false;   // a field exists (run, set_state)
    bool norm_set = false;  // normC holds the target modulus
    std::vector<int> cc1, cc2;  // the cut sections as 0/1 (section constructor)
    int Nzz = 0;
    int last_n = 0;         // n of the last runRec (numloops)
    int i = 0, j = 0;       // host copy of the loop state
    unsigned long long call = 0;
    int n_recorded = 0;
    bool profiling = false;
    double pass_ms[8] = {0};
    long long pass_count[8] = {0};
    cudaEvent_t ev[9] = {};
    cudaGraphExec_t g_loop = nullptr, g_thr = nullptr;
    long long launches = 0;

    ~m3d_rec() {
        if (g_loop) cudaGraphExecDestroy(g_loop);
        if (g_thr) cudaGraphExecDestroy(g_thr);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        cudaFree(m); cudaFree(A); cudaFree(twx); cudaFree(twy); cudaFree(twz);
        cudaFree(R); cudaFree(normC); cudaFree(part); cudaFree(errs); cudaFree(real); cudaFree(d_ctl);
        if (h_ctl) cudaFreeHost(h_ctl);
        if (stream) cudaStreamDestroy(stream);
    }
    size_t z_smem() const { return (size_t)Nz * 16 + 3 * (size_t)G * Nz * 16; }
    size_t zi_smem() const { return z_smem() + (size_t)G * Nz * 8; }
    size_t y_smem() const { return (size_t)Ny * 16 + 3 * (size_t)Ny * TZ * 16; }
    size_t x_smem() const { return (size_t)Nx * 16 + 3 * (size_t)Nx * TZX * 16 + 2 * (size_t)Nx * TZX * 8; }
    size_t xr_smem() const { return (size_t)Nx * 16 + 3 * (size_t)Nx * TZX * 16; }
    int grid1d() const { return (int)std::min<long long>(148 * 8, (xyz + kThreads - 1) / kThreads); }

    // the kernels of one pass, in order; `prof` brackets each with events
    template <int MaxR>
    int launch_pass_t(bool prof) {
        const int nbz = (int)((zlines + G - 1) / G);
        auto mark = [&](int k) { if (prof) cudaEventRecord(ev[k], stream); };
        mark(0);
        krec_z<Z_RAND, MaxR><<<grid_z, kThreads, z_smem(), stream>>>(A, m, twz, pz, G, zlines, nbz, d_ctl);
        krec_y<Y_RAND, MaxR><<<grid_y, kThreads, y_smem(), stream>>>(A, twy, py, Nz, TZ, ntz, nb_y, d_ctl);
        krec_xout<XO_ANGLE, MaxR><<<grid_xr, kThreads, xr_smem(), stream>>>(A, R, twx, px, Ny, Nz, TZX, ntzx, nb_x, -1, d_ctl);
        mark(1);
        krec_z<Z_FWD, MaxR><<<grid_z, kThreads, z_smem(), stream>>>(A, m, twz, pz, G, zlines, nbz, d_ctl);
        mark(2);
        krec_y<Y_FWD, MaxR><<<grid_y, kThreads, y_smem(), stream>>>(A, twy, py, Nz, TZ, ntz, nb_y, d_ctl);
        mark(3);
        krec_xturn<MaxR><<<grid_x, kThreads, x_smem(), stream>>>(A, normC, R, twx, px, Ny, Nz, TZX, ntzx, nb_x, part, errs, d_ctl);
        mark(4);
        krec_y<Y_INV, MaxR><<<grid_y, kThreads, y_smem(), stream>>>(A, twy, py, Nz, TZ, ntz, nb_y, d_ctl);
        mark(5);
        krec_z<Z_INV, MaxR><<<grid_zi, kThreads, zi_smem(), stream>>>(A, m, twz, pz, G, zlines, nbz, d_ctl);
        mark(6);
        launches += 8;
        MR_CUDA(cudaGetLastError());
        return M3D_OK;
    }
    // one plain 3-D transform of m (sign -1 forward, +1 inverse, unnormalised):
    // into A (out_norm false) or sqrt|.| into R (out_norm true)
    template <int MaxR>
    int transform_t(int sign, bool out_norm) {
        const int nbz = (int)((zlines + G - 1) / G);
        auto check = [&](const char* what) -> int {
            const cudaError_t e = cudaGetLastError();
            return e == cudaSuccess ? M3D_OK : failr(M3D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        };
        if (int rc = check("before the transform")) return rc;
        if (sign < 0) krec_z<Z_FWD, MaxR><<<grid_z, kThreads, z_smem(), stream>>>(A, m, twz, pz, G, zlines, nbz, d_ctl);
        else krec_z<Z_BWD, MaxR><<<grid_z, kThreads, z_smem(), stream>>>(A, m, twz, pz, G, zlines, nbz, d_ctl);
        if (int rc = check("z pass")) return rc;
        if (sign < 0) krec_y<Y_FWD, MaxR><<<grid_y, kThreads, y_smem(), stream>>>(A, twy, py, Nz, TZ, ntz, nb_y, d_ctl);
        else krec_y<Y_INV, MaxR><<<grid_y, kThreads, y_smem(), stream>>>(A, twy, py, Nz, TZ, ntz, nb_y, d_ctl);
        if (int rc = check("y pass")) return rc;
        if (out_norm)
            krec_xout<XO_NORM, MaxR><<<grid_xr, kThreads, xr_smem(), stream>>>(A, R, twx, px, Ny, Nz, TZX, ntzx, nb_x, sign, d_ctl);
        else
            krec_xout<XO_COPY, MaxR><<<grid_xr, kThreads, xr_smem(), stream>>>(A, R, twx, px, Ny, Nz, TZX, ntzx, nb_x, sign, d_ctl);
        launches += 3;
        MR_CUDA(cudaGetLastError());
        return M3D_OK;
    }
    int transform(int sign, bool out_norm) {
        RecCtl c{};  // i = 0, not done: the pass kernels' early exits stay closed
        c.xyz = xyz;
        *h_ctl = c;
        MR_CUDA(cudaMemcpyAsync(d_ctl, h_ctl, sizeof(RecCtl), cudaMemcpyHostToDevice, stream));
        switch (maxr) {
            case 5: return transform_t<5>(sign, out_norm);
            case 13: return transform_t<13>(sign, out_norm);
            case 19: return transform_t<19>(sign, out_norm);
            default: return transform_t<31>(sign, out_norm);
        }
    }
    template <int MaxR>
    void set_smem_t() {
        const int zs = (int)z_smem(), ys = (int)y_smem(), xs = (int)x_smem();
        allow_smem(krec_z<Z_FWD, MaxR>);
        allow_smem(krec_z<Z_RAND, MaxR>);
        allow_smem(krec_z<Z_INV, MaxR>);
        allow_smem(krec_y<Y_FWD, MaxR>);
        allow_smem(krec_y<Y_RAND, MaxR>);
        allow_smem(krec_y<Y_INV, MaxR>);
        allow_smem(krec_xout<XO_ANGLE, MaxR>);
        allow_smem(krec_xout<XO_COPY, MaxR>);
        allow_smem(krec_xout<XO_NORM, MaxR>);
        allow_smem(krec_z<Z_BWD, MaxR>);
        allow_smem(krec_xturn<MaxR>);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        sms = std::max(1, sms);
        auto fill = [&](auto kern, size_t smem, int tiles) {
            int per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
            return std::max(1, std::min(tiles, std::max(1, per_sm) * sms));
        };
        grid_y = fill(krec_y<Y_FWD, MaxR>, (size_t)ys, nb_y);
        grid_z = fill(krec_z<Z_FWD, MaxR>, (size_t)zs, (int)((zlines + G - 1) / G));
        grid_zi = fill(krec_z<Z_INV, MaxR>, zi_smem(), (int)((zlines + G - 1) / G));
        grid_x = fill(krec_xturn<MaxR>, (size_t)xs, nb_x);
        grid_xr = fill(krec_xout<XO_ANGLE, MaxR>, xr_smem(), nb_x);
    }
    // kernels are instantiated for the largest odd radix of the grid's plans
    // in buckets, so a grid of small factors does not pay the registers of a
    // 31-point butterfly
    int maxr = 5;
    int launch_pass(bool prof) {
        switch (maxr) {
            case 5: return launch_pass_t<5>(prof);
            case 13: return launch_pass_t<13>(prof);
            case 19: return launch_pass_t<19>(prof);
            default: return launch_pass_t<31>(prof);
        }
    }
    void set_smem() {
        switch (maxr) {
            case 5: set_smem_t<5>(); break;
            case 13: set_smem_t<13>(); break;
            case 19: set_smem_t<19>(); break;
            default: set_smem_t<31>(); break;
        }
    }

    // grow the error track, keeping what it holds
    int ensure_err(int n) {
        if (n <= err_cap) return M3D_OK;
        double* e = nullptr;
        if (cudaMalloc(&e, (size_t)n * sizeof(double)) != cudaSuccess) {
            (void)cudaGetLastError();
            return failr(M3D_ERR_OOM, "device allocation failed");
        }
        MR_CUDA(cudaMemsetAsync(e, 0, (size_t)n * sizeof(double), stream));
        if (err_cap > 0) MR_CUDA(cudaMemcpyAsync(e, errs, (size_t)err_cap * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        cudaFree(errs);
        errs = e;
        err_cap = n;
        if (g_loop) { cudaGraphExecDestroy(g_loop); g_loop = nullptr; }  // the graph holds the old pointer
        return M3D_OK;
    }

    int build_loop_graph() {
        cudaGraph_t top = nullptr;
        MR_CUDA(cudaGraphCreate(&top, 0));
        cudaGraphConditionalHandle h;
        cudaGraphNode_t node;
        cudaGraph_t body = nullptr;
        cudaError_t e = cudaGraphConditionalHandleCreate(&h, top, 1, cudaGraphCondAssignDefault);
        if (e == cudaSuccess) e = add_while(top, nullptr, 0, h, &node, &body);
        if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            const long long kl = launches;
            const int rc = launch_pass(false);
            krec_cond<<<1, 1, 0, stream>>>(h, d_ctl);
            launches = kl;
            cudaGraph_t got = nullptr;
            e = rc ? cudaErrorLaunchFailure : cudaGetLastError();
            const cudaError_t e2 = cudaStreamEndCapture(stream, &got);
            if (e == cudaSuccess) e = e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&g_loop, top, 0);
        cudaGraphDestroy(top);
        if (e != cudaSuccess) {
            g_loop = nullptr;
            (void)cudaGetLastError();
            return failr(M3D_ERR_CUDA, std::string("reconstruction graph: ") + cudaGetErrorString(e));
        }
        return M3D_OK;
    }

    int build_thr_graph() {
        cudaGraph_t top = nullptr;
        MR_CUDA(cudaGraphCreate(&top, 0));
        cudaGraphConditionalHandle h;
        cudaGraphNode_t node;
        cudaGraph_t body = nullptr;
        cudaError_t e = cudaGraphConditionalHandleCreate(&h, top, 1, cudaGraphCondAssignDefault);
        if (e == cudaSuccess) e = add_while(top, nullptr, 0, h, &node, &body);
        if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            krec_thr_try<<<grid1d(), kThreads, 0, stream>>>(R, d_ctl, xyz, h, 1);
            cudaGraph_t got = nullptr;
            e = cudaGetLastError();
            const cudaError_t e2 = cudaStreamEndCapture(stream, &got);
            if (e == cudaSuccess) e = e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&g_thr, top, 0);
        cudaGraphDestroy(top);
        if (e != cudaSuccess) {
            g_thr = nullptr;
            (void)cudaGetLastError();
            return failr(M3D_ERR_CUDA, std::string("threshold graph: ") + cudaGetErrorString(e));
        }
        return M3D_OK;
    }

    int pull_ctl() {
        MR_CUDA(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(RecCtl), cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        return M3D_OK;
    }

    // continue the loop until converged or i reaches n_stop
    int iterate(int n_stop, double beta) {
        if (n_stop > err_cap) {
            const int rc = ensure_err(std::max(n_stop, 2 * err_cap));
            if (rc) return rc;
        }
        // errors recorded before this call stay (the device array keeps them)
        RecCtl c{};
        c.i = i; c.j = j; c.n = n_stop; c.done = 0; c.hio = 1; c.trips = 0;
        c.seed = seed; c.call = call; c.beta = beta; c.normC0 = normC0; c.xyz = xyz;
        *h_ctl = c;
        MR_CUDA(cudaMemcpyAsync(d_ctl, h_ctl, sizeof(RecCtl), cudaMemcpyHostToDevice, stream));
        if (i < n_stop) {
            if (profiling) {
                for (int t = 0; t < n_stop - i + 1; ++t) {
                    int rc = launch_pass(true);
                    if (rc) return rc;
                    rc = pull_ctl();
                    if (rc) return rc;
                    float ms;
                    for (int k = 0; k < 6; ++k) {
                        cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
                        pass_ms[k] += ms;
                        pass_count[k] += 1;
                    }
                    if (h_ctl->done || h_ctl->i >= n_stop) break;
                }
            } else {
                if (!g_loop) {
                    const int rc = build_loop_graph();
                    if (rc) return rc;
                }
                MR_CUDA(cudaGraphLaunch(g_loop, stream));
                launches += 1;
                const int rc = pull_ctl();
                if (rc) return rc;
                launches += 9LL * h_ctl->trips;
            }
        }
        const int rc = pull_ctl();
        if (rc) return rc;
        if (h_ctl->trips > n_stop + 2) return failr(M3D_ERR_CUDA, "reconstruction loop exceeded its trip bound");
        i = h_ctl->i;
        j = h_ctl->j;
        call = h_ctl->call;
        n_recorded = h_ctl->done ? i + 1 : i;
        return M3D_OK;
    }

    int threshold() {
        RecCtl c{};
        c.normC0 = normC0; c.xyz = xyz; c.x = 0; c.ctr = 0; c.count_lt = 0; c.trips = 0;
        c.i = i; c.j = j; c.seed = seed; c.call = call;
        *h_ctl = c;
        MR_CUDA(cudaMemcpyAsync(d_ctl, h_ctl, sizeof(RecCtl), cudaMemcpyHostToDevice, stream));
        krec_thr_prep<<<grid1d(), kThreads, 0, stream>>>(m, R, xyz);  // R is free between passes
        launches += 1;
        if (profiling) {
            for (int t = 0; t < 203; ++t) {
                krec_thr_try<<<grid1d(), kThreads, 0, stream>>>(R, d_ctl, xyz, cudaGraphConditionalHandle{}, 0);
                launches += 1;
                MR_CUDA(cudaGetLastError());
                const int rc = pull_ctl();
                if (rc) return rc;
                if (h_ctl->thr_done) break;
            }
        } else {
            if (!g_thr) {
                const int rc = build_thr_graph();
                if (rc) return rc;
            }
            MR_CUDA(cudaGraphLaunch(g_thr, stream));
            launches += 1;
        }
        krec_thr_apply<<<grid1d(), kThreads, 0, stream>>>(m, d_ctl, xyz);
        launches += 1;
        MR_CUDA(cudaGetLastError());
        const int rc = pull_ctl();
        if (rc) return rc;
        if (!profiling) launches += h_ctl->trips;
        if (!h_ctl->thr_done) return failr(M3D_ERR_CUDA, "threshold walk did not finish");
        return M3D_OK;
    }
};

extern "C" {

}  // extern "C"

// a handle of the given grid with every buffer allocated; normC not set
static int rec_alloc(int Nx, int Ny, int Nz, int device, m3d_rec** out) {
    *out = nullptr;
    if (Nx < 1 || Ny < 1 || Nz < 1 || Nx > 2048 || Ny > 2048 || Nz > 2048)
        return failr(M3D_ERR_ARG, "grid sizes must be in [1, 2048]");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return failr(M3D_ERR_CUDA, "no CUDA device");
    if (device < 0 || device >= ndev) return failr(M3D_ERR_ARG, "device out of range");
    MR_CUDA(cudaSetDevice(device));
    m3d_rec* h = new m3d_rec();
    h->Nx = Nx; h->Ny = Ny; h->Nz = Nz;
    h->xyz = (long long)Nx * Ny * Nz;
    h->device = device;
    if (!make_plan(Nx, h->px, true) || !make_plan(Ny, h->py, true) || !make_plan(Nz, h->pz, true)) {
        delete h;
        return failr(M3D_ERR_UNSUPPORTED, "grid sizes need prime factors <= 32");
    }
    // ~48 KB of shared memory per CTA (two buffers of 16-byte elements) so
    // that several CTAs share an SM
    // z tiles: three 16-byte buffers plus the old field's 8-byte values in
    // about 75 KB, so that three CTAs share an SM
    h->G = std::max(1, std::min(16, (int)((75 * 1024 - 16 * (size_t)Nz) / (56 * (size_t)Nz))));
    const int nmax = std::max(Nx, Ny);
    h->TZ = std::max(1, std::min(16, (int)(48 * 1024 / (32 * (size_t)nmax))));
    h->TZ = std::min(h->TZ, Nz);
    h->ntz = (Nz + h->TZ - 1) / h->TZ;
    h->zlines = (long long)Nx * Ny;
    h->nb_y = Nx * h->ntz;
    // the x turnaround also double-buffers normC: a narrower tile, so that
    // three CTAs still share an SM (227 KB)
    h->TZX = std::max(1, std::min(h->TZ, (int)((75 * 1024 - 16 * (size_t)Nx) / (64 * (size_t)Nx))));
    h->ntzx = (Nz + h->TZX - 1) / h->TZX;
    h->nb_x = Ny * h->ntzx;
    if (h->zi_smem() > 220 * 1024 || h->y_smem() > 220 * 1024 || h->x_smem() > 220 * 1024) {
        delete h;
        return failr(M3D_ERR_UNSUPPORTED, "grid too large for the shared-memory line FFTs");
    }
    const size_t c16 = (size_t)h->xyz * sizeof(double2), c8 = (size_t)h->xyz * sizeof(double);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&h->m, c16) != cudaSuccess || cudaMalloc(&h->A, c16) != cudaSuccess ||
        cudaMalloc(&h->R, c8) != cudaSuccess || cudaMalloc(&h->normC, c8) != cudaSuccess ||
        cudaMalloc(&h->part, (size_t)h->nb_x * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->twx, Nx * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&h->twy, Ny * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&h->twz, Nz * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&h->d_ctl, sizeof(RecCtl)) != cudaSuccess ||
        cudaMallocHost(&h->h_ctl, sizeof(RecCtl)) != cudaSuccess) {
        delete h;
        (void)cudaGetLastError();
        return failr(M3D_ERR_OOM, "device allocation failed");
    }
    for (auto& e : h->ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            delete h;
            return failr(M3D_ERR_CUDA, "event creation failed");
        }
    const auto tx = twiddles<double>(Nx), ty = twiddles<double>(Ny), tz = twiddles<double>(Nz);
    cudaMemset(h->normC, 0, c8);
    cudaMemcpy(h->twx, tx.data(), Nx * sizeof(double2), cudaMemcpyHostToDevice);
    cudaMemcpy(h->twy, ty.data(), Ny * sizeof(double2), cudaMemcpyHostToDevice);
    cudaMemcpy(h->twz, tz.data(), Nz * sizeof(double2), cudaMemcpyHostToDevice);
    cudaMemset(h->m, 0, c16);
    cudaMemset(h->R, 0, c8);
    cudaMemset(h->d_ctl, 0, sizeof(RecCtl));
    int mr = 5;
    for (const LinePlan* pl : {&h->px, &h->py, &h->pz})
        for (int k = 0; k < pl->nstages; ++k) mr = std::max(mr, pl->radix[k] == 8 ? 5 : pl->radix[k]);
    h->maxr = mr <= 5 ? 5 : mr <= 13 ? 13 : mr <= 19 ? 19 : 31;
    h->set_smem();
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        delete h;
        return failr(M3D_ERR_CUDA, "device set-up failed");
    }
    *out = h;
    return M3D_OK;
}

// host complex array (xyz (re, im) pairs) -> m; transform; A -> host
static int rec_fft_host(m3d_rec* h, const double* in, double* out, int sign) {
    const size_t c16 = (size_t)h->xyz * sizeof(double2);
    MR_CUDA(cudaMemcpyAsync(h->m, in, c16, cudaMemcpyHostToDevice, h->stream));
    int rc = h->transform(sign, false);
    if (rc) return rc;
    MR_CUDA(cudaMemcpyAsync(out, h->A, c16, cudaMemcpyDeviceToHost, h->stream));
    MR_CUDA(cudaStreamSynchronize(h->stream));
    return M3D_OK;
}

// two's-complement wrap of an int product, as the reference's int arithmetic
static double int_product(long long a, long long b, long long c, long long d) {
    const unsigned long long u = (unsigned long long)a * (unsigned long long)b * (unsigned long long)c *
                                 (unsigned long long)d;
    return (double)(int)(unsigned)(u & 0xFFFFFFFFull);
}

// writers -----------------------------------------------------------------
struct Crc32Table {
    unsigned t[256];
    Crc32Table() {
        for (unsigned i = 0; i < 256; ++i) {
            unsigned c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            t[i] = c;
        }
    }
};
static unsigned crc32_of(const unsigned char* p, size_t n, unsigned crc = 0xFFFFFFFFu) {
    static const Crc32Table table;  // initialised once, thread-safely
    for (size_t i = 0; i < n; ++i) crc = table.t[(crc ^ p[i]) & 0xFF] ^ (crc >> 8);
    return crc;
}

// 8-bit greyscale PNG (zlib stream of stored deflate blocks: no compression library needed)
static bool write_png_gray(const std::string& path, int w, int h, const unsigned char* px) {
    std::vector<unsigned char> raw;
    raw.reserve((size_t)(w + 1) * h);
    for (int y = 0; y < h; ++y) {
        raw.push_back(0);  // filter: none
        raw.insert(raw.end(), px + (size_t)y * w, px + (size_t)(y + 1) * w);
    }
    std::vector<unsigned char> z = {0x78, 0x01};
    unsigned a = 1, b = 0;
    for (unsigned char c : raw) { a = (a + c) % 65521u; b = (b + a) % 65521u; }
    for (size_t off = 0; off < raw.size() || off == 0;) {
        const size_t len = std::min<size_t>(65535, raw.size() - off);
        const bool final = off + len >= raw.size();
        z.push_back(final ? 1 : 0);
        z.push_back(len & 0xFF); z.push_back(len >> 8);
        z.push_back(~len & 0xFF); z.push_back((~len >> 8) & 0xFF);
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
        off += len;
        if (final) break;
    }
    const unsigned ad = (b << 16) | a;
    for (int k = 3; k >= 0; --k) z.push_back((ad >> (8 * k)) & 0xFF);
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    auto be32 = [](unsigned v, unsigned char* o) { o[0] = v >> 24; o[1] = v >> 16; o[2] = v >> 8; o[3] = v; };
    auto chunk = [&](const char* type, const std::vector<unsigned char>& data) {
        unsigned char hdr[8];
        be32((unsigned)data.size(), hdr);
        std::memcpy(hdr + 4, type, 4);
        std::fwrite(hdr, 1, 8, f);
        if (!data.empty()) std::fwrite(data.data(), 1, data.size(), f);
        unsigned crc = crc32_of((const unsigned char*)type, 4);
        crc = crc32_of(data.data(), data.size(), crc) ^ 0xFFFFFFFFu;
        unsigned char c4[4];
        be32(crc, c4);
        std::fwrite(c4, 1, 4, f);
    };
    static const unsigned char sig[8] = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    std::fwrite(sig, 1, 8, f);
    std::vector<unsigned char> ihdr(13);
    be32(w, ihdr.data());
    be32(h, ihdr.data() + 4);
    ihdr[8] = 8; ihdr[9] = 0; ihdr[10] = 0; ihdr[11] = 0; ihdr[12] = 0;  // 8-bit grey, no interlace
    chunk("IHDR", ihdr);
    chunk("IDAT", z);
    chunk("IEND", {});
    return std::fclose(f) == 0;
}

extern "C" {

int m3drec_create(int Nx, int Ny, int Nz, const double* tpcf, int device, m3d_rec** out) {
    if (!out) return failr(M3D_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!tpcf) return failr(M3D_ERR_ARG, "tpcf is NULL");
    m3d_rec* h = nullptr;
    int rc = rec_alloc(Nx, Ny, Nz, device, &h);
    if (rc) return rc;
    // normC = sqrt(|TPCF| * xyz) (:238-239)
    std::vector<double> nc((size_t)h->xyz);
    for (long long v = 0; v < h->xyz; ++v) nc[v] = std::sqrt(std::fabs(tpcf[v]) * (double)h->xyz);
    h->normC0 = nc[0];
    if (cudaMemcpy(h->normC, nc.data(), nc.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        delete h;
        return failr(M3D_ERR_CUDA, "normC upload failed");
    }
    h->norm_set = true;
    *out = h;
    return M3D_OK;
}

// recPlan(CImg c1, CImg c2) :145-206: two perpendicular cut sections, 8-bit
// images stored x fastest (CImg's layout: pixel (x, y) at x + width * y).
// The grid is width1 x height1 x height2.  Each section becomes 0/1 by the
// reference's integer division pixel / max(pixel).  The reference fills the
// second section's array over the first one's extent, so both must have the
// same size (other sizes overrun its arrays); an all-zero section divides by
// zero there -- both are rejected here.
int m3drec_create_from_sections(const unsigned char* c1, int w1, int h1, const unsigned char* c2, int w2, int h2,
                                int device, m3d_rec** out) {
    if (!out) return failr(M3D_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!c1 || !c2) return failr(M3D_ERR_ARG, "NULL section");
    if (w1 != w2 || h1 != h2) return failr(M3D_ERR_ARG, "the two sections must have the same size");
    int max1 = 0, max2 = 0;
    for (int i = 0; i < w1; ++i)
        for (int j = 0; j < h1; ++j) {
            max1 = std::max(max1, (int)c1[i + (size_t)w1 * j]);
            max2 = std::max(max2, (int)c2[i + (size_t)w2 * j]);
        }
    if (max1 == 0 || max2 == 0) return failr(M3D_ERR_ARG, "a section has no nonzero pixel");
    m3d_rec* h = nullptr;
    int rc = rec_alloc(w1, h1, h2, device, &h);
    if (rc) return rc;
    h->Nzz = w2;
    h->cc1.resize((size_t)w1 * h1);
    h->cc2.resize((size_t)w1 * h1);
    for (int j = 0; j < w1; ++j)
        for (int k = 0; k < h1; ++k) {
            h->cc1[k + (size_t)j * h1] = (int)c1[j + (size_t)w1 * k] / max1;
            h->cc2[k + (size_t)j * h1] = (int)c2[j + (size_t)w2 * k] / max2;
        }
    *out = h;
    return M3D_OK;
}

// estimateNormFFT_RVE :245-281: the sections' autocorrelations by 2-D
// transforms, the separable two-point estimate, normC = sqrt|FFT3(estimate)|
int m3drec_estimate_norm(m3d_rec* h) {
    if (!h) return failr(M3D_ERR_ARG, "NULL handle");
    if (h->cc1.empty()) return failr(M3D_ERR_STATE, "the handle was not made from cut sections");
    MR_CUDA(cudaSetDevice(h->device));
    const int Nx = h->Nx, Ny = h->Ny, Nz = h->Nz, Nzz = h->Nzz;
    auto autocorr = [&](const std::vector<int>& cc, int a, int b, std::vector<double>& res) -> int {
        m3d_rec* t = nullptr;
        int rc = rec_alloc(a, b, 1, h->device, &t);
        if (rc) return rc;
        const size_t n = (size_t)a * b;
        std::vector<double> in(2 * n), sp(2 * n);
        for (size_t i = 0; i < n; ++i) { in[2 * i] = (double)cc[i]; in[2 * i + 1] = 0; }
        rc = rec_fft_host(t, in.data(), sp.data(), -1);
        const double den = int_product(a, b, a, b);
        for (size_t i = 0; i < n && !rc; ++i) {
            in[2 * i] = (sp[2 * i] * sp[2 * i] + sp[2 * i + 1] * sp[2 * i + 1]) / den;
            in[2 * i + 1] = 0;
        }
        res.resize(2 * n);
        if (!rc) rc = rec_fft_host(t, in.data(), res.data(), +1);
        m3drec_destroy(t);
        return rc;
    };
    std::vector<double> cc3, cc4;
    int rc = autocorr(h->cc1, Nx, Ny, cc3);
    if (!rc) rc = autocorr(h->cc2, Nz, Nzz, cc4);
    if (rc) return rc;
    const double f1 = cc3[0];
    const double dxyz = (double)h->xyz;
    std::vector<double> mh(2 * (size_t)h->xyz);
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j) {
            const double c3 = cc3[2 * ((size_t)i * Ny + j)];
            for (int k = 0; k < Nz; ++k) {
                const double c4 = cc4[2 * (size_t)k];
                const double a = c3 * c4 / f1;
                const double b = (f1 - c3) * (f1 - c4) / (1 - f1);
                const size_t v = k + (size_t)j * Nz + (size_t)i * Nz * Ny;
                mh[2 * v] = (a + b) * dxyz;
                mh[2 * v + 1] = 0;
            }
        }
    MR_CUDA(cudaMemcpyAsync(h->m, mh.data(), mh.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    rc = h->transform(-1, true);  // R = sqrt(sqrt(|MHat|^2))
    if (rc) return rc;
    MR_CUDA(cudaMemcpyAsync(h->normC, h->R, (size_t)h->xyz * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    MR_CUDA(cudaMemcpyAsync(&h->normC0, h->normC, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MR_CUDA(cudaStreamSynchronize(h->stream));
    h->norm_set = true;
    return M3D_OK;
}

// the modulus the loop targets (xyz doubles)
int m3drec_get_norm(m3d_rec* h, double* out) {
    if (!h || !out) return failr(M3D_ERR_ARG, "NULL argument");
    MR_CUDA(cudaSetDevice(h->device));
    MR_CUDA(cudaMemcpyAsync(out, h->normC, (size_t)h->xyz * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MR_CUDA(cudaStreamSynchronize(h->stream));
    return M3D_OK;
}

// one unnormalised 3-D complex transform of host arrays on the GPU (sign -1
// forward, +1 inverse; xyz (re, im) pairs, index z + Nz (y + Ny x))
int m3drec_fft3(const double* in, double* out, int Nx, int Ny, int Nz, int sign, int device) {
    if (!in || !out) return failr(M3D_ERR_ARG, "NULL argument");
    if (sign != -1 && sign != 1) return failr(M3D_ERR_ARG, "sign must be -1 or +1");
    m3d_rec* t = nullptr;
    int rc = rec_alloc(Nx, Ny, Nz, device, &t);
    if (rc) return rc;
    rc = rec_fft_host(t, in, out, sign);
    m3drec_destroy(t);
    return rc;
}

int m3drec_destroy(m3d_rec* h) {
    if (h) {
        cudaSetDevice(h->device);
        cudaStreamSynchronize(h->stream);
        delete h;
    }
    return M3D_OK;
}

int m3drec_seed(m3d_rec* h, unsigned long long seed) {
    if (!h) return failr(M3D_ERR_ARG, "NULL handle");
    h->seed = seed;
    h->call = 0;
    return M3D_OK;
}

// runRec(n, beta) :283-400: fresh random field, the loop, the threshold
int m3drec_run(m3d_rec* h, int n, double beta) {
    if (!h) return failr(M3D_ERR_ARG, "NULL handle");
    if (n < 0 || n > 10000000) return failr(M3D_ERR_ARG, "n must be in [0, 1e7]");
    if (!h->norm_set) return failr(M3D_ERR_STATE, "no target modulus (estimate_norm first)");
    h->last_n = n;
    MR_CUDA(cudaSetDevice(h->device));
    RecCtl c{};
    c.seed = h->seed;
    *h->h_ctl = c;
    MR_CUDA(cudaMemcpyAsync(h->d_ctl, h->h_ctl, sizeof(RecCtl), cudaMemcpyHostToDevice, h->stream));
    krec_init<<<h->grid1d(), kThreads, 0, h->stream>>>(h->m, h->d_ctl, h->xyz);
    h->launches += 1;
    MR_CUDA(cudaGetLastError());
    h->i = 0; h->j = 0; h->call = 1; h->n_recorded = 0;
    h->started = true;
    if (n > 0) {
        int rc = h->ensure_err(n);
        if (rc) return rc;
        MR_CUDA(cudaMemsetAsync(h->errs, 0, (size_t)n * sizeof(double), h->stream));
        rc = h->iterate(n, beta);
        if (rc) return rc;
    }
    return h->threshold();
}

// more passes of the loop from the current state (no threshold): until
// converged or `iters` further passes
int m3drec_iterate(m3d_rec* h, int iters, double beta) {
    if (!h) return failr(M3D_ERR_ARG, "NULL handle");
    if (!h->norm_set) return failr(M3D_ERR_STATE, "no target modulus (estimate_norm first)");
    if (!h->started) return failr(M3D_ERR_STATE, "no field yet (run or set_state first)");
    if (iters < 0 || iters > 10000000) return failr(M3D_ERR_ARG, "iters must be in [0, 1e7]");
    MR_CUDA(cudaSetDevice(h->device));
    return h->iterate(h->i + iters, beta);
}

int m3drec_threshold(m3d_rec* h) {
    if (!h) return failr(M3D_ERR_ARG, "NULL handle");
    if (!h->started) return failr(M3D_ERR_STATE, "no field yet (run or set_state first)");
    MR_CUDA(cudaSetDevice(h->device));
    return h->threshold();
}

int m3drec_set_state(m3d_rec* h, const double* field, int i, int j, unsigned long long call) {
    if (!h || !field) return failr(M3D_ERR_ARG, "NULL argument");
    if (i < 0 || j < 0 || j > 201) return failr(M3D_ERR_ARG, "need i >= 0 and 0 <= j <= 201");
    MR_CUDA(cudaSetDevice(h->device));
    MR_CUDA(cudaMemcpyAsync(h->m, field, (size_t)h->xyz * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    const int rc = h->ensure_err(i + 1);
    if (rc) return rc;
    MR_CUDA(cudaMemsetAsync(h->errs, 0, (size_t)h->err_cap * sizeof(double), h->stream));
    MR_CUDA(cudaStreamSynchronize(h->stream));
    h->i = i; h->j = j; h->call = call;
    h->n_recorded = i;
    h->started = true;
    return M3D_OK;
}

int m3drec_get_state(m3d_rec* h, double* field, int* i, int* j, unsigned long long* call) {
    if (!h) return failr(M3D_ERR_ARG, "NULL handle");
    MR_CUDA(cudaSetDevice(h->device));
    if (field) {
        MR_CUDA(cudaMemcpyAsync(field, h->m, (size_t)h->xyz * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
        MR_CUDA(cudaStreamSynchronize(h->stream));
    }
    if (i) *i = h->i;
    if (j) *j = h->j;
    if (call) *call = h->call;
    return M3D_OK;
}

// mTilda's real part (after run: the 0/1 phase field), xyz doubles
int m3drec_get_field(m3d_rec* h, double* out) {
    if (!h || !out) return failr(M3D_ERR_ARG, "NULL argument");
    MR_CUDA(cudaSetDevice(h->device));
    if (!h->real && cudaMalloc(&h->real, (size_t)h->xyz * sizeof(double)) != cudaSuccess) {
        (void)cudaGetLastError();
        h->real = nullptr;
        return failr(M3D_ERR_OOM, "device allocation failed");
    }
    krec_real<<<h->grid1d(), kThreads, 0, h->stream>>>(h->m, h->real, h->xyz);
    h->launches += 1;
    MR_CUDA(cudaGetLastError());
    MR_CUDA(cudaMemcpyAsync(out, h->real, (size_t)h->xyz * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MR_CUDA(cudaStreamSynchronize(h->stream));
    return M3D_OK;
}

// trackrealerrorA: the first min(cap, recorded) errors; *count = recorded
int m3drec_get_error(m3d_rec* h, double* out, int cap, int* count) {
    if (!h) return failr(M3D_ERR_ARG, "NULL handle");
    MR_CUDA(cudaSetDevice(h->device));
    const int k = std::min(std::max(cap, 0), h->n_recorded);
    if (out && k > 0) {
        MR_CUDA(cudaMemcpyAsync(out, h->errs, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        MR_CUDA(cudaStreamSynchronize(h->stream));
    }
    if (count) *count = h->n_recorded;
    return M3D_OK;
}

int m3drec_set_profiling(m3d_rec* h, int on) {
    if (!h) return failr(M3D_ERR_ARG, "NULL handle");
    h->profiling = on != 0;
    for (int k = 0; k < 8; ++k) { h->pass_ms[k] = 0; h->pass_count[k] = 0; }
    return M3D_OK;
}

// summed event times of the host-driven passes: [restart (3 launches), zfwd, yfwd, xturn, yinv, zinv]
int m3drec_profile(const m3d_rec* h, double* ms6, long long* passes) {
    if (!h || !ms6) return failr(M3D_ERR_ARG, "NULL argument");
    for (int k = 0; k < 6; ++k) ms6[k] = h->pass_ms[k];
    if (passes) *passes = h->pass_count[1];
    return M3D_OK;
}

long long m3drec_kernel_launches(const m3d_rec* h) { return h ? h->launches : 0; }
void* m3drec_get_stream(const m3d_rec* h) { return h ? (void*)h->stream : nullptr; }

// recon::fftshift / recon::ifftshift (:47-140): per axis, element k moves to
// (k + s) mod n with s = floor(n / 2) for fftshift and s = floor((n + 1) / 2)
// for ifftshift (the inverse permutation; the two differ for odd n only)
static void shift3(const double* in, double* out, int Nx, int Ny, int Nz, bool inverse) {
    auto sh = [&](int n) { return inverse ? (n + 1) / 2 : n / 2; };
    const int sx = sh(Nx), sy = sh(Ny), sz = sh(Nz);
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y)
            for (int z = 0; z < Nz; ++z)
                out[((size_t)((x + sx) % Nx) * Ny + (y + sy) % Ny) * Nz + (z + sz) % Nz] =
                    in[((size_t)x * Ny + y) * Nz + z];
}

// saveRecImages :403-432: folder/<i+1>.png for every x slice (pixel (j, k) =
// 255 m(x = i, y = j, z = k), an Ny x Nz image -- the reference's Nx x Ny image
// for cubic grids), folder/rve_rec.txt (the field, one value per line) and
// folder/err.txt ("voloum fraction= " + mean, then the errors of passes
// 0 .. numloops-2, 0 past the last pass run)
int m3drec_save_images(m3d_rec* h, const char* folder) {
    if (!h || !folder) return failr(M3D_ERR_ARG, "NULL argument");
    std::vector<double> f((size_t)h->xyz);
    int rc = m3drec_get_field(h, f.data());
    if (rc) return rc;
    std::vector<double> e((size_t)std::max(h->last_n, 0), 0.0);
    int cnt = 0;
    rc = m3drec_get_error(h, e.data(), (int)e.size(), &cnt);
    if (rc) return rc;
    const std::string dir(folder);
    mkdir(dir.c_str(), 0775);
    const int Nx = h->Nx, Ny = h->Ny, Nz = h->Nz;
    std::vector<unsigned char> img((size_t)Ny * Nz);
    for (int i = 0; i < Nx; ++i) {
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k)
                img[j + (size_t)Ny * k] = (unsigned char)(f[k + (size_t)j * Nz + (size_t)i * Ny * Nz] * 255);
        if (!write_png_gray(dir + "/" + std::to_string(i + 1) + ".png", Ny, Nz, img.data()))
            return failr(M3D_ERR_ARG, "cannot write " + dir + "/" + std::to_string(i + 1) + ".png");
    }
    std::ofstream op2(dir + "/rve_rec.txt");
    double sum = 0;
    for (long long v = 0; v < h->xyz; ++v) {
        op2 << f[v] << std::endl;
        sum += f[v];
    }
    sum = sum / h->xyz;
    std::ofstream op1(dir + "/err.txt");
    op1 << "voloum fraction= " << sum << std::endl;
    for (int i = 0; i < h->last_n - 1; ++i) op1 << e[i] << std::endl;
    if (!op1 || !op2) return failr(M3D_ERR_ARG, "cannot write into " + dir);
    return M3D_OK;
}

// vtiWriter :435-470: VTK XML image data with two Float64 components per
// point, (field, tpcf[len]), in flat index order (VTK's x-fastest loop over
// the reference's flat arrays)
int m3drec_write_vti(m3d_rec* h, const char* file, const double* tpcf) {
    if (!h || !file || !tpcf) return failr(M3D_ERR_ARG, "NULL argument");
    std::vector<double> f((size_t)h->xyz);
    int rc = m3drec_get_field(h, f.data());
    if (rc) return rc;
    std::ofstream o(file);
    if (!o) return failr(M3D_ERR_ARG, std::string("cannot open ") + file);
    o << "<?xml version=\"1.0\"?>\n";
    o << "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    o << "  <ImageData WholeExtent=\"0 " << h->Nx - 1 << " 0 " << h->Ny - 1 << " 0 " << h->Nz - 1
      << "\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n";
    o << "    <Piece Extent=\"0 " << h->Nx - 1 << " 0 " << h->Ny - 1 << " 0 " << h->Nz - 1 << "\">\n";
    o << "      <PointData Scalars=\"ImageScalars\">\n";
    o << "        <DataArray type=\"Float64\" Name=\"ImageScalars\" NumberOfComponents=\"2\" format=\"ascii\">\n";
    o.precision(10);
    for (long long v = 0; v < h->xyz; ++v) o << f[v] << " " << tpcf[v] << "\n";
    o << "        </DataArray>\n      </PointData>\n      <CellData/>\n    </Piece>\n  </ImageData>\n</VTKFile>\n";
    if (!o) return failr(M3D_ERR_ARG, std::string("write failed: ") + file);
    return M3D_OK;
}

int m3drec_fftshift(const double* in, double* out, int Nx, int Ny, int Nz) {
    if (!in || !out || in == out || Nx < 1 || Ny < 1 || Nz < 1) return failr(M3D_ERR_ARG, "bad arguments");
    shift3(in, out, Nx, Ny, Nz, false);
    return M3D_OK;
}

int m3drec_ifftshift(const double* in, double* out, int Nx, int Ny, int Nz) {
    if (!in || !out || in == out || Nx < 1 || Ny < 1 || Nz < 1) return failr(M3D_ERR_ARG, "bad arguments");
    shift3(in, out, Nx, Ny, Nz, true);
    return M3D_OK;
}

}  // extern "C"
