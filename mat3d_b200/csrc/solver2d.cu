// solver2d.cu -- the 2-D elastic solver of the reference (FFT_Analysis2D,
// src/2d/FFT_analysis2D.cpp) on the GPU: plane problem with 3 components
// [11, 22, 12] (tensor shear), complex fields, the basic scheme
//     sigma = C(x) eps ; tau = sigma - C0 eps ; eps = IFFT( -Gamma0 : FFT(tau) ), eps^(0) = E
// for a fixed number of iterations, and the 3-load-case homogenization.
//
// Layout: complex FP64 fields component-major, f[c*xy + v], v = y + Ny*x
// (the reference's voxel order).  One iteration = 4 launches: the pointwise
// constitutive step, forward FFTs of the rows (y), the column turnaround (x
// forward FFT, Green operator, x inverse FFT) and inverse FFTs of the rows
// with the 1/xy scaling.  Transforms are the generic shared-memory Stockham
// line FFTs (any length with prime factors up to 32).
//
// The Green operator follows setGF/multiplyGF (:49-137) including their
// conventions: frequencies x <= (Nx-1)/2 positive else -(Ny - x) (x wraps with
// Ny, so non-square grids can hit a zero wave vector away from the origin and
// produce non-finite values exactly as the reference does), y likewise with
// Ny; six independent components per mode; the shear component counted twice.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mat3d_b200.h"
#include "fft_plan.hpp"
#include "fft_smem.cuh"

using namespace m3d;

void m3d_internal_set_error(const std::string& msg);

namespace {

int fail2d(int code, const std::string& msg) {
    m3d_internal_set_error(msg);
    return code;
}

#define M2_CUDA(call)                                                                 \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) return fail2d(M3D_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

struct Consts2D {
    double Cm[9], Ci[9], C0[9];  // row-major 3 x 3
    double d1, d2;               // Green-operator constants (:51-52)
    double2 E[3];                // macroscopic strain (complex)
};

// sigma = C(x) eps ; tau = sigma - C0 eps   (multipCx :106-116, runAnalysis :240)
__global__ void k2d_pointwise(const double2* __restrict__ eps, double2* __restrict__ sig, double2* __restrict__ tau,
                              const uint8_t* __restrict__ phase, Consts2D k, long long xy) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < xy; v += (long long)gridDim.x * blockDim.x) {
        double2 e[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) e[c] = eps[c * xy + v];
        const double* M = phase[v] ? k.Cm : k.Ci;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double sr = 0, si = 0, tr = 0, ti = 0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                sr += M[i * 3 + j] * e[j].x;
                si += M[i * 3 + j] * e[j].y;
                tr += k.C0[i * 3 + j] * e[j].x;
                ti += k.C0[i * 3 + j] * e[j].y;
            }
            sig[i * xy + v] = make_double2(sr, si);
            tau[i * xy + v] = make_double2(sr - tr, si - ti);
        }
    }
}

// 16-byte global -> shared copies that complete asynchronously (zero-filled when !ok)
__device__ __forceinline__ void cp16(void* sdst, const void* gsrc, bool ok) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(ok ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Row FFTs (along y, contiguous): tiles of G lines of length Ny, walked by
// persistent CTAs with three shared buffers -- the next tile streams in by
// cp.async while the current one is transformed.  Inverse rows finish the
// iteration: eps = result / xy (FFTBCKWRD_epsilon :140-145).
// (nbuf = 2 for the longest rows, whose third buffer does not fit: each tile
// is then fetched after the previous one is stored)
__global__ void k2d_rows(double2* __restrict__ buf, double2* __restrict__ eps, const double2* __restrict__ twy,
                         LinePlan py, int G, int nlines, int sign, long long xy, int nbuf) {
    extern __shared__ __align__(16) char smem_raw[];
    const int Ny = py.n;
    const int tsz = G * Ny;
    const int ntiles = (nlines + G - 1) / G;
    double2* tw = (double2*)smem_raw;
    double2* S[3];
    S[0] = tw + Ny;
    S[1] = S[0] + tsz;
    S[2] = S[1] + tsz;
    // a tile's lines are one contiguous run: elements tile * G * Ny ..
    auto valid_of = [&](int tile) { return min(G, nlines - tile * G) * Ny; };
    auto fetch = [&](double2* D, int tile) {
        const long long v0 = (long long)tile * tsz;
        const int valid = valid_of(tile);
        for (int i = threadIdx.x; i < tsz; i += blockDim.x) cp16(D + i, i < valid ? buf + v0 + i : buf, i < valid);
    };
    const bool pre = nbuf == 3;
    int tile = blockIdx.x;
    if (pre && tile < ntiles) fetch(S[0], tile);
    cp_commit();
    for (int i = threadIdx.x; i < Ny; i += blockDim.x) tw[i] = twy[i];
    const LineLayout L{G, G, Ny, 0, 1, false};
    int d = 0;
    for (; tile < ntiles; tile += gridDim.x) {
        if (!pre) {
            __syncthreads();  // the previous tile's stores are done with the buffers
            fetch(S[0], tile);
            cp_commit();
        }
        cp_wait_all();
        __syncthreads();  // tile landed; the previous tile's stores are done with its buffers
        const int f = d == 0 ? 2 : d - 1;
        const int nxt = tile + gridDim.x;
        if (pre) {
            if (nxt < ntiles) fetch(S[f], nxt);
            cp_commit();
        }
        double2* r = fft_lines(S[d], S[d == 2 ? 0 : d + 1], tw, py, L, sign);
        const long long v0 = (long long)tile * tsz;
        const int valid = valid_of(tile);
        if (eps) {
            for (int i = threadIdx.x; i < valid; i += blockDim.x) {
                const double2 w = r[i];
                eps[v0 + i] = make_double2(w.x / (double)xy, w.y / (double)xy);
            }
        } else {
            for (int i = threadIdx.x; i < valid; i += blockDim.x) buf[v0 + i] = r[i];
        }
        if (pre) d = f;
    }
    cp_wait_all();
}

// Column turnaround: TZ consecutive columns y of all Nx rows and 3 components;
// forward FFT along x, -Gamma0 : tau^ per mode (k = 0 -> E * xy), inverse FFT.
__global__ void k2d_cols(double2* __restrict__ buf, const double2* __restrict__ twx, LinePlan px, int Ny, int TZ,
                         Consts2D k, long long xy) {
    extern __shared__ __align__(16) char smem_raw[];
    const int Nx = px.n;
    double2* tw = (double2*)smem_raw;
    double2* A = tw + Nx;  // [c][x][tz]
    double2* B = A + (size_t)3 * Nx * TZ;
    const int y0 = blockIdx.x * TZ;
    for (int i = threadIdx.x; i < Nx; i += blockDim.x) tw[i] = twx[i];
    for (int i = threadIdx.x; i < 3 * Nx * TZ; i += blockDim.x) {
        const int tz = i % TZ, cx = i / TZ, x = cx % Nx, c = cx / Nx;
        const int y = y0 + tz;
        A[i] = y < Ny ? buf[c * xy + (long long)x * Ny + y] : make_double2(0, 0);
    }
    __syncthreads();
    LineLayout L{3 * TZ, TZ, 1, Nx * TZ, TZ, false};
    double2* r = fft_lines(A, B, tw, px, L, -1);
    double2* o = (r == A) ? B : A;
    // Green operator (setGF :49-103, multiplyGF :105-138)
    for (int i = threadIdx.x; i < Nx * TZ; i += blockDim.x) {
        const int tz = i % TZ, x = i / TZ, y = y0 + tz;
        double2 t[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) t[c] = r[(c * Nx + x) * TZ + tz];
        double2 u[3];
        if (x == 0 && y == 0) {
#pragma unroll
            for (int c = 0; c < 3; ++c) u[c] = make_double2(k.E[c].x * (double)xy, k.E[c].y * (double)xy);
        } else {
            const double z[2] = {(double)(x <= (Nx - 1) / 2 ? x : -(Ny - x)), (double)(y <= (Ny - 1) / 2 ? y : -(Ny - y))};
            const double n2 = z[0] * z[0] + z[1] * z[1];
            const int q[6][4] = {{0, 0, 0, 0}, {0, 0, 1, 1}, {0, 0, 0, 1}, {1, 1, 1, 1}, {1, 1, 0, 1}, {0, 1, 0, 1}};
            double gf[6];
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                const int a = q[s][0], b = q[s][1], c = q[s][2], h = q[s][3];
                gf[s] = (k.d1 / n2) * ((c == a ? 1.0 : 0.0) * z[h] * z[b] + (h == a ? 1.0 : 0.0) * z[c] * z[b] +
                                       (c == b ? 1.0 : 0.0) * z[h] * z[a] + (h == b ? 1.0 : 0.0) * z[c] * z[a]) -
                        (k.d2 * z[a] * z[b] * z[c] * z[h]) / (n2 * n2);
            }
            const int w[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                u[j].x = -(gf[w[j][0]] * t[0].x + gf[w[j][1]] * t[1].x + gf[w[j][2]] * t[2].x * 2);
                u[j].y = -(gf[w[j][0]] * t[0].y + gf[w[j][1]] * t[1].y + gf[w[j][2]] * t[2].y * 2);
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) o[(c * Nx + x) * TZ + tz] = u[c];
    }
    __syncthreads();
    double2* s = fft_lines(o, r, tw, px, L, +1);
    for (int i = threadIdx.x; i < 3 * Nx * TZ; i += blockDim.x) {
        const int tz = i % TZ, cx = i / TZ, x = cx % Nx, c = cx / Nx;
        const int y = y0 + tz;
        if (y < Ny) buf[c * xy + (long long)x * Ny + y] = s[i];
    }
}

// per-block sums of the real parts of eps and sigma (6 values)
__global__ void k2d_means(const double2* __restrict__ eps, const double2* __restrict__ sig, long long xy,
                          double* __restrict__ part) {
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < xy; v += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a[c] += eps[c * xy + v].x;
            a[3 + c] += sig[c * xy + v].x;
        }
    __shared__ double red[6][256];
#pragma unroll
    for (int s = 0; s < 6; ++s) red[s][threadIdx.x] = a[s];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int s = 0; s < 6; ++s) {
            double t = 0;
            for (int i = 0; i < (int)blockDim.x; ++i) t += red[s][i];
            part[s * gridDim.x + blockIdx.x] = t;
        }
}

// AoS export: out[(v*3 + c)] = f[c*xy + v]
__global__ void k2d_aos(const double2* __restrict__ f, double2* __restrict__ out, long long xy) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < xy; v += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int c = 0; c < 3; ++c) out[v * 3 + c] = f[c * xy + v];
}

// setLoad(E) :226-233: eps = E everywhere
__global__ void k2d_fill(double2* eps, double2 e0, double2 e1, double2 e2, long long xy) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < xy; v += (long long)gridDim.x * blockDim.x) {
        eps[v] = e0;
        eps[xy + v] = e1;
        eps[2 * xy + v] = e2;
    }
}

void inv3(const double* a, double* o) {
    // Gauss-Jordan with partial pivoting on a row-major 3 x 3
    double m[3][6];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 6; ++j) m[i][j] = j < 3 ? a[i * 3 + j] : (j - 3 == i ? 1.0 : 0.0);
    for (int c = 0; c < 3; ++c) {
        int p = c;
        for (int r = c + 1; r < 3; ++r)
            if (std::fabs(m[r][c]) > std::fabs(m[p][c])) p = r;
        if (p != c)
            for (int j = 0; j < 6; ++j) std::swap(m[c][j], m[p][j]);
        const double d = m[c][c];
        for (int j = 0; j < 6; ++j) m[c][j] /= d;
        for (int r = 0; r < 3; ++r) {
            if (r == c) continue;
            const double f = m[r][c];
            for (int j = 0; j < 6; ++j) m[r][j] -= f * m[c][j];
        }
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) o[i * 3 + j] = m[i][j + 3];
}

}  // namespace

struct m3d_solver2d {
    int Nx = 0, Ny = 0;
    long long xy = 0;
    cudaStream_t stream = nullptr;
    double2 *eps = nullptr, *sig = nullptr, *buf = nullptr, *twx = nullptr, *twy = nullptr;
    uint8_t* phase = nullptr;
    double* part = nullptr;
    LinePlan px{}, py{};
    int G = 1, TZ = 1;
    Consts2D k{};
    bool material_set = false, load_set = false;
    long long launches = 0;
    ~m3d_solver2d() {
        cudaFree(eps); cudaFree(sig); cudaFree(buf); cudaFree(twx); cudaFree(twy); cudaFree(phase); cudaFree(part);
        if (stream) cudaStreamDestroy(stream);
    }
    int rows_nbuf = 3;  // shared buffers of the row passes (3: the next tile prefetched)
    int rows_grid = 1;  // persistent CTAs of the row passes
    size_t rows_smem() const { return (size_t)Ny * 16 + (size_t)rows_nbuf * G * Ny * 16; }
    size_t cols_smem() const { return (size_t)Nx * 16 + 2 * (size_t)3 * Nx * TZ * 16; }
    int iterate() {
        const int nb = 592;
        k2d_pointwise<<<nb, 256, 0, stream>>>(eps, sig, buf, phase, k, xy);
        const int nlines = 3 * Nx;
        k2d_rows<<<rows_grid, 256, rows_smem(), stream>>>(buf, nullptr, twy, py, G, nlines, -1, xy, rows_nbuf);
        k2d_cols<<<(Ny + TZ - 1) / TZ, 256, cols_smem(), stream>>>(buf, twx, px, Ny, TZ, k, xy);
        k2d_rows<<<rows_grid, 256, rows_smem(), stream>>>(buf, eps, twy, py, G, nlines, +1, xy, rows_nbuf);
        launches += 4;
        M2_CUDA(cudaGetLastError());
        return M3D_OK;
    }
};

extern "C" {

int m3d2d_create(int Nx, int Ny, m3d_solver2d** out) {
    if (!out) return fail2d(M3D_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (Nx < 2 || Ny < 2 || Nx > 4096 || Ny > 4096) return fail2d(M3D_ERR_ARG, "grid sizes must be in [2, 4096]");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail2d(M3D_ERR_CUDA, "no CUDA device");
    m3d_solver2d* h = new m3d_solver2d();
    h->Nx = Nx;
    h->Ny = Ny;
    h->xy = (long long)Nx * Ny;
    if (!make_plan(Nx, h->px) || !make_plan(Ny, h->py)) {
        delete h;
        return fail2d(M3D_ERR_UNSUPPORTED, "grid sizes need prime factors <= 32");
    }
    // rows: G lines per CTA in ~48 KB; columns: TZ columns of 3 components in ~96 KB
    h->G = std::max(1, std::min(16, (int)(48 * 1024 / (32 * (size_t)Ny))));
    if ((size_t)Ny * 16 + 3 * (size_t)h->G * Ny * 16 > 220 * 1024) h->rows_nbuf = 2;
    h->TZ = std::max(1, std::min(16, (int)(96 * 1024 / (96 * (size_t)Nx))));
    if (h->rows_smem() > 220 * 1024 || h->cols_smem() > 220 * 1024) {
        delete h;
        return fail2d(M3D_ERR_UNSUPPORTED, "grid too large for the shared-memory line FFTs");
    }
    const size_t f = (size_t)3 * h->xy * sizeof(double2);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&h->eps, f) != cudaSuccess || cudaMalloc(&h->sig, f) != cudaSuccess ||
        cudaMalloc(&h->buf, f) != cudaSuccess || cudaMalloc(&h->phase, (size_t)h->xy) != cudaSuccess ||
        cudaMalloc(&h->part, 6 * 592 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->twx, Nx * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&h->twy, Ny * sizeof(double2)) != cudaSuccess) {
        delete h;
        (void)cudaGetLastError();
        return fail2d(M3D_ERR_OOM, "device allocation failed");
    }
    const auto tx = twiddles<double>(Nx), ty = twiddles<double>(Ny);
    cudaMemcpy(h->twx, tx.data(), Nx * sizeof(double2), cudaMemcpyHostToDevice);
    cudaMemcpy(h->twy, ty.data(), Ny * sizeof(double2), cudaMemcpyHostToDevice);
    cudaMemset(h->eps, 0, f);
    cudaMemset(h->sig, 0, f);
// one limit per kernel for every handle (a per-handle value would lower it
    // under a larger handle made earlier): the device maximum
    for (const void* k : {(const void*)k2d_rows, (const void*)k2d_cols}) {
        cudaFuncAttributes a;
        if (cudaFuncGetAttributes(&a, k) == cudaSuccess)
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024 - (int)a.sharedSizeBytes);
    }
    {
        int per_sm = 0, sms = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2d_rows, 256, h->rows_smem());
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int tiles = (3 * Nx + h->G - 1) / h->G;
        h->rows_grid = std::max(1, std::min(tiles, std::max(1, per_sm) * std::max(1, sms)));
    }
    (void)cudaGetLastError();
    *out = h;
    return M3D_OK;
}

int m3d2d_destroy(m3d_solver2d* h) {
    if (h) {
        cudaStreamSynchronize(h->stream);
        delete h;
    }
    return M3D_OK;
}

// material(properties, RVE) :189-224; props = [E matrix, nu matrix, E inclusion, nu inclusion]
int m3d2d_material(m3d_solver2d* h, const double* props, const int32_t* phase) {
    if (!h || !props || !phase) return fail2d(M3D_ERR_ARG, "NULL argument");
    const double Em = props[0], vm = props[1], Ei = props[2], vi = props[3];
    if (!(Em > 0) || !(Ei > 0) || !(vm > -1 && vm < 0.5) || !(vi > -1 && vi < 0.5))
        return fail2d(M3D_ERR_ARG, "need E > 0 and -1 < nu < 0.5 for both phases");
    const double mum = Em / (1 + vm) / 2, lam = vm * Em / (1 + vm) / (1 - 2 * vm);
    const double mui = Ei / (1 + vi) / 2, lai = vi * Ei / (1 + vi) / (1 - 2 * vi);
    const double Cm[9] = {lam + 2 * mum, lam, 0, lam, lam + 2 * mum, 0, 0, 0, 2 * mum};
    const double Ci[9] = {lai + 2 * mui, lai, 0, lai, lai + 2 * mui, 0, 0, 0, 2 * mui};
    for (int i = 0; i < 9; ++i) {
        h->k.Cm[i] = Cm[i];
        h->k.Ci[i] = Ci[i];
        h->k.C0[i] = 1.0 * (Cm[i] + Ci[i]) / 2.0;
    }
    const double la0 = 1.0 * (lai + lam) / 2.0, mu0 = 1.0 * (mui + mum) / 2.0;
    h->k.d1 = 1 / (4 * mu0);
    h->k.d2 = (la0 + mu0) / (mu0 * (la0 + 2 * mu0));
    // RVE(i) == 1 is the matrix (:110-113)
    std::vector<uint8_t> ph((size_t)h->xy);
    for (long long v = 0; v < h->xy; ++v) ph[v] = phase[v] == 1 ? 1 : 0;
    M2_CUDA(cudaMemcpyAsync(h->phase, ph.data(), (size_t)h->xy, cudaMemcpyHostToDevice, h->stream));
    M2_CUDA(cudaStreamSynchronize(h->stream));
    h->material_set = true;
    return M3D_OK;
}

int m3d2d_set_load(m3d_solver2d* h, const double* E) {
    if (!h || !E) return fail2d(M3D_ERR_ARG, "NULL argument");
    for (int c = 0; c < 3; ++c) h->k.E[c] = make_double2(E[2 * c], E[2 * c + 1]);
    k2d_fill<<<592, 256, 0, h->stream>>>(h->eps, h->k.E[0], h->k.E[1], h->k.E[2], h->xy);
    h->launches += 1;
    M2_CUDA(cudaGetLastError());
    h->load_set = true;
    return M3D_OK;
}

// runAnalysis() :235-247 (the reference runs 25 iterations)
int m3d2d_run(m3d_solver2d* h, int iterations) {
    if (!h) return fail2d(M3D_ERR_ARG, "NULL handle");
    if (!h->material_set || !h->load_set) return fail2d(M3D_ERR_STATE, "material and load must be set first");
    if (iterations < 1 || iterations > 100000) return fail2d(M3D_ERR_ARG, "iterations must be in [1, 100000]");
    for (int i = 0; i < iterations; ++i) {
        const int rc = h->iterate();
        if (rc) return rc;
    }
    M2_CUDA(cudaStreamSynchronize(h->stream));
    return M3D_OK;
}

static int means2d(m3d_solver2d* h, double* m6) {
    k2d_means<<<592, 256, 0, h->stream>>>(h->eps, h->sig, h->xy, h->part);
    h->launches += 1;
    M2_CUDA(cudaGetLastError());
    std::vector<double> p(6 * 592);
    M2_CUDA(cudaMemcpyAsync(p.data(), h->part, p.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    M2_CUDA(cudaStreamSynchronize(h->stream));
    for (int s = 0; s < 6; ++s) {
        double t = 0;
        for (int b = 0; b < 592; ++b) t += p[s * 592 + b];
        m6[s] = t / (double)h->xy;
    }
    return M3D_OK;
}

// homogenization() :250-283: three load cases E(w) = 0.005, each continuing from
// the previous field (the reference does not reset it), CHomo = epHomo^-1 sigHomo.
// Outputs row-major 3 x 3 (any may be NULL).
int m3d2d_homogenize(m3d_solver2d* h, int iterations, double* CHomo, double* epHomo, double* sigHomo) {
    if (!h) return fail2d(M3D_ERR_ARG, "NULL handle");
    if (!h->material_set || !h->load_set) return fail2d(M3D_ERR_STATE, "material and load must be set first");
    double ep[9], sg[9];
    for (int w = 0; w < 3; ++w) {
        for (int c = 0; c < 3; ++c) h->k.E[c] = make_double2(c == w ? 0.005 : 0.0, 0.0);
        int rc = m3d2d_run(h, iterations);
        if (rc) return rc;
        double m[6];
        rc = means2d(h, m);
        if (rc) return rc;
        for (int c = 0; c < 3; ++c) {
            ep[w * 3 + c] = m[c];
            sg[c * 3 + w] = m[3 + c];
        }
    }
    double ei[9], C[9];
    inv3(ep, ei);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int kk = 0; kk < 3; ++kk) s += ei[i * 3 + kk] * sg[kk * 3 + j];
            C[i * 3 + j] = s;
        }
    if (CHomo) std::memcpy(CHomo, C, sizeof(C));
    if (epHomo) std::memcpy(epHomo, ep, sizeof(ep));
    if (sigHomo) std::memcpy(sigHomo, sg, sizeof(sg));
    return M3D_OK;
}

// eps and sigma as the reference stores them: 3 complex values per voxel
// (re, im pairs), voxel order y + Ny*x.  Either pointer may be NULL.
int m3d2d_get_fields(m3d_solver2d* h, double* eps, double* sig) {
    if (!h) return fail2d(M3D_ERR_ARG, "NULL handle");
    const size_t f = (size_t)3 * h->xy * sizeof(double2);
    for (int w = 0; w < 2; ++w) {
        double* out = w ? sig : eps;
        if (!out) continue;
        k2d_aos<<<592, 256, 0, h->stream>>>(w ? h->sig : h->eps, h->buf, h->xy);
        h->launches += 1;
        M2_CUDA(cudaGetLastError());
        M2_CUDA(cudaMemcpyAsync(out, h->buf, f, cudaMemcpyDeviceToHost, h->stream));
        M2_CUDA(cudaStreamSynchronize(h->stream));
    }
    return M3D_OK;
}

long long m3d2d_kernel_launches(const m3d_solver2d* h) { return h ? h->launches : 0; }

void* m3d2d_get_stream(const m3d_solver2d* h) { return h ? (void*)h->stream : nullptr; }

}  // extern "C"
