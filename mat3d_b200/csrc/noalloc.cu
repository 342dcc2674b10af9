// noalloc.cu -- a thermal solve that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool or arena (which owns all device memory and forbids
// outside allocations), real-time or serving paths that must never block on
// the allocator or fail half-way with an out-of-memory error, and embedded
// uses that want a fixed, known memory footprint.  For them,
// m3d_thermal_solve_noalloc runs the same Lippmann-Schwinger sweeps as the
// handle API (FP64, the rms-residual stop rule) on device buffers the caller
// already owns, and keeps all of its own working memory -- half spectrum,
// per-block partial sums, control block, twiddle and phase tables -- in one
// file-scope device array of kScratchBytes (32 MiB).  That array exists on
// every GPU that loads this library, from module load until process exit.
//
// Rules of use:
//  * Every call looks up the array's device address with
//    cudaGetSymbolAddress, with the calling device current (nothing is cached,
//    so the address stays right after cudaDeviceReset reloads the module);
//    the first call on a device also sets the kernels' shared-memory limits.
//    Make that first call before any stream capture.
//  * All calls share the one array and it keeps the last call's contents;
//    every call clears what must start at zero itself.  Calls that overlap on
//    the GPU (two streams, or two host threads) race on the array: serialise
//    them.
//  * Grids whose working set exceeds the array are rejected with
//    M3D_ERR_ARG and a message giving the limit (about 96^3 here).
// It calls no cudaMalloc, cudaFree or allocating library routine.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mat3d_b200.h"
#include "physics.cuh"

using namespace m3d;

void m3d_internal_set_error(const std::string& msg);

namespace {

constexpr size_t kScratchBytes = (size_t)32 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_noalloc_mu;
bool g_noalloc_attrs[kMaxDevices] = {};  // kernel attributes set on this device (guarded by g_noalloc_mu)

int nfail(int st, const std::string& msg) {
    m3d_internal_set_error("m3d_thermal_solve_noalloc: " + msg);
    return st;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

bool plan_of(int n, LinePlan& p) {
    std::vector<int> f;
    int m = n;
    while (m % 8 == 0) { f.push_back(8); m /= 8; }
    while (m % 4 == 0) { f.push_back(4); m /= 4; }
    while (m % 2 == 0) { f.push_back(2); m /= 2; }
    for (int q = 3; q <= m; q += 2)
        while (m % q == 0) { f.push_back(q); m /= q; }
    if ((int)f.size() > kMaxStages) return false;
    for (int r : f)
        if (r > kMaxGenericRadix) return false;
    p.n = n;
    p.nstages = (int)f.size();
    for (int i = 0; i < kMaxStages; ++i) p.radix[i] = i < (int)f.size() ? f[i] : 1;
    return true;
}

// phase ids -> 0 (inclusion) / 1 (matrix, any nonzero id), and the sum of the
// raw ids (the reference's RVE.sum(), which picks the scheme)
__global__ void k_noalloc_phase(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, long long V,
                                unsigned long long* idsum) {
    unsigned long long c = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        const uint8_t id = in[v];
        out[v] = id != 0;
        c += id;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(idsum, c);
}

__global__ void k_noalloc_fill(double* x, long long V, double e0, double e1, double e2) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        x[v] = e0;
        x[V + v] = e1;
        x[2 * V + v] = e2;
    }
}

// flux -> gradient (g = q / k) in place, for the flux-based scheme
__global__ void k_noalloc_to_grad(double* x, const uint8_t* __restrict__ ph, long long V, double rki, double rkm) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        const double r = ph[v] ? rkm : rki;
        x[v] *= r;
        x[V + v] *= r;
        x[2 * V + v] *= r;
    }
}

template <class K>
void allow_dyn(K kernel) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, kernel) == cudaSuccess)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024 - (int)a.sharedSizeBytes);
    (void)cudaGetLastError();
}

}  // namespace

extern "C" int m3d_thermal_solve_noalloc(int Nx, int Ny, int Nz, double km, double ki, const uint8_t* d_phase,
                                         const double* E, double tol, int max_iter, double* d_grad, int* iters_out,
                                         double* residual_out, void* stream_ptr) {
    if (!d_phase || !E || !d_grad) return nfail(M3D_ERR_ARG, "NULL argument");
    if (Nx < 2 || Ny < 2 || Nz < 2 || Nx > 1024 || Ny > 1024 || Nz > 1024) return nfail(M3D_ERR_ARG, "grid sizes must be in [2, 1024]");
    if (!(km > 0) || !(ki > 0)) return nfail(M3D_ERR_ARG, "conductivities must be positive");
    if (!(tol > 0)) return nfail(M3D_ERR_ARG, "tol must be positive");
    if (max_iter <= 0) max_iter = 500;
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    LinePlan px, py, pz;
    if (!plan_of(Nx, px) || !plan_of(Ny, py) || !plan_of(Nz, pz))
        return nfail(M3D_ERR_UNSUPPORTED, "grid sizes need prime factors <= 32");

    GridDims g;
    g.Nx = Nx; g.Ny = Ny; g.Nz = Nz;
    g.Hz = Nz / 2 + 1;
    g.Hzp = (g.Hz + 1) & ~1;
    g.V = (long long)Nx * Ny * Nz;
    g.NL = (long long)Nx * Ny;
    constexpr int C = 3;
    // launch geometry of the generic passes (as the handle API picks it)
    int G = (int)(48 * 1024 / ((size_t)C * Nz * sizeof(double2)));
    G = std::max(2, std::min(16, G)) & ~1;
    auto pick_tz = [](int ncomp, int n, int maxtz) {
        int tz = maxtz;
        while (tz > 1 && 2 * (size_t)ncomp * n * tz * sizeof(double2) > 64 * 1024) tz >>= 1;
        return tz;
    };
    const int TZy = pick_tz(1, Ny, 8), TZx = pick_tz(C, Nx, 8);
    const int zblk = (int)((g.NL + G - 1) / G);

    // scratch layout
    const size_t o_spec = 0;
    const size_t o_part = up256(o_spec + (size_t)C * g.NL * g.Hzp * sizeof(double2));
    const size_t o_ctl = up256(o_part + (size_t)zblk * 2 * sizeof(double));
    const size_t o_cnt = up256(o_ctl + sizeof(Ctl));
    const size_t o_ones = up256(o_cnt + sizeof(int));
    const size_t o_tw = up256(o_ones + sizeof(unsigned long long));
    const size_t o_mats = up256(o_tw + (size_t)(Nx + Ny + Nz) * sizeof(double2));
    const size_t o_ph = up256(o_mats + 64 * sizeof(double));
    const size_t need = up256(o_ph + (size_t)g.V);
    if (need > kScratchBytes)
        return nfail(M3D_ERR_ARG, "grid " + std::to_string(Nx) + "x" + std::to_string(Ny) + "x" + std::to_string(Nz) +
                                      " needs " + std::to_string(need >> 20) + " MiB of scratch; the limit is " +
                                      std::to_string(kScratchBytes >> 20) + " MiB (about 96^3)");

    // the array's device address, looked up with the calling device current
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nfail(M3D_ERR_CUDA, "no current CUDA device");
    unsigned char* base = nullptr;
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return nfail(M3D_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        base = (unsigned char*)p;
    }
    double2* spec = (double2*)(base + o_spec);
    double* part = (double*)(base + o_part);
    Ctl* ctl = (Ctl*)(base + o_ctl);
    int* counter = (int*)(base + o_cnt);
    unsigned long long* idsum = (unsigned long long*)(base + o_ones);
    double2* tw = (double2*)(base + o_tw);
    double* mats = (double*)(base + o_mats);
    uint8_t* ph = base + o_ph;

#define NA_CUDA(call)                                                                                   \
    do {                                                                                                \
        const cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return nfail(M3D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

    // what must start at zero: the completion counter and the id sum
    NA_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), stream));
    NA_CUDA(cudaMemsetAsync(idsum, 0, sizeof(unsigned long long), stream));
    k_noalloc_phase<<<296, 256, 0, stream>>>(d_phase, ph, g.V, idsum);
    NA_CUDA(cudaGetLastError());
    unsigned long long ids = 0;
    NA_CUDA(cudaMemcpyAsync(&ids, idsum, sizeof(ids), cudaMemcpyDeviceToHost, stream));
    NA_CUDA(cudaStreamSynchronize(stream));

    // scheme (the reference's integer-division rule on the raw id sum,
    // src/3dTherm/FFT_thermal3D.cpp:399-410, as m3d_set_material_thermal)
    const long long vol_1 = (long long)ids / g.V;
    const int scheme = ((vol_1 >= 1 && km > ki) || (vol_1 < 1 && km < ki)) ? 1 : 2;
    const double k0 = std::sqrt(ki * km);
    const double kk[2] = {ki, km};
    double hm[64] = {};
    // P (2 x 3x3) at 0, A (2 x 3x3) at 18, Osum (2 x 3) at 36
    for (int p = 0; p < 2; ++p) {
        const double k = kk[p];
        double pv, av, ov;
        if (scheme == 1) { pv = k - k0; av = 2 * k0 / (k + k0); ov = k; }
        else { const double r = 1 / k, r0 = 1 / k0; pv = r - r0; av = 2 * r0 / (r + r0); ov = r; }
        for (int i = 0; i < 3; ++i) {
            hm[p * 9 + i * 4] = pv;
            hm[18 + p * 9 + i * 4] = av;
            hm[36 + p * 3 + i] = ov;
        }
    }
    std::vector<double2> htw((size_t)Nx + Ny + Nz);
    {
        const long double two_pi = 6.283185307179586476925286766559L;
        size_t o = 0;
        for (int n : {Nx, Ny, Nz})
            for (int m = 0; m < n; ++m, ++o) {
                const long double a = -two_pi * (long double)m / (long double)n;
                htw[o].x = (double)cosl(a);
                htw[o].y = (double)sinl(a);
            }
    }
    Ctl hc;
    std::memset(&hc, 0, sizeof(hc));
    hc.max_iter = max_iter;
    hc.tol_field = tol;
    double en = 0;
    for (int i = 0; i < 3; ++i) {
        hc.E[i] = E[i];
        hc.kzero[i] = E[i] * (double)g.V;
        en += E[i] * E[i];
    }
    hc.enorm = en > 0 ? std::sqrt(en) : 1.0;
    hc.gxw = Nx;
    if (scheme == 1) { hc.gkind = GREEN_TGRAD; hc.gnyq = 1; hc.gp1 = 1.0 / k0; }
    else { hc.gkind = GREEN_TFLUX; hc.gxw = Ny; hc.gp1 = k0; }
    NA_CUDA(cudaMemcpyAsync(mats, hm, sizeof(hm), cudaMemcpyHostToDevice, stream));
    NA_CUDA(cudaMemcpyAsync(tw, htw.data(), htw.size() * sizeof(double2), cudaMemcpyHostToDevice, stream));
    NA_CUDA(cudaMemcpyAsync(ctl, &hc, sizeof(hc), cudaMemcpyHostToDevice, stream));
    k_noalloc_fill<<<296, 256, 0, stream>>>(d_grad, g.V, E[0], E[1], E[2]);

    ProMat<double, C> pro{ph, d_grad, g.V, mats, 2, nullptr};
    SpecGreen<double, C> sg;
    sg.g = g;
    sg.zero_k0 = 0;
    sg.xwrap = Nx;
    sg.pos_nyq = 0;
    if (scheme == 1) { sg.kind = GREEN_TGRAD; sg.pos_nyq = 1; sg.p1 = 1.0 / k0; }
    else { sg.kind = GREEN_TFLUX; sg.xwrap = Ny; sg.p1 = k0; }
    sg.p2 = 0;
    EpiEM<double, C> epi{ph, d_grad, nullptr, g.V, mats + 18, mats + 36, 2, nullptr};
    FinLinear fin{POL_RESIDUAL, (double)g.V, nullptr, counter};

    const size_t extra = 2 * (C * C + C) * sizeof(double) + 64;
    const size_t zsmem = (size_t)Nz * sizeof(double2) + 2 * (size_t)(G / 2) * C * Nz * sizeof(double2) + 16 + 32 * 32 * 8 + extra;
    const size_t ysmem = (size_t)Ny * sizeof(double2) + 2 * (size_t)Ny * TZy * sizeof(double2);
    const size_t xsmem = (size_t)Nx * sizeof(double2) + 2 * (size_t)C * Nx * TZx * sizeof(double2) + 16 + 32 * 32 * 8;
    const int ntzy = (g.Hzp + TZy - 1) / TZy, ntzx = (g.Hzp + TZx - 1) / TZx;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);  // kernel attributes are per device
        if (!g_noalloc_attrs[dev]) {
            allow_dyn(k_zfwd<double, C, ProMat<double, C>>);
            allow_dyn(k_ypass<double>);
            allow_dyn(k_xturn<double, C, SpecGreen<double, C>>);
            allow_dyn(k_zinv<double, C, EpiEM<double, C>, FinLinear>);
            g_noalloc_attrs[dev] = true;
        }
    }
    const double2* twx = tw;
    const double2* twy = tw + Nx;
    const double2* twz = tw + Nx + Ny;
    for (;;) {
        for (int k = 0; k < 8; ++k) {
            k_zfwd<double, C, ProMat<double, C>><<<dim3(zblk, 1), 256, zsmem, stream>>>(g, pz, twz, spec, pro, ctl, G, part);
            k_ypass<double><<<dim3(Nx * ntzy, C), 256, ysmem, stream>>>(g, py, twy, spec, TZy, C, -1, ctl);
            k_xturn<double, C, SpecGreen<double, C>><<<dim3(Ny * ntzx, 1), 256, xsmem, stream>>>(g, px, twx, spec, TZx, sg, ctl, part);
            k_ypass<double><<<dim3(Nx * ntzy, C), 256, ysmem, stream>>>(g, py, twy, spec, TZy, C, +1, ctl);
            k_zinv<double, C, EpiEM<double, C>, FinLinear><<<dim3(zblk, 1), 256, zsmem, stream>>>(g, pz, twz, spec, epi, ctl, G, part, fin);
        }
        NA_CUDA(cudaGetLastError());
        NA_CUDA(cudaMemcpyAsync(&hc, ctl, sizeof(hc), cudaMemcpyDeviceToHost, stream));
        NA_CUDA(cudaStreamSynchronize(stream));
        if (hc.done) break;
    }
    if (scheme == 2) {
        k_noalloc_to_grad<<<296, 256, 0, stream>>>(d_grad, ph, g.V, 1.0 / ki, 1.0 / km);
        NA_CUDA(cudaGetLastError());
        NA_CUDA(cudaStreamSynchronize(stream));
    }
#undef NA_CUDA
    if (iters_out) *iters_out = hc.iters;
    if (residual_out) *residual_out = hc.residual;
    if (hc.status == 2) return nfail(M3D_ERR_NAN, "non-finite residual");
    if (hc.status == 1) return M3D_NOT_CONVERGED;
    return M3D_OK;
}
