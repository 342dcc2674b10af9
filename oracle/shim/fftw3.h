/*
 * oracle/shim/fftw3.h -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
 *
 * Stand-in for the subset of FFTW 3 (third-party, not vendored with the
 * reference, version unpinned by its CMakeLists.txt:40-44) that the
 * reference solver sources call, so that those sources compile unmodified:
 *   src/3d/FFT_analysis3D.cpp:101-150,253,261-263,268,276,354,1137-1142
 *   src/3dTherm/FFT_thermal3D.cpp:31-89,216,223,306,760-763
 *
 * What is restated is FFTW's published contract for the guru64 interface:
 *   r2c:  Y[k] = sum_n x[n] exp(-2 pi i k.n / N)  over a rank-r grid, the last
 *         dimension halved to n/2+1 outputs; unnormalised.
 *   c2r:  x[n] = sum_k Y[k] exp(+2 pi i k.n / N) with the missing half taken
 *         from Hermitian symmetry along the last dimension; unnormalised.
 *         Complex passes run over the leading dimensions first and the
 *         1-D c2r along the last dimension runs last, so the imaginary parts
 *         of its DC and Nyquist bins are ignored (FFTW's hc2r codelets read
 *         only their real parts).  Numerically this is the real part of the
 *         full inverse DFT of the Hermitian extension.
 *   dims[i].n / .is / .os and howmany_dims give element strides.
 * The arithmetic is a project-written mixed-radix decimation-in-time FFT
 * (factors 4, 2, 3, 5 and a direct DFT for any other prime), twiddles from
 * long-double sin/cos, threaded over lines with OpenMP using the thread
 * count set by fftw_plan_with_nthreads (3 in the reference).
 * Only the calls listed above are provided.
 */
#ifndef M3D_ORACLE_FFTW3_SHIM_H
#define M3D_ORACLE_FFTW3_SHIM_H

#include <cstddef>
#include <cstring>
#include <cmath>
#include <vector>
#include <complex>
#include <omp.h>

typedef double fftw_complex[2];

typedef struct {
    std::ptrdiff_t n;
    std::ptrdiff_t is;
    std::ptrdiff_t os;
} fftw_iodim64;

#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE (0U)

namespace m3d_fftw_shim {

typedef std::complex<double> cplx;

/* One 1-D complex transform of length n (any n >= 1), forward sign -1. */
struct Line1D {
    int n = 0;
    std::vector<int> factors;
    std::vector<cplx> tw; /* tw[j] = exp(-2 pi i j / n) */

    void init(int n_) {
        n = n_;
        factors.clear();
        int m = n;
        while (m % 4 == 0) { factors.push_back(4); m /= 4; }
        while (m % 2 == 0) { factors.push_back(2); m /= 2; }
        for (int p = 3; p * p <= m; p += 2)
            while (m % p == 0) { factors.push_back(p); m /= p; }
        if (m > 1) factors.push_back(m);
        if (factors.empty()) factors.push_back(1);
        tw.resize(n);
        const long double two_pi = 6.283185307179586476925286766559L;
        for (int j = 0; j < n; ++j) {
            long double a = -two_pi * (long double)j / (long double)n;
            tw[j] = cplx((double)cosl(a), (double)sinl(a));
        }
    }

    /* Recursive DIT: out[0..len) = DFT_len of in[0], in[stride], ...
       level twiddle w_len^a = tw[a * tws] with tws = n / len. */
    void rec(const cplx* in, cplx* out, int len, int stride, int fi, int tws, int sign) const {
        if (len == 1) { out[0] = in[0]; return; }
        const int p = factors[fi];
        const int m = len / p;
        for (int q = 0; q < p; ++q)
            rec(in + (std::ptrdiff_t)q * stride, out + q * m, m, stride * p, fi + 1, tws * p, sign);
        cplx tmp[64];
        std::vector<cplx> big;
        cplx* t = tmp;
        if (p > 64) { big.resize(p); t = big.data(); }
        for (int k = 0; k < m; ++k) {
            for (int q = 0; q < p; ++q) {
                cplx w = tw[(std::size_t)((long long)q * k % len) * tws];
                if (sign > 0) w = std::conj(w);
                t[q] = out[q * m + k] * w;
            }
            if (p == 2) {
                out[k] = t[0] + t[1];
                out[k + m] = t[0] - t[1];
            } else if (p == 4) {
                cplx a0 = t[0] + t[2], a1 = t[0] - t[2];
                cplx b0 = t[1] + t[3], b1 = t[1] - t[3];
                /* multiply b1 by -i (forward) or +i (inverse) */
                cplx b1r = (sign < 0) ? cplx(b1.imag(), -b1.real()) : cplx(-b1.imag(), b1.real());
                out[k] = a0 + b0;
                out[k + m] = a1 + b1r;
                out[k + 2 * m] = a0 - b0;
                out[k + 3 * m] = a1 - b1r;
            } else {
                for (int s = 0; s < p; ++s) {
                    cplx acc(0.0, 0.0);
                    for (int q = 0; q < p; ++q) {
                        cplx w = tw[(std::size_t)((long long)q * s % p) * (std::size_t)m * tws];
                        if (sign > 0) w = std::conj(w);
                        acc += t[q] * w;
                    }
                    out[k + s * m] = acc;
                }
            }
        }
    }

    void exec(const cplx* in, cplx* out, int sign) const { rec(in, out, n, 1, 0, 1, sign); }
};

struct Plan {
    int kind = 0; /* 0 = r2c, 1 = c2r, 2 = c2c forward, 3 = c2c backward (cin -> cbuf) */
    fftw_complex* cin = nullptr;
    int rank = 0;
    std::vector<fftw_iodim64> dims;
    std::vector<fftw_iodim64> howmany;
    double* rbuf = nullptr;
    fftw_complex* cbuf = nullptr;
    int nthreads = 1;
    std::vector<Line1D> lines;
};

inline int& nthreads_setting() {
    static int nt = 1;
    return nt;
}

/* Iterate over every index of the dims except dimension `skip`, calling f(offset_in, offset_out). */
template <class F>
inline void for_each_line(const std::vector<fftw_iodim64>& d, const std::vector<std::ptrdiff_t>& is,
                          const std::vector<std::ptrdiff_t>& os, const std::vector<std::ptrdiff_t>& ext,
                          int skip, int nthreads, F f) {
    const int r = (int)d.size();
    std::ptrdiff_t total = 1;
    for (int i = 0; i < r; ++i)
        if (i != skip) total *= ext[i];
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (std::ptrdiff_t lin = 0; lin < total; ++lin) {
        std::ptrdiff_t rem = lin, oi = 0, oo = 0;
        for (int i = r - 1; i >= 0; --i) {
            if (i == skip) continue;
            std::ptrdiff_t idx = rem % ext[i];
            rem /= ext[i];
            oi += idx * is[i];
            oo += idx * os[i];
        }
        f(oi, oo);
    }
}

inline void execute(Plan* p) {
    const int r = p->rank;
    const std::ptrdiff_t nlast = p->dims[r - 1].n;
    const std::ptrdiff_t hlast = nlast / 2 + 1;
    std::ptrdiff_t hm_n = 1, hm_is = 0, hm_os = 0;
    if (!p->howmany.empty()) { hm_n = p->howmany[0].n; hm_is = p->howmany[0].is; hm_os = p->howmany[0].os; }
    const int nt = p->nthreads;

    for (std::ptrdiff_t h = 0; h < hm_n; ++h) {
        if (p->kind >= 2) {
            /* complex to complex: gather the input (input strides), scatter it
               to the output strides, then in-place 1-D transforms along every
               dimension of the output */
            const fftw_complex* in = p->cin + h * hm_is;
            fftw_complex* out = p->cbuf + h * hm_os;
            const int sign = (p->kind == 2) ? -1 : +1;
            std::vector<std::ptrdiff_t> is(r), os(r), ext(r);
            for (int i = 0; i < r; ++i) { is[i] = p->dims[i].is; os[i] = p->dims[i].os; ext[i] = p->dims[i].n; }
            {
                std::ptrdiff_t total = 1;
                for (int i = 0; i < r; ++i) total *= ext[i];
                std::vector<cplx> tmp((std::size_t)total);
                for (std::ptrdiff_t lin = 0; lin < total; ++lin) {
                    std::ptrdiff_t rem = lin, oi = 0;
                    for (int i = r - 1; i >= 0; --i) { oi += (rem % ext[i]) * is[i]; rem /= ext[i]; }
                    tmp[(std::size_t)lin] = cplx(in[oi][0], in[oi][1]);
                }
                for (std::ptrdiff_t lin = 0; lin < total; ++lin) {
                    std::ptrdiff_t rem = lin, oo = 0;
                    for (int i = r - 1; i >= 0; --i) { oo += (rem % ext[i]) * os[i]; rem /= ext[i]; }
                    out[oo][0] = tmp[(std::size_t)lin].real();
                    out[oo][1] = tmp[(std::size_t)lin].imag();
                }
            }
            for (int ax = r - 1; ax >= 0; --ax) {
                const Line1D& L = p->lines[ax];
                const std::ptrdiff_t n = p->dims[ax].n, s = p->dims[ax].os;
                for_each_line(p->dims, os, os, ext, ax, nt, [&](std::ptrdiff_t oi, std::ptrdiff_t) {
                    std::vector<cplx> a(n), b(n);
                    for (std::ptrdiff_t j = 0; j < n; ++j) a[j] = cplx(out[oi + j * s][0], out[oi + j * s][1]);
                    L.exec(a.data(), b.data(), sign);
                    for (std::ptrdiff_t j = 0; j < n; ++j) { out[oi + j * s][0] = b[j].real(); out[oi + j * s][1] = b[j].imag(); }
                });
            }
            continue;
        }
        if (p->kind == 0) {
            const double* in = p->rbuf + h * hm_is;
            fftw_complex* out = p->cbuf + h * hm_os;
            /* 1) real lines along the last dim -> half spectrum */
            {
                std::vector<std::ptrdiff_t> is(r), os(r), ext(r);
                for (int i = 0; i < r; ++i) { is[i] = p->dims[i].is; os[i] = p->dims[i].os; ext[i] = p->dims[i].n; }
                const Line1D& L = p->lines[r - 1];
                const std::ptrdiff_t sis = p->dims[r - 1].is, sos = p->dims[r - 1].os;
                for_each_line(p->dims, is, os, ext, r - 1, nt, [&](std::ptrdiff_t oi, std::ptrdiff_t oo) {
                    std::vector<cplx> a(nlast), b(nlast);
                    for (std::ptrdiff_t j = 0; j < nlast; ++j) a[j] = cplx(in[oi + j * sis], 0.0);
                    L.exec(a.data(), b.data(), -1);
                    for (std::ptrdiff_t j = 0; j < hlast; ++j) {
                        out[oo + j * sos][0] = b[j].real();
                        out[oo + j * sos][1] = b[j].imag();
                    }
                });
            }
            /* 2) complex passes over the leading dims, in place on the output */
            for (int ax = r - 2; ax >= 0; --ax) {
                std::vector<std::ptrdiff_t> os(r), ext(r);
                for (int i = 0; i < r; ++i) { os[i] = p->dims[i].os; ext[i] = p->dims[i].n; }
                ext[r - 1] = hlast;
                const Line1D& L = p->lines[ax];
                const std::ptrdiff_t n = p->dims[ax].n, s = p->dims[ax].os;
                for_each_line(p->dims, os, os, ext, ax, nt, [&](std::ptrdiff_t oi, std::ptrdiff_t) {
                    std::vector<cplx> a(n), b(n);
                    for (std::ptrdiff_t j = 0; j < n; ++j) a[j] = cplx(out[oi + j * s][0], out[oi + j * s][1]);
                    L.exec(a.data(), b.data(), -1);
                    for (std::ptrdiff_t j = 0; j < n; ++j) { out[oi + j * s][0] = b[j].real(); out[oi + j * s][1] = b[j].imag(); }
                });
            }
        } else {
            fftw_complex* in = p->cbuf + h * hm_is;
            double* out = p->rbuf + h * hm_os;
            /* 1) complex inverse passes over the leading dims, in place on the input
                  (FFTW's c2r may overwrite its input by default, too) */
            for (int ax = 0; ax <= r - 2; ++ax) {
                std::vector<std::ptrdiff_t> is(r), ext(r);
                for (int i = 0; i < r; ++i) { is[i] = p->dims[i].is; ext[i] = p->dims[i].n; }
                ext[r - 1] = hlast;
                const Line1D& L = p->lines[ax];
                const std::ptrdiff_t n = p->dims[ax].n, s = p->dims[ax].is;
                for_each_line(p->dims, is, is, ext, ax, nt, [&](std::ptrdiff_t oi, std::ptrdiff_t) {
                    std::vector<cplx> a(n), b(n);
                    for (std::ptrdiff_t j = 0; j < n; ++j) a[j] = cplx(in[oi + j * s][0], in[oi + j * s][1]);
                    L.exec(a.data(), b.data(), +1);
                    for (std::ptrdiff_t j = 0; j < n; ++j) { in[oi + j * s][0] = b[j].real(); in[oi + j * s][1] = b[j].imag(); }
                });
            }
            /* 2) 1-D c2r along the last dim: Hermitian extension, DC/Nyquist imaginary parts dropped */
            {
                std::vector<std::ptrdiff_t> is(r), os(r), ext(r);
                for (int i = 0; i < r; ++i) { is[i] = p->dims[i].is; os[i] = p->dims[i].os; ext[i] = p->dims[i].n; }
                const Line1D& L = p->lines[r - 1];
                const std::ptrdiff_t sis = p->dims[r - 1].is, sos = p->dims[r - 1].os;
                for_each_line(p->dims, is, os, ext, r - 1, nt, [&](std::ptrdiff_t oi, std::ptrdiff_t oo) {
                    std::vector<cplx> a(nlast), b(nlast);
                    for (std::ptrdiff_t j = 0; j < hlast; ++j) a[j] = cplx(in[oi + j * sis][0], in[oi + j * sis][1]);
                    a[0] = cplx(a[0].real(), 0.0);
                    if (nlast % 2 == 0) a[nlast / 2] = cplx(a[nlast / 2].real(), 0.0);
                    for (std::ptrdiff_t j = hlast; j < nlast; ++j) a[j] = std::conj(a[nlast - j]);
                    L.exec(a.data(), b.data(), +1);
                    for (std::ptrdiff_t j = 0; j < nlast; ++j) out[oo + j * sos] = b[j].real();
                });
            }
        }
    }
}

} /* namespace m3d_fftw_shim */

typedef m3d_fftw_shim::Plan* fftw_plan;

inline int fftw_init_threads(void) { return 1; }
inline void fftw_plan_with_nthreads(int n) { m3d_fftw_shim::nthreads_setting() = n > 0 ? n : 1; }
inline void fftw_cleanup(void) {}
inline void fftw_cleanup_threads(void) {}

inline fftw_plan m3d_fftw_make_plan(int kind, int rank, const fftw_iodim64* dims, int howmany_rank,
                                    const fftw_iodim64* howmany_dims, double* r, fftw_complex* c) {
    m3d_fftw_shim::Plan* p = new m3d_fftw_shim::Plan();
    p->kind = kind;
    p->rank = rank;
    p->dims.assign(dims, dims + rank);
    if (howmany_rank > 0) p->howmany.assign(howmany_dims, howmany_dims + howmany_rank);
    p->rbuf = r;
    p->cbuf = c;
    p->nthreads = m3d_fftw_shim::nthreads_setting();
    p->lines.resize(rank);
    for (int i = 0; i < rank; ++i) p->lines[i].init((int)dims[i].n);
    return p;
}

inline fftw_plan fftw_plan_guru64_dft_r2c(int rank, const fftw_iodim64* dims, int howmany_rank,
                                          const fftw_iodim64* howmany_dims, double* in, fftw_complex* out,
                                          unsigned) {
    return m3d_fftw_make_plan(0, rank, dims, howmany_rank, howmany_dims, in, out);
}

inline fftw_plan fftw_plan_guru64_dft_c2r(int rank, const fftw_iodim64* dims, int howmany_rank,
                                          const fftw_iodim64* howmany_dims, fftw_complex* in, double* out,
                                          unsigned) {
    return m3d_fftw_make_plan(1, rank, dims, howmany_rank, howmany_dims, out, in);
}

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

inline fftw_plan fftw_plan_guru64_dft(int rank, const fftw_iodim64* dims, int howmany_rank,
                                      const fftw_iodim64* howmany_dims, fftw_complex* in, fftw_complex* out, int sign,
                                      unsigned) {
    fftw_plan p = m3d_fftw_make_plan(sign < 0 ? 2 : 3, rank, dims, howmany_rank, howmany_dims, nullptr, out);
    p->cin = in;
    return p;
}

/* row-major complex transforms (last index fastest), in -> out */
inline fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign, unsigned f) {
    const fftw_iodim64 d[3] = {{n0, (std::ptrdiff_t)n1 * n2, (std::ptrdiff_t)n1 * n2}, {n1, n2, n2}, {n2, 1, 1}};
    return fftw_plan_guru64_dft(3, d, 0, nullptr, in, out, sign, f);
}
inline fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned f) {
    const fftw_iodim64 d[2] = {{n0, n1, n1}, {n1, 1, 1}};
    return fftw_plan_guru64_dft(2, d, 0, nullptr, in, out, sign, f);
}

inline void fftw_execute(const fftw_plan p) { m3d_fftw_shim::execute(p); }
inline void fftw_destroy_plan(fftw_plan p) { delete p; }

#endif
