// solver_inelastic.inl -- host driver of the J2 / damage path (included by solver.cu).
//
// Increment loop of runAnalysis ep/ed (src/3d/FFT_analysis3D.cpp:796-853):
//   dE = E / nInc; eps = dE everywhere (setLoad); for each increment:
//   constitutive; sweeps until the stop rule; softening stop (ed);
//   export_homogen_var; update_old_Variable.

void InelasticState::free_all() {
    cudaFree(eps); cudaFree(sig); cudaFree(eps_old); cudaFree(sig_old); cudaFree(ep); cudaFree(dmg);
    cudaFree(d_ph); cudaFree(d_S0); cudaFree(d_nrfail);
    eps = sig = eps_old = sig_old = ep = dmg = nullptr;
    d_ph = nullptr; d_S0 = nullptr; d_nrfail = nullptr;
    batch = 0;
}

int InelasticState::setup(m3d_solver* h) {
    free_all();
    const size_t w = 8;  // FP64 state in both precisions (the transforms carry the precision)
    const size_t V = (size_t)h->g.V, B = (size_t)h->B;
    M3D_CUDA(cudaMalloc(&eps, B * 6 * V * w));
    M3D_CUDA(cudaMalloc(&sig, B * 6 * V * w));
    M3D_CUDA(cudaMalloc(&eps_old, B * 6 * V * w));
    if (h->behav == M3D_BEHAV_J2) {
        M3D_CUDA(cudaMalloc(&sig_old, B * 6 * V * w));
        M3D_CUDA(cudaMalloc(&ep, B * V * w));
    } else {
        M3D_CUDA(cudaMalloc(&dmg, B * V * w));
    }
    std::vector<PhaseMech> ph(h->nph);
    for (int p = 0; p < h->nph; ++p) {
        for (int i = 0; i < 36; ++i) ph[p].C[i] = h->Cp[p][i];
        const double El = h->mat[p * 7 + 0], nu = h->mat[p * 7 + 1];
        ph[p].mu = El / (1 + nu) / 2.;
        ph[p].Sy = h->mat[p * 7 + 2];
        ph[p].H = h->mat[p * 7 + 3];
        ph[p].n = h->mat[p * 7 + 4];
        ph[p].P = h->mat[p * 7 + 5];
        ph[p].Y0 = h->mat[p * 7 + 6];
    }
    M3D_CUDA(cudaMalloc(&d_ph, ph.size() * sizeof(PhaseMech)));
    M3D_CUDA(cudaMemcpy(d_ph, ph.data(), ph.size() * sizeof(PhaseMech), cudaMemcpyHostToDevice));
    M3D_CUDA(cudaMalloc(&d_S0, 36 * sizeof(double)));
    M3D_CUDA(cudaMemcpy(d_S0, h->S0.data(), 36 * sizeof(double), cudaMemcpyHostToDevice));
    M3D_CUDA(cudaMalloc(&d_nrfail, sizeof(int)));
    batch = B;
    return M3D_OK;
}

template <typename TX>
__global__ void k_colsum(const TX* __restrict__ x, int C, int b, long long V, double* __restrict__ part) {
    double acc[6] = {};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < C; ++c) acc[c] += (double)x[((long long)b * C + c) * V + v];
    __shared__ double red[32 * 6];
    block_reduce_store<6>(acc, red, part, 0, gridDim.x, blockIdx.x);
}

template <typename TX>
static int colsum_mean(m3d_solver* h, const void* x, int C, int b, double* out) {
    const int nblk = 296;
    k_colsum<TX><<<nblk, 256, 0, h->stream>>>((const TX*)x, C, b, h->g.V, h->d_part);
    h->st.kernel_launches += 1;
    M3D_CUDA(cudaGetLastError());
    std::vector<double> hp((size_t)nblk * 6);
    M3D_CUDA(cudaMemcpyAsync(hp.data(), h->d_part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    M3D_CUDA(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < C; ++c) {
        double s = 0;
        for (int i = 0; i < nblk; ++i) s += hp[(size_t)c * nblk + i];
        out[c] = s / (double)h->g.V;
    }
    return M3D_OK;
}

int InelasticState::means(m3d_solver* h, int b, double* strain_mean, double* stress_mean) {
    const bool f32 = false;  // FP64 state
    int rc = M3D_OK;
    if (strain_mean) rc = f32 ? colsum_mean<float>(h, eps, 6, b, strain_mean) : colsum_mean<double>(h, eps, 6, b, strain_mean);
    if (rc) return rc;
    if (stress_mean) rc = f32 ? colsum_mean<float>(h, sig, 6, b, stress_mean) : colsum_mean<double>(h, sig, 6, b, stress_mean);
    return rc;
}

template <typename TX>
__global__ void k_copy_scalar(const TX* __restrict__ x, int b, long long V, double* __restrict__ out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x)
        out[v] = (double)x[(long long)b * V + v];
}

int InelasticState::get_field(m3d_solver* h, int which, int b, double* out) {
    const bool f32 = false;  // FP64 state
    if (which == M3D_FIELD_STRAIN)
        return f32 ? export_field<float, 6>(h, eps, nullptr, b, out) : export_field<double, 6>(h, eps, nullptr, b, out);
    if (which == M3D_FIELD_STRESS)
        return f32 ? export_field<float, 6>(h, sig, nullptr, b, out) : export_field<double, 6>(h, sig, nullptr, b, out);
    void* s = (which == M3D_FIELD_EPS_P) ? ep : (which == M3D_FIELD_DAMAGE ? dmg : nullptr);
    if (!s) return fail(M3D_ERR_ARG, "field not available for this behaviour");
    const long long V = h->g.V;
    if (!h->d_out) {
        if (cudaMalloc(&h->d_out, (size_t)6 * V * sizeof(double)) != cudaSuccess) return fail(M3D_ERR_OOM, "export buffer");
    }
    if (f32) k_copy_scalar<float><<<592, 256, 0, h->stream>>>((const float*)s, b, V, h->d_out);
    else k_copy_scalar<double><<<592, 256, 0, h->stream>>>((const double*)s, b, V, h->d_out);
    h->st.kernel_launches += 1;
    M3D_CUDA(cudaGetLastError());
    M3D_CUDA(cudaMemcpyAsync(out, h->d_out, (size_t)V * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    M3D_CUDA(cudaStreamSynchronize(h->stream));
    return M3D_OK;
}

template <typename T>
__global__ void k_fill(T* x, long long n, T v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) x[i] = v;
}

template <typename T, int CC>
int m3d_solver::run_inelastic(double tol_field, double tol_eq, int nInc, int criterion, int max_iter) {
    typedef typename Cx<T>::t C2;
    static_assert(CC == 6, "inelastic path is mechanical");
    const long long V = g.V;
    const int bj = (behav == M3D_BEHAV_J2) ? BEHAV_J2 : BEHAV_DAMAGE;
    typedef double S;  // state type (FP64 in both precisions)
    S* eps = (S*)in.eps;
    S* sig = (S*)in.sig;
    S* eps_old = (S*)in.eps_old;
    S* sig_old = (S*)in.sig_old;
    S* ep = (S*)in.ep;
    S* dmg = (S*)in.dmg;
    C2* sp = (C2*)d_spec;
    // initial state: eps = dE, sig = eps_old = sig_old = 0, eps_p = 1.236547e-9 (:56-98, :799)
    std::vector<double> dE((size_t)B * 6);
    for (int b = 0; b < B; ++b)
        for (int c = 0; c < 6; ++c) dE[b * 6 + c] = E[b * 6 + c] / (nInc * 1.);
    for (int b = 0; b < B; ++b)
        for (int c = 0; c < 6; ++c)
            k_fill<S><<<256, 256, 0, stream>>>(eps + ((long long)b * 6 + c) * V, V, dE[b * 6 + c]);
    M3D_CUDA(cudaMemsetAsync(sig, 0, (size_t)B * 6 * V * sizeof(S), stream));
    M3D_CUDA(cudaMemsetAsync(eps_old, 0, (size_t)B * 6 * V * sizeof(S), stream));
    if (sig_old) M3D_CUDA(cudaMemsetAsync(sig_old, 0, (size_t)B * 6 * V * sizeof(S), stream));
    if (ep) k_fill<S><<<256, 256, 0, stream>>>(ep, (long long)B * V, 1.236547e-9);
    st.kernel_launches += (long long)B * 6 + (ep ? 1 : 0);
    if (dmg) M3D_CUDA(cudaMemsetAsync(dmg, 0, (size_t)B * V * sizeof(S), stream));
    M3D_CUDA(cudaMemsetAsync(in.d_nrfail, 0, sizeof(int), stream));

    for (int b = 0; b < B; ++b) {
        Ctl c;
        std::memset(&c, 0, sizeof(c));
        c.max_iter = max_iter;
        c.tol_field = tol_field;
        c.tol_eq = tol_eq;
        c.crit_residual = (criterion == M3D_CRIT_RESIDUAL);
        double en = 0;
        for (int i = 0; i < 6; ++i) en += ((i >= 3) ? 2.0 : 1.0) * dE[b * 6 + i] * dE[b * 6 + i];
        c.enorm = en > 0 ? std::sqrt(en) : 1.0;
        c.den = den_ref;
        set_green(c, 0);
        const double* X = &X0[b * 6];
        double y[6];
        for (int i = 0; i < 6; ++i) {
            double s = 0;
            for (int j = 0; j < 6; ++j) s += S0[i * 6 + j] * X[j];
            y[i] = s;
            c.aux[AUX_X0 + i] = X[i];
            c.aux[AUX_S0 + i] = y[i];
        }
        c.aux[AUX_PXY] = y[0] * X[0] + y[1] * X[1] + y[2] * X[2] + 2 * (y[3] * X[3] + y[4] * X[4] + y[5] * X[5]);
        if (c.aux[AUX_PXY] == 0) return fail(M3D_ERR_ARG, "X0 must be a nonzero stress direction for ep/ed");
        for (int i = 0; i < 6; ++i) c.E[i] = dE[b * 6 + i];
        h_ctl[b] = c;
    }
    int t_comp = 0;
    for (int j = 0; j < 6; ++j)
        if (X0[j] != 0) { t_comp = j; break; }

    InelasticPtrs<S> P{d_phase, eps, sig, eps_old, sig_old, ep, dmg, V, in.d_ph, nph, bj, in.d_nrfail};
    EpiConstitutive<T> cons{P, nullptr};
    EpiBasic<T> epi{cons};
    ProStress<T> pro{sig, V};
    // FP32 transforms under the residual rule: transform the load step's
    // stress increment (J2 keeps the previous step's stress)
    if (sizeof(T) == 4 && criterion == M3D_CRIT_RESIDUAL && sig_old) pro.sig_old = sig_old;
    SpecBasic<T> spec{green<T, 6>(0), SpecEqVar<T, 6>{g}};
    const size_t phb = (size_t)nph * sizeof(PhaseMech) + 64;
    const int cblk = 592;
    const size_t csmem = 32 * 32 * 8 + phb;
    allow_smem(k_constitutive<T>);
    allow_smem(k_commit);
    prop.assign((size_t)nInc * 9, 0.0);
    long long total = 0;
    int nx = 0, done_inc = nInc, status = M3D_OK;
    const int chunk = 8;
    for (int inc = 0; inc < nInc; ++inc) {
        for (int b = 0; b < B; ++b) {
            double s = 0;
            for (int i = 0; i < 6; ++i) s += dE[b * 6 + i];
            h_ctl[b].done = 0;
            h_ctl[b].iters = 0;
            h_ctl[b].aux[AUX_DESUM] = s * (inc + 1);
        }
        M3D_CUDA(cudaMemcpyAsync(d_ctl, h_ctl, B * sizeof(Ctl), cudaMemcpyHostToDevice, stream));
        k_constitutive<T><<<dim3(cblk, B), 256, csmem, stream>>>(cons, d_ctl, d_part);
        k_finalize_j2<<<B, 256, 0, stream>>>(d_ctl, d_part, 13, cblk, POLJ2_START, (double)V, in.d_S0);
        st.kernel_launches += 2;
        int before = 0;
        for (;;) {
            for (int k = 0; k < chunk; ++k) {
                prof_mark(k);
                prof_pass(0);
                pass_zfwd<T, 6>(pro, d_ctl, sp);
                prof_pass(1);
                pass_y<T>(-1, 6, d_ctl, sp);
                prof_pass(2);
                const int xblk = pass_x<T, 6>(spec, d_ctl, sp);
                if (criterion == M3D_CRIT_REFERENCE) {
                    k_finalize_j2<<<B, 256, 0, stream>>>(d_ctl, d_part, 2, xblk, POLJ2_CHECK, (double)V, in.d_S0);
                    st.kernel_launches += 1;
                }
                prof_pass(3);
                pass_y<T>(+1, 6, d_ctl, sp);
                prof_pass(4);
                pass_zinv<T, 6>(epi, d_ctl, sp, FinJ2{POLJ2_SWEEP, (double)V, in.d_S0, d_counter});
                prof_pass(5);
            }
            M3D_CUDA(cudaGetLastError());
            prof_mark(chunk);
            int rc = sync_ctl(d_ctl);
            if (rc) return rc;
            prof_collect(max_iters() - before, sizeof(T) == 8);
            before = max_iters();
            bool all = true;
            for (int b = 0; b < B; ++b) all = all && h_ctl[b].done;
            if (all) break;
        }
        for (int b = 0; b < B; ++b) {
            total += h_ctl[b].iters;
            if (h_ctl[b].status == 1 && status == M3D_OK) status = M3D_NOT_CONVERGED;
            if (h_ctl[b].status == 2) status = M3D_ERR_NAN;
        }
        // softening stop (:829-847), on the increment's fresh averages
        std::vector<double> cur(6, 0.0);
        {
            double sm[6];
            int rc = in.means(this, 0, nullptr, sm);
            if (rc) return rc;
            for (int j = 0; j < 6; ++j) cur[j] = sm[j];
        }
        if (behav == M3D_BEHAV_DAMAGE && inc != 0) {
            for (int j = 0; j < 6; ++j)
                if (X0[j] != 0 && cur[j] < prop[(size_t)(inc - 1) * 9 + 1 + j]) nx += 1;
        }
        if (nx == 3) { done_inc = inc; break; }
        // export_homogen_var + update_old_Variable (entry 0 is reported)
        k_commit<<<dim3(cblk, B), 256, csmem, stream>>>(P, eps_old, sig_old, ep, t_comp, d_part);
        st.kernel_launches += 1;
        M3D_CUDA(cudaGetLastError());
        std::vector<double> hp((size_t)cblk * 9);
        M3D_CUDA(cudaMemcpyAsync(hp.data(), d_part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
        M3D_CUDA(cudaStreamSynchronize(stream));
        for (int k = 0; k < 9; ++k) {
            double s = 0;
            for (int i = 0; i < cblk; ++i) s += hp[(size_t)k * cblk + i];
            prop[(size_t)inc * 9 + k] = s / (double)V;
        }
        if (behav == M3D_BEHAV_DAMAGE) prop[(size_t)inc * 9 + 8] = 0;
    }
    int nrfail = 0;
    M3D_CUDA(cudaMemcpy(&nrfail, in.d_nrfail, sizeof(int), cudaMemcpyDeviceToHost));
    st.sweeps = total;
    if (sizeof(T) == 8) { st.sweeps_fp64 = total; st.sweeps_fp32 = 0; } else { st.sweeps_fp32 = total; st.sweeps_fp64 = 0; }
    st.iters = h_ctl[0].iters;
    st.residual = h_ctl[0].residual;
    st.eqvar = h_ctl[0].eqvar;
    st.diff_sum = h_ctl[0].diff_sum;
    st.diff_eq = h_ctl[0].diff_eq;
    st.n_increments = done_inc;
    prop.resize((size_t)done_inc * 9);
    if (nrfail) return fail(M3D_ERR_NAN, "J2 Newton-Raphson did not converge in some voxel");
    return status;
}
