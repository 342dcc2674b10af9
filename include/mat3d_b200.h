/*
 * mat3d_b200.h -- C ABI of the B200 FFT-homogenization solver (libmat3d_b200.so).
 *
 * Plain C: opaque handle, plain pointers and sizes, int status codes.  The
 * drop-in C++ classes FFT_Analysis3D / FFT_analysis3d_thermal
 * (include/FFT_analysis3D.hpp, include/FFT_thermal3D.hpp) and the Python
 * package are thin layers over these calls.
 *
 * Each entry point replaces a public method of the reference classes
 * (paths are relative to the reference project, FayyazNo/MAT3d):
 *   m3d_create                 FFT_Analysis3D(Nx,Ny,Nz,mater_behav)      include/FFT_analysis3D.hpp:196
 *                              FFT_analysis3d_thermal(Nx,Ny,Nz)          include/FFT_thermal3D.hpp:133
 *   m3d_set_material_mech      FFT_Analysis3D::material(mat,RVE,noPh)    include/FFT_analysis3D.hpp:200
 *   m3d_set_material_thermal   FFT_analysis3d_thermal::material(km,ki,RVE) include/FFT_thermal3D.hpp:138
 *   m3d_set_load               setLoad(E,X0) / setLoad(E)                include/FFT_analysis3D.hpp:202, FFT_thermal3D.hpp:140
 *   m3d_run                    runAnalysis(tol_field,tol_eq[,nInc])      include/FFT_analysis3D.hpp:206, FFT_thermal3D.hpp:145
 *   m3d_homogenize             homogenization(tol_field,tol_eq,name)     include/FFT_analysis3D.hpp:209, FFT_thermal3D.hpp:148
 *   m3d_get_field              public fields epsilon/sigma, tempGradient/heatFlux,
 *                              epsilon_p_eff, d                          include/FFT_analysis3D.hpp:98-99,146,152;
 *                                                                        FFT_thermal3D.hpp:82,92
 *   m3d_get_means / m3d_get_stats / m3d_get_increments
 *                              epHomo/sigHomo, prop_homogenized, the per-iteration
 *                              console report of convergenceCheck        src/3d/FFT_analysis3D.cpp:394-412,722-746
 *   m3d_destroy                ~FFT_Analysis3D / ~FFT_analysis3d_thermal
 *   m3d_get_stream / m3d_set_stream
 *                              no counterpart (the reference is CPU-only); lets a
 *                              caller order the solve on its own CUDA stream
 *   m3d_create_multi / m3d_set_material_mech_rve / m3d_set_material_thermal_rve
 *                              no counterpart: the reference solves one RVE per
 *                              object; these run many RVEs of one grid size in
 *                              one batch, each with the reference's per-RVE
 *                              material() setup (own scheme and reference medium)
 *
 * Layout conventions (as the reference): grid Nx x Ny x Nz, voxel index
 * v = z + Nz*(y + Ny*x); fields exchanged as AoS doubles out[v*c + comp]
 * (the reference's Eigen 6 x N^3 / 3 x N^3 column-major storage); Voigt order
 * [11,22,33,23,13,12] with tensor (not engineering) shear; phase id 1 =
 * matrix, 0 = inclusion.
 *
 * Errors: every call returns an m3d_status; none exits the process.  The
 * message of the last failure on the calling thread is m3d_last_error().
 * Threading: one handle = one CUDA stream; a handle must not be used by two
 * threads at once; different handles are independent.
 */
#ifndef MAT3D_B200_H
#define MAT3D_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define M3D_ABI_VERSION 2

typedef enum {
    M3D_OK = 0,
    M3D_ERR_ARG = 1,           /* invalid argument */
    M3D_ERR_CUDA = 2,          /* CUDA runtime error (no device, launch failure...) */
    M3D_ERR_OOM = 3,           /* device allocation failed */
    M3D_NOT_CONVERGED = 4,     /* iteration cap reached (results still available) */
    M3D_ERR_NAN = 5,           /* non-finite residual */
    M3D_ERR_STATE = 6,         /* call order violated (e.g. run before material) */
    M3D_ERR_UNSUPPORTED = 7,   /* valid request this build does not provide */
    M3D_ERR_TIMEOUT = 8,       /* a bounded device wait expired */
    M3D_PENDING = 9            /* serving: the request has not finished yet */
} m3d_status;

enum { M3D_KIND_MECH = 1, M3D_KIND_THERMAL = 2 };
/* mater_behav "e", "ep", "ed" (src/3d/FFT_analysis3D.cpp:56-98,610-617) */
enum { M3D_BEHAV_ELASTIC = 0, M3D_BEHAV_J2 = 1, M3D_BEHAV_DAMAGE = 2 };
/* arithmetic of the sweeps: FP64; FP32; FP32 sweeps with FP64 defect correction */
enum { M3D_PREC_FP64 = 0, M3D_PREC_FP32 = 1, M3D_PREC_FP32_REFINE = 2 };
/* stop rule: the reference's stationarity test (convergenceCheck), or the
   rms residual |x_c - x| / |E| of the accelerated scheme */
enum { M3D_CRIT_REFERENCE = 0, M3D_CRIT_RESIDUAL = 1 };
/* scheme: automatic as the reference, strain/gradient-based, stress/flux-based */
enum { M3D_SCHEME_AUTO = 0, M3D_SCHEME_PRIMAL = 1, M3D_SCHEME_DUAL = 2 };
/* fields: strain (temperature gradient), stress (heat flux), eq. plastic strain, damage */
enum { M3D_FIELD_STRAIN = 0, M3D_FIELD_STRESS = 1, M3D_FIELD_EPS_P = 2, M3D_FIELD_DAMAGE = 3 };

typedef struct m3d_solver m3d_solver;

typedef struct {
    long long sweeps;        /* all sweeps (FP32 + FP64) of the last run, summed over the batch */
    long long sweeps_fp64;   /* FP64 sweeps among them */
    long long sweeps_fp32;   /* FP32 sweeps among them */
    int iters;               /* sweeps of batch entry 0 in its last solve (reference itNo) */
    int scheme;              /* 1 strain/gradient-based, 2 stress/flux-based */
    int status;              /* status of the last run */
    int n_increments;        /* increments completed (ep/ed) */
    double residual;         /* last residual of entry 0 */
    double eqvar;            /* last reference equilibrium variable of entry 0 */
    double diff_sum;         /* last reference diff_sum_field of entry 0 */
    double diff_eq;          /* last reference diff_avr_eqVar of entry 0 */
    double solve_ms;         /* wall time of the last run/homogenize on the stream */
    double la0, mu0;         /* reference medium (mech) */
    double k0;               /* reference conductivity (thermal) */
    double vol_fraction[16]; /* per phase id */
    long long kernel_launches; /* kernels this handle launched since creation */
    int passes_per_sweep;    /* launches per linear sweep of the last run: 5 (z, y, x, y, z passes) or
                                2 (x turnaround + the y-z slab pass, per-component operators) */
} m3d_stats;

/* Create a solver for an Nx x Ny x Nz grid.  `batch` independent solves
   (load cases) share the phase map and run together. */
int m3d_create(int kind, int Nx, int Ny, int Nz, int behav, int precision, int batch, m3d_solver** out);
/* A linear (elastic or thermal) solver whose batch holds nrve RVEs of one
   grid size with nload load cases each: entry b = r * nload + l solves RVE r.
   Each RVE takes its phase map and properties from the _rve setters below;
   m3d_set_material_mech / _thermal set RVE 0.  m3d_homogenize then runs all
   RVEs (6 or 3 load cases each) and writes nrve consecutive tensors. */
int m3d_create_multi(int kind, int Nx, int Ny, int Nz, int precision, int nrve, int nload, m3d_solver** out);
int m3d_destroy(m3d_solver* h);
/* Device bytes a solver of this shape holds (nrve RVEs, batch entries in all;
   m3d_create: nrve = 1), without the lazily allocated field-export buffer.
   -1 for invalid arguments.  Used for admission by HBM footprint. */
long long m3d_footprint_bytes(int kind, int Nx, int Ny, int Nz, int behav, int precision, int nrve, int batch);

/* Phase properties, rows [E, nu, sigma_y, H, n, P, Y0] (row-major nph x 7), and
   the phase id of every voxel (0 <= id < nph, at most 16 phases). */
int m3d_set_material_mech(m3d_solver* h, const double* mat, int nph, const int32_t* phase, int scheme);
/* km: matrix (id != 0), ki: inclusion (id == 0). */
int m3d_set_material_thermal(m3d_solver* h, double km, double ki, const int32_t* phase, int scheme);
/* The same for RVE r of a multi-RVE solver (0 <= r < nrve). */
int m3d_set_material_mech_rve(m3d_solver* h, int r, const double* mat, int nph, const int32_t* phase, int scheme);
int m3d_set_material_thermal_rve(m3d_solver* h, int r, double km, double ki, const int32_t* phase, int scheme);

/* Load of batch entry b (b = -1: all entries): E has 6 (mech) or 3 (thermal)
   values; X0 (mech, may be NULL) is the stress direction of mixed control. */
int m3d_set_load(m3d_solver* h, int b, const double* E, const double* X0);

/* One analysis of every batch entry (runAnalysis). nInc is the number of load
   increments (ep/ed; ignored for e and thermal).  max_iter <= 0 picks the
   reference's caps (2000 mech, 500 thermal). */
int m3d_run(m3d_solver* h, double tol_field, double tol_eq, int nInc, int criterion, int max_iter);

/* Effective tensor from 6 (mech) / 3 (thermal) load cases run as one batch
   (homogenization).  Ceff, Seff: 36 or 9 doubles, row-major.  ep_means,
   sig_means (optional): the reference's epHomo / sigHomo matrices.  On a
   multi-RVE solver every array holds nrve such blocks, RVE r at r*36 (r*9). */
int m3d_homogenize(m3d_solver* h, double tol_field, double tol_eq, int criterion, int max_iter, double* Ceff,
                   double* Seff, double* ep_means, double* sig_means);

/* Copy a field of batch entry b to host memory: AoS doubles out[v*c + comp]
   (c = 6 mech, 3 thermal; scalar fields: out[v]). */
int m3d_get_field(m3d_solver* h, int which, int b, double* out);
/* As m3d_get_field, but returns once the copy to host memory is enqueued: the
   field is first written, on the device, into the handle's export buffer (the
   state may then be overwritten by the next solve at once) and read into `out`
   on a copy stream of the handle, so the copy overlaps the handle's next work
   (material upload, solve).  `out` must stay valid until m3d_wait_field
   returns, and should be page-locked (pinned) memory, or the copy does not run
   asynchronously.  A later m3d_get_field(_async) on the handle waits for the
   pending copy before reusing the export buffer.  Inelastic fields are copied
   synchronously.  No counterpart in the reference (its fields are host
   arrays); it serves callers that stream results back while solving. */
int m3d_get_field_async(m3d_solver* h, int which, int b, double* out);
/* Wait for the handle's pending m3d_get_field_async copy (no-op if none). */
int m3d_wait_field(m3d_solver* h);
/* Volume averages of the strain-like and stress-like fields of entry b. */
int m3d_get_means(m3d_solver* h, int b, double* strain_mean, double* stress_mean);
int m3d_get_stats(const m3d_solver* h, m3d_stats* out);
/* Entry b's own result of the last linear run (no counterpart in the reference,
   which solves one load case per object): its sweep count (for FP32+FP64
   refinement: FP64 defect sweeps, while *sweeps adds its FP32 sweeps), final
   residual and status. */
int m3d_get_entry_stats(const m3d_solver* h, int b, int* iters, long long* sweeps, double* residual, int* status);
/* Per-increment averages of the ep/ed path (prop_homogenized, nInc x 9). */
int m3d_get_increments(const m3d_solver* h, double* out, int max_rows);

/* Device time of the sweeps, from CUDA events recorded on the handle's stream
   around every sweep while profiling is enabled (off by default).  Sweeps that
   only found converged entries are not counted.  No counterpart in the
   reference, which has no timers. */
typedef struct {
    double ms_fp64;      /* summed device time of FP64 sweeps */
    long long n_fp64;    /* FP64 sweeps timed */
    double ms_fp32;      /* summed device time of FP32 sweeps */
    long long n_fp32;    /* FP32 sweeps timed */
    /* the same time split by pass (events around each pass of the linear
       sweeps): z forward, y forward, x turnaround, y inverse, z inverse; on
       two-pass sweeps (m3d_stats.passes_per_sweep == 2) slot 2 holds the x
       turnaround and slot 4 the y-z slab pass, slots 0, 1 and 3 stay 0 */
    double pass_ms_fp64[5];
    double pass_ms_fp32[5];
} m3d_profile;
int m3d_set_profiling(m3d_solver* h, int enable);  /* enabling also resets the counters */
int m3d_get_profile(const m3d_solver* h, m3d_profile* out);

/* Thermal solve for callers that cannot allocate device memory (they run
   inside another framework's memory pool, or on a serving path that must not
   block on the allocator or fail with out-of-memory half-way).  No
   counterpart in the reference.  Steady conduction on an Nx x Ny x Nz grid,
   FP64, rms-residual stop rule |x_c - x| / |E| < tol, scheme chosen as by
   m3d_set_material_thermal; E is the macroscopic temperature gradient
   (gradient-based scheme) or heat flux (flux-based), as for m3d_set_load.
   The caller passes device pointers: d_phase (V bytes, 0 = inclusion with
   conductivity ki, nonzero = matrix with km) and d_grad (3*V doubles, output,
   component-major: d_grad[c*V + v]).  All working memory is a fixed 32 MiB
   device array inside the library (held by every GPU that loads it until
   exit); grids that need more (beyond about 96^3) are rejected with
   M3D_ERR_ARG.  Every call looks up that array's address with the calling
   device current (so it stays valid after cudaDeviceReset); the first call on
   a device also sets kernel attributes, so make it before any stream
   capture.  Calls share the array: calls that
   overlap on the GPU race, serialise them.  stream: cudaStream_t (NULL = the
   legacy default stream).  Calls no cudaMalloc, cudaFree or allocating
   library routine. */
int m3d_thermal_solve_noalloc(int Nx, int Ny, int Nz, double km, double ki, const uint8_t* d_phase,
                              const double* E, double tol, int max_iter, double* d_grad, int* iters_out,
                              double* residual_out, void* stream);

/* ---- batched homogenization of many RVEs (no counterpart in the reference,
   which homogenizes one RVE per object, src/3d/FFT_analysis3D.cpp:856-903) --
   RVEs of any grid sizes are added, then m3d_batch_homogenize gives each its
   effective tensor, as m3d_homogenize would for it alone (residual stop rule).
   RVEs of one grid size run together as one multi-RVE solve (all their load
   cases in one graph launch); the groups of different grid sizes run
   concurrently (one host thread and CUDA stream each) when they fit the
   device-memory budget together, else one after another, each split only
   where the budget requires.  Each group's handle is created, its materials
   set, its schedule tuned (m3d_batch_set_autotune) and its solve graph
   captured (a one-sweep solve) before the timed launches; device_ms is the
   span from the first group's start to the last group's end on the device,
   wall_ms the whole call. */
typedef struct m3d_batch m3d_batch;
typedef struct {
    long long sweeps, sweeps_fp64, sweeps_fp32;  /* summed over all entries (RVE x load case) */
    long long voxel_iters;   /* sum over entries of voxels x sweeps */
    double device_ms;        /* device time of the solves (events around each launch's homogenize) */
    double wall_ms;          /* wall time of m3d_batch_homogenize, host staging included */
    int rves;                /* RVEs homogenized */
    int groups;              /* distinct grid sizes */
    int launches;            /* multi-RVE solves (groups x memory chunks) */
    long long kernel_launches;
    int autotuned;           /* groups whose launch schedule the autotuner picked */
    int concurrent;          /* 1: the grid-size groups ran at once (one stream each), 0: one after another */
} m3d_batch_stats;
/* mem_budget_bytes <= 0: 85% of the free device memory at creation. */
int m3d_batch_create(int kind, int precision, double mem_budget_bytes, m3d_batch** out);
int m3d_batch_add_mech(m3d_batch* b, int Nx, int Ny, int Nz, const double* mat, int nph, const int32_t* phase,
                       int scheme, int* index);
int m3d_batch_add_thermal(m3d_batch* b, int Nx, int Ny, int Nz, double km, double ki, const int32_t* phase,
                          int scheme, int* index);
/* Ceff, Seff: one C x C block per added RVE, in the order of addition. */
int m3d_batch_homogenize(m3d_batch* b, double tol_field, int max_iter, double* Ceff, double* Seff);
int m3d_batch_get_stats(const m3d_batch* b, m3d_batch_stats* out);
/* on != 0: before the first solve of each grid size, time the launch
   schedules (m3d_autotune, 3 sweeps each) and use the fastest for that size. */
int m3d_batch_set_autotune(m3d_batch* b, int on);
int m3d_batch_clear(m3d_batch* b);
int m3d_batch_destroy(m3d_batch* b);

/* ---- serving (no counterpart in the reference) ------------------------------
   A device-resident request loop: requests of any kind, behaviour, grid and
   precision are submitted from any host thread; worker threads admit them
   as soon as a worker is free and their device footprint fits the memory
   budget (idle solvers of other shapes are released to make room), each on
   its own CUDA stream so the solves of different requests overlap on the
   device.  Finished solvers stay resident (buffers, twiddles, captured
   graphs) and are reused by the next request of the same shape.  A request
   gives the result it would give alone: each runs on its own solver. */
typedef struct m3d_server m3d_server;
typedef struct {
    int kind;             /* M3D_KIND_MECH / M3D_KIND_THERMAL */
    int behav;            /* M3D_BEHAV_* (mech) */
    int Nx, Ny, Nz;
    int precision;        /* M3D_PREC_*; J2/damage: FP64 or FP32 */
    const double* mat;    /* mech: nph x 7 rows as m3d_set_material_mech */
    int nph;
    double km, ki;        /* thermal conductivities */
    const int32_t* phase; /* Nx*Ny*Nz phase ids */
    int scheme;           /* M3D_SCHEME_* */
    const double* E;      /* load: 6 (mech) or 3 (thermal) values */
    const double* X0;     /* J2/damage stress direction (6), else NULL */
    int nInc;             /* J2/damage increments (>= 1) */
    double tol;           /* residual tolerance (M3D_CRIT_RESIDUAL) */
    int max_iter;         /* <= 0: the reference's caps */
    int keep_field;       /* 1: keep the strain field for m3d_serve_get_field */
} m3d_request;
typedef struct {
    int status;                  /* m3d_status of the solve */
    int iters;                   /* sweeps of the (last) solve */
    long long sweeps;            /* all sweeps (FP32 + FP64) */
    double residual;
    double strain_mean[6], stress_mean[6];
    double queue_ms;             /* submit -> admitted */
    double solve_ms;             /* admitted -> finished */
    double latency_ms;           /* submit -> finished */
} m3d_result;
typedef struct {
    long long submitted, completed, failed;
    int queued, running, peak_running;
    int resident_solvers;        /* solvers held (running + idle) */
    double resident_bytes, budget_bytes;
    long long merged_solves;     /* solves that ran several requests as one multi-RVE batch */
    long long merged_requests;   /* requests served by those solves */
} m3d_serve_stats;
/* mem_budget_bytes <= 0: 85% of the free device memory; workers: concurrent solves. */
int m3d_serve_create(double mem_budget_bytes, int workers, m3d_server** out);
/* Copies the request's arrays; thread safe.  ticket > 0 identifies it. */
int m3d_serve_submit(m3d_server* s, const m3d_request* req, long long* ticket);
/* M3D_OK and *out filled once finished (the result is then released unless
   keep_field asked for the field), M3D_PENDING before, M3D_ERR_ARG for an
   unknown ticket. */
int m3d_serve_poll(m3d_server* s, long long ticket, m3d_result* out);
/* Blocks up to timeout_ms (< 0: no limit); M3D_PENDING on timeout. */
int m3d_serve_wait(m3d_server* s, long long ticket, double timeout_ms, m3d_result* out);
/* AoS strain field (c values per voxel) of a finished keep_field request; releases it. */
int m3d_serve_get_field(m3d_server* s, long long ticket, double* out);
int m3d_serve_get_stats(m3d_server* s, m3d_serve_stats* out);
/* Finishes the queued and running requests, then frees every solver. */
int m3d_serve_destroy(m3d_server* s);

/* ---- autotuner (no counterpart in the reference) ----------------------------
   Times the launch schedules that compute the same sweep -- the compile-time
   warp-split FFT kernels or the generic shared-memory ones, the TMA-staged or
   the register-staged y pass, and the generic kernels' tile sizes -- over
   `sweeps` full sweeps of the handle's own batch (after its material is set;
   its field state is overwritten), keeps the fastest on the handle and
   remembers it for the shape and precision.  sweeps = 0 applies the
   remembered schedule without timing (M3D_ERR_STATE if there is none).
   Schedules agree to rounding (the generic and the compile-time FFTs
   associate differently); the y-pass variants agree bitwise. */
typedef struct {
    int fast;         /* 1: compile-time warp-split kernels, 0: generic kernels */
    int tma_y;        /* 1: TMA-staged y pass (compile-time kernels only) */
    int G, tzy, tzx;  /* generic kernels: z lines per CTA, y / x tile columns */
    double sweep_us;  /* measured time of one sweep with this schedule */
    int candidates;   /* schedules timed */
    int slab;         /* 1: two-pass sweeps (x turnaround + y-z slab pass) */
    int schedule;     /* generic line FFTs: order of the radix stages (0 largest odd factor first,
                         1 smallest odd first, 2 powers of two first, 3 radix-4 for the powers of two) */
} m3d_tune;
int m3d_autotune(m3d_solver* h, int sweeps, m3d_tune* out);

/* ---- the 2-D elastic solver -------------------------------------------------
   Replaces FFT_Analysis2D (include/FFT_analysis2D.hpp:20-100,
   src/2d/FFT_analysis2D.cpp): plane problem on an Nx x Ny grid, 3 components
   [11, 22, 12] with tensor shear, complex FP64 fields, the basic scheme for
   a fixed number of iterations (the reference runs 25, :236).  Fields are
   exchanged as the reference stores them: 3 complex values (re, im) per
   voxel, voxel index y + Ny*x.
     m3d2d_create       FFT_Analysis2D(Nx, Ny)                 src/2d/FFT_analysis2D.cpp:3
     m3d2d_material     material(properties, RVE)              :189-224 (props = E_m, nu_m, E_i, nu_i;
                                                                         phase 1 = matrix)
     m3d2d_set_load     setLoad(E)                             :226-233 (E = 3 complex values)
     m3d2d_run          runAnalysis()                          :235-247
     m3d2d_homogenize   homogenization()                       :250-283 (row-major 3 x 3 outputs)
     m3d2d_get_fields   the public fields epsilon, sigma       include/FFT_analysis2D.hpp:35-36 */
typedef struct m3d_solver2d m3d_solver2d;
int m3d2d_create(int Nx, int Ny, m3d_solver2d** out);
int m3d2d_destroy(m3d_solver2d* h);
int m3d2d_material(m3d_solver2d* h, const double* props, const int32_t* phase);
int m3d2d_set_load(m3d_solver2d* h, const double* E);
int m3d2d_run(m3d_solver2d* h, int iterations);
int m3d2d_homogenize(m3d_solver2d* h, int iterations, double* CHomo, double* epHomo, double* sigHomo);
int m3d2d_get_fields(m3d_solver2d* h, double* eps, double* sig);
long long m3d2d_kernel_launches(const m3d_solver2d* h);
void* m3d2d_get_stream(const m3d_solver2d* h);

/* ---- microstructure reconstruction by phase retrieval ---------------------
   Replaces recon::recPlan (include/reconstruction.hpp:46-96,
   src/rec/reconstruction.cpp) built from a full two-point correlation
   function: complex FP64 fields, voxel index z + Nz*(y + Ny*x).
     m3drec_create        recPlan(TPCF, Nx, Ny, Nz)            src/rec/reconstruction.cpp:213-240
                          (normC = sqrt(|TPCF| * xyz))
     m3drec_seed          the seed of the random draws (Eigen setRandom in the
                          reference): draw `call` of voxel v is 2u - 1 with
                          u = (mix(mix(seed * 0x100000001B3 + call) + v) >> 11) * 2^-53,
                          mix = the SplitMix64 finaliser; draw 0 makes the
                          initial field, each restart pass takes the next
     m3drec_run           runRec(n, beta)                      :283-400 (loop + threshold)
     m3drec_get_field     the public member mTilda (real part) include/reconstruction.hpp:74
     m3drec_get_error     the public member trackrealerrorA    include/reconstruction.hpp:73
     m3drec_fftshift      recon::fftshift                      :47-90
     m3drec_ifftshift     recon::ifftshift                     :97-140
     m3drec_create_from_sections
                          recPlan(CImg c1, CImg c2)            :145-206 (8-bit sections, x fastest;
                                                                         both of one size, grid w x h x h)
     m3drec_estimate_norm estimateNormFFT_RVE()                :245-281
     m3drec_save_images   saveRecImages(folder)                :403-432 (PNG slices, rve_rec.txt, err.txt)
     m3drec_write_vti     vtiWriter(file, tpcf)                :435-470
     m3drec_fft3          the example's fftw_plan_dft_3d + fftw_execute (example/reconst3d/main.cpp:85-107)
   Beyond the reference: m3drec_iterate continues the loop from the current
   state without the closing threshold, m3drec_threshold applies it, and
   m3drec_set_state / m3drec_get_state move the complete loop state (field as
   xyz complex (re, im) pairs, counters i and j, draws taken) for checkpoints. */
typedef struct m3d_rec m3d_rec;
int m3drec_create(int Nx, int Ny, int Nz, const double* tpcf, int device, m3d_rec** out);
int m3drec_destroy(m3d_rec* h);
int m3drec_seed(m3d_rec* h, unsigned long long seed);
int m3drec_run(m3d_rec* h, int n, double beta);
int m3drec_iterate(m3d_rec* h, int iters, double beta);
int m3drec_threshold(m3d_rec* h);
int m3drec_set_state(m3d_rec* h, const double* field, int i, int j, unsigned long long call);
int m3drec_get_state(m3d_rec* h, double* field, int* i, int* j, unsigned long long* call);
int m3drec_get_field(m3d_rec* h, double* out);
int m3drec_get_error(m3d_rec* h, double* out, int cap, int* count);
/* Per-kernel event timing (host-driven passes instead of the graph) and the
   summed times [restart transform, zfwd, yfwd, xturn, yinv, zinv] in ms. */
int m3drec_set_profiling(m3d_rec* h, int on);
int m3drec_profile(const m3d_rec* h, double* ms6, long long* passes);
long long m3drec_kernel_launches(const m3d_rec* h);
void* m3drec_get_stream(const m3d_rec* h);
int m3drec_create_from_sections(const unsigned char* c1, int w1, int h1, const unsigned char* c2, int w2, int h2,
                                int device, m3d_rec** out);
int m3drec_estimate_norm(m3d_rec* h);
int m3drec_get_norm(m3d_rec* h, double* out);
int m3drec_save_images(m3d_rec* h, const char* folder);
int m3drec_write_vti(m3d_rec* h, const char* file, const double* tpcf);
int m3drec_fft3(const double* in, double* out, int Nx, int Ny, int Nz, int sign, int device);
int m3drec_fftshift(const double* in, double* out, int Nx, int Ny, int Nz);
int m3drec_ifftshift(const double* in, double* out, int Nx, int Ny, int Nz);

/* The CUDA stream (cudaStream_t) all work of the handle is ordered on.
   m3d_set_stream replaces it with a caller-owned stream (NULL: the handle's own). */
void* m3d_get_stream(const m3d_solver* h);
int m3d_set_stream(m3d_solver* h, void* stream);

const char* m3d_status_string(int status);
const char* m3d_last_error(void);
int m3d_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
