/*
 * askja_gpu.h -- C ABI of the askja B200 engine (libaskja_b200.so).
 *
 * A drop-in for the HMC path of paro8929/askja.  The reference has no FFI: its
 * in-process seam is a set of global-state functions in sun.cpp operating on
 * the globals u, U, pi, Pi, uconf (sun.cpp:82-89).  Each entry point below
 * names the reference routine it replaces.  A context owns the device copy of
 * those globals plus one CUDA stream; all work is ordered on that stream.
 *
 * Conventions
 *  - Every call returns ASKJA_OK (0) or a negative ASKJA_ERR_* status; the
 *    message is available from askja_last_error().  Nothing aborts or exits
 *    and no C++ exception crosses the ABI.  (The reference prints and sets a
 *    global ABORT flag: sun.cpp:48, 934-935, 1053-1054.)
 *  - Host field buffers use the reference's U-conf byte order
 *    (sun.cpp:289-302, gsl_matrix_complex_fwrite per link):
 *        [site][dir][row][col][re,im]   as doubles,
 *    i.e. V*DIM*NC*NC*2 doubles, site index with x0 slowest
 *    (structs.h:130-165).  Buffers are caller-owned and copied synchronously.
 *  - There is no CPU fallback: askja_create fails when no CUDA device is
 *    present or the kernels cannot load.
 *  - One host thread per context.
 */
#ifndef ASKJA_GPU_H
#define ASKJA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define ASKJA_API __attribute__((visibility("default")))
#else
#define ASKJA_API
#endif

#define ASKJA_OK 0
#define ASKJA_ERR_ARG (-1)         /* invalid argument or unsupported shape */
#define ASKJA_ERR_CUDA (-2)        /* a CUDA call failed (message says which) */
#define ASKJA_ERR_IO (-3)          /* file missing, short or unwritable */
#define ASKJA_ERR_NONFINITE (-4)   /* NaN/Inf in an uploaded host buffer */
#define ASKJA_ERR_NODEVICE (-5)    /* no CUDA device */
#define ASKJA_ERR_PARSE (-6)       /* malformed params file */

#define ASKJA_FP64 0 /* links, momenta and arithmetic in FP64 (the reference's precision) */
#define ASKJA_FP32 1 /* FP32-mixed: FP32 arithmetic, FP64 reductions and dH.  NC <= 4 (automatic
                        kernel path): links and momenta carry bfloat16 residual planes, the
                        kick and link update accumulate into them exactly, links are projected
                        onto SU(NC) in FP64 before every trajectory (residual-plane mode).
                        NC > 4 or kernel paths 1/3: FP32 fields, reunitarised per update. */
#define ASKJA_FP32_LEAN 2 /* FP32 fields without residual planes for every NC, reunitarised per
                             update (the FP32 storage of ASKJA_FP32 for NC > 4) */

#define ASKJA_MAX_DIM 16
#define ASKJA_MAX_NC 64

typedef struct askja_ctx askja_ctx;

/* Lattice and integrator settings: the params-file keys NC, DIM, N0..N{DIM-1},
 * BETA, DT, LEVEL (sun.cpp:803-888) plus the engine's own precision/seed. */
typedef struct {
  int nc;              /* NC, 2..64 */
  int dim;             /* DIM, 1..16 */
  int n[ASKJA_MAX_DIM];/* N0..N{DIM-1}, each >= 1 */
  double beta;         /* BETA */
  double dt;           /* DT (used by askja_trajectory) */
  int level;           /* LEVEL: Taylor order of exp(i dt P); outside 0..8 acts as 8 (sunmat.h:215-246) */
  int precision;       /* ASKJA_FP64, ASKJA_FP32 or ASKJA_FP32_LEAN */
  int reunitarise;     /* -1 default (on for FP32, off for FP64), 0 off, 1 on.  On: every
                          link update is projected back onto SU(NC); the FP32 row kernels
                          (NC > 4) and tensor cores project onto U(NC) per update and
                          askja_trajectory / askja_run_trajectories run the full SU(NC)
                          projection before every 10th trajectory */
  int device;          /* CUDA device ordinal */
  int kernel_path;     /* 0 automatic; 1 row-per-thread kernels for every NC (testing);
                          2 tensor cores (FP32 with NC = 16, 32 or 64 and DIM >= 2 only);
                          3 site pairs in packed FP32 (NC = 3, FP32, DIM >= 2 and
                            an even extent N{DIM-1} only) */
  uint64_t seed;       /* Philox key for momenta, Metropolis uniforms and hot start */
} askja_params;

/* Outcome of one trajectory (sun.cpp:1249-1318). */
typedef struct {
  double h_old;        /* CRITENERGY: beta*(EnergyMag + simpleenergyEl(pi)/(2 NC)) before */
  double h_new;        /* myenergy after the closing half kick */
  double dh;           /* h_new - h_old */
  double u;            /* Metropolis uniform */
  int accepted;        /* 0 reject, 1 "ACCEPT case 1" (dH<0), 2 "ACCEPT case 2" */
  int pad;
  unsigned long long traj;                  /* trajectories run by this context */
  unsigned long long n_acc, n_acc1, n_rej;  /* NACC, NAC1, NREC (sun.cpp:42-45) */
  unsigned long long n_tot;                 /* NTOT */
} askja_traj_result;

/* ---- lifetime ---------------------------------------------------------- */
/* Allocates the device fields (u, pi, Pi, uconf and a second link buffer) and
 * neighbour tables; replaces allocate_memory/xygrid.init/generators
 * (sun.cpp:96-125, structs.h:109-147, sun.cpp:142-189). */
ASKJA_API int askja_create(const askja_params* p, askja_ctx** out);
ASKJA_API void askja_destroy(askja_ctx* ctx);
ASKJA_API const char* askja_last_error(const askja_ctx* ctx); /* ctx may be NULL: last create() error */
ASKJA_API const char* askja_version(void);
ASKJA_API long askja_volume(const askja_ctx* ctx);            /* V = prod N_d (xygrid.SIZE) */
ASKJA_API void* askja_stream(askja_ctx* ctx);                 /* the context's cudaStream_t */
ASKJA_API int askja_sync(askja_ctx* ctx);

/* ---- fields (U-conf layout) ------------------------------------------- */
/* u := conf and uconf := conf (loadconf + takeconfiguration, sun.cpp:744-765,
 * 1164-1170).  Rejects non-finite input with ASKJA_ERR_NONFINITE. */
ASKJA_API int askja_set_links(askja_ctx* ctx, const double* conf);
/* The same upload without blocking the host (not in the reference): the
 * host->device copy runs on a copy stream into one of two device staging
 * buffers (used in turn), overlapping the work already enqueued on the
 * context's stream; the conversion into u and uconf is ordered after that
 * work, so a trajectory enqueued next starts from conf.  Returns once the
 * copy is enqueued.  conf should be page-locked (askja_host_alloc) and must
 * stay unchanged until a synchronising call (askja_sync, askja_trajectory,
 * a getter) has returned.  Non-finite input is counted on the device and
 * reported as ASKJA_ERR_NONFINITE by the next synchronising call (u then
 * holds the converted values). */
ASKJA_API int askja_set_links_async(askja_ctx* ctx, const double* conf);
ASKJA_API int askja_get_links(askja_ctx* ctx, double* conf);          /* current u */
ASKJA_API int askja_get_saved_links(askja_ctx* ctx, double* conf);    /* uconf (what storeconf writes, sun.cpp:289-302) */
/* which = 0: pi (current momenta), 1: Pi (updated momenta).  Momenta are
 * Hermitian (P_ij = conj(P_ji), real diagonal) as the reference's are; the
 * FP32 SU(3) link update relies on it (P^2, tr P and det P are formed from
 * the real diagonal and the upper triangle).  The residual-plane mode stores
 * momenta as coordinates of Hermitian traceless matrices: an uploaded matrix
 * is replaced by its Hermitian traceless part. */
ASKJA_API int askja_set_momenta(askja_ctx* ctx, int which, const double* conf);
ASKJA_API int askja_get_momenta(askja_ctx* ctx, int which, double* conf);
ASKJA_API int askja_initializeU(askja_ctx* ctx);                       /* cold start, sun.cpp:194-207; also uconf */
ASKJA_API int askja_hot_start(askja_ctx* ctx, uint64_t seed);          /* Haar SU(NC) links (not in the reference); also uconf */
/* pi := sqrt(2NC/beta) sum_a xi_a T_a with Philox normals keyed by (seed,
 * counter): replaces initializeE (sun.cpp:209-252), whose GSL stream is
 * time-seeded and not reproducible. */
ASKJA_API int askja_initializeE(askja_ctx* ctx, uint64_t seed, uint64_t counter);

/* ---- the reference's in-process seam ---------------------------------- */
ASKJA_API int askja_updateE(askja_ctx* ctx, double eps);              /* Pi = pi - eps*Adjoint(staples): sun.cpp:672-723 */
ASKJA_API int askja_updateUandcopyDown(askja_ctx* ctx, double eps);   /* u = mexpi(eps*Pi,L)*u; pi = Pi: sun.cpp:774-790 */
ASKJA_API int askja_copyDown(askja_ctx* ctx);                         /* pi = Pi: sun.cpp:792-801 */
ASKJA_API int askja_takeconfiguration(askja_ctx* ctx);                /* uconf = u: sun.cpp:725-732 */
ASKJA_API int askja_loadconfiguration(askja_ctx* ctx);                /* u = uconf: sun.cpp:734-742 */
ASKJA_API int askja_reunitarise(askja_ctx* ctx);                      /* project u onto SU(NC) (not in the reference) */
ASKJA_API int askja_EnergyMag(askja_ctx* ctx, double* out);           /* sun.cpp:507-537 */
ASKJA_API int askja_simpleenergyEl(askja_ctx* ctx, int which, double* out); /* sun.cpp:540-548, which 0 = pi, 1 = Pi */
ASKJA_API int askja_EnergyEl(askja_ctx* ctx, double* out);            /* sun.cpp:560-567 */
ASKJA_API int askja_TotalEnergy(askja_ctx* ctx, double* out);         /* sun.cpp:571-576 */
ASKJA_API int askja_GaussLaw(askja_ctx* ctx, double* out);            /* sun.cpp:415-438 */
ASKJA_API int askja_UViol(askja_ctx* ctx, double* out);               /* sun.cpp:441-471 */
ASKJA_API int askja_WilsonLoop(askja_ctx* ctx, double* out);          /* sun.cpp:307-362 (evs[0]) */

/* ---- measure4d observables on the current u --------------------------- */
ASKJA_API int askja_PolyakovLoop(askja_ctx* ctx, double* out);                 /* measurements4d.cpp:410-466 */
ASKJA_API int askja_WilsonLoopDir(askja_ctx* ctx, int dir, double* out);       /* measurements4d.cpp:311-355 */
ASKJA_API int askja_PlaqExp(askja_ctx* ctx, double* temporal, double* spatial);/* measurements4d.cpp:885-927 */
ASKJA_API int askja_scalarLoopcorr(askja_ctx* ctx, double* out /* N0 values */); /* measurements4d.cpp:357-408 */

/* ---- short names for the seam (the same calls as above) --------------- */
ASKJA_API int askja_force_step(askja_ctx* ctx, double eps);          /* = askja_updateE (sun.cpp:672-723) */
ASKJA_API int askja_link_step(askja_ctx* ctx, double eps);           /* = askja_updateUandcopyDown (sun.cpp:774-790) */
ASKJA_API int askja_action(askja_ctx* ctx, double* s_over_beta);     /* = askja_EnergyMag (sun.cpp:507-537) */
ASKJA_API int askja_kinetic(askja_ctx* ctx, double* trp2);           /* = askja_simpleenergyEl(ctx, 0, .) (sun.cpp:540-548) */
ASKJA_API int askja_refresh_momenta(askja_ctx* ctx, uint64_t seed, uint64_t counter); /* = askja_initializeE */
/* The measurements of one configuration (DIM >= 2), DIM+4 values:
 * out[0], out[1] PlaqExp temporal / spatial; out[2] PolyakovLoop;
 * out[2+d] WilsonLoop(dir d), d = 1..DIM-1 (measurements4d.cpp:311-466, 885-927);
 * out[DIM+2] GaussLaw; out[DIM+3] UViol (sun.cpp:415-471). */
ASKJA_API int askja_measure(askja_ctx* ctx, double* out);

/* ---- diagnostics the reference defines but never calls ---------------- */
/* FourierTrafo (sun.cpp:365-411): coefficients[j] = |x_j|, x the inverse DFT
 * (1/N0 normalised, as gsl_fft_complex_inverse) of the plaquette energy
 * sum_{a<b} (1 - ReTr P_ab / NC) of sites 0 .. N0-1 (site numbers, as the
 * reference loops them).  N0 values; NC <= 64. */
ASKJA_API int askja_FourierTrafo(askja_ctx* ctx, double* coefficients);
/* Tab (sun.cpp:580-670): adds site i's energy-momentum tensor terms, built
 * from the clover field strength of u and from pi + Pi, to mdata[0..Npt-1]
 * (mdata accumulates, as in the reference).  2 <= Npt <= DIM+2, DIM <= 8,
 * NC <= 64. */
ASKJA_API int askja_Tab(askja_ctx* ctx, long i, double* mdata, int Npt);
/* Tab for every site: out[s*Npt + m] = site s's contribution to mdata[m]. */
ASKJA_API int askja_Tab_all(askja_ctx* ctx, int Npt, double* out /* V*Npt */);
/* getevs (measurements4d.cpp:185-309): eigenphases of the N0 Wilson lines
 * along direction 1 through (x0,0,..) and of the N1 Polyakov lines along
 * direction 0 through (0,x1,0,..); per line the NC phases arg(lambda) are
 * re-centred by the winding (sum/2pi) when it exceeds 0.1 in magnitude and
 * sorted; w[i] and p[i] are the i-th sorted phase averaged over the lines
 * (NC values each).  Eigenvalues on the GPU (Hessenberg + shifted QR in
 * FP64), the sort and average on the host.  DIM >= 2. */
ASKJA_API int askja_eigenphases(askja_ctx* ctx, double* w, double* p);

/* ---- whole trajectories, on the device -------------------------------- */
/* One HMC trajectory as in sun.cpp:1249-1318 with `nsteps` link updates:
 * momentum refresh, H_old, half kick, (drift, kick) x nsteps with the last
 * kick halved, H_new, Metropolis, then uconf = u (accept) or u = uconf
 * (reject).  No host synchronisation inside. */
ASKJA_API int askja_trajectory(askja_ctx* ctx, int nsteps, askja_traj_result* out);
/* askja_trajectory without waiting (not in the reference): enqueues the
 * trajectory (a CUDA-graph replay, as askja_run_trajectories) and the copy of
 * its outcome to *out (may be NULL), and returns.  *out is valid after the
 * next askja_sync; it should be page-locked, or the copy blocks the host
 * until the trajectory has run. */
ASKJA_API int askja_trajectory_async(askja_ctx* ctx, int nsteps, askja_traj_result* out);
/* `ntraj` trajectories; with use_graph != 0 each is a CUDA-graph replay.
 * `log` (may be NULL) receives 4 doubles per trajectory: h_old, h_new, dh, accepted. */
ASKJA_API int askja_run_trajectories(askja_ctx* ctx, int ntraj, int nsteps, int use_graph, askja_traj_result* last,
                           double* log);
/* Only the leapfrog part of askja_trajectory (refresh, H and Metropolis
 * excluded): K(eps/2) [D(eps) K(eps)]^(nsteps-1) D(eps) K(eps/2) with fused
 * kick+drift kernels. */
ASKJA_API int askja_leapfrog(askja_ctx* ctx, int nsteps, double eps);

/* `nsteps` repetitions of the reference's inner MD step
 * "updateUandcopyDown(eps); updateE(eps)" (sun.cpp:1216-1218), computed with
 * fused kick+drift kernels; afterwards pi and Pi hold exactly what the
 * reference's globals would. */
ASKJA_API int askja_md_steps(askja_ctx* ctx, int nsteps, double eps);

/* ---- autotuning (not in the reference) ---------------------------------- */
/* Kernel mapping for the force / link-update kernel of one (NC, DIM,
 * precision): thread-per-link (NC <= 4, all matrices in registers) or
 * row-per-thread (NC threads per link, shared-memory tiles) or tensor cores
 * (FP32, NC = 16, 32 or 64: every complex product a split-TF32 MMA) or site pairs
 * (FP32 SU(3): two adjacent sites' links per thread in packed FP32x2
 * arithmetic), the number of sites per CTA of the row kernels, and the
 * register budget of the thread-per-link kernels. */
typedef struct {
  int path;       /* 0 thread-per-link, 1 row-per-thread, 2 tensor cores, 3 site pairs */
  int groups;     /* row-per-thread: sites per CTA (0 = default) */
  int occupancy;  /* thread-per-link, and row-per-thread FP32 with 5 <= NC <= 8: 0 default registers, 1 and 2
                     tighter budgets / more resident CTAs */
  int ncand;      /* candidates timed */
  double best_us; /* fused kick+drift launch time of the choice, microseconds */
  int cand_path[24], cand_groups[24], cand_occ[24];
  double cand_us[24];
} askja_tuning;

/* Times every candidate on this context's lattice (reps launches each, on
 * scratch copies of the fields -- u and pi are left unchanged, Pi is
 * overwritten), switches the context to the fastest and remembers it for
 * later contexts with the same (NC, DIM, precision) in this process. */
ASKJA_API int askja_autotune(askja_ctx* ctx, int reps, askja_tuning* out);
/* Applies a previously found mapping (for example read back from a file). */
ASKJA_API int askja_set_tuning(askja_ctx* ctx, const askja_tuning* t);

/* ---- batched independent chains (not in the reference) ----------------- */
/* Many independent HMC chains of uneven shape -- a beta scan, several colour
 * numbers, dimensions and volumes -- advanced together: per MD step one force
 * launch per colour number covers every chain of that colour number (the
 * launches of different colour numbers run concurrently), the reductions,
 * momentum refresh, Metropolis test and accept/reject copy are one launch
 * each for all chains, and a whole trajectory of all chains is one CUDA graph.
 * Each chain follows sun.cpp:1249-1318 with its own BETA, DT, LEVEL and seed. */
typedef struct {
  int nc, dim, n[ASKJA_MAX_DIM];
  double beta, dt;
  int level;
  uint64_t seed;
} askja_chain_params;

typedef struct askja_batch askja_batch;

ASKJA_API int askja_batch_create(const askja_chain_params* chains, int nchains, int precision, int device,
                                 askja_batch** out);
ASKJA_API void askja_batch_destroy(askja_batch* b);
ASKJA_API const char* askja_batch_last_error(const askja_batch* b); /* b may be NULL: last create() error */
ASKJA_API void* askja_batch_stream(askja_batch* b);
ASKJA_API int askja_batch_hot_start(askja_batch* b, uint64_t seed); /* Haar SU(NC) links for every chain */
ASKJA_API int askja_batch_set_links(askja_batch* b, int chain, const double* conf); /* U-conf layout */
ASKJA_API int askja_batch_get_links(askja_batch* b, int chain, double* conf);
/* ntraj trajectories of nsteps MD steps for all chains; results[c] (may be
 * NULL) receives chain c's outcome of the last trajectory and its counters. */
ASKJA_API int askja_batch_run(askja_batch* b, int ntraj, int nsteps, int use_graph, askja_traj_result* results);
/* out[c] = mean plaquette 1 - EnergyMag / (V D (D-1)/2) of chain c */
ASKJA_API int askja_batch_plaquette(askja_batch* b, double* out);

/* ---- allocation-free plaquette sums ------------------------------------ */
/* No counterpart in the reference.  For callers that cannot let a library
 * allocate GPU memory -- their device memory is owned by their own pool
 * allocator, or they run on a fixed memory budget where a cudaMalloc would
 * fail or synchronise the device mid-step.  Computes the same temporal and
 * spatial plaquette sums as askja_PlaqExp (out[0] temporal, out[1] spatial,
 * FP64) for a link field the caller already holds in device memory in plain
 * structure-of-arrays order (element (r,c) of link (site s, dir d) at
 * ((d*NC + r)*NC + c)*V + s, double2 for ASKJA_FP64 or float2 for ASKJA_FP32
 * per p->precision); `out` is device memory for 2 doubles.  Only p->nc,
 * p->dim, p->n, p->precision and p->device are read.
 *  - Allocates nothing: the per-block partial sums go to a fixed 128 KiB
 *    static device array that every GPU loading the library keeps until exit.
 *    Volumes above 2,097,152 sites are rejected with ASKJA_ERR_ARG.
 *  - The first call on a device looks up that array's device address
 *    (cudaGetSymbolAddress) and keeps it for the life of the process; make
 *    that first call before any stream capture.  Resetting the device
 *    (cudaDeviceReset) while the library is loaded is not supported: the kept
 *    address would no longer be valid.
 *  - p->device is made current for the call and the caller's own current
 *    device is restored before returning.
 *  - Work is enqueued on `stream` (NULL: the default stream) and the call
 *    returns without waiting; `out` is valid once the stream reaches it.
 *  - All calls share the one array (it keeps the last call's partials, each
 *    call overwrites every slot it reads, nothing needs clearing), so calls
 *    that overlap on the GPU race: serialise them on one stream.
 *  - Errors are reported through askja_last_error(NULL). */
ASKJA_API int askja_plaqexp_static(const askja_params* p, const void* links, double* out, void* stream);

/* ---- domain decomposition (not in the reference) ------------------------ */
/* Restricts the plaquette and link sums (askja_EnergyMag, askja_PlaqExp,
 * askja_simpleenergyEl, askja_EnergyEl, askja_UViol, and the Hamiltonian of
 * askja_trajectory) to the sites [s0, s1) of this context's lattice (site
 * order of the U-conf layout, x0 slowest), 0 <= s0 < s1 <= V.  A rank that
 * holds one x0 slab of a larger lattice plus halo slabs (askja_b200/slabs.py)
 * counts only the slab it owns; the sums of all ranks then add up to the
 * whole lattice's.  Default: every site. */
ASKJA_API int askja_set_reduction_range(askja_ctx* ctx, long s0, long s1);
/* Current links of the sites [s0, s0 + nsites) copied to (to_buf = 1) or from
 * (to_buf = 0) buf in the U-conf order ([site][dir][row][col][re,im] doubles,
 * nsites * DIM * NC * NC * 2 of them); buf may be host or device memory.
 * Returns when the copy is complete.  With x0 slowest, one x0 slab is the
 * nsites = V / N0 sites from s0 = x0 * V / N0: the halo exchange of a
 * domain-decomposed chain. */
ASKJA_API int askja_slab(askja_ctx* ctx, long s0, long nsites, double* buf, int to_buf);

/* ---- diagnostics (not in the reference) -------------------------------- */
/* Exercises the tensor-core path's bounded wait (context on the tensor-core
 * mapping, kernel path 2, only): one CTA sets up as the tensor-core link update
 * does and waits `cycles` clock cycles on an mbarrier that nothing completes
 * (no tensor-core instruction is issued), records the timeout as the link
 * update would and releases its tensor memory.  Returns once enqueued; the
 * next synchronising call (askja_sync) then reports ASKJA_ERR_CUDA with the
 * message of a link update that gave up waiting, and the context stays usable. */
ASKJA_API int askja_tc_wait_selftest(askja_ctx* ctx, long long cycles);

/* ---- host I/O (no GPU needed) ----------------------------------------- */
/* Contents of the positional params file (sun.cpp:803-938).  Key names are
 * read but not checked; the order is: header, NC, DIM, N0..N{DIM-1}, BETA, DT,
 * STEPS, UPDATE, UPDATE2, CONFTAKE, LEVEL, VERBOSE, RUNCONTINUE, RANDOM, and,
 * when RUNCONTINUE, TIME-STEP TAKEN NACC NAC1 NREC NTOT. */
typedef struct {
  int nc, dim, n[ASKJA_MAX_DIM];
  double beta, dt;
  int steps, update, update2, conftake, level, verbose, runcontinue, random;
  int start, taken, nacc, nac1, nrec, ntot; /* resume trailer (START = TIME-STEP) */
} askja_run_params;

ASKJA_API int askja_params_load(const char* path, askja_run_params* out);
/* store_parameters (sun.cpp:940-1057): copy `infile`'s key names with the
 * run's values, RUNCONTINUE forced to 1, plus the TIME-STEP/TAKEN/NACC/NAC1/
 * NREC/NTOT trailer. */
ASKJA_API int askja_params_store(const char* infile, const char* outfile, const askja_run_params* p, int timestep, int taken);
/* File stem "<dir>/<kind>-N%i-Nt%i-Ns%i-BETA%.2f-DT%.4f-U%.4f-CT%i" (sun.cpp:1124). */
ASKJA_API int askja_file_stem(const askja_run_params* p, const char* dir, const char* kind, char* out, size_t cap);
ASKJA_API int askja_conf_write(const char* path, const double* conf, long n_doubles); /* storeconf byte format */
ASKJA_API int askja_conf_read(const char* path, double* conf, long n_doubles);        /* loadconf; short file = error */

/* Pinned host memory for fast uploads (cudaMallocHost); NULL on failure. */
ASKJA_API void* askja_host_alloc(size_t bytes);
ASKJA_API void askja_host_free(void* p);

#ifdef __cplusplus
}
#endif

#endif
