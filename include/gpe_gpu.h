/*
 * gpe_gpu.h -- C-ABI of the B200 (sm_100a) Gross-Pitaevskii time stepper.
 *
 * This is the drop-in boundary for the reference solver's hot path
 * (liangjj/gpe, Fortran 90 + MPI).  The reference reaches that path through
 * the module procedure solver(var_in, var_out) (src/solve.f90:25-53, called
 * from src/gpe.f90:228) plus get_norm / energy / renormalise
 * (src/variables.f90:537-587, 698-709).  Those procedures read and write
 * module globals (dt, t, im_t, p, scheme, eqn_to_solve, bcs, order, dx..,
 * g, mu, omx.., Urhs, diss_amp: src/parameters.f90:24-127); here the
 * globals are the explicit gpe_params / gpe_time structs.
 *
 * Plain C types only: no C++ types, exceptions or torch objects cross this
 * boundary.  A context owns all device memory; psi stays resident on the GPU
 * between calls and crosses PCIe only in set_state / get_state (or the
 * host-array form gpe_gpu_solver_host).  Every call is stream-ordered on the
 * context's own CUDA stream and has completed when it returns.  One context
 * per host thread.
 *
 * Host arrays are the reference's interior layout: complex, Fortran order,
 * x fastest, psi[(k*ny + j)*nx + i]; elem_bytes 8 = complex64 (single
 * precision `pr`), 16 = complex128 (double precision `pr`,
 * src/parameters.in:21-23).
 *
 * Status codes: 0 = success, otherwise one of GPE_ERR_*; the message is
 * available from gpe_gpu_last_error().  The reference has no status codes --
 * it calls emergency_stop (src/error.f90:24-46); a driver maps a non-zero
 * status to that behaviour.
 */
#ifndef GPE_GPU_H
#define GPE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPE_GPU_ABI_VERSION 1

/* status codes */
#define GPE_OK 0
#define GPE_ERR_INVALID 1    /* bad argument or configuration */
#define GPE_ERR_SCHEME 2     /* 'ERROR: Unrecognised time stepping scheme.'
                                (src/solve.f90:47-49) */
#define GPE_ERR_CUDA 3       /* CUDA runtime/driver error */
#define GPE_ERR_OOM 4        /* device allocation failed */
#define GPE_ERR_NAN 5        /* non-finite value in a reduction */
#define GPE_ERR_TIMEOUT 6    /* a bounded device-side wait expired */
#define GPE_ERR_NODEVICE 7   /* no usable sm_100 device */
#define GPE_ERR_UNDERFLOW 8  /* rk45 step underflow (a warning in
                                src/solve.f90:203-211; reported, not fatal) */

/* scheme values (the reference's character(5) scheme) */
#define GPE_SCHEME_EULER 0   /* 'euler', src/solve.f90:57-74 */
#define GPE_SCHEME_RK2 1     /* 'rk2',   src/solve.f90:78-105 */
#define GPE_SCHEME_RK4 2     /* 'rk4',   src/solve.f90:109-154 */
#define GPE_SCHEME_RK45 3    /* 'rk45',  src/solve.f90:158-378 */

/* Run configuration.  Mirrors run_params / eqn_params
 * (src/parameters.f90:24-55) and the compile-time grid of parameters.in
 * (nx, ny, nz, pr); the remaining fields select the B200 storage form. */
typedef struct gpe_params {
  int32_t struct_size;  /* sizeof(gpe_params), for ABI checks */
  int32_t nx, ny, nz;   /* grid points (parameters.in nx, ny, nz) */
  double xr, yr, zr;    /* box half-widths; dx = 2 xr/(nx-1) (ic.f90:43-48) */
  int32_t scheme;       /* GPE_SCHEME_* */
  int32_t eqn_to_solve; /* 1..4 (src/solve.f90:414-437) */
  int32_t bcs;          /* 1 periodic, 2 reflective */
  int32_t order;        /* 2 or 4 (centred differences) */
  int32_t real_time;    /* 1 real time, 0 imaginary time */
  int32_t precision;    /* storage: 8 = complex64, 16 = complex128 */
  double Urhs, diss_amp, scal, g, mu, nn, omx, omy, omz;
  int32_t kahan;        /* complex64 only: compensated (Kahan) accumulation
                           of the step increment, FP32 compensation field */
  int32_t device;       /* CUDA device ordinal */
  int32_t tile_y;       /* 0 = auto; else rows per tile (4 or 8) */
  int32_t zchunk;       /* 0 = auto; else z-planes per block */
  double fd_match;      /* order 4 only, 0 = the centred 4th-order Laplacian.
                           r in (0, 1.5): per-axis coefficients
                           c1 = (4 - r^2)/(3 h^2), c2 = (r^2 - 1)/(12 h^2),
                           whose symbol k^2 - k^4 (r h)^2 / 12 + O(k^6 h^4)
                           is that of the 2nd-order Laplacian on a grid of
                           spacing r h: a coarse grid that disperses like a
                           finer one (the learned correction's base).  No
                           reference counterpart. */
} gpe_params;

/* The solver's time globals: t, im_t, dt (complex), p
 * (src/parameters.f90:115-127). */
typedef struct gpe_time {
  double t, im_t;
  double dt_re, dt_im;
  int32_t p;
  int32_t reserved;
} gpe_time;

/* Per-call diagnostics of solver(); for rk45: the accepted errmax
 * (errmaxr(1), src/solve.f90:184-193), number of rkck attempts, the step
 * actually taken (dt_did, :223) and an underflow flag (tnew == t, :203-211). */
typedef struct gpe_step_info {
  double errmax;
  double dt_did_re, dt_did_im;
  int32_t attempts;
  int32_t underflow;
} gpe_step_info;

/* Per-kernel-family device times collected while timing is on. */
#define GPE_TIMING_FAMILIES 8
typedef struct gpe_timing {
  double ms[GPE_TIMING_FAMILIES];      /* summed CUDA-event time */
  int64_t launches[GPE_TIMING_FAMILIES];
  int64_t sites[GPE_TIMING_FAMILIES];  /* grid sites processed */
} gpe_timing;
/* families */
#define GPE_FAM_STAGE_FIRST 0  /* first stage of a step (reads psi only) */
#define GPE_FAM_STAGE_MID 1    /* middle stages */
#define GPE_FAM_STAGE_LAST 2   /* final stage (writes psi, fused norm) */
#define GPE_FAM_REDUCE 3       /* reduction finalisers */
#define GPE_FAM_ENERGY 4
#define GPE_FAM_COPY 5         /* state pack/unpack, ghost fill, scale */
#define GPE_FAM_OTHER 6        /* cuFFT transforms and the rest */
#define GPE_FAM_SPECTRUM 7     /* spectrum / condensate reduction pass */

typedef struct gpe_ctx gpe_ctx;

/* Fill *prm with the reference defaults for an nx x ny x nz grid. */
void gpe_gpu_default_params(gpe_params* prm, int32_t nx, int32_t ny,
                            int32_t nz);

/* Allocate a context on prm->device: all fields, tensor maps and scratch.
 * Replaces the reference's allocation of psi%old/psi%new and work arrays
 * (src/gpe.f90:56-68) and its grid set-up get_grid (src/ic.f90:32-69). */
int gpe_gpu_create(const gpe_params* prm, gpe_ctx** out);
void gpe_gpu_destroy(gpe_ctx* ctx);

/* Last error message of ctx (or of the last failed create when ctx is
 * NULL).  Valid until the next call on ctx. */
const char* gpe_gpu_last_error(const gpe_ctx* ctx);

/* Grid coordinates x(0:nx-1), y, z (src/ic.f90:24-26, 53-66). */
int gpe_gpu_grid(const gpe_ctx* ctx, double* x, double* y, double* z);

/* Load / read the resident state from / to a HOST array (interior layout).
 * set_state also fills the boundary ghosts, which is what the caller's
 * halo exchange did before solver() (src/gpe.f90:165-174). */
int gpe_gpu_set_state(gpe_ctx* ctx, const void* psi, int32_t elem_bytes);
int gpe_gpu_get_state(gpe_ctx* ctx, void* psi, int32_t elem_bytes);
/* Same with DEVICE arrays on the context's device.  The copy is ordered on
 * the context's own (non-blocking) stream only: the caller must have
 * finished writing psi (set) or reading its previous contents (get) on its
 * own streams before the call, e.g. with cudaStreamSynchronize.  The call
 * returns after the copy is complete. */
int gpe_gpu_set_state_device(gpe_ctx* ctx, const void* psi,
                             int32_t elem_bytes);
int gpe_gpu_get_state_device(gpe_ctx* ctx, void* psi, int32_t elem_bytes);

/* psi at the interior site (i, j, k) of this context (k counts the
 * context's own planes) into re_im[2] (HOST): the point value save_time
 * writes to psi_time.dat (src/io.f90:147-195), without copying the field. */
int gpe_gpu_get_site(gpe_ctx* ctx, int32_t i, int32_t j, int32_t k, double* re_im);

/* The z-plane k of this context (k counts its own planes) into a HOST array
 * out[ny][nx] (x fastest) of elem_bytes complexes: the slice save_surface
 * writes (src/io.f90:449-485, psi*.dat at nz/2), without copying the field. */
int gpe_gpu_get_plane(gpe_ctx* ctx, int32_t k, void* out, int32_t elem_bytes);

/* One call of solver(var_in, var_out) (src/solve.f90:25-53) on the
 * resident state: advances psi by one step of the configured scheme and
 * updates tm->t, tm->im_t and (rk45) tm->dt exactly as the reference updates
 * its globals (src/solve.f90:70-71, 101-102, 150-151, 222-229).  tm->p is
 * not changed (the caller's loop increments it, src/gpe.f90:277).  info may
 * be NULL.  The fused final-stage norm of the new state is cached for
 * gpe_gpu_norm. */
int gpe_gpu_solver(gpe_ctx* ctx, gpe_time* tm, gpe_step_info* info);

/* The literal host-array form of solver(var_in, var_out): copies var_in
 * (interior, HOST) to the device, steps, copies the result to var_out.
 * The halo of the reference's var_in is not needed: boundary ghosts are
 * rebuilt on the device. */
int gpe_gpu_solver_host(gpe_ctx* ctx, const void* var_in, void* var_out,
                        int32_t elem_bytes, gpe_time* tm,
                        gpe_step_info* info);

/* nsteps solver() calls with get_norm after every step as the reference
 * loop does (src/gpe.f90:241-243); norms (HOST, may be NULL) receives nsteps
 * values; tm->p is advanced by the steps taken.  euler/rk2/rk4 steps are
 * enqueued back to back with no host synchronisation until the end.  rk45
 * takes nsteps accepted steps with the rkqs step control on the device
 * (src/solve.f90:158-244): each step is one CUDA graph, a conditional WHILE
 * node around the six Cash-Karp stages, the error and norm reductions and a
 * one-thread control kernel that accepts and grows dt or shrinks it and
 * retries, so no attempt waits for the host (contexts joined to NCCL, or
 * with timing on, run the same kernels with one read-back per attempt).  A
 * non-finite error estimate or 10000 rejected attempts stop the run early
 * (GPE_ERR_NAN / GPE_ERR_UNDERFLOW, tm then holds the last accepted step).
 * With a post-step correction attached, rk45 steps go one at a time. */
int gpe_gpu_advance(gpe_ctx* ctx, int64_t nsteps, gpe_time* tm,
                    double* norms);

/* The accepted dt (real part) and attempt count of the first n steps of the
 * last rk45 gpe_gpu_advance (HOST arrays, either may be NULL); n beyond the
 * steps it took is GPE_ERR_INVALID.  No reference counterpart: the
 * reference writes dt to timestep.dat every save_rate steps (rkqs). */
int gpe_gpu_step_series(gpe_ctx* ctx, int64_t n, double* dt_did, int32_t* attempts);

/* get_norm (src/variables.f90:537-559 with integrate_x/y/z :713-823) of the
 * resident state, FP64. */
int gpe_gpu_norm(gpe_ctx* ctx, double* norm);

/* energy (src/variables.f90:563-587): *E = sum Re(-lap psi conj(psi)
 * + 0.5|psi|^4) dx dy dz (energy.dat holds E/(nx ny nz), src/io.f90:213).
 * *H4 (may be NULL) = the discrete Hamiltonian of equation 4,
 * sum [0.5 Re(-lap psi conj psi) + V|psi|^2 + 0.5 g|psi|^4 - mu|psi|^2]
 * dx dy dz, which that equation conserves (no reference counterpart). */
int gpe_gpu_energy(gpe_ctx* ctx, double* E, double* H4);
/* mass (src/variables.f90:590-610: plain sum of |psi|^2 dx dy dz) and
 * momentum (:615-694: per axis the extended-Simpson integral of
 * (Re psi - 1) Im(d conj psi) - Im psi Re(d psi)) of the resident state, in
 * one device pass with FP64 sums; mom has 3 entries. */
int gpe_gpu_diagnostics(gpe_ctx* ctx, double* mass, double* mom);

/* Spectral initial condition and diagnostics on cuFFT (single-domain
 * contexts; a z-slab context returns GPE_ERR_INVALID).  Transforms follow
 * the reference's fft (src/ic.f90:905-1000): 'forward' = exp(-i k.x),
 * 'backward' = exp(+i k.x), both scaled by 1/sqrt(nx ny nz); the integer
 * wavenumber of index i along an axis of n points is i for
 * i <= (n-1)/2 + 1 and n - i above (src/ic.f90:221-238).  libcufft.so.11 is
 * opened on first use; without it the calls return GPE_ERR_CUDA.  The first
 * call on a context creates its two cuFFT plans (with cuFFT's work areas),
 * kept until the context is destroyed.
 *
 * gpe_gpu_random_phase replaces ics' random_phase (src/ic.f90:190-252) with
 * get_kc_amp (:256-269): every mode with |k|^2 <= kc2 gets amplitude
 * comp_amp and phase 2 pi phi, all others zero, and psi is the forward
 * transform, ghosts filled.  phi for the mode at dense index
 * q = (k ny + j) nx + i is the top 53 bits of SplitMix64(seed + (q+1) G),
 * G = 0x9E3779B97F4A7C15, times 2^-53 (the reference draws Fortran
 * random_number from a clock seed; this is reproducible).  *amp_out and
 * *kc2_out (may be NULL) receive comp_amp and kc2. */
int gpe_gpu_random_phase(gpe_ctx* ctx, double nv, double enerv, uint64_t seed,
                         double* amp_out, double* kc2_out);

/* condensed_particles (src/io.f90:315-404) and spectrum (:632-725) of the
 * resident state in one pass over its backward transform a:
 *   row[0..6] = M/(8 xr yr zr), n0/V, M, n0, temp, temp2, H/V (columns 3-9
 *     of mass.dat; M = sum |psi|^2 dx dy dz, here by Parseval over a);
 *   eta[7], nharm[7] = mean occupation and mode count of the 7 logarithmic
 *     shells (spectrum*.dat);
 *   F[nf] = the integral distribution function F(kk), kk = 1..nf, nf = nx/2
 *     (idf*.dat; nf must equal nx/2; nx up to 5120, the bins living in
 *     shared memory).
 * Any output pointer may be NULL (HOST arrays). */
int gpe_gpu_condensed_particles(gpe_ctx* ctx, double* row, double* eta,
                                int64_t* nharm, double* F, int32_t nf);

/* filtered_surface (src/io.f90:533-628): a = backward transform of psi,
 * a(k) *= max(1 - m |k|^2 / filter_kc^2, 0), out = forward transform
 * (interior layout, x fastest; HOST when device_out = 0, else DEVICE). */
int gpe_gpu_filtered_field(gpe_ctx* ctx, double filter_kc, double m, void* out,
                           int32_t elem_bytes, int32_t device_out);

/* linelength (src/variables.f90:879-1145): total vortex line length of the
 * resident state (single-domain contexts), from the zero lines of Re psi and
 * Im psi on the faces of every interior cell, times dx (the reference
 * assumes dx = dy = dz).  The reference carries its point arrays from cell
 * to cell and leaves their start undefined; here they start at zero on
 * every call. */
int gpe_gpu_linelength(gpe_ctx* ctx, double* length);
/* The same for a DEVICE array in the interior layout on the context's grid
 * (complex64 when elem_bytes = 8, complex128 when 16), e.g. the field of
 * gpe_gpu_filtered_field: save_linelength(filtered, 1) of
 * filtered_surface (src/io.f90:583-585), filtered_ll.dat.  The array must
 * be complete (written on the caller's streams and synchronised). */
int gpe_gpu_linelength_field(gpe_ctx* ctx, const void* field, int32_t elem_bytes,
                             double* length);

/* get_zeros, get_extra_zeros and get_re_im_zeros (src/io.f90:895-1402):
 * the zero points of the resident state (single-domain contexts) that the
 * reference writes to zeros*.dat, re_zeros*.dat and im_zeros*.dat, in its
 * order, as 12 sections: 0-2 edges along x, y, z where Re and Im cross
 * together; 3-5 xy, xz, yz faces crossed alternately by Re and Im; 6-8 the
 * x, y, z edges where Re crosses; 9-11 the same for Im.  counts[12] (HOST)
 * receives each section's number of points.  With points non-NULL (HOST,
 * room for cap points of 3 doubles) the points follow, sections
 * concatenated; a cap below the total returns GPE_ERR_INVALID with counts
 * filled.  Call with points = NULL to size the buffer.  The device copy of
 * the points (24 bytes each) is kept by the context for the next call and
 * freed with it. */
#define GPE_ZERO_SECTIONS 12
int gpe_gpu_zeros(gpe_ctx* ctx, int64_t* counts, double* points, int64_t cap);

/* Failure-detection self-test (no reference counterpart): runs, on the
 * context's stream, a device wait on a flag that nothing sets, bounded by
 * limit_ns (at most 1 s) with the same bounded-wait code as the stage
 * kernels; returns GPE_ERR_TIMEOUT read back from the device status word,
 * after which the context is still usable. */
int gpe_gpu_wait_probe(gpe_ctx* ctx, uint64_t limit_ns);

/* Limit of every bounded wait inside this context's stage kernels (the TMA
 * ring hand-over between the producer warp and the compute warps); 0 restores
 * the default of 2 s.  A wait that runs out makes the kernel stop, record
 * GPE_ERR_TIMEOUT in the status word and return; the step that hit it
 * returns GPE_ERR_TIMEOUT and its output is undefined, but the context stays
 * usable (set the state again).  Copies already in flight are always waited
 * for with a limit of at least 2 s before a block exits.  No reference
 * counterpart: failure detection of the device pipeline. */
int gpe_gpu_set_wait_limit(gpe_ctx* ctx, uint64_t limit_ns);

/* Failure-detection test hook: with plane >= 0, the producer warp of every
 * block of this context's later stage launches stops issuing loads when it
 * reaches that plane (counted from the start of a work item, whose first
 * planes are its z-chunk's halo; every item has at least 2), so the compute
 * warps' bounded wait for it runs out (GPE_ERR_TIMEOUT, as above) without any
 * fault; -1 turns it off.  Results of the launches it affects are undefined.
 * No reference counterpart. */
int gpe_gpu_test_stall(gpe_ctx* ctx, int32_t plane);

/* renormalise (src/variables.f90:698-709): psi = sqrt(nn) psi / sqrt(norm). */
int gpe_gpu_renormalise(gpe_ctx* ctx, double norm);

/* get_rhs (src/solve.f90:382-440) and laplacian (src/variables.f90:55-71)
 * of the resident state into a HOST array (interior layout). */
int gpe_gpu_rhs(gpe_ctx* ctx, void* out, int32_t elem_bytes);
int gpe_gpu_laplacian(gpe_ctx* ctx, void* out, int32_t elem_bytes);

/* Switch the time direction in place, as the imaginary-to-real switch of
 * src/gpe.f90:251-268 does (real_time flag used by rk45 step control). */
int gpe_gpu_set_real_time(gpe_ctx* ctx, int32_t real_time);

/* z-slab decomposition (one process per GPU).  The reference distributes
 * its grid over a (y, z) MPI process grid with a two-plane halo
 * (src/variables.f90:98-358) and all-reduces its sums and the rk45 error
 * maximum (src/variables.f90:581, 772, 816; src/solve.f90:189).  Here x and
 * y stay whole and ranks own consecutive z-slabs.
 *
 * gpe_gpu_set_slab: this context (created with nz = the slab's planes) holds
 * planes z_offset .. z_offset+nz-1 of a global axis of nz_global planes
 * (prm->zr is the global half-width).  Call before gpe_gpu_set_state. */
int gpe_gpu_set_slab(gpe_ctx* ctx, int32_t nz_global, int32_t z_offset);
/* A 128-byte NCCL unique id, made on one rank; the caller broadcasts it. */
int gpe_gpu_comm_unique_id(void* id128);
/* Join the ranks' NCCL communicator (rank r owns the r-th slab from the
 * bottom).  From then on every kernel that writes a stencil field is
 * followed by a send of its two boundary planes into the z-neighbours' ghost
 * planes, and every norm / energy / rk45 error reduction by an all-reduce,
 * so all ranks take the same rk45 decision.  On a slab of 8 planes or more
 * the stage computes its boundary planes first and the send runs on a side
 * stream while the interior planes are computed; the context's stream waits
 * for it before the next stage. */
int gpe_gpu_comm_init(gpe_ctx* ctx, const void* id128, int32_t rank,
                      int32_t nranks);

/* Batched ensembles (no reference counterpart; the reference runs one grid
 * per job).  Independent runs of uneven grids, each a full member context,
 * are stepped together with rk4: every stage is ONE persistent launch over a
 * work list of (run, tile, z-range) items of all members, and a whole step
 * (4 stage launches + per-run norm) is captured once in a CUDA graph and
 * replayed.  Members share scheme (rk4), order, bcs, equation, precision,
 * kahan, device and time direction; grids, box sizes, g, mu and trap may
 * differ. */
/* In-process slab group: z-slab contexts of one grid on one device (each
 * created with its slab's nz and placed with gpe_gpu_set_slab, consecutive
 * from z = 0, covering the global axis), stepped together as the reference
 * steps its MPI ranks (src/variables.f90:98-358, src/solve.f90:189): every
 * stage runs on every member, then each member's two boundary planes go to
 * its neighbours' ghost planes (cudaMemcpyAsync, the same planes the NCCL
 * path sends; on a side stream beside the interior planes when every slab
 * has 8 planes or more), and the norm, energy and rk45 error are
 * combined across members (sum / max) so every member takes the same rk45
 * decision.  Members keep their own fields and tables; while grouped they run
 * on the group's stream and the per-context step / reduce entry points
 * refuse them (GPE_ERR_INVALID).  State is loaded and read per member
 * (gpe_gpu_set_state / get_state); the group refreshes the z ghosts before
 * its next step.  Destroying the group returns the members to their own
 * streams; destroying a member first empties the group. */
typedef struct gpe_group gpe_group;
int gpe_group_create(gpe_ctx* const* members, int32_t n, gpe_group** out);
/* One solver() step of every member (t, im_t, dt, info as gpe_gpu_solver). */
int gpe_group_solver(gpe_group* g, gpe_time* tm, gpe_step_info* info);
/* get_norm / energy of the whole grid. */
int gpe_group_norm(gpe_group* g, double* norm);
int gpe_group_energy(gpe_group* g, double* E, double* H4);
void gpe_group_destroy(gpe_group* g);
const char* gpe_group_last_error(const gpe_group* g);

typedef struct gpe_batch gpe_batch;
typedef struct gpe_batch_opts {
  int32_t struct_size;  /* sizeof(gpe_batch_opts) */
  int32_t tile_y;       /* 0 = auto (8); else 4 or 8 */
  int32_t zchunk;       /* 0 = auto (min(nz, 64)); z-planes per work item */
  int32_t ctas_per_sm;  /* 0 = as many as fit */
  int32_t use_graph;    /* 1 = replay a captured CUDA graph per step */
} gpe_batch_opts;
void gpe_batch_default_opts(gpe_batch_opts* opts);
int gpe_batch_create(const gpe_params* prms, int32_t nruns,
                     const gpe_batch_opts* opts, gpe_batch** out);
void gpe_batch_destroy(gpe_batch* batch);
const char* gpe_batch_last_error(const gpe_batch* batch);
/* Member context of run `run` (for set_state / get_state / norm / energy;
 * owned by the batch). */
int gpe_batch_member(gpe_batch* batch, int32_t run, gpe_ctx** ctx);
/* nsteps rk4 steps of every member with time step dt; norms (HOST, may be
 * NULL) receives nruns x nsteps values, run-major. */
int gpe_batch_advance(gpe_batch* batch, int64_t nsteps, double dt_re,
                      double dt_im, double* norms);
/* Re-plan the launches with new options (the autotuner's knob); the members'
 * states are kept. */
int gpe_batch_set_opts(gpe_batch* batch, const gpe_batch_opts* opts);
void* gpe_batch_stream(const gpe_batch* batch);
int64_t gpe_batch_launch_count(const gpe_batch* batch);
int gpe_batch_info(const gpe_batch* batch, int64_t* sites, int32_t* nitems,
                   int32_t* grid, int32_t* tile_y);

/* Per-kernel-family CUDA-event timing (off by default). */
int gpe_gpu_set_timing(gpe_ctx* ctx, int32_t on);
int gpe_gpu_get_timing(gpe_ctx* ctx, gpe_timing* out);
/* Number of kernels this context has launched (graph replays count their
 * kernels). */
int64_t gpe_gpu_launch_count(const gpe_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or CUDA events against the solver's. */
void* gpe_gpu_stream(const gpe_ctx* ctx);

/* Device bytes held by the context. */
int64_t gpe_gpu_device_bytes(const gpe_ctx* ctx);

/* Pinned host memory for the host-array calls (cudaHostAlloc/FreeHost). */
void* gpe_gpu_host_alloc(size_t bytes);
void gpe_gpu_host_free(void* p);

int32_t gpe_gpu_abi_version(void);

/* No counterpart in the reference: an allocation-free get_norm.
 *
 * For callers that cannot call cudaMalloc -- hosts whose device memory is
 * owned by another allocator (a framework's caching allocator, or a driver
 * that sizes all device memory up front and treats a later allocation as an
 * error).  Computes the extended-Simpson norm of get_norm
 * (src/variables.f90:537-559) of psi, a DEVICE array on the current device
 * in the interior layout (complex64 when elem_bytes = 8, complex128 when 16),
 * for the grid nx x ny x nz with half-widths xr, yr, zr, and writes it to
 * *norm_out, a DEVICE double.  No context is needed and nothing is
 * allocated: the only scratch is a fixed per-process array of
 * GPE_NOALLOC_MAX_PLANES doubles (one partial sum per z-plane) that every GPU
 * loading this library holds until exit; nz above that limit is rejected
 * with GPE_ERR_INVALID.  The work is queued on `stream` (a cudaStream_t, NULL
 * for the default stream) and is complete once that stream is synchronised.
 * The first call on a device looks up the scratch array's device address;
 * make that first call before any stream capture.  Every call uses the same
 * scratch array, so calls that overlap on the GPU (two streams, two host
 * threads) race and must be serialised by the caller.  Each call writes every
 * scratch entry it reads, so nothing needs clearing between calls.  Errors:
 * the status code, with the message from gpe_gpu_last_error(NULL). */
#define GPE_NOALLOC_MAX_PLANES 8192
int gpe_gpu_norm_noalloc(const void* psi, int32_t elem_bytes, int32_t nx,
                         int32_t ny, int32_t nz, double xr, double yr,
                         double zr, double* norm_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GPE_GPU_H */
