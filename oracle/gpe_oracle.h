/*
 * gpe_oracle.h -- CPU FP64 restatement of the reference GPE solver's
 * finite-difference time-stepping path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product path and the timed CPU baseline.  Nothing in the product
 * (gpe_b200/, include/) links, imports or calls it.
 *
 * PARITY UNPINNED: the reference (Fortran 90 + MPI + FFTW2) ships no golden
 * vectors or known-answer tests, and it cannot be compiled here (no Fortran
 * compiler, MPI or FFTW2 in the image).  This restatement is therefore pinned
 * only against analytic known-answer tests written by this project
 * (plane-wave RK recurrences, reflective cosine eigenmodes, Taylor orders,
 * integration-weight identities) and against an independent numpy
 * restatement.
 *
 * Layout: every field is complex FP64 stored as interleaved (re, im) doubles,
 * Fortran order (x fastest), interior only: psi[((k*ny)+j)*nx+i].
 * Internally the solver uses the reference's haloed shape
 * (0:nx-1, -2:ny+1, -2:nz+1) and a single-rank halo exchange.
 */
#ifndef GPE_ORACLE_H
#define GPE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Time-stepping schemes, as the reference's character(5) `scheme`
 * (src/solve.f90:34-50). */
enum { ORA_EULER = 0, ORA_RK2 = 1, ORA_RK4 = 2, ORA_RK45 = 3 };

/* Run parameters: the subset of run_params / eqn_params
 * (src/parameters.f90:24-55) plus the compile-time grid (parameters.in). */
typedef struct ora_params {
  int nx, ny, nz;
  double xr, yr, zr;
  int scheme;        /* ORA_* */
  int eqn_to_solve;  /* 1..4 */
  int bcs;           /* 1 periodic, 2 reflective */
  int order;         /* 2 or 4 */
  int real_time;     /* 1 real time, 0 imaginary time */
  double Urhs, diss_amp, scal, g, mu, nn, omx, omy, omz;
} ora_params;

/* Module globals the solver reads and updates (src/parameters.f90:115-127). */
typedef struct ora_time {
  double t, im_t;
  double dt_re, dt_im;
  int p;
} ora_time;

typedef struct ora_ctx ora_ctx;

ora_ctx* ora_create(const ora_params* prm);
void ora_destroy(ora_ctx* c);
void ora_set_threads(int n);
int ora_get_threads(void);

/* Grid of src/ic.f90:32-69 (x has nx entries, etc.). */
void ora_grid(const ora_ctx* c, double* x, double* y, double* z);

/* One call of solver(var_in, var_out) (src/solve.f90:25-53).  psi_in is the
 * interior field; the single-rank halo exchange of src/gpe.f90:171-174 is
 * done internally.  Updates tm like the reference updates t, im_t, dt.
 * For rk45, *errmax receives the accepted errmax and *attempts the number of
 * rkck attempts (may be NULL).  Returns 0, or -1 on an unknown scheme. */
int ora_solver(ora_ctx* c, const double* psi_in, double* psi_out,
               ora_time* tm, double* errmax, int* attempts);

/* get_rhs (src/solve.f90:382-440) on an interior field. */
void ora_rhs(ora_ctx* c, const double* psi, double* rhs);
/* laplacian (src/variables.f90:55-71) and deriv_x/y/z
 * (src/derivs.f90:25-142) on an interior field. */
void ora_laplacian(ora_ctx* c, const double* psi, double* lap);
void ora_deriv(ora_ctx* c, int axis, int second, const double* psi,
               double* out);

/* get_norm (src/variables.f90:537-559, integrate_x/y/z :713-823). */
double ora_get_norm(ora_ctx* c, const double* psi);
/* energy (src/variables.f90:563-587): returns E (already times dx dy dz;
 * energy.dat holds E/(nx ny nz), src/io.f90:213). */
double ora_energy(ora_ctx* c, const double* psi);
/* Discrete Hamiltonian of equation 4 (not in the reference; used for energy
 * drift): sum[ 0.5 Re(-lap psi . conj psi) + V|psi|^2 + 0.5 g|psi|^4
 * - mu|psi|^2 ] dx dy dz. */
double ora_hamiltonian4(ora_ctx* c, const double* psi);
/* mass (src/variables.f90:590-610) and momentum (:615-694). */
double ora_mass(ora_ctx* c, const double* psi);
void ora_momentum(ora_ctx* c, const double* psi, double mom[3]);
/* renormalise (src/variables.f90:698-709): psi = sqrt(nn)*psi/sqrt(norm). */
void ora_renormalise(ora_ctx* c, double* psi, double norm);

/* Initial-condition generators of src/ic.f90 (interior fields). */
void ora_ic_vortex_line(ora_ctx* c, double x0, double y0, double z0,
                        double amp1, double amp2, double ll, double sgn,
                        char dir, int imprint_phase, double* out);
void ora_ic_vortex_ring(ora_ctx* c, const char* plane, double x0, double y0,
                        double z0, double r0, double amp, int mm, double r1,
                        int kk, double dir, double* out);
void ora_ic_pade_pulse_ring(ora_ctx* c, const char* pulse_or_ring, double x0,
                            double y0, double z0, double r0, double* out);
void ora_ic_fermi(ora_ctx* c, double* out);
/* get_rr (src/ic.f90:888-901) on a scalar. */
double ora_get_rr(double r);

/* linelength (src/variables.f90:879-1145) of a single-domain interior psi
 * (nz, ny, nx complex, x fastest) with grid spacing dx.  st[18] holds the
 * work arrays x(1:6), y(1:6), z(1:6), whose values carry over from cell to
 * cell in the reference (a cell with one zero point measures to the x(2)
 * left by an earlier cell); the caller passes their starting values (the
 * reference leaves them undefined) and gets the final ones back. */
double ora_linelength(const double* psi, int nx, int ny, int nz, double dx, double* st);

/* get_zeros, get_extra_zeros and get_re_im_zeros (src/io.f90:895-1402) of a
 * single-domain interior psi on the grid x, y, z: the points of the 12
 * sections in the reference's order (zeros: x-, y-, z-edges, then the
 * xy-, xz-, yz-face extras; re_zeros: x-, y-, z-edges; im_zeros: the
 * same).  counts[12] receives each section's number of points; points (may
 * be NULL) receives 3 doubles per point, sections concatenated, at most cap
 * points.  Returns the total. */
long long ora_zeros(const double* psi, int nx, int ny, int nz, const double* x,
                    const double* y, const double* z, long long* counts, double* points,
                    long long cap);

#ifdef __cplusplus
}
#endif
#endif
