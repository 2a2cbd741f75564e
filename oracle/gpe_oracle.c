/*
 * gpe_oracle.c -- CPU FP64 restatement of the reference GPE solver's
 * finite-difference time-stepping path (liangjj/gpe, Fortran 90 + MPI).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline.  The product never links or calls this file.
 *
 * PARITY UNPINNED against reference outputs: the reference ships no golden
 * vectors and cannot be compiled here (no Fortran compiler, MPI or FFTW2).
 * It is pinned by analytic known-answer tests and a numpy restatement.
 *
 * "Faithful" structure: each routine keeps the reference's pass structure
 * and temporaries -- the dissipation array and deriv_x on every RHS
 * (src/solve.f90:401-411), three separate second-derivative sweeps with a
 * per-point boundary-index call (src/derivs.f90:146-272, 276-398), a Vtrap
 * array per RHS (src/ic.f90:708-726), haloed stage temporaries with a
 * single-rank halo exchange after every stage (src/solve.f90:93-141,
 * src/variables.f90:186-358).  OpenMP threads over z-planes stand in for the
 * reference's MPI ranks when the baseline is timed on several cores.
 *
 * Built with -fcx-fortran-rules so complex multiply/divide follow gfortran's
 * rules.
 */
#include "gpe_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* Adaptive step constants, src/parameters.f90:89-92. */
static const double EPS_RK = 1e-6;
static const double SAFETY = 0.9;
static const double DT_DECREASE = -0.25;
static const double DT_INCREASE = -0.20;

/* Extended-Simpson end weights, src/variables.f90:49-51. */
static const double W1 = 3.0 / 8.0, W2 = 7.0 / 6.0, W3 = 23.0 / 24.0;

struct ora_ctx {
  ora_params p;
  int nx, ny, nz;
  double *x, *y, *z;
  double dx, dy, dz, dx2, dy2, dz2;
  size_t ni, nh;
  /* haloed temporaries (0:nx-1, -2:ny+1, -2:nz+1) */
  cplx *in_h, *tmp_h;
  /* interior temporaries */
  cplx *kk[6], *rhs_tmp, *psi_scal, *err, *tmp_var;
  /* get_rhs temporaries */
  double *diss, *vtrap, *sph;
  cplx *dpsidx, *dxx, *dyy, *dzz, *lap;
};

static inline size_t HX(const ora_ctx* c, int i, int j, int k) {
  return ((size_t)(k + 2) * (size_t)(c->ny + 4) + (size_t)(j + 2)) *
             (size_t)c->nx + (size_t)i;
}
static inline size_t IX(const ora_ctx* c, int i, int j, int k) {
  return ((size_t)k * (size_t)c->ny + (size_t)j) * (size_t)c->nx + (size_t)i;
}

void ora_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int ora_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* get_grid, src/ic.f90:32-69 */
static void make_grid(ora_ctx* c) {
  const ora_params* p = &c->p;
  double xl = -p->xr, yl = -p->yr, zl = -p->zr;
  c->dx = (p->xr - xl) / (double)(p->nx - 1);
  c->dy = (p->yr - yl) / (double)(p->ny - 1);
  c->dz = (p->zr - zl) / (double)(p->nz - 1);
  c->dx2 = c->dx * c->dx;
  c->dy2 = c->dy * c->dy;
  c->dz2 = c->dz * c->dz;
  for (int i = 0; i < p->nx; i++) c->x[i] = xl + (double)i * c->dx;
  for (int j = 0; j < p->ny; j++) c->y[j] = yl + (double)j * c->dy;
  for (int k = 0; k < p->nz; k++) c->z[k] = zl + (double)k * c->dz;
}

static void* xcalloc(size_t n, size_t sz) {
  void* q = calloc(n, sz);
  if (!q) {
    fprintf(stderr, "gpe_oracle: out of memory (%zu x %zu)\n", n, sz);
    abort();
  }
  return q;
}

ora_ctx* ora_create(const ora_params* prm) {
  ora_ctx* c = (ora_ctx*)xcalloc(1, sizeof(ora_ctx));
  c->p = *prm;
  c->nx = prm->nx;
  c->ny = prm->ny;
  c->nz = prm->nz;
  c->ni = (size_t)c->nx * c->ny * c->nz;
  c->nh = (size_t)c->nx * (c->ny + 4) * (c->nz + 4);
  c->x = (double*)xcalloc(c->nx, sizeof(double));
  c->y = (double*)xcalloc(c->ny, sizeof(double));
  c->z = (double*)xcalloc(c->nz, sizeof(double));
  make_grid(c);
  c->in_h = (cplx*)xcalloc(c->nh, sizeof(cplx));
  c->tmp_h = (cplx*)xcalloc(c->nh, sizeof(cplx));
  for (int s = 0; s < 6; s++) c->kk[s] = (cplx*)xcalloc(c->ni, sizeof(cplx));
  c->rhs_tmp = (cplx*)xcalloc(c->ni, sizeof(cplx));
  c->psi_scal = (cplx*)xcalloc(c->ni, sizeof(cplx));
  c->err = (cplx*)xcalloc(c->ni, sizeof(cplx));
  c->tmp_var = (cplx*)xcalloc(c->ni, sizeof(cplx));
  c->diss = (double*)xcalloc(c->ni, sizeof(double));
  c->vtrap = (double*)xcalloc(c->ni, sizeof(double));
  c->sph = (double*)xcalloc(c->ni, sizeof(double));
  c->dpsidx = (cplx*)xcalloc(c->ni, sizeof(cplx));
  c->dxx = (cplx*)xcalloc(c->ni, sizeof(cplx));
  c->dyy = (cplx*)xcalloc(c->ni, sizeof(cplx));
  c->dzz = (cplx*)xcalloc(c->ni, sizeof(cplx));
  c->lap = (cplx*)xcalloc(c->ni, sizeof(cplx));
  return c;
}

void ora_destroy(ora_ctx* c) {
  if (!c) return;
  free(c->x); free(c->y); free(c->z);
  free(c->in_h); free(c->tmp_h);
  for (int s = 0; s < 6; s++) free(c->kk[s]);
  free(c->rhs_tmp); free(c->psi_scal); free(c->err); free(c->tmp_var);
  free(c->diss); free(c->vtrap); free(c->sph);
  free(c->dpsidx); free(c->dxx); free(c->dyy); free(c->dzz); free(c->lap);
  free(c);
}

void ora_grid(const ora_ctx* c, double* x, double* y, double* z) {
  memcpy(x, c->x, sizeof(double) * c->nx);
  memcpy(y, c->y, sizeof(double) * c->ny);
  memcpy(z, c->z, sizeof(double) * c->nz);
}

/* ------------------------------------------------------------------------ */
/* Boundary index maps, src/derivs.f90:276-398.                              */

static void second_index(int bcs, int indx, int n, int* minus, int* plus,
                         int x_deriv) {
  if (bcs == 1) {
    minus[0] = indx - 1;
    plus[0] = indx + 1;
    if (x_deriv) {
      if (indx == 0) { minus[0] = n; plus[0] = 1; }
      if (indx == n) { minus[0] = n - 1; plus[0] = 0; }
    }
  } else {
    minus[0] = indx - 1;
    plus[0] = indx + 1;
    if (indx == 0) { minus[0] = 1; plus[0] = 1; }
    if (indx == n) { minus[0] = n - 1; plus[0] = n - 1; }
  }
}

static void fourth_index(int bcs, int indx, int n, int* minus, int* plus,
                         int x_deriv) {
  if (bcs == 1) {
    minus[0] = indx - 1; minus[1] = indx - 2;
    plus[0] = indx + 1; plus[1] = indx + 2;
    if (x_deriv) {
      if (indx == 0) { minus[0] = n; minus[1] = n - 1; plus[0] = 1; plus[1] = 2; }
      if (indx == 1) { minus[0] = 0; minus[1] = n; plus[0] = 2; plus[1] = 3; }
      if (indx == n - 1) { minus[0] = n - 2; minus[1] = n - 3; plus[0] = n; plus[1] = 0; }
      if (indx == n) { minus[0] = n - 1; minus[1] = n - 2; plus[0] = 0; plus[1] = 1; }
    }
  } else {
    minus[0] = indx - 1; minus[1] = indx - 2;
    plus[0] = indx + 1; plus[1] = indx + 2;
    if (indx == 0) { minus[0] = 1; minus[1] = 2; plus[0] = 1; plus[1] = 2; }
    if (indx == 1) { minus[0] = 0; minus[1] = 1; plus[0] = 2; plus[1] = 3; }
    if (indx == n - 1) { minus[0] = n - 2; minus[1] = n - 3; plus[0] = n; plus[1] = n - 1; }
    if (indx == n) { minus[0] = n - 1; minus[1] = n - 2; plus[0] = n - 1; plus[1] = n - 2; }
  }
}

/* ------------------------------------------------------------------------ */
/* Single-rank halo exchange: send_recv_z + pack_y/send_recv_y/unpack_y      */
/* (src/variables.f90:186-358).  With one rank and periodic BCs every        */
/* neighbour is the rank itself (itable wrap, :123-128), so the exchange is  */
/* a periodic copy of two planes.  With reflective BCs the neighbours are    */
/* MPI_PROC_NULL and the halo is left untouched (never read).               */

static void halo(ora_ctx* c, cplx* f) {
  if (c->p.bcs != 1) return;
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  /* z: two rounds, first the planes two away from the boundary. Only
   * j in js..je (message of nx*jlen starting at (0,js,k)). */
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      f[HX(c, i, j, -2)] = f[HX(c, i, j, nz - 2)];
      f[HX(c, i, j, nz + 1)] = f[HX(c, i, j, 1)];
    }
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      f[HX(c, i, j, -1)] = f[HX(c, i, j, nz - 1)];
      f[HX(c, i, j, nz)] = f[HX(c, i, j, 0)];
    }
  /* y: packed faces for k in kks..kke = 0..nz-1. */
  for (int k = 0; k < nz; k++)
    for (int i = 0; i < nx; i++) {
      cplx a = f[HX(c, i, ny - 2, k)], b = f[HX(c, i, ny - 1, k)];
      cplx d = f[HX(c, i, 0, k)], e = f[HX(c, i, 1, k)];
      f[HX(c, i, -2, k)] = a;
      f[HX(c, i, -1, k)] = b;
      f[HX(c, i, ny, k)] = d;
      f[HX(c, i, ny + 1, k)] = e;
    }
}

/* copy interior -> haloed, then halo exchange (src/gpe.f90:165-174) */
static void to_haloed(ora_ctx* c, const cplx* in, cplx* h) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      memcpy(&h[HX(c, 0, j, k)], &in[IX(c, 0, j, k)], sizeof(cplx) * nx);
  halo(c, h);
}

/* ------------------------------------------------------------------------ */
/* Derivatives, src/derivs.f90:25-272.  f is haloed, out is interior.        */

static void deriv_x(ora_ctx* c, const cplx* f, cplx* fx) {
  const int nx = c->nx, ny = c->ny, nz = c->nz, bcs = c->p.bcs;
  const double dx = c->dx;
  if (c->p.order == 2) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          int m[2] = {0, 0}, pl[2] = {0, 0};
          second_index(bcs, i, nx - 1, m, pl, 1);
          fx[IX(c, i, j, k)] =
              (f[HX(c, pl[0], j, k)] - f[HX(c, m[0], j, k)]) / (2.0 * dx);
        }
  } else {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          int m[2] = {0, 0}, pl[2] = {0, 0};
          fourth_index(bcs, i, nx - 1, m, pl, 1);
          fx[IX(c, i, j, k)] =
              (-f[HX(c, pl[1], j, k)] + 8.0 * f[HX(c, pl[0], j, k)] -
               8.0 * f[HX(c, m[0], j, k)] + f[HX(c, m[1], j, k)]) /
              (12.0 * dx);
        }
  }
}

static void deriv_y(ora_ctx* c, const cplx* f, cplx* fy) {
  const int nx = c->nx, ny = c->ny, nz = c->nz, bcs = c->p.bcs;
  const double dy = c->dy;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      int m[2] = {0, 0}, pl[2] = {0, 0};
      if (c->p.order == 2) {
        second_index(bcs, j, ny - 1, m, pl, 0);
        for (int i = 0; i < nx; i++)
          fy[IX(c, i, j, k)] =
              (f[HX(c, i, pl[0], k)] - f[HX(c, i, m[0], k)]) / (2.0 * dy);
      } else {
        fourth_index(bcs, j, ny - 1, m, pl, 0);
        for (int i = 0; i < nx; i++)
          fy[IX(c, i, j, k)] =
              (-f[HX(c, i, pl[1], k)] + 8.0 * f[HX(c, i, pl[0], k)] -
               8.0 * f[HX(c, i, m[0], k)] + f[HX(c, i, m[1], k)]) /
              (12.0 * dy);
      }
    }
}

static void deriv_z(ora_ctx* c, const cplx* f, cplx* fz) {
  const int nx = c->nx, ny = c->ny, nz = c->nz, bcs = c->p.bcs;
  const double dz = c->dz;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      int m[2] = {0, 0}, pl[2] = {0, 0};
      if (c->p.order == 2) {
        second_index(bcs, k, nz - 1, m, pl, 0);
        for (int i = 0; i < nx; i++)
          fz[IX(c, i, j, k)] =
              (f[HX(c, i, j, pl[0])] - f[HX(c, i, j, m[0])]) / (2.0 * dz);
      } else {
        fourth_index(bcs, k, nz - 1, m, pl, 0);
        for (int i = 0; i < nx; i++)
          fz[IX(c, i, j, k)] =
              (-f[HX(c, i, j, pl[1])] + 8.0 * f[HX(c, i, j, pl[0])] -
               8.0 * f[HX(c, i, j, m[0])] + f[HX(c, i, j, m[1])]) /
              (12.0 * dz);
      }
    }
}

static void deriv_xx(ora_ctx* c, const cplx* f, cplx* fxx) {
  const int nx = c->nx, ny = c->ny, nz = c->nz, bcs = c->p.bcs;
  const double dx2 = c->dx2;
  if (c->p.order == 2) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          int m[2] = {0, 0}, pl[2] = {0, 0};
          second_index(bcs, i, nx - 1, m, pl, 1);
          fxx[IX(c, i, j, k)] = (f[HX(c, pl[0], j, k)] -
                                 2.0 * f[HX(c, i, j, k)] +
                                 f[HX(c, m[0], j, k)]) / dx2;
        }
  } else {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          int m[2] = {0, 0}, pl[2] = {0, 0};
          fourth_index(bcs, i, nx - 1, m, pl, 1);
          fxx[IX(c, i, j, k)] =
              (-f[HX(c, pl[1], j, k)] + 16.0 * f[HX(c, pl[0], j, k)] -
               30.0 * f[HX(c, i, j, k)] + 16.0 * f[HX(c, m[0], j, k)] -
               f[HX(c, m[1], j, k)]) / (12.0 * dx2);
        }
  }
}

static void deriv_yy(ora_ctx* c, const cplx* f, cplx* fyy) {
  const int nx = c->nx, ny = c->ny, nz = c->nz, bcs = c->p.bcs;
  const double dy2 = c->dy2;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      int m[2] = {0, 0}, pl[2] = {0, 0};
      if (c->p.order == 2) {
        second_index(bcs, j, ny - 1, m, pl, 0);
        for (int i = 0; i < nx; i++)
          fyy[IX(c, i, j, k)] = (f[HX(c, i, pl[0], k)] -
                                 2.0 * f[HX(c, i, j, k)] +
                                 f[HX(c, i, m[0], k)]) / dy2;
      } else {
        fourth_index(bcs, j, ny - 1, m, pl, 0);
        for (int i = 0; i < nx; i++)
          fyy[IX(c, i, j, k)] =
              (-f[HX(c, i, pl[1], k)] + 16.0 * f[HX(c, i, pl[0], k)] -
               30.0 * f[HX(c, i, j, k)] + 16.0 * f[HX(c, i, m[0], k)] -
               f[HX(c, i, m[1], k)]) / (12.0 * dy2);
      }
    }
}

static void deriv_zz(ora_ctx* c, const cplx* f, cplx* fzz) {
  const int nx = c->nx, ny = c->ny, nz = c->nz, bcs = c->p.bcs;
  const double dz2 = c->dz2;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      int m[2] = {0, 0}, pl[2] = {0, 0};
      if (c->p.order == 2) {
        second_index(bcs, k, nz - 1, m, pl, 0);
        for (int i = 0; i < nx; i++)
          fzz[IX(c, i, j, k)] = (f[HX(c, i, j, pl[0])] -
                                 2.0 * f[HX(c, i, j, k)] +
                                 f[HX(c, i, j, m[0])]) / dz2;
      } else {
        fourth_index(bcs, k, nz - 1, m, pl, 0);
        for (int i = 0; i < nx; i++)
          fzz[IX(c, i, j, k)] =
              (-f[HX(c, i, j, pl[1])] + 16.0 * f[HX(c, i, j, pl[0])] -
               30.0 * f[HX(c, i, j, k)] + 16.0 * f[HX(c, i, j, m[0])] -
               f[HX(c, i, j, m[1])]) / (12.0 * dz2);
      }
    }
}

/* laplacian, src/variables.f90:55-71 */
static void laplacian_h(ora_ctx* c, const cplx* f, cplx* lap) {
  deriv_xx(c, f, c->dxx);
  deriv_yy(c, f, c->dyy);
  deriv_zz(c, f, c->dzz);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < c->nz; k++) {
    size_t b = IX(c, 0, 0, k), e = b + (size_t)c->nx * c->ny;
    for (size_t q = b; q < e; q++) lap[q] = c->dxx[q] + c->dyy[q] + c->dzz[q];
  }
}

/* Vtrap, src/ic.f90:708-726 */
static void vtrap(ora_ctx* c, double* v) {
  const ora_params* p = &c->p;
  double om[3] = {p->omx, p->omy, p->omz};
#pragma omp parallel for schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++)
        v[IX(c, i, j, k)] = 0.5 * ((om[0] * om[0]) * (c->x[i] * c->x[i]) +
                                   (om[1] * om[1]) * (c->y[j] * c->y[j]) +
                                   (om[2] * om[2]) * (c->z[k] * c->z[k]));
}

/* sphere, src/ic.f90:635-657 */
static void sphere(ora_ctx* c, double* s) {
  const double rad = 10.0, eps1 = 2.0;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++)
        s[IX(c, i, j, k)] =
            0.5 * (1.0 + tanh(sqrt(c->x[i] * c->x[i] + c->y[j] * c->y[j] +
                                   c->z[k] * c->z[k]) -
                              rad - eps1));
}

/* get_rhs, src/solve.f90:382-440.  in is haloed, rhs interior. */
static void get_rhs(ora_ctx* c, const cplx* in, cplx* rhs) {
  const ora_params* p = &c->p;
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  const double a = c->x[nx - 3], b = c->y[ny - 3], cc = c->z[nz - 3];
  double* diss = c->diss;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        diss[IX(c, i, j, k)] =
            p->diss_amp *
            ((1.0 + tanh(c->x[i] - a) * tanh(c->x[i] + a)) +
             (1.0 + tanh(c->y[j] - b) * tanh(c->y[j] + b)) +
             (1.0 + tanh(c->z[k] - cc) * tanh(c->z[k] + cc)));

  deriv_x(c, in, c->dpsidx);

  switch (p->eqn_to_solve) {
    case 1:
    case 3: {
      laplacian_h(c, in, c->lap);
      if (p->eqn_to_solve == 3) sphere(c, c->sph);
#pragma omp parallel for schedule(static)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) {
            size_t q = IX(c, i, j, k);
            cplx psi = in[HX(c, i, j, k)];
            double ab = cabs(psi);
            cplx r = 0.5 * (I + diss[q]) *
                         (c->lap[q] + (1.0 - ab * ab) * psi) +
                     p->Urhs * c->dpsidx[q];
            if (p->eqn_to_solve == 3) r = r * c->sph[q];
            rhs[q] = r;
          }
      break;
    }
    case 2: {
      laplacian_h(c, in, c->lap);
#pragma omp parallel for schedule(static)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) {
            size_t q = IX(c, i, j, k);
            cplx psi = in[HX(c, i, j, k)];
            double ab = cabs(psi);
            rhs[q] = I * (c->lap[q] - (ab * ab) * psi) + p->Urhs * c->dpsidx[q];
          }
      break;
    }
    case 4: {
      laplacian_h(c, in, c->lap);
      vtrap(c, c->vtrap);
#pragma omp parallel for schedule(static)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) {
            size_t q = IX(c, i, j, k);
            cplx psi = in[HX(c, i, j, k)];
            cplx inner = -0.5 * c->lap[q] + c->vtrap[q] * psi +
                         p->g * (cabs(psi * psi) * psi) - p->mu * psi;
            rhs[q] = -I * inner;
          }
      break;
    }
    default:
      memset(rhs, 0, sizeof(cplx) * c->ni);
  }
}

/* ------------------------------------------------------------------------ */
/* Time integrators, src/solve.f90:57-378.                                   */

#define INTERIOR_LOOP(body)                                  \
  _Pragma("omp parallel for schedule(static)")               \
  for (int k = 0; k < nz; k++)                               \
    for (int j = 0; j < ny; j++)                             \
      for (int i = 0; i < nx; i++) {                         \
        size_t q = IX(c, i, j, k);                           \
        size_t h = HX(c, i, j, k);                           \
        (void)h;                                             \
        body                                                 \
      }

static void euler(ora_ctx* c, const cplx* old, cplx* out, cplx dt) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  cplx* rhs = c->kk[0];
  get_rhs(c, old, rhs);
  INTERIOR_LOOP(out[q] = old[h] + dt * rhs[q];)
}

static void rk2(ora_ctx* c, const cplx* old, cplx* out, cplx dt) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  cplx *k1 = c->kk[0], *k2 = c->kk[1], *tmp = c->tmp_h;
  const cplx hdt = 0.5 * dt;
  get_rhs(c, old, k1);
  INTERIOR_LOOP(tmp[h] = old[h] + hdt * k1[q];)
  halo(c, tmp);
  get_rhs(c, tmp, k2);
  INTERIOR_LOOP(out[q] = old[h] + dt * k2[q];)
}

static void rk4(ora_ctx* c, const cplx* old, cplx* out, cplx dt) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  cplx *k1 = c->kk[0], *k2 = c->kk[1], *k3 = c->kk[2], *k4 = c->kk[3];
  cplx* tmp = c->tmp_h;
  const cplx hdt = 0.5 * dt;
  get_rhs(c, old, k1);
  INTERIOR_LOOP(tmp[h] = old[h] + hdt * k1[q];)
  halo(c, tmp);
  get_rhs(c, tmp, k2);
  INTERIOR_LOOP(tmp[h] = old[h] + hdt * k2[q];)
  halo(c, tmp);
  get_rhs(c, tmp, k3);
  INTERIOR_LOOP(tmp[h] = old[h] + dt * k3[q];)
  halo(c, tmp);
  get_rhs(c, tmp, k4);
  INTERIOR_LOOP(out[q] = old[h] + dt * (k1[q] / 6.0 + k2[q] / 3.0 +
                                        k3[q] / 3.0 + k4[q] / 6.0);)
}

/* rkck: Cash-Karp coefficients, src/solve.f90:255-281 */
static const double B21 = 0.2;
static const double B31 = 0.075, B32 = 0.225;
static const double B41 = 0.3, B42 = -0.9, B43 = 1.2;
#define B51 (-11.0 / 54.0)
#define B52 (2.5)
#define B53 (-70.0 / 27.0)
#define B54 (35.0 / 27.0)
#define B61 (1631.0 / 55296.0)
#define B62 (175.0 / 512.0)
#define B63 (575.0 / 13824.0)
#define B64 (44275.0 / 110592.0)
#define B65 (253.0 / 4096.0)
#define C1 (37.0 / 378.0)
#define C2 (0.0)
#define C3 (250.0 / 621.0)
#define C4 (125.0 / 594.0)
#define C5 (0.0)
#define C6 (512.0 / 1771.0)
#define DC1 (C1 - 2825.0 / 27648.0)
#define DC2 (C2 - 0.0)
#define DC3 (C3 - 18575.0 / 48384.0)
#define DC4 (C4 - 13525.0 / 55296.0)
#define DC5 (C5 - 277.0 / 14336.0)
#define DC6 (C6 - 0.25)

static void rkck(ora_ctx* c, const cplx* old, cplx* out, cplx* err, cplx dt) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  cplx *k1 = c->kk[0], *k2 = c->kk[1], *k3 = c->kk[2], *k4 = c->kk[3],
       *k5 = c->kk[4], *k6 = c->kk[5];
  cplx* tmp = c->tmp_h;
  get_rhs(c, old, k1);
  INTERIOR_LOOP(k1[q] = dt * k1[q]; tmp[h] = old[h] + B21 * k1[q];)
  halo(c, tmp);
  get_rhs(c, tmp, k2);
  INTERIOR_LOOP(k2[q] = dt * k2[q];
                tmp[h] = old[h] + B31 * k1[q] + B32 * k2[q];)
  halo(c, tmp);
  get_rhs(c, tmp, k3);
  INTERIOR_LOOP(k3[q] = dt * k3[q];
                tmp[h] = old[h] + B41 * k1[q] + B42 * k2[q] + B43 * k3[q];)
  halo(c, tmp);
  get_rhs(c, tmp, k4);
  INTERIOR_LOOP(k4[q] = dt * k4[q];
                tmp[h] = old[h] + B51 * k1[q] + B52 * k2[q] + B53 * k3[q] +
                         B54 * k4[q];)
  halo(c, tmp);
  get_rhs(c, tmp, k5);
  INTERIOR_LOOP(k5[q] = dt * k5[q];
                tmp[h] = old[h] + B61 * k1[q] + B62 * k2[q] + B63 * k3[q] +
                         B64 * k4[q] + B65 * k5[q];)
  halo(c, tmp);
  get_rhs(c, tmp, k6);
  INTERIOR_LOOP(k6[q] = dt * k6[q];)
  INTERIOR_LOOP(out[q] = old[h] + C1 * k1[q] + C2 * k2[q] + C3 * k3[q] +
                         C4 * k4[q] + C5 * k5[q] + C6 * k6[q];
                err[q] = DC1 * k1[q] + DC2 * k2[q] + DC3 * k3[q] +
                         DC4 * k4[q] + DC5 * k5[q] + DC6 * k6[q];)
}

/* rkqs, src/solve.f90:158-244 (the timestep.dat write is the caller's). */
static void rkqs(ora_ctx* c, const cplx* in, cplx* out, ora_time* tm,
                 double* errmax_out, int* attempts) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  const double errcon = pow(5.0 / SAFETY, 1.0 / DT_INCREASE);
  cplx dt = tm->dt_re + I * tm->dt_im;
  cplx* ps = c->psi_scal;
  get_rhs(c, in, ps);
  INTERIOR_LOOP(ps[q] = cabs(in[h]) + dt * cabs(ps[q]) + 1e-30;)
  double errmax = 0.0;
  int n_att = 0;
  for (;;) {
    n_att++;
    rkck(c, in, c->tmp_var, c->err, dt);
    /* maxval(abs(err/psi_scal))/eps, then MPI_ALLREDUCE(MAXLOC) */
    double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
    for (size_t q = 0; q < c->ni; q++) {
      double v = cabs(c->err[q] / ps[q]);
      if (v > m) m = v;
    }
    errmax = m / EPS_RK;
    if (errmax <= 1.0) break;
    cplx dt_temp = SAFETY * dt * pow(errmax, DT_DECREASE);
    double mag = fmax(cabs(dt_temp), 0.1 * cabs(dt));
    if (!c->p.real_time)
      dt = 0.0 - I * mag;
    else
      dt = mag + 0.0 * I;
    if (n_att > 10000) break; /* guard: reference loops forever */
  }
  cplx dt_next;
  if (errmax > errcon)
    dt_next = SAFETY * dt * pow(errmax, DT_INCREASE);
  else
    dt_next = 5.0 * dt;
  tm->t = tm->t + creal(dt);
  dt = dt_next;
  tm->im_t = tm->im_t + fabs(cimag(dt));
  tm->dt_re = creal(dt);
  tm->dt_im = cimag(dt);
  memcpy(out, c->tmp_var, sizeof(cplx) * c->ni);
  if (errmax_out) *errmax_out = errmax;
  if (attempts) *attempts = n_att;
}

int ora_solver(ora_ctx* c, const double* psi_in, double* psi_out,
               ora_time* tm, double* errmax, int* attempts) {
  const cplx* in = (const cplx*)psi_in;
  cplx* out = (cplx*)psi_out;
  to_haloed(c, in, c->in_h);
  cplx dt = tm->dt_re + I * tm->dt_im;
  if (errmax) *errmax = 0.0;
  if (attempts) *attempts = 1;
  switch (c->p.scheme) {
    case ORA_EULER: euler(c, c->in_h, out, dt); break;
    case ORA_RK2: rk2(c, c->in_h, out, dt); break;
    case ORA_RK4: rk4(c, c->in_h, out, dt); break;
    case ORA_RK45: rkqs(c, c->in_h, out, tm, errmax, attempts); return 0;
    default: return -1;
  }
  tm->t = tm->t + creal(dt);
  tm->im_t = tm->im_t + fabs(cimag(dt));
  return 0;
}

void ora_rhs(ora_ctx* c, const double* psi, double* rhs) {
  to_haloed(c, (const cplx*)psi, c->in_h);
  get_rhs(c, c->in_h, (cplx*)rhs);
}

void ora_laplacian(ora_ctx* c, const double* psi, double* lap) {
  to_haloed(c, (const cplx*)psi, c->in_h);
  laplacian_h(c, c->in_h, (cplx*)lap);
}

void ora_deriv(ora_ctx* c, int axis, int second, const double* psi,
               double* out) {
  to_haloed(c, (const cplx*)psi, c->in_h);
  cplx* o = (cplx*)out;
  if (second) {
    if (axis == 0) deriv_xx(c, c->in_h, o);
    else if (axis == 1) deriv_yy(c, c->in_h, o);
    else deriv_zz(c, c->in_h, o);
  } else {
    if (axis == 0) deriv_x(c, c->in_h, o);
    else if (axis == 1) deriv_y(c, c->in_h, o);
    else deriv_z(c, c->in_h, o);
  }
}

/* ------------------------------------------------------------------------ */
/* Reductions, src/variables.f90:537-587, 698-823.                           */

double ora_get_norm(ora_ctx* c, const double* psi_) {
  const cplx* psi = (const cplx*)psi_;
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  double* int_x = (double*)xcalloc((size_t)ny * nz, sizeof(double));
  double* int_y = (double*)xcalloc((size_t)nz, sizeof(double));
  /* integrate_x */
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      const cplx* r = &psi[IX(c, 0, j, k)];
#define IV(ii) (cabs(r[ii]) * cabs(r[ii]))
      double s = 0.0;
      for (int i = 3; i <= nx - 4; i++) s += IV(i);
      int_x[(size_t)k * ny + j] =
          (W1 * IV(0) + W2 * IV(1) + W3 * IV(2) + s + W3 * IV(nx - 3) +
           W2 * IV(nx - 2) + W1 * IV(nx - 1)) * c->dx;
#undef IV
    }
  /* integrate_y */
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++) {
    double s = 0.0;
    for (int j = 0; j < ny; j++) {
      double v = int_x[(size_t)k * ny + j], tv = v;
      if (j == 0) tv = W1 * v;
      if (j == 1) tv = W2 * v;
      if (j == 2) tv = W3 * v;
      if (j == ny - 3) tv = W3 * v;
      if (j == ny - 2) tv = W2 * v;
      if (j == ny - 1) tv = W1 * v;
      s += tv;
    }
    int_y[k] = s * c->dy;
  }
  /* integrate_z */
  double s = 0.0;
  for (int k = 0; k < nz; k++) {
    double v = int_y[k], tv = v;
    if (k == 0) tv = W1 * v;
    if (k == 1) tv = W2 * v;
    if (k == 2) tv = W3 * v;
    if (k == nz - 3) tv = W3 * v;
    if (k == nz - 2) tv = W2 * v;
    if (k == nz - 1) tv = W1 * v;
    s += tv;
  }
  free(int_x);
  free(int_y);
  return s * c->dz;
}

/* integrate_x / integrate_y / integrate_z (src/variables.f90:713-823) of a
 * real interior field: the extended-Simpson rule as get_norm applies it. */
static double integrate_xyz(ora_ctx* c, const double* f) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  double* int_x = (double*)xcalloc((size_t)ny * nz, sizeof(double));
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      const double* r = &f[IX(c, 0, j, k)];
      double s = 0.0;
      for (int i = 3; i <= nx - 4; i++) s += r[i];
      int_x[(size_t)k * ny + j] = (W1 * r[0] + W2 * r[1] + W3 * r[2] + s + W3 * r[nx - 3] +
                                   W2 * r[nx - 2] + W1 * r[nx - 1]) * c->dx;
    }
  double tot = 0.0;
  for (int k = 0; k < nz; k++) {
    double sy = 0.0;
    for (int j = 0; j < ny; j++) {
      double v = int_x[(size_t)k * ny + j], tv = v;
      if (j == 0) tv = W1 * v;
      if (j == 1) tv = W2 * v;
      if (j == 2) tv = W3 * v;
      if (j == ny - 3) tv = W3 * v;
      if (j == ny - 2) tv = W2 * v;
      if (j == ny - 1) tv = W1 * v;
      sy += tv;
    }
    double v = sy * c->dy, tv = v;
    if (k == 0) tv = W1 * v;
    if (k == 1) tv = W2 * v;
    if (k == 2) tv = W3 * v;
    if (k == nz - 3) tv = W3 * v;
    if (k == nz - 2) tv = W2 * v;
    if (k == nz - 1) tv = W1 * v;
    tot += tv;
  }
  free(int_x);
  return tot * c->dz;
}

/* mass (src/variables.f90:590-610): plain sum of |psi|^2 times dx dy dz. */
double ora_mass(ora_ctx* c, const double* psi_) {
  const cplx* psi = (const cplx*)psi_;
  const size_t n = (size_t)c->nx * c->ny * c->nz;
  double s = 0.0;
  for (size_t q = 0; q < n; q++) s += creal(psi[q]) * creal(psi[q]) + cimag(psi[q]) * cimag(psi[q]);
  return s * c->dx * c->dy * c->dz;
}

/* momentum (src/variables.f90:615-694): for each axis d,
 * integral of (Re psi - 1) Im(d conj(psi)) - Im psi Re(d psi). */
void ora_momentum(ora_ctx* c, const double* psi_, double mom[3]) {
  const cplx* psi = (const cplx*)psi_;
  const size_t n = (size_t)c->nx * c->ny * c->nz;
  cplx* d = (cplx*)xcalloc(n, sizeof(cplx));
  double* f = (double*)xcalloc(n, sizeof(double));
  for (int a = 0; a < 3; a++) {
    ora_deriv(c, a, 0, psi_, (double*)d);
    for (size_t q = 0; q < n; q++) {
      const cplx dstar = conj(d[q]); /* deriv of conj(psi): the stencil is real */
      f[q] = (creal(psi[q]) - 1.0) * cimag(dstar) - cimag(psi[q]) * creal(d[q]);
    }
    mom[a] = integrate_xyz(c, f);
  }
  free(d);
  free(f);
}

double ora_energy(ora_ctx* c, const double* psi_) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  to_haloed(c, (const cplx*)psi_, c->in_h);
  laplacian_h(c, c->in_h, c->lap);
  double* part = (double*)xcalloc((size_t)nz, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++) {
    double s = 0.0;
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        cplx psi = c->in_h[HX(c, i, j, k)];
        double a = cabs(psi);
        double a2 = a * a;
        s += creal(-c->lap[IX(c, i, j, k)] * conj(psi) + 0.5 * (a2 * a2));
      }
    part[k] = s;
  }
  double E = 0.0;
  for (int k = 0; k < nz; k++) E += part[k];
  free(part);
  return E * c->dx * c->dy * c->dz;
}

double ora_hamiltonian4(ora_ctx* c, const double* psi_) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  const ora_params* p = &c->p;
  to_haloed(c, (const cplx*)psi_, c->in_h);
  laplacian_h(c, c->in_h, c->lap);
  vtrap(c, c->vtrap);
  double* part = (double*)xcalloc((size_t)nz, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++) {
    double s = 0.0;
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t q = IX(c, i, j, k);
        cplx psi = c->in_h[HX(c, i, j, k)];
        double a2 = creal(psi) * creal(psi) + cimag(psi) * cimag(psi);
        s += 0.5 * creal(-c->lap[q] * conj(psi)) + c->vtrap[q] * a2 +
             0.5 * p->g * a2 * a2 - p->mu * a2;
      }
    part[k] = s;
  }
  double H = 0.0;
  for (int k = 0; k < nz; k++) H += part[k];
  free(part);
  return H * c->dx * c->dy * c->dz;
}

void ora_renormalise(ora_ctx* c, double* psi_, double norm) {
  cplx* psi = (cplx*)psi_;
  const double snn = sqrt(c->p.nn), sn = sqrt(norm);
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < c->ni; q++) psi[q] = snn * psi[q] / sn;
}

/* ------------------------------------------------------------------------ */
/* Initial conditions, src/ic.f90.                                          */

double ora_get_rr(double r) {
  return sqrt((0.3437 + 0.0286 * r * r) /
              (1.0 + (0.3333 * r * r) + (0.0286 * (r * r) * (r * r))));
}

/* vortex_line with get_theta / get_r / amp, src/ic.f90:309-348, 730-884 */
void ora_ic_vortex_line(ora_ctx* c, double x0, double y0, double z0,
                        double a1, double a2, double ll, double sgn, char dir,
                        int imprint_phase, double* out_) {
  cplx* out = (cplx*)out_;
  const double scal = c->p.scal, pi = 3.1415926535897932384626433832795;
  double safe1 = 0.0, safe2 = 0.0;
  if (fabs(ll) < 2.220446049250313e-16) {
    if (fabs(a1) < 2.220446049250313e-16) safe1 = 1.0;
    if (fabs(a2) < 2.220446049250313e-16) safe2 = 1.0;
  }
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double X = c->x[i], Y = c->y[j], Z = c->z[k], th, r;
        if (dir == 'x') {
          double u = scal * (Y - y0 - a1 * sin(2.0 * pi * (X - x0) / (ll + safe1)));
          double v = scal * (Z - z0 - a2 * cos(2.0 * pi * (X - x0) / (ll + safe2)));
          th = sgn * atan2(v, u);
          r = sqrt(scal * pow(Y - y0 - a1 * sin(2.0 * pi * (X - x0) / (ll + safe1)), 2) +
                   scal * pow(Z - z0 - a2 * cos(2.0 * pi * (X - x0) / (ll + safe2)), 2));
        } else if (dir == 'y') {
          double u = scal * (Z - z0 - a1 * sin(2.0 * pi * (Y - y0) / (ll + safe1)));
          double v = scal * (X - x0 - a2 * cos(2.0 * pi * (Y - y0) / (ll + safe2)));
          th = sgn * atan2(v, u);
          r = sqrt(scal * pow(Z - z0 - a1 * sin(2.0 * pi * (Y - y0) / (ll + safe1)), 2) +
                   scal * pow(X - x0 - a2 * cos(2.0 * pi * (Y - y0) / (ll + safe2)), 2));
        } else {
          double u = scal * (X - x0 - a1 * sin(2.0 * pi * (Z - z0) / (ll + safe1)));
          double v = scal * (Y - y0 - a2 * cos(2.0 * pi * (Z - z0) / (ll + safe2)));
          th = sgn * atan2(v, u);
          r = sqrt(scal * pow(X - x0 - a1 * sin(2.0 * pi * (Z - z0) / (ll + safe1)), 2) +
                   scal * pow(Y - y0 - a2 * cos(2.0 * pi * (Z - z0) / (ll + safe2)), 2));
        }
        cplx ph = cexp(I * th);
        if (imprint_phase)
          out[IX(c, i, j, k)] = ph;
        else
          out[IX(c, i, j, k)] = (1.0 - exp(-0.7 * pow(r, 1.15))) * ph;
      }
}

/* vortex_ring, src/ic.f90:352-509 */
void ora_ic_vortex_ring(ora_ctx* c, const char* plane, double x0, double y0,
                        double z0, double r0, double amp, int mm, double r1,
                        int kk, double dir, double* out_) {
  cplx* out = (cplx*)out_;
  const double scal = c->p.scal;
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double X = c->x[i], Y = c->y[j], Z = c->z[k];
        double a, b, along, c0, ctr;  /* plane coords, axis coord */
        if (plane[0] == 'x' && plane[1] == 'y') {
          a = X - x0; b = Y - y0; along = Z; ctr = z0;
        } else if (plane[0] == 'x' && plane[1] == 'z') {
          a = X - x0; b = Z - z0; along = Y; ctr = y0;
        } else {
          a = Y - y0; b = Z - z0; along = X; ctr = x0;
        }
        (void)c0;
        double theta = atan2(b, a);
        double s = sqrt(a * a + b * b) - r1 * sin((double)kk * theta);
        double dist = amp * cos((double)mm * theta);
        double pp = along - r1 * cos((double)kk * theta);
        double d1 = sqrt(pow(scal * (pp - ctr), 2) + pow(scal * (s + r0 - dist), 2));
        double d2 = sqrt(pow(scal * (pp - ctr), 2) + pow(scal * (s - r0 - dist), 2));
        double rr1 = ora_get_rr(d1), rr2 = ora_get_rr(d2);
        out[IX(c, i, j, k)] =
            rr1 * ((scal * (pp - ctr)) + dir * I * (scal * (s + r0 - dist))) *
            rr2 * ((scal * (pp - ctr)) - dir * I * (scal * (s - r0 - dist)));
      }
}

/* pade_pulse_ring, src/ic.f90:513-582 */
void ora_ic_pade_pulse_ring(ora_ctx* c, const char* pulse_or_ring, double x0,
                            double y0, double z0, double r0, double* out_) {
  cplx* out = (cplx*)out_;
  double a[9], U, m;
  if (strcmp(pulse_or_ring, "pulse") == 0) {
    const double t[9] = {-0.79792, 0.00388059, 0.00882276, -0.7981,
                         -0.012783, -0.0574092, 0.0399, 0.199, 0.0058};
    memcpy(a, t, sizeof a);
    U = 0.63; m = 8.37;
  } else {
    const double t[9] = {-1.1, 0.0170524, 0.0289452, -0.953, -0.0049767,
                         -0.0594346, 0.04, 0.21, 0.00612};
    memcpy(a, t, sizeof a);
    U = 0.6; m = 8.97;
  }
  const double pw = 7.0 / 4.0;
  const double one_2u = 1.0 - 2.0 * U * U;
  const double a9p = pow(a[8], pw);
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++) {
      double s = sqrt(pow(c->y[j] - y0, 2) + pow(c->z[k] - z0, 2));
      double s2 = pow(s - r0, 2);
      for (int i = 0; i < c->nx; i++) {
        double x2 = pow(c->x[i] - x0, 2);
        double q = x2 + one_2u * s2;
        double denom = pow(1.0 + a[7] * x2 + a[6] * s2 + a[8] * q * q, pw);
        double uu = 1.0 + (a[0] + a[2] * x2 + a[1] * s2 +
                           m * a9p * U * (2.0 * x2 - one_2u * s2)) * q / denom;
        double vv = (c->x[i] - x0) *
                    (a[3] + a[5] * x2 + a[4] * s2 - m * a9p * q * q) / denom;
        out[IX(c, i, j, k)] = uu + I * vv;
      }
    }
}

/* fermi, src/ic.f90:273-305 */
void ora_ic_fermi(ora_ctx* c, double* out_) {
  cplx* out = (cplx*)out_;
  vtrap(c, c->vtrap);
  for (size_t q = 0; q < c->ni; q++) {
    double f = (c->p.mu - c->vtrap[q]) / c->p.g;
    out[q] = (f >= 0.0) ? sqrt(f) : 0.0;
  }
}


/* ------------------------------------------------------------------------
 * linelength (src/variables.f90:879-1145), the reference's loops literally.
 * Cells (i, j, k) with 1 <= i <= nx-2 and the same for j, k; on each of the
 * 6 faces the zero lines of Re psi and Im psi are located by linear
 * interpolation along the face edges and intersected; two points found on
 * the cell's faces give a segment.  Faces: 1 front (k), 2 back (k+1),
 * 3 right (i+1), 4 left (i), 5 top (j+1), 6 bottom (j). */
static void face_corners(const double* psi, int nx, int ny, int i, int j, int k, int n,
                         double u[6], double v[6]) {
  /* corner (di, dj, dk) of corners 1..4 for each face */
  static const int cor[6][4][3] = {
      {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}},
      {{0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}},
      {{1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {1, 1, 0}},
      {{0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}},
      {{0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}},
      {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}}};
  for (int q = 0; q < 4; q++) {
    const int* d = cor[n - 1][q];
    const size_t at = (((size_t)(k + d[2]) * ny + (j + d[1])) * nx + (i + d[0])) * 2;
    u[q + 1] = psi[at];
    v[q + 1] = psi[at + 1];
  }
  u[5] = u[1];
  v[5] = v[1];
}

/* The zero points of one component along the face edges (the q loops of
 * src/variables.f90:990-1072): returns lu (or lv). */
static int edge_zeros(const double w[6], double xw[7], double yw[7]) {
  int l = 1;
  for (int q = 1; q <= 4; q++) {
    if (w[q] == 0.0) {
      switch (q) {
        case 1: xw[l] = 0.0; yw[l] = 0.0; break;
        case 2: xw[l] = 1.0; yw[l] = 0.0; break;
        case 3: xw[l] = 1.0; yw[l] = 1.0; break;
        default: xw[l] = 0.0; yw[l] = 1.0; break;
      }
    } else if (w[q] * w[q + 1] < 0.0) {
      switch (q) {
        case 1: xw[l] = fabs(w[q] / (w[q] - w[q + 1])); yw[l] = 0.0; break;
        case 2: xw[l] = 1.0; yw[l] = fabs(w[q] / (w[q] - w[q + 1])); break;
        case 3: xw[l] = fabs(w[q + 1] / (w[q] - w[q + 1])); yw[l] = 1.0; break;
        default: xw[l] = 0.0; yw[l] = fabs(w[q + 1] / (w[q] - w[q + 1])); break;
      }
      if (l == 1 || xw[l] != xw[l - 1] || yw[l] != yw[l - 1]) l++;
    }
  }
  return l;
}

double ora_linelength(const double* psi, int nx, int ny, int nz, double dx, double* st) {
  double* x = st - 1;       /* x(1:6) */
  double* y = st + 6 - 1;   /* y(1:6) */
  double* z = st + 12 - 1;  /* z(1:6) */
  double xu[7] = {0}, yu[7] = {0}, xv[7] = {0}, yv[7] = {0};
  double L = 0.0;
  for (int k = 1; k <= nz - 2; k++)
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        int m = 1;
        int skip = 0;
        for (int n = 1; n <= 6 && !skip; n++) {
          double u[6], v[6];
          face_corners(psi, nx, ny, i, j, k, n, u, v);
          /* a zero plane of one component crossed by the other */
          if ((u[1] == 0.0 && u[2] == 0.0 && u[3] == 0.0 && u[4] == 0.0 &&
               (v[1] * v[2] < 0.0 || v[2] * v[3] < 0.0 || v[3] * v[4] < 0.0 ||
                v[4] * v[1] < 0.0)) ||
              (v[1] == 0.0 && v[2] == 0.0 && v[3] == 0.0 && v[4] == 0.0 &&
               (u[1] * u[2] < 0.0 || u[2] * u[3] < 0.0 || u[3] * u[4] < 0.0 ||
                u[4] * u[1] < 0.0))) {
            L += 0.5;
            skip = 1;
            break;
          }
          /* a zero edge of both components */
          for (int q = 1; q <= 4; q++)
            if (u[q] == 0.0 && u[q + 1] == 0.0 && v[q] == 0.0 && v[q + 1] == 0.0) {
              L += 0.25;
              skip = 1;
              break;
            }
          if (skip) break;
          const int lu = edge_zeros(u, xu, yu);
          const int lv = edge_zeros(v, xv, yv);
          if (lu > 2 && lv > 2) {
            double den = xv[2] * (yu[1] - yu[2]) + xv[1] * (yu[2] - yu[1]) +
                         (xu[1] - xu[2]) * (yv[1] - yv[2]);
            if (den == 0.0) den = den + 0.0000001;
            const double xx = (xu[1] * (xv[2] * (yv[1] - yu[2]) + xv[1] * (yu[2] - yv[2])) +
                               xu[2] * (xv[2] * (yu[1] - yv[1]) + xv[1] * (yv[2] - yu[1]))) /
                              den;
            const double yy = (xv[2] * (yu[1] - yu[2]) * yv[1] + xu[1] * yu[2] * yv[1] -
                               xv[1] * yu[1] * yv[2] - xu[1] * yu[2] * yv[2] +
                               xv[1] * yu[2] * yv[2] + xu[2] * yu[1] * (yv[2] - yv[1])) /
                              den;
            if (xx >= 0.0 && xx <= 1.0 && yy >= 0.0 && yy <= 1.0) {
              switch (n) {
                case 1: x[m] = xx; y[m] = yy; z[m] = 0.0; break;
                case 2: x[m] = xx; y[m] = yy; z[m] = 1.0; break;
                case 3: x[m] = 1.0; y[m] = yy; z[m] = xx; break;
                case 4: x[m] = 0.0; y[m] = yy; z[m] = xx; break;
                case 5: x[m] = xx; y[m] = 1.0; z[m] = yy; break;
                default: x[m] = xx; y[m] = 0.0; z[m] = yy; break;
              }
              m++;
            }
          }
        }
        if (skip) continue;
        if (m > 1) {
          double a = 1.0;
          const int ex = x[1] == x[2] && (x[1] == 0.0 || x[1] == 1.0);
          const int ey = y[1] == y[2] && (y[1] == 0.0 || y[1] == 1.0);
          const int ez = z[1] == z[2] && (z[1] == 0.0 || z[1] == 1.0);
          /* the reference tests y twice where z may have been meant */
          if (ex || ey || ey) {
            a *= 0.5;
            if ((ex && (ey || ey)) || (ey && ez)) a *= 0.5;
          }
          L += a * sqrt((x[1] - x[2]) * (x[1] - x[2]) + (y[1] - y[2]) * (y[1] - y[2]) +
                        (z[1] - z[2]) * (z[1] - z[2]));
        }
      }
  return L * dx;
}


/* ------------------------------------------------------------------------
 * Zero finders (src/io.f90:895-1402), the reference's loops literally. */
typedef struct {
  double* pts;
  long long cap, n;
} zsink;

static void zput(zsink* s, double a, double b, double c) {
  if (s->pts && s->n < s->cap) {
    s->pts[3 * s->n] = a;
    s->pts[3 * s->n + 1] = b;
    s->pts[3 * s->n + 2] = c;
  }
  s->n++;
}

#define ZRE(i, j, k) psi[(((size_t)(k) * ny + (j)) * nx + (i)) * 2]
#define ZIM(i, j, k) psi[(((size_t)(k) * ny + (j)) * nx + (i)) * 2 + 1]

/* get_zeros on one edge direction (d = 0 x, 1 y, 2 z). */
static void zeros_edge_both(const double* psi, int nx, int ny, int nz, const double* x,
                            const double* y, const double* z, int d, zsink* s) {
  for (int k = 1; k <= nz - 2; k++)
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        const int i2 = i + (d == 0), j2 = j + (d == 1), k2 = k + (d == 2);
        const double r = ZRE(i, j, k), m = ZIM(i, j, k);
        const double rn = ZRE(i2, j2, k2), mn = ZIM(i2, j2, k2);
        if ((r == 0.0 && m == 0.0) || (r == 0.0 && m * mn < 0.0) ||
            (m == 0.0 && r * rn < 0.0) || (r * rn < 0.0 && m * mn < 0.0)) {
          const double den = r - rn;
          if (den == 0.0) continue;
          const double* c = d == 0 ? x : (d == 1 ? y : z);
          const int a = d == 0 ? i : (d == 1 ? j : k);
          const double zero = -rn * c[a] / den + r * c[a + 1] / den;
          if (d == 0) zput(s, zero, y[j], z[k]);
          else if (d == 1) zput(s, x[i], zero, z[k]);
          else zput(s, x[i], y[j], zero);
        }
      }
}

/* get_re_im_zeros on one component (comp 0 re, 1 im) and edge direction;
 * the z-edge test has .and. where the others have .or. (kept). */
static void zeros_edge_one(const double* psi, int nx, int ny, int nz, const double* x,
                           const double* y, const double* z, int comp, int d, zsink* s) {
  for (int k = 1; k <= nz - 2; k++)
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        const int i2 = i + (d == 0), j2 = j + (d == 1), k2 = k + (d == 2);
        const double w = comp ? ZIM(i, j, k) : ZRE(i, j, k);
        const double wn = comp ? ZIM(i2, j2, k2) : ZRE(i2, j2, k2);
        const int hit = d == 2 ? (w == 0.0 && w * wn < 0.0) : (w == 0.0 || w * wn < 0.0);
        if (hit) {
          const double den = w - wn;
          if (den == 0.0) continue;
          const double* c = d == 0 ? x : (d == 1 ? y : z);
          const int a = d == 0 ? i : (d == 1 ? j : k);
          const double zero = -wn * c[a] / den + w * c[a + 1] / den;
          if (d == 0) zput(s, zero, y[j], z[k]);
          else if (d == 1) zput(s, x[i], zero, z[k]);
          else zput(s, x[i], y[j], zero);
        }
      }
}

/* get_extra_zeros on one face orientation: f = 0 xy (corners (i,j), (i+1,j),
 * (i+1,j+1), (i,j+1) at k), 1 xz (x then z), 2 yz (z then y, at i). */
static void zeros_face(const double* psi, int nx, int ny, int nz, const double* x,
                       const double* y, const double* z, int f, zsink* s) {
  for (int k = 1; k <= nz - 2; k++)
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        /* corners c0..c3 around the face and the coordinates along its two
           axes: u runs c0 -> c1 (and c3 -> c2), w runs c1 -> c2 (and c0 -> c3) */
        int ci[4], cj[4], ck[4];
        double u0, u1, w0, w1;
        if (f == 0) {
          int a[4][3] = {{i, j, k}, {i + 1, j, k}, {i + 1, j + 1, k}, {i, j + 1, k}};
          for (int q = 0; q < 4; q++) { ci[q] = a[q][0]; cj[q] = a[q][1]; ck[q] = a[q][2]; }
          u0 = x[i]; u1 = x[i + 1]; w0 = y[j]; w1 = y[j + 1];
        } else if (f == 1) {
          int a[4][3] = {{i, j, k}, {i + 1, j, k}, {i + 1, j, k + 1}, {i, j, k + 1}};
          for (int q = 0; q < 4; q++) { ci[q] = a[q][0]; cj[q] = a[q][1]; ck[q] = a[q][2]; }
          u0 = x[i]; u1 = x[i + 1]; w0 = z[k]; w1 = z[k + 1];
        } else {
          int a[4][3] = {{i, j, k}, {i, j, k + 1}, {i, j + 1, k + 1}, {i, j + 1, k}};
          for (int q = 0; q < 4; q++) { ci[q] = a[q][0]; cj[q] = a[q][1]; ck[q] = a[q][2]; }
          u0 = z[k]; u1 = z[k + 1]; w0 = y[j]; w1 = y[j + 1];
        }
        double re[4], im[4];
        for (int q = 0; q < 4; q++) {
          re[q] = ZRE(ci[q], cj[q], ck[q]);
          im[q] = ZIM(ci[q], cj[q], ck[q]);
        }
        for (int pass = 0; pass < 2; pass++) {
          /* pass 0: re crosses c0-c1 and c2-c3, im crosses c1-c2 and c3-c0;
             pass 1: the other way round */
          const double* A = pass ? im : re; /* crosses on the u edges */
          const double* B = pass ? re : im; /* crosses on the w edges */
          if ((A[0] * A[1] < 0.0 && B[0] * B[1] >= 0.0) &&
              (B[1] * B[2] < 0.0 && A[1] * A[2] >= 0.0) &&
              (A[2] * A[3] < 0.0 && B[2] * B[3] >= 0.0) &&
              (B[3] * B[0] < 0.0 && A[3] * A[0] >= 0.0)) {
            double zr[4], den;
            den = A[0] - A[1];
            zr[0] = -A[1] * u0 / den + A[0] * u1 / den;
            den = B[1] - B[2];
            zr[1] = -B[2] * w0 / den + B[1] * w1 / den;
            den = A[2] - A[3];
            zr[2] = -A[3] * u1 / den + A[2] * u0 / den;
            den = B[3] - B[0];
            zr[3] = -B[0] * w1 / den + B[3] * w0 / den;
            const double m1 = (w0 - w1) / (zr[0] - zr[2]);
            const double m2 = (zr[1] - zr[3]) / (u1 - u0);
            const double up = (zr[3] - u0 * m2 - w0 + zr[0] * m1) / (m1 - m2);
            const double wp = up * m1 + w0 - zr[0] * m1;
            if (f == 0) zput(s, up, wp, z[k]);
            else if (f == 1) zput(s, up, y[j], wp);
            else zput(s, x[i], wp, up);
            break;
          }
        }
      }
}

long long ora_zeros(const double* psi, int nx, int ny, int nz, const double* x,
                    const double* y, const double* z, long long* counts, double* points,
                    long long cap) {
  zsink s = {points, cap, 0};
  long long prev = 0;
  for (int sec = 0; sec < 12; sec++) {
    if (sec < 3) zeros_edge_both(psi, nx, ny, nz, x, y, z, sec, &s);
    else if (sec < 6) zeros_face(psi, nx, ny, nz, x, y, z, sec - 3, &s);
    else zeros_edge_one(psi, nx, ny, nz, x, y, z, sec >= 9, (sec - 6) % 3, &s);
    counts[sec] = s.n - prev;
    prev = s.n;
  }
  return s.n;
}
#undef ZRE
#undef ZIM
