// aux_kernels.cuh -- state transfer, scaling and reduction kernels.
#pragma once

#include "device_utils.cuh"

namespace gpe {

struct Geom {
  int nx, ny, nz;  // interior
  int Nx, Ny;      // padded pitches
  int bcs;
  int zg_lo, zg_hi;  // fill z ghosts below / above locally
};

__device__ __forceinline__ size_t padded_index(const Geom& g, int i, int j,
                                               int k) {
  return ((size_t)(k + 2) * g.Ny + (size_t)(j + 2)) * g.Nx + (size_t)(i + 2);
}

// Dense interior array (any complex type TI) -> padded field of TS, with the
// boundary ghosts filled (the caller's halo exchange, src/gpe.f90:165-174).
template <typename TS, typename TI>
__global__ void unpack_kernel(const TI* __restrict__ src, TS* __restrict__ dst,
                              Geom g) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx);
    const size_t r = q / g.nx;
    const int j = (int)(r % g.ny);
    const int k = (int)(r / g.ny);
    const TS vr = (TS)src[2 * q], vi = (TS)src[2 * q + 1];
    st_one<TS>(dst + 2 * padded_index(g, i, j, k), vr, vi);
    int a, b;
    ghost_targets(i, g.nx, g.bcs, a, b);
    if (a != NO_GHOST) st_one<TS>(dst + 2 * padded_index(g, a, j, k), vr, vi);
    if (b != NO_GHOST) st_one<TS>(dst + 2 * padded_index(g, b, j, k), vr, vi);
    ghost_targets(j, g.ny, g.bcs, a, b);
    if (a != NO_GHOST) st_one<TS>(dst + 2 * padded_index(g, i, a, k), vr, vi);
    if (b != NO_GHOST) st_one<TS>(dst + 2 * padded_index(g, i, b, k), vr, vi);
    ghost_targets(k, g.nz, g.bcs, a, b);
    if (a != NO_GHOST && ((a < 0) ? g.zg_lo : g.zg_hi))
      st_one<TS>(dst + 2 * padded_index(g, i, j, a), vr, vi);
    if (b != NO_GHOST && ((b < 0) ? g.zg_lo : g.zg_hi))
      st_one<TS>(dst + 2 * padded_index(g, i, j, b), vr, vi);
  }
}

// Padded field -> dense interior array of TO.
template <typename TS, typename TO>
__global__ void pack_kernel(const TS* __restrict__ src, TO* __restrict__ dst,
                            Geom g) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx);
    const size_t r = q / g.nx;
    const int j = (int)(r % g.ny);
    const int k = (int)(r / g.ny);
    const size_t s = padded_index(g, i, j, k);
    dst[2 * q] = (TO)src[2 * s];
    dst[2 * q + 1] = (TO)src[2 * s + 1];
  }
}

// renormalise (src/variables.f90:698-709): f = (sqrt(nn) f) / sqrt(norm)
// over the whole padded buffer, ghosts included (they stay exact copies).
template <typename TS>
__global__ void scale_kernel(TS* __restrict__ f, size_t nscalars, double snn,
                             double sn) {
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nscalars;
       q += (size_t)gridDim.x * blockDim.x) {
    f[q] = (TS)(((double)f[q] * snn) / sn);
  }
}

// The same rescaling with the factor sqrt(target / current) read on the
// device (both norms left in device memory by earlier reductions).
template <typename TS>
__global__ void rescale_to_kernel(TS* __restrict__ f, size_t nscalars,
                                  const double* __restrict__ target,
                                  const double* __restrict__ current) {
  const double s = sqrt(target[0] / current[0]);
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nscalars;
       q += (size_t)gridDim.x * blockDim.x) {
    f[q] = (TS)((double)f[q] * s);
  }
}

// Weighted |psi|^2 per CTA into partials[2*blk] (get_norm without a stencil).
template <typename TS>
__global__ void norm_kernel(const TS* __restrict__ f, Geom g,
                            const double* __restrict__ wx,
                            const double* __restrict__ wy,
                            const double* __restrict__ wz,
                            double* __restrict__ partials) {
  __shared__ double s[32];
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  double acc = 0.0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx);
    const size_t r = q / g.nx;
    const int j = (int)(r % g.ny);
    const int k = (int)(r / g.ny);
    const size_t pi = padded_index(g, i, j, k);
    const double a = (double)f[2 * pi], b = (double)f[2 * pi + 1];
    acc += (wx[i] * wy[j]) * wz[k] * (a * a + b * b);
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s[w];
    partials[2 * blockIdx.x] = t;
    partials[2 * blockIdx.x + 1] = 0.0;
  }
}

// Fixed-order reduction of partials[2*b + slot], b < nblk, by one CTA of
// 1024 threads.  op 0 = sum, 1 = max.  out[0] = result * scale; when
// `series` is non-null also series[*counter] = out[0] and ++*counter.
// Fixed-order reduction of slot `slot` of the per-CTA partials by one block
// (sum, or max for op 1); the result is s[0] for every thread on return.
__device__ __forceinline__ void reduce_partials(const double* __restrict__ partials, int nblk,
                                                int slot, int op, double* s) {
  double a = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    const double v = partials[2 * (size_t)b + slot];
    a = op ? fmax(a, v) : a + v;
  }
  s[threadIdx.x] = a;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      const double v = s[threadIdx.x + w];
      s[threadIdx.x] = op ? fmax(s[threadIdx.x], v) : s[threadIdx.x] + v;
    }
    __syncthreads();
  }
}

__global__ void finalize_kernel(const double* __restrict__ partials, int nblk,
                                int slot, int op, double scale,
                                double* __restrict__ out,
                                double* __restrict__ series,
                                int* __restrict__ counter) {
  __shared__ double s[1024];
  reduce_partials(partials, nblk, slot, op, s);
  if (threadIdx.x == 0) {
    const double r = s[0] * scale;
    out[0] = r;
    if (series) {
      series[*counter] = r;
      *counter = *counter + 1;
    }
  }
}

// ---------------------------------------------------------------------------
// rkqs step control on the device (src/solve.f90:158-244).  A step is: begin
// (first attempt's dt), then attempts of the six Cash-Karp stages, each
// followed by rk45_control_kernel, until one is accepted.  The stage kernels
// read dt from `dt_r, dt_i, dt0_r, dt0_i` (contiguous, in this order).

struct DevTime {
  double dt_r, dt_i, dt0_r, dt0_i;  // this attempt's dt, the step's first dt
  double t, im_t;
  double errmax, did_r, did_i;       // last accepted attempt
  double errcon;                     // (5 / safety)^(1 / dt_increase)
  int attempts, underflow, halt, steps;  // halt: 0, or the GPE status code
  int real_time, pad;
};

// Sets the while node's condition (when it is one) and starts a step.
__global__ void rk45_begin_kernel(DevTime* T, cudaGraphConditionalHandle h, int use_cond) {
  if (threadIdx.x != 0) return;
  T->attempts = 0;
  T->dt0_r = T->dt_r;
  T->dt0_i = T->dt_i;
  if (use_cond) cudaGraphSetConditional(h, T->halt ? 0u : 1u);
}

// After an attempt whose error maximum (over all sites, already reduced
// across slabs) is scal[3] and whose trial-state norm is scal[0]: accept and
// advance t, dt (recording the step in the series), or shrink dt and retry.
// The arithmetic is the reference's: errmax <= 1 accepts; a rejected dt
// shrinks to max(safety dt errmax^dt_decrease, dt / 10) along the time
// direction; an accepted one grows to safety dt errmax^dt_increase, or 5 dt
// when errmax <= errcon; t advances by the accepted dt and im_t by the new
// |Im dt|.
__device__ void rk45_control(DevTime* T, const double* __restrict__ scal,
                             double* __restrict__ s_norm, double* __restrict__ s_dt,
                             int* __restrict__ s_att, int cap, cudaGraphConditionalHandle h,
                             int use_cond) {
  const double safety = 0.9, dt_decrease = -0.25, dt_increase = -0.20;
  if (T->halt) {
    if (use_cond) cudaGraphSetConditional(h, 0u);
    return;
  }
  const double errmax = scal[3];
  T->attempts += 1;
  T->errmax = errmax;
  bool done = false;
  // the error maximum skips NaN sites (fmax, as maxval does), so a state
  // that went non-finite shows in the fused norm of the trial state
  if (!isfinite(errmax) || !isfinite(scal[0])) {
    T->halt = 5;  // GPE_ERR_NAN
    done = true;
  } else if (errmax <= 1.0) {
    const double dr = T->dt_r, di = T->dt_i;
    double nr, ni;
    if (errmax > T->errcon) {
      const double f = pow(errmax, dt_increase);
      nr = (safety * dr) * f;
      ni = (safety * di) * f;
    } else {
      nr = 5.0 * dr;
      ni = 5.0 * di;
    }
    T->t = T->t + dr;
    T->did_r = dr;
    T->did_i = di;
    T->dt_r = nr;
    T->dt_i = ni;
    T->im_t = T->im_t + fabs(ni);
    const int k = T->steps;
    if (k < cap) {
      if (s_norm) s_norm[k] = scal[0];
      if (s_dt) s_dt[k] = dr;
      if (s_att) s_att[k] = T->attempts;
    }
    T->steps = k + 1;
    done = true;
  } else {
    const double dr = T->dt_r, di = T->dt_i;
    const double f = pow(errmax, dt_decrease);
    const double tr = (safety * dr) * f, ti = (safety * di) * f;
    const double mag = fmax(hypot(tr, ti), 0.1 * hypot(dr, di));
    if (T->real_time) {
      T->dt_r = mag;
      T->dt_i = 0.0;
      if (T->t + mag == T->t) T->underflow = 1;
    } else {
      T->dt_r = 0.0;
      T->dt_i = -mag;
    }
    if (T->attempts > 10000) {
      T->halt = 8;  // GPE_ERR_UNDERFLOW
      done = true;
    }
  }
  if (use_cond) cudaGraphSetConditional(h, done ? 0u : 1u);
}

__global__ void rk45_control_kernel(DevTime* T, const double* __restrict__ scal,
                                    double* __restrict__ s_norm, double* __restrict__ s_dt,
                                    int* __restrict__ s_att, int cap,
                                    cudaGraphConditionalHandle h, int use_cond) {
  if (threadIdx.x == 0) rk45_control(T, scal, s_norm, s_dt, s_att, cap, h, use_cond);
}

// A context with no neighbours: the attempt's two reductions (error maximum
// into scal[3], trial-state norm into scal[0], each as finalize_kernel forms
// it) and the step control in one launch of 1024 threads.
__global__ void rk45_reduce_control_kernel(const double* __restrict__ partials, int nblk,
                                           double err_scale, double norm_scale,
                                           double* __restrict__ scal, DevTime* T,
                                           double* __restrict__ s_norm,
                                           double* __restrict__ s_dt, int* __restrict__ s_att,
                                           int cap, cudaGraphConditionalHandle h,
                                           int use_cond) {
  __shared__ double s[1024];
  reduce_partials(partials, nblk, 1, 1, s);
  if (threadIdx.x == 0) scal[3] = s[0] * err_scale;
  __syncthreads();
  reduce_partials(partials, nblk, 0, 0, s);
  if (threadIdx.x == 0) {
    scal[0] = s[0] * norm_scale;
    rk45_control(T, scal, s_norm, s_dt, s_att, cap, h, use_cond);
  }
}

// Slab group: combine d_scal[idx] of n members in member order (sum, or max
// for op 1) and write the result back to every member.
__global__ void combine_scalars_kernel(double* const* __restrict__ scal, int n, int idx,
                                       int op) {
  if (threadIdx.x != 0) return;
  double a = scal[0][idx];
  for (int m = 1; m < n; m++) {
    const double v = scal[m][idx];
    a = op ? fmax(a, v) : a + v;
  }
  for (int m = 0; m < n; m++) scal[m][idx] = a;
}

// Batched ensembles: one CTA per run sums slot 0 of the partials of every
// work item of that run (fixed item order), times scale[r]; out[r] gets the
// value and, when series is non-null, series[r * cap + *counter] too.
__global__ void batch_finalize_kernel(const double* __restrict__ partials,
                                      const int* __restrict__ item_run, int nitems,
                                      const double* __restrict__ scale,
                                      double* __restrict__ out,
                                      double* __restrict__ series, int cap,
                                      const int* __restrict__ counter) {
  __shared__ double s[256];
  const int r = blockIdx.x;
  double a = 0.0;
  for (int i = threadIdx.x; i < nitems; i += blockDim.x)
    if (item_run[i] == r) a += partials[2 * (size_t)i];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double v = s[0] * scale[r];
    out[r] = v;
    if (series) series[(size_t)r * cap + *counter] = v;
  }
}

__global__ void bump_counter_kernel(int* counter) { *counter = *counter + 1; }

// Failure-detection probe: waits, bounded by limit_ns, on an mbarrier phase
// that nothing completes, then records the timeout in *status exactly as
// the stage kernels do.
__global__ void wait_probe_kernel(unsigned long long limit_ns, int* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0, limit_ns)) atomicExch(status, 1);
}

// mass (src/variables.f90:590-610) and momentum (:615-694) in one pass:
// per block, [4] partials = { sum |psi|^2, and for d = x, y, z the weighted
// sum of (Re psi - 1) Im(d conj psi) - Im psi Re(d psi) }.  First
// derivatives use the face ghosts: c1 (f+1 - f-1) + c2 (f+2 - f-2).
template <typename TS>
__global__ void diag_kernel(const TS* __restrict__ f, Geom g, double c1x, double c2x,
                            double c1y, double c2y, double c1z, double c2z,
                            const double* __restrict__ wx, const double* __restrict__ wy,
                            const double* __restrict__ wz, double* __restrict__ partials) {
  __shared__ double red[4][32];
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  const size_t sx = 1, sy = (size_t)g.Nx, sz = (size_t)g.Nx * g.Ny;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx);
    const size_t r = q / g.nx;
    const int j = (int)(r % g.ny);
    const int k = (int)(r / g.ny);
    const size_t pi = padded_index(g, i, j, k);
    const double re = (double)f[2 * pi], im = (double)f[2 * pi + 1];
    acc[0] += re * re + im * im;
    const size_t st[3] = {sx, sy, sz};
    const double c1[3] = {c1x, c1y, c1z}, c2[3] = {c2x, c2y, c2z};
    const double w = (wx[i] * wy[j]) * wz[k];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const size_t p1 = pi + st[a], m1 = pi - st[a], p2 = pi + 2 * st[a], m2 = pi - 2 * st[a];
      double dr = c1[a] * ((double)f[2 * p1] - (double)f[2 * m1]);
      double di = c1[a] * ((double)f[2 * p1 + 1] - (double)f[2 * m1 + 1]);
      if (c2[a] != 0.0) {
        dr += c2[a] * ((double)f[2 * p2] - (double)f[2 * m2]);
        di += c2[a] * ((double)f[2 * p2 + 1] - (double)f[2 * m2 + 1]);
      }
      // Im(d conj psi) = -Im(d psi)
      acc[1 + a] += w * (-(re - 1.0) * di - im * dr);
    }
  }
#pragma unroll
  for (int v = 0; v < 4; v++) {
    const double t = warp_sum(acc[v]);
    if ((threadIdx.x & 31) == 0) red[v][threadIdx.x >> 5] = t;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[threadIdx.x][w];
    partials[4 * (size_t)blockIdx.x + threadIdx.x] = t;
  }
}

// [nblk][4] partials -> out[0..3] * scale, fixed order (one CTA of 256).
__global__ void diag_finalize_kernel(const double* __restrict__ partials, int nblk, double scale,
                                     double* __restrict__ out) {
  __shared__ double s[4][256];
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
    for (int v = 0; v < 4; v++) a[v] += partials[4 * (size_t)b + v];
#pragma unroll
  for (int v = 0; v < 4; v++) s[v][threadIdx.x] = a[v];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int v = 0; v < 4; v++) s[v][threadIdx.x] += s[v][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = s[threadIdx.x][0] * scale;
}

}  // namespace gpe
