// spectral_kernels.cuh -- random-phase initial condition, spectrum and
// condensate reduction, and the spectral filter, on dense transformed fields
// (x fastest, complex of T = float or double).
//
// The transforms themselves are cuFFT's (spectral.cu); these kernels are the
// element-wise and reduction passes around them, each one streaming pass
// over the dense field (HBM-bound).
#pragma once

#include <cstdint>

namespace gpe {
namespace spec {

constexpr int NSHELLS = 7;
constexpr int S_THREADS = 256;
constexpr int S_WARPS = S_THREADS / 32;
// Per-block partial row: [0] sum |a|^2, [1] the temperature denominator,
// [2, 9) shell sums, [9, 16) shell counts, then nf bins of F.
constexpr int HEAD = 16;

// Integer wavenumber square of index i on an axis of n points: i <= (n-1)/2
// + 1 -> i^2, else (n - i)^2 (src/ic.f90:221-238, src/io.f90:652-669).
__host__ __device__ __forceinline__ long long index_k2(int i, int n) {
  return (i <= (n - 1) / 2 + 1) ? (long long)i * i : (long long)(n - i) * (n - i);
}

__device__ __forceinline__ int index_k2i(int i, int n) {
  return (i <= (n - 1) / 2 + 1) ? i * i : (n - i) * (n - i);
}

// SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): the finaliser of state seed + (q+1) G, top 53
// bits as a double in [0, 1).
__host__ __device__ __forceinline__ double splitmix_u01(uint64_t seed, uint64_t q) {
  uint64_t z = seed + (q + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * 0x1.0p-53;
}

// random_phase (src/ic.f90:220-248): amp e^{2 pi i phi} inside |k|^2 <= kc2,
// zero outside.  amp already carries the transform's 1/sqrt(N).
template <typename T>
__global__ void random_phase_kernel(T* __restrict__ a, int nx, int ny, int nz, double amp,
                                    double kc2, uint64_t seed) {
  const size_t n = (size_t)nx * ny * nz;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const size_t r = q / nx;
    const int j = (int)(r % ny);
    const int k = (int)(r / ny);
    const long long k2 = index_k2(i, nx) + index_k2(j, ny) + index_k2(k, nz);
    double re = 0.0, im = 0.0;
    if ((double)k2 <= kc2) {
      double s, c;
      sincospi(2.0 * splitmix_u01(seed, q), &s, &c);
      re = amp * c;
      im = amp * s;
    }
    a[2 * q] = (T)re;
    a[2 * q + 1] = (T)im;
  }
}

// filtered_surface (src/io.f90:549-572): a(k) *= max(1 - m k^2 / kc^2, 0),
// times `scale` (the two transforms' 1/N).
template <typename T>
__global__ void filter_kernel(T* __restrict__ a, int nx, int ny, int nz, double m,
                              double kc_sq, double scale) {
  const size_t n = (size_t)nx * ny * nz;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const size_t r = q / nx;
    const int j = (int)(r % ny);
    const int k = (int)(r / ny);
    const long long k2 = index_k2(i, nx) + index_k2(j, ny) + index_k2(k, nz);
    const double f = fmax(1.0 - (m * (double)k2) / kc_sq, 0.0) * scale;
    a[2 * q] = (T)((double)a[2 * q] * f);
    a[2 * q + 1] = (T)((double)a[2 * q + 1] * f);
  }
}

// Smallest b with b^2 >= k2 (k2 < 2^31): the first kk of F(kk) that holds
// the mode, as the reference's sqrt(real(k2)) <= kk test (src/io.f90:673-677).
// The approximate FP32 root is within one of the true root for every k2 here;
// integer checks make it exact.
__device__ __forceinline__ int ceil_sqrt(int k2) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"((float)k2));
  int b = (int)r;
  if (b * b > k2) b--;
  if ((b + 1) * (b + 1) <= k2) b++;
  return b + (b * b < k2 ? 1 : 0);
}

// Shell thresholds of spectrum (src/io.f90:679-687), m-1 <= |log2(|k| /
// (2 pi))| < m, in integer k2: with T = 4 pi^2, shell s >= 0 holds
// up[s] <= k2 < up[s+1] (up[s] = ceil(T 4^s)) on the |k| >= 2 pi side and
// dn[s+1] < k2 <= dn[s] (dn[s] = floor(T 4^-s)) below it.  No T 4^s with
// |s| <= 7 lies within 1e-9 of an integer, so these integer tests and the
// reference's logarithms agree for every k2.
struct Shells {
  int up[NSHELLS + 1];
  int dn[NSHELLS + 1];
};

// Shell index of k2 >= 1 (NSHELLS for none) as 0..7 on the |k| < 2 pi side
// and 8..15 on the other, so equal codes mean one interval of k2.
__device__ __forceinline__ int shell_code(int k2, const int* up, const int* dn) {
  int s = 0;
  if (k2 >= up[0]) {
#pragma unroll
    for (int q = 1; q <= NSHELLS; q++) s += (k2 >= up[q]) ? 1 : 0;
    return 8 + s;
  }
#pragma unroll
  for (int q = 1; q <= NSHELLS; q++) s += (k2 <= dn[q]) ? 1 : 0;
  return s;
}

// 1/d by Newton-Raphson iteration r <- r + r (1 - d r) from the hardware's
// approximate reciprocal; three steps take any start within 2^-10 to full
// double precision.  d is a normal nonzero double wherever the result is
// used (d = 0 is discarded by the caller).
__device__ __forceinline__ double recip_newton(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
#pragma unroll
  for (int q = 0; q < 3; q++) r = fma(r, fma(-d, r, 1.0), r);
  return r;
}

struct SpecArgs {
  int nx, ny, nz, nf;
  double inv_n;     // |buffer|^2 -> |a|^2 (the backward transform's 1/N)
  double inv_v;     // 1 / (nx ny nz)
  Shells shells;
  const double* ax;  // finite-difference symbols per axis (src/io.f90:354-361)
  const double* ay;
  const double* az;
  double* partials;  // [gridDim.x][HEAD + nf]
};

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

constexpr int S_NONE = 0x7fffffff;

// One pass over the unnormalised backward transform: Parseval mass, the
// temperature denominator sum (k2+rho0)/(k2^2+2 rho0 k2) over the
// finite-difference symbol (src/io.f90:347-366), shell sums and counts, and
// the F bins.  Warps own whole x-rows and walk each row in its two halves
// (i below (nx-1)/2+1, then the rest), along each of which |k| and so the F
// bin is monotone in i.  A lane takes S_E consecutive sites (32 S_E about
// half a row, at most 256 sites per pass): equal-bin runs
// inside the lane are summed in registers, a run strictly inside the lane is
// the only one with its bin and goes straight to the warp's bin array, and
// the runs at lane edges are joined across lanes by one segmented warp scan.
// Every bin then has one writer per instruction, so the bins need no
// atomics and the sums come out the same bit for bit on every run.  Shells
// change rarely along a row: a lane whose first and last site share a shell
// (and side) adds its sum once.
template <typename T, int S_E>
__global__ void __launch_bounds__(S_THREADS, S_E <= 4 ? 4 : 3) spectrum_kernel(
    const T* __restrict__ a, SpecArgs p) {
  extern __shared__ double smem_f[];            // [S_WARPS][nf]
  __shared__ double eta_s[S_WARPS][32][NSHELLS];  // per lane
  __shared__ int cnt_s[S_WARPS][32][NSHELLS];
  __shared__ double red[S_WARPS][2];
  using V2 = typename Vec2<T>::type;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nx = p.nx, nf = p.nf;
  double* fw = smem_f + (size_t)warp * nf;
  for (int b = threadIdx.x; b < S_WARPS * nf; b += S_THREADS) smem_f[b] = 0.0;
#pragma unroll
  for (int m = 0; m < NSHELLS; m++) {
    eta_s[warp][lane][m] = 0.0;
    cnt_s[warp][lane][m] = 0;
  }
  __syncthreads();

  __shared__ int sh_up[NSHELLS + 1], sh_dn[NSHELLS + 1];
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q <= NSHELLS; q++) {
      sh_up[q] = p.shells.up[q];
      sh_dn[q] = p.shells.dn[q];
    }
  }
  __syncthreads();

  // sums are of |buffer|^2; the finaliser applies the transform's 1/N
  const V2 a0 = reinterpret_cast<const V2*>(a)[0];
  const double rho0 = (((double)a0.x * a0.x + (double)a0.y * a0.y) * p.inv_n) * p.inv_v;
  const double two_rho0 = 2.0 * rho0;
  const double m12 = -(1.0 / 12.0);
  double mass = 0.0, tot = 0.0;
  // |k| rises along i < h and falls from h on (h = (nx-1)/2 + 1 is the peak)
  const int h = min((nx - 1) / 2 + 1, nx);
  const long long nrows = (long long)p.ny * p.nz;
  for (long long row = (long long)blockIdx.x * S_WARPS + warp; row < nrows;
       row += (long long)gridDim.x * S_WARPS) {
    const int j = (int)(row % p.ny), k = (int)(row / p.ny);
    const int c2 = index_k2i(j, p.ny) + index_k2i(k, p.nz);
    const double ayz = __ldg(p.ay + j);
    const double azk = __ldg(p.az + k);
    const V2* arow = reinterpret_cast<const V2*>(a) + (size_t)row * nx;
    for (int half = 0; half < 2; half++) {
      const int start = half ? h : 0, end = half ? nx - 1 : h - 1;
      for (int base = start; base <= end; base += 32 * S_E) {
        const int i0 = base + lane * S_E;
        V2 v[S_E];
#pragma unroll
        for (int e = 0; e < S_E; e++) {
          v[e].x = v[e].y = (T)0;
          if (i0 + e <= end) v[e] = arow[i0 + e];
        }
        // shells: k2 is monotone along the lane's sites, so equal shell codes
        // at its two ends put every site in that shell
        const int ilast = min(i0 + S_E - 1, end);
        const int k2f = index_k2i(i0, nx) + c2, k2l = index_k2i(ilast, nx) + c2;
        const bool any = i0 <= end;
        const int sf = (any && k2f > 0) ? shell_code(k2f, sh_up, sh_dn) : -1;
        const int sl = (any && k2l > 0) ? shell_code(k2l, sh_up, sh_dn) : -2;
        const bool one_shell = sf == sl;
        double lane_sum = 0.0;
        int lane_cnt = 0;
        // F runs: current (cb, cv), first (fb, fv)
        int cb = S_NONE, fb = S_NONE;
        double cv = 0.0, fv = 0.0;
        bool split = false;
#pragma unroll
        for (int e = 0; e < S_E; e++) {
          const int i = i0 + e;
          const bool valid = i <= end;
          const double pw = (double)v[e].x * v[e].x + (double)v[e].y * v[e].y;
          mass += pw;  // zero past the end
          const int ic = min(i, nx - 1);
          const double k2p = m12 * ((__ldg(p.ax + ic) + ayz) + azk);
          const double term = (k2p + rho0) * recip_newton(k2p * (k2p + two_rho0));
          tot += (valid && k2p != 0.0) ? term : 0.0;
          const int k2 = index_k2i(ic, nx) + c2;
          const bool live = valid && k2 > 0;
          if (one_shell) {
            lane_sum += live ? pw : 0.0;
            lane_cnt += live ? 1 : 0;
          } else if (live) {
            const int s = shell_code(k2, sh_up, sh_dn) & 7;
            if (s < NSHELLS) {
              eta_s[warp][lane][s] += pw;
              cnt_s[warp][lane][s]++;
            }
          }
          const int bb = ceil_sqrt(k2);
          const int b = (live && bb <= nf) ? bb : S_NONE;
          const double val = (b != S_NONE) ? pw : 0.0;
          if (e == 0) {
            cb = b;
            cv = val;
          } else {
            const bool same = b == cb;
            const bool first = !same && !split;
            const bool inner = !same && split && cb != S_NONE;
            if (inner) fw[cb - 1] += cv;  // a run inside the lane: no other lane has this bin
            fb = first ? cb : fb;
            fv = first ? cv : fv;
            split = split || !same;
            cv = same ? cv + val : val;
            cb = b;
          }
        }
        if (one_shell && sf >= 0 && (sf & 7) < NSHELLS && lane_cnt > 0) {
          eta_s[warp][lane][sf & 7] += lane_sum;
          cnt_s[warp][lane][sf & 7] += lane_cnt;
        }
        const int lb = cb;
        const double lv = cv;
        if (!split) {
          fb = lb;
          fv = 0.0;
        }
        // join edge runs across lanes: trailing-run chains by a segmented scan
        int prev_lb = __shfl_up_sync(0xffffffffu, lb, 1);
        if (lane == 0) prev_lb = -1;
        const bool cont = (fb != S_NONE) && (fb == prev_lb);
        double co = lv;
        int flag = (split || !cont) ? 1 : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const double o = __shfl_up_sync(0xffffffffu, co, d);
          const int of = __shfl_up_sync(0xffffffffu, flag, d);
          if (lane >= d && !flag) {
            co += o;
            flag = of;
          }
        }
        const double carry_in = __shfl_up_sync(0xffffffffu, co, 1);
        const int next_cont = __shfl_down_sync(0xffffffffu, cont ? 1 : 0, 1);
        if (split && fb != S_NONE) fw[fb - 1] += fv + (cont ? carry_in : 0.0);
        if ((lane == 31 || !next_cont) && lb != S_NONE) fw[lb - 1] += co;
      }
    }
  }
  // block partial row in a fixed order
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    mass += __shfl_down_sync(0xffffffffu, mass, d);
    tot += __shfl_down_sync(0xffffffffu, tot, d);
  }
  if (lane == 0) {
    red[warp][0] = mass;
    red[warp][1] = tot;
  }
  __syncthreads();
  double* out = p.partials + (size_t)blockIdx.x * (HEAD + nf);
  if (threadIdx.x < 2) {
    double x = 0.0;
    for (int w = 0; w < S_WARPS; w++) x += red[w][threadIdx.x];
    out[threadIdx.x] = x;
  } else if (threadIdx.x < 2 + NSHELLS) {
    const int m = threadIdx.x - 2;
    double x = 0.0;
    for (int w = 0; w < S_WARPS; w++)
      for (int l = 0; l < 32; l++) x += eta_s[w][l][m];
    out[threadIdx.x] = x;
  } else if (threadIdx.x < 2 + 2 * NSHELLS) {
    const int m = threadIdx.x - 2 - NSHELLS;
    long long x = 0;
    for (int w = 0; w < S_WARPS; w++)
      for (int l = 0; l < 32; l++) x += cnt_s[w][l][m];
    out[threadIdx.x] = (double)x;
  }
  for (int b = threadIdx.x; b < nf; b += S_THREADS) {
    double x = 0.0;
    for (int w = 0; w < S_WARPS; w++) x += smem_f[(size_t)w * nf + b];
    out[HEAD + b] = x;
  }
}

struct SpecFinal {
  int nblk, nf;
  double inv_n, volume_v;  // V = nx ny nz
  double cell;             // dx dy dz
  double box8;             // 8 xr yr zr
  double* out;  // [0,7) row, [7,14) eta, [14,21) nharm, [21, 21+nf) F
};

constexpr int F_FIN_THREADS = 1024;

// Sums the block partials (each column by one warp, lanes over blocks, then
// a fixed shuffle tree), then the mass.dat row (src/io.f90:369-382), eta =
// shell sum / count (:701-704) and F(kk) as the running sum of the bins
// (:673-677).
template <typename T>
__global__ void __launch_bounds__(F_FIN_THREADS) spectrum_finalize_kernel(
    const T* __restrict__ a, const double* __restrict__ partials, SpecFinal f) {
  extern __shared__ double col[];  // [HEAD + nf]
  using V2 = typename Vec2<T>::type;
  const int ncol = HEAD + f.nf;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = warp; c < ncol; c += F_FIN_THREADS / 32) {
    double x = 0.0;
    for (int b = lane; b < f.nblk; b += 32) x += partials[(size_t)b * ncol + c];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
    if (lane == 0) col[c] = x;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const V2 a0 = reinterpret_cast<const V2*>(a)[0];
  const double a0r = (double)a0.x, a0i = (double)a0.y;
  const double V = f.volume_v;
  const double n0 = (a0r * a0r + a0i * a0i) * f.inv_n;
  const double M = (col[0] * f.inv_n) * f.cell;
  const double tot = col[1];
  const double temp = (M - n0) / tot;
  const double E0 = (1.0 / (2.0 * V)) * (M * M + (M - n0) * (M - n0));
  const double H = E0 + temp * (V - 1.0);
  const double temp2 = ((M / f.box8) - (n0 / V)) / tot;
  double* o = f.out;
  o[0] = M / f.box8;
  o[1] = n0 / V;
  o[2] = M;
  o[3] = n0;
  o[4] = temp;
  o[5] = temp2;
  o[6] = H / V;
  for (int m = 0; m < NSHELLS; m++) {
    const double s = col[2 + m] * f.inv_n, n = col[2 + NSHELLS + m];
    o[7 + m] = (s == 0.0) ? 0.0 : s / n;
    o[14 + m] = n;
  }
  double run = 0.0;
  for (int b = 0; b < f.nf; b++) {
    run += col[HEAD + b];
    o[21 + b] = run * f.inv_n;
  }
}

}  // namespace spec
}  // namespace gpe
