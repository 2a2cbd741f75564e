// spectral.cu -- random-phase initial condition, condensate / spectrum
// diagnostics and the filtered field on cuFFT (include/gpe_gpu.h).
//
// Each call works on the context's dense staging buffer (nx ny nz elements
// of 16 bytes; complex64 fields use the first half): the backward transform
// reads psi's interior straight from the padded field into it (a cuFFT plan
// with the padded pitches), and the reduction or filter runs there; the
// initial condition is built there, transformed in place and loaded into
// psi with its ghosts.  libcufft is opened at first use so that the
// library still loads where it is absent.
#include <cuda_runtime.h>
#include <cufft.h>
#include <dlfcn.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "gpe_gpu.h"
#include "internal.h"
#include "spectral_kernels.cuh"

using namespace gpe;
using namespace gpe::spec;

namespace {

struct CufftApi {
  bool ok = false;
  std::string why;
  cufftResult (*Plan3d)(cufftHandle*, int, int, int, cufftType) = nullptr;
  cufftResult (*PlanMany)(cufftHandle*, int, int*, int*, int, int, int*, int, int, cufftType,
                          int) = nullptr;
  cufftResult (*SetStream)(cufftHandle, cudaStream_t) = nullptr;
  cufftResult (*ExecZ2Z)(cufftHandle, cufftDoubleComplex*, cufftDoubleComplex*, int) = nullptr;
  cufftResult (*ExecC2C)(cufftHandle, cufftComplex*, cufftComplex*, int) = nullptr;
  cufftResult (*Destroy)(cufftHandle) = nullptr;
};

CufftApi g_fft;
std::once_flag g_fft_once;

void load_cufft() {
  void* h = dlopen("libcufft.so.11", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libcufft.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h) {
    g_fft.why = std::string("libcufft.so.11 not found: ") + dlerror();
    return;
  }
#define GPE_FFT_SYM(field, name)                                            \
  g_fft.field = reinterpret_cast<decltype(g_fft.field)>(dlsym(h, name));    \
  if (!g_fft.field) {                                                       \
    g_fft.why = std::string("libcufft lacks ") + name;                      \
    return;                                                                 \
  }
  GPE_FFT_SYM(Plan3d, "cufftPlan3d")
  GPE_FFT_SYM(PlanMany, "cufftPlanMany")
  GPE_FFT_SYM(SetStream, "cufftSetStream")
  GPE_FFT_SYM(ExecZ2Z, "cufftExecZ2Z")
  GPE_FFT_SYM(ExecC2C, "cufftExecC2C")
  GPE_FFT_SYM(Destroy, "cufftDestroy")
#undef GPE_FFT_SYM
  g_fft.ok = true;
}

struct Spectral : Extension {
  cufftHandle plan = 0;      // in place on the dense staging buffer
  cufftHandle plan_psi = 0;  // padded psi interior -> dense staging buffer
  bool has_plan = false, has_plan_psi = false;
  double* d_axes = nullptr;      // ax[nx], ay[ny], az[nz]
  double* d_partials = nullptr;  // [nblk][HEAD + nf]
  double* d_out = nullptr;       // [21 + nf]
  int nblk = 0, nf = 0;
  ~Spectral() override {
    if (has_plan && g_fft.ok) g_fft.Destroy(plan);
    if (has_plan_psi && g_fft.ok) g_fft.Destroy(plan_psi);
    cudaFree(d_axes);
    cudaFree(d_partials);
    cudaFree(d_out);
  }
};

#define SP_CU(c, call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return gpe_internal_fail((c), GPE_ERR_CUDA,                                       \
                               std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

#define SP_FFT(c, call)                                                                 \
  do {                                                                                  \
    cufftResult r_ = (call);                                                            \
    if (r_ != CUFFT_SUCCESS)                                                            \
      return gpe_internal_fail((c), GPE_ERR_CUDA,                                       \
                               std::string(#call) + ": cufftResult " + std::to_string((int)r_)); \
  } while (0)

int elementwise_grid(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b < 148 * 16 ? b : 148 * 16);
}

// Finite-difference symbol of one axis as condensed_particles evaluates it
// (src/io.f90:333-361): k = -pi + i dk with dk = 2 pi / (nx - 1) on every
// axis, term (-2 cos(2 k h) + 32 cos(k h) - 30) / h^2.
void axis_terms(int n, double h, double dk, double* out) {
  const double kc = M_PI;
  for (int i = 0; i < n; i++) {
    const double k = -kc + (double)i * dk;
    out[i] = (-2.0 * std::cos(2.0 * k * h) + 32.0 * std::cos(k * h) - 30.0) / (h * h);
  }
}

// View, extension (plan, tables, partials) and the device made current.
int prepare(gpe_ctx* c, FieldView* v, Spectral** out) {
  if (!c || gpe_internal_field_view(c, v)) return GPE_ERR_INVALID;
  SP_CU(c, cudaSetDevice(v->dev));
  if (!v->single_domain)
    return gpe_internal_fail(c, GPE_ERR_INVALID,
                             "spectral calls need a single-domain context (the whole grid)");
  std::call_once(g_fft_once, load_cufft);
  if (!g_fft.ok) return gpe_internal_fail(c, GPE_ERR_CUDA, g_fft.why);
  auto& slot = gpe_internal_extension(c, GPE_EXT_SPECTRAL);
  if (!slot) slot.reset(new Spectral());
  Spectral* s = static_cast<Spectral*>(slot.get());
  if (!s->has_plan) {
    SP_FFT(c, g_fft.Plan3d(&s->plan, v->nz, v->ny, v->nx, v->es == 16 ? CUFFT_Z2Z : CUFFT_C2C));
    s->has_plan = true;
    SP_FFT(c, g_fft.SetStream(s->plan, v->stream));
  }
  if (!s->has_plan_psi) {
    // reads the interior of the padded field (row pitch Nx, plane pitch Nx Ny)
    int n[3] = {v->nz, v->ny, v->nx};
    int inembed[3] = {v->nz + 4, v->Ny, v->Nx};
    int onembed[3] = {v->nz, v->ny, v->nx};
    SP_FFT(c, g_fft.PlanMany(&s->plan_psi, 3, n, inembed, 1, (v->nz + 4) * v->Ny * v->Nx, onembed,
                             1, v->nz * v->ny * v->nx, v->es == 16 ? CUFFT_Z2Z : CUFFT_C2C, 1));
    s->has_plan_psi = true;
    SP_FFT(c, g_fft.SetStream(s->plan_psi, v->stream));
  }
  if (!s->d_axes) {
    const int nx = v->nx, ny = v->ny, nz = v->nz;
    const double dk = 2.0 * M_PI / (double)(nx - 1);
    std::vector<double> t((size_t)nx + ny + nz);
    axis_terms(nx, v->dx, dk, t.data());
    axis_terms(ny, v->dy, dk, t.data() + nx);
    axis_terms(nz, v->dz, dk, t.data() + nx + ny);
    SP_CU(c, cudaMalloc(&s->d_axes, sizeof(double) * t.size()));
    SP_CU(c, cudaMemcpyAsync(s->d_axes, t.data(), sizeof(double) * t.size(),
                             cudaMemcpyHostToDevice, v->stream));
    SP_CU(c, cudaStreamSynchronize(v->stream));
  }
  *out = s;
  return GPE_OK;
}

// In-place transform of the staging buffer (timed as GPE_FAM_OTHER).
int exec(gpe_ctx* c, Spectral* s, const FieldView& v, int dir) {
  TimedRegion t;
  gpe_internal_time_begin(c, &t, GPE_FAM_OTHER, (int64_t)v.nx * v.ny * v.nz);
  if (v.es == 16) {
    auto* p = static_cast<cufftDoubleComplex*>(v.stage);
    SP_FFT(c, g_fft.ExecZ2Z(s->plan, p, p, dir));
  } else {
    auto* p = static_cast<cufftComplex*>(v.stage);
    SP_FFT(c, g_fft.ExecC2C(s->plan, p, p, dir));
  }
  gpe_internal_time_end(c, &t);
  return GPE_OK;
}

template <typename T, int E>
int launch_spectrum(gpe_ctx* c, Spectral* s, const FieldView& v, const SpecArgs& a,
                    const SpecFinal& f0, size_t smem, int64_t sites) {
  SP_CU(c, cudaFuncSetAttribute(spectrum_kernel<T, E>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  int per_sm = 1, sms = 148;
  SP_CU(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spectrum_kernel<T, E>, S_THREADS,
                                                         smem));
  SP_CU(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, v.dev));
  const long long nrows = (long long)v.ny * v.nz;
  const long long want = (nrows + S_WARPS - 1) / S_WARPS;
  const long long cap = (long long)sms * (per_sm > 0 ? per_sm : 1);
  const int nblk = (int)(want < cap ? want : cap);
  if (nblk != s->nblk || f0.nf != s->nf) {
    cudaFree(s->d_partials);
    cudaFree(s->d_out);
    s->d_partials = s->d_out = nullptr;
    // mark the cache empty first: a failed allocation below must not leave
    // sizes that let the next call launch on null buffers
    s->nblk = 0;
    s->nf = -1;
    SP_CU(c, cudaMalloc(&s->d_partials, sizeof(double) * (size_t)nblk * (HEAD + f0.nf)));
    SP_CU(c, cudaMalloc(&s->d_out, sizeof(double) * (size_t)(21 + f0.nf)));
    s->nblk = nblk;
    s->nf = f0.nf;
  }
  SpecArgs args = a;
  args.partials = s->d_partials;
  SpecFinal f = f0;
  f.nblk = nblk;
  f.out = s->d_out;
  const size_t fsmem = sizeof(double) * (size_t)(HEAD + f.nf);
  const T* buf = static_cast<const T*>(v.stage);
  TimedRegion t1, t2;
  gpe_internal_time_begin(c, &t1, GPE_FAM_SPECTRUM, sites);
  spectrum_kernel<T, E><<<nblk, S_THREADS, smem, v.stream>>>(buf, args);
  SP_CU(c, cudaGetLastError());
  gpe_internal_time_end(c, &t1);
  gpe_internal_time_begin(c, &t2, GPE_FAM_REDUCE, 0);
  spectrum_finalize_kernel<T><<<1, F_FIN_THREADS, fsmem, v.stream>>>(buf, s->d_partials, f);
  SP_CU(c, cudaGetLastError());
  gpe_internal_time_end(c, &t2);
  gpe_internal_count_launches(c, 2);
  return GPE_OK;
}

// Backward transform of psi straight from the padded field into the dense
// staging buffer (out of place: psi is only read).
int backward_from_psi(gpe_ctx* c, Spectral* s, const FieldView& v) {
  TimedRegion t;
  gpe_internal_time_begin(c, &t, GPE_FAM_OTHER, (int64_t)v.nx * v.ny * v.nz);
  const size_t origin = ((size_t)2 * v.Ny + 2) * v.Nx + 2;
  if (v.es == 16) {
    auto* in = static_cast<cufftDoubleComplex*>(v.psi) + origin;
    SP_FFT(c, g_fft.ExecZ2Z(s->plan_psi, in, static_cast<cufftDoubleComplex*>(v.stage),
                            CUFFT_INVERSE));
  } else {
    auto* in = static_cast<cufftComplex*>(v.psi) + origin;
    SP_FFT(c, g_fft.ExecC2C(s->plan_psi, in, static_cast<cufftComplex*>(v.stage),
                            CUFFT_INVERSE));
  }
  gpe_internal_time_end(c, &t);
  return GPE_OK;
}

int spectrum_pass(gpe_ctx* c, Spectral* s, const FieldView& v) {
  const int nf = v.nx / 2;
  const size_t smem = sizeof(double) * (size_t)S_WARPS * (nf > 0 ? nf : 1);
  if (smem > 160 * 1024)
    return gpe_internal_fail(c, GPE_ERR_INVALID, "spectrum supports nx up to 5120");
  const double N = (double)v.nx * v.ny * v.nz;
  SpecArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = v.nx; a.ny = v.ny; a.nz = v.nz; a.nf = nf;
  a.inv_n = 1.0 / N;
  a.inv_v = 1.0 / N;
  // shell thresholds in integer k2 (T 4^s is never within 1e-9 of an integer)
  const double T4 = 4.0 * M_PI * M_PI;
  for (int q = 0; q <= NSHELLS; q++) {
    a.shells.up[q] = (int)std::ceil(T4 * std::ldexp(1.0, 2 * q));
    a.shells.dn[q] = (int)std::floor(T4 * std::ldexp(1.0, -2 * q));
  }
  a.ax = s->d_axes;
  a.ay = s->d_axes + v.nx;
  a.az = s->d_axes + v.nx + v.ny;
  SpecFinal f;
  memset(&f, 0, sizeof(f));
  f.nf = nf; f.inv_n = 1.0 / N; f.volume_v = N;
  f.cell = v.dx * v.dy * v.dz;
  f.box8 = 8.0 * v.xr * v.yr * v.zr;
  const int64_t sites = (int64_t)v.nx * v.ny * v.nz;
  // sites per lane: a warp pass (32 E sites) about half a row, 2 to 8
  const int half = (v.nx + 1) / 2;
  if (v.es == 16) {
    if (half <= 64) return launch_spectrum<double, 2>(c, s, v, a, f, smem, sites);
    if (half <= 128) return launch_spectrum<double, 4>(c, s, v, a, f, smem, sites);
    return launch_spectrum<double, 8>(c, s, v, a, f, smem, sites);
  }
  if (half <= 64) return launch_spectrum<float, 2>(c, s, v, a, f, smem, sites);
  if (half <= 128) return launch_spectrum<float, 4>(c, s, v, a, f, smem, sites);
  return launch_spectrum<float, 8>(c, s, v, a, f, smem, sites);
}

}  // namespace

extern "C" {

int gpe_gpu_random_phase(gpe_ctx* c, double nv, double enerv, uint64_t seed, double* amp_out,
                         double* kc2_out) {
  FieldView v;
  Spectral* s = nullptr;
  int rc = prepare(c, &v, &s);
  if (rc) return rc;
  if (!(nv > 0.0) || !(enerv > 0.0))
    return gpe_internal_fail(c, GPE_ERR_INVALID, "nv and enerv must be positive");
  // get_kc_amp (src/ic.f90:256-269)
  const double N = (double)v.nx * v.ny * v.nz;
  const double ek = 0.5 * v.nx / M_PI;
  const double ev = (ek * ek) * enerv;
  const double amp = std::sqrt((0.11095279993106999 * std::pow(nv, 2.5)) * N / std::pow(ev, 1.5));
  const double kc2 = (1.666666666666666 * ev) / nv;
  if (amp_out) *amp_out = amp;
  if (kc2_out) *kc2_out = kc2;
  const size_t n = (size_t)v.nx * v.ny * v.nz;
  const int nb = elementwise_grid(n);
  if (v.es == 16)
    random_phase_kernel<double><<<nb, 256, 0, v.stream>>>(static_cast<double*>(v.stage), v.nx,
                                                         v.ny, v.nz, amp / std::sqrt(N), kc2,
                                                         seed);
  else
    random_phase_kernel<float><<<nb, 256, 0, v.stream>>>(static_cast<float*>(v.stage), v.nx,
                                                        v.ny, v.nz, amp / std::sqrt(N), kc2,
                                                        seed);
  SP_CU(c, cudaGetLastError());
  gpe_internal_count_launches(c, 1);
  if ((rc = exec(c, s, v, CUFFT_FORWARD))) return rc;
  if ((rc = gpe_internal_load_stage(c))) return rc;
  SP_CU(c, cudaStreamSynchronize(v.stream));
  return GPE_OK;
}

int gpe_gpu_condensed_particles(gpe_ctx* c, double* row, double* eta, int64_t* nharm, double* F,
                                int32_t nf) {
  FieldView v;
  Spectral* s = nullptr;
  int rc = prepare(c, &v, &s);
  if (rc) return rc;
  if (F && nf != v.nx / 2)
    return gpe_internal_fail(c, GPE_ERR_INVALID, "F needs nf = nx/2 entries");
  if ((rc = backward_from_psi(c, s, v))) return rc;
  if ((rc = spectrum_pass(c, s, v))) return rc;
  std::vector<double> h((size_t)21 + s->nf);
  SP_CU(c, cudaMemcpyAsync(h.data(), s->d_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                           v.stream));
  SP_CU(c, cudaStreamSynchronize(v.stream));
  if (row) memcpy(row, h.data(), sizeof(double) * 7);
  if (eta) memcpy(eta, h.data() + 7, sizeof(double) * NSHELLS);
  if (nharm)
    for (int m = 0; m < NSHELLS; m++) nharm[m] = (int64_t)h[14 + m];
  if (F) memcpy(F, h.data() + 21, sizeof(double) * (size_t)s->nf);
  return GPE_OK;
}

int gpe_gpu_filtered_field(gpe_ctx* c, double filter_kc, double m, void* out, int32_t elem_bytes,
                           int32_t device_out) {
  FieldView v;
  Spectral* s = nullptr;
  int rc = prepare(c, &v, &s);
  if (rc) return rc;
  if (!out) return gpe_internal_fail(c, GPE_ERR_INVALID, "null output");
  if (elem_bytes != v.es)
    return gpe_internal_fail(c, GPE_ERR_INVALID, "elem_bytes must match the field's precision");
  if (!(filter_kc > 0.0)) return gpe_internal_fail(c, GPE_ERR_INVALID, "filter_kc must be positive");
  if ((rc = backward_from_psi(c, s, v))) return rc;
  const size_t n = (size_t)v.nx * v.ny * v.nz;
  const int nb = elementwise_grid(n);
  const double scale = 1.0 / (double)n;
  if (v.es == 16)
    filter_kernel<double><<<nb, 256, 0, v.stream>>>(static_cast<double*>(v.stage), v.nx, v.ny,
                                                   v.nz, m, filter_kc * filter_kc, scale);
  else
    filter_kernel<float><<<nb, 256, 0, v.stream>>>(static_cast<float*>(v.stage), v.nx, v.ny,
                                                  v.nz, m, filter_kc * filter_kc, scale);
  SP_CU(c, cudaGetLastError());
  gpe_internal_count_launches(c, 1);
  if ((rc = exec(c, s, v, CUFFT_FORWARD))) return rc;
  SP_CU(c, cudaMemcpyAsync(out, v.stage, n * (size_t)elem_bytes,
                           device_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           v.stream));
  SP_CU(c, cudaStreamSynchronize(v.stream));
  return GPE_OK;
}

}  // extern "C"
