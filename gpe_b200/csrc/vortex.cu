// vortex.cu -- gpe_gpu_linelength (include/gpe_gpu.h): total vortex line
// length of the resident state; kernels in vortex_kernels.cuh.
#include <cuda_runtime.h>

#include <string>

#include "gpe_gpu.h"
#include "internal.h"
#include "vortex_kernels.cuh"

using namespace gpe;
using namespace gpe::vortex;

namespace {

struct Vortex : Extension {
  int nblk = 0;
  void* mem = nullptr;
  ~Vortex() override { cudaFree(mem); }
};

#define VX_CU(c, call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return gpe_internal_fail((c), GPE_ERR_CUDA,                                   \
                               std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
int run(gpe_ctx* c, const FieldView& v, double* length) {
  LineArgs p;
  p.psi = v.psi;
  p.nx = v.nx;
  p.ny = v.ny;
  p.nz = v.nz;
  p.Nx = v.Nx;
  p.Ny = v.Ny;
  p.cx = v.nx - 2;
  const long long rows = (long long)(v.ny - 2) * (v.nz - 2);
  p.ncell = rows * p.cx;
  int sms = 148, per_sm = 1;
  VX_CU(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, v.dev));
  VX_CU(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, line_cells_kernel<T>,
                                                         L_THREADS, 0));
  // two waves of resident blocks, each block whole rows in loop order
  const long long want = (long long)sms * (per_sm > 0 ? per_sm : 1) * 2;
  const long long rows_per_block = (rows + want - 1) / want;
  const int nblk = (int)((rows + rows_per_block - 1) / rows_per_block);
  p.per_block = rows_per_block * p.cx;
  auto& slot = gpe_internal_extension(c, GPE_EXT_VORTEX);
  if (!slot) slot.reset(new Vortex());
  Vortex* x = static_cast<Vortex*>(slot.get());
  // per block: bsum, blast[4], bbuf[L_CAP][3], bres, incoming[3] doubles,
  // bfirst (long long), bunres (int); plus the total
  const size_t per = sizeof(double) * (1 + 4 + L_CAP * 3 + 1 + 3) + sizeof(long long) +
                     sizeof(int);
  if (x->nblk < nblk) {
    cudaFree(x->mem);
    x->mem = nullptr;
    x->nblk = 0;
    VX_CU(c, cudaMalloc(&x->mem, per * (size_t)nblk + 64));
    x->nblk = nblk;
  }
  double* d = static_cast<double*>(x->mem);
  p.bsum = d;
  d += nblk;
  p.blast = d;
  d += 4 * (size_t)nblk;
  p.bbuf = d;
  d += (size_t)L_CAP * 3 * nblk;
  p.bres = d;
  d += nblk;
  p.incoming = d;
  d += 3 * (size_t)nblk;
  p.out = d;
  d += 1;
  p.bfirst = reinterpret_cast<long long*>(d);
  p.bunres = reinterpret_cast<int*>(p.bfirst + nblk);
  TimedRegion t;
  gpe_internal_time_begin(c, &t, GPE_FAM_OTHER, (int64_t)p.ncell);
  line_cells_kernel<T><<<nblk, L_THREADS, 0, v.stream>>>(p);
  VX_CU(c, cudaGetLastError());
  gpe_internal_time_end(c, &t);
  line_chain_kernel<<<1, 32, 0, v.stream>>>(p, nblk);
  VX_CU(c, cudaGetLastError());
  line_resolve_kernel<T><<<nblk, L_THREADS, 0, v.stream>>>(p);
  VX_CU(c, cudaGetLastError());
  line_total_kernel<<<1, L_THREADS, 0, v.stream>>>(p, nblk, v.dx);
  VX_CU(c, cudaGetLastError());
  gpe_internal_count_launches(c, 4);
  VX_CU(c, cudaMemcpyAsync(length, p.out, sizeof(double), cudaMemcpyDeviceToHost, v.stream));
  VX_CU(c, cudaStreamSynchronize(v.stream));
  return GPE_OK;
}

}  // namespace

extern "C" int gpe_gpu_linelength(gpe_ctx* c, double* length) {
  FieldView v;
  if (!c || gpe_internal_field_view(c, &v)) return GPE_ERR_INVALID;
  if (!length) return gpe_internal_fail(c, GPE_ERR_INVALID, "null output");
  VX_CU(c, cudaSetDevice(v.dev));
  if (!v.single_domain)
    return gpe_internal_fail(c, GPE_ERR_INVALID,
                             "linelength needs a single-domain context (the whole grid)");
  if (v.nx < 3 || v.ny < 3 || v.nz < 3) {
    *length = 0.0;
    return GPE_OK;
  }
  return v.es == 16 ? run<double>(c, v, length) : run<float>(c, v, length);
}
