// vortex.cu -- gpe_gpu_linelength (include/gpe_gpu.h): total vortex line
// length of the resident state; kernels in vortex_kernels.cuh.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "gpe_gpu.h"
#include "internal.h"
#include "vortex_kernels.cuh"

using namespace gpe;
using namespace gpe::vortex;

namespace {

struct Vortex : Extension {
  int nblk = 0;
  void* mem = nullptr;
  // zero finders: grid tables, per-block counts / offsets, point list
  double* grid = nullptr;
  long long* zcount = nullptr;
  int znblk = 0;
  double* zpts = nullptr;
  long long zcap = 0;
  ~Vortex() override {
    cudaFree(mem);
    cudaFree(grid);
    cudaFree(zcount);
    cudaFree(zpts);
  }
};

Vortex* vortex_ext(gpe_ctx* c) {
  auto& slot = gpe_internal_extension(c, GPE_EXT_VORTEX);
  if (!slot) slot.reset(new Vortex());
  return static_cast<Vortex*>(slot.get());
}

#define VX_CU(c, call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return gpe_internal_fail((c), GPE_ERR_CUDA,                                   \
                               std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// field: the resident padded psi (dense = false) or a dense interior array.
template <typename T>
int run(gpe_ctx* c, const FieldView& v, const void* field, bool dense, double* length) {
  LineArgs p;
  p.psi = field;
  p.nx = v.nx;
  p.ny = v.ny;
  p.nz = v.nz;
  p.Nx = dense ? v.nx : v.Nx;
  p.Ny = dense ? v.ny : v.Ny;
  p.ghost = dense ? 0 : 2;
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
  Vortex* x = vortex_ext(c);
  // per block: bsum, blast[4], bbuf[L_CAP][3], bres doubles,
  // bfirst (long long), bunres (int); plus the total
  const size_t per = sizeof(double) * (1 + 4 + L_CAP * 3 + 1) + sizeof(long long) +
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
  p.out = d;
  d += 1;
  p.bfirst = reinterpret_cast<long long*>(d);
  p.bunres = reinterpret_cast<int*>(p.bfirst + nblk);
  TimedRegion t;
  gpe_internal_time_begin(c, &t, GPE_FAM_OTHER, (int64_t)p.ncell);
  line_cells_kernel<T><<<nblk, L_THREADS, 0, v.stream>>>(p);
  VX_CU(c, cudaGetLastError());
  gpe_internal_time_end(c, &t);
  line_resolve_kernel<T><<<nblk, L_THREADS, 0, v.stream>>>(p);
  VX_CU(c, cudaGetLastError());
  line_total_kernel<<<1, L_THREADS, 0, v.stream>>>(p, nblk, v.dx);
  VX_CU(c, cudaGetLastError());
  gpe_internal_count_launches(c, 3);
  VX_CU(c, cudaMemcpyAsync(length, p.out, sizeof(double), cudaMemcpyDeviceToHost, v.stream));
  VX_CU(c, cudaStreamSynchronize(v.stream));
  return GPE_OK;
}

template <typename T>
int run_zeros(gpe_ctx* c, const FieldView& v, int64_t* counts, double* points, int64_t cap) {
  Vortex* x = vortex_ext(c);
  ZeroArgs p;
  p.psi = v.psi;
  p.nx = v.nx;
  p.ny = v.ny;
  p.nz = v.nz;
  p.Nx = v.Nx;
  p.Ny = v.Ny;
  p.cx = v.nx - 2;
  const long long rows = (long long)(v.ny - 2) * (v.nz - 2);
  p.ncell = rows * p.cx;
  int sms = 148;
  VX_CU(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, v.dev));
  const long long want = (long long)sms * 4;
  const long long rows_per_block = (rows + want - 1) / want;
  const int nblk = (int)((rows + rows_per_block - 1) / rows_per_block);
  p.per_block = rows_per_block * p.cx;
  if (!x->grid) {
    std::vector<double> g((size_t)v.nx + v.ny + v.nz);
    if (gpe_gpu_grid(c, g.data(), g.data() + v.nx, g.data() + v.nx + v.ny))
      return gpe_internal_fail(c, GPE_ERR_INVALID, "grid unavailable");
    VX_CU(c, cudaMalloc(&x->grid, sizeof(double) * g.size()));
    VX_CU(c, cudaMemcpyAsync(x->grid, g.data(), sizeof(double) * g.size(),
                             cudaMemcpyHostToDevice, v.stream));
  }
  p.x = x->grid;
  p.y = x->grid + v.nx;
  p.z = x->grid + v.nx + v.ny;
  if (x->znblk < nblk) {
    cudaFree(x->zcount);
    x->zcount = nullptr;
    x->znblk = 0;
    VX_CU(c, cudaMalloc(&x->zcount, sizeof(long long) * 2 * Z_SECTIONS * (size_t)nblk));
    x->znblk = nblk;
  }
  p.bcount = x->zcount;
  p.boff = x->zcount + (size_t)Z_SECTIONS * nblk;
  p.pts = nullptr;
  zeros_count_kernel<T><<<nblk, L_THREADS, 0, v.stream>>>(p);
  VX_CU(c, cudaGetLastError());
  std::vector<long long> cnt((size_t)Z_SECTIONS * nblk), off((size_t)Z_SECTIONS * nblk);
  VX_CU(c, cudaMemcpyAsync(cnt.data(), p.bcount, sizeof(long long) * cnt.size(),
                           cudaMemcpyDeviceToHost, v.stream));
  VX_CU(c, cudaStreamSynchronize(v.stream));
  gpe_internal_count_launches(c, 1);
  // slots: section by section, blocks in order within a section
  long long total = 0;
  for (int s = 0; s < Z_SECTIONS; s++) {
    long long sec = 0;
    for (int b = 0; b < nblk; b++) {
      off[(size_t)b * Z_SECTIONS + s] = total;
      total += cnt[(size_t)b * Z_SECTIONS + s];
      sec += cnt[(size_t)b * Z_SECTIONS + s];
    }
    if (counts) counts[s] = sec;
  }
  if (!points) return GPE_OK;
  if (total > cap)
    return gpe_internal_fail(c, GPE_ERR_INVALID,
                             "points holds " + std::to_string(cap) + " points, " +
                                 std::to_string(total) + " needed (counts are filled)");
  if (total == 0) return GPE_OK;
  if (x->zcap < total) {
    cudaFree(x->zpts);
    x->zpts = nullptr;
    x->zcap = 0;
    VX_CU(c, cudaMalloc(&x->zpts, sizeof(double) * 3 * (size_t)total));
    x->zcap = total;
  }
  p.pts = x->zpts;
  VX_CU(c, cudaMemcpyAsync(const_cast<long long*>(p.boff), off.data(),
                           sizeof(long long) * off.size(), cudaMemcpyHostToDevice, v.stream));
  zeros_write_kernel<T><<<nblk, L_THREADS, 0, v.stream>>>(p);
  VX_CU(c, cudaGetLastError());
  gpe_internal_count_launches(c, 1);
  VX_CU(c, cudaMemcpyAsync(points, p.pts, sizeof(double) * 3 * (size_t)total,
                           cudaMemcpyDeviceToHost, v.stream));
  VX_CU(c, cudaStreamSynchronize(v.stream));
  return GPE_OK;
}

}  // namespace

extern "C" int gpe_gpu_zeros(gpe_ctx* c, int64_t* counts, double* points, int64_t cap) {
  FieldView v;
  if (!c || gpe_internal_field_view(c, &v)) return GPE_ERR_INVALID;
  VX_CU(c, cudaSetDevice(v.dev));
  if (!v.single_domain)
    return gpe_internal_fail(c, GPE_ERR_INVALID,
                             "zero finders need a single-domain context (the whole grid)");
  if (!counts) return gpe_internal_fail(c, GPE_ERR_INVALID, "null counts");
  return v.es == 16 ? run_zeros<double>(c, v, counts, points, cap)
                    : run_zeros<float>(c, v, counts, points, cap);
}

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
  return v.es == 16 ? run<double>(c, v, v.psi, false, length)
                    : run<float>(c, v, v.psi, false, length);
}

extern "C" int gpe_gpu_linelength_field(gpe_ctx* c, const void* field, int32_t elem_bytes,
                                        double* length) {
  FieldView v;
  if (!c || gpe_internal_field_view(c, &v)) return GPE_ERR_INVALID;
  if (!length || !field) return gpe_internal_fail(c, GPE_ERR_INVALID, "null argument");
  if (elem_bytes != 8 && elem_bytes != 16)
    return gpe_internal_fail(c, GPE_ERR_INVALID, "elem_bytes must be 8 or 16");
  VX_CU(c, cudaSetDevice(v.dev));
  if (!v.single_domain)
    return gpe_internal_fail(c, GPE_ERR_INVALID,
                             "linelength needs a single-domain context (the whole grid)");
  if (v.nx < 3 || v.ny < 3 || v.nz < 3) {
    *length = 0.0;
    return GPE_OK;
  }
  return elem_bytes == 16 ? run<double>(c, v, field, true, length)
                          : run<float>(c, v, field, true, length);
}
