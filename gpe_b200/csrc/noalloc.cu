// noalloc.cu -- get_norm of a caller-owned device array without allocating.
//
// Some hosts cannot call cudaMalloc: their device memory belongs to another
// allocator (a framework's caching allocator, or a driver program that sizes
// all device memory up front and treats any later allocation as an error).
// gpe_gpu_norm_noalloc serves them: it needs no context and allocates
// nothing.  Its only scratch is the file-scope array below, one FP64 partial
// sum per z-plane, which every GPU that loads this library holds until the
// process exits.
//
// The reduction is the extended-Simpson norm of the reference's get_norm
// (src/variables.f90:537-559, integrate_x/y/z :713-823): each CTA sums one
// z-plane, sum_j wy(j) sum_i wx(i) |psi|^2, into the scratch array, and one
// CTA then forms sum_k wz(k) * plane(k) * dx dy dz in a fixed order.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "device_utils.cuh"
#include "gpe_gpu.h"

// defined in gpe_gpu.cu: the message gpe_gpu_last_error(NULL) returns
void gpe_internal_set_last_error(const std::string& msg);

namespace {

constexpr int kMaxPlanes = GPE_NOALLOC_MAX_PLANES;
constexpr int kMaxDevices = 64;

// The scratch.  In host code this name is only a stand-in for the device
// array; its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double g_plane_scratch[kMaxPlanes];

std::mutex g_mutex;
double* g_scratch_addr[kMaxDevices] = {};

// Extended-Simpson weights (src/variables.f90:49-51).  Along x every term of
// integrate_x that names index i contributes; along y and z the last
// matching assignment of integrate_y / integrate_z wins.
__device__ __forceinline__ double weight_x(int i, int n) {
  double w = 0.0;
  if (i == 0) w += 3.0 / 8.0;
  if (i == 1) w += 7.0 / 6.0;
  if (i == 2) w += 23.0 / 24.0;
  if (i >= 3 && i <= n - 4) w += 1.0;
  if (i == n - 3) w += 23.0 / 24.0;
  if (i == n - 2) w += 7.0 / 6.0;
  if (i == n - 1) w += 3.0 / 8.0;
  return w;
}

__device__ __forceinline__ double weight_yz(int j, int n) {
  double w = 1.0;
  if (j == 0) w = 3.0 / 8.0;
  if (j == 1) w = 7.0 / 6.0;
  if (j == 2) w = 23.0 / 24.0;
  if (j == n - 3) w = 23.0 / 24.0;
  if (j == n - 2) w = 7.0 / 6.0;
  if (j == n - 1) w = 3.0 / 8.0;
  return w;
}

// One CTA per z-plane: plane[k] = sum_j wy(j) sum_i wx(i) |psi(i,j,k)|^2.
template <typename T>
__global__ void plane_sums_kernel(const T* __restrict__ psi, int nx, int ny,
                                  double* __restrict__ plane) {
  __shared__ double s[32];
  const int k = blockIdx.x;
  const size_t off = (size_t)k * ny * nx;
  double acc = 0.0;
  const long long nq = (long long)nx * ny;
  for (long long q = threadIdx.x; q < nq; q += blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const double a = (double)psi[2 * (off + q)], b = (double)psi[2 * (off + q) + 1];
    acc += weight_x(i, nx) * weight_yz(j, ny) * (a * a + b * b);
  }
  acc = gpe::warp_sum(acc);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s[w];
    plane[k] = t;  // every slot this call reads is written first
  }
}

// Single CTA: out = sum_k wz(k) plane[k] * dV, fixed order.
__global__ void planes_to_norm_kernel(const double* __restrict__ plane, int nz,
                                      double dv, double* __restrict__ out) {
  __shared__ double s[1024];
  double a = 0.0;
  for (int k = threadIdx.x; k < nz; k += blockDim.x) a += weight_yz(k, nz) * plane[k];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0] * dv;
}

int noalloc_fail(int code, const std::string& msg) {
  gpe_internal_set_last_error(msg);  // read back with gpe_gpu_last_error(NULL)
  return code;
}

// Device address of the scratch array on the current device, looked up once
// per device.
int scratch_address(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(GPE_ERR_NODEVICE, "gpe_gpu_norm_noalloc: no current CUDA device");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_plane_scratch);
    if (e != cudaSuccess || !ptr)
      return noalloc_fail(GPE_ERR_CUDA, std::string("gpe_gpu_norm_noalloc: "
                                                    "cudaGetSymbolAddress failed: ") +
                                            cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double*>(ptr);
  }
  *out = g_scratch_addr[dev];
  return GPE_OK;
}

}  // namespace

extern "C" int gpe_gpu_norm_noalloc(const void* psi, int32_t elem_bytes, int32_t nx,
                                    int32_t ny, int32_t nz, double xr, double yr,
                                    double zr, double* norm_out, void* stream) {
  if (!psi || !norm_out)
    return noalloc_fail(GPE_ERR_INVALID, "gpe_gpu_norm_noalloc: null array");
  if (elem_bytes != 8 && elem_bytes != 16)
    return noalloc_fail(GPE_ERR_INVALID, "gpe_gpu_norm_noalloc: elem_bytes must be 8 or 16");
  if (nx < 6 || ny < 6 || nz < 6)
    return noalloc_fail(GPE_ERR_INVALID, "gpe_gpu_norm_noalloc: nx, ny, nz must be >= 6");
  if (nz > kMaxPlanes)
    return noalloc_fail(GPE_ERR_INVALID,
                        "gpe_gpu_norm_noalloc: nz = " + std::to_string(nz) +
                            " exceeds the fixed scratch of " + std::to_string(kMaxPlanes) +
                            " z-planes (GPE_NOALLOC_MAX_PLANES)");
  if ((long long)nx * (long long)ny > 0x7fffffffLL)
    return noalloc_fail(GPE_ERR_INVALID, "gpe_gpu_norm_noalloc: nx*ny too large");
  if (!(xr > 0.0 && yr > 0.0 && zr > 0.0))
    return noalloc_fail(GPE_ERR_INVALID, "gpe_gpu_norm_noalloc: xr, yr, zr must be positive");
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  // get_grid (src/ic.f90:46-48)
  const double dx = (xr - (-xr)) / (double)(nx - 1);
  const double dy = (yr - (-yr)) / (double)(ny - 1);
  const double dz = (zr - (-zr)) / (double)(nz - 1);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (elem_bytes == 8)
    plane_sums_kernel<float><<<nz, 256, 0, st>>>(static_cast<const float*>(psi), nx, ny,
                                                  scratch);
  else
    plane_sums_kernel<double><<<nz, 256, 0, st>>>(static_cast<const double*>(psi), nx, ny,
                                                   scratch);
  planes_to_norm_kernel<<<1, 1024, 0, st>>>(scratch, nz, dx * dy * dz, norm_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return noalloc_fail(GPE_ERR_CUDA, std::string("gpe_gpu_norm_noalloc: launch failed: ") +
                                          cudaGetErrorString(e));
  return GPE_OK;
}
