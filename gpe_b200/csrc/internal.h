// internal.h -- library-internal access between translation units (not part
// of the C-ABI).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>

#include "gpe_gpu.h"

namespace gpe {

// The resident psi of a context: padded field (2 ghosts per side, pitches
// Nx >= nx + 4, Ny = ny + 4), complex of es bytes.
struct FieldView {
  void* psi;
  int nx, ny, nz, Nx, Ny;
  int es;
  int bcs;
  int dev;
  int single_domain;
  cudaStream_t stream;
  int* status;  // the context's device status word (wait timeouts)
  double dx, dy, dz;  // grid spacings, 2 xr / (nx - 1) etc.
  double xr, yr, zr;  // box half-widths
  void* stage;        // dense staging buffer, nx ny nz elements of 16 bytes
};

// A timed region on a context's stream (recorded only while the context's
// timing is on; collected by gpe_gpu_get_timing under `family`).
struct TimedRegion {
  cudaEvent_t a = nullptr, b = nullptr;
  int family = 0;
  int64_t sites = 0;
};

// Per-context state of another translation unit, owned by the context and
// deleted with it (with the context's device current, its stream drained).
struct Extension {
  virtual ~Extension() = default;
};

}  // namespace gpe

// Fills *v; marks the context's cached norm stale (the caller may write psi).
int gpe_internal_field_view(gpe_ctx* c, gpe::FieldView* v);
// fn(arg, c) is called after every completed step of c (enqueueing work on
// c's stream); null detaches.
void gpe_internal_set_post_step(gpe_ctx* c, int (*fn)(void*, gpe_ctx*), void* arg);
void gpe_internal_set_last_error(const std::string& msg);
// Records msg as the context's last error and returns code.
int gpe_internal_fail(gpe_ctx* c, int code, const std::string& msg);
// The context's extension slots (0 spectral, 1 vortex line length).
constexpr int GPE_EXT_SPECTRAL = 0, GPE_EXT_VORTEX = 1, GPE_EXT_SLOTS = 2;
std::unique_ptr<gpe::Extension>& gpe_internal_extension(gpe_ctx* c, int slot);
// Dense staging buffer (x fastest, elements of the field's own es bytes) ->
// psi with the boundary ghosts filled; invalidates the cached norm.
int gpe_internal_load_stage(gpe_ctx* c);
void gpe_internal_time_begin(gpe_ctx* c, gpe::TimedRegion* r, int family, int64_t sites);
void gpe_internal_time_end(gpe_ctx* c, gpe::TimedRegion* r);
// Enqueues psi *= sqrt(norm of the last step / norm of psi now) (the norm
// kept through a post-step correction).
int gpe_internal_restore_norm(gpe_ctx* c);
// Adds n to the context's launch counter (kernels enqueued by other units).
void gpe_internal_count_launches(gpe_ctx* c, int64_t n);
