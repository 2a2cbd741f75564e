// internal.h -- library-internal access between translation units (not part
// of the C-ABI).
#pragma once

#include <cuda_runtime.h>

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
};

}  // namespace gpe

// Fills *v; marks the context's cached norm stale (the caller may write psi).
int gpe_internal_field_view(gpe_ctx* c, gpe::FieldView* v);
// fn(arg, c) is called after every completed step of c (enqueueing work on
// c's stream); null detaches.
void gpe_internal_set_post_step(gpe_ctx* c, int (*fn)(void*, gpe_ctx*), void* arg);
void gpe_internal_set_last_error(const std::string& msg);
