// cnn.cu -- host side of the learned coarse-grid correction (include/gpe_cnn.h).
//
// Buffers (bf16 activations, layout of cnn_kernels.cuh): inference uses
// A0 (one channel half: Re, Im, 0 ...) and two 16-channel buffers A1, A2 in
// turn; training keeps every layer's input (T0 with both halves, T1..T3)
// and pre-activation (P0..P2) for the backward pass, plus two gradient
// buffers GA, GB used in turn.
//
// Training step (all on the context's stream):
//   pack u -> T0; conv0..2 (GELU, keep pre) -> T1..T3; conv3 -> delta;
//   loss -> GA (dL/d out of layer 3);
//   for l = 3..0: wgrad(T_l, G) -> dW_l; channel sums of G -> db_l;
//                 l > 0: dgrad conv of G with mirrored, transposed W_l times
//                 gelu'(P_{l-1}) -> the other G buffer;
//   Adam; repack bf16 weight tiles.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cnn_kernels.cuh"
#include "gpe_cnn.h"
#include "internal.h"

using namespace gpe;
using namespace gpe::cnn;

namespace {

thread_local std::string g_cnn_error;
constexpr unsigned long long CNN_WAIT_LIMIT_NS = 2000000000ull;

struct Act {
  __nv_bfloat16* p = nullptr;
  int H = 2;
};

}  // namespace

struct gpe_cnn {
  gpe_cnn_params prm;
  int dev = 0;
  int num_sms = 148;
  int nx, ny, nz, Xp, Yp, Zp;
  size_t nint = 0;
  // weights
  std::vector<float> hw, hb;
  float* d_w = nullptr;      // fp32 [4][27][16][16]
  float* d_b = nullptr;      // fp32 [4][16]
  __nv_bfloat16* d_wf = nullptr;
  __nv_bfloat16* d_wt = nullptr;
  __nv_bfloat16* d_wf2 = nullptr;  // last layer, N = 32 layout
  unsigned char* d_mask = nullptr;  // [weights + biases]
  float* d_grad = nullptr;   // [weights + biases]
  float* d_m = nullptr;
  float* d_v = nullptr;
  int64_t adam_t = 0;
  // activations
  Act A0, A1, A2;                       // inference
  Act T[4], P[3], GA, GB;               // training
  float* d_delta = nullptr;
  float* d_wpart = nullptr;
  float* d_bpart = nullptr;
  double* d_lpart = nullptr;
  int* d_status = nullptr;
  int wgrad_grid = 0;
  int ew_blocks = 0;
  int64_t launches = 0;
  std::string err;
};

namespace {

int cfail(gpe_cnn* n, int code, const std::string& msg) {
  if (n) n->err = msg;
  else g_cnn_error = msg;
  return code;
}

#define CNN_CU(n, call)                                                     \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess)                                                  \
      return cfail((n), GPE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

size_t act_bytes(const gpe_cnn* n, int H) {
  return (size_t)n->Zp * n->Yp * H * n->Xp * 16;
}

int alloc_act(gpe_cnn* n, Act& a, int H) {
  a.H = H;
  CNN_CU(n, cudaMalloc(&a.p, act_bytes(n, H)));
  CNN_CU(n, cudaMemset(a.p, 0, act_bytes(n, H)));
  return GPE_OK;
}

uint32_t round1k(uint32_t b) { return (b + 1023u) & ~1023u; }

// Items of a conv launch: y-slabs of TYF rows x z-chunks, about one per SM.
void conv_items(const gpe_cnn* n, int rows, int* nslab, int* nzc, int* zchunk) {
  *nslab = (n->ny + rows - 1) / rows;
  int want = std::max(1, F_CTAS_PER_SM * n->num_sms / *nslab);
  want = std::min(want, n->nz);
  *zchunk = (n->nz + want - 1) / want;
  *nzc = (n->nz + *zchunk - 1) / *zchunk;
}

template <int EPI>
int launch_conv(gpe_cnn* n, cudaStream_t st, const Act& in, int layer, bool dgrad,
                ConvParams& p) {
  // the last layer's 2 output channels use the N = 32 kernel
  constexpr int CO = (EPI == EPI_RESID || EPI == EPI_DELTA) ? 2 : 16;
  p.in = in.p;
  p.w = CO == 2 ? n->d_wf2
                : (dgrad ? n->d_wt : n->d_wf) + (size_t)layer * W_TILES * WT_BYTES / 2;
  p.bias = dgrad ? nullptr : n->d_b + layer * 16;
  p.nx = n->nx; p.ny = n->ny; p.nz = n->nz;
  p.Xp = n->Xp; p.Yp = n->Yp; p.Zp = n->Zp; p.Hin = in.H;
  conv_items(n, TYF, &p.nslab, &p.nzc, &p.zchunk);
  p.nitems = p.nslab * p.nzc;
  p.box_bytes = (uint32_t)((TYF + 2) * in.H * n->Xp * 16);
  p.slot_bytes = round1k(p.box_bytes);
  p.out_scale = n->prm.out_scale;
  if (!p.status) p.status = n->d_status;
  p.wait_limit_ns = CNN_WAIT_LIMIT_NS;
  const size_t smem = 1024 + (size_t)FSLOTS * p.slot_bytes + 4096 +
                      W_TILES * OutShape<CO>::WTB + F_TAIL_BYTES;
  auto fn = conv_fwd_kernel<EPI, CO>;
  CNN_CU(n, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::min(p.nitems, F_CTAS_PER_SM * n->num_sms);
  fn<<<grid, F_THREADS, smem, st>>>(p);
  CNN_CU(n, cudaGetLastError());
  n->launches++;
  return GPE_OK;
}

int launch_wgrad(gpe_cnn* n, cudaStream_t st, const Act& x, const Act& dy) {
  WgradParams p;
  memset(&p, 0, sizeof(p));
  p.x = x.p;
  p.dy = dy.p;
  p.nx = n->nx; p.ny = n->ny; p.nz = n->nz;
  p.Xp = n->Xp; p.Yp = n->Yp; p.Zp = n->Zp;
  p.nslab = (n->ny + TYW - 1) / TYW;
  const int want = std::min(n->nz, std::max(1, (2 * n->num_sms + p.nslab - 1) / p.nslab));
  p.zchunk = (n->nz + want - 1) / want;
  p.nzc = (n->nz + p.zchunk - 1) / p.zchunk;
  p.nitems = p.nslab * p.nzc;
  p.xbox_bytes = (uint32_t)(XROWS * 2 * n->Xp * 16);
  p.xslot_bytes = round1k(p.xbox_bytes);
  p.dbox_bytes = (uint32_t)(TYW * 2 * n->Xp * 16);
  p.dslot_bytes = round1k(p.dbox_bytes);
  p.partials = n->d_wpart;
  p.status = n->d_status;
  p.wait_limit_ns = CNN_WAIT_LIMIT_NS;
  const size_t smem = 1024 + (size_t)WSLOTS * p.xslot_bytes + (size_t)DSLOTS * p.dslot_bytes +
                      16 * 8 + 16;
  CNN_CU(n, cudaFuncSetAttribute(conv_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  conv_wgrad_kernel<<<n->wgrad_grid, W_THREADS, smem, st>>>(p);
  CNN_CU(n, cudaGetLastError());
  n->launches++;
  return GPE_OK;
}

int check_view(gpe_cnn* n, const FieldView& v) {
  if (v.nx != n->nx || v.ny != n->ny || v.nz != n->nz)
    return cfail(n, GPE_ERR_INVALID, "context grid differs from the network's grid");
  if (v.es != 8) return cfail(n, GPE_ERR_INVALID, "the learned correction needs complex64 psi");
  if (v.bcs != 1) return cfail(n, GPE_ERR_INVALID, "the learned correction needs periodic bcs");
  if (!v.single_domain) return cfail(n, GPE_ERR_INVALID, "z-slab contexts are not supported");
  if (v.dev != n->dev) return cfail(n, GPE_ERR_INVALID, "context on another device");
  return GPE_OK;
}

int pack_input(gpe_cnn* n, const FieldView& v, const Act& dst) {
  pack_input_kernel<float><<<n->Zp * n->Yp, 128, 0, v.stream>>>(
      static_cast<const float*>(v.psi), v.Nx, v.Ny, n->nx, n->ny, n->nz, dst.p, dst.H);
  CNN_CU(n, cudaGetLastError());
  n->launches++;
  return GPE_OK;
}

int sync_status(gpe_cnn* n, cudaStream_t st) {
  CNN_CU(n, cudaStreamSynchronize(st));
  int s = 0;
  CNN_CU(n, cudaMemcpy(&s, n->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (s) {
    cudaMemset(n->d_status, 0, sizeof(int));
    return cfail(n, GPE_ERR_TIMEOUT, "device-side wait limit expired in a conv kernel");
  }
  return GPE_OK;
}

// Inference: enqueue psi += delta(psi) on the view's stream.  A wait
// timeout is recorded in `status` (the network's own word, or the
// context's when the correction runs as part of the context's steps).
int enqueue_apply(gpe_cnn* n, const FieldView& v, int* status) {
  int rc = pack_input(n, v, n->A0);
  if (rc) return rc;
  ConvParams p;
  memset(&p, 0, sizeof(p));
  p.status = status;
  p.act_out = n->A1.p;
  if ((rc = launch_conv<EPI_GELU>(n, v.stream, n->A0, 0, false, p))) return rc;
  memset(&p, 0, sizeof(p));
  p.status = status;
  p.act_out = n->A2.p;
  if ((rc = launch_conv<EPI_GELU>(n, v.stream, n->A1, 1, false, p))) return rc;
  memset(&p, 0, sizeof(p));
  p.status = status;
  p.act_out = n->A1.p;
  if ((rc = launch_conv<EPI_GELU>(n, v.stream, n->A2, 2, false, p))) return rc;
  memset(&p, 0, sizeof(p));
  p.status = status;
  p.psi = static_cast<float*>(v.psi);
  p.psi_Nx = v.Nx;
  p.psi_Ny = v.Ny;
  return launch_conv<EPI_RESID>(n, v.stream, n->A1, 3, false, p);
}

int post_step_hook(void* arg, gpe_ctx* c) {
  gpe_cnn* n = static_cast<gpe_cnn*>(arg);
  FieldView v;
  if (gpe_internal_field_view(c, &v)) return GPE_ERR_INVALID;
  const int rc = enqueue_apply(n, v, v.status);
  if (rc || !n->prm.preserve_norm) return rc;
  return gpe_internal_restore_norm(c);
}

// Training-path forward into d_delta (keeps T1..T3, P0..P2).
int enqueue_train_forward(gpe_cnn* n, const FieldView& v) {
  int rc = pack_input(n, v, n->T[0]);
  if (rc) return rc;
  for (int l = 0; l < 3; l++) {
    ConvParams p;
    memset(&p, 0, sizeof(p));
    p.act_out = n->T[l + 1].p;
    p.pre_out = n->P[l].p;
    if ((rc = launch_conv<EPI_GELU_PRE>(n, v.stream, n->T[l], l, false, p))) return rc;
  }
  ConvParams p;
  memset(&p, 0, sizeof(p));
  p.delta = n->d_delta;
  return launch_conv<EPI_DELTA>(n, v.stream, n->T[3], 3, false, p);
}

// Loss and gradients into d_grad (weights then biases); loss partials in d_lpart.
int enqueue_backward(gpe_cnn* n, const FieldView& v, const void* target, int eb) {
  const int nb = n->ew_blocks;
  if (eb == 8)
    loss_kernel<float, float><<<nb, 256, 0, v.stream>>>(
        n->d_delta, static_cast<const float*>(v.psi), v.Nx, v.Ny,
        static_cast<const float*>(target), n->nx, n->ny, n->nz, n->prm.out_scale, n->GA.p,
        n->d_lpart);
  else
    loss_kernel<float, double><<<nb, 256, 0, v.stream>>>(
        n->d_delta, static_cast<const float*>(v.psi), v.Nx, v.Ny,
        static_cast<const double*>(target), n->nx, n->ny, n->nz, n->prm.out_scale, n->GA.p,
        n->d_lpart);
  CNN_CU(n, cudaGetLastError());
  n->launches++;
  Act* g = &n->GA;
  Act* other = &n->GB;
  for (int l = 3; l >= 0; l--) {
    int rc = launch_wgrad(n, v.stream, n->T[l], *g);
    if (rc) return rc;
    channel_sum_kernel<<<nb, 256, 0, v.stream>>>(g->p, n->nx, n->ny, n->nz, n->d_bpart);
    CNN_CU(n, cudaGetLastError());
    grad_finalize_kernel<<<(NTAP * 256 + 16 + 255) / 256, 256, 0, v.stream>>>(
        n->d_wpart, n->wgrad_grid, n->d_bpart, nb, n->d_grad + (size_t)l * NTAP * 256,
        n->d_grad + GPE_CNN_WEIGHTS + l * 16);
    CNN_CU(n, cudaGetLastError());
    n->launches += 2;
    if (l > 0) {
      ConvParams p;
      memset(&p, 0, sizeof(p));
      p.act_out = other->p;
      p.pre_in = n->P[l - 1].p;
      if ((rc = launch_conv<EPI_DGELU>(n, v.stream, *g, l, true, p))) return rc;
      std::swap(g, other);
    }
  }
  return GPE_OK;
}

int read_loss(gpe_cnn* n, cudaStream_t st, double* loss) {
  std::vector<double> part(n->ew_blocks);
  CNN_CU(n, cudaMemcpyAsync(part.data(), n->d_lpart, sizeof(double) * part.size(),
                            cudaMemcpyDeviceToHost, st));
  int rc = sync_status(n, st);
  if (rc) return rc;
  double t = 0.0;
  for (double x : part) t += x;
  if (loss) *loss = t / (double)n->nint;
  return GPE_OK;
}

int repack_weights(gpe_cnn* n, cudaStream_t st) {
  pack_weights_kernel<<<(NLAYER * W_TILES * 2 * NSTACK * 8 + 255) / 256, 256, 0, st>>>(n->d_w, n->d_wf, n->d_wt);
  CNN_CU(n, cudaGetLastError());
  pack_out2_kernel<<<(W_TILES * 2 * OutShape<2>::NB * 8 + 255) / 256, 256, 0, st>>>(n->d_w, n->d_wf2);
  CNN_CU(n, cudaGetLastError());
  n->launches += 2;
  return GPE_OK;
}

bool real_weight(int l, int co, int ci) {
  if (l == 0 && ci >= 2) return false;
  if (l == NLAYER - 1 && co >= 2) return false;
  return true;
}

int view_of(gpe_cnn* n, gpe_ctx* ctx, FieldView* v) {
  if (!ctx || gpe_internal_field_view(ctx, v)) return cfail(n, GPE_ERR_INVALID, "bad context");
  int rc = check_view(n, *v);
  if (rc) return rc;
  CNN_CU(n, cudaSetDevice(n->dev));
  return GPE_OK;
}

}  // namespace

extern "C" {

void gpe_cnn_default_params(gpe_cnn_params* p, int32_t nx, int32_t ny, int32_t nz) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->struct_size = (int32_t)sizeof(gpe_cnn_params);
  p->nx = nx;
  p->ny = ny;
  p->nz = nz;
  p->out_scale = 0.01f;
}

int gpe_cnn_create(const gpe_cnn_params* p, gpe_cnn** out) {
  if (!p || !out) return cfail(nullptr, GPE_ERR_INVALID, "null argument");
  *out = nullptr;
  if (p->struct_size != (int32_t)sizeof(gpe_cnn_params))
    return cfail(nullptr, GPE_ERR_INVALID, "gpe_cnn_params struct_size mismatch");
  if (p->nx < 16 || p->nx > 128 || p->nx % 16 != 0)
    return cfail(nullptr, GPE_ERR_INVALID, "nx must be a multiple of 16 in [16, 128]");
  if (p->ny < 1 || p->nz < 1) return cfail(nullptr, GPE_ERR_INVALID, "ny, nz must be >= 1");
  if (!(std::isfinite(p->out_scale) && p->out_scale != 0.f))
    return cfail(nullptr, GPE_ERR_INVALID, "out_scale must be finite and non-zero");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return cfail(nullptr, GPE_ERR_NODEVICE, "no CUDA device");
  }
  if (p->device < 0 || p->device >= ndev) return cfail(nullptr, GPE_ERR_INVALID, "bad device");
  gpe_cnn* n = new gpe_cnn();
  n->prm = *p;
  n->dev = p->device;
  n->nx = p->nx; n->ny = p->ny; n->nz = p->nz;
  n->Xp = n->nx + 2; n->Yp = n->ny + 2; n->Zp = n->nz + 2;
  n->nint = (size_t)n->nx * n->ny * n->nz;
  auto bail = [&](int rc) {
    g_cnn_error = n->err;
    gpe_cnn_destroy(n);
    return rc;
  };
  if (cudaSetDevice(n->dev) != cudaSuccess) {
    n->err = "cudaSetDevice failed";
    return bail(GPE_ERR_CUDA);
  }
  cudaDeviceGetAttribute(&n->num_sms, cudaDevAttrMultiProcessorCount, n->dev);
  int maj = 0;
  cudaDeviceGetAttribute(&maj, cudaDevAttrComputeCapabilityMajor, n->dev);
  if (maj != 10) {
    n->err = "the tcgen05 kernels need an sm_100 device";
    return bail(GPE_ERR_NODEVICE);
  }
  n->ew_blocks = (int)std::min<size_t>((n->nint + 255) / 256, (size_t)n->num_sms * 8);
  n->hw.assign(GPE_CNN_WEIGHTS, 0.f);
  n->hb.assign(GPE_CNN_BIASES, 0.f);
  const size_t np = GPE_CNN_WEIGHTS + GPE_CNN_BIASES;
  int rc;
  if (cudaMalloc(&n->d_w, sizeof(float) * np) != cudaSuccess ||
      cudaMalloc(&n->d_wf, (size_t)NLAYER * W_TILES * WT_BYTES) != cudaSuccess ||
      cudaMalloc(&n->d_wt, (size_t)NLAYER * W_TILES * WT_BYTES) != cudaSuccess ||
      cudaMalloc(&n->d_wf2, (size_t)W_TILES * OutShape<2>::WTB) != cudaSuccess ||
      cudaMalloc(&n->d_status, sizeof(int)) != cudaSuccess) {
    n->err = "cudaMalloc failed";
    return bail(GPE_ERR_OOM);
  }
  n->d_b = n->d_w + GPE_CNN_WEIGHTS;
  cudaMemset(n->d_w, 0, sizeof(float) * np);
  cudaMemset(n->d_status, 0, sizeof(int));
  if ((rc = alloc_act(n, n->A0, 1)) || (rc = alloc_act(n, n->A1, 2)) ||
      (rc = alloc_act(n, n->A2, 2)))
    return bail(rc);
  if (p->train) {
    for (int l = 0; l < 4; l++)
      if ((rc = alloc_act(n, n->T[l], 2))) return bail(rc);
    for (int l = 0; l < 3; l++)
      if ((rc = alloc_act(n, n->P[l], 2))) return bail(rc);
    if ((rc = alloc_act(n, n->GA, 2)) || (rc = alloc_act(n, n->GB, 2))) return bail(rc);
    n->wgrad_grid = n->num_sms;
    std::vector<unsigned char> mask(np, 1);
    for (int l = 0; l < NLAYER; l++)
      for (int t = 0; t < NTAP; t++)
        for (int co = 0; co < 16; co++)
          for (int ci = 0; ci < 16; ci++)
            mask[((size_t)(l * NTAP + t) * 16 + co) * 16 + ci] = real_weight(l, co, ci);
    for (int co = 2; co < 16; co++) mask[GPE_CNN_WEIGHTS + 3 * 16 + co] = 0;
    if (cudaMalloc(&n->d_delta, sizeof(float) * 2 * n->nint) != cudaSuccess ||
        cudaMalloc(&n->d_wpart, sizeof(float) * n->wgrad_grid * NACC * 128 * 16) != cudaSuccess ||
        cudaMalloc(&n->d_bpart, sizeof(float) * n->ew_blocks * 16) != cudaSuccess ||
        cudaMalloc(&n->d_lpart, sizeof(double) * n->ew_blocks) != cudaSuccess ||
        cudaMalloc(&n->d_grad, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&n->d_m, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&n->d_v, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&n->d_mask, np) != cudaSuccess) {
      n->err = "cudaMalloc of training buffers failed";
      return bail(GPE_ERR_OOM);
    }
    cudaMemset(n->d_m, 0, sizeof(float) * np);
    cudaMemset(n->d_v, 0, sizeof(float) * np);
    cudaMemset(n->d_grad, 0, sizeof(float) * np);
    cudaMemcpy(n->d_mask, mask.data(), np, cudaMemcpyHostToDevice);
  }
  if ((rc = repack_weights(n, 0))) return bail(rc);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    n->err = "device synchronisation failed in gpe_cnn_create";
    return bail(GPE_ERR_CUDA);
  }
  *out = n;
  return GPE_OK;
}

void gpe_cnn_destroy(gpe_cnn* n) {
  if (!n) return;
  cudaSetDevice(n->dev);
  cudaDeviceSynchronize();
  void* ptrs[] = {n->d_w, n->d_wf, n->d_wt, n->d_wf2, n->d_mask, n->d_grad, n->d_m, n->d_v,
                  n->A0.p, n->A1.p, n->A2.p, n->T[0].p, n->T[1].p, n->T[2].p, n->T[3].p,
                  n->P[0].p, n->P[1].p, n->P[2].p, n->GA.p, n->GB.p, n->d_delta,
                  n->d_wpart, n->d_bpart, n->d_lpart, n->d_status};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete n;
}

const char* gpe_cnn_last_error(const gpe_cnn* n) {
  return n ? n->err.c_str() : g_cnn_error.c_str();
}

int gpe_cnn_set_weights(gpe_cnn* n, const float* w, const float* b) {
  if (!n || !w || !b) return cfail(n, GPE_ERR_INVALID, "null argument");
  for (int l = 0; l < NLAYER; l++)
    for (int t = 0; t < NTAP; t++)
      for (int co = 0; co < 16; co++)
        for (int ci = 0; ci < 16; ci++) {
          const size_t i = ((size_t)(l * NTAP + t) * 16 + co) * 16 + ci;
          if (!std::isfinite(w[i])) return cfail(n, GPE_ERR_INVALID, "non-finite weight");
          n->hw[i] = real_weight(l, co, ci) ? w[i] : 0.f;
        }
  for (int l = 0; l < NLAYER; l++)
    for (int c = 0; c < 16; c++) {
      const float v = b[l * 16 + c];
      if (!std::isfinite(v)) return cfail(n, GPE_ERR_INVALID, "non-finite bias");
      n->hb[l * 16 + c] = (l == NLAYER - 1 && c >= 2) ? 0.f : v;
    }
  CNN_CU(n, cudaSetDevice(n->dev));
  CNN_CU(n, cudaMemcpy(n->d_w, n->hw.data(), sizeof(float) * GPE_CNN_WEIGHTS, cudaMemcpyHostToDevice));
  CNN_CU(n, cudaMemcpy(n->d_b, n->hb.data(), sizeof(float) * GPE_CNN_BIASES, cudaMemcpyHostToDevice));
  int rc = repack_weights(n, 0);
  if (rc) return rc;
  CNN_CU(n, cudaDeviceSynchronize());
  return GPE_OK;
}

int gpe_cnn_get_weights(const gpe_cnn* cn, float* w, float* b) {
  gpe_cnn* n = const_cast<gpe_cnn*>(cn);
  if (!n) return cfail(nullptr, GPE_ERR_INVALID, "null network");
  CNN_CU(n, cudaSetDevice(n->dev));
  CNN_CU(n, cudaDeviceSynchronize());
  if (w) CNN_CU(n, cudaMemcpy(w, n->d_w, sizeof(float) * GPE_CNN_WEIGHTS, cudaMemcpyDeviceToHost));
  if (b) CNN_CU(n, cudaMemcpy(b, n->d_b, sizeof(float) * GPE_CNN_BIASES, cudaMemcpyDeviceToHost));
  return GPE_OK;
}

int gpe_cnn_apply(gpe_cnn* n, gpe_ctx* ctx) {
  if (!n) return cfail(nullptr, GPE_ERR_INVALID, "null network");
  FieldView v;
  int rc = view_of(n, ctx, &v);
  if (rc) return rc;
  rc = enqueue_apply(n, v, n->d_status);
  if (rc) return rc;
  return sync_status(n, v.stream);
}

int gpe_cnn_attach(gpe_cnn* n, gpe_ctx* ctx) {
  if (!ctx) return cfail(n, GPE_ERR_INVALID, "null context");
  if (!n) {
    gpe_internal_set_post_step(ctx, nullptr, nullptr);
    return GPE_OK;
  }
  FieldView v;
  int rc = view_of(n, ctx, &v);
  if (rc) return rc;
  gpe_internal_set_post_step(ctx, post_step_hook, n);
  return GPE_OK;
}

int gpe_cnn_delta(gpe_cnn* n, gpe_ctx* ctx, float* delta_dev) {
  if (!n || !delta_dev) return cfail(n, GPE_ERR_INVALID, "null argument");
  if (!n->prm.train) return cfail(n, GPE_ERR_INVALID, "network created without training buffers");
  FieldView v;
  int rc = view_of(n, ctx, &v);
  if (rc) return rc;
  if ((rc = enqueue_train_forward(n, v))) return rc;
  CNN_CU(n, cudaMemcpyAsync(delta_dev, n->d_delta, sizeof(float) * 2 * n->nint,
                            cudaMemcpyDeviceToDevice, v.stream));
  return sync_status(n, v.stream);
}

int gpe_cnn_grad(gpe_cnn* n, gpe_ctx* ctx, const void* target, int32_t eb, double* loss,
                 float* dw, float* db) {
  if (!n || !target || (eb != 8 && eb != 16)) return cfail(n, GPE_ERR_INVALID, "bad argument");
  if (!n->prm.train) return cfail(n, GPE_ERR_INVALID, "network created without training buffers");
  FieldView v;
  int rc = view_of(n, ctx, &v);
  if (rc) return rc;
  if ((rc = enqueue_train_forward(n, v)) || (rc = enqueue_backward(n, v, target, eb))) return rc;
  if ((rc = read_loss(n, v.stream, loss))) return rc;
  if (dw) CNN_CU(n, cudaMemcpy(dw, n->d_grad, sizeof(float) * GPE_CNN_WEIGHTS, cudaMemcpyDeviceToHost));
  if (db)
    CNN_CU(n, cudaMemcpy(db, n->d_grad + GPE_CNN_WEIGHTS, sizeof(float) * GPE_CNN_BIASES,
                         cudaMemcpyDeviceToHost));
  return GPE_OK;
}

int gpe_cnn_train_step(gpe_cnn* n, gpe_ctx* ctx, const void* target, int32_t eb, float lr,
                       double* loss) {
  if (!n || !target || (eb != 8 && eb != 16) || !(lr > 0.f))
    return cfail(n, GPE_ERR_INVALID, "bad argument");
  if (!n->prm.train) return cfail(n, GPE_ERR_INVALID, "network created without training buffers");
  FieldView v;
  int rc = view_of(n, ctx, &v);
  if (rc) return rc;
  if ((rc = enqueue_train_forward(n, v)) || (rc = enqueue_backward(n, v, target, eb))) return rc;
  n->adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - (float)std::pow((double)b1, (double)n->adam_t);
  const float c2 = 1.f - (float)std::pow((double)b2, (double)n->adam_t);
  const int np = GPE_CNN_WEIGHTS + GPE_CNN_BIASES;
  adam_kernel<<<(np + 255) / 256, 256, 0, v.stream>>>(n->d_w, n->d_grad, n->d_m, n->d_v,
                                                       n->d_mask, np, lr, b1, b2, 1e-8f, c1, c2);
  CNN_CU(n, cudaGetLastError());
  n->launches++;
  if ((rc = repack_weights(n, v.stream))) return rc;
  return read_loss(n, v.stream, loss);
}

int gpe_cnn_adam_reset(gpe_cnn* n) {
  if (!n || !n->prm.train) return cfail(n, GPE_ERR_INVALID, "no training state");
  const size_t np = GPE_CNN_WEIGHTS + GPE_CNN_BIASES;
  CNN_CU(n, cudaSetDevice(n->dev));
  CNN_CU(n, cudaMemset(n->d_m, 0, sizeof(float) * np));
  CNN_CU(n, cudaMemset(n->d_v, 0, sizeof(float) * np));
  n->adam_t = 0;
  return GPE_OK;
}

int gpe_cnn_restrict(gpe_ctx* fine, void* coarse, int32_t eb) {
  FieldView v;
  if (!fine || !coarse || (eb != 8 && eb != 16) || gpe_internal_field_view(fine, &v))
    return cfail(nullptr, GPE_ERR_INVALID, "bad argument");
  if (v.nx % 2 || v.ny % 2 || v.nz % 2 || !v.single_domain)
    return cfail(nullptr, GPE_ERR_INVALID, "restriction needs even single-domain grids");
  CNN_CU(nullptr, cudaSetDevice(v.dev));
  const int nxc = v.nx / 2, nyc = v.ny / 2, nzc = v.nz / 2;
  const size_t nc = (size_t)nxc * nyc * nzc;
  const int nb = (int)std::min<size_t>((nc + 255) / 256, 148 * 8);
  if (v.es == 16 && eb == 16)
    restrict_kernel<double, double><<<nb, 256, 0, v.stream>>>(
        (const double*)v.psi, v.Nx, v.Ny, nxc, nyc, nzc, (double*)coarse);
  else if (v.es == 16)
    restrict_kernel<double, float><<<nb, 256, 0, v.stream>>>(
        (const double*)v.psi, v.Nx, v.Ny, nxc, nyc, nzc, (float*)coarse);
  else if (eb == 16)
    restrict_kernel<float, double><<<nb, 256, 0, v.stream>>>(
        (const float*)v.psi, v.Nx, v.Ny, nxc, nyc, nzc, (double*)coarse);
  else
    restrict_kernel<float, float><<<nb, 256, 0, v.stream>>>(
        (const float*)v.psi, v.Nx, v.Ny, nxc, nyc, nzc, (float*)coarse);
  CNN_CU(nullptr, cudaGetLastError());
  CNN_CU(nullptr, cudaStreamSynchronize(v.stream));
  return GPE_OK;
}

int64_t gpe_cnn_launch_count(const gpe_cnn* n) { return n ? n->launches : -1; }

}  // extern "C"
