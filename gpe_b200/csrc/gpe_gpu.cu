// gpe_gpu.cu -- context, stage scheduling and the C-ABI of include/gpe_gpu.h.
//
// One context = one run on one device.  Fields live in a ghost-padded layout
// (2 ghost layers on every axis, x pitch rounded to 4 elements) so that each
// stage kernel reads its stencil plane as one TMA box; ghosts are refreshed by
// the kernel that writes the field (see stage_kernel.cuh), which replaces the
// reference's halo exchange (src/variables.f90:186-358).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "aux_kernels.cuh"
#include "gpe_gpu.h"
#include "internal.h"
#include "stage_kernel.cuh"

using cd = std::complex<double>;
using namespace gpe;

namespace {

// Cash-Karp coefficients (src/solve.f90:255-281).
constexpr double B21 = 0.2;
constexpr double B31 = 0.075, B32 = 0.225;
constexpr double B41 = 0.3, B42 = -0.9, B43 = 1.2;
constexpr double B51 = -11.0 / 54.0, B52 = 2.5, B53 = -70.0 / 27.0,
                 B54 = 35.0 / 27.0;
constexpr double B61 = 1631.0 / 55296.0, B62 = 175.0 / 512.0,
                 B63 = 575.0 / 13824.0, B64 = 44275.0 / 110592.0,
                 B65 = 253.0 / 4096.0;
constexpr double C1 = 37.0 / 378.0, C3 = 250.0 / 621.0, C4 = 125.0 / 594.0,
                 C6 = 512.0 / 1771.0;
constexpr double DC1 = C1 - 2825.0 / 27648.0, DC3 = C3 - 18575.0 / 48384.0,
                 DC4 = C4 - 13525.0 / 55296.0, DC5 = 0.0 - 277.0 / 14336.0,
                 DC6 = C6 - 0.25;
// Adaptive step constants (src/parameters.f90:89-92); dt_decrease (-0.25)
// is applied in rk45_control_kernel.
constexpr double RK_EPS = 1e-6, SAFETY = 0.9,
                 DT_INCREASE = -0.20;
// Extended-Simpson end weights (src/variables.f90:49-51).
constexpr double W1 = 3.0 / 8.0, W2 = 7.0 / 6.0, W3 = 23.0 / 24.0;

constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull;  // 2 s

enum FieldId {
  F_PSI = 0, F_ALT, F_ACC, F_UA, F_UB, F_C, F_CALT,
  F_K1, F_K2, F_K3, F_K4, F_K5, F_COUNT
};

thread_local std::string g_last_create_error;

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

// NCCL, resolved at run time so that the library loads without it and uses
// the libnccl.so.2 already present in the process when there is one.
struct NcclApi {
  bool ok = false;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t,
                       cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t,
                       cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t,
                            ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  const char* (*GetErrorString)(ncclResult_t) = nullptr;
};
NcclApi g_nccl;

bool load_nccl(std::string* why) {
  if (g_nccl.ok) return true;
  void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h) {
    *why = "libnccl.so.2 not found";
    return false;
  }
#define GPE_SYM(field, name)                                             \
  g_nccl.field = reinterpret_cast<decltype(g_nccl.field)>(dlsym(h, name)); \
  if (!g_nccl.field) {                                                   \
    *why = std::string("NCCL symbol missing: ") + name;                  \
    return false;                                                        \
  }
  GPE_SYM(GetUniqueId, "ncclGetUniqueId")
  GPE_SYM(CommInitRank, "ncclCommInitRank")
  GPE_SYM(CommDestroy, "ncclCommDestroy")
  GPE_SYM(Send, "ncclSend")
  GPE_SYM(Recv, "ncclRecv")
  GPE_SYM(AllReduce, "ncclAllReduce")
  GPE_SYM(GroupStart, "ncclGroupStart")
  GPE_SYM(GroupEnd, "ncclGroupEnd")
  GPE_SYM(GetErrorString, "ncclGetErrorString")
#undef GPE_SYM
  g_nccl.ok = true;
  return true;
}

struct LaunchShape {
  int TY, S, zchunk, ntx, nty, nchunks;
  int rows = 1;  // tile rows per compute warp (rows_per_warp of the recipe)
  size_t smem;
  unsigned halo_box, pt_box, halo_smem, pt_smem;
};

struct Launch {
  int family;
  cudaEvent_t a, b;
  int64_t sites;
};

}  // namespace

// Shared with noalloc.cu, which has no context to hold its messages.
void gpe_internal_set_last_error(const std::string& msg) { g_last_create_error = msg; }

struct gpe_ctx {
  gpe_params prm;
  int dev = 0;
  cudaStream_t stream = nullptr;
  int nx, ny, nz, Nx, Ny, Nz;
  int num_sms = 148;
  // z-slab of a global grid (single domain: nzg == nz, z_off == 0)
  int nzg = 0, z_off = 0;
  ncclComm_t comm = nullptr;
  int rank = 0, nranks = 1, nbr_lo = 0, nbr_hi = 0;
  bool exch_lo = false, exch_hi = false;  // z ghosts come from a neighbour
  size_t npad, nint;
  int es;  // bytes per stored complex element (8 or 16)
  double dx, dy, dz;
  std::vector<double> x, y, z;
  void* fld[F_COUNT] = {};
  int psi_id = F_PSI, alt_id = F_ALT, c_id = F_C, calt_id = F_CALT;
  // tables: per axis padded to tab_n entries
  int tab_n[3];
  float* tabVf[3] = {};
  float* tabDf[3] = {};
  double* tabVd[3] = {};
  double* tabDd[3] = {};
  double* tabW[3] = {};
  double* tabX[3] = {};
  void* d_tables = nullptr;
  double* d_partials = nullptr;
  size_t partials_cap = 0;  // CTAs
  double* d_scal = nullptr;  // [0] norm [1] E [2] H4 [3] errmax
  double* d_series = nullptr;
  size_t series_cap = 0;
  int64_t series_steps = 0;  // steps the last rk45 advance recorded
  int* d_counter = nullptr;
  int* d_status = nullptr;
  void* d_stage = nullptr;  // dense staging, nint * 16 bytes
  void* h_pinned = nullptr;
  size_t h_pinned_bytes = 0;
  bool norm_valid = false;
  unsigned long long wait_limit_ns = 2000000000ull;
  int stall_plane = -1;  // failure-detection test hook (gpe_gpu_test_stall)
  int64_t launches = 0;
  int last_nblk = 0;
  int64_t device_bytes = 0;
  std::map<std::tuple<int, int, int, int>, CUtensorMap> maps;
  std::map<const void*, LaunchShape> shapes;
  bool timing = false;
  std::vector<Launch> timed;
  gpe_timing acc_timing;
  std::vector<cudaEvent_t> ev_pool;
  // enqueued after every completed step (the learned correction)
  int (*post_step)(void*, gpe_ctx*) = nullptr;
  void* post_arg = nullptr;
  std::unique_ptr<gpe::Extension> ext[GPE_EXT_SLOTS];
  // member of an in-process slab group (gpe_group_create): the group steps
  // all members on its stream; the context's own stream is kept aside
  gpe_group* group = nullptr;
  cudaStream_t own_stream = nullptr;
  // the ghost exchange overlapping a stage's interior planes (communicator)
  cudaStream_t xstream = nullptr;
  cudaEvent_t xev[2] = {nullptr, nullptr};  // boundary planes done, exchange done
  // rk45 step control on the device: time state, per-step series of the
  // last advance (dt taken, attempts) and one captured step per psi buffer
  gpe::DevTime* d_time = nullptr;
  double* d_ser_dt = nullptr;
  int* d_ser_att = nullptr;
  cudaGraph_t rk_graph[2] = {nullptr, nullptr};
  cudaGraphExec_t rk_exec[2] = {nullptr, nullptr};
  int rk_psi[2] = {-1, -1};  // psi buffer each captured step starts from
  bool ghosts_dirty = false;  // psi loaded alone; its z ghosts await the group
  std::string err;
};

// z-slab contexts of one grid on one device, in z order, stepped together.
struct gpe_group {
  std::vector<gpe_ctx*> m;
  int dev = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t xstream = nullptr;           // ghost copies beside the interiors
  cudaEvent_t xev[2] = {nullptr, nullptr};  // boundary planes done, copies done
  double** d_scal = nullptr;  // the members' d_scal pointers (device array)
  std::string err;
};

void gpe_internal_set_post_step(gpe_ctx* c, int (*fn)(void*, gpe_ctx*), void* arg) {
  if (!c) return;
  c->post_step = fn;
  c->post_arg = arg;
}

int gpe_internal_field_view(gpe_ctx* c, gpe::FieldView* v) {
  if (!c || !v) return GPE_ERR_INVALID;
  v->psi = c->fld[c->psi_id];
  v->nx = c->nx; v->ny = c->ny; v->nz = c->nz; v->Nx = c->Nx; v->Ny = c->Ny;
  v->es = c->es;
  v->bcs = c->prm.bcs;
  v->dev = c->dev;
  v->single_domain = (c->nranks == 1 && c->nzg == c->nz) ? 1 : 0;
  v->stream = c->stream;
  v->status = c->d_status;
  v->dx = c->dx; v->dy = c->dy; v->dz = c->dz;
  v->xr = c->prm.xr; v->yr = c->prm.yr; v->zr = c->prm.zr;
  v->stage = c->d_stage;
  c->norm_valid = false;
  return GPE_OK;
}

std::unique_ptr<gpe::Extension>& gpe_internal_extension(gpe_ctx* c, int slot) {
  return c->ext[slot];
}

void gpe_internal_count_launches(gpe_ctx* c, int64_t n) {
  if (c) c->launches += n;
}

namespace {

int fail(gpe_ctx* c, int code, const std::string& msg) {
  if (c)
    c->err = msg;
  else
    g_last_create_error = msg;
  return code;
}

#define CU_CHECK(c, call)                                                    \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      return fail((c), GPE_ERR_CUDA,                                         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)

size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }

int ensure_encode(gpe_ctx* c) {
  if (g_encode) return GPE_OK;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn,
                                          cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
    return fail(c, GPE_ERR_CUDA, "cuTensorMapEncodeTiled entry point not found");
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return GPE_OK;
}

// kind 0: halo box (64+4) x (TY+2R); kind 1: pointwise box 64 x TY.
int get_map(gpe_ctx* c, int field, int kind, int TY, int R,
            CUtensorMap* out) {
  auto key = std::make_tuple(field, kind, TY, kind == 0 ? R : 0);
  auto it = c->maps.find(key);
  if (it != c->maps.end()) {
    *out = it->second;
    return GPE_OK;
  }
  int rc = ensure_encode(c);
  if (rc) return rc;
  const cuuint64_t W = (cuuint64_t)(c->es / 8);
  cuuint64_t dims[3] = {W * (cuuint64_t)c->Nx, (cuuint64_t)c->Ny,
                        (cuuint64_t)c->Nz};
  cuuint64_t strides[2] = {(cuuint64_t)c->Nx * c->es,
                           (cuuint64_t)c->Nx * c->Ny * c->es};
  cuuint32_t box[3];
  if (kind == 0) {
    box[0] = (cuuint32_t)(W * (TX + 4));
    box[1] = (cuuint32_t)(TY + 2 * R);
  } else {
    box[0] = (cuuint32_t)(W * TX);
    box[1] = (cuuint32_t)TY;
  }
  box[2] = 1;
  cuuint32_t estr[3] = {1, 1, 1};
  CUtensorMap m;
  CUresult r = g_encode(&m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, c->fld[field],
                        dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(c, GPE_ERR_CUDA,
                "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  c->maps[key] = m;
  *out = m;
  return GPE_OK;
}

// ---------------------------------------------------------------------------
// z-slab halo exchange.  The two boundary planes of a stencil field go to
// the z-neighbours' ghost planes: sends "up" (my top planes -> the upper
// neighbour's lower ghosts) then "down", receives "from below" (into my
// lower ghosts) then "from above".  NCCL matches sends and receives per peer
// in issue order, so this order is right for any rank count, including two
// ranks (both neighbours are the same peer) and one rank with periodic
// wrap-around (both neighbours are the rank itself).

#define NCCL_CHECK(c, call)                                                  \
  do {                                                                       \
    ncclResult_t r_ = (call);                                                \
    if (r_ != ncclSuccess)                                                   \
      return fail((c), GPE_ERR_CUDA, std::string(#call) + ": " +             \
                                         g_nccl.GetErrorString(r_));         \
  } while (0)

int exchange_ghosts(gpe_ctx* c, int field, cudaStream_t st = nullptr) {
  if (!c->comm || !(c->exch_lo || c->exch_hi)) return GPE_OK;
  if (!st) st = c->stream;
  const size_t plane = (size_t)c->Nx * c->Ny * (size_t)c->es;  // bytes
  unsigned char* f = static_cast<unsigned char*>(c->fld[field]);
  // padded plane index pz = z + 2
  unsigned char* bottom = f + 2 * plane;                    // z = 0, 1
  unsigned char* top = f + (size_t)c->nz * plane;           // z = nz-2, nz-1
  unsigned char* ghost_lo = f;                              // z = -2, -1
  unsigned char* ghost_hi = f + (size_t)(c->nz + 2) * plane; // z = nz, nz+1
  const size_t n = 2 * plane;
  NCCL_CHECK(c, g_nccl.GroupStart());
  if (c->exch_hi) NCCL_CHECK(c, g_nccl.Send(top, n, ncclUint8, c->nbr_hi, c->comm, st));
  if (c->exch_lo) NCCL_CHECK(c, g_nccl.Send(bottom, n, ncclUint8, c->nbr_lo, c->comm, st));
  if (c->exch_lo) NCCL_CHECK(c, g_nccl.Recv(ghost_lo, n, ncclUint8, c->nbr_lo, c->comm, st));
  if (c->exch_hi) NCCL_CHECK(c, g_nccl.Recv(ghost_hi, n, ncclUint8, c->nbr_hi, c->comm, st));
  NCCL_CHECK(c, g_nccl.GroupEnd());
  return GPE_OK;
}

// Sum (op 0) or max (op 1) of `count` doubles of d_scal across the ranks.
int allreduce_scalars(gpe_ctx* c, int first, int count, int op) {
  if (!c->comm || c->nranks < 2) return GPE_OK;
  NCCL_CHECK(c, g_nccl.AllReduce(c->d_scal + first, c->d_scal + first, (size_t)count,
                                 ncclFloat64, op ? ncclMax : ncclSum, c->comm, c->stream));
  return GPE_OK;
}

// ---------------------------------------------------------------------------
// Stage description, independent of precision.

struct StageSpec {
  int stencil = F_PSI;
  int stencil2 = -1;  // second stencil field: the kernel steps stencil + stencil2
  int np = 0;
  int pt[MAXP] = {0, 0, 0, 0, 0, 0};
  int nout = 0;
  int out[2] = {0, 0};
  int ghost_mask = 0;
  // out[o] = alpha[o]*s0 + alpha2[o]*s1 + sum_q beta[o][q]*P_q + a[o]*f(u),
  // u = s0 (+ s1) the stencil field(s)
  double alpha[2] = {0.0, 0.0};
  double alpha2[2] = {0.0, 0.0};
  double beta[2][MAXP] = {};
  cd a[2] = {cd(0), cd(0)};
  int epi = 0;
  // rkqs error: err = sum_q ce[q]*P_q + cek*f(u)
  double ce[MAXP] = {};
  cd cek = cd(0);
  cd dt0 = cd(0);
  double inv_absdt = 0.0;
  // rk45 with device step control: a[o] = a_mul[o] dt, cek = cek_mul dt,
  // dt and dt0 read from device memory by the kernel
  const double* dyn = nullptr;
  double a_mul[2] = {0.0, 0.0};
  double cek_mul = 0.0;
  int family = GPE_FAM_OTHER;
};

using KernelFn = const void*;

// Ring depth S and tile height TY from the shared-memory budget: as many
// slots (up to 8) as fit two CTAs per SM, as long as that leaves the R + 1
// slots the compute warps hold plus one in flight, else one CTA per SM, else
// TY = 4.  (Two CTAs with four slots beat one CTA with eight on the rk4
// last stage at 512^3: 1.30 against 1.49 ms; the second CTA's warps hide
// the first's latency better than a deeper ring.)
LaunchShape ring_shape(int es, int R, int np, int tile_y, int ns = 1, int max_ctas = 2) {
  LaunchShape s{};
  int TY = tile_y > 0 ? tile_y : 8;
  for (int attempt = 0; attempt < 2; attempt++) {
    s.TY = TY;
    s.halo_box = (unsigned)((TX + 4) * (TY + 2 * R) * es);
    s.pt_box = (unsigned)(TX * TY * es);
    s.halo_smem = (unsigned)round_up(s.halo_box, 128);
    s.pt_smem = (unsigned)round_up(s.pt_box, 128);
    const size_t stage = (size_t)ns * s.halo_smem + (size_t)np * s.pt_smem;
    if (max_ctas >= 3) {
      // three CTAs per SM when their rings still keep two planes in flight
      const int S3 = (int)std::min<size_t>(8, (72 * 1024 - 128) / stage);
      if (S3 >= R + 3) {
        s.S = S3;
        break;
      }
    }
    int S = (int)std::min<size_t>(8, (110 * 1024 - 128) / stage);
    if (S < R + 2) S = (int)std::min<size_t>(8, (220 * 1024 - 128) / stage);
    if (S >= R + 2 || attempt == 1 || tile_y > 0) {
      s.S = std::max(S, R + 2);
      break;
    }
    TY = 4;
  }
  s.smem = 128 + (size_t)s.S * ((size_t)ns * s.halo_smem + (size_t)np * s.pt_smem);
  return s;
}

// Then the
// z-chunking from the kernel's real occupancy: among chunk counts, pick the
// one that minimises (waves of CTAs) x (planes per CTA + pipeline fill),
// which trades the last wave's idle SMs against the R extra halo planes and
// the fill latency every chunk pays.
int choose_shape(gpe_ctx* c, KernelFn fn, int R, int np, int ns, bool occ3, LaunchShape* out) {
  auto hit = c->shapes.find(fn);
  if (hit != c->shapes.end()) {
    *out = hit->second;
    return GPE_OK;
  }
  // occ3_recipe: complex64 stencil-only recipes are built for 3 CTAs/SM (the
  // energy recipe computes in FP64 and is not one of them)
  const int max_ctas = occ3 ? 3 : 2;
  LaunchShape s = ring_shape(c->es, R, np, c->prm.tile_y, ns, max_ctas);
  s.rows = (occ3 && ns == 2) ? 2 : 1;  // rows_per_warp of the occ3 recipes
  s.ntx = (c->nx + TX - 1) / TX;
  s.nty = (c->ny + s.TY - 1) / s.TY;
  CU_CHECK(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)s.smem));
  int occ = 0;
  CU_CHECK(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 32 * (s.TY / s.rows + 1),
                                                            s.smem));
  if (occ < 1) return fail(c, GPE_ERR_INVALID, "stage kernel cannot be resident");
  const long slots = (long)occ * c->num_sms;
  const long ntiles = (long)s.ntx * s.nty;
  int zc = c->prm.zchunk;
  if (zc <= 0) {
    double best = 1e300;
    const int nmax = std::min(c->nz, 256);
    for (int n = 1; n <= nmax; n++) {
      const int z = (c->nz + n - 1) / n;
      const long nch = (c->nz + z - 1) / z;
      const long waves = (ntiles * nch + slots - 1) / slots;
      const double cost = (double)waves * (double)(z + R + 3);
      if (cost < best - 1e-9) {
        best = cost;
        zc = z;
      }
    }
  }
  s.zchunk = zc;
  s.nchunks = (c->nz + zc - 1) / zc;
  c->shapes[fn] = s;
  *out = s;
  return GPE_OK;
}

// The stage recipes that the schemes use; see stage_kernel.cuh for the
// meaning of (NP, NOUT, EPI, AMASK, BMASK).  BMASK bit o*8+q: beta[o][q] != 0.
// The recipes built for three CTAs per SM (stage_kernel_occ3): complex64
// single-run stages that stage only stencil planes.
template <typename TS, typename TC>
constexpr bool occ3_recipe(int np, bool full, bool batch) {
  return std::is_same<TS, float>::value && std::is_same<TC, float>::value && np == 0 && !full &&
         !batch;
}

// The entry of one recipe (only that one is instantiated).
template <typename TS, typename TC, int R, int NS, int NP, int NOUT, int EPI, int AM, int BM,
          int FORM, bool BATCH>
KernelFn kernel_for() {
  if constexpr (rows_per_warp<TS, TC>(R, NS, NP, FORM, BATCH) == 2)
    return reinterpret_cast<KernelFn>(
        &stage_kernel_rows2<TS, TC, R, NS, NP, NOUT, EPI, AM, BM, FORM, BATCH>);
  else if constexpr (occ3_recipe<TS, TC>(NP, FORM == FORM_FULL, BATCH))
    return reinterpret_cast<KernelFn>(
        &stage_kernel_occ3<TS, TC, R, NS, NP, NOUT, EPI, AM, BM, FORM, BATCH>);
  else
    return reinterpret_cast<KernelFn>(
        &stage_kernel<TS, TC, R, NS, NP, NOUT, EPI, AM, BM, FORM, BATCH>);
}

// FORM_TRAP recipes exist for rk4 only; the other schemes step a trap with
// the FORM_FULL recipes (nullptr here, and the caller falls back).
template <typename TS, typename TC, int R, int FORM, bool BATCH>
KernelFn pick_kernel(int ns, int np, int nout, int epi, int am, int bm) {
#define GPE_CASE(NS_, NP_, NOUT_, EPI_, AM_, BM_)                                      \
  if (ns == NS_ && np == NP_ && nout == NOUT_ && epi == (EPI_) && am == AM_ && bm == BM_) \
    return kernel_for<TS, TC, R, NS_, NP_, NOUT_, (EPI_), AM_, BM_, FORM, BATCH>();
  if constexpr (BATCH) {
    // batched ensembles step with rk4
    if constexpr (std::is_same<TS, TC>::value) {
      GPE_CASE(1, 0, 1, 0, 0, 0)                   // rk4 stage 1
      GPE_CASE(2, 0, 1, 0, 0, 0)                   // rk4 stages 2, 3
      GPE_CASE(2, 2, 1, EPI_NORM, 5, 0x3)          // rk4 stage 4
      if constexpr (std::is_same<TS, float>::value) {
        GPE_CASE(2, 3, 2, EPI_KAHAN | EPI_NORM, 4, 0x3)   // rk4 stage 4 (compensated)
      }
    }
  } else if constexpr (FORM == FORM_TRAP) {
    if constexpr (std::is_same<TS, TC>::value) {
      GPE_CASE(1, 0, 1, 0, 0, 0)                   // rk4 stage 1, get_rhs
      GPE_CASE(2, 0, 1, 0, 0, 0)                   // rk4 stages 2, 3
      GPE_CASE(2, 2, 1, EPI_NORM, 5, 0x3)          // rk4 stage 4
      if constexpr (std::is_same<TS, float>::value) {
        GPE_CASE(2, 3, 2, EPI_KAHAN | EPI_NORM, 4, 0x3)   // rk4 stage 4 (compensated)
      }
    }
  } else {
  if constexpr (std::is_same<TC, double>::value && FORM == FORM_PLAIN) {
    GPE_CASE(1, 0, 0, EPI_ENERGY, 0, 0)
  }
  if constexpr (std::is_same<TS, TC>::value) {
    GPE_CASE(1, 0, 1, EPI_NORM, 1, 0)            // euler
    GPE_CASE(1, 0, 1, 0, 1, 0)                   // rk2 stage 1
    GPE_CASE(1, 1, 1, EPI_NORM, 0, 0x1)          // rk2 stage 2
    GPE_CASE(1, 0, 1, 0, 0, 0)                   // rk4 stage 1, get_rhs
    GPE_CASE(2, 0, 1, 0, 0, 0)                   // rk4 stages 2, 3
    GPE_CASE(2, 2, 1, EPI_NORM, 5, 0x3)          // rk4 stage 4
    GPE_CASE(1, 0, 2, 0, 2, 0)                   // rkck stage 1
    GPE_CASE(1, 2, 2, 0, 0, 0x300)               // rkck stage 2
    GPE_CASE(1, 3, 2, 0, 0, 0x700)               // rkck stage 3
    GPE_CASE(1, 4, 2, 0, 0, 0xF00)               // rkck stage 4
    GPE_CASE(1, 5, 2, 0, 0, 0x1F00)              // rkck stage 5
    GPE_CASE(1, 5, 1, EPI_NORM | EPI_ERR, 0, 0xF)  // rkck stage 6
    if constexpr (FORM == FORM_PLAIN) {
      GPE_CASE(1, 0, 1, EPI_LAP, 0, 0)           // laplacian
    }
    if constexpr (std::is_same<TS, float>::value) {
      GPE_CASE(1, 1, 2, EPI_KAHAN | EPI_NORM, 0, 0)       // euler (compensated)
      GPE_CASE(1, 2, 2, EPI_KAHAN | EPI_NORM, 0, 0)       // rk2 stage 2
      GPE_CASE(2, 3, 2, EPI_KAHAN | EPI_NORM, 4, 0x3)     // rk4 stage 4
      GPE_CASE(1, 6, 2, EPI_KAHAN | EPI_NORM | EPI_ERR, 0, 0xE)  // rkck stage 6
    }
  }
  }
#undef GPE_CASE
  return nullptr;
}

cudaEvent_t pool_event(gpe_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void fill_rhs_coeffs(const gpe_ctx* c, double& ar0, double& ard, double& ai,
                     double& cL, double& c0, double& cV, double& cn,
                     double& U, int& use_diss, int& use_V, int& use_sphere,
                     int& use_grad) {
  const gpe_params& p = c->prm;
  // f = m * ( A*(cL*L + (c0 + cV*V + cn*|u|^2) u) + U*u_x ), A = ar + i ai
  // (src/solve.f90:414-437)
  ar0 = 0; ard = 0; ai = 1; cL = 1; c0 = 0; cV = 0; cn = -1; U = 0;
  use_diss = 0; use_V = 0; use_sphere = 0; use_grad = 0;
  switch (p.eqn_to_solve) {
    case 1:
    case 3:
      ai = 0.5; ard = 0.5; cL = 1; c0 = 1; cn = -1; U = p.Urhs;
      use_diss = p.diss_amp != 0.0;
      use_grad = p.Urhs != 0.0;
      use_sphere = p.eqn_to_solve == 3;
      break;
    case 2:
      ai = 1; cL = 1; c0 = 0; cn = -1; U = p.Urhs;
      use_grad = p.Urhs != 0.0;
      break;
    default:  // 4
      ai = 1; cL = 0.5; c0 = p.mu; cV = -1; cn = -p.g;
      use_V = (p.omx != 0.0 || p.omy != 0.0 || p.omz != 0.0);
      break;
  }
}

// The right-hand side coefficients of a context, in the form the kernels
// take: without sponge, gradient or sphere terms
// f = i*ai*(cL*L + (c0 + cV*V + cn|u|^2)u); the kernel forms K = ai*(...) and
// the factor i moves into the output coefficients (`fold`), with the trap
// (`trap`, FORM_TRAP recipes) or without it.
struct RhsForm {
  double ar0, ard, ai, cL, c0, cV, cn, U;
  int ud, uv, us, ug;
  bool full, trap;
};

RhsForm rhs_form(const gpe_ctx* c) {
  RhsForm f;
  fill_rhs_coeffs(c, f.ar0, f.ard, f.ai, f.cL, f.c0, f.cV, f.cn, f.U, f.ud, f.uv, f.us, f.ug);
  f.full = f.ud || f.us || f.ug;
  f.trap = f.uv && !f.full;
  return f;
}

int form_of(const RhsForm& f) {
  return f.full ? FORM_FULL : f.trap ? FORM_TRAP : FORM_PLAIN;
}

// Recipe bit masks of a stage (see stage_kernel.cuh).
void recipe_masks(const StageSpec& sp, int* am, int* bm) {
  *am = 0;
  *bm = 0;
  for (int o = 0; o < sp.nout; o++) {
    if (sp.alpha[o] != 0.0) *am |= 1 << o;
    if (sp.alpha2[o] != 0.0) *am |= 4 << o;
    for (int q = 0; q < sp.np; q++)
      if (sp.beta[o][q] != 0.0) *bm |= 1 << (o * 8 + q);
  }
}

// Per-run part of a stage launch.
template <typename TS, typename TC>
int fill_run(gpe_ctx* c, const StageSpec& sp, int R, const LaunchShape& sh,
             RhsForm f, RunDesc<TS, TC>* rd, int force_full = -1) {
  if (force_full >= 0) f.full = force_full != 0;
  memset(rd, 0, sizeof(*rd));
  int rc = get_map(c, sp.stencil, 0, sh.TY, R, &rd->maps.halo);
  if (rc) return rc;
  if (sp.stencil2 >= 0) {
    rc = get_map(c, sp.stencil2, 0, sh.TY, R, &rd->maps.halo2);
    if (rc) return rc;
  }
  for (int q = 0; q < sp.np; q++) {
    rc = get_map(c, sp.pt[q], 1, sh.TY, R, &rd->maps.pt[q]);
    if (rc) return rc;
  }
  rd->nx = c->nx; rd->ny = c->ny; rd->nz = c->nz; rd->Nx = c->Nx; rd->Ny = c->Ny;
  rd->ntx = sh.ntx; rd->nty = sh.nty; rd->zchunk = sh.zchunk; rd->nchunks = sh.nchunks;
  rd->bcs = c->prm.bcs;
  rd->zg_lo = c->exch_lo ? 0 : 1;
  rd->zg_hi = c->exch_hi ? 0 : 1;
  rd->stencil = static_cast<const TS*>(c->fld[sp.stencil]);
  rd->stencil2 = sp.stencil2 >= 0 ? static_cast<const TS*>(c->fld[sp.stencil2]) : nullptr;
  for (int o = 0; o < sp.nout; o++) rd->out[o] = static_cast<TS*>(c->fld[sp.out[o]]);
  const double h2[3] = {c->dx * c->dx, c->dy * c->dy, c->dz * c->dz};
  double c1[3], c2[3];
  const double r2 = c->prm.fd_match * c->prm.fd_match;
  for (int a = 0; a < 3; a++) {
    if (R == 1) { c1[a] = 1.0 / h2[a]; c2[a] = 0.0; }
    else if (c->prm.fd_match > 0.0) {
      c1[a] = (4.0 - r2) / (3.0 * h2[a]);
      c2[a] = (r2 - 1.0) / (12.0 * h2[a]);
    } else { c1[a] = 16.0 / (12.0 * h2[a]); c2[a] = -1.0 / (12.0 * h2[a]); }
  }
  rd->cx1 = (TC)c1[0]; rd->cx2 = (TC)c2[0];
  rd->cy1 = (TC)c1[1]; rd->cy2 = (TC)c2[1];
  rd->cz1 = (TC)c1[2]; rd->cz2 = (TC)c2[2];
  rd->c0lap = (TC)(-2.0 * (c1[0] + c2[0] + c1[1] + c2[1] + c1[2] + c2[2]));
  if (R == 1) { rd->gx1 = (TC)(1.0 / (2.0 * c->dx)); rd->gx2 = (TC)0; }
  else { rd->gx1 = (TC)(8.0 / (12.0 * c->dx)); rd->gx2 = (TC)(-1.0 / (12.0 * c->dx)); }
  const double sc = f.full ? 1.0 : f.ai;
  rd->ar0 = (TC)f.ar0; rd->ard = (TC)f.ard; rd->ai = (TC)f.ai; rd->cL = (TC)(sc * f.cL);
  rd->c0 = (TC)(sc * f.c0); rd->cV = (TC)(sc * f.cV); rd->cn = (TC)(sc * f.cn); rd->U = (TC)f.U;
  rd->use_diss = f.ud; rd->use_V = f.uv; rd->use_sphere = f.us; rd->use_grad = f.ug;
  for (int a = 0; a < 3; a++) {
    if (std::is_same<TC, float>::value) {
      rd->tabV[a] = reinterpret_cast<const TC*>(c->tabVf[a]);
      rd->tabD[a] = reinterpret_cast<const TC*>(c->tabDf[a]);
    } else {
      rd->tabV[a] = reinterpret_cast<const TC*>(c->tabVd[a]);
      rd->tabD[a] = reinterpret_cast<const TC*>(c->tabDd[a]);
    }
    rd->tabW[a] = c->tabW[a];
    rd->tabX[a] = c->tabX[a];
  }
  rd->eg = c->prm.g;
  rd->emu = c->prm.mu;
  return GPE_OK;
}

// Per-launch part (recipe coefficients, ring shape).
template <typename TS, typename TC>
void fill_common(const StageSpec& sp, bool fold, const LaunchShape& sh,
                 StageParams<TS, TC>* p) {
  const cd I(0.0, 1.0);
  p->TY = sh.TY;
  p->stages = sh.S;
  p->halo_box_bytes = sh.halo_box; p->pt_box_bytes = sh.pt_box;
  p->halo_smem_bytes = sh.halo_smem; p->pt_smem_bytes = sh.pt_smem;
  p->ghost_mask = sp.ghost_mask;
  for (int o = 0; o < 2; o++) {
    p->alpha[o] = (TC)sp.alpha[o];
    p->alpha2[o] = (TC)sp.alpha2[o];
    const cd a = fold ? I * sp.a[o] : sp.a[o];
    p->a_r[o] = (TC)a.real(); p->a_i[o] = (TC)a.imag();
    for (int q = 0; q < MAXP; q++) p->beta[o][q] = (TC)sp.beta[o][q];
  }
  for (int q = 0; q < MAXP; q++) p->ce[q] = sp.ce[q];
  const cd cek = fold ? I * sp.cek : sp.cek;
  p->cek_r = cek.real(); p->cek_i = cek.imag();
  p->dt0_r = sp.dt0.real(); p->dt0_i = sp.dt0.imag();
  p->inv_absdt = sp.inv_absdt;
  p->dyn = sp.dyn;
  p->a_mul[0] = sp.a_mul[0];
  p->a_mul[1] = sp.a_mul[1];
  p->cek_mul = sp.cek_mul;
  p->fold = fold ? 1 : 0;
  p->wait_limit_ns = WAIT_LIMIT_NS;
  p->stall_plane = -1;
}

template <typename TS, typename TC, int R, bool BATCH>
KernelFn select_form(int form, const StageSpec& sp, int am, int bm) {
  const int ns = sp.stencil2 >= 0 ? 2 : 1;
  if (form == FORM_FULL)
    return pick_kernel<TS, TC, R, FORM_FULL, BATCH>(ns, sp.np, sp.nout, sp.epi, am, bm);
  if (form == FORM_TRAP)
    return pick_kernel<TS, TC, R, FORM_TRAP, BATCH>(ns, sp.np, sp.nout, sp.epi, am, bm);
  return pick_kernel<TS, TC, R, FORM_PLAIN, BATCH>(ns, sp.np, sp.nout, sp.epi, am, bm);
}

// The kernel of a stage in right-hand-side form *form; a trap recipe that
// has no FORM_TRAP build steps with FORM_FULL (and *form says so).
template <typename TS, typename TC, bool BATCH>
KernelFn select_kernel(int R, int* form, const StageSpec& sp, int am, int bm) {
  for (;;) {
    KernelFn fn = R == 1 ? select_form<TS, TC, 1, BATCH>(*form, sp, am, bm)
                         : select_form<TS, TC, 2, BATCH>(*form, sp, am, bm);
    if (fn || *form != FORM_TRAP) return fn;
    *form = FORM_FULL;
  }
}

// part 0: the whole slab; part 1: its boundary planes z = 0, 1 and nz-2,
// nz-1 (the planes the z-neighbours' ghosts take); part 2: the planes
// between them.  Parts 1 and 2 write their per-CTA partials one after the
// other, so a finalize after part 2 reduces both.
template <typename TS, typename TC>
int launch_stage_t(gpe_ctx* c, const StageSpec& sp, int part) {
  const int R = c->prm.order / 2;
  const RhsForm f = rhs_form(c);
  const bool special = (sp.epi & (EPI_LAP | EPI_ENERGY)) != 0;
  int form = special ? FORM_PLAIN : form_of(f);
  int am, bm;
  recipe_masks(sp, &am, &bm);
  KernelFn fn = select_kernel<TS, TC, false>(R, &form, sp, am, bm);
  if (!fn) return fail(c, GPE_ERR_INVALID, "no kernel for this stage shape");
  const bool fold = form != FORM_FULL && !special;
  LaunchShape sh;
  int rc = choose_shape(c, fn, R, sp.np, sp.stencil2 >= 0 ? 2 : 1,
                        occ3_recipe<TS, TC>(sp.np, form == FORM_FULL, false), &sh);
  if (rc) return rc;
  StageParams<TS, TC> p;
  memset(&p, 0, sizeof(p));
  rc = fill_run<TS, TC>(c, sp, R, sh, f, &p.run, special ? -1 : (form == FORM_FULL ? 1 : 0));
  if (rc) return rc;
  fill_common<TS, TC>(sp, fold, sh, &p);
  p.wait_limit_ns = c->wait_limit_ns;
  p.stall_plane = c->stall_plane;
  p.status = c->d_status;
  int nchunks = sh.nchunks, planes = c->nz;
  size_t first_blk = 0;
  p.zr[0] = 0; p.zr[1] = c->nz; p.zr[2] = p.zr[3] = 0;
  if (part == 1) {
    p.run.zchunk = 2;
    p.zr[1] = 2; p.zr[2] = c->nz - 2; p.zr[3] = c->nz;
    nchunks = 2;
    planes = 4;
  } else if (part == 2) {
    p.zr[0] = 2; p.zr[1] = c->nz - 2;
    planes = c->nz - 4;
    nchunks = (planes + sh.zchunk - 1) / sh.zchunk;
    first_blk = (size_t)c->last_nblk;
  }
  p.nch_a = part == 1 ? 1 : nchunks;
  const size_t nblk = (size_t)sh.ntx * sh.nty * nchunks;
  if (first_blk + nblk > c->partials_cap)
    return fail(c, GPE_ERR_INVALID, "partials buffer too small");
  p.partials = c->d_partials + 2 * first_blk;
  p.nitems = (int)nblk;
  dim3 grid((unsigned)nblk, 1, 1);
  dim3 block(32, (unsigned)(sh.TY / sh.rows) + 1, 1);
  void* args[] = {&p};
  Launch L{};
  if (c->timing) {
    L.family = sp.family;
    L.a = pool_event(c);
    L.b = pool_event(c);
    L.sites = (int64_t)c->nx * c->ny * planes;
    cudaEventRecord(L.a, c->stream);
  }
  CU_CHECK(c, cudaLaunchKernel(fn, grid, block, args, sh.smem, c->stream));
  if (c->timing) {
    cudaEventRecord(L.b, c->stream);
    c->timed.push_back(L);
  }
  c->launches++;
  c->last_nblk = (int)(first_blk + nblk);
  return GPE_OK;
}

}  // namespace

namespace {

int launch_stage_one(gpe_ctx* c, const StageSpec& sp, int part = 0) {
  if (sp.epi & EPI_ENERGY) {
    if (c->es == 8) return launch_stage_t<float, double>(c, sp, part);
    return launch_stage_t<double, double>(c, sp, part);
  }
  if (c->es == 8) return launch_stage_t<float, float>(c, sp, part);
  return launch_stage_t<double, double>(c, sp, part);
}

// Copies of the two boundary planes of `field` into the z-neighbours' ghost
// planes for every member of a slab group (the in-process form of
// exchange_ghosts: the same planes, moved by cudaMemcpyAsync on the group's
// stream after every member's kernel of the stage).
int group_exchange(gpe_group* g, int field, cudaStream_t st = nullptr) {
  if (!st) st = g->stream;
  const int n = (int)g->m.size();
  for (int r = 0; r < n; r++) {
    gpe_ctx* c = g->m[r];
    const size_t plane = (size_t)c->Nx * c->Ny * (size_t)c->es;
    unsigned char* f = static_cast<unsigned char*>(c->fld[field]);
    if (c->exch_lo) {
      const gpe_ctx* lo = g->m[c->nbr_lo];
      const unsigned char* src = static_cast<const unsigned char*>(lo->fld[field]) +
                                 (size_t)lo->nz * plane;  // its z = nz-2, nz-1
      CU_CHECK(c, cudaMemcpyAsync(f, src, 2 * plane, cudaMemcpyDeviceToDevice, st));
    }
    if (c->exch_hi) {
      const gpe_ctx* hi = g->m[c->nbr_hi];
      const unsigned char* src = static_cast<const unsigned char*>(hi->fld[field]) +
                                 2 * plane;  // its z = 0, 1
      CU_CHECK(c, cudaMemcpyAsync(f + (size_t)(c->nz + 2) * plane, src, 2 * plane,
                                  cudaMemcpyDeviceToDevice, st));
    }
  }
  return GPE_OK;
}

// The boundary planes go first when a stage's ghosts cross to a neighbour
// and the slab is deep enough: the exchange then runs on the side stream
// while the interior planes are computed, and the next stage waits for it.
// Not inside a stream capture (the rk45 step graphs keep one stream).
bool split_stage(const gpe_ctx* c) {
  if (c->nz < 8) return false;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(c->stream, &cs) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return cs == cudaStreamCaptureStatusNone;
}

// Side stream and the two events of the split form, made on first use.
int ensure_side(gpe_ctx* c, cudaStream_t* xs, cudaEvent_t* ev) {
  if (!*xs && cudaStreamCreateWithFlags(xs, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    *xs = nullptr;
    return fail(c, GPE_ERR_CUDA, "side stream creation failed");
  }
  for (int k = 0; k < 2; k++)
    if (!ev[k] && cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      ev[k] = nullptr;
      return fail(c, GPE_ERR_CUDA, "event creation failed");
    }
  return GPE_OK;
}

// One stage: on a single context, or on every member of its slab group
// followed by the group's ghost exchange; the z ghosts of a context with a
// communicator go to its neighbours through NCCL.
int launch_stage(gpe_ctx* c, const StageSpec& sp) {
  bool ghosts = false;
  for (int o = 0; o < sp.nout; o++) ghosts = ghosts || (sp.ghost_mask & (1 << o));
  if (c->group) {
    gpe_group* g = c->group;
    bool split = ghosts;
    for (gpe_ctx* m : g->m) split = split && split_stage(m);
    if (split) {
      const int rc = ensure_side(c, &g->xstream, g->xev);
      if (rc) return rc;
    }
    for (gpe_ctx* m : g->m) {
      const int rc = launch_stage_one(m, sp, split ? 1 : 0);
      if (rc) return fail(c, rc, m->err);
    }
    if (split) {
      CU_CHECK(c, cudaEventRecord(g->xev[0], g->stream));
      CU_CHECK(c, cudaStreamWaitEvent(g->xstream, g->xev[0], 0));
    }
    for (int o = 0; o < sp.nout; o++)
      if (sp.ghost_mask & (1 << o)) {
        const int rc = group_exchange(g, sp.out[o], split ? g->xstream : g->stream);
        if (rc) return rc;
      }
    if (split) {
      CU_CHECK(c, cudaEventRecord(g->xev[1], g->xstream));
      for (gpe_ctx* m : g->m) {
        const int rc = launch_stage_one(m, sp, 2);
        if (rc) return fail(c, rc, m->err);
      }
      CU_CHECK(c, cudaStreamWaitEvent(g->stream, g->xev[1], 0));
    }
    return GPE_OK;
  }
  const bool split = ghosts && c->comm && (c->exch_lo || c->exch_hi) && split_stage(c);
  int rc = split ? ensure_side(c, &c->xstream, c->xev) : GPE_OK;
  if (rc) return rc;
  rc = launch_stage_one(c, sp, split ? 1 : 0);
  if (rc) return rc;
  if (split) {
    CU_CHECK(c, cudaEventRecord(c->xev[0], c->stream));
    CU_CHECK(c, cudaStreamWaitEvent(c->xstream, c->xev[0], 0));
  }
  for (int o = 0; o < sp.nout; o++)
    if (sp.ghost_mask & (1 << o)) {
      rc = exchange_ghosts(c, sp.out[o], split ? c->xstream : c->stream);
      if (rc) return rc;
    }
  if (split) {
    CU_CHECK(c, cudaEventRecord(c->xev[1], c->xstream));
    rc = launch_stage_one(c, sp, 2);
    if (rc) return rc;
    CU_CHECK(c, cudaStreamWaitEvent(c->stream, c->xev[1], 0));
  }
  return GPE_OK;
}

// psi and its spare buffer (and the Kahan pair) trade roles on a context or
// on every member of its group.
void swap_psi(gpe_ctx* c) {
  if (c->group) {
    for (gpe_ctx* m : c->group->m) std::swap(m->psi_id, m->alt_id);
  } else {
    std::swap(c->psi_id, c->alt_id);
  }
}
void swap_comp(gpe_ctx* c) {
  if (c->group) {
    for (gpe_ctx* m : c->group->m) std::swap(m->c_id, m->calt_id);
  } else {
    std::swap(c->c_id, c->calt_id);
  }
}

Geom geom(const gpe_ctx* c) {
  Geom g;
  g.nx = c->nx; g.ny = c->ny; g.nz = c->nz; g.Nx = c->Nx; g.Ny = c->Ny;
  g.bcs = c->prm.bcs;
  g.zg_lo = c->exch_lo ? 0 : 1;
  g.zg_hi = c->exch_hi ? 0 : 1;
  return g;
}

int elementwise_blocks(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)std::min<size_t>(b, 148 * 16);
}

void begin_timed(gpe_ctx* c, Launch& L, int family, int64_t sites) {
  if (!c->timing) return;
  L.family = family;
  L.a = pool_event(c);
  L.b = pool_event(c);
  L.sites = sites;
  cudaEventRecord(L.a, c->stream);
}
void end_timed(gpe_ctx* c, Launch& L) {
  if (!c->timing) return;
  cudaEventRecord(L.b, c->stream);
  c->timed.push_back(L);
}

// partials -> d_scal[slot_out] (and optionally the per-step series).
int finalize_one(gpe_ctx* c, int nblk, int slot, int op, double scale,
                 int out_index, bool series) {
  Launch L{};
  begin_timed(c, L, GPE_FAM_REDUCE, 0);
  finalize_kernel<<<1, 1024, 0, c->stream>>>(
      c->d_partials, nblk, slot, op, scale, c->d_scal + out_index,
      series ? c->d_series : nullptr, c->d_counter);
  CU_CHECK(c, cudaGetLastError());
  end_timed(c, L);
  c->launches++;
  return allreduce_scalars(c, out_index, 1, op);
}

// partials -> d_scal[out_index] (sum or max over blocks); in a slab group
// each member reduces its own partials and the members' values are combined
// in member order and written back to every member.
int finalize(gpe_ctx* c, int nblk, int slot, int op, double scale,
             int out_index, bool series) {
  if (!c->group) return finalize_one(c, nblk, slot, op, scale, out_index, series);
  gpe_group* g = c->group;
  for (gpe_ctx* m : g->m) {
    const int rc = finalize_one(m, m->last_nblk, slot, op, scale, out_index, false);
    if (rc) return fail(c, rc, m->err);
  }
  combine_scalars_kernel<<<1, 32, 0, g->stream>>>(g->d_scal, (int)g->m.size(), out_index, op);
  CU_CHECK(c, cudaGetLastError());
  c->launches++;
  return GPE_OK;
}

double cell_volume(const gpe_ctx* c) { return c->dx * c->dy * c->dz; }

int read_scalars(gpe_ctx* c, double* dst, int first, int count) {
  CU_CHECK(c, cudaMemcpyAsync(dst, c->d_scal + first, sizeof(double) * count,
                              cudaMemcpyDeviceToHost, c->stream));
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  return GPE_OK;
}

int check_status_one(gpe_ctx* c) {
  int st = 0;
  CU_CHECK(c, cudaMemcpyAsync(&st, c->d_status, sizeof(int),
                              cudaMemcpyDeviceToHost, c->stream));
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  if (st != 0) {
    cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream);
    return fail(c, GPE_ERR_TIMEOUT,
                "device-side wait limit expired in a stage kernel");
  }
  return GPE_OK;
}

int check_status(gpe_ctx* c) {
  if (!c->group) return check_status_one(c);
  for (gpe_ctx* m : c->group->m) {
    const int rc = check_status_one(m);
    if (rc) return fail(c, rc, m->err);
  }
  return GPE_OK;
}

// --------------------------------------------------------------------------
// Schemes.  Each function enqueues one full step; the fused final-stage norm
// lands in the partials and is finalised into d_scal[0].

int step_euler(gpe_ctx* c, cd dt) {
  StageSpec s;
  s.stencil = c->psi_id;
  s.nout = c->prm.kahan ? 2 : 1;
  s.out[0] = c->alt_id;
  s.ghost_mask = 1;
  s.a[0] = dt;
  s.family = GPE_FAM_STAGE_LAST;
  if (c->prm.kahan) {
    // delta = dt f(psi); compensated psi' = psi + delta, c updated in place
    s.np = 1; s.pt[0] = c->c_id;
    s.out[1] = c->c_id;
    s.epi = EPI_KAHAN | EPI_NORM;
  } else {
    s.alpha[0] = 1.0;
    s.epi = EPI_NORM;
  }
  int rc = launch_stage(c, s);
  if (rc) return rc;
  swap_psi(c);
  return finalize(c, c->last_nblk, 0, 0, cell_volume(c), 0, false);
}

int step_rk2(gpe_ctx* c, cd dt) {
  StageSpec s1;
  s1.stencil = c->psi_id; s1.nout = 1; s1.out[0] = F_UA; s1.ghost_mask = 1;
  s1.alpha[0] = 1.0; s1.a[0] = 0.5 * dt; s1.family = GPE_FAM_STAGE_FIRST;
  int rc = launch_stage(c, s1);
  if (rc) return rc;
  StageSpec s2;
  s2.stencil = F_UA; s2.out[0] = c->psi_id; s2.ghost_mask = 1;
  s2.family = GPE_FAM_STAGE_LAST;
  if (c->prm.kahan) {
    s2.np = 2; s2.pt[0] = c->psi_id; s2.pt[1] = c->c_id;
    s2.nout = 2; s2.out[1] = c->c_id;
    s2.a[0] = dt;
    s2.epi = EPI_KAHAN | EPI_NORM;
  } else {
    s2.np = 1; s2.pt[0] = c->psi_id; s2.nout = 1;
    s2.beta[0][0] = 1.0; s2.a[0] = dt;
    s2.epi = EPI_NORM;
  }
  rc = launch_stage(c, s2);
  if (rc) return rc;
  return finalize(c, c->last_nblk, 0, 0, cell_volume(c), 0, false);
}

// The four classic RK4 stages (src/solve.f90:109-154) as stage recipes, in
// increment form.  With f1 = f(psi), d2 = dt/2 f1, d3 = dt/2 f(psi + d2),
// d4 = dt f(psi + d3), classic RK4 is
//   psi' = psi + dt/6 (f1 + 2 f2 + 2 f3 + f4)
//        = psi + [d2/3 + 2 d3/3 + d4/3 + dt/6 f(psi + d4)],
// and every stage after the first steps psi + d, staged from both fields
// with their halos (the kernel's second stencil field), so neither the stage
// values nor an accumulator are stored.  Traffic per site: S1 reads psi and
// writes d2; S2, S3 read psi, d and write the next d; S4 reads psi, d4, d2,
// d3 (and c) and writes psi' (and c): 16 + 24 + 24 + 48 (56 with Kahan)
// bytes at complex64, against 128 (152) for stage values plus accumulator.
// psi' is written over d2 (read at the same site only), then psi and that
// buffer trade roles; the bracket is summed smallest terms first and added
// to psi last (Kahan-compensated when enabled).
void rk4_specs(const gpe_ctx* c, cd dt, StageSpec sp[4]) {
  const bool K = c->prm.kahan != 0;
  const int psi = c->psi_id, d2 = c->alt_id, d3 = F_UB, d4 = F_ACC;
  // S1: d2 = dt/2 f(psi)
  StageSpec& s1 = sp[0];
  s1 = StageSpec();
  s1.stencil = psi; s1.nout = 1; s1.out[0] = d2; s1.ghost_mask = 1;
  s1.a[0] = 0.5 * dt;
  s1.family = GPE_FAM_STAGE_FIRST;
  // S2: d3 = dt/2 f(psi + d2)
  StageSpec& s2 = sp[1];
  s2 = StageSpec();
  s2.stencil = psi; s2.stencil2 = d2; s2.nout = 1; s2.out[0] = d3; s2.ghost_mask = 1;
  s2.a[0] = 0.5 * dt;
  s2.family = GPE_FAM_STAGE_MID;
  // S3: d4 = dt f(psi + d3)
  sp[2] = s2;
  sp[2].stencil2 = d3; sp[2].out[0] = d4; sp[2].a[0] = dt;
  // S4: psi' = psi (+) [d2/3 + 2 d3/3 + d4/3 + dt/6 f(psi + d4)], into d2's buffer
  StageSpec& s4 = sp[3];
  s4 = StageSpec();
  s4.stencil = psi; s4.stencil2 = d4; s4.out[0] = d2; s4.ghost_mask = 1;
  s4.family = GPE_FAM_STAGE_LAST;
  s4.pt[0] = d2; s4.pt[1] = d3;
  s4.beta[0][0] = 1.0 / 3.0; s4.beta[0][1] = 2.0 / 3.0;
  s4.alpha2[0] = 1.0 / 3.0;
  s4.a[0] = dt / 6.0;
  if (K) {
    s4.np = 3; s4.pt[2] = c->c_id;
    s4.nout = 2; s4.out[1] = c->c_id;
    s4.epi = EPI_KAHAN | EPI_NORM;
  } else {
    s4.np = 2; s4.nout = 1;
    s4.alpha[0] = 1.0;
    s4.epi = EPI_NORM;
  }
}

int step_rk4(gpe_ctx* c, cd dt) {
  StageSpec sp[4];
  rk4_specs(c, dt, sp);
  for (int st = 0; st < 4; st++) {
    const int rc = launch_stage(c, sp[st]);
    if (rc) return rc;
  }
  swap_psi(c);
  return finalize(c, c->last_nblk, 0, 0, cell_volume(c), 0, false);
}

// rkck (src/solve.f90:248-378) with the psi_scal / errmax reduction of rkqs
// (:176-190) fused into the last stage.  Writes the trial state to alt.
// reduce = false leaves the error maximum and the norm in the per-CTA
// partials for rk45_reduce_control_kernel.
int attempt_rkck(gpe_ctx* c, cd dt, cd dt0, const double* dyn = nullptr, bool reduce = true) {
  const bool K = c->prm.kahan != 0;
  const int psi = c->psi_id;
  const int stencils[6] = {psi, F_UA, F_UB, F_UA, F_UB, F_UA};
  const int ks[5] = {F_K1, F_K2, F_K3, F_K4, F_K5};
  const double B[5][5] = {{B21, 0, 0, 0, 0},
                          {B31, B32, 0, 0, 0},
                          {B41, B42, B43, 0, 0},
                          {B51, B52, B53, B54, 0},
                          {B61, B62, B63, B64, B65}};
  int rc;
  for (int st = 0; st < 5; st++) {
    // stage st+1: k = dt f(u_st); u_{st+1} = psi + sum_j B[st][j] k_j
    StageSpec s;
    s.stencil = stencils[st];
    s.nout = 2;
    s.out[0] = ks[st];
    s.out[1] = (st % 2 == 0) ? F_UA : F_UB;
    s.ghost_mask = 2;
    s.a[0] = dt;
    if (st == 0) {
      s.np = 0;
      s.alpha[1] = 1.0;
    } else {
      s.np = st + 1;
      s.pt[0] = psi;
      s.beta[1][0] = 1.0;
      for (int jj = 0; jj < st; jj++) {
        s.pt[jj + 1] = ks[jj];
        s.beta[1][jj + 1] = B[st][jj];
      }
    }
    s.a[1] = B[st][st] * dt;
    s.dyn = dyn;
    s.a_mul[0] = 1.0;
    s.a_mul[1] = B[st][st];
    s.family = st == 0 ? GPE_FAM_STAGE_FIRST : GPE_FAM_STAGE_MID;
    rc = launch_stage(c, s);
    if (rc) return rc;
  }
  // stage 6: psi_new = psi + c1 k1 + c3 k3 + c4 k4 + c6 dt f(u6)  (c2=c5=0)
  //          err     = dc1 k1 + dc3 k3 + dc4 k4 + dc5 k5 + dc6 dt f(u6)
  StageSpec s;
  s.stencil = F_UA;
  s.out[0] = c->alt_id;
  s.ghost_mask = 1;
  s.family = GPE_FAM_STAGE_LAST;
  s.dt0 = dt0;
  s.inv_absdt = 1.0 / std::abs(dt);
  s.a[0] = C6 * dt;
  s.cek = DC6 * dt;
  s.dyn = dyn;
  s.a_mul[0] = C6;
  s.cek_mul = DC6;
  // pointwise slots: psi, k1, k3, k4, k5 [, c]  (the kernel takes psi from
  // slot 0, k1 from slot 1 and the compensation from the last slot)
  s.pt[0] = psi;
  s.pt[1] = F_K1; s.pt[2] = F_K3; s.pt[3] = F_K4; s.pt[4] = F_K5;
  s.beta[0][1] = C1; s.beta[0][2] = C3; s.beta[0][3] = C4;
  s.ce[1] = DC1; s.ce[2] = DC3; s.ce[3] = DC4; s.ce[4] = DC5;
  if (K) {
    s.np = 6;
    s.pt[5] = c->c_id;
    s.nout = 2; s.out[1] = c->calt_id;
    s.epi = EPI_KAHAN | EPI_NORM | EPI_ERR;
  } else {
    s.np = 5;
    s.beta[0][0] = 1.0;
    s.nout = 1;
    s.epi = EPI_NORM | EPI_ERR;
  }
  rc = launch_stage(c, s);
  if (rc) return rc;
  if (!reduce) return GPE_OK;
  rc = finalize(c, c->last_nblk, 1, 1, 1.0 / RK_EPS, 3, false);
  if (rc) return rc;
  return finalize(c, c->last_nblk, 0, 0, cell_volume(c), 0, false);
}

// ---------------------------------------------------------------------------
// rkqs (src/solve.f90:158-244) with the step control on the device
// (rk45_control_kernel): an attempt is the six Cash-Karp stages reading dt
// from the context's DevTime, the error-maximum and norm reductions, then the
// control kernel, which accepts (advancing t and dt) or shrinks dt.  A step
// repeats attempts until one is accepted.  Where the stream can be captured
// (one context or a slab group; not with NCCL or per-launch timing) a step is
// one CUDA graph, a conditional WHILE node around the attempt, so a run of
// steps needs no host synchronisation; otherwise the host repeats the
// attempt, reading back two integers after each.  Both run the same kernels,
// so their step sequences are identical.

double rk45_errcon() { return std::pow(5.0 / SAFETY, 1.0 / DT_INCREASE); }

// The leader's DevTime (the group's first member steps the group).
DevTime* rk45_time(gpe_ctx* c) { return c->group ? c->group->m[0]->d_time : c->d_time; }

void rk45_drop_graphs(gpe_ctx* c) {
  for (int k = 0; k < 2; k++) {
    if (c->rk_exec[k]) cudaGraphExecDestroy(c->rk_exec[k]);
    if (c->rk_graph[k]) cudaGraphDestroy(c->rk_graph[k]);
    c->rk_exec[k] = nullptr;
    c->rk_graph[k] = nullptr;
    c->rk_psi[k] = -1;
  }
}

bool rk45_capturable(const gpe_ctx* c) { return !c->comm && !c->timing; }

// Enqueues one attempt and its control kernel (use_cond: inside the WHILE
// node whose handle is h).
// A context with no z-neighbours reduces the attempt's error maximum and norm
// in the step-control launch itself; slabs combine them across slabs first.
bool rk45_fused_control(const gpe_ctx* c) { return !c->group && !c->comm; }

// Launches of one attempt: the six stages, then either the fused reduction
// and control or two reductions and the control.
int rk45_launches_per_attempt(const gpe_ctx* c) { return rk45_fused_control(c) ? 7 : 9; }

int rk45_attempt(gpe_ctx* c, cudaGraphConditionalHandle h, int use_cond) {
  DevTime* T = rk45_time(c);
  const double* dyn = reinterpret_cast<const double*>(T);  // dt_r, dt_i, dt0_r, dt0_i
  const bool fused = rk45_fused_control(c);
  int rc = attempt_rkck(c, cd(1.0, 0.0), cd(1.0, 0.0), dyn, !fused);
  if (rc) return rc;
  if (fused) {
    rk45_reduce_control_kernel<<<1, 1024, 0, c->stream>>>(
        c->d_partials, c->last_nblk, 1.0 / RK_EPS, cell_volume(c), c->d_scal, T, c->d_series,
        c->d_ser_dt, c->d_ser_att, (int)c->series_cap, h, use_cond);
  } else {
    rk45_control_kernel<<<1, 32, 0, c->stream>>>(T, c->d_scal, c->d_series, c->d_ser_dt,
                                                  c->d_ser_att, (int)c->series_cap, h, use_cond);
  }
  CU_CHECK(c, cudaGetLastError());
  c->launches++;
  return GPE_OK;
}

// Captures the step that starts from the current psi buffer into slot k.
int rk45_build_graph(gpe_ctx* c, int k) {
  cudaGraph_t g = nullptr;
  CU_CHECK(c, cudaGraphCreate(&g, 0));
  auto bail = [&](int rc) {
    cudaGraphDestroy(g);
    return rc;
  };
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess)
    return bail(fail(c, GPE_ERR_CUDA, "cudaGraphConditionalHandleCreate failed"));
  const bool timing = c->timing;
  c->timing = false;
  // the begin kernel, then the WHILE node around one attempt
  cudaError_t e = cudaStreamBeginCaptureToGraph(c->stream, g, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rk45_begin_kernel<<<1, 32, 0, c->stream>>>(rk45_time(c), h, 1);
    cudaGraph_t tmp = nullptr;
    e = cudaStreamEndCapture(c->stream, &tmp);
  }
  if (e != cudaSuccess) {
    c->timing = timing;
    return bail(fail(c, GPE_ERR_CUDA, std::string("rk45 graph capture: ") + cudaGetErrorString(e)));
  }
  cudaGraphNode_t begin = nullptr;
  size_t nn = 1;
  cudaGraphGetNodes(g, &begin, &nn);
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cond = nullptr;
  e = cudaGraphAddNode(&cond, g, &begin, 1, &cp);
  if (e != cudaSuccess) {
    c->timing = timing;
    return bail(fail(c, GPE_ERR_CUDA, std::string("rk45 WHILE node: ") + cudaGetErrorString(e)));
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  int rc = GPE_OK;
  if (e == cudaSuccess) {
    rc = rk45_attempt(c, h, 1);
    cudaGraph_t tmp = nullptr;
    e = cudaStreamEndCapture(c->stream, &tmp);
  }
  c->timing = timing;
  if (rc) return bail(rc);
  if (e != cudaSuccess)
    return bail(fail(c, GPE_ERR_CUDA, std::string("rk45 attempt capture: ") + cudaGetErrorString(e)));
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  if (e != cudaSuccess)
    return bail(fail(c, GPE_ERR_CUDA, std::string("rk45 graph instantiate: ") + cudaGetErrorString(e)));
  c->rk_graph[k] = g;
  c->rk_exec[k] = x;
  c->rk_psi[k] = c->psi_id;
  return GPE_OK;
}

// Reads the DevTime back (one synchronisation).
int rk45_read(gpe_ctx* c, DevTime* h) {
  CU_CHECK(c, cudaMemcpyAsync(h, rk45_time(c), sizeof(DevTime), cudaMemcpyDeviceToHost,
                              c->stream));
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  return GPE_OK;
}

// Up to n steps from the time state in the DevTime; returns the steps taken
// in *done (fewer than n only if the control halted).  psi (and the Kahan
// pair) end in the buffers of the last accepted step.
int rk45_steps(gpe_ctx* c, int64_t n, int64_t* done) {
  *done = 0;
  if (n <= 0) return GPE_OK;
  DevTime h{};
  if (rk45_capturable(c)) {
    for (int k = 0; k < 2; k++) {
      // slot k starts from the psi buffer (k == 0: the current one)
      const int want = (k == 0) ? c->psi_id : c->alt_id;
      if (c->rk_psi[k] != want || !c->rk_exec[k]) {
        if (c->rk_exec[k]) cudaGraphExecDestroy(c->rk_exec[k]);
        if (c->rk_graph[k]) cudaGraphDestroy(c->rk_graph[k]);
        c->rk_exec[k] = nullptr;
        c->rk_graph[k] = nullptr;
        if (k == 1) {
          swap_psi(c);
          if (c->prm.kahan) swap_comp(c);
        }
        const int rc = rk45_build_graph(c, k);
        if (k == 1) {
          swap_psi(c);
          if (c->prm.kahan) swap_comp(c);
        }
        if (rc) return rc;
      }
    }
    for (int64_t s = 0; s < n; s++)
      CU_CHECK(c, cudaGraphLaunch(c->rk_exec[s & 1], c->stream));
    int rc = rk45_read(c, &h);
    if (rc) return rc;
    *done = h.steps;
    // graph replays: per step a begin kernel and per attempt 6 stages, 2
    // reductions and the control kernel
  } else {
    for (int64_t s = 0; s < n; s++) {
      rk45_begin_kernel<<<1, 32, 0, c->stream>>>(rk45_time(c), 0, 0);
      CU_CHECK(c, cudaGetLastError());
      c->launches++;
      for (;;) {
        int rc = rk45_attempt(c, 0, 0);
        if (rc) return rc;
        rc = rk45_read(c, &h);
        if (rc) return rc;
        if (h.halt || h.steps > s) break;
      }
      if (h.halt) break;
      swap_psi(c);
      if (c->prm.kahan) swap_comp(c);
    }
    *done = h.steps;
    return GPE_OK;
  }
  if (*done & 1) {
    swap_psi(c);
    if (c->prm.kahan) swap_comp(c);
  }
  return GPE_OK;
}

// Loads the host time state into the DevTime (steps counted from 0).
int rk45_load(gpe_ctx* c, const gpe_time* tm) {
  DevTime h{};
  h.dt_r = tm->dt_re;
  h.dt_i = tm->dt_im;
  h.dt0_r = tm->dt_re;
  h.dt0_i = tm->dt_im;
  h.t = tm->t;
  h.im_t = tm->im_t;
  h.errcon = rk45_errcon();
  h.real_time = c->prm.real_time ? 1 : 0;
  CU_CHECK(c, cudaMemcpyAsync(rk45_time(c), &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  return GPE_OK;
}

int rk45_halted(gpe_ctx* c, const DevTime& h) {
  if (h.halt == GPE_ERR_NAN)
    return fail(c, GPE_ERR_NAN, "non-finite rk45 error estimate or trial-state norm");
  if (h.halt) return fail(c, GPE_ERR_UNDERFLOW, "rk45: step size control did not converge");
  return GPE_OK;
}

int step_rk45(gpe_ctx* c, gpe_time* tm, gpe_step_info* info) {
  int rc = rk45_load(c, tm);
  if (rc) return rc;
  int64_t done = 0;
  rc = rk45_steps(c, 1, &done);
  if (rc) return rc;
  DevTime h{};
  rc = rk45_read(c, &h);
  if (rc) return rc;
  // a timed-out stage leaves no valid error estimate
  rc = check_status(c);
  if (rc) return rc;
  if (done != 1) return rk45_halted(c, h);
  c->launches += rk45_capturable(c) ? 1 + rk45_launches_per_attempt(c) * (int64_t)h.attempts : 0;
  tm->t = h.t;
  tm->im_t = h.im_t;
  tm->dt_re = h.dt_r;
  tm->dt_im = h.dt_i;
  if (info) {
    info->errmax = h.errmax;
    info->attempts = h.attempts;
    info->underflow = h.underflow;
    info->dt_did_re = h.did_r;
    info->dt_did_im = h.did_i;
  }
  return GPE_OK;
}

int do_step(gpe_ctx* c, gpe_time* tm, gpe_step_info* info) {
  const cd dt(tm->dt_re, tm->dt_im);
  int rc;
  c->norm_valid = false;
  switch (c->prm.scheme) {
    case GPE_SCHEME_EULER: rc = step_euler(c, dt); break;
    case GPE_SCHEME_RK2: rc = step_rk2(c, dt); break;
    case GPE_SCHEME_RK4: rc = step_rk4(c, dt); break;
    case GPE_SCHEME_RK45: rc = step_rk45(c, tm, info); break;
    default:
      return fail(c, GPE_ERR_SCHEME, "ERROR: Unrecognised time stepping scheme.");
  }
  if (rc) return rc;
  if (c->post_step) {
    rc = c->post_step(c->post_arg, c);
    if (rc) return fail(c, rc, "post-step correction failed");
  }
  if (c->prm.scheme != GPE_SCHEME_RK45) {
    tm->t = tm->t + dt.real();
    tm->im_t = tm->im_t + std::fabs(dt.imag());
    if (info) {
      info->errmax = 0.0;
      info->attempts = 1;
      info->underflow = 0;
      info->dt_did_re = dt.real();
      info->dt_did_im = dt.imag();
    }
  }
  // the fused norm is of the stepped state, before any post-step correction
  c->norm_valid = c->post_step == nullptr;
  return GPE_OK;
}

// --------------------------------------------------------------------------
// Tables and allocation.

// Per-axis tables.  Along z a context may hold the slab z_off .. z_off+nz-1
// of a global axis of nzg planes: coordinates, sponge edge and norm weights
// follow the global index.
int build_tables(gpe_ctx* c) {
  const gpe_params& p = c->prm;
  const int n[3] = {c->nx, c->ny, c->nz};
  const int ng[3] = {c->nx, c->ny, c->nzg};
  const int zoff[3] = {0, 0, c->z_off};
  const std::vector<double>* crd[3] = {&c->x, &c->y, &c->z};
  const double om[3] = {p.omx, p.omy, p.omz};
  size_t total = 0;
  for (int a = 0; a < 3; a++) {
    c->tab_n[a] = (int)round_up((size_t)n[a], 64) + 64;
    total += (size_t)c->tab_n[a];
  }
  // per axis: Vf, Df (float) + Vd, Dd, W, X (double)
  const size_t bytes = total * (2 * sizeof(float) + 4 * sizeof(double));
  CU_CHECK(c, cudaMalloc(&c->d_tables, bytes));
  c->device_bytes += (int64_t)bytes;
  std::vector<unsigned char> h(bytes, 0);
  size_t off = 0;
  auto take = [&](size_t nbytes) {
    size_t o = off;
    off += round_up(nbytes, 256);
    return o;
  };
  // recompute offsets with alignment
  off = 0;
  size_t offs[3][6];
  for (int a = 0; a < 3; a++) {
    offs[a][0] = take(sizeof(float) * c->tab_n[a]);
    offs[a][1] = take(sizeof(float) * c->tab_n[a]);
    for (int k = 2; k < 6; k++) offs[a][k] = take(sizeof(double) * c->tab_n[a]);
  }
  if (off > bytes) {
    cudaFree(c->d_tables);
    c->device_bytes -= (int64_t)bytes;
    CU_CHECK(c, cudaMalloc(&c->d_tables, off));
    c->device_bytes += (int64_t)off;
    h.assign(off, 0);
  }
  for (int a = 0; a < 3; a++) {
    float* vf = reinterpret_cast<float*>(&h[offs[a][0]]);
    float* df = reinterpret_cast<float*>(&h[offs[a][1]]);
    double* vd = reinterpret_cast<double*>(&h[offs[a][2]]);
    double* dd = reinterpret_cast<double*>(&h[offs[a][3]]);
    double* w = reinterpret_cast<double*>(&h[offs[a][4]]);
    double* xx = reinterpret_cast<double*>(&h[offs[a][5]]);
    const std::vector<double>& X = *crd[a];
    const int N = n[a], NG = ng[a], O = zoff[a];
    const double h = (a == 0) ? c->dx : (a == 1) ? c->dy : c->dz;
    const double r = (a == 0) ? p.xr : (a == 1) ? p.yr : p.zr;
    // sponge edge a = x(nx-3) of the global axis (src/solve.f90:397-409)
    const double edge = -r + (double)(NG - 3) * h;
    for (int i = 0; i < N; i++) {
      const double v = 0.5 * ((om[a] * om[a]) * (X[i] * X[i]));
      const double d = p.diss_amp * (1.0 + std::tanh(X[i] - edge) * std::tanh(X[i] + edge));
      vd[i] = v; vf[i] = (float)v;
      dd[i] = d; df[i] = (float)d;
      xx[i] = X[i];
    }
    // norm weights (src/variables.f90:713-823): x sums every term that
    // names an index, y and z take the last matching assignment.
    if (a == 0) {
      for (int i = 0; i < N; i++) w[i] = 0.0;
      w[0] += W1; w[1] += W2; w[2] += W3;
      for (int i = 3; i <= N - 4; i++) w[i] += 1.0;
      w[N - 3] += W3; w[N - 2] += W2; w[N - 1] += W1;
    } else {
      for (int i = 0; i < N; i++) {
        const int gi = O + i;
        double t = 1.0;
        if (gi == 0) t = W1;
        if (gi == 1) t = W2;
        if (gi == 2) t = W3;
        if (gi == NG - 3) t = W3;
        if (gi == NG - 2) t = W2;
        if (gi == NG - 1) t = W1;
        w[i] = t;
      }
    }
  }
  CU_CHECK(c, cudaMemcpy(c->d_tables, h.data(), h.size(), cudaMemcpyHostToDevice));
  unsigned char* base = static_cast<unsigned char*>(c->d_tables);
  for (int a = 0; a < 3; a++) {
    c->tabVf[a] = reinterpret_cast<float*>(base + offs[a][0]);
    c->tabDf[a] = reinterpret_cast<float*>(base + offs[a][1]);
    c->tabVd[a] = reinterpret_cast<double*>(base + offs[a][2]);
    c->tabDd[a] = reinterpret_cast<double*>(base + offs[a][3]);
    c->tabW[a] = reinterpret_cast<double*>(base + offs[a][4]);
    c->tabX[a] = reinterpret_cast<double*>(base + offs[a][5]);
  }
  return GPE_OK;
}

int alloc_field(gpe_ctx* c, int id) {
  const size_t bytes = c->npad * (size_t)c->es;
  cudaError_t e = cudaMalloc(&c->fld[id], bytes);
  if (e != cudaSuccess) {
    c->fld[id] = nullptr;
    cudaGetLastError();
    return fail(c, GPE_ERR_OOM, "cudaMalloc of a field failed: " +
                                    std::string(cudaGetErrorString(e)));
  }
  c->device_bytes += (int64_t)bytes;
  CU_CHECK(c, cudaMemset(c->fld[id], 0, bytes));
  return GPE_OK;
}

// d_stage (dense, elements of elem_bytes) -> psi with ghosts.
int load_stage(gpe_ctx* c, int elem_bytes) {
  Launch L{};
  begin_timed(c, L, GPE_FAM_COPY, (int64_t)c->nint);
  const Geom g = geom(c);
  const int nb = elementwise_blocks(c->nint);
  void* dst = c->fld[c->psi_id];
  if (c->es == 8) {
    if (elem_bytes == 8)
      unpack_kernel<float, float><<<nb, 256, 0, c->stream>>>(
          (const float*)c->d_stage, (float*)dst, g);
    else
      unpack_kernel<float, double><<<nb, 256, 0, c->stream>>>(
          (const double*)c->d_stage, (float*)dst, g);
  } else {
    if (elem_bytes == 8)
      unpack_kernel<double, float><<<nb, 256, 0, c->stream>>>(
          (const float*)c->d_stage, (double*)dst, g);
    else
      unpack_kernel<double, double><<<nb, 256, 0, c->stream>>>(
          (const double*)c->d_stage, (double*)dst, g);
  }
  CU_CHECK(c, cudaGetLastError());
  end_timed(c, L);
  c->launches++;
  if (c->prm.kahan && c->fld[c->c_id])
    CU_CHECK(c, cudaMemsetAsync(c->fld[c->c_id], 0, c->npad * (size_t)c->es,
                                c->stream));
  c->norm_valid = false;
  // a slab-group member's z ghosts come from its neighbours, which may not
  // be loaded yet: the group refreshes them before its next step
  if (c->group) c->ghosts_dirty = true;
  return exchange_ghosts(c, c->psi_id);
}

int stage_in(gpe_ctx* c, const void* src, int elem_bytes, bool device) {
  const size_t bytes = c->nint * (size_t)elem_bytes;
  CU_CHECK(c, cudaMemcpyAsync(c->d_stage, src, bytes,
                              device ? cudaMemcpyDeviceToDevice
                                     : cudaMemcpyHostToDevice,
                              c->stream));
  return load_stage(c, elem_bytes);
}

// field -> d_stage (dense, elements of elem_bytes).
int pack_stage(gpe_ctx* c, int field, int elem_bytes) {
  Launch L{};
  begin_timed(c, L, GPE_FAM_COPY, (int64_t)c->nint);
  const Geom g = geom(c);
  const int nb = elementwise_blocks(c->nint);
  const void* src = c->fld[field];
  if (c->es == 8) {
    if (elem_bytes == 8)
      pack_kernel<float, float><<<nb, 256, 0, c->stream>>>(
          (const float*)src, (float*)c->d_stage, g);
    else
      pack_kernel<float, double><<<nb, 256, 0, c->stream>>>(
          (const float*)src, (double*)c->d_stage, g);
  } else {
    if (elem_bytes == 8)
      pack_kernel<double, float><<<nb, 256, 0, c->stream>>>(
          (const double*)src, (float*)c->d_stage, g);
    else
      pack_kernel<double, double><<<nb, 256, 0, c->stream>>>(
          (const double*)src, (double*)c->d_stage, g);
  }
  CU_CHECK(c, cudaGetLastError());
  end_timed(c, L);
  c->launches++;
  return GPE_OK;
}

int stage_out(gpe_ctx* c, int field, void* dst, int elem_bytes, bool device) {
  int rc = pack_stage(c, field, elem_bytes);
  if (rc) return rc;
  CU_CHECK(c, cudaMemcpyAsync(dst, c->d_stage, c->nint * (size_t)elem_bytes,
                              device ? cudaMemcpyDeviceToDevice
                                     : cudaMemcpyDeviceToHost,
                              c->stream));
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  return GPE_OK;
}

int check_ctx(gpe_ctx* c) {
  if (!c) return GPE_ERR_INVALID;
  CU_CHECK(c, cudaSetDevice(c->dev));
  return GPE_OK;
}

// Entry points that step or reduce a whole grid refuse a slab-group member:
// the group steps and reduces its members together.
int check_solo(gpe_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (c->group)
    return fail(c, GPE_ERR_INVALID, "context is a member of a slab group; use gpe_group_*");
  return GPE_OK;
}

int check_elem(gpe_ctx* c, int elem_bytes, const void* ptr) {
  if (elem_bytes != 8 && elem_bytes != 16)
    return fail(c, GPE_ERR_INVALID, "elem_bytes must be 8 or 16");
  if (!ptr) return fail(c, GPE_ERR_INVALID, "null array");
  return GPE_OK;
}

}  // namespace

int gpe_internal_fail(gpe_ctx* c, int code, const std::string& msg) { return fail(c, code, msg); }
void gpe_internal_time_begin(gpe_ctx* c, gpe::TimedRegion* r, int family, int64_t sites) {
  Launch L{};
  begin_timed(c, L, family, sites);
  r->a = L.a;
  r->b = L.b;
  r->family = family;
  r->sites = sites;
}
void gpe_internal_time_end(gpe_ctx* c, gpe::TimedRegion* r) {
  if (!r->a) return;
  Launch L{r->family, r->a, r->b, r->sites};
  end_timed(c, L);
}
int gpe_internal_load_stage(gpe_ctx* c) { return load_stage(c, c->es); }

// psi rescaled on the context's stream so that its norm equals the norm the
// last step fused into d_scal[0] (before any post-step correction); the
// norm of psi as it stands goes to d_scal[8].  No host synchronisation.
int gpe_internal_restore_norm(gpe_ctx* c) {
  const Geom g = geom(c);
  const int nb = elementwise_blocks(c->nint);
  if (c->es == 8)
    norm_kernel<float><<<nb, 256, 0, c->stream>>>((const float*)c->fld[c->psi_id], g,
                                                  c->tabW[0], c->tabW[1], c->tabW[2],
                                                  c->d_partials);
  else
    norm_kernel<double><<<nb, 256, 0, c->stream>>>((const double*)c->fld[c->psi_id], g,
                                                   c->tabW[0], c->tabW[1], c->tabW[2],
                                                   c->d_partials);
  CU_CHECK(c, cudaGetLastError());
  finalize_kernel<<<1, 1024, 0, c->stream>>>(c->d_partials, nb, 0, 0, cell_volume(c),
                                              c->d_scal + 8, nullptr, c->d_counter);
  const size_t n = c->npad * 2;
  const int sb = elementwise_blocks(n);
  if (c->es == 8)
    rescale_to_kernel<float><<<sb, 256, 0, c->stream>>>((float*)c->fld[c->psi_id], n,
                                                        c->d_scal, c->d_scal + 8);
  else
    rescale_to_kernel<double><<<sb, 256, 0, c->stream>>>((double*)c->fld[c->psi_id], n,
                                                         c->d_scal, c->d_scal + 8);
  CU_CHECK(c, cudaGetLastError());
  c->launches += 3;
  return GPE_OK;
}

// ==========================================================================
// Batched ensembles: independent runs of uneven grids stepped by one
// persistent launch per RK4 stage.  Each member is a full context (fields,
// tables, tensor maps); the batch adds one work list of (run, tile, z-range)
// items for all members, per-stage arrays of their RunDescs in device memory,
// and a CUDA graph of one whole step (4 stage launches + per-run norm).

struct gpe_batch {
  int dev = 0;
  cudaStream_t stream = nullptr;
  std::vector<gpe_ctx*> runs;
  gpe_batch_opts opts;
  int es = 8, R = 1;
  int form = FORM_PLAIN;  // the highest right-hand-side form among the members
  int TY = 8;
  WorkItem* d_items = nullptr;
  int* d_item_run = nullptr;
  int nitems = 0;
  double* d_partials = nullptr;
  double* d_scale = nullptr;
  double* d_norm = nullptr;
  double* d_series = nullptr;
  size_t series_cap = 0;
  int64_t series_steps = 0;  // steps the last rk45 advance recorded  // steps per run
  int* d_counter = nullptr;
  int* d_status = nullptr;
  // Two prepared step forms: RK4 leaves psi in the members' other buffer
  // (rk4_specs), so [0] steps from the members' current psi and [1] from the
  // buffer the step after it starts from; steps alternate between them.
  void* d_rundesc[2][4] = {};
  struct Stage {
    KernelFn fn = nullptr;
    LaunchShape sh{};
    int grid = 0;
    std::vector<unsigned char> params;  // StageParams bytes
  } st[2][4];
  cd prepared_dt = cd(0.0, 0.0);
  bool prepared = false;
  std::vector<int> prepared_psi;  // each member's psi buffer that [0] starts from
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  double* graph_series = nullptr;
  int64_t launches = 0;
  int64_t sites = 0;
  std::string err;
};

namespace {

int bfail(gpe_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  else g_last_create_error = msg;
  return code;
}

#define BCU(b, call)                                                          \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return bfail((b), GPE_ERR_CUDA,                                         \
                   std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)

// Kernels, shapes and RunDesc arrays of the four stages for time step dt.
template <typename TS, typename TC>
int batch_prepare_par(gpe_batch* b, cd dt, int par) {
  for (int s = 0; s < 4; s++) {
    std::vector<RunDesc<TS, TC>> rds(b->runs.size());
    StageSpec sp0[4];
    rk4_specs(b->runs[0], dt, sp0);
    const StageSpec& sp = sp0[s];
    int am, bm;
    recipe_masks(sp, &am, &bm);
    int form = b->form;
    KernelFn fn = select_kernel<TS, TC, true>(b->R, &form, sp, am, bm);
    if (!fn) return bfail(b, GPE_ERR_INVALID, "no batched kernel for this stage");
    const int ns = sp.stencil2 >= 0 ? 2 : 1;
    const int rows = rows_per_warp<TS, TC>(b->R, ns, sp.np, form, true);
    // two-row recipes: rings for three CTAs per SM, as their registers allow
    LaunchShape sh = ring_shape(b->es, b->R, sp.np, b->TY, ns, rows == 2 ? 3 : 2);
    sh.rows = rows;
    BCU(b, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem));
    int occ = 0;
    BCU(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 32 * (sh.TY / sh.rows + 1),
                                                         sh.smem));
    if (occ < 1) return bfail(b, GPE_ERR_INVALID, "batched stage kernel cannot be resident");
    const int per_sm = b->opts.ctas_per_sm > 0 ? std::min(b->opts.ctas_per_sm, occ) : occ;
    const int grid = std::min(b->nitems, per_sm * b->runs[0]->num_sms);
    for (size_t r = 0; r < b->runs.size(); r++) {
      gpe_ctx* c = b->runs[r];
      StageSpec spr[4];
      rk4_specs(c, dt, spr);
      LaunchShape shr = sh;
      shr.ntx = (c->nx + TX - 1) / TX;
      shr.nty = (c->ny + sh.TY - 1) / sh.TY;
      shr.zchunk = 0;
      shr.nchunks = 0;
      const int rc = fill_run<TS, TC>(c, spr[s], b->R, shr, rhs_form(c), &rds[r],
                                      form == FORM_FULL ? 1 : 0);
      if (rc) return bfail(b, rc, c->err);
    }
    BCU(b, cudaMemcpy(b->d_rundesc[par][s], rds.data(), sizeof(RunDesc<TS, TC>) * rds.size(),
                      cudaMemcpyHostToDevice));
    StageParams<TS, TC> p;
    memset(&p, 0, sizeof(p));
    fill_common<TS, TC>(sp, form != FORM_FULL, sh, &p);
    p.runs = static_cast<const RunDesc<TS, TC>*>(b->d_rundesc[par][s]);
    p.items = b->d_items;
    p.nitems = b->nitems;
    p.partials = b->d_partials;
    p.status = b->d_status;
    b->st[par][s].fn = fn;
    b->st[par][s].sh = sh;
    b->st[par][s].grid = grid;
    b->st[par][s].params.assign(reinterpret_cast<unsigned char*>(&p),
                                reinterpret_cast<unsigned char*>(&p) + sizeof(p));
  }
  return GPE_OK;
}

void batch_swap_members(gpe_batch* b) {
  for (auto* c : b->runs) std::swap(c->psi_id, c->alt_id);
}

template <typename TS, typename TC>
int batch_prepare_t(gpe_batch* b, cd dt) {
  int rc = batch_prepare_par<TS, TC>(b, dt, 0);
  if (rc) return rc;
  batch_swap_members(b);
  rc = batch_prepare_par<TS, TC>(b, dt, 1);
  batch_swap_members(b);
  if (rc) return rc;
  b->prepared_dt = dt;
  b->prepared = true;
  b->prepared_psi.clear();
  for (auto* c : b->runs) b->prepared_psi.push_back(c->psi_id);
  return GPE_OK;
}

int batch_prepare(gpe_batch* b, cd dt) {
  if (b->es == 8) return batch_prepare_t<float, float>(b, dt);
  return batch_prepare_t<double, double>(b, dt);
}

// One RK4 step of every member: 4 persistent stage launches, per-run norm
// into d_norm and the series, step counter bump.
int batch_enqueue_step(gpe_batch* b, int par) {
  for (int s = 0; s < 4; s++) {
    auto& S = b->st[par][s];
    void* args[] = {S.params.data()};
    BCU(b, cudaLaunchKernel(S.fn, dim3((unsigned)S.grid), dim3(32, (unsigned)(S.sh.TY / S.sh.rows) + 1),
                            args, S.sh.smem, b->stream));
  }
  batch_finalize_kernel<<<(unsigned)b->runs.size(), 256, 0, b->stream>>>(
      b->d_partials, b->d_item_run, b->nitems, b->d_scale, b->d_norm, b->d_series,
      (int)b->series_cap, b->d_counter);
  bump_counter_kernel<<<1, 1, 0, b->stream>>>(b->d_counter);
  BCU(b, cudaGetLastError());
  return GPE_OK;
}

const char* bad_opts(const gpe_batch_opts& o) {
  if (o.tile_y != 0 && o.tile_y != 4 && o.tile_y != 8) return "tile_y must be 0, 4 or 8";
  if (o.zchunk < 0 || o.ctas_per_sm < 0) return "zchunk and ctas_per_sm must be >= 0";
  return nullptr;
}

// The work list of b->opts: every member's (tile, z-range) items, sorted by
// the sites they touch (warm-up planes included), largest first, so the
// persistent CTAs' round-robin walk ends on the small items.
int batch_plan(gpe_batch* b) {
  const gpe_batch_opts& o = b->opts;
  b->TY = o.tile_y > 0 ? o.tile_y : 8;
  std::vector<WorkItem> items;
  std::vector<long> work;
  for (int r = 0; r < (int)b->runs.size(); r++) {
    const gpe_ctx* c = b->runs[r];
    const int ntx = (c->nx + TX - 1) / TX, nty = (c->ny + b->TY - 1) / b->TY;
    const int zc = o.zchunk > 0 ? std::min(o.zchunk, c->nz) : std::min(c->nz, 64);
    for (int z0 = 0; z0 < c->nz; z0 += zc)
      for (int t = 0; t < ntx * nty; t++) {
        const int tx = t % ntx, tyy = t / ntx;
        const int z1 = std::min(z0 + zc, c->nz);
        items.push_back(WorkItem{r, t, z0, z1});
        work.push_back((long)(z1 - z0 + 2 * b->R) * std::min(TX, c->nx - tx * TX) *
                       std::min(b->TY, c->ny - tyy * b->TY));
      }
  }
  std::vector<size_t> order(items.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t x, size_t y) { return work[x] > work[y]; });
  std::vector<WorkItem> sorted;
  std::vector<int> item_run;
  for (size_t i : order) {
    sorted.push_back(items[i]);
    item_run.push_back(items[i].run);
  }
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_item_run) cudaFree(b->d_item_run);
  if (b->d_partials) cudaFree(b->d_partials);
  b->d_items = nullptr;
  b->d_item_run = nullptr;
  b->d_partials = nullptr;
  b->nitems = (int)sorted.size();
  if (cudaMalloc(&b->d_items, sizeof(WorkItem) * sorted.size()) != cudaSuccess ||
      cudaMalloc(&b->d_item_run, sizeof(int) * item_run.size()) != cudaSuccess ||
      cudaMalloc(&b->d_partials, 2 * sizeof(double) * sorted.size()) != cudaSuccess) {
    cudaGetLastError();
    b->err = "cudaMalloc of the batch work list failed";
    return GPE_ERR_OOM;
  }
  if (cudaMemcpy(b->d_items, sorted.data(), sizeof(WorkItem) * sorted.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_item_run, item_run.data(), sizeof(int) * item_run.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess) {
    b->err = "upload of the batch work list failed";
    return GPE_ERR_CUDA;
  }
  b->prepared = false;
  return GPE_OK;
}

void batch_drop_graph(gpe_batch* b) {
  for (int k = 0; k < 2; k++) {
    if (b->exec[k]) cudaGraphExecDestroy(b->exec[k]);
    if (b->graph[k]) cudaGraphDestroy(b->graph[k]);
    b->exec[k] = nullptr;
    b->graph[k] = nullptr;
  }
}

// After an odd number of steps the members' psi is in their other buffer:
// swap their ids and the two prepared forms, so [0] again starts from psi.
void batch_flip(gpe_batch* b) {
  batch_swap_members(b);
  for (size_t r = 0; r < b->runs.size() && r < b->prepared_psi.size(); r++)
    b->prepared_psi[r] = b->runs[r]->psi_id;
  for (int s = 0; s < 4; s++) {
    std::swap(b->st[0][s], b->st[1][s]);
    std::swap(b->d_rundesc[0][s], b->d_rundesc[1][s]);
  }
  std::swap(b->graph[0], b->graph[1]);
  std::swap(b->exec[0], b->exec[1]);
}

}  // namespace

// ==========================================================================
// C-ABI

extern "C" {

int32_t gpe_gpu_abi_version(void) { return GPE_GPU_ABI_VERSION; }

void gpe_gpu_default_params(gpe_params* p, int32_t nx, int32_t ny,
                            int32_t nz) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->struct_size = (int32_t)sizeof(gpe_params);
  p->nx = nx; p->ny = ny; p->nz = nz;
  p->xr = p->yr = p->zr = 1.0;
  p->scheme = GPE_SCHEME_RK4;
  p->eqn_to_solve = 4;
  p->bcs = 1;
  p->order = 2;
  p->real_time = 1;
  p->precision = 16;
  p->scal = 1.0; p->g = 1.0; p->mu = 1.0; p->nn = 1.0;
}

int gpe_gpu_create(const gpe_params* prm, gpe_ctx** out) {
  if (!out) return fail(nullptr, GPE_ERR_INVALID, "out is null");
  *out = nullptr;
  if (!prm) return fail(nullptr, GPE_ERR_INVALID, "params is null");
  if (prm->struct_size != (int32_t)sizeof(gpe_params))
    return fail(nullptr, GPE_ERR_INVALID, "gpe_params struct_size mismatch");
  const gpe_params& p = *prm;
  if (p.nx < 6 || p.ny < 6 || p.nz < 6)
    return fail(nullptr, GPE_ERR_INVALID, "nx, ny, nz must be >= 6");
  if (p.order != 2 && p.order != 4)
    return fail(nullptr, GPE_ERR_INVALID, "order must be 2 or 4");
  if (p.bcs != 1 && p.bcs != 2)
    return fail(nullptr, GPE_ERR_INVALID, "bcs must be 1 or 2");
  if (p.eqn_to_solve < 1 || p.eqn_to_solve > 4)
    return fail(nullptr, GPE_ERR_INVALID, "eqn_to_solve must be 1..4");
  if (p.precision != 8 && p.precision != 16)
    return fail(nullptr, GPE_ERR_INVALID, "precision must be 8 or 16");
  if (p.kahan && p.precision != 8)
    return fail(nullptr, GPE_ERR_INVALID, "kahan applies to precision 8 only");
  if (p.tile_y != 0 && p.tile_y != 4 && p.tile_y != 8)
    return fail(nullptr, GPE_ERR_INVALID, "tile_y must be 0, 4 or 8");
  if (p.xr <= 0 || p.yr <= 0 || p.zr <= 0)
    return fail(nullptr, GPE_ERR_INVALID, "xr, yr, zr must be positive");
  if (p.fd_match != 0.0 && (p.order != 4 || !(p.fd_match > 0.0 && p.fd_match < 1.5)))
    return fail(nullptr, GPE_ERR_INVALID, "fd_match needs order 4 and 0 < fd_match < 1.5");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= p.device || p.device < 0) {
    cudaGetLastError();
    return fail(nullptr, GPE_ERR_NODEVICE, "no CUDA device available");
  }
  cudaDeviceProp dp;
  if (cudaGetDeviceProperties(&dp, p.device) != cudaSuccess || dp.major != 10)
    return fail(nullptr, GPE_ERR_NODEVICE, "device is not sm_100 (B200)");

  gpe_ctx* c = new gpe_ctx();
  c->prm = p;
  c->num_sms = dp.multiProcessorCount;
  c->dev = p.device;
  memset(&c->acc_timing, 0, sizeof(c->acc_timing));
  auto bail = [&](int rc) {
    g_last_create_error = c->err;
    gpe_gpu_destroy(c);
    return rc;
  };
  if (cudaSetDevice(c->dev) != cudaSuccess) {
    c->err = "cudaSetDevice failed";
    return bail(GPE_ERR_CUDA);
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    c->err = "cudaStreamCreate failed";
    return bail(GPE_ERR_CUDA);
  }
  c->nx = p.nx; c->ny = p.ny; c->nz = p.nz;
  c->Nx = (int)round_up((size_t)p.nx + 4, 4);
  c->Ny = p.ny + 4;
  c->Nz = p.nz + 4;
  c->npad = (size_t)c->Nx * c->Ny * c->Nz;
  c->nint = (size_t)p.nx * p.ny * p.nz;
  c->es = p.precision;
  c->nzg = p.nz;
  c->z_off = 0;
  // get_grid, src/ic.f90:32-69
  c->dx = (p.xr - (-p.xr)) / (double)(p.nx - 1);
  c->dy = (p.yr - (-p.yr)) / (double)(p.ny - 1);
  c->dz = (p.zr - (-p.zr)) / (double)(p.nz - 1);
  c->x.resize(p.nx); c->y.resize(p.ny); c->z.resize(p.nz);
  for (int i = 0; i < p.nx; i++) c->x[i] = -p.xr + (double)i * c->dx;
  for (int j = 0; j < p.ny; j++) c->y[j] = -p.yr + (double)j * c->dy;
  for (int k = 0; k < p.nz; k++) c->z[k] = -p.zr + (double)k * c->dz;

  int rc = build_tables(c);
  if (rc) return bail(rc);
  std::vector<int> need = {F_PSI, F_ALT};
  switch (p.scheme) {
    case GPE_SCHEME_RK2: need.push_back(F_UA); break;
    case GPE_SCHEME_RK4:
      need.insert(need.end(), {F_UB, F_ACC});
      break;
    case GPE_SCHEME_RK45:
      need.insert(need.end(), {F_UA, F_UB, F_K1, F_K2, F_K3, F_K4, F_K5});
      break;
    default: break;
  }
  if (p.kahan) {
    need.push_back(F_C);
    if (p.scheme == GPE_SCHEME_RK45) need.push_back(F_CALT);
  }
  for (int id : need) {
    rc = alloc_field(c, id);
    if (rc) return bail(rc);
  }
  // partials: upper bound over every launch shape (TY >= 4, zchunk >= 1)
  const size_t ntiles_max = (size_t)((p.nx + TX - 1) / TX) * ((p.ny + 3) / 4);
  c->partials_cap = std::max<size_t>(ntiles_max * (size_t)p.nz, 148 * 16);
  if (cudaMalloc(&c->d_partials, 2 * sizeof(double) * c->partials_cap) != cudaSuccess ||
      cudaMalloc(&c->d_scal, 16 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_counter, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->d_stage, c->nint * 16) != cudaSuccess) {
    cudaGetLastError();
    c->err = "cudaMalloc of scratch buffers failed";
    return bail(GPE_ERR_OOM);
  }
  c->device_bytes += (int64_t)(2 * sizeof(double) * c->partials_cap +
                               16 * sizeof(double) + 2 * sizeof(int) + c->nint * 16);
  if (p.scheme == GPE_SCHEME_RK45) {
    if (cudaMalloc(&c->d_time, sizeof(DevTime)) != cudaSuccess) {
      cudaGetLastError();
      c->err = "cudaMalloc of the rk45 time state failed";
      return bail(GPE_ERR_OOM);
    }
    cudaMemset(c->d_time, 0, sizeof(DevTime));
    c->device_bytes += (int64_t)sizeof(DevTime);
  }
  cudaMemset(c->d_scal, 0, 16 * sizeof(double));
  cudaMemset(c->d_status, 0, sizeof(int));
  cudaMemset(c->d_counter, 0, sizeof(int));
  if (cudaDeviceSynchronize() != cudaSuccess) {
    c->err = "device synchronisation failed during create";
    return bail(GPE_ERR_CUDA);
  }
  *out = c;
  return GPE_OK;
}

void gpe_gpu_destroy(gpe_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->group) {  // the group outlives no member: it stops stepping this one
    gpe_group* g = c->group;
    cudaStreamSynchronize(g->stream);
    for (gpe_ctx* m : g->m) {
      m->stream = m->own_stream;
      m->group = nullptr;
      rk45_drop_graphs(m);
    }
    g->m.clear();
  }
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& e : c->ext) e.reset();
  if (c->comm && g_nccl.ok) g_nccl.CommDestroy(c->comm);
  for (int i = 0; i < F_COUNT; i++)
    if (c->fld[i]) cudaFree(c->fld[i]);
  if (c->d_tables) cudaFree(c->d_tables);
  if (c->d_partials) cudaFree(c->d_partials);
  if (c->d_scal) cudaFree(c->d_scal);
  if (c->d_series) cudaFree(c->d_series);
  if (c->d_counter) cudaFree(c->d_counter);
  if (c->d_status) cudaFree(c->d_status);
  if (c->d_stage) cudaFree(c->d_stage);
  rk45_drop_graphs(c);
  if (c->d_time) cudaFree(c->d_time);
  if (c->d_ser_dt) cudaFree(c->d_ser_dt);
  if (c->d_ser_att) cudaFree(c->d_ser_att);
  for (auto& L : c->timed) {
    cudaEventDestroy(L.a);
    cudaEventDestroy(L.b);
  }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  if (c->xstream) {
    cudaStreamSynchronize(c->xstream);
    cudaStreamDestroy(c->xstream);
  }
  for (auto e : c->xev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* gpe_gpu_last_error(const gpe_ctx* c) {
  if (!c) return g_last_create_error.c_str();
  return c->err.c_str();
}

int gpe_gpu_grid(const gpe_ctx* c, double* x, double* y, double* z) {
  if (!c) return GPE_ERR_INVALID;
  if (x) memcpy(x, c->x.data(), sizeof(double) * c->nx);
  if (y) memcpy(y, c->y.data(), sizeof(double) * c->ny);
  if (z) memcpy(z, c->z.data(), sizeof(double) * c->nz);
  return GPE_OK;
}

int gpe_gpu_set_state(gpe_ctx* c, const void* psi, int32_t elem_bytes) {
  int rc = check_ctx(c);
  if (rc) return rc;
  rc = check_elem(c, elem_bytes, psi);
  if (rc) return rc;
  rc = stage_in(c, psi, elem_bytes, false);
  if (rc) return rc;
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  return GPE_OK;
}

int gpe_gpu_get_state(gpe_ctx* c, void* psi, int32_t elem_bytes) {
  int rc = check_ctx(c);
  if (rc) return rc;
  rc = check_elem(c, elem_bytes, psi);
  if (rc) return rc;
  return stage_out(c, c->psi_id, psi, elem_bytes, false);
}

int gpe_gpu_set_state_device(gpe_ctx* c, const void* psi, int32_t elem_bytes) {
  int rc = check_ctx(c);
  if (rc) return rc;
  rc = check_elem(c, elem_bytes, psi);
  if (rc) return rc;
  rc = stage_in(c, psi, elem_bytes, true);
  if (rc) return rc;
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  return GPE_OK;
}

int gpe_gpu_get_state_device(gpe_ctx* c, void* psi, int32_t elem_bytes) {
  int rc = check_ctx(c);
  if (rc) return rc;
  rc = check_elem(c, elem_bytes, psi);
  if (rc) return rc;
  return stage_out(c, c->psi_id, psi, elem_bytes, true);
}

int gpe_gpu_get_site(gpe_ctx* c, int32_t i, int32_t j, int32_t k, double* re_im) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!re_im) return fail(c, GPE_ERR_INVALID, "null output");
  if (i < 0 || i >= c->nx || j < 0 || j >= c->ny || k < 0 || k >= c->nz)
    return fail(c, GPE_ERR_INVALID, "site outside the grid");
  const size_t q = ((size_t)(k + 2) * c->Ny + (size_t)(j + 2)) * c->Nx + (size_t)(i + 2);
  unsigned char buf[16];
  CU_CHECK(c, cudaMemcpyAsync(buf, static_cast<const unsigned char*>(c->fld[c->psi_id]) +
                                       q * (size_t)c->es,
                              (size_t)c->es, cudaMemcpyDeviceToHost, c->stream));
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  if (c->es == 8) {
    float f[2];
    memcpy(f, buf, sizeof(f));
    re_im[0] = f[0];
    re_im[1] = f[1];
  } else {
    memcpy(re_im, buf, 2 * sizeof(double));
  }
  return GPE_OK;
}

int gpe_gpu_get_plane(gpe_ctx* c, int32_t k, void* out, int32_t elem_bytes) {
  int rc = check_ctx(c);
  if (rc) return rc;
  rc = check_elem(c, elem_bytes, out);
  if (rc) return rc;
  if (k < 0 || k >= c->nz) return fail(c, GPE_ERR_INVALID, "plane outside the grid");
  const size_t first = ((size_t)(k + 2) * c->Ny + 2) * c->Nx + 2;
  const unsigned char* src = static_cast<const unsigned char*>(c->fld[c->psi_id]) +
                             first * (size_t)c->es;
  const size_t n = (size_t)c->nx * c->ny;
  std::vector<unsigned char> tmp;
  void* dst = out;
  if (elem_bytes != c->es) {
    tmp.resize(n * (size_t)c->es);
    dst = tmp.data();
  }
  CU_CHECK(c, cudaMemcpy2DAsync(dst, (size_t)c->nx * c->es, src, (size_t)c->Nx * c->es,
                                (size_t)c->nx * c->es, c->ny, cudaMemcpyDeviceToHost,
                                c->stream));
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  if (elem_bytes != c->es) {
    if (c->es == 8) {
      const float* f = reinterpret_cast<const float*>(tmp.data());
      double* o = static_cast<double*>(out);
      for (size_t q = 0; q < 2 * n; q++) o[q] = f[q];
    } else {
      const double* f = reinterpret_cast<const double*>(tmp.data());
      float* o = static_cast<float*>(out);
      for (size_t q = 0; q < 2 * n; q++) o[q] = (float)f[q];
    }
  }
  return GPE_OK;
}

int gpe_gpu_solver(gpe_ctx* c, gpe_time* tm, gpe_step_info* info) {
  int rc = check_solo(c);
  if (rc) return rc;
  if (!tm) return fail(c, GPE_ERR_INVALID, "tm is null");
  rc = do_step(c, tm, info);
  if (rc) return rc;
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  return check_status(c);
}

int gpe_gpu_solver_host(gpe_ctx* c, const void* var_in, void* var_out,
                        int32_t elem_bytes, gpe_time* tm, gpe_step_info* info) {
  int rc = check_solo(c);
  if (rc) return rc;
  rc = check_elem(c, elem_bytes, var_in);
  if (rc) return rc;
  rc = check_elem(c, elem_bytes, var_out);
  if (rc) return rc;
  if (!tm) return fail(c, GPE_ERR_INVALID, "tm is null");
  rc = stage_in(c, var_in, elem_bytes, false);
  if (rc) return rc;
  rc = do_step(c, tm, info);
  if (rc) return rc;
  rc = stage_out(c, c->psi_id, var_out, elem_bytes, false);
  if (rc) return rc;
  return check_status(c);
}

int gpe_gpu_advance(gpe_ctx* c, int64_t nsteps, gpe_time* tm, double* norms) {
  int rc = check_solo(c);
  if (rc) return rc;
  if (!tm || nsteps < 0) return fail(c, GPE_ERR_INVALID, "bad advance arguments");
  if ((size_t)nsteps > c->series_cap) {
    // the captured rk45 steps hold the old series pointers
    CU_CHECK(c, cudaStreamSynchronize(c->stream));
    rk45_drop_graphs(c);
    if (c->d_series) cudaFree(c->d_series);
    if (c->d_ser_dt) cudaFree(c->d_ser_dt);
    if (c->d_ser_att) cudaFree(c->d_ser_att);
    c->d_series = nullptr;
    c->d_ser_dt = nullptr;
    c->d_ser_att = nullptr;
    c->series_cap = 0;
    const size_t cap = std::max<size_t>((size_t)nsteps, 1024);
    CU_CHECK(c, cudaMalloc(&c->d_series, cap * sizeof(double)));
    CU_CHECK(c, cudaMalloc(&c->d_ser_dt, cap * sizeof(double)));
    CU_CHECK(c, cudaMalloc(&c->d_ser_att, cap * sizeof(int)));
    c->series_cap = cap;
  }
  if (c->prm.scheme == GPE_SCHEME_RK45 && !c->post_step) {
    // nsteps accepted steps with the step control on the device
    c->norm_valid = false;
    rc = rk45_load(c, tm);
    if (rc) return rc;
    int64_t done = 0;
    rc = rk45_steps(c, nsteps, &done);
    if (rc) return rc;
    DevTime h{};
    rc = rk45_read(c, &h);
    if (rc) return rc;
    rc = check_status(c);
    if (rc) return rc;
    tm->t = h.t;
    tm->im_t = h.im_t;
    tm->dt_re = h.dt_r;
    tm->dt_im = h.dt_i;
    tm->p += (int32_t)done;
    if (done > 0) {
      if (norms)
        CU_CHECK(c, cudaMemcpy(norms, c->d_series, sizeof(double) * done, cudaMemcpyDeviceToHost));
      if (rk45_capturable(c)) {
        std::vector<int> att((size_t)done);
        CU_CHECK(c, cudaMemcpy(att.data(), c->d_ser_att, sizeof(int) * done,
                               cudaMemcpyDeviceToHost));
        for (int a : att) c->launches += rk45_launches_per_attempt(c) * (int64_t)a;
        c->launches += done;
      }
    }
    c->series_steps = done;
    if (done < nsteps) return rk45_halted(c, h);
    c->norm_valid = true;
    return GPE_OK;
  }
  CU_CHECK(c, cudaMemsetAsync(c->d_counter, 0, sizeof(int), c->stream));
  for (int64_t s = 0; s < nsteps; s++) {
    rc = do_step(c, tm, nullptr);
    if (rc) return rc;
    // copy the fused norm into the per-step series
    CU_CHECK(c, cudaMemcpyAsync(c->d_series + s, c->d_scal, sizeof(double),
                                cudaMemcpyDeviceToDevice, c->stream));
    tm->p += 1;
  }
  if (norms && nsteps > 0)
    CU_CHECK(c, cudaMemcpyAsync(norms, c->d_series, sizeof(double) * nsteps,
                                cudaMemcpyDeviceToHost, c->stream));
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  return check_status(c);
}

int gpe_gpu_norm(gpe_ctx* c, double* norm) {
  int rc = check_solo(c);
  if (rc) return rc;
  if (!norm) return fail(c, GPE_ERR_INVALID, "norm is null");
  if (!c->norm_valid) {
    const Geom g = geom(c);
    const int nb = elementwise_blocks(c->nint);
    Launch L{};
    begin_timed(c, L, GPE_FAM_REDUCE, (int64_t)c->nint);
    if (c->es == 8)
      norm_kernel<float><<<nb, 256, 0, c->stream>>>(
          (const float*)c->fld[c->psi_id], g, c->tabW[0], c->tabW[1], c->tabW[2],
          c->d_partials);
    else
      norm_kernel<double><<<nb, 256, 0, c->stream>>>(
          (const double*)c->fld[c->psi_id], g, c->tabW[0], c->tabW[1], c->tabW[2],
          c->d_partials);
    CU_CHECK(c, cudaGetLastError());
    end_timed(c, L);
    c->launches++;
    rc = finalize(c, nb, 0, 0, cell_volume(c), 0, false);
    if (rc) return rc;
    c->norm_valid = true;
  }
  rc = read_scalars(c, norm, 0, 1);
  if (rc) return rc;
  if (!std::isfinite(*norm)) return fail(c, GPE_ERR_NAN, "non-finite norm");
  return GPE_OK;
}

int gpe_gpu_wait_probe(gpe_ctx* c, uint64_t limit_ns) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (limit_ns == 0 || limit_ns > 1000000000ull)
    return fail(c, GPE_ERR_INVALID, "wait probe limit must be in (0, 1 s]");
  wait_probe_kernel<<<1, 32, 0, c->stream>>>(limit_ns, c->d_status);
  CU_CHECK(c, cudaGetLastError());
  c->launches++;
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  return check_status(c);
}

int gpe_gpu_set_wait_limit(gpe_ctx* c, uint64_t limit_ns) {
  if (!c) return GPE_ERR_INVALID;
  c->wait_limit_ns = limit_ns ? (unsigned long long)limit_ns : WAIT_LIMIT_NS;
  cudaStreamSynchronize(c->stream);
  rk45_drop_graphs(c);
  return GPE_OK;
}

int gpe_gpu_test_stall(gpe_ctx* c, int32_t plane) {
  if (!c) return GPE_ERR_INVALID;
  c->stall_plane = plane >= 0 ? plane : -1;
  cudaStreamSynchronize(c->stream);
  rk45_drop_graphs(c);
  return GPE_OK;
}

int gpe_gpu_step_series(gpe_ctx* c, int64_t n, double* dt_did, int32_t* attempts) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (n < 0 || n > c->series_steps)
    return fail(c, GPE_ERR_INVALID, "the last rk45 advance recorded fewer steps");
  if (n == 0) return GPE_OK;
  if (dt_did)
    CU_CHECK(c, cudaMemcpy(dt_did, c->d_ser_dt, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (attempts)
    CU_CHECK(c, cudaMemcpy(attempts, c->d_ser_att, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
  return GPE_OK;
}

int gpe_gpu_diagnostics(gpe_ctx* c, double* mass, double* mom) {
  int rc = check_solo(c);
  if (rc) return rc;
  if (!mass || !mom) return fail(c, GPE_ERR_INVALID, "null output");
  const Geom g = geom(c);
  const int nb = (int)std::min<size_t>((size_t)elementwise_blocks(c->nint), c->partials_cap / 2);
  double c1[3], c2[3];
  const double h[3] = {c->dx, c->dy, c->dz};
  for (int a = 0; a < 3; a++) {
    if (c->prm.order == 2) { c1[a] = 1.0 / (2.0 * h[a]); c2[a] = 0.0; }
    else { c1[a] = 8.0 / (12.0 * h[a]); c2[a] = -1.0 / (12.0 * h[a]); }
  }
  if (c->es == 8)
    diag_kernel<float><<<nb, 256, 0, c->stream>>>((const float*)c->fld[c->psi_id], g, c1[0], c2[0],
                                                  c1[1], c2[1], c1[2], c2[2], c->tabW[0],
                                                  c->tabW[1], c->tabW[2], c->d_partials);
  else
    diag_kernel<double><<<nb, 256, 0, c->stream>>>((const double*)c->fld[c->psi_id], g, c1[0],
                                                   c2[0], c1[1], c2[1], c1[2], c2[2], c->tabW[0],
                                                   c->tabW[1], c->tabW[2], c->d_partials);
  CU_CHECK(c, cudaGetLastError());
  diag_finalize_kernel<<<1, 256, 0, c->stream>>>(c->d_partials, nb, cell_volume(c), c->d_scal + 4);
  CU_CHECK(c, cudaGetLastError());
  c->launches += 2;
  rc = allreduce_scalars(c, 4, 4, 0);
  if (rc) return rc;
  double v[4];
  rc = read_scalars(c, v, 4, 4);
  if (rc) return rc;
  *mass = v[0];
  mom[0] = v[1];
  mom[1] = v[2];
  mom[2] = v[3];
  if (!std::isfinite(v[0])) return fail(c, GPE_ERR_NAN, "non-finite mass");
  return GPE_OK;
}

int gpe_gpu_energy(gpe_ctx* c, double* E, double* H4) {
  int rc = check_solo(c);
  if (rc) return rc;
  if (!E) return fail(c, GPE_ERR_INVALID, "E is null");
  StageSpec s;
  s.stencil = c->psi_id;
  s.epi = EPI_ENERGY;
  s.family = GPE_FAM_ENERGY;
  rc = launch_stage(c, s);
  if (rc) return rc;
  const int nb = c->last_nblk;
  rc = finalize(c, nb, 0, 0, cell_volume(c), 1, false);
  if (rc) return rc;
  rc = finalize(c, nb, 1, 0, cell_volume(c), 2, false);
  if (rc) return rc;
  double v[2];
  rc = read_scalars(c, v, 1, 2);
  if (rc) return rc;
  *E = v[0];
  if (H4) *H4 = v[1];
  return check_status(c);
}

int gpe_gpu_renormalise(gpe_ctx* c, double norm) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!(norm > 0.0)) return fail(c, GPE_ERR_INVALID, "norm must be positive");
  const size_t n = c->npad * 2;
  const int nb = elementwise_blocks(n);
  Launch L{};
  begin_timed(c, L, GPE_FAM_COPY, (int64_t)c->nint);
  if (c->es == 8)
    scale_kernel<float><<<nb, 256, 0, c->stream>>>((float*)c->fld[c->psi_id], n,
                                                     std::sqrt(c->prm.nn), std::sqrt(norm));
  else
    scale_kernel<double><<<nb, 256, 0, c->stream>>>((double*)c->fld[c->psi_id], n,
                                                      std::sqrt(c->prm.nn), std::sqrt(norm));
  CU_CHECK(c, cudaGetLastError());
  end_timed(c, L);
  c->launches++;
  c->norm_valid = false;
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  return GPE_OK;
}

static int rhs_like(gpe_ctx* c, void* out, int32_t elem_bytes, bool lap) {
  int rc = check_solo(c);
  if (rc) return rc;
  rc = check_elem(c, elem_bytes, out);
  if (rc) return rc;
  StageSpec s;
  s.stencil = c->psi_id;
  s.nout = 1;
  s.out[0] = c->alt_id;
  s.a[0] = 1.0;
  s.epi = lap ? EPI_LAP : 0;
  rc = launch_stage(c, s);
  if (rc) return rc;
  rc = stage_out(c, c->alt_id, out, elem_bytes, false);
  if (rc) return rc;
  return check_status(c);
}

int gpe_gpu_rhs(gpe_ctx* c, void* out, int32_t elem_bytes) {
  return rhs_like(c, out, elem_bytes, false);
}

int gpe_gpu_laplacian(gpe_ctx* c, void* out, int32_t elem_bytes) {
  return rhs_like(c, out, elem_bytes, true);
}

int gpe_gpu_set_real_time(gpe_ctx* c, int32_t real_time) {
  if (!c) return GPE_ERR_INVALID;
  c->prm.real_time = real_time ? 1 : 0;
  return GPE_OK;
}

int gpe_gpu_set_timing(gpe_ctx* c, int32_t on) {
  if (!c) return GPE_ERR_INVALID;
  c->timing = on != 0;
  return GPE_OK;
}

int gpe_gpu_get_timing(gpe_ctx* c, gpe_timing* out) {
  int rc = check_ctx(c);
  if (rc) return rc;
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  for (auto& L : c->timed) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, L.a, L.b);
    if (L.family >= 0 && L.family < GPE_TIMING_FAMILIES) {
      c->acc_timing.ms[L.family] += ms;
      c->acc_timing.launches[L.family] += 1;
      c->acc_timing.sites[L.family] += L.sites;
    }
    c->ev_pool.push_back(L.a);
    c->ev_pool.push_back(L.b);
  }
  c->timed.clear();
  if (out) *out = c->acc_timing;
  memset(&c->acc_timing, 0, sizeof(c->acc_timing));
  return GPE_OK;
}

int64_t gpe_gpu_launch_count(const gpe_ctx* c) { return c ? c->launches : -1; }

int64_t gpe_gpu_device_bytes(const gpe_ctx* c) { return c ? c->device_bytes : -1; }

int gpe_gpu_set_slab(gpe_ctx* c, int32_t nz_global, int32_t z_offset) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nz_global < 6 || z_offset < 0 || z_offset + c->nz > nz_global)
    return fail(c, GPE_ERR_INVALID, "slab does not fit in the global z axis");
  if (c->prm.bcs == 2 && c->nz < 4 && nz_global > c->nz)
    return fail(c, GPE_ERR_INVALID, "reflective slabs need at least 4 planes");
  CU_CHECK(c, cudaStreamSynchronize(c->stream));
  rk45_drop_graphs(c);
  c->nzg = nz_global;
  c->z_off = z_offset;
  // get_grid on the global axis, keeping this slab's planes
  c->dz = (c->prm.zr - (-c->prm.zr)) / (double)(nz_global - 1);
  for (int k = 0; k < c->nz; k++) c->z[k] = -c->prm.zr + (double)(z_offset + k) * c->dz;
  if (c->d_tables) {
    cudaFree(c->d_tables);
    c->d_tables = nullptr;
  }
  rc = build_tables(c);
  if (rc) return rc;
  c->norm_valid = false;
  return GPE_OK;
}

int gpe_gpu_comm_unique_id(void* id128) {
  if (!id128) return fail(nullptr, GPE_ERR_INVALID, "id buffer is null");
  std::string why;
  if (!load_nccl(&why)) return fail(nullptr, GPE_ERR_CUDA, why);
  ncclUniqueId id;
  const ncclResult_t r = g_nccl.GetUniqueId(&id);
  if (r != ncclSuccess)
    return fail(nullptr, GPE_ERR_CUDA, std::string("ncclGetUniqueId: ") + g_nccl.GetErrorString(r));
  memcpy(id128, &id, sizeof(id));
  return GPE_OK;
}

int gpe_gpu_comm_init(gpe_ctx* c, const void* id128, int32_t rank, int32_t nranks) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!id128 || nranks < 1 || rank < 0 || rank >= nranks)
    return fail(c, GPE_ERR_INVALID, "bad communicator arguments");
  if (c->comm) return fail(c, GPE_ERR_INVALID, "communicator already set");
  std::string why;
  if (!load_nccl(&why)) return fail(c, GPE_ERR_CUDA, why);
  ncclUniqueId id;
  memcpy(&id, id128, sizeof(id));
  NCCL_CHECK(c, g_nccl.CommInitRank(&c->comm, nranks, id, rank));
  c->rank = rank;
  c->nranks = nranks;
  c->nbr_lo = (rank - 1 + nranks) % nranks;
  c->nbr_hi = (rank + 1) % nranks;
  // periodic: every rank trades both faces (one rank trades with itself);
  // reflective: the bottom and top ranks mirror their outer faces locally
  const bool periodic = c->prm.bcs == 1;
  c->exch_lo = periodic || rank > 0;
  c->exch_hi = periodic || rank < nranks - 1;
  c->norm_valid = false;
  return GPE_OK;
}

void* gpe_gpu_stream(const gpe_ctx* c) {
  return c ? static_cast<void*>(c->stream) : nullptr;
}

void* gpe_gpu_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void gpe_gpu_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

// ----------------------------------------------------------------------------
// In-process slab groups

static int gfail(gpe_group* g, int code, const std::string& msg) {
  if (g) g->err = msg;
  else g_last_create_error = msg;
  return code;
}

int gpe_group_create(gpe_ctx* const* members, int32_t n, gpe_group** out) {
  if (!out || !members || n < 2) return gfail(nullptr, GPE_ERR_INVALID, "a slab group needs >= 2 members");
  *out = nullptr;
  const gpe_ctx* c0 = members[0];
  if (!c0) return gfail(nullptr, GPE_ERR_INVALID, "null member");
  int z = 0;
  for (int r = 0; r < n; r++) {
    const gpe_ctx* c = members[r];
    if (!c) return gfail(nullptr, GPE_ERR_INVALID, "null member");
    if (c->group || c->comm)
      return gfail(nullptr, GPE_ERR_INVALID, "member already in a group or joined to a communicator");
    const gpe_params &a = c->prm, &b = c0->prm;
    if (c->dev != c0->dev || c->nx != c0->nx || c->ny != c0->ny || c->es != c0->es ||
        a.scheme != b.scheme || a.order != b.order || a.bcs != b.bcs ||
        a.eqn_to_solve != b.eqn_to_solve || a.kahan != b.kahan || a.real_time != b.real_time ||
        a.xr != b.xr || a.yr != b.yr || a.zr != b.zr || a.fd_match != b.fd_match ||
        c->nzg != c0->nzg)
      return gfail(nullptr, GPE_ERR_INVALID,
                   "members must share device, nx, ny, precision, scheme, order, boundary, "
                   "equation, time direction, box and global z axis");
    if (c->z_off != z) return gfail(nullptr, GPE_ERR_INVALID, "members must be consecutive z-slabs from z = 0");
    if (c->nz < (c->prm.bcs == 2 ? 4 : 2))
      return gfail(nullptr, GPE_ERR_INVALID, "slab too thin");
    z += c->nz;
  }
  if (z != c0->nzg) return gfail(nullptr, GPE_ERR_INVALID, "slabs do not cover the global z axis");
  gpe_group* g = new gpe_group();
  g->dev = c0->dev;
  if (cudaSetDevice(g->dev) != cudaSuccess ||
      cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&g->d_scal, sizeof(double*) * n) != cudaSuccess) {
    cudaGetLastError();
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
    return gfail(nullptr, GPE_ERR_CUDA, "group stream or scalar table allocation failed");
  }
  std::vector<double*> ptrs;
  for (int r = 0; r < n; r++) {
    gpe_ctx* c = members[r];
    cudaStreamSynchronize(c->stream);
    g->m.push_back(c);
    ptrs.push_back(c->d_scal);
    c->group = g;
    c->own_stream = c->stream;
    c->stream = g->stream;
    c->rank = r;
    c->nranks = n;
    c->nbr_lo = (r - 1 + n) % n;
    c->nbr_hi = (r + 1) % n;
    const bool periodic = c->prm.bcs == 1;
    c->exch_lo = periodic || r > 0;
    c->exch_hi = periodic || r < n - 1;
    c->ghosts_dirty = true;
    c->norm_valid = false;
    c->maps.clear();
    c->shapes.clear();
    rk45_drop_graphs(c);
  }
  cudaMemcpy(g->d_scal, ptrs.data(), sizeof(double*) * n, cudaMemcpyHostToDevice);
  *out = g;
  return GPE_OK;
}

void gpe_group_destroy(gpe_group* g) {
  if (!g) return;
  cudaSetDevice(g->dev);
  cudaStreamSynchronize(g->stream);
  for (gpe_ctx* c : g->m) {
    c->stream = c->own_stream;
    c->group = nullptr;
    c->rank = 0;
    c->nranks = 1;
    c->exch_lo = c->exch_hi = false;
    c->maps.clear();
    c->shapes.clear();
    rk45_drop_graphs(c);
  }
  if (g->d_scal) cudaFree(g->d_scal);
  if (g->xstream) {
    cudaStreamSynchronize(g->xstream);
    cudaStreamDestroy(g->xstream);
  }
  for (auto e : g->xev)
    if (e) cudaEventDestroy(e);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

const char* gpe_group_last_error(const gpe_group* g) {
  return g ? g->err.c_str() : g_last_create_error.c_str();
}

static int group_ready(gpe_group* g) {
  if (!g || g->m.empty()) return gfail(g, GPE_ERR_INVALID, "empty or destroyed group");
  gpe_ctx* c = g->m[0];
  if (cudaSetDevice(g->dev) != cudaSuccess) return gfail(g, GPE_ERR_CUDA, "cudaSetDevice failed");
  bool dirty = false;
  for (gpe_ctx* m : g->m) dirty = dirty || m->ghosts_dirty;
  if (dirty) {
    const int rc = group_exchange(g, c->psi_id);
    if (rc) return gfail(g, rc, c->err);
    for (gpe_ctx* m : g->m) m->ghosts_dirty = false;
  }
  return GPE_OK;
}

int gpe_group_solver(gpe_group* g, gpe_time* tm, gpe_step_info* info) {
  int rc = group_ready(g);
  if (rc) return rc;
  if (!tm) return gfail(g, GPE_ERR_INVALID, "tm is null");
  gpe_ctx* c = g->m[0];
  rc = do_step(c, tm, info);
  if (rc) return gfail(g, rc, c->err);
  if (cudaStreamSynchronize(g->stream) != cudaSuccess)
    return gfail(g, GPE_ERR_CUDA, "group stream synchronisation failed");
  rc = check_status(c);
  if (rc) return gfail(g, rc, c->err);
  for (gpe_ctx* m : g->m) m->norm_valid = c->norm_valid;
  return GPE_OK;
}

int gpe_group_norm(gpe_group* g, double* norm) {
  int rc = group_ready(g);
  if (rc) return rc;
  if (!norm) return gfail(g, GPE_ERR_INVALID, "norm is null");
  gpe_ctx* c = g->m[0];
  if (!c->norm_valid) {
    for (gpe_ctx* m : g->m) {
      const Geom gm = geom(m);
      const int nb = elementwise_blocks(m->nint);
      if (m->es == 8)
        norm_kernel<float><<<nb, 256, 0, g->stream>>>((const float*)m->fld[m->psi_id], gm,
                                                      m->tabW[0], m->tabW[1], m->tabW[2],
                                                      m->d_partials);
      else
        norm_kernel<double><<<nb, 256, 0, g->stream>>>((const double*)m->fld[m->psi_id], gm,
                                                       m->tabW[0], m->tabW[1], m->tabW[2],
                                                       m->d_partials);
      m->launches++;
      rc = finalize_one(m, nb, 0, 0, cell_volume(m), 0, false);
      if (rc) return gfail(g, rc, m->err);
    }
    combine_scalars_kernel<<<1, 32, 0, g->stream>>>(g->d_scal, (int)g->m.size(), 0, 0);
    if (cudaGetLastError() != cudaSuccess) return gfail(g, GPE_ERR_CUDA, "norm launch failed");
  }
  if (cudaMemcpyAsync(norm, c->d_scal, sizeof(double), cudaMemcpyDeviceToHost, g->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(g->stream) != cudaSuccess)
    return gfail(g, GPE_ERR_CUDA, "norm read-back failed");
  for (gpe_ctx* m : g->m) m->norm_valid = true;
  if (!std::isfinite(*norm)) return gfail(g, GPE_ERR_NAN, "non-finite norm");
  return GPE_OK;
}

int gpe_group_energy(gpe_group* g, double* E, double* H4) {
  int rc = group_ready(g);
  if (rc) return rc;
  if (!E) return gfail(g, GPE_ERR_INVALID, "E is null");
  gpe_ctx* c = g->m[0];
  StageSpec s;
  s.stencil = c->psi_id;
  s.epi = EPI_ENERGY;
  s.family = GPE_FAM_ENERGY;
  rc = launch_stage(c, s);
  if (!rc) rc = finalize(c, c->last_nblk, 0, 0, cell_volume(c), 1, false);
  if (!rc) rc = finalize(c, c->last_nblk, 1, 0, cell_volume(c), 2, false);
  double v[2] = {0.0, 0.0};
  if (!rc) rc = read_scalars(c, v, 1, 2);
  if (!rc) rc = check_status(c);
  if (rc) return gfail(g, rc, c->err);
  *E = v[0];
  if (H4) *H4 = v[1];
  return GPE_OK;
}

// ----------------------------------------------------------------------------
// Batched ensembles

void gpe_batch_default_opts(gpe_batch_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->struct_size = (int32_t)sizeof(gpe_batch_opts);
  o->use_graph = 1;
}

int gpe_batch_create(const gpe_params* prms, int32_t nruns, const gpe_batch_opts* opts,
                     gpe_batch** out) {
  if (!out || !prms || nruns < 1) return bfail(nullptr, GPE_ERR_INVALID, "bad batch arguments");
  *out = nullptr;
  gpe_batch_opts o;
  gpe_batch_default_opts(&o);
  if (opts) {
    if (opts->struct_size != (int32_t)sizeof(gpe_batch_opts))
      return bfail(nullptr, GPE_ERR_INVALID, "gpe_batch_opts struct_size mismatch");
    o = *opts;
  }
  if (const char* why = bad_opts(o)) return bfail(nullptr, GPE_ERR_INVALID, why);
  const gpe_params& p0 = prms[0];
  for (int r = 0; r < nruns; r++) {
    const gpe_params& p = prms[r];
    if (p.scheme != GPE_SCHEME_RK4)
      return bfail(nullptr, GPE_ERR_INVALID, "batched ensembles step with scheme rk4");
    if (p.order != p0.order || p.bcs != p0.bcs || p.eqn_to_solve != p0.eqn_to_solve ||
        p.precision != p0.precision || p.kahan != p0.kahan || p.device != p0.device ||
        p.real_time != p0.real_time)
      return bfail(nullptr, GPE_ERR_INVALID,
                   "batch members must share order, bcs, equation, precision, kahan, "
                   "device and time direction");
  }
  gpe_batch* b = new gpe_batch();
  b->opts = o;
  b->dev = p0.device;
  b->es = p0.precision;
  b->R = p0.order / 2;
  b->TY = o.tile_y > 0 ? o.tile_y : 8;
  auto bail = [&](int rc) {
    g_last_create_error = b->err;
    gpe_batch_destroy(b);
    return rc;
  };
  for (int r = 0; r < nruns; r++) {
    gpe_ctx* c = nullptr;
    gpe_params pr = prms[r];
    pr.tile_y = b->TY;
    const int rc = gpe_gpu_create(&pr, &c);
    if (rc) {
      b->err = std::string("member ") + std::to_string(r) + ": " + g_last_create_error;
      return bail(rc);
    }
    b->runs.push_back(c);
    b->form = std::max(b->form, form_of(rhs_form(c)));
    b->sites += (int64_t)c->nint;
  }
  if (cudaSetDevice(b->dev) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    b->err = "stream creation failed";
    return bail(GPE_ERR_CUDA);
  }
  {
    const int rc = batch_plan(b);
    if (rc) return bail(rc);
  }
  std::vector<double> scale;
  for (auto* c : b->runs) scale.push_back(cell_volume(c));
  size_t rdsz = (b->es == 8) ? sizeof(RunDesc<float, float>) : sizeof(RunDesc<double, double>);
  if (cudaMalloc(&b->d_scale, sizeof(double) * nruns) != cudaSuccess ||
      cudaMalloc(&b->d_norm, sizeof(double) * nruns) != cudaSuccess ||
      cudaMalloc(&b->d_counter, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&b->d_status, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    b->err = "cudaMalloc of batch buffers failed";
    return bail(GPE_ERR_OOM);
  }
  for (int k = 0; k < 2; k++)
    for (int s = 0; s < 4; s++)
      if (cudaMalloc(&b->d_rundesc[k][s], rdsz * nruns) != cudaSuccess) {
        cudaGetLastError();
        b->err = "cudaMalloc of run descriptors failed";
        return bail(GPE_ERR_OOM);
      }
  cudaMemcpy(b->d_scale, scale.data(), sizeof(double) * nruns, cudaMemcpyHostToDevice);
  cudaMemset(b->d_counter, 0, sizeof(int));
  cudaMemset(b->d_status, 0, sizeof(int));
  if (cudaDeviceSynchronize() != cudaSuccess) {
    b->err = "device synchronisation failed during batch create";
    return bail(GPE_ERR_CUDA);
  }
  *out = b;
  return GPE_OK;
}

void gpe_batch_destroy(gpe_batch* b) {
  if (!b) return;
  cudaSetDevice(b->dev);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graph(b);
  for (auto* c : b->runs) gpe_gpu_destroy(c);
  for (int k = 0; k < 2; k++)
    for (int s = 0; s < 4; s++)
      if (b->d_rundesc[k][s]) cudaFree(b->d_rundesc[k][s]);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_item_run) cudaFree(b->d_item_run);
  if (b->d_partials) cudaFree(b->d_partials);
  if (b->d_scale) cudaFree(b->d_scale);
  if (b->d_norm) cudaFree(b->d_norm);
  if (b->d_series) cudaFree(b->d_series);
  if (b->d_counter) cudaFree(b->d_counter);
  if (b->d_status) cudaFree(b->d_status);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

const char* gpe_batch_last_error(const gpe_batch* b) {
  if (!b) return g_last_create_error.c_str();
  return b->err.c_str();
}

int gpe_batch_member(gpe_batch* b, int32_t run, gpe_ctx** ctx) {
  if (!b || !ctx || run < 0 || run >= (int32_t)b->runs.size())
    return bfail(b, GPE_ERR_INVALID, "no such batch member");
  *ctx = b->runs[run];
  return GPE_OK;
}

int gpe_batch_advance(gpe_batch* b, int64_t nsteps, double dt_re, double dt_im,
                      double* norms) {
  if (!b || nsteps < 0) return bfail(b, GPE_ERR_INVALID, "bad batch advance arguments");
  BCU(b, cudaSetDevice(b->dev));
  const cd dt(dt_re, dt_im);
  const size_t nr = b->runs.size();
  if ((size_t)nsteps > b->series_cap) {
    batch_drop_graph(b);
    if (b->d_series) cudaFree(b->d_series);
    b->d_series = nullptr;
    const size_t cap = std::max<size_t>((size_t)nsteps, 64);
    BCU(b, cudaMalloc(&b->d_series, sizeof(double) * cap * nr));
    b->series_cap = cap;
  }
  bool moved = false;  // a member was stepped on its own since the batch prepared
  for (size_t r = 0; r < nr && b->prepared; r++)
    moved = moved || b->prepared_psi[r] != b->runs[r]->psi_id;
  if (!b->prepared || dt != b->prepared_dt || moved) {
    batch_drop_graph(b);
    const int rc = batch_prepare(b, dt);
    if (rc) return rc;
  }
  // members' own kernels (state loads) must be done before the batch runs
  for (auto* c : b->runs) BCU(b, cudaStreamSynchronize(c->stream));
  BCU(b, cudaMemsetAsync(b->d_counter, 0, sizeof(int), b->stream));
  for (int par = 0; par < 2 && b->opts.use_graph; par++) {
    if (b->exec[par]) continue;
    BCU(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_enqueue_step(b, par);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return bfail(b, GPE_ERR_CUDA, "graph capture failed");
    b->graph[par] = g;
    BCU(b, cudaGraphInstantiate(&b->exec[par], b->graph[par], 0));
  }
  for (int64_t k = 0; k < nsteps; k++) {
    const int par = (int)(k & 1);
    if (b->exec[par]) {
      BCU(b, cudaGraphLaunch(b->exec[par], b->stream));
    } else {
      const int rc = batch_enqueue_step(b, par);
      if (rc) return rc;
    }
    b->launches += 6;
  }
  if (nsteps & 1) batch_flip(b);
  for (auto* c : b->runs) c->norm_valid = false;
  if (norms && nsteps > 0) {
    // series is [run][cap]: copy the first nsteps of each run
    BCU(b, cudaMemcpy2DAsync(norms, sizeof(double) * nsteps, b->d_series,
                             sizeof(double) * b->series_cap, sizeof(double) * nsteps, nr,
                             cudaMemcpyDeviceToHost, b->stream));
  }
  BCU(b, cudaStreamSynchronize(b->stream));
  int st = 0;
  BCU(b, cudaMemcpy(&st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) return bfail(b, GPE_ERR_TIMEOUT, "device-side wait limit expired in a batched stage");
  return GPE_OK;
}

int gpe_batch_set_opts(gpe_batch* b, const gpe_batch_opts* opts) {
  if (!b || !opts) return bfail(b, GPE_ERR_INVALID, "bad batch arguments");
  if (opts->struct_size != (int32_t)sizeof(gpe_batch_opts))
    return bfail(b, GPE_ERR_INVALID, "gpe_batch_opts struct_size mismatch");
  if (const char* why = bad_opts(*opts)) return bfail(b, GPE_ERR_INVALID, why);
  BCU(b, cudaSetDevice(b->dev));
  BCU(b, cudaStreamSynchronize(b->stream));
  batch_drop_graph(b);
  b->opts = *opts;
  return batch_plan(b);
}

void* gpe_batch_stream(const gpe_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

int64_t gpe_batch_launch_count(const gpe_batch* b) { return b ? b->launches : -1; }

int gpe_batch_info(const gpe_batch* b, int64_t* sites, int32_t* nitems, int32_t* grid,
                   int32_t* tile_y) {
  if (!b) return GPE_ERR_INVALID;
  if (sites) *sites = b->sites;
  if (nitems) *nitems = b->nitems;
  if (grid) *grid = b->st[0][1].grid;
  if (tile_y) *tile_y = b->TY;
  return GPE_OK;
}

}  // extern "C"

