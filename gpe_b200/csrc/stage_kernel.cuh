// stage_kernel.cuh -- the fused finite-difference stage kernel.
//
// One launch evaluates f(u) = get_rhs(u) (src/solve.f90:382-440) for every
// interior site of a stencil field u and combines it with up to MAXP
// pointwise fields into one or two output fields -- one Runge-Kutta stage of
// euler / rk2 / rk4 / rkck (src/solve.f90:57-378) per launch.  Fused in the
// same pass:
//   * the 2nd/4th-order centred Laplacian and x-gradient of
//     src/derivs.f90:25-272 (periodic or reflective), read from ghosted
//     storage;
//   * the boundary ghost fill of the output field, which replaces the MPI
//     halo exchange after every stage (src/variables.f90:186-358);
//   * FP64 block partials of the extended-Simpson norm
//     (src/variables.f90:537-559, 713-823), the rkqs error maximum
//     (src/solve.f90:176-190) or the energy sum (src/variables.f90:563-587).
//
// Tiling: a CTA owns a 64 x TY tile in (x, y) and marches a chunk of
// z-planes.  TY / ROWS compute warps each own ROWS adjacent rows (one, or two
// for the recipes rows_per_warp names; two consecutive x sites per lane);
// one more warp is the producer: its lane 0 issues, plane by plane,
// TMA tile loads (no multicast) of the stencil plane with its halo and of the
// pointwise input tiles into a ring of `stages` shared-memory slots.  A slot
// is handed over on a "full" mbarrier (TMA transaction count) and handed back
// on an "empty" mbarrier that every compute warp arrives on once it no longer
// reads the slot, so no block-wide barrier is taken per plane.  The
// z-neighbours come from a register queue of 2R+1 planes per row (R = order/2),
// rotated by unrolling the plane loop 2R+1 times; x and y neighbours are read
// from the staged halo plane.  Outputs go straight from registers to global
// memory as 16-byte stores.
//
// The combination each stage performs is fixed at compile time ("recipe"):
//   out[o] = alpha[o]*s0 + alpha2[o]*s1 + sum_q beta[o][q]*P_q + a[o] (x) K
// where the stencil field u = s0 (+ s1) is one stored field or the sum of two
// (NS = 2: both staged with their halos and added as they are read, so a
// stage can step psi + d from an increment d without storing psi + d),
// s0 and s1 are those fields at the site, P_q the pointwise inputs, alpha
// and beta real Runge-Kutta weights present only where AMASK/BMASK say so,
// a[o] one complex coefficient per output (it carries dt), and K the
// right-hand side.  Without sponge, gradient or sphere terms the
// right-hand side of every equation is i*B with
// B = cL*lap(u) + (c0 + cV*V + cn|u|^2) u, so K = B and the host folds the
// factor i into a[o]: FORM_PLAIN without a trap (V = 0), FORM_TRAP with
// V = Vx[i] + Vy[j] + Vz[k]; with FORM_FULL K = f(u) is formed site by site
// with every term the equation may have.
#pragma once

#include <type_traits>

#include "device_utils.cuh"
#include "vec2.cuh"

namespace gpe {

constexpr int TX = 64;   // x sites per tile: one warp row, two per lane
constexpr int GH = 2;    // ghost width of every stored field
constexpr int MAXP = 6;  // maximum pointwise inputs of one stage

enum : int {
  EPI_NORM = 1,    // reduce sum w_ijk |out0|^2 into partial slot 0
  EPI_ERR = 2,     // reduce max |err / psi_scal| into partial slot 1
  EPI_KAHAN = 4,   // out0 = psi + delta with compensation, out1 = new c
  EPI_ENERGY = 8,  // no outputs; reduce E (slot 0) and H4 (slot 1)
  EPI_LAP = 16,    // K is the Laplacian itself
};

// Right-hand-side forms of a recipe (see the top of this file).
enum : int { FORM_PLAIN = 0, FORM_TRAP = 1, FORM_FULL = 2 };

// Rows of the tile each compute warp owns.  Two for the complex64 recipes
// that stage two stencil fields and nothing else (rk4 stages 2 and 3, in
// single-run and batched launches):
// their shared-memory loads (both fields at every x and y neighbour) bound
// them, and a warp with two adjacent rows loads the y-neighbour rows the two
// share once (rows -2, -1, +2, +3 of its first row for four, each row's own
// centre serving as the other's nearest neighbour).  Measured at 512^3: the
// stage 0.655 -> 0.605 ms; the one-field stage 1 lost (0.429 -> 0.443 ms:
// instruction-bound, and its warps per SM fell from 27 to 15), so it keeps
// one row per warp.
// A batched launch holds its run descriptor in registers too; with two rows
// its order-4 recipes spill, so batched launches take two rows at order 2.
template <typename TS, typename TC>
__host__ __device__ constexpr int rows_per_warp(int r, int ns, int np, int form, bool batch) {
  return (std::is_same<TS, float>::value && std::is_same<TC, float>::value && ns == 2 &&
          np == 0 && form != FORM_FULL && !(batch && r > 1))
             ? 2
             : 1;
}

struct TileMaps {
  CUtensorMap halo;      // stencil field, box (64+4) x (TY+2R) x 1
  CUtensorMap halo2;     // second stencil field (NS = 2), same box
  CUtensorMap pt[MAXP];  // pointwise fields, box 64 x TY x 1
};

// Everything one run contributes to a stage launch: its geometry, fields,
// tensor maps, discretisation coefficients and tables.
template <typename TS, typename TC>
struct alignas(64) RunDesc {
  TileMaps maps;        // 64-byte aligned tensor maps (first member)
  int nx, ny, nz;       // interior extents
  int Nx, Ny;           // padded pitches (complex elements)
  int ntx, nty, zchunk, nchunks;
  int bcs;
  int zg_lo, zg_hi;     // fill the z ghosts below / above locally (else a
                        // neighbouring rank sends them)
  const TS* stencil;    // stencil field (padded layout), warm-up planes
  const TS* stencil2;   // second stencil field (NS = 2)
  TS* out[2];           // output fields (padded layout)
  // Laplacian: T = sum_axes c1*(f1+f-1) + c2*(f2+f-2); L = T + c0*f0
  TC cx1, cx2, cy1, cy2, cz1, cz2, c0lap;
  // x gradient: gx1*(f1-f-1) + gx2*(f2-f-2)
  TC gx1, gx2;
  // FULL: f = m * ( A*(cL*L + (c0 + cV*V + cn*|u|^2) u) + U*u_x ),
  //       A = (ar0 + ard*diss) + i*ai
  // plain: K = cL*L + (c0 + cn*|u|^2) u   (the factor i is folded into a[o])
  TC ar0, ard, ai, cL, c0, cV, cn, U;
  int use_diss, use_V, use_sphere, use_grad;
  const TC* tabV[3];      // per-axis trap terms, V = Vx[i]+Vy[j]+Vz[k]
  const TC* tabD[3];      // per-axis sponge terms (times diss_amp)
  const double* tabW[3];  // per-axis norm weights
  const double* tabX[3];  // coordinates (sphere mask)
  double eg, emu;         // energy: g, mu
};

// A work item: run, tile (tile_x + ntx * tile_y) and z range [z0, z1).
struct WorkItem {
  int run, tile, z0, z1;
};

template <typename TS, typename TC>
struct StageParams {
  RunDesc<TS, TC> run;           // single-run launch: item i = (tile, chunk)
  const RunDesc<TS, TC>* runs;   // batched launch: per-run descriptors
  const WorkItem* items;         // batched launch: the work list
  int nitems;
  // single-run launch: planes [zr[0], zr[1]) in nch_a chunks, then planes
  // [zr[2], zr[3]) (a slab's boundary planes, or its interior, alone)
  int zr[4], nch_a;
  int TY, stages;
  unsigned int halo_box_bytes, pt_box_bytes;    // bytes one TMA box delivers
  unsigned int halo_smem_bytes, pt_smem_bytes;  // 128-aligned slot strides
  int ghost_mask;       // bit o set: out[o] gets its boundary ghosts filled
  TC alpha[2];           // weight of stencil field 0 at the site
  TC alpha2[2];          // weight of stencil field 1 at the site (NS = 2)
  TC beta[2][MAXP];
  TC a_r[2], a_i[2];
  // rkqs error: err = sum_q ce[q]*P_q + cek (x) K (FP64)
  double ce[MAXP], cek_r, cek_i;
  double dt0_r, dt0_i;    // dt of the first attempt (psi_scal)
  double inv_absdt;       // 1/|dt| of this attempt (|f(psi)| = |k1|/|dt|)
  double* partials;       // 2 doubles per work item
  int* status;
  unsigned long long wait_limit_ns;
  int stall_plane;        // >= 0: failure-detection test, the producer stops
                          // issuing when it reaches this plane of an item
  // rk45 with device step control: dt lives in device memory ([0..1] dt of
  // this attempt, [2..3] dt of the step's first attempt) and a[o] =
  // a_mul[o] dt, cek = cek_mul dt (times i when fold), replacing a_r, a_i,
  // cek_r, cek_i, dt0_r, dt0_i and inv_absdt above
  const double* dyn;
  double a_mul[2], cek_mul;
  int fold;
};

__device__ __forceinline__ bool near_edge(int i, int n) {
  return i < 3 || i >= n - 3;
}

template <int K>
using IC = std::integral_constant<int, K>;

// The kernel body; the __global__ entries below differ only in their
// register budget.
template <typename TS, typename TC, int R, int NS, int NP, int NOUT, int EPI, int AMASK,
          int BMASK, int FORM, bool BATCH>
__device__ __forceinline__ void stage_body(const StageParams<TS, TC>& p) {
  using V = typename VT<TC>::T;
  using RD = RunDesc<TS, TC>;
  constexpr bool FULL = FORM == FORM_FULL, TRAP = FORM == FORM_TRAP;
  constexpr int ROWS = rows_per_warp<TS, TC>(R, NS, NP, FORM, BATCH);
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int s_abort, s_issued, s_stop;
  __shared__ double s_red[2][32];

  constexpr int W = (int)(sizeof(TS) / 4);  // 8-byte TMA units per complex
  constexpr int HW = TX + 4;                // halo tile row width (complex)
  constexpr int QN = 2 * R + 1;             // z-queue length
  constexpr unsigned ES = 2 * sizeof(TS);   // bytes per stored complex
  const int TY = p.TY, S = p.stages;
  const int NW = TY / ROWS;  // compute warps; warp NW is the producer
  const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;

  // item it -> run descriptor, tile and z range
  auto item_of = [&](int it) -> WorkItem {
    if (BATCH) return p.items[it];
    // the chunks of the launch's first z range, then those of its second
    const int ntiles = p.run.ntx * p.run.nty;
    const int ch = it / ntiles;
    const bool first = ch < p.nch_a;
    const int z0 = (first ? p.zr[0] : p.zr[2]) + (first ? ch : ch - p.nch_a) * p.run.zchunk;
    return WorkItem{0, it - ch * ntiles, z0, min(z0 + p.run.zchunk, first ? p.zr[1] : p.zr[3])};
  };
  auto run_of = [&](const WorkItem& w) -> const RD& {
    if (BATCH) return p.runs[w.run];
    return p.run;
  };

  // shared memory: full[S] and empty[S] barriers (S <= 8), then the slots
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + 8;
  unsigned char* sbase = smem + 128;
  const unsigned hstride = (unsigned)NS * p.halo_smem_bytes;  // halo boxes of a slot
  const unsigned stride = hstride + (unsigned)NP * p.pt_smem_bytes;

  if (tid == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], (uint32_t)NW);
    }
    fence_mbar_init();
    s_abort = 0;
    s_issued = 0;
    s_stop = 0;
  }
  __syncthreads();

  if (ty == NW) {
    // ---------------- producer warp: lane 0 streams the planes -------------
    // Planes of successive items follow each other through the ring, so the
    // next item's first planes load while the current item drains.
    if (lane == 0) {
      int slot = 0, issued = 0;
      uint32_t cyc = 0;  // completed passes over the ring
      bool stop = false;
      for (int it = blockIdx.x; it < p.nitems && !stop; it += gridDim.x) {
        const WorkItem w = item_of(it);
        const RD& rd = run_of(w);
        const int tile_x = w.tile % rd.ntx, tile_y = w.tile / rd.ntx;
        const int niters = (w.z1 - w.z0) + R;
        prefetch_tmap(&rd.maps.halo);
        if (NS == 2) prefetch_tmap(&rd.maps.halo2);
#pragma unroll
        for (int qq = 0; qq < NP; qq++) prefetch_tmap(&rd.maps.pt[qq]);
        for (int u = 0; u < niters; u++) {
          if (u == p.stall_plane) {
            // the plane is never loaded: the compute warps' wait for it runs
            // out and takes the abort path
            stop = true;
            break;
          }
          if (cyc > 0) {
            // the slot's previous plane must have been released by every
            // compute warp
            if (!mbar_wait_bounded(&empty[slot], (cyc - 1) & 1u, p.wait_limit_ns)) {
              s_abort = 1;
              atomicExch(p.status, 6);
              stop = true;
              break;
            }
            fence_proxy_async();
          }
          unsigned char* st = sbase + (size_t)slot * stride;
          const bool with_pt = (NP > 0) && (u >= R);
          mbar_arrive_expect_tx(&full[slot],
                                NS * p.halo_box_bytes + (with_pt ? NP * p.pt_box_bytes : 0u));
          tma_load_3d(st, &rd.maps.halo, &full[slot], W * tile_x * TX,
                      tile_y * TY + GH - R, w.z0 + u + GH);
          if (NS == 2)
            tma_load_3d(st + p.halo_smem_bytes, &rd.maps.halo2, &full[slot], W * tile_x * TX,
                        tile_y * TY + GH - R, w.z0 + u + GH);
          if (with_pt) {
#pragma unroll
            for (int qq = 0; qq < NP; qq++)
              tma_load_3d(st + hstride + (size_t)qq * p.pt_smem_bytes,
                          &rd.maps.pt[qq], &full[slot], W * (tile_x * TX + GH),
                          tile_y * TY + GH, w.z0 + u - R + GH);
          }
          s_issued = ++issued;
          if (++slot == S) {
            slot = 0;
            ++cyc;
          }
          if (*(volatile int*)&s_abort) {
            stop = true;
            break;
          }
        }
      }
    }
  } else {
  // ------------------------------ compute warps ------------------------------
  int slot = 0, cslot = 0;
  uint32_t phase = 0;
  // the warp's first row; row rr of the warp sits rr rows further on
  const unsigned row_off = ES * (unsigned)((ty * ROWS + R) * HW + 2 * lane + 2);
  const unsigned pt_off = ES * (unsigned)(ty * ROWS * TX + 2 * lane);
  V ar[2], aix[2], alv[2], alv2[2], bev[2][NP > 0 ? NP : 1];
  TC a_re[2] = {p.a_r[0], p.a_r[1]}, a_im[2] = {p.a_i[0], p.a_i[1]};
  double cek_r = p.cek_r, cek_i = p.cek_i, dt0_r = p.dt0_r, dt0_i = p.dt0_i,
         inv_absdt = p.inv_absdt;
  if (p.dyn) {
    // the same arithmetic as the host's coefficient set-up: m * dt, and for
    // fold the complex product (0, 1) * (m dt)
    const double dr = p.dyn[0], di = p.dyn[1];
    auto coef = [&](double mul, double& cr, double& ci) {
      const double xr = __dmul_rn(mul, dr), xi = __dmul_rn(mul, di);
      if (p.fold) {
        cr = __dsub_rn(__dmul_rn(0.0, xr), xi);
        ci = __dadd_rn(__dmul_rn(0.0, xi), xr);
      } else {
        cr = xr;
        ci = xi;
      }
    };
#pragma unroll
    for (int o = 0; o < 2; o++) {
      double cr, ci;
      coef(p.a_mul[o], cr, ci);
      a_re[o] = (TC)cr;
      a_im[o] = (TC)ci;
    }
    coef(p.cek_mul, cek_r, cek_i);
    dt0_r = p.dyn[2];
    dt0_i = p.dyn[3];
    inv_absdt = __drcp_rn(hypot(dr, di));
  }
#pragma unroll
  for (int o = 0; o < 2; o++) {
    ar[o] = vsplat(a_re[o]);
    aix[o] = vpair(-a_im[o], a_im[o]);
    alv[o] = vsplat(p.alpha[o]);
    alv2[o] = vsplat(p.alpha2[o]);
#pragma unroll
    for (int qq = 0; qq < (NP > 0 ? NP : 1); qq++) bev[o][qq] = vsplat(p.beta[o][qq]);
  }
  const V mone = vsplat(TC(-1));

  for (int it = blockIdx.x; it < p.nitems; it += gridDim.x) {
  const WorkItem w = item_of(it);
  const RD& rd = run_of(w);
  const int nx = rd.nx, ny = rd.ny, nz = rd.nz, bcs = rd.bcs;
  const int zg_lo = rd.zg_lo, zg_hi = rd.zg_hi;
  const int tile_x = w.tile % rd.ntx, tile_y = w.tile / rd.ntx;
  const int z0 = w.z0;
  const int niters = (w.z1 - w.z0) + R;
  const int i0 = tile_x * TX + 2 * lane;
  const int j0 = tile_y * TY + ty * ROWS;  // the warp's first row
  bool ok0[ROWS], ok1[ROWS];
#pragma unroll
  for (int rr = 0; rr < ROWS; rr++) {
    ok0[rr] = (i0 < nx) && (j0 + rr < ny);
    ok1[rr] = (i0 + 1 < nx) && (j0 + rr < ny);
  }
  const size_t Nx = (size_t)rd.Nx, NxNy = (size_t)rd.Nx * (size_t)rd.Ny;
  TS* const outp[2] = {rd.out[0], rd.out[1]};
  const TC c0s = rd.c0, cns = rd.cn, cVs = rd.cV, ar0 = rd.ar0, ard = rd.ard, ais = rd.ai;
  const TC Us = rd.U, gx1 = rd.gx1, gx2 = rd.gx2;
  const int useV = rd.use_V, useD = rd.use_diss, useS = rd.use_sphere, useG = rd.use_grad;
  const TC* const tabVz = rd.tabV[2];
  const TC* const tabDz = rd.tabD[2];
  const double* const tabWz = rd.tabW[2];
  const double eg = rd.eg, emu = rd.emu;
  const V cx1 = vsplat(rd.cx1), cx2 = vsplat(rd.cx2), cy1 = vsplat(rd.cy1),
          cy2 = vsplat(rd.cy2), cz1 = vsplat(rd.cz1), cz2 = vsplat(rd.cz2),
          c0l = vsplat(rd.c0lap), cLv = vsplat(rd.cL);
  double red0 = 0.0, red1 = 0.0;

  // Per-thread constants of this item, per row.
  TC Vxy[ROWS][2], Dxy[ROWS][2];
  double Wxy[ROWS][2];
  // Ghost copies this thread's sites feed, as element offsets from the site
  // (x and y fixed per thread and row; z per plane, uniform across the CTA).
  int gxo[2][2], gyo[ROWS][2];
  bool edge_xy[ROWS];
  {
    int a, b;
    for (int e = 0; e < 2; e++) {
      ghost_targets(i0 + e, nx, bcs, a, b);
      gxo[e][0] = (a != NO_GHOST) ? a - (i0 + e) : 0;
      gxo[e][1] = (b != NO_GHOST) ? b - (i0 + e) : 0;
    }
#pragma unroll
    for (int rr = 0; rr < ROWS; rr++) {
      const int j = j0 + rr;
      Vxy[rr][0] = Vxy[rr][1] = Dxy[rr][0] = Dxy[rr][1] = TC(0);
      Wxy[rr][0] = Wxy[rr][1] = 0.0;
      if (TRAP || ((FULL || (EPI & EPI_ENERGY)) && useV)) {
        Vxy[rr][0] = rd.tabV[0][i0] + rd.tabV[1][j];
        Vxy[rr][1] = rd.tabV[0][i0 + 1] + rd.tabV[1][j];
      }
      if (FULL && useD) {
        Dxy[rr][0] = rd.tabD[0][i0] + rd.tabD[1][j];
        Dxy[rr][1] = rd.tabD[0][i0 + 1] + rd.tabD[1][j];
      }
      if (EPI & EPI_NORM) {
        Wxy[rr][0] = rd.tabW[0][i0] * rd.tabW[1][j];
        Wxy[rr][1] = rd.tabW[0][i0 + 1] * rd.tabW[1][j];
      }
      ghost_targets(j, ny, bcs, a, b);
      gyo[rr][0] = (a != NO_GHOST) ? (a - j) * rd.Nx : 0;
      gyo[rr][1] = (b != NO_GHOST) ? (b - j) * rd.Nx : 0;
      edge_xy[rr] = (gxo[0][0] | gxo[0][1] | gxo[1][0] | gxo[1][1] | gyo[rr][0] | gyo[rr][1]) != 0;
    }
  }
  // element offset of this thread's first site (first row) in plane z0
  size_t base = (size_t)(z0 + GH) * NxNy + (size_t)(j0 + GH) * Nx + (size_t)(i0 + GH);

  // z-queues, one per row: physical slot of push number c is c % QN; after
  // push c the plane d above the one being computed sits in slot
  // (c + 1 + R + d) % QN.
  CPair<TC> q[ROWS][QN];
#pragma unroll
  for (int rr = 0; rr < ROWS; rr++) {
#pragma unroll
    for (int w = 0; w < R; w++) {
      CPair<TC> v = {vsplat(TC(0)), vsplat(TC(0))};
      if (ok0[rr]) {
        const size_t off = 2 * (base + rr * Nx - (size_t)(R - w) * NxNy);
        v = ld_cpair<TS, TC>(rd.stencil + off);
        if (NS == 2) {
          const CPair<TC> v2 = ld_cpair<TS, TC>(rd.stencil2 + off);
          v = {vadd(v.a, v2.a), vadd(v.b, v2.b)};
        }
      }
      q[rr][w] = v;
    }
#pragma unroll
    for (int w = R; w < QN; w++) q[rr][w] = {vsplat(TC(0)), vsplat(TC(0))};
  }

  int t = 0;

  auto step = [&](auto kc) -> bool {
    constexpr int KK = decltype(kc)::value;
    if (t >= niters) return false;
    if (!mbar_wait_bounded(&full[slot], phase, p.wait_limit_ns)) {
      s_abort = 1;
      atomicExch(p.status, 6);
      return false;
    }
#pragma unroll
    for (int rr = 0; rr < ROWS; rr++) {
      // the stencil value is the sum of the NS stencil fields
      const unsigned char* sp = sbase + (size_t)slot * stride + row_off + ES * rr * HW;
      CPair<TC> v = ld_cpair<TS, TC>(reinterpret_cast<const TS*>(sp));
      if (NS == 2) {
        const CPair<TC> v2 =
            ld_cpair<TS, TC>(reinterpret_cast<const TS*>(sp + p.halo_smem_bytes));
        v = {vadd(v.a, v2.a), vadd(v.b, v2.b)};
      }
      q[rr][(R + KK) % QN] = v;
    }
    if (t >= R) {
      const int z = z0 + t - R;
      const unsigned char* hc = sbase + (size_t)cslot * stride + row_off;
      auto lds = [&](int drow, int dcol) {
        const unsigned char* a = hc + (int)ES * (drow * HW + dcol);
        CPair<TC> v = ld_cpair<TS, TC>(reinterpret_cast<const TS*>(a));
        if (NS == 2) {
          const CPair<TC> v2 = ld_cpair<TS, TC>(reinterpret_cast<const TS*>(a + p.halo_smem_bytes));
          v = {vadd(v.a, v2.a), vadd(v.b, v2.b)};
        }
        return v;
      };
      auto zq = [&](int rr, int d) -> const CPair<TC>& {
        return q[rr][(R + KK + 1 + R + d + 2 * QN) % QN];
      };
      // y-neighbour rows of the warp's rows, each loaded once: the rows
      // below (-R.. -1 relative to its first row) and above (ROWS..
      // ROWS-1+R) from the halo box; its own rows are their z-queue centres
      CPair<TC> ylo[R], yhi[R];
#pragma unroll
      for (int k = 0; k < R; k++) {
        ylo[k] = lds(k - R, 0);
        yhi[k] = lds(ROWS + k, 0);
      }
      auto yrow = [&](int dr) -> const CPair<TC>& {
        return dr < 0 ? ylo[R + dr] : dr >= ROWS ? yhi[dr - ROWS] : zq(dr, 0);
      };
      TC Vz = TC(0), Dz = TC(0);
      double Wz = 0.0;
      if (TRAP || ((FULL || (EPI & EPI_ENERGY)) && useV)) Vz = tabVz[z];
      if (FULL && useD) Dz = tabDz[z];
      if (EPI & EPI_NORM) Wz = tabWz[z];
      // z ghosts this plane feeds (element offsets): once per plane for
      // several rows, at the store for one (fewer registers held through
      // the stencil)
      auto z_ghosts = [&](long* gzo) {
        gzo[0] = gzo[1] = 0;
        if (near_edge(z, nz)) {
          int a, b;
          ghost_targets(z, nz, bcs, a, b);
          if (a != NO_GHOST && !((a < 0) ? zg_lo : zg_hi)) a = NO_GHOST;
          if (b != NO_GHOST && !((b < 0) ? zg_lo : zg_hi)) b = NO_GHOST;
          gzo[0] = (a != NO_GHOST) ? (long)(a - z) * (long)NxNy : 0;
          gzo[1] = (b != NO_GHOST) ? (long)(b - z) * (long)NxNy : 0;
        }
      };
      long gzo_plane[2] = {0, 0};
      if (ROWS > 1 && !(EPI & EPI_ENERGY)) z_ghosts(gzo_plane);

#pragma unroll
      for (int rr = 0; rr < ROWS; rr++) {
        const unsigned char* hr = hc + ES * rr * HW;  // the row's centre
        // NS = 2: the two stencil fields at the site, kept apart for the
        // pointwise part of the recipe
        CPair<TC> sc0, sc1;
        if (NS == 2) {
          sc0 = ld_cpair<TS, TC>(reinterpret_cast<const TS*>(hr));
          sc1 = ld_cpair<TS, TC>(reinterpret_cast<const TS*>(hr + p.halo_smem_bytes));
        }
        const CPair<TC> xa = lds(rr, -2);
        const CPair<TC> xc = lds(rr, 2);
        const CPair<TC>& yp1 = yrow(rr + 1);
        const CPair<TC>& ym1 = yrow(rr - 1);
        const CPair<TC>& yp2 = yrow(R == 2 ? rr + 2 : rr + 1);
        const CPair<TC>& ym2 = yrow(R == 2 ? rr - 2 : rr - 1);
        CPair<TC> P[NP > 0 ? NP : 1];
        if (NP > 0) {
          const unsigned char* pb =
              sbase + (size_t)slot * stride + hstride + pt_off + ES * rr * TX;
#pragma unroll
          for (int qq = 0; qq < NP; qq++)
            P[qq] = ld_cpair<TS, TC>(reinterpret_cast<const TS*>(pb + (size_t)qq * p.pt_smem_bytes));
        }

        V res[2][2];  // [output][site]
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const CPair<TC>& ctr = zq(rr, 0);
          const V f0 = e ? ctr.b : ctr.a;
          const V xm1 = e ? ctr.a : xa.b, xp1 = e ? xc.a : ctr.b;
          const V xm2 = e ? xa.b : xa.a, xp2 = e ? xc.b : xc.a;
          V L = vmul(cx1, vadd(xp1, xm1));
          L = vfma(cy1, vadd(e ? yp1.b : yp1.a, e ? ym1.b : ym1.a), L);
          L = vfma(cz1, vadd(e ? zq(rr, 1).b : zq(rr, 1).a, e ? zq(rr, -1).b : zq(rr, -1).a), L);
          if (R == 2) {
            L = vfma(cx2, vadd(xp2, xm2), L);
            L = vfma(cy2, vadd(e ? yp2.b : yp2.a, e ? ym2.b : ym2.a), L);
            L = vfma(cz2, vadd(e ? zq(rr, 2).b : zq(rr, 2).a, e ? zq(rr, -2).b : zq(rr, -2).a), L);
          }
          L = vfma(c0l, f0, L);
          const bool ok = e ? ok1[rr] : ok0[rr];

          if (EPI & EPI_ENERGY) {
            if (ok) {
              const double lr = (double)L.x, li = (double)L.y;
              const double fr = (double)f0.x, fi = (double)f0.y;
              const double d2 = fr * fr + fi * fi;
              const double kin = -(lr * fr + li * fi);
              red0 += kin + 0.5 * (d2 * d2);
              red1 += 0.5 * kin + (double)(Vxy[rr][e] + Vz) * d2 + 0.5 * eg * d2 * d2 -
                      emu * d2;
            }
            continue;
          }

          const TC a2 = fma(f0.y, f0.y, f0.x * f0.x);
          V Kv;
          if (EPI & EPI_LAP) {
            Kv = L;
          } else if (!FULL) {
            const TC s = TRAP ? fma(cns, a2, fma(cVs, Vxy[rr][e] + Vz, c0s)) : fma(cns, a2, c0s);
            Kv = vfma(vsplat(s), f0, vmul(cLv, L));
          } else {
            const TC Vs = useV ? Vxy[rr][e] + Vz : TC(0);
            const TC s = c0s + cVs * Vs + cns * a2;
            const V B = vfma(vsplat(s), f0, vmul(cLv, L));
            const TC arr = useD ? ar0 + ard * (Dxy[rr][e] + Dz) : ar0;
            Kv = vfma(vsplat(arr), B, vmul(vpair(-ais, ais), vswap(B)));
            if (useG) {
              V gx = vmul(vsplat(gx1), vfma(xm1, mone, xp1));
              if (R == 2) gx = vfma(vsplat(gx2), vfma(xm2, mone, xp2), gx);
              Kv = vfma(vsplat(Us), gx, Kv);
            }
            if (useS) {
              const double X = rd.tabX[0][i0 + e], Y = rd.tabX[1][j0 + rr], Z = rd.tabX[2][z];
              const TC m = (TC)(0.5 * (1.0 + tanh(sqrt(X * X + Y * Y + Z * Z) - 10.0 - 2.0)));
              Kv = vmul(vsplat(m), Kv);
            }
          }

          const V Ks = vswap(Kv);
#pragma unroll
          for (int o = 0; o < NOUT; o++) {
            // smallest terms first: a (x) K, field 1, pointwise, field 0
            V v = vfma(ar[o], Kv, vmul(aix[o], Ks));
            if (NS == 2 && (AMASK & (4 << o))) v = vfma(alv2[o], e ? sc1.b : sc1.a, v);
#pragma unroll
            for (int qq = 0; qq < NP; qq++)
              if (BMASK & (1 << (o * 8 + qq))) v = vfma(bev[o][qq], e ? P[qq].b : P[qq].a, v);
            if (AMASK & (1 << o)) v = vfma(alv[o], NS == 2 ? (e ? sc0.b : sc0.a) : f0, v);
            res[o][e] = v;
          }

          if (EPI & EPI_KAHAN) {
            // res[0] is the increment delta; compensated add to psi.  Slots:
            // psi = P[0] when NP >= 2 (else the stencil field), c = P[NP-1].
            // psi: stencil field 0 at the site when there are two, else
            // P[0] when NP >= 2, else the stencil field
            const V psi = (NS == 2) ? (e ? sc0.b : sc0.a)
                                    : (NP >= 2) ? (e ? P[0].b : P[0].a) : f0;
            const V cc = e ? P[NP > 0 ? NP - 1 : 0].b : P[NP > 0 ? NP - 1 : 0].a;
            const V y = vfma(cc, mone, res[0][e]);
            const V tt = vadd(psi, y);
            res[1][e] = vfma(y, mone, vfma(psi, mone, tt));
            res[0][e] = tt;
          }

          if (ok && (EPI & EPI_NORM)) {
            const double vr = (double)res[0][e].x, vi = (double)res[0][e].y;
            red0 = fma(Wxy[rr][e] * Wz, fma(vr, vr, vi * vi), red0);
          }
          if (ok && (EPI & EPI_ERR)) {
            // err = sum_q ce[q] P_q + cek (x) K; psi = P[0], k1 = P[1]
            const double kr = (double)Kv.x, ki = (double)Kv.y;
            double er = cek_r * kr - cek_i * ki;
            double ei = cek_r * ki + cek_i * kr;
#pragma unroll
            for (int qq = 1; qq < NP; qq++) {
              const V pv = e ? P[qq].b : P[qq].a;
              er = fma(p.ce[qq], (double)pv.x, er);
              ei = fma(p.ce[qq], (double)pv.y, ei);
            }
            const V psi0 = e ? P[0].b : P[0].a;
            const V k1 = e ? P[NP > 1 ? 1 : 0].b : P[NP > 1 ? 1 : 0].a;
            const double apsi = hypot((double)psi0.x, (double)psi0.y);
            const double m = hypot((double)k1.x, (double)k1.y) * inv_absdt;
            const double sr = apsi + dt0_r * m + 1e-30, si = dt0_i * m;
            red1 = fmax(red1, hypot(er, ei) / hypot(sr, si));
          }
        }

        if (!(EPI & EPI_ENERGY)) {
          long gzo[2] = {gzo_plane[0], gzo_plane[1]};
          if (ROWS == 1) z_ghosts(gzo);
          const bool edge = edge_xy[rr] || ((gzo[0] | gzo[1]) != 0);
#pragma unroll
          for (int o = 0; o < NOUT; o++) {
            TS* out = outp[o] + 2 * (base + rr * Nx);
            if (ok1[rr]) {
              st_cpair<TS, typename VT<TS>::T>(out, cvt_v<TS>(res[o][0]),
                                                cvt_v<TS>(res[o][1]));
            } else if (ok0[rr]) {
              st_c1<TS>(out, res[o][0]);
            }
            if (edge && (p.ghost_mask & (1 << o))) {
#pragma unroll
              for (int e = 0; e < 2; e++) {
                if (!(e ? ok1[rr] : ok0[rr])) continue;
                TS* o1 = out + 2 * e;
                const V v = res[o][e];
                if (gxo[e][0]) st_c1<TS>(o1 + 2 * (ptrdiff_t)gxo[e][0], v);
                if (gxo[e][1]) st_c1<TS>(o1 + 2 * (ptrdiff_t)gxo[e][1], v);
                if (gyo[rr][0]) st_c1<TS>(o1 + 2 * (ptrdiff_t)gyo[rr][0], v);
                if (gyo[rr][1]) st_c1<TS>(o1 + 2 * (ptrdiff_t)gyo[rr][1], v);
                if (gzo[0]) st_c1<TS>(o1 + 2 * gzo[0], v);
                if (gzo[1]) st_c1<TS>(o1 + 2 * gzo[1], v);
              }
            }
          }
        }
      }  // rows

      base += NxNy;
    }
    if (t >= R) {
      // this warp no longer reads plane t-R's slot
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[cslot]);
      if (++cslot == S) cslot = 0;
    }
    if (++slot == S) {
      slot = 0;
      phase ^= 1u;
    }
    ++t;
    return true;
  };

  while (!*(volatile int*)&s_abort) {
    if (!step(IC<0>())) break;
    if (!step(IC<1>())) break;
    if (!step(IC<2>())) break;
    if constexpr (QN > 3) {
      if (!step(IC<3>())) break;
      if (!step(IC<4>())) break;
    }
  }
  // A warp whose wait ran out (or that saw another's) leaves the item early.
  const bool aborted = t < niters;
  if (!aborted) {
    // Hand back the item's last R planes, still held for their x/y
    // neighbours.
#pragma unroll
    for (int k = 0; k < R; k++) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[cslot]);
      if (++cslot == S) cslot = 0;
    }
  }

  if (EPI & (EPI_NORM | EPI_ERR | EPI_ENERGY)) {
    // Per-item partials; only the compute warps take part (named barrier 1).
    // Every compute warp reaches both barriers of every item it starts, an
    // aborted one included, and all of them leave the item loop on the same
    // decision (s_stop, read once between the barriers), so no warp can be
    // left waiting at a barrier that a sibling will never reach.
    red0 = warp_sum(red0);
    red1 = (EPI & EPI_ERR) ? warp_max(red1) : warp_sum(red1);
    if (lane == 0) {
      s_red[0][ty] = red0;
      s_red[1][ty] = red1;
    }
    named_barrier_sync(1, 32 * NW);
    if (tid == 0) {
      double a = 0.0, b = 0.0;
      for (int w2 = 0; w2 < NW; w2++) {
        a += s_red[0][w2];
        b = (EPI & EPI_ERR) ? fmax(b, s_red[1][w2]) : b + s_red[1][w2];
      }
      p.partials[2 * (size_t)it + 0] = a;
      p.partials[2 * (size_t)it + 1] = b;
      s_stop = *(volatile int*)&s_abort;
    }
    named_barrier_sync(1, 32 * NW);
    if (*(volatile int*)&s_stop) break;
  } else if (aborted) {
    break;  // no barrier among the compute warps in this recipe
  }
  }  // items
  }  // compute warps

  __syncthreads();
  // After a timed-out wait, let the copies already in flight land (bounded)
  // before the CTA's shared memory is released: the last load issued into
  // each slot completes phase (u / S) of that slot's full barrier.  This
  // wait has its own limit of at least 2 s, so that a short wait limit set
  // for the pipeline cannot release shared memory under a copy in flight.
  if (s_abort && tid == 0) {
    const int issued = s_issued;
    const unsigned long long drain =
        p.wait_limit_ns > 2000000000ull ? p.wait_limit_ns : 2000000000ull;
    for (int u = max(0, issued - S); u < issued; u++)
      mbar_wait_bounded(&full[u % S], (uint32_t)((u / S) & 1), drain);
  }
}

// Budget left to the compiler (one to two CTAs per SM, by shared memory).
template <typename TS, typename TC, int R, int NS, int NP, int NOUT, int EPI, int AMASK,
          int BMASK, int FORM, bool BATCH>
__global__ void __launch_bounds__(288)
    stage_kernel(const __grid_constant__ StageParams<TS, TC> p) {
  stage_body<TS, TC, R, NS, NP, NOUT, EPI, AMASK, BMASK, FORM, BATCH>(p);
}

// Registers capped for three resident CTAs per SM: the complex64 recipes
// that stage only stencil planes, whose warps mostly wait on fixed-latency
// and shared-memory dependencies, so more warps per scheduler hide more of
// it (their three rings of slots fit in shared memory).  One row per warp:
// 8 compute warps + the producer.
template <typename TS, typename TC, int R, int NS, int NP, int NOUT, int EPI, int AMASK,
          int BMASK, int FORM, bool BATCH>
__global__ void __launch_bounds__(288, 3)
    stage_kernel_occ3(const __grid_constant__ StageParams<TS, TC> p) {
  stage_body<TS, TC, R, NS, NP, NOUT, EPI, AMASK, BMASK, FORM, BATCH>(p);
}

// The same for the two-row recipes (rows_per_warp == 2): 4 compute warps +
// the producer on an 8-row tile, three CTAs per SM.
template <typename TS, typename TC, int R, int NS, int NP, int NOUT, int EPI, int AMASK,
          int BMASK, int FORM, bool BATCH>
__global__ void __launch_bounds__(160, 3)
    stage_kernel_rows2(const __grid_constant__ StageParams<TS, TC> p) {
  stage_body<TS, TC, R, NS, NP, NOUT, EPI, AMASK, BMASK, FORM, BATCH>(p);
}

}  // namespace gpe
