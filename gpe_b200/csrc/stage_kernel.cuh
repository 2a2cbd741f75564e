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
// z-planes.  TY compute warps each own one row (two consecutive x sites per
// lane); one more warp is the producer: its lane 0 issues, plane by plane,
// TMA tile loads (no multicast) of the stencil plane with its halo and of the
// pointwise input tiles into a ring of `stages` shared-memory slots.  A slot
// is handed over on a "full" mbarrier (TMA transaction count) and handed back
// on an "empty" mbarrier that every compute warp arrives on once it no longer
// reads the slot, so no block-wide barrier is taken per plane.  The
// z-neighbours come from a register queue of 2R+1 planes (R = order/2),
// rotated by unrolling the plane loop 2R+1 times; x and y neighbours are read
// from the staged halo plane.  Outputs go straight from registers to global
// memory as 16-byte stores.
//
// The combination each stage performs is fixed at compile time ("recipe"):
//   out[o] = alpha[o]*u + sum_q beta[o][q]*P_q + a[o] (x) K
// where u is the stencil field at the site, P_q the pointwise inputs, alpha
// and beta real Runge-Kutta weights present only where AMASK/BMASK say so,
// a[o] one complex coefficient per output (it carries dt), and K the
// right-hand side.  Without trap, sponge, gradient or sphere terms (FULL =
// false) the right-hand side of every equation is i*B with
// B = cL*lap(u) + (c0 + cn|u|^2) u, so K = B and the host folds the factor i
// into a[o]; with FULL = true K = f(u) is formed site by site.
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

struct TileMaps {
  CUtensorMap halo;      // stencil field, box (64+4) x (TY+2R) x 1
  CUtensorMap pt[MAXP];  // pointwise fields, box 64 x TY x 1
};

template <typename TS, typename TC>
struct StageParams {
  TileMaps maps;
  int nx, ny, nz;       // interior extents
  int Nx, Ny;           // padded pitches (complex elements)
  int ntx, zchunk, bcs, TY, stages;
  unsigned int halo_box_bytes, pt_box_bytes;    // bytes one TMA box delivers
  unsigned int halo_smem_bytes, pt_smem_bytes;  // 128-aligned slot strides
  const TS* stencil;    // stencil field (padded layout), warm-up planes
  TS* out[2];           // output fields (padded layout)
  int ghost_mask;       // bit o set: out[o] gets its boundary ghosts filled
  int zg_lo, zg_hi;     // fill the z ghosts below / above locally (else a
                        // neighbouring rank sends them)
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
  TC alpha[2];
  TC beta[2][MAXP];
  TC a_r[2], a_i[2];
  // rkqs error: err = sum_q ce[q]*P_q + cek (x) K (FP64)
  double ce[MAXP], cek_r, cek_i;
  double dt0_r, dt0_i;    // dt of the first attempt (psi_scal)
  double inv_absdt;       // 1/|dt| of this attempt (|f(psi)| = |k1|/|dt|)
  double eg, emu;         // energy: g, mu
  double* partials;       // 2 doubles per CTA
  int* status;
  unsigned long long wait_limit_ns;
};

__device__ __forceinline__ bool near_edge(int i, int n) {
  return i < 3 || i >= n - 3;
}

template <int K>
using IC = std::integral_constant<int, K>;

template <typename TS, typename TC, int R, int NP, int NOUT, int EPI, int AMASK,
          int BMASK, bool FULL>
__global__ void __launch_bounds__(288)
    stage_kernel(const __grid_constant__ StageParams<TS, TC> p) {
  using V = typename VT<TC>::T;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int s_abort, s_issued;
  __shared__ double s_red[2][32];

  constexpr int W = (int)(sizeof(TS) / 4);  // 8-byte TMA units per complex
  constexpr int HW = TX + 4;                // halo tile row width (complex)
  constexpr int QN = 2 * R + 1;             // z-queue length
  constexpr unsigned ES = 2 * sizeof(TS);   // bytes per stored complex
  const int TY = p.TY, S = p.stages;
  const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;
  const int tile_x = blockIdx.x % p.ntx, tile_y = blockIdx.x / p.ntx;
  const int z0 = blockIdx.y * p.zchunk;
  const int z1 = min(z0 + p.zchunk, p.nz);
  const int niters = (z1 - z0) + R;
  const int i0 = tile_x * TX + 2 * lane;
  const int j = tile_y * TY + ty;
  const bool ok0 = (i0 < p.nx) && (j < p.ny);
  const bool ok1 = (i0 + 1 < p.nx) && (j < p.ny);

  // shared memory: full[S] and empty[S] barriers (S <= 8), then the slots
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + 8;
  unsigned char* sbase = smem + 128;
  const unsigned stride = p.halo_smem_bytes + (unsigned)NP * p.pt_smem_bytes;
  const size_t Nx = (size_t)p.Nx, NxNy = (size_t)p.Nx * (size_t)p.Ny;

  if (tid == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], (uint32_t)TY);
    }
    fence_mbar_init();
    s_abort = 0;
    s_issued = 0;
  }
  __syncthreads();

  double red0 = 0.0, red1 = 0.0;
  if (ty == TY) {
    // ---------------- producer warp: lane 0 streams the planes -------------
    if (lane == 0) {
      prefetch_tmap(&p.maps.halo);
#pragma unroll
      for (int qq = 0; qq < NP; qq++) prefetch_tmap(&p.maps.pt[qq]);
      int slot = 0;
      uint32_t cyc = 0;  // completed passes over the ring
      for (int u = 0; u < niters; u++) {
        if (cyc > 0) {
          // the slot's previous plane must have been released by every
          // compute warp
          if (!mbar_wait_bounded(&empty[slot], (cyc - 1) & 1u, p.wait_limit_ns)) {
            s_abort = 1;
            atomicExch(p.status, 6);
            break;
          }
          fence_proxy_async();
        }
        unsigned char* st = sbase + (size_t)slot * stride;
        const bool with_pt = (NP > 0) && (u >= R);
        mbar_arrive_expect_tx(&full[slot],
                              p.halo_box_bytes + (with_pt ? NP * p.pt_box_bytes : 0u));
        tma_load_3d(st, &p.maps.halo, &full[slot], W * tile_x * TX,
                    tile_y * TY + GH - R, z0 + u + GH);
        if (with_pt) {
#pragma unroll
          for (int qq = 0; qq < NP; qq++)
            tma_load_3d(st + p.halo_smem_bytes + (size_t)qq * p.pt_smem_bytes,
                        &p.maps.pt[qq], &full[slot], W * (tile_x * TX + GH),
                        tile_y * TY + GH, z0 + u - R + GH);
        }
        s_issued = u + 1;
        if (++slot == S) {
          slot = 0;
          ++cyc;
        }
        if (*(volatile int*)&s_abort) break;
      }
    }
  } else {
  // Per-thread constants.
  TC Vxy[2] = {TC(0), TC(0)}, Dxy[2] = {TC(0), TC(0)};
  double Wxy[2] = {0.0, 0.0};
  if ((FULL || (EPI & EPI_ENERGY)) && p.use_V) {
    Vxy[0] = p.tabV[0][i0] + p.tabV[1][j];
    Vxy[1] = p.tabV[0][i0 + 1] + p.tabV[1][j];
  }
  if (FULL && p.use_diss) {
    Dxy[0] = p.tabD[0][i0] + p.tabD[1][j];
    Dxy[1] = p.tabD[0][i0 + 1] + p.tabD[1][j];
  }
  if (EPI & EPI_NORM) {
    Wxy[0] = p.tabW[0][i0] * p.tabW[1][j];
    Wxy[1] = p.tabW[0][i0 + 1] * p.tabW[1][j];
  }
  const V cx1 = vsplat(p.cx1), cx2 = vsplat(p.cx2), cy1 = vsplat(p.cy1),
          cy2 = vsplat(p.cy2), cz1 = vsplat(p.cz1), cz2 = vsplat(p.cz2),
          c0l = vsplat(p.c0lap), cLv = vsplat(p.cL);
  V ar[2], aix[2], alv[2], bev[2][NP > 0 ? NP : 1];
#pragma unroll
  for (int o = 0; o < 2; o++) {
    ar[o] = vsplat(p.a_r[o]);
    aix[o] = vpair(-p.a_i[o], p.a_i[o]);
    alv[o] = vsplat(p.alpha[o]);
#pragma unroll
    for (int qq = 0; qq < (NP > 0 ? NP : 1); qq++) bev[o][qq] = vsplat(p.beta[o][qq]);
  }
  const V mone = vsplat(TC(-1));
  // Ghost copies this thread's sites feed, as element offsets from the site
  // (x and y fixed per thread; z per plane, uniform across the CTA).
  int gxo[2][2], gyo[2];
  {
    int a, b;
    for (int e = 0; e < 2; e++) {
      ghost_targets(i0 + e, p.nx, p.bcs, a, b);
      gxo[e][0] = (a != NO_GHOST) ? a - (i0 + e) : 0;
      gxo[e][1] = (b != NO_GHOST) ? b - (i0 + e) : 0;
    }
    ghost_targets(j, p.ny, p.bcs, a, b);
    gyo[0] = (a != NO_GHOST) ? (a - j) * p.Nx : 0;
    gyo[1] = (b != NO_GHOST) ? (b - j) * p.Nx : 0;
  }
  const bool edge_xy = (gxo[0][0] | gxo[0][1] | gxo[1][0] | gxo[1][1] | gyo[0] | gyo[1]) != 0;
  // element offset of this thread's first site in plane z0
  size_t base = (size_t)(z0 + GH) * NxNy + (size_t)(j + GH) * Nx + (size_t)(i0 + GH);

  // z-queue: physical slot of push number c is c % QN; after push c the
  // plane d above the one being computed sits in slot (c + 1 + R + d) % QN.
  CPair<TC> q[QN];
#pragma unroll
  for (int w = 0; w < R; w++) {
    CPair<TC> v = {vsplat(TC(0)), vsplat(TC(0))};
    if (ok0) v = ld_cpair<TS, TC>(p.stencil + 2 * (base - (size_t)(R - w) * NxNy));
    q[w] = v;
  }
#pragma unroll
  for (int w = R; w < QN; w++) q[w] = {vsplat(TC(0)), vsplat(TC(0))};

  int t = 0, slot = 0, cslot = 0;
  uint32_t phase = 0;
  const unsigned row_off = ES * (unsigned)((ty + R) * HW + 2 * lane + 2);
  const unsigned pt_off = ES * (unsigned)(ty * TX + 2 * lane);

  auto step = [&](auto kc) -> bool {
    constexpr int KK = decltype(kc)::value;
    if (t >= niters) return false;
    if (!mbar_wait_bounded(&full[slot], phase, p.wait_limit_ns)) {
      s_abort = 1;
      atomicExch(p.status, 6);
      return false;
    }
    q[(R + KK) % QN] = ld_cpair<TS, TC>(
        reinterpret_cast<const TS*>(sbase + (size_t)slot * stride + row_off));
    if (t >= R) {
      const int z = z0 + t - R;
      const unsigned char* hc = sbase + (size_t)cslot * stride + row_off;
      auto lds = [&](int drow, int dcol) {
        return ld_cpair<TS, TC>(reinterpret_cast<const TS*>(hc + (int)ES * (drow * HW + dcol)));
      };
      auto zq = [&](int d) -> const CPair<TC>& { return q[(R + KK + 1 + R + d + 2 * QN) % QN]; };
      const CPair<TC> xa = lds(0, -2);
      const CPair<TC> xc = lds(0, 2);
      const CPair<TC> yp1 = lds(1, 0), ym1 = lds(-1, 0);
      CPair<TC> yp2 = yp1, ym2 = ym1;
      if (R == 2) {
        yp2 = lds(2, 0);
        ym2 = lds(-2, 0);
      }
      CPair<TC> P[NP > 0 ? NP : 1];
      if (NP > 0) {
        const unsigned char* pb = sbase + (size_t)slot * stride + p.halo_smem_bytes + pt_off;
#pragma unroll
        for (int qq = 0; qq < NP; qq++)
          P[qq] = ld_cpair<TS, TC>(reinterpret_cast<const TS*>(pb + (size_t)qq * p.pt_smem_bytes));
      }
      TC Vz = TC(0), Dz = TC(0);
      double Wz = 0.0;
      if ((FULL || (EPI & EPI_ENERGY)) && p.use_V) Vz = p.tabV[2][z];
      if (FULL && p.use_diss) Dz = p.tabD[2][z];
      if (EPI & EPI_NORM) Wz = p.tabW[2][z];

      V res[2][2];  // [output][site]
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const CPair<TC>& ctr = zq(0);
        const V f0 = e ? ctr.b : ctr.a;
        const V xm1 = e ? ctr.a : xa.b, xp1 = e ? xc.a : ctr.b;
        const V xm2 = e ? xa.b : xa.a, xp2 = e ? xc.b : xc.a;
        V L = vmul(cx1, vadd(xp1, xm1));
        L = vfma(cy1, vadd(e ? yp1.b : yp1.a, e ? ym1.b : ym1.a), L);
        L = vfma(cz1, vadd(e ? zq(1).b : zq(1).a, e ? zq(-1).b : zq(-1).a), L);
        if (R == 2) {
          L = vfma(cx2, vadd(xp2, xm2), L);
          L = vfma(cy2, vadd(e ? yp2.b : yp2.a, e ? ym2.b : ym2.a), L);
          L = vfma(cz2, vadd(e ? zq(2).b : zq(2).a, e ? zq(-2).b : zq(-2).a), L);
        }
        L = vfma(c0l, f0, L);
        const bool ok = e ? ok1 : ok0;

        if (EPI & EPI_ENERGY) {
          if (ok) {
            const double lr = (double)L.x, li = (double)L.y;
            const double fr = (double)f0.x, fi = (double)f0.y;
            const double d2 = fr * fr + fi * fi;
            const double kin = -(lr * fr + li * fi);
            red0 += kin + 0.5 * (d2 * d2);
            red1 += 0.5 * kin + (double)(Vxy[e] + Vz) * d2 + 0.5 * p.eg * d2 * d2 -
                    p.emu * d2;
          }
          continue;
        }

        const TC a2 = fma(f0.y, f0.y, f0.x * f0.x);
        V Kv;
        if (EPI & EPI_LAP) {
          Kv = L;
        } else if (!FULL) {
          const TC s = fma(p.cn, a2, p.c0);
          Kv = vfma(vsplat(s), f0, vmul(cLv, L));
        } else {
          const TC Vs = p.use_V ? Vxy[e] + Vz : TC(0);
          const TC s = p.c0 + p.cV * Vs + p.cn * a2;
          const V B = vfma(vsplat(s), f0, vmul(cLv, L));
          const TC arr = p.use_diss ? p.ar0 + p.ard * (Dxy[e] + Dz) : p.ar0;
          Kv = vfma(vsplat(arr), B, vmul(vpair(-p.ai, p.ai), vswap(B)));
          if (p.use_grad) {
            V gx = vmul(vsplat(p.gx1), vfma(xm1, mone, xp1));
            if (R == 2) gx = vfma(vsplat(p.gx2), vfma(xm2, mone, xp2), gx);
            Kv = vfma(vsplat(p.U), gx, Kv);
          }
          if (p.use_sphere) {
            const double X = p.tabX[0][i0 + e], Y = p.tabX[1][j], Z = p.tabX[2][z];
            const TC m = (TC)(0.5 * (1.0 + tanh(sqrt(X * X + Y * Y + Z * Z) - 10.0 - 2.0)));
            Kv = vmul(vsplat(m), Kv);
          }
        }

        const V Ks = vswap(Kv);
#pragma unroll
        for (int o = 0; o < NOUT; o++) {
          V v = vfma(ar[o], Kv, vmul(aix[o], Ks));
          if (AMASK & (1 << o)) v = vfma(alv[o], f0, v);
#pragma unroll
          for (int qq = 0; qq < NP; qq++)
            if (BMASK & (1 << (o * 8 + qq))) v = vfma(bev[o][qq], e ? P[qq].b : P[qq].a, v);
          res[o][e] = v;
        }

        if (EPI & EPI_KAHAN) {
          // res[0] is the increment delta; compensated add to psi.  Slots:
          // psi = P[0] when NP >= 2 (else the stencil field), c = P[NP-1].
          const V psi = (NP >= 2) ? (e ? P[0].b : P[0].a) : f0;
          const V cc = e ? P[NP > 0 ? NP - 1 : 0].b : P[NP > 0 ? NP - 1 : 0].a;
          const V y = vfma(cc, mone, res[0][e]);
          const V tt = vadd(psi, y);
          res[1][e] = vfma(y, mone, vfma(psi, mone, tt));
          res[0][e] = tt;
        }

        if (ok && (EPI & EPI_NORM)) {
          const double vr = (double)res[0][e].x, vi = (double)res[0][e].y;
          red0 = fma(Wxy[e] * Wz, fma(vr, vr, vi * vi), red0);
        }
        if (ok && (EPI & EPI_ERR)) {
          // err = sum_q ce[q] P_q + cek (x) K; psi = P[0], k1 = P[1]
          const double kr = (double)Kv.x, ki = (double)Kv.y;
          double er = p.cek_r * kr - p.cek_i * ki;
          double ei = p.cek_r * ki + p.cek_i * kr;
#pragma unroll
          for (int qq = 1; qq < NP; qq++) {
            const V pv = e ? P[qq].b : P[qq].a;
            er = fma(p.ce[qq], (double)pv.x, er);
            ei = fma(p.ce[qq], (double)pv.y, ei);
          }
          const V psi0 = e ? P[0].b : P[0].a;
          const V k1 = e ? P[NP > 1 ? 1 : 0].b : P[NP > 1 ? 1 : 0].a;
          const double apsi = hypot((double)psi0.x, (double)psi0.y);
          const double m = hypot((double)k1.x, (double)k1.y) * p.inv_absdt;
          const double sr = apsi + p.dt0_r * m + 1e-30, si = p.dt0_i * m;
          red1 = fmax(red1, hypot(er, ei) / hypot(sr, si));
        }
      }

      if (!(EPI & EPI_ENERGY)) {
        long gzo[2] = {0, 0};
        if (near_edge(z, p.nz)) {
          int a, b;
          ghost_targets(z, p.nz, p.bcs, a, b);
          if (a != NO_GHOST && !((a < 0) ? p.zg_lo : p.zg_hi)) a = NO_GHOST;
          if (b != NO_GHOST && !((b < 0) ? p.zg_lo : p.zg_hi)) b = NO_GHOST;
          gzo[0] = (a != NO_GHOST) ? (long)(a - z) * (long)NxNy : 0;
          gzo[1] = (b != NO_GHOST) ? (long)(b - z) * (long)NxNy : 0;
        }
        const bool edge = edge_xy || ((gzo[0] | gzo[1]) != 0);
#pragma unroll
        for (int o = 0; o < NOUT; o++) {
          TS* out = p.out[o] + 2 * base;
          if (ok1) {
            st_cpair<TS, typename VT<TS>::T>(out, cvt_v<TS>(res[o][0]),
                                              cvt_v<TS>(res[o][1]));
          } else if (ok0) {
            st_c1<TS>(out, res[o][0]);
          }
          if (edge && (p.ghost_mask & (1 << o))) {
#pragma unroll
            for (int e = 0; e < 2; e++) {
              if (!(e ? ok1 : ok0)) continue;
              TS* o1 = out + 2 * e;
              const V v = res[o][e];
              if (gxo[e][0]) st_c1<TS>(o1 + 2 * (ptrdiff_t)gxo[e][0], v);
              if (gxo[e][1]) st_c1<TS>(o1 + 2 * (ptrdiff_t)gxo[e][1], v);
              if (gyo[0]) st_c1<TS>(o1 + 2 * (ptrdiff_t)gyo[0], v);
              if (gyo[1]) st_c1<TS>(o1 + 2 * (ptrdiff_t)gyo[1], v);
              if (gzo[0]) st_c1<TS>(o1 + 2 * gzo[0], v);
              if (gzo[1]) st_c1<TS>(o1 + 2 * gzo[1], v);
            }
          }
        }
      }
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
  }  // compute warps

  __syncthreads();
  // After a timed-out wait, let the copies already in flight land (bounded)
  // before the CTA's shared memory is released: the last load issued into
  // each slot completes phase (u / S) of that slot's full barrier.
  if (s_abort && tid == 0) {
    const int issued = s_issued;
    for (int u = max(0, issued - S); u < issued; u++)
      mbar_wait_bounded(&full[u % S], (uint32_t)((u / S) & 1), p.wait_limit_ns);
  }

  if (EPI & (EPI_NORM | EPI_ERR | EPI_ENERGY)) {
    red0 = warp_sum(red0);
    red1 = (EPI & EPI_ERR) ? warp_max(red1) : warp_sum(red1);
    if (lane == 0) {
      s_red[0][ty] = red0;
      s_red[1][ty] = red1;
    }
    __syncthreads();
    if (tid == 0) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < TY; w++) {
        a += s_red[0][w];
        b = (EPI & EPI_ERR) ? fmax(b, s_red[1][w]) : b + s_red[1][w];
      }
      const size_t blk = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
      p.partials[2 * blk + 0] = a;
      p.partials[2 * blk + 1] = b;
    }
  }
}

}  // namespace gpe
