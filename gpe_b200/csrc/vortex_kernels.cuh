// vortex_kernels.cuh -- total vortex line length (linelength,
// src/variables.f90:879-1145) on the resident padded field.
//
// Cells (i, j, k), 1 <= i <= nx-2 (likewise j, k), in the reference's loop
// order (k outer, i inner).  On each of a cell's 6 faces the zero lines of
// Re psi and Im psi are located by linear interpolation along the face edges
// and intersected; the first two points found on the cell's faces give a
// segment.  The reference keeps its point arrays x(1:6), y(1:6), z(1:6) from
// cell to cell, so a cell that finds one point measures to the x(2) left by
// the last earlier cell that found two: that carried value is resolved here
// by block scans in loop order (the cells of a block are contiguous), each
// block's last x(2), looked up by the next blocks, and a pass over each
// block's cells that came before its first writer.  The arithmetic is compiled
// without FMA contraction and in the reference's order, so every cell's
// points and segment equal a sequential evaluation bit for bit; only the
// final sum is reassociated (a fixed tree, the same on every run).
#pragma once

#include <cstdint>

namespace gpe {
namespace vortex {

constexpr int L_THREADS = 256;
constexpr int L_WARPS = L_THREADS / 32;
constexpr int L_CAP = 64;  // unresolved one-point cells kept per block

struct Pt {
  double x, y, z;
};

struct CellOut {
  int skip;     // the cell ended on a zero plane / zero edge ("cycle iloop")
  double add;   // 0.5 or 0.25 for those
  int npts;     // points written to x(1..) before the cell ended
  Pt p1, p2;
};

template <typename T> struct C2;
template <> struct C2<double> { using type = double2; };
template <> struct C2<float> { using type = float2; };

// Accepted zero points of one component along the 4 edges of a face: the
// first two (the only ones used) and their count.  An exact zero at a
// corner writes the reference's xu(lu) without advancing lu and is always
// overwritten before it is read, so it has no effect here.
__device__ __forceinline__ int edge_zeros(const double w[5], double& x1, double& y1, double& x2,
                                          double& y2) {
  int cnt = 0;
  double px = 0.0, py = 0.0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const double a = w[q], b = w[q + 1];
    if (a != 0.0 && a * b < 0.0) {
      double cx, cy;
      if (q == 0) {
        cx = fabs(a / (a - b));
        cy = 0.0;
      } else if (q == 1) {
        cx = 1.0;
        cy = fabs(a / (a - b));
      } else if (q == 2) {
        cx = fabs(b / (a - b));
        cy = 1.0;
      } else {
        cx = 0.0;
        cy = fabs(b / (a - b));
      }
      if (cnt == 0 || cx != px || cy != py) {
        if (cnt == 0) {
          x1 = cx;
          y1 = cy;
        }
        if (cnt == 1) {
          x2 = cx;
          y2 = cy;
        }
        px = cx;
        py = cy;
        cnt++;
      }
    }
  }
  return cnt;
}

// Corners q = 0..3 of faces front, back, right, left, top, bottom
// (src/variables.f90:901-958), one nibble each, corner = di | dj << 1 | dk << 2.
__constant__ unsigned kFaceCorners[6] = {0x2310u, 0x6754u, 0x3751u, 0x2640u, 0x6732u, 0x4510u};

// Outcome of one face (the body of the reference's nloop for face n).
constexpr int F_NONE = 0, F_POINT = 1, F_PLANE = 2, F_EDGE = 3;

// Corner values of face n from the cell's 8 corners (selects, no indexing).
__device__ __forceinline__ void face_values(const double cu[8], const double cv[8], int n,
                                            double u[5], double v[5]) {
  const unsigned tab = kFaceCorners[n];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = (tab >> (4 * q)) & 0xf;
    double uu = cu[0], vv = cv[0];
#pragma unroll
    for (int r = 1; r < 8; r++) {
      uu = (c == r) ? cu[r] : uu;
      vv = (c == r) ? cv[r] : vv;
    }
    u[q] = uu;
    v[q] = vv;
  }
  u[4] = u[0];
  v[4] = v[0];
}

// A component of one strict sign on the face's corners rules out every test
// of face_eval: no zero plane, no zero edge, no crossing to intersect.
__device__ __forceinline__ bool face_active(const double u[5], const double v[5]) {
  const bool u_one = (u[0] > 0.0 && u[1] > 0.0 && u[2] > 0.0 && u[3] > 0.0) ||
                     (u[0] < 0.0 && u[1] < 0.0 && u[2] < 0.0 && u[3] < 0.0);
  const bool v_one = (v[0] > 0.0 && v[1] > 0.0 && v[2] > 0.0 && v[3] > 0.0) ||
                     (v[0] < 0.0 && v[1] < 0.0 && v[2] < 0.0 && v[3] < 0.0);
  return !(u_one || v_one);
}

__device__ __forceinline__ int face_eval(const double u[5], const double v[5], double& xx,
                                         double& yy) {
  const bool uz = u[0] == 0.0 && u[1] == 0.0 && u[2] == 0.0 && u[3] == 0.0;
  const bool vz = v[0] == 0.0 && v[1] == 0.0 && v[2] == 0.0 && v[3] == 0.0;
  const bool vcross = v[0] * v[1] < 0.0 || v[1] * v[2] < 0.0 || v[2] * v[3] < 0.0 ||
                      v[3] * v[0] < 0.0;
  const bool ucross = u[0] * u[1] < 0.0 || u[1] * u[2] < 0.0 || u[2] * u[3] < 0.0 ||
                      u[3] * u[0] < 0.0;
  if ((uz && vcross) || (vz && ucross)) return F_PLANE;
  bool edge = false;
#pragma unroll
  for (int q = 0; q < 4; q++)
    edge = edge || (u[q] == 0.0 && u[q + 1] == 0.0 && v[q] == 0.0 && v[q + 1] == 0.0);
  if (edge) return F_EDGE;
  double xu1 = 0, yu1 = 0, xu2 = 0, yu2 = 0, xv1 = 0, yv1 = 0, xv2 = 0, yv2 = 0;
  const int nu = edge_zeros(u, xu1, yu1, xu2, yu2);
  const int nv = edge_zeros(v, xv1, yv1, xv2, yv2);
  if (nu >= 2 && nv >= 2) {
    double den = xv2 * (yu1 - yu2) + xv1 * (yu2 - yu1) + (xu1 - xu2) * (yv1 - yv2);
    if (den == 0.0) den = den + 0.0000001;
    xx = (xu1 * (xv2 * (yv1 - yu2) + xv1 * (yu2 - yv2)) +
          xu2 * (xv2 * (yu1 - yv1) + xv1 * (yv2 - yu1))) / den;
    yy = (xv2 * (yu1 - yu2) * yv1 + xu1 * yu2 * yv1 - xv1 * yu1 * yv2 - xu1 * yu2 * yv2 +
          xv1 * yu2 * yv2 + xu2 * yu1 * (yv2 - yv1)) / den;
    if (xx >= 0.0 && xx <= 1.0 && yy >= 0.0 && yy <= 1.0) return F_POINT;
  }
  return F_NONE;
}

// The cell-local point of a face's (xx, yy) (src/variables.f90:1088-1113).
__device__ __forceinline__ Pt face_point(int n, double xx, double yy) {
  switch (n) {
    case 0: return Pt{xx, yy, 0.0};
    case 1: return Pt{xx, yy, 1.0};
    case 2: return Pt{1.0, yy, xx};
    case 3: return Pt{0.0, yy, xx};
    case 4: return Pt{xx, 1.0, yy};
    default: return Pt{xx, 0.0, yy};
  }
}

// Folds a face outcome into the cell in face order (the reference's m, its
// "cycle iloop" on a zero plane or edge).  Returns false once the cell ended.
__device__ __forceinline__ bool fold_face(CellOut& o, int& m, int n, int code, double xx,
                                          double yy) {
  if (code == F_PLANE || code == F_EDGE) {
    o.skip = 1;
    o.add = code == F_PLANE ? 0.5 : 0.25;
    o.npts = m;
    return false;
  }
  if (code == F_POINT) {
    const Pt p = face_point(n, xx, yy);
    if (m == 0) o.p1 = p;
    if (m == 1) o.p2 = p;
    m++;
  }
  return true;
}

// One cell of the reference's iloop body, faces in order.
__device__ __forceinline__ void cell_line(const double cu[8], const double cv[8], CellOut& o) {
  o.skip = 0;
  o.add = 0.0;
  o.npts = 0;
  int m = 0;
#pragma unroll 1
  for (int n = 0; n < 6; n++) {
    double u[5], v[5];
    face_values(cu, cv, n, u, v);
    if (!face_active(u, v)) continue;
    double xx = 0.0, yy = 0.0;
    const int code = face_eval(u, v, xx, yy);
    if (!fold_face(o, m, n, code, xx, yy)) return;
  }
  o.npts = m;
}

// The segment of a cell with points p1 and x(2) = p2
// (src/variables.f90:1118-1134; the reference tests y twice where z may
// have been meant, kept).
__device__ __forceinline__ double segment(const Pt& p1, const Pt& p2) {
  double a = 1.0;
  const bool ex = p1.x == p2.x && (p1.x == 0.0 || p1.x == 1.0);
  const bool ey = p1.y == p2.y && (p1.y == 0.0 || p1.y == 1.0);
  const bool ez = p1.z == p2.z && (p1.z == 0.0 || p1.z == 1.0);
  if (ex || ey) {
    a = a * 0.5;
    if ((ex && ey) || (ey && ez)) a = a * 0.5;
  }
  const double dx = p1.x - p2.x, dy = p1.y - p2.y, dz = p1.z - p2.z;
  return a * sqrt(dx * dx + dy * dy + dz * dz);
}

struct LineArgs {
  const void* psi;        // the resident padded field, or a dense interior array
  int nx, ny, nz, Nx, Ny;
  int ghost;              // 2 for the padded field, 0 for a dense array
  int cx;               // cells per row, nx - 2
  long long ncell;      // (nx-2)(ny-2)(nz-2)
  long long per_block;  // cells per block (whole rows)
  double* bsum;         // [nblk] sums of the cells resolved in the block
  double* blast;        // [nblk][4] has-writer flag, last x(2) written
  int* bunres;          // [nblk] one-point cells before the block's first writer
  long long* bfirst;    // [nblk] cell offset of the block's first writer
  double* bbuf;         // [nblk][L_CAP][3] their first points
  double* bres;         // [nblk] sums of those cells once resolved
  double* out;          // [0] total length
};

template <typename T>
__device__ __forceinline__ void load_cell(const LineArgs& p, long long c, double cu[8],
                                          double cv[8]) {
  using V = typename C2<T>::type;
  const V* f = static_cast<const V*>(p.psi);
  const long long row = c / p.cx;
  const int i = 1 + (int)(c - row * p.cx);
  const int j = 1 + (int)(row % (p.ny - 2));
  const int k = 1 + (int)(row / (p.ny - 2));
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int di = q & 1, dj = (q >> 1) & 1, dk = q >> 2;
    const size_t at = ((size_t)(k + dk + p.ghost) * p.Ny + (size_t)(j + dj + p.ghost)) * p.Nx +
                      (size_t)(i + di + p.ghost);
    const V w = f[at];
    cu[q] = (double)w.x;
    cv[q] = (double)w.y;
  }
}

// A cell can hold a point, a zero plane or a zero edge only if neither
// component keeps one strict sign on all 8 corners.
__device__ __forceinline__ bool may_hold_line(const double cu[8], const double cv[8]) {
  bool up = true, un = true, vp = true, vn = true;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    up = up && cu[q] > 0.0;
    un = un && cu[q] < 0.0;
    vp = vp && cv[q] > 0.0;
    vn = vn && cv[q] < 0.0;
  }
  return !(up || un || vp || vn);
}

// Exclusive block scan over a flag: the largest tid' < tid with the flag
// set (-1 if none), and the block's first and last flagged tid.
__device__ __forceinline__ int last_flag_before(bool flag, int* s_warp, int& first, int& last) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(0xffffffffu, flag);
  const unsigned below = bal & ((1u << lane) - 1u);
  const int in_warp = below ? (warp * 32 + 31 - __clz(below)) : -1;
  __syncthreads();
  if (lane == 0) {
    s_warp[warp] = bal ? (warp * 32 + 31 - __clz(bal)) : -1;
    s_warp[L_WARPS + warp] = bal ? (warp * 32 + __ffs(bal) - 1) : -1;
  }
  __syncthreads();
  int before = in_warp;
  if (before < 0)
    for (int w = warp - 1; w >= 0; w--)
      if (s_warp[w] >= 0) {
        before = s_warp[w];
        break;
      }
  first = -1;
  last = -1;
  for (int w = 0; w < L_WARPS; w++)
    if (s_warp[L_WARPS + w] >= 0) {
      first = s_warp[L_WARPS + w];
      break;
    }
  for (int w = L_WARPS - 1; w >= 0; w--)
    if (s_warp[w] >= 0) {
      last = s_warp[w];
      break;
    }
  return before;
}

__device__ __forceinline__ double block_sum(double x, double* s_red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
  __syncthreads();
  if (lane == 0) s_red[warp] = x;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < L_WARPS; w++) t += s_red[w];
  return t;
}

// Block-wide exclusive prefix sum of one small count per thread (thread
// order) and the block's total.
__device__ __forceinline__ int block_excl_sum(int x, int* s_cnt, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += o;
  }
  __syncthreads();
  if (lane == 31) s_cnt[warp] = inc;
  __syncthreads();
  int pos = inc - x;
  total = 0;
  for (int w = 0; w < L_WARPS; w++) {
    if (w < warp) pos += s_cnt[w];
    total += s_cnt[w];
  }
  return pos;
}

// Block-wide exclusive position of a flagged thread among the flagged ones
// (thread order) and the block's total.
__device__ __forceinline__ int flag_position(bool flag, int* s_cnt, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned b = __ballot_sync(0xffffffffu, flag);
  __syncthreads();
  if (lane == 0) s_cnt[warp] = __popc(b);
  __syncthreads();
  int pos = __popc(b & ((1u << lane) - 1u));
  total = 0;
  for (int w = 0; w < L_WARPS; w++) {
    if (w < warp) pos += s_cnt[w];
    total += s_cnt[w];
  }
  return pos;
}

// Pass 1: the block's cells in loop order.  Cells that may hold a line
// (most do not) are queued in order and processed 256 at a time; their
// faces on which neither component keeps one sign are queued again and
// evaluated one per thread, so the warps doing the face arithmetic are
// dense; one-point cells are resolved inside the block wherever an earlier
// queued cell of the block wrote x(2).
// Resident blocks per SM the cell pass is compiled for (registers per thread
// 65536 / (256 x this)).
#ifndef GPE_LINE_MIN_BLOCKS
#define GPE_LINE_MIN_BLOCKS 2
#endif

template <typename T>
__global__ void __launch_bounds__(L_THREADS, GPE_LINE_MIN_BLOCKS) line_cells_kernel(LineArgs p) {
  __shared__ double s_p2[L_THREADS][3];
  __shared__ long long s_q[2 * L_THREADS];
  __shared__ double s_fx[6 * L_THREADS], s_fy[6 * L_THREADS];
  __shared__ unsigned char s_fc[6 * L_THREADS];
  __shared__ unsigned short s_face[6 * L_THREADS];
  __shared__ int s_warp[2 * L_WARPS];
  __shared__ int s_cnt[L_WARPS];
  __shared__ double s_red[L_WARPS];
  const int tid = threadIdx.x;
  const long long c0 = (long long)blockIdx.x * p.per_block;
  const long long c1 = min(c0 + p.per_block, p.ncell);
  double acc = 0.0;
  bool carry_ok = false;
  Pt carry = {0.0, 0.0, 0.0};
  long long first_writer = c1 - c0;
  int unresolved = 0;
  int qn = 0;
  long long scan = c0;
  while (scan < c1 || qn > 0) {
    // fill the queue with candidate cells, in order
    while (qn < L_THREADS && scan < c1) {
      const long long c = scan + tid;
      bool cand = false;
      if (c < c1) {
        double cu[8], cv[8];
        load_cell<T>(p, c, cu, cv);
        cand = may_hold_line(cu, cv);
      }
      int total;
      const int pos = flag_position(cand, s_cnt, total);
      if (cand) s_q[qn + pos] = c;
      qn += total;
      scan += L_THREADS;
      __syncthreads();
    }
    if (qn == 0) break;
    const int nb = min(qn, L_THREADS);
    const bool valid = tid < nb;
    const long long c = valid ? s_q[tid] : 0;
    // the batch's faces: each active one evaluated by whichever thread takes
    // it from the face queue, outcomes folded per cell in face order
    unsigned amask = 0;
    if (valid) {
      double cu[8], cv[8];
      load_cell<T>(p, c, cu, cv);
#pragma unroll
      for (int n = 0; n < 6; n++) {
        double u[5], v[5];
        face_values(cu, cv, n, u, v);
        if (face_active(u, v)) amask |= 1u << n;
        s_fc[tid * 6 + n] = (unsigned char)F_NONE;
      }
    }
    int nface;
    int at = block_excl_sum(__popc(amask), s_cnt, nface);
#pragma unroll
    for (int n = 0; n < 6; n++)
      if ((amask >> n) & 1u) s_face[at++] = (unsigned short)((tid << 3) | n);
    __syncthreads();
    for (int q = tid; q < nface; q += L_THREADS) {
      const int t = s_face[q] >> 3, n = s_face[q] & 7;
      double cu[8], cv[8];
      load_cell<T>(p, s_q[t], cu, cv);
      double u[5], v[5];
      face_values(cu, cv, n, u, v);
      double xx = 0.0, yy = 0.0;
      const int code = face_eval(u, v, xx, yy);
      s_fc[t * 6 + n] = (unsigned char)code;
      s_fx[t * 6 + n] = xx;
      s_fy[t * 6 + n] = yy;
    }
    __syncthreads();
    CellOut o;
    o.skip = 0;
    o.add = 0.0;
    o.npts = 0;
    o.p1 = o.p2 = Pt{0.0, 0.0, 0.0};
    if (valid) {
      int m = 0;
      bool live = true;
#pragma unroll
      for (int n = 0; n < 6; n++)
        if (live)
          live = fold_face(o, m, n, s_fc[tid * 6 + n], s_fx[tid * 6 + n], s_fy[tid * 6 + n]);
      if (live) o.npts = m;
    }
    const bool writer = o.npts >= 2;
    const bool pending = !o.skip && o.npts == 1;
    if (o.skip)
      acc += o.add;
    else if (o.npts >= 2)
      acc += segment(o.p1, o.p2);
    s_p2[tid][0] = o.p2.x;
    s_p2[tid][1] = o.p2.y;
    s_p2[tid][2] = o.p2.z;
    int first, last;
    const int before = last_flag_before(writer, s_warp, first, last);
    bool unres = false;
    if (pending) {
      if (before >= 0)
        acc += segment(o.p1, Pt{s_p2[before][0], s_p2[before][1], s_p2[before][2]});
      else if (carry_ok)
        acc += segment(o.p1, carry);
      else
        unres = true;
    }
    // unresolved cells keep their first point, in cell order
    int total;
    const int off = unresolved + flag_position(unres, s_cnt, total);
    if (unres && off < L_CAP) {
      double* b = p.bbuf + ((size_t)blockIdx.x * L_CAP + off) * 3;
      b[0] = o.p1.x;
      b[1] = o.p1.y;
      b[2] = o.p1.z;
    }
    unresolved += total;
    if (first >= 0 && !carry_ok) first_writer = s_q[first] - c0;
    if (last >= 0) {
      carry = Pt{s_p2[last][0], s_p2[last][1], s_p2[last][2]};
      carry_ok = true;
    }
    // drop the processed entries
    __syncthreads();
    const long long keep = (tid < qn - nb) ? s_q[nb + tid] : 0;
    __syncthreads();
    if (tid < qn - nb) s_q[tid] = keep;
    qn -= nb;
    __syncthreads();
  }
  const double s = block_sum(acc, s_red);
  if (tid == 0) {
    p.bsum[blockIdx.x] = s;
    double* L = p.blast + (size_t)blockIdx.x * 4;
    L[0] = carry_ok ? 1.0 : 0.0;
    L[1] = carry.x;
    L[2] = carry.y;
    L[3] = carry.z;
    p.bunres[blockIdx.x] = unresolved;
    p.bfirst[blockIdx.x] = first_writer;
  }
}

// Pass 2: the one-point cells before each block's first writer, measured
// to the carried x(2): from the kept points, or by walking those cells
// again when there were more than L_CAP of them.
template <typename T>
__global__ void __launch_bounds__(L_THREADS) line_resolve_kernel(LineArgs p) {
  __shared__ double s_red[L_WARPS];
  __shared__ Pt s_in;
  const int b = blockIdx.x;
  const int cnt = p.bunres[b];
  if (cnt == 0) {  // block-uniform
    if (threadIdx.x == 0) p.bres[b] = 0.0;
    return;
  }
  // the x(2) carried in: the last written by the nearest earlier block that
  // wrote one (zero if none), found by the first warp 32 blocks at a time
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int found = -1;
    for (int top = b - 1; top >= 0 && found < 0; top -= 32) {
      const int q = top - lane;
      const bool w = q >= 0 && p.blast[(size_t)q * 4] != 0.0;
      const unsigned bal = __ballot_sync(0xffffffffu, w);
      if (bal) found = top - (__ffs(bal) - 1);
    }
    if (lane == 0)
      s_in = found < 0 ? Pt{0.0, 0.0, 0.0}
                       : Pt{p.blast[(size_t)found * 4 + 1], p.blast[(size_t)found * 4 + 2],
                            p.blast[(size_t)found * 4 + 3]};
  }
  __syncthreads();
  const Pt in = s_in;
  double acc = 0.0;
  if (cnt <= L_CAP) {
    for (int t = threadIdx.x; t < cnt; t += L_THREADS) {
      const double* q = p.bbuf + ((size_t)b * L_CAP + t) * 3;
      acc += segment(Pt{q[0], q[1], q[2]}, in);
    }
  } else {
    const long long c0 = (long long)b * p.per_block;
    const long long c1 = c0 + p.bfirst[b];
    for (long long base = c0; base < c1; base += L_THREADS) {
      const long long c = base + threadIdx.x;
      if (c < c1) {
        double cu[8], cv[8];
        load_cell<T>(p, c, cu, cv);
        CellOut o;
        o.skip = 0;
        o.add = 0.0;
        o.npts = 0;
        o.p1 = o.p2 = Pt{0.0, 0.0, 0.0};
        if (may_hold_line(cu, cv)) cell_line(cu, cv, o);
        if (!o.skip && o.npts == 1) acc += segment(o.p1, in);
      }
    }
  }
  const double s = block_sum(acc, s_red);
  if (threadIdx.x == 0) p.bres[b] = s;
}

// Total in block order (a fixed tree), times dx.
__global__ void __launch_bounds__(L_THREADS) line_total_kernel(LineArgs p, int nblk, double dx) {
  __shared__ double s_red[L_WARPS];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblk; b += L_THREADS) acc += p.bsum[b] + p.bres[b];
  const double s = block_sum(acc, s_red);
  if (threadIdx.x == 0) p.out[0] = s * dx;
}

}  // namespace vortex
}  // namespace gpe

// ===========================================================================
// Zero finders: get_zeros, get_extra_zeros, get_re_im_zeros
// (src/io.f90:895-1402).  Twelve sections, in the reference's file order:
//   0-2  zeros, x / y / z edges where Re and Im cross together
//   3-5  zeros, xy / xz / yz faces crossed alternately by Re and Im
//   6-8  re_zeros, x / y / z edges of Re;  9-11 im_zeros, the same of Im
// Every section walks the interior cells in loop order with at most one
// point per cell; points are compacted in that order (a count pass, block
// offsets, a write pass), so the lists equal the reference's line by line.
namespace gpe {
namespace vortex {

constexpr int Z_SECTIONS = 12;

struct ZeroArgs {
  const void* psi;
  int nx, ny, nz, Nx, Ny;
  int cx;
  long long ncell, per_block;
  const double* x;  // grid coordinates (src/ic.f90:53-66)
  const double* y;
  const double* z;
  long long* bcount;  // [nblk][Z_SECTIONS]
  const long long* boff;  // [nblk][Z_SECTIONS] first output slot
  double* pts;        // [total][3]
};

// Corners of a cell used by the sections: 0 (i,j,k), 1 (i+1,j,k), 2 (i,j+1,k),
// 3 (i,j,k+1), 4 (i+1,j+1,k), 5 (i+1,j,k+1), 6 (i,j+1,k+1).
template <typename T>
__device__ __forceinline__ void load_zero_corners(const ZeroArgs& p, long long c, double re[7],
                                                  double im[7], int& i, int& j, int& k) {
  using V = typename C2<T>::type;
  const V* f = static_cast<const V*>(p.psi);
  const long long row = c / p.cx;
  i = 1 + (int)(c - row * p.cx);
  j = 1 + (int)(row % (p.ny - 2));
  k = 1 + (int)(row / (p.ny - 2));
  const int di[7] = {0, 1, 0, 0, 1, 1, 0}, dj[7] = {0, 0, 1, 0, 1, 0, 1},
            dk[7] = {0, 0, 0, 1, 0, 1, 1};
#pragma unroll
  for (int q = 0; q < 7; q++) {
    const size_t at = ((size_t)(k + dk[q] + 2) * p.Ny + (size_t)(j + dj[q] + 2)) * p.Nx +
                      (size_t)(i + di[q] + 2);
    const V w = f[at];
    re[q] = (double)w.x;
    im[q] = (double)w.y;
  }
}

__device__ __forceinline__ double select7(const double v[7], int q) {
  double r = v[0];
#pragma unroll
  for (int t = 1; t < 7; t++) r = (q == t) ? v[t] : r;
  return r;
}

// Section s of one cell: whether it writes a point, and the point.
__device__ __forceinline__ bool zero_section(int s, const double re[7], const double im[7],
                                             int i, int j, int k, const ZeroArgs& p, Pt& o) {
  if (s < 3 || s >= 6) {
    const int d = s < 3 ? s : (s - 6) % 3;  // 0 x, 1 y, 2 z
    const int n = 1 + d;                    // corner across the edge
    const double* cc = d == 0 ? p.x : (d == 1 ? p.y : p.z);  // device grid table
    const int a = d == 0 ? i : (d == 1 ? j : k);
    double w, wn;
    bool hit;
    if (s < 3) {
      const double r = re[0], m = im[0], rn = select7(re, n), mn = select7(im, n);
      hit = (r == 0.0 && m == 0.0) || (r == 0.0 && m * mn < 0.0) ||
            (m == 0.0 && r * rn < 0.0) || (r * rn < 0.0 && m * mn < 0.0);
      w = r;
      wn = rn;
    } else {
      const bool use_im = s >= 9;
      w = use_im ? im[0] : re[0];
      wn = use_im ? select7(im, n) : select7(re, n);
      // the z edges test .and. where the x and y edges test .or. (kept)
      hit = d == 2 ? (w == 0.0 && w * wn < 0.0) : (w == 0.0 || w * wn < 0.0);
    }
    if (!hit) return false;
    const double den = w - wn;
    if (den == 0.0) return false;
    const double zero = -wn * cc[a] / den + w * cc[a + 1] / den;
    o = Pt{d == 0 ? zero : p.x[i], d == 1 ? zero : p.y[j], d == 2 ? zero : p.z[k]};
    return true;
  }
  // faces: corners c0..c3 around the face; u runs c0 -> c1, w runs c1 -> c2
  const int f = s - 3;
  int q0, q1, q2, q3;
  double u0, u1, w0, w1;
  if (f == 0) {
    q0 = 0; q1 = 1; q2 = 4; q3 = 2;
    u0 = p.x[i]; u1 = p.x[i + 1]; w0 = p.y[j]; w1 = p.y[j + 1];
  } else if (f == 1) {
    q0 = 0; q1 = 1; q2 = 5; q3 = 3;
    u0 = p.x[i]; u1 = p.x[i + 1]; w0 = p.z[k]; w1 = p.z[k + 1];
  } else {
    q0 = 0; q1 = 3; q2 = 6; q3 = 2;
    u0 = p.z[k]; u1 = p.z[k + 1]; w0 = p.y[j]; w1 = p.y[j + 1];
  }
#pragma unroll
  for (int pass = 0; pass < 2; pass++) {
    // pass 0: Re crosses the u edges and Im the w edges; pass 1 the reverse
    const double r0 = select7(re, q0), r1 = select7(re, q1), r2 = select7(re, q2),
                 r3 = select7(re, q3);
    const double i0 = select7(im, q0), i1 = select7(im, q1), i2 = select7(im, q2),
                 i3 = select7(im, q3);
    const double A0 = pass ? i0 : r0, A1 = pass ? i1 : r1, A2 = pass ? i2 : r2,
                 A3 = pass ? i3 : r3;
    const double B0 = pass ? r0 : i0, B1 = pass ? r1 : i1, B2 = pass ? r2 : i2,
                 B3 = pass ? r3 : i3;
    if ((A0 * A1 < 0.0 && B0 * B1 >= 0.0) && (B1 * B2 < 0.0 && A1 * A2 >= 0.0) &&
        (A2 * A3 < 0.0 && B2 * B3 >= 0.0) && (B3 * B0 < 0.0 && A3 * A0 >= 0.0)) {
      double den = A0 - A1;
      const double z0 = -A1 * u0 / den + A0 * u1 / den;
      den = B1 - B2;
      const double z1 = -B2 * w0 / den + B1 * w1 / den;
      den = A2 - A3;
      const double z2 = -A3 * u1 / den + A2 * u0 / den;
      den = B3 - B0;
      const double z3 = -B0 * w1 / den + B3 * w0 / den;
      const double m1 = (w0 - w1) / (z0 - z2);
      const double m2 = (z1 - z3) / (u1 - u0);
      const double up = (z3 - u0 * m2 - w0 + z0 * m1) / (m1 - m2);
      const double wp = up * m1 + w0 - z0 * m1;
      if (f == 0) o = Pt{up, wp, p.z[k]};
      else if (f == 1) o = Pt{up, p.y[j], wp};
      else o = Pt{p.x[i], wp, up};
      return true;
    }
  }
  return false;
}

// Pass 1: points per block and section.
template <typename T>
__global__ void __launch_bounds__(L_THREADS) zeros_count_kernel(ZeroArgs p) {
  __shared__ int s_cnt[L_WARPS][Z_SECTIONS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long c0 = (long long)blockIdx.x * p.per_block;
  const long long c1 = min(c0 + p.per_block, p.ncell);
  int cnt[Z_SECTIONS];
#pragma unroll
  for (int s = 0; s < Z_SECTIONS; s++) cnt[s] = 0;
  for (long long c = c0 + threadIdx.x; c < c1; c += L_THREADS) {
    double re[7], im[7];
    int i, j, k;
    load_zero_corners<T>(p, c, re, im, i, j, k);
    Pt o;
#pragma unroll
    for (int s = 0; s < Z_SECTIONS; s++) cnt[s] += zero_section(s, re, im, i, j, k, p, o) ? 1 : 0;
  }
#pragma unroll
  for (int s = 0; s < Z_SECTIONS; s++) {
    int x = cnt[s];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
    if (lane == 0) s_cnt[warp][s] = x;
  }
  __syncthreads();
  if (threadIdx.x < Z_SECTIONS) {
    long long t = 0;
    for (int w = 0; w < L_WARPS; w++) t += s_cnt[w][threadIdx.x];
    p.bcount[(size_t)blockIdx.x * Z_SECTIONS + threadIdx.x] = t;
  }
}

// Pass 2: the points, each at its place in loop order.  A chunk of 256
// cells finds its hits in all 12 sections, places them (block-wide counts
// per warp and section), and queues them section by section; the queue is
// then worked one hit per thread, so the point arithmetic runs in dense,
// mostly same-section warps.
template <typename T>
__global__ void __launch_bounds__(L_THREADS) zeros_write_kernel(ZeroArgs p) {
  __shared__ int s_cnt[L_WARPS][Z_SECTIONS];
  __shared__ long long s_run[Z_SECTIONS];
  __shared__ long long s_qat[Z_SECTIONS * L_THREADS];
  __shared__ unsigned short s_qts[Z_SECTIONS * L_THREADS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long c0 = (long long)blockIdx.x * p.per_block;
  const long long c1 = min(c0 + p.per_block, p.ncell);
  if (threadIdx.x < Z_SECTIONS)
    s_run[threadIdx.x] = p.boff[(size_t)blockIdx.x * Z_SECTIONS + threadIdx.x];
  const unsigned below = (1u << lane) - 1u;
  for (long long base = c0; base < c1; base += L_THREADS) {
    const long long c = base + threadIdx.x;
    const bool valid = c < c1;
    unsigned mask = 0;
    if (valid) {
      double re[7], im[7];
      int i, j, k;
      load_zero_corners<T>(p, c, re, im, i, j, k);
      Pt o;
#pragma unroll
      for (int s = 0; s < Z_SECTIONS; s++)
        if (zero_section(s, re, im, i, j, k, p, o)) mask |= 1u << s;
    }
#pragma unroll
    for (int s = 0; s < Z_SECTIONS; s++) {
      const unsigned bal = __ballot_sync(0xffffffffu, (mask >> s) & 1u);
      if (lane == 0) s_cnt[warp][s] = __popc(bal);
    }
    __syncthreads();
    // queue: sections in order, each in thread (= cell) order
    int qbase = 0, nq = 0;
#pragma unroll
    for (int s = 0; s < Z_SECTIONS; s++) {
      const unsigned bal = __ballot_sync(0xffffffffu, (mask >> s) & 1u);
      int before = __popc(bal & below), tot = 0;
      for (int w = 0; w < L_WARPS; w++) {
        if (w < warp) before += s_cnt[w][s];
        tot += s_cnt[w][s];
      }
      if ((mask >> s) & 1u) {
        s_qat[qbase + before] = s_run[s] + before;
        s_qts[qbase + before] = (unsigned short)((threadIdx.x << 4) | s);
      }
      qbase += tot;
    }
    nq = qbase;
    __syncthreads();
    for (int q = threadIdx.x; q < nq; q += L_THREADS) {
      const int t = s_qts[q] >> 4, sec = s_qts[q] & 15;
      double re[7], im[7];
      int i, j, k;
      load_zero_corners<T>(p, base + t, re, im, i, j, k);
      Pt o = {0.0, 0.0, 0.0};
      zero_section(sec, re, im, i, j, k, p, o);
      double* out = p.pts + 3 * s_qat[q];
      out[0] = o.x;
      out[1] = o.y;
      out[2] = o.z;
    }
    __syncthreads();
    if (threadIdx.x < Z_SECTIONS) {
      int t = 0;
      for (int w = 0; w < L_WARPS; w++) t += s_cnt[w][threadIdx.x];
      s_run[threadIdx.x] += t;
    }
    __syncthreads();
  }
}

}  // namespace vortex
}  // namespace gpe
