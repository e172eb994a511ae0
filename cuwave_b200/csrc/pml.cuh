// The pml memory update of one 3D forward step along axes 1 and 2, over their slab nodes.
//
// The blocked 3D step writes the update of every interior node with the axis-0 memory
// terms already in (an axis-0 slab row is a whole plane of its march). These two
// kernels then add, axis by axis in the reference's order, each lined axis' share: for
// a node of an axis-d slab they advance its memory (psi+, psi-, zeta) from the plain cell
// differences of u^(t-1) along d and add minv (f (g psi+ - g psi-) + zeta) to u^t, as
// cuwave's pml_kernel does after fd_kernel (scalar.cu:500-532). Launched in order, axis
// 1 then axis 2, so a node in both slabs takes its shares in the reference's order.
//
// A thread owns four consecutive axis-2 nodes (a quad, 16-byte aligned) of one row, so
// the field, update and memory rows move as 16-byte vectors:
//
//   axis 1: a block per (plane, 4 slab rows, 32 quads), a warp along each row; taps are
//           the 2R rows of four around the row (the block's rows share them in L1)
//   axis 2: a thread per (row, slab quad); taps are the quad's run of 4 + 2H values;
//           the quad's memory is loaded for all its lanes before any is written back
//           (four blocks an SM bound its registers, so the early loads cost no warps)
//
// Taps past a wall take their mirrors (cuwave common.cuh:50-54). The stiffness is
// uniform (the blocked step's domain), so the harmonic means are one constant.
#pragma once

#include "step.cuh"

namespace cwb {

constexpr int PML1_THREADS = 128;
constexpr int PML1_QUADS = 32, PML1_ROWS = PML1_THREADS / PML1_QUADS;  // an axis-1 block's tile
constexpr int PML2_THREADS = 256;

template <typename T>
struct Pml3Params {
  Geometry g;
  T w[MAXR];
  T f;       // the axis' step factor
  T gconst;  // k k / (k + k) of the uniform stiffness
  T sconst;  // the uniform stiffness
  int flags;  // K_DERIVE, K_ADV
  DLevel u1, u2;
  const T *minv;
  const T *prof;  // (4, n[d]) a_node, b_node, a_half, b_half
  T *aux;         // 3 rows of `auxrow`: psi+, psi-, zeta
  long long auxrow;
  int nlo, nhi, xhi;  // axis 2: slab quads on each side, the first high one's x
  int fold;           // axis 2: the face ghosts refilled here (1 low, 2 high) from final mirrors
  int *ctr;
};

// one node's memory step and share of the update (pml_kernel's order)
template <typename T>
__device__ __forceinline__ void pml_node(const T f, const T gg, const T an, const T bn,
                                         const T ah, const T bh, const T ah1, const T bh1,
                                         const T Dpu, const T Dmu, T &m0, T &m1, T &m2,
                                         T &v, const T mi, const bool held) {
  const T pp = bh * m0 + ah * Dpu;
  const T pm = bh1 * m1 + ah1 * Dmu;
  const T zz = bn * m2 + an * f * (gg * (Dpu + pp) - gg * (Dmu + pm));
  m0 = pp;
  m1 = pm;
  m2 = zz;
  if (!held)
    v += mi * (f * (gg * pp - gg * pm) + zz);
}

template <typename T>
__device__ __forceinline__ void get4m(const T *base, T *dst, const int mask) {
  if (mask == 15) {
    load4(dst, base);
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i)
      dst[i] = ((mask >> i) & 1) ? base[i] : (T)0;
  }
}

template <typename T>
__device__ __forceinline__ void put4m(T *base, const T *src, const int mask) {
  if (mask == 15) {
    store4(base, src);
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if ((mask >> i) & 1)
        base[i] = src[i];
  }
}

template <typename T, int R>
__global__ void __launch_bounds__(PML1_THREADS) pml_axis1_kernel(const __grid_constant__ Pml3Params<T> p) {
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  const int N0 = g.n[0], NM = g.n[1], NF = g.n[2];
  const int lo = g.lo[1], hi = g.hi[1];
  // a warp a slab row, PML1_ROWS consecutive slab rows a block, so their taps' rows are
  // shared in L1
  const int r = blockIdx.y * PML1_ROWS + threadIdx.x / PML1_QUADS;  // the slab row
  const int z = 1 + blockIdx.z;                                      // the plane
  const int y = r < lo ? 1 + r : NM - 1 - hi + (r - lo);
  const int xq = 4 * (blockIdx.x * PML1_QUADS + threadIdx.x % PML1_QUADS);
  if (r < lo + hi && xq <= NF - 2) {
    const T *__restrict__ u1 = level<T>(p.u1, t);
    T *u2 = level<T>(p.u2, t);
    int mask = 0, xheld = 0;
    const int dirF = (g.dir >> 4) & 3, dirM = (g.dir >> 2) & 3;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int x = xq + i;
      if (x < 1 || x > NF - 2)
        continue;
      mask |= 1 << i;
      if (held_wall(x, NF, dirF))
        xheld |= 1 << i;
    }
    const int held = (held_wall(y, NM, dirM) || held_wall(z, N0, g.dir & 3)) ? mask : xheld;
    const long long s1 = g.s[1];
    const long long idx = (long long)z * g.s[0] + y * s1 + xq;
    // u^(t-1) on rows y - R .. y + R over the quad, past a wall off its mirror
    T rows[2 * R + 1][4];
    load4(rows[R], u1 + idx);
#pragma unroll
    for (int j = -R; j <= R; ++j) {
      if (j == 0)
        continue;
      int sg = 1;
      const int m = (y + j >= 0 && y + j <= NM - 1) ? y + j : mirror_node(y + j, NM, dirM, sg);
      load4(rows[R + j], u1 + idx + (m - y) * s1);
      if (sg < 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          rows[R + j][i] = -rows[R + j][i];
      }
    }
    T v[4], mi[4], m0[4], m1[4], m2[4];
    load4(v, u2 + idx);
    if (p.flags & K_DERIVE) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        mi[i] = (T)1 / p.sconst;
    } else {
      load4(mi, p.minv + idx);
    }
    T *aux = p.aux + ((long long)z * (lo + hi) + r) * g.ext[2] + xq;
    const long long sz = p.auxrow;
    get4m(aux, m0, mask);
    get4m(aux + sz, m1, mask);
    get4m(aux + 2 * sz, m2, mask);
    const T *prof = p.prof;
    const T an = prof[y], bn = prof[NM + y];
    const T ah = prof[2 * NM + y], bh = prof[3 * NM + y];
    const T ah1 = prof[2 * NM + y - 1], bh1 = prof[3 * NM + y - 1];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (!((mask >> i) & 1))
        continue;
      const auto tap = [&](const int j) { return rows[R + j][i]; };
      T Dpu, Dmu;
      diffs_plain<T, R>(tap, rows[R][i], p.w, Dpu, Dmu);
      pml_node(p.f, p.gconst, an, bn, ah, bh, ah1, bh1, Dpu, Dmu, m0[i], m1[i], m2[i], v[i],
               mi[i], (held >> i) & 1);
    }
    put4m(aux, m0, mask);
    put4m(aux + sz, m1, mask);
    put4m(aux + 2 * sz, m2, mask);
    put4m(u2 + idx, v, mask);
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

template <typename T, int R>
__global__ void __launch_bounds__(PML2_THREADS, 4) pml_axis2_kernel(const __grid_constant__ Pml3Params<T> p) {
  constexpr int H = (R + 3) / 4 * 4;  // the run's halo, whole quads
  constexpr int XR = 4 + 2 * H;
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  const int N0 = g.n[0], NM = g.n[1], NF = g.n[2];
  const int lo = g.lo[2], hi = g.hi[2];
  const int nq = p.nlo + p.nhi;
  const int rows_per_block = PML2_THREADS / nq;
  const int qi = threadIdx.x % nq, yl = threadIdx.x / nq;
  const int y = 1 + blockIdx.y * rows_per_block + yl;
  const int z = 1 + blockIdx.z;
  if (yl < rows_per_block && y <= NM - 2) {
    const T *__restrict__ u1 = level<T>(p.u1, t);
    T *u2 = level<T>(p.u2, t);
    const bool low = qi < p.nlo;
    const int xq = low ? 4 * qi : p.xhi + 4 * (qi - p.nlo);
    const int dirF = (g.dir >> 4) & 3, dirM = (g.dir >> 2) & 3;
    int in = 0, xheld = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      // the nodes of this side's slab (a quad both slabs reach is two threads' work)
      const int x = xq + i;
      if (x < 1 || x > NF - 2 || (low ? x > lo : x < NF - 1 - hi))
        continue;
      in |= 1 << i;
      if (held_wall(x, NF, dirF))
        xheld |= 1 << i;
    }
    if (in) {
      const int held = (held_wall(y, NM, dirM) || held_wall(z, N0, g.dir & 3)) ? in : xheld;
      const long long idx = (long long)z * g.s[0] + (long long)y * g.s[1] + xq;
      // the quad's run along axis 2, mirrored past the walls
      const int ext = g.ext[2];
      T xr[XR];
#pragma unroll
      for (int c = 0; c < XR / 4; ++c) {
        const int x = xq - H + 4 * c;
        if (x >= 0 && x + 3 <= ext - 1) {
          load4(xr + 4 * c, u1 + idx - H + 4 * c);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            xr[4 * c + i] = (T)0;
        }
      }
      if (xq - H < 0)
        mirror_run_lo_at<T, XR, H>(xr, (dirF & 1) ? (T)-1 : (T)1, H - xq);
      const int e_hi = NF - (xq - H);
      if (e_hi <= XR - 1)
        mirror_run_hi_at<T, XR, H + 2>(xr, (dirF & 2) ? (T)-1 : (T)1, e_hi);
      T v[4], mi[4];
      load4(v, u2 + idx);
      if (p.flags & K_DERIVE) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          mi[i] = (T)1 / p.sconst;
      } else {
        load4(mi, p.minv + idx);
      }
      const long long sz = p.auxrow;
      // the quad's slab nodes are consecutive slab indices of one side: the memory of
      // lane i at m + i, loaded for every lane before the first is written back
      const int f = __ffs(in) - 1;
      T *m = p.aux + ((long long)z * NM + y) * (lo + hi) + (slab_row(xq + f, NF, lo, hi) - f);
      T m0[4], m1[4], m2[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const bool on = (in >> i) & 1;
        m0[i] = on ? m[i] : (T)0;
        m1[i] = on ? m[sz + i] : (T)0;
        m2[i] = on ? m[2 * sz + i] : (T)0;
      }
      const T *prof = p.prof;
      // the half-point profile one node down is the lane before's own: loaded once for
      // the quad's first lane (xq >= 0: the slab nodes have x >= 1)
      T ah_prev = xq >= 1 ? prof[2 * NF + xq - 1] : (T)0;
      T bh_prev = xq >= 1 ? prof[3 * NF + xq - 1] : (T)0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int x = xq + i;
        // (the quad's last lanes may lie past the row's last node, NF - 1)
        const T ah = x <= NF - 1 ? prof[2 * NF + x] : (T)0;
        const T bh = x <= NF - 1 ? prof[3 * NF + x] : (T)0;
        if ((in >> i) & 1) {
          const auto tap = [&](const int j) { return xr[H + i + j]; };
          T Dpu, Dmu;
          diffs_plain<T, R>(tap, xr[H + i], p.w, Dpu, Dmu);
          pml_node(p.f, p.gconst, prof[x], prof[NF + x], ah, bh, ah_prev, bh_prev, Dpu, Dmu,
                   m0[i], m1[i], m2[i], v[i], mi[i], (held >> i) & 1);
        }
        ah_prev = ah;
        bh_prev = bh;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if ((in >> i) & 1) {
          m[i] = m0[i];
          m[sz + i] = m1[i];
          m[2 * sz + i] = m2[i];
        }
      // the face ghosts of axis 2 in this quad, refilled from their mirrors two nodes in
      // (homogeneous_neumann/dirichlet_kernel, scalar.cu:535-555), whose values are final
      // here: the host folds a face only when no source sits on its mirror column (the
      // sources come after the pml), its wall node held at zero already on a Dirichlet face
      int wmask = in;
      if ((p.fold & 1) && xq == 0) {
        v[0] = (dirF & 1) ? -v[2] : v[2];
        wmask |= 1;
      }
      if ((p.fold & 2) && xq + 2 <= NF - 1 && NF - 1 <= xq + 3) {
#pragma unroll
        for (int a = 2; a < 4; ++a)
          if (NF - 1 - xq == a) {
            v[a] = (dirF & 2) ? -v[a - 2] : v[a - 2];
            wmask |= 1 << a;
          }
      }
      put4m(u2 + idx, v, wmask);
    }
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

}  // namespace cwb
