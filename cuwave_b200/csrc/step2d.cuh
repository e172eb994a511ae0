// The 2D forward step of a uniform stiffness: quads of four fast-axis nodes marching rows.
//
// A thread owns four consecutive axis-1 nodes (a quad, 16-byte aligned) and marches a
// chunk of axis-0 rows. It keeps, per node, the 2R values u(z-R+1) .. u(z+R) of its
// column in a register queue fed one row per step and carries g * D+ of the row before as
// this row's g * D- (the same expression of the same values, so the reuse is bit-exact).
// The axis-1 taps are the quad's run of 4 + 2H values: the queue's centre row and two
// 16-byte loads beside it, which neighbouring threads share through L1. There is no
// shared memory and no barrier: every load is a coalesced 16-byte row and warps run
// independently.
//
// The node arithmetic is step.cuh's (cuwave fd_kernel, scalar.cu:347-427) in the same
// order, Dirichlet wall nodes held at zero. An axis-0 pml slab row is a whole row of the
// march, so its memory terms apply uniformly over the row; the axis-1 slab columns apply
// theirs quad by quad after it (cuwave pml_kernel, scalar.cu:500-532, axes in order).
// The sources and the ghost refill follow as launches of their own, in the order of
// cuwave's step. Values past a wall take their mirrors (cuwave common.cuh:50-54): along
// axis 1 in the run's registers, along axis 0 by reading the mirror row.
#pragma once

#include <cooperative_groups.h>

#include "step.cuh"
#include "transfer.cuh"

namespace cwb {

constexpr int S2_THREADS = 128;

template <typename T, int R>
struct Step2Shape {
  static constexpr int H = (R + 3) / 4 * 4;  // the run's halo, whole quads
  static constexpr int XR = 4 + 2 * H;
  // float (16-byte quads of four); the queue of 2R rows of four fits four blocks of 128
  // threads an SM up to radius 5, two from 6 on
  static constexpr bool SUPPORTED = sizeof(T) == 4 && R <= 8;
  static constexpr int MIN_BLOCKS = R <= 5 ? 4 : 2;
};

// The sources and the ghost refill a multi-step march folds into the step: the sources
// added node by node after the pml (cuwave excitation_kernel, common.cuh:456-464), the
// ghosts written from their mirror rows (cuwave scalar.cu:535-555). None in a plain step.
template <typename T>
struct Fold2 {
  const int *lin;       // flat source nodes
  const T *weight;      // their weights
  const T *signal;      // (rows, nsrc)
  int nsrc, sig_mul, sig_add;
  int refill;           // faces whose ghosts are written
};

// unit k (a quad and a chunk of rows) of the step at t; HOLD: the grid has a Dirichlet
// face (without one, the faces' masks are zero at compile time and the wall tests fold);
// PML: the pml memory terms are applied here (else pml2d_kernel applies them after)
template <typename T, int R, bool HOLD = true, bool PML = true>
__device__ __forceinline__ void step2d_rows(const StepParams<T> &p, const int t, const long long k,
                                            const Fold2<T> &fold) {
  using S = Step2Shape<T, R>;
  constexpr int H = S::H, XR = S::XR;
  const Geometry &g = p.g;
  const int N0 = g.n[0], NF = g.n[1], ext = g.ext[1];
  const int nq = (NF - 2) / 4 + 1;  // quads covering nodes 0 .. NF - 2
  const int quad = (int)(k % nq);
  const int cz = (int)(k / nq);
  const int c0 = 1 + cz * p.chunk;
  const int c1 = min(N0 - 1, c0 + p.chunk);
  const int xq = 4 * quad;
  if (c0 < c1 && xq <= NF - 2) {
    const T *__restrict__ u0 = level<T>(p.u0, t);
    const T *__restrict__ u1 = level<T>(p.u1, t);
    T *u2 = level<T>(p.u2, t);
    const T *__restrict__ minv = p.minv;
    const int dir0 = HOLD ? g.dir & 3 : 0, dirF = HOLD ? (g.dir >> 2) & 3 : 0;
    const int s0 = g.s[0];
    const int flags = p.flags;
    const T gg = p.gconst;
    // the quad's interior nodes, its Dirichlet wall nodes, its axis-1 slab nodes
    int inner = 0, xheld = 0, xslab = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int x = xq + i;
      if (x < 1 || x > NF - 2)
        continue;
      inner |= 1 << i;
      if (held_wall(x, NF, dirF))
        xheld |= 1 << i;
      if (PML && (flags & K_PML) && slab_row(x, NF, g.lo[1], g.hi[1]) >= 0)
        xslab |= 1 << i;
    }
    const bool fix_lo = xq - H < 0;
    const int e_hi = NF - (xq - H);
    const bool fix_hi = e_hi <= XR - 1;
    const T slo = (dirF & 1) ? (T)-1 : (T)1, shi = (dirF & 2) ? (T)-1 : (T)1;
    const T mi_derived = (flags & K_DERIVE) ? (T)1 / p.sconst : (T)0;
    // u^(t-1) over the quad at row b, through its mirror past the axis-0 walls
    const auto row4 = [&](const int b, T *dst) {
      int sg = 1;
      const int m = (b >= 0 && b <= N0 - 1) ? b : mirror_node(b, N0, dir0, sg);
      load4(dst, u1 + (long long)m * s0 + xq);
      if (sg < 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          dst[i] = -dst[i];
      }
    };
    // the queue q[k] = u(z - R + 1 + k) and g * D+ of the row before (which reads u(c0 - R))
    T q[2 * R][4], pz[4];
    {
      T first[4];
      row4(c0 - R, first);
#pragma unroll
      for (int j = 0; j < 2 * R - 1; ++j)
        row4(c0 - R + 1 + j, q[j]);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const auto tap = [&](const int j) { return j == -R + 1 ? first[i] : q[R - 2 + j][i]; };
        pz[i] = mul_rn(dplus<T, R>(tap, tap(0), p.w), gg);
      }
    }
    for (int z = c0; z < c1; ++z) {
      row4(z + R, q[2 * R - 1]);
      const long long row = (long long)z * s0 + xq;
      // the run along axis 1: left quad, the queue's centre, right quad; mirrored
      T xr[XR];
#pragma unroll
      for (int c = 0; c < XR / 4; ++c) {
        const int x = xq - H + 4 * c;
        if (c == H / 4) {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            xr[4 * c + i] = q[R - 1][i];
        } else if (x >= 0 && x + 3 <= ext - 1) {
          load4(xr + 4 * c, u1 + row - H + 4 * c);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            xr[4 * c + i] = (T)0;
        }
      }
      if (fix_lo)
        mirror_run_lo_at<T, XR, H>(xr, slo, H - xq);
      if (fix_hi)
        mirror_run_hi_at<T, XR, H + 2>(xr, shi, e_hi);
      T old[4], mi[4];
      load4(old, u0 + row);
      if (flags & K_DERIVE) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          mi[i] = mi_derived;
      } else {
        load4(mi, minv + row);
      }
      // axis 1: D+ at faces x0 - 1 .. x0 + 3; axis 0 from the queue; the laplacian
      T dx[5];
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const auto tap = [&](const int kk) { return xr[H - 1 + j + kk]; };
        dx[j] = dplus<T, R>(tap, xr[H - 1 + j], p.w);
      }
      T v[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const auto tap = [&](const int j) { return q[R - 1 + j][i]; };
        const T dpz = dplus<T, R>(tap, q[R - 1][i], p.w);
        const T ddz = fma_rn(dpz, gg, -pz[i]);
        pz[i] = mul_rn(dpz, gg);
        const T ddx = fma_rn(dx[i + 1], gg, -mul_rn(dx[i], gg));
        const T lap = R == 1 ? fma_rn(p.f[0], ddz, mul_rn(p.f[1], ddx))
                             : fma_rn(p.f[1], ddx, mul_rn(p.f[0], ddz));
        const T uc = q[R - 1][i];
        if (flags & K_DAMP) {
          const T dmp = ((inner >> i) & 1) ? p.damping[row + i] : (T)0;
          const T beta = (T)0.5 * mi[i] * dmp * p.dt;
          v[i] = ((T)2 * uc - old[i] * ((T)1 - beta) + mi[i] * lap) / ((T)1 + beta);
        } else {
          v[i] = -old[i] + (T)2 * uc + mi[i] * lap;
        }
      }
      const int held = held_wall(z, N0, dir0) ? inner : xheld;
      if (held) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if ((held >> i) & 1)
            v[i] = (T)0;
      }
      if (PML && (flags & K_PML)) {
        // one node's memory step and share of the update along axis d (pml_kernel's order)
        const auto node = [&](const int i, const int d, const int a, const int N, const T Dpu,
                              const T Dmu, T &m0, T &m1, T &m2) {
          const T *prof = p.prof[d];
          const T an = prof[a], bn = prof[N + a];
          const T ah = prof[2 * N + a], bh = prof[3 * N + a];
          const T ah1 = prof[2 * N + a - 1], bh1 = prof[3 * N + a - 1];
          const T f = p.f[d];
          const T pp = bh * m0 + ah * Dpu;
          const T pm = bh1 * m1 + ah1 * Dmu;
          const T zz = bn * m2 + an * f * (gg * (Dpu + pp) - gg * (Dmu + pm));
          m0 = pp;
          m1 = pm;
          m2 = zz;
          if (!((held >> i) & 1))
            v[i] += mi[i] * (f * (gg * pp - gg * pm) + zz);
        };
        const int zrow = slab_row(z, N0, g.lo[0], g.hi[0]);
        if (zrow >= 0) {
          // an axis-0 slab row: its memory row is contiguous over the quad
          T last[4];
          row4(z - R, last);
          T *aux = p.aux[0];
          const long long sz = p.auxrow[0], si = (long long)zrow * ext + xq;
          T m0[4], m1[4], m2[4];
          load4(m0, aux + si);
          load4(m1, aux + sz + si);
          load4(m2, aux + 2 * sz + si);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            if (!((inner >> i) & 1))
              continue;
            const auto tap = [&](const int j) { return j == -R ? last[i] : q[R - 1 + j][i]; };
            T Dpu, Dmu;
            diffs_plain<T, R>(tap, q[R - 1][i], p.w, Dpu, Dmu);
            node(i, 0, z, N0, Dpu, Dmu, m0[i], m1[i], m2[i]);
          }
          // the quad's nodes outside the interior keep their memory
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if ((inner >> i) & 1) {
              aux[si + i] = m0[i];
              aux[sz + si + i] = m1[i];
              aux[2 * sz + si + i] = m2[i];
            }
        }
        if (xslab) {
          // the quad's memories loaded before any is stored, so their loads are in flight
          // together (a store between them would order each load after it)
          T *aux = p.aux[1];
          const long long sz = p.auxrow[1];
          const int lo = g.lo[1], hi = g.hi[1];
          const long long base = (long long)z * (lo + hi);
          long long si[4];
          T m0[4], m1[4], m2[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            si[i] = base + ((xslab >> i) & 1 ? slab_row(xq + i, NF, lo, hi) : 0);
            if ((xslab >> i) & 1) {
              m0[i] = aux[si[i]];
              m1[i] = aux[sz + si[i]];
              m2[i] = aux[2 * sz + si[i]];
            }
          }
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            if (!((xslab >> i) & 1))
              continue;
            const int x = xq + i;
            const auto tap = [&](const int j) { return xr[H + i + j]; };
            T Dpu, Dmu;
            diffs_plain<T, R>(tap, xr[H + i], p.w, Dpu, Dmu);
            node(i, 1, x, NF, Dpu, Dmu, m0[i], m1[i], m2[i]);
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if ((xslab >> i) & 1) {
              aux[si[i]] = m0[i];
              aux[sz + si[i]] = m1[i];
              aux[2 * sz + si[i]] = m2[i];
            }
        }
      }
      if (fold.nsrc) {
        // the sources of this quad, in the list's order
        const long long srow = (long long)fold.sig_mul * t + fold.sig_add;
        for (int e = 0; e < fold.nsrc; ++e) {
          const long long n = fold.lin[e] - row;
          if (n >= 0 && n < 4) {
            const T add = fold.weight[e] * fold.signal[srow * fold.nsrc + e];
#pragma unroll
            for (int i = 0; i < 4; ++i)
              if (n == i)
                v[i] += add;
          }
        }
      }
      if (inner == 15) {
        store4(u2 + row, v);
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if ((inner >> i) & 1)
            u2[row + i] = v[i];
      }
      if (fold.refill) {
        const int fr = fold.refill;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (!((inner >> i) & 1))
            continue;
          const int x = xq + i;
          if ((fr & 1) && z == 2)
            u2[row + i - 2LL * s0] = (dir0 & 1) ? -v[i] : v[i];
          if ((fr & 2) && z == N0 - 3)
            u2[row + i + 2LL * s0] = (dir0 & 2) ? -v[i] : v[i];
          if ((fr & 4) && x == 2)
            u2[row + i - 2] = (dirF & 1) ? -v[i] : v[i];
          if ((fr & 8) && x == NF - 3)
            u2[row + i + 2] = (dirF & 2) ? -v[i] : v[i];
        }
      }
#pragma unroll
      for (int j = 0; j < 2 * R - 1; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i)
          q[j][i] = q[j + 1][i];
    }
  }
}

template <typename T, int R, bool UNIF, bool HOLD = true, bool PML = true>
__global__ void __launch_bounds__(S2_THREADS, Step2Shape<T, R>::MIN_BLOCKS)
    step2d_kernel(const StepParams<T> p) {
  static_assert(Step2Shape<T, R>::SUPPORTED && UNIF,
                "the 2D quad step is built for float and a uniform stiffness");
  const Fold2<T> none{};
  step2d_rows<T, R, HOLD, PML>(p, step_index(p.ctr), (long long)blockIdx.x * S2_THREADS + threadIdx.x,
                               none);
  finish_step(p.ctr, p.flags & K_ADV);
}

// The pml memory terms of a 2D quad step, after step2d_kernel<..., PML = false> wrote the
// update and before the sources: the nodes of the axis-0 slab rows (every quad of those
// rows; a quad there holding axis-1 slab nodes takes that axis' share after axis 0's),
// then, in the other rows, the axis-1 slab quads of each side. A thread per quad and
// row, its update, 1/m and memories loaded, the memory advanced from the plain
// differences of u^(t-1) along the axis and the share added unless the node is held
// (cuwave pml_kernel, scalar.cu:500-532, in step2d_rows' arithmetic and order). Kept out
// of the update kernel, whose every thread would otherwise carry the slab code's
// registers and wait on the memory's loads in the few warps that hold slab nodes.
struct Pml2Layout {
  int nq;            // quads a row
  int nlo, nhi, xhi;  // axis-1 slab quads on each side, the first high one's x
  long long na;      // threads of the axis-0 slab rows
  long long total;   // all threads
  int fold;          // face ghosts refilled here (1 row 0, 2 row N0-1, 4 column 0, 8 column NF-1)
};

// `src`: the step's sources when none sits on a node this launch writes (its num 0
// otherwise): threads past the slab quads add them, as excite_kernel would after it.
// `rec`: the record op that follows the step, when its nodes are final before this launch
// (interior, no slab node, no source): threads past those read them, as record_kernel would
template <typename T, int R, bool HOLD>
__global__ void __launch_bounds__(S2_THREADS) pml2d_kernel(const StepParams<T> p, const Pml2Layout lay,
                                                           const TransferParams<T> src,
                                                           const TransferParams<T> rec) {
  using S = Step2Shape<T, R>;
  constexpr int H = S::H, XR = S::XR;
  const long long k = (long long)blockIdx.x * S2_THREADS + threadIdx.x;
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  if (k < lay.total) {
    const int N0 = g.n[0], NF = g.n[1], ext = g.ext[1];
    const int lo0 = g.lo[0], hi0 = g.hi[0], lo1 = g.lo[1], hi1 = g.hi[1];
    int z, xq, side = 0;  // side: 0 both axes' slab nodes, 1 the low axis-1 slab, 2 the high
    if (k < lay.na) {
      const int ra = (int)(k / lay.nq);
      z = ra < lo0 ? 1 + ra : N0 - 1 - hi0 + (ra - lo0);
      xq = 4 * (int)(k % lay.nq);
    } else {
      const long long kb = k - lay.na;
      const int nqs = lay.nlo + lay.nhi;
      const int qi = (int)(kb % nqs);
      z = lo0 + 1 + (int)(kb / nqs);
      side = qi < lay.nlo ? 1 : 2;
      xq = side == 1 ? 4 * qi : lay.xhi + 4 * (qi - lay.nlo);
    }
    const T *__restrict__ u1 = level<T>(p.u1, t);
    T *u2 = level<T>(p.u2, t);
    const int dir0 = HOLD ? g.dir & 3 : 0, dirF = HOLD ? (g.dir >> 2) & 3 : 0;
    const int s0 = g.s[0];
    const T gg = p.gconst;
    int inner = 0, xheld = 0, xslab = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int x = xq + i;
      if (x < 1 || x > NF - 2)
        continue;
      inner |= 1 << i;
      if (held_wall(x, NF, dirF))
        xheld |= 1 << i;
      const bool lo_node = lo1 && x <= lo1, hi_node = hi1 && x >= NF - 1 - hi1;
      if (side == 0 ? (lo_node || hi_node) : side == 1 ? lo_node : hi_node)
        xslab |= 1 << i;
    }
    const int mine = side == 0 ? inner : xslab;  // the nodes this thread writes
    if (mine) {
      const long long row = (long long)z * s0 + xq;
      T v[4], mi[4];
      load4(v, u2 + row);
      if (p.flags & K_DERIVE) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          mi[i] = (T)1 / p.sconst;
      } else {
        load4(mi, p.minv + row);
      }
      const int held = held_wall(z, N0, dir0) ? inner : xheld;
      const auto node = [&](const int i, const int d, const int a, const int N, const T Dpu,
                            const T Dmu, T &m0, T &m1, T &m2) {
        const T *prof = p.prof[d];
        const T an = prof[a], bn = prof[N + a];
        const T ah = prof[2 * N + a], bh = prof[3 * N + a];
        const T ah1 = prof[2 * N + a - 1], bh1 = prof[3 * N + a - 1];
        const T f = p.f[d];
        const T pp = bh * m0 + ah * Dpu;
        const T pm = bh1 * m1 + ah1 * Dmu;
        const T zz = bn * m2 + an * f * (gg * (Dpu + pp) - gg * (Dmu + pm));
        m0 = pp;
        m1 = pm;
        m2 = zz;
        if (!((held >> i) & 1))
          v[i] += mi[i] * (f * (gg * pp - gg * pm) + zz);
      };
      if (side == 0) {
        // an axis-0 slab row: u^(t-1) on rows z - R .. z + R through the axis-0 mirrors
        T col[2 * R + 1][4];
#pragma unroll
        for (int j = -R; j <= R; ++j) {
          const int b = z + j;
          int sg = 1;
          const int m = (b >= 0 && b <= N0 - 1) ? b : mirror_node(b, N0, dir0, sg);
          load4(col[R + j], u1 + (long long)m * s0 + xq);
          if (sg < 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
              col[R + j][i] = -col[R + j][i];
          }
        }
        T *aux = p.aux[0];
        const long long sz = p.auxrow[0], si = (long long)slab_row(z, N0, lo0, hi0) * ext + xq;
        T m0[4], m1[4], m2[4];
        load4(m0, aux + si);
        load4(m1, aux + sz + si);
        load4(m2, aux + 2 * sz + si);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (!((inner >> i) & 1))
            continue;
          const auto tap = [&](const int j) { return col[R + j][i]; };
          T Dpu, Dmu;
          diffs_plain<T, R>(tap, col[R][i], p.w, Dpu, Dmu);
          node(i, 0, z, N0, Dpu, Dmu, m0[i], m1[i], m2[i]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if ((inner >> i) & 1) {
            aux[si + i] = m0[i];
            aux[sz + si + i] = m1[i];
            aux[2 * sz + si + i] = m2[i];
          }
      }
      if (xslab) {
        // the quad's run of u^(t-1) along axis 1, mirrored past the walls
        T xr[XR];
#pragma unroll
        for (int c = 0; c < XR / 4; ++c) {
          const int x = xq - H + 4 * c;
          if (x >= 0 && x + 3 <= ext - 1) {
            load4(xr + 4 * c, u1 + row - H + 4 * c);
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
        // the quad's slab nodes are consecutive slab indices of one side: the memory of
        // lane i at m + i, loaded for every lane before the first is written back
        const long long sz = p.auxrow[1];
        const int f = __ffs(xslab) - 1;
        T *m = p.aux[1] + (long long)z * (lo1 + hi1) + (slab_row(xq + f, NF, lo1, hi1) - f);
        T m0[4], m1[4], m2[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const bool on = (xslab >> i) & 1;
          m0[i] = on ? m[i] : (T)0;
          m1[i] = on ? m[sz + i] : (T)0;
          m2[i] = on ? m[2 * sz + i] : (T)0;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (!((xslab >> i) & 1))
            continue;
          const int x = xq + i;
          const auto tap = [&](const int j) { return xr[H + i + j]; };
          T Dpu, Dmu;
          diffs_plain<T, R>(tap, xr[H + i], p.w, Dpu, Dmu);
          node(i, 1, x, NF, Dpu, Dmu, m0[i], m1[i], m2[i]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if ((xslab >> i) & 1) {
            m[i] = m0[i];
            m[sz + i] = m1[i];
            m[2 * sz + i] = m2[i];
          }
      }
      // the face ghosts whose mirrors this thread holds, refilled from them (cuwave
      // scalar.cu:535-555): the host folds a face here only when no source sits on its
      // mirror row or column (the sources come after the pml, the refill after them)
      int wmask = mine;
      if ((lay.fold & 4) && xq == 0) {
        v[0] = (dirF & 1) ? -v[2] : v[2];
        wmask |= 1;
      }
      if ((lay.fold & 8) && xq + 2 <= NF - 1 && NF - 1 <= xq + 3) {
#pragma unroll
        for (int a = 2; a < 4; ++a)
          if (NF - 1 - xq == a) {
            v[a] = (dirF & 2) ? -v[a - 2] : v[a - 2];
            wmask |= 1 << a;
          }
      }
      if (wmask == 15) {
        store4(u2 + row, v);
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if ((wmask >> i) & 1)
            u2[row + i] = v[i];
      }
      if (side == 0 && (((lay.fold & 1) && z == 2) || ((lay.fold & 2) && z == N0 - 3))) {
        const bool top = z == 2;
        const T sg = (dir0 & (top ? 1 : 2)) ? (T)-1 : (T)1;
        T *ghost = u2 + row + (top ? -2LL : 2LL) * s0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if ((inner >> i) & 1)
            ghost[i] = sg * v[i];
      }
    }
  } else if (k < lay.total + src.num) {
    // a source (excite_kernel's add): its node is no slab node, so no thread above
    // writes it, and no face this launch refills mirrors it
    const int j = (int)(k - lay.total);
    T *a = level<T>(src.a, t);
    const long long srow = (long long)src.row_mul * t + src.row_add;
    atomic_add_exact(&a[src.lin[j]], src.weight[j] * record_read(src, srow * src.num + j));
  } else if (k < lay.total + src.num + rec.num) {
    // a receiver (record_kernel's read) of a node no launch of the step writes after the
    // update
    const int j = (int)(k - lay.total - src.num);
    const T *a = level<T>(rec.a, t);
    const long long rrow = (long long)rec.row_mul * t + rec.row_add;
    record_write(rec, rrow * rec.num + j, a[rec.lin[j]]);
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// The multi-step march of an L2-resident 2D grid: one cooperative launch runs `steps`
// steps of [step (sources and refill folded), records] with a grid-wide barrier between a
// step and its records, where the plain march launches four kernels a step. It stands in
// for cuwave's blocked_kernel (several steps per launch, excitation, refill and record
// folded in; scalar.cu:571-791) on a grid whose fields stay in L2 between steps.
constexpr int MARCH2_RECORDS = 4;

template <typename T>
struct March2Params {
  StepParams<T> s;
  Fold2<T> fold;
  TransferParams<T> rec[MARCH2_RECORDS];  // store, level and rows of each record
  int nrec;
  int t0, steps;
  long long units;  // quads x row chunks
};

template <typename T, int R, bool HOLD = true, bool PML = true>
__global__ void __launch_bounds__(S2_THREADS, Step2Shape<T, R>::MIN_BLOCKS)
    march2d_kernel(const __grid_constant__ March2Params<T> mp) {
  static_assert(Step2Shape<T, R>::SUPPORTED, "the 2D quad step is built for float");
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gsize = (long long)gridDim.x * blockDim.x;
  for (int s = 0; s < mp.steps; ++s) {
    const int t = mp.t0 + s;
    for (long long k = gtid; k < mp.units; k += gsize)
      step2d_rows<T, R, HOLD, PML>(mp.s, t, k, mp.fold);
    grid.sync();  // the step's nodes and ghosts are all written
    for (int r = 0; r < mp.nrec; ++r) {
      const TransferParams<T> &rp = mp.rec[r];
      const T *a = level<T>(rp.a, t);
      const long long row = (long long)rp.row_mul * t + rp.row_add;
      for (long long j = gtid; j < rp.num; j += gsize)
        record_write(rp, row * rp.num + j, a[rp.lin[j]]);
    }
    // the next step writes the level two back and reads this one: no barrier needed
  }
  if (gtid == 0) {
    mp.s.ctr[1] = 0;
    mp.s.ctr[0] = mp.t0 + mp.steps;
  }
}

}  // namespace cwb
