// The pml memory update of one forward step along the axes after axis 0, over their slab
// nodes only.
//
// The blocked 3D step writes the update of every interior node with the axis-0 memory
// terms already in (an axis-0 slab row is a whole plane of its march); this kernel then
// visits the nodes of the slabs of axes 1 and 2 and, axis by axis in order, advances
// the node's memory (psi+, psi-, zeta) and adds its share to the update, as cuwave's
// pml_kernel does after fd_kernel (scalar.cu:429-532). The slab union is cut into
// disjoint boxes so that every node is visited once and applies its lined axes in the
// reference's order:
//
//   axis-1 slabs: every interior axis-0 plane, axis-1 rows of the slab (3D)
//   axis-2 slabs: every interior axis-0 plane, the axis-1 interior, the fast slab columns
//
// A thread owns four consecutive fast-axis nodes (a quad, 16-byte aligned) of one row,
// so the field, update and memory rows move as 16-byte vectors and consecutive threads
// read consecutive quads; axis-1 taps are the 2R rows of four around the node, axis-2
// taps the quad's run of 4 + 2H values. Taps past a wall take their mirrors (cuwave
// common.cuh:50-54).
#pragma once

#include "step.cuh"

namespace cwb {

constexpr int PML_THREADS = 256;

template <typename T>
struct PmlStepParams {
  Geometry g;
  T w[MAXR];
  T f[3];
  T gconst, sconst;
  int flags;  // K_DERIVE, K_ADV
  DLevel u1, u2;
  const T *stiff, *minv;
  const T *prof[3];
  T *aux[3];
  int auxrow[3];
  int nbox;
  int org[6][3], ext[6][3];  // per box: first node and extent along each axis
  long long end[6];          // running thread count at each box's end
  int *ctr;
};

template <typename T, int NDIM, int R, bool UNIF>
__global__ void __launch_bounds__(PML_THREADS, 4) pml_step_kernel(const __grid_constant__ PmlStepParams<T> p) {
  constexpr int F = NDIM - 1;
  constexpr int H = (R + 3) / 4 * 4;  // the run's halo, whole quads
  constexpr int XR = 4 + 2 * H;
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  const long long k = (long long)blockIdx.x * PML_THREADS + threadIdx.x;
  if (k < p.end[p.nbox - 1]) {
    const T *__restrict__ u1 = level<T>(p.u1, t);
    T *u2 = level<T>(p.u2, t);
    int b = 0;
    while (k >= p.end[b])
      ++b;
    int local = (int)(k - (b ? p.end[b - 1] : 0));  // a box holds fewer than 2^31 threads
    // the thread's quad (fast axis), its axis-1 row (3D) and its axis-0 plane
    const int x0 = p.org[b][F], x1 = p.org[b][F] + p.ext[b][F] - 1;
    const int nq = (x1 >> 2) - (x0 >> 2) + 1;
    int q = local / nq;
    const int xq = ((x0 >> 2) + (local - q * nq)) * 4;
    local = q;
    int y = 0;
    if (NDIM == 3) {  // the box's axis-1 extent
      const int e = p.ext[b][1];
      q = local / e;
      y = p.org[b][1] + (local - q * e);
      local = q;
    }
    const int z = p.org[b][0] + local;
    const int N0 = g.n[0], NF = g.n[F];
    const int dir0 = g.dir & 3, dirF = (g.dir >> (2 * F)) & 3;
    const long long s0 = g.s[0];
    const long long col = (NDIM == 3 ? (long long)y * g.s[1] : 0) + xq;
    // the quad's nodes in the box, their Dirichlet walls, their place in the fast slab
    int mask = 0, xheld = 0, in = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int x = xq + i;
      if (x < x0 || x > x1)
        continue;
      mask |= 1 << i;
      if (held_wall(x, NF, dirF))
        xheld |= 1 << i;
      if (slab_row(x, NF, g.lo[F], g.hi[F]) >= 0)
        in |= 1 << i;
    }
    const bool yheld = NDIM == 3 && held_wall(y, g.n[1], (g.dir >> 2) & 3);
    const int yrow = NDIM == 3 ? slab_row(y, g.n[1], g.lo[1], g.hi[1]) : -1;
    const auto get4 = [&](const T *base, T *dst) {
      if (mask == 15) {
        load4(dst, base);
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          dst[i] = ((mask >> i) & 1) ? base[i] : (T)0;
      }
    };
    const auto put4 = [&](T *base, const T *src) {
      if (mask == 15) {
        store4(base, src);
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if ((mask >> i) & 1)
            base[i] = src[i];
      }
    };
    {
      const long long idx = z * s0 + col;
      T v[4], uc[4], mi[4], sc[4];
      get4(u2 + idx, v);
      get4(u1 + idx, uc);
      if (UNIF) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          sc[i] = p.sconst;
      } else {
        get4(p.stiff + idx, sc);
      }
      if (p.flags & K_DERIVE) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          mi[i] = (T)1 / sc[i];
      } else {
        get4(p.minv + idx, mi);
      }
      const int held = (yheld || held_wall(z, N0, dir0)) ? mask : xheld;
      // one node's memory step and share of the update along axis d (pml_kernel's order)
      const auto node = [&](const int i, const int d, const int a, const int N, const T Dpu,
                            const T Dmu, T &m0, T &m1, T &m2) {
        const long long st = g.s[d];
        T gp = p.gconst, gm = p.gconst;
        if (!UNIF) {
          const T sp = p.stiff[idx + i + st], sm = p.stiff[idx + i - st];
          gp = sc[i] * sp / (sc[i] + sp);
          gm = sc[i] * sm / (sc[i] + sm);
        }
        const T *prof = p.prof[d];
        const T an = prof[a], bn = prof[N + a];
        const T ah = prof[2 * N + a], bh = prof[3 * N + a];
        const T ah1 = prof[2 * N + a - 1], bh1 = prof[3 * N + a - 1];
        const T f = p.f[d];
        const T pp = bh * m0 + ah * Dpu;
        const T pm = bh1 * m1 + ah1 * Dmu;
        const T zz = bn * m2 + an * f * (gp * (Dpu + pp) - gm * (Dmu + pm));
        m0 = pp;
        m1 = pm;
        m2 = zz;
        if (!((held >> i) & 1))
          v[i] += mi[i] * (f * (gp * pp - gm * pm) + zz);
      };
      // the memory rows of a slow axis: contiguous over the quad
      const auto slow = [&](const int d, const int a, const int N, const long long si,
                            const T (*tq)[4]) {
        T *aux = p.aux[d];
        const long long sz = p.auxrow[d];
        T m0[4], m1[4], m2[4];
        get4(aux + si, m0);
        get4(aux + sz + si, m1);
        get4(aux + 2 * sz + si, m2);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (!((mask >> i) & 1))
            continue;
          const auto tap = [&](const int j) { return tq[R + j][i]; };
          T Dpu, Dmu;
          diffs_plain<T, R>(tap, uc[i], p.w, Dpu, Dmu);
          node(i, d, a, N, Dpu, Dmu, m0[i], m1[i], m2[i]);
        }
        put4(aux + si, m0);
        put4(aux + sz + si, m1);
        put4(aux + 2 * sz + si, m2);
      };
      if (NDIM == 3 && yrow >= 0) {
        const int N1 = g.n[1], odd = (g.dir >> 2) & 3;
        const long long s1 = g.s[1];
        T tq[2 * R + 1][4];
#pragma unroll
        for (int j = -R; j <= R; ++j) {
          if (j == 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
              tq[R][i] = uc[i];
            continue;
          }
          int sg = 1;
          const int m = (y + j >= 0 && y + j <= N1 - 1) ? y + j : mirror_node(y + j, N1, odd, sg);
          get4(u1 + idx + (long long)(m - y) * s1, tq[R + j]);
          if (sg < 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
              tq[R + j][i] = -tq[R + j][i];
          }
        }
        const int rows = g.lo[1] + g.hi[1];
        slow(1, y, N1, ((long long)z * rows + yrow) * g.ext[2] + xq, tq);
      }
      if (in) {
        // the fast axis: the quad's run, mirrored past the walls
        const int ext = g.ext[F];
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
          mirror_run_lo<T, XR, H>(xr, (dirF & 1) ? (T)-1 : (T)1);
        const int e_hi = NF - (xq - H);
        if (e_hi <= XR - 1)
          mirror_run_hi_at<T, XR, H + 2>(xr, (dirF & 2) ? (T)-1 : (T)1, e_hi);
        const int lo = g.lo[F], hi = g.hi[F];
        T *aux = p.aux[F];
        const long long sz = p.auxrow[F];
        const long long row = NDIM == 3 ? ((long long)z * g.n[1] + y) * (lo + hi)
                                        : (long long)z * (lo + hi);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (!((in >> i) & 1))
            continue;
          const int x = xq + i;
          const auto tap = [&](const int j) { return xr[H + i + j]; };
          T Dpu, Dmu;
          diffs_plain<T, R>(tap, uc[i], p.w, Dpu, Dmu);
          const long long si = row + slab_row(x, NF, lo, hi);
          node(i, F, x, NF, Dpu, Dmu, aux[si], aux[sz + si], aux[2 * sz + si]);
        }
      }
      put4(u2 + idx, v);
    }
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

}  // namespace cwb
