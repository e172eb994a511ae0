// The 2D transposed step of a uniform stiffness, with or without the gradient densities:
// quads of four fast-axis nodes marching rows, like step2d.cuh.
//
// MODE_STEP       lambda^n = 2 lambda^(n+1) - lambda^(n+2) + dt^2/m (W^-1 A^T W lambda^(n+1))
//                 (cuwave adjoint_kernel, scalar_sensitivity.cu:388-441), the pml transpose
//                 (pml_adjoint_kernel, 545-597) gathered after it by adjoint2d_pml_kernel
//                 over the nodes within R of a slab;
// MODE_STEP_GRAD  the same, accumulating g_mass and g_stiff against u^n
//                 (adjoint_gradient_kernel, scalar_sensitivity.cu:444-515).
//
// A thread owns a quad and marches a chunk of rows, reading the axis-0 taps (lambda^(n+1)
// over rows z-R .. z+R, u^n over rows z-R+1 .. z+R) row by row as 16-byte rows of its
// column, which the rows before brought into L1 (register queues of them measured
// slower: their 68 registers and shifts cost more than the L1 reads), and the quad's
// axis-1 runs of 4 + 2H values. The taps read through the node image (a stored ghost is
// never read; lambda and u odd across a Dirichlet face) and read zero on a held wall
// node, as cuwave's `reflected` does (scalar_sensitivity.cu:177-184). Along axis 1 the quad shares its runs' first
// differences and the plain D+ of u between neighbouring nodes: the same subtractions and
// products of the same values the per-node form performs, so the sums are bit-identical;
// a node on a held wall keeps the per-node form (its own value is not its taps' zero).
// The arithmetic order is transposed_divergence_taps and stiffness_gradient_taps
// (scalar_sensitivity.cu:119-154).
#pragma once

#include <type_traits>

#include "adjoint.cuh"
#include "step.cuh"

namespace cwb {

constexpr int A2_THREADS = 128;
constexpr int A2_MIN_BLOCKS = 4;  // blocks an SM (128 registers a thread)

template <typename T, int R>
struct Adj2Shape {
  static constexpr int H = (R + 3) / 4 * 4;
  static constexpr int XR = 4 + 2 * H;
  static constexpr bool SUPPORTED = sizeof(T) == 4 && R <= 4;
};

// xr[c] = 0 at the run index c = e (a held wall node), e known at run time
template <typename T, int XR>
__device__ __forceinline__ void zero_at(T *xr, const int e) {
#pragma unroll
  for (int c = 0; c < XR; ++c)
    if (c == e)
      xr[c] = (T)0;
}

// A run of nodes xq - H .. xq + 3 + H along the fast axis read through the node image
// (node b < 1 reads 2 - b, b > N - 2 reads 2(N - 2) - b, odd across a Dirichlet face),
// zero on a held wall node
template <typename T, int XR, int H>
__device__ __forceinline__ void image_run(T *xr, const T *row, const int xq, const int N,
                                          const int ext, const int odd) {
#pragma unroll
  for (int c = 0; c < XR / 4; ++c) {
    const int x = xq - H + 4 * c;
    if (x >= 0 && x + 3 <= ext - 1) {
      load4(xr + 4 * c, row - H + 4 * c);
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        xr[4 * c + i] = (T)0;
    }
  }
  if (xq - H < 1 || xq + 3 + H > N - 2) {
    // rebuild the positions past the walls from the stored interior ones
    T raw[XR];
#pragma unroll
    for (int c = 0; c < XR; ++c)
      raw[c] = xr[c];
#pragma unroll
    for (int c = 0; c < XR; ++c) {
      const int b = xq - H + c;
      if (b < 1 || b > N - 2) {
        int sg;
        const int m = node_image(b, N, odd, sg);
        const int cm = m - (xq - H);
        T v = (T)0;
#pragma unroll
        for (int s = 0; s < XR; ++s)
          if (s == cm)
            v = raw[s];
        xr[c] = sg < 0 ? -v : v;
      }
    }
  }
  if (odd & 1)
    zero_at<T, XR>(xr, 1 - (xq - H));
  if (odd & 2)
    zero_at<T, XR>(xr, N - 2 - (xq - H));
}

// HOLD: the grid has a Dirichlet face (without one, the faces' masks are zero at compile
// time and every wall test folds away); DAMP: a damping field (without one, no code for it)
template <typename T, int R, int MODE, bool HOLD = true, bool DAMP = true>
__global__ void __launch_bounds__(A2_THREADS, A2_MIN_BLOCKS) adjoint2d_kernel(const AdjointParams<T> p) {
  using S = Adj2Shape<T, R>;
  static_assert(S::SUPPORTED && MODE != MODE_GRAD, "the 2D quad adjoint: float, radius <= 4");
  constexpr bool GR = MODE == MODE_STEP_GRAD;
  constexpr int H = S::H, XR = S::XR;
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  const int N0 = g.n[0], NF = g.n[1], ext = g.ext[1];
  const int nq = (NF - 2) / 4 + 1;
  const long long k = (long long)blockIdx.x * A2_THREADS + threadIdx.x;
  const int quad = (int)(k % nq), cz = (int)(k / nq);
  const int c0 = 1 + cz * p.chunk, c1 = min(N0 - 1, c0 + p.chunk);
  const int xq = 4 * quad;
  if (c0 < c1 && xq <= NF - 2) {
    T *l0 = level<T>(p.l0, t);
    const T *__restrict__ l1 = level<T>(p.l1, t);
    const T *__restrict__ u1 = GR ? level<T>(p.u1, t) : nullptr;
    const int dir0 = HOLD ? g.dir & 3 : 0, dirF = HOLD ? (g.dir >> 2) & 3 : 0;
    const int s0 = g.s[0];
    const int flags = p.flags;
    const T gg = p.gconst, dg = p.dgconst;
    int inner = 0, xheld = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int x = xq + i;
      if (x < 1 || x > NF - 2)
        continue;
      inner |= 1 << i;
      if (held_wall(x, NF, dirF))
        xheld |= 1 << i;
    }
    const T mi_derived = (flags & K_DERIVE) ? (T)1 / p.sconst : (T)0;
    // a field over the quad at row b through the node image along axis 0
    const auto row4 = [&](const T *f, const int b, T *dst) {
      int sg = 1;
      const int m = (b >= 1 && b <= N0 - 2) ? b : node_image(b, N0, dir0, sg);
      load4(dst, f + (long long)m * s0 + xq);
      if (sg < 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          dst[i] = -dst[i];
      }
    };
    const auto held_row = [&](const int b) {
      return ((dir0 & 1) && b == 1) || ((dir0 & 2) && b == N0 - 2);
    };
    // the queues hold taps: a held wall row reads zero there (its own centre is read
    // again from memory when the march reaches it)
    const auto tap4 = [&](const T *f, const int b, T *dst) {
      row4(f, b, dst);
      if (held_row(b)) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          dst[i] = (T)0;
      }
    };
    // The axis-0 taps are read row by row as the march needs them (the thread read the
    // same rows of its column in the rows before, so they come from L1): lambda rows
    // z-R .. z+R and u rows z-R+1 .. z+R. dmz carries the plain D+ of u at the row before
    // (this row's D-); for the chunk's first row it reads u rows c0 - R .. c0 + R - 1.
    T dmz[4];
    if constexpr (GR) {
      T uc[4], a[4], b[4];
      tap4(u1, c0 - 1, uc);
      tap4(u1, c0, a);
      // (u on a held wall row is zero, so its tap is its centre)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        dmz[i] = p.w[0] * (a[i] - uc[i]);
#pragma unroll
      for (int kk = 2; kk <= R; ++kk) {
        tap4(u1, c0 - 1 + kk, a);
        tap4(u1, c0 - kk, b);
#pragma unroll
        for (int i = 0; i < 4; ++i)
          dmz[i] += p.w[kk - 1] * (a[i] - b[i]);
      }
    }
    // Rows two or more from either wall read their taps as stored: a chunk whose taps
    // all lie there marches without the wall logic (the same values, fewer instructions)
    const bool plain = c0 - R >= 2 && c1 - 1 + R <= N0 - 3;
    const auto march = [&](auto plain_tag) {
      constexpr bool PLAIN = decltype(plain_tag)::value;
      const auto tapz = [&](const T *f, const int b, T *dst) {
        if constexpr (PLAIN)
          load4(dst, f + (long long)b * s0 + xq);
        else
          tap4(f, b, dst);
      };
      const auto rowz = [&](const T *f, const int b, T *dst) {
        if constexpr (PLAIN)
          load4(dst, f + (long long)b * s0 + xq);
        else
          row4(f, b, dst);
      };
      for (int z = c0; z < c1; ++z) {
        const long long row = (long long)z * s0 + xq;
        const bool zheld = held_row(z);
        // the row's point reads first, so their latency passes under the taps' arithmetic
        // (issued later they wait behind the row's taps, and cannot pass the row before's
        // stores)
        T lov[4], miv[4], gm[4], gs4[4];
        load4(lov, l0 + row);
        if (flags & K_DERIVE) {
  #pragma unroll
          for (int i = 0; i < 4; ++i)
            miv[i] = mi_derived;
        } else {
          load4(miv, p.minv + row);
        }
        if constexpr (GR) {
          load4(gm, p.g_mass + row);
          load4(gs4, p.g_stiff + row);
        }
        // the row's own lambda and u, as stored (a held wall row's own value is not the
        // zero its taps read)
        T lcz[4], ucz[4];
        rowz(l1, z, lcz);
        if constexpr (GR)
          rowz(u1, z, ucz);
        // axis 0: the per-node differences of lambda, rows z +- 1 .. z +- R in turn; the
        // first rows on either side kept for the stiffness densities
        T div0[4], lp1[4], lm1[4];
        {
          T lh[4], ll[4];
  #pragma unroll
          for (int i = 0; i < 4; ++i) {
            div0[i] = (T)0;
            lh[i] = ll[i] = lcz[i];
          }
  #pragma unroll
          for (int j = 1; j <= R; ++j) {
            T hi[4], lo[4];
            tapz(l1, z + j, hi);
            tapz(l1, z - j, lo);
            if (j == 1) {
  #pragma unroll
              for (int i = 0; i < 4; ++i) {
                lp1[i] = hi[i];
                lm1[i] = lo[i];
              }
            }
  #pragma unroll
            for (int i = 0; i < 4; ++i) {
              div0[i] += p.w[j - 1] * (gg * (hi[i] - lh[i]) - gg * (ll[i] - lo[i]));
              lh[i] = hi[i];
              ll[i] = lo[i];
            }
          }
        }
        // the plain D+ of u along axis 0 at this row
        T dpz[4];
        if constexpr (GR) {
          T a[4], b[4];
          tapz(u1, z + 1, a);
  #pragma unroll
          for (int i = 0; i < 4; ++i)
            dpz[i] = p.w[0] * (a[i] - ucz[i]);
  #pragma unroll
          for (int kk = 2; kk <= R; ++kk) {
            tapz(u1, z + kk, a);
            tapz(u1, z + 1 - kk, b);
  #pragma unroll
            for (int i = 0; i < 4; ++i)
              dpz[i] += p.w[kk - 1] * (a[i] - b[i]);
          }
        }
        // the axis-1 runs through the node image, zero on a held wall node
        T lr[XR], ur[XR];
        image_run<T, XR, H>(lr, l1 + row, xq, NF, ext, dirF);
        if constexpr (GR)
          image_run<T, XR, H>(ur, u1 + row, xq, NF, ext, dirF);
        // shared along axis 1: g times the first differences of lambda, the plain D+ of u
        T ge[XR];
  #pragma unroll
        for (int c = H - R + 1; c <= H + 3 + R; ++c)
          ge[c] = gg * (lr[c] - lr[c - 1]);
        T dpx[5];
        if constexpr (GR) {
  #pragma unroll
          for (int j = 0; j < 5; ++j) {
            const int c = H - 1 + j;
            T d = p.w[0] * (ur[c + 1] - ur[c]);
  #pragma unroll
            for (int kk = 2; kk <= R; ++kk)
              d += p.w[kk - 1] * (ur[c + kk] - ur[c + 1 - kk]);
            dpx[j] = d;
          }
        }
        T ln[4], uc[4], lc[4];
  #pragma unroll
        for (int i = 0; i < 4; ++i) {
          lc[i] = lcz[i];
          uc[i] = GR ? ucz[i] : (T)0;
          const bool held = zheld || ((xheld >> i) & 1);
          const T lw = held ? (T)0 : lc[i];
          // axis 1: shared differences, or the per-node form on a held wall node
          const int c = H + i;
          T div1 = (T)0;
          if (!((xheld >> i) & 1)) {
  #pragma unroll
            for (int j = 1; j <= R; ++j)
              div1 += p.w[j - 1] * (ge[c + j] - ge[c - j + 1]);
          } else {
            T lh = lc[i], ll = lc[i];
  #pragma unroll
            for (int j = 1; j <= R; ++j) {
              const T lh1 = lr[c + j], ll1 = lr[c - j];
              div1 += p.w[j - 1] * (gg * (lh1 - lh) - gg * (ll - ll1));
              lh = lh1;
              ll = ll1;
            }
          }
          T div_l = (T)0;
          div_l += p.f[0] * div0[i];
          div_l += p.f[1] * div1;
          T gsum = (T)0;
          if constexpr (GR) {
            // the stiffness densities (stiffness_gradient_taps), axis 0 then axis 1
            const T sd0 = p.f[0] * (dg * dpz[i] * (lp1[i] - lw) + dg * dmz[i] * (lw - lm1[i]));
            dmz[i] = dpz[i];
            const T sd1 = p.f[1] * (dg * dpx[i + 1] * (lr[c + 1] - lw) + dg * dpx[i] * (lw - lr[c - 1]));
            gsum += sd0;
            gsum += sd1;
          }
          const T lo = lov[i], mi = miv[i];
          T v;
          if (DAMP && (flags & K_DAMP)) {
            const T dmp = ((inner >> i) & 1) ? p.damping[row + i] : (T)0;
            const T beta = (T)0.5 * mi * dmp * p.dt;
            v = ((T)2 * lc[i] - lo * ((T)1 - beta) + mi * div_l) / ((T)1 + beta);
          } else {
            v = -lo + (T)2 * lc[i] + mi * div_l;
          }
          if (held)
            v = (T)0;
          ln[i] = v;
          if constexpr (GR) {
            gm[i] = gm[i] - p.mf * uc[i] * (v - (T)2 * lc[i] + lo);
            gs4[i] = gs4[i] - p.mf * gsum;
          }
        }
        if (inner == 15) {
          store4(l0 + row, ln);
          if constexpr (GR) {
            store4(p.g_mass + row, gm);
            store4(p.g_stiff + row, gs4);
          }
        } else {
  #pragma unroll
          for (int i = 0; i < 4; ++i)
            if ((inner >> i) & 1) {
              l0[row + i] = ln[i];
              if constexpr (GR) {
                p.g_mass[row + i] = gm[i];
                p.g_stiff[row + i] = gs4[i];
              }
            }
        }
      }
    };
    if (plain)
      march(std::true_type{});
    else
      march(std::false_type{});
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// The nodes the 2D pml transpose reaches: those within R of a lined axis' slab. Rows
// 1 .. za_lo and za_hi .. N0 - 2 (axis 0) are gathered whole; the rows between them over
// columns 1 .. xb_lo and xb_hi .. NF - 2 (axis 1). The host merges ranges that meet.
struct Adj2Reach {
  int za_lo, za_hi;
  int xb_lo, xb_hi;
};

constexpr int A2P_THREADS = 256;

// The pml transpose of the 2D adjoint step, after adjoint2d_kernel has written lambda^n
// (and g_mass): node by node over the reached nodes, each lined axis in turn, the taps of
// the memories' c+ and c- rows around the node summed in stencil order, then the reads
// past the walls that land on it folded back (odd on a Dirichlet face), scaled by 1/m and
// the wall cells' half weights; lambda^n takes the sum, g_mass its share against u^n
// (pml_adjoint_kernel and pml_tap, scalar_sensitivity.cu:545-597, 237-251; the order of
// adjoint_gradient_kernel's update and then pml_adjoint_kernel's, as cuwave launches
// them).
// `ld`: the adjoint load that follows the step, when none of its nodes is reached (its
// num 0 otherwise): threads past the reached nodes apply it, as load_kernel would after
template <typename T, int R, int MODE>
__global__ void __launch_bounds__(A2P_THREADS) adjoint2d_pml_kernel(const AdjointParams<T> p,
                                                                    const Adj2Reach reach,
                                                                    const TransferParams<T> ld,
                                                                    T *ld_mass) {
  constexpr bool GR = MODE == MODE_STEP_GRAD;
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  const int N0 = g.n[0], NF = g.n[1], ext = g.ext[1];
  const int nzlo = reach.za_lo, nzhi = N0 - 1 - reach.za_hi;
  const long long nA = (long long)(nzlo + nzhi) * (NF - 2);
  const int nxlo = reach.xb_lo, nxhi = NF - 1 - reach.xb_hi, nx = nxlo + nxhi;
  const long long nB = (long long)(reach.za_hi - 1 - reach.za_lo) * nx;
  const long long k = (long long)blockIdx.x * A2P_THREADS + threadIdx.x;
  int z = -1, x = -1;
  if (k < nA) {
    const int r = (int)(k / (NF - 2));
    z = r < nzlo ? 1 + r : reach.za_hi + (r - nzlo);
    x = 1 + (int)(k % (NF - 2));
  } else if (k - nA < nB) {
    const long long kb = k - nA;
    z = reach.za_lo + 1 + (int)(kb / nx);
    const int c = (int)(kb % nx);
    x = c < nxlo ? 1 + c : reach.xb_hi + (c - nxlo);
  }
  if (z >= 0) {
    T *l0 = level<T>(p.l0, t);
    const long long row = (long long)z * g.s[0] + x;
    const T mi = (p.flags & K_DERIVE) ? (T)1 / p.sconst : p.minv[row];
    const int A[2] = {z, x};
    T wcell = (T)1;
#pragma unroll
    for (int e = 0; e < 2; ++e)
      if (A[e] == 1 || A[e] == g.n[e] - 2)
        wcell *= (T)0.5;
    T ln = l0[row];
    T gm = GR ? p.g_mass[row] : (T)0;
    const T uc = GR ? level<T>(p.u1, t)[row] : (T)0;
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const int lo_d = g.lo[d], hi_d = g.hi[d];
      if (!(lo_d + hi_d))
        continue;
      const int a = A[d], N = g.n[d];
      const bool reached = (lo_d && a >= 1 && a <= lo_d + R) ||
                           (hi_d && a <= N - 2 && a >= N - 1 - (hi_d + R));
      if (!reached)
        continue;
      const T *mem = p.mem[d];
      const long long sz = p.memrow[d];
      const int rows = lo_d + hi_d;
      const auto tap = [&](const int ai, const int q) -> T {
        const int r = slab_row(ai, N, lo_d, hi_d);
        const long long si = d == 0 ? (long long)r * ext + A[1] : (long long)A[0] * rows + r;
        return mem[3 * sz + si] * plus_tap<T, R>(p.w, q) + mem[4 * sz + si] * minus_tap<T, R>(p.w, q);
      };
      T sum = (T)0;
#pragma unroll
      for (int m = -R; m <= R; ++m)
        if (slab_row(a + m, N, lo_d, hi_d) >= 0)
          sum += tap(a + m, -m);
#pragma unroll
      for (int high = 0; high < 2; ++high) {
        // the reads past the wall that land on a, folded back, odd on a Dirichlet face;
        // none reaches a node more than R + 1 from the wall (skipping its zero fold
        // leaves the sum's bits as they are: it starts at +0 and cannot turn -0)
        if (high ? a < N - 2 - R : a > R + 1)
          continue;
        const int ghost = high ? 2 * (N - 2) - a : 2 - a;
        if (high ? ghost < N - 1 : ghost > 0)
          continue;
        T fold = (T)0;
#pragma unroll
        for (int kk = 1; kk <= R; ++kk) {
          const int ai = high ? N - 1 - kk : kk;
          if (slab_row(ai, N, lo_d, hi_d) >= 0 && ghost - ai >= -R && ghost - ai <= R)
            fold += tap(ai, ghost - ai);
        }
        sum += ((g.dir >> (2 * d + high)) & 1) ? -fold : fold;
      }
      const T delta = mi * sum / wcell;
      ln += delta;
      if constexpr (GR)
        gm -= p.mf * uc * delta;
    }
    l0[row] = ln;
    if constexpr (GR)
      p.g_mass[row] = gm;
  } else if (k >= nA + nB && k < nA + nB + ld.num) {
    // a receiver's load (load_kernel's adds): no reached node, so no thread above
    // writes its lambda or g_mass
    const int j = (int)(k - nA - nB);
    T *a = level<T>(ld.a, t);
    const long long srow = (long long)ld.row_mul * t + ld.row_add;
    const int n = ld.lin[j];
    const T load = ld.weight[j] * record_read(ld, srow * ld.num + j);
    atomic_add_exact(&a[n], load);
    if (ld.flags & K_MASS)
      atomic_add_exact(&ld_mass[n], -ld.scale * level<T>(ld.c, t)[n] * load);
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

}  // namespace cwb
