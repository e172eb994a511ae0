// The transposed step and the gradient densities, marched along axis 0 like the step.
//
// MODE_STEP       lambda^n = 2 lambda^(n+1) - lambda^(n+2) + dt^2/m (W^-1 A^T W lambda^(n+1)),
//                 the pml transpose gathered in: adjoint_kernel + pml_adjoint_kernel
//                 (cuwave/kernels/scalar_sensitivity.cu:388-441, 545-597).
// MODE_STEP_GRAD  the same, accumulating g_mass and g_stiff against u^n:
//                 adjoint_gradient_kernel (scalar_sensitivity.cu:444-515).
// MODE_GRAD       both densities of a forward triplet against lambda:
//                 gradient_kernel (scalar_sensitivity.cu:303-350).
//
// The adjoint reads lambda, u and k through the node image, never a stored ghost,
// lambda and u odd across a Dirichlet face and zero on its wall node
// (`reflected`, scalar_sensitivity.cu:177-184); the queues and tiles hold the image
// values and a tap landing on a held wall node is zeroed where it is read. The
// transposed divergence is transposed_divergence_taps (scalar_sensitivity.cu:140-154)
// and the stiffness density stiffness_gradient_taps (scalar_sensitivity.cu:119-135),
// in their order of operations.
#pragma once

#include <type_traits>

#include "params.cuh"

namespace cwb {

template <int NDIM, int R, int BX, int BY>
struct AdjShape {
  static constexpr int HY = NDIM == 3 ? R : 0;
  static constexpr int TW = BX + 2 * R;
  static constexpr int TH = BY + 2 * HY;
  static constexpr int PLANE = TW * TH;
};

// fields an adjoint mode reads with taps: lambda always, u with gradients, k unless
// uniform
template <int MODE, bool UNIF>
struct AdjFields {
  static constexpr bool U = MODE != MODE_STEP;
  static constexpr bool K = !UNIF;
  static constexpr int COUNT = 1 + (U ? 1 : 0) + (K ? 1 : 0);
};

// PML: the pml transpose gathered here where the flags ask (else a launch of its own, or
// none, and no code for it)
template <typename T, int NDIM, int R, bool UNIF, int MODE, int BX, int BY, bool PML = true>
// (three blocks of 256 an SM for a uniform stiffness in 3D up to radius 4: its registers
// fit, and the march waits on loads more warps hide)
__global__ void __launch_bounds__(BX *BY, NDIM == 3 && UNIF && R <= 4 ? 3 : 1) adjoint_kernel(const AdjointParams<T> p) {
  using S = AdjShape<NDIM, R, BX, BY>;
  using FL = AdjFields<MODE, UNIF>;
  constexpr int HY = S::HY, TW = S::TW, F = NDIM - 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *tiles = reinterpret_cast<T *>(smem_raw);

  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  // MODE_STEP*: l0 = lambda^(n+2) -> lambda^n, l1 = lambda^(n+1), u1 = u^n
  // MODE_GRAD:  u0, u1, u2 the forward triplet, l1 = lambda
  T *l0 = MODE == MODE_GRAD ? nullptr : level<T>(p.l0, t);
  const T *__restrict__ l1 = level<T>(p.l1, t);
  const T *__restrict__ u1 = FL::U ? level<T>(p.u1, t) : nullptr;
  const T *__restrict__ u0 = MODE == MODE_GRAD ? level<T>(p.u0, t) : nullptr;
  const T *__restrict__ u2 = MODE == MODE_GRAD ? level<T>(p.u2, t) : nullptr;
  const T *__restrict__ stiff = p.stiff;

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x0 = blockIdx.x * BX;
  const int y0 = NDIM == 3 ? blockIdx.y * BY : 0;
  const int cz = NDIM == 3 ? blockIdx.z : blockIdx.y;
  const int N0 = g.n[0], NF = g.n[F], NM = NDIM == 3 ? g.n[1] : 1;
  const int s0 = g.s[0], sM = NDIM == 3 ? g.s[1] : 0;
  const int px = x0 + tx, py = y0 + ty;
  const int c0 = 1 + cz * p.chunk;
  const int c1 = min(N0 - 1, c0 + p.chunk);
  // only an interior column keeps queues: a ghost column's cell holds its image
  const bool inner = px >= 1 && px <= NF - 2 && (NDIM == 2 || (py >= 1 && py <= NM - 2));
  const bool own = inner;
  const int col = (NDIM == 3 ? py * sM : 0) + px;
  const int dir0 = g.dir & 3;
  const int dirM = NDIM == 3 ? (g.dir >> 2) & 3 : 0;
  const int dirF = (g.dir >> (2 * F)) & 3;
  const int flags = p.flags;

  // field at row b of this column through the node image along axis 0
  const auto row_val = [&](const T *f, const int b, const bool odd) -> T {
    int sg;
    const int m = node_image(b, N0, odd ? dir0 : 0, sg);
    const T v = f[m * s0 + col];
    return sg < 0 ? -v : v;
  };
  // field at in-plane node (bm, bf) of plane a0 through its images; out of reach zero
  const auto plane_val = [&](const T *f, const int a0, const int bm, const int bf,
                             const bool odd) -> T {
    int sf, sm = 1, mm = 0;
    const int mf = node_image(bf, NF, odd ? dirF : 0, sf);
    if (NDIM == 3)
      mm = node_image(bm, NM, odd ? dirM : 0, sm);
    if (mf < 0 || mf > NF - 1 || mm < 0 || mm > NM - 1)
      return (T)0;
    const T v = f[a0 * s0 + mm * sM + mf];
    return sf * sm < 0 ? -v : v;
  };

  // queues along axis 0: lambda, u, k on rows a0 - R .. a0 + R
  T ql[2 * R + 1], qu[2 * R + 1], qk[2 * R + 1];
  if (own && c0 < c1) {
#pragma unroll
    for (int k = 0; k < 2 * R; ++k) {
      ql[k] = row_val(l1, c0 - R + k, true);
      if constexpr (FL::U)
        qu[k] = row_val(u1, c0 - R + k, true);
      if constexpr (FL::K)
        qk[k] = row_val(stiff, c0 - R + k, false);
    }
  }

  // the loads of a plane, issued one plane ahead so that they arrive during the plane
  // before's arithmetic: the queues' feed (plane a + R) and the tile's halo at plane a
  // (a thread holds at most one halo node per side along each in-plane axis: R <= BX, BY)
  static_assert(R <= BX && (NDIM == 2 || R <= BY), "one halo node a side per thread");
  const bool xh = tx < R, yh = NDIM == 3 && ty < R;
  T nq[3] = {(T)0, (T)0, (T)0}, nx[3][2], ny[3][2];
  // the node's own lambda^(n+2), 1/m and gradient densities at plane a (the transposed
  // update's point reads), fetched with the rest
  T nn[4] = {(T)0, (T)0, (T)0, (T)0};
  const auto fetch = [&](const int a) {
    if constexpr (MODE != MODE_GRAD) {
      if (inner) {
        const long long i2 = (long long)a * s0 + col;
        nn[0] = l0[i2];
        if (!(p.flags & K_DERIVE))
          nn[1] = p.minv[i2];
        if constexpr (MODE == MODE_STEP_GRAD) {
          nn[2] = p.g_mass[i2];
          nn[3] = p.g_stiff[i2];
        }
      }
    }
    if (own) {
      nq[0] = row_val(l1, a + R, true);
      if constexpr (FL::U)
        nq[1] = row_val(u1, a + R, true);
      if constexpr (FL::K)
        nq[2] = row_val(stiff, a + R, false);
    }
    if (xh) {
      nx[0][0] = plane_val(l1, a, py, x0 - R + tx, true);
      nx[0][1] = plane_val(l1, a, py, x0 + BX + tx, true);
      if constexpr (FL::U) {
        nx[1][0] = plane_val(u1, a, py, x0 - R + tx, true);
        nx[1][1] = plane_val(u1, a, py, x0 + BX + tx, true);
      }
      if constexpr (FL::K) {
        nx[2][0] = plane_val(stiff, a, py, x0 - R + tx, false);
        nx[2][1] = plane_val(stiff, a, py, x0 + BX + tx, false);
      }
    }
    if (yh) {
      ny[0][0] = plane_val(l1, a, y0 - R + ty, px, true);
      ny[0][1] = plane_val(l1, a, y0 + BY + ty, px, true);
      if constexpr (FL::U) {
        ny[1][0] = plane_val(u1, a, y0 - R + ty, px, true);
        ny[1][1] = plane_val(u1, a, y0 + BY + ty, px, true);
      }
      if constexpr (FL::K) {
        ny[2][0] = plane_val(stiff, a, y0 - R + ty, px, false);
        ny[2][1] = plane_val(stiff, a, y0 + BY + ty, px, false);
      }
    }
  };
  if (c0 < c1)
    fetch(c0);

  for (int a0 = c0; a0 < c1; ++a0) {
    T *tL = tiles + ((a0 - c0) & 1) * FL::COUNT * S::PLANE;
    T *tU = tL + S::PLANE;
    T *tK = tL + (FL::U ? 2 : 1) * S::PLANE;
    if (own) {
      ql[2 * R] = nq[0];
      if constexpr (FL::U)
        qu[2 * R] = nq[1];
      if constexpr (FL::K)
        qk[2 * R] = nq[2];
    }
    const int cc = (ty + HY) * TW + tx + R;
    if (xh) {
      const int cl = (ty + HY) * TW + tx, cr = (ty + HY) * TW + BX + R + tx;
      tL[cl] = nx[0][0];
      tL[cr] = nx[0][1];
      if constexpr (FL::U) {
        tU[cl] = nx[1][0];
        tU[cr] = nx[1][1];
      }
      if constexpr (FL::K) {
        tK[cl] = nx[2][0];
        tK[cr] = nx[2][1];
      }
    }
    if (yh) {
      const int ct = ty * TW + tx + R, cb = (BY + HY + ty) * TW + tx + R;
      tL[ct] = ny[0][0];
      tL[cb] = ny[0][1];
      if constexpr (FL::U) {
        tU[ct] = ny[1][0];
        tU[cb] = ny[1][1];
      }
      if constexpr (FL::K) {
        tK[ct] = ny[2][0];
        tK[cb] = ny[2][1];
      }
    }
    const T cur_lo = nn[0], cur_mi = nn[1], cur_gm = nn[2], cur_gs = nn[3];
    if (a0 + 1 < c1)
      fetch(a0 + 1);
    tL[cc] = own ? ql[R] : plane_val(l1, a0, py, px, true);
    if constexpr (FL::U)
      tU[cc] = own ? qu[R] : plane_val(u1, a0, py, px, true);
    if constexpr (FL::K)
      tK[cc] = own ? qk[R] : plane_val(stiff, a0, py, px, false);
    __syncthreads();

    if (inner) {
      const int idx = a0 * s0 + col;
      const int A[3] = {a0, NDIM == 3 ? py : px, px};
      const int dirs[3] = {dir0, NDIM == 3 ? dirM : dirF, dirF};
      const bool held = held_wall(a0, N0, dir0) || (NDIM == 3 && held_wall(py, NM, dirM)) ||
                        held_wall(px, NF, dirF);
      // whether a tap of this node can land on a held wall node
      bool near = false;
#pragma unroll
      for (int d = 0; d < NDIM; ++d)
        near |= ((dirs[d] & 1) && A[d] <= R + 1) || ((dirs[d] & 2) && A[d] >= g.n[d] - 2 - R);
      const T sc = UNIF ? p.sconst : qk[R];
      const T uc = FL::U ? qu[R] : (T)0;
      const T lc = ql[R];
      const T lw = held ? (T)0 : lc;

      const auto body = [&](auto check) {
        constexpr bool CHK = decltype(check)::value;
        // the taps of axis d; lambda and u read zero on a held wall node
        const auto tapL = [&](const int d, const int j) -> T {
          T v = d == 0 ? ql[R + j] : (d == F ? tL[cc + j] : tL[cc + j * TW]);
          if (CHK) {
            const int b = A[d] + j;
            if (((dirs[d] & 1) && b == 1) || ((dirs[d] & 2) && b == g.n[d] - 2))
              v = (T)0;
          }
          return v;
        };
        const auto tapU = [&](const int d, const int j) -> T {
          T v = d == 0 ? qu[R + j] : (d == F ? tU[cc + j] : tU[cc + j * TW]);
          if (CHK) {
            const int b = A[d] + j;
            if (((dirs[d] & 1) && b == 1) || ((dirs[d] & 2) && b == g.n[d] - 2))
              v = (T)0;
          }
          return v;
        };
        const auto tapK = [&](const int d, const int j) -> T {
          if (UNIF)
            return p.sconst;
          return d == 0 ? qk[R + j] : (d == F ? tK[cc + j] : tK[cc + j * TW]);
        };
        // the stiffness density of one axis, its outer minus left to the caller
        const auto stiff_density = [&](const int d) -> T {
          T dgp, dgm;
          if (UNIF) {
            dgp = p.dgconst;
            dgm = p.dgconst;
          } else {
            const T sp = tapK(d, 1), sm = tapK(d, -1);
            dgp = sp * sp / ((sc + sp) * (sc + sp));
            dgm = sm * sm / ((sc + sm) * (sc + sm));
          }
          T Dp = p.w[0] * (tapU(d, 1) - uc);
          T Dm = p.w[0] * (uc - tapU(d, -1));
#pragma unroll
          for (int j = 2; j <= R; ++j) {
            Dp += p.w[j - 1] * (tapU(d, j) - tapU(d, 1 - j));
            Dm += p.w[j - 1] * (tapU(d, j - 1) - tapU(d, -j));
          }
          return p.f[d] * (dgp * Dp * (tapL(d, 1) - lw) + dgm * Dm * (lw - tapL(d, -1)));
        };

        if constexpr (MODE == MODE_GRAD) {
          // dJ/dmass of the triplet, then dJ/dstiff (gradient_kernel)
          p.g_mass[idx] -= p.mf * lc * (u2[idx] - (T)2 * uc + u0[idx]);
          T gs = (T)0;
#pragma unroll
          for (int d = 0; d < NDIM; ++d)
            gs += stiff_density(d);
          p.g_stiff[idx] -= gs;
        } else {
          const T lo = cur_lo;
          const T mi = (flags & K_DERIVE) ? (T)1 / sc : cur_mi;
          T div_l = (T)0, gs = (T)0;
#pragma unroll
          for (int d = 0; d < NDIM; ++d) {
            T div = (T)0, sh = sc, sl = sc, lh = lc, ll = lc;
#pragma unroll
            for (int j = 1; j <= R; ++j) {
              const T sh1 = tapK(d, j), sl1 = tapK(d, -j);
              const T lh1 = tapL(d, j), ll1 = tapL(d, -j);
              T ghi, glo;
              if (UNIF) {
                ghi = p.gconst;
                glo = p.gconst;
              } else {
                ghi = sh * sh1 / (sh + sh1);
                glo = sl * sl1 / (sl + sl1);
              }
              div += p.w[j - 1] * (ghi * (lh1 - lh) - glo * (ll - ll1));
              sh = sh1;
              sl = sl1;
              lh = lh1;
              ll = ll1;
            }
            div_l += p.f[d] * div;
            if constexpr (MODE == MODE_STEP_GRAD)
              gs += stiff_density(d);
          }
          T ln;
          if (flags & K_DAMP) {
            const T beta = (T)0.5 * mi * p.damping[idx] * p.dt;
            ln = ((T)2 * lc - lo * ((T)1 - beta) + mi * div_l) / ((T)1 + beta);
          } else {
            ln = -lo + (T)2 * lc + mi * div_l;
          }
          if (held)
            ln = (T)0;
          T gmass = (T)0, gstiff = (T)0;
          if constexpr (MODE == MODE_STEP_GRAD) {
            gmass = cur_gm - p.mf * uc * (ln - (T)2 * lc + lo);
            gstiff = cur_gs - p.mf * gs;
          }

          if (PML && (flags & K_PML)) {
            const T wcell = cell_weight<T>(g, A);
#pragma unroll 1
            for (int d = 0; d < NDIM; ++d) {
              const int lo_d = g.lo[d], hi_d = g.hi[d];
              if (!(lo_d + hi_d))
                continue;
              const int a = A[d], N = g.n[d];
              const bool reached = (lo_d && a >= 1 && a <= lo_d + R) ||
                                   (hi_d && a <= N - 2 && a >= N - 1 - (hi_d + R));
              if (!reached)
                continue;
              const T *mem = p.mem[d];
              const int sz = p.memrow[d];
              int B[3] = {A[0], A[1], A[2]};
              // what the memories of layer row ai give the node q rows off it
              // (pml_tap, scalar_sensitivity.cu:237-251, its c+ and c- precomputed)
              const auto tap = [&](const int ai, const int q) -> T {
                const int r = slab_row(ai, N, lo_d, hi_d);
                B[d] = ai;
                const int i = slab_index(g, d, r, B);
                return mem[3 * sz + i] * plus_tap<T, R>(p.w, q) +
                       mem[4 * sz + i] * minus_tap<T, R>(p.w, q);
              };
              T sum = (T)0;
#pragma unroll 1
              for (int m = -R; m <= R; ++m)
                if (slab_row(a + m, N, lo_d, hi_d) >= 0)
                  sum += tap(a + m, -m);
#pragma unroll 1
              for (int high = 0; high < 2; ++high) {
                // the reads past the wall that land on a, folded back, odd on a
                // Dirichlet face
                const int ghost = high ? 2 * (N - 2) - a : 2 - a;
                if (high ? ghost < N - 1 : ghost > 0)
                  continue;
                T fold = (T)0;
#pragma unroll 1
                for (int k = 1; k <= R; ++k) {
                  const int ai = high ? N - 1 - k : k;
                  if (slab_row(ai, N, lo_d, hi_d) >= 0 && ghost - ai >= -R && ghost - ai <= R)
                    fold += tap(ai, ghost - ai);
                }
                sum += ((g.dir >> (2 * d + high)) & 1) ? -fold : fold;
              }
              const T delta = mi * sum / wcell;
              ln += delta;
              if constexpr (MODE == MODE_STEP_GRAD)
                gmass -= p.mf * uc * delta;
            }
          }
          l0[idx] = ln;
          if constexpr (MODE == MODE_STEP_GRAD) {
            p.g_mass[idx] = gmass;
            p.g_stiff[idx] = gstiff;
          }
        }
      };
      if (near)
        body(std::true_type{});
      else
        body(std::false_type{});
    }
#pragma unroll
    for (int k = 0; k < 2 * R; ++k) {
      ql[k] = ql[k + 1];
      if constexpr (FL::U)
        qu[k] = qu[k + 1];
      if constexpr (FL::K)
        qk[k] = qk[k + 1];
    }
  }
  finish_step(p.ctr, flags & K_ADV);
}

// The nodes the 3D pml transpose reaches: those within R of a lined axis' slab, as three
// disjoint regions -- the planes axis 0's slabs reach, whole; in the planes between, the
// rows axis 1's reach, whole; in the rest, the columns axis 2's reach. `lo[d]` is the last
// reached index near the low wall (0: none) and `hi[d]` the first near the high one
// (n[d] - 1: none); the host merges ranges that meet.
struct Adj3Reach {
  int lo[3], hi[3];
};

constexpr int A3P_THREADS = 256;

// The pml transpose of the 3D adjoint step, after the march has written lambda^n (and
// g_mass) without it: node by node over the reached nodes, each lined axis in turn, the
// taps of the memories' c+ and c- rows around the node summed in stencil order, then
// the reads past the walls that land on it folded back (odd on a Dirichlet face), scaled
// by 1/m and the wall cells' half weights; lambda^n takes the sum, g_mass its share
// against u^n (pml_adjoint_kernel and pml_tap, scalar_sensitivity.cu:545-597, 237-251,
// after adjoint_gradient_kernel's update, in the order cuwave launches them). The same
// gather, in the same order, as the one adjoint_kernel runs inline.
template <typename T, int R, bool UNIF, int MODE>
__global__ void __launch_bounds__(A3P_THREADS) adjoint3d_pml_kernel(const AdjointParams<T> p,
                                                                    const Adj3Reach reach) {
  constexpr bool GR = MODE == MODE_STEP_GRAD;
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  const int n0 = g.n[0] - 2, n1 = g.n[1] - 2, n2 = g.n[2] - 2;  // interior extents
  // reached and unreached counts along each axis
  int rc[3], uc_[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    rc[d] = reach.lo[d] + (g.n[d] - 1 - reach.hi[d]);
    uc_[d] = g.n[d] - 2 - rc[d];
  }
  const long long nA = (long long)rc[0] * n1 * n2;
  const long long nB = (long long)uc_[0] * rc[1] * n2;
  const long long nC = (long long)uc_[0] * uc_[1] * rc[2];
  long long k = (long long)blockIdx.x * A3P_THREADS + threadIdx.x;
  // index j of a reached (or unreached) coordinate along axis d
  const auto reached_at = [&](const int d, const int j) {
    return j < reach.lo[d] ? 1 + j : reach.hi[d] + (j - reach.lo[d]);
  };
  const auto unreached_at = [&](const int d, const int j) { return reach.lo[d] + 1 + j; };
  int A[3] = {-1, -1, -1};
  if (k < nA) {
    A[2] = 1 + (int)(k % n2);
    k /= n2;
    A[1] = 1 + (int)(k % n1);
    A[0] = reached_at(0, (int)(k / n1));
  } else if ((k -= nA) < nB) {
    A[2] = 1 + (int)(k % n2);
    k /= n2;
    A[1] = reached_at(1, (int)(k % rc[1]));
    A[0] = unreached_at(0, (int)(k / rc[1]));
  } else if ((k -= nB) < nC) {
    A[2] = reached_at(2, (int)(k % rc[2]));
    k /= rc[2];
    A[1] = unreached_at(1, (int)(k % uc_[1]));
    A[0] = unreached_at(0, (int)(k / uc_[1]));
  }
  if (A[0] >= 0) {
    T *l0 = level<T>(p.l0, t);
    const long long idx = (long long)A[0] * g.s[0] + (long long)A[1] * g.s[1] + A[2];
    T mi;
    if (p.flags & K_DERIVE)
      mi = (T)1 / (UNIF ? p.sconst : p.stiff[idx]);
    else
      mi = p.minv[idx];
    T wcell = (T)1;  // the cell weight: a half per axis on whose wall the node sits
#pragma unroll
    for (int e = 0; e < 3; ++e)
      if (A[e] == 1 || A[e] == g.n[e] - 2)
        wcell *= (T)0.5;
    T ln = l0[idx];
    T gm = GR ? p.g_mass[idx] : (T)0;
    const T uc = GR ? level<T>(p.u1, t)[idx] : (T)0;
    // the axes in order, every loop unrolled: a tap's memory index is base + r * rs for
    // its slab row r (the grid with axis d replaced by its slab rows)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int lo_d = g.lo[d], hi_d = g.hi[d];
      if (!(lo_d + hi_d))
        continue;
      const int a = A[d], N = g.n[d];
      const bool reached = (lo_d && a >= 1 && a <= lo_d + R) ||
                           (hi_d && a <= N - 2 && a >= N - 1 - (hi_d + R));
      if (!reached)
        continue;
      const T *mem = p.mem[d];
      const int sz = p.memrow[d];
      const int rows = lo_d + hi_d;
      const int e1 = g.ext[1], e2 = g.ext[2];
      const int base = d == 0 ? A[1] * e2 + A[2]
                     : d == 1 ? A[0] * rows * e2 + A[2]
                              : (A[0] * e1 + A[1]) * rows;
      const int rs = d == 0 ? e1 * e2 : d == 1 ? e2 : 1;
      const auto tap = [&](const int ai, const int q) -> T {
        const int i = base + slab_row(ai, N, lo_d, hi_d) * rs;
        return mem[3 * sz + i] * plus_tap<T, R>(p.w, q) +
               mem[4 * sz + i] * minus_tap<T, R>(p.w, q);
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
      if (GR)
        gm -= p.mf * uc * delta;
    }
    l0[idx] = ln;
    if (GR)
      p.g_mass[idx] = gm;
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

}  // namespace cwb
