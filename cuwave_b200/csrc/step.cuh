// The forward leapfrog step: fd update, pml memory, folded sources and refill.
//
// A block owns a tile of the plane orthogonal to axis 0 (BX fast-axis nodes by BY
// axis-1 nodes in 3D, BX nodes in 2D) and marches `chunk` planes along axis 0. Each
// thread keeps its column's 2R + 1 values of u^(t-1) along axis 0 in a register queue,
// so every value of the field is read from DRAM once per step; the in-plane taps come
// from the current plane staged in shared memory with an R-wide halo (double
// buffered, one barrier a plane).
//
// Per node the arithmetic is cuwave's fd_kernel (cuwave/kernels/scalar.cu:347-496):
// the pinned cell differences of flux_divergence_taps (scalar.cu:15-32) with the
// harmonic cell stiffness of flux_divergence_axis (scalar.cu:43-65), the axes summed
// in the same fused order, and the (damped) update. The pml terms of pml_kernel
// (scalar.cu:500-532) are added in axis order from the same taps, re-forming the cell
// differences unfused as cell_differences (scalar.cu:69-83) does; the folded sources
// add `weight * signal` as excitation_kernel (cuwave/kernels/common.cuh:456-464), and
// the folded refill writes a face ghost from its mirror as the refill kernels
// (scalar.cu:535-555) do after the excitation.
#pragma once

#include "params.cuh"

namespace cwb {

// D+ and D- of one axis rounded as flux_divergence_taps pins them
template <typename T, int R, class Tap>
__device__ __forceinline__ void diffs_pinned(const Tap &u, const T uc, const T *w, T &Dp,
                                             T &Dm) {
  Dp = u(1) - uc;
  Dm = uc - u(-1);
  if (R > 1) {
    Dp = mul_rn(w[0], Dp);
    Dm = mul_rn(w[0], Dm);
  }
#pragma unroll
  for (int k = 2; k <= R; ++k) {
    Dp = fma_rn(w[k - 1], u(k) - u(1 - k), Dp);
    Dm = fma_rn(w[k - 1], u(k - 1) - u(-k), Dm);
  }
}

// D+ of a node with the fused products of the pinned form (diffs_pinned's D+)
template <typename T, int R, class Tap>
__device__ __forceinline__ T dplus(const Tap &u, const T uc, const T *w) {
  T d = u(1) - uc;
  if (R > 1)
    d = mul_rn(w[0], d);
#pragma unroll
  for (int k = 2; k <= R; ++k)
    d = fma_rn(w[k - 1], u(k) - u(1 - k), d);
  return d;
}

// D+ and D- with products and sums rounded apart, as cell_differences forms them
template <typename T, int R, class Tap>
__device__ __forceinline__ void diffs_plain(const Tap &u, const T uc, const T *w, T &Dp,
                                            T &Dm) {
  Dp = w[0] * (u(1) - uc);
  Dm = w[0] * (uc - u(-1));
#pragma unroll
  for (int k = 2; k <= R; ++k) {
    Dp += w[k - 1] * (u(k) - u(1 - k));
    Dm += w[k - 1] * (u(k - 1) - u(-k));
  }
}

// One axis of a masked node's operator: each cell at its own radius from the table
// rows, a closed cell carrying no flux and a held one a flux onto a zero at its
// midpoint, taps read as stored (flux_divergence_cells, cuwave/kernels/scalar.cu:86-118).
template <typename T, int R, bool UNIF>
__device__ __forceinline__ T cell_axis(const StepParams<T> &p, const T *__restrict__ u1,
                                       const long long idx, const long long s, const T uc,
                                       const T sc, const T f, const int rp, const int rm) {
  T Dp = (T)0, Dm = (T)0;
  if (rp == CELL_HELD) {
    Dp = -uc * sc;
  } else if (rp) {
    const T sp = UNIF ? p.sconst : p.stiff[idx + s];
    const T *w = p.ctab + (rp - 1) * R;
    Dp = w[0] * (u1[idx + s] - uc);
#pragma unroll
    for (int k = 2; k <= R; ++k)
      if (k <= rp)
        Dp += w[k - 1] * (u1[idx + k * s] - u1[idx - (k - 1) * s]);
    Dp *= sc * sp / (sc + sp);
  }
  if (rm == CELL_HELD) {
    Dm = uc * sc;
  } else if (rm) {
    const T sm = UNIF ? p.sconst : p.stiff[idx - s];
    const T *w = p.ctab + (rm - 1) * R;
    Dm = w[0] * (uc - u1[idx - s]);
#pragma unroll
    for (int k = 2; k <= R; ++k)
      if (k <= rm)
        Dm += w[k - 1] * (u1[idx + (k - 1) * s] - u1[idx - k * s]);
    Dm *= sc * sm / (sc + sm);
  }
  return f * (Dp - Dm);
}

template <int NDIM, int R, int BX, int BY>
struct StepShape {
  static constexpr int HY = NDIM == 3 ? R : 0;
  static constexpr int TW = BX + 2 * R;
  static constexpr int TH = BY + 2 * HY;
  static constexpr int PLANE = TW * TH;
};

// One block's tile of step t: the tile (bx, by) of the plane, chunk bz along axis 0 (in
// 2D: bx, chunk by), of a grid of nbx x nby tiles; `tiles` the block's shared memory.
template <typename T, int NDIM, int R, bool UNIF, int BX, int BY>
__device__ __forceinline__ void step_block(const StepParams<T> &p, const int t, const int bx,
                                           const int by, const int bz, const int nbx,
                                           const int nby, T *tiles) {
  using S = StepShape<NDIM, R, BX, BY>;
  constexpr int HY = S::HY, TW = S::TW, F = NDIM - 1;

  const Geometry &g = p.g;
  const T *u0 = level<T>(p.u0, t);
  const T *__restrict__ u1 = level<T>(p.u1, t);
  T *u2 = level<T>(p.u2, t);

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x0 = bx * BX;
  const int y0 = NDIM == 3 ? by * BY : 0;
  const int cz = NDIM == 3 ? bz : by;
  const int N0 = g.n[0], NF = g.n[F], NM = NDIM == 3 ? g.n[1] : 1;
  const int s0 = g.s[0], sM = NDIM == 3 ? g.s[1] : 0;
  const int px = x0 + tx, py = y0 + ty;
  const int c0 = 1 + cz * p.chunk;
  const int c1 = min(N0 - 1, c0 + p.chunk);
  const bool own = px <= NF - 1 && (NDIM == 2 || py <= NM - 1);
  const bool inner = px >= 1 && px <= NF - 2 && (NDIM == 2 || (py >= 1 && py <= NM - 2));
  const int col = (NDIM == 3 ? py * sM : 0) + px;
  const int dir0 = g.dir & 3;
  const int dirM = NDIM == 3 ? (g.dir >> 2) & 3 : 0;
  const int dirF = (g.dir >> (2 * F)) & 3;
  const int flags = p.flags;

  // u^(t-1) at row b of this column, past a wall off its mirror
  const auto row_val = [&](const int b) -> T {
    int sg;
    const int m = mirror_node(b, N0, dir0, sg);
    const T v = u1[m * s0 + col];
    return sg < 0 ? -v : v;
  };
  // u^(t-1) at in-plane node (bm, bf) of plane a0, past a wall off its mirror; a node
  // no interior tap reaches is left zero
  const auto plane_val = [&](const int a0, const int bm, const int bf) -> T {
    int sf, sm = 1, mm = 0;
    const int mf = mirror_node(bf, NF, dirF, sf);
    if (NDIM == 3)
      mm = mirror_node(bm, NM, dirM, sm);
    if (mf < 0 || mf > NF - 1 || mm < 0 || mm > NM - 1)
      return (T)0;
    const T v = u1[a0 * s0 + mm * sM + mf];
    return sf * sm < 0 ? -v : v;
  };

  T q[2 * R + 1];  // u^(t-1) on rows a0 - R .. a0 + R of this column
  if (own && c0 < c1) {
#pragma unroll
    for (int k = 0; k < 2 * R; ++k)
      q[k] = row_val(c0 - R + k);
  }

  int sfirst = 0, slast = 0, srow = 0;
  const int lane = ty * BX + tx;
  if (flags & K_SRC) {
    const int blk = bx + nbx * (by + nby * bz);
    sfirst = p.src_start[blk];
    slast = p.src_start[blk + 1];
    srow = p.sig_mul * t + p.sig_add;
  }

  for (int a0 = c0; a0 < c1; ++a0) {
    T *tl = tiles + ((a0 - c0) & 1) * S::PLANE;
    if (own)
      q[2 * R] = row_val(a0 + R);
    tl[(ty + HY) * TW + tx + R] = own ? q[R] : plane_val(a0, py, px);
    for (int e = tx; e < R; e += BX) {
      tl[(ty + HY) * TW + e] = plane_val(a0, py, x0 - R + e);
      tl[(ty + HY) * TW + BX + R + e] = plane_val(a0, py, x0 + BX + e);
    }
    if (NDIM == 3) {
      for (int e = ty; e < R; e += BY) {
        tl[e * TW + tx + R] = plane_val(a0, y0 - R + e, px);
        tl[(BY + HY + e) * TW + tx + R] = plane_val(a0, y0 + BY + e, px);
      }
    }
    __syncthreads();

    if (inner) {
      const int idx = a0 * s0 + col;
      const T uc = q[R];
      const T *trow = tl + (ty + HY) * TW + tx + R;
      const auto tap0 = [&](const int j) { return q[R + j]; };
      const auto tapM = [&](const int j) { return trow[j * TW]; };
      const auto tapF = [&](const int j) { return trow[j]; };
      const int A[3] = {a0, NDIM == 3 ? py : px, px};
      const int strides[3] = {s0, NDIM == 3 ? sM : 1, 1};

      T Dp[NDIM], Dm[NDIM], gp[NDIM], gm[NDIM], dd[NDIM];
      diffs_pinned<T, R>(tap0, uc, p.w, Dp[0], Dm[0]);
      if (NDIM == 3)
        diffs_pinned<T, R>(tapM, uc, p.w, Dp[1], Dm[1]);
      diffs_pinned<T, R>(tapF, uc, p.w, Dp[F], Dm[F]);
      T sc = p.sconst;
      if (!UNIF)
        sc = p.stiff[idx];
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        if (UNIF) {
          gp[d] = p.gconst;
          gm[d] = p.gconst;
        } else {
          const T sp = p.stiff[idx + strides[d]], sm = p.stiff[idx - strides[d]];
          gp[d] = sc * sp / (sc + sp);
          gm[d] = sc * sm / (sc + sm);
        }
        dd[d] = fma_rn(Dp[d], gp[d], -mul_rn(Dm[d], gm[d]));
      }
      T lap;
      if (NDIM == 2)
        lap = R == 1 ? fma_rn(p.f[0], dd[0], mul_rn(p.f[1], dd[1 % NDIM]))
                     : fma_rn(p.f[1], dd[1 % NDIM], mul_rn(p.f[0], dd[0]));
      else
        lap = fma_rn(p.f[2], dd[2 % NDIM], fma_rn(p.f[0], dd[0], mul_rn(p.f[1], dd[1 % NDIM])));

      // a masked domain: a node outside is not stepped; a node by its wall takes each
      // cell at its own radius, the axes summed plainly (wall_laplacian, scalar.cu:131-158)
      bool stepped = true;
      if (flags & K_CELLS) {
        const int code = p.cells[idx];
        stepped = code != 0;
        if (stepped && !(code & CELL_DEEP)) {
#pragma unroll
          for (int d = 0; d < NDIM; ++d) {
            const T term = cell_axis<T, R, UNIF>(p, u1, idx, strides[d], uc, sc, p.f[d],
                                                 (code >> (6 * d)) & 7, (code >> (6 * d + 3)) & 7);
            lap = d == 0 ? term : lap + term;
          }
        }
      }
      const T mi = (flags & K_DERIVE) ? (T)1 / sc : p.minv[idx];
      const T old = u0[idx];
      T v;
      if (flags & K_DAMP) {
        const T beta = (T)0.5 * mi * p.damping[idx] * p.dt;
        v = ((T)2 * uc - old * ((T)1 - beta) + mi * lap) / ((T)1 + beta);
      } else {
        v = -old + (T)2 * uc + mi * lap;
      }
      const bool held = held_wall(a0, N0, dir0) || (NDIM == 3 && held_wall(py, NM, dirM)) ||
                        held_wall(px, NF, dirF);
      if (held)
        v = (T)0;

      if (flags & K_PML) {
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
          const int lo = g.lo[d], hi = g.hi[d];
          if (!(lo + hi))
            continue;
          const int a = A[d], N = g.n[d];
          const int r = slab_row(a, N, lo, hi);
          if (r < 0)
            continue;
          T Dpu, Dmu;
          if (d == 0)
            diffs_plain<T, R>(tap0, uc, p.w, Dpu, Dmu);
          else if (d == F)
            diffs_plain<T, R>(tapF, uc, p.w, Dpu, Dmu);
          else
            diffs_plain<T, R>(tapM, uc, p.w, Dpu, Dmu);
          const T *prof = p.prof[d];
          const T an = prof[a], bn = prof[N + a];
          const T ah = prof[2 * N + a], bh = prof[3 * N + a];
          const T ah1 = prof[2 * N + a - 1], bh1 = prof[3 * N + a - 1];
          T *aux = p.aux[d];
          const int sz = p.auxrow[d];
          const int si = slab_index(g, d, r, A);
          const T f = p.f[d];
          const T pp = bh * aux[si] + ah * Dpu;
          const T pm = bh1 * aux[sz + si] + ah1 * Dmu;
          const T z = bn * aux[2 * sz + si] + an * f * (gp[d] * (Dpu + pp) - gm[d] * (Dmu + pm));
          aux[si] = pp;
          aux[sz + si] = pm;
          aux[2 * sz + si] = z;
          if (!held)
            v += mi * (f * (gp[d] * pp - gm[d] * pm) + z);
        }
      }

      if (flags & K_SRC) {
        for (int k = sfirst; k < slast; ++k) {
          const int4 e = p.src_entry[k];
          if (e.x == a0 && e.y == lane)
            v += p.src_weight[e.z] * p.signal[srow * p.nsrc + e.z];
        }
      }
      if ((flags & K_REFILL) && held)
        v = (T)0;
      // outside a masked domain nothing is written
      if (stepped) {
        if (flags & K_SUPER) {
          // superposed_kernel (scalar_sensitivity.cu:600-668): the mass density of the
          // triplet before, whose oldest level c still holds, and the stiffness density
          // of this one, central differences of its middle level read as stored
          const T dudt = uc - u2[idx];
          p.acc_mass[idx] += p.ft * dudt * dudt;
          T sum = (T)0;
#pragma unroll
          for (int d = 0; d < NDIM; ++d) {
            const T gd = u1[idx + strides[d]] - u1[idx - strides[d]];
            sum = d == 0 ? p.f[0] * gd * gd : sum + p.f[d] * gd * gd;
          }
          p.acc_stiff[idx] += p.fs * sum;
        }
        u2[idx] = v;
        if (flags & K_REFILL) {
#pragma unroll
          for (int d = 0; d < NDIM; ++d) {
            const int a = A[d], N = g.n[d], st = strides[d];
            if (((p.refill >> (2 * d)) & 1) && a == 2)
              u2[idx - 2 * st] = ((g.dir >> (2 * d)) & 1) ? -v : v;
            if (((p.refill >> (2 * d + 1)) & 1) && a == N - 3)
              u2[idx + 2 * st] = ((g.dir >> (2 * d + 1)) & 1) ? -v : v;
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 2 * R; ++k)
      q[k] = q[k + 1];
  }
}

template <typename T, int NDIM, int R, bool UNIF, int BX, int BY>
__global__ void __launch_bounds__(BX *BY) step_kernel(const StepParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  step_block<T, NDIM, R, UNIF, BX, BY>(p, step_index(p.ctr), blockIdx.x, blockIdx.y, blockIdx.z,
                                       gridDim.x, gridDim.y, reinterpret_cast<T *>(smem_raw));
  finish_step(p.ctr, p.flags & K_ADV);
}

}  // namespace cwb
