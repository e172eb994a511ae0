// The forward step with TMA-staged planes.
//
// A block owns a BX x BY tile of the plane orthogonal to axis 0 (BX x 1 in 2D) and marches
// `chunk` planes along axis 0. One thread issues, per plane, three tensor-map tile loads
// into a ring of shared-memory stages: u^(t-1) over the tile and an R-wide halo, u^(t-2)
// and 1/m over the tile. The ring runs R + 1 + PREFETCH planes ahead, so a block keeps
// several planes of loads in flight without holding them in registers. Each thread
// steps RY rows of its column, keeping each row's 2R + 1 values along axis 0 in a
// register queue fed from the staged planes; in-plane taps read the current plane's stage.
//
// Tiles at the domain's edge rewrite the halo cells past a wall with their mirrors (the
// TMA fills them with zeros), in the forward convention of cuwave common.cuh:50-69. The
// node arithmetic is step.cuh's, i.e. cuwave fd_kernel + pml_kernel (scalar.cu:347-532).
#pragma once

#include <type_traits>

#include "step.cuh"
#include "tma.cuh"

namespace cwb {

#ifndef TMA_MIN_BLOCKS
#define TMA_MIN_BLOCKS 3  // resident blocks per SM the register budget is cut for
#endif

template <typename T>
struct StepTmaParams {
  StepParams<T> s;
  CUtensorMap map_u1;   // levels of operand b: (ext_F, NM, n0, levels), box (WB, HB, 1, 1)
  CUtensorMap map_u0;   // levels of operand a: box (BX, BY, 1, 1)
  CUtensorMap map_minv; // (ext_F, NM, n0), box (BX, BY, 1)
  int level_u1[3];      // mul, add, period of b's level index
  int level_u0[3];
  int *err;
};

template <typename T, int NDIM, int R, int BX, int BY>
struct TmaShape {
  static constexpr int H = ((R * (int)sizeof(T) + 15) / 16) * 16 / (int)sizeof(T);  // x halo
  static constexpr int HY = NDIM == 3 ? R : 0;
  static constexpr int WB = BX + 2 * H;
  static constexpr int HB = BY + 2 * HY;
  // planes in flight past the queue's lead: deeper where the ring still fits 3 blocks
  static constexpr int PREFETCH = R <= 4 ? 3 : 2;
  static constexpr int STAGES = R + 1 + PREFETCH;
  static constexpr int U1_BYTES = WB * HB * (int)sizeof(T);
  static constexpr int TILE_BYTES = BX * BY * (int)sizeof(T);
  static constexpr int align128(int b) { return (b + 127) / 128 * 128; }
  static constexpr int U0_OFF = align128(U1_BYTES);
  static constexpr int MINV_OFF = U0_OFF + align128(TILE_BYTES);
  static constexpr int STAGE_BYTES = MINV_OFF + align128(TILE_BYTES);
  static constexpr int SMEM = STAGES * STAGE_BYTES + 128;
};

__device__ __forceinline__ int level_index(const int *L, const int t) {
  int k = L[0] * t + L[1];
  if (L[2] > 0) {
    k %= L[2];
    if (k < 0)
      k += L[2];
  }
  return k;
}

// resident blocks an SM the register budget is cut for: three, or two for the 3D rows
// of radius 5 and up, whose queues would otherwise spill (364 bytes a thread at radius 8)
template <int NDIM, int R>
constexpr int tma_min_blocks() {
  return NDIM == 3 && R >= 5 ? 2 : TMA_MIN_BLOCKS;
}

template <typename T, int NDIM, int R, bool UNIF, int BX, int BY, int RY>
__global__ void __launch_bounds__(BX *(BY / RY), tma_min_blocks<NDIM, R>())
    step_tma_kernel(const __grid_constant__ StepTmaParams<T> P) {
  using S = TmaShape<T, NDIM, R, BX, BY>;
  constexpr int H = S::H, HY = S::HY, WB = S::WB, NS = S::STAGES, F = NDIM - 1;
  constexpr int TY = BY / RY;
  static_assert(NDIM == 3 || (BY == 1 && RY == 1), "a 2D tile is one row");
  extern __shared__ __align__(128) unsigned char tma_smem[];
  __shared__ __align__(8) uint64_t full[NS];
  unsigned char *ring =
      align_smem128(tma_smem);

  const StepParams<T> &p = P.s;
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  const T *u0 = level<T>(p.u0, t);
  const T *__restrict__ u1 = level<T>(p.u1, t);
  T *u2 = level<T>(p.u2, t);
  const int lev1 = level_index(P.level_u1, t), lev0 = level_index(P.level_u0, t);

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x0 = blockIdx.x * BX;
  const int y0 = NDIM == 3 ? blockIdx.y * BY : 0;
  const int cz = NDIM == 3 ? blockIdx.z : blockIdx.y;
  const int N0 = g.n[0], NF = g.n[F], NM = NDIM == 3 ? g.n[1] : 1;
  const int s0 = g.s[0], sM = NDIM == 3 ? g.s[1] : 0;
  const int c0 = 1 + cz * p.chunk;
  const int c1 = min(N0 - 1, c0 + p.chunk);
  const int dir0 = g.dir & 3;
  const int dirM = NDIM == 3 ? (g.dir >> 2) & 3 : 0;
  const int dirF = (g.dir >> (2 * F)) & 3;
  const int flags = p.flags;
  const bool leader = tx == 0 && ty == 0;
  // whether the box reaches past a wall or into the padding, so its halo needs mirrors
  const bool edge = x0 - H < 0 || x0 + BX + H > NF || (NDIM == 3 && (y0 - HY < 0 || y0 + BY + HY > NM));

  const auto stage = [&](const int plane) { return ring + ((unsigned)plane % NS) * S::STAGE_BYTES; };
  int issued = c0 - 1, arrived = c0 - 1;  // the last plane issued (leader) and waited for
  const auto issue = [&](const int plane) {
    issued = plane;
    unsigned char *st = stage(plane);
    uint64_t *bar = &full[(unsigned)plane % NS];
    const bool node_tiles = plane < c1;  // u^(t-2) and 1/m only for planes stepped here
    unsigned bytes = S::U1_BYTES;
    if (node_tiles)
      bytes += S::TILE_BYTES * ((flags & K_DERIVE) ? 1 : 2);
    mbar_expect(bar, bytes);
    tma_load_4d(st, &P.map_u1, bar, x0 - H, y0 - HY, plane, lev1);
    if (node_tiles) {
      tma_load_4d(st + S::U0_OFF, &P.map_u0, bar, x0, y0, plane, lev0);
      if (!(flags & K_DERIVE))
        tma_load_3d(st + S::MINV_OFF, &P.map_minv, bar, x0, y0, plane);
    }
  };

  // planes c0 .. c1 - 1 + R are staged; the ones past the last row read zeros there
  const int last = c1 - 1 + R;
  if (leader) {
    for (int i = 0; i < NS; ++i)
      mbar_init(&full[i], 1);
    fence_barrier_init();
    prefetch_map(&P.map_u1);
    prefetch_map(&P.map_u0);
    if (!(flags & K_DERIVE))
      prefetch_map(&P.map_minv);
  }
  __syncthreads();
  if (leader && c0 < c1)
    for (int pl = c0; pl < c0 + NS - 1 && pl <= last; ++pl)
      issue(pl);

  // rows of this thread and their columns
  int py[RY], col[RY];
  bool own[RY], inner[RY];
  const int px = x0 + tx;
#pragma unroll
  for (int k = 0; k < RY; ++k) {
    py[k] = y0 + ty + k * TY;
    own[k] = px <= NF - 1 && (NDIM == 2 || py[k] <= NM - 1);
    inner[k] = px >= 1 && px <= NF - 2 && (NDIM == 2 || (py[k] >= 1 && py[k] <= NM - 2));
    col[k] = (NDIM == 3 ? py[k] * sM : 0) + px;
  }
  // u^(t-1) at row b of column c, through its mirror along axis 0, from global memory
  const auto row_val = [&](const int b, const int c) -> T {
    int sg;
    const int m = mirror_node(b, N0, dir0, sg);
    const T v = u1[m * s0 + c];
    return sg < 0 ? -v : v;
  };
  T q[RY][2 * R + 1];
  if (c0 < c1) {
#pragma unroll
    for (int k = 0; k < RY; ++k)
      if (own[k]) {
#pragma unroll
        for (int j = 0; j < 2 * R; ++j)
          q[k][j] = row_val(c0 - R + j, col[k]);
      }
  }
  int sfirst = 0, slast = 0, srow = 0;
  if (flags & K_SRC) {
    const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    sfirst = p.src_start[blk];
    slast = p.src_start[blk + 1];
    srow = p.sig_mul * t + p.sig_add;
  }
  // An edge tile's box past the walls takes the mirrored values (the copy zero-filled
  // it). Only the out-of-range columns and rows are visited; a cell out of range on both
  // axes is never read by a star stencil and is zeroed.
  const int xlo_end = max(0, min(WB, H - x0));        // columns with x < 0
  const int xhi_beg = max(0, min(WB, NF - (x0 - H)));  // columns with x > NF - 1
  const int ylo_end = NDIM == 3 ? max(0, min(S::HB, HY - y0)) : 0;
  const int yhi_beg = NDIM == 3 ? max(0, min(S::HB, NM - (y0 - HY))) : S::HB;
  const auto fix_cell = [&](T *box, const int bx, const int by) {
    const int xg = x0 - H + bx, yg = y0 - HY + by;
    const bool xin = xg >= 0 && xg <= NF - 1;
    const bool yin = NDIM == 2 || (yg >= 0 && yg <= NM - 1);
    if (xin && yin)
      return;
    T v = (T)0;
    if (xin != yin) {
      int sx = 1, sy = 1;
      const int mx = xin ? xg : mirror_node(xg, NF, dirF, sx);
      const int my = (NDIM == 2 || yin) ? yg : mirror_node(yg, NM, dirM, sy);
      const int lx = mx - (x0 - H), ly = my - (y0 - HY);
      const bool mine = mx >= 0 && mx <= NF - 1 && my >= 0 && (NDIM == 2 || my <= NM - 1);
      if (mine && lx >= 0 && lx < WB && ly >= 0 && ly < S::HB) {
        const T m = box[ly * WB + lx];
        v = sx * sy < 0 ? -m : m;
      }
    }
    box[by * WB + bx] = v;
  };
  const auto fix = [&](const int plane) {
    T *box = reinterpret_cast<T *>(stage(plane));
    const int nthreads = BX * TY, tid = ty * BX + tx;
    const int ncols = xlo_end + (WB - xhi_beg);
    for (int c = tid; c < ncols * S::HB; c += nthreads) {
      const int ci = c % ncols, by = c / ncols;
      fix_cell(box, ci < xlo_end ? ci : xhi_beg + (ci - xlo_end), by);
    }
    const int nrows = ylo_end + (S::HB - yhi_beg);
    for (int c = tid; c < nrows * WB; c += nthreads) {
      const int ri = c / WB, bx = c % WB;
      fix_cell(box, bx, ri < ylo_end ? ri : yhi_beg + (ri - ylo_end));
    }
  };
  // wait for a staged plane: the leader polls the barrier, the block learns the outcome
  // at the barrier after; then an edge tile's halo takes its mirrors. False if the
  // bounded wait ran out.
  const auto arrive = [&](const int plane) -> bool {
    bool good = true;
    if (leader && plane <= last)
      good = mbar_wait(&full[(unsigned)plane % NS], ((unsigned)(plane - c0) / NS) & 1u);
    if (!__syncthreads_and(good))
      return false;
    arrived = plane;
    if (plane <= last && edge) {
      fix(plane);
      __syncthreads();
    }
    return true;
  };

  // what the tile's nodes can meet, fixed for the block: pml slabs of the in-plane axes,
  // the mirror rows the folded refill writes from, Dirichlet wall nodes, sources
  const int xa = max(x0, 1), xb = min(x0 + BX - 1, NF - 2);
  const int ya = NDIM == 3 ? max(y0, 1) : 0, yb = NDIM == 3 ? min(y0 + BY - 1, NM - 2) : 0;
  const auto meets = [](const int a, const int b, const int lo, const int hi) {
    return a <= hi && lo <= b;
  };
  bool tile_general = (flags & K_DAMP) || sfirst < slast;
  if (flags & K_PML) {
    const int loF = g.lo[F], hiF = g.hi[F];
    tile_general |= (loF && meets(xa, xb, 1, loF)) || (hiF && meets(xa, xb, NF - 1 - hiF, NF - 2));
    if (NDIM == 3) {
      const int loM = g.lo[1], hiM = g.hi[1];
      tile_general |= (loM && meets(ya, yb, 1, loM)) || (hiM && meets(ya, yb, NM - 1 - hiM, NM - 2));
    }
  }
  if (flags & K_REFILL) {
    tile_general |= meets(xa, xb, 2, 2) || meets(xa, xb, NF - 3, NF - 3);
    if (NDIM == 3)
      tile_general |= meets(ya, yb, 2, 2) || meets(ya, yb, NM - 3, NM - 3);
  }
  tile_general |= ((dirF & 1) && meets(xa, xb, 1, 1)) || ((dirF & 2) && meets(xa, xb, NF - 2, NF - 2));
  if (NDIM == 3)
    tile_general |= ((dirM & 1) && meets(ya, yb, 1, 1)) || ((dirM & 2) && meets(ya, yb, NM - 2, NM - 2));

  bool ok = true;
  if (c0 < c1)
    for (int pl = c0; pl < c0 + R && ok; ++pl)
      ok = arrive(pl);

  for (int a0 = c0; a0 < c1 && ok; ++a0) {
    const int ahead = a0 + R;  // the plane whose arrival feeds the queue
    if (!arrive(ahead)) {
      ok = false;
      break;
    }
    // refill the stage freed by the plane before this one, after every thread left it
    if (leader) {
      const int next = a0 + NS - 1;
      if (next <= last) {
        fence_proxy_async();
        issue(next);
      }
    }
    const T *cur = reinterpret_cast<const T *>(stage(a0));
    const T *nxt = reinterpret_cast<const T *>(stage(ahead));
#pragma unroll
    for (int k = 0; k < RY; ++k) {
      if (!own[k])
        continue;
      const int cell = (ty + k * TY + HY) * WB + tx + H;
      q[k][2 * R] = ahead <= N0 - 1 ? nxt[cell] : row_val(ahead, col[k]);
    }
    // the plane's own slab, refill row or wall send it down the general path
    bool general = tile_general;
    if (flags & K_PML)
      general |= (g.lo[0] && a0 <= g.lo[0]) || (g.hi[0] && a0 >= N0 - 1 - g.hi[0]);
    if (flags & K_REFILL)
      general |= a0 == 2 || a0 == N0 - 3;
    general |= ((dir0 & 1) && a0 == 1) || ((dir0 & 2) && a0 == N0 - 2);
    const T *tile0 = reinterpret_cast<const T *>(stage(a0) + S::U0_OFF);
    const T *tilem = reinterpret_cast<const T *>(stage(a0) + S::MINV_OFF);

    const auto node = [&](const int k, auto full_path) {
      constexpr bool GEN = decltype(full_path)::value;
      const int idx = a0 * s0 + col[k];
      const T uc = q[k][R];
      const T *trow = cur + (ty + k * TY + HY) * WB + tx + H;
      const auto tap0 = [&](const int j) { return q[k][R + j]; };
      const auto tapM = [&](const int j) { return trow[j * WB]; };
      const auto tapF = [&](const int j) { return trow[j]; };
      const int tc = (ty + k * TY) * BX + tx;

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
          const int st = d == 0 ? s0 : (d == F ? 1 : sM);
          const T sp = p.stiff[idx + st], sm = p.stiff[idx - st];
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
      const T mi = (flags & K_DERIVE) ? (T)1 / sc : tilem[tc];
      const T old = tile0[tc];
      T v;
      if (GEN && (flags & K_DAMP)) {
        const T beta = (T)0.5 * mi * p.damping[idx] * p.dt;
        v = ((T)2 * uc - old * ((T)1 - beta) + mi * lap) / ((T)1 + beta);
      } else {
        v = -old + (T)2 * uc + mi * lap;
      }
      if constexpr (GEN) {
        const int pyk = NDIM == 3 ? py[k] : 0;
        const bool held = held_wall(a0, N0, dir0) || (NDIM == 3 && held_wall(pyk, NM, dirM)) ||
                          held_wall(px, NF, dirF);
        if (held)
          v = (T)0;
        if (flags & K_PML) {
#pragma unroll
          for (int d = 0; d < NDIM; ++d) {
            const int lo = g.lo[d], hi = g.hi[d];
            if (!(lo + hi))
              continue;
            const int a = d == 0 ? a0 : (d == F ? px : pyk);
            const int N = g.n[d];
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
            const int rows = lo + hi, extF = g.ext[F];
            // the memory's own layout: the padded grid with axis d replaced by its rows
            int si;
            if (NDIM == 3)
              si = d == 0 ? (r * NM + pyk) * extF + px
                          : (d == 1 ? (a0 * rows + r) * extF + px : (a0 * NM + pyk) * rows + r);
            else
              si = d == 0 ? r * extF + px : a0 * rows + r;
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
          const int lane = (ty + k * TY) * BX + tx;
          for (int e = sfirst; e < slast; ++e) {
            const int4 en = p.src_entry[e];
            if (en.x == a0 && en.y == lane)
              v += p.src_weight[en.z] * p.signal[srow * p.nsrc + en.z];
          }
        }
        if ((flags & K_REFILL) && held)
          v = (T)0;
        u2[idx] = v;
        if (flags & K_REFILL) {
#pragma unroll
          for (int d = 0; d < NDIM; ++d) {
            const int a = d == 0 ? a0 : (d == F ? px : pyk), N = g.n[d];
            const int st = d == 0 ? s0 : (d == F ? 1 : sM);
            if (((p.refill >> (2 * d)) & 1) && a == 2)
              u2[idx - 2 * st] = ((g.dir >> (2 * d)) & 1) ? -v : v;
            if (((p.refill >> (2 * d + 1)) & 1) && a == N - 3)
              u2[idx + 2 * st] = ((g.dir >> (2 * d + 1)) & 1) ? -v : v;
          }
        }
      } else {
        u2[idx] = v;
      }
    };
    if (general) {
#pragma unroll
      for (int k = 0; k < RY; ++k)
        if (inner[k])
          node(k, std::true_type{});
    } else {
#pragma unroll
      for (int k = 0; k < RY; ++k)
        if (inner[k])
          node(k, std::false_type{});
    }
#pragma unroll
    for (int k = 0; k < RY; ++k)
#pragma unroll
      for (int j = 0; j < 2 * R; ++j)
        q[k][j] = q[k][j + 1];
  }

  if (!ok) {
    // a tile never arrived: flag it, and drain what is still in flight before leaving
    if (leader) {
      atomicExch(P.err, 1);
      for (int pl = arrived + 1; pl <= issued; ++pl)
        mbar_wait(&full[(unsigned)pl % NS], ((unsigned)(pl - c0) / NS) & 1u);
    }
  }
  finish_step(p.ctr, flags & K_ADV);
}

}  // namespace cwb
