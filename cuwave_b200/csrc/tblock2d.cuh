// Temporal blocking of the 2D forward step: K leapfrog steps per pass over HBM.
//
// A block owns a tile of TB_TQ quads (four fast-axis nodes each) across the fast axis and a
// chunk of rows along axis 0, and advances it K steps in one pass, a group of TB_TQ
// threads (one per quad, whole warps) per level:
// level 0 is u^(t-1) and level -1 u^(t-2), read from HBM once; level j = 1 .. K is
// u^(t+j-1). The levels move down the rows as a wavefront, TB_M rows a tick, level j
// working on rows r - (j-1) L .. + TB_M - 1 at the tick where level 1 works on rows
// r .. r + TB_M - 1, with L = R + TB_M: the rows a level reads of the level before it
// (its taps, +- R) and of the one before that (its old value) are all from earlier
// ticks, so the levels of a tick are independent and one block barrier a tick orders
// them. Each level's recent rows (2L + TB_M of them) sit in a shared-memory ring; levels
// K - 1 and K, the pass's results, are written to HBM over the tile's own rows and quads.
// A thread steps consecutive rows of its column, so g D+ of a row is carried in a
// register as the next row's g D- (as step2d.cuh's queue carries it, bit for bit). Compulsory HBM traffic per node and pass: three reads
// (u^(t-2), u^(t-1), 1/m) and two writes, for K updates, against 16 bytes for each
// update stepped alone.
//
// A level's reach shrinks by one quad on each side per level (R <= 4), and the rows by R,
// so the tile overlaps its neighbours by K quads and the chunk by K R rows, recomputed in
// each: every level of every node is stepped with the same arithmetic and order as
// step2d.cuh's quad step (cuwave fd_kernel, scalar.cu:347-427, D- formed as the row
// before's D+), so the overlap is bit-identical and the result equals K single steps to
// the bit.
//
// Within a pass, as in cuwave's step (wave.py:1119-1127): the update, Dirichlet wall
// nodes held at zero, the sources added in list order (every copy of a node, the
// overlap's included, so later levels read them), the face ghosts refilled from their
// mirrors (cuwave scalar.cu:535-555; the rings keep a level's ghost columns, taps past
// a ghost row read its mirror row), then the receivers of the tile's own nodes recorded.
// Rings hold interior rows only; a tap row b past a wall reads row 2 - b or 2 (N0 - 2) - b,
// negated past a Dirichlet face (cuwave common.cuh:50-54).
//
// With a pml (the PML instance), each level advances the memory of its slab nodes after
// the update, axis 0 then axis 1 (cuwave pml_kernel, scalar.cu:500-532; the order and
// arithmetic of step2d.cuh's): an axis-0 slab row takes its taps from the window of the
// level before, an axis-1 slab node from its run. Every level reads the memory the level
// before it wrote and writes its own copy (K + 1 copies, the pass's input the first), so
// a node that neighbouring tiles or chunks both recompute is written twice with the same
// value and no block reads a copy another block may still be writing.
#pragma once

#include <type_traits>

#include "pairs.cuh"
#include "step2d.cuh"
#include "transfer.cuh"

namespace cwb {

constexpr int TB_TQ = 64;       // quads per tile row at the widest level, a level's threads
constexpr int TB_K = 4;         // steps per pass
constexpr int TB_M = 2;         // rows a level steps a tick
constexpr int TB_RECORDS = 4;   // record ops a pass writes

template <typename T>
struct TBlock2Params {
  StepParams<T> s;        // geometry, stencil row, factors, 1/m (its levels unused)
  const T *A, *B;         // u^(t-2), u^(t-1): the pass's inputs
  T *outA, *outB;         // u^(t+K-2), u^(t+K-1): its outputs (not the inputs' memory)
  int t;                  // the pass's first step
  int chunk;              // output rows per block
  int qx_step;            // output quads per tile, TB_TQ - 2K
  int refill;             // faces whose ghosts are refilled
  // folded sources listed per block over the rows and quads it steps: (row, x, index)
  const int *src_start;
  const int4 *src_entry;
  const T *src_weight;
  const T *signal;
  int nsrc, sig_mul, sig_add;
  // receivers listed per block over its own nodes: (row, x, index, record op), by row
  const int *rec_start;
  const int4 *rec_entry;
  TransferParams<T> rec[TB_RECORDS];
  int nrec;
  // the pml memory, axes 0 and 1, in the plan's (3, slab) layout: [0] the pass's input,
  // [j] what level j writes
  T *psi[TB_K + 1][2];
};

template <int R>
struct TBlockShape {
  static constexpr int M = TB_M;
  static constexpr int L = R + M;           // rows between consecutive levels' fronts
  static constexpr int NR = 2 * L + M;      // ring rows per level
  static constexpr int W = 2 * R + M;       // rows of the level before a tick reads
  static_assert(R <= 4, "the tile shrinks by one quad a level: radius 4 at most");
  static constexpr int H = 4;               // the run's halo: one quad each side
  static constexpr int XR = 12;
};

template <int R, int K>
constexpr int tblock_smem() {
  return K * TBlockShape<R>::NR * TB_TQ * 16;
}

template <int R, int K, bool HOLD, bool PML>
__global__ void __launch_bounds__(TB_TQ * K, 2) tblock2d_kernel(const __grid_constant__ TBlock2Params<float> P) {
  using T = float;
  using S = TBlockShape<R>;
  constexpr int L = S::L, NR = S::NR, H = S::H, XR = S::XR, M = S::M, W = S::W;
  extern __shared__ __align__(16) float4 tb_ring[];  // [K][NR][TB_TQ]: levels 0 .. K-1
  const StepParams<T> &p = P.s;
  const Geometry &g = p.g;
  const int N0 = g.n[0], NF = g.n[1];
  const long long s0 = g.s[0];
  const int dir0 = HOLD ? g.dir & 3 : 0, dirF = HOLD ? (g.dir >> 2) & 3 : 0;
  const T gg = p.gconst;
  const int qi = threadIdx.x % TB_TQ;
  const int lev = 1 + threadIdx.x / TB_TQ;      // the level this thread's group steps
  const int qx0 = blockIdx.x * P.qx_step - K;  // the tile's first quad (of the widest level)
  const int xq = 4 * (qx0 + qi);
  const int c0 = 1 + blockIdx.y * P.chunk;
  const int c1 = min(N0 - 1, c0 + P.chunk);
  // level j steps rows [row_lo(j), row_hi(j)) and local quads [j, TB_TQ - j)
  const auto row_lo = [&](const int j) { return max(1, c0 - (K - j) * R); };
  const auto row_hi = [&](const int j) { return min(N0 - 1, c1 + (K - j) * R); };
  const auto slot_of = [&](const int row) { return (unsigned)row % NR; };
  const auto at = [&](const int j, const int slot) -> float4 * {
    return tb_ring + (j * NR + slot) * TB_TQ;
  };
  // the thread's nodes, its Dirichlet wall nodes, its axis-1 slab nodes
  int inner = 0, xheld = 0, xslab = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int x = xq + i;
    if (x < 1 || x > NF - 2)
      continue;
    inner |= 1 << i;
    if (HOLD && held_wall(x, NF, dirF))
      xheld |= 1 << i;
    if (PML && slab_row(x, NF, g.lo[1], g.hi[1]) >= 0)
      xslab |= 1 << i;
  }
  const bool fix_lo = xq - H < 0;
  const int e_hi = NF - (xq - H);
  const bool fix_hi = e_hi <= XR - 1;
  const T slo = (dirF & 1) ? (T)-1 : (T)1, shi = (dirF & 2) ? (T)-1 : (T)1;
  const T sgl = (dir0 & 1) ? (T)-1 : (T)1, sgh = (dir0 & 2) ? (T)-1 : (T)1;
  const bool own_x = qi >= K && qi < TB_TQ - K;
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const int ext = g.ext[1];
  const bool in_row = xq >= 0 && xq + 3 <= ext - 1;  // the quad lies in memory
  const bool works = qi >= lev && qi < TB_TQ - lev && inner;
  const int gx = NF - 1 - xq;  // the high ghost's lane (4 .. 5: in the next quad)
  const bool hi_mirror = (P.refill & 8) && NF - 3 >= xq && NF - 3 <= xq + 3;
  const int rlo = row_lo(lev), rhi = row_hi(lev);
  const int step = P.t + lev - 1;
  const int bid = blockIdx.y * gridDim.x + blockIdx.x;
  const int first = row_lo(1);  // level 1's first row: the front at tick 0

  // level 0 (u^(t-1)): the rows level 1 reads at the first tick, from HBM
  if (lev == 1)
    for (int b = max(1, first - L); b <= min(N0 - 2, first + M - 1 + R); ++b)
      at(0, slot_of(b))[qi] = in_row ? *reinterpret_cast<const float4 *>(P.B + b * s0 + xq) : zero4;
  // the next tick's rows' 1/m and (level 1) u^(t-2), fetched a tick ahead
  float4 mi_next[M], old_next[M];
  const auto fetch_rows = [&](const int r0) {
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int r = r0 + m;
      mi_next[m] = old_next[m] = zero4;
      if (r < rlo || r >= rhi || !works)
        continue;
      const long long row = (long long)r * s0 + xq;
      if (!(p.flags & K_DERIVE))
        mi_next[m] = *reinterpret_cast<const float4 *>(p.minv + row);
      if (lev == 1)
        old_next[m] = *reinterpret_cast<const float4 *>(P.A + row);
    }
  };
  fetch_rows(first - (lev - 1) * L);
  __syncthreads();

  const int rec_hi = P.rec_start ? P.rec_start[bid + 1] : 0;
  int rec_cur = P.rec_start ? P.rec_start[bid] : 0;
  const int src_lo = P.src_start ? P.src_start[bid] : 0;
  const int src_hi = P.src_start ? P.src_start[bid + 1] : 0;
  const T mi_derived = (p.flags & K_DERIVE) ? (T)1 / p.sconst : (T)0;
  // -g D+ of the row before this thread's next row, a pair per half quad
  float2 npz[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  float2 w2[R];
#pragma unroll
  for (int k = 0; k < R; ++k)
    w2[k] = p_splat(p.w[k]);
  const float2 g2 = p_splat(gg), ng2 = p_splat(-gg);
  const float2 f0 = p_splat(p.f[0]), f1 = p_splat(p.f[1]);
  // ring slots of this level's rows at the first tick (rows are >= 1 - R - 2 M; the
  // offset keeps the modulo's argument positive)
  int wslot0 = (int)(((unsigned)(first - (lev - 1) * L - R + 64 * NR)) % NR);
  int rslot0 = (int)(((unsigned)(first - (lev - 1) * L + 64 * NR)) % NR);

  // a block whose rows or quads (the widest level's) meet no slab runs the march without
  // the pml's code: one kernel, two bodies, the choice uniform over the block
  const auto slab_block = [&]() {
    const int lo0 = g.lo[0], hi0 = g.hi[0], lo1 = g.lo[1], hi1 = g.hi[1];
    const int ra = row_lo(1), rb = row_hi(1) - 1;  // rows, inclusive
    const int xa = 4 * (qx0 + 1), xb = 4 * (qx0 + TB_TQ - 1) - 1;  // nodes, inclusive
    return (lo0 && ra <= lo0) || (hi0 && rb >= N0 - 1 - hi0) || (lo1 && xa <= lo1) ||
           (hi1 && xb >= NF - 1 - hi1);
  };
  const auto march = [&](auto pml_c) {
  constexpr bool DO_PML = decltype(pml_c)::value;
  for (int front = first; front - (K - 1) * L < row_hi(K); front += M) {
    // level 1's group fetches the rows of u^(t-1) it reads M ahead next tick
    float4 next[M];
    bool fetch[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int b = front + M + R + m;
      fetch[m] = lev == 1 && b >= 1 && b <= N0 - 2 && b <= row_hi(1) - 1 + R;
      next[m] = fetch[m] && in_row ? *reinterpret_cast<const float4 *>(P.B + b * s0 + xq) : zero4;
    }
    const int r0 = front - (lev - 1) * L;
    // the ring slots of r0 - R (the window's first row) and r0, advanced by M a tick
    const int wslot = wslot0, rslot = rslot0;
    wslot0 = wslot0 + M >= NR ? wslot0 + M - NR : wslot0 + M;
    rslot0 = rslot0 + M >= NR ? rslot0 + M - NR : rslot0 + M;
    float4 mi4[M], o4p[M];
#pragma unroll
    for (int m = 0; m < M; ++m)
      mi4[m] = mi_next[m], o4p[m] = old_next[m];
    fetch_rows(r0 + M);
    if (works && r0 + M > rlo && r0 < rhi) {
      const int pj = lev - 1;  // the level read
      // rows r0 - R .. r0 + M - 1 + R of the level before; a row past a wall reads its
      // mirror row (2 - b, 2 (N0 - 2) - b), negated past a Dirichlet face
      T win[W][4];
      if (r0 - R >= 1 && r0 + M - 1 + R <= N0 - 2) {
        int sl = wslot;
#pragma unroll
        for (int w = 0; w < W; ++w) {
          const float4 a = at(pj, sl)[qi];
          win[w][0] = a.x, win[w][1] = a.y, win[w][2] = a.z, win[w][3] = a.w;
          sl = sl + 1 == NR ? 0 : sl + 1;
        }
      } else {
#pragma unroll
        for (int w = 0; w < W; ++w) {
          const int b = r0 - R + w;
          const T sg = b > N0 - 2 ? sgh : b < 1 ? sgl : (T)1;
          const int mb = b > N0 - 2 ? 2 * (N0 - 2) - b : b < 1 ? 2 - b : b;
          float4 a = zero4;
          if (mb >= 1 && mb <= N0 - 2)
            a = at(pj, slot_of(mb))[qi];
          win[w][0] = sg * a.x, win[w][1] = sg * a.y, win[w][2] = sg * a.z, win[w][3] = sg * a.w;
        }
      }
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int r = r0 + m;
        if (r < rlo || r >= rhi)
          continue;
        const int c = R + m;  // the row's place in the window
        // rows of the window as pairs of nodes (half h of the quad)
        const auto pair = [&](const int w, const int h) {
          return make_float2(win[w][2 * h], win[w][2 * h + 1]);
        };
        if (r == rlo) {
          // the carry's start: D+ of the row before, from its own taps
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const auto tb = [&](const int k) { return pair(c - 1 + k, h); };
            npz[h] = p_mul(p_dplus<R>(tb, pair(c - 1, h), w2), ng2);
          }
        }
        const long long row = (long long)r * s0 + xq;
        const int cs = rslot + m >= NR ? rslot + m - NR : rslot + m;
        // the row's run along the fast axis, from the level before's ring
        T xr[XR];
        {
          const float4 *rr = at(pj, cs);
          const float4 a = rr[qi - 1], b = rr[qi + 1];
          xr[0] = a.x, xr[1] = a.y, xr[2] = a.z, xr[3] = a.w;
#pragma unroll
          for (int i = 0; i < 4; ++i)
            xr[H + i] = win[c][i];
          xr[8] = b.x, xr[9] = b.y, xr[10] = b.z, xr[11] = b.w;
        }
        if (fix_lo)
          mirror_run_lo_at<T, XR, H>(xr, slo, H - xq);
        if (fix_hi)
          mirror_run_hi_at<T, XR, H + 2>(xr, shi, e_hi);
        float4 o4;
        if (lev == 1)
          o4 = o4p[m];
        else
          o4 = at(lev - 2, cs)[qi];
        const T old[4] = {o4.x, o4.y, o4.z, o4.w};
        T mi[4] = {mi4[m].x, mi4[m].y, mi4[m].z, mi4[m].w};
        if (p.flags & K_DERIVE) {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            mi[i] = mi_derived;
        }
        // axis 1: D+ at faces x0 - 1 .. x0 + 3; axis 0: D+ here and the carried g D-
        T dx[5];
#pragma unroll
        for (int jj = 0; jj < 5; ++jj) {
          const auto tx = [&](const int kk) { return xr[H - 1 + jj + kk]; };
          dx[jj] = dplus<T, R>(tx, xr[H - 1 + jj], p.w);
        }
        T v[4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          // axis 0 on the pair; the laplacian; (2u - u0) + (1/m) lap, the product lane by
          // lane (a packed one would be contracted into the sum)
          const auto tz = [&](const int k) { return pair(c + k, h); };
          const float2 dpz = p_dplus<R>(tz, pair(c, h), w2);
          const float2 ddz = p_fma(dpz, g2, npz[h]);
          npz[h] = p_mul(dpz, ng2);
          const float2 ddx = make_float2(fma_rn(dx[2 * h + 1], gg, -mul_rn(dx[2 * h], gg)),
                                         fma_rn(dx[2 * h + 2], gg, -mul_rn(dx[2 * h + 1], gg)));
          const float2 lap = R == 1 ? p_fma(f0, ddz, p_mul(f1, ddx)) : p_fma(f1, ddx, p_mul(f0, ddz));
          const float2 uc = make_float2(xr[H + 2 * h], xr[H + 2 * h + 1]);
          const float2 o = make_float2(old[2 * h], old[2 * h + 1]);
          const float2 r2 = p_add(p_sub(p_add(uc, uc), o),
                                  make_float2(mul_rn(mi[2 * h], lap.x), mul_rn(mi[2 * h + 1], lap.y)));
          v[2 * h] = r2.x;
          v[2 * h + 1] = r2.y;
        }
        const int held = HOLD ? (held_wall(r, N0, dir0) ? inner : xheld) : 0;
        if (HOLD) {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if ((held >> i) & 1)
              v[i] = (T)0;
        }
        if constexpr (DO_PML) {
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
          const int zrow = slab_row(r, N0, g.lo[0], g.hi[0]);
          if (zrow >= 0) {
            // an axis-0 slab row: its taps from the window, its memory row contiguous
            const T *src = P.psi[lev - 1][0];
            T *dst = P.psi[lev][0];
            const long long sz = p.auxrow[0], si = (long long)zrow * ext + xq;
            T m0[4], m1[4], m2[4];
            load4(m0, src + si);
            load4(m1, src + sz + si);
            load4(m2, src + 2 * sz + si);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              if (!((inner >> i) & 1))
                continue;
              const auto tap = [&](const int j) { return win[c + j][i]; };
              T Dpu, Dmu;
              diffs_plain<T, R>(tap, win[c][i], p.w, Dpu, Dmu);
              node(i, 0, r, N0, Dpu, Dmu, m0[i], m1[i], m2[i]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
              if ((inner >> i) & 1) {
                dst[si + i] = m0[i];
                dst[sz + si + i] = m1[i];
                dst[2 * sz + si + i] = m2[i];
              }
          }
          if (xslab) {
            const T *src = P.psi[lev - 1][1];
            T *dst = P.psi[lev][1];
            const long long sz = p.auxrow[1];
            const int lo = g.lo[1], hi = g.hi[1];
            const long long base = (long long)r * (lo + hi);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              if (!((xslab >> i) & 1))
                continue;
              const auto tap = [&](const int j) { return xr[H + i + j]; };
              T Dpu, Dmu;
              diffs_plain<T, R>(tap, xr[H + i], p.w, Dpu, Dmu);
              const long long si = base + slab_row(xq + i, NF, lo, hi);
              T m0 = src[si], m1 = src[sz + si], m2 = src[2 * sz + si];
              node(i, 1, xq + i, NF, Dpu, Dmu, m0, m1, m2);
              dst[si] = m0;
              dst[sz + si] = m1;
              dst[2 * sz + si] = m2;
            }
          }
        }
        // the sources on this quad, in the list's order
        if (src_hi > src_lo) {
          const long long srow = (long long)P.sig_mul * step + P.sig_add;
          for (int e = src_lo; e < src_hi; ++e) {
            const int4 en = P.src_entry[e];
            if (en.x == r && en.y >= xq && en.y < xq + 4) {
              const T add = P.src_weight[en.z] * P.signal[srow * P.nsrc + en.z];
#pragma unroll
              for (int i = 0; i < 4; ++i)
                if (en.y - xq == i)
                  v[i] += add;
            }
          }
        }
        // the ghost columns of this level's row: refilled from their mirrors (lane 0 of
        // quad 0 from lane 2; node NF - 1 from NF - 3, in this quad or the next)
        T out[4] = {v[0], v[1], v[2], v[3]};
        int ghost_lanes = 0;
        if ((P.refill & 4) && xq == 0) {
          out[0] = (dirF & 1) ? -v[2] : v[2];
          ghost_lanes |= 1;
        }
        bool ghost_next = false;
        T ghost_val = (T)0;
        if (hi_mirror) {
          // this quad holds node NF - 3: its ghost NF - 1 takes its value
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            if (NF - 3 - xq != a)
              continue;
            const T gv = (dirF & 2) ? -v[a] : v[a];
            if (a + 2 <= 3) {
              out[a + 2 < 4 ? a + 2 : 3] = gv;
              ghost_lanes |= 1 << (a + 2);
            } else {
              ghost_next = true;
              ghost_val = gv;
            }
          }
        }
        if (lev < K) {
          at(lev, cs)[qi] = make_float4(out[0], out[1], out[2], out[3]);
          if (ghost_next)
            reinterpret_cast<T *>(at(lev, cs) + qi + 1)[gx - 4] = ghost_val;
        }
        // the pass's results over the tile's own nodes, ghosts included (no corner)
        if (lev >= K - 1 && own_x && r >= c0 && r < c1) {
          T *dst = lev == K ? P.outB : P.outA;
          const int mask = inner | ghost_lanes;
          if (mask == 15) {
            store4(dst + row, out);
          } else {
#pragma unroll
            for (int i = 0; i < 4; ++i)
              if ((mask >> i) & 1)
                dst[row + i] = out[i];
          }
          if (ghost_next)
            dst[row + gx] = ghost_val;
          // ghost rows: refilled from rows 2 and N0 - 3 over the interior columns
          if ((P.refill & 1) && r == 2) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
              if ((inner >> i) & 1)
                dst[row - 2 * s0 + i] = (dir0 & 1) ? -v[i] : v[i];
          }
          if ((P.refill & 2) && r == N0 - 3) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
              if ((inner >> i) & 1)
                dst[row + 2 * s0 + i] = (dir0 & 2) ? -v[i] : v[i];
          }
        }
        // the receivers of the tile's own nodes on this row (the block's list is by row)
        if (P.nrec && own_x) {
          while (rec_cur < rec_hi && P.rec_entry[rec_cur].x < r)
            ++rec_cur;
          for (int e = rec_cur; e < rec_hi; ++e) {
            const int4 en = P.rec_entry[e];
            if (en.x != r)
              break;
            if (en.y >= xq && en.y < xq + 4) {
              const TransferParams<T> &rp2 = P.rec[en.w];
              const long long rrow = (long long)rp2.row_mul * step + rp2.row_add;
              T val = v[0];
#pragma unroll
              for (int i = 1; i < 4; ++i)
                if (en.y - xq == i)
                  val = v[i];
              record_write(rp2, rrow * rp2.num + en.z, val);
            }
          }
        }
      }
    }
#pragma unroll
    for (int m = 0; m < M; ++m)
      if (fetch[m])
        at(0, slot_of(front + M + R + m))[qi] = next[m];
    __syncthreads();
  }
  };
  if (PML && slab_block())
    march(std::true_type{});
  else
    march(std::false_type{});
}

}  // namespace cwb
