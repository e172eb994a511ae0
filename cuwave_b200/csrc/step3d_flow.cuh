// The 3D forward step of a uniform stiffness, with no block-wide barrier in its march.
//
// The tiling is step3d.cuh's: a block of 256 threads owns a 64 x 16 tile of the
// (axis-1, axis-2) plane and marches a chunk of planes along axis 0, each thread a quad
// of four consecutive axis-2 nodes of one axis-1 row, the axis-0 taps in a register
// queue, the in-plane taps from TMA-staged boxes in a shared-memory ring. What differs:
//
//   * One stage per plane z: the box of u^(t-1) that the queue takes in at z (plane
//     z + R, with its in-plane halo) and the tile of u^(t-2) and 1/m at z, completing
//     on one mbarrier. Every warp waits for its stage itself and no warp waits for
//     another, so warps drift apart by up to the ring's slack and one warp's arithmetic
//     overlaps another's wait instead of all eight meeting at a barrier every plane.
//   * A stage's slots are refilled by the warp that leaves them last: each warp counts
//     itself past its plane on the stage's counter (an acquire-release shared atomic)
//     and the one that completes the count issues the stage NT planes on. No thread
//     waits for a slot to empty.
//   * The plane body is built in four forms, chosen per block and per plane by uniform
//     branches: interior tiles (every thread steps a whole quad with no wall in reach)
//     against edge tiles (mirrors along axes 1 and 2, partial quads, held wall nodes),
//     and ordinary planes against special ones (an axis-0 pml slab plane, a held wall
//     plane, a feed past the last plane). The interior form of an ordinary plane, the
//     bulk of a large grid, carries no test at all.
//   * Two nodes of a quad share each instruction along axes 0 and 1 and in the update:
//     sm_100's packed f32x2 add, subtract, multiply and fused multiply-add. Each lane
//     rounds as its scalar operation does, so the node arithmetic, its order and its
//     roundings are step.cuh's (cuwave fd_kernel, scalar.cu:347-427), bit for bit. One
//     exception is kept scalar: ptxas contracts a packed product into a packed sum it
//     feeds (measured: one rounding instead of two, whatever --fmad says), so a product
//     that a sum consumes is formed lane by lane.
//   * Rows of a box past an axis-1 wall are not rewritten in place; a thread of an edge
//     tile reads its axis-1 taps through the mirrored row instead (cuwave
//     common.cuh:50-69), negated past a Dirichlet face.
//
// Every wait is bounded (tma.cuh); a warp whose wait runs out raises the launch's error
// flag and leaves the march, and the block drains every copy still in flight before it
// exits.
#pragma once

#include <type_traits>

#include "pairs.cuh"
#include "step3d.cuh"

namespace cwb {

// a quad as two pairs, from 16-byte aligned memory and back
struct Quad2 {
  float2 lo, hi;
  __device__ __forceinline__ float2 &operator[](const int h) { return h ? hi : lo; }
  __device__ __forceinline__ const float2 &operator[](const int h) const { return h ? hi : lo; }
};
__device__ __forceinline__ Quad2 ldq(const float *src) {
  const float4 v = *reinterpret_cast<const float4 *>(src);
  return {make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ void stq(float *dst, const Quad2 &v) {
  *reinterpret_cast<float4 *>(dst) = make_float4(v.lo.x, v.lo.y, v.hi.x, v.hi.y);
}
__device__ __forceinline__ float lane_of(const Quad2 &v, const int i) {
  return i == 0 ? v.lo.x : i == 1 ? v.lo.y : i == 2 ? v.hi.x : v.hi.y;
}
__device__ __forceinline__ void set_lane(Quad2 &v, const int i, const float x) {
  if (i == 0)
    v.lo.x = x;
  else if (i == 1)
    v.lo.y = x;
  else if (i == 2)
    v.hi.x = x;
  else
    v.hi.y = x;
}

// one warp's count past a stage; true for the warp that completes the count of `warps`
// (the last to leave the stage's plane)
__device__ __forceinline__ bool release_stage(unsigned *count, const unsigned warps) {
  unsigned old;
  asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], 1;"
               : "=r"(old)
               : "r"(smem_addr(count))
               : "memory");
  return old % warps == warps - 1;
}

// the wait of a whole warp on a stage: one test, then the bounded loop if it is not in
__device__ __forceinline__ bool warp_wait(uint64_t *bar, const unsigned parity) {
  bool good = mbar_try(bar, parity);
  if (!__all_sync(0xffffffffu, good))
    good = __all_sync(0xffffffffu, mbar_wait(bar, parity));
  return good;
}

// HOLD: the grid has a Dirichlet face; DERIVE: 1/m = 1/k; DAMP: a damping field
template <typename T, int R, bool HOLD, bool DERIVE, bool DAMP>
__global__ void __launch_bounds__(S3_THREADS, 2)
    step3d_flow_kernel(const __grid_constant__ Step3Params<T> P) {
  using S = Step3Shape<T, R>;
  static_assert(S::SUPPORTED, "the blocked 3D step is built for float up to radius 4");
  static_assert(sizeof(T) == 4, "packed pairs of float");
  constexpr int H = S::H, WB = S::WB, HB = S::HB, XR = S::XR;
  constexpr int NB = S::NS1;  // boxes: the centre plane's through the feed's, and the slack
  constexpr int NT = S::NS0;  // tiles, stages and their barriers
  constexpr int BX = S3_BX, BY = S3_BY, NW = S3_THREADS / 32;
  constexpr int BOXF = S::BOX_BYTES / (int)sizeof(T), TILEF = 2 * S::TILE_BYTES / (int)sizeof(T);
  extern __shared__ __align__(128) unsigned char s3_smem[];
  __shared__ __align__(8) uint64_t stage_bar[NT];
  __shared__ __align__(8) uint64_t first_bar;  // the boxes of the chunk's first R planes
  __shared__ unsigned done[NT];                // warps past each stage's plane, counted up
  __shared__ int last[NT];                     // the last stage issued on each barrier
  T *ring1 = reinterpret_cast<T *>(align_smem128(s3_smem));
  T *ring0 = ring1 + NB * BOXF;

  const StepParams<T> &p = P.s;
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  T *u2 = level<T>(p.u2, t);
  const T *__restrict__ u1 = level<T>(p.u1, t);
  const int lev1 = level_index(P.level_u1, t), lev0 = level_index(P.level_u0, t);

  const int tid = threadIdx.x, lane = tid & 31;
  const int tq = tid % (BX / 4), ty = tid / (BX / 4);  // the thread's quad along axis 2, its row
  const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY;
  const int xq = x0 + 4 * tq, py = y0 + ty;
  const int N0 = g.n[0], NM = g.n[1], NF = g.n[2];
  const int s0 = g.s[0], sM = g.s[1];
  const int c0 = 1 + blockIdx.z * p.chunk;
  const int c1 = min(N0 - 1, c0 + p.chunk);
  const int dir0 = g.dir & 3, dirM = (g.dir >> 2) & 3, dirF = (g.dir >> 4) & 3;
  const T gg = p.gconst;
  const int lastbox = min(c1 - 1 + R, N0 - 1);

  // plane p's box in slot (p - c0) % NB, stage k's tile and barrier in slot (k - c0) % NT
  const auto box = [&](const int plane) { return ring1 + ((unsigned)(plane - c0) % NB) * BOXF; };
  const auto tile = [&](const int k) { return ring0 + ((unsigned)(k - c0) % NT) * TILEF; };
  const auto parity = [&](const int k) { return ((unsigned)(k - c0) / NT) & 1u; };
  // stage k: the box of plane k + R (while there is one) and the tile of plane k
  const auto issue = [&](const int k) {
    const unsigned s = (unsigned)(k - c0) % NT;
    last[s] = k;
    const bool boxed = k + R <= lastbox;
    mbar_expect(&stage_bar[s], (boxed ? WB * HB * (int)sizeof(T) : 0) +
                                   S::TILE_BYTES * (DERIVE ? 1 : 2));
    if (boxed)
      tma_load_4d(box(k + R), &P.map_u1, &stage_bar[s], x0 - H, y0 - R, k + R, lev1);
    T *dst = tile(k);
    tma_load_4d(dst, &P.map_u0, &stage_bar[s], x0, y0, k, lev0);
    if (!DERIVE)
      tma_load_3d(dst + BX * BY, &P.map_minv, &stage_bar[s], x0, y0, k);
  };

  if (tid == 0) {
    for (int i = 0; i < NT; ++i) {
      mbar_init(&stage_bar[i], 1);
      done[i] = 0;
      last[i] = -1;
    }
    mbar_init(&first_bar, 1);
    fence_barrier_init();
    prefetch_map(&P.map_u1);
    prefetch_map(&P.map_u0);
    if (!DERIVE)
      prefetch_map(&P.map_minv);
  }
  __syncthreads();
  const int first_end = min(c0 + R - 1, lastbox);  // the first R planes' boxes
  if (tid == 0 && c0 < c1) {
    mbar_expect(&first_bar, (first_end - c0 + 1) * WB * HB * (int)sizeof(T));
    for (int pl = c0; pl <= first_end; ++pl)
      tma_load_4d(box(pl), &P.map_u1, &first_bar, x0 - H, y0 - R, pl, lev1);
    for (int k = c0; k < c0 + NT && k < c1; ++k)
      issue(k);
  }

  // the thread's nodes
  const bool own = c0 < c1 && py >= 1 && py <= NM - 2 && xq + 3 >= 1 && xq <= NF - 2;
  const int e_hi = NF - (xq - H);  // run index of node NF
  const bool fix_lo = xq - H < 0, fix_hi = e_hi <= XR - 1;
  const T slo = (dirF & 1) ? (T)-1 : (T)1, shi = (dirF & 2) ? (T)-1 : (T)1;
  // an interior tile: every thread a whole quad, no wall within the taps' reach; an
  // axis-1 edge: box rows past a wall, read through their mirrors
  const bool interior = x0 - H >= 0 && x0 + BX + H <= NF && y0 - R >= 1 && y0 + BY + R <= NM - 1;
  const bool yedge = y0 - R < 0 || y0 + BY + R > NM;
  const int ccol = 4 * tq + H;  // the thread's first node in a box row
  const int crow = (ty + R) * WB + ccol;
  const int ctile = ty * BX + 4 * tq;
  const long long gcol = (long long)py * sM + xq;
  int inner = 0, xheld = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int px = xq + i;
    if (px < 1 || px > NF - 2)
      continue;
    inner |= 1 << i;
    if (HOLD && held_wall(px, NF, dirF))
      xheld |= 1 << i;
  }
  const bool yheld = HOLD && held_wall(py, NM, dirM);
  const T mi_derived = DERIVE ? (T)1 / p.sconst : (T)0;

  // u^(t-1) at plane b over the quad, through its mirror along axis 0, from global memory
  const auto gquad = [&](const int b) {
    int sg;
    const int m = mirror_node(b, N0, dir0, sg);
    Quad2 v = ldq(u1 + (long long)m * s0 + gcol);
    if (sg < 0) {
      v.lo = make_float2(-v.lo.x, -v.lo.y);
      v.hi = make_float2(-v.hi.x, -v.hi.y);
    }
    return v;
  };

  float2 w2[R];
#pragma unroll
  for (int k = 0; k < R; ++k)
    w2[k] = p_splat(p.w[k]);
  const float2 g2 = p_splat(gg), ng2 = p_splat(-gg);
  const float2 f0 = p_splat(p.f[0]), f1 = p_splat(p.f[1]), f2 = p_splat(p.f[2]);

  // the queue q[k] = u(z - R + 1 + k), k < 2R (what D+ at plane z reads), and -g * D+
  // of the plane before (its g * D- negated: -(a b) = a (-b) exactly); D+ at plane
  // c0 - 1 also reads u(c0 - R)
  Quad2 q[2 * R];
  float2 npz[2];
  if (own) {
    const Quad2 first = gquad(c0 - R);
#pragma unroll
    for (int k = 0; k < 2 * R - 1; ++k)
      q[k] = gquad(c0 - R + 1 + k);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const auto tap = [&](const int j) { return j == -R + 1 ? first[h] : q[R - 2 + j][h]; };
      npz[h] = p_mul(p_dplus<R>(tap, tap(0), w2), ng2);
    }
  }

  // One plane of the thread's quad. EDGE: the tile meets a wall (the checks of partial
  // quads, mirrors and held wall nodes); SPECIAL: an axis-0 pml slab plane, a held wall
  // plane or a feed past the last plane (what an ordinary plane never meets).
  const auto plane = [&](auto edge_c, auto special_c, const int z) {
    constexpr bool EDGE = decltype(edge_c)::value, SPECIAL = decltype(special_c)::value;
    const int feed = z + R;
    const T *cb = box(z);
    const T *tz = tile(z);
    if (!SPECIAL || feed <= N0 - 1)
      q[2 * R - 1] = ldq(box(feed) + crow);
    else
      q[2 * R - 1] = gquad(feed);

    // the row's run along axis 2, mirrored past the walls
    T xr[XR];
#pragma unroll
    for (int k = 0; k < XR / 4; ++k) {
      const float4 v = *reinterpret_cast<const float4 *>(cb + crow - H + 4 * k);
      xr[4 * k] = v.x, xr[4 * k + 1] = v.y, xr[4 * k + 2] = v.z, xr[4 * k + 3] = v.w;
    }
    if constexpr (EDGE) {
      if (fix_lo)
        mirror_run_lo<T, XR, H>(xr, slo);
      if (fix_hi) {
        switch (e_hi) {
        case H + 2: mirror_run_hi<T, XR, H + 2>(xr, shi); break;
        case H + 3: mirror_run_hi<T, XR, H + 3>(xr, shi); break;
        case H + 4: mirror_run_hi<T, XR, H + 4>(xr, shi); break;
        case H + 5: mirror_run_hi<T, XR, H + 5>(xr, shi); break;
        case H + 6: mirror_run_hi<T, XR, H + 6>(xr, shi); break;
        case H + 7: mirror_run_hi<T, XR, H + 7>(xr, shi); break;
        default: break;
        }
      }
    }
    Quad2 uc;
    uc.lo = make_float2(xr[H], xr[H + 1]);
    uc.hi = make_float2(xr[H + 2], xr[H + 3]);

    // axis 2: D+ at faces x0 - 1 .. x0 + 3, then g D+ - g D- per node
    T dx[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const auto tap = [&](const int k) { return xr[H - 1 + j + k]; };
      dx[j] = dplus<T, R>(tap, xr[H - 1 + j], p.w);
    }
    T ndx[5];
#pragma unroll
    for (int j = 0; j < 5; ++j)
      ndx[j] = mul_rn(dx[j], -gg);
    Quad2 v;
    v.lo = make_float2(fma_rn(dx[1], gg, ndx[0]), fma_rn(dx[2], gg, ndx[1]));
    v.hi = make_float2(fma_rn(dx[3], gg, ndx[2]), fma_rn(dx[4], gg, ndx[3]));

    // axis 1: rows +k and -k of the box, through the mirrored row in an edge tile
    Quad2 rp[R + 1], rm[R + 1];
    rp[0] = rm[0] = uc;
    const auto yrow = [&](const int b) {
      int sg;
      const int my = mirror_node(b, NM, dirM, sg);
      const int ly = my - (y0 - R);
      Quad2 r{make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
      if (my >= 0 && my <= NM - 1 && ly >= 0 && ly < HB) {
        r = ldq(cb + ly * WB + ccol);
        if (sg < 0) {
          r.lo = make_float2(-r.lo.x, -r.lo.y);
          r.hi = make_float2(-r.hi.x, -r.hi.y);
        }
      }
      return r;
    };
#pragma unroll
    for (int k = 1; k <= R; ++k) {
      if (!EDGE || !yedge) {
        rp[k] = ldq(cb + crow + k * WB);
        rm[k] = ldq(cb + crow - k * WB);
      } else {
        rp[k] = yrow(py + k);
        rm[k] = yrow(py - k);
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float2 a = p_sub(rp[1][h], uc[h]), b = p_sub(uc[h], rm[1][h]);
      if (R > 1) {
        a = p_mul(w2[0], a);
        b = p_mul(w2[0], b);
      }
#pragma unroll
      for (int k = 2; k <= R; ++k) {
        a = p_fma(w2[k - 1], p_sub(rp[k][h], rm[k - 1][h]), a);
        b = p_fma(w2[k - 1], p_sub(rp[k - 1][h], rm[k][h]), b);
      }
      const float2 ddy = p_fma(a, g2, p_mul(b, ng2));
      // axis 0 from the queue, then the laplacian f2 ddx + (f0 ddz + f1 ddy)
      const auto tap = [&](const int j) { return q[R - 1 + j][h]; };
      const float2 dpz = p_dplus<R>(tap, q[R - 1][h], w2);
      const float2 ddz = p_fma(dpz, g2, npz[h]);
      npz[h] = p_mul(dpz, ng2);
      v[h] = p_fma(f2, v[h], p_fma(f0, ddz, p_mul(f1, ddy)));
    }
    const Quad2 old = ldq(tz + ctile);
    Quad2 mi;
    if constexpr (DERIVE)
      mi.lo = mi.hi = p_splat(mi_derived);
    else
      mi = ldq(tz + BX * BY + ctile);
    const long long row = (long long)z * s0 + gcol;

    if constexpr (!DAMP) {
      // -u^(t-2) + 2 u^(t-1) + (1/m) lap, as (2u - u0) + (1/m) lap. The product is taken
      // lane by lane: ptxas fuses a packed product into the packed sum it feeds (an FMA,
      // rounded once), which the reference does not do.
#pragma unroll
      for (int h = 0; h < 2; ++h)
        v[h] = p_add(p_sub(p_add(uc[h], uc[h]), old[h]),
                     make_float2(__fmul_rn(mi[h].x, v[h].x), __fmul_rn(mi[h].y, v[h].y)));
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const T m_i = lane_of(mi, i);
        const T dmp = ((inner >> i) & 1) ? p.damping[row + i] : (T)0;
        const T beta = (T)0.5 * m_i * dmp * p.dt;
        set_lane(v, i, ((T)2 * lane_of(uc, i) - lane_of(old, i) * ((T)1 - beta) + m_i * lane_of(v, i)) /
                           ((T)1 + beta));
      }
    }
    // Dirichlet wall nodes hold zero
    int held = 0;
    if constexpr (HOLD && (EDGE || SPECIAL)) {
      const bool zheld = held_wall(z, N0, dir0);
      held = EDGE ? ((yheld || zheld) ? inner : xheld) : (zheld ? 15 : 0);
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if ((held >> i) & 1)
          set_lane(v, i, (T)0);
    }
    if constexpr (SPECIAL) {
      const int zrow = (p.flags & K_PML) ? slab_row(z, N0, g.lo[0], g.hi[0]) : -1;
      if (zrow >= 0) {
        // an axis-0 slab row: the plane's pml memory (pml_kernel's axis 0), its taps from
        // the queue and the one plane the queue no longer holds
        const Quad2 lastq = gquad(z - R);
        T Dpu[4], Dmu[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const auto tap = [&](const int j) {
            return j == -R ? lane_of(lastq, i) : lane_of(q[R - 1 + j], i);
          };
          diffs_plain<T, R>(tap, lane_of(uc, i), p.w, Dpu[i], Dmu[i]);
        }
        const T *prof = p.prof[0];
        const T an = prof[z], bn = prof[N0 + z];
        const T ah = prof[2 * N0 + z], bh = prof[3 * N0 + z];
        const T ah1 = prof[2 * N0 + z - 1], bh1 = prof[3 * N0 + z - 1];
        const T f = p.f[0];
        T *aux = p.aux[0];
        const long long sz = p.auxrow[0];
        T *m = aux + ((long long)zrow * NM + py) * g.ext[2] + xq;
        T m0[4], m1[4], m2[4];
        if (!EDGE || inner == 15) {
          ld4(m0, m), ld4(m1, m + sz), ld4(m2, m + 2 * sz);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const bool on = (inner >> i) & 1;
            m0[i] = on ? m[i] : (T)0;
            m1[i] = on ? m[sz + i] : (T)0;
            m2[i] = on ? m[2 * sz + i] : (T)0;
          }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const T pp = bh * m0[i] + ah * Dpu[i];
          const T pm = bh1 * m1[i] + ah1 * Dmu[i];
          const T zz = bn * m2[i] + an * f * (gg * (Dpu[i] + pp) - gg * (Dmu[i] + pm));
          m0[i] = pp;
          m1[i] = pm;
          m2[i] = zz;
          if (!((held >> i) & 1))
            set_lane(v, i, lane_of(v, i) + lane_of(mi, i) * (f * (gg * pp - gg * pm) + zz));
        }
        if (!EDGE || inner == 15) {
          st4(m, m0), st4(m + sz, m1), st4(m + 2 * sz, m2);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if ((inner >> i) & 1) {
              m[i] = m0[i];
              m[sz + i] = m1[i];
              m[2 * sz + i] = m2[i];
            }
        }
      }
    }
    if (!EDGE || inner == 15) {
      stq(u2 + row, v);
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if ((inner >> i) & 1)
          u2[row + i] = lane_of(v, i);
    }
#pragma unroll
    for (int k = 0; k < 2 * R - 1; ++k)
      q[k] = q[k + 1];
  };

  // a plane is special where it lines the pml along axis 0, holds its wall nodes or
  // feeds the queue past the last plane
  const int lo0 = (p.flags & K_PML) ? g.lo[0] : 0, hi0 = (p.flags & K_PML) ? g.hi[0] : 0;
  const auto special = [&](const int z) {
    return z <= lo0 || z >= N0 - 1 - hi0 || z + R > N0 - 1 || (HOLD && held_wall(z, N0, dir0));
  };
  const auto march = [&](auto edge_c) {
    constexpr bool EDGE = decltype(edge_c)::value;
    if (!warp_wait(&first_bar, 0u))
      return false;
    for (int z = c0; z < c1; ++z) {
      if (!warp_wait(&stage_bar[(unsigned)(z - c0) % NT], parity(z)))
        return false;
      if (!EDGE || own) {
        if (special(z))
          plane(std::integral_constant<bool, EDGE>{}, std::true_type{}, z);
        else
          plane(std::integral_constant<bool, EDGE>{}, std::false_type{}, z);
      }
      // this warp is done with stage z's box and tile; the last warp out issues the
      // stage NT planes on into the same slots
      __syncwarp();
      if (lane == 0 && release_stage(&done[(unsigned)(z - c0) % NT], NW) && z + NT < c1) {
        fence_proxy_async();
        issue(z + NT);
      }
    }
    return true;
  };
  if (c0 < c1) {
    const bool ok = interior ? march(std::false_type{}) : march(std::true_type{});
    if (!ok && lane == 0)
      atomicExch(P.err, 1);
  }
  // no copy may still be writing into the ring when the block leaves: wait (bounded)
  // for the last stage issued on every barrier, which the march consumed unless it
  // broke off
  __syncthreads();
  if (tid == 0 && c0 < c1) {
    mbar_wait(&first_bar, 0u);
    for (int i = 0; i < NT; ++i)
      if (last[i] >= 0)
        mbar_wait(&stage_bar[i], parity(last[i]));
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

}  // namespace cwb
