// The 3D forward step of a uniform stiffness, register-blocked over TMA-staged planes.
//
// A block of 256 threads owns a 64 x 16 tile of the (axis-1, axis-2) plane and marches a
// chunk of planes along axis 0. Each thread steps four consecutive axis-2 nodes of one
// axis-1 row, so every tap it reads is a 16-byte row of four values.
//
//   * Axis 0 (the march) keeps, per node, the 2R values u(z-R+1) .. u(z+R) in a
//     register queue fed one plane ahead from the staged planes, and carries g * D+ of
//     the plane before as this plane's g * D- (the two are the same expression of the
//     same values, so the reuse is bit-exact).
//   * Axis 2 (fast) reads the row's 4 + 2H values once and forms D+ at the five faces
//     x0 - 1 .. x0 + 3, each face's D+ serving as the next node's D-.
//   * Axis 1 reads 2R rows of four from the staged box.
//
// One elected thread issues, per plane, a tensor-map copy of u^(t-1) over the tile and an
// R-wide halo into a ring of R + 1 + PREFETCH boxes (the planes the axis-1/2 taps and the
// queue's feed reach), and a copy of u^(t-2) and 1/m over the tile into a second ring.
// Values past a wall take their mirrors (cuwave common.cuh:50-69): along axis 2 in the
// row's registers, along axis 1 in the box rows past the wall (edge tiles only), along
// axis 0 by reading the mirror plane from global memory at the chunk's ends.
//
// The node arithmetic is step.cuh's (cuwave fd_kernel, scalar.cu:347-427) in the same
// order, Dirichlet wall nodes held at zero. An axis-0 pml slab row is a whole plane of
// the march, so its memory terms (pml_kernel's axis 0) are applied here, uniformly over
// the plane; those of axes 1 and 2 (pml.cuh), the sources and the ghost refill follow as
// launches of their own, in the order of cuwave's step, so no quad branches apart from
// the others of its plane. Every wait on a copy is bounded
// (tma.cuh): a lost copy raises the launch's error flag, the block drains what it issued
// and leaves.
#pragma once

#include <type_traits>

#include "step_tma.cuh"  // level_index, the pinned differences, the copies

namespace cwb {

constexpr int S3_BX = 64, S3_BY = 16, S3_THREADS = 256;

template <typename T, int R, int PF = 3>
struct Step3Shape {
  static constexpr int V = 16 / (int)sizeof(T);            // values per 16-byte row
  static constexpr int H = (R + V - 1) / V * V;             // axis-2 halo, whole 16-byte rows
  static constexpr int WB = S3_BX + 2 * H;                  // box width
  static constexpr int HB = S3_BY + 2 * R;                  // box height
  static constexpr int PREFETCH = PF;                       // planes issued past the feed
  static constexpr int NS1 = R + 1 + PREFETCH;              // boxes of u^(t-1)
  static constexpr int NS0 = PREFETCH + 1;                  // tiles of u^(t-2) and 1/m
  static constexpr int BOX_BYTES = (WB * HB * (int)sizeof(T) + 127) / 128 * 128;
  static constexpr int TILE_BYTES = S3_BX * S3_BY * (int)sizeof(T);
  static constexpr int RING1 = NS1 * BOX_BYTES;
  static constexpr int SMEM = RING1 + NS0 * 2 * TILE_BYTES + 128;
  static constexpr int XR = 4 + 2 * H;                      // the row's run along axis 2
  // the kernel is built for single precision up to radius 4 (its registers); the host
  // sends other cases to the row kernel
  static constexpr bool SUPPORTED = sizeof(T) == 4 && R <= 4;
};

template <typename T>
struct Step3Params {
  StepParams<T> s;
  CUtensorMap map_u1;    // levels of b: (ext_F, n1, n0, levels), box (WB, HB, 1, 1)
  CUtensorMap map_u0;    // levels of a: box (64, 16, 1, 1)
  CUtensorMap map_minv;  // (ext_F, n1, n0), box (64, 16, 1)
  int level_u1[3];
  int level_u0[3];
  int *err;
  int flow;  // 1: the barrier-free march (step3d_flow.cuh), 0: the per-plane barrier one
};

// four values from 16-byte aligned memory
template <typename T>
__device__ __forceinline__ void ld4(T *dst, const T *src) {
  static_assert(sizeof(T) == 4, "16-byte rows of four");
  const float4 v = *reinterpret_cast<const float4 *>(src);
  dst[0] = v.x, dst[1] = v.y, dst[2] = v.z, dst[3] = v.w;
}

template <typename T>
__device__ __forceinline__ void st4(T *dst, const T *v) {
  static_assert(sizeof(T) == 4, "16-byte rows of four");
  *reinterpret_cast<float4 *>(dst) = make_float4(v[0], v[1], v[2], v[3]);
}

// HOLD: the grid has a Dirichlet face, whose wall nodes the step holds at zero (without
// one, no node is held and the step carries no wall test)
template <typename T, int R, bool UNIF, bool HOLD = true>
__global__ void __launch_bounds__(S3_THREADS, 2)
    step3d_kernel(const __grid_constant__ Step3Params<T> P) {
  using S = Step3Shape<T, R>;
  static_assert(S::SUPPORTED, "the blocked 3D step is built for float up to radius 4");
  static_assert(UNIF, "the blocked 3D step is built for a uniform stiffness");
  constexpr int H = S::H, WB = S::WB, HB = S::HB, NS1 = S::NS1, NS0 = S::NS0, XR = S::XR;
  constexpr int BX = S3_BX, BY = S3_BY;
  extern __shared__ __align__(128) unsigned char s3_smem[];
  __shared__ __align__(8) uint64_t full1[NS1];
  __shared__ __align__(8) uint64_t full0[NS0];
  unsigned char *ring1 = align_smem128(s3_smem);
  unsigned char *ring0 = ring1 + S::RING1;

  const StepParams<T> &p = P.s;
  const Geometry &g = p.g;
  const int t = step_index(p.ctr);
  T *u2 = level<T>(p.u2, t);
  const T *__restrict__ u1 = level<T>(p.u1, t);
  const int lev1 = level_index(P.level_u1, t), lev0 = level_index(P.level_u0, t);

  const int tid = threadIdx.x;
  const int tq = tid % (BX / 4), ty = tid / (BX / 4);  // the thread's quad along axis 2, its row
  const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY;
  const int xq = x0 + 4 * tq, py = y0 + ty;
  const int N0 = g.n[0], NM = g.n[1], NF = g.n[2];
  const int s0 = g.s[0], sM = g.s[1];
  const int c0 = 1 + blockIdx.z * p.chunk;
  const int c1 = min(N0 - 1, c0 + p.chunk);
  const int dir0 = g.dir & 3, dirM = (g.dir >> 2) & 3, dirF = (g.dir >> 4) & 3;
  const int flags = p.flags;
  const bool leader = tid == 0;
  const T gg = p.gconst;

  // ring 1 holds the boxes of planes c0 .. lastbox, ring 0 the tiles of c0 .. c1 - 1
  const int lastbox = min(c1 - 1 + R, N0 - 1);
  const auto box = [&](const int plane) {
    return reinterpret_cast<T *>(ring1 + ((unsigned)(plane - c0) % NS1) * S::BOX_BYTES);
  };
  const auto tile = [&](const int plane) {
    return reinterpret_cast<T *>(ring0 + ((unsigned)(plane - c0) % NS0) * 2 * S::TILE_BYTES);
  };
  const auto parity1 = [&](const int plane) { return ((unsigned)(plane - c0) / NS1) & 1u; };
  const auto parity0 = [&](const int plane) { return ((unsigned)(plane - c0) / NS0) & 1u; };
  int issued1 = c0 - 1, issued0 = c0 - 1, arrived1 = c0 - 1, arrived0 = c0 - 1;
  const auto issue1 = [&](const int plane) {
    issued1 = plane;
    uint64_t *bar = &full1[(unsigned)(plane - c0) % NS1];
    mbar_expect(bar, WB * HB * (int)sizeof(T));
    tma_load_4d(box(plane), &P.map_u1, bar, x0 - H, y0 - R, plane, lev1);
  };
  const auto issue0 = [&](const int plane) {
    issued0 = plane;
    uint64_t *bar = &full0[(unsigned)(plane - c0) % NS0];
    const bool derive = flags & K_DERIVE;
    mbar_expect(bar, S::TILE_BYTES * (derive ? 1 : 2));
    T *dst = tile(plane);
    tma_load_4d(dst, &P.map_u0, bar, x0, y0, plane, lev0);
    if (!derive)
      tma_load_3d(dst + BX * BY, &P.map_minv, bar, x0, y0, plane);
  };

  if (leader) {
    for (int i = 0; i < NS1; ++i)
      mbar_init(&full1[i], 1);
    for (int i = 0; i < NS0; ++i)
      mbar_init(&full0[i], 1);
    fence_barrier_init();
    prefetch_map(&P.map_u1);
    prefetch_map(&P.map_u0);
    if (!(flags & K_DERIVE))
      prefetch_map(&P.map_minv);
  }
  __syncthreads();
  if (leader && c0 < c1) {
    for (int pl = c0; pl < c0 + NS1 - 1 && pl <= lastbox; ++pl)
      issue1(pl);
    for (int pl = c0; pl < c0 + NS0 - 1 && pl < c1; ++pl)
      issue0(pl);
  }

  // box rows past an axis-1 wall take the mirrored rows; cells past both walls are read
  // by no star stencil and are zeroed
  const bool yedge = y0 - R < 0 || y0 + BY + R > NM;
  const int ylo_end = max(0, min(HB, R - y0));
  const int yhi_beg = max(0, min(HB, NM - (y0 - R)));
  const auto yfix = [&](T *b) {
    const int nrows = ylo_end + (HB - yhi_beg);
    for (int c = tid; c < nrows * WB; c += S3_THREADS) {
      const int ri = c / WB, bx = c % WB;
      const int by = ri < ylo_end ? ri : yhi_beg + (ri - ylo_end);
      const int xg = x0 - H + bx, yg = y0 - R + by;
      T v = (T)0;
      if (xg >= 0 && xg <= NF - 1) {
        int sy;
        const int my = mirror_node(yg, NM, dirM, sy);
        const int ly = my - (y0 - R);
        if (my >= 0 && my <= NM - 1 && ly >= 0 && ly < HB) {
          const T m = b[ly * WB + bx];
          v = sy < 0 ? -m : m;
        }
      }
      b[by * WB + bx] = v;
    }
    // these generic-proxy writes precede the copy that later refills the stage
    fence_proxy_async();
  };

  // the thread's nodes
  const bool own = c0 < c1 && py >= 1 && py <= NM - 2 && xq + 3 >= 1 && xq <= NF - 2;
  const bool full_quad = xq >= 1 && xq + 3 <= NF - 2;
  const int e_hi = NF - (xq - H);  // run index of node NF
  const bool fix_lo = xq - H < 0, fix_hi = e_hi <= XR - 1;
  const T slo = (dirF & 1) ? (T)-1 : (T)1, shi = (dirF & 2) ? (T)-1 : (T)1;
  const int crow = (ty + R) * WB + 4 * tq + H;  // the thread's first node in a box
  const int ctile = ty * BX + 4 * tq;           // ... and in a tile
  const long long gcol = (long long)py * sM + xq;
  // u^(t-1) at plane b over the quad, through its mirror along axis 0, from global memory
  const auto gquad = [&](const int b, T *dst) {
    int sg;
    const int m = mirror_node(b, N0, dir0, sg);
    ld4(dst, u1 + (long long)m * s0 + gcol);
    if (sg < 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        dst[i] = -dst[i];
    }
  };

  // the queue q[k] = u(z - R + 1 + k), k < 2R (what D+ at plane z reads), and g * D+
  // of the plane before; D+ at plane c0 - 1 also reads u(c0 - R)
  T q[2 * R][4];
  T pz[4];
  if (own) {
    T first[4];
    gquad(c0 - R, first);
#pragma unroll
    for (int k = 0; k < 2 * R - 1; ++k)
      gquad(c0 - R + 1 + k, q[k]);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const auto tap = [&](const int j) { return j == -R + 1 ? first[i] : q[R - 2 + j][i]; };
      pz[i] = mul_rn(dplus<T, R>(tap, tap(0), p.w), gg);
    }
  }

  // What the thread's nodes meet: Dirichlet wall nodes, which hold zero. The pml memory
  // of axes 1 and 2, the sources and the ghost refill run as launches of their own after
  // this one, in the order of cuwave's step (fd, pml, excitation, refill).
  const bool damp = flags & K_DAMP;
  int inner = 0, xheld = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int px = xq + i;
    if (px < 1 || px > NF - 2)
      continue;
    inner |= 1 << i;
    if (held_wall(px, NF, dirF))
      xheld |= 1 << i;
  }
  const bool yheld = held_wall(py, NM, dirM);
  const T mi_derived = (flags & K_DERIVE) ? (T)1 / p.sconst : (T)0;

  // the boxes of planes c0 .. c0 + R - 1 before the first plane reads them
  bool ok = true;
  if (c0 < c1) {
    bool good = true;
    if (leader)
      for (int pl = c0; pl < c0 + R && pl <= lastbox && good; ++pl) {
        good = mbar_wait(&full1[(unsigned)(pl - c0) % NS1], parity1(pl));
        if (good)
          arrived1 = pl;
      }
    ok = __syncthreads_and(good);
    if (ok && yedge) {
      for (int pl = c0; pl < c0 + R && pl <= lastbox; ++pl)
        yfix(box(pl));
      __syncthreads();
    }
  }

  for (int z = c0; z < c1 && ok; ++z) {
    const int feed = z + R;  // the plane the queue takes in
    bool good = true;
    if (leader) {
      if (feed <= lastbox)
        good = mbar_wait(&full1[(unsigned)(feed - c0) % NS1], parity1(feed));
      if (good)
        good = mbar_wait(&full0[(unsigned)(z - c0) % NS0], parity0(z));
    }
    if (!__syncthreads_and(good)) {
      ok = false;
      break;
    }
    if (feed <= lastbox)
      arrived1 = feed;
    arrived0 = z;
    // every thread is past plane z - 1: its stages take the planes PREFETCH ahead
    if (leader) {
      fence_proxy_async();
      if (z + NS1 - 1 <= lastbox)
        issue1(z + NS1 - 1);
      if (z + NS0 - 1 < c1)
        issue0(z + NS0 - 1);
    }
    // the feed's box is read along axis 1 from plane `feed` on, after barriers to come
    if (yedge && feed <= lastbox)
      yfix(box(feed));
    if (!own)
      continue;

    const int held = !HOLD ? 0 : (yheld || held_wall(z, N0, dir0)) ? inner : xheld;
    const int zrow = (flags & K_PML) ? slab_row(z, N0, g.lo[0], g.hi[0]) : -1;

    const T *cb = box(z);
    if (feed <= N0 - 1)
      ld4(q[2 * R - 1], box(feed) + crow);
    else
      gquad(feed, q[2 * R - 1]);
    // the row's run along axis 2, mirrored past the walls
    const auto load_run = [&](T *xr) {
#pragma unroll
      for (int k = 0; k < XR / 4; ++k)
        ld4(xr + 4 * k, cb + crow - H + 4 * k);
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
    };
    T xr[XR];
    load_run(xr);
    T uc[4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
      uc[i] = xr[H + i];

    // axis 2: D+ at faces x0 - 1 .. x0 + 3
    T dx[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const auto tap = [&](const int k) { return xr[H - 1 + j + k]; };
      dx[j] = dplus<T, R>(tap, xr[H - 1 + j], p.w);
    }
    // axis 1: D+ and D- from rows +k and -k
    T dpy[4], dmy[4];
    {
      T rp[R + 1][4], rm[R + 1][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        rp[0][i] = rm[0][i] = uc[i];
#pragma unroll
      for (int k = 1; k <= R; ++k) {
        ld4(rp[k], cb + crow + k * WB);
        ld4(rm[k], cb + crow - k * WB);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        T a = rp[1][i] - uc[i], b = uc[i] - rm[1][i];
        if (R > 1) {
          a = mul_rn(p.w[0], a);
          b = mul_rn(p.w[0], b);
        }
#pragma unroll
        for (int k = 2; k <= R; ++k) {
          a = fma_rn(p.w[k - 1], rp[k][i] - rm[k - 1][i], a);
          b = fma_rn(p.w[k - 1], rp[k - 1][i] - rm[k][i], b);
        }
        dpy[i] = a;
        dmy[i] = b;
      }
    }
    // axis 0 from the queue; the laplacian
    T lap[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const auto tap = [&](const int j) { return q[R - 1 + j][i]; };
      const T dpz = dplus<T, R>(tap, q[R - 1][i], p.w);
      const T ddz = fma_rn(dpz, gg, -pz[i]);
      pz[i] = mul_rn(dpz, gg);
      const T ddy = fma_rn(dpy[i], gg, -mul_rn(dmy[i], gg));
      const T ddx = fma_rn(dx[i + 1], gg, -mul_rn(dx[i], gg));
      lap[i] = fma_rn(p.f[2], ddx, fma_rn(p.f[0], ddz, mul_rn(p.f[1], ddy)));
    }
    const T *tz = tile(z);
    T old[4], mi[4];
    ld4(old, tz + ctile);
    if (flags & K_DERIVE) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        mi[i] = mi_derived;
    } else {
      ld4(mi, tz + BX * BY + ctile);
    }
    const long long row = (long long)z * s0 + gcol;

    T v[4];
    if (!damp) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        v[i] = -old[i] + (T)2 * uc[i] + mi[i] * lap[i];
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const T dmp = ((inner >> i) & 1) ? p.damping[row + i] : (T)0;
        const T beta = (T)0.5 * mi[i] * dmp * p.dt;
        v[i] = ((T)2 * uc[i] - old[i] * ((T)1 - beta) + mi[i] * lap[i]) / ((T)1 + beta);
      }
    }
    // Dirichlet wall nodes hold zero
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if ((held >> i) & 1)
        v[i] = (T)0;
    if (zrow >= 0) {
      // an axis-0 slab row: the plane's pml memory (pml_kernel's axis 0), its taps from
      // the queue and the one plane the queue no longer holds
      T last[4], Dpu[4], Dmu[4];
      gquad(z - R, last);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const auto tap = [&](const int j) { return j == -R ? last[i] : q[R - 1 + j][i]; };
        diffs_plain<T, R>(tap, uc[i], p.w, Dpu[i], Dmu[i]);
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
      if (inner == 15) {
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
          v[i] += mi[i] * (f * (gg * pp - gg * pm) + zz);
      }
      if (inner == 15) {
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
    if (inner == 15) {
      st4(u2 + row, v);
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if ((inner >> i) & 1)
          u2[row + i] = v[i];
    }
#pragma unroll
    for (int k = 0; k < 2 * R - 1; ++k)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        q[k][i] = q[k + 1][i];
  }
  if (!ok && leader) {
    // a copy never arrived: flag it and drain what is in flight before leaving
    atomicExch(P.err, 1);
    for (int pl = arrived1 + 1; pl <= issued1; ++pl)
      mbar_wait(&full1[(unsigned)(pl - c0) % NS1], parity1(pl));
    for (int pl = arrived0 + 1; pl <= issued0; ++pl)
      mbar_wait(&full0[(unsigned)(pl - c0) % NS0], parity0(pl));
  }
  finish_step(p.ctr, flags & K_ADV);
}

}  // namespace cwb
