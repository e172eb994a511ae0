/*
 * CPU ORACLE -- test infrastructure, not the product. Only tests/, the smoke check and
 * bench.py's cpu_baseline leg load it, and only as the checker.
 *
 * A plain-C restatement of cmpmech/cuwave's scalar-wave kernels, one function per
 * kernel launch, looping over the nodes the launch's threads cover. Included twice by
 * oracle.c with REAL = float / double and SFX = _f32 / _f64. Arithmetic follows the
 * reference's expression order; the library is built with -ffp-contract=off, as the
 * reference's host fallback is (cuwave/cpu.py), and FMA_RN / MUL_RN map to fma and a
 * plain product (cuwave/kernels/cpu.hpp:36-39).
 *
 * Geometry: fields are C-contiguous over (n[0], .., ext[ndim-1]), the last axis padded
 * to a multiple of 32 (cuwave/wave.py:120-122); s[] are the strides. A lined axis d
 * keeps its pml memory over its lo + hi slab rows, laid out as the grid with axis d
 * replaced by the rows (row r < lo is node 1 + r, row lo + k node n - 1 - hi + k).
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

static inline REAL FN(fma_r)(REAL a, REAL b, REAL c) { return FMAF(a, b, c); }

/* node b past the stored ghost: its mirror about the wall node (common.cuh:50-54) */
static inline int FN(mirror_node)(int b, int N, int odd, int *sign) {
  *sign = ((b < 0 && (odd & 1)) || (b > N - 1 && (odd & 2))) ? -1 : 1;
  return b < 0 ? 2 - b : (b > N - 1 ? 2 * (N - 2) - b : b);
}

/* node b past the wall node: its image (common.cuh:73-77) */
static inline int FN(node_image)(int b, int N, int odd, int *sign) {
  *sign = ((b < 1 && (odd & 1)) || (b > N - 2 && (odd & 2))) ? -1 : 1;
  return b < 1 ? 2 - b : (b > N - 2 ? 2 * (N - 2) - b : b);
}

static inline int FN(held_wall)(int a, int N, int odd) {
  return ((odd & 1) && a == 1) || ((odd & 2) && a == N - 2);
}

/* u at node a + j along axis d from idx, read through mirror_node (common.cuh:62-69) */
static inline REAL FN(mirrored)(const REAL *u, long idx, const orc_geo *g, int d, int a,
                                int j) {
  int sign;
  int odd = (g->dir >> (2 * d)) & 3;
  int b = FN(mirror_node)(a + j, g->n[d], odd, &sign);
  REAL v = u[idx + (long)(b - a) * g->s[d]];
  return sign > 0 ? v : -v;
}

/* a field at node a + j through node_image, zero on a held node when odd
 * (reflected, scalar_sensitivity.cu:177-184) */
static inline REAL FN(reflected)(const REAL *u, long idx, const orc_geo *g, int d, int a,
                                 int j, int odd) {
  int sign;
  int b = FN(node_image)(a + j, g->n[d], odd, &sign);
  if (FN(held_wall)(b, g->n[d], odd))
    sign = 0;
  REAL v = u[idx + (long)(b - a) * g->s[d]];
  return sign > 0 ? v : (sign < 0 ? -v : (REAL)0);
}

/* node coordinates of flat index idx */
static inline void FN(coords)(const orc_geo *g, long idx, int *A) {
  long rest = idx;
  for (int d = 0; d < g->ndim; ++d) {
    A[d] = (int)(rest / g->s[d]);
    rest -= (long)A[d] * g->s[d];
  }
}

static inline int FN(interior)(const orc_geo *g, const int *A) {
  for (int d = 0; d < g->ndim; ++d)
    if (A[d] < 1 || A[d] > g->n[d] - 2)
      return 0;
  return 1;
}

static inline int FN(held_node)(const orc_geo *g, const int *A) {
  int held = 0;
  for (int d = 0; d < g->ndim; ++d)
    held |= FN(held_wall)(A[d], g->n[d], (g->dir >> (2 * d)) & 3);
  return held;
}

static inline long FN(total)(const orc_geo *g) {
  long t = 1;
  for (int d = 0; d < g->ndim; ++d)
    t *= g->ext[d];
  return t;
}

/* ---------------------------------------------------------------- forward step */
/* flux_divergence_axis + flux_divergence_taps (scalar.cu:15-65): every tap through
 * its mirror (the in-place read of a deep slow axis reads the same values) */
static REAL FN(flux_axis)(const orc_geo *g, const REAL *w, const REAL *u1,
                          const REAL *stiff, long idx, int d, int a, REAL uc, REAL sc) {
  const int R = g->R;
  REAL taps[2 * 8 + 1];
  for (int j = -R; j <= R; ++j)
    taps[j + R] = FN(mirrored)(u1, idx, g, d, a, j);
  const REAL sp = stiff[idx + g->s[d]], sm = stiff[idx - g->s[d]];
  const REAL gp = sc * sp / (sc + sp), gm = sc * sm / (sc + sm);
  REAL Dp = taps[R + 1] - uc, Dm = uc - taps[R - 1];
  if (R > 1) {
    Dp = w[0] * Dp;
    Dm = w[0] * Dm;
  }
  for (int k = 2; k <= R; ++k) {
    Dp = FN(fma_r)(w[k - 1], taps[R + k] - taps[R + 1 - k], Dp);
    Dm = FN(fma_r)(w[k - 1], taps[R + k - 1] - taps[R - k], Dm);
  }
  return (REAL)1 * FN(fma_r)(Dp, gp, -(Dm * gm));
}

/* fd_kernel, per-thread form (scalar.cu:347-496), damping when `damping` is set */
void FN(orc_step)(const orc_geo *g, const REAL *w, const REAL *f, REAL dt, const REAL *u0,
                  const REAL *u1, REAL *u2, const REAL *stiff, const REAL *minv,
                  const REAL *damping, int derive) {
  const long total = FN(total)(g);
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < total; ++idx) {
    int A[3];
    FN(coords)(g, idx, A);
    if (!FN(interior)(g, A))
      continue;
    const REAL uc = u1[idx], sc = stiff[idx];
    REAL lap;
    if (g->ndim == 2) {
      const REAL d0 = FN(flux_axis)(g, w, u1, stiff, idx, 0, A[0], uc, sc);
      const REAL d1 = FN(flux_axis)(g, w, u1, stiff, idx, 1, A[1], uc, sc);
      lap = g->R == 1 ? FN(fma_r)(f[0], d0, f[1] * d1) : FN(fma_r)(f[1], d1, f[0] * d0);
    } else {
      const REAL d0 = FN(flux_axis)(g, w, u1, stiff, idx, 0, A[0], uc, sc);
      const REAL d1 = FN(flux_axis)(g, w, u1, stiff, idx, 1, A[1], uc, sc);
      const REAL d2 = FN(flux_axis)(g, w, u1, stiff, idx, 2, A[2], uc, sc);
      lap = FN(fma_r)(f[2], d2, FN(fma_r)(f[0], d0, f[1] * d1));
    }
    const REAL mi = derive ? (REAL)1 / sc : minv[idx];
    REAL v;
    if (damping) {
      const REAL beta = (REAL)0.5 * mi * damping[idx] * dt;
      v = ((REAL)2 * uc - u0[idx] * ((REAL)1 - beta) + mi * lap) / ((REAL)1 + beta);
    } else {
      v = -u0[idx] + (REAL)2 * uc + mi * lap;
    }
    if (FN(held_node)(g, A))
      v = 0;
    u2[idx] = v;
  }
}

/* flux_divergence_cells (scalar.cu:86-118): one axis with each cell at its own radius,
 * taps as stored; table row r - 1 holds OP_W(r, 1..r), 7 marks a cell onto a held node */
static REAL FN(cells_axis)(const orc_geo *g, const REAL *table, const REAL *u1,
                           const REAL *stiff, long idx, long s, REAL uc, REAL sc, REAL f,
                           int rp, int rm) {
  const int R = g->R;
  REAL Dp = 0, Dm = 0;
  if (rp == 7) {
    Dp = -uc * sc;
  } else if (rp) {
    const REAL sp = stiff[idx + s];
    const REAL *w = table + (rp - 1) * R;
    Dp = w[0] * (u1[idx + s] - uc);
    for (int k = 2; k <= rp; ++k)
      Dp += w[k - 1] * (u1[idx + k * s] - u1[idx - (k - 1) * s]);
    Dp *= sc * sp / (sc + sp);
  }
  if (rm == 7) {
    Dm = uc * sc;
  } else if (rm) {
    const REAL sm = stiff[idx - s];
    const REAL *w = table + (rm - 1) * R;
    Dm = w[0] * (uc - u1[idx - s]);
    for (int k = 2; k <= rm; ++k)
      Dm += w[k - 1] * (u1[idx + (k - 1) * s] - u1[idx - k * s]);
    Dm *= sc * sm / (sc + sm);
  }
  return f * (Dp - Dm);
}

/* fd_kernel under USE_DOMAIN (scalar.cu:434-452): a node of code 0 is not written, a
 * node by a wall (code without bit 30) takes wall_laplacian (scalar.cu:131-158) */
void FN(orc_step_cells)(const orc_geo *g, const REAL *w, const REAL *f, REAL dt,
                        const REAL *u0, const REAL *u1, REAL *u2, const REAL *stiff,
                        const REAL *minv, const REAL *damping, int derive, const int *cells,
                        const REAL *table) {
  const long total = FN(total)(g);
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < total; ++idx) {
    int A[3];
    FN(coords)(g, idx, A);
    if (!FN(interior)(g, A))
      continue;
    const int code = cells[idx];
    if (!code)
      continue;
    const REAL uc = u1[idx], sc = stiff[idx];
    REAL lap;
    if (g->ndim == 2) {
      const REAL d0 = FN(flux_axis)(g, w, u1, stiff, idx, 0, A[0], uc, sc);
      const REAL d1 = FN(flux_axis)(g, w, u1, stiff, idx, 1, A[1], uc, sc);
      lap = g->R == 1 ? FN(fma_r)(f[0], d0, f[1] * d1) : FN(fma_r)(f[1], d1, f[0] * d0);
    } else {
      const REAL d0 = FN(flux_axis)(g, w, u1, stiff, idx, 0, A[0], uc, sc);
      const REAL d1 = FN(flux_axis)(g, w, u1, stiff, idx, 1, A[1], uc, sc);
      const REAL d2 = FN(flux_axis)(g, w, u1, stiff, idx, 2, A[2], uc, sc);
      lap = FN(fma_r)(f[2], d2, FN(fma_r)(f[0], d0, f[1] * d1));
    }
    if (!(code >> 30)) {
      lap = 0;
      for (int d = 0; d < g->ndim; ++d) {
        const REAL term = FN(cells_axis)(g, table, u1, stiff, idx, g->s[d], uc, sc, f[d],
                                         (code >> (6 * d)) & 7, (code >> (6 * d + 3)) & 7);
        lap = d == 0 ? term : lap + term;
      }
    }
    const REAL mi = derive ? (REAL)1 / sc : minv[idx];
    REAL v;
    if (damping) {
      const REAL beta = (REAL)0.5 * mi * damping[idx] * dt;
      v = ((REAL)2 * uc - u0[idx] * ((REAL)1 - beta) + mi * lap) / ((REAL)1 + beta);
    } else {
      v = -u0[idx] + (REAL)2 * uc + mi * lap;
    }
    if (FN(held_node)(g, A))
      v = 0;
    u2[idx] = v;
  }
}

/* slab row of node a on a lined axis, -1 off the slab */
static inline int FN(slab_row)(int a, int N, int lo, int hi) {
  if (lo && a >= 1 && a <= lo)
    return a - 1;
  if (hi && a >= N - 1 - hi && a <= N - 2)
    return lo + a - (N - 1 - hi);
  return -1;
}

static inline long FN(slab_index)(const orc_geo *g, int d, int r, const int *A) {
  long idx = 0;
  for (int e = 0; e < g->ndim; ++e) {
    const int extent = e == d ? g->lo[d] + g->hi[d] : g->ext[e];
    idx = idx * extent + (e == d ? r : A[e]);
  }
  return idx;
}

long FN(orc_slab_size)(const orc_geo *g, int d) {
  long size = 1;
  for (int e = 0; e < g->ndim; ++e)
    size *= e == d ? g->lo[d] + g->hi[d] : g->ext[e];
  return size;
}

static inline REAL FN(cell_weight)(const orc_geo *g, const int *A) {
  REAL w = 1;
  for (int e = 0; e < g->ndim; ++e)
    if (A[e] == 1 || A[e] == g->n[e] - 2)
      w *= (REAL)0.5;
  return w;
}

/* pml_kernel (scalar.cu:500-532) for lined axis d: aux holds 3 slab rows */
void FN(orc_pml)(const orc_geo *g, const REAL *w, int d, REAL f, const REAL *u1, REAL *u2,
                 const REAL *stiff, const REAL *minv, int derive, REAL *aux,
                 const REAL *profile) {
  const long total = FN(total)(g);
  const int N = g->n[d], lo = g->lo[d], hi = g->hi[d], R = g->R, o = g->s[d];
  const long size = FN(orc_slab_size)(g, d);
  const REAL *an = profile, *bn = profile + N, *ah = profile + 2 * N, *bh = profile + 3 * N;
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < total; ++idx) {
    int A[3];
    FN(coords)(g, idx, A);
    if (!FN(interior)(g, A))
      continue;
    const int a = A[d];
    const int r = FN(slab_row)(a, N, lo, hi);
    if (r < 0)
      continue;
    const long t = FN(slab_index)(g, d, r, A);
    const REAL uc = u1[idx], sc = stiff[idx];
    /* cell_differences (scalar.cu:69-83): products and sums rounded apart */
    REAL Dp = w[0] * (FN(mirrored)(u1, idx, g, d, a, 1) - uc);
    REAL Dm = w[0] * (uc - FN(mirrored)(u1, idx, g, d, a, -1));
    for (int k = 2; k <= R; ++k) {
      Dp += w[k - 1] * (FN(mirrored)(u1, idx, g, d, a, k) -
                        FN(mirrored)(u1, idx, g, d, a, 1 - k));
      Dm += w[k - 1] * (FN(mirrored)(u1, idx, g, d, a, k - 1) -
                        FN(mirrored)(u1, idx, g, d, a, -k));
    }
    const REAL sp = stiff[idx + o], sm = stiff[idx - o];
    const REAL gp = sc * sp / (sc + sp), gm = sc * sm / (sc + sm);
    const REAL pp = bh[a] * aux[t] + ah[a] * Dp;
    const REAL pm = bh[a - 1] * aux[size + t] + ah[a - 1] * Dm;
    const REAL z = bn[a] * aux[2 * size + t] + an[a] * f * (gp * (Dp + pp) - gm * (Dm + pm));
    aux[t] = pp;
    aux[size + t] = pm;
    aux[2 * size + t] = z;
    const REAL mi = derive ? (REAL)1 / sc : minv[idx];
    if (!FN(held_node)(g, A))
      u2[idx] += mi * (f * (gp * pp - gm * pm) + z);
  }
}

/* excitation_kernel (common.cuh:456-464), in point order */
void FN(orc_excite)(REAL *u, const int *lin, const REAL *weight, const REAL *row, int num) {
  for (int j = 0; j < num; ++j)
    u[lin[j]] += weight[j] * row[j];
}

/* adjoint_excitation_kernel (common.cuh:467-480), in point order */
void FN(orc_load)(REAL *l2, const int *lin, const REAL *weight, const REAL *row, int num,
                  REAL *g_mass, const REAL *u1, REAL mf) {
  for (int j = 0; j < num; ++j) {
    const int n = lin[j];
    const REAL load = weight[j] * row[j];
    l2[n] += load;
    if (g_mass)
      g_mass[n] += -mf * u1[n] * load;
  }
}

void FN(orc_record)(const REAL *u, const int *lin, REAL *row, int num) {
  for (int j = 0; j < num; ++j)
    row[j] = u[lin[j]];
}

void FN(orc_replay)(REAL *u, const int *lin, const REAL *row, int num) {
  for (int j = 0; j < num; ++j)
    u[lin[j]] = row[j];
}

/* homogeneous_neumann_kernel / homogeneous_dirichlet_kernel (scalar.cu:535-555):
 * the Neumann faces first, then the Dirichlet ones, as two launches */
void FN(orc_refill)(const orc_geo *g, REAL *u, int neumann, int dirichlet) {
  for (int pass = 0; pass < 2; ++pass) {
    const int faces = pass == 0 ? neumann : dirichlet;
    for (int d = 0; d < g->ndim; ++d)
      for (int side = 0; side < 2; ++side) {
        if (!((faces >> (2 * d + side)) & 1))
          continue;
        long count = 1;
        for (int e = 0; e < g->ndim; ++e)
          if (e != d)
            count *= g->n[e] - 2;
        for (long k = 0; k < count; ++k) {
          long rest = k, off = 0;
          for (int e = g->ndim - 1; e >= 0; --e)
            if (e != d) {
              off += (rest % (g->n[e] - 2) + 1) * g->s[e];
              rest /= g->n[e] - 2;
            }
          const long ghost = off + (long)(side ? g->n[d] - 1 : 0) * g->s[d];
          const long normal = side ? -g->s[d] : g->s[d];
          if (pass == 0) {
            u[ghost] = u[ghost + 2 * normal];
          } else {
            u[ghost] = -u[ghost + 2 * normal];
            u[ghost + normal] = 0;
          }
        }
      }
  }
}

/* ---------------------------------------------------------------- adjoint */
/* stiffness_gradient_taps on reflected taps (scalar_sensitivity.cu:119-135, 188-203) */
static REAL FN(stiff_density)(const orc_geo *g, const REAL *w, const REAL *u1,
                              const REAL *l1, const REAL *stiff, long idx, int d, int a,
                              REAL uc, REAL lc, REAL sc, REAL factor) {
  const int R = g->R, odd = (g->dir >> (2 * d)) & 3;
#define U_(j) FN(reflected)(u1, idx, g, d, a, (j), odd)
#define L_(j) FN(reflected)(l1, idx, g, d, a, (j), odd)
#define K_(j) FN(reflected)(stiff, idx, g, d, a, (j), 0)
  const REAL sp = K_(1), sm = K_(-1);
  const REAL dgp = sp * sp / ((sc + sp) * (sc + sp));
  const REAL dgm = sm * sm / ((sc + sm) * (sc + sm));
  REAL Dp = w[0] * (U_(1) - uc);
  REAL Dm = w[0] * (uc - U_(-1));
  for (int j = 2; j <= R; ++j) {
    Dp += w[j - 1] * (U_(j) - U_(1 - j));
    Dm += w[j - 1] * (U_(j - 1) - U_(-j));
  }
  return factor * (dgp * Dp * (L_(1) - lc) + dgm * Dm * (lc - L_(-1)));
}

/* transposed_divergence_taps on reflected taps (scalar_sensitivity.cu:140-154) */
static REAL FN(transposed_div)(const orc_geo *g, const REAL *w, const REAL *l1,
                               const REAL *stiff, long idx, int d, int a, REAL lc, REAL sc) {
  const int R = g->R, odd = (g->dir >> (2 * d)) & 3;
  REAL div = 0, sh = sc, sl = sc, lh = lc, ll = lc;
  for (int j = 1; j <= R; ++j) {
    const REAL sh1 = K_(j), sl1 = K_(-j);
    const REAL lh1 = L_(j), ll1 = L_(-j);
    div += w[j - 1] * (sh * sh1 / (sh + sh1) * (lh1 - lh) - sl * sl1 / (sl + sl1) * (ll - ll1));
    sh = sh1;
    sl = sl1;
    lh = lh1;
    ll = ll1;
  }
  return div;
#undef U_
#undef L_
#undef K_
}

/* adjoint_gradient_kernel (grad != 0) or adjoint_kernel (grad == 0)
 * (scalar_sensitivity.cu:388-515); l2 may be l0 */
void FN(orc_adjoint)(const orc_geo *g, const REAL *w, const REAL *f, REAL dt, const REAL *l0,
                     const REAL *l1, REAL *l2, const REAL *u1, REAL *g_mass, REAL *g_stiff,
                     const REAL *stiff, const REAL *minv, const REAL *damping, int derive,
                     REAL mf, int grad) {
  const long total = FN(total)(g);
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < total; ++idx) {
    int A[3];
    FN(coords)(g, idx, A);
    if (!FN(interior)(g, A))
      continue;
    const REAL lc = l1[idx], sc = stiff[idx], lo = l0[idx];
    const REAL uc = grad ? u1[idx] : 0;
    const REAL mi = derive ? (REAL)1 / sc : minv[idx];
    const int held = FN(held_node)(g, A);
    const REAL lw = held ? (REAL)0 : lc;
    REAL div_l = 0, gs = 0;
    for (int d = 0; d < g->ndim; ++d) {
      div_l += f[d] * FN(transposed_div)(g, w, l1, stiff, idx, d, A[d], lc, sc);
      if (grad)
        gs += FN(stiff_density)(g, w, u1, l1, stiff, idx, d, A[d], uc, lw, sc, f[d]);
    }
    REAL ln;
    if (damping) {
      const REAL beta = (REAL)0.5 * mi * damping[idx] * dt;
      ln = ((REAL)2 * lc - lo * ((REAL)1 - beta) + mi * div_l) / ((REAL)1 + beta);
    } else {
      ln = -lo + (REAL)2 * lc + mi * div_l;
    }
    if (held)
      ln = 0;
    if (grad) {
      const REAL gm = g_mass[idx], gsum = g_stiff[idx];
      g_mass[idx] = gm - mf * uc * (ln - (REAL)2 * lc + lo);
      g_stiff[idx] = gsum - mf * gs;
    }
    l2[idx] = ln;
  }
}

/* gradient_kernel (scalar_sensitivity.cu:303-350): F are f_d / dt^2 */
void FN(orc_gradient)(const orc_geo *g, const REAL *w, const REAL *F, const REAL *u0,
                      const REAL *u1, const REAL *u2, const REAL *l1, REAL *g_mass,
                      REAL *g_stiff, const REAL *stiff, REAL inv_dt2) {
  const long total = FN(total)(g);
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < total; ++idx) {
    int A[3];
    FN(coords)(g, idx, A);
    if (!FN(interior)(g, A))
      continue;
    const REAL uc = u1[idx], lc = l1[idx];
    g_mass[idx] -= inv_dt2 * lc * (u2[idx] - (REAL)2 * uc + u0[idx]);
    const REAL sc = stiff[idx];
    const int held = FN(held_node)(g, A);
    const REAL lw = held ? (REAL)0 : lc;
    REAL gs = 0;
    for (int d = 0; d < g->ndim; ++d)
      gs += FN(stiff_density)(g, w, u1, l1, stiff, idx, d, A[d], uc, lw, sc, F[d]);
    g_stiff[idx] -= gs;
  }
}

/* pml_aux_kernel (scalar_sensitivity.cu:518-542): eta holds 3 slab rows */
void FN(orc_pml_aux)(const orc_geo *g, int d, REAL f, const REAL *l1, const REAL *stiff,
                     REAL *eta, const REAL *profile) {
  const long total = FN(total)(g);
  const int N = g->n[d], lo = g->lo[d], hi = g->hi[d], o = g->s[d];
  const long size = FN(orc_slab_size)(g, d);
  const REAL *an = profile, *bn = profile + N, *bh = profile + 3 * N;
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < total; ++idx) {
    int A[3];
    FN(coords)(g, idx, A);
    if (!FN(interior)(g, A))
      continue;
    const int a = A[d];
    const int r = FN(slab_row)(a, N, lo, hi);
    if (r < 0)
      continue;
    const long t = FN(slab_index)(g, d, r, A);
    const REAL sc = stiff[idx], sp = stiff[idx + o], sm = stiff[idx - o];
    const REAL gp = sc * sp / (sc + sp), gm = sc * sm / (sc + sm);
    const REAL q = FN(held_node)(g, A) ? (REAL)0 : FN(cell_weight)(g, A) * l1[idx];
    const REAL ez = eta[2 * size + t];
    eta[t] = bh[a] * (eta[t] + an[a] * f * gp * ez) + f * gp * q;
    eta[size + t] = bh[a - 1] * (eta[size + t] - an[a] * f * gm * ez) - f * gm * q;
    eta[2 * size + t] = bn[a] * ez + q;
  }
}

/* d(D+)/du_q and d(D-)/du_q (scalar_sensitivity.cu:221-234) */
static inline REAL FN(plus_tap)(const REAL *w, int R, int q) {
  if (q >= 1)
    return q <= R ? w[q - 1] : (REAL)0;
  return 1 - q <= R ? -w[-q] : (REAL)0;
}
static inline REAL FN(minus_tap)(const REAL *w, int R, int q) {
  if (q >= 0)
    return q + 1 <= R ? w[q] : (REAL)0;
  return -q <= R ? -w[-q - 1] : (REAL)0;
}

/* pml_tap (scalar_sensitivity.cu:237-251) of the slab node at row ai of node A's line */
static REAL FN(pml_tap)(const orc_geo *g, const REAL *w, int d, REAL f, const REAL *eta,
                        const REAL *stiff, const REAL *profile, const int *A, int ai, int q) {
  const int N = g->n[d], o = g->s[d];
  const long size = FN(orc_slab_size)(g, d);
  int B[3] = {A[0], A[1], A[2]};
  B[d] = ai;
  const int r = FN(slab_row)(ai, N, g->lo[d], g->hi[d]);
  const long i = FN(slab_index)(g, d, r, B);
  long iidx = 0;
  for (int e = 0; e < g->ndim; ++e)
    iidx += (long)B[e] * g->s[e];
  const REAL *an = profile, *ah = profile + 2 * N;
  const REAL sc = stiff[iidx], sp = stiff[iidx + o], sm = stiff[iidx - o];
  const REAL gp = sc * sp / (sc + sp), gm = sc * sm / (sc + sm);
  const REAL ez = an[ai] * f * eta[2 * size + i];
  const REAL cp = ah[ai] * eta[i] + gp * (1 + ah[ai]) * ez;
  const REAL cm = ah[ai - 1] * eta[size + i] - gm * (1 + ah[ai - 1]) * ez;
  return cp * FN(plus_tap)(w, g->R, q) + cm * FN(minus_tap)(w, g->R, q);
}

/* pml_adjoint_kernel (scalar_sensitivity.cu:545-597) */
void FN(orc_pml_adjoint)(const orc_geo *g, const REAL *w, int d, REAL f, REAL *l2,
                         REAL *g_mass, const REAL *u1, REAL mf, int with_mass,
                         const REAL *stiff, const REAL *minv, int derive, const REAL *eta,
                         const REAL *profile) {
  const long total = FN(total)(g);
  const int N = g->n[d], lo = g->lo[d], hi = g->hi[d], R = g->R;
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < total; ++idx) {
    int A[3];
    FN(coords)(g, idx, A);
    if (!FN(interior)(g, A))
      continue;
    const int a = A[d];
    const int reached = (lo && a >= 1 && a <= lo + R) || (hi && a <= N - 2 && a >= N - 1 - (hi + R));
    if (!reached)
      continue;
    REAL sum = 0;
    for (int m = -R; m <= R; ++m)
      if (FN(slab_row)(a + m, N, lo, hi) >= 0)
        sum += FN(pml_tap)(g, w, d, f, eta, stiff, profile, A, a + m, -m);
    for (int high = 0; high < 2; ++high) {
      const int ghost = high ? 2 * (N - 2) - a : 2 - a;
      if (high ? ghost < N - 1 : ghost > 0)
        continue;
      REAL fold = 0;
      for (int k = 1; k <= R; ++k) {
        const int ai = high ? N - 1 - k : k;
        if (FN(slab_row)(ai, N, lo, hi) >= 0 && ghost - ai >= -R && ghost - ai <= R)
          fold += FN(pml_tap)(g, w, d, f, eta, stiff, profile, A, ai, ghost - ai);
      }
      sum += ((g->dir >> (2 * d + high)) & 1) ? -fold : fold;
    }
    const REAL mi = derive ? (REAL)1 / stiff[idx] : minv[idx];
    const REAL delta = mi * sum / FN(cell_weight)(g, A);
    l2[idx] += delta;
    if (with_mass)
      g_mass[idx] -= mf * u1[idx] * delta;
  }
}
