// Point transfers, the ghost refill and the adjoint pml memory step.
#pragma once

#include "params.cuh"

namespace cwb {

constexpr int TRANSFER_THREADS = 256;

// float32 rounded to the nearest even bfloat16, as wave.narrow does it
// (cuwave/wave.py:848-853): the high half after adding 0x7FFF plus the kept lsb
__device__ __forceinline__ unsigned short narrow_bf16(const float v) {
  const unsigned bits = __float_as_uint(v);
  return (unsigned short)((bits + 0x7FFFu + ((bits >> 16) & 1u)) >> 16);
}
__device__ __forceinline__ float widen_bf16(const unsigned short b) {
  return __uint_as_float(((unsigned)b) << 16);
}

template <typename T>
__device__ __forceinline__ T record_read(const TransferParams<T> &p, const long long at) {
  if (p.store == 1)
    return (T)widen_bf16(reinterpret_cast<const unsigned short *>(p.record)[at]);
  if (p.store == 2)
    return (T)reinterpret_cast<const float *>(p.record)[at];
  return reinterpret_cast<const T *>(p.record)[at];
}

template <typename T>
__device__ __forceinline__ void record_write(const TransferParams<T> &p, const long long at,
                                             const T v) {
  if (p.store == 1)
    reinterpret_cast<unsigned short *>(p.record)[at] = narrow_bf16((float)v);
  else if (p.store == 2)
    reinterpret_cast<float *>(p.record)[at] = (float)v;
  else
    reinterpret_cast<T *>(p.record)[at] = v;
}

// a[lin] += weight * record[row] (excitation_kernel, cuwave/kernels/common.cuh:456-464)
template <typename T>
__global__ void excite_kernel(const TransferParams<T> p) {
  const int t = step_index(p.ctr);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < p.num) {
    T *a = level<T>(p.a, t);
    const long long row = (long long)p.row_mul * t + p.row_add;
    atomic_add_exact(&a[p.lin[j]], p.weight[j] * record_read(p, row * p.num + j));
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// the adjoint load, and with K_MASS its share of the inertia gradient against c
// (adjoint_excitation_kernel, common.cuh:467-480)
template <typename T>
__global__ void load_kernel(const TransferParams<T> p, T *g_mass) {
  const int t = step_index(p.ctr);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < p.num) {
    T *a = level<T>(p.a, t);
    const long long row = (long long)p.row_mul * t + p.row_add;
    const int n = p.lin[j];
    const T load = p.weight[j] * record_read(p, row * p.num + j);
    atomic_add_exact(&a[n], load);
    if (p.flags & K_MASS) {
      const T *u1 = level<T>(p.c, t);
      atomic_add_exact(&g_mass[n], -p.scale * u1[n] * load);
    }
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// record[row] = a[lin] (get_signal_kernel, common.cuh:483-491)
template <typename T>
__global__ void record_kernel(const TransferParams<T> p) {
  const int t = step_index(p.ctr);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < p.num) {
    const T *a = level<T>(p.a, t);
    const long long row = (long long)p.row_mul * t + p.row_add;
    record_write(p, row * p.num + j, a[p.lin[j]]);
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// a[lin] = record[row] (set_signal_kernel, common.cuh:494-503)
template <typename T>
__global__ void replay_kernel(const TransferParams<T> p) {
  const int t = step_index(p.ctr);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < p.num) {
    T *a = level<T>(p.a, t);
    const long long row = (long long)p.row_mul * t + p.row_add;
    a[p.lin[j]] = record_read(p, row * p.num + j);
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// One thread per face ghost, edges and corners excluded: the ghost takes its mirror
// two nodes in, negated on a Dirichlet face whose wall node is zeroed
// (homogeneous_neumann_kernel / homogeneous_dirichlet_kernel, scalar.cu:535-555).
template <typename T>
__global__ void refill_kernel(const TransferParams<T> p, const int faces) {
  const int t = step_index(p.ctr);
  const Geometry &g = p.g;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  T *u = level<T>(p.a, t);
  for (int d = 0; d < g.ndim; ++d) {
    int face = 1;
    for (int e = 0; e < g.ndim; ++e)
      if (e != d)
        face *= g.n[e] - 2;
    for (int side = 0; side < 2; ++side) {
      if (!((faces >> (2 * d + side)) & 1))
        continue;
      if (k >= 0 && k < face) {
        int rest = k, off = 0;
        for (int e = g.ndim - 1; e >= 0; --e)
          if (e != d) {
            off += (rest % (g.n[e] - 2) + 1) * g.s[e];
            rest /= g.n[e] - 2;
          }
        const int ghost = off + (side ? g.n[d] - 1 : 0) * g.s[d];
        const int normal = side ? -g.s[d] : g.s[d];
        const bool odd = (g.dir >> (2 * d + side)) & 1;
        const T v = u[ghost + 2 * normal];
        u[ghost] = odd ? -v : v;
        if (odd)
          u[ghost + normal] = (T)0;
      }
      k -= face;
    }
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// The same refill on a 3D grid, the faces of axes 0 and 1 a quad of four fast-axis nodes
// a thread (their ghost rows are contiguous along axis 2), those of axis 2 a row a
// thread (both sides): for each face asked, the threads of its (side, row, quad) or
// (plane, row) come one after another on the launch. The values and the nodes written are
// refill_kernel's; a wall node of a Dirichlet face is zeroed as there.
struct Refill3Layout {
  int faces;
  int nq;            // quads covering nodes 0 .. NF - 2 of a row
  long long n0, n1;  // threads of axis 0's faces, of axis 1's (both sides each)
  long long total;
};

// `src`, `rec`: the step's sources and the record op that follows, when neither touches a
// node another thread of the launch reads or writes (no source on a refilled face's
// mirror, no receiver on a ghost, a held wall node or a source): threads past the faces'
// add the sources as excite_kernel would before the refill and read the receivers as
// record_kernel would after it (num 0 where they run as launches of their own)
template <typename T>
__global__ void refill3d_kernel(const TransferParams<T> p, const Refill3Layout lay,
                                const TransferParams<T> src, const TransferParams<T> rec) {
  const int t = step_index(p.ctr);
  const Geometry &g = p.g;
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= lay.total) {
    k -= lay.total;
    if (k < src.num) {
      T *a = level<T>(src.a, t);
      const long long srow = (long long)src.row_mul * t + src.row_add;
      atomic_add_exact(&a[src.lin[k]], src.weight[k] * record_read(src, srow * src.num + k));
    } else if (k - src.num < rec.num) {
      const int j = (int)(k - src.num);
      const T *a = level<T>(rec.a, t);
      const long long rrow = (long long)rec.row_mul * t + rec.row_add;
      record_write(rec, rrow * rec.num + j, a[rec.lin[j]]);
    }
  } else {
    T *u = level<T>(p.a, t);
    const int N0 = g.n[0], NM = g.n[1], NF = g.n[2];
    const long long s0 = g.s[0], s1 = g.s[1];
    if (k < lay.n0 + lay.n1) {
      // a quad of a ghost row of axis 0 or 1: side, the other in-plane index, the quad
      const int d = k < lay.n0 ? 0 : 1;
      if (d == 1)
        k -= lay.n0;
      const int q = (int)(k % lay.nq);
      k /= lay.nq;
      const int other = 1 + (int)(k % (d == 0 ? NM - 2 : N0 - 2));
      const int side = (int)(k / (d == 0 ? NM - 2 : N0 - 2));
      if (((lay.faces >> (2 * d + side)) & 1)) {
        const int N = g.n[d];
        const long long sd = d == 0 ? s0 : s1;
        const long long base = (d == 0 ? other * s1 : other * s0) + 4LL * q;
        const long long ghost = base + (side ? N - 1 : 0) * sd;
        const long long normal = side ? -sd : sd;
        const bool odd = (g.dir >> (2 * d + side)) & 1;
        const int xq = 4 * q;
        T v[4];
        load4(v, u + ghost + 2 * normal);
        int mask = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (xq + i >= 1 && xq + i <= NF - 2)
            mask |= 1 << i;
#pragma unroll
        for (int i = 0; i < 4; ++i)
          v[i] = odd ? -v[i] : v[i];
        if (mask == 15) {
          store4(u + ghost, v);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if ((mask >> i) & 1)
              u[ghost + i] = v[i];
        }
        if (odd) {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if ((mask >> i) & 1)
              u[ghost + normal + i] = (T)0;
        }
      }
    } else {
      // a row of axis 2's faces: both sides
      k -= lay.n0 + lay.n1;
      const int y = 1 + (int)(k % (NM - 2));
      const int z = 1 + (int)(k / (NM - 2));
      const long long row = z * s0 + y * s1;
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        if (!((lay.faces >> (4 + side)) & 1))
          continue;
        const long long ghost = row + (side ? NF - 1 : 0);
        const long long normal = side ? -1 : 1;
        const bool odd = (g.dir >> (4 + side)) & 1;
        const T v = u[ghost + 2 * normal];
        u[ghost] = odd ? -v : v;
        if (odd)
          u[ghost + normal] = (T)0;
      }
    }
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// The adjoint pml memory of one lined axis from lambda^(n+1), then the coefficients
// c+ and c- the transposed step gathers (pml_aux_kernel and pml_tap,
// cuwave/kernels/scalar_sensitivity.cu:518-542, 237-251). One thread per slab node.
// One launch for every lined axis (PmlAuxSet): a block finds its axis by its index.
template <typename T>
__global__ void pml_aux_kernel(const __grid_constant__ PmlAuxSet<T> set) {
  int ai = 0;
  while (ai + 1 < set.nax && (int)blockIdx.x >= set.first[ai + 1])
    ++ai;
  const PmlAuxParams<T> &p = set.ax[ai];
  const int t = step_index(set.ctr);
  const Geometry &g = p.g;
  const int d = p.d;
  const int lo = g.lo[d], hi = g.hi[d], N = g.n[d];
  long long k = (long long)(blockIdx.x - set.first[ai]) * blockDim.x + threadIdx.x;
  const bool active = k < p.memrow;
  if (active) {
    // decompose the slab index over the grid with axis d replaced by its rows
    int A[3] = {0, 0, 0};
    int rest = (int)k;  // below memrow, an int
    int r = 0;
    for (int e = g.ndim - 1; e >= 0; --e) {
      const int extent = e == d ? lo + hi : g.ext[e];
      const int c = rest % extent;
      rest /= extent;
      if (e == d)
        r = c;
      else
        A[e] = c;
    }
    const int a = r < lo ? 1 + r : N - 1 - hi + (r - lo);
    A[d] = a;
    bool interior = true;
    for (int e = 0; e < g.ndim; ++e)
      if (e != d && (A[e] < 1 || A[e] > g.n[e] - 2))
        interior = false;
    if (interior) {
      const T *l1 = level<T>(p.l1, t);
      int idx = 0;
      bool held = false;
      for (int e = 0; e < g.ndim; ++e) {
        idx += A[e] * g.s[e];
        held |= held_wall(A[e], g.n[e], (g.dir >> (2 * e)) & 3);
      }
      const int o = g.s[d];
      T sc, sp, sm;
      if (p.uniform) {
        sc = sp = sm = p.sconst;
      } else {
        sc = p.stiff[idx];
        sp = p.stiff[idx + o];
        sm = p.stiff[idx - o];
      }
      const T gp = sc * sp / (sc + sp), gm = sc * sm / (sc + sm);
      const T w = cell_weight<T>(g, A);
      const T q = held ? (T)0 : w * l1[idx];
      const T *an = p.prof, *bn = p.prof + N, *ah = p.prof + 2 * N, *bh = p.prof + 3 * N;
      T *mem = p.mem;
      const long long sz = p.memrow;
      const T f = p.f;
      const T ez = mem[2 * sz + k];
      const T e0 = bh[a] * (mem[k] + an[a] * f * gp * ez) + f * gp * q;
      const T e1 = bh[a - 1] * (mem[sz + k] - an[a] * f * gm * ez) - f * gm * q;
      const T e2 = bn[a] * ez + q;
      mem[k] = e0;
      mem[sz + k] = e1;
      mem[2 * sz + k] = e2;
      const T ez2 = an[a] * f * e2;
      mem[3 * sz + k] = ah[a] * e0 + gp * (1 + ah[a]) * ez2;
      mem[4 * sz + k] = ah[a - 1] * e1 - gm * (1 + ah[a - 1]) * ez2;
    }
  }
  finish_step(set.ctr, set.flags & K_ADV);
}

// A running DFT at the points: acc[k * num + j] += table[row * columns + k] * a[lin[j]],
// one thread per point (dft_kernel, cuwave/kernels/common.cuh:506-518).
template <typename T>
__global__ void dft_kernel(const TransferParams<T> p, T *acc) {
  const int t = step_index(p.ctr);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < p.num) {
    const T *a = level<T>(p.a, t);
    const T uc = a[p.lin[j]];
    const T *table = reinterpret_cast<const T *>(p.record) +
                     ((long long)p.row_mul * t + p.row_add) * p.columns;
    for (int k = 0; k < p.columns; ++k)
      acc[(long long)k * p.num + j] += table[k] * uc;
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// Both Frechet densities of one triplet a, b, c of the interior, added into the
// accumulators: ft (c - a)^2 to acc_mass and sum_d F_d (b[+s_d] - b[-s_d])^2 to
// acc_stiff (frechet_kernel, cuwave/kernels/scalar_sensitivity.cu:353-385). One thread
// per node of the padded grid.
template <typename T>
__global__ void frechet_kernel(const FrechetParams<T> p) {
  const int t = step_index(p.ctr);
  const Geometry &g = p.g;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)g.n[0] * g.s[0];
  if (k < total) {
    int rest = (int)k, inside = 1;
    for (int d = 0; d < g.ndim; ++d) {
      const int a = rest / g.s[d];
      rest -= a * g.s[d];
      inside &= a > 0 && a < g.n[d] - 1;
    }
    if (inside) {
      const T *a = level<T>(p.a, t);
      const T *b = level<T>(p.b, t);
      const T *c = level<T>(p.c, t);
      const T dudt = c[k] - a[k];
      p.acc_mass[k] += p.ft * dudt * dudt;
      T sum = (T)0;
      for (int d = 0; d < g.ndim; ++d) {
        const T gd = b[k + g.s[d]] - b[k - g.s[d]];
        sum = d == 0 ? p.F[0] * gd * gd : sum + p.F[d] * gd * gd;
      }
      p.acc_stiff[k] += sum;
    }
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

}  // namespace cwb
