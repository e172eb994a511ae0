// Kernel parameter blocks, filled by the host march and passed by value.
#pragma once

#include "device.cuh"

namespace cwb {

constexpr int MAXR = 8;

template <typename T>
struct StepParams {
  Geometry g;
  T w[MAXR];  // OP_W(R, 1..R)
  T f[3];     // step factors
  T dt;
  T gconst;   // k k / (k + k) of a uniform stiffness
  T sconst;   // the uniform stiffness
  int flags;
  int refill;  // faces whose ghosts the fold writes
  int chunk;   // planes of axis 0 one block marches
  DLevel u0, u1, u2;
  const T *stiff, *minv, *damping;
  const T *prof[3];
  T *aux[3];
  int auxrow[3];
  // folded sources, listed per block (CSR): entry (plane, lane, column j, 0)
  const int *src_start;
  const int4 *src_entry;
  const T *src_weight;
  const T *signal;
  int nsrc, sig_mul, sig_add;
  // K_SUPER: acc_mass += ft (b - c_old)^2, acc_stiff += fs sum_d f_d (b[+s_d] - b[-s_d])^2
  T *acc_mass, *acc_stiff;
  T ft, fs;
  // K_CELLS: per-node cell codes and the (R, R) table of OP_W rows
  const int *cells;
  const T *ctab;
  int *ctr;
};

enum : int { MODE_STEP = 0, MODE_STEP_GRAD = 1, MODE_GRAD = 2 };

template <typename T>
struct AdjointParams {
  Geometry g;
  T w[MAXR];
  T f[3];     // per-axis factors: f_d (adjoint) or F_d (gradient)
  T dt;
  T gconst, dgconst, sconst;  // uniform stiffness: k k/(k+k), k^2/(k+k)^2, k
  T mf;       // 1 / dt^2
  int flags;
  int chunk;
  DLevel l0, l1, u0, u1, u2;  // see each mode
  const T *stiff, *minv, *damping;
  const T *prof[3];
  T *mem[3];  // adjoint pml memory: rows eta+, eta-, eta_zeta, c+, c-
  int memrow[3];
  T *g_mass, *g_stiff;
  int *ctr;
};

template <typename T>
struct TransferParams {
  Geometry g;
  DLevel a, c;
  const int *lin;
  const T *weight;
  void *record;
  int num, row_mul, row_add, store;  // store: 0 T, 1 bfloat16 bits, 2 float32
  int columns;                       // DFT: phase factors per table row
  T scale;
  int flags;
  int *ctr;
};

// both Frechet densities of a triplet a, b, c (frechet_kernel)
template <typename T>
struct FrechetParams {
  Geometry g;
  DLevel a, b, c;
  T *acc_mass, *acc_stiff;
  T ft;     // the mass density factor
  T F[3];   // the stiffness density factors, per axis
  int flags;
  int *ctr;
};

template <typename T>
struct PmlAuxParams {
  Geometry g;
  T f;  // the axis' step factor
  int d;
  DLevel l1;
  const T *stiff, *minv;
  const T *prof;
  T *mem;
  int memrow;
  T sconst;
  int uniform;
  int flags;
  int *ctr;
};

// the adjoint pml memory of every lined axis in one launch: axis ax[i]'s slab elements
// on blocks first[i] .. first[i + 1] - 1
template <typename T>
struct PmlAuxSet {
  PmlAuxParams<T> ax[3];
  int nax;
  int first[4];
  int flags;  // K_ADV
  int *ctr;
};

}  // namespace cwb
