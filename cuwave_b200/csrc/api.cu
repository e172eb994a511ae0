// The C ABI: plans, and the march that runs an op list for a range of steps.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "cuwave_b200.h"
#include "launch.cuh"
#include "march3d.cuh"
#include "pml.cuh"
#include "batch.cuh"
#include "conv.cuh"
#include "adjoint2d.cuh"
#include "step2d.cuh"
#include "step3d.cuh"
#include "step_tma.cuh"
#include "tblock2d.cuh"

namespace {

thread_local std::string g_error;
std::atomic<long long> g_launches{0};

int fail(const int code, const std::string &what) {
  g_error = what;
  return code;
}

#define CWB_CUDA(call)                                                                   \
  do {                                                                                   \
    const cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                               \
      return fail(CWB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

// steps a captured graph holds
constexpr int GRAPH_STEPS = 32;

struct Scratch {
  int *start = nullptr;
  int4 *entry = nullptr;
  size_t start_cap = 0, entry_cap = 0;
};

}  // namespace

struct cwb_plan {
  cwb_grid grid;
  cwb::Geometry geo;
  int *ctr = nullptr;
  int *err = nullptr;  // raised by a kernel whose bounded wait ran out
  bool tma = true;     // stage planes with tensor-map copies where the layout allows
  bool blocked3 = true;  // uniform-stiffness steps on the register-blocked kernels (CWB_STEP3D=0: off)
  // all steps of a 3D grid whose fields fit march3_bytes in one cooperative launch
  // (CWB_MARCH3D=0: off; 2: any size)
  int march3 = 1;
  long long march3_bytes = 8LL << 20;
  int flow3 = 1;  // the 3D blocked step without a block barrier per plane (CWB_FLOW3D=0: with; 2: deeper ring)
  int pml2d = 1;  // the 2D quad step's pml terms by a launch of their own (CWB_PML2D=0: inside the update kernel)
  int src2d = 1;  // that launch adds the step's sources too where none is on a slab node (CWB_SRC2D=0: a launch of their own)
  int fold3d = 1;  // the 3D refill launch adds the sources and reads the next record op where they touch no refilled node (CWB_FOLD3D=0: their own launches)
  int rec2d = 1;  // that launch also reads the record op that follows where its nodes are final (CWB_REC2D=0: its own launch)
  int load2d = 1;  // the 2D adjoint's gather applies the load that follows where none of its nodes is reached (CWB_LOAD2D=0: its own launch)
  cudaStream_t lane = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // the adjoint's pml memory beside its march (CWB_AUXPAR=0: before it), on this stream
  int aux_par = 1;
  cudaStream_t side = nullptr;
  cudaEvent_t side_fork = nullptr, side_join = nullptr;
  int sms = 148;
  int chunk_override = 0;
  std::vector<Scratch> scratch;
  long long pml_row[3] = {0, 0, 0};
  // a march run without a plan keeps its source lists in the library's static device
  // array (cwb_march_static) instead of the plan's scratch
  unsigned char *fixed = nullptr;
  size_t fixed_cap = 0, fixed_used = 0;
  // the temporally blocked 2D march: its second pair of field slots (the passes alternate
  // between the caller's and these) and its per-block source and receiver lists
  // temporal blocking of 2D marches (CWB_TBLOCK=1: grids too large for L2; 2: any size).
  // Off by default: one step a launch measured faster on every grid once the update
  // kernel lost its slab code (8192^2: 233 against 214 Gpt-updates/s)
  int tblock = 0;
  bool adj_split = true;  // the 3D adjoint's pml transpose as a launch of its own (CWB_ADJSPLIT=0: inline)
  void *tb_fields = nullptr;
  size_t tb_fields_bytes = 0;
  void *tb_psi = nullptr;  // temporal blocking with a pml: the levels' copies of the memory
  size_t tb_psi_bytes = 0;
  Scratch tb_src, tb_rec;
};

namespace {

using cwb::Geometry;

bool lined(const cwb_plan *p, const int d) { return p->geo.lo[d] + p->geo.hi[d] > 0; }

// planes of axis 0 a block marches: enough blocks to fill the device a few times over
int chunk_for(const cwb_plan *p, const int plane_blocks) {
  if (p->chunk_override > 0)
    return p->chunk_override;
  const int rows = p->geo.n[0] - 2;
  if (p->geo.ndim == 3) {
    // 32 planes, the fastest of 32 .. 255 measured on 512^3; fewer (down to 8) where
    // 32-plane chunks would leave the device short of blocks (two a slot of every SM):
    // a chunk's planes are a chain of waits on staged tiles, so a small grid in long
    // chunks is as slow as a large one
    const long long want = 2LL * p->sms;
    const long long chunk = (rows * (long long)plane_blocks + want - 1) / want;
    return (int)std::min<long long>(rows, std::max<long long>(8, std::min<long long>(32, chunk)));
  }
  const long long want = 8LL * p->sms;
  const long long chunk = (rows * (long long)plane_blocks + want - 1) / want;
  return (int)std::max<long long>(8, std::min<long long>(rows, chunk));
}

void stencil_grid(const cwb_plan *p, dim3 &grid, int &chunk) {
  int bx, by;
  cwb::block_shape(p->geo.ndim, bx, by);
  const Geometry &g = p->geo;
  const int F = g.ndim - 1;
  const int gx = (g.ext[F] + bx - 1) / bx;
  const int gy = g.ndim == 3 ? (g.n[1] + by - 1) / by : 1;
  chunk = chunk_for(p, gx * gy);
  const int gz = (g.n[0] - 2 + chunk - 1) / chunk;
  grid = g.ndim == 3 ? dim3(gx, gy, gz) : dim3(gx, gz, 1);
}

// the TMA step's grid: BX x BY tiles of the plane, chunks of axis 0
void tma_grid(const cwb_plan *p, const int bx, const int by, dim3 &grid, int &chunk) {
  const Geometry &g = p->geo;
  const int F = g.ndim - 1;
  const int gx = (g.ext[F] + bx - 1) / bx;
  const int gy = g.ndim == 3 ? (g.n[1] + by - 1) / by : 1;
  chunk = chunk_for(p, gx * gy);
  const int gz = (g.n[0] - 2 + chunk - 1) / chunk;
  grid = g.ndim == 3 ? dim3(gx, gy, gz) : dim3(gx, gz, 1);
}

cwb::DLevel to_level(const cwb_level &L, const int bytes) {
  cwb::DLevel d;
  d.base = static_cast<char *>(L.base);
  d.stride = L.stride * bytes;
  d.mul = L.mul;
  d.add = L.add;
  d.period = L.period;
  return d;
}

template <typename T>
int fill_material(const cwb_plan *p, const cwb_material &m, const T **stiff, const T **minv,
                  const T **damping, const T **prof, T &sconst, T &gconst, T &dgconst,
                  int &flags, bool &uniform, const bool pml) {
  uniform = m.stiff_uniform != 0;
  *stiff = static_cast<const T *>(m.stiff);
  *minv = static_cast<const T *>(m.minv);
  *damping = static_cast<const T *>(m.damping);
  if (!uniform && !m.stiff)
    return fail(CWB_ERR_ARG, "a non-uniform stiffness needs the stiff field");
  if (!m.derive_inertia && !m.minv)
    return fail(CWB_ERR_ARG, "minv is required unless derive_inertia is set");
  for (int d = 0; d < 3; ++d) {
    prof[d] = static_cast<const T *>(m.profile[d]);
    if (pml && d < p->geo.ndim && lined(p, d) && !prof[d])
      return fail(CWB_ERR_ARG, "a lined axis needs its pml profile");
  }
  sconst = (T)m.stiff_value;
  const T s = sconst;
  gconst = s * s / (s + s);
  dgconst = s * s / ((s + s) * (s + s));
  if (m.derive_inertia)
    flags |= cwb::K_DERIVE;
  if (m.damping)
    flags |= cwb::K_DAMP;
  return CWB_OK;
}

int check_level(const cwb_level &L, const char *what) {
  if (!L.base)
    return fail(CWB_ERR_ARG, std::string("op level ") + what + " has no base pointer");
  if (L.period < 0)
    return fail(CWB_ERR_ARG, std::string("op level ") + what + " has a negative period");
  return CWB_OK;
}

using Launch = std::function<cudaError_t(cudaStream_t, bool)>;

// the folded sources of a step, listed per block of its grid
template <typename T>
int build_sources(cwb_plan *p, const size_t slot, const cwb_points &pts, const dim3 grid,
                  const int chunk, const int bx, const int by, cudaStream_t stream,
                  const int **start, const int4 **entry) {
  const Geometry &g = p->geo;
  const int nblocks = grid.x * grid.y * grid.z;
  std::vector<int> lin(pts.num);
  if (pts.num) {
    CWB_CUDA(cudaMemcpyAsync(lin.data(), pts.lin, sizeof(int) * pts.num,
                             cudaMemcpyDeviceToHost, stream));
    CWB_CUDA(cudaStreamSynchronize(stream));
  }
  const int F = g.ndim - 1;
  std::vector<std::vector<int4>> per(nblocks);
  for (int j = 0; j < pts.num; ++j) {
    int rest = lin[j], A[3] = {0, 0, 0};
    for (int d = 0; d < g.ndim; ++d) {
      A[d] = rest / g.s[d];
      rest -= A[d] * g.s[d];
    }
    for (int d = 0; d < g.ndim; ++d)
      if (A[d] < 1 || A[d] > g.n[d] - 2)
        return fail(CWB_ERR_ARG, "a folded source must sit on an interior node");
    const int gx = A[F] / bx, lx = A[F] % bx;
    const int gy = g.ndim == 3 ? A[1] / by : 0, ly = g.ndim == 3 ? A[1] % by : 0;
    const int gz = (A[0] - 1) / chunk;
    const int blk = g.ndim == 3 ? gx + grid.x * (gy + grid.y * gz) : gx + grid.x * gz;
    per[blk].push_back(make_int4(A[0], ly * bx + lx, j, 0));
  }
  std::vector<int> starts(nblocks + 1, 0);
  std::vector<int4> entries;
  entries.reserve(std::max(1, pts.num));
  for (int b = 0; b < nblocks; ++b) {
    std::stable_sort(per[b].begin(), per[b].end(), [](const int4 &x, const int4 &y) {
      return x.x != y.x ? x.x < y.x : x.z < y.z;
    });
    entries.insert(entries.end(), per[b].begin(), per[b].end());
    starts[b + 1] = (int)entries.size();
  }
  if (entries.empty())
    entries.push_back(make_int4(-1, -1, 0, 0));
  if (p->fixed) {
    // no allocation: both lists go into the caller-less static region, 16-byte aligned
    const size_t off = (p->fixed_used + 15) / 16 * 16;
    const size_t start_bytes = (sizeof(int) * starts.size() + 15) / 16 * 16;
    const size_t need = off + start_bytes + sizeof(int4) * entries.size();
    if (need > p->fixed_cap)
      return fail(CWB_ERR_ARG, "the folded sources need " + std::to_string(need) +
                                   " bytes of static scratch, more than the " +
                                   std::to_string(p->fixed_cap) + " it holds");
    int *sdev = reinterpret_cast<int *>(p->fixed + off);
    int4 *edev = reinterpret_cast<int4 *>(p->fixed + off + start_bytes);
    CWB_CUDA(cudaMemcpyAsync(sdev, starts.data(), sizeof(int) * starts.size(),
                             cudaMemcpyHostToDevice, stream));
    CWB_CUDA(cudaMemcpyAsync(edev, entries.data(), sizeof(int4) * entries.size(),
                             cudaMemcpyHostToDevice, stream));
    CWB_CUDA(cudaStreamSynchronize(stream));
    p->fixed_used = need;
    *start = sdev;
    *entry = edev;
    return CWB_OK;
  }
  if (p->scratch.size() <= slot)
    p->scratch.resize(slot + 1);
  Scratch &sc = p->scratch[slot];
  if (sc.start_cap < starts.size()) {
    if (sc.start)
      cudaFree(sc.start);
    if (cudaMalloc(&sc.start, sizeof(int) * starts.size()) != cudaSuccess)
      return fail(CWB_ERR_ALLOC, "source list allocation failed");
    sc.start_cap = starts.size();
  }
  if (sc.entry_cap < entries.size()) {
    if (sc.entry)
      cudaFree(sc.entry);
    if (cudaMalloc(&sc.entry, sizeof(int4) * entries.size()) != cudaSuccess)
      return fail(CWB_ERR_ALLOC, "source list allocation failed");
    sc.entry_cap = entries.size();
  }
  CWB_CUDA(cudaMemcpyAsync(sc.start, starts.data(), sizeof(int) * starts.size(),
                           cudaMemcpyHostToDevice, stream));
  CWB_CUDA(cudaMemcpyAsync(sc.entry, entries.data(), sizeof(int4) * entries.size(),
                           cudaMemcpyHostToDevice, stream));
  CWB_CUDA(cudaStreamSynchronize(stream));
  *start = sc.start;
  *entry = sc.entry;
  return CWB_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

// a tiled tensor map, dims fastest first, strides in bytes of dims 1 .. rank - 1
template <typename T>
bool encode_map(CUtensorMap *map, const void *base, const int rank, const cuuint64_t *dims,
                const cuuint64_t *strides, const cuuint32_t *box) {
  const auto fn = encode_fn();
  if (!fn || (reinterpret_cast<uintptr_t>(base) & 15))
    return false;
  for (int i = 0; i < rank - 1; ++i)
    if (strides[i] % 16 || strides[i] >= (1ULL << 40))
      return false;
  const cuuint32_t elem[5] = {1, 1, 1, 1, 1};
  const CUresult r = fn(map, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                        rank, const_cast<void *>(base), dims, strides, box, elem,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename T, int NDIM>
int tma_halo_nd(const int R) {
  switch (R) {
  case 1: return cwb::step_tma_halo<T, NDIM, 1>();
  case 2: return cwb::step_tma_halo<T, NDIM, 2>();
  case 3: return cwb::step_tma_halo<T, NDIM, 3>();
  case 4: return cwb::step_tma_halo<T, NDIM, 4>();
  case 5: return cwb::step_tma_halo<T, NDIM, 5>();
  case 6: return cwb::step_tma_halo<T, NDIM, 6>();
  case 7: return cwb::step_tma_halo<T, NDIM, 7>();
  default: return cwb::step_tma_halo<T, NDIM, 8>();
  }
}

template <typename T, int NDIM>
cudaError_t step_tma_nd(const cwb::StepTmaParams<T> &p, const int R, const bool u,
                        const dim3 grid, cudaStream_t s) {
  switch (R) {
  case 1: return cwb::step_tma_unit<T, NDIM, 1>(p, u, grid, s);
  case 2: return cwb::step_tma_unit<T, NDIM, 2>(p, u, grid, s);
  case 3: return cwb::step_tma_unit<T, NDIM, 3>(p, u, grid, s);
  case 4: return cwb::step_tma_unit<T, NDIM, 4>(p, u, grid, s);
  case 5: return cwb::step_tma_unit<T, NDIM, 5>(p, u, grid, s);
  case 6: return cwb::step_tma_unit<T, NDIM, 6>(p, u, grid, s);
  case 7: return cwb::step_tma_unit<T, NDIM, 7>(p, u, grid, s);
  case 8: return cwb::step_tma_unit<T, NDIM, 8>(p, u, grid, s);
  }
  return cudaErrorInvalidValue;
}

// The tensor maps of a TMA step: the level stacks of operands b (box with halo) and a,
// and 1/m. False where the layout does not allow tensor-map copies.
// `bx` x `by` tiles, the box of b wider by `H` on each side of the fast axis.
template <typename T, class Params>
bool tma_maps(const cwb_plan *p, const cwb_op &op, const bool derive, const T *minv,
              Params &tp, const int bx, const int by, const int H) {
  const cwb::Geometry &g = p->geo;
  const int nd = g.ndim, F = nd - 1, R = p->grid.radius;
  const cuuint64_t ext = g.ext[F], nm = nd == 3 ? g.n[1] : 1, n0 = g.n[0];
  const cuuint64_t row = ext * sizeof(T), plane = row * nm;
  const int hy = nd == 3 ? R : 0;
  for (const cwb_level *L : {&op.b, &op.a})
    if (L->count < 1 || (L->period > 0 && L->period > L->count))
      return false;
  {
    const cuuint64_t dims[4] = {ext, nm, n0, (cuuint64_t)op.b.count};
    const cuuint64_t strides[3] = {row, plane, (cuuint64_t)op.b.stride * sizeof(T)};
    const cuuint32_t box[4] = {(cuuint32_t)(bx + 2 * H), (cuuint32_t)(by + 2 * hy), 1, 1};
    if (op.b.count > 1 && op.b.stride * (long long)sizeof(T) < (long long)(plane * n0))
      return false;
    if (!encode_map<T>(&tp.map_u1, op.b.base, 4, dims, strides, box))
      return false;
  }
  {
    const cuuint64_t dims[4] = {ext, nm, n0, (cuuint64_t)op.a.count};
    const cuuint64_t strides[3] = {row, plane, (cuuint64_t)op.a.stride * sizeof(T)};
    const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, 1};
    if (op.a.count > 1 && op.a.stride * (long long)sizeof(T) < (long long)(plane * n0))
      return false;
    if (!encode_map<T>(&tp.map_u0, op.a.base, 4, dims, strides, box))
      return false;
  }
  if (!derive) {
    const cuuint64_t dims[3] = {ext, nm, n0};
    const cuuint64_t strides[2] = {row, plane};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    if (!encode_map<T>(&tp.map_minv, minv, 3, dims, strides, box))
      return false;
  } else {
    tp.map_minv = tp.map_u0;  // never read
  }
  tp.level_u1[0] = op.b.mul, tp.level_u1[1] = op.b.add, tp.level_u1[2] = op.b.period;
  tp.level_u0[0] = op.a.mul, tp.level_u0[1] = op.a.add, tp.level_u0[2] = op.a.period;
  return true;
}

template <typename T, int NDIM>
cudaError_t step_nd(const cwb::StepParams<T> &p, const int R, const bool u, const dim3 grid,
                    cudaStream_t s) {
  switch (R) {
  case 1: return cwb::step_unit<T, NDIM, 1>(p, u, grid, s);
  case 2: return cwb::step_unit<T, NDIM, 2>(p, u, grid, s);
  case 3: return cwb::step_unit<T, NDIM, 3>(p, u, grid, s);
  case 4: return cwb::step_unit<T, NDIM, 4>(p, u, grid, s);
  case 5: return cwb::step_unit<T, NDIM, 5>(p, u, grid, s);
  case 6: return cwb::step_unit<T, NDIM, 6>(p, u, grid, s);
  case 7: return cwb::step_unit<T, NDIM, 7>(p, u, grid, s);
  case 8: return cwb::step_unit<T, NDIM, 8>(p, u, grid, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T, int NDIM>
cudaError_t adjoint_nd(const cwb::AdjointParams<T> &p, const int R, const bool u,
                       const int mode, const dim3 grid, cudaStream_t s) {
  switch (R) {
  case 1: return cwb::adjoint_unit<T, NDIM, 1>(p, u, mode, grid, s);
  case 2: return cwb::adjoint_unit<T, NDIM, 2>(p, u, mode, grid, s);
  case 3: return cwb::adjoint_unit<T, NDIM, 3>(p, u, mode, grid, s);
  case 4: return cwb::adjoint_unit<T, NDIM, 4>(p, u, mode, grid, s);
  case 5: return cwb::adjoint_unit<T, NDIM, 5>(p, u, mode, grid, s);
  case 6: return cwb::adjoint_unit<T, NDIM, 6>(p, u, mode, grid, s);
  case 7: return cwb::adjoint_unit<T, NDIM, 7>(p, u, mode, grid, s);
  case 8: return cwb::adjoint_unit<T, NDIM, 8>(p, u, mode, grid, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t step_dispatch(const cwb::StepParams<T> &p, const int ndim, const int R,
                          const bool u, const dim3 grid, cudaStream_t s) {
  return ndim == 3 ? step_nd<T, 3>(p, R, u, grid, s) : step_nd<T, 2>(p, R, u, grid, s);
}

template <typename T>
cudaError_t step_tma_dispatch(const cwb::StepTmaParams<T> &p, const int ndim, const int R,
                              const bool u, const dim3 grid, cudaStream_t s) {
  return ndim == 3 ? step_tma_nd<T, 3>(p, R, u, grid, s) : step_tma_nd<T, 2>(p, R, u, grid, s);
}

template <typename T>
int step3d_halo_r(const int R) {
  switch (R) {
  case 1: return cwb::step3d_halo<T, 1>();
  case 2: return cwb::step3d_halo<T, 2>();
  case 3: return cwb::step3d_halo<T, 3>();
  case 4: return cwb::step3d_halo<T, 4>();
  case 5: return cwb::step3d_halo<T, 5>();
  case 6: return cwb::step3d_halo<T, 6>();
  case 7: return cwb::step3d_halo<T, 7>();
  case 8: return cwb::step3d_halo<T, 8>();
  }
  return -1;
}

template <typename T>
bool step2d_built_r(const int R) {
  switch (R) {
  case 1: return cwb::step2d_built<T, 1>();
  case 2: return cwb::step2d_built<T, 2>();
  case 3: return cwb::step2d_built<T, 3>();
  case 4: return cwb::step2d_built<T, 4>();
  case 5: return cwb::step2d_built<T, 5>();
  case 6: return cwb::step2d_built<T, 6>();
  case 7: return cwb::step2d_built<T, 7>();
  case 8: return cwb::step2d_built<T, 8>();
  }
  return false;
}

template <typename T>
cudaError_t pml2d_r(const cwb::StepParams<T> &p, const cwb::Pml2Layout &lay,
                    const cwb::TransferParams<T> &src, const cwb::TransferParams<T> &rec, const int R,
                    cudaStream_t s) {
  switch (R) {
  case 1: return cwb::pml2d_unit<T, 1>(p, lay, src, rec, s);
  case 2: return cwb::pml2d_unit<T, 2>(p, lay, src, rec, s);
  case 3: return cwb::pml2d_unit<T, 3>(p, lay, src, rec, s);
  case 4: return cwb::pml2d_unit<T, 4>(p, lay, src, rec, s);
  case 5: return cwb::pml2d_unit<T, 5>(p, lay, src, rec, s);
  case 6: return cwb::pml2d_unit<T, 6>(p, lay, src, rec, s);
  case 7: return cwb::pml2d_unit<T, 7>(p, lay, src, rec, s);
  case 8: return cwb::pml2d_unit<T, 8>(p, lay, src, rec, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t step2d_r(const cwb::StepParams<T> &p, const int R, const bool u, const dim3 grid,
                     cudaStream_t s) {
  switch (R) {
  case 1: return cwb::step2d_unit<T, 1>(p, u, grid, s);
  case 2: return cwb::step2d_unit<T, 2>(p, u, grid, s);
  case 3: return cwb::step2d_unit<T, 3>(p, u, grid, s);
  case 4: return cwb::step2d_unit<T, 4>(p, u, grid, s);
  case 5: return cwb::step2d_unit<T, 5>(p, u, grid, s);
  case 6: return cwb::step2d_unit<T, 6>(p, u, grid, s);
  case 7: return cwb::step2d_unit<T, 7>(p, u, grid, s);
  case 8: return cwb::step2d_unit<T, 8>(p, u, grid, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t adjoint2d_pml_r(const cwb::AdjointParams<T> &p, const cwb::Adj2Reach &reach,
                            const int R, const int mode, const cwb::TransferParams<T> &ld,
                            T *ld_mass, const dim3 grid, cudaStream_t s) {
  switch (R) {
  case 1: return cwb::adjoint2d_pml_unit<T, 1>(p, reach, mode, ld, ld_mass, grid, s);
  case 2: return cwb::adjoint2d_pml_unit<T, 2>(p, reach, mode, ld, ld_mass, grid, s);
  case 3: return cwb::adjoint2d_pml_unit<T, 3>(p, reach, mode, ld, ld_mass, grid, s);
  case 4: return cwb::adjoint2d_pml_unit<T, 4>(p, reach, mode, ld, ld_mass, grid, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t adjoint3d_pml_r(const cwb::AdjointParams<T> &p, const cwb::Adj3Reach &reach,
                            const int R, const bool u, const int mode, const dim3 grid,
                            cudaStream_t s) {
  switch (R) {
  case 1: return cwb::adjoint3d_pml_unit<T, 1>(p, reach, u, mode, grid, s);
  case 2: return cwb::adjoint3d_pml_unit<T, 2>(p, reach, u, mode, grid, s);
  case 3: return cwb::adjoint3d_pml_unit<T, 3>(p, reach, u, mode, grid, s);
  case 4: return cwb::adjoint3d_pml_unit<T, 4>(p, reach, u, mode, grid, s);
  case 5: return cwb::adjoint3d_pml_unit<T, 5>(p, reach, u, mode, grid, s);
  case 6: return cwb::adjoint3d_pml_unit<T, 6>(p, reach, u, mode, grid, s);
  case 7: return cwb::adjoint3d_pml_unit<T, 7>(p, reach, u, mode, grid, s);
  case 8: return cwb::adjoint3d_pml_unit<T, 8>(p, reach, u, mode, grid, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t adjoint2d_r(const cwb::AdjointParams<T> &p, const int R, const int mode,
                        const dim3 grid, cudaStream_t s) {
  switch (R) {
  case 1: return cwb::adjoint2d_unit<T, 1>(p, mode, grid, s);
  case 2: return cwb::adjoint2d_unit<T, 2>(p, mode, grid, s);
  case 3: return cwb::adjoint2d_unit<T, 3>(p, mode, grid, s);
  case 4: return cwb::adjoint2d_unit<T, 4>(p, mode, grid, s);
  case 5: return cwb::adjoint2d_unit<T, 5>(p, mode, grid, s);
  case 6: return cwb::adjoint2d_unit<T, 6>(p, mode, grid, s);
  case 7: return cwb::adjoint2d_unit<T, 7>(p, mode, grid, s);
  case 8: return cwb::adjoint2d_unit<T, 8>(p, mode, grid, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t step3d_r(const cwb::Step3Params<T> &p, const int R, const bool u, const dim3 grid,
                     cudaStream_t s) {
  switch (R) {
  case 1: return cwb::step3d_unit<T, 1>(p, u, grid, s);
  case 2: return cwb::step3d_unit<T, 2>(p, u, grid, s);
  case 3: return cwb::step3d_unit<T, 3>(p, u, grid, s);
  case 4: return cwb::step3d_unit<T, 4>(p, u, grid, s);
  case 5: return cwb::step3d_unit<T, 5>(p, u, grid, s);
  case 6: return cwb::step3d_unit<T, 6>(p, u, grid, s);
  case 7: return cwb::step3d_unit<T, 7>(p, u, grid, s);
  case 8: return cwb::step3d_unit<T, 8>(p, u, grid, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t adjoint_dispatch(const cwb::AdjointParams<T> &p, const int ndim, const int R,
                             const bool u, const int mode, const dim3 grid, cudaStream_t s) {
  return ndim == 3 ? adjoint_nd<T, 3>(p, R, u, mode, grid, s)
                   : adjoint_nd<T, 2>(p, R, u, mode, grid, s);
}

template <typename T>
void fill_weights(const cwb_plan *p, T *w, T *f) {
  for (int k = 0; k < cwb::MAXR; ++k)
    w[k] = k < p->grid.radius ? (T)p->grid.coeffs[k] : (T)0;
  for (int d = 0; d < 3; ++d)
    f[d] = d < p->geo.ndim ? (T)p->grid.factors[d] : (T)0;
}

template <typename T>
cudaError_t pml3d_r(const cwb::Pml3Params<T> &p, const int R, const int axis, const dim3 grid,
                    cudaStream_t s) {
  switch (R) {
  case 1: return cwb::pml3d_unit<T, 1>(p, axis, grid, s);
  case 2: return cwb::pml3d_unit<T, 2>(p, axis, grid, s);
  case 3: return cwb::pml3d_unit<T, 3>(p, axis, grid, s);
  case 4: return cwb::pml3d_unit<T, 4>(p, axis, grid, s);
  case 5: return cwb::pml3d_unit<T, 5>(p, axis, grid, s);
  case 6: return cwb::pml3d_unit<T, 6>(p, axis, grid, s);
  case 7: return cwb::pml3d_unit<T, 7>(p, axis, grid, s);
  case 8: return cwb::pml3d_unit<T, 8>(p, axis, grid, s);
  }
  return cudaErrorInvalidValue;
}

// The pml launches of axes 1 and 2 after the blocked 3D step (which advanced axis 0's
// memory in its march): a launch per lined axis, axis 1 first, so a node in both slabs
// takes its shares in the reference's order.
template <typename T>
int pml_launch(const cwb_plan *p, const cwb::StepParams<T> &sp, const int fold,
               std::vector<Launch> &out) {
  const Geometry &g = p->geo;
  const int R = p->grid.radius;
  if (g.ndim != 3)
    return fail(CWB_ERR_UNSUPPORTED, "the pml slab launches step 3D grids");
  cwb::Pml3Params<T> pp;
  std::memset(&pp, 0, sizeof pp);
  pp.g = g;
  for (int k = 0; k < cwb::MAXR; ++k)
    pp.w[k] = sp.w[k];
  pp.gconst = sp.gconst;
  pp.sconst = sp.sconst;
  pp.flags = sp.flags & cwb::K_DERIVE;
  pp.u1 = sp.u1;
  pp.u2 = sp.u2;
  pp.minv = sp.minv;
  pp.ctr = sp.ctr;
  if (g.lo[1] + g.hi[1] > 0) {
    cwb::Pml3Params<T> q1 = pp;
    q1.f = sp.f[1];
    q1.prof = sp.prof[1];
    q1.aux = sp.aux[1];
    q1.auxrow = sp.auxrow[1];
    const int quads = (g.n[2] - 2) / 4 + 1;
    const dim3 grid((quads + cwb::PML1_QUADS - 1) / cwb::PML1_QUADS,
                    (g.lo[1] + g.hi[1] + cwb::PML1_ROWS - 1) / cwb::PML1_ROWS, g.n[0] - 2);
    out.push_back([q1, R, grid](cudaStream_t s, bool adv) {
      cwb::Pml3Params<T> q = q1;
      if (adv)
        q.flags |= cwb::K_ADV;
      return pml3d_r<T>(q, R, 1, grid, s);
    });
  }
  if (g.lo[2] + g.hi[2] > 0) {
    cwb::Pml3Params<T> q2 = pp;
    q2.f = sp.f[2];
    q2.prof = sp.prof[2];
    q2.aux = sp.aux[2];
    q2.auxrow = sp.auxrow[2];
    const int NF = g.n[2];
    // quads of four holding a slab node: x in 1 .. lo on the low side, NF - 1 - hi ..
    // NF - 2 on the high side
    q2.nlo = g.lo[2] > 0 ? g.lo[2] / 4 + 1 : 0;
    q2.xhi = (NF - 1 - g.hi[2]) / 4 * 4;
    q2.nhi = g.hi[2] > 0 ? (NF - 2) / 4 - (NF - 1 - g.hi[2]) / 4 + 1 : 0;
    q2.fold = fold;
    const int nq = q2.nlo + q2.nhi;
    if (nq > cwb::PML2_THREADS)
      return fail(CWB_ERR_UNSUPPORTED, "pml slabs wider than 500 nodes along axis 2");
    const int rows = cwb::PML2_THREADS / nq;
    const dim3 grid(1, (g.n[1] - 2 + rows - 1) / rows, g.n[0] - 2);
    out.push_back([q2, R, grid](cudaStream_t s, bool adv) {
      cwb::Pml3Params<T> q = q2;
      if (adv)
        q.flags |= cwb::K_ADV;
      return pml3d_r<T>(q, R, 2, grid, s);
    });
  }
  return CWB_OK;
}

// The step op's common parameters: geometry, stencil row, factors, materials, pml memory.
template <typename T>
int step_setup(const cwb_plan *p, const cwb_op &op, cwb::StepParams<T> &sp, int &flags,
               bool &uniform) {
  int rc;
  if ((rc = check_level(op.a, "a")) || (rc = check_level(op.b, "b")) ||
      (rc = check_level(op.c, "c")))
    return rc;
  sp.g = p->geo;
  fill_weights(p, sp.w, sp.f);
  sp.dt = (T)p->grid.dt;
  T dgconst;
  flags = 0;
  if ((rc = fill_material<T>(p, op.mat, &sp.stiff, &sp.minv, &sp.damping, sp.prof, sp.sconst,
                             sp.gconst, dgconst, flags, uniform, op.flags & CWB_PML)))
    return rc;
  if (op.flags & CWB_PML) {
    flags |= cwb::K_PML;
    for (int d = 0; d < p->geo.ndim; ++d) {
      sp.aux[d] = static_cast<T *>(op.memory[d]);
      sp.auxrow[d] = (int)p->pml_row[d];
      if (lined(p, d) && !sp.aux[d])
        return fail(CWB_ERR_ARG, "a lined axis needs its pml memory");
    }
  }
  return CWB_OK;
}

// An internal refill op's flags: the faces (bit 2d low, 2d + 1 high of axis d, times
// this) that an earlier launch of the step refilled already.
constexpr int OP_REFILLED = 1 << 24;

// The sources' mirror positions on `axis`: whether a folded source sits at index a there.
int sources_at(const cwb_plan *p, const cwb_op &op, cudaStream_t stream, const int axis,
               const int a, const int b, bool &at_a, bool &at_b) {
  const Geometry &g = p->geo;
  at_a = at_b = false;
  const cwb_points &src = op.points;
  if (!(op.flags & CWB_FOLD_SOURCES) || src.num <= 0)
    return CWB_OK;
  std::vector<int> lin(src.num);
  CWB_CUDA(cudaMemcpyAsync(lin.data(), src.lin, sizeof(int) * src.num, cudaMemcpyDeviceToHost, stream));
  CWB_CUDA(cudaStreamSynchronize(stream));
  for (const int l : lin) {
    const int c = axis == 0 ? l / g.s[0] : (l % g.s[axis - 1]) / g.s[axis];
    at_a = at_a || c == a;
    at_b = at_b || c == b;
  }
  return CWB_OK;
}

// The 2D quad step's face ghosts pml2d_kernel may refill itself (1 row 0, 2 row N0 - 1,
// 4 column 0, 8 column NF - 1): a face refilled this step whose mirror row or column the
// pml launch's threads hold (an axis-0 slab reaching row 2 or N0 - 3; an axis-1 slab on
// that side with ghost and mirror in one quad that only that side's threads write) and
// no folded source on it.
int ghost_fold_2d(const cwb_plan *p, const cwb_op &op, cudaStream_t stream, int &fold) {
  const Geometry &g = p->geo;
  fold = 0;
  if (g.ndim != 2 || !(op.flags & CWB_FOLD_REFILL))
    return CWB_OK;
  const int N0 = g.n[0], NF = g.n[1];
  const int faces = p->grid.neumann | p->grid.dirichlet;
  if ((faces & 1) && g.lo[0] >= 2)
    fold |= 1;
  if ((faces & 2) && g.hi[0] >= 2)
    fold |= 2;
  if ((faces & 4) && g.lo[1] > 0 && NF - 1 - g.hi[1] > 3)
    fold |= 4;
  if ((faces & 8) && g.hi[1] > 0 && (NF - 1) % 4 >= 2 && g.lo[1] < (NF - 1) / 4 * 4)
    fold |= 8;
  bool r2, rn, c2, cn;
  int rc;
  if (fold && ((rc = sources_at(p, op, stream, 0, 2, N0 - 3, r2, rn)) ||
               (rc = sources_at(p, op, stream, 1, 2, NF - 3, c2, cn))))
    return rc;
  if (fold) {
    if (r2) fold &= ~1;
    if (rn) fold &= ~2;
    if (c2) fold &= ~4;
    if (cn) fold &= ~8;
  }
  return CWB_OK;
}

// The 3D step's fast-axis face ghosts the axis-2 pml launch may refill itself (1 low,
// 2 high): the face lined by the pml and refilled this step, its ghost and mirror in one
// quad that only that side's slab threads write, and no folded source on the mirror
// column (the sources are added after the pml, the refill after them).
template <typename T>
int x_ghost_fold(const cwb_plan *p, const cwb_op &op, cudaStream_t stream, int &fold) {
  const Geometry &g = p->geo;
  fold = 0;
  if (g.ndim != 3 || !(op.flags & CWB_FOLD_REFILL))
    return CWB_OK;
  const int NF = g.n[2], lo = g.lo[2], hi = g.hi[2];
  const int faces = p->grid.neumann | p->grid.dirichlet;
  if (lo > 0 && ((faces >> 4) & 1) && NF - 1 - hi > 3)
    fold |= 1;
  if (hi > 0 && ((faces >> 5) & 1) && (NF - 1) % 4 >= 2 && lo < (NF - 1) / 4 * 4)
    fold |= 2;
  bool at_lo, at_hi;
  if (fold) {
    if (const int rc = sources_at(p, op, stream, 2, 2, NF - 3, at_lo, at_hi))
      return rc;
    if (at_lo)
      fold &= ~1;
    if (at_hi)
      fold &= ~2;
  }
  return CWB_OK;
}

// the launches of one op, each taking (stream, advance)
template <typename T>
int translate(cwb_plan *p, const cwb_op &op, const size_t slot, cudaStream_t stream,
              std::vector<Launch> &out, const cwb_op *next = nullptr, bool *took_next = nullptr) {
  const Geometry &g = p->geo;
  const int ndim = g.ndim, R = p->grid.radius;
  const int bytes = sizeof(T);
  int rc;
  switch (op.kind) {
  case CWB_OP_STEP:
  case CWB_OP_SUPERPOSED: {
    cwb::StepTmaParams<T> tp;
    std::memset(&tp, 0, sizeof tp);
    cwb::StepParams<T> &sp = tp.s;
    bool uniform;
    int flags = 0;
    if ((rc = step_setup<T>(p, op, sp, flags, uniform)))
      return rc;
    // a masked domain: the plain kernel with the cell radii, no pml
    const bool masked = op.mat.cells != nullptr;
    if (masked) {
      if (flags & cwb::K_PML)
        return fail(CWB_ERR_UNSUPPORTED, "a pml takes no domain mask");
      if (!op.mat.cell_table)
        return fail(CWB_ERR_ARG, "a masked domain needs its cell table");
      flags |= cwb::K_CELLS;
      sp.cells = op.mat.cells;
      sp.ctab = static_cast<const T *>(op.mat.cell_table);
    }
    // the superposed step: the plain kernel with the density epilogue, lossless only
    const bool super = op.kind == CWB_OP_SUPERPOSED;
    if (super) {
      if ((flags & (cwb::K_PML | cwb::K_DAMP)))
        return fail(CWB_ERR_UNSUPPORTED, "the superposed step is lossless: no pml, no damping");
      if (!op.g_mass || !op.g_stiff)
        return fail(CWB_ERR_ARG, "the superposed step needs both accumulators");
      flags |= cwb::K_SUPER;
      sp.acc_mass = static_cast<T *>(op.g_mass);
      sp.acc_stiff = static_cast<T *>(op.g_stiff);
      sp.ft = (T)op.scale;
      sp.fs = (T)op.factors[0];
    }
    // 3D, a uniform stiffness: the blocked kernel. It stores rows of four and keeps the
    // taps it mirrors in its own run, so it wants an output level on 16-byte boundaries
    // and axes of at least 3R nodes. Elsewhere the TMA row kernel, else the plain one.
    const bool derive = flags & cwb::K_DERIVE;
    cwb::Step3Params<T> s3;
    std::memset(&s3, 0, sizeof s3);
    const bool c_aligned = reinterpret_cast<uintptr_t>(op.c.base) % 16 == 0 &&
                           (op.c.stride * (long long)sizeof(T)) % 16 == 0;
    const bool roomy = ndim == 3 && g.n[0] >= 3 * R && g.n[1] >= 3 * R && g.n[2] >= 3 * R;
    const int H3 = ndim == 3 ? step3d_halo_r<T>(R) : -1;
    const bool blocked = !super && !masked && p->tma && p->blocked3 && uniform && c_aligned && roomy && H3 >= 0 &&
                         tma_maps<T>(p, op, derive, sp.minv, s3, cwb::S3_BX, cwb::S3_BY, H3);
    const int Hrow = ndim == 3 ? tma_halo_nd<T, 3>(R) : tma_halo_nd<T, 2>(R);
    const bool tma = !blocked && !super && !masked && p->tma &&
                     tma_maps<T>(p, op, derive, sp.minv, tp, ndim == 3 ? cwb::TMA_BX3 : cwb::TMA_BX2,
                                 ndim == 3 ? cwb::TMA_BY3 : 1, Hrow);
    // 2D, a uniform stiffness, float: the quad step, which reads u^(t-1),
    // u^(t-2) and 1/m as 16-byte rows (levels and 1/m on 16-byte boundaries)
    const auto aligned16 = [](const void *ptr, const long long stride_elems) {
      return reinterpret_cast<uintptr_t>(ptr) % 16 == 0 && (stride_elems * (long long)sizeof(T)) % 16 == 0;
    };
    const bool quad2 = !super && !masked && ndim == 2 && p->blocked3 && uniform && step2d_built_r<T>(R) &&
                       aligned16(op.a.base, op.a.stride) && aligned16(op.b.base, op.b.stride) &&
                       aligned16(op.c.base, op.c.stride) && (derive || aligned16(sp.minv, 0)) &&
                       g.n[0] >= 3 * R && g.n[1] >= 3 * R;
    int refilled = 0;  // face ghosts a launch before the refill has written (face bits)
    bool sources_done = false;  // the sources added by a launch before the excitation's
    if (quad2) {
      // enough quads x row chunks to give every SM a few blocks of 128 threads
      const long long rows = g.n[0] - 2, quads = (g.n[1] - 2) / 4 + 1;
      const long long want = (long long)p->sms * 1024;
      const int chunk = (int)std::max<long long>(1, std::min<long long>(rows, rows * quads / want));
      sp.chunk = p->chunk_override > 0 ? p->chunk_override : chunk;
      const long long threads = quads * ((rows + sp.chunk - 1) / sp.chunk);
      const dim3 grid((unsigned)((threads + cwb::S2_THREADS - 1) / cwb::S2_THREADS));
      sp.flags = flags;
      sp.u0 = to_level(op.a, bytes);
      sp.u1 = to_level(op.b, bytes);
      sp.u2 = to_level(op.c, bytes);
      sp.ctr = p->ctr;
      // the pml terms by a launch of their own over the slab nodes, the update kernel
      // built without them (CWB_PML2D=0: inside the update kernel)
      const bool split = (flags & cwb::K_PML) && p->pml2d;
      cwb::StepParams<T> su = sp;
      if (split)
        su.flags &= ~cwb::K_PML;
      out.push_back([su, R, uniform, grid](cudaStream_t s, bool adv) {
        cwb::StepParams<T> q = su;
        if (adv)
          q.flags |= cwb::K_ADV;
        return step2d_r<T>(q, R, uniform, grid, s);
      });
      if (split) {
        cwb::Pml2Layout lay;
        const int NF = g.n[1], lo1 = g.lo[1], hi1 = g.hi[1];
        lay.nq = (int)quads;
        lay.nlo = lo1 > 0 ? lo1 / 4 + 1 : 0;
        lay.xhi = (NF - 1 - hi1) / 4 * 4;
        lay.nhi = hi1 > 0 ? (NF - 2) / 4 - (NF - 1 - hi1) / 4 + 1 : 0;
        lay.na = (long long)(g.lo[0] + g.hi[0]) * quads;
        lay.total = lay.na + (long long)(g.n[0] - 2 - g.lo[0] - g.hi[0]) * (lay.nlo + lay.nhi);
        if ((rc = ghost_fold_2d(p, op, stream, lay.fold)))
          return rc;
        if (lay.total <= 0)
          lay.fold = 0;
        refilled = lay.fold;
        // the sources ride on the pml launch where none sits on a node it writes (a slab
        // node; its ghost folds are interior-free): the pml's share of a node comes
        // before its source in cuwave's step, and no slab node holds one
        cwb::TransferParams<T> src;
        std::memset(&src, 0, sizeof src);
        const cwb_points &pt = op.points;
        if (lay.total > 0 && p->src2d && (op.flags & CWB_FOLD_SOURCES) && pt.num > 0 && pt.lin &&
            pt.weight && pt.record && pt.store >= 0 && pt.store <= 1) {
          std::vector<int> lin(pt.num);
          CWB_CUDA(cudaMemcpyAsync(lin.data(), pt.lin, sizeof(int) * pt.num, cudaMemcpyDeviceToHost, stream));
          CWB_CUDA(cudaStreamSynchronize(stream));
          const int N0 = g.n[0], lo0 = g.lo[0], hi0 = g.hi[0];
          bool clear = true;
          for (const int l : lin) {
            const int z = l / g.s[0], x = l % g.s[0];
            const bool interior = z >= 1 && z <= N0 - 2 && x >= 1 && x <= NF - 2;
            const bool slab = (lo0 && z <= lo0) || (hi0 && z >= N0 - 1 - hi0) || (lo1 && x <= lo1) ||
                              (hi1 && x >= NF - 1 - hi1);
            clear = clear && interior && !slab;
          }
          if (clear) {
            src.g = g;
            src.a = to_level(op.c, bytes);
            src.lin = pt.lin;
            src.weight = static_cast<const T *>(pt.weight);
            src.record = pt.record;
            src.num = pt.num;
            src.row_mul = pt.row_mul;
            src.row_add = pt.row_add;
            src.store = pt.store;
            src.ctr = p->ctr;
            sources_done = true;
          }
        }
        // the record op that follows rides on the launch too where its nodes are final
        // after the update: interior, no slab node (the pml's), no source's node
        cwb::TransferParams<T> rec;
        std::memset(&rec, 0, sizeof rec);
        if (lay.total > 0 && p->rec2d && next && took_next && next->kind == CWB_OP_RECORD &&
            next->points.num > 0 && next->points.num <= 65536 && next->points.lin && next->points.record &&
            next->points.store >= 0 && next->points.store <= 2 &&
            !(next->points.store == 2 && sizeof(T) == 4) && !check_level(next->a, "a")) {
          const cwb_points &rp = next->points;
          std::vector<int> rlin(rp.num), slin;
          CWB_CUDA(cudaMemcpyAsync(rlin.data(), rp.lin, sizeof(int) * rp.num, cudaMemcpyDeviceToHost, stream));
          if ((op.flags & CWB_FOLD_SOURCES) && pt.num > 0 && pt.lin) {
            slin.resize(pt.num);
            CWB_CUDA(cudaMemcpyAsync(slin.data(), pt.lin, sizeof(int) * pt.num, cudaMemcpyDeviceToHost, stream));
          }
          CWB_CUDA(cudaStreamSynchronize(stream));
          std::sort(slin.begin(), slin.end());
          const int N0 = g.n[0], lo0 = g.lo[0], hi0 = g.hi[0];
          bool clear = true;
          for (const int l : rlin) {
            const int z = l / g.s[0], x = l % g.s[0];
            const bool interior = z >= 1 && z <= N0 - 2 && x >= 1 && x <= NF - 2;
            const bool slab = (lo0 && z <= lo0) || (hi0 && z >= N0 - 1 - hi0) || (lo1 && x <= lo1) ||
                              (hi1 && x >= NF - 1 - hi1);
            clear = clear && interior && !slab && !std::binary_search(slin.begin(), slin.end(), l);
          }
          if (clear) {
            rec.g = g;
            rec.a = to_level(next->a, bytes);
            rec.lin = rp.lin;
            rec.record = rp.record;
            rec.num = rp.num;
            rec.row_mul = rp.row_mul;
            rec.row_add = rp.row_add;
            rec.store = rp.store;
            rec.ctr = p->ctr;
            *took_next = true;
          }
        }
        if (lay.total > 0)
          out.push_back([sp, lay, src, rec, R](cudaStream_t s, bool adv) {
            cwb::StepParams<T> q = sp;
            if (adv)
              q.flags |= cwb::K_ADV;
            return pml2d_r<T>(q, lay, src, rec, R, s);
          });
      }
    }
    if (blocked || quad2) {
      int fold = 0;  // fast-axis face ghosts the pml launch refills
      // after the update (and its pml memory), the sources and the refill, each a
      // launch of its own in the order of cuwave's step
      if (blocked) {
        dim3 grid;
        tma_grid(p, cwb::S3_BX, cwb::S3_BY, grid, sp.chunk);
        sp.flags = flags;
        sp.u0 = to_level(op.a, bytes);
        sp.u1 = to_level(op.b, bytes);
        sp.u2 = to_level(op.c, bytes);
        sp.ctr = p->ctr;
        s3.s = sp;
        s3.err = p->err;
        s3.flow = p->flow3;
        out.push_back([s3, R, uniform, grid](cudaStream_t s, bool adv) {
          cwb::Step3Params<T> q = s3;
          if (adv)
            q.s.flags |= cwb::K_ADV;
          return step3d_r<T>(q, R, uniform, grid, s);
        });
        if (op.flags & CWB_PML) {
          if ((rc = x_ghost_fold<T>(p, op, stream, fold)))
            return rc;
          if ((rc = pml_launch<T>(p, sp, fold, out)))
            return rc;
          refilled = fold << 4;
        }
      }
      // 3D: the refill launch adds the sources and reads the record op that follows where
      // neither touches a node the refill reads or writes (a refilled face's mirror, a ghost,
      // a held wall node) and no receiver sits on a source
      cwb::TransferParams<T> src3, rec3;
      std::memset(&src3, 0, sizeof src3);
      std::memset(&rec3, 0, sizeof rec3);
      const int faces3 = (p->grid.neumann | p->grid.dirichlet) & ~refilled;
      if (blocked && p->fold3d && (op.flags & CWB_FOLD_REFILL)) {
        const auto place = [&](const int l, int A[3]) {
          A[0] = l / g.s[0];
          A[1] = (l % g.s[0]) / g.s[1];
          A[2] = l % g.s[1];
        };
        // along axis d: whether index a is a refilled face's mirror, a ghost or a held wall
        const auto touched = [&](const int d, const int a, const bool reads) {
          const int N = g.n[d];
          bool hit = a <= 0 || a >= N - 1;
          for (int side = 0; side < 2; ++side) {
            if (!((faces3 >> (2 * d + side)) & 1))
              continue;
            if (reads && a == (side ? N - 3 : 2))
              hit = true;
            if (((p->grid.dirichlet >> (2 * d + side)) & 1) && a == (side ? N - 2 : 1))
              hit = true;
          }
          return hit;
        };
        const cwb_points &sp3 = op.points;
        std::vector<int> slin;
        if ((op.flags & CWB_FOLD_SOURCES) && sp3.num > 0 && sp3.num <= 65536 && sp3.lin && sp3.weight &&
            sp3.record && sp3.store >= 0 && sp3.store <= 1) {
          slin.resize(sp3.num);
          CWB_CUDA(cudaMemcpyAsync(slin.data(), sp3.lin, sizeof(int) * sp3.num, cudaMemcpyDeviceToHost, stream));
          CWB_CUDA(cudaStreamSynchronize(stream));
          bool clear = true;
          for (const int l : slin) {
            int A[3];
            place(l, A);
            for (int d = 0; d < 3; ++d)
              clear = clear && !touched(d, A[d], true);
          }
          if (clear) {
            src3.g = g;
            src3.a = to_level(op.c, bytes);
            src3.lin = sp3.lin;
            src3.weight = static_cast<const T *>(sp3.weight);
            src3.record = sp3.record;
            src3.num = sp3.num;
            src3.row_mul = sp3.row_mul;
            src3.row_add = sp3.row_add;
            src3.store = sp3.store;
            src3.ctr = p->ctr;
            sources_done = true;
          }
        }
        if (next && took_next && next->kind == CWB_OP_RECORD && next->points.num > 0 &&
            next->points.num <= 65536 && next->points.lin && next->points.record &&
            next->points.store >= 0 && next->points.store <= 2 &&
            !(next->points.store == 2 && sizeof(T) == 4) && !check_level(next->a, "a")) {
          const cwb_points &rp = next->points;
          std::vector<int> rlin(rp.num);
          CWB_CUDA(cudaMemcpyAsync(rlin.data(), rp.lin, sizeof(int) * rp.num, cudaMemcpyDeviceToHost, stream));
          CWB_CUDA(cudaStreamSynchronize(stream));
          std::vector<int> sorted;
          if (src3.num)
            sorted = slin;
          std::sort(sorted.begin(), sorted.end());
          bool clear = true;
          for (const int l : rlin) {
            int A[3];
            place(l, A);
            for (int d = 0; d < 3; ++d)
              clear = clear && !touched(d, A[d], false);
            clear = clear && !std::binary_search(sorted.begin(), sorted.end(), l);
          }
          if (clear) {
            rec3.g = g;
            rec3.a = to_level(next->a, bytes);
            rec3.lin = rp.lin;
            rec3.record = rp.record;
            rec3.num = rp.num;
            rec3.row_mul = rp.row_mul;
            rec3.row_add = rp.row_add;
            rec3.store = rp.store;
            rec3.ctr = p->ctr;
            *took_next = true;
          }
        }
      }
      if ((op.flags & CWB_FOLD_SOURCES) && op.points.num > 0 && !sources_done) {
        if (!op.points.weight || !op.points.record)
          return fail(CWB_ERR_ARG, "folded sources need weights and a signal");
        cwb_op ex;
        std::memset(&ex, 0, sizeof ex);
        ex.kind = CWB_OP_EXCITE;
        ex.a = op.c;
        ex.points = op.points;
        if ((rc = translate<T>(p, ex, slot, stream, out)))
          return rc;
      }
      if (src3.num || rec3.num) {
        cwb::TransferParams<T> tp;
        std::memset(&tp, 0, sizeof tp);
        tp.g = g;
        tp.a = to_level(op.c, bytes);
        tp.ctr = p->ctr;
        out.push_back([tp, faces3, src3, rec3](cudaStream_t s, bool adv) {
          cwb::TransferParams<T> q = tp;
          if (adv)
            q.flags |= cwb::K_ADV;
          return cwb::launch_refill3d<T>(q, faces3, src3.num ? &src3 : nullptr,
                                         rec3.num ? &rec3 : nullptr, s);
        });
      } else if (op.flags & CWB_FOLD_REFILL) {
        cwb_op rf;
        std::memset(&rf, 0, sizeof rf);
        rf.kind = CWB_OP_REFILL;
        rf.flags = refilled * OP_REFILLED;  // faces the pml launch refilled
        rf.a = op.c;
        if ((rc = translate<T>(p, rf, slot, stream, out)))
          return rc;
      }
      return CWB_OK;
    }
    dim3 grid;
    int bx, by;
    if (tma) {
      bx = ndim == 3 ? cwb::TMA_BX3 : cwb::TMA_BX2;
      by = ndim == 3 ? cwb::TMA_BY3 : 1;
      tma_grid(p, bx, by, grid, sp.chunk);
    } else {
      cwb::block_shape(ndim, bx, by);
      stencil_grid(p, grid, sp.chunk);
    }
    if (op.flags & CWB_FOLD_REFILL) {
      flags |= cwb::K_REFILL;
      sp.refill = p->grid.neumann | p->grid.dirichlet;
    }
    if ((op.flags & CWB_FOLD_SOURCES) && op.points.num > 0) {
      flags |= cwb::K_SRC;
      if (!op.points.weight || !op.points.record)
        return fail(CWB_ERR_ARG, "folded sources need weights and a signal");
      if ((rc = build_sources<T>(p, slot, op.points, grid, sp.chunk, bx, by, stream,
                                 &sp.src_start, &sp.src_entry)))
        return rc;
      sp.src_weight = static_cast<const T *>(op.points.weight);
      sp.signal = static_cast<const T *>(op.points.record);
      sp.nsrc = op.points.num;
      sp.sig_mul = op.points.row_mul;
      sp.sig_add = op.points.row_add;
    }
    sp.flags = flags;
    sp.u0 = to_level(op.a, bytes);
    sp.u1 = to_level(op.b, bytes);
    sp.u2 = to_level(op.c, bytes);
    sp.ctr = p->ctr;
    tp.err = p->err;
    if (tma) {
      out.push_back([tp, ndim, R, uniform, grid](cudaStream_t s, bool adv) {
        cwb::StepTmaParams<T> q = tp;
        if (adv)
          q.s.flags |= cwb::K_ADV;
        return step_tma_dispatch<T>(q, ndim, R, uniform, grid, s);
      });
    } else {
      out.push_back([sp, ndim, R, uniform, grid](cudaStream_t s, bool adv) {
        cwb::StepParams<T> q = sp;
        if (adv)
          q.flags |= cwb::K_ADV;
        return step_dispatch<T>(q, ndim, R, uniform, grid, s);
      });
    }
    return CWB_OK;
  }
  case CWB_OP_ADJOINT:
  case CWB_OP_GRADIENT: {
    if (op.mat.cells)
      return fail(CWB_ERR_UNSUPPORTED,
                  "the transposed and gradient kernels grade no masked wall: step a masked "
                  "domain's adjoint with CWB_OP_STEP, its own transpose");
    const bool grad_only = op.kind == CWB_OP_GRADIENT;
    cwb::AdjointParams<T> ap;
    std::memset(&ap, 0, sizeof ap);
    ap.g = g;
    fill_weights(p, ap.w, ap.f);
    ap.dt = (T)p->grid.dt;
    bool uniform;
    int flags = 0;
    const T *prof[3];
    if ((rc = fill_material<T>(p, op.mat, &ap.stiff, &ap.minv, &ap.damping, prof, ap.sconst,
                               ap.gconst, ap.dgconst, flags, uniform,
                               !grad_only && (op.flags & CWB_PML))))
      return rc;
    for (int d = 0; d < 3; ++d)
      ap.prof[d] = prof[d];
    ap.mf = (T)op.scale;
    int mode;
    if (grad_only) {
      mode = cwb::MODE_GRAD;
      if ((rc = check_level(op.a, "a")) || (rc = check_level(op.b, "b")) ||
          (rc = check_level(op.c, "c")) || (rc = check_level(op.d, "d")))
        return rc;
      if (!op.g_mass || !op.g_stiff)
        return fail(CWB_ERR_ARG, "the gradient op needs both accumulators");
      ap.u0 = to_level(op.a, bytes);
      ap.u1 = to_level(op.b, bytes);
      ap.u2 = to_level(op.c, bytes);
      ap.l1 = to_level(op.d, bytes);
      for (int d = 0; d < 3; ++d)
        ap.f[d] = d < ndim ? (T)op.factors[d] : (T)0;
    } else {
      if ((rc = check_level(op.a, "a")) || (rc = check_level(op.b, "b")))
        return rc;
      ap.l0 = to_level(op.a, bytes);
      ap.l1 = to_level(op.b, bytes);
      mode = cwb::MODE_STEP;
      if (op.flags & CWB_GRAD) {
        if ((rc = check_level(op.c, "c")))
          return rc;
        if (!op.g_mass || !op.g_stiff)
          return fail(CWB_ERR_ARG, "gradients need both accumulators");
        mode = cwb::MODE_STEP_GRAD;
        ap.u1 = to_level(op.c, bytes);
      }
      if (op.flags & CWB_PML) {
        flags |= cwb::K_PML;
        for (int d = 0; d < ndim; ++d) {
          ap.mem[d] = static_cast<T *>(op.memory[d]);
          ap.memrow[d] = (int)p->pml_row[d];
          if (lined(p, d) && !ap.mem[d])
            return fail(CWB_ERR_ARG, "a lined axis needs its adjoint pml memory");
        }
      }
    }
    ap.g_mass = static_cast<T *>(op.g_mass);
    ap.g_stiff = static_cast<T *>(op.g_stiff);
    ap.flags = flags;
    ap.ctr = p->ctr;
    // 2D, a uniform stiffness, float, radius <= 4: the quad adjoint (16-byte rows of the
    // levels, 1/m and the accumulators)
    const auto aligned16 = [](const void *ptr, const long long stride_elems) {
      return reinterpret_cast<uintptr_t>(ptr) % 16 == 0 &&
             (stride_elems * (long long)sizeof(T)) % 16 == 0;
    };
    if (ndim == 2 && mode != cwb::MODE_GRAD && p->blocked3 && uniform && step2d_built_r<T>(R) &&
        aligned16(op.a.base, op.a.stride) && aligned16(op.b.base, op.b.stride) &&
        (mode != cwb::MODE_STEP_GRAD ||
         (aligned16(op.c.base, op.c.stride) && aligned16(op.g_mass, 0) && aligned16(op.g_stiff, 0))) &&
        ((flags & cwb::K_DERIVE) || aligned16(ap.minv, 0)) && g.n[0] >= 3 * R && g.n[1] >= 3 * R) {
      // the shortest chunks that fit the grid in one wave of resident blocks: a partial
      // second wave idles most SMs for its length (measured on 2048^2 with the pml
      // gathered apart: 14 rows, one wave, 97 us a step; 9 rows, 1.5 waves, 110 us)
      const long long rows = g.n[0] - 2, quads = (g.n[1] - 2) / 4 + 1;
      const long long wave = (long long)p->sms * cwb::A2_MIN_BLOCKS * cwb::A2_THREADS;
      const int chunk = (int)std::min<long long>(rows, (rows * quads + wave - 1) / wave);
      ap.chunk = p->chunk_override > 0 ? p->chunk_override : std::max(2, chunk);
      const long long threads = quads * ((rows + ap.chunk - 1) / ap.chunk);
      const dim3 grid((unsigned)((threads + cwb::A2_THREADS - 1) / cwb::A2_THREADS));
      out.push_back([ap, R, mode, grid](cudaStream_t s, bool adv) {
        cwb::AdjointParams<T> q = ap;
        if (adv)
          q.flags |= cwb::K_ADV;
        return adjoint2d_r<T>(q, R, mode, grid, s);
      });
      if (flags & cwb::K_PML) {
        // the pml transpose over the nodes within R of a slab: the rows that axis 0's
        // slabs reach, whole, then the other rows' columns that axis 1's reach
        const int N0 = g.n[0], NF = g.n[1];
        cwb::Adj2Reach reach;
        reach.za_lo = g.lo[0] ? std::min(g.lo[0] + R, N0 - 2) : 0;
        reach.za_hi = g.hi[0] ? std::max(N0 - 1 - (g.hi[0] + R), 1) : N0 - 1;
        if (reach.za_lo >= reach.za_hi)
          reach.za_lo = N0 - 2, reach.za_hi = N0 - 1;
        reach.xb_lo = g.lo[1] ? std::min(g.lo[1] + R, NF - 2) : 0;
        reach.xb_hi = g.hi[1] ? std::max(NF - 1 - (g.hi[1] + R), 1) : NF - 1;
        if (reach.xb_lo >= reach.xb_hi)
          reach.xb_lo = NF - 2, reach.xb_hi = NF - 1;
        const long long nodes =
            (long long)(reach.za_lo + N0 - 1 - reach.za_hi) * (NF - 2) +
            (long long)(reach.za_hi - 1 - reach.za_lo) * (reach.xb_lo + NF - 1 - reach.xb_hi);
        // the adjoint load that follows this op rides on the gather where none of its nodes
        // is reached: the gather adds nothing to them, so the load applied beside it is
        // the load applied after it
        cwb::TransferParams<T> ld;
        std::memset(&ld, 0, sizeof ld);
        T *ld_mass = nullptr;
        if (next && took_next && p->load2d && next->kind == CWB_OP_LOAD && next->points.num > 0 &&
            next->points.num <= 65536 &&
            next->points.lin && next->points.weight && next->points.record &&
            next->points.store >= 0 && next->points.store <= 1 && !check_level(next->a, "a") &&
            (!next->g_mass || !check_level(next->c, "c"))) {
          const cwb_points &pt = next->points;
          std::vector<int> lin(pt.num);
          CWB_CUDA(cudaMemcpyAsync(lin.data(), pt.lin, sizeof(int) * pt.num, cudaMemcpyDeviceToHost, stream));
          CWB_CUDA(cudaStreamSynchronize(stream));
          bool clear = true;
          for (const int l : lin) {
            const int z = l / g.s[0], x = l % g.s[0];
            const bool interior = z >= 1 && z <= N0 - 2 && x >= 1 && x <= NF - 2;
            const bool reached = z <= reach.za_lo || z >= reach.za_hi || x <= reach.xb_lo || x >= reach.xb_hi;
            clear = clear && interior && !reached;
          }
          if (clear) {
            ld.g = g;
            ld.a = to_level(next->a, bytes);
            ld.lin = pt.lin;
            ld.weight = static_cast<const T *>(pt.weight);
            ld.record = pt.record;
            ld.num = pt.num;
            ld.row_mul = pt.row_mul;
            ld.row_add = pt.row_add;
            ld.store = pt.store;
            ld.ctr = p->ctr;
            if (next->g_mass) {
              ld.flags |= cwb::K_MASS;
              ld.c = to_level(next->c, bytes);
              ld.scale = (T)next->scale;
              ld_mass = static_cast<T *>(next->g_mass);
            }
            *took_next = true;
          }
        }
        const long long threads = nodes + ld.num;
        const dim3 pgrid((unsigned)std::max<long long>(1, (threads + cwb::A2P_THREADS - 1) / cwb::A2P_THREADS));
        out.push_back([ap, reach, R, mode, ld, ld_mass, pgrid](cudaStream_t s, bool adv) {
          cwb::AdjointParams<T> q = ap;
          if (adv)
            q.flags |= cwb::K_ADV;
          return adjoint2d_pml_r<T>(q, reach, R, mode, ld, ld_mass, pgrid, s);
        });
      }
      return CWB_OK;
    }
    dim3 grid;
    stencil_grid(p, grid, ap.chunk);
    // 3D with a pml: the march without the pml transpose, which a launch of its own then
    // gathers over the nodes within R of a slab (the same gather, in the same order)
    const bool split = ndim == 3 && (flags & cwb::K_PML) && mode != cwb::MODE_GRAD && p->adj_split;
    cwb::AdjointParams<T> am = ap;
    if (split)
      am.flags &= ~cwb::K_PML;
    out.push_back([am, ndim, R, uniform, mode, grid](cudaStream_t s, bool adv) {
      cwb::AdjointParams<T> q = am;
      if (adv)
        q.flags |= cwb::K_ADV;
      return adjoint_dispatch<T>(q, ndim, R, uniform, mode, grid, s);
    });
    if (split) {
      cwb::Adj3Reach reach;
      long long counts[3][2];
      for (int d = 0; d < 3; ++d) {
        const int N = g.n[d];
        reach.lo[d] = g.lo[d] ? std::min(g.lo[d] + R, N - 2) : 0;
        reach.hi[d] = g.hi[d] ? std::max(N - 1 - (g.hi[d] + R), 1) : N - 1;
        if (reach.lo[d] >= reach.hi[d])
          reach.lo[d] = N - 2, reach.hi[d] = N - 1;
        counts[d][0] = reach.lo[d] + (N - 1 - reach.hi[d]);  // reached
        counts[d][1] = N - 2 - counts[d][0];                 // not
      }
      const long long nodes = counts[0][0] * (g.n[1] - 2) * (g.n[2] - 2) +
                              counts[0][1] * counts[1][0] * (g.n[2] - 2) +
                              counts[0][1] * counts[1][1] * counts[2][0];
      const dim3 pgrid((unsigned)std::max<long long>(1, (nodes + cwb::A3P_THREADS - 1) / cwb::A3P_THREADS));
      out.push_back([ap, reach, R, uniform, mode, pgrid](cudaStream_t s, bool adv) {
        cwb::AdjointParams<T> q = ap;
        if (adv)
          q.flags |= cwb::K_ADV;
        return adjoint3d_pml_r<T>(q, reach, R, uniform, mode, pgrid, s);
      });
    }
    return CWB_OK;
  }
  case CWB_OP_FRECHET: {
    if ((rc = check_level(op.a, "a")) || (rc = check_level(op.b, "b")) ||
        (rc = check_level(op.c, "c")))
      return rc;
    if (!op.g_mass || !op.g_stiff)
      return fail(CWB_ERR_ARG, "the Frechet densities need both accumulators");
    cwb::FrechetParams<T> fp;
    std::memset(&fp, 0, sizeof fp);
    fp.g = g;
    fp.a = to_level(op.a, bytes);
    fp.b = to_level(op.b, bytes);
    fp.c = to_level(op.c, bytes);
    fp.acc_mass = static_cast<T *>(op.g_mass);
    fp.acc_stiff = static_cast<T *>(op.g_stiff);
    fp.ft = (T)op.scale;
    for (int d = 0; d < 3; ++d)
      fp.F[d] = (T)op.factors[d];
    fp.ctr = p->ctr;
    out.push_back([fp](cudaStream_t s, bool adv) {
      cwb::FrechetParams<T> q = fp;
      q.flags = adv ? cwb::K_ADV : 0;
      return cwb::launch_frechet<T>(q, s);
    });
    return CWB_OK;
  }
  case CWB_OP_PML_AUX: {
    if ((rc = check_level(op.a, "a")))
      return rc;
    const T *stiff, *minv, *damping, *prof[3];
    T sconst, gconst, dgconst;
    bool uniform;
    int flags = 0;
    if ((rc = fill_material<T>(p, op.mat, &stiff, &minv, &damping, prof, sconst, gconst,
                               dgconst, flags, uniform, true)))
      return rc;
    cwb::PmlAuxSet<T> set;
    std::memset(&set, 0, sizeof set);
    set.ctr = p->ctr;
    for (int d = 0; d < ndim; ++d) {
      if (!lined(p, d))
        continue;
      cwb::PmlAuxParams<T> pa;
      std::memset(&pa, 0, sizeof pa);
      pa.g = g;
      pa.f = (T)p->grid.factors[d];
      pa.d = d;
      pa.l1 = to_level(op.a, bytes);
      pa.stiff = stiff;
      pa.minv = minv;
      pa.prof = prof[d];
      pa.mem = static_cast<T *>(op.memory[d]);
      if (!pa.mem)
        return fail(CWB_ERR_ARG, "a lined axis needs its adjoint pml memory");
      pa.memrow = (int)p->pml_row[d];
      pa.sconst = sconst;
      pa.uniform = uniform;
      pa.ctr = p->ctr;
      set.ax[set.nax] = pa;
      set.first[set.nax + 1] =
          set.first[set.nax] + (pa.memrow + cwb::TRANSFER_THREADS - 1) / cwb::TRANSFER_THREADS;
      ++set.nax;
    }
    if (set.nax)
      out.push_back([set](cudaStream_t s, bool adv) {
        cwb::PmlAuxSet<T> q = set;
        q.flags = adv ? cwb::K_ADV : 0;
        return cwb::launch_pml_aux<T>(q, s);
      });
    return CWB_OK;
  }
  case CWB_OP_EXCITE:
  case CWB_OP_LOAD:
  case CWB_OP_RECORD:
  case CWB_OP_REPLAY:
  case CWB_OP_DFT:
  case CWB_OP_REFILL: {
    if ((rc = check_level(op.a, "a")))
      return rc;
    cwb::TransferParams<T> tp;
    std::memset(&tp, 0, sizeof tp);
    tp.g = g;
    tp.a = to_level(op.a, bytes);
    tp.ctr = p->ctr;
    int kind, total = 0, faces = 0;
    T *g_mass = nullptr;
    if (op.kind == CWB_OP_REFILL) {
      kind = cwb::TR_REFILL;
      faces = p->grid.neumann | p->grid.dirichlet;
      // an internal refill after the pml launch: the faces that launch refilled are left out
      faces &= ~((op.flags / OP_REFILLED) & 63);
      for (int d = 0; d < ndim; ++d) {
        int face = 1;
        for (int e = 0; e < ndim; ++e)
          if (e != d)
            face *= g.n[e] - 2;
        total += face * (((faces >> (2 * d)) & 1) + ((faces >> (2 * d + 1)) & 1));
      }
    } else {
      const cwb_points &pt = op.points;
      if (pt.num <= 0)
        return CWB_OK;  // nothing to move
      if (!pt.lin || !pt.record)
        return fail(CWB_ERR_ARG, "a transfer needs indices and a record");
      if (pt.store < 0 || pt.store > 2 || (pt.store == 2 && sizeof(T) == 4))
        return fail(CWB_ERR_ARG, "unknown record storage");
      tp.lin = pt.lin;
      tp.weight = static_cast<const T *>(pt.weight);
      tp.record = pt.record;
      tp.num = pt.num;
      tp.row_mul = pt.row_mul;
      tp.row_add = pt.row_add;
      tp.store = pt.store;
      total = pt.num;
      if (op.kind == CWB_OP_EXCITE || op.kind == CWB_OP_LOAD) {
        if (!pt.weight)
          return fail(CWB_ERR_ARG, "an excitation needs weights");
      }
      kind = op.kind == CWB_OP_EXCITE   ? cwb::TR_EXCITE
             : op.kind == CWB_OP_LOAD   ? cwb::TR_LOAD
             : op.kind == CWB_OP_RECORD ? cwb::TR_RECORD
             : op.kind == CWB_OP_DFT    ? cwb::TR_DFT
                                        : cwb::TR_REPLAY;
      if (op.kind == CWB_OP_DFT) {
        if (!op.g_mass || op.columns <= 0 || pt.store != 0)
          return fail(CWB_ERR_ARG, "a DFT needs an accumulator, its columns and a native table");
        tp.columns = op.columns;
        g_mass = static_cast<T *>(op.g_mass);
      }
      if (op.kind == CWB_OP_LOAD && op.g_mass) {
        if ((rc = check_level(op.c, "c")))
          return rc;
        tp.flags |= cwb::K_MASS;
        tp.c = to_level(op.c, bytes);
        tp.scale = (T)op.scale;
        g_mass = static_cast<T *>(op.g_mass);
      }
    }
    if (total <= 0)
      return CWB_OK;
    out.push_back([tp, kind, g_mass, faces, total](cudaStream_t s, bool adv) {
      cwb::TransferParams<T> q = tp;
      if (adv)
        q.flags |= cwb::K_ADV;
      return cwb::launch_transfer<T>(kind, q, g_mass, faces, total, s);
    });
    return CWB_OK;
  }
  }
  return fail(CWB_ERR_ARG, "unknown op kind " + std::to_string(op.kind));
}

int enqueue_step(const std::vector<Launch> &launches, cudaStream_t s) {
  for (size_t i = 0; i < launches.size(); ++i) {
    const cudaError_t e = launches[i](s, i + 1 == launches.size());
    if (e != cudaSuccess)
      return fail(CWB_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  }
  g_launches += (long long)launches.size();
  return CWB_OK;
}

template <typename T>
cudaError_t march3d_r(const cwb::March3Params<T> &mp, const int R, const bool uniform,
                      const int sms, cudaStream_t s) {
  switch (R) {
  case 1: return cwb::march3d_unit<T, 1>(mp, uniform, sms, s);
  case 2: return cwb::march3d_unit<T, 2>(mp, uniform, sms, s);
  case 3: return cwb::march3d_unit<T, 3>(mp, uniform, sms, s);
  case 4: return cwb::march3d_unit<T, 4>(mp, uniform, sms, s);
  case 5: return cwb::march3d_unit<T, 5>(mp, uniform, sms, s);
  case 6: return cwb::march3d_unit<T, 6>(mp, uniform, sms, s);
  case 7: return cwb::march3d_unit<T, 7>(mp, uniform, sms, s);
  case 8: return cwb::march3d_unit<T, 8>(mp, uniform, sms, s);
  }
  return cudaErrorInvalidValue;
}

// A 3D op list [step (sources and refill folded), records] on a grid small enough for its
// fields to stay in L2 runs as one cooperative launch of all its steps (march3d_kernel:
// the generic tile step, a grid barrier before the records). Returns false where the
// list is another shape or the grid too large, leaving it to the per-step march.
template <typename T>
bool march3d_path(cwb_plan *p, const cwb_op *ops, const int nops, const int t0, const int steps,
                  cudaStream_t user, int &rc) {
  const Geometry &g = p->geo;
  const int R = p->grid.radius;
  if (!p->march3 || g.ndim != 3 || steps < 16 || nops < 1 || nops > 1 + cwb::MARCH3_RECORDS ||
      ops[0].kind != CWB_OP_STEP || ops[0].mat.cells || !(ops[0].flags & CWB_FOLD_REFILL))
    return false;
  for (int i = 1; i < nops; ++i)
    if (ops[i].kind != CWB_OP_RECORD || ops[i].points.num <= 0 || !ops[i].points.lin ||
        !ops[i].points.record || ops[i].points.store < 0 || ops[i].points.store > 2 ||
        (ops[i].points.store == 2 && sizeof(T) == 4) || check_level(ops[i].a, "a"))
      return false;
  // fields L2 holds between steps, where a step's launches cost more than its work
  const long long field = (long long)g.n[0] * g.n[1] * g.ext[2] * (long long)sizeof(T);
  if (p->march3 < 2 && 3 * field > p->march3_bytes)
    return false;
  const cwb_op &op = ops[0];
  cwb::March3Params<T> mp;
  std::memset(&mp, 0, sizeof mp);
  cwb::StepParams<T> &sp = mp.s;
  int flags = 0;
  bool uniform = false;
  if (step_setup<T>(p, op, sp, flags, uniform))
    return false;
  const int bytes = sizeof(T);
  int bx, by;
  cwb::block_shape(3, bx, by);
  const int gx = (g.ext[2] + bx - 1) / bx, gy = (g.n[1] + by - 1) / by;
  const int rows = g.n[0] - 2;
  // about two tiles a resident block slot, no chunk under two planes
  const long long want = 2LL * p->sms;
  int chunk = (int)std::max<long long>(2, ((long long)rows * gx * gy + want - 1) / want);
  if (p->chunk_override > 0)
    chunk = p->chunk_override;
  chunk = std::min(chunk, rows);
  const int gz = (rows + chunk - 1) / chunk;
  sp.chunk = chunk;
  flags |= cwb::K_REFILL;
  sp.refill = p->grid.neumann | p->grid.dirichlet;
  rc = CWB_OK;
  if ((op.flags & CWB_FOLD_SOURCES) && op.points.num > 0) {
    if (!op.points.weight || !op.points.record)
      return rc = fail(CWB_ERR_ARG, "folded sources need weights and a signal"), true;
    flags |= cwb::K_SRC;
    if ((rc = build_sources<T>(p, 0, op.points, dim3(gx, gy, gz), chunk, bx, by, user,
                               &sp.src_start, &sp.src_entry)))
      return true;
    sp.src_weight = static_cast<const T *>(op.points.weight);
    sp.signal = static_cast<const T *>(op.points.record);
    sp.nsrc = op.points.num;
    sp.sig_mul = op.points.row_mul;
    sp.sig_add = op.points.row_add;
  }
  sp.flags = flags;
  sp.u0 = to_level(op.a, bytes);
  sp.u1 = to_level(op.b, bytes);
  sp.u2 = to_level(op.c, bytes);
  sp.ctr = p->ctr;
  mp.nbx = gx;
  mp.nby = gy;
  mp.nbz = gz;
  mp.nrec = nops - 1;
  for (int i = 1; i < nops; ++i) {
    cwb::TransferParams<T> &tp = mp.rec[i - 1];
    tp.g = g;
    tp.a = to_level(ops[i].a, bytes);
    tp.lin = ops[i].points.lin;
    tp.record = ops[i].points.record;
    tp.num = ops[i].points.num;
    tp.row_mul = ops[i].points.row_mul;
    tp.row_add = ops[i].points.row_add;
    tp.store = ops[i].points.store;
    tp.ctr = p->ctr;
  }
  mp.t0 = t0;
  mp.steps = steps;
  const auto run = [&]() -> int {
    CWB_CUDA(cudaEventRecord(p->fork, user));
    CWB_CUDA(cudaStreamWaitEvent(p->lane, p->fork, 0));
    cudaStream_t s = p->lane;
    CWB_CUDA(cwb::launch_set_counter(p->ctr, t0, s));
    CWB_CUDA(march3d_r<T>(mp, R, uniform, p->sms, s));
    g_launches += 2;
    CWB_CUDA(cudaEventRecord(p->join, s));
    CWB_CUDA(cudaStreamWaitEvent(user, p->join, 0));
    return CWB_OK;
  };
  rc = run();
  return true;
}

template <typename T>
cudaError_t march2d_r(const cwb::March2Params<T> &mp, const int R, const int sms, cudaStream_t s) {
  switch (R) {
  case 1: return cwb::march2d_unit<T, 1>(mp, sms, s);
  case 2: return cwb::march2d_unit<T, 2>(mp, sms, s);
  case 3: return cwb::march2d_unit<T, 3>(mp, sms, s);
  case 4: return cwb::march2d_unit<T, 4>(mp, sms, s);
  case 5: return cwb::march2d_unit<T, 5>(mp, sms, s);
  case 6: return cwb::march2d_unit<T, 6>(mp, sms, s);
  case 7: return cwb::march2d_unit<T, 7>(mp, sms, s);
  case 8: return cwb::march2d_unit<T, 8>(mp, sms, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t tblock2d_r(const cwb::TBlock2Params<float> &tp, const int R, const dim3 grid,
                       cudaStream_t s) {
  switch (R) {
  case 1: return cwb::tblock2d_unit<T, 1>(tp, grid, s);
  case 2: return cwb::tblock2d_unit<T, 2>(tp, grid, s);
  case 3: return cwb::tblock2d_unit<T, 3>(tp, grid, s);
  case 4: return cwb::tblock2d_unit<T, 4>(tp, grid, s);
  }
  return cudaErrorInvalidValue;
}

// A 2D op list [step, records] of a uniform stiffness (float) runs as one
// cooperative launch of all its steps, sources and refill folded into the step and a
// grid-wide barrier before the records (march2d_kernel). Returns false where the list is
// another shape, leaving it to the per-step march.
template <typename T>
bool march2d_path(cwb_plan *p, const cwb_op *ops, const int nops, const int t0, const int steps,
                  cudaStream_t user, int &rc) {
  const Geometry &g = p->geo;
  const int R = p->grid.radius;
  if (!p->blocked3 || g.ndim != 2 || steps < 16 || nops < 1 || nops > 1 + cwb::MARCH2_RECORDS ||
      ops[0].kind != CWB_OP_STEP || ops[0].mat.cells || !step2d_built_r<T>(R) ||
      g.n[0] < 3 * R || g.n[1] < 3 * R)
    return false;
  for (int i = 1; i < nops; ++i)
    if (ops[i].kind != CWB_OP_RECORD || ops[i].points.num <= 0 || !ops[i].points.lin ||
        !ops[i].points.record || ops[i].points.store < 0 || ops[i].points.store > 2 ||
        (ops[i].points.store == 2 && sizeof(T) == 4) || check_level(ops[i].a, "a"))
      return false;
  const cwb_op &op = ops[0];
  const cwb_points &src = op.points;
  if ((op.flags & CWB_FOLD_SOURCES) && src.num > 0 &&
      (src.num > 32 || !src.lin || !src.weight || !src.record))
    return false;
  cwb::March2Params<T> mp;
  std::memset(&mp, 0, sizeof mp);
  cwb::StepParams<T> &sp = mp.s;
  int flags = 0;
  bool uniform = false;
  if (step_setup<T>(p, op, sp, flags, uniform) || !uniform)
    return false;
  const auto aligned16 = [](const void *ptr, const long long stride_elems) {
    return reinterpret_cast<uintptr_t>(ptr) % 16 == 0 && (stride_elems * (long long)sizeof(T)) % 16 == 0;
  };
  if (!aligned16(op.a.base, op.a.stride) || !aligned16(op.b.base, op.b.stride) ||
      !aligned16(op.c.base, op.c.stride) || (!(flags & cwb::K_DERIVE) && !aligned16(sp.minv, 0)))
    return false;
  const int bytes = sizeof(T);
  const long long rows = g.n[0] - 2, quads = (g.n[1] - 2) / 4 + 1;
  // a grid whose rows the co-resident threads cover about once: larger ones keep more
  // rows in flight launched step by step (measured: 512^2 10.8 us a step here against
  // 16 us launched; 2048^2 69 us against 52 us)
  if (rows * quads > (long long)p->sms * 1024)
    return false;
  const long long want = (long long)p->sms * 1024;
  sp.chunk = (int)std::max<long long>(1, std::min<long long>(rows, rows * quads / want));
  if (p->chunk_override > 0)
    sp.chunk = p->chunk_override;
  sp.flags = flags;
  sp.u0 = to_level(op.a, bytes);
  sp.u1 = to_level(op.b, bytes);
  sp.u2 = to_level(op.c, bytes);
  sp.ctr = p->ctr;
  mp.units = quads * ((rows + sp.chunk - 1) / sp.chunk);
  if ((op.flags & CWB_FOLD_SOURCES) && src.num > 0) {
    mp.fold.lin = src.lin;
    mp.fold.weight = static_cast<const T *>(src.weight);
    mp.fold.signal = static_cast<const T *>(src.record);
    mp.fold.nsrc = src.num;
    mp.fold.sig_mul = src.row_mul;
    mp.fold.sig_add = src.row_add;
  }
  if (op.flags & CWB_FOLD_REFILL)
    mp.fold.refill = p->grid.neumann | p->grid.dirichlet;
  mp.nrec = nops - 1;
  for (int i = 1; i < nops; ++i) {
    cwb::TransferParams<T> &tp = mp.rec[i - 1];
    tp.g = g;
    tp.a = to_level(ops[i].a, bytes);
    tp.lin = ops[i].points.lin;
    tp.record = ops[i].points.record;
    tp.num = ops[i].points.num;
    tp.row_mul = ops[i].points.row_mul;
    tp.row_add = ops[i].points.row_add;
    tp.store = ops[i].points.store;
    tp.ctr = p->ctr;
  }
  mp.t0 = t0;
  mp.steps = steps;
  rc = CWB_OK;
  const auto run = [&]() -> int {
    CWB_CUDA(cudaEventRecord(p->fork, user));
    CWB_CUDA(cudaStreamWaitEvent(p->lane, p->fork, 0));
    cudaStream_t s = p->lane;
    CWB_CUDA(cwb::launch_set_counter(p->ctr, t0, s));
    CWB_CUDA(march2d_r<T>(mp, R, p->sms, s));
    g_launches += 2;
    CWB_CUDA(cudaEventRecord(p->join, s));
    CWB_CUDA(cudaStreamWaitEvent(user, p->join, 0));
    return CWB_OK;
  };
  rc = run();
  return true;
}

// per-block lists (CSR) uploaded into a plan scratch: starts[nblocks + 1], entries
int upload_lists(Scratch &sc, const std::vector<std::vector<int4>> &per, cudaStream_t s) {
  std::vector<int> starts(per.size() + 1, 0);
  std::vector<int4> entries;
  for (size_t b = 0; b < per.size(); ++b) {
    entries.insert(entries.end(), per[b].begin(), per[b].end());
    starts[b + 1] = (int)entries.size();
  }
  if (entries.empty())
    entries.push_back(make_int4(-1, -1, 0, 0));
  if (sc.start_cap < starts.size()) {
    if (sc.start)
      cudaFree(sc.start);
    sc.start = nullptr;
    if (cudaMalloc(&sc.start, sizeof(int) * starts.size()) != cudaSuccess)
      return fail(CWB_ERR_ALLOC, "list allocation failed");
    sc.start_cap = starts.size();
  }
  if (sc.entry_cap < entries.size()) {
    if (sc.entry)
      cudaFree(sc.entry);
    sc.entry = nullptr;
    if (cudaMalloc(&sc.entry, sizeof(int4) * entries.size()) != cudaSuccess)
      return fail(CWB_ERR_ALLOC, "list allocation failed");
    sc.entry_cap = entries.size();
  }
  CWB_CUDA(cudaMemcpyAsync(sc.start, starts.data(), sizeof(int) * starts.size(),
                           cudaMemcpyHostToDevice, s));
  CWB_CUDA(cudaMemcpyAsync(sc.entry, entries.data(), sizeof(int4) * entries.size(),
                           cudaMemcpyHostToDevice, s));
  CWB_CUDA(cudaStreamSynchronize(s));
  return CWB_OK;
}

// A 2D op list [step (sources and refill folded), records] of a uniform stiffness
// (float, radius <= 4, no damping; a pml or none) on a grid too large for L2, its levels
// the two slots a simulation rotates (u^s in slot (s + add) mod 2), runs TB_K steps per
// pass over HBM (tblock2d_kernel): the passes alternate between the caller's slots and
// the plan's second pair (the pml memory around a ring of K + 1 copies), the last result
// is copied back, and the steps short of a whole pass are left to the per-step march.
// Returns false where the list is another shape.
bool tblock2d_path(cwb_plan *p, const cwb_op *ops, const int nops, const int t0, int &steps,
                   cudaStream_t user, int &rc, int &done) {
  using T = float;
  constexpr int K = cwb::TB_K;
  const Geometry &g = p->geo;
  const int R = p->grid.radius;
  done = 0;
  if (!p->tblock || p->fixed || p->grid.precision != 4 || g.ndim != 2 || R > 4 ||
      steps < 2 * K || nops < 1 || nops > 1 + cwb::TB_RECORDS || ops[0].kind != CWB_OP_STEP ||
      ops[0].mat.cells || !(ops[0].flags & CWB_FOLD_REFILL) ||
      ((p->grid.neumann | p->grid.dirichlet) & 15) != 15 || g.n[0] < 3 * R + 2 || g.n[1] < 3 * R + 2)
    return false;
  const cwb_op &op = ops[0];
  // the two slots a simulation rotates: a and c the same slot, b the other
  const cwb_level &A = op.a, &B = op.b, &C = op.c;
  if (A.base != B.base || A.base != C.base || A.stride != B.stride || A.stride != C.stride ||
      A.period != 2 || B.period != 2 || C.period != 2 || A.mul != 1 || B.mul != 1 || C.mul != 1 ||
      ((A.add - C.add) % 2) != 0 || (((B.add - C.add) % 2 + 2) % 2) != 1)
    return false;
  for (int i = 1; i < nops; ++i) {
    const cwb_points &pt = ops[i].points;
    if (ops[i].kind != CWB_OP_RECORD || pt.num <= 0 || !pt.lin || !pt.record || pt.store < 0 ||
        pt.store > 1 || ops[i].a.base != C.base || ops[i].a.stride != C.stride ||
        ops[i].a.period != 2 || ops[i].a.mul != 1 || ((ops[i].a.add - C.add) % 2) != 0)
      return false;
  }
  cwb::TBlock2Params<T> tp;
  std::memset(&tp, 0, sizeof tp);
  cwb::StepParams<T> &sp = tp.s;
  int flags = 0;
  bool uniform = false;
  if (step_setup<T>(p, op, sp, flags, uniform) || !uniform || (flags & cwb::K_DAMP))
    return false;
  const auto aligned16 = [](const void *ptr, const long long stride_elems) {
    return reinterpret_cast<uintptr_t>(ptr) % 16 == 0 && (stride_elems * (long long)sizeof(T)) % 16 == 0;
  };
  if (!aligned16(A.base, A.stride) || (!(flags & cwb::K_DERIVE) && !aligned16(sp.minv, 0)))
    return false;
  const long long rows = g.n[0] - 2, quads = (g.n[1] - 2) / 4 + 1;
  // grids L2 holds step well one step a launch; this pays where the fields stream from HBM.
  // With a pml it is bit-exact but slower than one step a launch on every grid measured
  // (2048^2 .. 8192^2, 20-cell slabs): only CWB_TBLOCK=2 takes it
  if (p->tblock < 2 && ((flags & cwb::K_PML) ||
                        rows * quads * 4 * (long long)sizeof(T) * 3 < 96LL * 1024 * 1024))
    return false;
  const int qx_step = cwb::TB_TQ - 2 * K;
  const int gx = (int)((quads + qx_step - 1) / qx_step);
  // rows per block: about two waves of blocks two a SM, no fewer than 64
  const long long want_blocks = 4LL * p->sms;
  int chunk = (int)std::max<long long>(64, (rows * gx + want_blocks - 1) / want_blocks);
  if (p->chunk_override > 0)
    chunk = p->chunk_override;
  chunk = (int)std::min<long long>(chunk, rows);
  const int gy = (int)((rows + chunk - 1) / chunk);
  const int nblocks = gx * gy;
  const int N0 = g.n[0];
  sp.flags = flags;
  sp.ctr = p->ctr;
  tp.chunk = chunk;
  tp.qx_step = qx_step;
  tp.refill = p->grid.neumann | p->grid.dirichlet;
  rc = CWB_OK;
  // the per-block lists: sources over the rows and quads a block steps, receivers over
  // the nodes it owns
  const auto block_rows = [&](const int by, int &lo, int &hi, int &own_lo, int &own_hi) {
    own_lo = 1 + by * chunk;
    own_hi = std::min(N0 - 1, own_lo + chunk);
    lo = std::max(1, own_lo - (K - 1) * R);
    hi = std::min(N0 - 1, own_hi + (K - 1) * R);
  };
  const auto copy_lin = [&](const int *lin, const int num, std::vector<int> &out) -> int {
    out.resize(num);
    if (num) {
      CWB_CUDA(cudaMemcpyAsync(out.data(), lin, sizeof(int) * num, cudaMemcpyDeviceToHost, user));
      CWB_CUDA(cudaStreamSynchronize(user));
    }
    return CWB_OK;
  };
  const int s0 = g.s[0];
  const cwb_points &src = op.points;
  if ((op.flags & CWB_FOLD_SOURCES) && src.num > 0) {
    if (!src.weight || !src.record)
      return rc = fail(CWB_ERR_ARG, "folded sources need weights and a signal"), true;
    std::vector<int> lin;
    if ((rc = copy_lin(src.lin, src.num, lin)))
      return true;
    std::vector<std::vector<int4>> per(nblocks);
    for (int e = 0; e < src.num; ++e) {
      const int r = lin[e] / s0, x = lin[e] % s0;
      if (r < 1 || r > N0 - 2 || x < 1 || x > g.n[1] - 2)
        return rc = fail(CWB_ERR_ARG, "a folded source must sit on an interior node"), true;
      for (int by = 0; by < gy; ++by) {
        int lo, hi, olo, ohi;
        block_rows(by, lo, hi, olo, ohi);
        if (r < lo || r >= hi)
          continue;
        for (int bx = 0; bx < gx; ++bx) {
          const int q0 = bx * qx_step - K, q = x / 4;
          if (q >= q0 && q < q0 + cwb::TB_TQ)
            per[by * gx + bx].push_back(make_int4(r, x, e, 0));
        }
      }
    }
    if ((rc = upload_lists(p->tb_src, per, user)))
      return true;
    tp.src_start = p->tb_src.start;
    tp.src_entry = p->tb_src.entry;
    tp.src_weight = static_cast<const T *>(src.weight);
    tp.signal = static_cast<const T *>(src.record);
    tp.nsrc = src.num;
    tp.sig_mul = src.row_mul;
    tp.sig_add = src.row_add;
  }
  tp.nrec = nops - 1;
  if (tp.nrec) {
    std::vector<std::vector<int4>> per(nblocks);
    for (int i = 1; i < nops; ++i) {
      const cwb_points &pt = ops[i].points;
      std::vector<int> lin;
      if ((rc = copy_lin(pt.lin, pt.num, lin)))
        return true;
      for (int j = 0; j < pt.num; ++j) {
        const int r = lin[j] / s0, x = lin[j] % s0;
        if (r < 1 || r > N0 - 2 || x < 1 || x > g.n[1] - 2)
          return false;  // a receiver off the interior: the per-step march records it
        const int by = (r - 1) / chunk, bx = (x / 4) / qx_step;
        per[by * gx + bx].push_back(make_int4(r, x, j, i - 1));
      }
      cwb::TransferParams<T> &rp = tp.rec[i - 1];
      rp.g = g;
      rp.lin = pt.lin;
      rp.record = pt.record;
      rp.num = pt.num;
      rp.row_mul = pt.row_mul;
      rp.row_add = pt.row_add;
      rp.store = pt.store;
    }
    for (auto &v : per)
      std::stable_sort(v.begin(), v.end(), [](const int4 &a, const int4 &b) { return a.x < b.x; });
    if ((rc = upload_lists(p->tb_rec, per, user)))
      return true;
    tp.rec_start = p->tb_rec.start;
    tp.rec_entry = p->tb_rec.entry;
  }
  // the second pair of slots, a copy of the caller's so the nodes no pass writes (corner
  // ghosts, padding) match
  const size_t slot_bytes = (size_t)A.stride * sizeof(T);
  if (p->tb_fields_bytes < 2 * slot_bytes) {
    if (p->tb_fields)
      cudaFree(p->tb_fields);
    p->tb_fields = nullptr;
    p->tb_fields_bytes = 0;
    if (cudaMalloc(&p->tb_fields, 2 * slot_bytes) != cudaSuccess)
      return rc = fail(CWB_ERR_ALLOC, "temporal blocking's second slots"), true;
    p->tb_fields_bytes = 2 * slot_bytes;
  }
  // with a pml, K + 1 copies of the memory of axes 0 and 1 in a ring: the plan's own
  // (copy 0) and K of the plan's scratch; a pass reads copy `in` and its level j writes
  // copy in + j, so the next pass reads copy in + K (mod K + 1)
  const bool pml = flags & cwb::K_PML;
  size_t psi_copy = 0;  // floats of one copy, both axes
  size_t psi_off[2] = {0, 0};
  for (int d = 0; d < 2 && pml; ++d) {
    psi_off[d] = psi_copy;
    if (sp.aux[d])
      psi_copy += 3 * (size_t)sp.auxrow[d];
  }
  if (pml && p->tb_psi_bytes < K * psi_copy * sizeof(T)) {
    if (p->tb_psi)
      cudaFree(p->tb_psi);
    p->tb_psi = nullptr;
    p->tb_psi_bytes = 0;
    if (cudaMalloc(&p->tb_psi, K * psi_copy * sizeof(T)) != cudaSuccess)
      return rc = fail(CWB_ERR_ALLOC, "temporal blocking's copies of the pml memory"), true;
    p->tb_psi_bytes = K * psi_copy * sizeof(T);
  }
  const auto psi_at = [&](const int copy, const int d) -> T * {
    if (!pml || !sp.aux[d])
      return nullptr;
    if (copy == 0)
      return sp.aux[d];
    return static_cast<T *>(p->tb_psi) + (size_t)(copy - 1) * psi_copy + psi_off[d];
  };
  T *mine[2] = {static_cast<T *>(A.base), static_cast<T *>(A.base) + A.stride};
  T *other[2] = {static_cast<T *>(p->tb_fields), static_cast<T *>(p->tb_fields) + A.stride};
  const auto slot_of = [&](const int m) { return ((m + C.add) % 2 + 2) % 2; };  // u^m's slot
  const int passes = steps / K;
  const auto run = [&]() -> int {
    CWB_CUDA(cudaEventRecord(p->fork, user));
    CWB_CUDA(cudaStreamWaitEvent(p->lane, p->fork, 0));
    cudaStream_t s = p->lane;
    CWB_CUDA(cudaMemcpyAsync(other[0], mine[0], 2 * slot_bytes, cudaMemcpyDeviceToDevice, s));
    int in = 0;  // the pml memory copy the pass reads
    for (int k = 0; k < passes; ++k) {
      const int t = t0 + k * K;
      T **from = k % 2 ? other : mine, **to = k % 2 ? mine : other;
      for (int j = 0; j <= K; ++j)
        for (int d = 0; d < 2; ++d)
          tp.psi[j][d] = psi_at((in + j) % (K + 1), d);
      in = (in + K) % (K + 1);
      tp.t = t;
      tp.A = from[slot_of(t - 2)];
      tp.B = from[slot_of(t - 1)];
      tp.outA = to[slot_of(t + K - 2)];
      tp.outB = to[slot_of(t + K - 1)];
      CWB_CUDA(tblock2d_r<T>(tp, R, dim3(gx, gy), s));
      ++g_launches;
    }
    if (passes % 2)
      CWB_CUDA(cudaMemcpyAsync(mine[0], other[0], 2 * slot_bytes, cudaMemcpyDeviceToDevice, s));
    for (int d = 0; d < 2 && in != 0; ++d)
      if (psi_at(0, d))
        CWB_CUDA(cudaMemcpyAsync(psi_at(0, d), psi_at(in, d), 3 * (size_t)sp.auxrow[d] * sizeof(T),
                                 cudaMemcpyDeviceToDevice, s));
    CWB_CUDA(cudaEventRecord(p->join, s));
    CWB_CUDA(cudaStreamWaitEvent(user, p->join, 0));
    return CWB_OK;
  };
  rc = run();
  done = passes * K;
  return true;
}

template <typename T>
int march(cwb_plan *p, const cwb_op *ops, const int nops, const int t0, const int steps,
          const int graph, cudaStream_t user) {
  {
    // small 2D grids: all steps in one cooperative launch; large ones: TB_K steps per
    // pass over HBM (CWB_TBLOCK=2 takes that path first, whatever the grid's size)
    int rc = CWB_OK, done = 0, left = steps;
    const auto blocked = [&]() {
      return sizeof(T) == 4 && tblock2d_path(p, ops, nops, t0, left, user, rc, done);
    };
    if (p->tblock == 2 && blocked()) {
      if (rc || done == steps)
        return rc;
      return march<T>(p, ops, nops, t0 + done, steps - done, graph, user);
    }
    if (march2d_path<T>(p, ops, nops, t0, steps, user, rc))
      return rc;
    if (march3d_path<T>(p, ops, nops, t0, steps, user, rc))
      return rc;
    if (p->tblock == 1 && blocked()) {
      if (rc || done == steps)
        return rc;
      return march<T>(p, ops, nops, t0 + done, steps - done, graph, user);
    }
  }
  std::vector<Launch> launches;
  for (int i = 0; i < nops; ++i) {
    // the adjoint's pml memory [PML_AUX, ADJOINT with its gather apart]: the memory launch
    // reads lambda^(n+1) and writes only the memory, which the march neither reads nor
    // writes; it runs beside the march on the side stream and the gather, which reads the
    // memory, waits for it
    if (p->aux_par && p->side && ops[i].kind == CWB_OP_PML_AUX && i + 1 < nops &&
        ops[i + 1].kind == CWB_OP_ADJOINT) {
      std::vector<Launch> aux, adj;
      bool took = false;
      int rc = translate<T>(p, ops[i], (size_t)i, user, aux);
      if (!rc)
        rc = translate<T>(p, ops[i + 1], (size_t)(i + 1), user, adj, i + 2 < nops ? &ops[i + 2] : nullptr,
                          &took);
      if (rc)
        return rc;
      if (aux.size() == 1 && adj.size() == 2) {
        const Launch mem = aux[0], gather = adj[1];
        cudaStream_t side = p->side;
        cudaEvent_t sf = p->side_fork, sj = p->side_join;
        launches.push_back([mem, side, sf](cudaStream_t s, bool) {
          cudaError_t e = cudaEventRecord(sf, s);
          if (e == cudaSuccess)
            e = cudaStreamWaitEvent(side, sf, 0);
          return e == cudaSuccess ? mem(side, false) : e;  // never a step's last launch
        });
        launches.push_back(adj[0]);
        launches.push_back([gather, side, sj](cudaStream_t s, bool adv) {
          cudaError_t e = cudaEventRecord(sj, side);
          if (e == cudaSuccess)
            e = cudaStreamWaitEvent(s, sj, 0);
          return e == cudaSuccess ? gather(s, adv) : e;
        });
      } else {
        launches.insert(launches.end(), aux.begin(), aux.end());
        launches.insert(launches.end(), adj.begin(), adj.end());
      }
      i += took ? 2 : 1;
      continue;
    }
    // an op may take the one after it into its own launches (the 2D adjoint its load)
    bool took = false;
    const int rc = translate<T>(p, ops[i], (size_t)i, user, launches, i + 1 < nops ? &ops[i + 1] : nullptr,
                                &took);
    if (rc)
      return rc;
    if (took)
      ++i;
  }
  if (launches.empty() || steps <= 0)
    return CWB_OK;
  // the march runs on the plan's own stream, ordered after and before the caller's
  CWB_CUDA(cudaEventRecord(p->fork, user));
  CWB_CUDA(cudaStreamWaitEvent(p->lane, p->fork, 0));
  cudaStream_t s = p->lane;
  CWB_CUDA(cudaMemsetAsync(p->err, 0, sizeof(int), s));
  CWB_CUDA(cwb::launch_set_counter(p->ctr, t0, s));
  ++g_launches;
  int done = 0;
  if (graph && steps >= 2 * GRAPH_STEPS) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    CWB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int rc = CWB_OK;
    for (int k = 0; k < GRAPH_STEPS && !rc; ++k)
      rc = enqueue_step(launches, s);
    const cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (rc)
      return rc;
    if (ce != cudaSuccess)
      return fail(CWB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    g_launches -= (long long)GRAPH_STEPS * launches.size();  // captured, not run
    CWB_CUDA(cudaGraphInstantiate(&exec, g, 0));
    cudaGraphDestroy(g);
    for (; done + GRAPH_STEPS <= steps; done += GRAPH_STEPS) {
      const cudaError_t e = cudaGraphLaunch(exec, s);
      if (e != cudaSuccess) {
        cudaGraphExecDestroy(exec);
        return fail(CWB_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
      }
      g_launches += (long long)GRAPH_STEPS * launches.size();
    }
    cudaGraphExecDestroy(exec);
  }
  for (; done < steps; ++done) {
    const int rc = enqueue_step(launches, s);
    if (rc)
      return rc;
  }
  CWB_CUDA(cudaEventRecord(p->join, s));
  CWB_CUDA(cudaStreamWaitEvent(user, p->join, 0));
  // a bounded wait that ran out leaves its step incomplete: report it
  int err = 0;
  CWB_CUDA(cudaMemcpyAsync(&err, p->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CWB_CUDA(cudaStreamSynchronize(s));
  if (err)
    return fail(CWB_ERR_CUDA, "a staged tile never arrived: the step was abandoned");
  return CWB_OK;
}

// A plan's geometry from its grid, validated: the stencil and precision built here,
// the padded extents and strides, the pml slabs and their memory rows, the device's SM
// count and the environment's overrides. cwb_plan_create and cwb_march_static both
// start from it, so the two step the same geometry.
int plan_geometry(const cwb_grid &G, cwb_plan &p) {
  if (G.ndim != 2 && G.ndim != 3)
    return fail(CWB_ERR_UNSUPPORTED, "the steps are 2D and 3D");
  if (G.radius < 1 || G.radius > CWB_MAX_RADIUS)
    return fail(CWB_ERR_UNSUPPORTED, "radius runs 1 .. 8");
  if (G.precision != 4 && G.precision != 8)
    return fail(CWB_ERR_UNSUPPORTED, "precision is 4 or 8 bytes");
  if ((G.dirichlet & G.neumann) != 0)
    return fail(CWB_ERR_ARG, "a face is either Neumann or Dirichlet");
  cwb::Geometry &geo = p.geo;
  std::memset(&geo, 0, sizeof geo);
  geo.ndim = G.ndim;
  long long total = 1;
  for (int d = 0; d < G.ndim; ++d) {
    if (G.nx[d] < G.radius + 3)
      return fail(CWB_ERR_ARG, "every axis needs at least radius + 3 nodes");
    geo.n[d] = G.nx[d];
    geo.ext[d] = d == G.ndim - 1 ? (G.nx[d] + 31) / 32 * 32 : G.nx[d];
    total *= geo.ext[d];
  }
  if (total >= (1LL << 31))
    return fail(CWB_ERR_ARG, "the padded grid overflows int32 flat indices");
  geo.s[G.ndim - 1] = 1;
  for (int d = G.ndim - 2; d >= 0; --d)
    geo.s[d] = geo.s[d + 1] * geo.ext[d + 1];
  geo.dir = G.dirichlet;
  for (int d = 0; d < G.ndim; ++d) {
    geo.lo[d] = G.pml_lo[d];
    geo.hi[d] = G.pml_hi[d];
    if (geo.lo[d] < 0 || geo.hi[d] < 0 ||
        (geo.lo[d] + geo.hi[d] > 0 &&
         (geo.lo[d] ? geo.lo[d] + G.radius : 0) + (geo.hi[d] ? geo.hi[d] + G.radius : 0) >=
             G.nx[d] - 2))
      return fail(CWB_ERR_ARG, "the pml layers and their reach leave no interior");
    if (geo.lo[d] + geo.hi[d] == 0)
      continue;
    long long row = 1;
    for (int e = 0; e < G.ndim; ++e)
      row *= e == d ? geo.lo[d] + geo.hi[d] : geo.ext[e];
    p.pml_row[d] = row;
  }
  p.grid = G;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&p.sms, cudaDevAttrMultiProcessorCount, dev);
  if (const char *env = std::getenv("CWB_CHUNK"))
    p.chunk_override = std::atoi(env);
  if (const char *env = std::getenv("CWB_NO_TMA"))
    p.tma = std::atoi(env) == 0;
  if (const char *env = std::getenv("CWB_STEP3D"))
    p.blocked3 = std::atoi(env) != 0;
  if (const char *env = std::getenv("CWB_MARCH3D"))
    p.march3 = std::atoi(env);
  if (const char *env = std::getenv("CWB_PML2D"))
    p.pml2d = std::atoi(env);
  if (const char *env = std::getenv("CWB_SRC2D"))
    p.src2d = std::atoi(env) != 0;
  if (const char *env = std::getenv("CWB_LOAD2D"))
    p.load2d = std::atoi(env) != 0;
  if (const char *env = std::getenv("CWB_REC2D"))
    p.rec2d = std::atoi(env) != 0;
  if (const char *env = std::getenv("CWB_FOLD3D"))
    p.fold3d = std::atoi(env) != 0;
  if (const char *env = std::getenv("CWB_FLOW3D"))
    p.flow3 = std::atoi(env);
  if (const char *env = std::getenv("CWB_AUXPAR"))
    p.aux_par = std::atoi(env) != 0;
  if (const char *env = std::getenv("CWB_TBLOCK"))
    p.tblock = std::atoi(env);
  if (const char *env = std::getenv("CWB_ADJSPLIT"))
    p.adj_split = std::atoi(env) != 0;
  return CWB_OK;
}

// ------------------------------------------------------------------------------ batches
template <typename T>
cudaError_t batch2d_r(const cwb::Batch2Params<T> &p, const int R, const dim3 grid,
                      cudaStream_t s) {
  switch (R) {
  case 1: return cwb::batch2d_unit<T, 1>(p, grid, s);
  case 2: return cwb::batch2d_unit<T, 2>(p, grid, s);
  case 3: return cwb::batch2d_unit<T, 3>(p, grid, s);
  case 4: return cwb::batch2d_unit<T, 4>(p, grid, s);
  case 5: return cwb::batch2d_unit<T, 5>(p, grid, s);
  case 6: return cwb::batch2d_unit<T, 6>(p, grid, s);
  case 7: return cwb::batch2d_unit<T, 7>(p, grid, s);
  case 8: return cwb::batch2d_unit<T, 8>(p, grid, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace

struct cwb_batch {
  std::vector<cwb_batch_item> items;
  int *ctr = nullptr;
  cudaStream_t lane = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr, t_begin = nullptr, t_end = nullptr;
  int sms = 148;
  long long want = 0;  // threads a launch aims at
  struct Group {
    int R = 0;
    void *items = nullptr;  // device Batch2Item<float>[count]
    int count = 0;
    long long total = 0;
    bool hold = true;  // an item of the group has a Dirichlet face
    bool pml = true;   // an item of the group has a pml
  };
  std::vector<Group> groups;
  void *recs = nullptr;  // device BatchRecord<float>[items]
  int *owner = nullptr, *col = nullptr;
  int nsens = 0;
  int max_steps = 0;
  // the radius groups of a step run side by side, each on a stream of its own
  static constexpr int SIDES = CWB_MAX_RADIUS;
  cudaStream_t side[SIDES] = {};
  cudaEvent_t step_fork = nullptr, side_done[SIDES] = {};
};

namespace {

void batch_free_groups(cwb_batch *b) {
  for (auto &g : b->groups)
    if (g.items)
      cudaFree(g.items);
  b->groups.clear();
}

// Lay out the items' launches for a launch of about `want` threads: every item marches
// chunks of the same number of rows (its own rows at most), so the threads carry equal
// work; items padded to whole blocks, grouped by radius.
int batch_layout(cwb_batch *b, const long long want) {
  using T = float;
  batch_free_groups(b);
  b->want = want;
  long long units = 0;
  for (const auto &it : b->items) {
    const Geometry &g = it.plan->geo;
    units += (long long)(g.n[0] - 2) * ((g.n[1] - 2) / 4 + 1);
  }
  const long long rows_per = std::max<long long>(1, (units + want - 1) / want);
  std::vector<int> radii;
  for (const auto &it : b->items)
    if (std::find(radii.begin(), radii.end(), it.plan->grid.radius) == radii.end())
      radii.push_back(it.plan->grid.radius);
  std::sort(radii.begin(), radii.end());
  for (const int R : radii) {
    std::vector<cwb::Batch2Item<T>> host;
    long long first = 0;
    for (const auto &it : b->items) {
      if (it.plan->grid.radius != R)
        continue;
      cwb::Batch2Item<T> bi;
      std::memset(&bi, 0, sizeof bi);
      int flags = 0;
      bool uniform = false;
      int rc;
      if ((rc = step_setup<T>(it.plan, it.step, bi.s, flags, uniform)))
        return rc;
      const Geometry &g = it.plan->geo;
      const long long rows = g.n[0] - 2, quads = (g.n[1] - 2) / 4 + 1;
      bi.s.chunk = (int)std::min<long long>(rows, rows_per);
      bi.s.flags = flags;
      bi.s.u0 = to_level(it.step.a, 4);
      bi.s.u1 = to_level(it.step.b, 4);
      bi.s.u2 = to_level(it.step.c, 4);
      bi.s.ctr = b->ctr;
      if ((it.step.flags & CWB_FOLD_SOURCES) && it.step.points.num > 0) {
        const cwb_points &src = it.step.points;
        bi.fold.lin = src.lin;
        bi.fold.weight = static_cast<const T *>(src.weight);
        bi.fold.signal = static_cast<const T *>(src.record);
        bi.fold.nsrc = src.num;
        bi.fold.sig_mul = src.row_mul;
        bi.fold.sig_add = src.row_add;
      }
      if (it.step.flags & CWB_FOLD_REFILL)
        bi.fold.refill = it.plan->grid.neumann | it.plan->grid.dirichlet;
      bi.first = first;
      bi.steps = it.steps;
      const long long threads = quads * ((rows + bi.s.chunk - 1) / bi.s.chunk);
      first += (threads + cwb::S2_THREADS - 1) / cwb::S2_THREADS * cwb::S2_THREADS;
      host.push_back(bi);
    }
    cwb_batch::Group grp;
    grp.R = R;
    grp.count = (int)host.size();
    grp.total = first;
    grp.hold = false;
    grp.pml = false;
    for (const auto &it : host) {
      grp.hold = grp.hold || it.s.g.dir != 0;
      grp.pml = grp.pml || (it.s.flags & cwb::K_PML) != 0;
    }
    CWB_CUDA(cudaMalloc(&grp.items, sizeof(cwb::Batch2Item<T>) * host.size()));
    b->groups.push_back(grp);
    CWB_CUDA(cudaMemcpy(grp.items, host.data(), sizeof(cwb::Batch2Item<T>) * host.size(),
                        cudaMemcpyHostToDevice));
  }
  return CWB_OK;
}

// the launches of one step of the batch: a step per radius group, then the receivers
std::vector<Launch> batch_launches(cwb_batch *b, const bool records) {
  using T = float;
  std::vector<Launch> out;
  for (const auto &g : b->groups) {
    cwb::Batch2Params<T> bp;
    std::memset(&bp, 0, sizeof bp);
    bp.items = static_cast<const cwb::Batch2Item<T> *>(g.items);
    bp.count = g.count;
    bp.total = g.total;
    bp.hold = g.hold ? 1 : 0;
    bp.pml = g.pml ? 1 : 0;
    bp.ctr = b->ctr;
    const dim3 grid((unsigned)((g.total + cwb::S2_THREADS - 1) / cwb::S2_THREADS));
    const int R = g.R;
    out.push_back([bp, R, grid](cudaStream_t s, bool adv) {
      cwb::Batch2Params<T> q = bp;
      q.flags = adv ? cwb::K_ADV : 0;
      return batch2d_r<T>(q, R, grid, s);
    });
  }
  if (records && b->nsens > 0) {
    cwb::BatchRecordParams<T> rp;
    std::memset(&rp, 0, sizeof rp);
    rp.recs = static_cast<const cwb::BatchRecord<T> *>(b->recs);
    rp.owner = b->owner;
    rp.col = b->col;
    rp.total = b->nsens;
    rp.ctr = b->ctr;
    out.push_back([rp](cudaStream_t s, bool adv) {
      cwb::BatchRecordParams<T> q = rp;
      q.flags = adv ? cwb::K_ADV : 0;
      return cwb::launch_batch_record<T>(q, s);
    });
  }
  return out;
}

// one step: with several radius groups and the receivers' launch last, the groups run
// side by side on their own streams, joined before the receivers' launch (which ends the
// step); otherwise in order
int batch_step(cwb_batch *b, const std::vector<Launch> &launches, cudaStream_t s) {
  const int groups = (int)b->groups.size();
  if (groups < 2 || (int)launches.size() != groups + 1 || groups > cwb_batch::SIDES)
    return enqueue_step(launches, s);
  CWB_CUDA(cudaEventRecord(b->step_fork, s));
  for (int i = 0; i < groups; ++i) {
    CWB_CUDA(cudaStreamWaitEvent(b->side[i], b->step_fork, 0));
    const cudaError_t e = launches[i](b->side[i], false);
    if (e != cudaSuccess)
      return fail(CWB_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    CWB_CUDA(cudaEventRecord(b->side_done[i], b->side[i]));
    CWB_CUDA(cudaStreamWaitEvent(s, b->side_done[i], 0));
  }
  const cudaError_t e = launches.back()(s, true);
  if (e != cudaSuccess)
    return fail(CWB_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  g_launches += (long long)launches.size();
  return CWB_OK;
}

int batch_run(cwb_batch *b, const std::vector<Launch> &launches, const int t0, const int steps,
              const bool graph, cudaStream_t s) {
  CWB_CUDA(cwb::launch_set_counter(b->ctr, t0, s));
  ++g_launches;
  int done = 0;
  if (graph && steps >= 2 * GRAPH_STEPS) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    CWB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int rc = CWB_OK;
    for (int k = 0; k < GRAPH_STEPS && !rc; ++k)
      rc = batch_step(b, launches, s);
    const cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (rc)
      return rc;
    if (ce != cudaSuccess)
      return fail(CWB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    g_launches -= (long long)GRAPH_STEPS * launches.size();
    CWB_CUDA(cudaGraphInstantiate(&exec, g, 0));
    cudaGraphDestroy(g);
    for (; done + GRAPH_STEPS <= steps; done += GRAPH_STEPS) {
      const cudaError_t e = cudaGraphLaunch(exec, s);
      if (e != cudaSuccess) {
        cudaGraphExecDestroy(exec);
        return fail(CWB_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
      }
      g_launches += (long long)GRAPH_STEPS * launches.size();
    }
    cudaGraphExecDestroy(exec);
  }
  for (; done < steps; ++done) {
    const int rc = batch_step(b, launches, s);
    if (rc)
      return rc;
  }
  return CWB_OK;
}

// zero a level stack and the pml memory an item steps
int batch_rest(const cwb_batch_item &it, cudaStream_t s) {
  const cwb_level *levels[3] = {&it.step.a, &it.step.b, &it.step.c};
  for (const cwb_level *L : levels) {
    const long long count = std::max(1, L->count);
    CWB_CUDA(cudaMemsetAsync(L->base, 0, (size_t)(count * L->stride) * 4, s));
  }
  for (int d = 0; d < 3; ++d)
    if (it.step.memory[d] && it.plan->pml_row[d] > 0)
      CWB_CUDA(cudaMemsetAsync(it.step.memory[d], 0, (size_t)(3 * it.plan->pml_row[d]) * 4, s));
  return CWB_OK;
}

}  // namespace

extern "C" {

int cwb_batch_destroy(cwb_batch *b) {
  if (!b)
    return CWB_OK;
  if (b->lane)
    cudaStreamSynchronize(b->lane);
  batch_free_groups(b);
  if (b->recs)
    cudaFree(b->recs);
  if (b->owner)
    cudaFree(b->owner);
  if (b->col)
    cudaFree(b->col);
  if (b->ctr)
    cudaFree(b->ctr);
  cudaEvent_t events[4] = {b->fork, b->join, b->t_begin, b->t_end};
  for (cudaEvent_t e : events)
    if (e)
      cudaEventDestroy(e);
  if (b->step_fork)
    cudaEventDestroy(b->step_fork);
  for (int i = 0; i < cwb_batch::SIDES; ++i) {
    if (b->side_done[i])
      cudaEventDestroy(b->side_done[i]);
    if (b->side[i])
      cudaStreamDestroy(b->side[i]);
  }
  if (b->lane)
    cudaStreamDestroy(b->lane);
  delete b;
  return CWB_OK;
}

int cwb_batch_create(const cwb_batch_item *items, const int32_t n, cwb_batch **out) {
  if (!items || n <= 0 || !out)
    return fail(CWB_ERR_ARG, "null argument");
  *out = nullptr;
  const auto aligned16 = [](const void *ptr, const long long stride_elems) {
    return reinterpret_cast<uintptr_t>(ptr) % 16 == 0 && (stride_elems * 4LL) % 16 == 0;
  };
  int max_steps = 0;
  for (int i = 0; i < n; ++i) {
    const cwb_batch_item &it = items[i];
    const std::string at = "batch item " + std::to_string(i) + ": ";
    if (!it.plan)
      return fail(CWB_ERR_ARG, at + "no plan");
    const cwb_plan *p = it.plan;
    if (p->geo.ndim != 2 || p->grid.precision != 4)
      return fail(CWB_ERR_UNSUPPORTED, at + "a batch steps 2D float grids");
    if (p->geo.n[0] < 3 * p->grid.radius || p->geo.n[1] < 3 * p->grid.radius)
      return fail(CWB_ERR_UNSUPPORTED, at + "axes of at least 3 radii");
    const cwb_op &op = it.step;
    if (op.kind != CWB_OP_STEP || !op.mat.stiff_uniform || op.mat.cells)
      return fail(CWB_ERR_UNSUPPORTED, at + "a step of a uniform stiffness, unmasked");
    if (!aligned16(op.a.base, op.a.stride) || !aligned16(op.b.base, op.b.stride) ||
        !aligned16(op.c.base, op.c.stride) || (!op.mat.derive_inertia && !aligned16(op.mat.minv, 0)))
      return fail(CWB_ERR_ARG, at + "levels and 1/m on 16-byte boundaries");
    if ((op.flags & CWB_FOLD_SOURCES) && op.points.num > 0 &&
        (op.points.num > 32 || !op.points.lin || !op.points.weight || !op.points.record))
      return fail(CWB_ERR_ARG, at + "at most 32 folded sources, with weights and a signal");
    if (it.record.num > 0 && (!it.record.lin || !it.record.record || it.record.store != 0))
      return fail(CWB_ERR_ARG, at + "a record needs indices and native storage");
    if (it.steps < 0)
      return fail(CWB_ERR_ARG, at + "a negative step count");
    max_steps = std::max(max_steps, it.steps);
  }
  cwb_batch *b = new cwb_batch();
  b->items.assign(items, items + n);
  b->max_steps = max_steps;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaMalloc(&b->ctr, 2 * sizeof(int)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->lane, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&b->t_begin) != cudaSuccess || cudaEventCreate(&b->t_end) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->step_fork, cudaEventDisableTiming) != cudaSuccess) {
    cwb_batch_destroy(b);
    return fail(CWB_ERR_ALLOC, "batch resources");
  }
  for (int i = 0; i < cwb_batch::SIDES; ++i)
    if (cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->side_done[i], cudaEventDisableTiming) != cudaSuccess) {
      cwb_batch_destroy(b);
      return fail(CWB_ERR_ALLOC, "batch streams");
    }
  cudaMemset(b->ctr, 0, 2 * sizeof(int));
  // the receivers: one table entry per item, one (owner, column) pair per sensor
  std::vector<cwb::BatchRecord<float>> recs(n);
  std::vector<int> owner, col;
  for (int i = 0; i < n; ++i) {
    const cwb_batch_item &it = items[i];
    std::memset(&recs[i], 0, sizeof recs[i]);
    recs[i].a = to_level(it.step.c, 4);
    recs[i].lin = it.record.lin;
    recs[i].record = static_cast<float *>(it.record.record);
    recs[i].num = it.record.num;
    recs[i].steps = it.steps;
    for (int j = 0; j < it.record.num; ++j) {
      owner.push_back(i);
      col.push_back(j);
    }
  }
  b->nsens = (int)owner.size();
  int rc = CWB_OK;
  if (cudaMalloc(&b->recs, sizeof(cwb::BatchRecord<float>) * n) != cudaSuccess ||
      (b->nsens && (cudaMalloc(&b->owner, sizeof(int) * b->nsens) != cudaSuccess ||
                    cudaMalloc(&b->col, sizeof(int) * b->nsens) != cudaSuccess))) {
    cwb_batch_destroy(b);
    return fail(CWB_ERR_ALLOC, "batch receivers");
  }
  cudaMemcpy(b->recs, recs.data(), sizeof(cwb::BatchRecord<float>) * n, cudaMemcpyHostToDevice);
  if (b->nsens) {
    cudaMemcpy(b->owner, owner.data(), sizeof(int) * b->nsens, cudaMemcpyHostToDevice);
    cudaMemcpy(b->col, col.data(), sizeof(int) * b->nsens, cudaMemcpyHostToDevice);
  }
  if ((rc = batch_layout(b, (long long)b->sms * 1024))) {
    cwb_batch_destroy(b);
    return rc;
  }
  *out = b;
  return CWB_OK;
}

int cwb_batch_tune(cwb_batch *b, const int32_t steps, void *stream) {
  if (!b || steps <= 0)
    return fail(CWB_ERR_ARG, "null batch or no steps");
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  CWB_CUDA(cudaEventRecord(b->fork, user));
  CWB_CUDA(cudaStreamWaitEvent(b->lane, b->fork, 0));
  cudaStream_t s = b->lane;
  const int run = std::min(steps, std::max(1, b->max_steps));
  const long long candidates[] = {256, 512, 1024, 2048, 4096};
  long long best = (long long)b->sms * 1024;
  float best_ms = 1e30f;
  int rc;
  for (const long long per : candidates) {
    if ((rc = batch_layout(b, per * b->sms)))
      return rc;
    const std::vector<Launch> launches = batch_launches(b, false);
    if ((rc = batch_run(b, launches, 0, 1, false, s)))  // warm: the first launch loads code
      return rc;
    CWB_CUDA(cudaEventRecord(b->t_begin, s));
    if ((rc = batch_run(b, launches, 0, run, false, s)))
      return rc;
    CWB_CUDA(cudaEventRecord(b->t_end, s));
    CWB_CUDA(cudaEventSynchronize(b->t_end));
    float ms = 0.f;
    CWB_CUDA(cudaEventElapsedTime(&ms, b->t_begin, b->t_end));
    if (ms < best_ms) {
      best_ms = ms;
      best = per * b->sms;
    }
  }
  for (const auto &it : b->items)
    if ((rc = batch_rest(it, s)))
      return rc;
  if ((rc = batch_layout(b, best)))
    return rc;
  CWB_CUDA(cudaEventRecord(b->join, s));
  CWB_CUDA(cudaStreamWaitEvent(user, b->join, 0));
  return CWB_OK;
}

int cwb_batch_march(cwb_batch *b, const int32_t t0, const int32_t steps, const int32_t graph,
                    void *stream) {
  if (!b)
    return fail(CWB_ERR_ARG, "null batch");
  if (steps <= 0)
    return CWB_OK;
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  CWB_CUDA(cudaEventRecord(b->fork, user));
  CWB_CUDA(cudaStreamWaitEvent(b->lane, b->fork, 0));
  const std::vector<Launch> launches = batch_launches(b, true);
  int rc;
  if ((rc = batch_run(b, launches, t0, steps, graph != 0, b->lane)))
    return rc;
  CWB_CUDA(cudaEventRecord(b->join, b->lane));
  CWB_CUDA(cudaStreamWaitEvent(user, b->join, 0));
  return CWB_OK;
}

int64_t cwb_batch_threads(const cwb_batch *b) { return b ? b->want : 0; }

namespace {
int conv_shape(const int32_t batch, const int32_t height, const int32_t width, const int32_t cin,
               const int32_t cout, cwb::ConvShape &s) {
  if (batch <= 0 || height <= 0 || width <= 0 || cin < 2 || cin % 2 || cout < 1 ||
      cout > cwb::CONV_MAX_N)
    return fail(CWB_ERR_ARG, "conv: positive sizes, an even cin, at most 32 output channels");
  s.batch = batch;
  s.h = height;
  s.w = width;
  s.cin = cin;
  s.cout = cout;
  s.kpad = (25 * cin + 15) / 16 * 16;
  return CWB_OK;
}
}  // namespace

int cwb_conv_bf16_fwd(const void *x, const void *w, const float *bias, const void *mask,
                      void *y_bf16, float *y_f32, const int32_t batch, const int32_t height,
                      const int32_t width, const int32_t cin, const int32_t cout,
                      const int32_t relu, void *stream) {
  cwb::ConvShape s;
  int rc;
  if ((rc = conv_shape(batch, height, width, cin, cout, s)))
    return rc;
  if (!x || !w || (!y_bf16 && !y_f32))
    return fail(CWB_ERR_ARG, "conv: null input, weights or output");
  CWB_CUDA(cwb::conv_forward(x, w, bias, mask, y_bf16, y_f32, s, relu,
                             static_cast<cudaStream_t>(stream)));
  ++g_launches;
  return CWB_OK;
}

int cwb_conv_bf16_bwd(const void *dy, const void *x, float *dw, float *db, const int32_t batch,
                      const int32_t height, const int32_t width, const int32_t cin,
                      const int32_t cout, void *stream) {
  cwb::ConvShape s;
  int rc;
  if ((rc = conv_shape(batch, height, width, cin, cout, s)))
    return rc;
  if (!dy || !x || !dw)
    return fail(CWB_ERR_ARG, "conv: null gradient, input or weight gradient");
  CWB_CUDA(cwb::conv_weight_grad(dy, x, dw, db, s, static_cast<cudaStream_t>(stream)));
  g_launches += db ? 2 : 1;
  return CWB_OK;
}

const char *cwb_last_error(void) { return g_error.c_str(); }

int32_t cwb_version(void) { return 1; }

int64_t cwb_launches(void) { return g_launches.load(); }

int cwb_plan_create(const cwb_grid *grid, cwb_plan **out) {
  if (!grid || !out)
    return fail(CWB_ERR_ARG, "null argument");
  *out = nullptr;
  cwb_plan *p = new cwb_plan();
  if (const int rc = plan_geometry(*grid, *p)) {
    delete p;
    return rc;
  }
  if (cudaMalloc(&p->ctr, 2 * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&p->err, sizeof(int)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&p->lane, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->side_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->side_join, cudaEventDisableTiming) != cudaSuccess) {
    cwb_plan_destroy(p);
    return fail(CWB_ERR_ALLOC, std::string("plan resources: ") +
                                   cudaGetErrorString(cudaGetLastError()));
  }
  cudaMemset(p->ctr, 0, 2 * sizeof(int));
  cudaMemset(p->err, 0, sizeof(int));
  *out = p;
  return CWB_OK;
}

int cwb_plan_destroy(cwb_plan *p) {
  if (!p)
    return CWB_OK;
  if (p->lane)
    cudaStreamSynchronize(p->lane);
  for (Scratch *s : {&p->tb_src, &p->tb_rec})
    p->scratch.push_back(*s);
  for (Scratch &s : p->scratch) {
    if (s.start)
      cudaFree(s.start);
    if (s.entry)
      cudaFree(s.entry);
  }
  if (p->tb_fields)
    cudaFree(p->tb_fields);
  if (p->tb_psi)
    cudaFree(p->tb_psi);
  if (p->ctr)
    cudaFree(p->ctr);
  if (p->err)
    cudaFree(p->err);
  if (p->fork)
    cudaEventDestroy(p->fork);
  if (p->join)
    cudaEventDestroy(p->join);
  if (p->side) {
    cudaStreamSynchronize(p->side);
    cudaStreamDestroy(p->side);
  }
  if (p->side_fork)
    cudaEventDestroy(p->side_fork);
  if (p->side_join)
    cudaEventDestroy(p->side_join);
  if (p->lane)
    cudaStreamDestroy(p->lane);
  delete p;
  return CWB_OK;
}

int64_t cwb_pml_row(const cwb_plan *p, const int32_t d) {
  if (!p || d < 0 || d > 2)
    return 0;
  return p->pml_row[d];
}

int cwb_march(cwb_plan *p, const cwb_op *ops, const int32_t nops, const int32_t t0,
              const int32_t steps, const int32_t graph, void *stream) {
  if (!p || (!ops && nops > 0) || nops < 0)
    return fail(CWB_ERR_ARG, "null argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return p->grid.precision == 4 ? march<float>(p, ops, nops, t0, steps, graph, s)
                                : march<double>(p, ops, nops, t0, steps, graph, s);
}

}  // extern "C"

// ------------------------------------------------------------- march without allocation
// Some callers cannot let a library allocate device memory: a host application (an
// inference server, or a service embedding this library through its C ABI) that owns
// the whole GPU through its own memory pool and forbids allocations behind its back,
// or that budgets every byte of a device shared with other work. For them
// cwb_march_static runs the same op list as cwb_march with no plan at all: its step
// counter, its error flag and its folded-source lists live in g_static_scratch, a
// fixed array every GPU that loads this library holds until the process exits.
namespace {

// 16 bytes of counter and flag, the rest for folded-source lists
__device__ __align__(256) unsigned char g_static_scratch[CWB_STATIC_SCRATCH_BYTES];

// The device address of g_static_scratch on the current device. In host code the
// symbol's name is only a host-side stand-in, so the address is asked from the runtime,
// with the device current, on every call: a cached address could outlive the module it
// points into (a device reset, or a primary context torn down and made again, loads the
// module anew), and one lookup costs nothing next to a march.
int static_scratch(void **out) {
  void *ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
  if (e != cudaSuccess)
    return fail(CWB_ERR_CUDA,
                std::string("cudaGetSymbolAddress(g_static_scratch): ") + cudaGetErrorString(e));
  *out = ptr;
  return CWB_OK;
}

template <typename T>
int march_static(cwb_plan &p, const cwb_op *ops, const int nops, const int t0, const int steps,
                 cudaStream_t s) {
  std::vector<Launch> launches;
  for (int i = 0; i < nops; ++i) {
    const int rc = translate<T>(&p, ops[i], (size_t)i, s, launches);
    if (rc)
      return rc;
  }
  if (launches.empty() || steps <= 0)
    return CWB_OK;
  // the counter and the flag start at zero every call; the lists were written above
  CWB_CUDA(cudaMemsetAsync(p.err, 0, sizeof(int), s));
  CWB_CUDA(cwb::launch_set_counter(p.ctr, t0, s));
  ++g_launches;
  for (int k = 0; k < steps; ++k) {
    const int rc = enqueue_step(launches, s);
    if (rc)
      return rc;
  }
  int err = 0;
  CWB_CUDA(cudaMemcpyAsync(&err, p.err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CWB_CUDA(cudaStreamSynchronize(s));
  if (err)
    return fail(CWB_ERR_CUDA, "a staged tile never arrived: the step was abandoned");
  return CWB_OK;
}

}  // namespace

extern "C" int cwb_march_static(const cwb_grid *grid, const cwb_op *ops, const int32_t nops,
                                const int32_t t0, const int32_t steps, void *stream) {
  if (!grid || (!ops && nops > 0) || nops < 0)
    return fail(CWB_ERR_ARG, "null argument");
  void *base = nullptr;
  int rc = static_scratch(&base);
  if (rc)
    return rc;
  cwb_plan p;  // on the stack: no stream, event or device memory of its own
  if ((rc = plan_geometry(*grid, p)))
    return rc;
  unsigned char *bytes = static_cast<unsigned char *>(base);
  p.ctr = reinterpret_cast<int *>(bytes);      // step counter and blocks done
  p.err = reinterpret_cast<int *>(bytes + 8);  // error flag
  p.fixed = bytes + 16;
  p.fixed_cap = CWB_STATIC_SCRATCH_BYTES - 16;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return grid->precision == 4 ? march_static<float>(p, ops, nops, t0, steps, s)
                              : march_static<double>(p, ops, nops, t0, steps, s);
}
