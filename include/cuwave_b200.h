/*
 * cuwave_b200.h -- C ABI of the B200 scalar-wave hot path.
 *
 * One shared library, libcuwave_b200.so, steps the scalar (pressure) wave equation's
 * leapfrog update with its perfectly matched layer, source injection, ghost refill and
 * receiver recording, and the transposed (adjoint) update with the material-gradient
 * accumulation, on one sm_100a GPU.
 *
 * Every pointer below is a DEVICE pointer unless its comment says otherwise. Fields are
 * C-contiguous over the padded grid (nx[0], .., ceil32(nx[ndim-1])); a flat node index
 * is sum_d i_d * stride_d over that grid, int32. Every call returns CWB_OK (0) or a
 * negative CWB_ERR_* code, and cwb_last_error() then holds one line of text. Nothing is
 * allocated outside a plan: a plan owns its scratch (counters, source lists, graphs)
 * and its two streams (the march's, and a side stream the adjoint's pml memory runs on).
 * The one entry point that runs without a plan, cwb_march_static, allocates nothing at
 * all: its scratch is a fixed static device array.
 *
 * The reference (cmpmech/cuwave) launches one CUDA C kernel per operation from Python;
 * on its host fallback each kernel is bound through the C ABI
 *     extern "C" void launch_<kernel>(gx, gy, gz, bx, by, bz, void **args)
 * (cuwave/kernels/cpu.hpp:93-98). The entry points here replace those launches, grouped
 * per time step: see each op kind for the reference kernels it stands in for.
 */
#ifndef CUWAVE_B200_H
#define CUWAVE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CWB_OK 0
#define CWB_ERR_ARG (-1)         /* an argument out of range or inconsistent */
#define CWB_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define CWB_ERR_UNSUPPORTED (-3) /* a configuration this build does not step */
#define CWB_ERR_ALLOC (-4)       /* a plan could not allocate its scratch */

#define CWB_MAX_RADIUS 8

/* Grid geometry and the stencil, fixed for a plan.
 * Replaces the compile-time configuration of cuwave/kernels/scalar.cu:1-12 (NDIM,
 * USE_FLOAT, STENCIL_RADIUS, OP_COEFFS, DIRICHLET_FACES) and the geometry arguments
 * of wave.axis_geometry (cuwave/wave.py:830-837). */
typedef struct cwb_grid {
  int32_t ndim;                  /* 2 or 3 */
  int32_t nx[3];                 /* logical nodes per axis, ghost ring included */
  int32_t radius;                /* R = space_order / 2, 1 .. 8 */
  int32_t precision;             /* bytes per value: 4 (float32) or 8 (float64) */
  double coeffs[CWB_MAX_RADIUS]; /* OP_W(R, 1..R), rounded to `precision` on use */
  double factors[3];             /* the per-axis step factors f_d */
  double dt;                     /* the time step, read by the damped update */
  int32_t dirichlet;             /* faces held at zero, bit 2 * axis + side */
  int32_t neumann;               /* faces refilled evenly, bit 2 * axis + side */
  int32_t pml_lo[3], pml_hi[3];  /* layer depth behind each face, 0 for none */
} cwb_grid;

typedef struct cwb_plan cwb_plan;

/* Where the field of time step t lives: base + ((mul * t + add) mod period) * stride
 * elements (period 0: no wrap), one of `count` levels stacked from `base`. Two slots
 * rotate as period 2, a history as period 0. */
typedef struct cwb_level {
  void *base;
  int64_t stride;
  int32_t mul, add, period;
  int32_t count; /* levels in the stack; every step's index must fall in 0 .. count - 1 */
} cwb_level;

/* The material a step reads. Replaces PressureWave.step_kernel_args
 * (cuwave/scalar.py:739-745) and the pml profiles (cuwave/boundary.py:327-361). */
typedef struct cwb_material {
  const void *stiff;       /* k over the padded grid; unread when stiff_uniform */
  const void *minv;        /* 1 / m over the padded grid; unread when derive_inertia */
  const void *damping;     /* d over the padded grid, or NULL for a lossless step */
  const void *profile[3];  /* (4, nx[d]) rows a_node, b_node, a_half, b_half per lined axis */
  int32_t derive_inertia;  /* 1 / m = 1 / k (ScalarWave) */
  int32_t stiff_uniform;   /* k is stiff_value everywhere the step reads it */
  double stiff_value;
  /* A masked domain, or NULL: per node of the padded grid 0 (not stepped), 1 << 30
   * (every cell at the full radius), else the radii of its two cells along each axis d,
   * (r_plus | r_minus << 3) << 6 d, 7 for a cell open onto a held node. Replaces the
   * cells of cuwave/wave.py:675-726 read by fd_kernel under USE_DOMAIN (scalar.cu:86-158,
   * 434-452). */
  const int32_t *cells;
  const void *cell_table;  /* with cells: (R, R) OP_W(r, k) at [r - 1][k - 1] */
} cwb_material;

/* A transfer list: `num` flat node indices, a per-point weight and a (rows, num)
 * record whose row for step t is row_mul * t + row_add. */
typedef struct cwb_points {
  const int32_t *lin;
  const void *weight;   /* per point, or NULL where the op reads none */
  void *record;         /* (rows, num) values */
  int32_t num;
  int32_t row_mul, row_add;
  int32_t store;        /* record elements: 0 the plan's precision, 1 bfloat16 bits
                           (uint16, round to nearest even), 2 float32 under float64 */
} cwb_points;

/* Op kinds of a march step, run in order for every step t. */
enum {
  /* The leapfrog update u^t = 2u^(t-1) - u^(t-2) + dt^2/m div(k grad u^(t-1)) of the
   * interior, its pml memory terms, and, per flags, the folded sources and ghost refill.
   * a = u^(t-2) (read), b = u^(t-1) (read), c = u^t (written; may alias a).
   * Replaces fd_kernel (cuwave/kernels/scalar.cu:347-496) and pml_kernel
   * (scalar.cu:500-532), and with CWB_FOLD_* excitation_kernel
   * (cuwave/kernels/common.cuh:456-464) and the refill kernels (scalar.cu:535-555). */
  CWB_OP_STEP = 1,
  /* a[lin] += weight * record[row], atomically. Replaces excitation_kernel
   * (common.cuh:456-464). */
  CWB_OP_EXCITE = 2,
  /* a[lin] = record[row]. Replaces set_signal_kernel (common.cuh:494-503). */
  CWB_OP_REPLAY = 3,
  /* Ghosts of every face refilled from their mirror, negated and the wall node zeroed on
   * a Dirichlet face. Replaces homogeneous_neumann_kernel / homogeneous_dirichlet_kernel
   * (scalar.cu:535-555). */
  CWB_OP_REFILL = 4,
  /* record[row] = a[lin], narrowed as points.store asks. Replaces
   * get_signal_kernel (common.cuh:483-491) and wave.narrow (cuwave/wave.py:848-853). */
  CWB_OP_RECORD = 5,
  /* The adjoint pml memory step from a = lambda^(n+1), before CWB_OP_ADJOINT reads it.
   * Replaces pml_aux_kernel (cuwave/kernels/scalar_sensitivity.cu:518-542). */
  CWB_OP_PML_AUX = 6,
  /* The transposed update lambda^n from a = lambda^(n+2) (overwritten) and
   * b = lambda^(n+1), with the pml transpose gathered in; with CWB_GRAD also
   * g_mass and g_stiff against c = u^n. Replaces adjoint_kernel and
   * adjoint_gradient_kernel (scalar_sensitivity.cu:388-515) and pml_adjoint_kernel
   * (scalar_sensitivity.cu:545-597). */
  CWB_OP_ADJOINT = 7,
  /* The adjoint load a[lin] += weight * record[row]; with g_mass also
   * g_mass[lin] -= scale * c[lin] * load. Replaces adjoint_excitation_kernel
   * (common.cuh:467-480). */
  CWB_OP_LOAD = 8,
  /* Both gradient densities of one forward triplet a, b, c = u^(t-2), u^(t-1), u^t
   * against d = lambda^t, with scale = 1 / dt^2 and factors F_d. Replaces
   * gradient_kernel (scalar_sensitivity.cu:303-350). */
  CWB_OP_GRADIENT = 9,
  /* The leapfrog update of CWB_OP_STEP (a, b read, c written; lossless: no pml, no
   * damping) that first adds the superposition densities into g_mass and g_stiff: the
   * mass density of the triplet before, scale * (b - c)^2 with c's old value, and the
   * stiffness density of this triplet, factors[0] * sum_d f_d (b[+s_d] - b[-s_d])^2.
   * c must not alias a. Replaces superposed_kernel (scalar_sensitivity.cu:600-668). */
  CWB_OP_SUPERPOSED = 10,
  /* Both Frechet densities of the triplet a, b, c over the interior: g_mass +=
   * scale * (c - a)^2, g_stiff += sum_d factors[d] * (b[+s_d] - b[-s_d])^2. Replaces
   * frechet_kernel (scalar_sensitivity.cu:353-385). */
  CWB_OP_FRECHET = 11,
  /* A running DFT at `points`: acc[k * num + j] += table[row * columns + k] * a[lin[j]]
   * for the `columns` phase factors of table row `row` (points.record is the (rows,
   * columns) table), acc = g_mass. Replaces dft_kernel (common.cuh:506-518). */
  CWB_OP_DFT = 12,
};

/* op flags */
#define CWB_PML 1          /* STEP, ADJOINT: step the pml memory of the lined axes */
#define CWB_FOLD_SOURCES 2 /* STEP: add `points` (interior nodes only) inside the step */
#define CWB_FOLD_REFILL 4  /* STEP: write the face ghosts from their mirrors */
#define CWB_GRAD 8         /* ADJOINT: accumulate g_mass and g_stiff */

typedef struct cwb_op {
  int32_t kind;
  int32_t flags;
  cwb_level a, b, c, d;
  cwb_material mat;
  cwb_points points;
  void *memory[3];   /* pml memory per lined axis: 3 slab rows forward, 5 adjoint */
  void *g_mass;
  void *g_stiff;
  double scale;      /* ADJOINT / LOAD / GRADIENT: 1 / dt^2; SUPERPOSED / FRECHET: the
                        mass density factor */
  double factors[3]; /* GRADIENT: F_d = f_d / dt^2; SUPERPOSED: [0] the stiffness density
                        factor; FRECHET: the per-axis stiffness density factors */
  int32_t columns;   /* DFT: phase factors per table row, rows of the accumulator */
} cwb_op;

/* Create and destroy a plan. Replaces compile_kernels (cuwave/wave.py:637-647): one
 * build serves every order, stencil and face layout, the table a runtime argument. */
int cwb_plan_create(const cwb_grid *grid, cwb_plan **plan);
int cwb_plan_destroy(cwb_plan *plan);

/* Run `steps` steps t = t0 .. t0 + steps - 1 of the op list on `stream` (a
 * cudaStream_t, NULL for the legacy stream). With `graph` nonzero, chunks of steps
 * are captured once as a CUDA graph and replayed. Replaces wave.march
 * (cuwave/wave.py:890-952) and the step closures handed to it. */
int cwb_march(cwb_plan *plan, const cwb_op *ops, int32_t nops, int32_t t0,
              int32_t steps, int32_t graph, void *stream);

/* Bytes of the static device scratch cwb_march_static uses (per GPU, until exit). */
#define CWB_STATIC_SCRATCH_BYTES (256 * 1024)

/* cwb_march for callers that cannot let a library allocate device memory, e.g. a host
 * that owns the GPU through its own memory pool and forbids allocations behind its
 * back. No counterpart in the reference. Runs the op list of cwb_march for `steps` steps
 * directly on `stream`, without a plan: it allocates nothing, captures no graph, and
 * keeps its step counter, error flag and folded-source lists (16 bytes per source plus
 * 4 bytes per block of the step's grid) in one static device array of
 * CWB_STATIC_SCRATCH_BYTES. It asks the runtime for the array's device address on
 * every call, with the caller's device current (the first call on a device may load the
 * library's device code: make it before any stream capture). A march whose
 * lists do not fit is refused with CWB_ERR_ARG. Every call shares the array: calls that
 * overlap on the GPU (two streams, two host threads) race and must not be issued. The
 * call returns after the march has finished on the GPU. */
int cwb_march_static(const cwb_grid *grid, const cwb_op *ops, int32_t nops, int32_t t0,
                     int32_t steps, void *stream);

/* ------------------------------------------------------------------ batches
 * Many 2D problems (shots, designs of uneven size and order) stepped together: each
 * item is one problem's forward step on its own plan, and the batch runs every item's
 * step t in one launch per stencil radius, then every item's receivers in one launch,
 * chunks of steps replayed as a CUDA graph. No counterpart in the reference, which runs
 * a problem at a time (cuwave/utils.py:50-73 spreads shots over GPUs, one simulate
 * each). */
typedef struct cwb_batch cwb_batch;

typedef struct cwb_batch_item {
  cwb_plan *plan;     /* the item's plan: 2D, float */
  cwb_op step;        /* CWB_OP_STEP of a uniform stiffness, sources (at most 32, interior
                         nodes) and refill folded; levels, material and pml memory as
                         cwb_march takes them, on 16-byte boundaries */
  cwb_points record;  /* receivers read after every step into (steps, num) native
                         values at row t, or num 0 */
  int32_t steps;      /* the item's own step count: it rests from t = steps on */
} cwb_batch_item;

/* Check the items and lay out their launches; the pointers they hold must outlive the
 * batch. */
int cwb_batch_create(const cwb_batch_item *items, int32_t n, cwb_batch **batch);
/* Choose the launches' thread count by timing `steps` steps of each candidate on the
 * items' own fields, which it zeroes afterwards with their pml memory: call it before
 * the march, on fields at rest. */
int cwb_batch_tune(cwb_batch *batch, int32_t steps, void *stream);
/* Steps t = t0 .. t0 + steps - 1 of every item, as cwb_march. */
int cwb_batch_march(cwb_batch *batch, int32_t t0, int32_t steps, int32_t graph, void *stream);
/* Threads a launch of the batch aims at (the tuned choice). */
int64_t cwb_batch_threads(const cwb_batch *batch);
int cwb_batch_destroy(cwb_batch *batch);

/* ---------------------------------------------------------------- corrector
 * The 5x5 convolutions (stride 1, zero padding 2) of the learned dispersion corrector,
 * on the tensor cores: BF16 operands, FP32 accumulation. Activations are channels-last
 * BF16 (batch, height, width, channels); a layer's weights are (cout, kpad) BF16 with
 * k = (5 ky + kx) cin + ci and kpad = 25 cin rounded up to 16 (the padding zero). cin is
 * even (pad a channel), cout at most 32. No counterpart in the reference. */

/* y = conv(x, w) + bias (optional), ReLU when `relu`; zeroed where `mask` (BF16, the
 * shape of y, optional) is not positive; written to y_bf16 and/or y_f32 (either may be
 * NULL). The data gradient of a layer is this call on dy with the weights flipped and
 * transposed (wt[ci][(5 ky + kx) cout + co] = w[co][(5 (4 - ky) + 4 - kx) cin + ci]) and
 * the layer input's activation as the mask. */
int cwb_conv_bf16_fwd(const void *x, const void *w, const float *bias, const void *mask,
                      void *y_bf16, float *y_f32, int32_t batch, int32_t height, int32_t width,
                      int32_t cin, int32_t cout, int32_t relu, void *stream);
/* dw += the weight gradient sum over pixels of dy[p][co] im2col(x)[p][k] (FP32,
 * (cout, kpad)), db += sum over pixels of dy (optional). */
int cwb_conv_bf16_bwd(const void *dy, const void *x, float *dw, float *db, int32_t batch,
                      int32_t height, int32_t width, int32_t cin, int32_t cout, void *stream);

/* Elements per row of the pml memory of axis d (0 for an unlined axis); a forward
 * memory holds 3 such rows, an adjoint one 5. */
int64_t cwb_pml_row(const cwb_plan *plan, int32_t d);

/* Kernels the library launched since it was loaded (a diagnostic counter). */
int64_t cwb_launches(void);

const char *cwb_last_error(void);
int32_t cwb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CUWAVE_B200_H */
