"""ctypes binding of libcuwave_b200.so (include/cuwave_b200.h).

The library is the product's only compute path: importing this module without it, or
calling it without a CUDA device, raises. There is no fallback.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import torch

LIBRARY = Path(__file__).resolve().parent / "libcuwave_b200.so"

CWB_OK = 0
ERRORS = {-1: "bad argument", -2: "CUDA error", -3: "unsupported", -4: "allocation failed"}

OP_STEP, OP_EXCITE, OP_REPLAY, OP_REFILL, OP_RECORD = 1, 2, 3, 4, 5
OP_PML_AUX, OP_ADJOINT, OP_LOAD, OP_GRADIENT = 6, 7, 8, 9
OP_SUPERPOSED, OP_FRECHET, OP_DFT = 10, 11, 12
PML, FOLD_SOURCES, FOLD_REFILL, GRAD = 1, 2, 4, 8
STORE_NATIVE, STORE_BF16, STORE_F32 = 0, 1, 2


class Grid(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int32),
        ("nx", ctypes.c_int32 * 3),
        ("radius", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("coeffs", ctypes.c_double * 8),
        ("factors", ctypes.c_double * 3),
        ("dt", ctypes.c_double),
        ("dirichlet", ctypes.c_int32),
        ("neumann", ctypes.c_int32),
        ("pml_lo", ctypes.c_int32 * 3),
        ("pml_hi", ctypes.c_int32 * 3),
    ]


class Level(ctypes.Structure):
    _fields_ = [
        ("base", ctypes.c_void_p),
        ("stride", ctypes.c_int64),
        ("mul", ctypes.c_int32),
        ("add", ctypes.c_int32),
        ("period", ctypes.c_int32),
        ("count", ctypes.c_int32),
    ]


class Material(ctypes.Structure):
    _fields_ = [
        ("stiff", ctypes.c_void_p),
        ("minv", ctypes.c_void_p),
        ("damping", ctypes.c_void_p),
        ("profile", ctypes.c_void_p * 3),
        ("derive_inertia", ctypes.c_int32),
        ("stiff_uniform", ctypes.c_int32),
        ("stiff_value", ctypes.c_double),
        ("cells", ctypes.c_void_p),
        ("cell_table", ctypes.c_void_p),
    ]


class Points(ctypes.Structure):
    _fields_ = [
        ("lin", ctypes.c_void_p),
        ("weight", ctypes.c_void_p),
        ("record", ctypes.c_void_p),
        ("num", ctypes.c_int32),
        ("row_mul", ctypes.c_int32),
        ("row_add", ctypes.c_int32),
        ("store", ctypes.c_int32),
    ]


class Op(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("a", Level),
        ("b", Level),
        ("c", Level),
        ("d", Level),
        ("mat", Material),
        ("points", Points),
        ("memory", ctypes.c_void_p * 3),
        ("g_mass", ctypes.c_void_p),
        ("g_stiff", ctypes.c_void_p),
        ("scale", ctypes.c_double),
        ("factors", ctypes.c_double * 3),
        ("columns", ctypes.c_int32),
    ]


class BatchItem(ctypes.Structure):
    _fields_ = [
        ("plan", ctypes.c_void_p),
        ("step", Op),
        ("record", Points),
        ("steps", ctypes.c_int32),
    ]


_lib = None


def library() -> ctypes.CDLL:
    """The loaded library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(
                f"{LIBRARY.name} is not built: run `python -m cuwave_b200.build` "
                "(there is no CPU fallback)"
            )
        lib = ctypes.CDLL(str(LIBRARY))
        lib.cwb_plan_create.argtypes = [ctypes.POINTER(Grid), ctypes.POINTER(ctypes.c_void_p)]
        lib.cwb_plan_create.restype = ctypes.c_int
        lib.cwb_plan_destroy.argtypes = [ctypes.c_void_p]
        lib.cwb_plan_destroy.restype = ctypes.c_int
        lib.cwb_march.argtypes = [
            ctypes.c_void_p,
            ctypes.POINTER(Op),
            ctypes.c_int32,
            ctypes.c_int32,
            ctypes.c_int32,
            ctypes.c_int32,
            ctypes.c_void_p,
        ]
        lib.cwb_march.restype = ctypes.c_int
        lib.cwb_batch_create.argtypes = [ctypes.POINTER(BatchItem), ctypes.c_int32,
                                         ctypes.POINTER(ctypes.c_void_p)]
        lib.cwb_batch_create.restype = ctypes.c_int
        lib.cwb_batch_tune.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
        lib.cwb_batch_tune.restype = ctypes.c_int
        lib.cwb_batch_march.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_void_p]
        lib.cwb_batch_march.restype = ctypes.c_int
        lib.cwb_batch_threads.argtypes = [ctypes.c_void_p]
        lib.cwb_batch_threads.restype = ctypes.c_int64
        lib.cwb_batch_destroy.argtypes = [ctypes.c_void_p]
        lib.cwb_batch_destroy.restype = ctypes.c_int
        vp, i32 = ctypes.c_void_p, ctypes.c_int32
        lib.cwb_conv_bf16_fwd.argtypes = [vp, vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, i32, vp]
        lib.cwb_conv_bf16_fwd.restype = ctypes.c_int
        lib.cwb_conv_bf16_bwd.argtypes = [vp, vp, vp, vp, i32, i32, i32, i32, i32, vp]
        lib.cwb_conv_bf16_bwd.restype = ctypes.c_int
        lib.cwb_pml_row.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        lib.cwb_pml_row.restype = ctypes.c_int64
        lib.cwb_launches.restype = ctypes.c_int64
        lib.cwb_last_error.restype = ctypes.c_char_p
        lib.cwb_version.restype = ctypes.c_int32
        _lib = lib
    return _lib


def check(code: int) -> None:
    if code != CWB_OK:
        message = library().cwb_last_error().decode()
        raise RuntimeError(f"cuwave_b200: {ERRORS.get(code, code)}: {message}")


def require_cuda() -> torch.device:
    """The current CUDA device; the product runs on a GPU only."""
    if not torch.cuda.is_available():
        raise RuntimeError("cuwave_b200 steps on a CUDA device, and none is available")
    library()
    return torch.device("cuda", torch.cuda.current_device())


class Plan:
    """A native plan: one grid geometry, stencil row, factors and face layout."""

    def __init__(self, grid: Grid):
        self._lib = library()
        handle = ctypes.c_void_p()
        check(self._lib.cwb_plan_create(ctypes.byref(grid), ctypes.byref(handle)))
        self.handle = handle
        self.grid = grid

    def pml_row(self, d: int) -> int:
        return int(self._lib.cwb_pml_row(self.handle, d))

    def march(self, ops: list[Op], t0: int, steps: int, graph: bool = True) -> None:
        if steps <= 0 or not ops:
            return
        array = (Op * len(ops))(*ops)
        stream = torch.cuda.current_stream().cuda_stream
        check(
            self._lib.cwb_march(
                self.handle, array, len(ops), int(t0), int(steps), int(graph),
                ctypes.c_void_p(stream),
            )
        )

    def __del__(self):
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            try:
                self._lib.cwb_plan_destroy(handle)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None


def ptr(tensor: torch.Tensor | None) -> int | None:
    return None if tensor is None else tensor.data_ptr()


def level(stack: torch.Tensor, *, mul: int = 1, add: int = 0, period: int = 0) -> Level:
    """Level `(mul * t + add) mod period` (no wrap for period 0) of a stack of fields."""
    return Level(stack.data_ptr(), int(stack[0].numel()), int(mul), int(add), int(period),
                 int(stack.shape[0]))


def fixed(field: torch.Tensor) -> Level:
    """A level that is the same field every step."""
    return Level(field.data_ptr(), 0, 0, 0, 0, 1)


def points(lin: torch.Tensor | None, record: torch.Tensor | None, *, weight=None,
           row_mul: int = 1, row_add: int = 0, store: int = STORE_NATIVE) -> Points:
    if lin is None or lin.numel() == 0:
        return Points(None, None, None, 0, 0, 0, 0)
    return Points(
        lin.data_ptr(), ptr(weight), ptr(record), int(lin.numel()), int(row_mul),
        int(row_add), int(store),
    )


def op(kind: int, **fields) -> Op:
    o = Op()
    o.kind = kind
    for name, value in fields.items():
        if name == "memory":
            for d, m in enumerate(value):
                o.memory[d] = None if m is None else m.data_ptr()
        elif name == "factors":
            for d, f in enumerate(value):
                o.factors[d] = float(f)
        elif name in ("g_mass", "g_stiff"):
            setattr(o, name, ptr(value))
        else:
            setattr(o, name, value)
    return o


def launches() -> int:
    """Kernels the library has launched in this process."""
    return int(library().cwb_launches())


class Batch:
    """A native batch of 2D forward steps (cwb_batch_*), one item a problem."""

    def __init__(self, items: list[BatchItem]):
        self._lib = library()
        array = (BatchItem * len(items))(*items)
        handle = ctypes.c_void_p()
        check(self._lib.cwb_batch_create(array, len(items), ctypes.byref(handle)))
        self.handle = handle

    def tune(self, steps: int) -> int:
        stream = torch.cuda.current_stream().cuda_stream
        check(self._lib.cwb_batch_tune(self.handle, int(steps), ctypes.c_void_p(stream)))
        return int(self._lib.cwb_batch_threads(self.handle))

    def march(self, t0: int, steps: int, graph: bool = True) -> None:
        stream = torch.cuda.current_stream().cuda_stream
        check(self._lib.cwb_batch_march(self.handle, int(t0), int(steps), int(graph),
                                        ctypes.c_void_p(stream)))

    def __del__(self):
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            try:
                self._lib.cwb_batch_destroy(handle)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None


def conv_fwd(x, w, bias, y16=None, y32=None, *, relu=False, mask=None) -> None:
    """cwb_conv_bf16_fwd: x (B, H, W, cin) bf16, w (cout, kpad) bf16, into y16 / y32."""
    B, H, W, cin = x.shape
    out = y16 if y16 is not None else y32
    cout = out.shape[-1]
    stream = torch.cuda.current_stream().cuda_stream
    check(library().cwb_conv_bf16_fwd(ptr(x), ptr(w), ptr(bias), ptr(mask), ptr(y16), ptr(y32),
                                      B, H, W, cin, cout, int(relu), ctypes.c_void_p(stream)))


def conv_bwd(dy, x, dw, db=None) -> None:
    """cwb_conv_bf16_bwd: dw (cout, kpad) += weight gradient, db (cout) += bias gradient."""
    B, H, W, cin = x.shape
    cout = dy.shape[-1]
    stream = torch.cuda.current_stream().cuda_stream
    check(library().cwb_conv_bf16_bwd(ptr(dy), ptr(x), ptr(dw), ptr(db), B, H, W, cin, cout,
                                      ctypes.c_void_p(stream)))

