"""The allocation-free march (`cwb_march_static`) against the plan-based `cwb_march`.

`cwb_march_static` serves callers that cannot let this library allocate device memory
(a host that owns the GPU through its own pool): it keeps its step counter, error flag
and folded-source lists in a static device array instead of a plan. It must step
exactly what `cwb_march` steps, call after call, since every call reuses that array.
Collected last on purpose, so a failure here cannot hide any other test's result.
"""

import ctypes

import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu


def _forward_ops(sim, mat, shot, U, um, sensor_lin):
    from cuwave_b200 import _native as nat
    from cuwave_b200.wave import forward_ops, pml_memory

    memory = pml_memory(sim, 3, U.device)
    ops = forward_ops(sim, mat, nat.level(U, add=0, period=2), nat.level(U, add=1, period=2),
                      nat.level(U, add=0, period=2), shot, memory,
                      records=[(sensor_lin, um, 1, 0, nat.STORE_NATIVE)])
    return ops, memory


@pytest.mark.parametrize("name", ["fwd3d_r4_pml", "fwd2d_r3_pml_mixed"])
def test_static_march_matches_plan_march(name):
    from cuwave_b200 import _native as nat
    from cuwave_b200.wave import flatten_indices, prepare_shot

    lib = nat.library()
    lib.cwb_march_static.argtypes = [ctypes.POINTER(nat.Grid), ctypes.POINTER(nat.Op),
                                     ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                     ctypes.c_void_p]
    lib.cwb_march_static.restype = ctypes.c_int

    fx = cases.load(name)
    sim, design = cases.product_sim(fx)
    N = int(fx["N"])
    mat = sim.build_materials(design.copy())
    shot = prepare_shot(sim, mat, fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
    assert shot.foldable, "the case must fold its sources, so the static lists are used"
    sensor_lin = flatten_indices(sim, fx["sensors"])
    dev = torch.device("cuda")

    def fresh():
        U = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
        um = torch.zeros((N, sensor_lin.numel()), dtype=sim.dtype, device=dev)
        return U, um

    # the existing entry point, through its plan
    U_ref, um_ref = fresh()
    ops, memory = _forward_ops(sim, mat, shot, U_ref, um_ref, sensor_lin)
    sim.plan().march(ops, 0, N)
    torch.cuda.synchronize()
    ref_field = U_ref[(N - 1) % 2].cpu().numpy()
    ref_traces = um_ref.cpu().numpy()

    # the allocation-free entry point, twice in a row on fresh fields
    grid = sim.plan().grid
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        U, um = fresh()
        ops, memory = _forward_ops(sim, mat, shot, U, um, sensor_lin)
        array = (nat.Op * len(ops))(*ops)
        rc = lib.cwb_march_static(ctypes.byref(grid), array, len(ops), 0, N, stream)
        assert rc == 0, lib.cwb_last_error().decode()
        field = U[(N - 1) % 2].cpu().numpy()
        traces = um.cpu().numpy()
        assert cases.rel_l2(field, ref_field) <= 1e-5, call
        assert cases.rel_l2(traces, ref_traces) <= 1e-5, call
        np.testing.assert_array_equal(field, ref_field)
        np.testing.assert_array_equal(traces, ref_traces)


def test_static_march_builds_its_source_lists_in_the_array():
    """A heterogeneous stiffness (a ScalarWave design) steps on the row kernel, which folds
    the sources into the step through per-block lists; with two shots in one op list both
    lists land in the static array one after the other. Each shot must equal what the
    plan-based march gives and what the reference gives, on two calls in a row."""
    from cuwave_b200 import _native as nat
    from cuwave_b200.wave import flatten_indices, forward_ops, pml_memory, prepare_shot

    lib = nat.library()
    lib.cwb_march_static.restype = ctypes.c_int
    fx = cases.load("fwd2d_scalar_r2")
    sim, design = cases.product_sim(fx)
    N = int(fx["N"])
    mat = sim.build_materials(design.copy())
    assert not mat["uniform"], "the case must have a heterogeneous stiffness"
    signal = fx["signal"].astype(np.float32)
    # the fixture's shot, and a second one of two sources elsewhere with its own signal
    second = np.array([[5, int(fx["Nx"][0]) - 6], [int(fx["Nx"][1]) - 5, 4]], np.int32)
    signal2 = np.ascontiguousarray(np.stack([signal[:, 0], -0.5 * signal[:, 0]], axis=1))
    shots = [prepare_shot(sim, mat, fx["source"], signal), prepare_shot(sim, mat, second, signal2)]
    assert all(s.foldable for s in shots)
    sensor_lin = flatten_indices(sim, fx["sensors"])
    dev = torch.device("cuda")

    def marched(run):
        fields = []
        ops = []
        for shot in shots:
            U = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
            um = torch.zeros((N, sensor_lin.numel()), dtype=sim.dtype, device=dev)
            ops += forward_ops(sim, mat, nat.level(U, add=0, period=2), nat.level(U, add=1, period=2),
                               nat.level(U, add=0, period=2), shot, pml_memory(sim, 3, dev),
                               records=[(sensor_lin, um, 1, 0, nat.STORE_NATIVE)])
            fields.append((U, um))
        assert sum(1 for op in ops if op.flags & nat.FOLD_SOURCES) == 2
        run(ops)
        torch.cuda.synchronize()
        return [(U[(N - 1) % 2].cpu().numpy(), um.cpu().numpy()) for U, um in fields]

    ref = marched(lambda ops: sim.plan().march(ops, 0, N))
    grid = sim.plan().grid
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def static(ops):
        array = (nat.Op * len(ops))(*ops)
        rc = lib.cwb_march_static(ctypes.byref(grid), array, len(ops), 0, N, stream)
        assert rc == 0, lib.cwb_last_error().decode()

    logical = tuple(slice(0, int(n)) for n in fx["Nx"])
    # the second shot through the oracle, the fixture holding only the first
    case = cases.oracle_case(fx)
    case.source_lin = cases.flat(fx, second)
    case.signal = signal2
    case.source_weight = case.excitation_weights(case.source_lin)
    oracle_field, oracle_traces = case.forward(N)
    for call in range(2):
        got = marched(static)
        for (field, traces), (rf, rt) in zip(got, ref):
            np.testing.assert_array_equal(field, rf)
            np.testing.assert_array_equal(traces, rt)
        np.testing.assert_array_equal(got[0][0][logical], fx["field"])
        np.testing.assert_array_equal(got[0][1], fx["traces"])
        np.testing.assert_array_equal(got[1][0][logical], oracle_field[logical])
        np.testing.assert_array_equal(got[1][1], oracle_traces)


def test_static_march_refuses_lists_past_its_array():
    """A march whose source lists cannot fit the static array is refused, not truncated.
    (A heterogeneous stiffness: its step folds the sources through per-block lists,
    which the register-blocked steps of a uniform stiffness do not build.)"""
    from cuwave_b200 import _native as nat
    from cuwave_b200.wave import prepare_shot

    lib = nat.library()
    lib.cwb_march_static.restype = ctypes.c_int
    fx = cases.load("fwd2d_r8")
    sim, design = cases.product_sim(fx)
    mat = sim.build_materials(design.copy())
    mat["stiff"] = mat["stiff"] * (1.0 + 0.1 * torch.rand_like(mat["stiff"]))
    mat["uniform"] = False
    # 20000 sources on interior nodes: 320 kB of list entries, past the 256 kB array
    rng = np.random.default_rng(0)
    count = 20000
    position = np.stack([rng.integers(1, n - 1, count) for n in sim.Nx]).astype(np.int32)
    signal = np.zeros((int(fx["N"]), count), np.float32)
    shot = prepare_shot(sim, mat, position, signal)
    U = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device="cuda")
    from cuwave_b200.wave import forward_ops, pml_memory

    ops = forward_ops(sim, mat, nat.level(U, add=0, period=2), nat.level(U, add=1, period=2),
                      nat.level(U, add=0, period=2), shot, pml_memory(sim, 3, U.device))
    array = (nat.Op * len(ops))(*ops)
    rc = lib.cwb_march_static(ctypes.byref(sim.plan().grid), array, len(ops), 0, 1,
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == -1
    assert "static scratch" in lib.cwb_last_error().decode()
