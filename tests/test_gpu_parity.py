"""The CUDA path against the reference's outputs and the CPU oracle.

Fixture cases come from the reference itself (tests/golden); the larger cases are
seeded and checked against the oracle. The kernels keep the reference's order of
operations and are built without fused multiply-adds the source does not ask for, so
the bar is equality; a 1e-5 relative L2 tolerance is checked as well so
a failure says how far off it is.
"""

import numpy as np
import pytest
import torch

import cases
from oracle import oracle as o

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2, float32 wavefields and traces


def _interior(fx):
    return tuple(slice(0, int(n)) for n in fx["Nx"])


@pytest.mark.parametrize("name", cases.FORWARD)
def test_simulate_matches_reference(name):
    from cuwave_b200 import Source, simulate

    fx = cases.load(name)
    sim, design = cases.product_sim(fx)
    src = Source(fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
    field, traces = simulate(sim, src, design.copy(), fx["sensors"])
    field, traces = field.cpu().numpy(), traces.cpu().numpy()
    assert cases.rel_l2(field, fx["field"]) <= TOL
    assert cases.rel_l2(traces, fx["traces"]) <= TOL
    np.testing.assert_array_equal(field, fx["field"])
    np.testing.assert_array_equal(traces, fx["traces"])


@pytest.mark.parametrize("name", cases.GRADIENT)
def test_sensitivity_matches_reference(name):
    from cuwave_b200 import Source
    from cuwave_b200.sensitivity import l2_misfit, sensitivity, source_sensitivity

    fx = cases.load(name)
    sim, design = cases.product_sim(fx)
    src = Source(fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
    cost, grads, traces, info = sensitivity(sim, src, design.copy(), fx["sensors"], l2_misfit(fx["observed"]))
    assert info == {}
    np.testing.assert_array_equal(traces.cpu().numpy(), fx["traces"])
    for key, ref in (("mass", fx["g_mass"]), ("stiff", fx["g_stiff"])):
        got = grads[key].cpu().numpy()
        assert cases.rel_l2(got, ref) <= 1e-4, key
        np.testing.assert_array_equal(got, ref)
    assert cost == pytest.approx(float(fx["cost"]), rel=1e-4)
    _, gradient, _, _ = source_sensitivity(sim, src, design.copy(), fx["sensors"], l2_misfit(fx["observed"]))
    np.testing.assert_array_equal(gradient.cpu().numpy(), fx["source_gradient"])


def _random_case(ndim, R, *, dirichlet=0, pml=0, uniform=False, damping=False, seed=1,
                 dtype=np.float32, nsrc=3, nsens=5, Nx=None, faces=None):
    """A seeded case with a heterogeneous stiffness, for the oracle and the product."""
    rng = np.random.default_rng(seed)
    if Nx is None:
        Nx = (27, 29) if ndim == 2 else (19, 21, 23)
    Nx = tuple(n + 2 * pml for n in Nx)
    shape = o.padded(Nx)
    stiff = np.zeros(shape, dtype)
    minv = np.zeros(shape, dtype)
    logical = tuple(slice(0, n) for n in Nx)
    stiff[logical] = 1.0 if uniform else rng.uniform(0.6, 1.4, Nx)
    minv[logical] = rng.uniform(0.7, 1.3, Nx)
    o.mirror_ghosts(Nx, stiff)
    o.mirror_ghosts(Nx, minv)
    dt = 0.4 * o.stable_dt((1.0,) * ndim, 1.3 * 1.2, 2 * R, "optimized")
    widths = None
    if pml:
        lined = set(range(2 * ndim)) if faces is None else set(faces)
        widths = tuple(tuple(pml if 2 * d + side in lined else 0 for side in (0, 1)) for d in range(ndim))
    profiles = o.pml_profiles(Nx, (1.0,) * ndim, dt, widths, pml, 1.6, 1e-6, 0.0, dtype) if pml else None
    src = np.stack([rng.integers(2, n - 2, nsrc) for n in Nx]).astype(np.int32)
    sens = np.stack([rng.integers(1, n - 1, nsens) for n in Nx]).astype(np.int32)
    N = 40
    signal = rng.standard_normal((N, nsrc)).astype(dtype)
    damp = None
    if damping:
        damp = np.zeros(shape, dtype)
        damp[logical] = rng.uniform(0.0, 0.5, Nx)
    neumann = ((1 << (2 * ndim)) - 1) & ~dirichlet
    case = o.Case(Nx=Nx, R=R, coeffs=o.cell_coefficients(R, "optimized"),
                  factors=[dtype(2 * dt**2)] * ndim, dt=dt, stiff=stiff, minv=minv, dtype=dtype,
                  dirichlet=dirichlet, neumann=neumann, damping=damp, widths=widths,
                  profiles=profiles, source_lin=cases.flat({"Nx": np.array(Nx)}, src),
                  signal=signal, sensor_lin=cases.flat({"Nx": np.array(Nx)}, sens))
    case.source_weight = case.excitation_weights(case.source_lin)
    return case, dict(Nx=Nx, dt=dt, src=src, sens=sens, N=N, pml=pml, dirichlet=dirichlet, faces=faces)


def _product(case, meta):
    """Run the native march on the oracle case's own arrays (materials bypass the hooks)."""
    from cuwave_b200 import _native as nat
    from cuwave_b200 import AcousticWave, Dirichlet, Neumann, Pml
    from cuwave_b200.wave import Shot, forward_ops, pml_memory

    ndim = len(meta["Nx"])
    boundary = tuple(
        tuple(Dirichlet if (meta["dirichlet"] >> (2 * d + s)) & 1 else Neumann for s in (0, 1))
        for d in range(ndim)
    )
    pml = Pml(width=meta["pml"], wavespeed=1.6, faces=meta.get("faces")) if meta["pml"] else None
    precision = "float32" if case.dtype == np.float32 else "float64"
    sim = AcousticWave(Nx=meta["Nx"], dx=(1.0,) * ndim, N=meta["N"], dt=meta["dt"],
                       precision=precision, space_order=2 * case.R, boundary=boundary, pml=pml,
                       rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=2.0,
                       damping=case.damping)
    dev = torch.device("cuda")
    t = lambda a: None if a is None else torch.as_tensor(a, device=dev)  # noqa: E731
    stiff = t(case.stiff)
    mat = {"stiff": stiff, "minv": t(case.minv), "damping": t(case.damping),
           "profiles": [t(p) for p in (case.profiles or [None] * 3)] + [None] * (3 - ndim),
           "uniform": bool((case.stiff[tuple(slice(0, n) for n in meta["Nx"])] == case.stiff.flat[0]).all()),
           "stiff_value": float(case.stiff.flat[0])}
    mat["profiles"] = mat["profiles"][:3]
    shot = Shot(t(meta["src"]), t(case.source_lin), t(case.source_weight), t(case.signal),
                foldable=bool(((meta["src"] >= 1) & (meta["src"] <= np.array(meta["Nx"])[:, None] - 2)).all()))
    U = torch.zeros((2, *case.shape), dtype=stiff.dtype, device=dev)
    memory = pml_memory(sim, 3, dev)
    um = torch.zeros((meta["N"], case.sensor_lin.size), dtype=stiff.dtype, device=dev)
    ops = forward_ops(sim, mat, nat.level(U, add=0, period=2), nat.level(U, add=1, period=2),
                      nat.level(U, add=0, period=2), shot, memory,
                      records=[(t(case.sensor_lin), um, 1, 0, 0)])
    sim.plan().march(ops, 0, meta["N"])
    return U[(meta["N"] - 1) % 2].cpu().numpy(), um.cpu().numpy()


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("R", [1, 2, 3, 4, 5, 6, 7, 8])
def test_heterogeneous_step_matches_oracle(ndim, R):
    case, meta = _random_case(ndim, R, dirichlet=0b0110 if ndim == 2 else 0b100110)
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    assert cases.rel_l2(field, ref_field) <= TOL
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


@pytest.mark.parametrize("ndim,R,pml", [(2, 4, 5), (3, 4, 4), (3, 8, 3), (2, 1, 3), (3, 2, 4)])
def test_pml_step_matches_oracle(ndim, R, pml):
    case, meta = _random_case(ndim, R, pml=pml, seed=3)
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


@pytest.mark.parametrize("ndim", [2, 3])
def test_damped_float64_step_matches_oracle(ndim):
    case, meta = _random_case(ndim, 3, damping=True, dtype=np.float64, seed=5)
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


def test_uniform_stiffness_path_matches_oracle():
    case, meta = _random_case(3, 4, uniform=True, pml=3, seed=7)
    field, _ = _product(case, meta)
    ref_field, _ = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)


@pytest.mark.parametrize("R,dirichlet,pml,damping", [
    (1, 0b000000, 0, False), (2, 0b100110, 0, False), (3, 0b011001, 3, False),
    (4, 0b100110, 4, False), (4, 0b000000, 0, True), (4, 0b111111, 0, False), (2, 0b010101, 6, False),
    (4, 0b011010, 13, False), (3, 0b000000, 23, False),
])
def test_blocked_uniform_step_matches_oracle(R, dirichlet, pml, damping):
    """Several 64 x 16 tiles and 32-plane chunks, an axis-2 extent with padding, Dirichlet
    and Neumann faces, pml slabs, damping and folded sources on the blocked 3D kernel of a
    uniform stiffness. Slabs of 13 and 23 cells give the axis-1 pml kernel several
    segments of rows a side, the last one short."""
    case, meta = _random_case(3, R, dirichlet=dirichlet, pml=pml, uniform=True, damping=damping,
                              seed=11 + R, nsrc=6, nsens=9, Nx=(45, 37, 139))
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


@pytest.mark.parametrize("R,faces,pml,dirichlet", [
    (4, (1, 2, 5), 20, 0b000000), (4, (0, 3, 4), 9, 0b100001), (3, (2, 3), 17, 0b000100),
    (2, (4, 5), 70, 0b000000), (1, (0, 1, 3, 4), 5, 0b110000),
])
def test_blocked_step_with_pml_on_some_faces(R, faces, pml, dirichlet):
    """The blocked 3D step's pml on a subset of faces (a side lined, the other not), the
    slabs of axes 1 and 2 taken inside the step's own tiles: tiles that meet a slab but no
    wall, an axis-2 slab wider than a tile, Dirichlet faces beside a lined one."""
    case, meta = _random_case(3, R, dirichlet=dirichlet, pml=pml, uniform=True, seed=200 + R,
                              nsrc=4, nsens=9, Nx=(41, 53, 97), faces=faces)
    meta["N"] = 24
    case.signal = case.signal[:24]
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


@pytest.mark.parametrize("dirichlet,on_mirrors", [(0b0000, True), (0b1010, True),
                                                   (0b0101, False), (0b0000, False)])
def test_quad_2d_pml_step_ghosts_folded_or_not(dirichlet, on_mirrors):
    """The 2D quad step with a pml refills the face ghosts inside its pml launch where no
    source sits on the mirror rows and columns (2, N0 - 3; 2, NF - 3), and leaves a face to
    the refill launch where one does: both equal to the oracle, on a grid of several row
    chunks too large for the multi-step march."""
    case, meta = _random_case(2, 4, dirichlet=dirichlet, pml=6, uniform=True, seed=57, nsrc=4,
                              nsens=9, Nx=(611, 1090))
    meta["N"] = 12
    case.signal = case.signal[:12]
    if on_mirrors:
        Nx = meta["Nx"]
        src = meta["src"].copy()
        src[:, 0] = (2, Nx[1] // 2)
        src[:, 1] = (Nx[0] - 3, Nx[1] // 3)
        src[:, 2] = (Nx[0] // 2, 2)
        src[:, 3] = (Nx[0] // 3, Nx[1] - 3)
        meta["src"] = src
        case.source_lin = cases.flat({"Nx": np.array(Nx)}, src)
        case.source_weight = case.excitation_weights(case.source_lin)
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


@pytest.mark.parametrize("inside,dirichlet,receivers", [
    (False, 0b0000, "clear"), (False, 0b1001, "clear"), (True, 0b0000, "clear"),
    (False, 0b0000, "on a source"), (False, 0b0000, "in a slab"),
])
def test_quad_2d_pml_launch_adds_the_sources(inside, dirichlet, receivers):
    """The 2D quad step's pml launch adds the step's sources itself when none sits on a
    slab node (two of them on one node here), and leaves them to a launch of their own
    when one does; it reads the receivers that follow when they are final after the update
    (clear of the slabs and the sources), and leaves them to the record launch when one
    sits on a source or a slab node: all equal to the oracle."""
    pml = 6
    case, meta = _random_case(2, 4, dirichlet=dirichlet, pml=pml, uniform=True, seed=63, nsrc=4,
                              nsens=9, Nx=(611, 1090))
    meta["N"] = 12
    case.signal = case.signal[:12]
    Nx = meta["Nx"]
    src = np.array([[pml + 3, Nx[0] // 2, Nx[0] // 2, Nx[0] - pml - 4],
                    [Nx[1] // 3, Nx[1] // 2, Nx[1] // 2, Nx[1] - pml - 4]], np.int32)
    if inside:
        src[:, 3] = (Nx[0] // 3, pml)  # a node of the axis-1 slab
    meta["src"] = src
    case.source_lin = cases.flat({"Nx": np.array(Nx)}, src)
    case.source_weight = case.excitation_weights(case.source_lin)
    sens = np.stack([np.full(9, Nx[0] // 4), np.linspace(pml + 2, Nx[1] - pml - 3, 9).astype(int)]).astype(np.int32)
    if receivers == "on a source":
        sens[:, 4] = src[:, 1]
    elif receivers == "in a slab":
        sens[:, 4] = (pml - 1, Nx[1] // 2)
    meta["sens"] = sens
    case.sensor_lin = cases.flat({"Nx": np.array(Nx)}, sens)
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


@pytest.mark.parametrize("dirichlet", [0b000000, 0b110000])
def test_blocked_step_with_sources_on_the_ghost_mirrors(dirichlet):
    """Sources on the columns whose values the fast axis' face ghosts copy (x = 2 and
    NF - 3): the ghosts must take the value after the excitation, so the axis-2 pml
    launch leaves those faces to the refill; the other cases fold them into it."""
    case, meta = _random_case(3, 4, dirichlet=dirichlet, pml=4, uniform=True, seed=91, nsrc=3,
                              nsens=9, Nx=(45, 37, 139))
    Nx = meta["Nx"]
    src = meta["src"].copy()
    src[2, 0] = 2
    src[2, 1] = Nx[2] - 3
    meta["src"] = src
    case.source_lin = cases.flat({"Nx": np.array(Nx)}, src)
    case.source_weight = case.excitation_weights(case.source_lin)
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


@pytest.mark.parametrize("R,dirichlet,pml,damping", [
    (1, 0b0000, 0, False), (2, 0b0110, 0, False), (3, 0b1001, 3, False),
    (4, 0b0110, 4, False), (4, 0b0000, 0, True), (4, 0b1111, 0, False), (2, 0b0101, 6, False),
    (5, 0b0110, 0, False), (6, 0b1001, 7, False), (7, 0b0000, 0, True), (8, 0b0101, 9, False),
])
def test_quad_2d_uniform_step_matches_oracle(R, dirichlet, pml, damping):
    """The 2D quad step of a uniform stiffness on a grid of many row chunks and quads, an
    axis-1 extent with padding, Dirichlet and Neumann faces, pml slabs, damping and
    sources."""
    case, meta = _random_case(2, R, dirichlet=dirichlet, pml=pml, uniform=True, damping=damping,
                              seed=31 + R, nsrc=6, nsens=9, Nx=(187, 139))
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


def test_quad_2d_step_by_step_on_a_large_grid():
    """A 2D grid past the multi-step march's size runs the quad step launch by launch
    (sources and refill as their own launches): still equal to the oracle's."""
    case, meta = _random_case(2, 4, dirichlet=0b0110, pml=5, uniform=True, seed=77, nsrc=3,
                              nsens=9, Nx=(603, 1101))
    meta["N"] = 20
    case.signal = case.signal[:20]
    field, traces = _product(case, meta)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(field, ref_field)
    np.testing.assert_array_equal(traces, ref_traces)


@pytest.mark.parametrize("ndim,R,dirichlet,pml,damping,Nx", [
    (2, 1, 0b0000, 0, False, (67, 91)), (2, 2, 0b0110, 0, False, (81, 73)),
    (2, 3, 0b1001, 4, False, (67, 91)), (2, 4, 0b0110, 5, False, (75, 139)),
    (2, 4, 0b0000, 0, True, (67, 91)), (2, 4, 0b1111, 0, False, (59, 101)),
    (3, 2, 0b100110, 3, False, (23, 21, 27)),
    # 3D: several chunks of planes and tiles, radius 1 to 4, walls, a pml, damping
    (3, 1, 0b000000, 0, False, (37, 29, 71)), (3, 3, 0b011001, 4, False, (30, 41, 75)),
    (3, 4, 0b000000, 5, False, (29, 35, 77)), (3, 4, 0b111111, 0, False, (27, 25, 45)),
    (3, 4, 0b000000, 0, True, (27, 31, 53)), (3, 2, 0b010100, 6, False, (19, 33, 23)),
    # the narrowest grids a pml allows (its width + R on both sides leaves one interior
    # node): the transpose's gathered rows and columns leave one row or a few columns
    (2, 4, 0b0110, 6, False, (11, 13)), (2, 3, 0b1001, 5, False, (9, 61)),
    (2, 2, 0b0101, 4, False, (53, 7)), (2, 1, 0b0000, 3, False, (41, 37)),
])
def test_uniform_sensitivity_matches_oracle(ndim, R, dirichlet, pml, damping, Nx):
    """sensitivity of a uniform stiffness (the quad adjoint in 2D) on grids of many row
    chunks and quads, Dirichlet and Neumann faces, pml slabs and damping: the gradients
    and traces equal the oracle's to the bit."""
    from cuwave_b200 import AcousticWave, Dirichlet, Neumann, Pml, Source
    from cuwave_b200.sensitivity import l2_misfit, sensitivity

    case, meta = _random_case(ndim, R, dirichlet=dirichlet, pml=pml, uniform=True, damping=damping,
                              seed=51 + R, nsrc=2, nsens=7, Nx=Nx)
    rng = np.random.default_rng(9)
    observed = rng.standard_normal((meta["N"], meta["sens"].shape[1])).astype(case.dtype) * 1e-3
    _, ref, ref_traces = case.sensitivity(meta["N"], o.l2(observed))
    boundary = tuple(
        tuple(Dirichlet if (dirichlet >> (2 * d + s)) & 1 else Neumann for s in (0, 1))
        for d in range(ndim)
    )
    sim = AcousticWave(Nx=meta["Nx"], dx=(1.0,) * ndim, N=meta["N"], dt=meta["dt"],
                       precision="float32", space_order=2 * R, boundary=boundary,
                       pml=Pml(width=pml, wavespeed=1.6) if pml else None,
                       rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=2.0, damping=case.damping)
    dev = torch.device("cuda")
    t = lambda a: None if a is None else torch.as_tensor(a, device=dev)  # noqa: E731
    mat = {"stiff": t(case.stiff), "minv": t(case.minv), "damping": t(case.damping),
           "profiles": ([t(p) for p in case.profiles] if case.profiles else [None] * ndim) + [None] * (3 - ndim),
           "uniform": True, "stiff_value": float(case.stiff.flat[0])}
    source = Source(meta["src"], case.signal)
    _, grads, traces, _ = sensitivity(sim, source, None, meta["sens"], l2_misfit(t(observed)), _mat=mat)
    np.testing.assert_array_equal(traces.cpu().numpy(), ref_traces)
    for key in ("mass", "stiff"):
        np.testing.assert_array_equal(grads[key].cpu().numpy(), ref[key])


@pytest.mark.parametrize("inside", [False, True])
def test_quad_adjoint_gather_applies_the_load(inside):
    """The 2D quad adjoint's pml gather applies the adjoint load that follows it when no
    receiver sits on a node the gather reaches (two receivers on one node here), and
    leaves it to a launch of its own when one does: the gradients and traces equal the
    oracle's to the bit either way."""
    from cuwave_b200 import AcousticWave, Neumann, Pml, Source
    from cuwave_b200.sensitivity import l2_misfit, sensitivity

    R, pml = 4, 5
    case, meta = _random_case(2, R, pml=pml, uniform=True, seed=71, nsrc=2, nsens=6, Nx=(75, 139))
    Nx = meta["Nx"]
    reach = pml + R
    sens = np.array([[reach + 2, Nx[0] // 2, Nx[0] // 2, Nx[0] - reach - 3, 30, 40],
                     [reach + 2, Nx[1] // 2, Nx[1] // 2, Nx[1] - reach - 3, 60, 90]], np.int32)
    if inside:
        sens[:, 5] = (Nx[0] // 2, reach - 1)  # within R of the axis-1 slab
    meta["sens"] = sens
    case.sensor_lin = cases.flat({"Nx": np.array(Nx)}, sens)
    rng = np.random.default_rng(9)
    observed = rng.standard_normal((meta["N"], sens.shape[1])).astype(case.dtype) * 1e-3
    _, ref, ref_traces = case.sensitivity(meta["N"], o.l2(observed))
    sim = AcousticWave(Nx=Nx, dx=(1.0, 1.0), N=meta["N"], dt=meta["dt"], precision="float32",
                       space_order=2 * R, boundary=((Neumann, Neumann), (Neumann, Neumann)),
                       pml=Pml(width=pml, wavespeed=1.6), rho1=1.0, rho2=1.0, kappa1=1.0,
                       kappa2=2.0)
    dev = torch.device("cuda")
    t = lambda a: torch.as_tensor(a, device=dev)  # noqa: E731
    mat = {"stiff": t(case.stiff), "minv": t(case.minv), "damping": None,
           "profiles": [t(p) for p in case.profiles] + [None],
           "uniform": True, "stiff_value": float(case.stiff.flat[0])}
    source = Source(meta["src"], case.signal)
    _, grads, traces, _ = sensitivity(sim, source, None, sens, l2_misfit(t(observed)), _mat=mat)
    np.testing.assert_array_equal(traces.cpu().numpy(), ref_traces)
    for key in ("mass", "stiff"):
        np.testing.assert_array_equal(grads[key].cpu().numpy(), ref[key])


@pytest.mark.parametrize("name", cases.GRADIENT)
def test_reconstruction_matches_reference(name):
    """The strip-replay adjoint with two checkpoints against the reference's own run."""
    from cuwave_b200 import Source
    from cuwave_b200.sensitivity import l2_misfit, reconstruction_sensitivity

    fx = cases.load(name)
    sim, design = cases.product_sim(fx)
    src = Source(fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
    cost, grads, traces, info = reconstruction_sensitivity(
        sim, src, design.copy(), fx["sensors"], l2_misfit(fx["observed"]), checkpoints=2
    )
    assert info["strip"] == int(fx["rec_strip"])
    assert info["segment"] == int(fx["rec_segment"])
    assert info["sweeps"] == pytest.approx(float(fx["rec_sweeps"]))
    np.testing.assert_array_equal(traces.cpu().numpy(), fx["traces"])
    for key, ref in (("mass", fx["rec_g_mass"]), ("stiff", fx["rec_g_stiff"])):
        got = grads[key].cpu().numpy()
        assert cases.rel_l2(got, ref) <= 1e-4, key
        np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("name", ["grad2d_r4_pml", "grad3d_r2_pml", "grad2d_r4_damped"])
@pytest.mark.parametrize("checkpoints", [None, 0, 1, 64])
def test_reconstruction_matches_sensitivity(name, checkpoints):
    """Replaying the strip reads only reversible nodes: the gradient equals the stored-
    history one where the strip shields it, at round-off in float64 as the reference pins
    it (cuwave sensitivity_test.py:910-1113)."""
    from cuwave_b200 import Source
    from cuwave_b200.sensitivity import l2_misfit, reconstruction_sensitivity, sensitivity

    fx = dict(cases.load(name))
    fx["precision"] = np.array("float64")
    sim, design = cases.product_sim(fx)
    src = Source(fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
    objective = l2_misfit(fx["observed"])
    _, ref, _, _ = sensitivity(sim, src, design.copy(), fx["sensors"], objective)
    _, got, _, info = reconstruction_sensitivity(sim, src, design.copy(), fx["sensors"], objective,
                                                 checkpoints=checkpoints)
    from cuwave_b200.sensitivity import reconstruction_nodes

    _, valid = reconstruction_nodes(sim, design.copy())
    for key in ("mass", "stiff"):
        a = got[key][valid].cpu().numpy()
        b = ref[key][valid].cpu().numpy()
        assert cases.rel_l2(a, b) <= 1e-7, key
    assert info["drift"] < 1e-7


@pytest.mark.parametrize("name", [n for n in cases.FORWARD + cases.GRADIENT if "damped" in n])
def test_sponge_matches_reference(name):
    """`sponge` builds the reference's damping field from the design (boundary.py:238-269)."""
    from cuwave_b200 import sponge

    fx = cases.load(name)
    sim, design = cases.product_sim(fx)
    field = sponge(sim, design.copy(), width=4, beta=0.3)
    np.testing.assert_array_equal(field, fx["damping_field"])


@pytest.mark.parametrize("name", ["grad2d_r4_pml", "grad3d_r2_pml", "grad2d_r4_damped"])
@pytest.mark.parametrize("precision,stored,tolerance", [("float64", "float32", 1e-6),
                                                        ("float64", "bfloat16", 1e-2),
                                                        ("float32", "bfloat16", 1e-2)])
def test_narrower_strip_trades_exactness_for_memory(name, precision, stored, tolerance):
    """A strip stored narrower than the field (bfloat16 bits, or float32 under float64)
    rebuilds the forward field from rounded values: the gradient stays within the
    reference's own bounds of the stored-history one where the strip shields it
    (cuwave sensitivity_test.py:1015-1035: 1e-6 for float32 under float64, 1e-2 for
    bfloat16), on the mass-and-stiffness combination the design sees."""
    from cuwave_b200 import Source
    from cuwave_b200.sensitivity import (l2_misfit, reconstruction_nodes, reconstruction_sensitivity,
                                         sensitivity)

    fx = dict(cases.load(name))
    fx["precision"] = np.array(precision)
    sim, design = cases.product_sim(fx)
    src = Source(fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
    objective = l2_misfit(fx["observed"].astype(cases.dtype_of(fx)))
    _, ref, _, _ = sensitivity(sim, src, design.copy(), fx["sensors"], objective)
    _, got, _, info = reconstruction_sensitivity(sim, src, design.copy(), fx["sensors"], objective,
                                                 strip_dtype=stored)
    _, valid = reconstruction_nodes(sim, design.copy())
    d_mass, d_stiff = sim.parametrization_jacobian(None)

    def combine(g):
        return (d_mass * g["mass"] + d_stiff * g["stiff"])[valid].double().cpu().numpy()

    a, b = combine(got), combine(ref)
    rel = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    assert rel < tolerance, rel
    if stored == "bfloat16":
        assert rel > 0, "a bfloat16 strip rounds what it stores"


def test_strip_no_narrower_is_refused():
    from cuwave_b200 import Source
    from cuwave_b200.sensitivity import l2_misfit, reconstruction_sensitivity

    fx = cases.load("grad2d_r4_pml")
    sim, design = cases.product_sim(fx)
    src = Source(fx["source"], fx["signal"])
    with pytest.raises(ValueError):
        reconstruction_sensitivity(sim, src, design.copy(), fx["sensors"], l2_misfit(fx["observed"]),
                                   strip_dtype="float32")
