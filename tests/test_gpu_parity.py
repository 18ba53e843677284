"""Parity of the sm_100a solid path with the CPU oracle (the reference's own kernels).

Tolerances (relative L2 of displacement unless stated):
* FP64 form vs the FP64 oracle: <= 1e-12;
* FP32-state form vs the FP64 oracle: <= 1e-5;
* one-time FP64 set-up arrays (templates, mass, load, assembled blocks): <= 1e-13 max-relative.
"""
import os

import numpy as np
import pytest
import torch

from cvfes_b200 import _lib
from cvfes_b200._lib import call, ptr
from cvfes_b200.mesh import SolidMesh
from cvfes_b200.plan import SolidPlan, color_greedy
from cvfes_b200.solver import GPUSolidSolver, LocalComm
from oracle import solid_oracle as so

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
FP64_TOL = 1e-12
FP32_TOL = 1e-5


class Cfg:
    def __init__(self, dt, nSmp, precision=64, **kw):
        self.dt = dt
        self.nSmp = nSmp
        self.gpu = type("G", (), dict(precision=precision, use_graph=True, graph_chunk=kw.get("chunk", 6),
                                      watchdog=True, device=0, state=kw.get("state", "auto"),
                                      norms_every=kw.get("norms_every", 0),
                                      semantics=kw.get("semantics", "cpu")))()
        self.dt_f = 0.01
        self.exportBdyStressFilename = None
        self.useConstantStress = False
        self.constant_T = 1.0
        self.constant_pressure = 0.0
        self.pressure_ramp = "linear"


def golden(name):
    return dict(np.load(os.path.join(GOLD, name)))


def golden_mesh(g, **kw):
    return SolidMesh(g["nodes"], g["elements"], g["boundary"], g["coefK"].shape[1],
                     density=float(g["density"]), v=float(g["v"]), damp=float(g["damp"]),
                     coefK=g["coefK"], gthick=g["gthick"])


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


@pytest.mark.parametrize("name", ["tube8x6_element.npz", "tube6x5_nodal.npz"])
def test_setup_kernels_match_reference_assembly(lib, cuda, name):
    """Templates, lumped mass, unit load and block-CSR assembly vs the reference's outputs."""
    g = golden(name)
    nodes, elems = g["nodes"], g["elements"]
    N, E, S = len(nodes), len(elems), g["coefK"].shape[1]
    plan = SolidPlan(nodes, elems, 0, 0.0, float(g["v"]), float(g["density"]), cuda,
                     precisions=(32, 64), keep_full=True)
    plan.set_material(g["coefK"], g["gthick"])
    Kt, T, area = so.element_templates(nodes, elems, float(g["v"]))
    assert rel(plan.kt_full.view(E, 9, 9).cpu().numpy(), Kt) < 1e-13
    assert rel(plan.area.cpu().numpy(), area) < 1e-14
    lm = plan.lm.cpu().numpy()
    assert rel(np.repeat(lm, 3, axis=0), g["LM"]) < 1e-13
    fh = plan.fhat64.cpu().numpy()[:, :3].ravel()
    assert rel(fh, g["f"]) < 1e-13
    # block-CSR assembly in the reference layout, one launch per colour
    colors, nc = color_greedy(elems, N)
    order = np.argsort(colors, kind="stable").astype(np.int32)
    cptr = np.zeros(nc + 1, dtype=np.int64)
    cptr[1:] = np.cumsum(np.bincount(colors, minlength=nc))
    pos = so.block_positions(g["indptr"], g["indices"], elems).reshape(E, 9).astype(np.int32)
    K = torch.zeros((len(g["indices"]), S, 3, 3), dtype=torch.float64, device=cuda)
    pos_d = torch.from_numpy(pos).to(cuda)
    order_d = torch.from_numpy(order).to(cuda)
    call("cvfes_solid_assemble_bsr_f64", E, S, ptr(plan.kt_full), ptr(plan.coef64), ptr(pos_d),
         nc, ptr(cptr), ptr(order_d), ptr(K), torch.cuda.current_stream().cuda_stream)
    assert rel(K.cpu().numpy(), g["K"]) < 1e-13
    # and the reference-layout SpMV on it
    rng = np.random.default_rng(3)
    v = rng.standard_normal((3 * N, S))
    res = torch.zeros((3 * N, S), dtype=torch.float64, device=cuda)
    ip = torch.from_numpy(g["indptr"]).to(cuda)
    ix = torch.from_numpy(g["indices"]).to(cuda)
    vd = torch.from_numpy(v).to(cuda)
    call("cvfes_bsr_spmv_f64", N, S, ptr(ip), ptr(ix), ptr(K), ptr(vd), ptr(res),
         torch.cuda.current_stream().cuda_stream)
    ref = so.multiply_by_vector(g["indptr"], g["indices"], g["K"], v)
    assert rel(res.cpu().numpy(), ref) < 1e-13
    # template K*u equals the assembled block-CSR K*u
    d64 = plan.desc(64)
    out = torch.empty_like(res)
    call("cvfes_solid_kmul_f64", _lib.C.byref(d64), ptr(plan.coef64), ptr(vd), ptr(out), 0,
         torch.cuda.current_stream().cuda_stream)
    assert rel(out.cpu().numpy(), ref) < 1e-13
    d32 = plan.desc(32)
    v32 = vd.float()
    out32 = torch.empty_like(v32)
    call("cvfes_solid_kmul_f32", _lib.C.byref(d32), ptr(plan.coef32), ptr(v32), ptr(out32), 0,
         torch.cuda.current_stream().cuda_stream)
    assert rel(out32.double().cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("name", ["tube8x6_element.npz", "tube6x5_nodal.npz"])
@pytest.mark.parametrize("precision", [64, 32])
def test_solver_class_reproduces_golden_history(lib, cuda, name, precision):
    """GPUSolidSolver.Solve step by step against the reference kernels' history."""
    g = golden(name)
    mesh = golden_mesh(g)
    solver = GPUSolidSolver(LocalComm(), mesh, Cfg(float(g["dt"]), mesh.nSmp, precision))
    tol = FP64_TOL if precision == 64 else FP32_TOL
    k = 0
    for n, p in enumerate(g["pressures"]):
        solver.pressure = float(p)
        solver.Solve(n * float(g["dt"]), float(g["dt"]))
        if (n + 1) % 5 == 0:
            assert so.rel_l2(solver.displacement(), g["hist"][k]) < tol
            k += 1
    assert k == len(g["hist"])


def c0_mesh(S=8):
    from cvfes_b200.cases import CASES, build_mesh
    return build_mesh(CASES["tube64x128"], n_samples=S)


@pytest.fixture(scope="module")
def c0_oracle():
    """FP64 oracle history of the 64x128 tube, 8 samples, 400 steps (every 50 steps)."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    mesh = c0_mesh()
    coefK, gthick = mesh.element_coefficients()
    backend = "reference" if so.load_reference_module() is not None else "numpy"
    o = so.OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick,
                             mesh.density, mesh.v, mesh.damp, case.dt, backend=backend)
    hist = o.run(case.pressures(), history_every=50)
    return mesh, case, hist, backend


@pytest.mark.parametrize("precision,use_graph", [(64, True), (64, False), (32, True)])
def test_tube64x128_400_steps(lib, cuda, c0_oracle, precision, use_graph):
    """The 64x128 tube, 8 samples, 400 steps: FP64 <= 1e-12, FP32 <= 1e-5 at every 50th step."""
    mesh, case, hist, backend = c0_oracle
    cfg = Cfg(case.dt, mesh.nSmp, precision, chunk=24)
    solver = GPUSolidSolver(LocalComm(), mesh, cfg)
    pres = case.pressures()
    worst = 0.0
    for k in range(8):
        solver.Advance(pres[50 * k:50 * (k + 1)], use_graph=use_graph)
        err = so.rel_l2(solver.displacement(), hist[k])
        worst = max(worst, err)
    tol = FP64_TOL if precision == 64 else FP32_TOL
    print(f"precision={precision} graph={use_graph} oracle={backend} max rel-L2 = {worst:.3e}")
    assert worst < tol


def test_graph_replay_is_bitwise_equal_to_plain_launches(lib, cuda):
    mesh = c0_mesh(4)
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    out = []
    for use_graph in (True, False):
        s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 4, 32, chunk=12))
        s.Advance(case.pressures(100), use_graph=use_graph)
        out.append(s.local_displacement().clone())
    assert torch.equal(out[0], out[1])


def test_norms_and_watchdog(lib, cuda):
    mesh = c0_mesh(4)
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 4, 64))
    s.Advance(case.pressures(150))
    nrm = s.Norms()
    u = s.bufs[s.cur].cpu().numpy()
    up = s.bufs[s.prev].cpu().numpy()
    m = np.repeat(s.plan.lm.cpu().numpy(), 3, axis=0)
    assert np.allclose(nrm[:, 0], (u ** 2).sum(0), rtol=1e-12)
    assert np.allclose(nrm[:, 1], ((u - up) ** 2).sum(0), rtol=1e-12)
    assert np.allclose(nrm[:, 2], (m * (u - up) ** 2).sum(0), rtol=1e-10)
    assert np.all(nrm[:, 3] == 0)
    # a NaN planted in a host buffer and uploaded into the state trips the watchdog
    bad = u.copy()
    bad[100, 2] = np.nan
    s.bufs[s.cur].copy_(torch.from_numpy(bad))
    with pytest.raises(_lib.NonFiniteError):
        s.Norms()
    assert s.Norms(check_finite=False)[2, 3] == 1


@pytest.mark.parametrize("state", ["velocity", "previous"])
@pytest.mark.parametrize("norms_every", [0, 1])
def test_fp32_norms_against_fp64_sums(lib, cuda, state, norms_every):
    """FP32 state, separate pass and fused into the step: the norms against FP64 sums of
    the same FP32 values.  Each node's three-value term is formed in FP32 (three
    roundings; the mass-weighted term also a reciprocal of at most 1 ulp and a product),
    so the bound is 2e-7 (4e-7)."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    mesh = c0_mesh(64)
    s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 64, 32, chunk=12, state=state,
                                              norms_every=norms_every))
    pres = case.pressures(150)
    for n in range(150):
        s.pressure = float(pres[n])
        s.Solve(None, case.dt)
    nrm = s.Norms()
    assert s._norms_step == (s.step_count if norms_every else -1)
    u = s.bufs[s.cur].double().cpu().numpy()
    other = s.bufs[s.prev].double().cpu().numpy()
    du = other if state == "velocity" else u - other
    im = s.plan.invm(32).double().cpu().numpy()
    m = np.repeat(np.where(im != 0, 1.0 / np.where(im != 0, im, 1.0), 0.0), 3, axis=0)
    np.testing.assert_allclose(nrm[:, 0], (u ** 2).sum(0), rtol=2e-7, atol=0)
    np.testing.assert_allclose(nrm[:, 1], (du ** 2).sum(0), rtol=2e-7, atol=0)
    np.testing.assert_allclose(nrm[:, 2], (m * du ** 2).sum(0), rtol=4e-7, atol=0)
    assert np.all(nrm[:, 3] == 0)


def test_invalid_arguments_are_rejected(lib, cuda):
    mesh = c0_mesh(4)
    s = GPUSolidSolver(LocalComm(), mesh, Cfg(2e-6, 4, 64))
    with pytest.raises(_lib.CvfesError):
        call("cvfes_solid_step_f64", _lib.C.byref(s._desc), None, None, None, None, None, None,
             None, 0, 0.0, None, 2e-6, 0.0, None)
    with pytest.raises(_lib.CvfesError):
        call("cvfes_solid_step_f64", _lib.C.byref(s._desc), ptr(s.plan.coef64),
             ptr(s.plan.invm64), ptr(s.bufs[0]), ptr(s.bufs[1]), ptr(s.bufs[2]), None, None, 0,
             0.0, None, -1.0, 0.0, None)


VARIANTS = {32: [(0, 4, 8, 1), (1, 4, 4, 2), (2, 4, 4, 2), (3, 4, 2, 2), (4, 4, 4, 2), (4, 4, 4, 3),
                 (4, 2, 8, 3), (3, 2, 4, 3), (1, 1, 8, 4), (6, 4, 2, 1), (7, 2, 2, 2),
                 (7, 1, 2, 2), (8, 4, 2, 1), (8, 4, 2, 2), (8, 2, 2, 3), (5, 4, 2, 1)],
            64: [(0, 2, 8, 1), (1, 2, 4, 2), (3, 2, 2, 2), (4, 2, 4, 2), (4, 1, 6, 3), (3, 1, 4, 3),
                 (6, 2, 4, 2), (7, 1, 2, 2), (8, 2, 2, 2), (8, 1, 4, 3)]}


@pytest.mark.parametrize("precision,state", [(32, "previous"), (32, "velocity"),
                                             (64, "previous"), (64, "velocity")])
def test_step_kernel_variants_are_bitwise_identical(lib, cuda, precision, state):
    """Every step-kernel variant (L1 gather, TMA-staged, cp.async gather, fan rotation,
    pipelined persistent, persistent fan, TMA-tiled strips, two-ahead fan, burst gather)
    computes the same floating-point operations in the same order: their states after
    60 steps must be bitwise equal, in either state form."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    S = 128 if precision == 32 else 64
    mesh = c0_mesh(S)
    saved = _lib.get_step_tuning(precision)
    outs = []
    try:
        for staged, vec, npb, minb in VARIANTS[precision]:
            _lib.set_step_tuning(precision, vec, npb, staged, minb)
            s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, S, precision, chunk=12,
                                                      state=state))
            s.Advance(case.pressures(60))
            s.plan.check_status()
            outs.append(((staged, vec, npb, minb), s.local_displacement().clone()))
            s.release_graphs()
    finally:
        _lib.set_step_tuning(precision, **saved)
    ref_cfg, ref = outs[0]
    assert torch.isfinite(ref).all()
    for cfg, out in outs[1:]:
        assert torch.equal(out, ref), f"variant {cfg} differs from {ref_cfg}"


def test_large_sample_chunk_against_oracle(lib, cuda):
    """S = 128 (the warp-per-node kernels) on the 64x128 tube, 40 steps, vs the FP64 oracle."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    mesh = c0_mesh(128)
    coefK, gthick = mesh.element_coefficients()
    o = so.OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick,
                             mesh.density, mesh.v, mesh.damp, case.dt, backend="template")
    pres = case.pressures(40)
    o.run(pres)
    for precision, tol in ((64, FP64_TOL), (32, FP32_TOL)):
        s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 128, precision, chunk=12))
        s.Advance(pres)
        assert so.rel_l2(s.displacement(), o.u) < tol


def test_full_size_mesh_sample_chunk_against_oracle(lib, cuda):
    """The 256x1024 tube (262,144 nodes, 523,776 triangles, row-sum mass), a seeded
    64-sample chunk of its ensemble, 6 steps: the default step kernels (fan rotation
    with the L2 prefetch) against the oracle's element-template form, FP64 and FP32."""
    from cvfes_b200.cases import CASES, build_mesh
    case = CASES["tube256x1024"]
    mesh = build_mesh(case, n_samples=64)
    assert case.mass_lumping == "rowsum"  # the reference's lumping with 3x the density
    coefK, gthick = mesh.element_coefficients()
    o = so.OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick,
                             3.0 * mesh.density, mesh.v, mesh.damp, case.dt,
                             backend="template")
    pres = 1.33e5 * np.arange(6) / 6.0
    o.run(pres)
    assert np.linalg.norm(o.u) > 0
    for precision, tol in ((64, FP64_TOL), (32, FP32_TOL)):
        s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 64, precision, chunk=3))
        s.Advance(pres)
        s.plan.check_status()
        err = so.rel_l2(s.displacement(), o.u)
        s.release_graphs()
        assert err < tol, (precision, err)


@pytest.mark.parametrize("S", [200, 72])
def test_partial_sample_chunks_against_oracle(lib, cuda, S):
    """S/VEC above 32 and not a multiple of 32 (last sample chunk of a node block partly
    filled): every sample still steps, FP64 and FP32, single mesh and batch."""
    from cvfes_b200.batched import BatchedSolidSolver
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    mesh = c0_mesh(S)
    coefK, gthick = mesh.element_coefficients()
    o = so.OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick,
                             mesh.density, mesh.v, mesh.damp, case.dt, backend="template")
    pres = case.pressures(30)
    o.run(pres)
    for precision, tol in ((64, FP64_TOL), (32, FP32_TOL)):
        s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, S, precision, chunk=12))
        s.Advance(pres)
        assert so.rel_l2(s.displacement(), o.u) < tol
        b = BatchedSolidSolver([mesh], [case.dt], precision=precision, device=cuda,
                               graph_chunk=12)
        b.Advance(pres)
        assert so.rel_l2(b.displacement(0), o.u) < tol


def test_burst_step_variant_matches_fan(lib, cuda):
    """The burst-gather step kernel gives the fan kernel's bits (FP32 and FP64)."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    pres = case.pressures(36)
    for precision, S, tunes in ((32, 128, [(4, 2, 3, 2), (4, 2, 5, 1), (2, 2, 5, 2)]),
                                (64, 64, [(2, 2, 3, 2), (2, 2, 5, 1), (1, 2, 5, 2)])):
        mesh = c0_mesh(S)
        saved = _lib.get_step_tuning(precision)
        outs = []
        try:
            for vec, npb, staged, minb in tunes:
                _lib.set_step_tuning(precision, vec, npb, staged, minb)
                s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, S, precision, chunk=12))
                s.Advance(pres)
                outs.append(s.local_displacement().clone())
        finally:
            _lib.set_step_tuning(precision, **saved)
        for o in outs[1:]:
            assert torch.equal(o, outs[0])


def test_fan_prefetch_distance_leaves_results_unchanged(lib, cuda):
    """L2 prefetch of the nodes ahead (1, 80, the automatic distance and past the mesh
    end; node rows, coefficient rows or both) gives the fan kernel's bits with prefetch
    off (FP32 and FP64)."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    pres = case.pressures(36)
    for precision, S, vec in ((32, 128, 4), (64, 64, 2)):
        mesh = c0_mesh(S)
        saved, saved_pf = _lib.get_step_tuning(precision), _lib.get_step_prefetch(precision)
        outs = []
        try:
            _lib.set_step_tuning(precision, vec, 2, 3, 2)
            for dist, parts in ((0, 0), (1, 3), (80, 1), (80, 2), (-1, -1), (1 << 20, 3),
                                (80, 7), (0, 4)):
                _lib.set_step_prefetch(precision, dist, parts)
                s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, S, precision, chunk=12))
                s.Advance(pres)
                s.plan.check_status()
                outs.append(s.local_displacement().clone())
                s.release_graphs()
        finally:
            _lib.set_step_tuning(precision, **saved)
            _lib.set_step_prefetch(precision, **saved_pf)
        for o in outs[1:]:
            assert torch.equal(o, outs[0])


@pytest.mark.parametrize("name", ["tube8x6_geo1.npz", "tube8x6_geo3.npz"])
@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("path", ["solve", "advance"])
def test_geometric_update_reproduces_golden_history(lib, cuda, name, precision, path):
    """Stiffness and follower pressure on x + u (every step / every 3 steps) against the
    reference's OptimizedSolidAssembleUpdate run, step by step and as one Advance."""
    g = golden(name)
    mesh = golden_mesh(g)
    cfg = Cfg(float(g["dt"]), mesh.nSmp, precision)
    cfg.update_interval = int(g["update_interval"])
    solver = GPUSolidSolver(LocalComm(), mesh, cfg)
    tol = FP64_TOL if precision == 64 else FP32_TOL
    pres = g["pressures"]
    for k in range(len(g["hist"])):
        chunk = pres[5 * k:5 * k + 5]
        if path == "solve":
            for p in chunk:
                solver.pressure = float(p)
                solver.Solve(None, float(g["dt"]))
        else:
            solver.Advance(chunk)
        assert so.rel_l2(solver.displacement(), g["hist"][k]) < tol, k


def test_geometric_update_large_samples_against_oracle(lib, cuda):
    """Every-step geometric update on a 24x20 tube with 72 samples (S/VEC above 32 and not a
    multiple of it), 24 steps of a large load, against the NumPy restatement."""
    from cvfes_b200.cases import TubeCase, build_mesh, case_dt
    case = TubeCase("geo72", 24, 20, 2.0, n_samples=72, dt=None, seed_E=41, seed_h=42)
    mesh = build_mesh(case)
    dt = case_dt(case, mesh)
    coefK, gthick = mesh.element_coefficients()
    o = so.OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick,
                             mesh.density, mesh.v, mesh.damp, dt, backend="template",
                             update_interval=1)
    pres = case.pressures(24) * 5.0  # a large load: 8% away from the undeformed stiffness
    o.run(pres)
    for precision, tol in ((64, FP64_TOL), (32, FP32_TOL)):
        cfg = Cfg(dt, 72, precision, chunk=12)
        cfg.update_interval = 1
        s = GPUSolidSolver(LocalComm(), mesh, cfg)
        s.Advance(pres)
        assert so.rel_l2(s.displacement(), o.u) < tol


@pytest.mark.parametrize("name", ["tube8x6_element.npz", "tube6x5_nodal.npz",
                                  "tube8x6_geo1.npz", "tube8x6_geo3.npz"])
@pytest.mark.parametrize("precision", [64, 32])
def test_stress_recovery_matches_golden(lib, cuda, name, precision, tmp_path):
    """GPUSolidSolver.Stress after the golden run against the reference's
    OptimizedCalculateStress; Save writes the same stresses next to the displacement."""
    g = golden(name)
    mesh = golden_mesh(g)
    if "vE" in g:
        mesh = SolidMesh(g["nodes"], g["elements"], g["boundary"], g["coefK"].shape[1],
                         density=float(g["density"]), v=float(g["v"]), damp=float(g["damp"]),
                         vE=g["vE"], vthickness=g["vthickness"])
    cfg = Cfg(float(g["dt"]), mesh.nSmp, precision)
    cfg.update_interval = int(g["update_interval"])
    solver = GPUSolidSolver(LocalComm(), mesh, cfg)
    for p in g["pressures"]:
        solver.pressure = float(p)
        solver.Solve(None, float(g["dt"]))
    st = solver.Stress().double().cpu().numpy()
    tol = 1e-12 if precision == 64 else 1e-4
    assert rel(st, g["stress"]) < tol
    solver.Save(str(tmp_path / "out.npz"), 7)
    saved = np.load(str(tmp_path / "out7.npz"))
    assert np.array_equal(saved["stress"], st)
    assert saved["u"].shape == (mesh.nSmp, mesh.nNodes, 3)


@pytest.mark.parametrize("interval", [0, 1])
@pytest.mark.parametrize("constant", [False, True])
def test_traction_series_input_against_oracle(lib, cuda, tmp_path, constant, interval):
    """Fluid wall traction read from the .npy series of RefreshContext (ramped, then
    interpolated between files every dt_f; or one constant file), added as nodal force,
    on the undeformed stiffness (interval 0) and with the stiffness and follower pressure
    rebuilt every step (interval 1: assemble_K_P with calc_u_appTrac)."""
    import math
    g = golden("tube8x6_element.npz")
    mesh = golden_mesh(g)
    N, dt = mesh.nNodes, float(g["dt"])
    rng = np.random.default_rng(9)
    base = str(tmp_path / "trac")
    files = [2e3 * rng.standard_normal((N, 3)) for _ in range(6)]
    if constant:
        np.save(base + ".npy", files[0])
    else:
        for i, f in enumerate(files):
            np.save(f"{base}{i}.npy", f)
    cfg = Cfg(dt, mesh.nSmp, 64)
    cfg.exportBdyStressFilename = base
    cfg.useConstantStress = constant
    cfg.constant_T, cfg.dt_f, cfg.constant_pressure = 10 * dt, 4 * dt, 5e4
    cfg.update_interval = interval
    solver = GPUSolidSolver(LocalComm(), mesh, cfg)
    coefK, gthick = mesh.element_coefficients()
    o = so.OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick,
                             mesh.density, mesh.v, mesh.damp, dt, backend="numpy",
                             update_interval=interval)
    bdy = (3 * np.asarray(mesh.boundary)[:, None] + np.arange(3)).ravel()

    class Clock:
        t = 0.0
    clock = Clock()
    T, dtf = cfg.constant_T, cfg.dt_f
    strac, etrac, nt = files[0], files[1], 0
    for n in range(30):
        clock.t = t = n * dt
        solver.RefreshContext(clock)
        solver.Solve(t, dt)
        # expected load (physicsSolverSDampGPUs.py:287-322), boundary rows held clamped
        if constant:
            tr = files[0] if t > T else files[0] / 2 - files[0] / 2 * math.cos(math.pi / T * t)
        elif t > T:
            if int((t - T) / dtf) > nt:
                nt += 1
                strac, etrac = etrac, files[nt + 1]
            tr = strac + (t - T - nt * dtf) * (etrac - strac) / dtf
        else:
            tr = strac / 2 - strac / 2 * math.cos(math.pi / T * t)
        tr = np.array(tr, dtype=np.float64).reshape(-1)
        tr[bdy] = 0.0
        p = 5e4 if t > T else 5e4 * t / T  # the configuration's linear ramp
        o.step(p, tr)
    assert so.rel_l2(solver.displacement(), o.u) < FP64_TOL


@pytest.mark.parametrize("precision", [32, 64])
def test_tiled_step_with_outliers_matches_fan(lib, cuda, precision):
    """The TMA-tiled step with one node window and one element window per tile, so most
    neighbour and coefficient rows are read from global memory: the fan kernel's bits."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    S = 128 if precision == 32 else 64
    mesh = c0_mesh(S)
    pres = case.pressures(36)
    saved = _lib.get_step_tuning(precision)
    try:
        _lib.set_step_tuning(precision, 4 if precision == 32 else 2, 2, 3, 2)
        ref = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, S, precision, chunk=12))
        ref.Advance(pres)
        _lib.set_step_tuning(precision, 2 if precision == 32 else 1, 2, 7, 2)
        s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, S, precision, chunk=12))
        s.plan.build_tiles(P=16, H=18, W=1, EH=36, WE=1)
        assert s.plan.tile_stats["node_outliers"] > 0 and s.plan.tile_stats["element_outliers"] > 0
        s.refresh_desc()
        s.Advance(pres)
        s.plan.check_status()
    finally:
        _lib.set_step_tuning(precision, **saved)
    assert torch.equal(s.local_displacement(), ref.local_displacement())


@pytest.mark.parametrize("precision", [32, 64])
def test_geometric_step_tunings_are_bitwise_identical(lib, cuda, precision):
    """Samples per thread and block size of the geometric step change no bits."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    mesh = c0_mesh(64)
    pres = case.pressures(24) * 5.0
    saved = [C_int() for C_int in (_lib.C.c_int32, _lib.C.c_int32)]
    call("cvfes_get_geo_tuning", precision, _lib.C.byref(saved[0]), _lib.C.byref(saved[1]))
    outs = []
    try:
        for vec, block in ([(1, 64), (2, 128), (4, 256), (4, 128)] if precision == 32
                           else [(1, 64), (2, 128), (2, 256)]):
            call("cvfes_set_geo_tuning", precision, vec, block)
            cfg = Cfg(case.dt, 64, precision, chunk=12)
            cfg.update_interval = 1
            s = GPUSolidSolver(LocalComm(), mesh, cfg)
            s.Advance(pres)
            outs.append(s.local_displacement().clone())
    finally:
        call("cvfes_set_geo_tuning", precision, saved[0].value, saved[1].value)
    for o in outs[1:]:
        assert torch.equal(o, outs[0])


@pytest.mark.parametrize("precision,state,S", [(32, "velocity", 128), (32, "previous", 128),
                                               (64, "previous", 64), (64, "velocity", 64),
                                               (32, "velocity", 16)])
def test_fused_step_norms_match_separate_pass(lib, cuda, precision, state, S):
    """Solve with the norms fused into the step (persistent fan kernel; with 16 samples
    the shape has no fused kernel and the step falls back to the separate pass): the
    state bits of the plain step, and norms equal to the separate pass's to summation-
    order rounding (1e-13)."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    mesh = c0_mesh(S)
    pres = case.pressures(24)
    plain = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, S, precision, chunk=12, state=state))
    fused = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, S, precision, chunk=12, state=state,
                                                  norms_every=1))
    for n in range(24):
        for s in (plain, fused):
            s.pressure = float(pres[n])
            s.Solve(n * case.dt, case.dt)
        nf, npl = fused.Norms(), plain.Norms()
        assert fused._norms_step == fused.step_count
        assert np.all(nf[:, 3] == 0) and np.all(npl[:, 3] == 0)
        if n > 0:
            np.testing.assert_allclose(nf[:, :3], npl[:, :3], rtol=1e-13, atol=0)
    assert torch.equal(fused.local_displacement(), plain.local_displacement())


@pytest.mark.parametrize("precision,state", [(32, "velocity"), (64, "previous")])
def test_norms_memory_modes_agree_bitwise(lib, cuda, precision, state):
    """The fused norms kept in tensor memory (default) and in shared memory
    (cvfes_set_norms_memory(1)): the same state and bitwise the same norms."""
    from cvfes_b200.cases import CASES
    case = CASES["tube64x128"]
    mesh = c0_mesh(128)
    pres = case.pressures(12)
    runs = []
    try:
        for mode in (0, 1):
            call("cvfes_set_norms_memory", mode)
            s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 128, precision, chunk=12,
                                                      state=state, norms_every=1))
            out = []
            for n in range(12):
                s.pressure = float(pres[n])
                s.Solve(None, case.dt)
                out.append(s.Norms())
            assert s._norms_step == s.step_count
            runs.append((s.local_displacement().clone(), np.stack(out)))
    finally:
        call("cvfes_set_norms_memory", 0)
    assert torch.equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


@pytest.mark.parametrize("precision", [64, 32])
def test_opencl_semantics_against_restatement(lib, cuda, precision):
    """[gpu] semantics = opencl (the OpenCL class's numerics: mean(E h) over the element's
    nodes, its lumping of nodal thickness, damping force per dof with LHS = LM, no damping
    in the start-up acceleration, stiffness and follower pressure on x + u every step)
    against the NumPy restatement of its kernels, with nodal material that varies node
    by node and damping 100: FP64 <= 1e-12, FP32 <= 1e-5 at every 10th step."""
    from cvfes_b200.mesh import TubeGeometry, tube_mesh
    from oracle.opencl_oracle import OpenCLSolidOracle
    nodes, elems, inl, outl = tube_mesh(TubeGeometry(16, 12, 3.0, 0.3))
    bdy = np.concatenate([inl, outl])
    N, S = len(nodes), 4
    rng = np.random.default_rng(11)
    vE = 7e6 * np.exp(0.2 * rng.standard_normal((N, S)))
    vh = 0.04 * np.exp(0.1 * rng.standard_normal((N, S)))
    dt, damp = 2e-6, 100.0
    mesh = SolidMesh(nodes, elems, bdy, S, density=1.0, v=0.49, damp=damp, vE=vE, vthickness=vh)
    ocl = OpenCLSolidOracle(nodes, elems, bdy, vE, vh, 1.0, 0.49, damp, dt)
    s = GPUSolidSolver(LocalComm(), mesh, Cfg(dt, S, precision, chunk=12, semantics="opencl"))
    assert s.update_interval == 1 and s._desc.damping_form == 1
    pres = 1.33e5 * np.minimum(np.arange(40) / 10.0, 1.0)
    tol = FP64_TOL if precision == 64 else FP32_TOL
    worst = 0.0
    for n, p in enumerate(pres):
        s.pressure = float(p)
        s.Solve(n * dt, dt)
        ref = ocl.step(p)
        if (n + 1) % 10 == 0:
            worst = max(worst, so.rel_l2(s.displacement(), ref))
    print(f"opencl semantics FP{precision}: max rel-L2 {worst:.3e}")
    assert np.abs(ref).max() > 0 and worst < tol
