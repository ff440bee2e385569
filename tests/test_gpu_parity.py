"""GPU parity suite: the CUDA operators and solver against the FP64 oracle.

Tolerances (relative to max |reference|):
  FP64 operators          1e-12   (different but exact-in-FP64 formula order)
  FP32 operators          2e-5    (FP32 arithmetic, FP64 input/output)
  FP64 GMRES vs LU        1e-8 on moments at tol 1e-10, 1e-9 on C_ext
  FP32+refine vs LU       1e-6 on C_ext (the north-star gate)
"""
import math
import threading

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from lumina_b200.geometry import Sphere, discretise_primitive
from lumina_b200.lattice import LatticeSpec, SubstrateRuntime
from oracle import oracle as orc
from tests.conftest import rand_vec, rel_err

pytestmark = pytest.mark.gpu


def _workload(kind, rng):
    if kind == "sphere_fcd":
        pos = discretise_primitive(Sphere((0, 0, 0), 6.0), 2.0)
        w = configs.au_workload("s", pos, 2.0, 520.0)
        return w.positions, w.alpha, w.k, True, 2.0
    if kind == "sphere_point":
        pos = discretise_primitive(Sphere((0, 0, 0), 6.0), 2.0)
        w = configs.au_workload("s", pos, 2.0, 600.0)
        return w.positions, w.alpha, w.k, False, 2.0
    if kind == "jitter_aniso":
        base = discretise_primitive(Sphere((1.0, -2.0, 0.5), 5.0), 1.5)
        pos = base + rng.uniform(-0.2, 0.2, base.shape)
        n = pos.shape[0]
        alpha = (np.eye(3) * (3.0 + 1.5j))[None] + 0.3 * (rng.standard_normal((n, 3, 3))
                                                          + 1j * rng.standard_normal((n, 3, 3)))
        return pos, alpha, 2 * math.pi / 480.0, True, 1.5
    raise KeyError(kind)


KINDS = ["sphere_fcd", "sphere_point", "jitter_aniso"]


@pytest.mark.parametrize("kind", KINDS)
def test_onthefly_fp64_matches_oracle(backend, rng, kind):
    pos, alpha, k, fcd, cell = _workload(kind, rng)
    inv = lb.invert_polarisability(alpha)
    x = rand_vec(rng, 3 * pos.shape[0])
    y_ref = orc.matvec_onthefly(pos, alpha, x, k, fcd, cell)
    with backend.create_onthefly_session(pos, inv, k, fcd, cell) as s:
        y = s.matvec(x, "fp64")
    assert rel_err(y, y_ref) < 1e-12


@pytest.mark.parametrize("kind", KINDS)
def test_onthefly_fp32_matches_oracle(backend, rng, kind):
    pos, alpha, k, fcd, cell = _workload(kind, rng)
    inv = lb.invert_polarisability(alpha)
    x = rand_vec(rng, 3 * pos.shape[0])
    y_ref = orc.matvec_onthefly(pos, alpha, x, k, fcd, cell)
    with backend.create_onthefly_session(pos, inv, k, fcd, cell) as s:
        y = s.matvec(x, "fp32")
    assert rel_err(y, y_ref) < 2e-5


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
def test_onthefly_substrate_matches_oracle(backend, rng, precision, tol):
    pos = discretise_primitive(Sphere((0, 0, 12.0), 5.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 560.0)
    sub = SubstrateRuntime(0.0, complex(0.45 / 2.45))
    inv = lb.invert_polarisability(w.alpha)
    x = rand_vec(rng, 3 * w.n)
    y_ref = orc.matvec_onthefly(w.positions, w.alpha, x, w.k, True, 2.0, substrate=sub)
    with backend.create_onthefly_session(w.positions, inv, w.k, True, 2.0, substrate=sub) as s:
        y = s.matvec(x, precision)
    assert rel_err(y, y_ref) < tol


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
def test_device_assembly_matches_oracle(backend, rng, kind, precision, tol):
    pos, alpha, k, fcd, cell = _workload(kind, rng)
    inv = lb.invert_polarisability(alpha)
    A = orc.assemble(pos, alpha, k, fcd, cell)
    x = rand_vec(rng, 3 * pos.shape[0])
    with backend.assemble_and_create_session(pos, k, inv, use_fcd=fcd, cell_size=cell,
                                             precision=precision) as s:
        y = s.matvec(x, precision)
    assert rel_err(y, A @ x) < tol


@pytest.mark.parametrize("lat", ["planar", "planar_sub", "chain"])
def test_ewald_matvec_matches_oracle(backend, rng, lat):
    pos = discretise_primitive(Sphere((0, 0, 10.0), 3.0), 2.0)
    n = pos.shape[0]
    k = 2 * math.pi / 600.0
    alpha = np.broadcast_to(np.eye(3) * (40.0 + 12.0j), (n, 3, 3)).copy()
    sub = None
    if lat == "chain":
        L = LatticeSpec.chain((80.0, 0.0, 0.0))
    else:
        L = LatticeSpec.planar((100.0, 0.0, 0.0), (0.0, 100.0, 0.0))
        if lat == "planar_sub":
            sub = SubstrateRuntime(0.0, complex(0.2, 0.01))
    kb = (k * math.sin(math.radians(10.0)), 0.0, 0.0)
    inv = lb.invert_polarisability(alpha)
    x = rand_vec(rng, 3 * n)
    y_ref = orc.matvec_onthefly(pos, alpha, x, k, True, 2.0, lattice=L, k_bloch=kb, substrate=sub)
    with backend.create_onthefly_session(pos, inv, k, True, 2.0, lattice=L, k_bloch=kb,
                                         substrate=sub) as s:
        y = s.matvec(x, "fp64")
    assert rel_err(y, y_ref) < 1e-10
    A = orc.assemble(pos, alpha, k, True, 2.0, lattice=L, k_bloch=kb, substrate=sub)
    with backend.assemble_and_create_session(pos, k, inv, use_fcd=True, cell_size=2.0, lattice=L,
                                             k_bloch=kb, substrate=sub, precision="fp64") as s:
        y2 = s.matvec(x, "fp64")
    assert rel_err(y2, A @ x) < 1e-10


@pytest.fixture(scope="module")
def c1():
    w = configs.sphere_au_925()
    A = orc.assemble(w.positions, w.alpha, w.k, True, w.cell_size)
    b = orc.incident_field(w.positions, w.k)
    x_lu = orc.lu_solve(A, b)
    cs_lu = orc.cross_sections(w.positions, w.alpha, x_lu, w.k)
    return w, A, b, x_lu, cs_lu


def test_c1_fp64_gmres_matches_lu(backend, c1):
    w, A, b, x_lu, cs_lu = c1
    inv = lb.invert_polarisability(w.alpha)
    with backend.create_onthefly_session(w.positions, inv, w.k, True, w.cell_size) as s:
        x, info = s.solve(b, 1e-10, 5000, 30, "fp64")
    assert info["converged"] == 1
    assert rel_err(x, x_lu) < 1e-8
    cs = lb.cross_sections(w.positions, inv, x, w.k, lb.IncidentField())
    assert abs(cs[0] - cs_lu[0]) / abs(cs_lu[0]) < 1e-9
    assert abs(cs[1] - cs_lu[1]) / abs(cs_lu[1]) < 1e-9


def test_c1_fp32_refine_meets_gate(backend, c1):
    w, A, b, x_lu, cs_lu = c1
    inv = lb.invert_polarisability(w.alpha)
    with backend.create_onthefly_session(w.positions, inv, w.k, True, w.cell_size) as s:
        x, info = s.solve(b, 1e-8, 5000, 30, "fp32_refine")
    assert info["converged"] == 1
    assert info["matvecs_fp32"] > info["matvecs_fp64"]
    cs = lb.cross_sections(w.positions, inv, x, w.k, lb.IncidentField())
    assert abs(cs[0] - cs_lu[0]) / abs(cs_lu[0]) < 1e-6


def test_gmres_iterations_match_oracle(backend):
    pos = discretise_primitive(Sphere((0, 0, 0), 6.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 520.0)
    b = orc.incident_field(w.positions, w.k)
    ref = orc.gmres_onthefly(w.positions, w.alpha, b, w.k, True, 2.0, tol=1e-10, max_iter=2000)
    inv = lb.invert_polarisability(w.alpha)
    with backend.create_onthefly_session(w.positions, inv, w.k, True, 2.0) as s:
        x, info = s.solve(b, 1e-10, 2000, 30, "fp64")
    assert ref.converged and info["converged"]
    assert abs(info["iterations"] - ref.iterations) <= 1
    assert info["matvecs_reference"] in (ref.matvecs, ref.matvecs + 1, ref.matvecs - 1)
    assert rel_err(x, ref.x) < 1e-8


def test_cdasolver_dispatch_paths(backend):
    w = configs.sphere_au_925()
    ds = lb.DipoleSet(w.positions, w.alpha)
    params = lb.SimulationParams(solver_tolerance=1e-10, max_iterations=5000)
    direct = lb.CdaSolver.with_fcd(1000, True, 2.0, backend=backend)
    cached = lb.CdaSolver.with_fcd(0, True, 2.0, backend=backend)
    otf = lb.CdaSolver.with_fcd(0, True, 2.0, backend=backend, matrix_memory_budget=0)
    res = [s.compute_cross_sections(ds, 520.0, params) for s in (direct, cached, otf)]
    for r in res[1:]:
        assert abs(r.extinction - res[0].extinction) / res[0].extinction < 1e-8


def test_cdasolver_fft_branch(backend):
    """The solver's FFT branch (cda/mod.rs:286-298, widened to FCD and the
    substrate forms) agrees with the matrix-free branch at the C_ext gate.
    Tolerance 1e-8 as in the bench: FP32+refine through the FP32 FFT product
    stalls near 1e-9 on this system."""
    from lumina_b200.lattice import SommerfeldRuntime
    w = configs.cuboid_au((20.0, 20.0, 10.0), 1.0, 520.0)
    pos = w.positions.copy()
    pos[:, 2] += 8.0
    ds = lb.DipoleSet(pos, w.alpha)
    for sub in (None, SommerfeldRuntime(0.0, 520.0, 2.25, 1.0)):
        params = lb.SimulationParams(solver_tolerance=1e-8, max_iterations=5000,
                                     substrate_runtime=sub)
        fft = lb.CdaSolver.with_fcd(0, True, 1.0, backend=backend, precision="fp32_refine")
        otf = lb.CdaSolver.with_fcd(0, True, 1.0, backend=backend, precision="fp32_refine",
                                    matrix_memory_budget=0, use_fft=False)
        assert fft._fft_worthwhile(pos) and not otf._fft_worthwhile(pos)
        a = fft.compute_cross_sections(ds, 520.0, params).extinction
        b = otf.compute_cross_sections(ds, 520.0, params).extinction
        assert abs(a - b) / abs(b) < 1e-6


# --- edge cases -----------------------------------------------------------

def test_single_dipole_rayleigh(backend):
    # cda_diagnostic.rs:121-166: one dipole, C_ext = k Im(alpha) within 1 %
    k = 2 * math.pi / 600.0
    eps = complex(-10.0, 1.5)
    vol = 4.0 / 3.0 * math.pi * 10.0 ** 3
    a = lb.radiative_correction(lb.clausius_mossotti(vol, eps, 1.0), k)
    ds = lb.DipoleSet.isotropic([[0.0, 0.0, 0.0]], a)
    cs = lb.CdaSolver(backend=backend).compute_cross_sections(ds, 600.0, lb.SimulationParams())
    assert abs(cs.extinction - k * a.imag) / (k * a.imag) < 0.01


def test_two_dipoles_and_n1_sessions(backend, rng):
    pos = np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0]])
    alpha = np.broadcast_to(np.eye(3) * (50 + 5j), (2, 3, 3)).copy()
    inv = lb.invert_polarisability(alpha)
    k = 2 * math.pi / 500.0
    x = rand_vec(rng, 6)
    for fcd in (False, True):
        y_ref = orc.matvec_onthefly(pos, alpha, x, k, fcd, 3.0)
        with backend.create_onthefly_session(pos, inv, k, fcd, 3.0) as s:
            assert rel_err(s.matvec(x, "fp64"), y_ref) < 1e-13
    one = np.zeros((1, 3))
    with backend.create_onthefly_session(one, inv[:1], k, True, 3.0) as s:
        y = s.matvec(x[:3], "fp64")
    assert rel_err(y, inv[0] @ x[:3]) < 1e-15


def test_invalid_inputs_raise(backend):
    k = 0.01
    inv = np.broadcast_to(np.eye(3, dtype=complex), (2, 3, 3)).copy()
    with pytest.raises(lb.InvalidGeometry):
        backend.create_onthefly_session(np.zeros((2, 3)), inv, k, True, 1.0)  # coincident
    with pytest.raises(lb.InvalidGeometry):
        backend.create_onthefly_session(np.zeros((0, 3)), inv[:0], k, True, 1.0)
    with pytest.raises(lb.InvalidGeometry):
        backend.create_onthefly_session(np.array([[0, 0, 0], [1, 0, 0.0]]), inv, -1.0, True, 1.0)
    with pytest.raises(lb.InvalidGeometry):
        lb.invert_polarisability(np.zeros((1, 3, 3)))


def test_not_converged_and_zero_rhs(backend):
    w = configs.sphere_au_925()
    inv = lb.invert_polarisability(w.alpha)
    b = orc.incident_field(w.positions, w.k)
    with backend.create_onthefly_session(w.positions, inv, w.k, True, 2.0) as s:
        with pytest.raises(lb.ConvergenceFailure) as ei:
            s.solve(b, 1e-14, 3, 30, "fp64")
        assert ei.value.info["iterations"] == 3
        x, info = s.solve(np.zeros_like(b), 1e-8, 10, 30, "fp64")
        assert np.all(x == 0) and info["converged"] == 1


def test_set_wavelength_matches_fresh_session(backend, rng):
    pos = discretise_primitive(Sphere((0, 0, 0), 6.0), 2.0)
    w1 = configs.au_workload("a", pos, 2.0, 520.0)
    w2 = configs.au_workload("b", pos, 2.0, 640.0)
    x = rand_vec(rng, 3 * w1.n)
    inv1, inv2 = lb.invert_polarisability(w1.alpha), lb.invert_polarisability(w2.alpha)
    with backend.create_onthefly_session(pos, inv1, w1.k, True, 2.0) as s:
        s.set_wavelength(w2.k, inv2)
        y = s.matvec(x, "fp64")
    y_ref = orc.matvec_onthefly(pos, w2.alpha, x, w2.k, True, 2.0)
    assert rel_err(y, y_ref) < 1e-12


# --- ports of the reference's wgpu backend tests (gpu.rs:690-1073) ---------

def test_ref_gpu_matvec_identity_and_complex(backend):
    dim = 6
    v = np.array([complex(i + 1.0, 0.5 * i) for i in range(dim)])
    assert np.max(np.abs(backend.matvec(np.eye(dim), v, "fp32") - v)) < 1e-4
    A = np.array([[2 + 1j, -1 + .5j, 0], [.3 - .2j, 3, -.5 + .1j], [0, .7 - .3j, 4 - 1j]])
    x = np.array([1, 1j, -1 + .5j])
    assert np.max(np.abs(backend.matvec(A, x, "fp32") - A @ x)) < 1e-4


def test_ref_gpu_matvec_300(backend):
    dim = 300
    A = np.diag(np.full(dim, 4 + .5j)) + np.diag(np.full(dim - 1, -1 + .1j), 1) \
        + np.diag(np.full(dim - 1, -1 - .1j), -1)
    v = np.array([complex(math.sin(i), math.cos(i)) for i in range(dim)])
    e = A @ v
    assert np.max(np.abs(backend.matvec(A, v, "fp32") - e)) / np.linalg.norm(e) < 1e-4


def test_ref_session_repeated(backend):
    dim = 9
    A = np.array([[3 + .5j if i == j else complex(.1 * np.sign(i - j), .05) for j in range(dim)]
                  for i in range(dim)])
    with backend.create_session(dim, "fp32") as s:
        s.upload_matrix(A)
        for trial in range(5):
            v = np.array([complex((i + trial) * .4, (trial - i) * .1) for i in range(dim)])
            assert np.max(np.abs(s.matvec(v, "fp32") - A @ v)) < 1e-4


def test_ref_gpu_assembly_collinear(backend):
    n = 20
    pos = np.array([[i * 3.0, 0.0, 0.0] for i in range(n)])
    k = 2 * math.pi / 600.0
    alpha = np.broadcast_to(np.eye(3) * (1000 + 200j), (n, 3, 3)).copy()
    inv = lb.invert_polarisability(alpha)
    A = orc.assemble(pos, alpha, k, False, 3.0)
    with backend.assemble_and_create_session(pos, k, inv, precision="fp32") as s:
        err = 0.0
        for col in range(3 * n):
            e = np.zeros(3 * n, complex)
            e[col] = 1.0
            err = max(err, np.max(np.abs(s.matvec(e, "fp32") - A[:, col])))
    assert err < 5e-5
    # the reference's own FP32 shader arithmetic lands in the same band
    Aw = orc.wgsl_assemble_f32(pos, inv, k)
    assert np.max(np.abs(Aw - A)) < 5e-5


def test_ref_gpu_assembly_diagonal_and_n1(backend):
    pos = np.array([[0.0, 0, 0], [1000.0, 0, 0], [2000.0, 0, 0]])
    k = 2 * math.pi / 600.0
    inv = lb.invert_polarisability(np.broadcast_to(np.eye(3) * (500 + 100j), (3, 3, 3)).copy())
    with backend.assemble_and_create_session(pos, k, inv, precision="fp32") as s:
        for i in range(3):
            for a in range(3):
                e = np.zeros(9, complex)
                e[3 * i + a] = 1
                y = s.matvec(e, "fp32")
                for b in range(3):
                    assert abs(y[3 * i + b] - inv[i][b, a]) < 1e-3
    inv1 = np.eye(3, dtype=complex)[None] * (0.001 + 0.0001j)
    with backend.assemble_and_create_session(np.zeros((1, 3)), 0.01, inv1, precision="fp32") as s:
        y = s.matvec(np.array([1, 0, 0], complex), "fp32")
    assert abs(y[0] - (0.001 + 0.0001j)) < 1e-4


def test_ref_parallel_sessions(backend):
    dim = 12
    A = np.array([[5 + 1j if i == j else complex(-.1, .05 * (i - j)) for j in range(dim)]
                  for i in range(dim)])
    errs = [None] * 4

    def work(tid):
        with backend.create_session(dim, "fp32") as s:
            s.upload_matrix(A)
            v = np.array([complex(i, tid * .1) for i in range(dim)])
            errs[tid] = np.max(np.abs(s.matvec(v, "fp32") - A @ v))

    ts = [threading.Thread(target=work, args=(t,)) for t in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert all(e is not None and e < 1e-4 for e in errs)


# --- the reference's benchmark-as-test (tests/gpu_benchmark.rs) ---------------
def _bench_matrix(dim):
    """gpu_benchmark.rs:16-30: a deterministic complex matrix made diagonally
    dominant, and the vector of :33-41."""
    i = np.arange(dim)[:, None]
    j = np.arange(dim)[None, :]
    A = (((i * 137 + j * 251 + 31) % 997) / 997.0 - 0.5) + \
        1j * (((i * 173 + j * 311 + 59) % 991) / 991.0 - 0.5)
    A[np.arange(dim), np.arange(dim)] += dim
    q = np.arange(dim)
    v = (((q * 193 + 41) % 983) / 983.0 - 0.5) + 1j * (((q * 229 + 67) % 977) / 977.0 - 0.5)
    return A, v


@pytest.mark.parametrize("dim", [300, 1000, 3000])
def test_ref_benchmark_matvec_and_gmres(backend, dim):
    """gpu_benchmark.rs:86-200: the FP32 session matvec agrees with the FP64
    product to < 1e-4, and GMRES through it (tol 1e-6) with the FP64 GMRES at
    1e-10 to < 1e-3 -- here the FP32+refine solve at 1e-10 is held to 1e-8."""
    A, v = _bench_matrix(dim)
    y_ref = A @ v
    x_ref = np.linalg.solve(A, v)
    with backend.create_session(dim, "fp32") as s:
        s.upload_matrix(A)
        assert rel_err(s.matvec(v, "fp32"), y_ref) < 1e-4
        x, info = s.solve(v, 1e-6, 1000, 30, "fp64")
        assert rel_err(x, x_ref) < 1e-3
    with backend.create_session(dim, "fp64") as s:
        s.upload_matrix(A)
        x, info = s.solve(v, 1e-10, 1000, 30, "fp32_refine")
        assert info["converged"] and rel_err(x, x_ref) < 1e-8


@pytest.mark.parametrize("branch", ["direct", "cached", "onthefly", "fft", "onthefly_sommerfeld"])
def test_cdasolver_session_reuse_matches_fresh(backend, branch):
    """A wavelength sweep through one solver re-targets its kept session; the
    results equal those of a fresh session per call, and a new geometry gets
    a new session."""
    from lumina_b200.lattice import SommerfeldRuntime, SubstrateSpec, SubstrateRuntime
    if branch == "fft":
        w = configs.cuboid_au((20.0, 20.0, 10.0), 1.0, 520.0)
        kw = dict(iterative_threshold=0, cell_size=1.0)
    else:
        w = configs.sphere_au_925()
        kw = dict(iterative_threshold=1000 if branch == "direct" else 0, cell_size=2.0,
                  matrix_memory_budget=0 if branch.startswith("onthefly") else 2 << 30)
    pos = w.positions.copy()
    pos[:, 2] += 20.0
    reuse = lb.CdaSolver(backend=backend, **kw)
    fresh = lb.CdaSolver(backend=backend, reuse_session=False, **kw)
    spec = SubstrateSpec(0.0, "glass", True, branch.endswith("sommerfeld"))
    kept = []
    for wl in (520.0, 600.0, 700.0):
        ds = lb.DipoleSet(pos, configs.au_workload("s", pos, kw["cell_size"], wl).alpha)
        sub = SubstrateRuntime.from_spec(spec, 2.25, 1.0, wl) if "sommerfeld" in branch else None
        params = lb.SimulationParams(solver_tolerance=1e-8, max_iterations=20000,
                                     substrate_runtime=sub)
        a = reuse.compute_cross_sections(ds, wl, params)
        b = fresh.compute_cross_sections(ds, wl, params)
        assert abs(a.extinction - b.extinction) <= 1e-9 * abs(b.extinction)
        assert abs(a.absorption - b.absorption) <= 1e-9 * abs(b.absorption)
        kept.append(reuse._kept[1])
    assert kept[0] is kept[1] is kept[2]
    moved = lb.DipoleSet(pos + 2.0 * kw["cell_size"], ds.polarisability)
    reuse.compute_cross_sections(moved, 700.0, params)
    assert reuse._kept[1] is not kept[0]
    reuse.close()
    assert reuse._kept is None


def test_cdasolver_shared_between_threads(backend):
    """Two threads on one solver: the kept session is never used by both at
    once (a busy session makes the other call build its own)."""
    w = configs.sphere_au_925()
    solver = lb.CdaSolver(backend=backend, iterative_threshold=0, cell_size=2.0,
                          matrix_memory_budget=0)
    params = lb.SimulationParams(solver_tolerance=1e-10, max_iterations=20000)
    wls = [520.0, 560.0, 600.0, 640.0]
    ref = {wl: lb.CdaSolver(backend=backend, iterative_threshold=0, cell_size=2.0,
                            matrix_memory_budget=0, reuse_session=False).compute_cross_sections(
        lb.DipoleSet(w.positions, configs.au_workload("s", w.positions, 2.0, wl).alpha), wl,
        params).extinction for wl in wls}
    out, errs = {}, []

    def run(ws):
        try:
            for wl in ws:
                ds = lb.DipoleSet(w.positions, configs.au_workload("s", w.positions, 2.0, wl).alpha)
                out[wl] = solver.compute_cross_sections(ds, wl, params).extinction
        except Exception as e:  # noqa: BLE001
            errs.append(e)

    th = [threading.Thread(target=run, args=(wls[i::2],)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs
    for wl in wls:
        assert abs(out[wl] - ref[wl]) <= 1e-8 * abs(ref[wl])
    solver.close()
