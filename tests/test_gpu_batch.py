"""Batched systems (lum_batch_*) on the GPU against the oracle.

Seeded Drude ellipsoid clusters with the reference's anisotropic ellipsoid
polarisability tensors (scene.rs:507-517, types.rs:286-317), each solved for
x and y polarisation as separate systems of one batch.  Every system's
segment of the batched matvec must equal the oracle's single-system
on-the-fly matvec (assembly.rs:209-318), and every system's batched GMRES
must reproduce the oracle's GMRES (iterative.rs:33-206).

Tolerances: matvec FP64 1e-12, FP32 2e-5 (max-norm relative); FP64 solve
x 1e-8 and C_ext 1e-9 against the oracle's GMRES at the same tolerance,
iteration counts within one step (summation order differs); FP32+refine
C_ext 1e-6.
"""
import os

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from oracle import oracle as orc
from tests.conftest import rand_vec, rel_err

pytestmark = pytest.mark.gpu


def small_batch(count=4, seed=3, n_range=(200, 700)):
    return configs.batch_clusters(count, seed, n_range=n_range)


def batch_inputs(w):
    systems = w.systems()
    specs = [(p, lb.invert_polarisability(a), k, cell) for p, a, k, cell, _ in systems]
    return systems, specs


def test_batch_matvec_matches_oracle(backend, rng):
    w = small_batch()
    systems, specs = batch_inputs(w)
    for use_fcd in (True, False):
        with backend.create_batch(specs, use_fcd=use_fcd) as B:
            x = rand_vec(rng, B.dim)
            y64 = B.split(B.matvec(x, "fp64"))
            y32 = B.split(B.matvec(x, "fp32"))
            xs = B.split(x)
            for s, (p, a, k, cell, _) in enumerate(systems):
                y_ref = orc.matvec_onthefly(p, a, xs[s], k, use_fcd, cell)
                assert rel_err(y64[s], y_ref) < 1e-12, (use_fcd, s)
                assert rel_err(y32[s], y_ref) < 2e-5, (use_fcd, s)
            info = B.info()
            assert info["systems"] == len(systems)
            assert info["items32"] >= len(systems)


def test_batch_uneven_k_and_cell(backend, rng):
    """Systems of one batch may differ in wave number and FCD cell."""
    w = small_batch(count=3, seed=5)
    systems, _ = batch_inputs(w)
    ks = [0.009, 0.0105, 0.0125, 0.011, 0.0098, 0.0131]
    cells = [1.5, 2.0, 1.5, 3.0, 1.5, 2.5]
    specs, refs = [], []
    for s, (p, a, _, _, _) in enumerate(systems):
        specs.append((p, lb.invert_polarisability(a), ks[s], cells[s]))
        refs.append((p, a, ks[s], cells[s]))
    with backend.create_batch(specs) as B:
        x = rand_vec(rng, B.dim)
        ys = B.split(B.matvec(x, "fp64"))
        xs = B.split(x)
    for s, (p, a, k, cell) in enumerate(refs):
        assert rel_err(ys[s], orc.matvec_onthefly(p, a, xs[s], k, True, cell)) < 1e-12


def test_batch_solve_matches_oracle_gmres(backend):
    w = small_batch()
    systems, specs = batch_inputs(w)
    rhs = [lb.incident_field(p, k, inc) for p, _, k, _, inc in systems]
    b = np.concatenate(rhs)
    tol = 1e-10
    with backend.create_batch(specs) as B:
        x64, info64 = B.solve(b, tol, 3000, 30, "fp64")
        x32, info32 = B.solve(b, tol, 3000, 30, "fp32_refine")
        x64s, x32s = B.split(x64), B.split(x32)
    for s, (p, a, k, cell, inc) in enumerate(systems):
        ref = orc.gmres_onthefly(p, a, rhs[s], k, True, cell, tol=tol, max_iter=3000)
        assert ref.converged
        assert info64[s]["converged"] == 1 and info32[s]["converged"] == 1
        assert abs(info64[s]["iterations"] - ref.iterations) <= 1, (s, info64[s], ref.iterations)
        assert rel_err(x64s[s], ref.x) < 1e-8, s
        inv = specs[s][1]
        cs_ref = lb.cross_sections(p, inv, ref.x, k, inc)
        cs64 = lb.cross_sections(p, inv, x64s[s], k, inc)
        cs32 = lb.cross_sections(p, inv, x32s[s], k, inc)
        assert abs(cs64[0] - cs_ref[0]) / abs(cs_ref[0]) < 1e-9, s
        assert abs(cs32[0] - cs_ref[0]) / abs(cs_ref[0]) < 1e-6, s
        assert abs(cs32[1] - cs_ref[1]) / abs(cs_ref[1]) < 1e-6, s


def test_batch_solve_equals_single_sessions(backend):
    """The batch gives each system what its own session gives."""
    w = small_batch(count=2, seed=11)
    systems, specs = batch_inputs(w)
    rhs = [lb.incident_field(p, k, inc) for p, _, k, _, inc in systems]
    with backend.create_batch(specs) as B:
        xb, infob = B.solve(np.concatenate(rhs), 1e-9, 2000, 30, "fp32_refine")
        xbs = B.split(xb)
    for s, (p, inv, k, cell) in enumerate(specs):
        with backend.create_onthefly_session(p, inv, k, True, cell) as S:
            xs, info = S.solve(rhs[s], 1e-9, 2000, 30, "fp32_refine")
        assert rel_err(xbs[s], xs) < 1e-6
        assert abs(infob[s]["iterations"] - info["iterations"]) <= 2


def test_batch_graph_replay_is_bitwise_equal(backend):
    w = small_batch(count=2, seed=7)
    systems, specs = batch_inputs(w)
    b = np.concatenate([lb.incident_field(p, k, inc) for p, _, k, _, inc in systems])
    out = []
    for flag in ("0", "1"):
        os.environ["LUMINA_BATCH_GRAPH"] = flag
        try:
            with backend.create_batch(specs) as B:
                x, _ = B.solve(b, 1e-8, 2000, 30, "fp32_refine")
                x2, _ = B.solve(b, 1e-8, 2000, 30, "fp32_refine")  # replays the captured cycle
        finally:
            os.environ.pop("LUMINA_BATCH_GRAPH", None)
        assert np.array_equal(x, x2)
        out.append(x)
    assert np.array_equal(out[0], out[1])


def test_batch_edge_cases(backend, rng):
    w = small_batch(count=2, seed=9)
    systems, specs = batch_inputs(w)
    # a one-dipole system (GMRES restart min(30, 3) = 3) and a zero right-hand side
    p1 = np.array([[0.3, -0.2, 0.1]])
    a1 = np.broadcast_to(np.diag([800 + 60j, 900 + 40j, 700 + 90j]), (1, 3, 3)).copy()
    specs = specs + [(p1, lb.invert_polarisability(a1), 0.0105, 1.5)]
    rhs = [lb.incident_field(p, k, inc) for p, _, k, _, inc in systems]
    rhs[1] = np.zeros_like(rhs[1])
    rhs.append(np.array([1.0 + 0.5j, -0.25j, 0.75]))
    with backend.create_batch(specs) as B:
        x, info = B.solve(np.concatenate(rhs), 1e-10, 5000, 30, "fp64")
        xs = B.split(x)
        assert info[1]["converged"] == 1 and info[1]["iterations"] == 0
        assert np.all(xs[1] == 0)
        A1 = orc.assemble(p1, a1, 0.0105, True, 1.5)
        assert rel_err(xs[-1], np.linalg.solve(A1, rhs[-1])) < 1e-12
        # too few iterations for the clusters: NOT_CONVERGED with per-system info
        with pytest.raises(lb.ConvergenceFailure):
            B.solve(np.concatenate(rhs), 1e-12, 3, 30, "fp64")
        _, info = B.solve(np.concatenate(rhs), 1e-12, 3, 30, "fp64", raise_on_failure=False)
        assert info[0]["converged"] == 0 and info[0]["iterations"] == 3
        assert info[1]["converged"] == 1


def test_batch_rejects_invalid_input(backend):
    p = np.array([[0.0, 0.0, 0.0], [1.5, 0.0, 0.0], [0.0, 0.0, 0.0]])
    inv = lb.invert_polarisability(np.broadcast_to(np.eye(3) * (500 + 50j), (3, 3, 3)).copy())
    with pytest.raises(lb.InvalidGeometry):
        backend.create_batch([(p, inv, 0.01, 1.5)])
    with pytest.raises(lb.InvalidGeometry):
        backend.create_batch([])
    bad = p.copy()
    bad[2] = [np.nan, 0.0, 0.0]
    with pytest.raises(lb.InvalidGeometry):
        backend.create_batch([(bad, inv, 0.01, 1.5)])


@pytest.mark.parametrize("variant", ["1", "2", "3", "4"])
def test_batch_symmetric_scheme_matches_oracle(backend, rng, monkeypatch, variant):
    """The symmetric FP32 scheme over the batch (each unordered pair once per
    system, superblock pairs drawn from one work list; LUMINA_BATCH_SYM=v
    forces build v): systems of 200-1400 dipoles, so superblock edges and
    diagonal blocks are crossed; every system against the oracle, and the
    FP32+refine solve against the FP64 one."""
    monkeypatch.setenv("LUMINA_BATCH_SYM", variant)
    monkeypatch.setenv("LUMINA_BATCH_SYM_MIN_ITEMS", "0")  # every FP32 cycle symmetric
    w = small_batch(count=3, seed=7, n_range=(200, 1400))
    systems, specs = batch_inputs(w)
    with backend.create_batch(specs) as B:
        cfg = B.kernel_config()
        assert cfg["fp32_scheme"] == "symmetric" and cfg["sym32"] == int(variant)
        assert cfg["sym_min_items"] == 0
        x = rand_vec(rng, B.dim)
        y32 = B.split(B.matvec(x, "fp32"))
        xs = B.split(x)
        for s, (p, a, k, cell, _) in enumerate(systems):
            y_ref = orc.matvec_onthefly(p, a, xs[s], k, True, cell)
            assert rel_err(y32[s], y_ref) < 2e-5, (variant, s)
        b = np.concatenate([lb.incident_field(p, k, inc) for p, _, k, _, inc in systems])
        x32, i32 = B.solve(b, 1e-10, 5000, 30, "fp32_refine")
        x64, i64 = B.solve(b, 1e-10, 5000, 30, "fp64")
        for s, ((p, inv, k, cell), (_, _, _, _, inc)) in enumerate(zip(specs, systems)):
            c32 = lb.cross_sections(p, inv, B.split(x32)[s], k, inc)[0]
            c64 = lb.cross_sections(p, inv, B.split(x64)[s], k, inc)[0]
            assert abs(c32 - c64) <= 1e-6 * abs(c64), (variant, s)


def test_batch_scheme_switch_mid_solve(backend, monkeypatch):
    """A cycle runs the symmetric build while the active systems hold at
    least LUMINA_BATCH_SYM_MIN_ITEMS symmetric items, the split list below
    that.  With the threshold at the batch's full item count the first cycles
    are symmetric and the rest, once a system has converged, split: the
    FP32+refine solve still matches the FP64 one and the solves under either
    scheme alone (tolerance 1e-8, the clusters benchmark's; these Drude
    clusters take thousands of iterations)."""
    monkeypatch.setenv("LUMINA_BATCH_SYM", "2")
    w = small_batch(count=4, seed=11, n_range=(300, 1500))
    systems, specs = batch_inputs(w)
    total = sum(((p.shape[0] + 511) // 512) * ((p.shape[0] + 511) // 512 + 1) // 2
                for p, _, _, _ in specs)
    b = np.concatenate([lb.incident_field(p, k, inc) for p, _, k, _, inc in systems])
    cext = {}
    for label, min_items in (("hybrid", total), ("sym", 0), ("split", 10 ** 9)):
        monkeypatch.setenv("LUMINA_BATCH_SYM_MIN_ITEMS", str(min_items))
        with backend.create_batch(specs) as B:
            assert B.kernel_config()["sym_min_items"] == min_items
            x32, i32 = B.solve(b, 1e-8, 20000, 30, "fp32_refine")
            x64, _ = B.solve(b, 1e-8, 20000, 30, "fp64")
            cext[label] = []
            for s, ((p, inv, k, cell), (_, _, _, _, inc)) in enumerate(zip(specs, systems)):
                c32 = lb.cross_sections(p, inv, B.split(x32)[s], k, inc)[0]
                c64 = lb.cross_sections(p, inv, B.split(x64)[s], k, inc)[0]
                assert i32[s]["converged"] == 1, (label, s)
                assert abs(c32 - c64) <= 1e-6 * abs(c64), (label, s)
                cext[label].append(c32)
    for s in range(len(specs)):
        for label in ("hybrid", "sym"):
            assert abs(cext[label][s] - cext["split"][s]) <= 1e-6 * abs(cext["split"][s])
