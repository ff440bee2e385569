"""Generate the golden fixtures in tests/golden/ (committed with this script).

An independent, vectorised numpy restatement of the reference's Green's
tensor (greens.rs:34-71), its FCD cell average (greens.rs:94-167), the
interaction matrix (assembly.rs:45-175) and the cross sections
(cda/mod.rs:175-236), solved with numpy's LAPACK LU.  It shares no code with
the C++ oracle, so agreement between the two (and with the CUDA library)
checks all three.

Cases (seeded, synthetic):
  sphere_au_r6_d2    Au sphere R = 6 nm, 2 nm lattice (N = 123), 520 nm, FCD
  sphere_au_r12_d2   the 925-dipole Au sphere at 520 nm, FCD (cell = 2 nm)
  jitter_aniso       jittered 1.5 nm lattice, random anisotropic alpha, 480 nm, FCD
  substrate_r5       Au sphere above an n = 1.45 substrate (retarded r), 560 nm

Each fixture stores positions, alpha (N x 3 x 3), k, flags, the solved
moments, C_ext/C_abs/C_sca and y = A x for a seeded x.
Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lumina_b200 import configs, geometry  # noqa: E402


def greens_np(d, k):
    """Point tensors for displacements d (M, 3) -> (M, 3, 3) complex."""
    r = np.sqrt(np.sum(d * d, axis=1))
    kr = k * r
    pf = k * k * np.exp(1j * kr) / (4 * np.pi * r)
    a = 1 + (1j * kr - 1) / kr ** 2
    b = (3 - 3j * kr - kr ** 2) / kr ** 2
    rh = d / r[:, None]
    return pf[:, None, None] * (a[:, None, None] * np.eye(3)[None]
                                + b[:, None, None] * rh[:, :, None] * rh[:, None, :])


def fcd_np(ri, rj, k, cell):
    nodes = np.array([-np.sqrt(0.6), 0.0, np.sqrt(0.6)])
    w = np.array([5 / 9, 8 / 9, 5 / 9])
    acc = np.zeros((3, 3), complex)
    tw = 0.0
    for ix in range(3):
        for iy in range(3):
            for iz in range(3):
                rp = rj + cell / 2 * np.array([nodes[ix], nodes[iy], nodes[iz]])
                dd = ri - rp
                if dd @ dd < 1e-20:
                    continue
                wt = w[ix] * w[iy] * w[iz]
                acc += wt * greens_np(dd[None], k)[0]
                tw += wt
    return acc / tw


def assemble_np(pos, alpha, k, use_fcd, cell, sub=None):
    n = len(pos)
    A = np.zeros((3 * n, 3 * n), complex)
    for i in range(n):
        A[3 * i:3 * i + 3, 3 * i:3 * i + 3] = np.linalg.inv(alpha[i])
        d = pos[i] - pos
        mask = np.arange(n) != i
        G = np.zeros((n, 3, 3), complex)
        G[mask] = greens_np(d[mask], k)
        if use_fcd:
            dist = np.sqrt(np.sum(d * d, axis=1))
            for j in np.nonzero(mask & ~(dist > 2.0 * cell))[0]:
                G[j] = fcd_np(pos[i], pos[j], k, cell)
        A[3 * i:3 * i + 3, :] -= G.transpose(1, 0, 2).reshape(3, 3 * n)
        if sub is not None:
            z0, refl = sub
            img = pos.copy()
            img[:, 2] = 2 * z0 - img[:, 2]
            dimg = pos[i] - img
            ok = np.sum(dimg * dimg, axis=1) >= 1e-20
            Gi = np.zeros((n, 3, 3), complex)
            Gi[ok] = greens_np(dimg[ok], k)
            m = np.array([-refl, -refl, refl])
            A[3 * i:3 * i + 3, :] -= (Gi * m[None, None, :]).transpose(1, 0, 2).reshape(3, 3 * n)
    return A


def cross_np(pos, alpha, p, k):
    e = np.exp(1j * k * pos[:, 2])[:, None] * np.array([1.0, 0, 0])[None]
    P = p.reshape(-1, 3)
    cext = k * np.sum((np.conj(e) * P).imag)
    inv = np.linalg.inv(alpha)
    cabs = 0.0
    for i in range(len(pos)):
        cabs += (P[i] @ np.conj(inv[i]) @ np.conj(P[i])).imag - (2 / 3) * k ** 3 * np.sum(np.abs(P[i]) ** 2)
    cabs *= k
    return np.array([cext, cabs, max(cext - cabs, 0.0)])


def case(name, pos, alpha, k, use_fcd, cell, sub=None, seed=0):
    A = assemble_np(pos, alpha, k, use_fcd, cell, sub)
    b = (np.exp(1j * k * pos[:, 2])[:, None] * np.array([1.0, 0, 0])[None]).ravel()
    p = np.linalg.solve(A, b)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(3 * len(pos)) + 1j * rng.standard_normal(3 * len(pos))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), positions=pos, alpha=alpha, k=k,
                        use_fcd=use_fcd, cell=cell,
                        substrate=np.array(sub if sub else (np.nan, np.nan), complex),
                        moments=p, cross=cross_np(pos, alpha, p, k), x=x, y=A @ x)
    print(name, len(pos))


def main():
    w = configs.au_workload("s", geometry.discretise_primitive(geometry.Sphere((0, 0, 0), 6.0), 2.0),
                            2.0, 520.0)
    case("sphere_au_r6_d2", w.positions, w.alpha, w.k, True, 2.0)
    w = configs.sphere_au_925()
    case("sphere_au_r12_d2", w.positions, w.alpha, w.k, True, 2.0)
    rng = np.random.default_rng(11)
    base = geometry.discretise_primitive(geometry.Sphere((1.0, -2.0, 0.5), 5.0), 1.5)
    pos = base + rng.uniform(-0.2, 0.2, base.shape)
    n = len(pos)
    alpha = (np.eye(3) * (3.0 + 1.5j))[None] + 0.3 * (rng.standard_normal((n, 3, 3))
                                                      + 1j * rng.standard_normal((n, 3, 3)))
    case("jitter_aniso", pos, alpha, 2 * np.pi / 480.0, True, 1.5)
    base = geometry.discretise_primitive(geometry.Sphere((0, 0, 12.0), 5.0), 2.0)
    w = configs.au_workload("sub", base, 2.0, 560.0)
    case("substrate_r5", w.positions, w.alpha, w.k, True, 2.0, sub=(0.0, 0.45 / 2.45))


if __name__ == "__main__":
    main()
