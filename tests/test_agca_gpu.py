"""Adaptive GCA (the app's gca == 2; here tn_stokes_params.gca = 3): the element collector's marks
(tn_gca_elements_f64), the selectively Galerkin coarse matrices (tn_gca_coarsen_f64 +
tn_agca_unmarked_local_matrices_f64) applied with the stored-matrix kernel against the reference's own adaptive
GCA apply (tests/golden/ref_L2.npz) and the oracle, a two-step coarsening, and the Stokes solve with it."""
import os
import sys

import numpy as np
import pytest
import torch

from helpers import rel, random_vector
from oracle_lib import Mesh

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_L2.npz")


def _scalar(shell, pm, a):
    v = shell.VectorQ1Scalar(pm)
    v.set_numpy(a)
    return v


@pytest.mark.parametrize("bc", G.AGCA_CASES)
def test_agca_apply_matches_reference(bc):
    from terraneo_b200 import shell
    g = np.load(GOLDEN)
    fine, coarse, k, kc, src = G.agca_inputs()
    pf, pc = shell.ShellMesh(G.AGCA_L), shell.ShellMesh(G.AGCA_L - 1)
    kv, kcv = _scalar(shell, pf, k), _scalar(shell, pc, kc)
    marks = shell.gca_elements(pf, kv, 2)
    assert np.array_equal(marks.cpu().numpy(), g["agca_marks"])
    mats = shell.agca_coarsen(pf, pc, marks, 1, k_coarse=kcv, k_fine=kv)
    bcc, bcs, diag = bc
    op = shell.StoredEpsilonDivDiv(pc, mats, bcc, bcs, diagonal=bool(diag))
    u, v = shell.VectorQ1Vec(pc), shell.VectorQ1Vec(pc)
    u.set_numpy(src)
    shell.apply(op, u, v)
    assert rel(v.numpy(), g[f"agca_{bcc}{bcs}{diag}"]) <= 1e-12


def test_agca_two_coarsenings_match_oracle():
    """level 4 -> 3 -> 2 with the marks on level 1 (level ranges 3, 2, 1): the second coarsening starts from the
    first one's selective matrices, as the app's hierarchy does"""
    from terraneo_b200 import shell
    f, c1, c2 = Mesh(4), Mesh(3), Mesh(2)
    k, k1, k2 = G.blob_viscosity(f), G.blob_viscosity(c1), G.blob_viscosity(c2)
    marks = f.gca_elements(k, 3)
    assert 0 < marks.sum() < marks.size
    m1 = f.agca_coarsen(c1, marks, 2, k1, k=k)
    m2 = c1.agca_coarsen(c2, marks, 1, k2, mats_fine=m1)
    src = random_vector(c2, seed=4)
    want = c2.stored_apply(m2, src, 2, 2)
    pf, p1, p2 = shell.ShellMesh(4), shell.ShellMesh(3), shell.ShellMesh(2)
    kv, k1v, k2v = _scalar(shell, pf, k), _scalar(shell, p1, k1), _scalar(shell, p2, k2)
    gm = shell.gca_elements(pf, kv, 3)
    assert np.array_equal(gm.cpu().numpy(), marks)
    g1 = shell.agca_coarsen(pf, p1, gm, 2, k_coarse=k1v, k_fine=kv)
    g2 = shell.agca_coarsen(p1, p2, gm, 1, k_coarse=k2v, mats_fine=g1)
    u, v = shell.VectorQ1Vec(p2), shell.VectorQ1Vec(p2)
    u.set_numpy(src)
    shell.apply(shell.StoredEpsilonDivDiv(p2, g2, 2, 2), u, v)
    assert rel(v.numpy(), want) <= 1e-12


@pytest.mark.parametrize("bc", [(1, 1), (2, 1)])
def test_stokes_solve_with_adaptive_gca(bc):
    """the Stokes solver with gca = 3 at level 4 (blob viscosity, a part of the coarsest cells marked): the FP64
    true residual under the oracle operators reaches the tolerance, in a few more or fewer iterations than the
    full GCA (free-slip on both radii is left out: with a random right-hand side the rigid rotations make it
    nearly singular)"""
    from terraneo_b200 import shell
    L = 4
    om, oc = Mesh(L), Mesh(L - 1)
    k = G.blob_viscosity(om)
    pm = shell.ShellMesh(L)
    kv = _scalar(shell, pm, k)
    f = random_vector(om, seed=21)
    if bc[0] == 1:
        f[:, :, :, :, 0] = 0
    if bc[1] == 1:
        f[:, :, :, :, -1] = 0
    fu, fp = shell.VectorQ1Vec(pm), shell.VectorQ1Scalar(shell.ShellMesh(L - 1))
    fu.set_numpy(f)
    fu.halo_sum()
    if 2 in bc:
        shell.freeslip_project(fu, bc[0] == 2, bc[1] == 2)
    its = {}
    for gca in (1, 3):
        s = shell.StokesSolver(L, kv, mg_levels=3, bc_cmb=bc[0], bc_surface=bc[1], mg_fp32=False, gca=gca,
                               relative_tolerance=1e-9, max_iterations=400, restart=100)
        xu, xp = shell.VectorQ1Vec(pm), shell.VectorQ1Scalar(fp.mesh)
        its[gca], rr = s.solve(fu, fp, xu, xp)
        u, p = xu.numpy(), xp.numpy()[0]
        b = fu.numpy()
        ru = om.kerngen(k, u, *bc) + om.gradient(oc, p, *bc) - b
        rp = om.divergence(oc, u, *bc)
        true_rr = np.sqrt(om.dot(ru, ru) + oc.dot(rp, rp)) / np.sqrt(om.dot(b, b))
        assert true_rr <= 1e-8, (gca, its[gca], rr, true_rr)
    assert its[3] <= 2 * its[1] + 10, its
