"""Pins the oracle (the C restatement under oracle/) to the reference.

The golden fixture tests/golden/ref_L2.npz holds outputs of the reference's
own operators (compiled from its sources by oracle/ref_build) on a seeded L2
mesh; make_golden.py beside it regenerates it.  Every case is recomputed here
by the oracle from the same seeded inputs.  When the compiled reference is
present (oracle/_ref/ref_dump), a second test compares oracle and reference
live on an L3 mesh.  CPU only.
"""
import os
import sys
import tempfile

import numpy as np
import pytest

from helpers import rel
from oracle_lib import (Mesh, xdmf_geometry, xdmf_grid_bytes, xdmf_metadata, xdmf_read_grid, xdmf_step_xml,
                        xdmf_topology, xdmf_write_dir, chebyshev_smoother, fgmres, kerngen_vcycles, laplace_vcycles, pbicgstab, pminres, power_iteration, ref_available, run_ref, stokes_block_fgmres,
                        stokes_block_minres)

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as G  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_L2.npz")
TOL = 1e-12


@pytest.fixture(scope="module")
def case():
    g = np.load(GOLDEN)
    fine, coarse = Mesh(int(g["level"])), Mesh(int(g["level"]) - 1)
    x = G.inputs(fine, coarse)
    return g, fine, coarse, x


def test_inputs_regenerate(case):
    g, _, _, x = case
    for name, a in x.items():
        assert np.allclose(G.checksum(a), g["checksum_" + name], rtol=1e-13, atol=0), name


def test_mesh_matches_reference(case):
    g, fine, _, _ = case
    assert np.abs(fine.coords - g["coords"]).max() <= 1e-15
    assert np.abs(fine.radii - g["radii"]).max() <= 1e-15
    assert np.array_equal(fine.bmask, g["bmask"])
    assert np.array_equal(fine.omask, g["omask"])


@pytest.mark.parametrize("bcc,bcs,diag", G.KERNGEN_CASES)
def test_kerngen_matches_reference(case, bcc, bcs, diag):
    g, fine, _, x = case
    assert rel(fine.kerngen(x["k"], x["u"], bcc, bcs, diag), g[f"kerngen_{bcc}{bcs}{diag}"]) <= TOL


@pytest.mark.parametrize("treat,diag", G.LAPLACE_CASES)
def test_laplace_matches_reference(case, treat, diag):
    g, fine, _, x = case
    assert rel(fine.laplace(x["s"], treat, diag), g[f"laplace_{treat}{diag}"]) <= TOL


@pytest.mark.parametrize("bcc,bcs", G.STOKES_BCS)
def test_stokes_blocks_match_reference(case, bcc, bcs):
    g, fine, coarse, x = case
    assert rel(fine.divergence(coarse, x["u"], bcc, bcs), g[f"divergence_{bcc}{bcs}"]) <= TOL
    assert rel(fine.gradient(coarse, x["p"], bcc, bcs), g[f"gradient_{bcc}{bcs}"]) <= TOL


@pytest.mark.parametrize("bcc,bcs", G.STOKES_OP_BCS)
def test_stokes_operator_matches_reference(case, bcc, bcs):
    """EpsDivDivStokes (epsilon_divdiv_stokes.hpp:55-90): A (no halo) + B^T (Add, halo) on the velocity block,
    B on the pressure block, equals the composition of the pinned oracle blocks."""
    g, fine, coarse, x = case
    u = fine.kerngen(x["k"], x["u"], bcc, bcs) + fine.gradient(coarse, x["p"], bcc, bcs)
    p = fine.divergence(coarse, x["u"], bcc, bcs)
    assert rel(u, g[f"stokes_u_{bcc}{bcs}"]) <= TOL
    assert rel(p, g[f"stokes_p_{bcc}{bcs}"]) <= TOL


def test_power_iteration_matches_reference(case):
    """power_iteration.hpp:13-48 on D^-1 A (the Chebyshev smoother's estimate, 50 iterations) from the start
    vector the reference drew: the same eigenvalue estimate."""
    g, fine, _, _ = case
    inv = 1.0 / fine.laplace(np.ones(fine.shape), True, True)
    lam = power_iteration(lambda v: inv * fine.laplace(v, True, False), fine.dot, g["power_start"],
                          G.CHEBYSHEV_CASE["pits"])
    assert abs(lam - float(g["chebyshev_lambda"])) <= 1e-12 * abs(lam)


def test_chebyshev_smoother_matches_reference(case):
    """Chebyshev smoothing (chebyshev.hpp:100-160; order 3, 2 sweeps, rho carried across sweeps) from x = 0 with
    the eigenvalue estimate the reference's smoother computed (its power iteration starts from a seeded
    random vector, reproducible on one thread): the same iterate."""
    g, fine, _, x = case
    C = G.CHEBYSHEV_CASE
    inv = 1.0 / fine.laplace(np.ones(fine.shape), True, True)
    xo = chebyshev_smoother(lambda v: fine.laplace(v, True, False), inv, G.cg_rhs(x["s"]), np.zeros(fine.shape),
                            C["order"], C["iters"], float(g["chebyshev_lambda"]))
    assert rel(xo, g["chebyshev_x"]) <= TOL


def test_pbicgstab_matches_reference(case):
    """PBiCGStab(2) (pbicgstab.hpp:98-260) on the Dirichlet Laplace from x = 0, with the shadow residual the
    reference drew: the same number of steps and the same solution; residuals to 1e-5 relative above 1e-14."""
    g, fine, _, x = case
    B = G.BICGSTAB_CASE
    xo, ho = pbicgstab(lambda v: fine.laplace(v, True, False), fine.dot, G.cg_rhs(x["s"]), B["l"], B["maxit"],
                       B["tol"], g["bicgstab_rshadow"])
    assert len(ho) == len(g["bicgstab_hist"])
    np.testing.assert_allclose(ho, g["bicgstab_hist"], rtol=1e-5, atol=1e-14)
    assert rel(xo, g["bicgstab_x"]) <= TOL


def test_pminres_matches_reference(case):
    """PMINRES (pminres.hpp:30-175) on the Dirichlet Laplace from x = 0: the same iterations and solution as the
    reference's; residual estimates to 1e-6 relative above 1e-14 (amplified rounding)."""
    g, fine, _, x = case
    M = G.MINRES_CASE
    xo, ho = pminres(lambda v: fine.laplace(v, True, False), fine.dot, G.cg_rhs(x["s"]), M["maxit"], M["tol"])
    assert len(ho) == len(g["minres_hist"])
    np.testing.assert_allclose(ho, g["minres_hist"], rtol=1e-6, atol=1e-14)
    assert rel(xo, g["minres_x"]) <= TOL


def test_fgmres_matches_reference(case):
    """FGMRES(10) (fgmres.hpp:100-330) on the Dirichlet Laplace from x = 0, three restarts: the same number of
    iterations and the same solution as the reference's FGMRES; the residual estimates agree to rounding
    amplified by the Krylov process (reduction orders differ), checked to 1e-6 relative above 1e-14."""
    g, fine, _, x = case
    F = G.FGMRES_CASE
    xo, ho = fgmres(lambda v: fine.laplace(v, True, False), fine.dot, G.cg_rhs(x["s"]), F["restart"], F["maxit"],
                    F["tol"])
    assert len(ho) == len(g["fgmres_hist"])
    np.testing.assert_allclose(ho, g["fgmres_hist"], rtol=1e-6, atol=1e-14)
    assert rel(xo, g["fgmres_x"]) <= TOL


@pytest.mark.parametrize("bcc,bcs", G.STOKES_FGMRES["bcs"])
def test_stokes_block_fgmres_matches_reference(case, bcc, bcs):
    """The Stokes solve's composition (FGMRES, EpsDivDivStokes, the app's block-triangular preconditioner with
    the lumped inverse KMass(1/eta) Schur block), with a deterministic Jacobi velocity block in place of the
    multigrid: the same residual history and solution as the reference's own composition."""
    g, fine, coarse, x = case
    S = G.STOKES_FGMRES
    u, p, hist = stokes_block_fgmres(fine, coarse, x["k"], G.pressure_viscosity(x), x["u"], x["p"], bcc, bcs,
                                     S["restart"], S["maxit"], S["tol"], S["sweeps"], S["omega"])
    np.testing.assert_allclose(hist, g[f"stokes_fgmres_hist_{bcc}{bcs}"], rtol=1e-10, atol=1e-16)
    assert rel(u, g[f"stokes_fgmres_u_{bcc}{bcs}"]) <= TOL
    assert rel(p, g[f"stokes_fgmres_p_{bcc}{bcs}"]) <= TOL


@pytest.mark.parametrize("bcc,bcs", G.STOKES_MINRES["bcs"])
def test_stokes_block_minres_matches_reference(case, bcc, bcs):
    """PMINRES on the Stokes block operator with the block-diagonal preconditioner (block_preconditioner_2x2.hpp:
    38-100; the Stokes solver's outer = 1): the same history and solution as the reference's composition."""
    g, fine, coarse, x = case
    S = G.STOKES_MINRES
    u, p, hist = stokes_block_minres(fine, coarse, x["k"], G.pressure_viscosity(x), x["u"], x["p"], bcc, bcs,
                                     S["maxit"], S["tol"], S["sweeps"], S["omega"])
    np.testing.assert_allclose(hist, g[f"stokes_minres_hist_{bcc}{bcs}"], rtol=1e-10, atol=1e-16)
    assert rel(u, g[f"stokes_minres_u_{bcc}{bcs}"]) <= TOL
    assert rel(p, g[f"stokes_minres_p_{bcc}{bcs}"]) <= TOL


def test_laplace_vcycles_match_reference(case):
    """Multigrid (multigrid.hpp:108-211) with Jacobi smoothing, constant transfers and the coarse PCG: two
    V-cycles over levels 1-3 from x = 0 against the reference's own Multigrid<Laplace, ...>."""
    g = case[0]
    V = G.VCYCLE
    b = G.vcycle_rhs()
    assert np.allclose(G.checksum(b), g["checksum_vcycle_b"], rtol=1e-13, atol=0)
    meshes = [Mesh(level) for level in range(V["lmin"], V["lmax"] + 1)]
    x = laplace_vcycles(meshes, b, V["omega"], V["smooth"], V["cycles"], V["cmaxit"])
    assert rel(x, g["vcycle_x"]) <= TOL


def test_kerngen_vcycles_match_reference(case):
    """The velocity block's V-cycle structure: two V-cycles over levels 1-3 on the free-slip epsilon-div-div
    operator (rotation penalty included) with Jacobi smoothing, constant vector transfers and the coarse PCG,
    against the reference's own Multigrid<EpsilonDivDivKerngen, ...>.  The 50-iteration coarse CG amplifies
    rounding, hence 1e-10."""
    g = case[0]
    K = G.KVCYCLE
    ks, b = G.kvcycle_inputs()
    assert np.allclose(G.checksum(b), g["checksum_kvcycle_b"], rtol=1e-13, atol=0)
    meshes = [Mesh(level) for level in range(K["lmin"], K["lmax"] + 1)]
    x = kerngen_vcycles(meshes, ks, b, *K["bcs"], K["omega"], K["smooth"], K["cycles"], K["cmaxit"])
    assert rel(x, g["kvcycle_x"]) <= 1e-10


def test_transfers_match_reference(case):
    g, fine, coarse, x = case
    assert rel(fine.prolong(coarse, x["uc"]), g["prolong"]) <= TOL
    assert rel(fine.restrict(coarse, x["u"]), g["restrict"]) <= TOL


def test_linear_transfers_match_reference(case):
    g, fine, coarse, x = case
    assert rel(fine.prolong_linear(coarse, x["pc"]), g["prolong_linear"]) <= TOL
    assert rel(fine.restrict_linear(coarse, x["s"]), g["restrict_linear"]) <= TOL


@pytest.mark.parametrize("mode", G.MASS_MODES)
def test_mass_is_kmass_with_unit_k(case, mode):
    """Mass (mass.hpp) equals KMass with k = 1: the oracle's kmass with unit k reproduces it."""
    g, fine, _, x = case
    assert rel(fine.kmass(np.ones(fine.shape), x["s"], mode), g[f"mass_{mode}"]) <= TOL


@pytest.mark.parametrize("mode", G.VMASS_MODES)
def test_vector_mass_is_componentwise_mass(case, mode):
    """VectorMass (vector_mass.hpp) applies Mass to each component."""
    g, fine, _, x = case
    ref = np.stack([fine.kmass(np.ones(fine.shape), x["u"][c], mode) for c in range(3)])
    assert rel(ref, g[f"vmass_{mode}"]) <= TOL


@pytest.mark.parametrize("mode", G.KMASS_MODES)
def test_kmass_matches_reference(case, mode):
    g, fine, _, x = case
    assert rel(fine.kmass(x["k"], x["s"], mode), g[f"kmass_{mode}"]) <= TOL


@pytest.mark.parametrize("treat,diag", G.EPSDIVDIV_CASES)
def test_epsdivdiv3x2_matches_reference(case, treat, diag):
    g, fine, _, x = case
    assert rel(fine.epsdivdiv3x2(x["k"], x["u"], treat, diag), g[f"epsdivdiv_{treat}{diag}"]) <= TOL


@pytest.mark.parametrize("treat,diag,single", G.DIVKGRAD_CASES)
def test_divkgrad_matches_reference(case, treat, diag, single):
    g, fine, _, x = case
    assert rel(fine.divkgrad(x["k"], x["s"], treat, diag, single), g[f"divkgrad_{treat}{diag}{single}"]) <= TOL


@pytest.mark.parametrize("bcc,bcs,diag", G.VLAPLACE_CASES)
def test_vector_laplace_matches_reference(case, bcc, bcs, diag):
    g, fine, _, x = case
    assert rel(fine.vector_laplace(x["u"], bcc, bcs, diag), g[f"vlaplace_{bcc}{bcs}{diag}"]) <= TOL


@pytest.mark.parametrize("kappa,bc", G.FCT_CASES)
def test_fct_matches_reference(case, kappa, bc):
    g, fine, _, _ = case
    vel, T, src = G.fct_inputs(fine)
    c = fine.fv_cell_centers()
    assert np.abs(c - g["fct_centers"]).max() <= 1e-15
    tag = f"fct_{kappa:g}_{bc}"
    dt_stable, dt = g[tag + "_dt"]
    assert fine.fct_dt_stable(c, vel, kappa) == pytest.approx(dt_stable, rel=1e-13)
    T0 = fine.fct_dirichlet(T) if bc else T.copy()
    Tn, TL = fine.fct_step(c, vel, fine.fv_ghost_update(T0), dt, kappa, src, True, (1.0, 0.0, 1, 1) if bc else None)
    N = fine.N
    inner = (slice(None), slice(1, N + 1), slice(1, N + 1), slice(1, N + 1))
    assert rel(Tn[inner], g[tag + "_T"][inner]) <= TOL
    assert rel(TL[inner], g[tag + "_TL"][inner]) <= TOL
    assert rel(Tn, g[tag + "_T"]) <= TOL  # ghost layers included


@pytest.mark.parametrize("bcc,bcs,diag", G.KSLOW_CASES)
def test_stored_matrices_and_slow_path_match_reference(case, bcc, bcs, diag):
    """The kerngen wedge matrices (assemble_local_matrix, epsilon_divdiv_kerngen.hpp:2051-2110) and the slow
    path that applies them with the boundary treatment at apply time (:823-1052): the oracle's
    or_kerngen_local_matrices + or_stored_apply against the reference's own matrices stored in Full mode."""
    g, fine, _, x = case
    mats = fine.local_matrices(x["k"])
    assert rel(mats[G.KSLOW_CELLS], g["kslow_mats"]) <= TOL
    assert rel(fine.stored_apply(mats, x["u"], bcc, bcs, diag), g[f"kslow_{bcc}{bcs}{diag}"]) <= TOL


@pytest.mark.parametrize("mode,bcc,bcs,diag", G.GCA_CASES)
def test_gca_coarse_operator_matches_reference(case, mode, bcc, bcs, diag):
    """TwoGridGCA (gca/gca.hpp:154-528; constant and linear interpolation) of the Neumann kerngen operator into
    the coarser level, applied through the slow path with the coarse boundary conditions: the oracle's
    or_gca_coarsen + or_stored_apply against the reference's coarse operator."""
    g, fine, coarse, x = case
    mc = fine.gca_coarsen(coarse, k=x["k"], mode=mode)
    assert rel(coarse.stored_apply(mc, x["uc"], bcc, bcs, diag), g[f"gca_{mode}_{bcc}{bcs}{diag}"]) <= TOL


@pytest.mark.skipif(not ref_available(), reason="compiled reference (oracle/_ref/ref_dump) not built here")
def test_slow_path_and_gca_match_live_reference_L3():
    """Level 3 (its coarse level 2), live against the compiled reference: every wedge matrix, the slow-path
    apply and the GCA coarse operators of both interpolation modes."""
    L = 3
    f, c = Mesh(L), Mesh(L - 1)
    rs = np.random.RandomState(11)
    k = f.make_consistent(np.exp(2.0 * rs.normal(size=f.shape)))
    u = f.make_consistent(rs.normal(size=(3,) + f.shape))
    uc = c.make_consistent(rs.normal(size=(3,) + c.shape))
    mats = f.local_matrices(k)
    with tempfile.TemporaryDirectory() as d:
        k.tofile(f"{d}/k.bin")
        u.tofile(f"{d}/src.bin")
        for bcc, bcs, diag in [(2, 2, 0), (1, 2, 0), (2, 1, 1)]:
            run_ref(["kerngen_slow", L, 0.55, 1.0, bcc, bcs, diag, d], d)
            assert rel(mats, np.fromfile(f"{d}/mats.bin").reshape(mats.shape)) <= TOL
            ref = np.fromfile(f"{d}/dst.bin").reshape((3,) + f.shape)
            assert rel(f.stored_apply(mats, u, bcc, bcs, diag), ref) <= TOL
        uc.tofile(f"{d}/src.bin")
        for mode in (0, 1):
            mc = f.gca_coarsen(c, k=k, mode=mode)
            for bcc, bcs, diag in [(2, 2, 0), (1, 1, 0), (2, 1, 1)]:
                run_ref(["gca", L, 0.55, 1.0, bcc, bcs, diag, mode, d], d)
                ref = np.fromfile(f"{d}/dst.bin").reshape((3,) + c.shape)
                assert rel(c.stored_apply(mc, uc, bcc, bcs, diag), ref) <= TOL


@pytest.mark.parametrize("lumped", G.L2PROJ_MODES)
def test_l2_projection_matches_reference(case, lumped):
    """l2_project_fv_to_fe (Q1 mass + PCG to 1e-12, conversion.hpp:131-205) and its lumped form (:243-300) of a
    seeded FV field: the oracle against the reference (the consistent form to the solver's tolerance)."""
    g, fine, _, _ = case
    fv, T = G.timestep_inputs(fine)
    assert np.allclose(G.checksum(fv), g["checksum_ts_fv"], rtol=1e-13, atol=0)
    tol = TOL if lumped else 1e-10
    assert rel(fine.l2_project_fv_to_fe(fv, lumped=bool(lumped)), g[f"l2proj_{lumped}"]) <= tol


@pytest.mark.parametrize("bcc,bcs", G.STOKES_RHS_BCS)
def test_stokes_buoyancy_rhs_matches_reference(case, bcc, bcs):
    """The app's Stokes right-hand side (mantlecirculation.cpp:876-899): VectorMass of Ra T n with the strong
    Dirichlet / free-slip enforcement on the boundary get_shell_boundary_flag names."""
    g, fine, _, _ = case
    fv, T = G.timestep_inputs(fine)
    assert np.allclose(G.checksum(T), g["checksum_ts_T"], rtol=1e-13, atol=0)
    assert rel(fine.stokes_buoyancy_rhs(T, G.STOKES_RHS_RA, bcc, bcs), g[f"stokes_rhs_{bcc}{bcs}"]) <= TOL


def test_fe_to_fv_matches_reference(case):
    """l2_project_fe_to_fv (conversion.hpp:349-416): cell averages of the seeded FE temperature, lateral ghosts
    updated, against the reference"""
    g, fine, _, _ = case
    _, T = G.timestep_inputs(fine)
    ref = g["fe2fv"]
    assert np.abs(fine.l2_project_fe_to_fv(T) - ref).max() <= 1e-15 * np.abs(ref).max()


def _xdmf_grids(fine, coarse, step):
    return [dict(label=lab, in_bytes=ib, out_bytes=ob, vec=v, data=a)
            for lab, ib, ob, v, a in G.xdmf_fields(fine, coarse, step)]


def test_xdmf_restatement_matches_reference_files(case):
    """Every file io::XDMFOutput wrote for the fixture (tests/golden/xdmf_L2: geometry, topology, metadata, the
    six grids of both writes, both .xmf steps) is byte for byte the restatement's"""
    _, fine, coarse, _ = case
    d = G.XDMF_DIR

    def raw(name):
        with open(os.path.join(d, name), "rb") as f:
            return f.read()
    assert raw("geometry.bin") == xdmf_geometry(fine, G.XDMF_PTS)
    assert raw("topology.bin") == xdmf_topology(fine, G.XDMF_CONN)
    assert raw("checkpoint_metadata.bin") == xdmf_metadata(fine, _xdmf_grids(fine, coarse, 0), G.XDMF_PTS)
    for step in (0, 1):
        grids = _xdmf_grids(fine, coarse, step)
        for gr in grids:
            assert raw(f'{gr["label"]}_{step}.bin') == xdmf_grid_bytes(gr["data"], gr["vec"], gr["out_bytes"]), gr["label"]
        assert raw(f"step_{step}.xmf").decode() == xdmf_step_xml(fine, grids, step, G.XDMF_PTS, G.XDMF_CONN)
    assert sorted(os.listdir(d)) == sorted(
        ["README.md", "geometry.bin", "topology.bin", "checkpoint_metadata.bin"]
        + [f"{lab}_{s}.bin" for lab, *_ in G.XDMF_GRIDS for s in (0, 1)] + ["step_0.xmf", "step_1.xmf"])


def test_xdmf_reader_restatement(case):
    """read_xdmf_checkpoint_grid restated: every grid of the reference's checkpoint reads back as written
    (FP32 outputs as the cast of the input)"""
    _, fine, coarse, _ = case
    for step in (0, 1):
        for gr in _xdmf_grids(fine, coarse, step):
            want = gr["data"].astype(np.float32 if gr["out_bytes"] == 4 else np.float64).astype(np.float64)
            got = xdmf_read_grid(G.XDMF_DIR, gr["label"], step, fine, gr["vec"] == 3)
            assert np.array_equal(got, want), gr["label"]


@pytest.mark.skipif(not ref_available(), reason="compiled reference not built")
def test_xdmf_live_against_reference():
    """Live, at level 3: FP64 points and int32 connectivity written by the reference equal the restatement;
    the reference's reader recovers the grids of a checkpoint the restatement wrote with the diamonds' chunks
    in a shuffled order (the metadata's subdomain ids say where each is)."""
    fine, coarse = Mesh(3), Mesh(2)
    rs = np.random.RandomState(77)
    T = fine.make_consistent(rs.normal(size=fine.shape)).reshape(fine.shape)
    u = rs.normal(size=(3,) + fine.shape)
    with tempfile.TemporaryDirectory() as d:
        T.tofile(f"{d}/T.bin")
        u.tofile(f"{d}/u.bin")
        run_ref(["xdmf_write", 3, 0.55, 1.0, 8, 4, d], d)
        # FP64 coordinates to one unit in the last place: this build of the reference contracts the sum of
        # squares of its normalisation (dense/vec.hpp:76-97) into FMAs (-march=x86-64-v3); the oracle does not
        ref_geo = np.fromfile(f"{d}/xdmf/geometry.bin")
        geo = np.frombuffer(xdmf_geometry(fine, 8), dtype=np.float64)
        assert np.abs(ref_geo - geo).max() <= 2.3e-16
        with open(f"{d}/xdmf/topology.bin", "rb") as f:
            assert f.read() == xdmf_topology(fine, 4)
        with open(f"{d}/xdmf/u64_1.bin", "rb") as f:
            assert f.read() == xdmf_grid_bytes(2 * u, 3, 8)
        order = [3, 7, 0, 9, 1, 5, 2, 8, 6, 4]
        grids = [dict(label="T", in_bytes=8, out_bytes=8, vec=1, data=T),
                 dict(label="u_u", in_bytes=8, out_bytes=4, vec=3, data=u)]
        xdmf_write_dir(f"{d}/ck", fine, [grids], pts=4, conn=8, order=order)
        run_ref(["xdmf_read", 3, 0.55, 1.0, "T", 0, 0, f"{d}/ck", d], d)
        assert np.array_equal(np.fromfile(f"{d}/out.bin").reshape(fine.shape), T)
        run_ref(["xdmf_read", 3, 0.55, 1.0, "u_u", 0, 1, f"{d}/ck", d], d)
        got = np.fromfile(f"{d}/out.bin").reshape((3,) + fine.shape)
        assert np.array_equal(got, u.astype(np.float32).astype(np.float64))
        assert np.array_equal(xdmf_read_grid(f"{d}/ck", "u_u", 0, fine, True), got)


@pytest.mark.skipif(not ref_available(), reason="compiled reference not built")
def test_fe_to_fv_live_against_reference():
    fine = Mesh(3)
    T = fine.make_consistent(np.random.RandomState(78).uniform(size=fine.shape)).reshape(fine.shape)
    with tempfile.TemporaryDirectory() as d:
        T.tofile(f"{d}/T.bin")
        run_ref(["fe2fv", 3, 0.55, 1.0, d], d)
        ref = np.fromfile(f"{d}/fv.bin").reshape(fine.fv_shape)
    assert np.abs(fine.l2_project_fe_to_fv(T) - ref).max() <= 1e-15 * np.abs(ref).max()


def _supg_key(c):
    return "supg_" + "_".join(str(v) for v in c)


@pytest.mark.parametrize("c", G.SUPG_CASES)
def test_supg_matches_reference(case, c):
    """UnsteadyAdvectionDiffusionSUPG (unsteady_advection_diffusion_supg.hpp:199-420) with its mass lumping,
    boundary mask and diagonal mode, against the reference on the seeded level-2 inputs"""
    g, fine, _, _ = case
    vel, src = G.supg_inputs(fine)
    assert np.allclose(G.checksum(vel), g["checksum_supg_vel"], rtol=1e-13, atol=0)
    kappa, dt, ms, lumped, treat, diag = c
    out = fine.supg(vel, src, kappa, dt, ms, bool(lumped), bool(treat), bool(diag))
    assert rel(out, g[_supg_key(c)]) <= TOL


@pytest.mark.skipif(not ref_available(), reason="compiled reference not built")
def test_supg_live_against_reference():
    fine = Mesh(3)
    rs = np.random.RandomState(81)
    vel = rs.normal(size=(3,) + fine.shape)
    src = rs.normal(size=fine.shape)
    with tempfile.TemporaryDirectory() as d:
        vel.tofile(f"{d}/vel.bin")
        src.tofile(f"{d}/src.bin")
        for c in [(1e-3, 1e-2, 1.0, 0, 1, 0), (0.05, 0.1, 2.0, 1, 0, 0)]:
            run_ref(["supg", 3, 0.55, 1.0, *c, d], d)
            ref = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)
            kappa, dt, ms, lumped, treat, diag = c
            assert rel(fine.supg(vel, src, kappa, dt, ms, bool(lumped), bool(treat), bool(diag)), ref) <= TOL


@pytest.mark.parametrize("bc", G.AGCA_CASES)
def test_agca_matches_reference(case, bc):
    """Adaptive GCA (GCAElementsCollector marks on level 1 from the level-3 viscosity, Selective storage on
    level 2, TwoGridGCA on the marked elements, the level-2 kerngen matrices elsewhere) and the coarse apply,
    against the reference"""
    g = case[0]
    fine, coarse, k, kc, src = G.agca_inputs()
    assert np.allclose(G.checksum(src), g["checksum_agca_src"], rtol=1e-13, atol=0)
    marks = fine.gca_elements(k, 2)
    assert np.array_equal(marks, g["agca_marks"]) and 0 < marks.sum() < marks.size
    mats = fine.agca_coarsen(coarse, marks, 1, kc, k=k)
    bcc, bcs, diag = bc
    assert rel(coarse.stored_apply(mats, src, bcc, bcs, bool(diag)), g[f"agca_{bcc}{bcs}{diag}"]) <= TOL


def test_golden_fixture_is_not_trivial(case):
    """A planted error in the oracle's input must break the comparison."""
    g, fine, _, x = case
    u = x["u"].copy()
    u[0, 3, 1, 2, 2] += 1e-3
    assert rel(fine.kerngen(x["k"], u, 1, 1, 0), g["kerngen_110"]) > 1e-8


def test_laplace_pcg_matches_reference(case):
    """The PCG restatement reaches the reference solver's solution in the same number of iterations."""
    g, fine, _, x = case
    sol, its = fine.laplace_pcg(G.cg_rhs(x["s"]), G.CG_MAXIT, G.CG_TOL)
    assert its == int(g["laplace_cg_iterations"])
    assert rel(sol, g["laplace_cg_x"]) <= 1e-11


@pytest.mark.skipif(not ref_available(), reason="compiled reference (oracle/_ref/ref_dump) not built here")
def test_oracle_matches_live_reference_L3():
    L = 3
    m = Mesh(L)
    rs = np.random.RandomState(7)
    k = m.make_consistent(np.exp(rs.normal(size=m.shape)))
    u = m.make_consistent(rs.normal(size=(3,) + m.shape))
    with tempfile.TemporaryDirectory() as d:
        k.tofile(f"{d}/k.bin")
        u.tofile(f"{d}/src.bin")
        for bcc, bcs in [(2, 2), (1, 2)]:
            run_ref(["kerngen", L, 0.55, 1.0, bcc, bcs, 0, d], d)
            ref = np.fromfile(f"{d}/dst.bin").reshape((3,) + m.shape)
            assert rel(m.kerngen(k, u, bcc, bcs, False), ref) <= TOL
