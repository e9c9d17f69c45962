"""Generate the golden fixtures in this folder from the reference itself.

Runs the reference's own operators, compiled from its sources into
oracle/_ref/ref_dump (recipe: oracle/ref_build/Makefile), on small seeded
meshes and writes their outputs to ref_L2.npz.  Inputs are not stored: they
are regenerated from numpy's frozen legacy generator (RandomState) with the
seeds below, and the fixture keeps their checksums so a drift in generation
shows up as a failing check instead of a silent mismatch.

Usage (in a container that has the reference sources and a built ref_dump):
    python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle_lib import Mesh, run_ref  # noqa: E402

L = 2
R_MIN, R_MAX = 0.55, 1.0
KERNGEN_CASES = [(1, 1, 0), (2, 2, 0), (2, 1, 0), (1, 2, 0), (0, 0, 0), (0, 1, 0), (1, 1, 1), (2, 2, 1)]
LAPLACE_CASES = [(1, 0), (0, 0), (1, 1)]
STOKES_BCS = [(1, 1), (2, 2), (0, 0)]
KMASS_MODES = [0, 1, 2]
DIVKGRAD_CASES = [(1, 0, 0), (0, 0, 0), (1, 1, 0), (1, 0, 1)]
VLAPLACE_CASES = [(1, 1, 0), (0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 1)]


def inputs(fine, coarse):
    """Seeded inputs (numpy RandomState is stream-stable across versions)."""
    rs = np.random.RandomState(20240601)
    k = fine.make_consistent(np.exp(rs.normal(size=fine.shape)))
    u = fine.make_consistent(rs.normal(size=(3,) + fine.shape))
    s = fine.make_consistent(rs.normal(size=fine.shape))
    p = coarse.make_consistent(rs.normal(size=coarse.shape))
    uc = coarse.make_consistent(rs.normal(size=(3,) + coarse.shape))
    pc = coarse.make_consistent(rs.normal(size=coarse.shape))
    return dict(k=k, u=u, s=s, p=p, uc=uc, pc=pc)


def checksum(a):
    a = np.asarray(a, dtype=np.float64)
    return np.array([a.sum(), (a * a).sum(), np.abs(a).max()])


def main():
    fine, coarse = Mesh(L), Mesh(L - 1)
    x = inputs(fine, coarse)
    out = {"level": np.array(L), "r_range": np.array([R_MIN, R_MAX])}
    for name, a in x.items():
        out["checksum_" + name] = checksum(a)
    with tempfile.TemporaryDirectory() as d:
        run_ref(["mesh", L, R_MIN, R_MAX, d], d)
        out["coords"] = np.fromfile(f"{d}/coords.bin").reshape(fine.coords.shape)
        out["radii"] = np.fromfile(f"{d}/radii.bin").reshape(fine.radii.shape)
        out["bmask"] = np.fromfile(f"{d}/bmask.bin", np.uint8).reshape(fine.shape)
        out["omask"] = np.fromfile(f"{d}/omask.bin", np.uint8).reshape(fine.shape)

        x["k"].tofile(f"{d}/k.bin")
        x["u"].tofile(f"{d}/src.bin")
        for bcc, bcs, diag in KERNGEN_CASES:
            run_ref(["kerngen", L, R_MIN, R_MAX, bcc, bcs, diag, d], d)
            out[f"kerngen_{bcc}{bcs}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)

        x["s"].tofile(f"{d}/src.bin")
        for treat, diag in LAPLACE_CASES:
            run_ref(["laplace", L, R_MIN, R_MAX, treat, diag, d], d)
            out[f"laplace_{treat}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)

        for bcc, bcs in STOKES_BCS:
            x["u"].tofile(f"{d}/src.bin")
            run_ref(["divergence", L, R_MIN, R_MAX, bcc, bcs, d], d)
            out[f"divergence_{bcc}{bcs}"] = np.fromfile(f"{d}/dst.bin").reshape(coarse.shape)
            x["p"].tofile(f"{d}/src.bin")
            run_ref(["gradient", L, R_MIN, R_MAX, bcc, bcs, d], d)
            out[f"gradient_{bcc}{bcs}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)

        x["uc"].tofile(f"{d}/src.bin")
        run_ref(["prolong", L, R_MIN, R_MAX, d], d)
        out["prolong"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)
        x["u"].tofile(f"{d}/src.bin")
        run_ref(["restrict", L, R_MIN, R_MAX, d], d)
        out["restrict"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + coarse.shape)

        x["pc"].tofile(f"{d}/src.bin")
        run_ref(["prolong_linear", L, R_MIN, R_MAX, d], d)
        out["prolong_linear"] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)
        x["s"].tofile(f"{d}/src.bin")
        run_ref(["restrict_linear", L, R_MIN, R_MAX, d], d)
        out["restrict_linear"] = np.fromfile(f"{d}/dst.bin").reshape(coarse.shape)

        x["k"].tofile(f"{d}/k.bin")
        x["s"].tofile(f"{d}/src.bin")
        for mode in KMASS_MODES:
            run_ref(["kmass", L, R_MIN, R_MAX, mode, d], d)
            out[f"kmass_{mode}"] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)
        for treat, diag, single in DIVKGRAD_CASES:
            run_ref(["divkgrad", L, R_MIN, R_MAX, treat, diag, single, d], d)
            out[f"divkgrad_{treat}{diag}{single}"] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)
        x["u"].tofile(f"{d}/src.bin")
        for bcc, bcs, diag in VLAPLACE_CASES:
            run_ref(["vlaplace", L, R_MIN, R_MAX, bcc, bcs, diag, d], d)
            out[f"vlaplace_{bcc}{bcs}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)
    path = os.path.join(HERE, f"ref_L{L}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
