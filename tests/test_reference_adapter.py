"""The drop-in boundary compiled against the reference's own headers (CPU, no GPU needed).

tests/adapter/reference_concepts.cpp static_asserts the reference's VectorLike / Block2VectorLike /
OperatorLike / SolverLike concepts (linalg/vector.hpp:8-52, linalg/operator.hpp:57-71,
linalg/solvers/solver.hpp:19-29) on the library's C++ layer, explicitly instantiates the reference's PCG,
Chebyshev, FGMRES and power iteration over the library's operators and vectors, and instantiates PCG over
the reference-side binding terraneo_b200/cpp/reference/epsilon_divdiv_kerngen_b200.hpp on the reference's
own VectorQ1Vec.  Compiled with g++ -fsyntax-only and the Kokkos include set of oracle/ref_build.  Skipped
where the reference's source tree is absent."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("TERRANEO_REFERENCE", "/root/reference")
CUDA_INC = "/usr/local/cuda/include"


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src", "terra")) or shutil.which("g++") is None
                    or not os.path.isdir(CUDA_INC), reason="reference sources, g++ or CUDA headers absent")
def test_reference_concepts_and_solvers_compile_over_the_library():
    kok = os.path.join(REF, "extern", "kokkos-4.6.01")
    rb = os.path.join(ROOT, "oracle", "ref_build")
    inc = [os.path.join(rb, "config"), os.path.join(kok, "core", "src"), os.path.join(kok, "containers", "src"),
           os.path.join(kok, "algorithms", "src"), os.path.join(kok, "simd", "src"),
           os.path.join(kok, "tpls", "desul", "include"), os.path.join(kok, "tpls", "mdspan", "include"),
           os.path.join(rb, "mpi_stub"), os.path.join(REF, "src"), os.path.join(REF, "src", "terra"),
           os.path.join(REF, "extern", "cli11-2.5.0"), CUDA_INC, os.path.join(ROOT, "include"),
           os.path.join(ROOT, "terraneo_b200", "cpp")]
    cmd = (["g++", "-std=c++20", "-fsyntax-only", "-w", "-fopenmp"] + [f"-I{p}" for p in inc]
           + ["-isystem", os.path.join(REF, "extern", "eigen-3.4.0"),
              os.path.join(ROOT, "tests", "adapter", "reference_concepts.cpp")])
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-4000:]
