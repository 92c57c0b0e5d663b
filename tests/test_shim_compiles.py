"""The maintainer-side shim (tests/shim/ginkgo_b200_cuda_shim.cpp: Ginkgo's
CUDA kernel functions defined over the C ABI, and the Cg solver hook)
compiled against the reference's own headers, kernel declarations and
instantiation macros: a signature check of the drop-in boundary.  Needs the
reference source tree (GINKGO_REFERENCE_DIR); skipped where it is absent."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("GINKGO_REFERENCE_DIR", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "include", "ginkgo")),
                    reason="reference source tree not available")
def test_shim_compiles_against_reference_headers(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    obj = tmp_path / "shim.o"
    cmd = [cxx, "-std=c++17", "-c", "-o", str(obj),
           "-I", os.path.join(ROOT, "tests", "shim", "include"),
           "-I", os.path.join(REF, "include"), "-I", REF,
           "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "shim", "ginkgo_b200_cuda_shim.cpp")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    # the kernel functions libginkgo_cuda would export are defined here
    nm = shutil.which("nm")
    if nm:
        syms = subprocess.run([nm, "-C", str(obj)], capture_output=True, text=True).stdout
        for name in ("gko::kernels::cuda::csr::spmv<double, double, double, int>",
                     "gko::kernels::cuda::csr::spmv<float, double, double, int>",
                     "gko::kernels::cuda::csr::advanced_spmv<double, float, float, int>",
                     "gko::kernels::cuda::csr::spgemm<double, int>",
                     "gko::kernels::cuda::ell::spmv<double, double, double, int>",
                     "gko::kernels::cuda::sellp::compute_slice_sets<int>"):
            assert name in syms, name
