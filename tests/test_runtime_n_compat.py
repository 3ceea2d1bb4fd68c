"""The drop-in for the reference's runtime-n solver header (src/nvrtc/nvrtc_solver.hpp), CPU side.

include/sbg/compat/nvrtc/nvrtc_solver.hpp re-declares the reference's public API
(NvrtcGeneigSolver, TuningMode, CacheMode, ModuleCacheKey, make_streams, destroy_streams) over
the C ABI.  Two checks:

* A caller using every member of that API compiles against the header and links against
  libsbg_geneig.so.
* When the reference tree is present, its own runtime-n tests compile unchanged against the
  header: tests/test_nvrtc_n54.cpp, test_nvrtc_multiN.cpp, test_autotune_n32.cpp,
  test_autotune_n54.cpp, test_bpb_sweep_n54.cpp, test_blockdim_n32.cpp, test_cache_n54.cpp and
  test_cache_invalidation.cpp.  The oracle/Makefile target `nvrtc-drivers` builds them and links
  them against libsbg_geneig.so in place of the reference's NVRTC build.

Running any of them needs a GPU.
"""
from __future__ import annotations

import os
import subprocess

import pytest

from conftest import REPO

INC = os.path.join(REPO, "include")
LIB_DIR = os.path.join(REPO, "sunny-batched-geneig_b200", "sbg")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")

CALLER = r'''
#include "nvrtc/nvrtc_solver.hpp"
#include <cstdio>
int main(int argc, char**) {
    if (argc > 1) {                        // never taken here: only compiled and linked
        NvrtcGeneigSolver s(54, 0, 0, 0, TuningMode::Autotune, CacheMode::NoDisk);
        std::vector<CUstream> st = make_streams(2);
        CUdeviceptr p = 0;
        s.launch(p, p, p, p, p, 0, st[0]);
        s.launch_chunked(p, p, p, p, p, 0, 1, 2, st);
        dim3 b = s.block_dim();
        std::printf("%d %d %u %u %d %d %d %s %f %s %s\n", s.matrix_size(), s.batches_per_block(), b.x,
                    s.shared_mem_bytes(), s.autotuned_block_dim_x(), int(s.was_autotuned()),
                    int(s.autotune_sweep_ran()), s.cache_layer_used(), s.acquire_module_ms(),
                    NvrtcGeneigSolver::cache_dir().c_str(), NvrtcGeneigSolver::cubin_path(ModuleCacheKey{}).c_str());
        destroy_streams(st);
    }
    return 0;
}
'''


def _lib():
    so = os.path.join(LIB_DIR, "libsbg_geneig.so")
    if not os.path.exists(so):
        pytest.skip("libsbg_geneig.so not built")
    return so


def test_every_member_compiles_and_links(tmp_path):
    _lib()
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    exe = tmp_path / "caller"
    cmd = ["g++", "-std=c++17", "-Wall", "-Werror", f"-I{os.path.join(INC, 'sbg', 'compat')}", f"-I{INC}",
           f"-I{CUDA}/include", str(src), "-o", str(exe), f"-L{LIB_DIR}", "-l:libsbg_geneig.so",
           f"-Wl,-rpath,{LIB_DIR}", f"-L{CUDA}/lib64/stubs", "-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr


def test_reference_runtime_n_tests_compile_unchanged():
    _lib()
    from oracle import oracle as O
    ref = O.reference_dir()
    if not os.path.isdir(os.path.join(ref, "tests")):
        pytest.skip("the reference tree is not present")
    r = subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), f"SBG_REFERENCE_DIR={ref}", "nvrtc-drivers"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for name in ("test_nvrtc_n54", "test_nvrtc_multiN", "test_autotune_n32", "test_autotune_n54",
                 "test_bpb_sweep_n54", "test_blockdim_n32", "test_cache_n54", "test_cache_invalidation"):
        exe = os.path.join(REPO, "oracle", "_ref", name)
        assert os.access(exe, os.X_OK), name
