"""The persistent kernel's launch plan on CPU: tests/plan_check.cu is built
against libedzt.so and runs lz_cut (the device-free part of lz_plan in
dmft-ed-zt_b200/csrc/lanczos.cu) on 3,000 seeded random job sets and grid
sizes, checking the tile lists, the cost-balanced CTA ranges, every job's run
of participating CTAs, the partial-sum slots and the column phase's slab
order (a bijection numbering the participants' tiles by round).  No GPU is
needed: lz_cut makes no CUDA call."""

import os
import shutil
import subprocess

import pytest

from conftest import PKG_DIR, ROOT

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not available")
def test_lz_cut_invariants(tmp_path):
    lib = os.path.join(PKG_DIR, "libedzt.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", PKG_DIR], check=True, capture_output=True)
    exe = str(tmp_path / "plan_check")
    subprocess.run([NVCC, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(PKG_DIR, "csrc"), os.path.join(ROOT, "tests", "plan_check.cu"),
                    "-o", exe, "-L", PKG_DIR, "-ledzt", "-lcudart", f"-Xlinker=-rpath,{PKG_DIR}"],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok 3000"), r.stdout
