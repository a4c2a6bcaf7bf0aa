"""The traversal plans (execution order, register forwarding and shared-memory stack positions
of the 4-state stack kernels) checked on the CPU: tests/cpp/plan_check.cpp includes
gems_b200/csrc/plan.h, plans random postorder op lists (whole trees, partly computed trees,
lists with a slot written twice) and executes each plan symbolically: every child read through
the plan must be what the caller's order gives, and the slots must end the same."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_plans_execute_like_the_callers_order(tmp_path):
    exe = str(tmp_path / "plan_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "gems_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "plan_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
    # whole-tree lists need at most a handful of stack positions (up to 600 taxa)
    depth = int(r.stdout.split("max_depth_full=")[1].split()[0])
    assert depth <= 8
