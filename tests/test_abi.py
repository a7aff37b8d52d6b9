"""The C-ABI library loads and exports every symbol include/gpt.h declares;
host-side logic that needs no GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def header_symbols():
    src = open(os.path.join(ROOT, "include", "gpt.h")).read()
    return sorted(set(re.findall(r"\b(gpt_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(gpt):
    L = gpt.lib()
    declared = header_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(gpt.EXPORTED) == declared


def test_default_configs_match_reference_settings(gpt):
    pc = gpt.default_problem_config()
    sc = gpt.default_solver_config()
    assert (pc.state_size, pc.control_size) == (14, 7)
    assert abs(pc.timestep - 1 / 64) < 1e-9 and pc.integrator == 0 and pc.mu == 10.0
    assert sc.sqp_max_iter == 40 and abs(sc.rho_factor - 1.2) < 1e-6 and sc.rho_max == 10.0
    assert abs(sc.rho_min - 1e-3) < 1e-9


def test_create_rejects_bad_sizes(gpt):
    L = gpt.lib()
    h = C.c_void_p()
    pc = gpt.default_problem_config(state_size=12)
    sc = gpt.default_solver_config()
    assert L.gpt_create(C.byref(pc), C.byref(sc), C.byref(h)) == 1  # BAD_ARG before touching the GPU
    pc = gpt.default_problem_config(max_knot_points=4096)
    assert L.gpt_create(C.byref(pc), C.byref(sc), C.byref(h)) == 1
    assert L.gpt_create(None, C.byref(sc), C.byref(h)) == 1


def test_prep_csr_matches_oracle_pattern(gpt, oracle):
    for N in (2, 3, 8):
        cp, ri = gpt.prep_csr(N)
        ocp, ori = oracle.csc_pattern(N)
        np.testing.assert_array_equal(cp, ocp)
        np.testing.assert_array_equal(ri, ori)


def test_no_gpu_means_no_silent_fallback(gpt):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(gpt.GptError) as ei:
        gpt.Solver(max_knot_points=8)
    assert ei.value.status == 3  # NO_DEVICE


def test_problem_generator_is_seeded(problem_mod):
    a = problem_mod.make_problem(16, 3)
    b = problem_mod.make_problem(16, 3)
    c = problem_mod.make_problem(16, 4)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert np.abs(a["goal"] - c["goal"]).max() > 1e-3
    assert a["xu"].shape == (21 * 16 - 7,) and a["goal"].shape == (6 * 16,)
    np.testing.assert_array_equal(a["xu"][:14], a["xs"])
    assert np.abs(a["xu"][7:14]).max() == 0.0  # x_s has zero velocity
    batch = problem_mod.make_batch([4, 8], seed0=3)
    np.testing.assert_array_equal(batch["xu"][:21 * 4 - 7], problem_mod.make_problem(4, 3)["xu"])


def test_cpp_dropin_header_compiles_and_links(tmp_path):
    """include/gpt_toplevel.hpp (the sqpSolve and track drop-ins) compiles with the
    reference's macros defined and links against libgpt.so."""
    import subprocess
    src = tmp_path / "dropin.cpp"
    src.write_text(
        '#define QD_COST 1e-4\n#define R_COST 1e-4\n#define RHO_FACTOR 1.2\n#define RHO_MAX 10\n'
        '#define SIMULATION_PERIOD 2000\n#define REMOVE_JITTERS 1\n'
        '#include "gpt_toplevel.hpp"\n'
        'int main(){ pcg_config cfg; float rho = 1e-3f;\n'
        '  if (0) { auto t = sqpSolve<float>(14, 7, 32, 0.015625f, (float*)0, (float*)0, (float*)0,\n'
        '              gpt_dynamics_const_mem<float>(), cfg, rho, 1e-3f); (void)t;\n'
        '    auto r = track<float, uint32_t>(14, 7, 32, 666, 0.015625f, (float*)0, (float*)0, (float*)0,\n'
        '              0, 0, 0, 1e-5f, "out"); (void)r; }\n'
        '  gpt_problem_config pc; gpt_default_problem_config(&pc); return pc.state_size == 14 ? 0 : 1; }\n')
    exe = tmp_path / "dropin"
    lib_dir = os.path.join(ROOT, "gpu-pcg-tracking_b200")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
                    str(src), "-L", lib_dir, "-lgpt", "-L", os.path.join(cuda, "lib64"), "-lcudart",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    assert subprocess.run([str(exe)]).returncode == 0
