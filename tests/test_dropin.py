"""The C++ drop-in (include/gpt_toplevel.hpp) run on the GPU: a program written against the
reference's interface -- sqpSolve<float>(...) and track<float, uint32_t>(...) with the reference's
compile-time macros, toplevel.cuh:24-25,507-510 -- solves the reference's own trajectory
testfiles/0_0_traj.csv, and its outputs (the updated buffers and the returned tuples,
toplevel.cuh:502,819-823) equal the C ABI's gpt_sqp_solve / gpt_track called directly."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, ref_problem

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

PROGRAM = r"""
#define QD_COST 1e-4
#define R_COST 1e-4
#define RHO_FACTOR 1.2
#define RHO_MAX 10
#define SQP_MAX_ITER 8
#define PCG_MAX_ITER 167
#define SIMULATION_PERIOD 2000
#define REMOVE_JITTERS 0
#include "gpt_toplevel.hpp"
#include <cstdio>
#include <cstdlib>
#include <vector>

static std::vector<float> load(const char *path, size_t n)
{
    std::vector<float> v(n);
    FILE *f = std::fopen(path, "rb");
    if (!f || std::fread(v.data(), sizeof(float), n, f) != n) std::exit(3);
    std::fclose(f);
    return v;
}
static float *upload(const std::vector<float> &v)
{
    float *d = nullptr;
    if (cudaMalloc((void **)&d, sizeof(float) * v.size()) != cudaSuccess) std::exit(4);
    cudaMemcpy(d, v.data(), sizeof(float) * v.size(), cudaMemcpyHostToDevice);
    return d;
}
static std::vector<float> download(const float *d, size_t n)
{
    std::vector<float> v(n);
    cudaMemcpy(v.data(), d, sizeof(float) * n, cudaMemcpyDeviceToHost);
    return v;
}

int main(int argc, char **argv)
{
    const uint32_t N = (uint32_t)std::atoi(argv[1]), S = (uint32_t)std::atoi(argv[2]);
    const std::string dir = argv[3];
    const float dt = 0.015625f;
    // ---- one sqpSolve on the first N rows (runme.cu:145-161 layout)
    float *d_xu = upload(load((dir + "/xu.bin").c_str(), 21 * N - 7));
    float *d_goal = upload(load((dir + "/goal.bin").c_str(), 6 * N));
    float *d_lam = upload(std::vector<float>(14 * N, 0.f));
    pcg_config cfg;
    cfg.pcg_exit_tol = 1e-5f;
    cfg.pcg_max_iter = PCG_MAX_ITER;
    float rho = 1e-3f;
    auto t = sqpSolve<float>(14, 7, N, dt, d_goal, d_lam, d_xu, gpt_dynamics_const_mem<float>(), cfg, rho, 1e-3f);
    FILE *o = std::fopen((dir + "/solve.txt").c_str(), "w");
    std::fprintf(o, "%u %d %.9g\n", std::get<3>(t), (int)std::get<4>(t), rho);
    for (int v : std::get<0>(t)) std::fprintf(o, "%d ", v);
    std::fprintf(o, "\n");
    for (bool v : std::get<5>(t)) std::fprintf(o, "%d ", (int)v);
    std::fprintf(o, "\n");
    std::fclose(o);
    auto xu_out = download(d_xu, 21 * N - 7), lam_out = download(d_lam, 14 * N);
    FILE *b = std::fopen((dir + "/solve.bin").c_str(), "wb");
    std::fwrite(xu_out.data(), sizeof(float), xu_out.size(), b);
    std::fwrite(lam_out.data(), sizeof(float), lam_out.size(), b);
    std::fclose(b);
    // ---- track over S rows of the trajectory
    float *d_traj = upload(load((dir + "/traj.bin").c_str(), 21 * S));
    float *d_ee = upload(load((dir + "/ee.bin").c_str(), 6 * S));
    float *d_xs = upload(load((dir + "/xs.bin").c_str(), 14));
    auto r = track<float, uint32_t>(14, 7, N, S, dt, d_ee, d_traj, d_xs, 0, 0, 0, 1e-5f, "unused");
    FILE *q = std::fopen((dir + "/track.txt").c_str(), "w");
    std::fprintf(q, "%.9g\n", (double)std::get<2>(r));
    for (uint32_t v : std::get<0>(r)) std::fprintf(q, "%u ", v);
    std::fprintf(q, "\n");
    for (float v : std::get<1>(r)) std::fprintf(q, "%.9g ", (double)v);
    std::fprintf(q, "\n");
    std::fclose(q);
    auto xs_out = download(d_xs, 14);
    FILE *x = std::fopen((dir + "/xs_out.bin").c_str(), "wb");
    std::fwrite(xs_out.data(), sizeof(float), 14, x);
    std::fclose(x);
    return 0;
}
"""


def build_program(tmp_path):
    src = tmp_path / "dropin_run.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "dropin_run"
    lib_dir = os.path.join(ROOT, "gpu-pcg-tracking_b200")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
                    str(src), "-L", lib_dir, "-lgpt", "-L", os.path.join(cuda, "lib64"), "-lcudart",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    return exe


def test_cpp_dropin_runs_and_equals_the_c_abi(gpt, golden, tmp_path):
    N, S = 16, 40
    p = ref_problem(golden, N)
    traj = golden["traj_0_0"][1:1 + S].astype(np.float32)
    ee = golden["eepos_0_0"][1:1 + S].astype(np.float32)
    xs = traj[0, :14].copy()
    for name, arr in (("xu", p["xu"]), ("goal", p["goal"]), ("traj", traj.reshape(-1)), ("ee", ee.reshape(-1)),
                      ("xs", xs)):
        arr.astype(np.float32).tofile(tmp_path / f"{name}.bin")
    exe = build_program(tmp_path)
    subprocess.run([str(exe), str(N), str(S), str(tmp_path)], check=True, timeout=300)

    # the same calls through the C ABI (Python front end), same settings as the macros above
    sv = gpt.Solver(max_knot_points=N, timestep=0.015625, qd_cost=1e-4, r_cost=1e-4)
    try:
        sv.set_solver(sqp_max_iter=8, pcg_max_iter=167, pcg_exit_tol=1e-5, rho_factor=1.2, rho_max=10.0)
        xu = torch.as_tensor(p["xu"], device="cuda")
        lam = torch.zeros(14 * N, device="cuda")
        res = sv.sqp_solve(N, torch.as_tensor(p["goal"], device="cuda"), lam, xu, 1e-3)
        lines = (tmp_path / "solve.txt").read_text().split("\n")
        sqp_iter, time_exit, rho = lines[0].split()
        assert int(sqp_iter) == res.sqp_iters
        assert bool(int(time_exit)) == (not (res.stats["exit_flags"] & gpt.EXIT_RHO_MAX))
        assert np.float32(float(rho)) == np.float32(res.rho)
        assert [int(v) for v in lines[1].split()] == res.pcg_iters
        assert [bool(int(v)) for v in lines[2].split()] == res.pcg_exit
        out = np.fromfile(tmp_path / "solve.bin", np.float32)
        assert np.array_equal(out[:21 * N - 7], xu.cpu().numpy())
        assert np.array_equal(out[21 * N - 7:], lam.cpu().numpy())

        xs_d = torch.as_tensor(xs, device="cuda")
        log = torch.zeros(100000, dtype=torch.int32, device="cuda")
        errs, st = sv.track(N, torch.as_tensor(ee.reshape(-1), device="cuda"),
                            torch.as_tensor(traj.reshape(-1), device="cuda"), xs_d,
                            gpt.default_track_config(sim_period_us=2000.0), sqp_iters_log=log)
        tl = (tmp_path / "track.txt").read_text().split("\n")
        assert np.float32(float(tl[0])) == np.float32(st["final_tracking_error"])
        iters_cpp = [int(v) for v in tl[1].split()]
        assert len(iters_cpp) == st["control_updates"]
        assert iters_cpp == log[:st["control_updates"]].cpu().tolist()
        err_cpp = np.array([float(v) for v in tl[2].split()], np.float32)
        assert np.array_equal(err_cpp, errs.cpu().numpy().astype(np.float32))
        assert np.array_equal(np.fromfile(tmp_path / "xs_out.bin", np.float32), xs_d.cpu().numpy())
        assert st["shifts"] == S
    finally:
        sv.close()
