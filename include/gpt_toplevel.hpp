// gpt_toplevel.hpp -- drop-in replacement for the sqpSolve of gpu-pcg-tracking
// (toplevel.cuh:24-503) on top of the C ABI in gpt.h.
//
// A program that includes the reference's toplevel.cuh and calls
//     auto stats = sqpSolve<float>(state_size, control_size, knot_points, timestep,
//                                  d_eePos_traj, d_lambda, d_xu, d_dynMem_const,
//                                  config, rho, rho_reset);
// includes this header instead.  The returned tuple has the reference's
// element types (toplevel.cuh:502): PCG iterations per SQP iteration, linear
// solve times (empty: no per-solve host timing), solve time in microseconds,
// SQP iterations, the "time exit" flag (1 unless the rho > rho_max exit fired,
// as in toplevel.cuh:402) and PCG max-iteration flags.
//
// The reference's compile-time settings map onto gpt_problem_config /
// gpt_solver_config: QD_COST, R_COST, RHO_FACTOR, RHO_MAX, PCG_MAX_ITER and
// SQP_MAX_ITER are read here when defined.  The wall-clock cap
// SQP_MAX_TIME_US is not applied (solves are deterministic).
#pragma once

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "gpt.h"

#ifndef GPT_DEFAULT_QD_COST
#ifdef QD_COST
#define GPT_DEFAULT_QD_COST (QD_COST)
#else
#define GPT_DEFAULT_QD_COST 1e-4
#endif
#endif
#ifndef GPT_DEFAULT_R_COST
#ifdef R_COST
#define GPT_DEFAULT_R_COST (R_COST)
#else
#define GPT_DEFAULT_R_COST 1e-4
#endif
#endif

// GPU-PCG's configuration struct (toplevel.cuh:573-576 sets these three fields).
#ifndef GPT_HAVE_PCG_CONFIG
struct pcg_config {
    uint32_t pcg_block = 128;
    float pcg_exit_tol = 1e-5f;
    uint32_t pcg_max_iter = 167;
};
#endif

namespace gpt_dropin {

// One handle per (knot_points, timestep), created on first use and kept for
// the life of the process (the reference allocates per call).
inline gpt_handle *handle_for(uint32_t knot_points, float timestep)
{
    struct Entry {
        uint32_t n;
        float dt;
        gpt_handle *h;
    };
    static std::vector<Entry> cache;
    for (auto &e : cache)
        if (e.n == knot_points && e.dt == timestep) return e.h;
    gpt_problem_config pc;
    gpt_solver_config sc;
    gpt_default_problem_config(&pc);
    gpt_default_solver_config(&sc);
    pc.max_knot_points = knot_points;
    pc.timestep = timestep;
    pc.qd_cost = (float)GPT_DEFAULT_QD_COST;
    pc.r_cost = (float)GPT_DEFAULT_R_COST;
#ifdef RHO_FACTOR
    sc.rho_factor = (float)(RHO_FACTOR);
#endif
#ifdef RHO_MAX
    sc.rho_max = (float)(RHO_MAX);
#endif
#ifdef SQP_MAX_ITER
    sc.sqp_max_iter = (uint32_t)(SQP_MAX_ITER);
#endif
    gpt_handle *h = nullptr;
    if (gpt_create(&pc, &sc, &h) != GPT_OK) throw std::runtime_error(gpt_last_error());
    cache.push_back({knot_points, timestep, h});
    return h;
}

}  // namespace gpt_dropin

// Replacement for gato_plant::initializeDynamicsConstMem (the model is compiled in).
template <typename T>
void *gpt_dynamics_const_mem()
{
    static int token = 0;
    return &token;
}

template <typename T>
std::tuple<std::vector<int>, std::vector<double>, double, uint32_t, bool, std::vector<bool>> sqpSolve(
    uint32_t state_size, uint32_t control_size, uint32_t knot_points, float timestep, T *d_eePos_traj, T *d_lambda,
    T *d_xu, void * /*d_dynMem_const*/, pcg_config &config, T &rho, T rho_reset)
{
    static_assert(sizeof(T) == sizeof(float), "the B200 path computes in float32 (pcg_t = float)");
    if (state_size != 14 || control_size != 7) throw std::runtime_error("iiwa14: state 14, control 7");
    gpt_handle *h = gpt_dropin::handle_for(knot_points, timestep);
    gpt_solver_config sc;
    gpt_default_solver_config(&sc);
#ifdef SQP_MAX_ITER
    sc.sqp_max_iter = (uint32_t)(SQP_MAX_ITER);
#endif
#ifdef RHO_FACTOR
    sc.rho_factor = (float)(RHO_FACTOR);
#endif
#ifdef RHO_MAX
    sc.rho_max = (float)(RHO_MAX);
#endif
    sc.pcg_exit_tol = config.pcg_exit_tol;
    sc.pcg_max_iter = config.pcg_max_iter;
    if (gpt_set_solver_config(h, &sc) != GPT_OK) throw std::runtime_error(gpt_last_error());
    std::vector<uint32_t> iters(sc.sqp_max_iter);
    std::vector<uint8_t> maxit(sc.sqp_max_iter);
    gpt_sqp_stats st;
    float r = (float)rho;
    const auto t0 = std::chrono::steady_clock::now();
    const gpt_status s = gpt_sqp_solve(h, knot_points, (const float *)d_eePos_traj, (float *)d_lambda, (float *)d_xu,
                                       &r, (float)rho_reset, &st, iters.data(), maxit.data(), nullptr);
    const auto t1 = std::chrono::steady_clock::now();
    if (s != GPT_OK && s != GPT_ERR_NONFINITE) throw std::runtime_error(gpt_last_error());
    rho = (T)r;
    std::vector<int> pcg_iter_vec(iters.begin(), iters.begin() + st.sqp_iters);
    std::vector<bool> pcg_exit_vec(maxit.begin(), maxit.begin() + st.sqp_iters);
    const double us = std::chrono::duration<double, std::micro>(t1 - t0).count();
    const bool sqp_time_exit = (st.exit_flags & GPT_EXIT_RHO_MAX) == 0;
    return std::make_tuple(pcg_iter_vec, std::vector<double>{}, us, st.sqp_iters, sqp_time_exit, pcg_exit_vec);
}

// Replacement for track<T, return_type> (toplevel.cuh:507-510): the receding-horizon loop
// runs on the device (gpt_track).  Returns the reference's tuple: per-update SQP iterations
// (TIME_LINSYS 0), the per-shift tracking errors and the final tracking error.  The
// experiment bookkeeping arguments (start/goal indices, test_iter, output prefix) only named
// the reference's CSV dumps and are ignored.  SIMULATION_PERIOD is read when defined.
template <typename T, typename return_type>
std::tuple<std::vector<return_type>, std::vector<T>, T> track(
    uint32_t state_size, uint32_t control_size, uint32_t knot_points, const uint32_t traj_steps, float timestep,
    T *d_eePos_traj, T *d_xu_traj, T *d_xs, uint32_t /*start_state_ind*/, uint32_t /*goal_state_ind*/,
    uint32_t /*test_iter*/, T pcg_exit_tol, const std::string & /*test_output_prefix*/ = std::string())
{
    static_assert(sizeof(T) == sizeof(float), "the B200 path computes in float32 (pcg_t = float)");
    if (state_size != 14 || control_size != 7) throw std::runtime_error("iiwa14: state 14, control 7");
    gpt_handle *h = gpt_dropin::handle_for(knot_points, timestep);
    gpt_solver_config sc;
    gpt_default_solver_config(&sc);
#ifdef SQP_MAX_ITER
    sc.sqp_max_iter = (uint32_t)(SQP_MAX_ITER);
#endif
#ifdef RHO_FACTOR
    sc.rho_factor = (float)(RHO_FACTOR);
#endif
#ifdef RHO_MAX
    sc.rho_max = (float)(RHO_MAX);
#endif
#ifdef PCG_MAX_ITER
    sc.pcg_max_iter = (uint32_t)(PCG_MAX_ITER);
#endif
    sc.pcg_exit_tol = (float)pcg_exit_tol;
    if (gpt_set_solver_config(h, &sc) != GPT_OK) throw std::runtime_error(gpt_last_error());
    gpt_track_config tc;
    gpt_default_track_config(&tc);
#ifdef SIMULATION_PERIOD
    tc.sim_period_us = (float)(SIMULATION_PERIOD);
#endif
#if defined(REMOVE_JITTERS) && REMOVE_JITTERS
    tc.jitter_solves = 100;  // toplevel.cuh:584
#endif
    float *d_err = nullptr;
    uint32_t *d_log = nullptr;
    const uint32_t cap = tc.max_control_updates;
    // the reference allocates its loop buffers per call too (toplevel.cuh:545-566)
    if (cudaMalloc((void **)&d_err, sizeof(float) * traj_steps) != cudaSuccess ||
        cudaMalloc((void **)&d_log, sizeof(uint32_t) * cap) != cudaSuccess) {
        cudaFree(d_err);
        throw std::runtime_error("track: cudaMalloc failed");
    }
    gpt_track_stats st;
    const gpt_status s = gpt_track(h, knot_points, traj_steps, (const float *)d_eePos_traj, (const float *)d_xu_traj,
                                   (float *)d_xs, &tc, d_err, d_log, cap, &st, nullptr);
    std::vector<float> err(st.shifts);
    std::vector<uint32_t> log(st.control_updates < cap ? st.control_updates : cap);
    if (s == GPT_OK || s == GPT_ERR_NONFINITE) {
        cudaMemcpy(err.data(), d_err, sizeof(float) * err.size(), cudaMemcpyDeviceToHost);
        cudaMemcpy(log.data(), d_log, sizeof(uint32_t) * log.size(), cudaMemcpyDeviceToHost);
    }
    cudaFree(d_err);
    cudaFree(d_log);
    if (s != GPT_OK && s != GPT_ERR_NONFINITE) throw std::runtime_error(gpt_last_error());
    return std::make_tuple(std::vector<return_type>(log.begin(), log.end()), std::vector<T>(err.begin(), err.end()),
                           (T)st.final_tracking_error);
}
