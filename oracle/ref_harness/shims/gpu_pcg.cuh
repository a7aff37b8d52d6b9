// gpu_pcg.cuh -- stand-in for the GPU-PCG submodule header that
// toplevel.cuh:16 includes (.gitmodules:1-3, empty in the reference tree).
// The harness builds the reference with PCG_SOLVE=0, its qdldl path, so only
// the configuration struct sqpSolve's signature names is needed (fields set
// at toplevel.cuh:573-576).  Test infrastructure only.
#pragma once
#include <cstdint>

struct pcg_config {
    uint32_t pcg_block = 128;
    float pcg_exit_tol = 1e-5f;
    uint32_t pcg_max_iter = 167;
};
