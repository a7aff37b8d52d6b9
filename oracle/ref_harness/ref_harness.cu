// ref_harness.cu -- the reference's own KKT, Schur, dz kernels and its qdldl
// helper, compiled unmodified from the reference's sources with the
// stand-ins in shims/ for its three empty submodules, behind a small C ABI.
//
// Test infrastructure only (a parity oracle): nothing in the product links
// it.  Built by oracle/Makefile (target `ref`) into oracle/_ref/, once per
// cost setting, because the reference takes QD_COST / R_COST as compile-time
// macros (iiwa_eepos_plant.cuh:60-64).
//
// Not exposed: compute_merit, ls_gato_compute_merit and sqpSolve (which calls
// both).  Their launches request less dynamic shared memory than the
// forward-dynamics call inside integratorError uses: forwardDynamics places
// its temporaries 1008 floats into the buffer (iiwa_eepos_plant.cuh:104) and
// direct_minv_inner / inverse_dynamics_inner reach about 750 floats past that
// (iiwa_eepos_grid.cuh:3753-4383), about 1815 floats from the start of the
// merit kernels' buffer, while get_merit_smem_size (merit.cuh:11-14) requests
// 1672 floats for compute_merit (and 1658 + 2N for the line-search kernel).
// On B200 the reference's compute_merit stopped with an illegal-address error.
//
// Calls follow the reference's own launch sites:
//   refh_form_kkt       gato_form_kkt launch of toplevel.cuh:256
//   refh_form_schur     form_schur (schur.cuh:545-559)
//   refh_form_schur_qdl form_schur_qdl (schur.cuh:528-543); refh_prep_csr: toplevel.cuh:178
//   refh_compute_dz     compute_dz (schur.cuh:562-566)
//   refh_qdldl_solve    qdl::qdldl_solve_schur (qdldl_helper.cuh:62-180), host arrays
#include <fstream>
#include <iostream>

#include "toplevel.cuh"

namespace {
void *g_dyn = nullptr;
void *dyn()
{
    if (!g_dyn) g_dyn = gato_plant::initializeDynamicsConstMem<float>();
    return g_dyn;
}
int finish()
{
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}
}  // namespace

extern "C" {

int refh_form_kkt(uint32_t N, float dt, int integrator, float *d_G, float *d_C, float *d_g, float *d_c,
                  float *d_eePos, float *d_xs, float *d_xu)
{
    const size_t smem = 2 * oldschur::get_kkt_smem_size<float>(14, 7);
    void *dm = dyn();
    if (integrator == 0)
        gato_form_kkt<float, 0><<<N, KKT_THREADS, smem>>>(14, 7, N, d_G, d_C, d_g, d_c, dm, dt, d_eePos, d_xs, d_xu);
    else
        gato_form_kkt<float, 1><<<N, KKT_THREADS, smem>>>(14, 7, N, d_G, d_C, d_g, d_c, dm, dt, d_eePos, d_xs, d_xu);
    return finish();
}

int refh_form_schur(uint32_t N, float rho, float *d_G, float *d_C, float *d_g, float *d_c, float *d_S, float *d_Pinv,
                    float *d_gamma)
{
    form_schur<float>(14, 7, N, d_G, d_C, d_g, d_c, d_S, d_Pinv, d_gamma, rho);
    return finish();
}

int refh_form_schur_qdl(uint32_t N, float rho, float *d_G, float *d_C, float *d_g, float *d_c, float *d_val,
                        float *d_gamma)
{
    form_schur_qdl<float>(14, 7, N, d_G, d_C, d_g, d_c, d_val, d_gamma, rho);
    return finish();
}

int refh_prep_csr(uint32_t N, int32_t *d_col_ptr, int32_t *d_row_ind)
{
    prep_csr<<<N, 64>>>(14, N, d_col_ptr, d_row_ind);
    return finish();
}

int refh_compute_dz(uint32_t N, float *d_Ginv, float *d_C, float *d_g, float *d_lambda, float *d_dz)
{
    compute_dz<float>(14, 7, N, d_Ginv, d_C, d_g, d_lambda, d_dz);
    return finish();
}

int refh_qdldl_solve(uint32_t N, int32_t *h_col_ptr, int32_t *h_row_ind, float *h_val, float *h_gamma,
                     float *h_lambda)
{
    const QDLDL_int An = 14 * N;
    std::vector<QDLDL_int> etree(An), Lnz(An), Lp(An + 1), iwork(3 * An);
    std::vector<QDLDL_float> D(An), Dinv(An), fwork(An);
    std::vector<QDLDL_bool> bwork(An);
    const QDLDL_int sumLnz = QDLDL_etree(An, h_col_ptr, h_row_ind, iwork.data(), Lnz.data(), etree.data());
    if (sumLnz < 0) return -1;
    std::vector<QDLDL_int> Li(sumLnz);
    std::vector<QDLDL_float> Lx(sumLnz);
    qdl::qdldl_solve_schur(An, h_col_ptr, h_row_ind, h_val, h_gamma, h_lambda, Lp.data(), Li.data(), Lx.data(),
                           D.data(), Dinv.data(), Lnz.data(), etree.data(), bwork.data(), iwork.data(), fwork.data());
    return 0;
}

}  // extern "C"
