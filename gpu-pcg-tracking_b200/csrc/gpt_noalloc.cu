// gpt_noalloc.cu -- the line-search merit entry point for callers that cannot
// allocate device memory (gpt_ls_compute_merit_noalloc in include/gpt.h).
//
// Who needs it: a real-time control loop that allocates everything once at
// start-up and may not call cudaMalloc (or wait on an allocator's locks)
// between control ticks, and a plug-in that runs inside a host framework whose
// own pool owns every device allocation.  gpt_ls_compute_merit needs a
// gpt_handle, and gpt_create allocates the handle's workspace; this variant
// needs no handle.
//
// Its scratch -- the per-knot merits of the 8 step sizes, reduced to the 8
// outputs -- lives in the file-scope array below, so the library holds
// 16 KiB on every GPU that loads it, until the process exits.  The caller
// still passes every input and the output.  Every call on a device shares the
// array and leaves its contents behind; each call writes every entry it then
// reads, so nothing has to start at zero.  Two calls whose kernels overlap on
// the GPU (on different streams, or from different host threads) race on the
// array.
#include <mutex>

#include "gpt_common.cuh"
#include "gpt_internal.h"

using namespace gpt;

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;

// 8 step sizes x GPT_NOALLOC_MAX_KNOTS knots of per-knot merits (16 KiB).
// In host code this name is a host-side stand-in for the symbol, not a device
// address: the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) float g_ls_knot_merit[NUM_ALPHAS * GPT_NOALLOC_MAX_KNOTS];

struct DeviceScratch {
    float *knot_merit = nullptr;
    int num_sms = 0;
};

std::mutex g_setup_mutex;
DeviceScratch g_scratch[NOALLOC_MAX_DEVICES];

// Once per device, with that device current: the device address of the
// scratch array and the SM count.  Runs inside the first call on each device.
gpt_status device_scratch(DeviceScratch *out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return record_error(GPT_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return record_error(GPT_ERR_BAD_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceScratch &d = g_scratch[dev];
    if (!d.knot_merit) {
        float *ptr = nullptr;
        e = cudaGetSymbolAddress((void **)&ptr, g_ls_knot_merit);
        if (e != cudaSuccess) return record_error(GPT_ERR_CUDA, cudaGetErrorString(e));
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return record_error(GPT_ERR_CUDA, cudaGetErrorString(e));
        d.num_sms = sms;
        d.knot_merit = ptr;
    }
    *out = d;
    return GPT_OK;
}

}  // namespace

extern "C" gpt_status gpt_ls_compute_merit_noalloc(const gpt_problem_config *pc, uint32_t N, const float *d_xs,
                                                   const float *d_xu, const float *d_goal, const float *d_dz,
                                                   float *d_merits, gpt_stream_t stream)
{
    if (!pc || !d_xs || !d_xu || !d_goal || !d_dz || !d_merits) return record_error(GPT_ERR_BAD_ARG, "null argument");
    if (pc->state_size != NS || pc->control_size != NC)
        return record_error(GPT_ERR_BAD_ARG, "state_size must be 14 and control_size 7");
    if (N < 2 || N > GPT_NOALLOC_MAX_KNOTS)
        return record_error(GPT_ERR_BAD_ARG,
                            "knot_points out of range: the no-allocation merit takes 2..GPT_NOALLOC_MAX_KNOTS (512)");
    DeviceScratch d;
    const gpt_status st = device_scratch(&d);
    if (st != GPT_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    BatchView bv;
    bv.B = 1;
    bv.total_knots = (int)N;
    bv.knot_off = nullptr;
    bv.knot_inst = nullptr;
    bv.st = nullptr;
    SolverParams unused{};
    cudaError_t e = launch_merit(bv, problem_params(*pc), NUM_ALPHAS, d_xu, d_dz, d_goal, d_xs, d.knot_merit,
                                 d.num_sms, s);
    if (e == cudaSuccess)
        e = launch_accept(bv, 2, unused, d.knot_merit, nullptr, nullptr, d_merits, nullptr, d.num_sms, s);
    if (e != cudaSuccess) return record_error(GPT_ERR_CUDA, cudaGetErrorString(e));
    return GPT_OK;
}
