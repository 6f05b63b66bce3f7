// context.h -- the sarbp_ctx handle behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>

#include "runner.h"
#include "sarbp_b200.h"

struct sarbp_ctx {
    sarbp::DeviceInfo dev;
    std::unique_ptr<sarbp::Runner> runner;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    sarbp::DeviceBuffer io;  // device copies of host-API inputs and outputs
    sarbp::DeviceBuffer out_aux;
    sarbp::DeviceBuffer resize_buf;  // resize weights, bounds and intermediates
    std::map<std::string, sarbp_opts> tuned;  // autotuner results by job-set key
    // host-buffer entry points: copies in, second compute stream, copies out,
    // and the events that pipeline row slabs between them
    static constexpr int kMaxSlabs = 12;
    cudaStream_t copy_in = nullptr, aux = nullptr, copy_out = nullptr;
    cudaEvent_t ev_out = nullptr;
    cudaEvent_t ev_ready[kMaxSlabs] = {}, ev_done[kMaxSlabs] = {};
};

namespace sarbp {
// makes the context's device current (SARBP_ERR_INVALID for a NULL ctx)
int ctx_set_device(sarbp_ctx *ctx);
}  // namespace sarbp
