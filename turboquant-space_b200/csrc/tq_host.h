// tq_host.h -- host-side internals shared by the C ABI translation units
// (tq_capi.cu, tq_serve.cu): the space object and error/device helpers.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "turboquant_b200.h"
#include "tq_internal.h"
#include "tq_tables.h"

struct tq_space {
    size_t dim = 0, D = 0, packed_bytes = 0, code_size = 0;
    int bits = 0, levels = 0, num_threads = 1, device = -1;
    bool padded = false;
    uint64_t rot_seed = 0, qjl_seed = 0;
    std::vector<float> centroids, boundaries, rot_signs, qjl_signs;
    tq::QuantLut qlut;
    tq::Params P{};
    tq::DevTables T{};
    void *dev_block = nullptr;  // single device allocation holding the tables
    std::mutex host_mu;         // serialises the host-pointer entry points
    cudaStream_t host_stream[2] = {nullptr, nullptr};
    // scan kernel timer (tq_space_scan_timer): event pairs around each 1->N
    // scan launch while enabled
    std::mutex timer_mu;
    bool timer_on = false;
    size_t timer_used = 0;
    std::vector<cudaEvent_t> timer_events;  // 2 per recorded launch
};

namespace tq {

// Record a message for tq_last_error() and return `st`.
tq_status fail(tq_status st, const char *fmt, ...);
// TQ_ERR_OUT_OF_MEMORY for allocation failures, TQ_ERR_CUDA otherwise.
tq_status cuda_fail(cudaError_t e, const char *what);
// TQ_ERR_NO_DEVICE unless the space is bound to a device.
tq_status need_device(const tq_space *sp);

#define TQ_CUDA(call, what)                                       \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return ::tq::cuda_fail(e_, what);  \
    } while (0)

// Makes `dev` current for the scope and restores the caller's device.
struct DeviceGuard {
    int prev = -1, want = -1;
    explicit DeviceGuard(int dev) : want(dev) {
        cudaGetDevice(&prev);
        if (prev != want) cudaSetDevice(want);
    }
    ~DeviceGuard() {
        if (prev >= 0 && prev != want) cudaSetDevice(prev);
    }
};

}  // namespace tq
