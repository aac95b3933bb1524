// internal.h — definitions shared by the engine's translation units
// (engine.cu: single cases; batch.cu: batches of cases).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/lbm_ddf.h"

struct lbm_case {
    lbm_params p;
    lbm_derived d;
    int64_t nodes = 0, ps = 0;
    int64_t step = 0;
    bool swapped = false;
    bool initialised = false;
    bool rest_phi = false;               // next step uses phi = 0.5 (reference rest state)
    // f and g: separate arrays of 27 rows (FP64, FP32), or for 16-bit
    // storage one array of (f, g) pairs with g = f + one element
    void *f = nullptr, *g = nullptr, *phip = nullptr;
    int32_t kernel = LBM_KERNEL_AUTO;    // step kernel choice
    int32_t collision = LBM_COLLISION_BGK;
    lbm_batch *batch = nullptr;          // the batch the case is a member of
    int *d_err = nullptr;                // set by a step kernel whose bulk-copy wait timed out
    uint32_t debug_extra_tx = 0;         // lbm_debug_row_wait_extra_bytes (0: off)
    double *partial = nullptr;           // obs partial sums
    lbm_observables *d_obs = nullptr;    // reduced observables (device)
    int obs_blocks = 0;                  // partial rows (most reduction blocks)
    int sms = 148;                       // SM count of the case's device
    double *obs_rows = nullptr;          // lbm_step_observed: per-warp rows + chunk partials
    lbm_observables *obs_series = nullptr;
    int obs_series_cap = 0;
};

namespace lbm_internal {

// 16-bit storage keeps f and g interleaved (lattice.cuh elem_stride)
inline bool interleaved(const lbm_case *c) {
    return c->p.storage == LBM_STORE_F16S || c->p.storage == LBM_STORE_BF16S;
}

// records `msg` for lbm_last_error() on this thread and returns `code`
int fail(int code, const std::string &msg);
size_t store_bytes(int storage);
int64_t round_up(int64_t v, int64_t m);
void derive(const lbm_params *p, lbm_derived *d);
int check_params(const lbm_params *p);
// drops a case that is being destroyed from its batch (batch.cu)
void batch_forget(lbm_batch *b, lbm_case *c);
// enqueues the observables reduction of c's current state into dst (device
// memory) on st, without synchronising (engine.cu)
int enqueue_observables(const lbm_case *c, lbm_observables *dst, cudaStream_t st);
// enqueues one node-kernel step of c from layout `swapped` on st; the host
// state (step count, layout flag) is the caller's to advance (engine.cu)
int enqueue_case_step(const lbm_case *c, bool swapped, cudaStream_t st);

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace lbm_internal

#define CUDA_TRY(call)                                                                                   \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return lbm_internal::fail(LBM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
