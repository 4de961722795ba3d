// Host-side helpers shared by the C-ABI translation units: error recording, CUDA checks.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "../../include/ldg_b200.h"

namespace ldg {

void set_error(const std::string& msg);
void clear_error();

// Checks a CUDA call; on failure records the message and returns LDG_ERR_CUDA from the caller.
#define LDG_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t e__ = (call);                                                               \
        if (e__ != cudaSuccess) {                                                               \
            ::ldg::set_error(std::string(#call) + ": " + cudaGetErrorString(e__));              \
            return LDG_ERR_CUDA;                                                                \
        }                                                                                       \
    } while (0)

// Checks the last launch.
#define LDG_LAUNCHED(name)                                                                      \
    do {                                                                                        \
        cudaError_t e__ = cudaGetLastError();                                                   \
        if (e__ != cudaSuccess) {                                                               \
            ::ldg::set_error(std::string("launch of ") + (name) + ": " + cudaGetErrorString(e__)); \
            return LDG_ERR_CUDA;                                                                \
        }                                                                                       \
    } while (0)

#define LDG_REQUIRE(cond, code, msg)                                                            \
    do {                                                                                        \
        if (!(cond)) {                                                                          \
            ::ldg::set_error(msg);                                                              \
            return (code);                                                                      \
        }                                                                                       \
    } while (0)

// Makes a handle's device current for the scope of an entry point and restores the caller's
// device afterwards, so handles created on different GPUs can be used from one thread.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        int cur = -1;
        if (dev < 0 || cudaGetDevice(&cur) != cudaSuccess || cur == dev) return;
        if (cudaSetDevice(dev) == cudaSuccess) prev = cur;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

}  // namespace ldg
