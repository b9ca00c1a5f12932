// Shared host-side helpers of libkcfd: error text, status codes, CUDA checks.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>

#include "kcfd.h"

namespace kcfd {

// Records the text of the last failure of this thread (read by kcfd_last_error).
void set_error(const char* fmt, ...);
const std::string& last_error();

}  // namespace kcfd

#define KCFD_REQUIRE(cond, ...)                 \
    do {                                        \
        if (!(cond)) {                          \
            ::kcfd::set_error(__VA_ARGS__);     \
            return KCFD_BAD_INPUT;              \
        }                                       \
    } while (0)

#ifdef __CUDACC__
#define KCFD_CUDA(call)                                                                     \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            ::kcfd::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return KCFD_CUDA_ERROR;                                                         \
        }                                                                                   \
    } while (0)
#endif
