// common.h — host-side error reporting shared by the C-ABI translation units.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>

#include <cuda_runtime.h>

#include "../../include/strelka_b200.h"

namespace sb {

// Message of the most recent failure on the calling thread.
std::string& last_error();

inline int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    last_error() = buf;
    return code;
}

inline int cuda_fail(cudaError_t e, const char* what)
{
    return fail(e == cudaErrorMemoryAllocation ? STRELKA_ERR_OUT_OF_MEMORY : STRELKA_ERR_CUDA, "%s: %s (%d)", what,
                cudaGetErrorString(e), (int)e);
}

#define SB_CUDA_TRY(expr)                                  \
    do {                                                   \
        cudaError_t sb_err_ = (expr);                      \
        if (sb_err_ != cudaSuccess) return sb::cuda_fail(sb_err_, #expr); \
    } while (0)

}  // namespace sb
