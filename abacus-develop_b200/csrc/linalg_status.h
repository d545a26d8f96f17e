// Status checks of the vendor linear-algebra calls (cuBLAS, cuSOLVER): a failed call becomes a b200::Error
// with the call's text and status, which the C-ABI turns into a status code.
#pragma once
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <string>

#include "common.h"

#define B200_CUBLAS(call)                                                                                       \
    do {                                                                                                        \
        cublasStatus_t st_ = (call);                                                                            \
        if (st_ != CUBLAS_STATUS_SUCCESS)                                                                       \
            throw ::b200::Error(::b200::kCublasError, std::string(#call) + " failed with status " +           \
                                                          std::to_string(int(st_)));                           \
    } while (0)

#define B200_CUSOLVER(call)                                                                                     \
    do {                                                                                                        \
        cusolverStatus_t st_ = (call);                                                                          \
        if (st_ != CUSOLVER_STATUS_SUCCESS)                                                                     \
            throw ::b200::Error(::b200::kCusolverError, std::string(#call) + " failed with status " +         \
                                                            std::to_string(int(st_)));                         \
    } while (0)
