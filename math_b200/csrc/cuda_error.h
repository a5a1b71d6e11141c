// Errors of CUDA runtime calls.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace nbpt
{
// A failed CUDA runtime call.  It carries the cudaError_t, so that callers
// decide by the code (cudaErrorMemoryAllocation: the device is full) and
// not by the wording of the message.
class CudaError final : public std::runtime_error
{
        cudaError_t code_;

public:
        CudaError(const std::string& what, const cudaError_t code)
                : std::runtime_error(what + ": " + cudaGetErrorString(code)),
                  code_(code)
        {
        }

        cudaError_t code() const noexcept
        {
                return code_;
        }
};

inline void cuda_check(const cudaError_t e, const char* what)
{
        if (e != cudaSuccess)
        {
                throw CudaError(what, e);
        }
}
} // namespace nbpt
