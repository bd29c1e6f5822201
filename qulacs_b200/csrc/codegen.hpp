// Run-time compiled kernels (csrc/pass_codegen.cpp): CUDA C source compiled for sm_100a with NVRTC,
// loaded with cudaLibraryLoadData and cached by source text for the life of the process.
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace qs {

// Kernel `name` (extern "C") of `src`; *compile_ms receives the compile time (0 on a cache hit).
// QS_ERR_NOT_SUPPORTED when NVRTC cannot be loaded.  The handle stays valid until exit.
int nvrtc_kernel(const std::string& src, const char* name, void** kernel, double* compile_ms);
// cudaLaunchKernel of such a kernel, its dynamic shared-memory limit raised to `smem_limit` bytes once
// per device.
int launch_nvrtc_kernel(void* kernel, dim3 grid, dim3 block, void** args, size_t smem, size_t smem_limit,
    cudaStream_t st, const char* what);

}  // namespace qs
