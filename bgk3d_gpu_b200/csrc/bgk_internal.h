// Internal helpers shared by the library's translation units.
#pragma once
#include <cstdarg>
#include <cuda_runtime.h>

namespace bgk {
// Record a formatted message as the calling thread's last error; returns code.
int set_error(int code, const char* fmt, ...);
// cudaGetLastError after a launch, recorded as an error when it failed.
int check_launch(const char* what);
// Block shape for one-thread-per-node sweeps over (i, j) rows: TX x TY = 256.
dim3 row_block(int l);
}  // namespace bgk
