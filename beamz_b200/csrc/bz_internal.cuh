// Shared helpers of libbeamz_b200: status/error plumbing and launch utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/beamz_b200.h"

namespace bz {

// Records the message of a failed call for bz_last_error() (thread-local) and
// returns the code so call sites can `return fail(...)`.
int fail(int code, const char* fmt, ...);
void clear_error();

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Checks the launch that was just issued; maps a CUDA failure to BZ_ERR_CUDA.
int check_launch(const char* what);

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace bz

#define BZ_REQUIRE(cond, ...)                                   \
  do {                                                          \
    if (!(cond)) return ::bz::fail(BZ_ERR_INVALID, __VA_ARGS__); \
  } while (0)
