// Error plumbing and library info of the C ABI.
#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "common.cuh"

namespace {
thread_local std::string g_err;
}

extern "C" void uva_set_error(const char* msg) { g_err = msg ? msg : ""; }

int uva_cuda_status(cudaError_t e, const char* where) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s: CUDA error %d (%s)", where, static_cast<int>(e), cudaGetErrorString(e));
    uva_set_error(buf);
    return UVA_E_CUDA;
}

extern "C" const char* uva_last_error(void) { return g_err.c_str(); }

extern "C" int uva_version(void) { return 1; }
