/*
 * Host definitions of the CUDA runtime calls that the reference's GPU-aligner
 * driver code makes (test infrastructure only; see host_operators.cpp).  The
 * oracle's reference build runs that driver code on the CPU: one "device",
 * streams that are plain handles, and nothing asynchronous, because every
 * stand-in operator finishes before it returns.
 */
#include <cuda_runtime_api.h>

#include <atomic>

namespace {
std::atomic<unsigned long> g_next_stream(1);
}

extern "C" {

cudaError_t cudaGetDeviceCount(int *count) {
  *count = 1;
  return cudaSuccess;
}

cudaError_t cudaSetDevice(int device) { return device == 0 ? cudaSuccess : cudaErrorInvalidDevice; }

cudaError_t cudaDeviceReset(void) { return cudaSuccess; }

const char *cudaGetErrorString(cudaError_t error) {
  return error == cudaSuccess ? "no error" : "host stand-in error";
}

cudaError_t cudaStreamCreate(cudaStream_t *stream) {
  *stream = reinterpret_cast<cudaStream_t>(g_next_stream.fetch_add(1));
  return cudaSuccess;
}

cudaError_t cudaStreamDestroy(cudaStream_t) { return cudaSuccess; }

cudaError_t cudaStreamQuery(cudaStream_t) { return cudaSuccess; }

cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }

}  // extern "C"
