// twi_diag.cu -- diagnostics of the library's failure path.
//
// Every wait in the step kernels is bounded: when a copy never lands, the
// CTA raises the device error word, waits (bounded) for its other copies and
// returns, so the host sees TWI_ERR_DEVICE and the context stays usable.
// twi_check_wait_timeout exercises exactly that path without any fault: its
// kernel waits on a shared-memory barrier that nothing ever arrives at.
// twi_check_counter_wait does the same for the counter wait of chained and
// persistent launches: a counter that never reaches its target, or an error
// word that another CTA has already raised.
#include <cuda_runtime.h>

#include <string>

#include "twi_b200.h"
#include "twi_persist.cuh"
#include "twi_ptx.cuh"

namespace twi {
void set_last_error(const std::string& msg);
}

namespace {

__device__ int g_diag_err;
__device__ unsigned g_diag_count;

__global__ void counter_wait_kernel(unsigned long long limit_ns, int preset) {
    // the counter stays 0: a target of 1 is never reached
    if (threadIdx.x == 0) {
        if (preset) atomicOr(&g_diag_err, 4);   // another CTA's error, raised first
        twi::wait_count_for(&g_diag_count, 1u, &g_diag_err, limit_ns);
    }
}

__global__ void wait_timeout_kernel(unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        twi::mbar_init(&bar, 1);
        twi::fence_barrier_init();
    }
    __syncthreads();
    const bool ok = twi::mbar_wait_for(&bar, 0, limit_ns);   // phase 0 never completes
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(&g_diag_err, 1);
}

int dfail(int code, const std::string& msg) {
    twi::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" int twi_check_wait_timeout(int limit_us, float* elapsed_ms, void* stream) {
    if (limit_us < 1 || limit_us > 2000000) return dfail(TWI_ERR_INVALID, "limit_us must be in [1, 2e6]");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int* err = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&err), g_diag_err) != cudaSuccess)
        return dfail(TWI_ERR_CUDA, "error word address lookup failed");
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return dfail(TWI_ERR_CUDA, "event create failed");
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return dfail(TWI_ERR_CUDA, "event create failed");
    }
    int host = 0;
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaEventRecord(e0, st);
    if (e == cudaSuccess) {
        wait_timeout_kernel<<<1, 32, 0, st>>>(1000ull * (unsigned long long)limit_us);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return dfail(TWI_ERR_CUDA, std::string("wait-timeout check: ") + cudaGetErrorString(e));
    if (elapsed_ms) *elapsed_ms = ms;
    if (!(host & 1)) return dfail(TWI_ERR_DEVICE, "the bounded wait did not report running out");
    return TWI_OK;
}

// The counter wait of chained and persistent launches.  preset_error = 0: the
// wait must run out after `limit_us` and raise bit 1 of the error word;
// preset_error = 1: the word holds another CTA's error (bit 2) beforehand and
// the wait must leave without raising bit 1.
extern "C" int twi_check_counter_wait(int limit_us, int preset_error, float* elapsed_ms, void* stream) {
    if (limit_us < 1 || limit_us > 2000000) return dfail(TWI_ERR_INVALID, "limit_us must be in [1, 2e6]");
    if (preset_error != 0 && preset_error != 1) return dfail(TWI_ERR_INVALID, "preset_error must be 0 or 1");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int* err = nullptr;
    unsigned* count = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&err), g_diag_err) != cudaSuccess ||
        cudaGetSymbolAddress(reinterpret_cast<void**>(&count), g_diag_count) != cudaSuccess)
        return dfail(TWI_ERR_CUDA, "diagnostic word address lookup failed");
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return dfail(TWI_ERR_CUDA, "event create failed");
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return dfail(TWI_ERR_CUDA, "event create failed");
    }
    int host = 0;
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaEventRecord(e0, st);
    if (e == cudaSuccess) {
        counter_wait_kernel<<<1, 32, 0, st>>>(1000ull * (unsigned long long)limit_us, preset_error);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return dfail(TWI_ERR_CUDA, std::string("counter-wait check: ") + cudaGetErrorString(e));
    if (elapsed_ms) *elapsed_ms = ms;
    if (preset_error ? host != 4 : host != 2)
        return dfail(TWI_ERR_DEVICE, "the counter wait did not end as designed (error word " + std::to_string(host) + ")");
    return TWI_OK;
}
