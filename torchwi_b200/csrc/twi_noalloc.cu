// twi_noalloc.cu -- forward modelling of one shot without any device
// allocation, for callers that cannot allocate GPU memory: code running
// inside another framework's memory pool or a pre-sized arena, real-time or
// embedded hosts that forbid allocation after start-up, and callers that must
// not trigger the implicit synchronisation an allocation can cause.
//
// The wavefield scratch (padded velocity, four wavefield slots, wavelet,
// shot cells and the device error word) lives in one file-scope
// __device__ array of kNoAllocScratchBytes (32 MiB).  Every GPU that loads
// this library reserves that much for the lifetime of the process.  The
// caller passes only inputs and outputs.
//
// Rules that follow from the shared array:
//   * every call looks up the array's device address with
//     cudaGetSymbolAddress on the current device before it does anything
//     else, so the address is never stale (after a device reset the module
//     may load again at another address);
//   * every call reuses the same array and leaves its contents behind: the
//     call clears what must start at zero (the zero wavefield slot and the
//     error word) itself;
//   * two calls whose work overlaps on the GPU (different streams, or
//     different host threads on the same device) race on the array: issue
//     them on one stream or synchronise between them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "twi_b200.h"
#include "twi_kernels.h"
#include "twi_plan_internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;   // 32 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

int nofail(int code, const std::string& msg) {
    twi::set_last_error(msg);
    return code;
}

// Device address of g_noalloc_scratch on the current device, looked up on
// every call (host code must not use the symbol's name as an address).
int scratch_address(unsigned char** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
        return nofail(TWI_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    *out = static_cast<unsigned char*>(p);
    return TWI_OK;
}

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" int twi_fdm_forward_only_noalloc(float* frd, const float* vel, const float* w,
                                            int order, int dimx, int dimy, int nt, float h,
                                            float dt, float sx, float sy, float ry,
                                            void* stream) {
    using namespace twi;
    if (!frd || !vel || !w) return nofail(TWI_ERR_INVALID, "null array");
    int s = check_order(order);
    if (s != TWI_OK) return s;
    const int ne = order / 2, nx = dimx - order, nz = dimy - order;
    if (nx < 1 || nz < 1 || nt < 1)
        return nofail(TWI_ERR_INVALID, "dimx, dimy must exceed order and nt >= 1");
    if (!(h > 0.f) || !(dt > 0.f)) return nofail(TWI_ERR_INVALID, "h and dt must be positive");
    int host_coords[3];   // padded source row, source column, receiver row
    s = shot_cells(sx, sy, ry, h, nx, nz, ne, dimy, &host_coords[0], &host_coords[1], &host_coords[2]);
    if (s != TWI_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // layout inside the fixed scratch: velocity slot, 4 wavefield slots
    // (slot 0 stays zero), wavelet, shot cells, error word; sizes in 64 bits
    // so that no grid overflows before it is rejected
    const long long pitch_ll = ((long long)dimx + kTileX - 1) / kTileX * kTileX;
    const long long slot_ll = pitch_ll * dimy * 4;
    if (slot_ll > (long long)kNoAllocScratchBytes)
        return nofail(TWI_ERR_INVALID,
                      "grid too large for the no-allocation scratch: one wavefield of " +
                          std::to_string(dimx) + " x " + std::to_string(dimy) + " cells needs " +
                          std::to_string(slot_ll) + " bytes, the fixed scratch holds " +
                          std::to_string(kNoAllocScratchBytes));
    const int pitch = (int)pitch_ll;
    const size_t slot_bytes = (size_t)slot_ll;
    const size_t off_vpad = 0;
    const size_t off_fields = up256(off_vpad + slot_bytes);
    const size_t off_wav = up256(off_fields + 4 * slot_bytes);
    const size_t off_coords = up256(off_wav + (size_t)nt * 4);
    const size_t off_err = up256(off_coords + 3 * 4);
    const size_t need = up256(off_err + 4);
    if (need > kNoAllocScratchBytes)
        return nofail(TWI_ERR_INVALID,
                      "grid too large for the no-allocation scratch: needs " + std::to_string(need) +
                          " bytes, the fixed scratch holds " + std::to_string(kNoAllocScratchBytes) +
                          " (5 * roundup(dimx,128) * dimy * 4 + nt * 4 bytes plus a few hundred)");

    unsigned char* base = nullptr;
    s = scratch_address(&base);
    if (s != TWI_OK) return s;
    float* vpad = reinterpret_cast<float*>(base + off_vpad);
    float* fields = reinterpret_cast<float*>(base + off_fields);
    int* coords = reinterpret_cast<int*>(base + off_coords);
    int* err = reinterpret_cast<int*>(base + off_err);

#define NOALLOC_CUDA(expr)                                                                     \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess) return nofail(TWI_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

    // what must start at zero: the zero slot (u^{-1} = u^0) and the error word
    NOALLOC_CUDA(cudaMemsetAsync(fields, 0, slot_bytes, st));
    NOALLOC_CUDA(cudaMemsetAsync(err, 0, 4, st));
    NOALLOC_CUDA(cudaMemcpy2DAsync(vpad, (size_t)pitch * 4, vel, (size_t)dimx * 4, (size_t)dimx * 4,
                                   dimy, cudaMemcpyDeviceToDevice, st));
    NOALLOC_CUDA(cudaMemcpyAsync(base + off_wav, w, (size_t)nt * 4, cudaMemcpyDefault, st));
    NOALLOC_CUDA(cudaMemcpyAsync(coords, host_coords, sizeof(host_coords), cudaMemcpyHostToDevice, st));

    const LaunchShape shape{4, 4};
    const int TZ = 16, HZ = zhalo(order);
    CUtensorMap tm_u2, tm_u1, tm_vel;
    if ((s = make_map(&tm_u2, fields, dimx, dimy, 4, pitch, kBoxX, TZ + 2 * HZ)) != TWI_OK) return s;
    if ((s = make_map(&tm_u1, fields, dimx, dimy, 4, pitch, kTileX, TZ)) != TWI_OK) return s;
    if ((s = make_map(&tm_vel, vpad, dimx, dimy, 0, pitch, kTileX, TZ)) != TWI_OK) return s;
    NOALLOC_CUDA(prepare_step(order, true, shape));

    StepArgs a{};
    a.dimx = dimx, a.dimz = dimy, a.pitch = pitch, a.nx = nx, a.nz = nz;
    a.slot_elems = (long long)pitch * dimy;
    a.fields = fields;
    a.vel = vpad;
    a.nshots = 1, a.spc = 1;
    const float dt2 = dt * dt, h2 = h * h;
    a.dt2 = dt2, a.h2 = h2, a.dtoh2 = dt2 / h2, a.hdt = h * dt;
    a.cons = static_cast<float>(-2.0 / static_cast<double>(dt2));
    a.src_rc = coords;
    a.rec_row = coords + 2;
    a.wav = reinterpret_cast<const float*>(base + off_wav);
    a.wav_stride = 0;
    a.frd = frd;
    a.frd_stride = (long long)nt * nx;
    a.err = err;
    for (int it = 0; it < nt; ++it) {
        // u^k lives in slot 0 for k <= 0 and in slot 1 + k % 3 afterwards
        auto slot = [](long long k) { return k <= 0 ? 0 : 1 + (int)(k % 3); };
        a.it = it;
        a.prev_base = slot(it - 1), a.cur_base = slot(it), a.next_base = slot(it + 1);
        NOALLOC_CUDA(launch_step(order, true, kModeForward, shape, tm_u2, tm_u1, tm_vel, a, st));
    }
    int herr = 0;
    NOALLOC_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
    NOALLOC_CUDA(cudaStreamSynchronize(st));
#undef NOALLOC_CUDA
    if (herr) return nofail(TWI_ERR_DEVICE, "device error word " + std::to_string(herr));
    return TWI_OK;
}
