// prog_noalloc.cu -- gral_prog_check_speeds_noalloc: the unrealistic-wind-speed check of a solved
// flow field on caller-owned device arrays, with no device allocation.
//
// Who needs it: a caller that keeps the flow field on the GPU after the solve (for the dispersion
// step that follows, or to write GRAL's flow-field files from device memory) and cannot call
// cudaMalloc at that point -- because its device memory is already committed to its own pool
// (a caching allocator that holds the rest of HBM, where a cudaMalloc fails or forces that pool
// to release), or because cudaMalloc/cudaFree would synchronise the whole device while its other
// solver streams run.  Such a caller cannot create a solver context, so this entry point takes
// plain device pointers in the host layout and keeps its scratch in a fixed static array.
//
// The check itself is the one gral_prog_store runs (k_postcheck): per ADVDOM column, levels
// 1..min(NKK-1, KKART+vert_cells_ff), counts |U| or |V| above 55 m/s or above 10*GESCHW_MAX,
// |W| above 20 m/s or 10*GESCHW_MAX, plus non-finite values.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "gral_prog.h"

namespace {

// Scratch: per-row partial counts (4 ints per row i) after a 256-byte header holding the
// completion ticket (word 0) and the final counts (words 4..7).  Fixed size, held by every device
// that loads the library until the process exits.
constexpr int kHeaderWords = 64;
constexpr int kScratchWords = kHeaderWords + 4 * GRAL_NOALLOC_MAX_ROWS;
static __device__ __align__(256) unsigned int g_speed_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned int *g_addr[kMaxDevices] = {};   // device address of g_speed_scratch per device

constexpr int kThreads = 256;

__device__ __forceinline__ int warp_sum(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One block per row i (1..nii); warps stride over j, lanes over k.  Each block stores its row's
// four counts into the scratch, the last block to finish (completion ticket) sums the rows in
// ascending order into the header and re-arms the ticket.
__global__ void __launch_bounds__(kThreads) k_check_speeds(int nii, int njj, int nkk, int vcff, float limit,
                                                           const float *__restrict__ uk,
                                                           const float *__restrict__ vk,
                                                           const float *__restrict__ wk,
                                                           const uint8_t *__restrict__ advdom,
                                                           const int16_t *__restrict__ kkart,
                                                           unsigned int *scratch) {
    __shared__ int red[kThreads / 32][4];
    __shared__ bool last;
    const int i = blockIdx.x + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nj2 = njj + 2, nk2 = nkk + 2;
    int cu = 0, cv = 0, cw = 0, cn = 0;
    for (int j = 1 + warp; j <= njj; j += kThreads / 32) {
        const size_t c = (size_t)i * nj2 + j;
        if (advdom[c] != 1) continue;
        const int ktop = min(nkk - 1, (int)kkart[c] + vcff);
        const size_t base = c * nk2;
        for (int k = 1 + lane; k <= ktop; k += 32) {
            const float u = uk[base + k], v = vk[base + k], w = wk[base + k];
            cu += (fabsf(u) > 55.f || fabsf(u) > limit);
            cv += (fabsf(v) > 55.f || fabsf(v) > limit);
            cw += (fabsf(w) > 20.f || fabsf(w) > limit);
            cn += (!isfinite(u) || !isfinite(v) || !isfinite(w));
        }
    }
    cu = warp_sum(cu); cv = warp_sum(cv); cw = warp_sum(cw); cn = warp_sum(cn);
    if (lane == 0) { red[warp][0] = cu; red[warp][1] = cv; red[warp][2] = cw; red[warp][3] = cn; }
    __syncthreads();
    if (threadIdx.x < 4) {
        int s = 0;
        for (int w = 0; w < kThreads / 32; ++w) s += red[w][threadIdx.x];
        scratch[kHeaderWords + 4 * (i - 1) + threadIdx.x] = (unsigned int)s;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(&scratch[0], 1u) == (unsigned int)(nii - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < 4) {
        const volatile unsigned int *rows = scratch + kHeaderWords;
        unsigned int s = 0;
        for (int r = 0; r < nii; ++r) s += rows[4 * r + threadIdx.x];
        scratch[4 + threadIdx.x] = s;
    }
    if (threadIdx.x == 0) scratch[0] = 0u;
}

// True for memory the kernel on device `dev` may read: device memory of `dev` itself, or managed
// memory.  Device memory of another GPU is refused: without peer access a kernel reading it faults.
bool on_device(const void *p, int dev) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();   // clears only the error of this lookup (none was pending on entry)
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    return at.type == cudaMemoryTypeDevice && at.device == dev;
}

}  // namespace

extern "C" int gral_prog_check_speeds_noalloc(int32_t nii, int32_t njj, int32_t nkk, int32_t vert_cells_ff,
                                              double geschw_max, const float *uk, const float *vk,
                                              const float *wk, const uint8_t *advdom, const int16_t *kkart,
                                              int32_t counts[4], void *stream) {
    if (!counts || nii < 1 || njj < 1 || nkk < 2 || vert_cells_ff < 0) return GRAL_EINVAL;
    if (nii > GRAL_NOALLOC_MAX_ROWS) return GRAL_ETOOLARGE;
    if (!uk || !vk || !wk || !advdom || !kkart) return GRAL_EINVAL;
    // an error left pending by the caller's own work is reported, not cleared: the error checks
    // below then see only what this call causes
    if (cudaPeekAtLastError() != cudaSuccess) return GRAL_ECUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return GRAL_ENODEV;
    }
    if (dev < 0 || dev >= kMaxDevices) return GRAL_ENODEV;
    if (!on_device(uk, dev) || !on_device(vk, dev) || !on_device(wk, dev) || !on_device(advdom, dev) ||
        !on_device(kkart, dev))
        return GRAL_EINVAL;
    unsigned int *scratch = nullptr;
    {
        // first call on this device: resolve the device address of the static scratch (the
        // current device is the one the kernel will run on).  The address is kept for the life of
        // the process; cudaDeviceReset of this device would make it stale.
        std::lock_guard<std::mutex> lk(g_mutex);
        if (!g_addr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_speed_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return GRAL_ECUDA;
            }
            g_addr[dev] = static_cast<unsigned int *>(p);
        }
        scratch = g_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the ticket and the result words must start at zero; the per-row words are all overwritten
    if (cudaMemsetAsync(scratch, 0, 8 * sizeof(unsigned int), st) != cudaSuccess) return GRAL_ECUDA;
    const float limit = (float)(10 * geschw_max);
    k_check_speeds<<<nii, kThreads, 0, st>>>(nii, njj, nkk, vert_cells_ff, limit, uk, vk, wk, advdom, kkart,
                                             scratch);
    if (cudaGetLastError() != cudaSuccess) return GRAL_ECUDA;
    unsigned int out[4] = {0, 0, 0, 0};
    if (cudaMemcpyAsync(out, scratch + 4, sizeof(out), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return GRAL_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return GRAL_ECUDA;
    for (int q = 0; q < 4; ++q) counts[q] = (int32_t)out[q];
    return GRAL_OK;
}
