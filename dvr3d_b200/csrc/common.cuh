// common.cuh -- shared device helpers for the DVR3DRJZ kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dvr3d {

// Number of kernels this library has launched (host side; read by the solve entry
// points to report the launches of one solve).
extern long long g_kernel_launches;
#define DVR3D_COUNT_LAUNCH(k) (::dvr3d::g_kernel_launches += (k))

// Kernel attributes such as cudaFuncAttributeMaxDynamicSharedMemorySize are per device:
// launchers that raise them keep one "done" flag per device ordinal below this bound (and set
// the attribute on every launch for ordinals beyond it).
constexpr int kMaxAttrDevices = 64;

// Device-side error flags written by kernels (never __trap): the host reads them after a
// stage and turns them into DVR3D_ERR_* codes.
enum DeviceErr : int {
    kDevOk = 0,
    kDevBarrierTimeout = 1,   // a grid barrier wait ran past its iteration limit
    kDevNoConv = 2,           // an iterative device solver hit its iteration limit
    kDevBadPes = 3,           // non-finite potential value
    kDevOverflow = 4,         // a selection exceeded the caller's MAX2D / MAX3D
    kDevNotPosDef = 5         // a Cholesky pivot was not positive
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum; `red` is shared scratch of >= 32 doubles. All threads get the result.
__device__ __forceinline__ double block_sum(double v, double *red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = (threadIdx.x < (unsigned)nw) ? red[threadIdx.x] : 0.0;
    if (wid == 0) {
        t = warp_sum(t);
        if (lane == 0) red[0] = t;
    }
    __syncthreads();
    double r = red[0];
    __syncthreads();
    return r;
}

// Grid-wide barrier for kernels launched with cudaLaunchCooperativeKernel (all CTAs
// co-resident). Sense by generation counter. The wait is bounded: after `limit` polls the
// CTA records kDevBarrierTimeout in *err and returns false; callers must then leave the
// kernel. Returns false as well when another CTA already flagged an error.
struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

__device__ __forceinline__ bool grid_sync(GridBarrier *b, int *err, unsigned long long limit = (1ull << 26)) {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        volatile unsigned int *vgen = &b->gen;
        const unsigned int g = *vgen;
        __threadfence();
        const unsigned int arrived = atomicAdd(&b->count, 1u);
        if (arrived == gridDim.x * gridDim.y * gridDim.z - 1) {
            b->count = 0;
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            unsigned long long spins = 0;
            while (*vgen == g) {
                if (++spins > limit) {
                    atomicExch(err, (int)kDevBarrierTimeout);
                    break;
                }
                if (spins > 4096) __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = (*(volatile int *)err == 0);
    }
    __syncthreads();
    return s_ok != 0;
}

// Grid barrier on a counter that only grows: barrier number e of a sequence completes when
// the counter reaches (e + 1) * gridDim; `target` carries the running count (start it at the
// arrivals made by earlier launches on the same counter, which is zeroed once before them).
// No reset step, so the last arrival releases everybody at once. Bounded like grid_sync (a
// limit of 0 means the default 2^26 polls); a CTA that sees another's error flag while
// waiting returns false as well.
__device__ __forceinline__ bool grid_sync_counted(unsigned int *count, unsigned int &target, int *err,
                                                  unsigned long long limit = (1ull << 26)) {
    if (limit == 0) limit = 1ull << 26;
    __syncthreads();
    __shared__ int s_okc;
    target += gridDim.x * gridDim.y * gridDim.z;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(count, 1u);
        volatile unsigned int *vc = count;
        unsigned long long spins = 0;
        int ok = 1;
        while (*vc < target) {
            ++spins;
            if ((spins & 1023ull) == 0 && *(volatile int *)err != 0) {
                ok = 0;
                break;
            }
            if (spins > limit) {
                atomicExch(err, (int)kDevBarrierTimeout);
                ok = 0;
                break;
            }
            if (spins > 4096) __nanosleep(32);
        }
        __threadfence();
        s_okc = ok;
    }
    __syncthreads();
    return s_okc != 0;
}

}  // namespace dvr3d
