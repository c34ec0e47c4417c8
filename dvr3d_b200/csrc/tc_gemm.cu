// tc_gemm.cu -- split-BF16 GEMMs on the 5th-generation tensor cores (sm_100a).
//
// One CTA computes one 128 x BN output tile:
//   * warp 0 / lane 0 streams K in 64-element steps with TMA (cp.async.bulk.tensor, 128-byte
//     swizzle, no multicast) into a ring of shared-memory stages, one mbarrier per stage for
//     "full" (transaction bytes) and one for "empty";
//   * warp 1 / lane 0 issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) on each stage, the
//     accumulator living in tensor memory (BN columns of 128 lanes), and frees the stage with
//     tcgen05.commit on its "empty" barrier; a last commit signals "done";
//   * all four warps then drain tensor memory (tcgen05.ld, warp w owns lanes 32w..32w+31 =
//     tile rows) and apply the epilogue in FP64.
// With two slices per operand a stage holds A_hi, A_lo, B_hi, B_lo of the same K step and the
// three BF16x3 products are issued back to back into the same accumulator, so every operand
// byte is read from HBM once.
//
// Every wait is bounded in time (globaltimer); a wait that runs out sets the error flag, the
// CTA stops issuing, waits (bounded again) for its own copies and products in flight, frees
// its tensor memory and leaves its tile unwritten.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "common.cuh"
#include "tc_gemm.cuh"
#include "tcgen05.cuh"

namespace dvr3d {

namespace {

constexpr int kBM = 128;       // tile rows = UMMA M = tensor-memory lanes
constexpr int kBK = 64;        // K elements per stage: one 128-byte swizzle row per tile row
constexpr int kUK = 16;        // K of one kind::f16 MMA
constexpr int kThreads = 128;  // 4 warps
constexpr unsigned long long kDefaultWaitNs = 4000000000ull;

template <int BN>
struct TcCfg {
    static constexpr int kA = kBM * kBK * 2;  // bytes of one A slice tile (16 KB)
    static constexpr int kB = BN * kBK * 2;   // bytes of one B slice tile
    static constexpr int kStage = 2 * kA + 2 * kB;
    static constexpr int kStages = (192 * 1024) / kStage;
    static constexpr int kSmem = kStages * kStage + 1024;  // + slack to align the ring to 1 KB
    static_assert(kStages >= 2, "at least double buffering");
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "UMMA N / TMEM allocation");
};

struct TcMaps {
    CUtensorMap a[2];
    CUtensorMap b[2];
};

struct TcArgs {
    int M, N, K, nslice;
    double *C;
    long long cm, cn;
    double alpha, beta;
    const int *g;
    const double *T;
    int ldt;
    const double *e2;
    double *H;
    __nv_bfloat16 *H_hi, *H_lo;
    long long ldh;
    int *err;
    unsigned long long wait_ns;
};

using tc::fence_after;
using tc::fence_before;
using tc::global_ns;
using tc::mbar_expect_tx;
using tc::mbar_init;
using tc::mbar_wait;
using tc::smem_u32;
using tc::tma_load_2d;
using tc::umma_commit;

// Shared-memory matrix descriptor of a K-major tile written by TMA with the 128-byte swizzle:
// rows of 128 bytes, 8-row groups 1024 bytes apart (stride byte offset), version 1, layout
// SWIZZLE_128B. Advancing the start address by 32 bytes selects the next K = 16 slice.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

// 32 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    tc::tmem_ld32(taddr, r);
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void split_store(__nv_bfloat16 *hi, __nv_bfloat16 *lo, long long idx, double v) {
    const __nv_bfloat16 h = __double2bfloat16(v);
    hi[idx] = h;
    lo[idx] = __double2bfloat16(v - (double)__bfloat162float(h));
}

template <int BN, int EPI>
__global__ void __launch_bounds__(kThreads, 1) tc_gemm_kernel(const __grid_constant__ TcMaps maps, const TcArgs p) {
    using Cfg = TcCfg<BN>;
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long bar_full[Cfg::kStages];
    __shared__ __align__(8) unsigned long long bar_empty[Cfg::kStages];
    __shared__ __align__(8) unsigned long long bar_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_abort;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long wait_ns = p.wait_ns;
    const unsigned long long t_end = global_ns() + wait_ns;

    int ti, tj;
    if (EPI == kTcAssemble) {  // lower tile pair (ti >= tj) from the linear block index
        const long long t = blockIdx.x;
        ti = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
        while ((long long)ti * (ti + 1) / 2 > t) --ti;
        while ((long long)(ti + 1) * (ti + 2) / 2 <= t) ++ti;
        tj = (int)(t - (long long)ti * (ti + 1) / 2);
    } else {
        ti = blockIdx.x;
        tj = blockIdx.y;
    }
    const int m0 = ti * kBM, n0 = tj * BN;

    const uint32_t ring = (smem_u32(tc_smem) + 1023u) & ~1023u;
    const uint32_t full0 = smem_u32(&bar_full[0]), empty0 = smem_u32(&bar_empty[0]), done = smem_u32(&bar_done);
    if (threadIdx.x == 0) {
        for (int s = 0; s < Cfg::kStages; ++s) {
            mbar_init(full0 + 8u * s, 1);
            mbar_init(empty0 + 8u * s, 1);
        }
        mbar_init(done, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"((uint32_t)BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;

    const int nk = (p.K + kBK - 1) / kBK;
    const int ns = p.nslice;
    const uint32_t tx_bytes = (uint32_t)(ns * (Cfg::kA + Cfg::kB));
    if (threadIdx.x == 0) {
        // ---- TMA producer
        int it = 0;
        bool ok = true;
        for (; it < nk; ++it) {
            const int s = it % Cfg::kStages;
            const uint32_t ph = (uint32_t)(it / Cfg::kStages) & 1u;
            if (!mbar_wait(empty0 + 8u * s, ph ^ 1u, t_end) || *(volatile int *)&s_abort) {
                ok = false;
                break;
            }
            const uint32_t sa = ring + (uint32_t)(s * Cfg::kStage), sb = sa + 2u * Cfg::kA;
            mbar_expect_tx(full0 + 8u * s, tx_bytes);
            const int kx = it * kBK;
            for (int sl = 0; sl < ns; ++sl) {
                tma_load_2d(sa + (uint32_t)(sl * Cfg::kA), &maps.a[sl], full0 + 8u * s, kx, m0);
                tma_load_2d(sb + (uint32_t)(sl * Cfg::kB), &maps.b[sl], full0 + 8u * s, kx, n0);
            }
        }
        if (!ok) {
            atomicExch(&s_abort, 1);
            if (p.err) atomicExch(p.err, (int)kDevBarrierTimeout);
        }
        // the copies issued last (one per stage at most) have landed before the CTA goes on
        for (int j = (it > Cfg::kStages ? it - Cfg::kStages : 0); j < it; ++j)
            mbar_wait(full0 + 8u * (j % Cfg::kStages), (uint32_t)(j / Cfg::kStages) & 1u, t_end + wait_ns);
    } else if (threadIdx.x == 32) {
        // ---- MMA issuer
        const uint32_t idesc = (1u << 4)                         // D: FP32
                               | (1u << 7) | (1u << 10)           // A, B: BF16
                               | ((uint32_t)(BN >> 3) << 17)      // N
                               | ((uint32_t)(kBM >> 4) << 24);    // M
        const int nterm = ns == 1 ? 1 : 3;
        bool ok = true;
        for (int it = 0; it < nk; ++it) {
            const int s = it % Cfg::kStages;
            const uint32_t ph = (uint32_t)(it / Cfg::kStages) & 1u;
            if (!mbar_wait(full0 + 8u * s, ph, t_end) || *(volatile int *)&s_abort) {
                ok = false;
                break;
            }
            fence_after();
            const uint32_t sa = ring + (uint32_t)(s * Cfg::kStage), sb = sa + 2u * Cfg::kA;
            for (int t = 0; t < nterm; ++t) {
                // terms: A_hi B_hi, A_hi B_lo, A_lo B_hi
                const uint64_t da = sw128_desc(sa + (t == 2 ? (uint32_t)Cfg::kA : 0u));
                const uint64_t db = sw128_desc(sb + (t == 1 ? (uint32_t)Cfg::kB : 0u));
#pragma unroll
                for (int kk = 0; kk < kBK / kUK; ++kk)
                    umma_bf16(tmem, da + (uint64_t)(2 * kk), db + (uint64_t)(2 * kk), idesc,
                              (it | t | kk) != 0 ? 1u : 0u);
            }
            umma_commit(empty0 + 8u * s);
        }
        if (!ok) {
            atomicExch(&s_abort, 1);
            if (p.err) atomicExch(p.err, (int)kDevBarrierTimeout);
        }
        umma_commit(done);  // arrives once every product issued above has completed
    }
    __syncwarp();

    // ---- epilogue: tensor memory -> FP64
    const bool got = mbar_wait(done, 0u, t_end + wait_ns);
    fence_after();
    const bool warp_ok = __all_sync(0xffffffffu, got && *(volatile int *)&s_abort == 0);
    if (!got && lane == 0 && p.err) atomicExch(p.err, (int)kDevBarrierTimeout);
    if (warp_ok) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            if (n0 + c0 >= p.N) break;  // uniform over the warp
            float v[32];
            tmem_ld32(tmem + lane_base + (uint32_t)c0, v);
            if (row >= p.M) continue;
            if (EPI == kTcStore) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = n0 + c0 + j;
                    if (col >= p.N) continue;
                    double *pc = p.C + (long long)row * p.cm + (long long)col * p.cn;
                    double val = p.alpha * (double)v[j];
                    if (p.beta != 0.0) val += p.beta * *pc;
                    *pc = val;
                }
            } else {
                const int gi = p.g[row];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = n0 + c0 + j;
                    if (col >= p.N || (ti == tj && col > row)) continue;
                    double val = (double)v[j] * p.T[(long long)p.g[col] * p.ldt + gi];
                    if (col == row) val += p.e2[row];
                    const long long a = (long long)col * p.ldh + row, b = (long long)row * p.ldh + col;
                    if (p.H) {
                        p.H[a] = val;
                        p.H[b] = val;
                    } else {
                        split_store(p.H_hi, p.H_lo, a, val);
                        split_store(p.H_hi, p.H_lo, b, val);
                    }
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
    }
}

__global__ void split_bf16_kernel(const double *__restrict__ X, long long ldx, int R, int K,
                                  __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo, long long ldo) {
    for (int r = blockIdx.y; r < R; r += gridDim.y) {
        const double *x = X + (long long)r * ldx;
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
            const double v = x[k];
            const __nv_bfloat16 h = __double2bfloat16(v);
            hi[(long long)r * ldo + k] = h;
            if (lo) lo[(long long)r * ldo + k] = __double2bfloat16(v - (double)__bfloat162float(h));
        }
    }
}

__global__ void split_sum_kernel(const __nv_bfloat16 *__restrict__ hi, const __nv_bfloat16 *__restrict__ lo,
                                 long long lds, int n, double *__restrict__ S) {
    for (int c = blockIdx.y; c < n; c += gridDim.y)
        for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
            const long long e = (long long)c * lds + r;
            S[e] = (double)__bfloat162float(hi[e]) + (double)__bfloat162float(lo[e]);
        }
}

using tc::EncodeTiledFn;
using tc::encode_tiled;

// Row-major rows x K BF16 matrix (row stride ld elements), boxes of 64 K-elements x box_rows.
bool make_map(EncodeTiledFn fn, CUtensorMap &m, const __nv_bfloat16 *ptr, int rows, int K, long long ld,
              int box_rows) {
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(ptr), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, int EPI>
cudaError_t launch_cfg(const TcMaps &maps, const TcArgs &a, dim3 grid, cudaStream_t st) {
    using Cfg = TcCfg<BN>;
    static bool attr_done[kMaxAttrDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= kMaxAttrDevices || !attr_done[dev]) {
        e = cudaFuncSetAttribute(tc_gemm_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::kSmem);
        if (e != cudaSuccess) return e;
        if (dev < kMaxAttrDevices) attr_done[dev] = true;
    }
    DVR3D_COUNT_LAUNCH(1);
    tc_gemm_kernel<BN, EPI><<<grid, kThreads, Cfg::kSmem, st>>>(maps, a);
    return cudaGetLastError();
}

bool aligned16(const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; }

}  // namespace

cudaError_t launch_split_bf16(const double *X, long long ldx, int R, int K, __nv_bfloat16 *hi, __nv_bfloat16 *lo,
                              long long ldo, cudaStream_t st) {
    if (R <= 0 || K <= 0) return cudaSuccess;
    if (!X || !hi || ldx < K || ldo < K) return cudaErrorInvalidValue;
    const int bx = (K + 255) / 256;
    dim3 grid((unsigned)(bx < 16 ? bx : 16), (unsigned)(R < 65535 ? R : 65535));
    DVR3D_COUNT_LAUNCH(1);
    split_bf16_kernel<<<grid, 256, 0, st>>>(X, ldx, R, K, hi, lo, ldo);
    return cudaGetLastError();
}

cudaError_t launch_split_sum(const __nv_bfloat16 *hi, const __nv_bfloat16 *lo, long long lds, int n, double *S,
                             cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (!hi || !lo || !S || lds < n) return cudaErrorInvalidValue;
    const int bx = (n + 255) / 256;
    dim3 grid((unsigned)(bx < 16 ? bx : 16), (unsigned)(n < 65535 ? n : 65535));
    DVR3D_COUNT_LAUNCH(1);
    split_sum_kernel<<<grid, 256, 0, st>>>(hi, lo, lds, n, S);
    return cudaGetLastError();
}

cudaError_t launch_tc_gemm(const TcGemm &p, cudaStream_t st) {
    if (p.M <= 0 || p.N <= 0) return cudaSuccess;
    if (p.K <= 0 || (p.nslice != 1 && p.nslice != 2)) return cudaErrorInvalidValue;
    if (!p.A_hi || !p.B_hi || !aligned16(p.A_hi) || !aligned16(p.B_hi)) return cudaErrorInvalidValue;
    if (p.nslice == 2 && (!p.A_lo || !p.B_lo || !aligned16(p.A_lo) || !aligned16(p.B_lo)))
        return cudaErrorInvalidValue;
    if (p.lda % 8 != 0 || p.ldb % 8 != 0 || p.lda < p.K || p.ldb < p.K) return cudaErrorInvalidValue;
    if (p.epilogue == kTcStore && !p.C) return cudaErrorInvalidValue;
    if (p.epilogue == kTcAssemble &&
        (p.M != p.N || !p.g || !p.T || !p.e2 || p.ldh < p.N || (!p.H && (!p.H_hi || !p.H_lo))))
        return cudaErrorInvalidValue;
    if (p.epilogue != kTcStore && p.epilogue != kTcAssemble) return cudaErrorInvalidValue;
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return cudaErrorNotSupported;
    const int BN = (p.epilogue == kTcAssemble || p.N > 64) ? 128 : 64;
    TcMaps maps;
    std::memset(&maps, 0, sizeof(maps));
    for (int sl = 0; sl < p.nslice; ++sl) {
        if (!make_map(fn, maps.a[sl], sl ? p.A_lo : p.A_hi, p.M, p.K, p.lda, kBM)) return cudaErrorInvalidValue;
        if (!make_map(fn, maps.b[sl], sl ? p.B_lo : p.B_hi, p.N, p.K, p.ldb, BN)) return cudaErrorInvalidValue;
    }
    TcArgs a{};
    a.M = p.M;
    a.N = p.N;
    a.K = p.K;
    a.nslice = p.nslice;
    a.C = p.C;
    a.cm = p.cm;
    a.cn = p.cn;
    a.alpha = p.alpha;
    a.beta = p.beta;
    a.g = p.g;
    a.T = p.T;
    a.ldt = p.ldt;
    a.e2 = p.e2;
    a.H = p.H;
    a.H_hi = p.H_hi;
    a.H_lo = p.H_lo;
    a.ldh = p.ldh;
    a.err = p.err;
    a.wait_ns = p.wait_ns ? p.wait_ns : kDefaultWaitNs;
    if (p.epilogue == kTcAssemble) {
        const long long tiles = (p.N + kBM - 1) / kBM;
        const long long nblk = tiles * (tiles + 1) / 2;
        if (nblk > 0x7fffffffLL) return cudaErrorInvalidValue;
        return launch_cfg<128, kTcAssemble>(maps, a, dim3((unsigned)nblk), st);
    }
    const int tm = (p.M + kBM - 1) / kBM, tn = (p.N + BN - 1) / BN;
    if (tn > 65535) return cudaErrorInvalidValue;
    if (BN == 128) return launch_cfg<128, kTcStore>(maps, a, dim3((unsigned)tm, (unsigned)tn), st);
    return launch_cfg<64, kTcStore>(maps, a, dim3((unsigned)tm, (unsigned)tn), st);
}

double tc_gemm_alg_flops(const TcGemm &p) {
    if (p.epilogue == kTcAssemble) return (double)p.N * (double)(p.N + 1) * (double)p.K;
    return 2.0 * (double)p.M * (double)p.N * (double)p.K;
}

}  // namespace dvr3d
