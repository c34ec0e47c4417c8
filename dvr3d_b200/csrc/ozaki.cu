// ozaki.cu -- FP64-accurate GEMM on the 5th-generation int8 tensor cores (sm_100a), after
// the Ozaki scheme (Ozaki, Ogita, Oishi and Rump 2012) in its integer form (Ootomo, Ozaki and
// Yokota 2024): each FP64 operand is cut into signed 7-bit slices that int8 products multiply
// exactly.
//
// Slicing: row r of op(A) (and column c of op(B)) is scaled by 2^-e_r, e_r the smallest
// exponent with max_k |A(r, k)| < 2^e_r, then x = A(r, k) 2^(7 - e_r) (|x| < 128) gives the
// digits d_1 = trunc(x), d_{i+1} = trunc(128 (x_i - d_i)), |d_i| <= 127, so that
//     A(r, k) = 2^e_r sum_i d_i 128^-i  + remainder below 2^e_r 128^-s   (s slices);
// every step is exact in FP64.
// Product: (op(A) op(B))(r, c) = 2^(e_r + f_c) sum_{i+j <= s+1} 128^-(i+j) P_ij(r, c) with
// P_ij = D^A_i (D^B_j)^T, an int8 GEMM with exact int32 accumulation. Products of the same
// weight share one accumulator (group g = i + j - 2, s groups); the dropped terms (i + j > s + 1)
// and the slice remainders weigh below 2^-49 of max|A(r,:)| max|B(:,c)| per term at 8 slices,
// under the FP64 unit roundoff times the term count that bounds a DMMA product's error.
//
// Kernels: a row-maximum pass (atomicMax on the bit pattern of |x|, which orders like the
// value), a slicing pass (64 x 64 tiles through shared memory, written K-contiguous, the
// triangle of a triangular operand masked to zero), and the GEMM: one CTA per 128 x 64 output
// tile, warp 0 / lane 0 streams 64-byte K steps of all slices of both operands with TMA
// (64-byte swizzle, no multicast) into a two-stage ring, warp 1 / lane 0 issues the
// s (s + 1) / 2 slice products of a stage as tcgen05.mma kind::i8 into s int32 accumulators in
// tensor memory (64 columns each), all four warps drain tensor memory and combine the groups
// in FP64 (Horner in 1/128, then the row and column scales). Waits are bounded in time as in
// tc_gemm.cu; a timeout sets the error flag and leaves the tile unwritten.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "common.cuh"
#include "ozaki.cuh"
#include "tcgen05.cuh"

namespace dvr3d {

namespace {

constexpr int kBM = 128;       // tile rows = UMMA M = tensor-memory lanes
constexpr int kBK = 64;        // K bytes (= int8 elements) per stage: one 64-byte swizzle row
constexpr int kUK = 32;        // K of one kind::i8 MMA
constexpr int kThreads = 128;  // 4 warps
constexpr unsigned long long kDefaultWaitNs = 4000000000ull;
constexpr unsigned long long kNanBits = 0x7ff8000000000000ull;

// BN = tile columns = UMMA N = tensor-memory columns of one accumulator (64, or 32 for the
// thin right-hand sides of the Krylov steps)
template <int S, int BN>
struct OzCfg {
    static constexpr int kA = kBM * kBK;  // bytes of one A slice tile (8 KB)
    static constexpr int kB = BN * kBK;   // bytes of one B slice tile
    static constexpr int kStage = S * (kA + kB);
    static constexpr int kStages = (200 * 1024) / kStage;
    static constexpr int kSmem = kStages * kStage + 1024;  // + slack to align the ring to 1 KB
    static constexpr int kCols = S * BN <= 32 ? 32 : (S * BN <= 64 ? 64 : (S * BN <= 128 ? 128 : (S * BN <= 256 ? 256 : 512)));
    static_assert(kStages >= 2, "at least double buffering");
    static_assert(S * BN <= 512, "one accumulator of BN columns per weight group");
};

struct OzMaps {
    CUtensorMap a[kOzMaxSlices];
    CUtensorMap b[kOzMaxSlices];
};

struct OzArgs {
    int M, N, K;
    int tri, tri_b, lower_out;
    int kchunk;    // > 0: CTA z sums K range [z kchunk, (z + 1) kchunk) into part (no alpha, beta)
    double *part;  // chunk z, element (i, j) at part[z M N + j M + i]
    double alpha, beta;
    double *C;
    long long ldc;
    const unsigned long long *umax_a, *umax_b;
    int *err;
    unsigned long long wait_ns;
};

// One operand seen as rows of K: X(r, k) = P[r rs + k ks], keep = 0 all, 1 k <= r, 2 k >= r.
struct OzOperand {
    const double *P;
    long long rs, ks;
    int rows, K, Kp, keep;
    unsigned long long *umax;
    signed char *S;  // slice sl, row r, k at S[sl sls + r Kp + k]
    long long sls;
};

__device__ __forceinline__ double oz_val(const OzOperand &o, int r, int k) {
    if (r >= o.rows || k >= o.K) return 0.0;
    if ((o.keep == 1 && k > r) || (o.keep == 2 && k < r)) return 0.0;
    return o.P[(long long)r * o.rs + (long long)k * o.ks];
}

__device__ __forceinline__ unsigned long long abs_bits(double v) {
    const double a = fabs(v);
    return isfinite(a) ? (unsigned long long)__double_as_longlong(a) : kNanBits;
}

// Row maxima of |X| over a 64 x 64 tile, folded into umax[r] by atomicMax on the bit pattern
// (non-negative doubles order like their bits; a non-finite entry records the NaN pattern,
// which is above every finite one).
template <bool KC>
__global__ void __launch_bounds__(256) oz_rowmax_kernel(OzOperand o) {
    const int r0 = blockIdx.y * 64, k0 = blockIdx.x * 64, t = threadIdx.x;
    if (KC) {  // k contiguous: 64 threads along k, four rows at a time
        const int kk = t & 63;
        for (int rr = t >> 6; rr < 64; rr += 4) {
            const int r = r0 + rr;
            unsigned long long m = abs_bits(oz_val(o, r, k0 + kk));
#pragma unroll
            for (int w = 16; w > 0; w >>= 1) {
                const unsigned long long q = __shfl_xor_sync(0xffffffffu, m, w);
                m = q > m ? q : m;
            }
            if ((t & 31) == 0 && m != 0 && r < o.rows) atomicMax(&o.umax[r], m);
        }
    } else {  // rows contiguous: one row per thread, 16 k each
        const int rr = t & 63, r = r0 + rr;
        unsigned long long m = 0;
        for (int kk = t >> 6; kk < 64; kk += 4) {
            const unsigned long long q = abs_bits(oz_val(o, r, k0 + kk));
            m = q > m ? q : m;
        }
        if (m != 0 && r < o.rows) atomicMax(&o.umax[r], m);
    }
}

// Slices of a 64 x 64 tile: loaded through shared memory along the contiguous direction of
// the source, then each thread cuts 16 consecutive k of one row into nslice digits and stores
// 16 bytes per slice (k beyond K, and masked entries, are zero digits).
template <bool KC>
__global__ void __launch_bounds__(256) oz_slice_kernel(OzOperand o, int nslice) {
    __shared__ double tile[64][65];
    const int r0 = blockIdx.y * 64, k0 = blockIdx.x * 64, t = threadIdx.x;
    if (KC) {
        for (int rr = t >> 6; rr < 64; rr += 4) tile[rr][t & 63] = oz_val(o, r0 + rr, k0 + (t & 63));
    } else {
        for (int kk = t >> 6; kk < 64; kk += 4) tile[t & 63][kk] = oz_val(o, r0 + (t & 63), k0 + kk);
    }
    __syncthreads();
    const int rr = t >> 2, kb = (t & 3) * 16, r = r0 + rr;
    if (r >= o.rows) return;
    const double mx = __longlong_as_double((long long)o.umax[r]);
    double sc = 0.0;
    if (mx > 0.0 && isfinite(mx)) {
        int e = 0;
        frexp(mx, &e);  // mx = f 2^e, 0.5 <= f < 1: every |x| of the row is below 2^e
        sc = ldexp(1.0, 7 - e);
    }
    double x[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = tile[rr][kb + j] * sc;  // |x| < 128, exact scaling
    signed char *dst = o.S + (long long)r * o.Kp + k0 + kb;
    for (int sl = 0; sl < nslice; ++sl) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const double d = trunc(x[j]);
            x[j] = (x[j] - d) * 128.0;
            w[j >> 2] |= ((uint32_t)(int)d & 0xffu) << (8 * (j & 3));
        }
        *reinterpret_cast<uint4 *>(dst + (long long)sl * o.sls) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with the 64-byte swizzle:
// rows of 64 bytes, 8-row groups 512 bytes apart (stride byte offset), version 1, layout
// SWIZZLE_64B. Advancing the start address by 32 bytes selects the second K = 32 half.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(512 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ int scale_exp(unsigned long long bits, bool &bad) {
    const double mx = __longlong_as_double((long long)bits);
    if (!isfinite(mx)) {
        bad = true;
        return 0;
    }
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    return e;
}

template <int S, int BN>
__global__ void __launch_bounds__(kThreads, 1) oz_gemm_kernel(const __grid_constant__ OzMaps maps, const OzArgs p) {
    using Cfg = OzCfg<S, BN>;
    extern __shared__ __align__(1024) unsigned char oz_smem[];
    __shared__ __align__(8) unsigned long long bar_full[Cfg::kStages];
    __shared__ __align__(8) unsigned long long bar_empty[Cfg::kStages];
    __shared__ __align__(8) unsigned long long bar_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_abort;
    __shared__ int s_cexp[BN];
    __shared__ int s_cbad[BN];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // grouped launch order: consecutive CTAs walk 16 row tiles of one column tile, then the
    // next column tile, so that a wave of CTAs shares a compact block of operand rows in L2
    // (row-tile-fastest order made every wave read all of op(A)'s slices from HBM)
    int ti, tj;
    {
        constexpr int G = 16;
        const int tm = (int)gridDim.x, tn = (int)gridDim.y;
        const long long t = (long long)blockIdx.y * tm + blockIdx.x, per = (long long)G * tn;
        const int g = (int)(t / per), first = g * G, gm = min(G, tm - first);
        const int r = (int)(t - (long long)g * per);
        ti = first + r % gm;
        tj = r / gm;
    }
    const int m0 = ti * kBM, n0 = tj * BN;
    if (p.lower_out && n0 > m0 + kBM - 1) return;  // tile strictly above the diagonal (uniform)
    const unsigned long long wait_ns = p.wait_ns;
    const unsigned long long t_end = tc::global_ns() + wait_ns;

    // K range holding nonzero terms of this tile
    int kb = 0, ke = p.K;
    if (p.tri == 1) ke = min(ke, m0 + kBM);
    if (p.tri == 2) kb = max(kb, m0);
    if (p.tri_b == 1) kb = max(kb, n0);
    if (p.tri_b == 2) ke = min(ke, n0 + BN);
    double *part = nullptr;
    if (p.kchunk > 0) {
        kb = max(kb, (int)blockIdx.z * p.kchunk);
        ke = min(ke, ((int)blockIdx.z + 1) * p.kchunk);
        part = p.part + (long long)blockIdx.z * p.M * p.N;
    }
    kb &= ~(kBK - 1);
    const int nk = ke > kb ? (ke - kb + kBK - 1) / kBK : 0;
    if (part && nk == 0) {  // an empty chunk of this tile: its partial sum is zero (uniform)
        for (int q = threadIdx.x; q < kBM * BN; q += kThreads) {
            const int i = m0 + (q % kBM), j = n0 + q / kBM;
            if (i < p.M && j < p.N) part[(long long)j * p.M + i] = 0.0;
        }
        return;
    }

    const uint32_t ring = (tc::smem_u32(oz_smem) + 1023u) & ~1023u;
    const uint32_t full0 = tc::smem_u32(&bar_full[0]), empty0 = tc::smem_u32(&bar_empty[0]);
    const uint32_t done = tc::smem_u32(&bar_done);
    if (threadIdx.x == 0) {
        for (int s = 0; s < Cfg::kStages; ++s) {
            tc::mbar_init(full0 + 8u * s, 1);
            tc::mbar_init(empty0 + 8u * s, 1);
        }
        tc::mbar_init(done, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < BN) {
        const int c = n0 + threadIdx.x;
        bool bad = false;
        s_cexp[threadIdx.x] = c < p.N ? scale_exp(p.umax_b[c], bad) : 0;
        s_cbad[threadIdx.x] = bad ? 1 : 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         tc::smem_u32(&tmem_slot)),
                     "r"((uint32_t)Cfg::kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tmem_slot;

    constexpr uint32_t tx_bytes = (uint32_t)(S * (Cfg::kA + Cfg::kB));
    if (threadIdx.x == 0) {
        // ---- TMA producer: all slices of both operands for one K step per stage
        int it = 0;
        bool ok = true;
        for (; it < nk; ++it) {
            const int s = it % Cfg::kStages;
            const uint32_t ph = (uint32_t)(it / Cfg::kStages) & 1u;
            if (!tc::mbar_wait(empty0 + 8u * s, ph ^ 1u, t_end) || *(volatile int *)&s_abort) {
                ok = false;
                break;
            }
            const uint32_t sa = ring + (uint32_t)(s * Cfg::kStage), sb = sa + (uint32_t)(S * Cfg::kA);
            tc::mbar_expect_tx(full0 + 8u * s, tx_bytes);
            const int kx = kb + it * kBK;
#pragma unroll
            for (int sl = 0; sl < S; ++sl) {
                tc::tma_load_2d(sa + (uint32_t)(sl * Cfg::kA), &maps.a[sl], full0 + 8u * s, kx, m0);
                tc::tma_load_2d(sb + (uint32_t)(sl * Cfg::kB), &maps.b[sl], full0 + 8u * s, kx, n0);
            }
        }
        if (!ok) {
            atomicExch(&s_abort, 1);
            if (p.err) atomicExch(p.err, (int)kDevBarrierTimeout);
        }
        for (int j = (it > Cfg::kStages ? it - Cfg::kStages : 0); j < it; ++j)
            tc::mbar_wait(full0 + 8u * (j % Cfg::kStages), (uint32_t)(j / Cfg::kStages) & 1u, t_end + wait_ns);
    } else if (threadIdx.x == 32) {
        // ---- MMA issuer: pairs (i, j), i + j <= S - 1 (0-based), into accumulator i + j
        const uint32_t idesc = (2u << 4)                          // D: S32
                               | (1u << 7) | (1u << 10)            // A, B: signed 8-bit
                               | ((uint32_t)(BN >> 3) << 17)       // N
                               | ((uint32_t)(kBM >> 4) << 24);     // M
        bool ok = true;
        for (int it = 0; it < nk; ++it) {
            const int s = it % Cfg::kStages;
            const uint32_t ph = (uint32_t)(it / Cfg::kStages) & 1u;
            if (!tc::mbar_wait(full0 + 8u * s, ph, t_end) || *(volatile int *)&s_abort) {
                ok = false;
                break;
            }
            tc::fence_after();
            const uint32_t sa = ring + (uint32_t)(s * Cfg::kStage), sb = sa + (uint32_t)(S * Cfg::kA);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                const uint64_t da = sw64_desc(sa + (uint32_t)(i * Cfg::kA));
#pragma unroll
                for (int j = 0; j + i < S; ++j) {
                    const uint64_t db = sw64_desc(sb + (uint32_t)(j * Cfg::kB));
                    const uint32_t dst = tmem + (uint32_t)((i + j) * BN);
#pragma unroll
                    for (int kk = 0; kk < kBK / kUK; ++kk)  // the first product of a group starts it
                        umma_i8(dst, da + (uint64_t)(2 * kk), db + (uint64_t)(2 * kk), idesc,
                                (it | i | kk) != 0 ? 1u : 0u);
                }
            }
            tc::umma_commit(empty0 + 8u * s);
        }
        if (!ok) {
            atomicExch(&s_abort, 1);
            if (p.err) atomicExch(p.err, (int)kDevBarrierTimeout);
        }
        tc::umma_commit(done);  // arrives once every product issued above has completed
    }
    __syncwarp();

    // ---- epilogue: s int32 accumulators -> FP64
    const bool got = tc::mbar_wait(done, 0u, t_end + wait_ns);
    tc::fence_after();
    const bool warp_ok = __all_sync(0xffffffffu, got && *(volatile int *)&s_abort == 0);
    if (!got && lane == 0 && p.err) atomicExch(p.err, (int)kDevBarrierTimeout);
    if (warp_ok) {
        const int row = m0 + warp * 32 + lane;
        bool rbad = false;
        const int er = row < p.M ? scale_exp(p.umax_a[row], rbad) : 0;
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            if (n0 + c0 >= p.N) break;  // uniform over the warp
            double t[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) t[j] = 0.0;
            if (nk > 0) {
#pragma unroll 1
                for (int q = S - 1; q >= 0; --q) {  // t = sum_q acc_q 128^-q (Horner, smallest first)
                    uint32_t r[32];
                    tc::tmem_ld32(tmem + lane_base + (uint32_t)(q * BN + c0), r);
#pragma unroll
                    for (int j = 0; j < 32; ++j) t[j] = (double)(int)r[j] + t[j] * 0.0078125;
                }
            }
            if (row >= p.M) continue;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int col = n0 + c0 + j;
                if (col >= p.N || (p.lower_out && col > row)) continue;
                double val = ldexp(t[j], er + s_cexp[c0 + j] - 14);
                if (rbad || s_cbad[c0 + j]) val = __longlong_as_double((long long)kNanBits);
                if (part) {
                    part[(long long)col * p.M + row] = val;
                    continue;
                }
                double *pc = p.C + (long long)col * p.ldc + row;
                double out = p.alpha * val;
                if (p.beta != 0.0) out += p.beta * *pc;
                *pc = out;
            }
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)Cfg::kCols));
    }
}

bool make_map(tc::EncodeTiledFn fn, CUtensorMap &m, const signed char *ptr, int rows, int Kp, int box_rows) {
    const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)Kp};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<signed char *>(ptr), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The kernel's shared-memory opt-in, once per device (kept outside stream capture by callers
// that capture: ozaki_set_attributes).
template <int S, int BN>
cudaError_t set_attr() {
    static bool attr_done[kMaxAttrDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= kMaxAttrDevices || !attr_done[dev]) {
        e = cudaFuncSetAttribute(oz_gemm_kernel<S, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 OzCfg<S, BN>::kSmem);
        if (e != cudaSuccess) return e;
        if (dev < kMaxAttrDevices) attr_done[dev] = true;
    }
    return cudaSuccess;
}

template <int S, int BN>
cudaError_t launch_cfg(const OzMaps &maps, const OzArgs &a, dim3 grid, cudaStream_t st) {
    cudaError_t e = set_attr<S, BN>();
    if (e != cudaSuccess) return e;
    DVR3D_COUNT_LAUNCH(1);
    oz_gemm_kernel<S, BN><<<grid, kThreads, OzCfg<S, BN>::kSmem, st>>>(maps, a);
    return cudaGetLastError();
}

template <int BN>
cudaError_t launch_bn(int nslice, const OzMaps &maps, const OzArgs &a, dim3 grid, cudaStream_t st) {
    switch (nslice) {
        case 4: return launch_cfg<4, BN>(maps, a, grid, st);
        case 5: return launch_cfg<5, BN>(maps, a, grid, st);
        case 6: return launch_cfg<6, BN>(maps, a, grid, st);
        case 7: return launch_cfg<7, BN>(maps, a, grid, st);
        default: return launch_cfg<8, BN>(maps, a, grid, st);
    }
}

template <int BN>
cudaError_t set_attr_bn(int nslice) {
    switch (nslice) {
        case 4: return set_attr<4, BN>();
        case 5: return set_attr<5, BN>();
        case 6: return set_attr<6, BN>();
        case 7: return set_attr<7, BN>();
        default: return set_attr<8, BN>();
    }
}

// C = alpha sum_z part[z] + beta C, the chunks summed in a fixed order (deterministic).
__global__ void oz_reduce_kernel(const double *__restrict__ part, int nchunk, int M, int N, double alpha,
                                 double beta, double *C, long long ldc) {
    const long long tot = (long long)M * N, stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += stride) {
        double v = 0.0;
        for (int z = 0; z < nchunk; ++z) v += part[(long long)z * tot + t];
        const int j = (int)(t / M), i = (int)(t % M);
        double *pc = C + (long long)j * ldc + i;
        *pc = beta != 0.0 ? alpha * v + beta * *pc : alpha * v;
    }
}

long long rup(long long a, long long b) { return (a + b - 1) / b * b; }

int tile_n_of(const GemmOp &p) { return p.N <= 32 && !p.lower_out ? 32 : 64; }

struct Layout {
    int Kp;
    bool shared;  // op(B)'s rows are op(A)'s rows (A A^T): one set of slices
    bool pre;     // op(A) sliced beforehand (OzPresliced): no A slices here
    int nchunk;
    size_t umax_a, umax_b, sa, sb, part, total;
};

Layout layout_of(const GemmOp &p, int nslice, bool pre, int kchunk) {
    Layout L{};
    L.Kp = (int)rup(std::max(p.K, 1), kBK);
    L.pre = pre;
    L.shared = !pre && p.A == p.B && p.lda == p.ldb && p.ta != p.tb && p.tri == 0 && p.tri_b == 0 && p.M == p.N;
    L.nchunk = kchunk > 0 ? (p.K + kchunk - 1) / kchunk : 0;
    size_t off = 0;
    L.umax_a = off;
    if (!pre) off = (size_t)rup(off + 8 * (size_t)p.M, 1024);
    L.umax_b = off;
    off = (size_t)rup(off + 8 * (size_t)p.N, 1024);
    L.sa = off;
    if (!pre) off = (size_t)rup(off + (size_t)nslice * p.M * L.Kp, 1024);
    L.sb = L.shared ? L.sa : off;
    if (!L.shared) off = (size_t)rup(off + (size_t)nslice * p.N * L.Kp, 1024);
    L.part = off;
    off = (size_t)rup(off + 8 * (size_t)L.nchunk * p.M * p.N, 1024);
    L.total = off;
    return L;
}

OzOperand a_operand(const GemmOp &p, int Kp, unsigned long long *umax, signed char *S) {
    // op(A)(i, k) = ta ? A[i lda + k] : A[k lda + i]; rows of the A side are i
    return OzOperand{p.A, p.ta ? p.lda : 1, p.ta ? 1 : p.lda, p.M, p.K, Kp, p.tri == 1 ? 1 : (p.tri == 2 ? 2 : 0),
                     umax, S, (long long)p.M * Kp};
}

cudaError_t slice_operand(const OzOperand &o, int nslice, cudaStream_t st) {
    const dim3 grid((unsigned)(o.Kp / 64), (unsigned)((o.rows + 63) / 64));
    if (grid.y > 65535) return cudaErrorInvalidValue;
    const bool kc = o.ks == 1;
    DVR3D_COUNT_LAUNCH(2);
    if (kc) oz_rowmax_kernel<true><<<grid, 256, 0, st>>>(o);
    else oz_rowmax_kernel<false><<<grid, 256, 0, st>>>(o);
    if (kc) oz_slice_kernel<true><<<grid, 256, 0, st>>>(o, nslice);
    else oz_slice_kernel<false><<<grid, 256, 0, st>>>(o, nslice);
    return cudaGetLastError();
}

}  // namespace

bool ozaki_supported(const GemmOp &p, int nslice) {
    if (nslice < kOzMinSlices || nslice > kOzMaxSlices) return false;
    if (p.M <= 0 || p.N <= 0 || p.K <= 0 || p.K > kOzMaxK) return false;
    if (p.lower_out && p.M != p.N) return false;
    if (!p.A || !p.B || !p.C || p.tri < 0 || p.tri > 2 || p.tri_b < 0 || p.tri_b > 2) return false;
    if ((p.M + 63) / 64 > 65535 || (p.N + 31) / 32 > 65535) return false;
    return true;
}

bool ozaki_profitable(const GemmOp &p) {
    // below a few thousand output tiles of work the slicing passes and the single-CTA-per-SM
    // occupancy cost more than the DMMA main loop they replace
    return p.M >= 1536 && p.N >= 1536 && p.K >= 1024;
}

size_t ozaki_work_bytes(const GemmOp &p, int nslice, bool presliced_a, int kchunk) {
    return layout_of(p, nslice, presliced_a, kchunk).total;
}

size_t ozaki_preslice_bytes(const GemmOp &p, int nslice) {
    return (size_t)rup(8 * (size_t)p.M, 1024) + (size_t)nslice * p.M * rup(std::max(p.K, 1), kBK);
}

cudaError_t ozaki_preslice_a(const GemmOp &p, int nslice, void *buf, size_t bytes, OzPresliced &out,
                             cudaStream_t st) {
    if (!ozaki_supported(p, nslice)) return cudaErrorInvalidValue;
    if (!buf || bytes < ozaki_preslice_bytes(p, nslice) || (reinterpret_cast<uintptr_t>(buf) & 1023u))
        return cudaErrorInvalidValue;
    const int Kp = (int)rup(p.K, kBK);
    unsigned char *w = static_cast<unsigned char *>(buf);
    auto *umax = reinterpret_cast<unsigned long long *>(w);
    auto *S = reinterpret_cast<signed char *>(w + rup(8 * (size_t)p.M, 1024));
    cudaError_t e = cudaMemsetAsync(umax, 0, 8 * (size_t)p.M, st);
    if (e != cudaSuccess) return e;
    if ((e = slice_operand(a_operand(p, Kp, umax, S), nslice, st)) != cudaSuccess) return e;
    out = OzPresliced{S, umax, p.M, p.K, nslice, p.tri};
    return cudaSuccess;
}

double ozaki_alg_flops(const GemmOp &p) { return gemm_alg_flops(p); }

cudaError_t ozaki_set_attributes(const GemmOp &p, int nslice) {
    if (nslice < kOzMinSlices || nslice > kOzMaxSlices) return cudaErrorInvalidValue;
    tc::encode_tiled();
    return tile_n_of(p) == 32 ? set_attr_bn<32>(nslice) : set_attr_bn<64>(nslice);
}

cudaError_t launch_ozaki_gemm(const GemmOp &p, int nslice, void *work, size_t work_bytes, int *err,
                              cudaStream_t st, const OzPresliced *pre, int kchunk) {
    if (p.M <= 0 || p.N <= 0) return cudaSuccess;
    if (!ozaki_supported(p, nslice)) return cudaErrorInvalidValue;
    if (pre && (pre->rows != p.M || pre->K != p.K || pre->nslice != nslice || pre->tri != p.tri || !pre->S))
        return cudaErrorInvalidValue;
    if (kchunk < 0 || (kchunk > 0 && (kchunk % kBK != 0 || p.lower_out || (p.K + kchunk - 1) / kchunk > 65535)))
        return cudaErrorInvalidValue;
    const Layout L = layout_of(p, nslice, pre != nullptr, kchunk);
    if (!work || work_bytes < L.total || (reinterpret_cast<uintptr_t>(work) & 1023u)) return cudaErrorInvalidValue;
    tc::EncodeTiledFn fn = tc::encode_tiled();
    if (!fn) return cudaErrorNotSupported;
    unsigned char *w = static_cast<unsigned char *>(work);
    const unsigned long long *umax_a = pre ? pre->umax : reinterpret_cast<unsigned long long *>(w + L.umax_a);
    auto *umax_b = L.shared ? const_cast<unsigned long long *>(umax_a)
                            : reinterpret_cast<unsigned long long *>(w + L.umax_b);
    const signed char *sa = pre ? pre->S : reinterpret_cast<signed char *>(w + L.sa);
    auto *sb = reinterpret_cast<signed char *>(w + L.sb);
    cudaError_t e = cudaMemsetAsync(w, 0, L.sa, st);
    if (e != cudaSuccess) return e;

    if (!pre) {
        const OzOperand oa = a_operand(p, L.Kp, const_cast<unsigned long long *>(umax_a), const_cast<signed char *>(sa));
        if ((e = slice_operand(oa, nslice, st)) != cudaSuccess) return e;
    }
    // op(B)(k, j) = tb ? B[k ldb + j] : B[j ldb + k]; rows of the B side are j; op(B) lower
    // (tri_b = 1) keeps k >= j, upper keeps k <= j
    const OzOperand ob{p.B, p.tb ? 1 : p.ldb, p.tb ? p.ldb : 1, p.N, p.K, L.Kp,
                       p.tri_b == 1 ? 2 : (p.tri_b == 2 ? 1 : 0), umax_b, sb, (long long)p.N * L.Kp};
    if (!L.shared && (e = slice_operand(ob, nslice, st)) != cudaSuccess) return e;

    const int bn = tile_n_of(p);
    OzMaps maps;
    std::memset(&maps, 0, sizeof(maps));
    for (int sl = 0; sl < nslice; ++sl) {
        if (!make_map(fn, maps.a[sl], sa + (size_t)sl * p.M * L.Kp, p.M, L.Kp, kBM)) return cudaErrorInvalidValue;
        if (!make_map(fn, maps.b[sl], sb + (size_t)sl * p.N * L.Kp, p.N, L.Kp, bn)) return cudaErrorInvalidValue;
    }
    OzArgs a{};
    a.M = p.M;
    a.N = p.N;
    a.K = p.K;
    a.tri = p.tri;
    a.tri_b = p.tri_b;
    a.lower_out = p.lower_out;
    a.kchunk = kchunk;
    a.part = kchunk > 0 ? reinterpret_cast<double *>(w + L.part) : nullptr;
    a.alpha = p.alpha;
    a.beta = p.beta;
    a.C = p.C;
    a.ldc = p.ldc;
    a.umax_a = umax_a;
    a.umax_b = umax_b;
    a.err = err;
    a.wait_ns = kDefaultWaitNs;
    const dim3 grid((unsigned)((p.M + kBM - 1) / kBM), (unsigned)((p.N + bn - 1) / bn),
                    (unsigned)std::max(1, L.nchunk));
    e = bn == 32 ? launch_bn<32>(nslice, maps, a, grid, st) : launch_bn<64>(nslice, maps, a, grid, st);
    if (e != cudaSuccess || kchunk == 0) return e;
    const long long tot = (long long)p.M * p.N;
    DVR3D_COUNT_LAUNCH(1);
    oz_reduce_kernel<<<(unsigned)std::min<long long>((tot + 255) / 256, 148LL * 8), 256, 0, st>>>(
        a.part, L.nchunk, p.M, p.N, p.alpha, p.beta, p.C, p.ldc);
    return cudaGetLastError();
}

}  // namespace dvr3d
