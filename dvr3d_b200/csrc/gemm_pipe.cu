// gemm_pipe.cu -- pipelined FP64 tensor-core GEMM (DMMA mma.sync m8n8k4 .f64, cp.async
// double buffering) with the options the shift-invert Krylov solver needs:
//   * either operand stored column-major or transposed (no copies),
//   * a triangular first operand (K range limited per output row tile),
//   * lower-triangle output only (SYRK-style updates of a symmetric matrix),
//   * split-K over gridDim.y: up to 8 slices as one thread-block cluster whose partial tiles
//     are summed through distributed shared memory (deterministic, no second kernel), more
//     slices through a scratch buffer and a second-pass reduction.
//
// Tiles are BM x BN = 64 x 64 (or 64 x 32 for thin right-hand sides), BK = 16; four warps,
// 2 x 2, each a 32 x (BN/2) sub-tile. Shared-memory layouts follow the contiguous direction
// of the source so that every cp.async moves 16 bytes: [m][k] (stride 20 doubles) for
// k-contiguous operands, [k][m] (stride BM+4) for m-contiguous ones; both strides make the
// DMMA fragment reads bank-conflict free.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "gemm64.cuh"

namespace dvr3d {

namespace {

constexpr int kBM = 64, kBK = 16, kThr = 128;
constexpr int kSK = kBK + 4;  // stride of [m][k] tiles
constexpr int kMaxClusterSplit = 8;  // portable cluster size
// Instruction shape of the inner product: m16n8k16 (one instruction per 16-deep k tile and
// 16 x 8 output block) or the m8n8k4 of sm_80.
#ifndef DVR3D_GEMM_K16
#define DVR3D_GEMM_K16 1
#endif
constexpr bool kUseK16 = DVR3D_GEMM_K16 != 0;

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// The larger FP64 shape of sm_90+: one instruction does a 16 x 8 x 16 product. With
// g = lane / 4 and t = lane % 4 the fragments are A(g + 8 (i % 2), t + 4 (i / 2)) for
// a[0..7], B(k = t + 4 i, n = g) for b[0..3], and C(g, 2t), C(g, 2t+1), C(g+8, 2t),
// C(g+8, 2t+1) for c[0..3].
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
        "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
          "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

__device__ __forceinline__ void cp16(void *smem, const void *gmem, int bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}

// Tile of ROWS x kBK elements, element (r, k) of the operand at src(r, k).
//   KC = true : source contiguous in k   -> smem [ROWS][kSK]
//   KC = false: source contiguous in r   -> smem [kBK][ROWS + 4]
template <int ROWS, bool KC>
struct TileLoader {
    static constexpr int kStride = KC ? kSK : ROWS + 4;
    static constexpr int kElems = KC ? ROWS * kSK : kBK * (ROWS + 4);
    // base points at element (r0, k0); ld is the stride between consecutive k (r-contiguous)
    // or consecutive r (k-contiguous); rmax / kmax: valid extents from (r0, k0)
    __device__ static void load(double *sm, const double *base, long long ld, int rmax, int kmax, int tid) {
        constexpr int kChunks = ROWS * kBK / 2;
#pragma unroll
        for (int q = 0; q < (kChunks + kThr - 1) / kThr; ++q) {
            const int e = tid + q * kThr;
            if (kChunks % kThr != 0 && e >= kChunks) break;
            int r, k, valid;
            if (KC) {
                r = e >> 3;
                k = (e & 7) * 2;
                valid = (r < rmax) ? min(max(kmax - k, 0), 2) : 0;
            } else {
                k = e / (ROWS / 2);
                r = (e % (ROWS / 2)) * 2;
                valid = (k < kmax) ? min(max(rmax - r, 0), 2) : 0;
            }
            double *dst = KC ? sm + r * kSK + k : sm + k * kStride + r;
            const double *src = valid ? (KC ? base + (size_t)r * ld + k : base + (size_t)k * ld + r) : base;
            cp16(dst, src, valid * 8);
        }
    }
    __device__ static double at(const double *sm, int r, int k) { return KC ? sm[r * kSK + k] : sm[k * kStride + r]; }
};

// op(A)(i, k): TA ? A[i * lda + k] : A[k * lda + i]   (k-contiguous when TA)
// op(B)(k, j): TB ? B[k * ldb + j] : B[j * ldb + k]   (k-contiguous when !TB)
template <bool TA, bool TB, int BN, bool CL, bool K16 = kUseK16>
__global__ void __launch_bounds__(kThr) gemm_pipe_kernel(GemmOp p, int tiles_m) {
    using LA = TileLoader<kBM, TA>;
    using LB = TileLoader<BN, !TB>;
    constexpr int WN = BN / 2, FN = WN / 8;
    // stages in flight: three for thin right-hand sides (two loads outstanding while one
    // stage is multiplied), two for 64-wide tiles (static shared memory limit)
    constexpr int NS = (BN == 32) ? 3 : 2;
    constexpr int kSmem = NS * LA::kElems + NS * LB::kElems;
    static_assert(kSmem >= kBM * BN, "staging of the cluster reduction fits the operand buffers");
    __shared__ __align__(16) double smem_all[kSmem];
    double(*As)[LA::kElems] = reinterpret_cast<double(*)[LA::kElems]>(smem_all);
    double(*Bs)[LB::kElems] = reinterpret_cast<double(*)[LB::kElems]>(smem_all + NS * LA::kElems);
    int tm, tn;
    if (p.lower_out) {
        const long long t = blockIdx.x;
        int ti = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
        while ((long long)ti * (ti + 1) / 2 > t) --ti;
        while ((long long)(ti + 1) * (ti + 2) / 2 <= t) ++ti;
        tm = ti;
        tn = (int)(t - (long long)ti * (ti + 1) / 2);
    } else {
        tm = blockIdx.x % tiles_m;
        tn = blockIdx.x / tiles_m;
        // triangular operands: the tiles with the longest K ranges first (lower op(A): the
        // bottom row tiles; upper op(B): the right column tiles), so they do not form the tail
        if (p.tri == 1) tm = tiles_m - 1 - tm;
        if (p.tri_b == 2) tn = (int)((gridDim.x / tiles_m) - 1) - tn;
    }
    const int i0 = tm * kBM, j0 = tn * BN;
    // K range of this tile (triangular op(A)) and of this split
    int kb = 0, ke = p.K;
    if (p.tri == 1) ke = min(ke, i0 + kBM);
    else if (p.tri == 2) kb = (i0 / kBK) * kBK;
    if (p.tri_b == 1) kb = max(kb, (j0 / kBK) * kBK);
    else if (p.tri_b == 2) ke = min(ke, j0 + BN);
    const int ntk = ke > kb ? (ke - kb + kBK - 1) / kBK : 0;
    const int S = gridDim.y, z = blockIdx.y;
    const int t0 = (int)((long long)ntk * z / S), t1 = (int)((long long)ntk * (z + 1) / S);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * WN;
    // accumulators: K16 -> [two 16-row tiles][FN 8-column tiles][4]; else [four 8-row
    // tiles][FN][2]; either way 8 FN doubles per thread
    double acc[K16 ? 2 : 4][FN][K16 ? 4 : 2];
#pragma unroll
    for (int a = 0; a < (K16 ? 2 : 4); ++a)
#pragma unroll
        for (int b = 0; b < FN; ++b)
#pragma unroll
            for (int h = 0; h < (K16 ? 4 : 2); ++h) acc[a][b][h] = 0.0;
    // row / column of accumulator element (a, b, h) within the CTA tile
    auto acc_row = [&](int a, int h) { return K16 ? wm + a * 16 + (lane >> 2) + 8 * (h >> 1) : wm + a * 8 + (lane >> 2); };
    auto acc_col = [&](int b, int h) { return wn + b * 8 + (lane & 3) * 2 + (K16 ? (h & 1) : h); };
    auto load = [&](int st, int kt) {
        const int k0 = kb + kt * kBK;
        const int kmax = ke - k0;
        const double *a = TA ? p.A + (size_t)i0 * p.lda + k0 : p.A + (size_t)k0 * p.lda + i0;
        LA::load(As[st], a, p.lda, p.M - i0, kmax, tid);
        const double *b = TB ? p.B + (size_t)k0 * p.ldb + j0 : p.B + (size_t)j0 * p.ldb + k0;
        LB::load(Bs[st], b, p.ldb, p.N - j0, kmax, tid);
        asm volatile("cp.async.commit_group;\n" ::);
    };
    const int r = lane >> 2, c = lane & 3;
#pragma unroll
    for (int q = 0; q < NS - 1; ++q)
        if (t0 + q < t1) load(q, t0 + q);
    for (int kt = t0; kt < t1; ++kt) {
        const int st = (kt - t0) % NS;
        // tile kt + NS - 1 goes into the stage freed by tile kt - 1 (the barrier at the end
        // of the previous iteration); then wait until tile kt has landed
        if (kt + NS - 1 < t1) {
            load((kt - t0 + NS - 1) % NS, kt + NS - 1);
            asm volatile("cp.async.wait_group %0;\n" ::"n"(NS - 1));
        } else if (NS == 3 && kt + 1 < t1) {
            asm volatile("cp.async.wait_group 1;\n" ::);
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::);
        }
        __syncthreads();
        if constexpr (K16) {
            double af[2][8], bf[FN][4];
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int i = 0; i < 8; ++i) af[a][i] = LA::at(As[st], wm + a * 16 + r + 8 * (i & 1), c + 4 * (i >> 1));
#pragma unroll
            for (int b = 0; b < FN; ++b)
#pragma unroll
                for (int i = 0; i < 4; ++i) bf[b][i] = LB::at(Bs[st], wn + b * 8 + r, c + 4 * i);
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < FN; ++b) dmma16(*reinterpret_cast<double(*)[4]>(acc[a][b]), af[a], bf[b]);
        } else {
#pragma unroll
            for (int kk = 0; kk < kBK; kk += 4) {
                double af[4], bf[FN];
#pragma unroll
                for (int t = 0; t < 4; ++t) af[t] = LA::at(As[st], wm + t * 8 + r, kk + c);
#pragma unroll
                for (int t = 0; t < FN; ++t) bf[t] = LB::at(Bs[st], wn + t * 8 + r, kk + c);
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < FN; ++b) dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
            }
        }
        __syncthreads();
    }
    constexpr int NA = K16 ? 2 : 4, NH = K16 ? 4 : 2;
    if constexpr (CL) {
        // cluster split-K: stage this slice's tile, sum the S slices through distributed
        // shared memory, each CTA of the cluster finishing 64/S rows of the tile
        namespace cg = cooperative_groups;
        cg::cluster_group cluster = cg::this_cluster();
        __syncthreads();
        double *stage = smem_all;
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int b = 0; b < FN; ++b)
#pragma unroll
                for (int h = 0; h < NH; ++h) stage[acc_row(a, h) * BN + acc_col(b, h)] = acc[a][b][h];
        cluster.sync();
        const int rank = (int)cluster.block_rank();
        const int r0 = rank * kBM / S, r1 = (rank + 1) * kBM / S;
        for (int q = threadIdx.x; q < (r1 - r0) * BN; q += kThr) {
            const int rr = r0 + q / BN, cc = q % BN;
            const int i = i0 + rr, j = j0 + cc;
            double sum = 0.0;
            for (int u = 0; u < S; ++u) sum += cluster.map_shared_rank(stage, u)[rr * BN + cc];
            if (i < p.M && j < p.N && !(p.lower_out && j > i)) {
                double *cp = p.C + (size_t)j * p.ldc + i;
                const double old = (p.beta != 0.0) ? *cp : 0.0;
                *cp = p.alpha * sum + p.beta * old;
            }
        }
        cluster.sync();
        return;
    }
    const bool split = (S > 1);
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < FN; ++b)
#pragma unroll
            for (int h = 0; h < NH; ++h) {
                const int i = i0 + acc_row(a, h), j = j0 + acc_col(b, h);
                if (i >= p.M || j >= p.N) continue;
                if (p.lower_out && j > i) continue;
                if (split) {
                    p.work[((size_t)z * p.N + j) * p.M + i] = acc[a][b][h];
                } else {
                    double *cp = p.C + (size_t)j * p.ldc + i;
                    const double old = (p.beta != 0.0) ? *cp : 0.0;
                    *cp = p.alpha * acc[a][b][h] + p.beta * old;
                }
            }
}

// Sum of the S partial tiles: a block covers 32 consecutive rows of one column; its eight
// warps take every eighth slice (eight independent loads in flight per thread) and add
// their sums through shared memory.
__global__ void __launch_bounds__(256) splitk_reduce_kernel(GemmOp p, int S) {
    __shared__ double part[8][33];
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + lane, j = blockIdx.y;
    const bool live = i < p.M && !(p.lower_out && j > i);
    double s = 0.0;
    if (live) {
        const double *w = p.work + (size_t)j * p.M + i;
        const size_t zs = (size_t)p.N * p.M;
        for (int z0 = g; z0 < S; z0 += 64) {
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int z = z0 + 8 * u;
                s += (z < S) ? w[(size_t)z * zs] : 0.0;
            }
        }
    }
    part[g][lane] = s;
    __syncthreads();
    if (g == 0 && live) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) t += part[q][lane];
        double *cp = p.C + (size_t)j * p.ldc + i;
        const double old = (p.beta != 0.0) ? *cp : 0.0;
        *cp = p.alpha * t + p.beta * old;
    }
}

template <bool TA, bool TB, int BN, bool CL>
cudaError_t launch_one(const GemmOp &p, dim3 grid, int S, int tiles_m, cudaStream_t st) {
    if (!CL) {
        gemm_pipe_kernel<TA, TB, BN, false><<<grid, kThr, 0, st>>>(p, tiles_m);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kThr);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = S;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, gemm_pipe_kernel<TA, TB, BN, true>, p, tiles_m);
}

template <int BN, bool CL>
cudaError_t launch_bn(const GemmOp &p, int S, cudaStream_t st) {
    const int tiles_m = (p.M + kBM - 1) / kBM, tiles_n = (p.N + BN - 1) / BN;
    const long long nt = p.lower_out ? (long long)tiles_m * (tiles_m + 1) / 2 : (long long)tiles_m * tiles_n;
    dim3 grid((unsigned)nt, (unsigned)S);
    DVR3D_COUNT_LAUNCH(1);
    if (!p.ta && !p.tb) return launch_one<false, false, BN, CL>(p, grid, S, tiles_m, st);
    if (p.ta && !p.tb) return launch_one<true, false, BN, CL>(p, grid, S, tiles_m, st);
    if (!p.ta && p.tb) return launch_one<false, true, BN, CL>(p, grid, S, tiles_m, st);
    return launch_one<true, true, BN, CL>(p, grid, S, tiles_m, st);
}

}  // namespace

size_t gemm_splitk_work(int M, int N, int S) { return S > kMaxClusterSplit ? (size_t)S * M * N : 0; }

double gemm_alg_flops(const GemmOp &p) {
    const double M = p.M, N = p.N, K = p.K;
    if (p.M <= 0 || p.N <= 0 || p.K <= 0) return 0.0;
    // sum over i < n of min(i + 1, k), and of max(k - i, 0)
    auto head = [](double n, double k) { return n <= k ? n * (n + 1.0) * 0.5 : k * (k + 1.0) * 0.5 + (n - k) * k; };
    auto tail = [](double n, double k) {
        const double t = n < k ? n : k;
        return t * k - t * (t - 1.0) * 0.5;
    };
    if (p.lower_out) return 2.0 * K * M * (M + 1.0) * 0.5;
    if (p.tri == 1) return 2.0 * N * head(M, K);
    if (p.tri == 2) return 2.0 * N * tail(M, K);
    if (p.tri_b == 1) return 2.0 * M * tail(N, K);
    if (p.tri_b == 2) return 2.0 * M * head(N, K);
    return 2.0 * M * N * K;
}

namespace {
thread_local GemmLaunchLog *t_gemm_log = nullptr;
cudaError_t launch_gemm_kernels(const GemmOp &p0, cudaStream_t st);
}  // namespace

void set_gemm_launch_log(GemmLaunchLog *log) { t_gemm_log = log; }

double gemm_launch_log_ms(const GemmLaunchLog &log) {
    if (log.used < 2) return 0.0;
    cudaEventSynchronize(log.ev[log.used - 1]);
    double ms = 0.0;
    for (int q = 0; q + 1 < log.used; q += 2) {
        float m = 0.f;
        if (cudaEventElapsedTime(&m, log.ev[q], log.ev[q + 1]) == cudaSuccess) ms += m;
    }
    return ms;
}

cudaError_t launch_gemm(const GemmOp &p, cudaStream_t st) {
    GemmLaunchLog *lg = t_gemm_log;
    if (!lg || p.M <= 0 || p.N <= 0) return launch_gemm_kernels(p, st);
    if (lg->used + 2 > lg->nev) {
        ++lg->untimed;
        return launch_gemm_kernels(p, st);
    }
    cudaEventRecord(lg->ev[lg->used], st);
    const cudaError_t e = launch_gemm_kernels(p, st);
    cudaEventRecord(lg->ev[lg->used + 1], st);
    lg->used += 2;
    ++lg->launches;
    lg->flops += gemm_alg_flops(p);
    return e;
}

namespace {

cudaError_t launch_gemm_kernels(const GemmOp &p0, cudaStream_t st) {
    GemmOp p = p0;
    if (p.M <= 0 || p.N <= 0) return cudaSuccess;
    if (p.lower_out && p.M != p.N) return cudaErrorInvalidValue;
    // 16-byte cp.async: every operand base and leading dimension must be even in doubles
    if ((p.lda & 1) || (p.ldb & 1) || (reinterpret_cast<uintptr_t>(p.A) & 15) ||
        (reinterpret_cast<uintptr_t>(p.B) & 15))
        return cudaErrorInvalidValue;
    int S = std::max(1, p.splitk);
    if (p.K <= 0) S = 1;
    const bool cl = (S > 1 && S <= kMaxClusterSplit);
    if (S > 1 && !cl && (!p.work || p.N > 65535)) return cudaErrorInvalidValue;
    const int bn = (p.N <= 32 && !p.lower_out) ? 32 : 64;
    cudaError_t e;
    if (cl) e = (bn == 32) ? launch_bn<32, true>(p, S, st) : launch_bn<64, true>(p, S, st);
    else e = (bn == 32) ? launch_bn<32, false>(p, S, st) : launch_bn<64, false>(p, S, st);
    if (e != cudaSuccess || S == 1 || cl) return e;
    DVR3D_COUNT_LAUNCH(1);
    splitk_reduce_kernel<<<dim3((unsigned)((p.M + 31) / 32), (unsigned)p.N), 256, 0, st>>>(p, S);
    return cudaGetLastError();
}

}  // namespace

}  // namespace dvr3d
