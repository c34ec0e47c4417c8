// tc_gemm.cuh -- Blackwell tensor-core GEMMs (tcgen05.mma kind::f16, BF16 operands, FP32
// accumulation in tensor memory) over split-BF16 operands, with TMA-staged shared memory.
//
// A double x is carried as two BF16 slices, x ~= hi + lo with hi = bf16(x) and
// lo = bf16(x - hi) (16 significant bits). The "BF16x3" product of two split matrices keeps
// the three leading slice products,
//     A B^T ~= A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T,
// each term exact in FP32 (8 x 8 significant bits) and summed in the FP32 accumulator; the
// dropped A_lo B_lo^T term and the slice rounding leave a relative error of order 2^-16.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace dvr3d {

// FP64 -> BF16 slices of a K-major operand: rows r < R, element (r, k) of the source at
// X[r * ldx + k]; hi / lo are row-major with row stride ldo (elements, a multiple of 8).
// lo may be null (one slice).
cudaError_t launch_split_bf16(const double *X, long long ldx, int R, int K, __nv_bfloat16 *hi,
                              __nv_bfloat16 *lo, long long ldo, cudaStream_t st);

// S (n x n, lds) = hi + lo in FP64 (the split matrix as the products see it).
cudaError_t launch_split_sum(const __nv_bfloat16 *hi, const __nv_bfloat16 *lo, long long lds, int n, double *S,
                             cudaStream_t st);

enum TcEpilogue : int {
    kTcStore = 0,     // C[i * cm + j * cn] = alpha * acc + beta * C[...]  (FP64 C)
    kTcAssemble = 1,  // contracted-Hamiltonian assembly, see TcGemm
};

// C (M x N) = sum of the slice products of A (M x K) and B (N x K), both row-major BF16 with
// K contiguous (row strides lda / ldb in elements, multiples of 8; 16-byte aligned bases).
//   nslice = 1: A_hi B_hi^T;  nslice = 2: the BF16x3 product above.
// kTcAssemble: A == B == the contracted basis (row i = basis function i over the P grid
//   points, K = P, M = N = n); only lower 128 x 128 tiles run and each value
//       v(i, j) = acc(i, j) * T[g(j) * ldt + g(i)] + (i == j ? e2[i] : 0)
//   is written to (i, j) and (j, i) of H (FP64, ldh) or, when H is null, split into the BF16
//   slices H_hi / H_lo (ldh) of the Hamiltonian the split products then use.
struct TcGemm {
    int M = 0, N = 0, K = 0;
    int nslice = 2;
    const __nv_bfloat16 *A_hi = nullptr, *A_lo = nullptr;
    long long lda = 0;
    const __nv_bfloat16 *B_hi = nullptr, *B_lo = nullptr;
    long long ldb = 0;
    int epilogue = kTcStore;
    // kTcStore
    double *C = nullptr;
    long long cm = 0, cn = 0;
    double alpha = 1.0, beta = 0.0;
    // kTcAssemble
    const int *g = nullptr;
    const double *T = nullptr;
    int ldt = 0;
    const double *e2 = nullptr;
    double *H = nullptr;
    __nv_bfloat16 *H_hi = nullptr, *H_lo = nullptr;
    long long ldh = 0;
    // error flag (device int, may be null): set to kDevBarrierTimeout when a pipeline wait
    // ran past wait_ns nanoseconds (0: 4 s); the tile is then left unwritten
    int *err = nullptr;
    unsigned long long wait_ns = 0;
};

// Checks the operands (sizes, alignment, strides) and launches; cudaErrorInvalidValue when a
// requirement does not hold, before anything is launched.
cudaError_t launch_tc_gemm(const TcGemm &p, cudaStream_t st);

// Algorithmic FP64-equivalent flops of one launch: 2 M N K (kTcAssemble: the lower tiles'
// share of 2 n^2 K), independent of the number of slice products.
double tc_gemm_alg_flops(const TcGemm &p);

}  // namespace dvr3d
