// ozaki.cuh -- FP64-accurate GEMM on the int8 tensor cores (Ozaki scheme with integer slices).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "gemm64.cuh"

namespace dvr3d {

constexpr int kOzMinSlices = 4;
constexpr int kOzMaxSlices = 8;
constexpr int kOzDefaultSlices = 8;
// Exactness limit of the int32 accumulators: one accumulator sums up to nslice slice products
// of K terms each of magnitude <= 127^2, so nslice * 127^2 * K < 2^31 (K <= 16640 at 8 slices).
constexpr int kOzMaxK = 16384;
// K chunk of the thin Krylov products (one CTA per 128-row tile and chunk)
constexpr int kOzKrylovChunk = 1024;

// Same operation and operand conventions as launch_gemm (GemmOp: op(A) M x K, op(B) K x N,
// column-major C, tri / tri_b / lower_out, alpha, beta; splitk and work are ignored), computed
// from nslice signed 7-bit slices of each operand with exact int32 accumulation.
// False when the product is outside the exactness limits (K > kOzMaxK) or malformed.
bool ozaki_supported(const GemmOp &p, int nslice);
// Products large enough that slicing pays for itself (the tensor-core main loop dominates).
bool ozaki_profitable(const GemmOp &p);
// op(A) of a product sliced once and kept (the shift-invert solve slices inv(L) once per
// factorisation and multiplies it into every Krylov block).
struct OzPresliced {
    const signed char *S = nullptr;          // nslice slices of rows x Kp bytes
    const unsigned long long *umax = nullptr;  // per-row max |op(A)| bit patterns
    int rows = 0, K = 0, nslice = 0, tri = 0;
};
size_t ozaki_preslice_bytes(const GemmOp &p, int nslice);
cudaError_t ozaki_preslice_a(const GemmOp &p, int nslice, void *buf, size_t bytes, OzPresliced &out,
                             cudaStream_t st);
// Device workspace (bytes) launch_ozaki_gemm needs for this product (with op(A) presliced or
// not, with K chunks of kchunk or not).
size_t ozaki_work_bytes(const GemmOp &p, int nslice, bool presliced_a = false, int kchunk = 0);
// err (device int, may be null) receives kDevBarrierTimeout if a pipeline wait runs out.
// pre: op(A) from ozaki_preslice_a of the same operand (A, lda, ta, tri, M, K) instead of
// slicing it here. kchunk (multiple of 64, 0 = off): the K range is split into chunks of
// kchunk, one CTA per (tile, chunk) writing its partial sum, then one reduction kernel sums
// the chunks in order (deterministic) -- for thin products (N <= 32) with few row tiles.
cudaError_t launch_ozaki_gemm(const GemmOp &p, int nslice, void *work, size_t work_bytes, int *err,
                              cudaStream_t st, const OzPresliced *pre = nullptr, int kchunk = 0);
// The per-device kernel attribute (and the tensor-map encoder lookup) that the first launch of
// this product's configuration would set: call before capturing such launches in a CUDA graph.
cudaError_t ozaki_set_attributes(const GemmOp &p, int nslice);
// Algorithmic FP64-equivalent flops of the product (as gemm_alg_flops).
double ozaki_alg_flops(const GemmOp &p);

}  // namespace dvr3d
