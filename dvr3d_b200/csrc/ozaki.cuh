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

// Same operation and operand conventions as launch_gemm (GemmOp: op(A) M x K, op(B) K x N,
// column-major C, tri / tri_b / lower_out, alpha, beta; splitk and work are ignored), computed
// from nslice signed 7-bit slices of each operand with exact int32 accumulation.
// False when the product is outside the exactness limits (K > kOzMaxK) or malformed.
bool ozaki_supported(const GemmOp &p, int nslice);
// Products large enough that slicing pays for itself (the tensor-core main loop dominates).
bool ozaki_profitable(const GemmOp &p);
// Device workspace (bytes) launch_ozaki_gemm needs for this product.
size_t ozaki_work_bytes(const GemmOp &p, int nslice);
// err (device int, may be null) receives kDevBarrierTimeout if a pipeline wait runs out.
cudaError_t launch_ozaki_gemm(const GemmOp &p, int nslice, void *work, size_t work_bytes, int *err,
                              cudaStream_t st);
// Algorithmic FP64-equivalent flops of the product (as gemm_alg_flops).
double ozaki_alg_flops(const GemmOp &p);

}  // namespace dvr3d
