// h3_apply.cu -- the contracted Hamiltonian applied in FP64 without forming it.
//
// The assembly (bloc3d / blc2d2 / vecmul, :3455-3595, Radau; mkham3 / loadh, :2301-2609,
// Jacobi) builds H3 block pair by block pair as T[g, g'] C_g^T C_g' plus the 2D eigenvalues
// on the diagonal, C_g the contracted functions of block (angle) g over the P grid points.
// Its product with vectors factorises through the grid:
//     (H3 X)_g = C_g^T Z_g + e2_g o X_g,   Z_g = sum_g' T[g, g'] Y_g',   Y_g' = C_g' X_g',
// 4 P N + 2 P G^2 flops per vector (G blocks) against 2 N^2 for the assembled matrix. The
// split-BF16 solve uses it as its FP64 operator (the residual correction).
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "gemm64.cuh"
#include "pipeline.cuh"

#define CK(x)                                          \
    do {                                               \
        cudaError_t e_ = (x);                          \
        if (e_ != cudaSuccess) throw CudaFail{e_, #x}; \
    } while (0)

namespace dvr3d {

namespace {

// Y[:, j] += e2 o X[:, j]
__global__ void add_diag_kernel(const double *e2, const double *X, long long ldx, int N, int nvec, double *Y,
                                long long ldy) {
    const int j = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        Y[(size_t)j * ldy + i] += e2[i] * X[(size_t)j * ldx + i];
}

template <class T>
T *upload_vec(dvr3d_ctx *ctx, const char *name, const std::vector<T> &v) {
    T *p = ctx->arena.get_t<T>(name, v.size());
    CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    note_h2d((long long)(v.size() * sizeof(T)));
    return p;
}

}  // namespace

void apply_h3_fp64(dvr3d_ctx *ctx, const Contracted &C, const double *X, long long ldx, int nvec, double *Y,
                   long long ldy) {
    if (nvec <= 0 || C.N <= 0) return;
    cudaStream_t st = ctx->stream;
    const int nb = C.nblocks, P = C.P;
    const long long pn = (long long)P * nvec;
    double *Yg = ctx->arena.get_t<double>("ha_y", (size_t)pn * nb);
    double *Zg = ctx->arena.get_t<double>("ha_z", (size_t)pn * nb);
    // per-block offsets and 64 x 64 tile counts of the two grouped products
    std::vector<int> M1(nb), K1(nb), ts1(nb + 1, 0), M3(nb), K3(nb), ts3(nb + 1, 0);
    std::vector<long long> a1(nb), b1(nb), c1(nb), a3(nb), b3(nb), c3(nb);
    const int tn = (nvec + 63) / 64;
    int col0 = 0;
    for (int g = 0; g < nb; ++g) {
        const int s = C.iv2[g];
        // Y_g (P x nvec, ld P) = C_g (P x s, columns col0.. of Vt) X_g (rows col0.. of X)
        M1[g] = P;
        K1[g] = s;
        a1[g] = (long long)col0 * C.ldv;
        b1[g] = col0;
        c1[g] = (long long)g * pn;
        ts1[g + 1] = ts1[g] + ((P + 63) / 64) * tn;
        // (H3 X)_g (s x nvec) = C_g^T Z_g
        M3[g] = s;
        K3[g] = P;
        a3[g] = (long long)col0 * C.ldv;
        b3[g] = (long long)g * pn;
        c3[g] = col0;
        ts3[g + 1] = ts3[g] + ((s + 63) / 64) * tn;
        col0 += s;
    }
    GroupedGemm g1{};
    g1.ngroups = nb;
    g1.tile_start = upload_vec(ctx, "ha_ts1", ts1);
    g1.M = upload_vec(ctx, "ha_m1", M1);
    g1.K = upload_vec(ctx, "ha_k1", K1);
    g1.N = nvec;
    g1.A = C.Vt;
    g1.aoff = upload_vec(ctx, "ha_a1", a1);
    g1.lda = C.ldv;
    g1.B = X;
    g1.boff = upload_vec(ctx, "ha_b1", b1);
    g1.ldb = ldx;
    g1.C = Yg;
    g1.coff = upload_vec(ctx, "ha_c1", c1);
    g1.ldc = P;
    g1.alpha = 1.0;
    g1.beta = 0.0;
    launch_grouped_dgemm(g1, false, ts1[nb], st);
    CK(cudaGetLastError());
    // Z (P nvec x G) = Y (P nvec x G) T^T, T[g' * ldt + g] = T(g, g')
    launch_dgemm(false, true, (int)pn, nb, nb, 1.0, Yg, pn, C.T, C.ldt, 0.0, Zg, pn, st);
    CK(cudaGetLastError());
    GroupedGemm g3{};
    g3.ngroups = nb;
    g3.tile_start = upload_vec(ctx, "ha_ts3", ts3);
    g3.M = upload_vec(ctx, "ha_m3", M3);
    g3.K = upload_vec(ctx, "ha_k3", K3);
    g3.N = nvec;
    g3.A = C.Vt;
    g3.aoff = upload_vec(ctx, "ha_a3", a3);
    g3.lda = C.ldv;
    g3.B = Zg;
    g3.boff = upload_vec(ctx, "ha_b3", b3);
    g3.ldb = P;
    g3.C = Y;
    g3.coff = upload_vec(ctx, "ha_c3", c3);
    g3.ldc = ldy;
    g3.alpha = 1.0;
    g3.beta = 0.0;
    launch_grouped_dgemm(g3, true, ts3[nb], st);
    CK(cudaGetLastError());
    DVR3D_COUNT_LAUNCH(1);
    add_diag_kernel<<<dim3((unsigned)std::min(64, (C.N + 255) / 256), (unsigned)nvec), 256, 0, st>>>(
        C.e2, X, ldx, C.N, nvec, Y, ldy);
    CK(cudaGetLastError());
}

}  // namespace dvr3d
