// chol.cu -- FP64 Cholesky factorisation fused with the triangular inverse, recursive, on
// the DMMA GEMM (gemm_pipe.cu).
//
// For A = [[A11, .], [A21, A22]] (n1 + n2 rows, n1 a multiple of 64):
//   (1) recurse on A11                      -> inv(L11) in place
//   (2) L21 = A21 inv(L11)^T                 (GEMM, triangular second operand) -> scratch
//   (3) A22 <- A22 - L21 L21^T               (GEMM, lower tiles only)
//   (4) recurse on A22                      -> inv(L22) in place
//   (5) A21 <- -inv(L22) L21 inv(L11)        (two triangular GEMMs)
// so that on exit the lower triangle holds inv(L) with L L^T = A (the factor itself is never
// needed by the shift-invert solver). Leaves (<= 64) are factored and inverted by one CTA in
// shared memory. Work: n^3/3 (factorisation) + n^3/3 (inverse) flop, the top levels as a few
// large GEMMs instead of one thin GEMM per 64-column panel.
#include <algorithm>
#include <cmath>

#include "chol.cuh"
#include "common.cuh"
#include "gemm64.cuh"
#include "ozaki.cuh"

namespace dvr3d {

namespace {

constexpr int NB = kCholNb;
constexpr int kLeafThreads = 256;

__global__ void shift_copy_lower_kernel(const double *H, long long ldh, int n, double sigma, double *A,
                                        long long lda) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * lda) return;
    const int j = (int)(t / lda), i = (int)(t % lda);
    if (i >= n) return;
    double v = 0.0;
    if (i >= j) v = H[(size_t)j * ldh + i] - (i == j ? sigma : 0.0);
    A[(size_t)j * lda + i] = v;
}

// Cholesky of the nb x nb block at (j0, j0) (nb <= 64, lower triangle read) and inverse of
// its factor. in_place_inv = 0: the factor goes back into A; 1: the inverse replaces the
// block's lower triangle. inv_out (optional): the inverse (ld 64, zeros above).
// One right-looking sweep forms A = U D U^T (U unit lower) and, in the same steps, the
// forward substitution X = inv(U) (row k of X is final when step k starts; step k
// subtracts U[i][k] X[k] from the rows below); then L = U D^{1/2}, inv(L) = D^{-1/2} X.
// Thread (row ti, group tg) keeps columns 16 tg .. 16 tg + 15 of the matrix and of X in
// registers. The pivot column is published with zeros on and above the diagonal and row k
// of X has zeros right of its diagonal, so every step is the same 32 unmasked FMAs per
// thread (finished columns and the upper triangle take zero updates); one barrier per step.
__global__ void __launch_bounds__(kLeafThreads, 1) potrf_leaf_kernel(double *A, long long lda, int j0, int nb,
                                                                     double *inv_out, int in_place_inv,
                                                                     double rel_tol, int *err) {
    if (*(volatile int *)err != 0) return;
    __shared__ __align__(16) double colb[2][NB];
    __shared__ __align__(16) double rowb[2][NB];
    __shared__ double piv[2], rdb[2];
    __shared__ double sq[NB], rsq[NB];
    __shared__ double s_thr;
    const int tid = threadIdx.x;
    const int ti = tid & (NB - 1), tg = tid >> 6;
    constexpr int U = NB / 4;
    const int jb = tg * U;
    double own[U], x[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int j = jb + u;
        own[u] = (ti < nb && j < nb && ti >= j) ? A[(size_t)(j0 + j) * lda + j0 + ti] : 0.0;
        x[u] = (ti == j) ? 1.0 : 0.0;
        if (ti == j) sq[ti] = own[u];  // diagonal, for the pivot threshold
        if (ti == 0) rowb[0][j] = x[u];
    }
    if (tg == 0) {
        colb[0][ti] = (ti > 0) ? own[0] : 0.0;
        if (ti == 0) {
            piv[0] = own[0];
            rdb[0] = 1.0 / own[0];
        }
    }
    __syncthreads();
    if (tid < 32) {  // threshold relative to the largest diagonal entry
        double mx = 0.0;
        for (int i = tid; i < nb; i += 32) mx = fmax(mx, sq[i]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (tid == 0) s_thr = rel_tol * mx;
    }
    bool bad = false;
    for (int k = 0; k < nb; ++k) {
        const int cb = k & 1, nbuf = cb ^ 1;
        __syncthreads();
        const double d = piv[cb];
        if (!(d > s_thr) || !isfinite(d)) {  // uniform: every thread reads the same d
            bad = true;
            break;
        }
        const double lik = colb[cb][ti] * rdb[cb];  // zero on and above the pivot
        double cv[U], rv[U];
#pragma unroll
        for (int u = 0; u < U; u += 2) {
            const double2 c2 = *reinterpret_cast<const double2 *>(&colb[cb][jb + u]);
            const double2 r2 = *reinterpret_cast<const double2 *>(&rowb[cb][jb + u]);
            cv[u] = c2.x;
            cv[u + 1] = c2.y;
            rv[u] = r2.x;
            rv[u + 1] = r2.y;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            own[u] = fma(-lik, cv[u], own[u]);
            x[u] = fma(-lik, rv[u], x[u]);
        }
        const int kn = k + 1;
        if (tg == (kn >> 4) && kn < NB) {  // column k+1 is final after this step
            double v = 0.0;
            switch (kn & 15) {
#define DVR3D_PICK(c) \
    case c:           \
        v = own[c];   \
        break;
                DVR3D_PICK(0) DVR3D_PICK(1) DVR3D_PICK(2) DVR3D_PICK(3) DVR3D_PICK(4) DVR3D_PICK(5) DVR3D_PICK(6)
                DVR3D_PICK(7) DVR3D_PICK(8) DVR3D_PICK(9) DVR3D_PICK(10) DVR3D_PICK(11) DVR3D_PICK(12)
                DVR3D_PICK(13) DVR3D_PICK(14) DVR3D_PICK(15)
#undef DVR3D_PICK
            }
            colb[nbuf][ti] = (ti > kn) ? v : 0.0;
            if (ti == kn) {
                piv[nbuf] = v;
                rdb[nbuf] = 1.0 / v;
            }
        }
        if (ti == kn) {  // so is row k+1 of X
#pragma unroll
            for (int u = 0; u < U; ++u) rowb[nbuf][jb + u] = x[u];
        }
    }
    if (bad) {
        if (tid == 0) atomicExch(err, (int)kDevNotPosDef);
        return;
    }
    // L = U D^{1/2} (column j of the unscaled factor times 1/sqrt(d_j), diagonal sqrt(d_j));
    // inv(L) = D^{-1/2} X
    __syncthreads();
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int j = jb + u;
        if (ti == j && ti < nb) {
            const double r = sqrt(own[u]);
            sq[j] = r;
            rsq[j] = 1.0 / r;
        }
    }
    __syncthreads();
    const double rrow = (ti < nb) ? rsq[ti] : 0.0;
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int j = jb + u;
        const bool in = (ti < nb && j < nb && ti >= j);
        const double l = (ti == j) ? sq[j] : own[u] * rsq[j];
        const double xi = x[u] * rrow;
        if (in) A[(size_t)(j0 + j) * lda + j0 + ti] = in_place_inv ? xi : l;
        if (inv_out) inv_out[(size_t)j * NB + ti] = in ? xi : 0.0;
    }
}

// Cholesky and inverse of a b x b block (b <= 32) in one warp: lane i keeps row i of the
// matrix and of X = inv(U) in registers; step k broadcasts the pivot and column k / row k
// by shuffles (no barriers). Same results as the leaf kernel: G's lower triangle receives
// L, inv_out (ld 64) the inverse with zeros above the diagonal.
__global__ void __launch_bounds__(32) chol_warp_kernel(double *G, int b, double *inv_out, double rel_tol, int *err) {
    if (*(volatile int *)err != 0) return;
    const int i = threadIdx.x;
    constexpr unsigned kAll = 0xffffffffu;
    double own[32], x[32];
#pragma unroll
    for (int c = 0; c < 32; ++c) {
        own[c] = (i < b && c < b && c <= i) ? G[(size_t)c * b + i] : 0.0;
        x[c] = (c == i) ? 1.0 : 0.0;
    }
    double dmax = 0.0;
#pragma unroll
    for (int c = 0; c < 32; ++c)
        if (c == i) dmax = own[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(kAll, dmax, o));
    const double thr = rel_tol * dmax;
    // the step loop stays a loop (a fully unrolled one is too long for the instruction cache);
    // column k of this lane's row is picked by selects, the other rows' entries by shuffles
    bool bad = false;
#pragma unroll 1
    for (int k = 0; k < b; ++k) {
        double colk = 0.0;
#pragma unroll
        for (int c = 0; c < 32; ++c) colk = (c == k) ? own[c] : colk;
        const double d = __shfl_sync(kAll, colk, k);
        if (!(d > thr) || !isfinite(d)) {  // uniform: every lane holds the same d
            bad = true;
            break;
        }
        const double lik = (i > k && i < b) ? colk * (1.0 / d) : 0.0;
#pragma unroll
        for (int c = 0; c < 32; ++c) {
            const double ack = __shfl_sync(kAll, colk, c);  // row c's entry of column k
            own[c] -= (c > k) ? lik * ack : 0.0;
            x[c] -= lik * __shfl_sync(kAll, x[c], k);      // row k of X (zero right of k)
        }
    }
    if (bad) {
        if (i == 0) atomicExch(err, (int)kDevNotPosDef);
        return;
    }
    double di = 0.0;
#pragma unroll
    for (int c = 0; c < 32; ++c)
        if (c == i) di = own[c];
    const double sq = (i < b) ? sqrt(di) : 1.0;
    const double rs = 1.0 / sq;
#pragma unroll
    for (int c = 0; c < 32; ++c) {
        const double rsc = __shfl_sync(kAll, rs, c);
        const double sqc = __shfl_sync(kAll, sq, c);
        const bool in = (i < b && c < b && c <= i);
        if (in) G[(size_t)c * b + i] = (c == i) ? sqc : own[c] * rsc;
        if (inv_out && c < 64) inv_out[(size_t)c * NB + i] = in ? x[c] * rs : 0.0;
    }
    if (inv_out) {  // rows b..63 of the 64-row inverse block stay zero
        for (int q = i; q < NB * NB; q += 32) {
            const int c = q / NB, r = q % NB;
            if (r >= 32 || c >= 32) inv_out[q] = 0.0;
        }
    }
}

cudaError_t leaf(double *A, long long lda, int j0, int nb, double *inv_out, int in_place, double rel_tol, int *err,
                 cudaStream_t st) {
    DVR3D_COUNT_LAUNCH(1);
    potrf_leaf_kernel<<<1, kLeafThreads, 0, st>>>(A, lda, j0, nb, inv_out, in_place, rel_tol, err);
    return cudaGetLastError();
}

__global__ void copy_block_kernel(const double *S, long long lds, double *D, long long ldd, int m, int n) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)m * n) return;
    const int j = (int)(t / m), i = (int)(t % m);
    D[(size_t)j * ldd + i] = S[(size_t)j * lds + i];
}

constexpr size_t kSplitWork = (size_t)4 << 20;  // doubles of split-K scratch

int split_of(int M, int N, int K, bool lower) {
    const long long tm = (M + 63) / 64, tn = (N + 63) / 64;
    const long long tiles = lower ? tm * (tm + 1) / 2 : tm * tn;
    if (tiles >= 296) return 1;
    long long s = (600 + tiles - 1) / tiles;
    s = std::min<long long>(s, 16);
    s = std::min<long long>(s, (K + 63) / 64);
    s = std::min<long long>(s, (long long)(kSplitWork / ((size_t)M * N + 1)));
    return (int)std::max<long long>(s, 1);
}

struct Rec {
    double *A;
    long long lda;
    double *stack;     // scratch for L21 blocks, used depth-first
    double *work;      // split-K scratch
    int *err;
    cudaStream_t st;
    CholOzaki oz;      // int8-sliced products for the large GEMMs (oz.work null: DMMA only)

    cudaError_t gemm(GemmOp g) {
        if (oz.work && ozaki_profitable(g) && ozaki_supported(g, oz.nslice) &&
            ozaki_work_bytes(g, oz.nslice) <= oz.bytes) {
            ++oz.launches;
            return launch_ozaki_gemm(g, oz.nslice, oz.work, oz.bytes, err, st);
        }
        g.splitk = split_of(g.M, g.N, g.K, g.lower_out != 0);
        g.work = work;
        return launch_gemm(g, st);
    }

    cudaError_t run(int off, int n, double *sp) {
        cudaError_t e;
        if (n <= NB) return leaf(A, lda, off, n, nullptr, 1, 0.0, err, st);
        int n1 = ((n / 2 + NB - 1) / NB) * NB;
        if (n1 >= n) n1 = n - NB;
        const int n2 = n - n1;
        double *A11 = A + (size_t)off * lda + off;
        double *A21 = A11 + n1;
        double *A22 = A + (size_t)(off + n1) * lda + off + n1;
        const long long ldt = (n2 + 7) / 8 * 8;
        double *L21 = sp;
        if ((e = run(off, n1, sp)) != cudaSuccess) return e;
        GemmOp a;  // L21 = A21 inv(L11)^T
        a.M = n2;
        a.N = n1;
        a.K = n1;
        a.A = A21;
        a.lda = lda;
        a.B = A11;
        a.ldb = lda;
        a.tb = true;
        a.tri_b = 2;
        a.C = L21;
        a.ldc = ldt;
        if ((e = gemm(a)) != cudaSuccess) return e;
        GemmOp s;  // A22 -= L21 L21^T
        s.M = n2;
        s.N = n2;
        s.K = n1;
        s.alpha = -1.0;
        s.beta = 1.0;
        s.A = L21;
        s.lda = ldt;
        s.B = L21;
        s.ldb = ldt;
        s.tb = true;
        s.C = A22;
        s.ldc = lda;
        s.lower_out = 1;
        if ((e = gemm(s)) != cudaSuccess) return e;
        if ((e = run(off + n1, n2, sp + (size_t)ldt * n1)) != cudaSuccess) return e;
        GemmOp z;  // A21 <- inv(L22) L21
        z.M = n2;
        z.N = n1;
        z.K = n2;
        z.A = A22;
        z.lda = lda;
        z.tri = 1;
        z.B = L21;
        z.ldb = ldt;
        z.C = A21;
        z.ldc = lda;
        if ((e = gemm(z)) != cudaSuccess) return e;
        GemmOp c;  // L21 <- -A21 inv(L11), then back into A21
        c.M = n2;
        c.N = n1;
        c.K = n1;
        c.alpha = -1.0;
        c.A = A21;
        c.lda = lda;
        c.B = A11;
        c.ldb = lda;
        c.tri_b = 1;
        c.C = L21;
        c.ldc = ldt;
        if ((e = gemm(c)) != cudaSuccess) return e;
        DVR3D_COUNT_LAUNCH(1);
        copy_block_kernel<<<(unsigned)(((long long)n2 * n1 + 255) / 256), 256, 0, st>>>(L21, ldt, A21, lda, n2, n1);
        return cudaGetLastError();
    }
};

size_t stack_need(int n) {
    if (n <= NB) return 0;
    int n1 = ((n / 2 + NB - 1) / NB) * NB;
    if (n1 >= n) n1 = n - NB;
    const int n2 = n - n1;
    const size_t mine = (size_t)((n2 + 7) / 8 * 8) * n1;
    return std::max(stack_need(n1), mine + stack_need(n2));
}

// Largest Ozaki workspace any product of the recursion asks for (shapes as in Rec::run).
size_t oz_need(int n, int nslice) {
    if (n <= NB) return 0;
    int n1 = ((n / 2 + NB - 1) / NB) * NB;
    if (n1 >= n) n1 = n - NB;
    const int n2 = n - n1;
    static const double dummy[2] = {0.0, 0.0};
    size_t m = 0;
    const int shapes[4][4] = {{n2, n1, n1, 0}, {n2, n2, n1, 1}, {n2, n1, n2, 0}, {n2, n1, n1, 0}};
    for (const auto &sh : shapes) {
        GemmOp g;
        g.M = sh[0];
        g.N = sh[1];
        g.K = sh[2];
        g.lower_out = sh[3];
        g.A = dummy;
        g.B = dummy + 1;
        g.C = const_cast<double *>(dummy);
        if (ozaki_profitable(g) && ozaki_supported(g, nslice)) m = std::max(m, ozaki_work_bytes(g, nslice));
    }
    return std::max({m, oz_need(n1, nslice), oz_need(n2, nslice)});
}

}  // namespace

size_t chol_work_doubles(int n) { return stack_need(n) + kSplitWork + 64; }

size_t chol_ozaki_work_bytes(int n, int nslice) { return oz_need(n, nslice); }

cudaError_t launch_shift_copy_lower(const double *H, long long ldh, int n, double sigma, double *A, long long lda,
                                    cudaStream_t st) {
    const long long tot = (long long)n * lda;
    DVR3D_COUNT_LAUNCH(1);
    shift_copy_lower_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(H, ldh, n, sigma, A, lda);
    return cudaGetLastError();
}

cudaError_t launch_potrf_inv_lower(double *A, long long lda, int n, double *work, int *err, cudaStream_t st,
                                   CholOzaki *oz) {
    if (n <= 0) return cudaSuccess;
    if (lda & 1) return cudaErrorInvalidValue;
    Rec r{A, lda, work + kSplitWork + 64, work, err, st, oz ? *oz : CholOzaki{}};
    const cudaError_t e = r.run(0, n, r.stack);
    if (oz) oz->launches = r.oz.launches;
    return e;
}

cudaError_t launch_chol_small(double *G, int b, double *ginv, double rel_tol, int *err, cudaStream_t st) {
    if (b > NB) return cudaErrorInvalidValue;
    if (b <= 32) {
        DVR3D_COUNT_LAUNCH(1);
        chol_warp_kernel<<<1, 32, 0, st>>>(G, b, ginv, rel_tol, err);
        return cudaGetLastError();
    }
    return leaf(G, b, 0, b, ginv, 0, rel_tol, err, st);
}

}  // namespace dvr3d
