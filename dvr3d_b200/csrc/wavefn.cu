// wavefn.cu -- wavefunction amplitudes on the DVR grid (the reference's trans / transr).
//
// The reference writes, when ZTRAN is set, every returned level as its amplitudes on the
// DVR grid: transr (:3596-3643, Radau) sums vecs2d(irs, j) ham3(j, level) over the kept 2D
// states j of each angle; trans (:3649-3843, Jacobi) forms phi = 1D x 2D vectors on the
// (a, b) grid of every last-coordinate point and sums phi ham3(., level). Both are, per block
// g of the contracted basis,
//     psi_g (P x nlev) = C_g (P x s_g) Z_g (s_g x nlev),
// with C_g the block's basis functions on its P grid points and Z_g the block's rows of the
// final eigenvectors. Here C_g is the block's slice of the device-resident contracted basis
// Vt (whose rows carry the sqrt(w_p) factor of the assembly, divided out again), so the
// back-transform is one DMMA GEMM per block (gemm_pipe.cu) and one scatter into the record
// layout; only the records come back to the host.
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

// Zp[colp[b] + i, l] = Z[col0[b] + i, l] for i < s[b]: block b's rows at an even row offset
// (16-byte aligned GEMM operand). One thread per (row of the packed layout, level).
__global__ void wave_pack_kernel(const double *Z, long long ldz, const int *blk_of_row, const int *col0,
                                 const int *colp, int nrowp, int nlev, double *Zp, long long ldzp) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nrowp * nlev) return;
    const int r = (int)(t % nrowp), l = (int)(t / nrowp);
    const int b = blk_of_row[r];
    double v = 0.0;
    if (b >= 0) v = Z[(size_t)l * ldz + col0[b] + (r - colp[b])];
    Zp[(size_t)l * ldzp + r] = v;
}

// out[l * len + fidx[q]] = Psi[q + l * ldpsi] / sw[q % P] for q < nblk * P (fidx < 0: unused)
__global__ void wave_scatter_kernel(const double *Psi, long long ldpsi, const long long *fidx, const double *sw,
                                    int P, long long nq, int nlev, long long len, double *out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nq * nlev) return;
    const long long q = t % nq;
    const int l = (int)(t / nq);
    const long long f = fidx[q];
    if (f < 0) return;
    out[(size_t)l * len + f] = Psi[(size_t)l * ldpsi + q] / sw[q % P];
}

inline unsigned nb256(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

void compute_wavefunctions(dvr3d_ctx *ctx, const BlockPlan &p, const Contracted &C, const double *Z, long long ldz,
                           int nlev, WaveOut &wave) {
    cudaStream_t st = ctx->stream;
    const int nb = C.nblocks, P = C.P;
    wave.nlev = nlev;
    wave.psi.clear();
    if (nlev <= 0 || nb <= 0 || !Z) return;
    // record layout: fidx[b * P + q] = position of block b's grid point q in one record
    std::vector<long long> fidx((size_t)nb * P, -1);
    long long len;
    if (p.radau) {
        // transr: wvfunc(index), index running over the pair irs (outer) and the angles
        // with kept states (inner); nbass = iang * max2d entries (zero beyond)
        int iang = 0;
        std::vector<int> rank(nb, -1);
        for (int b = 0; b < nb; ++b)
            if (C.iv2[b] > 0) rank[b] = iang++;
        len = (long long)iang * p.max2d;
        for (int b = 0; b < nb; ++b)
            if (rank[b] >= 0)
                for (int q = 0; q < P; ++q) fidx[(size_t)b * P + q] = (long long)q * iang + rank[b];
    } else {
        // trans: psi(idvr, npnt1, npnt2), Fortran order; grid point q = ia * npntb + ib of the
        // (a, b) pair of block ic, the coordinate order set by ZTHETA and ZR2R1
        const long long I = p.idvr, n1 = p.npnt1;
        len = I * p.npnt1 * p.npnt2;
        for (int ic = 0; ic < nb; ++ic)
            for (int ia = 0; ia < p.npnta; ++ia)
                for (int ib = 0; ib < p.npntb; ++ib) {
                    long long f;
                    if (!p.ztheta) f = p.zr2r1 ? ic + I * (ib + n1 * ia) : ic + I * (ia + n1 * ib);
                    else f = p.zr2r1 ? ia + I * (ic + n1 * ib) : ia + I * (ib + n1 * ic);
                    fidx[(size_t)ic * P + (size_t)ia * p.npntb + ib] = f;
                }
    }
    wave.len = len;
    // packed eigenvector rows: block b at an even offset colp[b]
    std::vector<int> col0(nb, 0), colp(nb, 0), sz(nb, 0);
    int c = 0, cp = 0;
    for (int b = 0; b < nb; ++b) {
        col0[b] = c;
        colp[b] = cp;
        sz[b] = C.iv2[b];
        c += sz[b];
        cp += (sz[b] + 1) & ~1;
    }
    const int nrowp = std::max(cp, 2);
    std::vector<int> blk_of_row(nrowp, -1);
    for (int b = 0; b < nb; ++b)
        for (int i = 0; i < sz[b]; ++i) blk_of_row[colp[b] + i] = b;
    auto up = [&](const char *name, const auto &v) {
        using T = typename std::decay_t<decltype(v)>::value_type;
        T *d = ctx->arena.get_t<T>(name, std::max<size_t>(v.size(), 1));
        CK(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        note_h2d((long long)(v.size() * sizeof(T)));
        return d;
    };
    const long long ldzp = (nrowp + 1) & ~1LL;
    double *Zp = ctx->arena.get_t<double>("wf_zp", (size_t)ldzp * nlev);
    DVR3D_COUNT_LAUNCH(1);
    wave_pack_kernel<<<nb256((long long)nrowp * nlev), 256, 0, st>>>(Z, ldz, up("wf_bor", blk_of_row), up("wf_c0", col0),
                                                                       up("wf_cp", colp), nrowp, nlev, Zp, ldzp);
    CK(cudaGetLastError());
    const long long nq = (long long)nb * P;
    double *Psi = ctx->arena.get_t<double>("wf_psi", (size_t)nq * nlev);
    for (int b = 0; b < nb; ++b) {
        if (sz[b] == 0) continue;
        GemmOp g;  // Psi[b P : (b+1) P, :] = Vt[:, col0 b ...] Zp[colp b ..., :]
        g.M = P;
        g.N = nlev;
        g.K = sz[b];
        g.A = C.Vt + (size_t)col0[b] * C.ldv;
        g.lda = C.ldv;
        g.B = Zp + colp[b];
        g.ldb = ldzp;
        g.C = Psi + (size_t)b * P;
        g.ldc = nq;
        CK(launch_gemm(g, st));
    }
    double *out = ctx->arena.get_t<double>("wf_out", (size_t)len * nlev);
    CK(cudaMemsetAsync(out, 0, sizeof(double) * len * nlev, st));
    DVR3D_COUNT_LAUNCH(1);
    wave_scatter_kernel<<<nb256(nq * nlev), 256, 0, st>>>(Psi, nq, up("wf_fidx", fidx), up("wf_sw", C.sw), P, nq, nlev,
                                                         len, out);
    CK(cudaGetLastError());
    wave.psi.resize((size_t)len * nlev);
    CK(cudaMemcpyAsync(wave.psi.data(), out, sizeof(double) * len * nlev, cudaMemcpyDeviceToHost, st));
    note_d2h((long long)(sizeof(double) * len * nlev));
    CK(cudaStreamSynchronize(st));
}

}  // namespace dvr3d
