// davidson.cu -- block-Davidson solver for the lowest levels of the contracted Hamiltonian.
//
// The reference diagonalises the assembled final Hamiltonian completely (diag3d -> dsyev,
// :2661-2764) although only NEVAL levels are kept. Here the lowest levels are found
// iteratively, and the Hamiltonian is never formed: with C_g the sqrt(w)-scaled contracted
// basis functions of block g (columns of Vt, P rows each),
//     H3 v = blockdiag(C_g^T) (T (x) I_P) blockdiag(C_g) v + e2 o v,
// i.e. per block of vectors: Y_g = C_g V_g (grouped GEMM), Z = Y T (GEMM over blocks),
// (HV)_g = C_g^T Z_g (grouped GEMM). That is ~(4 P N + 2 P nblk^2) flop per vector instead
// of 2 N^2, and only Vt (P x N) is read instead of an N x N matrix.
//
// Iteration (thick-restarted block Davidson with locking):
//   Rayleigh-Ritz on the current basis S (G = S^T H S, m <= 160, solved in shared memory)
//   -> Ritz pairs and FP64 residuals -> leading converged pairs are locked (removed from
//   the search space, later corrections are orthogonalised against them) -> corrections for
//   the next `block` unconverged pairs from the preconditioner -> orthogonalised against the
//   locked vectors and the Ritz vectors (classical Gram-Schmidt, twice), orthonormalised
//   through the eigen-decomposition of their Gram matrix (near-dependent directions dropped)
//   -> appended with their H images.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "gemm64.cuh"
#include "pipeline.cuh"
#include "small_syev.cuh"

#define CK(x)                                          \
    do {                                               \
        cudaError_t e_ = (x);                          \
        if (e_ != cudaSuccess) throw CudaFail{e_, #x}; \
    } while (0)

namespace dvr3d {

namespace {

constexpr int kMaxSub = kSmallSyevMax;  // largest Rayleigh-Ritz problem (shared memory)

// diag(H3)_i = e2_i + T[g_i, g_i] ||Vt[:, i]||^2 ; one warp per column
__global__ void hdiag_kernel(const double *Vt, long long ldv, int P, int N, const int *g, const double *T,
                             int ldt, const double *e2, double *hd) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= N) return;
    const double *c = Vt + (size_t)w * ldv;
    double s = 0.0;
    for (int p = lane; p < P; p += 32) s += c[p] * c[p];
    s = warp_sum(s);
    if (lane == 0) hd[w] = e2[w] + T[(size_t)g[w] * ldt + g[w]] * s;
}

__global__ void unit_columns_kernel(double *S, long long ld, int N, const int *idx, int m) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * m) return;
    const int j = (int)(t / N), i = (int)(t % N);
    S[(size_t)j * ld + i] = (i == idx[j]) ? 1.0 : 0.0;
}

// HV += e2 o V
__global__ void add_diag_kernel(const double *e2, const double *V, long long ldv, double *HV, long long ldh, int N,
                                int b) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * b) return;
    const int j = (int)(t / N), i = (int)(t % N);
    HV[(size_t)j * ldh + i] += e2[i] * V[(size_t)j * ldv + i];
}

// R[:, j] = HX[:, j] - w_j X[:, j], rn[j] = ||R[:, j]||; one CTA per column
__global__ void residual_kernel(const double *X, const double *HX, long long ld, const double *w, int N, double *R,
                                double *rn) {
    const int j = blockIdx.x;
    const double wj = w[j];
    double s = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const double r = HX[(size_t)j * ld + i] - wj * X[(size_t)j * ld + i];
        R[(size_t)j * ld + i] = r;
        s += r * r;
    }
    __shared__ double red[32];
    s = block_sum(s, red);
    if (threadIdx.x == 0) rn[j] = sqrt(s);
}

// Davidson (diagonal) preconditioner: t_i = r_i / (theta - d_i), safeguarded
__global__ void precond_diag_kernel(const double *R, long long ldr, const double *w, const double *hd, int N, int nb,
                                    double *Tc, long long ldt) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * nb) return;
    const int j = (int)(t / N), i = (int)(t % N);
    double den = w[j] - hd[i];
    const double eps = 1.0e-6;
    if (fabs(den) < eps) den = (den < 0.0) ? -eps : eps;
    Tc[(size_t)j * ldt + i] = R[(size_t)j * ldr + i] / den;
}

// dst[:, j] = src[:, j] for j < ncol (contiguous columns, same leading dimension)
__global__ void copy_cols_kernel(const double *src, double *dst, long long ld, int N, int ncol) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * ncol) return;
    const int j = (int)(t / N), i = (int)(t % N);
    dst[(size_t)j * ld + i] = src[(size_t)j * ld + i];
}

// Q[:, j] *= s[j]
__global__ void scale_cols_kernel(double *Q, long long ld, int n, const double *s, int ncol) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * ncol) return;
    const int j = (int)(t / n), i = (int)(t % n);
    Q[(size_t)j * ld + i] *= s[j];
}

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

// The contracted-basis operator.
class MatFree {
  public:
    MatFree(dvr3d_ctx *ctx, const Contracted &C) : ctx_(ctx), C_(C) {
        const int nb = C.nblocks;
        col0_.assign(nb, 0);
        s_.assign(nb, 0);
        int c = 0;
        for (int b = 0; b < nb; ++b) {
            col0_[b] = c;
            s_[b] = C.iv2[b];
            c += s_[b];
        }
    }
    // HV (ld ldh) = H3 V (ld ldv), b columns
    void apply(const double *V, long long ldv, int b, double *HV, long long ldh, DavidsonStats &st) {
        cudaStream_t s = ctx_->stream;
        const int nbk = C_.nblocks, P = C_.P;
        const long long PB = (long long)P * b;
        double *Y = ctx_->arena.get_t<double>("dv_Y", (size_t)PB * nbk);
        double *Z = ctx_->arena.get_t<double>("dv_Zm", (size_t)PB * nbk);
        const int tn = (b + 63) / 64;
        // metadata of the two grouped products
        std::vector<int> ts1(nbk + 1), ts2(nbk + 1), M1(nbk), K1(nbk), M2(nbk), K2(nbk);
        std::vector<long long> a1(nbk), b1(nbk), c1(nbk), b2(nbk), c2(nbk);
        ts1[0] = ts2[0] = 0;
        for (int g = 0; g < nbk; ++g) {
            M1[g] = P;
            K1[g] = s_[g];
            a1[g] = (long long)col0_[g] * C_.ldv;
            b1[g] = col0_[g];
            c1[g] = (long long)g * PB;
            ts1[g + 1] = ts1[g] + ((P + 63) / 64) * tn;
            M2[g] = s_[g];
            K2[g] = P;
            b2[g] = (long long)g * PB;
            c2[g] = col0_[g];
            ts2[g + 1] = ts2[g] + ((s_[g] + 63) / 64) * tn;
        }
        auto up = [&](const char *nm, const auto &v) {
            using T = typename std::decay_t<decltype(v)>::value_type;
            T *p = ctx_->arena.get_t<T>(nm, v.size());
            CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
            return p;
        };
        if (!ev_[0]) {
            CK(cudaEventCreate(&ev_[0]));
            CK(cudaEventCreate(&ev_[1]));
        }
        CK(cudaEventRecord(ev_[0], s));
        GroupedGemm g1{};
        g1.ngroups = nbk;
        g1.tile_start = up("mf_ts1", ts1);
        g1.M = up("mf_M1", M1);
        g1.K = up("mf_K1", K1);
        g1.N = b;
        g1.A = C_.Vt;
        g1.aoff = up("mf_a1", a1);
        g1.lda = C_.ldv;
        g1.B = V;
        g1.boff = up("mf_b1", b1);
        g1.ldb = ldv;
        g1.C = Y;
        g1.coff = up("mf_c1", c1);
        g1.ldc = P;
        g1.alpha = 1.0;
        g1.beta = 0.0;
        launch_grouped_dgemm(g1, false, ts1[nbk], s);
        launch_dgemm(false, false, (int)PB, nbk, nbk, 1.0, Y, PB, C_.T, C_.ldt, 0.0, Z, PB, s);
        GroupedGemm g2{};
        g2.ngroups = nbk;
        g2.tile_start = up("mf_ts2", ts2);
        g2.M = up("mf_M2", M2);
        g2.K = up("mf_K2", K2);
        g2.N = b;
        g2.A = C_.Vt;
        g2.aoff = g1.aoff;
        g2.lda = C_.ldv;
        g2.B = Z;
        g2.boff = up("mf_b2", b2);
        g2.ldb = P;
        g2.C = HV;
        g2.coff = up("mf_c2", c2);
        g2.ldc = ldh;
        g2.alpha = 1.0;
        g2.beta = 0.0;
        launch_grouped_dgemm(g2, true, ts2[nbk], s);
        add_diag_kernel<<<nblk((long long)C_.N * b, 256), 256, 0, s>>>(C_.e2, V, ldv, HV, ldh, C_.N, b);
        DVR3D_COUNT_LAUNCH(2);
        CK(cudaGetLastError());
        CK(cudaEventRecord(ev_[1], s));
        pending_ = true;
        st.matvecs += b;
        st.hv_flops += (4.0 * P * (double)C_.N + 2.0 * P * (double)nbk * nbk) * b;
        st.hv_launches += 4;
    }
    // accumulate the device time of the last application (after a stream sync)
    void collect(DavidsonStats &st) {
        if (!pending_) return;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
        st.hv_ms += ms;
        pending_ = false;
    }
    ~MatFree() {
        for (auto e : ev_)
            if (e) cudaEventDestroy(e);
    }

  private:
    dvr3d_ctx *ctx_;
    const Contracted &C_;
    std::vector<int> col0_, s_;
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    bool pending_ = false;
};

template <class T>
std::vector<T> d2h(dvr3d_ctx *ctx, const T *p, size_t n) {
    std::vector<T> v(n);
    if (n) CK(cudaMemcpyAsync(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return v;
}

// Eigen-decomposition of one m x m matrix (lower triangle) on the device.
void syev_small(dvr3d_ctx *ctx, const double *G, int m, double *w, double *Zv) {
    cudaStream_t s = ctx->stream;
    int *dn = ctx->arena.get_t<int>("ss_n", 1);
    long long *doff = ctx->arena.get_t<long long>("ss_off", 1);
    CK(cudaMemcpyAsync(dn, &m, sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(doff, 0, sizeof(long long), s));
    double *work = ctx->arena.get_t<double>("ss_work", (size_t)small_syev_work_doubles(kMaxSub));
    SmallSyev p{};
    p.nmat = 1;
    p.n = dn;
    p.A = G;
    p.aoff = doff;
    p.lda = nullptr;
    p.W = w;
    p.woff = doff;
    p.Z = Zv;
    p.zoff = doff;
    p.work = work;
    p.workoff = doff;
    CK(launch_small_syev(p, m, s));
}

}  // namespace

void davidson_solve(dvr3d_ctx *ctx, const Contracted &C, const dvr3d_options &opt, int nwant, double *wv_dev,
                    std::vector<double> &rn_host, double *evec_dev, DavidsonStats &stats) {
    cudaStream_t st = ctx->stream;
    const int N = C.N;
    nwant = std::min(nwant, N);
    const int bsz = std::max(8, std::min(opt.block > 0 ? opt.block : 48, kMaxSub / 3));
    const int mmax = std::min(kMaxSub, N);
    const int nkeep = std::max(1, mmax - bsz);  // Ritz vectors kept at each restart
    const double tol_cm = opt.tol_cm > 0.0 ? opt.tol_cm : 1.0e-4;
    // residual bound for an eigenvalue error of tol_cm with gaps >= 1e-5 Eh
    const double rtol = std::sqrt(tol_cm / 2.19474624e5 * 1.0e-5);
    const int max_iter = opt.max_iter > 0 ? opt.max_iter : 400;
    const long long ld = N;
    double *S = ctx->arena.get_t<double>("dv_S", (size_t)ld * mmax);
    double *HS = ctx->arena.get_t<double>("dv_HS", (size_t)ld * mmax);
    double *X = ctx->arena.get_t<double>("dv_X", (size_t)ld * mmax);
    double *HX = ctx->arena.get_t<double>("dv_HX", (size_t)ld * mmax);
    double *R = ctx->arena.get_t<double>("dv_R", (size_t)ld * mmax);
    double *Tc = ctx->arena.get_t<double>("dv_T", (size_t)ld * bsz);
    double *T2 = ctx->arena.get_t<double>("dv_T2", (size_t)ld * bsz);
    double *L = ctx->arena.get_t<double>("dv_L", (size_t)ld * (nwant + mmax));
    double *G = ctx->arena.get_t<double>("dv_G", (size_t)mmax * mmax);
    double *Yr = ctx->arena.get_t<double>("dv_Yr", (size_t)mmax * mmax);
    double *wr = ctx->arena.get_t<double>("dv_wr", mmax);
    double *rn = ctx->arena.get_t<double>("dv_rn", mmax);
    double *proj = ctx->arena.get_t<double>("dv_proj", (size_t)(nwant + mmax) * bsz);
    double *hd = ctx->arena.get_t<double>("dv_hd", N);
    double *dsc = ctx->arena.get_t<double>("dv_sc", mmax);
    MatFree H(ctx, C);
    hdiag_kernel<<<nblk((long long)N * 32, 256), 256, 0, st>>>(C.Vt, C.ldv, C.P, N, C.g, C.T, C.ldt, C.e2, hd);
    DVR3D_COUNT_LAUNCH(1);
    // start: unit vectors at the lowest diagonal entries
    std::vector<double> hdh = d2h(ctx, hd, N);
    std::vector<int> order(N);
    std::iota(order.begin(), order.end(), 0);
    const int m0 = std::min(mmax - bsz, N);
    std::partial_sort(order.begin(), order.begin() + m0, order.end(),
                      [&](int a, int b) { return hdh[a] < hdh[b]; });
    order.resize(m0);
    int *didx = ctx->arena.get_t<int>("dv_idx", m0);
    CK(cudaMemcpyAsync(didx, order.data(), sizeof(int) * m0, cudaMemcpyHostToDevice, st));
    unit_columns_kernel<<<nblk((long long)N * m0, 256), 256, 0, st>>>(S, ld, N, didx, m0);
    DVR3D_COUNT_LAUNCH(1);
    H.apply(S, ld, m0, HS, ld, stats);
    int m = m0, nl = 0;
    std::vector<double> lval, lres;
    int it = 0;
    for (; it < max_iter && nl < nwant; ++it) {
        // Rayleigh-Ritz
        launch_dgemm(true, false, m, m, N, 1.0, S, ld, HS, ld, 0.0, G, m, st);
        syev_small(ctx, G, m, wr, Yr);
        const int nx = std::min(m, nkeep);
        launch_dgemm(false, false, N, nx, m, 1.0, S, ld, Yr, m, 0.0, X, ld, st);
        launch_dgemm(false, false, N, nx, m, 1.0, HS, ld, Yr, m, 0.0, HX, ld, st);
        residual_kernel<<<nx, 256, 0, st>>>(X, HX, ld, wr, N, R, rn);
        DVR3D_COUNT_LAUNCH(1);
        CK(cudaGetLastError());
        std::vector<double> wh = d2h(ctx, wr, nx);
        std::vector<double> rh = d2h(ctx, rn, nx);
        H.collect(stats);
        // lock the leading converged Ritz pairs
        int c = 0;
        while (c < nx && nl + c < nwant && rh[c] < rtol) ++c;
        if (c > 0) {
            copy_cols_kernel<<<nblk((long long)N * c, 256), 256, 0, st>>>(X, L + (size_t)nl * ld, ld, N, c);
            DVR3D_COUNT_LAUNCH(1);
            for (int j = 0; j < c; ++j) {
                lval.push_back(wh[j]);
                lres.push_back(rh[j]);
            }
            nl += c;
            if (nl >= nwant) break;
        }
        // restart from the unlocked Ritz vectors
        const int keep = nx - c;
        std::swap(S, X);
        std::swap(HS, HX);
        if (c > 0) {
            // shift columns c..nx-1 to the front (through the other buffer pair)
            copy_cols_kernel<<<nblk((long long)N * keep, 256), 256, 0, st>>>(S + (size_t)c * ld, X, ld, N, keep);
            copy_cols_kernel<<<nblk((long long)N * keep, 256), 256, 0, st>>>(HS + (size_t)c * ld, HX, ld, N, keep);
            DVR3D_COUNT_LAUNCH(2);
            std::swap(S, X);
            std::swap(HS, HX);
        }
        m = keep;
        // corrections for the next unconverged pairs
        const int nb = std::min(bsz, keep);
        if (nb <= 0) break;
        precond_diag_kernel<<<nblk((long long)N * nb, 256), 256, 0, st>>>(R + (size_t)c * ld, ld, wr + c, hd, N, nb,
                                                                          Tc, ld);
        DVR3D_COUNT_LAUNCH(1);
        // orthogonalise against locked and current vectors, twice
        for (int pass = 0; pass < 2; ++pass) {
            if (nl > 0) {
                launch_dgemm(true, false, nl, nb, N, 1.0, L, ld, Tc, ld, 0.0, proj, nl, st);
                launch_dgemm(false, false, N, nb, nl, -1.0, L, ld, proj, nl, 1.0, Tc, ld, st);
            }
            launch_dgemm(true, false, m, nb, N, 1.0, S, ld, Tc, ld, 0.0, proj, m, st);
            launch_dgemm(false, false, N, nb, m, -1.0, S, ld, proj, m, 1.0, Tc, ld, st);
        }
        // orthonormalise the corrections: Tc^T Tc = Q diag(l) Q^T, keep l > 1e-10 max
        launch_dgemm(true, false, nb, nb, N, 1.0, Tc, ld, Tc, ld, 0.0, G, nb, st);
        syev_small(ctx, G, nb, wr, Yr);
        std::vector<double> lg = d2h(ctx, wr, nb);
        const double lmax = lg[nb - 1];
        int first = 0;
        while (first < nb && !(lg[first] > 1.0e-10 * lmax)) ++first;
        const int nk = nb - first;
        if (nk <= 0) break;
        std::vector<double> sc(nk);
        for (int j = 0; j < nk; ++j) sc[j] = 1.0 / std::sqrt(lg[first + j]);
        CK(cudaMemcpyAsync(dsc, sc.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, st));
        scale_cols_kernel<<<nblk((long long)nb * nk, 256), 256, 0, st>>>(Yr + (size_t)first * nb, nb, nb, dsc, nk);
        DVR3D_COUNT_LAUNCH(1);
        double *Snew = S + (size_t)m * ld;
        launch_dgemm(false, false, N, nk, nb, 1.0, Tc, ld, Yr + (size_t)first * nb, nb, 0.0, Snew, ld, st);
        H.apply(Snew, ld, nk, HS + (size_t)m * ld, ld, stats);
        m += nk;
        (void)T2;
    }
    stats.iterations = it;
    if (nl < nwant) throw HostError{DVR3D_ERR_NOCONV, "Davidson did not converge all requested levels"};
    // order the locked pairs by energy
    std::vector<int> perm(nl);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return lval[a] < lval[b]; });
    std::vector<double> ws(nwant);
    rn_host.assign(nwant, 0.0);
    stats.max_resid = 0.0;
    for (int j = 0; j < nwant; ++j) {
        ws[j] = lval[perm[j]];
        rn_host[j] = lres[perm[j]];
        stats.max_resid = std::max(stats.max_resid, rn_host[j]);
    }
    CK(cudaMemcpyAsync(wv_dev, ws.data(), sizeof(double) * nwant, cudaMemcpyHostToDevice, st));
    if (evec_dev) {
        for (int j = 0; j < nwant; ++j)
            CK(cudaMemcpyAsync(evec_dev + (size_t)j * ld, L + (size_t)perm[j] * ld, sizeof(double) * N,
                               cudaMemcpyDeviceToDevice, st));
    }
    CK(cudaStreamSynchronize(st));
    H.collect(stats);
}

}  // namespace dvr3d
