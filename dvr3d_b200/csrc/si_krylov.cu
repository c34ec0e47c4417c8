// si_krylov.cu -- lowest levels of the contracted Hamiltonian by a shift-invert block Krylov
// (block Lanczos) solve with full reorthogonalisation, judged by FP64 residuals.
//
// The reference diagonalises the final Hamiltonian completely (diag3d -> dsyev, :2661-2764)
// and keeps the lowest NEVAL levels. Here:
//   (1) sigma below the spectrum: H3 = C^T (T (x) W) C + diag(e2) with T (the angular
//       kinetic L matrix, lmatrx :1846-1911) positive semi-definite and W > 0, so
//       lambda_min(H3) >= min(e2); sigma = min(e2) - margin makes H3 - sigma SPD
//       (a failed pivot lowers sigma and retries);
//   (2) H3 - sigma = L L^T and B = L^{-1} (chol.cu: recursive, DMMA GEMMs, 2/3 N^3 flop);
//   (3) block Krylov space of M = (H3 - sigma)^{-1} = B^T B: each step W = B^T (B Q_k) (two
//       triangular GEMMs), classical Gram-Schmidt against all previous blocks twice, and
//       Cholesky-QR twice inside the block; the projections give T = Q^T M Q column block
//       by column block;
//   (4) at check points: eigenpairs of T (the dense device eigensolver on -T gives the
//       largest mu first), Ritz vectors X = Q Y, FP64 H3 X, Rayleigh quotients and residual
//       norms; a level is accepted when rho^2 / gap <= tol (the quadratic residual bound),
//       otherwise the Krylov space grows and the check repeats; past the size limit the
//       caller falls back to the dense FP64 eigensolve.
// All heavy work is DMMA GEMM (gemm_pipe.cu); the levels returned are the FP64 Rayleigh
// quotients of the accepted Ritz vectors.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "band_eig.cuh"
#include "chol.cuh"
#include "ozaki.cuh"
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

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Q[:, 0:b] <- uniform(-1, 1) from a counter hash (deterministic)
__global__ void rand_block_kernel(double *Q, long long ld, int n, int b, unsigned long long seed) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * b) return;
    const int j = (int)(t / n), i = (int)(t % n);
    const unsigned long long h = mix64(seed ^ mix64((unsigned long long)t));
    Q[(size_t)j * ld + i] = (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// T[0:m, 0:b] += P (ld m)
__global__ void add_block_kernel(double *T, long long ldt, const double *P, int m, int b) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)m * b) return;
    const int j = (int)(t / m), i = (int)(t % m);
    T[(size_t)j * ldt + i] += P[(size_t)j * m + i];
}

// A = -(T symmetrised from its upper triangle), m x m
__global__ void upper_sym_neg_kernel(const double *T, long long ldt, int m, double *A, long long lda) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)m * m) return;
    const int j = (int)(t / m), i = (int)(t % m);
    const int r = i < j ? i : j, c = i < j ? j : i;
    A[(size_t)j * lda + i] = -T[(size_t)c * ldt + r];
}

// theta_j = x^T H x / x^T x, rho_j = ||H x - theta x|| / ||x||; one CTA per column
__global__ void rq_resid_kernel(const double *X, const double *HX, long long ld, int n, double *theta, double *rho) {
    const int j = blockIdx.x;
    const double *x = X + (size_t)j * ld, *hx = HX + (size_t)j * ld;
    __shared__ double red[32];
    double xx = 0.0, xh = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        xx += x[i] * x[i];
        xh += x[i] * hx[i];
    }
    xx = block_sum(xx, red);
    xh = block_sum(xh, red);
    const double th = xh / xx;
    double rr = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double r = hx[i] - th * x[i];
        rr += r * r;
    }
    rr = block_sum(rr, red);
    if (threadIdx.x == 0) {
        theta[j] = th;
        rho[j] = sqrt(rr / xx);
    }
}

// Z[:, q] = X[:, perm[q]] / ||X[:, perm[q]]||
__global__ void gather_norm_kernel(const double *X, long long ldx, const int *perm, int n, double *Z, long long ldz) {
    const int q = blockIdx.x;
    const double *x = X + (size_t)perm[q] * ldx;
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i] * x[i];
    s = block_sum(s, red);
    const double inv = 1.0 / sqrt(s);
    for (int i = threadIdx.x; i < n; i += blockDim.x) Z[(size_t)q * ldz + i] = x[i] * inv;
}

inline unsigned nb256(long long n) { return (unsigned)((n + 255) / 256); }
inline long long rup(long long x, long long m) { return (x + m - 1) / m * m; }

// split-K factor for about `target` CTAs; at most 8 (one thread-block cluster, no second
// reduction kernel) once that already gives two waves of CTAs
int splits(int tiles, int ktiles, int target, int smax) {
    int s = (target + tiles - 1) / std::max(tiles, 1);
    s = std::max(1, std::min({s, smax, ktiles}));
    if (s > 8 && tiles * 8 >= 296) s = 8;
    return s;
}

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer() {
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    void start(cudaStream_t s) { CK(cudaEventRecord(a, s)); }
    void stop(cudaStream_t s) { CK(cudaEventRecord(b, s)); }
    double ms() {
        CK(cudaEventSynchronize(b));
        float m = 0.f;
        CK(cudaEventElapsedTime(&m, a, b));
        return m;
    }
};

// Autotuned split-K of the Krylov triangular products (L^-1 Q and its transpose have the same
// shape): on the first solve of an (N, b) shape in a context, each candidate split is timed by
// CUDA events (one untimed launch, then two timed) on the start block and the fastest is kept
// for every later block step and solve; candidates are the fixed rule's choice and 4..8 slices
// (reduced by the thread-block cluster through distributed shared memory). DVR3D_NO_AUTOTUNE=1
// keeps the rule.
int tuned_trmm_split(dvr3d_ctx *ctx, GemmOp y, int rule, cudaStream_t st) {
    const long long key = ((long long)y.M << 16) | (long long)y.N;
    auto it = ctx->tuned_split.find(key);
    if (it != ctx->tuned_split.end()) return it->second;
    const char *env = std::getenv("DVR3D_NO_AUTOTUNE");
    if (env && env[0] == '1') return rule;
    const int ktiles = (y.K + 15) / 16;
    Timer t;
    int best = rule;
    double best_ms = 1.0e30;
    std::vector<int> cand{rule};
    for (int c = 4; c <= 8; ++c)
        if (c != rule && c <= ktiles) cand.push_back(c);
    for (int c : cand) {
        y.splitk = c;
        CK(launch_gemm(y, st));
        t.start(st);
        CK(launch_gemm(y, st));
        CK(launch_gemm(y, st));
        t.stop(st);
        const double ms = t.ms();
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    ctx->tuned_split[key] = best;
    return best;
}

}  // namespace

int si_krylov_first_size(int nwant, int block) {
    // about 5 Krylov vectors per wanted level, and at least 20 block steps (the polynomial
    // degree, not only the dimension, sets the convergence of the last wanted levels);
    // DVR3D_SI_FIRST overrides the vectors per level (tuning)
    double per = 5.2;
    if (const char *e = std::getenv("DVR3D_SI_FIRST")) {
        const double v = std::atof(e);
        if (v >= 1.5 && v <= 10.0) per = v;
    }
    const int b = block;
    return (int)std::max(rup((long long)std::ceil(per * nwant) + b, b), 20LL * b);
}

bool si_krylov_solve(dvr3d_ctx *ctx, const double *H3, long long ldh, int N, double emin_bound,
                     const dvr3d_options &opt, int nwant, double *wv_dev, std::vector<double> &rn_host,
                     double *evec_dev, KrylovStats &ks) {
    cudaStream_t st = ctx->stream;
    const int bdef = nwant <= 48 ? 8 : (nwant <= 160 ? 16 : 32);
    const int b = std::max(8, std::min(opt.block > 0 ? opt.block : bdef, 64)) & ~1;  // even: 16-byte rows
    if (ldh & 1) return false;
    const int guard = std::min(32, std::max(8, nwant / 10));
    const int kw = nwant + guard;
    const int mfirst = si_krylov_first_size(nwant, b);
    const int mmax = (int)std::min<long long>(std::max(rup((long long)std::ceil(7.0 * nwant) + 2 * b, b), 40LL * b),
                                              (N / b - 1) * (long long)b);
    if (mfirst > mmax || kw > mfirst) return false;
    const double tolE = (opt.tol_cm > 0.0 ? opt.tol_cm : 1.0e-4) / 2.19474624e5;
    const long long ldw = rup(N, 8), ldq = ldw, ldT = rup(mmax, 8);
    // ---- buffers
    double *Lb = ctx->arena.get_t<double>("si_L", (size_t)ldw * N);
    const size_t wk = std::max({chol_work_doubles(N), (size_t)16 * N * b, (size_t)64 * mmax * b, (size_t)64 * 64 * 64});
    double *work = ctx->arena.get_t<double>("si_work", wk);
    int *err = ctx->arena.get_t<int>("si_err", 2);
    double *Q = ctx->arena.get_t<double>("si_Q", (size_t)ldq * (mmax + b));
    double *T = ctx->arena.get_t<double>("si_T", (size_t)ldT * mmax);
    double *Y1 = ctx->arena.get_t<double>("si_Y1", (size_t)ldq * b);
    double *G = ctx->arena.get_t<double>("si_G", 64 * 64);
    double *Gi = ctx->arena.get_t<double>("si_Gi", 64 * 64);
    double *proj = ctx->arena.get_t<double>("si_P", (size_t)mmax * b);
    Timer tf, tk, tr;
    const char *trace_env = std::getenv("DVR3D_SI_TRACE");
    const bool trace = trace_env && trace_env[0] == '1';
    ks = KrylovStats{};
    ks.block = b;
    // with DVR3D_GEMM_EVENTS=1, every GEMM launch of this solve is timed by an event pair
    // (4096 launches at most); off by default: the event records and the read-out after the
    // solve cost host time that delays the next solve
    const char *gev = std::getenv("DVR3D_GEMM_EVENTS");
    const bool log_gemms = gev && gev[0] == '1';
    if (log_gemms && ctx->gemm_ev.empty()) {
        ctx->gemm_ev.resize(8192);
        for (auto &e : ctx->gemm_ev) CK(cudaEventCreate(&e));
    }
    GemmLaunchLog glog;
    glog.ev = ctx->gemm_ev.data();
    glog.nev = (int)ctx->gemm_ev.size();
    struct LogScope {
        explicit LogScope(GemmLaunchLog *l) { set_gemm_launch_log(l); }
        ~LogScope() { set_gemm_launch_log(nullptr); }
    } log_scope(log_gemms ? &glog : nullptr);
    // ---- (1)+(2) shift, factor, invert
    tf.start(st);
    double sigma = emin_bound - std::max(1.0e-6, 1.0e-3 * std::fabs(emin_bound));
    // the large products of the factorisation on the int8 tensor cores (Ozaki slices, FP64
    // accuracy); DVR3D_OZAKI=0 keeps every product on the DMMA path, DVR3D_OZAKI_SLICES sets
    // the slice count (4..8)
    CholOzaki oz;
    {
        const char *oe = std::getenv("DVR3D_OZAKI");
        const char *se = std::getenv("DVR3D_OZAKI_SLICES");
        if (se) oz.nslice = std::max(kOzMinSlices, std::min(kOzMaxSlices, std::atoi(se)));
        const size_t ob = (oe && oe[0] == '0') ? 0 : chol_ozaki_work_bytes(N, oz.nslice);
        if (ob > 0) {
            oz.work = ctx->arena.get_t<unsigned char>("si_oz", ob + 1024);
            oz.bytes = ob + 1024;
            const uintptr_t mis = reinterpret_cast<uintptr_t>(oz.work) & 1023u;
            if (mis) {  // 1 KB alignment for the slice buffers
                oz.work = static_cast<unsigned char *>(oz.work) + (1024 - mis);
                oz.bytes -= 1024 - mis;
            }
        }
    }
    bool spd = false;
    for (int attempt = 0; attempt < 4 && !spd; ++attempt) {
        CK(launch_shift_copy_lower(H3, ldh, N, sigma, Lb, ldw, st));
        CK(cudaMemsetAsync(err, 0, 2 * sizeof(int), st));
        CK(launch_potrf_inv_lower(Lb, ldw, N, work, err, st, &oz));
        int e = 0;
        CK(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        note_d2h(sizeof(int));
        if (e == kDevBarrierTimeout) return false;  // a tensor-core pipeline wait ran out
        if (e == 0) spd = true;
        else {
            ++ks.retries;
            sigma -= std::max(1.0e-2, 2.0 * std::fabs(sigma));
        }
    }
    if (!spd) return false;
    ks.sigma = sigma;
    // optionally (DVR3D_OZAKI_KRYLOV=1) the Krylov products inv(L) Q_k and inv(L)^T Y on the
    // int8 tensor cores: inv(L) sliced once in both orientations (rows of inv(L) for the
    // first, its columns for the second), each product slicing only its 32-column block and
    // splitting K into chunks. Off by default: with 32-column tiles every int8 MMA re-reads its
    // 128-row slice tile from shared memory for only 32 output columns, and the Krylov steps
    // took 62.7 ms against 54.4 ms on the DMMA path at N = 12202.
    OzPresliced ozl1, ozl2;
    bool oz_krylov = false;
    int oz_kslices = kOzDefaultSlices;
    unsigned char *ozk_work = nullptr;
    size_t ozk_bytes = 0;
    {
        const char *ke = std::getenv("DVR3D_OZAKI_KRYLOV");
        const char *se = std::getenv("DVR3D_OZAKI_KRYLOV_SLICES");
        if (se) oz_kslices = std::max(kOzMinSlices, std::min(kOzMaxSlices, std::atoi(se)));
        GemmOp y;
        y.M = N;
        y.N = b;
        y.K = N;
        y.A = Lb;
        y.lda = ldw;
        y.tri = 1;
        y.B = Q;
        y.ldb = ldq;
        y.C = Y1;
        y.ldc = ldq;
        GemmOp w = y;
        w.ta = true;
        w.tri = 2;
        w.B = Y1;
        w.C = Q;
        if (oz.work && ke && ke[0] == '1' && ozaki_supported(y, oz_kslices) && N >= 2048) {
            auto aligned = [&](const char *name, size_t bytes) {
                auto *p = ctx->arena.get_t<unsigned char>(name, bytes + 1024);
                const uintptr_t mis = reinterpret_cast<uintptr_t>(p) & 1023u;
                return mis ? p + (1024 - mis) : p;
            };
            const size_t pb = ozaki_preslice_bytes(y, oz_kslices);
            CK(ozaki_preslice_a(y, oz_kslices, aligned("si_ozL1", pb), pb, ozl1, st));
            CK(ozaki_preslice_a(w, oz_kslices, aligned("si_ozL2", pb), pb, ozl2, st));
            ozk_bytes = std::max(ozaki_work_bytes(y, oz_kslices, true, kOzKrylovChunk),
                                 ozaki_work_bytes(w, oz_kslices, true, kOzKrylovChunk));
            ozk_work = aligned("si_ozK", ozk_bytes);
            CK(ozaki_set_attributes(y, oz_kslices));  // before any graph capture of these launches
            oz_krylov = true;
        }
    }
    tf.stop(st);
    // ---- (3) block Krylov
    auto cholqr = [&](double *Wp) {
        for (int pass = 0; pass < 2; ++pass) {
            GemmOp g;
            g.M = b;
            g.N = b;
            g.K = N;
            g.A = Wp;
            g.lda = ldq;
            g.ta = true;
            g.B = Wp;
            g.ldb = ldq;
            g.C = G;
            g.ldc = b;
            g.splitk = splits(1, (N + 15) / 16, 256, 128);
            g.work = work;
            CK(launch_gemm(g, st));
            CK(launch_chol_small(G, b, Gi, 1.0e-24, err + 1, st));
            GemmOp s;
            s.M = N;
            s.N = b;
            s.K = b;
            s.A = Wp;
            s.lda = ldq;
            s.B = Gi;
            s.ldb = 64;
            s.tb = true;
            s.C = Wp;
            s.ldc = ldq;
            CK(launch_gemm(s, st));
        }
    };
    DVR3D_COUNT_LAUNCH(1);
    rand_block_kernel<<<nb256((long long)N * b), 256, 0, st>>>(Q, ldq, N, b, 0x5eed1234abcdull);
    CK(cudaGetLastError());
    cholqr(Q);
    const int tiles_n = (N + 63) / 64;
    int trmm_s = splits(tiles_n, (N + 15) / 16, 1200, 16);
    {
        GemmOp y;
        y.M = N;
        y.N = b;
        y.K = N;
        y.A = Lb;
        y.lda = ldw;
        y.tri = 1;
        y.B = Q;
        y.ldb = ldq;
        y.C = Y1;
        y.ldc = ldq;
        y.work = work;
        if (!oz_krylov) trmm_s = tuned_trmm_split(ctx, y, trmm_s, st);
    }
    ks.trmm_split = trmm_s;
    double flops = 0.0;
    int s = 0;  // blocks with their T column computed
    int next = mfirst / b;
    double tk_ms = 0.0, tr_ms = 0.0;
    bool done = false, breakdown = false;
    std::vector<double> theta, rho;
    std::vector<int> perm;
    // The block steps between two checks have no host synchronisation: outside GEMM timing they
    // run as one CUDA graph, captured on the first solve of a shape (and buffers) in this
    // context and replayed by later solves (DVR3D_NO_GRAPH=1 launches them one by one).
    const char *ng = std::getenv("DVR3D_NO_GRAPH");
    const bool use_graph = !log_gemms && !(ng && ng[0] == '1');
    while (!done) {
        tk.start(st);
        std::string gkey;
        bool replayed = false, capturing = false;
        const long long kernels0 = g_kernel_launches;
        if (use_graph && next > s) {
            char kb[256];
            std::snprintf(kb, sizeof(kb), "si:%d:%d:%d:%d:%d:%lld:%lld:%p:%p:%p:%p:%p:%p:%d:%p:%p:%p", N, b, s, next,
                          trmm_s, ldq, ldT, (void *)Lb, (void *)Q, (void *)T, (void *)Y1, (void *)work, (void *)proj,
                          oz_krylov ? oz_kslices : 0, (void *)ozk_work, (const void *)ozl1.S, (const void *)ozl2.S);
            gkey = kb;
            auto it = ctx->graphs.find(gkey);
            if (it != ctx->graphs.end()) {
                CK(cudaGraphLaunch(it->second.exec, st));
                DVR3D_COUNT_LAUNCH(it->second.kernels);
                replayed = true;
            } else {
                CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                capturing = true;
            }
        }
        // a failure while capturing ends the capture before the error propagates
        struct CaptureGuard {
            cudaStream_t st;
            bool &on;
            ~CaptureGuard() {
                if (on) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(st, &g);
                    if (g) cudaGraphDestroy(g);
                    cudaGetLastError();
                }
            }
        } guard{st, capturing};
        const int s_first = s;
        if (replayed) {
            for (; s < next; ++s) {
                const int m = (s + 1) * b;
                flops += 2.0 * (double)N * N * b + 8.0 * (double)N * m * b + 8.0 * (double)N * b * b;
            }
        }
        for (; s < next; ++s) {
            const double *Qk = Q + (size_t)s * b * ldq;
            const int m = (s + 1) * b;
            GemmOp y;
            y.M = N;
            y.N = b;
            y.K = N;
            y.A = Lb;
            y.lda = ldw;
            y.tri = 1;
            y.B = Qk;
            y.ldb = ldq;
            y.C = Y1;
            y.ldc = ldq;
            y.splitk = trmm_s;
            y.work = work;
            if (oz_krylov) CK(launch_ozaki_gemm(y, oz_kslices, ozk_work, ozk_bytes, err, st, &ozl1, kOzKrylovChunk));
            else CK(launch_gemm(y, st));
            // the new block is formed in place in its slot of Q (not read by the projections)
            double *W = Q + (size_t)(s + 1) * b * ldq;
            GemmOp w = y;
            w.ta = true;
            w.tri = 2;
            w.B = Y1;
            w.C = W;
            if (oz_krylov) CK(launch_ozaki_gemm(w, oz_kslices, ozk_work, ozk_bytes, err, st, &ozl2, kOzKrylovChunk));
            else CK(launch_gemm(w, st));
            double *Tk = T + (size_t)s * b * ldT;
            const int tm = (m + 63) / 64;
            for (int pass = 0; pass < 2; ++pass) {
                GemmOp c;
                c.M = m;
                c.N = b;
                c.K = N;
                c.A = Q;
                c.lda = ldq;
                c.ta = true;
                c.B = W;
                c.ldb = ldq;
                c.C = pass == 0 ? Tk : proj;
                c.ldc = pass == 0 ? ldT : m;
                c.splitk = splits(tm, (N + 15) / 16, 1200, 64);
                c.work = work;
                CK(launch_gemm(c, st));
                GemmOp u;
                u.M = N;
                u.N = b;
                u.K = m;
                u.alpha = -1.0;
                u.beta = 1.0;
                u.A = Q;
                u.lda = ldq;
                u.B = c.C;
                u.ldb = c.ldc;
                u.C = W;
                u.ldc = ldq;
                u.splitk = splits(tiles_n, (m + 15) / 16, 1200, 8);
                u.work = work;
                CK(launch_gemm(u, st));
                if (pass == 1) {
                    DVR3D_COUNT_LAUNCH(1);
                    add_block_kernel<<<nb256((long long)m * b), 256, 0, st>>>(Tk, ldT, proj, m, b);
                    CK(cudaGetLastError());
                }
            }
            cholqr(W);
            flops += 2.0 * (double)N * N * b + 8.0 * (double)N * m * b + 8.0 * (double)N * b * b;
        }
        if (capturing) {
            cudaGraph_t graph = nullptr;
            capturing = false;
            CK(cudaStreamEndCapture(st, &graph));
            cudaGraphExec_t exec = nullptr;
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            CK(ie);
            dvr3d_ctx::Graph g;
            g.exec = exec;
            g.kernels = g_kernel_launches - kernels0;
            ctx->graphs[gkey] = g;
            CK(cudaGraphLaunch(exec, st));
        }
        (void)s_first;
        tk.stop(st);
        tk_ms += tk.ms();
        int qe[2] = {0, 0};
        CK(cudaMemcpyAsync(qe, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        note_d2h(2 * sizeof(int));
        if (qe[0] == kDevBarrierTimeout) return false;  // an int8 tensor-core pipeline wait ran out
        breakdown = (qe[1] != 0);
        // ---- (4) Rayleigh-Ritz on T, FP64 judge
        tr.start(st);
        const int m = s * b;
        const long long lda = rup(m, 8);
        double *A = ctx->arena.get_t<double>("si_A", (size_t)lda * m);
        DVR3D_COUNT_LAUNCH(1);
        upper_sym_neg_kernel<<<nb256((long long)m * m), 256, 0, st>>>(T, ldT, m, A, lda);
        CK(cudaGetLastError());
        double *lam = ctx->arena.get_t<double>("si_lam", kw);
        double *Yv = ctx->arena.get_t<double>("si_Yv", (size_t)m * kw);
        Timer td;
        td.start(st);
        // T is block tridiagonal up to the rounding-level reorthogonalisation coefficients:
        // chase its band unless those are not small (then the dense reduction)
        double dropped = 0.0;
        const char *be = std::getenv("DVR3D_BAND_EIG");
        const bool bisect = be && std::strcmp(be, "bisect") == 0;
        bool banded = false;
        if (b <= kBandMaxBw && bisect) banded = band_lowest_bisect(ctx, A, lda, m, b, kw, lam, Yv, m, 1.0e-11, &dropped);
        if (!banded && bisect && b <= kBandMaxBw) {  // the factors overwrote nothing; redo the copy for the chase
            DVR3D_COUNT_LAUNCH(1);
            upper_sym_neg_kernel<<<nb256((long long)m * m), 256, 0, st>>>(T, ldT, m, A, lda);
            CK(cudaGetLastError());
        }
        if (!banded) banded = b <= kBandMaxBw && band_lowest(ctx, A, lda, m, b, kw, lam, Yv, m, 1.0e-11, &dropped);
        if (!banded) {
            DVR3D_COUNT_LAUNCH(1);
            upper_sym_neg_kernel<<<nb256((long long)m * m), 256, 0, st>>>(T, ldT, m, A, lda);
            CK(cudaGetLastError());
            dense_lowest(ctx, A, lda, m, kw, true, lam, Yv, m, "si_", false, nullptr);
        }
        td.stop(st);
        double *X = ctx->arena.get_t<double>("si_X", (size_t)ldq * kw);
        double *HX = ctx->arena.get_t<double>("si_HX", (size_t)ldq * kw);
        GemmOp x;
        x.M = N;
        x.N = kw;
        x.K = m;
        x.A = Q;
        x.lda = ldq;
        x.B = Yv;
        x.ldb = m;
        x.C = X;
        x.ldc = ldq;
        CK(launch_gemm(x, st));
        GemmOp h;
        h.M = N;
        h.N = kw;
        h.K = N;
        h.A = H3;
        h.lda = ldh;
        h.B = X;
        h.ldb = ldq;
        h.C = HX;
        h.ldc = ldq;
        CK(launch_gemm(h, st));
        double *dth = ctx->arena.get_t<double>("si_th", kw);
        double *drh = ctx->arena.get_t<double>("si_rh", kw);
        DVR3D_COUNT_LAUNCH(1);
        rq_resid_kernel<<<kw, 256, 0, st>>>(X, HX, ldq, N, dth, drh);
        CK(cudaGetLastError());
        theta.assign(kw, 0.0);
        rho.assign(kw, 0.0);
        CK(cudaMemcpyAsync(theta.data(), dth, sizeof(double) * kw, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(rho.data(), drh, sizeof(double) * kw, cudaMemcpyDeviceToHost, st));
        tr.stop(st);
        tr_ms += tr.ms();
        note_d2h(2 * sizeof(double) * kw);
        ++ks.checks;
        perm.resize(kw);
        std::iota(perm.begin(), perm.end(), 0);
        std::sort(perm.begin(), perm.end(), [&](int a, int c) { return theta[a] < theta[c]; });
        int nconv = 0;
        double worst = 0.0;
        for (int q = 0; q < nwant; ++q) {
            const double t = theta[perm[q]], r = rho[perm[q]];
            double gap = theta[perm[q + 1]] - t;
            if (q > 0) gap = std::min(gap, t - theta[perm[q - 1]]);
            const double bound = r * r / std::max(gap, r);
            worst = std::max(worst, bound);
            if (bound <= tolE && std::isfinite(bound)) ++nconv;
        }
        ks.nconv = nconv;
        ks.worst_bound = worst;
        ks.m = m;
        if (trace)
            std::fprintf(stderr, "si_krylov: N=%d b=%d sigma=%.6e retries=%d m=%d converged %d/%d worst bound %.3e Eh "
                                 "(krylov %.2f ms, rr %.2f ms so far)\n",
                         N, b, sigma, ks.retries, m, nconv, nwant, worst, tk_ms, tr_ms);
        if (trace)
            std::fprintf(stderr, "si_krylov: %s eigensolve of T (m=%d, %d vectors, entries beyond the band %.2e of max) %.2f ms\n",
                         banded ? "band" : "dense", m, kw, dropped, td.ms());
        if (nconv == nwant) {
            done = true;
            break;
        }
        if (breakdown) break;
        // grow by about ten vectors per level still outside the tolerance (the levels near
        // the top of the wanted window converge last, at a roughly steady rate per block)
        const int inc = std::max(2, (int)((10LL * (nwant - nconv) + b - 1) / b));
        if (s * b >= mmax) break;
        next = std::min(s + inc, mmax / b);
    }
    ks.factor_ms = tf.ms();
    if (trace)
        std::fprintf(stderr, "si_krylov: factorisation %.2f ms, %d products on the int8 tensor cores (%d slices); "
                             "Krylov products %s\n",
                     ks.factor_ms, oz.launches, oz.nslice, oz_krylov ? "on the int8 tensor cores" : "DMMA");
    ks.krylov_ms = tk_ms;
    ks.rr_ms = tr_ms;
    ks.gemm_ms = log_gemms ? gemm_launch_log_ms(glog) : 0.0;
    ks.gemm_flops = glog.flops;
    ks.gemm_launches = glog.launches;
    ks.gemm_untimed = glog.untimed;
    ks.blocks = s;
    ks.flops = flops + 2.0 / 3.0 * (double)N * N * N;
    if (!done) return false;
    std::vector<double> ws(nwant);
    rn_host.assign(nwant, 0.0);
    ks.max_resid = 0.0;
    for (int q = 0; q < nwant; ++q) {
        ws[q] = theta[perm[q]];
        rn_host[q] = rho[perm[q]];
        ks.max_resid = std::max(ks.max_resid, rn_host[q]);
    }
    CK(cudaMemcpyAsync(wv_dev, ws.data(), sizeof(double) * nwant, cudaMemcpyHostToDevice, st));
    note_h2d(sizeof(double) * nwant);
    if (evec_dev) {
        int *dp = ctx->arena.get_t<int>("si_perm", nwant);
        CK(cudaMemcpyAsync(dp, perm.data(), sizeof(int) * nwant, cudaMemcpyHostToDevice, st));
        note_h2d(sizeof(int) * nwant);
        const double *X = ctx->arena.get_t<double>("si_X", (size_t)ldq * kw);
        DVR3D_COUNT_LAUNCH(1);
        gather_norm_kernel<<<nwant, 256, 0, st>>>(X, ldq, dp, N, evec_dev, N);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(st));
    return true;
}

}  // namespace dvr3d
