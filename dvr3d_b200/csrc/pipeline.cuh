// pipeline.cuh -- device context and the per-k-block solve pipeline.
#pragma once

#include <chrono>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/dvr3d_b200.h"
#include "common.cuh"
#include "host_setup.h"
#include "learned_precond.cuh"
#include "pes.cuh"

namespace dvr3d {

// Device buffers keyed by name, grown on demand and reused across solves.
class DeviceArena {
  public:
    ~DeviceArena();
    void *get(const std::string &name, size_t bytes);
    template <class T>
    T *get_t(const std::string &name, size_t count) {
        return static_cast<T *>(get(name, count * sizeof(T)));
    }
    size_t bytes_held() const;
    void release_all();

  private:
    struct Buf {
        void *p = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buf> bufs_;
};

struct CudaFail {
    cudaError_t err;
    std::string where;
};

}  // namespace dvr3d

struct dvr3d_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;     // stream all work of this context is issued on
    cudaStream_t own_stream = nullptr; // the stream the context created (destroyed with it)
    std::string last_error;
    dvr3d::PesParams pes{};
    std::vector<double> pes_grid;  // host copy of a tabulated PES
    std::map<int, std::vector<double>> pes_grid_k;  // tables of single k blocks (their own grids)
    // the table of k block kz: its own, else the common one
    const std::vector<double> &pes_table(int kz) const {
        const auto it = pes_grid_k.find(kz);
        return it == pes_grid_k.end() ? pes_grid : it->second;
    }
    dvr3d::DeviceArena arena;
    cudaEvent_t ev[8] = {};
    int sm_count = 0;
    int dense_grid = 0;
    std::vector<cudaEvent_t> panel_ev;  // timing pool for the reduction panels
    unsigned long long wait_limit = 0;  // polls of each bounded device wait (0: kernel defaults)
    std::vector<cudaEvent_t> gemm_ev;   // timing pool of the GEMM launches of an iterative solve
    bool lp_trained = false;            // arena "lp_w" holds a trained preconditioner network
    std::map<long long, int> tuned_split;  // autotuned split-K of the Krylov products per (N, b)
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        long long kernels = 0;          // kernel launches the graph replays
    };
    std::map<std::string, Graph> graphs;  // captured Krylov step sequences, by shape and buffers
    struct LpSet {                      // training pairs of the last training solve
        bool valid = false;
        int N = 0, nwant = 0, npair = 0;
        long long ld = 0;
        std::vector<int> snap_m;        // basis size of each snapshot (arena "lp_V<s>")
        dvr3d::ChanPrec cp;
    } lp_set;
};

namespace dvr3d {

// Output of the 1D/2D stages: the contracted basis, ready for assembly or for the
// matrix-free operator H3 = blockdiag(C_g^T) (T x I_P) blockdiag(C_g) + diag(e2).
struct Contracted {
    double *Vt = nullptr;   // ldv x ncol (zero padded), column i = sqrt(w)-scaled basis function
    long long ldv = 0;
    int P = 0, N = 0;
    int *g = nullptr;       // [N] block of each column (device)
    double *e2 = nullptr;   // [N] 2D eigenvalues (device)
    const double *T = nullptr;  // block coupling matrix (device), T[g' * ldt + g]
    int ldt = 0;
    std::vector<int> iv2;   // per block selected counts (host)
    int nblocks = 0;
    std::vector<double> sw; // [P] the row scaling sqrt(w_p) applied to Vt (1 where none; host)
};

// Wavefunction amplitudes of the returned levels on the DVR grid, in the record layout of the
// reference's wavefunction file (filled by solve_block when requested): psi holds `nlev`
// records of `len` doubles (Jacobi: psi(idvr, npnt1, npnt2) as trans writes it, :3733-3841;
// Radau: wvfunc(nbass) as transr writes it, :3596-3643).
struct WaveOut {
    long long len = 0;
    int nlev = 0;
    std::vector<double> psi;
};

// The assembled H3 as the iterative solvers see it: FP64 full symmetric storage (H3, ldh
// even), or, in the split-BF16 form (H3 null), its BF16 slices hi + lo (full symmetric
// storage, ld a multiple of 8) for the tensor-core products, the FP64 products then coming
// from the matrix-free operator of the contracted basis (apply_h3_fp64).
struct H3Op {
    const double *H3 = nullptr;
    long long ldh = 0;
    const __nv_bfloat16 *hi = nullptr, *lo = nullptr;
    long long ld = 0;
};

// Y (N x nvec, ldy) = H3 X (ldx) in FP64 without H3: per block g of the contracted basis
//   Y_g = C_g^T sum_g' T[g, g'] (C_g' X_g')  +  e2_g o X_g
// (three DMMA GEMM launches: block products, the block mix by T, the transposed block
// products; then the diagonal). 4 P N + 2 P G^2 flops per vector instead of 2 N^2.
void apply_h3_fp64(dvr3d_ctx *ctx, const Contracted &C, const double *X, long long ldx, int nvec, double *Y,
                   long long ldy);

// Channel blocks of the assembled H3 and their eigen-decompositions, with the per-mode
// features of the learned correction (learned_precond.cuh). lam_host / chan_of_mode
// (optional): the channel eigenvalues and the channel of every mode.
void channel_setup(dvr3d_ctx *ctx, const H3Op &op, const Contracted &C, ChanPrec &cp,
                   std::vector<double> *lam_host = nullptr, std::vector<int> *chan_of_mode = nullptr);

// Block-Davidson for the lowest `nwant` levels of H3 with the channel-block preconditioner.
// mode 0: exact channel inverse; 1: with the learned correction (parameters lp_w, device);
// 2: exact channel inverse, record (residual, correction) pairs and fit the network into
// lp_w. Block b = nwant + max(8, nwant/2) up to kDavidsonMaxLevels levels (b <= 48), else
// nwant + max(16, nwant/4); Rayleigh-Ritz on the shared-memory eigensolver up to 160 basis
// vectors, on the dense FP64 eigensolver beyond.
// Split-BF16 form: the products H3 V are BF16x3 tensor-core GEMMs until the largest residual
// stops falling (by less than 30 % in an iteration); then the residual correction: the
// products of the whole basis are recomputed in FP64 (apply_h3_fp64) and the iteration goes
// on with FP64 products until the FP64 residual test holds. Writes the levels (device wv_dev),
// FP64 residual norms and optionally the vectors (N x nwant, ld N). Returns false when it
// does not converge within its limits (the caller falls back).
constexpr int kDavidsonMaxLevels = 32;
constexpr int kDavidsonMaxBlock = 48;
struct DavidsonStats {
    int iterations = 0;
    int matvecs = 0;
    int low_iterations = 0;    // split-BF16 form: iterations with tensor-core products
    int low_matvecs = 0;       //                  vectors multiplied on the tensor cores
    double max_resid = 0.0;
    int pairs = 0;             // training pairs recorded (mode 2)
    bool trained = false;
    double loss_first = 0.0, loss_last = 0.0;
};
bool davidson_solve(dvr3d_ctx *ctx, const H3Op &op, const Contracted &C, const dvr3d_options &opt, int nwant,
                    int mode, double *lp_w, double *wv_dev, std::vector<double> &rn_host, double *evec_dev,
                    DavidsonStats &stats);

// Training loss of the learned correction (and, when grad is not null, its gradient, device)
// at parameters w (device) on the pairs recorded by the context's last training solve.
double lp_train_loss(dvr3d_ctx *ctx, const double *w, double *grad);

// Host<->device byte counters of the current solve (reported in dvr3d_result).
void note_h2d(long long bytes);
void note_d2h(long long bytes);

// Lowest nev eigenvalues (ascending, device w) and optionally eigenvectors (device Z, ldz)
// of the symmetric n x n matrix A (lower triangle read, lda a multiple of 8; overwritten by
// the reduction). Device scratch is taken from the arena under names starting with `tag`.
// When time_panels is set, the reduction's panel launches are timed into *out.
struct DenseOut {
    double panel_ms = 0.0;
    int npanel = 0;
};
void dense_lowest(dvr3d_ctx *ctx, double *A, long long lda, int n, int nev, bool vecs, double *w, double *Z,
                  long long ldz, const char *tag, bool time_panels, DenseOut *out);
// Lowest nev eigenpairs of a symmetric matrix (lower triangle of A, lda) treated as a band
// of half-bandwidth b (<= 32): bulge chasing, tridiagonal eigensolve, back-transform into Z.
// Returns false (nothing computed) when the entries beyond the band exceed drop_rel times
// the largest entry inside it; *dropped_rel receives that ratio.
bool band_lowest(dvr3d_ctx *ctx, double *A, long long lda, int n, int b, int nev, double *w, double *Z,
                 long long ldz, double drop_rel, double *dropped_rel);

// The same eigenpairs by Sturm-count bisection and inverse iteration on LDL^T factors of the
// band (no reduction); false when the band check fails or inverse iteration does not grow.
bool band_lowest_bisect(dvr3d_ctx *ctx, double *A, long long lda, int n, int b, int nev, double *w, double *Z,
                        long long ldz, double drop_rel, double *dropped_rel);

// Shift-invert block Krylov solve for the lowest `nwant` levels of the assembled H3
// (full symmetric storage, ldh even). emin_bound: a lower bound of the spectrum (min e2).
// Returns false when it gives up (Krylov space limit, breakdown, no SPD shift found); the
// caller then uses the dense eigensolver.
struct KrylovStats {
    double sigma = 0.0;
    int retries = 0;       // shifts that failed the Cholesky pivot test
    int block = 0;
    int blocks = 0;        // Krylov blocks built
    int m = 0;             // final subspace size
    int checks = 0;        // Rayleigh-Ritz checks
    int nconv = 0;
    double worst_bound = 0.0;
    double factor_ms = 0.0, krylov_ms = 0.0, rr_ms = 0.0;
    double flops = 0.0;    // algorithmic flops of the factorisation, Krylov steps and checks
    double max_resid = 0.0;
    // the GEMM launches of the solve, each timed with CUDA events (gemm64.cuh GemmLaunchLog)
    double gemm_ms = 0.0, gemm_flops = 0.0;
    int gemm_launches = 0, gemm_untimed = 0;
    int trmm_split = 0;    // split-K of the Krylov triangular products (autotuned)
};
int si_krylov_first_size(int nwant, int block);
bool si_krylov_solve(dvr3d_ctx *ctx, const double *H3, long long ldh, int N, double emin_bound,
                     const dvr3d_options &opt, int nwant, double *wv_dev, std::vector<double> &rn_host,
                     double *evec_dev, KrylovStats &ks);

// Solve one k block. Throws HostError / CudaFail. With `wave`, the eigenvectors of the
// returned levels are also back-transformed to the DVR grid (wavefn.cu).
void solve_block(dvr3d_ctx *ctx, const dvr3d_deck &deck, int kk, const dvr3d_options &opt,
                 dvr3d_result &res, WaveOut *wave = nullptr);

// The 2D stages of several independent Radau k blocks (each with its own surface) as one
// batched device workload; outs[i] is problem i's contracted basis.
void radau_stage_batch(dvr3d_ctx *ctx, const std::vector<BlockPlan> &plans, const std::vector<PesParams> &pes,
                       std::vector<Contracted> &outs);

// The error flag of the batched eigenvector kernels (cleared by the caller before a stage) and
// its check (throws DVR3D_ERR_NOCONV when raised).
int *eigvec_err_flag(dvr3d_ctx *ctx);
void check_eigvec_err(dvr3d_ctx *ctx, const char *stage);

// The part of solve_block after the 1D/2D stages (assembly, final eigensolve, outputs), for a
// block whose contracted basis C is already on the device (ev[0] / ev[1] bracket its stage).
void solve_contracted(dvr3d_ctx *ctx, const BlockPlan &p, const Contracted &C, const dvr3d_options &opt,
                      dvr3d_result &res, WaveOut *wave, std::chrono::steady_clock::time_point th0,
                      std::chrono::steady_clock::time_point th1, long long launches0);

// psi = the contracted basis (Vt with its sqrt(w) row scaling removed) times the eigenvector
// coefficients Z (N x nlev, ldz), per block one DMMA GEMM, scattered into the record layout
// of the wavefunction file. Downloads the records into wave.
void compute_wavefunctions(dvr3d_ctx *ctx, const BlockPlan &p, const Contracted &C, const double *Z,
                           long long ldz, int nlev, WaveOut &wave);

}  // namespace dvr3d
