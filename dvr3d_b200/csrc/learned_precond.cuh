// learned_precond.cuh -- the Davidson preconditioner of the contracted Hamiltonian: exact
// channel blocks, with a small learned spectral correction, and the kernels that train it.
//
// Channels. In block (angle) g the contracted functions are the 2D states of that angle in
// ascending energy; channel c collects the c-th state of every block (one function per block
// that has more than c states). Coupling between the same state at different angles (through
// the angular kinetic matrix) dominates the off-diagonal part of H3, so the channel blocks
// H_c = H3[ix_c, ix_c] (at most one row per angle) carry most of what a diagonal
// preconditioner misses. With H_c = Q_c diag(lambda_c) Q_c^T, the correction of a residual r
// for the Ritz value theta is
//     t[ix_c] = Q_c diag( g_cq / (lambda_cq - theta) ) Q_c^T r[ix_c],
// where g = 1 (exact channel inverse) or g = 1 + f(phi) with f a per-mode MLP
// (4 -> 16 -> 16 -> 1, tanh) of
//     phi = ((lambda_cq - theta)/s, (lambda_cq - mean_c e2)/s, c/nch, q/(n_c - 1)),
// s a per-problem energy scale. The last layer starts at zero (g = 1).
//
// Training data are pairs (r_j, theta_j, e_j) recorded by the Davidson solver, e_j the part of
// (x_final - x_j) outside the search space V_j of that moment. The loss is the mean over pairs
// of 1 - (t.e)^2 / (|P t|^2 |e|^2), P = I - V V^T (only the new direction of a correction
// matters). Its gradient runs back through the channel transforms to per-mode deltas
// dL/dg = (Q^T dL/dt) o (Q^T r)/(lambda - theta), then through the MLP.
#pragma once

#include <cuda_runtime.h>

namespace dvr3d {

constexpr int kLpFeat = 4;
constexpr int kLpHidden = 16;
// W1[16][4], b1[16], W2[16][16], b2[16], w3[16], b3
constexpr int kLpParams = kLpHidden * kLpFeat + kLpHidden + kLpHidden * kLpHidden + kLpHidden + kLpHidden + 1;

// Per-mode inputs of the features (device arrays of length n = number of modes = N).
struct LpModes {
    const double *lam = nullptr;  // channel eigenvalues
    const double *f1 = nullptr;   // (lambda - mean e2 of the channel) / s
    const double *f2 = nullptr;   // channel position
    const double *f3 = nullptr;   // position inside the channel
    int n = 0;
    double scale = 0.1;           // s (Eh)
};

struct ChanPrec {
    int nch = 0, nmax = 0;
    const int *n = nullptr;          // [nch] channel sizes
    const int *off = nullptr;        // [nch] first mode / member of each channel
    const long long *qoff = nullptr; // [nch] offset of Q_c (n_c x n_c, ld n_c)
    const int *idx = nullptr;        // [N] basis function of each member, channel by channel
    const double *Q = nullptr;
    LpModes modes;
};

// T[:, j] = correction of R[:, j] for theta[j] (ncol columns). w: network parameters (device)
// or null for the exact channel inverse. zraw (optional, N x ncol, ld N): the unscaled mode
// coefficients (Q^T r)/(lambda - theta), kept for the backward pass.
cudaError_t launch_chan_apply(const ChanPrec &cp, const double *w, const double *R, long long ldr,
                              const double *theta, int ncol, double *T, long long ldt, double *zraw,
                              cudaStream_t st);

// delta[m, j] = (Q_c^T G[ix_c, j])_q * zraw[m, j]  (dL/dg from dL/dt = G), N x ncol, ld N.
cudaError_t launch_chan_back(const ChanPrec &cp, const double *G, long long ldg, const double *zraw, int ncol,
                             double *delta, cudaStream_t st);

// Network outputs g = 1 + f for all (mode, column) items: gout (n x ncol, ld n).
cudaError_t launch_lp_forward(const LpModes &m, const double *w, const double *theta, int ncol, double *gout,
                              cudaStream_t st);

// grad = sum over items of delta[m, j] * d g[m, j] / d w (device, kLpParams);
// work: lp_grad_work_doubles() doubles.
size_t lp_grad_work_doubles();
cudaError_t lp_mlp_grad(const LpModes &m, const double *w, const double *theta, int ncol, const double *delta,
                        double *grad, double *work, cudaStream_t st);

// One Adam step on the device (step counts from 1).
cudaError_t lp_adam_step(double *w, const double *grad, double *mom, double *vel, int step, double lr,
                         cudaStream_t st);

// Loss pieces: per pair j (one CTA per column) te = T.E, ptt = PT.PT, ee = E.E -> sums[3 j..];
// then coefficients a_j, b_j of dL/dT = a E + b PT and the loss (mean over valid pairs).
cudaError_t launch_lp_pair_terms(const double *T, const double *PT, const double *E, long long ld, int n,
                                 int npair, double *sums, double *coef, double *loss, cudaStream_t st);
// G = a_j E + b_j PT
cudaError_t launch_lp_dldt(const double *E, const double *PT, long long ld, int n, int npair, const double *coef,
                           double *G, cudaStream_t st);

}  // namespace dvr3d
