// blocks.cu -- block-build kernels of the 2D (Radau) and 1D/2D (Jacobi) stages and the
// transforms that turn selected block eigenvectors into the columns of the contracted
// basis matrix Vt (P x N) used by the 3D assembly.
#include <cmath>

#include "blocks.cuh"
#include "common.cuh"

namespace dvr3d {

namespace {

// Radau 2D Hamiltonian of one angle (blc2d1 :3125-3219; z_blc2d1 :4038-4127 for the z-perp
// embedding) in the symmetrised pair basis (alpha <= beta - ipar, beta outer), full
// symmetric storage. One thread per element.
__global__ void radau_build_kernel(RadauBuild rb, double *H) {
    const int g = blockIdx.y;
    const int n = rb.n;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * n) return;
    const int row = (int)(idx % n), col = (int)(idx / n);
    const int ap = rb.pa[row], bp = rb.pb[row];  // (alpha', beta'), 0-based radial indices
    const int a = rb.pa[col], b = rb.pb[col];
    const double q = rb.ipar ? -1.0 : 1.0;
    const double x = rb.xalf[g];
    const int np = rb.npnt;
    auto hr = [&](int i, int j) { return rb.hr[(size_t)j * np + i]; };
    double h = 0.0;
    if (row == col && rb.jrot != 0 && rb.zperp) {
        // z-perp J > 0 diagonal (:4059-4085): k^2/4 (+ the Q term x / (1 - x^2) for k = 1) and
        // the s (J(J+1) - k^2)/4 / (1 - x^2) term; doubled for alpha = beta as in the reference
        double fact = rb.term;
        if (rb.kz == 1) fact = fact + rb.term3 * x / (1.0 - x * x);
        const double fact2 = rb.term2 / (1.0 - x * x);
        const double wa = 0.5 / (rb.r[a] * rb.r[a] * rb.urr1), wb = 0.5 / (rb.r[b] * rb.r[b] * rb.urr1);
        const double ws = (wa + wb) * fact + (wa + wb) * fact2;
        h += (a == b && rb.ipar == 0) ? 2.0 * ws : ws;
    } else if (row == col && rb.jrot != 0) {
        // J > 0 diagonal term (:3155-3177); doubled for alpha = beta as in the reference
        double fact = rb.term + rb.term2 / (1.0 - x);
        if (rb.kz == 1) fact += rb.term3 * (1.0 + x) / (1.0 - x);
        const double wa = 0.5 / (rb.r[a] * rb.r[a]), wb = 0.5 / (rb.r[b] * rb.r[b]);
        const double ws = (wa + wb) * fact / rb.urr1 - (wa + wb) * rb.xterm / (1.0 - x * x);
        h += (a == b && rb.ipar == 0) ? 2.0 * ws : ws;
    }
    if (b == bp) h += hr(ap, a);
    if (b == ap) h += q * hr(bp, a);
    if (a == bp) h += q * hr(ap, b);
    if (a == ap) h += hr(bp, b);
    if (a == ap && b == bp) h += pes_eval(rb.pes, rb.r[a], rb.r[b], x, a, b, g);
    if (a == bp && b == ap) h += q * pes_eval(rb.pes, rb.r[b], rb.r[a], x, b, a, g);
    const double f2 = 0.70710678118654752440;  // sqrt(0.5)
    if (ap == bp) h *= f2;
    if (a == b) h *= f2;
    H[(size_t)g * n * n + idx] = h;
}

// Jacobi 1D Hamiltonian of block (ic, ib) (mkham1 :2121-2225), full storage, n = npnta.
__global__ void jacobi_build1d_kernel(Jacobi1D jb, double *H) {
    const int blk = blockIdx.y;  // = ic * npntb + ib
    const int ic = blk / jb.npntb, ib = blk - ic * jb.npntb;
    const int n = jb.npnta;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * n) return;
    const int i = idx % n, j = idx / n;
    double h;
    if (jb.ztheta) {
        // theta first: a = angle; (ic, ib) index (r1, r2) = zr2r1 ? (ic, ib) : (ib, ic)
        const int i1 = jb.zr2r1 ? ic : ib, i2 = jb.zr2r1 ? ib : ic;
        const double w1 = 0.5 / (jb.r1[i1] * jb.r1[i1] * jb.ur1);
        const double w2 = 0.5 / (jb.r2[i2] * jb.r2[i2] * jb.ur2);
        h = jb.ta[(size_t)j * jb.lda + i] * (w1 + w2);
        if (i == j) {
            double wterm = 0.0;
            if (jb.jrot > 0) wterm = jb.zembed ? jb.term * w2 * jb.ur2 / jb.urr2 : jb.term * w1 * jb.ur1 / jb.urr1;
            double v = pes_eval(jb.pes, jb.r1[i1], jb.r2[i2], jb.xalf[i], i1, i2, i);
            if (jb.w3k != 0.0) {  // the extra term when the vibrational and rotational masses differ
                const double w3 = jb.w3k * ((jb.ur1 / jb.urr1 - 1.0) * w1 + (jb.ur2 / jb.urr2 - 1.0) * w2);
                v = v + w3 / (1.0 - jb.xalf[i] * jb.xalf[i]);
            }
            h += v + wterm;
        }
    } else {
        h = jb.ta[(size_t)j * jb.lda + i];
        if (i == j) {
            double v, wterm = 0.0;
            if (jb.zr2r1) {  // a = r2, b = r1, c = angle
                v = pes_eval(jb.pes, jb.r1[ib], jb.r2[i], jb.xalf[ic], ib, i, ic);
                if (jb.jrot > 0)
                    wterm = jb.zembed ? (jb.term * 0.5) / (jb.r2[i] * jb.r2[i] * jb.ur2)
                                      : (jb.term * 0.5) / (jb.r1[ib] * jb.r1[ib] * jb.ur1);
            } else {         // a = r1, b = r2, c = angle
                v = pes_eval(jb.pes, jb.r1[i], jb.r2[ib], jb.xalf[ic], i, ib, ic);
                if (jb.jrot > 0)
                    wterm = jb.zembed ? (jb.term * 0.5) / (jb.r2[ib] * jb.r2[ib] * jb.ur2)
                                      : (jb.term * 0.5) / (jb.r1[i] * jb.r1[i] * jb.ur1);
            }
            h += v + wterm;
        }
    }
    H[(size_t)blk * n * n + idx] = h;
}

// Jacobi 2D Hamiltonian of block ic (mkham2 :2228-2298):
// H2[j,j'] = Tb[b(j), b(j')] (u_j . u_j') + delta_jj' e1_j, full storage.
__global__ void jacobi_build2d_kernel(Jacobi2D jb, double *H2) {
    const int ic = blockIdx.y;
    const int n2 = jb.n2[ic];
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n2 * n2) return;
    const int i = idx % n2, j = idx / n2;
    const long long ub = jb.uoff[ic];  // U (npnta x n2) of this block
    const double *ui = jb.U + ub + (size_t)i * jb.npnta;
    const double *uj = jb.U + ub + (size_t)j * jb.npnta;
    double s = 0.0;
    for (int k = 0; k < jb.npnta; ++k) s += ui[k] * uj[k];
    const int bi = jb.bidx[jb.e1off[ic] + i], bj = jb.bidx[jb.e1off[ic] + j];
    double h = s * jb.tb[(size_t)bj * jb.ldb + bi];
    if (i == j) h += jb.e1[jb.e1off[ic] + i];
    H2[jb.hoff[ic] + idx] = h;
}

// Contracted basis of one Jacobi block (mkham3 :2362-2407):
// Vt[(k*npntb + b), col0 + j] = sw[k,b] * sum_{i in group b} V2[i, j] U[k, i].
__global__ void jacobi_ctrans_kernel(Jacobi2D jb, CTrans ct, const double *V2, double *Vt) {
    const int ic = blockIdx.y;
    const int s = ct.s2[ic];
    if (s == 0) return;
    const int P = jb.npnta * jb.npntb;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)P * s) return;
    const int p = (int)(idx % P), j = (int)(idx / P);
    const int k = p / jb.npntb, b = p - k * jb.npntb;
    const int n2 = jb.n2[ic];
    const double *v2 = V2 + ct.v2off[ic] + (size_t)j * n2;
    const double *U = jb.U + jb.uoff[ic];
    const int g0 = ct.gstart[ic * (jb.npntb + 1) + b], g1 = ct.gstart[ic * (jb.npntb + 1) + b + 1];
    double acc = 0.0;
    for (int i = g0; i < g1; ++i) acc += v2[i] * U[(size_t)i * jb.npnta + k];
    Vt[(size_t)(ct.col0[ic] + j) * ct.ldv + p] = acc * ct.sw[p];
}

// Radau: scale rows of the selected 2D eigenvectors by sqrt(w_p) (blc2d2 :3509-3566 has a
// diagonal pair-basis kernel L(g,g') w_p, so H3 = (sqrt(w) V)^T (sqrt(w) V) o L).
__global__ void scale_rows_kernel(double *Vt, int P, long long ncol, const double *sw) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)P * ncol) return;
    Vt[idx] *= sw[idx % P];
}

// gather: dst[i] = src[map[i]]
__global__ void gather_kernel(const double *src, const long long *map, double *dst, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[map[i]];
}

}  // namespace

void launch_radau_build(const RadauBuild &rb, int nalf, double *H, cudaStream_t st) {
    const long long nn = (long long)rb.n * rb.n;
    dim3 grid((unsigned)((nn + 255) / 256), nalf);
    DVR3D_COUNT_LAUNCH(1);
    radau_build_kernel<<<grid, 256, 0, st>>>(rb, H);
}

void launch_jacobi_build1d(const Jacobi1D &jb, int nblk, double *H, cudaStream_t st) {
    const int nn = jb.npnta * jb.npnta;
    dim3 grid((nn + 127) / 128, nblk);
    DVR3D_COUNT_LAUNCH(1);
    jacobi_build1d_kernel<<<grid, 128, 0, st>>>(jb, H);
}

void launch_jacobi_build2d(const Jacobi2D &jb, int nblk, int n2max, double *H2, cudaStream_t st) {
    const long long nn = (long long)n2max * n2max;
    dim3 grid((unsigned)((nn + 255) / 256), nblk);
    DVR3D_COUNT_LAUNCH(1);
    jacobi_build2d_kernel<<<grid, 256, 0, st>>>(jb, H2);
}

void launch_jacobi_ctrans(const Jacobi2D &jb, const CTrans &ct, int nblk, int s2max,
                          const double *V2, double *Vt, cudaStream_t st) {
    const long long P = (long long)jb.npnta * jb.npntb;
    const long long tot = P * s2max;
    if (tot == 0) return;
    dim3 grid((unsigned)((tot + 255) / 256), nblk);
    DVR3D_COUNT_LAUNCH(1);
    jacobi_ctrans_kernel<<<grid, 256, 0, st>>>(jb, ct, V2, Vt);
}

void launch_scale_rows(double *Vt, int P, long long ncol, const double *sw, cudaStream_t st) {
    const long long tot = (long long)P * ncol;
    if (tot == 0) return;
    DVR3D_COUNT_LAUNCH(1);
    scale_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(Vt, P, ncol, sw);
}

void launch_gather(const double *src, const long long *map, double *dst, long long n, cudaStream_t st) {
    if (n == 0) return;
    DVR3D_COUNT_LAUNCH(1);
    gather_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, map, dst, n);
}

}  // namespace dvr3d
