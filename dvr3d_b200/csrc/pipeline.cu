// pipeline.cu -- the per-k-block solve on one GPU.
//
// Stage order follows nfmain (:3006-3121) for Radau idia=-2 and jhmain (:1915-2118) for
// the Jacobi / idia=-1 orderings; the reference's scratch units (ivecs1, ieigs1, intvec,
// ivint, iband ...) become device buffers that stay resident between stages. The host
// only plans sizes (selection counts come back as a few integers per block).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "blocks.cuh"
#include "eig_batched.cuh"
#include "band_eig.cuh"
#include "eig_dense.cuh"
#include "gemm64.cuh"
#include "learned_precond.cuh"
#include "pipeline.cuh"
#include "tc_gemm.cuh"

#define CK(x)                                          \
    do {                                               \
        cudaError_t e_ = (x);                          \
        if (e_ != cudaSuccess) throw CudaFail{e_, #x}; \
    } while (0)

namespace dvr3d {

long long g_kernel_launches = 0;

namespace {
thread_local long long t_h2d = 0, t_d2h = 0;
}

void note_h2d(long long bytes) { t_h2d += bytes; }
void note_d2h(long long bytes) { t_d2h += bytes; }

// ---------------------------------------------------------------- arena
DeviceArena::~DeviceArena() { release_all(); }

void *DeviceArena::get(const std::string &name, size_t bytes) {
    if (bytes == 0) bytes = 16;
    Buf &b = bufs_[name];
    if (b.bytes < bytes) {
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
        size_t nb = std::max(bytes, b.bytes + b.bytes / 4);
        nb = (nb + 255) & ~(size_t)255;
        cudaError_t e = cudaMalloc(&b.p, nb);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw HostError{DVR3D_ERR_NOMEM, "device allocation of " + std::to_string(nb) + " bytes for " + name + " failed"};
        }
        b.bytes = nb;
    }
    return b.p;
}

size_t DeviceArena::bytes_held() const {
    size_t s = 0;
    for (auto &kv : bufs_) s += kv.second.bytes;
    return s;
}

void DeviceArena::release_all() {
    for (auto &kv : bufs_)
        if (kv.second.p) cudaFree(kv.second.p);
    bufs_.clear();
}

namespace {

template <class T>
T *upload(dvr3d_ctx *ctx, const std::string &name, const std::vector<T> &v) {
    T *p = ctx->arena.get_t<T>(name, std::max<size_t>(v.size(), 1));
    if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    t_h2d += (long long)(v.size() * sizeof(T));
    return p;
}

template <class T>
std::vector<T> download(dvr3d_ctx *ctx, const T *p, size_t n) {
    std::vector<T> v(n);
    if (n) CK(cudaMemcpyAsync(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    t_d2h += (long long)(n * sizeof(T));
    CK(cudaStreamSynchronize(ctx->stream));
    return v;
}

inline long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

void check_dev_err(dvr3d_ctx *ctx, const int *err_dev, const char *stage) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, err_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    t_d2h += sizeof(int);
    CK(cudaStreamSynchronize(ctx->stream));
    if (e == kDevBarrierTimeout) throw HostError{DVR3D_ERR_NOCONV, std::string(stage) + ": grid barrier wait exceeded its limit"};
    if (e == kDevNoConv) {
        int f[4];
        invit_fail_info(ctx->stream, f);
        std::string where;
        if (f[0]) where = " (block " + std::to_string(f[1] + 1) + ", vector " + std::to_string(f[2] + 1) + " of order " +
                          std::to_string(f[3]) + ")";
        throw HostError{DVR3D_ERR_NOCONV, std::string(stage) + ": did not converge" + where};
    }
    if (e != 0) throw HostError{DVR3D_ERR_NOCONV, std::string(stage) + ": device error flag " + std::to_string(e)};
}

// Flag raised by the batched eigenvector kernels when inverse iteration fails its growth
// test; cleared at the start of each solve, read after the 1D/2D stage and at the end.
int *ev_err(dvr3d_ctx *ctx) { return ctx->arena.get_t<int>("ev_err", 1); }

// ---------------------------------------------------------------- Radau (nfmain)
void radau_stage(dvr3d_ctx *ctx, const BlockPlan &p, Contracted &out) {
    cudaStream_t st = ctx->stream;
    const int npnt = p.npnt1, ipar = p.ipar, nalf = p.nalf;
    const int n = npnt * (npnt + 1 - 2 * ipar) / 2;
    if (n > 1024) throw HostError{DVR3D_ERR_UNSUPPORTED, "Radau 2D block larger than 1024"};
    std::vector<int> pa, pb;
    for (int beta = 1; beta <= npnt; ++beta)
        for (int alpha = 1; alpha <= beta - ipar; ++alpha) {
            pa.push_back(alpha - 1);
            pb.push_back(beta - 1);
        }
    double *r = upload(ctx, "r1", p.r1);
    double *hr = upload(ctx, "xk1", p.xk1);
    double *xalf = upload(ctx, "xalf", p.xalf);
    double *xl = upload(ctx, "xlmatr", p.xlmatr);
    int *dpa = upload(ctx, "pa", pa);
    int *dpb = upload(ctx, "pb", pb);
    double *H = ctx->arena.get_t<double>("blk2", (size_t)nalf * n * n);
    RadauBuild rb{};
    rb.n = n;
    rb.npnt = npnt;
    rb.ipar = ipar;
    rb.jrot = p.jrot;
    rb.kz = p.kz;
    rb.pa = dpa;
    rb.pb = dpb;
    rb.r = r;
    rb.hr = hr;
    rb.xalf = xalf;
    rb.term = p.nf_term;
    rb.term2 = p.nf_term2;
    rb.term3 = p.nf_term3;
    rb.zperp = p.zperp ? 1 : 0;
    rb.urr1 = p.urr1;
    rb.xterm = p.zperp ? 0.0 : (double)(p.kz * p.kz) * (1.0 / p.ur1 - 1.0 / p.urr1) * p.xp0;
    rb.pes = ctx->pes;
    if (rb.pes.kind == DVR3D_PES_GRID) {
        const std::vector<double> &tab = ctx->pes_table(p.kz);
        if (tab.size() < (size_t)nalf * p.npnt1 * p.npnt1)
            throw HostError{DVR3D_ERR_ARG, "tabulated PES smaller than the DVR grid"};
        rb.pes.grid = upload(ctx, "pesgrid", tab);
        rb.pes.npnt1 = p.npnt1;
        rb.pes.npnt2 = p.npnt1;
    }
    launch_radau_build(rb, nalf, H, st);
    CK(cudaGetLastError());
    std::vector<int> nv(nalf, n);
    std::vector<long long> aoff(nalf), voff(nalf);
    for (int b = 0; b < nalf; ++b) {
        aoff[b] = (long long)b * n * n;
        voff[b] = (long long)b * n;
    }
    BatchDesc bd{nalf, upload(ctx, "bd_n", nv), upload(ctx, "bd_aoff", aoff), upload(ctx, "bd_voff", voff)};
    double *d = ctx->arena.get_t<double>("bd_d", (size_t)nalf * n);
    double *e = ctx->arena.get_t<double>("bd_e", (size_t)nalf * n);
    double *tau = ctx->arena.get_t<double>("bd_tau", (size_t)nalf * n);
    double *w = ctx->arena.get_t<double>("bd_w", (size_t)nalf * n);
    int *cnt = ctx->arena.get_t<int>("bd_cnt", nalf);
    launch_tridiag_batched(bd, H, d, e, tau, n, st);
    launch_eigvals_batched(bd, d, e, w, cnt, p.zcut ? 1 : 0, p.emax2_au, st);
    CK(cudaGetLastError());
    // selection: cut2dr (:3323-3377) or choosr (:3223-3319), then testiv (:3380-3451)
    std::vector<int> sel = download(ctx, cnt, nalf);
    if (p.zcut) {
        long long tot = 0;
        for (int b = 0; b < nalf; ++b) {
            tot += sel[b];
            if (tot > p.max3d) throw HostError{DVR3D_ERR_CORE_MAX3D, "number of 2d eigenvalues greater than max3d"};
        }
    } else {
        std::vector<double> all = download(ctx, w, (size_t)nalf * n);
        std::vector<double> srt = all;
        std::sort(srt.begin(), srt.end());
        const double emax = ((long long)srt.size() <= p.max3d) ? srt.back() : srt[p.max3d - 1];
        for (int b = 0; b < nalf; ++b) {
            int c = 0;
            while (c < n && all[(size_t)b * n + c] <= emax) ++c;
            sel[b] = c;
        }
    }
    if (p.jrot > 0) {
        int iend = nalf;
        for (int i = nalf / 2; i <= nalf; ++i)
            if (i >= 1 && sel[i - 1] == 0) {
                iend = i;
                break;
            }
        for (int i = iend + 1; i <= nalf; ++i) sel[i - 1] = 0;
        if (sel[nalf - 1] > 0) {
            if (p.zlin) sel[nalf - 1] = 0;
            else throw HostError{DVR3D_ERR_THETA0, "bisector embedding: wavefunction has amplitude for theta = 0"};
        }
    }
    const int N = std::accumulate(sel.begin(), sel.end(), 0);
    out.iv2 = sel;
    out.nblocks = nalf;
    out.N = N;
    out.P = n;
    out.ldv = round_up(n, 16);
    if (N == 0) return;
    const long long ncol = round_up(N, 64);
    out.Vt = ctx->arena.get_t<double>("vt", (size_t)out.ldv * ncol);
    CK(cudaMemsetAsync(out.Vt, 0, sizeof(double) * out.ldv * ncol, st));
    std::vector<long long> zoff(nalf);
    std::vector<int> zld(nalf, (int)out.ldv);
    std::vector<int> gcol(N);
    std::vector<long long> emap(N);
    long long col = 0;
    for (int b = 0; b < nalf; ++b) {
        zoff[b] = col * out.ldv;
        for (int j = 0; j < sel[b]; ++j) {
            gcol[col + j] = b;
            emap[col + j] = voff[b] + j;
        }
        col += sel[b];
    }
    launch_eigvecs_batched_fast(bd, H, d, e, tau, w, upload(ctx, "sel", sel), upload(ctx, "zoff", zoff),
                                upload(ctx, "zld", zld), out.Vt, n, ev_err(ctx), st);
    CK(cudaGetLastError());
    // sqrt of the pair weight w_p = 1/(2 mu r_a^2) + 1/(2 mu r_b^2) (blc2d2 :3537-3539)
    std::vector<double> sw(out.ldv, 0.0);
    for (int q = 0; q < n; ++q) {
        const double ra = p.r1[pa[q]], rbv = p.r1[pb[q]];
        sw[q] = std::sqrt(0.5 / (ra * ra * p.ur1) + 0.5 / (rbv * rbv * p.ur1));
    }
    launch_scale_rows(out.Vt, (int)out.ldv, N, upload(ctx, "sw", sw), st);
    out.sw.assign(sw.begin(), sw.begin() + n);
    out.g = upload(ctx, "gcol", gcol);
    out.e2 = ctx->arena.get_t<double>("e2", N);
    launch_gather(w, upload(ctx, "emap", emap), out.e2, N, st);
    out.T = xl;
    out.ldt = p.idvr;
    CK(cudaGetLastError());
}

// ---------------------------------------------------------------- Jacobi (jhmain)
void jacobi_stage(dvr3d_ctx *ctx, const BlockPlan &p, Contracted &out) {
    cudaStream_t st = ctx->stream;
    const int na = p.npnta, nbp = p.npntb, ncp = p.npntc;
    if (na > 1024) throw HostError{DVR3D_ERR_UNSUPPORTED, "1D block larger than 1024"};
    double *r1 = upload(ctx, "r1", p.r1);
    double *r2 = upload(ctx, "r2", p.r2);
    double *xalf = upload(ctx, "xalf", p.xalf);
    double *xk1 = upload(ctx, "xk1", p.xk1);
    double *xk2 = upload(ctx, "xk2", p.xk2);
    double *xl = upload(ctx, "xlmatr", p.xlmatr);
    // ---- 1D stage (mkham1 / diag / cut1d, :1975-2003)
    Jacobi1D j1{};
    j1.npnta = na;
    j1.npntb = nbp;
    j1.npntc = ncp;
    j1.ztheta = p.ztheta;
    j1.zr2r1 = p.zr2r1;
    j1.zembed = p.zembed;
    j1.jrot = p.jrot;
    j1.r1 = r1;
    j1.r2 = r2;
    j1.xalf = xalf;
    if (p.ztheta) {
        j1.ta = xl;
        j1.lda = p.idvr;
    } else {
        j1.ta = p.zr2r1 ? xk2 : xk1;
        j1.lda = p.zr2r1 ? p.npnt2 : p.npnt1;
    }
    j1.ur1 = p.ur1;
    j1.ur2 = p.ur2;
    j1.urr1 = p.urr1;
    j1.urr2 = p.urr2;
    j1.term = p.term;
    j1.w3k = (p.ztheta && p.jrot > 0 && p.kz > 0) ? (double)(p.kz * p.kz) * p.xp0 : 0.0;
    j1.pes = ctx->pes;
    if (j1.pes.kind == DVR3D_PES_GRID) {
        const std::vector<double> &tab = ctx->pes_table(p.kz);
        if (tab.size() < (size_t)p.idvr * p.npnt1 * p.npnt2)
            throw HostError{DVR3D_ERR_ARG, "tabulated PES smaller than the DVR grid"};
        j1.pes.grid = upload(ctx, "pesgrid", tab);
        j1.pes.npnt1 = p.npnt1;
        j1.pes.npnt2 = p.npnt2;
    }
    const int nb1 = ncp * nbp;
    double *H1 = ctx->arena.get_t<double>("blk1", (size_t)nb1 * na * na);
    launch_jacobi_build1d(j1, nb1, H1, st);
    std::vector<int> nv1(nb1, na);
    std::vector<long long> aoff1(nb1), voff1(nb1);
    for (int b = 0; b < nb1; ++b) {
        aoff1[b] = (long long)b * na * na;
        voff1[b] = (long long)b * na;
    }
    BatchDesc bd1{nb1, upload(ctx, "bd1_n", nv1), upload(ctx, "bd1_aoff", aoff1), upload(ctx, "bd1_voff", voff1)};
    double *d1 = ctx->arena.get_t<double>("bd1_d", (size_t)nb1 * na);
    double *e1 = ctx->arena.get_t<double>("bd1_e", (size_t)nb1 * na);
    double *t1 = ctx->arena.get_t<double>("bd1_tau", (size_t)nb1 * na);
    double *w1 = ctx->arena.get_t<double>("bd1_w", (size_t)nb1 * na);
    int *c1 = ctx->arena.get_t<int>("bd1_cnt", nb1);
    launch_tridiag_batched(bd1, H1, d1, e1, t1, na, st);
    launch_eigvals_batched(bd1, d1, e1, w1, c1, p.zall ? 0 : 2, p.emax1_au, st);
    CK(cudaGetLastError());
    std::vector<int> iv1 = download(ctx, c1, nb1);
    std::vector<int> n2(ncp, 0);
    std::vector<long long> uoff(ncp), zoff1(nb1), e1off(ncp);
    long long ut = 0, et = 0;
    for (int ic = 0; ic < ncp; ++ic) {
        uoff[ic] = ut;
        e1off[ic] = et;
        int s = 0;
        for (int ib = 0; ib < nbp; ++ib) {
            zoff1[ic * nbp + ib] = ut + (long long)na * s;
            s += iv1[ic * nbp + ib];
            if (s > p.max2d && !p.zall) throw HostError{DVR3D_ERR_CORE_MAX2D, "core exceeded: reduce cut-off emax1"};
        }
        n2[ic] = s;
        ut += (long long)na * s;
        et += s;
    }
    double *U = ctx->arena.get_t<double>("u1", (size_t)std::max<long long>(ut, 1));
    {
        std::vector<int> zld1(nb1, na);
        launch_eigvecs_batched_fast(bd1, H1, d1, e1, t1, w1, upload(ctx, "sel1", iv1), upload(ctx, "zoff1", zoff1),
                                    upload(ctx, "zld1", zld1), U, na, ev_err(ctx), st);
        CK(cudaGetLastError());
    }
    // 1D eigenvalues and coordinate-b index of each 2D basis function
    std::vector<long long> e1map(std::max<long long>(et, 1));
    std::vector<int> bidx(std::max<long long>(et, 1));
    for (int ic = 0; ic < ncp; ++ic) {
        long long q = e1off[ic];
        for (int ib = 0; ib < nbp; ++ib)
            for (int jj = 0; jj < iv1[ic * nbp + ib]; ++jj) {
                e1map[q] = voff1[ic * nbp + ib] + jj;
                bidx[q] = ib;
                ++q;
            }
    }
    double *e1v = ctx->arena.get_t<double>("e1v", (size_t)std::max<long long>(et, 1));
    launch_gather(w1, upload(ctx, "e1map", e1map), e1v, et, st);
    // ---- 2D stage (mkham2 / diag / cut2d | choose, :2019-2053)
    std::vector<int> blocks;  // ic with n2 > 0
    for (int ic = 0; ic < ncp; ++ic)
        if (n2[ic] > 0) blocks.push_back(ic);
    const int nb2 = (int)blocks.size();
    int n2max = 0;
    std::vector<long long> hoff(ncp, 0), aoff2, voff2;
    std::vector<int> nv2;
    long long ht = 0, vt = 0;
    for (int ic = 0; ic < ncp; ++ic) {
        hoff[ic] = ht;
        ht += (long long)n2[ic] * n2[ic];
        n2max = std::max(n2max, n2[ic]);
    }
    for (int ic : blocks) {
        nv2.push_back(n2[ic]);
        aoff2.push_back(hoff[ic]);
        voff2.push_back(vt);
        vt += n2[ic];
    }
    if (n2max > 1024) throw HostError{DVR3D_ERR_UNSUPPORTED, "2D block larger than 1024"};
    Jacobi2D j2{};
    j2.npnta = na;
    j2.npntb = nbp;
    j2.n2 = upload(ctx, "n2", n2);
    j2.uoff = upload(ctx, "uoff", uoff);
    j2.U = U;
    j2.bidx = upload(ctx, "bidx", bidx);
    j2.e1off = upload(ctx, "e1off", e1off);
    j2.e1 = e1v;
    if (p.ztheta) {
        j2.tb = p.zr2r1 ? xk2 : xk1;
        j2.ldb = p.zr2r1 ? p.npnt2 : p.npnt1;
    } else {
        j2.tb = p.zr2r1 ? xk1 : xk2;
        j2.ldb = p.zr2r1 ? p.npnt1 : p.npnt2;
    }
    j2.hoff = upload(ctx, "hoff", hoff);
    double *H2 = ctx->arena.get_t<double>("blk2", (size_t)std::max<long long>(ht, 1));
    std::vector<int> sel2(nb2, 0);
    std::vector<int> s2(ncp, 0);
    double *d2 = nullptr, *e2d = nullptr, *t2 = nullptr, *w2 = nullptr;
    BatchDesc bd2{};
    if (nb2 > 0) {
        launch_jacobi_build2d(j2, ncp, n2max, H2, st);
        bd2 = BatchDesc{nb2, upload(ctx, "bd2_n", nv2), upload(ctx, "bd2_aoff", aoff2), upload(ctx, "bd2_voff", voff2)};
        d2 = ctx->arena.get_t<double>("bd2_d", (size_t)vt);
        e2d = ctx->arena.get_t<double>("bd2_e", (size_t)vt);
        t2 = ctx->arena.get_t<double>("bd2_tau", (size_t)vt);
        w2 = ctx->arena.get_t<double>("bd2_w", (size_t)vt);
        int *c2 = ctx->arena.get_t<int>("bd2_cnt", nb2);
        launch_tridiag_batched(bd2, H2, d2, e2d, t2, n2max, st);
        const bool zcut = p.zcut;
        launch_eigvals_batched(bd2, d2, e2d, w2, c2, zcut ? 2 : 0, p.emax2_au, st);
        CK(cudaGetLastError());
        sel2 = download(ctx, c2, nb2);
        if (zcut) {
            long long tot = 0;
            for (int q = 0; q < nb2; ++q) {
                tot += sel2[q];
                if (tot > p.max3d && !p.zall) throw HostError{DVR3D_ERR_CORE_MAX3D, "core exceeded: reduce cut-off emax2"};
            }
        } else {
            // choose (:2767-2867): the max3d lowest over all blocks, ties to the lower block
            std::vector<double> all = download(ctx, w2, (size_t)vt);
            long long nhamsm = vt;
            long long low3d = std::min<long long>(p.max3d, nhamsm);
            std::vector<int> ptr(nb2, 0);
            for (long long q = 0; q < low3d; ++q) {
                int best = -1;
                double bv = 0.0;
                for (int bb = 0; bb < nb2; ++bb) {
                    if (ptr[bb] >= nv2[bb]) continue;
                    const double v = all[voff2[bb] + ptr[bb]];
                    if (best < 0 || v < bv) {
                        best = bb;
                        bv = v;
                    }
                }
                ptr[best] += 1;
            }
            sel2 = ptr;
        }
        for (int q = 0; q < nb2; ++q) s2[blocks[q]] = sel2[q];
    }
    const int N = std::accumulate(s2.begin(), s2.end(), 0);
    out.iv2 = s2;
    out.nblocks = ncp;
    out.N = N;
    out.P = na * nbp;
    out.ldv = round_up(out.P, 16);
    if (N == 0) return;
    // 2D eigenvectors of the selected levels
    std::vector<long long> v2off(ncp, 0), zoff2(nb2);
    std::vector<int> zld2(nb2);
    long long v2t = 0;
    for (int q = 0; q < nb2; ++q) {
        const int ic = blocks[q];
        v2off[ic] = v2t;
        zoff2[q] = v2t;
        zld2[q] = n2[ic];
        v2t += (long long)n2[ic] * sel2[q];
    }
    double *V2 = ctx->arena.get_t<double>("v2", (size_t)std::max<long long>(v2t, 1));
    {
        launch_eigvecs_batched_fast(bd2, H2, d2, e2d, t2, w2, upload(ctx, "sel2", sel2), upload(ctx, "zoff2", zoff2),
                                    upload(ctx, "zld2", zld2), V2, n2max, ev_err(ctx), st);
        CK(cudaGetLastError());
    }
    // contracted basis (mkham3 first part :2362-2411)
    const long long ncol = round_up(N, 64);
    out.Vt = ctx->arena.get_t<double>("vt", (size_t)out.ldv * ncol);
    CK(cudaMemsetAsync(out.Vt, 0, sizeof(double) * out.ldv * ncol, st));
    std::vector<int> gstart((size_t)ncp * (nbp + 1));
    std::vector<long long> col0(ncp);
    std::vector<int> gcol(N);
    std::vector<long long> emap(N);
    long long col = 0;
    int s2max = 0;
    for (int ic = 0; ic < ncp; ++ic) {
        int s = 0;
        for (int ib = 0; ib < nbp; ++ib) {
            gstart[(size_t)ic * (nbp + 1) + ib] = s;
            s += iv1[ic * nbp + ib];
        }
        gstart[(size_t)ic * (nbp + 1) + nbp] = s;
        col0[ic] = col;
        s2max = std::max(s2max, s2[ic]);
        col += s2[ic];
    }
    for (int q = 0; q < nb2; ++q) {
        const int ic = blocks[q];
        for (int j = 0; j < sel2[q]; ++j) {
            gcol[col0[ic] + j] = ic;
            emap[col0[ic] + j] = voff2[q] + j;
        }
    }
    std::vector<double> sw(out.P, 1.0);
    if (!p.ztheta) {
        for (int ia = 0; ia < na; ++ia)
            for (int ib = 0; ib < nbp; ++ib) {
                const int i1 = p.zr2r1 ? ib : ia, i2 = p.zr2r1 ? ia : ib;
                const double wsum = 0.5 / (p.r1[i1] * p.r1[i1] * p.ur1) + 0.5 / (p.r2[i2] * p.r2[i2] * p.ur2);
                sw[(size_t)ia * nbp + ib] = std::sqrt(wsum);
            }
    }
    CTrans ct{};
    ct.s2 = upload(ctx, "s2", s2);
    ct.v2off = upload(ctx, "v2off", v2off);
    ct.gstart = upload(ctx, "gstart", gstart);
    ct.col0 = upload(ctx, "col0", col0);
    ct.sw = upload(ctx, "sw", sw);
    out.sw = sw;
    ct.ldv = out.ldv;
    launch_jacobi_ctrans(j2, ct, ncp, s2max, V2, out.Vt, st);
    out.g = upload(ctx, "gcol", gcol);
    out.e2 = ctx->arena.get_t<double>("e2", N);
    launch_gather(w2, upload(ctx, "emap", emap), out.e2, N, st);
    if (p.ztheta) {
        out.T = p.zr2r1 ? xk1 : xk2;
        out.ldt = p.zr2r1 ? p.npnt1 : p.npnt2;
    } else {
        out.T = xl;
        out.ldt = p.idvr;
    }
    CK(cudaGetLastError());
}

__global__ void resid_kernel(const double *R, const double *Z, const double *w, int n, long long ld, int nev,
                             double *res) {
    const int j = blockIdx.x;
    if (j >= nev) return;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double r = R[(size_t)j * ld + i] - w[j] * Z[(size_t)j * ld + i];
        s += r * r;
    }
    __shared__ double red[32];
    s = block_sum(s, red);
    if (threadIdx.x == 0) res[j] = sqrt(s);
}

}  // namespace

// ---------------------------------------------------------------- channel blocks of H3
namespace {
// H null: the entries come from the split-BF16 slices (hi + lo).
__global__ void chan_gather_kernel(const double *H, const __nv_bfloat16 *hi, const __nv_bfloat16 *lo, long long ldh,
                                   const int *idx, const int *off, const long long *qoff, const int *n, double *A) {
    const int c = blockIdx.y, nc = n[c];
    const int *ix = idx + off[c];
    double *a = A + qoff[c];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nc * nc; t += gridDim.x * blockDim.x) {
        const int p = t % nc, q = t / nc;
        const size_t e = (size_t)ix[q] * ldh + ix[p];
        a[t] = H ? H[e] : (double)__bfloat162float(hi[e]) + (double)__bfloat162float(lo[e]);
    }
}
}  // namespace

void channel_setup(dvr3d_ctx *ctx, const H3Op &op, const Contracted &C, ChanPrec &cp,
                   std::vector<double> *lam_host, std::vector<int> *chan_of_mode) {
    cudaStream_t st = ctx->stream;
    const int N = C.N, nb = C.nblocks;
    std::vector<int> col0(nb, 0);
    for (int b = 1; b < nb; ++b) col0[b] = col0[b - 1] + C.iv2[b - 1];
    const int kmax = *std::max_element(C.iv2.begin(), C.iv2.end());
    std::vector<int> n(kmax, 0), off(kmax, 0), idx;
    std::vector<long long> qoff(kmax, 0), voff(kmax, 0);
    idx.reserve(N);
    long long qt = 0;
    int nmax = 0;
    for (int c = 0; c < kmax; ++c) {
        off[c] = (int)idx.size();
        voff[c] = off[c];
        for (int b = 0; b < nb; ++b)
            if (C.iv2[b] > c) idx.push_back(col0[b] + c);
        n[c] = (int)idx.size() - off[c];
        qoff[c] = qt;
        qt += (long long)n[c] * n[c];
        nmax = std::max(nmax, n[c]);
    }
    if (nmax > 1024) throw HostError{DVR3D_ERR_UNSUPPORTED, "channel block larger than 1024"};
    int *dn = upload(ctx, "ch_n", n);
    int *doff = upload(ctx, "ch_off", off);
    long long *dq = upload(ctx, "ch_qoff", qoff);
    long long *dv = upload(ctx, "ch_voff", voff);
    int *didx = upload(ctx, "ch_idx", idx);
    double *A = ctx->arena.get_t<double>("ch_A", (size_t)qt);
    double *Q = ctx->arena.get_t<double>("ch_Q", (size_t)qt);
    DVR3D_COUNT_LAUNCH(1);
    chan_gather_kernel<<<dim3((unsigned)((nmax * nmax + 255) / 256), kmax), 256, 0, st>>>(
        op.H3, op.hi, op.lo, op.H3 ? op.ldh : op.ld, didx, doff, dq, dn, A);
    CK(cudaGetLastError());
    BatchDesc bd{kmax, dn, dq, dv};
    double *d = ctx->arena.get_t<double>("ch_d", N), *e = ctx->arena.get_t<double>("ch_e", N);
    double *tau = ctx->arena.get_t<double>("ch_tau", N), *lam = ctx->arena.get_t<double>("ch_lam", N);
    int *cnt = ctx->arena.get_t<int>("ch_cnt", kmax);
    launch_tridiag_batched(bd, A, d, e, tau, nmax, st);
    launch_eigvals_batched(bd, d, e, lam, cnt, 0, 0.0, st);
    launch_eigvecs_batched_fast(bd, A, d, e, tau, lam, dn, dq, dn, Q, nmax, ev_err(ctx), st);
    CK(cudaGetLastError());
    // per-mode features
    std::vector<double> lh = download(ctx, lam, N), e2h = download(ctx, C.e2, N);
    std::vector<double> f1(N), f2(N), f3(N);
    const auto mm = std::minmax_element(lh.begin(), lh.end());
    const double s = std::max(1.0e-6, 0.25 * (*mm.second - *mm.first));
    for (int c = 0; c < kmax; ++c) {
        double me = 0.0;
        for (int p = 0; p < n[c]; ++p) me += e2h[idx[off[c] + p]];
        me /= std::max(1, n[c]);
        for (int q = 0; q < n[c]; ++q) {
            const int m = off[c] + q;
            f1[m] = (lh[m] - me) / s;
            f2[m] = (double)c / kmax;
            f3[m] = n[c] > 1 ? (double)q / (n[c] - 1) : 0.0;
        }
    }
    if (lam_host) *lam_host = lh;
    if (chan_of_mode) {
        chan_of_mode->assign(N, 0);
        for (int c = 0; c < kmax; ++c)
            for (int q = 0; q < n[c]; ++q) (*chan_of_mode)[off[c] + q] = c;
    }
    cp.nch = kmax;
    cp.nmax = nmax;
    cp.n = dn;
    cp.off = doff;
    cp.qoff = dq;
    cp.idx = didx;
    cp.Q = Q;
    cp.modes.lam = lam;
    cp.modes.f1 = upload(ctx, "ch_f1", f1);
    cp.modes.f2 = upload(ctx, "ch_f2", f2);
    cp.modes.f3 = upload(ctx, "ch_f3", f3);
    cp.modes.n = N;
    cp.modes.scale = s;
}

// ---------------------------------------------------------------- dense eigensolver
void dense_lowest(dvr3d_ctx *ctx, double *A, long long lda, int n, int nev, bool vecs, double *w, double *Z,
                  long long ldz, const char *tag, bool time_panels, DenseOut *out) {
    cudaStream_t st = ctx->stream;
    const std::string t(tag);
    DenseTri dt{};
    dt.A = A;
    dt.lda = lda;
    dt.n = n;
    dt.d = ctx->arena.get_t<double>(t + "d", n);
    dt.e = ctx->arena.get_t<double>(t + "e", n);
    dt.tau = ctx->arena.get_t<double>(t + "tau", n);
    int G = ctx->dense_grid;
    if ((long long)n > 256LL * G) throw HostError{DVR3D_ERR_UNSUPPORTED, "matrix too large for the dense eigensolver"};
    dt.nbmax = dense_panel_width();
    dt.NT = (n + 63) / 64;
    dt.V = ctx->arena.get_t<double>(t + "V", (size_t)n * dt.nbmax);
    dt.W = ctx->arena.get_t<double>(t + "W", (size_t)n * dt.nbmax);
    // the panel kernel reads all panel columns of V and W unconditionally: finite values
    CK(cudaMemsetAsync(dt.V, 0, sizeof(double) * n * dt.nbmax, st));
    CK(cudaMemsetAsync(dt.W, 0, sizeof(double) * n * dt.nbmax, st));
    dt.acol = ctx->arena.get_t<double>(t + "acol", n);
    dt.ybuf = ctx->arena.get_t<double>(t + "y", n);
    dt.P = ctx->arena.get_t<double>(t + "P", (size_t)dt.NT * dt.NT * 64);
    dt.part = ctx->arena.get_t<double>(t + "part", (size_t)G * (2 + 2 * dt.nbmax));
    dt.bar = ctx->arena.get_t<GridBarrier>(t + "bar", 1);
    dt.err = ctx->arena.get_t<int>(t + "err", 1);
    CK(cudaMemsetAsync(dt.bar, 0, sizeof(GridBarrier), st));
    CK(cudaMemsetAsync(dt.err, 0, sizeof(int), st));
    dt.wait_limit = ctx->wait_limit;
    const char *prof_env = std::getenv("DVR3D_PROF");
    const bool prof = prof_env && prof_env[0] == '1';
    if (prof) {
        dt.prof = ctx->arena.get_t<long long>(t + "prof", 8);
        CK(cudaMemsetAsync(dt.prof, 0, 8 * sizeof(long long), st));
    }
    if (time_panels) {
        const int npan = (n + dt.nbmax - 1) / dt.nbmax + 1;
        if ((int)ctx->panel_ev.size() < 2 * npan) {
            const size_t old = ctx->panel_ev.size();
            ctx->panel_ev.resize(2 * npan);
            for (size_t q = old; q < ctx->panel_ev.size(); ++q) CK(cudaEventCreate(&ctx->panel_ev[q]));
        }
        dt.ev = ctx->panel_ev.data();
        dt.nev = (int)ctx->panel_ev.size();
    }
    {
        int gres = 0;
        const int slots = dense_resident_plan(ctx->device, n, &gres);
        if (slots > 0 && gres <= G) {
            dt.cache_tiles = slots;
            G = gres;
        }
    }
    CK(launch_dense_tridiag(dt, G, st));
    if (prof) {
        std::vector<long long> pc = download(ctx, dt.prof, 6);
        int khz = 0;
        cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, ctx->device);
        std::fprintf(stderr, "dense reduction N=%d grid=%d phase ms (at %d MHz):", n, G, khz / 1000);
        for (int q = 0; q < 6; ++q) std::fprintf(stderr, " %.2f", (double)pc[q] / (double)khz);
        std::fprintf(stderr, "\n");
    }
    double *e2s = ctx->arena.get_t<double>(t + "e2", n);
    double *info = ctx->arena.get_t<double>(t + "info", 4);
    launch_dense_eigvals(dt.d, dt.e, n, nev, e2s, info, w, st);
    CK(cudaGetLastError());
    if (vecs) {
        const int T = std::min(nev, 1024);
        const bool smem = invit_smem_bytes(n) <= (size_t)kInvitSmemMax;
        double *fac = smem ? nullptr : ctx->arena.get_t<double>(t + "fac", (size_t)5 * n * T);
        double *X = smem ? nullptr : ctx->arena.get_t<double>(t + "x", (size_t)n * nev);
        int *cs = ctx->arena.get_t<int>(t + "cs", nev + 1);
        int *ncl = ctx->arena.get_t<int>(t + "ncl", 1);
        double *bt = ctx->arena.get_t<double>(t + "bt", dense_bt_work_doubles(n, nev));
        launch_dense_eigvecs(A, lda, n, dt.d, dt.e, dt.tau, w, nev, info, cs, ncl, fac, T, X, Z, ldz, bt, st);
        CK(cudaGetLastError());
    }
    check_dev_err(ctx, dt.err, "dense tridiagonal reduction");
    if (out && time_panels) {
        out->npanel = dt.npanel;
        out->panel_ms = 0.0;
        for (int q = 0; q < dt.npanel && 2 * q + 1 < dt.nev; ++q) {
            float m = 0.f;
            CK(cudaEventElapsedTime(&m, ctx->panel_ev[2 * q], ctx->panel_ev[2 * q + 1]));
            out->panel_ms += m;
        }
    }
}

// ---------------------------------------------------------------- band eigensolver
bool band_lowest(dvr3d_ctx *ctx, double *A, long long lda, int n, int b, int nev, double *w, double *Z,
                 long long ldz, double drop_rel, double *dropped_rel) {
    cudaStream_t st = ctx->stream;
    if (b < 1 || b > kBandMaxBw || n < 3 || nev > n) return false;
    auto *mx = ctx->arena.get_t<unsigned long long>("bd_max", 2);
    CK(launch_band_prepare(A, lda, n, b, mx, st));
    unsigned long long hb[2] = {0, 0};
    CK(cudaMemcpyAsync(hb, mx, sizeof(hb), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    note_d2h(sizeof(hb));
    double dropped, inside;
    std::memcpy(&dropped, &hb[0], sizeof(double));
    std::memcpy(&inside, &hb[1], sizeof(double));
    const double rel = inside > 0.0 ? dropped / inside : (dropped > 0.0 ? 1.0 : 0.0);
    if (dropped_rel) *dropped_rel = rel;
    if (!(rel <= drop_rel)) return false;
    BandTri t{};
    t.A = A;
    t.lda = lda;
    t.n = n;
    t.b = b;
    t.d = ctx->arena.get_t<double>("bd_d", n);
    t.e = ctx->arena.get_t<double>("bd_e", n);
    t.vs = ctx->arena.get_t<double>("bd_vs", band_reflector_doubles(n, b));
    t.taus = ctx->arena.get_t<double>("bd_tau", band_tau_doubles(n, b));
    t.progress = ctx->arena.get_t<unsigned int>("bd_prog", n);
    t.err = ctx->arena.get_t<int>("bd_err", 1);
    t.wait_limit = ctx->wait_limit;
    CK(cudaMemsetAsync(t.err, 0, sizeof(int), st));
    CK(launch_band_chase(t, st));
    check_dev_err(ctx, t.err, "band reduction");
    double *e2s = ctx->arena.get_t<double>("bd_e2", n);
    double *info = ctx->arena.get_t<double>("bd_info", 4);
    launch_dense_eigvals(t.d, t.e, n, nev, e2s, info, w, st);
    CK(cudaGetLastError());
    const int T = std::min(nev, 1024);
    const bool smem = invit_smem_bytes(n) <= (size_t)kInvitSmemMax;
    double *fac = smem ? nullptr : ctx->arena.get_t<double>("bd_fac", (size_t)5 * n * T);
    double *X = smem ? nullptr : ctx->arena.get_t<double>("bd_x", (size_t)n * nev);
    int *cs = ctx->arena.get_t<int>("bd_cs", nev + 1);
    int *ncl = ctx->arena.get_t<int>("bd_ncl", 1);
    launch_tridiag_eigvecs(t.d, t.e, n, w, nev, info, cs, ncl, fac, T, X, Z, ldz, 1.0e-10, st);
    CK(cudaGetLastError());
    CK(launch_band_backtransform(t, Z, ldz, nev, st));
    return true;
}

// Lowest eigenpairs of the band matrix by bisection and inverse iteration on LDL^T factors
// (band_bisect.cu), with the same band check as band_lowest. Returns false (nothing usable)
// when the band check fails or a vector's inverse iteration does not grow.
bool band_lowest_bisect(dvr3d_ctx *ctx, double *A, long long lda, int n, int b, int nev, double *w, double *Z,
                        long long ldz, double drop_rel, double *dropped_rel) {
    cudaStream_t st = ctx->stream;
    if (b < 1 || b > kBandMaxBw || n < 3 || nev > n) return false;
    auto *mx = ctx->arena.get_t<unsigned long long>("bd_max", 2);
    CK(launch_band_prepare(A, lda, n, b, mx, st));
    double *bounds = ctx->arena.get_t<double>("bb_bounds", 4);
    CK(launch_band_bounds(A, lda, n, b, bounds, st));
    CK(launch_band_bisect(A, lda, n, b, nev, bounds, w, st));
    unsigned long long hb[2] = {0, 0};
    double hbd[3] = {0, 0, 0};
    std::vector<double> wh(nev);
    CK(cudaMemcpyAsync(hb, mx, sizeof(hb), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hbd, bounds, sizeof(hbd), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(wh.data(), w, sizeof(double) * nev, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    note_d2h(sizeof(hb) + sizeof(hbd) + sizeof(double) * nev);
    double dropped, inside;
    std::memcpy(&dropped, &hb[0], sizeof(double));
    std::memcpy(&inside, &hb[1], sizeof(double));
    const double rel = inside > 0.0 ? dropped / inside : (dropped > 0.0 ? 1.0 : 0.0);
    if (dropped_rel) *dropped_rel = rel;
    if (!(rel <= drop_rel)) return false;
    // clusters: eigenvalues closer than 1e-10 ||A|| share a warp (Gram-Schmidt inside)
    const double anorm = std::max(hbd[2], 1e-300);
    std::vector<int> cs{0};
    for (int j = 1; j < nev; ++j)
        if (wh[j] - wh[j - 1] > 1.0e-10 * anorm) cs.push_back(j);
    cs.push_back(nev);
    const int ncl = (int)cs.size() - 1;
    int *dcs = ctx->arena.get_t<int>("bb_cs", cs.size());
    CK(cudaMemcpyAsync(dcs, cs.data(), sizeof(int) * cs.size(), cudaMemcpyHostToDevice, st));
    note_h2d(sizeof(int) * cs.size());
    double *scr = ctx->arena.get_t<double>("bb_scr", band_bisect_scratch_doubles(n, b, ncl));
    int *err = ctx->arena.get_t<int>("bb_err", 1);
    CK(cudaMemsetAsync(err, 0, sizeof(int), st));
    CK(launch_band_invit(A, lda, n, b, w, dcs, ncl, bounds, scr, Z, ldz, 1.0 / (1.0e-8 * anorm), err, st));
    int he = 0;
    CK(cudaMemcpyAsync(&he, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return he == 0;
}

// ---------------------------------------------------------------- one k block
// ---------------------------------------------------------------- many Radau problems at once
// The 2D stage of independent Radau problems (the repeated DVR3DRJZ runs of a fitting
// driver) as one workload: the blocks of every problem are built into one buffer and go
// through ONE launch of each batched eigensolver phase (tridiagonalisation, eigenvalues,
// eigenvectors of the kept states), so the GPU works on the blocks of all problems together
// instead of on one problem's few dozen angles. All eigenvalues come back in one copy and
// each problem's selection (cut2dr / choosr, testiv) is made on the host. Per-problem
// buffers are named with the problem index so every contracted basis stays resident until
// its problem's assembly and final solve (solve_contracted).
void radau_stage_batch(dvr3d_ctx *ctx, const std::vector<BlockPlan> &plans, const std::vector<PesParams> &pes,
                       std::vector<Contracted> &outs) {
    cudaStream_t st = ctx->stream;
    const int np = (int)plans.size();
    outs.assign(np, Contracted{});
    std::vector<int> nb_n, first(np + 1, 0);  // per block: dimension; first block of each problem
    std::vector<long long> aoff, voff;
    long long at = 0, vt = 0;
    int nmax = 0;
    for (int i = 0; i < np; ++i) {
        const BlockPlan &p = plans[i];
        const int n = p.npnt1 * (p.npnt1 + 1 - 2 * p.ipar) / 2;
        if (n > 1024) throw HostError{DVR3D_ERR_UNSUPPORTED, "Radau 2D block larger than 1024"};
        nmax = std::max(nmax, n);
        first[i] = (int)nb_n.size();
        for (int b = 0; b < p.nalf; ++b) {
            nb_n.push_back(n);
            aoff.push_back(at);
            voff.push_back(vt);
            at += (long long)n * n;
            vt += n;
        }
    }
    first[np] = (int)nb_n.size();
    const int nblk = (int)nb_n.size();
    double *H = ctx->arena.get_t<double>("bt_blk2", (size_t)at);
    std::vector<std::vector<int>> pa(np), pb(np);
    for (int i = 0; i < np; ++i) {
        const BlockPlan &p = plans[i];
        const int npnt = p.npnt1;
        for (int beta = 1; beta <= npnt; ++beta)
            for (int alpha = 1; alpha <= beta - p.ipar; ++alpha) {
                pa[i].push_back(alpha - 1);
                pb[i].push_back(beta - 1);
            }
        const std::string sfx = "_" + std::to_string(i);
        RadauBuild rb{};
        rb.n = (int)pa[i].size();
        rb.npnt = npnt;
        rb.ipar = p.ipar;
        rb.jrot = p.jrot;
        rb.kz = p.kz;
        rb.pa = upload(ctx, "bt_pa" + sfx, pa[i]);
        rb.pb = upload(ctx, "bt_pb" + sfx, pb[i]);
        rb.r = upload(ctx, "bt_r1" + sfx, p.r1);
        rb.hr = upload(ctx, "bt_xk1" + sfx, p.xk1);
        rb.xalf = upload(ctx, "bt_xalf" + sfx, p.xalf);
        rb.term = p.nf_term;
        rb.term2 = p.nf_term2;
        rb.term3 = p.nf_term3;
        rb.zperp = p.zperp ? 1 : 0;
        rb.urr1 = p.urr1;
        rb.xterm = p.zperp ? 0.0 : (double)(p.kz * p.kz) * (1.0 / p.ur1 - 1.0 / p.urr1) * p.xp0;
        rb.pes = pes[i];
        if (rb.pes.kind != DVR3D_PES_MORSE_SUM)
            throw HostError{DVR3D_ERR_ARG, "batched problems take DVR3D_PES_MORSE_SUM surfaces"};
        launch_radau_build(rb, p.nalf, H + aoff[first[i]], st);
        outs[i].T = upload(ctx, "bt_xl" + sfx, p.xlmatr);
        outs[i].ldt = p.idvr;
    }
    CK(cudaGetLastError());
    BatchDesc bd{nblk, upload(ctx, "bt_n", nb_n), upload(ctx, "bt_aoff", aoff), upload(ctx, "bt_voff", voff)};
    double *d = ctx->arena.get_t<double>("bt_d", (size_t)vt);
    double *e = ctx->arena.get_t<double>("bt_e", (size_t)vt);
    double *tau = ctx->arena.get_t<double>("bt_tau", (size_t)vt);
    double *w = ctx->arena.get_t<double>("bt_w", (size_t)vt);
    int *cnt = ctx->arena.get_t<int>("bt_cnt", nblk);
    launch_tridiag_batched(bd, H, d, e, tau, nmax, st);
    launch_eigvals_batched(bd, d, e, w, cnt, 0, 0.0, st);  // every eigenvalue: selection on the host
    CK(cudaGetLastError());
    const std::vector<double> all = download(ctx, w, (size_t)vt);
    std::vector<int> sel(nblk, 0);
    std::vector<long long> zoff(nblk, 0);
    std::vector<int> zld(nblk, 0);
    std::vector<long long> vtoff(np, 0);
    long long vtot = 0;
    for (int i = 0; i < np; ++i) {
        const BlockPlan &p = plans[i];
        const int n = nb_n[first[i]], nalf = p.nalf;
        const double *wi = all.data() + voff[first[i]];
        int *si = sel.data() + first[i];
        if (p.zcut) {  // cut2dr (:3323-3377)
            long long tot = 0;
            for (int b = 0; b < nalf; ++b) {
                int c = 0;
                while (c < n && wi[(size_t)b * n + c] < p.emax2_au) ++c;
                si[b] = c;
                tot += c;
                if (tot > p.max3d) throw HostError{DVR3D_ERR_CORE_MAX3D, "number of 2d eigenvalues greater than max3d"};
            }
        } else {  // choosr (:3223-3319)
            std::vector<double> srt(wi, wi + (size_t)nalf * n);
            std::sort(srt.begin(), srt.end());
            const double emax = ((long long)srt.size() <= p.max3d) ? srt.back() : srt[p.max3d - 1];
            for (int b = 0; b < nalf; ++b) {
                int c = 0;
                while (c < n && wi[(size_t)b * n + c] <= emax) ++c;
                si[b] = c;
            }
        }
        if (p.jrot > 0) {  // testiv (:3380-3451)
            int iend = nalf;
            for (int q = nalf / 2; q <= nalf; ++q)
                if (q >= 1 && si[q - 1] == 0) {
                    iend = q;
                    break;
                }
            for (int q = iend + 1; q <= nalf; ++q) si[q - 1] = 0;
            if (si[nalf - 1] > 0) {
                if (p.zlin) si[nalf - 1] = 0;
                else throw HostError{DVR3D_ERR_THETA0, "bisector embedding: wavefunction has amplitude for theta = 0"};
            }
        }
        Contracted &o = outs[i];
        o.iv2.assign(si, si + nalf);
        o.nblocks = nalf;
        o.N = std::accumulate(o.iv2.begin(), o.iv2.end(), 0);
        o.P = n;
        o.ldv = round_up(n, 16);
        vtoff[i] = vtot;
        long long col = 0;
        for (int b = 0; b < nalf; ++b) {
            zoff[first[i] + b] = vtot + col * o.ldv;
            zld[first[i] + b] = (int)o.ldv;
            col += si[b];
        }
        vtot += o.ldv * round_up(std::max(o.N, 1), 64);
    }
    double *Vpool = ctx->arena.get_t<double>("bt_vt", (size_t)vtot);
    CK(cudaMemsetAsync(Vpool, 0, sizeof(double) * vtot, st));
    launch_eigvecs_batched_fast(bd, H, d, e, tau, w, upload(ctx, "bt_sel", sel), upload(ctx, "bt_zoff", zoff),
                                upload(ctx, "bt_zld", zld), Vpool, nmax, ev_err(ctx), st);
    CK(cudaGetLastError());
    for (int i = 0; i < np; ++i) {
        const BlockPlan &p = plans[i];
        Contracted &o = outs[i];
        o.Vt = Vpool + vtoff[i];
        const std::string sfx = "_" + std::to_string(i);
        std::vector<double> sw(o.ldv, 0.0);
        for (int q = 0; q < o.P; ++q) {
            const double ra = p.r1[pa[i][q]], rbv = p.r1[pb[i][q]];
            sw[q] = std::sqrt(0.5 / (ra * ra * p.ur1) + 0.5 / (rbv * rbv * p.ur1));
        }
        if (o.N == 0) continue;
        launch_scale_rows(o.Vt, (int)o.ldv, o.N, upload(ctx, "bt_sw" + sfx, sw), st);
        o.sw.assign(sw.begin(), sw.begin() + o.P);
        std::vector<int> gcol(o.N);
        std::vector<long long> emap(o.N);
        long long col = 0;
        for (int b = 0; b < o.nblocks; ++b) {
            for (int j = 0; j < o.iv2[b]; ++j) {
                gcol[col + j] = b;
                emap[col + j] = voff[first[i] + b] + j;
            }
            col += o.iv2[b];
        }
        o.g = upload(ctx, "bt_gcol" + sfx, gcol);
        o.e2 = ctx->arena.get_t<double>("bt_e2" + sfx, o.N);
        launch_gather(w, upload(ctx, "bt_emap" + sfx, emap), o.e2, o.N, st);
    }
    CK(cudaGetLastError());
}

// The eigenvector error flag of a solve, for callers outside this file that run the stages
// themselves (batched problems): cleared before the stage, checked after it.
int *eigvec_err_flag(dvr3d_ctx *ctx) { return ev_err(ctx); }
void check_eigvec_err(dvr3d_ctx *ctx, const char *stage) { check_dev_err(ctx, ev_err(ctx), stage); }

// Everything after the 1D/2D stages of one block: selection outputs, assembly, the final
// eigensolve (plain, Davidson or shift-invert), levels, vectors, timings and counters.
// ev[0] / ev[1] of the context bracket the stage that produced C.
void solve_contracted(dvr3d_ctx *ctx, const BlockPlan &p, const Contracted &C, const dvr3d_options &opt,
                      dvr3d_result &res, WaveOut *wave, std::chrono::steady_clock::time_point th0,
                      std::chrono::steady_clock::time_point th1, long long launches0) {
    cudaStream_t st = ctx->stream;
    const int N = C.N;
    res.kz = p.kz;
    res.ipar = p.ipar;
    res.nham3 = N;
    res.nblocks = C.nblocks;
    res.iterations = 0;
    res.fallback = 0;
    res.path = DVR3D_PATH_DENSE;
    res.matvecs = 0;
    res.lp_pairs = 0;
    res.lp_loss_first = res.lp_loss_last = 0.0;
    ctx->lp_set.valid = false;  // recorded pairs refer to the buffers of the last solve only
    if (res.iv2 && res.iv2_cap >= C.nblocks)
        for (int b = 0; b < C.nblocks; ++b) res.iv2[b] = C.iv2[b];
    const int meval = std::min(opt.nlevels > 0 ? opt.nlevels : p.neval, N);
    res.meval = meval;
    if (N == 0) {
        res.max_resid = 0.0;
        return;
    }
    if (res.eval && res.eval_cap < meval) throw HostError{DVR3D_ERR_BUFFER, "eval buffer smaller than min(neval, N)"};
    const bool mixed = (opt.precision == DVR3D_PREC_MIXED_DAVIDSON);
    const bool split_form = (opt.precision == DVR3D_PREC_SPLIT_BF16);
    res.low_iterations = 0;
    res.low_matvecs = 0;
    auto finish_times = [&](double &ms1, double &ms2, double &ms3) {
        CK(cudaStreamSynchronize(st));
        float a = 0, b = 0, c = 0;
        CK(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]));
        CK(cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]));
        CK(cudaEventElapsedTime(&c, ctx->ev[2], ctx->ev[3]));
        ms1 = a;
        ms2 = b;
        ms3 = c;
        res.stage_ms[0] = std::chrono::duration<double, std::milli>(th1 - th0).count();
        res.stage_ms[1] = ms1;
        res.stage_ms[2] = ms2;
        res.stage_ms[3] = ms3;
        res.stage_ms[4] = ms1 + ms2 + ms3;
        res.stage_ms[5] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - th0).count();
    };
    auto put_levels = [&](const double *wv, const double *Z) {
        if (res.eval) {
            CK(cudaMemcpyAsync(res.eval, wv, sizeof(double) * meval, cudaMemcpyDeviceToHost, st));
            t_d2h += (long long)sizeof(double) * meval;
        }
        if (res.evec && Z) {
            if (res.evec_cap < (size_t)N * meval) throw HostError{DVR3D_ERR_BUFFER, "evec buffer too small"};
            CK(cudaMemcpyAsync(res.evec, Z, sizeof(double) * N * meval, cudaMemcpyDeviceToHost, st));
            t_d2h += (long long)sizeof(double) * N * meval;
        }
    };
    // ---- assembly (bloc3d / mkham3+loadh): FP64 DMMA, or BF16x3 on the tensor cores into the
    // split matrix of the split-BF16 form
    const long long ldh = (mixed || split_form) ? round_up(N, 8) : N;
    double *H3 = nullptr;
    auto assemble_fp64 = [&]() {
        H3 = ctx->arena.get_t<double>("h3", (size_t)ldh * N);
        AsmParams ap{};
        ap.Vt = C.Vt;
        ap.ldv = C.ldv;
        ap.n = N;
        ap.g = C.g;
        ap.T = C.T;
        ap.ldt = C.ldt;
        ap.e2 = C.e2;
        ap.H = H3;
        ap.ldh = ldh;
        launch_assemble_h3(ap, st);
        CK(cudaGetLastError());
    };
    H3Op op;
    int *tc_err = nullptr;
    if (split_form) {
        const long long ldk = round_up(C.P, 8);
        auto *vh = ctx->arena.get_t<__nv_bfloat16>("vt_hi", (size_t)ldk * N);
        auto *vl = ctx->arena.get_t<__nv_bfloat16>("vt_lo", (size_t)ldk * N);
        auto *hh = ctx->arena.get_t<__nv_bfloat16>("h3_hi", (size_t)ldh * N);
        auto *hl = ctx->arena.get_t<__nv_bfloat16>("h3_lo", (size_t)ldh * N);
        tc_err = ctx->arena.get_t<int>("tc_err", 1);
        CK(cudaMemsetAsync(tc_err, 0, sizeof(int), st));
        CK(launch_split_bf16(C.Vt, C.ldv, N, C.P, vh, vl, ldk, st));
        TcGemm g;
        g.M = N;
        g.N = N;
        g.K = C.P;
        g.nslice = 2;
        g.A_hi = g.B_hi = vh;
        g.A_lo = g.B_lo = vl;
        g.lda = g.ldb = ldk;
        g.epilogue = kTcAssemble;
        g.g = C.g;
        g.T = C.T;
        g.ldt = C.ldt;
        g.e2 = C.e2;
        g.H_hi = hh;
        g.H_lo = hl;
        g.ldh = ldh;
        g.err = tc_err;
        CK(launch_tc_gemm(g, st));
        op.hi = hh;
        op.lo = hl;
        op.ld = ldh;
        int herr = 0;
        CK(cudaMemcpyAsync(&herr, tc_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (herr != 0) throw HostError{DVR3D_ERR_NOCONV, "tensor-core assembly: a pipeline wait timed out"};
    } else {
        assemble_fp64();
        op.H3 = H3;
        op.ldh = ldh;
    }
    CK(cudaEventRecord(ctx->ev[2], st));
    if (opt.want_h3 && res.h3) {
        if (res.h3_cap < (size_t)N * N) throw HostError{DVR3D_ERR_BUFFER, "h3 buffer too small"};
        const double *src = H3;
        if (split_form) {  // the split matrix as the solver uses it: hi + lo
            double *hs = ctx->arena.get_t<double>("h3_sum", (size_t)ldh * N);
            CK(launch_split_sum(op.hi, op.lo, ldh, N, hs, st));
            src = hs;
        }
        CK(cudaMemcpy2DAsync(res.h3, (size_t)N * sizeof(double), src, (size_t)ldh * sizeof(double),
                             (size_t)N * sizeof(double), N, cudaMemcpyDeviceToHost, st));
        t_d2h += (long long)sizeof(double) * N * N;
    }
    if (opt.learned_precond == 1 && !ctx->lp_trained)
        throw HostError{DVR3D_ERR_ARG, "no trained preconditioner (train one with learned_precond = 2 or load weights)"};
    if ((mixed && meval <= kDavidsonMaxLevels) || split_form) {
        // ---- block-Davidson with the channel-block preconditioner (few levels in the mixed
        // form; any number in the split-BF16 form)
        double *wv = ctx->arena.get_t<double>("dt_w", meval);
        double *Z = (res.evec || wave) ? ctx->arena.get_t<double>("dv_z", (size_t)N * meval) : nullptr;
        double *lpw = ctx->arena.get_t<double>("lp_w", kLpParams);
        const int mode = opt.learned_precond == 2 ? 2 : (opt.learned_precond == 1 ? 1 : 0);
        std::vector<double> rn;
        DavidsonStats ds;
        const bool ok = davidson_solve(ctx, op, C, opt, meval, mode, lpw, wv, rn, Z, ds);
        check_dev_err(ctx, ev_err(ctx), "batched inverse iteration (channel blocks)");
        res.iterations = ds.iterations;
        res.matvecs = ds.matvecs;
        res.low_iterations = ds.low_iterations;
        res.low_matvecs = ds.low_matvecs;
        if (ds.trained) {
            ctx->lp_trained = true;
            res.lp_pairs = ds.pairs;
            res.lp_loss_first = ds.loss_first;
            res.lp_loss_last = ds.loss_last;
        }
        if (ok) {
            CK(cudaEventRecord(ctx->ev[3], st));
            put_levels(wv, Z);
            if (wave) compute_wavefunctions(ctx, p, C, Z, N, meval, *wave);
            if (res.resid)
                for (int j = 0; j < std::min(meval, res.resid_cap); ++j) res.resid[j] = rn[j];
            res.max_resid = ds.max_resid;
            res.path = DVR3D_PATH_DAVIDSON;
            double ms1, ms2, ms3;
            finish_times(ms1, ms2, ms3);
            // dominant work: the H3 V products (2 N^2 flop per vector), timed with the solve
            res.dom_ms = ms3;
            res.dom_bytes = 0.0;
            res.dom_flops = 2.0 * (double)N * N * ds.matvecs;
            res.dom_launches = 0;
            std::snprintf(res.dom_kernel, sizeof(res.dom_kernel), split_form ? "tc_gemm_kernel" : "gemm_pipe_kernel");
            res.launches = (int)(g_kernel_launches - launches0);
            res.h2d_bytes = t_h2d;
            res.d2h_bytes = t_d2h;
            return;
        }
        if (split_form) {
            res.fallback = 1;
            assemble_fp64();  // the dense FP64 fallback below works on the assembled FP64 matrix
        }
    }
    if (mixed) {
        // ---- shift-invert block Krylov for the lowest levels; dense FP64 fallback below
        std::vector<double> e2h = download(ctx, C.e2, N);
        const double emin = *std::min_element(e2h.begin(), e2h.end());
        double *wv = ctx->arena.get_t<double>("dt_w", meval);
        double *Z = (res.evec || wave) ? ctx->arena.get_t<double>("dv_z", (size_t)N * meval) : nullptr;
        std::vector<double> rn;
        KrylovStats ks;
        const bool ok = si_krylov_solve(ctx, H3, ldh, N, emin, opt, meval, wv, rn, Z, ks);
        if (ok) {
            res.path = DVR3D_PATH_SHIFT_INVERT;
            res.matvecs = ks.m;
            CK(cudaEventRecord(ctx->ev[3], st));
            put_levels(wv, Z);
            if (wave) compute_wavefunctions(ctx, p, C, Z, N, meval, *wave);
            if (res.resid)
                for (int j = 0; j < std::min(meval, res.resid_cap); ++j) res.resid[j] = rn[j];
            res.max_resid = ks.max_resid;
            res.iterations = ks.blocks;
            double ms1, ms2, ms3;
            finish_times(ms1, ms2, ms3);
            // dominant kernel family: the DMMA GEMM (Cholesky-inverse, Krylov steps, Ritz
            // vectors, H3 X): its launches' own event-timed durations and algorithmic flops
            // when they were logged (DVR3D_GEMM_EVENTS=1), else zero
            res.dom_ms = ks.gemm_ms;
            res.dom_bytes = 0.0;
            res.dom_flops = ks.gemm_ms > 0.0 ? ks.gemm_flops : 0.0;
            res.dom_launches = ks.gemm_launches;
            std::snprintf(res.dom_kernel, sizeof(res.dom_kernel), "gemm_pipe_kernel");
            res.launches = (int)(g_kernel_launches - launches0);
            res.h2d_bytes = t_h2d;
            res.d2h_bytes = t_d2h;
            return;
        }
        res.fallback = 1;
    }
    // ---- final eigensolve (diag3d), dense FP64
    const long long ldw = round_up(N, 8);
    double *Hw = ctx->arena.get_t<double>("h3w", (size_t)ldw * N);
    CK(cudaMemcpy2DAsync(Hw, ldw * sizeof(double), H3, (size_t)ldh * sizeof(double), (size_t)N * sizeof(double), N,
                         cudaMemcpyDeviceToDevice, st));
    double *wv = ctx->arena.get_t<double>("dt_w", meval);
    const bool vecs = opt.want_vectors || res.evec || res.resid || wave;
    double *Z = vecs ? ctx->arena.get_t<double>("dv_z", (size_t)N * meval) : nullptr;
    DenseOut dout;
    dense_lowest(ctx, Hw, ldw, N, meval, vecs, wv, Z, N, "dt_", true, &dout);
    CK(cudaEventRecord(ctx->ev[3], st));
    res.max_resid = -1.0;
    if (vecs && (res.resid || opt.want_vectors)) {
        double *R = ctx->arena.get_t<double>("dv_r", (size_t)N * meval);
        double *rn = ctx->arena.get_t<double>("dv_rn", meval);
        launch_dgemm(false, false, N, meval, N, 1.0, H3, ldh, Z, N, 0.0, R, N, st);
        resid_kernel<<<meval, 256, 0, st>>>(R, Z, wv, N, N, meval, rn);
        DVR3D_COUNT_LAUNCH(1);
        CK(cudaGetLastError());
        std::vector<double> rv = download(ctx, rn, meval);
        res.max_resid = 0.0;
        for (double v : rv) res.max_resid = std::max(res.max_resid, v);
        if (res.resid)
            for (int j = 0; j < std::min(meval, res.resid_cap); ++j) res.resid[j] = rv[j];
    }
    put_levels(wv, Z);
    if (wave) compute_wavefunctions(ctx, p, C, Z, N, meval, *wave);
    double ms1, ms2, ms3;
    finish_times(ms1, ms2, ms3);
    // dominant kernel: the panel kernel of the Householder reduction; its algorithmic
    // traffic is one read of the trailing lower triangle per column
    double bytes = 0.0;
    for (int k = 0; k + 2 < N; ++k) {
        const double m = (double)(N - k - 1);
        bytes += 8.0 * m * (m + 1.0) * 0.5;
    }
    res.dom_ms = dout.panel_ms;
    res.dom_bytes = bytes;
    res.dom_flops = 0.0;
    res.dom_launches = dout.npanel;
    std::snprintf(res.dom_kernel, sizeof(res.dom_kernel), "dense_panel_kernel");
    res.launches = (int)(g_kernel_launches - launches0);
    res.h2d_bytes = t_h2d;
    res.d2h_bytes = t_d2h;
}

void solve_block(dvr3d_ctx *ctx, const dvr3d_deck &deck, int kk, const dvr3d_options &opt,
                 dvr3d_result &res, WaveOut *wave) {
    auto th0 = std::chrono::steady_clock::now();
    if (ctx->pes.kind != DVR3D_PES_MORSE_SUM && ctx->pes.kind != DVR3D_PES_GRID)
        throw HostError{DVR3D_ERR_ARG, "no potential selected (dvr3d_b200_set_pes)"};
    BlockPlan p;
    plan_block(deck, kk, p);
    auto th1 = std::chrono::steady_clock::now();
    const long long launches0 = g_kernel_launches;
    t_h2d = 0;
    t_d2h = 0;
    res.dom_ms = res.dom_bytes = res.dom_flops = 0.0;
    res.dom_launches = 0;
    std::memset(res.dom_kernel, 0, sizeof(res.dom_kernel));
    cudaStream_t st = ctx->stream;
    CK(cudaMemsetAsync(ev_err(ctx), 0, sizeof(int), st));
    invit_fail_clear(st);
    CK(cudaEventRecord(ctx->ev[0], st));
    Contracted C;
    if (p.radau) radau_stage(ctx, p, C);
    else jacobi_stage(ctx, p, C);
    CK(cudaEventRecord(ctx->ev[1], st));
    check_dev_err(ctx, ev_err(ctx), ("batched inverse iteration (1D/2D eigenvectors, k = " + std::to_string(p.kz) + ")").c_str());
    solve_contracted(ctx, p, C, opt, res, wave, th0, th1, launches0);
}

}  // namespace dvr3d
