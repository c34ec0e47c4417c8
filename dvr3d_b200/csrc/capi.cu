// capi.cu -- extern "C" entry points declared in include/dvr3d_b200.h.
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dvr3d_b200.h"
#include "eig_batched.cuh"
#include "eig_dense.cuh"
#include "learned_precond.cuh"
#include "pipeline.cuh"
#include "rotlev.cuh"
#include "dipole.cuh"
#include "tc_gemm.cuh"
#include "ozaki.cuh"

#define CK(x)                                          \
    do {                                               \
        cudaError_t e_ = (x);                          \
        if (e_ != cudaSuccess) throw CudaFail{e_, #x}; \
    } while (0)

using dvr3d::CudaFail;
using dvr3d::HostError;

namespace {

int fail_ctx(dvr3d_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

template <class F>
int guarded(dvr3d_ctx *ctx, F &&f) {
    try {
        return f();
    } catch (HostError &e) {
        return fail_ctx(ctx, e.code, e.msg);
    } catch (CudaFail &e) {
        cudaGetLastError();
        return fail_ctx(ctx, DVR3D_ERR_CUDA, e.where + ": " + cudaGetErrorString(e.err));
    } catch (std::bad_alloc &) {
        return fail_ctx(ctx, DVR3D_ERR_NOMEM, "host allocation failed");
    }
}

void appendf(std::string &s, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    s += buf;
}

// Fortran Dw.d edit descriptor (0.ddddD+ee form) for the level tables of diag3d.
std::string fortran_d(double v, int w, int d) {
    char buf[64];
    if (v == 0.0) {
        snprintf(buf, sizeof(buf), "0.%0*dD+00", d, 0);
    } else {
        int ex = (int)std::floor(std::log10(std::fabs(v))) + 1;
        double mant = std::fabs(v) / std::pow(10.0, ex);
        // rounding may carry into the next decade
        double scale = std::pow(10.0, d);
        double rm = std::round(mant * scale);
        if (rm >= scale) {
            rm /= 10.0;
            ex += 1;
        }
        if (rm < scale / 10.0) {
            rm *= 10.0;
            ex -= 1;
        }
        snprintf(buf, sizeof(buf), "%s0.%0*.0fD%c%02d", v < 0 ? "-" : "", d, rm, ex < 0 ? '-' : '+', std::abs(ex));
    }
    std::string s(buf);
    if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
    return s;
}

void copy_out(const std::string &s, char *out, size_t cap, size_t *len) {
    if (len) *len = s.size() + 1;
    if (out && cap > 0) {
        const size_t n = std::min(cap - 1, s.size());
        std::memcpy(out, s.data(), n);
        out[n] = '\0';
    }
}

}  // namespace

extern "C" {

const char *dvr3d_b200_strerror(int code) {
    switch (code) {
    case DVR3D_OK: return "ok";
    case DVR3D_ERR_ARG: return "invalid argument or inconsistent input";
    case DVR3D_ERR_CORE_MAX2D: return "core exceeded: reduce cut-off emax1 (MAX2D)";
    case DVR3D_ERR_CORE_MAX3D: return "core exceeded: increase max3d or reduce emax2 (MAX3D)";
    case DVR3D_ERR_QUADRATURE: return "points & weights in error (quadrature self-check failed)";
    case DVR3D_ERR_NOCONV: return "eigensolver did not converge within its limits";
    case DVR3D_ERR_CUDA: return "CUDA runtime error";
    case DVR3D_ERR_NOMEM: return "out of memory";
    case DVR3D_ERR_UNSUPPORTED: return "option not supported on this path";
    case DVR3D_ERR_THETA0: return "bisector embedding: wavefunction has amplitude for theta = 0";
    case DVR3D_ERR_PES: return "potential returned a non-finite value";
    case DVR3D_ERR_DECK: return "job deck could not be parsed";
    case DVR3D_ERR_NO_DEVICE: return "no usable CUDA device";
    case DVR3D_ERR_BUFFER: return "caller buffer too small";
    case DVR3D_ERR_SCRATCH: return "request exceeds the 64 MiB fixed scratch of dvr3d_b200_diag_batched_noalloc";
    default: return "unknown error";
    }
}

const char *dvr3d_b200_last_error(const dvr3d_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int dvr3d_b200_init(int device, dvr3d_ctx **out) {
    if (!out) return DVR3D_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
        cudaGetLastError();
        return DVR3D_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
        cudaGetLastError();
        return DVR3D_ERR_NO_DEVICE;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return DVR3D_ERR_NO_DEVICE;
    }
    dvr3d_ctx *ctx = new dvr3d_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return DVR3D_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    for (auto &e : ctx->ev) cudaEventCreate(&e);
    ctx->dense_grid = dvr3d::dense_tridiag_grid(device);
    ctx->pes.kind = DVR3D_PES_NONE;
    *out = ctx;
    return DVR3D_OK;
}

void dvr3d_b200_destroy(dvr3d_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->arena.release_all();
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : ctx->panel_ev) cudaEventDestroy(e);
    for (auto &e : ctx->gemm_ev) cudaEventDestroy(e);
    for (auto &g : ctx->graphs)
        if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

int dvr3d_b200_set_stream(dvr3d_ctx *ctx, void *stream) {
    if (!ctx) return DVR3D_ERR_ARG;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return DVR3D_OK;
}

int dvr3d_b200_parse_deck(const char *text, dvr3d_deck *out) {
    if (!text || !out) return DVR3D_ERR_ARG;
    try {
        dvr3d::parse_deck(text, *out);
        return DVR3D_OK;
    } catch (HostError &e) {
        return e.code;
    }
}

int dvr3d_b200_set_pes(dvr3d_ctx *ctx, int kind, const double *params, int nparams) {
    if (!ctx) return DVR3D_ERR_ARG;
    if (kind == DVR3D_PES_MORSE_SUM) {
        if (!params || nparams < DVR3D_PES_MORSE_SUM_NPARAM) return fail_ctx(ctx, DVR3D_ERR_ARG, "MORSE_SUM needs 13 parameters");
        for (int i = 0; i < DVR3D_PES_MORSE_SUM_NPARAM; ++i) {
            if (!std::isfinite(params[i])) return fail_ctx(ctx, DVR3D_ERR_PES, "non-finite PES parameter");
            ctx->pes.p[i] = params[i];
        }
        ctx->pes.kind = kind;
        return DVR3D_OK;
    }
    if (kind == DVR3D_PES_GRID) {
        if (ctx->pes_grid.empty() && ctx->pes_grid_k.empty())
            return fail_ctx(ctx, DVR3D_ERR_ARG, "call dvr3d_b200_set_pes_grid first");
        ctx->pes.kind = kind;
        return DVR3D_OK;
    }
    return fail_ctx(ctx, DVR3D_ERR_ARG, "unknown PES kind");
}

int dvr3d_b200_set_pes_grid(dvr3d_ctx *ctx, const double *v, size_t n) {
    if (!ctx || !v || n == 0) return DVR3D_ERR_ARG;
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return fail_ctx(ctx, DVR3D_ERR_PES, "non-finite value in the PES table");
    ctx->pes_grid.assign(v, v + n);
    ctx->pes.kind = DVR3D_PES_GRID;
    return DVR3D_OK;
}

int dvr3d_b200_set_pes_grid_k(dvr3d_ctx *ctx, int kz, const double *v, size_t n) {
    if (!ctx || kz < 0 || (n > 0 && !v)) return DVR3D_ERR_ARG;
    if (n == 0) {
        ctx->pes_grid_k.erase(kz);
        return DVR3D_OK;
    }
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return fail_ctx(ctx, DVR3D_ERR_PES, "non-finite value in the PES table");
    ctx->pes_grid_k[kz].assign(v, v + n);
    ctx->pes.kind = DVR3D_PES_GRID;
    return DVR3D_OK;
}

int dvr3d_b200_grid(dvr3d_ctx *ctx, const dvr3d_deck *deck, int kz, double *r1, int n1cap, double *r2,
                    int n2cap, double *xalf, int nacap) {
    if (!deck) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        dvr3d::BlockPlan p;
        dvr3d::plan_block(*deck, kz, p);
        if ((r1 && n1cap < p.npnt1) || (r2 && n2cap < p.npnt2) || (xalf && nacap < (int)p.xalf.size()))
            return fail_ctx(ctx, DVR3D_ERR_BUFFER, "grid buffers too small");
        if (r1) std::memcpy(r1, p.r1.data(), sizeof(double) * p.npnt1);
        if (r2) std::memcpy(r2, p.r2.data(), sizeof(double) * p.r2.size());
        if (xalf) std::memcpy(xalf, p.xalf.data(), sizeof(double) * p.xalf.size());
        return DVR3D_OK;
    });
}

int dvr3d_b200_solve_block(dvr3d_ctx *ctx, const dvr3d_deck *deck, int kz, const dvr3d_options *opt,
                           dvr3d_result *res) {
    if (!ctx || !deck || !res) return DVR3D_ERR_ARG;
    dvr3d_options o{};
    if (opt) o = *opt;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        dvr3d::solve_block(ctx, *deck, kz, o, *res);
        return DVR3D_OK;
    });
}

int dvr3d_b200_solve_batch(dvr3d_ctx *ctx, const dvr3d_deck *decks, const double *pes_params, int nprob,
                           const dvr3d_options *opt, dvr3d_result *res) {
    if (!ctx || !decks || !pes_params || !res || nprob <= 0) return DVR3D_ERR_ARG;
    dvr3d_options o{};
    if (opt) o = *opt;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        const dvr3d::PesParams saved = ctx->pes;
        struct Restore {
            dvr3d_ctx *c;
            dvr3d::PesParams p;
            ~Restore() { c->pes = p; }
        } restore{ctx, saved};
        const auto th0 = std::chrono::steady_clock::now();
        std::vector<dvr3d::BlockPlan> plans(nprob);
        std::vector<dvr3d::PesParams> pes(nprob);
        bool radau = true;
        for (int i = 0; i < nprob; ++i) {
            int kd, ku;
            dvr3d::k_range(decks[i], kd, ku);
            dvr3d::plan_block(decks[i], kd, plans[i]);
            radau = radau && plans[i].radau;
            pes[i] = dvr3d::PesParams{};
            pes[i].kind = DVR3D_PES_MORSE_SUM;
            for (int k = 0; k < DVR3D_PES_MORSE_SUM_NPARAM; ++k)
                pes[i].p[k] = pes_params[(size_t)i * DVR3D_PES_MORSE_SUM_NPARAM + k];
        }
        if (!radau) {  // Jacobi problems: one pipeline each
            for (int i = 0; i < nprob; ++i) {
                ctx->pes = pes[i];
                int kd, ku;
                dvr3d::k_range(decks[i], kd, ku);
                dvr3d::solve_block(ctx, decks[i], kd, o, res[i]);
            }
            return DVR3D_OK;
        }
        // Radau problems: the 2D stages of all of them as one batched workload, then each
        // problem's assembly and final eigensolve on its own resident contracted basis
        const auto th1 = std::chrono::steady_clock::now();
        const long long launches0 = dvr3d::g_kernel_launches;
        cudaStream_t st = ctx->stream;
        if (cudaMemsetAsync(dvr3d::eigvec_err_flag(ctx), 0, sizeof(int), st) != cudaSuccess ||
            cudaEventRecord(ctx->ev[0], st) != cudaSuccess)
            throw CudaFail{cudaGetLastError(), "solve_batch"};
        std::vector<dvr3d::Contracted> cs;
        dvr3d::radau_stage_batch(ctx, plans, pes, cs);
        if (cudaEventRecord(ctx->ev[1], st) != cudaSuccess) throw CudaFail{cudaGetLastError(), "solve_batch"};
        dvr3d::check_eigvec_err(ctx, "batched inverse iteration (2D eigenvectors)");
        for (int i = 0; i < nprob; ++i) {
            res[i].dom_ms = res[i].dom_bytes = res[i].dom_flops = 0.0;
            res[i].dom_launches = 0;
            std::memset(res[i].dom_kernel, 0, sizeof(res[i].dom_kernel));
            dvr3d::solve_contracted(ctx, plans[i], cs[i], o, res[i], nullptr, th0, th1, launches0);
        }
        return DVR3D_OK;
    });
}

int dvr3d_b200_diag_batched(dvr3d_ctx *ctx, int nblk, const int *n_host, const long long *off_host,
                            const long long *woff_host, double *a_dev, double *w_dev, int vecs) {
    if (!ctx || nblk <= 0 || !n_host || !off_host || !woff_host || !a_dev || !w_dev) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        cudaStream_t st = ctx->stream;
        std::vector<int> n(n_host, n_host + nblk);
        std::vector<long long> aoff(off_host, off_host + nblk), voff(nblk);
        int nmax = 0;
        long long vt = 0;
        for (int b = 0; b < nblk; ++b) {
            if (n[b] < 1 || n[b] > 1024) return fail_ctx(ctx, DVR3D_ERR_ARG, "block dimension must be 1..1024");
            nmax = std::max(nmax, n[b]);
            voff[b] = vt;
            vt += n[b];
        }
        auto up = [&](const char *name, const auto &v) {
            using T = typename std::decay_t<decltype(v)>::value_type;
            T *p = ctx->arena.get_t<T>(name, v.size());
            cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
            return p;
        };
        dvr3d::BatchDesc bd{nblk, up("dg_n", n), up("dg_aoff", aoff), up("dg_voff", voff)};
        double *d = ctx->arena.get_t<double>("dg_d", vt), *e = ctx->arena.get_t<double>("dg_e", vt);
        double *tau = ctx->arena.get_t<double>("dg_tau", vt), *w = ctx->arena.get_t<double>("dg_w", vt);
        int *cnt = ctx->arena.get_t<int>("dg_cnt", nblk);
        // the reflectors overwrite a copy of the blocks; eigenvectors are written back to a
        std::vector<long long> asz(nblk);
        long long at = 0;
        for (int b = 0; b < nblk; ++b) {
            asz[b] = at;
            at += (long long)n[b] * n[b];
        }
        double *ac = ctx->arena.get_t<double>("dg_a", at);
        for (int b = 0; b < nblk; ++b)
            cudaMemcpyAsync(ac + asz[b], a_dev + aoff[b], sizeof(double) * n[b] * n[b], cudaMemcpyDeviceToDevice, st);
        // the reference reads the lower triangle only: mirror it into full storage
        std::vector<int> dummy;
        (void)dummy;
        dvr3d::BatchDesc bdc{nblk, bd.n, up("dg_asz", asz), bd.voff};
        dvr3d::launch_symmetrize_lower(bdc, ac, nmax, st);
        dvr3d::launch_tridiag_batched(bdc, ac, d, e, tau, nmax, st);
        dvr3d::launch_eigvals_batched(bdc, d, e, w, cnt, 0, 0.0, st);
        for (int b = 0; b < nblk; ++b)
            cudaMemcpyAsync(w_dev + woff_host[b], w + voff[b], sizeof(double) * n[b], cudaMemcpyDeviceToDevice, st);
        int *err = ctx->arena.get_t<int>("err", 1);
        int err_host = 0;
        if (vecs) {
            std::vector<int> zld(n);
            std::vector<long long> woff(nblk);
            long long wt = 0;
            for (int b = 0; b < nblk; ++b) {
                woff[b] = wt;
                wt += 5LL * n[b] * std::min(128, n[b]) + (long long)n[b] * n[b];
            }
            double *work = ctx->arena.get_t<double>("dg_work", wt);
            cudaMemsetAsync(err, 0, sizeof(int), st);
            dvr3d::launch_eigvecs_batched(bdc, ac, d, e, tau, w, bd.n, up("dg_zoff", aoff), up("dg_zld", n), a_dev,
                                          work, up("dg_woff", woff), nmax, err, st);
            cudaMemcpyAsync(&err_host, err, sizeof(int), cudaMemcpyDeviceToHost, st);
        }
        cudaError_t ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) throw CudaFail{ce, "diag_batched"};
        if (err_host != 0) return fail_ctx(ctx, DVR3D_ERR_NOCONV, "inverse iteration did not converge for some eigenvector");
        return DVR3D_OK;
    });
}

int dvr3d_b200_set_wait_limit(dvr3d_ctx *ctx, long long polls) {
    if (!ctx || polls < 0) return DVR3D_ERR_ARG;
    ctx->wait_limit = (unsigned long long)polls;
    return DVR3D_OK;
}

int dvr3d_b200_rotlev3b(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, double *levels, int cap,
                        int *nlev, char *out, size_t outcap, size_t *outlen) {
    if (!ctx || !deck_text || !wave_path || !nlev) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        std::vector<double> lv;
        std::string table;
        dvr3d::RotInfo info;
        dvr3d::rotlev3b_solve(ctx, deck_text, wave_path, lv, table, info);
        *nlev = (int)lv.size();
        if (levels) {
            if (cap < (int)lv.size()) return fail_ctx(ctx, DVR3D_ERR_BUFFER, "levels buffer smaller than neval");
            std::memcpy(levels, lv.data(), sizeof(double) * lv.size());
        }
        copy_out(table, out, outcap, outlen);
        return DVR3D_OK;
    });
}

int dvr3d_b200_rotlev3b_trans(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, const char *kvec_path,
                              double *levels, int cap, int *nlev, char *out, size_t outcap, size_t *outlen) {
    if (!ctx || !deck_text || !wave_path || !kvec_path || !kvec_path[0] || !nlev) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        std::vector<double> lv;
        std::string table;
        dvr3d::RotInfo info;
        dvr3d::rotlev3b_solve(ctx, deck_text, wave_path, lv, table, info, kvec_path);
        *nlev = (int)lv.size();
        if (levels) {
            if (cap < (int)lv.size()) return fail_ctx(ctx, DVR3D_ERR_BUFFER, "levels buffer smaller than neval");
            std::memcpy(levels, lv.data(), sizeof(double) * lv.size());
        }
        copy_out(table, out, outcap, outlen);
        return DVR3D_OK;
    });
}

int dvr3d_b200_rotlev3b_pair(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, const char *kvec_path,
                             const char *kvec2_path, double *levels_e, int cap_e, int *nlev_e, double *levels_f,
                             int cap_f, int *nlev_f, char *out, size_t outcap, size_t *outlen) {
    if (!ctx || !deck_text || !wave_path || !nlev_e || !nlev_f) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        std::vector<double> le, lf;
        std::string table;
        dvr3d::RotInfo info;
        dvr3d::rotlev3b_solve(ctx, deck_text, wave_path, le, table, info, kvec_path, &lf, kvec2_path);
        *nlev_e = (int)le.size();
        *nlev_f = (int)lf.size();
        if (levels_e) {
            if (cap_e < (int)le.size()) return fail_ctx(ctx, DVR3D_ERR_BUFFER, "e levels buffer smaller than neval");
            std::memcpy(levels_e, le.data(), sizeof(double) * le.size());
        }
        if (levels_f) {
            if (cap_f < (int)lf.size()) return fail_ctx(ctx, DVR3D_ERR_BUFFER, "f levels buffer smaller than neval2");
            std::memcpy(levels_f, lf.data(), sizeof(double) * lf.size());
        }
        copy_out(table, out, outcap, outlen);
        return DVR3D_OK;
    });
}

int dvr3d_b200_rotlev3(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, const char *kvec_path,
                       const char *kvec2_path, double *levels, int cap, int *nlev, double *levels_f, int cap_f,
                       int *nlev_f, char *out, size_t outcap, size_t *outlen) {
    if (!ctx || !deck_text || !wave_path || !nlev) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        std::vector<double> le, lf;
        std::string text;
        dvr3d::RotInfo info;
        dvr3d::rotlev3_solve(ctx, deck_text, wave_path, le, lf, text, info, kvec_path, kvec2_path);
        *nlev = (int)le.size();
        if (nlev_f) *nlev_f = (int)lf.size();
        if (levels) {
            if (cap < (int)le.size()) return fail_ctx(ctx, DVR3D_ERR_BUFFER, "levels buffer smaller than neval");
            std::memcpy(levels, le.data(), sizeof(double) * le.size());
        }
        if (levels_f && !lf.empty()) {
            if (cap_f < (int)lf.size()) return fail_ctx(ctx, DVR3D_ERR_BUFFER, "f levels buffer smaller than neval2");
            std::memcpy(levels_f, lf.data(), sizeof(double) * lf.size());
        }
        copy_out(text, out, outcap, outlen);
        return DVR3D_OK;
    });
}

int dvr3d_b200_dipole3(dvr3d_ctx *ctx, const char *deck_text, const char *ket_path, const char *bra_path,
                       dvr3d_dipd_fn dipd, dvr3d_dipsa_fn dipsa, void *user, const char *tra_path,
                       dvr3d_dipole_result *res, char *out, size_t outcap, size_t *outlen) {
    if (!ctx || !deck_text || !ket_path || !bra_path || !res || (!dipd == !dipsa)) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        std::string text;
        dvr3d::dipole3_run(ctx, deck_text, ket_path, bra_path, dipd, dipsa, user, tra_path, *res, text);
        copy_out(text, out, outcap, outlen);
        return DVR3D_OK;
    });
}

int dvr3d_b200_split_gemm(dvr3d_ctx *ctx, int m, int n, int k, const double *a, long long lda, const double *b,
                          long long ldb, int nslice, double *c, long long ldc) {
    if (!ctx || m < 0 || n < 0 || k < 1 || !a || !b || !c || lda < k || ldb < k || ldc < m ||
        (nslice != 1 && nslice != 2))
        return DVR3D_ERR_ARG;
    if (m == 0 || n == 0) return DVR3D_OK;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        cudaStream_t st = ctx->stream;
        const long long lds = (k + 7) / 8 * 8;
        double *da = ctx->arena.get_t<double>("sg_a", (size_t)m * k), *db = ctx->arena.get_t<double>("sg_b", (size_t)n * k);
        double *dc = ctx->arena.get_t<double>("sg_c", (size_t)m * n);
        auto *ah = ctx->arena.get_t<__nv_bfloat16>("sg_ah", (size_t)m * lds);
        auto *al = ctx->arena.get_t<__nv_bfloat16>("sg_al", (size_t)m * lds);
        auto *bh = ctx->arena.get_t<__nv_bfloat16>("sg_bh", (size_t)n * lds);
        auto *bl = ctx->arena.get_t<__nv_bfloat16>("sg_bl", (size_t)n * lds);
        int *err = ctx->arena.get_t<int>("sg_err", 1);
        CK(cudaMemcpy2DAsync(da, sizeof(double) * k, a, sizeof(double) * lda, sizeof(double) * k, m,
                             cudaMemcpyHostToDevice, st));
        CK(cudaMemcpy2DAsync(db, sizeof(double) * k, b, sizeof(double) * ldb, sizeof(double) * k, n,
                             cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(err, 0, sizeof(int), st));
        CK(dvr3d::launch_split_bf16(da, k, m, k, ah, al, lds, st));
        CK(dvr3d::launch_split_bf16(db, k, n, k, bh, bl, lds, st));
        dvr3d::TcGemm g;
        g.M = m;
        g.N = n;
        g.K = k;
        g.nslice = nslice;
        g.A_hi = ah;
        g.A_lo = al;
        g.lda = lds;
        g.B_hi = bh;
        g.B_lo = bl;
        g.ldb = lds;
        g.C = dc;
        g.cm = 1;
        g.cn = m;
        g.err = err;
        CK(dvr3d::launch_tc_gemm(g, st));
        int err_host = 0;
        CK(cudaMemcpyAsync(&err_host, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpy2DAsync(c, sizeof(double) * ldc, dc, sizeof(double) * m, sizeof(double) * m, n,
                             cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (err_host != 0) return fail_ctx(ctx, DVR3D_ERR_NOCONV, "tensor-core pipeline wait timed out");
        return DVR3D_OK;
    });
}

int dvr3d_b200_ozaki_gemm(dvr3d_ctx *ctx, int ta, int tb, int tri, int tri_b, int lower_out, int m, int n, int k,
                          double alpha, const double *a, long long lda, const double *b, long long ldb, double beta,
                          double *c, long long ldc, int nslice) {
    const long long arow = ta ? k : m, acol = ta ? m : k, brow = tb ? n : k, bcol = tb ? k : n;
    if (!ctx || m < 0 || n < 0 || k < 1 || !a || !b || !c || lda < arow || ldb < brow || ldc < m || (lda & 1) ||
        (ldb & 1) || tri < 0 || tri > 2 || tri_b < 0 || tri_b > 2 || (lower_out && m != n) ||
        (nslice != 0 && (nslice < dvr3d::kOzMinSlices || nslice > dvr3d::kOzMaxSlices)))
        return DVR3D_ERR_ARG;
    if (m == 0 || n == 0) return DVR3D_OK;
    dvr3d::GemmOp g;
    g.M = m;
    g.N = n;
    g.K = k;
    g.alpha = alpha;
    g.beta = beta;
    g.ta = ta != 0;
    g.tb = tb != 0;
    g.tri = tri;
    g.tri_b = tri_b;
    g.lower_out = lower_out != 0;
    g.lda = lda;
    g.ldb = ldb;
    g.ldc = ldc;
    if (nslice != 0) {
        g.A = a;  // host pointers stand in for the support check (shapes only)
        g.B = b;
        g.C = c;
        if (!dvr3d::ozaki_supported(g, nslice)) return DVR3D_ERR_ARG;
    }
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        cudaStream_t st = ctx->stream;
        double *da = ctx->arena.get_t<double>("oz_a", (size_t)lda * acol);
        double *db = ctx->arena.get_t<double>("oz_b", (size_t)ldb * bcol);
        double *dc = ctx->arena.get_t<double>("oz_c", (size_t)ldc * n);
        int *err = ctx->arena.get_t<int>("oz_err", 1);
        CK(cudaMemcpyAsync(da, a, sizeof(double) * lda * acol, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(db, b, sizeof(double) * ldb * bcol, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(dc, c, sizeof(double) * ldc * n, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(err, 0, sizeof(int), st));
        g.A = da;
        g.B = db;
        g.C = dc;
        if (nslice == 0) {
            g.splitk = 1;
            CK(dvr3d::launch_gemm(g, st));
        } else {
            // thin products with few row tiles split K into chunks, as the Krylov steps do
            const int kchunk = (n <= 32 && !lower_out && (m + 127) / 128 < 148) ? dvr3d::kOzKrylovChunk : 0;
            const size_t wb = dvr3d::ozaki_work_bytes(g, nslice, false, kchunk) + 1024;
            unsigned char *w = ctx->arena.get_t<unsigned char>("oz_w", wb);
            const uintptr_t mis = reinterpret_cast<uintptr_t>(w) & 1023u;
            if (mis) w += 1024 - mis;
            CK(dvr3d::launch_ozaki_gemm(g, nslice, w, wb - 1024, err, st, nullptr, kchunk));
        }
        int err_host = 0;
        CK(cudaMemcpyAsync(&err_host, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(c, dc, sizeof(double) * ldc * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (err_host != 0) return fail_ctx(ctx, DVR3D_ERR_NOCONV, "tensor-core pipeline wait timed out");
        return DVR3D_OK;
    });
}

namespace {

// Sequential unformatted Fortran records: each record's bytes framed by its length as a
// 4-byte little-endian count before and after (the sequential unformatted layout of gfortran
// and of ifort's default record type). Logicals are 4-byte integers, .TRUE. = -1 (ifort's
// default representation, read as true by ifort and gfortran alike).
struct FortranRecords {
    FILE *f = nullptr;
    std::vector<unsigned char> rec;
    void i4(int v) { put(&v, 4); }
    void l4(bool v) { i4(v ? -1 : 0); }
    void r8(double v) { put(&v, 8); }
    void r8s(const double *v, size_t n) { put(v, 8 * n); }
    void put(const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        rec.insert(rec.end(), c, c + n);
    }
    void end() {
        if (rec.size() > 0x7fffffffu) throw HostError{DVR3D_ERR_UNSUPPORTED, "wavefunction record above 2 GiB"};
        const unsigned int n = (unsigned int)rec.size();
        if (std::fwrite(&n, 4, 1, f) != 1 || (n && std::fwrite(rec.data(), 1, n, f) != n) ||
            std::fwrite(&n, 4, 1, f) != 1)
            throw HostError{DVR3D_ERR_ARG, "writing the wavefunction file failed"};
        rec.clear();
    }
};

struct FileCloser {
    FILE *f;
    ~FileCloser() {
        if (f) std::fclose(f);
    }
};

// Records of the wavefunction file that precede the k loop: setcon's header (:1176-1184)
// and ccmain's r**(-2) term or basis sizes plus the radial grids (:820-845).
void write_wave_header(FortranRecords &wr, const dvr3d_deck &d, int kd, int ku) {
    dvr3d::BlockPlan p0;
    dvr3d::plan_block(d, kd, p0);
    const bool radau = p0.radau;
    int nlim = 0;
    if (p0.zrot) nlim = p0.zembed ? p0.npnt2 : p0.npnt1;  // zquad2 = T on this path
    wr.i4(d.idia);
    wr.i4(p0.ipar);
    wr.i4(p0.idvr);
    wr.i4(p0.npnt1);
    wr.i4(radau ? p0.npnt1 : p0.npnt2);
    wr.i4(p0.jrot);
    wr.i4(p0.kmin);
    wr.i4(d.neval);
    wr.i4(nlim);
    wr.end();
    wr.l4(p0.zembed);
    wr.l4(true);  // zmors1
    wr.l4(true);  // zmors2 (Radau: zmors1 again)
    wr.r8s(d.xmass, 3);
    wr.r8(p0.g1);
    wr.r8(p0.g2);
    wr.l4(!p0.zrot);  // zncor
    wr.l4(true);      // zquad2
    wr.end();
    const double rad[6] = {d.re1, d.diss1, d.we1, radau ? d.re1 : d.re2, radau ? d.diss1 : d.diss2,
                           radau ? d.we1 : d.we2};
    wr.r8s(rad, 6);
    wr.end();
    if (ku > kd) {
        // (symmetric Radau: one radial grid, r2 = r1)
        if (p0.zembed && !radau)
            for (int i = 0; i < p0.npnt2; ++i) wr.r8(0.5 / (p0.r2[i] * p0.r2[i] * p0.urr2));
        else
            for (int i = 0; i < p0.npnt1; ++i) wr.r8(0.5 / (p0.r1[i] * p0.r1[i] * p0.urr1));
    } else {
        const int jdia = std::max(1, d.idia);
        int jstart = p0.kmin;
        if (jstart % jdia != p0.ipar) ++jstart;
        const int nang = (p0.maxleg - jstart) / jdia + 1;
        const int mbass = radau ? p0.idvr * p0.max2d : p0.idvr * p0.npnt1 * p0.npnt2;
        wr.i4(mbass);
        wr.i4(jstart);
        wr.i4(nang);
        wr.i4(mbass);
    }
    wr.end();
    wr.r8s(p0.r1.data(), p0.npnt1);
    wr.end();
    if (!radau) {
        wr.r8s(p0.r2.data(), p0.npnt2);
        wr.end();
    }
}

// Records of one k block: angular grid and polynomials (:972-976), for Radau testiv's
// selection (:3446-3448), then the levels and one amplitude record per level (trans
// :3733-3841, transr :3622-3641).
void write_wave_block(FortranRecords &wr, const dvr3d::BlockPlan &p, const dvr3d_result &r, const int *iv2,
                      const double *ev, const dvr3d::WaveOut &wave) {
    wr.r8s(p.xalf.data(), p.idvr);
    wr.end();
    wr.i4(p.kz);
    wr.i4(p.maxleg);
    wr.i4(p.nidvr);
    wr.i4(p.lincr);
    wr.end();
    wr.r8s(p.pleg_walf.data(), p.pleg_walf.size());
    wr.end();
    if (p.radau) {
        int iang = 0;
        for (int b = 0; b < r.nblocks; ++b) iang += (iv2[b] > 0);
        wr.i4(iang);
        wr.i4(iang * p.max2d);
        wr.end();
        for (int b = 0; b < r.nblocks; ++b) wr.i4(iv2[b]);
        wr.end();
    }
    wr.i4(r.meval);
    wr.end();
    wr.r8s(ev, r.meval);
    wr.end();
    for (int l = 0; l < wave.nlev; ++l) {
        wr.r8s(wave.psi.data() + (size_t)l * wave.len, (size_t)wave.len);
        wr.end();
    }
}

}  // namespace

static int run_deck_impl(dvr3d_ctx *ctx, const char *deck_text, const dvr3d_options *opt, char *out, size_t outcap,
                         size_t *outlen, char *lev, size_t levcap, size_t *levlen, const char *wave_path) {
    if (!ctx || !deck_text) return DVR3D_ERR_ARG;
    dvr3d_options o{};
    if (opt) o = *opt;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        dvr3d_deck d;
        dvr3d::parse_deck(deck_text, d);
        int kd, ku;
        dvr3d::k_range(d, kd, ku);
        const double autocm = 2.19474624e+05;
        std::string s, lv;
        // the wavefunction file (unit IWAVE): written when the deck sets ZTRAN and a path is given
        const bool ztran = d.ztran && wave_path && wave_path[0];
        FortranRecords wr;
        FileCloser closer{nullptr};
        if (ztran) {
            closer.f = std::fopen(wave_path, "wb");
            if (!closer.f) throw HostError{DVR3D_ERR_ARG, std::string("cannot open ") + wave_path};
            wr.f = closer.f;
            write_wave_header(wr, d, kd, ku);
        }
        appendf(s, "     Program DVR3DRJZ (B200 hot path)\n\n     Title: %s\n", d.title);
        for (int kk = kd; kk <= ku; ++kk) {
            dvr3d::BlockPlan p;
            dvr3d::plan_block(d, kk, p);
            std::vector<double> ev(std::max(p.neval, 1));
            std::vector<int> iv2(std::max(p.radau ? p.nalf : p.npntc, 1));
            dvr3d_result r{};
            r.eval = ev.data();
            r.eval_cap = (int)ev.size();
            r.iv2 = iv2.data();
            r.iv2_cap = (int)iv2.size();
            dvr3d::WaveOut wave;
            dvr3d::solve_block(ctx, d, kk, o, r, ztran ? &wave : nullptr);
            if (ztran) write_wave_block(wr, p, r, iv2.data(), ev.data(), wave);
            if (d.jrot != 0 && p.zrot) appendf(s, "\n     Solutions with J =%3d k =%3d\n", p.jrot, p.kz);
            if (p.radau && d.jrot != 0 && p.zrot)
                appendf(s, p.ipar == 0 ? "\n     even parity solutions\n" : "\n     odd parity solutions\n");
            for (int b = 0; b < r.nblocks && p.radau; ++b)
                appendf(s, "     for gamma = %2d selected %3d energies.\n", b + 1, iv2[b]);
            appendf(s, "                         total = %5d\n", r.nham3);
            const int meval = r.meval;
            if (!d.zpmin) {
                appendf(s, "\n     lowest%4d eigenvalues in hartrees:\n\n", meval);
                for (int i = 0; i < meval; ++i) {
                    s += fortran_d(ev[i], 24, 12);
                    if (i % 5 == 4 || i == meval - 1) s += "\n\n";
                }
            }
            appendf(s, "\n\n     Lowest%4d eigenvalues in wavenumbers:\n\n", meval);
            for (int i = 0; i < meval; ++i) {
                s += fortran_d(ev[i] * autocm, 24, 12);
                if (i % 5 == 4 || i == meval - 1) s += "\n\n";
            }
            // zpfun levels file (:2708-2719): header 6i4, then 4d20.12
            const int ip = d.jrot - p.kmin;
            if (d.zpfun && (d.jrot == 0 || ip == 1)) {
                const int jdia = std::max(0, d.idia), jpar = std::min(jdia, p.ipar);
                int isym = std::abs(std::min(0, d.idia));
                if (p.ipar == 1) isym = -isym;
                appendf(lv, "%4d%4d%4d%4d%4d%4d\n", d.jrot, ip, jdia, jpar, isym, meval);
                for (int i = 0; i < meval; ++i) {
                    lv += fortran_d(ev[i], 20, 12);
                    if (i % 4 == 3 || i == meval - 1) lv += "\n";
                }
            }
            if (d.jrot == 0 && meval > 0) {  // band origins (:2748-2761)
                double ezero;
                int ii;
                if (std::abs(d.idia) == 2 && p.ipar == 1) {
                    ezero = d.have_ezero ? d.ezero : 0.0;
                    ii = 0;
                } else {
                    ezero = ev[0] * autocm;
                    ii = 1;
                }
                appendf(s, "\n  Band origins in wavenumbers:\n\n");
                int c = 0;
                for (int i = ii; i < meval; ++i, ++c) {
                    appendf(s, "%15.6f", ev[i] * autocm - ezero);
                    if (c % 5 == 4 || i == meval - 1) s += "\n\n";
                }
            }
        }
        copy_out(s, out, outcap, outlen);
        copy_out(lv, lev, levcap, levlen);
        return DVR3D_OK;
    });
}

int dvr3d_b200_run_deck(dvr3d_ctx *ctx, const char *deck_text, const dvr3d_options *opt, char *out, size_t outcap,
                        size_t *outlen, char *lev, size_t levcap, size_t *levlen) {
    return run_deck_impl(ctx, deck_text, opt, out, outcap, outlen, lev, levcap, levlen, nullptr);
}

int dvr3d_b200_run_deck_wave(dvr3d_ctx *ctx, const char *deck_text, const dvr3d_options *opt, char *out,
                             size_t outcap, size_t *outlen, char *lev, size_t levcap, size_t *levlen,
                             const char *wave_path) {
    if (!wave_path) return DVR3D_ERR_ARG;
    return run_deck_impl(ctx, deck_text, opt, out, outcap, outlen, lev, levcap, levlen, wave_path);
}

int dvr3d_b200_lp_get_weights(dvr3d_ctx *ctx, double *w, int n) {
    if (!ctx || !w) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        if (!ctx->lp_trained) throw HostError{DVR3D_ERR_ARG, "no trained preconditioner in this context"};
        if (n < dvr3d::kLpParams) throw HostError{DVR3D_ERR_BUFFER, "weight buffer smaller than DVR3D_LP_NPARAM"};
        cudaSetDevice(ctx->device);
        const double *d = ctx->arena.get_t<double>("lp_w", dvr3d::kLpParams);
        cudaError_t e = cudaMemcpyAsync(w, d, sizeof(double) * dvr3d::kLpParams, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) throw CudaFail{e, "lp_get_weights"};
        return dvr3d::kLpParams;
    });
}

int dvr3d_b200_lp_set_weights(dvr3d_ctx *ctx, const double *w, int n) {
    if (!ctx || !w) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        if (n != dvr3d::kLpParams) throw HostError{DVR3D_ERR_ARG, "expected DVR3D_LP_NPARAM parameters"};
        for (int p = 0; p < n; ++p)
            if (!std::isfinite(w[p])) throw HostError{DVR3D_ERR_ARG, "non-finite preconditioner parameter"};
        cudaSetDevice(ctx->device);
        double *d = ctx->arena.get_t<double>("lp_w", dvr3d::kLpParams);
        cudaError_t e = cudaMemcpyAsync(d, w, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) throw CudaFail{e, "lp_set_weights"};
        ctx->lp_trained = true;
        return DVR3D_OK;
    });
}

int dvr3d_b200_lp_eval(dvr3d_ctx *ctx, const double *w, int nmode, int ncol, const double *lam,
                       const double *f1, const double *f2, const double *f3, double scale,
                       const double *theta, const double *delta, double *gout, double *grad) {
    if (!ctx || !w || !lam || !f1 || !f2 || !f3 || !theta || !delta || !gout || !grad || nmode <= 0 || ncol <= 0 ||
        !(scale > 0.0))
        return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        cudaStream_t st = ctx->stream;
        auto up = [&](const char *nm, const double *src, size_t cnt) {
            double *d = ctx->arena.get_t<double>(nm, cnt);
            const cudaError_t e = cudaMemcpyAsync(d, src, sizeof(double) * cnt, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) throw CudaFail{e, "lp_eval upload"};
            return d;
        };
        dvr3d::LpModes m;
        m.lam = up("lpe_lam", lam, nmode);
        m.f1 = up("lpe_f1", f1, nmode);
        m.f2 = up("lpe_f2", f2, nmode);
        m.f3 = up("lpe_f3", f3, nmode);
        m.n = nmode;
        m.scale = scale;
        const double *dth = up("lpe_th", theta, ncol);
        const double *dd = up("lpe_delta", delta, (size_t)nmode * ncol);
        const double *dw = up("lpe_w", w, dvr3d::kLpParams);
        double *dg = ctx->arena.get_t<double>("lpe_g", (size_t)nmode * ncol);
        double *dgr = ctx->arena.get_t<double>("lpe_grad", dvr3d::kLpParams);
        double *work = ctx->arena.get_t<double>("lpe_work", dvr3d::lp_grad_work_doubles());
        cudaError_t e = dvr3d::launch_lp_forward(m, dw, dth, ncol, dg, st);
        if (e == cudaSuccess) e = dvr3d::lp_mlp_grad(m, dw, dth, ncol, dd, dgr, work, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(gout, dg, sizeof(double) * nmode * ncol, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(grad, dgr, sizeof(double) * dvr3d::kLpParams, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) throw CudaFail{e, "lp_eval"};
        return DVR3D_OK;
    });
}

int dvr3d_b200_lp_train_loss(dvr3d_ctx *ctx, const double *w, double *loss, double *grad) {
    if (!ctx || !w || !loss) return DVR3D_ERR_ARG;
    return guarded(ctx, [&]() -> int {
        cudaSetDevice(ctx->device);
        cudaStream_t st = ctx->stream;
        double *dw = ctx->arena.get_t<double>("lpt_w", dvr3d::kLpParams);
        double *dg = ctx->arena.get_t<double>("lpt_g", dvr3d::kLpParams);
        cudaError_t e = cudaMemcpyAsync(dw, w, sizeof(double) * dvr3d::kLpParams, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) throw CudaFail{e, "lp_train_loss upload"};
        *loss = dvr3d::lp_train_loss(ctx, dw, grad ? dg : nullptr);
        if (grad) {
            e = cudaMemcpyAsync(grad, dg, sizeof(double) * dvr3d::kLpParams, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) throw CudaFail{e, "lp_train_loss"};
        }
        return DVR3D_OK;
    });
}

}  // extern "C"
