/*
 * dvr3d_b200.h -- C ABI of the B200-native DVR3DRJZ hot path.
 *
 * The library replaces, for one GPU, the numerical core of the DVR3DRJZ program of the
 * DVR3D suite (reference file source/dvr3drjz_segmented.f90):
 *
 *   radial / angular DVR set-up  ->  per-angle 2D (or 1D+2D) block builds and FP64
 *   eigensolves with energy-cut-off truncation  ->  contracted 3D Hamiltonian assembly
 *   ->  final eigensolve for the lowest levels.
 *
 * Conventions (they follow the Fortran reference so a Fortran/ISO_C_BINDING or ctypes
 * host can bind the entry points directly):
 *   - plain C types and pointers only; every array is caller-owned host memory unless
 *     stated; matrices are column-major FP64 (Fortran order);
 *   - energies are in hartree (Eh) unless the name says _cm (wavenumbers);
 *   - every entry point returns 0 on success or a negative DVR3D_ERR_* code; the library
 *     never calls exit() or stop (the reference's STOP conditions become error codes);
 *   - one dvr3d_ctx per host thread; the library owns all device memory in the ctx.
 */
#ifndef DVR3D_B200_H
#define DVR3D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DVR3D_B200_ABI_VERSION 1

/* ---- error codes ------------------------------------------------------------------ */
enum dvr3d_status {
    DVR3D_OK = 0,
    DVR3D_ERR_ARG = -1,          /* invalid argument or inconsistent input cards          */
    DVR3D_ERR_CORE_MAX2D = -2,   /* cut1d: "core exceeded: reduce cut-off emax1"  (:2925) */
    DVR3D_ERR_CORE_MAX3D = -3,   /* cut2d/cut2dr: "core exceeded ... emax2" (:2981,:3359) */
    DVR3D_ERR_QUADRATURE = -4,   /* lagpt/jacobi: "points & weights in error" (:1360,:939) */
    DVR3D_ERR_NOCONV = -5,       /* an eigensolver did not converge within its limits     */
    DVR3D_ERR_CUDA = -6,         /* CUDA runtime error (message via strerror of the ctx)  */
    DVR3D_ERR_NOMEM = -7,        /* device allocation failed                              */
    DVR3D_ERR_UNSUPPORTED = -8,  /* option of the reference not implemented on this path */
    DVR3D_ERR_THETA0 = -9,       /* testiv: wavefunction amplitude at theta = 0 (:3430)  */
    DVR3D_ERR_PES = -10,         /* potential returned a non-finite value                 */
    DVR3D_ERR_DECK = -11,        /* job deck could not be parsed                          */
    DVR3D_ERR_NO_DEVICE = -12,   /* no CUDA device / extension not usable                 */
    DVR3D_ERR_BUFFER = -13,      /* caller buffer too small                               */
    DVR3D_ERR_SCRATCH = -14      /* request larger than the fixed scratch of the
                                    allocation-free entry point                          */
};

typedef struct dvr3d_ctx dvr3d_ctx;

/* ---- job deck: the reference's stdin input (namelist PRT + fixed-format cards) -------- */
/* Field meaning, defaults and card order follow block data (:83-168), insize (:171-638)
 * and setcon (:1016-1188). Logical flags are 0/1. */
typedef struct dvr3d_deck {
    /* Line 1: namelist /PRT/ */
    int zpham, zprad, zp1d, zp2d, zpmin, zpvec, zlmat, zcut, zrot, zperp, zembed, zlin;
    int zmors1, zmors2, zladd, ztwod, zvec, zall, ztheta, zr2r1, ztran, zquad2, zdiag;
    int zpfun, zx, zs0, zs1;
    /* Line 2 */
    int ncoord;
    /* Line 3: NPNT2,JROT,NEVAL,NALF,MAX2D,MAX3D,IDIA,KMIN,NPNT1,IPAR,MAX3D2 (11I5) */
    int npnt2, jrot, neval, nalf, max2d, max3d, idia, kmin, npnt1, ipar, max3d2;
    /* Line 4 */
    char title[80];
    /* Lines 5-10 (F20.0 fields) */
    double fixcos;
    double xmass[3], xmassr[3];
    double emax1, emax2;                 /* cm-1 */
    double re1, diss1, we1, re2, diss2, we2;
    /* optional trailing card read by diag3d for odd-parity band origins (:2751) */
    double ezero;
    int have_ezero;
} dvr3d_deck;

/* ---- potential energy surface ------------------------------------------------------ */
/* The reference's plugin is SUBROUTINE POTV(V,R1,R2,XCOS) (docum.tex:30-47; called from
 * mkham1 :2178-2183 and blc2d1 :3199,:3204). A host callback cannot run on the GPU, so a
 * potential is either one of the device-built families below, or a table of V that the
 * host evaluated with its own POTV at the DVR grid returned by dvr3d_b200_grid(). */
typedef enum dvr3d_pes_kind {
    DVR3D_PES_NONE = 0,
    /* V = D1 (1-exp(-a1 (r1-re1)))^2 + D2 (1-exp(-a2 (r2-re2)))^2
     *   + kb (cos t - c0)^2 + c12 (r1-re1)(r2-re2) + sum_{l=1..4} cl P_l(cos t)
     * params[13] = {D1, a1, re1, D2, a2, re2, kb, c0, c12, c1, c2, c3, c4} (Eh, bohr) */
    DVR3D_PES_MORSE_SUM = 1,
    /* V tabulated on the grid: v[(ic*npnt2 + i2)*npnt1 + i1] = V(r1[i1], r2[i2], xalf[ic]);
     * for Radau (idia=-2) r2 == r1. Set with dvr3d_b200_set_pes_grid(). */
    DVR3D_PES_GRID = 2
} dvr3d_pes_kind;

#define DVR3D_PES_MORSE_SUM_NPARAM 13

/* ---- solve options and results ------------------------------------------------------- */
typedef enum dvr3d_precision {
    DVR3D_PREC_FP64 = 0,             /* plain FP64 GPU path: dense FP64 final eigensolve  */
    DVR3D_PREC_MIXED_DAVIDSON = 1,   /* iterative lowest-level solve on the FP64 tensor
                                        cores: block-Davidson (<= 32 levels; channel-block
                                        preconditioner, optionally with the learned
                                        correction) or shift-invert block Krylov; FP64
                                        Rayleigh-Ritz and residual judge; dense FP64
                                        fallback                                          */
    DVR3D_PREC_SPLIT_BF16 = 2        /* split-BF16 form: assembly and H3 V as BF16x3
                                        products on the BF16 tensor cores (tcgen05, FP32
                                        accumulation), block-Davidson for any number of
                                        levels with FP64 Rayleigh-Ritz and residual norms;
                                        once the BF16x3 residuals stop falling, the FP64
                                        residual correction (products of the basis with
                                        the matrix-free FP64 operator) until the FP64
                                        residual test holds; dense FP64 fallback           */
} dvr3d_precision;

typedef enum dvr3d_path {
    DVR3D_PATH_DENSE = 0,            /* dense FP64 reduction (plain path or fallback)     */
    DVR3D_PATH_SHIFT_INVERT = 1,     /* shift-invert block Krylov                         */
    DVR3D_PATH_DAVIDSON = 2          /* block-Davidson                                    */
} dvr3d_path;

/* Number of parameters of the learned preconditioner correction (4 -> 16 -> 16 -> 1 MLP). */
#define DVR3D_LP_NPARAM 369

typedef struct dvr3d_options {
    int precision;          /* dvr3d_precision                                              */
    int nlevels;            /* levels wanted (0: NEVAL of the deck)                         */
    double tol_cm;          /* Davidson: max eigenvalue error target in cm-1 (0: 1e-4)      */
    int max_iter;           /* Davidson iteration limit (0: 200)                            */
    int block;              /* Davidson block size (0: automatic)                           */
    int learned_precond;    /* Davidson (<= 32 levels, channel-block preconditioner):
                               0 exact channel blocks; 1 with the trained correction of this
                               context; 2 train the correction on this solve (recorded
                               residual / ideal-correction pairs) and keep it in the context */
    int want_vectors;       /* 1: return eigenvectors of the final Hamiltonian in evec      */
    int want_h3;            /* 1: copy the assembled final Hamiltonian (lower) into h3      */
} dvr3d_options;

typedef struct dvr3d_result {
    /* outputs */
    int kz, ipar;           /* k block and parity solved                                    */
    int nham3;              /* dimension of the final contracted Hamiltonian                */
    int meval;              /* levels written to eval (min(neval, nham3))                   */
    int nblocks;            /* number of angular (Radau) / last-coordinate (Jacobi) blocks  */
    int iterations;         /* Davidson iterations (0 on the dense path)                    */
    int fallback;           /* 1 if the Davidson path fell back to the dense FP64 solve     */
    double stage_ms[6];     /* device time: 0 set-up, 1 block builds+eigensolves+selection,
                               2 assembly, 3 final eigensolve, 4 total, 5 host set-up       */
    double max_resid;       /* max FP64 residual ||H x - e x|| over returned levels (Eh)    */
    /* measurement counters of this solve (CUDA events on the context's stream) */
    double dom_ms;          /* device time of the dominant kernel's launches                */
    double dom_bytes;       /* algorithmic bytes those launches must move (or flops, below) */
    double dom_flops;       /* algorithmic flops of those launches (0 if bandwidth-bound)   */
    int dom_launches;       /* number of launches of the dominant kernel                    */
    int launches;           /* kernels launched by the library for this solve               */
    long long h2d_bytes;    /* host -> device bytes copied by this solve                    */
    long long d2h_bytes;    /* device -> host bytes copied by this solve                    */
    char dom_kernel[48];    /* name of the dominant kernel                                  */
    /* caller-provided buffers (may be NULL / 0) */
    double *eval;   int eval_cap;     /* levels (Eh), ascending                               */
    int *iv2;       int iv2_cap;      /* per-block selection counts (blocks in solve order)   */
    double *resid;  int resid_cap;    /* per-level FP64 residual norms (Eh)                   */
    double *evec;   size_t evec_cap;  /* nham3 x meval, column-major                          */
    double *h3;     size_t h3_cap;    /* nham3 x nham3, column-major, lower triangle valid    */
    /* solver path and iterative-solver counters (appended; outputs) */
    int path;               /* dvr3d_path: which eigensolver produced the levels            */
    int matvecs;            /* Davidson: H3 products (vectors); shift-invert: Krylov size   */
    int lp_pairs;           /* training pairs recorded when learned_precond = 2              */
    double lp_loss_first;   /* learned preconditioner loss before / after training          */
    double lp_loss_last;
    int low_iterations;     /* split-BF16 form: Davidson iterations on tensor-core products */
    int low_matvecs;        /* split-BF16 form: vectors multiplied on the BF16 tensor cores */
} dvr3d_result;

/* ---- entry points ----------------------------------------------------------------- */

/* Create a context on CUDA device `device`. Fails with DVR3D_ERR_NO_DEVICE when no
 * usable sm_100 device is present (no CPU fallback exists). */
int dvr3d_b200_init(int device, dvr3d_ctx **out);
void dvr3d_b200_destroy(dvr3d_ctx *ctx);
const char *dvr3d_b200_strerror(int code);
/* Last detailed error message of this context (CUDA error text, offending sizes). */
const char *dvr3d_b200_last_error(const dvr3d_ctx *ctx);
/* Use `stream` (a cudaStream_t) for all work of this context; NULL = the ctx's own. */
int dvr3d_b200_set_stream(dvr3d_ctx *ctx, void *stream);

/* Every device-side wait of the library is bounded: the grid barriers of the cooperative
 * dense reduction (default 2^26 polls) and the hand-off waits of the band reduction's bulge
 * chase (default 2^24 polls). A wait that runs out raises the kernel's error flag, every CTA
 * leaves its kernel, and the solve returns DVR3D_ERR_NOCONV with the context still usable.
 * This sets the poll limit of every such wait of later solves on the context (0 restores the
 * defaults); a small limit lets a caller check that the waits end. No counterpart in the
 * reference (which has no device waits). */
int dvr3d_b200_set_wait_limit(dvr3d_ctx *ctx, long long polls);

/* The second variational step for J > 0, symmetrised Radau coordinates with the bisector
 * embedding: the reference's program ROTLEV3B (source/rotlev3b_segmented.f90). deck_text is
 * ROTLEV3B's stdin (namelist PRT, card NVIB,NEVAL,KMIN,IBASS,NEVAL2,NPNT (12i5, insize
 * :157-161), title, optional EZERO card, vrmain :593-596); wave_path the first step's
 * wavefunction file (unit IVEC = 26) as dvr3d_b200_run_deck_wave writes it for k = kmin..J
 * (ZROT, ZTRAN). The Coriolis-coupled Hamiltonian (select :306-510, solrt :1339-1620,
 * angin1/angin2 :719-873, solofd :1682-1729) is built on the device and its lowest NEVAL levels
 * (Eh, dgrot :1731-1800) go to levels (cap entries); *nlev receives their number; out / outlen
 * as for dvr3d_b200_run_deck receive the printed level table. One parity per call: KMIN = 1
 * (e, k = 0..J) or 0 (f, k = 1..J) from a file of the same KMIN (KMIN = 1 also reads a KMIN = 2
 * file's first J + 1 blocks); KMIN = 2 (both sets) returns DVR3D_ERR_ARG here and is run by
 * dvr3d_b200_rotlev3b_pair. */
int dvr3d_b200_rotlev3b(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, double *levels, int cap,
                        int *nlev, char *out, size_t outcap, size_t *outlen);

/* The same with ROTLEV3B's ZTRAN: the eigenvectors are also transformed back to the first
 * step's basis, the angular DVR of each k block taken to associated Legendre functions
 * (dstore :1917-2049, tofbr :2175-2228, jtran :2230-2274), and written to kvec_path (unit
 * KVEC = 8) in the record layout DIPOLE3 reads: the DVR3D header, (nend, lmin, lbasis, nkbas),
 * the radial grid, nval, the levels (Eh), then one record d(nkbas(k), nval) per k block. */
int dvr3d_b200_rotlev3b_trans(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, const char *kvec_path,
                              double *levels, int cap, int *nlev, char *out, size_t outcap, size_t *outlen);

/* ROTLEV3B with KMIN = 2 on a KMIN = 2 first-step file: the e set (k = 0..J), then the second
 * pass (vrmain :600-660), the f set (k = 1..J) with the file's f-type k = 1 block (stored after
 * the e blocks) in place of the e-type one; its Coriolis blocks with k = 2 and 3 formed anew
 * (solrt :1529-1617), those among k >= 2 as in the first pass; NEVAL2 f levels. With ZTRAN
 * (non-empty paths) the e vectors go to kvec_path (unit KVEC = 8) and the f vectors to
 * kvec2_path (KVEC2 = 9); for J = 1 the f set is the f-type k = 1 block itself, copied in the
 * layout of a one-block file (dstore1 :2051-2173). out receives both printed tables. */
int dvr3d_b200_rotlev3b_pair(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, const char *kvec_path,
                             const char *kvec2_path, double *levels_e, int cap_e, int *nlev_e, double *levels_f,
                             int cap_f, int *nlev_f, char *out, size_t outcap, size_t *outlen);

/* The second variational step for J > 0 with the z axis along r1 or r2 (Jacobi coordinates,
 * IDIA = 1 or 2, and unsymmetrised Radau): the reference's program ROTLEV3 (source/rotlev3.f90).
 * deck_text is ROTLEV3's stdin (namelist PRT, card NVIB,NEVAL,KMIN,IBASS,NEVAL2 (12i5, insize
 * :150-151), title, optional EZERO card, vrmain :519-522); wave_path the first step's ZTRAN file
 * (unit IWAVE = 26; KMIN = 1 or 2 need a file of KMIN = 1, :287). The Hamiltonian in the lowest
 * first-step functions of each k block (select :301-480) with the Coriolis blocks of k-1, k
 * (solrt :671-837 on the vectors taken to associated Legendre functions, jtran :839-905) is built
 * on the device; its lowest NEVAL levels (Eh, dgrot :1046-1199) go to levels (cap), their number
 * to *nlev: the e set for KMIN = 1, the f set for KMIN = 0; KMIN = 2 also gives the f set (the
 * Hamiltonian without its k = 0 block, NEVAL2 levels, vrmain :600-660) in levels_f (cap_f,
 * *nlev_f; may be NULL otherwise). Non-empty kvec_path / kvec2_path (ZTRAN) receive the first /
 * second set's vectors in the first step's basis (dstore :1201-1342, units KVEC = 8 and
 * KVEC2 = 9); the J = 1 f set is the file's second k block copied as a one-block file (dstore1
 * :1344-1476), written to kvec2_path also when KMIN = 0, as the reference writes it to KVEC2.
 * out / outlen receive the printed level lists. */
int dvr3d_b200_rotlev3(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, const char *kvec_path,
                       const char *kvec2_path, double *levels, int cap, int *nlev, double *levels_f, int cap_f,
                       int *nlev_f, char *out, size_t outcap, size_t *outlen);

/* ---- DIPOLE3: transition moments between two sets of vib-rot states ------------------- */
/* The user's dipole surface, the two plug-ins of source/dipole3_segmented.f90:
 *   DIPD(DIPC, R1, R2, XCOS, NU) (:2054): component nu (0: along the embedding z axis, 1: x)
 *     at the scattering / Radau / bond coordinates of the wavefunction files;
 *   DIPSA(DIPX, DIPY, Q1, Q2, COST) (:2108): the bond-frame components, called by the
 *     reference's own DIPD, which does the coordinate transform and the rotation to the
 *     embedding (bond-angle, scattering, general and bisector branches, :2065-2192). */
typedef double (*dvr3d_dipd_fn)(double r1, double r2, double xcos, int nu, void *user);
typedef void (*dvr3d_dipsa_fn)(double *dipx, double *dipy, double q1, double q2, double cost, void *user);

typedef struct dvr3d_dipole_result {
    int cap1, cap2;      /* in: capacity of e1 (cap1), e2 (cap2); tz, tx, sint hold cap1 x cap2 */
    double *e1, *e2;     /* out: ket and bra energies (Eh) of the states taken                 */
    double *tz, *tx;     /* out: z and x transition moments (a.u.) without the common factor
                            sqrt((2j1+1)(2j2+1)), column-major, leading dimension cap1          */
    double *sint;        /* out: S(f-i) in a.u. (the values written to unit ITRA)              */
    int neval1, neval2;  /* out: ket and bra states taken (NV1, NV2, IBASE1, IBASE2)           */
    int j1, j2, kmin1, kmin2;
    int nblocks;         /* out: k -> k' blocks computed                                        */
    double dev_ms;       /* out: device time (CUDA events) of the vector uploads, the angular
                            transforms and the moment products                                */
    double flops;        /* out: their algorithmic floating-point operations                   */
} dvr3d_dipole_result;

/* DIPOLE3 (source/dipole3_segmented.f90): deck_text is its stdin (namelist PRT, title, card
 * NPOT,NV1,NV2,IBASE1,IBASE2 (5i5), optional EZERO card (f20.0), insize :198-620, spect
 * :1825-1954); ket_path and bra_path the two wavefunction files (units IKET = 11, IBRA = 12):
 * a J = 0 file as dvr3d_b200_run_deck_wave writes it, or a J > 0 file as
 * dvr3d_b200_rotlev3b_trans writes it. Exactly one of dipd / dipsa is given; it is called on
 * the host at the radial DVR points and NPOT Gauss-Legendre points (lagpt :1141-1232). The
 * vectors of every k block are evaluated at the angular points (dsrd :1412-1562, jtran
 * :1564-1646) and the transition moments of each k -> k' block (trans :1648-1776) formed on the
 * device as FP64 tensor-core (DMMA) GEMMs. Results go to res; out / outlen receive the printed
 * table; with ZTRA (the default) and a non-empty tra_path the records of outpt (:1956-2003) are
 * written to tra_path (appended unless ZSTART). Symmetrised Radau files (IDIA = -2, bisector
 * embedding) and Jacobi files; both files without Coriolis coupling (ZNCOR), and restart runs
 * (IRES), return DVR3D_ERR_UNSUPPORTED. */
int dvr3d_b200_dipole3(dvr3d_ctx *ctx, const char *deck_text, const char *ket_path, const char *bra_path,
                       dvr3d_dipd_fn dipd, dvr3d_dipsa_fn dipsa, void *user, const char *tra_path,
                       dvr3d_dipole_result *res, char *out, size_t outcap, size_t *outlen);

/* The split-BF16 tensor-core product of the mixed-precision form, on host buffers:
 *     c (m x n, ldc) = a^T b,   a: k x m (lda), b: k x n (ldb), all column-major FP64.
 * Each operand is split on the device into BF16 slices (x ~= hi + lo); nslice = 1 keeps hi
 * only (one BF16 product), nslice = 2 forms the BF16x3 product hi.hi + hi.lo + lo.hi with FP32
 * accumulation in tensor memory (relative error of order 2^-16 of |a|^T |b|). The same
 * kernel assembles the contracted Hamiltonian (mkham3 :2508-2523, bloc3d :3455-3505) and
 * forms H3 V in the mixed-precision solve. No counterpart in the reference; exposed for tests
 * and for callers that want the product itself. */
int dvr3d_b200_split_gemm(dvr3d_ctx *ctx, int m, int n, int k, const double *a, long long lda, const double *b,
                          long long ldb, int nslice, double *c, long long ldc);

/* An FP64 GEMM on the int8 tensor cores (Ozaki scheme), on host buffers, as the shift-invert
 * solve uses it for the large products of its Cholesky-inverse:
 *     c (m x n, ldc) = alpha op(a) op(b) + beta c,   column-major FP64,
 *     op(a) = ta ? a^T (a: k x m, lda) : a (m x k, lda);  op(b) = tb ? b^T (b: n x k) : b (k x n);
 *     tri = 1 / 2: op(a) lower / upper triangular; tri_b = 1 / 2: op(b) lower / upper
 *     (ignored outside the triangle; the DMMA path, nslice = 0, needs zeros there);
 *     lower_out: m == n, only c(i, j), i >= j.
 * Each row of op(a) and column of op(b) is scaled by a power of two and cut into nslice
 * (4..8) signed 7-bit slices; the slice products are exact int32 sums (k <= 16384) combined in
 * FP64: with 8 slices the error per term is below 2^-49 max|op(a)(i,:)| max|op(b)(:,j)|.
 * nslice = 0 runs the same product on the FP64 DMMA path instead (for comparisons).
 * No counterpart in the reference (its products are LAPACK / BLAS calls). lda, ldb even. */
int dvr3d_b200_ozaki_gemm(dvr3d_ctx *ctx, int ta, int tb, int tri, int tri_b, int lower_out, int m, int n, int k,
                          double alpha, const double *a, long long lda, const double *b, long long ldb, double beta,
                          double *c, long long ldc, int nslice);

/* Reads a job deck in the reference's stdin format: namelist PRT (dvr3d :65, defaults of
 * block data :158-167), card 2 (insize :232), card 3 (:238), title (:372) and the setcon
 * cards (:1042-1095, in the source's order FIXCOS, XMASS, XMASSR, EMAX1/EMAX2, r1 Morse,
 * r2 Morse), plus the optional EZERO card (:2751). Host-only; needs no GPU. */
int dvr3d_b200_parse_deck(const char *text, dvr3d_deck *out);

/* Select the potential. Replaces linking a POTV routine (docum.tex:30-47). */
int dvr3d_b200_set_pes(dvr3d_ctx *ctx, int kind, const double *params, int nparams);
/* Table of V for DVR3D_PES_GRID (layout documented at DVR3D_PES_GRID). */
int dvr3d_b200_set_pes_grid(dvr3d_ctx *ctx, const double *v, size_t n);
/* The table of k block kz alone, in the same layout on that block's own grid (the angular
 * points of block k are those of its associated Legendre quadrature, dvr3d_b200_grid(kz)):
 * with ZROT every k block of a run calls the reference's POTV at its own points. Takes
 * precedence over the common table for that block; n = 0 removes it. */
int dvr3d_b200_set_pes_grid_k(dvr3d_ctx *ctx, int kz, const double *v, size_t n);

/* DVR grid of one k block, so a host can evaluate its own POTV there: r1[npnt1],
 * r2[npnt2] (bohr; r2 = r1 for Radau idia=-2) and xalf[nalf] (cos theta, full range),
 * as computed by lagpt (:1290-1366), jacobi/allpts (:1635-1772). */
int dvr3d_b200_grid(dvr3d_ctx *ctx, const dvr3d_deck *deck, int kz,
                    double *r1, int n1cap, double *r2, int n2cap, double *xalf, int nacap);

/* Solve one k block of one deck. Replaces, for that block, the per-k driver call of
 * ccmain (:988-1006): nfmain(hr,htheta,r,theta,kz) (:3006, Radau idia=-2 in-plane) or
 * jhmain(xk1,xk2,xlmatr,r1,r2,xalf,r2m2t,kz) (:1915, Jacobi/scattering and idia=-1),
 * including their calls of diag -> dsyev (:2638-2659) and diag3d (:2661-2764). */
int dvr3d_b200_solve_block(dvr3d_ctx *ctx, const dvr3d_deck *deck, int kz,
                           const dvr3d_options *opt, dvr3d_result *res);

/* Solve `nprob` independent J=0 decks, each with its own PES parameter row
 * (pes_params[i*DVR3D_PES_MORSE_SUM_NPARAM ...]), as one batched device workload. This is
 * the repeated-caller pattern of the reference's fitting driver (SFIT_DVR3D runs DVR3DRJZ
 * once per trial surface, SFIT_DVR3D/H2S/dvr3d_sfit.f90:746-832). */
int dvr3d_b200_solve_batch(dvr3d_ctx *ctx, const dvr3d_deck *decks, const double *pes_params,
                           int nprob, const dvr3d_options *opt, dvr3d_result *res);

/* Run a whole job like `program DVR3DRJZ` (:1-80): parse, loop over k blocks as ccmain
 * (:857-1007) does, and write the level tables of diag3d (:2703-2761) into `out` (NUL-
 * terminated; *outlen receives the length needed). Levels in the fort.14 layout of zpfun
 * (:2708-2719) go to `lev` when non-NULL. */
int dvr3d_b200_run_deck(dvr3d_ctx *ctx, const char *deck_text, const dvr3d_options *opt,
                        char *out, size_t outcap, size_t *outlen,
                        char *lev, size_t levcap, size_t *levlen);

/* dvr3d_b200_run_deck plus the wavefunction file the reference writes to unit IWAVE
 * (fort.26) when the deck sets ZTRAN, written to `wave_path` record by record as DVR3DRJZ
 * writes it: the setcon header (:1176-1184), the ccmain records (:820-845), per k block the
 * angular grid and polynomials (:972-976), for Radau testiv's selection (:3446-3448), and the
 * levels and each level's amplitudes on the DVR grid from trans (Jacobi, psi(idvr, npnt1,
 * npnt2), :3733-3841) or transr (Radau, wvfunc(nbass), :3622-3641). Records are sequential
 * unformatted with a 4-byte length count before and after each; logicals are 4-byte with
 * .TRUE. = -1. Amplitudes are defined up to the sign of each eigenvector. The readers are
 * ROTLEV3 / ROTLEV3B / DIPOLE3 (source/wfnread.f90:101-215 reads the same records). */
int dvr3d_b200_run_deck_wave(dvr3d_ctx *ctx, const char *deck_text, const dvr3d_options *opt,
                             char *out, size_t outcap, size_t *outlen,
                             char *lev, size_t levcap, size_t *levlen, const char *wave_path);

/* Batched replacement of diag(ham,maxham,nham,eig) -> dsyev('V','L',...) (:2638-2659) for
 * many independent symmetric blocks already on the device: block b is n[b] x n[b] at
 * a + off[b] with leading dimension n[b] (lower triangle read). Eigenvalues ascending go
 * to w + woff[b]; when vecs != 0 the eigenvectors overwrite the blocks. Device pointers. */
int dvr3d_b200_diag_batched(dvr3d_ctx *ctx, int nblk, const int *n_host,
                            const long long *off_host, const long long *woff_host,
                            double *a_dev, double *w_dev, int vecs);

/* ---- learned Davidson preconditioner (no counterpart in the reference) ---------------- */
/* A solve with options.learned_precond = 2 records (residual, ideal correction) pairs and
 * trains the context's network; later solves with learned_precond = 1 use it (for example
 * trained on k = 0 and reused for the other k blocks, or on one surface of a fit and reused
 * for the next). Its parameters can be read out and loaded into another context. */
/* Copies the trained parameters into w (n >= DVR3D_LP_NPARAM); returns DVR3D_LP_NPARAM, or
 * DVR3D_ERR_ARG when the context holds no trained network. */
int dvr3d_b200_lp_get_weights(dvr3d_ctx *ctx, double *w, int n);
/* Loads parameters (n == DVR3D_LP_NPARAM) as the context's trained network. */
int dvr3d_b200_lp_set_weights(dvr3d_ctx *ctx, const double *w, int n);
/* The network on its own, by the device kernels the solver and trainer use: for nmode modes
 * (channel eigenvalue lam, features f1, f2, f3, energy scale) and ncol Ritz values theta,
 * gout[m + j nmode] = 1 + f(phi(m, theta_j)) and grad = sum_mj delta[m + j nmode] dg/dw
 * (DVR3D_LP_NPARAM entries). Host arrays. */
int dvr3d_b200_lp_eval(dvr3d_ctx *ctx, const double *w, int nmode, int ncol, const double *lam,
                       const double *f1, const double *f2, const double *f3, double scale,
                       const double *theta, const double *delta, double *gout, double *grad);
/* Training loss (and its gradient when grad is not NULL) at parameters w (host) on the pairs
 * recorded by this context's last solve, which must have been a training solve
 * (learned_precond = 2). */
int dvr3d_b200_lp_train_loss(dvr3d_ctx *ctx, const double *w, double *loss, double *grad);

/* ---- allocation-free variant ---------------------------------------------------------- */
/* No counterpart in the reference. Same computation and arguments as
 * dvr3d_b200_diag_batched, for callers that must not allocate device memory (a host whose
 * framework's memory pool owns the GPU memory and forbids outside cudaMalloc, or a latency-
 * critical loop where cudaMalloc/cudaFree and their device-wide synchronisation must not
 * happen). No context is needed: the work runs on `stream` (a cudaStream_t, 0 = default
 * stream) of the current device, and all scratch comes from one array of
 * DVR3D_NOALLOC_SCRATCH_BYTES compiled into the library, held by every GPU that loads it.
 * Limit: requests needing more scratch than that -- about 8*(4n + 2n^2 + 5n*min(n,128)) bytes
 * summed over the blocks with vecs != 0 -- return DVR3D_ERR_SCRATCH; split them into several
 * calls. At most 65535 blocks per call (DVR3D_ERR_ARG beyond). A failed launch returns
 * DVR3D_ERR_CUDA before the caller's a_dev / w_dev are written; inverse iteration that does
 * not converge returns DVR3D_ERR_NOCONV, as dvr3d_b200_diag_batched does. The first call on a device looks the array up (do it before any stream capture on
 * that device). All calls share the array: calls that may overlap on the GPU race and must
 * be serialised by the caller. Synchronises `stream` before returning. */
#define DVR3D_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
int dvr3d_b200_diag_batched_noalloc(void *stream, int nblk, const int *n_host,
                                    const long long *off_host, const long long *woff_host,
                                    double *a_dev, double *w_dev, int vecs);

#ifdef __cplusplus
}
#endif
#endif /* DVR3D_B200_H */
