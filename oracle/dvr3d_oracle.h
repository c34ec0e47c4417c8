/*
 * dvr3d_oracle.h -- CPU FP64 restatement of the DVR3DRJZ hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker: it is loaded by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the product
 * library. It restates source/dvr3drjz_segmented.f90 of the reference routine by routine
 * (each function cites the lines it follows) and calls LAPACK dsyev like the reference.
 */
#ifndef DVR3D_ORACLE_H
#define DVR3D_ORACLE_H
#include <stddef.h>
#include "../include/dvr3d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Resolve dsyev/dsyevd/dgemm from a LAPACK shared object (scipy's OpenBLAS exports them
 * as scipy_dsyev_ ...). `prefix` is the symbol prefix ("scipy_" or ""). */
int oracle_load_lapack(const char *path, const char *prefix);

/* All eigenpairs of the symmetric n x n matrix a (lower triangle read, column-major) by the
 * loaded dsyev('V','L'): ascending w, vectors over a. */
int oracle_dsyev_lower(double *a, int n, double *w);

/* The oracle's own reader of a job deck (deck_reader.cpp), independent of the product's
 * dvr3d_b200_parse_deck: namelist PRT, cards 2-10 and the optional EZERO card. */
int oracle_parse_deck(const char *text, dvr3d_deck *out);

/* Quadrature known-answer data of one k block (what lagpt / jacobi print). */
typedef struct oracle_quad {
    int npnt1, npnt2, nang2, nidvr;
    double y1[128], wt1[128], r1[128];   /* Gauss-Laguerre points, weights, r (r1) */
    double csx1, csa1, tsx1, tsa1;
    double y2[128], wt2[128], r2[128];   /* same for r2 (idia > -2) */
    double csx2, csa2, tsx2, tsa2;
    double xhalf[128], whalf[128];       /* jacobi() output before allpts (printed)  */
    double cswalf, tswalf;
    double xalf[256], walf[256];         /* after allpts (walf = sqrt(scale w))      */
    double ur1, ur2, urr1, urr2, beta1, beta2, a1, a2, g1, g2;
    int iu1, iu2;
    int status;                          /* 0 or DVR3D_ERR_QUADRATURE                */
} oracle_quad;

int oracle_quadrature(const dvr3d_deck *deck, int kk, oracle_quad *q);

/* Optional intermediate outputs of one k block. All pointers may be NULL. */
typedef struct oracle_trace {
    int nblocks;                 /* nalf (Radau) or npntc (Jacobi)                        */
    int npnta, npntb, npntc, max2d, max3d, kz, ipar;
    int *iv1; int iv1_cap;       /* Jacobi: 1D counts iv1(ione,itwo) as [ione*npntb+itwo]  */
    int *iv2; int iv2_cap;       /* per-block 2D selection counts                          */
    int *n2d; int n2d_cap;       /* per-block 2D Hamiltonian dimension                     */
    double *eig2all; int eig2all_cap;   /* all 2D eigenvalues, blocks concatenated         */
    double *eigs2d; int eigs2d_cap;     /* selected 2D eigenvalues in final-basis order     */
    double *h3; size_t h3_cap;          /* assembled final Hamiltonian (lower valid)        */
    double stage_s[4];           /* wall seconds: 1D/2D stage, assembly, final diag, total */
    int nham3;
    /* wavefunction amplitudes of the returned levels on the DVR grid (trans :3649-3843 /
     * transr :3596-3643): psi_nlev records of psi_len doubles, as the reference writes them */
    double *psi; size_t psi_cap;
    long long psi_len; int psi_nlev;
    /* the angular record of the block as a ZTRAN file holds it (ccmain :972-976): pleg(l, i)
     * walf(i), (maxleg + 1) x nidvr, with the kz line's maxleg, nidvr and lincr */
    double *pleg_walf; size_t pleg_cap;
    int maxleg, nidvr, lincr;
} oracle_trace;

/* final_mode: 0 = dsyev('V','L') with lwork = 3*N as diag() does (:2650-2654);
 *             1 = dsyevd (the divide-and-conquer variant kept commented in :2612-2636);
 *             2 = stop after assembly (no final diagonalisation);
 *             3 = stop after the 2D selection (sizes and counts only). */
int oracle_solve_block(const dvr3d_deck *deck, int kk, int pes_kind, const double *pes,
                       int npes, const double *vgrid, size_t nvgrid, int final_mode,
                       oracle_trace *trace, dvr3d_result *res);

/* Stepwise run of oracle_solve_block (same arguments and results), for timing one complete
 * solve as a sequence of bounded steps: _begin sets the block up and starts a worker thread
 * that waits before each unit of work (per block of the 1D and 2D stages, the selection,
 * per block row of the assembly, the final diagonalisation); _step lets it run `units`
 * more units and returns the units left (0 when the solve is complete, < 0 on error);
 * _end cancels an unfinished run or collects the results, and frees the session. */
int oracle_session_begin(const dvr3d_deck *deck, int kk, int pes_kind, const double *pes, int npes,
                         const double *vgrid, size_t nvgrid, int final_mode, void **out);
int oracle_session_units(void *session);
int oracle_session_step(void *session, int units);
/* Between steps, after the selection unit: per block kept 2D states (iv2) and 2D dimension
 * (n2d); returns the number of blocks (0 before the selection has run). */
int oracle_session_counts(void *session, int *iv2, int *n2d, int cap);
int oracle_session_end(void *session, oracle_trace *trace, dvr3d_result *res);

/* ROTLEV3B (source/rotlev3b_segmented.f90) for one parity on a first-step wavefunction file:
 * lowest NEVAL levels (Eh) of the Coriolis-coupled Hamiltonian, diagonalised in core. */
int oracle_rotlev3b(const char *deck_text, const char *wave_path, double *levels, int cap, int *nlev);
/* DIPOLE3 (source/dipole3_segmented.f90) on two wavefunction files, arguments as
 * dvr3d_b200_dipole3 (without the context). */
int oracle_dipole3(const char *deck_text, const char *ket_path, const char *bra_path, dvr3d_dipd_fn dipd,
                   dvr3d_dipsa_fn dipsa, void *user, const char *tra_path, dvr3d_dipole_result *res, char *out,
                   size_t outcap, size_t *outlen);
/* lagpt's angular rule (jacobi :1311-1368, alf = bta = 0): the npot/2 largest points, weights,
 * computed and exact half sums of the weights. */
int oracle_dipole_quadrature(int npot, double *x, double *w, double *csa, double *tsa);
/* threej :1778-1823 */
double oracle_threej(int j1, int j2, int j3, int m1, int m2, int m3);
/* KMIN = 2: both passes (e levels, then the f levels of the second pass, vrmain :600-660),
 * with ZTRAN the e vectors to kvec_path and the f vectors to kvec2_path (either may be empty). */
int oracle_rotlev3b_pair(const char *deck_text, const char *wave_path, const char *kvec_path, const char *kvec2_path,
                         double *levels, int cap, int *nlev, double *levels2, int cap2, int *nlev2);
/* The same with ZTRAN: the transformed vectors (dstore :1917-2049) written to kvec_path. */
int oracle_rotlev3b_trans(const char *deck_text, const char *wave_path, const char *kvec_path, double *levels,
                          int cap, int *nlev);
/* ROTLEV3 (rotlev3_oracle.cpp): the second step for z along r1 or r2 on a first-step ZTRAN
 * file. levels: the e set (KMIN = 1, 2) or the f set (KMIN = 0); levels_f: the f set of
 * KMIN = 2. With ZTRAN the first set's vectors go to kvec_path and the KMIN = 2 f set's to
 * kvec2_path; J = 1 f (KMIN = 0) writes its single block to kvec2_path as the reference does. */
int oracle_rotlev3(const char *deck_text, const char *wave_path, const char *kvec_path, const char *kvec2_path,
                   double *levels, int cap, int *nlev, double *levels_f, int cap_f, int *nlev_f);
/* ROTLEV3B's Gauss-associated Legendre rule (jacobi :941-1007): the npnt2 = (npnt+1)/2 points
 * of the half range (descending from 1) and weights, computed and exact sums of weights. */
int oracle_rot_quadrature(int npnt, int k, double *x, double *w, double *cswalf, double *tswalf);

/* Derived sizes of insize (:171-638) for one k block (kk = loop index of ccmain :857). */
int oracle_sizes(const dvr3d_deck *deck, int kk, int *out16);

/* Potential family DVR3D_PES_MORSE_SUM at one point (for fixtures). */
double oracle_pes_morse_sum(const double *p, double r1, double r2, double xcos);

/* Time `reps` dsyev('V','L') calls on a seeded random symmetric n x n (CPU baseline
 * samples of the final eigensolve). Returns seconds per call. */
double oracle_time_dsyev(int n, int reps, int mode);

#ifdef __cplusplus
}
#endif
#endif
