/*
 * crt_oracle.h -- CPU FP64 restatement of CRTomo's forward / sensitivity /
 * Gauss-Newton inner-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle and the timed
 * CPU baseline.  The product (crtomo_stable_b200, libcrt_b200.so) never links,
 * loads or calls it; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg do.
 *
 * Every function restates one Fortran routine of geophysics-ubonn/crtomo_stable
 * (cited as src/<file>.f90:<lines>).  Array layouts follow the Fortran module
 * arrays exactly: column-major, with 1-based node / element / electrode numbers
 * stored in the integer arrays.  Complex quantities are C99 double complex
 * (layout-compatible with Fortran COMPLEX(KIND(0D0))).
 */
#ifndef CRT_ORACLE_H
#define CRT_ORACLE_H

#include <complex.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double complex dcplx;

/* Mirror of the module state the hot path reads (elemmod, electrmod, datmod,
 * wavenmod, femmod, randbmod).  All pointers are borrowed. */
typedef struct {
    /* elemmod (src/elemmod.f90) */
    int32_t sanz, typanz, mb;
    int32_t elanz, relanz, maxnodes;     /* max_nr_element_nodes */
    const int32_t *typ, *nelanz, *selanz;/* [typanz] */
    const int32_t *snr;                  /* [sanz]  */
    const double *sx, *sy;               /* [sanz]  */
    const int32_t *nrel;                 /* nrel(elanz+relanz, maxnodes) */
    const int32_t *rnr;                  /* [relanz] */
    /* electrmod */
    int32_t eanz;
    const int32_t *enr;                  /* [eanz] */
    /* datmod */
    int32_t nanz;
    const int32_t *strnr, *vnr;          /* [nanz] */
    /* wavenmod */
    int32_t kwnanz, swrtr;
    const double *kwn, *kwnwi;           /* [kwnanz] */
    /* femmod precal outputs */
    const double *elbg;                  /* elbg(elanz, nmn, kwnanz) */
    const double *relbg;                 /* relbg(relanz, nmn)       */
    const double *kg;                    /* kg(relanz, eanz, kwnanz) */
    int32_t lbeta, lrandb, lrandb2, lsink, nsink;
    /* randbmod (boundary.dat values) */
    int32_t rwdanz;
    const int32_t *rwdnr;                /* [rwdanz] node numbers */
    const dcplx *rwd;                    /* [rwdanz] values        */
} orc_problem;

/* src/rwaven.f90:22-171 (+ gauleg.f90, gaulag.f90).  kwn/kwnwi need room for
 * 30 entries.  Returns errnr. */
int orc_rwaven(const orc_problem *p, int32_t *kwnanz, double *kwn,
               double *kwnwi, double *amin, double *amax);

/* src/gauleg.f90:17-38, src/gaulag.f90:16-42 */
void orc_gauleg(double x1, double x2, double *x, double *w, int n);
void orc_gaulag(double *x, double *w, int n, double alf);

/* src/bessk0.f90, bessk1.f90, bessi0.f90, bessi1.f90 */
double orc_bessk0(double x);
double orc_bessk1(double x);

/* src/precal.f90:13-222 with elem1/elem3/elem5/elem8/beta/bsytop.
 * elbg, relbg, kg caller-allocated (sizes as in orc_problem).  lbeta/lrandb
 * are returned.  Returns errnr. */
int orc_precal(const orc_problem *p, int lsytop, double *elbg, double *relbg,
               double *kg, int32_t *lbeta, int32_t *lrandb);

/* Forward loop of src/inv.f90:343-484 (and src/fem.f90:328-397): for each
 * wavenumber k and electrode l assemble (kompab/kompadc), apply Dirichlet
 * nodes (randb/randdc, randb2/randbdc2), scale (scalab/scaldc), factor
 * (chol/choldc), or only rebuild the RHS (kompb/kompbdc), solve (vre/vredc)
 * and store kpot(j,l,k) = pot(j)*fak(j).  ldc selects the real path (kpot
 * then has zero imaginary parts).  OpenMP over k with nthreads threads,
 * as the reference does.  kpot(sanz, eanz, kwnanz).  Returns errnr. */
int orc_forward(const orc_problem *p, const dcplx *sigma, int ldc,
                int nthreads, dcplx *kpot);

/* Single-system pieces, exposed for unit tests (0-based slices of the
 * Fortran arrays, band a((mb+1)*sanz)). */
int orc_kompab(const orc_problem *p, int nelec, int ki, const dcplx *sigma,
               dcplx *a, dcplx *b);
int orc_scalab(const orc_problem *p, dcplx *a, dcplx *b, double *fak);
int orc_chol(const orc_problem *p, dcplx *a);
void orc_vre(const orc_problem *p, const dcplx *a, const dcplx *b, dcplx *pot);

/* src/rtrafo.f90:46-90.  hpot(sanz, eanz). */
void orc_rtrafo(const orc_problem *p, const dcplx *kpot, dcplx *hpot);
/* src/bvolti.f90:43-89.  Returns errnr (82 on zero voltage). */
int orc_bvolti(const orc_problem *p, const dcplx *hpot, dcplx *volt,
               dcplx *sigmaa);
/* src/bvolt.f90:40-79 (kfak NULL = 1). */
void orc_bvolt(const orc_problem *p, const dcplx *hpot, const double *kfak,
               dcplx *volt, dcplx *sigmaa);
/* src/bkfak.f90:46-136.  Returns errnr (93). */
int orc_bkfak(const orc_problem *p, double *kfak);

/* src/bsensi.f90:82-188 (normalised complex), src/bsendc.f90:62-179 (real:
 * result in the real parts), src/bsens.f90:82-193 (CRMod, strom==NULL means
 * unit currents).  sens(nanz, elanz). OpenMP over measurements. */
void orc_bsensi(const orc_problem *p, const dcplx *kpot, const dcplx *sigma,
                const dcplx *volt, int nthreads, dcplx *sens);
void orc_bsendc(const orc_problem *p, const dcplx *kpot, const dcplx *sigma,
                const dcplx *volt, int nthreads, double *sensdc);
void orc_bsens(const orc_problem *p, const dcplx *kpot, const double *strom,
               int nthreads, dcplx *sens);

/* src/refsig.f90:7-73 */
dcplx orc_refsig(const orc_problem *p, const dcplx *sigma);

/* src/bnachbar.f90:52-90.  nachbar(elanz, maxnodes+1) */
void orc_bnachbar(const orc_problem *p, int32_t *nachbar);
/* element midpoints as src/relem.f90 sets espx/espy */
void orc_esp(const orc_problem *p, double *espx, double *espy);
/* src/bsmatm_mod.f90:364-460 (ltri 1/2): smatm(elanz, maxnodes+1) */
void orc_bsmatmtri(const orc_problem *p, const int32_t *nachbar,
                   const double *espx, const double *espy, double alfx,
                   double alfz, double *smatm);
/* src/bsmatm_mod.f90:190-362 (ltri 0): smatm(nx*nz, 3) */
void orc_bsmatmreg(const orc_problem *p, int nx, int nz, double alfx,
                   double alfz, double *smatm);

/* Inner solve parameters (konvmod / cjgmod / invmod state). */
typedef struct {
    int32_t manz, nanz;
    int32_t ltri, nx;           /* regulariser: 0 = five point, 1/2 = nachbar */
    int32_t nnb;                /* max_nr_element_nodes (smatm columns - 1)   */
    int32_t ldc, lfpi;
    int32_t ncgmax;
    double lam, eps;
    const double *smatm;        /* smatm(manz, 3) or smatm(manz, nnb+1)       */
    const int32_t *nachbar;     /* nachbar(manz, nnb+1) for ltri 1/2          */
    const double *wmatd;        /* [nanz] */
    const int32_t *wdfak;       /* [nanz] */
} orc_cg_params;

/* src/update.f90:55-351 for lprior = ldiff = lw_ref = .false.:
 * builds bvec (regularisation gradient, RHS) and cgfac, runs cjggra/cjggdc
 * (src/cg_mod.f90:426-518 / :106-199), rescales dpar and applies
 * par += step*dpar.  sens is the complex Jacobian (nanz, manz); for ldc the
 * real Jacobian sensdc is used instead.  cgres must hold ncgmax+1 values.
 * Outputs: dpar[manz], cgfac[manz], bvec_rhs[manz] (the scaled RHS before
 * CG), cgres, ncg, bdpar. par is updated in place. */
void orc_update(const orc_cg_params *c, const dcplx *sens, const double *sensdc,
                const dcplx *dat, const dcplx *sigmaa, double step,
                dcplx *par, dcplx *dpar, double *cgfac, dcplx *bvec_rhs,
                double *cgres, int32_t *ncg, double *bdpar);

/* CG only (src/cg_mod.f90:426-518 complex, :106-199 real).  bvec is the
 * scaled RHS on entry and scratch on exit. */
void orc_cjggra(const orc_cg_params *c, const dcplx *sens, const double *cgfac,
                dcplx *bvec, dcplx *dpar, double *cgres, int32_t *ncg);
void orc_cjggdc(const orc_cg_params *c, const dcplx *sens, const double *sensdc,
                const double *cgfac, dcplx *bvec, dcplx *dpar, double *cgres,
                int32_t *ncg);

/* src/brough_mod.f90 (tri / reg, lprior = .false.) */
double orc_brough(const orc_cg_params *c, const dcplx *par);

/* src/blam0.f90:131-167: lambda_0 from the Jacobian (no preset), the
 * reference's O(nanz manz^2) loop; uses c->wmatd, c->wdfak, c->ldc,
 * c->lfpi. */
double orc_blam0(const orc_cg_params *c, const dcplx *sens, const double *sensdc, double alfx, double alfz);
/* src/parfit.f90:38-186: step length from the misfits at steps 0, 0.5, 1. */
double orc_parfit(double fa, double fb, double fc, double fmin, double smin);

/* src/dmisft.f90:73-137 with chkpo2 (lrobust = ldiff = .false.).
 * Returns nrmsd; betrms/pharms optional. */
double orc_dmisft(int nanz, const dcplx *dat, const dcplx *sigmaa,
                  const double *wmatd, const double *wmatdr,
                  const double *wmatdp, int lfpi, int lpol, double *betrms,
                  double *pharms, int32_t *npol);

#ifdef __cplusplus
}
#endif
#endif
