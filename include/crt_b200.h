/*
 * crt_b200.h -- C ABI of the B200-native CRTomo forward / sensitivity /
 * Gauss-Newton inner-solve path (libcrt_b200.so).
 *
 * The ABI replaces the Fortran call sites of geophysics-ubonn/crtomo_stable
 * listed beside each entry point.  Conventions:
 *   - every entry point returns the reference's integer error number
 *     (src/error.txt: 0 ok, 19 band width, 26 element orientation, 27 zero
 *     diagonal, 28 non-positive pivot, 35 boundary geometry, 73 duplicate
 *     electrodes, 82 zero voltage, 93 zero geometric factor, 97 allocation),
 *     plus 200 for a CUDA runtime failure and 201 for an option outside the
 *     implemented path; crt_last_error() gives the message (fetxt);
 *   - arrays use the Fortran module layouts (column-major) and the
 *     reference's 1-based node / element / electrode numbers;
 *   - complex arrays are interleaved (re, im) doubles, the layout of
 *     COMPLEX(KIND(0D0)) / C99 double _Complex;
 *   - host arrays are borrowed for the duration of a call only; kpot, the
 *     Jacobian and the CG vectors stay in device memory inside the context
 *     between crt_forward -> crt_jacobian -> crt_update;
 *   - a context is bound to one device and one host thread; calls are
 *     synchronous.
 */
#ifndef CRT_B200_H
#define CRT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CRT_B200_ABI_VERSION 2

typedef struct crt_ctx crt_ctx;

/* Mesh: the elemmod arrays read by src/relem.f90 (elem.dat). */
typedef struct {
    int32_t sanz, typanz, mb;
    const int32_t *typ, *nelanz, *selanz; /* [typanz] */
    const int32_t *snr;                   /* [sanz] coordinate row of each node */
    const double *sx, *sy;                /* [sanz] */
    const int32_t *nrel;                  /* nrel(elanz+relanz, max(selanz)) */
    const int32_t *rnr;                   /* rnr(relanz) */
} crt_mesh;

/* Electrodes, measurements, wavenumbers and boundary options
 * (electrmod, datmod, wavenmod, femmod, randbmod). */
typedef struct {
    int32_t eanz;
    const int32_t *enr;                   /* [eanz] node numbers */
    int32_t nanz;
    const int32_t *strnr, *vnr;           /* [nanz] C1 + 10000*C2, P1 + 10000*P2 */
    int32_t kwnanz, swrtr;                /* swrtr 0: 2D (kwnanz 1), 1: 2.5D */
    const double *kwn, *kwnwi;            /* [kwnanz] from rwaven (crt_rwaven) */
    /* precal results in Fortran layout, or NULL to compute them on the
     * device (src/precal.f90): elbg(elanz, nmn, kwnanz), relbg(relanz, nmn),
     * kg(relanz, eanz, kwnanz), nmn = m(m+1)/2, m = max(selanz). */
    const double *elbg, *relbg, *kg;
    int32_t lsink, nsink;                 /* fictitious sink node */
    int32_t rwdanz;                       /* boundary.dat (lrandb2) */
    const int32_t *rwdnr;                 /* [rwdanz] node numbers */
    const double *rwd;                    /* [rwdanz] complex values */
    int32_t lsytop;                       /* mswitch bit 8: mirror about sytop */
} crt_survey;

/* Inner-solve controls (konvmod / cjgmod / invmod). */
typedef struct {
    double lam;        /* regularisation parameter */
    double eps;        /* stop when |r|^2 <= eps |r0|^2 (reference default 1e-4) */
    int32_t ncgmax;    /* iteration cap (reference: manz/10 for ltri < 5) */
    int32_t ldc;       /* DC inversion: real Jacobian (bsendc), cjggdc */
    int32_t lfpi;      /* final phase improvement: real part of J, imaginary RHS */
    double step;       /* model step length applied by crt_update */
    int32_t precond;   /* CRT_PRECOND_JACOBI (the reference's cjggra / cjggdc) or
                          CRT_PRECOND_BLOCK (no reference counterpart) */
} crt_cg_params;

/* CG forms.
 * CRT_PRECOND_JACOBI: the reference iteration, preconditioned by cgfac only.
 * CRT_PRECOND_BLOCK:  additionally preconditioned by S^-1, S the sparse part
 *   diag(C^2 J^H W J) + lam C R C of the scaled operator (C = diag(cgfac)),
 *   factored block-tridiagonally in FP32 after a reverse Cuthill-McKee
 *   ordering of the regulariser's graph; flexible (Polak-Ribiere) beta, the
 *   reference's stop rule on the true residual.  Falls back to the Jacobi
 *   form when the ordered bandwidth exceeds 192 or a pivot breaks down
 *   (crt_cg_info reports which form ran). */
#define CRT_PRECOND_JACOBI 0
#define CRT_PRECOND_BLOCK 1
/* The learned correction (crt_gnn_*) added to the identity (Jacobi form) or
 * to the block preconditioner; used when the network was trained on records
 * of the same base, else the form without it runs. */
#define CRT_PRECOND_GNN 2
#define CRT_PRECOND_BLOCK_GNN 3

/* Precision forms.
 * CRT_PREC_FP64:  everything in FP64 / complex128 (the reference's arithmetic).
 * CRT_PREC_MIXED: the complex band systems are assembled and scaled in FP64,
 *                 factored and solved in complex64, and refined in FP64
 *                 (crt_set_refinement); the Jacobian is computed in FP64 and
 *                 stored in complex64; the CG accumulates in FP64.  Dot
 *                 products, quadrature weights, misfit and model update stay
 *                 FP64.  The DC (real) systems stay FP64. */
#define CRT_PREC_FP64 0
#define CRT_PREC_MIXED 1

/* Steps of FP64 iterative refinement after the complex64 factorisation of
 * the mixed form: at most `steps` (default 8; 0 leaves the complex64
 * solution).  Each step forms the residual of the scaled system in FP64
 * (from the FP64 entries of the prepared matrix) and its normwise
 * backward error max_r |r_r| / max_r (sum_c |a_rc| |z_c| + |b_r|), and adds
 * a complex64 correction solve; a system whose backward error is at most
 * the tolerance (crt_set_refinement_tol, default 1e-14, the FP64 floor)
 * takes no further steps, so well-conditioned systems stop after a few
 * while the ill-conditioned low-wavenumber systems keep refining.  No
 * reference counterpart. */
int32_t crt_set_refinement(crt_ctx *ctx, int32_t steps);
/* Normwise backward error at which a system's refinement stops (default
 * 1e-14; 0 runs every step for every system).  No reference counterpart. */
int32_t crt_set_refinement_tol(crt_ctx *ctx, double tau);

/* Forms of the forward model with mixed boundaries.
 * CRT_FORWARD_DIRECT: the reference's loop -- one assembled, scaled and
 *   factored band system per wavenumber and source electrode (kompab,
 *   scalab, chol, vre), in the context's precision form.
 * CRT_FORWARD_SCHUR: the same systems solved by block elimination of the
 *   mixed-boundary nodes G (every node of a type-11 segment), the only rows
 *   and columns in which the systems of different electrodes differ
 *   (src/kompab.f90:113-117): per wavenumber one band factorisation of the
 *   interior matrix and a multi-RHS solve of the source vectors and the
 *   interior-boundary couplings; per (wavenumber, electrode) a dense
 *   Cholesky of the m x m Schur complement on G and the rebuild of the
 *   interior potentials.  FP64 / complex128 arithmetic throughout in both
 *   precision forms (no refinement needed); needs no Dirichlet nodes and
 *   m <= 768.  The same potentials up to rounding.  No reference
 *   counterpart.
 * CRT_FORWARD_AUTO (default): the Schur form where it applies (and its
 *   workspaces fit a workspace limit set by crt_set_workspace_limit), the
 *   direct form otherwise. */
#define CRT_FORWARD_AUTO 0
#define CRT_FORWARD_DIRECT 1
#define CRT_FORWARD_SCHUR 2
int32_t crt_set_forward_form(crt_ctx *ctx, int32_t form);
/* Form of the last forward (CRT_FORWARD_DIRECT / _SCHUR; _AUTO before the
 * first), the boundary and interior node counts of the Schur split and the
 * interior half-bandwidth (0 when the Schur form does not apply).  Any
 * pointer may be NULL.  No reference counterpart. */
int32_t crt_forward_info(const crt_ctx *ctx, int32_t *form, int32_t *nboundary, int32_t *ninterior,
                         int32_t *mb_interior);

/* Creates a context on `device`: uploads the mesh, builds the gather lists
 * of the streamed assembly, and evaluates precal on the device unless the
 * survey provides elbg/relbg/kg.  Replaces the set-up part of
 * src/inv.f90:179-248 / src/fem.f90:308-326 (precal + ALLOCATEs). */
crt_ctx *crt_create(int32_t device, const crt_mesh *mesh, const crt_survey *survey,
                    int32_t precision, int32_t *errnr);
void crt_destroy(crt_ctx *ctx);
const char *crt_last_error(const crt_ctx *ctx);
int32_t crt_abi_version(void);

/* Wavenumbers and weights: src/rwaven.f90:22-171 (FP64, host).  kwn and
 * kwnwi need room for 30 values. */
int32_t crt_rwaven(const crt_mesh *mesh, int32_t eanz, const int32_t *enr, int32_t nanz,
                   const int32_t *strnr, const int32_t *vnr, int32_t *kwnanz, double *kwn,
                   double *kwnwi);

/* Copies the device precal results to the host in Fortran layout
 * (src/precal.f90 outputs elbg, relbg, kg) and reports lbeta / lrandb. */
int32_t crt_precal(crt_ctx *ctx, double *elbg, double *relbg, double *kg, int32_t *lbeta,
                   int32_t *lrandb);

/* Forward model for conductivities sigma(elanz) (complex):
 * the wavenumber x electrode loop of src/inv.f90:343-484 / src/fem.f90:
 * 328-397 (kompab/kompadc, randb/randb2, scalab/scaldc, chol/choldc,
 * kompb, vre/vredc), then rtrafo (src/rtrafo.f90) at the electrode nodes
 * and bvolti (mode 0, src/bvolti.f90: sigmaa = -ln V) or bvolt (mode 1,
 * src/bvolt.f90: sigmaa = kfak V, kfak NULL = 1).
 * ldc != 0 solves the real systems with Re(sigma).
 * volt / sigmaa: complex [nanz]; kpot: complex kpot(sanz, eanz, kwnanz) or
 * NULL (kept on the device for crt_jacobian / crt_potentials). */
int32_t crt_forward(crt_ctx *ctx, const double *sigma, int32_t ldc, int32_t mode,
                    const double *kfak, double *volt, double *sigmaa, double *kpot);

/* Potentials of the last forward call at all nodes, hpot(sanz, eanz)
 * (rtrafo, src/rtrafo.f90:46-90, used by bpot/wpot). */
int32_t crt_potentials(crt_ctx *ctx, double *hpot);

/* Jacobian of the last forward call: mode 0 bsensi (src/bsensi.f90),
 * 1 bsendc (src/bsendc.f90, real), 2 bsens (src/bsens.f90, CRMod).
 * strom: [nanz] currents for mode 2 (NULL = 1).  sens: sens(nanz, elanz),
 * complex (modes 0, 2) or real (mode 1), or NULL to keep it on the device. */
int32_t crt_jacobian(crt_ctx *ctx, int32_t mode, const double *strom, double *sens);

/* Uploads a Jacobian computed elsewhere (complex sens(nanz, manz), or real
 * sensdc when real != 0), replacing the device-resident one. */
int32_t crt_set_jacobian(crt_ctx *ctx, int32_t real, const double *sens);

/* Replaces the measurement configurations (same nanz), e.g. after the
 * polarity check of src/chkpol.f90 swapped potential electrodes.  A reading
 * whose new vnr is its old one with the two potential electrodes swapped
 * (same strnr) also gets the stored response of the last forward flipped,
 * as chkpol does (volt -> -volt, the phase of sigmaa moved by pi), so that
 * crt_jacobian after this call matches the swapped configuration. */
int32_t crt_set_configs(crt_ctx *ctx, const int32_t *strnr, const int32_t *vnr);

/* Regularisation operator R (src/bsmatm_mod.f90): ltri 0 five-point
 * smatm(manz, 3) with nx cells per row; ltri 1/2 neighbour form
 * smatm(manz, nnb+1) with nachbar(manz, nnb+1). */
int32_t crt_set_regularizer(crt_ctx *ctx, int32_t ltri, int32_t nx, int32_t nnb,
                            const double *smatm, const int32_t *nachbar);

/* Data and weights (datmod / invmod): dat complex [nanz] (-ln|R|, -phase),
 * wmatd [nanz], wdfak [nanz] (NULL = 1). */
int32_t crt_set_data(crt_ctx *ctx, const double *dat, const double *wmatd, const int32_t *wdfak);

/* src/update.f90:27-353 (lprior = ldiff = lw_ref = .false.): regularisation
 * gradient, Jacobi factors cgfac, scaled RHS, the CG of src/cg_mod.f90
 * (cjggra, or cjggdc for ldc / lfpi) on the device-resident Jacobian and
 * the model step par += step * dpar.  sigmaa: complex [nanz] forward
 * response (NULL = from the last crt_forward); par: complex [manz] in/out.
 * Optional outputs (NULL to skip): dpar [manz] complex, cgfac [manz],
 * cgres [ncgmax+1] (cgres[0] = ncg, cgres[k] = eps |r_k|^2/|r_0|^2 as
 * float), ncg, bdpar. */
int32_t crt_update(crt_ctx *ctx, const crt_cg_params *prm, const double *sigmaa, double *par,
                   double *dpar, double *cgfac, double *cgres, int32_t *ncg, double *bdpar);

/* Lambda candidates side by side.  The reference's inversion loop
 * (src/inv.f90:769-912) tries one lambda after another, each trial one
 * src/update.f90 pass with cjggra / cjggdc on the same Jacobian; this call
 * runs nlam (1 .. 8) such updates at once, and every CG iteration reads J
 * once for all candidates.  Candidate b is crt_update with prm->lam =
 * lams[b] (prm->lam is ignored) from the same sigmaa (NULL = the last
 * crt_forward) and par (complex [manz], not modified), in the Jacobi form,
 * or with prm->precond CRT_PRECOND_BLOCK (or _BLOCK_GNN: the learned
 * correction is not batched) in the block form with one factor per
 * candidate; if the block preconditioner is unavailable or any
 * candidate's factor breaks down, the batch runs in the Jacobi form
 * (crt_cg_info reports which).  par_out: complex [nlam][manz], par + step * dpar_b.
 * Optional (NULL to skip): dpar complex [nlam][manz], ncg [nlam],
 * bdpar [nlam]. */
int32_t crt_update_lambdas(crt_ctx *ctx, const crt_cg_params *prm, int32_t nlam, const double *lams,
                           const double *sigmaa, const double *par, double *par_out, double *dpar,
                           int32_t *ncg, double *bdpar);

/* lambda_0 of src/blam0.f90:131-167 from the device-resident Jacobian and
 * the weights of crt_set_data (wmatd * wdfak): lammax = 5 * 2/(alfx+alfz)
 * * sum_j |sum_i conj(J_ij) w_i sum_k J_ik| / manz, with the real Jacobian
 * (ldc, as stored by crt_jacobian mode 1) or the real part of the complex
 * one (lfpi).  Two passes over J instead of the reference's O(N M^2) loop;
 * the presets of src/blam0.f90:45-77 are the caller's. */
int32_t crt_blam0(crt_ctx *ctx, int32_t ldc, int32_t lfpi, double alfx, double alfz, double *lammax);

/* Coverage of src/bbsens.f90:52-78 from the device-resident Jacobian:
 * csens[j] = sum_i |J_ij| w_i (part 0; |Re J_ij| for part 1, the final
 * phase improvement's csens_fpi; the real Jacobian of crt_jacobian mode 1
 * takes part 0).  weight: [nanz] per-reading weights (bbsens's
 * sqrt(wmatd_cri | wmatdr | wmatd) * wdfak), or NULL for sqrt(wmatd * wdfak)
 * of crt_set_data.  The normalisation and log10 of the written file are
 * the caller's. */
int32_t crt_coverage(crt_ctx *ctx, int32_t part, const double *weight, double *csens);

/* One Gauss-Newton step of the reference loop (src/inv.f90:426-495,
 * :739-743, :924-933): sigma = exp(par); forward + bvolti; bsensi (or
 * bsendc); update.  par is updated in place.  Outputs as crt_update plus
 * sigmaa (complex [nanz], the response of the model the step started
 * from; NULL to skip). */
int32_t crt_gn_step(crt_ctx *ctx, const crt_cg_params *prm, double *par, double *sigmaa,
                    double *cgres, int32_t *ncg, double *bdpar);

/* Device-resident variant used for throughput measurement: the same step
 * on a model already in device memory (crt_set_model) without host
 * copies.  Returns after the work is enqueued and completed. */
int32_t crt_set_model(crt_ctx *ctx, const double *par);
int32_t crt_gn_step_device(crt_ctx *ctx, const crt_cg_params *prm, int32_t *ncg);
int32_t crt_get_model(crt_ctx *ctx, double *par);
/* Device-side copy of the current model: save (0) to or restore (1) from a
 * backup buffer, so repeated steps can restart from one model without host
 * traffic. */
int32_t crt_model_backup(crt_ctx *ctx, int32_t restore);

/* Timings of the phases of the last crt_gn_step / crt_gn_step_device
 * (milliseconds, CUDA events on the context stream): [0] forward factor,
 * [1] forward solves, [2] voltages, [3] Jacobian, [4] CG set-up, [5] CG
 * iterations, [6] total. */
int32_t crt_last_timings(const crt_ctx *ctx, double *ms7);

/* The same and more, up to n entries: [0..6] as crt_last_timings, [7] the
 * preparation pass of the forward factor (assembly, Dirichlet edits and
 * scaling of all rows), [8] the factor kernels alone, [9] the number of
 * factor-kernel launches (one per chunk of systems), [10] the FP64
 * residuals and [11] the correction solves of the mixed form's refinement
 * (both inside [1]), [12] the panel width of the blocked band factorisation
 * (chosen by the autotuner; 0 for the unblocked kernel), and in the Schur
 * form (inside [1]) [13] the forward sweep of the interior columns, [14]
 * their Gram products, [15] the electrode systems' solves (the iteration
 * with its reference factors, or the per-system Cholesky), [16] the rebuild
 * and the back sweep into the potentials, [17] the mean number of
 * iterations per electrode system when they were solved by the iteration,
 * 0 when by the Cholesky.
 * Milliseconds except [9], [12] and [17].  No reference counterpart. */
int32_t crt_last_timings_ex(const crt_ctx *ctx, double *ms, int32_t n);

/* Kernel launches enqueued by the context since creation. */
int64_t crt_launch_count(const crt_ctx *ctx);

/* Form of the last inner CG (CRT_PRECOND_*), block size B of the block
 * preconditioner (0 when unavailable for this regulariser) and the
 * regulariser's half-bandwidth after reverse Cuthill-McKee.  Any pointer
 * may be NULL.  No reference counterpart. */
int32_t crt_cg_info(const crt_ctx *ctx, int32_t *form, int32_t *block, int32_t *bandwidth);

/* Learned correction of the CG preconditioner (no reference counterpart).
 * A mesh graph network over the model cells (the regulariser's graph, three
 * message-passing layers of width 32, tanh, no biases, bf16 weights with FP32
 * sums) maps the normalised residual and the base preconditioner's output to
 * a correction: z = base(r) + net(r, base(r)).  It is trained on the GPU on
 * residual / error pairs recorded from the plain (Jacobi-form) CG of the
 * inversion itself and used by crt_update / crt_gn_step through
 * CRT_PRECOND_GNN / CRT_PRECOND_BLOCK_GNN.  The network weights are a flat
 * FP32 vector of crt_gnn_nparam() entries, matrices stored [in][out]:
 *   Win[4][32] | (Ws[32][32], Wn[32][32]) x 3 layers | Wout[32][2].
 * form: 0 trained on the identity base, 1 on the block preconditioner. */
int32_t crt_gnn_nparam(void);
/* Whether the network is available for this regulariser, trained, the base
 * it was trained on, the records held, and whether the last solve's guard
 * switched it off (a non-descent direction, or |r|^2 not halving over 50
 * iterations: the CG then finishes with the base preconditioner). */
int32_t crt_gnn_status(const crt_ctx *ctx, int32_t *available, int32_t *trained, int32_t *form, int32_t *nrec,
                       int32_t *guard_fired);
int32_t crt_gnn_init(crt_ctx *ctx, uint64_t seed);
int32_t crt_gnn_set_weights(crt_ctx *ctx, const float *w, int32_t n, int32_t form);
int32_t crt_gnn_get_weights(crt_ctx *ctx, float *w, int32_t n, int32_t *form);
/* Runs the plain CG of the current Gauss-Newton system (as crt_update would,
 * without changing the model) and records (r_k, x* - x_k) every `stride`
 * iterations, at most nmax; *nrec = records held in total. */
int32_t crt_gnn_collect(crt_ctx *ctx, const crt_cg_params *prm, int32_t base_block, int32_t stride,
                        int32_t nmax, int32_t *nrec);
int32_t crt_gnn_clear(crt_ctx *ctx);
/* Adam, seeded shuffles, mini-batches; loss_hist[epochs] = mean record loss
 * |z - e|^2 / |e - base|^2 (normalised units). */
int32_t crt_gnn_train(crt_ctx *ctx, int32_t epochs, int32_t batch, float lr, uint64_t seed, float *loss_hist);
/* One record's features x[M][4], target t[M][2], message weights a[M][4],
 * neighbours nbr[M][4] (-1 none) and |t|^2, and its loss and gradient with
 * the current weights (for checking against a CPU restatement). */
int32_t crt_gnn_record(crt_ctx *ctx, int32_t idx, float *x, float *t, float *a, int32_t *nbr, float *tnorm2);
int32_t crt_gnn_record_grad(crt_ctx *ctx, int32_t idx, float *grad, double *loss);

/* Reverse Cuthill-McKee ordering of an undirected graph in CSR form
 * (xadj[n+1], adj[xadj[n]], 0-based, both directions of every edge listed):
 * order[k] = the vertex placed at position k; *bandwidth (may be NULL) =
 * max |pos(v) - pos(w)| over the edges.  Host-only, no device needed.  The
 * ordering the block preconditioner uses for the regulariser's graph; the
 * reference renumbers mesh nodes with Cuthill-McKee in cutmckee/cutmck.f. */
int32_t crt_rcm_order(int32_t n, const int32_t *xadj, const int32_t *adj, int32_t *order, int32_t *bandwidth);

/* Allocation-free voltages.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory (all of their device memory is
 * allocated up front, e.g. from their own pool or a framework allocator, or
 * allocation is forbidden after start-up).  Computes what crt_forward's
 * last step does -- rtrafo at the electrode nodes and bvolti (mode 0,
 * sigmaa = -ln V) or bvolt (mode 1, sigmaa = kfak V) -- from a caller-held
 * kpot.  Every pointer except `stream` is DEVICE memory: kpot complex
 * kpot(sanz, eanz, kwnanz), kwnwi [kwnanz], enr [eanz] (1-based nodes),
 * strnr / vnr [nanz], kfak [nanz] or NULL, outputs volt / sigmaa complex
 * [nanz].  stream: a cudaStream_t (NULL = legacy default stream); the call
 * synchronises it before returning the errnr (82 zero voltage, 46 / 29 bad
 * electrode numbers, 3 bad arguments; 200 when a CUDA error from earlier
 * work was already pending on entry, which is left pending for its owner
 * and named on stderr).  It calls no cudaMalloc / cudaFree:
 * its scratch (the eanz x eanz table of electrode potentials) is a static
 * device array for at most 512 electrodes (4 MiB per GPU, held until
 * exit); eanz > 512 is rejected with errnr 3 and a message on stderr.  The
 * first call on a device looks up the array's device address (once per
 * device); make that first call before any stream capture.  All calls
 * share the array, so calls that overlap on the GPU race. */
int32_t crt_voltages_noalloc(const double *kpot, const double *kwnwi, const int32_t *enr,
                             const int32_t *strnr, const int32_t *vnr, int32_t sanz, int32_t eanz,
                             int32_t kwnanz, int32_t nanz, int32_t swrtr, int32_t ldc, int32_t mode,
                             const double *kfak, double *volt, double *sigmaa, void *stream);

/* Data misfit: src/dmisft.f90:73-137 with chkpo2 (FP64, host).
 * Returns nrmsd; betrms / pharms / npol optional. */
double crt_dmisft(int32_t nanz, const double *dat, const double *sigmaa, const double *wmatd,
                  const double *wmatdr, const double *wmatdp, int32_t lfpi, int32_t lpol,
                  double *betrms, double *pharms, int32_t *npol);

/* ---------------------------------------------------------------------
 * Batches of independent instances (no reference counterpart: CRMod runs
 * one tomodir per process).  Each instance is its own context (mesh,
 * survey, precision); a batch runs the forward of every instance -- and,
 * with jacobian_mode >= 0, its Jacobian (0 bsensi, 1 bsendc, 2 bsens) --
 * as one CUDA graph in which the instances are independent branches.
 * The first crt_batch_run runs every instance once eagerly (allocating
 * workspaces and autotuning the band panel width per precision and mb),
 * then captures and replays the graph; later runs replay it.  The contexts
 * must live on one device and outlive the batch, and may not be used by
 * other calls while the batch runs.  ms receives the device time of the
 * replay.  The results stay on the device in each context as its last
 * forward (and Jacobian), which later calls on that context use;
 * crt_batch_results copies them out. */
typedef struct crt_batch crt_batch;
crt_batch *crt_batch_create(crt_ctx *const *ctxs, int32_t count, int32_t ldc, int32_t jacobian_mode,
                            int32_t *err);
void crt_batch_destroy(crt_batch *b);
const char *crt_batch_error(const crt_batch *b);
/* sigma[i]: complex conductivity of instance i (E_i interleaved pairs). */
int32_t crt_batch_set_models(crt_batch *b, const double *const *sigma);
int32_t crt_batch_run(crt_batch *b, double *ms);
/* errnr of instance i in the last run (0 = ok). */
int32_t crt_batch_status(const crt_batch *b, int32_t i);
/* volt / sigmaa: [N_i] complex; sens: [N_i, E_i] as crt_jacobian (NULL skips). */
int32_t crt_batch_results(crt_batch *b, int32_t i, double *volt, double *sigmaa, double *sens);
/* Upper bound of a context's band-factor workspace in bytes (0: default);
 * the forward is chunked to fit.  Meant for batches, whose contexts hold
 * their workspaces side by side. */
int32_t crt_set_workspace_limit(crt_ctx *ctx, int64_t bytes);

#ifdef __cplusplus
}
#endif
#endif /* CRT_B200_H */
