// crt_api.cu -- the C ABI (include/crt_b200.h): context, uploads, the
// forward / Jacobian / update drivers and the Gauss-Newton step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/crt_b200.h"
#include "crt_band.h"
#include "crt_cg.h"
#include "crt_common.cuh"
#include "crt_schur.h"
#include "crt_sens.h"
#include "crt_setup.h"
#include "crt_spc.h"
#include "crt_gnn.h"
#include "crt_volt.h"

template <typename T> void launch_band_solve_with_scratch(const SolveArgs<T>&, T*, cudaStream_t);

struct crt_ctx {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[10] = {};
    double timings[CRT_NTIMINGS] = {};
    int64_t launches = 0;
    std::string err;

    // sizes
    int n = 0, mb = 0, W = 0, E = 0, R = 0, ntot = 0, maxnodes = 0, nmn = 0;
    int L = 0, N = 0, K = 0, swrtr = 1;
    int lbeta = 0, lrandb = 0, lrandb2 = 0, lsink = 0, nsink = 0;
    int nkmax = 0;
    double pi = 0.0;

    // host copies
    std::vector<double> kwnwi_h, kwn_h;
    std::vector<int> strnr_h, vnr_h;

    // device mesh / survey
    int *d_nrel0 = nullptr, *d_snr0 = nullptr, *d_etyp = nullptr, *d_enk = nullptr;
    int *d_enr0 = nullptr, *d_mixed_rel = nullptr, *d_strnr = nullptr, *d_vnr = nullptr;
    int4* d_elec = nullptr;
    double *d_sx = nullptr, *d_sy = nullptr, *d_kwn = nullptr, *d_kwnwi = nullptr;
    double *d_elbg = nullptr, *d_relbg = nullptr, *d_kg = nullptr;
    int *d_row_ptr = nullptr, *d_ent_d = nullptr, *d_ent_ptr = nullptr, *d_con_code = nullptr,
        *d_con_sig = nullptr;
    // entries above the diagonal of every row r: (entry e of row c > r with
    // offset c - r, row c), for the FP64 residual of the refinement
    int *d_up_ptr = nullptr, *d_up_ent = nullptr, *d_up_row = nullptr;
    int nent_rows = 0;         // gather entries per system (row_ptr[n])
    cd* d_aval = nullptr;      // [chunk][nent_rows] prepared FP64 entries (mixed form)
    size_t aval_chunk = 0;
    // iterative refinement of the complex64 forward: at most nref steps; a
    // system stops once its componentwise backward error is at most ref_tau
    int nref = 8;
    double ref_tau = 1e-14;
    unsigned long long* d_omega = nullptr;   // [2 steps][chunk * L][2] backward-error maxima
    size_t omega_cap = 0;
    unsigned char* d_dflag = nullptr;
    cd* d_dval = nullptr;
    // randb2 right-hand-side moves of non-zero boundary.dat values: the rows
    // coupled to such a node, per row the gather entries and the nodes
    // (CSR), and the per-system moves of the current chunk [chunk][n]
    int ndc_rows = 0;
    int *d_dc_rows = nullptr, *d_dc_ptr = nullptr, *d_dc_ent = nullptr, *d_dc_node = nullptr;
    cd* d_bdir = nullptr;
    size_t bdir_chunk = 0;
    int* d_status = nullptr;    // [max(K*L, K) + 8] per-system errnr; [last] global
    int nstatus = 0;

    // forward state
    cd *d_sigma = nullptr, *d_kpot = nullptr, *d_kpt = nullptr, *d_volt = nullptr,
       *d_sigmaa = nullptr, *d_hel = nullptr;
    int last_ldc = 0, have_forward = 0;
    // band workspaces (chunked)
    void* d_Lws = nullptr;
    void* d_yws = nullptr;
    double* d_fakws = nullptr;
    void* d_scratch = nullptr;
    size_t lws_slot_bytes = 0;
    int chunk = 0;

    // Jacobian / inversion state
    void* d_sens = nullptr;
    int sens_real = 0, have_sens = 0;
    cd* d_part_sens = nullptr;
    double* d_strom = nullptr;
    int ltri = -1, nx = 0, nnb = 0;
    double* d_smatm = nullptr;
    int* d_nachbar = nullptr;
    cd* d_dat = nullptr;
    double* d_wd = nullptr;
    double *d_cgfac = nullptr, *d_cgres = nullptr, *d_bdpar = nullptr;
    cd *d_rhs = nullptr, *d_p = nullptr, *d_r = nullptr, *d_bvec = nullptr, *d_dpar = nullptr,
       *d_ap = nullptr, *d_cgpart = nullptr, *d_par = nullptr, *d_par_backup = nullptr;
    CGState* d_cgst = nullptr;
    int cg_nsplit = 1, cg_ncgmax_alloc = 0;
    // block preconditioner of the CG (built with the regulariser)
    SpcPlan spc;
    std::string spc_why;
    cd *d_z = nullptr, *d_rold = nullptr, *d_zb = nullptr;
    CGState* d_live = nullptr;   // a never-done CG state for preconditioner applications outside the CG
    double* d_vred = nullptr;    // partial sums of the CG head and tail
    cd* d_sfac = nullptr;        // per-reading factors of the Gram-form Jacobian
    // the forward sweep concurrent with the interior factor: the factor's
    // progress per wavenumber and its count of started CTAs, the stream and
    // the fork / join events
    int* d_fprog = nullptr;
    cudaStream_t ovl_st = nullptr;
    cudaEvent_t ovl_ev[2] = {};
    // fused matvec of the CG (k_cg_fused): reduction ring, tickets, error word
    unsigned char* d_cgf = nullptr;
    size_t cgf_bytes = 0;
    int cgf_grid = 0;
    // lambda candidates side by side (crt_update_lambdas): one slab for all
    // candidates' vectors, grown on demand
    unsigned char* d_cgl = nullptr;
    size_t cgl_bytes = 0;
    // block form of the batch: each candidate's preconditioner factor
    // buffers, and streams on which the candidates' one-CTA factor and
    // sweep kernels run side by side
    std::vector<SpcPlan> spc_c;
    cudaStream_t cstr[CGL_MAX] = {};
    cudaEvent_t cev_fork = nullptr;
    cudaEvent_t cev_join[CGL_MAX] = {};
    int cg_form = 0;      // form of the last CG: CRT_PRECOND_*
    // learned correction of the preconditioner
    Gnn gnn;
    int gnn_guard = 0;   // the last solve switched the learned correction off
    int prec = CRT_PREC_FP64;
    // enqueue-only pass (stream capture into a batch graph): no host
    // synchronisation, no timing reads, no allocation, status read later
    int capture = 0;
    size_t ws_budget = 0;   // factor workspace budget in bytes (0: default)
    int panel = 0;          // panel width of the last blocked factorisation
    // timing events of the forward, read after the forward's one host
    // synchronisation (the status read) instead of one wait per phase
    std::vector<cudaEvent_t> tev;
    int tev_n = 0;
    struct FwdMark {
        int e0, e8, e1, e2;            // chunk start, after preparation, after factor, end
        bool blk;
        std::vector<int> ref;          // per refinement step: residual start, solve start, end
    };
    std::vector<FwdMark> fwd_marks;
    int vol_e0 = -1, vol_e1 = -1;
    // forward by elimination of the mixed-boundary nodes (crt_schur.cu):
    // the plan (host and device), its workspaces and the phase events of the
    // last run
    int fwd_form = CRT_FORWARD_AUTO;
    int schur_ok = 0, schur_used = 0;
    SchurHost schur_h;
    SchurArgs schur{};
    std::vector<void*> schur_bufs;    // plan arrays
    int *d_sI_row_ptr = nullptr, *d_sI_ent_d = nullptr, *d_sI_ent_ptr = nullptr, *d_sI_con_code = nullptr,
        *d_sI_con_sig = nullptr;
    unsigned char* d_sI_dflag = nullptr;
    void *d_sLI = nullptr, *d_sLrev = nullptr, *d_sX = nullptr, *d_sC = nullptr, *d_sS = nullptr, *d_sxg = nullptr,
         *d_scval = nullptr, *d_sS0 = nullptr, *d_sDv = nullptr;
    double* d_sfak = nullptr;
    int* d_snonconv = nullptr;   // systems the iterative Schur solve did not converge on
    int sS_chunk = 0;
    double schur_iter_mean = 0;  // the last Schur forward's iterations per electrode system (0: the Cholesky)
    int sev[5] = {-1, -1, -1, -1, -1};   // after the forward sweep, the Gram products, the Cholesky, the back sweep
};

namespace {

bool ck(crt_ctx* c, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return true;
    c->err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

#define CK(call)                                   \
    do {                                           \
        if (!ck(ctx, (call), #call)) return CRT_ERR_CUDA; \
    } while (0)

template <typename T>
bool dalloc(crt_ctx* ctx, T** p, size_t count)
{
    if (*p) {
        cudaFree(*p);
        *p = nullptr;
    }
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) {
        ctx->err = std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) + " bytes: " +
                   cudaGetErrorString(e);
        *p = nullptr;
        return false;
    }
    return true;
}

template <typename T>
bool upload(crt_ctx* ctx, T** p, const T* h, size_t count)
{
    if (!dalloc(ctx, p, count)) return false;
    if (count && h) return ck(ctx, cudaMemcpyAsync(*p, h, count * sizeof(T), cudaMemcpyHostToDevice, ctx->st), "upload");
    return true;
}

int set_err(crt_ctx* ctx, int code, const std::string& msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

// First non-zero per-system status (the reference stops at the first error).
int collect_status(crt_ctx* ctx, int count)
{
    if (ctx->capture) return CRT_OK;
    std::vector<int> h(count);
    if (!ck(ctx, cudaMemcpyAsync(h.data(), ctx->d_status, sizeof(int) * count, cudaMemcpyDeviceToHost, ctx->st),
            "status copy"))
        return CRT_ERR_CUDA;
    if (!ck(ctx, cudaStreamSynchronize(ctx->st), "stream sync")) return CRT_ERR_CUDA;
    for (int i = 0; i < count; ++i)
        if (h[i]) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "device status %d in system %d", h[i], i);
            ctx->err = buf;
            return h[i];
        }
    return CRT_OK;
}

int kernel_check(crt_ctx* ctx, const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(ctx, CRT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return CRT_OK;
}

// Phase timing by the context's events; a captured pass records and reads
// nothing.
bool ev_rec(crt_ctx* ctx, int i) { return ctx->capture || ck(ctx, cudaEventRecord(ctx->ev[i], ctx->st), "event record"); }
bool ev_sync(crt_ctx* ctx, int i) { return ctx->capture || ck(ctx, cudaEventSynchronize(ctx->ev[i]), "event sync"); }
float ev_ms(crt_ctx* ctx, int a, int b)
{
    float ms = 0.0f;
    if (!ctx->capture) cudaEventElapsedTime(&ms, ctx->ev[a], ctx->ev[b]);
    return ms;
}

// A pooled timing event recorded on the context stream (-1 while capturing).
int tev_rec(crt_ctx* ctx)
{
    if (ctx->capture) return -1;
    if (ctx->tev_n == (int)ctx->tev.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return -1;
        ctx->tev.push_back(e);
    }
    if (cudaEventRecord(ctx->tev[ctx->tev_n], ctx->st) != cudaSuccess) return -1;
    return ctx->tev_n++;
}
float tev_ms(crt_ctx* ctx, int a, int b)
{
    float ms = 0.0f;
    if (a >= 0 && b >= 0) cudaEventElapsedTime(&ms, ctx->tev[a], ctx->tev[b]);
    return ms;
}

size_t sens_elem_bytes(const crt_ctx* ctx, bool real)
{
    const bool f32 = ctx->prec == CRT_PREC_MIXED;
    if (real) return f32 ? sizeof(float) : sizeof(double);
    return f32 ? sizeof(cf) : sizeof(cd);
}

// Workspace chunk: how many band systems are factored per launch.
int plan_chunk(crt_ctx* ctx, int nsys, size_t tsize)
{
    const size_t slot = (size_t)ctx->n * ctx->W * tsize;
    size_t budget = (size_t)48 << 30;
    if (const char* env = std::getenv("CRT_B200_WORKSPACE_GB")) budget = (size_t)(std::atof(env) * (1u << 30));
    if (ctx->ws_budget) budget = std::min(budget, ctx->ws_budget);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) budget = std::min(budget, free_b / 2);
    int c = (int)std::max<size_t>(1, budget / std::max<size_t>(slot + (size_t)ctx->n * (tsize + 8), 1));
    // one factor CTA per SM (the window fills the shared memory): round the
    // chunk down to whole waves so no wave runs part-empty
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    if (c >= nsm && c < nsys) c = (c / nsm) * nsm;
    return std::min(c, nsys);
}

bool upload_upper_lists(crt_ctx* ctx, const AssemblyLists& lists)
{
    const int n = (int)lists.row_ptr.size() - 1;
    std::vector<int> cnt(n + 1, 0);
    for (int c = 0; c < n; ++c)
        for (int e = lists.row_ptr[c]; e < lists.row_ptr[c + 1]; ++e)
            if (lists.ent_d[e] > 0) cnt[c - lists.ent_d[e] + 1]++;
    for (int r = 0; r < n; ++r) cnt[r + 1] += cnt[r];
    std::vector<int> ue(cnt[n]), ur(cnt[n]), fill(cnt.begin(), cnt.end() - 1);
    for (int c = 0; c < n; ++c)
        for (int e = lists.row_ptr[c]; e < lists.row_ptr[c + 1]; ++e)
            if (lists.ent_d[e] > 0) {
                const int r = c - lists.ent_d[e];
                ue[fill[r]] = e;
                ur[fill[r]] = c;
                fill[r]++;
            }
    return upload(ctx, &ctx->d_up_ptr, cnt.data(), cnt.size()) && upload(ctx, &ctx->d_up_ent, ue.data(), ue.size()) &&
           upload(ctx, &ctx->d_up_row, ur.data(), ur.size());
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" int32_t crt_abi_version(void) { return CRT_B200_ABI_VERSION; }

extern "C" const char* crt_last_error(const crt_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

extern "C" int64_t crt_launch_count(const crt_ctx* ctx) { return ctx ? ctx->launches : 0; }

extern "C" int32_t crt_cg_info(const crt_ctx* ctx, int32_t* form, int32_t* block, int32_t* bandwidth)
{
    if (!ctx) return CRT_ERR_ARG;
    if (form) *form = ctx->cg_form;
    if (block) *block = ctx->spc.ok ? ctx->spc.B : 0;
    if (bandwidth) *bandwidth = ctx->spc.bw;
    return CRT_OK;
}

extern "C" int32_t crt_last_timings(const crt_ctx* ctx, double* ms7)
{
    if (!ctx || !ms7) return CRT_ERR_ARG;
    for (int i = 0; i < 7; ++i) ms7[i] = ctx->timings[i];
    return CRT_OK;
}

extern "C" int32_t crt_set_refinement(crt_ctx* ctx, int32_t steps)
{
    if (!ctx || steps < 0 || steps > 16) return CRT_ERR_ARG;
    ctx->nref = steps;
    return CRT_OK;
}

extern "C" int32_t crt_set_refinement_tol(crt_ctx* ctx, double tau)
{
    if (!ctx || !(tau >= 0.0) || !(tau < 1.0)) return CRT_ERR_ARG;
    ctx->ref_tau = tau;
    return CRT_OK;
}

extern "C" int32_t crt_set_forward_form(crt_ctx* ctx, int32_t form)
{
    if (!ctx) return CRT_ERR_ARG;
    if (form != CRT_FORWARD_AUTO && form != CRT_FORWARD_DIRECT && form != CRT_FORWARD_SCHUR)
        return set_err(ctx, CRT_ERR_ARG, "unknown forward form");
    if (form == CRT_FORWARD_SCHUR && !ctx->schur_ok)
        return set_err(ctx, CRT_ERR_UNSUPPORTED,
                       "the Schur form needs mixed boundaries, no Dirichlet nodes and at most 768 boundary nodes");
    ctx->fwd_form = form;
    return CRT_OK;
}

extern "C" int32_t crt_forward_info(const crt_ctx* ctx, int32_t* form, int32_t* nboundary, int32_t* ninterior,
                                    int32_t* mb_interior)
{
    if (!ctx) return CRT_ERR_ARG;
    if (form) *form = ctx->have_forward ? (ctx->schur_used ? CRT_FORWARD_SCHUR : CRT_FORWARD_DIRECT) : CRT_FORWARD_AUTO;
    if (nboundary) *nboundary = ctx->schur_ok ? ctx->schur_h.m : 0;
    if (ninterior) *ninterior = ctx->schur_ok ? ctx->schur_h.nI : 0;
    if (mb_interior) *mb_interior = ctx->schur_ok ? ctx->schur_h.mbI : 0;
    return CRT_OK;
}

extern "C" int32_t crt_last_timings_ex(const crt_ctx* ctx, double* ms, int32_t n)
{
    if (!ctx || !ms || n < 0) return CRT_ERR_ARG;
    for (int i = 0; i < n && i < CRT_NTIMINGS; ++i) ms[i] = ctx->timings[i];
    return CRT_OK;
}

extern "C" int32_t crt_rwaven(const crt_mesh* mesh, int32_t eanz, const int32_t* enr, int32_t nanz,
                              const int32_t* strnr, const int32_t* vnr, int32_t* kwnanz, double* kwn,
                              double* kwnwi)
{
    (void)eanz;
    if (!mesh || !enr || !strnr || !vnr || !kwnanz || !kwn || !kwnwi) return CRT_ERR_ARG;
    return crt_rwaven_host(nanz, strnr, vnr, enr, mesh->snr, mesh->sx, mesh->sy, kwnanz, kwn, kwnwi, nullptr,
                           nullptr);
}

extern "C" void crt_destroy(crt_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    for (void* p : ctx->schur_bufs)
        if (p) cudaFree(p);
    void* sws[] = {ctx->d_sLI, ctx->d_sLrev, ctx->d_sX, ctx->d_sC, ctx->d_sS, ctx->d_sxg, ctx->d_scval, ctx->d_sfak,
                   ctx->d_sS0, ctx->d_sDv, ctx->d_snonconv};
    for (void* p : sws)
        if (p) cudaFree(p);
    void* ptrs[] = {ctx->d_nrel0, ctx->d_snr0, ctx->d_etyp, ctx->d_enk, ctx->d_enr0, ctx->d_mixed_rel,
                    ctx->d_strnr, ctx->d_vnr, ctx->d_elec, ctx->d_sx, ctx->d_sy, ctx->d_kwn, ctx->d_kwnwi,
                    ctx->d_elbg, ctx->d_relbg, ctx->d_kg, ctx->d_row_ptr, ctx->d_ent_d, ctx->d_ent_ptr,
                    ctx->d_con_code, ctx->d_con_sig, ctx->d_up_ptr, ctx->d_up_ent, ctx->d_up_row, ctx->d_aval, ctx->d_dflag, ctx->d_dval, ctx->d_status, ctx->d_sigma,
                    ctx->d_kpot, ctx->d_kpt, ctx->d_volt, ctx->d_sigmaa, ctx->d_hel, ctx->d_Lws, ctx->d_yws,
                    ctx->d_fakws, ctx->d_scratch, ctx->d_sens, ctx->d_part_sens, ctx->d_strom, ctx->d_smatm,
                    ctx->d_nachbar, ctx->d_dat, ctx->d_wd, ctx->d_cgfac, ctx->d_cgres, ctx->d_bdpar,
                    ctx->d_rhs, ctx->d_p, ctx->d_r, ctx->d_bvec, ctx->d_dpar, ctx->d_ap, ctx->d_cgpart,
                    ctx->d_par, ctx->d_par_backup, ctx->d_cgst, ctx->d_z, ctx->d_rold, ctx->d_zb, ctx->d_live, ctx->d_cgl, ctx->d_omega, ctx->d_cgf, ctx->d_vred, ctx->d_sfac, ctx->d_fprog,
                    ctx->d_dc_rows, ctx->d_dc_ptr, ctx->d_dc_ent, ctx->d_dc_node, ctx->d_bdir};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (SpcPlan& c : ctx->spc_c) spc_plan_free_clone(c);
    spc_plan_free(ctx->spc);
    if (ctx->ovl_st) cudaStreamDestroy(ctx->ovl_st);
    for (cudaEvent_t e : ctx->ovl_ev)
        if (e) cudaEventDestroy(e);
    for (int b = 0; b < CGL_MAX; ++b) {
        if (ctx->cstr[b]) cudaStreamDestroy(ctx->cstr[b]);
        if (ctx->cev_join[b]) cudaEventDestroy(ctx->cev_join[b]);
    }
    if (ctx->cev_fork) cudaEventDestroy(ctx->cev_fork);
    gnn_free(ctx->gnn);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->tev) cudaEventDestroy(e);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
}

extern "C" crt_ctx* crt_create(int32_t device, const crt_mesh* mesh, const crt_survey* sv, int32_t precision,
                               int32_t* errnr)
{
    auto fail = [&](crt_ctx* c, int code) -> crt_ctx* {
        if (errnr) *errnr = code;
        if (c && !c->err.empty()) std::fprintf(stderr, "crt_create: %s\n", c->err.c_str());
        crt_destroy(c);
        return nullptr;
    };
    if (errnr) *errnr = CRT_OK;
    if (!mesh || !sv) return fail(nullptr, CRT_ERR_ARG);
    if (precision != CRT_PREC_FP64 && precision != CRT_PREC_MIXED) return fail(nullptr, CRT_ERR_UNSUPPORTED);
    crt_ctx* ctx = new crt_ctx();
    ctx->prec = precision;
    ctx->device = device;
    ctx->pi = std::acos(-1.0);
    if (!ck(ctx, cudaSetDevice(device), "cudaSetDevice")) return fail(ctx, CRT_ERR_CUDA);
    if (!ck(ctx, cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking), "stream")) return fail(ctx, CRT_ERR_CUDA);
    for (auto& e : ctx->ev)
        if (!ck(ctx, cudaEventCreate(&e), "event")) return fail(ctx, CRT_ERR_CUDA);

    // ---- mesh
    MeshHost m{};
    m.sanz = mesh->sanz;
    m.mb = mesh->mb;
    m.typanz = mesh->typanz;
    m.typ = mesh->typ;
    m.nelanz = mesh->nelanz;
    m.selanz = mesh->selanz;
    m.nrel = mesh->nrel;
    m.rnr = mesh->rnr;
    m.snr = mesh->snr;
    m.sx = mesh->sx;
    m.sy = mesh->sy;
    m.elanz = m.relanz = m.maxnodes = 0;
    for (int t = 0; t < m.typanz; ++t) {
        if (m.typ[t] > 10) m.relanz += m.nelanz[t];
        else m.elanz += m.nelanz[t];
        m.maxnodes = std::max(m.maxnodes, (int)m.selanz[t]);
    }
    m.ntot = m.elanz + m.relanz;
    ctx->n = m.sanz;
    ctx->mb = m.mb;
    ctx->W = m.mb + 1;
    ctx->E = m.elanz;
    ctx->R = m.relanz;
    ctx->ntot = m.ntot;
    ctx->maxnodes = m.maxnodes;
    ctx->nmn = m.maxnodes * (m.maxnodes + 1) / 2;
    ctx->L = sv->eanz;
    ctx->N = sv->nanz;
    ctx->K = sv->kwnanz;
    ctx->swrtr = sv->swrtr;
    ctx->lsink = sv->lsink;
    ctx->nsink = sv->nsink;
    if (ctx->n <= 0 || ctx->E <= 0 || ctx->L <= 0 || ctx->K <= 0 || m.maxnodes > 4)
        return fail(ctx, set_err(ctx, CRT_ERR_ARG, "empty mesh / survey or element with > 4 nodes"));
    if (band_factor_smem<cd>(ctx->W) > 227 * 1024)
        return fail(ctx, set_err(ctx, CRT_ERR_UNSUPPORTED, "half bandwidth too large for the FP64 window"));

    // element table: 0-based nodes, types, node counts, boundary flags
    std::vector<int> nrel0((size_t)m.ntot * m.maxnodes, 0);
    {
        // area elements must precede the boundary segments (the reference's
        // sigma(iel) and nrel(elanz + rel, .) indexing relies on it)
        bool seen_boundary = false;
        for (int t = 0; t < m.typanz; ++t) {
            if (m.typ[t] > 10) seen_boundary = true;
            else if (seen_boundary)
                return fail(ctx, set_err(ctx, CRT_ERR_ARG, "area element types listed after boundary types"));
        }
    }
    std::vector<int> et(m.elanz), enk(m.elanz), mixed_rel;
    std::vector<unsigned char> dflag(ctx->n, 0), t13(ctx->n, 0);
    std::vector<cd> dval(ctx->n, cd{0.0, 0.0});
    {
        int row = 0;
        for (int t = 0; t < m.typanz; ++t)
            for (int j = 0; j < m.nelanz[t]; ++j, ++row) {
                for (int q = 0; q < m.selanz[t]; ++q) {
                    int node = m.nrel[(size_t)q * m.ntot + row];
                    if (node < 1 || node > m.sanz)
                        return fail(ctx, set_err(ctx, CRT_ERR_ARG, "node number out of range in nrel"));
                    nrel0[(size_t)row * m.maxnodes + q] = node - 1;
                }
                if (m.typ[t] <= 10) {
                    et[row] = m.typ[t];
                    enk[row] = m.selanz[t];
                    ctx->nkmax = std::max(ctx->nkmax, (int)m.selanz[t]);
                } else if (m.typ[t] == 11) {
                    ctx->lbeta = 1;
                    const int rel = row - m.elanz;
                    if (m.rnr[rel] < 1 || m.rnr[rel] > m.elanz)
                        return fail(ctx, set_err(ctx, 111, "border to element context is wrong (errnr 111)"));
                    mixed_rel.push_back(rel);
                } else if (m.typ[t] == 13) {
                    ctx->lrandb = 1;
                    for (int q = 0; q < m.selanz[t]; ++q) {
                        const int node = m.nrel[(size_t)q * m.ntot + row] - 1;
                        dflag[node] = 1;
                        t13[node] = 1;
                    }
                }
            }
    }
    if (ctx->lbeta && ctx->lrandb)
        return fail(ctx, set_err(ctx, 101, "mixed boundary and Dirichlet elements together (errnr 101)"));
    if (sv->rwdanz > 0) {
        ctx->lrandb2 = 1;
        for (int i = 0; i < sv->rwdanz; ++i) {
            int node = sv->rwdnr[i] - 1;
            if (node < 0 || node >= ctx->n)
                return fail(ctx, set_err(ctx, CRT_ERR_ARG, "boundary.dat node number out of range"));
            dflag[node] = 2;
            dval[node] = cd{sv->rwd[2 * i], sv->rwd[2 * i + 1]};
        }
    }
    AssemblyLists lists;
    int e = build_assembly_lists(m, lists);
    if (e) return fail(ctx, set_err(ctx, e, "band width violated in kompab (errnr 19)"));
    // randb2 (src/randb2.f90:39-79): a free row r coupled to a boundary.dat
    // node c with a non-zero value receives value(c) a(r, c) on its right-hand
    // side.  randb runs first and has zeroed the rows and columns of the
    // type-13 nodes, so a boundary.dat node that is also a type-13 node
    // couples to nothing, and type-13 rows keep b = 0.
    std::vector<int> dc_rows, dc_ptr(1, 0), dc_ent, dc_node;
    if (ctx->lrandb2) {
        std::vector<std::vector<std::pair<int, int>>> per_row(ctx->n);
        auto coupled = [&](int c) { return dflag[c] == 2 && !t13[c] && (dval[c].x != 0.0 || dval[c].y != 0.0); };
        for (int r = 0; r < ctx->n; ++r)
            for (int q = lists.row_ptr[r]; q < lists.row_ptr[r + 1]; ++q) {
                const int d = lists.ent_d[q];
                if (d == 0) continue;
                const int c = r - d;   // entry (r, c) = (c, r), c < r
                if (dflag[r] == 0 && coupled(c)) per_row[r].push_back({q, c});
                if (dflag[c] == 0 && coupled(r)) per_row[c].push_back({q, r});
            }
        for (int r = 0; r < ctx->n; ++r) {
            if (per_row[r].empty()) continue;
            dc_rows.push_back(r);
            for (auto& pr : per_row[r]) {
                dc_ent.push_back(pr.first);
                dc_node.push_back(pr.second);
            }
            dc_ptr.push_back((int)dc_ent.size());
        }
        ctx->ndc_rows = (int)dc_rows.size();
    }

    std::vector<int> snr0(ctx->n), enr0(ctx->L);
    for (int i = 0; i < ctx->n; ++i) snr0[i] = mesh->snr[i] - 1;
    for (int i = 0; i < ctx->L; ++i) {
        enr0[i] = sv->enr[i] - 1;
        if (enr0[i] < 0 || enr0[i] >= ctx->n) return fail(ctx, set_err(ctx, 29, "electrode node > sanz (errnr 29)"));
    }
    std::vector<int4> elec(ctx->N);
    for (int i = 0; i < ctx->N; ++i) {
        int s = sv->strnr[i], v = sv->vnr[i];
        int e1 = s % 10000, e2 = s / 10000, e3 = v % 10000, e4 = v / 10000;
        if (std::min({e1, e2, e3, e4}) < 0 || std::max({e1, e2, e3, e4}) > ctx->L)
            return fail(ctx, set_err(ctx, 46, "electrode number out of range (errnr 46)"));
        elec[i] = make_int4(e1 - 1, e2 - 1, e3 - 1, e4 - 1);
    }
    ctx->strnr_h.assign(sv->strnr, sv->strnr + ctx->N);
    ctx->vnr_h.assign(sv->vnr, sv->vnr + ctx->N);
    ctx->kwn_h.assign(sv->kwn, sv->kwn + ctx->K);
    ctx->kwnwi_h.assign(sv->kwnwi, sv->kwnwi + ctx->K);

    bool ok = upload(ctx, &ctx->d_nrel0, nrel0.data(), nrel0.size()) &&
              upload(ctx, &ctx->d_snr0, snr0.data(), snr0.size()) &&
              upload(ctx, &ctx->d_etyp, et.data(), et.size()) && upload(ctx, &ctx->d_enk, enk.data(), enk.size()) &&
              upload(ctx, &ctx->d_enr0, enr0.data(), enr0.size()) &&
              upload(ctx, &ctx->d_mixed_rel, mixed_rel.data(), mixed_rel.size()) &&
              upload(ctx, &ctx->d_strnr, sv->strnr, (size_t)ctx->N) && upload(ctx, &ctx->d_vnr, sv->vnr, (size_t)ctx->N) &&
              upload(ctx, &ctx->d_elec, elec.data(), elec.size()) && upload(ctx, &ctx->d_sx, mesh->sx, (size_t)ctx->n) &&
              upload(ctx, &ctx->d_sy, mesh->sy, (size_t)ctx->n) && upload(ctx, &ctx->d_kwn, sv->kwn, (size_t)ctx->K) &&
              upload(ctx, &ctx->d_kwnwi, sv->kwnwi, (size_t)ctx->K) &&
              upload(ctx, &ctx->d_row_ptr, lists.row_ptr.data(), lists.row_ptr.size()) &&
              upload(ctx, &ctx->d_ent_d, lists.ent_d.data(), lists.ent_d.size()) &&
              upload(ctx, &ctx->d_ent_ptr, lists.ent_ptr.data(), lists.ent_ptr.size()) &&
              upload(ctx, &ctx->d_con_code, lists.con_code.data(), lists.con_code.size()) &&
              upload(ctx, &ctx->d_con_sig, lists.con_sig.data(), lists.con_sig.size()) &&
              upload_upper_lists(ctx, lists) && (ctx->nent_rows = lists.row_ptr.back(), true) &&
              upload(ctx, &ctx->d_dflag, dflag.data(), dflag.size()) &&
              upload(ctx, &ctx->d_dval, dval.data(), dval.size());
    if (ok && ctx->ndc_rows > 0)
        ok = upload(ctx, &ctx->d_dc_rows, dc_rows.data(), dc_rows.size()) &&
             upload(ctx, &ctx->d_dc_ptr, dc_ptr.data(), dc_ptr.size()) &&
             upload(ctx, &ctx->d_dc_ent, dc_ent.data(), dc_ent.size()) &&
             upload(ctx, &ctx->d_dc_node, dc_node.data(), dc_node.size());
    if (!ok) return fail(ctx, CRT_ERR_ALLOC);
    // Schur form of the forward: mixed boundaries without Dirichlet nodes;
    // the boundary set is every node of a type-11 segment
    if (ctx->lbeta && !ctx->lrandb && !ctx->lrandb2) {
        std::vector<int> gnodes;
        for (int rel : mixed_rel)
            for (int q = 0; q < 2; ++q) gnodes.push_back(nrel0[(size_t)(m.elanz + rel) * m.maxnodes + q]);
        SchurHost& H = ctx->schur_h;
        // forward-sweep column blocks: 16 columns (two CTAs per SM with the
        // rows one block ahead: 11.0 ms after the factor on the 60k-triangle
        // mesh) or 32 (one CTA per SM, 11.7 ms; CRT_B200_SCHUR_R=32)
        // (16 also where the 32-column block's buffers exceed shared memory)
        const char* rv = std::getenv("CRT_B200_SCHUR_R");
        int sweep_r = (rv && std::strcmp(rv, "32") == 0) ? SCHUR_MS_R : 16;
        int plan_e = schur_plan_host(lists, ctx->n, gnodes, enr0, ctx->lsink, ctx->nsink - 1, H, sweep_r);
        if (plan_e == CRT_OK && sweep_r != 16 && schur_sweep_smem<cd>(H.mbI, H.mbI + 1, sweep_r) > 227 * 1024) {
            sweep_r = 16;
            H = SchurHost{};
            plan_e = schur_plan_host(lists, ctx->n, gnodes, enr0, ctx->lsink, ctx->nsink - 1, H, sweep_r);
        }
        if (plan_e == CRT_OK &&
            schur_sweep_smem<cd>(H.mbI, H.mbI + 1, sweep_r) <= 227 * 1024 &&
            (size_t)(16 + 1) * H.m * sizeof(cd) <= 227 * 1024 && band_factor_smem<cd>(H.mbI + 1) <= 227 * 1024) {
            auto up = [&](int** d, const std::vector<int>& v) {
                const std::vector<int> one(1, 0);
                const std::vector<int>& src = v.empty() ? one : v;
                if (!upload(ctx, d, src.data(), src.size())) return false;
                ctx->schur_bufs.push_back(*d);
                return true;
            };
            SchurArgs& S = ctx->schur;
            int *p_permI = nullptr, *p_gam = nullptr, *p_pis = nullptr, *p_pgs = nullptr, *p_gip = nullptr,
                *p_gipos = nullptr, *p_gient = nullptr, *p_gig = nullptr, *p_ggg = nullptr, *p_ggh = nullptr,
                *p_gge = nullptr, *p_co = nullptr, *p_bs = nullptr, *p_first = nullptr, *p_gsort = nullptr,
                *p_gfirst = nullptr, *p_bdp = nullptr, *p_bdc = nullptr, *p_bde = nullptr;
            const AssemblyLists& li = H.lists_I;
            std::vector<unsigned char> zf(H.nI, 0);
            bool su = up(&p_permI, H.permI) && up(&p_gam, H.gam) && up(&p_pis, H.posI_src) && up(&p_pgs, H.posG_src) &&
                      up(&p_gip, H.gi_ptr) && up(&p_gipos, H.gi_pos) && up(&p_gient, H.gi_ent) && up(&p_gig, H.gi_g) &&
                      up(&p_ggg, H.gg_g) && up(&p_ggh, H.gg_h) && up(&p_gge, H.gg_ent) && up(&p_co, H.col_order) &&
                      up(&p_bs, H.blk_start) && up(&p_first, H.first) && up(&p_gsort, H.gsort) &&
                      up(&p_gfirst, H.gfirst) && up(&p_bdp, H.bd_ptr) && up(&p_bdc, H.bd_col) && up(&p_bde, H.bd_ent) &&
                      up(&ctx->d_sI_row_ptr, li.row_ptr) && up(&ctx->d_sI_ent_d, li.ent_d) &&
                      up(&ctx->d_sI_ent_ptr, li.ent_ptr) && up(&ctx->d_sI_con_code, li.con_code) &&
                      up(&ctx->d_sI_con_sig, li.con_sig) && upload(ctx, &ctx->d_sI_dflag, zf.data(), zf.size());
            if (!su) return fail(ctx, CRT_ERR_ALLOC);
            ctx->schur_bufs.push_back(ctx->d_sI_dflag);
            S.nI = H.nI;
            S.m = H.m;
            S.L = ctx->L;
            S.K = ctx->K;
            S.ncol = ctx->L + H.m;
            S.mbI = H.mbI;
            S.nblk = (int)H.blk_start.size();
            S.R = H.R;
            S.ncpl = (int)H.gi_pos.size();
            S.ngg = (int)H.gg_ent.size();
            S.permI = p_permI;
            S.gam = p_gam;
            S.posI_src = p_pis;
            S.posG_src = p_pgs;
            S.posI_sink = H.posI_sink;
            S.posG_sink = H.posG_sink;
            S.lsink = ctx->lsink;
            S.gi_ptr = p_gip;
            S.gi_pos = p_gipos;
            S.gi_ent = p_gient;
            S.gi_g = p_gig;
            S.gg_g = p_ggg;
            S.gg_h = p_ggh;
            S.gg_ent = p_gge;
            S.col_order = p_co;
            S.blk_start = p_bs;
            S.first = p_first;
            S.gsort = p_gsort;
            S.gfirst = p_gfirst;
            S.bd_ptr = p_bdp;
            S.bd_col = p_bdc;
            S.bd_ent = p_bde;
            S.grp = 0;
            S.ngrp = 0;
            ctx->schur_ok = 1;
        }
    }
    ctx->nstatus = std::max(ctx->K * ctx->L, ctx->K) + 8;
    if (!dalloc(ctx, &ctx->d_status, (size_t)ctx->nstatus)) return fail(ctx, CRT_ERR_ALLOC);
    if (!ck(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int) * ctx->nstatus, ctx->st), "memset")) return fail(ctx, CRT_ERR_CUDA);

    // ---- precal: elbg [K][E][nmn], relbg [R][3], kg [K][L][R]
    const size_t n_elbg = (size_t)ctx->K * ctx->E * ctx->nmn;
    const size_t n_kg = (size_t)ctx->K * ctx->L * std::max(ctx->R, 1);
    if (!dalloc(ctx, &ctx->d_elbg, n_elbg) || !dalloc(ctx, &ctx->d_relbg, (size_t)std::max(ctx->R, 1) * 3) ||
        !dalloc(ctx, &ctx->d_kg, n_kg))
        return fail(ctx, CRT_ERR_ALLOC);
    cudaMemsetAsync(ctx->d_relbg, 0, sizeof(double) * std::max(ctx->R, 1) * 3, ctx->st);
    cudaMemsetAsync(ctx->d_kg, 0, sizeof(double) * n_kg, ctx->st);
    if (sv->elbg) {
        // Fortran elbg(elanz, nmn, kwnanz) -> [K][E][nmn]
        std::vector<double> h(n_elbg);
        for (int k = 0; k < ctx->K; ++k)
            for (int q = 0; q < ctx->nmn; ++q)
                for (int el = 0; el < ctx->E; ++el)
                    h[((size_t)k * ctx->E + el) * ctx->nmn + q] = sv->elbg[((size_t)k * ctx->nmn + q) * ctx->E + el];
        if (!ck(ctx, cudaMemcpyAsync(ctx->d_elbg, h.data(), sizeof(double) * n_elbg, cudaMemcpyHostToDevice, ctx->st), "elbg"))
            return fail(ctx, CRT_ERR_CUDA);
        if (ctx->R > 0 && sv->relbg && sv->kg) {
            std::vector<double> hr((size_t)ctx->R * 3), hk(n_kg);
            for (int q = 0; q < 3; ++q)
                for (int r = 0; r < ctx->R; ++r) hr[(size_t)r * 3 + q] = sv->relbg[(size_t)q * ctx->R + r];
            std::memcpy(hk.data(), sv->kg, sizeof(double) * n_kg);   // kg(R, L, K) is already [K][L][R]
            if (!ck(ctx, cudaMemcpyAsync(ctx->d_relbg, hr.data(), sizeof(double) * hr.size(), cudaMemcpyHostToDevice, ctx->st), "relbg") ||
                !ck(ctx, cudaMemcpyAsync(ctx->d_kg, hk.data(), sizeof(double) * n_kg, cudaMemcpyHostToDevice, ctx->st), "kg"))
                return fail(ctx, CRT_ERR_CUDA);
        }
        if (!ck(ctx, cudaStreamSynchronize(ctx->st), "sync")) return fail(ctx, CRT_ERR_CUDA);
    } else {
        SetupArgs A{};
        A.E = ctx->E;
        A.R = std::max(ctx->R, 1);
        A.K = ctx->K;
        A.L = ctx->L;
        A.maxnodes = ctx->maxnodes;
        A.nmn = ctx->nmn;
        A.nmixed = (int)mixed_rel.size();
        A.nrel0 = ctx->d_nrel0;
        A.snr0 = ctx->d_snr0;
        A.etyp = ctx->d_etyp;
        A.enk = ctx->d_enk;
        A.enr0 = ctx->d_enr0;
        A.mixed_rel = ctx->d_mixed_rel;
        A.sx = ctx->d_sx;
        A.sy = ctx->d_sy;
        A.kwn = ctx->d_kwn;
        A.sytop = sv->lsytop ? crt_sytop_host(m) : 0.0;
        A.elbg = ctx->d_elbg;
        A.relbg = ctx->d_relbg;
        A.kg = ctx->d_kg;
        A.status = ctx->d_status + ctx->nstatus - 1;
        int64_t t1 = (int64_t)ctx->E * ctx->K;
        k_elem_matrices<<<(unsigned)((t1 + 255) / 256), 256, 0, ctx->st>>>(A);
        ctx->launches++;
        if (A.nmixed > 0) {
            int64_t t2 = (int64_t)A.nmixed * ctx->L * ctx->K;
            k_beta<<<(unsigned)((t2 + 255) / 256), 256, 0, ctx->st>>>(A);
            ctx->launches++;
        }
        if (kernel_check(ctx, "precal kernels")) return fail(ctx, CRT_ERR_CUDA);
        int st = collect_status(ctx, ctx->nstatus);
        if (st) return fail(ctx, st);
    }
    return ctx;
}

extern "C" int32_t crt_precal(crt_ctx* ctx, double* elbg, double* relbg, double* kg, int32_t* lbeta, int32_t* lrandb)
{
    if (!ctx) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    const size_t n_elbg = (size_t)ctx->K * ctx->E * ctx->nmn;
    if (elbg) {
        std::vector<double> h(n_elbg);
        CK(cudaMemcpyAsync(h.data(), ctx->d_elbg, sizeof(double) * n_elbg, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        for (int k = 0; k < ctx->K; ++k)
            for (int q = 0; q < ctx->nmn; ++q)
                for (int el = 0; el < ctx->E; ++el)
                    elbg[((size_t)k * ctx->nmn + q) * ctx->E + el] = h[((size_t)k * ctx->E + el) * ctx->nmn + q];
    }
    if (relbg && ctx->R > 0) {
        std::vector<double> h((size_t)ctx->R * 3);
        CK(cudaMemcpyAsync(h.data(), ctx->d_relbg, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        // relbg(relanz, nmn): only the first three columns are used by 2-node segments
        for (int q = 0; q < ctx->nmn; ++q)
            for (int r = 0; r < ctx->R; ++r) relbg[(size_t)q * ctx->R + r] = q < 3 ? h[(size_t)r * 3 + q] : 0.0;
    }
    if (kg && ctx->R > 0) {
        CK(cudaMemcpyAsync(kg, ctx->d_kg, sizeof(double) * (size_t)ctx->K * ctx->L * ctx->R, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    if (lbeta) *lbeta = ctx->lbeta;
    if (lrandb) *lrandb = ctx->lrandb;
    return CRT_OK;
}

// ---------------------------------------------------------------------------
// Forward.
namespace {

template <typename T>
int run_forward(crt_ctx* ctx)
{
    const int n = ctx->n, L = ctx->L, K = ctx->K;
    // column stride of the factor workspace: mb + 1, rounded up to even for
    // complex64 so every column starts on a 16-byte boundary (the solve's
    // asynchronous block copies need that)
    const int W = std::is_same<T, cf>::value ? (ctx->W + 1) / 2 * 2 : ctx->W;
    const bool mixed = ctx->lbeta != 0;
    const int nfac = mixed ? K * L : K;
    const size_t slot_bytes = (size_t)n * W * sizeof(T);
    int chunk = ctx->capture ? ctx->chunk : plan_chunk(ctx, nfac, sizeof(T));
    if (ctx->capture && (ctx->lws_slot_bytes != slot_bytes || !ctx->d_Lws))
        return set_err(ctx, CRT_ERR_ARG, "captured forward without a prepared workspace");
    // factor workspace
    if (ctx->lws_slot_bytes != slot_bytes || ctx->chunk < chunk || !ctx->d_Lws) {
        if (ctx->d_Lws) cudaFree(ctx->d_Lws);
        if (ctx->d_yws) cudaFree(ctx->d_yws);
        if (ctx->d_fakws) cudaFree(ctx->d_fakws);
        if (ctx->d_scratch) cudaFree(ctx->d_scratch);
        ctx->d_Lws = ctx->d_yws = ctx->d_scratch = nullptr;
        ctx->d_fakws = nullptr;
        CK(cudaMalloc(&ctx->d_Lws, slot_bytes * chunk));
        CK(cudaMalloc(&ctx->d_yws, (size_t)n * sizeof(cd) * chunk));
        CK(cudaMalloc((void**)&ctx->d_fakws, (size_t)n * sizeof(double) * chunk));
        if (!mixed) CK(cudaMalloc(&ctx->d_scratch, (size_t)n * sizeof(cd) * chunk * L));
        ctx->lws_slot_bytes = slot_bytes;
        ctx->chunk = chunk;
    }
    if (std::is_same<T, cf>::value && ctx->omega_cap < (size_t)ctx->chunk * L) {
        if (ctx->capture) return set_err(ctx, CRT_ERR_ARG, "captured forward without a prepared workspace");
        if (ctx->d_omega) cudaFree(ctx->d_omega);
        ctx->d_omega = nullptr;
        ctx->omega_cap = 0;
        CK(cudaMalloc((void**)&ctx->d_omega, 4 * sizeof(unsigned long long) * (size_t)ctx->chunk * L));
        ctx->omega_cap = (size_t)ctx->chunk * L;
    }
    if (ctx->ndc_rows > 0 && ctx->bdir_chunk < (size_t)ctx->chunk) {
        if (ctx->capture) return set_err(ctx, CRT_ERR_ARG, "captured forward without a prepared workspace");
        if (ctx->d_bdir) cudaFree(ctx->d_bdir);
        ctx->d_bdir = nullptr;
        ctx->bdir_chunk = 0;
        CK(cudaMalloc((void**)&ctx->d_bdir, sizeof(cd) * (size_t)n * ctx->chunk));
        // rows without couplings stay zero; the coupled rows are rewritten
        // for every chunk
        CK(cudaMemsetAsync(ctx->d_bdir, 0, sizeof(cd) * (size_t)n * ctx->chunk, ctx->st));
        ctx->bdir_chunk = ctx->chunk;
    }
    chunk = ctx->chunk;
    ctx->tev_n = 0;
    ctx->fwd_marks.clear();
    int nfl = 0;
    bool blk = false;
    for (int s0 = 0; s0 < nfac; s0 += chunk) {
        const int ns = std::min(chunk, nfac - s0);
        BandArgs<T> A{};
        A.n = n;
        A.mb = ctx->mb;
        A.W = W;
        A.sys0 = s0;
        A.nsys = ns;
        A.L = L;
        A.K = K;
        A.mixed = mixed;
        A.fuse_rhs = 1;
        A.E = ctx->E;
        A.R = std::max(ctx->R, 1);
        A.nmn = ctx->nmn;
        A.row_ptr = ctx->d_row_ptr;
        A.ent_d = ctx->d_ent_d;
        A.ent_ptr = ctx->d_ent_ptr;
        A.con_code = ctx->d_con_code;
        A.con_sig = ctx->d_con_sig;
        A.elbg = ctx->d_elbg;
        A.relbg = ctx->d_relbg;
        A.kg = ctx->d_kg;
        A.sigma = ctx->d_sigma;
        A.dflag = ctx->d_dflag;
        A.dval = ctx->d_dval;
        A.bdir = ctx->ndc_rows > 0 ? ctx->d_bdir : nullptr;
        A.enr0 = ctx->d_enr0;
        A.lsink = ctx->lsink;
        A.nsink0 = ctx->nsink - 1;
        A.Lws = static_cast<T*>(ctx->d_Lws);
        A.lstride = (size_t)n * W;
        A.yws = static_cast<T*>(ctx->d_yws);
        A.fakws = ctx->d_fakws;
        A.status = ctx->d_status;
        A.aval = nullptr;
        A.aval_stride = (size_t)ctx->nent_rows;
        if constexpr (std::is_same<T, cf>::value) {
            // the refinement's residual reads the prepared entries in FP64
            if (ctx->aval_chunk < (size_t)chunk) {
                if (!dalloc(ctx, &ctx->d_aval, (size_t)chunk * ctx->nent_rows)) return CRT_ERR_ALLOC;
                ctx->aval_chunk = chunk;
            }
            A.aval = ctx->d_aval;
        }
        crt_ctx::FwdMark mk{};
        mk.e0 = tev_rec(ctx);
        if (ctx->ndc_rows > 0) {
            launch_band_dir_rhs<T>(A, ctx->ndc_rows, ctx->d_dc_rows, ctx->d_dc_ptr, ctx->d_dc_ent, ctx->d_dc_node,
                                   ctx->d_bdir, ctx->st);
            ctx->launches++;
        }
        {
            const char* fv = std::getenv("CRT_B200_FACTOR");
            const bool force_v0 = fv && std::strcmp(fv, "v0") == 0;
            if (!force_v0 && band_blk_fits<T>(ctx->mb)) {
                const int pb = band_panel<T>(A, !ctx->capture, ctx->st);
                ctx->panel = pb & BAND_PANEL_MASK;
                launch_band_prep<T>(A, ctx->st);
                mk.e8 = tev_rec(ctx);
                launch_band_factor_blk<T>(A, pb, ctx->st);
                ctx->launches += 3;
                blk = true;
            } else {
                if constexpr (std::is_same<T, cf>::value) {
                    return set_err(ctx, CRT_ERR_UNSUPPORTED, "complex64 factorisation needs the panel-blocked kernel");
                } else {
                    launch_band_factor<T>(A, ctx->st);
                }
                mk.e8 = tev_rec(ctx);
                ctx->launches++;
                blk = false;
            }
            ++nfl;
        }
        if (int e = kernel_check(ctx, "band factor")) return e;
        mk.e1 = tev_rec(ctx);
        mk.blk = blk;
        SolveArgs<T> S{};
        S.n = n;
        S.mb = ctx->mb;
        S.W = W;
        S.L = L;
        S.mixed = mixed;
        S.lsink = ctx->lsink;
        S.nsink0 = ctx->nsink - 1;
        S.enr0 = ctx->d_enr0;
        S.Lws = A.Lws;
        S.lstride = A.lstride;
        S.fakws = ctx->d_fakws;
        S.yws = A.yws;
        S.kpot = ctx->d_kpot;
        S.status = ctx->d_status;
        T* scr = static_cast<T*>(mixed ? ctx->d_yws : ctx->d_scratch);
        if (mixed) {
            S.sys0 = s0;
            S.nsys = ns;
            S.factor_of_sys_div = 1;
        } else {
            S.sys0 = s0 * L;
            S.nsys = ns * L;
            S.factor_of_sys_div = L;
        }
        launch_band_solve_with_scratch<T>(S, scr, ctx->st);
        ctx->launches++;
        if constexpr (std::is_same<T, cf>::value) {
            // iterative refinement of the complex64 solution: FP64 residual of
            // the scaled system and its componentwise backward error, complex64
            // correction solve, FP64 update of kpot; a system whose backward
            // error has reached ref_tau (the FP64 floor) takes no further steps
            for (int it = 0; it < ctx->nref; ++it) {
                unsigned long long* om_cur = ctx->d_omega + (size_t)(it & 1) * 2 * ctx->omega_cap;
                const unsigned long long* om_prev =
                    it ? ctx->d_omega + (size_t)((it - 1) & 1) * 2 * ctx->omega_cap : nullptr;
                CK(cudaMemsetAsync(om_cur, 0, 2 * sizeof(unsigned long long) * S.nsys, ctx->st));
                mk.ref.push_back(tev_rec(ctx));
                launch_band_residual<T>(A, S.sys0, S.nsys, S.factor_of_sys_div, ctx->d_up_ptr, ctx->d_up_ent,
                                        ctx->d_up_row, ctx->d_kpot, scr, om_prev, om_cur, ctx->ref_tau, ctx->st);
                mk.ref.push_back(tev_rec(ctx));
                SolveArgs<T> C = S;
                C.rhs = scr;
                C.accumulate = 1;
                C.skip_omega = om_cur;
                C.skip_tau = ctx->ref_tau;
                launch_band_solve_with_scratch<T>(C, scr, ctx->st);
                mk.ref.push_back(tev_rec(ctx));
                ctx->launches += 2;
            }
        }
        if (int e = kernel_check(ctx, "band solve")) return e;
        mk.e2 = tev_rec(ctx);
        ctx->fwd_marks.push_back(mk);
    }
    ctx->timings[9] = nfl;
    ctx->timings[12] = blk ? ctx->panel : 0;
    return CRT_OK;   // per-system status and phase times: read by forward_common
}

// Bytes of the Schur form's workspaces (sized for complex128).
size_t schur_bytes(const crt_ctx* ctx, int chunk)
{
    const SchurHost& H = ctx->schur_h;
    const size_t K = ctx->K, L = ctx->L, nI = H.nI, m = H.m;
    return sizeof(cd) * (2 * K * nI * (H.mbI + 2) + K * (L + m) * nI + K * std::max<size_t>(H.gi_pos.size(), 1) +
                         K * (L + m) * m + K * L * m + (size_t)chunk * m * m) +
           sizeof(double) * K * nI;
}

// Whether this forward runs in the Schur form.
bool use_schur(const crt_ctx* ctx)
{
    if (!ctx->schur_ok || ctx->fwd_form == CRT_FORWARD_DIRECT) return false;
    const char* fv = std::getenv("CRT_B200_FORWARD");
    if (fv && std::strcmp(fv, "direct") == 0) return false;
    if (ctx->d_sLI) return true;   // workspaces exist (a captured forward may not allocate)
    const size_t chunk = std::min<size_t>((size_t)ctx->K * ctx->L, 2048);
    return ctx->ws_budget == 0 || schur_bytes(ctx, (int)chunk) <= ctx->ws_budget;
}

// Forward in the Schur form (crt_schur.h): interior factorisation per
// wavenumber, forward sweep of [F r_I | F A_IG], Gram products V^T [u^ | V^],
// dense Cholesky of every S_l with its boundary solve, z^ = u^ - V^ p_G and
// the back sweep into kpot.  FP64 arithmetic (T = complex128, or double for
// the real DC systems).
template <typename T>
int run_forward_schur(crt_ctx* ctx)
{
    const SchurHost& H = ctx->schur_h;
    const int K = ctx->K, L = ctx->L, nI = H.nI, m = H.m;
    // column stride of the interior factor: mbI + 1, even for real entries
    // so that every column starts on a 16-byte boundary (bulk copies)
    const int WI = std::is_same<T, double>::value ? (H.mbI + 2) / 2 * 2 : H.mbI + 1;
    const int ncol = L + m, ncpl = (int)H.gi_pos.size();
    if (!ctx->d_sLI) {
        if (ctx->capture) return set_err(ctx, CRT_ERR_ARG, "captured forward without a prepared workspace");
        // the per-(k, l) Schur matrices in chunks of at most 8 GiB
        const size_t per = sizeof(cd) * (size_t)m * m;
        ctx->sS_chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)K * L, (8ull << 30) / per));
        CK(cudaMalloc(&ctx->d_sLI, sizeof(cd) * (size_t)K * nI * (H.mbI + 2)));
        CK(cudaMalloc(&ctx->d_sLrev, sizeof(cd) * (size_t)K * nI * (H.mbI + 2)));
        CK(cudaMalloc((void**)&ctx->d_sfak, sizeof(double) * (size_t)K * nI));
        CK(cudaMalloc(&ctx->d_sX, sizeof(cd) * (size_t)K * ncol * nI));
        CK(cudaMalloc(&ctx->d_scval, sizeof(cd) * (size_t)K * std::max(ncpl, 1)));
        CK(cudaMalloc(&ctx->d_sC, sizeof(cd) * (size_t)K * ncol * m));
        CK(cudaMalloc(&ctx->d_sxg, sizeof(cd) * (size_t)K * L * m));
        CK(cudaMalloc(&ctx->d_sS, per * ctx->sS_chunk));
    }
    T* X = static_cast<T*>(ctx->d_sX);
    T* cval = static_cast<T*>(ctx->d_scval);
    T* Cg = static_cast<T*>(ctx->d_sC);
    T* xg = static_cast<T*>(ctx->d_sxg);
    T* Sws = static_cast<T*>(ctx->d_sS);
    T* LI = static_cast<T*>(ctx->d_sLI);
    T* Lrev = static_cast<T*>(ctx->d_sLrev);
    SchurArgs S = ctx->schur;
    S.WI = WI;
    S.k0 = 0;
    S.nk = K;
    S.status = ctx->d_status;
    // the full mesh's assembly data (entries of A_IG and A_GG(l))
    BandArgs<T> Af{};
    Af.n = ctx->n;
    Af.mb = ctx->mb;
    Af.L = L;
    Af.K = K;
    Af.mixed = 1;
    Af.E = ctx->E;
    Af.R = std::max(ctx->R, 1);
    Af.nmn = ctx->nmn;
    Af.row_ptr = ctx->d_row_ptr;
    Af.ent_d = ctx->d_ent_d;
    Af.ent_ptr = ctx->d_ent_ptr;
    Af.con_code = ctx->d_con_code;
    Af.con_sig = ctx->d_con_sig;
    Af.elbg = ctx->d_elbg;
    Af.relbg = ctx->d_relbg;
    Af.kg = ctx->d_kg;
    Af.sigma = ctx->d_sigma;
    Af.status = ctx->d_status;
    // the interior systems A_II, one per wavenumber
    BandArgs<T> AI = Af;
    AI.n = nI;
    AI.mb = H.mbI;
    AI.W = WI;
    AI.sys0 = 0;
    AI.nsys = K;
    AI.mixed = 0;
    AI.fuse_rhs = 0;
    AI.row_ptr = ctx->d_sI_row_ptr;
    AI.ent_d = ctx->d_sI_ent_d;
    AI.ent_ptr = ctx->d_sI_ent_ptr;
    AI.con_code = ctx->d_sI_con_code;
    AI.con_sig = ctx->d_sI_con_sig;
    AI.dflag = ctx->d_sI_dflag;
    AI.dval = ctx->d_dval;
    AI.bdir = nullptr;
    AI.enr0 = S.posI_src;
    AI.lsink = 0;
    AI.nsink0 = 0;
    AI.Lws = LI;
    AI.lstride = (size_t)nI * WI;
    AI.yws = nullptr;
    AI.fakws = ctx->d_sfak;
    AI.aval = nullptr;
    ctx->tev_n = 0;
    ctx->fwd_marks.clear();
    crt_ctx::FwdMark mk{};
    mk.e0 = tev_rec(ctx);
    const bool blk = band_blk_fits<T>(H.mbI);
    int pb = 0;
    if (blk) {
        pb = band_panel<T>(AI, !ctx->capture, ctx->st);
        ctx->panel = pb & BAND_PANEL_MASK;
        launch_band_prep<T>(AI, ctx->st);   // the scaling factors for the right-hand sides
    }
    CK(cudaMemsetAsync(X, 0, sizeof(T) * (size_t)K * ncol * nI, ctx->st));
    // The forward sweep follows the interior factor column block by column
    // block on a second stream (the factor occupies K SMs for its whole
    // run); CRT_B200_SCHUR_OVERLAP=0, graph capture and the streamed
    // factor keep the two in sequence.
    const char* ov = std::getenv("CRT_B200_SCHUR_OVERLAP");
    const bool overlap = blk && !ctx->capture && !(ov && std::strcmp(ov, "0") == 0);
    if (overlap) {
        if (!ctx->d_fprog && !dalloc(ctx, &ctx->d_fprog, (size_t)K + 1)) return CRT_ERR_ALLOC;
        CK(cudaMemsetAsync(ctx->d_fprog, 0, sizeof(int) * ((size_t)K + 1), ctx->st));
        if (!ctx->ovl_st) CK(cudaStreamCreateWithFlags(&ctx->ovl_st, cudaStreamNonBlocking));
        if (!ctx->ovl_ev[0]) {
            CK(cudaEventCreateWithFlags(&ctx->ovl_ev[0], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->ovl_ev[1], cudaEventDisableTiming));
        }
    }
    mk.e8 = tev_rec(ctx);
    if (blk) {
        launch_schur_rhs<T>(S, Af, ctx->d_sfak, X, cval, ctx->st);
        if (overlap) {
            AI.progress = ctx->d_fprog;
            AI.started = ctx->d_fprog + K;
            CK(cudaEventRecord(ctx->ovl_ev[0], ctx->st));
        }
        launch_band_factor_blk<T>(AI, pb, ctx->st);
    } else {
        launch_band_factor<T>(AI, ctx->st);   // forms fak as it goes
        launch_schur_rhs<T>(S, Af, ctx->d_sfak, X, cval, ctx->st);
    }
    if (overlap) {
        SchurArgs So = S;
        So.progress = ctx->d_fprog;
        CK(cudaStreamWaitEvent(ctx->ovl_st, ctx->ovl_ev[0], 0));
        launch_wait_started(ctx->d_fprog + K, K, S.status, ctx->ovl_st);
        launch_schur_forward<T>(So, LI, X, ctx->ovl_st);
        CK(cudaEventRecord(ctx->ovl_ev[1], ctx->ovl_st));
        ctx->launches += 2;
    }
    if (int e = kernel_check(ctx, "interior factor")) return e;
    mk.e1 = tev_rec(ctx);
    mk.blk = blk;
    launch_schur_transpose<T>(S, LI, Lrev, ctx->st);
    if (overlap) CK(cudaStreamWaitEvent(ctx->st, ctx->ovl_ev[1], 0));
    else launch_schur_forward<T>(S, LI, X, ctx->st);
    ctx->sev[0] = tev_rec(ctx);
    launch_schur_gram<T>(S, X, Cg, ctx->st);
    ctx->sev[1] = tev_rec(ctx);
    // The electrode systems S_l = S0 + D_l: by the iteration preconditioned
    // with one factor per group of electrodes (the mixed-boundary parts D_l
    // of nearby electrodes differ little), or each by its own Cholesky
    // (CRT_B200_SCHUR_SOLVE=direct, a capture, or when the iteration does
    // not converge on every system).
    const char* sv_env = std::getenv("CRT_B200_SCHUR_SOLVE");
    const bool want_iter = !(sv_env && std::strcmp(sv_env, "direct") == 0);
    const char* gv = std::getenv("CRT_B200_SCHUR_GROUP");
    int grp = gv ? std::atoi(gv) : 16;
    grp = std::max(1, std::min(grp, L));
    const int ngrp = (L + grp - 1) / grp;
    // the iteration pays where its CTAs (eight systems each) fill the GPU
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    bool iter = want_iter && !ctx->capture && L >= 2 && ctx->sS_chunk >= K * ngrp &&
                schur_iter_smem<T>(m) <= 227 * 1024 &&
                (K * L / 8 >= nsm || (sv_env && std::strcmp(sv_env, "iter") == 0));
    ctx->schur_iter_mean = 0.0;
    if (iter) {
        if (!ctx->d_sS0) CK(cudaMalloc(&ctx->d_sS0, sizeof(T) * (size_t)K * m * m));
        const int nbd = (int)ctx->schur_h.bd_col.size();
        if (!ctx->d_sDv) CK(cudaMalloc(&ctx->d_sDv, sizeof(T) * std::max<size_t>(1, (size_t)K * L * nbd)));
        S.nbd = nbd;
        if (!ctx->d_snonconv) CK(cudaMalloc((void**)&ctx->d_snonconv, 2 * sizeof(int)));
        S.grp = grp;
        S.ngrp = ngrp;
        T* S0 = static_cast<T*>(ctx->d_sS0);
        CK(cudaMemsetAsync(ctx->d_snonconv, 0, 2 * sizeof(int), ctx->st));
        T* Dv = static_cast<T*>(ctx->d_sDv);
        launch_schur_s0<T>(S, Af, Cg, S0, ctx->st);
        launch_schur_dvals<T>(S, Af, Dv, ctx->st);
        launch_schur_ref<T>(S, Af, S0, Sws, ctx->d_snonconv, ctx->st);
        launch_schur_iter<T>(S, Af, Cg, S0, Sws, Dv, xg, 40, 1e-15, ctx->d_snonconv, ctx->st);
        int nc[2] = {0, 0};
        CK(cudaMemcpyAsync(nc, ctx->d_snonconv, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        ctx->launches += 5;
        if (nc[0] == 0) ctx->schur_iter_mean = (double)nc[1] / (double)(K * L);
        else iter = false;
    }
    if (!iter)
        for (int s0 = 0; s0 < K * L; s0 += ctx->sS_chunk)
            launch_schur_chol<T>(S, Af, Cg, Sws, xg, s0, std::min(ctx->sS_chunk, K * L - s0), ctx->st);
    ctx->sev[2] = tev_rec(ctx);
    launch_schur_zrebuild<T>(S, X, xg, ctx->st);
    launch_schur_back<T>(S, Lrev, ctx->d_sfak, X, xg, ctx->n, ctx->d_kpot, ctx->st);
    if (int e = kernel_check(ctx, "Schur kernels")) return e;
    mk.e2 = tev_rec(ctx);
    ctx->sev[3] = mk.e2;
    ctx->fwd_marks.push_back(mk);
    ctx->launches += 11 + (K * L + ctx->sS_chunk - 1) / ctx->sS_chunk;
    ctx->timings[9] = 1;
    ctx->timings[12] = blk ? ctx->panel : 0;
    return CRT_OK;
}

// Phase times of the last forward from its pooled events (after a host
// synchronisation that covers them).
void resolve_forward_timings(crt_ctx* ctx)
{
    float ms_f = 0, ms_s = 0, ms_prep = 0, ms_fk = 0, ms_res = 0, ms_cor = 0;
    for (const crt_ctx::FwdMark& m : ctx->fwd_marks) {
        const float a = tev_ms(ctx, m.e0, m.e1), b = tev_ms(ctx, m.e1, m.e2), c = tev_ms(ctx, m.e0, m.e8);
        ms_f += a;
        ms_s += b;
        if (m.blk) ms_prep += c;
        ms_fk += m.blk ? a - c : a;
        for (size_t i = 0; i + 2 < m.ref.size(); i += 3) {
            ms_res += tev_ms(ctx, m.ref[i], m.ref[i + 1]);
            ms_cor += tev_ms(ctx, m.ref[i + 1], m.ref[i + 2]);
        }
    }
    ctx->timings[0] = ms_f;
    ctx->timings[1] = ms_s;
    ctx->timings[2] = tev_ms(ctx, ctx->vol_e0, ctx->vol_e1);
    ctx->timings[7] = ms_prep;
    ctx->timings[8] = ms_fk;
    ctx->timings[10] = ms_res;
    ctx->timings[11] = ms_cor;
    // Schur form: forward sweep, Gram products, boundary Cholesky, rebuild
    // + back sweep
    if (ctx->schur_used && !ctx->fwd_marks.empty()) {
        const crt_ctx::FwdMark& m0 = ctx->fwd_marks[0];
        ctx->timings[13] = tev_ms(ctx, m0.e1, ctx->sev[0]);
        ctx->timings[14] = tev_ms(ctx, ctx->sev[0], ctx->sev[1]);
        ctx->timings[15] = tev_ms(ctx, ctx->sev[1], ctx->sev[2]);
        ctx->timings[16] = tev_ms(ctx, ctx->sev[2], ctx->sev[3]);
        ctx->timings[17] = ctx->schur_iter_mean;
    } else {
        ctx->timings[13] = ctx->timings[14] = ctx->timings[15] = ctx->timings[16] = ctx->timings[17] = 0.0;
    }
}

int forward_common(crt_ctx* ctx, int ldc, int mode, const double* kfak_h)
{
    const size_t nk = (size_t)ctx->n * ctx->L * ctx->K;
    if (!ctx->d_kpot) {
        if (!dalloc(ctx, &ctx->d_kpot, nk)) return CRT_ERR_ALLOC;
        if (!dalloc(ctx, &ctx->d_volt, (size_t)ctx->N) || !dalloc(ctx, &ctx->d_sigmaa, (size_t)ctx->N) ||
            !dalloc(ctx, &ctx->d_hel, (size_t)ctx->L * ctx->L))
            return CRT_ERR_ALLOC;
    }
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int) * ctx->nstatus, ctx->st));
    // the mixed form factors the complex systems in complex64 and refines
    const char* fv = std::getenv("CRT_B200_FACTOR");
    const bool c64 = !ldc && ctx->prec == CRT_PREC_MIXED && band_blk_fits<cf>(ctx->mb) && !(fv && std::strcmp(fv, "v0") == 0);
    ctx->schur_used = use_schur(ctx);
    int e;
    if (ctx->schur_used)
        e = ldc ? run_forward_schur<double>(ctx) : run_forward_schur<cd>(ctx);
    else
        e = ldc ? run_forward<double>(ctx) : (c64 ? run_forward<cf>(ctx) : run_forward<cd>(ctx));
    if (e) return e;
    double* d_kfak = nullptr;
    if (kfak_h && mode == 1) {
        CK(cudaMalloc((void**)&d_kfak, sizeof(double) * ctx->N));
        CK(cudaMemcpyAsync(d_kfak, kfak_h, sizeof(double) * ctx->N, cudaMemcpyHostToDevice, ctx->st));
    }
    VoltArgs V{};
    V.n = ctx->n;
    V.L = ctx->L;
    V.K = ctx->K;
    V.N = ctx->N;
    V.swrtr = ctx->swrtr;
    V.ldc = ldc;
    V.mode = mode;
    V.pi = ctx->pi;
    V.kpot = ctx->d_kpot;
    V.kwnwi = ctx->d_kwnwi;
    V.enr0 = ctx->d_enr0;
    V.strnr = ctx->d_strnr;
    V.vnr = ctx->d_vnr;
    V.kfak = d_kfak;
    V.hel = ctx->d_hel;
    V.volt = ctx->d_volt;
    V.sigmaa = ctx->d_sigmaa;
    V.status = ctx->d_status + ctx->nstatus - 1;
    ctx->vol_e0 = tev_rec(ctx);
    launch_voltages(V, ctx->st);
    ctx->launches += 2;
    ctx->vol_e1 = tev_rec(ctx);
    if (int k = kernel_check(ctx, "voltages")) return k;
    // the forward's one host synchronisation: per-system status of the
    // factorisations and voltages, then the phase times
    int st = collect_status(ctx, ctx->nstatus);
    if (d_kfak) cudaFree(d_kfak);
    if (!ctx->capture) resolve_forward_timings(ctx);
    if (st) return st;
    ctx->last_ldc = ldc;
    ctx->have_forward = 1;
    // the Jacobian stays that of the model it was computed at (the
    // reference's sens is kept across the lambda and step-length trials,
    // src/inv.f90:769-912, until the next accepted iterate recomputes it)
    return CRT_OK;
}

}  // namespace

extern "C" int32_t crt_forward(crt_ctx* ctx, const double* sigma, int32_t ldc, int32_t mode, const double* kfak,
                               double* volt, double* sigmaa, double* kpot)
{
    if (!ctx || !sigma) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    if (!ctx->d_sigma && !dalloc(ctx, &ctx->d_sigma, (size_t)ctx->E)) return CRT_ERR_ALLOC;
    CK(cudaMemcpyAsync(ctx->d_sigma, sigma, sizeof(cd) * ctx->E, cudaMemcpyHostToDevice, ctx->st));
    int e = forward_common(ctx, ldc, mode, kfak);
    if (e) return e;
    if (volt) CK(cudaMemcpyAsync(volt, ctx->d_volt, sizeof(cd) * ctx->N, cudaMemcpyDeviceToHost, ctx->st));
    if (sigmaa) CK(cudaMemcpyAsync(sigmaa, ctx->d_sigmaa, sizeof(cd) * ctx->N, cudaMemcpyDeviceToHost, ctx->st));
    if (kpot)
        CK(cudaMemcpyAsync(kpot, ctx->d_kpot, sizeof(cd) * (size_t)ctx->n * ctx->L * ctx->K, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return CRT_OK;
}

extern "C" int32_t crt_potentials(crt_ctx* ctx, double* hpot)
{
    if (!ctx || !hpot) return CRT_ERR_ARG;
    if (!ctx->have_forward) return set_err(ctx, CRT_ERR_ARG, "crt_potentials before crt_forward");
    CK(cudaSetDevice(ctx->device));
    cd* d_h = nullptr;
    CK(cudaMalloc((void**)&d_h, sizeof(cd) * (size_t)ctx->n * ctx->L));
    VoltArgs V{};
    V.n = ctx->n;
    V.L = ctx->L;
    V.K = ctx->K;
    V.swrtr = ctx->swrtr;
    V.pi = ctx->pi;
    V.kpot = ctx->d_kpot;
    V.kwnwi = ctx->d_kwnwi;
    launch_hpot_full(V, d_h, ctx->st);
    ctx->launches++;
    if (int e = kernel_check(ctx, "hpot")) {
        cudaFree(d_h);
        return e;
    }
    CK(cudaMemcpyAsync(hpot, d_h, sizeof(cd) * (size_t)ctx->n * ctx->L, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    cudaFree(d_h);
    return CRT_OK;
}

// ---------------------------------------------------------------------------
// Jacobian.
namespace {
int jacobian_device(crt_ctx* ctx, int mode, const double* strom_h)
{
    const bool real = (mode == 1);
    const size_t ne = (size_t)ctx->E * ctx->N;
    if (!ctx->d_kpt && !dalloc(ctx, &ctx->d_kpt, (size_t)ctx->n * ctx->L * ctx->K)) return CRT_ERR_ALLOC;
    if (!ctx->d_sens || ctx->sens_real != (int)real) {
        if (ctx->d_sens) cudaFree(ctx->d_sens);
        ctx->d_sens = nullptr;
        CK(cudaMalloc(&ctx->d_sens, ne * sens_elem_bytes(ctx, real)));
        ctx->sens_real = real;
    }
    if (strom_h && mode == 2) {
        if (!upload(ctx, &ctx->d_strom, strom_h, (size_t)ctx->N)) return CRT_ERR_ALLOC;
    }
    if (!ev_rec(ctx, 5)) return CRT_ERR_CUDA;
    launch_transpose_kpot(ctx->d_kpot, ctx->d_kpt, ctx->n, ctx->L, ctx->K, ctx->st);
    ctx->launches++;
    int kc = 0;
    size_t smem = sens_smem(ctx->L, ctx->K, ctx->nkmax, ctx->nmn, &kc, 200 * 1024, real);
    SensArgs S{};
    S.n = ctx->n;
    S.E = ctx->E;
    S.L = ctx->L;
    S.K = ctx->K;
    S.N = ctx->N;
    S.nmn = ctx->nmn;
    S.maxnodes = ctx->maxnodes;
    S.swrtr = ctx->swrtr;
    S.mode = mode;
    S.kchunk = kc;
    S.pi = ctx->pi;
    S.kpt = ctx->d_kpt;
    S.elbg = ctx->d_elbg;
    S.kwnwi = ctx->d_kwnwi;
    S.nrel0 = ctx->d_nrel0;
    S.enk = ctx->d_enk;
    S.elec = ctx->d_elec;
    S.sigma = ctx->d_sigma;
    S.volt = ctx->d_volt;
    S.strom = (mode == 2 && strom_h) ? ctx->d_strom : nullptr;
    S.sens = ctx->d_sens;
    S.out_prec = ctx->prec == CRT_PREC_MIXED;
    if (kc < ctx->K) {
        if (!ctx->d_part_sens && !dalloc(ctx, &ctx->d_part_sens, ne)) return CRT_ERR_ALLOC;
    }
    S.part = ctx->d_part_sens;
    if (!ctx->d_sfac && !dalloc(ctx, &ctx->d_sfac, (size_t)ctx->N)) return CRT_ERR_ALLOC;
    S.rfac = ctx->d_sfac;
    int LP = 0, gkc = 0, gnt = 0;
    size_t gsmem = 0;
    const char* sv = std::getenv("CRT_B200_SENS");
    const bool force_direct = sv && std::strcmp(sv, "direct") == 0;
    if (!force_direct && sens_gram_plan(ctx->L, ctx->K, ctx->nkmax, real, &LP, &gkc, &gsmem, &gnt)) {
        launch_sens_gram(S, LP, gkc, gsmem, gnt, real, ctx->st);
        ctx->launches += S.out_prec ? 2 : 1;
    } else {
        launch_sens(S, smem, real, ctx->st);
        ctx->launches++;
    }
    if (!ev_rec(ctx, 6)) return CRT_ERR_CUDA;
    if (int e = kernel_check(ctx, "sensitivities")) return e;
    if (!ev_sync(ctx, 6)) return CRT_ERR_CUDA;
    float ms = 0;
    ms = ev_ms(ctx, 5, 6);
    ctx->timings[3] = ms;
    ctx->have_sens = 1;
    return CRT_OK;
}
// Host copy of the device Jacobian in FP64 (complex values interleaved).
int download_sens(crt_ctx* ctx, double* sens)
{
    const size_t ne = (size_t)ctx->E * ctx->N;
    const size_t vals = ne * (ctx->sens_real ? 1 : 2);
    if (ctx->prec == CRT_PREC_MIXED) {
        std::vector<float> h(vals);
        CK(cudaMemcpyAsync(h.data(), ctx->d_sens, vals * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        for (size_t q = 0; q < vals; ++q) sens[q] = (double)h[q];
    } else {
        CK(cudaMemcpyAsync(sens, ctx->d_sens, vals * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    return CRT_OK;
}
}  // namespace

extern "C" int32_t crt_jacobian(crt_ctx* ctx, int32_t mode, const double* strom, double* sens)
{
    if (!ctx || mode < 0 || mode > 2) return CRT_ERR_ARG;
    if (!ctx->have_forward) return set_err(ctx, CRT_ERR_ARG, "crt_jacobian before crt_forward");
    CK(cudaSetDevice(ctx->device));
    int e = jacobian_device(ctx, mode, strom);
    if (e) return e;
    return sens ? download_sens(ctx, sens) : CRT_OK;
}

extern "C" int32_t crt_set_jacobian(crt_ctx* ctx, int32_t real, const double* sens)
{
    if (!ctx || !sens) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    const size_t ne = (size_t)ctx->E * ctx->N;
    const size_t vals = ne * (real ? 1 : 2);
    const size_t bytes = ne * sens_elem_bytes(ctx, real != 0);
    if (!ctx->d_sens || ctx->sens_real != (real != 0)) {
        if (ctx->d_sens) cudaFree(ctx->d_sens);
        ctx->d_sens = nullptr;
        CK(cudaMalloc(&ctx->d_sens, bytes));
        ctx->sens_real = real != 0;
    }
    if (ctx->prec == CRT_PREC_MIXED) {
        std::vector<float> h(vals);
        for (size_t q = 0; q < vals; ++q) h[q] = (float)sens[q];
        CK(cudaMemcpyAsync(ctx->d_sens, h.data(), bytes, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    } else {
        CK(cudaMemcpyAsync(ctx->d_sens, sens, bytes, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    ctx->have_sens = 1;
    return CRT_OK;
}

extern "C" int32_t crt_set_configs(crt_ctx* ctx, const int32_t* strnr, const int32_t* vnr)
{
    if (!ctx || !strnr || !vnr) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    std::vector<int4> elec(ctx->N);
    for (int i = 0; i < ctx->N; ++i) {
        int s = strnr[i], v = vnr[i];
        int e1 = s % 10000, e2 = s / 10000, e3 = v % 10000, e4 = v / 10000;
        if (std::min({e1, e2, e3, e4}) < 0 || std::max({e1, e2, e3, e4}) > ctx->L)
            return set_err(ctx, 46, "electrode number out of range (errnr 46)");
        elec[i] = make_int4(e1 - 1, e2 - 1, e3 - 1, e4 - 1);
    }
    // Readings whose potential electrodes were swapped (chkpol.f90:84-87,
    // :113-116): the stored response follows, volt -> -volt and sigmaa's
    // phase moved by pi into (-pi, pi], so that the Jacobian of the last
    // forward (dV / V) keeps its sign.
    std::vector<int> swapped;
    if (ctx->have_forward && (int)ctx->vnr_h.size() == ctx->N)
        for (int i = 0; i < ctx->N; ++i) {
            const int o = ctx->vnr_h[i], v = vnr[i];
            if (o != v && (o % 10000) == v / 10000 && o / 10000 == (v % 10000) && strnr[i] == ctx->strnr_h[i])
                swapped.push_back(i);
        }
    if (!swapped.empty()) {
        std::vector<cd> vo(ctx->N), sa(ctx->N);
        CK(cudaMemcpyAsync(vo.data(), ctx->d_volt, sizeof(cd) * ctx->N, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(sa.data(), ctx->d_sigmaa, sizeof(cd) * ctx->N, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        for (int i : swapped) {
            vo[i] = -vo[i];
            sa[i].y += sa[i].y > 0.0 ? -ctx->pi : ctx->pi;
        }
        CK(cudaMemcpyAsync(ctx->d_volt, vo.data(), sizeof(cd) * ctx->N, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->d_sigmaa, sa.data(), sizeof(cd) * ctx->N, cudaMemcpyHostToDevice, ctx->st));
    }
    CK(cudaMemcpyAsync(ctx->d_strnr, strnr, sizeof(int) * ctx->N, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->d_vnr, vnr, sizeof(int) * ctx->N, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->d_elec, elec.data(), sizeof(int4) * ctx->N, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->strnr_h.assign(strnr, strnr + ctx->N);
    ctx->vnr_h.assign(vnr, vnr + ctx->N);
    return CRT_OK;
}

// ---------------------------------------------------------------------------
// Inversion pieces.
extern "C" int32_t crt_set_regularizer(crt_ctx* ctx, int32_t ltri, int32_t nx, int32_t nnb, const double* smatm,
                                       const int32_t* nachbar)
{
    if (!ctx || !smatm) return CRT_ERR_ARG;
    if (!(ltri == 0 || ltri == 1 || ltri == 2))
        return set_err(ctx, CRT_ERR_UNSUPPORTED, "only the smoothness regularisers ltri 0/1/2 are implemented");
    CK(cudaSetDevice(ctx->device));
    const int M = ctx->E;
    ctx->ltri = ltri;
    ctx->nx = nx;
    ctx->nnb = nnb;
    if (ltri == 0) {
        if (nx < 1 || M % nx != 0) return set_err(ctx, 89, "five-point regulariser needs manz = nx * nz (errnr 89)");
        if (!upload(ctx, &ctx->d_smatm, smatm, (size_t)M * 3)) return CRT_ERR_ALLOC;
    } else {
        if (!nachbar || nnb < 1) return CRT_ERR_ARG;
        for (size_t q = 0; q < (size_t)M * nnb; ++q)
            if (nachbar[q] < 0 || nachbar[q] > M) return set_err(ctx, CRT_ERR_ARG, "nachbar entry out of range");
        if (!upload(ctx, &ctx->d_smatm, smatm, (size_t)M * (nnb + 1)) ||
            !upload(ctx, &ctx->d_nachbar, nachbar, (size_t)M * (nnb + 1)))
            return CRT_ERR_ALLOC;
    }
    CK(cudaStreamSynchronize(ctx->st));
    ctx->spc_why.clear();
    // the lambda candidates' factor buffers follow the plan they were cloned from
    for (SpcPlan& c : ctx->spc_c) spc_plan_free_clone(c);
    ctx->spc_c.clear();
    if (int e = spc_plan_build(ctx->spc, M, ltri, nx, nnb, smatm, nachbar, ctx->spc_why))
        return set_err(ctx, e, "block preconditioner set-up failed");
    // learned correction: same graph; a graph it cannot hold (more than four
    // neighbours, not symmetric) leaves it unavailable, which is not an error
    const int ge = gnn_setup(ctx->gnn, M, ltri, nx, nnb, nachbar);
    if (ge == CRT_ERR_ALLOC || ge == CRT_ERR_CUDA) return set_err(ctx, ge, "learned preconditioner set-up failed");
    if (ctx->gnn.ready && gnn_init(ctx->gnn, 1)) return set_err(ctx, CRT_ERR_CUDA, "learned preconditioner init");
    return CRT_OK;
}

extern "C" int32_t crt_set_data(crt_ctx* ctx, const double* dat, const double* wmatd, const int32_t* wdfak)
{
    if (!ctx || !dat || !wmatd) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    std::vector<double> wd(ctx->N);
    for (int i = 0; i < ctx->N; ++i) wd[i] = wmatd[i] * (double)(wdfak ? wdfak[i] : 1);
    if (!upload(ctx, &ctx->d_dat, reinterpret_cast<const cd*>(dat), (size_t)ctx->N) ||
        !upload(ctx, &ctx->d_wd, wd.data(), wd.size()))
        return CRT_ERR_ALLOC;
    CK(cudaStreamSynchronize(ctx->st));
    return CRT_OK;
}

namespace {

int ensure_cg_buffers(crt_ctx* ctx, int ncgmax)
{
    const int M = ctx->E, N = ctx->N;
    if (!ctx->d_cgfac) {
        int nsplit = std::max(1, std::min(64, (148 * 8) / std::max(1, (N + 255) / 256)));
        ctx->cg_nsplit = nsplit;
        bool ok = dalloc(ctx, &ctx->d_cgfac, (size_t)M) && dalloc(ctx, &ctx->d_rhs, (size_t)M) &&
                  dalloc(ctx, &ctx->d_p, (size_t)M) && dalloc(ctx, &ctx->d_r, (size_t)M) &&
                  dalloc(ctx, &ctx->d_bvec, (size_t)M) && dalloc(ctx, &ctx->d_dpar, (size_t)M) &&
                  dalloc(ctx, &ctx->d_ap, (size_t)N) && dalloc(ctx, &ctx->d_cgpart, (size_t)nsplit * N) &&
                  dalloc(ctx, &ctx->d_cgst, (size_t)1) && dalloc(ctx, &ctx->d_bdpar, (size_t)1) &&
                  dalloc(ctx, &ctx->d_par, (size_t)M) && dalloc(ctx, &ctx->d_z, (size_t)M) &&
                  dalloc(ctx, &ctx->d_rold, (size_t)M) && dalloc(ctx, &ctx->d_zb, (size_t)M) &&
                  dalloc(ctx, &ctx->d_live, (size_t)1) && dalloc(ctx, &ctx->d_vred, (size_t)32 * 8);
        if (!ok) return CRT_ERR_ALLOC;
        if (cudaMemset(ctx->d_live, 0, sizeof(CGState)) != cudaSuccess) return CRT_ERR_CUDA;
    }
    if (ctx->cg_ncgmax_alloc < ncgmax + 2) {
        if (!dalloc(ctx, &ctx->d_cgres, (size_t)ncgmax + 2)) return CRT_ERR_ALLOC;
        ctx->cg_ncgmax_alloc = ncgmax + 2;
    }
    return CRT_OK;
}

CGArgs make_cg_args(crt_ctx* ctx, const crt_cg_params* prm)
{
    CGArgs a{};
    a.M = ctx->E;
    a.N = ctx->N;
    a.jmode = prm->ldc ? 1 : (prm->lfpi ? 2 : 0);
    a.jprec = ctx->prec == CRT_PREC_MIXED ? 1 : 0;
    a.ltri = ctx->ltri;
    a.nx = ctx->nx;
    a.nnb = ctx->nnb;
    a.ncgmax = prm->ncgmax;
    a.lam = prm->lam;
    a.eps = prm->eps;
    a.J = ctx->d_sens;
    a.wd = ctx->d_wd;
    a.smatm = ctx->d_smatm;
    a.nachbar = ctx->d_nachbar;
    a.cgfac = ctx->d_cgfac;
    a.rhs = ctx->d_rhs;
    a.p = ctx->d_p;
    a.r = ctx->d_r;
    a.bvec = ctx->d_bvec;
    a.dpar = ctx->d_dpar;
    a.ap = ctx->d_ap;
    a.part = ctx->d_cgpart;
    a.nsplit = ctx->cg_nsplit;
    a.cgres = ctx->d_cgres;
    a.st = ctx->d_cgst;
    a.pc = 0;
    a.z = ctx->d_z;
    a.rold = ctx->d_rold;
    a.pc_gnn = 0;
    a.zb = nullptr;
    a.vred = ctx->d_vred;
    return a;
}

// The fused matvec (one read of J per CG iteration, complex64 Jacobians)
// when CRT_B200_CG_FUSED=1 asks for it; the two-pass kernels otherwise (on
// the 60k-cell benchmark the fused form is slower: every row block waits
// for a grid-wide exchange).  Sets the fused fields of `a`; allocates the
// reduction ring once per context.
int setup_cg_fused(crt_ctx* ctx, CGArgs* a)
{
    a->fused = 0;
    const char* ev = std::getenv("CRT_B200_CG_FUSED");
    if (!ev || std::strcmp(ev, "1") != 0) return CRT_OK;
    int nsm = 0, smem = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
    CK(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    if (!cg_fused_fits(*a, nsm, (size_t)smem)) return CRT_OK;
    const size_t part = (size_t)CGF_Q * nsm * CGF_R * sizeof(cd), v = (size_t)CGF_Q * CGF_R * sizeof(cd);
    const size_t words = (size_t)CGF_Q * 8 + 8 + (size_t)CGF_Q * 4 + 4;
    const size_t bytes = part + v + words;
    if (ctx->cgf_bytes < bytes) {
        if (ctx->d_cgf) cudaFree(ctx->d_cgf);
        ctx->d_cgf = nullptr;
        ctx->cgf_bytes = 0;
        if (cudaMalloc(&ctx->d_cgf, bytes) != cudaSuccess) return set_err(ctx, CRT_ERR_ALLOC, "fused CG workspace");
        CK(cudaMemsetAsync(ctx->d_cgf, 0, bytes, ctx->st));
        ctx->cgf_bytes = bytes;
    }
    ctx->cgf_grid = nsm;
    // row blocks between the two uses of a tile: long enough for the grid's
    // partial sums to arrive, short enough for the tiles to stay in L2
    int lag = 8;
    if (const char* lv = std::getenv("CRT_B200_CG_FUSED_LAG")) lag = std::atoi(lv);
    a->flag_lag = std::max(CGF_S, std::min(CGF_Q - 1, lag));
    a->fused = 1;
    a->fper = (a->M + nsm - 1) / nsm;
    a->fpart = reinterpret_cast<cd*>(ctx->d_cgf);
    a->fv = reinterpret_cast<cd*>(ctx->d_cgf + part);
    a->fflag = reinterpret_cast<unsigned long long*>(ctx->d_cgf + part + v);
    a->fepoch = a->fflag + CGF_Q;
    a->fcnt = reinterpret_cast<int*>(a->fepoch + 1);
    a->ferr = a->fcnt + CGF_Q;
    return CRT_OK;
}

// Block factor and / or message weights of the learned correction for the
// system whose cgfac was just formed.  A requested piece that is not
// available (bandwidth, pivot breakdown, untrained network, network trained
// on the other base) is left out, down to the Jacobi form.
int prepare_preconditioner(crt_ctx* ctx, const crt_cg_params* prm, bool* use_block, bool* use_gnn)
{
    const int pc = prm->precond;
    *use_block = false;
    *use_gnn = false;
    if ((pc == CRT_PRECOND_BLOCK || pc == CRT_PRECOND_BLOCK_GNN) && ctx->spc.ok) {
        // S from cgfac and lam, factored once per update; a breakdown
        // (non-positive pivot) drops the block part
        launch_spc_factor(ctx->spc, ctx->d_cgfac, ctx->d_smatm, prm->lam, ctx->st);
        ctx->launches += 3 + (ctx->spc.nb > 1 ? 1 : 0);
        int flag = 0;
        CK(cudaMemcpyAsync(&flag, ctx->spc.d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (int e = kernel_check(ctx, "block preconditioner factor")) return e;
        *use_block = flag == 0;
    }
    if ((pc == CRT_PRECOND_GNN || pc == CRT_PRECOND_BLOCK_GNN) && ctx->gnn.ready && ctx->gnn.trained &&
        ctx->gnn.form == (*use_block ? 1 : 0)) {
        launch_gnn_edges(ctx->gnn, ctx->d_cgfac, ctx->d_smatm, prm->lam, ctx->st);
        ctx->launches++;
        *use_gnn = true;
    }
    return CRT_OK;
}

// update.f90 on device-resident J, data, response and model (d_par).
int update_device(crt_ctx* ctx, const crt_cg_params* prm, const cd* d_sigmaa, int* ncg_out)
{
    if (ctx->ltri < 0) return set_err(ctx, CRT_ERR_ARG, "regulariser not set (crt_set_regularizer)");
    if (!ctx->d_dat) return set_err(ctx, CRT_ERR_ARG, "data not set (crt_set_data)");
    if (!ctx->have_sens) return set_err(ctx, CRT_ERR_ARG, "no Jacobian (crt_jacobian / crt_set_jacobian)");
    if (prm->ldc != ctx->sens_real) return set_err(ctx, CRT_ERR_ARG, "ldc does not match the Jacobian type");
    if (int e = ensure_cg_buffers(ctx, prm->ncgmax)) return e;
    CGArgs a = make_cg_args(ctx, prm);
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    launch_cg_setup(a, ctx->d_dat, d_sigmaa, ctx->d_par, ctx->st);
    ctx->launches += 1;
    bool use_block = false, use_gnn = false;
    if (int e = prepare_preconditioner(ctx, prm, &use_block, &use_gnn)) return e;
    a.pc = (use_block || use_gnn) ? 1 : 0;
    a.pc_gnn = use_gnn ? 1 : 0;
    a.zb = (use_block && use_gnn) ? ctx->d_zb : nullptr;
    ctx->cg_form = use_block ? (use_gnn ? CRT_PRECOND_BLOCK_GNN : CRT_PRECOND_BLOCK)
                             : (use_gnn ? CRT_PRECOND_GNN : CRT_PRECOND_JACOBI);
    if (int e = setup_cg_fused(ctx, &a)) return e;
    launch_cg_init(a, ctx->st);
    ctx->launches += 1;
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    if (int e = kernel_check(ctx, "cg setup")) return e;
    // iterate in batches; the device-side stop flag makes surplus launches no-ops
    CGState hs{};
    int done_iters = 0;
    const int batch = 16;
    while (done_iters < prm->ncgmax) {
        int it = std::min(batch, prm->ncgmax - done_iters);
        launch_cg_iterations(a, it, use_block ? &ctx->spc : nullptr, use_gnn ? &ctx->gnn : nullptr, ctx->d_zb,
                             ctx->st);
        ctx->launches += ((a.fused ? 5 : 7) + (a.pc ? 1 : 0) + (use_block ? 2 : 0) + (use_gnn ? 7 : 0)) * it;
        done_iters += it;
        CK(cudaMemcpyAsync(&hs, ctx->d_cgst, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (hs.done) break;
    }
    if (int e = kernel_check(ctx, "cg iterations")) return e;
    if (a.fused) {
        int ferr = 0;
        CK(cudaMemcpyAsync(&ferr, a.ferr, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (ferr) {
            // the ring's counters are left mid-block: start it afresh
            CK(cudaMemsetAsync(ctx->d_cgf, 0, ctx->cgf_bytes, ctx->st));
            CK(cudaStreamSynchronize(ctx->st));
            return set_err(ctx, CRT_ERR_CUDA, "fused CG matvec: a wait for the grid's partial sums gave up");
        }
    }
    launch_cg_finish(a, prm->lfpi, prm->step, ctx->d_par, ctx->d_bdpar, ctx->st);
    ctx->launches++;
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    CK(cudaEventSynchronize(ctx->ev[2]));
    float a1 = 0, a2 = 0;
    cudaEventElapsedTime(&a1, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&a2, ctx->ev[1], ctx->ev[2]);
    ctx->timings[4] = a1;
    ctx->timings[5] = a2;
    CK(cudaMemcpyAsync(&hs, ctx->d_cgst, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (ncg_out) *ncg_out = hs.ncg;
    ctx->gnn_guard = use_gnn ? hs.no_gnn : 0;
    return CRT_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// blam0 (src/blam0.f90:131-167): jtj(j) = |sum_i sum_k conj(J_ij) J_ik w_i|
// = |sum_i conj(J_ij) w_i s_i| with the row sums s = J 1: two passes over
// the device-resident Jacobian instead of the reference's O(N M^2) loop.
// `real` selects the real Jacobian (ldc: sensdc) or, with `re_part`, the
// real part of the complex one (final phase improvement).
namespace {

template <typename S> __device__ __forceinline__ cd jval(const S* J, size_t idx);
template <> __device__ __forceinline__ cd jval<cd>(const cd* J, size_t idx) { return J[idx]; }
template <> __device__ __forceinline__ cd jval<cf>(const cf* J, size_t idx)
{
    return cd{(double)J[idx].x, (double)J[idx].y};
}
template <> __device__ __forceinline__ cd jval<double>(const double* J, size_t idx) { return cd{J[idx], 0.0}; }
template <> __device__ __forceinline__ cd jval<float>(const float* J, size_t idx) { return cd{(double)J[idx], 0.0}; }

template <typename S>
__global__ void k_blam0_rowsum(const S* __restrict__ J, int N, int M, int re_part, cd* s)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    cd acc{0.0, 0.0};
    for (int j = 0; j < M; ++j) acc += jval<S>(J, (size_t)j * N + i);
    if (re_part) acc.y = 0.0;
    s[i] = acc;
}

// one warp per model cell: |sum_i conj(J_ij) wd_i s_i|
template <typename S>
__global__ void k_blam0_col(const S* __restrict__ J, int N, int M, int re_part, const double* __restrict__ wd,
                            const cd* __restrict__ s, double* jtj)
{
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (j >= M) return;
    cd acc{0.0, 0.0};
    for (int i = lane; i < N; i += 32) {
        cd a = jval<S>(J, (size_t)j * N + i);
        if (re_part) a.y = 0.0;
        acc += conj(a) * (s[i] * wd[i]);
    }
    for (int off = 16; off > 0; off >>= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, off);
    }
    if (lane == 0) jtj[j] = hypot(acc.x, acc.y);
}

// Coverage (bbsens.f90:52-78): one warp per model cell, sum_i |J_ij| w_i
// (|Re J_ij| for part 1); w = the caller's weights or sqrt(wmatd wdfak).
template <typename S>
__global__ void k_coverage_col(const S* __restrict__ J, int N, int M, int re_part, const double* __restrict__ w,
                               int w_is_sq, double* csens)
{
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (j >= M) return;
    double acc = 0.0;
    for (int i = lane; i < N; i += 32) {
        const cd a = jval<S>(J, (size_t)j * N + i);
        const double wi = w_is_sq ? sqrt(w[i]) : w[i];
        acc += (re_part ? fabs(a.x) : hypot(a.x, a.y)) * wi;
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) csens[j] = acc;
}

template <typename S>
void blam0_launch(const crt_ctx* ctx, int re_part, cd* s, double* jtj)
{
    const S* J = static_cast<const S*>(ctx->d_sens);
    k_blam0_rowsum<S><<<(ctx->N + 255) / 256, 256, 0, ctx->st>>>(J, ctx->N, ctx->E, re_part, s);
    k_blam0_col<S><<<(ctx->E * 32 + 255) / 256, 256, 0, ctx->st>>>(J, ctx->N, ctx->E, re_part, ctx->d_wd, s, jtj);
}

}  // namespace

extern "C" int32_t crt_blam0(crt_ctx* ctx, int32_t ldc, int32_t lfpi, double alfx, double alfz, double* lammax)
{
    if (!ctx || !lammax || !(alfx + alfz > 0.0)) return CRT_ERR_ARG;
    if (!ctx->have_sens || !ctx->d_sens) return set_err(ctx, CRT_ERR_ARG, "crt_blam0 before crt_jacobian");
    if (!ctx->d_wd) return set_err(ctx, CRT_ERR_ARG, "crt_blam0 before crt_set_data");
    if ((ldc != 0) != (ctx->sens_real != 0))
        return set_err(ctx, CRT_ERR_ARG, "crt_blam0: ldc does not match the stored Jacobian");
    CK(cudaSetDevice(ctx->device));
    cd* s = nullptr;
    double* jtj = nullptr;
    CK(cudaMalloc((void**)&s, sizeof(cd) * (size_t)ctx->N));
    if (cudaMalloc((void**)&jtj, sizeof(double) * (size_t)ctx->E) != cudaSuccess) {
        cudaFree(s);
        return set_err(ctx, CRT_ERR_CUDA, "cudaMalloc of the blam0 sums");
    }
    const bool f32 = ctx->prec == CRT_PREC_MIXED;
    if (ldc) {
        if (f32) blam0_launch<float>(ctx, 0, s, jtj);
        else blam0_launch<double>(ctx, 0, s, jtj);
    } else {
        if (f32) blam0_launch<cf>(ctx, lfpi != 0, s, jtj);
        else blam0_launch<cd>(ctx, lfpi != 0, s, jtj);
    }
    ctx->launches += 2;
    std::vector<double> h(ctx->E);
    int e = kernel_check(ctx, "blam0");
    if (!e && cudaMemcpyAsync(h.data(), jtj, sizeof(double) * ctx->E, cudaMemcpyDeviceToHost, ctx->st) != cudaSuccess)
        e = set_err(ctx, CRT_ERR_CUDA, "blam0 copy");
    if (!e && cudaStreamSynchronize(ctx->st) != cudaSuccess) e = set_err(ctx, CRT_ERR_CUDA, "blam0 sync");
    cudaFree(s);
    cudaFree(jtj);
    if (e) return e;
    double tot = 0.0;
    for (double v : h) tot += v;
    *lammax = tot / (double)ctx->E * 2.0 / (alfx + alfz) * 5.0;
    return CRT_OK;
}

extern "C" int32_t crt_coverage(crt_ctx* ctx, int32_t part, const double* weight, double* csens)
{
    if (!ctx || !csens || part < 0 || part > 1) return CRT_ERR_ARG;
    if (!ctx->have_sens || !ctx->d_sens) return set_err(ctx, CRT_ERR_ARG, "crt_coverage before crt_jacobian");
    if (!weight && !ctx->d_wd) return set_err(ctx, CRT_ERR_ARG, "crt_coverage without weights before crt_set_data");
    CK(cudaSetDevice(ctx->device));
    double *w = nullptr, *cs = nullptr;
    CK(cudaMalloc((void**)&cs, sizeof(double) * (size_t)ctx->E));
    if (weight) {
        if (cudaMalloc((void**)&w, sizeof(double) * (size_t)ctx->N) != cudaSuccess) {
            cudaFree(cs);
            return set_err(ctx, CRT_ERR_CUDA, "cudaMalloc of the coverage weights");
        }
        if (cudaMemcpyAsync(w, weight, sizeof(double) * ctx->N, cudaMemcpyHostToDevice, ctx->st) != cudaSuccess) {
            cudaFree(cs);
            cudaFree(w);
            return set_err(ctx, CRT_ERR_CUDA, "coverage weights copy");
        }
    }
    const double* wd = weight ? w : ctx->d_wd;
    const int sq = weight ? 0 : 1, g = (ctx->E * 32 + 255) / 256;
    const bool f32 = ctx->prec == CRT_PREC_MIXED;
    if (ctx->sens_real) {
        if (f32) k_coverage_col<float><<<g, 256, 0, ctx->st>>>(static_cast<const float*>(ctx->d_sens), ctx->N, ctx->E, 0, wd, sq, cs);
        else k_coverage_col<double><<<g, 256, 0, ctx->st>>>(static_cast<const double*>(ctx->d_sens), ctx->N, ctx->E, 0, wd, sq, cs);
    } else {
        if (f32) k_coverage_col<cf><<<g, 256, 0, ctx->st>>>(static_cast<const cf*>(ctx->d_sens), ctx->N, ctx->E, part, wd, sq, cs);
        else k_coverage_col<cd><<<g, 256, 0, ctx->st>>>(static_cast<const cd*>(ctx->d_sens), ctx->N, ctx->E, part, wd, sq, cs);
    }
    ctx->launches++;
    int e = kernel_check(ctx, "coverage");
    if (!e && cudaMemcpyAsync(csens, cs, sizeof(double) * ctx->E, cudaMemcpyDeviceToHost, ctx->st) != cudaSuccess)
        e = set_err(ctx, CRT_ERR_CUDA, "coverage copy");
    if (!e && cudaStreamSynchronize(ctx->st) != cudaSuccess) e = set_err(ctx, CRT_ERR_CUDA, "coverage sync");
    cudaFree(cs);
    if (w) cudaFree(w);
    return e;
}

extern "C" int32_t crt_set_model(crt_ctx* ctx, const double* par)
{
    if (!ctx || !par) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    if (!ctx->d_par && !dalloc(ctx, &ctx->d_par, (size_t)ctx->E)) return CRT_ERR_ALLOC;
    CK(cudaMemcpyAsync(ctx->d_par, par, sizeof(cd) * ctx->E, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return CRT_OK;
}

extern "C" int32_t crt_get_model(crt_ctx* ctx, double* par)
{
    if (!ctx || !par || !ctx->d_par) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(par, ctx->d_par, sizeof(cd) * ctx->E, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return CRT_OK;
}

extern "C" int32_t crt_model_backup(crt_ctx* ctx, int32_t restore)
{
    if (!ctx || !ctx->d_par) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    if (!ctx->d_par_backup) {
        if (restore) return set_err(ctx, CRT_ERR_ARG, "no model backup");
        if (!dalloc(ctx, &ctx->d_par_backup, (size_t)ctx->E)) return CRT_ERR_ALLOC;
    }
    if (restore)
        CK(cudaMemcpyAsync(ctx->d_par, ctx->d_par_backup, sizeof(cd) * ctx->E, cudaMemcpyDeviceToDevice, ctx->st));
    else
        CK(cudaMemcpyAsync(ctx->d_par_backup, ctx->d_par, sizeof(cd) * ctx->E, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return CRT_OK;
}

extern "C" int32_t crt_update(crt_ctx* ctx, const crt_cg_params* prm, const double* sigmaa, double* par, double* dpar,
                              double* cgfac, double* cgres, int32_t* ncg, double* bdpar)
{
    if (!ctx || !prm || !par) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    if (int e = ensure_cg_buffers(ctx, prm->ncgmax)) return e;
    CK(cudaMemcpyAsync(ctx->d_par, par, sizeof(cd) * ctx->E, cudaMemcpyHostToDevice, ctx->st));
    const cd* d_sa = ctx->d_sigmaa;
    cd* tmp = nullptr;
    if (sigmaa) {
        CK(cudaMalloc((void**)&tmp, sizeof(cd) * ctx->N));
        CK(cudaMemcpyAsync(tmp, sigmaa, sizeof(cd) * ctx->N, cudaMemcpyHostToDevice, ctx->st));
        d_sa = tmp;
    } else if (!ctx->have_forward) {
        return set_err(ctx, CRT_ERR_ARG, "no forward response for crt_update");
    }
    int n_cg = 0;
    int e = update_device(ctx, prm, d_sa, &n_cg);
    if (tmp) cudaFree(tmp);
    if (e) return e;
    CK(cudaMemcpyAsync(par, ctx->d_par, sizeof(cd) * ctx->E, cudaMemcpyDeviceToHost, ctx->st));
    if (dpar) CK(cudaMemcpyAsync(dpar, ctx->d_dpar, sizeof(cd) * ctx->E, cudaMemcpyDeviceToHost, ctx->st));
    if (cgfac) CK(cudaMemcpyAsync(cgfac, ctx->d_cgfac, sizeof(double) * ctx->E, cudaMemcpyDeviceToHost, ctx->st));
    if (cgres) CK(cudaMemcpyAsync(cgres, ctx->d_cgres, sizeof(double) * (n_cg + 1), cudaMemcpyDeviceToHost, ctx->st));
    if (bdpar) CK(cudaMemcpyAsync(bdpar, ctx->d_bdpar, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (ncg) *ncg = n_cg;
    return CRT_OK;
}

// Lambda candidates side by side: update.f90 + cjggra / cjggdc for every
// lambda of a trial set on the same Jacobian, data, response and model.
extern "C" int32_t crt_update_lambdas(crt_ctx* ctx, const crt_cg_params* prm, int32_t nlam, const double* lams,
                                      const double* sigmaa, const double* par, double* par_out, double* dpar,
                                      int32_t* ncg, double* bdpar)
{
    if (!ctx || !prm || !lams || !par || !par_out) return CRT_ERR_ARG;
    if (nlam < 1 || nlam > CGL_MAX) return set_err(ctx, CRT_ERR_ARG, "nlam must be 1 .. 8");
    for (int b = 0; b < nlam; ++b)
        if (!(lams[b] >= 0.0) || !std::isfinite(lams[b]))
            return set_err(ctx, CRT_ERR_ARG, "lambda candidates must be finite and non-negative");
    if (prm->ncgmax < 0) return set_err(ctx, CRT_ERR_ARG, "ncgmax must be non-negative");
    CK(cudaSetDevice(ctx->device));
    if (ctx->ltri < 0) return set_err(ctx, CRT_ERR_ARG, "regulariser not set (crt_set_regularizer)");
    if (!ctx->d_dat) return set_err(ctx, CRT_ERR_ARG, "data not set (crt_set_data)");
    if (!ctx->have_sens) return set_err(ctx, CRT_ERR_ARG, "no Jacobian (crt_jacobian / crt_set_jacobian)");
    if (prm->ldc != ctx->sens_real) return set_err(ctx, CRT_ERR_ARG, "ldc does not match the Jacobian type");
    if (!sigmaa && !ctx->have_forward) return set_err(ctx, CRT_ERR_ARG, "no forward response for crt_update_lambdas");
    if (int e = ensure_cg_buffers(ctx, prm->ncgmax)) return e;
    const size_t M = (size_t)ctx->E, N = (size_t)ctx->N, nl = (size_t)nlam, ns = (size_t)ctx->cg_nsplit;
    const size_t ncr = (size_t)prm->ncgmax + 2;
    // slab: cd vectors first (16-byte aligned), then doubles, then the states
    const size_t n_cd = nl * (8 * M + N + ns * N) + N;   // rhs p r bvec dpar par_out z rold, ap, part; sigmaa
    const size_t n_d = nl * (M + ncr + 1);                // cgfac, cgres, bdpar
    const size_t bytes = n_cd * sizeof(cd) + n_d * sizeof(double) + nl * sizeof(CGState);
    if (ctx->cgl_bytes < bytes) {
        if (ctx->d_cgl) cudaFree(ctx->d_cgl);
        ctx->d_cgl = nullptr;
        ctx->cgl_bytes = 0;
        if (!dalloc(ctx, &ctx->d_cgl, bytes)) return CRT_ERR_ALLOC;
        ctx->cgl_bytes = bytes;
    }
    cd* pc = reinterpret_cast<cd*>(ctx->d_cgl);
    auto take_cd = [&](size_t n) { cd* q = pc; pc += n; return q; };
    cd* v_rhs = take_cd(nl * M);
    cd* v_p = take_cd(nl * M);
    cd* v_r = take_cd(nl * M);
    cd* v_bvec = take_cd(nl * M);
    cd* v_dpar = take_cd(nl * M);
    cd* v_par = take_cd(nl * M);
    cd* v_z = take_cd(nl * M);
    cd* v_rold = take_cd(nl * M);
    cd* v_ap = take_cd(nl * N);
    cd* v_part = take_cd(nl * ns * N);
    cd* v_sa = take_cd(N);
    double* pd = reinterpret_cast<double*>(pc);
    double* v_cgfac = pd;
    double* v_cgres = v_cgfac + nl * M;
    double* v_bdpar = v_cgres + nl * ncr;
    CGState* v_st = reinterpret_cast<CGState*>(v_bdpar + nl);

    CK(cudaMemcpyAsync(ctx->d_par, par, sizeof(cd) * M, cudaMemcpyHostToDevice, ctx->st));
    const cd* d_sa = ctx->d_sigmaa;
    if (sigmaa) {
        CK(cudaMemcpyAsync(v_sa, sigmaa, sizeof(cd) * N, cudaMemcpyHostToDevice, ctx->st));
        d_sa = v_sa;
    }
    crt_cg_params p1 = *prm;
    p1.precond = CRT_PRECOND_JACOBI;
    CGLArgs L{};
    L.a = make_cg_args(ctx, &p1);
    L.a.cgfac = v_cgfac;
    L.a.rhs = v_rhs;
    L.a.p = v_p;
    L.a.r = v_r;
    L.a.bvec = v_bvec;
    L.a.dpar = v_dpar;
    L.a.ap = v_ap;
    L.a.part = v_part;
    L.a.cgres = v_cgres;
    L.a.st = v_st;
    L.a.z = v_z;
    L.a.rold = v_rold;
    L.a.pc = 0;
    L.a.pc_gnn = 0;
    L.a.zb = nullptr;
    L.nl = nlam;
    for (int b = 0; b < nlam; ++b) {
        L.lam[b] = lams[b];
        L.slot[b] = b;
    }
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    launch_cgl_setup(L, ctx->d_dat, d_sa, ctx->d_par, ctx->st);
    ctx->launches += 1;
    // block form: every candidate's S from its cgfac and lambda, factored
    // side by side; a breakdown of any candidate's factor runs the whole
    // batch in the Jacobi form
    bool use_block = false;
    if ((prm->precond == CRT_PRECOND_BLOCK || prm->precond == CRT_PRECOND_BLOCK_GNN) && ctx->spc.ok) {
        if (ctx->spc_c.size() < nl) ctx->spc_c.resize(nl);
        for (size_t b = 0; b < nl; ++b) {
            if (!ctx->spc_c[b].ok)
                if (int e = spc_plan_clone(ctx->spc, ctx->spc_c[b]))
                    return set_err(ctx, e, "block preconditioner buffers of a lambda candidate");
            if (!ctx->cstr[b]) CK(cudaStreamCreateWithFlags(&ctx->cstr[b], cudaStreamNonBlocking));
            if (!ctx->cev_join[b]) CK(cudaEventCreateWithFlags(&ctx->cev_join[b], cudaEventDisableTiming));
        }
        if (!ctx->cev_fork) CK(cudaEventCreateWithFlags(&ctx->cev_fork, cudaEventDisableTiming));
        CK(cudaEventRecord(ctx->cev_fork, ctx->st));
        for (size_t b = 0; b < nl; ++b) {
            CK(cudaStreamWaitEvent(ctx->cstr[b], ctx->cev_fork, 0));
            launch_spc_factor(ctx->spc_c[b], v_cgfac + b * M, ctx->d_smatm, lams[b], ctx->cstr[b]);
            CK(cudaEventRecord(ctx->cev_join[b], ctx->cstr[b]));
            CK(cudaStreamWaitEvent(ctx->st, ctx->cev_join[b], 0));
            ctx->launches += 3 + (ctx->spc.nb > 1 ? 1 : 0);
        }
        std::vector<int> flags(nl, 0);
        for (size_t b = 0; b < nl; ++b)
            CK(cudaMemcpyAsync(&flags[b], ctx->spc_c[b].d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (int e = kernel_check(ctx, "lambda-batch block preconditioner factors")) return e;
        use_block = true;
        for (int f : flags) use_block = use_block && f == 0;
    }
    L.a.pc = use_block ? 1 : 0;
    launch_cgl_init(L, ctx->st);
    ctx->launches += 1;
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    if (int e = kernel_check(ctx, "lambda-batch cg setup")) return e;
    std::vector<CGState> hs(nl);
    int done_iters = 0;
    // iterations between host reads of the candidates' states; at each read
    // the candidates still iterating are compacted into the first positions
    // (fewer slots in the matvecs, fewer sweeps)
    const int batch = 8;
    while (done_iters < prm->ncgmax) {
        const int it = std::min(batch, prm->ncgmax - done_iters);
        if (use_block) {
            for (int k = 0; k < it; ++k) {
                // z = S^-1 r of every active candidate on its stream, then the batched iteration
                CK(cudaEventRecord(ctx->cev_fork, ctx->st));
                for (int q = 0; q < L.nl; ++q) {
                    const size_t b = (size_t)L.slot[q];
                    CK(cudaStreamWaitEvent(ctx->cstr[b], ctx->cev_fork, 0));
                    launch_spc_apply(ctx->spc_c[b], v_r + b * M, v_z + b * M, v_st + b, ctx->cstr[b]);
                    CK(cudaEventRecord(ctx->cev_join[b], ctx->cstr[b]));
                    CK(cudaStreamWaitEvent(ctx->st, ctx->cev_join[b], 0));
                }
                ctx->launches += 2 * L.nl + launch_cgl_iteration_pc(L, ctx->st);
            }
        } else {
            ctx->launches += launch_cgl_iterations(L, it, ctx->st);
        }
        done_iters += it;
        CK(cudaMemcpyAsync(hs.data(), v_st, sizeof(CGState) * nl, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        int na = 0;
        for (int b = 0; b < nlam; ++b)
            if (!hs[b].done) L.slot[na++] = b;
        if (na == 0) break;
        L.nl = na;
    }
    // finish every candidate
    L.nl = nlam;
    for (int b = 0; b < nlam; ++b) L.slot[b] = b;
    if (int e = kernel_check(ctx, "lambda-batch cg iterations")) return e;
    launch_cgl_finish(L, prm->lfpi, prm->step, ctx->d_par, v_par, v_bdpar, ctx->st);
    ctx->launches++;
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    CK(cudaEventSynchronize(ctx->ev[2]));
    float a1 = 0, a2 = 0;
    cudaEventElapsedTime(&a1, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&a2, ctx->ev[1], ctx->ev[2]);
    ctx->timings[4] = a1;
    ctx->timings[5] = a2;
    CK(cudaMemcpyAsync(hs.data(), v_st, sizeof(CGState) * nl, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(par_out, v_par, sizeof(cd) * nl * M, cudaMemcpyDeviceToHost, ctx->st));
    if (dpar) CK(cudaMemcpyAsync(dpar, v_dpar, sizeof(cd) * nl * M, cudaMemcpyDeviceToHost, ctx->st));
    if (bdpar) CK(cudaMemcpyAsync(bdpar, v_bdpar, sizeof(double) * nl, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (ncg)
        for (int b = 0; b < nlam; ++b) ncg[b] = hs[b].ncg;
    ctx->cg_form = use_block ? CRT_PRECOND_BLOCK : CRT_PRECOND_JACOBI;
    return CRT_OK;
}

// ---------------------------------------------------------------------------
// Gauss-Newton step.
namespace {
__global__ void k_exp_model(const cd* par, cd* sigma, int M)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    // sigma = cdexp(par) (src/bsigma.f90)
    const cd p = par[i];
    const double r = exp(p.x);
    double s, c;
    sincos(p.y, &s, &c);
    sigma[i] = cd{r * c, r * s};
}

int gn_step_device(crt_ctx* ctx, const crt_cg_params* prm, int* ncg)
{
    if (!ctx->d_par) return set_err(ctx, CRT_ERR_ARG, "no model (crt_set_model)");
    if (!ctx->d_sigma && !dalloc(ctx, &ctx->d_sigma, (size_t)ctx->E)) return CRT_ERR_ALLOC;
    cudaEvent_t t0 = ctx->ev[7];
    CK(cudaEventRecord(t0, ctx->st));
    k_exp_model<<<(ctx->E + 255) / 256, 256, 0, ctx->st>>>(ctx->d_par, ctx->d_sigma, ctx->E);
    ctx->launches++;
    double tm[CRT_NTIMINGS] = {0};
    int e = forward_common(ctx, prm->ldc, 0, nullptr);
    if (e) return e;
    for (int i = 0; i < 3; ++i) tm[i] = ctx->timings[i];
    for (int i = 7; i < CRT_NTIMINGS; ++i) tm[i] = ctx->timings[i];
    e = jacobian_device(ctx, prm->ldc ? 1 : 0, nullptr);
    if (e) return e;
    tm[3] = ctx->timings[3];
    e = update_device(ctx, prm, ctx->d_sigmaa, ncg);
    if (e) return e;
    tm[4] = ctx->timings[4];
    tm[5] = ctx->timings[5];
    CK(cudaEventRecord(ctx->ev[3], ctx->st));
    CK(cudaEventSynchronize(ctx->ev[3]));
    float tot = 0;
    cudaEventElapsedTime(&tot, t0, ctx->ev[3]);
    tm[6] = tot;
    for (int i = 0; i < CRT_NTIMINGS; ++i) ctx->timings[i] = tm[i];
    return CRT_OK;
}
}  // namespace

extern "C" int32_t crt_gn_step_device(crt_ctx* ctx, const crt_cg_params* prm, int32_t* ncg)
{
    if (!ctx || !prm) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    int n = 0;
    int e = gn_step_device(ctx, prm, &n);
    if (ncg) *ncg = n;
    return e;
}

extern "C" int32_t crt_gn_step(crt_ctx* ctx, const crt_cg_params* prm, double* par, double* sigmaa, double* cgres,
                               int32_t* ncg, double* bdpar)
{
    if (!ctx || !prm || !par) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    if (int e = ensure_cg_buffers(ctx, prm->ncgmax)) return e;
    CK(cudaMemcpyAsync(ctx->d_par, par, sizeof(cd) * ctx->E, cudaMemcpyHostToDevice, ctx->st));
    int n = 0;
    int e = gn_step_device(ctx, prm, &n);
    if (e) return e;
    CK(cudaMemcpyAsync(par, ctx->d_par, sizeof(cd) * ctx->E, cudaMemcpyDeviceToHost, ctx->st));
    if (sigmaa) CK(cudaMemcpyAsync(sigmaa, ctx->d_sigmaa, sizeof(cd) * ctx->N, cudaMemcpyDeviceToHost, ctx->st));
    if (cgres) CK(cudaMemcpyAsync(cgres, ctx->d_cgres, sizeof(double) * (n + 1), cudaMemcpyDeviceToHost, ctx->st));
    if (bdpar) CK(cudaMemcpyAsync(bdpar, ctx->d_bdpar, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (ncg) *ncg = n;
    return CRT_OK;
}

// ---------------------------------------------------------------------------
// Data misfit (src/dmisft.f90:73-137 with chkpo2, lrobust = ldiff = .false.).
extern "C" double crt_dmisft(int32_t nanz, const double* dat, const double* sigmaa, const double* wmatd,
                             const double* wmatdr, const double* wmatdp, int32_t lfpi, int32_t lpol, double* betrms,
                             double* pharms, int32_t* npol)
{
    const double pi = std::acos(-1.0);
    double nrm = 0.0, br = 0.0, ph = 0.0;
    int ok = 0;
    for (int i = 0; i < nanz; ++i) {
        int wdlok = 1;
        double rd = dat[2 * i], id = dat[2 * i + 1], rs = sigmaa[2 * i], is = sigmaa[2 * i + 1];
        int idat = id > pi / 2 ? -1 : (id <= -pi / 2 ? 1 : 0);
        int isig = is > pi / 2 ? -1 : (is <= -pi / 2 ? 1 : 0);
        if (idat == 0 && isig != 0) {
            is += (double)isig * pi;
            if (!lpol) id = id - std::copysign(pi, id);
            wdlok = 0;
        } else if (idat != 0 && isig == 0) {
            if (lpol) id = id + (double)idat * pi;
            wdlok = 0;
        } else if (idat != 0 && isig != 0) {
            is += (double)isig * pi;
            id += (double)idat * pi;
        }
        const double cr = rd - rs, ci = id - is;
        const double psi = lfpi ? std::sqrt(wmatd[i]) * std::fabs(ci) : std::sqrt(wmatd[i]) * std::hypot(cr, ci);
        ok += wdlok;
        nrm += psi * psi * (double)wdlok;
        if (wmatdr) br += wmatdr[i] * (double)wdlok * cr * cr;
        if (wmatdp) ph += wmatdp[i] * (double)wdlok * ci * ci;
    }
    if (npol) *npol = nanz - ok;
    if (ok == 0) return -1.0;
    if (betrms) *betrms = std::sqrt(br / ok);
    if (pharms) *pharms = std::sqrt(ph / ok);
    return std::sqrt(nrm / ok);
}

// ---------------------------------------------------------------------------
// Learned correction of the CG preconditioner (no reference counterpart).

extern "C" int32_t crt_gnn_nparam(void) { return GNN_NPARAM; }

extern "C" int32_t crt_gnn_status(const crt_ctx* ctx, int32_t* available, int32_t* trained, int32_t* form,
                                  int32_t* nrec, int32_t* guard_fired)
{
    if (!ctx) return CRT_ERR_ARG;
    if (available) *available = ctx->gnn.ready;
    if (trained) *trained = ctx->gnn.trained;
    if (form) *form = ctx->gnn.form;
    if (nrec) *nrec = (int32_t)ctx->gnn.recs.size();
    if (guard_fired) *guard_fired = ctx->gnn_guard;
    return CRT_OK;
}

extern "C" int32_t crt_gnn_init(crt_ctx* ctx, uint64_t seed)
{
    if (!ctx) return CRT_ERR_ARG;
    if (!ctx->gnn.ready) return set_err(ctx, CRT_ERR_UNSUPPORTED, "learned preconditioner unavailable (regulariser)");
    CK(cudaSetDevice(ctx->device));
    if (gnn_init(ctx->gnn, seed)) return set_err(ctx, CRT_ERR_CUDA, "learned preconditioner init");
    ctx->gnn.trained = 0;
    return CRT_OK;
}

extern "C" int32_t crt_gnn_set_weights(crt_ctx* ctx, const float* w, int32_t n, int32_t form)
{
    if (!ctx || !w || n != GNN_NPARAM || (form != 0 && form != 1)) return CRT_ERR_ARG;
    if (!ctx->gnn.ready) return set_err(ctx, CRT_ERR_UNSUPPORTED, "learned preconditioner unavailable (regulariser)");
    CK(cudaSetDevice(ctx->device));
    if (gnn_set_weights(ctx->gnn, w)) return set_err(ctx, CRT_ERR_CUDA, "learned preconditioner weights");
    ctx->gnn.trained = 1;
    ctx->gnn.form = form;
    return CRT_OK;
}

extern "C" int32_t crt_gnn_get_weights(crt_ctx* ctx, float* w, int32_t n, int32_t* form)
{
    if (!ctx || !w || n != GNN_NPARAM) return CRT_ERR_ARG;
    if (!ctx->gnn.ready) return set_err(ctx, CRT_ERR_UNSUPPORTED, "learned preconditioner unavailable (regulariser)");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaMemcpy(w, ctx->gnn.d_w, GNN_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    if (form) *form = ctx->gnn.form;
    return CRT_OK;
}

extern "C" int32_t crt_gnn_clear(crt_ctx* ctx)
{
    if (!ctx) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    for (auto& r : ctx->gnn.recs) {
        cudaFree(r.x);
        cudaFree(r.t);
    }
    for (float* p : ctx->gnn.edge_sets) cudaFree(p);
    ctx->gnn.recs.clear();
    ctx->gnn.edge_sets.clear();
    return CRT_OK;
}

// Runs the plain (Jacobi-form) CG of the current Gauss-Newton system -- the
// Jacobian, data, response and model already on the device, as for
// crt_update -- and records every `stride` iterations the residual r_k and
// the iterate x_k; after convergence each record becomes the pair
// (r_k, e_k = x* - x_k) with its base b_k (r_k, or S^-1 r_k when base_block).
// The model is not changed.
extern "C" int32_t crt_gnn_collect(crt_ctx* ctx, const crt_cg_params* prm, int32_t base_block, int32_t stride,
                                   int32_t nmax, int32_t* nrec)
{
    if (!ctx || !prm || stride < 1 || nmax < 1) return CRT_ERR_ARG;
    Gnn& G = ctx->gnn;
    if (!G.ready) return set_err(ctx, CRT_ERR_UNSUPPORTED, "learned preconditioner unavailable (regulariser)");
    if (ctx->ltri < 0) return set_err(ctx, CRT_ERR_ARG, "regulariser not set (crt_set_regularizer)");
    if (!ctx->d_dat) return set_err(ctx, CRT_ERR_ARG, "data not set (crt_set_data)");
    if (!ctx->have_sens) return set_err(ctx, CRT_ERR_ARG, "no Jacobian (crt_jacobian / crt_set_jacobian)");
    if (!ctx->have_forward || !ctx->d_par) return set_err(ctx, CRT_ERR_ARG, "no forward response / model");
    if (prm->ldc != ctx->sens_real) return set_err(ctx, CRT_ERR_ARG, "ldc does not match the Jacobian type");
    if (!G.recs.empty() && G.form != (base_block ? 1 : 0))
        return set_err(ctx, CRT_ERR_ARG, "records of the other base exist (crt_gnn_clear first)");
    if (base_block && !ctx->spc.ok) return set_err(ctx, CRT_ERR_UNSUPPORTED, "block preconditioner unavailable");
    CK(cudaSetDevice(ctx->device));
    if (int e = ensure_cg_buffers(ctx, prm->ncgmax)) return e;
    const int M = ctx->E;
    CGArgs a = make_cg_args(ctx, prm);
    launch_cg_setup(a, ctx->d_dat, ctx->d_sigmaa, ctx->d_par, ctx->st);
    if (base_block) {
        launch_spc_factor(ctx->spc, ctx->d_cgfac, ctx->d_smatm, prm->lam, ctx->st);
        int flag = 0;
        CK(cudaMemcpyAsync(&flag, ctx->spc.d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (flag) return set_err(ctx, CRT_ERR_PIVOT, "block preconditioner breakdown");
    }
    launch_gnn_edges(G, ctx->d_cgfac, ctx->d_smatm, prm->lam, ctx->st);
    float* edges = nullptr;
    CK(cudaMalloc(&edges, (size_t)M * GNN_D * sizeof(float)));
    CK(cudaMemcpyAsync(edges, G.d_a, (size_t)M * GNN_D * sizeof(float), cudaMemcpyDeviceToDevice, ctx->st));
    launch_cg_init(a, ctx->st);
    cd* raw = nullptr;   // [nmax][2][M]: r_k, x_k
    if (cudaMalloc(&raw, (size_t)nmax * 2 * M * sizeof(cd)) != cudaSuccess) {
        cudaFree(edges);
        return set_err(ctx, CRT_ERR_ALLOC, "record buffers");
    }
    int nraw = 0, it = 0;
    CGState hs{};
    while (it < prm->ncgmax) {
        launch_cg_iterations(a, 1, nullptr, nullptr, nullptr, ctx->st);
        ++it;
        if (it % stride == 0 || it % 16 == 0) {
            CK(cudaMemcpyAsync(&hs, ctx->d_cgst, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->st));
            CK(cudaStreamSynchronize(ctx->st));
            if (hs.done) break;
            if (it % stride == 0 && nraw < nmax) {
                CK(cudaMemcpyAsync(raw + (size_t)nraw * 2 * M, ctx->d_r, M * sizeof(cd), cudaMemcpyDeviceToDevice,
                                   ctx->st));
                CK(cudaMemcpyAsync(raw + (size_t)nraw * 2 * M + M, ctx->d_dpar, M * sizeof(cd),
                                   cudaMemcpyDeviceToDevice, ctx->st));
                ++nraw;
            }
        }
    }
    if (int e = kernel_check(ctx, "record CG")) {
        cudaFree(raw);
        cudaFree(edges);
        return e;
    }
    const int sys = (int)G.edge_sets.size();
    G.edge_sets.push_back(edges);
    for (int k = 0; k < nraw; ++k) {
        const cd* rk = raw + (size_t)k * 2 * M;
        const cd* xk = rk + M;
        const cd* bk = nullptr;
        if (base_block) {
            launch_spc_apply(ctx->spc, rk, ctx->d_zb, ctx->d_live, ctx->st);
            bk = ctx->d_zb;
        }
        GnnRecordSet R;
        R.sys = sys;
        if (cudaMalloc(&R.x, (size_t)2 * M * sizeof(cf)) != cudaSuccess ||
            cudaMalloc(&R.t, (size_t)M * sizeof(cf)) != cudaSuccess) {
            cudaFree(R.x);
            cudaFree(raw);
            return set_err(ctx, CRT_ERR_ALLOC, "record buffers");
        }
        launch_gnn_make_record(G, R, rk, bk, xk, ctx->d_dpar, ctx->st);
        double t2 = 0.0;
        CK(cudaMemcpyAsync(&t2, G.d_scal + 2, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        R.tnorm2 = (float)t2;
        if (t2 > 0.0) {
            G.recs.push_back(R);
        } else {
            cudaFree(R.x);
            cudaFree(R.t);
        }
    }
    cudaFree(raw);
    if (int e = kernel_check(ctx, "records")) return e;
    G.form = base_block ? 1 : 0;
    if (nrec) *nrec = (int32_t)G.recs.size();
    return CRT_OK;
}

// Adam on the recorded pairs: `epochs` passes in a seeded random order,
// mini-batches of `batch` records; loss_hist[epoch] = mean record loss.
extern "C" int32_t crt_gnn_train(crt_ctx* ctx, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                                 float* loss_hist)
{
    if (!ctx || epochs < 1 || batch < 1 || !(lr > 0.0f)) return CRT_ERR_ARG;
    Gnn& G = ctx->gnn;
    if (!G.ready) return set_err(ctx, CRT_ERR_UNSUPPORTED, "learned preconditioner unavailable (regulariser)");
    if (G.recs.empty()) return set_err(ctx, CRT_ERR_ARG, "no records (crt_gnn_collect)");
    CK(cudaSetDevice(ctx->device));
    const int nr = (int)G.recs.size();
    std::vector<int> order(nr);
    for (int i = 0; i < nr; ++i) order[i] = i;
    unsigned long long st = seed ^ 0x9e3779b97f4a7c15ULL;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int i = nr - 1; i > 0; --i) {   // Fisher-Yates with a 64-bit LCG
            st = st * 6364136223846793005ULL + 1442695040888963407ULL;
            const int j = (int)((st >> 33) % (unsigned long long)(i + 1));
            std::swap(order[i], order[j]);
        }
        CK(cudaMemsetAsync(G.d_scal + 1, 0, sizeof(double), ctx->st));
        for (int b0 = 0; b0 < nr; b0 += batch) {
            const int b1 = std::min(nr, b0 + batch);
            for (int q = b0; q < b1; ++q) launch_gnn_record_grad(G, G.recs[order[q]], 1.0f / (b1 - b0), ctx->st);
            launch_gnn_adam(G, lr, ctx->st);
        }
        double L = 0.0;
        CK(cudaMemcpyAsync(&L, G.d_scal + 1, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (int e = kernel_check(ctx, "training")) return e;
        if (loss_hist) loss_hist[ep] = (float)(L / nr);
    }
    G.trained = 1;
    return CRT_OK;
}

// One record's data (for checking the network against a CPU restatement):
// x [M][4] features, t [M][2] target, a [M][4] message weights, nbr [M][4]
// neighbours (-1 none), |t|^2.  Any output may be NULL.
extern "C" int32_t crt_gnn_record(crt_ctx* ctx, int32_t idx, float* x, float* t, float* a, int32_t* nbr,
                                  float* tnorm2)
{
    if (!ctx) return CRT_ERR_ARG;
    Gnn& G = ctx->gnn;
    if (idx < 0 || idx >= (int)G.recs.size()) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    const GnnRecordSet& R = G.recs[idx];
    const size_t M = G.M;
    if (x) CK(cudaMemcpy(x, R.x, M * 2 * sizeof(cf), cudaMemcpyDeviceToHost));
    if (t) CK(cudaMemcpy(t, R.t, M * sizeof(cf), cudaMemcpyDeviceToHost));
    if (a) CK(cudaMemcpy(a, G.edge_sets[R.sys], M * GNN_D * sizeof(float), cudaMemcpyDeviceToHost));
    if (nbr) CK(cudaMemcpy(nbr, G.d_nbr, M * GNN_D * sizeof(int), cudaMemcpyDeviceToHost));
    if (tnorm2) *tnorm2 = R.tnorm2;
    return CRT_OK;
}

// Loss and weight gradient of one record with the current weights (the
// weights are not changed).
extern "C" int32_t crt_gnn_record_grad(crt_ctx* ctx, int32_t idx, float* grad, double* loss)
{
    if (!ctx || !grad) return CRT_ERR_ARG;
    Gnn& G = ctx->gnn;
    if (idx < 0 || idx >= (int)G.recs.size()) return CRT_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemsetAsync(G.d_g, 0, GNN_NPARAM * sizeof(float), ctx->st));
    CK(cudaMemsetAsync(G.d_scal + 1, 0, sizeof(double), ctx->st));
    launch_gnn_record_grad(G, G.recs[idx], 1.0f, ctx->st);
    CK(cudaMemcpyAsync(grad, G.d_g, GNN_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    double L = 0.0;
    CK(cudaMemcpyAsync(&L, G.d_scal + 1, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaMemsetAsync(G.d_g, 0, GNN_NPARAM * sizeof(float), ctx->st));
    if (int e = kernel_check(ctx, "record gradient")) return e;
    if (loss) *loss = L;
    return CRT_OK;
}

// ---------------------------------------------------------------------------
// Batches of independent instances under one CUDA graph.
//
// Every context keeps its own stream, device data and workspaces.  The first
// crt_batch_run runs each context's forward (and Jacobian) once eagerly --
// which allocates the workspaces and autotunes the band panel width for
// every (precision, mb) of the batch -- and then captures all of them into
// one graph: the batch stream records a fork event that every context
// stream waits on, each context enqueues its forward and Jacobian with host
// synchronisation, timing reads and allocation switched off, and the batch
// stream joins all context streams again.  The instances are independent
// branches of the graph, so uneven instances fill the SMs side by side; a
// replay is one cudaGraphLaunch.  Per-system status words are read after
// the replay.
struct crt_batch {
    int device = 0;
    std::vector<crt_ctx*> ctx;
    int ldc = 0, jac = -1;
    cudaStream_t st = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<int> status;
    std::string err;
};

namespace {
int batch_enqueue(crt_batch* b, crt_ctx* c)
{
    int e = forward_common(c, b->ldc, 0, nullptr);
    if (!e && b->jac >= 0) e = jacobian_device(c, b->jac, nullptr);
    return e;
}

void batch_release(crt_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}
}  // namespace

extern "C" crt_batch* crt_batch_create(crt_ctx* const* ctxs, int32_t count, int32_t ldc, int32_t jacobian_mode,
                                       int32_t* err)
{
    auto fail = [&](int code) -> crt_batch* {
        if (err) *err = code;
        return nullptr;
    };
    if (!ctxs || count < 1 || jacobian_mode < -1 || jacobian_mode > 2) return fail(CRT_ERR_ARG);
    for (int i = 0; i < count; ++i)
        if (!ctxs[i] || ctxs[i]->device != ctxs[0]->device) return fail(CRT_ERR_ARG);
    if (jacobian_mode == 1 && !ldc) return fail(CRT_ERR_ARG);   // bsendc belongs to the DC forward
    auto* b = new crt_batch();
    b->device = ctxs[0]->device;
    b->ctx.assign(ctxs, ctxs + count);
    b->ldc = ldc != 0;
    b->jac = jacobian_mode;
    b->status.assign(count, 0);
    bool ok = cudaSetDevice(b->device) == cudaSuccess &&
              cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreate(&b->t0) == cudaSuccess && cudaEventCreate(&b->t1) == cudaSuccess;
    b->join.assign(count, nullptr);
    for (int i = 0; ok && i < count; ++i)
        ok = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        crt_batch_destroy(b);
        return fail(CRT_ERR_CUDA);
    }
    if (err) *err = CRT_OK;
    return b;
}

extern "C" void crt_batch_destroy(crt_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    batch_release(b);
    for (cudaEvent_t e : b->join)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->t0) cudaEventDestroy(b->t0);
    if (b->t1) cudaEventDestroy(b->t1);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

extern "C" const char* crt_batch_error(const crt_batch* b) { return b ? b->err.c_str() : "no batch"; }

extern "C" int32_t crt_batch_set_models(crt_batch* b, const double* const* sigma)
{
    if (!b || !sigma) return CRT_ERR_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return CRT_ERR_CUDA;
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        crt_ctx* ctx = b->ctx[i];
        if (!sigma[i]) return CRT_ERR_ARG;
        if (!ctx->d_sigma && !dalloc(ctx, &ctx->d_sigma, (size_t)ctx->E)) return CRT_ERR_ALLOC;
        CK(cudaMemcpyAsync(ctx->d_sigma, sigma[i], sizeof(cd) * ctx->E, cudaMemcpyHostToDevice, ctx->st));
    }
    for (crt_ctx* ctx : b->ctx) CK(cudaStreamSynchronize(ctx->st));
    return CRT_OK;
}

extern "C" int32_t crt_batch_run(crt_batch* b, double* ms)
{
    if (!b) return CRT_ERR_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return CRT_ERR_CUDA;
    for (crt_ctx* c : b->ctx)
        if (!c->d_sigma) {
            b->err = "crt_batch_run before crt_batch_set_models";
            return CRT_ERR_ARG;
        }
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        b->err = std::string(what) + ": " + cudaGetErrorString(e);
        return CRT_ERR_CUDA;
    };
    if (!b->exec) {
        // eager pass: allocations, panel autotuning, status of every instance
        for (size_t i = 0; i < b->ctx.size(); ++i) {
            if (int e = batch_enqueue(b, b->ctx[i])) {
                b->err = "instance " + std::to_string(i) + ": " + b->ctx[i]->err;
                return e;
            }
        }
        cudaError_t ce = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal);
        if (ce != cudaSuccess) return cuda_fail(ce, "begin capture");
        int failed = 0;
        ce = cudaEventRecord(b->fork, b->st);
        for (size_t i = 0; ce == cudaSuccess && !failed && i < b->ctx.size(); ++i) {
            crt_ctx* c = b->ctx[i];
            ce = cudaStreamWaitEvent(c->st, b->fork, 0);
            if (ce != cudaSuccess) break;
            c->capture = 1;
            const int e = batch_enqueue(b, c);
            c->capture = 0;
            if (e) {
                b->err = "capturing instance " + std::to_string(i) + ": " + c->err;
                failed = e;
                break;
            }
            ce = cudaEventRecord(b->join[i], c->st);
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->st, b->join[i], 0);
        }
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(b->st, &g);
        if (failed || ce != cudaSuccess || ee != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            if (failed) return failed;
            return cuda_fail(ce != cudaSuccess ? ce : ee, "graph capture");
        }
        b->graph = g;
        ce = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (ce != cudaSuccess) {
            batch_release(b);
            return cuda_fail(ce, "graph instantiate");
        }
    }
    cudaError_t ce = cudaEventRecord(b->t0, b->st);
    if (ce == cudaSuccess) ce = cudaGraphLaunch(b->exec, b->st);
    if (ce == cudaSuccess) ce = cudaEventRecord(b->t1, b->st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(b->t1);
    if (ce != cudaSuccess) return cuda_fail(ce, "graph launch");
    float t = 0.0f;
    cudaEventElapsedTime(&t, b->t0, b->t1);
    if (ms) *ms = t;
    int first = CRT_OK;
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        crt_ctx* c = b->ctx[i];
        b->status[i] = collect_status(c, c->nstatus);
        if (b->status[i] == CRT_OK) {
            c->last_ldc = b->ldc;
            c->have_forward = 1;
            c->have_sens = b->jac >= 0;
        } else if (first == CRT_OK) {
            first = b->status[i];
            b->err = "instance " + std::to_string(i) + ": " + c->err;
        }
    }
    return first;
}

extern "C" int32_t crt_batch_status(const crt_batch* b, int32_t i)
{
    if (!b || i < 0 || i >= (int)b->ctx.size()) return CRT_ERR_ARG;
    return b->status[i];
}

extern "C" int32_t crt_batch_results(crt_batch* b, int32_t i, double* volt, double* sigmaa, double* sens)
{
    if (!b || i < 0 || i >= (int)b->ctx.size()) return CRT_ERR_ARG;
    crt_ctx* ctx = b->ctx[i];
    if (!ctx->have_forward) return set_err(ctx, CRT_ERR_ARG, "no batch result for this instance");
    CK(cudaSetDevice(ctx->device));
    if (volt) CK(cudaMemcpyAsync(volt, ctx->d_volt, sizeof(cd) * ctx->N, cudaMemcpyDeviceToHost, ctx->st));
    if (sigmaa) CK(cudaMemcpyAsync(sigmaa, ctx->d_sigmaa, sizeof(cd) * ctx->N, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (sens) {
        if (!ctx->have_sens) return set_err(ctx, CRT_ERR_ARG, "the batch computes no Jacobian");
        return download_sens(ctx, sens);
    }
    return CRT_OK;
}

extern "C" int32_t crt_set_workspace_limit(crt_ctx* ctx, int64_t bytes)
{
    if (!ctx || bytes < 0) return CRT_ERR_ARG;
    ctx->ws_budget = (size_t)bytes;
    return CRT_OK;
}
