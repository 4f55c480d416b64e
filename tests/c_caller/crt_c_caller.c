/*
 * crt_c_caller.c -- a plain C99 caller of include/crt_b200.h, as a Fortran
 * driver's ISO_C_BINDING calls would reach it: no Python, no ctypes.
 *
 * Test program: tests/test_c_caller.py writes the inputs of one tomodir
 * (mesh, electrodes, readings, conductivities, regulariser, data) to a
 * record file, runs this program, and compares what it writes back with the
 * FP64 oracle.  The sequence is the first pass of the CRTomo loop
 * (src/inv.f90): rwaven (crt_rwaven), precal + ALLOCATEs (crt_create), the
 * forward + rtrafo + bvolti (crt_forward), bsensi (crt_jacobian), the
 * regulariser and data (crt_set_regularizer, crt_set_data), dmisft
 * (crt_dmisft) and update + cjggra (crt_update), then crt_destroy.
 *
 * Record file: a sequence of records, each an int64 byte count followed by
 * that many bytes, in the order read below (and written on output).
 *
 *     crt_c_caller <inputs> <outputs>
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "crt_b200.h"

static void* read_rec(FILE* f, int64_t* nbytes)
{
    int64_t n = 0;
    if (fread(&n, sizeof n, 1, f) != 1 || n < 0) {
        fprintf(stderr, "crt_c_caller: truncated input\n");
        exit(2);
    }
    void* p = malloc(n > 0 ? (size_t)n : 1);
    if (!p || (n > 0 && fread(p, 1, (size_t)n, f) != (size_t)n)) {
        fprintf(stderr, "crt_c_caller: truncated input\n");
        exit(2);
    }
    if (nbytes) *nbytes = n;
    return p;
}

static int32_t read_i32(FILE* f)
{
    int64_t n = 0;
    int32_t* p = (int32_t*)read_rec(f, &n);
    int32_t v = n == 4 ? p[0] : -1;
    free(p);
    return v;
}

static double read_f64(FILE* f)
{
    int64_t n = 0;
    double* p = (double*)read_rec(f, &n);
    double v = n == 8 ? p[0] : 0.0;
    free(p);
    return v;
}

static void write_rec(FILE* f, const void* p, int64_t nbytes)
{
    fwrite(&nbytes, sizeof nbytes, 1, f);
    if (nbytes) fwrite(p, 1, (size_t)nbytes, f);
}

static int fail(const char* what, int32_t errnr, crt_ctx* ctx)
{
    fprintf(stderr, "crt_c_caller: %s: errnr %d (%s)\n", what, (int)errnr, ctx ? crt_last_error(ctx) : "");
    if (ctx) crt_destroy(ctx);
    return errnr ? (int)errnr : 1;
}

int main(int argc, char** argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: crt_c_caller <inputs> <outputs>\n");
        return 2;
    }
    if (crt_abi_version() != CRT_B200_ABI_VERSION) {
        fprintf(stderr, "crt_c_caller: header ABI %d, library ABI %d\n", CRT_B200_ABI_VERSION, (int)crt_abi_version());
        return 2;
    }
    FILE* in = fopen(argv[1], "rb");
    if (!in) return 2;
    crt_mesh mesh;
    memset(&mesh, 0, sizeof mesh);
    mesh.sanz = read_i32(in);
    mesh.typanz = read_i32(in);
    mesh.mb = read_i32(in);
    mesh.typ = (const int32_t*)read_rec(in, NULL);
    mesh.nelanz = (const int32_t*)read_rec(in, NULL);
    mesh.selanz = (const int32_t*)read_rec(in, NULL);
    mesh.snr = (const int32_t*)read_rec(in, NULL);
    mesh.sx = (const double*)read_rec(in, NULL);
    mesh.sy = (const double*)read_rec(in, NULL);
    mesh.nrel = (const int32_t*)read_rec(in, NULL);
    mesh.rnr = (const int32_t*)read_rec(in, NULL);
    const int32_t elanz = read_i32(in);
    int64_t nb = 0;
    crt_survey sv;
    memset(&sv, 0, sizeof sv);
    sv.enr = (const int32_t*)read_rec(in, &nb);
    sv.eanz = (int32_t)(nb / 4);
    sv.strnr = (const int32_t*)read_rec(in, &nb);
    sv.nanz = (int32_t)(nb / 4);
    sv.vnr = (const int32_t*)read_rec(in, NULL);
    double* sigma = (double*)read_rec(in, NULL);   /* complex [elanz] */
    const int32_t ltri = read_i32(in), nx = read_i32(in), nnb = read_i32(in);
    double* smatm = (double*)read_rec(in, NULL);
    int32_t* nachbar = (int32_t*)read_rec(in, &nb);
    double* dat = (double*)read_rec(in, NULL);     /* complex [nanz] */
    double* wmatd = (double*)read_rec(in, NULL);
    crt_cg_params prm;
    memset(&prm, 0, sizeof prm);
    prm.lam = read_f64(in);
    prm.eps = read_f64(in);
    prm.ncgmax = read_i32(in);
    prm.step = 1.0;
    prm.precond = CRT_PRECOND_JACOBI;
    fclose(in);

    /* src/rwaven.f90: wavenumbers and weights on the host */
    double kwn[30], kwnwi[30];
    int32_t kwnanz = 0;
    int32_t e = crt_rwaven(&mesh, sv.eanz, sv.enr, sv.nanz, sv.strnr, sv.vnr, &kwnanz, kwn, kwnwi);
    if (e) return fail("crt_rwaven", e, NULL);
    sv.kwnanz = kwnanz;
    sv.swrtr = 1;
    sv.kwn = kwn;
    sv.kwnwi = kwnwi;

    int32_t err = 0;
    crt_ctx* ctx = crt_create(0, &mesh, &sv, CRT_PREC_FP64, &err);
    if (!ctx) return fail("crt_create", err, NULL);

    const size_t N = (size_t)sv.nanz, M = (size_t)elanz;
    double* volt = (double*)calloc(2 * N, sizeof(double));
    double* sigmaa = (double*)calloc(2 * N, sizeof(double));
    double* sens = (double*)calloc(2 * N * M, sizeof(double));
    double* par = (double*)calloc(2 * M, sizeof(double));
    double* dpar = (double*)calloc(2 * M, sizeof(double));
    double* cgfac = (double*)calloc(M, sizeof(double));
    double* cgres = (double*)calloc((size_t)prm.ncgmax + 2, sizeof(double));
    if (!volt || !sigmaa || !sens || !par || !dpar || !cgfac || !cgres) return fail("allocation", 97, ctx);

    if ((e = crt_forward(ctx, sigma, 0, 0, NULL, volt, sigmaa, NULL))) return fail("crt_forward", e, ctx);
    if ((e = crt_jacobian(ctx, 0, NULL, sens))) return fail("crt_jacobian", e, ctx);
    if ((e = crt_set_regularizer(ctx, ltri, nx, nnb, smatm, nachbar))) return fail("crt_set_regularizer", e, ctx);
    if ((e = crt_set_data(ctx, dat, wmatd, NULL))) return fail("crt_set_data", e, ctx);
    double betrms = 0.0, pharms = 0.0;
    int32_t npol = 0;
    const double nrmsd = crt_dmisft(sv.nanz, dat, sigmaa, wmatd, NULL, NULL, 0, 0, &betrms, &pharms, &npol);
    /* par = log(sigma) */
    for (size_t j = 0; j < M; ++j) {
        const double re = sigma[2 * j], im = sigma[2 * j + 1];
        par[2 * j] = 0.5 * log(re * re + im * im);
        par[2 * j + 1] = atan2(im, re);
    }
    int32_t ncg = 0;
    double bdpar = 0.0;
    if ((e = crt_update(ctx, &prm, NULL, par, dpar, cgfac, cgres, &ncg, &bdpar))) return fail("crt_update", e, ctx);
    int32_t form = -1;
    crt_cg_info(ctx, &form, NULL, NULL);
    crt_destroy(ctx);

    FILE* out = fopen(argv[2], "wb");
    if (!out) return 2;
    write_rec(out, &kwnanz, 4);
    write_rec(out, kwn, 8 * (int64_t)kwnanz);
    write_rec(out, kwnwi, 8 * (int64_t)kwnanz);
    write_rec(out, volt, 16 * (int64_t)N);
    write_rec(out, sigmaa, 16 * (int64_t)N);
    write_rec(out, sens, 16 * (int64_t)(N * M));
    write_rec(out, &nrmsd, 8);
    write_rec(out, par, 16 * (int64_t)M);
    write_rec(out, dpar, 16 * (int64_t)M);
    write_rec(out, cgfac, 8 * (int64_t)M);
    write_rec(out, &ncg, 4);
    write_rec(out, &bdpar, 8);
    write_rec(out, &form, 4);
    fclose(out);
    printf("crt_c_caller: ok (sanz %d, eanz %d, nanz %d, kwnanz %d, ncg %d)\n", (int)mesh.sanz, (int)sv.eanz,
           (int)sv.nanz, (int)kwnanz, (int)ncg);
    return 0;
}
