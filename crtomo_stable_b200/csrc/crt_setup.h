// crt_setup.h -- set-up stage (wavenumbers, element matrices, mixed-boundary
// coefficients, gather lists for the streamed assembly).
#pragma once

#include <stdint.h>

#include <vector>

#include "crt_common.cuh"

// Host view of the mesh in the reference's layout (src/elemmod.f90):
// nrel(ntot, maxnodes) column-major with 1-based node numbers.
struct MeshHost {
    int sanz, mb, typanz, elanz, relanz, maxnodes, ntot;
    const int32_t *typ, *nelanz, *selanz, *nrel, *rnr, *snr;
    const double *sx, *sy;
};

// Gather form of kompab (src/kompab.f90:80-128): row r owns entries
// ent [row_ptr[r], row_ptr[r+1]); entry e sits at band offset ent_d[e]
// (column r - d) and sums contributions [ent_ptr[e], ent_ptr[e+1]) in element
// order.  A contribution code >= 0 indexes elbg[k] (e*nmn + imn); a code < 0
// is -(rel*3 + imn) - 1 for a mixed-boundary segment (relbg * kg).  con_sig
// is the element whose conductivity multiplies the coefficient.
struct AssemblyLists {
    std::vector<int> row_ptr, ent_d, ent_ptr, con_code, con_sig;
    int max_row_entries = 0;
};

struct SetupArgs {
    int E, R, K, L, maxnodes, nmn, nmixed;
    const int* nrel0;     // [ntot][maxnodes] 0-based node numbers
    const int* snr0;      // [sanz] 0-based coordinate rows
    const int* etyp;      // [E] element type
    const int* enk;       // [E] nodes per element
    const int* enr0;      // [L] 0-based electrode nodes
    const int* mixed_rel; // [nmixed] 0-based boundary indices of type-11 segments
    const double *sx, *sy, *kwn;
    double sytop;
    double* elbg;         // [K][E][nmn]
    double* relbg;        // [R][3]
    double* kg;           // [K][L][R]
    int* status;
};

__global__ void k_elem_matrices(SetupArgs A);
__global__ void k_beta(SetupArgs A);
__host__ __device__ double crt_bessk0(double x);
__host__ __device__ double crt_bessk1(double x);

int crt_rwaven_host(int nanz, const int32_t* strnr, const int32_t* vnr, const int32_t* enr,
                    const int32_t* snr, const double* sx, const double* sy, int32_t* kwnanz,
                    double* kwn, double* kwnwi, double* amin, double* amax);
double crt_sytop_host(const MeshHost& m);
int build_assembly_lists(const MeshHost& m, AssemblyLists& out);
