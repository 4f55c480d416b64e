// crt_gnn.h -- learned correction of the CG preconditioner (no counterpart
// in the reference, whose CG is preconditioned by cgfac alone).
//
// A mesh graph network over the model cells, with the regulariser's
// neighbour graph and, as message weights, the off-diagonal entries
// a_ij = lam C_i R_ij C_j of the scaled sparse operator S:
//   x_i  = [Re r_i, Im r_i, Re b_i, Im b_i] * s      (b = base(r), s = 1 / rms(r))
//   h0_i = tanh(Win^T x_i)
//   h_l,i = tanh(Ws_l^T h_{l-1},i + Wn_l^T sum_j a_ij h_{l-1},j),  l = 1..3
//   z_i  = b_i + (Wout^T h3_i) / s                     (complex: the two outputs)
// Width 32, no biases: tanh is odd and the input is normalised, so the
// correction is an odd, degree-1 homogeneous map of r (z(alpha r) = alpha z(r)
// for real alpha), which keeps the preconditioned CG scale-invariant.  The
// base is the identity (the cgfac-scaled system has a unit diagonal) or the
// block preconditioner S^-1.  Weights are kept as an FP32 master copy for
// training and rounded to bf16 for every forward pass; all sums are FP32.
//
// Training data are (residual, error) pairs of the plain (Jacobi-form) CG:
// every `stride` iterations r_k and the iterate x_k are recorded, and after
// convergence e_k = x* - x_k, so A e_k = r_k.  The loss of a record is
// |z(r_k) - e_k|^2 / |e_k - b_k|^2 in the normalised units.
#pragma once

#include <vector>

#include "crt_common.cuh"

constexpr int GNN_W = 32;          // channels
constexpr int GNN_L = 3;           // message-passing layers
constexpr int GNN_F = 4;           // input features
constexpr int GNN_O = 2;           // outputs (Re, Im)
constexpr int GNN_D = 4;           // max neighbours per cell
// flat parameter layout, all matrices [in][out]:
//   Win [F][W] | (Ws_l [W][W], Wn_l [W][W]) for l = 1..L | Wout [W][O]
constexpr int GNN_OFF_IN = 0;
constexpr int GNN_OFF_L = GNN_F * GNN_W;
constexpr int GNN_LSTRIDE = 2 * GNN_W * GNN_W;
constexpr int GNN_OFF_OUT = GNN_OFF_L + GNN_L * GNN_LSTRIDE;
constexpr int GNN_NPARAM = GNN_OFF_OUT + GNN_W * GNN_O;

struct CGState;
struct SpcPlan;

struct GnnRecordSet {
    int sys = 0;          // index into the edge-weight sets
    cf *x = nullptr;      // [M][2] normalised features r s and b s (interleaved complex pairs)
    cf *t = nullptr;      // [M] normalised target (e - b) s
    float tnorm2 = 0.0f;  // |t|^2
};

struct Gnn {
    int M = 0, ready = 0, trained = 0, form = -1;   // form: base of the training records (0 identity, 1 block)
    int* d_nbr = nullptr;            // [M][D] neighbour cell or -1
    int* d_nsm = nullptr;            // [M][D] smatm index of the coupling
    float* d_a = nullptr;            // [M][D] message weights of the current system
    float* d_w = nullptr;            // [NPARAM] FP32 master weights
    unsigned short* d_wb = nullptr;  // [NPARAM] bf16 weights of the forward pass
    float *d_m = nullptr, *d_v = nullptr, *d_g = nullptr;   // Adam moments, gradient
    float* d_part = nullptr;         // per-block gradient partials
    int nblk = 0;
    float* d_h = nullptr;            // [(L+1)][M][W] activations
    float* d_agg = nullptr;          // [L][M][W] aggregated messages
    float* d_du = nullptr;           // [2][M][W] backward work
    float* d_x = nullptr;            // [M][4] features of the current application
    float* d_out = nullptr;          // [M][2] network output
    double* d_scal = nullptr;        // [4] scale and loss scratch
    int t_adam = 0;
    std::vector<float*> edge_sets;   // message weights of recorded systems
    std::vector<GnnRecordSet> recs;
};

// Host set-up from the regulariser (same graph as the block preconditioner).
int gnn_setup(Gnn& G, int M, int ltri, int nx, int nnb, const int* nachbar);
void gnn_free(Gnn& G);
// Seeded Glorot-uniform initialisation (output layer near zero), or given
// FP32 master weights; both reset the optimiser.
int gnn_init(Gnn& G, unsigned long long seed);
int gnn_set_weights(Gnn& G, const float* w);
// Message weights a_ij = lam C_i R_ij C_j of the current system into G.d_a.
void launch_gnn_edges(const Gnn& G, const double* cgfac, const double* smatm, double lam, cudaStream_t s);
// z = base + correction(r, base); base = r (zb == nullptr) or zb.  Skipped
// once the CG state reports done (st may be nullptr).
void launch_gnn_apply(Gnn& G, const cd* r, const cd* zb, cd* z, const CGState* st, cudaStream_t s);
// One record: forward with stored activations, loss, backward; adds the
// weight gradient (scaled by gscale) to G.d_g and the loss to G.d_scal[1].
void launch_gnn_record_grad(Gnn& G, const GnnRecordSet& R, float gscale, cudaStream_t s);
// Adam step on G.d_w from G.d_g (then clears G.d_g), bf16 copy to G.d_wb.
void launch_gnn_adam(Gnn& G, float lr, cudaStream_t s);
// bf16 copy of the master weights.
void launch_gnn_round(Gnn& G, cudaStream_t s);
// Records of one Jacobi-form CG run: rk, xk (complex128, device), the final
// iterate xs and the base of each rk (nullptr: identity).
void launch_gnn_make_record(Gnn& G, GnnRecordSet& R, const cd* rk, const cd* bk, const cd* xk, const cd* xs,
                            cudaStream_t s);
