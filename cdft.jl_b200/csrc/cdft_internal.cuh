// Internal device/host structures of libcdft_b200.
//
// Memory model: every system (one DFTSystem of the reference) owns contiguous
// device buffers; a "batch" is a device array of SysDev records plus task and
// chunk lists, so every kernel launch covers all systems of the batch.
// Vectors follow the reference's Julia layout (grid fastest, then field,
// then component): element e = i*N + j of component i at grid point j.
#pragma once
#include <cstdint>
#include "../../include/cdft_b200.h"

#define CDFT_NF_MAX 9          // 6 + nd fields, nd <= 3
#define CDFT_NCONV_MAX 8       // NF - 1 convolved fields

// 1D circulant convolution tiling (see conv1d_kernel)
#define CONV_R 4               // outputs per thread (strided by 32)
#define CONV_WARPS 4
#define CONV_TILE (CONV_WARPS * 32 * CONV_R)   // outputs per block
#define CONV_QC 1024           // taps per block (split-K chunk)

// vector (Anderson) chunking
#define ELEM_CHUNK 1024        // elements per block of the vector kernels
#define ELEM_THREADS 256
#define POINT_THREADS 128      // points per block of the pointwise Phi kernel
#define RED_SLOTS (CDFT_MAX_M + 2)   // partial sums per chunk

// solver modes (the phase of aasol a system is in when its next G evaluation runs)
enum { MODE_EVAL_INIT = 0, MODE_EVAL_PICARD = 1, MODE_EVAL_AA = 2, MODE_DONE = 3 };

// vector-slot operations between two fixed-point evaluations (see ctl_kernel): the CGS2
// QR update of aa_qr_update! (anderson.jl:498-540) in three passes over the elements, and
// the solution update
enum {
    OP_NONE = 0,
    OP_NORM_DF = 1,        // partial ||df||^2 (first column of the QR factor)
    OP_DOT_H1 = 2,         // partial h1 = Q^T df
    OP_SUB_DOT_NORM = 3,   // df <- df - Q h1; partial h2 = Q^T df and ||df||^2
    OP_SETQ_DOT_TRES = 4,  // q = (df - Q h2) / r; partial [Q q]^T res; store q, or [Q q] Qx
                           // when the next step starts with the QR downdate
    OP_SOL_AA = 5,         // sol = gx - DG theta; rho = exp(sol)
    OP_SOL_COPY = 6        // sol = gx; rho = exp(sol)
};
#define N_VEC_SLOTS 4

struct PhiParams {
    int nc, nd;
    double T;
    double m[CDFT_MAX_NC];
    double d[CDFT_MAX_NC];                       // reduced hard-sphere diameters d_i / L
    double c1[CDFT_MAX_NC * CDFT_MAX_NC];        // m_i m_j (sigma_ij/L)^3 eps_ij/T
    double c2[CDFT_MAX_NC * CDFT_MAX_NC];        // c1 * eps_ij/T
    int has_assoc, a_ic, a_jc;                   // has_assoc: number of pairs (1: analytic, >1: general)
    double a_nia, a_njb, a_dij, a_K;             // d_ij (reduced) and (sigma_ij/L)^3 (exp(eps/T)-1) kappa
    // several pairs (assoc.jl:771-828): sites s < a_ns of component g_sc[s], multiplicity g_sm[s];
    // pair p bonds site g_pa[p] (multiplicity g_nia[p]) with g_pb[p] (g_njb[p])
    int a_ns;
    int g_sc[CDFT_MAX_SITES];
    double g_sm[CDFT_MAX_SITES];
    int g_pa[CDFT_MAX_ASSOC], g_pb[CDFT_MAX_ASSOC];
    double g_nia[CDFT_MAX_ASSOC], g_njb[CDFT_MAX_ASSOC], g_dij[CDFT_MAX_ASSOC], g_K[CDFT_MAX_ASSOC];
};

struct SysDev {
    int nd, N, nc, NF, nconv;
    int ngrid[3];
    int ksplit;                  // split-K factor of the 1D circulant convolutions
    int n_elem;                  // N * nc
    int mixed;                   // 1: FP32 convolution/Phi buffers
    int chunk_begin, chunk_count;  // element chunks of this system (reductions)
    double NA;                   // N_A L^3
    double cprd[CDFT_MAX_NC];    // mu_res + ln rho_bulk
    PhiParams phi;
    // tables
    const double* taps;          // [(i*nconv+f)*N + q] = Re(IDFT(omega_hat))[q]
    const float* taps32;
    const double* vext;          // [e] or nullptr
    // work buffers
    double* rho;                 // exp(sol)
    double* sol;
    double* gx;
    double* res;
    double* df;
    double* Q;                   // QR history, row-major: [e*qs + c]
    double* DG;                  // [slot*n_elem + e]
    int qs;                      // row stride of Q (doubles, even: rows start 16-byte aligned)
    void* part;                  // convolution partials [((i*nconv+f)*ksplit+ks)*N + j] (double or float)
    void* dfield;                // dPhi/dn [(i*NF+a)*N + j] (double or float)
    double* fval;                // Phi per point
    double* out;                 // scratch output (functional derivative)
    void* adj;                   // 3D: adjoint sum sum_f ±omega_f * dPhi/dn_f per element (T), else nullptr
    const double* mats;          // radial grids: dense operators [(stage*nc + i)*nconv + f][j][q], else nullptr
    const double* qw;            // radial grids: quadrature weights of the integral, else nullptr (Simpson)
    double wscale;               // Cartesian grids: product over dimensions of dz / 3 (Simpson)
};

struct AAState {
    int mode, k, picard_it, nevals;
    int errcode, idid, toosoon, m;
    int maxit, picard_maxit;
    int head, dg_slot, kq, mk;
    int downdate;                // the next Anderson step starts from the downdated QR (Rn, Qx)
    int pad0;                    // persistent engine: a warp-parallel downdate is pending
    int op[N_VEC_SLOTS + 1];
    double beta, picard_beta, rtol, atol, picard_rtol, picard_atol;
    double resnorm, tol, picard_tol, up_bd;
    double rnorm;                // norm of the vector being orthonormalised
    double coef[CDFT_MAX_M];     // coefficients of the current slot op
    double h1[CDFT_MAX_M];
    double R[CDFT_MAX_M * CDFT_MAX_M];     // column-major m x m
    double Rn[CDFT_MAX_M * CDFT_MAX_M];    // the downdated R of the next step (column-major m x m)
    double Qx[CDFT_MAX_M * CDFT_MAX_M];    // column-major m x (m-1)
    double tau[CDFT_MAX_M], v1[CDFT_MAX_M];  // Householder reflectors of the downdate
    double* history;
    int history_cap, pad1;
};

struct ConvTask {
    int sys, comp, field, tile_ks;   // tile_ks = tile * ksplit + ks
};

struct Chunk {
    int sys, begin;
};
