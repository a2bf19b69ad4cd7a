// Persistent converge! engine: one CTA per system runs the whole aasol loop.
//
// Every fixed-point evaluation and every Anderson step of a system happens
// inside one thread block, separated by __syncthreads instead of kernel
// launches; the batch is ONE launch whose blocks finish independently (each
// system stops at its own aasol exit, the launch ends with the slowest one).
// The circulant taps, the periodically extended convolution inputs, the
// weighted densities / dPhi/dn and the adjoint partial sums live in shared
// memory; the Anderson vectors (sol, gx, res, df, Q, DG) stay in global
// memory (L2-resident at these sizes).  Arithmetic and operation order are
// the ones of the grid engine (kernels.cuh), so both engines follow the same
// aasol trajectory.
#pragma once
#include <cooperative_groups.h>
#include "kernels.cuh"

#define PERS_THREADS 384
#define PERS_WARPS (PERS_THREADS / 32)
#define PERS_R 8
#define PERS_TILE (32 * PERS_R)
#define PERS_MAX_M 8           // Anderson depth bound of the persistent engine (deeper: grid engine)

// extended periodic window of one convolution input: logical ext[k] = in[(k - OFF) mod N],
// k < EXTN; OFF is a multiple of 16.  The FP64 (tensor-core) path stores logical element k at
// pers_pos(k) = k + 4 floor(k / 16): a warp's 8 x 4 B-fragment loads then fall on each
// double-wide bank pair exactly twice (2 wavefronts, the minimum for 32 doubles).  Rows are
// pers_extp(N) long.  Taps of a field are stored with PERS_TPAD zeros on either side.
#define PERS_TPAD 16
__host__ __device__ __forceinline__ int pers_off(int N) { return (N + 32 + 15) & ~15; }
__host__ __device__ __forceinline__ int pers_extn(int N) { return pers_off(N) + N + 32 * (PERS_R + 1) + 16; }
__host__ __device__ __forceinline__ int pers_pos(int k) { return k + 4 * (k >> 4); }
__host__ __device__ __forceinline__ int pers_extp(int N) { return pers_extn(N) + 4 * ((pers_extn(N) + 15) >> 4); }
__host__ __device__ __forceinline__ int pers_ts(int N) { return N + 2 * PERS_TPAD; }

__host__ __device__ __forceinline__ size_t pers_smem_bytes(int N, int nc, int nconv, int NF, size_t esz)
{
    return esz * ((size_t)nc * nconv * pers_ts(N)      // taps (zero-padded)
                  + (size_t)nc * nconv * pers_extp(N)  // extended inputs
                  + (size_t)nc * NF * N                // n, then dPhi/dn
                  + (size_t)nc * nconv * N);           // adjoint partials
}

// byte offset of the shared-memory Anderson vectors, and their size for n_elem
// elements and m history columns (rho, sol, gx, res, df, V_ext, Q row-major, DG)
__host__ __device__ __forceinline__ size_t pers_vec_offset(int N, int nc, int nconv, int NF, size_t esz)
{
    return (pers_smem_bytes(N, nc, nconv, NF, esz) + 15) & ~(size_t)15;
}
// row stride of the shared-memory QR history: m rounded up to even (16-byte aligned rows)
__host__ __device__ __forceinline__ int pers_qs(int m) { return m + (m & 1); }
__host__ __device__ __forceinline__ size_t pers_vec_bytes(int n_elem, int m)
{
    return sizeof(double) * (size_t)n_elem * (6 + (size_t)pers_qs(m) + (size_t)m);
}

// Sums of K per-thread values over the block into sums[0..K), for thread 0 only: the
// caller lets thread 0 consume them and then synchronises the block.  Threads with
// index >= active hold exact zeros (they had no element); their warps skip the shuffles
// and store +0.0, which is what the shuffles would give, so the sums do not change.
template <int BLOCK>
__device__ __forceinline__ void block_reduce_to_smem(double* vals, int K, double* sums, int active)
{
    __shared__ double red[BLOCK / 32][RED_SLOTS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp * 32 < active) {
#pragma unroll
        for (int c = 0; c < RED_SLOTS; ++c) {
            if (c >= K) break;
            double v = vals[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][c] = v;
        }
    } else if (lane < K) {
        red[warp][lane] = 0.0;
    }
    __syncthreads();
    if (threadIdx.x < K) {   // warp 0
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < BLOCK / 32; ++w) s += red[w][threadIdx.x];
        sums[threadIdx.x] = s;
    }
    __syncwarp();
}

// all circulant convolutions of one stage: out[(i*nconv+f)*N + j] = scale * sum_q taps_if[q] in_if[j-q]
//
// A warp owns PERS_TILE = 32 * PERS_R outputs of one field; lane l accumulates
// j = j0 + 32 r (r < PERS_R).  For each residue q0 = q mod 32 the inputs
// in[j0 + 32 r - q] form a window that moves by one register per q += 32; the
// window is a ring of PERS_R registers whose rotation is resolved at compile time
// (the q loop is unrolled by PERS_R), so a step is one tap load, one window load
// and PERS_R independent FMAs.
// The fields f = frank, frank + fstride, ... of the stage (a cluster of fstride CTAs splits
// the fields between them); out2, when not null, receives a second copy of every output
// (the peer CTA's buffer).
template <typename T, int NC>
__device__ __forceinline__ void pers_conv(const T* __restrict__ ext, bool shared_input, const T* __restrict__ taps,
                                          T* __restrict__ out, int out_comp_stride, int N, int nconv, T scale,
                                          int frank, int fstride, T* out2)
{
    const int lane = threadIdx.x & 31;
    const int EXTN = pers_extp(N), OFF = pers_off(N);   // FP32 rows: logical positions, row stride extp
    const int ntiles = (N + PERS_TILE - 1) / PERS_TILE;
    const int nfm = (nconv - frank + fstride - 1) / fstride;
    const int ntask = NC * nfm * ntiles;
    for (int task = threadIdx.x >> 5; task < ntask; task += PERS_WARPS) {
        const int tile = task % ntiles;
        const int f = ((task / ntiles) % nfm) * fstride + frank;
        const int i = task / (ntiles * nfm);
        const T* in = ext + (size_t)(shared_input ? i : i * nconv + f) * EXTN + OFF;
        const T* tp = taps + (size_t)(i * nconv + f) * pers_ts(N) + PERS_TPAD;
        const int j0 = tile * PERS_TILE + lane;
        T acc[PERS_R];
#pragma unroll
        for (int r = 0; r < PERS_R; ++r) acc[r] = T(0);
        const int q0_end = min(32, N);
        for (int q0 = 0; q0 < q0_end; ++q0) {
            T W[PERS_R];   // W[r] = in[j0 + 32 r - q] at the start of each unrolled block
#pragma unroll
            for (int r = 0; r < PERS_R; ++r) W[r] = in[j0 + 32 * r - q0];
            for (int q = q0; q < N; q += 32 * PERS_R) {
#pragma unroll
                for (int s = 0; s < PERS_R; ++s) {
                    const int qs = q + 32 * s;
                    if (qs < N) {
                        const T t = tp[qs];
#pragma unroll
                        for (int r = 0; r < PERS_R; ++r) acc[r] = fma(t, W[(r - s + PERS_R) % PERS_R], acc[r]);
                        // the slot of output r = PERS_R-1 is free: it takes the input of step s+1, output 0
                        W[PERS_R - 1 - s] = in[j0 - qs - 32];
                    }
                }
            }
        }
        const size_t ob = (size_t)i * out_comp_stride + (size_t)f * N;
#pragma unroll
        for (int r = 0; r < PERS_R; ++r) {
            const int j = j0 + 32 * r;
            if (j < N) {
                const T v = acc[r] * scale;
                out[ob + j] = v;
                if (out2) out2[ob + j] = v;
            }
        }
    }
}

// FP64 tensor-core form of pers_conv (mma.sync m8n8k4 f64; the FP64 tensor path
// of sm_100a).  With e[k] = in[k] the periodic extension and outputs grouped as
// OUT[a][u] = out[8u + a] (a < 8):
//   OUT[a][u] = sum_d sum_{c<8} t(8d + a - c) e[8(u - d) + c],  t(q) = 0 outside [0, N)
// i.e. OUT = sum_d A_d B_d with A_d an 8x8 Toeplitz block of taps and
// B_d[c][u] = e[8(u - d) + c] an 8-column slab of the extended input.  A warp owns
// 8 columns (64 outputs) of one field and runs the k = (d, c) loop as 2 D mma of
// k = 4 into two accumulators (c < 4, c >= 4).  Every q in [0, N) is visited once
// per output, so the result is the circulant up to summation order.
// (dmma_m8n8k4 is defined in kernels.cuh.)

// Extended inputs at bank-spread positions (pers_pos), taps zero-padded: the loop has no
// bounds test.  The d loop runs two tap blocks per step into four independent accumulator
// pairs (even / odd d, c < 4 / c >= 4), summed at the end.
template <int NC>
__device__ __forceinline__ void pers_conv_dmma(const double* __restrict__ ext, bool shared_input,
                                               const double* __restrict__ taps, double* __restrict__ out,
                                               int out_comp_stride, int N, int nconv, double scale, int frank,
                                               int fstride, double* out2)
{
    const int lane = threadIdx.x & 31;
    const int EXTP = pers_extp(N), OFF = pers_off(N), TS = pers_ts(N);
    const int U = (N + 7) / 8;          // 8-output columns
    const int nut = (U + 7) / 8;        // warp tiles of 8 columns
    const int D = (N + 14) / 8;         // tap blocks: 8 (D - 1) + 7 >= N - 1
    const int nfm = (nconv - frank + fstride - 1) / fstride;   // fields of this CTA: f = frank + fstride fl
    const int ntask = NC * nfm * nut;
    const int r = lane >> 2, k = lane & 3;   // A row / C row, A column / B row
    for (int task = threadIdx.x >> 5; task < ntask; task += PERS_WARPS) {
        const int ut = task % nut;
        const int f = ((task / nut) % nfm) * fstride + frank;
        const int i = task / (nut * nfm);
        const double* tp = taps + (size_t)(i * nconv + f) * TS + PERS_TPAD;   // tp[q] = 0 outside [0, N)
        const double* in = ext + (size_t)(shared_input ? i : i * nconv + f) * EXTP;
        const int u0 = ut * 8;
        double c0 = 0.0, c1 = 0.0, e0 = 0.0, e1 = 0.0, g0 = 0.0, g1 = 0.0, h0 = 0.0, h1 = 0.0;
        // B: e[8 (u0 + r - d) + c] at logical OFF + 8 (u0 + r) + c - 8 d; A: t(8 d + r - c)
        const int xb = OFF + 8 * (u0 + r) + k;
        int d = 0;
        for (; d + 1 < D; d += 2) {
            const int q0 = 8 * d + r - k;
            const int x0 = xb - 8 * d, x1 = x0 - 8;
            const double a0 = tp[q0], a1 = tp[q0 - 4], a2 = tp[q0 + 8], a3 = tp[q0 + 4];
            const double b0 = in[pers_pos(x0)], b1 = in[pers_pos(x0 + 4)];
            const double b2 = in[pers_pos(x1)], b3 = in[pers_pos(x1 + 4)];
            dmma_m8n8k4(c0, c1, a0, b0);
            dmma_m8n8k4(e0, e1, a1, b1);
            dmma_m8n8k4(g0, g1, a2, b2);
            dmma_m8n8k4(h0, h1, a3, b3);
        }
        if (d < D) {
            const int q0 = 8 * d + r - k;
            const int x0 = xb - 8 * d;
            dmma_m8n8k4(c0, c1, tp[q0], in[pers_pos(x0)]);
            dmma_m8n8k4(e0, e1, tp[q0 - 4], in[pers_pos(x0 + 4)]);
        }
        const size_t ob = (size_t)i * out_comp_stride + (size_t)f * N;
        const int j0 = 8 * (u0 + 2 * k) + r, j1 = j0 + 8;
        const double v0 = ((c0 + e0) + (g0 + h0)) * scale, v1 = ((c1 + e1) + (g1 + h1)) * scale;
        if (j0 < N) {
            out[ob + j0] = v0;
            if (out2) out2[ob + j0] = v0;
        }
        if (j1 < N) {
            out[ob + j1] = v1;
            if (out2) out2[ob + j1] = v1;
        }
    }
}

template <typename T, int NC>
__device__ __forceinline__ void pers_conv_any(const T* __restrict__ ext, bool shared_input, const T* __restrict__ taps,
                                              T* __restrict__ out, int out_comp_stride, int N, int nconv, T scale,
                                              int frank, int fstride, T* out2)
{
    if constexpr (sizeof(T) == 8)
        pers_conv_dmma<NC>(ext, shared_input, taps, out, out_comp_stride, N, nconv, scale, frank, fstride, out2);
    else
        pers_conv<T, NC>(ext, shared_input, taps, out, out_comp_stride, N, nconv, scale, frank, fstride, out2);
}

// The Anderson section of one fixed-point step (the QR downdate and the vector slots
// between two evaluations) on one warp: each slot's partial sums are reduced by
// shuffles and lane 0 applies the step, so the slots need no block barrier.  For the
// small systems of a batch (a few hundred elements per system) the slots are bound by
// those barriers and the serial control step, not by the element loops.
__device__ __forceinline__ void pers_anderson_warp(const SysDev& S, AAState& A, double* sums, int* done_counter,
                                                   int lane)
{
    for (int slot = 1; slot <= N_VEC_SLOTS; ++slot) {
        const int op = A.op[slot];
        if (op == OP_NONE) break;
        double acc[RED_SLOTS];
#pragma unroll
        for (int k = 0; k < RED_SLOTS; ++k) acc[k] = 0.0;
        const int K = vec_op_range<PERS_MAX_M>(op, S, A, lane, S.n_elem, 32, acc);
        if (K > 0) {
#pragma unroll
            for (int c = 0; c < RED_SLOTS; ++c) {
                if (c >= K) break;
                double v = acc[c];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) sums[c] = v;
            }
            __syncwarp();
            if (lane == 0) ctl_apply(A, op, slot, sums, done_counter, true);
            __syncwarp();
            if (A.pad0) {   // the next step's QR downdate, from this step's R
                aa_downdate_warp(A, lane);
                if (lane == 0) A.pad0 = 0;
            }
        }
        __syncwarp();
    }
}

// warp_aa_max_elem: a system of at most this many elements (N * nc) runs the Anderson
// section on warp 0 (pers_anderson_warp), a larger one on the whole block.  The choice
// depends on the system alone, so a system gets the same arithmetic alone or in a batch.
//
// CL = 2: a cluster of two CTAs per system (launched with cluster dimension 2; only with
// the Anderson vectors in shared memory).  The convolution tasks and the Phi points are
// split between the two CTAs; each writes its results into its own shared memory and into
// the peer's (distributed shared memory), and a cluster barrier follows each of the three
// stages.  The Euler-Lagrange step and the Anderson section run in both CTAs on identical
// data, so both hold the same solver state and take the same branches; every value is
// computed by the same code as with CL = 1, so the results are bit for bit the same.
// Rank 0 alone writes the state, the profile and the done count back.
template <typename T, int NC, int ND, int CL>
__global__ void __launch_bounds__(PERS_THREADS, 1)
persistent_kernel(const SysDev* __restrict__ sys, AAState* __restrict__ st, int* done_counter, int max_evals,
                  int vec_m, int warp_aa_max_elem)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ AAState sA;
    __shared__ SysDev sS;
    __shared__ double sums[RED_SLOTS];
    __shared__ int done_local;
    constexpr int NF = 6 + ND, NCONV = 5 + ND;
    const int rank = (CL == 2) ? (int)(blockIdx.x & 1u) : 0;
    const int sid = (CL == 2) ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    int* done_ptr = rank == 0 ? done_counter : &done_local;
    const SysDev& G = sys[sid];
    const int N = G.N, n_elem = G.n_elem;
    const int EXTN = pers_extn(N), EXTP = pers_extp(N), OFF = pers_off(N), TS = pers_ts(N);
    const int tid = threadIdx.x;
    T* taps = reinterpret_cast<T*>(smem_raw);
    T* ext = taps + (size_t)NC * NCONV * TS;
    T* nf = ext + (size_t)NC * NCONV * EXTP;
    T* ip = nf + (size_t)NC * NF * N;
    if (tid == 0) {
        sA = st[sid];
        sS = G;
        done_local = 0;
    }
    // the peer CTA's copies of the stage buffers (CL = 2), and the stage split
    T* nf_peer = nullptr;
    T* ip_peer = nullptr;
    if constexpr (CL == 2) {
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        nf_peer = cl.map_shared_rank(nf, rank ^ 1);
        ip_peer = cl.map_shared_rank(ip, rank ^ 1);
    }
    auto stage_sync = [&]() {
        if constexpr (CL == 2) cooperative_groups::this_cluster().sync();
        else __syncthreads();
    };
    {
        const T* src = (sizeof(T) == 8) ? reinterpret_cast<const T*>(G.taps) : reinterpret_cast<const T*>(G.taps32);
        for (int k = tid; k < NC * NCONV * TS; k += PERS_THREADS) {
            const int slot = k / TS, q = k - slot * TS - PERS_TPAD;
            taps[k] = (q >= 0 && q < N) ? src[(size_t)slot * N + q] : T(0);
        }
    }
    // vec_m >= 0: the Anderson vectors (rho, sol, gx, res, df, V_ext, vec_m columns
    // of Q and of DG) live in shared memory after the convolution buffers; rho and
    // sol are read in here and written back at the end.
    double* vs = reinterpret_cast<double*>(smem_raw + pers_vec_offset(N, NC, NCONV, NF, sizeof(T)));
    if (vec_m >= 0) {
        for (int e = tid; e < n_elem; e += PERS_THREADS) {
            vs[e] = G.rho[e];
            vs[n_elem + e] = G.sol[e];
            vs[5 * n_elem + e] = G.vext ? G.vext[e] : 0.0;
        }
        // gx, res, df and the history start at zero (the solver writes them before it reads
        // them; defined contents keep the two CTAs of a cluster bit-identical regardless)
        for (size_t e = tid; e < 3 * (size_t)n_elem; e += PERS_THREADS) vs[2 * (size_t)n_elem + e] = 0.0;
        const size_t nhist = ((size_t)pers_qs(vec_m) + (size_t)vec_m) * n_elem;
        for (size_t e = tid; e < nhist; e += PERS_THREADS) vs[6 * (size_t)n_elem + e] = 0.0;
    }
    __syncthreads();
    if (vec_m >= 0 && tid == 0) {
        sS.rho = vs;
        sS.sol = vs + n_elem;
        sS.gx = vs + 2 * (size_t)n_elem;
        sS.res = vs + 3 * (size_t)n_elem;
        sS.df = vs + 4 * (size_t)n_elem;
        if (G.vext) sS.vext = vs + 5 * (size_t)n_elem;
        sS.Q = vs + 6 * (size_t)n_elem;
        sS.qs = pers_qs(vec_m);
        sS.DG = vs + (6 + (size_t)pers_qs(vec_m)) * n_elem;
    }
    __syncthreads();
    const SysDev& S = sS;
    const T NA = T(S.NA);
    const bool warp_aa = n_elem <= warp_aa_max_elem;
    for (int it = 0; it < max_evals; ++it) {
        if (sA.mode == MODE_DONE) break;
        // ---- weighted densities (evaluate_field!) ----
        for (int k = tid; k < NC * EXTN; k += PERS_THREADS) {
            const int i = k / EXTN, u = k - i * EXTN;
            int j = (u - OFF) % N;
            j += (j < 0) ? N : 0;
            ext[(size_t)i * EXTP + (sizeof(T) == 8 ? pers_pos(u) : u)] = T(S.rho[i * N + j]);
        }
        for (int e = tid; e < n_elem; e += PERS_THREADS) {
            const int i = e / N, j = e - i * N;
            nf[(i * NF) * N + j] = T(S.NA * S.rho[e]);
        }
        __syncthreads();
        pers_conv_any<T, NC>(ext, true, taps, nf + N, NF * N, N, NCONV, NA, rank, CL,
                             nf_peer ? nf_peer + N : nullptr);
        stage_sync();
        // ---- fused Phi / dPhi/dn, in place: two threads per point ----
        // items j < N: hard sphere + association (fields 1 .. 2 + ND); items N + j: chain +
        // dispersion (fields 0, 3 + ND .. 5 + ND).  The two halves read and write disjoint
        // fields, and they fall in different warps except around item N.
        // (CL = 2: rank 0 takes the hard-sphere halves, rank 1 the chain + dispersion halves)
        const int w_end = (CL == 2) ? (rank + 1) * N : 2 * N;
        for (int w = ((CL == 2) ? rank * N : 0) + tid; w < w_end; w += PERS_THREADS) {
            const bool first = w < N;
            const int j = first ? w : w - N;
            T n[NC][NF], g[NC][NF];
#pragma unroll
            for (int i = 0; i < NC; ++i)
#pragma unroll
                for (int a = 0; a < NF; ++a) {
                    const bool mine = (a >= 1 && a <= 2 + ND) == first;
                    n[i][a] = mine ? nf[(i * NF + a) * N + j] : T(1);
                }
            if (first) phi_grad<T, NC, ND, false, 1>(S.phi, n, g);
            else phi_grad<T, NC, ND, false, 2>(S.phi, n, g);
#pragma unroll
            for (int i = 0; i < NC; ++i)
#pragma unroll
                for (int a = 0; a < NF; ++a)
                    if ((a >= 1 && a <= 2 + ND) == first) {
                        nf[(i * NF + a) * N + j] = g[i][a];
                        if (nf_peer) nf_peer[(i * NF + a) * N + j] = g[i][a];
                    }
        }
        stage_sync();
        // ---- adjoint convolutions (integrate_field!) ----
        {
            // the extended inputs of this CTA's fields only (f = rank + CL fl)
            constexpr int NFM0 = (NCONV + CL - 1) / CL;
            const int nfm = (NCONV - rank + CL - 1) / CL;
            for (int k = tid; k < NC * NFM0 * EXTN; k += PERS_THREADS) {
                const int ms = k / EXTN, u = k - ms * EXTN;
                const int i = ms / NFM0, fl = ms - i * NFM0;
                if (fl >= nfm) continue;
                const int f = fl * CL + rank, slot = i * NCONV + f;
                int j = (u - OFF) % N;
                j += (j < 0) ? N : 0;
                ext[(size_t)slot * EXTP + (sizeof(T) == 8 ? pers_pos(u) : u)] = nf[(i * NF + f + 1) * N + j];
            }
            __syncthreads();
            pers_conv_any<T, NC>(ext, false, taps, ip, NCONV * N, N, NCONV, T(1), rank, CL, ip_peer);
        }
        stage_sync();
        // ---- Euler-Lagrange step + aa_point! bookkeeping ----
        {
            const int mode = sA.mode;
            const double beta = (mode == MODE_EVAL_PICARD) ? sA.picard_beta : sA.beta;
            const bool aa = (mode == MODE_EVAL_AA);
            double* DGs = (aa && sA.m > 0) ? S.DG + (size_t)sA.dg_slot * n_elem : nullptr;
            double ss[1] = {0.0};
            for (int e = tid; e < n_elem; e += PERS_THREADS) {
                const int i = e / N, j = e - i * N;
                double dF = double(nf[(i * NF) * N + j]);
#pragma unroll
                for (int f = 0; f < NCONV; ++f) {
                    const double v = double(ip[(i * NCONV + f) * N + j]);
                    if (f >= 2 && f < 2 + ND) dF -= v;
                    else dF += v;
                }
                if (S.vext) dF += S.vext[e];
                ss[0] += el_elem(S, e, i, dF, beta, aa, DGs);
            }
            block_reduce_to_smem<PERS_THREADS>(ss, 1, sums, n_elem);
            if (tid == 0) ctl_apply(sA, -1, 0, sums, done_ptr, true);
            __syncthreads();
        }
        // ---- Anderson vector slots ----
        if (warp_aa) {
            if (tid < 32) pers_anderson_warp(S, sA, sums, done_ptr, tid);
            __syncthreads();
            continue;
        }
        for (int slot = 1; slot <= N_VEC_SLOTS; ++slot) {
            const int op = sA.op[slot];
            if (op == OP_NONE) break;
            double acc[RED_SLOTS];
#pragma unroll
            for (int k = 0; k < RED_SLOTS; ++k) acc[k] = 0.0;
            const int K = vec_op_range<PERS_MAX_M>(op, S, sA, tid, n_elem, PERS_THREADS, acc);
            if (K > 0) {
                block_reduce_to_smem<PERS_THREADS>(acc, K, sums, n_elem);
                if (tid == 0) ctl_apply(sA, op, slot, sums, done_ptr, true);
            }
            __syncthreads();
            if (sA.pad0) {   // the next step's QR downdate, from this step's R, by one thread
                __syncthreads();
                if (tid == 0) {
                    aa_downdate_fast(sA);
                    sA.pad0 = 0;
                }
                __syncthreads();
            }
        }
    }
    if (vec_m >= 0 && rank == 0) {
        for (int e = tid; e < n_elem; e += PERS_THREADS) {
            G.rho[e] = S.rho[e];
            G.sol[e] = S.sol[e];
        }
    }
    if (tid == 0 && rank == 0) st[sid] = sA;
    // no CTA of a cluster leaves while its peer may still write into its shared memory
    if constexpr (CL == 2) cooperative_groups::this_cluster().sync();
}
