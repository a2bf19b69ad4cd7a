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
#include "kernels.cuh"

#define PERS_THREADS 384
#define PERS_WARPS (PERS_THREADS / 32)
#define PERS_R 4
#define PERS_TILE (32 * PERS_R)

// extended periodic window of one convolution input: ext[k] = in[(k - OFF) mod N]
__host__ __device__ __forceinline__ int pers_extn(int N) { return 2 * N + 32 * (PERS_R + 2); }
__host__ __device__ __forceinline__ int pers_off(int N) { return N + 32; }

__host__ __device__ __forceinline__ size_t pers_smem_bytes(int N, int nc, int nconv, int NF, size_t esz)
{
    return esz * ((size_t)nc * nconv * N              // taps
                  + (size_t)nc * nconv * pers_extn(N)  // extended inputs
                  + (size_t)nc * NF * N                // n, then dPhi/dn
                  + (size_t)nc * nconv * N);           // adjoint partials
}

template <int BLOCK>
__device__ __forceinline__ void block_reduce_to_smem(double* vals, int K, double* sums)
{
    __shared__ double red[BLOCK / 32][RED_SLOTS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = 0; c < K; ++c) {
        double v = vals[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < BLOCK / 32; ++w) s += red[w][threadIdx.x];
        sums[threadIdx.x] = s;
    }
    __syncthreads();
}

// all circulant convolutions of one stage: out[(i*nconv+f)*N + j] = scale * sum_q taps_if[q] in_if[j-q]
template <typename T, int NC>
__device__ __forceinline__ void pers_conv(const T* __restrict__ ext, bool shared_input, const T* __restrict__ taps,
                                          T* __restrict__ out, int out_comp_stride, int N, int nconv, T scale)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int EXTN = pers_extn(N), OFF = pers_off(N);
    const int ntiles = (N + PERS_TILE - 1) / PERS_TILE;
    const int ntask = NC * nconv * ntiles;
    for (int task = warp; task < ntask; task += PERS_WARPS) {
        const int tile = task % ntiles;
        const int f = (task / ntiles) % nconv;
        const int i = task / (ntiles * nconv);
        const T* in = ext + (size_t)(shared_input ? i : i * nconv + f) * EXTN + OFF;
        const T* tp = taps + (size_t)(i * nconv + f) * N;
        const int j0 = tile * PERS_TILE + lane;
        T acc[PERS_R];
#pragma unroll
        for (int r = 0; r < PERS_R; ++r) acc[r] = T(0);
        const int q0_end = min(32, N);
        for (int q0 = 0; q0 < q0_end; ++q0) {
            T W[PERS_R];
#pragma unroll
            for (int r = 0; r < PERS_R; ++r) W[r] = in[j0 + 32 * r - q0];
            for (int q = q0; q < N; q += 32) {
                const T t = tp[q];
#pragma unroll
                for (int r = 0; r < PERS_R; ++r) acc[r] = fma(t, W[r], acc[r]);
#pragma unroll
                for (int r = PERS_R - 1; r > 0; --r) W[r] = W[r - 1];
                W[0] = in[j0 - q - 32];
            }
        }
        T* o = out + (size_t)i * out_comp_stride + (size_t)f * N;
#pragma unroll
        for (int r = 0; r < PERS_R; ++r) {
            const int j = j0 + 32 * r;
            if (j < N) o[j] = acc[r] * scale;
        }
    }
}

template <typename T, int NC, int ND>
__global__ void __launch_bounds__(PERS_THREADS, 1)
persistent_kernel(const SysDev* __restrict__ sys, AAState* __restrict__ st, int* done_counter, int max_evals)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ AAState sA;
    __shared__ double sums[RED_SLOTS];
    constexpr int NF = 6 + ND, NCONV = 5 + ND;
    const SysDev& S = sys[blockIdx.x];
    const int N = S.N, n_elem = S.n_elem;
    const int EXTN = pers_extn(N), OFF = pers_off(N);
    const int tid = threadIdx.x;
    T* taps = reinterpret_cast<T*>(smem_raw);
    T* ext = taps + (size_t)NC * NCONV * N;
    T* nf = ext + (size_t)NC * NCONV * EXTN;
    T* ip = nf + (size_t)NC * NF * N;
    if (tid == 0) sA = st[blockIdx.x];
    {
        const T* src = (sizeof(T) == 8) ? reinterpret_cast<const T*>(S.taps) : reinterpret_cast<const T*>(S.taps32);
        for (int k = tid; k < NC * NCONV * N; k += PERS_THREADS) taps[k] = src[k];
    }
    __syncthreads();
    const T NA = T(S.NA);
    for (int it = 0; it < max_evals; ++it) {
        if (sA.mode == MODE_DONE) break;
        // ---- weighted densities (evaluate_field!) ----
        for (int k = tid; k < NC * EXTN; k += PERS_THREADS) {
            const int i = k / EXTN, u = k - i * EXTN;
            int j = (u - OFF) % N;
            j += (j < 0) ? N : 0;
            ext[k] = T(S.rho[i * N + j]);
        }
        for (int e = tid; e < n_elem; e += PERS_THREADS) {
            const int i = e / N, j = e - i * N;
            nf[(i * NF) * N + j] = T(S.NA * S.rho[e]);
        }
        __syncthreads();
        pers_conv<T, NC>(ext, true, taps, nf + N, NF * N, N, NCONV, NA);
        __syncthreads();
        // ---- fused Phi / dPhi/dn, in place ----
        for (int j = tid; j < N; j += PERS_THREADS) {
            T n[NC][NF], g[NC][NF];
#pragma unroll
            for (int i = 0; i < NC; ++i)
#pragma unroll
                for (int a = 0; a < NF; ++a) n[i][a] = nf[(i * NF + a) * N + j];
            phi_grad<T, NC, ND>(S.phi, n, g);
#pragma unroll
            for (int i = 0; i < NC; ++i)
#pragma unroll
                for (int a = 0; a < NF; ++a) nf[(i * NF + a) * N + j] = g[i][a];
        }
        __syncthreads();
        // ---- adjoint convolutions (integrate_field!) ----
        for (int k = tid; k < NC * NCONV * EXTN; k += PERS_THREADS) {
            const int slot = k / EXTN, u = k - slot * EXTN;
            const int i = slot / NCONV, f = slot - i * NCONV;
            int j = (u - OFF) % N;
            j += (j < 0) ? N : 0;
            ext[k] = nf[(i * NF + f + 1) * N + j];
        }
        __syncthreads();
        pers_conv<T, NC>(ext, false, taps, ip, NCONV * N, N, NCONV, T(1));
        __syncthreads();
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
            block_reduce_to_smem<PERS_THREADS>(ss, 1, sums);
            if (tid == 0) ctl_apply(sA, -1, 0, sums, done_counter);
            __syncthreads();
        }
        // ---- Anderson vector slots ----
        for (int slot = 1; slot <= N_VEC_SLOTS; ++slot) {
            const int op = sA.op[slot];
            if (op == OP_NONE) break;
            double acc[RED_SLOTS];
#pragma unroll
            for (int k = 0; k < RED_SLOTS; ++k) acc[k] = 0.0;
            const int K = vec_op_range(op, S, sA, tid, n_elem, PERS_THREADS, acc);
            if (K > 0) {
                block_reduce_to_smem<PERS_THREADS>(acc, K, sums);
                if (tid == 0) ctl_apply(sA, op, slot, sums, done_counter);
            }
            __syncthreads();
        }
    }
    if (tid == 0) st[blockIdx.x] = sA;
}
