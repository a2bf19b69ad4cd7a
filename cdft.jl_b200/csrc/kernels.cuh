// Device kernels of the converge! path (1D Cartesian engine).
//
// One fixed-point evaluation G(x) (GFix!, src/methods/converge.jl:235-242) is
//   conv1d_kernel(stage 0)  weighted densities n_alpha  (evaluate_field!, fields.jl:26-48)
//   phi_kernel              dPhi/dn_alpha, Phi          (δFδρ_res! AD stage, models.jl:145-179)
//   conv1d_kernel(stage 1)  adjoint convolutions        (integrate_field!, fields.jl:50-61)
//   el_kernel               ln G = mu - dF/drho - Vext, clamp, Anderson bookkeeping
//                           (get_new_profile!, converge.jl:108-153; aa_point!/betafix!,
//                            anderson.jl:470-491)
// followed by up to five vector slots (vec_kernel) interleaved with one-warp
// control kernels (ctl_kernel) that run aasol's state machine
// (anderson.jl:301-443) and the QR update/downdate (anderson.jl:498-583).
#pragma once
#include "cdft_internal.cuh"
#include "functional.cuh"

__device__ __forceinline__ bool sys_active(const AAState* st, int s)
{
    return st == nullptr || st[s].mode != MODE_DONE;
}

// ---------------------------------------------------------------------------
// Circulant convolution  out[j] = sum_q taps[q] * in[(j - q) mod N].
//
// taps are Re(IDFT(omega_hat)) of the reference's sampled kernel, so this is
// the same linear operator as real(ifft(fft(in) .* omega_hat))
// (convolve!, src/utils/integrals.jl:88-96), evaluated without transforms.
// Block = (system, component, field, output tile, tap chunk).  Each lane owns
// CONV_R outputs strided by 32 and walks its tap chunk in stride-32 order so
// that the input window slides by one register per step: per step one
// broadcast tap load, one conflict-free window load, CONV_R FMAs.
// Tap chunks (split-K) write separate partial sums, reduced by the consumer.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T conv_in(const SysDev& S, int stage, int comp, int field, int j)
{
    if (stage == 0) return T(S.rho[comp * S.N + j]);
    return reinterpret_cast<const T*>(S.dfield)[(comp * S.NF + field + 1) * S.N + j];
}

template <typename T>
__global__ void __launch_bounds__(CONV_WARPS * 32)
conv1d_kernel(const ConvTask* __restrict__ tasks, const SysDev* __restrict__ sys,
              const AAState* __restrict__ st, int stage)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* staps = reinterpret_cast<T*>(smem_raw);
    T* swin = staps + CONV_QC;
    const ConvTask tk = tasks[blockIdx.x];
    if (!sys_active(st, tk.sys)) return;
    const SysDev& S = sys[tk.sys];
    const int N = S.N;
    const int ks = tk.tile_ks % S.ksplit;
    const int tile = tk.tile_ks / S.ksplit;
    const int slot = tk.comp * S.nconv + tk.field;
    const T* taps = (sizeof(T) == 8) ? reinterpret_cast<const T*>(S.taps) : reinterpret_cast<const T*>(S.taps32);
    taps += (size_t)slot * N;

    const int q_lo = ks * CONV_QC;
    const int q_hi = min(N, q_lo + CONV_QC);
    const int QN = q_hi - q_lo;
    const int j_lo = tile * CONV_TILE;
    const int u_lo = j_lo - q_hi + 1 - 32;
    const int u_n = CONV_TILE + QN - 1 + 32;
    for (int t = threadIdx.x; t < QN; t += blockDim.x) staps[t] = taps[q_lo + t];
    for (int t = threadIdx.x; t < u_n; t += blockDim.x) {
        int u = u_lo + t;
        int idx = ((u % N) + N) % N;
        swin[t] = conv_in<T>(S, stage, tk.comp, tk.field, idx);
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wbase = j_lo + warp * 32 * CONV_R;
    if (wbase >= N) return;   // no further barriers below
    const int j0 = wbase + lane;
    T acc[CONV_R];
#pragma unroll
    for (int r = 0; r < CONV_R; ++r) acc[r] = T(0);
    const int q0_end = min(32, QN);
    for (int q0 = 0; q0 < q0_end; ++q0) {
        T W[CONV_R];
#pragma unroll
        for (int r = 0; r < CONV_R; ++r) W[r] = swin[j0 + 32 * r - (q_lo + q0) - u_lo];
        for (int q = q0; q < QN; q += 32) {
            const T tp = staps[q];
#pragma unroll
            for (int r = 0; r < CONV_R; ++r) acc[r] = fma(tp, W[r], acc[r]);
#pragma unroll
            for (int r = CONV_R - 1; r > 0; --r) W[r] = W[r - 1];
            W[0] = swin[j0 - (q_lo + q) - 32 - u_lo];
        }
    }
    T* out = reinterpret_cast<T*>(S.part) + ((size_t)slot * S.ksplit + ks) * N;
    const T scale = (stage == 0) ? T(S.NA) : T(1);   // n = real(conv) * N_A L^3 (weighted_densities.jl:137)
#pragma unroll
    for (int r = 0; r < CONV_R; ++r) {
        const int j = j0 + 32 * r;
        if (j < N) out[j] = acc[r] * scale;
    }
}

// ---------------------------------------------------------------------------
// Fused Phi / dPhi/dn at every grid point (one thread per point).
// ---------------------------------------------------------------------------
template <typename T, int NC, int ND>
__device__ __forceinline__ void load_n(const SysDev& S, int j, T (&n)[NC][6 + ND])
{
    const T* part = reinterpret_cast<const T*>(S.part);
#pragma unroll
    for (int i = 0; i < NC; ++i) {
        n[i][0] = T(S.NA * S.rho[i * S.N + j]);
#pragma unroll
        for (int f = 0; f < 5 + ND; ++f) {
            const T* p = part + ((size_t)(i * S.nconv + f) * S.ksplit) * S.N + j;
            T v = p[0];
            for (int ks = 1; ks < S.ksplit; ++ks) v += p[(size_t)ks * S.N];
            n[i][f + 1] = v;
        }
    }
}

template <typename T, int NC, int ND>
__device__ __forceinline__ void phi_point(const Chunk* __restrict__ pchunks, const SysDev* __restrict__ sys,
                                          const AAState* __restrict__ st)
{
    const Chunk c = pchunks[blockIdx.x];
    if (!sys_active(st, c.sys)) return;
    const SysDev& S = sys[c.sys];
    const int j = c.begin + threadIdx.x;
    if (j >= S.N) return;
    T n[NC][6 + ND], g[NC][6 + ND];
    load_n<T, NC, ND>(S, j, n);
    const T f = phi_grad<T, NC, ND>(S.phi, n, g);
    T* df = reinterpret_cast<T*>(S.dfield);
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int a = 0; a < 6 + ND; ++a) df[(i * (6 + ND) + a) * S.N + j] = g[i][a];
    S.fval[j] = double(f);
}

template <typename T, int NC, int ND>
__global__ void __launch_bounds__(POINT_THREADS)
phi_kernel(const Chunk* __restrict__ pchunks, const SysDev* __restrict__ sys, const AAState* __restrict__ st)
{
    phi_point<T, NC, ND>(pchunks, sys, st);
}

// The 3D grids' Phi pass streams millions of points: five resident blocks per SM (at
// most 96 registers, ~100 B of spills; 146 unbounded gave three) keep more loads in
// flight (128^3 FP64 iteration: 4 blocks 1.228 ms, 5 blocks 1.210 ms).
template <typename T, int NC>
__global__ void __launch_bounds__(POINT_THREADS, 5)
phi_kernel3d(const Chunk* __restrict__ pchunks, const SysDev* __restrict__ sys, const AAState* __restrict__ st)
{
    phi_point<T, NC, 3>(pchunks, sys, st);
}

// standalone pointwise evaluation (cdft_phi_pointwise): n, dphi are (npts, NF, nc) column-major
template <int NC, int ND>
__global__ void phi_points_kernel(PhiParams P, const double* __restrict__ n_in, int npts,
                                  double* __restrict__ fval, double* __restrict__ dphi)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npts) return;
    double n[NC][6 + ND], g[NC][6 + ND];
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int a = 0; a < 6 + ND; ++a) n[i][a] = n_in[(size_t)(i * (6 + ND) + a) * npts + p];
    fval[p] = phi_grad<double, NC, ND>(P, n, g);
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int a = 0; a < 6 + ND; ++a) dphi[(size_t)(i * (6 + ND) + a) * npts + p] = g[i][a];
}

// ---------------------------------------------------------------------------
// Block reduction of K partial sums (deterministic order).
// ---------------------------------------------------------------------------
template <int BLOCK, int NS = RED_SLOTS>
__device__ __forceinline__ void block_reduce_store(double* vals, int K, double* out)
{
    __shared__ double red[BLOCK / 32][RED_SLOTS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < NS; ++c) {
        if (c >= K) break;
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
        out[threadIdx.x] = s;
    }
}

// ---------------------------------------------------------------------------
// dF/drho + Vext (standalone functional derivative).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ double dfdrho_elem(const SysDev& S, int e)
{
    const int i = e / S.N, j = e - i * S.N;
    const T* df = reinterpret_cast<const T*>(S.dfield);
    const T* part = reinterpret_cast<const T*>(S.part);
    double v = double(df[(i * S.NF) * S.N + j]);   // rho field: δfδρ_res .= profile
    if (S.adj) {   // 3D: the adjoint convolutions were summed in the spectral domain
        v += double(reinterpret_cast<const T*>(S.adj)[e]);
        if (S.vext) v += S.vext[e];
        return v;
    }
    for (int f = 0; f < S.nconv; ++f) {
        const T* p = part + ((size_t)(i * S.nconv + f) * S.ksplit) * S.N + j;
        T acc = p[0];
        for (int ks = 1; ks < S.ksplit; ++ks) acc += p[(size_t)ks * S.N];
        // scalar fields accumulate, vector fields subtract (weighted_densities.jl:160,381)
        if (f >= 2 && f < 2 + S.nd) v -= double(acc);
        else v += double(acc);
    }
    if (S.vext) v += S.vext[e];
    return v;
}

template <typename T>
__global__ void dfdrho_out_kernel(const Chunk* __restrict__ echunks, const SysDev* __restrict__ sys)
{
    const Chunk c = echunks[blockIdx.x];
    const SysDev& S = sys[c.sys];
    for (int t = threadIdx.x; t < ELEM_CHUNK; t += blockDim.x) {
        const int e = c.begin + t;
        if (e < S.n_elem) S.out[e] = dfdrho_elem<T>(S, e);
    }
}

// ---------------------------------------------------------------------------
// Euler-Lagrange step + aa_point!/betafix! bookkeeping + ||res||^2 partials.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ double el_range(const SysDev& S, const AAState& A, int e0, int e1, int stride);

template <typename T>
__global__ void __launch_bounds__(ELEM_THREADS)
el_kernel(const Chunk* __restrict__ echunks, const SysDev* __restrict__ sys,
          const AAState* __restrict__ st, double* __restrict__ partials)
{
    const Chunk c = echunks[blockIdx.x];
    if (!sys_active(st, c.sys)) return;
    const SysDev& S = sys[c.sys];
    const int e1 = min(c.begin + ELEM_CHUNK, S.n_elem);
    double v[1] = {el_range<T>(S, st[c.sys], c.begin + threadIdx.x, e1, ELEM_THREADS)};
    block_reduce_store<ELEM_THREADS>(v, 1, partials + (size_t)blockIdx.x * RED_SLOTS);
}

// ---------------------------------------------------------------------------
// Vector slot operations of the Anderson step (see OP_* in cdft_internal.cuh).
// ---------------------------------------------------------------------------
// Applies slot operation `op` to the elements e = e0, e0 + stride, ... < e1 of
// one system and accumulates this thread's partial sums into acc[0..K).
// Returns K (0 for the solution updates, which reduce nothing).
// The history Q is row-major (one element's row of Q contiguous, qs doubles, 16-byte
// aligned), so a row arrives in 16-byte loads and stays in registers; column loops are
// unrolled to the compile-time bound MB (>= m) and left early.
//
// One Anderson step's CGS2 update (Orthogonalize!, anderson.jl:525-540) in three passes:
//   DOT_H1:        h1 = Q^T df
//   SUB_DOT_NORM:  df1 = df - Q h1 (stored);  h2 = Q^T df1,  ||df1||^2
//   SETQ_DOT_TRES: df2 = df1 - Q h2,  q = df2 / r,  tres = [Q q]^T res
// with r = ||df2|| = sqrt(||df1||^2 - ||h2||^2), exact for orthonormal Q (the reference
// forms df2 in a third pass and takes its norm).  When the next step starts with the QR
// downdate (downdate_aaqr!, anderson.jl:552-583), its Qx is known before SETQ_DOT_TRES,
// which then stores the rotated row [Q q] Qx instead of q alone.
template <int MB>
__device__ __forceinline__ void load_qrow(const double* __restrict__ p, int cnt, double (&row)[MB])
{
#pragma unroll
    for (int c = 0; c < MB; c += 2) {
        if (c >= cnt) break;
        const double2 v = *reinterpret_cast<const double2*>(p + c);
        row[c] = v.x;
        if (c + 1 < MB) row[c + 1] = v.y;
    }
}

template <int MB = CDFT_MAX_M>
__device__ __forceinline__ int vec_op_range(int op, const SysDev& S, const AAState& A, int e0, int e1, int stride,
                                            double* acc)
{
    const int n = S.n_elem;
    const int m = A.m;
    const int qs = S.qs;
    double* __restrict__ Q = S.Q;
    switch (op) {
    case OP_NORM_DF:
        for (int e = e0; e < e1; e += stride) {
            const double v = S.df[e];
            acc[0] += v * v;
        }
        return 1;
    case OP_DOT_H1: {
        const int kq = A.kq;
        for (int e = e0; e < e1; e += stride) {
            double q[MB];
            load_qrow<MB>(Q + (size_t)e * qs, kq, q);
            const double dv = S.df[e];
#pragma unroll
            for (int cc = 0; cc < MB; ++cc) {
                if (cc >= kq) break;
                acc[cc] += q[cc] * dv;
            }
        }
        return kq;
    }
    case OP_SUB_DOT_NORM: {
        const int kq = A.kq;
        for (int e = e0; e < e1; e += stride) {
            double q[MB];
            load_qrow<MB>(Q + (size_t)e * qs, kq, q);
            double v = S.df[e];
#pragma unroll
            for (int cc = 0; cc < MB; ++cc) {
                if (cc >= kq) break;
                v += (-A.coef[cc]) * q[cc];   // gemv, alpha = -1
            }
            S.df[e] = v;
#pragma unroll
            for (int cc = 0; cc < MB; ++cc) {
                if (cc >= kq) break;
                acc[cc] += q[cc] * v;
            }
#pragma unroll
            for (int cc = 0; cc <= MB; ++cc)
                if (cc == kq) acc[cc] += v * v;   // ||df1||^2 in slot kq
        }
        return kq + 1;
    }
    case OP_SETQ_DOT_TRES: {
        const int kq = A.kq;   // the new column's index; mk = kq + 1 columns enter tres
        const double r = A.rnorm;
        const bool down = A.downdate;
        for (int e = e0; e < e1; e += stride) {
            double q[MB];
            double* row = Q + (size_t)e * qs;
            load_qrow<MB>(row, kq, q);
            double v = S.df[e];
#pragma unroll
            for (int cc = 0; cc < MB; ++cc) {
                if (cc >= kq) break;
                v += (-A.coef[cc]) * q[cc];   // df2 = df1 - Q h2
            }
            const double qn = v / r;
            const double rv = S.res[e];
#pragma unroll
            for (int cc = 0; cc < MB; ++cc) {
                if (cc >= kq) break;
                acc[cc] += q[cc] * rv;
            }
#pragma unroll
            for (int cc = 0; cc <= MB; ++cc)
                if (cc == kq) acc[cc] += qn * rv;
            if (down) {   // next step's Q[:, 1:m-1] = [Q q] Qx (here kq = m - 1)
#pragma unroll
                for (int cc = 0; cc < MB; cc += 2) {
                    if (cc >= kq) break;
                    const double* x0 = A.Qx + cc * m;
                    double o0 = qn * x0[kq], o1 = 0.0;
#pragma unroll
                    for (int rr = 0; rr < MB; ++rr) {
                        if (rr >= kq) break;
                        o0 += q[rr] * x0[rr];
                    }
                    if (cc + 1 < kq) {
                        const double* x1 = x0 + m;
                        o1 = qn * x1[kq];
#pragma unroll
                        for (int rr = 0; rr < MB; ++rr) {
                            if (rr >= kq) break;
                            o1 += q[rr] * x1[rr];
                        }
                    }
                    *reinterpret_cast<double2*>(row + cc) = make_double2(o0, o1);
                }
            } else {
                row[kq] = qn;
            }
        }
        return kq + 1;
    }
    case OP_SOL_AA: {
        const int mk = A.mk;
        for (int e = e0; e < e1; e += stride) {
            double v = S.gx[e];
#pragma unroll
            for (int cc = 0; cc < MB; ++cc) {
                if (cc >= mk) break;
                int slotc = A.head + cc;
                slotc -= (slotc >= m) ? m : 0;
                v += (-A.coef[cc]) * S.DG[(size_t)slotc * n + e];
            }
            S.sol[e] = v;
            S.rho[e] = exp(v);
        }
        return 0;
    }
    case OP_SOL_COPY:
        for (int e = e0; e < e1; e += stride) {
            const double v = S.gx[e];
            S.sol[e] = v;
            S.rho[e] = exp(v);
        }
        return 0;
    default:
        return 0;
    }
}

// MB: compile-time bound of the Anderson depth m (MB >= m), chosen by the host; the
// per-thread history rows and partial sums scale with it.  Three resident blocks per SM
// (80 registers; no spills up to MB = 12) keep enough loads in flight: with the
// unbounded 128 registers two blocks left this memory-bound kernel latency-bound.
template <int MB>
__global__ void __launch_bounds__(ELEM_THREADS, 3)
vec_kernel(const Chunk* __restrict__ echunks, const SysDev* __restrict__ sys,
           const AAState* __restrict__ st, double* __restrict__ partials, int slot)
{
    const Chunk c = echunks[blockIdx.x];
    const AAState& A = st[c.sys];
    const int op = A.op[slot];
    if (op == OP_NONE) return;
    const SysDev& S = sys[c.sys];
    double acc[MB + 1];
#pragma unroll
    for (int k = 0; k < MB + 1; ++k) acc[k] = 0.0;
    const int e1 = min(c.begin + ELEM_CHUNK, S.n_elem);
    const int K = vec_op_range<MB>(op, S, A, c.begin + threadIdx.x, e1, ELEM_THREADS, acc);
    if (K == 0) return;   // block-uniform
    block_reduce_store<ELEM_THREADS, MB + 1>(acc, K, partials + (size_t)blockIdx.x * RED_SLOTS);
}

// Euler-Lagrange step on a range of elements: ln G = mu - dF/drho, clamp, betafix!,
// aa_point! bookkeeping; returns this thread's sum of res^2.
// One element of the Euler-Lagrange step given dF/drho + Vext; returns res^2.
__device__ __forceinline__ double el_elem(const SysDev& S, int e, int i, double dF, double beta, bool aa, double* DGs)
{
    double lnG = S.cprd[i] - dF;
    // clamp!(ln_Gx, -100, 100) with Julia's clamp semantics: a NaN stays NaN (fmin/fmax
    // would turn it into a bound and hide a failed evaluation inside a finite residual)
    lnG = (lnG > 100.0) ? 100.0 : ((lnG < -100.0) ? -100.0 : lnG);
    const double s = S.sol[e];
    const double gxn = (beta == 1.0) ? lnG : (1.0 - beta) * s + beta * lnG;  // betafix!
    const double rn = gxn - s;
    if (aa) {                                          // aa_point!: dg = G_new - G_old, df = res_new - res_old
        const double dgv = gxn - S.gx[e];
        const double dfv = -S.res[e] + rn;
        S.df[e] = dfv;
        if (DGs) DGs[e] = dgv;
    }
    S.res[e] = rn;
    S.gx[e] = gxn;
    return rn * rn;
}

template <typename T>
__device__ __forceinline__ double el_range(const SysDev& S, const AAState& A, int e0, int e1, int stride)
{
    const int mode = A.mode;
    const double beta = (mode == MODE_EVAL_PICARD) ? A.picard_beta : A.beta;
    const bool aa = (mode == MODE_EVAL_AA);
    double* DGs = (aa && A.m > 0) ? S.DG + (size_t)A.dg_slot * S.n_elem : nullptr;
    double ss = 0.0;
    for (int e = e0; e < e1; e += stride) ss += el_elem(S, e, e / S.N, dfdrho_elem<T>(S, e), beta, aa, DGs);
    return ss;
}

// ---------------------------------------------------------------------------
// Control: one warp per system.
// ---------------------------------------------------------------------------
__device__ void aa_finish(AAState& A, int* done_counter)
{
    // AndersonOK, anderson.jl:727-737
    if (A.toosoon) { A.idid = 1; A.errcode = -1; }
    else if (A.resnorm >= A.up_bd) { A.idid = 0; A.errcode = -2; }
    else if (A.resnorm <= A.tol) { A.idid = 1; A.errcode = 0; }
    else { A.idid = 0; A.errcode = 10; }
    A.mode = MODE_DONE;
    atomicAdd(done_counter, 1);
}

__device__ __forceinline__ int aa_next_dg_slot(const AAState& A)
{
    // BuildDG!(DG, m, k+1, dg), anderson.jl:450-461, as a ring: the next dg lands in
    // the slot of the column that is dropped (the oldest) once the history is full.
    if (A.m <= 1) return 0;
    return (A.k > A.m) ? A.head : A.k - 1;
}

__device__ void aa_anderson_start(AAState& A)
{
    // copy!(sol, gx); k += 1; aa_point!  (anderson.jl:369-380)
    A.op[1] = OP_SOL_COPY;
    A.k = 1;
    A.mode = MODE_EVAL_AA;
    A.dg_slot = aa_next_dg_slot(A);
}

// Householder QR of R[:, 2:m] (m x (m-1)) with LAPACK dlarfg conventions;
// downdate_aaqr!, anderson.jl:552-583.  R[:, 2:m] of an upper triangular R is
// upper Hessenberg, and every reflector keeps it so: the vector below the
// diagonal of column j has the single entry at row j+1, each reflector touches
// rows j and j+1 only.  The loops run over those rows (the dense loops add
// exact zeros).  The downdate of the NEXT Anderson step is formed while this
// step still needs R for its solve: it works on the copy Rn (with the column
// offset of the slice) and leaves the thin Q factor in Qx; after this step's
// solve Rn replaces R (aa_apply_downdate).
__device__ void aa_downdate(AAState& A)
{
    const int m = A.m, n = m - 1;
    double* R = A.Rn;
    for (int k = 0; k < m * m; ++k) R[k] = A.R[k];
    double* tau = A.tau;
    double* v1 = A.v1;
    for (int j = 0; j < n; ++j) {
        const double alpha = R[j + (j + 1) * m];
        const double x = R[j + 1 + (j + 1) * m];
        const double xnorm = sqrt(x * x);
        if (xnorm == 0.0) {
            tau[j] = 0.0;
            v1[j] = 0.0;
            continue;
        }
        const double beta = -copysign(hypot(alpha, xnorm), alpha);
        tau[j] = (beta - alpha) / beta;
        v1[j] = x * (1.0 / (alpha - beta));
        R[j + (j + 1) * m] = beta;
        R[j + 1 + (j + 1) * m] = 0.0;
        for (int c = j + 1; c < n; ++c) {
            const double w = fma(v1[j], R[j + 1 + (c + 1) * m], R[j + (c + 1) * m]);
            R[j + (c + 1) * m] = fma(-tau[j], w, R[j + (c + 1) * m]);
            R[j + 1 + (c + 1) * m] = fma(-(tau[j] * v1[j]), w, R[j + 1 + (c + 1) * m]);
        }
    }
    // thin Q (m x n) = H_0 ... H_{n-1} [I; 0]
    double* Qx = A.Qx;
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < m; ++r) Qx[r + c * m] = (r == c) ? 1.0 : 0.0;
    for (int j = n - 1; j >= 0; --j) {
        for (int c = 0; c < n; ++c) {
            const double w = fma(v1[j], Qx[j + 1 + c * m], Qx[j + c * m]);
            Qx[j + c * m] = fma(-tau[j], w, Qx[j + c * m]);
            Qx[j + 1 + c * m] = fma(-(tau[j] * v1[j]), w, Qx[j + 1 + c * m]);
        }
    }
    // Rn[1:m-1, 1:m-1] = upper triangle of the slice; Rn[:, m] = 0
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < m; ++r) R[r + c * m] = (r <= c) ? R[r + (c + 1) * m] : 0.0;
    for (int r = 0; r < m; ++r) R[r + (m - 1) * m] = 0.0;
}

// aa_downdate for a compile-time depth M, by one thread with R and Qx in registers: the same
// operations in the same order (so the same bits) without the round trips through the
// solver state's memory between dependent steps.  Not inlined: its registers are its own.
template <int M>
__device__ __noinline__ void aa_downdate_reg(AAState& A)
{
    constexpr int n = M - 1;
    double R[M][M];
#pragma unroll
    for (int c = 0; c < M; ++c)
#pragma unroll
        for (int r = 0; r < M; ++r) R[r][c] = A.R[r + c * M];
    double tau[n], v1[n];
#pragma unroll
    for (int j = 0; j < n; ++j) {
        const double alpha = R[j][j + 1];
        const double x = R[j + 1][j + 1];
        const double xnorm = sqrt(x * x);
        if (xnorm == 0.0) {
            tau[j] = 0.0;
            v1[j] = 0.0;
            continue;
        }
        const double beta = -copysign(hypot(alpha, xnorm), alpha);
        tau[j] = (beta - alpha) / beta;
        v1[j] = x * (1.0 / (alpha - beta));
        R[j][j + 1] = beta;
        R[j + 1][j + 1] = 0.0;
#pragma unroll
        for (int c = j + 1; c < n; ++c) {
            const double w = fma(v1[j], R[j + 1][c + 1], R[j][c + 1]);
            R[j][c + 1] = fma(-tau[j], w, R[j][c + 1]);
            R[j + 1][c + 1] = fma(-(tau[j] * v1[j]), w, R[j + 1][c + 1]);
        }
    }
    double Qx[M][n];
#pragma unroll
    for (int c = 0; c < n; ++c) {
#pragma unroll
        for (int r = 0; r < M; ++r) Qx[r][c] = (r == c) ? 1.0 : 0.0;
#pragma unroll
        for (int j = n - 1; j >= 0; --j) {
            const double w = fma(v1[j], Qx[j + 1][c], Qx[j][c]);
            Qx[j][c] = fma(-tau[j], w, Qx[j][c]);
            Qx[j + 1][c] = fma(-(tau[j] * v1[j]), w, Qx[j + 1][c]);
        }
    }
#pragma unroll
    for (int j = 0; j < n; ++j) {
        A.tau[j] = tau[j];
        A.v1[j] = v1[j];
    }
#pragma unroll
    for (int c = 0; c < n; ++c)
#pragma unroll
        for (int r = 0; r < M; ++r) {
            A.Qx[r + c * M] = Qx[r][c];
            A.Rn[r + c * M] = (r <= c) ? R[r][c + 1] : 0.0;
        }
#pragma unroll
    for (int r = 0; r < M; ++r) A.Rn[r + n * M] = 0.0;
}

// aa_downdate through the register form for depths up to 12 (deeper histories: the loop form)
__device__ void aa_downdate_fast(AAState& A)
{
    switch (A.m) {
    case 2: aa_downdate_reg<2>(A); return;
    case 3: aa_downdate_reg<3>(A); return;
    case 4: aa_downdate_reg<4>(A); return;
    case 5: aa_downdate_reg<5>(A); return;
    case 6: aa_downdate_reg<6>(A); return;
    case 7: aa_downdate_reg<7>(A); return;
    case 8: aa_downdate_reg<8>(A); return;
    case 9: aa_downdate_reg<9>(A); return;
    case 10: aa_downdate_reg<10>(A); return;
    case 11: aa_downdate_reg<11>(A); return;
    case 12: aa_downdate_reg<12>(A); return;
    default: aa_downdate(A); return;
    }
}

// aa_downdate by one warp: lane 0 forms each reflector, the lanes update the trailing
// columns and build Qx column by column; per element the arithmetic of aa_downdate (a
// reflector with tau = v1 = 0 leaves the columns unchanged).  A lives in shared memory.
__device__ void aa_downdate_warp(AAState& A, int lane)
{
    const int m = A.m, n = m - 1;
    double* R = A.Rn;
    for (int k = lane; k < m * m; k += 32) R[k] = A.R[k];
    __syncwarp();
    double* tau = A.tau;
    double* v1 = A.v1;
    for (int j = 0; j < n; ++j) {
        if (lane == 0) {
            const double alpha = R[j + (j + 1) * m];
            const double x = R[j + 1 + (j + 1) * m];
            const double xnorm = sqrt(x * x);
            if (xnorm == 0.0) {
                tau[j] = 0.0;
                v1[j] = 0.0;
            } else {
                const double beta = -copysign(hypot(alpha, xnorm), alpha);
                tau[j] = (beta - alpha) / beta;
                v1[j] = x * (1.0 / (alpha - beta));
                R[j + (j + 1) * m] = beta;
                R[j + 1 + (j + 1) * m] = 0.0;
            }
        }
        __syncwarp();
        const double tj = tau[j], vj = v1[j];
        for (int c = j + 1 + lane; c < n; c += 32) {
            const double w = fma(vj, R[j + 1 + (c + 1) * m], R[j + (c + 1) * m]);
            R[j + (c + 1) * m] = fma(-tj, w, R[j + (c + 1) * m]);
            R[j + 1 + (c + 1) * m] = fma(-(tj * vj), w, R[j + 1 + (c + 1) * m]);
        }
        __syncwarp();
    }
    double* Qx = A.Qx;
    for (int c = lane; c < n; c += 32) {   // thin Q = H_0 ... H_{n-1} [I; 0], one column per lane
        for (int r = 0; r < m; ++r) Qx[r + c * m] = (r == c) ? 1.0 : 0.0;
        for (int j = n - 1; j >= 0; --j) {
            const double w = fma(v1[j], Qx[j + 1 + c * m], Qx[j + c * m]);
            Qx[j + c * m] = fma(-tau[j], w, Qx[j + c * m]);
            Qx[j + 1 + c * m] = fma(-(tau[j] * v1[j]), w, Qx[j + 1 + c * m]);
        }
    }
    // Rn[1:m-1, 1:m-1] = upper triangle of the slice; Rn[:, m] = 0 (read all, then write)
    double v[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int idx = lane + 32 * t;
        if (idx < n * m) {
            const int c = idx / m, r = idx - c * m;
            v[t] = (r <= c) ? R[r + (c + 1) * m] : 0.0;
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int idx = lane + 32 * t;
        if (idx < n * m) R[idx] = v[t];
    }
    if (lane < m) R[lane + (m - 1) * m] = 0.0;
    __syncwarp();
}

__device__ void aa_after_eval(AAState& A, double r, int* done_counter)
{
    A.resnorm = r;
    if (A.history && A.nevals < A.history_cap) A.history[A.nevals] = r;
    A.nevals++;
    for (int s = 1; s <= N_VEC_SLOTS; ++s) A.op[s] = OP_NONE;
    if (!isfinite(r)) {   // a non-finite evaluation ends the run as a divergence
        A.idid = 0;
        A.errcode = -2;
        A.mode = MODE_DONE;
        atomicAdd(done_counter, 1);
        return;
    }
    switch (A.mode) {
    case MODE_EVAL_INIT: {
        A.up_bd = 1.0e4 * r;
        A.tol = A.rtol * r + A.atol;
        A.picard_tol = A.picard_rtol * r + A.picard_atol;
        A.toosoon = (r <= A.tol);
        if (A.toosoon) { aa_finish(A, done_counter); return; }
        if (A.picard_maxit > 0) {
            A.picard_it = 0;
            if (A.picard_maxit - 1 > 0) {   // copy!(sol, gx); Picard loop
                A.mode = MODE_EVAL_PICARD;
                A.op[1] = OP_SOL_COPY;
                return;
            }
        }
        aa_anderson_start(A);
        return;
    }
    case MODE_EVAL_PICARD: {
        A.picard_it++;
        if (r <= A.picard_tol || r >= A.up_bd) {   // break (sol keeps the previous iterate)
            A.toosoon = (r <= A.tol);
            if (A.toosoon) { aa_finish(A, done_counter); return; }
            aa_anderson_start(A);
            return;
        }
        // copy!(sol, gx)
        A.op[1] = OP_SOL_COPY;
        if (A.picard_it >= A.picard_maxit - 1) {   // loop exhausted
            A.toosoon = (r <= A.tol);
            if (A.toosoon) { aa_finish(A, done_counter); return; }   // pending copy still runs
            aa_anderson_start(A);
        }
        return;
    }
    case MODE_EVAL_AA: {
        if (!((A.k < A.maxit + A.picard_maxit) && (r > A.tol) && (r < A.up_bd))) {
            aa_finish(A, done_counter);
            return;
        }
        if (A.m == 0) {
            A.op[1] = OP_SOL_COPY;
            A.k++;
            return;
        }
        if (A.m > 1 && A.k > A.m) A.head = (A.head + 1) % A.m;   // BuildDG! shift
        const int kqr = A.k - 1;
        A.mk = min(A.m, A.k);
        // the QR downdate of this step (kqr > m - 1) was applied to Q and R at the end of
        // the previous step, as soon as that step's R column was known
        if (kqr == 0 || A.m == 1) {
            A.kq = 0;
            A.op[1] = OP_NORM_DF;
            return;
        }
        A.kq = min(kqr, A.m - 1);
        A.op[1] = OP_DOT_H1;
        return;
    }
    default:
        return;
    }
}

// Number of partial sums that slot operation `op` produced (-1 = the EL stage).
__device__ __forceinline__ int ctl_nsums(const AAState& A, int op)
{
    switch (op) {
    case -1: case OP_NORM_DF: return 1;
    case OP_DOT_H1: return A.kq;
    case OP_SUB_DOT_NORM: case OP_SETQ_DOT_TRES: return A.kq + 1;
    default: return 0;
    }
}

// After this step's R column: when the next Anderson step starts with a full history
// (its counter k + 1 > m), its QR downdate is formed now (Rn, Qx) so that the SETQ pass
// can store the rotated Q.  defer: leave it to the caller (flag pad0), which runs it
// warp-parallel (aa_downdate_warp).
__device__ __forceinline__ void aa_plan_downdate(AAState& A, bool defer)
{
    A.downdate = (A.m > 1 && A.k >= A.m) ? 1 : 0;
    if (A.downdate) {
        if (defer) A.pad0 = 1;
        else aa_downdate_fast(A);
    }
}

// Finish slot `slot_done` (0 = EL) of a system given its reduced sums; sets the
// operation of the next slot.  One thread.
__device__ void ctl_apply(AAState& A, int op, int slot_done, const double* sums, int* done_counter,
                          bool defer_downdate = false)
{
    const int next = slot_done + 1;
    switch (op) {
    case -1:
        aa_after_eval(A, sqrt(sums[0]), done_counter);
        break;
    case OP_NORM_DF: {   // k == 0 branch of aa_qr_update!: R[1,1] = norm(df)
        const double r = sqrt(sums[0]);
        A.R[0] = r;
        A.rnorm = r;
        A.kq = 0;
        aa_plan_downdate(A, defer_downdate);
        if (next <= N_VEC_SLOTS) A.op[next] = OP_SETQ_DOT_TRES;
        break;
    }
    case OP_DOT_H1:
        for (int k = 0; k < A.kq; ++k) { A.h1[k] = sums[k]; A.coef[k] = sums[k]; }
        if (next <= N_VEC_SLOTS) A.op[next] = OP_SUB_DOT_NORM;
        break;
    case OP_SUB_DOT_NORM: {
        // hv[1:k] = h1 + h2; hv[k+1] = norm(df2), ||df2||^2 = ||df1||^2 - ||h2||^2
        double h2sq = 0.0;
        for (int k = 0; k < A.kq; ++k) {
            A.R[k + A.kq * A.m] = A.h1[k] + sums[k];
            A.coef[k] = sums[k];
            h2sq += sums[k] * sums[k];
        }
        const double r = sqrt(fmax(sums[A.kq] - h2sq, 0.0));
        A.R[A.kq + A.kq * A.m] = r;
        A.rnorm = r;
        aa_plan_downdate(A, defer_downdate);
        if (next <= N_VEC_SLOTS) A.op[next] = OP_SETQ_DOT_TRES;
        break;
    }
    case OP_SETQ_DOT_TRES: {
        // theta = R[1:mk,1:mk] \ tres (upper triangular back substitution)
        const int mk = A.mk, m = A.m;
        double th[CDFT_MAX_M];
        for (int i = mk - 1; i >= 0; --i) {
            double v = sums[i];
            for (int j = i + 1; j < mk; ++j) v -= A.R[i + j * m] * th[j];
            th[i] = v / A.R[i + i * m];
        }
        for (int i = 0; i < mk; ++i) A.coef[i] = th[i];
        if (A.downdate)   // the next step starts from the downdated factor
            for (int k = 0; k < m * m; ++k) A.R[k] = A.Rn[k];
        if (next <= N_VEC_SLOTS) A.op[next] = OP_SOL_AA;
        A.k++;
        A.mode = MODE_EVAL_AA;
        A.dg_slot = aa_next_dg_slot(A);
        break;
    }
    default:
        break;
    }
}

// One block of CTL_THREADS per system: threads stride over the system's chunk
// partials in a fixed order, a fixed-shape tree reduces them (deterministic, and
// independent of the other systems of the batch), thread 0 applies the step.
#define CTL_THREADS 128
__global__ void __launch_bounds__(CTL_THREADS)
ctl_kernel(const SysDev* __restrict__ sys, AAState* __restrict__ st, const double* __restrict__ partials,
           int nsys, int slot_done, int* done_counter)
{
    const int s = blockIdx.x;
    if (s >= nsys) return;
    AAState& A = st[s];
    const SysDev& S = sys[s];
    if (A.mode == MODE_DONE) {
        if (slot_done == 0 && threadIdx.x == 0)
            for (int k = 1; k <= N_VEC_SLOTS; ++k) A.op[k] = OP_NONE;
        return;
    }
    const int op = (slot_done == 0) ? -1 : A.op[slot_done];
    if (op == OP_NONE || op == OP_SOL_AA || op == OP_SOL_COPY) return;
    const int K = ctl_nsums(A, op);
    __shared__ double red[CTL_THREADS / 32][RED_SLOTS];
    __shared__ double sums[RED_SLOTS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // one sum at a time: the chunk loop of a sum unrolls into independent loads (a loop
    // over the K sums of a row instead leaves one load in flight per thread behind its
    // bound check, measured 60% slower)
#pragma unroll
    for (int k = 0; k < RED_SLOTS; ++k) {
        if (k >= K) break;
        double v = 0.0;
        for (int ch = threadIdx.x; ch < S.chunk_count; ch += CTL_THREADS)
            v += partials[(size_t)(S.chunk_begin + ch) * RED_SLOTS + k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < CTL_THREADS / 32; ++w) v += red[w][threadIdx.x];
        sums[threadIdx.x] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) ctl_apply(A, op, slot_done, sums, done_counter);
}

// initial iterate: sol = log(rho0); rho = exp(sol)   (converge.jl:244, GFix! :236)
__global__ void init_kernel(const Chunk* __restrict__ echunks, const SysDev* __restrict__ sys)
{
    const Chunk c = echunks[blockIdx.x];
    const SysDev& S = sys[c.sys];
    for (int t = threadIdx.x; t < ELEM_CHUNK; t += blockDim.x) {
        const int e = c.begin + t;
        if (e >= S.n_elem) break;
        const double x = log(S.rho[e]);
        S.sol[e] = x;
        S.rho[e] = exp(x);
    }
}

// Device-array copies of a batch in one launch (block row y = one system): the caller's
// profiles into the plans' buffers and back, instead of one cudaMemcpyAsync per system.
struct CopyTask {
    const double* src;
    double* dst;
    long long n;
};

__global__ void batch_copy_kernel(const CopyTask* __restrict__ tasks)
{
    const CopyTask c = tasks[blockIdx.y];
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < c.n; e += (long long)gridDim.x * blockDim.x)
        c.dst[e] = c.src[e];
}

// The solver state of every system at the start of a phase, written on the device: all
// zero, then aasol's options and the system's slice of the residual history.
struct AAInit {
    double* history;
    int history_cap, picard_maxit;
    double rtol, atol;
};
struct AACommon {
    int m, maxit;
    double beta, picard_beta, picard_rtol, picard_atol;
};

__global__ void state_init_kernel(AAState* __restrict__ st, const AAInit* __restrict__ init, AACommon c)
{
    static_assert(sizeof(AAState) % sizeof(double) == 0, "AAState is zeroed in doubles");
    AAState& A = st[blockIdx.x];
    double* w = reinterpret_cast<double*>(&A);
    for (int k = threadIdx.x; k < (int)(sizeof(AAState) / sizeof(double)); k += blockDim.x) w[k] = 0.0;
    __syncthreads();
    if (threadIdx.x != 0) return;
    const AAInit& I = init[blockIdx.x];
    A.mode = MODE_EVAL_INIT;
    A.m = c.m;
    A.maxit = c.maxit;
    A.picard_maxit = I.picard_maxit;
    A.beta = c.beta;
    A.picard_beta = c.picard_beta;
    A.rtol = I.rtol;
    A.atol = I.atol;
    A.picard_rtol = c.picard_rtol;
    A.picard_atol = c.picard_atol;
    A.history = I.history;
    A.history_cap = I.history_cap;
}

// The fields of the final solver states that the host reads (status, counts, residuals).
struct AASummary {
    int mode, idid, errcode, k, nevals, pad;
    double resnorm, tol;
};

__global__ void state_summary_kernel(const AAState* __restrict__ st, AASummary* __restrict__ out, int n)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const AAState& A = st[s];
    AASummary r;
    r.mode = A.mode;
    r.idid = A.idid;
    r.errcode = A.errcode;
    r.k = A.k;
    r.nevals = A.nevals;
    r.pad = 0;
    r.resnorm = A.resnorm;
    r.tol = A.tol;
    out[s] = r;
}

// ---------------------------------------------------------------------------
// Circulant taps of the 1D kernels: t[q] = Re((1/N) sum_k Omega_k exp(2 pi i k q / N)).
// Omega_k are the reference's closed forms (weighted_densities.jl:28-80,193-246)
// sampled at the reduced FFT frequencies L * fftfreq(N, N/(ub-lb))
// (structure_fftfreq/structure_ω, src/structure/structure.jl:153-185).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double kernel_hat_1d(int type, double w, double R, int vector_comp)
{
    // type: 1 int rho dz, 2 int rho z^2 dz, 3 vector int rho z dz (imaginary part returned)
    const double PI = 3.14159265358979323846, TWO_PI = 2.0 * PI;
    const double wb = fabs(w);
    if (type == 1) return (wb == 0.0) ? 2.0 * R / TWO_PI : 2.0 * sin(wb * R) / wb / TWO_PI;
    if (type == 2) {
        if (wb == 0.0) return 4.0 * PI * R * R * R / 3.0 / (TWO_PI * TWO_PI * TWO_PI);
        return 4.0 * PI / (wb * wb * wb) * (sin(wb * R) - R * wb * cos(wb * R)) / (TWO_PI * TWO_PI * TWO_PI);
    }
    if (wb == 0.0) return 4.0 * PI * R / (TWO_PI * TWO_PI * TWO_PI);
    return 4.0 * PI * w / (wb * wb * wb) * (sin(wb * R) - R * wb * cos(wb * R)) / (TWO_PI * TWO_PI * TWO_PI);
}

__global__ void taps1d_kernel(int N, double span, double L, int type, double width_red, double* __restrict__ taps)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= N) return;
    const double R = 2.0 * 3.14159265358979323846 * width_red;
    double acc = 0.0;
    const int half = (N + 1) / 2;   // ceil(N/2)
    for (int k = 0; k < N; ++k) {
        const int kk = (k < half) ? k : k - N;
        const double w = (double)kk / span * L;
        const long long ph = ((long long)k * (long long)q) % N;
        double sn, cs;
        sincospi(2.0 * (double)ph / (double)N, &sn, &cs);
        const double K = kernel_hat_1d(type, w, R, 0);
        acc += (type == 3) ? -K * sn : K * cs;
    }
    taps[q] = acc / (double)N;
}

// ---------------------------------------------------------------------------
// Radial (spherical / cylindrical) grids: the weighted densities and their adjoint
// are dense operators (the reference's QDHT convolution and its materialised vector
// operator, weighted_densities.jl:92-116,248-343).  One warp per output:
// out[(i*nconv + f)*N + j] = scale * sum_q A[j][q] x[q], x = rho_i (stage 0, scale N_A L^3)
// or dPhi/dn_{i,f} (stage 1); written where the Cartesian convolutions write.
// ---------------------------------------------------------------------------
#define DENSE_THREADS 256
template <typename T>
__global__ void __launch_bounds__(DENSE_THREADS)
dense1d_kernel(const SysDev* __restrict__ sys, int s, int stage, const AAState* __restrict__ st)
{
    if (!sys_active(st, s)) return;
    const SysDev& S = sys[s];
    const int N = S.N, nconv = S.nconv;
    const int row = (blockIdx.x * DENSE_THREADS + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= S.nc * nconv * N) return;
    const int slot = row / N, j = row - slot * N;
    const int i = slot / nconv, f = slot - i * nconv;
    const double* A = S.mats + (((size_t)stage * S.nc * nconv + slot) * N + j) * N;
    double acc = 0.0;
    if (stage == 0) {
        const double* x = S.rho + (size_t)i * N;
        for (int q = lane; q < N; q += 32) acc = fma(A[q], x[q], acc);
    } else {
        const T* x = reinterpret_cast<const T*>(S.dfield) + (size_t)(i * S.NF + f + 1) * N;
        for (int q = lane; q < N; q += 32) acc = fma(A[q], double(x[q]), acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) reinterpret_cast<T*>(S.part)[(size_t)slot * N + j] = T(stage == 0 ? acc * S.NA : acc);
}

// mma.sync m8n8k4 f64 (the FP64 tensor path of sm_100a): D += A B with A 8x4 (row),
// B 4x8 (col); lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Radial operators of a whole batch as FP64 tensor-core GEMMs.  Plans of one geometry,
// length unit and set of diameters share one operator buffer (an isotherm of a pore:
// every pressure), so those systems' matrix-vector products are one product of the
// operator with a matrix whose columns are the systems' inputs.  Column tiles of up to
// DGRP_COLS systems of one buffer are built with the batch; a CTA computes, for one
// slot (component i, field f) and 8 output rows, the 8 x 8 tile Y = A X with
// mma.sync m8n8k4.  The k = 4 blocks of [0, N) are dealt round-robin to the CTA's
// DGRP_WARPS warps (four accumulator pairs each) and the warps' tiles are summed in a
// fixed order in shared memory.  Each output element is a sum over its own operator row
// and input column only, so a system gets the same bits alone or inside any column tile;
// each operator row is read once per column tile instead of once per system.
#define DGRP_COLS 8
#define DGRP_WARPS 8
struct DenseGroup {
    int ns;                   // systems in this column tile (1..DGRP_COLS)
    int sys[DGRP_COLS];       // their batch indices (unused entries repeat sys[0])
};

// RT: 8-row tiles per CTA (1 or 2).  With RT = 2 the two tiles share each input fragment
// (12 loads in flight per lane instead of 8, half the CTAs); every output element runs the
// same sequence of products and additions as with RT = 1, so the bits are the same.
template <typename T, int RT>
__global__ void __launch_bounds__(DGRP_WARPS * 32)
dense_group_kernel(const SysDev* __restrict__ sys, const DenseGroup* __restrict__ groups, int stage,
                   const AAState* __restrict__ st)
{
    __shared__ double red[DGRP_WARPS][RT][32][2];
    const DenseGroup& G = groups[blockIdx.y];
    const SysDev& S0 = sys[G.sys[0]];
    const int N = S0.N, nconv = S0.nconv, nc = S0.nc;
    const int rtiles = (N + 8 * RT - 1) / (8 * RT);   // CTA row blocks of 8 RT rows
    if ((int)blockIdx.x >= nc * nconv * rtiles) return;
    const int slot = blockIdx.x / rtiles, j0 = (blockIdx.x - slot * rtiles) * 8 * RT;
    const int i = slot / nconv, f = slot - i * nconv;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = lane >> 2, k = lane & 3;
    // A: operator rows j0 + 8 t + r (rows past N read row N - 1 and are not stored)
    const double* Abase = S0.mats + ((size_t)stage * nc * nconv + slot) * N * (size_t)N;
    const double* Arow[RT];
#pragma unroll
    for (int t = 0; t < RT; ++t) Arow[t] = Abase + (size_t)min(j0 + 8 * t + r, N - 1) * N;
    // B: column r is the input of the tile's r-th system (zero past ns or once converged)
    const bool cval = r < G.ns && sys_active(st, G.sys[r]);
    const SysDev& Sc = sys[G.sys[cval ? r : 0]];
    const double* x64 = Sc.rho + (size_t)i * N;
    const T* xT = reinterpret_cast<const T*>(Sc.dfield) + (size_t)(i * Sc.NF + f + 1) * N;
    const int nk4 = (N + 3) >> 2;
    double c[RT][4][2];
#pragma unroll
    for (int t = 0; t < RT; ++t)
#pragma unroll
        for (int u = 0; u < 4; ++u) c[t][u][0] = c[t][u][1] = 0.0;
    for (int kb = warp; kb < nk4; kb += 4 * DGRP_WARPS) {   // warp-uniform trip count
        double a[RT][4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int q = (kb + u * DGRP_WARPS) * 4 + k;
            const bool in = q < N;
#pragma unroll
            for (int t = 0; t < RT; ++t) a[t][u] = in ? __ldg(Arow[t] + q) : 0.0;
            b[u] = (in && cval) ? (stage == 0 ? __ldg(x64 + q) : double(xT[q])) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int t = 0; t < RT; ++t) dmma_m8n8k4(c[t][u][0], c[t][u][1], a[t][u], b[u]);
    }
#pragma unroll
    for (int t = 0; t < RT; ++t) {
        red[warp][t][lane][0] = (c[t][0][0] + c[t][1][0]) + (c[t][2][0] + c[t][3][0]);
        red[warp][t][lane][1] = (c[t][0][1] + c[t][1][1]) + (c[t][2][1] + c[t][3][1]);
    }
    __syncthreads();
    if (warp >= RT) return;   // warp t sums and stores row tile t
    const int j = j0 + 8 * warp + r;
    if (j >= N) return;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        double acc = 0.0;
#pragma unroll
        for (int w = 0; w < DGRP_WARPS; ++w) acc += red[w][warp][lane][h];
        const int col = 2 * k + h;
        if (col < G.ns && sys_active(st, G.sys[col])) {
            const SysDev& So = sys[G.sys[col]];
            reinterpret_cast<T*>(So.part)[(size_t)slot * N + j] = T(stage == 0 ? acc * So.NA : acc);
        }
    }
}

// ---------------------------------------------------------------------------
// Parameter gradient of F_res (1D): derivative taps, rho * dtaps, per-point terms.
// ---------------------------------------------------------------------------
// d omega_hat / dR of kernel_hat_1d (same type codes; type 3 returns the imaginary part)
__device__ __forceinline__ double kernel_hat_1d_dR(int type, double w, double R)
{
    const double PI = 3.14159265358979323846, TWO_PI = 2.0 * PI;
    const double wb = fabs(w);
    if (type == 1) return 2.0 * cos(wb * R) / TWO_PI;
    if (type == 2) {
        if (wb == 0.0) return 4.0 * PI * R * R / (TWO_PI * TWO_PI * TWO_PI);
        return 4.0 * PI * R * sin(wb * R) / wb / (TWO_PI * TWO_PI * TWO_PI);
    }
    if (wb == 0.0) return 4.0 * PI / (TWO_PI * TWO_PI * TWO_PI);
    return 4.0 * PI * w * R * sin(wb * R) / wb / (TWO_PI * TWO_PI * TWO_PI);
}

// d taps / dR: Re(IDFT(d omega_hat / dR)), the derivative of taps1d_kernel's output
__global__ void dtaps1d_kernel(int N, double span, double L, int type, double width_red, double* __restrict__ dtaps)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= N) return;
    const double R = 2.0 * 3.14159265358979323846 * width_red;
    double acc = 0.0;
    const int half = (N + 1) / 2;
    for (int k = 0; k < N; ++k) {
        const int kk = (k < half) ? k : k - N;
        const double w = (double)kk / span * L;
        const long long ph = ((long long)k * (long long)q) % N;
        double sn, cs;
        sincospi(2.0 * (double)ph / (double)N, &sn, &cs);
        const double K = kernel_hat_1d_dR(type, w, R);
        acc += (type == 3) ? -K * sn : K * cs;
    }
    dtaps[q] = acc / (double)N;
}

// All circulant taps of one plan in one launch: block (task, q-range) tabulates the
// closed forms Omega at the non-negative frequencies k <= N/2 and the twiddles
// cos/sin(2 pi j / N), j < N, in shared memory once, then every thread sums its
// output q from the tables.  Omega depends on |w| (types 1, 2: the even kernels) or is
// odd in w (type 3, the vector kernel), so the frequencies k and N - k pair up:
//   even: t[q] = (1/N) [Omega_0 + 2 sum_{k=1}^{M} Omega_k cos(2 pi k q / N) + (N even) Omega_{N/2} (-1)^q]
//   odd:  t[q] = (1/N) [-2 sum_{k=1}^{M} Omega_k sin(2 pi k q / N)]          (M = (N-1)/2)
// the same sum as taps1d_kernel / dtaps1d_kernel (Re of the inverse DFT of the sampled
// kernel), with O(N) instead of O(N^2) transcendentals per field.  deriv: d Omega / dR.
#define TAPS_MAX_TASKS 24          // 6 fields x CDFT_MAX_NC components
#define TAPS_TABLE_MAX_N 8192      // shared tables: (2.5 N + 1) doubles <= 164 KB
#define TAPS_THREADS 256
struct TapsArgs {
    int N, ntask, deriv;
    double span, L;
    int type[TAPS_MAX_TASKS];
    double R[TAPS_MAX_TASKS];      // 2 pi x reduced kernel width
    double* out[TAPS_MAX_TASKS];
};

__host__ __device__ __forceinline__ size_t taps_smem_bytes(int N) { return sizeof(double) * (2 * (size_t)N + N / 2 + 1); }

__global__ void __launch_bounds__(TAPS_THREADS) taps_table_kernel(TapsArgs a)
{
    extern __shared__ double tsh[];
    const int N = a.N, H = N / 2 + 1, M = (N - 1) / 2;
    double* cs = tsh;
    double* sn = tsh + N;
    double* om = tsh + 2 * N;
    const int task = blockIdx.x;
    const int type = a.type[task];
    const double R = a.R[task];
    for (int j = threadIdx.x; j < N; j += TAPS_THREADS) sincospi(2.0 * (double)j / (double)N, &sn[j], &cs[j]);
    for (int k = threadIdx.x; k < H; k += TAPS_THREADS) {
        const double w = (double)k / a.span * a.L;
        om[k] = a.deriv ? kernel_hat_1d_dR(type, w, R) : kernel_hat_1d(type, w, R, 0);
    }
    __syncthreads();
    const int q = blockIdx.y * TAPS_THREADS + threadIdx.x;
    if (q >= N) return;
    const double* tab = (type == 3) ? sn : cs;
    double acc0 = 0.0, acc1 = 0.0;
    int j = 0;
    int k = 1;
    for (; k + 1 <= M; k += 2) {   // two accumulators: independent FMA chains
        j += q; j -= (j >= N) ? N : 0;
        acc0 = fma(om[k], tab[j], acc0);
        j += q; j -= (j >= N) ? N : 0;
        acc1 = fma(om[k + 1], tab[j], acc1);
    }
    if (k <= M) {
        j += q; j -= (j >= N) ? N : 0;
        acc0 = fma(om[k], tab[j], acc0);
    }
    double t;
    if (type == 3) {
        t = -2.0 * (acc0 + acc1);
    } else {
        t = om[0] + 2.0 * (acc0 + acc1);
        if ((N & 1) == 0) t += (q & 1) ? -om[N / 2] : om[N / 2];
    }
    a.out[task][q] = t / (double)N;
}

// dn[(i*nconv + f)*N + j] = scale[f] * sum_q dtaps[(i*nconv + f)*N + q] rho[i*N + (j - q) mod N]
__global__ void dconv1d_kernel(int N, int nconv, const double* __restrict__ dtaps, const double* __restrict__ rho,
                               const double* __restrict__ scale, double* __restrict__ dn)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int slot = blockIdx.y;   // i * nconv + f
    if (j >= N) return;
    const int i = slot / nconv, f = slot - i * nconv;
    const double* t = dtaps + (size_t)slot * N;
    const double* r = rho + (size_t)i * N;
    double acc = 0.0;
    int src = j;
    for (int q = 0; q < N; ++q) {
        acc = fma(t[q], r[src], acc);
        src = (src == 0) ? N - 1 : src - 1;
    }
    dn[(size_t)slot * N + j] = acc * scale[f];
}

// per point j: gp[q*N + j] = dPhi/dP_q (explicit parameters) and
// kt[i*N + j] = sum_f dPhi/dn_{i,f} * dn_{i,f}/dd_i (kernels)
template <int NC, int ND>
__global__ void grad_points_kernel(const SysDev* __restrict__ sys, const double* __restrict__ dn,
                                   double* __restrict__ gp_out, double* __restrict__ kt_out)
{
    const SysDev& S = sys[0];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= S.N) return;
    double n[NC][6 + ND], g[NC][6 + ND];
    double gp[PhiParamIdx<NC>::NP];
    load_n<double, NC, ND>(S, j, n);
    phi_grad<double, NC, ND, true>(S.phi, n, g, gp);
    for (int q = 0; q < PhiParamIdx<NC>::NP; ++q) gp_out[(size_t)q * S.N + j] = gp[q];
#pragma unroll
    for (int i = 0; i < NC; ++i) {
        double acc = 0.0;
        for (int f = 0; f < S.nconv; ++f) acc += g[i][f + 1] * dn[((size_t)i * S.nconv + f) * S.N + j];
        kt_out[(size_t)i * S.N + j] = acc;
    }
}

__global__ void to_float_kernel(const double* __restrict__ a, float* __restrict__ b, size_t n)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

// ---------------------------------------------------------------------------
// Integrals of a system at its current profile, one block per system: the free energies
// and the amounts that surface_tension (surface_tension.jl:31-53), adsorption
// (adsorption.jl:26-32) and free_energy (utils/base.jl:8-10) need.  out[(3 + nc) s + q]:
//   q = 0        sum_j w_j Phi_j          (F_res L^3, k_B T)
//   q = 1        sum_j w_j f_ideal_j      (F_ideal, k_B T; BasicIdeal.jl:34-38)
//   q = 2 + i    sum_j w_j rho_ij         (int rho_i)
//   q = 2 + nc   sum_j w_j                (int 1)
// w_j: Simpson's 1, 4, 2, ..., 4, 1 per dimension times dz/3 (integrals.jl:17,28-41), or the
// radial quadrature weights.  Grid (chunks, systems): a block sums INTEG_CHUNK consecutive
// points of one system, each thread with Neumaier's compensation, and writes the block's
// (sum, compensation) pair per amount; integrals_reduce_kernel then combines the chunks of
// a system in chunk order.  The order of every addition is fixed (deterministic).
// ---------------------------------------------------------------------------
#define INTEG_THREADS 256
#define INTEG_CHUNK (INTEG_THREADS * 32)
struct NSum {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x)
    {
        const double t = s + x;
        c += (fabs(s) >= fabs(x)) ? ((s - t) + x) : ((x - t) + s);
        s = t;
    }
};

__device__ __forceinline__ double simpson_coef(int k, int n)   // k = 0 .. n-1
{
    return (k == 0 || k == n - 1) ? 1.0 : (((k + 1) & 1) == 0 ? 4.0 : 2.0);
}

// part[((s * nchunk + chunk) * nq + q) * 2 + {0, 1}] = (sum, compensation)
__global__ void __launch_bounds__(INTEG_THREADS)
integrals_kernel(const SysDev* __restrict__ sys, double T, double* __restrict__ part, int nchunk)
{
    const SysDev& S = sys[blockIdx.y];
    const int nc = S.nc, nq = 3 + nc;
    const double kNA = 6.02214076e23, lnT = log(T);
    NSum acc[3 + CDFT_MAX_NC];
    const int j0 = blockIdx.x * INTEG_CHUNK;
    const int j1 = min(S.N, j0 + INTEG_CHUNK);
    for (int j = j0 + threadIdx.x; j < j1; j += INTEG_THREADS) {
        double w;
        if (S.qw) {
            w = S.qw[j];
        } else if (S.nd == 1) {
            w = simpson_coef(j, S.N) * S.wscale;
        } else {
            const int L = S.ngrid[0];
            const int x = j % L, y = (j / L) % L, z = j / (L * L);
            w = simpson_coef(x, L) * simpson_coef(y, L) * simpson_coef(z, L) * S.wscale;
        }
        acc[0].add(w * S.fval[j]);
        double fid = 0.0;
        for (int i = 0; i < nc; ++i) {
            const double r = S.rho[(size_t)i * S.N + j];
            fid += kNA * r * (log(r) - 1.5 * lnT - 1.0);
            acc[2 + i].add(w * r);
        }
        acc[1].add(w * fid);
        acc[2 + nc].add(w);
    }
    __shared__ double ps[INTEG_THREADS][3 + CDFT_MAX_NC];
    __shared__ double pc[INTEG_THREADS][3 + CDFT_MAX_NC];
    for (int q = 0; q < nq; ++q) {
        ps[threadIdx.x][q] = acc[q].s;
        pc[threadIdx.x][q] = acc[q].c;
    }
    __syncthreads();
    if (threadIdx.x < nq) {
        const int q = threadIdx.x;
        NSum tot;
        double comp = 0.0;
        for (int t = 0; t < INTEG_THREADS; ++t) {
            tot.add(ps[t][q]);
            comp += pc[t][q];
        }
        double* o = part + (((size_t)blockIdx.y * nchunk + blockIdx.x) * nq + q) * 2;
        o[0] = tot.s;
        o[1] = tot.c + comp;
    }
}

// One block per system: out[s * nq + q] from the chunk pairs, in chunk order.
__global__ void integrals_reduce_kernel(const double* __restrict__ part, int nchunk, int nq, double* __restrict__ out)
{
    const int q = threadIdx.x;
    if (q >= nq) return;
    NSum tot;
    double comp = 0.0;
    for (int c = 0; c < nchunk; ++c) {
        const double* o = part + (((size_t)blockIdx.x * nchunk + c) * nq + q) * 2;
        tot.add(o[0]);
        comp += o[1];
    }
    out[(size_t)blockIdx.x * nq + q] = tot.s + (tot.c + comp);
}

// ---------------------------------------------------------------------------
// DDFT right-hand side in ln rho (ext/SciMLBasecDFTExt.jl:10-61, ddft_rhs_log!):
//   d eta/dt = lap(eta) + lap(mu) + sum_d [ (d_d eta)^2 + d_d mu d_d eta ],
// mu = dF/drho_res + V_ext.  The reference applies the spectral maps 2 pi i k_d and
// -(2 pi)^2 |k|^2 by FFT (convolve!, integrals.jl:88-96: real part of the inverse
// transform); both maps are sums of one-axis maps, so each term is a periodic circulant
// along one axis whose taps are the real inverse DFT of the one-axis map.
// ddft_prep_kernel: rho = exp(clamp(eta, -50, 30)).
// ddft_axis_kernel: one block per (line, output tile) of one axis; the line of eta and mu
// in shared memory; adds lap_d(eta + mu) + g_eta^2 + g_mu g_eta into deta (first axis
// writes).  tg / tl: gradient and second-derivative taps of the axis.
// ---------------------------------------------------------------------------
#define DDFT_THREADS 256
__global__ void ddft_prep_kernel(const double* __restrict__ eta, double* __restrict__ rho, size_t n)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        rho[e] = exp(fmin(fmax(eta[e], -50.0), 30.0));
}

__global__ void __launch_bounds__(DDFT_THREADS)
ddft_axis_kernel(const double* __restrict__ eta, const double* __restrict__ mu, double* __restrict__ deta,
                 const double* __restrict__ tg, const double* __restrict__ tl, int len, long long stride,
                 long long inner, long long nlines, int first)
{
    extern __shared__ double ddft_smem[];
    double* se = ddft_smem;        // eta of the line
    double* sm = ddft_smem + len;  // mu of the line
    const long long line = blockIdx.x;
    if (line >= nlines) return;
    // line -> base offset: lines are (outer, inner) pairs around the axis
    const long long o = line / inner, i = line - o * inner;
    const long long base = o * inner * len + i;
    for (int q = threadIdx.x; q < len; q += DDFT_THREADS) {
        se[q] = eta[base + q * stride];
        sm[q] = mu[base + q * stride];
    }
    __syncthreads();
    const int j = blockIdx.y * DDFT_THREADS + threadIdx.x;
    if (j >= len) return;
    double lap = 0.0, ge = 0.0, gm = 0.0;
    int src = j;   // (j - q) mod len
    for (int q = 0; q < len; ++q) {
        const double a = tg[q], b = tl[q];
        const double xe = se[src], xm = sm[src];
        lap = fma(b, xe + xm, lap);
        ge = fma(a, xe, ge);
        gm = fma(a, xm, gm);
        src = (src == 0) ? len - 1 : src - 1;
    }
    const double v = lap + ge * ge + gm * ge;
    const long long e = base + j * stride;
    deta[e] = first ? v : deta[e] + v;
}
