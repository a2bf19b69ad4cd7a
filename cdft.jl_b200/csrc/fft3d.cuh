// 3D periodic Cartesian weighted densities by FFT (cubic box, N a power of two).
//
// The reference convolves with real(ifft(fft(rho) .* omega_hat)) on complex
// FFTs (convolve!, src/utils/integrals.jl:88-96) with the analytic kernels of
// weighted_densities.jl:28-80,193-246 sampled at L*fftfreq.  Here the same
// operator runs on the half spectrum (x is the real-to-complex axis):
//   spectrum layout [field][z][y][kx], kx in [0, N/2] valid, rows padded to KXP = N/2 + 2
//   entries (a row of either precision is a multiple of 16 bytes: tensor-map strides),
//   y and z in [0, N)
//   x pass: two real rows packed into one complex N-point FFT and split
//   y, z passes: in place, LINES consecutive kx per block (coalesced rows)
// The kernel multiply is fused into the z pass: one kernel turns the spectrum
// of rho into all convolved-field spectra, another accumulates the adjoint
// products of all fields into one spectrum.  Kernel values come from tables
// indexed by |k|^2 (cubic box: omega_bar depends on kx^2+ky^2+kz^2 only).
// Vector kernels are i * omega_d * Omega_n3(omega_bar) with the Nyquist plane of
// their own axis and k = 0 set to zero: that is the Hermitian part of the
// reference's kernel, i.e. exactly what real(ifft(...)) keeps.
//
// FFTs: two register passes per transform (L = R1 R2 Cooley-Tukey, radix-2 DFTs in
// registers, one shared-memory exchange), twiddles exp(-2 pi i q / N) from sincospi.
#pragma once
#include "cdft_internal.cuh"

#define FFT_THREADS 256

// lines per block for a given transform length and element size: more resident blocks
// beat more lines per block once a line exceeds 512 B (measured at 128^3 and 256^3)
template <typename T, int L> struct FftLines { static constexpr int value = (L * (int)sizeof(T) <= 512) ? 16 : 8; };

// resident blocks per SM the register allocation must allow: unbounded, the FP64 transforms
// of 128 and 256 points took 96-132 registers (two blocks of 256 threads; shared memory
// allows five); at 80 registers three fit (+5-8% per 3D iteration, measured).  The other
// instances used at most 64-72 registers unbounded and get that cap.
template <typename T, int L> struct FftMinBlocks { static constexpr int value = (sizeof(T) == 8 && L >= 128) ? 3 : 4; };

template <typename T> struct V2;
template <> struct V2<double> { typedef double2 t; };
template <> struct V2<float> { typedef float2 t; };

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) { C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r; }
template <typename C>
__device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }

// twiddle table tw[q] = exp(-2 pi i q / L), q < L/2, in shared memory
template <typename T, int L>
__device__ __forceinline__ void fft_twiddles(typename V2<T>::t* tw)
{
    for (int q = threadIdx.x; q < L / 2; q += blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)q / (double)L, &s, &c);
        tw[q].x = T(c);
        tw[q].y = T(s);
    }
}

// Split of an L-point transform into two register passes, L = R1 * R2.
template <int L> struct FftSplit;
template <> struct FftSplit<32> { static constexpr int R1 = 4, R2 = 8; };
template <> struct FftSplit<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct FftSplit<128> { static constexpr int R1 = 8, R2 = 16; };
template <> struct FftSplit<256> { static constexpr int R1 = 16, R2 = 16; };

__host__ __device__ constexpr int fft_bitrev(int i, int R)
{
    int r = 0;
    for (int b = 1; b < R; b <<= 1) {
        r = (r << 1) | (i & 1);
        i >>= 1;
    }
    return r;
}

// w_L^m = exp(-+2 pi i m / L), m in [0, L), from the half table tw[q], q < L/2
template <typename C, int L>
__device__ __forceinline__ C fft_tw(const C* tw, int m, bool inverse)
{
    C w = tw[m & (L / 2 - 1)];
    if (m >= L / 2) { w.x = -w.x; w.y = -w.y; }
    if (inverse) w.y = -w.y;
    return w;
}

// R-point DFT of v in registers (radix-2, decimation in time, all indices compile-time);
// twiddles w_R^q = w_L^(q L / R) from the block's table
template <typename C, int R, int L>
__device__ __forceinline__ void fft_reg(C (&v)[R], const C* tw, bool inverse)
{
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int jr = fft_bitrev(i, R);
        if (jr > i) { const C t = v[i]; v[i] = v[jr]; v[jr] = t; }
    }
#pragma unroll
    for (int half = 1; half < R; half <<= 1) {
#pragma unroll
        for (int q = 0; q < half; ++q) {
            const C w = fft_tw<C, L>(tw, q * (L / (2 * half)), inverse);
#pragma unroll
            for (int b = 0; b < R; b += 2 * half) {
                const C a = v[b + q], c = cmul(v[b + q + half], w);
                v[b + q] = cadd(a, c);
                v[b + q + half] = csub(a, c);
            }
        }
    }
}

// L-point transforms of LINES lines stored as x[n * LS + line] (LS = LINES + 1 avoids bank
// conflicts).  Two register passes, L = R1 R2 (decimation in time):
//   pass 1, for each (t < R2, line): DFT over s of x[t + R2 s] -> u[k1], times w_L^(t k1),
//           stored at y[k1 R2 + t]
//   pass 2, for each (k1 < R1, line): DFT over t of y[k1 R2 + t] -> X[k1 + R1 k2] into x
// since w_L^((t + R2 s)(k1 + R1 k2)) = w_L^(t k1) w_R2^(t k2) w_R1^(s k1).  The caller has
// synchronised after filling x; the result is in x (returned) after a barrier.
template <typename T, int L, int LINES, int LS>
__device__ __forceinline__ typename V2<T>::t* fft_lines(typename V2<T>::t* x, typename V2<T>::t* y,
                                                        const typename V2<T>::t* tw, bool inverse)
{
    typedef typename V2<T>::t C;
    constexpr int R1 = FftSplit<L>::R1, R2 = FftSplit<L>::R2;
    for (int it = threadIdx.x; it < R2 * LINES; it += blockDim.x) {
        const int line = it % LINES, t = it / LINES;
        C v[R1];
#pragma unroll
        for (int s = 0; s < R1; ++s) v[s] = x[(t + R2 * s) * LS + line];
        fft_reg<C, R1, L>(v, tw, inverse);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) y[(k1 * R2 + t) * LS + line] = cmul(v[k1], fft_tw<C, L>(tw, t * k1, inverse));
    }
    __syncthreads();
    for (int it = threadIdx.x; it < R1 * LINES; it += blockDim.x) {
        const int line = it % LINES, k1 = it / LINES;
        C v[R2];
#pragma unroll
        for (int t = 0; t < R2; ++t) v[t] = y[(k1 * R2 + t) * LS + line];
        fft_reg<C, R2, L>(v, tw, inverse);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) x[(k1 + R1 * k2) * LS + line] = v[k2];
    }
    __syncthreads();
    return x;
}

// row length of the half spectrum: KX = L/2 + 1 valid entries, KXP = L/2 + 2 stored
template <int L> struct Spec3 {
    static constexpr int KX = L / 2 + 1;
    static constexpr int KXP = L / 2 + 2;
};

struct Grid3 {
    int N;          // points per dimension
    int Kx;         // N/2 + 1
    size_t npts;    // N^3
    size_t nspec;   // Kx N^2
};

// ---------------------------------------------------------------------------
// x pass, real -> half spectrum.  in: nfields real arrays (stride in_stride),
// out: nfields spectra (stride out_stride).  Block: 2*LINES rows of one field.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool fft_skip(const AAState* st) { return st != nullptr && st[0].mode == MODE_DONE; }

template <typename T, typename Tin, int L, int LINES>
__global__ void __launch_bounds__(FFT_THREADS, (FftMinBlocks<T, L>::value))
fft_x_r2c(const Tin* __restrict__ in, size_t in_stride, typename V2<T>::t* __restrict__ out, size_t out_stride,
          const AAState* __restrict__ st)
{
    typedef typename V2<T>::t C;
    constexpr int LS = LINES + 1;
    constexpr int KX = L / 2 + 1;
    if (fft_skip(st)) return;
    extern __shared__ __align__(16) unsigned char fft_smem[];
    C* bufA = reinterpret_cast<C*>(fft_smem);
    C* bufB = bufA + L * LS;
    C* tw = bufB + L * LS;
    fft_twiddles<T, L>(tw);
    const int field = blockIdx.y;
    const size_t row0 = (size_t)blockIdx.x * 2 * LINES;   // rows are (z, y) pairs, N*N of them
    const Tin* src = in + field * in_stride + row0 * L;
    for (int idx = threadIdx.x; idx < 2 * LINES * L; idx += blockDim.x) {
        const int r = idx / L, n = idx - r * L;
        const T v = T(src[idx]);
        C& c = bufA[n * LS + (r >> 1)];
        if (r & 1) c.y = v; else c.x = v;
    }
    __syncthreads();
    const C* Z = fft_lines<T, L, LINES, LS>(bufA, bufB, tw, false);
    constexpr int KXP = Spec3<L>::KXP;
    C* dst = out + field * out_stride + row0 * KXP;
    for (int idx = threadIdx.x; idx < LINES * KX; idx += blockDim.x) {
        const int line = idx / KX, k = idx - line * KX;
        const C zk = Z[k * LS + line];
        const C zm = cconj(Z[((L - k) % L) * LS + line]);
        C a, b;   // X_a = (Z_k + conj Z_{L-k}) / 2,  X_b = (Z_k - conj Z_{L-k}) / (2i)
        a.x = T(0.5) * (zk.x + zm.x);
        a.y = T(0.5) * (zk.y + zm.y);
        b.x = T(0.5) * (zk.y - zm.y);
        b.y = T(-0.5) * (zk.x - zm.x);
        dst[(size_t)(2 * line) * KXP + k] = a;
        dst[(size_t)(2 * line + 1) * KXP + k] = b;
    }
}

// ---------------------------------------------------------------------------
// x pass, half spectrum -> real, times `scale`.
// ---------------------------------------------------------------------------
template <typename T, int L, int LINES>
__global__ void __launch_bounds__(FFT_THREADS, (FftMinBlocks<T, L>::value))
fft_x_c2r(const typename V2<T>::t* __restrict__ in, size_t in_stride, T* __restrict__ out, size_t out_stride, T scale,
          const AAState* __restrict__ st)
{
    typedef typename V2<T>::t C;
    constexpr int LS = LINES + 1;
    constexpr int KX = L / 2 + 1;
    if (fft_skip(st)) return;
    extern __shared__ __align__(16) unsigned char fft_smem[];
    C* bufA = reinterpret_cast<C*>(fft_smem);
    C* bufB = bufA + L * LS;
    C* tw = bufB + L * LS;
    fft_twiddles<T, L>(tw);
    const int field = blockIdx.y;
    const size_t row0 = (size_t)blockIdx.x * 2 * LINES;
    constexpr int KXP = Spec3<L>::KXP;
    const C* src = in + field * in_stride + row0 * KXP;
    for (int idx = threadIdx.x; idx < LINES * L; idx += blockDim.x) {
        const int line = idx / L, k = idx - line * L;
        const int kk = (k <= L / 2) ? k : L - k;
        C a = src[(size_t)(2 * line) * KXP + kk];
        C b = src[(size_t)(2 * line + 1) * KXP + kk];
        if (k > L / 2) { a = cconj(a); b = cconj(b); }
        C z;   // Z = X_a + i X_b
        z.x = a.x - b.y;
        z.y = a.y + b.x;
        bufA[k * LS + line] = z;
    }
    __syncthreads();
    const C* z = fft_lines<T, L, LINES, LS>(bufA, bufB, tw, true);
    T* dst = out + field * out_stride + row0 * L;
    for (int idx = threadIdx.x; idx < 2 * LINES * L; idx += blockDim.x) {
        const int r = idx / L, n = idx - r * L;
        const C c = z[n * LS + (r >> 1)];
        dst[idx] = ((r & 1) ? c.y : c.x) * scale;
    }
}

// ---------------------------------------------------------------------------
// in-place y or z pass on spectra.  axis 1: y (stride Kx), axis 2: z (stride N Kx).
// Block: LINES consecutive kx at one (z) [axis y] or one (y) [axis z].
// ---------------------------------------------------------------------------
template <typename T, int L, int LINES>
__device__ __forceinline__ size_t yz_base(int axis, int outer, int kx0)
{
    constexpr int KXP = Spec3<L>::KXP;
    return axis == 1 ? (size_t)outer * L * KXP + kx0 : (size_t)outer * KXP + kx0;
}

template <typename T, int L, int LINES>
__global__ void __launch_bounds__(FFT_THREADS, (FftMinBlocks<T, L>::value))
fft_yz(typename V2<T>::t* __restrict__ data, size_t stride, int axis, int inverse, const AAState* __restrict__ st)
{
    typedef typename V2<T>::t C;
    constexpr int LS = LINES + 1;
    constexpr int KX = L / 2 + 1;
    if (fft_skip(st)) return;
    extern __shared__ __align__(16) unsigned char fft_smem[];
    C* bufA = reinterpret_cast<C*>(fft_smem);
    C* bufB = bufA + L * LS;
    C* tw = bufB + L * LS;
    fft_twiddles<T, L>(tw);
    const int ntile = (KX + LINES - 1) / LINES;
    const int kx0 = (blockIdx.x % ntile) * LINES;
    const int outer = blockIdx.x / ntile;
    const size_t estride = axis == 1 ? Spec3<L>::KXP : (size_t)L * Spec3<L>::KXP;
    C* d = data + blockIdx.y * stride + yz_base<T, L, LINES>(axis, outer, kx0);
    const int nl = min(LINES, KX - kx0);
    for (int idx = threadIdx.x; idx < L * LINES; idx += blockDim.x) {
        const int n = idx / LINES, line = idx - n * LINES;
        if (line < nl) bufA[n * LS + line] = d[n * estride + line];
        else { bufA[n * LS + line].x = T(0); bufA[n * LS + line].y = T(0); }
    }
    __syncthreads();
    const C* r = fft_lines<T, L, LINES, LS>(bufA, bufB, tw, inverse != 0);
    for (int idx = threadIdx.x; idx < L * LINES; idx += blockDim.x) {
        const int n = idx / LINES, line = idx - n * LINES;
        if (line < nl) d[n * estride + line] = r[n * LS + line];
    }
}

// ---------------------------------------------------------------------------
// kernel multiplier at (kx, y, z) for convolved field f of component i
// ---------------------------------------------------------------------------
struct KTab3 {
    const double* tab;     // [(i*5 + t) * (k2max+1) + k2], t: 0 n2(d/2) 1 n3(d/2) 2 n3(d) 3 n2(d) 4 n3(psi d)
    int k2max;
    double w0;             // reduced frequency per index: L / period
    int nconv;             // 8
};

// field f (0..7) of the 3D list -> table type; vectors use the n3(d/2) table
__device__ __forceinline__ int k3_table(int f) { return f == 0 ? 0 : (f <= 4 ? 1 : f - 3); }

template <typename T, int L>
__device__ __forceinline__ typename V2<T>::t k3_apply(const KTab3& K, int comp, int f, int kx, int ky, int kz,
                                                      typename V2<T>::t v)
{
    typedef typename V2<T>::t C;
    const int sy = ky < L / 2 ? ky : ky - L, sz = kz < L / 2 ? kz : kz - L;
    const int k2 = kx * kx + sy * sy + sz * sz;
    const T t = T(K.tab[((size_t)comp * 5 + k3_table(f)) * (K.k2max + 1) + k2]);
    C r;
    if (f < 2 || f > 4) {   // real, even kernel
        r.x = v.x * t;
        r.y = v.y * t;
        return r;
    }
    const int d = f - 2;    // vector component: i * omega_d * Omega_n3, zero on its Nyquist plane
    const int kd = d == 0 ? kx : (d == 1 ? ky : kz);
    const int sd = d == 0 ? kx : (d == 1 ? sy : sz);
    if (kd == L / 2) { r.x = T(0); r.y = T(0); return r; }
    const T wv = T(K.w0 * (double)sd) * t;
    r.x = -v.y * wv;
    r.y = v.x * wv;
    return r;
}

// z pass of the weighted densities: forward z-FFT of the rho spectrum, then for
// every convolved field: multiply by the kernel and inverse z-FFT into its spectrum.
template <typename T, int L, int LINES>
__global__ void __launch_bounds__(FFT_THREADS, (FftMinBlocks<T, L>::value))
fft_z_eval(const typename V2<T>::t* __restrict__ R, size_t r_stride, typename V2<T>::t* __restrict__ out,
           size_t out_stride, KTab3 K, const AAState* __restrict__ st)
{
    typedef typename V2<T>::t C;
    constexpr int LS = LINES + 1;
    constexpr int KX = L / 2 + 1;
    if (fft_skip(st)) return;
    extern __shared__ __align__(16) unsigned char fft_smem[];
    C* bufA = reinterpret_cast<C*>(fft_smem);
    C* bufB = bufA + L * LS;
    C* bufC = bufB + L * LS;
    C* tw = bufC + L * LS;
    fft_twiddles<T, L>(tw);
    const int ntile = (KX + LINES - 1) / LINES;
    const int kx0 = (blockIdx.x % ntile) * LINES;
    const int y = blockIdx.x / ntile;
    const int comp = blockIdx.y;
    const size_t estride = (size_t)L * Spec3<L>::KXP;
    const size_t base = (size_t)y * Spec3<L>::KXP + kx0;
    const int nl = min(LINES, KX - kx0);
    const C* src = R + comp * r_stride + base;
    for (int idx = threadIdx.x; idx < L * LINES; idx += blockDim.x) {
        const int n = idx / LINES, line = idx - n * LINES;
        if (line < nl) bufA[n * LS + line] = src[n * estride + line];
        else { bufA[n * LS + line].x = T(0); bufA[n * LS + line].y = T(0); }
    }
    __syncthreads();
    C* spec = fft_lines<T, L, LINES, LS>(bufA, bufB, tw, false);   // spec is bufA or bufB
    C* w1 = (spec == bufA) ? bufB : bufA;
    for (int f = 0; f < K.nconv; ++f) {
        for (int idx = threadIdx.x; idx < L * LINES; idx += blockDim.x) {
            const int n = idx / LINES, line = idx - n * LINES;
            if (line < nl) {
                w1[n * LS + line] = k3_apply<T, L>(K, comp, f, kx0 + line, y, n, spec[n * LS + line]);
            } else {   // padding lines of the last kx tile: kx > N/2 has no table entry
                w1[n * LS + line].x = T(0);
                w1[n * LS + line].y = T(0);
            }
        }
        __syncthreads();
        const C* r = fft_lines<T, L, LINES, LS>(w1, bufC, tw, true);
        C* dst = out + ((size_t)comp * K.nconv + f) * out_stride + base;
        for (int idx = threadIdx.x; idx < L * LINES; idx += blockDim.x) {
            const int n = idx / LINES, line = idx - n * LINES;
            if (line < nl) dst[n * estride + line] = r[n * LS + line];
        }
        __syncthreads();
    }
}

// z pass of the adjoint: forward z-FFT of every field's dPhi/dn spectrum,
// accumulate sign_f * kernel_f * spectrum_f, inverse z-FFT of the sum.
template <typename T, int L, int LINES>
__global__ void __launch_bounds__(FFT_THREADS, (FftMinBlocks<T, L>::value))
fft_z_adjoint(const typename V2<T>::t* __restrict__ in, size_t in_stride, typename V2<T>::t* __restrict__ out,
              size_t out_stride, KTab3 K, const AAState* __restrict__ st)
{
    typedef typename V2<T>::t C;
    constexpr int LS = LINES + 1;
    constexpr int KX = L / 2 + 1;
    if (fft_skip(st)) return;
    extern __shared__ __align__(16) unsigned char fft_smem[];
    C* bufA = reinterpret_cast<C*>(fft_smem);
    C* bufB = bufA + L * LS;
    C* acc = bufB + L * LS;
    C* tw = acc + L * LS;
    fft_twiddles<T, L>(tw);
    const int ntile = (KX + LINES - 1) / LINES;
    const int kx0 = (blockIdx.x % ntile) * LINES;
    const int y = blockIdx.x / ntile;
    const int comp = blockIdx.y;
    const size_t estride = (size_t)L * Spec3<L>::KXP;
    const size_t base = (size_t)y * Spec3<L>::KXP + kx0;
    const int nl = min(LINES, KX - kx0);
    // every slot of the padded [n * LS + line] layout starts at zero
    for (int idx = threadIdx.x; idx < L * LS; idx += blockDim.x) { acc[idx].x = T(0); acc[idx].y = T(0); }
    for (int f = 0; f < K.nconv; ++f) {
        const C* src = in + ((size_t)comp * K.nconv + f) * in_stride + base;
        for (int idx = threadIdx.x; idx < L * LINES; idx += blockDim.x) {
            const int n = idx / LINES, line = idx - n * LINES;
            if (line < nl) bufA[n * LS + line] = src[n * estride + line];
            else { bufA[n * LS + line].x = T(0); bufA[n * LS + line].y = T(0); }
        }
        __syncthreads();
        const C* r = fft_lines<T, L, LINES, LS>(bufA, bufB, tw, false);
        const T sign = (f >= 2 && f <= 4) ? T(-1) : T(1);   // vector fields: δfδρ .-= (weighted_densities.jl:381)
        for (int idx = threadIdx.x; idx < L * LINES; idx += blockDim.x) {
            const int n = idx / LINES, line = idx - n * LINES;
            if (line >= nl) continue;   // padding lines of the last kx tile
            const C v = k3_apply<T, L>(K, comp, f, kx0 + line, y, n, r[n * LS + line]);
            acc[n * LS + line].x += sign * v.x;
            acc[n * LS + line].y += sign * v.y;
        }
        __syncthreads();
    }
    const C* r = fft_lines<T, L, LINES, LS>(acc, bufA, tw, true);
    C* dst = out + comp * out_stride + base;
    for (int idx = threadIdx.x; idx < L * LINES; idx += blockDim.x) {
        const int n = idx / LINES, line = idx - n * LINES;
        if (line < nl) dst[n * estride + line] = r[n * LS + line];
    }
}
