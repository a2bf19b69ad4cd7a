// Strided FFT passes of the 3D weighted densities with TMA tile movement (sm_100a).
//
// The y and z passes of the half spectrum (layout [field][z][y][kx], rows of KXP
// complex, fft3d.cuh) read and write tiles of LINES consecutive kx by L rows that lie
// a row (y) or a plane (z) apart in memory.  Here every block is persistent over tiles:
// a tensor-map load (cp.async.bulk.tensor, completion on an mbarrier) brings the next
// tile into shared memory while the block transforms the current one, and the result
// leaves by a tensor-map store (bulk group) that the block does not wait for until the
// buffer is needed again.  No thread issues per-element global loads; the tile layout
// in shared memory is [n][line] with 16-byte complex (8-byte in FP32) entries, which the
// two register passes of fft_lines read without bank conflicts.
//
// Tensor maps describe a spectrum buffer as a 4D tensor of T: {2 KX (re/im of kx),
// L (y), L (z), fields}, row strides 2 KXP T (a multiple of 16 bytes), box {2 LINES,
// L, 1, 1} (y pass) or {2 LINES, 1, L, 1} (z pass).  The kx tile of the Nyquist entry
// runs past 2 KX: loads fill zeros there and stores clip it.  Every coordinate is >= 0
// and the innermost one, 2 kx0 T, is a multiple of 16 bytes (kx0 a multiple of LINES).
// No load uses cluster multicast, and the maps only ever cover this GPU's own buffers.
//
// Every wait on an mbarrier is bounded (TMA_WAIT_LIMIT polls): a wait that runs out
// sets the error word (TMA_ERR_TIMEOUT), waits, again bounded, for the block's own
// copies in flight and leaves the kernel; the host reports the error.
#pragma once
#include <cuda.h>
#include <cstdint>
#include "fft3d.cuh"

#define TMA_WAIT_LIMIT (1LL << 22)
#define TMA_ERR_TIMEOUT 1
#define FFT_TMA_THREADS 128

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// bounded wait for the completion of phase `parity` of the barrier
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_addr(bar);
    for (long long it = 0; it < TMA_WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, const void* src, int c0, int c1, int c2, int c3)
{
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(smem_addr(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
}

__device__ __forceinline__ void tma_store_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// at most N store groups of this thread still reading shared memory
template <int N>
__device__ __forceinline__ void tma_store_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// every store group of this thread complete (written to global memory)
__device__ __forceinline__ void tma_store_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// shared-memory writes of the threads become visible to the async (TMA) proxy
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// The dynamic shared memory of every kernel here starts at a 128-byte boundary (tensor
// copies need it; the extern array is only guaranteed 16 bytes): the host adds
// TMA_SMEM_SLACK bytes and the kernel rounds its base up.  The kernels declare no static
// shared memory; their block-uniform flag lives after the mbarriers.
#define TMA_SMEM_SLACK 256
#define TMA_ERR_ALIGN 2
extern __shared__ __align__(128) unsigned char tma_smem_raw[];
__device__ __forceinline__ unsigned char* tma_smem_base()
{
    return tma_smem_raw + ((128u - (smem_addr(tma_smem_raw) & 127u)) & 127u);
}

// kx tiles of a half-spectrum row
template <int L, int LINES>
struct TmaTiles {
    static constexpr int KX = L / 2 + 1;
    static constexpr int NT = (KX + LINES - 1) / LINES;
};

// tensor coordinates {2 kx0, y, z, field} of tile t of a y pass (outer = z) or z pass (outer = y)
template <int L, int LINES>
__device__ __forceinline__ void tma_tile_coords(int t, int axis, int& c0, int& c1, int& c2, int& c3)
{
    constexpr int NT = TmaTiles<L, LINES>::NT;
    const int kt = t % NT;
    const int r = t / NT;
    const int outer = r % L;
    c3 = r / L;
    c0 = 2 * kt * LINES;
    c1 = (axis == 1) ? 0 : outer;
    c2 = (axis == 1) ? outer : 0;
}

// block-uniform error exit: the block's own loads in flight on `pending` (or nullptr) and its
// stores complete, then the error word is set
__device__ __forceinline__ void tma_error_exit(int* err, uint64_t* pending, uint32_t parity)
{
    if (threadIdx.x == 0) {
        if (pending) mbar_wait(pending, parity);
        tma_store_wait_all();
        atomicExch(err, TMA_ERR_TIMEOUT);
    }
}

// ---------------------------------------------------------------------------
// in-place y or z pass over `nfields` spectra (axis 1: y, 2: z)
// shared memory: two tile buffers (current, next), the FFT scratch tile, twiddles, 2 mbarriers
// ---------------------------------------------------------------------------
template <typename T, int L, int LINES>
__host__ __device__ constexpr size_t fft_tma_smem_yz()
{
    return (3 * (size_t)L * LINES + L / 2) * sizeof(typename V2<T>::t) + 2 * sizeof(uint64_t) + 16 + TMA_SMEM_SLACK;
}

template <typename T, int L, int LINES>
__global__ void __launch_bounds__(FFT_TMA_THREADS)
fft_yz_tma(const __grid_constant__ CUtensorMap tm, int axis, int inverse, int nfields, const AAState* __restrict__ st,
           int* __restrict__ err)
{
    typedef typename V2<T>::t C;
    constexpr int TILE = L * LINES;
    constexpr uint32_t TBYTES = TILE * sizeof(C);
    if (fft_skip(st)) return;
    unsigned char* smem = tma_smem_base();
    C* buf0 = reinterpret_cast<C*>(smem);
    C* buf1 = buf0 + TILE;
    C* work = buf1 + TILE;
    C* tw = work + TILE;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tw + L / 2);
    int& ok_s = *reinterpret_cast<int*>(bar + 2);
    const int ntiles = nfields * L * TmaTiles<L, LINES>::NT;
    int t = blockIdx.x;
    if (t >= ntiles) return;
    if ((smem_addr(smem) & 127u) || (smem_addr(bar) & 7u)) {   // cannot happen: base rounded up above
        if (threadIdx.x == 0) atomicExch(err, TMA_ERR_ALIGN);
        return;
    }
    fft_twiddles<T, L>(tw);
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
        int c0, c1, c2, c3;
        tma_tile_coords<L, LINES>(t, axis, c0, c1, c2, c3);
        mbar_expect_tx(&bar[0], TBYTES);
        tma_load_4d(buf0, &tm, &bar[0], c0, c1, c2, c3);
    }
    for (int i = 0; t < ntiles; ++i, t += gridDim.x) {
        const int cur = i & 1;
        C* x = cur ? buf1 : buf0;
        C* nx = cur ? buf0 : buf1;
        const int tn = t + gridDim.x;
        if (threadIdx.x == 0) {
            if (tn < ntiles) {   // prefetch: the store that last read nx has finished reading
                tma_store_wait_read<0>();
                int c0, c1, c2, c3;
                tma_tile_coords<L, LINES>(tn, axis, c0, c1, c2, c3);
                mbar_expect_tx(&bar[cur ^ 1], TBYTES);
                tma_load_4d(nx, &tm, &bar[cur ^ 1], c0, c1, c2, c3);
            }
            ok_s = mbar_wait(&bar[cur], (i >> 1) & 1);
        }
        __syncthreads();
        if (!ok_s) {
            tma_error_exit(err, tn < ntiles ? &bar[cur ^ 1] : nullptr, ((i + 1) >> 1) & 1);
            return;
        }
        fft_lines<T, L, LINES, LINES>(x, work, tw, inverse != 0);   // result in x, block synchronised
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            int c0, c1, c2, c3;
            tma_tile_coords<L, LINES>(t, axis, c0, c1, c2, c3);
            tma_store_4d(&tm, x, c0, c1, c2, c3);
            tma_store_commit();
        }
    }
    if (threadIdx.x == 0) tma_store_wait_all();
}

// ---------------------------------------------------------------------------
// z pass of the weighted densities: forward z-FFT of a tile of the rho spectrum, then for
// every convolved field the kernel multiply and the inverse z-FFT, stored to that field's
// spectrum.  Tiles (comp, y, kx tile).  Shared memory: two input buffers (current spectrum,
// prefetch), FFT scratch, two output buffers (alternating, each released when its store
// has read it), twiddles, 2 mbarriers.
// ---------------------------------------------------------------------------
template <typename T, int L, int LINES>
__host__ __device__ constexpr size_t fft_tma_smem_zeval()
{
    return (5 * (size_t)L * LINES + L / 2) * sizeof(typename V2<T>::t) + 2 * sizeof(uint64_t) + 16 + TMA_SMEM_SLACK;
}

template <typename T, int L, int LINES>
__global__ void __launch_bounds__(FFT_TMA_THREADS)
fft_z_eval_tma(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout, KTab3 K, int nc,
               const AAState* __restrict__ st, int* __restrict__ err)
{
    typedef typename V2<T>::t C;
    constexpr int TILE = L * LINES;
    constexpr uint32_t TBYTES = TILE * sizeof(C);
    constexpr int KX = L / 2 + 1;
    if (fft_skip(st)) return;
    unsigned char* smem = tma_smem_base();
    C* in0 = reinterpret_cast<C*>(smem);
    C* in1 = in0 + TILE;
    C* work = in1 + TILE;
    C* out0 = work + TILE;
    C* out1 = out0 + TILE;
    C* tw = out1 + TILE;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tw + L / 2);
    int& ok_s = *reinterpret_cast<int*>(bar + 2);
    const int ntiles = nc * L * TmaTiles<L, LINES>::NT;
    int t = blockIdx.x;
    if (t >= ntiles) return;
    if ((smem_addr(smem) & 127u) || (smem_addr(bar) & 7u)) {   // cannot happen: base rounded up above
        if (threadIdx.x == 0) atomicExch(err, TMA_ERR_ALIGN);
        return;
    }
    fft_twiddles<T, L>(tw);
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
        int c0, c1, c2, c3;
        tma_tile_coords<L, LINES>(t, 2, c0, c1, c2, c3);
        mbar_expect_tx(&bar[0], TBYTES);
        tma_load_4d(in0, &tin, &bar[0], c0, c1, c2, c3);
    }
    int nstore = 0;
    for (int i = 0; t < ntiles; ++i, t += gridDim.x) {
        const int cur = i & 1;
        C* x = cur ? in1 : in0;
        C* nx = cur ? in0 : in1;
        const int tn = t + gridDim.x;
        if (threadIdx.x == 0) {
            if (tn < ntiles) {   // nx was last read by this block's threads (previous tile), not by a store
                int c0, c1, c2, c3;
                tma_tile_coords<L, LINES>(tn, 2, c0, c1, c2, c3);
                mbar_expect_tx(&bar[cur ^ 1], TBYTES);
                tma_load_4d(nx, &tin, &bar[cur ^ 1], c0, c1, c2, c3);
            }
            ok_s = mbar_wait(&bar[cur], (i >> 1) & 1);
        }
        __syncthreads();
        if (!ok_s) {
            tma_error_exit(err, tn < ntiles ? &bar[cur ^ 1] : nullptr, ((i + 1) >> 1) & 1);
            return;
        }
        int c0, c1, c2, comp;
        tma_tile_coords<L, LINES>(t, 2, c0, c1, c2, comp);
        const int kx0 = c0 / 2, y = c1;
        C* spec = fft_lines<T, L, LINES, LINES>(x, work, tw, false);   // forward z: spectrum of rho in x
        for (int f = 0; f < K.nconv; ++f) {
            C* o = (nstore & 1) ? out1 : out0;
            if (threadIdx.x == 0) tma_store_wait_read<1>();   // the store two back has read o
            __syncthreads();
            for (int idx = threadIdx.x; idx < TILE; idx += blockDim.x) {
                const int n = idx / LINES, line = idx - n * LINES;
                if (kx0 + line < KX) {
                    o[idx] = k3_apply<T, L>(K, comp, f, kx0 + line, y, n, spec[idx]);
                } else {   // lines past the Nyquist entry: no kernel value (their store is clipped)
                    o[idx].x = T(0);
                    o[idx].y = T(0);
                }
            }
            __syncthreads();
            fft_lines<T, L, LINES, LINES>(o, work, tw, true);
            fence_proxy_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                tma_store_4d(&tout, o, c0, y, 0, comp * K.nconv + f);
                tma_store_commit();
            }
            ++nstore;
        }
    }
    if (threadIdx.x == 0) tma_store_wait_all();
}

// ---------------------------------------------------------------------------
// z pass of the adjoint: for every convolved field the forward z-FFT of its dPhi/dn
// spectrum tile, times sign_f * kernel_f, accumulated; the inverse z-FFT of the sum is
// stored to the component's spectrum.  Loads run one (tile, field) unit ahead.
// Shared memory: two input buffers, FFT scratch, the accumulator, twiddles, 2 mbarriers.
// ---------------------------------------------------------------------------
template <typename T, int L, int LINES>
__host__ __device__ constexpr size_t fft_tma_smem_zadj()
{
    return (4 * (size_t)L * LINES + L / 2) * sizeof(typename V2<T>::t) + 2 * sizeof(uint64_t) + 16 + TMA_SMEM_SLACK;
}

template <typename T, int L, int LINES>
__global__ void __launch_bounds__(FFT_TMA_THREADS)
fft_z_adjoint_tma(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout, KTab3 K, int nc,
                  const AAState* __restrict__ st, int* __restrict__ err)
{
    typedef typename V2<T>::t C;
    constexpr int TILE = L * LINES;
    constexpr uint32_t TBYTES = TILE * sizeof(C);
    constexpr int KX = L / 2 + 1;
    if (fft_skip(st)) return;
    unsigned char* smem = tma_smem_base();
    C* in0 = reinterpret_cast<C*>(smem);
    C* in1 = in0 + TILE;
    C* work = in1 + TILE;
    C* acc = work + TILE;
    C* tw = acc + TILE;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tw + L / 2);
    int& ok_s = *reinterpret_cast<int*>(bar + 2);
    const int NF = K.nconv;
    const int ntiles = nc * L * TmaTiles<L, LINES>::NT;
    int t = blockIdx.x;
    if (t >= ntiles) return;
    if ((smem_addr(smem) & 127u) || (smem_addr(bar) & 7u)) {   // cannot happen: base rounded up above
        if (threadIdx.x == 0) atomicExch(err, TMA_ERR_ALIGN);
        return;
    }
    fft_twiddles<T, L>(tw);
    // unit (t, f): field f of the component of tile t, fields comp * NF + f of the input
    auto issue = [&](int tt, int f, int b) {
        int c0, c1, c2, comp;
        tma_tile_coords<L, LINES>(tt, 2, c0, c1, c2, comp);
        mbar_expect_tx(&bar[b], TBYTES);
        tma_load_4d(b ? in1 : in0, &tin, &bar[b], c0, c1, c2, comp * NF + f);
    };
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
        issue(t, 0, 0);
    }
    int v = 0;   // units consumed by this block
    for (; t < ntiles; t += gridDim.x) {
        int c0, c1, c2, comp;
        tma_tile_coords<L, LINES>(t, 2, c0, c1, c2, comp);
        const int kx0 = c0 / 2, y = c1;
        if (threadIdx.x == 0) tma_store_wait_read<0>();   // the previous tile's store has read acc
        __syncthreads();
        for (int idx = threadIdx.x; idx < TILE; idx += blockDim.x) {
            acc[idx].x = T(0);
            acc[idx].y = T(0);
        }
        for (int f = 0; f < NF; ++f, ++v) {
            const int b = v & 1;
            C* x = b ? in1 : in0;
            // prefetch the next unit into the other buffer (its previous unit was consumed)
            const bool more = (f + 1 < NF) || (t + (int)gridDim.x < ntiles);
            if (threadIdx.x == 0) {
                if (more) issue(f + 1 < NF ? t : t + gridDim.x, f + 1 < NF ? f + 1 : 0, b ^ 1);
                ok_s = mbar_wait(&bar[b], (v >> 1) & 1);
            }
            __syncthreads();
            if (!ok_s) {
                tma_error_exit(err, more ? &bar[b ^ 1] : nullptr, ((v + 1) >> 1) & 1);
                return;
            }
            const C* r = fft_lines<T, L, LINES, LINES>(x, work, tw, false);
            const T sign = (f >= 2 && f <= 4) ? T(-1) : T(1);   // vector fields: δfδρ .-= (weighted_densities.jl:381)
            for (int idx = threadIdx.x; idx < TILE; idx += blockDim.x) {
                const int n = idx / LINES, line = idx - n * LINES;
                if (kx0 + line >= KX) continue;   // lines past the Nyquist entry
                const C w = k3_apply<T, L>(K, comp, f, kx0 + line, y, n, r[idx]);
                acc[idx].x += sign * w.x;
                acc[idx].y += sign * w.y;
            }
            __syncthreads();
        }
        fft_lines<T, L, LINES, LINES>(acc, work, tw, true);
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tma_store_4d(&tout, acc, c0, y, 0, comp);
            tma_store_commit();
        }
    }
    if (threadIdx.x == 0) tma_store_wait_all();
}

// ---------------------------------------------------------------------------
// Fused x pass of the functional derivative: inverse x-FFT of the 8 convolved-field
// spectra, Phi / dPhi/dn (fused reverse sweep, functional.cuh), forward x-FFT of the 8
// dPhi/dn fields, for 2 LF real rows of every component per block.  The weighted
// densities and their derivatives never leave shared memory; each field's block of rows
// is one contiguous run of 2 LF x KXP complex in the spectrum, moved by 1D bulk copies
// (cp.async.bulk, load on an mbarrier, store in a bulk group), double-buffered.
// Per line and per point the arithmetic of fft_x_c2r, phi_point and fft_x_r2c.
// Global writes: the 8 spectra (in place of the ones read) and dPhi/dn of the rho field.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)),
                 "r"(bytes)
                 : "memory");
}

#define FUSED_THREADS 512   // Phi runs on two threads per point (hard sphere + association / chain + dispersion)
#define FUSED_SMEM_MAX 232448   // dynamic shared memory of one block on sm_100

template <typename T, int L, int NC, int LF>
__host__ __device__ constexpr size_t fused_smem_bytes()
{
    typedef typename V2<T>::t C;
    return (size_t)NC * 9 * 2 * LF * L * sizeof(T)               // the 9 fields of every component, 2 LF rows
           + 2 * (size_t)2 * LF * Spec3<L>::KXP * sizeof(C)      // two staging blocks of spectrum rows
           + 2 * (size_t)L * (LF + 1) * sizeof(C)                // FFT line buffers
           + (size_t)(L / 2) * sizeof(C) + 2 * sizeof(uint64_t)  // twiddles, mbarriers
           + 16 + TMA_SMEM_SLACK;                                 // flag, alignment slack
}

// lines (row pairs) per block: the largest power of two up to FftLines whose block fits
template <typename T, int L, int NC>
struct FusedLines {
    static constexpr int L16 = 16, L8 = 8, L4 = 4, L2 = 2;
    static constexpr int top = FftLines<T, L>::value;
    static constexpr int value = (top >= 16 && fused_smem_bytes<T, L, NC, L16>() <= FUSED_SMEM_MAX) ? 16
                                 : (top >= 8 && fused_smem_bytes<T, L, NC, L8>() <= FUSED_SMEM_MAX) ? 8
                                 : (fused_smem_bytes<T, L, NC, L4>() <= FUSED_SMEM_MAX) ? 4 : 2;
};

template <typename T, int L, int NC, int LF>
__global__ void __launch_bounds__(FUSED_THREADS, 1)
fft_x_phi_fused(typename V2<T>::t* __restrict__ spec, size_t nspec, const SysDev* __restrict__ sys, T scale_in,
                const AAState* __restrict__ st, int* __restrict__ err)
{
    typedef typename V2<T>::t C;
    constexpr int ROWS = 2 * LF, KX = L / 2 + 1, KXP = Spec3<L>::KXP, LS = LF + 1, NF = 9, NCONV = 8;
    constexpr int FIELD = ROWS * L;                 // reals of one field in the block
    constexpr int SROW = ROWS * KXP;                // complex of one staged spectrum block
    constexpr uint32_t SBYTES = SROW * sizeof(C);
    constexpr int NU = NC * NCONV;                  // (component, field) units
    if (fft_skip(st)) return;
    unsigned char* smem = tma_smem_base();
    T* F = reinterpret_cast<T*>(smem);
    C* stage0 = reinterpret_cast<C*>(F + (size_t)NC * NF * FIELD);
    C* stage1 = stage0 + SROW;
    C* bufA = stage1 + SROW;
    C* bufB = bufA + L * LS;
    C* tw = bufB + L * LS;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tw + L / 2);
    int& ok_s = *reinterpret_cast<int*>(bar + 2);
    const SysDev& S = sys[0];
    const size_t npts = (size_t)L * L * L;
    const size_t row0 = (size_t)blockIdx.x * ROWS;
    auto unit_src = [&](int u) { return spec + (size_t)u * nspec + row0 * KXP; };   // u = i * NCONV + f
    if ((smem_addr(smem) & 127u) || (smem_addr(bar) & 7u)) {   // cannot happen: base rounded up above
        if (threadIdx.x == 0) atomicExch(err, TMA_ERR_ALIGN);
        return;
    }
    fft_twiddles<T, L>(tw);
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
        mbar_expect_tx(&bar[0], SBYTES);
        bulk_load(stage0, unit_src(0), SBYTES, &bar[0]);
    }
    // ---- inverse x pass of the convolved fields, into F (scaled by N_A L^3 / N^3) ----
    for (int u = 0; u < NU; ++u) {
        const int b = u & 1;
        C* sg = b ? stage1 : stage0;
        if (threadIdx.x == 0) {
            if (u + 1 < NU) {   // the other staging block was consumed by unit u - 1
                mbar_expect_tx(&bar[b ^ 1], SBYTES);
                bulk_load(b ? stage0 : stage1, unit_src(u + 1), SBYTES, &bar[b ^ 1]);
            }
            ok_s = mbar_wait(&bar[b], (u >> 1) & 1);
        }
        __syncthreads();
        if (!ok_s) {
            tma_error_exit(err, u + 1 < NU ? &bar[b ^ 1] : nullptr, ((u + 1) >> 1) & 1);
            return;
        }
        for (int idx = threadIdx.x; idx < LF * L; idx += blockDim.x) {
            const int line = idx / L, k = idx - line * L;
            const int kk = (k <= L / 2) ? k : L - k;
            C a = sg[(2 * line) * KXP + kk];
            C c = sg[(2 * line + 1) * KXP + kk];
            if (k > L / 2) { a = cconj(a); c = cconj(c); }
            C z;   // Z = X_a + i X_b
            z.x = a.x - c.y;
            z.y = a.y + c.x;
            bufA[k * LS + line] = z;
        }
        __syncthreads();
        const C* z = fft_lines<T, L, LF, LS>(bufA, bufB, tw, true);
        const int i = u / NCONV, f = u - i * NCONV;
        T* dst = F + ((size_t)i * NF + f + 1) * FIELD;
        for (int idx = threadIdx.x; idx < FIELD; idx += blockDim.x) {
            const int r = idx / L, n = idx - r * L;
            const C c = z[n * LS + (r >> 1)];
            dst[idx] = ((r & 1) ? c.y : c.x) * scale_in;
        }
        __syncthreads();
    }
    // ---- the rho field: n_0 = N_A L^3 rho ----
    for (int idx = threadIdx.x; idx < NC * FIELD; idx += blockDim.x) {
        const int i = idx / FIELD, p = idx - i * FIELD;
        F[(size_t)i * NF * FIELD + p] = T(S.NA * S.rho[(size_t)i * npts + row0 * L + p]);
    }
    __syncthreads();
    // ---- Phi / dPhi/dn at every point of the block, in place, two threads per point ----
    // items w < FIELD: hard sphere + association (fields 1 .. 5: n2, n3, the vector n2);
    // items FIELD + p: chain + dispersion (fields 0, 6, 7, 8).  The halves read and write
    // disjoint fields (phi_grad's PART split), so no barrier sits between them.
    T* dfield = reinterpret_cast<T*>(S.dfield);
    for (int w = threadIdx.x; w < 2 * FIELD; w += blockDim.x) {
        const bool first = w < FIELD;
        const int p = first ? w : w - FIELD;
        T n[NC][NF], g[NC][NF];
#pragma unroll
        for (int i = 0; i < NC; ++i)
#pragma unroll
            for (int a = 0; a < NF; ++a) {
                const bool mine = (a >= 1 && a <= 5) == first;
                n[i][a] = mine ? F[((size_t)i * NF + a) * FIELD + p] : T(1);
            }
        if (first) phi_grad<T, NC, 3, false, 1>(S.phi, n, g);
        else phi_grad<T, NC, 3, false, 2>(S.phi, n, g);
#pragma unroll
        for (int i = 0; i < NC; ++i) {
#pragma unroll
            for (int a = 1; a < NF; ++a)
                if ((a >= 1 && a <= 5) == first) F[((size_t)i * NF + a) * FIELD + p] = g[i][a];
            if (!first) dfield[(size_t)i * NF * npts + row0 * L + p] = g[i][0];   // the rho field (EL step)
        }
    }
    __syncthreads();
    // ---- forward x pass of the 8 dPhi/dn fields, stored over the spectra read above ----
    for (int u = 0; u < NU; ++u) {
        C* o = (u & 1) ? stage1 : stage0;
        if (threadIdx.x == 0) tma_store_wait_read<1>();   // the store two units back has read o
        const int i = u / NCONV, f = u - i * NCONV;
        const T* src = F + ((size_t)i * NF + f + 1) * FIELD;
        for (int idx = threadIdx.x; idx < FIELD; idx += blockDim.x) {
            const int r = idx / L, n = idx - r * L;
            C& c = bufA[n * LS + (r >> 1)];
            if (r & 1) c.y = src[idx]; else c.x = src[idx];
        }
        __syncthreads();
        const C* Z = fft_lines<T, L, LF, LS>(bufA, bufB, tw, false);
        for (int idx = threadIdx.x; idx < LF * KX; idx += blockDim.x) {
            const int line = idx / KX, k = idx - line * KX;
            const C zk = Z[k * LS + line];
            const C zm = cconj(Z[((L - k) % L) * LS + line]);
            C a, c;   // X_a = (Z_k + conj Z_{L-k}) / 2,  X_b = (Z_k - conj Z_{L-k}) / (2i)
            a.x = T(0.5) * (zk.x + zm.x);
            a.y = T(0.5) * (zk.y + zm.y);
            c.x = T(0.5) * (zk.y - zm.y);
            c.y = T(-0.5) * (zk.x - zm.x);
            o[(2 * line) * KXP + k] = a;
            o[(2 * line + 1) * KXP + k] = c;
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            bulk_store(unit_src(u), o, SBYTES);
            tma_store_commit();
        }
    }
    if (threadIdx.x == 0) tma_store_wait_all();
}
