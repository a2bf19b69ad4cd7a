"""CPU emulations of the index maps of two device kernels, step by step as the CUDA code
computes them, against direct NumPy results (no GPU).

- `pers_conv_dmma` (csrc/persistent.cuh): the exact circulant convolution of the persistent
  engine as a sum of 8x8 Toeplitz tap blocks times 8-column input slabs on the FP64
  m8n8k4 tensor-core path, reading zero-padded taps and the periodically extended input at
  bank-spread positions; the index ranges are checked against their buffers and the bank
  pairs of every warp load counted.
- `fft_lines` / `fft_reg` / the two-rows-in-one packing of `fft_x_r2c` and `fft_x_c2r`
  (csrc/fft3d.cuh): L = R1 R2 two-pass Cooley-Tukey with radix-2 register DFTs.
"""
import numpy as np
import pytest

PERS_R = 8
FFT_SPLIT = {32: (4, 8), 64: (8, 8), 128: (8, 16), 256: (16, 16)}   # FftSplit<L>


PERS_TPAD = 16


def pers_off(N):
    return (N + 32 + 15) & ~15


def pers_extn(N):
    return pers_off(N) + N + 32 * (PERS_R + 1) + 16


def pers_pos(k):
    return k + 4 * (k >> 4)


def pers_extp(N):
    return pers_extn(N) + 4 * ((pers_extn(N) + 15) >> 4)


def dmma_conv(taps, x):
    """out[j] = sum_q taps[q] x[(j - q) mod N] as pers_conv_dmma forms it: per warp task
    (8 output columns u0..u0+7 of 8 outputs each), m8n8k4 products A_d B_d with
    A_d[a][c] = t(8d + a - c) from the zero-padded taps and B_d[c][n] = x[8(u0 + n - d) + c]
    from the extended input stored at bank-spread positions; tap blocks in pairs into four
    accumulators.  Every read is checked against its buffer, and the B loads of a warp
    must hit each 8-byte bank pair at most twice (2 shared-memory wavefronts)."""
    N = len(taps)
    U = (N + 7) // 8
    nut = (U + 7) // 8
    D = (N + 14) // 8
    EXTN, EXTP, OFF, TS = pers_extn(N), pers_extp(N), pers_off(N), N + 2 * PERS_TPAD
    ext = np.full(EXTP, np.nan)
    for k in range(EXTN):
        ext[pers_pos(k)] = x[(k - OFF) % N]
    tp = np.zeros(TS)
    tp[PERS_TPAD:PERS_TPAD + N] = taps
    out = np.zeros(N)

    def A(q):
        assert 0 <= q + PERS_TPAD < TS, (N, q)
        return tp[q + PERS_TPAD]

    def B(xl):
        assert 0 <= xl < EXTN, (N, xl)
        v = ext[pers_pos(xl)]
        assert np.isfinite(v)
        return v

    for ut in range(nut):
        u0 = 8 * ut
        acc = [np.zeros((8, 8)) for _ in range(4)]

        def step(d, chains):
            for half, ch in zip((0, 4), chains):
                Am = np.zeros((8, 4))
                Bm = np.zeros((4, 8))
                banks = {}
                for r in range(8):
                    for k in range(4):
                        Am[r, k] = A(8 * d + r - k - half)
                        xl = OFF + 8 * (u0 + r) + k - 8 * d + half
                        Bm[k, r] = B(xl)
                        b = pers_pos(xl) % 16
                        banks[b] = banks.get(b, 0) + 1
                assert max(banks.values()) <= 2, (N, d, banks)
                acc[ch] += Am @ Bm

        d = 0
        while d + 1 < D:
            step(d, (0, 1))
            step(d + 1, (2, 3))
            d += 2
        if d < D:
            step(d, (0, 1))
        Dm = (acc[0] + acc[1]) + (acc[2] + acc[3])
        for a in range(8):
            for n in range(8):
                j = 8 * (u0 + n) + a
                if j < N:
                    out[j] = Dm[a, n]
    return out


@pytest.mark.parametrize("N", [8, 9, 15, 16, 17, 64, 100, 186, 257, 400])
def test_dmma_circulant_index_map(N):
    rng = np.random.default_rng(N)
    taps = rng.standard_normal(N)
    x = rng.standard_normal(N)
    ref = np.array([sum(taps[q] * x[(j - q) % N] for q in range(N)) for j in range(N)])
    got = dmma_conv(taps, x)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def bitrev(i, R):
    r, b = 0, 1
    while b < R:
        r = (r << 1) | (i & 1)
        i >>= 1
        b <<= 1
    return r


def fft_tw(L, m, inverse):
    """w_L^m from the half table tw[q] = exp(-2 pi i q / L), q < L/2, as fft_tw reads it."""
    w = np.exp(-2j * np.pi * (m & (L // 2 - 1)) / L)
    if m >= L // 2:
        w = -w
    return np.conj(w) if inverse else w


def fft_reg(v, L, inverse):
    v = list(v)
    R = len(v)
    for i in range(R):
        jr = bitrev(i, R)
        if jr > i:
            v[i], v[jr] = v[jr], v[i]
    half = 1
    while half < R:
        for q in range(half):
            w = fft_tw(L, q * (L // (2 * half)), inverse)
            for b in range(0, R, 2 * half):
                a, c = v[b + q], v[b + q + half] * w
                v[b + q], v[b + q + half] = a + c, a - c
        half <<= 1
    return v


def fft_lines(x, inverse):
    L = len(x)
    R1, R2 = FFT_SPLIT[L]
    y = np.zeros(L, complex)
    for t in range(R2):
        u = fft_reg([x[t + R2 * s] for s in range(R1)], L, inverse)
        for k1 in range(R1):
            y[k1 * R2 + t] = u[k1] * fft_tw(L, t * k1, inverse)
    X = np.zeros(L, complex)
    for k1 in range(R1):
        v = fft_reg([y[k1 * R2 + t] for t in range(R2)], L, inverse)
        for k2 in range(R2):
            X[k1 + R1 * k2] = v[k2]
    return X


@pytest.mark.parametrize("L", sorted(FFT_SPLIT))
def test_fft_two_pass_split(L):
    R1, R2 = FFT_SPLIT[L]
    assert R1 * R2 == L and R1 & (R1 - 1) == 0 and R2 & (R2 - 1) == 0
    rng = np.random.default_rng(L)
    x = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    np.testing.assert_allclose(fft_lines(x, False), np.fft.fft(x), atol=1e-12 * L)
    np.testing.assert_allclose(fft_lines(x, True), np.fft.ifft(x) * L, atol=1e-12 * L)


@pytest.mark.parametrize("L", [32, 128])
def test_fft_two_real_rows_packing(L):
    """fft_x_r2c: rows a, b as z = a + i b, X_a = (Z_k + conj Z_{L-k}) / 2,
    X_b = (Z_k - conj Z_{L-k}) / (2i); fft_x_c2r: the Hermitian extension of X_a + i X_b
    back, real part L a, imaginary part L b."""
    rng = np.random.default_rng(L + 1)
    a, b = rng.standard_normal(L), rng.standard_normal(L)
    Z = fft_lines(a + 1j * b, False)
    KX = L // 2 + 1
    Xa = np.array([(Z[k] + np.conj(Z[(L - k) % L])) / 2 for k in range(KX)])
    Xb = np.array([(Z[k] - np.conj(Z[(L - k) % L])) / 2j for k in range(KX)])
    np.testing.assert_allclose(Xa, np.fft.rfft(a), atol=1e-12 * L)
    np.testing.assert_allclose(Xb, np.fft.rfft(b), atol=1e-12 * L)
    z = np.zeros(L, complex)
    for k in range(L):
        kk = k if k <= L // 2 else L - k
        xa, xb = Xa[kk], Xb[kk]
        if k > L // 2:
            xa, xb = np.conj(xa), np.conj(xb)
        z[k] = xa + 1j * xb
    back = fft_lines(z, True) / L
    np.testing.assert_allclose(back.real, a, atol=1e-12)
    np.testing.assert_allclose(back.imag, b, atol=1e-12)


# ---------------------------------------------------------------------------
# taps_table_kernel (csrc/kernels.cuh): the circulant taps from tabulated closed forms
# at k <= N/2 and twiddles, frequencies k and N - k folded into one term.
# ---------------------------------------------------------------------------
def _kernel_hat_1d(ktype, w, R):
    """kernel_hat_1d (type 3 returns the coefficient of i of the odd vector kernel)."""
    two_pi = 2 * np.pi
    wb = abs(w)
    if ktype == 1:
        return 2 * R / two_pi if wb == 0 else 2 * np.sin(wb * R) / wb / two_pi
    if ktype == 2:
        if wb == 0:
            return 4 * np.pi * R ** 3 / 3 / two_pi ** 3
        return 4 * np.pi / wb ** 3 * (np.sin(wb * R) - R * wb * np.cos(wb * R)) / two_pi ** 3
    if wb == 0:
        return 4 * np.pi * R / two_pi ** 3
    return 4 * np.pi * w / wb ** 3 * (np.sin(wb * R) - R * wb * np.cos(wb * R)) / two_pi ** 3


def taps_table(N, span, L, ktype, R):
    """The kernel's arithmetic, thread by thread: om[k] for k <= N/2, the index j = k q
    mod N advanced by q per step (two accumulators), the pair/Nyquist terms."""
    H, M = N // 2 + 1, (N - 1) // 2
    cs = np.cos(2 * np.pi * np.arange(N) / N)
    sn = np.sin(2 * np.pi * np.arange(N) / N)
    om = np.array([_kernel_hat_1d(ktype, k / span * L, R) for k in range(H)])
    tab = sn if ktype == 3 else cs
    out = np.empty(N)
    for q in range(N):
        acc = [0.0, 0.0]
        j = 0
        k = 1
        while k + 1 <= M:
            j = (j + q) - (N if j + q >= N else 0)
            assert 0 <= j < N
            acc[0] += om[k] * tab[j]
            j = (j + q) - (N if j + q >= N else 0)
            acc[1] += om[k + 1] * tab[j]
            k += 2
        if k <= M:
            j = (j + q) - (N if j + q >= N else 0)
            acc[0] += om[k] * tab[j]
        if ktype == 3:
            t = -2 * (acc[0] + acc[1])
        else:
            t = om[0] + 2 * (acc[0] + acc[1])
            if N % 2 == 0:
                t += -om[N // 2] if q % 2 else om[N // 2]
        out[q] = t / N
    return out


@pytest.mark.parametrize("N", [8, 9, 100, 143, 201, 256])
@pytest.mark.parametrize("ktype", [1, 2, 3])
def test_taps_table_equals_inverse_dft(N, ktype):
    """Re(ifft(Omega sampled at L fftfreq(N, N/span))) of the reference's sampled kernel
    (weighted_densities.jl:28-80,193-246; fftfreq convention of structure.jl:153-162)."""
    span, L = 4.0 * 3.7, 3.7
    R = 2 * np.pi * 0.5 * 0.95
    w = np.fft.fftfreq(N) * N / span * L
    K = np.array([_kernel_hat_1d(ktype, x, R) for x in w])
    spec = 1j * K if ktype == 3 else K.astype(complex)
    ref = np.real(np.fft.ifft(spec))
    got = taps_table(N, span, L, ktype, R)
    assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))


# ---------------------------------------------------------------------------
# TMA tiles of the strided 3D passes (csrc/fft3d_tma.cuh, tensor maps of
# make_spectrum_map in csrc/cdft_b200.cu)
# ---------------------------------------------------------------------------
def fft_lines_of(fp32, L):
    return (16 if L * 4 <= 512 else 8) if fp32 else (16 if L * 8 <= 512 else 8)


def tma_tile_coords(t, axis, L, LINES):
    KX = L // 2 + 1
    NT = (KX + LINES - 1) // LINES
    kt, r = t % NT, t // NT
    outer, field = r % L, r // L
    return 2 * kt * LINES, (0 if axis == 1 else outer), (outer if axis == 1 else 0), field


@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("L", [32, 64, 128, 256])
@pytest.mark.parametrize("axis", [1, 2])
def test_tma_tiles_cover_each_spectrum_entry_once(fp32, L, axis):
    es = 4 if fp32 else 8
    LINES = fft_lines_of(fp32, L)
    KX, KXP = L // 2 + 1, L // 2 + 2
    nfields = 2
    dims = (2 * KX, L, L, nfields)
    strides = (2 * KXP * es, 2 * KXP * es * L, 2 * KXP * es * L * L)
    box = (2 * LINES, L if axis == 1 else 1, 1 if axis == 1 else L, 1)
    # tensor-map rules: 16-byte strides, box rows a multiple of 16 bytes, box dims <= 256
    assert all(s % 16 == 0 for s in strides)
    assert (box[0] * es) % 16 == 0 and max(box) <= 256
    NT = (KX + LINES - 1) // LINES
    cover = np.zeros((nfields, L, L, KX), dtype=np.int32)   # [field][z][y][kx]
    for t in range(nfields * L * NT):
        c0, c1, c2, c3 = tma_tile_coords(t, axis, L, LINES)
        assert min(c0, c1, c2, c3) >= 0                         # no negative store coordinate
        assert (c0 * es) % 16 == 0                              # innermost coordinate on 16 bytes
        assert c1 + box[1] <= dims[1] and c2 + box[2] <= dims[2] and c3 < dims[3]
        kx = np.arange(c0 // 2, c0 // 2 + LINES)
        kx = kx[kx < KX]                                        # past 2 KX: zero-filled, store clipped
        assert kx.size >= 1
        if axis == 1:
            cover[c3, c2, :, kx[0]:kx[-1] + 1] += 1
        else:
            cover[c3, :, c1, kx[0]:kx[-1] + 1] += 1
    assert np.all(cover == 1)


@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("L", [32, 128, 256])
def test_tma_shared_memory_fits(fp32, L):
    """fft_tma_smem_*: the tile buffers and mbarriers of the three kernels fit the 227 KB of
    one block, with the barriers 8-byte aligned and each tile buffer 128-byte aligned."""
    cs = 8 if fp32 else 16
    LINES = fft_lines_of(fp32, L)
    tile = L * LINES * cs
    assert tile % 128 == 0                     # every tile buffer starts on 128 bytes (tensor copies)
    slack = 256                                # TMA_SMEM_SLACK: the base is rounded up to 128 bytes
    for ntiles in (3, 5, 4):
        off_bar = ntiles * tile + (L // 2) * cs
        assert off_bar % 8 == 0
        assert off_bar + 16 + 16 + slack <= 227 * 1024


DGRP_COLS, DGRP_WARPS = 8, 8


def dense_group_emulate(mats, xs, N, slots, active, RT=1):
    """dense_group_kernel<T, RT> (csrc/kernels.cuh) step by step for one column tile: per CTA
    (slot, RT 8-row tiles) and warp, the k = 4 blocks kb = warp, warp + 8, ... in unrolled
    groups of four into four accumulator pairs per row tile, every index checked against its
    buffer; then the fixed-order sum over warps.  Returns out[col][slot][j] (NaN where not
    stored) and the number of times each (row, q) product was formed for column 0."""
    ns = len(xs)
    rtiles = (N + 8 * RT - 1) // (8 * RT)
    nk4 = (N + 3) >> 2
    out = np.full((ns, slots, N), np.nan)
    seen = np.zeros((slots, N, N), dtype=np.int64)
    for bx in range(slots * rtiles):
        slot, j0 = bx // rtiles, (bx % rtiles) * 8 * RT
        red = np.zeros((DGRP_WARPS, RT, 8, 8))
        for warp in range(DGRP_WARPS):
            acc = np.zeros((RT, 4, 8, 8))
            kb = warp
            while kb < nk4:
                for u in range(4):
                    for t in range(RT):
                        for r in range(8):
                            row = min(j0 + 8 * t + r, N - 1)
                            assert 0 <= row < N
                            for k in range(4):
                                q = (kb + u * DGRP_WARPS) * 4 + k
                                if q >= N:
                                    continue
                                assert 0 <= slot * N * N + row * N + q < slots * N * N
                                for c in range(8):
                                    if c < ns and active[c]:
                                        acc[t, u, r, c] += mats[slot, row, q] * xs[c][slot, q]
                                        if j0 + 8 * t + r < N and c == 0:
                                            seen[slot, j0 + 8 * t + r, q] += 1
                kb += 4 * DGRP_WARPS
            for t in range(RT):
                red[warp, t] = (acc[t, 0] + acc[t, 1]) + (acc[t, 2] + acc[t, 3])
        for t in range(RT):
            tot = np.zeros((8, 8))
            for w in range(DGRP_WARPS):
                tot += red[w, t]
            for r in range(8):
                j = j0 + 8 * t + r
                if j >= N:
                    continue
                for c in range(8):
                    if c < ns and active[c]:
                        assert np.isnan(out[c, slot, j])   # every output is stored once
                        out[c, slot, j] = tot[r, c]
    return out, seen


@pytest.mark.parametrize("RT", [1, 2])
@pytest.mark.parametrize("N,ns", [(13, 3), (61, 8), (40, 1)])
def test_dense_group_index_map(N, ns, RT):
    """Every operator row meets every input entry exactly once per output, the loads stay
    inside the operator and input buffers, rows past N and inactive columns are not
    written, and the result is A x per system; 16-row CTAs (RT = 2) give the same bits as
    8-row ones."""
    rng = np.random.default_rng(N)
    slots = 2
    mats = rng.standard_normal((slots, N, N))
    xs = [rng.standard_normal((slots, N)) for _ in range(ns)]
    active = [c != 1 for c in range(8)]
    out, seen = dense_group_emulate(mats, xs, N, slots, active, RT)
    if RT == 2:
        ref, _ = dense_group_emulate(mats, xs, N, slots, active, 1)
        assert np.array_equal(np.nan_to_num(out, nan=7.0), np.nan_to_num(ref, nan=7.0))
    if active[0]:
        assert np.all(seen == 1)
    for c in range(ns):
        if not active[c]:
            assert np.all(np.isnan(out[c]))
            continue
        want = np.einsum("sjq,sq->sj", mats, xs[c])
        np.testing.assert_allclose(out[c], want, rtol=1e-12, atol=1e-12)
