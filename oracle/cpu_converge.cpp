// CPU restatement of the reference's converge! path for 1D Cartesian PC-SAFT systems
// (TEST INFRASTRUCTURE and the timed CPU baseline; never part of the product path).
//
// ClapeyronThermo/cDFT.jl runs converge! on the CPU as Julia code over FFTW, Enzyme and
// KernelAbstractions threads; none of that can run here (no Julia).  This file restates
// the same algorithm in C++17 with OpenMP, so the CPU side of a benchmark is compiled code
// on every host core rather than an interpreter:
//
//  * weighted densities and their adjoint by FFT, as convolve! does
//    (src/utils/integrals.jl:88-96): n_a = Re(IFFT(FFT(rho) .* omega_a)) N_A L^3 with the
//    analytic kernels of src/fields/weighted_densities.jl:28-80,193-246 sampled at
//    L * fftfreq(N, N/(ub - lb)) (src/structure/structure.jl:153-185); the adjoint adds
//    scalar fields and subtracts the vector field (weighted_densities.jl:140-164,368-385).
//    One forward transform of rho per component serves all fields (the reference
//    re-transforms rho per field); arbitrary N by Bluestein's chirp-z algorithm over a
//    radix-2 FFT.
//  * dPhi/dn by forward-mode differentiation of f_res (PCSAFT.jl:110-211, FMT.jl:17-46,
//    assoc.jl:702-769), all NF*nc tangent directions in one pass (the reference's
//    :forward_batch mode, models.jl:399-411) with dual numbers.
//  * the Euler-Lagrange map get_new_profile! (src/methods/converge.jl:108-153) and aasol
//    (src/utils/anderson.jl:301-443: Picard warm-up, Anderson with the CGS2 QR update and
//    the Householder downdate of R, AndersonOK exit codes).
//  * a batch of independent state points is converged with one OpenMP thread per system.
//
// Inputs use the library's own C types (include/cdft_b200.h); only 1D Cartesian FP64
// systems with at most one association pair are handled.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include <omp.h>

#include "../include/cdft_b200.h"

namespace {

using cplx = std::complex<double>;
constexpr double PI = 3.14159265358979323846;
constexpr double NAVO = 6.02214076e23;
constexpr double PSI = 1.3862;   // PCSAFT.jl:53,160

// Gross & Sadowski (2001) universal constants a_ki, b_ki, [k*3 + i] (PCSAFT.jl:86-103)
const double GS_A[21] = {
    0.9105631445, -0.3084016918, -0.0906148351, 0.6361281449, 0.1860531159, 0.4527842806,
    2.6861347891, -2.5030047259, 0.5962700728, -26.547362491, 21.419793629, -1.7241829131,
    97.759208784, -65.25588533, -4.1302112531, -159.59154087, 83.318680481, 13.77663187,
    91.297774084, -33.74692293, -8.6728470368};
const double GS_B[21] = {
    0.7240946941, -0.5755498075, 0.0976883116, 2.2382791861, 0.6995095521, -0.2557574982,
    -4.0025849485, 3.892567339, -9.155856153, -21.003576815, -17.215471648, 20.642075974,
    26.855641363, 192.67226447, -38.804430052, 206.55133841, -161.82646165, 93.626774077,
    -355.60235612, -165.20769346, -29.666905585};

// ---------------------------------------------------------------------------
// FFT: radix-2 for powers of two, Bluestein (chirp-z) otherwise
// ---------------------------------------------------------------------------
struct Fft {
    int N = 0, M = 0;
    bool pow2 = false;
    std::vector<cplx> tw;      // exp(-2 pi i j / M), j < M/2
    std::vector<int> rev;
    std::vector<cplx> chirp;   // exp(-i pi k^2 / N), k < N
    std::vector<cplx> bhat;    // FFT_M of conj(chirp) wrapped to length M
    std::vector<cplx> work;

    void init(int n)
    {
        N = n;
        pow2 = (n & (n - 1)) == 0;
        M = 1;
        if (pow2) M = n;
        else
            while (M < 2 * n - 1) M <<= 1;
        tw.resize(M / 2 > 0 ? M / 2 : 1);
        for (int j = 0; j < M / 2; ++j) tw[j] = std::polar(1.0, -2.0 * PI * j / M);
        rev.assign(M, 0);
        int lg = 0;
        while ((1 << lg) < M) ++lg;
        for (int i = 0; i < M; ++i) {
            int r = 0;
            for (int b = 0; b < lg; ++b) r |= ((i >> b) & 1) << (lg - 1 - b);
            rev[i] = r;
        }
        work.assign(M, 0.0);
        if (pow2) return;
        chirp.resize(N);
        for (long long k = 0; k < N; ++k) {
            const long long k2 = (k * k) % (2LL * N);   // exact argument reduction
            chirp[k] = std::polar(1.0, -PI * (double)k2 / N);
        }
        bhat.assign(M, 0.0);
        bhat[0] = std::conj(chirp[0]);
        for (int k = 1; k < N; ++k) bhat[k] = bhat[M - k] = std::conj(chirp[k]);
        radix2(bhat.data(), false);
    }

    void radix2(cplx* a, bool inverse) const
    {
        for (int i = 0; i < M; ++i)
            if (rev[i] > i) std::swap(a[i], a[rev[i]]);
        for (int len = 2; len <= M; len <<= 1) {
            const int half = len >> 1, step = M / len;
            for (int i = 0; i < M; i += len)
                for (int j = 0; j < half; ++j) {
                    cplx w = tw[j * step];
                    if (inverse) w = std::conj(w);
                    const cplx u = a[i + j], v = a[i + j + half] * w;
                    a[i + j] = u + v;
                    a[i + j + half] = u - v;
                }
        }
    }

    // unnormalised DFT in place: forward sum_j x_j exp(-2 pi i jk/N), inverse with +
    void run(cplx* x, bool inverse)
    {
        if (pow2) {
            radix2(x, inverse);
            return;
        }
        if (inverse)
            for (int j = 0; j < N; ++j) x[j] = std::conj(x[j]);
        for (int j = 0; j < N; ++j) work[j] = x[j] * chirp[j];
        for (int j = N; j < M; ++j) work[j] = 0.0;
        radix2(work.data(), false);
        for (int j = 0; j < M; ++j) work[j] *= bhat[j];
        radix2(work.data(), true);
        const double s = 1.0 / M;
        for (int k = 0; k < N; ++k) x[k] = work[k] * s * chirp[k];
        if (inverse)
            for (int j = 0; j < N; ++j) x[j] = std::conj(x[j]);
    }
};

// ---------------------------------------------------------------------------
// forward-mode dual numbers with K tangents
// ---------------------------------------------------------------------------
template <int K>
struct Dual {
    double v;
    double d[K];
};
template <int K> inline Dual<K> mk(double v) { Dual<K> r; r.v = v; for (int k = 0; k < K; ++k) r.d[k] = 0.0; return r; }
template <int K> inline Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) { Dual<K> r; r.v = a.v + b.v; for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k]; return r; }
template <int K> inline Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) { Dual<K> r; r.v = a.v - b.v; for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k]; return r; }
template <int K> inline Dual<K> operator-(const Dual<K>& a) { Dual<K> r; r.v = -a.v; for (int k = 0; k < K; ++k) r.d[k] = -a.d[k]; return r; }
template <int K> inline Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) { Dual<K> r; r.v = a.v * b.v; for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k]; return r; }
template <int K> inline Dual<K> operator/(const Dual<K>& a, const Dual<K>& b)
{
    Dual<K> r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int K> inline Dual<K> operator+(const Dual<K>& a, double b) { Dual<K> r = a; r.v += b; return r; }
template <int K> inline Dual<K> operator+(double b, const Dual<K>& a) { return a + b; }
template <int K> inline Dual<K> operator-(const Dual<K>& a, double b) { Dual<K> r = a; r.v -= b; return r; }
template <int K> inline Dual<K> operator-(double b, const Dual<K>& a) { Dual<K> r = -a; r.v += b; return r; }
template <int K> inline Dual<K> operator*(const Dual<K>& a, double b) { Dual<K> r; r.v = a.v * b; for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b; return r; }
template <int K> inline Dual<K> operator*(double b, const Dual<K>& a) { return a * b; }
template <int K> inline Dual<K> operator/(const Dual<K>& a, double b) { return a * (1.0 / b); }
template <int K> inline Dual<K> operator/(double a, const Dual<K>& b)
{
    Dual<K> r;
    r.v = a / b.v;
    const double f = -r.v / b.v;
    for (int k = 0; k < K; ++k) r.d[k] = f * b.d[k];
    return r;
}
template <int K> inline Dual<K> dlog(const Dual<K>& a)   // log|a| (Base.log(abs(x)) of the reference)
{
    Dual<K> r;
    r.v = std::log(std::fabs(a.v));
    const double ia = 1.0 / a.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * ia;
    return r;
}
template <int K> inline Dual<K> dsqrt(const Dual<K>& a)
{
    Dual<K> r;
    r.v = std::sqrt(a.v);
    const double f = 0.5 / r.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * f;
    return r;
}
inline double dlog(double a) { return std::log(std::fabs(a)); }
inline double dsqrt(double a) { return std::sqrt(a); }
template <int K> inline double val(const Dual<K>& a) { return a.v; }
inline double val(double a) { return a; }

// ---------------------------------------------------------------------------
// PC-SAFT free-energy density f_res at one point, 1D (NF = 7 fields per component):
// 0 rho, 1 n2-type int rho dz (d/2), 2 n3-type int rho z^2 dz (d/2), 3 vector (d/2),
// 4 int rho z^2 dz (d) [chain], 5 int rho dz (d) [chain lambda], 6 int rho z^2 dz (psi d) [dispersion]
// ---------------------------------------------------------------------------
struct Params {
    int nc;
    double T;
    double m[CDFT_MAX_NC], d[CDFT_MAX_NC];
    double s3[CDFT_MAX_NC * CDFT_MAX_NC];    // (sigma_ij / L)^3
    double eT[CDFT_MAX_NC * CDFT_MAX_NC];    // eps_ij / T
    int has_assoc, aic, ajc;
    double aK;                                // (sigma_ij/L)^3 (exp(eps_AB/T) - 1) kappa_AB
};

// true: the reference's closed White-Bear bracket everywhere (FMT.jl:39-45), including
// |n3| < 0.05 where the series form replaces it by default
bool g_wb_closed = false;

template <typename T>
T wb_bracket(const T& n3, const T& dn, const T& log1dn)
{
    // B(n3) = ln(1-n3)/(12 pi n3^2) + 1/(12 pi n3 (1-n3)^2) (FMT.jl:42-43); for |n3| < 0.05 its
    // Taylor series 12 pi B = sum_j (j+1)(j+3)/(j+2) n3^j (16 terms), where the closed form
    // cancels (the oracle's and the library's form)
    if (!g_wb_closed && std::fabs(val(n3)) < 0.05) {
        T s = n3 * 0.0 + (16.0 * 18.0 / 17.0);
        for (int j = 14; j >= 0; --j) s = s * n3 + ((j + 1.0) * (j + 3.0) / (j + 2.0));
        return s / (12.0 * PI);
    }
    return log1dn / (12.0 * PI * n3 * n3) + 1.0 / (12.0 * PI * n3 * dn * dn);
}

template <typename T, int NC>
T f_res(const T (&n)[NC][7], const Params& P)
{
    // --- hard spheres, White-Bear (FMT.jl:17-46) ---
    T n0 = n[0][0] * 0.0, n1 = n0, n2 = n0, n3 = n0, nv1 = n0, nv2 = n0;
    for (int i = 0; i < NC; ++i) {
        const T nim = n[i][1] * P.m[i];
        n0 = n0 + nim / P.d[i];
        n1 = n1 + 0.5 * nim;
        n2 = n2 + PI * nim * P.d[i];
        nv1 = nv1 + n[i][3] * (P.m[i] / P.d[i]);
        nv2 = nv2 - (2.0 * PI * P.m[i]) * n[i][3];
        n3 = n3 + n[i][2] * P.m[i];
    }
    const T nv1v2 = nv1 * nv2, nv2sq = nv2 * nv2;
    const T dn = 1.0 - n3;
    const T log1dn = dlog(dn);
    const T bkt = wb_bracket(n3, dn, log1dn);
    T res = -n0 * log1dn + (n1 * n2 - nv1v2) / dn + (n2 * n2 * n2 / 3.0 - n2 * nv2sq) * bkt;
    // --- chain (PCSAFT.jl:123-144) ---
    T z3 = n0 * 0.0, z2 = z3;
    for (int i = 0; i < NC; ++i) {
        z3 = z3 + P.m[i] * n[i][4];
        z2 = z2 + (P.m[i] / P.d[i]) * n[i][4];
    }
    z3 = z3 / 8.0;
    z2 = z2 / 8.0;
    const T inv1 = 1.0 / (1.0 - z3);
    for (int i = 0; i < NC; ++i) {
        const T lam = n[i][5] / (2.0 * P.d[i]);
        const T ydd = inv1 + 1.5 * P.d[i] * z2 * inv1 * inv1 + 0.5 * P.d[i] * P.d[i] * z2 * z2 * inv1 * inv1 * inv1;
        res = res - (P.m[i] - 1.0) * n[i][0] * dlog(ydd * lam / n[i][0]);
    }
    // --- dispersion (PCSAFT.jl:150-211) ---
    const double factor = 3.0 / (4.0 * PSI * PSI * PSI * PI);
    T rz[NC];
    T rzs = n0 * 0.0, rzm = rzs, etad = rzs;
    for (int i = 0; i < NC; ++i) {
        rz[i] = n[i][6] * (factor / (P.d[i] * P.d[i] * P.d[i]));
        rzs = rzs + rz[i];
        rzm = rzm + rz[i] * P.m[i];
        etad = etad + (P.m[i] * P.d[i] * P.d[i] * P.d[i]) * rz[i];
    }
    const T mbar = rzm / rzs;
    etad = etad * (PI / 6.0);
    T s1 = n0 * 0.0, s2 = s1;
    for (int i = 0; i < NC; ++i)
        for (int j = 0; j < NC; ++j) {
            const double c = P.m[i] * P.m[j] * P.s3[i * CDFT_MAX_NC + j];
            const double e = P.eT[i * CDFT_MAX_NC + j];
            const T cij = rz[i] * rz[j] * c;
            s1 = s1 + cij * e;
            s2 = s2 + cij * (e * e);
        }
    const T e2 = etad * etad;
    const T ome = 1.0 - etad, tme = 2.0 - etad;
    const T C1 = 1.0 + mbar * (8.0 * etad - 2.0 * e2) / (ome * ome * ome * ome)
                 + (1.0 - mbar) * (20.0 * etad - 27.0 * e2 + 12.0 * etad * e2 - 2.0 * e2 * e2) / (ome * ome * tme * tme);
    const T c1 = (mbar - 1.0) / mbar;
    const T c2 = c1 * (mbar - 2.0) / mbar;
    T I1 = n0 * 0.0, I2 = I1;
    for (int k = 6; k >= 0; --k) {   // evalpoly (Horner)
        I1 = I1 * etad + (GS_A[3 * k] + c1 * GS_A[3 * k + 1] + c2 * GS_A[3 * k + 2]);
        I2 = I2 * etad + (GS_B[3 * k] + c1 * GS_B[3 * k + 1] + c2 * GS_B[3 * k + 2]);
    }
    res = res - 2.0 * PI * I1 * s1 - PI * mbar * I2 * s2 / C1;
    // --- association, one pair analytic (assoc.jl:702-769) ---
    if (P.has_assoc) {
        const int ic = P.aic, jc = P.ajc;
        T n2m = n0 * 0.0, n3m = n2m, vm = n2m;
        for (int i = 0; i < NC; ++i) {
            n2m = n2m + (PI * P.m[i] * P.d[i]) * n[i][1];
            n3m = n3m + P.m[i] * n[i][2];
            vm = vm - (2.0 * PI * P.m[i]) * n[i][3];
        }
        const T xim = 1.0 - vm * vm / (n2m * n2m);
        const double dij = P.d[ic] * P.d[jc] / (P.d[ic] + P.d[jc]);
        const T inv1n3 = 1.0 / (1.0 - n3m);
        const T ghs = inv1n3 + 0.5 * dij * xim * n2m * inv1n3 * inv1n3
                      + dij * dij * n2m * n2m * xim * inv1n3 * inv1n3 * inv1n3 / 18.0;
        const T delta = ghs * P.aK;
        auto comp = [&](int c, T& n0c, T& xic) {
            n0c = n[c][1] / P.d[c];
            const T n2c = (PI * P.d[c]) * n[c][1];
            const T v = (-2.0 * PI) * n[c][3];
            xic = 1.0 - v * v / (n2c * n2c);
        };
        T n0i, xii, n0j, xij;
        comp(ic, n0i, xii);
        comp(jc, n0j, xij);
        const T kia = n0i * xii * delta, kjb = n0j * xij * delta;
        const T b = 1.0 - kia + kjb;
        const T Xa = 2.0 / (b + dsqrt(b * b + 4.0 * kia));
        const T Xb = 1.0 / (1.0 + kia * Xa);
        res = res + n0i * xii * (dlog(Xa) - 0.5 * Xa + 0.5) + n0j * xij * (dlog(Xb) - 0.5 * Xb + 0.5);
    }
    return res;
}

// dPhi/dn for every (component, field) at one point, one forward pass with 7 NC tangents
template <int NC>
void phi_grad(const double (&n)[NC][7], const Params& P, double& f, double (&g)[NC][7])
{
    constexpr int K = 7 * NC;
    Dual<K> x[NC][7];
    for (int i = 0; i < NC; ++i)
        for (int a = 0; a < 7; ++a) {
            x[i][a] = mk<K>(n[i][a]);
            x[i][a].d[i * 7 + a] = 1.0;
        }
    const Dual<K> r = f_res<Dual<K>, NC>(x, P);
    f = r.v;
    for (int i = 0; i < NC; ++i)
        for (int a = 0; a < 7; ++a) g[i][a] = r.d[i * 7 + a];
}

// omega_hat closed forms (weighted_densities.jl:48-69,210-236) at reduced frequency w
double kernel_hat(int type, double w, double R)
{
    const double TP = 2.0 * PI, wb = std::fabs(w);
    if (type == 1) return (wb == 0.0) ? 2.0 * R / TP : 2.0 * std::sin(wb * R) / wb / TP;
    if (type == 2) {
        if (wb == 0.0) return 4.0 * PI * R * R * R / 3.0 / (TP * TP * TP);
        return 4.0 * PI / (wb * wb * wb) * (std::sin(wb * R) - R * wb * std::cos(wb * R)) / (TP * TP * TP);
    }
    if (wb == 0.0) return 4.0 * PI * R / (TP * TP * TP);   // vector kernel: coefficient of i
    return 4.0 * PI * w / (wb * wb * wb) * (std::sin(wb * R) - R * wb * std::cos(wb * R)) / (TP * TP * TP);
}

// ---------------------------------------------------------------------------
// one system
// ---------------------------------------------------------------------------
struct System {
    int N = 0, nc = 0;
    double NA = 0.0;
    Params P;
    double cprd[CDFT_MAX_NC];
    std::vector<cplx> K;        // [(i*6 + f)*N + k] sampled kernels
    std::vector<double> vext;   // [i*N + j] or empty
    Fft fft;
    std::vector<cplx> spec, buf, acc;
    std::vector<double> n, g;   // [(i*7 + a)*N + j]

    int build(const cdft_system_desc& d)
    {
        if (d.nd != 1 || d.coord != CDFT_COORD_CART || d.nc < 1 || d.nc > CDFT_MAX_NC || d.ngrid[0] < 2 ||
            d.n_assoc < 0 || d.n_assoc > 1)
            return CDFT_E_UNSUPPORTED;
        N = d.ngrid[0];
        nc = d.nc;
        const double L = d.L, T = d.T;
        NA = NAVO * L * L * L;
        P.nc = nc;
        P.T = T;
        for (int i = 0; i < nc; ++i) {
            P.m[i] = d.m[i];
            P.d[i] = d.hsd[i] / L;
            cprd[i] = d.mu_res_plus_ln_rhob[i];
        }
        for (int i = 0; i < nc; ++i)
            for (int j = 0; j < nc; ++j) {
                const double s = d.sigma[i * nc + j] / L;
                P.s3[i * CDFT_MAX_NC + j] = s * s * s;
                P.eT[i * CDFT_MAX_NC + j] = d.eps[i * nc + j] / T;
            }
        P.has_assoc = d.n_assoc;
        if (d.n_assoc) {
            const cdft_assoc_pair& a = d.assoc[0];
            P.aic = a.icomp;
            P.ajc = a.jcomp;
            const double s = d.sigma[a.icomp * nc + a.jcomp] / L;
            P.aK = s * s * s * (std::exp(a.eps_ab / T) - 1.0) * a.kappa_ab;
        }
        const int types[6] = {1, 2, 3, 2, 1, 2};
        const double wf[6] = {0.5, 0.5, 0.5, 1.0, 1.0, PSI};
        const double span = d.bounds[0][1] - d.bounds[0][0];
        K.assign((size_t)nc * 6 * N, 0.0);
        const int half = (N + 1) / 2;
        for (int i = 0; i < nc; ++i)
            for (int f = 0; f < 6; ++f) {
                const double R = 2.0 * PI * (wf[f] * P.d[i]);
                for (int k = 0; k < N; ++k) {
                    const int kk = (k < half) ? k : k - N;   // fftfreq order
                    const double w = (double)kk / span * L;
                    const double v = kernel_hat(types[f], w, R);
                    K[((size_t)i * 6 + f) * N + k] = (types[f] == 3) ? cplx(0.0, v) : cplx(v, 0.0);
                }
            }
        if (d.vext) vext.assign(d.vext, d.vext + (size_t)nc * N);
        fft.init(N);
        spec.assign(N, 0.0);
        buf.assign(N, 0.0);
        acc.assign(N, 0.0);
        n.assign((size_t)nc * 7 * N, 0.0);
        g.assign((size_t)nc * 7 * N, 0.0);
        return 0;
    }

    // delta F_res / delta rho + V_ext (delta F delta rho_res!, models.jl:131-186, + Steele)
    template <int NC>
    void dFdrho_nc(const double* rho, double* out)
    {
        const double invN = 1.0 / N;
        for (int i = 0; i < NC; ++i) {   // evaluate_field!
            for (int j = 0; j < N; ++j) {
                spec[j] = rho[(size_t)i * N + j];
                n[((size_t)i * 7) * N + j] = rho[(size_t)i * N + j] * NA;
            }
            fft.run(spec.data(), false);
            for (int f = 0; f < 6; ++f) {
                const cplx* k = K.data() + ((size_t)i * 6 + f) * N;
                for (int j = 0; j < N; ++j) buf[j] = spec[j] * k[j];
                fft.run(buf.data(), true);
                double* o = n.data() + ((size_t)i * 7 + f + 1) * N;
                for (int j = 0; j < N; ++j) o[j] = buf[j].real() * invN * NA;
            }
        }
        for (int j = 0; j < N; ++j) {   // AD stage
            double x[NC][7], gg[NC][7], fv;
            for (int i = 0; i < NC; ++i)
                for (int a = 0; a < 7; ++a) x[i][a] = n[((size_t)i * 7 + a) * N + j];
            phi_grad<NC>(x, P, fv, gg);
            for (int i = 0; i < NC; ++i)
                for (int a = 0; a < 7; ++a) g[((size_t)i * 7 + a) * N + j] = gg[i][a];
        }
        for (int i = 0; i < NC; ++i) {   // integrate_field!
            for (int j = 0; j < N; ++j) acc[j] = 0.0;
            for (int f = 0; f < 6; ++f) {
                const double* src = g.data() + ((size_t)i * 7 + f + 1) * N;
                for (int j = 0; j < N; ++j) buf[j] = src[j];
                fft.run(buf.data(), false);
                const cplx* k = K.data() + ((size_t)i * 6 + f) * N;
                const double sgn = (f == 2) ? -1.0 : 1.0;   // vector field: δfδρ .-= (weighted_densities.jl:381)
                for (int j = 0; j < N; ++j) acc[j] += sgn * buf[j] * k[j];
            }
            fft.run(acc.data(), true);
            for (int j = 0; j < N; ++j) {
                double v = g[((size_t)i * 7) * N + j] + acc[j].real() * invN;
                if (!vext.empty()) v += vext[(size_t)i * N + j];
                out[(size_t)i * N + j] = v;
            }
        }
    }

    void dFdrho(const double* rho, double* out)
    {
        switch (nc) {
        case 1: dFdrho_nc<1>(rho, out); break;
        case 2: dFdrho_nc<2>(rho, out); break;
        case 3: dFdrho_nc<3>(rho, out); break;
        default: dFdrho_nc<4>(rho, out); break;
        }
    }

    // GFix!: rho = exp(ln x); ln G = mu_res + ln rho_b - dF/drho, clamp!(+-100) (converge.jl:108-153,235-242)
    std::vector<double> rho_w, d_w;
    void gfix(const double* lnx, double* lnG)
    {
        const size_t ne = (size_t)nc * N;
        rho_w.resize(ne);
        d_w.resize(ne);
        for (size_t e = 0; e < ne; ++e) rho_w[e] = std::exp(lnx[e]);
        dFdrho(rho_w.data(), d_w.data());
        for (int i = 0; i < nc; ++i)
            for (int j = 0; j < N; ++j) {
                const size_t e = (size_t)i * N + j;
                double v = cprd[i] - d_w[e];
                v = (v > 100.0) ? 100.0 : ((v < -100.0) ? -100.0 : v);   // a NaN stays NaN
                lnG[e] = v;
            }
    }
};

// ---------------------------------------------------------------------------
// aasol (anderson.jl:301-443) for one system
// ---------------------------------------------------------------------------
double nrm2(const std::vector<double>& x)
{
    double s = 0.0;
    for (double v : x) s += v * v;
    return std::sqrt(s);
}

// thin Householder QR of the m x (m-1) matrix A (column-major, leading dimension m), LAPACK
// dlarfg signs: Q (m x (m-1)) and R ((m-1) x (m-1)) -- downdate_aaqr!, anderson.jl:552-583
void householder_qr(int m, int n, std::vector<double>& A, std::vector<double>& Q, std::vector<double>& R)
{
    std::vector<double> tau(n), V((size_t)m * n, 0.0);
    for (int j = 0; j < n; ++j) {
        const double alpha = A[j + (size_t)j * m];
        double xn = 0.0;
        for (int r = j + 1; r < m; ++r) xn += A[r + (size_t)j * m] * A[r + (size_t)j * m];
        xn = std::sqrt(xn);
        V[j + (size_t)j * m] = 1.0;
        if (xn == 0.0) {
            tau[j] = 0.0;
            continue;
        }
        const double beta = -std::copysign(std::hypot(alpha, xn), alpha);
        tau[j] = (beta - alpha) / beta;
        const double sc = 1.0 / (alpha - beta);
        for (int r = j + 1; r < m; ++r) V[r + (size_t)j * m] = A[r + (size_t)j * m] * sc;
        A[j + (size_t)j * m] = beta;
        for (int r = j + 1; r < m; ++r) A[r + (size_t)j * m] = 0.0;
        for (int c = j + 1; c < n; ++c) {
            double w = 0.0;
            for (int r = j; r < m; ++r) w += V[r + (size_t)j * m] * A[r + (size_t)c * m];
            for (int r = j; r < m; ++r) A[r + (size_t)c * m] -= tau[j] * V[r + (size_t)j * m] * w;
        }
    }
    R.assign((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c)
        for (int r = 0; r <= c; ++r) R[r + (size_t)c * n] = A[r + (size_t)c * m];
    Q.assign((size_t)m * n, 0.0);
    for (int c = 0; c < n; ++c) Q[c + (size_t)c * m] = 1.0;
    for (int j = n - 1; j >= 0; --j)
        for (int c = 0; c < n; ++c) {
            double w = 0.0;
            for (int r = j; r < m; ++r) w += V[r + (size_t)j * m] * Q[r + (size_t)c * m];
            for (int r = j; r < m; ++r) Q[r + (size_t)c * m] -= tau[j] * V[r + (size_t)j * m] * w;
        }
}

int aasol(System& S, std::vector<double>& sol, const cdft_solver_opts& o, cdft_result* res)
{
    const size_t n = sol.size();
    const int m = o.m;
    const double beta = o.beta;
    std::vector<double> gx(n), r(n), tmp(n);
    int evals = 0, k = 0;
    auto record = [&](double v) {
        if (res && res->history && evals < res->history_cap) res->history[evals] = v;
        ++evals;
    };
    auto betafix = [](std::vector<double>& g, const std::vector<double>& s, double b) {
        if (b != 1.0)
            for (size_t e = 0; e < g.size(); ++e) g[e] = (1.0 - b) * s[e] + b * g[e];
    };
    S.gfix(sol.data(), gx.data());
    betafix(gx, sol, beta);
    for (size_t e = 0; e < n; ++e) r[e] = gx[e] - sol[e];
    double resnorm = nrm2(r);
    record(resnorm);
    const double up_bd = 1.0e4 * resnorm;
    const double tol = o.rtol * resnorm + o.atol;
    const double picard_tol = o.picard_rtol * resnorm + o.picard_atol;
    bool toosoon = resnorm <= tol;
    if (!toosoon && o.picard_maxit > 0) {   // Picard warm-up (anderson.jl:345-364)
        sol = gx;
        for (int it = 0; it < o.picard_maxit - 1; ++it) {
            S.gfix(sol.data(), gx.data());
            betafix(gx, sol, o.picard_beta);
            for (size_t e = 0; e < n; ++e) r[e] = gx[e] - sol[e];
            resnorm = nrm2(r);
            record(resnorm);
            if (resnorm <= picard_tol || resnorm >= up_bd) break;
            sol = gx;
        }
        toosoon = resnorm <= tol;
    }
    const int mm = std::max(m, 1);
    std::vector<double> Q(n * mm, 0.0), DG(n * mm, 0.0), R((size_t)mm * mm, 0.0), dg(n), df(n);
    auto aa_point = [&]() {   // anderson.jl:470-481
        for (size_t e = 0; e < n; ++e) dg[e] = -gx[e];
        S.gfix(sol.data(), gx.data());
        betafix(gx, sol, beta);
        for (size_t e = 0; e < n; ++e) {
            dg[e] += gx[e];
            df[e] = -r[e];
            r[e] = gx[e] - sol[e];
            df[e] += r[e];
        }
        resnorm = nrm2(r);
        record(resnorm);
    };
    if (!toosoon) {
        sol = gx;
        ++k;
        aa_point();
    }
    std::vector<double> Qx, Rd, Rp, h1, h2, th, tres;
    while (k < o.maxit + o.picard_maxit && resnorm > tol && !toosoon && resnorm < up_bd) {
        if (m == 0) {
            sol = gx;
        } else {
            const int kk = k + 1;   // BuildDG!(DG, m, k+1, dg), anderson.jl:450-461
            if (m == 1) std::copy(dg.begin(), dg.end(), DG.begin());
            else if (kk > m + 1) {
                std::copy(DG.begin() + n, DG.begin() + n * m, DG.begin());
                std::copy(dg.begin(), dg.end(), DG.begin() + n * (m - 1));
            } else {
                std::copy(dg.begin(), dg.end(), DG.begin() + n * (kk - 2));
            }
            const int kq0 = k - 1;   // aa_qr_update!(Q, R, df, m, k-1), anderson.jl:498-512
            if (kq0 == 0) {
                const double nv = nrm2(df);
                R[0] = nv;
                for (size_t e = 0; e < n; ++e) Q[e] = df[e] / nv;
            } else {
                if (kq0 > m - 1) {   // downdate_aaqr!
                    Rp.assign((size_t)m * (m - 1), 0.0);
                    for (int c = 0; c < m - 1; ++c)
                        for (int rr = 0; rr < m; ++rr) Rp[rr + (size_t)c * m] = R[rr + (size_t)(c + 1) * m];
                    householder_qr(m, m - 1, Rp, Qx, Rd);
                    std::fill(R.begin(), R.end(), 0.0);
                    for (int c = 0; c < m - 1; ++c)
                        for (int rr = 0; rr < m - 1; ++rr) R[rr + (size_t)c * m] = Rd[rr + (size_t)c * (m - 1)];
                    std::vector<double> row(m);
                    for (size_t e = 0; e < n; ++e) {
                        for (int c = 0; c < m; ++c) row[c] = Q[e + n * c];
                        for (int c = 0; c < m - 1; ++c) {
                            double v = 0.0;
                            for (int rr = 0; rr < m; ++rr) v += row[rr] * Qx[rr + (size_t)c * m];
                            Q[e + n * c] = v;
                        }
                        Q[e + n * (m - 1)] = 0.0;
                    }
                }
                const int kq = std::min(kq0, m - 1);   // Orthogonalize! CGS2, anderson.jl:525-540
                h1.assign(kq, 0.0);
                h2.assign(kq, 0.0);
                for (int c = 0; c < kq; ++c) {
                    double s = 0.0;
                    for (size_t e = 0; e < n; ++e) s += Q[e + n * c] * df[e];
                    h1[c] = s;
                }
                for (int c = 0; c < kq; ++c)
                    for (size_t e = 0; e < n; ++e) df[e] += (-h1[c]) * Q[e + n * c];
                for (int c = 0; c < kq; ++c) {
                    double s = 0.0;
                    for (size_t e = 0; e < n; ++e) s += Q[e + n * c] * df[e];
                    h2[c] = s;
                }
                for (int c = 0; c < kq; ++c)
                    for (size_t e = 0; e < n; ++e) df[e] += (-h2[c]) * Q[e + n * c];
                for (int c = 0; c < kq; ++c) R[c + (size_t)kq * m] = h1[c] + h2[c];
                const double nv = nrm2(df);
                R[kq + (size_t)kq * m] = nv;
                for (size_t e = 0; e < n; ++e) Q[e + n * kq] = df[e] / nv;
            }
            const int mk = std::min(m, k);   // theta = R \ (Q' res), anderson.jl:405-416
            tres.assign(mk, 0.0);
            for (int c = 0; c < mk; ++c) {
                double s = 0.0;
                for (size_t e = 0; e < n; ++e) s += Q[e + n * c] * r[e];
                tres[c] = s;
            }
            th.assign(mk, 0.0);
            for (int i = mk - 1; i >= 0; --i) {
                double v = tres[i];
                for (int j = i + 1; j < mk; ++j) v -= R[i + (size_t)j * m] * th[j];
                th[i] = v / R[i + (size_t)i * m];
            }
            sol = gx;
            for (int c = 0; c < mk; ++c)
                for (size_t e = 0; e < n; ++e) sol[e] += (-th[c]) * DG[e + n * c];
        }
        ++k;
        aa_point();
    }
    int errcode;   // AndersonOK, anderson.jl:727-737
    if (toosoon) errcode = -1;
    else if (resnorm >= up_bd || !std::isfinite(resnorm)) errcode = -2;
    else if (resnorm <= tol) errcode = 0;
    else errcode = 10;
    if (res) {
        res->idid = (errcode == -1 || errcode == 0) ? 1 : 0;
        res->errcode = errcode;
        res->iterations = k;
        res->evaluations = evals;
        res->resnorm = resnorm;
        res->tol = tol;
        res->history_len = res->history ? std::min(evals, res->history_cap) : 0;
    }
    return 0;
}

}  // namespace

extern "C" {

// dF/drho (residual + external field) of one 1D system at rho (nc x N, grid fastest).
int cdft_cpu_functional_derivative(const cdft_system_desc* desc, const double* rho, double* out)
{
    if (!desc || !rho || !out) return CDFT_E_INVALID;
    System S;
    const int rc = S.build(*desc);
    if (rc) return rc;
    S.dFdrho(rho, out);
    return 0;
}

// converge! of n independent systems on `nthreads` OpenMP threads (<= 0: all), one system
// per thread at a time (dynamic schedule, largest first).  rho_inout[s] holds the initial
// profile on entry and exp(result.solution) on exit, as converge! returns it (converge.jl:246).
int cdft_cpu_batch_converge(const cdft_system_desc* descs, int n, double* const* rho_inout,
                            const cdft_solver_opts* opts, cdft_result* results, int nthreads)
{
    if (!descs || n <= 0 || !rho_inout || !opts) return CDFT_E_INVALID;
    if (opts->m < 0 || opts->m > CDFT_MAX_M || !(std::fabs(opts->beta) > 0 && std::fabs(opts->beta) <= 1))
        return CDFT_E_INVALID;
    std::vector<int> order(n);
    for (int s = 0; s < n; ++s) order[s] = s;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return descs[a].ngrid[0] * descs[a].nc > descs[b].ngrid[0] * descs[b].nc; });
    int err = 0;
    const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int t = 0; t < n; ++t) {
        const int s = order[t];
        System S;
        int rc = S.build(descs[s]);
        if (rc) {
#pragma omp atomic write
            err = rc;
            continue;
        }
        const size_t ne = (size_t)S.nc * S.N;
        std::vector<double> sol(ne);
        for (size_t e = 0; e < ne; ++e) sol[e] = std::log(rho_inout[s][e]);
        aasol(S, sol, *opts, results ? &results[s] : nullptr);
        for (size_t e = 0; e < ne; ++e) rho_inout[s][e] = std::exp(sol[e]);
    }
    return err;
}

int cdft_cpu_max_threads(void) { return omp_get_max_threads(); }

// 1: evaluate the reference's closed White-Bear bracket everywhere; 0: the series near n3 = 0
void cdft_cpu_set_wb_closed(int closed) { g_wb_closed = closed != 0; }

}  // extern "C"
