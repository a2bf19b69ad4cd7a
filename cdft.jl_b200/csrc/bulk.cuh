// Bulk PC-SAFT at fixed temperature and composition on the device: the density roots
// behind a system's bulk state (get_species / volume(model, p, T, x), PCSAFT.jl:65-72;
// adsorption(model, surface, p, T) builds one per state point, adsorption.jl:48-65).
//
// Residual Helmholtz energy per molecule (Gross & Sadowski, Ind. Eng. Chem. Res. 40 (2001)
// 1244; 2B self-association: Ind. Eng. Chem. Res. 41 (2002) 5510) in forward-mode dual
// numbers in the number density, so the compressibility Z = 1 + rho d(a_res)/d(rho) and the
// pressure p = rho k_B T Z come out exactly.  Roots of p(eta) = p_target as the host
// molar_density finds them: the sign changes of p - p_target on 40 log-spaced packing
// fractions in [1e-12, 10^-1.3] and 70 linear ones in [0.051, 0.74], the densest bracket
// for the liquid, the most dilute for the vapour, refined to 1e-15 relative (Illinois
// false position).  The stable phase is the root of lower Gibbs energy per molecule,
// a_res + Z + ln rho (the terms common to both roots dropped).
#pragma once

struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual dc(double v) { return Dual{v, 0.0}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return Dual{q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator*(double s, Dual a) { return Dual{s * a.v, s * a.d}; }
__device__ __forceinline__ Dual operator+(double s, Dual a) { return Dual{s + a.v, a.d}; }
__device__ __forceinline__ Dual operator-(double s, Dual a) { return Dual{s - a.v, -a.d}; }
__device__ __forceinline__ Dual operator+(Dual a, double s) { return Dual{a.v + s, a.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double s) { return Dual{a.v - s, a.d}; }
__device__ __forceinline__ Dual dlog(Dual a) { return Dual{log(a.v), a.d / a.v}; }
__device__ __forceinline__ Dual dsqrt(Dual a)
{
    const double r = sqrt(a.v);
    return Dual{r, 0.5 * a.d / r};
}

struct BulkModel {
    int nc;
    double T;
    double m[CDFT_MAX_NC], d[CDFT_MAX_NC];        // segments, hard-sphere diameters (m)
    double s3[CDFT_MAX_NC * CDFT_MAX_NC];         // sigma_ij^3 (m^3)
    double eT[CDFT_MAX_NC * CDFT_MAX_NC];         // eps_ij / T
    double aK[CDFT_MAX_NC];                       // 2B self-association: sigma_ii^3 kappa (exp(eps_AB/T) - 1), 0 = none
};

__constant__ double kBulkA[7][3] = {
    {0.9105631445, -0.3084016918, -0.0906148351}, {0.6361281449, 0.1860531159, 0.4527842806},
    {2.6861347891, -2.5030047259, 0.5962700728}, {-26.547362491, 21.419793629, -1.7241829131},
    {97.759208784, -65.25588533, -4.1302112531}, {-159.59154087, 83.318680481, 13.77663187},
    {91.297774084, -33.74692293, -8.6728470368}};
__constant__ double kBulkB[7][3] = {
    {0.7240946941, -0.5755498075, 0.0976883116}, {2.2382791861, 0.6995095521, -0.2557574982},
    {-4.0025849485, 3.892567339, -9.155856153}, {-21.003576815, -17.215471648, 20.642075974},
    {26.855641363, 192.67226447, -38.804430052}, {206.55133841, -161.82646165, 93.626774077},
    {-355.60235612, -165.20769346, -29.666905585}};

// a_res per molecule (k_B T) at number density rho (1/m^3) and mole fractions x, with its
// derivative in rho
__device__ Dual bulk_ares(const BulkModel& M, const double* x, Dual rho)
{
    const double PI = 3.14159265358979323846;
    const int nc = M.nc;
    Dual z[4];
    for (int k = 0; k < 4; ++k) {
        double c = 0.0;
        for (int i = 0; i < nc; ++i) {
            double dk = 1.0;
            for (int q = 0; q < k; ++q) dk *= M.d[i];
            c += x[i] * M.m[i] * dk;
        }
        z[k] = (PI / 6.0 * c) * rho;
    }
    const Dual e = z[3], ome = 1.0 - e;
    const Dual lno = dlog(ome);
    const Dual ahs = (3.0 * (z[1] * z[2] / ome) + z[2] * z[2] * z[2] / (e * ome * ome) +
                      (z[2] * z[2] * z[2] / (e * e) - z[0]) * lno) / z[0];
    auto gij = [&](double dd) {   // g_hs at contact, dd = d_i d_j / (d_i + d_j)
        return dc(1.0) / ome + (3.0 * dd) * (z[2] / (ome * ome)) + (2.0 * dd * dd) * (z[2] * z[2] / (ome * ome * ome));
    };
    double mb = 0.0;
    for (int i = 0; i < nc; ++i) mb += x[i] * M.m[i];
    Dual ahc = mb * ahs;
    for (int i = 0; i < nc; ++i)
        if (M.m[i] != 1.0) ahc = ahc - (x[i] * (M.m[i] - 1.0)) * dlog(gij(0.5 * M.d[i]));
    const double c1 = (mb - 1.0) / mb, c2 = (mb - 1.0) * (mb - 2.0) / (mb * mb);
    Dual I1 = dc(0.0), I2 = dc(0.0);
    for (int k = 6; k >= 0; --k) {
        I1 = I1 * e + dc(kBulkA[k][0] + c1 * kBulkA[k][1] + c2 * kBulkA[k][2]);
        I2 = I2 * e + dc(kBulkB[k][0] + c1 * kBulkB[k][1] + c2 * kBulkB[k][2]);
    }
    const Dual e2 = e * e;
    const Dual C1 = dc(1.0) / (1.0 + mb * (8.0 * e - 2.0 * e2) / (ome * ome * ome * ome) +
                           (1.0 - mb) * (20.0 * e - 27.0 * e2 + 12.0 * e2 * e - 2.0 * e2 * e2) /
                               ((ome * (2.0 - e)) * (ome * (2.0 - e))));
    double m2es3 = 0.0, m2e2s3 = 0.0;
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            const double t = x[i] * x[j] * M.m[i] * M.m[j] * M.s3[i * CDFT_MAX_NC + j];
            const double et = M.eT[i * CDFT_MAX_NC + j];
            m2es3 += t * et;
            m2e2s3 += t * et * et;
        }
    const Dual adisp = (-2.0 * PI * m2es3) * (rho * I1) - (PI * mb * m2e2s3) * (rho * C1 * I2);
    Dual aas = dc(0.0);
    for (int i = 0; i < nc; ++i)
        if (M.aK[i] != 0.0) {
            const Dual D = M.aK[i] * gij(0.5 * M.d[i]);
            const Dual q = (x[i] * D) * rho;
            const Dual X = dc(2.0) / (1.0 + dsqrt(1.0 + 4.0 * q));
            aas = aas + (2.0 * x[i]) * (dlog(X) - 0.5 * X + 0.5);
        }
    return ahc + adisp + aas;
}

// pressure (Pa) and Gibbs term a_res + Z + ln rho at number density rho
__device__ __forceinline__ double bulk_pressure(const BulkModel& M, const double* x, double rho, double* g = nullptr)
{
    const double kB = 1.380649e-23;
    const Dual a = bulk_ares(M, x, Dual{rho, 1.0});
    const double Z = 1.0 + rho * a.d;
    if (g) *g = a.v + Z + log(rho);
    return rho * kB * M.T * Z;
}

#define BULK_GRID 110
__device__ __forceinline__ double bulk_grid_eta(int k)
{
    if (k < 40) return pow(10.0, -12.0 + k * (10.7 / 39.0));   // numpy.logspace(-12, -1.3, 40)
    return 0.051 + (k - 40) * (0.689 / 69.0);                   // numpy.linspace(0.051, 0.74, 70)
}

// root of p(eta / scale) = p0 in the bracket [a, b] (f(a), f(b) of opposite signs)
__device__ double bulk_refine(const BulkModel& M, const double* x, double scale, double p0, double a, double b,
                              double fa, double fb)
{
    int side = 0;
    for (int it = 0; it < 400; ++it) {
        if (fabs(b - a) <= 1e-15 * fabs(b) + 1e-300) break;
        double c = (a * fb - b * fa) / (fb - fa);
        if (!(c > fmin(a, b) && c < fmax(a, b))) c = 0.5 * (a + b);
        const double fc = bulk_pressure(M, x, c / scale) - p0;
        if (fc == 0.0) return c;
        if ((fc > 0) == (fb > 0)) {
            b = c;
            fb = fc;
            if (side == -1) fa *= 0.5;   // Illinois: halve the retained end
            side = -1;
        } else {
            a = c;
            fa = fc;
            if (side == 1) fb *= 0.5;
            side = 1;
        }
    }
    return 0.5 * (a + b);
}

// one warp per state point: rho[s] (mol/m^3) of the requested phase; status[s] = 0 ok, 1 no root
__global__ void bulk_density_kernel(BulkModel M, int n, const double* __restrict__ p, const double* __restrict__ xin,
                                    int phase, double* __restrict__ rho_out, int* __restrict__ status)
{
    const double NAVO = 6.02214076e23;
    const int s = blockIdx.x;
    if (s >= n) return;
    const int lane = threadIdx.x;
    __shared__ double fgrid[BULK_GRID];
    double x[CDFT_MAX_NC];
    double sx = 0.0;
    for (int i = 0; i < M.nc; ++i) sx += xin[(size_t)s * M.nc + i];
    double scale = 0.0;
    for (int i = 0; i < M.nc; ++i) {
        x[i] = xin[(size_t)s * M.nc + i] / sx;
        scale += x[i] * M.m[i] * M.d[i] * M.d[i] * M.d[i];
    }
    const double PI = 3.14159265358979323846;
    scale *= PI / 6.0;   // eta per (molecule / m^3)
    const double p0 = p[s];
    for (int k = lane; k < BULK_GRID; k += 32) fgrid[k] = bulk_pressure(M, x, bulk_grid_eta(k) / scale) - p0;
    __syncwarp();
    if (lane != 0) return;
    auto sgn = [](double v) { return v > 0 ? 1 : (v < 0 ? -1 : 0); };
    int first = -1, last = -1;
    for (int k = 0; k + 1 < BULK_GRID; ++k)
        if (sgn(fgrid[k]) != sgn(fgrid[k + 1])) {
            if (first < 0) first = k;
            last = k;
        }
    if (first < 0) {
        rho_out[s] = __longlong_as_double(0x7ff8000000000000LL);
        status[s] = 1;
        return;
    }
    auto root = [&](int k) {
        const double e = bulk_refine(M, x, scale, p0, bulk_grid_eta(k), bulk_grid_eta(k + 1), fgrid[k], fgrid[k + 1]);
        return e / scale;   // molecules / m^3
    };
    double r;
    if (phase == 1) r = root(last);
    else if (phase == 2) r = root(first);
    else {
        const double rl = root(last), rv = root(first);
        if (fabs(rl / rv - 1.0) < 1e-10) r = rl;
        else {
            double gl, gv;
            bulk_pressure(M, x, rl, &gl);
            bulk_pressure(M, x, rv, &gv);
            r = (gl <= gv) ? rl : rv;
        }
    }
    rho_out[s] = r / NAVO;
    status[s] = 0;
}

// Pure-component vapour-liquid coexistence, one warp per temperature (models[s] holds the
// component at T_s).  Start as the host solver does: the densest root of p = p_start (the
// warp scans the packing-fraction grid of bulk_density_kernel, lane 0 refines it) and the ideal-gas vapour
// p_start / k_B T.  Then Newton on y = (ln rho_l, ln rho_v) for
//   F1 = rho_l Z_l - rho_v Z_v   (p_l - p_v over k_B T),   F2 = g_l - g_v   (mu_l - mu_v over k_B T).
// Gibbs-Duhem (d mu = dp / rho at fixed T) gives the Jacobian from P' = d(p / k_B T)/d rho
// alone: dF1/dy_l = rho_l P'_l, dF2/dy_l = P'_l (and minus the vapour's), so the step is
//   dy_l = (rho_v F2 - F1) / (P'_l (rho_v - rho_l)),   dy_v = (rho_l F2 - F1) / (P'_v (rho_v - rho_l)),
// halved until no component exceeds 0.5, at most 100 steps, converged when both are below
// 1e-13.  Outputs p_sat = p(rho_v) (Pa) and the densities in mol/m^3; status 0 ok, 1 no
// liquid root at p_start, 2 not converged, 3 the trivial solution rho_l = rho_v or a
// non-finite iterate.
__global__ void saturation_kernel(const BulkModel* __restrict__ models, int n, double p_start,
                                  double* __restrict__ p_out, double* __restrict__ rl_out,
                                  double* __restrict__ rv_out, int* __restrict__ status)
{
    const double NAVO = 6.02214076e23, kB = 1.380649e-23, PI = 3.14159265358979323846;
    const int s = blockIdx.x;
    if (s >= n) return;
    const int lane = threadIdx.x;
    const BulkModel& M = models[s];
    __shared__ double fgrid[BULK_GRID];
    const double x[1] = {1.0};
    const double scale = PI / 6.0 * M.m[0] * M.d[0] * M.d[0] * M.d[0];
    for (int k = lane; k < BULK_GRID; k += 32) fgrid[k] = bulk_pressure(M, x, bulk_grid_eta(k) / scale) - p_start;
    __syncwarp();
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    auto fail = [&](int code) {
        if (lane != 0) return;
        p_out[s] = nan;
        rl_out[s] = nan;
        rv_out[s] = nan;
        status[s] = code;
    };
    // lane 0 finds the densest sign change and refines the liquid root there
    int last = -1;
    double rl0 = 0.0;
    if (lane == 0) {
        auto sgn = [](double v) { return v > 0 ? 1 : (v < 0 ? -1 : 0); };
        for (int k = 0; k + 1 < BULK_GRID; ++k)
            if (sgn(fgrid[k]) != sgn(fgrid[k + 1])) last = k;
        if (last >= 0)
            rl0 = bulk_refine(M, x, scale, p_start, bulk_grid_eta(last), bulk_grid_eta(last + 1), fgrid[last],
                              fgrid[last + 1]) / scale;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    rl0 = __shfl_sync(0xffffffffu, rl0, 0);
    if (last < 0) return fail(1);
    // Newton on the whole warp: lanes 0-2 evaluate a_res (dual numbers: a and a') at rho_l,
    // rho_l + h, rho_l - h and lanes 3-5 at rho_v, rho_v + h, rho_v - h, h = 1e-5 rho (the other
    // lanes repeat one of them); every lane then forms the same step from the shuffled values:
    // Z = 1 + rho a', g = a + Z + ln rho, and P' = d(p / k_B T)/d rho = 1 + 2 rho a' + rho^2 a''
    // with a'' the central difference of a' (it only sets Newton's rate; the residuals are
    // exact), so the warp takes the same steps as one lane would
    const int ph = lane < 3 ? 0 : 1, kind = lane % 3;
    double yl = log(rl0), yv = log(p_start / (kB * M.T));
    bool conv = false;
    for (int it = 0; it < 100; ++it) {
        const double rl = exp(yl), rv = exp(yv);
        const double r = ph == 0 ? rl : rv;
        const double h = 1e-5 * r;
        const Dual a = bulk_ares(M, x, Dual{kind == 0 ? r : (kind == 1 ? r + h : r - h), 1.0});
        const double avl = __shfl_sync(0xffffffffu, a.v, 0), adl = __shfl_sync(0xffffffffu, a.d, 0);
        const double apl = __shfl_sync(0xffffffffu, a.d, 1), aml = __shfl_sync(0xffffffffu, a.d, 2);
        const double avv = __shfl_sync(0xffffffffu, a.v, 3), adv = __shfl_sync(0xffffffffu, a.d, 3);
        const double apv = __shfl_sync(0xffffffffu, a.d, 4), amv = __shfl_sync(0xffffffffu, a.d, 5);
        const double hl = 1e-5 * rl, hv = 1e-5 * rv;
        const double a2l = (apl - aml) / (2.0 * hl), a2v = (apv - amv) / (2.0 * hv);
        const double Zl = 1.0 + rl * adl, Zv = 1.0 + rv * adv;
        const double gl = avl + Zl + log(rl), gv = avv + Zv + log(rv);
        const double Pl = 1.0 + 2.0 * rl * adl + rl * rl * a2l, Pv = 1.0 + 2.0 * rv * adv + rv * rv * a2v;
        const double F1 = rl * Zl - rv * Zv, F2 = gl - gv;
        const double dl = (rv * F2 - F1) / (Pl * (rv - rl)), dv = (rl * F2 - F1) / (Pv * (rv - rl));
        if (!isfinite(dl) || !isfinite(dv)) return fail(3);
        double lam = 1.0;
        while (fmax(fabs(lam * dl), fabs(lam * dv)) > 0.5) lam *= 0.5;
        yl -= lam * dl;
        yv -= lam * dv;
        if (fmax(fabs(dl), fabs(dv)) < 1e-13) {
            conv = true;
            break;
        }
    }
    const double rl = exp(yl), rv = exp(yv);
    if (!conv) return fail(2);
    if (!(fabs(rl / rv - 1.0) > 1e-6)) return fail(3);
    if (lane != 0) return;
    p_out[s] = bulk_pressure(M, x, rv);   // the vapour side: Z_l ~ 1e-6 at low T makes p(rho_l) ill-conditioned
    rl_out[s] = rl / NAVO;
    rv_out[s] = rv / NAVO;
    status[s] = 0;
}
