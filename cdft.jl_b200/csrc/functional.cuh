// Fused pointwise PC-SAFT free-energy density Phi(n) and its gradient dPhi/dn.
//
// Restates f_res (src/models/DFT/SAFT/PCSAFT/PCSAFT.jl:110-117):
//   f_hs   White-Bear FMT            src/models/DFT/FMT.jl:17-46
//   f_hc   Sauer-Gross chain          PCSAFT.jl:123-144
//   f_disp weighted dispersion        PCSAFT.jl:150-211
//   f_assoc one-pair analytic Wertheim  src/models/DFT/assoc.jl:159-168,702-769
//   f_assoc with several pairs          assoc.jl:251-413,771-828 (solve), :830-960 (IFT gradient)
// The reference differentiates f_res with Enzyme (models.jl:355-411, NF*nc
// forward passes by default).  Here the gradient is a hand-written reverse
// sweep computed in the same pass as Phi: one evaluation per point gives all
// NF*nc partial derivatives.
//
// Field order (get_fields, PCSAFT.jl:47-62): 0 rho, 1 int rho dz (d/2),
// 2 int rho z^2 dz (d/2), 3..3+nd-1 vector int rho z dz (d/2), 3+nd
// int rho z^2 dz (d), 4+nd int rho dz (d), 5+nd int rho z^2 dz (psi d).
#pragma once
#include "cdft_internal.cuh"

__constant__ double c_pcsaft_a[21];   // Gross & Sadowski (2001) a_0i, a_1i, a_2i, i = 0..6
__constant__ double c_pcsaft_b[21];   // b_0i, b_1i, b_2i

#define PSI_DISP 1.3862   // PCSAFT.jl:53

template <typename T>
__device__ __forceinline__ T fabs_t(T x) { return x < T(0) ? -x : x; }

// log|x| evaluated in double (the near-close-packing log(1 - n3) and the
// association logs stay FP64 in the mixed mode).
__device__ __forceinline__ double logabs64(double x) { return log(fabs(x)); }

// White-Bear bracket B(n3) = [ln(1 - n3) / n3^2 + 1 / (n3 (1 - n3)^2)] / (12 pi) and
// dB/dn3 (FMT.jl:39-43 writes B in this closed form).  For small |n3| the two
// terms cancel from O(1/n3) to O(1) (from O(1/n3^3) in dB/dn3), which makes the
// closed form lose all digits where n3 passes through zero: the ringing of the
// sampled kernels next to hard solutes puts grid points there.  Below |n3| = 0.05
// the Taylor series 12 pi B = sum_j (j+1)(j+3)/(j+2) n3^j is used instead; 16
// terms reach the FP64 rounding level on that interval.
__device__ __forceinline__ void wb_bracket(double n3, double D, double Lg, double invD, double& B, double& dB)
{
    const double c12 = 12.0 * 3.14159265358979323846;
    if (fabs(n3) < 0.05) {
        double b = 16.0 * 18.0 / 17.0, db = 0.0;   // j = 15
#pragma unroll
        for (int j = 14; j >= 0; --j) {
            db = db * n3 + b;
            b = b * n3 + (j + 1.0) * (j + 3.0) / (j + 2.0);
        }
        B = b / c12;
        dB = db / c12;
        return;
    }
    B = Lg / (c12 * n3 * n3) + 1.0 / (c12 * n3 * D * D);
    dB = -invD / (c12 * n3 * n3) - 2.0 * Lg / (c12 * n3 * n3 * n3)
         - 1.0 / (c12 * n3 * n3 * D * D) + 2.0 / (c12 * n3 * D * D * D);
}

// Wertheim association with several pairs at one point (assoc.jl:771-828), FP64.
// Inputs: u_c = n0_c xi_c per component, I = 1/(1 - n3), the mixture n2 and xi of g_hs.
// X_s by _assoc_solve (:405-413): X0 = 0.9, 5 NS blended substitutions
// X_s <- (X_s + 1/(1 + C_s(X)))/2 (:251-285), then 5 NS Newton steps on F_s = X_s (1 + C_s) - 1,
// J_st = (1 + C_s) delta_st + X_s dC_s/dX_t, solved by Gaussian elimination without pivoting;
// a candidate outside (0, 1) falls back to the plain substitution (:294-385).  Returns
// f = sum_s u_c(s) n_s (ln X_s - X_s/2 + 1/2) and its gradient in (u, I, n2, xi): the
// implicit-function derivative at the final X (:830-960, reverse: J^T lambda = df/dX).
// Not inlined, so the plain functional keeps its own register allocation.
__device__ __noinline__ double assoc_general(const PhiParams& P, const double* u, double I, double n2m, double xim,
                                             double* gu, double& gI, double& gn2, double& gxi)
{
    const int ns = P.a_ns, np = P.has_assoc;
    double D[CDFT_MAX_ASSOC], ca[CDFT_MAX_ASSOC], cb[CDFT_MAX_ASSOC];
    for (int p = 0; p < np; ++p) {
        const double dij = P.g_dij[p];
        const double ghs = I + 0.5 * dij * xim * n2m * I * I + dij * dij * n2m * n2m * xim * (I * I * I) / 18.0;
        D[p] = ghs * P.g_K[p];
        ca[p] = P.g_njb[p] * u[P.g_sc[P.g_pb[p]]] * D[p];   // coefficient of X_pb in C_pa
        cb[p] = P.g_nia[p] * u[P.g_sc[P.g_pa[p]]] * D[p];   // coefficient of X_pa in C_pb
    }
    double X[CDFT_MAX_SITES], C[CDFT_MAX_SITES];
    for (int s = 0; s < ns; ++s) X[s] = 0.9;
    auto fill_C = [&]() {
        for (int s = 0; s < ns; ++s) C[s] = 0.0;
        for (int p = 0; p < np; ++p) {
            C[P.g_pa[p]] += ca[p] * X[P.g_pb[p]];
            C[P.g_pb[p]] += cb[p] * X[P.g_pa[p]];
        }
    };
    double J[CDFT_MAX_SITES][CDFT_MAX_SITES + 1];
    auto fill_J = [&]() {   // J | F
        for (int s = 0; s < ns; ++s) {
            for (int t = 0; t < ns; ++t) J[s][t] = (s == t) ? 1.0 + C[s] : 0.0;
            J[s][ns] = X[s] * (1.0 + C[s]) - 1.0;
        }
        for (int p = 0; p < np; ++p) {
            J[P.g_pa[p]][P.g_pb[p]] += X[P.g_pa[p]] * ca[p];
            J[P.g_pb[p]][P.g_pa[p]] += X[P.g_pb[p]] * cb[p];
        }
    };
    for (int it = 0; it < 5 * ns; ++it) {
        fill_C();
        for (int s = 0; s < ns; ++s) X[s] = 0.5 * (X[s] + 1.0 / (1.0 + C[s]));
    }
    double dX[CDFT_MAX_SITES];
    for (int it = 0; it < 5 * ns; ++it) {
        fill_C();
        fill_J();
        for (int k = 0; k < ns; ++k)
            for (int i = k + 1; i < ns; ++i) {
                const double f = J[i][k] / J[k][k];
                for (int j = k + 1; j <= ns; ++j) J[i][j] -= f * J[k][j];
            }
        for (int k = ns - 1; k >= 0; --k) {
            double r = J[k][ns];
            for (int j = k + 1; j < ns; ++j) r -= J[k][j] * dX[j];
            dX[k] = r / J[k][k];
        }
        for (int s = 0; s < ns; ++s) {
            const double cand = X[s] - dX[s];
            X[s] = (cand > 0.0 && cand < 1.0) ? cand : 1.0 / (1.0 + C[s]);
        }
    }
    // value and the adjoint at the final X
    fill_C();
    fill_J();
    double f = 0.0, lam[CDFT_MAX_SITES];
    for (int c = 0; c < CDFT_MAX_NC; ++c) gu[c] = 0.0;
    for (int s = 0; s < ns; ++s) {
        const double h = logabs64(X[s]) - 0.5 * X[s] + 0.5;
        const double us = u[P.g_sc[s]];
        f += us * P.g_sm[s] * h;
        gu[P.g_sc[s]] += P.g_sm[s] * h;
        lam[s] = us * P.g_sm[s] * (1.0 / X[s] - 0.5);   // df/dX_s, overwritten by lambda
    }
    // J^T lambda = df/dX: elimination on the transpose, no pivoting
    double A[CDFT_MAX_SITES][CDFT_MAX_SITES];
    for (int s = 0; s < ns; ++s)
        for (int t = 0; t < ns; ++t) A[s][t] = J[t][s];
    for (int k = 0; k < ns; ++k)
        for (int i = k + 1; i < ns; ++i) {
            const double q = A[i][k] / A[k][k];
            for (int j = k + 1; j < ns; ++j) A[i][j] -= q * A[k][j];
            lam[i] -= q * lam[k];
        }
    for (int k = ns - 1; k >= 0; --k) {
        double r = lam[k];
        for (int j = k + 1; j < ns; ++j) r -= A[k][j] * lam[j];
        lam[k] = r / A[k][k];
    }
    // df/dtheta = explicit - lambda^T dF/dtheta, theta = (u_c, D_p)
    gI = gn2 = gxi = 0.0;
    for (int p = 0; p < np; ++p) {
        const int sa = P.g_pa[p], sb = P.g_pb[p];
        const int ca_c = P.g_sc[sb], cb_c = P.g_sc[sa];
        // F_sa gets X_sa * ca[p] * X_sb, F_sb gets X_sb * cb[p] * X_sa
        const double wa = lam[sa] * X[sa] * X[sb], wb = lam[sb] * X[sb] * X[sa];
        gu[ca_c] -= wa * P.g_njb[p] * D[p];
        gu[cb_c] -= wb * P.g_nia[p] * D[p];
        const double gD = -(wa * P.g_njb[p] * u[ca_c] + wb * P.g_nia[p] * u[cb_c]);
        const double gg = gD * P.g_K[p], dij = P.g_dij[p];
        gI += gg * (1.0 + dij * xim * n2m * I + dij * dij * n2m * n2m * xim * I * I / 6.0);
        gn2 += gg * (0.5 * dij * xim * I * I + dij * dij * n2m * xim * I * I * I / 9.0);
        gxi += gg * (0.5 * dij * n2m * I * I + dij * dij * n2m * n2m * I * I * I / 18.0);
    }
    return f;
}

// Layout of the parameter gradient of Phi (phi_grad with PG = true): the entries of
// PhiParams the functional depends on, m_i, d_i, c1_ij, c2_ij, the association d_ij and K.
template <int NC> struct PhiParamIdx {
    static constexpr int M = 0, D = NC, C1 = 2 * NC, C2 = 2 * NC + NC * NC, ADIJ = 2 * NC + 2 * NC * NC,
                         AK = ADIJ + 1, NP = AK + 1;
};

// Phi and dPhi/dn at one point (reverse sweep).  PG = true also accumulates
// dPhi/dP into gp[PhiParamIdx<NC>::NP] (same sweep, FP64): the explicit parameter
// dependence used by the parameter gradient of F_res; PG = false compiles to the
// plain evaluation.
// PART selects the terms: 0 all; 1 hard sphere + association (they read and write the
// n2, n3 and vector fields only); 2 chain + dispersion (rho, chain, lambda, dispersion
// fields only).  The two parts of one point can run on two threads, in place.
template <typename T, int NC, int ND, bool PG = false, int PART = 0>
__device__ __forceinline__ T phi_grad(const PhiParams& P, const T (&n)[NC][6 + ND], T (&g)[NC][6 + ND],
                                      double* gp = nullptr)
{
    using PI_ = PhiParamIdx<NC>;
    if constexpr (PG) {
        for (int q = 0; q < PI_::NP; ++q) gp[q] = 0.0;
    }
    constexpr int NF = 6 + ND;
    constexpr int F2 = 1, F3 = 2, FV = 3, IHC = 3 + ND, ILAM = 4 + ND, IDISP = 5 + ND;
    const T pi = T(3.14159265358979323846);
    const T two_pi = T(2.0) * pi;
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int a = 0; a < NF; ++a) g[i][a] = T(0);

    T phi = T(0);
    if constexpr (PART != 2) {
    // ---------------- hard sphere (FMT.jl:17-46) ----------------
    T n0 = 0, n1 = 0, n2 = 0, n3 = 0;
    T nv1[ND], nv2[ND];
#pragma unroll
    for (int k = 0; k < ND; ++k) { nv1[k] = 0; nv2[k] = 0; }
#pragma unroll
    for (int i = 0; i < NC; ++i) {
        const T mi = T(P.m[i]), di = T(P.d[i]);
        const T nim = n[i][F2] * mi;
        n0 += nim / di;
        n1 += T(0.5) * nim;
        n2 += pi * nim * di;
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            const T nvi = n[i][FV + k];
            nv1[k] += nvi * mi / di;
            nv2[k] -= two_pi * nvi * mi;
        }
        n3 += n[i][F3] * mi;
    }
    T nv1v2 = 0, nv2sq = 0;
#pragma unroll
    for (int k = 0; k < ND; ++k) { nv1v2 += nv1[k] * nv2[k]; nv2sq += nv2[k] * nv2[k]; }
    // log(1 - n3) and the White-Bear bracket in FP64
    const double n3d = double(n3);
    const double Dd = 1.0 - n3d;
    const double Lg = logabs64(Dd);
    const double invD = 1.0 / Dd;
    double Bd, dBd;
    wb_bracket(n3d, Dd, Lg, invD, Bd, dBd);
    const T A3 = n2 * n2 * n2 / T(3) - n2 * nv2sq;
    const T A2 = n1 * n2 - nv1v2;
    phi = T(-double(n0) * Lg) + A2 * T(invD) + A3 * T(Bd);
    {
        const T g_n0 = T(-Lg);
        const T g_n1 = n2 * T(invD);
        const T g_n2 = n1 * T(invD) + (n2 * n2 - nv2sq) * T(Bd);
        const T g_n3 = T(double(n0) * invD + double(A2) * invD * invD + double(A3) * dBd);
        T g_nv1[ND], g_nv2[ND];
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            g_nv1[k] = -nv2[k] * T(invD);
            g_nv2[k] = -nv1[k] * T(invD) - T(2) * n2 * nv2[k] * T(Bd);
        }
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            const T mi = T(P.m[i]), di = T(P.d[i]);
            g[i][F2] += mi * (g_n0 / di + T(0.5) * g_n1 + pi * di * g_n2);
            g[i][F3] += mi * g_n3;
#pragma unroll
            for (int k = 0; k < ND; ++k) g[i][FV + k] += mi * (g_nv1[k] / di - two_pi * g_nv2[k]);
        }
        if constexpr (PG) {
            // n0, n1, n2, nv1, nv2, n3 are linear in m_i; n0, n2, nv1 carry d_i
#pragma unroll
            for (int i = 0; i < NC; ++i) {
                const double mi = P.m[i], di = P.d[i];
                const double f2 = double(n[i][F2]), f3 = double(n[i][F3]);
                double gm = double(g_n0) * f2 / di + 0.5 * double(g_n1) * f2 + 3.14159265358979323846 * double(g_n2) * f2 * di
                            + double(g_n3) * f3;
                double gd = -double(g_n0) * f2 * mi / (di * di) + 3.14159265358979323846 * double(g_n2) * f2 * mi;
#pragma unroll
                for (int k = 0; k < ND; ++k) {
                    const double nvi = double(n[i][FV + k]);
                    gm += double(g_nv1[k]) * nvi / di - 2.0 * 3.14159265358979323846 * double(g_nv2[k]) * nvi;
                    gd -= double(g_nv1[k]) * nvi * mi / (di * di);
                }
                gp[PI_::M + i] += gm;
                gp[PI_::D + i] += gd;
            }
        }
    }

    }   // hard sphere

    if constexpr (PART != 1) {
    // ---------------- hard chain (PCSAFT.jl:123-144) ----------------
    {
        T z3 = 0, z2 = 0;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            z3 += T(P.m[i]) * n[i][IHC];
            z2 += T(P.m[i]) * n[i][IHC] / T(P.d[i]);
        }
        z3 /= T(8);
        z2 /= T(8);
        const T I = T(1) / (T(1) - z3);
        const T I2 = I * I, I3 = I2 * I, I4 = I3 * I;
        T gz3 = 0, gz2 = 0;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            const T am1 = T(P.m[i]) - T(1);
            if (am1 == T(0)) {   // exact zero contribution (m_i = 1); its m_i-derivative is not zero
                if constexpr (PG) {
                    const double di = P.d[i];
                    const double lam = double(n[i][ILAM]) / (2.0 * di);
                    const double y = double(I) + 1.5 * di * double(z2) * double(I2)
                                     + 0.5 * di * di * double(z2) * double(z2) * double(I3);
                    gp[PI_::M + i] += -double(n[i][0]) * log(fabs(y * lam / double(n[i][0])));
                }
                continue;
            }
            const T rho = n[i][0];
            // exact zeros (rho inside a hard wall, lambda as rounded FP32 FFT noise) make
            // rho ln(y lambda / rho) 0/0 or 0 * inf: the point contributes nothing
            if (rho == T(0) || n[i][ILAM] == T(0)) continue;
            const T di = T(P.d[i]);
            const T lam = n[i][ILAM] / (T(2) * di);
            const T y = I + T(1.5) * di * z2 * I2 + T(0.5) * di * di * z2 * z2 * I3;
            const T lg = T(log(fabs(double(y * lam / rho))));
            phi -= rho * am1 * lg;
            g[i][0] += -am1 * (lg - T(1));
            g[i][ILAM] += -rho * am1 / n[i][ILAM];
            const T gy = -rho * am1 / y;
            gz3 += gy * (I2 + T(3) * di * z2 * I3 + T(1.5) * di * di * z2 * z2 * I4);
            gz2 += gy * (T(1.5) * di * I2 + di * di * z2 * I3);
            if constexpr (PG) {
                // (m_i - 1) factor; explicit d_i in y and in lambda = n / (2 d_i)
                gp[PI_::M + i] += -double(rho) * double(lg);
                gp[PI_::D + i] += double(gy) * (1.5 * double(z2) * double(I2) + double(di) * double(z2) * double(z2) * double(I3))
                                  + double(rho) * double(am1) / double(di);
            }
        }
#pragma unroll
        for (int i = 0; i < NC; ++i) g[i][IHC] += T(P.m[i]) / T(8) * (gz3 + gz2 / T(P.d[i]));
        if constexpr (PG) {
            // z3 = sum m_i n_i / 8, z2 = sum m_i n_i / (8 d_i)
#pragma unroll
            for (int i = 0; i < NC; ++i) {
                const double nh = double(n[i][IHC]), di = P.d[i];
                gp[PI_::M + i] += double(gz3) * nh / 8.0 + double(gz2) * nh / (8.0 * di);
                gp[PI_::D + i] += -double(gz2) * P.m[i] * nh / (8.0 * di * di);
            }
        }
    }

    // ---------------- dispersion (PCSAFT.jl:150-211) ----------------
    {
        const T psi = T(PSI_DISP);
        const T factor = T(3) / (T(4) * psi * psi * psi * pi);
        T r[NC];
        T S = 0, M = 0, eta = 0;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            const T di = T(P.d[i]);
            const T d3 = di * di * di;
            r[i] = n[i][IDISP] * factor / d3;
            S += r[i];
            M += r[i] * T(P.m[i]);
            eta += T(P.m[i]) * r[i] * d3;
        }
        // mbar = sum r_i m_i / sum r_i (PCSAFT.jl:165-170).  One component: mbar = m
        // exactly, with no division.  Where a mixture's dispersion density is exactly zero
        // (FP32 FFT noise inside a hard solute rounds to 0.0 at some points) the ratio is
        // 0/0 while the term and its gradient vanish with r: any finite mbar serves there
        // and the composition derivatives are dropped.
        const bool S0 = (NC > 1) && (S == T(0));
        T mbar;
        if constexpr (NC == 1) mbar = T(P.m[0]);
        else mbar = S0 ? T(P.m[0]) : M / S;
        eta = eta * pi / T(6);
        T s1 = 0, s2 = 0;
        T rc1[NC], rc2[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            rc1[i] = 0; rc2[i] = 0;
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                rc1[i] += r[j] * T(P.c1[i * CDFT_MAX_NC + j]);
                rc2[i] += r[j] * T(P.c2[i * CDFT_MAX_NC + j]);
            }
            s1 += r[i] * rc1[i];
            s2 += r[i] * rc2[i];
        }
        const T e2 = eta * eta;
        const T om = T(1) - eta;
        const T om2 = om * om;
        const T om4 = om2 * om2;
        const T iv1 = T(1) / om;
        const T iv2 = T(1) / (T(2) - eta);
        const T Pp = (T(8) * eta - T(2) * e2) / om4;
        const T Qn = T(20) * eta - T(27) * e2 + T(12) * (eta * e2) - T(2) * (e2 * e2);
        const T Qq = Qn * iv1 * iv1 * iv2 * iv2;
        const T C1 = T(1) + mbar * Pp + (T(1) - mbar) * Qq;
        const T c1m = (mbar - T(1)) / mbar;
        const T c2m = c1m * (mbar - T(2)) / mbar;
        const T dc1 = T(1) / (mbar * mbar);
        const T dc2 = (T(3) * mbar - T(4)) / (mbar * mbar * mbar);
        // Horner for I1, I2 and their derivatives in eta and mbar
        T I1 = 0, I2 = 0, dI1e = 0, dI2e = 0, dI1m = 0, dI2m = 0;
#pragma unroll
        for (int k = 6; k >= 0; --k) {
            const T a = T(c_pcsaft_a[3 * k]) + c1m * T(c_pcsaft_a[3 * k + 1]) + c2m * T(c_pcsaft_a[3 * k + 2]);
            const T b = T(c_pcsaft_b[3 * k]) + c1m * T(c_pcsaft_b[3 * k + 1]) + c2m * T(c_pcsaft_b[3 * k + 2]);
            const T am = dc1 * T(c_pcsaft_a[3 * k + 1]) + dc2 * T(c_pcsaft_a[3 * k + 2]);
            const T bm = dc1 * T(c_pcsaft_b[3 * k + 1]) + dc2 * T(c_pcsaft_b[3 * k + 2]);
            dI1e = dI1e * eta + I1;
            dI2e = dI2e * eta + I2;
            I1 = I1 * eta + a;
            I2 = I2 * eta + b;
            dI1m = dI1m * eta + am;
            dI2m = dI2m * eta + bm;
        }
        phi += -T(2) * (pi * I1 * s1) - pi * mbar * I2 * s2 / C1;
        const T g_s1 = -T(2) * pi * I1;
        const T g_s2 = -pi * mbar * I2 / C1;
        const T g_I1 = -T(2) * pi * s1;
        const T g_I2 = -pi * mbar * s2 / C1;
        const T g_C1 = pi * mbar * I2 * s2 / (C1 * C1);
        const T dP = (T(8) - T(4) * eta) / om4 + T(4) * (T(8) * eta - T(2) * e2) / (om4 * om);
        const T dQn = T(20) - T(54) * eta + T(36) * e2 - T(8) * eta * e2;
        const T Qd = om2 * (T(2) - eta) * (T(2) - eta);
        const T dQd = -T(2) * om * (T(2) - eta) * (T(3) - T(2) * eta);
        const T dQ = (dQn * Qd - Qn * dQd) / (Qd * Qd);
        const T g_m = -pi * I2 * s2 / C1 + g_C1 * (Pp - Qq) + g_I1 * dI1m + g_I2 * dI2m;
        const T g_e = g_C1 * (mbar * dP + (T(1) - mbar) * dQ) + g_I1 * dI1e + g_I2 * dI2e;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            const T di = T(P.d[i]);
            const T d3 = di * di * di;
            const T gm_i = (NC == 1 || S0) ? T(0) : g_m * (T(P.m[i]) - mbar) / S;
            const T gr = gm_i + g_e * pi / T(6) * T(P.m[i]) * d3
                         + g_s1 * T(2) * rc1[i] + g_s2 * T(2) * rc2[i];
            g[i][IDISP] += gr * factor / d3;
            if constexpr (PG) {
                // r_i = n_i factor / d_i^3; mbar = M / S; eta = pi/6 sum m_i r_i d_i^3 (explicit d_i^3)
                const double ri = double(r[i]);
                const double dmbar = (NC == 1) ? 1.0 : (S0 ? 0.0 : ri / double(S));   // d mbar / d m_i
                gp[PI_::M + i] += double(g_m) * dmbar + double(g_e) * 3.14159265358979323846 / 6.0 * ri * double(d3);
                gp[PI_::D + i] += double(gr) * (-3.0 * ri / double(di))
                                  + double(g_e) * 3.14159265358979323846 / 2.0 * P.m[i] * ri * double(di) * double(di);
#pragma unroll
                for (int j = 0; j < NC; ++j) {
                    gp[PI_::C1 + i * NC + j] += double(g_s1) * ri * double(r[j]);
                    gp[PI_::C2 + i * NC + j] += double(g_s2) * ri * double(r[j]);
                }
            }
        }
    }

    }   // chain and dispersion

    // ---------------- association, one pair (assoc.jl:702-769), FP64 ----------------
    if (PART != 2 && P.has_assoc == 1) {
        const double PI = 3.14159265358979323846, TWO_PI = 2.0 * PI;
        double n2m = 0, n3m = 0, nv2m[ND];
#pragma unroll
        for (int k = 0; k < ND; ++k) nv2m[k] = 0;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            n2m += PI * double(n[i][F2]) * P.m[i] * P.d[i];
            n3m += double(n[i][F3]) * P.m[i];
#pragma unroll
            for (int k = 0; k < ND; ++k) nv2m[k] -= TWO_PI * double(n[i][FV + k]) * P.m[i];
        }
        // xi = 1 - |nv2|^2 / n2^2 (assoc.jl:734) is 0/0 where n2 is exactly zero (in the
        // mixed mode the weighted densities are FP32 FFT output, which rounds to 0.0 inside
        // hard walls at some points); there u = n0 xi and every xi term vanish with n2, so
        // xi = 1 and the vector fields drop out.
        if (n2m == 0.0) {
#pragma unroll
            for (int k = 0; k < ND; ++k) nv2m[k] = 0.0;
        }
        const double d2m = (n2m == 0.0) ? 1.0 : n2m;
        double nv2sqm = 0;
#pragma unroll
        for (int k = 0; k < ND; ++k) nv2sqm += nv2m[k] * nv2m[k];
        const double xim = 1.0 - nv2sqm / (d2m * d2m);
        const double dij = P.a_dij;
        const double I = 1.0 / (1.0 - n3m);
        const double ghs = I + 0.5 * dij * xim * n2m * I * I + dij * dij * n2m * n2m * xim * (I * I * I) / 18.0;
        const double Delta = ghs * P.a_K;
        const int ic = P.a_ic, jc = P.a_jc;
        double n0c[2], n2c[2], sqc[2], xic[2], uc[2];
        bool zc[2];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int c = s == 0 ? ic : jc;
            double nc_f2 = 0, vv[ND];
#pragma unroll
            for (int i = 0; i < NC; ++i)
                if (i == c) {
                    nc_f2 = double(n[i][F2]);
#pragma unroll
                    for (int k = 0; k < ND; ++k) vv[k] = double(n[i][FV + k]);
                }
            n0c[s] = nc_f2 / P.d[c];
            n2c[s] = PI * nc_f2 * P.d[c];
            zc[s] = (n2c[s] == 0.0);   // as above: xi_c = 1 where n2_c is exactly zero
            double sq = 0;
#pragma unroll
            for (int k = 0; k < ND; ++k) { const double t = -TWO_PI * vv[k]; sq += t * t; }
            sqc[s] = zc[s] ? 0.0 : sq;
            if (zc[s]) n2c[s] = 1.0;   // denominator only: n0_c = 0 carries the zero
            xic[s] = 1.0 - sqc[s] / (n2c[s] * n2c[s]);
            uc[s] = n0c[s] * xic[s];
        }
        const double nia = P.a_nia, njb = P.a_njb;
        const double kia = nia * uc[0] * Delta;
        const double kjb = njb * uc[1] * Delta;
        const double b = 1.0 - kia + kjb;
        const double sr = sqrt(b * b + 4.0 * kia);
        const double Xa = 2.0 / (b + sr);
        const double Xb = 1.0 / (1.0 + kia * Xa);
        const double phA = logabs64(Xa) - 0.5 * Xa + 0.5;
        const double phB = logabs64(Xb) - 0.5 * Xb + 0.5;
        phi += T(uc[0] * nia * phA + uc[1] * njb * phB);
        // reverse sweep
        const double gXa = nia * uc[0] * (1.0 / Xa - 0.5);
        const double gXb = njb * uc[1] * (1.0 / Xb - 0.5);
        const double bs2 = (b + sr) * (b + sr);
        const double dXa_db = -2.0 / bs2 * (1.0 + b / sr);
        const double dXa_dks = -4.0 / (bs2 * sr);
        const double dXa_dkia = -dXa_db + dXa_dks;
        const double dXa_dkjb = dXa_db;
        const double dXb_dkia = -Xb * Xb * (Xa + kia * dXa_dkia);
        const double dXb_dkjb = -Xb * Xb * kia * dXa_dkjb;
        const double gkia = gXa * dXa_dkia + gXb * dXb_dkia;
        const double gkjb = gXa * dXa_dkjb + gXb * dXb_dkjb;
        const double gu[2] = {nia * phA + gkia * nia * Delta, njb * phB + gkjb * njb * Delta};
        const double gDelta = gkia * nia * uc[0] + gkjb * njb * uc[1];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int c = s == 0 ? ic : jc;
            const double g_n0 = gu[s] * xic[s];
            const double g_xi = gu[s] * n0c[s];
            const double g_n2 = g_xi * 2.0 * sqc[s] / (n2c[s] * n2c[s] * n2c[s]);
#pragma unroll
            for (int i = 0; i < NC; ++i)
                if (i == c) {
                    g[i][F2] += T(g_n0 / P.d[c] + g_n2 * PI * P.d[c]);
#pragma unroll
                    for (int k = 0; k < ND; ++k)
                        if (!zc[s]) g[i][FV + k] += T(g_xi * (-2.0 * TWO_PI * TWO_PI * double(n[i][FV + k]) / (n2c[s] * n2c[s])));
                }
        }
        const double gg = gDelta * P.a_K;
        const double dg_dI = 1.0 + dij * xim * n2m * I + dij * dij * n2m * n2m * xim * I * I / 6.0;
        const double dg_dn2 = 0.5 * dij * xim * I * I + dij * dij * n2m * xim * I * I * I / 9.0;
        const double dg_dxi = 0.5 * dij * n2m * I * I + dij * dij * n2m * n2m * I * I * I / 18.0;
        const double g_n2m = gg * (dg_dn2 + dg_dxi * 2.0 * nv2sqm / (d2m * d2m * d2m));
        const double g_n3m = gg * dg_dI * I * I;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            g[i][F2] += T(g_n2m * PI * P.m[i] * P.d[i]);
            g[i][F3] += T(g_n3m * P.m[i]);
#pragma unroll
            for (int k = 0; k < ND; ++k)
                g[i][FV + k] += T(gg * dg_dxi * (-2.0 * nv2m[k] / (d2m * d2m)) * (-TWO_PI * P.m[i]));
        }
        if constexpr (PG) {
            gp[PI_::AK] += gDelta * ghs;
            gp[PI_::ADIJ] += gg * (0.5 * xim * n2m * I * I + dij * n2m * n2m * xim * I * I * I / 9.0);
#pragma unroll
            for (int i = 0; i < NC; ++i) {
                const double f2 = double(n[i][F2]);
                double gm = g_n2m * PI * f2 * P.d[i] + g_n3m * double(n[i][F3]);
#pragma unroll
                for (int k = 0; k < ND; ++k)
                    gm += gg * dg_dxi * (-2.0 * nv2m[k] / (d2m * d2m)) * (-TWO_PI * double(n[i][FV + k]));
                gp[PI_::M + i] += gm;
                gp[PI_::D + i] += g_n2m * PI * f2 * P.m[i];
            }
#pragma unroll
            for (int s = 0; s < 2; ++s) {   // u_c = n0_c xi_c with n0_c = n_F2 / d_c, n2_c = pi n_F2 d_c
                const int c = s == 0 ? ic : jc;
                const double dc = P.d[c];
                const double du = xic[s] * (-n0c[s] / dc) + n0c[s] * (2.0 * sqc[s] / (n2c[s] * n2c[s] * n2c[s])) * (n2c[s] / dc);
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    if (i == c) gp[PI_::D + i] += gu[s] * du;
            }
        }
    }
    // ---------------- association, several pairs (assoc.jl:771-828), FP64 ----------------
    // Compiled for mixtures only (plans with one component and several pairs are refused):
    // the call keeps its own registers, but the caller must save its live values around it,
    // which would cost the one-component kernels spills they do not need.
    if constexpr (NC >= 2) if (PART != 2 && P.has_assoc > 1) {
        const double PI = 3.14159265358979323846, TWO_PI = 2.0 * PI;
        double n2m = 0, n3m = 0, nv2m[ND];
#pragma unroll
        for (int k = 0; k < ND; ++k) nv2m[k] = 0;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            n2m += PI * double(n[i][F2]) * P.m[i] * P.d[i];
            n3m += double(n[i][F3]) * P.m[i];
#pragma unroll
            for (int k = 0; k < ND; ++k) nv2m[k] -= TWO_PI * double(n[i][FV + k]) * P.m[i];
        }
        if (n2m == 0.0) {   // exact zero (FP32 weighted densities): xi = 1, as in the one-pair path
#pragma unroll
            for (int k = 0; k < ND; ++k) nv2m[k] = 0.0;
        }
        const double d2m = (n2m == 0.0) ? 1.0 : n2m;
        double nv2sqm = 0;
#pragma unroll
        for (int k = 0; k < ND; ++k) nv2sqm += nv2m[k] * nv2m[k];
        const double xim = 1.0 - nv2sqm / (d2m * d2m);
        const double I = 1.0 / (1.0 - n3m);
        double u[CDFT_MAX_NC], n0c[NC], n2c[NC], sqc[NC], xic[NC];
        bool zc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const double f2 = double(n[c][F2]);
            n0c[c] = f2 / P.d[c];
            n2c[c] = PI * f2 * P.d[c];
            zc[c] = (n2c[c] == 0.0);
            double sq = 0;
#pragma unroll
            for (int k = 0; k < ND; ++k) { const double t = -TWO_PI * double(n[c][FV + k]); sq += t * t; }
            sqc[c] = zc[c] ? 0.0 : sq;
            if (zc[c]) n2c[c] = 1.0;
            xic[c] = 1.0 - sqc[c] / (n2c[c] * n2c[c]);
            u[c] = n0c[c] * xic[c];
        }
        double gu[CDFT_MAX_NC], gI, gn2, gxi;
        phi += T(assoc_general(P, u, I, n2m, xim, gu, gI, gn2, gxi));
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const double g_n0 = gu[c] * xic[c];
            const double g_xi = gu[c] * n0c[c];
            const double g_n2 = g_xi * 2.0 * sqc[c] / (n2c[c] * n2c[c] * n2c[c]);
            g[c][F2] += T(g_n0 / P.d[c] + g_n2 * PI * P.d[c]);
#pragma unroll
            for (int k = 0; k < ND; ++k)
                if (!zc[c]) g[c][FV + k] += T(g_xi * (-2.0 * TWO_PI * TWO_PI * double(n[c][FV + k]) / (n2c[c] * n2c[c])));
        }
        const double g_n2m = gn2 + gxi * 2.0 * nv2sqm / (d2m * d2m * d2m);
        const double g_n3m = gI * I * I;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            g[i][F2] += T(g_n2m * PI * P.m[i] * P.d[i]);
            g[i][F3] += T(g_n3m * P.m[i]);
#pragma unroll
            for (int k = 0; k < ND; ++k)
                g[i][FV + k] += T(gxi * (-2.0 * nv2m[k] / (d2m * d2m)) * (-TWO_PI * P.m[i]));
        }
    }
    return phi;
}
