// libcdft_b200: host side of the C ABI declared in include/cdft_b200.h.
//
// A plan (one DFTSystem) owns its device tables and work buffers.  A batch is
// a set of plans converged together: every kernel launch covers all of them
// and the per-iteration kernel sequence is captured once into a CUDA graph
// holding `iters_per_launch` fixed-point evaluations; the host only polls a
// device counter of finished systems between graph launches.
#include <cuda_runtime.h>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <algorithm>

#include "persistent.cuh"
#include "fft3d.cuh"
#include "fft3d_tma.cuh"
#include "tuning.cuh"
#include "bulk.cuh"

namespace {

thread_local int g_err_code = 0;
thread_local char g_err_msg[512] = {0};
thread_local long long g_launches = 0;

int set_error(int code, const char* fmt, ...)
{
    g_err_code = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err_msg, sizeof(g_err_msg), fmt, ap);
    va_end(ap);
    return code;
}

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t _e = (call);                                                                   \
        if (_e != cudaSuccess)                                                                     \
            return set_error(CDFT_E_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), \
                             __FILE__, __LINE__);                                                  \
    } while (0)

#define CHECK_LAUNCH()                                                                             \
    do {                                                                                           \
        cudaError_t _e = cudaGetLastError();                                                       \
        if (_e != cudaSuccess)                                                                     \
            return set_error(CDFT_E_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(_e), \
                             __FILE__, __LINE__);                                                  \
    } while (0)

const double kNA = 6.02214076e23;
const double kPCSAFT_A[21] = {
    0.9105631445, -0.3084016918, -0.0906148351, 0.6361281449, 0.1860531159, 0.4527842806,
    2.6861347891, -2.5030047259, 0.5962700728, -26.547362491, 21.419793629, -1.7241829131,
    97.759208784, -65.25588533, -4.1302112531, -159.59154087, 83.318680481, 13.77663187,
    91.297774084, -33.74692293, -8.6728470368};
const double kPCSAFT_B[21] = {
    0.7240946941, -0.5755498075, 0.0976883116, 2.2382791861, 0.6995095521, -0.2557574982,
    -4.0025849485, 3.892567339, -9.155856153, -21.003576815, -17.215471648, 20.642075974,
    26.855641363, 192.67226447, -38.804430052, 206.55133841, -161.82646165, 93.626774077,
    -355.60235612, -165.20769346, -29.666905585};

std::mutex g_const_mu;
bool g_const_done[64] = {false};   // per device: PC-SAFT constants uploaded to its __constant__ bank

}  // namespace

struct Batch;

// Dense radial operators on one device, shared by every plan of the same geometry,
// length unit and diameters (an isotherm in one pore builds them once); freed with the
// last plan that holds them.
struct RadialOps {
    int device = 0;
    double* d_mats = nullptr;
    RadialOps() = default;
    RadialOps(const RadialOps&) = delete;
    RadialOps& operator=(const RadialOps&) = delete;
    ~RadialOps()
    {
        int cur = -1;
        const bool other = cudaGetDevice(&cur) == cudaSuccess && cur != device;
        if (other) cudaSetDevice(device);
        cudaFree(d_mats);
        if (other) cudaSetDevice(cur);
    }
};

struct cdft_plan {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    cdft_system_desc desc;
    SysDev sys;            // host copy holding device pointers
    int N = 0, m_cap = -1;
    double dz[3] = {0, 0, 0};
    double* d_taps = nullptr;
    float* d_taps32 = nullptr;
    double* d_vext = nullptr;
    double* d_vec = nullptr;      // rho, sol, gx, res, df, out
    double* d_Q = nullptr;
    double* d_DG = nullptr;
    void* d_part = nullptr;
    void* d_dfield = nullptr;
    double* d_fval = nullptr;
    std::shared_ptr<RadialOps> rops;   // radial: dense weighted-density operators (both stages)
    double* d_rw = nullptr;       // radial: quadrature weights on the device
    std::vector<double> rw;       // radial: quadrature weights of the integral (angular factor included)
    void* d_spec = nullptr;       // 3D: convolved-field spectra [comp][field][z][y][kx]
    void* d_R = nullptr;          // 3D: spectrum of rho / accumulated adjoint spectrum
    void* d_adj = nullptr;        // 3D: adjoint sum in real space
    double* d_ktab = nullptr;     // 3D: kernel tables by |k|^2
    CUtensorMap tmaps[2][2][2];   // 3D: [FP32][R, spec][y box, z box] tensor maps of the spectra
    int tma_ready = 0;
    int L3 = 0, k2max = 0;        // 3D: points per dimension, max |k|^2 index
    double w0 = 0.0;              // 3D: reduced frequency per index
    double* d_ddft = nullptr;     // DDFT: [tg, tl] per axis, then eta and deta scratch
    size_t ddft_eta = 0;          // DDFT: offset of the eta scratch in d_ddft
    Batch* self = nullptr;        // batch of this plan alone
};

// host profiles of a batch of at most this many doubles in all are staged through one pinned buffer
#define CDFT_STAGE_MAX_ELEMS (4LL << 20)

struct Batch {
    std::vector<cdft_plan*> plans;
    int nsys = 0, nc = 0, nd = 0, mixed = 0, coord = 0;
    cudaStream_t stream = nullptr;
    SysDev* d_sys = nullptr;
    AAState* d_st = nullptr;
    ConvTask* d_tasks = nullptr;
    int ntasks = 0;
    Chunk* d_pchunks = nullptr;
    int npchunks = 0;
    Chunk* d_echunks = nullptr;
    int nechunks = 0;
    double* d_partials = nullptr;
    int* d_done = nullptr;
    int* h_done = nullptr;
    double* d_hist = nullptr;
    int hist_cap = 0;
    int cur32 = 0;                          // arithmetic of the running phase: 1 FP32, 0 FP64
    cudaGraphExec_t graph[2] = {nullptr, nullptr};   // indexed by cur32
    int graph_iters[2] = {0, 0};
    int vec_mb = CDFT_MAX_M;                          // compile-time depth bound of vec_kernel
    int graph_mb[2] = {0, 0};                         // ... captured in each graph
    TunedShapes graph_tuned[2];                       // ... and the launch shapes they were captured with
    long long graph_launches[2] = {0, 0};             // kernel launches captured in each graph
    CopyTask* d_copy = nullptr;                       // profile copies in [0, nsys) and out [nsys, 2 nsys)
    CopyTask* h_copy = nullptr;                       // ... their pinned host staging
    AAInit* d_init = nullptr;                         // per-system solver-state initialisation
    AAInit* h_init = nullptr;
    AASummary* d_sum = nullptr;                       // the final states' status fields
    AASummary* h_sum = nullptr;
    double* h_stage = nullptr;                        // host profiles staged back to back (pinned) ...
    double* d_stage = nullptr;                        // ... and on the device; small batches only
    long long stage_elems = 0;
    DenseGroup* d_groups = nullptr;                   // radial: column tiles of systems sharing an operator
    int ngroups = 0, group_blocks = 0;                // ... and the largest slots x row tiles among them
    int group_blocks2 = 0;                            // ... the same in tiles of 16 rows
};

namespace {

std::mutex g_batch_mu;
std::map<std::vector<cdft_plan*>, Batch*> g_batches;

// Upload the dispersion constants to the __constant__ bank of the current device (once per device).
int upload_constants()
{
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(CDFT_E_UNSUPPORTED, "device ordinal %d", dev);
    std::lock_guard<std::mutex> lk(g_const_mu);
    if (g_const_done[dev]) return 0;
    CU(cudaMemcpyToSymbol(c_pcsaft_a, kPCSAFT_A, sizeof(kPCSAFT_A)));
    CU(cudaMemcpyToSymbol(c_pcsaft_b, kPCSAFT_B, sizeof(kPCSAFT_B)));
    g_const_done[dev] = true;
    return 0;
}

void free_batch(Batch* b)
{
    if (!b) return;
    for (int k = 0; k < 2; ++k)
        if (b->graph[k]) cudaGraphExecDestroy(b->graph[k]);
    cudaFree(b->d_sys);
    cudaFree(b->d_st);
    cudaFree(b->d_tasks);
    cudaFree(b->d_pchunks);
    cudaFree(b->d_echunks);
    cudaFree(b->d_partials);
    cudaFree(b->d_groups);
    cudaFree(b->d_copy);
    cudaFree(b->d_init);
    cudaFree(b->d_sum);
    if (b->h_copy) cudaFreeHost(b->h_copy);
    if (b->h_init) cudaFreeHost(b->h_init);
    if (b->h_sum) cudaFreeHost(b->h_sum);
    if (b->h_stage) cudaFreeHost(b->h_stage);
    cudaFree(b->d_stage);
    cudaFree(b->d_done);
    cudaFree(b->d_hist);
    if (b->h_done) cudaFreeHost(b->h_done);
    delete b;
}

// ---------------------------------------------------------------------------
// plan construction
// ---------------------------------------------------------------------------
int validate_desc(const cdft_system_desc* d)
{
    if (!d) return set_error(CDFT_E_INVALID, "desc is NULL");
    if (d->nd != 1 && d->nd != 3) return set_error(CDFT_E_UNSUPPORTED, "nd=%d: 1D and 3D Cartesian systems are supported", d->nd);
    if (d->nd == 3) {
        const int n = d->ngrid[0];
        if (d->ngrid[1] != n || d->ngrid[2] != n || !(n == 32 || n == 64 || n == 128 || n == 256))
            return set_error(CDFT_E_UNSUPPORTED, "3D grids must be cubic with N in {32, 64, 128, 256} points per side");
        for (int k = 0; k < 3; ++k)
            if (!(d->bounds[k][1] > d->bounds[k][0]) ||
                std::fabs((d->bounds[k][1] - d->bounds[k][0]) - (d->bounds[0][1] - d->bounds[0][0])) >
                    1e-12 * (d->bounds[0][1] - d->bounds[0][0]))
                return set_error(CDFT_E_UNSUPPORTED, "3D boxes must be cubic (equal periods)");
        if (d->nc > 2) return set_error(CDFT_E_UNSUPPORTED, "3D systems support nc <= 2");
    }
    if (d->coord != CDFT_COORD_CART && d->coord != CDFT_COORD_SPH && d->coord != CDFT_COORD_CYL)
        return set_error(CDFT_E_INVALID, "coord=%d", d->coord);
    if (d->coord != CDFT_COORD_CART && (d->nd != 1 || d->ngrid[0] < 4))
        return set_error(CDFT_E_UNSUPPORTED, "spherical and cylindrical grids are 1D (radial) with at least 4 points");
    if (d->nc < 1 || d->nc > CDFT_MAX_NC) return set_error(CDFT_E_INVALID, "nc=%d out of [1,%d]", d->nc, CDFT_MAX_NC);
    if (d->ngrid[0] < 2) return set_error(CDFT_E_INVALID, "ngrid[0]=%d < 2", d->ngrid[0]);
    if (!(d->bounds[0][1] > d->bounds[0][0])) return set_error(CDFT_E_INVALID, "bounds must satisfy ub > lb");
    if (!(d->L > 0) || !(d->T > 0)) return set_error(CDFT_E_INVALID, "L and T must be positive");
    if (d->n_assoc < 0 || d->n_assoc > CDFT_MAX_ASSOC)
        return set_error(CDFT_E_UNSUPPORTED, "n_assoc=%d out of [0,%d]", d->n_assoc, CDFT_MAX_ASSOC);
    for (int i = 0; i < d->nc; ++i)
        if (!(d->hsd[i] > 0) || !(d->m[i] > 0)) return set_error(CDFT_E_INVALID, "component %d: hsd and m must be positive", i);
    {
        int keys[2 * CDFT_MAX_ASSOC], mult[2 * CDFT_MAX_ASSOC], nk = 0;
        for (int p = 0; p < d->n_assoc; ++p) {
            const cdft_assoc_pair& a = d->assoc[p];
            if (a.icomp < 0 || a.icomp >= d->nc || a.jcomp < 0 || a.jcomp >= d->nc)
                return set_error(CDFT_E_INVALID, "association pair %d: component out of range", p);
            if (a.isite < 0 || a.isite >= 64 || a.jsite < 0 || a.jsite >= 64 || a.n_ia < 1 || a.n_jb < 1)
                return set_error(CDFT_E_INVALID, "association pair %d: site index or multiplicity out of range", p);
            if (!(a.kappa_ab >= 0) || !std::isfinite(a.eps_ab))
                return set_error(CDFT_E_INVALID, "association pair %d: eps_ab and kappa_ab", p);
            const int ka = a.icomp * 64 + a.isite, kb = a.jcomp * 64 + a.jsite;
            const int ma = a.n_ia, mb = a.n_jb;
            for (int e = 0; e < 2; ++e) {
                const int key = e ? kb : ka, mu = e ? mb : ma;
                int q = 0;
                while (q < nk && keys[q] != key) ++q;
                if (q == nk) { keys[nk] = key; mult[nk++] = mu; }
                else if (mult[q] != mu)
                    return set_error(CDFT_E_INVALID, "association site (%d, %d): two multiplicities", key / 64, key % 64);
            }
        }
        if (nk > CDFT_MAX_SITES) return set_error(CDFT_E_UNSUPPORTED, "%d association sites (at most %d)", nk, CDFT_MAX_SITES);
        if (d->n_assoc > 1 && d->nc < 2)
            return set_error(CDFT_E_UNSUPPORTED, "several association pairs are supported for mixtures (nc >= 2)");
    }
    if (d->precision != CDFT_PREC_FP64 && d->precision != CDFT_PREC_MIXED)
        return set_error(CDFT_E_INVALID, "precision=%d", d->precision);
    return 0;
}

// Circulant taps (deriv: their derivatives in the kernel radius) of the 6 convolved
// fields of every component of a 1D Cartesian system, written to out[(i*6 + f)*N + q]:
// one launch (taps_table_kernel); grids above TAPS_TABLE_MAX_N points take the
// per-output kernels.  Fields of get_fields(::PCSAFTModel) in 1D (PCSAFT.jl:55-61).
int launch_taps(cudaStream_t stream, int N, double span, double L, int nc, const double* dred, double* out, bool deriv)
{
    const int types[6] = {1, 2, 3, 2, 1, 2};
    const double wf[6] = {0.5, 0.5, 0.5, 1.0, 1.0, PSI_DISP};
    if (nc * 6 > TAPS_MAX_TASKS) return set_error(CDFT_E_UNSUPPORTED, "nc=%d", nc);
    if (N > TAPS_TABLE_MAX_N) {
        for (int i = 0; i < nc; ++i)
            for (int f = 0; f < 6; ++f) {
                double* o = out + ((size_t)i * 6 + f) * N;
                if (deriv) dtaps1d_kernel<<<(N + 127) / 128, 128, 0, stream>>>(N, span, L, types[f], wf[f] * dred[i], o);
                else taps1d_kernel<<<(N + 127) / 128, 128, 0, stream>>>(N, span, L, types[f], wf[f] * dred[i], o);
                g_launches += 1;
            }
        CHECK_LAUNCH();
        return 0;
    }
    TapsArgs a;
    memset(&a, 0, sizeof(a));
    a.N = N;
    a.ntask = nc * 6;
    a.deriv = deriv ? 1 : 0;
    a.span = span;
    a.L = L;
    for (int i = 0; i < nc; ++i)
        for (int f = 0; f < 6; ++f) {
            const int t = i * 6 + f;
            a.type[t] = types[f];
            a.R[t] = 2.0 * 3.14159265358979323846 * (wf[f] * dred[i]);
            a.out[t] = out + (size_t)t * N;
        }
    const size_t smem = taps_smem_bytes(N);
    CU(cudaFuncSetAttribute(taps_table_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    taps_table_kernel<<<dim3(a.ntask, (N + TAPS_THREADS - 1) / TAPS_THREADS), TAPS_THREADS, smem, stream>>>(a);
    CHECK_LAUNCH();
    g_launches += 1;
    return 0;
}

int plan_alloc_m(cdft_plan* p, int m)
{
    if (m <= p->m_cap) return 0;
    cudaFree(p->d_Q);
    cudaFree(p->d_DG);
    p->d_Q = p->d_DG = nullptr;
    const size_t ne = (size_t)p->sys.n_elem;
    const size_t cols = (size_t)(m > 0 ? m : 1);
    const int qs = (int)(cols + (cols & 1));   // row-major QR history, 16-byte aligned rows
    CU(cudaMalloc(&p->d_Q, ne * qs * sizeof(double)));
    CU(cudaMalloc(&p->d_DG, ne * cols * sizeof(double)));
    CU(cudaMemsetAsync(p->d_Q, 0, ne * qs * sizeof(double), p->stream));
    CU(cudaMemsetAsync(p->d_DG, 0, ne * cols * sizeof(double), p->stream));
    p->m_cap = m;
    p->sys.Q = p->d_Q;
    p->sys.DG = p->d_DG;
    p->sys.qs = qs;
    return 0;
}

int plan_build3d(cdft_plan* p);

// ---------------------------------------------------------------------------
// Radial grids (Uniform1DSphr / Uniform1DCyl, src/base/structure.jl:355-433).
// The reference transforms with Hankel.jl's QDHT(0, n, ub, N) (n = 2 sphere, 1
// cylinder).  Restated from the published quasi-discrete Hankel transform
// (Guizar-Sicairos & Gutierrez-Vega, JOSA A 21 (2004) 53) for radially symmetric
// functions in n + 1 dimensions: Bessel order nu = (n - 1) / 2, zeros j_1..j_{N+1},
// S = j_{N+1}, r_m = j_m R / S, k_m = j_m / R, the symmetric matrix
// T_mq = 2 J_nu(j_m j_q / S) / (|J_{nu+1}(j_m)| |J_{nu+1}(j_q)| S) for both directions,
// and point weights a_m = r_m^nu / |J_{nu+1}(j_m)|.  A convolution with multiplier
// w(k) is then the dense operator diag(1/a) T diag(w) T diag(a).
// ---------------------------------------------------------------------------
std::vector<double> bessel_zeros(double nu, int count)
{
    std::vector<double> z(count);
    const double PI = 3.14159265358979323846;
    for (int m = 1; m <= count; ++m) {
        if (nu == 0.5) {   // J_{1/2}(x) = sqrt(2 / (pi x)) sin x
            z[m - 1] = m * PI;
            continue;
        }
        double x = (m - 0.25) * PI;   // McMahon's first term for J_0, then Newton (J_0' = -J_1)
        x += 1.0 / (8.0 * x);
        for (int it = 0; it < 60; ++it) {
            const double dx = std::cyl_bessel_j(0.0, x) / std::cyl_bessel_j(1.0, x);
            x += dx;
            if (std::fabs(dx) < 1e-16 * x) break;
        }
        z[m - 1] = x;
    }
    return z;
}

struct RadialKey {
    int device, coord, N, nc, nconv, pad;   // no padding bytes: compared by memcmp
    uint64_t R, L, d[CDFT_MAX_NC];          // bit patterns
    bool operator<(const RadialKey& o) const { return std::memcmp(this, &o, sizeof(RadialKey)) < 0; }
};
std::mutex g_rops_mu;
std::map<RadialKey, std::weak_ptr<RadialOps>> g_rops;

int radial_build(cdft_plan* p)
{
    const cdft_system_desc& d = p->desc;
    SysDev& S = p->sys;
    const int N = d.ngrid[0], nc = d.nc, nconv = S.nconv;
    const double PI = 3.14159265358979323846, TWO_PI = 2.0 * PI;
    const double nu = (d.coord == CDFT_COORD_SPH) ? 0.5 : 0.0;
    const double R = d.bounds[0][1], L = d.L;
    const std::vector<double> j = bessel_zeros(nu, N + 1);
    const double Sz = j[N];
    std::vector<double> r(N), k(N), a(N), jn1(N), T((size_t)N * N);
    p->rw.assign(N, 0.0);
    const double ang = (d.coord == CDFT_COORD_SPH) ? 4.0 * PI : TWO_PI;   // integrals.jl:18-19
    for (int m = 0; m < N; ++m) {
        r[m] = j[m] * R / Sz;
        k[m] = j[m] / R;
        jn1[m] = std::fabs(std::cyl_bessel_j(nu + 1.0, j[m]));
        a[m] = std::pow(r[m], nu) / jn1[m];
        // int_0^R f r^(2 nu + 1) dr: Fourier-Bessel quadrature of the k -> 0 limit
        p->rw[m] = ang * 2.0 * R * R / (Sz * Sz * jn1[m] * jn1[m]) * std::pow(r[m], 2.0 * nu);
    }
    CU(cudaMalloc(&p->d_rw, (size_t)N * sizeof(double)));
    CU(cudaMemcpyAsync(p->d_rw, p->rw.data(), (size_t)N * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    S.qw = p->d_rw;
    // the operators depend on the grid (coordinates, N, R), L and the diameters only
    RadialKey key;
    std::memset(&key, 0, sizeof(key));
    key.device = p->device;
    key.coord = d.coord;
    key.N = N;
    key.nc = nc;
    key.nconv = nconv;
    std::memcpy(&key.R, &R, sizeof(double));
    std::memcpy(&key.L, &L, sizeof(double));
    for (int i = 0; i < nc; ++i) std::memcpy(&key.d[i], &S.phi.d[i], sizeof(double));
    {
        std::lock_guard<std::mutex> lk(g_rops_mu);
        auto it = g_rops.find(key);
        if (it != g_rops.end()) {
            if (auto ops = it->second.lock()) {
                p->rops = ops;
                S.mats = ops->d_mats;
                CU(cudaStreamSynchronize(p->stream));
                return 0;
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (int m = 0; m < N; ++m)
        for (int q = 0; q < N; ++q)
            T[(size_t)m * N + q] = 2.0 * std::cyl_bessel_j(nu, j[m] * j[q] / Sz) / (jn1[m] * jn1[q] * Sz);
    // radial_derivative_matrix (src/structure/transforms.jl:43-64) on the physical grid
    std::vector<double> D((size_t)N * N, 0.0);
    for (int i = 1; i < N - 1; ++i) {
        const double h1 = r[i] - r[i - 1], h2 = r[i + 1] - r[i];
        D[(size_t)i * N + i - 1] = -h2 / (h1 * (h1 + h2));
        D[(size_t)i * N + i] = (h2 - h1) / (h1 * h2);
        D[(size_t)i * N + i + 1] = h1 / (h2 * (h1 + h2));
    }
    {
        double h1 = r[1] - r[0], h2 = r[2] - r[1];
        D[0] = -(2 * h1 + h2) / (h1 * (h1 + h2));
        D[1] = (h1 + h2) / (h1 * h2);
        D[2] = -h1 / (h2 * (h1 + h2));
        h1 = r[N - 2] - r[N - 3];
        h2 = r[N - 1] - r[N - 2];
        D[(size_t)(N - 1) * N + N - 3] = h2 / (h1 * (h1 + h2));
        D[(size_t)(N - 1) * N + N - 2] = -(h1 + h2) / (h1 * h2);
        D[(size_t)(N - 1) * N + N - 1] = (2 * h2 + h1) / (h2 * (h1 + h2));
    }
    auto conv = [&](const std::vector<double>& w, std::vector<double>& M) {   // diag(1/a) T diag(w) T diag(a)
        std::vector<double> TW((size_t)N * N);
        for (int m = 0; m < N; ++m)
            for (int q = 0; q < N; ++q) TW[(size_t)m * N + q] = T[(size_t)m * N + q] * w[q];
        M.assign((size_t)N * N, 0.0);
#pragma omp parallel for schedule(static)
        for (int m = 0; m < N; ++m)
            for (int t = 0; t < N; ++t) {
                const double v = TW[(size_t)m * N + t];
                for (int q = 0; q < N; ++q) M[(size_t)m * N + q] += v * T[(size_t)t * N + q];
            }
        for (int m = 0; m < N; ++m)
            for (int q = 0; q < N; ++q) M[(size_t)m * N + q] *= a[q] / a[m];
    };
    // fields of get_fields(::PCSAFTModel) (PCSAFT.jl:55-61): types and widths as in 1D Cartesian
    const int types[6] = {1, 2, 3, 2, 1, 2};
    const double wf[6] = {0.5, 0.5, 0.5, 1.0, 1.0, PSI_DISP};
    const size_t NN = (size_t)N * N;
    std::vector<double> mats(2 * (size_t)nc * nconv * NN);
    std::vector<double> w(N), M;
    for (int i = 0; i < nc; ++i)
        for (int f = 0; f < nconv; ++f) {
            const double width = wf[f] * S.phi.d[i];
            double* A0 = mats.data() + ((size_t)(0 * nc + i) * nconv + f) * NN;
            double* A1 = mats.data() + ((size_t)(1 * nc + i) * nconv + f) * NN;
            if (types[f] != 3) {   // SWeightedDensity(::RadialFrequency): omega_bar scaled by L, R = 2 pi width
                const double Rr = TWO_PI * width;
                for (int m = 0; m < N; ++m) {
                    const double wb = k[m] / TWO_PI * L;
                    w[m] = (types[f] == 1) ? 2.0 * std::sin(wb * Rr) / wb / TWO_PI
                                           : 4.0 * PI / (wb * wb * wb) * (std::sin(wb * Rr) - Rr * wb * std::cos(wb * Rr))
                                                 / (TWO_PI * TWO_PI * TWO_PI);
                }
                conv(w, M);
                std::copy(M.begin(), M.end(), A0);
                std::copy(M.begin(), M.end(), A1);   // integrate_field! applies the same convolution
            } else {   // VWeightedDensity(::RadialFrequency): D QDHT^-1 diag(H) QDHT, raw omega, physical width
                const double Rk = TWO_PI * width * L;
                for (int m = 0; m < N; ++m) {
                    const double wr = k[m] / TWO_PI;
                    w[m] = 4.0 * PI / (wr * wr * wr) * (std::sin(wr * Rk) - Rk * wr * std::cos(wr * Rk))
                           / (TWO_PI * TWO_PI * TWO_PI);
                }
                conv(w, M);
                // D has nonzeros in columns m - 1..m + 1 (rows 0 and N - 1: 0..2, N - 3..N - 1), so
                // the sum over t runs over that band only (the skipped terms are exact zeros)
#pragma omp parallel for schedule(static)
                for (int m = 0; m < N; ++m)
                    for (int q = 0; q < N; ++q) {
                        double v = 0.0;
                        const int t0 = std::max(0, m - 2), t1 = std::min(N - 1, m + 2);
                        for (int t = t0; t <= t1; ++t) v += D[(size_t)m * N + t] * M[(size_t)t * N + q];
                        A0[(size_t)m * N + q] = v;
                    }
                // adjoint: the transpose, added (weighted_densities.jl:368-385); stored negated because
                // the EL assembly subtracts the vector field's adjoint term (the Cartesian sign)
                for (int m = 0; m < N; ++m)
                    for (int q = 0; q < N; ++q) A1[(size_t)m * N + q] = -A0[(size_t)q * N + m];
            }
        }
    auto ops = std::make_shared<RadialOps>();
    ops->device = p->device;
    CU(cudaMalloc(&ops->d_mats, mats.size() * sizeof(double)));
    CU(cudaMemcpyAsync(ops->d_mats, mats.data(), mats.size() * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    CU(cudaStreamSynchronize(p->stream));
    p->rops = ops;
    S.mats = ops->d_mats;
    std::lock_guard<std::mutex> lk(g_rops_mu);
    for (auto it = g_rops.begin(); it != g_rops.end();)   // drop the entries whose plans are gone
        it = it->second.expired() ? g_rops.erase(it) : std::next(it);
    g_rops[key] = ops;
    return 0;
}

// Association tables of PhiParams from the descriptor's pairs (pack_assoc_params,
// assoc.jl:18-56): one pair fills the analytic path's fields, several the general
// solve's site and pair tables (sites numbered by (component, site) in ascending order).
static void fill_assoc_params(PhiParams& P, const cdft_system_desc& d)
{
    const int nc = d.nc;
    const double L = d.L, T = d.T;
    P.has_assoc = d.n_assoc;
    P.a_ns = 0;
    auto K_of = [&](const cdft_assoc_pair& a) {
        const double sg = d.sigma[a.icomp * nc + a.jcomp] / L;
        return sg * sg * sg * (exp(a.eps_ab / T) - 1.0) * a.kappa_ab;
    };
    auto dij_of = [&](const cdft_assoc_pair& a) {
        const double di = P.d[a.icomp], dj = P.d[a.jcomp];
        return di * dj / (di + dj);
    };
    if (d.n_assoc == 1) {
        const cdft_assoc_pair& a = d.assoc[0];
        P.a_ic = a.icomp;
        P.a_jc = a.jcomp;
        P.a_nia = a.n_ia;
        P.a_njb = a.n_jb;
        P.a_dij = dij_of(a);
        P.a_K = K_of(a);
    } else if (d.n_assoc > 1) {
        int keys[2 * CDFT_MAX_ASSOC], nk = 0;   // key = component * 64 + site
        for (int p = 0; p < d.n_assoc; ++p) {
            const int ka = d.assoc[p].icomp * 64 + d.assoc[p].isite, kb = d.assoc[p].jcomp * 64 + d.assoc[p].jsite;
            for (int key : {ka, kb}) {
                bool seen = false;
                for (int q = 0; q < nk; ++q) seen |= keys[q] == key;
                if (!seen) keys[nk++] = key;
            }
        }
        std::sort(keys, keys + nk);
        P.a_ns = nk;
        auto site_of = [&](int key) { return int(std::lower_bound(keys, keys + nk, key) - keys); };
        for (int p = 0; p < d.n_assoc; ++p) {
            const cdft_assoc_pair& a = d.assoc[p];
            const int sa = site_of(a.icomp * 64 + a.isite), sb = site_of(a.jcomp * 64 + a.jsite);
            P.g_pa[p] = sa;
            P.g_pb[p] = sb;
            P.g_sc[sa] = a.icomp;
            P.g_sc[sb] = a.jcomp;
            P.g_sm[sa] = a.n_ia;
            P.g_sm[sb] = a.n_jb;
            P.g_nia[p] = a.n_ia;
            P.g_njb[p] = a.n_jb;
            P.g_dij[p] = dij_of(a);
            P.g_K[p] = K_of(a);
        }
    }
}

int plan_build(cdft_plan* p)
{
    if (p->desc.nd == 3) return plan_build3d(p);
    const cdft_system_desc& d = p->desc;
    SysDev& S = p->sys;
    memset(&S, 0, sizeof(S));
    const int N = d.ngrid[0];
    const int nc = d.nc;
    p->N = N;
    S.nd = d.nd;
    S.N = N;
    S.nc = nc;
    S.NF = 6 + d.nd;
    S.nconv = S.NF - 1;
    S.ngrid[0] = N; S.ngrid[1] = 1; S.ngrid[2] = 1;
    S.ksplit = (d.coord == CDFT_COORD_CART) ? (N + CONV_QC - 1) / CONV_QC : 1;
    S.n_elem = N * nc;
    S.mixed = d.precision == CDFT_PREC_MIXED;
    const double L = d.L, T = d.T;
    S.NA = kNA * L * L * L;
    p->dz[0] = (d.bounds[0][1] - d.bounds[0][0]) / N;
    S.wscale = p->dz[0] / 3.0;
    for (int i = 0; i < nc; ++i) S.cprd[i] = d.mu_res_plus_ln_rhob[i];
    PhiParams& P = S.phi;
    P.nc = nc;
    P.nd = d.nd;
    P.T = T;
    for (int i = 0; i < nc; ++i) {
        P.m[i] = d.m[i];
        P.d[i] = d.hsd[i] / L;
    }
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            const double s = d.sigma[i * nc + j] / L;
            const double e = d.eps[i * nc + j];
            const double c1 = d.m[i] * d.m[j] * s * s * s * e / T;
            P.c1[i * CDFT_MAX_NC + j] = c1;
            P.c2[i * CDFT_MAX_NC + j] = c1 * e / T;
        }
    fill_assoc_params(P, d);

    const size_t ne = (size_t)S.n_elem;
    const size_t ntap = (size_t)S.nconv * nc * N;
    const size_t esz = sizeof(double);   // mixed plans finish with an FP64 phase in the same buffers
    CU(cudaMalloc(&p->d_taps, ntap * sizeof(double)));
    CU(cudaMalloc(&p->d_vec, ne * 6 * sizeof(double)));
    CU(cudaMemsetAsync(p->d_vec, 0, ne * 6 * sizeof(double), p->stream));
    CU(cudaMalloc(&p->d_part, ntap * S.ksplit * esz));
    CU(cudaMalloc(&p->d_dfield, (size_t)S.NF * nc * N * esz));
    CU(cudaMalloc(&p->d_fval, (size_t)N * sizeof(double)));
    if (d.vext) {
        CU(cudaMalloc(&p->d_vext, ne * sizeof(double)));
        CU(cudaMemcpyAsync(p->d_vext, d.vext, ne * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    }
    S.rho = p->d_vec;
    S.sol = p->d_vec + ne;
    S.gx = p->d_vec + 2 * ne;
    S.res = p->d_vec + 3 * ne;
    S.df = p->d_vec + 4 * ne;
    S.out = p->d_vec + 5 * ne;
    S.part = p->d_part;
    S.dfield = p->d_dfield;
    S.fval = p->d_fval;
    S.vext = p->d_vext;
    S.taps = p->d_taps;

    if (d.coord != CDFT_COORD_CART) {
        const int rc = radial_build(p);
        CU(cudaStreamSynchronize(p->stream));
        return rc;
    }
    // kernels of get_fields(::PCSAFTModel) (PCSAFT.jl:55-61), fields 2..7 in 1D
    const double span = d.bounds[0][1] - d.bounds[0][0];
    int rc = launch_taps(p->stream, N, span, L, nc, P.d, p->d_taps, false);
    if (rc) return rc;
    if (S.mixed) {
        CU(cudaMalloc(&p->d_taps32, ntap * sizeof(float)));
        to_float_kernel<<<(unsigned)((ntap + 255) / 256), 256, 0, p->stream>>>(p->d_taps, p->d_taps32, ntap);
        CHECK_LAUNCH();
        S.taps32 = p->d_taps32;
    }
    CU(cudaStreamSynchronize(p->stream));
    return 0;
}


// Reduced PC-SAFT parameters of preallocate_params (PCSAFT.jl:213-285) for a system record.
void fill_phi_params(const cdft_system_desc& d, SysDev& S)
{
    const double L = d.L, T = d.T;
    const int nc = d.nc;
    PhiParams& P = S.phi;
    P.nc = nc;
    P.nd = d.nd;
    P.T = T;
    for (int i = 0; i < nc; ++i) {
        P.m[i] = d.m[i];
        P.d[i] = d.hsd[i] / L;
    }
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            const double sg = d.sigma[i * nc + j] / L;
            const double e = d.eps[i * nc + j];
            const double c1 = d.m[i] * d.m[j] * sg * sg * sg * e / T;
            P.c1[i * CDFT_MAX_NC + j] = c1;
            P.c2[i * CDFT_MAX_NC + j] = c1 * e / T;
        }
    fill_assoc_params(P, d);
}

// omega_hat of SWeightedDensity (weighted_densities.jl:48-69) at reduced |omega|
double kernel_hat(int type, double wb, double R)
{
    const double PI = 3.14159265358979323846, TWO_PI = 2.0 * PI;
    if (type == 1) return (wb == 0.0) ? 2.0 * R / TWO_PI : 2.0 * std::sin(wb * R) / wb / TWO_PI;
    if (wb == 0.0) return 4.0 * PI * R * R * R / 3.0 / (TWO_PI * TWO_PI * TWO_PI);
    return 4.0 * PI / (wb * wb * wb) * (std::sin(wb * R) - R * wb * std::cos(wb * R)) / (TWO_PI * TWO_PI * TWO_PI);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int get_encode_tiled(EncodeTiledFn* out)
{
    static std::mutex mu;
    static EncodeTiledFn fn = nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        CU(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p)
            return set_error(CDFT_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    *out = fn;
    return 0;
}

// Tensor map of `nfields` half spectra of L^3 points in precision fp32/fp64 at `base`:
// a 4D tensor {2 KX, L, L, nfields} of reals with rows of 2 KXP reals (KXP = L/2 + 2, so every
// stride is a multiple of 16 bytes), box {2 lines, L, 1, 1} (axis 1, y) or {2 lines, 1, L, 1}.
int make_spectrum_map(CUtensorMap* m, bool fp32, void* base, int L, int lines, int nfields, int axis)
{
    EncodeTiledFn enc = nullptr;
    int rc = get_encode_tiled(&enc);
    if (rc) return rc;
    const size_t es = fp32 ? sizeof(float) : sizeof(double);
    const int KX = L / 2 + 1, KXP = L / 2 + 2;
    const cuuint64_t dims[4] = {(cuuint64_t)(2 * KX), (cuuint64_t)L, (cuuint64_t)L, (cuuint64_t)nfields};
    const cuuint64_t strides[3] = {(cuuint64_t)(2 * KXP * es), (cuuint64_t)(2 * KXP * es) * L,
                                   (cuuint64_t)(2 * KXP * es) * L * L};
    const cuuint32_t box[4] = {(cuuint32_t)(2 * lines), (cuuint32_t)(axis == 1 ? L : 1), (cuuint32_t)(axis == 1 ? 1 : L), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    if (((uintptr_t)base & 15) || (strides[0] & 15) || ((2 * lines * es) & 15))
        return set_error(CDFT_E_INVALID, "spectrum tensor map: 16-byte alignment violated");
    const CUresult r = enc(m, fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims,
                           strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(CDFT_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return 0;
}

// lines per tile of the transforms of L points in each precision (FftLines of fft3d.cuh)
int fft_lines_of(bool fp32, int L)
{
    return fp32 ? ((L * 4 <= 512) ? 16 : 8) : ((L * 8 <= 512) ? 16 : 8);
}

// 3D periodic cubic box: FFT weighted densities (fft3d.cuh)
int plan_build3d(cdft_plan* p)
{
    const cdft_system_desc& d = p->desc;
    SysDev& S = p->sys;
    memset(&S, 0, sizeof(S));
    const int L3 = d.ngrid[0], nc = d.nc;
    const size_t npts = (size_t)L3 * L3 * L3;
    const size_t nspec = (size_t)(L3 / 2 + 2) * L3 * L3;   // rows padded to KXP = L/2 + 2
    p->N = (int)npts;
    p->L3 = L3;
    S.nd = 3;
    S.N = (int)npts;
    S.nc = nc;
    S.NF = 9;
    S.nconv = 8;
    S.ngrid[0] = S.ngrid[1] = S.ngrid[2] = L3;
    S.ksplit = 1;
    S.n_elem = (int)(npts * nc);
    S.mixed = d.precision == CDFT_PREC_MIXED;
    const double Lr = d.L;
    S.NA = kNA * Lr * Lr * Lr;
    for (int k = 0; k < 3; ++k) p->dz[k] = (d.bounds[k][1] - d.bounds[k][0]) / L3;
    S.wscale = (p->dz[0] / 3.0) * (p->dz[1] / 3.0) * (p->dz[2] / 3.0);
    for (int i = 0; i < nc; ++i) S.cprd[i] = d.mu_res_plus_ln_rhob[i];
    fill_phi_params(d, S);
    const size_t ne = (size_t)S.n_elem;
    CU(cudaMalloc(&p->d_vec, ne * 6 * sizeof(double)));
    CU(cudaMemsetAsync(p->d_vec, 0, ne * 6 * sizeof(double), p->stream));
    CU(cudaMalloc(&p->d_part, (size_t)S.nconv * nc * npts * sizeof(double)));
    CU(cudaMalloc(&p->d_dfield, (size_t)S.NF * nc * npts * sizeof(double)));
    CU(cudaMalloc(&p->d_adj, ne * sizeof(double)));
    CU(cudaMalloc(&p->d_spec, (size_t)S.nconv * nc * nspec * 2 * sizeof(double)));
    CU(cudaMalloc(&p->d_R, (size_t)nc * nspec * 2 * sizeof(double)));
    CU(cudaMalloc(&p->d_fval, npts * sizeof(double)));
    if (d.vext) {
        CU(cudaMalloc(&p->d_vext, ne * sizeof(double)));
        CU(cudaMemcpyAsync(p->d_vext, d.vext, ne * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    }
    // kernel tables by integer |k|^2: omega_bar = sqrt(k2) * L / period (structure_ω + _scaled_ω)
    const int half = L3 / 2;
    p->k2max = 3 * half * half;
    p->w0 = Lr / (d.bounds[0][1] - d.bounds[0][0]);
    const int types[5] = {1, 2, 2, 1, 2};                 // n2(d/2), n3(d/2), n3(d), n2(d), n3(psi d)
    const double wf[5] = {0.5, 0.5, 1.0, 1.0, PSI_DISP};
    std::vector<double> tab((size_t)nc * 5 * (p->k2max + 1));
    for (int i = 0; i < nc; ++i)
        for (int t = 0; t < 5; ++t) {
            const double R = 2.0 * 3.14159265358979323846 * wf[t] * S.phi.d[i];
            for (int k2 = 0; k2 <= p->k2max; ++k2)
                tab[((size_t)i * 5 + t) * (p->k2max + 1) + k2] = kernel_hat(types[t], std::sqrt((double)k2) * p->w0, R);
        }
    CU(cudaMalloc(&p->d_ktab, tab.size() * sizeof(double)));
    CU(cudaMemcpyAsync(p->d_ktab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    // tensor maps of the spectra for the TMA y/z passes, both precisions (mixed plans run both)
    for (int f32 = 0; f32 < 2; ++f32)
        for (int axis = 1; axis <= 2; ++axis) {
            const int lines = fft_lines_of(f32 != 0, L3);
            int rc = make_spectrum_map(&p->tmaps[f32][0][axis - 1], f32 != 0, p->d_R, L3, lines, nc, axis);
            if (!rc) rc = make_spectrum_map(&p->tmaps[f32][1][axis - 1], f32 != 0, p->d_spec, L3, lines, nc * S.nconv, axis);
            if (rc) return rc;
        }
    p->tma_ready = 1;
    S.rho = p->d_vec;
    S.sol = p->d_vec + ne;
    S.gx = p->d_vec + 2 * ne;
    S.res = p->d_vec + 3 * ne;
    S.df = p->d_vec + 4 * ne;
    S.out = p->d_vec + 5 * ne;
    S.part = p->d_part;
    S.dfield = p->d_dfield;
    S.adj = p->d_adj;
    S.fval = p->d_fval;
    S.vext = p->d_vext;
    CU(cudaStreamSynchronize(p->stream));
    return 0;
}

void plan_free(cdft_plan* p)
{
    cudaFree(p->d_rw);
    p->rops.reset();
    cudaFree(p->d_taps);
    cudaFree(p->d_taps32);
    cudaFree(p->d_vext);
    cudaFree(p->d_vec);
    cudaFree(p->d_Q);
    cudaFree(p->d_DG);
    cudaFree(p->d_part);
    cudaFree(p->d_dfield);
    cudaFree(p->d_fval);
    cudaFree(p->d_spec);
    cudaFree(p->d_R);
    cudaFree(p->d_adj);
    cudaFree(p->d_ktab);
    cudaFree(p->d_ddft);
    if (p->own_stream) cudaStreamDestroy(p->own_stream);
}

// ---------------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------------
int batch_build(const std::vector<cdft_plan*>& plans, Batch** out)
{
    Batch* b = new Batch();
    b->plans = plans;
    b->nsys = (int)plans.size();
    b->nc = plans[0]->desc.nc;
    b->nd = plans[0]->desc.nd;
    b->coord = plans[0]->desc.coord;
    b->mixed = plans[0]->sys.mixed;
    b->cur32 = b->mixed;
    b->stream = plans[0]->stream;
    for (auto* p : plans) {
        if (p->desc.nc != b->nc || p->desc.nd != b->nd || p->sys.mixed != b->mixed || p->desc.coord != b->coord) {
            free_batch(b);
            return set_error(CDFT_E_UNSUPPORTED, "systems of one batch must share nc, nd, coordinates and precision");
        }
        if (p->device != plans[0]->device) {
            free_batch(b);
            return set_error(CDFT_E_INVALID, "systems of one batch must live on one device");
        }
    }
    if (b->nd == 3 && b->nsys != 1) {
        free_batch(b);
        return set_error(CDFT_E_UNSUPPORTED, "3D systems are converged one per batch");
    }
    std::vector<ConvTask> tasks;
    std::vector<Chunk> pch, ech;
    for (int s = 0; s < b->nsys; ++s) {
        SysDev& S = plans[s]->sys;
        const int tiles = (S.N + CONV_TILE - 1) / CONV_TILE;
        if (b->nd == 1 && b->coord == CDFT_COORD_CART)
            for (int i = 0; i < S.nc; ++i)
                for (int f = 0; f < S.nconv; ++f)
                    for (int t = 0; t < tiles; ++t)
                        for (int ks = 0; ks < S.ksplit; ++ks) tasks.push_back({s, i, f, t * S.ksplit + ks});
        for (int j = 0; j < S.N; j += POINT_THREADS) pch.push_back({s, j});
        S.chunk_begin = (int)ech.size();
        for (int e = 0; e < S.n_elem; e += ELEM_CHUNK) ech.push_back({s, e});
        S.chunk_count = (int)ech.size() - S.chunk_begin;
    }
    // radial: systems whose plans share one operator buffer, in tiles of DGRP_COLS (batch order)
    std::vector<DenseGroup> groups;
    if (b->coord != CDFT_COORD_CART) {
        std::vector<const double*> keys;
        std::vector<std::vector<int>> members;
        for (int s = 0; s < b->nsys; ++s) {
            const double* m = plans[s]->sys.mats;
            size_t g = std::find(keys.begin(), keys.end(), m) - keys.begin();
            if (g == keys.size()) {
                keys.push_back(m);
                members.emplace_back();
            }
            members[g].push_back(s);
        }
        for (const auto& mem : members)
            for (size_t t = 0; t < mem.size(); t += DGRP_COLS) {
                DenseGroup G;
                G.ns = (int)std::min<size_t>(DGRP_COLS, mem.size() - t);
                for (int c = 0; c < DGRP_COLS; ++c) G.sys[c] = mem[t + (c < G.ns ? c : 0)];
                const SysDev& S = plans[G.sys[0]]->sys;
                b->group_blocks = std::max(b->group_blocks, S.nc * S.nconv * ((S.N + 7) / 8));
                b->group_blocks2 = std::max(b->group_blocks2, S.nc * S.nconv * ((S.N + 15) / 16));
                groups.push_back(G);
            }
    }
    b->ngroups = (int)groups.size();
    if (b->ngroups > 65535) {
        free_batch(b);
        return set_error(CDFT_E_UNSUPPORTED, "radial batch of %d column tiles (at most 65535)", b->ngroups);
    }
    b->ntasks = (int)tasks.size();
    b->npchunks = (int)pch.size();
    b->nechunks = (int)ech.size();
#define BCU(call)                      \
    do {                               \
        cudaError_t _e = (call);       \
        if (_e != cudaSuccess) {       \
            free_batch(b);             \
            return set_error(CDFT_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e)); \
        }                              \
    } while (0)
    BCU(cudaMalloc(&b->d_sys, sizeof(SysDev) * b->nsys));
    BCU(cudaMalloc(&b->d_st, sizeof(AAState) * b->nsys));
    BCU(cudaMalloc(&b->d_tasks, sizeof(ConvTask) * std::max<size_t>(tasks.size(), 1)));
    BCU(cudaMalloc(&b->d_pchunks, sizeof(Chunk) * pch.size()));
    BCU(cudaMalloc(&b->d_echunks, sizeof(Chunk) * ech.size()));
    BCU(cudaMalloc(&b->d_partials, sizeof(double) * RED_SLOTS * ech.size()));
    BCU(cudaMalloc(&b->d_done, 2 * sizeof(int)));        // [0] finished systems, [1] kernel error word
    BCU(cudaMallocHost(&b->h_done, 2 * sizeof(int)));
    BCU(cudaMalloc(&b->d_copy, sizeof(CopyTask) * 2 * b->nsys));
    BCU(cudaMallocHost(&b->h_copy, sizeof(CopyTask) * 2 * b->nsys));
    BCU(cudaMalloc(&b->d_init, sizeof(AAInit) * b->nsys));
    BCU(cudaMallocHost(&b->h_init, sizeof(AAInit) * b->nsys));
    BCU(cudaMalloc(&b->d_sum, sizeof(AASummary) * b->nsys));
    BCU(cudaMallocHost(&b->h_sum, sizeof(AASummary) * b->nsys));
    if (!tasks.empty())
        BCU(cudaMemcpy(b->d_tasks, tasks.data(), sizeof(ConvTask) * tasks.size(), cudaMemcpyHostToDevice));
    if (!groups.empty()) {
        BCU(cudaMalloc(&b->d_groups, sizeof(DenseGroup) * groups.size()));
        BCU(cudaMemcpy(b->d_groups, groups.data(), sizeof(DenseGroup) * groups.size(), cudaMemcpyHostToDevice));
    }
    BCU(cudaMemcpy(b->d_pchunks, pch.data(), sizeof(Chunk) * pch.size(), cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->d_echunks, ech.data(), sizeof(Chunk) * ech.size(), cudaMemcpyHostToDevice));
#undef BCU
    *out = b;
    return 0;
}

int batch_upload_sys(Batch* b)
{
    std::vector<SysDev> h(b->nsys);
    for (int s = 0; s < b->nsys; ++s) h[s] = b->plans[s]->sys;
    CU(cudaMemcpyAsync(b->d_sys, h.data(), sizeof(SysDev) * b->nsys, cudaMemcpyHostToDevice, b->stream));
    return 0;
}

template <typename T>
int launch_phi(Batch* b, const AAState* st)
{
#define PHI_CASE(NC_, ND_)                                                                              \
    if (b->nc == NC_ && b->nd == ND_) {                                                                 \
        phi_kernel<T, NC_, ND_><<<b->npchunks, POINT_THREADS, 0, b->stream>>>(b->d_pchunks, b->d_sys, st); \
        return 0;                                                                                       \
    }
    PHI_CASE(1, 1) PHI_CASE(2, 1) PHI_CASE(3, 1) PHI_CASE(4, 1)
#undef PHI_CASE
    if (b->nd == 3 && b->nc == 1) {
        phi_kernel3d<T, 1><<<b->npchunks, POINT_THREADS, 0, b->stream>>>(b->d_pchunks, b->d_sys, st);
        return 0;
    }
    if (b->nd == 3 && b->nc == 2) {
        phi_kernel3d<T, 2><<<b->npchunks, POINT_THREADS, 0, b->stream>>>(b->d_pchunks, b->d_sys, st);
        return 0;
    }
    return set_error(CDFT_E_UNSUPPORTED, "no Phi kernel for nc=%d nd=%d", b->nc, b->nd);
}

template <typename K>
int fft_attr(K kern, size_t smem)
{
    CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return 0;
}

// Grid of a persistent tile kernel: as many blocks as are resident at once (occupancy x SMs),
// at most one per tile.  Cached per (kernel, device).
int persistent_grid(const void* kern, int threads, size_t smem, int ntiles, int* grid)
{
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> cache;
    int dev = 0;
    CU(cudaGetDevice(&dev));
    int per = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find({kern, dev});
        if (it != cache.end()) per = it->second;
    }
    if (!per) {
        int occ = 0, nsm = 0;
        CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem));
        CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        per = std::max(occ, 1) * nsm;
        std::lock_guard<std::mutex> lk(mu);
        cache[{kern, dev}] = per;
    }
    *grid = std::min(ntiles, per);
    return 0;
}

// the fused inverse x pass + Phi + forward x pass (fft_x_phi_fused) for nc components
template <typename T, int L, int NC>
int launch_fused_nc(Batch* b, const AAState* st, typename V2<T>::t* spec, size_t nspec, int* err)
{
    constexpr int LF = FusedLines<T, L, NC>::value;
    constexpr size_t smem = fused_smem_bytes<T, L, NC, LF>();
    static_assert(smem <= FUSED_SMEM_MAX, "fused x pass does not fit one block");
    const SysDev& S = b->plans[0]->sys;
    const size_t npts = (size_t)L * L * L;
    CU(cudaFuncSetAttribute(fft_x_phi_fused<T, L, NC, LF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fft_x_phi_fused<T, L, NC, LF><<<L * L / (2 * LF), FUSED_THREADS, smem, b->stream>>>(
        spec, nspec, b->d_sys, T(S.NA / (double)npts), st, err);
    g_launches += 1;
    return 0;
}

// weighted densities, Phi and (with_int) the adjoint of a 3D system by FFT
template <typename T, int L>
int launch_eval3d_L(Batch* b, const AAState* st, bool with_int)
{
    typedef typename V2<T>::t C;
    constexpr int LINES = FftLines<T, L>::value;
    cdft_plan* p = b->plans[0];
    const SysDev& S = p->sys;
    const int nc = S.nc;
    const int KX = L / 2 + 1;
    const size_t npts = (size_t)L * L * L, nspec = (size_t)Spec3<L>::KXP * L * L;
    const int ntile = (KX + LINES - 1) / LINES;
    const int xblocks = L * L / (2 * LINES);
    const size_t smem2 = (size_t)(2 * L * (LINES + 1) + L / 2) * sizeof(C);
    const size_t smem3 = (size_t)(3 * L * (LINES + 1) + L / 2) * sizeof(C);
    int rc = 0;
    if ((rc = fft_attr(fft_x_r2c<T, double, L, LINES>, smem2)) || (rc = fft_attr(fft_x_r2c<T, T, L, LINES>, smem2)) ||
        (rc = fft_attr(fft_x_c2r<T, L, LINES>, smem2)) || (rc = fft_attr(fft_yz<T, L, LINES>, smem2)) ||
        (rc = fft_attr(fft_z_eval<T, L, LINES>, smem3)) || (rc = fft_attr(fft_z_adjoint<T, L, LINES>, smem3)))
        return rc;
    C* R = reinterpret_cast<C*>(p->d_R);
    C* spec = reinterpret_cast<C*>(p->d_spec);
    T* part = reinterpret_cast<T*>(S.part);
    T* dfield = reinterpret_cast<T*>(S.dfield);
    T* adj = reinterpret_cast<T*>(S.adj);
    KTab3 K;
    K.tab = p->d_ktab;
    K.k2max = p->k2max;
    K.w0 = p->w0;
    K.nconv = S.nconv;
    cudaStream_t str = b->stream;
    // the strided y and z passes: TMA tile kernels (fft3d_tma.cuh) or the per-thread-load kernels
    const bool tma = g_tuned.fft3d_tma && p->tma_ready;
    const int f32 = (sizeof(T) == 4) ? 1 : 0;
    int* err = b->d_done + 1;
    const size_t sm_yz = fft_tma_smem_yz<T, L, LINES>(), sm_ze = fft_tma_smem_zeval<T, L, LINES>(),
                 sm_za = fft_tma_smem_zadj<T, L, LINES>();
    const int tiles1 = L * ntile;   // tiles of one field in a y or z pass
    auto yz_pass = [&](int buf, int nfields, int axis, int inverse) -> int {
        if (!tma) {
            C* d = buf ? spec : R;
            fft_yz<T, L, LINES><<<dim3(L * ntile, nfields), FFT_THREADS, smem2, str>>>(d, nspec, axis, inverse, st);
            return 0;
        }
        int grid = 0;
        int r = persistent_grid((const void*)fft_yz_tma<T, L, LINES>, FFT_TMA_THREADS, sm_yz, tiles1 * nfields, &grid);
        if (r) return r;
        fft_yz_tma<T, L, LINES><<<grid, FFT_TMA_THREADS, sm_yz, str>>>(p->tmaps[f32][buf][axis - 1], axis, inverse,
                                                                      nfields, st, err);
        return 0;
    };
    fft_x_r2c<T, double, L, LINES><<<dim3(xblocks, nc), FFT_THREADS, smem2, str>>>(S.rho, npts, R, nspec, st);
    if ((rc = yz_pass(0, nc, 1, 0))) return rc;
    if (tma) {
        int grid = 0;
        if ((rc = persistent_grid((const void*)fft_z_eval_tma<T, L, LINES>, FFT_TMA_THREADS, sm_ze, tiles1 * nc, &grid)))
            return rc;
        fft_z_eval_tma<T, L, LINES><<<grid, FFT_TMA_THREADS, sm_ze, str>>>(p->tmaps[f32][0][1], p->tmaps[f32][1][1], K,
                                                                          nc, st, err);
    } else {
        fft_z_eval<T, L, LINES><<<dim3(L * ntile, nc), FFT_THREADS, smem3, str>>>(R, nspec, spec, nspec, K, st);
    }
    if ((rc = yz_pass(1, nc * S.nconv, 1, 1))) return rc;
    // the functional derivative takes the fused x pass (weighted densities, Phi and dPhi/dn
    // stay in shared memory); the free energy needs Phi in global memory: separate kernels
    const bool fused = with_int && g_tuned.fft3d_fused_phi && p->tma_ready;
    g_launches += 4;
    if (fused) {
        rc = (nc == 1) ? launch_fused_nc<T, L, 1>(b, st, spec, nspec, err) : launch_fused_nc<T, L, 2>(b, st, spec, nspec, err);
        if (rc) return rc;
    } else {
        fft_x_c2r<T, L, LINES><<<dim3(xblocks, nc * S.nconv), FFT_THREADS, smem2, str>>>(spec, nspec, part, npts,
                                                                                        T(S.NA / (double)npts), st);
        rc = launch_phi<T>(b, st);
        if (rc) return rc;
        g_launches += 2;
    }
    if (with_int) {
        if (!fused) {
            for (int i = 0; i < nc; ++i)
                fft_x_r2c<T, T, L, LINES><<<dim3(xblocks, S.nconv), FFT_THREADS, smem2, str>>>(
                    dfield + ((size_t)i * S.NF + 1) * npts, npts, spec + (size_t)i * S.nconv * nspec, nspec, st);
            g_launches += nc;
        }
        if ((rc = yz_pass(1, nc * S.nconv, 1, 0))) return rc;
        if (tma) {
            int grid = 0;
            if ((rc = persistent_grid((const void*)fft_z_adjoint_tma<T, L, LINES>, FFT_TMA_THREADS, sm_za, tiles1 * nc,
                                      &grid)))
                return rc;
            fft_z_adjoint_tma<T, L, LINES><<<grid, FFT_TMA_THREADS, sm_za, str>>>(p->tmaps[f32][1][1],
                                                                                 p->tmaps[f32][0][1], K, nc, st, err);
        } else {
            fft_z_adjoint<T, L, LINES><<<dim3(L * ntile, nc), FFT_THREADS, smem3, str>>>(spec, nspec, R, nspec, K, st);
        }
        if ((rc = yz_pass(0, nc, 1, 1))) return rc;
        fft_x_c2r<T, L, LINES><<<dim3(xblocks, nc), FFT_THREADS, smem2, str>>>(R, nspec, adj, npts,
                                                                              T(1.0 / (double)npts), st);
        g_launches += 4;
    }
    CHECK_LAUNCH();
    return 0;
}

template <typename T>
int launch_eval3d(Batch* b, const AAState* st, bool with_int)
{
    switch (b->plans[0]->L3) {
    case 32: return launch_eval3d_L<T, 32>(b, st, with_int);
    case 64: return launch_eval3d_L<T, 64>(b, st, with_int);
    case 128: return launch_eval3d_L<T, 128>(b, st, with_int);
    case 256: return launch_eval3d_L<T, 256>(b, st, with_int);
    default: return set_error(CDFT_E_UNSUPPORTED, "3D grid size %d", b->plans[0]->L3);
    }
}

template <typename T>
int launch_dense_stage(Batch* b, const AAState* st, int stage)
{
    if (g_tuned.radial_dmma == 2) {
        dense_group_kernel<T, 2><<<dim3(b->group_blocks2, b->ngroups), DGRP_WARPS * 32, 0, b->stream>>>(
            b->d_sys, b->d_groups, stage, st);
        g_launches += 1;
        CHECK_LAUNCH();
        return 0;
    }
    if (g_tuned.radial_dmma) {
        dense_group_kernel<T, 1><<<dim3(b->group_blocks, b->ngroups), DGRP_WARPS * 32, 0, b->stream>>>(
            b->d_sys, b->d_groups, stage, st);
        g_launches += 1;
        CHECK_LAUNCH();
        return 0;
    }
    for (int s = 0; s < b->nsys; ++s) {
        const SysDev& S = b->plans[s]->sys;
        const long long rows = (long long)S.nc * S.nconv * S.N;
        const int blocks = (int)((rows * 32 + DENSE_THREADS - 1) / DENSE_THREADS);
        dense1d_kernel<T><<<blocks, DENSE_THREADS, 0, b->stream>>>(b->d_sys, s, stage, st);
        g_launches += 1;
    }
    CHECK_LAUNCH();
    return 0;
}

template <typename T>
int launch_eval_radial(Batch* b, const AAState* st, bool with_int)
{
    int rc = launch_dense_stage<T>(b, st, 0);
    if (rc) return rc;
    rc = launch_phi<T>(b, st);
    if (rc) return rc;
    g_launches += 1;
    if (with_int) rc = launch_dense_stage<T>(b, st, 1);
    return rc;
}

template <typename T>
int launch_eval_stages(Batch* b, const AAState* st, bool with_int)
{
    if (b->nd == 3) return launch_eval3d<T>(b, st, with_int);
    if (b->coord != CDFT_COORD_CART) return launch_eval_radial<T>(b, st, with_int);
    const size_t smem = (size_t)(CONV_QC + CONV_TILE + CONV_QC + 31) * sizeof(T);
    conv1d_kernel<T><<<b->ntasks, CONV_WARPS * 32, smem, b->stream>>>(b->d_tasks, b->d_sys, st, 0);
    int rc = launch_phi<T>(b, st);
    if (rc) return rc;
    g_launches += 2;
    if (with_int) {
        conv1d_kernel<T><<<b->ntasks, CONV_WARPS * 32, smem, b->stream>>>(b->d_tasks, b->d_sys, st, 1);
        g_launches += 1;
    }
    return 0;
}

template <typename T>
int launch_iteration(Batch* b)
{
    int rc = launch_eval_stages<T>(b, b->d_st, true);
    if (rc) return rc;
    el_kernel<T><<<b->nechunks, ELEM_THREADS, 0, b->stream>>>(b->d_echunks, b->d_sys, b->d_st, b->d_partials);
    const int ctl_blocks = b->nsys;
    ctl_kernel<<<ctl_blocks, CTL_THREADS, 0, b->stream>>>(b->d_sys, b->d_st, b->d_partials, b->nsys, 0, b->d_done);
    auto vec = (b->vec_mb <= 8) ? vec_kernel<8> : (b->vec_mb <= 12) ? vec_kernel<12> : vec_kernel<CDFT_MAX_M>;
    for (int slot = 1; slot <= N_VEC_SLOTS; ++slot) {
        vec<<<b->nechunks, ELEM_THREADS, 0, b->stream>>>(b->d_echunks, b->d_sys, b->d_st, b->d_partials, slot);
        if (slot < N_VEC_SLOTS)
            ctl_kernel<<<ctl_blocks, CTL_THREADS, 0, b->stream>>>(b->d_sys, b->d_st, b->d_partials, b->nsys, slot, b->d_done);
    }
    g_launches += 2 * N_VEC_SLOTS + 1;   // el, ctl0, N_VEC_SLOTS vec, N_VEC_SLOTS - 1 ctl (eval stages counted above)
    CHECK_LAUNCH();
    return 0;
}

// Two CTAs per system (a cluster of two, persistent_kernel<..., 2>) when the Anderson vectors
// live in shared memory, the arithmetic is FP64, the pairs fit the device in one wave and the
// tuned entry allows it; otherwise one CTA per system.  Both forms give the same bits.
template <typename T, int NC>
int launch_persistent_nc(Batch* b, int max_evals, size_t smem, int vec_m)
{
    const int dev = b->plans[0]->device;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if constexpr (sizeof(T) == 8) {
        if (g_tuned.pers_cluster && vec_m >= 0 && 2 * b->nsys <= nsm) {
            auto kern2 = persistent_kernel<T, NC, 1, 2>;
            CU(cudaFuncSetAttribute(kern2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(2 * b->nsys);
            cfg.blockDim = dim3(PERS_THREADS);
            cfg.dynamicSmemBytes = smem;
            cfg.stream = b->stream;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = 2;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, kern2, &cfg) == cudaSuccess && nclusters >= b->nsys) {
                CU(cudaLaunchKernelEx(&cfg, kern2, (const SysDev*)b->d_sys, b->d_st, b->d_done, max_evals, vec_m,
                                      g_tuned.pers_warp_aa_max_elem));
                g_launches += 1;
                return 0;
            }
            cudaGetLastError();   // the occupancy query's status, if it failed: fall back to one CTA per system
        }
    }
    auto kern = persistent_kernel<T, NC, 1, 1>;
    CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<b->nsys, PERS_THREADS, smem, b->stream>>>(b->d_sys, b->d_st, b->d_done, max_evals, vec_m,
                                                     g_tuned.pers_warp_aa_max_elem);
    CHECK_LAUNCH();
    g_launches += 1;
    return 0;
}

template <typename T>
int launch_persistent(Batch* b, int max_evals, size_t smem, int vec_m)
{
    switch (b->nc) {
    case 1: return launch_persistent_nc<T, 1>(b, max_evals, smem, vec_m);
    case 2: return launch_persistent_nc<T, 2>(b, max_evals, smem, vec_m);
    case 3: return launch_persistent_nc<T, 3>(b, max_evals, smem, vec_m);
    case 4: return launch_persistent_nc<T, 4>(b, max_evals, smem, vec_m);
    default: return set_error(CDFT_E_UNSUPPORTED, "nc=%d", b->nc);
    }
}

// dynamic shared memory the persistent kernel needs for the largest system of the batch
size_t persistent_smem_need(const Batch* b)
{
    int nmax = 0;
    for (auto* p : b->plans) nmax = std::max(nmax, p->N);
    const SysDev& S = b->plans[0]->sys;
    return pers_smem_bytes(nmax, S.nc, S.nconv, S.NF, b->cur32 ? sizeof(float) : sizeof(double));
}

template <typename T, int NC>
size_t persistent_static_smem()
{
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, persistent_kernel<T, NC, 1, 1>) != cudaSuccess) return 1u << 30;
    size_t stat = a.sharedSizeBytes;
    if (cudaFuncGetAttributes(&a, persistent_kernel<T, NC, 1, 2>) != cudaSuccess) return 1u << 30;
    return std::max(stat, (size_t)a.sharedSizeBytes);
}

size_t persistent_smem_limit(const Batch* b)
{
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->plans[0]->device);
    size_t stat = 0;
    switch ((b->cur32 ? 10 : 0) + b->nc) {
    case 1: stat = persistent_static_smem<double, 1>(); break;
    case 2: stat = persistent_static_smem<double, 2>(); break;
    case 3: stat = persistent_static_smem<double, 3>(); break;
    case 4: stat = persistent_static_smem<double, 4>(); break;
    case 11: stat = persistent_static_smem<float, 1>(); break;
    case 12: stat = persistent_static_smem<float, 2>(); break;
    case 13: stat = persistent_static_smem<float, 3>(); break;
    case 14: stat = persistent_static_smem<float, 4>(); break;
    default: return 0;
    }
    return (size_t)optin > stat ? (size_t)optin - stat : 0;
}

int batch_capture(Batch* b, int iters)
{
    const int g32 = b->cur32;
    if (b->graph[g32] && b->graph_iters[g32] == iters && b->graph_mb[g32] == b->vec_mb &&
        std::memcmp(&b->graph_tuned[g32], &g_tuned, sizeof(TunedShapes)) == 0)
        return 0;
    if (b->graph[g32]) {
        cudaGraphExecDestroy(b->graph[g32]);
        b->graph[g32] = nullptr;
    }
    cudaGraph_t g;
    CU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const long long before = g_launches;
    int rc = 0;
    for (int it = 0; it < iters && !rc; ++it) rc = g32 ? launch_iteration<float>(b) : launch_iteration<double>(b);
    b->graph_launches[g32] = g_launches - before;   // kernel nodes of the graph, counted when it runs
    g_launches = before;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return set_error(CDFT_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph[g32], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_error(CDFT_E_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    b->graph_iters[g32] = iters;
    b->graph_mb[g32] = b->vec_mb;
    b->graph_tuned[g32] = g_tuned;
    return 0;
}

int get_batch(const std::vector<cdft_plan*>& plans, Batch** out)
{
    std::lock_guard<std::mutex> lk(g_batch_mu);
    auto it = g_batches.find(plans);
    if (it != g_batches.end()) {
        *out = it->second;
        return 0;
    }
    Batch* b = nullptr;
    int rc = batch_build(plans, &b);
    if (rc) return rc;
    g_batches[plans] = b;
    *out = b;
    return 0;
}

void drop_batches_of(cdft_plan* p)
{
    std::lock_guard<std::mutex> lk(g_batch_mu);
    for (auto it = g_batches.begin(); it != g_batches.end();) {
        bool hit = false;
        for (auto* q : it->first) hit |= (q == p);
        if (hit) {
            free_batch(it->second);
            it = g_batches.erase(it);
        } else {
            ++it;
        }
    }
}

int validate_opts(const cdft_solver_opts* o)
{
    if (!o) return set_error(CDFT_E_INVALID, "opts is NULL");
    if (o->m < 0 || o->m > CDFT_MAX_M) return set_error(CDFT_E_INVALID, "m=%d out of [0,%d]", o->m, CDFT_MAX_M);
    if (!(std::fabs(o->beta) > 0 && std::fabs(o->beta) <= 1)) return set_error(CDFT_E_INVALID, "abs(beta) must be in (0,1]");
    if (o->maxit < 0 || o->picard_maxit < 0) return set_error(CDFT_E_INVALID, "maxit and picard_maxit must be >= 0");
    return 0;
}

// One aasol run over the batch from the profiles currently in the plans' rho
// buffers, with the arithmetic of b->cur32.  hist_off[s]: history entries already
// written for system s by an earlier phase.
// atol_sys (optional): one absolute tolerance per system, replacing rtol/atol
// (a negative entry keeps rtol/atol for that system).
int run_phase(Batch* b, const cdft_solver_opts* opts, double rtol, double atol, const std::vector<int>& hist_off,
              std::vector<AAState>& st, std::chrono::steady_clock::time_point t0, bool* budget_hit,
              const std::vector<double>* atol_sys = nullptr)
{
    const long long max_evals = (long long)opts->maxit + 2LL * opts->picard_maxit + 4;
    // every state starts zeroed with aasol's options (state_init_kernel); per system the
    // tolerances and its slice of the residual history
    for (int s = 0; s < b->nsys; ++s) {
        AAInit& I = b->h_init[s];
        const bool abs_tol = atol_sys && (*atol_sys)[s] >= 0.0;
        I.rtol = abs_tol ? 0.0 : rtol;
        I.atol = abs_tol ? (*atol_sys)[s] : atol;
        // an FP64 polish of an FP32 result starts with Anderson: the Picard warm-up of
        // aasol targets picard_rtol times the residual of its first iterate, which is
        // already small here, and damped Picard does not reach it
        I.picard_maxit = abs_tol ? 0 : opts->picard_maxit;
        const int off = std::min(hist_off[s], b->hist_cap);
        I.history = b->d_hist + (size_t)s * b->hist_cap + off;
        I.history_cap = b->hist_cap - off;
    }
    const AACommon common{opts->m, opts->maxit, opts->beta, opts->picard_beta, opts->picard_rtol, opts->picard_atol};
    CU(cudaMemcpyAsync(b->d_init, b->h_init, sizeof(AAInit) * b->nsys, cudaMemcpyHostToDevice, b->stream));
    state_init_kernel<<<b->nsys, 128, 0, b->stream>>>(b->d_st, b->d_init, common);
    CHECK_LAUNCH();
    g_launches += 1;
    CU(cudaMemsetAsync(b->d_done, 0, 2 * sizeof(int), b->stream));
    init_kernel<<<b->nechunks, ELEM_THREADS, 0, b->stream>>>(b->d_echunks, b->d_sys);
    CHECK_LAUNCH();
    g_launches += 1;
    bool use_persistent = false;
    if (b->nd == 3 && opts->engine == CDFT_ENGINE_PERSISTENT)
        return set_error(CDFT_E_UNSUPPORTED, "3D systems run on the grid engine");
    if (opts->engine != CDFT_ENGINE_AUTO && opts->engine != CDFT_ENGINE_GRID && opts->engine != CDFT_ENGINE_PERSISTENT)
        return set_error(CDFT_E_INVALID, "engine=%d", opts->engine);
    if (b->coord != CDFT_COORD_CART && opts->engine == CDFT_ENGINE_PERSISTENT)
        return set_error(CDFT_E_UNSUPPORTED, "spherical and cylindrical systems run on the grid engine");
    const bool snapshots = opts->snapshot_every > 0 && opts->snapshot;
    if (snapshots && opts->engine == CDFT_ENGINE_PERSISTENT)
        return set_error(CDFT_E_UNSUPPORTED, "snapshots run on the grid engine (one graph launch per interval)");
    if (!snapshots && b->nd == 1 && b->coord == CDFT_COORD_CART &&
        (opts->engine == CDFT_ENGINE_AUTO || opts->engine == CDFT_ENGINE_PERSISTENT)) {
        const size_t need = persistent_smem_need(b), limit = persistent_smem_limit(b);
        use_persistent = need <= limit && opts->m <= PERS_MAX_M;
        if (!use_persistent && opts->engine == CDFT_ENGINE_PERSISTENT) {
            if (opts->m > PERS_MAX_M)
                return set_error(CDFT_E_UNSUPPORTED, "persistent engine takes Anderson depths m <= %d", PERS_MAX_M);
            return set_error(CDFT_E_UNSUPPORTED, "persistent engine needs %zu B of shared memory per system (limit %zu)",
                             need, limit);
        }
    }
    int rc = 0;
    if (use_persistent) {
        // one launch: every block runs its system's aasol loop to the end (bounded by max_evals);
        // the Anderson vectors join the block's shared memory when they fit
        size_t smem = persistent_smem_need(b);
        int vec_m = -1;
        {
            int nmax = 0;
            for (auto* p : b->plans) nmax = std::max(nmax, p->N);
            const SysDev& S0 = b->plans[0]->sys;
            const size_t with_vec = pers_vec_offset(nmax, S0.nc, S0.nconv, S0.NF, b->cur32 ? sizeof(float) : sizeof(double))
                                    + pers_vec_bytes(nmax * S0.nc, opts->m);
            if (with_vec <= persistent_smem_limit(b)) {
                smem = with_vec;
                vec_m = opts->m;
            }
        }
        const int cap = (int)std::min<long long>(max_evals, 1 << 30);
        rc = b->cur32 ? launch_persistent<float>(b, cap, smem, vec_m) : launch_persistent<double>(b, cap, smem, vec_m);
        if (rc) return rc;
    } else {
        const int K = snapshots ? opts->snapshot_every : (opts->iters_per_launch > 0 ? opts->iters_per_launch : 16);
        // the vector kernel instance whose history bound covers m (8, 12 or CDFT_MAX_M)
        b->vec_mb = (opts->m <= 8) ? 8 : (opts->m <= 12) ? 12 : CDFT_MAX_M;
        rc = batch_capture(b, K);
        if (rc) return rc;
        long long launched_evals = 0;
        while (true) {
            CU(cudaGraphLaunch(b->graph[b->cur32], b->stream));
            g_launches += b->graph_launches[b->cur32];
            launched_evals += K;
            CU(cudaMemcpyAsync(b->h_done, b->d_done, 2 * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
            CU(cudaStreamSynchronize(b->stream));
            if (b->h_done[1])
                return set_error(CDFT_E_CUDA, "a tensor-memory transfer did not complete in time (kernel error %d)",
                                 b->h_done[1]);
            if (snapshots && *b->h_done < b->nsys) {
                // every system still running has made K more evaluations: hand its iterate out
                CU(cudaMemcpyAsync(st.data(), b->d_st, sizeof(AAState) * b->nsys, cudaMemcpyDeviceToHost, b->stream));
                CU(cudaStreamSynchronize(b->stream));
                for (int s = 0; s < b->nsys; ++s) {
                    if (st[s].mode == MODE_DONE) continue;
                    cdft_plan* p = b->plans[s];
                    std::vector<double> h((size_t)p->sys.n_elem);
                    CU(cudaMemcpy(h.data(), p->sys.rho, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
                    opts->snapshot(opts->snapshot_user, s, st[s].nevals + hist_off[s], h.data());
                }
            }
            if (*b->h_done >= b->nsys) break;
            if (launched_evals > max_evals + K) break;   // cannot happen: aasol's caps end every system
            if (opts->time_budget_s > 0) {
                const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                if (el > opts->time_budget_s) {
                    *budget_hit = true;
                    break;
                }
            }
        }
    }
    // the host reads the status fields of the final states (AASummary), not the whole states
    state_summary_kernel<<<(b->nsys + 127) / 128, 128, 0, b->stream>>>(b->d_st, b->d_sum, b->nsys);
    CHECK_LAUNCH();
    g_launches += 1;
    CU(cudaMemcpyAsync(b->h_sum, b->d_sum, sizeof(AASummary) * b->nsys, cudaMemcpyDeviceToHost, b->stream));
    CU(cudaStreamSynchronize(b->stream));
    for (int s = 0; s < b->nsys; ++s) {
        AAState& A = st[s];
        memset(&A, 0, sizeof(A));
        const AASummary& r = b->h_sum[s];
        A.mode = r.mode;
        A.idid = r.idid;
        A.errcode = r.errcode;
        A.k = r.k;
        A.nevals = r.nevals;
        A.resnorm = r.resnorm;
        A.tol = r.tol;
    }
    return 0;
}

// rho pointers: host (is_dev = false) or device arrays of n_elem doubles per system.
// FP64 plans run one aasol.  Mixed plans run aasol with FP32 convolutions and Phi
// until ||r|| <= max(rtol, s) ||r0|| + atol (s = mixed_switch_rtol), then a
// second aasol in FP64 from that profile until the FP64 residual meets the
// stopping test of a plain FP64 run, rtol ||r0|| + atol with r0 the residual
// of the initial profile (taken from the first phase).  A system whose FP32 phase
// diverges (errcode -2, which includes a non-finite evaluation) is converged again
// in FP64 from its initial profile; its evaluation count includes both phases.
int batch_converge(const std::vector<cdft_plan*>& plans, double* const* rho, bool is_dev,
                   const cdft_solver_opts* opts, cdft_result* results)
{
    int rc = validate_opts(opts);
    if (rc) return rc;
    for (size_t s = 0; s < plans.size(); ++s) {
        if (!plans[s]) return set_error(CDFT_E_INVALID, "plan %zu is NULL", s);
        if (!rho || !rho[s]) return set_error(CDFT_E_INVALID, "rho %zu is NULL", s);
    }
    auto t0 = std::chrono::steady_clock::now();
    Batch* b = nullptr;
    rc = get_batch(plans, &b);
    if (rc) return rc;
    b->stream = plans[0]->stream;
    CU(cudaSetDevice(plans[0]->device));
    for (auto* p : plans) {
        rc = plan_alloc_m(p, opts->m);
        if (rc) return rc;
    }
    rc = batch_upload_sys(b);
    if (rc) return rc;
    const long long max_evals = (long long)opts->maxit + 2LL * opts->picard_maxit + 4;
    const int phases = b->mixed ? 2 : 1;
    int hist_cap = (int)std::min<long long>(phases * max_evals, 1 << 20);
    if (b->hist_cap < hist_cap) {
        cudaFree(b->d_hist);
        b->d_hist = nullptr;
        CU(cudaMalloc(&b->d_hist, sizeof(double) * (size_t)hist_cap * b->nsys));
        b->hist_cap = hist_cap;
    }
    // device profiles move in and out by one batch_copy_kernel launch each; host ones by one
    // copy per system
    long long max_elem = 0;
    for (int s = 0; s < b->nsys; ++s) {
        cdft_plan* p = plans[s];
        max_elem = std::max<long long>(max_elem, p->sys.n_elem);
        b->h_copy[s] = CopyTask{rho[s], p->sys.rho, (long long)p->sys.n_elem};
        b->h_copy[b->nsys + s] = CopyTask{p->sys.rho, rho[s], (long long)p->sys.n_elem};
    }
    const dim3 copy_grid((unsigned)std::min<long long>((max_elem + 255) / 256, 64), (unsigned)b->nsys);
    // host profiles of a small batch (at most CDFT_STAGE_MAX_ELEMS doubles in all) go through one
    // pinned staging buffer: one host-to-device copy and the scatter kernel, instead of a
    // pageable copy per system; larger ones (3D grids) are copied directly
    long long total_elem = 0;
    for (auto* p : plans) total_elem += p->sys.n_elem;
    const bool staged = !is_dev && total_elem <= CDFT_STAGE_MAX_ELEMS;
    if (staged && b->stage_elems < total_elem) {
        if (b->h_stage) cudaFreeHost(b->h_stage);
        cudaFree(b->d_stage);
        b->h_stage = nullptr;
        b->d_stage = nullptr;
        b->stage_elems = 0;
        CU(cudaMallocHost(&b->h_stage, sizeof(double) * (size_t)total_elem));
        CU(cudaMalloc(&b->d_stage, sizeof(double) * (size_t)total_elem));
        b->stage_elems = total_elem;
    }
    if (staged) {
        long long off = 0;
        for (int s = 0; s < b->nsys; ++s) {
            const long long ne = plans[s]->sys.n_elem;
            std::memcpy(b->h_stage + off, rho[s], sizeof(double) * (size_t)ne);
            b->h_copy[s].src = b->d_stage + off;
            b->h_copy[b->nsys + s].dst = b->d_stage + off;
            off += ne;
        }
        CU(cudaMemcpyAsync(b->d_stage, b->h_stage, sizeof(double) * (size_t)total_elem, cudaMemcpyHostToDevice,
                           b->stream));
    }
    if (is_dev || staged) {
        CU(cudaMemcpyAsync(b->d_copy, b->h_copy, sizeof(CopyTask) * 2 * b->nsys, cudaMemcpyHostToDevice, b->stream));
        batch_copy_kernel<<<copy_grid, 256, 0, b->stream>>>(b->d_copy);
        CHECK_LAUNCH();
        g_launches += 1;
    } else {
        for (int s = 0; s < b->nsys; ++s) {
            cdft_plan* p = plans[s];
            const size_t bytes = (size_t)p->sys.n_elem * sizeof(double);
            CU(cudaMemcpyAsync(p->sys.rho, rho[s], bytes, cudaMemcpyHostToDevice, b->stream));
        }
    }
    std::vector<AAState> st(b->nsys), st1;
    std::vector<int> hist_off(b->nsys, 0);
    bool budget_hit = false, phase2 = false;
    // 1D Cartesian mixed plans that run on the persistent engine converge in FP64 directly:
    // there the FP32 circulant (FFMA) is no faster than the FP64 tensor-core one, and the
    // FP32 phase only adds evaluations.  The FP32 phase pays on the 3D FFT path.
    bool mixed_fp32 = b->mixed;
    if (b->mixed && b->nd == 1 && b->coord == CDFT_COORD_CART && opts->engine != CDFT_ENGINE_GRID &&
        opts->m <= PERS_MAX_M && !(opts->snapshot_every > 0 && opts->snapshot)) {
        b->cur32 = 0;
        mixed_fp32 = persistent_smem_need(b) > persistent_smem_limit(b);
    }
    if (mixed_fp32) {
        const double sw = opts->mixed_switch_rtol > 0 ? opts->mixed_switch_rtol : 1e-5;
        b->cur32 = 1;
        rc = run_phase(b, opts, std::max(opts->rtol, sw), opts->atol, hist_off, st, t0, &budget_hit);
        if (rc) return rc;
        st1 = st;
        for (int s = 0; s < b->nsys; ++s) hist_off[s] = st1[s].nevals;
        if (!budget_hit) {
            // phase-1 tol = max(rtol, sw) ||r0|| + atol gives back ||r0||
            const double r1 = std::max(opts->rtol, sw);
            std::vector<double> target(b->nsys);
            for (int s = 0; s < b->nsys; ++s) {
                target[s] = opts->rtol * ((st1[s].tol - opts->atol) / r1) + opts->atol;
                if (st1[s].errcode == -2) {
                    // the FP32 phase diverged (residual blow-up or a non-finite evaluation):
                    // this system restarts in FP64 from its initial profile, which the
                    // caller's buffer still holds, under the stopping test of a plain FP64
                    // run (target < 0: rtol ||r0|| + atol with its own r0)
                    target[s] = -1.0;
                    cdft_plan* p = plans[s];
                    const size_t bytes = (size_t)p->sys.n_elem * sizeof(double);
                    CU(cudaMemcpyAsync(p->sys.rho, rho[s], bytes,
                                       is_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->stream));
                }
            }
            b->cur32 = 0;
            phase2 = true;
            rc = run_phase(b, opts, opts->rtol, opts->atol, hist_off, st, t0, &budget_hit, &target);
            b->cur32 = 1;
            if (rc) return rc;
        }
    } else {
        b->cur32 = 0;
        rc = run_phase(b, opts, opts->rtol, opts->atol, hist_off, st, t0, &budget_hit);
        if (rc) return rc;
    }
    if (is_dev || staged) {
        batch_copy_kernel<<<copy_grid, 256, 0, b->stream>>>(b->d_copy + b->nsys);
        CHECK_LAUNCH();
        g_launches += 1;
        if (staged)
            CU(cudaMemcpyAsync(b->h_stage, b->d_stage, sizeof(double) * (size_t)total_elem, cudaMemcpyDeviceToHost,
                               b->stream));
    } else {
        for (int s = 0; s < b->nsys; ++s) {
            cdft_plan* p = plans[s];
            const size_t bytes = (size_t)p->sys.n_elem * sizeof(double);
            CU(cudaMemcpyAsync(rho[s], p->sys.rho, bytes, cudaMemcpyDeviceToHost, b->stream));
        }
    }
    CU(cudaStreamSynchronize(b->stream));
    if (staged) {
        long long off = 0;
        for (int s = 0; s < b->nsys; ++s) {
            const long long ne = plans[s]->sys.n_elem;
            std::memcpy(rho[s], b->h_stage + off, sizeof(double) * (size_t)ne);
            off += ne;
        }
    }
    if (results) {
        for (int s = 0; s < b->nsys; ++s) {
            cdft_result& r = results[s];
            // st holds the last phase that ran; a mixed run counts the evaluations of both
            const AAState& A = st[s];
            const int prev_evals = phase2 ? st1[s].nevals : 0;
            const int prev_k = phase2 ? st1[s].k : 0;
            const bool two = phase2;
            r.idid = A.idid;
            r.errcode = A.errcode;
            r.iterations = two ? prev_k + A.k : A.k;
            r.evaluations = two ? prev_evals + A.nevals : A.nevals;
            r.resnorm = A.resnorm;
            r.tol = A.tol;
            r.history_len = 0;
            if (r.history && r.history_cap > 0) {
                const int n = std::min(std::min(r.evaluations, r.history_cap), b->hist_cap);
                CU(cudaMemcpy(r.history, b->d_hist + (size_t)s * b->hist_cap, sizeof(double) * n, cudaMemcpyDeviceToHost));
                r.history_len = n;
            }
        }
    }
    if (budget_hit) return set_error(CDFT_E_BUDGET, "time budget of %.3f s exhausted", opts->time_budget_s);
    return 0;
}

int self_batch(cdft_plan* p, Batch** b)
{
    std::vector<cdft_plan*> v{p};
    int rc = get_batch(v, b);
    if (rc) return rc;
    (*b)->stream = p->stream;
    return batch_upload_sys(*b);
}

int launch_stage(Batch* b, int stage)
{
    const bool mixed = b->cur32;
    if (b->nd == 3 && stage != 3) return set_error(CDFT_E_UNSUPPORTED, "3D systems time stage 3 only");
    const size_t smem = (size_t)(CONV_QC + CONV_TILE + CONV_QC + 31) * (mixed ? sizeof(float) : sizeof(double));
    if (b->coord != CDFT_COORD_CART && (stage == 0 || stage == 2))
        return mixed ? launch_dense_stage<float>(b, nullptr, stage / 2) : launch_dense_stage<double>(b, nullptr, stage / 2);
    switch (stage) {
    case 0:
    case 2:
        if (mixed)
            conv1d_kernel<float><<<b->ntasks, CONV_WARPS * 32, smem, b->stream>>>(b->d_tasks, b->d_sys, nullptr, stage / 2);
        else
            conv1d_kernel<double><<<b->ntasks, CONV_WARPS * 32, smem, b->stream>>>(b->d_tasks, b->d_sys, nullptr, stage / 2);
        g_launches += 1;
        break;
    case 1: {
        int rc = mixed ? launch_phi<float>(b, nullptr) : launch_phi<double>(b, nullptr);
        if (rc) return rc;
        g_launches += 1;
        break;
    }
    case 3: {
        int rc = mixed ? launch_eval_stages<float>(b, nullptr, true) : launch_eval_stages<double>(b, nullptr, true);
        if (rc) return rc;
        if (mixed)
            dfdrho_out_kernel<float><<<b->nechunks, ELEM_THREADS, 0, b->stream>>>(b->d_echunks, b->d_sys);
        else
            dfdrho_out_kernel<double><<<b->nechunks, ELEM_THREADS, 0, b->stream>>>(b->d_echunks, b->d_sys);
        g_launches += 1;
        break;
    }
    default:
        return set_error(CDFT_E_INVALID, "stage %d", stage);
    }
    CHECK_LAUNCH();
    return 0;
}

// the kernel error word of a batch (d_done[1]): cleared before a stand-alone evaluation and
// checked after it (the converge loop checks it with every poll)
int clear_kernel_error(Batch* b)
{
    CU(cudaMemsetAsync(b->d_done + 1, 0, sizeof(int), b->stream));
    return 0;
}

int check_kernel_error(Batch* b)
{
    int e = 0;
    CU(cudaMemcpyAsync(&e, b->d_done + 1, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    CU(cudaStreamSynchronize(b->stream));
    if (e) return set_error(CDFT_E_CUDA, "a tensor-memory transfer did not complete in time (kernel error %d)", e);
    return 0;
}

int functional_derivative(cdft_plan* p, const double* rho, double* out, bool is_dev)
{
    if (!p || !rho || !out) return set_error(CDFT_E_INVALID, "NULL argument");
    CU(cudaSetDevice(p->device));
    Batch* b = nullptr;
    int rc = self_batch(p, &b);
    if (rc) return rc;
    const size_t bytes = (size_t)p->sys.n_elem * sizeof(double);
    CU(cudaMemcpyAsync(p->sys.rho, rho, bytes, is_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, p->stream));
    if ((rc = clear_kernel_error(b))) return rc;
    rc = p->sys.mixed ? launch_eval_stages<float>(b, nullptr, true) : launch_eval_stages<double>(b, nullptr, true);
    if (rc) return rc;
    if (p->sys.mixed)
        dfdrho_out_kernel<float><<<b->nechunks, ELEM_THREADS, 0, p->stream>>>(b->d_echunks, b->d_sys);
    else
        dfdrho_out_kernel<double><<<b->nechunks, ELEM_THREADS, 0, p->stream>>>(b->d_echunks, b->d_sys);
    CHECK_LAUNCH();
    g_launches += 1;
    CU(cudaMemcpyAsync(out, p->sys.out, bytes, is_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, p->stream));
    CU(cudaStreamSynchronize(p->stream));
    return check_kernel_error(b);
}

// compensated (Neumaier) sum
struct KSum {
    double s = 0, c = 0;
    void add(double x)
    {
        const double t = s + x;
        if (std::fabs(s) >= std::fabs(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    double value() const { return s + c; }
};

// DDFT taps of one axis: the real inverse DFT of the one-axis maps of ddft_rhs_log!
// (ext/SciMLBasecDFTExt.jl:17-19), 2 pi i k and -(2 pi)^2 k^2 with k = m / B, m the fftfreq
// integers and B the reduced box length.  Angles by exact integer reduction of m q mod n;
// the points where sin or cos is exactly 0 or +-1 are set exactly (the Nyquist bin of the
// gradient then drops out, as the real part of the reference's inverse transform drops it).
void ddft_axis_taps(int n, double B, double* tg, double* tl)
{
    const double two_pi = 6.283185307179586476925286766559;
    for (int q = 0; q < n; ++q) {
        KSum sg, sl;
        for (int idx = 0; idx < n; ++idx) {
            const long long m = idx < (n + 1) / 2 ? idx : idx - n;
            long long r = (m * q) % n;
            if (r < 0) r += n;
            double sn, cs;
            if (r == 0) { sn = 0.0; cs = 1.0; }
            else if (2 * r == n) { sn = 0.0; cs = -1.0; }
            else if (4 * r == n) { sn = 1.0; cs = 0.0; }
            else if (4 * r == 3 * (long long)n) { sn = -1.0; cs = 0.0; }
            else {
                const double th = two_pi * double(r) / double(n);
                sn = std::sin(th);
                cs = std::cos(th);
            }
            sg.add(double(m) * sn);
            sl.add(double(m) * double(m) * cs);
        }
        tg[q] = -(two_pi / (double(n) * B)) * sg.value();
        tl[q] = -(two_pi * two_pi / (double(n) * B * B)) * sl.value();
    }
}

int ddft_rhs(cdft_plan* p, const double* eta, double* deta, bool is_dev)
{
    if (!p || !eta || !deta) return set_error(CDFT_E_INVALID, "NULL argument");
    const cdft_system_desc& d = p->desc;
    if (d.coord != CDFT_COORD_CART)
        return set_error(CDFT_E_UNSUPPORTED, "the DDFT right-hand side is defined on Cartesian grids");
    const int nd = d.nd;
    int len[3] = {1, 1, 1};
    for (int k = 0; k < nd; ++k) len[k] = d.ngrid[k];
    int maxlen = 0;
    for (int k = 0; k < nd; ++k) maxlen = std::max(maxlen, len[k]);
    const size_t smem = 2 * (size_t)maxlen * sizeof(double);
    if (smem > 200 * 1024) return set_error(CDFT_E_UNSUPPORTED, "DDFT axis of %d points (at most 12800)", maxlen);
    CU(cudaSetDevice(p->device));
    const size_t ne = (size_t)p->sys.n_elem;
    if (!p->d_ddft) {
        size_t ntap = 0;
        for (int k = 0; k < nd; ++k) ntap += 2 * (size_t)len[k];
        std::vector<double> taps(ntap);
        size_t off = 0;
        for (int k = 0; k < nd; ++k) {
            const double B = (d.bounds[k][1] - d.bounds[k][0]) / d.L;
            ddft_axis_taps(len[k], B, taps.data() + off, taps.data() + off + len[k]);
            off += 2 * (size_t)len[k];
        }
        CU(cudaMalloc(&p->d_ddft, (ntap + 2 * ne) * sizeof(double)));
        CU(cudaMemcpy(p->d_ddft, taps.data(), ntap * sizeof(double), cudaMemcpyHostToDevice));
        p->ddft_eta = ntap;
        CU(cudaFuncSetAttribute(ddft_axis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    }
    double* d_eta = p->d_ddft + p->ddft_eta;
    double* d_out = is_dev ? deta : d_eta + ne;
    Batch* b = nullptr;
    int rc = self_batch(p, &b);
    if (rc) return rc;
    CU(cudaMemcpyAsync(d_eta, eta, ne * sizeof(double), is_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                       p->stream));
    ddft_prep_kernel<<<std::min<size_t>((ne + 255) / 256, 4096), 256, 0, p->stream>>>(d_eta, p->sys.rho, ne);
    CHECK_LAUNCH();
    if ((rc = clear_kernel_error(b))) return rc;
    rc = p->sys.mixed ? launch_eval_stages<float>(b, nullptr, true) : launch_eval_stages<double>(b, nullptr, true);
    if (rc) return rc;
    if (p->sys.mixed)
        dfdrho_out_kernel<float><<<b->nechunks, ELEM_THREADS, 0, p->stream>>>(b->d_echunks, b->d_sys);
    else
        dfdrho_out_kernel<double><<<b->nechunks, ELEM_THREADS, 0, p->stream>>>(b->d_echunks, b->d_sys);
    CHECK_LAUNCH();
    // mu = dF/drho_res + V_ext is in sys.out; the axes in x, y, z order, grid [comp][z][y][x]
    size_t off = 0;
    long long stride = 1;
    for (int k = 0; k < nd; ++k) {
        const long long inner = stride;
        const long long nlines = (long long)(ne / len[k]);
        dim3 grid((unsigned)nlines, (unsigned)((len[k] + DDFT_THREADS - 1) / DDFT_THREADS));
        ddft_axis_kernel<<<grid, DDFT_THREADS, 2 * (size_t)len[k] * sizeof(double), p->stream>>>(
            d_eta, p->sys.out, d_out, p->d_ddft + off, p->d_ddft + off + len[k], len[k], stride, inner, nlines,
            k == 0 ? 1 : 0);
        CHECK_LAUNCH();
        off += 2 * (size_t)len[k];
        stride *= len[k];
    }
    g_launches += 2 + nd;
    if (!is_dev) CU(cudaMemcpyAsync(deta, d_out, ne * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    CU(cudaStreamSynchronize(p->stream));
    return check_kernel_error(b);
}


}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
// per-point terms of the parameter gradient of F_res (cdft_free_energy_res_grad)
template <int NC>
int launch_grad_points(cdft_plan* p, Batch* b, const double* dn, double* gp, double* kt)
{
    if (p->desc.nd == 3)
        grad_points_kernel<NC, 3><<<(p->N + 127) / 128, 128, 0, p->stream>>>(b->d_sys, dn, gp, kt);
    else
        grad_points_kernel<NC, 1><<<(p->N + 127) / 128, 128, 0, p->stream>>>(b->d_sys, dn, gp, kt);
    CHECK_LAUNCH();
    return 0;
}

extern "C" {

int cdft_plan_create(const cdft_system_desc* desc, cdft_plan** plan)
{
    g_err_code = 0;
    if (!plan) return set_error(CDFT_E_INVALID, "plan output pointer is NULL");
    *plan = nullptr;
    int rc = validate_desc(desc);
    if (rc) return rc;
    int dev = 0;
    CU(cudaGetDevice(&dev));
    rc = upload_constants();
    if (rc) return rc;
    cdft_plan* p = new cdft_plan();
    p->device = dev;
    p->desc = *desc;
    p->desc.vext = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete p;
        return set_error(CDFT_E_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    p->stream = p->own_stream;
    cdft_system_desc tmp = *desc;
    p->desc = tmp;
    rc = plan_build(p);
    p->desc.vext = nullptr;
    if (rc) {
        plan_free(p);
        delete p;
        return rc;
    }
    *plan = p;
    return 0;
}

int cdft_plan_destroy(cdft_plan* plan)
{
    if (!plan) return 0;
    cudaSetDevice(plan->device);
    drop_batches_of(plan);
    plan_free(plan);
    delete plan;
    return 0;
}

int cdft_functional_derivative(cdft_plan* plan, const double* rho, double* dFdrho)
{
    g_err_code = 0;
    return functional_derivative(plan, rho, dFdrho, false);
}

int cdft_functional_derivative_dev(cdft_plan* plan, const double* d_rho, double* d_dFdrho)
{
    g_err_code = 0;
    return functional_derivative(plan, d_rho, d_dFdrho, true);
}

}  // extern "C"

// The bulk model of desc's components at temperature T with hard-sphere diameters hsd (m).
static int bulk_model_at(const cdft_system_desc& d, double T, const double* hsd, BulkModel& M)
{
    M = BulkModel{};
    M.nc = d.nc;
    M.T = T;
    for (int i = 0; i < d.nc; ++i) {
        if (!(d.m[i] > 0) || !(hsd[i] > 0)) return set_error(CDFT_E_INVALID, "component %d: m and hsd", i);
        M.m[i] = d.m[i];
        M.d[i] = hsd[i];
        for (int j = 0; j < d.nc; ++j) {
            const double sg = d.sigma[i * d.nc + j];
            M.s3[i * CDFT_MAX_NC + j] = sg * sg * sg;
            M.eT[i * CDFT_MAX_NC + j] = d.eps[i * d.nc + j] / T;
        }
    }
    for (int q = 0; q < d.n_assoc; ++q) {   // the closed form covers 2B self-association
        const cdft_assoc_pair& a = d.assoc[q];
        if (a.icomp != a.jcomp || a.isite == a.jsite || a.n_ia != 1 || a.n_jb != 1 || a.icomp < 0 || a.icomp >= d.nc ||
            M.aK[a.icomp] != 0.0)
            return set_error(CDFT_E_UNSUPPORTED, "device bulk densities cover 2B self-association only");
        const double sg = d.sigma[a.icomp * d.nc + a.icomp];
        M.aK[a.icomp] = sg * sg * sg * a.kappa_ab * (exp(a.eps_ab / T) - 1.0);
    }
    return 0;
}

extern "C" {

int cdft_bulk_density(const cdft_system_desc* desc, int n, const double* p, const double* x, int phase,
                      double* rho, int* status)
{
    g_err_code = 0;
    if (!desc || n < 0 || (n > 0 && (!p || !x || !rho || !status))) return set_error(CDFT_E_INVALID, "invalid argument");
    if (phase < 0 || phase > 2) return set_error(CDFT_E_INVALID, "phase=%d (0 stable, 1 liquid, 2 vapour)", phase);
    const cdft_system_desc& d = *desc;
    if (d.nc < 1 || d.nc > CDFT_MAX_NC || !(d.T > 0)) return set_error(CDFT_E_INVALID, "nc and T");
    if (n == 0) return 0;
    BulkModel M{};
    int rc = bulk_model_at(d, d.T, d.hsd, M);
    if (rc) return rc;
    double* dbuf = nullptr;
    const size_t nb = (size_t)n * (2 + d.nc) * sizeof(double) + (size_t)n * sizeof(int);
    CU(cudaMalloc(&dbuf, nb));
    double* dp = dbuf;
    double* dx = dp + n;
    double* dr = dx + (size_t)n * d.nc;
    int* ds = reinterpret_cast<int*>(dr + n);
    cudaError_t e = cudaMemcpy(dp, p, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dx, x, (size_t)n * d.nc * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        bulk_density_kernel<<<n, 32>>>(M, n, dp, dx, phase, dr, ds);
        e = cudaGetLastError();
        g_launches += 1;
    }
    if (e == cudaSuccess) e = cudaMemcpy(rho, dr, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(status, ds, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(dbuf);
    if (e != cudaSuccess) return set_error(CDFT_E_CUDA, "bulk densities: %s", cudaGetErrorString(e));
    return 0;
}

int cdft_saturation_pure(const cdft_system_desc* desc, int n, const double* T, double* p_sat, double* rho_liquid,
                         double* rho_vapour, int* status)
{
    g_err_code = 0;
    if (!desc || n < 0 || (n > 0 && (!T || !p_sat || !rho_liquid || !rho_vapour || !status)))
        return set_error(CDFT_E_INVALID, "invalid argument");
    const cdft_system_desc& d = *desc;
    if (d.nc != 1) return set_error(CDFT_E_UNSUPPORTED, "saturation of a pure component: nc=%d", d.nc);
    if (n == 0) return 0;
    std::vector<BulkModel> M(n);
    for (int s = 0; s < n; ++s) {
        if (!(T[s] > 0)) return set_error(CDFT_E_INVALID, "T[%d]=%g", s, T[s]);
        // PC-SAFT's temperature-dependent diameter d = sigma (1 - 0.12 exp(-3 eps / T))
        const double hsd = d.sigma[0] * (1.0 - 0.12 * exp(-3.0 * d.eps[0] / T[s]));
        const int rc = bulk_model_at(d, T[s], &hsd, M[s]);
        if (rc) return rc;
    }
    BulkModel* dm = nullptr;
    double* dbuf = nullptr;
    CU(cudaMalloc(&dm, sizeof(BulkModel) * n));
    cudaError_t e = cudaMalloc(&dbuf, (size_t)n * (3 * sizeof(double) + sizeof(int)));
    double* dp = dbuf;
    double* dl = dp + n;
    double* dv = dl + n;
    int* ds = reinterpret_cast<int*>(dv + n);
    if (e == cudaSuccess) e = cudaMemcpy(dm, M.data(), sizeof(BulkModel) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        saturation_kernel<<<n, 32>>>(dm, n, 1e3, dp, dl, dv, ds);
        e = cudaGetLastError();
        g_launches += 1;
    }
    if (e == cudaSuccess) e = cudaMemcpy(p_sat, dp, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(rho_liquid, dl, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(rho_vapour, dv, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(status, ds, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(dm);
    cudaFree(dbuf);
    if (e != cudaSuccess) return set_error(CDFT_E_CUDA, "saturation: %s", cudaGetErrorString(e));
    return 0;
}

int cdft_ddft_rhs(cdft_plan* plan, const double* eta, double* deta)
{
    g_err_code = 0;
    return ddft_rhs(plan, eta, deta, false);
}

int cdft_ddft_rhs_dev(cdft_plan* plan, const double* d_eta, double* d_deta)
{
    g_err_code = 0;
    return ddft_rhs(plan, d_eta, d_deta, true);
}

int cdft_phi_field(cdft_plan* plan, const double* rho, double* fval)
{
    g_err_code = 0;
    if (!plan || !rho || !fval) return set_error(CDFT_E_INVALID, "NULL argument");
    CU(cudaSetDevice(plan->device));
    Batch* b = nullptr;
    int rc = self_batch(plan, &b);
    if (rc) return rc;
    CU(cudaMemcpyAsync(plan->sys.rho, rho, (size_t)plan->sys.n_elem * sizeof(double), cudaMemcpyHostToDevice,
                       plan->stream));
    if ((rc = clear_kernel_error(b))) return rc;
    rc = launch_eval_stages<double>(b, nullptr, false);
    if (rc) return rc;
    CU(cudaMemcpyAsync(fval, plan->sys.fval, sizeof(double) * plan->N, cudaMemcpyDeviceToHost, plan->stream));
    CU(cudaStreamSynchronize(plan->stream));
    return check_kernel_error(b);
}

int cdft_free_energy_res(cdft_plan* plan, const double* rho, double* F)
{
    g_err_code = 0;
    if (!plan || !rho || !F) return set_error(CDFT_E_INVALID, "NULL argument");
    CU(cudaSetDevice(plan->device));
    Batch* b = nullptr;
    int rc = self_batch(plan, &b);
    if (rc) return rc;
    const size_t bytes = (size_t)plan->sys.n_elem * sizeof(double);
    CU(cudaMemcpyAsync(plan->sys.rho, rho, bytes, cudaMemcpyHostToDevice, plan->stream));
    if ((rc = clear_kernel_error(b))) return rc;
    // the free-energy integral is FP64 in every precision mode
    rc = launch_eval_stages<double>(b, nullptr, false);
    if (rc) return rc;
    if ((rc = check_kernel_error(b))) return rc;
    std::vector<double> f(plan->N);
    CU(cudaMemcpyAsync(f.data(), plan->sys.fval, sizeof(double) * plan->N, cudaMemcpyDeviceToHost, plan->stream));
    CU(cudaStreamSynchronize(plan->stream));
    // Simpson coefficients of _∫ (integrals.jl:28-41): 1, 4, 2, 4, ..., 1 per dimension (outer
    // product in nD), times prod(dz/3); compensated summation
    auto coef = [](int k, int n) { return (k == 1 || k == n) ? 1.0 : ((k % 2 == 0) ? 4.0 : 2.0); };
    KSum acc;
    const double L = plan->desc.L;
    if (plan->desc.coord != CDFT_COORD_CART) {   // 4 pi / 2 pi integrateR (integrals.jl:18-19)
        for (int k = 0; k < plan->N; ++k) acc.add(plan->rw[k] * f[k]);
        *F = acc.value() / (L * L * L);
    } else if (plan->desc.nd == 1) {
        const int N = plan->N;
        for (int k = 1; k <= N; ++k) acc.add(coef(k, N) * f[k - 1]);
        *F = acc.value() * (plan->dz[0] / 3.0) / (L * L * L);
    } else {
        const int n = plan->L3;
        for (int z = 1; z <= n; ++z)
            for (int y = 1; y <= n; ++y) {
                const double cyz = coef(z, n) * coef(y, n);
                for (int x = 1; x <= n; ++x)
                    acc.add(cyz * coef(x, n) * f[((size_t)(z - 1) * n + (y - 1)) * n + (x - 1)]);
            }
        *F = acc.value() * (plan->dz[0] / 3.0) * (plan->dz[1] / 3.0) * (plan->dz[2] / 3.0) / (L * L * L);
    }
    return 0;
}

int cdft_phi_pointwise(cdft_plan* plan, const double* n, int npts, double* fval, double* dphi)
{
    g_err_code = 0;
    if (!plan || !n || !fval || !dphi || npts <= 0) return set_error(CDFT_E_INVALID, "invalid argument");
    CU(cudaSetDevice(plan->device));
    const int nc = plan->desc.nc, NF = plan->sys.NF;
    const size_t nin = (size_t)npts * NF * nc;
    double *d_n = nullptr, *d_f = nullptr, *d_g = nullptr;
    CU(cudaMalloc(&d_n, nin * sizeof(double)));
    CU(cudaMalloc(&d_f, (size_t)npts * sizeof(double)));
    CU(cudaMalloc(&d_g, nin * sizeof(double)));
    CU(cudaMemcpyAsync(d_n, n, nin * sizeof(double), cudaMemcpyHostToDevice, plan->stream));
    const int blocks = (npts + 127) / 128;
    const PhiParams& P = plan->sys.phi;
    int rc = 0;
    if (plan->desc.nd == 1) {
        switch (nc) {
        case 1: phi_points_kernel<1, 1><<<blocks, 128, 0, plan->stream>>>(P, d_n, npts, d_f, d_g); break;
        case 2: phi_points_kernel<2, 1><<<blocks, 128, 0, plan->stream>>>(P, d_n, npts, d_f, d_g); break;
        case 3: phi_points_kernel<3, 1><<<blocks, 128, 0, plan->stream>>>(P, d_n, npts, d_f, d_g); break;
        case 4: phi_points_kernel<4, 1><<<blocks, 128, 0, plan->stream>>>(P, d_n, npts, d_f, d_g); break;
        default: rc = set_error(CDFT_E_UNSUPPORTED, "nc");
        }
    } else if (plan->desc.nd == 3 && nc <= 2) {
        if (nc == 1) phi_points_kernel<1, 3><<<blocks, 128, 0, plan->stream>>>(P, d_n, npts, d_f, d_g);
        else phi_points_kernel<2, 3><<<blocks, 128, 0, plan->stream>>>(P, d_n, npts, d_f, d_g);
    } else {
        rc = set_error(CDFT_E_UNSUPPORTED, "nd");
    }
    g_launches += 1;
    cudaError_t e = cudaGetLastError();
    if (!rc && e != cudaSuccess) rc = set_error(CDFT_E_CUDA, "phi_points_kernel: %s", cudaGetErrorString(e));
    if (!rc) {
        cudaMemcpyAsync(fval, d_f, (size_t)npts * sizeof(double), cudaMemcpyDeviceToHost, plan->stream);
        cudaMemcpyAsync(dphi, d_g, nin * sizeof(double), cudaMemcpyDeviceToHost, plan->stream);
        e = cudaStreamSynchronize(plan->stream);
        if (e != cudaSuccess) rc = set_error(CDFT_E_CUDA, "phi_pointwise: %s", cudaGetErrorString(e));
    }
    cudaFree(d_n);
    cudaFree(d_f);
    cudaFree(d_g);
    return rc;
}

int cdft_converge(cdft_plan* plan, double* rho_inout, const cdft_solver_opts* opts, cdft_result* result)
{
    g_err_code = 0;
    std::vector<cdft_plan*> v{plan};
    double* r[1] = {rho_inout};
    return batch_converge(v, r, false, opts, result);
}

int cdft_converge_dev(cdft_plan* plan, double* d_rho_inout, const cdft_solver_opts* opts, cdft_result* result)
{
    g_err_code = 0;
    std::vector<cdft_plan*> v{plan};
    double* r[1] = {d_rho_inout};
    return batch_converge(v, r, true, opts, result);
}

int cdft_batch_converge(cdft_plan* const* plans, int nplans, double* const* rho_inout,
                        const cdft_solver_opts* opts, cdft_result* results)
{
    g_err_code = 0;
    if (!plans || nplans <= 0) return set_error(CDFT_E_INVALID, "no plans");
    std::vector<cdft_plan*> v(plans, plans + nplans);
    return batch_converge(v, rho_inout, false, opts, results);
}

int cdft_batch_converge_dev(cdft_plan* const* plans, int nplans, double* const* d_rho_inout,
                            const cdft_solver_opts* opts, cdft_result* results)
{
    g_err_code = 0;
    if (!plans || nplans <= 0) return set_error(CDFT_E_INVALID, "no plans");
    std::vector<cdft_plan*> v(plans, plans + nplans);
    return batch_converge(v, d_rho_inout, true, opts, results);
}

int cdft_plan_set_stream(cdft_plan* plan, void* stream)
{
    g_err_code = 0;
    if (!plan) return set_error(CDFT_E_INVALID, "plan is NULL");
    CU(cudaSetDevice(plan->device));
    CU(cudaStreamSynchronize(plan->stream));
    plan->stream = stream ? (cudaStream_t)stream : plan->own_stream;
    return 0;
}

int cdft_batch_time_stage(cdft_plan* const* plans, int nplans, int stage, int reps, double* ms_per_launch)
{
    g_err_code = 0;
    if (!plans || nplans <= 0 || reps <= 0 || !ms_per_launch) return set_error(CDFT_E_INVALID, "invalid argument");
    std::vector<cdft_plan*> v(plans, plans + nplans);
    Batch* b = nullptr;
    int rc = get_batch(v, &b);
    if (rc) return rc;
    b->stream = v[0]->stream;
    CU(cudaSetDevice(v[0]->device));
    rc = batch_upload_sys(b);
    if (rc) return rc;
    for (int w = 0; w < 3 && !rc; ++w) rc = launch_stage(b, stage);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    CU(cudaEventRecord(e0, b->stream));
    for (int r = 0; r < reps && !rc; ++r) rc = launch_stage(b, stage);
    CU(cudaEventRecord(e1, b->stream));
    CU(cudaEventSynchronize(e1));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    *ms_per_launch = (double)ms / reps;
    return 0;
}

int cdft_batch_integrals(cdft_plan* const* plans, int nplans, double* const* rho, int rho_on_device, double* out)
{
    g_err_code = 0;
    if (!plans || nplans <= 0 || !out) return set_error(CDFT_E_INVALID, "invalid argument");
    std::vector<cdft_plan*> v(plans, plans + nplans);
    for (int s = 0; s < nplans; ++s)
        if (!v[s]) return set_error(CDFT_E_INVALID, "plan %d is NULL", s);
    Batch* b = nullptr;
    int rc = get_batch(v, &b);
    if (rc) return rc;
    b->stream = v[0]->stream;
    CU(cudaSetDevice(v[0]->device));
    rc = batch_upload_sys(b);
    if (rc) return rc;
    if (rho)
        for (int s = 0; s < nplans; ++s) {
            if (!rho[s]) return set_error(CDFT_E_INVALID, "rho %d is NULL", s);
            CU(cudaMemcpyAsync(v[s]->sys.rho, rho[s], (size_t)v[s]->sys.n_elem * sizeof(double),
                               rho_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->stream));
        }
    if ((rc = clear_kernel_error(b))) return rc;
    rc = launch_eval_stages<double>(b, nullptr, false);   // weighted densities and Phi, FP64
    if (rc) return rc;
    const int nq = 3 + b->nc;
    int maxn = 1;
    for (int s = 0; s < nplans; ++s) maxn = std::max(maxn, v[s]->sys.N);
    const int nchunk = (maxn + INTEG_CHUNK - 1) / INTEG_CHUNK;
    double* d_out = nullptr;
    CU(cudaMalloc(&d_out, sizeof(double) * nq * nplans * (1 + 2 * (size_t)nchunk)));
    double* d_part = d_out + (size_t)nq * nplans;
    integrals_kernel<<<dim3(nchunk, nplans), INTEG_THREADS, 0, b->stream>>>(b->d_sys, v[0]->desc.T, d_part, nchunk);
    integrals_reduce_kernel<<<nplans, 32, 0, b->stream>>>(d_part, nchunk, nq, d_out);
    g_launches += 2;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, sizeof(double) * nq * nplans, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    cudaFree(d_out);
    if (e != cudaSuccess) return set_error(CDFT_E_CUDA, "batch integrals: %s", cudaGetErrorString(e));
    for (int s = 0; s < nplans; ++s) {   // F_res in k_B T per unit area (1D) or total (3D, radial)
        const double L = v[s]->desc.L;
        out[(size_t)s * nq] /= L * L * L;
    }
    return check_kernel_error(b);
}

long long cdft_launch_count(int reset)
{
    const long long v = g_launches;
    if (reset) g_launches = 0;
    return v;
}

int cdft_last_error(char* buf, size_t len)
{
    if (buf && len) {
        strncpy(buf, g_err_msg, len - 1);
        buf[len - 1] = 0;
    }
    return g_err_code;
}

const char* cdft_version(void) { return "cdft_b200 0.2 (sm_100a)"; }

int cdft_tuning_get(const char* name, int* value)
{
    g_err_code = 0;
    const TunedEntry* e = tuned_entry(name);
    if (!e || !value) return set_error(CDFT_E_INVALID, "unknown tuning entry %s", name ? name : "(null)");
    *value = g_tuned.*(e->field);
    return 0;
}

int cdft_tuning_set(const char* name, int value)
{
    g_err_code = 0;
    const TunedEntry* e = tuned_entry(name);
    if (!e) return set_error(CDFT_E_INVALID, "unknown tuning entry %s", name ? name : "(null)");
    if (value < e->lo || value > e->hi) return set_error(CDFT_E_INVALID, "%s=%d out of [%d, %d]", name, value, e->lo, e->hi);
    g_tuned.*(e->field) = value;
    return 0;
}

// ---------------------------------------------------------------------------
// Parameter gradient of F_res and of the excess grand potential (1D)
// ---------------------------------------------------------------------------
// uniform = false: the Simpson weights of F_res (integrals.jl:28-41); true: the uniform
// weights dz of the discrete functional whose gradient the pointwise Euler-Lagrange equation
// of converge! is (what cdft_grad_params differentiates)
static int fres_grad_impl(cdft_plan* plan, const double* rho, double* dF, bool uniform);
static int fres_grad_chain(cdft_plan* plan, const std::vector<double>& G, const std::vector<double>& Gd, double* dF);
static int fres_grad3d(cdft_plan* plan, Batch* b, bool uniform, int NP, double* dF);

int cdft_free_energy_res_grad(cdft_plan* plan, const double* rho, double* dF)
{
    g_err_code = 0;
    return fres_grad_impl(plan, rho, dF, false);
}

static int fres_grad_impl(cdft_plan* plan, const double* rho, double* dF, bool uniform)
{
    if (!plan || !rho || !dF) return set_error(CDFT_E_INVALID, "NULL argument");
    const cdft_system_desc& d = plan->desc;
    if (d.coord != CDFT_COORD_CART || (d.nd != 1 && d.nd != 3))
        return set_error(CDFT_E_UNSUPPORTED, "the parameter gradient is implemented for 1D and 3D Cartesian grids");
    if (d.n_assoc > 1)
        return set_error(CDFT_E_UNSUPPORTED, "the parameter gradient covers one association pair");
    const int nc = d.nc, N = plan->N;
    const double L = d.L, T = d.T;
    // the chain below assumes PC-SAFT's diameter d_i = sigma_i (1 - 0.12 exp(-3 eps_i / T)) and the
    // combining rule sigma_ij = (sigma_i + sigma_j) / 2 (eps_ij = sqrt(eps_i eps_j)(1 - k_ij), any k_ij)
    for (int i = 0; i < nc; ++i) {
        const double si = d.sigma[i * nc + i], ei = d.eps[i * nc + i];
        const double dd = si * (1.0 - 0.12 * exp(-3.0 * ei / T));
        if (fabs(dd / d.hsd[i] - 1.0) > 1e-9)
            return set_error(CDFT_E_UNSUPPORTED, "hsd[%d] is not the PC-SAFT diameter of sigma and eps", i);
        for (int j = 0; j < nc; ++j)
            if (fabs(d.sigma[i * nc + j] / (0.5 * (si + d.sigma[j * nc + j])) - 1.0) > 1e-12)
                return set_error(CDFT_E_UNSUPPORTED, "sigma[%d,%d] does not follow (sigma_i + sigma_j) / 2", i, j);
    }
    CU(cudaSetDevice(plan->device));
    Batch* b = nullptr;
    int rc = self_batch(plan, &b);
    if (rc) return rc;
    SysDev& S = plan->sys;
    const int nconv = S.nconv;
    const size_t ne = (size_t)S.n_elem;
    CU(cudaMemcpyAsync(S.rho, rho, ne * sizeof(double), cudaMemcpyHostToDevice, plan->stream));
    const int NP = 2 * nc + 2 * nc * nc + 2;
    if (d.nd == 3) return fres_grad3d(plan, b, uniform, NP, dF);
    // weighted densities (FP64 in every precision mode)
    {
        const size_t smem = (size_t)(CONV_QC + CONV_TILE + CONV_QC + 31) * sizeof(double);
        conv1d_kernel<double><<<b->ntasks, CONV_WARPS * 32, smem, plan->stream>>>(b->d_tasks, b->d_sys, nullptr, 0);
        CHECK_LAUNCH();
    }
    const double wf[6] = {0.5, 0.5, 0.5, 1.0, 1.0, PSI_DISP};
    double *d_dt = nullptr, *d_dn = nullptr, *d_gp = nullptr, *d_kt = nullptr, *d_scale = nullptr;
    const size_t ntap = (size_t)nc * nconv * N;
    CU(cudaMalloc(&d_dt, ntap * sizeof(double)));
    CU(cudaMalloc(&d_dn, ntap * sizeof(double)));
    CU(cudaMalloc(&d_gp, (size_t)NP * N * sizeof(double)));
    CU(cudaMalloc(&d_kt, (size_t)nc * N * sizeof(double)));
    CU(cudaMalloc(&d_scale, nconv * sizeof(double)));
    double scale[6];
    for (int f = 0; f < nconv; ++f) scale[f] = S.NA * 2.0 * 3.14159265358979323846 * wf[f];   // N_A L^3 dR/dd
    CU(cudaMemcpyAsync(d_scale, scale, nconv * sizeof(double), cudaMemcpyHostToDevice, plan->stream));
    const double span = d.bounds[0][1] - d.bounds[0][0];
    rc = launch_taps(plan->stream, N, span, L, nc, S.phi.d, d_dt, true);
    if (rc) {
        cudaFree(d_dt);
        cudaFree(d_dn);
        cudaFree(d_gp);
        cudaFree(d_kt);
        cudaFree(d_scale);
        return rc;
    }
    dconv1d_kernel<<<dim3((N + 127) / 128, nc * nconv), 128, 0, plan->stream>>>(N, nconv, d_dt, S.rho, d_scale, d_dn);
    CHECK_LAUNCH();
    switch (nc) {
    case 1: rc = launch_grad_points<1>(plan, b, d_dn, d_gp, d_kt); break;
    case 2: rc = launch_grad_points<2>(plan, b, d_dn, d_gp, d_kt); break;
    case 3: rc = launch_grad_points<3>(plan, b, d_dn, d_gp, d_kt); break;
    case 4: rc = launch_grad_points<4>(plan, b, d_dn, d_gp, d_kt); break;
    default: rc = set_error(CDFT_E_UNSUPPORTED, "nc=%d", nc);
    }
    std::vector<double> gp((size_t)NP * N), kt((size_t)nc * N);
    if (!rc) {
        CU(cudaMemcpyAsync(gp.data(), d_gp, gp.size() * sizeof(double), cudaMemcpyDeviceToHost, plan->stream));
        CU(cudaMemcpyAsync(kt.data(), d_kt, kt.size() * sizeof(double), cudaMemcpyDeviceToHost, plan->stream));
        CU(cudaStreamSynchronize(plan->stream));
    }
    cudaFree(d_dt);
    cudaFree(d_dn);
    cudaFree(d_gp);
    cudaFree(d_kt);
    cudaFree(d_scale);
    if (rc) return rc;
    // Simpson (as cdft_free_energy_res) or uniform integrals: G[q] = dF_res / dP_q, Gd[i] = dF_res / dd_i
    // via the kernels
    auto coef = [uniform](int k, int n) {
        return uniform ? 3.0 : ((k == 1 || k == n) ? 1.0 : ((k % 2 == 0) ? 4.0 : 2.0));
    };
    const double w = (plan->dz[0] / 3.0) / (L * L * L);
    std::vector<double> G(NP), Gd(nc);
    for (int q = 0; q < NP; ++q) {
        KSum acc;
        for (int k = 1; k <= N; ++k) acc.add(coef(k, N) * gp[(size_t)q * N + k - 1]);
        G[q] = acc.value() * w;
    }
    for (int i = 0; i < nc; ++i) {
        KSum acc;
        for (int k = 1; k <= N; ++k) acc.add(coef(k, N) * kt[(size_t)i * N + k - 1]);
        Gd[i] = acc.value() * w;
    }
    return fres_grad_chain(plan, G, Gd, dF);
}

// dF_res/dP_q (G) and dF_res/dd_i through the kernels (Gd) chained to theta = (sigma_k [A],
// eps_k / k_B [K], m_k) with the length unit L held fixed
static int fres_grad_chain(cdft_plan* plan, const std::vector<double>& G, const std::vector<double>& Gd, double* dF)
{
    const cdft_system_desc& d = plan->desc;
    const SysDev& S = plan->sys;
    const int nc = d.nc;
    const double L = d.L, T = d.T;
    const int iM = 0, iD = nc, iC1 = 2 * nc, iC2 = 2 * nc + nc * nc, iAD = 2 * nc + 2 * nc * nc, iAK = iAD + 1;
    const PhiParams& P = S.phi;
    for (int k = 0; k < nc; ++k) {
        const double sk = d.sigma[k * nc + k], ek = d.eps[k * nc + k];
        const double ex = exp(-3.0 * ek / T);
        // reduced diameter d_k / L: derivatives per m of sigma and per K of eps
        const double dd_ds = (1.0 - 0.12 * ex) / L;
        const double dd_de = sk * 0.36 / T * ex / L;
        double g_s = 0.0, g_e = 0.0, g_m = 0.0;
        // explicit dependence on d_k (FMT, chain, dispersion, association u_c) and through the kernels
        g_s += (G[iD + k] + Gd[k]) * dd_ds;
        g_e += (G[iD + k] + Gd[k]) * dd_de;
        g_m += G[iM + k];
        for (int i = 0; i < nc; ++i)
            for (int j = 0; j < nc; ++j) {
                const int dik = (i == k) + (j == k);
                if (!dik) continue;
                const double sg = d.sigma[i * nc + j] / L, e = d.eps[i * nc + j];
                const double mm = d.m[i] * d.m[j];
                const double c1 = mm * sg * sg * sg * e / T;
                // c1 = m_i m_j sg^3 e / T, c2 = c1 e / T; d sg / d sigma_k = dik / (2 L); d e / d eps_k = e dik / (2 eps_k)
                const double dc1_dm = ((i == k) * d.m[j] + (j == k) * d.m[i]) * sg * sg * sg * e / T;
                const double dc1_ds = mm * 3.0 * sg * sg * (0.5 * dik / L) * e / T;
                const double dc1_de = mm * sg * sg * sg / T * (e * 0.5 * dik / ek);
                const double de = e * 0.5 * dik / ek;
                g_m += G[iC1 + i * nc + j] * dc1_dm + G[iC2 + i * nc + j] * dc1_dm * e / T;
                g_s += G[iC1 + i * nc + j] * dc1_ds + G[iC2 + i * nc + j] * dc1_ds * e / T;
                g_e += G[iC1 + i * nc + j] * dc1_de + G[iC2 + i * nc + j] * (dc1_de * e / T + c1 * de / T);
            }
        if (P.has_assoc) {
            const int ic = P.a_ic, jc = P.a_jc;
            const double di = P.d[ic], dj = P.d[jc], den = (di + dj) * (di + dj);
            // a_dij = d_i d_j / (d_i + d_j)
            const double dA_dk = (ic == k ? dj * dj / den : 0.0) + (jc == k ? di * di / den : 0.0);
            g_s += G[iAD] * dA_dk * dd_ds;
            g_e += G[iAD] * dA_dk * dd_de;
            // a_K = sg^3 (exp(eps_AB / T) - 1) kappa_AB with sg = sigma_{ic,jc} / L
            const int dik = (ic == k) + (jc == k);
            if (dik) {
                const double sg = d.sigma[ic * nc + jc] / L;
                g_s += G[iAK] * 3.0 * (P.a_K / sg) * (0.5 * dik / L);
            }
        }
        dF[3 * k + 0] = g_s * 1e-10;   // per Angstrom
        dF[3 * k + 1] = g_e;
        dF[3 * k + 2] = g_m;
    }
    return 0;
}

// 3D parameter gradient of F_res.  The weighted densities' dependence on the diameters goes
// through the FFT pipeline with derivative kernel tables: d omega_hat / dR of each table's
// kernel times dR/dd = 2 pi w_t (type 1: 2 cos(wR) / 2 pi; type 2: 4 pi R sin(wR) / w / (2 pi)^3,
// 4 pi R^2 / (2 pi)^3 at w = 0; the vector fields take the type-2 table times i w_d, as the
// kernels do).  The pipeline with those tables gives dn_f = N_A L^3 rho (*) d omega_f / d d_i in
// the plan's field buffer; the pipeline with the plan's own tables then leaves the weighted
// densities there for the per-point terms.
static int fres_grad3d(cdft_plan* p, Batch* b, bool uniform, int NP, double* dF)
{
    const cdft_system_desc& d = p->desc;
    SysDev& S = p->sys;
    const int nc = d.nc, L3 = p->L3;
    const size_t npts = (size_t)L3 * L3 * L3;
    const double PI = 3.14159265358979323846, TWO_PI = 2.0 * PI;
    const int types[5] = {1, 2, 2, 1, 2};
    const double wf[5] = {0.5, 0.5, 1.0, 1.0, PSI_DISP};
    std::vector<double> tab((size_t)nc * 5 * (p->k2max + 1));
    for (int i = 0; i < nc; ++i)
        for (int t = 0; t < 5; ++t) {
            const double dR = TWO_PI * wf[t], R = dR * S.phi.d[i];
            for (int k2 = 0; k2 <= p->k2max; ++k2) {
                const double w = std::sqrt((double)k2) * p->w0;
                double v;
                if (types[t] == 1) v = 2.0 * std::cos(w * R) / TWO_PI;
                else v = (w == 0.0 ? 4.0 * PI * R * R : 4.0 * PI * R * std::sin(w * R) / w) / (TWO_PI * TWO_PI * TWO_PI);
                tab[((size_t)i * 5 + t) * (p->k2max + 1) + k2] = v * dR;
            }
        }
    double *d_tab = nullptr, *d_dn = nullptr, *d_gp = nullptr, *d_kt = nullptr;
    const size_t nfield = (size_t)nc * S.nconv * npts;
    int rc = 0;
    auto cleanup = [&]() {
        cudaFree(d_tab);
        cudaFree(d_dn);
        cudaFree(d_gp);
        cudaFree(d_kt);
    };
    if (cudaMalloc(&d_tab, tab.size() * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&d_dn, nfield * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&d_gp, (size_t)NP * npts * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&d_kt, (size_t)nc * npts * sizeof(double)) != cudaSuccess) {
        cleanup();
        return set_error(CDFT_E_CUDA, "3D parameter gradient: out of device memory");
    }
    cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, p->stream);
    double* keep = p->d_ktab;
    p->d_ktab = d_tab;
    rc = launch_eval_stages<double>(b, nullptr, false);   // S.part = d n_f / d d_i (Phi of it is unused)
    p->d_ktab = keep;
    if (!rc) {
        cudaMemcpyAsync(d_dn, S.part, nfield * sizeof(double), cudaMemcpyDeviceToDevice, p->stream);
        rc = launch_eval_stages<double>(b, nullptr, false);   // S.part = the weighted densities
    }
    if (!rc) {
        switch (nc) {
        case 1: rc = launch_grad_points<1>(p, b, d_dn, d_gp, d_kt); break;
        case 2: rc = launch_grad_points<2>(p, b, d_dn, d_gp, d_kt); break;
        case 3: rc = launch_grad_points<3>(p, b, d_dn, d_gp, d_kt); break;
        case 4: rc = launch_grad_points<4>(p, b, d_dn, d_gp, d_kt); break;
        default: rc = set_error(CDFT_E_UNSUPPORTED, "nc=%d", nc);
        }
    }
    std::vector<double> gp, kt;
    if (!rc) {
        gp.resize((size_t)NP * npts);
        kt.resize((size_t)nc * npts);
        cudaMemcpyAsync(gp.data(), d_gp, gp.size() * sizeof(double), cudaMemcpyDeviceToHost, p->stream);
        cudaMemcpyAsync(kt.data(), d_kt, kt.size() * sizeof(double), cudaMemcpyDeviceToHost, p->stream);
        const cudaError_t e = cudaStreamSynchronize(p->stream);
        if (e != cudaSuccess) rc = set_error(CDFT_E_CUDA, "3D parameter gradient: %s", cudaGetErrorString(e));
    }
    cleanup();
    if (rc) return rc;
    // Simpson weights per dimension (integrals.jl:28-41) or the uniform dz^3
    auto coef = [uniform](int k, int n) {
        return uniform ? 3.0 : ((k == 1 || k == n) ? 1.0 : ((k % 2 == 0) ? 4.0 : 2.0));
    };
    const double Lr = d.L;
    const double w = (p->dz[0] / 3.0) * (p->dz[1] / 3.0) * (p->dz[2] / 3.0) / (Lr * Lr * Lr);
    std::vector<double> G(NP), Gd(nc);
    auto wsum = [&](const double* f) {
        KSum acc;
        for (int z = 1; z <= L3; ++z)
            for (int y = 1; y <= L3; ++y) {
                const double cyz = coef(z, L3) * coef(y, L3);
                const double* row = f + ((size_t)(z - 1) * L3 + (y - 1)) * L3;
                for (int x = 1; x <= L3; ++x) acc.add(cyz * coef(x, L3) * row[x - 1]);
            }
        return acc.value() * w;
    };
    for (int q = 0; q < NP; ++q) G[q] = wsum(gp.data() + (size_t)q * npts);
    for (int i = 0; i < nc; ++i) Gd[i] = wsum(kt.data() + (size_t)i * npts);
    return fres_grad_chain(p, G, Gd, dF);
}

}  // extern "C"

namespace {

int grad_params_impl(cdft_plan* plan, const double* rho, const double* dmu_dtheta, const double* dp_dtheta,
                     const double* dvext_dtheta, double* dOmega)
{
    if (!plan || !rho || !dOmega) return set_error(CDFT_E_INVALID, "NULL argument");
    const cdft_system_desc& d = plan->desc;
    if (plan->d_vext && !dvext_dtheta)
        return set_error(CDFT_E_UNSUPPORTED,
                         "the external field depends on the parameters: pass its derivative (cdft_grad_params_ext)");
    const int nc = d.nc, N = plan->N, np = 3 * nc;
    std::vector<double> dF(np);
    g_err_code = 0;
    int rc = fres_grad_impl(plan, rho, dF.data(), true);
    if (rc) return rc;
    // The envelope theorem needs the quadrature in which the converged profile is stationary:
    // the pointwise Euler-Lagrange equation is the gradient of the functional summed with
    // uniform weights dz (the adjoint of the periodic convolution), so every integral below
    // uses them.  surface_tension's Simpson weights differ from it where the profile is not
    // resolved on the grid (sharp adsorbed layers); for resolved profiles the two agree.
    const double dz = (d.nd == 3) ? plan->dz[0] * plan->dz[1] * plan->dz[2] : plan->dz[0];   // volume per point
    std::vector<double> nint(nc);
    for (int i = 0; i < nc; ++i) {
        KSum acc;
        for (int k = 0; k < N; ++k) acc.add(rho[(size_t)i * N + k]);
        nint[i] = acc.value() * dz;
    }
    const double one = (double)N * dz;
    const double kB = 1.380649e-23, NAVO = 6.02214076e23;
    for (int t = 0; t < np; ++t) {
        double v = kB * d.T * dF[t];
        if (dmu_dtheta)
            for (int i = 0; i < nc; ++i) v -= dmu_dtheta[(size_t)i * np + t] * nint[i];
        if (dp_dtheta) v += dp_dtheta[t] * one;
        if (dvext_dtheta)   // R T sum_i int rho_i dV_i/dtheta (rho in mol/m^3, V in units of k_B T)
            for (int i = 0; i < nc; ++i) {
                KSum acc;
                const double* dv = dvext_dtheta + ((size_t)t * nc + i) * N;
                for (int k = 0; k < N; ++k) acc.add(rho[(size_t)i * N + k] * dv[k]);
                v += NAVO * kB * d.T * acc.value() * dz;
            }
        dOmega[t] = v;
    }
    return 0;
}

}  // namespace

extern "C" {

int cdft_grad_params(cdft_plan* plan, const double* rho, const double* dmu_dtheta, const double* dp_dtheta,
                     double* dOmega)
{
    g_err_code = 0;
    return grad_params_impl(plan, rho, dmu_dtheta, dp_dtheta, nullptr, dOmega);
}

int cdft_grad_params_ext(cdft_plan* plan, const double* rho, const double* dmu_dtheta, const double* dp_dtheta,
                         const double* dvext_dtheta, double* dOmega)
{
    g_err_code = 0;
    if (!dvext_dtheta) return set_error(CDFT_E_INVALID, "dvext_dtheta is NULL");
    return grad_params_impl(plan, rho, dmu_dtheta, dp_dtheta, dvext_dtheta, dOmega);
}

}  // extern "C"

// ===========================================================================
// Allocation-free functional derivative (cdft_functional_derivative_noalloc).
//
// For callers that cannot call cudaMalloc (see the header).  The scratch is a
// file-scope device array; host code never dereferences its name (in host code
// it is only a stand-in for the symbol): the device address is obtained once
// per device with cudaGetSymbolAddress and handed to the kernels.
// ===========================================================================
static __device__ __align__(256) double g_noalloc_scratch[CDFT_NOALLOC_SCRATCH_BYTES / sizeof(double)];

namespace {

std::mutex g_noalloc_mu;
double* g_noalloc_addr[64] = {nullptr};

// device address of the scratch array on the current device (looked up on first use)
int noalloc_scratch_addr(double** out)
{
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(CDFT_E_UNSUPPORTED, "device ordinal %d", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[dev];
    return 0;
}

size_t noalloc_align(size_t n) { return (n + 31) & ~size_t(31); }   // 256-byte steps, in doubles

}  // namespace

extern "C" int cdft_functional_derivative_noalloc(const cdft_system_desc* desc, const double* d_rho, double* d_dFdrho,
                                                  void* stream_ptr)
{
    g_err_code = 0;
    if (!d_rho || !d_dFdrho) return set_error(CDFT_E_INVALID, "NULL device array");
    int rc = validate_desc(desc);
    if (rc) return rc;
    const cdft_system_desc& d = *desc;
    if (d.nd != 1 || d.coord != CDFT_COORD_CART)
        return set_error(CDFT_E_UNSUPPORTED, "the allocation-free entry point handles 1D Cartesian grids only");
    if (d.precision != CDFT_PREC_FP64)
        return set_error(CDFT_E_UNSUPPORTED, "the allocation-free entry point computes in FP64 only");
    const int N = d.ngrid[0], nc = d.nc;
    if (N > CDFT_NOALLOC_MAX_N || (long long)N * nc > CDFT_NOALLOC_MAX_ELEM)
        return set_error(CDFT_E_UNSUPPORTED,
                         "system too large for the allocation-free scratch: N=%d nc=%d (limits N<=%d, N*nc<=%d)",
                         N, nc, CDFT_NOALLOC_MAX_N, CDFT_NOALLOC_MAX_ELEM);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    if (stream) {   // the stream must belong to the current device, where the scratch address is looked up
        int dev = 0, sdev = 0;
        CU(cudaGetDevice(&dev));
        CU(cudaStreamGetDevice(stream, &sdev));
        if (sdev != dev)
            return set_error(CDFT_E_INVALID, "stream belongs to device %d, the current device is %d", sdev, dev);
    }
    rc = upload_constants();
    if (rc) return rc;
    double* base = nullptr;
    rc = noalloc_scratch_addr(&base);
    if (rc) return rc;

    // system record (reduced parameters as in plan creation), pointers into the scratch
    SysDev S;
    memset(&S, 0, sizeof(S));
    S.nd = 1;
    S.N = N;
    S.nc = nc;
    S.NF = 7;
    S.nconv = 6;
    S.ngrid[0] = N; S.ngrid[1] = 1; S.ngrid[2] = 1;
    S.ksplit = (d.coord == CDFT_COORD_CART) ? (N + CONV_QC - 1) / CONV_QC : 1;
    S.n_elem = N * nc;
    const double L = d.L, T = d.T;
    S.NA = kNA * L * L * L;
    for (int i = 0; i < nc; ++i) S.cprd[i] = d.mu_res_plus_ln_rhob[i];
    PhiParams& P = S.phi;
    P.nc = nc;
    P.nd = 1;
    P.T = T;
    for (int i = 0; i < nc; ++i) {
        P.m[i] = d.m[i];
        P.d[i] = d.hsd[i] / L;
    }
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            const double sg = d.sigma[i * nc + j] / L;
            const double e = d.eps[i * nc + j];
            const double c1 = d.m[i] * d.m[j] * sg * sg * sg * e / T;
            P.c1[i * CDFT_MAX_NC + j] = c1;
            P.c2[i * CDFT_MAX_NC + j] = c1 * e / T;
        }
    fill_assoc_params(P, d);

    // task and chunk lists on the host stack (bounded by the size limits)
    ConvTask tasks[1024];
    Chunk pch[(CDFT_NOALLOC_MAX_N + POINT_THREADS - 1) / POINT_THREADS];
    Chunk ech[(CDFT_NOALLOC_MAX_ELEM + ELEM_CHUNK - 1) / ELEM_CHUNK];
    int ntasks = 0, npch = 0, nech = 0;
    const int tiles = (N + CONV_TILE - 1) / CONV_TILE;
    for (int i = 0; i < nc; ++i)
        for (int f = 0; f < S.nconv; ++f)
            for (int t = 0; t < tiles; ++t)
                for (int ks = 0; ks < S.ksplit; ++ks) {
                    if (ntasks >= 1024) return set_error(CDFT_E_UNSUPPORTED, "task list overflow");
                    tasks[ntasks++] = {0, i, f, t * S.ksplit + ks};
                }
    for (int j = 0; j < N; j += POINT_THREADS) pch[npch++] = {0, j};
    for (int e = 0; e < S.n_elem; e += ELEM_CHUNK) ech[nech++] = {0, e};

    // scratch layout (offsets in doubles, 256-byte aligned)
    size_t off = 0;
    const size_t o_sys = off;   off += noalloc_align((sizeof(SysDev) + 7) / 8);
    const size_t o_task = off;  off += noalloc_align((sizeof(ConvTask) * ntasks + 7) / 8);
    const size_t o_pch = off;   off += noalloc_align((sizeof(Chunk) * npch + 7) / 8);
    const size_t o_ech = off;   off += noalloc_align((sizeof(Chunk) * nech + 7) / 8);
    const size_t ntap = (size_t)S.nconv * nc * N;
    const size_t o_taps = off;  off += noalloc_align(ntap);
    const size_t o_part = off;  off += noalloc_align(ntap * S.ksplit);
    const size_t o_df = off;    off += noalloc_align((size_t)S.NF * nc * N);
    const size_t o_fval = off;  off += noalloc_align((size_t)N);
    const size_t o_vext = off;  off += d.vext ? noalloc_align((size_t)S.n_elem) : 0;
    if (off * sizeof(double) > CDFT_NOALLOC_SCRATCH_BYTES)
        return set_error(CDFT_E_UNSUPPORTED, "scratch of %zu B exceeds %u B", off * sizeof(double),
                         (unsigned)CDFT_NOALLOC_SCRATCH_BYTES);
    S.taps = base + o_taps;
    S.part = base + o_part;
    S.dfield = base + o_df;
    S.fval = base + o_fval;
    S.vext = d.vext ? base + o_vext : nullptr;
    S.rho = const_cast<double*>(d_rho);   // read only by the kernels below
    S.out = d_dFdrho;
    SysDev* d_sys = reinterpret_cast<SysDev*>(base + o_sys);
    ConvTask* d_tasks = reinterpret_cast<ConvTask*>(base + o_task);
    Chunk* d_pch = reinterpret_cast<Chunk*>(base + o_pch);
    Chunk* d_ech = reinterpret_cast<Chunk*>(base + o_ech);
    CU(cudaMemcpyAsync(d_sys, &S, sizeof(SysDev), cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(d_tasks, tasks, sizeof(ConvTask) * ntasks, cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(d_pch, pch, sizeof(Chunk) * npch, cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(d_ech, ech, sizeof(Chunk) * nech, cudaMemcpyHostToDevice, stream));
    if (d.vext)
        CU(cudaMemcpyAsync(base + o_vext, d.vext, sizeof(double) * S.n_elem, cudaMemcpyHostToDevice, stream));

    // kernels of get_fields(::PCSAFTModel) in 1D (PCSAFT.jl:55-61), same tables as plan creation
    const double span = d.bounds[0][1] - d.bounds[0][0];
    rc = launch_taps(stream, N, span, L, nc, P.d, base + o_taps, false);
    if (rc) return rc;
    const size_t smem = (size_t)(CONV_QC + CONV_TILE + CONV_QC + 31) * sizeof(double);
    conv1d_kernel<double><<<ntasks, CONV_WARPS * 32, smem, stream>>>(d_tasks, d_sys, nullptr, 0);
    switch (nc) {
    case 1: phi_kernel<double, 1, 1><<<npch, POINT_THREADS, 0, stream>>>(d_pch, d_sys, nullptr); break;
    case 2: phi_kernel<double, 2, 1><<<npch, POINT_THREADS, 0, stream>>>(d_pch, d_sys, nullptr); break;
    case 3: phi_kernel<double, 3, 1><<<npch, POINT_THREADS, 0, stream>>>(d_pch, d_sys, nullptr); break;
    default: phi_kernel<double, 4, 1><<<npch, POINT_THREADS, 0, stream>>>(d_pch, d_sys, nullptr); break;
    }
    conv1d_kernel<double><<<ntasks, CONV_WARPS * 32, smem, stream>>>(d_tasks, d_sys, nullptr, 1);
    dfdrho_out_kernel<double><<<nech, ELEM_THREADS, 0, stream>>>(d_ech, d_sys);
    CHECK_LAUNCH();
    g_launches += 4;
    CU(cudaStreamSynchronize(stream));
    return 0;
}
