// C-ABI of the B200 MDFT engine (declared in include/mdft_b200.h).
#include "../../include/mdft_b200.h"

#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <string>
#include <thread>

#include "common.cuh"
#include "setup_host.cuh"
#include "k_angular.cuh"
#include "k_fft.cuh"
#include "k_fft2.cuh"
#include "k_oz.cuh"
#include "k_oz2.cuh"
#include "k_vec.cuh"
#include "k_lbfgs.cuh"
#include "k_gather_tma.cuh"
#include "k_ozp.cuh"
#include "k_project_tma.cuh"
#include "k_angular_umma.cuh"
#include "k_vext.cuh"
#include "k_bridge.cuh"

namespace mdft {

static thread_local std::string g_error;
void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
}
const char *last_error() { return g_error.c_str(); }

constexpr double kBoltz = 1.3806488e-23;  // src/module_constants.f90:26
constexpr double kNavo = 6.02214129e23;   // src/module_constants.f90:24

enum Stage { ST_PROJECT = 0, ST_FFT_FWD, ST_OZ, ST_FFT_INV, ST_GATHER, ST_COUNT };

struct FftAxis {
    FftAxisArgs args;
    int grid;
    size_t smem;
    const void *tw;  // device twiddles (double2 or float2) of this length
};

}  // namespace mdft

using namespace mdft;

struct mdft_handle {
    Grid g;
    // set on species 0's handle while mdft_mixture_minimize runs: the minimiser's vectors
    // span every species and its evaluations are the mixture's
    mdft_mixture *mix = nullptr;
    CTable ct;
    int precision = MDFT_PREC_FP64;
    int device = 0;
    cudaStream_t stream = nullptr;
    double const_corr = 0.0;
    bool have_vext = false;
    // device state
    DevBuf<double> xi, vext, df, w, A, B, partial, sums;
    DevBuf<float> vext32;  // FP32 copy of vext for the FP32 phase of mixed solves (made per solve)
    DevBuf<double2> planes, ctab;
    DevBuf<double2> tw64[3];
    // mixed path: FP32 projections, c table, twiddles and angular matrices
    DevBuf<float> A32, B32;
    DevBuf<float2> planes32, ctab32, tw32[3];
    int eval_prec = MDFT_PREC_FP64;  // precision of the evaluations run_pipeline performs
    double *h_sums = nullptr;  // pinned {F_id, F_ext, sum_exc}
    int bm_project = 64, bm_gather = 64;
    long long nblk_project = 0, nblk_gather = 0;
    int nsm = 148;
    int gt_ncol64 = 0, gt_ncol32 = 0;  // k_gather_tma columns of 32 per precision (0: not usable)
    bool pt_ok64 = false, pt_ok32 = false;  // k_project_tma usable per precision
    int pt_grid_x32 = 0;                    // resident CTAs of k_project_tma<float, float>
    int xy_grid_cap64 = 0, xy_grid_cap32 = 0;  // CTAs of the persistent xy FFT (resident count)
    DevBuf<int> kerr;                  // set by a pipeline kernel whose bounded wait ran out
    int *h_kerr = nullptr;
    FftAxis fft[3];
    Oz2Args oz{};
    DevBuf<int> oz_ints;
    DevBuf<double> oz_dbls;
    int oz_grid = 0, oz_warps = 8, oz_grid32 = 0, oz_warps32 = 8;
    // FP32 evaluations: angular contractions on the tensor cores (k_project_umma,
    // k_gather_umma), with the packed split-BF16 images of A^T and B^T
    bool um_ok = false;
    UmmaShape um_ps{}, um_gs{};
    DevBuf<uint16_t> um_pimg, um_gimg;
    int um_grid_p = 0, um_grid_g = 0;
    bool ring_p = false, ring_g = false;  // FP32 phase: the bulk-copy ring forms (one CTA per SM)
    bool ring_p_ok = false, ring_g_ok = false;  // ... where they fit
    // autotuning of the FP32 forms (project: register/ring, OZ: factored/unfactored, gather:
    // ring/register), once per handle on its first FP32 phase; tune_ms[stage][config] are the
    // measured stage times of the two configurations timed (-1: not measured)
    bool tune_on = false, tuned = false;
    double tune_ms[3][2] = {{-1, -1}, {-1, -1}, {-1, -1}};
    bool ozp_ok = false;  // FP32 evaluations use the thread-per-pair k_ozp
    bool ozd = false;     // ... in its factored-rotation form k_ozd (MDFT_OZ=ozp: the unfactored one)
    OzpParams ozp{};
    DevBuf<float2> ozp_cq;  // c interpolated at every |q|^2 of a cubic grid (empty: interpolate per pair)
    size_t oz_smem = 0, oz_smem32 = 0;
    // timing
    bool timing = false;
    bool trace = false;  // MDFT_TRACE=1 in the environment at create: per-iteration log on stderr
    cudaEvent_t ev[ST_COUNT + 1] = {};
    double stage_ms[ST_COUNT] = {0};
    int stage_count = 0;
    long long launches = 0;  // kernels launched by this handle
    // the evaluation pipeline as CUDA graphs, one per set of buffers and flags (MDFT_GRAPHS=0:
    // direct launches); never used while stage timing is on
    struct PipeGraph {
        const void *x, *dvec, *vext, *vext32;
        double *g;
        int do_ideal, df_mode, prec;
        bool v32, x32;
        cudaGraphExec_t exec;
        long long nlaunch;
    };
    std::vector<PipeGraph> pipe_graphs;
    bool graphs_on = true;
    bool wait_fail = false;  // mdft_set_wait_failure: gathers report a timed-out wait (tests)
    // vector reductions
    DevBuf<double> vpart, vsc;
    double *h_vsc = nullptr;
    // minimiser work (allocated on first use)
    LbfgsState lb;
    // learned warm start (mdft_set_warm_net): the network, its input channels, the
    // orientation table {u_x, u_y, u_z, w} and the solute sites, allocated on first use
    mdft_warm_net *warm = nullptr;
    DevBuf<float> wfeat;
    DevBuf<double4> wdir;
    DevBuf<double> wsite;
    long long warm_starts = 0, warm_fallbacks = 0;
    // bridge = "cgb" (mdft_set_bridge_cgb): 0 none, 1 'sla', 2 'wda'; the transformed kernel,
    // two work planes, n(r) and the block partials
    int cgb = 0;
    CgbArgs cgb_args{};
    DevBuf<double2> cgb_kk, cgb_a, cgb_b;
    DevBuf<double> cgb_dens, cgb_part;
    // bridge = "hard_sphere" (mdft_set_bridge_fmt): 0 none, 1 PY, 2 CS; seven work planes,
    // the hard-sphere c(k) and the partials {density 2B | stats 2 | Phi 4B | gradient 4B}
    int fmt = 0;
    FmtArgs fmt_args{};
    DevBuf<double2> fmt_pl;
    DevBuf<double> fmt_cs, fmt_part;
};

namespace {
bool has_bridge(const mdft_handle *h) { return h->cgb || h->fmt; }
}

namespace {

int check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return MDFT_E_CUDA;
    }
    return 0;
}

int alloc_check(cudaError_t e, const char *what, size_t bytes) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        set_error("device allocation of %zu bytes for %s failed", bytes, what);
        return MDFT_E_NOMEM;
    }
    return check_cuda(e, what);
}

// Let `fn` use all opt-in shared memory that its static allocation leaves.
int allow_smem(const void *fn, int optin) {
    cudaFuncAttributes at{};
    int rc = check_cuda(cudaFuncGetAttributes(&at, fn), "cudaFuncGetAttributes");
    if (rc) return rc;
    return check_cuda(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)at.sharedSizeBytes),
                      "cudaFuncSetAttribute");
}

int upload_twiddles(DevBuf<double2> &buf, int n) {
    std::vector<double2> h(n);
    for (int t = 0; t < n; ++t) {
        long double ang = 2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)n;
        h[t] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    int rc = alloc_check(buf.alloc(n), "fft twiddles", n * sizeof(double2));
    if (rc) return rc;
    return check_cuda(cudaMemcpy(buf.p, h.data(), n * sizeof(double2), cudaMemcpyHostToDevice), "twiddle upload");
}

// BF16 bits of an FP32 value, rounded to nearest even (finite inputs)
uint16_t bf16_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
float bf16_value(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
// hi and lo BF16 images (hi then lo) of an [Rp][Kp] operand in the packed tcgen05 layout;
// value(r, k) is the FP64 entry (0 in the padding)
template <typename F>
void pack_split_bf16(int Rp, int Kp, F value, std::vector<uint16_t> &img) {
    const size_t half = (size_t)Rp * Kp;
    img.assign(2 * half, 0);
    for (int r = 0; r < Rp; ++r)
        for (int k = 0; k < Kp; ++k) {
            const double v = value(r, k);
            const uint16_t hi = bf16_bits((float)v);
            const uint16_t lo = bf16_bits((float)(v - (double)bf16_value(hi)));
            const size_t off = umma::elem_offset(r, k, Kp, 2) / 2;
            img[off] = hi;
            img[half + off] = lo;
        }
}

int pick_tl(long long lines_divisor, int n) {
    int best = 1;
    const int cands[] = {32, 16, 8, 4, 2, 1};
    for (int c : cands) {
        if (lines_divisor % c) continue;
        if (c == 32 && n > 32) continue;
        best = c;
        break;
    }
    return best;
}

int setup_fft(mdft_handle *h) {
    const Grid &g = h->g;
    const int dims[3] = {g.nx, g.ny, g.nz};
    for (int ax = 0; ax < 3; ++ax) {
        FftAxis &F = h->fft[ax];
        F.args.axis = ax;
        F.args.nx = g.nx;
        F.args.ny = g.ny;
        F.args.nz = g.nz;
        F.args.nplanes = g.np;
        if (!make_plan1d(dims[ax], F.args.plan)) {
            set_error("grid size %d is not of the form 2^a 3^b", dims[ax]);
            return MDFT_E_ARG;
        }
        long long lines_div = (ax == 0) ? (long long)g.np * g.ny * g.nz : g.nx;
        F.args.TL = pick_tl(lines_div, dims[ax]);
        long long nlines = (long long)g.np * g.N / dims[ax];
        F.grid = (int)(nlines / F.args.TL);
        F.smem = fft_smem_bytes<double>(dims[ax], F.args.TL);
        int rc = upload_twiddles(h->tw64[ax], dims[ax]);
        if (rc) return rc;
        F.tw = h->tw64[ax].p;
        std::vector<double2> t64(dims[ax]);
        cudaMemcpy(t64.data(), h->tw64[ax].p, dims[ax] * sizeof(double2), cudaMemcpyDeviceToHost);
        std::vector<float2> t32(dims[ax]);
        for (int t = 0; t < dims[ax]; ++t) t32[t] = make_float2((float)t64[t].x, (float)t64[t].y);
        if ((rc = alloc_check(h->tw32[ax].alloc(dims[ax]), "fft twiddles", dims[ax] * sizeof(float2)))) return rc;
        cudaMemcpy(h->tw32[ax].p, t32.data(), dims[ax] * sizeof(float2), cudaMemcpyHostToDevice);
    }
    return 0;
}

// Specialised plane (x,y) and column (z) transforms for the supported lengths; the
// generic per-axis kernel otherwise.
template <typename T, int N>
cudaError_t fft_xy_n(typename Cplx<T>::t *data, long long nplanes, const typename Cplx<T>::t *tw, int sign, cudaStream_t st,
                     bool prepare, int grid_cap, int *err) {
    if constexpr (xy_tma_fits<T, N>()) {
        // persistent bulk-copy form: grid_cap CTAs at most (the device's resident count)
        if (prepare)
            return cudaFuncSetAttribute(k_fft_xy_tma<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xy_tma_smem_bytes<T, N>());
        const long long grid = std::min<long long>(nplanes, std::max(1, grid_cap));
        k_fft_xy_tma<T, N><<<(unsigned)grid, xy_threads<T, N>(), xy_tma_smem_bytes<T, N>(), st>>>(data, tw, sign, nplanes, err);
        return cudaGetLastError();
    } else {
        if (prepare)
            return cudaFuncSetAttribute(k_fft_xy<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xy_smem_bytes<T, N>());
        k_fft_xy<T, N><<<(unsigned)nplanes, xy_threads<T, N>(), xy_smem_bytes<T, N>(), st>>>(data, tw, sign);
        return cudaGetLastError();
    }
}
template <typename T, int N>
cudaError_t fft_z_n(typename Cplx<T>::t *data, long long nplanes, int nx, int ny, const typename Cplx<T>::t *tw, int sign,
                    cudaStream_t st, bool prepare) {
    if (prepare)
        return cudaFuncSetAttribute(k_fft_z<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)z_smem_bytes<T, N>());
    const long long grid = nplanes * ny * (nx / z_tl<T>());
    k_fft_z<T, N><<<(unsigned)grid, 256, z_smem_bytes<T, N>(), st>>>(data, tw, nx, ny, sign);
    return cudaGetLastError();
}

// resident CTAs per SM of the persistent xy FFT for length n (0: not used for n)
template <typename T, int N>
int xy_tma_per_sm_n() {
    if constexpr (xy_tma_fits<T, N>()) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_fft_xy_tma<T, N>, xy_threads<T, N>(), xy_tma_smem_bytes<T, N>());
        return b;
    } else {
        return 0;
    }
}
template <typename T>
int xy_tma_per_sm(int n) {
    switch (n) {
    case 8: return xy_tma_per_sm_n<T, 8>();
    case 12: return xy_tma_per_sm_n<T, 12>();
    case 16: return xy_tma_per_sm_n<T, 16>();
    case 24: return xy_tma_per_sm_n<T, 24>();
    case 32: return xy_tma_per_sm_n<T, 32>();
    case 48: return xy_tma_per_sm_n<T, 48>();
    case 64: return xy_tma_per_sm_n<T, 64>();
    case 96: return xy_tma_per_sm_n<T, 96>();
    default: return 0;
    }
}

// returns cudaErrorNotSupported when no specialised kernel exists for n
template <typename T>
cudaError_t fft_xy(int n, typename Cplx<T>::t *data, long long nplanes, const typename Cplx<T>::t *tw, int sign, cudaStream_t st,
                   bool prepare, int grid_cap = 0, int *err = nullptr) {
    switch (n) {
    case 8: return fft_xy_n<T, 8>(data, nplanes, tw, sign, st, prepare, grid_cap, err);
    case 12: return fft_xy_n<T, 12>(data, nplanes, tw, sign, st, prepare, grid_cap, err);
    case 16: return fft_xy_n<T, 16>(data, nplanes, tw, sign, st, prepare, grid_cap, err);
    case 24: return fft_xy_n<T, 24>(data, nplanes, tw, sign, st, prepare, grid_cap, err);
    case 32: return fft_xy_n<T, 32>(data, nplanes, tw, sign, st, prepare, grid_cap, err);
    case 48: return fft_xy_n<T, 48>(data, nplanes, tw, sign, st, prepare, grid_cap, err);
    case 64: return fft_xy_n<T, 64>(data, nplanes, tw, sign, st, prepare, grid_cap, err);
    case 96: return fft_xy_n<T, 96>(data, nplanes, tw, sign, st, prepare, grid_cap, err);
    default: return cudaErrorNotSupported;
    }
}
template <typename T>
cudaError_t fft_z(int n, typename Cplx<T>::t *data, long long nplanes, int nx, int ny, const typename Cplx<T>::t *tw, int sign,
                  cudaStream_t st, bool prepare) {
    if (nx % z_tl<T>()) return cudaErrorNotSupported;
    switch (n) {
    case 8: return fft_z_n<T, 8>(data, nplanes, nx, ny, tw, sign, st, prepare);
    case 12: return fft_z_n<T, 12>(data, nplanes, nx, ny, tw, sign, st, prepare);
    case 16: return fft_z_n<T, 16>(data, nplanes, nx, ny, tw, sign, st, prepare);
    case 24: return fft_z_n<T, 24>(data, nplanes, nx, ny, tw, sign, st, prepare);
    case 32: return fft_z_n<T, 32>(data, nplanes, nx, ny, tw, sign, st, prepare);
    case 48: return fft_z_n<T, 48>(data, nplanes, nx, ny, tw, sign, st, prepare);
    case 64: return fft_z_n<T, 64>(data, nplanes, nx, ny, tw, sign, st, prepare);
    case 96: return fft_z_n<T, 96>(data, nplanes, nx, ny, tw, sign, st, prepare);
    case 128: return fft_z_n<T, 128>(data, nplanes, nx, ny, tw, sign, st, prepare);
    default: return cudaErrorNotSupported;
    }
}

template <typename T>
int launch_fft_t(mdft_handle *h, typename Cplx<T>::t *planes, const void *const *tw, int sign) {
    using C = typename Cplx<T>::t;
    const Grid &g = h->g;
    bool xy_done = false;
    if (g.nx == g.ny && sizeof(C) * (size_t)g.nx * (g.nx + 2) <= 200 * 1024) {
        cudaError_t e = fft_xy<T>(g.nx, planes, (long long)g.np * g.nz, (const C *)tw[0], sign, h->stream, false,
                                  sizeof(T) == 8 ? h->xy_grid_cap64 : h->xy_grid_cap32, h->kerr.p);
        if (e == cudaSuccess) { xy_done = true; h->launches += 1; }
        else if (e != cudaErrorNotSupported) return check_cuda(e, "fft xy launch");
        else cudaGetLastError();
    }
    for (int ax = 0; ax < 2 && !xy_done; ++ax) {
        FftAxis &F = h->fft[ax];
        FftAxisArgs a = F.args;
        a.sign = sign;
        k_fft_axis<T><<<F.grid, kFftThreads, fft_smem_bytes<T>(a.plan.n, a.TL), h->stream>>>(planes, (const C *)tw[ax], a);
        h->launches += 1;
    }
    cudaError_t e = fft_z<T>(g.nz, planes, g.np, g.nx, g.ny, (const C *)tw[2], sign, h->stream, false);
    if (e == cudaSuccess) {
        h->launches += 1;
    } else if (e == cudaErrorNotSupported) {
        cudaGetLastError();
        FftAxis &F = h->fft[2];
        FftAxisArgs a = F.args;
        a.sign = sign;
        k_fft_axis<T><<<F.grid, kFftThreads, fft_smem_bytes<T>(a.plan.n, a.TL), h->stream>>>(planes, (const C *)tw[2], a);
        h->launches += 1;
    } else {
        return check_cuda(e, "fft z launch");
    }
    return check_cuda(cudaGetLastError(), "fft launch");
}

// FP32 OZ, thread per pair: the instantiation for (mmax, mrso); factored: the form with the
// rotation matrices split into phases and a real matrix (k_ozd), else k_ozp
template <int MM, int MR>
const void *ozp_fn(bool factored) { return factored ? (const void *)k_ozd<MM, MR> : (const void *)k_ozp<MM, MR>; }
const void *ozp_kernel(int mmax, int mrso, bool factored = false) {
    if (mrso == 2) {
        switch (mmax) {
            case 0: return ozp_fn<0, 2>(factored);
            case 1: return ozp_fn<1, 2>(factored);
            case 2: return ozp_fn<2, 2>(factored);
            case 3: return ozp_fn<3, 2>(factored);
        }
    } else if (mrso == 1) {
        switch (mmax) {
            case 0: return ozp_fn<0, 1>(factored);
            case 1: return ozp_fn<1, 1>(factored);
            case 2: return ozp_fn<2, 1>(factored);
        }
    }
    return nullptr;
}
void launch_ozp(mdft_handle *h, float2 *planes, const float2 *ctab, const Oz2Args &oz) {
    const Grid &g = h->g;
    const unsigned grid = (unsigned)((oz.nk + kOzpThreads - 1) / kOzpThreads);
    const size_t smem = ozp_smem_bytes(g.np);
    const float2 *cq = h->ozp_cq.p;
    void *args[] = {(void *)&planes, (void *)&ctab, (void *)&oz, (void *)&h->ozp, (void *)&cq};
    cudaLaunchKernel(ozp_kernel(g.mmax, g.mrso, h->ozd), dim3(grid), dim3(kOzpThreads), args, smem, h->stream);
}

void stage_mark(mdft_handle *h, int i) {
    if (h->timing) cudaEventRecord(h->ev[i], h->stream);
}

// Arguments of the S7 gather.  The excess prefactor -kT 2 (4 pi^2) / mrso / n0
// (src/module_energy_cproj_mrso.f90:728) carries a species' mole fraction as `scale` in a
// multi-species evaluation (src/module_energy_cproj_mrso_mixture.f90:791).
GatherArgs gather_args(const mdft_handle *h, int df_mode, int do_ideal, const void *dvec, double scale) {
    const Grid &g = h->g;
    GatherArgs ga;
    ga.fail_wait = h->wait_fail ? 1 : 0;
    ga.N = g.N;
    ga.no = g.no;
    ga.np = g.np;
    ga.rho0 = g.rho0;
    ga.kT = g.kT;
    ga.dv = g.dv;
    const double fourpisq = 4.0 * kPi * kPi;
    ga.prefactor = -g.kT * 2.0 * fourpisq / g.mrso / g.n0;
    if (scale != 1.0) ga.prefactor *= scale;
    ga.cst = 1.0 / (double)(g.nx * g.ny * g.nz);
    ga.do_ideal = do_ideal;
    ga.df_mode = df_mode;
    ga.dvec = dvec;
    return ga;
}

// batched FFT over planes (defined with the solver, solve.cuh)
int launch_fft_planes(mdft_handle *h, double2 *data, int nplanes, int sign);

// The bridge term after the pipeline of a full FP64 evaluation: F_b into sums[6]; with d_df,
// the bridge gradient added to d_df and sums[3..5] recomputed over the final gradient.
int launch_fmt(mdft_handle *h, const double *d_xi, double *d_df, const double *dvec) {
    const FmtArgs &a = h->fmt_args;
    const unsigned nb = kRedBlocks;
    const long long N = h->g.N;
    double2 *pl = h->fmt_pl.p;
    double *pd = h->fmt_part.p, *stats = pd + 2 * nb, *pphi = stats + 2, *pgr = pphi + 4 * nb;
    int rc;
    k_fmt_density<<<nb, kBrThreads, 0, h->stream>>>(d_xi, h->w.p, a, pl, pd);
    k_fmt_stats<<<1, kBrThreads, 0, h->stream>>>(pd, (int)nb, stats);
    if ((rc = launch_fft_planes(h, pl, 2, -1))) return rc;
    k_fmt_weigh<<<nb, kBrThreads, 0, h->stream>>>(pl, h->fmt_cs.p, a);
    if ((rc = launch_fft_planes(h, pl + N, 5, +1))) return rc;
    k_fmt_phi<<<nb, kBrThreads, 0, h->stream>>>(pl, a, d_df ? 1 : 0, pphi);
    h->launches += 4;
    if (d_df) {
        if ((rc = launch_fft_planes(h, pl + 2 * N, 4, -1))) return rc;
        k_fmt_combine<<<nb, kBrThreads, 0, h->stream>>>(pl, a);
        if ((rc = launch_fft_planes(h, pl + 6 * N, 1, +1))) return rc;
        h->launches += 1;
    }
    k_fmt_grad<<<nb, kBrThreads, 0, h->stream>>>(d_xi, h->w.p, a, pl, stats, d_df, dvec, pgr);
    k_fmt_finish<<<1, kBrThreads, 0, h->stream>>>(pphi, pgr, (int)nb, stats, a, d_df ? 1 : 0, h->sums.p);
    h->launches += 2;
    return check_cuda(cudaGetLastError(), "bridge launch");
}

int launch_bridge(mdft_handle *h, const double *d_xi, double *d_df, const double *dvec) {
    if (h->fmt) return launch_fmt(h, d_xi, d_df, dvec);
    const Grid &g = h->g;
    const CgbArgs &a = h->cgb_args;
    const unsigned nb = kRedBlocks;
    int rc;
    k_cgb_density<<<nb, kBrThreads, 0, h->stream>>>(d_xi, h->w.p, a, h->cgb_dens.p, h->cgb_a.p);
    if ((rc = launch_fft_planes(h, h->cgb_a.p, 1, -1))) return rc;
    k_cgb_cmul<<<nb, kBrThreads, 0, h->stream>>>(h->cgb_a.p, h->cgb_kk.p, g.N);
    if ((rc = launch_fft_planes(h, h->cgb_a.p, 1, +1))) return rc;
    k_cgb_phi<<<nb, kBrThreads, 0, h->stream>>>(h->cgb_a.p, h->cgb_dens.p, a, d_df ? 1 : 0, h->cgb_b.p, h->cgb_part.p);
    h->launches += 4;
    if (d_df) {
        if ((rc = launch_fft_planes(h, h->cgb_b.p, 1, -1))) return rc;
        k_cgb_cmul<<<nb, kBrThreads, 0, h->stream>>>(h->cgb_b.p, h->cgb_kk.p, g.N);
        if ((rc = launch_fft_planes(h, h->cgb_b.p, 1, +1))) return rc;
        k_cgb_grad<<<nb, kBrThreads, 0, h->stream>>>(d_xi, h->w.p, a, h->cgb_a.p, h->cgb_b.p, h->cgb_dens.p, d_df, dvec,
                                                     h->cgb_part.p + kRedBlocks);
        h->launches += 2;
    }
    k_cgb_finish<<<1, kBrThreads, 0, h->stream>>>(h->cgb_part.p, kRedBlocks, h->cgb_part.p + kRedBlocks, d_df ? kRedBlocks : 0,
                                                  h->sums.p);
    h->launches += 1;
    return check_cuda(cudaGetLastError(), "bridge launch");
}

// S1 on CUDA cores, FP64 point: the bulk-copy projection where it fits and xi is 16-byte
// aligned, else the tiled one.
template <typename T>
void launch_project_cc(mdft_handle *h, const double *d_xi, const T *A, typename Cplx<T>::t *planes, const AngularArgs &aa) {
    const Grid &g = h->g;
    if ((sizeof(T) == 8 ? h->pt_ok64 : h->pt_ok32) && ((uintptr_t)d_xi & 15u) == 0) {
        const int ntiles = (int)(g.N / kPtBM);
        k_project_tma<T><<<std::min(ntiles, h->nsm), 256, project_tma_smem_bytes<T>(g.np, g.no), h->stream>>>(d_xi, A, planes,
                                                                                                             h->kerr.p, aa, ntiles);
    } else if (h->bm_project == 64)
        k_project<T, 64><<<(unsigned)h->nblk_project, kAngThreads, project_smem_bytes<T>(64, g.no), h->stream>>>(d_xi, A, planes, aa);
    else
        k_project<T, 32><<<(unsigned)h->nblk_project, kAngThreads, project_smem_bytes<T>(32, g.no), h->stream>>>(d_xi, A, planes, aa);
}

// S7 + ideal/external on CUDA cores, FP64 point and gradient: the bulk-copy gather with
// gt_ncol column groups (gt_ncol > 0), else the tiled one.  Returns the number of partial
// rows k_reduce_sums folds.
template <typename T>
long long launch_gather_cc(mdft_handle *h, const typename Cplx<T>::t *planes, const T *B, const double *d_xi, double *d_df,
                           const GatherArgs &ga, int gt_ncol) {
    const Grid &g = h->g;
    if (gt_ncol > 0) {
        const int ntiles = (int)(g.N / gt_bm<T>());
        const int grid = std::min(ntiles, h->nsm * (sizeof(T) == 8 ? 1 : 2));
        const size_t smem = gather_tma_smem_bytes<T>(g.np, g.no, gt_ncol);
        if (gt_ncol == 1)
            k_gather_tma<T, 1, double><<<grid, kGtThreads, smem, h->stream>>>(planes, B, d_xi, h->vext.p, h->w.p, d_df, h->partial.p, h->kerr.p, ga, ntiles);
        else if (gt_ncol == 2)
            k_gather_tma<T, 2, double><<<grid, kGtThreads, smem, h->stream>>>(planes, B, d_xi, h->vext.p, h->w.p, d_df, h->partial.p, h->kerr.p, ga, ntiles);
        else
            k_gather_tma<T, 3, double><<<grid, kGtThreads, smem, h->stream>>>(planes, B, d_xi, h->vext.p, h->w.p, d_df, h->partial.p, h->kerr.p, ga, ntiles);
        return grid;
    }
    if (h->bm_gather == 64)
        k_gather<T, 64><<<(unsigned)h->nblk_gather, kAngThreads, gather_smem_bytes<T>(64, g.np), h->stream>>>(
            planes, B, d_xi, h->vext.p, h->w.p, d_df, h->partial.p, ga);
    else
        k_gather<T, 32><<<(unsigned)h->nblk_gather, kAngThreads, gather_smem_bytes<T>(32, g.np), h->stream>>>(
            planes, B, d_xi, h->vext.p, h->w.p, d_df, h->partial.p, ga);
    return h->nblk_gather;
}

// The excess-term pipeline plus (optionally) the ideal/external term on device
// arrays, in precision T; leaves {F_id, F_ext, sum_exc, df.dvec, max|df|} in h->sums.
template <typename T>
int run_pipeline_t(mdft_handle *h, const void *xin, double *d_df, int do_ideal, int df_mode, const void *dvec, bool vec32,
                   bool x32) {
    using C = typename Cplx<T>::t;
    const double *d_xi = static_cast<const double *>(xin);  // FP64 point unless x32
    const Grid &g = h->g;
    const bool dbl = sizeof(T) == 8;
    if (has_bridge(h) && do_ideal && (!dbl || vec32 || x32)) {
        set_error("the bridge term is evaluated in FP64 only (an FP64 handle and FP64 solves)");
        return MDFT_E_STATE;
    }
    C *planes = dbl ? (C *)h->planes.p : (C *)h->planes32.p;
    const T *A = dbl ? (const T *)h->A.p : (const T *)h->A32.p;
    const T *B = dbl ? (const T *)h->B.p : (const T *)h->B32.p;
    const C *ctab = dbl ? (const C *)h->ctab.p : (const C *)h->ctab32.p;
    const void *tw[3];
    for (int ax = 0; ax < 3; ++ax) tw[ax] = dbl ? (const void *)h->tw64[ax].p : (const void *)h->tw32[ax].p;
    stage_mark(h, 0);
    AngularArgs aa{g.N, g.no, g.np, g.rho0};
    if (x32 && (dbl || (!h->pt_ok32 && !h->um_ok) || !h->vext32.p || ((uintptr_t)xin & 15u) != 0)) {
        set_error("an FP32 point needs the FP32 bulk-copy kernels");
        return MDFT_E_STATE;
    }
    const bool umma = !dbl && h->um_ok;
    if (umma) {
        // tensor-core projection (split BF16); FP32 point in the FP32 phase, else the FP64 xi
        const int ntiles = (int)(g.N / kUmBM);
        const unsigned grid = (unsigned)std::min(ntiles, h->um_grid_p);
        const size_t smem = umma_smem_bytes(h->um_ps);
        const bool vec = g.no % 4 == 0 && ((uintptr_t)xin & 15u) == 0;
        if (x32 && h->ring_p) {
            const unsigned rgrid = (unsigned)std::min(ntiles, h->nsm);
            const size_t rsmem = project_ring_smem_bytes(h->um_ps, g.no);
            if (vec) k_project_ring<4><<<rgrid, kRingThreads, rsmem, h->stream>>>(static_cast<const float *>(xin), h->um_pimg.p, (float2 *)planes, h->kerr.p, aa, h->um_ps, ntiles);
            else k_project_ring<1><<<rgrid, kRingThreads, rsmem, h->stream>>>(static_cast<const float *>(xin), h->um_pimg.p, (float2 *)planes, h->kerr.p, aa, h->um_ps, ntiles);
        } else if (x32) {
            if (vec) k_project_umma<float, 4><<<grid, kPjThreads, smem, h->stream>>>(static_cast<const float *>(xin), h->um_pimg.p, (float2 *)planes, h->kerr.p, aa, h->um_ps, ntiles);
            else k_project_umma<float, 1><<<grid, kPjThreads, smem, h->stream>>>(static_cast<const float *>(xin), h->um_pimg.p, (float2 *)planes, h->kerr.p, aa, h->um_ps, ntiles);
        } else {
            if (vec) k_project_umma<double, 4><<<grid, kPjThreads, smem, h->stream>>>(d_xi, h->um_pimg.p, (float2 *)planes, h->kerr.p, aa, h->um_ps, ntiles);
            else k_project_umma<double, 1><<<grid, kPjThreads, smem, h->stream>>>(d_xi, h->um_pimg.p, (float2 *)planes, h->kerr.p, aa, h->um_ps, ntiles);
        }
    } else if (x32) {
        const int ntiles = (int)(g.N / kPtBM);
        k_project_tma<float, float><<<std::min(ntiles, h->pt_grid_x32), 256, project_tma_smem_bytes<float, float>(g.np, g.no), h->stream>>>(
            static_cast<const float *>(xin), (const float *)A, (float2 *)planes, h->kerr.p, aa, ntiles);
    } else {
        launch_project_cc<T>(h, d_xi, A, planes, aa);
    }
    int rc = check_cuda(cudaGetLastError(), "project launch");
    if (rc) return rc;
    stage_mark(h, 1);
    if ((rc = launch_fft_t<T>(h, planes, tw, +1))) return rc;
    stage_mark(h, 2);
    Oz2Args oz = h->oz;
    oz.quirks = dbl ? 1 : 0;
    const int ozw = dbl ? h->oz_warps : h->oz_warps32;
    if (!dbl && h->ozp_ok)
        launch_ozp(h, (float2 *)planes, (const float2 *)ctab, oz);
    else
        k_oz2<T><<<dbl ? h->oz_grid : h->oz_grid32, 32 * ozw, dbl ? h->oz_smem : h->oz_smem32, h->stream>>>(planes, ctab, h->oz_ints.p,
                                                                                                           h->oz_dbls.p, oz, nullptr, OzMix{});
    if ((rc = check_cuda(cudaGetLastError(), "oz launch"))) return rc;
    stage_mark(h, 3);
    if ((rc = launch_fft_t<T>(h, planes, tw, -1))) return rc;
    stage_mark(h, 4);
    const GatherArgs ga = gather_args(h, d_df ? df_mode : 0, do_ideal, dvec, 1.0);
    const int gt_ncol = dbl ? h->gt_ncol64 : h->gt_ncol32;
    auto al16 = [](const void *p) { return ((uintptr_t)p & 15u) == 0; };
    long long red_blocks = h->nblk_gather;
    const bool tma_gather = gt_ncol > 0 && ga.df_mode != 2 && al16(d_xi) && al16(dvec);
    const bool umma_gather = umma && ga.df_mode != 2;
    if ((vec32 || x32) && !tma_gather && !umma_gather) {
        set_error("FP32 gradient vectors need the bulk-copy gather");
        return MDFT_E_STATE;
    }
    if (umma_gather) {
        // tensor-core gather (split BF16) with the FP32 element-wise epilogue
        const int ntiles = (int)(g.N / kUmBM);
        const int grid = std::min(ntiles, h->um_grid_g);
        const size_t smem = gather_umma_smem_bytes(h->um_gs, g.no);
        const float2 *pl = (const float2 *)planes;
        // 4-element vector epilogue with a compile-time orientation count (mmax 3, water), else scalar
        const bool v84 = g.no == 84 && al16(xin) && al16(dvec) && al16(d_df);
        float *df32 = reinterpret_cast<float *>(d_df);
        const float *x32p = static_cast<const float *>(xin);
        if (x32 && v84 && h->ring_g) {
            const int rgrid = std::min(ntiles, h->nsm);
            const size_t rs = gather_ring_smem_bytes(h->um_gs, 84);
            constexpr int rt = gather_ring_block<84>();
            k_gather_ring<84><<<rgrid, rt, rs, h->stream>>>(pl, h->um_gimg.p, x32p, h->vext32.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, h->um_gs, ntiles);
            red_blocks = rgrid;
        } else if (x32 && v84)
            k_gather_umma<float, float, 84><<<grid, kUmThreads, smem, h->stream>>>(pl, h->um_gimg.p, x32p, h->vext32.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, h->um_gs, ntiles);
        else if (x32)
            k_gather_umma<float, float, 0><<<grid, kUmThreads, smem, h->stream>>>(pl, h->um_gimg.p, x32p, h->vext32.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, h->um_gs, ntiles);
        else if (vec32 && v84)
            k_gather_umma<double, float, 84><<<grid, kUmThreads, smem, h->stream>>>(pl, h->um_gimg.p, d_xi, h->vext.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, h->um_gs, ntiles);
        else if (vec32)
            k_gather_umma<double, float, 0><<<grid, kUmThreads, smem, h->stream>>>(pl, h->um_gimg.p, d_xi, h->vext.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, h->um_gs, ntiles);
        else if (v84)
            k_gather_umma<double, double, 84><<<grid, kUmThreads, smem, h->stream>>>(pl, h->um_gimg.p, d_xi, h->vext.p, h->w.p, d_df, h->partial.p, h->kerr.p, ga, h->um_gs, ntiles);
        else
            k_gather_umma<double, double, 0><<<grid, kUmThreads, smem, h->stream>>>(pl, h->um_gimg.p, d_xi, h->vext.p, h->w.p, d_df, h->partial.p, h->kerr.p, ga, h->um_gs, ntiles);
        if (!(x32 && v84 && h->ring_g)) red_blocks = grid;
    } else if (tma_gather && (x32 || vec32)) {
        const int ntiles = (int)(g.N / gt_bm<T>());
        const int grid = std::min(ntiles, h->nsm * (dbl ? 1 : 2));
        const size_t smem = gather_tma_smem_bytes<T>(g.np, g.no, gt_ncol);
        if (x32) {
            // FP32 phase of a mixed solve: point, vext, gradient and direction in FP32
            float *df32 = reinterpret_cast<float *>(d_df);
            const float *x32p = static_cast<const float *>(xin);
            const float2 *pl = (const float2 *)planes;
            const float *B32 = (const float *)B;
            if (gt_ncol == 1)
                k_gather_tma<float, 1, float, float><<<grid, kGtThreads, smem, h->stream>>>(pl, B32, x32p, h->vext32.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, ntiles);
            else if (gt_ncol == 2)
                k_gather_tma<float, 2, float, float><<<grid, kGtThreads, smem, h->stream>>>(pl, B32, x32p, h->vext32.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, ntiles);
            else
                k_gather_tma<float, 3, float, float><<<grid, kGtThreads, smem, h->stream>>>(pl, B32, x32p, h->vext32.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, ntiles);
        } else {
            float *df32 = reinterpret_cast<float *>(d_df);
            if (gt_ncol == 1)
                k_gather_tma<T, 1, float><<<grid, kGtThreads, smem, h->stream>>>(planes, B, d_xi, h->vext.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, ntiles);
            else if (gt_ncol == 2)
                k_gather_tma<T, 2, float><<<grid, kGtThreads, smem, h->stream>>>(planes, B, d_xi, h->vext.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, ntiles);
            else
                k_gather_tma<T, 3, float><<<grid, kGtThreads, smem, h->stream>>>(planes, B, d_xi, h->vext.p, h->w.p, df32, h->partial.p, h->kerr.p, ga, ntiles);
        }
        red_blocks = grid;
    } else {
        red_blocks = launch_gather_cc<T>(h, planes, B, d_xi, d_df, ga, tma_gather ? gt_ncol : 0);
    }
    if ((rc = check_cuda(cudaGetLastError(), "gather launch"))) return rc;
    k_reduce_sums<<<1, 256, 0, h->stream>>>(h->partial.p, red_blocks, h->sums.p);
    h->launches += 4;  // project, oz, gather, reduce (the FFT launches are counted in launch_fft_t)
    if ((rc = check_cuda(cudaGetLastError(), "reduce launch"))) return rc;
    if (has_bridge(h) && do_ideal && (rc = launch_bridge(h, d_xi, ga.df_mode == 1 ? d_df : nullptr, static_cast<const double *>(dvec))))
        return rc;
    stage_mark(h, 5);
    return MDFT_OK;
}

// dvec (df_mode 1 only): h_sums[3] = df.dvec, h_sums[4] = max|df| after finish_sums.
// vec32 (bulk-copy gather only): df and dvec are FP32 vectors (the minimiser's mixed solves);
// x32 (FP32 evaluations, with vec32): the point is FP32 too and vext is read from h->vext32.
// The pipeline is a fixed sequence of launches for given buffers and flags: it runs as a CUDA
// graph captured on first use (one graph launch instead of about a dozen kernel launches per
// evaluation), falling back to direct launches when capture is not possible.
constexpr size_t kMaxPipeGraphs = 8;
void drop_pipe_graphs(mdft_handle *h) {
    for (auto &pg : h->pipe_graphs) cudaGraphExecDestroy(pg.exec);
    h->pipe_graphs.clear();
}
int run_pipeline(mdft_handle *h, const void *d_xi, double *d_df, int do_ideal, int df_mode, const void *dvec = nullptr,
                 bool vec32 = false, bool x32 = false) {
    auto direct = [&]() {
        if (h->eval_prec == MDFT_PREC_MIXED) return run_pipeline_t<float>(h, d_xi, d_df, do_ideal, df_mode, dvec, vec32, x32);
        return run_pipeline_t<double>(h, d_xi, d_df, do_ideal, df_mode, dvec, vec32, x32);
    };
    if (!h->graphs_on || h->timing) return direct();
    for (auto &pg : h->pipe_graphs)
        if (pg.x == d_xi && pg.g == d_df && pg.dvec == dvec && pg.do_ideal == do_ideal && pg.df_mode == df_mode &&
            pg.prec == h->eval_prec && pg.v32 == vec32 && pg.x32 == x32 && pg.vext == h->vext.p && pg.vext32 == h->vext32.p) {
            h->launches += pg.nlaunch;
            return check_cuda(cudaGraphLaunch(pg.exec, h->stream), "pipeline graph launch");
        }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return direct();  // inside a caller's capture: launch into it
    }
    const long long l0 = h->launches;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return direct();
    }
    const int rc = direct();
    const long long nl = h->launches - l0;  // counted during capture; nothing has run yet
    h->launches = l0;
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    const bool ok = rc == 0 && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (rc) return rc;  // a launch was refused (nothing ran)
    if (!ok) {
        h->graphs_on = false;  // this handle's pipeline does not capture: launch directly from now on
        return direct();
    }
    if (h->pipe_graphs.size() >= kMaxPipeGraphs) {
        cudaGraphExecDestroy(h->pipe_graphs.front().exec);
        h->pipe_graphs.erase(h->pipe_graphs.begin());
    }
    h->pipe_graphs.push_back(mdft_handle::PipeGraph{d_xi, dvec, h->vext.p, h->vext32.p, d_df, do_ideal, df_mode, h->eval_prec, vec32, x32, exec, nl});
    h->launches += nl;
    return check_cuda(cudaGraphLaunch(exec, h->stream), "pipeline graph launch");
}

int finish_sums(mdft_handle *h, double *fid, double *fext, double *fexc) {
    // {F_id, F_ext, sum_exc, df.dvec, max|df|, sum w df, F_b, bridge error}
    int rc = check_cuda(cudaMemcpyAsync(h->h_sums, h->sums.p, (kGatherSums + 2) * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "sums copy");
    if (rc) return rc;
    if ((rc = check_cuda(cudaMemcpyAsync(h->h_kerr, h->kerr.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "flag copy"))) return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "evaluation"))) return rc;
    if (*h->h_kerr) {
        cudaMemsetAsync(h->kerr.p, 0, sizeof(int), h->stream);
        set_error("a pipeline wait in the projection or gather timed out (bulk copy never completed)");
        return MDFT_E_CUDA;
    }
    if (h->fmt && h->h_sums[7] != 0.0) {
        const int code = (int)h->h_sums[7];
        cudaMemsetAsync(h->sums.p + 7, 0, sizeof(double), h->stream);
        set_error(code == 1 ? "hard-sphere bridge: a weighted density n3 >= 1 (log(1 - n3) undefined)"
                  : code == 2 ? "hard-sphere bridge (CS): a weighted density n3 <= 0"
                              : "hard-sphere bridge: 1 - n3 or n3 at zero in the gradient");
        return MDFT_E_NUMERIC;
    }
    if (h->timing) {
        for (int i = 0; i < ST_COUNT; ++i) {
            float ms = 0;
            cudaEventElapsedTime(&ms, h->ev[i], h->ev[i + 1]);
            h->stage_ms[i] += ms;
        }
        h->stage_count++;
    }
    *fid = h->h_sums[0];
    *fext = h->h_sums[1];
    *fexc = h->h_sums[2] * 0.5 * h->g.dv;
    if (!std::isfinite(*fid) || !std::isfinite(*fext) || !std::isfinite(*fexc)) {
        set_error("non-finite functional (F_id=%g F_ext=%g F_exc=%g)", *fid, *fext, *fexc);
        return MDFT_E_NUMERIC;
    }
    return 0;
}

double combine(const mdft_handle *h, double fid, double fext, double fexc) {
    // src/module_energy_and_gradient.f90:89-217
    double f = 0.0;
    f = f + fid + fext;
    f = f + fexc;
    f = f + (has_bridge(h) ? h->h_sums[6] : 0.0);  // bridge: F_b of this evaluation ("no": 0)
    f = f + h->const_corr;
    return f;
}

// create-time tuning of the FP32 kernel forms (defined with the solver, solve.cuh)
int autotune_at_create(mdft_handle *h);

}  // namespace

// -------------------------------------------------------------------------
extern "C" {

const char *mdft_last_error(void) { return last_error(); }

int mdft_create(const mdft_desc *d, mdft_handle **out) {
    if (!d || !out) { set_error("null argument"); return MDFT_E_ARG; }
    *out = nullptr;
    if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0 || (d->nx & 1) || (d->ny & 1) || (d->nz & 1)) {
        set_error("grid sizes must be positive and even (got %d %d %d)", d->nx, d->ny, d->nz);
        return MDFT_E_ARG;
    }
    if (!(d->lx > 0 && d->ly > 0 && d->lz > 0)) { set_error("box lengths must be positive"); return MDFT_E_ARG; }
    if (d->mmax < 0 || d->mmax > kMaxMmax) { set_error("mmax must be in [0, %d]", kMaxMmax); return MDFT_E_ARG; }
    if (d->mrso < 1) { set_error("mrso must be >= 1"); return MDFT_E_ARG; }
    if (!(d->temperature > 0) || !(d->n0 > 0)) { set_error("temperature and n0 must be positive"); return MDFT_E_ARG; }
    if (d->precision != MDFT_PREC_FP64 && d->precision != MDFT_PREC_MIXED) { set_error("unknown precision %d", d->precision); return MDFT_E_ARG; }
    std::unique_ptr<mdft_handle> h(new mdft_handle());
    {
        const char *tr = std::getenv("MDFT_TRACE");
        h->trace = tr && tr[0] && tr[0] != '0';
        const char *gr = std::getenv("MDFT_GRAPHS");
        h->graphs_on = !(gr && std::strcmp(gr, "0") == 0);
    }
    h->precision = d->precision;
    h->device = d->device;
    // host-side set-up first: argument and c(k) errors do not depend on the device
    const double kT = kBoltz * kNavo * d->temperature * 1.0e-3;  // src/module_thermo.f90:62
    if (build_grid(h->g, d->nx, d->ny, d->nz, d->lx, d->ly, d->lz, d->mmax, d->mrso, kT, d->n0)) return MDFT_E_ARG;
    const Grid &g = h->g;
    if (g.np > kMaxNpConst) { set_error("too many projections (%d)", g.np); return MDFT_E_ARG; }
    {
        FftPlan1D tmp;
        const int dims[3] = {d->nx, d->ny, d->nz};
        for (int ax = 0; ax < 3; ++ax)
            if (!make_plan1d(dims[ax], tmp)) { set_error("grid size %d is not of the form 2^a 3^b", dims[ax]); return MDFT_E_ARG; }
    }
    if (read_ctable(g, d->ck_path, h->ct)) return MDFT_E_IO;
    int rc = check_cuda(cudaSetDevice(d->device), "cudaSetDevice");
    if (rc) return rc;
    if ((rc = check_cuda(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream"))) return rc;
    for (int i = 0; i <= ST_COUNT; ++i)
        if ((rc = check_cuda(cudaEventCreate(&h->ev[i]), "event"))) return rc;
    const size_t nf = (size_t)g.N * g.no;
    if ((rc = alloc_check(h->xi.alloc(nf), "xi", nf * 8))) return rc;
    if ((rc = alloc_check(h->vext.alloc(nf), "vext", nf * 8))) return rc;
    if ((rc = alloc_check(h->df.alloc(nf), "df", nf * 8))) return rc;
    if ((rc = alloc_check(h->planes.alloc((size_t)g.np * g.N), "projection planes", (size_t)g.np * g.N * 16))) return rc;
    if ((rc = check_cuda(cudaMemsetAsync(h->vext.p, 0, nf * 8, h->stream), "vext clear"))) return rc;
    std::vector<double> A, B;
    build_angular_matrices(g, A, B);
    if ((rc = alloc_check(h->A.alloc(A.size()), "A", A.size() * 8))) return rc;
    if ((rc = alloc_check(h->B.alloc(B.size()), "B", B.size() * 8))) return rc;
    if ((rc = alloc_check(h->w.alloc(g.no), "w", g.no * 8))) return rc;
    cudaMemcpy(h->A.p, A.data(), A.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(h->B.p, B.data(), B.size() * 8, cudaMemcpyHostToDevice);
    {
        std::vector<float> A32(A.begin(), A.end()), B32(B.begin(), B.end());
        if ((rc = alloc_check(h->A32.alloc(A32.size()), "A32", A32.size() * 4))) return rc;
        if ((rc = alloc_check(h->B32.alloc(B32.size()), "B32", B32.size() * 4))) return rc;
        cudaMemcpy(h->A32.p, A32.data(), A32.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(h->B32.p, B32.data(), B32.size() * 4, cudaMemcpyHostToDevice);
        if ((rc = alloc_check(h->planes32.alloc((size_t)g.np * g.N), "FP32 projection planes", (size_t)g.np * g.N * 8))) return rc;
    }
    cudaMemcpy(h->w.p, g.w.data(), g.no * 8, cudaMemcpyHostToDevice);
    if ((rc = alloc_check(h->ctab.alloc((size_t)h->ct.nq * h->ct.ncoef), "c table", h->ct.c.size() * 8))) return rc;
    cudaMemcpy(h->ctab.p, h->ct.c.data(), h->ct.c.size() * 8, cudaMemcpyHostToDevice);
    {
        std::vector<float> c32(h->ct.c.begin(), h->ct.c.end());
        if ((rc = alloc_check(h->ctab32.alloc((size_t)h->ct.nq * h->ct.ncoef), "FP32 c table", c32.size() * 4))) return rc;
        cudaMemcpy(h->ctab32.p, c32.data(), c32.size() * 4, cudaMemcpyHostToDevice);
    }
    if ((rc = check_cuda(cudaGetLastError(), "table upload"))) return rc;
    // launch shapes
    int maxsmem = 0;
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->device);
    const size_t dyn_max = (size_t)maxsmem - 1024;  // static shared memory of these kernels is < 1 KB
    h->bm_project = project_smem_bytes<double>(64, g.no) <= dyn_max ? 64 : 32;
    h->bm_gather = gather_smem_bytes<double>(64, g.np) <= dyn_max ? 64 : 32;
    if (project_smem_bytes<double>(h->bm_project, g.no) > dyn_max || gather_smem_bytes<double>(h->bm_gather, g.np) > dyn_max) {
        set_error("angular transform tiles do not fit in shared memory");
        return MDFT_E_ARG;
    }
    {
        const void *fns[] = {(const void *)k_project<double, 64>, (const void *)k_project<double, 32>,
                             (const void *)k_gather<double, 64>,  (const void *)k_gather<double, 32>,
                             (const void *)k_project<float, 64>,  (const void *)k_project<float, 32>,
                             (const void *)k_gather<float, 64>,   (const void *)k_gather<float, 32>,
                             (const void *)k_fft_axis<double>,    (const void *)k_fft_axis<float>,
                             (const void *)k_oz2<double>,         (const void *)k_oz2<float>};
        for (const void *fn : fns)
            if ((rc = allow_smem(fn, maxsmem))) return rc;
    }
    for (int n : {g.nx, g.nz}) {
        cudaError_t e[4] = {fft_xy<double>(n, nullptr, 0, nullptr, 1, nullptr, true),
                            fft_z<double>(n, nullptr, 0, g.nx, g.ny, nullptr, 1, nullptr, true),
                            fft_xy<float>(n, nullptr, 0, nullptr, 1, nullptr, true),
                            fft_z<float>(n, nullptr, 0, g.nx, g.ny, nullptr, 1, nullptr, true)};
        for (cudaError_t x : e)
            if (x != cudaSuccess && x != cudaErrorNotSupported) return check_cuda(x, "fft attribute");
        cudaGetLastError();
    }
    h->nblk_project = (g.N + h->bm_project - 1) / h->bm_project;
    h->nblk_gather = (g.N + h->bm_gather - 1) / h->bm_gather;
    cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, d->device);
    h->xy_grid_cap64 = h->nsm * std::max(1, xy_tma_per_sm<double>(g.nx));
    h->xy_grid_cap32 = h->nsm * std::max(1, xy_tma_per_sm<float>(g.nx));
    {
        // persistent bulk-copy gather: N in whole 32-point tiles, no <= 96, stages that fit
        const int ncol = (g.no + 31) / 32;
        const bool shape_ok = g.N % kGtBM == 0 && ncol <= 3;  // kGtBM32 divides kGtBM
        h->gt_ncol64 = (shape_ok && gather_tma_smem_bytes<double>(g.np, g.no, ncol) <= dyn_max) ? ncol : 0;
        h->gt_ncol32 = (shape_ok && gather_tma_smem_bytes<float>(g.np, g.no, ncol) <= dyn_max) ? ncol : 0;
        // persistent bulk-copy projection: N in whole 64-point tiles, np <= 32
        const bool pshape = g.N % kPtBM == 0 && g.np <= 32;
        h->pt_ok64 = pshape && project_tma_smem_bytes<double>(g.np, g.no) <= dyn_max;
        h->pt_ok32 = pshape && project_tma_smem_bytes<float>(g.np, g.no) <= dyn_max;
        if ((rc = allow_smem((const void *)k_project_tma<double>, maxsmem))) return rc;
        if ((rc = allow_smem((const void *)k_project_tma<float>, maxsmem))) return rc;
        if ((rc = allow_smem((const void *)k_project_tma<float, float>, maxsmem))) return rc;
        {
            int b = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_project_tma<float, float>, 256,
                                                          project_tma_smem_bytes<float, float>(g.np, g.no));
            h->pt_grid_x32 = h->nsm * std::max(1, b);
        }
        const void *fns[] = {(const void *)k_gather_tma<double, 1, double>, (const void *)k_gather_tma<double, 2, double>,
                             (const void *)k_gather_tma<double, 3, double>, (const void *)k_gather_tma<float, 1, double>,
                             (const void *)k_gather_tma<float, 2, double>,  (const void *)k_gather_tma<float, 3, double>,
                             (const void *)k_gather_tma<double, 1, float>,  (const void *)k_gather_tma<double, 2, float>,
                             (const void *)k_gather_tma<double, 3, float>,  (const void *)k_gather_tma<float, 1, float>,
                             (const void *)k_gather_tma<float, 2, float>,   (const void *)k_gather_tma<float, 3, float>,
                             (const void *)k_gather_tma<float, 1, float, float>, (const void *)k_gather_tma<float, 2, float, float>,
                             (const void *)k_gather_tma<float, 3, float, float>};
        for (const void *fn : fns)
            if ((rc = allow_smem(fn, maxsmem))) return rc;
    }
    {
        // tensor-core angular contractions for FP32 evaluations: N in whole 128-point tiles,
        // no <= 96, 2np <= 64 (mmax <= 3 for water); MDFT_ANGULAR=ffma keeps the FFMA kernels
        const char *ang = std::getenv("MDFT_ANGULAR");
        const bool want = !(ang && std::strcmp(ang, "ffma") == 0);
        // "umma": register forms only; "ring": the bulk-copy ring forms of both contractions;
        // default: register projection (measured faster) and ring gather
        const bool want_ring = !(ang && std::strcmp(ang, "umma") == 0);
        const bool want_ring_p = ang && std::strcmp(ang, "ring") == 0;
        h->um_ps = umma_shape(g.no, 2 * g.np);
        h->um_gs = umma_shape(2 * g.np, g.no);
        if (want && g.N % kUmBM == 0 && h->um_ps.Kp <= 96 && h->um_gs.Kp <= 64 &&
            gather_umma_smem_bytes(h->um_gs, g.no) <= dyn_max && umma_smem_bytes(h->um_ps) <= dyn_max) {
            std::vector<uint16_t> pimg, gimg;
            const int np2 = 2 * g.np, no = g.no;
            pack_split_bf16(h->um_ps.Np, h->um_ps.Kp, [&](int n, int io) { return (n < np2 && io < no) ? A[(size_t)io * np2 + n] : 0.0; }, pimg);
            pack_split_bf16(h->um_gs.Np, h->um_gs.Kp, [&](int io, int k) { return (io < no && k < np2) ? B[(size_t)k * no + io] : 0.0; }, gimg);
            if ((rc = alloc_check(h->um_pimg.alloc(pimg.size()), "angular operand images", pimg.size() * 2))) return rc;
            if ((rc = alloc_check(h->um_gimg.alloc(gimg.size()), "angular operand images", gimg.size() * 2))) return rc;
            cudaMemcpy(h->um_pimg.p, pimg.data(), pimg.size() * 2, cudaMemcpyHostToDevice);
            cudaMemcpy(h->um_gimg.p, gimg.data(), gimg.size() * 2, cudaMemcpyHostToDevice);
            const void *pf[] = {(const void *)k_project_umma<float, 4>, (const void *)k_project_umma<float, 1>,
                                (const void *)k_project_umma<double, 4>, (const void *)k_project_umma<double, 1>};
            const void *gf[] = {(const void *)k_gather_umma<float, float, 84>, (const void *)k_gather_umma<double, float, 84>,
                                (const void *)k_gather_umma<double, double, 84>, (const void *)k_gather_umma<float, float, 0>,
                                (const void *)k_gather_umma<double, float, 0>, (const void *)k_gather_umma<double, double, 0>};
            for (const void *fn : pf)
                if ((rc = allow_smem(fn, maxsmem))) return rc;
            for (const void *fn : gf)
                if ((rc = allow_smem(fn, maxsmem))) return rc;
            int bp = 0, bg = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bp, k_project_umma<float, 4>, kPjThreads, umma_smem_bytes(h->um_ps));
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bg, k_gather_umma<float, float, 84>, kUmThreads,
                                                          gather_umma_smem_bytes(h->um_gs, g.no));
            h->um_grid_p = h->nsm * std::max(1, bp);
            h->um_grid_g = h->nsm * std::max(1, bg);
            h->um_ok = true;
            h->ring_p_ok = project_ring_smem_bytes(h->um_ps, g.no) <= dyn_max;
            h->ring_g_ok = g.no == 84 && gather_ring_smem_bytes(h->um_gs, 84) <= dyn_max;
            h->ring_p = want_ring_p && h->ring_p_ok;
            h->ring_g = want_ring && h->ring_g_ok;
            if (h->ring_p_ok) {
                if ((rc = allow_smem((const void *)k_project_ring<4>, maxsmem))) return rc;
                if ((rc = allow_smem((const void *)k_project_ring<1>, maxsmem))) return rc;
            }
            if (h->ring_g_ok && (rc = allow_smem((const void *)k_gather_ring<84>, maxsmem))) return rc;
            // the FP32 forms are measured on the first FP32 phase unless chosen in the environment
            const char *at = std::getenv("MDFT_AUTOTUNE");
            h->tune_on = !(at && std::strcmp(at, "0") == 0) && !ang && !std::getenv("MDFT_OZ");
        }
    }
    {
        const size_t rows = std::max<long long>({h->nblk_gather, 2LL * h->nsm, (long long)h->um_grid_g});
        if ((rc = alloc_check(h->partial.alloc(kGatherSums * rows), "partials", 8 * kGatherSums * rows))) return rc;
    }
    if ((rc = alloc_check(h->kerr.alloc(1), "error flag", 4))) return rc;
    cudaMemset(h->kerr.p, 0, sizeof(int));
    if ((rc = check_cuda(cudaMallocHost(&h->h_kerr, sizeof(int)), "pinned flag"))) return rc;
    if ((rc = alloc_check(h->sums.alloc(8), "sums", 64))) return rc;
    cudaMemset(h->sums.p, 0, 8 * sizeof(double));
    if ((rc = check_cuda(cudaMallocHost(&h->h_sums, 8 * sizeof(double)), "pinned sums"))) return rc;
    if ((rc = alloc_check(h->vpart.alloc((size_t)kMaxRows * kRedBlocks), "reduction partials", 8 * kMaxRows * kRedBlocks))) return rc;
    if ((rc = alloc_check(h->vsc.alloc(kScalarSlots), "reduction scalars", 8 * kScalarSlots))) return rc;
    if ((rc = check_cuda(cudaMallocHost(&h->h_vsc, sizeof(double) * kScalarSlots), "pinned scalars"))) return rc;
    if ((rc = setup_fft(h.get()))) return rc;
    for (int ax = 0; ax < 3; ++ax)
        if (h->fft[ax].smem > (size_t)maxsmem) { set_error("FFT tile does not fit in shared memory"); return MDFT_E_ARG; }
    {
        OzTables tb;
        if (!build_oz_tables(g, h->ct, tb)) { set_error("OZ term tables exceed their index encoding"); return MDFT_E_ARG; }
        if ((rc = alloc_check(h->oz_ints.alloc(tb.ints.size()), "OZ tables", tb.ints.size() * 4))) return rc;
        if ((rc = alloc_check(h->oz_dbls.alloc(std::max<size_t>(1, tb.dbls.size())), "OZ tables", tb.dbls.size() * 8))) return rc;
        cudaMemcpy(h->oz_ints.p, tb.ints.data(), tb.ints.size() * 4, cudaMemcpyHostToDevice);
        if (!tb.dbls.empty()) cudaMemcpy(h->oz_dbls.p, tb.dbls.data(), tb.dbls.size() * 8, cudaMemcpyHostToDevice);
        Oz2Args &oz = h->oz;
        oz.nx = g.nx; oz.ny = g.ny; oz.nz = g.nz; oz.N = g.N;
        oz.nk = (long long)g.nx * g.ny * (g.nz / 2 + 1);
        oz.mmax = g.mmax; oz.np = g.np; oz.ncoef = h->ct.ncoef; oz.nq = h->ct.nq; oz.dq = h->ct.dq;
        oz.twopi_lx = 2.0 * kPi / g.lx; oz.twopi_ly = 2.0 * kPi / g.ly; oz.twopi_lz = 2.0 * kPi / g.lz;
        oz.quirks = 1;
        oz.n_ints = (int)tb.ints.size(); oz.n_dbls = (int)tb.dbls.size(); oz.nrot = tb.nrot;
        oz.fwd_off = tb.fwd_off; oz.fwd_terms = tb.fwd_terms; oz.oz_off = tb.oz_off; oz.oz_terms = tb.oz_terms;
        oz.bwd_off = tb.bwd_off; oz.bwd_terms = tb.bwd_terms; oz.sign = tb.sign; oz.lvl_off = tb.lvl_off;
        oz.rec_int = tb.rec_int;
        h->oz_warps = 8;
        while (h->oz_warps > 1 && oz2_smem_bytes<double>(oz, h->oz_warps) > dyn_max) h->oz_warps /= 2;
        h->oz_smem = oz2_smem_bytes<double>(oz, h->oz_warps);
        if (h->oz_smem > dyn_max) { set_error("OZ tile does not fit in shared memory"); return MDFT_E_ARG; }
        // persistent grid: as many CTAs as fit on the device at once (tables staged once per CTA)
        auto oz_grid_of = [&](const void *fn, int warps, size_t smem) {
            int per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * warps, smem);
            const long long groups = (oz.nk + warps - 1) / warps;
            return (int)std::min<long long>(groups, (long long)std::max(1, per_sm) * h->nsm);
        };
        h->oz_grid = oz_grid_of((const void *)k_oz2<double>, h->oz_warps, h->oz_smem);
        h->oz_warps32 = 8;
        while (h->oz_warps32 > 1 && oz2_smem_bytes<float>(oz, h->oz_warps32) > dyn_max) h->oz_warps32 /= 2;
        h->oz_smem32 = oz2_smem_bytes<float>(oz, h->oz_warps32);
        h->oz_grid32 = oz_grid_of((const void *)k_oz2<float>, h->oz_warps32, h->oz_smem32);
        // thread-per-pair FP32 OZ where an instantiation exists and its slice fits
        const void *fn = ozp_kernel(g.mmax, g.mrso);
        if (fn && build_ozp_params(g, h->ct, h->ozp) && ozp_smem_bytes(g.np) <= dyn_max) {
            if ((rc = allow_smem(fn, maxsmem))) return rc;
            h->ozp_ok = true;
            const char *ozsel = std::getenv("MDFT_OZ");
            h->ozd = !(ozsel && std::strcmp(ozsel, "ozp") == 0);
            if ((rc = allow_smem(ozp_kernel(g.mmax, g.mrso, true), maxsmem))) return rc;
            std::vector<float2> c32(h->ct.c.size() / 2);  // the FP32 table as the kernels read it
            for (size_t i = 0; i < c32.size(); ++i) c32[i] = make_float2((float)h->ct.c[2 * i], (float)h->ct.c[2 * i + 1]);
            std::vector<float2> cq = build_ozp_cq(g, h->ct, c32);
            if (!cq.empty()) {
                if ((rc = alloc_check(h->ozp_cq.alloc(cq.size()), "OZ c rows", cq.size() * 8))) return rc;
                cudaMemcpy(h->ozp_cq.p, cq.data(), cq.size() * 8, cudaMemcpyHostToDevice);
            }
        }
    }
    h->eval_prec = h->precision;
    if ((rc = autotune_at_create(h.get()))) return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "create"))) return rc;
    *out = h.release();
    return MDFT_OK;
}

int mdft_destroy(mdft_handle *h) {
    if (!h) return MDFT_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    // an attached warm-start network goes back to its own stream before this one is destroyed
    if (h->warm) mdft_warm_net_set_stream(h->warm, nullptr);
    h->warm = nullptr;
    drop_pipe_graphs(h);
    h->ozp_cq.free();
    h->um_pimg.free();
    h->um_gimg.free();
    h->xi.free(); h->vext.free(); h->vext32.free(); h->df.free(); h->w.free(); h->A.free(); h->B.free();
    h->partial.free(); h->sums.free(); h->planes.free(); h->ctab.free(); h->oz_ints.free(); h->oz_dbls.free();
    for (int i = 0; i < 3; ++i) {
        h->tw64[i].free();
        h->tw32[i].free();
    }
    h->A32.free(); h->B32.free(); h->planes32.free(); h->ctab32.free();
    lbfgs_free(h->lb);
    h->vpart.free();
    h->vsc.free();
    if (h->h_vsc) cudaFreeHost(h->h_vsc);
    if (h->h_sums) cudaFreeHost(h->h_sums);
    if (h->h_kerr) cudaFreeHost(h->h_kerr);
    h->kerr.free();
    for (int i = 0; i <= ST_COUNT; ++i)
        if (h->ev[i]) cudaEventDestroy(h->ev[i]);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MDFT_OK;
}

int mdft_get_sizes(const mdft_handle *h, mdft_sizes *o) {
    if (!h || !o) { set_error("null argument"); return MDFT_E_ARG; }
    o->ntheta = h->g.ntheta; o->nphi = h->g.nphi; o->npsi = h->g.npsi;
    o->no = h->g.no; o->np = h->g.np;
    o->ncoef = h->ct.ncoef; o->nq = h->ct.nq;
    o->dv = h->g.dv; o->rho0 = h->g.rho0; o->kT = h->g.kT; o->dq = h->ct.dq;
    return MDFT_OK;
}

int mdft_get_stream(const mdft_handle *h, void **s) {
    if (!h || !s) { set_error("null argument"); return MDFT_E_ARG; }
    *s = (void *)h->stream;
    return MDFT_OK;
}

int mdft_get_weights(const mdft_handle *h, double *w) {
    if (!h || !w) { set_error("null argument"); return MDFT_E_ARG; }
    std::memcpy(w, h->g.w.data(), sizeof(double) * h->g.no);
    return MDFT_OK;
}

int mdft_set_vext(mdft_handle *h, const double *v) {
    if (!h || !v) { set_error("null argument"); return MDFT_E_ARG; }
    size_t n = (size_t)h->g.N * h->g.no;
    int rc = check_cuda(cudaMemcpyAsync(h->vext.p, v, n * 8, cudaMemcpyHostToDevice, h->stream), "vext upload");
    if (rc) return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "vext upload"))) return rc;
    h->have_vext = true;
    return MDFT_OK;
}

int mdft_get_vext(const mdft_handle *h, double *v) {
    if (!h || !v) { set_error("null argument"); return MDFT_E_ARG; }
    size_t n = (size_t)h->g.N * h->g.no;
    int rc = check_cuda(cudaMemcpyAsync(v, h->vext.p, n * 8, cudaMemcpyDeviceToHost, h->stream), "vext download");
    if (rc) return rc;
    return check_cuda(cudaStreamSynchronize(h->stream), "vext download");
}

int mdft_set_constant_correction(mdft_handle *h, double c) {
    if (!h) { set_error("null argument"); return MDFT_E_ARG; }
    h->const_corr = c;
    return MDFT_OK;
}

// c00_000 by solvent(1)%name and grid%mmax (src/module_coarse_grained_gageat_bridge.f90:260-263)
int mdft_cgb_c00(const char *solvent, int mmax, double *c00) {
    if (!solvent || !c00) { set_error("null argument"); return MDFT_E_ARG; }
    if (std::strcmp(solvent, "spce") == 0) *c00 = mmax == 0 ? -14.64872 : -13.665;
    else if (std::strcmp(solvent, "tip3p") == 0) *c00 = -11.9078;
    else {
        set_error("no c00_000 for solvent '%s' (the reference has values for spce and tip3p only)", solvent);
        return MDFT_E_ARG;
    }
    return MDFT_OK;
}

}  // extern "C"

namespace {
// bridge = "no": drop both terms and their buffers
int clear_bridges(mdft_handle *h) {
    drop_pipe_graphs(h);  // the captured pipelines carry the bridge's launches
    h->cgb = 0;
    h->fmt = 0;
    h->cgb_kk.free(); h->cgb_a.free(); h->cgb_b.free(); h->cgb_dens.free(); h->cgb_part.free();
    h->fmt_pl.free(); h->fmt_cs.free(); h->fmt_part.free();
    return check_cuda(cudaMemsetAsync(h->sums.p + 6, 0, 2 * sizeof(double), h->stream), "sums reset");
}
}  // namespace

extern "C" {

int mdft_set_bridge_cgb(mdft_handle *h, int version, double B6, double sigma, double c00) {
    if (!h) { set_error("null argument"); return MDFT_E_ARG; }
    if (version < MDFT_BRIDGE_NONE || version > MDFT_BRIDGE_CGB_WDA) { set_error("unknown cgb version %d", version); return MDFT_E_ARG; }
    if (version != MDFT_BRIDGE_NONE && h->precision != MDFT_PREC_FP64) {
        set_error("the bridge term needs an FP64 handle");
        return MDFT_E_ARG;
    }
    if (version != MDFT_BRIDGE_NONE && !(sigma > 0.0 && std::isfinite(sigma) && std::isfinite(B6) && std::isfinite(c00))) {
        set_error("cgb parameters must be finite, sigma > 0");
        return MDFT_E_ARG;
    }
    int rc = clear_bridges(h);
    if (rc || version == MDFT_BRIDGE_NONE) return rc;
    const Grid &g = h->g;
    if ((rc = alloc_check(h->cgb_kk.alloc(g.N), "bridge kernel", g.N * 16))) return rc;
    if ((rc = alloc_check(h->cgb_a.alloc(g.N), "bridge plane", g.N * 16))) return rc;
    if ((rc = alloc_check(h->cgb_b.alloc(g.N), "bridge plane", g.N * 16))) return rc;
    if ((rc = alloc_check(h->cgb_dens.alloc(g.N), "bridge density", g.N * 8))) return rc;
    if ((rc = alloc_check(h->cgb_part.alloc(4 * kRedBlocks), "bridge partials", 32 * kRedBlocks))) return rc;
    // fill_kernel (src/module_coarse_grained_gageat_bridge.f90:123-210)
    const double pi = std::acos(-1.0);
    const double sp = sigma * std::sqrt(2.0 * pi);
    const double gp = 1.0 / (sp * sp * sp), oo = 1.0 / (2.0 * sigma * sigma);
    const double cut = -1.0 / oo * std::log(1.0e-10 / gp);
    const double nf = (double)(float)(g.nx * g.ny * g.nz);  // real(nx*ny*nz): single precision
    k_cgb_kernel<<<kRedBlocks, kBrThreads, 0, h->stream>>>(h->cgb_kk.p, g.nx, g.ny, g.nz, g.lx / g.nx, g.ly / g.ny, g.lz / g.nz,
                                                           gp, oo, cut);
    if ((rc = launch_fft_planes(h, h->cgb_kk.p, 1, -1))) return rc;
    k_cgb_scale<<<kRedBlocks, kBrThreads, 0, h->stream>>>(h->cgb_kk.p, g.N, nf, g.lx * g.ly * g.lz);
    h->launches += 2;
    if ((rc = check_cuda(cudaGetLastError(), "bridge kernel"))) return rc;
    CgbArgs &a = h->cgb_args;
    a.N = g.N;
    a.no = g.no;
    a.version = version;
    a.rho0 = g.rho0;
    a.n0 = g.n0;
    a.kT = g.kT;
    a.vvox = (g.lx / g.nx) * (g.ly / g.ny) * (g.lz / g.nz);
    a.nf = nf;
    a.A3 = 1.0 - c00 / 2.0;
    a.B6 = B6;
    h->cgb = version;
    return check_cuda(cudaStreamSynchronize(h->stream), "bridge set-up");
}

// The bulk hard-sphere parameters (src/module_hardspheres.f90:83-189) and the hard-sphere
// c(k) (src/cs_of_k_hard_sphere.f90:56-157) on nb_k points of the c(k) file's step.
int mdft_set_bridge_fmt(mdft_handle *h, int functional, double R) {
    if (!h) { set_error("null argument"); return MDFT_E_ARG; }
    if (functional < MDFT_BRIDGE_NONE || functional > MDFT_BRIDGE_HS_CS) { set_error("unknown hard-sphere functional %d", functional); return MDFT_E_ARG; }
    if (functional != MDFT_BRIDGE_NONE && h->precision != MDFT_PREC_FP64) {
        set_error("the bridge term needs an FP64 handle");
        return MDFT_E_ARG;
    }
    if (functional != MDFT_BRIDGE_NONE && !(R > 0.0 && std::isfinite(R))) { set_error("the hard-sphere radius must be positive"); return MDFT_E_ARG; }
    int rc = clear_bridges(h);
    if (rc || functional == MDFT_BRIDGE_NONE) return rc;
    const Grid &g = h->g;
    const double pi = kPi, kT = g.kT, n0 = g.n0;
    const double pf = (double)(4.0f / 3.0f) * pi * n0 * (R * R * R);  // fourthird = 4./3. (single)
    if (pf >= 0.74) { set_error("hard-sphere packing fraction %g is above 0.74", pf); return MDFT_E_ARG; }
    // excess chemical potential and bulk grand potential
    const double b1 = n0 * R, b2 = n0 * 4 * pi * (R * R), b3 = n0 * 4 * pi * (R * R * R) / 3;
    double dp[4];
    dp[0] = -std::log(1 - b3);
    dp[1] = b2 / (1 - b3);
    if (functional == MDFT_BRIDGE_HS_PY) {
        dp[2] = b1 / (1 - b3) + (b2 * b2) / (8 * pi * ((1 - b3) * (1 - b3)));
        dp[3] = n0 / (1 - b3) + b1 * b2 / ((1 - b3) * (1 - b3)) + (b2 * b2 * b2) / (12 * pi * ((1 - b3) * (1 - b3) * (1 - b3)));
    } else {
        const double m = b3 - 1;
        dp[2] = (b3 * ((b2 * b2) - 12 * b1 * m * b3 * pi) + (b2 * b2) * (m * m) * std::log(1 - b3)) / (12 * pi * (m * m) * (b3 * b3));
        dp[3] = (b3 * ((b2 * b2 * b2) * (2 - 5 * b3 + (b3 * b3)) + 36 * b1 * b2 * m * (b3 * b3) * pi - 36 * n0 * (m * m) * (b3 * b3) * pi) -
                 2 * (b2 * b2 * b2) * (m * m * m) * std::log(1 - b3)) /
                (36 * pi * (m * m * m) * (b3 * b3 * b3));
    }
    const double dn[4] = {1, R, 4 * pi * (R * R), 4 * pi * (R * R * R) / 3.0};
    double acc = 0.0;
    for (int i = 0; i < 4; ++i) acc += dp[i] * dn[i];
    const double mu = kT * acc;
    double f0 = functional == MDFT_BRIDGE_HS_PY
                    ? kT * (-n0 * std::log(1 - b3) + b1 * b2 / (1 - b3) + (b2 * b2 * b2) / (24 * pi * ((1 - b3) * (1 - b3))))
                    : kT * (((1.0 / (36 * pi)) * (b2 * b2 * b2) / (b3 * b3) - n0) * std::log(1 - b3) + b1 * b2 / (1 - b3) +
                            (1.0 / (36 * pi)) * (b2 * b2 * b2) / (((1 - b3) * (1 - b3)) * b3));
    f0 = (f0 - mu * n0) * (g.lx * g.ly * g.lz);
    // c_hs(k) at k = (i-1) dq with the bulk weighted densities
    const double twopi = 2.0 * pi;
    const double kxm = (double)(g.nx / 2) * twopi / g.lx, kym = (double)(g.ny / 2) * twopi / g.ly, kzm = (double)(g.nz / 2) * twopi / g.lz;
    const double dq = h->ct.dq;
    const int nbk = (int)(std::sqrt(kxm * kxm + kym * kym + kzm * kzm) / dq) + 1;
    std::vector<double> cs(nbk);
    // the bulk weighted densities as cs_of_k_hard_sphere forms them: n0 times w_a(k = 0)
    const double c0 = n0 * 1.0, c1 = n0 * R, c2 = n0 * (4.0 * pi * (R * R)), c3 = n0 * (4.0 * pi / 3.0 * (R * R * R));
    const double u = 1.0 - c3, m1 = -1.0 + c3;
    if (std::fabs(c3 - 1) <= kEpsDp) { set_error("n3 = 1 in the hard-sphere c(k)"); return MDFT_E_ARG; }
    double d[4][4] = {{0}};
    if (functional == MDFT_BRIDGE_HS_PY) {
        d[0][3] = 1.0 / u;
        d[1][2] = 1.0 / u;
        d[1][3] = c2 / (u * u);
        d[2][2] = c2 / (4 * pi * (u * u));
        d[2][3] = c1 / (u * u) + (c2 * c2) / (4 * pi * (u * u * u));
        d[3][3] = (2.0 * c1 * c2) / (u * u * u) + c0 / (u * u) + (c2 * c2 * c2) / (4.0 * pi * ((u * u) * (u * u)));
    } else {
        d[0][3] = 1.0 / (1 - c3);
        d[1][2] = 1.0 / (1.0 - c3);
        d[1][3] = c2 / ((1.0 - c3) * (1.0 - c3));
        d[2][2] = c2 / (6.0 * ((1.0 - c3) * (1.0 - c3)) * c3 * pi) + (c2 * std::log(1.0 - c3)) / (6.0 * (c3 * c3) * pi);
        d[2][3] = (c3 * ((c2 * c2) * (2.0 - 5.0 * c3 + (c3 * c3)) + 12.0 * c1 * m1 * (c3 * c3) * pi) -
                   2.0 * (c2 * c2) * (m1 * m1 * m1) * std::log(1 - c3)) /
                  (12.0 * (m1 * m1 * m1) * (c3 * c3 * c3) * pi);
        d[3][3] = (c3 * ((c2 * c2 * c2) * (6.0 - 21.0 * c3 + 26.0 * (c3 * c3) - 5.0 * (c3 * c3 * c3)) -
                         72.0 * c1 * c2 * m1 * (c3 * c3 * c3) * pi + 36.0 * c0 * (m1 * m1) * (c3 * c3 * c3) * pi) +
                   6.0 * (c2 * c2 * c2) * ((m1 * m1) * (m1 * m1)) * std::log(1.0 - c3)) /
                  (36.0 * ((m1 * m1) * (m1 * m1)) * ((c3 * c3) * (c3 * c3)) * pi);
    }
    d[2][1] = d[1][2];
    d[3][0] = d[0][3];
    d[3][1] = d[1][3];
    d[3][2] = d[2][3];
    for (int i = 0; i < nbk; ++i) {
        const double k = i * dq;
        double w[4];
        if (std::fabs(k) <= kEpsDp) {
            w[0] = 1.0; w[1] = R; w[2] = 4.0 * pi * (R * R); w[3] = 4.0 * pi / 3.0 * (R * R * R);
        } else {
            const double kR = k * R, sk = std::sin(kR), ck = std::cos(kR);
            w[0] = ck + kR * sk / 2.0;
            w[1] = (sk + kR * ck) / (2.0 * k);
            w[2] = (4.0 * pi * R * sk) / k;
            w[3] = 4.0 * pi * (sk - kR * ck) / (k * k * k);
        }
        double sum = 0.0;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) sum += d[a][b] * w[a] * w[b];
        cs[i] = -sum;
    }
    const size_t nb = kRedBlocks;
    if ((rc = alloc_check(h->fmt_pl.alloc(7 * (size_t)g.N), "bridge planes", 7 * 16 * (size_t)g.N))) return rc;
    if ((rc = alloc_check(h->fmt_cs.alloc(nbk), "hard-sphere c(k)", 8 * (size_t)nbk))) return rc;
    if ((rc = alloc_check(h->fmt_part.alloc(10 * nb + 2), "bridge partials", 8 * (10 * nb + 2)))) return rc;
    if ((rc = check_cuda(cudaMemcpy(h->fmt_cs.p, cs.data(), 8 * (size_t)nbk, cudaMemcpyHostToDevice), "hard-sphere c(k)"))) return rc;
    FmtArgs &a = h->fmt_args;
    a.N = g.N;
    a.no = g.no;
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    a.version = functional;
    a.rho0 = g.rho0;
    a.kT = kT;
    a.dv = g.dv;
    a.R = R;
    a.mu = mu;
    a.fexc0 = f0;
    a.shift = (twopi * (4.0 * pi)) / (double)g.mrso;
    a.nd = (double)(g.nx * g.ny * g.nz);
    a.dq = dq;
    a.lx = g.lx;
    a.ly = g.ly;
    a.lz = g.lz;
    a.nbk = nbk;
    h->fmt = functional;
    return MDFT_OK;
}

int mdft_get_bridge_fmt_params(const mdft_handle *h, double *out) {
    if (!h || !out) { set_error("null argument"); return MDFT_E_ARG; }
    if (!h->fmt) { set_error("no hard-sphere bridge set"); return MDFT_E_STATE; }
    out[0] = h->fmt_args.R;
    out[1] = h->fmt_args.mu;
    out[2] = h->fmt_args.fexc0;
    out[3] = h->fmt_args.nbk;
    return MDFT_OK;
}

int mdft_bridge_energy(mdft_handle *h, const double *xi, double *fb, double *df) {
    if (!h || !xi || !fb) { set_error("null argument"); return MDFT_E_ARG; }
    *fb = 0.0;
    if (!has_bridge(h)) return MDFT_OK;  // bridge "no"
    const size_t n = (size_t)h->g.N * h->g.no;
    int rc = check_cuda(cudaMemcpyAsync(h->xi.p, xi, n * 8, cudaMemcpyHostToDevice, h->stream), "xi upload");
    if (rc) return rc;
    if (df && (rc = check_cuda(cudaMemcpyAsync(h->df.p, df, n * 8, cudaMemcpyHostToDevice, h->stream), "df upload"))) return rc;
    if ((rc = launch_bridge(h, h->xi.p, df ? h->df.p : nullptr, nullptr))) return rc;
    if ((rc = check_cuda(cudaMemcpyAsync(h->h_sums + 6, h->sums.p + 6, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "sums copy")))
        return rc;
    if (df && (rc = check_cuda(cudaMemcpyAsync(df, h->df.p, n * 8, cudaMemcpyDeviceToHost, h->stream), "df download"))) return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "bridge"))) return rc;
    if (h->fmt && h->h_sums[7] != 0.0) {
        cudaMemsetAsync(h->sums.p + 7, 0, sizeof(double), h->stream);
        set_error("hard-sphere bridge: a weighted density left (0, 1) (code %d)", (int)h->h_sums[7]);
        return MDFT_E_NUMERIC;
    }
    *fb = h->h_sums[6];
    if (!std::isfinite(*fb)) { set_error("non-finite bridge energy"); return MDFT_E_NUMERIC; }
    return MDFT_OK;
}

int mdft_energy_and_gradient_device(mdft_handle *h, const double *d_xi, double *d_df, double *f, double *terms) {
    if (!h || !d_xi || !f) { set_error("null argument"); return MDFT_E_ARG; }
    int rc = run_pipeline(h, d_xi, d_df, 1, 1);
    if (rc) return rc;
    double fid, fext, fexc;
    if ((rc = finish_sums(h, &fid, &fext, &fexc))) return rc;
    *f = combine(h, fid, fext, fexc);
    if (terms) {
        terms[0] = fid;
        terms[1] = fext;
        terms[2] = fexc;
        terms[3] = h->const_corr;
    }
    return MDFT_OK;
}

int mdft_energy_and_gradient(mdft_handle *h, const double *xi, double *f, double *df, double *terms) {
    if (!h || !xi || !f) { set_error("null argument"); return MDFT_E_ARG; }
    size_t n = (size_t)h->g.N * h->g.no;
    int rc = check_cuda(cudaMemcpyAsync(h->xi.p, xi, n * 8, cudaMemcpyHostToDevice, h->stream), "xi upload");
    if (rc) return rc;
    if ((rc = mdft_energy_and_gradient_device(h, h->xi.p, df ? h->df.p : nullptr, f, terms))) return rc;
    if (df) {
        if ((rc = check_cuda(cudaMemcpyAsync(df, h->df.p, n * 8, cudaMemcpyDeviceToHost, h->stream), "df download"))) return rc;
        if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "df download"))) return rc;
    }
    return MDFT_OK;
}

int mdft_excess_energy(mdft_handle *h, const double *xi, double *fexc, double *df) {
    if (!h || !xi || !fexc) { set_error("null argument"); return MDFT_E_ARG; }
    size_t n = (size_t)h->g.N * h->g.no;
    int rc = check_cuda(cudaMemcpyAsync(h->xi.p, xi, n * 8, cudaMemcpyHostToDevice, h->stream), "xi upload");
    if (rc) return rc;
    if (df && (rc = check_cuda(cudaMemcpyAsync(h->df.p, df, n * 8, cudaMemcpyHostToDevice, h->stream), "df upload"))) return rc;
    if ((rc = run_pipeline(h, h->xi.p, df ? h->df.p : nullptr, 0, 2))) return rc;
    double a, b;
    if ((rc = finish_sums(h, &a, &b, fexc))) return rc;
    if (df) {
        if ((rc = check_cuda(cudaMemcpyAsync(df, h->df.p, n * 8, cudaMemcpyDeviceToHost, h->stream), "df download"))) return rc;
        if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "df download"))) return rc;
    }
    return MDFT_OK;
}

int mdft_set_timing(mdft_handle *h, int on) {
    if (!h) { set_error("null argument"); return MDFT_E_ARG; }
    h->timing = on != 0;
    for (int i = 0; i < ST_COUNT; ++i) h->stage_ms[i] = 0;
    h->stage_count = 0;
    return MDFT_OK;
}

int mdft_set_wait_failure(mdft_handle *h, int on) {
    if (!h) { set_error("null argument"); return MDFT_E_ARG; }
    h->wait_fail = on != 0;
    drop_pipe_graphs(h);  // the captured launches carry the flag
    return MDFT_OK;
}

int mdft_get_kernel_forms(const mdft_handle *h, int *forms, double *ms) {
    if (!h || !forms) { set_error("null argument"); return MDFT_E_ARG; }
    forms[0] = h->ring_p ? 1 : 0;
    forms[1] = h->ring_g ? 1 : 0;
    forms[2] = h->ozd;
    forms[3] = h->tuned && h->tune_ms[0][0] >= 0 ? 1 : 0;
    if (ms)
        for (int i = 0; i < 3; ++i)
            for (int c = 0; c < 2; ++c) ms[2 * i + c] = h->tune_ms[i][c];
    return MDFT_OK;
}

int mdft_get_launch_count(const mdft_handle *h, long long *count) {
    if (!h || !count) { set_error("null argument"); return MDFT_E_ARG; }
    *count = h->launches;
    return MDFT_OK;
}

int mdft_get_stage_times(const mdft_handle *h, double *ms5, int *count) {
    if (!h || !ms5) { set_error("null argument"); return MDFT_E_ARG; }
    for (int i = 0; i < ST_COUNT; ++i) ms5[i] = h->stage_ms[i];
    if (count) *count = h->stage_count;
    return MDFT_OK;
}

}  // extern "C"

#include "solve.cuh"
#include "mixture.cuh"
