// Solve-level entry points: external potential, initial guess, the L-BFGS
// minimisation on the device and the pressure-corrected solvation free
// energy.  Included by mdft_b200.cu after the handle definition.
#pragma once

namespace {

constexpr double kQfact = 1.602176565e-19 * 1.602176565e-19 * 1.0e-3 * 6.02214129e23 /
                          (4.0 * 3.14159265358979323846 * 8.854187817e-12 * 1.0e-10);  // src/module_constants.f90:25

inline unsigned vec_grid() { return kRedBlocks; }

// multi-species minimisation (mixture.cuh): vector length, gradient buffer and the two
// halves of an evaluation of every species
long long mixture_len(const mdft_mixture *m);
double *mixture_grad(mdft_mixture *m);
int mixture_eval_launch(mdft_mixture *m, const double *x, double *g, const double *dvec);
int mixture_eval_finish(mdft_mixture *m, double *f, double *gd, double *gmax, double *guni, double *fscale);

// Evaluation in two halves so that more work can be queued before the synchronise:
// eval_launch queues the pipeline at x (gradient into g; with dvec also g.dvec and max|g|
// from the gather pass), eval_finish waits and reads f, g.dvec, max|g| and sum w g dv.
int eval_launch(mdft_handle *h, const void *x, double *g, const void *dvec, bool v32 = false, bool x32 = false) {
    if (h->mix) return mixture_eval_launch(h->mix, static_cast<const double *>(x), g, static_cast<const double *>(dvec));
    return run_pipeline(h, x, g, 1, 1, dvec, v32, x32);
}

int eval_finish(mdft_handle *h, double *f, double *gd, double *gmax, double *guni = nullptr, double *fscale = nullptr) {
    if (h->mix) return mixture_eval_finish(h->mix, f, gd, gmax, guni, fscale);
    double fid, fext, fexc;
    int rc = finish_sums(h, &fid, &fext, &fexc);
    if (rc) return rc;
    *f = combine(h, fid, fext, fexc);
    if (fscale) *fscale = std::fabs(fid) + std::fabs(fext) + std::fabs(fexc) + std::fabs(h->const_corr);
    const double gdv = h->h_sums[3], gmx = h->h_sums[4], gun = h->h_sums[5] * h->g.dv;
    if (gd) *gd = gdv;
    if (gmax) *gmax = gmx;
    if (guni) *guni = gun;
    if (!std::isfinite(gdv) || !std::isfinite(gmx) || !std::isfinite(gun)) {
        set_error("non-finite gradient");
        return MDFT_E_NUMERIC;
    }
    return 0;
}

// x, g device vectors of n; dvec may be null.  Leaves f, g.dvec and max|g|.  v32: g and dvec
// are FP32 vectors (the minimiser's mixed solves).
int eval_fg(mdft_handle *h, const void *x, double *g, const void *dvec, double *f, double *gd, double *gmax,
            bool v32 = false, bool x32 = false, double *guni = nullptr, double *fscale = nullptr) {
    int rc = eval_launch(h, x, g, dvec, v32, x32);
    if (rc) return rc;
    return eval_finish(h, f, gd, gmax, guni, fscale);
}

// Autotuner of the FP32 forms: the pipeline at the FP32 point x (gradient into the scratch
// vector g) under two configurations -- the defaults (register projection, ring gather,
// factored OZ) and the alternatives (ring projection, register gather, complex-rotation
// OZ) -- one untimed and three timed evaluations each, stage times by CUDA events (the
// fastest of the three); each stage keeps its default form unless the alternative is more
// than 5 % faster.
constexpr double kTuneMargin = 0.05;
int autotune_fp32(mdft_handle *h, const void *x, double *g) {
    if (h->tuned) return 0;
    h->tuned = true;
    if (!h->tune_on || !h->um_ok) return 0;
    const bool timing0 = h->timing;
    double ms0[ST_COUNT];
    for (int i = 0; i < ST_COUNT; ++i) ms0[i] = h->stage_ms[i];
    const int cnt0 = h->stage_count;
    struct Cfg {
        bool rp, rg, oz;
    };
    const Cfg cfg[2] = {{false, h->ring_g_ok, h->ozp_ok ? true : h->ozd}, {h->ring_p_ok, false, false}};
    double ms[2][ST_COUNT] = {};
    int rc = 0;
    for (int c = 0; c < 2 && !rc; ++c) {
        h->ring_p = cfg[c].rp;
        h->ring_g = cfg[c].rg;
        h->ozd = cfg[c].oz;
        double fid, fext, fexc;
        h->timing = false;
        if ((rc = run_pipeline(h, x, g, 1, 1, nullptr, true, true)) || (rc = finish_sums(h, &fid, &fext, &fexc))) break;
        h->timing = true;
        for (int i = 0; i < ST_COUNT; ++i) ms[c][i] = -1.0;
        for (int r = 0; r < 3 && !rc; ++r) {  // the fastest of three evaluations, stage by stage
            for (int i = 0; i < ST_COUNT; ++i) h->stage_ms[i] = 0;
            h->stage_count = 0;
            if (!(rc = run_pipeline(h, x, g, 1, 1, nullptr, true, true))) rc = finish_sums(h, &fid, &fext, &fexc);
            for (int i = 0; i < ST_COUNT && !rc; ++i)
                if (ms[c][i] < 0.0 || h->stage_ms[i] < ms[c][i]) ms[c][i] = h->stage_ms[i];
        }
    }
    h->timing = timing0;
    for (int i = 0; i < ST_COUNT; ++i) h->stage_ms[i] = ms0[i];
    h->stage_count = cnt0;
    drop_pipe_graphs(h);  // graphs captured under either configuration are stale
    if (rc) {  // keep the defaults
        h->ring_p = cfg[0].rp;
        h->ring_g = cfg[0].rg;
        h->ozd = cfg[0].oz;
        return rc;
    }
    const int stage[3] = {ST_PROJECT, ST_OZ, ST_GATHER};
    for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 2; ++c) h->tune_ms[i][c] = ms[c][stage[i]];
    const bool diff_p = cfg[0].rp != cfg[1].rp, diff_g = cfg[0].rg != cfg[1].rg, diff_o = cfg[0].oz != cfg[1].oz;
    // an alternative replaces a default only when it is faster by more than kTuneMargin, so
    // that timing noise does not flip a choice
    auto better = [](double alt, double def) { return alt < (1.0 - kTuneMargin) * def; };
    h->ring_p = diff_p && better(ms[1][ST_PROJECT], ms[0][ST_PROJECT]) ? cfg[1].rp : cfg[0].rp;
    h->ring_g = diff_g && better(ms[1][ST_GATHER], ms[0][ST_GATHER]) ? cfg[1].rg : cfg[0].rg;
    h->ozd = diff_o && better(ms[1][ST_OZ], ms[0][ST_OZ]) ? cfg[1].oz : cfg[0].oz;
    if (h->trace)
        std::fprintf(stderr, "mdft-trace autotune: project %s (%.4f / %.4f ms), oz %s (%.4f / %.4f), gather %s (%.4f / %.4f)\n",
                     h->ring_p ? "ring" : "register", ms[0][ST_PROJECT], ms[1][ST_PROJECT], h->ozd ? "factored" : "complex",
                     ms[0][ST_OZ], ms[1][ST_OZ], h->ring_g ? "ring" : "register", ms[0][ST_GATHER], ms[1][ST_GATHER]);
    return 0;
}

__global__ void k_fill_f32(float *__restrict__ p, float v, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = v;
}

// Create-time tuning of a mixed handle, shared by every handle of the same shape on the same
// device in this process (the first one measures, under a lock, at the bulk density with no
// external potential -- the kernels' times do not depend on the values).
struct TuneKey {
    int dev, nx, ny, nz, mmax, mrso, no;
    bool operator<(const TuneKey &o) const {
        return std::tie(dev, nx, ny, nz, mmax, mrso, no) < std::tie(o.dev, o.nx, o.ny, o.nz, o.mmax, o.mrso, o.no);
    }
};
struct TuneResult {
    bool rp, rg, oz;
    double ms[3][2];
};
int autotune_at_create(mdft_handle *h) {
    if (!h->tune_on || !h->um_ok || !h->pt_ok32 || h->gt_ncol32 <= 0 || h->precision != MDFT_PREC_MIXED) return 0;
    static std::mutex mu;
    static std::map<TuneKey, TuneResult> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const Grid &g = h->g;
    const TuneKey key{dev, g.nx, g.ny, g.nz, g.mmax, g.mrso, g.no};
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it == cache.end()) {
        const long long nf = g.N * g.no;
        int rc;
        if (!h->vext32.p && (rc = alloc_check(h->vext32.alloc((size_t)nf), "FP32 vext", (size_t)nf * 4))) return rc;
        cudaMemsetAsync(h->vext32.p, 0, (size_t)nf * 4, h->stream);
        float *x = reinterpret_cast<float *>(h->xi.p);  // the FP64 buffer holds the FP32 point
        k_fill_f32<<<vec_grid(), 256, 0, h->stream>>>(x, 1.0f, nf);
        h->launches += 1;
        const int ep = h->eval_prec;
        h->eval_prec = MDFT_PREC_MIXED;
        rc = autotune_fp32(h, x, h->df.p);
        h->eval_prec = ep;
        if (rc) return rc;
        TuneResult r{h->ring_p, h->ring_g, h->ozd, {}};
        for (int i = 0; i < 3; ++i)
            for (int c = 0; c < 2; ++c) r.ms[i][c] = h->tune_ms[i][c];
        cache[key] = r;
    } else {
        h->ring_p = it->second.rp;
        h->ring_g = it->second.rg;
        h->ozd = it->second.oz;
        for (int i = 0; i < 3; ++i)
            for (int c = 0; c < 2; ++c) h->tune_ms[i][c] = it->second.ms[i][c];
        h->tuned = true;
    }
    return 0;
}

int lbfgs_alloc(mdft_handle *h, int m) {
    LbfgsState &L = h->lb;
    const long long n = h->mix ? mixture_len(h->mix) : h->g.N * h->g.no;
    if (L.n == n && L.m == m) return 0;
    lbfgs_free(L);
    L.n = n;
    L.m = m;
    int rc;
    DevBuf<double> *v[] = {&L.x, &L.d, &L.t, &L.r};
    for (auto *b : v)
        if ((rc = alloc_check(b->alloc(n), "L-BFGS vector", n * 8))) return rc;
    if ((rc = alloc_check(L.S.alloc((size_t)m * n), "L-BFGS s history", (size_t)m * n * 8))) return rc;
    return alloc_check(L.Y.alloc((size_t)m * n), "L-BFGS y history", (size_t)m * n * 8);
}

// Moré-Thuente search of src/module_lbfgs_nocedal_mdft.f90:1653-1959 (dcsrch/dcstep),
// with the reference's single-precision constants.
struct LineSearch {
    int brackt = 0, stage = 1;
    double ginit = 0, gtest = 0, gx = 0, gy = 0, finit = 0, fx = 0, fy = 0, stx = 0, sty = 0, stmin = 0, stmax = 0,
           width = 0, width1 = 0;
};
enum { LS_FG = 0, LS_CONV = 1, LS_WARN = 2, LS_ERROR = 3 };

void dcstep(double &stx, double &fx, double &dx, double &sty, double &fy, double &dy, double &stp, double fp, double dp,
            int &brackt, double stpmin, double stpmax) {
    const double p66 = (double)0.66f;
    double gamma, p, q, r, s, stpc, stpf, stpq, theta;
    double sgnd = dp * (dx / std::fabs(dx));
    if (fp > fx) {
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
        s = std::max(std::max(std::fabs(theta), std::fabs(dx)), std::fabs(dp));
        gamma = s * std::sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
        if (stp < stx) gamma = -gamma;
        p = (gamma - dx) + theta;
        q = ((gamma - dx) + gamma) + dp;
        r = p / q;
        stpc = stx + r * (stp - stx);
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx);
        stpf = (std::fabs(stpc - stx) < std::fabs(stpq - stx)) ? stpc : stpc + (stpq - stpc) / 2.0;
        brackt = 1;
    } else if (sgnd < 0.0) {
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
        s = std::max(std::max(std::fabs(theta), std::fabs(dx)), std::fabs(dp));
        gamma = s * std::sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
        if (stp > stx) gamma = -gamma;
        p = (gamma - dp) + theta;
        q = ((gamma - dp) + gamma) + dx;
        r = p / q;
        stpc = stp + r * (stx - stp);
        stpq = stp + (dp / (dp - dx)) * (stx - stp);
        stpf = (std::fabs(stpc - stp) > std::fabs(stpq - stp)) ? stpc : stpq;
        brackt = 1;
    } else if (std::fabs(dp) < std::fabs(dx)) {
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
        s = std::max(std::max(std::fabs(theta), std::fabs(dx)), std::fabs(dp));
        gamma = s * std::sqrt(std::max(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
        if (stp > stx) gamma = -gamma;
        p = (gamma - dp) + theta;
        q = (gamma + (dx - dp)) + gamma;
        r = p / q;
        if (r < 0.0 && gamma != 0.0) stpc = stp + r * (stx - stp);
        else if (stp > stx) stpc = stpmax;
        else stpc = stpmin;
        stpq = stp + (dp / (dp - dx)) * (stx - stp);
        if (brackt) {
            stpf = (std::fabs(stpc - stp) < std::fabs(stpq - stp)) ? stpc : stpq;
            if (stp > stx) stpf = std::min(stp + p66 * (sty - stp), stpf);
            else stpf = std::max(stp + p66 * (sty - stp), stpf);
        } else {
            stpf = (std::fabs(stpc - stp) > std::fabs(stpq - stp)) ? stpc : stpq;
            stpf = std::min(stpmax, stpf);
            stpf = std::max(stpmin, stpf);
        }
    } else {
        if (brackt) {
            theta = 3.0 * (fp - fy) / (sty - stp) + dy + dp;
            s = std::max(std::max(std::fabs(theta), std::fabs(dy)), std::fabs(dp));
            gamma = s * std::sqrt((theta / s) * (theta / s) - (dy / s) * (dp / s));
            if (stp > sty) gamma = -gamma;
            p = (gamma - dp) + theta;
            q = ((gamma - dp) + gamma) + dy;
            r = p / q;
            stpc = stp + r * (sty - stp);
            stpf = stpc;
        } else if (stp > stx) stpf = stpmax;
        else stpf = stpmin;
    }
    if (fp > fx) {
        sty = stp; fy = fp; dy = dp;
    } else {
        if (sgnd < 0.0) { sty = stx; fy = fx; dy = dx; }
        stx = stp; fx = fp; dx = dp;
    }
    stp = stpf;
}

int dcsrch(double f, double g, double &stp, double ftol, double gtol, double xtol, double stpmin, double stpmax, bool start,
           LineSearch &S) {
    const double p5 = 0.5, p66 = (double)0.66f, xtrapl = (double)1.1f, xtrapu = 4.0;
    if (start) {
        if (stp < stpmin || stp > stpmax || g >= 0.0 || ftol < 0.0 || gtol < 0.0 || xtol < 0.0 || stpmin < 0.0 ||
            stpmax < stpmin)
            return LS_ERROR;
        S = LineSearch();
        S.brackt = 0; S.stage = 1; S.finit = f; S.ginit = g; S.gtest = ftol * S.ginit;
        S.width = stpmax - stpmin; S.width1 = S.width / p5;
        S.stx = 0.0; S.fx = S.finit; S.gx = S.ginit;
        S.sty = 0.0; S.fy = S.finit; S.gy = S.ginit;
        S.stmin = 0.0; S.stmax = stp + xtrapu * stp;
        return LS_FG;
    }
    int task = LS_FG;
    double ftest = S.finit + stp * S.gtest;
    if (S.stage == 1 && f <= ftest && g >= 0.0) S.stage = 2;
    if (S.brackt && (stp <= S.stmin || stp >= S.stmax)) task = LS_WARN;
    if (S.brackt && S.stmax - S.stmin <= xtol * S.stmax) task = LS_WARN;
    if (stp == stpmax && f <= ftest && g <= S.gtest) task = LS_WARN;
    if (stp == stpmin && (f > ftest || g >= S.gtest)) task = LS_WARN;
    if (f <= ftest && std::fabs(g) <= gtol * (-S.ginit)) task = LS_CONV;
    if (task != LS_FG) return task;
    if (S.stage == 1 && f <= S.fx && f > ftest) {
        double fm = f - stp * S.gtest, fxm = S.fx - S.stx * S.gtest, fym = S.fy - S.sty * S.gtest;
        double gm = g - S.gtest, gxm = S.gx - S.gtest, gym = S.gy - S.gtest;
        dcstep(S.stx, fxm, gxm, S.sty, fym, gym, stp, fm, gm, S.brackt, S.stmin, S.stmax);
        S.fx = fxm + S.stx * S.gtest;
        S.fy = fym + S.sty * S.gtest;
        S.gx = gxm + S.gtest;
        S.gy = gym + S.gtest;
    } else {
        dcstep(S.stx, S.fx, S.gx, S.sty, S.fy, S.gy, stp, f, g, S.brackt, S.stmin, S.stmax);
    }
    if (S.brackt) {
        if (std::fabs(S.sty - S.stx) >= p66 * S.width1) stp = S.stx + p5 * (S.sty - S.stx);
        S.width1 = S.width;
        S.width = std::fabs(S.sty - S.stx);
    }
    if (S.brackt) { S.stmin = std::min(S.stx, S.sty); S.stmax = std::max(S.stx, S.sty); }
    else { S.stmin = stp + xtrapl * (stp - S.stx); S.stmax = stp + xtrapu * (stp - S.stx); }
    stp = std::max(stp, stpmin);
    stp = std::min(stp, stpmax);
    if ((S.brackt && (stp <= S.stmin || stp >= S.stmax)) || (S.brackt && S.stmax - S.stmin <= xtol * S.stmax)) stp = S.stx;
    return LS_FG;
}

// Launch a batched FFT over `nplanes` planes starting at `data`: the specialised plane (xy)
// and column (z) kernels of the evaluation pipeline where they exist for the grid's
// lengths, the generic per-axis kernel otherwise.
int launch_fft_planes(mdft_handle *h, double2 *data, int nplanes, int sign) {
    const Grid &g = h->g;
    const int dims[3] = {g.nx, g.ny, g.nz};
    auto axis = [&](int ax) {
        FftAxisArgs a = h->fft[ax].args;
        a.nplanes = nplanes;
        a.sign = sign;
        long long lines_div = (ax == 0) ? (long long)nplanes * g.ny * g.nz : g.nx;
        a.TL = pick_tl(lines_div, dims[ax]);
        long long nlines = (long long)nplanes * g.N / dims[ax];
        size_t smem = fft_smem_bytes<double>(dims[ax], a.TL);
        k_fft_axis<double><<<(unsigned)(nlines / a.TL), kFftThreads, smem, h->stream>>>(data, (const double2 *)h->fft[ax].tw, a);
        h->launches += 1;
    };
    bool xy_done = false;
    if (g.nx == g.ny && sizeof(double2) * (size_t)g.nx * (g.nx + 2) <= 200 * 1024) {
        const cudaError_t e = fft_xy<double>(g.nx, data, (long long)nplanes * g.nz, h->tw64[0].p, sign, h->stream, false,
                                             h->xy_grid_cap64, h->kerr.p);
        if (e == cudaSuccess) { xy_done = true; h->launches += 1; }
        else if (e != cudaErrorNotSupported) return check_cuda(e, "fft xy launch");
        else cudaGetLastError();
    }
    if (!xy_done) {
        axis(0);
        axis(1);
    }
    const cudaError_t e = fft_z<double>(g.nz, data, nplanes, g.nx, g.ny, h->tw64[2].p, sign, h->stream, false);
    if (e == cudaSuccess) h->launches += 1;
    else if (e != cudaErrorNotSupported) return check_cuda(e, "fft z launch");
    else {
        cudaGetLastError();
        axis(2);
    }
    return check_cuda(cudaGetLastError(), "fft launch");
}

}  // namespace

extern "C" {

int mdft_compute_vext(mdft_handle *h, int nsite, const double *q, const double *sig, const double *eps, const double *xyz,
                      int nsv, const double *sq, const double *ssig, const double *seps, const double *sxyz, double rvdw,
                      double *lj_tail) {
    if (!h || nsite < 0 || (nsite > 0 && (!q || !sig || !eps || !xyz)) || nsv <= 0 || !sq || !ssig || !seps || !sxyz) {
        set_error("null or invalid argument");
        return MDFT_E_ARG;
    }
    const Grid &g = h->g;
    const long long N = g.N;
    const size_t nf = (size_t)N * g.no;
    int rc;
    // ---- electrostatics (vextq kept apart in the df buffer until the sum) ----
    bool charged = false;
    for (int s = 0; s < nsite; ++s)
        if (std::fabs(q[s]) > kEpsDp) charged = true;
    bool have_vq = false;
    if (charged) {
        std::vector<double> rho(N, 0.0);
        const int n3[3] = {g.nx, g.ny, g.nz};
        const double L3[3] = {g.lx, g.ly, g.lz};
        const double d3[3] = {g.lx / g.nx, g.ly / g.ny, g.lz / g.nz};
        for (int s = 0; s < nsite; ++s) {  // src/module_solute.f90:193-236
            if (!(std::fabs(q[s]) > kEpsDp)) continue;
            int mi[3], pi[3];
            double wp[3], wm[3];
            for (int d = 0; d < 3; ++d) {
                double x = xyz[3 * s + d];
                double r = std::fabs(x / d3[d] - std::floor(x / d3[d]));
                double md = std::fmod(x, L3[d]);
                if (md < 0) md += L3[d];
                mi[d] = (int)std::floor(md / d3[d]);
                if (mi[d] >= n3[d]) mi[d] = n3[d] - 1;
                pi[d] = (mi[d] + 1) % n3[d];
                wp[d] = r;
                wm[d] = 1.0 - r;
            }
            auto at = [&](int a, int b, int c) -> double & { return rho[((size_t)c * g.ny + b) * g.nx + a]; };
            at(mi[0], mi[1], mi[2]) += q[s] * wm[0] * wm[1] * wm[2];
            at(pi[0], mi[1], mi[2]) += q[s] * wp[0] * wm[1] * wm[2];
            at(mi[0], pi[1], mi[2]) += q[s] * wm[0] * wp[1] * wm[2];
            at(mi[0], mi[1], pi[2]) += q[s] * wm[0] * wm[1] * wp[2];
            at(pi[0], pi[1], mi[2]) += q[s] * wp[0] * wp[1] * wm[2];
            at(pi[0], mi[1], pi[2]) += q[s] * wp[0] * wm[1] * wp[2];
            at(mi[0], pi[1], pi[2]) += q[s] * wm[0] * wp[1] * wp[2];
            at(pi[0], pi[1], pi[2]) += q[s] * wp[0] * wp[1] * wp[2];
        }
        const double vol = d3[0] * d3[1] * d3[2];
        bool allzero = true;
        for (auto &v : rho) {
            v /= vol;
            if (std::fabs(v) > kEpsDp) allzero = false;
        }
        if (!allzero) {
            DevBuf<double> drho, dsq, dsx, drot;
            DevBuf<double2> vk;
            std::vector<double> cq, cx;
            for (int s = 0; s < nsv; ++s)
                if (std::fabs(sq[s]) > kEpsDp) {
                    cq.push_back(sq[s]);
                    cx.insert(cx.end(), sxyz + 3 * s, sxyz + 3 * s + 3);
                }
            if ((rc = alloc_check(drho.alloc(N), "charge density", N * 8))) return rc;
            if ((rc = alloc_check(vk.alloc(N), "V(k)", N * 16))) return rc;
            if ((rc = alloc_check(dsq.alloc(std::max<size_t>(1, cq.size())), "solvent charges", 64))) return rc;
            if ((rc = alloc_check(dsx.alloc(std::max<size_t>(3, cx.size())), "solvent sites", 64))) return rc;
            if ((rc = alloc_check(drot.alloc(9 * (size_t)g.no), "orientations", 72 * g.no))) return rc;
            cudaMemcpyAsync(drho.p, rho.data(), N * 8, cudaMemcpyHostToDevice, h->stream);
            if (!cq.empty()) {
                cudaMemcpyAsync(dsq.p, cq.data(), cq.size() * 8, cudaMemcpyHostToDevice, h->stream);
                cudaMemcpyAsync(dsx.p, cx.data(), cx.size() * 8, cudaMemcpyHostToDevice, h->stream);
            }
            cudaMemcpyAsync(drot.p, g.rotm.data(), 72 * (size_t)g.no, cudaMemcpyHostToDevice, h->stream);
            k_real_to_cplx<<<vec_grid(), 256, 0, h->stream>>>(drho.p, h->planes.p, N);
            if ((rc = launch_fft_planes(h, h->planes.p, 1, -1))) return rc;
            k_poisson<<<vec_grid(), 256, 0, h->stream>>>(h->planes.p, vk.p, g.nx, g.ny, g.nz, g.lx, g.ly, g.lz);
            const int batch = g.np;
            for (int io0 = 0; io0 < g.no; io0 += batch) {
                SigmaArgs sa{g.nx, g.ny, g.nz, g.no, 2.0 * kPi / g.lx, 2.0 * kPi / g.ly, 2.0 * kPi / g.lz, (int)cq.size(), io0,
                             std::min(batch, g.no - io0)};
                k_sigma_product<<<vec_grid(), 256, 0, h->stream>>>(vk.p, h->planes.p, drot.p, dsq.p, dsx.p, sa);
                if ((rc = launch_fft_planes(h, h->planes.p, sa.nbatch, +1))) return rc;
                k_sigma_store<<<vec_grid(), 256, 0, h->stream>>>(h->planes.p, h->df.p, g.no, io0, sa.nbatch, N, kQfact / (double)N);
            }
            if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "electrostatics"))) return rc;
            have_vq = true;
        }
    }
    // ---- Lennard-Jones (src/module_lennardjones.f90:9-226) ----
    const double cutoff = rvdw;
    if (cutoff > g.lx * 0.5 || cutoff > g.ly * 0.5 || cutoff > g.lz * 0.5) {
        set_error("LJ cut-off %g larger than half the box", cutoff);
        return MDFT_E_ARG;
    }
    const int n3[3] = {g.nx, g.ny, g.nz};
    const double L3[3] = {g.lx, g.ly, g.lz}, D3[3] = {g.dx, g.dy, g.dz};
    int tabsize[3];
    for (int d = 0; d < 3; ++d) tabsize[d] = (int)std::floor(2 * cutoff / D3[d]) + 1;
    bool only_origin = true;
    for (int s = 0; s < nsv; ++s)
        if (seps[s] != 0.0 && (sxyz[3 * s] != 0.0 || sxyz[3 * s + 1] != 0.0 || sxyz[3 * s + 2] != 0.0)) only_origin = false;
    std::vector<LJTerm> terms;
    double ljcorr = 0.0;
    for (int u = 0; u < nsite; ++u) {
        if (eps[u] <= kEpsDp) continue;
        LJTerm base{};
        base.px = xyz[3 * u]; base.py = xyz[3 * u + 1]; base.pz = xyz[3 * u + 2];
        for (int d = 0; d < 3; ++d) {
            double r = xyz[3 * u + d];
            int mn = (int)std::floor(std::fmod(r - cutoff + L3[d], L3[d]) / D3[d]) + 1;
            int mx = (int)std::floor(std::fmod(r + cutoff, L3[d]) / D3[d]) + 1;
            if (mn < 1 || mx > n3[d]) {
                set_error("LJ node range check failed for site %d", u + 1);
                return MDFT_E_ARG;
            }
            // the reference loops over the first tabsize entries of the realised table
            int ts = tabsize[d];
            base.lo[d][1] = 1; base.hi[d][1] = 0;  // empty
            if (mn < mx) {
                base.lo[d][0] = mn - 1;
                base.hi[d][0] = std::min(mx, mn + ts - 1) - 1;
            } else {
                int first = std::min(mx, ts);
                base.lo[d][0] = 0;
                base.hi[d][0] = first - 1;
                int rest = ts - first;
                if (rest > 0) {
                    base.lo[d][1] = mn - 1;
                    base.hi[d][1] = std::min(n3[d], mn + rest - 1) - 1;
                }
            }
        }
        for (int ss = 0; ss < nsv; ++ss) {
            if (seps[ss] <= kEpsDp) continue;
            LJTerm t = base;
            t.epsuv = std::sqrt(eps[u] * seps[ss]);
            t.siguv6 = powi((sig[u] + ssig[ss]) * 0.5, 6);
            t.sx = sxyz[3 * ss]; t.sy = sxyz[3 * ss + 1]; t.sz = sxyz[3 * ss + 2];
            ljcorr = ljcorr - (16.0 * 3.14159 / 3.0) * t.epsuv * t.siguv6 * g.n0 / powi(cutoff, 3);
            terms.push_back(t);
        }
    }
    if ((rc = check_cuda(cudaMemsetAsync(h->vext.p, 0, nf * 8, h->stream), "vext clear"))) return rc;
    if (!terms.empty()) {
        DevBuf<LJTerm> dt;
        DevBuf<double> drot;
        if ((rc = alloc_check(dt.alloc(terms.size()), "LJ terms", terms.size() * sizeof(LJTerm)))) return rc;
        if ((rc = alloc_check(drot.alloc(9 * (size_t)g.no), "orientations", 72 * g.no))) return rc;
        cudaMemcpyAsync(dt.p, terms.data(), terms.size() * sizeof(LJTerm), cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(drot.p, g.rotm.data(), 72 * (size_t)g.no, cudaMemcpyHostToDevice, h->stream);
        LJArgs la{g.nx, g.ny, g.nz, g.no, g.dx, g.dy, g.dz, g.lx, g.ly, g.lz, cutoff * cutoff, (int)terms.size(), only_origin ? 1 : 0};
        k_lj<<<vec_grid(), 256, 0, h->stream>>>(h->vext.p, dt.p, drot.p, la);
        if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "Lennard-Jones"))) return rc;
    }
    // ---- vext_total_sum ----
    DevBuf<int> flag;
    if ((rc = alloc_check(flag.alloc(1), "flag", 4))) return rc;
    cudaMemsetAsync(flag.p, 0, 4, h->stream);
    k_vext_total<<<vec_grid(), 256, 0, h->stream>>>(h->vext.p, have_vq ? h->df.p : nullptr, kQfact / 2.0, (long long)nf, flag.p);
    int hflag = 0;
    cudaMemcpyAsync(&hflag, flag.p, 4, cudaMemcpyDeviceToHost, h->stream);
    if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "vext sum"))) return rc;
    if (hflag & 1) { set_error("NaN or Inf in vext"); return MDFT_E_NUMERIC; }
    if (hflag & 2) { set_error("vext below -qfact/2 somewhere"); return MDFT_E_NUMERIC; }
    h->have_vext = true;
    if (lj_tail) *lj_tail = ljcorr;
    return MDFT_OK;
}

int mdft_guess_density(const mdft_handle *h, double *xi) {
    if (!h || !xi) { set_error("null argument"); return MDFT_E_ARG; }
    const size_t nf = (size_t)h->g.N * h->g.no;
    const double vmax = (-std::log(kEpsDp) - (double)0.05f) * h->g.kT;
    mdft_handle *hh = const_cast<mdft_handle *>(h);
    k_guess<<<vec_grid(), 256, 0, h->stream>>>(h->vext.p, hh->xi.p, vmax, (long long)nf);
    int rc = check_cuda(cudaMemcpyAsync(xi, h->xi.p, nf * 8, cudaMemcpyDeviceToHost, h->stream), "guess download");
    if (rc) return rc;
    return check_cuda(cudaStreamSynchronize(h->stream), "guess");
}

}  // extern "C"

namespace {

// The L-BFGS loop on L.x (already holding the start point).
// History of the compact limited-memory matrix.  Slots head, head+1, ... (mod m) hold the
// pairs oldest first; Gram entries are kept by slot: sy[i*m+j] = s_i.y_j (i not newer than
// j), yy[i*m+j] = y_i.y_j, and sg/yg = s_i.g, y_i.g at the current gradient.
// Relative rounding noise assumed for the FP32 phase of a mixed solve (FP32 planes and
// per-element arithmetic, FP64 sums), relative to the size of the terms F is the sum of
// (|F_id| + |F_ext| + |F_exc| + |constant|, which can exceed |F| by orders of magnitude):
// the tolerance of its approximate Wolfe test.
constexpr double kMixedNoiseRel = 1e-6;
// Trial points one line search of the FP32 phase may evaluate; more means the search is
// chasing rounding noise, and the phase ends as at a failed search (the FP64 phase goes on).
constexpr int kMixedMaxTrials = 8;

struct LbfgsHist {
    int m = 0, col = 0, head = 0;
    bool low = false;  // mixed solves: pairs stored in BF16, gradient and direction vectors in FP32
    double theta = 1.0, gg = 0.0, sty = 0.0;  // sty: s.y of the pair formed last, from the stored values
    std::vector<double> sy, yy, sg, yg;
    void reset(int mm, bool lowp = false) {
        m = mm;
        low = lowp;
        col = 0;
        head = 0;
        theta = 1.0;
        sy.assign((size_t)m * m, 0.0);
        yy.assign((size_t)m * m, 0.0);
        sg.assign(m, 0.0);
        yg.assign(m, 0.0);
    }
    int slot(int c) const { return (head + c) % m; }
};

constexpr int kRowsBase = 64;  // first device scalar slot of the history inner products

// slot j of the S or Y history in the storage type of H
inline void *hist_slot(const LbfgsHist &H, double *base, int j, long long n) {
    return H.low ? (void *)(reinterpret_cast<__nv_bfloat16 *>(base) + (size_t)j * n) : (void *)(base + (size_t)j * n);
}

template <typename TS, typename TV, int K, bool PAIR, bool SELF>
void launch_dots_v(const PairDotsArgs &a, cudaStream_t st) {
    // 16-byte accesses of the narrower of the vector and history types (8 FP32/BF16 elements)
    constexpr int V = 16 / (int)(sizeof(TS) < sizeof(TV) ? sizeof(TS) : sizeof(TV));
    if (a.n % V == 0) k_pair_dots<TS, TV, K, PAIR, SELF, V><<<vec_grid(), kRedThreads, 0, st>>>(a);
    else k_pair_dots<TS, TV, K, PAIR, SELF, 1><<<vec_grid(), kRedThreads, 0, st>>>(a);
}
template <int K>
void launch_dots(bool low, bool pair, bool self, const PairDotsArgs &a, cudaStream_t st) {
    if (low) {
        if (!pair) launch_dots_v<__nv_bfloat16, float, K, false, false>(a, st);
        else if (self) launch_dots_v<__nv_bfloat16, float, K, true, true>(a, st);
        else launch_dots_v<__nv_bfloat16, float, K, true, false>(a, st);
    } else {
        if (!pair) launch_dots_v<double, double, K, false, false>(a, st);
        else if (self) launch_dots_v<double, double, K, true, true>(a, st);
        else launch_dots_v<double, double, K, true, false>(a, st);
    }
}

// Inner products of the history with a gradient g, launched without waiting: `slots` are
// the history slots read; with pair, also those of the candidate pair (stp d, g - gold).
// The row layout of each launch goes to `plan`; the rows land in h->vsc from kRowsBase on
// and are copied to h->h_vsc in the same stream (read them after the next synchronise).
struct DotsPlan {
    std::vector<int> slots;
    bool pair = false;
    std::vector<int> base, kk;
    int end = kRowsBase;
};
int launch_history_dots(mdft_handle *h, const LbfgsHist &H, const double *g, const double *gold, const double *d, double stp,
                        DotsPlan &P) {
    LbfgsState &L = h->lb;
    const long long n = L.n;
    cudaStream_t st = h->stream;
    const int ns = (int)P.slots.size();
    const int ngroups = std::max(1, (ns + kPairGroup - 1) / kPairGroup);
    P.base.assign(ngroups, 0);
    P.kk.assign(ngroups, 0);
    int off = kRowsBase;
    for (int gi = 0; gi < ngroups; ++gi) {
        const int K = std::min(kPairGroup, ns - kPairGroup * gi);
        const bool self = P.pair && gi == 0;
        const int rows = pair_rows(K, P.pair, self);
        if (off + rows > kScalarSlots) {
            set_error("history too long for the scalar slots");
            return MDFT_E_ARG;
        }
        PairDotsArgs a{};
        a.g = g;
        a.gold = gold;
        a.d = d;
        for (int k = 0; k < K; ++k) {
            a.s[k] = hist_slot(H, L.S.p, P.slots[kPairGroup * gi + k], n);
            a.y[k] = hist_slot(H, L.Y.p, P.slots[kPairGroup * gi + k], n);
        }
        a.stp = stp;
        a.n = n;
        a.part = h->vpart.p;
        switch (K) {
            case 0: launch_dots<0>(H.low, P.pair, self, a, st); break;
            case 1: launch_dots<1>(H.low, P.pair, self, a, st); break;
            case 2: launch_dots<2>(H.low, P.pair, self, a, st); break;
            case 3: launch_dots<3>(H.low, P.pair, self, a, st); break;
            case 4: launch_dots<4>(H.low, P.pair, self, a, st); break;
            case 5: launch_dots<5>(H.low, P.pair, self, a, st); break;
            case 6: launch_dots<6>(H.low, P.pair, self, a, st); break;
            case 7: launch_dots<7>(H.low, P.pair, self, a, st); break;
            default: launch_dots<8>(H.low, P.pair, self, a, st); break;
        }
        k_finish_rows<<<rows, 256, 0, st>>>(h->vpart.p, (int)vec_grid(), h->vsc.p + off);
        h->launches += 2;
        P.base[gi] = off;
        P.kk[gi] = K;
        off += rows;
    }
    P.end = off;
    int rc = check_cuda(cudaGetLastError(), "history inner products");
    if (rc) return rc;
    return check_cuda(cudaMemcpyAsync(h->h_vsc + kRowsBase, h->vsc.p + kRowsBase, (off - kRowsBase) * sizeof(double),
                                      cudaMemcpyDeviceToHost, st), "history inner products");
}

// Candidate pair's products read back by read_history_dots
struct PairRows {
    std::vector<double> s_yn, y_yn;  // by slot
    double yy = 0, yg = 0, sg = 0, sy = 0;
};

// After the synchronise: s_i.g, y_i.g and g.g into H; the candidate's products into R.
int read_history_dots(const mdft_handle *h, LbfgsHist &H, const DotsPlan &P, PairRows *R) {
    const double *r = h->h_vsc;
    for (int i = kRowsBase; i < P.end; ++i)
        if (!std::isfinite(r[i])) {
            set_error("non-finite history inner product");
            return MDFT_E_NUMERIC;
        }
    if (R) {
        R->s_yn.assign(H.m, 0.0);
        R->y_yn.assign(H.m, 0.0);
    }
    for (size_t gi = 0; gi < P.base.size(); ++gi) {
        const int K = P.kk[gi], b = P.base[gi];
        for (int k = 0; k < K; ++k) {
            const int j = P.slots[kPairGroup * gi + k];
            H.sg[j] = r[b + k];
            H.yg[j] = r[b + K + k];
            if (P.pair && R) {
                R->s_yn[j] = r[b + 2 * K + 1 + k];
                R->y_yn[j] = r[b + 3 * K + 1 + k];
            }
        }
        if (gi == 0) {
            H.gg = r[b + 2 * K];
            if (P.pair && R) {
                R->yy = r[b + 4 * K + 1];
                R->yg = r[b + 4 * K + 2];
                R->sg = r[b + 4 * K + 3];
                R->sy = r[b + 4 * K + 4];
            }
        }
    }
    return 0;
}

// Blocking form: products of every current slot with g (no candidate pair).
int history_dots_now(mdft_handle *h, LbfgsHist &H, const double *g) {
    DotsPlan P;
    for (int c = 0; c < H.col; ++c) P.slots.push_back(H.slot(c));
    int rc = launch_history_dots(h, H, g, nullptr, nullptr, 0.0, P);
    if (rc) return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "history inner products"))) return rc;
    return read_history_dots(h, H, P, nullptr);
}

template <int K, bool NP>
void launch_direction_k(bool low, bool x32, const DirArgs &a, cudaStream_t st) {
    if (low && x32) {
        if (a.n % 4 == 0) k_direction<__nv_bfloat16, float, float, K, NP, 4><<<vec_grid(), kRedThreads, 0, st>>>(a);
        else k_direction<__nv_bfloat16, float, float, K, NP, 1><<<vec_grid(), kRedThreads, 0, st>>>(a);
    } else if (low) {
        if (a.n % 4 == 0) k_direction<__nv_bfloat16, float, double, K, NP, 4><<<vec_grid(), kRedThreads, 0, st>>>(a);
        else k_direction<__nv_bfloat16, float, double, K, NP, 1><<<vec_grid(), kRedThreads, 0, st>>>(a);
    } else {
        if (a.n % 2 == 0) k_direction<double, double, double, K, NP, 2><<<vec_grid(), kRedThreads, 0, st>>>(a);
        else k_direction<double, double, double, K, NP, 1><<<vec_grid(), kRedThreads, 0, st>>>(a);
    }
}
template <int K>
void launch_direction(bool low, bool x32, bool np, const DirArgs &a, cudaStream_t st) {
    if (np) launch_direction_k<K, true>(low, x32, a, st);
    else launch_direction_k<K, false>(low, x32, a, st);
}

// Pair accepted in the last step and not yet stored: k_direction forms it from the
// direction it replaces (s = stp d) and the previous gradient (y = g - gold).
struct PendingPair {
    int slot = -1;
    const double *gold = nullptr;
    double stp = 1.0;
};

// d = -H g with H the inverse of the compact L-BFGS matrix, H0 = I/theta:
//   H g = g/theta + S top - Y u/theta,  u = R^-1 S'g,  top = R^-T ((D + Y'Y/theta) u - Y'g/theta)
// (R = upper triangle of S'Y, D its diagonal; no history: d = -g/theta).  The slope g.d and
// d.d come from the Gram data (no synchronise); a pending pair is stored on the way.
// With x non-null the last launch also writes the first trial point xt = x + stp_t d.
// x, xt: FP32 when x32 (the FP32 phase of a mixed solve), else FP64.
int direction(mdft_handle *h, const LbfgsHist &H, const void *g, void *d, const PendingPair &pend, double *gd, double *dd,
              const void *x = nullptr, void *xt = nullptr, double stp_t = 1.0, bool x32 = false) {
    LbfgsState &L = h->lb;
    const long long n = L.n;
    const int k = H.col, m = H.m;
    cudaStream_t st = h->stream;
    const double gam = 1.0 / H.theta;
    std::vector<const void *> vec;
    std::vector<double> coef;
    double cs_n = 0.0, cy_n = 0.0;
    double slope = -gam * H.gg, dnorm2 = gam * gam * H.gg;
    if (k > 0) {
        std::vector<int> idx(k);
        for (int c = 0; c < k; ++c) idx[c] = H.slot(c);
        auto R = [&](int a, int b) { return H.sy[(size_t)idx[a] * m + idx[b]]; };
        auto YY = [&](int a, int b) { return H.yy[(size_t)idx[a] * m + idx[b]]; };
        std::vector<double> u(k), w(k), top(k);
        for (int a = k - 1; a >= 0; --a) {
            double s = H.sg[idx[a]];
            for (int b = a + 1; b < k; ++b) s -= R(a, b) * u[b];
            u[a] = s / R(a, a);
        }
        for (int a = 0; a < k; ++a) {
            double yu = 0.0;
            for (int b = 0; b < k; ++b) yu += YY(a, b) * u[b];
            w[a] = R(a, a) * u[a] + gam * yu - gam * H.yg[idx[a]];
        }
        for (int a = 0; a < k; ++a) {
            double s = w[a];
            for (int b = 0; b < a; ++b) s -= R(b, a) * top[b];
            top[a] = s / R(a, a);
        }
        for (int a = 0; a < k; ++a) {
            const double cs = -top[a], cy = gam * u[a];
            if (!std::isfinite(cs) || !std::isfinite(cy)) {
                set_error("non-finite search-direction coefficient");
                return MDFT_E_NUMERIC;
            }
            slope += cs * H.sg[idx[a]] + cy * H.yg[idx[a]];
            if (idx[a] == pend.slot) {
                cs_n = cs;
                cy_n = cy;
                continue;
            }
            vec.push_back(hist_slot(H, L.S.p, idx[a], n));
            coef.push_back(cs);
            vec.push_back(hist_slot(H, L.Y.p, idx[a], n));
            coef.push_back(cy);
        }
    }
    const int nv = (int)vec.size();
    constexpr int kV = 2 * kPairGroup;
    const int nl = std::max(1, (nv + kV - 1) / kV);
    for (int li = 0; li < nl; ++li) {
        DirArgs a{};
        a.g = g;
        a.cg = -gam;
        const bool np = li == 0 && pend.slot >= 0;
        if (np) {
            a.gold = pend.gold;
            a.stp = pend.stp;
            a.cs_n = cs_n;
            a.cy_n = cy_n;
            a.snew = hist_slot(H, L.S.p, pend.slot, n);
            a.ynew = hist_slot(H, L.Y.p, pend.slot, n);
        }
        const int K = std::min(kV, nv - kV * li);
        for (int j = 0; j < K; ++j) {
            a.v[j] = vec[kV * li + j];
            a.cv[j] = coef[kV * li + j];
        }
        a.d = d;
        a.accumulate = li > 0;
        a.n = n;
        if (li == nl - 1 && x) {
            a.x = x;
            a.xt = xt;
            a.stp_t = stp_t;
        }
        switch (K) {
            case 0: launch_direction<0>(H.low, x32, np, a, st); break;
            case 2: launch_direction<2>(H.low, x32, np, a, st); break;
            case 4: launch_direction<4>(H.low, x32, np, a, st); break;
            case 6: launch_direction<6>(H.low, x32, np, a, st); break;
            case 8: launch_direction<8>(H.low, x32, np, a, st); break;
            case 10: launch_direction<10>(H.low, x32, np, a, st); break;
            case 12: launch_direction<12>(H.low, x32, np, a, st); break;
            case 14: launch_direction<14>(H.low, x32, np, a, st); break;
            default: launch_direction<16>(H.low, x32, np, a, st); break;
        }
        h->launches += 1;
    }
    *gd = slope;
    *dd = dnorm2;
    if (!std::isfinite(slope)) {
        set_error("non-finite search direction");
        return MDFT_E_NUMERIC;
    }
    return check_cuda(cudaGetLastError(), "direction");
}

// MDFT_TRACE: one stderr line per accepted iteration with F, max|df| and the particle
// deficit dN of the current point (dG along the path = F - dN/n0 Pbulk + LJ tail).
void trace_iter(mdft_handle *h, const double *x, int iter, int nfgv, double f, double gmax, double stp) {
    if (!h->trace) return;
    const Grid &g = h->g;
    if (!x) {  // FP32 point: no dN
        std::fprintf(stderr, "mdft-trace it %d nfg %d prec %s f %.15e gmax %.6e stp %.6e dN nan\n", iter, nfgv,
                     h->eval_prec == MDFT_PREC_MIXED ? "mixed" : "fp64", f, gmax, stp);
        return;
    }
    k_density_sum<<<vec_grid(), 256, 0, h->stream>>>(x, h->w.p, g.no, (long long)h->lb.n, g.rho0, h->vpart.p);
    k_finish_dot_max<<<1, 256, 0, h->stream>>>(h->vpart.p, vec_grid(), h->vsc.p, 4);
    cudaMemcpyAsync(h->h_vsc + 4, h->vsc.p + 4, 8, cudaMemcpyDeviceToHost, h->stream);
    cudaStreamSynchronize(h->stream);
    const double dN = g.n0 * (g.lx * g.ly * g.lz) - h->h_vsc[4] * g.dv;
    std::fprintf(stderr, "mdft-trace it %d nfg %d prec %s f %.15e gmax %.6e stp %.6e dN %.15e\n", iter, nfgv,
                 h->eval_prec == MDFT_PREC_MIXED ? "mixed" : "fp64", f, gmax, stp, dN);
}

// The L-BFGS iteration of src/module_lbfgs_nocedal_mdft.f90 mainlb (no bounds): search
// direction, Moré-Thuente line search (lnsrlb/dcsrch), stopping tests, matupd.  The
// current and trial points (x, g) live in two buffer pairs that swap on acceptance, so a
// rejected trial costs no copies.  H carries the history in and out (an empty H starts
// from steepest descent with stp = 1/|d|); with stop_on_ls_fail a failed line search
// ends the run instead of restarting from an empty history; noise_rel > 0 adds the
// approximate Wolfe acceptance for an F with that relative rounding noise (the FP32
// phase).  The result is left in L.x.
int minimize_impl(mdft_handle *h, const mdft_minimize_opts *o, mdft_minimize_result *res, LbfgsHist &H,
                  bool stop_on_ls_fail, double noise_rel = 0.0) {
    int rc;
    LbfgsState &L = h->lb;
    const long long n = L.n;
    const int m = o->m;
    cudaStream_t st = h->stream;
    if (H.m != m) H.reset(m, H.low);
    double *const g0 = h->mix ? mixture_grad(h->mix) : h->df.p;  // the gradient's home buffer
    double *xc = L.x.p, *xt = L.t.p, *gc = g0, *gt = L.r.p;  // gc, gt and L.d hold TV values
    const bool v32 = H.low;  // mixed solves: FP32 gradient and direction vectors
    // FP32 phase of a mixed solve: the point too is FP32 (xc, xt then hold floats); the FP64
    // start point in L.x is converted into L.t first, and the result back into L.x at the end
    const bool x32 = v32 && h->eval_prec == MDFT_PREC_MIXED && h->pt_ok32 && h->gt_ncol32 > 0 && h->vext32.p;
    if (x32) {
        k_convert<double, float><<<vec_grid(), 256, 0, st>>>(reinterpret_cast<float *>(L.t.p), L.x.p, n);
        h->launches += 1;
        std::swap(xc, xt);
    }
    const double epsmch = kEpsDp;
    const double ftol = (double)0.001f, gtol = (double)0.9f, xtol = (double)0.1f, big = 1.0 + 10;
    double f = 0, fold = 0, stp = 0, gd = 0, gdold = 0, gmax = 0, dd = 0, guni = 0, fscale = 0, fscale_t = 0;
    int iter = 0, nfgv = 0, status = 3;
    const bool fresh = H.col == 0;
    PendingPair pend;
    // projgr's test (max|df| <= pgtol), plus, when asked, the uniform-mode gradient bound
    auto converged = [&](double gm, double gu) { return gm <= o->pgtol && (o->guni_tol <= 0.0 || std::fabs(gu) <= o->guni_tol); };
    if ((rc = eval_fg(h, xc, gc, nullptr, &f, nullptr, &gmax, v32, x32, &guni, &fscale))) return rc;
    nfgv = 1;
    trace_iter(h, x32 ? nullptr : xc, 0, nfgv, f, gmax, 0.0);
    double sbgnrm = gmax;
    if (converged(sbgnrm, guni)) { status = 0; goto done; }
    if ((rc = history_dots_now(h, H, gc))) return rc;  // s_i.g, y_i.g, g.g at the start point
    while (iter < o->itermax) {
        // ---- search direction (stores the pair accepted last step) and the first trial ----
        const double stpmx = big;
        // lnsrlb's first step: 1/|d| on the first iteration from an empty history, where
        // d = -g/theta and |d|^2 = g.g/theta^2, else 1
        stp = (iter == 0 && fresh) ? std::min(1.0 / std::sqrt(H.gg / (H.theta * H.theta)), stpmx) : 1.0;
        if ((rc = direction(h, H, gc, L.d.p, pend, &gd, &dd, xc, xt, stp, x32))) return rc;
        pend = PendingPair();
        // ---- line search (lnsrlb) ----
        fold = f;
        gdold = gd;
        int ifun = 0, iback = 0, info = 0;
        double gmax_t = gmax, guni_t = guni;
        // the slot a pair accepted in this step would take, and the slots that stay
        const int tnext = H.col < m ? H.slot(H.col) : H.head;
        DotsPlan P;
        P.pair = true;
        for (int c = 0; c < H.col; ++c)
            if (H.slot(c) != tnext) P.slots.push_back(H.slot(c));
        PairRows PR;
        LineSearch LS;
        if (gd >= 0.0) {
            info = -4;
        } else {
            int task = dcsrch(f, gd, stp, ftol, gtol, xtol, 0.0, stpmx, true, LS);
            while (task == LS_FG) {
                ++ifun;
                ++nfgv;
                iback = ifun - 1;
                if (iback >= 20) break;
                if (noise_rel > 0.0 && ifun > kMixedMaxTrials) {  // FP32 phase: the search chases noise
                    iback = 20;
                    break;
                }
                if (ifun > 1) {  // the first trial point came with the direction
                    if (x32) {
                        const float *d32 = reinterpret_cast<const float *>(L.d.p);
                        float *xt32 = reinterpret_cast<float *>(xt);
                        const float *xc32 = reinterpret_cast<const float *>(xc);
                        if (n % 4 == 0) k_trial<float, float, 4><<<vec_grid(), 256, 0, st>>>(xt32, xc32, d32, stp, n);
                        else k_trial<float, float, 1><<<vec_grid(), 256, 0, st>>>(xt32, xc32, d32, stp, n);
                    } else if (v32) {
                        const float *d32 = reinterpret_cast<const float *>(L.d.p);
                        if (n % 4 == 0) k_trial<float, double, 4><<<vec_grid(), 256, 0, st>>>(xt, xc, d32, stp, n);
                        else k_trial<float, double, 1><<<vec_grid(), 256, 0, st>>>(xt, xc, d32, stp, n);
                    } else {
                        if (n % 2 == 0) k_trial<double, double, 2><<<vec_grid(), 256, 0, st>>>(xt, xc, L.d.p, stp, n);
                        else k_trial<double, double, 1><<<vec_grid(), 256, 0, st>>>(xt, xc, L.d.p, stp, n);
                    }
                    h->launches += 1;
                }
                if ((rc = eval_launch(h, xt, gt, L.d.p, v32, x32))) return rc;
                // the history's products with this trial gradient, queued before the one
                // synchronise of the step (used if the trial is accepted)
                if ((rc = launch_history_dots(h, H, gt, gc, L.d.p, stp, P))) return rc;
                if ((rc = eval_finish(h, &f, &gd, &gmax_t, &guni_t, &fscale_t))) return rc;
                const double stp_eval = stp;
                task = dcsrch(f, gd, stp, ftol, gtol, xtol, 0.0, stpmx, false, LS);
                // Approximate Wolfe test (Hager and Zhang, SIAM J. Optim. 16 (2005) 170, eq. 4.1):
                // when F carries rounding noise of relative size noise_rel (relative to the
                // terms it sums), a trial whose F is within that noise of F(0) and whose slope
                // satisfies sigma g'(0) <= g'(stp) <= (2 delta - 1) g'(0) is accepted.
                if (task == LS_FG && noise_rel > 0.0 && f <= fold + noise_rel * fscale &&
                    gd >= 0.9 * gdold && gd <= -0.8 * gdold) {
                    stp = stp_eval;
                    task = LS_CONV;
                }
                if (task != LS_FG) stp = stp_eval;
            }
            if (task == LS_ERROR) info = -1;
        }
        if (info != 0 || iback >= 20) {
            f = fold;  // x and g stay at the last accepted point (H.gg still belongs to it)
            if (h->trace) std::fprintf(stderr, "mdft-trace line search failed (info %d, iback %d, col %d)\n", info, iback, H.col);
            if (H.col == 0 || stop_on_ls_fail) {
                status = 2;
                ++iter;
                goto done;
            }
            H.col = 0;
            H.head = 0;
            H.theta = 1.0;
            continue;
        }
        ++iter;
        std::swap(xc, xt);
        std::swap(gc, gt);
        gmax = gmax_t;
        guni = guni_t;
        fscale = fscale_t;
        sbgnrm = gmax;
        trace_iter(h, x32 ? nullptr : xc, iter, nfgv, f, gmax, stp);
        if (converged(sbgnrm, guni)) { status = 0; goto done; }
        if ((fold - f) <= o->ftol_abs) { status = 1; goto done; }
        // ---- BFGS update (matupd) ----
        double dr, ddum;
        if (stp == 1.0) { dr = gd - gdold; ddum = -gdold; }
        else { dr = (gd - gdold) * stp; ddum = -gdold * stp; }
        if (dr <= epsmch * ddum) {  // update skipped: products of every slot with the new g
            if ((rc = history_dots_now(h, H, gc))) return rc;
            continue;
        }
        if ((rc = read_history_dots(h, H, P, &PR))) return rc;
        if (H.col < m) ++H.col;
        else H.head = (H.head + 1) % m;
        const int t = tnext;
        for (int j : P.slots) {
            H.sy[(size_t)j * m + t] = PR.s_yn[j];
            H.yy[(size_t)j * m + t] = H.yy[(size_t)t * m + j] = PR.y_yn[j];
        }
        H.yy[(size_t)t * m + t] = PR.yy;
        H.sg[t] = PR.sg;
        H.yg[t] = PR.yg;
        // FP64 history: s.y = dr as the reference's matupd; BF16 history: s.y of the stored pair
        const double sty = H.low ? PR.sy : dr;
        H.sy[(size_t)t * m + t] = sty;
        H.theta = PR.yy / sty;
        pend.slot = t;
        pend.gold = gt;  // the previous gradient (buffers swapped above)
        pend.stp = stp;
    }
done:
    if (pend.slot >= 0) {
        // the last accepted pair is part of H (a later phase may continue with it): store it
        double gd2, dd2;
        if ((rc = direction(h, H, gc, L.d.p, pend, &gd2, &dd2))) return rc;
    }
    if (x32) {
        // the FP32 point back to FP64 in L.x (through L.t when it sits in L.x's storage)
        const float *x32p = reinterpret_cast<const float *>(xc);
        if (xc == L.t.p) {
            k_convert<float, double><<<vec_grid(), 256, 0, st>>>(L.x.p, x32p, n);
        } else {
            k_convert<float, double><<<vec_grid(), 256, 0, st>>>(L.t.p, x32p, n);
            cudaMemcpyAsync(L.x.p, L.t.p, n * 8, cudaMemcpyDeviceToDevice, st);
        }
        h->launches += 1;
    } else if (xc != L.x.p) {
        cudaMemcpyAsync(L.x.p, xc, n * 8, cudaMemcpyDeviceToDevice, st);
    }
    if (gc != g0) cudaMemcpyAsync(g0, gc, n * (v32 ? 4 : 8), cudaMemcpyDeviceToDevice, st);
    if ((rc = check_cuda(cudaStreamSynchronize(st), "minimize"))) return rc;
    res->f = f;
    res->pgnorm = sbgnrm;
    res->guni = guni;
    res->iterations = iter;
    res->evaluations = nfgv;
    res->status = status;
    return MDFT_OK;
}

int check_min_opts(const mdft_minimize_opts *o) {
    if (o->m < 1 || o->m > 64 || o->itermax < 1) { set_error("invalid minimiser options"); return MDFT_E_ARG; }
    if (o->precision != MDFT_PREC_FP64 && o->precision != MDFT_PREC_MIXED) { set_error("unknown precision %d", o->precision); return MDFT_E_ARG; }
    return 0;
}

// FP64 solve, or the mixed solve: L-BFGS with FP32-pipeline evaluations until its
// stopping test holds or its line search fails, then (polish) FP64 iterations from that
// point that keep the history, or one FP64 evaluation.  F, max|df| and the status are FP64's.
int solve_phases(mdft_handle *h, const mdft_minimize_opts *o, mdft_minimize_result *res) {
    const int saved = h->eval_prec;
    int rc;
    LbfgsHist H;
    // BF16 history and FP32 vectors for mixed solves where the bulk-copy gathers (FP32 and, for
    // the FP64 check and polish, FP64) can take FP32 vectors
    H.reset(o->m, o->precision == MDFT_PREC_MIXED && h->gt_ncol32 > 0 && h->gt_ncol64 > 0);
    res->evaluations_mixed = 0;
    if (o->precision == MDFT_PREC_MIXED) {
        if (H.low && h->pt_ok32) {
            // FP32 copy of vext for the FP32 phase (vext does not change during the solve)
            const size_t nf = (size_t)h->g.N * h->g.no;
            if (!h->vext32.p && (rc = alloc_check(h->vext32.alloc(nf), "FP32 vext", nf * 4))) return rc;
            k_convert<double, float><<<vec_grid(), 256, 0, h->stream>>>(h->vext32.p, h->vext.p, (long long)nf);
            h->launches += 1;
        }
        h->eval_prec = MDFT_PREC_MIXED;
        mdft_minimize_opts o1 = *o;
        if (o->pgtol_mixed > 0) o1.pgtol = o->pgtol_mixed;
        mdft_minimize_result r1{};
        rc = minimize_impl(h, &o1, &r1, H, true, kMixedNoiseRel);
        h->eval_prec = MDFT_PREC_FP64;
        if (!rc && o->polish) {
            rc = minimize_impl(h, o, res, H, false);
            res->iterations += r1.iterations;
        } else if (!rc) {
            double f = 0.0, gmax = 0.0, guni = 0.0;
            rc = eval_fg(h, h->lb.x.p, h->df.p, nullptr, &f, nullptr, &gmax, false, false, &guni);
            *res = r1;
            res->f = f;
            res->pgnorm = gmax;
            res->guni = guni;
            res->evaluations = 1;
        }
        res->evaluations_mixed = r1.evaluations;
    } else {
        h->eval_prec = MDFT_PREC_FP64;
        rc = minimize_impl(h, o, res, H, false);
    }
    h->eval_prec = saved;
    return rc;
}

}  // namespace

extern "C" {

int mdft_minimize(mdft_handle *h, double *xi, const mdft_minimize_opts *o, mdft_minimize_result *res) {
    if (!h || !xi || !o || !res) { set_error("null argument"); return MDFT_E_ARG; }
    int rc = check_min_opts(o);
    if (rc) return rc;
    if ((rc = lbfgs_alloc(h, o->m))) return rc;
    LbfgsState &L = h->lb;
    if ((rc = check_cuda(cudaMemcpyAsync(L.x.p, xi, L.n * 8, cudaMemcpyHostToDevice, h->stream), "xi upload"))) return rc;
    if ((rc = solve_phases(h, o, res))) return rc;
    if ((rc = check_cuda(cudaMemcpyAsync(xi, L.x.p, L.n * 8, cudaMemcpyDeviceToHost, h->stream), "xi download"))) return rc;
    return check_cuda(cudaStreamSynchronize(h->stream), "xi download");
}

int mdft_minimize_device(mdft_handle *h, double *d_xi, const mdft_minimize_opts *o, mdft_minimize_result *res) {
    if (!h || !d_xi || !o || !res) { set_error("null argument"); return MDFT_E_ARG; }
    int rc = check_min_opts(o);
    if (rc) return rc;
    if ((rc = lbfgs_alloc(h, o->m))) return rc;
    LbfgsState &L = h->lb;
    if ((rc = check_cuda(cudaMemcpyAsync(L.x.p, d_xi, L.n * 8, cudaMemcpyDeviceToDevice, h->stream), "xi copy"))) return rc;
    if ((rc = solve_phases(h, o, res))) return rc;
    if ((rc = check_cuda(cudaMemcpyAsync(d_xi, L.x.p, L.n * 8, cudaMemcpyDeviceToDevice, h->stream), "xi copy"))) return rc;
    return check_cuda(cudaStreamSynchronize(h->stream), "xi copy");
}

int mdft_guess_density_device(mdft_handle *h, double *d_xi) {
    if (!h || !d_xi) { set_error("null argument"); return MDFT_E_ARG; }
    const double vmax = (-std::log(kEpsDp) - (double)0.05f) * h->g.kT;
    k_guess<<<vec_grid(), 256, 0, h->stream>>>(h->vext.p, d_xi, vmax, (long long)h->g.N * h->g.no);
    h->launches += 1;
    return check_cuda(cudaGetLastError(), "guess launch");
}

}  // extern "C"

#include "warmstart.cuh"
#include "restart.cuh"

namespace {

// d_xi device; h->xi is overwritten (it holds the empty box afterwards)
int pressure_impl(mdft_handle *h, const double *d_xi, double ftot, double lj_tail, double *out) {
    const Grid &g = h->g;
    const size_t nf = (size_t)g.N * g.no;
    int rc;
    cudaStream_t st = h->stream;
    k_density_sum<<<vec_grid(), 256, 0, st>>>(d_xi, h->w.p, g.no, (long long)nf, g.rho0, h->vpart.p);
    h->launches += 2;
    k_finish_dot_max<<<1, 256, 0, st>>>(h->vpart.p, vec_grid(), h->vsc.p, 2);
    cudaMemcpyAsync(h->h_vsc + 2, h->vsc.p + 2, 8, cudaMemcpyDeviceToHost, st);
    if ((rc = check_cuda(cudaStreamSynchronize(st), "density integral"))) return rc;
    const double nwith = h->h_vsc[2] * g.dv;
    const double nwithout = g.n0 * (g.lx * g.ly * g.lz);
    const double deltaN = nwithout - nwith;
    // empty box: xi = 0, no charged-solute corrections (src/module_pressure_correction.f90:117-126)
    if ((rc = check_cuda(cudaMemsetAsync(h->xi.p, 0, nf * 8, st), "xi clear"))) return rc;
    const int saved = h->eval_prec;
    h->eval_prec = MDFT_PREC_FP64;  // the reported free energy is always an FP64 evaluation
    rc = run_pipeline(h, h->xi.p, nullptr, 1, 0);
    h->eval_prec = saved;
    if (rc) return rc;
    double fid, fext, fexc;
    if ((rc = finish_sums(h, &fid, &fext, &fexc))) return rc;
    double f0 = 0.0;
    f0 = f0 + fid + fext;
    f0 = f0 + fexc;
    f0 = f0 + (has_bridge(h) ? h->h_sums[6] : 0.0);  // the bridge term of the empty box
    const double pbulk = f0 / (g.lx * g.ly * g.lz);
    const double pmv = -deltaN / g.n0 * pbulk;
    out[0] = ftot + pmv + lj_tail;
    out[1] = pmv;
    out[2] = pbulk;
    out[3] = deltaN;
    return MDFT_OK;
}

}  // namespace

extern "C" {

int mdft_pressure_correction(mdft_handle *h, const double *xi, double ftot, double lj_tail, double *out) {
    if (!h || !xi || !out) { set_error("null argument"); return MDFT_E_ARG; }
    const size_t nf = (size_t)h->g.N * h->g.no;
    int rc = lbfgs_alloc(h, h->lb.m > 0 ? h->lb.m : 1);
    if (rc) return rc;
    if ((rc = check_cuda(cudaMemcpyAsync(h->lb.x.p, xi, nf * 8, cudaMemcpyHostToDevice, h->stream), "xi upload"))) return rc;
    return pressure_impl(h, h->lb.x.p, ftot, lj_tail, out);
}

int mdft_pressure_correction_device(mdft_handle *h, const double *d_xi, double ftot, double lj_tail, double *out) {
    if (!h || !d_xi || !out) { set_error("null argument"); return MDFT_E_ARG; }
    return pressure_impl(h, d_xi, ftot, lj_tail, out);
}

int mdft_solve(mdft_handle *h, int nsite, const double *q, const double *sig, const double *eps, const double *xyz, int nsv,
               const double *sq, const double *ssig, const double *seps, const double *sxyz, double rvdw, double eps_r,
               const mdft_minimize_opts *o, double *xi_out, double *out, mdft_minimize_result *res) {
    if (!h || !o || !out || !res || nsv <= 0 || !sq || !sxyz) { set_error("null argument"); return MDFT_E_ARG; }
    int rc = check_min_opts(o);
    if (rc) return rc;
    double lj = 0.0;
    auto t0 = std::chrono::steady_clock::now();
    auto lap = [&](const char *what) {
        if (!h->trace) return;
        cudaStreamSynchronize(h->stream);
        auto t1 = std::chrono::steady_clock::now();
        std::fprintf(stderr, "mdft-trace time %s %.3f ms\n", what, std::chrono::duration<double, std::milli>(t1 - t0).count());
        t0 = t1;
    };
    if ((rc = mdft_compute_vext(h, nsite, q, sig, eps, xyz, nsv, sq, ssig, seps, sxyz, rvdw, &lj))) return rc;
    lap("vext");
    // charged-solute corrections (src/module_energy_and_gradient.f90:191-204,281-344)
    double qnet = 0.0, quad = 0.0;
    for (int s = 0; s < nsite; ++s) qnet += q[s];
    for (int s = 0; s < nsv; ++s)
        quad += sq[s] * (sxyz[3 * s] * sxyz[3 * s] + sxyz[3 * s + 1] * sxyz[3 * s + 1] + sxyz[3 * s + 2] * sxyz[3 * s + 2]);
    double corr = 0.0;
    if (std::fabs(qnet) > 1e-7) {
        const Grid &g = h->g;
        double L = (g.lx == g.ly && g.ly == g.lz) ? g.lx : (g.lx + g.ly + g.lz) / 3.0;
        corr = -1971.01 * qnet * qnet / L * (1 - 1.0 / eps_r);
        corr = corr + (0.0 - quad * g.n0 * 2909.857 * qnet);
    }
    h->const_corr = corr;
    if ((rc = lbfgs_alloc(h, o->m))) return rc;
    LbfgsState &L = h->lb;
    const double vmax = (-std::log(kEpsDp) - (double)0.05f) * h->g.kT;
    const bool warm = h->warm != nullptr;
    if (warm) {
        if ((rc = warm_start_impl(h, nsite, q, sig, eps, xyz, nsv, ssig, seps, rvdw, L.x.p))) return rc;
        h->warm_starts += 1;
    } else {
        k_guess<<<vec_grid(), 256, 0, h->stream>>>(h->vext.p, L.x.p, vmax, L.n);
        h->launches += 1;
    }
    lap(warm ? "warm start" : "guess");
    if ((rc = solve_phases(h, o, res))) return rc;
    // a warm-started solve that stops without meeting its tests (line-search failure or the
    // iteration limit) is redone from the bulk guess; the result counts both solves' work
    if (warm && res->status != 0 && res->status != 1) {
        mdft_minimize_result r0 = *res;
        k_guess<<<vec_grid(), 256, 0, h->stream>>>(h->vext.p, L.x.p, vmax, L.n);
        h->launches += 1;
        if ((rc = solve_phases(h, o, res))) return rc;
        res->iterations += r0.iterations;
        res->evaluations += r0.evaluations;
        res->evaluations_mixed += r0.evaluations_mixed;
        h->warm_fallbacks += 1;
    }
    lap("minimise");
    double pc[4];
    if ((rc = pressure_impl(h, L.x.p, res->f, lj, pc))) return rc;
    lap("pressure");
    out[0] = pc[0];
    out[1] = res->f;
    out[2] = pc[1];
    out[3] = lj;
    out[4] = pc[2];
    out[5] = pc[3];
    if (xi_out) {
        if ((rc = check_cuda(cudaMemcpyAsync(xi_out, L.x.p, L.n * 8, cudaMemcpyDeviceToHost, h->stream), "xi download"))) return rc;
        if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "xi download"))) return rc;
    }
    return MDFT_OK;
}

}  // extern "C"

extern "C" int mdft_solve_batch(mdft_handle *const *handles, int nhandles, const mdft_solute *solutes, int nsolutes,
                                int nsv, const double *sq, const double *ssig, const double *seps, const double *sxyz, double rvdw,
                                double eps_r, const mdft_minimize_opts *opts, double *out, mdft_minimize_result *res, int *rc) {
    if (!handles || nhandles <= 0 || (nsolutes > 0 && !solutes) || !opts || (nsolutes > 0 && (!out || !res))) {
        set_error("null argument or no handle");
        return MDFT_E_ARG;
    }
    for (int k = 0; k < nhandles; ++k)
        if (!handles[k]) { set_error("null handle %d", k); return MDFT_E_ARG; }
    for (int i = 0; i < nsolutes; ++i)
        if (solutes[i].handle < -1 || solutes[i].handle >= nhandles) {
            set_error("solute %d: handle %d out of range", i, solutes[i].handle);
            return MDFT_E_ARG;
        }
    std::vector<int> codes(nsolutes, MDFT_OK);
    std::vector<std::string> msgs(nsolutes);
    std::atomic<int> next_free{0};
    auto worker = [&](int k) {
        mdft_handle *h = handles[k];
        if (cudaSetDevice(h->device) != cudaSuccess) {
            for (int i = 0; i < nsolutes; ++i)
                if (solutes[i].handle == k) { codes[i] = MDFT_E_CUDA; msgs[i] = "cudaSetDevice failed"; }
            return;
        }
        auto run = [&](int i) {
            const mdft_solute &u = solutes[i];
            codes[i] = mdft_solve(h, u.nsite, u.q, u.sig, u.eps, u.xyz, nsv, sq, ssig, seps, sxyz, rvdw, eps_r, opts, u.xi_out,
                                  out + 6 * (size_t)i, res + i);
            if (codes[i]) msgs[i] = last_error();
        };
        for (int i = 0; i < nsolutes; ++i)
            if (solutes[i].handle == k) run(i);
        // unassigned solutes, in order, to whichever handle is free
        for (;;) {
            int i = next_free.fetch_add(1);
            while (i < nsolutes && solutes[i].handle != -1) i = next_free.fetch_add(1);
            if (i >= nsolutes) break;
            run(i);
        }
    };
    if (nhandles == 1) {
        worker(0);
    } else {
        std::vector<std::thread> pool;
        for (int k = 0; k < nhandles; ++k) pool.emplace_back(worker, k);
        for (auto &t : pool) t.join();
    }
    int first = MDFT_OK;
    for (int i = 0; i < nsolutes; ++i) {
        if (rc) rc[i] = codes[i];
        if (codes[i] && first == MDFT_OK) {
            first = codes[i];
            set_error("solute %d: %s", i, msgs[i].c_str());
        }
    }
    return first;
}

