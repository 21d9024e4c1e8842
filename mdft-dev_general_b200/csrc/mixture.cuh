// Multi-species solvent: energy_and_gradient with nspec > 1 species
// (src/module_energy_and_gradient.f90:86-217, excess_energy => energy_cproj_mrso_mixture by
// src/module_init_simu.f90:67-71).
//
// A mixture binds nspec species handles on one grid, angular order, symmetry order,
// temperature and device, all FP64.  Each handle holds one species: its n0 (the pure
// fluid's times the mole fraction, src/module_solvent.f90:221-222), its c(k) table and its
// vext.  One evaluation:
//   * species s, on its handle's stream: the S1 projection of rho0_s (xi_s^2 - 1) into the
//     handle's planes and their forward FFT (src/module_energy_cproj_mrso_mixture.f90:283-344);
//   * species s2, on its stream once every forward FFT is done:
//     gamma_{s2} = sum_s OZ_{c(s2)}(drho_s) by one launch of k_oz2<double, 1> over every
//     source species' planes (:491-721), the inverse FFT of gamma_{s2} (:746-779), then the gather of species s2 with its ideal and external terms
//     and the excess prefactor times x_{s2} (:788-809,
//     src/module_energy_ideal_and_external.f90:46-72).
// The mixture owns the gamma planes (nspec x np x N complex) and the OZ term tables of the
// multi-species rotation form (build_oz_tables with mix = true).
#pragma once

#include <vector>

struct mdft_mixture {
    std::vector<mdft_handle *> sp;
    std::vector<double> x;
    int device = 0;
    DevBuf<double2> gam;  // [nspec][np][N]
    DevBuf<int> oz_ints;
    DevBuf<double> oz_dbls;
    int oz_grid = 0, oz_warps = 0;
    size_t oz_smem = 0;
    OzMix srcs{};  // every species' planes
    DevBuf<double> xi, df;  // staging of the host entry point and the minimiser's gradient, [nspec][N][no]
    std::vector<cudaEvent_t> ev_fwd, ev_done;  // per species: forward FFTs done, gather done
    cudaEvent_t ev_start = nullptr;            // species 0's stream: the point is ready
};

namespace {

int mixture_check(const mdft_mixture *m) {
    if (!m) { set_error("null mixture"); return MDFT_E_ARG; }
    return check_cuda(cudaSetDevice(m->device), "cudaSetDevice");
}

// Launches one evaluation; leaves each species' sums on its handle (finish_sums reads them).
// The point may come from work on species 0's stream (the minimiser's trial point): every
// species stream starts after it, and species 0's stream continues after every gather.
// dvec (may be null): the gathers also form df.dvec, as in single-species evaluations.
int mixture_launch(mdft_mixture *m, const double *d_xi, double *d_df, const double *dvec = nullptr) {
    const int ns = (int)m->sp.size();
    const Grid &g = m->sp[0]->g;
    const size_t n = (size_t)g.N * g.no;
    int rc;
    if ((rc = check_cuda(cudaEventRecord(m->ev_start, m->sp[0]->stream), "event record"))) return rc;
    for (int s = 1; s < ns; ++s)
        if ((rc = check_cuda(cudaStreamWaitEvent(m->sp[s]->stream, m->ev_start, 0), "stream wait"))) return rc;
    for (int s = 0; s < ns; ++s) {
        mdft_handle *h = m->sp[s];
        const void *tw[3] = {h->tw64[0].p, h->tw64[1].p, h->tw64[2].p};
        const AngularArgs aa{g.N, g.no, g.np, h->g.rho0};
        launch_project_cc<double>(h, d_xi + s * n, h->A.p, h->planes.p, aa);
        if ((rc = check_cuda(cudaGetLastError(), "project launch"))) return rc;
        if ((rc = launch_fft_t<double>(h, h->planes.p, tw, +1))) return rc;
        if ((rc = check_cuda(cudaEventRecord(m->ev_fwd[s], h->stream), "event record"))) return rc;
        h->launches += 1;
    }
    for (int s2 = 0; s2 < ns; ++s2) {
        mdft_handle *h = m->sp[s2];
        double2 *gam = m->gam.p + (size_t)s2 * g.np * g.N;
        for (int s = 0; s < ns; ++s)
            if ((rc = check_cuda(cudaStreamWaitEvent(h->stream, m->ev_fwd[s], 0), "stream wait"))) return rc;
        Oz2Args oz = h->oz;  // this species' c table: nq, dq
        oz.quirks = 1;
        k_oz2<double, 1><<<m->oz_grid, 32 * m->oz_warps, m->oz_smem, h->stream>>>(nullptr, h->ctab.p, m->oz_ints.p, m->oz_dbls.p,
                                                                                 oz, gam, m->srcs);
        if ((rc = check_cuda(cudaGetLastError(), "oz launch"))) return rc;
        const void *tw[3] = {h->tw64[0].p, h->tw64[1].p, h->tw64[2].p};
        if ((rc = launch_fft_t<double>(h, gam, tw, -1))) return rc;
        const double *dv = dvec ? dvec + s2 * n : nullptr;
        const GatherArgs ga = gather_args(h, d_df ? 1 : 0, 1, dv, m->x[s2]);
        const bool tma = h->gt_ncol64 > 0 && ((uintptr_t)(d_xi + s2 * n) & 15u) == 0 && ((uintptr_t)dv & 15u) == 0;
        const long long rows = launch_gather_cc<double>(h, gam, h->B.p, d_xi + s2 * n, d_df ? d_df + s2 * n : nullptr, ga,
                                                        tma ? h->gt_ncol64 : 0);
        if ((rc = check_cuda(cudaGetLastError(), "gather launch"))) return rc;
        k_reduce_sums<<<1, 256, 0, h->stream>>>(h->partial.p, rows, h->sums.p);
        if ((rc = check_cuda(cudaGetLastError(), "reduce launch"))) return rc;
        h->launches += 3;
        if ((rc = check_cuda(cudaEventRecord(m->ev_done[s2], h->stream), "event record"))) return rc;
    }
    for (int s = 1; s < ns; ++s)
        if ((rc = check_cuda(cudaStreamWaitEvent(m->sp[0]->stream, m->ev_done[s], 0), "stream wait"))) return rc;
    return MDFT_OK;
}

// Reads every species' sums (synchronising its stream): F, and with the gradient's
// reductions summed over species {df.dvec, max|df|, sum w df dv}; fscale the terms' sizes.
int mixture_finish(mdft_mixture *m, double *f, double *terms, double *gd, double *gmax, double *guni, double *fscale) {
    double fid = 0.0, fext = 0.0, sexc = 0.0, gdv = 0.0, gmx = 0.0, gun = 0.0;
    int first = 0;
    for (mdft_handle *h : m->sp) {
        double a = 0, b = 0, c = 0;
        const int r = finish_sums(h, &a, &b, &c);  // synchronises the species' stream
        if (r && !first) first = r;
        // src/module_energy_ideal_and_external.f90:46-72 sums F_id and F_ext over species in
        // order; F_exc = 0.5 dv sum_{s2} (...) (src/module_energy_cproj_mrso_mixture.f90:788-809)
        fid += a;
        fext += b;
        sexc += h->h_sums[2];
        gdv += h->h_sums[3];
        gmx = std::max(gmx, h->h_sums[4]);
        gun += h->h_sums[5];
    }
    if (first) return first;
    const mdft_handle *h0 = m->sp[0];
    const double fexc = sexc * 0.5 * h0->g.dv;
    *f = combine(h0, fid, fext, fexc);
    if (terms) {
        terms[0] = fid;
        terms[1] = fext;
        terms[2] = fexc;
        terms[3] = h0->const_corr;
    }
    if (gd) *gd = gdv;
    if (gmax) *gmax = gmx;
    if (guni) *guni = gun * h0->g.dv;
    if (fscale) *fscale = std::fabs(fid) + std::fabs(fext) + std::fabs(fexc) + std::fabs(h0->const_corr);
    if (!std::isfinite(gdv) || !std::isfinite(gmx) || !std::isfinite(gun)) {
        set_error("non-finite gradient");
        return MDFT_E_NUMERIC;
    }
    return MDFT_OK;
}

long long mixture_len(const mdft_mixture *m) { return (long long)m->sp.size() * m->sp[0]->g.N * m->sp[0]->g.no; }

double *mixture_grad(mdft_mixture *m) {
    const size_t n = (size_t)mixture_len(m);
    if (!m->df.p && alloc_check(m->df.alloc(n), "mixture df", n * 8)) return nullptr;
    return m->df.p;
}

int mixture_eval_launch(mdft_mixture *m, const double *x, double *g, const double *dvec) {
    const int rc = mixture_launch(m, x, g, dvec);
    if (rc)
        for (mdft_handle *h : m->sp) cudaStreamSynchronize(h->stream);
    return rc;
}

int mixture_eval_finish(mdft_mixture *m, double *f, double *gd, double *gmax, double *guni, double *fscale) {
    return mixture_finish(m, f, nullptr, gd, gmax, guni, fscale);
}

}  // namespace

extern "C" {

int mdft_mixture_create(mdft_handle *const *species, int nspec, const double *mole_fraction, mdft_mixture **out) {
    if (!species || !mole_fraction || !out) { set_error("null argument"); return MDFT_E_ARG; }
    *out = nullptr;
    if (nspec < 2 || nspec > kOzMaxSpecies) {
        set_error(nspec < 2 ? "a mixture needs at least two species (one species uses the handle itself)"
                            : "a mixture takes at most %d species", kOzMaxSpecies);
        return MDFT_E_ARG;
    }
    const mdft_handle *h0 = species[0];
    if (!h0) { set_error("null species handle"); return MDFT_E_ARG; }
    const Grid &g0 = h0->g;
    double xsum = 0.0;
    for (int s = 0; s < nspec; ++s) {
        const mdft_handle *h = species[s];
        if (!h) { set_error("null species handle"); return MDFT_E_ARG; }
        for (int t = 0; t < s; ++t)
            if (species[t] == h) { set_error("species %d and %d are the same handle", t, s); return MDFT_E_ARG; }
        const Grid &g = h->g;
        if (g.nx != g0.nx || g.ny != g0.ny || g.nz != g0.nz || g.lx != g0.lx || g.ly != g0.ly || g.lz != g0.lz ||
            g.mmax != g0.mmax || g.mrso != g0.mrso || g.kT != g0.kT || h->device != h0->device) {
            set_error("species %d differs from species 0 in grid, angular order, symmetry order, temperature or device", s);
            return MDFT_E_ARG;
        }
        if (h->precision != MDFT_PREC_FP64) { set_error("mixtures are evaluated in FP64: species %d is not", s); return MDFT_E_ARG; }
        if (has_bridge(h)) { set_error("species %d has a bridge term; the reference's bridges take one species", s); return MDFT_E_ARG; }
        if (h->ct.ncoef != h0->ct.ncoef) { set_error("species %d has another c(k) coefficient count", s); return MDFT_E_ARG; }
        const double x = mole_fraction[s];
        if (!(x > 0.0 && x <= 1.0)) { set_error("mole fraction of species %d is %g, outside (0, 1]", s, x); return MDFT_E_ARG; }
        xsum += x;
    }
    // src/module_solvent.f90:476-480: the fractions must sum to exactly one
    if (xsum != 1.0) { set_error("mole fractions sum to %.17g, not 1", xsum); return MDFT_E_ARG; }
    std::unique_ptr<mdft_mixture> m(new mdft_mixture());
    m->sp.assign(species, species + nspec);
    m->x.assign(mole_fraction, mole_fraction + nspec);
    m->device = h0->device;
    int rc;
    if ((rc = mixture_check(m.get()))) return rc;
    OzTables tb;
    if (!build_oz_tables(g0, h0->ct, tb, true)) { set_error("OZ term tables exceed their index encoding"); return MDFT_E_ARG; }
    if ((int)tb.ints.size() != h0->oz.n_ints || (int)tb.dbls.size() != h0->oz.n_dbls) {
        set_error("multi-species OZ tables differ in layout from the species tables");
        return MDFT_E_STATE;
    }
    const size_t planes = (size_t)nspec * g0.np * g0.N;
    if ((rc = alloc_check(m->gam.alloc(planes), "mixture gamma planes", planes * sizeof(double2)))) return rc;
    if ((rc = alloc_check(m->oz_ints.alloc(tb.ints.size()), "OZ tables", tb.ints.size() * 4))) return rc;
    if ((rc = alloc_check(m->oz_dbls.alloc(std::max<size_t>(1, tb.dbls.size())), "OZ tables", tb.dbls.size() * 8))) return rc;
    if ((rc = check_cuda(cudaMemcpy(m->oz_ints.p, tb.ints.data(), tb.ints.size() * 4, cudaMemcpyHostToDevice), "OZ tables"))) return rc;
    if (!tb.dbls.empty() &&
        (rc = check_cuda(cudaMemcpy(m->oz_dbls.p, tb.dbls.data(), tb.dbls.size() * 8, cudaMemcpyHostToDevice), "OZ tables")))
        return rc;
    int maxsmem = 0;
    if ((rc = check_cuda(cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, m->device), "device attribute")))
        return rc;
    if ((rc = allow_smem((const void *)k_oz2<double, 1>, maxsmem))) return rc;
    // warps per CTA: as many of 8 as fit with the two gamma accumulators per warp
    m->oz_warps = 8;
    while (m->oz_warps > 1 && oz2_smem_bytes<double>(h0->oz, m->oz_warps, 1) > (size_t)maxsmem) m->oz_warps /= 2;
    m->oz_smem = oz2_smem_bytes<double>(h0->oz, m->oz_warps, 1);
    if (m->oz_smem > (size_t)maxsmem) { set_error("multi-species OZ tile does not fit in shared memory"); return MDFT_E_ARG; }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_oz2<double, 1>, 32 * m->oz_warps, m->oz_smem);
    const long long nk = (long long)g0.nx * g0.ny * (g0.nz / 2 + 1);
    const long long groups = (nk + m->oz_warps - 1) / m->oz_warps;
    m->oz_grid = (int)std::min<long long>(groups, (long long)std::max(1, per_sm) * h0->nsm);
    m->srcs.ns = nspec;
    for (int s = 0; s < nspec; ++s) m->srcs.p[s] = m->sp[s]->planes.p;
    m->ev_fwd.assign(nspec, nullptr);
    m->ev_done.assign(nspec, nullptr);
    auto drop_events = [&]() {
        for (cudaEvent_t e : m->ev_fwd)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : m->ev_done)
            if (e) cudaEventDestroy(e);
        if (m->ev_start) cudaEventDestroy(m->ev_start);
    };
    for (int s = 0; s < nspec; ++s)
        if ((rc = check_cuda(cudaEventCreateWithFlags(&m->ev_fwd[s], cudaEventDisableTiming), "event create")) ||
            (rc = check_cuda(cudaEventCreateWithFlags(&m->ev_done[s], cudaEventDisableTiming), "event create"))) {
            drop_events();
            return rc;
        }
    if ((rc = check_cuda(cudaEventCreateWithFlags(&m->ev_start, cudaEventDisableTiming), "event create"))) {
        drop_events();
        return rc;
    }
    *out = m.release();
    return MDFT_OK;
}

int mdft_mixture_destroy(mdft_mixture *m) {
    if (!m) return MDFT_OK;
    cudaSetDevice(m->device);
    for (mdft_handle *h : m->sp) cudaStreamSynchronize(h->stream);
    for (cudaEvent_t e : m->ev_fwd)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : m->ev_done)
        if (e) cudaEventDestroy(e);
    if (m->ev_start) cudaEventDestroy(m->ev_start);
    m->gam.free(); m->oz_ints.free(); m->oz_dbls.free(); m->xi.free(); m->df.free();
    delete m;
    return MDFT_OK;
}

int mdft_mixture_energy_and_gradient_device(mdft_mixture *m, const double *d_xi, double *d_df, double *f, double *terms) {
    int rc = mixture_check(m);
    if (rc) return rc;
    if (!d_xi || !f) { set_error("null argument"); return MDFT_E_ARG; }
    for (const mdft_handle *h : m->sp)
        if (has_bridge(h)) { set_error("a species handle has a bridge term; the reference's bridges take one species"); return MDFT_E_STATE; }
    if ((rc = mixture_launch(m, d_xi, d_df))) {
        for (mdft_handle *h : m->sp) cudaStreamSynchronize(h->stream);
        return rc;
    }
    return mixture_finish(m, f, terms, nullptr, nullptr, nullptr, nullptr);
}

int mdft_mixture_energy_and_gradient(mdft_mixture *m, const double *xi, double *f, double *df, double *terms) {
    int rc = mixture_check(m);
    if (rc) return rc;
    if (!xi || !f) { set_error("null argument"); return MDFT_E_ARG; }
    const Grid &g = m->sp[0]->g;
    const size_t n = (size_t)m->sp.size() * g.N * g.no;
    if (!m->xi.p && (rc = alloc_check(m->xi.alloc(n), "mixture xi", n * 8))) return rc;
    if (df && !m->df.p && (rc = alloc_check(m->df.alloc(n), "mixture df", n * 8))) return rc;
    cudaStream_t st = m->sp[0]->stream;
    if ((rc = check_cuda(cudaMemcpyAsync(m->xi.p, xi, n * 8, cudaMemcpyHostToDevice, st), "xi upload"))) return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(st), "xi upload"))) return rc;
    if ((rc = mdft_mixture_energy_and_gradient_device(m, m->xi.p, df ? m->df.p : nullptr, f, terms))) return rc;
    if (df) {
        if ((rc = check_cuda(cudaMemcpyAsync(df, m->df.p, n * 8, cudaMemcpyDeviceToHost, st), "df download"))) return rc;
        if ((rc = check_cuda(cudaStreamSynchronize(st), "df download"))) return rc;
    }
    return MDFT_OK;
}

// energy_minimization over every species' xi at once (the reference's L-BFGS on the vector of
// all species): the FP64 minimiser of mdft_minimize with the mixture's evaluations.
int mdft_mixture_minimize(mdft_mixture *m, double *xi, const mdft_minimize_opts *o, mdft_minimize_result *res) {
    int rc = mixture_check(m);
    if (rc) return rc;
    if (!xi || !o || !res) { set_error("null argument"); return MDFT_E_ARG; }
    if ((rc = check_min_opts(o))) return rc;
    if (o->precision != MDFT_PREC_FP64) { set_error("mixtures are minimised in FP64"); return MDFT_E_ARG; }
    for (const mdft_handle *h : m->sp)
        if (has_bridge(h)) { set_error("a species handle has a bridge term; the reference's bridges take one species"); return MDFT_E_STATE; }
    mdft_handle *h0 = m->sp[0];
    struct Bind {  // species 0's handle runs the minimiser on the mixture while this lives
        mdft_handle *h;
        Bind(mdft_handle *hh, mdft_mixture *mm) : h(hh) { h->mix = mm; }
        ~Bind() { h->mix = nullptr; }
    } bind(h0, m);
    if (!mixture_grad(m)) return MDFT_E_NOMEM;
    if ((rc = lbfgs_alloc(h0, o->m))) return rc;
    LbfgsState &L = h0->lb;
    if ((rc = check_cuda(cudaMemcpyAsync(L.x.p, xi, L.n * 8, cudaMemcpyHostToDevice, h0->stream), "xi upload"))) return rc;
    if ((rc = solve_phases(h0, o, res))) {
        for (mdft_handle *h : m->sp) cudaStreamSynchronize(h->stream);
        return rc;
    }
    if ((rc = check_cuda(cudaMemcpyAsync(xi, L.x.p, L.n * 8, cudaMemcpyDeviceToHost, h0->stream), "xi download"))) return rc;
    return check_cuda(cudaStreamSynchronize(h0->stream), "xi download");
}

}  // extern "C"
