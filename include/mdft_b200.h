/*
 * mdft_b200.h -- C-ABI of the B200 MDFT energy-and-gradient engine.
 *
 * The engine replaces, behind plain pointers and sizes, the hot path of the
 * Fortran program dborgis/mdft-dev_general:
 *
 *   subroutine energy_and_gradient(f, df)      src/module_energy_and_gradient.f90:36
 *   procedure pointer excess_energy(ff, df)    src/module_proc_ptrs.f90:3-21
 *
 * and the set-up and callers those need (vext, guess_density, the L-BFGS
 * loop of energy_minimization, pressure_correction), with the functionals
 * beside the excess term on the same path: the bridges of energy_bridge
 * (src/module_energy_and_gradient.f90:246-275) and the multi-species excess
 * energy_cproj_mrso_mixture.  A Fortran host binds
 * these entry points with ISO_C_BINDING (one bind(C) interface per entry point,
 * with the structs below as bind(C) derived types).
 *
 * Layout: every per-orientation field (xi, vext, df) is the reference's
 * Fortran array (no, nx, ny, nz) with io fastest, i.e. the C index
 * ((iz*ny + iy)*nx + ix)*no + io.  Units follow the reference: Angstrom,
 * kJ/mol, molecules/Angstrom^3.  `df` is dF/dxi divided by the volume
 * element dv, exactly as the reference returns it.
 *
 * Errors: every entry point returns 0 on success and a negative MDFT_E_*
 * code on failure; mdft_last_error() gives the message of the last failure
 * on the calling thread.  Nothing aborts the process.
 *
 * Threading: one host thread per handle; each handle owns one CUDA stream
 * and all of its device memory.  Handles are independent.
 */
#ifndef MDFT_B200_H
#define MDFT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDFT_OK 0
#define MDFT_E_ARG (-1)     /* invalid argument or size                        */
#define MDFT_E_IO (-2)      /* c(k) file missing or malformed                   */
#define MDFT_E_CUDA (-3)    /* CUDA runtime error (message has the CUDA string) */
#define MDFT_E_NUMERIC (-4) /* NaN/Inf in inputs or outputs                     */
#define MDFT_E_STATE (-5)   /* call order (e.g. no vext yet)                    */
#define MDFT_E_NOMEM (-6)   /* device allocation failed                         */

/* Arithmetic of the excess-term pipeline. */
#define MDFT_PREC_FP64 0  /* every stage in FP64 (parity path)                          */
#define MDFT_PREC_MIXED 1 /* FP32 projections, FFTs, OZ and angular transforms, FP64 sums */

typedef struct mdft_handle mdft_handle;

/* System description: grid (src/module_grid.f90:51-212), solvent and thermo
 * (src/module_solvent.f90:209-226, src/module_thermo.f90:56-66), c(k) file
 * (src/module_read_c_luc.f90:6-124). */
typedef struct mdft_desc {
    int nx, ny, nz;         /* grid nodes (boxnod); even                          */
    double lx, ly, lz;      /* box lengths (boxlen), Angstrom                     */
    int mmax;               /* angular order, 0..5                               */
    int mrso;               /* molrotsymorder of the solvent (2 for water)       */
    double temperature;     /* K                                                 */
    double n0;              /* bulk number density, molecules/Angstrom^3         */
    const char *ck_path;    /* c^{mn}_{mu nu khi}(q) table in Luc's file format  */
    int precision;          /* MDFT_PREC_*                                       */
    int device;             /* CUDA device ordinal                               */
} mdft_desc;

/* Sizes derived from the description (filled by mdft_get_sizes). */
typedef struct mdft_sizes {
    int ntheta, nphi, npsi; /* angular grid                                       */
    int no;                 /* orientations  = ntheta*nphi*npsi                  */
    int np;                 /* projections   = sum_m (2m+1)(m/mrso+1)            */
    int ncoef;              /* c(k) coefficients used per k                      */
    int nq;                 /* c(k) rows used                                    */
    double dv;              /* volume element, Angstrom^3                        */
    double rho0;            /* n0 / (8 pi^2 / mrso)                              */
    double kT;              /* kJ/mol                                            */
    double dq;              /* c(k) abscissa step                                */
} mdft_sizes;

/* Create / destroy: replaces init_simu's grid, thermo, c(k) and FFT set-up
 * (src/module_init_simu.f90:24-36, src/module_energy_cproj_mrso.f90:151-267,362-431). */
int mdft_create(const mdft_desc *desc, mdft_handle **out);
int mdft_destroy(mdft_handle *h);
const char *mdft_last_error(void);
int mdft_get_sizes(const mdft_handle *h, mdft_sizes *out);

/* Stream of the handle (a cudaStream_t); every device call runs on it. */
int mdft_get_stream(const mdft_handle *h, void **stream);

/* Quadrature weights w(io) (src/module_grid.f90:116-139), host buffer of no doubles. */
int mdft_get_weights(const mdft_handle *h, double *w);

/* External potential vext(no,nx,ny,nz), host buffer: replaces the module state
 * solvent(1)%vext that energy_and_gradient reads (src/module_vext.f90:14-115). */
int mdft_set_vext(mdft_handle *h, const double *vext_host);
int mdft_get_vext(const mdft_handle *h, double *vext_host);

/* Constant added to F: the charged-solute corrections of
 * src/module_energy_and_gradient.f90:191-204,281-344 (0 for a neutral solute). */
int mdft_set_constant_correction(mdft_handle *h, double c);

/* energy_and_gradient(f, df): src/module_energy_and_gradient.f90:36-240.
 * xi, df: host arrays of no*nx*ny*nz doubles; df may be NULL (energy only).
 * terms (may be NULL) receives {F_id, F_ext, F_exc, constant correction}. */
int mdft_energy_and_gradient(mdft_handle *h, const double *xi, double *f, double *df, double *terms);

/* Same with device pointers (on the handle's stream); d_df may be NULL. */
int mdft_energy_and_gradient_device(mdft_handle *h, const double *d_xi, double *d_df, double *f, double *terms);

/* excess_energy(ff, df): the procedure-pointer seam bound to energy_cproj_mrso
 * (src/module_proc_ptrs.f90:3-21, src/module_energy_cproj_mrso.f90:61-782).
 * df (may be NULL) is ACCUMULATED into, as the reference does. */
int mdft_excess_energy(mdft_handle *h, const double *xi, double *fexc, double *df);

/* External potential from a solute (src/module_vext.f90:14-115,600-669):
 * Lennard-Jones (src/module_lennardjones.f90:9-226) plus the Poisson-solved
 * electrostatics (src/module_fastpoissonsolver.f90:121-288,
 * src/module_solvent.f90:367-438), clipped at qfact/2.  Solute sites are used
 * as given (callers apply mv_solute_to_center first, src/module_solute.f90:146-187).
 * The result becomes the handle's vext; lj_tail receives LJ_energy_correction. */
int mdft_compute_vext(mdft_handle *h, int nsite, const double *q, const double *sig, const double *eps,
                      const double *xyz, int nsolvsite, const double *sq, const double *ssig,
                      const double *seps, const double *sxyz, double rvdw, double *lj_tail);

/* guess_density (src/module_density.f90:267-284) into a host xi. */
int mdft_guess_density(const mdft_handle *h, double *xi);

/* Minimiser settings and result for mdft_minimize. */
typedef struct mdft_minimize_opts {
    int m;           /* L-BFGS history (lbfgsb%m)                                 */
    double pgtol;    /* stop when max|df| <= pgtol (lbfgsb%pgtol)                  */
    double ftol_abs; /* stop when f_old - f <= ftol_abs (factr*epsmch)             */
    int itermax;     /* maximum iterations (maximum_iteration_nbr)                 */
    int precision;   /* MDFT_PREC_* of the evaluations used by this solve          */
    double pgtol_mixed; /* MIXED: stop the FP32 phase at max|df| <= this (<= 0: pgtol) */
    int polish;      /* MIXED: 1 = continue with FP64 evaluations until pgtol holds;
                        0 = one FP64 evaluation at the FP32 phase's result          */
    double guni_tol; /* > 0: the pgtol test also needs |sum_{r,io} w(io) df dv| <= guni_tol,
                        the gradient along a uniform change of xi (kJ/mol); <= 0: off.
                        Not in the reference: the solvation free energy's error at a
                        stopping point follows this sum (about half of it, in kJ/mol),
                        which converges more slowly than max|df| for small solutes     */
} mdft_minimize_opts;

typedef struct mdft_minimize_result {
    double f;        /* functional at the returned xi                             */
    double pgnorm;   /* max|df| at the returned xi                                */
    int iterations;  /* L-BFGS iterations                                        */
    int evaluations; /* energy_and_gradient calls                                 */
    int status;      /* 0 pgtol, 1 f-reduction, 2 line-search failure, 3 itermax   */
    int evaluations_mixed; /* of which FP32-pipeline evaluations (MDFT_PREC_MIXED)   */
    double guni;     /* sum_{r,io} w(io) df dv at the returned xi (kJ/mol)          */
} mdft_minimize_result;

/* minimization_using_lbfgs (src/energy_minimization.f90:232-290) with the
 * unconstrained L-BFGS-B of src/module_lbfgs_nocedal_mdft.f90:136-534, run on
 * the device: xi is read from and written to the host buffer.  With
 * MDFT_PREC_MIXED the iterations use FP32 projections/FFTs/OZ until the
 * stopping test (pgtol_mixed) holds or a line search fails, then either
 * continue with FP64 evaluations, keeping the L-BFGS history, until pgtol
 * holds in FP64 (polish = 1) or end with one FP64 evaluation (polish = 0);
 * f and pgnorm are always FP64 values. */
int mdft_minimize(mdft_handle *h, double *xi, const mdft_minimize_opts *opts, mdft_minimize_result *res);

/* Device-pointer variants (on the handle's stream): d_xi is a device array of
 * no*nx*ny*nz doubles, read and overwritten. */
int mdft_guess_density_device(mdft_handle *h, double *d_xi);
int mdft_minimize_device(mdft_handle *h, double *d_xi, const mdft_minimize_opts *opts, mdft_minimize_result *res);

/* pressure_correction (src/module_pressure_correction.f90:7-156):
 * out = {dG_SFE, PMV correction, P_bulk, deltaN} for the density xi (host)
 * whose functional value is ftot; lj_tail as returned by mdft_compute_vext. */
int mdft_pressure_correction(mdft_handle *h, const double *xi, double ftot, double lj_tail, double *out);

/* One solute, end to end, as main.f90 runs it (src/main.f90:20-40): init_vext,
 * guess_density, the L-BFGS minimisation and pressure_correction.  Solute and
 * solvent sites are host arrays as in mdft_compute_vext; charged solutes get
 * the constant corrections of src/module_energy_and_gradient.f90:281-344 from
 * eps_r and the solvent quadrupole trace.  xi_out (host, may be NULL) receives
 * the converged density; out = {dG_SFE, F at the minimum, PMV correction,
 * LJ tail, P_bulk, deltaN}. */
int mdft_solve(mdft_handle *h, int nsite, const double *q, const double *sig, const double *eps, const double *xyz,
               int nsolvsite, const double *sq, const double *ssig, const double *seps, const double *sxyz, double rvdw,
               double eps_r, const mdft_minimize_opts *opts, double *xi_out, double *out, mdft_minimize_result *res);

int mdft_pressure_correction_device(mdft_handle *h, const double *d_xi, double ftot, double lj_tail, double *out);

/* One solute of a batch: sites as in mdft_solve; handle = index into the batch's handle
 * array to solve it on, or -1 for the next free handle; xi_out: host buffer for its
 * converged density (may be NULL). */
typedef struct mdft_solute {
    int nsite;
    const double *q, *sig, *eps, *xyz;
    int handle;
    double *xi_out;
} mdft_solute;

/* A batch of independent solves (no counterpart in the reference, which solves one solute
 * per run).  Each handle gets one host worker thread that runs mdft_solve for the solutes
 * assigned to it and then for unassigned ones (handle -1) as they come free, so solves on
 * different handles -- each with its own device buffers and stream -- run concurrently on
 * the GPU.  Handles may differ in grid and mmax (a solute with handle -1 must fit every
 * handle).  out: 6 doubles per solute as mdft_solve's; res: one result per solute; rc (may
 * be NULL): each solute's mdft_solve return code.  Returns MDFT_OK when every solve succeeded,
 * else the first failing code with its message in mdft_last_error.  The handles must not be
 * used by other threads during the call. */
int mdft_solve_batch(mdft_handle *const *handles, int nhandles, const mdft_solute *solutes, int nsolutes, int nsolvsite,
                     const double *sq, const double *ssig, const double *seps, const double *sxyz, double rvdw, double eps_r,
                     const mdft_minimize_opts *opts, double *out, mdft_minimize_result *res, int *rc);

/* Per-stage device time (ms) of the last evaluations, when timing is on:
 * stage order {project, fft_forward, oz, fft_inverse, gather}; count = calls. */
int mdft_set_timing(mdft_handle *h, int on);
int mdft_get_stage_times(const mdft_handle *h, double *ms5, int *count);

/* Ideal + external term without any device allocation (no counterpart in the
 * reference).  For callers that may not allocate GPU memory: a Fortran or C host that
 * embeds the engine inside a program whose own pool owns every device allocation, or a
 * time-critical loop that must not change the device's memory footprint.  Inputs and
 * outputs stay the caller's device buffers: xi and vext (npoints*no doubles, io
 * fastest), w (no doubles), df (may be NULL; receives the id+ext gradient, divided by dv
 * like the reference's df), out (2 doubles: F_id, F_ext).  Work is queued on `stream`
 * (a cudaStream_t, NULL for the default stream); nothing is synchronised.  The
 * per-block partial sums go to a fixed 256 KB array inside the library, one per GPU that
 * loads it, held until the process exits, so npoints is limited to 1,048,576 (larger
 * sizes return MDFT_E_ARG with a message).  The first call on a device looks up that
 * array's device address; make that first call before any stream capture.  After a
 * cudaDeviceReset the next call on that device looks the address up again (the array
 * may move with the new context), so that call too belongs before any capture.  Every call
 * shares the array: calls that overlap on the GPU race and must be serialised by the
 * caller.  Same arithmetic as src/module_energy_ideal_and_external.f90:46-73. */
int mdft_ideal_external_noalloc(const double *d_xi, const double *d_vext, const double *d_w, int no, long long npoints,
                                double kT, double rho0, double dv, double *d_df, double *d_out, void *stream);

/* Number of kernels this handle has launched since creation. */
int mdft_get_launch_count(const mdft_handle *h, long long *count);

/* Error-path test switch (no counterpart in the reference): with on != 0, this handle's
 * bulk-copy and tensor-core gather kernels behave as if their first mbarrier wait had run
 * out -- they set the device error flag and return before issuing any copy or allocating
 * tensor memory -- so every evaluation fails with MDFT_E_CUDA and the bounded-wait message.
 * Off again, the handle evaluates as before. */
int mdft_set_wait_failure(mdft_handle *h, int on);

/* The kernel forms of this handle's FP32 evaluations (no counterpart in the reference):
 * forms[4] = {projection: 0 register / 1 bulk-copy ring, gather: 0 register / 1 ring, OZ:
 * 0 complex rotations / 1 factored rotations, 1 when the autotuner chose them}.  The
 * autotuner times two configurations on the handle's first FP32 phase (the default forms,
 * and the alternatives) stage by stage and keeps the faster form of each stage; ms (may be
 * NULL) receives 6 doubles {project, oz, gather} x {configuration 0, 1} in ms, -1 when not
 * measured.  MDFT_AUTOTUNE=0, MDFT_ANGULAR or MDFT_OZ in the environment at create skip it. */
int mdft_get_kernel_forms(const mdft_handle *h, int *forms, double *ms);

/* ---- The reference's density file (output/density.bin, input/density.bin) ----
 *
 * Write (src/module_postprocessing.f90:45-95): Fortran unformatted sequential records with
 * 4-byte length markers -- ns (1; -1 when full), mmax, no, np, (nx, ny, nz), (dx, dy, dz),
 * nsite, one 176-byte site_type record per solute site (name blank, type and n_sites 0,
 * r, q, sig, eps, lambda1 = lambda2 = 0, Z), then per grid point (x fastest) one record of
 * np complex angl2proj(xi(:, point)), or with full != 0 no records of one real each.
 * xi: host array of no*nx*ny*nz doubles, or NULL for the handle's last solve; Z may be NULL. */
int mdft_write_density_bin(mdft_handle *h, const double *xi, int nsite, const double *q, const double *sig, const double *eps,
                           const double *xyz, const int *Z, int full, const char *path);
/* Restart (read_restart_file, src/module_density.f90:61-261): the file's projections become xi
 * on the file's grid (proj2angl with this handle's orientations; the file's mmax may be
 * lower), interpolated trilinearly onto this grid with the file's box centred in this one
 * (the reference's loop order: a point on a cell face takes the last cell's value; points
 * outside every cell keep xi's input value).  A full-density file needs this grid and
 * orientations.  The solute sites must match the file's (count no larger, positions equal
 * to the file's plus the centring offset, same sigma and epsilon).  xi (host, in/out). */
int mdft_read_density_bin(mdft_handle *h, const char *path, int nsite, const double *sig, const double *eps, const double *xyz,
                          double *xi);

/* ---- Input files of the reference (host only; no GPU needed) ----
 *
 * dft.in (src/module_input.f90): lines are 100-character records, cut at '#', blank lines
 * dropped (:654-732); a tag's value is list-directed-read from columns len(tag)+4 ..
 * len(tag)+50 of the first line that starts with the tag followed by a blank, i.e. after
 * "tag = " (:73-79); logicals take the first character of the first item, T/t or F/f
 * (:386-427).  The getters leave *out untouched and set *found = 0 when the tag is absent
 * (the caller's defaults stand); a value that does not read returns MDFT_E_IO. */
typedef struct mdft_input mdft_input;
int mdft_input_read(const char *path, mdft_input **out);
int mdft_input_free(mdft_input *in);
int mdft_input_nlines(const mdft_input *in, int *n);
int mdft_input_line(const mdft_input *in, int i, char *buf, int buflen);
/* n = 1..3 values (getinput%dp/dp2/dp3, getinput%int/int2/int3) */
int mdft_input_get_dp(const mdft_input *in, const char *tag, int n, double *out, int *found);
int mdft_input_get_int(const mdft_input *in, const char *tag, int n, int *out, int *found);
int mdft_input_get_log(const mdft_input *in, const char *tag, int *out, int *found);
/* character(50) value: the first list-directed item, NUL-terminated in out */
int mdft_input_get_char(const mdft_input *in, const char *tag, char *out, int outlen, int *found);
/* Grid and thermo of init_grid / init_thermo (src/module_grid.f90:62-95,
 * src/module_thermo.f90:25): molrotsymorder (default 2), boxlen (default 128 128 128),
 * boxnod (default nint(boxlen/0.3)), mmax (default 0), temperature (default 300); n0,
 * the c(k) path, precision and device come from the caller. */
int mdft_desc_from_input(const mdft_input *in, const char *ck_path, double n0, int precision, int device, mdft_desc *out);
/* solute.in (src/module_solute.f90:36-52): a comment line, the site count, a comment line,
 * then per site: index, q, sigma, epsilon, x, y, z, Z.  Charges are multiplied by
 * charge_scale (solute_charges_scale_factor).  With q == NULL only *nsite is returned;
 * otherwise the arrays hold cap sites (xyz 3 per site; Z may be NULL). */
int mdft_read_solute(const char *path, double charge_scale, int cap, int *nsite, double *q, double *sig, double *eps,
                     double *xyz, int *Z);
/* mv_solute_to_center (src/module_solute.f90:146-187): with translate, move the mean site
 * position to the box centre; then wrap every coordinate into [0, box) (Fortran MODULO). */
int mdft_center_solute(int nsite, double *xyz, const double *box, int translate);

/* ---- Learned warm start (no counterpart in the reference, whose solves always start
 * from guess_density, src/module_density.f90:267-284) ----
 *
 * A periodic 3-D convolutional encoder-decoder (4 levels, 16-128 channels, GELU,
 * 906,772 parameters; BF16 weights, FP32 activations and accumulation) maps 3 input
 * channels of a solute on the solver's grid -- Lennard-Jones energy, electrostatic
 * potential, Gaussian site density -- to the 4 m <= 1 projections of the converged
 * log-density ln(rho/rho0) in the real basis {1, u_x, u_y, u_z} (u: molecular z axis).
 * Device arrays are [channel][point], points in xi's order without io.  Grid
 * dimensions must be multiples of 8.  One network object serves one handle (it holds
 * the activation buffers and runs on one stream). */
typedef struct mdft_warm_net mdft_warm_net;

int mdft_warm_net_create(int nx, int ny, int nz, int device, mdft_warm_net **out);
int mdft_warm_net_destroy(mdft_warm_net *net);
int mdft_warm_net_num_params(const mdft_warm_net *net, long long *n);
/* He-normal weights from a seed (splitmix64 + Box-Muller), zero biases, head scaled 0.1. */
int mdft_warm_net_init(mdft_warm_net *net, unsigned long long seed);
/* FP32 master parameters (host arrays of num_params values); set resets Adam's moments. */
int mdft_warm_net_set_params(mdft_warm_net *net, const float *params, long long n);
int mdft_warm_net_get_params(const mdft_warm_net *net, float *params, long long n);
/* Run on this CUDA stream (NULL: the network's own stream). */
int mdft_warm_net_set_stream(mdft_warm_net *net, void *stream);
/* d_in: 3 x N channels; d_out (may be NULL): 4 x N projections; queued, not synchronised. */
int mdft_warm_net_forward(mdft_warm_net *net, const float *d_in, float *d_out);
/* Device address of the last forward's output (4 x N), valid until the next call. */
int mdft_warm_net_output(mdft_warm_net *net, const float **d_out);
/* Masked squared-error loss sum_v mask_v sum_c (y - t)^2 / (4 N) of one sample and its
 * gradient with respect to every parameter (host array of num_params FP32 values). */
int mdft_warm_net_gradients(mdft_warm_net *net, const float *d_in, const float *d_target, const float *d_mask, float *grad,
                            double *loss);
/* One Adam step (beta 0.9/0.999, eps 1e-8) on the mean gradient of nbatch samples
 * (device pointer arrays; d_mask may be NULL).  Queued, not synchronised. */
int mdft_warm_net_train_step(mdft_warm_net *net, const float *const *d_in, const float *const *d_target,
                             const float *const *d_mask, int nbatch, float lr);
/* Mean loss per sample of the training steps since the last call (synchronises). */
int mdft_warm_net_take_loss(mdft_warm_net *net, double *mean_loss);
int mdft_warm_net_launch_count(const mdft_warm_net *net, long long *count);
int mdft_warm_net_grid(const mdft_warm_net *net, int *nxyz);
/* A network with nout output channels (1..256): 4 is the m <= 1 form above; 2 np gives the
 * real and imaginary parts of all np complex projections of the log-density on a handle's
 * angular grid, in the order of the reference's angl2proj
 * (src/module_orientation_projection_transform.f90:159-199). */
int mdft_warm_net_create_n(int nx, int ny, int nz, int nout, int device, mdft_warm_net **out);
int mdft_warm_net_num_outputs(const mdft_warm_net *net, int *nout);

/* The network's 3 input channels for a solute on h's grid (sites as in mdft_solve). */
int mdft_warm_features(mdft_handle *h, int nsite, const double *q, const double *sig, const double *eps, const double *xyz,
                       int nsolvsite, const double *sq, const double *ssig, const double *seps, const double *sxyz,
                       double rvdw, float *d_feat);
/* Training target (4 x N) and loss mask (N, may be NULL) from a converged density d_xi
 * (device; NULL: the handle's last solve) with the handle's vext. */
int mdft_warm_target(mdft_handle *h, const double *d_xi, float *d_target, float *d_mask);
/* Starting density from 4 x N projections (d_xi device; NULL: the handle's solver point). */
int mdft_warm_expand(mdft_handle *h, const float *d_pred, double *d_xi);
/* Target and start of either output form: nout = 4 as above, or nout = 2 np (the log-density's
 * complex projections by the handle's angl2proj as real and imaginary planes; the start is
 * their proj2angl, src/module_orientation_projection_transform.f90:202-243, clamped and
 * exponentiated as in the m <= 1 form). */
int mdft_warm_target_n(mdft_handle *h, const double *d_xi, int nout, float *d_target, float *d_mask);
int mdft_warm_expand_n(mdft_handle *h, const float *d_pred, int nout, double *d_xi);
/* Make mdft_solve (and mdft_solve_batch on this handle) start from the network's
 * prediction instead of guess_density (either output form); NULL restores the bulk guess.  A warm-started
 * solve that ends in a line-search failure or at the iteration limit is redone from the
 * bulk guess.  The network must be built for the handle's grid; while attached it runs on
 * the handle's stream (detaching, or mdft_destroy of the handle, returns it to its own).
 * Detach a network before destroying it. */
int mdft_set_warm_net(mdft_handle *h, mdft_warm_net *net);
/* stats[0]: warm-started solves, stats[1]: of which redone from the bulk guess. */
int mdft_get_warm_stats(const mdft_handle *h, long long *stats);

/* ---- Bridge term, bridge = "cgb" (src/module_energy_and_gradient.f90:166-175, 246-275) ----
 *
 * The coarse-grained bridge of src/module_coarse_grained_gageat_bridge.f90:216-482 (one
 * species, FP64 handles only): n(r) = sum_io xi^2 rho0 w / n0, n_cg its convolution with a
 * normalised Gaussian of width sigma on the periodic grid, and F_b = sum kT dv n0 Phi(n_cg)
 * ('sla') or sum kT dv n0 (n - 1) Phi(n_cg) ('wda', cgb_version) with A3 = 1 - c00/2 and B6.
 * Once set, every full evaluation of the handle (mdft_energy_and_gradient*, the FP64
 * minimiser, mdft_solve, the batch) adds F_b to F and its gradient to df, and the stopping
 * quantities (max|df|, sum w df) include it; F = terms[0] + terms[1] + terms[2] + F_b +
 * terms[3].  FP32 evaluations (mixed solves) are refused while it is set; mdft_excess_energy
 * leaves it out, as the reference's excess seam does.  As in the reference, the 'wda'
 * gradient convolves Phi' before multiplying by (n - 1) (:349-419); it is not the
 * derivative of that F_b.  version MDFT_BRIDGE_NONE removes any bridge term. */
#define MDFT_BRIDGE_NONE 0     /* bridge = "no"              */
#define MDFT_BRIDGE_CGB_SLA 1  /* bridge = "cgb", cgb_version 'sla' (the default) */
#define MDFT_BRIDGE_CGB_WDA 2  /* bridge = "cgb", cgb_version 'wda' */
/* B6, sigma: cgb_B6 (default 0) and cgb_sigma (default 1 A); c00: c00_000 (mdft_cgb_c00). */
int mdft_set_bridge_cgb(mdft_handle *h, int version, double B6, double sigma, double c00);
/* c00_000 for the reference's solvent names: spce -14.64872 at mmax 0, -13.665 above;
 * tip3p -11.9078 (:260-263).  Other names: MDFT_E_ARG (the reference leaves it unset). */
int mdft_cgb_c00(const char *solvent, int mmax, double *c00);
/* bridge = "hard_sphere" (src/module_fmt.f90:5-317, one species, FP64 handles only): the
 * Kierlik-Rosinberg FMT functional (PY or CS, hs_functional) of the orientation-summed
 * density with hard spheres of radius R (hs_radius), minus the bulk excess chemical
 * potential and grand potential (src/module_hardspheres.f90:83-189) and minus the quadratic
 * part of the hard-sphere c(k) (src/cs_of_k_hard_sphere.f90, tabulated on the c(k) file's
 * step).  It enters evaluations as the "cgb" term does; setting one bridge replaces the
 * other.  An empty box (every |xi| <= epsilon) gives F_b = -Fexc0 and no gradient
 * (:46-49).  A weighted density n3 outside (0, 1) fails the evaluation with MDFT_E_NUMERIC
 * (the reference stops).  The reference computes the bulk parameters only with a
 * hard-sphere solute (src/compute_vext_hard_sphere.f90:46-53); here they are computed at set. */
#define MDFT_BRIDGE_HS_PY 1  /* hs_functional PY */
#define MDFT_BRIDGE_HS_CS 2  /* hs_functional CS */
int mdft_set_bridge_fmt(mdft_handle *h, int functional, double radius);
/* out[4] = {radius, excess chemical potential mu_exc0, bulk grand potential Fexc0, nb_k}. */
int mdft_get_bridge_fmt_params(const mdft_handle *h, double *out);
/* energy_bridge(fb, df) alone: fb, and df (host array, may be NULL) += the bridge
 * gradient; fb = 0 and df unchanged without a bridge. */
int mdft_bridge_energy(mdft_handle *h, const double *xi, double *fb, double *df);

/* ---- Multi-species solvent (nb_solvent > 1) ----
 *
 * energy_and_gradient of a solvent of nspec >= 2 species: replaces the excess pointer
 * set to energy_cproj_mrso_mixture (src/module_init_simu.f90:67-71,
 * src/module_energy_cproj_mrso_mixture.f90:67-850) with the ideal and external terms summed
 * over species (src/module_energy_ideal_and_external.f90:46-72).
 *
 * Up to 8 species.  Each species is an FP64 handle on one grid, mmax, mrso, temperature and device, created
 * with that species' n0 already multiplied by its mole fraction (as the reference stores
 * it, src/module_solvent.f90:221-222) and its own c(k) file, with its vext set
 * (mdft_set_vext or mdft_compute_vext with its own sites).  mole_fraction[s] must lie in
 * (0, 1] and the fractions must sum to exactly 1 (src/module_solvent.f90:476-485; a zero
 * fraction would give n0 = 0, which mdft_create refuses).  The mixture uses the species
 * handles' buffers and streams: while it is in use, do not evaluate on those handles
 * directly, and destroy it before them.  The reference takes the mixture routine only for
 * nspec > 1, so nspec = 1 is refused; that routine differs from the single-species one in
 * two ways, kept here: -q is rotated with R(m,mup,khi) (single species: R(m,mup,-khi)) and
 * at self-conjugate k-points the q result is kept.  As in the reference, species s2's
 * excess field is gamma_{s2} = sum_s c(s2) (x) drho_s (c_{s2,s} taken as c_{s2}).
 *
 * xi, df: [nspec][nz][ny][nx][no] doubles (each species' block in the single-species layout,
 * df as the reference's df(no,nx,ny,nz,nspec)); terms = {F_id, F_ext, F_exc, constant
 * corrections}, F_id and F_ext summed over species, the corrections species 0's
 * (mdft_set_constant_correction). */
typedef struct mdft_mixture mdft_mixture;
int mdft_mixture_create(mdft_handle *const *species, int nspec, const double *mole_fraction, mdft_mixture **out);
int mdft_mixture_destroy(mdft_mixture *m);
int mdft_mixture_energy_and_gradient(mdft_mixture *m, const double *xi, double *f, double *df, double *terms);
/* Device arrays (d_df may be NULL: energy only). */
int mdft_mixture_energy_and_gradient_device(mdft_mixture *m, const double *d_xi, double *d_df, double *f, double *terms);
/* energy_minimization of a mixture: the L-BFGS of mdft_minimize (FP64 only) over every
 * species' xi at once (xi: [nspec][N][no] host array, updated in place); the reference's
 * minimiser runs on the vector of all species. */
int mdft_mixture_minimize(mdft_mixture *m, double *xi, const mdft_minimize_opts *opts, mdft_minimize_result *res);

#ifdef __cplusplus
}
#endif
#endif /* MDFT_B200_H */
