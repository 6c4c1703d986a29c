/*
 * crowdphot_b200.h -- C ABI of the B200 crowded-field PSF-fitting library.
 *
 * The library replaces two Julia entry points of CrowdPhot.jl:
 *
 *   CrowdPhot.fit_all_stars_simultaneous(image, psf, sources, fit_rad; kws...)
 *       src/photometry/psf_photometry_simultaneous.jl:953-1431
 *   CrowdPhot.PSF.fit_star(model, image, inds; kws...)
 *       src/psf/psf_fitting.jl:229-308 (generic), :314-451 (CircularGaussianPSF),
 *       :1086-1173 (ImagePSF), :1177-1210 (GriddedPSFModel{T,<:ImagePSF})
 *
 * Conventions (all entry points):
 *   - Every image-shaped array is column-major (Julia layout): element (y, x),
 *     1-based, lives at offset (y-1) + (x-1)*ny.
 *   - Inputs and outputs are caller-owned host memory unless an entry point
 *     says "device".  Device state is owned by the context handle.
 *   - Return value 0 = success; negative = error (see CPB_ERR_*).  The text
 *     of the last error is available from cpb_last_error().  Argument errors
 *     carry the reference's ArgumentError message text.
 *   - Per-star failures are not errors: they are reported in valid[] /
 *     n_failed exactly as the reference does.
 *   - One call at a time per context (an internal mutex serialises callers).
 */
#ifndef CROWDPHOT_B200_H
#define CROWDPHOT_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define CPB_API __attribute__((visibility("default")))
#else
#define CPB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define CPB_OK 0
#define CPB_ERR_ARGUMENT (-1)  /* reference ArgumentError */
#define CPB_ERR_CUDA (-2)      /* CUDA runtime / launch error */
#define CPB_ERR_OOM (-3)       /* device memory exhausted or admission refused */
#define CPB_ERR_TIMEOUT (-4)   /* a bounded device-side wait gave up */
#define CPB_ERR_INTERNAL (-5)  /* also: a device index check failed (libcrowdphot_b200_checked.so) */
#define CPB_ERR_NO_DEVICE (-6) /* no CUDA device / library built without GPU */

/* ---- element types ----------------------------------------------------- */
#define CPB_F32 1
#define CPB_F64 2

/* ---- PSF kinds (the supported AbstractPSFModel subtypes) --------------- */
#define CPB_PSF_GRIDDED_IMAGE 1     /* GriddedPSFModel{T,<:ImagePSF{T}}  src/psf/gridded_psf.jl:51-62 */
#define CPB_PSF_IMAGE 2             /* ImagePSF{T}                        src/psf/empirical_models.jl:76-85 */
#define CPB_PSF_CIRCULAR_GAUSSIAN 3 /* CircularGaussianPSF{T}             src/psf/parametric_models.jl:62-115 */

/*
 * PSF descriptor.  For CPB_PSF_GRIDDED_IMAGE every node is an ImagePSF;
 * for CPB_PSF_IMAGE n_nodes == 1 (grid_y/grid_x ignored); for
 * CPB_PSF_CIRCULAR_GAUSSIAN n_nodes == 0 and only `fwhm` is read.
 * Node k's tabulated data is node_data[k], column-major node_ny[k] x node_nx[k]
 * (ImagePSF.data), node_os[2k], node_os[2k+1] = ImagePSF.oversampling[1] (x
 * factor), oversampling[2] (y factor); node_origin[2k], node_origin[2k+1] =
 * ImagePSF.origin.y, origin.x; node_fill_value[k] = ImagePSF.fill_value;
 * grid_y[k], grid_x[k] = GriddedPSFModel node positions.
 */
typedef struct cpb_psf_desc {
    int32_t kind;
    int32_t n_nodes;
    int32_t eltype; /* element type of node_data */
    int32_t reserved;
    const void* const* node_data;
    const int64_t* node_ny;
    const int64_t* node_nx;
    const int64_t* node_os;
    const double* node_origin;
    const double* node_fill_value;
    const double* grid_y;
    const double* grid_x;
    double fwhm;
} cpb_psf_desc;

/* free-parameter bits (order of the reference's getproperties) */
#define CPB_FREE_Y 1
#define CPB_FREE_X 2
#define CPB_FREE_FLUX 4
#define CPB_FREE_BKG 8  /* fit_star only */
#define CPB_FREE_FWHM 16 /* fit_star with CircularGaussianPSF only */

/* arithmetic of the device path */
#define CPB_PREC_FP64 0  /* plain form: every step in FP64 */
#define CPB_PREC_MIXED 1 /* FP32 stamps/render/residual/J products; FP64 solver scalars */

/* covariance estimator (levenberg_marquardt.jl:366-388) */
#define CPB_COV_AUTO 0          /* KnownWeights iff inv_var given */
#define CPB_COV_KNOWN_WEIGHTS 1
#define CPB_COV_REWEIGHTED 2

/* damping (levenberg_marquardt.jl:64-99) */
#define CPB_DAMP_MARQUARDT 0
#define CPB_DAMP_LEVENBERG 1
#define CPB_DAMP_NONE 2

/* inner Krylov solver of the simultaneous fit */
#define CPB_SOLVER_LSQR 0
#define CPB_SOLVER_LSMR 1 /* LSMR (Fong & Saunders); batched groups run through the full-field fit */

/*
 * Keyword arguments of fit_all_stars_simultaneous
 * (psf_photometry_simultaneous.jl:953-981).  Non-free y/x/flux take the
 * matching fixed_* value (the reference's `fixed` NamedTuple); bkg is always
 * fixed (contract :1019-1031); fixed_fwhm is the Gaussian's fixed FWHM.
 * model_rad_max < 0 means the default 10*fit_rad.
 */
typedef struct cpb_sim_params {
    double fit_rad;
    int32_t free_mask;
    int32_t inner_iterations; /* 10 */
    double fixed_y, fixed_x, fixed_flux, fixed_bkg, fixed_fwhm;
    double linear_tol;        /* 1e-6 */
    int32_t model_rad_auto;   /* 1 = :auto: per-star radii from the unit PSF's curve of growth (needs inv_var) */
    int32_t max_trials;       /* 8 */
    double model_rad;         /* used when model_rad_auto == 0 */
    double model_rad_max;     /* 10*fit_rad */
    double model_rad_nsigma;  /* 1 */
    double max_step;          /* 0.25 */
    int32_t max_iter;         /* 40 */
    int32_t covariance;       /* CPB_COV_* */
    double x_tol, f_tol, g_tol;                          /* 1e-5, 1e-4, 1e-4 */
    double lambda_init, lambda_up, lambda_down;          /* 1e-4, 10, 10 */
    double lambda_min, lambda_max;                       /* 1e-12, 1e12 */
    int32_t precision;        /* CPB_PREC_* */
    int32_t solver;           /* CPB_SOLVER_* */
    int32_t damping;          /* CPB_DAMP_* */
    /* precision == CPB_PREC_MIXED only: FP64 refinement iterations after the
     * FP32-stamp loop (every active star live again on the original data, from
     * the mixed-precision parameters, damping restarted at lambda_init, same
     * tests; converged flags accumulate).  0 = none: the final FP64 pass then
     * only re-evaluates errors, residual and diagnostics at the
     * mixed-precision parameters. */
    int32_t refine_iters;
    /* spread_model reference disk FWHM: NaN = from the PSF's effective area
     * (the reference default, _spread_fwhm); <= 0 = skip spread_model */
    double spread_model_fwhm;
} cpb_sim_params;

/*
 * Result of a simultaneous fit (MultiPassPhotResult,
 * psf_photometry_single.jl:99-122).  All arrays are caller-allocated with n
 * entries (catalogue order); NULL skips an optional output.  residual is
 * ny*nx column-major.  The dbg_* exports give the integer structures the
 * reference builds once per fit (active order, stamp pixel indices, model
 * radii) for bit-exact comparison; n_active and n_union are always written.
 */
typedef struct cpb_sim_result {
    double *y, *x, *flux, *bkg;
    double *y_err, *x_err, *flux_err, *bkg_err;
    uint8_t *converged, *valid;
    double* chisq;            /* optional */
    double *qfit, *qfit_expected, *qfit_z, *crowding; /* optional diagnostics */
    int32_t* n_iter;
    double* residual;         /* optional, ny*nx */
    int32_t* dbg_active;      /* optional, n: catalogue index (0-based) per active slot */
    int32_t* dbg_pixels;      /* optional, S2*n: 1-based flat pixel per stamp entry, 0 = unusable */
    int32_t* dbg_model_R;     /* optional, n: per active slot */
    int32_t n_passes;
    int32_t n_failed;
    int64_t n_active;
    int64_t n_union;
    /* work counters */
    int64_t n_trials;         /* damping trials run */
    int64_t n_lsqr_iters;     /* LSQR iterations run (summed over trials) */
    double model_px_evals;    /* stamp fills + renders, star-pixel evaluations */
    double lsqr_px_macs;      /* star-pixel products in J and J^T */
    double device_seconds;    /* device-timed fit, excluding host<->device copies */
    double *spread_model, *spread_model_err; /* optional, n */
} cpb_sim_result;

/*
 * Keyword arguments of fit_star / lm_irls (psf_fitting.jl:229-250,
 * levenberg_marquardt.jl:431-449), IRLS reweighting included (fields below).
 */
typedef struct cpb_lm_params {
    int32_t free_mask;        /* CPB_FREE_* bits */
    int32_t max_iter;         /* 200 */
    double fixed_y, fixed_x, fixed_flux, fixed_bkg, fixed_fwhm;
    double x_tol, f_tol, g_tol;                  /* 1e-8, 1e-4, 1e-4 */
    double lambda_init, lambda_up, lambda_down;  /* 1e-4, 10, 10 */
    double lambda_min, lambda_max;               /* 1e-12, 1e12 */
    double min_diagonal;      /* MarquardtDamping.min_diagonal, 1e-6 */
    int32_t damping;          /* CPB_DAMP_* */
    int32_t covariance;       /* CPB_COV_* */
    int32_t precision;        /* CPB_PREC_* */
    int32_t reserved;
    /* IRLS reweighting: lm_irls's reweight / scale_estimator / weight_reset_tol
     * (levenberg_marquardt.jl:105-355, 420-425, 611-645).  CPB_LOSS_NONE (the
     * zero value) is the plain fit. */
    int32_t reweight;         /* CPB_LOSS_* */
    int32_t scale_estimator;  /* CPB_SCALE_* */
    double loss_param;        /* HuberLoss d / TukeyLoss c */
    double scale_value;       /* FixedScale sigma */
    double mscale_delta, mscale_tol; /* MScale: 0.5, 1e-6 */
    int32_t mscale_max_iter;  /* MScale: 30 */
    int32_t reserved2;
    double weight_reset_tol;  /* 0.1 */
} cpb_lm_params;

/* IRLS losses (LossFunctions.L2DistLoss, LossFunctions.HuberLoss(d),
 * CrowdPhot.TukeyLoss(c)) and scale estimators (MADScale, FixedScale(sigma),
 * MScale(delta, tol, max_iter)); CPB_SCALE_AUTO is the reference's default:
 * FixedScale(sqrt(1 / mean(weights))) when inv_var is given, else MADScale. */
#define CPB_LOSS_NONE 0
#define CPB_LOSS_L2DIST 1
#define CPB_LOSS_HUBER 2
#define CPB_LOSS_TUKEY 3
#define CPB_LOSS_LOGITDIST 4 /* LossFunctions.jl LogitDistLoss: psi(r) = tanh(r/2), psi'(0) = 1/2 */
#define CPB_SCALE_AUTO 0
#define CPB_SCALE_MAD 1
#define CPB_SCALE_FIXED 2
#define CPB_SCALE_MSCALE 3

/*
 * Per-cutout result of the batched LM fit (LMResult, levenberg_marquardt.jl:28-41).
 * np = number of model parameters (4 for image/gridded: y,x,flux,bkg; 5 for
 * CircularGaussianPSF: y,x,fwhm,flux,bkg); nf = number of free ones.
 * params: n*np (fitted model parameters, fixed ones included);
 * cov: n*nf*nf column-major (optional).  status[c] is 0, or CPB_ERR_ARGUMENT
 * when cutout c fails the reference's input checks (too few valid pixels).
 */
typedef struct cpb_lm_result {
    double* params;
    double* cov;              /* optional */
    double *cost, *cost_init, *chisq, *lambda_final;
    uint8_t *converged, *x_converged, *f_converged, *g_converged;
    int32_t* iterations;
    int32_t* status;
    double device_seconds;
    double* sigma_final;      /* optional: the last IRLS scale estimate (NaN without IRLS) */
} cpb_lm_result;

typedef struct cpb_ctx cpb_ctx;
typedef struct cpb_psf cpb_psf;

/* ---- context ------------------------------------------------------------ */
/* Creates a context on CUDA device `device`. */
CPB_API int cpb_ctx_create(int device, cpb_ctx** out);
CPB_API int cpb_ctx_destroy(cpb_ctx* ctx);
/* Text of the last error on this context ("" if none); valid until the next call. */
CPB_API const char* cpb_last_error(const cpb_ctx* ctx);
/* Library version string. */
CPB_API const char* cpb_version(void);

/*
 * Instrumentation (no counterpart in the reference).  Every kernel launch of a
 * context is counted; with profiling enabled each launch is also bracketed by
 * CUDA events on the context stream and credited with its algorithmic bytes
 * (each distinct array element it must move, counted once).  Profiling adds
 * two event records per launch; leave it off for timed runs.
 */
typedef struct cpb_kernel_stat {
    char name[32];
    int64_t launches;
    double seconds;  /* summed event-timed duration */
    double bytes;    /* summed algorithmic bytes */
} cpb_kernel_stat;
CPB_API int cpb_ctx_set_profiling(cpb_ctx* ctx, int enable);

/*
 * Bounded device waits (no counterpart in the reference, which runs on one
 * thread).  The persistent fit_all_stars pass kernel spins on its ready queue
 * for at most `polls` polls of >= 64 ns per wait (<= 0: the default, 2^26, a few
 * seconds) before it gives up and the call returns CPB_ERR_TIMEOUT with the
 * reason in cpb_last_error; the context stays usable.
 */
CPB_API int cpb_ctx_set_wait_limit(cpb_ctx* ctx, int64_t polls);
/*
 * Host-side fault injection for testing the bounded waits above; no GPU fault
 * is involved.  CPB_FAULT_HOLD_READY_STAR: the next fit_all_stars call holds the
 * brightest star of its first pass back from the ready queue, so the stars that
 * wait for it never become ready and the waits run out (CPB_ERR_TIMEOUT).  The
 * injection applies to one call and then clears itself.
 */
#define CPB_FAULT_NONE 0
#define CPB_FAULT_HOLD_READY_STAR 1
CPB_API int cpb_ctx_inject_fault(cpb_ctx* ctx, int32_t fault);
/* Writes up to max_out per-kernel records, the number available to *n_out and
 * the total launch count to *launches; reset != 0 clears the counters. */
CPB_API int cpb_ctx_kernel_stats(cpb_ctx* ctx, cpb_kernel_stat* out, int max_out, int* n_out, int64_t* launches,
                                 int reset);

/* ---- PSF ---------------------------------------------------------------- */
/*
 * Validates and uploads a PSF once (GriddedPSFModel constructor checks,
 * gridded_psf.jl:64-135; ImagePSF checks, empirical_models.jl:91-140).
 * The node grid (ygrid, xgrid, index_grid) is derived here.
 */
CPB_API int cpb_psf_upload(cpb_ctx* ctx, const cpb_psf_desc* desc, cpb_psf** out);
CPB_API int cpb_psf_free(cpb_ctx* ctx, cpb_psf* psf);

/* ---- simultaneous fit (fit_all_stars_simultaneous) ---------------------- */
/*
 * image: ny*nx of `eltype`; inv_var (nullable) and background (nullable):
 * same shape and eltype.  The fitted data are image - background.  y0/x0/flux0:
 * the catalogue (sources.y, sources.x, sources.flux), n entries.
 * Replaces psf_photometry_simultaneous.jl:953-1431.
 */
CPB_API int cpb_fit_simultaneous(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params,
                         const void* image, int32_t eltype, int64_t ny, int64_t nx,
                         const void* inv_var, const void* background,
                         int64_t n, const double* y0, const double* x0, const double* flux0,
                         cpb_sim_result* out);

/*
 * Same fit with image / inv_var / background / catalogue already resident in
 * device memory ("device" pointers).  Outputs are still host arrays.
 */
CPB_API int cpb_fit_simultaneous_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params,
                                const void* d_image, int32_t eltype, int64_t ny, int64_t nx,
                                const void* d_inv_var, const void* d_background,
                                int64_t n, const double* d_y0, const double* d_x0,
                                const double* d_flux0, cpb_sim_result* out);

/*
 * No-allocation form of cpb_fit_simultaneous_device.  It has no counterpart in
 * the reference.  It exists for callers that cannot allocate device memory
 * while they fit: hosts whose device memory belongs to another allocator's
 * pool (CUDA.jl's pool allocator in Julia, PyTorch's caching allocator),
 * where a cudaMalloc behind the pool's back can fail or fragment the pool,
 * and loops that cannot take cudaMalloc's implicit device synchronisation.  It
 * allocates nothing: all scratch comes from one static 64 MiB device region
 * the library holds on each GPU that uses it until the process exits.  Fields
 * whose scratch would exceed that region (roughly beyond 512 x 512 pixels with
 * a few thousand 25 x 25 stamps) are rejected with CPB_ERR_ARGUMENT and a
 * message naming the size ("too large for the no-allocation entry point"),
 * before the fit's outer loop starts.  The first call on a device looks up
 * the region's address (cudaGetSymbolAddress); make that call before any
 * stream capture, and do not use this entry point on a device after a
 * cudaDeviceReset of it (the looked-up address would be stale).  All calls
 * share the region and find the previous call's contents in it (the fit
 * clears what must start at zero); calls whose GPU work overlaps race on it,
 * so serialise them.  The context must already exist.
 */
CPB_API int cpb_fit_simultaneous_device_noalloc(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params,
                                                const void* d_image, int32_t eltype, int64_t ny, int64_t nx,
                                                const void* d_inv_var, const void* d_background, int64_t n,
                                                const double* d_y0, const double* d_x0, const double* d_flux0,
                                                cpb_sim_result* out);

/* ---- sequential multi-pass photometry (fit_all_stars) ------------------- */
/*
 * Result of fit_all_stars (MultiPassPhotResult, psf_photometry_single.jl:99-122)
 * with the models' parameters in getproperties order (np per star: y, x, flux,
 * bkg for image PSFs; y, x, fwhm, flux, bkg for CircularGaussianPSF).
 * Arrays are caller-allocated host memory; NULL skips an optional one.
 */
typedef struct cpb_multipass_result {
    double* params;            /* n*np fitted parameters (fixed ones as given) */
    double* errors;            /* n*np (0 for fixed parameters, NaN before a star's first fit) */
    uint8_t *converged, *valid;
    double* chisq;
    double *qfit, *qfit_expected, *qfit_z, *crowding; /* optional */
    int32_t* n_iter;           /* LM iterations summed over the passes */
    double* residual;          /* optional, ny*nx: the data with every valid star's model subtracted */
    int32_t n_passes;
    int32_t n_failed;          /* fits that failed the reference's input checks */
    int64_t n_levels;          /* longest chain of dependent fits, summed over the passes */
    int64_t n_fits;            /* fit_star calls run */
    double device_seconds;
    double *spread_model, *spread_model_err; /* optional */
} cpb_multipass_result;

/*
 * CrowdPhot.fit_all_stars (psf_photometry_single.jl:267-469): n_passes
 * brightness-ordered passes; each valid star is added back (passes 2+),
 * fitted with fit_star on its +-fit_rad box of the running residual image and
 * subtracted again.  Two stars depend on each other only through pixels their
 * boxes share, and each pass fixes every box at its start, so a star waits
 * only for the brighter stars whose boxes meet its own; stars that are ready
 * together have disjoint boxes and are fitted concurrently (one device launch
 * per pass; IRLS and multi-node PSFs run the pass as batches of such stars).
 * The result equals the one-star-at-a-time order of the reference.  image:
 * ny*nx of eltype (background-subtracted); inv_var nullable; init: n*np
 * initial parameters (_extract_source_catalog: y, x from the catalogue, flux
 * from it or 1, bkg from it or 0, other parameters the PSF's own).  LM keyword
 * arguments (IRLS included) as cpb_fit_lm_batch.  Host arrays.  A pass whose
 * device queue stalls (a fault of the library, not of the data) returns
 * CPB_ERR_TIMEOUT after a bounded wait of a few seconds.
 * spread_model_fwhm: as cpb_sim_params.spread_model_fwhm.
 */
CPB_API int cpb_fit_all_stars(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* params, double fit_rad,
                              int32_t n_passes, double spread_model_fwhm, const void* image, int32_t eltype,
                              int64_t ny, int64_t nx, const void* inv_var, int64_t n, const double* init,
                              cpb_multipass_result* out);

/*
 * The spread_model reference disk (_exp_disk_kernel_bandlimited,
 * src/photometry/psf_photometry_diagnostics.jl:82-108): the circular
 * exponential disk of FWHM fwhm (scale length fwhm/16, a 6-Gaussian mixture)
 * band-limited to the pixel Nyquist frequency, (2 half + 1)^2 values
 * column-major into K, normalised to sum 1.  The fits use it with
 * half = ceil(fit_rad).  Host-only (no device work).
 */
CPB_API int cpb_exp_disk_kernel(double fwhm, int32_t half, double* K);

/* ---- many small simultaneous fits (star groups) ------------------------- */
/*
 * Results of a batch of independent fit_all_stars_simultaneous calls, one
 * per group (a small field holding a blend of stars).  Per-star arrays have
 * one entry per catalogue star, groups concatenated in order (group g's stars
 * at star_offsets[g] .. star_offsets[g+1]); they mean what the same-named
 * cpb_sim_result fields mean.  Per-group arrays have n_groups entries.
 * status[g] is 0, or CPB_ERR_ARGUMENT when group g fails one of the
 * reference's data checks (error_kind[g] = 1: the image holds non-finite
 * values but no inv_var was given; 2: a star's integer anchor is negative);
 * the per-star outputs of such a group hold its catalogue with NaN errors
 * and valid = 0.  residual (optional) is packed like the pixels.  NULL skips
 * an optional output.
 */
typedef struct cpb_group_result {
    double *y, *x, *flux;
    double *y_err, *x_err, *flux_err;
    uint8_t *converged, *valid;
    int32_t* n_iter;
    double* chisq;                                     /* optional */
    double *qfit, *qfit_expected, *qfit_z, *crowding;  /* optional */
    double* residual;                                  /* optional, packed like the pixels */
    int32_t *n_passes, *n_failed, *status;
    int32_t* error_kind;                               /* optional */
    int32_t *n_active, *n_union;                       /* optional */
    int32_t *n_trials, *n_lsqr_iters;                  /* optional */
    int64_t n_kernel_groups;  /* groups fitted by the one-block-per-group kernel */
    int64_t n_routed_groups;  /* groups too large for it, fitted by the full-field path */
    double device_seconds;
    double *spread_model, *spread_model_err;  /* optional (params->spread_model_fwhm sizes the disk) */
} cpb_group_result;

/*
 * n_groups independent fit_all_stars_simultaneous calls sharing one PSF and
 * one set of keyword arguments (psf_photometry_simultaneous.jl:953-1431,
 * applied to each group).  Group g's image is the column-major block
 * pixels[pix_offsets[g] .. pix_offsets[g] + ny[g]*nx[g]); inv_var and
 * background (nullable) share the layout; its catalogue is y0/x0/flux0
 * [star_offsets[g] .. star_offsets[g+1]) in the group's own 1-based pixel
 * coordinates (star_offsets has n_groups + 1 entries).  Results equal those of
 * cpb_fit_simultaneous on each group alone, within the parity tolerances
 * (the batch sums its reductions in a different order).  Groups of at most
 * 64 stars whose working set fits in shared memory are fitted by a
 * persistent kernel, one thread block per group, from a device work queue;
 * larger groups go through the full-field path.  precision must be
 * CPB_PREC_FP64.  Host arrays.
 */
CPB_API int cpb_fit_simultaneous_batch(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params,
                                       int64_t n_groups, const int64_t* pix_offsets, const int32_t* ny,
                                       const int32_t* nx, const void* pixels, int32_t eltype, const void* inv_var,
                                       const void* background, const int64_t* star_offsets, const double* y0,
                                       const double* x0, const double* flux0, cpb_group_result* out);

/*
 * cpb_fit_simultaneous_batch on device-resident groups (no counterpart in the
 * reference): every array argument and every pointer in `out` is a device
 * pointer on the context's device.  total_pixels = the pixel elements the
 * groups span (sizes the residual; 0 is allowed when out->residual is NULL).
 */
CPB_API int cpb_fit_simultaneous_batch_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params,
                                              int64_t n_groups, const int64_t* d_pix_offsets, const int32_t* d_ny,
                                              const int32_t* d_nx, const void* d_pixels, int32_t eltype,
                                              const void* d_inv_var, const void* d_background,
                                              const int64_t* d_star_offsets, const double* d_y0,
                                              const double* d_x0, const double* d_flux0, int64_t total_pixels,
                                              cpb_group_result* out);

/* ---- batched per-star LM (fit_star) ------------------------------------- */
/*
 * n_cutouts independent fit_star calls.  Cutout c is the column-major block
 * pixels[offsets[c] .. offsets[c] + ny[c]*nx[c]) holding image[inds] with
 * inds = (y_origin[c] : y_origin[c]+ny[c]-1, x_origin[c] : x_origin[c]+nx[c]-1)
 * (1-based image coordinates, which are the coordinates the model is evaluated
 * at).  inv_var (nullable) shares the layout.  init: n_cutouts*np initial
 * model parameters.  Replaces psf_fitting.jl:229-308, :314-451, :1086-1210.
 */
CPB_API int cpb_fit_lm_batch(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* params,
                     int64_t n_cutouts, const int64_t* offsets, const int32_t* ny,
                     const int32_t* nx, const int32_t* y_origin, const int32_t* x_origin,
                     const void* pixels, int32_t eltype, const void* inv_var,
                     const double* init, cpb_lm_result* out);

/*
 * cpb_fit_lm_batch on device-resident cutouts (no counterpart in the
 * reference, whose fit_star takes host arrays; this serves callers whose
 * cutouts already sit on the GPU, and the throughput measurement).  Every
 * array argument and every pointer in `out` is a device pointer on the
 * context's device; out->status is required, the other outputs may be null.
 * total_pixels = the pixel elements the cutouts span (used only to credit the
 * instrumentation's byte count; 0 is allowed).  Cutout dimensions are checked
 * on the device: a cutout with ny or nx <= 0 gets status CPB_ERR_ARGUMENT.
 * Returns when the fits are done; out->device_seconds is their GPU time.
 */
CPB_API int cpb_fit_lm_batch_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* params,
                                    int64_t n_cutouts, const int64_t* d_offsets, const int32_t* d_ny,
                                    const int32_t* d_nx, const int32_t* d_y_origin, const int32_t* d_x_origin,
                                    const void* d_pixels, int32_t eltype, const void* d_inv_var,
                                    const double* d_init, int64_t total_pixels, cpb_lm_result* out);

/* ---- one captured launch for a mixed batch (fit_star cutouts + groups) -- */
/*
 * No counterpart in the reference (whose fits run one call at a time on the
 * CPU).  A batch graph binds a batch of fit_star cutouts
 * (cpb_fit_lm_batch_device's arguments) and a batch of star groups
 * (cpb_fit_simultaneous_batch_device's arguments) to fixed device buffers and
 * captures both persistent kernels, each with its work-queue reset, in one
 * CUDA graph whose two branches run concurrently.  Every replay fits the
 * current contents of the bound input buffers into the bound output buffers:
 * refill the inputs in place (same sizes) and launch again.  Either half may
 * be empty (n_cutouts = 0 or n_groups = 0, other arguments of that half then
 * ignored).  Groups too large for one thread block are refused
 * (CPB_ERR_ARGUMENT): fit them with cpb_fit_simultaneous_batch.
 *
 * Launch shapes.  autotune = 0 uses the default shapes; 1 looks the batch's
 * signature up in the tuning cache at cache_path (NULL: the file named by the
 * CPB_TUNE_CACHE environment variable, else no file) and, when absent, times
 * every candidate shape on the bound batch itself (each candidate runs the
 * real fits once; outputs are overwritten), keeps the fastest and records it;
 * 2 re-tunes even when cached.  The shapes are: persistent blocks per SM (1
 * or 2) and whether the ePSF node is staged in shared memory for the fit_star
 * kernel; threads per block (64, 128 or 256) for each launch of the group
 * kernel (groups are launched in buckets of similar star count, each with a
 * shared-memory layout sized for its largest group).  `info` (nullable)
 * reports the choice; its grp_* fields describe the launch of the largest
 * groups.
 */
typedef struct cpb_tune_info {
    int32_t lm_blocks_per_sm;
    int32_t lm_node_in_smem;
    int32_t grp_threads;
    int32_t grp_blocks_per_sm;
    int32_t from_cache;   /* 1 when both choices came from the cache */
    int32_t n_timed;      /* candidate launches timed by this call */
    double lm_ms, grp_ms; /* device time of the chosen shapes (0 when not timed) */
} cpb_tune_info;

typedef struct cpb_batch_graph cpb_batch_graph;

CPB_API int cpb_batch_graph_create(cpb_ctx* ctx, const cpb_psf* psf,
                                   /* fit_star half */
                                   const cpb_lm_params* lm_params, int64_t n_cutouts, const int64_t* d_offsets,
                                   const int32_t* d_ny, const int32_t* d_nx, const int32_t* d_y_origin,
                                   const int32_t* d_x_origin, const void* d_pixels, int32_t lm_eltype,
                                   const void* d_inv_var, const double* d_init, int64_t lm_total_pixels,
                                   const cpb_lm_result* d_lm_out,
                                   /* group half */
                                   const cpb_sim_params* sim_params, int64_t n_groups, const int64_t* d_pix_offsets,
                                   const int32_t* d_gny, const int32_t* d_gnx, const void* d_gpixels,
                                   int32_t g_eltype, const void* d_ginv_var, const void* d_gbackground,
                                   const int64_t* d_star_offsets, const double* d_y0, const double* d_x0,
                                   const double* d_flux0, int64_t g_total_pixels, const cpb_group_result* d_g_out,
                                   /* launch shapes */
                                   int32_t autotune, const char* cache_path, cpb_batch_graph** out,
                                   cpb_tune_info* info);
/* Replays the graph on the context's stream and waits for it; *device_seconds
 * (nullable) receives its GPU time. */
CPB_API int cpb_batch_graph_launch(cpb_ctx* ctx, cpb_batch_graph* graph, double* device_seconds);
CPB_API int cpb_batch_graph_destroy(cpb_ctx* ctx, cpb_batch_graph* graph);

/* ---- serving: continuous batching of fit requests ------------------------ */
/*
 * No counterpart in the reference.  A server keeps PSFs resident on one GPU
 * and runs fit_all_stars_simultaneous requests (fields of any size) as they
 * arrive: up to max_inflight requests run at once, each on its own stream with
 * its own device working memory (kept between requests and reused), so their
 * kernels overlap on the GPU.  A queued request is admitted as soon as a slot
 * is free and its estimated device memory fits the budget (free device memory
 * at creation minus hbm_reserve_bytes, less what running requests and idle
 * slots hold; idle slots give their memory back when an admission needs it).
 * Queued requests are admitted first-fit in arrival order, so a large request
 * does not hold back smaller ones that fit.  A request whose estimate exceeds
 * the whole budget fails with CPB_ERR_OOM.  Each result is the one
 * cpb_fit_simultaneous gives for the same request alone (the fits are
 * deterministic and requests share no state).
 *
 * The host buffers a request names (inputs and cpb_sim_result arrays) must
 * stay valid and untouched until the request is done, failed or cancelled.
 * Calls are thread-safe.
 */
typedef struct cpb_server cpb_server;

typedef struct cpb_server_config {
    int32_t device;
    int32_t max_inflight;       /* concurrent requests; <= 0 means 4 */
    int64_t hbm_reserve_bytes;  /* device memory admission leaves free; < 0 means 2 GiB */
} cpb_server_config;

#define CPB_REQ_QUEUED 0
#define CPB_REQ_RUNNING 1
#define CPB_REQ_DONE 2
#define CPB_REQ_FAILED 3
#define CPB_REQ_CANCELLED 4

typedef struct cpb_request_info {
    int32_t state;            /* CPB_REQ_* */
    int32_t status;           /* the fit's return code once done / failed */
    int32_t slot;             /* slot that ran it, -1 if none */
    int32_t reserved;
    int64_t est_bytes;        /* admission estimate of its device memory */
    double queued_seconds;    /* submit -> start */
    double run_seconds;       /* start -> done (host clock) */
    double latency_seconds;   /* submit -> done */
    double device_seconds;    /* the fit's device time */
    double start_time;        /* start and end, seconds since the server was created */
    double end_time;
    char error[256];          /* cpb_last_error text when failed */
} cpb_request_info;

CPB_API int cpb_server_create(const cpb_server_config* config, cpb_server** out);
/* Uploads a PSF once (as cpb_psf_upload); *psf_id names it in submits. */
CPB_API int cpb_server_add_psf(cpb_server* server, const cpb_psf_desc* desc, int32_t* psf_id);
/* Queues one fit_all_stars_simultaneous request (cpb_fit_simultaneous's
 * arguments; host buffers).  Returns at once with *request_id. */
CPB_API int cpb_server_submit(cpb_server* server, int32_t psf_id, const cpb_sim_params* params, const void* image,
                              int32_t eltype, int64_t ny, int64_t nx, const void* inv_var, const void* background,
                              int64_t n, const double* y0, const double* x0, const double* flux0,
                              cpb_sim_result* out, int64_t* request_id);
CPB_API int cpb_server_poll(cpb_server* server, int64_t request_id, cpb_request_info* info);
/* Waits until the request is done, failed or cancelled, or timeout_seconds
 * pass (< 0: no limit); returns CPB_ERR_TIMEOUT on timeout. */
CPB_API int cpb_server_wait(cpb_server* server, int64_t request_id, double timeout_seconds, cpb_request_info* info);
/* Cancels a queued request (a running one finishes); CPB_ERR_ARGUMENT if it
 * is no longer queued. */
CPB_API int cpb_server_cancel(cpb_server* server, int64_t request_id);
/* Cancels queued requests, waits for running ones, frees everything. */
CPB_API int cpb_server_destroy(cpb_server* server);
/* Text of the server's last call error ("" if none). */
CPB_API const char* cpb_server_last_error(const cpb_server* server);

#ifdef __cplusplus
}
#endif

#endif /* CROWDPHOT_B200_H */
