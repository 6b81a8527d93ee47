/*
 * icar_adv.h -- C ABI of the B200 tracer-advection step for ICAR/HICAR.
 *
 * Drop-in boundary for ICAR's advection module (src/physics/advection_driver.f90,
 * module `advection`, public :: advect, adv_init, adv_var_request).  A Fortran
 * ISO_C_BINDING shim binds these functions one to one; plain pointers, sizes
 * and status codes only, no C++ or CUDA types in any signature.
 *
 * Data model.  One handle = one ICAR image's domain (domain_t) on one GPU.
 * Every 3-D field is passed in the Fortran layout of domain_t:
 *   data_3d(ims:ime, kms:kme, jms:jme), x fastest, then z, then y
 * with the staggered extents of the reference: u-grid fields (u, jacobian_u)
 * have nx+1 points in x, v-grid fields (v, jacobian_v) have ny+1 points in y
 * (src/objects/domain_obj.f90:1916-1931).  Host strides are given in elements
 * for the (x, z, y) axes; {1, nx', nx'*nz} is a contiguous Fortran array.
 * The handle owns the device copies: species, winds and metric fields stay
 * resident in GPU memory across steps and only move on set/get calls.
 *
 * Errors.  Every call returns an icar_adv_status; nothing aborts.  The message
 * of the last failure on a handle is icar_adv_last_error(h) (h may be NULL for
 * failures that happened before a handle existed).
 *
 * Threading.  A handle is used by one host thread at a time; its work goes on
 * the handle's CUDA stream.  Different handles may be driven concurrently.
 */
#ifndef ICAR_ADV_H
#define ICAR_ADV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ICAR_ADV_ABI_VERSION 1
#define ICAR_ADV_MAX_SPECIES 32

/* Scheme switches, src/constants/icar_constants.f90:419-422. */
enum { ICAR_ADV_STD = 1, ICAR_ADV_MPDATA = 2 };
enum { ICAR_FLUXCOR_NONE = 0, ICAR_FLUXCOR_MONO = 1 };

typedef enum {
    ICAR_ADV_OK = 0,
    ICAR_ADV_BAD_ARG = 1,        /* invalid size, id, option combination or pointer      */
    ICAR_ADV_OOM = 2,            /* device or pinned host allocation failed              */
    ICAR_ADV_CFL_VIOLATION = 3,  /* debug: a Courant number >= 1; compute_dt: dt < 0.1 s */
    ICAR_ADV_NAN_INPUT = 4,      /* debug option: a non-finite input value was found     */
    ICAR_ADV_TIMEOUT = 5,        /* a bounded device wait gave up                        */
    ICAR_ADV_CUDA_ERROR = 6,     /* a CUDA runtime call failed                           */
    ICAR_ADV_NOT_READY = 7,      /* a field the step needs was never set                 */
    ICAR_ADV_OVER_BUDGET = 8,    /* admission refused: the memory budget would be exceeded */
    ICAR_ADV_PHYSICS_STOP = 9    /* a physics routine met a condition where the reference stops */
} icar_adv_status;

/* Field ids.  Model variables use the reference's kVARS numbering
 * (src/constants/icar_constants.f90:42-110 and the constructor at :310);
 * domain_t members without a kVARS id use 1000+. */
enum {
    ICAR_F_U = 1,
    ICAR_F_V = 2,
    ICAR_F_W = 3,
    ICAR_F_THETA = 7,  /* potential_temperature */
    ICAR_F_QV = 9,     /* water_vapor */
    ICAR_F_QC = 10,    /* cloud_water */
    ICAR_F_NC = 11,    /* cloud_number_concentration */
    ICAR_F_QI = 12,    /* cloud_ice */
    ICAR_F_NI = 13,    /* ice_number_concentration */
    ICAR_F_QR = 14,    /* rain_in_air */
    ICAR_F_NR = 15,    /* rain_number_concentration */
    ICAR_F_QS = 16,    /* snow_in_air */
    ICAR_F_NS = 17,    /* snow_number_concentration */
    ICAR_F_QG = 18,    /* graupel_in_air */
    ICAR_F_NG = 19,    /* graupel_number_concentration */
    ICAR_F_ICE1_A = 20, ICAR_F_ICE1_C = 21, ICAR_F_ICE2_MASS = 22, ICAR_F_ICE2_NUMBER = 23,
    ICAR_F_ICE2_A = 24, ICAR_F_ICE2_C = 25, ICAR_F_ICE3_MASS = 26, ICAR_F_ICE3_NUMBER = 27,
    ICAR_F_ICE3_A = 28, ICAR_F_ICE3_C = 29,
    ICAR_F_PRESSURE = 5,         /* kVARS%pressure (nx, nz, ny), simple microphysics */
    ICAR_F_EXNER = 37,           /* kVARS%exner (nx, nz, ny), simple microphysics */
    ICAR_F_DENSITY = 39,
    ICAR_F_DZ_MASS = 42,         /* kVARS%dz = domain%dz_mass (nx, nz, ny), simple microphysics */
    ICAR_F_DZ_INTERFACE = 43,
    ICAR_F_JACOBIAN = 1001,      /* domain%jacobian   (nx, nz, ny)   */
    ICAR_F_JACOBIAN_U = 1002,    /* domain%jacobian_u (nx+1, nz, ny) */
    ICAR_F_JACOBIAN_V = 1003,    /* domain%jacobian_v (nx, nz, ny+1) */
    ICAR_F_JACOBIAN_W = 1004,    /* domain%jacobian_w (nx, nz, ny)   */
    ICAR_F_ADVECTION_DZ = 1005,  /* domain%advection_dz (nx, nz, ny) */
    ICAR_F_RELAX_FILTER = 1006,  /* domain%relax_filter_2d (nx, 1, ny); set by create, may be overridden */
    ICAR_F_FORCING_BASE = 2000,  /* + species id: forcing_hi%data_3d of that species (nx, nz, ny) */
    ICAR_F_DQDT_BASE = 3000      /* + species id: forcing_hi%dqdt_3d of that species  (nx, nz, ny) */
};

/* Domain description: the index bounds of one single-image domain_t
 * (ims=jms=kms=1, ime=nx, jme=ny, kme=nz) and its advected-variable list in
 * adv_vars order (src/objects/domain_obj.f90:62-89). */
typedef struct {
    int32_t nx, ny, nz;
    float dx;                                  /* domain%dx in metres */
    int32_t n_species;
    int32_t species[ICAR_ADV_MAX_SPECIES];     /* kVARS ids */
    int32_t north_boundary, south_boundary;    /* 1 where the edge is a physical boundary */
    int32_t east_boundary, west_boundary;      /* (all four are 1 for a single image)     */
    int32_t device;                            /* CUDA device ordinal                     */
} icar_adv_desc;

/* Options: the advection subset of options_t, field for field
 * (adv_options_type, src/objects/opt_types.f90:119-127; physics%advection;
 * time_options%RK3; parameters%advect_density and %debug). */
typedef struct {
    int32_t advection;        /* ICAR_ADV_STD or ICAR_ADV_MPDATA                 */
    int32_t mpdata_fct;       /* MPDATA_FCT, default 1                           */
    int32_t mpdata_order;     /* mpdata_order, default 2                         */
    int32_t flux_corr;        /* flux_corr, default 0                            */
    int32_t h_order;          /* h_order 1/3/5, default 1                        */
    int32_t v_order;          /* v_order 1/3/5, default 1                        */
    int32_t rk3;              /* time_options%RK3                                */
    int32_t advect_density;   /* parameters%advect_density                       */
    int32_t debug;            /* parameters%debug: NaN and Courant checks        */
    int32_t boundary_buffer;  /* boundary_buffer (accepted; unused by the path,   */
                              /* as in the reference)                            */
} icar_adv_opts;

typedef struct icar_adv_domain icar_adv_t;
typedef struct icar_adv_batch icar_adv_batch_t;

/* ABI version of the loaded library (ICAR_ADV_ABI_VERSION). */
int icar_adv_abi_version(void);

/* Default options, as adv_parameters_namelist sets them
 * (src/objects/options_obj.f90:1576-1582) with physics%advection = MPDATA. */
int icar_adv_default_opts(icar_adv_opts *opts);

/* adv_var_request(options), src/physics/advection_driver.f90:46-57 ->
 * adv_std_var_request, src/physics/advect.f90:94-108.  Writes the kVARS ids
 * the scheme needs allocated and the ids it marks as advected; *n_* are the
 * capacities on entry and the counts on return. */
int icar_adv_var_request(const icar_adv_opts *opts, int32_t *alloc_vars, int32_t *n_alloc,
                         int32_t *advect_vars, int32_t *n_advect);

/* Halo width the reference derives from the options
 * (src/objects/domain_obj.f90:2979-2986 and grid_obj.f90:153-154). */
int icar_adv_halo_size(const icar_adv_opts *opts);

/* adv_init(domain, options), src/physics/advection_driver.f90:26-44: create a
 * handle, allocate the resident device fields, build the relaxation filter
 * (init_relax_filters, src/objects/domain_obj.f90:3285-3400). */
int icar_adv_create(const icar_adv_desc *desc, const icar_adv_opts *opts, icar_adv_t **out);
/* Release a handle.  Its device memory goes back to a pool the library keeps
 * per device, in the order of the handle's stream (after the work queued
 * there), without waiting for the device; the pool reuses it for later
 * handles and holds it until the process exits. */
int icar_adv_destroy(icar_adv_t *h);

/* Copy one field between the host and the handle's resident device copy.
 * strides: element strides of the (x, z, y) axes of the host array, or NULL
 * for a contiguous Fortran-ordered array.  get_field returns after the data
 * has arrived in host memory. */
int icar_adv_set_field(icar_adv_t *h, int32_t field, const float *host, const int64_t *strides);
int icar_adv_get_field(icar_adv_t *h, int32_t field, float *host, const int64_t *strides);

/* Restarts.  icar_adv_restart_vars gives the field ids the reference lists
 * for advection restarts (options%restart_vars in adv_std_var_request,
 * src/physics/advect.f90:95-107, the same for both schemes): u, v, w,
 * dz_interface, water_vapor; vars may be NULL to ask for the count.
 * icar_adv_download copies n resident fields to host arrays (contiguous
 * Fortran order) with one wait at the end instead of one per field, and
 * icar_adv_upload writes them back -- every species and forcing field, the
 * winds and metric terms, pressure/exner/dz and dz_interface (which the
 * handle keeps only for restarts). */
int icar_adv_restart_vars(const icar_adv_opts *opts, int32_t *vars, int32_t *n);
int icar_adv_download(icar_adv_t *h, int32_t n, const int32_t *fields, float *const *host);
int icar_adv_upload(icar_adv_t *h, int32_t n, const int32_t *fields, const float *const *host);

/* Same with device memory on the handle's device (contiguous Fortran order).
 * Ordered on the handle's stream. */
int icar_adv_set_field_device(icar_adv_t *h, int32_t field, const float *dev);
int icar_adv_get_field_device(icar_adv_t *h, int32_t field, float *dev);

/* advect(domain, options, dt), src/physics/advection_driver.f90:59-126:
 * Courant fluxes from the winds, then every species in adv_vars order.
 * dt in seconds.  Asynchronous on the handle's stream. */
int icar_adv_advect(icar_adv_t *h, float dt);

/* apply_forcing, advected 3-D branch (src/objects/domain_obj.f90:3495-3506)
 * for every species with a forcing field: forcing += dqdt*dt, then the
 * relaxation-zone update.  dt_seconds is the real64 dt%seconds(). */
int icar_adv_apply_forcing(icar_adv_t *h, double dt_seconds);

/* enforce_limits (src/objects/domain_obj.f90:3124-3147): q = max(q, 0) for
 * every resident species. */
int icar_adv_enforce_limits(icar_adv_t *h);

/* One advection time step as time_step.f90:319-389 orders it for these
 * fields: apply_forcing(dt) -> advect(real(dt)) -> enforce_limits if
 * enforce_limits != 0.  Asynchronous on the handle's stream. */
int icar_adv_step(icar_adv_t *h, double dt_seconds, int32_t enforce_limits);

/* The same step for a caller whose species live in host memory, as the
 * reference's advect(domain, options, dt) sees them when CPU physics runs
 * between calls: q_in[s] holds species s (adv_vars order, contiguous
 * Fortran order) before the step, q_out[s] receives it after (q_out[s] may
 * equal q_in[s]).  Equivalent to icar_adv_set_field of every species,
 * icar_adv_step, then icar_adv_get_field of every species, with the same
 * results bit for bit; on the fused kernels the species go in groups (one
 * species each, up to 12 groups) so that the uploads of one group, the
 * step of the previous one and the downloads of the one before overlap
 * (copy streams of their own, which needs page-locked host arrays;
 * pageable ones are copied without overlap).  Returns when q_out is
 * complete. */
int icar_adv_step_host(icar_adv_t *h, double dt_seconds, int32_t enforce_limits, const float *const *q_in,
                       float *const *q_out);

/* balance_uvw(domain, options), src/physics/wind.f90:88-164, called every
 * step before advection when advect_density is set (time_step.f90:324):
 * rebuilds the resident w from the horizontal divergence of the resident u
 * and v (calc_divergence with horz_only, calc_w), density weighted when the
 * handle's advect_density is set.  Columns outside its-1..ite+1 x
 * jts-1..jte+1 get w = 0, as in the reference.  Asynchronous. */
int icar_adv_balance_uvw(icar_adv_t *h);

/* compute_dt(dx, u, v, w, rho, dz, ..., CFL, cfl_strictness, use_density),
 * src/main/time_step.f90:51-168, on the resident winds: the largest stable
 * step for cfl (options%time_options%cfl_reduction_factor) and
 * cfl_strictness 1..5, with dz_levels the host array of nz level
 * thicknesses (options%parameters%dz_levels).  Writes *dt and returns
 * ICAR_ADV_CFL_VIOLATION when dt < 0.1 s (where the reference stops).
 * Synchronises the handle's stream. */
int icar_adv_compute_dt(icar_adv_t *h, const float *dz_levels, float cfl, int32_t cfl_strictness,
                        int32_t use_density, float *dt);

/* mp(domain, options, dt) with physics%microphysics = kMP_SB04:
 * mp_simple_driver, src/physics/mp_simple.f90:595-646, as
 * src/physics/mp_driver.f90:548-568 calls it, on the resident fields:
 * potential temperature, qv, qc, qr and qs must be among the domain's
 * species, and pressure, exner, density and dz (dz_mass) set.  Works on
 * the tile its..ite x jts..jte, every level; the column rain and snow of the
 * call are added to the handle's real64 accumulations (accumulated_
 * precipitation, accumulated_snowfall), which start at zero.  Asynchronous;
 * the next sync reports ICAR_ADV_PHYSICS_STOP if a column met the
 * reference's stop in phase_change. */
int icar_adv_mp_simple(icar_adv_t *h, float dt);
/* Copy the real64 accumulations (nx*ny each, x fastest; either may be
 * NULL) to the host, or set them (NULL = zero).  Synchronous. */
int icar_adv_get_precipitation(icar_adv_t *h, double *rain, double *snow);
int icar_adv_set_precipitation(icar_adv_t *h, const double *rain, const double *snow);

/* Block until the handle's stream has drained; reports device-side errors. */
int icar_adv_sync(icar_adv_t *h);

/* Bounded wait (no reference counterpart; the reference's calls are
 * synchronous): like icar_adv_sync, but gives up after timeout_s seconds
 * and returns ICAR_ADV_TIMEOUT with the work still queued (a later sync
 * can wait for it).  timeout_s = 0 asks whether the work is done. */
int icar_adv_sync_timeout(icar_adv_t *h, double timeout_s);

/* Use an external CUDA stream (cudaStream_t passed as void*; NULL = the
 * handle's own stream).  Work already queued on the previous stream comes
 * first: the new stream waits for it (no host wait).  The stream must stay
 * valid while the handle uses it. */
int icar_adv_set_stream(icar_adv_t *h, void *cuda_stream);

/* Bytes of device memory the handle holds. */
int icar_adv_device_bytes(const icar_adv_t *h, int64_t *bytes);

/* Device memory a handle with this description and these options would
 * hold, without creating it (used for admission by memory footprint). */
int icar_adv_footprint(const icar_adv_desc *desc, const icar_adv_opts *opts, int64_t *bytes);

const char *icar_adv_last_error(const icar_adv_t *h);

/* Diagnostics (no reference counterpart; the reference times advect with
 * timer_t, src/objects/timer_obj.f90).  icar_adv_profile(h, 1) resets the
 * counters and brackets every per-species advection pass with CUDA events;
 * icar_adv_profile_read returns the summed device time of those passes, the
 * kernels they launched, all kernels launched since the reset and the number
 * of passes.  Reading synchronises the handle's stream. */
int icar_adv_profile(icar_adv_t *h, int32_t enable);
int icar_adv_profile_read(icar_adv_t *h, double *species_kernel_ms, int64_t *species_kernel_launches,
                          int64_t *all_launches, int64_t *species_passes);
/* Summed device time and launch count of the fused correction kernel alone
 * (the dominant kernel of the fused MPDATA step) since icar_adv_profile(h, 1). */
int icar_adv_profile_read_correction(icar_adv_t *h, double *ms, int64_t *launches);

/* ---------------------------------------------------------------------------
 * Batched form (no reference counterpart: the reference advances one domain
 * per process).  Many independent domains -- ensemble members or served
 * requests of uneven nx x ny x nz -- advance together: one step is a single
 * CUDA-graph launch holding the boundary update, the per-step wind fields,
 * the donor-cell pass and one correction kernel over a (member, species,
 * tile) work list (two-pass kernels, persistent CTAs), or one single-pass
 * launch over that work list with one CTA per item (icar_adv_batch_set_path
 * 2 or 3).  Each member keeps its own device
 * fields; while it is a member its work runs on the batch's stream, it
 * cannot be stepped on its own, and set/get_field stay available.  All
 * members must use MPDATA order 2 without RK3 and share MPDATA_FCT.
 * A step applies apply_forcing(dt) then advect(real(dt)) to every member,
 * with each member's own dt (icar_adv_step without enforce_limits).
 * ------------------------------------------------------------------------- */
int icar_adv_batch_create(int32_t device, icar_adv_batch_t **out);
int icar_adv_batch_destroy(icar_adv_batch_t *b);
int icar_adv_batch_add(icar_adv_batch_t *b, icar_adv_t *member, double dt_seconds);
int icar_adv_batch_remove(icar_adv_batch_t *b, icar_adv_t *member);
int icar_adv_batch_set_dt(icar_adv_batch_t *b, icar_adv_t *member, double dt_seconds);
int icar_adv_batch_set_tile_shape(icar_adv_batch_t *b, int32_t shape);
int icar_adv_batch_set_species_group(icar_adv_batch_t *b, int32_t group);
int icar_adv_batch_step(icar_adv_batch_t *b);
int icar_adv_batch_sync(icar_adv_batch_t *b);
/* Bounded wait for the batch's steps; ICAR_ADV_TIMEOUT after timeout_s. */
int icar_adv_batch_sync_timeout(icar_adv_batch_t *b, double timeout_s);
int icar_adv_batch_set_stream(icar_adv_batch_t *b, void *cuda_stream);
/* MPDATA kernels of the batch's step (no reference counterpart): 0 = the
 * donor-cell kernel then the fused correction (default), 2 = the single-pass
 * kernel with the reference's FP32 arithmetic (bit-identical results), 3 =
 * the single-pass kernel with fast arithmetic (hardware reciprocal
 * approximation and fused multiply-adds; results within the tolerance
 * stated with icar_adv_set_path). */
int icar_adv_batch_set_path(icar_adv_batch_t *b, int32_t path);
/* Event timing of every step launched while enabled; reading synchronises. */
int icar_adv_batch_profile(icar_adv_batch_t *b, int32_t enable);
int icar_adv_batch_profile_read(icar_adv_batch_t *b, double *step_ms, int64_t *steps, int64_t *kernels_per_step,
                                int64_t *cell_species_per_step);
const char *icar_adv_batch_last_error(const icar_adv_batch_t *b);

/* ---------------------------------------------------------------------------
 * MPDATA step on caller-owned device arrays that allocates nothing.  This
 * entry point has no counterpart in the reference.  It is for callers that
 * cannot call cudaMalloc: code running inside another framework's memory
 * pool or allocator (which must own every device allocation), inside a
 * captured CUDA graph or a stream-ordered region where an allocation would
 * synchronise or break the capture, or under a fixed device-memory budget.
 * The caller passes the inputs and outputs; the library's per-step scratch
 * (Courant fluxes, J*rho, dz*J*rho, W_m/dz and one pass-1 field) comes from a
 * file-scope __device__ array of 4 Mi floats (16 MiB) that every GPU that
 * loads the library holds until the process exits.
 *
 * Limit: the domain must fit that array: 6*round64(P*nz*ny) +
 * round64(P*nz*(ny+1)) <= 4*2^20 floats, with P = round_up(nx+1, 4) and
 * round64 rounding up to a multiple of 64 (about 600 thousand cells, e.g.
 * 128x128x32); larger domains get ICAR_ADV_BAD_ARG with the sizes in the
 * message.  The scheme is advect() with MPDATA order 2 (FCT on or off):
 * every species is read from q_in[s] and the new state written to q_out[s];
 * no boundary update.  No output may overlap any input or another output
 * (the species run one after another, so an overlap would feed updated
 * values into a later species): such calls get ICAR_ADV_BAD_ARG.
 *
 * Device layout of every array: the reference's Fortran order with row pitch
 * P floats, element (i,k,j) at i + P*(k + nz*j); x-face fields (u,
 * jacobian_u) use i <= nx, y-face fields (v, jacobian_v) have ny+1 rows, cell
 * fields i < nx.  Every array must start on a 16-byte boundary (rows are
 * staged with 16-byte copies); a misaligned pointer gets ICAR_ADV_BAD_ARG
 * before anything is launched.  Padding columns are ignored on input and
 * left untouched on output.
 *
 * The first call on a device sets that device up (it looks up the device
 * address of the static array and opts the kernel into its shared memory):
 * make it before any stream capture.  Every call on a device shares the one
 * array, and each call clears the part it uses at its start, so calls whose
 * work overlaps on the GPU (other streams, other host threads) race: order
 * them on one stream or synchronise between them.  Work is enqueued on
 * `stream` (NULL = the legacy default stream); the call returns without
 * waiting. */
typedef struct {
    int32_t nx, ny, nz;
    float dx;                 /* domain%dx in metres       */
    float dt;                 /* seconds                   */
    int32_t mpdata_fct;       /* MPDATA_FCT                */
    int32_t advect_density;   /* parameters%advect_density */
    int32_t n_species;
    const float *u, *v, *w, *density, *jacobian, *jacobian_u, *jacobian_v, *jacobian_w, *advection_dz;
    const float *q_in[ICAR_ADV_MAX_SPECIES];
    float *q_out[ICAR_ADV_MAX_SPECIES];
    void *stream;             /* cudaStream_t */
} icar_adv_noalloc_args;

int icar_adv_advect_noalloc(const icar_adv_noalloc_args *args);

/* Launch shape of the fused MPDATA kernels (no reference counterpart; chosen
 * per grid shape by the autotuner, hicar_b200/autotune.py).  The tile shape
 * selects the output rows per tile of the correction kernel;
 * icar_adv_tile_shapes reports how many shapes exist and the rows of each
 * (rows may be NULL).  The species group is the number of species one thread
 * of the donor-cell pass takes (0 = all, the default; 1..32).  Neither
 * changes any result. */
int icar_adv_set_tile_shape(icar_adv_t *h, int32_t shape);
int icar_adv_set_species_group(icar_adv_t *h, int32_t group);
int icar_adv_tile_shapes(int32_t *n_shapes, int32_t *rows);

/* Kernel selection (no reference counterpart).  MPDATA order 2 without
 * RK3 runs as:
 *   0  the donor-cell kernel then the fused correction kernel (default;
 *      the reference's FP32 arithmetic, bit-identical results);
 *   1  one kernel per reference stage (any mpdata_order; bit-identical);
 *   2  the single-pass kernel (donor-cell pass, pseudo-velocities, limiter
 *      and corrective pass in one launch for every species; bit-identical);
 *   3  the single-pass kernel with fast arithmetic: hardware reciprocal
 *      approximation, fused multiply-adds and reassociated pair sums.  Not
 *      bit-identical; tolerance as tested: max relative error (floor
 *      1e-6 * max|q|) <= 1e-5 after one step and <= 1e-4 after 100 steps on
 *      a smooth tracer, error against an FP64 evaluation within 5x the
 *      reference FP32 arithmetic's own, 99.9 % of cells within 1e-5 of the
 *      FP32 result, and mass conserved to 2e-6.
 * Other schemes and orders ignore 2 and 3 (the standard scheme always runs
 * its fused kernels on 0, 2 and 3). */
int icar_adv_set_path(icar_adv_t *h, int32_t path);

#ifdef __cplusplus
}
#endif

#endif /* ICAR_ADV_H */
