/*
 * CPU oracle for the ICAR tracer-advection step.
 *
 * TEST INFRASTRUCTURE ONLY: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library, and
 * only as the checker or the timed CPU baseline.  The product path
 * (libicar_adv.so) never links, loads or calls it.
 *
 * No Fortran compiler exists in the build image, so the reference sources
 * cannot be compiled; this file restates them in plain C:
 *   src/physics/advection_driver.f90:59-126      advect
 *   src/physics/adv_mpdata.f90:23-504             MPDATA
 *   src/physics/adv_mpdata_FCT_core.f90:47-116    FCT core
 *   src/physics/advect.f90:134-320,447-493        standard (upwind / 3rd / 5th)
 *   src/physics/adv_fluxcorr.f90:37-192           WRF monotonic flux correction
 *   src/objects/domain_obj.f90:3092-3149          enforce_limits
 *   src/objects/domain_obj.f90:3285-3400          init_relax_filters
 *   src/objects/domain_obj.f90:3457-3526          apply_forcing (advected part)
 *   src/physics/wind.f90:88-271                   balance_uvw, calc_w, calc_divergence
 *   src/main/time_step.f90:51-168                 compute_dt
 *   src/physics/mp_simple.f90:146-646             simple microphysics (SB04)
 *   src/physics/mp_driver.f90:477-481,548-568,741-749  its driver call and accumulation
 * The reference has no golden vectors for this path (its only MPDATA test,
 * src/tests/test_mpdata.f90, is print-only and disabled), so parity of this
 * restatement is pinned by the known-answer properties in
 * tests/test_oracle.py, not by reference outputs: "parity unpinned" by the
 * reference's own tests.
 *
 * Built twice into one shared object: *_f32 (the reference's real) and
 * *_f64 (the same scheme in double, for error reporting).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int advection;      /* 1 = kADV_STD, 2 = kADV_MPDATA (icar_constants.f90:419-420) */
    int mpdata_fct;     /* adv_options%MPDATA_FCT */
    int mpdata_order;   /* adv_options%mpdata_order */
    int flux_corr;      /* adv_options%flux_corr (1 = kFLUXCOR_MONO) */
    int h_order;        /* adv_options%h_order */
    int v_order;        /* adv_options%v_order */
    int rk3;            /* time_options%RK3 */
    int advect_density; /* parameters%advect_density */
    int halo;           /* grid%halo_size used for its/ite (grid_obj.f90:246-249) */
} oracle_opts;

#define REAL float
#define FN(x) x##_f32
#define EPS10 1e-10f
#define EPS15 1e-15f
#define RK3_THIRD 0.333f
#define RABS(a) fabsf(a)
#define RSQRT3 sqrtf(3.0f)
#define REXP(x) ((float)exp((double)(x)))  /* correctly rounded expf, see mp_simple below */
#include "oracle_body.inc"
#undef REAL
#undef FN
#undef EPS10
#undef EPS15
#undef RK3_THIRD
#undef RABS
#undef RSQRT3
#undef REXP
#undef C3
#undef UX

#define REAL double
#define FN(x) x##_f64
#define EPS10 1e-10
#define EPS15 1e-15
#define RK3_THIRD 0.333
#define RABS(a) fabs(a)
#define RSQRT3 sqrt(3.0)
#define REXP(x) exp(x)
#include "oracle_body.inc"
#undef REAL
#undef FN

/* ------------------------------------------------------------------------
 * init_relax_filters, src/objects/domain_obj.f90:3285-3400 (2-D filter only;
 * the 3-D copy is the same value on every level).  Boundary flags say which
 * edges of this image are physical; a single image has all four, so the
 * north+west corner branch applies.  filter is nx*ny, x fastest.
 * ------------------------------------------------------------------------ */
void init_relax_filters(int nx, int ny, int hs, int north, int south, int east, int west, float *filter)
{
    const float rs[7] = {0.9f, 0.75f, 0.6f, 0.5f, 0.4f, 0.25f, 0.1f};
    const float rs_r[7] = {0.1f, 0.25f, 0.4f, 0.5f, 0.6f, 0.75f, 0.9f};
    const int ims = 1, ime = nx, jms = 1, jme = ny;
    int corner = (west || east) && (north || south);
    int nr = 7;
    if (ime - ims - hs < nr) nr = ime - ims - hs;
    if (jme - jms - hs < nr) nr = jme - jms - hs;
#define SET(i, j, val)                                                                  \
    do {                                                                                \
        int ii_ = (i), jj_ = (j);                                                       \
        if (ii_ >= 1 && ii_ <= nx && jj_ >= 1 && jj_ <= ny)                             \
            filter[(size_t)(ii_ - 1) + (size_t)nx * (size_t)(jj_ - 1)] = (val);         \
    } while (0)
    for (size_t c = 0; c < (size_t)nx * ny; c++) filter[c] = 0.0f;
    if (!corner) {
        if (west) {
            for (int j = jms; j <= jme; j++)
                for (int i = ims; i <= ims + hs - 1; i++) SET(i, j, 1.0f);
            for (int k = jms; k <= jme; k++)
                for (int m = 1; m <= nr; m++) SET(ims + hs + m - 1, k, rs[m - 1]);
        } else if (east) {
            for (int j = jms; j <= jme; j++)
                for (int i = ime - hs + 1; i <= ime; i++) SET(i, j, 1.0f);
            for (int k = jms; k <= jme; k++)
                for (int m = 1; m <= nr; m++) SET(ime - hs - nr + m, k, rs_r[m - 1]);
        } else if (north) {
            for (int j = jme - hs - 1; j <= jme; j++)
                for (int i = ims; i <= ime; i++) SET(i, j, 1.0f);
            for (int k = ims; k <= ime; k++)
                for (int m = 1; m <= nr; m++) SET(k, jme - hs - nr + m, rs_r[m - 1]);
        } else if (south) {
            for (int j = jms; j <= jms + hs - 1; j++)
                for (int i = ims; i <= ime; i++) SET(i, j, 1.0f);
            for (int k = ims; k <= ime; k++)
                for (int m = 1; m <= nr; m++) SET(k, jms + hs + m - 1, rs[m - 1]);
        }
    } else {
        if (north && west) {
            for (int j = jms; j <= jme; j++)
                for (int i = ims; i <= ims + hs - 1; i++) SET(i, j, 1.0f);
            for (int j = jme - hs - 1; j <= jme; j++)
                for (int i = ims; i <= ime; i++) SET(i, j, 1.0f);
            for (int k = jms; k <= jme - hs; k++)
                for (int m = 1; m <= nr; m++) SET(ims + hs + m - 1, k, rs[m - 1]);
            for (int k = ims + hs; k <= ime; k++)
                for (int m = 1; m <= nr; m++) SET(k, jme - hs - nr + m, rs_r[m - 1]);
            for (int i = 1; i <= nr; i++)
                for (int k = 1; k <= nr; k++) SET(ims + hs + i - 1, jme - hs - k + 1, rs[(i < k ? i : k) - 1]);
        } else if (north && east) {
            for (int j = jms; j <= jme; j++)
                for (int i = ime - hs + 1; i <= ime; i++) SET(i, j, 1.0f);
            for (int j = jme - hs - 1; j <= jme; j++)
                for (int i = ims; i <= ime; i++) SET(i, j, 1.0f);
            for (int k = jms; k <= jme - hs; k++)
                for (int m = 1; m <= nr; m++) SET(ime - hs - nr + m, k, rs_r[m - 1]);
            for (int k = ims; k <= ime - hs; k++)
                for (int m = 1; m <= nr; m++) SET(k, jme - hs - nr + m, rs_r[m - 1]);
            for (int i = 1; i <= nr; i++)
                for (int k = 1; k <= nr; k++) SET(ime - hs - i + 1, jme - hs - k + 1, rs[(i < k ? i : k) - 1]);
        } else if (south && west) {
            for (int j = jms; j <= jme; j++)
                for (int i = ims; i <= ims + hs - 1; i++) SET(i, j, 1.0f);
            for (int j = jms; j <= jms + hs - 1; j++)
                for (int i = ims; i <= ime; i++) SET(i, j, 1.0f);
            for (int k = jms + hs; k <= jme; k++)
                for (int m = 1; m <= nr; m++) SET(ims + hs + m - 1, k, rs[m - 1]);
            for (int k = ims + hs; k <= ime; k++)
                for (int m = 1; m <= nr; m++) SET(k, jms + hs + m - 1, rs[m - 1]);
            for (int i = 1; i <= nr; i++)
                for (int k = 1; k <= nr; k++) SET(ims + hs + i - 1, jms + hs + k - 1, rs[(i < k ? i : k) - 1]);
        } else if (south && east) {
            for (int j = jms; j <= jme; j++)
                for (int i = ime - hs + 1; i <= ime; i++) SET(i, j, 1.0f);
            for (int j = jms; j <= jms + hs - 1; j++)
                for (int i = ims; i <= ime; i++) SET(i, j, 1.0f);
            for (int k = jms + hs; k <= jme; k++)
                for (int m = 1; m <= nr; m++) SET(ime - hs - nr + m, k, rs_r[m - 1]);
            for (int k = ims; k <= ime - hs; k++)
                for (int m = 1; m <= nr; m++) SET(k, jms + hs + m - 1, rs[m - 1]);
            for (int i = 1; i <= nr; i++)
                for (int k = 1; k <= nr; k++) SET(ime - hs - i + 1, jms + hs + k - 1, rs[(i < k ? i : k) - 1]);
        }
    }
#undef SET
}
