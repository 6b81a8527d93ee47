/* Plain-C consumer of the drop-in boundary.  Compiled as C99 against
 * include/icar_adv.h and linked to libicar_adv.so, it calls the host-only
 * entry points (no device work) the way a Fortran shim bound through
 * ISO_C_BINDING does: option defaults, the variable request, the halo rule,
 * the footprint with its validation, and NULL-handle errors.  Prints "ok"
 * and exits 0, or exits with the number of the first failed check. */
#include <stdio.h>
#include <string.h>

#include "icar_adv.h"

#define CHECK(n, cond)                                  \
    do {                                                \
        if (!(cond)) {                                  \
            fprintf(stderr, "check %d failed\n", (n));  \
            return (n);                                 \
        }                                               \
    } while (0)

int main(void)
{
    icar_adv_opts o;
    icar_adv_desc d;
    int32_t alloc_ids[64], adv_ids[64], n_alloc = 64, n_adv = 64, n_restart = 0, n_shapes = 0, rows[16];
    int64_t bytes = 0;
    int32_t i, has_qv = 0;

    CHECK(1, icar_adv_abi_version() == ICAR_ADV_ABI_VERSION);
    CHECK(2, icar_adv_default_opts(&o) == ICAR_ADV_OK);
    CHECK(3, o.advection == ICAR_ADV_MPDATA && o.mpdata_fct == 1 && o.mpdata_order == 2 && o.h_order == 1);
    CHECK(4, icar_adv_halo_size(&o) == 2);

    CHECK(5, icar_adv_var_request(&o, alloc_ids, &n_alloc, adv_ids, &n_adv) == ICAR_ADV_OK);
    CHECK(6, n_adv == 2 && adv_ids[0] == ICAR_F_QV && adv_ids[1] == ICAR_F_THETA);
    for (i = 0; i < n_alloc; i++) has_qv |= alloc_ids[i] == ICAR_F_QV;
    CHECK(7, has_qv);
    CHECK(8, icar_adv_restart_vars(&o, NULL, &n_restart) == ICAR_ADV_OK && n_restart == 5);

    memset(&d, 0, sizeof d);
    d.nx = 64;
    d.ny = 48;
    d.nz = 20;
    d.dx = 1000.0f;
    d.n_species = 2;
    d.species[0] = ICAR_F_QV;
    d.species[1] = ICAR_F_QC;
    d.north_boundary = d.south_boundary = d.east_boundary = d.west_boundary = 1;
    CHECK(9, icar_adv_footprint(&d, &o, &bytes) == ICAR_ADV_OK && bytes > (int64_t)4 * 64 * 48 * 20 * 10);
    d.nz = 2;
    CHECK(10, icar_adv_footprint(&d, &o, &bytes) == ICAR_ADV_BAD_ARG);
    CHECK(11, strstr(icar_adv_last_error(NULL), "too small") != NULL);

    CHECK(12, icar_adv_step(NULL, 4.0, 0) == ICAR_ADV_BAD_ARG);
    CHECK(13, icar_adv_advect(NULL, 4.0f) == ICAR_ADV_BAD_ARG);
    CHECK(14, icar_adv_destroy(NULL) == ICAR_ADV_OK);

    CHECK(15, icar_adv_tile_shapes(&n_shapes, NULL) == ICAR_ADV_OK && n_shapes >= 1 && n_shapes <= 16);
    CHECK(16, icar_adv_tile_shapes(&n_shapes, rows) == ICAR_ADV_OK && rows[0] > 0);

    printf("ok\n");
    return 0;
}
