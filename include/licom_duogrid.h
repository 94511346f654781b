/*
 * licom_duogrid.h - C-ABI of the cubed-sphere duogrid geometry generator.
 *
 * This is the input pipeline of the barotropic path: it produces the geometry
 * constants (rdx, rdy, rda, c_dy, d_dx, a_gct, a_sina, a_f, a_c2l, a_l2c,
 * k2e_coef, k2e_loc_i/j, a_pt, ...) that the reference obtains from its Fortran
 * library `libduogrid_coordinate` through ctypes and serialises to
 * `field/duogrid_C{nx}.npz`.
 *
 * Replaces (reference interface, path within the reference project):
 *   chtholly_global_grid_init / _end      src/duogrid_c/chtholly/chtholly_get_global_grid.F90:57-74
 *   chtholly_global_grid_get_*            src/duogrid_c/chtholly/chtholly_get_global_grid.F90:75-322
 *   ctypes bindings init_with_mp / end /
 *   get_all_a_grid / get_all_bc_d_grid    src/initial_field/_c_duogrid_function.py:207-307
 *   transpose + truncation + stacking     src/initial_field/main.py:57-142
 *
 * Unlike the reference (one Fortran call per tile, Fortran-ordered output that
 * Python transposes and truncates), one ldg_create() builds all six tiles and
 * every getter writes the final C-ordered layout the solver consumes:
 *   2-D fields   (6, M, M)        M = res + 6 (3-cell halo on each side)
 *   a_pt, b_pt,
 *   k2e_coef     (6, M, M, 2)
 *   2x2 matrices (6, M, M, 2, 2)  element [t,i,j,a,b] = Fortran (a+1,b+1,i,j)
 * Axis -2 is the Fortran i index, axis -1 the Fortran j index; python index
 * ii corresponds to Fortran i = ii - 2.
 *
 * All functions return 0 on success and a negative code on failure; the
 * message is available from ldg_last_error() (thread-local).
 */
#ifndef LICOM_DUOGRID_H
#define LICOM_DUOGRID_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ldg_grid ldg_grid;

#define LDG_OK 0
#define LDG_EINVAL -1
#define LDG_ENOMEM -2
#define LDG_ENOFIELD -3

/* Build the equal-edge (grid_type 0) duogrid at resolution res (res >= 6),
 * halo ng = 3, all six tiles.  Replaces chtholly_global_grid_init with
 * isd = jsd = -2, ied = jed = res + 3 (src/initial_field/main.py:54-55,105-109). */
int ldg_create(int res, ldg_grid** out);

/* Release a grid (replaces chtholly_global_grid_end). */
void ldg_destroy(ldg_grid* g);

/* Shape of a named field: writes ndim and shape[0..ndim-1]. */
int ldg_field_shape(const ldg_grid* g, const char* name, int* ndim, long* shape);

/* Number of exported field names and the i-th name (static storage). */
int ldg_num_fields(void);
const char* ldg_field_name(int i);

/* 1 if the named field is an int32 field (k2e_loc, k2e_loc_i, k2e_loc_j). */
int ldg_field_is_int(const char* name);

/* Copy a float64 field into out (C order, size from ldg_field_shape). */
int ldg_get_f64(const ldg_grid* g, const char* name, double* out);

/* Copy an int32 field into out (k2e_loc, k2e_loc_i, k2e_loc_j). */
int ldg_get_i32(const ldg_grid* g, const char* name, int* out);

const char* ldg_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* LICOM_DUOGRID_H */
