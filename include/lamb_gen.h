/*
 * lamb_gen.h -- synthetic water-box matrices in LAMB's single-rank sector
 * layout.  This is input staging, not part of the multiply: it plays the
 * role of the reference's matrix builders (lamb_matrix_X_create_random /
 * fill_sector, src/lamb_matrix_X_tests.F90:89-250, and lamb_load_dbcsr +
 * fill_local_sectors, src/lamb_io_operations.F90:267-756,
 * src/lamb_matrix_operations.F90:294-375) for geometries that the reference
 * does not ship.
 *
 * Geometry: n_mol rigid waters (O-H 0.96 A, H-O-H 104.5 deg) placed by random
 * sequential insertion with a minimum O-O distance in a periodic cubic box.
 * Atom order is molecule-major (O, H, H).  Block (i,j) is present iff the
 * minimum-image distance r_ij < cutoff (a single image per pair).
 * Values: element (p,q) of block (i,j) is u(seed,i,j,p,q)*exp(-r_ij/decay)
 * with u uniform in [-1,1) from a counter-based hash; diagonal blocks are
 * (X+X^T)/2 + I; with symmetric != 0 every block satisfies X_ji = X_ij^T.
 *
 * Sector layout at one rank: LAMB partitions space into n_cubes = 2 cubes
 * along x (src/lamb_plexus_operations.F90:115-126,
 * src/lamb_partition_operations.F90:62-108); atom subset =
 * 1 + mod(int(x*multiplier), 2) computed in float32 with multiplier =
 * 2/h11 (src/lamb_partition_methods.F90:85-96, src/lamb_partition_types.F90:139-143);
 * the local index is the running count in global order
 * (src/lamb_set_partition_methods.F90:69-144).  Sectors come in
 * (1,1),(1,2),(2,1),(2,2) order (fill_my_sectors,
 * src/lamb_plexus_operations.F90:454-488); blocks of a sector are stored
 * contiguously in row-major (row, col) order as fill_sector does.
 */
#ifndef LAMB_GEN_H
#define LAMB_GEN_H
#include <stdint.h>
#include "lamb_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lamb_gen_geom lamb_gen_geom;
typedef struct lamb_gen_matrix lamb_gen_matrix;

/* Returns 0 on success; the error text is available via lamb_gen_last_error(). */
LAMB_API int32_t lamb_gen_water_geometry(int32_t n_mol, double box, double cutoff, int32_t blk_o, int32_t blk_h,
                                uint64_t seed, double min_oo, int32_t n_x_cubes, lamb_gen_geom** geom);
LAMB_API int32_t lamb_gen_geom_free(lamb_gen_geom* geom);
LAMB_API int32_t lamb_gen_geom_n_atoms(const lamb_gen_geom* geom);
LAMB_API int64_t lamb_gen_geom_n_pairs(const lamb_gen_geom* geom);
/* positions[3*n_atoms] (x,y,z per atom, wrapped into [0,box)), blk[n_atoms], subset[n_atoms] (1-based). */
LAMB_API int32_t lamb_gen_geom_atoms(const lamb_gen_geom* geom, double* positions, int8_t* blk, int32_t* subset,
                            int32_t* local);

LAMB_API int32_t lamb_gen_water_matrix(const lamb_gen_geom* geom, uint64_t seed, double decay, int32_t symmetric,
                              lamb_gen_matrix** mat);
LAMB_API int32_t lamb_gen_matrix_free(lamb_gen_matrix* mat);
LAMB_API int32_t lamb_gen_matrix_n_sectors(const lamb_gen_matrix* mat);
/* Pointers stay valid until lamb_gen_matrix_free. */
LAMB_API int32_t lamb_gen_matrix_sector(const lamb_gen_matrix* mat, int32_t s, lamb_c_sector* out);
LAMB_API const char* lamb_gen_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
