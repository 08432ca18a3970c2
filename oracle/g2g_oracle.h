/* Test infrastructure only: the oracle. Never linked into the product library.
 *
 * CPU FP64 restatement of the reference's XC grid integration (LIO g2g, CPU
 * path, precision=1): grid generation and cube/sphere partition
 * (g2g/regenerate_partition.cpp:161-481), function screening
 * (g2g/classify_functions.cpp, g2g/partition.cpp:230-254), Becke weights
 * (g2g/cpu/weight.cpp), basis values (g2g/cpu/functions.cpp), the density
 * loops, functionals and Kohn-Sham accumulation (g2g/cpu/iteration.cpp,
 * g2g/pointxc headers). It exists for grids the compiled reference cannot run (the
 * 302-point angular table; the reference's table sizes are compile-time,
 * g2g/init.h:10-14) and is itself checked bit for bit (partition) and to
 * 1e-10 (E_xc, K) against the reference on the 194-point grid.
 */
#ifndef G2G_ORACLE_H
#define G2G_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int natoms;
  const double *x, *y, *z;     /* bohr */
  const int* Z;                /* atomic numbers */
  const double* rm_by_Z;       /* Rm indexed by Z */
  const unsigned* shells_by_Z; /* radial shells indexed by Z (Nr or Nr2) */
  int M;                       /* expanded functions */
  const int* nuc;              /* 0-based atom of each expanded function */
  const int* ncont;
  const double *a, *c;         /* M x 13 row-major */
  int s_funcs, p_funcs, d_funcs; /* simple counts */
  int normalize;
  int nang;
  const double *ex, *ey, *ez, *ew;
  double little_cube_size, sphere_radius;
  unsigned max_function_exponent, min_points_per_cube;
  int assign_all_functions, remove_zero_weights;
  long long mincost;
  int iexch, open;
} oracle_system;

/* Partition + one XC build. fock/fockb are accumulated (+=); *energy written.
 * Returns 0, or a negative code on invalid input. npoints/ngroups optional. */
int oracle_solve(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b,
                 double* fock, double* fockb, double* energy, long long* npoints, long long* ngroups);

/* Same, restricted to every `stride`-th group starting at `first` (a bounded
 * sample for CPU timing); counts only the points of the processed groups. */
int oracle_solve_sample(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b,
                        double* fock, double* fockb, double* energy, long long* npoints, long long* ngroups,
                        int first, int stride);

/* Same, restricted to the listed groups (indices in the partition's order:
 * cubes, then spheres, each sorted by cost); for checking a sharded build. */
int oracle_solve_subset(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b,
                        double* fock, double* fockb, double* energy, long long* npoints, long long* ngroups,
                        const int* group_ids, int nids);

/* Partition + XC forces (g2g_solve_groups_ types 2/3): each atom's XC force
 * added into forces (natoms x 3 column-major, leading dimension natoms),
 * *energy written, no Kohn-Sham contributions. */
int oracle_solve_forces(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b,
                        double* forces, double* energy, long long* npoints, long long* ngroups);

#ifdef __cplusplus
}
#endif
#endif
