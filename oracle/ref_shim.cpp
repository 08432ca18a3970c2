// Test infrastructure only (the oracle). Never linked into the product library.
//
// Plain-C accessors compiled against the reference g2g headers and linked into
// oracle/_ref/libg2g_ref.so next to the reference's own CPU sources. They walk
// the reference's process-global partition (the `::partition` object that
// g2g/init.cpp:27 declares and g2g_solve_groups_ drives) so the tests can
// compare the grid partition point by point, and they expose the reference's
// solve timing for the CPU baseline.
//
// Group numbering: cubes first (in the reference's cost-sorted order), then
// spheres, i.e. the same `ind` convention g2g/partition.cpp:478-484 uses.
#include <cstring>
#include <vector>
#include "common.h"
#include "init.h"
#include "partition.h"

extern G2G::Partition partition;

namespace {
G2G::PointGroup<double>* group_at(int g) {
  const int nc = (int)partition.cubes.size();
  if (g < 0) return nullptr;
  if (g < nc) return partition.cubes[g];
  const int ns = (int)partition.spheres.size();
  if (g < nc + ns) return partition.spheres[g - nc];
  return nullptr;
}
}  // namespace

extern "C" {

int ref_num_cubes(void) { return (int)partition.cubes.size(); }
int ref_num_spheres(void) { return (int)partition.spheres.size(); }

// meta[0]=npoints meta[1]=nfuncs_simple meta[2]=s meta[3]=p meta[4]=d
// meta[5]=total_functions meta[6]=nucleii meta[7]=is_sphere
int ref_group_meta(int g, int* meta) {
  G2G::PointGroup<double>* pg = group_at(g);
  if (!pg) return -1;
  meta[0] = (int)pg->number_of_points;
  meta[1] = (int)pg->total_functions_simple();
  meta[2] = (int)pg->s_functions;
  meta[3] = (int)pg->p_functions;
  meta[4] = (int)pg->d_functions;
  meta[5] = (int)pg->total_functions();
  meta[6] = (int)pg->total_nucleii();
  meta[7] = g >= (int)partition.cubes.size() ? 1 : 0;
  return 0;
}

// ids: npoints x 3 ints (atom, shell, point); xyzw: npoints x 4 doubles.
int ref_group_points(int g, int* ids, double* xyzw) {
  G2G::PointGroup<double>* pg = group_at(g);
  if (!pg) return -1;
  for (size_t i = 0; i < pg->points.size(); i++) {
    const G2G::Point& p = pg->points[i];
    ids[3 * i + 0] = (int)p.atom;
    ids[3 * i + 1] = (int)p.shell;
    ids[3 * i + 2] = (int)p.point;
    xyzw[4 * i + 0] = p.position.x;
    xyzw[4 * i + 1] = p.position.y;
    xyzw[4 * i + 2] = p.position.z;
    xyzw[4 * i + 3] = p.weight;
  }
  return 0;
}

// funcs: nfuncs_simple global function indices (0-based, first component);
// nucs: nucleii global atom indices (0-based).
int ref_group_lists(int g, int* funcs, int* nucs) {
  G2G::PointGroup<double>* pg = group_at(g);
  if (!pg) return -1;
  for (size_t i = 0; i < pg->local2global_func.size(); i++)
    funcs[i] = (int)pg->local2global_func[i];
  for (size_t i = 0; i < pg->local2global_nuc.size(); i++)
    nucs[i] = (int)pg->local2global_nuc[i];
  return 0;
}

long long ref_group_cost(int g) {
  G2G::PointGroup<double>* pg = group_at(g);
  return pg ? pg->cost() : -1;
}

int ref_cpu_threads(void) { return G2G::cpu_threads; }

// atoms the reference's g2g_parameter_init_ recorded (the state its analytic
// integrals read), for the link test of the drop-in
int ref_bound_atoms(void) { return (int)G2G::fortran_vars.atoms; }
}
