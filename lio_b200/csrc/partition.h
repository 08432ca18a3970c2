// Grid generation and partition into cubes/spheres (host, FP64, bit-exact with
// the reference's g2g/regenerate_partition.cpp:161-481, classify_functions.cpp
// and cpu/weight.cpp).
#pragma once
#include <cstdint>
#include <vector>

#include "system.h"

namespace lio {

struct GridPoint {
  int atom, shell, point;
  double x, y, z, w;
  // no zeroing when a point array is sized before it is filled (the grid build
  // places every point of a geometry, ~140 MB at 256 atoms, into sized arrays)
  GridPoint() {}
  GridPoint(int a, int s, int p, double x_, double y_, double z_, double w_)
      : atom(a), shell(s), point(p), x(x_), y(y_), z(z_), w(w_) {}
};

struct PointGroup {
  bool sphere = false;
  std::vector<GridPoint> points;
  std::vector<int> funcs;  // simple functions: global index of the first component
  std::vector<int> nucs;   // sorted global nuclei of the significant functions
  int s = 0, p = 0, d = 0;
  int total_functions() const { return s + 3 * p + 6 * d; }
  long long cost(long long mincost) const {  // g2g/partition.cpp:257-260
    long long np = (long long)points.size(), gm = total_functions();
    return 10 * ((np * gm * (1 + gm)) / 2) + mincost;
  }
};

struct Partition {
  std::vector<PointGroup> cubes, spheres;  // each sorted by cost
  long long mincost = 250000;
  int total_groups() const { return (int)(cubes.size() + spheres.size()); }
  const PointGroup& group(int g) const {
    return g < (int)cubes.size() ? cubes[g] : spheres[g - cubes.size()];
  }
};

// Becke weights of many groups at once (g2g/cpu/weight.cpp:13-112): every
// point's weight is multiplied by its atom's fuzzy-cell weight, restricted to
// the group's nuclei, bit for bit as the reference computes it. With
// `drop_zero` the points whose weight is then 0 are removed, keeping the order
// of the others (g2g/cpu/weight.cpp:100-111), in the same pass.
using WeightsFn = void (*)(const System& sys, const std::vector<PointGroup*>& groups, bool drop_zero);
// host implementation (OpenMP over each group's points)
void host_becke_weights(const System& sys, const std::vector<PointGroup*>& groups, bool drop_zero);
// the atomic-size adjustment of every atom pair (j, k), out[j * natoms + k],
// by the operations the host weights use (compiled without FMA contraction)
void becke_pair_table(const System& sys, double* out);

// Builds the partition. `grid_type` selects the radial shell table (0: Nr,
// otherwise Nr2) exactly as g2g/init.cpp:238-266 does. The Becke weights of all
// candidate groups are computed in one call of `weights` (default: the host
// implementation); zero-weight removal and the minimum-size filter follow, in
// the reference's group order.
void build_partition(const System& sys, const Options& opt, const AngularGrid& ang,
                     int grid_type, Partition& out, WeightsFn weights = nullptr);

}  // namespace lio
