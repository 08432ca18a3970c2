// Host-side description of one molecule + basis + options, as bound through the
// g2g C ABI (g2g/init.h:16-52 holds the reference's equivalent FortranVars).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace lio {

constexpr int kMaxContractions = 13;  // g2g/common.h:14

struct Options {  // g2g/init.cpp:395-404 defaults
  unsigned max_function_exponent = 10;
  double little_cube_size = 8.0;
  unsigned min_points_per_cube = 1;
  bool assign_all_functions = false;
  double sphere_radius = 0.6;
  bool remove_zero_weights = true;
  bool energy_all_iterations = false;
  double free_global_memory = 0.0;
  unsigned timer_level = 0;
  unsigned verbose = 0;
};

struct AngularGrid {
  std::vector<double> x, y, z, w;  // unit directions and weights (sum 4*pi)
  int size() const { return (int)w.size(); }
};

// One contracted Cartesian function shell as the grid and the device see it.
struct System {
  int natoms = 0;
  std::vector<double> ax, ay, az;       // atom positions (bohr)
  std::vector<int> atom_type;           // Iz - 1
  std::vector<unsigned> shells_grid0;   // Nr[Iz]
  std::vector<unsigned> shells_grid12;  // Nr2[Iz]
  std::vector<double> rm;               // Rm[Iz]
  std::vector<double> atom_dist;        // natoms x natoms, |Ri - Rj|

  int M = 0;                 // total (expanded) functions
  int s_funcs = 0, p_funcs = 0, d_funcs = 0;  // simple counts
  // shell type of every (expanded) function (0 s, 1 p, 2 d); empty: from the
  // counts above (all s, then p, then d). A batch of molecules joined into one
  // system keeps each molecule's own order, so it sets these explicitly.
  std::vector<int8_t> ftype;
  std::vector<int> nuc;      // per expanded function, 0-based atom
  std::vector<int> ncont;    // per expanded function
  std::vector<double> a, c;  // per expanded function x kMaxContractions (row-major)
  double d_norm = 1.0;       // 1/sqrt(3) when normalised d functions

  int iexch = 9;
  bool lda = false;
  bool open = false;
};

}  // namespace lio
