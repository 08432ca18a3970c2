// Grid generation, significant-function screening and Becke weights.
//
// Every floating-point expression below keeps the operand order of the
// reference so that points, weights and function lists come out bit-for-bit
// equal (this file is compiled with -ffp-contract=off and no -march, so no
// fused multiply-add is formed). The reference steps each function follows are
// cited inline.
#include "partition.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <set>
#include <stdexcept>

namespace lio {
namespace {

inline double len3(double x, double y, double z) { return std::sqrt(x * x + y * y + z * z); }

// The significance test of g2g/partition.cpp:230-254 (is_significative), split into its part that
// depends on the function alone (computed once per function) and the comparison
// with the squared distance (per cube or sphere): s functions compare
// exponent * d2 with a bound, p and d functions sqrt(d2) with a radius found by
// fixed-point iteration. Same expressions, so the same bits as calling
// is_significative per group.
struct Screen {
  std::vector<double> bound;  // per function index f (first component): s bound or p/d radius
};
Screen make_screen(const System& sys, const Options& opt, const std::vector<double>& min_exps) {
  Screen sc;
  sc.bound.assign(sys.M, 0.0);
  const unsigned mfe = opt.max_function_exponent;
  const int s_end = sys.s_funcs, p_end = sys.s_funcs + sys.p_funcs * 3,
            d_end = sys.s_funcs + sys.p_funcs * 3 + sys.d_funcs * 6;
  for (int f = 0; f < d_end; f += (f < s_end ? 1 : (f < p_end ? 3 : 6))) {
    const double exponent = min_exps[f];
    if (f < s_end) {
      sc.bound[f] = mfe - std::log(std::pow((2. * exponent / M_PI), 3)) / 4;
      continue;
    }
    const int type = f < p_end ? 3 : 6;
    double x = 1;
    double delta;
    const double e = 0.1;
    double factor = std::pow((2.0 * exponent / M_PI), 3);
    factor = std::sqrt(factor * 4.0 * exponent);
    double norm = (type == 3 ? std::sqrt(factor) : std::fabs(factor));
    do {
      double div = (type == 3 ? std::log(x) : 2 * std::log(x));
      double x1 = std::sqrt((mfe - std::log(norm) + div) / exponent);
      delta = std::fabs(x - x1);
      x = x1;
    } while (delta > e);
    sc.bound[f] = x;
  }
  return sc;
}

// g2g/classify_functions.cpp:13-65: walks s, then p (stride 3), then d (stride 6).
void assign_functions(const System& sys, const Options& opt, const std::vector<double>& dists,
                      const std::vector<double>& min_exps, const Screen& sc, PointGroup& g) {
  std::set<int> nuc_set;
  g.funcs.clear();
  int f = 0;
  const int s_end = sys.s_funcs, p_end = sys.s_funcs + sys.p_funcs * 3,
            d_end = sys.s_funcs + sys.p_funcs * 3 + sys.d_funcs * 6;
  for (; f < s_end; f++) {
    int atom = sys.nuc[f];
    if (opt.assign_all_functions || min_exps[f] * dists[atom] < sc.bound[f]) {
      g.funcs.push_back(f);
      g.s++;
      nuc_set.insert(atom);
    }
  }
  for (; f < p_end; f += 3) {
    int atom = sys.nuc[f];
    if (opt.assign_all_functions || std::sqrt(dists[atom]) < sc.bound[f]) {
      g.funcs.push_back(f);
      g.p++;
      nuc_set.insert(atom);
    }
  }
  for (; f < d_end; f += 6) {
    int atom = sys.nuc[f];
    if (opt.assign_all_functions || std::sqrt(dists[atom]) < sc.bound[f]) {
      g.funcs.push_back(f);
      g.d++;
      nuc_set.insert(atom);
    }
  }
  g.nucs.assign(nuc_set.begin(), nuc_set.end());
}

// Becke fuzzy-cell partition with the atomic-size adjustment, restricted to the
// group's nuclei: g2g/cpu/weight.cpp:13-112.
// the size adjustment a_jk of the pair (g2g/cpu/weight.cpp:40-44)
inline double becke_adjust(double rm_j, double rm_k) {
  double x = rm_j / rm_k;
  x = (x - 1.0) / (x + 1.0);
  return x / (x * x - 1.0);
}

inline double becke_step(double u, double rm_j, double rm_k) {
  u += becke_adjust(rm_j, rm_k) * (1.0 - u * u);
  u = 1.5 * u - 0.5 * (u * u * u);
  u = 1.5 * u - 0.5 * (u * u * u);
  u = 1.5 * u - 0.5 * (u * u * u);
  return 0.5 * (1.0 - u);
}

void compute_weights(const System& sys, PointGroup& g) {
  const int nn = (int)g.nucs.size();
  const int np = (int)g.points.size();
  const int* nucs = g.nucs.data();
#pragma omp parallel for schedule(static) if (np > 2048)
  for (int pi = 0; pi < np; pi++) {
    GridPoint& pt = g.points[pi];
    const int atom = pt.atom;
    double P_total = 0.0, P_atom = 0.0;
    bool own_found = false;
    for (int j = 0; j < nn; ++j) {
      double P_curr = 1.0;
      const int aj = nucs[j];
      const double dj = len3(pt.x - sys.ax[aj], pt.y - sys.ay[aj], pt.z - sys.az[aj]);
      for (int k = 0; k < nn; ++k) {
        const int ak = nucs[k];
        if (ak == aj) continue;
        double u = (dj - len3(pt.x - sys.ax[ak], pt.y - sys.ay[ak], pt.z - sys.az[ak])) /
                   sys.atom_dist[(size_t)aj * sys.natoms + ak];
        P_curr *= becke_step(u, sys.rm[aj], sys.rm[ak]);
        if (P_curr == 0.0) break;
      }
      if (aj == atom) {
        own_found = true;
        P_atom = P_curr;
        if (P_atom == 0.0) break;
      }
      P_total += P_curr;
    }
    if (!own_found) {
      // the point's own atom is not among the group's nuclei (weight.cpp:67-96)
      P_atom = 1.0;
      const double da = len3(pt.x - sys.ax[atom], pt.y - sys.ay[atom], pt.z - sys.az[atom]);
      for (int k = 0; k < nn; ++k) {
        const int ak = nucs[k];
        double u = (da - len3(pt.x - sys.ax[ak], pt.y - sys.ay[ak], pt.z - sys.az[ak])) /
                   sys.atom_dist[(size_t)atom * sys.natoms + ak];
        P_atom *= becke_step(u, sys.rm[atom], sys.rm[ak]);
        if (P_atom == 0.0) break;
      }
    }
    const double atom_weight = (P_total == 0.0 ? 0.0 : (P_atom / P_total));
    pt.w *= atom_weight;
  }
}

// zero-weight removal (g2g/cpu/weight.cpp:100-111)
void remove_zero_weights(PointGroup& g) {
  // in place, keeping the order (no fresh buffer to fault in)
  g.points.erase(std::remove_if(g.points.begin(), g.points.end(), [](const GridPoint& p) { return p.w == 0.0; }),
                 g.points.end());
}

long long env_int(const char* name, long long dflt) {
  const char* v = std::getenv(name);
  return v ? std::strtol(v, nullptr, 10) : dflt;
}

}  // namespace

void becke_pair_table(const System& sys, double* out) {
  const size_t na = (size_t)sys.natoms;
  for (size_t j = 0; j < na; j++)
    for (size_t k = 0; k < na; k++) out[j * na + k] = becke_adjust(sys.rm[j], sys.rm[k]);
}

void host_becke_weights(const System& sys, const std::vector<PointGroup*>& groups, bool drop_zero) {
  for (PointGroup* g : groups) {
    compute_weights(sys, *g);
    if (drop_zero) remove_zero_weights(*g);
  }
}

// Per-atom point buffers of the grid build, kept by each calling thread from one
// geometry to the next: allocating them afresh (a few hundred KB per atom) on
// every call costs page faults that the threads filling them in parallel take
// one at a time.
struct PointScratch {
  std::vector<std::vector<GridPoint>> pts;
  std::vector<std::vector<long long>> dst;
};
static thread_local PointScratch tl_point_scratch;

void build_partition(const System& sys, const Options& opt, const AngularGrid& ang,
                     int grid_type, Partition& out, WeightsFn weights) {
  out.cubes.clear();
  out.spheres.clear();
  const int natoms = sys.natoms;
  const std::vector<unsigned>& shells = grid_type == 0 ? sys.shells_grid0 : sys.shells_grid12;

  // smallest exponent per element and per function (regenerate_partition.cpp:165-186)
  std::vector<double> min_exps_type(120, std::numeric_limits<double>::max());
  for (int i = 0; i < sys.M; i++) {
    const int t = sys.atom_type[sys.nuc[i]];
    for (int j = 0; j < sys.ncont[i]; j++)
      min_exps_type[t] = std::min(min_exps_type[t], sys.a[(size_t)i * kMaxContractions + j]);
  }
  std::vector<double> min_exps_func(sys.M, std::numeric_limits<double>::max());
  for (int i = 0; i < sys.M; i++)
    for (int j = 0; j < sys.ncont[i]; j++)
      if (sys.a[(size_t)i * kMaxContractions + j] < min_exps_func[i])
        min_exps_func[i] = sys.a[(size_t)i * kMaxContractions + j];

  // bounding prism (:189-219)
  double x0[3] = {0, 0, 0}, x1[3] = {0, 0, 0};
  for (int atom = 0; atom < natoms; atom++) {
    const double pos[3] = {sys.ax[atom], sys.ay[atom], sys.az[atom]};
    const double r = 2 * std::sqrt(opt.max_function_exponent / min_exps_type[sys.atom_type[atom]]);
    for (int d = 0; d < 3; d++) {
      if (atom == 0) {
        x0[d] = pos[d] - r;
        x1[d] = pos[d] + r;
      } else {
        x0[d] = std::min(x0[d], pos[d] - r);
        x1[d] = std::max(x1[d], pos[d] + r);
      }
    }
  }
  const double lcs = opt.little_cube_size;
  unsigned psize[3];
  for (int d = 0; d < 3; d++) psize[d] = (unsigned)std::ceil((x1[d] - x0[d]) / lcs);

  // sphere radii (:227-248)
  std::vector<double> sphere_r(natoms, 0.0);
  if (opt.sphere_radius > 0) {
    for (int atom = 0; atom < natoms; atom++) {
      const unsigned ns = shells[atom];
      const unsigned inc = (unsigned)std::ceil(opt.sphere_radius * ns);
      if (inc == 0) {
        sphere_r[atom] = 0;
      } else {
        const double x = std::cos((M_PI / (ns + 1)) * (ns - inc + 1));
        sphere_r[atom] = sys.rm[atom] * (1.0 + x) / (1.0 - x);
      }
    }
  }

  // points: Gauss-Chebyshev radial (Becke mapping) x angular (:274-322). Each
  // atom's points are generated in parallel (in the reference's shell, point
  // order) with their destination (a cube, or the atom's sphere, -1); the cubes
  // are then filled by threads that each own a range of cubes and scan the atoms
  // in order, so every cube holds its points in the serial loop's order.
  const size_t ncubes_all = (size_t)psize[0] * psize[1] * psize[2];
  std::vector<std::vector<GridPoint>> prism(ncubes_all);
  std::vector<std::vector<GridPoint>> sph(opt.sphere_radius > 0 ? natoms : 0);
  PointScratch& scratch = tl_point_scratch;  // the calling thread's (the workers fill it)
  if ((int)scratch.pts.size() < natoms) {
    scratch.pts.resize(natoms);
    scratch.dst.resize(natoms);
  }
  std::vector<std::vector<GridPoint>>& apts = scratch.pts;
  std::vector<std::vector<long long>>& adst = scratch.dst;
  bool outside = false;
#pragma omp parallel for schedule(dynamic, 1) reduction(|| : outside)
  for (int atom = 0; atom < natoms; atom++) {
    const unsigned ns = shells[atom];
    const double t0 = M_PI / (ns + 1);
    const double rm = sys.rm[atom];
    const unsigned inc = (unsigned)std::ceil(opt.sphere_radius * ns);
    // filled through vectors on this thread's stack (swapped in and out of the
    // atom's slot): the slots' headers share cache lines between atoms, and a
    // push_back on them from several threads would bounce those lines
    std::vector<GridPoint> P;
    std::vector<long long> D;
    P.swap(apts[atom]);
    D.swap(adst[atom]);
    P.clear();
    D.clear();
    P.reserve((size_t)ns * ang.size());
    D.reserve((size_t)ns * ang.size());
    for (unsigned shell = 0; shell < ns; shell++) {
      const double t1 = t0 * (shell + 1);
      const double x = std::cos(t1);
      const double w = t0 * std::fabs(std::sin(t1));
      const double r1 = rm * (1.0 + x) / (1.0 - x);
      const double wrad = w * (r1 * r1) * rm * 2.0 / ((1.0 - x) * (1.0 - x));
      for (int p = 0; p < ang.size(); p++) {
        const double px = sys.ax[atom] + ang.x[p] * r1;
        const double py = sys.ay[atom] + ang.y[p] * r1;
        const double pz = sys.az[atom] + ang.z[p] * r1;
        const bool inside = (x0[0] <= px && px <= x1[0]) && (x0[1] <= py && py <= x1[1]) &&
                            (x0[2] <= pz && pz <= x1[2]);
        if (!inside) continue;
        P.push_back(GridPoint{atom, (int)shell, p, px, py, pz, wrad * ang.w[p]});
        if (shell >= (ns - inc)) {
          D.push_back(-1);
        } else {
          const unsigned cx = (unsigned)std::floor((px - x0[0]) / lcs);
          const unsigned cy = (unsigned)std::floor((py - x0[1]) / lcs);
          const unsigned cz = (unsigned)std::floor((pz - x0[2]) / lcs);
          if (cx >= psize[0] || cy >= psize[1] || cz >= psize[2]) outside = true;
          D.push_back((long long)(((size_t)cx * psize[1] + cy) * psize[2] + cz));
        }
      }
    }
    P.swap(apts[atom]);
    D.swap(adst[atom]);
  }
  if (outside) throw std::runtime_error("grid point outside the cube prism");
  const size_t ncount = (size_t)natoms * ncubes_all;
  if (ncount <= ((size_t)1 << 26)) {
    // counting sort: points per (atom, cube), start offsets by a prefix over the
    // atoms within each cube, then every atom's points written in parallel to
    // their places (atom-major, each atom's order: the serial loop's order)
    std::vector<int> at((size_t)ncount, 0);  // [atom][cube]: count, then start offset
#pragma omp parallel for schedule(dynamic, 1)
    for (int atom = 0; atom < natoms; atom++) {
      int* row = at.data() + (size_t)atom * ncubes_all;
      for (long long c : adst[atom])
        if (c >= 0) row[c]++;
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (long long c = 0; c < (long long)ncubes_all; c++) {
      int run = 0;
      for (int atom = 0; atom < natoms; atom++) {
        int& v = at[(size_t)atom * ncubes_all + (size_t)c];
        const int n = v;
        v = run;
        run += n;
      }
      prism[(size_t)c].resize((size_t)run);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int atom = 0; atom < natoms; atom++) {
      int* row = at.data() + (size_t)atom * ncubes_all;
      const std::vector<GridPoint>& P = apts[atom];
      const std::vector<long long>& D = adst[atom];
      std::vector<GridPoint> mine;  // the atom's sphere points (filled on this thread's stack)
      for (size_t q = 0; q < P.size(); q++) {
        if (D[q] >= 0)
          prism[(size_t)D[q]][(size_t)row[D[q]]++] = P[q];
        else if (atom < (int)sph.size())
          mine.push_back(P[q]);
      }
      if (atom < (int)sph.size()) sph[atom].swap(mine);
    }
  } else {
#pragma omp parallel
    {
      const int nt = omp_get_num_threads(), t = omp_get_thread_num();
      const long long c0 = (long long)(ncubes_all * t / nt), c1 = (long long)(ncubes_all * (t + 1) / nt);
      for (int atom = 0; atom < natoms; atom++) {
        const std::vector<GridPoint>& P = apts[atom];
        const std::vector<long long>& D = adst[atom];
        for (size_t q = 0; q < P.size(); q++)
          if (D[q] >= c0 && D[q] < c1) prism[(size_t)D[q]].push_back(P[q]);
      }
#pragma omp for schedule(dynamic, 8)
      for (int atom = 0; atom < (int)sph.size(); atom++) {
        std::vector<GridPoint> mine;
        for (size_t q = 0; q < apts[atom].size(); q++)
          if (adst[atom][q] < 0) mine.push_back(apts[atom][q]);
        sph[atom].swap(mine);
      }
    }
  }

  const Screen screen = make_screen(sys, opt, min_exps_func);

  // cubes (:331-399): screening against the cube box, then weights
  // every cube screened in parallel into its own slot, then the kept ones taken
  // in the serial loop's (i, j, k) order
  std::vector<PointGroup> cand_cubes, cand_spheres;
  std::vector<PointGroup> cube_slot(ncubes_all);
  std::vector<char> cube_kept(ncubes_all, 0);
#pragma omp parallel
  {
    std::vector<double> dists(natoms);
#pragma omp for schedule(dynamic, 4)
    for (long long c = 0; c < (long long)ncubes_all; c++) {
      const unsigned i = (unsigned)(c / ((long long)psize[1] * psize[2]));
      const unsigned j = (unsigned)((c / psize[2]) % psize[1]);
      const unsigned k = (unsigned)(c % psize[2]);
      std::vector<GridPoint>& pts = prism[(size_t)c];
      // an empty cube never becomes a group (it has fewer than min_points_per_cube >= 1 points)
      if (pts.empty() && opt.min_points_per_cube > 0) continue;
      const double cc[3] = {x0[0] + i * lcs, x0[1] + j * lcs, x0[2] + k * lcs};
      for (int a = 0; a < natoms; a++) {
        const double pos[3] = {sys.ax[a], sys.ay[a], sys.az[a]};
        double dv[3];
        for (int d = 0; d < 3; d++) {
          if (pos[d] < cc[d])
            dv[d] = cc[d] - pos[d];
          else if (pos[d] > (cc[d] + lcs))
            dv[d] = pos[d] - (cc[d] + lcs);
          else
            dv[d] = 0;
        }
        dists[a] = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
      }
      PointGroup& g = cube_slot[(size_t)c];
      g.sphere = false;
      assign_functions(sys, opt, dists, min_exps_func, screen, g);
      if (g.funcs.empty() || pts.size() < opt.min_points_per_cube) continue;
      g.points.swap(pts);
      cube_kept[(size_t)c] = 1;
    }
  }
  for (size_t c = 0; c < ncubes_all; c++)
    if (cube_kept[c]) cand_cubes.push_back(std::move(cube_slot[c]));
  std::vector<double> dists(natoms);

  // spheres (:402-462)
  if (opt.sphere_radius > 0) {
    for (int a = 0; a < natoms; a++) {
      for (int o = 0; o < natoms; o++) {
        if (o == a) {
          dists[o] = 0;
        } else {
          const double d = len3(sys.ax[o] - sys.ax[a], sys.ay[o] - sys.ay[a], sys.az[o] - sys.az[a]);
          const double dd = (sphere_r[a] > d ? 0 : d - sphere_r[a]);
          dists[o] = dd * dd;
        }
      }
      PointGroup g;
      g.sphere = true;
      assign_functions(sys, opt, dists, min_exps_func, screen, g);
      if (sph[a].size() < opt.min_points_per_cube) continue;
      g.points.swap(sph[a]);
      cand_spheres.push_back(std::move(g));
    }
  }

  // weights of every candidate group in one pass, then the filters in group order
  std::vector<PointGroup*> all;
  all.reserve(cand_cubes.size() + cand_spheres.size());
  for (PointGroup& g : cand_cubes) all.push_back(&g);
  for (PointGroup& g : cand_spheres) all.push_back(&g);
  (weights ? weights : host_becke_weights)(sys, all, opt.remove_zero_weights);
  for (int pass = 0; pass < 2; pass++) {
    std::vector<PointGroup>& cand = pass == 0 ? cand_cubes : cand_spheres;
    for (PointGroup& g : cand) {
      if (g.points.size() < opt.min_points_per_cube) continue;
      (pass == 0 ? out.cubes : out.spheres).push_back(std::move(g));
    }
  }

  const long long mc = out.mincost;
  auto by_cost = [mc](const PointGroup& l, const PointGroup& r) { return l.cost(mc) < r.cost(mc); };
  std::stable_sort(out.cubes.begin(), out.cubes.end(), by_cost);
  std::stable_sort(out.spheres.begin(), out.spheres.end(), by_cost);
}

}  // namespace lio
