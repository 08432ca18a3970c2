// The g2g C ABI (Fortran calling convention) over the B200 device engine.
//
// Process-global state, single caller thread, like the reference
// (g2g/init.cpp:27-33). Every entry point catches all exceptions: failures are
// recorded in a sticky status (g2g_last_error_) and, at verbose > 0, printed;
// nothing is thrown across the boundary and nothing calls exit().
//
// Linked beside the reference's library: lioamber also calls the reference's
// analytic-integral entry points (aint_*: the Coulomb fit and the QM/MM
// integrals, g2g/analytic_integral/aint_init.cpp), whose code reads the state
// the reference's own g2g_parameter_init_ and g2g_reload_atom_positions_ fill
// (atom positions, basis, density and Fock pointers). When this library is
// linked ahead of the reference's, the state-setting entry points here
// (g2g_init_, g2g_set_options_, g2g_parameter_init_,
// g2g_reload_atom_positions_, g2g_new_grid_, g2g_deinit_) first pass the call
// on to the next definition in the process's symbol search order (the
// reference's), so that state is kept exactly as before; the XC build,
// g2g_solve_groups_, is this library's alone. LIO_B200_NO_FORWARD set in the
// environment turns the passing on off.
#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#pragma GCC visibility push(default)
#include "../../include/g2g.h"
#pragma GCC visibility pop
#include "engine.h"
#include "partition.h"
#include "system.h"

namespace {

using lio::AngularGrid;
using lio::Options;
using lio::Partition;
using lio::System;

struct BoundArrays {  // caller-owned arrays (g2g/init.h:16-52)
  unsigned natoms = 0, max_atoms = 0, ngaussians = 0, M = 0;
  double* r = nullptr;
  unsigned* nuc = nullptr;
  unsigned* ncont = nullptr;
  double *a = nullptr, *c = nullptr;
  double *rho = nullptr, *fock = nullptr, *fockb = nullptr, *rhoa = nullptr, *rhob = nullptr;
  bool open = false;
};

struct State {
  Options opt;
  System sys;
  BoundArrays arr;
  bool params_set = false;
  std::map<unsigned, AngularGrid> grids;  // by grid_type
  int grid_type = -1;
  Partition part;
  std::unique_ptr<lio::DeviceEngine> engine;
  // precision mode (g2g_set_precision_): 0 FP64, 1 tensor core, 2 autotuned,
  // 3 (the default) tensor core where the grid can run it, else FP64
  unsigned mode = 3;
  lio::Precision precision = lio::Precision::TensorCore;  // the form of the current grid
  int status = 0;
  std::string message;
  double last_solve_ms = 0.0, last_grid_ms = 0.0;
  double grid_phase_ms[3] = {0.0, 0.0, 0.0};  // partition (incl. weights), device upload, autotune
  bool device_ready = false;
  void* stream = nullptr;
  bool graphs = true;
  bool device_weights = true;  // Becke weights of the grid build on the GPU when one is present
  bool lean = false;           // g2g_set_lean_: the blocked basis released once the operands are built
  int shard_rank = 0, shard_world = 1;  // this process's share of the groups (multi-GPU)
};

State& st() {
  static State s;
  return s;
}

void fail(const std::string& msg, int code = 1) {
  State& s = st();
  s.status = code;
  s.message = msg;
  if (s.opt.verbose > 0) std::fprintf(stderr, "g2g error: %s\n", msg.c_str());
}

template <class F>
void guarded(const char* where, F&& f) {
  try {
    f();
  } catch (const std::exception& e) {
    fail(std::string(where) + ": " + e.what());
  } catch (...) {
    fail(std::string(where) + ": unknown error");
  }
}

AngularGrid grid_from_fortran(const double* e, const double* w, unsigned n) {
  AngularGrid g;
  g.x.resize(n);
  g.y.resize(n);
  g.z.resize(n);
  g.w.resize(n);
  for (unsigned i = 0; i < n; i++) {  // column-major n x 3
    g.x[i] = e[i];
    g.y[i] = e[n + i];
    g.z[i] = e[2 * n + i];
    g.w[i] = w[i];
  }
  return g;
}

// Copies positions and basis parameters out of the bound arrays
// (g2g/init.cpp:286-294 re-reads the positions at every reload).
void refresh_system() {
  State& s = st();
  System& y = s.sys;
  const BoundArrays& b = s.arr;
  y.natoms = (int)b.natoms;
  y.ax.resize(b.natoms);
  y.ay.resize(b.natoms);
  y.az.resize(b.natoms);
  for (unsigned i = 0; i < b.natoms; i++) {
    y.ax[i] = b.r[i];
    y.ay[i] = b.r[b.max_atoms + i];
    y.az[i] = b.r[2 * (size_t)b.max_atoms + i];
  }
  y.atom_dist.assign((size_t)b.natoms * b.natoms, 0.0);
  for (unsigned i = 0; i < b.natoms; i++)
    for (unsigned j = 0; j < b.natoms; j++) {
      const double dx = y.ax[i] - y.ax[j], dy = y.ay[i] - y.ay[j], dz = y.az[i] - y.az[j];
      y.atom_dist[(size_t)i * b.natoms + j] = std::sqrt(dx * dx + dy * dy + dz * dz);
    }
  y.M = (int)b.M;
  y.nuc.resize(b.M);
  y.ncont.resize(b.M);
  y.a.assign((size_t)b.M * lio::kMaxContractions, 0.0);
  y.c.assign((size_t)b.M * lio::kMaxContractions, 0.0);
  for (unsigned i = 0; i < b.M; i++) {
    y.nuc[i] = (int)b.nuc[i] - 1;
    y.ncont[i] = (int)b.ncont[i];
    for (unsigned k = 0; k < b.ncont[i] && k < (unsigned)lio::kMaxContractions; k++) {
      y.a[(size_t)i * lio::kMaxContractions + k] = b.a[(size_t)k * b.ngaussians + i];
      y.c[(size_t)i * lio::kMaxContractions + k] = b.c[(size_t)k * b.ngaussians + i];
    }
  }
}

// Cost-balanced assignment of the partition's groups to `world` ranks: longest
// processing time first on the reference's group cost (g2g/partition.cpp:257-260),
// each group to the least-loaded rank (ties to the lower rank).
std::vector<int> shard_owners(const Partition& part, int world) {
  const int ng = part.total_groups();
  std::vector<int> order(ng), owner(ng, 0);
  for (int g = 0; g < ng; g++) order[g] = g;
  auto cost = [&](int g) { return part.group(g).cost(part.mincost); };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
  std::vector<long long> load(world, 0);
  for (int g : order) {
    int r = 0;
    for (int k = 1; k < world; k++)
      if (load[k] < load[r]) r = k;
    owner[g] = r;
    load[r] += cost(g);
  }
  return owner;
}

void build_grid(unsigned grid_type) {
  State& s = st();
  if (!s.params_set) throw std::runtime_error("g2g_parameter_init_ has not been called");
  auto it = s.grids.find(grid_type);
  if (it == s.grids.end()) throw std::runtime_error("unknown grid type " + std::to_string(grid_type));
  const auto t0 = std::chrono::steady_clock::now();
  refresh_system();
  const bool dev = s.device_weights && lio::DeviceEngine::available();
  lio::build_partition(s.sys, s.opt, it->second, (int)grid_type, s.part,
                       dev ? &lio::DeviceEngine::becke_weights : nullptr);
  s.grid_type = (int)grid_type;
  s.last_grid_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  s.grid_phase_ms[0] = s.last_grid_ms;
  s.grid_phase_ms[1] = s.grid_phase_ms[2] = 0.0;
  // The partition is host work and is kept even without a GPU (so it can be
  // inspected); the device upload and every solve need a CUDA device.
  if (!lio::DeviceEngine::available()) {
    s.device_ready = false;
    throw std::runtime_error("no CUDA device: the grid partition was built but the device engine is unavailable");
  }
  if (!s.engine) s.engine.reset(new lio::DeviceEngine());
  s.engine->set_lean(s.lean);
  s.engine->set_stream(s.stream);
  s.engine->set_graphs(s.graphs);
  s.precision = s.mode == 0 ? lio::Precision::FP64 : lio::Precision::TensorCore;
  s.engine->set_precision(s.precision);
  if (s.shard_world > 1) {
    const std::vector<int> owner = shard_owners(s.part, s.shard_world);
    std::vector<char> keep(owner.size());
    for (size_t g = 0; g < owner.size(); g++) keep[g] = owner[g] == s.shard_rank;
    s.engine->upload(s.sys, s.part, &keep);
  } else {
    s.engine->upload(s.sys, s.part);
  }
  const double t_up = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  s.grid_phase_ms[1] = t_up - s.grid_phase_ms[0];
  if (s.mode == 2) {
    s.precision = s.engine->autotune();
  } else if (s.mode == 3) {
    // the tensor-core operands are built now; a grid the form cannot run (a
    // point group beyond the Kohn-Sham accumulators' limit, or more functions
    // than a block's shared memory holds) gets the FP64 form instead
    try {
      s.engine->prepare();
    } catch (const std::exception&) {
      s.engine->drop_tensor_core();
      s.precision = lio::Precision::FP64;
      s.engine->set_precision(s.precision);
      s.engine->prepare();
    }
  }
  s.device_ready = true;
  s.last_grid_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  s.grid_phase_ms[2] = s.last_grid_ms - t_up;
}

// The definition of `name` that follows this library in the symbol search
// order (a g2g linked after it), or null (none, or passing on turned off).
template <class F>
F next_definition(const char* name, F self) {
  if (std::getenv("LIO_B200_NO_FORWARD")) return nullptr;
  F p = reinterpret_cast<F>(dlsym(RTLD_NEXT, name));
  return p == self ? nullptr : p;
}
// Calls the next definition of the enclosing entry point `name` with the same
// arguments; a failure there is recorded like one of this library's own.
#define LIO_PASS_ON(name, ...)                                                        \
  do {                                                                                \
    static const auto next_ = next_definition(#name, &name);                          \
    if (next_) guarded(#name " (passed on to the next g2g)", [&] { next_(__VA_ARGS__); }); \
  } while (0)

// ---- Fortran-named timers (g2g/timer.cpp:117-296): host wall clock
struct NamedTimer {
  double total = 0.0;
  std::chrono::steady_clock::time_point start;
  bool running = false;
};
std::map<std::string, NamedTimer>& timers() {
  static std::map<std::string, NamedTimer> t;
  return t;
}
void timer_start(const char* n, unsigned len) {
  NamedTimer& t = timers()[std::string(n, len)];
  t.start = std::chrono::steady_clock::now();
  t.running = true;
}
double timer_pause(const char* n, unsigned len) {
  NamedTimer& t = timers()[std::string(n, len)];
  if (t.running) {
    t.total += std::chrono::duration<double>(std::chrono::steady_clock::now() - t.start).count();
    t.running = false;
  }
  return t.total;
}

}  // namespace

extern "C" {

void g2g_init_(void) {
  LIO_PASS_ON(g2g_init_);
  guarded("g2g_init_", [] {
    if (!lio::DeviceEngine::available()) throw std::runtime_error("no CUDA device visible");
    if (!st().engine) st().engine.reset(new lio::DeviceEngine());
  });
}

void g2g_set_options_(double* fgm, double* lcs, double* sr, bool* aaf, bool* eai, bool* rzw, unsigned* mppc,
                      unsigned* mfe, unsigned* time, unsigned* verbose) {
  LIO_PASS_ON(g2g_set_options_, fgm, lcs, sr, aaf, eai, rzw, mppc, mfe, time, verbose);
  Options& o = st().opt;
  o.free_global_memory = *fgm;
  o.little_cube_size = *lcs;
  o.sphere_radius = *sr;
  o.assign_all_functions = *aaf;
  o.energy_all_iterations = *eai;
  o.remove_zero_weights = *rzw;
  o.min_points_per_cube = *mppc;
  o.max_function_exponent = *mfe;
  o.timer_level = *time;
  o.verbose = *verbose;
}

void g2g_parameter_init_(const unsigned* norm, const unsigned* natom, const unsigned* max_atoms,
                         const unsigned* ngaussians, double* r, double* Rm, const unsigned* Iz,
                         const unsigned* Nr, const unsigned* Nr2, unsigned* Nuc, const unsigned* M,
                         unsigned* ncont, const unsigned* nshell, double* c, double* a, double* rho_vec,
                         double* fock_vec, double* fockb_vec, double* rhoalpha, double* rhobeta,
                         const unsigned* nco, bool* OPEN, const unsigned* nunp, const unsigned* nopt,
                         const unsigned* Iexch, double* e, double* e2, double* e3, double* wang,
                         double* wang2, double* wang3, bool* use_libxc, const unsigned* ex_functional_id,
                         const unsigned* ec_functional_id) {
  LIO_PASS_ON(g2g_parameter_init_, norm, natom, max_atoms, ngaussians, r, Rm, Iz, Nr, Nr2, Nuc, M, ncont, nshell, c,
              a, rho_vec, fock_vec, fockb_vec, rhoalpha, rhobeta, nco, OPEN, nunp, nopt, Iexch, e, e2, e3, wang, wang2,
              wang3, use_libxc, ex_functional_id, ec_functional_id);
  guarded("g2g_parameter_init_", [&] {
    State& s = st();
    BoundArrays& b = s.arr;
    b.natoms = *natom;
    b.max_atoms = *max_atoms;
    b.ngaussians = *ngaussians;
    b.M = *M;
    b.r = r;
    b.nuc = Nuc;
    b.ncont = ncont;
    b.a = a;
    b.c = c;
    b.rho = rho_vec;
    b.fock = fock_vec;
    b.fockb = fockb_vec;
    b.rhoa = rhoalpha;
    b.rhob = rhobeta;
    b.open = *OPEN;
    for (unsigned i = 0; i < *M; i++)
      if (ncont[i] > (unsigned)lio::kMaxContractions)
        throw std::runtime_error("Maximum functions per contraction reached!");
    if (*Iexch < 1 || *Iexch > 9) throw std::runtime_error("Iexch out of range 1..9");
    // 1-3: LDA (Slater; + Gunnarsson-Lundqvist; + VWN); 4-9: GGA (closed shell:
    // 4 P86+P86, 5 B88+P86, 6 B88+VWN-form, 7 B88+LYP, 8 P86+LYP, 9 PBE; open
    // shell: PBE for every GGA value, as g2g/cpu/iteration.cpp:478-480 calls it)
    if (*Iexch < 1 || *Iexch > 9)
      throw std::runtime_error("Iexch " + std::to_string(*Iexch) + " is not implemented (supported: 1-3 LDA, 4-9 GGA)");
    if (*use_libxc) throw std::runtime_error("libxc functionals are not supported");
    System& y = s.sys;
    y.s_funcs = (int)nshell[0];
    y.p_funcs = (int)nshell[1] / 3;
    y.d_funcs = (int)nshell[2] / 6;
    y.d_norm = *norm ? (1.0 / std::sqrt(3)) : 1.0;
    y.iexch = (int)*Iexch;
    y.lda = (*Iexch <= 3);
    y.open = *OPEN;
    y.atom_type.resize(*natom);
    y.shells_grid0.resize(*natom);
    y.shells_grid12.resize(*natom);
    y.rm.resize(*natom);
    for (unsigned i = 0; i < *natom; i++) {
      y.atom_type[i] = (int)Iz[i] - 1;
      y.shells_grid0[i] = Nr[Iz[i]];
      y.shells_grid12[i] = Nr2[Iz[i]];
      y.rm[i] = Rm[Iz[i]];
    }
    s.grids[0] = grid_from_fortran(e, wang, 50);
    s.grids[1] = grid_from_fortran(e2, wang2, 116);
    s.grids[2] = grid_from_fortran(e3, wang3, 194);
    s.params_set = true;
    s.grid_type = -1;
    (void)nco;
    (void)nunp;
    (void)nopt;
    (void)ex_functional_id;
    (void)ec_functional_id;
  });
}

void g2g_set_angular_grid_(const unsigned* grid_type, const unsigned* npoints, const double* e,
                           const double* wang) {
  guarded("g2g_set_angular_grid_", [&] {
    if (*grid_type < 3) throw std::runtime_error("grid types 0-2 are bound by g2g_parameter_init_");
    st().grids[*grid_type] = grid_from_fortran(e, wang, *npoints);
  });
}

void g2g_reload_atom_positions_(const unsigned* grid_type) {
  LIO_PASS_ON(g2g_reload_atom_positions_, grid_type);
  guarded("g2g_reload_atom_positions_", [&] { build_grid(*grid_type); });
}

void g2g_new_grid_(const unsigned* grid_type) {
  LIO_PASS_ON(g2g_new_grid_, grid_type);
  guarded("g2g_new_grid_", [&] {
    if ((int)*grid_type != st().grid_type) build_grid(*grid_type);
  });
}

void g2g_solve_groups_(const unsigned* computation_type, double* fort_energy_ptr, double* fort_forces_ptr) {
  guarded("g2g_solve_groups_", [&] {
    State& s = st();
    if (s.grid_type < 0) throw std::runtime_error("no grid: call g2g_reload_atom_positions_ first");
    if (!s.engine || !s.device_ready) throw std::runtime_error("no CUDA device engine for the current grid");
    const unsigned ct = *computation_type;
    bool compute_energy = (ct == 1 || ct == 2);
    const bool compute_forces = (ct == 2 || ct == 3);
    const bool compute_rmm = (ct == 0);
    if (s.opt.energy_all_iterations) compute_energy = true;
    if (compute_forces && !fort_forces_ptr) throw std::runtime_error("XC forces requested with a null forces array");
    lio::SolveRequest req;
    req.compute_rmm = compute_rmm;
    req.compute_energy = compute_energy;
    if (s.sys.open) {
      req.rho_a = s.arr.rhoa;
      req.rho_b = s.arr.rhob;
      req.fock = s.arr.fock;
      req.fock_b = s.arr.fockb;
    } else {
      req.rho = s.arr.rho;
      req.fock = s.arr.fock;
    }
    s.engine->set_precision(s.precision);
    // forces: += into the caller's natoms x 3 column-major array, leading
    // dimension max_atoms (g2g/partition.cpp:516-526); no Kohn-Sham update
    const lio::SolveResult r = compute_forces
                                   ? s.engine->solve_forces(req, fort_forces_ptr, (int)s.arr.max_atoms)
                                   : s.engine->solve(req);
    s.last_solve_ms = r.device_ms;
    *fort_energy_ptr = compute_energy ? r.energy : 0.0;
    if (std::isnan(*fort_energy_ptr)) fail("XC energy is NaN", 2);
  });
}

void g2g_set_stream_(void* cuda_stream) {
  guarded("g2g_set_stream_", [&] {
    State& s = st();
    s.stream = cuda_stream;
    if (s.engine) s.engine->set_stream(cuda_stream);
  });
}

int g2g_solve_resident_(void) {
  int n = -1;
  guarded("g2g_solve_resident_", [&] {
    State& s = st();
    if (s.grid_type < 0 || !s.engine || !s.device_ready) throw std::runtime_error("no device grid");
    lio::SolveRequest req;
    req.resident = true;
    s.engine->set_precision(s.precision);
    s.engine->solve(req);
    n = s.engine->launches_per_solve();
  });
  return n;
}

void g2g_set_shard_(const int* rank, const int* world) {
  guarded("g2g_set_shard_", [&] {
    if (*world < 1 || *rank < 0 || *rank >= *world) throw std::runtime_error("shard rank must be in 0 .. world-1");
    State& s = st();
    s.shard_rank = *rank;
    s.shard_world = *world;
  });
}

int g2g_shard_groups_(const int* world, int* owner) {
  int n = -1;
  guarded("g2g_shard_groups_", [&] {
    if (*world < 1) throw std::runtime_error("world must be >= 1");
    const std::vector<int> o = shard_owners(st().part, *world);
    for (size_t g = 0; g < o.size(); g++) owner[g] = o[g];
    n = (int)o.size();
  });
  return n;
}

void g2g_copy_resident_results_(double* d_fock_a, double* d_fock_b, double* d_energy) {
  guarded("g2g_copy_resident_results_", [&] {
    State& s = st();
    if (!s.engine || !s.device_ready) throw std::runtime_error("no device grid");
    s.engine->copy_results(d_fock_a, d_fock_b, d_energy);
  });
}

void g2g_set_graphs_(const unsigned* on) {
  guarded("g2g_set_graphs_", [&] {
    State& s = st();
    s.graphs = *on != 0;
    if (s.engine) s.engine->set_graphs(s.graphs);
  });
}

void g2g_profile_(const unsigned* on) {
  guarded("g2g_profile_", [&] {
    State& s = st();
    if (s.engine) s.engine->set_profiling(*on != 0);
  });
}

void g2g_set_accumulators_(double* d_fock_a, double* d_fock_b, double* d_energy) {
  guarded("g2g_set_accumulators_", [&] {
    State& s = st();
    if (!s.engine) throw std::runtime_error("no device engine: build a grid first");
    s.engine->set_accumulators(d_fock_a, d_fock_b, d_energy);
  });
}

void g2g_set_device_weights_(const unsigned* on) {
  guarded("g2g_set_device_weights_", [&] { st().device_weights = *on != 0; });
}

double g2g_last_force_ms_(void) {
  double ms = -1.0;
  guarded("g2g_last_force_ms_", [&] {
    State& s = st();
    if (!s.engine) throw std::runtime_error("no device engine");
    ms = s.engine->last_force_kernel_ms();
  });
  return ms;
}

void g2g_last_transfer_bytes_(long long* h2d, long long* d2h) {
  guarded("g2g_last_transfer_bytes_", [&] {
    State& s = st();
    if (!s.engine) throw std::runtime_error("no device engine");
    s.engine->last_transfer_bytes(h2d, d2h);
  });
}

int g2g_stage_times_(double* ms, int* solves) {
  int n = 0;
  guarded("g2g_stage_times_", [&] {
    State& s = st();
    if (!s.engine) throw std::runtime_error("no device engine");
    n = s.engine->stage_times(ms, 5, solves);
  });
  return n;
}

int g2g_solve_device_noalloc_(const double* d_rho_a, const double* d_rho_b, double* d_fock_a, double* d_fock_b,
                              double* d_energy, void* stream) {
  int rc = -1;
  guarded("g2g_solve_device_noalloc_", [&] {
    State& s = st();
    if (s.grid_type < 0 || !s.engine || !s.device_ready) throw std::runtime_error("no device grid");
    s.engine->solve_noalloc(d_rho_a, d_rho_b, d_fock_a, d_fock_b, d_energy, stream);
    rc = 0;
  });
  return rc;
}

int g2g_selftest_bounded_wait_(const unsigned* polls, double* ms) {
  int rc = -1;
  guarded("g2g_selftest_bounded_wait_", [&] {
    if (!lio::DeviceEngine::available()) throw std::runtime_error("no CUDA device visible");
    unsigned checksum = 0;
    rc = lio::bounded_wait_selftest(*polls, ms, &checksum);
    if (rc == 1) {
      if (checksum != 32640u) throw std::runtime_error("bounded-wait self-test: the armed stage held wrong data");
      fail("bounded wait timed out after " + std::to_string(*polls) +
               " polls (self-test: the producer stopped early); the kernel returned and freed its TMEM",
           3);
    } else if (rc != 0) {
      throw std::runtime_error("bounded-wait self-test: status " + std::to_string(rc));
    }
  });
  return rc;
}

void g2g_deinit_(void) {
  LIO_PASS_ON(g2g_deinit_);
  guarded("g2g_deinit_", [] {
    State& s = st();
    s.part.cubes.clear();
    s.part.spheres.clear();
    if (s.engine) s.engine->release();
    s.grid_type = -1;
  });
}

int g2g_last_error_(char* msg, const unsigned* len) {
  State& s = st();
  const int code = s.status;
  if (msg && len && *len > 0) {
    std::strncpy(msg, s.message.c_str(), *len - 1);
    msg[*len - 1] = 0;
  }
  s.status = 0;
  s.message.clear();
  return code;
}

void g2g_set_lean_(const unsigned* on) {
  guarded("g2g_set_lean_", [&] {
    State& s = st();
    s.lean = *on != 0;
    if (s.engine) s.engine->set_lean(s.lean);
  });
}

void g2g_set_precision_(const unsigned* mode) {
  guarded("g2g_set_precision_", [&] {
    State& s = st();
    if (*mode > 3)
      throw std::runtime_error(
          "precision mode must be 0 (FP64), 1 (tensor core), 2 (autotuned) or 3 (tensor core, FP64 where it cannot run)");
    s.mode = *mode;
    // a change applies to the current grid at once when the device holds one
    if (s.mode == 0 || s.mode == 1) s.precision = s.mode == 1 ? lio::Precision::TensorCore : lio::Precision::FP64;
    if (s.engine && s.device_ready) {
      if (s.mode == 2) {
        s.precision = s.engine->autotune();
      } else if (s.mode == 3) {
        s.precision = lio::Precision::TensorCore;
        s.engine->set_precision(s.precision);
        try {
          s.engine->prepare();
        } catch (const std::exception&) {
          s.engine->drop_tensor_core();
          s.precision = lio::Precision::FP64;
          s.engine->set_precision(s.precision);
          s.engine->prepare();
        }
      }
    }
  });
}

void g2g_partition_stats_(long long* out) {
  const Partition& p = st().part;
  long long pts = 0, pm = 0, pm2 = 0;
  for (int g = 0; g < p.total_groups(); g++) {
    const lio::PointGroup& pg = p.group(g);
    const long long n = (long long)pg.points.size(), m = pg.total_functions();
    pts += n;
    pm += n * m;
    pm2 += n * m * m;
  }
  out[0] = p.total_groups();
  out[1] = (long long)p.cubes.size();
  out[2] = (long long)p.spheres.size();
  out[3] = pts;
  out[4] = pm;
  out[5] = pm2;
}

int g2g_partition_group_(const int* g, int* meta, int* ids, double* xyzw, int* funcs) {
  const Partition& p = st().part;
  if (*g < 0 || *g >= p.total_groups()) return -1;
  const lio::PointGroup& pg = p.group(*g);
  meta[0] = (int)pg.points.size();
  meta[1] = (int)pg.funcs.size();
  meta[2] = pg.s;
  meta[3] = pg.p;
  meta[4] = pg.d;
  meta[5] = pg.total_functions();
  meta[6] = (int)pg.nucs.size();
  meta[7] = pg.sphere ? 1 : 0;
  for (size_t i = 0; i < pg.points.size(); i++) {
    const lio::GridPoint& q = pg.points[i];
    if (ids) {
      ids[3 * i] = q.atom;
      ids[3 * i + 1] = q.shell;
      ids[3 * i + 2] = q.point;
    }
    if (xyzw) {
      xyzw[4 * i] = q.x;
      xyzw[4 * i + 1] = q.y;
      xyzw[4 * i + 2] = q.z;
      xyzw[4 * i + 3] = q.w;
    }
  }
  if (funcs)
    for (size_t i = 0; i < pg.funcs.size(); i++) funcs[i] = pg.funcs[i];
  return 0;
}

void g2g_last_timings_(double* solve_ms, double* grid_ms) {
  *solve_ms = st().last_solve_ms;
  *grid_ms = st().last_grid_ms;
}

void g2g_grid_timings_(double* phase_ms) {
  for (int i = 0; i < 3; i++) phase_ms[i] = st().grid_phase_ms[i];
}

void g2g_timer_start_(const char* n, unsigned len) { timer_start(n, len); }
void g2g_timer_stop_(const char* n, unsigned len) {
  const double t = timer_pause(n, len);
  if (st().opt.timer_level % 2 == 1) std::printf("TIMER [%.*s]: %.6f s\n", (int)len, n, t);
  timers().erase(std::string(n, len));
}
void g2g_timer_pause_(const char* n, unsigned len) { timer_pause(n, len); }
void g2g_timer_sum_start_(const char* n, unsigned len) { timer_start(n, len); }
void g2g_timer_sum_stop_(const char* n, unsigned len) { timer_pause(n, len); }
void g2g_timer_sum_pause_(const char* n, unsigned len) { timer_pause(n, len); }
void g2g_timer_clear_(void) { timers().clear(); }
void g2g_timer_summary_(void) {
  if (st().opt.timer_level > 1)
    for (const auto& kv : timers()) std::printf("TIMER SUMMARY [%s]: %.6f s\n", kv.first.c_str(), kv.second.total);
}

}  // extern "C"
