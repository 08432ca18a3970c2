// Many molecules' XC builds per kernel launch (C ABI: lio_batch_* in
// include/lio_serve.h).
//
// The molecules of a batch are grouped by functional class (LDA or GGA, closed
// or open shell, iexch, d normalisation): the kernels are specialised on the
// first two and the point functional on the third. Each class becomes one
// joined system: the atoms and functions of its molecules one after the other
// (each molecule's function types kept explicitly, since the joined order is
// no longer all s, then p, then d) and one partition holding every molecule's
// point groups in molecule order. The device engine uploads it with one
// BatchMember per molecule (function and packed-matrix offsets, group range),
// so one launch per stage covers every group of the class; the groups read
// and write their own molecule's packed matrices and the energy partials are
// summed per molecule. A group's functions all belong to one molecule, so
// joining changes nothing in the arithmetic of any group.
#pragma GCC visibility push(default)
#include "../../include/lio_serve.h"
#pragma GCC visibility pop

#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "engine.h"
#include "molecule.h"
#include "partition.h"
#include "system.h"

namespace {

struct BatchClass {
  lio::System sys;
  lio::Partition part;
  std::vector<lio::BatchMember> members;
  std::vector<int> mols;  // batch index of each member
  std::unique_ptr<lio::DeviceEngine> engine;
  std::vector<double> rho_a, rho_b, fock_a, fock_b, energies;  // concatenated packed vectors
};

std::string& create_error() {
  static std::string e;
  return e;
}

// Appends molecule `m` (its system and partition) to the class's joined system.
void join(BatchClass& c, lio::System&& m, lio::Partition&& part) {
  lio::System& y = c.sys;
  const int atom_off = y.natoms, f_off = y.M;
  y.natoms += m.natoms;
  y.ax.insert(y.ax.end(), m.ax.begin(), m.ax.end());
  y.ay.insert(y.ay.end(), m.ay.begin(), m.ay.end());
  y.az.insert(y.az.end(), m.az.begin(), m.az.end());
  for (int f = 0; f < m.M; f++) {
    y.nuc.push_back(m.nuc[f] + atom_off);
    y.ncont.push_back(m.ncont[f]);
    y.ftype.push_back((int8_t)(f < m.s_funcs ? 0 : (f < m.s_funcs + 3 * m.p_funcs ? 1 : 2)));
  }
  y.a.insert(y.a.end(), m.a.begin(), m.a.end());
  y.c.insert(y.c.end(), m.c.begin(), m.c.end());
  y.M += m.M;
  lio::BatchMember b;
  b.f_off = f_off;
  b.M = m.M;
  b.pk_off = c.members.empty() ? 0
                               : c.members.back().pk_off + (long long)c.members.back().M * (c.members.back().M + 1) / 2;
  b.g_begin = (int)c.part.cubes.size();
  for (std::vector<lio::PointGroup>* v : {&part.cubes, &part.spheres})
    for (lio::PointGroup& g : *v) {
      for (int& f : g.funcs) f += f_off;
      for (int& a : g.nucs) a += atom_off;
      c.part.cubes.push_back(std::move(g));  // the device engine does not tell cubes from spheres
    }
  b.g_end = (int)c.part.cubes.size();
  c.members.push_back(b);
}

}  // namespace

struct lio_batch {
  int device = 0;
  std::vector<BatchClass> classes;
  std::vector<int> mol_class, mol_member, mol_M, mol_open;
  long long points = 0;
  double build_s = 0.0;
  std::string error;
};

extern "C" {

lio_batch* lio_batch_create(int device, int nmol, const lio_molecule* mols, int precision) {
  try {
    if (nmol <= 0 || !mols) throw std::runtime_error("no molecules");
    if (precision < 0 || precision > 2) throw std::runtime_error("precision must be 0, 1 or 2");
    if (cudaSetDevice(device) != cudaSuccess) {
      cudaGetLastError();
      throw std::runtime_error("cannot select CUDA device " + std::to_string(device));
    }
    const auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<lio_batch> b(new lio_batch());
    b->device = device;
    // every molecule's system and partition, on all host threads (the partition
    // build's own parallel loops run inside one thread each)
    std::vector<lio::System> sys(nmol);
    std::vector<lio::Partition> part(nmol);
    std::vector<std::string> err(nmol);
    for (int i = 0; i < nmol; i++) sys[i] = lio::system_from_molecule(&mols[i]);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < nmol; i++) {
      try {
        lio::AngularGrid ang;
        ang.x.assign(mols[i].ang_x, mols[i].ang_x + mols[i].nang);
        ang.y.assign(mols[i].ang_y, mols[i].ang_y + mols[i].nang);
        ang.z.assign(mols[i].ang_z, mols[i].ang_z + mols[i].nang);
        ang.w.assign(mols[i].ang_w, mols[i].ang_w + mols[i].nang);
        lio::build_partition(sys[i], lio::Options(), ang, 3, part[i]);
      } catch (const std::exception& e) {
        err[i] = e.what();
      }
    }
    for (int i = 0; i < nmol; i++)
      if (!err[i].empty()) throw std::runtime_error("molecule " + std::to_string(i) + ": " + err[i]);
    // classes: (lda, open, iexch, d normalisation)
    std::map<std::tuple<int, int, int, double>, int> key_class;
    b->mol_class.resize(nmol);
    b->mol_member.resize(nmol);
    b->mol_M.resize(nmol);
    b->mol_open.resize(nmol);
    for (int i = 0; i < nmol; i++) {
      const auto key = std::make_tuple((int)sys[i].lda, (int)sys[i].open, sys[i].iexch, sys[i].d_norm);
      auto it = key_class.find(key);
      if (it == key_class.end()) {
        it = key_class.emplace(key, (int)b->classes.size()).first;
        b->classes.emplace_back();
        lio::System& y = b->classes.back().sys;
        y.lda = sys[i].lda;
        y.open = sys[i].open;
        y.iexch = sys[i].iexch;
        y.d_norm = sys[i].d_norm;
      }
      BatchClass& c = b->classes[it->second];
      for (int g = 0; g < part[i].total_groups(); g++) b->points += (long long)part[i].group(g).points.size();
      b->mol_class[i] = it->second;
      b->mol_member[i] = (int)c.members.size();
      b->mol_M[i] = sys[i].M;
      b->mol_open[i] = sys[i].open;
      c.mols.push_back(i);
      join(c, std::move(sys[i]), std::move(part[i]));
    }
    // one engine per class
    for (BatchClass& c : b->classes) {
      c.engine.reset(new lio::DeviceEngine());
      c.engine->set_precision(precision == 0 ? lio::Precision::FP64 : lio::Precision::TensorCore);
      c.engine->upload(c.sys, c.part, nullptr, &c.members);
      if (precision == 2) {
        c.engine->autotune();
      } else if (precision == 1) {
        try {  // a class the tensor-core form cannot run takes the FP64 form
          c.engine->prepare();
        } catch (const std::exception&) {
          c.engine->drop_tensor_core();
          c.engine->set_precision(lio::Precision::FP64);
        }
      }
      c.engine->prepare();
      const size_t np = c.engine->packed_size();
      c.rho_a.assign(np, 0.0);
      c.fock_a.assign(np, 0.0);
      if (c.sys.open) {
        c.rho_b.assign(np, 0.0);
        c.fock_b.assign(np, 0.0);
      }
      c.energies.assign(c.members.size(), 0.0);
    }
    b->build_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return b.release();
  } catch (const std::exception& e) {
    create_error() = std::string("lio_batch_create: ") + e.what();
    cudaGetLastError();
    return nullptr;
  }
}

const char* lio_batch_create_error(void) { return create_error().c_str(); }

int lio_batch_solve(lio_batch* b, const double* const* rho_a, const double* const* rho_b, double* const* fock_a,
                    double* const* fock_b, double* energies, double* device_ms) {
  if (!b) return -1;
  try {
    if (cudaSetDevice(b->device) != cudaSuccess) {
      cudaGetLastError();
      throw std::runtime_error("cannot select the batch's device");
    }
    const int nmol = (int)b->mol_class.size();
    // gather every molecule's densities into its class's vectors
    for (int i = 0; i < nmol; i++) {
      BatchClass& c = b->classes[b->mol_class[i]];
      const lio::BatchMember& m = c.members[b->mol_member[i]];
      const size_t n = (size_t)m.M * (m.M + 1) / 2;
      if (!rho_a[i] || (b->mol_open[i] && !rho_b[i])) throw std::runtime_error("molecule " + std::to_string(i) + ": null density");
      std::memcpy(c.rho_a.data() + m.pk_off, rho_a[i], n * sizeof(double));
      if (b->mol_open[i]) std::memcpy(c.rho_b.data() + m.pk_off, rho_b[i], n * sizeof(double));
    }
    // every class's build enqueued on its engine's stream, then completed
    std::vector<lio::SolveRequest> reqs(b->classes.size());
    for (size_t k = 0; k < b->classes.size(); k++) {
      BatchClass& c = b->classes[k];
      lio::SolveRequest& r = reqs[k];
      std::fill(c.fock_a.begin(), c.fock_a.end(), 0.0);
      if (c.sys.open) std::fill(c.fock_b.begin(), c.fock_b.end(), 0.0);
      if (c.sys.open) {
        r.rho_a = c.rho_a.data();
        r.rho_b = c.rho_b.data();
        r.fock = c.fock_a.data();
        r.fock_b = c.fock_b.data();
      } else {
        r.rho = c.rho_a.data();
        r.fock = c.fock_a.data();
      }
      c.engine->enqueue(r);
    }
    double ms = 0.0;
    for (size_t k = 0; k < b->classes.size(); k++) {
      BatchClass& c = b->classes[k];
      ms += c.engine->finish(reqs[k]).device_ms;
      c.engine->batch_energies(c.energies.data());
    }
    // scatter (=) every molecule's results
    for (int i = 0; i < nmol; i++) {
      const BatchClass& c = b->classes[b->mol_class[i]];
      const lio::BatchMember& m = c.members[b->mol_member[i]];
      const size_t n = (size_t)m.M * (m.M + 1) / 2;
      if (fock_a && fock_a[i]) std::memcpy(fock_a[i], c.fock_a.data() + m.pk_off, n * sizeof(double));
      if (b->mol_open[i] && fock_b && fock_b[i]) std::memcpy(fock_b[i], c.fock_b.data() + m.pk_off, n * sizeof(double));
      if (energies) energies[i] = c.energies[b->mol_member[i]];
    }
    if (device_ms) *device_ms = ms;
    return 0;
  } catch (const std::exception& e) {
    b->error = std::string("lio_batch_solve: ") + e.what();
    cudaGetLastError();
    return 1;
  }
}

const char* lio_batch_last_error(lio_batch* b) { return b ? b->error.c_str() : "no batch"; }

int lio_batch_stats(lio_batch* b, long long* points, int* nclasses, double* build_s, int max_classes, int* form,
                    int* members) {
  if (!b) return -1;
  if (points) *points = b->points;
  if (nclasses) *nclasses = (int)b->classes.size();
  if (build_s) *build_s = b->build_s;
  for (int k = 0; k < (int)b->classes.size() && k < max_classes; k++) {
    if (form) form[k] = b->classes[k].engine->precision() == lio::Precision::TensorCore ? 1 : 0;
    if (members) members[k] = (int)b->classes[k].members.size();
  }
  return 0;
}

void lio_batch_destroy(lio_batch* b) {
  if (!b) return;
  if (cudaSetDevice(b->device) != cudaSuccess) cudaGetLastError();
  delete b;
}

}  // extern "C"
