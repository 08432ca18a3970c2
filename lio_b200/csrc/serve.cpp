// XC build service with continuous batching (C ABI in include/lio_serve.h).
//
// Two threads make the service's CUDA calls; callers only enqueue requests and
// wait for them. The worker owns the running builds (one DeviceEngine per
// resident molecule, each with its own CUDA stream). Its loop:
//   1. completes requests whose device work has finished (event query) and
//      wakes their waiters;
//   2. admits queued requests in arrival order while fewer than max_inflight
//      run: a request whose molecule is busy or loading stays queued (one build
//      in flight per molecule: its engine holds one set of per-solve buffers)
//      and later requests may pass it; for a molecule that is not resident it
//      plans the room (plan_admission, least recently used idle molecules
//      first: their per-geometry caches, and only if that is not enough whole
//      molecules), books the bytes and hands the eviction and the upload to the
//      loader thread;
//   3. enqueues the admitted build on the molecule's stream and moves on, so
//      builds of different molecules overlap on the GPU.
// The loader frees the evicted memory and uploads (or, for a molecule whose
// caches were evicted, recomputes them on the device) without holding the
// lock, so requests for resident molecules keep being served meanwhile.
// Requests arriving while others run are therefore admitted as soon as a slot
// and memory free up (continuous batching), not after the current batch.
#pragma GCC visibility push(default)
#include "../../include/lio_serve.h"
#pragma GCC visibility pop

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "partition.h"
#include "system.h"

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

// Admission: does a molecule of `need` bytes fit `budget` with `used` bytes in
// use, if idle residents are evicted least recently used first? Fills `evict`.
bool plan_admission(int n, const unsigned long long* footprint, const int* busy, const unsigned long long* last_use,
                    unsigned long long budget, unsigned long long used, unsigned long long need,
                    std::vector<int>& evict) {
  evict.clear();
  if (need > budget) return false;
  if (used + need <= budget) return true;
  std::vector<int> idle;
  for (int i = 0; i < n; i++)
    if (!busy[i] && footprint[i] > 0) idle.push_back(i);
  std::sort(idle.begin(), idle.end(), [&](int a, int b) { return last_use[a] < last_use[b]; });
  unsigned long long freed = 0;
  for (int i : idle) {
    evict.push_back(i);
    freed += footprint[i];
    if (used - freed + need <= budget) return true;
  }
  evict.clear();
  return false;
}

struct Molecule {
  lio::System sys;
  lio::Options opt;
  lio::AngularGrid ang;
  lio::Partition part;
  std::unique_ptr<lio::DeviceEngine> engine;  // null while not resident
  unsigned long long footprint = 0;           // device bytes while resident
  bool measured = false;
  // cold: resident grid (points, tiles, buffers) without the per-geometry
  // caches (basis values, tensor-core operands), which the next build
  // recomputes on the device; core = the bytes a cold molecule still holds
  bool cold = false;
  unsigned long long core = 0;
  bool loading = false;    // in the loader's hands (being uploaded, restored or evicted)
  std::string load_error;  // an upload that failed: its requests fail with this
  int form = -1;  // the form it runs in (0 FP64, 1 tensor core) once resident
  double tuned_ms[2] = {0.0, 0.0};
  bool busy = false;
  unsigned long long last_use = 0;
  long long points = 0;
  size_t npacked = 0;
};

struct Request {
  int mol = -1;
  std::vector<double> rho_a, rho_b;
  std::vector<double> K_a, K_b;
  double energy = 0.0;
  std::string error;
  enum { kQueued, kRunning, kDone } state = kQueued;
  Clock::time_point t_submit;
  double latency_ms = 0.0;
  lio::SolveRequest sreq;
};

}  // namespace

struct LoadJob {
  int mol = -1;                                          // made resident (hot)
  std::vector<int> demote;                               // idle molecules whose caches go
  std::vector<std::unique_ptr<lio::DeviceEngine>> drop;  // engines of molecules evicted whole
  unsigned long long reserved = 0;                       // bytes booked for `mol`
  unsigned long long room = 0;                           // budget minus the other molecules' bytes, at booking
};

struct lio_server {
  int device = 0;
  lio::Precision precision = lio::Precision::TensorCore;
  bool autotune = false;  // per molecule: the faster form, timed at its first upload
  int max_inflight = 16;
  unsigned long long budget = 0, used = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_load;
  std::thread worker, loader;
  std::deque<LoadJob> jobs;
  unsigned long long epoch = 0;  // bumped by submissions and finished loads (the worker's wake-ups)
  bool stop = false;
  std::string error;
  std::vector<std::unique_ptr<Molecule>> mols;
  std::unordered_map<long long, std::unique_ptr<Request>> reqs;
  std::deque<long long> queue;
  std::vector<long long> running;
  long long next_id = 0;
  unsigned long long tick = 0;
  // statistics
  std::vector<double> lat_ms;
  double points_done = 0.0;
  bool any_submit = false;
  Clock::time_point t_first, t_last;
  long long evictions = 0, uploads = 0, oom_retries = 0;
  size_t peak_inflight = 0;

  void loop();
  void loader_loop();
  bool plan_load(int mi, std::string& why);
  bool any_loading() const {
    for (auto& x : mols)
      if (x->loading) return true;
    return false;
  }
};

// Under the lock: books room for molecule mi (not hot, not loading) and queues
// its load; false with `why` empty when it cannot fit yet, or a reason when it
// never can.
bool lio_server::plan_load(int mi, std::string& why) {
  Molecule& m = *mols[mi];
  // before the first upload: the estimate of its form (autotuned: the larger of
  // the two, held one after the other while both are timed); a cold molecule
  // needs its caches back only
  // Engines are lean: a tensor-core molecule holds its blocked basis only while
  // its operands are built, so every load that may build them books that room
  // as well (the booking is replaced by the measured footprint once resident).
  const bool may_tc = autotune ? m.form != 0 : precision == lio::Precision::TensorCore;
  const unsigned long long transient =
      may_tc ? lio::DeviceEngine::estimate_blocked_basis_bytes(m.sys, m.part) : 0;
  const unsigned long long resident_need =
      (m.engine ? m.footprint - m.core
       : m.measured ? m.footprint
       : autotune ? (unsigned long long)std::max(
                        lio::DeviceEngine::estimate_device_bytes(m.sys, m.part, lio::Precision::FP64, true),
                        lio::DeviceEngine::estimate_device_bytes(m.sys, m.part, lio::Precision::TensorCore, true))
                  : (unsigned long long)lio::DeviceEngine::estimate_device_bytes(m.sys, m.part, precision, true));
  // a molecule that fits the budget only without its transient books what it
  // keeps (a load that then runs out of device memory is retried as below)
  const unsigned long long need = resident_need + transient > budget ? resident_need : resident_need + transient;
  // Eviction in two levels, least recently used idle molecules first: their
  // caches (the bulk of a footprint; they go cold and keep their grid), and only
  // if that cannot make room, whole molecules (hot or cold).
  std::vector<unsigned long long> fp_cache, fp_all, lu;
  std::vector<int> busy;
  for (size_t i = 0; i < mols.size(); i++) {
    const Molecule& x = *mols[i];
    const bool cand = (int)i != mi && x.engine && !x.loading;
    fp_cache.push_back(cand && !x.cold ? (unsigned long long)x.engine->cache_bytes() : 0);
    fp_all.push_back(cand ? (x.cold ? x.core : x.footprint) : 0);
    busy.push_back(x.busy || x.loading ? 1 : 0);
    lu.push_back(x.last_use);
  }
  LoadJob job;
  std::vector<int> evict;
  if (plan_admission((int)mols.size(), fp_cache.data(), busy.data(), lu.data(), budget, used, need, evict)) {
    for (int i : evict) {
      Molecule& x = *mols[i];
      x.core = x.footprint > fp_cache[i] ? x.footprint - fp_cache[i] : 0;
      x.cold = true;
      x.loading = true;
      used -= fp_cache[i];
      evictions++;
      job.demote.push_back(i);
    }
  } else if (plan_admission((int)mols.size(), fp_all.data(), busy.data(), lu.data(), budget, used, need, evict)) {
    for (int i : evict) {
      Molecule& x = *mols[i];
      job.drop.push_back(std::move(x.engine));
      x.cold = false;
      used -= fp_all[i];
      evictions++;
    }
  } else {
    why = need > budget ? "molecule footprint exceeds the server's HBM budget" : "";
    return false;
  }
  job.room = budget > used ? budget - used : 0;
  used += need;
  job.mol = mi;
  job.reserved = need;
  m.loading = true;
  jobs.push_back(std::move(job));
  cv_load.notify_one();
  return true;
}

void lio_server::loader_loop() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  while (true) {
    cv_load.wait(lk, [&] { return stop || !jobs.empty(); });
    if (stop) break;
    LoadJob job = std::move(jobs.front());
    jobs.pop_front();
    Molecule& m = *mols[job.mol];
    std::vector<lio::DeviceEngine*> demote;
    for (int i : job.demote) demote.push_back(mols[i]->engine.get());
    lio::DeviceEngine* cold = m.engine.get();  // non-null: caches to rebuild
    const int form = m.form;
    lk.unlock();
    std::string err;
    std::unique_ptr<lio::DeviceEngine> e;
    int new_form = form;
    double tuned[2] = {0.0, 0.0};
    long long delta = 0;
    try {
      job.drop.clear();  // frees the memory of the molecules evicted whole
      for (lio::DeviceEngine* x : demote) x->release_caches();
      const long long before = lio::DeviceEngine::process_device_bytes();
      if (cold) {
        cold->prepare();
      } else {
        e.reset(new lio::DeviceEngine());
        e->set_graphs(true);
        e->set_lean(true);  // the tensor-core form keeps its operands, not the blocked basis
        if (autotune && form >= 0) {  // decided at an earlier upload
          e->set_precision(form ? lio::Precision::TensorCore : lio::Precision::FP64);
          e->upload(m.sys, m.part);
          e->prepare();
        } else if (autotune) {
          // both forms timed alone; the tensor-core form is kept only when it is
          // at least twice as fast, its time x device-bytes product (whole
          // footprint) is the smaller, and it takes at most half of the room the
          // molecule was booked in. Twice: its kernels are persistent (one CTA per
          // SM), so among other molecules' builds they lose the overlap the FP64
          // form's kernels get. Bytes: a form that buys time with proportionally
          // more HBM (small groups, whose 32-function tiles are mostly padding)
          // would crowd the other molecules out and turn into evictions.
          e->upload(m.sys, m.part);  // FP64 form: grid plus its basis cache
          const long long up = lio::DeviceEngine::process_device_bytes() - before;
          size_t c64 = 0, ctc = 0;
          e->autotune_measure(&tuned[0], &tuned[1], &c64, &ctc);
          const double core = (double)std::max<long long>(up - (long long)c64, 0);
          const double fp64 = core + (double)c64, fptc = core + (double)ctc;
          const bool faster = 2.0 * tuned[1] < tuned[0];
          const bool plenty = fptc <= 0.5 * (double)job.room;
          const bool tc = faster && plenty && tuned[1] * fptc < tuned[0] * fp64;
          e->keep_form(tc ? lio::Precision::TensorCore : lio::Precision::FP64);
          new_form = tc ? 1 : 0;
        } else {
          e->set_precision(precision);
          e->upload(m.sys, m.part);
          e->prepare();
          new_form = precision == lio::Precision::TensorCore ? 1 : 0;
        }
      }
      delta = lio::DeviceEngine::process_device_bytes() - before;
    } catch (const std::exception& ex) {
      err = ex.what();
      cudaGetLastError();  // an allocation failure is not sticky; clear it for this thread's next launches
      e.reset();           // a partial upload's memory goes before the lock is taken
      try {
        if (cold) cold->release_caches();
      } catch (...) {
      }
    }
    size_t free_now = 0, total = 0;
    const bool oom = err.find("out of memory") != std::string::npos;
    if (oom && cudaMemGetInfo(&free_now, &total) != cudaSuccess) {
      cudaGetLastError();
      free_now = 0;
    }
    lk.lock();
    for (int i : job.demote) mols[i]->loading = false;
    m.loading = false;
    if (!err.empty()) {
      used -= job.reserved;
      const unsigned long long fit = used + (unsigned long long)(0.9 * (double)free_now);
      if (oom && fit < budget) {
        // memory the accounting counted as free is held elsewhere (another user
        // of the GPU): the budget becomes what the server holds plus 90 % of
        // what is free now, and the request retries, evicting more
        budget = fit;
        oom_retries++;
      } else {
        m.load_error = err;
      }
    } else {
      used = (unsigned long long)std::max<long long>((long long)used - (long long)job.reserved + delta, 0);
      if (cold) {
        m.cold = false;
      } else {
        m.engine = std::move(e);
        m.footprint = (unsigned long long)std::max<long long>(delta, 1);
        m.measured = true;
        if (new_form != form) {
          m.form = new_form;
          m.tuned_ms[0] = tuned[0];
          m.tuned_ms[1] = tuned[1];
        }
      }
      uploads++;
    }
    epoch++;
    cv_work.notify_all();
  }
}

void lio_server::loop() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  while (!stop) {
    bool progressed = false;
    const unsigned long long seen = epoch;
    // 1. completions
    for (size_t k = 0; k < running.size();) {
      Request& r = *reqs[running[k]];
      Molecule& m = *mols[r.mol];
      bool done = false;
      try {
        done = m.engine->ready();
        if (done) {
          const lio::SolveResult res = m.engine->finish(r.sreq);
          r.energy = res.energy;
        }
      } catch (const std::exception& ex) {
        done = true;
        r.error = ex.what();
      }
      if (!done) {
        k++;
        continue;
      }
      r.state = Request::kDone;
      r.latency_ms = seconds_since(r.t_submit) * 1e3;
      lat_ms.push_back(r.latency_ms);
      points_done += (double)m.points;
      t_last = Clock::now();
      m.busy = false;
      m.last_use = ++tick;
      running.erase(running.begin() + (long)k);
      progressed = true;
    }
    if (progressed) cv_done.notify_all();
    // 2./3. admission and launch, in arrival order
    for (auto it = queue.begin(); it != queue.end() && (int)running.size() < max_inflight;) {
      Request& r = *reqs[*it];
      Molecule& m = *mols[r.mol];
      if (m.busy || m.loading) {
        ++it;
        continue;
      }
      if (!m.load_error.empty()) {
        r.error = m.load_error;
        r.state = Request::kDone;
        it = queue.erase(it);
        cv_done.notify_all();
        continue;
      }
      if (!m.engine || m.cold) {  // not resident: book room, the loader makes it so
        std::string why;
        bool ok = false;
        try {
          ok = plan_load(r.mol, why);
        } catch (const std::exception& ex) {
          why = ex.what();
        }
        if (!ok && (!why.empty() || (running.empty() && jobs.empty() && !any_loading()))) {
          // cannot fit now and nothing will free memory
          r.error = why.empty() ? "molecule does not fit the HBM budget" : why;
          r.state = Request::kDone;
          it = queue.erase(it);
          cv_done.notify_all();
          continue;
        }
        ++it;
        continue;
      }
      r.sreq = lio::SolveRequest();
      r.K_a.assign(m.npacked, 0.0);
      if (m.sys.open) r.K_b.assign(m.npacked, 0.0);
      if (m.sys.open) {
        r.sreq.rho_a = r.rho_a.data();
        r.sreq.rho_b = r.rho_b.data();
        r.sreq.fock = r.K_a.data();
        r.sreq.fock_b = r.K_b.data();
      } else {
        r.sreq.rho = r.rho_a.data();
        r.sreq.fock = r.K_a.data();
      }
      try {
        m.engine->enqueue(r.sreq);
      } catch (const std::exception& ex) {
        r.error = ex.what();
        r.state = Request::kDone;
        it = queue.erase(it);
        cv_done.notify_all();
        continue;
      }
      m.busy = true;
      m.last_use = ++tick;
      r.state = Request::kRunning;
      running.push_back(*it);
      peak_inflight = std::max(peak_inflight, running.size());
      it = queue.erase(it);
      progressed = true;
    }
    if (!progressed) {
      if (running.empty())  // nothing on the GPU: sleep until a submission or a finished load
        cv_work.wait(lk, [&] { return stop || epoch != seen; });
      else {  // device work in flight: poll its completion events
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lk.lock();
      }
    }
  }
  // drain: wait for the device work of requests still running
  for (long long id : running) {
    Request& r = *reqs[id];
    try {
      mols[r.mol]->engine->finish(r.sreq);
    } catch (...) {
    }
    r.error = "server stopped";
    r.state = Request::kDone;
  }
  running.clear();
  cv_done.notify_all();
}

namespace lio {
System system_from_molecule(const lio_molecule* d) {
  if (d->natoms <= 0 || d->M <= 0) throw std::runtime_error("empty molecule");
  if (d->iexch < 1 || d->iexch > 9) throw std::runtime_error("iexch must be 1-3 (LDA) or 4-9 (GGA)");
  if (d->s_funcs + 3 * d->p_funcs + 6 * d->d_funcs != d->M) throw std::runtime_error("s/p/d counts do not add up to M");
  lio::System y;
  y.natoms = d->natoms;
  y.ax.resize(d->natoms);
  y.ay.resize(d->natoms);
  y.az.resize(d->natoms);
  y.atom_type.resize(d->natoms);
  y.shells_grid0.resize(d->natoms);
  y.shells_grid12.resize(d->natoms);
  y.rm.resize(d->natoms);
  for (int i = 0; i < d->natoms; i++) {
    y.ax[i] = d->xyz[3 * i];
    y.ay[i] = d->xyz[3 * i + 1];
    y.az[i] = d->xyz[3 * i + 2];
    y.atom_type[i] = d->atomic_number[i] - 1;
    y.shells_grid0[i] = y.shells_grid12[i] = d->shells[i];
    y.rm[i] = d->rm[i];
  }
  y.atom_dist.assign((size_t)d->natoms * d->natoms, 0.0);
  for (int i = 0; i < d->natoms; i++)
    for (int j = 0; j < d->natoms; j++) {
      const double dx = y.ax[i] - y.ax[j], dy = y.ay[i] - y.ay[j], dz = y.az[i] - y.az[j];
      y.atom_dist[(size_t)i * d->natoms + j] = std::sqrt(dx * dx + dy * dy + dz * dz);
    }
  y.M = d->M;
  y.s_funcs = d->s_funcs;
  y.p_funcs = d->p_funcs;
  y.d_funcs = d->d_funcs;
  y.nuc.assign(d->nuc, d->nuc + d->M);
  y.ncont.assign(d->ncont, d->ncont + d->M);
  for (int i = 0; i < d->M; i++) {
    if (d->ncont[i] < 1 || d->ncont[i] > lio::kMaxContractions)
      throw std::runtime_error("primitives per function must be 1..13");
    if (d->nuc[i] < 0 || d->nuc[i] >= d->natoms) throw std::runtime_error("function on a nonexistent atom");
  }
  y.a.assign(d->a, d->a + (size_t)d->M * lio::kMaxContractions);
  y.c.assign(d->c, d->c + (size_t)d->M * lio::kMaxContractions);
  y.d_norm = d->normalize ? 1.0 / std::sqrt(3.0) : 1.0;
  y.iexch = d->iexch;
  y.lda = d->iexch <= 3;
  y.open = d->open != 0;
  return y;
}
}  // namespace lio

extern "C" {

lio_server* lio_srv_create(int device, unsigned long long hbm_budget_bytes, int precision, int max_inflight) {
  try {
    if (cudaSetDevice(device) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    std::unique_ptr<lio_server> s(new lio_server());
    s->device = device;
    s->precision = precision == 1 ? lio::Precision::TensorCore : lio::Precision::FP64;
    s->autotune = precision == 2;
    s->max_inflight = max_inflight > 0 ? max_inflight : 16;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return nullptr;
    s->budget = hbm_budget_bytes ? hbm_budget_bytes : (unsigned long long)(0.9 * (double)fr);
    lio_server* p = s.release();
    p->worker = std::thread([p] { p->loop(); });
    p->loader = std::thread([p] { p->loader_loop(); });
    return p;
  } catch (...) {
    return nullptr;
  }
}

void lio_srv_destroy(lio_server* srv) {
  if (!srv) return;
  {
    std::lock_guard<std::mutex> g(srv->mu);
    srv->stop = true;
  }
  srv->cv_work.notify_all();
  srv->cv_load.notify_all();
  if (srv->worker.joinable()) srv->worker.join();
  if (srv->loader.joinable()) srv->loader.join();
  delete srv;
}

const char* lio_srv_last_error(lio_server* srv) { return srv ? srv->error.c_str() : "no server"; }

int lio_srv_add_molecule(lio_server* srv, const lio_molecule* mol) {
  if (!srv || !mol) return -1;
  try {
    std::unique_ptr<Molecule> m(new Molecule());
    m->sys = lio::system_from_molecule(mol);
    m->ang.x.assign(mol->ang_x, mol->ang_x + mol->nang);
    m->ang.y.assign(mol->ang_y, mol->ang_y + mol->nang);
    m->ang.z.assign(mol->ang_z, mol->ang_z + mol->nang);
    m->ang.w.assign(mol->ang_w, mol->ang_w + mol->nang);
    m->opt = lio::Options();
    lio::build_partition(m->sys, m->opt, m->ang, 3, m->part);
    for (int g = 0; g < m->part.total_groups(); g++) m->points += (long long)m->part.group(g).points.size();
    m->npacked = (size_t)m->sys.M * (m->sys.M + 1) / 2;
    std::lock_guard<std::mutex> g(srv->mu);
    srv->mols.push_back(std::move(m));
    return (int)srv->mols.size() - 1;
  } catch (const std::exception& e) {
    std::lock_guard<std::mutex> g(srv->mu);
    srv->error = std::string("lio_srv_add_molecule: ") + e.what();
    return -1;
  }
}

int lio_srv_molecule_info(lio_server* srv, int mol, long long* points, unsigned long long* footprint, int* resident) {
  if (!srv) return 1;
  std::lock_guard<std::mutex> g(srv->mu);
  if (mol < 0 || mol >= (int)srv->mols.size()) {
    srv->error = "lio_srv_molecule_info: no such molecule";
    return 1;
  }
  Molecule& m = *srv->mols[mol];
  if (points) *points = m.points;
  if (footprint)
    *footprint = m.measured ? m.footprint
                            : (unsigned long long)lio::DeviceEngine::estimate_device_bytes(m.sys, m.part, srv->precision, true);
  if (resident) *resident = m.engine && !m.cold ? 1 : 0;
  return 0;
}

int lio_srv_molecule_form(lio_server* srv, int mol, int* form, double* fp64_ms, double* tc_ms) {
  if (!srv) return 1;
  std::lock_guard<std::mutex> g(srv->mu);
  if (mol < 0 || mol >= (int)srv->mols.size()) {
    srv->error = "lio_srv_molecule_form: no such molecule";
    return 1;
  }
  const Molecule& m = *srv->mols[mol];
  if (form) *form = m.form;
  if (fp64_ms) *fp64_ms = m.tuned_ms[0];
  if (tc_ms) *tc_ms = m.tuned_ms[1];
  return 0;
}

long long lio_srv_submit(lio_server* srv, int mol, const double* rho_a, const double* rho_b) {
  if (!srv) return -1;
  std::unique_ptr<Request> r(new Request());
  std::lock_guard<std::mutex> g(srv->mu);
  if (mol < 0 || mol >= (int)srv->mols.size() || !rho_a || (srv->mols[mol]->sys.open && !rho_b)) {
    srv->error = "lio_srv_submit: bad molecule handle or missing density";
    return -1;
  }
  const Molecule& m = *srv->mols[mol];
  r->mol = mol;
  r->rho_a.assign(rho_a, rho_a + m.npacked);
  if (m.sys.open) r->rho_b.assign(rho_b, rho_b + m.npacked);
  r->t_submit = Clock::now();
  if (!srv->any_submit) {
    srv->any_submit = true;
    srv->t_first = r->t_submit;
  }
  const long long id = srv->next_id++;
  srv->reqs[id] = std::move(r);
  srv->queue.push_back(id);
  srv->epoch++;
  srv->cv_work.notify_one();
  return id;
}

int lio_srv_wait(lio_server* srv, long long req, double* energy, double* fock_a, double* fock_b, double* latency_ms) {
  if (!srv) return 1;
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(req);
  if (it == srv->reqs.end()) {
    srv->error = "lio_srv_wait: no such request";
    return 1;
  }
  srv->cv_done.wait(lk, [&] { return it->second->state == Request::kDone; });
  Request& r = *it->second;
  int rc = 0;
  if (!r.error.empty()) {
    srv->error = r.error;
    rc = 2;
  } else {
    if (energy) *energy = r.energy;
    if (fock_a) std::copy(r.K_a.begin(), r.K_a.end(), fock_a);
    if (fock_b && !r.K_b.empty()) std::copy(r.K_b.begin(), r.K_b.end(), fock_b);
  }
  if (latency_ms) *latency_ms = r.latency_ms;
  srv->reqs.erase(it);
  return rc;
}

int lio_srv_stats(lio_server* srv, double* out) {
  if (!srv || !out) return 0;
  std::lock_guard<std::mutex> g(srv->mu);
  std::vector<double> v = srv->lat_ms;
  std::sort(v.begin(), v.end());
  auto pct = [&](double q) {
    if (v.empty()) return 0.0;
    const size_t k = (size_t)std::min<double>((double)v.size() - 1, std::ceil(q * (double)v.size()) - 1);
    return v[k];
  };
  out[0] = (double)v.size();
  out[1] = pct(0.50);
  out[2] = pct(0.99);
  out[3] = v.empty() ? 0.0 : std::accumulate(v.begin(), v.end(), 0.0) / (double)v.size();
  out[4] = srv->points_done;
  out[5] = srv->any_submit && !v.empty() ? std::chrono::duration<double>(srv->t_last - srv->t_first).count() : 0.0;
  out[6] = (double)srv->evictions;
  out[7] = (double)srv->uploads;
  out[8] = (double)srv->peak_inflight;
  out[9] = (double)srv->oom_retries;
  out[10] = (double)srv->budget;
  return 11;
}

void lio_srv_reset_stats(lio_server* srv) {
  if (!srv) return;
  std::lock_guard<std::mutex> g(srv->mu);
  srv->lat_ms.clear();
  srv->points_done = 0.0;
  srv->any_submit = false;
  srv->evictions = srv->uploads = srv->oom_retries = 0;
  srv->peak_inflight = 0;
}

int lio_srv_plan_admission(int n, const unsigned long long* footprint, const int* busy,
                           const unsigned long long* last_use, unsigned long long budget, unsigned long long used,
                           unsigned long long need, int* evict, int* nevict) {
  std::vector<int> ev;
  const bool ok = plan_admission(n, footprint, busy, last_use, budget, used, need, ev);
  for (size_t i = 0; i < ev.size(); i++) evict[i] = ev[i];
  *nevict = (int)ev.size();
  return ok ? 1 : 0;
}

}  // extern "C"
