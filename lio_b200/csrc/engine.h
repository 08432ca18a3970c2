// Device engine for the XC grid integration (one molecule, one GPU).
//
// Host code hands it a built partition once per geometry (upload_partition)
// and then calls solve() once per SCF/TD step with the caller's packed density
// matrices; solve() accumulates the Kohn-Sham (Fock) contributions into the
// caller's packed vectors and returns E_xc. No CUDA types appear here so the
// C-ABI layer compiles with the host compiler.
#pragma once
#include <cstddef>
#include <memory>
#include <string>
#include <vector>

#include "partition.h"
#include "system.h"

namespace lio {

enum class Precision { FP64 = 0, TensorCore = 1 };

struct SolveRequest {
  bool compute_rmm = true;      // accumulate into the Fock vector(s)
  bool compute_energy = true;
  const double* rho = nullptr;  // closed shell: packed total density (doubled off-diagonals)
  const double* rho_a = nullptr;  // open shell
  const double* rho_b = nullptr;
  double* fock = nullptr;       // closed shell, or alpha when open
  double* fock_b = nullptr;     // open shell beta
  // Device-resident mode: reuse the density already on the device, leave the
  // Kohn-Sham accumulator and the energy on the device, do not synchronise.
  bool resident = false;
};

struct SolveResult {
  double energy = 0.0;
  double device_ms = 0.0;
};

// One molecule of a batch uploaded as one system (DeviceEngine::upload with
// `batch`): its functions are [f_off, f_off + M) of the joined system's, its
// packed density and Kohn-Sham matrices occupy [pk_off, pk_off + M(M+1)/2) of
// the engine's vectors, and its point groups are [g_begin, g_end) of the
// joined partition (each molecule's groups one after the other).
struct BatchMember {
  int f_off = 0, M = 0;
  long long pk_off = 0;
  int g_begin = 0, g_end = 0;
};

class DeviceEngine {
 public:
  DeviceEngine();
  ~DeviceEngine();
  DeviceEngine(const DeviceEngine&) = delete;
  DeviceEngine& operator=(const DeviceEngine&) = delete;

  // Uploads basis parameters, points and function lists and evaluates the
  // basis values; with `keep`, only the groups g with (*keep)[g] (this rank's
  // shard of a multi-GPU build).
  // With `batch`, the system and partition join several molecules (see
  // BatchMember): one set of kernel launches per stage covers all of them, the
  // density and Kohn-Sham vectors of solve() are the molecules' packed
  // matrices one after the other, and batch_energies() gives each one's E_xc.
  void upload(const System& sys, const Partition& part, const std::vector<char>* keep = nullptr,
              const std::vector<BatchMember>* batch = nullptr);
  // E_xc of every batch member in the last host-array solve; returns their number
  int batch_energies(double* out) const;
  // elements of the packed density / Kohn-Sham vectors per spin
  size_t packed_size() const;
  // One XC build: enqueue() puts all of its device work on the engine's stream
  // (density upload unless resident, the kernels, result download into pinned
  // buffers) and returns; ready() polls it; finish() waits for it and delivers
  // the outputs (Kohn-Sham += into req.fock / fock_b, E_xc). solve() = both.
  // One solve in flight per engine.
  void enqueue(const SolveRequest& req);
  bool ready() const;
  SolveResult finish(const SolveRequest& req);
  SolveResult solve(const SolveRequest& req);
  // XC nuclear gradients (g2g_solve_groups_ types 2 and 3): a build without
  // the Kohn-Sham accumulation (E_xc and the per-point factors, in the current
  // form), then each atom's XC force from those factors (G = P F in FP64, or
  // on tcgen05 from the build's int8 slices in the tensor-core GGA form), added
  // (+=) into forces[atom + ld * axis] (the caller's natoms x 3 column-major array).
  SolveResult solve_forces(const SolveRequest& req, double* forces, int ld);
  // device ms of the last solve_forces' force kernel (CUDA events around it)
  double last_force_kernel_ms() const;
  // bytes the last host-array solve moved: densities in, Kohn-Sham values (and
  // the energy) out; only the packed entries the groups touch when those are at
  // most half of the matrix
  void last_transfer_bytes(long long* h2d, long long* d2h) const;
  // External accumulators for resident solves (nullptr: off): the Kohn-Sham
  // contraction's FP64 atomics and the energy sum add (+=) into these device
  // buffers, which the caller zeroes, instead of the engine's own. Shards of a
  // build on several GPUs can all add into one GPU's buffers, mapped into each
  // process over NVLink, so the contraction itself does the cross-GPU sum.
  void set_accumulators(double* d_fock_a, double* d_fock_b, double* d_energy);
  // Replay the kernels of a solve from a CUDA graph captured on first use
  // (re-captured after a new geometry or precision).
  void set_graphs(bool on);
  void set_precision(Precision p) {
    if (p != precision_) set_graphs_dirty();
    precision_ = p;
  }
  // Stream for all device work (nullptr: the engine's own stream).
  void set_stream(void* cuda_stream);
  // Kernel launches of one solve (for launch accounting).
  int launches_per_solve() const;
  // Per-stage device timing (CUDA events between the stages of every solve):
  // five stages (density operands, density contraction, functional and energy,
  // Kohn-Sham operands, Kohn-Sham contraction), accumulated over solves until reset.
  void set_profiling(bool on);
  int stage_times(double* ms, int max_stages, int* solves) const;
  Precision precision() const { return precision_; }
  void release();

  // Device-pointer solve that allocates nothing: every per-solve scratch
  // buffer lives in one file-scope __device__ array of kNoAllocScratchBytes
  // (engine.cu); groups are processed in batches that fit it. Inputs: packed
  // densities in device memory (rho_b only for open shell). Outputs: packed
  // Kohn-Sham vectors in device memory, accumulated (+=); the energy (one
  // double in device memory) is overwritten. Throws on sizes beyond the array,
  // and when the FP64 form's basis cache is not resident (a grid built or
  // autotuned in the tensor-core form): rebuilding it would allocate.
  void solve_noalloc(const double* rho_a, const double* rho_b, double* fock_a, double* fock_b,
                     double* energy, void* cuda_stream);
  static size_t noalloc_scratch_bytes();

  // true when a CUDA device can be used from this process
  static bool available();
  // Becke weights of a partition being built, on the current device: the
  // bit-exact device form of host_becke_weights (partition.h), for
  // build_partition's `weights` argument.
  static void becke_weights(const System& sys, const std::vector<PointGroup*>& groups, bool drop_zero);
  // builds the current form's per-geometry caches now (tensor-core operands or
  // the FP64 basis cache; otherwise the next solve does)
  void prepare();
  // releases the per-geometry caches (basis values, tensor-core operands), the
  // bulk of a molecule's device bytes; the grid, tiles and per-solve buffers stay
  // and the next prepare() or solve rebuilds the caches on the device
  void release_caches();
  // device bytes release_caches() would free
  size_t cache_bytes() const;
  // Times one build of this molecule in each form, keeps the faster (both meet
  // the accuracy bar; memory_aware: the smaller time x device-bytes product)
  // and releases the other's device buffers; returns it.
  Precision autotune(bool memory_aware = false);
  // The autotuner's measurement alone: ms per resident build of each form and
  // the bytes of each form's per-geometry caches; leaves the tensor-core form
  // active. keep_form() then keeps one form and releases the other's caches.
  void autotune_measure(double* fp64_ms, double* tc_ms, size_t* fp64_cache, size_t* tc_cache);
  void keep_form(Precision p);
  void tuned_times(double* fp64_ms, double* tc_ms) const;
  // releases the tensor-core operands (rebuilt by the next tensor-core solve)
  void drop_tensor_core();
  // device-to-device copy of the last resident solve's Kohn-Sham matrices and
  // energy into caller buffers, on the engine's stream
  void copy_results(double* d_fock_a, double* d_fock_b, double* d_energy);
  // device bytes held by all engines of the process, and an estimate of one
  // molecule's footprint before it is uploaded
  static long long process_device_bytes();
  // (lean: without the blocked basis, which a lean engine keeps only while it builds its operands)
  static size_t estimate_device_bytes(const System& sys, const Partition& part, Precision prec, bool lean = false);
  // lean: once the tensor-core operands are built the blocked FP64 basis is
  // released (about a third of the form's footprint for GGA); the Kohn-Sham
  // kernels then form F from the radial sums, and forces rebuild the blocked
  // basis for their call. Its size, which a lean engine still needs while it
  // builds its operands:
  void set_lean(bool on);
  bool lean() const;
  static size_t estimate_blocked_basis_bytes(const System& sys, const Partition& part);

  // statistics of the uploaded partition
  long long points() const;
  long long groups() const;

 private:
  void prepare_tensor_core();
  int run_kernels(bool compute_rmm, bool ext = false);
  void set_graphs_dirty();
  struct Impl;
  std::unique_ptr<Impl> impl_;
  Precision precision_ = Precision::FP64;
};

// Self-test of the bounded waits of the pipelined tensor-core kernels (a
// producer that stops early, one consumer wait of `polls` polls that runs out);
// returns 1 when that wait timed out and the kernel returned (0 would mean both
// stages arrived, 2 that even the armed stage did not), the device ms in *ms
// and a checksum of the stage that did land (32640 for its 256 values 0..255)
int bounded_wait_selftest(unsigned polls, double* ms, unsigned* checksum);

}  // namespace lio
