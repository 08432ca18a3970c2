/*
 * g2g C ABI of the B200 XC grid-integration library (lio_b200/libg2g_b200.so).
 *
 * The first block is the entry-point set lioamber's Fortran SCF/TD drivers bind
 * (Fortran name mangling: lower case + trailing underscore, every scalar passed
 * by reference, `bool` is one byte read from a Fortran LOGICAL). Each entry
 * cites the reference function it replaces; argument meaning, array layouts and
 * output semantics are the reference's:
 *   - the caller owns every array; the library keeps the pointers it is given
 *     at g2g_parameter_init_ and re-reads the density at every solve;
 *   - the Kohn-Sham (Fock) output is ACCUMULATED (+=) into the caller's packed
 *     vector(s); the energy is OVERWRITTEN;
 *   - packed storage is the lower triangle in Fortran 'L' order, packed index
 *     of 0-based (i <= j) = i*M - i*(i-1)/2 + (j-i); densities carry doubled
 *     off-diagonal elements, Fock vectors do not.
 * The library never throws or exits across this boundary: failures set a sticky
 * status readable through g2g_last_error_ (an addition; the reference throws
 * std::runtime_error or calls exit(1)).
 *
 * The second block holds additions with no counterpart in the reference ABI.
 */
#ifndef LIO_B200_G2G_H
#define LIO_B200_G2G_H

#ifdef __cplusplus
#include <cstddef>
extern "C" {
#else
#include <stdbool.h>
#include <stddef.h>
#endif

/* ---- entry points of the reference ABI ---------------------------------- */

/* g2g/init.cpp:38-61 (g2g_init_): device discovery. */
void g2g_init_(void);

/* g2g/init.cpp:409-433 (g2g_set_options_): free_global_memory, little_cube_size,
 * sphere_radius, assign_all_functions, energy_all_iterations,
 * remove_zero_weights, min_points_per_cube, max_function_exponent, timer level,
 * verbose. */
void g2g_set_options_(double* fort_fgm, double* fort_lcs, double* fort_sr,
                      bool* fort_aaf, bool* fort_eai, bool* fort_rzw,
                      unsigned int* fort_mppc, unsigned int* fort_mfe,
                      unsigned int* fort_time, unsigned int* fort_verbose);

/* g2g/init.cpp:69-219 (g2g_parameter_init_): binds the caller's arrays.
 * r: natom x 3 column-major, leading dimension max_atoms (bohr).
 * Rm, Nr, Nr2: indexed by atomic number (0..54). Iz, Nuc, ncont: 1-based.
 * c, a: M x 13 column-major, leading dimension ngaussians.
 * nshell[0] = #s, nshell[1] = 3 * #p, nshell[2] = 6 * #d.
 * e/e2/e3: 50/116/194 x 3 column-major angular directions; wang/wang2/wang3
 * their weights (already multiplied by 4*pi). */
void g2g_parameter_init_(const unsigned int* norm, const unsigned int* natom,
                         const unsigned int* max_atoms, const unsigned int* ngaussians,
                         double* r, double* Rm, const unsigned int* Iz,
                         const unsigned int* Nr, const unsigned int* Nr2,
                         unsigned int* Nuc, const unsigned int* M, unsigned int* ncont,
                         const unsigned int* nshell, double* c, double* a,
                         double* rho_vec, double* fock_vec, double* fockb_vec,
                         double* rhoalpha, double* rhobeta, const unsigned int* nco,
                         bool* OPEN, const unsigned int* nunp, const unsigned int* nopt,
                         const unsigned int* Iexch, double* e, double* e2, double* e3,
                         double* wang, double* wang2, double* wang3, bool* use_libxc,
                         const unsigned int* ex_functional_id,
                         const unsigned int* ec_functional_id);

/* g2g/init.cpp:282-306 (g2g_reload_atom_positions_): re-reads the positions
 * and rebuilds the grid partition for grid_type (0/1/2 -> 50/116/194 points;
 * types >= 3 are tables registered with g2g_set_angular_grid_). */
void g2g_reload_atom_positions_(const unsigned int* grid_type);

/* g2g/init.cpp:308-315 (g2g_new_grid_): rebuilds only if grid_type changed. */
void g2g_new_grid_(const unsigned int* grid_type);

/* g2g/init.cpp:332-391 (g2g_solve_groups_): computation_type 0 = Fock (RMM)
 * update, 1 = energy only, 2 = energy + forces, 3 = forces only. The energy is
 * written (0 when not computed); the Kohn-Sham vectors bound at parameter_init
 * are added to (type 0 only); types 2 and 3 add each atom's XC force into
 * fort_forces_ptr, natoms x 3 column-major with leading dimension max_atoms
 * (g2g/partition.cpp:516-526), with the reference's CPU formula
 * (g2g/cpu/iteration.cpp:213-267, open shell 496-563) from the per-point
 * factors of the build (whose form set_precision selects): G = P F in FP64 in
 * the FP64 form (and for LDA), on tcgen05 from the build's own int8 slices in
 * the tensor-core form, the gradient dots and sums in FP64 in both. */
void g2g_solve_groups_(const unsigned int* computation_type, double* fort_energy_ptr,
                       double* fort_forces_ptr);

/* g2g/init.cpp:221-236 (g2g_deinit_): releases the partition and device state. */
void g2g_deinit_(void);

/* g2g/timer.cpp:125-296: Fortran-named timers (hidden length argument). */
void g2g_timer_start_(const char* timer_name, unsigned int length_arg);
void g2g_timer_stop_(const char* timer_name, unsigned int length_arg);
void g2g_timer_pause_(const char* timer_name, unsigned int length_arg);
void g2g_timer_sum_start_(const char* timer_name, unsigned int length_arg);
void g2g_timer_sum_stop_(const char* timer_name, unsigned int length_arg);
void g2g_timer_sum_pause_(const char* timer_name, unsigned int length_arg);
void g2g_timer_clear_(void);
void g2g_timer_summary_(void);

/* ---- additions (no counterpart in the reference ABI) --------------------- */

/* Sticky status of the last failing call: 0 = ok. Copies up to len-1 bytes of
 * the message into msg (NUL-terminated) when msg != NULL. Reading clears it. */
int g2g_last_error_(char* msg, const unsigned int* len);

/* Registers an angular table for grid_type >= 3 (e: npoints x 3 column-major
 * unit directions, wang: weights summing to 4*pi); such grid types use the
 * Nr2 radial shell counts, as grid types 1 and 2 do. The reference supports
 * only its three compiled-in tables (g2g/init.h:10-14, g2g/init.cpp:238-266). */
void g2g_set_angular_grid_(const unsigned int* grid_type, const unsigned int* npoints,
                           const double* e, const double* wang);

/* Arithmetic of the two contractions (density and Kohn-Sham update):
 * 0 = FP64 on the CUDA cores (the plain form), 1 = tensor-core form (a grid it
 * cannot run is refused with an error), 2 = autotuned: after each grid upload
 * one build of each form is timed and the faster kept (both meet the accuracy
 * bar; small molecules, whose function tiles are mostly padding, often run
 * faster in FP64), 3 = the default for a caller that never calls this: the
 * tensor-core form, with the FP64 form for a grid the tensor-core form cannot
 * run (a point group above 87,296 padded points, or more significant
 * functions in one group than a block's shared memory holds). */
void g2g_set_precision_(const unsigned int* mode);

/* Lean tensor-core form (no reference counterpart): *on != 0 releases the
 * blocked FP64 basis values once the tensor-core operands are built (about a
 * third of the form's device footprint for GGA). The Kohn-Sham contraction then
 * forms the basis values it needs from the per-shell radial sums, and a force
 * request (g2g_solve_groups_ types 2/3) rebuilds the blocked values for its
 * call. Off by default; applies to the current grid at once and to later ones. */
void g2g_set_lean_(const unsigned int* on);

/* Partition statistics of the current grid: out[0] = groups, out[1] = cubes,
 * out[2] = spheres, out[3] = points kept, out[4] = sum over groups of
 * points * functions, out[5] = sum of points * functions^2. */
void g2g_partition_stats_(long long* out);

/* Copies group g of the current partition (groups numbered cubes first, then
 * spheres, each in cost order): meta[0..7] = points, simple functions, s, p, d,
 * total functions, nuclei, is_sphere; when non-NULL, ids (points x 3: atom,
 * shell, angular point), xyzw (points x 4: x, y, z, weight), funcs (simple
 * functions, 0-based global index of the first component). Returns 0 or -1. */
int g2g_partition_group_(const int* g, int* meta, int* ids, double* xyzw, int* funcs);

/* Device time of the last g2g_solve_groups_ (ms, CUDA events around the
 * device work) and of the last partition build (ms, host clock). */
void g2g_last_timings_(double* solve_ms, double* grid_ms);

/* No counterpart in the reference: wall ms of the last grid build's phases:
 * phase_ms[0] the partition (grid, screening, Becke weights, ordering),
 * phase_ms[1] the device upload (arrays, basis values), phase_ms[2] the
 * autotuner (precision mode 2; else 0). */
void g2g_grid_timings_(double* phase_ms);

/* Runs all device work of this library on the given cudaStream_t. NULL (the
 * legacy default stream's handle) selects the library's own non-blocking
 * stream, which does not order with the legacy default stream. */
void g2g_set_stream_(void* cuda_stream);

/* Device-resident solve: same work as g2g_solve_groups_(0) on the density that
 * the last g2g_solve_groups_ uploaded, with the Kohn-Sham accumulator and the
 * energy left in device memory and no host synchronisation (for callers that
 * keep the SCF state on the GPU, and for throughput measurement). Returns the
 * number of kernel launches it enqueued. */
int g2g_solve_resident_(void);

/* No counterpart in the reference, whose multi-GPU form shards groups inside
 * one process (g2g/partition.cpp:441-511) and sums on the host (:516-574).
 * Multi-GPU here is one process per GPU: g2g_set_shard_(rank, world) before a
 * grid build makes this process upload and solve only its share of the groups
 * (cost-balanced, longest processing time first on the reference's group cost);
 * g2g_solve_groups_ then returns this share's E_xc and adds this share's
 * Kohn-Sham contribution, and the caller sums both over the ranks (one
 * all-reduce). g2g_shard_groups_ writes the owner rank of every group of the
 * current partition (cubes, then spheres) and returns the group count.
 * g2g_copy_resident_results_ copies the last resident solve's Kohn-Sham
 * matrices (packed, per spin; beta may be NULL for closed shell) and energy
 * into caller device buffers on the library's stream, for a device-side
 * all-reduce. */
void g2g_set_shard_(const int* rank, const int* world);
int g2g_shard_groups_(const int* world, int* owner);
void g2g_copy_resident_results_(double* d_fock_a, double* d_fock_b, double* d_energy);

/* No counterpart in the reference: replay each solve's kernels from a CUDA
 * graph captured on the first solve after a new grid or precision (on by
 * default; 0 launches the kernels one by one). Profiled solves always launch
 * them one by one. */
void g2g_set_graphs_(const unsigned int* on);

/* Per-stage device timing with CUDA events recorded between the stages of
 * every solve. g2g_profile_(on) resets the sums; g2g_stage_times_ writes the
 * accumulated ms of five stages into ms[0..4]: 0 = density operand preparation
 * (the int8 slices of the density matrices; empty in the FP64 form), 1 = density
 * contraction, 2 = point functional and energy sum, 3 = Kohn-Sham operand
 * preparation (slices of f*F; empty in the FP64 form), 4 = Kohn-Sham
 * contraction, and the number of solves timed. Returns the number of stages. */
void g2g_profile_(const unsigned int* on);
int g2g_stage_times_(double* ms, int* solves);

/* No counterpart in the reference: external accumulators for device-resident
 * solves (g2g_solve_resident_). With device pointers set, each resident
 * solve's Kohn-Sham contraction adds (+=) its contributions into d_fock_a
 * (and d_fock_b for open shell) with its own FP64 atomics, and its E_xc into
 * *d_energy, instead of into the engine's buffers; the caller zeroes them. The
 * shards of a build (g2g_set_shard_) on several GPUs can all be given one
 * GPU's buffers, mapped into every process over NVLink (CUDA IPC or symmetric
 * memory), so that the contraction itself performs the cross-GPU sum and no
 * separate all-reduce follows. All three NULL: off. Replaces the result
 * buffers of g2g_copy_resident_results_ while set. */
void g2g_set_accumulators_(double* d_fock_a, double* d_fock_b, double* d_energy);

/* No counterpart in the reference: where the Becke weights of a grid build
 * (g2g_reload_atom_positions_, g2g_new_grid_) are computed. 1 (default): on
 * the GPU when one is present, one thread per point with explicitly rounded
 * FP64 operations in the reference's order, so the partition is the same bit
 * for bit; 0: on the host cores (OpenMP), as g2g/cpu/weight.cpp:13-112 does. */
void g2g_set_device_weights_(const unsigned int* on);

/* No counterpart in the reference: device ms of the force kernel of the last
 * g2g_solve_groups_ type 2 or 3 call (CUDA events around it; the build before
 * it is not included), or -1 without a device engine. */
double g2g_last_force_ms_(void);

/* No counterpart in the reference: bytes the last g2g_solve_groups_ moved
 * between the caller's arrays and the device (h2d: density values; d2h:
 * Kohn-Sham values and the energy). When the point groups touch at most half
 * of the packed matrix, only those entries travel: the density's are gathered
 * from the caller's vector and scattered on the device, the Kohn-Sham
 * contributions gathered on the device and added into the caller's vector
 * (every other entry's XC contribution is zero). */
void g2g_last_transfer_bytes_(long long* h2d, long long* d2h);

/* No counterpart in the reference: an XC build that allocates no device
 * memory, for callers that cannot call cudaMalloc (a host program whose
 * allocator already owns all of the GPU's memory, or code that must not
 * allocate while it runs). It performs the work of g2g_solve_groups_(0) on the
 * current grid with device pointers: d_rho_a (closed shell: the packed total
 * density; open shell: alpha) and d_rho_b (open shell: beta, else NULL) in the
 * packed, doubled-off-diagonal layout; d_fock_a/d_fock_b receive the packed
 * Kohn-Sham contributions ACCUMULATED (+=); d_energy (one double) is
 * overwritten with E_xc. Every intermediate lives in one fixed 32 MiB device
 * array inside the library (held by each GPU that loads it until the process
 * exits); groups are processed in batches that fit, and a grid whose single
 * largest group does not fit is rejected with an error (status -1, message in
 * g2g_last_error_). The first call on a device looks up that array's device
 * address (with the device current); make that first call before any stream
 * capture. All calls share the array: calls that overlap on the GPU (on
 * different streams or from different threads) race and corrupt each other.
 * The grid itself (points, basis values) must already be resident, built by
 * g2g_reload_atom_positions_ in the FP64 form (g2g_set_precision_(0) before
 * the grid build): the tensor-core form, the default, does not keep the FP64
 * basis values this path reads, and since building them would allocate, the
 * call is then refused with an error rather than run. stream: a cudaStream_t,
 * or NULL for the library's own stream. Returns 0 on success. */
int g2g_solve_device_noalloc_(const double* d_rho_a, const double* d_rho_b, double* d_fock_a,
                              double* d_fock_b, double* d_energy, void* stream);

/* Failure-path self-test (no counterpart in the reference, which aborts with
 * exit(1) on a failed build, g2g/partition.cpp:584-590). Every wait of the
 * pipelined tensor-core kernels on an mbarrier is bounded; when one runs out,
 * the kernel records the failure, lets its copies in flight land, frees its
 * TMEM and returns, and the host reports an error instead of hanging. This
 * runs that path on purpose: a one-CTA kernel whose producer arms and sends
 * the first of two ring stages and then stops, while the consumer waits for
 * both with a limit of *polls polls. Returns 1 when the second wait ran out
 * as intended (then the sticky status is 3 and g2g_last_error_ carries the
 * message), 0 if it did not run out, -1 on an error; *ms gets the kernel's
 * device time. The GPU context stays usable for the next build. */
int g2g_selftest_bounded_wait_(const unsigned int* polls, double* ms);

/* Diagnostic (no counterpart in the reference): runs one tcgen05 int8 tensor-
 * core product D[128 x N] = A[128 x K] * B[N x K]^T (row-major host arrays,
 * 16 <= N <= 256 with N % 16 == 0, 32 <= K <= 256 with K % 32 == 0) so the
 * shared-memory descriptor and TMEM layouts can be checked exactly. Returns 0
 * on success, 1 if the completion wait timed out, < 0 on a setup error. */
int lio_tc_selftest_(int N, int K, const signed char* A, const signed char* B, int* D);

#ifdef __cplusplus
}
#endif
#endif /* LIO_B200_G2G_H */
