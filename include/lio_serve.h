/* Handle-based XC build service: many molecules resident on one GPU, XC builds
 * submitted as requests and run with continuous batching.
 *
 * No counterpart in the reference, whose g2g keeps one molecule in process-
 * global state (g2g/init.cpp:27-33, `fortran_vars` and `::partition`) and runs
 * one synchronous build per g2g_solve_groups_ call (g2g/init.cpp:332-391). The
 * Fortran ABI of g2g.h stays the thin single-molecule wrapper; this API adds:
 *
 *   - molecule handles: each molecule's grid, partition, basis values and
 *     tensor-core operands are built once and kept on the device (resident);
 *   - requests: (molecule, density matrices) -> (E_xc, Kohn-Sham matrices),
 *     the same computation as g2g_solve_groups_(0) with energy on, but the
 *     Kohn-Sham output is written (=) into the request's result, not added;
 *   - continuous batching: a worker thread admits queued requests whenever a
 *     molecule is idle and the in-flight count allows, so requests that arrive
 *     while others run start at once and overlap with them on the GPU (one
 *     CUDA stream per resident molecule);
 *   - admission by HBM footprint: a molecule is made resident only when its
 *     device footprint fits the server's byte budget, evicting idle resident
 *     molecules least recently used first — their basis-value and tensor-core
 *     caches first (the molecule keeps its grid and rebuilds them on the device
 *     when next needed), whole molecules only if that is not enough; a request
 *     waits in the queue until its molecule fits. Evictions and uploads run on
 *     a loader thread, so builds of resident molecules continue meanwhile.
 *
 * Every call returns a status (0 = success) or a handle >= 0; on failure the
 * message is read with lio_srv_last_error. Calls are thread-safe; results are
 * identical (within floating-point summation order of the Kohn-Sham atomics)
 * whether a request runs alone or among others.
 */
#ifndef LIO_SERVE_H
#define LIO_SERVE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct lio_server lio_server;

/* One molecule with its basis, functional and angular grid. Positions in bohr.
 * Functions in LIO order: all s, then p (x,y,z consecutive), then d (xx, xy,
 * yy, xz, yz, zz), as g2g_parameter_init_ receives them
 * (g2g/init.cpp:100-104); nuc is 0-based here. a and c are M x 13 row-major
 * (primitive k of function i at [i * 13 + k]). rm and shells are per atom. */
typedef struct lio_molecule {
  int natoms;
  const double* xyz;        /* natoms x 3, row-major */
  const int* atomic_number; /* per atom */
  const double* rm;         /* per atom: the Becke radius the reference takes from Rm[Iz] */
  const unsigned* shells;   /* per atom: radial shells (Nr2[Iz] of the reference) */
  int M;
  const int* nuc;           /* per function, 0-based atom */
  const int* ncont;         /* per function, primitives (<= 13) */
  const double* a;          /* M x 13 exponents */
  const double* c;          /* M x 13 contraction coefficients */
  int s_funcs, p_funcs, d_funcs; /* simple function counts (a p counts once, not three times) */
  int normalize;            /* 1: d xx, yy, zz carry 1/sqrt(3) (LIO's norm) */
  int iexch;                /* 1-3: LDA; 4-9: GGA (4 P86, 5 B88+P86, 6 B88+VWN, 7 BLYP, 8 P86+LYP, 9 PBE; open shell: PBE) */
  int open;                 /* 1: open shell (alpha and beta densities) */
  int nang;                 /* angular grid: points and unit directions/weights (sum 4 pi) */
  const double *ang_x, *ang_y, *ang_z, *ang_w;
} lio_molecule;

/* A server on `device`. hbm_budget_bytes = 0 takes 90% of the free device
 * memory. precision: 0 FP64 form, 1 tensor-core form, 2 autotuned per molecule
 * (one build of each form timed at the molecule's first upload; the form with
 * the smaller time x device-bytes product is kept, so residency is not spent on
 * little speed). max_inflight: requests on the GPU at once (0 = 16). */
lio_server* lio_srv_create(int device, unsigned long long hbm_budget_bytes, int precision, int max_inflight);
void lio_srv_destroy(lio_server* srv);
const char* lio_srv_last_error(lio_server* srv);

/* Registers a molecule: copies its description and builds its grid partition
 * on the host (bit-exact with g2g_reload_atom_positions_). Device residency is
 * decided at admission. Returns the molecule handle, or -1. */
int lio_srv_add_molecule(lio_server* srv, const lio_molecule* mol);
/* Points of the molecule's grid and its device footprint in bytes (estimated
 * until it has been resident once, measured after). */
int lio_srv_molecule_info(lio_server* srv, int mol, long long* points, unsigned long long* footprint_bytes,
                          int* resident);

/* The form a molecule runs in (0 FP64, 1 tensor core, -1 not yet uploaded)
 * and, when autotuned, the measured ms per build of each form. */
int lio_srv_molecule_form(lio_server* srv, int mol, int* form, double* fp64_ms, double* tc_ms);

/* Submits one XC build. Closed shell: rho_a = the packed total density
 * (doubled off-diagonal elements, as rho_vec of g2g_parameter_init_), rho_b
 * ignored. Open shell: rho_a, rho_b = the packed alpha and beta densities. The
 * densities are copied before the call returns. Returns the request handle (>= 0) or -1. */
long long lio_srv_submit(lio_server* srv, int mol, const double* rho_a, const double* rho_b);
/* Blocks until the request is done; writes E_xc and the packed Kohn-Sham
 * matrices (fock_b only for open shell; either pointer may be NULL). Returns 0,
 * or a nonzero status with the request's error in lio_srv_last_error. The
 * request handle is released. latency_ms (optional) receives submit-to-done time. */
int lio_srv_wait(lio_server* srv, long long req, double* energy, double* fock_a, double* fock_b, double* latency_ms);

/* Service statistics since creation or the last reset: out[0] completed
 * requests, out[1] p50 latency ms, out[2] p99 latency ms, out[3] mean latency
 * ms, out[4] grid points processed, out[5] wall seconds from the first
 * submission to the last completion, out[6] evictions (whole molecules or their
 * caches), out[7] uploads (or cache rebuilds), out[8] peak requests in flight,
 * out[9] loads retried after the device ran out of memory (each shrinks the
 * budget), out[10] the current HBM budget in bytes. out must hold 11 values;
 * returns the number written (11). */
int lio_srv_stats(lio_server* srv, double* out);
void lio_srv_reset_stats(lio_server* srv);

/* Test hook for the admission policy alone (no device): given resident
 * molecules' footprints, busy flags and last-use ticks, the budget and the
 * bytes in use, decides whether a molecule of `need` bytes can be admitted and
 * which residents to evict (least recently used idle ones first). Writes up to
 * n indices into evict and their count into nevict; returns 1 if admissible. */
int lio_srv_plan_admission(int n, const unsigned long long* footprint, const int* busy,
                           const unsigned long long* last_use, unsigned long long budget,
                           unsigned long long used, unsigned long long need, int* evict, int* nevict);

/* ---- many molecules per launch --------------------------------------------
 * No counterpart in the reference, whose CPU path runs the point groups of one
 * molecule in one OpenMP loop (g2g/partition.cpp:441-511). A batch joins many
 * molecules into one device layout per functional class (LDA or GGA, closed or
 * open shell, one iexch): the point groups of all its molecules form one tile
 * list, so each stage of an XC build (density operands, density contraction,
 * functional, Kohn-Sham operands and contraction) is one kernel launch for the
 * whole class, however small its molecules. Each group carries its molecule's
 * packed-matrix dimension and offset; the densities of the molecules are read
 * from, and their Kohn-Sham matrices added into, one concatenated vector per
 * spin, and each molecule's E_xc is summed from its own groups' partials.
 *
 * lio_batch_create builds every molecule's grid and partition (host threads,
 * Becke weights on the host) and uploads one engine per class to `device`;
 * precision 0 FP64, 1 tensor core, 2 the faster of both per class (timed once).
 * It returns NULL on failure (message in lio_batch_create_error).
 * lio_batch_solve runs one XC build of every molecule: rho_a[i] (closed shell:
 * the packed total density; open shell: alpha) and rho_b[i] (open shell: beta,
 * else ignored) are molecule i's packed densities (doubled off-diagonals), its
 * packed Kohn-Sham matrices are WRITTEN (=) into fock_a[i] / fock_b[i] and its
 * E_xc into energies[i]; the classes run concurrently on their own streams.
 * *device_ms (optional) receives the sum over classes of their device time.
 * Returns 0, or a nonzero status with the message in lio_batch_last_error.
 * lio_batch_stats writes the grid points of all molecules, the number of
 * classes, the seconds the grids and uploads took and, per class (up to
 * max_classes), its form (0 FP64, 1 tensor core) and molecule count. */
typedef struct lio_batch lio_batch;
lio_batch* lio_batch_create(int device, int nmol, const lio_molecule* mols, int precision);
const char* lio_batch_create_error(void);
int lio_batch_solve(lio_batch* b, const double* const* rho_a, const double* const* rho_b, double* const* fock_a,
                    double* const* fock_b, double* energies, double* device_ms);
const char* lio_batch_last_error(lio_batch* b);
int lio_batch_stats(lio_batch* b, long long* points, int* nclasses, double* build_s, int max_classes, int* form,
                    int* members);
void lio_batch_destroy(lio_batch* b);

#ifdef __cplusplus
}
#endif
#endif
