// Device engine: HBM layout, kernels and per-solve orchestration (FP64 form).
//
// HBM layout of one molecule (built once per geometry by upload()):
//   groups[]      GroupDev records, cubes first then spheres (cost order)
//   px/py/pz/pw   point coordinates and weights, each group padded to ldp
//                 (a multiple of 64) slots; padded slots have weight 0
//   fn_glob[]     per group, the global (expanded) index of every local function
//   sf_glob/type  per group, its simple functions (s, p shell, d shell)
//   basis cache   per group NK x m x ldp doubles, function-major (points
//                 contiguous): NK = 1 (F) for LDA, 10 for GGA
//                 (F, dx, dy, dz, dxx, dyy, dzz, dxy, dxz, dyz)
// Per solve: packed density(ies) uploaded, partial densities per
// (function tile, quantity, point), per-point factors w*v_xc, the packed
// Kohn-Sham accumulator (FP64) and per-block energy partials.
//
// Math (g2g/cpu/iteration.cpp:90-291 restated as GEMMs): with D the dense
// symmetric group density (packed value, halved off the diagonal),
//   G = F D, Ga = (dF/da) D                               (tensor-shaped)
//   rho = sum_i F_i G_i, d rho/da = 2 sum_i dF_i/da G_i,
//   d2 rho/da db = 2 sum_i (d2F_i/da db G_i + dF_i/da Gb_i)  (row-dot epilogue)
//   K_ij += sum_p F_ip (w_p v_p) F_jp                      (tensor-shaped)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <cstdint>
#include <mutex>
#include <vector>

#include "engine.h"
#include "xc_functionals.cuh"

namespace lio {

#define LIO_CUDA(x)                                                                           \
  do {                                                                                        \
    cudaError_t err_ = (x);                                                                   \
    if (err_ != cudaSuccess)                                                                  \
      throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(err_) + " at " + \
                               __FILE__ + ":" + std::to_string(__LINE__));                    \
  } while (0)

namespace {

constexpr int kTile = 64;    // points / functions per GEMM tile
constexpr int kPointPad = 128;  // points per group padded to a multiple of this
constexpr int kTcChunkElems = 32 * 128;  // doubles of one (kind, 32-function, 128-point) block of the blocked basis
constexpr int kKStep = 16;   // reduction step of the FP64 GEMMs
constexpr int kBasisBlock = 128;
constexpr int kFuncBlock = 128;
constexpr int kNQ = 10;      // rho, grad[3], (xx,yy,zz), (xy,xz,yz)

struct GroupDev {
  int npts, ldp, m, nsimple;
  int nft, m32, nftc, pad2;  // m32: m rounded up to 32; nftc: 32-function tensor-core density tiles
  long long pt_off;    // point arrays
  long long fn_off;    // fn_glob, fn_sh, fn_cp
  long long sf_off;    // sf_glob / sf_type
  long long bas_off;   // basis cache (elements)
  long long part_off;  // partial densities (elements, one spin)
  long long bb_off;    // blocked FP64 basis of the tensor-core density (elements)
  long long sl_off;    // int8 slices of the density A operands (bytes)
  long long aexp_off;  // their per-point exponents (elements): NA x ldp
  long long ds_off;    // int8 slices of the density matrix (bytes, one spin)
  long long dexp_off;  // their exponents (elements): nftc x 32, one value per 32-function tile
  long long fa_off;    // int8 slices of F by function row for the Kohn-Sham contraction (bytes)
  long long fae_off;   // their per-row exponents (elements): nI x 128
  long long fbe_off;   // per-row exponents of f*F (elements): nJ x 32
  long long rad_off;   // radial sums of the tensor-core density (elements): per 128-point tile, shell, NR values
  // the packed density / Kohn-Sham matrices the group reads and adds into: dimension pk_M, starting at
  // element pk_off of the engine's vectors (a batch of molecules keeps one per molecule, one after the other)
  int pk_M, pk_pad;
  long long pk_off;
};

// Process-wide pinned host staging of the grid build (grow-only, one buffer per
// use, never returned until exit): a new geometry (every MD step) would
// otherwise fault in tens of bytes per point of fresh host memory and copy it
// pageable. Engines of many resident molecules share one buffer rather than
// each pinning its own; users hold the mutex while they fill and copy it.
struct PinnedStaging {
  std::mutex m;
  void* host = nullptr;
  size_t bytes = 0;
  // grows with 1/8 headroom: pinning is slow (~1 ms per 2-3 MB), and the next
  // geometry of a molecule in motion usually has a few more points
  void reserve(size_t need) {
    if (bytes >= need) return;
    if (host) cudaFreeHost(host);
    host = nullptr;
    bytes = 0;
    need += need / 8;
    const cudaError_t e = cudaMallocHost(&host, need);
    if (e != cudaSuccess) {
      cudaGetLastError();
      host = nullptr;
      throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e) + " pinning " +
                               std::to_string(need) + " bytes of host staging");
    }
    bytes = need;
  }
};
PinnedStaging& weights_staging() {  // Becke weights: points in, factors out
  static PinnedStaging* w = new PinnedStaging;  // never destroyed: no cudaFreeHost after the runtime's exit
  return *w;
}
PinnedStaging& point_staging() {  // the point arrays of an engine's upload
  static PinnedStaging* w = new PinnedStaging;
  return *w;
}

// Per device: a non-blocking stream for the grid build's host-to-device copies,
// which then overlap host work (the legacy stream's synchronous copies of other
// arrays do not wait for it). Never destroyed.
cudaStream_t copy_stream() {
  static std::mutex mu;
  static cudaStream_t streams[64] = {};
  int dev = 0;
  LIO_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw std::runtime_error("device ordinal out of range for the copy stream");
  std::lock_guard<std::mutex> lock(mu);
  if (!streams[dev]) LIO_CUDA(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking));
  return streams[dev];
}

// Waits for a copy stream when leaving a scope, normally or by an exception,
// so pinned staging is never reused, nor device buffers freed, under a copy.
struct StreamDrain {
  cudaStream_t s;
  ~StreamDrain() {
    if (cudaStreamSynchronize(s) != cudaSuccess) cudaGetLastError();
  }
};

// device bytes held by every DevBuf of the process (footprint accounting)
std::atomic<long long> g_devbuf_bytes{0};

// Device array with process-wide byte accounting. alloc() keeps the existing
// allocation when it is large enough (a new geometry of similar size reuses it:
// no cudaFree / cudaMalloc, which synchronise the device, per grid build).
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;    // elements in use
  size_t cap = 0;  // elements allocated
  void alloc(size_t count) {
    if (count == 0) count = 1;
    if (p && count <= cap) {
      n = count;
      return;
    }
    // a buffer that must grow (a new geometry with a few more points) gets
    // 1/16 headroom, so that the next small growth reuses it; first
    // allocations are exact
    const size_t want = p ? count + count / 16 : count;
    free();
    const cudaError_t e = cudaMalloc(&p, want * sizeof(T));
    if (e != cudaSuccess) {  // clear the thread's last error: later launch checks must not see it
      cudaGetLastError();
      p = nullptr;
      throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e) + " allocating " +
                               std::to_string(count * sizeof(T)) + " bytes");
    }
    n = count;
    cap = want;
    g_devbuf_bytes += (long long)(cap * sizeof(T));
  }
  void upload(const std::vector<T>& v) {
    alloc(v.size());
    if (!v.empty()) LIO_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  }
  void free() {
    if (p) {
      cudaFree(p);
      g_devbuf_bytes -= (long long)(cap * sizeof(T));
    }
    p = nullptr;
    n = cap = 0;
  }
  ~DevBuf() { free(); }
};

// Host copies of the packed matrices (millions of doubles for a few thousand
// functions), threaded: dst = src, and dst += src.
void host_copy(double* dst, const double* src, size_t n) {
#pragma omp parallel for schedule(static) if (n >= (1u << 15))
  for (long long i = 0; i < (long long)n; i++) dst[i] = src[i];
}
void host_accumulate(double* dst, const double* src, size_t n) {
#pragma omp parallel for schedule(static) if (n >= (1u << 15))
  for (long long i = 0; i < (long long)n; i++) dst[i] += src[i];
}

// Pieces of the compact Kohn-Sham download: eight, each added into the
// caller's vectors on all host threads while the next is in flight (the same
// sizes on both sides: enqueue downloads them, finish adds them)
size_t compact_piece(size_t total) { return std::max<size_t>((total + 7) / 8, (size_t)1 << 15); }

// Compact transfers of a host-array solve: only the packed entries some group
// touches (sorted, unique `idx`, n per spin) cross PCIe. The density's are
// scattered into the full device matrices (the kernels read no other entry);
// the Kohn-Sham matrices' are gathered before the download (no other entry
// receives an XC contribution).
__global__ void k_scatter_packed(const double* __restrict__ src, const long long* __restrict__ idx, long long n,
                                 int nspin, double* __restrict__ a, double* __restrict__ b) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n * nspin;
       k += (long long)gridDim.x * blockDim.x)
    (k < n ? a : b)[idx[k < n ? k : k - n]] = src[k];
}
__global__ void k_gather_packed(const double* __restrict__ a, const double* __restrict__ b,
                                const long long* __restrict__ idx, long long n, int nspin, double* __restrict__ dst) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n * nspin;
       k += (long long)gridDim.x * blockDim.x)
    dst[k] = (k < n ? a : b)[idx[k < n ? k : k - n]];
}

__device__ __forceinline__ long long packed_index(int gi, int gj, int M) {
  const long long lo = gi < gj ? gi : gj, hi = gi < gj ? gj : gi;
  return lo * M - (lo * (lo - 1)) / 2 + (hi - lo);
}

// ------------------------------------------------------------------ basis values
// Cartesian component exponents: s; p x,y,z; d xx,xy,yy,xz,yz,zz
__constant__ int c_comp_l[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                                    {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}};

__device__ __forceinline__ double ipow(double x, int n) { return n == 0 ? 1.0 : (n == 1 ? x : x * x); }
__device__ __forceinline__ double dpow(double x, int n) {  // d/dx x^n
  return n == 0 ? 0.0 : (n == 1 ? 1.0 : 2.0 * x);
}
__device__ __forceinline__ double d2pow(int n) { return n == 2 ? 2.0 : 0.0; }

// One thread per (group, point). For every simple function of the group the
// contracted radial part t = sum_k c_k exp(-a_k r^2) (primitives with
// a_k r^2 > 70 skipped, g2g/cpu/functions.cpp:68-79), tg = sum a_k t_k and
// th = sum a_k^2 t_k give, for the monomial P = x^lx y^ly z^lz,
//   F = P t,  dF/da = P_a t - 2 r_a P tg,
//   d2F/da db = P_ab t - 2 (r_b P_a + r_a P_b + delta_ab P) tg + 4 r_a r_b P th,
// the closed forms of g2g/cpu/functions.cpp:81-352; d xx/yy/zz carry dnorm.
__global__ void k_basis(const int2* __restrict__ tiles, const GroupDev* __restrict__ groups,
                        const double* __restrict__ px, const double* __restrict__ py,
                        const double* __restrict__ pz, const int* __restrict__ sf_glob,
                        const int* __restrict__ sf_type, const int* __restrict__ nuc,
                        const int* __restrict__ ncont, const double* __restrict__ ca,
                        const double* __restrict__ cc, const double* __restrict__ ax,
                        const double* __restrict__ ay, const double* __restrict__ az, double dnorm,
                        int kinds, double* __restrict__ basis, int nkb, int bscale = 1) {
  const int2 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int p = t.y * kBasisBlock + threadIdx.x;
  if (p >= G.ldp) return;
  const bool valid = p < G.npts;
  const double x = px[G.pt_off + p], y = py[G.pt_off + p], z = pz[G.pt_off + p];
  // function-major cache (nkb = 0): value (kind, i, p) at bas_off * bscale + kind * m * ldp + i * ldp + p
  // (bscale: kinds of this cache over the kinds bas_off was laid out for); blocked copy of the
  // tensor-core density (nkb kinds): per (128-point tile, 32-function tile) the kinds one after
  // the other, each [i mod 32][p mod 128]. kinds: 1 (F), 4 (F, gradient) or 10 (and Hessian).
  double* out = basis + (nkb ? G.bb_off : G.bas_off * bscale);
  const long long kstride = nkb ? (long long)kTcChunkElems : (long long)G.m * G.ldp;
  auto at = [&](int i) {
    return nkb ? ((long long)((p >> 7) * G.nftc + (i >> 5)) * nkb * kTcChunkElems + (i & 31) * 128 + (p & 127))
               : (long long)i * G.ldp + p;
  };
  int ii = 0;
  for (int sf = 0; sf < G.nsimple; sf++) {
    const int gf = sf_glob[G.sf_off + sf];
    const int type = sf_type[G.sf_off + sf];
    const int atom = nuc[gf];
    const double r[3] = {x - ax[atom], y - ay[atom], z - az[atom]};
    const double dist = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    double tt = 0.0, tg = 0.0, th = 0.0;
    const int nc = ncont[gf];
    for (int k = 0; k < nc; k++) {
      const double a = ca[gf * 13 + k], c = cc[gf * 13 + k];
      const double expo = a * dist;
      if (expo > 70.0) continue;
      const double t0 = exp(-expo) * c;
      tt += t0;
      tg += t0 * a;
      th += t0 * (a * a);
    }
    const int c0 = type == 0 ? 0 : (type == 1 ? 1 : 4);
    const int nc_comp = type == 0 ? 1 : (type == 1 ? 3 : 6);
    for (int q = 0; q < nc_comp; q++, ii++) {
      const int* l = c_comp_l[c0 + q];
      const double scale = (type == 2 && (q == 0 || q == 2 || q == 5)) ? dnorm : 1.0;
      const double P = ipow(r[0], l[0]) * ipow(r[1], l[1]) * ipow(r[2], l[2]);
      const long long o = at(ii);
      out[o] = valid ? scale * P * tt : 0.0;
      if (kinds < 4) continue;
      double Pa[3];
      Pa[0] = dpow(r[0], l[0]) * ipow(r[1], l[1]) * ipow(r[2], l[2]);
      Pa[1] = ipow(r[0], l[0]) * dpow(r[1], l[1]) * ipow(r[2], l[2]);
      Pa[2] = ipow(r[0], l[0]) * ipow(r[1], l[1]) * dpow(r[2], l[2]);
      for (int a = 0; a < 3; a++)
        out[(1 + a) * kstride + o] = valid ? scale * (Pa[a] * tt - 2.0 * r[a] * P * tg) : 0.0;
      if (kinds < 10) continue;
      // Hessian: (xx, yy, zz) then (xy, xz, yz)
      const int ha[6] = {0, 1, 2, 0, 0, 1}, hb[6] = {0, 1, 2, 1, 2, 2};
      for (int h = 0; h < 6; h++) {
        const int a = ha[h], b = hb[h];
        double Pab;
        if (a == b) {
          Pab = (a == 0 ? d2pow(l[0]) * ipow(r[1], l[1]) * ipow(r[2], l[2])
                        : (a == 1 ? ipow(r[0], l[0]) * d2pow(l[1]) * ipow(r[2], l[2])
                                  : ipow(r[0], l[0]) * ipow(r[1], l[1]) * d2pow(l[2])));
        } else {
          int e[3] = {0, 0, 0};
          e[a] = 1;
          e[b] = 1;
          Pab = (e[0] ? dpow(r[0], l[0]) : ipow(r[0], l[0])) * (e[1] ? dpow(r[1], l[1]) : ipow(r[1], l[1])) *
                (e[2] ? dpow(r[2], l[2]) : ipow(r[2], l[2]));
        }
        double v = Pab * tt - 2.0 * (r[b] * Pa[a] + r[a] * Pa[b] + (a == b ? P : 0.0)) * tg +
                   4.0 * r[a] * r[b] * P * th;
        out[(4 + h) * kstride + o] = valid ? scale * v : 0.0;
      }
    }
  }
}

// ------------------------------------------------------- density (FP64 GEMMs)
// Tile = (group, point tile, function tile); 256 threads, each 4 points x 4
// functions of the 64 x 64 output, NA = 1 (LDA: G) or 4 (GGA: G, Gx, Gy, Gz).
template <int NA>
__global__ void __launch_bounds__(256) k_density_fp64(const int4* __restrict__ tiles,
                                                      const GroupDev* __restrict__ groups,
                                                      const int* __restrict__ fn_glob,
                                                      const double* __restrict__ basis,
                                                      const double* __restrict__ P, int M,
                                                      double* __restrict__ partial, long long part_base) {
  constexpr int NQ = NA == 1 ? 1 : kNQ;
  __shared__ double As[NA][kKStep][kTile];
  __shared__ double Bs[kKStep][kTile + 1];
  const int4 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int pt0 = t.y * kTile, ft = t.z, ft0 = ft * kTile;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const long long kstride = (long long)G.m * G.ldp;
  const double* bas = basis + G.bas_off;
  const int* fg = fn_glob + G.fn_off;
  double acc[NA][4][4];
#pragma unroll
  for (int a = 0; a < NA; a++)
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[a][r][c] = 0.0;

  for (int j0 = 0; j0 < G.m; j0 += kKStep) {
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
      for (int rr = 0; rr < 4; rr++) {
        const int idx = tid + 256 * rr, kk = idx >> 6, pp = idx & 63;
        const int j = j0 + kk;
        As[a][kk][pp] = j < G.m ? bas[a * kstride + (long long)j * G.ldp + pt0 + pp] : 0.0;
      }
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
      const int idx = tid + 256 * rr, kk = idx >> 6, ii = idx & 63;
      const int j = j0 + kk, i = ft0 + ii;
      double v = 0.0;
      if (j < G.m && i < G.m) {
        const int gj = fg[j], gi = fg[i];
        v = P[G.pk_off + packed_index(gi, gj, G.pk_M)];
        if (gi != gj) v *= 0.5;
      }
      Bs[kk][ii] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kKStep; kk++) {
      double b[4];
#pragma unroll
      for (int c = 0; c < 4; c++) b[c] = Bs[kk][tx + 16 * c];
#pragma unroll
      for (int a = 0; a < NA; a++)
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const double av = As[a][kk][ty + 16 * r];
#pragma unroll
          for (int c = 0; c < 4; c++) acc[a][r][c] = fma(av, b[c], acc[a][r][c]);
        }
    }
    __syncthreads();
  }

  // row-dot epilogue
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int p = pt0 + ty + 16 * r;
    double q[NQ];
#pragma unroll
    for (int k = 0; k < NQ; k++) q[k] = 0.0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int i = ft0 + tx + 16 * c;
      if (i >= G.m) continue;
      const long long o = (long long)i * G.ldp + p;
      const double F = bas[o];
      q[0] += F * acc[0][r][c];
      if (NA == 4) {
        const double gx = bas[kstride + o], gy = bas[2 * kstride + o], gz = bas[3 * kstride + o];
        const double hxx = bas[4 * kstride + o], hyy = bas[5 * kstride + o], hzz = bas[6 * kstride + o];
        const double hxy = bas[7 * kstride + o], hxz = bas[8 * kstride + o], hyz = bas[9 * kstride + o];
        const double g0 = acc[0][r][c], gX = acc[NA > 1 ? 1 : 0][r][c], gY = acc[NA > 2 ? 2 : 0][r][c],
                     gZ = acc[NA > 3 ? 3 : 0][r][c];
        q[1] += 2.0 * gx * g0;
        q[2] += 2.0 * gy * g0;
        q[3] += 2.0 * gz * g0;
        q[4] += 2.0 * (gx * gX + hxx * g0);
        q[5] += 2.0 * (gy * gY + hyy * g0);
        q[6] += 2.0 * (gz * gZ + hzz * g0);
        q[7] += 2.0 * (gx * gY + hxy * g0);
        q[8] += 2.0 * (gx * gZ + hxz * g0);
        q[9] += 2.0 * (gy * gZ + hyz * g0);
      }
    }
#pragma unroll
    for (int k = 0; k < NQ; k++) {
      double v = q[k];
      v += __shfl_xor_sync(0xffffffffu, v, 8);
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      v += __shfl_xor_sync(0xffffffffu, v, 2);
      v += __shfl_xor_sync(0xffffffffu, v, 1);
      q[k] = v;
    }
    if (tx == 0) {
      double* dst = partial + (G.part_off - part_base);
#pragma unroll
      for (int k = 0; k < NQ; k++) dst[((long long)ft * NQ + k) * G.ldp + p] = q[k];
    }
  }
}

// --------------------------------------------------------- Becke weights
// One thread per grid point of the partition being built: its atom's
// fuzzy-cell weight over the group's nuclei with the atomic-size adjustment
// (g2g/cpu/weight.cpp:13-112), in the operation order of the host code
// (partition.cpp) and with every FP64 operation explicitly rounded (no fused
// multiply-add), so the factors equal the host's, and the reference's, bit
// for bit. Two values the host code recomputes in its inner loop are computed
// once instead, by the same operations: the size adjustment a_jk =
// x / (x^2 - 1), x = (rm_j / rm_k - 1) / (rm_j / rm_k + 1), per atom pair
// (becke_pair_table, three divisions out of every step), and the point's
// distance to each nucleus of its group (a per-thread cache, one square root
// per nucleus instead of one per pair). The host multiplies each point's
// weight by its factor.
__device__ __forceinline__ double len3_rn(double x, double y, double z) {
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

// s(u) with the pair's size adjustment a_jk (g2g/cpu/weight.cpp:40-48)
__device__ __forceinline__ double becke_step_rn(double u, double a_jk) {
  u = __dadd_rn(u, __dmul_rn(a_jk, __dsub_rn(1.0, __dmul_rn(u, u))));
#pragma unroll
  for (int it = 0; it < 3; it++) u = __dsub_rn(__dmul_rn(1.5, u), __dmul_rn(0.5, __dmul_rn(__dmul_rn(u, u), u)));
  return __dmul_rn(0.5, __dsub_rn(1.0, u));
}

constexpr int kBeckeCache = 64;  // nuclei whose distances a thread keeps (more: recomputed per pair)

__global__ void k_becke_weights(const double* __restrict__ px, const double* __restrict__ py,
                                const double* __restrict__ pz, const int* __restrict__ patom,
                                const int* __restrict__ pgroup, long long i0, long long n,
                                const int* __restrict__ nuc_off,
                                const int* __restrict__ nucs, const double* __restrict__ ax,
                                const double* __restrict__ ay, const double* __restrict__ az,
                                const double* __restrict__ pair_a, const double* __restrict__ adist, int natoms,
                                double* __restrict__ factor) {
  const long long i = i0 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = px[i], y = py[i], z = pz[i];
  const int atom = patom[i], g = pgroup[i];
  const int* nl = nucs + nuc_off[g];
  const int nn = nuc_off[g + 1] - nuc_off[g];
  const bool cached = nn <= kBeckeCache;
  double dc[kBeckeCache];
  auto dist_to = [&](int a) { return len3_rn(__dsub_rn(x, ax[a]), __dsub_rn(y, ay[a]), __dsub_rn(z, az[a])); };
  if (cached)
    for (int k = 0; k < nn; ++k) dc[k] = dist_to(nl[k]);
  auto dist_k = [&](int k) { return cached ? dc[k] : dist_to(nl[k]); };
  double P_total = 0.0, P_atom = 0.0;
  bool own_found = false;
  for (int j = 0; j < nn; ++j) {
    double P_curr = 1.0;
    const int aj = nl[j];
    const double dj = dist_k(j);
    const double* aj_dist = adist + (long long)aj * natoms;
    const double* aj_pair = pair_a + (long long)aj * natoms;
    for (int k = 0; k < nn; ++k) {
      const int ak = nl[k];
      if (ak == aj) continue;
      const double u = __ddiv_rn(__dsub_rn(dj, dist_k(k)), aj_dist[ak]);
      P_curr = __dmul_rn(P_curr, becke_step_rn(u, aj_pair[ak]));
      if (P_curr == 0.0) break;
    }
    if (aj == atom) {
      own_found = true;
      P_atom = P_curr;
      if (P_atom == 0.0) break;
    }
    P_total = __dadd_rn(P_total, P_curr);
  }
  if (!own_found) {  // the point's own atom is not among the group's nuclei
    P_atom = 1.0;
    const double da = dist_to(atom);
    const double* at_dist = adist + (long long)atom * natoms;
    const double* at_pair = pair_a + (long long)atom * natoms;
    for (int k = 0; k < nn; ++k) {
      const int ak = nl[k];
      const double u = __ddiv_rn(__dsub_rn(da, dist_k(k)), at_dist[ak]);
      P_atom = __dmul_rn(P_atom, becke_step_rn(u, at_pair[ak]));
      if (P_atom == 0.0) break;
    }
  }
  factor[i] = P_total == 0.0 ? 0.0 : __ddiv_rn(P_atom, P_total);
}

// ------------------------------------------------------- XC nuclear gradients
// g2g_solve_groups_ types 2 and 3 (g2g/cpu/iteration.cpp:213-267 closed,
// 496-563 open). Per point p and function i of a group, with the packed
// density's off-diagonals halved (the symmetric P),
//   w_i(p) = 2 sum_j P_ij F_j(p),
// and the atom of function i gets -f_p w_i(p) grad F_i(p) summed over the
// points, per spin with its own factor f_p = w_p v_xc(p) (the factors of the
// solve just run). Tile = (group, 64-point tile, 64-function tile) as the FP64
// density: G = F P in registers (one accumulator block per spin), then the
// factor-weighted gradient dots, summed over the tile's points, go to the
// atoms with FP64 atomics (summation order, not values, varies run to run).
struct BasisView {
  const double* base;  // function-major cache (nkb = 0) or the blocked copy (nkb kinds)
  int nkb;
  int bscale;          // function-major: kinds of this cache over the kinds bas_off counts
  __device__ __forceinline__ double at(const GroupDev& G, int kind, int i, int p) const {
    if (nkb == 0) return base[G.bas_off * bscale + ((long long)kind * G.m + i) * G.ldp + p];
    return base[G.bb_off + ((long long)((p >> 7) * G.nftc + (i >> 5)) * nkb + kind) * kTcChunkElems +
                (i & 31) * 128 + (p & 127)];
  }
};

template <int NS>
__global__ void __launch_bounds__(256) k_force_fp64(const int4* __restrict__ tiles, const GroupDev* __restrict__ groups,
                                                    const int* __restrict__ fn_glob, const int* __restrict__ fn_atom,
                                                    BasisView bv, const double* __restrict__ P_a,
                                                    const double* __restrict__ P_b, int M,
                                                    const double* __restrict__ fac_a,
                                                    const double* __restrict__ fac_b, double* __restrict__ force) {
  __shared__ double As[kKStep][kTile];
  __shared__ double Bs[NS][kKStep][kTile + 1];
  __shared__ double red[8][kTile][3];
  const int4 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int pt0 = t.y * kTile, ft0 = t.z * kTile;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int* fg = fn_glob + G.fn_off;
  double acc[NS][4][4];
#pragma unroll
  for (int sp = 0; sp < NS; sp++)
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[sp][r][c] = 0.0;

  for (int j0 = 0; j0 < G.m; j0 += kKStep) {
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
      const int idx = tid + 256 * rr, kk = idx >> 6, pp = idx & 63;
      const int j = j0 + kk;
      As[kk][pp] = j < G.m ? bv.at(G, 0, j, pt0 + pp) : 0.0;
    }
#pragma unroll
    for (int sp = 0; sp < NS; sp++)
#pragma unroll
      for (int rr = 0; rr < 4; rr++) {
        const int idx = tid + 256 * rr, kk = idx >> 6, ii = idx & 63;
        const int j = j0 + kk, i = ft0 + ii;
        double v = 0.0;
        if (j < G.m && i < G.m) {
          const int gj = fg[j], gi = fg[i];
          v = (sp == 0 ? P_a : P_b)[G.pk_off + packed_index(gi, gj, G.pk_M)];
          if (gi != gj) v *= 0.5;
        }
        Bs[sp][kk][ii] = v;
      }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kKStep; kk++) {
#pragma unroll
      for (int sp = 0; sp < NS; sp++) {
        double b[4];
#pragma unroll
        for (int c = 0; c < 4; c++) b[c] = Bs[sp][kk][tx + 16 * c];
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const double av = As[kk][ty + 16 * r];
#pragma unroll
          for (int c = 0; c < 4; c++) acc[sp][r][c] = fma(av, b[c], acc[sp][r][c]);
        }
      }
    }
    __syncthreads();
  }

  // sum_p f_p G_i(p) dF_i/da(p) over this thread's 4 points, per function c and axis a
  double sx[4][3];
#pragma unroll
  for (int c = 0; c < 4; c++)
#pragma unroll
    for (int a = 0; a < 3; a++) sx[c][a] = 0.0;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int p = pt0 + ty + 16 * r;
    const double fa = fac_a[G.pt_off + p], fb = NS == 2 ? fac_b[G.pt_off + p] : 0.0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int i = ft0 + tx + 16 * c;
      if (i >= G.m) continue;
      const double h = NS == 2 ? fa * acc[0][r][c] + fb * acc[NS - 1][r][c] : fa * acc[0][r][c];
#pragma unroll
      for (int a = 0; a < 3; a++) sx[c][a] = fma(h, bv.at(G, 1 + a, i, p), sx[c][a]);
    }
  }
  // over the 16 threads of a function column: the two of a warp by shuffle, the 8 warps in shared memory
  const int warp = tid >> 5;
#pragma unroll
  for (int c = 0; c < 4; c++)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double v = sx[c][a] + __shfl_xor_sync(0xffffffffu, sx[c][a], 16);
      if ((tid & 31) < 16) red[warp][tx + 16 * c][a] = v;
    }
  __syncthreads();
  for (int k = tid; k < kTile * 3; k += 256) {
    const int fn = k / 3, a = k - 3 * fn, i = ft0 + fn;
    if (i >= G.m) continue;
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < 8; w++) v += red[w][fn][a];
    atomicAdd(&force[fn_atom[G.fn_off + i] * 3 + a], -2.0 * v);
  }
}

// ------------------------------------------------------------- point functional
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  v = threadIdx.x < nw ? sh[threadIdx.x] : 0.0;
  if (w == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One thread per point: reduce the function-tile partials, evaluate the
// functional, write factor = w * v_xc, and a per-block energy sum of
// rho * w * (ex + ec) (g2g/cpu/iteration.cpp:106-114, 199-208, 482-492).
// MODE: 0 closed LDA, 1 closed GGA (PBE), 2 open GGA (PBE), 3 open LDA (the
// reference CPU path has no branch for it, g2g/cpu/iteration.cpp:362-363:
// energy and potential stay zero). Compile-time so the per-point sums live in
// registers.
template <int MODE>
__global__ void __launch_bounds__(kFuncBlock, 8) k_functional(const int2* __restrict__ tiles,
                                                           const GroupDev* __restrict__ groups,
                                                           const double* __restrict__ pw,
                                                           const double* __restrict__ part_a,
                                                           const double* __restrict__ part_b, int part_tile,
                                                           int iexch, double* __restrict__ fac_a,
                                                           double* __restrict__ fac_b,
                                                           double* __restrict__ energy_blocks, long long part_base,
                                                           long long pt_base) {
  constexpr bool kLda = MODE == 0 || MODE == 3, kOpen = MODE >= 2;
  constexpr int NQ = kLda ? 1 : kNQ;
  __shared__ double sh[32];
  const int2 t = tiles[blockIdx.x];
  const GroupDev& G = groups[t.x];
  const int p = t.y * kFuncBlock + threadIdx.x;
  const int ldp = G.ldp;
  double e = 0.0;
  if (p < ldp) {
    const double w = pw[G.pt_off + p];
    double qa[kNQ], qb[kNQ];
#pragma unroll
    for (int k = 0; k < kNQ; k++) qa[k] = qb[k] = 0.0;
    const int nparts = (G.m + part_tile - 1) / part_tile;  // partial tiles written by the density stage
    for (int f = 0; f < nparts; f++)
#pragma unroll
      for (int k = 0; k < NQ; k++) {
        const long long o = G.part_off - part_base + ((long long)f * NQ + k) * ldp + p;
        qa[k] += part_a[o];
        if (kOpen) qb[k] += part_b[o];
      }
    double va = 0.0, vb = 0.0;
    if (p < G.npts) {
      if (MODE == 2) {
        const xc::GgaOpenOut o = xc::pbe_open(qa[0], qb[0], qa + 1, qb + 1, qa + 4, qb + 4, qa + 7, qb + 7);
        e = ((qa[0] + qb[0]) * w) * (o.ex + o.ec);
        va = w * o.va;
        vb = w * o.vb;
      } else if (MODE == 0) {
        const xc::LdaOut o = xc::lda_closed(qa[0], iexch);
        e = (qa[0] * w) * (o.ex + o.ec);
        va = w * o.v;
      } else if (MODE == 1) {
        const xc::GgaOut o = iexch == 9 ? xc::pbe_closed(qa[0], qa + 1, qa + 4, qa + 7)
                                        : xc::gga_closed_other(qa[0], qa + 1, qa + 4, qa + 7, iexch);
        e = (qa[0] * w) * (o.ex + o.ec);
        va = w * o.v;
      }
    }
    fac_a[G.pt_off - pt_base + p] = va;
    if (kOpen) fac_b[G.pt_off - pt_base + p] = vb;
  }
  const double s = block_sum(e, sh);
  if (threadIdx.x == 0) energy_blocks[blockIdx.x] = s;
}

// part_base / pt_base: offsets (elements) subtracted from every group's
// part_off / pt_off when indexing the partials and the factors, for callers
// whose arrays hold only a batch of groups (the weights pw are always indexed
// by the group's own pt_off)
void launch_functional(bool lda, bool open, unsigned nblocks, cudaStream_t st, const int2* tiles,
                       const GroupDev* groups, const double* pw, const double* part_a, const double* part_b,
                       int part_tile, int iexch, double* fac_a, double* fac_b, double* eblocks,
                       long long part_base = 0, long long pt_base = 0) {
#define LIO_FUNCTIONAL(MODE)                                                                                \
  k_functional<MODE><<<nblocks, kFuncBlock, 0, st>>>(tiles, groups, pw, part_a, part_b, part_tile, iexch, fac_a, \
                                                     fac_b, eblocks, part_base, pt_base)
  if (!open && lda)
    LIO_FUNCTIONAL(0);
  else if (!open)
    LIO_FUNCTIONAL(1);
  else if (!lda)
    LIO_FUNCTIONAL(2);
  else
    LIO_FUNCTIONAL(3);
#undef LIO_FUNCTIONAL
}

// E_xc of the build from the per-block partials: written, or (accumulate) added
// to an external accumulator that other shards of the build also add to
__global__ void k_sum_blocks(const double* __restrict__ in, int n, double* __restrict__ out, int accumulate) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += in[i];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) {
    if (accumulate)
      atomicAdd(out, v);
    else
      *out = v;
  }
}

// E_xc of every molecule of a batch: block k sums the per-block partials of
// its molecule, [seg[k].x, seg[k].y)
__global__ void k_sum_segments(const double* __restrict__ in, const int2* __restrict__ seg,
                               double* __restrict__ out) {
  __shared__ double sh[32];
  const int2 r = seg[blockIdx.x];
  double v = 0.0;
  for (int i = r.x + threadIdx.x; i < r.y; i += blockDim.x) v += in[i];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = v;
}

// ------------------------------------------------ Kohn-Sham update (FP64 GEMM)
// Tile = (group, i tile, j tile) with i tile <= j tile; K_ij = sum_p F_ip f_p F_jp
// for i <= j, scattered with FP64 atomics into the packed accumulator(s).
template <int NS>
__global__ void __launch_bounds__(256) k_fock_fp64(const int4* __restrict__ tiles,
                                                   const GroupDev* __restrict__ groups,
                                                   const int* __restrict__ fn_glob,
                                                   const double* __restrict__ basis,
                                                   const double* __restrict__ fac_a,
                                                   const double* __restrict__ fac_b, int M,
                                                   double* __restrict__ K_a, double* __restrict__ K_b,
                                                   long long pt_base) {
  __shared__ double As[kKStep][kTile + 1];
  __shared__ double Bs[NS][kKStep][kTile + 1];
  const int4 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int i0 = t.y * kTile, j0 = t.z * kTile;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const double* F = basis + G.bas_off;
  double acc[NS][4][4];
#pragma unroll
  for (int s = 0; s < NS; s++)
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[s][r][c] = 0.0;
  for (int p0 = 0; p0 < G.ldp; p0 += kKStep) {
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
      const int idx = tid + 256 * rr, row = idx >> 4, kk = idx & 15;
      const int i = i0 + row, j = j0 + row, p = p0 + kk;
      As[kk][row] = i < G.m ? F[(long long)i * G.ldp + p] : 0.0;
      const double fj = j < G.m ? F[(long long)j * G.ldp + p] : 0.0;
      Bs[0][kk][row] = fj * fac_a[G.pt_off - pt_base + p];
      if (NS == 2) Bs[NS - 1][kk][row] = fj * fac_b[G.pt_off - pt_base + p];
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kKStep; kk++) {
      double av[4];
#pragma unroll
      for (int r = 0; r < 4; r++) av[r] = As[kk][ty + 16 * r];
#pragma unroll
      for (int s = 0; s < NS; s++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const double bv = Bs[s][kk][tx + 16 * c];
#pragma unroll
          for (int r = 0; r < 4; r++) acc[s][r][c] = fma(av[r], bv, acc[s][r][c]);
        }
    }
    __syncthreads();
  }
  const int* fg = fn_glob + G.fn_off;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int i = i0 + ty + 16 * r;
    if (i >= G.m) continue;
    const int gi = fg[i];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int j = j0 + tx + 16 * c;
      if (j >= G.m || (t.y == t.z && i > j)) continue;
      const long long o = G.pk_off + packed_index(gi, fg[j], G.pk_M);
      atomicAdd(K_a + o, acc[0][r][c]);
      if (NS == 2) atomicAdd(K_b + o, acc[NS - 1][r][c]);
    }
  }
}

#include "density_tc.cuh"
#include "fock_tc.cuh"
#include "force_tc.cuh"

}  // namespace

// ============================================================================ Impl
struct DeviceEngine::Impl {
  int M = 0, natoms = 0;
  bool lda = false, open = false;
  int iexch = 9;
  int nk = 1;   // kinds of the FP64 form's function-major basis cache: 1 (LDA) or 10 (GGA)
  int nkb = 1;  // kinds of the tensor-core form's blocked basis: F (LDA), or F and its gradient (GGA)
  long long npoints = 0, ngroups = 0, total_ldp = 0;
  std::vector<GroupDev> hgroups;
  DevBuf<GroupDev> groups;
  DevBuf<double> px, py, pz, pw;
  DevBuf<int> fn_glob, sf_glob, sf_type, nuc, ncont, fn_sh, fn_atom;
  DevBuf<int> sf_fn;  // per simple function (shell) of a group: the local index of its first component
  DevBuf<ShellInfo> sinfo;  // per (group, shell): atom position, type, first column (density epilogue)
  DevBuf<double> rad;  // radial sums per (tile, shell, point) of the tensor-core density
  long long rad_elems = 0;
  DevBuf<int8_t> fn_cp;
  // tensor-core form (built on first use per geometry)
  DevBuf<int2> slice_basis_tiles, slice_dens_tiles;
  DevBuf<int2> dens_tc_tiles;  // (group, 128-point tile), largest function count first
  int tc_fcap = 0, nsm = 148;

  DevBuf<double> bblk;  // blocked FP64 basis (tensor-core operands, forces)
  bool lean = false;    // the blocked basis is dropped once the operands are built
  int max_nftc = 0;
  DevBuf<int8_t> aslices, dslices_a, dslices_b;
  DevBuf<int16_t> aexp, dexp_a, dexp_b;
  DevBuf<int> tc_err;
  long long tc_sizes[5] = {0, 0, 0, 0, 0};
  // tensor-core Kohn-Sham contraction
  DevBuf<int2> fa_rows, fb_rows, fa_tiles32;  // rows of the Kohn-Sham operands, 32-row pieces of the A slices
  DevBuf<int4> fk_tiles, force_tc_tiles;
  DevBuf<int8_t> fa_slices;
  DevBuf<int16_t> fa_exp, fb_exp_a, fb_exp_b;
  long long fk_sizes[4] = {0, 0, 0, 0};
  bool tc_ready = false;
  double d_norm = 1.0;
  DevBuf<double> ca, cc, ax, ay, az;
  DevBuf<double> basis;
  DevBuf<int2> basis_tiles, func_tiles;
  DevBuf<int4> dens_tiles, fock_tiles;
  DevBuf<double> P_a, P_b, K_a, K_b, part_a, part_b, fac_a, fac_b, eblocks, energy;
  size_t npacked = 0;  // elements of the packed matrices per spin (a batch: its molecules' together)
  // a batch: per molecule the range of its energy partials, its E_xc (device, pinned copy)
  int nmembers = 0;
  DevBuf<int2> member_blocks;
  DevBuf<double> member_energy;
  std::vector<double> h_member_energy;
  double* hME = nullptr;
  size_t hme_elems = 0;
  // packed entries the groups touch (sorted); when they are at most half of the
  // packed matrix, host-array solves move only these (Pc, Kc: nspin x npairs)
  std::vector<long long> hpidx;
  DevBuf<long long> pidx;
  DevBuf<double> Pc, Kc;
  bool compact = false;
  long long last_h2d = 0, last_d2h = 0;  // bytes of the last host-array solve
  double* hK = nullptr;  // pinned: Kohn-Sham result of the last solve (nspin x npacked)
  double* hP = nullptr;  // pinned: staging of the caller's densities (nspin x npacked)
  size_t pinned_elems = 0;
  double* hE = nullptr;  // pinned: its energy
  int* hErr = nullptr;   // pinned: the tensor-core error flag
  bool enqueued = false;
  bool use_graphs = true;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_key = -1, graph_launches = 0;
  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    graph_key = -1;
  }
  double tuned_fp64_ms = 0.0, tuned_tc_ms = 0.0;
  long long basis_elems = 0, bblk_elems = 0;
  double basis_norm = 1.0;
  bool basis_valid = false;
  // the function-major cache of the FP64 form, or (blocked) the tensor-core
  // form's blocked copy; the padded functions of a blocked tile stay zero
  void compute_basis(bool blocked = false) {
    DevBuf<double>& dst = blocked ? bblk : basis;
    if (blocked) {
      bblk.alloc(bblk_elems);
      LIO_CUDA(cudaMemsetAsync(bblk.p, 0, bblk_elems * sizeof(double), stream));
    } else {
      basis.alloc(basis_elems);
    }
    if (basis_tiles.n > 0 && ngroups > 0) {
      k_basis<<<(unsigned)basis_tiles.n, kBasisBlock, 0, stream>>>(basis_tiles.p, groups.p, px.p, py.p, pz.p,
                                                                    sf_glob.p, sf_type.p, nuc.p, ncont.p, ca.p, cc.p,
                                                                    ax.p, ay.p, az.p, basis_norm, blocked ? nkb : nk,
                                                                    dst.p, blocked ? nkb : 0);
      LIO_CUDA(cudaGetLastError());
    }
    LIO_CUDA(cudaStreamSynchronize(stream));
    if (!blocked) basis_valid = true;
  }
  void free_pinned() {
    if (hK) cudaFreeHost(hK);
    if (hP) cudaFreeHost(hP);
    hP = nullptr;
    pinned_elems = 0;
    if (hE) cudaFreeHost(hE);
    if (hErr) cudaFreeHost(hErr);
    if (hME) cudaFreeHost(hME);
    hME = nullptr;
    hme_elems = 0;
    hK = hE = nullptr;
    hErr = nullptr;
  }
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t fev0 = nullptr, fev1 = nullptr;  // around the force kernel
  // chunked result download: the host adds each chunk of the Kohn-Sham matrices
  // into the caller's vectors while the next one is in flight
  static constexpr int kMaxChunks = 32;
  cudaEvent_t kev[kMaxChunks] = {};
  int nchunks = 0;
  double *ext_ka = nullptr, *ext_kb = nullptr, *ext_e = nullptr;  // external accumulators (resident solves)
  double last_force_ms = 0.0;
  int launches = 0;
  bool profiling = false;
  static constexpr int kNumStages = 5;
  cudaEvent_t sev[kNumStages + 1] = {};
  double stage_ms[kNumStages] = {};
  int profiled = 0;
  bool pending = false;
  void collect() {
    if (!pending) return;
    LIO_CUDA(cudaEventSynchronize(sev[kNumStages]));
    for (int i = 0; i < kNumStages; i++) {
      float ms = 0.f;
      LIO_CUDA(cudaEventElapsedTime(&ms, sev[i], sev[i + 1]));
      stage_ms[i] += ms;
    }
    profiled++;
    pending = false;
  }
  void mark(int i) {
    if (profiling) LIO_CUDA(cudaEventRecord(sev[i], stream));
  }

  Impl() {
    LIO_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    stream = own_stream;
    LIO_CUDA(cudaEventCreate(&ev0));
    LIO_CUDA(cudaEventCreate(&ev1));
    LIO_CUDA(cudaEventCreate(&fev0));
    LIO_CUDA(cudaEventCreate(&fev1));
    for (auto& e : kev) LIO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : sev) LIO_CUDA(cudaEventCreate(&e));
  }
  ~Impl() {
    drop_graph();
    free_pinned();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (fev0) cudaEventDestroy(fev0);
    if (fev1) cudaEventDestroy(fev1);
    for (auto& e : kev)
      if (e) cudaEventDestroy(e);
    for (auto& e : sev)
      if (e) cudaEventDestroy(e);
    if (own_stream) cudaStreamDestroy(own_stream);
  }
};

DeviceEngine::DeviceEngine() : impl_(new Impl) {}

bool DeviceEngine::available() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return n > 0;
}
DeviceEngine::~DeviceEngine() = default;

void DeviceEngine::release() {
  Impl* d = impl_.get();
  d->basis.free();
  d->basis_valid = false;
  d->part_a.free();
  d->part_b.free();
  d->ngroups = d->npoints = 0;
}

long long DeviceEngine::points() const { return impl_->npoints; }

namespace {
size_t align256(size_t b) { return (b + 255) / 256 * 256; }
}  // namespace

void DeviceEngine::becke_weights(const System& sys, const std::vector<PointGroup*>& groups, bool drop_zero) {
  const long long ng = (long long)groups.size();
  std::vector<long long> first(ng + 1, 0);  // first point of each group in the flat arrays
  for (long long gi = 0; gi < ng; gi++) first[gi + 1] = first[gi] + (long long)groups[gi]->points.size();
  const long long n = first[ng];
  if (n == 0) return;
  std::vector<int> hoff(groups.size() + 1, 0), hnucs;
  for (size_t gi = 0; gi < groups.size(); gi++) {
    hnucs.insert(hnucs.end(), groups[gi]->nucs.begin(), groups[gi]->nucs.end());
    hoff[gi + 1] = (int)hnucs.size();
  }
  const size_t na = (size_t)sys.natoms;
  // one layout for the pinned staging and the device block: per point x, y, z,
  // factor (FP64), atom, group (int); then the group offsets, their nuclei and
  // the atom tables
  const size_t o_x = 0, o_y = o_x + align256(n * 8), o_z = o_y + align256(n * 8), o_f = o_z + align256(n * 8);
  const size_t o_atom = o_f + align256(n * 8), o_group = o_atom + align256(n * 4);
  const size_t o_off = o_group + align256(n * 4), o_nucs = o_off + align256(hoff.size() * 4);
  const size_t o_ax = o_nucs + align256(std::max<size_t>(hnucs.size(), 1) * 4);
  const size_t o_ay = o_ax + align256(na * 8), o_az = o_ay + align256(na * 8), o_pair = o_az + align256(na * 8);
  const size_t o_dist = o_pair + align256(na * na * 8), total = o_dist + align256(na * na * 8);
  PinnedStaging& ws = weights_staging();
  std::lock_guard<std::mutex> lock(ws.m);  // one grid build at a time uses the staging
  ws.reserve(total);
  char* h = static_cast<char*>(ws.host);
  double* hx = reinterpret_cast<double*>(h + o_x);
  double* hy = reinterpret_cast<double*>(h + o_y);
  double* hz = reinterpret_cast<double*>(h + o_z);
  double* hf = reinterpret_cast<double*>(h + o_f);
  int* hatom = reinterpret_cast<int*>(h + o_atom);
  int* hgroup = reinterpret_cast<int*>(h + o_group);
  std::memcpy(h + o_off, hoff.data(), hoff.size() * 4);
  if (!hnucs.empty()) std::memcpy(h + o_nucs, hnucs.data(), hnucs.size() * 4);
  std::memcpy(h + o_ax, sys.ax.data(), na * 8);
  std::memcpy(h + o_ay, sys.ay.data(), na * 8);
  std::memcpy(h + o_az, sys.az.data(), na * 8);
  becke_pair_table(sys, reinterpret_cast<double*>(h + o_pair));
  std::memcpy(h + o_dist, sys.atom_dist.data(), na * na * 8);
  // the device block is kept per device too (grow-only, never freed): no
  // cudaMalloc / cudaFree of ~50 bytes per point on every geometry
  static DevBuf<char>* blocks[64] = {};
  int dev = 0;
  LIO_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw std::runtime_error("device ordinal out of range for the weights block");
  if (!blocks[dev]) blocks[dev] = new DevBuf<char>;
  blocks[dev]->alloc(total);
  char* d = blocks[dev]->p;
  // A pipeline over chunks of whole groups (about 1/8 of the points each): the
  // host packs chunk c while the device copies in, weighs and copies out the
  // chunks before it, and multiplies chunk c's weights while the device works
  // on the ones after it.
  const cudaStream_t cs = copy_stream();
  StreamDrain drain{cs};
  LIO_CUDA(cudaMemcpyAsync(d + o_off, h + o_off, total - o_off, cudaMemcpyHostToDevice, cs));
  constexpr int kChunks = 8;
  std::vector<long long> cut{0};  // group boundaries of the chunks
  for (long long gi = 0; gi < ng; gi++)
    if (first[gi + 1] - first[cut.back()] >= (n + kChunks - 1) / kChunks || gi + 1 == ng) cut.push_back(gi + 1);
  const int nc = (int)cut.size() - 1;
  struct Events {
    std::vector<cudaEvent_t> e;
    ~Events() {
      for (cudaEvent_t x : e) cudaEventDestroy(x);
    }
  } ev;
  for (int c = 0; c < nc; c++) {
#pragma omp parallel for schedule(dynamic, 4)
    for (long long gi = cut[c]; gi < cut[c + 1]; gi++) {
      long long k = first[gi];
      for (const GridPoint& p : groups[gi]->points) {
        hx[k] = p.x;
        hy[k] = p.y;
        hz[k] = p.z;
        hatom[k] = p.atom;
        hgroup[k] = (int)gi;
        k++;
      }
    }
    const long long p0 = first[cut[c]], p1 = first[cut[c + 1]], np = p1 - p0;
    cudaEvent_t e;
    LIO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ev.e.push_back(e);
    if (np == 0) {
      LIO_CUDA(cudaEventRecord(e, cs));
      continue;
    }
    for (size_t o : {o_x, o_y, o_z})
      LIO_CUDA(cudaMemcpyAsync(d + o + p0 * 8, h + o + p0 * 8, (size_t)np * 8, cudaMemcpyHostToDevice, cs));
    for (size_t o : {o_atom, o_group})
      LIO_CUDA(cudaMemcpyAsync(d + o + p0 * 4, h + o + p0 * 4, (size_t)np * 4, cudaMemcpyHostToDevice, cs));
    k_becke_weights<<<(unsigned)((np + 127) / 128), 128, 0, cs>>>(
        reinterpret_cast<const double*>(d + o_x), reinterpret_cast<const double*>(d + o_y),
        reinterpret_cast<const double*>(d + o_z), reinterpret_cast<const int*>(d + o_atom),
        reinterpret_cast<const int*>(d + o_group), p0, p1, reinterpret_cast<const int*>(d + o_off),
        reinterpret_cast<const int*>(d + o_nucs), reinterpret_cast<const double*>(d + o_ax),
        reinterpret_cast<const double*>(d + o_ay), reinterpret_cast<const double*>(d + o_az),
        reinterpret_cast<const double*>(d + o_pair), reinterpret_cast<const double*>(d + o_dist), sys.natoms,
        reinterpret_cast<double*>(d + o_f));
    LIO_CUDA(cudaGetLastError());
    LIO_CUDA(cudaMemcpyAsync(hf + p0, d + o_f + p0 * 8, (size_t)np * 8, cudaMemcpyDeviceToHost, cs));
    LIO_CUDA(cudaEventRecord(e, cs));
  }
  for (int c = 0; c < nc; c++) {
    LIO_CUDA(cudaEventSynchronize(ev.e[c]));
#pragma omp parallel for schedule(dynamic, 4)
    for (long long gi = cut[c]; gi < cut[c + 1]; gi++) {
      // weights times factors, the zero-weight points dropped in place (in order)
      std::vector<GridPoint>& pts = groups[gi]->points;
      const double* f = hf + first[gi];
      size_t kept = 0;
      for (size_t q = 0; q < pts.size(); q++) {
        const double w = pts[q].w * f[q];
        if (drop_zero && w == 0.0) continue;
        if (kept != q) pts[kept] = pts[q];
        pts[kept++].w = w;
      }
      pts.resize(kept);
    }
  }
}

double DeviceEngine::last_force_kernel_ms() const { return impl_->last_force_ms; }
void DeviceEngine::last_transfer_bytes(long long* h2d, long long* d2h) const {
  if (h2d) *h2d = impl_->last_h2d;
  if (d2h) *d2h = impl_->last_d2h;
}

void DeviceEngine::set_accumulators(double* d_fock_a, double* d_fock_b, double* d_energy) {
  Impl* d = impl_.get();
  if (d_fock_a && (!d_energy || (d->open && !d_fock_b)))
    throw std::runtime_error("accumulators: the energy (and for open shell the beta matrix) are needed too");
  d->ext_ka = d_fock_a;
  d->ext_kb = d_fock_a ? d_fock_b : nullptr;
  d->ext_e = d_fock_a ? d_energy : nullptr;
  d->drop_graph();  // the pointers are part of a captured build
}
void DeviceEngine::set_stream(void* s) {
  impl_->stream = s ? (cudaStream_t)s : impl_->own_stream;
}
int DeviceEngine::launches_per_solve() const { return impl_->launches; }
void DeviceEngine::set_profiling(bool on) {
  impl_->collect();
  impl_->profiling = on;
  impl_->profiled = 0;
  for (double& v : impl_->stage_ms) v = 0.0;
}
int DeviceEngine::stage_times(double* ms, int max_stages, int* solves) const {
  impl_->collect();
  for (int i = 0; i < Impl::kNumStages && i < max_stages; i++) ms[i] = impl_->stage_ms[i];
  if (solves) *solves = impl_->profiled;
  return Impl::kNumStages;
}
long long DeviceEngine::groups() const { return impl_->ngroups; }

void DeviceEngine::upload(const System& sys, const Partition& part, const std::vector<char>* keep,
                          const std::vector<BatchMember>* batch) {
  Impl* d = impl_.get();
  d->M = sys.M;
  d->natoms = sys.natoms;
  d->lda = sys.lda;
  d->open = sys.open;
  d->iexch = sys.iexch;
  d->nk = sys.lda ? 1 : 10;
  d->nkb = sys.lda ? 1 : 4;
  d->max_nftc = 0;
  d->d_norm = sys.d_norm;
  const int NQ = sys.lda ? 1 : kNQ;

  std::vector<GroupDev> gd;
  std::vector<int> hfn, hsf, hst, hfsh, hfat, hsffn;
  std::vector<ShellInfo> hsinfo;
  std::vector<int8_t> hfcp;
  std::vector<int2> btiles, ftiles, sbtiles, sdtiles;
  std::vector<int4> dtiles, ktiles, tctiles;
  long long pt_off = 0, fn_off = 0, sf_off = 0, bas_off = 0, part_off = 0;
  long long bb_off = 0, sl_off = 0, aexp_off = 0, ds_off = 0, dexp_off = 0;
  long long fa_off = 0, fae_off = 0, fbe_off = 0, rad_off = 0;
  const int NR = sys.lda ? 1 : 3;  // radial sums per (shell, point)
  std::vector<int2> farows, fbrows, fat32;
  std::vector<int4> fktiles, frtiles;
  long long npts_total = 0;
  int maxm = 0;
  const int NA = sys.lda ? 1 : 4;
  const int ngr = part.total_groups();
  if (batch && keep) throw std::runtime_error("a batch of molecules is not sharded across devices");
  size_t member = 0;                        // the batch member of group g
  std::vector<int2> member_ft;              // per member: its range of energy-partial blocks

  // The point arrays first: every device group's points, SoA at its padded
  // offset, packed on all host threads into the pinned staging (x, y, z, w one
  // after the other; padded slots hold a copy of the first point with zero
  // weight) and copied on the copy stream while the host builds the lists below.
  std::vector<int> src_group;  // partition group of each device group
  std::vector<long long> src_off;
  long long np_pad = 0;
  // sizes of the lists built below, so that each is allocated once
  size_t n_fn = 0, n_sf = 0, n_t128 = 0, n_t128f = 0, n_ftc = 0, n_dt = 0, n_kt = 0, n_fa = 0, n_fb = 0, n_fk = 0;
  for (int g = 0; g < ngr; g++) {
    if (keep && !(*keep)[g]) continue;  // another rank's group
    const PointGroup& pg = part.group(g);
    const int npts = (int)pg.points.size(), ldp = ((npts + kPointPad - 1) / kPointPad) * kPointPad;
    const int m = pg.total_functions(), nft = (m + kTile - 1) / kTile, nftc = (m + kTcFuncs - 1) / kTcFuncs;
    const int nI = (m + kFkRows - 1) / kFkRows, nJ = (m + kFkCols - 1) / kFkCols;
    src_group.push_back(g);
    src_off.push_back(np_pad);
    np_pad += ldp;
    n_fn += m;
    n_sf += pg.funcs.size();
    n_t128 += ldp / kTcPoints;
    n_t128f += (size_t)(ldp / kTcPoints) * nftc;
    n_ftc += nftc;
    n_dt += (size_t)(ldp / kTile) * nft;
    n_kt += (size_t)nft * (nft + 1) / 2;
    n_fa += (size_t)nI * kFkRows;
    n_fb += (size_t)nJ * kFkCols;
    n_fk += (size_t)nI * nJ;
  }
  for (auto* v : {&hfn, &hfsh, &hfat}) v->reserve(n_fn);
  hfcp.reserve(n_fn);
  for (auto* v : {&hsf, &hst, &hsffn}) v->reserve(n_sf);
  hsinfo.reserve(n_sf);
  farows.reserve(n_fa);
  fat32.reserve(n_fa / 32 + 1);
  fbrows.reserve(n_fb);
  fktiles.reserve(n_fk);
  frtiles.reserve(n_t128f * (sys.open ? 2 : 1));
  sbtiles.reserve(n_t128);
  sdtiles.reserve(n_ftc);
  dtiles.reserve(n_dt);
  ktiles.reserve(n_kt);
  btiles.reserve(n_t128 * kTcPoints / kBasisBlock + src_group.size());
  ftiles.reserve(n_t128 * kTcPoints / kFuncBlock + src_group.size());
  gd.reserve(src_group.size());
  PinnedStaging& ps = point_staging();
  std::lock_guard<std::mutex> ps_lock(ps.m);  // one upload at a time: held to the end of this upload
  ps.reserve(4 * (size_t)std::max(np_pad, 1LL) * sizeof(double));
  double* hx = static_cast<double*>(ps.host);
  double* hy = hx + np_pad;
  double* hz = hy + np_pad;
  double* hw = hz + np_pad;
#pragma omp parallel for schedule(dynamic, 4)
  for (long long gi = 0; gi < (long long)src_group.size(); gi++) {
    const PointGroup& pg = part.group(src_group[gi]);
    const int npts = (int)pg.points.size();
    const int ldp = ((npts + kPointPad - 1) / kPointPad) * kPointPad;
    for (int p = 0; p < ldp; p++) {
      const GridPoint& q = pg.points[p < npts ? p : 0];
      const long long o = src_off[gi] + p;
      hx[o] = q.x;
      hy[o] = q.y;
      hz[o] = q.z;
      hw[o] = p < npts ? q.w : 0.0;
    }
  }
  const cudaStream_t cs = copy_stream();
  StreamDrain drain{cs};
  for (auto [buf, src] : {std::pair<DevBuf<double>*, const double*>{&d->px, hx}, {&d->py, hy}, {&d->pz, hz},
                          {&d->pw, hw}}) {
    buf->alloc((size_t)np_pad);
    LIO_CUDA(cudaMemcpyAsync(buf->p, src, (size_t)np_pad * sizeof(double), cudaMemcpyHostToDevice, cs));
  }

  for (int g = 0; g < ngr; g++) {
    if (keep && !(*keep)[g]) continue;  // another rank's group
    const int gdev = (int)gd.size();    // its index on this device
    if (batch) {
      while (member < batch->size() && g >= (*batch)[member].g_end) member++;
      if (member >= batch->size() || g < (*batch)[member].g_begin)
        throw std::runtime_error("batch members must cover the partition's groups in order");
      if (member_ft.size() <= member) member_ft.resize(member + 1, make_int2(0, 0));
    }
    const BatchMember* bm = batch ? &(*batch)[member] : nullptr;
    const PointGroup& pg = part.group(g);
    GroupDev G{};
    G.npts = (int)pg.points.size();
    G.ldp = ((G.npts + kPointPad - 1) / kPointPad) * kPointPad;
    G.m = pg.total_functions();
    G.m32 = ((G.m + 31) / 32) * 32;
    G.nsimple = (int)pg.funcs.size();
    G.nft = (G.m + kTile - 1) / kTile;
    G.nftc = (G.m + kTcFuncs - 1) / kTcFuncs;
    G.pt_off = pt_off;
    G.fn_off = fn_off;
    G.sf_off = sf_off;
    G.bas_off = bas_off;
    G.part_off = part_off;
    G.bb_off = bb_off;
    G.sl_off = sl_off;
    G.aexp_off = aexp_off;
    G.ds_off = ds_off;
    G.dexp_off = dexp_off;
    G.fa_off = fa_off;
    G.fae_off = fae_off;
    G.fbe_off = fbe_off;
    G.rad_off = rad_off;
    G.pk_M = bm ? bm->M : sys.M;
    G.pk_off = bm ? bm->pk_off : 0;
    const int nI = (G.m + kFkRows - 1) / kFkRows, nJ = (G.m + kFkCols - 1) / kFkCols;
    for (int i = 0; i < nI * kFkRows; i++) farows.push_back({gdev, i});
    for (int j = 0; j < nJ * kFkCols; j++) fbrows.push_back({gdev, j});
    for (int i = 0; i < nI * kFkRows; i += 32) fat32.push_back({gdev, i});
    for (int I = 0; I < nI; I++)
      for (int J = 0; J < nJ; J++)
        if (J * kFkCols + kFkCols - 1 >= I * kFkRows) fktiles.push_back({gdev, I, J, 0});
    for (size_t i = 0; i < pg.funcs.size(); i++) {
      const int f = pg.funcs[i];
      const int type = !sys.ftype.empty() ? sys.ftype[f]
                                          : (f < sys.s_funcs ? 0 : (f < sys.s_funcs + 3 * sys.p_funcs ? 1 : 2));
      hsf.push_back(f);
      hst.push_back(type);
      hsffn.push_back((int)((long long)hfn.size() - G.fn_off));
      hsinfo.push_back(ShellInfo{sys.ax[sys.nuc[f]], sys.ay[sys.nuc[f]], sys.az[sys.nuc[f]], type,
                                 (int)((long long)hfn.size() - G.fn_off)});
      const int ncomp = type == 0 ? 1 : (type == 1 ? 3 : 6);
      const int c0 = type == 0 ? 0 : (type == 1 ? 1 : 4);
      for (int k = 0; k < ncomp; k++) {
        hfn.push_back(f + k - (bm ? bm->f_off : 0));  // its index in its molecule's packed matrices
        hfsh.push_back((int)i);
        hfat.push_back(sys.nuc[f]);
        const bool normed = type == 2 && (k == 0 || k == 2 || k == 5);
        hfcp.push_back((int8_t)((c0 + k) | (normed ? 16 : 0)));
      }
    }
    for (int b = 0; b < G.ldp / kBasisBlock + (G.ldp % kBasisBlock ? 1 : 0); b++) btiles.push_back({gdev, b});
    if (bm && member_ft[member].y == 0) member_ft[member] = make_int2((int)ftiles.size(), (int)ftiles.size());
    for (int b = 0; b < (G.ldp + kFuncBlock - 1) / kFuncBlock; b++) ftiles.push_back({gdev, b});
    if (bm) member_ft[member].y = (int)ftiles.size();
    for (int pt = 0; pt < G.ldp / kTile; pt++)
      for (int ft = 0; ft < G.nft; ft++) dtiles.push_back({gdev, pt, ft, 0});
    for (int it = 0; it < G.nft; it++)
      for (int jt = it; jt < G.nft; jt++) ktiles.push_back({gdev, it, jt, 0});
    for (int T = 0; T < G.ldp / kTcPoints; T++) sbtiles.push_back({gdev, T});
    maxm = std::max(maxm, G.m);
    for (int ft = 0; ft < G.nftc; ft++) sdtiles.push_back({gdev, ft});
    for (int T = 0; T < G.ldp / kTcPoints; T++)  // tensor-core forces: (tile, function tile, spin)
      for (int ft = 0; ft < G.nftc; ft++)
        for (int s = 0; s < (sys.open ? 2 : 1); s++) frtiles.push_back({gdev, T, ft, s});
    pt_off += G.ldp;
    fn_off += G.m;
    sf_off += G.nsimple;
    bas_off += (long long)d->nk * G.m * G.ldp;
    part_off += (long long)G.nft * NQ * G.ldp;
    bb_off += (long long)(G.ldp / kTcPoints) * G.nftc * d->nkb * kTcChunk;
    d->max_nftc = std::max(d->max_nftc, G.nftc);
    sl_off += (long long)(G.ldp / kTcPoints) * NA * (G.m32 / 32) * kTcStepA;
    aexp_off += (long long)NA * G.ldp;
    ds_off += (long long)G.nftc * (G.m32 / 32) * kTcStepD;
    dexp_off += (long long)G.nftc * kTcFuncs;
    for (int I = 0; I < nI; I++) fa_off += (long long)kSlices * fk_tile_rows(G.m, I) * G.ldp;
    fae_off += (long long)nI * kFkRows;
    fbe_off += (long long)nJ * kFkCols;
    rad_off += (long long)G.ldp * G.nsimple * NR;
    npts_total += G.npts;
    gd.push_back(G);
  }
  if (pt_off != np_pad) throw std::runtime_error("upload: point offsets disagree");
  d->tc_sizes[0] = bb_off;
  d->bblk_elems = bb_off;
  d->tc_sizes[1] = sl_off;
  d->tc_sizes[2] = aexp_off;
  d->tc_sizes[3] = ds_off;
  d->tc_sizes[4] = dexp_off;
  d->tc_ready = false;
  d->fk_sizes[0] = fa_off;
  d->fk_sizes[1] = fae_off;
  d->fk_sizes[3] = fbe_off;
  d->fa_rows.upload(farows);
  d->fb_rows.upload(fbrows);
  d->fa_tiles32.upload(fat32);
  d->fk_tiles.upload(fktiles);
  d->force_tc_tiles.upload(frtiles);
  d->hgroups = gd;
  d->ngroups = (long long)gd.size();
  d->npoints = npts_total;
  d->total_ldp = pt_off;

  std::vector<int> hnuc(sys.M), hnc(sys.M);
  for (int i = 0; i < sys.M; i++) {
    hnuc[i] = sys.nuc[i];
    hnc[i] = sys.ncont[i];
  }
  d->groups.upload(gd);
  d->fn_glob.upload(hfn);
  d->fn_sh.upload(hfsh);
  d->fn_atom.upload(hfat);
  d->fn_cp.upload(hfcp);
  d->slice_basis_tiles.upload(sbtiles);
  {
    // persistent tensor-core density: heaviest tiles first, dealt round-robin to the CTAs
    std::vector<int2> order = sbtiles;
    std::stable_sort(order.begin(), order.end(), [&](const int2& a, const int2& b) { return gd[a.x].m > gd[b.x].m; });
    d->dens_tc_tiles.upload(order);
    d->tc_fcap = ((maxm + 31) / 32) * 32;  // per-function table of the tensor-core density
  }
  d->slice_dens_tiles.upload(sdtiles);
  (void)tctiles;
  d->sf_glob.upload(hsf);
  d->sf_type.upload(hst);
  d->sf_fn.upload(hsffn);
  d->sinfo.upload(hsinfo);
  d->rad_elems = rad_off;
  d->nuc.upload(hnuc);
  d->ncont.upload(hnc);
  d->ca.upload(sys.a);
  d->cc.upload(sys.c);
  d->ax.upload(sys.ax);
  d->ay.upload(sys.ay);
  d->az.upload(sys.az);
  d->basis_tiles.upload(btiles);
  d->func_tiles.upload(ftiles);
  d->dens_tiles.upload(dtiles);
  d->fock_tiles.upload(ktiles);

  size_t npacked = (size_t)sys.M * (sys.M + 1) / 2;
  if (batch) {
    npacked = 0;
    for (const BatchMember& b : *batch) {
      if (b.pk_off != (long long)npacked) throw std::runtime_error("batch members' packed matrices must follow each other");
      npacked += (size_t)b.M * (b.M + 1) / 2;
    }
  }
  d->npacked = npacked;
  d->nmembers = batch ? (int)batch->size() : 0;
  if (batch) {
    member_ft.resize(batch->size(), make_int2(0, 0));
    d->member_blocks.upload(member_ft);
    d->member_energy.alloc(batch->size());
    d->h_member_energy.assign(batch->size(), 0.0);
  }
  if (batch) {
    // every molecule's whole matrices travel (small molecules' groups touch most of them)
    d->hpidx.clear();
    d->compact = false;
    d->pidx.free();
    d->Pc.free();
    d->Kc.free();
  } else {
    // the packed entries this engine's groups touch (fn_glob is increasing
    // within a group), marked by the groups on all host threads (relaxed
    // atomic byte stores: groups that share entries store the same 1)
    std::unique_ptr<std::atomic<unsigned char>[]> touched(new std::atomic<unsigned char>[npacked]);
#pragma omp parallel for schedule(static)
    for (long long e = 0; e < (long long)npacked; e++) touched[e].store(0, std::memory_order_relaxed);
    const long long Ml = sys.M;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long gi = 0; gi < (long long)gd.size(); gi++) {
      const GroupDev& G = gd[gi];
      const int* f = hfn.data() + G.fn_off;
      for (int a = 0; a < G.m; a++) {
        const long long lo = f[a], row = lo * Ml - (lo * (lo - 1)) / 2 - lo;
        for (int b = a; b < G.m; b++) touched[(size_t)(row + f[b])].store(1, std::memory_order_relaxed);
      }
    }
    // their indices in order: counted per chunk, then written per chunk
    constexpr long long kChunks = 256;
    const long long chunk = ((long long)npacked + kChunks - 1) / kChunks;
    std::vector<long long> at(kChunks + 1, 0);
#pragma omp parallel for schedule(static)
    for (long long c = 0; c < kChunks; c++) {
      long long cnt = 0;
      for (long long e = c * chunk; e < std::min((c + 1) * chunk, (long long)npacked); e++)
        cnt += touched[e].load(std::memory_order_relaxed);
      at[c + 1] = cnt;
    }
    for (long long c = 0; c < kChunks; c++) at[c + 1] += at[c];
    d->hpidx.resize((size_t)at[kChunks]);
#pragma omp parallel for schedule(static)
    for (long long c = 0; c < kChunks; c++) {
      long long o = at[c];
      for (long long e = c * chunk; e < std::min((c + 1) * chunk, (long long)npacked); e++)
        if (touched[e].load(std::memory_order_relaxed)) d->hpidx[(size_t)o++] = e;
    }
    d->compact = !d->hpidx.empty() && 2 * d->hpidx.size() <= npacked;
    const size_t nsp = sys.open ? 2 : 1;
    if (d->compact) {
      d->pidx.upload(d->hpidx);
      d->Pc.alloc(nsp * d->hpidx.size());
      d->Kc.alloc(nsp * d->hpidx.size());
    } else {
      d->pidx.free();
      d->Pc.free();
      d->Kc.free();
    }
  }
  d->P_a.alloc(npacked);
  LIO_CUDA(cudaMemset(d->P_a.p, 0, npacked * sizeof(double)));
  d->K_a.alloc(npacked);
  d->part_a.alloc(part_off);
  d->fac_a.alloc(pt_off);
  if (sys.open) {
    d->P_b.alloc(npacked);
    LIO_CUDA(cudaMemset(d->P_b.p, 0, npacked * sizeof(double)));
    d->K_b.alloc(npacked);
    d->part_b.alloc(part_off);
    d->fac_b.alloc(pt_off);
  } else {
    d->P_b.free();
    d->K_b.free();
    d->part_b.free();
    d->fac_b.free();
  }
  d->eblocks.alloc(ftiles.size());
  d->energy.alloc(1);
  d->drop_graph();
  const size_t pinned = npacked * (sys.open ? 2 : 1);
  if (!d->hK || d->pinned_elems != pinned) {  // a new geometry of the same molecule keeps them
    d->free_pinned();
    LIO_CUDA(cudaMallocHost(&d->hK, pinned * sizeof(double)));
    LIO_CUDA(cudaMallocHost(&d->hP, pinned * sizeof(double)));
    LIO_CUDA(cudaMallocHost(&d->hE, sizeof(double)));
    LIO_CUDA(cudaMallocHost(&d->hErr, sizeof(int)));
    d->pinned_elems = pinned;
  }
  if (batch && d->hme_elems < batch->size()) {
    if (d->hME) cudaFreeHost(d->hME);
    d->hME = nullptr;
    LIO_CUDA(cudaMallocHost(&d->hME, batch->size() * sizeof(double)));
    d->hme_elems = batch->size();
  }
  *d->hErr = 0;

  // basis values, computed once per geometry and kept resident (the tensor-core
  // form drops them once its operands are built, and recomputes them if the
  // FP64 form is asked for again)
  d->basis_elems = bas_off;
  d->basis_norm = sys.d_norm;
  d->basis.free();
  d->basis_valid = false;
  LIO_CUDA(cudaStreamSynchronize(cs));  // the point arrays are in place
  if (precision_ == Precision::FP64) d->compute_basis();
}

// Builds the tensor-core operands of the current geometry: the blocked FP64
// basis and the int8 slices of the density A operands (F, and for GGA its
// gradient) and of the Kohn-Sham A operand (F).
void DeviceEngine::prepare_tensor_core() {
  Impl* d = impl_.get();
  // The Kohn-Sham contraction sums over a group's points: its int32 level
  // accumulators hold (l + 1) * 64 * 64 * K at most, below 2^31 for K up to
  // 87,381 (the density and force contractions sum over functions, far fewer).
  constexpr int kTcMaxGroupPoints = 87296;  // a multiple of the 128-point padding
  for (const GroupDev& G : d->hgroups)
    if (G.ldp > kTcMaxGroupPoints)
      throw std::runtime_error("tensor-core form: a point group of " + std::to_string(G.ldp) +
                               " padded points exceeds its limit of " + std::to_string(kTcMaxGroupPoints) +
                               " (int32 level accumulators); use the FP64 form or a smaller little_cube_size");
  cudaStream_t st = d->stream;
  // the FP64 form's function-major cache is not needed (and not kept): every
  // tensor-core operand is built from the blocked copy, computed directly
  d->basis.free();
  d->basis_valid = false;
  d->compute_basis(true);
  d->aslices.alloc(d->tc_sizes[1]);
  d->aexp.alloc(d->tc_sizes[2]);
  d->dslices_a.alloc(d->tc_sizes[3]);
  d->dexp_a.alloc(d->tc_sizes[4]);
  if (d->open) {
    d->dslices_b.alloc(d->tc_sizes[3]);
    d->dexp_b.alloc(d->tc_sizes[4]);
  }
  d->tc_err.alloc(1);
  LIO_CUDA(cudaMemsetAsync(d->tc_err.p, 0, sizeof(int), st));
  // radial sums of every shell at every point, read by the density contraction's epilogue
  d->rad.alloc(d->rad_elems);
  if (d->lda)
    k_radial<1><<<(unsigned)d->slice_basis_tiles.n, kTcPoints, 0, st>>>(
        d->slice_basis_tiles.p, d->groups.p, d->px.p, d->py.p, d->pz.p, d->sf_glob.p, d->nuc.p, d->ncont.p, d->ca.p,
        d->cc.p, d->ax.p, d->ay.p, d->az.p, d->rad.p);
  else
    k_radial<3><<<(unsigned)d->slice_basis_tiles.n, kTcPoints, 0, st>>>(
        d->slice_basis_tiles.p, d->groups.p, d->px.p, d->py.p, d->pz.p, d->sf_glob.p, d->nuc.p, d->ncont.p, d->ca.p,
        d->cc.p, d->ax.p, d->ay.p, d->az.p, d->rad.p);
  LIO_CUDA(cudaGetLastError());
  if (d->lda)
    k_slice_basis<1><<<(unsigned)d->slice_basis_tiles.n, kTcPoints, 0, st>>>(d->slice_basis_tiles.p, d->groups.p,
                                                                            d->bblk.p, 1, d->aslices.p, d->aexp.p);
  else
    k_slice_basis<4><<<(unsigned)d->slice_basis_tiles.n, kTcPoints, 0, st>>>(d->slice_basis_tiles.p, d->groups.p,
                                                                            d->bblk.p, d->nkb, d->aslices.p,
                                                                            d->aexp.p);
  LIO_CUDA(cudaGetLastError());
  d->fa_slices.alloc(d->fk_sizes[0]);
  d->fa_exp.alloc(d->fk_sizes[1]);
  d->fb_exp_a.alloc(d->fk_sizes[3]);
  if (d->open) {
    d->fb_exp_b.alloc(d->fk_sizes[3]);
  }
  {
    const int nrows = (int)d->fa_rows.n;
    k_fock_rowexp<1, false><<<(unsigned)((nrows + 7) / 8), 256, 0, st>>>(
        d->fa_rows.p, nrows, d->groups.p, d->bblk.p, nullptr, nullptr, d->fa_exp.p, nullptr, 0, d->nkb,
        RadialSource{});
    LIO_CUDA(cudaGetLastError());
    k_fock_aslices<<<(unsigned)d->fa_tiles32.n, 256, 0, st>>>(d->fa_tiles32.p, d->groups.p, d->bblk.p,
                                                                d->fa_exp.p, d->fa_slices.p, d->nkb);
    LIO_CUDA(cudaGetLastError());
  }
  LIO_CUDA(cudaFuncSetAttribute(k_fock_tc<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FkCfg<1>::kSmem));
  LIO_CUDA(cudaFuncSetAttribute(k_fock_tc<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FkCfg<2>::kSmem));
  LIO_CUDA(cudaFuncSetAttribute(k_fock_tc<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FkCfg<1>::kSmem));
  LIO_CUDA(cudaFuncSetAttribute(k_fock_tc<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FkCfg<2>::kSmem));
  {
    int dev = 0;
    LIO_CUDA(cudaGetDevice(&dev));
    LIO_CUDA(cudaDeviceGetAttribute(&d->nsm, cudaDevAttrMultiProcessorCount, dev));
    const int cap = d->tc_fcap;
    int optin = 0;
    LIO_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t need = d->lda ? (d->open ? TcCfg<false, 2>::smem(cap) : TcCfg<false, 1>::smem(cap))
                               : (d->open ? TcCfg<true, 2>::smem(cap) : TcCfg<true, 1>::smem(cap));
    if (need + 256 > (size_t)optin)
      throw std::runtime_error("tensor-core density: a group with " + std::to_string(cap) +
                               " functions needs more shared memory than a block can have; use precision 0");
    // only the variant this system runs (the others may not fit at this cap), and
    // only ever raised: the limit belongs to the kernel, which every engine of the
    // process shares, and an engine with larger groups may launch it later
    auto raise_limit = [&](const void* fn) {
      static std::mutex mu;
      std::lock_guard<std::mutex> lock(mu);
      cudaFuncAttributes fa;
      LIO_CUDA(cudaFuncGetAttributes(&fa, fn));
      if ((int)need > fa.maxDynamicSharedSizeBytes)
        LIO_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
    };
    if (d->lda && d->open)
      raise_limit((const void*)k_density_tc<false, 2>);
    else if (d->lda)
      raise_limit((const void*)k_density_tc<false, 1>);
    else if (d->open)
      raise_limit((const void*)k_density_tc<true, 2>);
    else
      raise_limit((const void*)k_density_tc<true, 1>);
  }
  // a lean engine keeps the operands only: the Kohn-Sham kernels then form F
  // from the radial sums, and forces rebuild the blocked basis when asked
  if (d->lean) d->bblk.free();  // cudaFree waits for the kernels above
  d->tc_ready = true;
}

// The device work of one solve, from the densities in d->P_a / d->P_b to E_xc in
// d->energy and the Kohn-Sham contributions in d->K_a / d->K_b (ext: added into
// the external accumulators instead); captured once into a CUDA graph when
// graphs are on. Returns the number of kernel launches.
int DeviceEngine::run_kernels(bool compute_rmm, bool ext) {
  Impl* d = impl_.get();
  double* Ka = ext ? d->ext_ka : d->K_a.p;
  double* Kb = ext ? d->ext_kb : d->K_b.p;
  const size_t npacked = d->npacked;
  cudaStream_t st = d->stream;
  int launches = 0;
  const unsigned nd = (unsigned)d->dens_tiles.n, nf = (unsigned)d->func_tiles.n,
                 nk = (unsigned)d->fock_tiles.n;
  d->mark(0);
  const int nspin = d->open ? 2 : 1;
  const bool tc = precision_ == Precision::TensorCore;
  if (tc) {
    // D slices of each spin, then one launch for both spins (shared A slices and basis rebuild)
    for (int s = 0; s < nspin; s++) {
      const double* P = s == 0 ? d->P_a.p : d->P_b.p;
      int8_t* dsl = s == 0 ? d->dslices_a.p : d->dslices_b.p;
      int16_t* dex = s == 0 ? d->dexp_a.p : d->dexp_b.p;
      k_slice_density<<<(unsigned)d->slice_dens_tiles.n, kTcFuncs, 0, st>>>(d->slice_dens_tiles.p, d->groups.p,
                                                                          d->fn_glob.p, P, d->M, dsl, dex);
      LIO_CUDA(cudaGetLastError());
      launches++;
    }
    d->mark(1);
    const int ntiles = (int)d->dens_tc_tiles.n;
    const unsigned nt = (unsigned)std::min(ntiles, d->nsm);
    const int cap = d->tc_fcap;
#define LIO_DENSITY_TC(GGA, NS)                                                                                    \
  k_density_tc<GGA, NS><<<nt, TcCfg<GGA, NS>::kThreads, TcCfg<GGA, NS>::smem(cap), st>>>(                          \
      d->dens_tc_tiles.p, ntiles, d->groups.p, d->aslices.p, d->aexp.p, d->dslices_a.p, d->dexp_a.p,               \
      d->dslices_b.p, d->dexp_b.p, cap, d->px.p, d->py.p, d->pz.p, d->fn_sh.p, d->sinfo.p, d->rad.p, d->basis_norm,    \
      d->part_a.p, d->part_b.p, d->tc_err.p)
    if (d->lda) {
      if (d->open) LIO_DENSITY_TC(false, 2); else LIO_DENSITY_TC(false, 1);
    } else {
      if (d->open) LIO_DENSITY_TC(true, 2); else LIO_DENSITY_TC(true, 1);
    }
#undef LIO_DENSITY_TC
    LIO_CUDA(cudaGetLastError());
    launches++;
  } else {
    d->mark(1);  // no operand preparation in the FP64 form
    for (int s = 0; s < nspin; s++) {
      const double* P = s == 0 ? d->P_a.p : d->P_b.p;
      double* part = s == 0 ? d->part_a.p : d->part_b.p;
      if (d->lda)
        k_density_fp64<1><<<nd, 256, 0, st>>>(d->dens_tiles.p, d->groups.p, d->fn_glob.p, d->basis.p, P, d->M, part,
                                              0);
      else
        k_density_fp64<4><<<nd, 256, 0, st>>>(d->dens_tiles.p, d->groups.p, d->fn_glob.p, d->basis.p, P, d->M, part,
                                              0);
      LIO_CUDA(cudaGetLastError());
      launches++;
    }
  }
  d->mark(2);
  // the tensor-core density writes one partial per point, the FP64 one one per 64-function tile
  launch_functional(d->lda, d->open, nf, st, d->func_tiles.p, d->groups.p, d->pw.p, d->part_a.p,
                    d->open ? d->part_b.p : nullptr, tc ? (1 << 30) : kTile, d->iexch, d->fac_a.p,
                    d->open ? d->fac_b.p : nullptr, d->eblocks.p);
  LIO_CUDA(cudaGetLastError());
  k_sum_blocks<<<1, 1024, 0, st>>>(d->eblocks.p, (int)nf, ext ? d->ext_e : d->energy.p, ext ? 1 : 0);
  LIO_CUDA(cudaGetLastError());
  launches += 2;
  if (d->nmembers > 0) {  // a batch: each molecule's E_xc as well
    k_sum_segments<<<(unsigned)d->nmembers, 256, 0, st>>>(d->eblocks.p, d->member_blocks.p, d->member_energy.p);
    LIO_CUDA(cudaGetLastError());
    launches++;
  }
  d->mark(3);
  if (compute_rmm) {
    if (!ext) {  // an external accumulator is zeroed by its owner, once for all shards
      LIO_CUDA(cudaMemsetAsync(d->K_a.p, 0, npacked * sizeof(double), st));
      if (d->open) LIO_CUDA(cudaMemsetAsync(d->K_b.p, 0, npacked * sizeof(double), st));
    }
    if (tc) {
      // row exponents of f * F (both spins, one pass over F); the contraction
      // kernel cuts the f * F slices itself. F from the blocked basis, or (a lean
      // engine) from the radial sums.
      const int nrows = (int)d->fb_rows.n;
      const RadialSource rs{d->rad.p,    d->px.p, d->py.p, d->pz.p, d->fn_sh.p,      d->fn_cp.p,
                            d->fn_atom.p, d->ax.p, d->ay.p, d->az.p, d->basis_norm, d->lda ? 1 : 3};
      const unsigned nb = (unsigned)((nrows + 7) / 8);
      const double* fb = d->fac_b.p;
      int16_t* eb = d->fb_exp_b.p;
      if (!d->bblk.p) {
        if (d->open)
          k_fock_rowexp<2, true><<<nb, 256, 0, st>>>(d->fb_rows.p, nrows, d->groups.p, nullptr, d->fac_a.p, fb,
                                                     d->fb_exp_a.p, eb, 1, 0, rs);
        else
          k_fock_rowexp<1, true><<<nb, 256, 0, st>>>(d->fb_rows.p, nrows, d->groups.p, nullptr, d->fac_a.p, nullptr,
                                                     d->fb_exp_a.p, nullptr, 1, 0, rs);
      } else {
        if (d->open)
          k_fock_rowexp<2, false><<<nb, 256, 0, st>>>(d->fb_rows.p, nrows, d->groups.p, d->bblk.p, d->fac_a.p, fb,
                                                      d->fb_exp_a.p, eb, 1, d->nkb, rs);
        else
          k_fock_rowexp<1, false><<<nb, 256, 0, st>>>(d->fb_rows.p, nrows, d->groups.p, d->bblk.p, d->fac_a.p,
                                                      nullptr, d->fb_exp_a.p, nullptr, 1, d->nkb, rs);
      }
      LIO_CUDA(cudaGetLastError());
      launches++;
      d->mark(4);
      const unsigned nt = (unsigned)d->fk_tiles.n;
#define launch_fock(NS_, RAD_)                                                                                        \
  k_fock_tc<NS_, RAD_><<<nt, FkCfg<NS_>::kThreads, FkCfg<NS_>::kSmem, st>>>(                                      \
      d->fk_tiles.p, d->groups.p, d->fn_glob.p, d->fa_slices.p, d->fa_exp.p, d->bblk.p, d->nkb, d->fac_a.p,         \
      NS_ == 2 ? fb : nullptr, d->fb_exp_a.p, NS_ == 2 ? eb : nullptr, d->M, Ka, NS_ == 2 ? Kb : nullptr,           \
      d->tc_err.p, rs)
      if (d->open && !d->bblk.p)
        launch_fock(2, true);
      else if (d->open)
        launch_fock(2, false);
      else if (!d->bblk.p)
        launch_fock(1, true);
      else
        launch_fock(1, false);
#undef launch_fock
    } else if (d->open) {
      d->mark(4);  // no operand preparation in the FP64 form
      k_fock_fp64<2><<<nk, 256, 0, st>>>(d->fock_tiles.p, d->groups.p, d->fn_glob.p, d->basis.p, d->fac_a.p,
                                         d->fac_b.p, d->M, Ka, Kb, 0);
    } else {
      d->mark(4);
      k_fock_fp64<1><<<nk, 256, 0, st>>>(d->fock_tiles.p, d->groups.p, d->fn_glob.p, d->basis.p, d->fac_a.p,
                                         nullptr, d->M, Ka, nullptr, 0);
    }
    LIO_CUDA(cudaGetLastError());
    launches++;
  }
  if (!compute_rmm) d->mark(4);
  d->mark(5);
  return launches;
}

void DeviceEngine::set_graphs(bool on) {
  impl_->use_graphs = on;
  impl_->drop_graph();
}
void DeviceEngine::set_graphs_dirty() { impl_->drop_graph(); }

void DeviceEngine::copy_results(double* d_fock_a, double* d_fock_b, double* d_energy) {
  Impl* d = impl_.get();
  const size_t npacked = d->npacked;
  if (d_fock_a)
    LIO_CUDA(cudaMemcpyAsync(d_fock_a, d->K_a.p, npacked * sizeof(double), cudaMemcpyDeviceToDevice, d->stream));
  if (d_fock_b && d->open)
    LIO_CUDA(cudaMemcpyAsync(d_fock_b, d->K_b.p, npacked * sizeof(double), cudaMemcpyDeviceToDevice, d->stream));
  if (d_energy) LIO_CUDA(cudaMemcpyAsync(d_energy, d->energy.p, sizeof(double), cudaMemcpyDeviceToDevice, d->stream));
}

void DeviceEngine::prepare() {
  Impl* d = impl_.get();
  if (d->ngroups == 0) return;  // nothing to build (e.g. a shard that owns no group)
  if (precision_ == Precision::TensorCore && !d->tc_ready) {
    prepare_tensor_core();
    d->drop_graph();
    LIO_CUDA(cudaStreamSynchronize(d->stream));
  } else if (precision_ == Precision::FP64 && !d->basis_valid && d->ngroups > 0) {
    d->compute_basis();  // synchronises
    d->drop_graph();
  }
}

size_t DeviceEngine::cache_bytes() const {
  const Impl* d = impl_.get();
  size_t b = (d->basis.cap + d->bblk.cap + d->rad.cap) * sizeof(double);
  for (const auto* x : {&d->aslices, &d->dslices_a, &d->dslices_b, &d->fa_slices})
    b += x->cap;
  for (const auto* x : {&d->aexp, &d->dexp_a, &d->dexp_b, &d->fa_exp, &d->fb_exp_a, &d->fb_exp_b})
    b += x->cap * sizeof(int16_t);
  return b;
}

void DeviceEngine::release_caches() {
  Impl* d = impl_.get();
  LIO_CUDA(cudaStreamSynchronize(d->stream));  // no build in flight reads them
  d->basis.free();
  d->basis_valid = false;
  drop_tensor_core();
}

long long DeviceEngine::process_device_bytes() { return g_devbuf_bytes.load(); }

void DeviceEngine::drop_tensor_core() {
  Impl* d = impl_.get();
  for (auto* b : {&d->aslices, &d->dslices_a, &d->dslices_b, &d->fa_slices})
    b->free();
  for (auto* b : {&d->aexp, &d->dexp_a, &d->dexp_b, &d->fa_exp, &d->fb_exp_a, &d->fb_exp_b}) b->free();
  d->bblk.free();
  d->rad.free();
  d->tc_ready = false;
  d->drop_graph();
}

void DeviceEngine::autotune_measure(double* fp64_ms, double* tc_ms, size_t* fp64_cache, size_t* tc_cache) {
  Impl* d = impl_.get();
  auto time_form = [&](Precision p) {
    set_precision(p);
    SolveRequest req;
    req.resident = true;
    solve(req);  // builds the form's operands and captures its graph
    LIO_CUDA(cudaStreamSynchronize(d->stream));
    cudaEvent_t a, b;
    LIO_CUDA(cudaEventCreate(&a));
    LIO_CUDA(cudaEventCreate(&b));
    LIO_CUDA(cudaEventRecord(a, d->stream));
    for (int k = 0; k < 2; k++) solve(req);
    LIO_CUDA(cudaEventRecord(b, d->stream));
    LIO_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    LIO_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / 2;
  };
  d->tuned_fp64_ms = time_form(Precision::FP64);
  *fp64_cache = cache_bytes();
  try {
    d->tuned_tc_ms = time_form(Precision::TensorCore);  // its operands replace the FP64 cache
    *tc_cache = cache_bytes();
  } catch (const std::exception&) {
    // a form this molecule cannot run (e.g. a group too large for the tensor-core
    // kernel's shared memory): it is never the faster
    cudaGetLastError();
    drop_tensor_core();
    d->tuned_tc_ms = std::numeric_limits<double>::infinity();
    *tc_cache = 0;
  }
  *fp64_ms = d->tuned_fp64_ms;
  *tc_ms = d->tuned_tc_ms;
}

void DeviceEngine::keep_form(Precision p) {
  Impl* d = impl_.get();
  if (p == Precision::FP64) {
    drop_tensor_core();
    set_precision(Precision::FP64);
    if (!d->basis_valid && d->ngroups > 0) d->compute_basis();
  } else {
    set_precision(Precision::TensorCore);
    prepare();
  }
}

// The autotuner: one resident build of each form after a warm-up (the density
// contents do not change the work of either), the faster one kept and the
// other's caches released. Memory-aware: the tensor-core form is kept only when
// its time x cache-bytes product is the smaller.
Precision DeviceEngine::autotune(bool memory_aware) {
  Impl* d = impl_.get();
  if (d->ngroups == 0) return precision_;
  double t64 = 0, ttc = 0;
  size_t c64 = 0, ctc = 0;
  autotune_measure(&t64, &ttc, &c64, &ctc);
  const bool tc_wins = memory_aware ? ttc * (double)(ctc + 1) < t64 * (double)(c64 + 1) : ttc < t64;
  keep_form(tc_wins ? Precision::TensorCore : Precision::FP64);
  return precision_;
}

void DeviceEngine::tuned_times(double* fp64_ms, double* tc_ms) const {
  *fp64_ms = impl_->tuned_fp64_ms;
  *tc_ms = impl_->tuned_tc_ms;
}

void DeviceEngine::set_lean(bool on) {
  Impl* d = impl_.get();
  d->lean = on;
  if (on && d->tc_ready && precision_ == Precision::TensorCore && d->bblk.p) {
    LIO_CUDA(cudaStreamSynchronize(d->stream));  // no build in flight reads it
    d->bblk.free();
    d->drop_graph();  // the captured Kohn-Sham launches read it
  }
}
bool DeviceEngine::lean() const { return impl_->lean; }

size_t DeviceEngine::estimate_blocked_basis_bytes(const System& sys, const Partition& part) {
  double b = 0.0;
  for (int g = 0; g < part.total_groups(); g++) {
    const PointGroup& pg = part.group(g);
    const double ldp = (double)(((long long)pg.points.size() + kPointPad - 1) / kPointPad * kPointPad);
    const int nftc = (pg.total_functions() + kTcFuncs - 1) / kTcFuncs;
    b += ldp * nftc * kTcFuncs * (sys.lda ? 1 : 4) * 8.0;
  }
  return (size_t)b;
}

size_t DeviceEngine::estimate_device_bytes(const System& sys, const Partition& part, Precision prec, bool lean) {
  const int nk = sys.lda ? 1 : 10, na = sys.lda ? 1 : 4, nq = sys.lda ? 1 : kNQ, nspin = sys.open ? 2 : 1;
  const size_t npacked = (size_t)sys.M * (sys.M + 1) / 2;
  double b = (double)npacked * 8 * 2 * nspin;  // densities and Kohn-Sham accumulators
  for (int g = 0; g < part.total_groups(); g++) {
    const PointGroup& pg = part.group(g);
    const double ldp = (double)(((long long)pg.points.size() + kPointPad - 1) / kPointPad * kPointPad);
    const int m = pg.total_functions(), m32 = (m + 31) / 32 * 32;
    const int nft = (m + kTile - 1) / kTile, nftc = (m + kTcFuncs - 1) / kTcFuncs;
    const int nI = (m + kFkRows - 1) / kFkRows;
    b += ldp * (6 * 8 + nspin * (nq * (double)nft * 8 + 8));  // points, partials, factors
    if (prec == Precision::FP64) b += ldp * nk * (double)m * 8;  // function-major basis cache
    if (prec == Precision::TensorCore)
      b += ldp * ((lean ? 0.0 : (double)nftc * kTcFuncs * (sys.lda ? 1 : 4) * 8) +  // blocked basis
                  (double)pg.funcs.size() * (sys.lda ? 1 : 3) * 8 +
                  (double)na * m32 * kSlices + na * 2 +
                  (double)(nI > 0 ? (nI - 1) * kFkRows + fk_tile_rows(m, nI - 1) : 0) * kSlices) +
           (double)nspin * nftc * m32 * kTcTall;
  }
  return (size_t)(b * 1.05) + (16u << 20);
}

void DeviceEngine::enqueue(const SolveRequest& req) {
  Impl* d = impl_.get();
  const size_t npacked = d->npacked;
  d->enqueued = false;
  if (d->ngroups == 0) return;
  cudaStream_t st = d->stream;
  const bool tc = precision_ == Precision::TensorCore;
  if (tc && !d->tc_ready) {
    prepare_tensor_core();
    d->drop_graph();
  }
  if (!tc && !d->basis_valid) {
    d->compute_basis();
    d->drop_graph();
  }
  d->collect();
  LIO_CUDA(cudaEventRecord(d->ev0, st));
  if (!req.resident) {
    // the caller's (pageable) densities through pinned staging: a threaded host
    // copy, then one full-speed copy per spin
    const int nspin = d->open ? 2 : 1;
    if (d->compact) {
      // the touched entries only: gathered per spin by all host threads, each
      // spin sent while the next is gathered, then scattered on the device
      const long long np = (long long)d->hpidx.size();
      const long long* ix = d->hpidx.data();
      for (int s = 0; s < nspin; s++) {
        const double* src = d->open ? (s == 0 ? req.rho_a : req.rho_b) : req.rho;
        double* h = d->hP + (size_t)s * np;
#pragma omp parallel for schedule(static) if (np > (1 << 16))
        for (long long k = 0; k < np; k++) h[k] = src[ix[k]];
        LIO_CUDA(cudaMemcpyAsync(d->Pc.p + (size_t)s * np, h, (size_t)np * sizeof(double), cudaMemcpyHostToDevice,
                                 st));
      }
      k_scatter_packed<<<(unsigned)std::min<long long>((nspin * np + 255) / 256, 4096), 256, 0, st>>>(
          d->Pc.p, d->pidx.p, np, nspin, d->P_a.p, d->open ? d->P_b.p : nullptr);
      LIO_CUDA(cudaGetLastError());
      d->last_h2d = (long long)nspin * np * (long long)sizeof(double);
    } else {
      // in pieces, so that the host copy of one piece overlaps the transfer of the last
      const size_t piece = std::max<size_t>(npacked / 8, 1 << 16);
      for (int s = 0; s < nspin; s++) {
        const double* src = d->open ? (s == 0 ? req.rho_a : req.rho_b) : req.rho;
        double* dst = s == 0 ? d->P_a.p : d->P_b.p;
        for (size_t o = 0; o < npacked; o += piece) {
          const size_t n = std::min(piece, npacked - o);
          host_copy(d->hP + s * npacked + o, src + o, n);
          LIO_CUDA(
              cudaMemcpyAsync(dst + o, d->hP + s * npacked + o, n * sizeof(double), cudaMemcpyHostToDevice, st));
        }
      }
      d->last_h2d = (long long)nspin * (long long)npacked * (long long)sizeof(double);
    }
  }
  // graph replay when on (not while profiling: the stage events are recorded eagerly)
  const bool ext = req.resident && d->ext_ka != nullptr;
  const int key = (tc ? 2 : 0) | (req.compute_rmm ? 1 : 0) | (ext ? 4 : 0);
  if (d->use_graphs && !d->profiling) {
    if (!d->graph_exec || d->graph_key != key) {
      d->drop_graph();
      cudaGraph_t g = nullptr;
      LIO_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      int n = 0;
      try {
        n = run_kernels(req.compute_rmm, ext);
      } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      LIO_CUDA(cudaStreamEndCapture(st, &g));
      LIO_CUDA(cudaGraphInstantiate(&d->graph_exec, g, 0));
      LIO_CUDA(cudaGraphDestroy(g));
      d->graph_key = key;
      d->graph_launches = n;
    }
    LIO_CUDA(cudaGraphLaunch(d->graph_exec, st));
    d->launches = d->graph_launches;
  } else {
    d->launches = run_kernels(req.compute_rmm, ext);
    d->pending = d->profiling;
  }
  if (!req.resident) {
    const int nspin = d->open ? 2 : 1;
    LIO_CUDA(cudaMemcpyAsync(d->hE, d->energy.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (d->nmembers > 0)
      LIO_CUDA(cudaMemcpyAsync(d->hME, d->member_energy.p, (size_t)d->nmembers * sizeof(double),
                               cudaMemcpyDeviceToHost, st));
    if (tc) LIO_CUDA(cudaMemcpyAsync(d->hErr, d->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    d->nchunks = 0;
    d->last_d2h = (long long)sizeof(double);  // the energy
    if (req.compute_rmm && d->compact) {  // the touched entries, gathered, in pieces with an event after each
      const long long np = (long long)d->hpidx.size();
      k_gather_packed<<<(unsigned)std::min<long long>((nspin * np + 255) / 256, 4096), 256, 0, st>>>(
          d->K_a.p, d->open ? d->K_b.p : nullptr, d->pidx.p, np, nspin, d->Kc.p);
      LIO_CUDA(cudaGetLastError());
      const size_t total = (size_t)nspin * np;
      const size_t piece = compact_piece(total);
      for (size_t o = 0; o < total; o += piece, d->nchunks++) {
        LIO_CUDA(cudaMemcpyAsync(d->hK + o, d->Kc.p + o, std::min(piece, total - o) * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
        LIO_CUDA(cudaEventRecord(d->kev[d->nchunks], st));
      }
      d->last_d2h += (long long)total * (long long)sizeof(double);
    } else if (req.compute_rmm) {  // nspin x npacked values in up to kMaxChunks pieces, an event after each
      const size_t total = (size_t)nspin * npacked;
      d->last_d2h += (long long)total * (long long)sizeof(double);
      const size_t piece = std::max<size_t>((total + Impl::kMaxChunks - 1) / Impl::kMaxChunks, 1 << 16);
      for (size_t o = 0; o < total; o += piece, d->nchunks++) {
        const size_t n = std::min(piece, total - o);
        for (size_t e = o; e < o + n;) {  // a piece may span the two spins' device buffers
          const int s = (int)(e / npacked);
          const size_t in_s = e - (size_t)s * npacked, m = std::min(o + n - e, npacked - in_s);
          LIO_CUDA(cudaMemcpyAsync(d->hK + e, (s == 0 ? d->K_a.p : d->K_b.p) + in_s, m * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
          e += m;
        }
        LIO_CUDA(cudaEventRecord(d->kev[d->nchunks], st));
      }
    }
  }
  LIO_CUDA(cudaEventRecord(d->ev1, st));
  d->enqueued = true;
}

bool DeviceEngine::ready() const {
  Impl* d = impl_.get();
  if (!d->enqueued) return true;
  const cudaError_t e = cudaEventQuery(d->ev1);
  if (e == cudaErrorNotReady) return false;
  LIO_CUDA(e);
  return true;
}

SolveResult DeviceEngine::finish(const SolveRequest& req) {
  Impl* d = impl_.get();
  SolveResult res;
  if (!d->enqueued) return res;
  d->enqueued = false;
  if (req.resident) return res;
  const size_t npacked = d->npacked;
  // the energy and the error flag are downloaded before the first Kohn-Sham piece
  LIO_CUDA(cudaEventSynchronize(req.compute_rmm && d->nchunks > 0 ? d->kev[0] : d->ev1));
  if (precision_ == Precision::TensorCore && *d->hErr) {
    LIO_CUDA(cudaEventSynchronize(d->ev1));
    throw std::runtime_error("tensor-core density: an MMA completion wait timed out");
  }
  if (req.compute_rmm && d->compact) {  // scatter-added chunk by chunk as they arrive
    const int nspin = d->open ? 2 : 1;
    const long long np = (long long)d->hpidx.size();
    const long long* ix = d->hpidx.data();
    const size_t total = (size_t)nspin * np;
    const size_t piece = compact_piece(total);
    int c = 0;
    for (size_t o = 0; o < total; o += piece, c++) {
      LIO_CUDA(cudaEventSynchronize(d->kev[c]));
      const long long k1 = (long long)std::min(o + piece, total);
#pragma omp parallel for schedule(static) if (k1 - (long long)o >= (1 << 12))
      for (long long k = (long long)o; k < k1; k++) {
        double* f = k < np ? req.fock : req.fock_b;  // indices are unique: no two threads add to one entry
        f[ix[k < np ? k : k - np]] += d->hK[k];
      }
    }
  } else if (req.compute_rmm) {  // chunk by chunk as they arrive (the same pieces enqueue downloaded)
    const int nspin = d->open ? 2 : 1;
    const size_t total = (size_t)nspin * npacked;
    const size_t piece = std::max<size_t>((total + Impl::kMaxChunks - 1) / Impl::kMaxChunks, 1 << 16);
    int c = 0;
    for (size_t o = 0; o < total; o += piece, c++) {
      LIO_CUDA(cudaEventSynchronize(d->kev[c]));
      const size_t n = std::min(piece, total - o);
      for (size_t e = o; e < o + n;) {
        const int s = (int)(e / npacked);
        const size_t in_s = e - (size_t)s * npacked, m = std::min(o + n - e, npacked - in_s);
        host_accumulate((s == 0 ? req.fock : req.fock_b) + in_s, d->hK + e, m);
        e += m;
      }
    }
  }
  LIO_CUDA(cudaEventSynchronize(d->ev1));
  float ms = 0.f;
  LIO_CUDA(cudaEventElapsedTime(&ms, d->ev0, d->ev1));
  res.energy = *d->hE;
  res.device_ms = ms;
  for (int k = 0; k < d->nmembers; k++) d->h_member_energy[k] = d->hME[k];
  return res;
}

int DeviceEngine::batch_energies(double* out) const {
  const Impl* d = impl_.get();
  for (int k = 0; k < d->nmembers; k++) out[k] = d->h_member_energy[k];
  return d->nmembers;
}

size_t DeviceEngine::packed_size() const { return impl_->npacked; }

SolveResult DeviceEngine::solve(const SolveRequest& req) {
  enqueue(req);
  return finish(req);
}

SolveResult DeviceEngine::solve_forces(const SolveRequest& req, double* forces, int ld) {
  Impl* d = impl_.get();
  if (!forces || ld < d->natoms) throw std::runtime_error("forces: null array or leading dimension below natoms");
  SolveRequest r = req;
  r.compute_rmm = false;
  r.resident = false;
  const SolveResult res = solve(r);  // densities uploaded, factors in fac_a / fac_b
  if (d->ngroups == 0) return res;
  cudaStream_t st = d->stream;
  // F and its gradient: the resident cache of the GGA forms, or (LDA keeps F
  // only) a four-kind function-major cache built for this call
  DevBuf<double> grad;
  BasisView bv{nullptr, 0, 1};
  if (d->lda) {
    grad.alloc((size_t)4 * d->basis_elems);
    k_basis<<<(unsigned)d->basis_tiles.n, kBasisBlock, 0, st>>>(
        d->basis_tiles.p, d->groups.p, d->px.p, d->py.p, d->pz.p, d->sf_glob.p, d->sf_type.p, d->nuc.p, d->ncont.p,
        d->ca.p, d->cc.p, d->ax.p, d->ay.p, d->az.p, d->basis_norm, 4, grad.p, 0, 4);
    LIO_CUDA(cudaGetLastError());
    bv = BasisView{grad.p, 0, 4};
  } else if (precision_ == Precision::TensorCore) {
    if (!d->bblk.p) d->compute_basis(true);  // a lean engine: rebuilt for the forces
    bv = BasisView{d->bblk.p, d->nkb, 1};
  } else {
    bv = BasisView{d->basis.p, 0, 1};
  }
  DevBuf<double> frc;
  frc.alloc((size_t)3 * d->natoms);
  LIO_CUDA(cudaMemsetAsync(frc.p, 0, (size_t)3 * d->natoms * sizeof(double), st));
  const unsigned nd = (unsigned)d->dens_tiles.n;
  const bool tc = precision_ == Precision::TensorCore && !d->lda;
  LIO_CUDA(cudaEventRecord(d->fev0, st));
  if (tc) {
    // G from the build's own int8 operands (F slices, stacked density slices) on tcgen05
    LIO_CUDA(cudaFuncSetAttribute(k_force_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FtCfg::kSmem));
    const int nu = (int)d->force_tc_tiles.n;
    k_force_tc<<<(unsigned)std::min(nu, 2 * d->nsm), FtCfg::kThreads, FtCfg::kSmem, st>>>(
        d->force_tc_tiles.p, nu, d->groups.p, 4, d->aslices.p, d->aexp.p, d->dslices_a.p, d->dexp_a.p,
        d->open ? d->dslices_b.p : nullptr, d->open ? d->dexp_b.p : nullptr, d->bblk.p, d->nkb, d->fac_a.p,
        d->open ? d->fac_b.p : nullptr, d->fn_atom.p, frc.p, d->tc_err.p);
  } else if (d->open)
    k_force_fp64<2><<<nd, 256, 0, st>>>(d->dens_tiles.p, d->groups.p, d->fn_glob.p, d->fn_atom.p, bv, d->P_a.p,
                                        d->P_b.p, d->M, d->fac_a.p, d->fac_b.p, frc.p);
  else
    k_force_fp64<1><<<nd, 256, 0, st>>>(d->dens_tiles.p, d->groups.p, d->fn_glob.p, d->fn_atom.p, bv, d->P_a.p,
                                        nullptr, d->M, d->fac_a.p, nullptr, frc.p);
  LIO_CUDA(cudaGetLastError());
  LIO_CUDA(cudaEventRecord(d->fev1, st));
  std::vector<double> h((size_t)3 * d->natoms);
  LIO_CUDA(cudaMemcpyAsync(h.data(), frc.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  int terr = 0;
  if (tc) LIO_CUDA(cudaMemcpyAsync(&terr, d->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  LIO_CUDA(cudaStreamSynchronize(st));
  if (terr) throw std::runtime_error("tensor-core forces: an MMA completion wait timed out");
  if (d->lean && d->bblk.p) d->bblk.free();  // back to the operands-only footprint
  float fms = 0.f;
  LIO_CUDA(cudaEventElapsedTime(&fms, d->fev0, d->fev1));
  d->last_force_ms = fms;
  for (int a = 0; a < d->natoms; a++)
    for (int x = 0; x < 3; x++) forces[a + (size_t)ld * x] += h[(size_t)a * 3 + x];
  return res;
}

// ======================================================= no-allocation variant
// Callers that cannot allocate device memory (an MD engine or SCF driver that
// hands all of the GPU's memory to its own pool, or code running where a
// cudaMalloc is not allowed to happen) use this path: the per-solve scratch of
// the density, functional and energy stages sits in the fixed array below,
// which every GPU that loads this library holds until the process exits.
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
constexpr size_t kNoAllocDoubles = kNoAllocScratchBytes / sizeof(double);
constexpr size_t kNoAllocEnergySlots = 4096;  // one partial energy per batch
__device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[128] = {nullptr};

// The host-side name g_noalloc_scratch is only a stand-in for the symbol; the
// device address is looked up once per device, with that device current.
double* noalloc_scratch_address() {
  int dev = 0;
  LIO_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) throw std::runtime_error("device ordinal out of range for the no-alloc scratch table");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    LIO_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  return g_noalloc_ptr[dev];
}
}  // namespace

size_t DeviceEngine::noalloc_scratch_bytes() { return kNoAllocScratchBytes; }

void DeviceEngine::solve_noalloc(const double* rho_a, const double* rho_b, double* fock_a, double* fock_b,
                                 double* energy, void* cuda_stream) {
  Impl* d = impl_.get();
  if (d->ngroups == 0) throw std::runtime_error("no grid uploaded");
  if (!rho_a || !fock_a || !energy || (d->open && (!rho_b || !fock_b)))
    throw std::runtime_error("null device pointer");
  // The FP64 form's basis cache must be resident: building it would allocate
  // (gigabytes at a few hundred atoms), which is what this entry point's callers
  // cannot do. A grid built or autotuned into the tensor-core form does not keep it.
  if (!d->basis_valid)
    throw std::runtime_error(
        "the no-allocation entry point needs the FP64 form's resident basis values, which this grid does not hold "
        "(it was built or autotuned in the tensor-core form): call g2g_set_precision_(0) before "
        "g2g_reload_atom_positions_");
  double* scratch = noalloc_scratch_address();
  cudaStream_t st = cuda_stream ? (cudaStream_t)cuda_stream : d->stream;
  const int nspin = d->open ? 2 : 1;
  const int NQ = d->lda ? 1 : kNQ;
  const size_t usable = kNoAllocDoubles - kNoAllocEnergySlots;
  double* eparts = scratch;  // one partial energy per batch, all written before they are read
  double* region = scratch + kNoAllocEnergySlots;

  // per-group tile counts in the order upload() generated the tile lists
  auto ndt = [](const GroupDev& G) { return (long long)(G.ldp / kTile) * G.nft; };
  auto nft_ = [](const GroupDev& G) { return (long long)((G.ldp + kFuncBlock - 1) / kFuncBlock); };
  auto nkt = [](const GroupDev& G) { return (long long)G.nft * (G.nft + 1) / 2; };
  auto need = [&](const GroupDev& G) {
    return (size_t)nspin * ((size_t)G.nft * NQ * G.ldp + G.ldp) + (size_t)nft_(G);
  };
  long long dt0 = 0, ft0 = 0, kt0 = 0;
  int nbatch = 0;
  int g0 = 0;
  const int ng = (int)d->ngroups;
  while (g0 < ng) {
    size_t used = 0;
    int g1 = g0;
    long long nd = 0, nf = 0, nk = 0;
    while (g1 < ng && used + need(d->hgroups[g1]) <= usable) {
      used += need(d->hgroups[g1]);
      nd += ndt(d->hgroups[g1]);
      nf += nft_(d->hgroups[g1]);
      nk += nkt(d->hgroups[g1]);
      g1++;
    }
    if (g1 == g0)
      throw std::runtime_error("group " + std::to_string(g0) + " needs " +
                               std::to_string(need(d->hgroups[g0]) * sizeof(double)) +
                               " bytes of scratch; the no-alloc entry point holds " +
                               std::to_string(kNoAllocScratchBytes - kNoAllocEnergySlots * sizeof(double)));
    if (nbatch >= (int)kNoAllocEnergySlots) throw std::runtime_error("too many batches for the no-alloc scratch");
    const GroupDev& first = d->hgroups[g0];
    long long part_len = 0, fac_len = 0;
    for (int g = g0; g < g1; g++) {
      part_len += (long long)d->hgroups[g].nft * NQ * d->hgroups[g].ldp;
      fac_len += d->hgroups[g].ldp;
    }
    double* part_a = region;
    double* part_b = part_a + part_len;
    double* fac_a = part_b + (nspin == 2 ? part_len : 0);
    double* fac_b = fac_a + fac_len;
    double* eblk = fac_b + (nspin == 2 ? fac_len : 0);
    // the batch's partials and factors start at the region: the kernels index
    // them by each group's offset less the batch's first group's
    const long long part_base = first.part_off, pt_base = first.pt_off;
    for (int s = 0; s < nspin; s++) {
      const double* P = s == 0 ? rho_a : rho_b;
      if (d->lda)
        k_density_fp64<1><<<(unsigned)nd, 256, 0, st>>>(d->dens_tiles.p + dt0, d->groups.p, d->fn_glob.p, d->basis.p,
                                                          P, d->M, s == 0 ? part_a : part_b, part_base);
      else
        k_density_fp64<4><<<(unsigned)nd, 256, 0, st>>>(d->dens_tiles.p + dt0, d->groups.p, d->fn_glob.p, d->basis.p,
                                                          P, d->M, s == 0 ? part_a : part_b, part_base);
      LIO_CUDA(cudaGetLastError());
    }
    launch_functional(d->lda, d->open, (unsigned)nf, st, d->func_tiles.p + ft0, d->groups.p, d->pw.p, part_a,
                      d->open ? part_b : nullptr, kTile, d->iexch, fac_a, d->open ? fac_b : nullptr, eblk, part_base,
                      pt_base);
    LIO_CUDA(cudaGetLastError());
    k_sum_blocks<<<1, 1024, 0, st>>>(eblk, (int)nf, eparts + nbatch, 0);
    LIO_CUDA(cudaGetLastError());
    if (d->open)
      k_fock_fp64<2><<<(unsigned)nk, 256, 0, st>>>(d->fock_tiles.p + kt0, d->groups.p, d->fn_glob.p, d->basis.p,
                                                    fac_a, fac_b, d->M, fock_a, fock_b, pt_base);
    else
      k_fock_fp64<1><<<(unsigned)nk, 256, 0, st>>>(d->fock_tiles.p + kt0, d->groups.p, d->fn_glob.p, d->basis.p,
                                                    fac_a, nullptr, d->M, fock_a, nullptr, pt_base);
    LIO_CUDA(cudaGetLastError());
    dt0 += nd;
    ft0 += nf;
    kt0 += nk;
    nbatch++;
    g0 = g1;
  }
  k_sum_blocks<<<1, 1024, 0, st>>>(eparts, nbatch, energy, 0);
  LIO_CUDA(cudaGetLastError());
}

}  // namespace lio
