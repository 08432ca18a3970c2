// Tensor-core form of the density contraction (included by engine.cu inside its
// anonymous namespace; uses GroupDev, c_comp_l and the monomial helpers).
//
// G^a = A^a . D for the basis kinds a = F (LDA) or F, dF/dx, dF/dy, dF/dz (GGA),
// with D the group's dense density, computed with int8 tensor-core products
// (tcgen05 kind::i8, exact int32 accumulation in TMEM) on Ozaki-style slices:
//   A^a_pj = 2^(e_p) * sum_s a_s[p][j] 128^-(s+1),   |a_s| <= 64  (per point p)
//   D_ji   = 2^(f_i) * sum_t d_t[i][j] 128^-(t+1),   |d_t| <= 64  (per function i)
// and G_pi = 2^(e_p + f_i - 7(S+1)) * sum_l acc_l[p][i] 128^(S-1-l), where the
// level accumulator acc_l holds every slice pair s + t = l (pairs with
// s + t >= S are dropped). The level sum is formed exactly in int64 and
// converted to FP64 once. With S = 6 the dropped terms are ~2^-42 of
// max_j|A_pj| * max_j|D_ji| per term, far inside the 1e-7 / 1e-6 Ha tolerances.
//
// The row-dot epilogue needs F, dF and d2F at (p, i) in FP64; instead of
// re-reading ten cached values per (p, i) it rebuilds them from a per-shell
// radial cache (t, tg, th) and the point/atom coordinates (no exp), so the
// kernel's HBM traffic is dominated by the int8 slices.
#pragma once
#include "umma.cuh"

constexpr int kSlices = 6;       // Ozaki slices per operand
constexpr int kTcPoints = 128;   // UMMA M: points per tile
constexpr int kTcFuncs = 64;     // UMMA N: functions per tile (== kTile)
constexpr int kTcChunk = 64;     // K bytes (functions j) staged per step
constexpr uint32_t kTcTmemCols = 512;
constexpr size_t kTcSmemA = (size_t)kSlices * kTcPoints * kTcChunk;  // 48 KiB
constexpr size_t kTcSmemB = (size_t)kSlices * kTcFuncs * kTcChunk;   // 24 KiB

// exponent so that |x| * 2^-e <= 1/2 for every |x| <= amax
__device__ __forceinline__ int slice_exponent(double amax) { return amax > 0.0 ? ilogb(amax) + 2 : 0; }

// ---------------------------------------------------------------- A slices
// Per geometry: one thread per (group, point) and kind; reads the FP64 basis
// cache, writes the int8 slices in the K-major interleaved UMMA layout of each
// 128-point tile, and the per-point exponents.
template <int NA>
__global__ void k_slice_basis(const int2* __restrict__ tiles, const GroupDev* __restrict__ groups,
                              const double* __restrict__ basis, int8_t* __restrict__ aslices,
                              int16_t* __restrict__ aexp) {
  const int2 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int r = threadIdx.x;
  const int p = t.y * kTcPoints + r;
  const long long kstride = (long long)G.m * G.ldp;
  for (int a = 0; a < NA; a++) {
    const double* src = basis + G.bas_off + a * kstride + p;
    double amax = 0.0;
    for (int j = 0; j < G.m; j++) amax = fmax(amax, fabs(src[(long long)j * G.ldp]));
    const int e = slice_exponent(amax);
    aexp[G.aexp_off + (long long)a * G.ldp + p] = (int16_t)e;
    int8_t* dst = aslices + G.sl_off + ((long long)(t.y * NA + a) * kSlices) * kTcPoints * G.m32;
    for (int j = 0; j < G.m32; j++) {
      double x = j < G.m ? ldexp(src[(long long)j * G.ldp], -e) : 0.0;
      const uint32_t off = lio::umma::kmajor_offset(r, j, kTcPoints);
      for (int s = 0; s < kSlices; s++) {
        x *= 128.0;
        const double d = rint(x);
        x -= d;
        dst[(long long)s * kTcPoints * G.m32 + off] = (int8_t)d;
      }
    }
  }
}

// --------------------------------------------------------------- D slices
// Per solve and spin: one thread per (group, function i) of a 64-function tile;
// gathers column i of the group's density from the packed matrix (off-diagonal
// packed values halved), writes its slices and exponent.
__global__ void k_slice_density(const int2* __restrict__ tiles, const GroupDev* __restrict__ groups,
                                const int* __restrict__ fn_glob, const double* __restrict__ P, int M,
                                int8_t* __restrict__ dslices, int16_t* __restrict__ dexp) {
  const int2 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int r = threadIdx.x;  // row of the B tile
  const int i = t.y * kTcFuncs + r;
  const int* fg = fn_glob + G.fn_off;
  double amax = 0.0;
  const int gi = i < G.m ? fg[i] : 0;
  if (i < G.m)
    for (int j = 0; j < G.m; j++) {
      const int gj = fg[j];
      double v = P[packed_index(gi, gj, M)];
      if (gi != gj) v *= 0.5;
      amax = fmax(amax, fabs(v));
    }
  const int e = slice_exponent(amax);
  dexp[G.dexp_off + i] = (int16_t)e;
  int8_t* dst = dslices + G.ds_off + ((long long)t.y * kSlices) * kTcFuncs * G.m32;
  for (int j = 0; j < G.m32; j++) {
    double x = 0.0;
    if (i < G.m && j < G.m) {
      const int gj = fg[j];
      double v = P[packed_index(gi, gj, M)];
      if (gi != gj) v *= 0.5;
      x = ldexp(v, -e);
    }
    const uint32_t off = lio::umma::kmajor_offset(r, j, kTcFuncs);
    for (int s = 0; s < kSlices; s++) {
      x *= 128.0;
      const double d = rint(x);
      x -= d;
      dst[(long long)s * kTcFuncs * G.m32 + off] = (int8_t)d;
    }
  }
}

// ------------------------------------------------------- the fused kernel
struct TcFn {
  double ax, ay, az, scale;
  int sh, cp;
};

// basis value and derivatives of local function (f) at point r from the
// radial triplet (t, tg, th): the same closed forms as k_basis
__device__ __forceinline__ void rebuild(const TcFn& f, const double r[3], double t, double tg, double th, bool hess,
                                        double& F, double g[3], double h[6]) {
  const int* l = c_comp_l[f.cp];
  const double P = ipow(r[0], l[0]) * ipow(r[1], l[1]) * ipow(r[2], l[2]);
  double Pa[3];
  Pa[0] = dpow(r[0], l[0]) * ipow(r[1], l[1]) * ipow(r[2], l[2]);
  Pa[1] = ipow(r[0], l[0]) * dpow(r[1], l[1]) * ipow(r[2], l[2]);
  Pa[2] = ipow(r[0], l[0]) * ipow(r[1], l[1]) * dpow(r[2], l[2]);
  F = f.scale * P * t;
  for (int a = 0; a < 3; a++) g[a] = f.scale * (Pa[a] * t - 2.0 * r[a] * P * tg);
  if (!hess) return;
  const int ha[6] = {0, 1, 2, 0, 0, 1}, hb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const int a = ha[k], b = hb[k];
    double Pab;
    if (a == b) {
      Pab = (a == 0 ? d2pow(l[0]) * ipow(r[1], l[1]) * ipow(r[2], l[2])
                    : (a == 1 ? ipow(r[0], l[0]) * d2pow(l[1]) * ipow(r[2], l[2])
                              : ipow(r[0], l[0]) * ipow(r[1], l[1]) * d2pow(l[2])));
    } else {
      const int e0 = (a == 0 || b == 0), e1 = (a == 1 || b == 1), e2 = (a == 2 || b == 2);
      Pab = (e0 ? dpow(r[0], l[0]) : ipow(r[0], l[0])) * (e1 ? dpow(r[1], l[1]) : ipow(r[1], l[1])) *
            (e2 ? dpow(r[2], l[2]) : ipow(r[2], l[2]));
    }
    h[k] = f.scale * (Pab * t - 2.0 * (r[b] * Pa[a] + r[a] * Pa[b] + (a == b ? P : 0.0)) * tg + 4.0 * r[a] * r[b] * P * th);
  }
}

// Tile = (group, 128-point tile, 64-function tile); 128 threads = 4 warps, one
// TMEM lane (= one point) per thread. Per kind: stage 64-byte K chunks of all
// A and D slices in shared memory, one thread issues the slice-pair MMAs into
// the S level accumulators, then every thread combines its point's levels and
// accumulates the row-dot terms. Writes the same partial layout as
// k_density_fp64.
template <int NA>
__global__ void __launch_bounds__(128, 1)
    k_density_tc(const int4* __restrict__ tiles, const GroupDev* __restrict__ groups,
                 const int8_t* __restrict__ aslices, const int16_t* __restrict__ aexp,
                 const int8_t* __restrict__ dslices, const int16_t* __restrict__ dexp,
                 const double* __restrict__ radial, const double* __restrict__ px, const double* __restrict__ py,
                 const double* __restrict__ pz, const int* __restrict__ fn_sh, const int8_t* __restrict__ fn_cp,
                 const int* __restrict__ sf_glob, const int* __restrict__ nuc, const double* __restrict__ ax,
                 const double* __restrict__ ay, const double* __restrict__ az, double dnorm,
                 double* __restrict__ partial, int* __restrict__ err) {
  constexpr int NQ = NA == 1 ? 1 : kNQ;
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  uint8_t* sA = tc_smem;
  uint8_t* sB = tc_smem + kTcSmemA;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ TcFn fns[kTcFuncs];
  __shared__ int fexp[kTcFuncs];
  const int4 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int T = t.y, ft = t.z;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int p = T * kTcPoints + tid;
  if (warp == 0) lio::umma::tmem_alloc(&tmem_base, kTcTmemCols);
  if (tid == 0) lio::umma::mbar_init(&mbar, 1);
  if (tid < kTcFuncs) {
    const int i = ft * kTcFuncs + tid;
    TcFn f{0, 0, 0, 0, 0, 0};
    if (i < G.m) {
      f.sh = fn_sh[G.fn_off + i];
      const int code = fn_cp[G.fn_off + i];
      f.cp = code & 15;
      f.scale = (code & 16) ? dnorm : 1.0;
      const int atom = nuc[sf_glob[G.sf_off + f.sh]];
      f.ax = ax[atom];
      f.ay = ay[atom];
      f.az = az[atom];
    }
    fns[tid] = f;
    fexp[tid] = dexp[G.dexp_off + ft * kTcFuncs + tid];
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  lio::umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  const uint32_t lane_base = tbase + ((uint32_t)(warp * 32) << 16);
  const double rp[3] = {px[G.pt_off + p], py[G.pt_off + p], pz[G.pt_off + p]};
  double q[NQ];
#pragma unroll
  for (int k = 0; k < NQ; k++) q[k] = 0.0;
  const int nks = G.m32 / 32;       // 32-byte MMA K steps
  const int nch = (nks + 1) / 2;    // 64-byte chunks
  const uint32_t idesc = lio::umma::idesc_i8(kTcPoints, kTcFuncs);
  const uint32_t a_sm = lio::umma::smem_u32(sA), b_sm = lio::umma::smem_u32(sB);
  uint32_t phase = 0;
  bool ok = true;
  const double* rad = radial + G.rad_off;
  const long long rstride = (long long)G.nsimple * G.ldp;

  for (int a = 0; a < NA && ok; a++) {
    const int8_t* Ablk = aslices + G.sl_off + ((long long)(T * NA + a) * kSlices) * kTcPoints * G.m32;
    const int8_t* Bblk = dslices + G.ds_off + ((long long)ft * kSlices) * kTcFuncs * G.m32;
    for (int c = 0; c < nch && ok; c++) {
      const int halves = (2 * c + 1 < nks) ? 4 : 2;  // 16-byte K halves in this chunk
      // stage: A slice s bytes [c*4*16*128, +halves*16*128), B slice t bytes [c*4*16*64, ...)
      const int abytes = halves * 16 * kTcPoints, bbytes = halves * 16 * kTcFuncs;
      for (int s = 0; s < kSlices; s++) {
        const int4* srcA = reinterpret_cast<const int4*>(Ablk + (long long)s * kTcPoints * G.m32 + c * 4 * 16 * kTcPoints);
        int4* dstA = reinterpret_cast<int4*>(sA + s * kTcPoints * kTcChunk);
        for (int v = tid; v < abytes / 16; v += 128) dstA[v] = srcA[v];
        const int4* srcB = reinterpret_cast<const int4*>(Bblk + (long long)s * kTcFuncs * G.m32 + c * 4 * 16 * kTcFuncs);
        int4* dstB = reinterpret_cast<int4*>(sB + s * kTcFuncs * kTcChunk);
        for (int v = tid; v < bbytes / 16; v += 128) dstB[v] = srcB[v];
      }
      lio::umma::fence_proxy_async_smem();
      lio::umma::fence_before_sync();
      __syncthreads();
      lio::umma::fence_after_sync();
      if (tid == 0) {
        for (int kk = 0; kk < halves / 2; kk++) {
          for (int l = 0; l < kSlices; l++)
            for (int s = 0; s <= l; s++) {
              const int tt = l - s;
              const uint64_t ad =
                  lio::umma::smem_desc(a_sm + s * kTcPoints * kTcChunk + kk * 32 * kTcPoints, 16u * kTcPoints, 128u);
              const uint64_t bd =
                  lio::umma::smem_desc(b_sm + tt * kTcFuncs * kTcChunk + kk * 32 * kTcFuncs, 16u * kTcFuncs, 128u);
              const uint32_t acc = (c > 0 || kk > 0 || s > 0) ? 1u : 0u;
              lio::umma::mma_i8(tbase + (uint32_t)(l * kTcFuncs), ad, bd, idesc, acc);
            }
        }
        lio::umma::commit(&mbar);
      }
      ok = lio::umma::mbar_wait(&mbar, phase);
      phase ^= 1u;
      lio::umma::fence_after_sync();
      ok = __syncthreads_and(ok ? 1 : 0) != 0;
    }
    if (!ok) break;
    // epilogue for kind a: combine levels, rebuild basis values, row-dot
    const int ea = aexp[G.aexp_off + (long long)a * G.ldp + p];
    for (int cc = 0; cc < kTcFuncs; cc += 8) {
      int32_t lv[kSlices][8];
#pragma unroll
      for (int l = 0; l < kSlices; l++) lio::umma::tmem_ld8(lane_base + (uint32_t)(l * kTcFuncs + cc), lv[l]);
      lio::umma::tmem_wait_ld();
#pragma unroll
      for (int jj = 0; jj < 8; jj++) {
        const int il = cc + jj;
        const int i = ft * kTcFuncs + il;
        if (i >= G.m) continue;
        long long V = 0;
#pragma unroll
        for (int l = 0; l < kSlices; l++) V += (long long)lv[l][jj] * (1LL << (7 * (kSlices - 1 - l)));
        const double Gv = ldexp((double)V, ea + fexp[il] - 7 * (kSlices + 1));
        const TcFn f = fns[il];
        const double rr[3] = {rp[0] - f.ax, rp[1] - f.ay, rp[2] - f.az};
        const long long ro = (long long)f.sh * G.ldp + p;
        const double tv = rad[ro], tg = rad[rstride + ro], th = rad[2 * rstride + ro];
        double F, g[3], h[6];
        rebuild(f, rr, tv, tg, th, NA > 1 && a == 0, F, g, h);
        if (a == 0) {
          q[0] += F * Gv;
          if (NA > 1) {
            q[1 % NQ] += 2.0 * g[0] * Gv;
            q[2 % NQ] += 2.0 * g[1] * Gv;
            q[3 % NQ] += 2.0 * g[2] * Gv;
            q[4 % NQ] += 2.0 * h[0] * Gv;
            q[5 % NQ] += 2.0 * h[1] * Gv;
            q[6 % NQ] += 2.0 * h[2] * Gv;
            q[7 % NQ] += 2.0 * h[3] * Gv;
            q[8 % NQ] += 2.0 * h[4] * Gv;
            q[9 % NQ] += 2.0 * h[5] * Gv;
          }
        } else if (a == 1) {  // Gx: xx, xy (= gy.Gx), xz (= gz.Gx)
          q[4 % NQ] += 2.0 * g[0] * Gv;
          q[7 % NQ] += 2.0 * g[1] * Gv;
          q[8 % NQ] += 2.0 * g[2] * Gv;
        } else if (a == 2) {  // Gy: yy, yz (= gz.Gy)
          q[5 % NQ] += 2.0 * g[1] * Gv;
          q[9 % NQ] += 2.0 * g[2] * Gv;
        } else {  // Gz: zz
          q[6 % NQ] += 2.0 * g[2] * Gv;
        }
      }
    }
    // all TMEM reads of this kind must finish before the next kind's MMAs
    lio::umma::fence_before_sync();
    __syncthreads();
    lio::umma::fence_after_sync();
  }
  if (ok) {
    double* dst = partial + G.part_off;
#pragma unroll
    for (int k = 0; k < NQ; k++) dst[((long long)ft * NQ + k) * G.ldp + p] = q[k];
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) lio::umma::tmem_dealloc(tbase, kTcTmemCols);
}
