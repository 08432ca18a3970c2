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
constexpr int kTcFuncs = 16;     // UMMA N: functions per tile; all kinds x levels stay in TMEM
constexpr int kTcEpiWarps = 16;  // epilogue warps: kTcEpiWarps / 4 per TMEM lane quadrant
constexpr int kTcEpiCols = kTcFuncs / (kTcEpiWarps / 4);  // columns per epilogue warp
constexpr int kTcSliceA = 32 * kTcPoints;  // bytes of one A slice per 32-byte K step
constexpr int kTcSliceB = 32 * kTcFuncs;   // bytes of one B slice per K step
template <int NA>
struct TcCfg {
  static constexpr int kStageA = NA * kSlices * kTcSliceA;
  static constexpr int kStage = kStageA + kSlices * kTcSliceB;
  static constexpr size_t kSmem = 2 * (size_t)kStage;  // double-buffered K steps
  static constexpr uint32_t kCols = NA * kSlices * kTcFuncs;
  static constexpr uint32_t kTmem = kCols <= 128 ? 128 : (kCols <= 256 ? 256 : 512);
  static constexpr int kWarps = kTcEpiWarps + 2;  // epilogue warps, producer, MMA issuer
  static constexpr int kThreads = 32 * kWarps;
};

// exponent so that |x| * 2^-e <= 1/2 for every |x| <= amax
__device__ __forceinline__ int slice_exponent(double amax) { return amax > 0.0 ? ilogb(amax) + 2 : 0; }

// exact 2^k as a double (k within the normal range), else ldexp
__device__ __forceinline__ double pow2(int k) {
  return (k > -1022 && k < 1024) ? __longlong_as_double((long long)(k + 1023) << 52) : ldexp(1.0, k);
}

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
// Per solve and spin: one thread per (group, function i) of a kTcFuncs-function tile;
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
// basis value and derivatives of one Cartesian component x^LX y^LY z^LZ at
// displacement r from the radial triplet (t, tg, th); the closed forms of
// k_basis with every exponent a compile-time constant:
//   F = P t,  dF/da = P_a t - 2 r_a P tg,
//   d2F/da db = P_ab t - 2 (r_b P_a + r_a P_b + delta_ab P) tg + 4 r_a r_b P th
template <int L>
__device__ __forceinline__ double cpow(double x) { return L == 0 ? 1.0 : (L == 1 ? x : x * x); }
template <int L>
__device__ __forceinline__ double cdpow(double x) { return L == 0 ? 0.0 : (L == 1 ? 1.0 : 2.0 * x); }
template <int L>
__device__ __forceinline__ double cd2pow() { return L == 2 ? 2.0 : 0.0; }

template <int LX, int LY, int LZ, bool HESS>
__device__ __forceinline__ void rebuild_c(const double r[3], double t, double tg, double th, double sc, double& F,
                                          double g[3], double h[6]) {
  const double px = cpow<LX>(r[0]), py = cpow<LY>(r[1]), pz = cpow<LZ>(r[2]);
  const double dx = cdpow<LX>(r[0]), dy = cdpow<LY>(r[1]), dz = cdpow<LZ>(r[2]);
  const double P = px * py * pz;
  const double Pa[3] = {dx * py * pz, px * dy * pz, px * py * dz};
  const double st = sc * t, sv = sc * (-2.0 * tg), sw = sc * (4.0 * th);
  F = P * st;
  g[0] = Pa[0] * st + r[0] * P * sv;
  g[1] = Pa[1] * st + r[1] * P * sv;
  g[2] = Pa[2] * st + r[2] * P * sv;
  if (!HESS) return;
  const double Pxx = cd2pow<LX>() * py * pz, Pyy = px * cd2pow<LY>() * pz, Pzz = px * py * cd2pow<LZ>();
  const double Pxy = dx * dy * pz, Pxz = dx * py * dz, Pyz = px * dy * dz;
  const double wP = sw * P;
  h[0] = Pxx * st + (2.0 * r[0] * Pa[0] + P) * sv + r[0] * r[0] * wP;
  h[1] = Pyy * st + (2.0 * r[1] * Pa[1] + P) * sv + r[1] * r[1] * wP;
  h[2] = Pzz * st + (2.0 * r[2] * Pa[2] + P) * sv + r[2] * r[2] * wP;
  h[3] = Pxy * st + (r[1] * Pa[0] + r[0] * Pa[1]) * sv + r[0] * r[1] * wP;
  h[4] = Pxz * st + (r[2] * Pa[0] + r[0] * Pa[2]) * sv + r[0] * r[2] * wP;
  h[5] = Pyz * st + (r[2] * Pa[1] + r[1] * Pa[2]) * sv + r[1] * r[2] * wP;
}

// dispatch on the component code (0: s; 1-3: p x,y,z; 4-9: d xx,xy,yy,xz,yz,zz),
// which is the same for every lane of a warp
template <bool HESS>
__device__ __forceinline__ void rebuild_cp(int cp, const double r[3], double t, double tg, double th, double sc,
                                           double& F, double g[3], double h[6]) {
  switch (cp) {
    case 0: rebuild_c<0, 0, 0, HESS>(r, t, tg, th, sc, F, g, h); break;
    case 1: rebuild_c<1, 0, 0, HESS>(r, t, tg, th, sc, F, g, h); break;
    case 2: rebuild_c<0, 1, 0, HESS>(r, t, tg, th, sc, F, g, h); break;
    case 3: rebuild_c<0, 0, 1, HESS>(r, t, tg, th, sc, F, g, h); break;
    case 4: rebuild_c<2, 0, 0, HESS>(r, t, tg, th, sc, F, g, h); break;
    case 5: rebuild_c<1, 1, 0, HESS>(r, t, tg, th, sc, F, g, h); break;
    case 6: rebuild_c<0, 2, 0, HESS>(r, t, tg, th, sc, F, g, h); break;
    case 7: rebuild_c<1, 0, 1, HESS>(r, t, tg, th, sc, F, g, h); break;
    case 8: rebuild_c<0, 1, 1, HESS>(r, t, tg, th, sc, F, g, h); break;
    default: rebuild_c<0, 0, 2, HESS>(r, t, tg, th, sc, F, g, h); break;
  }
}

template <int N>
__device__ __forceinline__ void tmem_ld_cols(uint32_t taddr, int32_t (&v)[N]) {
  if constexpr (N == 8) {
    lio::umma::tmem_ld8(taddr, v);
  } else {
    lio::umma::tmem_ld4(taddr, *reinterpret_cast<int32_t(*)[4]>(v));
  }
}

// CTA = (group, 128-point tile), warp-specialised:
//   warps 0..kTcEpiWarps-1  epilogue: TMEM lane quadrant warp % 4 (one lane =
//                one point), columns kTcEpiCols * (warp / 4) .. of each tile;
//   next warp    producer: 1-D bulk copies of the A slices (all kinds) and the
//                D slices of each 32-byte K step into one of two stages;
//   last warp    MMA issuer: every kind's slice pairs into the NA x S level
//                accumulators, which stay resident in TMEM for a whole
//                16-function tile.
// mbarriers: full[s] (bytes landed), empty[s] (the stage's MMAs are done),
// tfull (a tile's accumulators are complete), tempty (the epilogue has read
// them). The epilogue hands TMEM back right after combining the levels, so the
// next tile's MMAs overlap its FP64 row-dot work. The four column groups of a
// point are summed through shared memory at the end and written once (one
// partial per point). Every wait is bounded.
template <int NA>
__global__ void __launch_bounds__(TcCfg<NA>::kThreads, 1)
    k_density_tc(const int2* __restrict__ tiles, const GroupDev* __restrict__ groups,
                 const int8_t* __restrict__ aslices, const int16_t* __restrict__ aexp,
                 const int8_t* __restrict__ dslices, const int16_t* __restrict__ dexp,
                 const double* __restrict__ radial, const double* __restrict__ px, const double* __restrict__ py,
                 const double* __restrict__ pz, const int* __restrict__ fn_sh, const int8_t* __restrict__ fn_cp,
                 const int* __restrict__ fn_atom, const double* __restrict__ ax, const double* __restrict__ ay,
                 const double* __restrict__ az, double dnorm, double* __restrict__ partial, int* __restrict__ err) {
  using Cfg = TcCfg<NA>;
  constexpr int NQ = NA == 1 ? 1 : kNQ;
  constexpr int kGroups = kTcEpiWarps / 4;  // column groups per lane quadrant
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ uint64_t full[2], empty[2], tfull, tempty;
  __shared__ uint32_t tmem_base;
  __shared__ int fail;
  const int2 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int T = t.y;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nks = G.m32 / 32;
  const int nft = (G.m + kTcFuncs - 1) / kTcFuncs;
  const int total = nft * nks;
  if (warp == 0) lio::umma::tmem_alloc(&tmem_base, Cfg::kTmem);
  if (tid == 0) {
    lio::umma::mbar_init(&full[0], 1);
    lio::umma::mbar_init(&full[1], 1);
    lio::umma::mbar_init(&empty[0], 1);
    lio::umma::mbar_init(&empty[1], 1);
    lio::umma::mbar_init(&tfull, 1);
    lio::umma::mbar_init(&tempty, kTcEpiWarps);
    lio::umma::fence_mbar_init();
    fail = 0;
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  lio::umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  double q[NQ];
#pragma unroll
  for (int k = 0; k < NQ; k++) q[k] = 0.0;
  const int quad = warp & 3, colg = warp >> 2;
  const int row = quad * 32 + lane;
  const int p = T * kTcPoints + row;

  if (warp == kTcEpiWarps) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      const int8_t* Abase = aslices + G.sl_off + (long long)T * NA * kSlices * kTcPoints * G.m32;
      const int8_t* Bbase = dslices + G.ds_off;
      for (int st = 0; st < total; st++) {
        const int buf = st & 1, use = st >> 1;
        if (use > 0 && !lio::umma::mbar_wait(&empty[buf], (use - 1) & 1)) {
          fail = 1;
          break;
        }
        const int ft = st / nks, kk = st - ft * nks;
        uint8_t* stage = tc_smem + buf * Cfg::kStage;
        lio::umma::mbar_expect_tx(&full[buf], (uint32_t)Cfg::kStage);
        for (int piece = 0; piece < NA * kSlices; piece++)
          lio::umma::bulk_copy_g2s(stage + piece * kTcSliceA,
                                   Abase + (long long)piece * kTcPoints * G.m32 + kk * kTcSliceA, kTcSliceA,
                                   &full[buf]);
        for (int s = 0; s < kSlices; s++)
          lio::umma::bulk_copy_g2s(stage + Cfg::kStageA + s * kTcSliceB,
                                   Bbase + ((long long)ft * kSlices + s) * kTcFuncs * G.m32 + kk * kTcSliceB,
                                   kTcSliceB, &full[buf]);
      }
    }
  } else if (warp == kTcEpiWarps + 1) {
    // ------------------------------------------- MMA issuer (all kinds)
    if (lane == 0) {
      const uint32_t idesc = lio::umma::idesc_i8(kTcPoints, kTcFuncs);
      const uint32_t smem0 = lio::umma::smem_u32(tc_smem);
      for (int st = 0; st < total; st++) {
        const int buf = st & 1, use = st >> 1;
        const int ft = st / nks, kk = st - ft * nks;
        if (kk == 0 && ft > 0) {
          if (!lio::umma::mbar_wait(&tempty, (ft - 1) & 1)) {
            fail = 1;
            break;
          }
          lio::umma::fence_after_sync();
        }
        if (!lio::umma::mbar_wait(&full[buf], use & 1)) {
          fail = 1;
          break;
        }
        lio::umma::fence_after_sync();
        // the descriptor start-address field advances by (byte offset >> 4)
        const uint64_t ad0 = lio::umma::smem_desc(smem0 + buf * Cfg::kStage, 16u * kTcPoints, 128u);
        const uint64_t bd0 = lio::umma::smem_desc(smem0 + buf * Cfg::kStage + Cfg::kStageA, 16u * kTcFuncs, 128u);
        const uint32_t keep = kk > 0 ? 1u : 0u;
#pragma unroll
        for (int a = 0; a < NA; a++)
#pragma unroll
          for (int l = 0; l < kSlices; l++)
#pragma unroll
            for (int s = 0; s <= l; s++)
              lio::umma::mma_i8(tbase + (uint32_t)((a * kSlices + l) * kTcFuncs),
                                ad0 + (uint64_t)(((a * kSlices + s) * kTcSliceA) >> 4),
                                bd0 + (uint64_t)(((l - s) * kTcSliceB) >> 4), idesc, s > 0 ? 1u : keep);
        lio::umma::commit(&empty[buf]);
        if (kk == nks - 1) lio::umma::commit(&tfull);
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const uint32_t lane_base = tbase + ((uint32_t)(quad * 32) << 16);
    double sp[NA];  // 2^(point exponent - 7(S+1)) per kind
#pragma unroll
    for (int a = 0; a < NA; a++) sp[a] = pow2(aexp[G.aexp_off + (long long)a * G.ldp + p] - 7 * (kSlices + 1));
    const double rp[3] = {px[G.pt_off + p], py[G.pt_off + p], pz[G.pt_off + p]};
    const double* rad = radial + G.rad_off;
    const long long rstride = (long long)G.nsimple * G.ldp;
    for (int ft = 0; ft < nft; ft++) {
      const int c0 = ft * kTcFuncs + colg * kTcEpiCols;  // first function of this warp's columns
      if (!lio::umma::mbar_wait(&tfull, ft & 1)) {
        fail = 1;
        break;
      }
      lio::umma::fence_after_sync();
      double Gv[NA][kTcEpiCols];
#pragma unroll
      for (int a = 0; a < NA; a++) {
        int32_t lv[kSlices][kTcEpiCols];
#pragma unroll
        for (int l = 0; l < kSlices; l++)
          tmem_ld_cols<kTcEpiCols>(lane_base + (uint32_t)((a * kSlices + l) * kTcFuncs + colg * kTcEpiCols), lv[l]);
        lio::umma::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < kTcEpiCols; c++) {
          // levels pairwise in int32 (|acc| < 2^23, so 128 acc_l + acc_l+1 fits), then exactly in int64
          long long V = 0;
#pragma unroll
          for (int l = 0; l < kSlices; l += 2) V = V * (1LL << 14) + (long long)(lv[l][c] * 128 + lv[l + 1][c]);
          Gv[a][c] = (double)V * sp[a];
        }
      }
      // accumulators read: hand TMEM back to the MMA issuer
      lio::umma::fence_before_sync();
      __syncwarp();
      if (lane == 0) lio::umma::mbar_arrive(&tempty);
#pragma unroll 1
      for (int c = 0; c < kTcEpiCols; c++) {
        const int i = c0 + c;
        if (i >= G.m) break;
        const int sh = fn_sh[G.fn_off + i];
        const int code = fn_cp[G.fn_off + i];
        const double sc = (code & 16) ? dnorm : 1.0;
        const int atom = fn_atom[G.fn_off + i];
        const double si = pow2(dexp[G.dexp_off + i]);
        const double rr[3] = {rp[0] - ax[atom], rp[1] - ay[atom], rp[2] - az[atom]};
        const long long ro = (long long)sh * G.ldp + p;
        const double tv = rad[ro], tg = rad[rstride + ro], th = rad[2 * rstride + ro];
        double F, g[3], h[6];
        rebuild_cp<(NA > 1)>(code & 15, rr, tv, tg, th, sc, F, g, h);
        double gg[4];
#pragma unroll
        for (int a = 0; a < 4; a++) gg[a] = Gv[a % NA][c] * si;
        q[0] += F * gg[0];
        if (NA > 1) {
          const double g0 = gg[0];
          q[1 % NQ] += 2.0 * g[0] * g0;
          q[2 % NQ] += 2.0 * g[1] * g0;
          q[3 % NQ] += 2.0 * g[2] * g0;
          q[4 % NQ] += 2.0 * (h[0] * g0 + g[0] * gg[1]);
          q[5 % NQ] += 2.0 * (h[1] * g0 + g[1] * gg[2]);
          q[6 % NQ] += 2.0 * (h[2] * g0 + g[2] * gg[3]);
          q[7 % NQ] += 2.0 * (h[3] * g0 + g[1] * gg[1]);  // xy: gy . Gx (= gx . Gy by symmetry of D)
          q[8 % NQ] += 2.0 * (h[4] * g0 + g[2] * gg[1]);  // xz: gz . Gx
          q[9 % NQ] += 2.0 * (h[5] * g0 + g[2] * gg[2]);  // yz: gz . Gy
        }
      }
    }
  }
  __syncthreads();  // every role done; all copies and MMAs have completed
  const bool ok = fail == 0;
  double* red = reinterpret_cast<double*>(tc_smem);  // [column group 1..][point][NQ]
  if (ok && warp < kTcEpiWarps && colg > 0) {
#pragma unroll
    for (int k = 0; k < NQ; k++) red[((colg - 1) * kTcPoints + row) * NQ + k] = q[k];
  }
  __syncthreads();
  if (ok && warp < kTcEpiWarps && colg == 0) {
    double* dst = partial + G.part_off;
#pragma unroll
    for (int k = 0; k < NQ; k++) {
      double v = q[k];
#pragma unroll
      for (int gi = 1; gi < kGroups; gi++) v += red[((gi - 1) * kTcPoints + row) * NQ + k];
      dst[(long long)k * G.ldp + p] = v;
    }
  } else if (!ok && tid == 0) {
    atomicExch(err, 1);
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) lio::umma::tmem_dealloc(tbase, Cfg::kTmem);
}
