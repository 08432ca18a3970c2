// Tensor-core form of the density contraction (included by engine.cu inside its
// anonymous namespace; uses GroupDev and packed_index).
//
// G^a = A^a . D for the basis kinds a = F (LDA) or F, dF/dx, dF/dy, dF/dz (GGA),
// with D the group's dense density, computed with int8 tensor-core products
// (tcgen05 kind::i8, exact int32 accumulation in TMEM) on Ozaki-style slices:
//   A^a_pj = 2^(e_p) * sum_s a_s[p][j] 128^-(s+1),   |a_s| <= 64  (per point p)
//   D_ji   = 2^(f_T) * sum_t d_t[i][j] 128^-(t+1),   |d_t| <= 64  (per 32-function tile T of i)
// and G_pi = 2^(e_p + f_T - 7(S+1)) * sum_l acc_l[p][i] 128^(S-1-l), where the
// level accumulator acc_l holds every slice pair s + t = l (pairs with
// s + t >= S are dropped). With S = 6 the dropped terms are ~2^-42 of
// max_j|A_pj| * max_(j, i in T)|D_ji| per term, far inside the 1e-7 / 1e-6 Ha
// absolute tolerances. One exponent per tile lets the epilogue scale a whole
// row dot once instead of every G_pi.
//
// Slice pairs in few, wide MMAs: the S slices of a 32-function D tile are
// stacked along N ("tall" B operand, row t * 32 + i holds d_t[i]). For A slice s
// one MMA with N = (S - s) * 32 multiplies a_s by d_0 .. d_(S-1-s) (a prefix of
// the tall operand) into TMEM columns starting at level s, so product (s, t)
// lands on level s + t: S MMAs per K step and kind instead of S(S+1)/2 narrow
// ones (an MMA costs about the same for every N up to 64 on this part).
//
// The row-dot epilogue needs F, dF and d2F at (p, i) in FP64. They come from a
// blocked copy of the basis cache (per 128-point tile, 32-function tile and
// kind one contiguous 32 KB chunk) that a dedicated warp streams into a
// shared-memory ring with bulk copies, so the epilogue does no global loads.
#pragma once
#include "umma.cuh"

constexpr int kSlices = 6;       // Ozaki slices per operand
constexpr int kTcPoints = 128;   // UMMA M: points per tile
constexpr int kTcFuncs = 32;     // functions per density tile (output columns per level)
constexpr int kTcTall = kSlices * kTcFuncs;  // rows of the stacked D operand
constexpr int kTcEpiWarps = 8;   // two per TMEM lane quadrant
constexpr int kTcCpw = kTcFuncs / 2;         // columns per epilogue warp
constexpr int kTcSliceA = 32 * kTcPoints;    // bytes of one A slice per 32-byte K step
constexpr int kTcStepA = kSlices * kTcSliceA;  // one kind's A slices per K step (contiguous)
constexpr int kTcStepD = 32 * kTcTall;         // one spin's stacked D slices per K step (contiguous)
constexpr int kTcChunk = kTcFuncs * kTcPoints;  // doubles of one blocked basis chunk (kind, 32 functions)

// KP = kinds per unit: all NS x KP x S x 32 level columns of a unit fit in 384
// TMEM columns. Open shell: one kind per unit (F, x, y, z); closed shell GGA:
// {F, dF/dx} then {dF/dy, dF/dz}; LDA: {F}.
template <bool GGA, int NS>
struct TcCfg {
  static constexpr int KP = (GGA && NS == 1) ? 2 : 1;
  static constexpr int NA = GGA ? 4 : 1;   // kinds of the contraction
  static constexpr int NK = GGA ? 10 : 1;  // kinds of the FP64 basis (F; dF; d2F)
  static constexpr int NP = NA / KP;       // units per function tile
  static constexpr int NQ = GGA ? 10 : 1;
  static constexpr int kStageA = KP * kTcStepA;
  static constexpr int kStage = kStageA + NS * kTcStepD;
  static constexpr uint32_t kCols = NS * KP * kSlices * kTcFuncs;
  static constexpr uint32_t kTmem = kCols <= 256 ? 256 : 512;
  // epilogue warps, operand producer, MMA issuer, basis producer
  static constexpr int kWarps = kTcEpiWarps + 3;
  static constexpr int kThreads = 32 * kWarps;
  static constexpr int kProd = kTcEpiWarps, kMma = kTcEpiWarps + 1, kBasisProd = kTcEpiWarps + 2;
  // dynamic shared memory: operand ring | basis ring | column-group reduction | function table
  static constexpr int kStages = 2;
  static constexpr int kBStages = 3;
  static constexpr size_t kRing = (size_t)kStages * kStage;
  static constexpr size_t kBRing = kRing;
  static constexpr size_t kRed = kBRing + (size_t)kBStages * kTcChunk * 8;
  static constexpr size_t kRedBytes = (size_t)NS * kTcPoints * NQ * 8;  // [spin][point][NQ] FP64
  static constexpr size_t kTab = kRed + kRedBytes;
  static constexpr size_t kTabEntry = NS * 8;  // 2^f_i per spin
  static size_t smem(int cap) { return kTab + (size_t)cap * kTabEntry; }
};

// exponent so that |x| * 2^-e <= 1/2 for every |x| <= amax
__device__ __forceinline__ int slice_exponent(double amax) { return amax > 0.0 ? ilogb(amax) + 2 : 0; }

// exact 2^k as a double (k within the normal range), else ldexp
__device__ __forceinline__ double pow2(int k) {
  return (k > -1022 && k < 1024) ? __longlong_as_double((long long)(k + 1023) << 52) : ldexp(1.0, k);
}

// The S = 6 base-128 digits of x (|x| < 1/2), all from one rounding on the
// FP64 adder: t = 2^52 + B + x 2^42 with B = 64 (128^6 - 1) / 127 (even) rounds
// x 2^42 to the nearest integer N, ties to even, and the low mantissa bits of
// t hold M = N + B >= 0. The base-128 digits m_k of M less 64 are balanced
// digits of N (|m_k - 64| <= 64), so
//   x = sum_s (m_(5-s) - 64) 128^-(s+1) + r,  |r| <= 2^-43,
// with two FP64 operations per value instead of three per digit for a
// digit-by-digit extraction. `s42` is 2^42 times the row's power-of-two scale
// (digit_scale). Returns t's two 32-bit halves (M = bits 0..42).
__device__ __forceinline__ void digits_m(double x, double s42, uint32_t& lo, uint32_t& hi) {
  const double t = fma(x, s42, 4505815965769792.0);  // 2^52 + B
  lo = (uint32_t)__double2loint(t);
  hi = (uint32_t)__double2hiint(t);
}
// `s42` for a row with exponent e: 2^(42 - e), or 0 (every digit zero) for a
// row whose values are all below 2^-981, where 2^(42 - e) would leave the
// double range; the dropped values are far below any tolerance
__device__ __forceinline__ double digit_scale(int e) { return e > -980 ? pow2(42 - e) : 0.0; }

// m_(5-s), the field of slice s (0 = most significant), in the low byte; for
// s >= 1 bit 7 of that byte belongs to the next field and is masked by
// pack_digits. t's exponent bits (from bit 20 of hi) never reach a low byte.
__device__ __forceinline__ uint32_t digit_field(uint32_t lo, uint32_t hi, int s) {
  switch (s) {
    case 0: return hi >> 3;                        // bits 35..42 (m_5 <= 128)
    case 1: return __funnelshift_r(lo, hi, 28);    // bits 28..34
    case 2: return lo >> 21;
    case 3: return lo >> 14;
    case 4: return lo >> 7;
    default: return lo;
  }
}
// four fields (low bytes, first point lowest) -> four int8 digits m - 64,
// byte-wise without carries between bytes; slice 0 keeps its bit 7 (m_5 = 128
// gives digit 64)
__device__ __forceinline__ uint32_t pack_digits(uint32_t f0, uint32_t f1, uint32_t f2, uint32_t f3, bool top) {
  const uint32_t w = __byte_perm(__byte_perm(f0, f1, 0x0040), __byte_perm(f2, f3, 0x0040), 0x5410);
  const uint32_t low = (w & 0x7F7F7F7Fu) + 0x40404040u;
  return top ? low ^ ((w ^ 0xC0C0C0C0u) & 0x80808080u) : low ^ 0x80808080u;
}

// ---------------------------------------------------------------- A slices
// Per geometry: one thread per (group, point) and kind; reads the blocked FP64
// basis (NK kinds per block), writes the per-point exponent and the int8
// slices. Layout per 128-point tile T, kind a and 32-function K step kk: the S
// slices one after the other (kTcStepA bytes, one bulk copy), each in the
// K-major interleaved UMMA layout of a 128-row x 32-byte block.
template <int NA>
__global__ void k_slice_basis(const int2* __restrict__ tiles, const GroupDev* __restrict__ groups,
                              const double* __restrict__ bblk, int NK, int8_t* __restrict__ aslices,
                              int16_t* __restrict__ aexp) {
  const int2 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int r = threadIdx.x;
  const int p = t.y * kTcPoints + r;
  const int nks = G.m32 / 32;
  // value (kind a, function j) of this point
  auto val = [&](int a, int j) {
    return bblk[G.bb_off + ((long long)(t.y * G.nftc + (j >> 5)) * NK + a) * kTcChunk + (j & 31) * kTcPoints + r];
  };
  for (int a = 0; a < NA; a++) {
    double amax = 0.0;
    for (int j = 0; j < G.m; j++) amax = fmax(amax, fabs(val(a, j)));
    const int e = slice_exponent(amax);
    const double s42 = digit_scale(e);
    aexp[G.aexp_off + (long long)a * G.ldp + p] = (int16_t)e;
    int8_t* dst = aslices + G.sl_off + (long long)(t.y * NA + a) * nks * kTcStepA;
    // 16 consecutive functions at a time: per slice their 16 digits are one
    // contiguous 16-byte row segment of the K-major block, one store
    for (int j0 = 0; j0 < G.m32; j0 += 16) {
      uint32_t lo[16], hi[16];
#pragma unroll
      for (int k = 0; k < 16; k++) digits_m(j0 + k < G.m ? val(a, j0 + k) : 0.0, s42, lo[k], hi[k]);
      int8_t* blk = dst + (j0 >> 5) * kTcStepA + lio::umma::kmajor_offset(r, j0 & 31, kTcPoints);
#pragma unroll
      for (int s = 0; s < kSlices; s++) {
        uint32_t w[4];
#pragma unroll
        for (int k4 = 0; k4 < 4; k4++)
          w[k4] = pack_digits(digit_field(lo[4 * k4], hi[4 * k4], s), digit_field(lo[4 * k4 + 1], hi[4 * k4 + 1], s),
                              digit_field(lo[4 * k4 + 2], hi[4 * k4 + 2], s),
                              digit_field(lo[4 * k4 + 3], hi[4 * k4 + 3], s), s == 0);
        *reinterpret_cast<uint4*>(blk + s * kTcSliceA) = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
  }
}

// --------------------------------------------------------------- D slices
// Per solve and spin: one thread per (group, function i) of a 32-function tile
// (one warp per tile); gathers column i of the group's density from the packed
// matrix (off-diagonal packed values halved), writes the tile's exponent (one
// per 32 columns, from the largest |D_ji| of the tile, stored for each of its
// functions) and its S slices into the stacked operand: per tile and
// 32-function K step kk a 192-row x 32-byte block (kTcStepD bytes, one bulk
// copy) whose row t * 32 + i holds d_t[i].
__global__ void k_slice_density(const int2* __restrict__ tiles, const GroupDev* __restrict__ groups,
                                const int* __restrict__ fn_glob, const double* __restrict__ P, int M,
                                int8_t* __restrict__ dslices, int16_t* __restrict__ dexp) {
  const int2 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int r = threadIdx.x;  // function within the tile
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
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  const int e = slice_exponent(amax);
  const double s42 = digit_scale(e);
  dexp[G.dexp_off + i] = (int16_t)e;
  const int nks = G.m32 / 32;
  int8_t* dst = dslices + G.ds_off + (long long)t.y * nks * kTcStepD;
  // 16 consecutive functions j at a time: per slice one 16-byte row segment
  for (int j0 = 0; j0 < G.m32; j0 += 16) {
    uint32_t lo[16], hi[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
      const int j = j0 + k;
      double v = 0.0;
      if (i < G.m && j < G.m) {
        const int gj = fg[j];
        v = P[packed_index(gi, gj, M)];
        if (gi != gj) v *= 0.5;
      }
      digits_m(v, s42, lo[k], hi[k]);
    }
    int8_t* blk = dst + (j0 >> 5) * kTcStepD;
#pragma unroll
    for (int s = 0; s < kSlices; s++) {
      uint32_t w[4];
#pragma unroll
      for (int k4 = 0; k4 < 4; k4++)
        w[k4] = pack_digits(digit_field(lo[4 * k4], hi[4 * k4], s), digit_field(lo[4 * k4 + 1], hi[4 * k4 + 1], s),
                            digit_field(lo[4 * k4 + 2], hi[4 * k4 + 2], s),
                            digit_field(lo[4 * k4 + 3], hi[4 * k4 + 3], s), s == 0);
      *reinterpret_cast<uint4*>(blk + lio::umma::kmajor_offset(s * kTcFuncs + r, j0 & 31, kTcTall)) =
          make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// ------------------------------------------------------- the fused kernel
// K (padded functions) up to which two adjacent levels combine exactly in
// int32: |acc_l| <= (l + 1) * 64 * 64 * K, so |128 acc_4 + acc_5| < 2^31 for K < 813
constexpr int kTcNarrowK = 768;

// sum_l acc_l 128^(S-1-l) of column c in FP64: level pairs in int32 (narrow)
// or each level converted (wide), then combined with one rounding, 2^-53 of
// the leading term and far below the dropped slice pairs
template <int W>
__device__ __forceinline__ double level_sum(const int32_t (&lv)[kSlices][W], int c, bool narrow) {
  double v0, v1, v2;
  if (narrow) {
    v0 = (double)(lv[0][c] * 128 + lv[1][c]);
    v1 = (double)(lv[2][c] * 128 + lv[3][c]);
    v2 = (double)(lv[4][c] * 128 + lv[5][c]);
  } else {
    v0 = fma((double)lv[0][c], 128.0, (double)lv[1][c]);
    v1 = fma((double)lv[2][c], 128.0, (double)lv[3][c]);
    v2 = fma((double)lv[4][c], 128.0, (double)lv[5][c]);
  }
  return fma(fma(v0, 16384.0, v1), 16384.0, v2);
}

// named barrier over the epilogue warps only; returns the OR of `pred` over them
__device__ __forceinline__ bool epi_sync_or(bool pred) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(out)
      : "r"((uint32_t)pred), "n"(kTcEpiWarps * 32)
      : "memory");
  return out != 0;
}

// Whether a later unit of the same function tile reads chunk k again (the dF/dy,
// dF/dz chunks after the F or x unit, dF/dx after F when x is a unit of its own):
// those are kept in L2, last uses are evicted first.
__device__ __forceinline__ bool chunk_reused(int first, int k, int KP) {
  if (k < 1 || k > 3) return false;
  const int next = first + KP;  // first kind of the next unit
  return next <= 3 && k >= next;
}

// FP64 basis kinds whose chunks a unit with first contraction kind `first`
// consumes, in order: F unit: all NK; x: dF/dx..dF/dz; y: dF/dy, dF/dz; z: dF/dz.
__host__ __device__ __forceinline__ int unit_klo(int first) { return first == 0 ? 0 : first; }
__host__ __device__ __forceinline__ int unit_khi(int first, int NK) { return first == 0 ? NK - 1 : 3; }

// Adds the row dots of basis-kind chunk k, d[sp][kp] = sum_i v_ki G^(kp)_i over
// this warp's columns, to the point's q = (rho; grad rho; d2rho xx, yy, zz, xy,
// xz, yz) per spin:
//   unit F : k = F: rho += d;  k = dF_a: grad_a += 2 d;  k = d2F_ab: d2_ab += 2 d
//            with KP = 2 also G^x: xx += 2 d(Fx), xy += 2 d(Fy), xz += 2 d(Fz)
//   unit x : xx += 2 d(Fx), xy += 2 d(Fy), xz += 2 d(Fz)   (Fy Gx = Fx Gy: D is symmetric)
//   unit y : yy += 2 d(Fy), yz += 2 d(Fz)   (with KP = 2 also zz += 2 d(Fz) of G^z)
//   unit z : zz += 2 d(Fz)
template <bool GGA, int NS, int NQ, int KP>
__device__ __forceinline__ void apply_chunk(int first, int k, const double (&d)[NS][KP], double (&q)[NS][NQ]) {
#pragma unroll
  for (int sp = 0; sp < NS; sp++) {
    if (!GGA) {
      q[sp][0] += d[sp][0];
      continue;
    }
    const double d0 = 2.0 * d[sp][0], d1 = 2.0 * d[sp][KP - 1];
    if (first == 0) {
      // kinds F, dF/dx, dF/dy, dF/dz, d2F xx .. yz map onto q[0 .. 9] in order
      switch (k) {
        case 0: q[sp][0] += d[sp][0]; break;
        case 1: q[sp][1 % NQ] += d0; if (KP == 2) q[sp][4 % NQ] += d1; break;
        case 2: q[sp][2 % NQ] += d0; if (KP == 2) q[sp][7 % NQ] += d1; break;
        case 3: q[sp][3 % NQ] += d0; if (KP == 2) q[sp][8 % NQ] += d1; break;
        case 4: q[sp][4 % NQ] += d0; break;
        case 5: q[sp][5 % NQ] += d0; break;
        case 6: q[sp][6 % NQ] += d0; break;
        case 7: q[sp][7 % NQ] += d0; break;
        case 8: q[sp][8 % NQ] += d0; break;
        default: q[sp][9 % NQ] += d0; break;
      }
    } else if (first == 1) {
      if (k == 1) q[sp][4 % NQ] += d0;
      else if (k == 2) q[sp][7 % NQ] += d0;
      else q[sp][8 % NQ] += d0;
    } else if (first == 2) {
      if (k == 2) {
        q[sp][5 % NQ] += d0;
      } else {
        q[sp][9 % NQ] += d0;
        if (KP == 2) q[sp][6 % NQ] += d1;
      }
    } else {
      q[sp][6 % NQ] += d0;
    }
  }
}

// CTA = one per SM, persistent over the 128-point tiles (all groups, largest
// function count first, tile w handled by CTA w mod gridDim.x); both spins
// (NS = 2) or one. A unit is (tile, 32-function tile, KP contraction kinds).
// Warp roles:
//   warps 0..7  epilogue: TMEM lane quadrant warp % 4 (one lane = one point),
//               columns 16 * (warp / 4) .. of the function tile;
//   warp 8      operand producer: per (unit, 32-function K step) one stage with
//               the unit's A slices (KP x kTcStepA) and every spin's stacked D
//               slices (kTcStepD), one bulk copy each;
//   warp 9      MMA issuer: per stage NS x KP x S MMAs into the unit's
//               NS x KP x S x 32 level columns in TMEM;
//   warp 10     basis producer: per unit the FP64 basis chunks its row dots
//               need (unit_klo .. unit_khi), one 32 KB bulk copy each, into a
//               three-slot ring.
// The epilogue reads the unit's levels (tfull), forms G in FP64 in registers,
// hands TMEM back (tempty) so the next unit's MMAs overlap its row dots, and
// consumes the basis chunks from shared memory. Every wait is bounded; a
// timeout sets `fail`, which the other roles poll, and the kernel drains its
// copies and MMAs before it frees TMEM and reports the error.
template <bool GGA, int NS>
__global__ void __launch_bounds__(TcCfg<GGA, NS>::kThreads, 1)
    k_density_tc(const int2* __restrict__ tiles, int ntiles, const GroupDev* __restrict__ groups,
                 const int8_t* __restrict__ aslices, const int16_t* __restrict__ aexp,
                 const int8_t* __restrict__ dsl_a, const int16_t* __restrict__ dexp_a,
                 const int8_t* __restrict__ dsl_b, const int16_t* __restrict__ dexp_b,
                 const double* __restrict__ bblk, int fcap, double* __restrict__ part_a,
                 double* __restrict__ part_b, int* __restrict__ err) {
  using Cfg = TcCfg<GGA, NS>;
  constexpr int KP = Cfg::KP, NP = Cfg::NP, NA = Cfg::NA, NK = Cfg::NK, NQ = Cfg::NQ, CPW = kTcCpw;
  constexpr int kStages = Cfg::kStages, kBStages = Cfg::kBStages;
  extern __shared__ __align__(128) uint8_t tc_smem[];
  __shared__ uint64_t full[kStages], empty[kStages], bfull[kBStages], bempty[kBStages], tfull, tempty, drain;
  __shared__ uint32_t tmem_base;
  __shared__ int fail, consumed, bconsumed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) lio::umma::tmem_alloc(&tmem_base, Cfg::kTmem);
  if (tid == 0) {
    for (int b = 0; b < kStages; b++) {
      lio::umma::mbar_init(&full[b], 1);
      lio::umma::mbar_init(&empty[b], 1);
    }
    for (int b = 0; b < kBStages; b++) {
      lio::umma::mbar_init(&bfull[b], 1);
      lio::umma::mbar_init(&bempty[b], kTcEpiWarps);
    }
    lio::umma::mbar_init(&tfull, 1);
    lio::umma::mbar_init(&tempty, kTcEpiWarps);
    lio::umma::mbar_init(&drain, 1);
    lio::umma::fence_mbar_init();
    fail = 0;
    consumed = 0;
    bconsumed = 0;
  }
  {
    // The basis ring starts zeroed: a chunk of a group's last function tile is
    // copied for its m - 32 ft valid functions only, and the rows after them
    // keep the finite values of earlier chunks, which meet G = 0 in the dots.
    double* ring = reinterpret_cast<double*>(tc_smem + Cfg::kBRing);
    for (int i = tid; i < kBStages * kTcChunk; i += blockDim.x) ring[i] = 0.0;
    lio::umma::fence_proxy_async_smem();
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  lio::umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  volatile int* vfail = &fail;
  int issued = 0;  // producers: stages / chunks issued

  if (warp == Cfg::kProd) {
    // ------------------------------------------------------------ operand producer
    if (lane == 0) {
      const uint64_t keep = lio::umma::l2_evict_last(), drop = lio::umma::l2_evict_first();
      int cnt = 0;
      for (int w = blockIdx.x; w < ntiles && !*vfail; w += gridDim.x) {
        const int2 t = tiles[w];
        const GroupDev& G = groups[t.x];
        const int nks = G.m32 / 32, nft = G.nftc;
        const int8_t* Abase = aslices + G.sl_off + (long long)t.y * NA * nks * kTcStepA;
        for (int tt = 0; tt < nft * NP && !*vfail; tt++) {
          const int ft = tt / NP, pass = tt - ft * NP;
          for (int kk = 0; kk < nks; kk++, cnt++) {
            const int buf = cnt % kStages, use = cnt / kStages;
            if (use > 0 && (*vfail || !lio::umma::mbar_wait(&empty[buf], (use - 1) & 1))) {
              *vfail = 1;
              break;
            }
            uint8_t* stage = tc_smem + buf * Cfg::kStage;
            lio::umma::mbar_expect_tx(&full[buf], (uint32_t)Cfg::kStage);
            // A is read again by the tile's next function tile; D by every tile of the group
            const uint64_t pa = ft + 1 < nft ? keep : drop;
            for (int kp = 0; kp < KP; kp++)
              lio::umma::bulk_copy_g2s_hint(stage + kp * kTcStepA,
                                            Abase + ((long long)(pass * KP + kp) * nks + kk) * kTcStepA, kTcStepA,
                                            &full[buf], pa);
            for (int sp = 0; sp < NS; sp++)
              lio::umma::bulk_copy_g2s_hint(
                  stage + Cfg::kStageA + sp * kTcStepD,
                  (sp == 0 ? dsl_a : dsl_b) + G.ds_off + ((long long)ft * nks + kk) * kTcStepD, kTcStepD, &full[buf],
                  keep);
            issued = cnt + 1;
          }
        }
      }
    }
  } else if (warp == Cfg::kBasisProd) {
    // ------------------------------------------------------------ basis producer
    if (lane == 0) {
      const uint64_t keep = lio::umma::l2_evict_last(), drop = lio::umma::l2_evict_first();
      int cnt = 0;
      for (int w = blockIdx.x; w < ntiles && !*vfail; w += gridDim.x) {
        const int2 t = tiles[w];
        const GroupDev& G = groups[t.x];
        const int nft = G.nftc;
        for (int tt = 0; tt < nft * NP && !*vfail; tt++) {
          const int ft = tt / NP, first = (tt - ft * NP) * KP;
          const double* src = bblk + G.bb_off + (long long)(t.y * nft + ft) * NK * kTcChunk;
          // rows (functions) of the chunk that exist: 1 KB each, contiguous from row 0
          const uint32_t bytes = (uint32_t)min(kTcFuncs, G.m - ft * kTcFuncs) * kTcPoints * 8;
          for (int k = unit_klo(first); k <= unit_khi(first, NK); k++, cnt++) {
            const int buf = cnt % kBStages, use = cnt / kBStages;
            if (use > 0 && (*vfail || !lio::umma::mbar_wait(&bempty[buf], (use - 1) & 1))) {
              *vfail = 1;
              break;
            }
            lio::umma::mbar_expect_tx(&bfull[buf], bytes);
            lio::umma::bulk_copy_g2s_hint(tc_smem + Cfg::kBRing + (size_t)buf * kTcChunk * 8,
                                          src + (long long)k * kTcChunk, bytes, &bfull[buf],
                                          chunk_reused(first, k, KP) ? keep : drop);
            issued = cnt + 1;
          }
        }
      }
    }
  } else if (warp == Cfg::kMma) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t smem0 = lio::umma::smem_u32(tc_smem);
      int cnt = 0, ucnt = 0;
      bool stop = false;
      for (int w = blockIdx.x; w < ntiles && !stop; w += gridDim.x) {
        const int2 t = tiles[w];
        const GroupDev& G = groups[t.x];
        const int nks = G.m32 / 32, nft = G.nftc;
        for (int tt = 0; tt < nft * NP && !stop; tt++, ucnt++) {
          if (ucnt > 0) {
            if (*vfail || !lio::umma::mbar_wait(&tempty, (ucnt - 1) & 1)) {
              stop = true;
              break;
            }
            lio::umma::fence_after_sync();
          }
          for (int kk = 0; kk < nks; kk++, cnt++) {
            const int buf = cnt % kStages, use = cnt / kStages;
            if (*vfail || !lio::umma::mbar_wait(&full[buf], use & 1)) {
              stop = true;
              break;
            }
            consumed = cnt + 1;
            lio::umma::fence_after_sync();
            const uint32_t sa = smem0 + buf * Cfg::kStage;
#pragma unroll
            for (int sp = 0; sp < NS; sp++) {
              // stacked D of this spin: K-major, 192 rows (LBO = 16 * 192 bytes between K halves)
              const uint64_t bd = lio::umma::smem_desc(sa + Cfg::kStageA + sp * kTcStepD, 16u * kTcTall, 128u);
#pragma unroll
              for (int kp = 0; kp < KP; kp++)
#pragma unroll
                for (int s = 0; s < kSlices; s++)
                  lio::umma::mma_i8(
                      tbase + (uint32_t)(((sp * KP + kp) * kSlices + s) * kTcFuncs),
                      lio::umma::smem_desc(sa + kp * kTcStepA + s * kTcSliceA, 16u * kTcPoints, 128u), bd,
                      lio::umma::idesc_i8(kTcPoints, (kSlices - s) * kTcFuncs), (kk > 0 || s > 0) ? 1u : 0u);
            }
            lio::umma::commit(&empty[buf]);
            if (kk == nks - 1) lio::umma::commit(&tfull);
          }
        }
      }
      if (stop) *vfail = 1;
      // every MMA issued so far has completed once this arrives
      lio::umma::commit(&drain);
      if (!lio::umma::mbar_wait(&drain, 0)) *vfail = 1;
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int quad = warp & 3, colg = warp >> 2;
    const int row = quad * 32 + lane;
    const int etid = tid;  // 0 .. 255
    const uint32_t lane_base = tbase + ((uint32_t)(quad * 32) << 16);
    const double* bring = reinterpret_cast<const double*>(tc_smem + Cfg::kBRing);
    double* red = reinterpret_cast<double*>(tc_smem + Cfg::kRed);
    double* tsa = reinterpret_cast<double*>(tc_smem + Cfg::kTab);  // 2^f_T per function, spin a
    double* tsb = tsa + fcap;                                        // spin b (NS = 2 only)
    bool lfail = false;
    int ucnt = 0, bcnt = 0;
    for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
      const int2 t = tiles[w];
      const GroupDev& G = groups[t.x];
      const int m = G.m, ldp = G.ldp, nft = G.nftc, ntt = nft * NP;
      const int p = t.y * kTcPoints + row;
      // per-function scales of this group (the previous tile's readers are past the last barrier)
      const int mt = nft * kTcFuncs;  // <= fcap: fcap covers the largest padded m
      for (int i = etid; i < mt; i += kTcEpiWarps * 32) {
        tsa[i] = i < m ? pow2(dexp_a[G.dexp_off + i]) : 0.0;
        if (NS == 2) tsb[i] = i < m ? pow2(dexp_b[G.dexp_off + i]) : 0.0;
      }
      epi_sync_or(false);
      double spx[NA];  // 2^(point exponent - 7(S+1)) per kind
#pragma unroll
      for (int a = 0; a < NA; a++) spx[a] = pow2(aexp[G.aexp_off + (long long)a * ldp + p] - 7 * (kSlices + 1));
      double q[NS][NQ];
#pragma unroll
      for (int sp = 0; sp < NS; sp++)
#pragma unroll
        for (int k = 0; k < NQ; k++) q[sp][k] = 0.0;
      const bool narrow = G.m32 <= kTcNarrowK;
      for (int tt = 0; tt < ntt; tt++, ucnt++) {
        const int ft = tt / NP, pass = tt - ft * NP, first = pass * KP;
        const int cb = ft * kTcFuncs + colg * CPW;  // first function of this warp's columns
        // ---- the unit's accumulators -> G / 2^(e_p + f_T - 7(S+1)) (FP64) in registers; the
        // scale is applied to each row dot
        double sc[NS][KP];
#pragma unroll
        for (int sp = 0; sp < NS; sp++)
#pragma unroll
          for (int kp = 0; kp < KP; kp++) sc[sp][kp] = spx[first + kp] * (sp == 0 ? tsa : tsb)[ft * kTcFuncs];
        bool ok = !lfail && !*vfail && lio::umma::mbar_wait(&tfull, ucnt & 1);
        ok = __all_sync(0xffffffffu, ok);
        lio::umma::fence_after_sync();
        double g[CPW][NS][KP];
        if (ok) {
#pragma unroll
          for (int sp = 0; sp < NS; sp++)
#pragma unroll
            for (int kp = 0; kp < KP; kp++)
#pragma unroll
              for (int h = 0; h < CPW / 8; h++) {
                int32_t lv[kSlices][8];
#pragma unroll
                for (int l = 0; l < kSlices; l++)
                  lio::umma::tmem_ld8(
                      lane_base + (uint32_t)(((sp * KP + kp) * kSlices + l) * kTcFuncs + colg * CPW + h * 8), lv[l]);
                lio::umma::tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < 8; c++) g[h * 8 + c][sp][kp] = level_sum(lv, c, narrow);
              }
        } else {
          lfail = true;
          *vfail = 1;
        }
        // accumulators read: hand TMEM back to the MMA issuer
        lio::umma::fence_before_sync();
        __syncwarp();
        if (lane == 0 && ok) lio::umma::mbar_arrive(&tempty);
        // ---- row dots against the unit's basis chunks (none for a column half past m)
        const int klo = unit_klo(first), khi = unit_khi(first, NK);
        const bool cols = cb < m;
        for (int k = klo; k <= khi; k++, bcnt++) {
          const int buf = bcnt % kBStages, use = bcnt / kBStages;
          bool okb = !lfail && !*vfail && lio::umma::mbar_wait(&bfull[buf], use & 1);
          okb = __all_sync(0xffffffffu, okb);
          if (!okb) {
            lfail = true;
            *vfail = 1;
          } else if (cols) {
            const double* ch = bring + (size_t)buf * kTcChunk + (colg * CPW) * kTcPoints + row;
            double d4[4][NS][KP];
#pragma unroll
            for (int c = 0; c < 4; c++)
#pragma unroll
              for (int sp = 0; sp < NS; sp++)
#pragma unroll
                for (int kp = 0; kp < KP; kp++) d4[c][sp][kp] = ch[c * kTcPoints] * g[c][sp][kp];
#pragma unroll
            for (int c = 4; c < CPW; c++) {
              const double v = ch[c * kTcPoints];
#pragma unroll
              for (int sp = 0; sp < NS; sp++)
#pragma unroll
                for (int kp = 0; kp < KP; kp++) d4[c & 3][sp][kp] = fma(v, g[c][sp][kp], d4[c & 3][sp][kp]);
            }
            double d[NS][KP];
#pragma unroll
            for (int sp = 0; sp < NS; sp++)
#pragma unroll
              for (int kp = 0; kp < KP; kp++)
                d[sp][kp] = ((d4[0][sp][kp] + d4[1][sp][kp]) + (d4[2][sp][kp] + d4[3][sp][kp])) * sc[sp][kp];
            apply_chunk<GGA, NS, NQ, KP>(first, k, d, q);
          }
          __syncwarp();
          if (lane == 0 && okb) lio::umma::mbar_arrive(&bempty[buf]);
        }
      }
      // tile done: column group 1 hands its sums to column group 0, which writes them
      if (colg == 1) {
#pragma unroll
        for (int sp = 0; sp < NS; sp++)
#pragma unroll
          for (int k = 0; k < NQ; k++) red[(sp * kTcPoints + row) * NQ + k] = q[sp][k];
      }
      const bool anyfail = epi_sync_or(lfail || *vfail);
      if (anyfail) break;
      if (colg == 0) {
#pragma unroll
        for (int sp = 0; sp < NS; sp++) {
          double* dst = (sp == 0 ? part_a : part_b) + G.part_off;
#pragma unroll
          for (int k = 0; k < NQ; k++) dst[(long long)k * ldp + p] = q[sp][k] + red[(sp * kTcPoints + row) * NQ + k];
        }
      }
      epi_sync_or(false);  // the table and the reduction area are free again
    }
    if (etid == 0) bconsumed = bcnt;
  }
  __syncthreads();  // every role done
  if ((warp == Cfg::kProd || warp == Cfg::kBasisProd) && lane == 0) {
    // copies issued but never consumed (after a timeout) land before the CTA exits
    const bool basis = warp == Cfg::kBasisProd;
    const int nb = basis ? kBStages : kStages;
    for (int k = basis ? bconsumed : consumed; k < issued; k++)
      if (!lio::umma::mbar_wait(basis ? &bfull[k % nb] : &full[k % nb], (k / nb) & 1)) break;
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  if (tid == 0 && fail) atomicExch(err, 1);
  if (warp == 0) lio::umma::tmem_dealloc(tbase, Cfg::kTmem);
}
