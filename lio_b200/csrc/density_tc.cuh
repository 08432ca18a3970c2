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
// The row-dot epilogue needs F, dF and d2F at (p, i) in FP64. They are not
// streamed from HBM (80 bytes per point and function, three quarters of the
// kernel's traffic before). Each value is P(r) R(r): a Cartesian monomial of the
// point's displacement from the function's atom times the shell's contracted
// radial part, whose sums t, tg, th (the only exponentials) are computed once per
// geometry (k_radial, 24 bytes per point and shell). The epilogue contracts G
// shell by shell in factored form: with S0 = sum_c P_c G_c, S1_a = sum_c
// dP_c/da G_c and S2_ab = sum_c d2P_c/da db G_c over the shell's components,
//   sum_c F_c G_c        = t S0
//   sum_c dF_c/da G_c    = t S1_a + r_a tg2 S0
//   sum_c d2F_c/dadb G_c = t S2_ab + tg2 (r_b S1_a + r_a S1_b + delta_ab S0) + th4 r_a r_b S0
// (tg2 = -2 tg, th4 = 4 th; the closed forms of g2g/cpu/functions.cpp:81-352
// summed over a shell): a few FP64 operations per function instead of ten
// values and their row dots.
#pragma once
#include <type_traits>

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
constexpr int kTcMaxWarpShells = 16;  // shells an epilogue warp's 16 columns touch, at most
template <bool GGA, int NS>
struct TcCfg {
  static constexpr int KP = (GGA && NS == 1) ? 2 : 1;
  static constexpr int NA = GGA ? 4 : 1;   // kinds of the contraction
  static constexpr int NP = NA / KP;       // units per function tile
  static constexpr int NQ = GGA ? 10 : 1;
  static constexpr int NR = GGA ? 3 : 1;   // radial sums per (shell, point): t (LDA); t, -2 tg, 4 th (GGA)
  static constexpr int kStageA = KP * kTcStepA;
  static constexpr int kStage = kStageA + NS * kTcStepD;
  static constexpr uint32_t kCols = NS * KP * kSlices * kTcFuncs;
  // after the level columns, the unit's G in FP64: per function column c the
  // NS x KP values, two 32-bit TMEM columns each (column kCols + c * kGPer + ...)
  static constexpr uint32_t kGPer = 2 * NS * KP;
  static constexpr uint32_t kTmemUsed = kCols + kTcFuncs * kGPer;
  static constexpr uint32_t kTmem = kTmemUsed <= 256 ? 256 : 512;
  static_assert(kTmemUsed <= 512, "levels and G fit the 512 TMEM columns");
  // epilogue warps, operand producer, MMA issuer
  static constexpr int kWarps = kTcEpiWarps + 2;
  static constexpr int kThreads = 32 * kWarps;
  static constexpr int kProd = kTcEpiWarps, kMma = kTcEpiWarps + 1;
  // dynamic shared memory: operand ring | radial sums (per epilogue warp: up to
  // 16 shells x NR values x 32 points, each thread's own) | per-group
  // density-tile scales. At the end of a tile each warp of column group 1 hands
  // its points' sums to column group 0 through its own radial area, which it
  // no longer reads by then. Two operand stages: a third (room for it only in
  // the open-shell form) measured slower at 256 atoms, 7.23 against 7.01 ms.
  static constexpr size_t kWarpRad = (size_t)kTcMaxWarpShells * NR * 32 * 8;
  static constexpr size_t kRadBytes = (size_t)kTcEpiWarps * kWarpRad;
  static constexpr size_t kRedBytes = (size_t)NS * 32 * NQ * 8;  // per warp: [spin][lane][NQ] FP64
  static_assert(kRedBytes <= kWarpRad, "a warp's sums fit its radial area");
  static constexpr int kStages = 2;
  static constexpr size_t kRing = (size_t)kStages * kStage;
  static constexpr size_t kRad = kRing;
  static constexpr size_t kTab = kRad + kRadBytes;
  static constexpr size_t kTabEntry = NS * 8;  // 2^f_T per function, per spin
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
      double v = P[G.pk_off + packed_index(gi, gj, G.pk_M)];
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
        v = P[G.pk_off + packed_index(gi, gj, G.pk_M)];
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

// ------------------------------------------------------------- radial sums
// Per geometry: one thread per (group, point) of a 128-point tile; for every
// shell (simple function) of the group the contracted radial sums at the point
// (g2g/cpu/functions.cpp:68-79: primitives with a_k r^2 > 70 skipped),
//   t = sum_k c_k e^(-a_k r^2),  tg2 = -2 sum_k a_k c_k e^(..),  th4 = 4 sum_k a_k^2 c_k e^(..)
// (t only for LDA, NR = 1). Layout per group and tile: [shell][NR][128 points],
// so the shells of one function tile are contiguous.
template <int NR>
__global__ void __launch_bounds__(kTcPoints) k_radial(const int2* __restrict__ tiles,
                                                      const GroupDev* __restrict__ groups,
                                                      const double* __restrict__ px, const double* __restrict__ py,
                                                      const double* __restrict__ pz, const int* __restrict__ sf_glob,
                                                      const int* __restrict__ nuc, const int* __restrict__ ncont,
                                                      const double* __restrict__ ca, const double* __restrict__ cc,
                                                      const double* __restrict__ ax, const double* __restrict__ ay,
                                                      const double* __restrict__ az, double* __restrict__ rad) {
  const int2 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int r = threadIdx.x;
  const long long p = G.pt_off + t.y * kTcPoints + r;
  const double x = px[p], y = py[p], z = pz[p];
  double* out = rad + G.rad_off + (long long)t.y * G.nsimple * NR * kTcPoints + r;
  for (int sh = 0; sh < G.nsimple; sh++) {
    const int gf = sf_glob[G.sf_off + sh];
    const int atom = nuc[gf];
    const double dx = x - ax[atom], dy = y - ay[atom], dz = z - az[atom];
    const double dist = dx * dx + dy * dy + dz * dz;
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
    out[(long long)sh * NR * kTcPoints] = tt;
    if (NR == 3) {
      out[((long long)sh * NR + 1) * kTcPoints] = -2.0 * tg;
      out[((long long)sh * NR + 2) * kTcPoints] = 4.0 * th;
    }
  }
}

// ------------------------------------------------ one shell's contribution
// Monomial sums of one shell for one (spin, kind) from its components' G values
// g[c] (0 for components outside this warp's columns): S0 = sum_c P_c g_c,
// S1[a] = sum_c dP_c/da g_c, S2 = sum_c d2P_c/da db g_c in the order xx, yy,
// zz, xy, xz, yz. TYPE 0 s (P = 1), 1 p (P = x, y, z), 2 d (P = xx, xy, yy,
// xz, yz, zz with xx, yy, zz times the normalisation n).
template <int TYPE>
struct ShellSums {
  double S0, S1[3], S2[6];
  __device__ __forceinline__ ShellSums(const double* g, const double (&r)[3], double n) {
    if constexpr (TYPE == 0) {
      S0 = g[0];
    } else if constexpr (TYPE == 1) {
      S0 = fma(r[0], g[0], fma(r[1], g[1], r[2] * g[2]));
      S1[0] = g[0];
      S1[1] = g[1];
      S1[2] = g[2];
    } else {
      const double gxx = n * g[0], gxy = g[1], gyy = n * g[2], gxz = g[3], gyz = g[4], gzz = n * g[5];
      const double x = r[0], y = r[1], z = r[2];
      S0 = fma(x * x, gxx, fma(y * y, gyy, fma(z * z, gzz, fma(x * y, gxy, fma(x * z, gxz, (y * z) * gyz)))));
      S1[0] = fma(2.0 * x, gxx, fma(y, gxy, z * gxz));
      S1[1] = fma(2.0 * y, gyy, fma(x, gxy, z * gyz));
      S1[2] = fma(2.0 * z, gzz, fma(x, gxz, y * gyz));
      S2[0] = 2.0 * gxx;
      S2[1] = 2.0 * gyy;
      S2[2] = 2.0 * gzz;
      S2[3] = gxy;
      S2[4] = gxz;
      S2[5] = gyz;
    }
  }
};

// A shell of a group as the density epilogue reads it, one 32-byte record per
// (group, shell), written per geometry: its atom's position, its type (0 s, 1 p,
// 2 d) and the group-local column of its first component. One load per shell
// instead of a chain through the shell's function, its atom and the positions.
struct ShellInfo {
  double x, y, z;
  int type, fcol;
};
static_assert(sizeof(ShellInfo) == 32, "one 32-byte record per shell");

// A shell at this thread's point: displacement from its atom and radial sums.
struct ShellPoint {
  double r[3], t, tg2, th4;
};

// Adds a shell's contribution of kind KIND (0 F, 1 dF/dx, 2 dF/dy, 3 dF/dz of
// the unit's G) to the point's q = (rho; grad rho; d2rho xx, yy, zz, xy, xz, yz);
// the factor 2 of every derivative term is applied once when q is written:
//   F : rho += t S0, grad_a += t S1_a + r_a tg2 S0,
//       d2_ab += t S2_ab + tg2 (r_b S1_a + r_a S1_b + delta_ab S0) + r_a r_b th4 S0
//   x : xx, xy, xz += t S1_(x, y, z) + r_(x, y, z) tg2 S0   (F_y G^x = F_x G^y: D is symmetric)
//   y : yy, yz += t S1_(y, z) + r_(y, z) tg2 S0
//   z : zz += t S1_z + r_z tg2 S0
template <int TYPE, int KIND, bool GGA, int NQ>
__device__ __forceinline__ void shell_finish(const ShellSums<TYPE>& S, const ShellPoint& sp, double (&q)[NQ]) {
  if constexpr (!GGA) {
    q[0] = fma(sp.t, S.S0, q[0]);
  } else if constexpr (KIND == 0) {
    q[0] = fma(sp.t, S.S0, q[0]);
    const double tg0 = sp.tg2 * S.S0, th0 = sp.th4 * S.S0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      double v = sp.r[a] * tg0;
      if constexpr (TYPE > 0) v = fma(sp.t, S.S1[a], v);
      q[(1 + a) % NQ] += v;
    }
#pragma unroll
    for (int h = 0; h < 6; h++) {
      constexpr int ha[6] = {0, 1, 2, 0, 0, 1}, hb[6] = {0, 1, 2, 1, 2, 2};
      const int a = ha[h], b = hb[h];
      double v = (sp.r[a] * sp.r[b]) * th0;     // r_a r_b th4 S0
      if (h < 3) v += tg0;                      // delta_ab tg2 S0
      if constexpr (TYPE > 0) v = fma(sp.tg2, fma(sp.r[b], S.S1[a], sp.r[a] * S.S1[b]), v);
      if constexpr (TYPE == 2) v = fma(sp.t, S.S2[h], v);
      q[(4 + h) % NQ] += v;
    }
  } else {
    // gradient kinds: rows xx, xy, xz (x); yy, yz (y); zz (z)
    constexpr int na = KIND == 1 ? 3 : (KIND == 2 ? 2 : 1);
    constexpr int qa[3][3] = {{4, 7, 8}, {5, 9, 0}, {6, 0, 0}};
    const double tg0 = sp.tg2 * S.S0;
#pragma unroll
    for (int j = 0; j < na; j++) {
      const int a = KIND - 1 + j;  // dF/da dotted with G^KIND
      double v = sp.r[a] * tg0;
      if constexpr (TYPE > 0) v = fma(sp.t, S.S1[a], v);
      q[qa[KIND - 1][j] % NQ] += v;
    }
  }
}

// One shell of this warp's columns for the current unit: its components' G
// (NS x KP doubles per column, parked in TMEM at gbase + column * GPER by the
// unit's read-out; columns outside [0, wlen) belong to another warp or function
// tile and count as 0), the monomial sums per (spin, kind) and their finishing
// step. `pass` selects the unit's first kind (F, x, y, z in units of KP).
template <int TYPE, bool GGA, int NS, int KP, int NQ, int GPER>
__device__ __forceinline__ void shell_unit(int pass, uint32_t gbase, int fcol, int wlen, const ShellPoint& spt,
                                           double dnorm, double (&q)[NS][NQ]) {
  constexpr int NC = TYPE == 0 ? 1 : (TYPE == 1 ? 3 : 6);
  uint32_t raw[NC][4];
#pragma unroll
  for (int c = 0; c < NC; c++) {
    const int col = fcol + c;
    if (col >= 0 && col < wlen) {  // warp-uniform
      if constexpr (GPER == 4)
        lio::umma::tmem_ld4u(gbase + (uint32_t)(col * GPER), raw[c][0], raw[c][1], raw[c][2], raw[c][3]);
      else
        lio::umma::tmem_ld2(gbase + (uint32_t)(col * GPER), raw[c][0], raw[c][1]);
    } else {
#pragma unroll
      for (int k = 0; k < 4; k++) raw[c][k] = 0u;  // the bits of +0.0
    }
  }
  lio::umma::tmem_wait_ld();
  auto run = [&](auto first_tag) {
    constexpr int FIRST = decltype(first_tag)::value;
#pragma unroll
    for (int kp = 0; kp < KP; kp++)
#pragma unroll
      for (int sp = 0; sp < NS; sp++) {
        const int sk = sp * KP + kp;
        double g[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) g[c] = __hiloint2double((int)raw[c][2 * sk + 1], (int)raw[c][2 * sk]);
        const ShellSums<TYPE> S(g, spt.r, dnorm);
        if (kp == 0)
          shell_finish<TYPE, FIRST, GGA, NQ>(S, spt, q[sp]);
        else
          shell_finish<TYPE, (FIRST + 1 < 4 ? FIRST + 1 : 3), GGA, NQ>(S, spt, q[sp]);
      }
  };
  if constexpr (!GGA) {
    run(std::integral_constant<int, 0>{});
  } else if constexpr (KP == 2) {
    if (pass == 0) run(std::integral_constant<int, 0>{});  // F and x
    else run(std::integral_constant<int, 2>{});            // y and z
  } else {
    if (pass == 0) run(std::integral_constant<int, 0>{});
    else if (pass == 1) run(std::integral_constant<int, 1>{});
    else if (pass == 2) run(std::integral_constant<int, 2>{});
    else run(std::integral_constant<int, 3>{});
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
//               NS x KP x S x 32 level columns in TMEM.
// Per 32-function tile each epilogue warp copies the radial sums of the shells
// its 16 columns touch (at its own points) into its part of shared memory
// while the tile's first unit runs. Per unit it reads the levels (tfull),
// forms G in FP64 and parks it in the TMEM columns after the levels, hands the
// level columns back (tempty) so the next unit's MMAs overlap its work, and
// contracts G shell by shell. The warps of a tile meet only at its start and
// end. Every wait is bounded; a timeout sets `fail`, which the other roles poll,
// and the kernel drains its copies and MMAs before it frees TMEM and reports
// the error.
template <bool GGA, int NS>
__global__ void __launch_bounds__(TcCfg<GGA, NS>::kThreads, 1)
    k_density_tc(const int2* __restrict__ tiles, int ntiles, const GroupDev* __restrict__ groups,
                 const int8_t* __restrict__ aslices, const int16_t* __restrict__ aexp,
                 const int8_t* __restrict__ dsl_a, const int16_t* __restrict__ dexp_a,
                 const int8_t* __restrict__ dsl_b, const int16_t* __restrict__ dexp_b, int fcap,
                 const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
                 const int* __restrict__ fn_sh, const ShellInfo* __restrict__ sinfo, const double* __restrict__ rad,
                 double dnorm, double* __restrict__ part_a, double* __restrict__ part_b, int* __restrict__ err) {
  using Cfg = TcCfg<GGA, NS>;
  constexpr int KP = Cfg::KP, NP = Cfg::NP, NA = Cfg::NA, NQ = Cfg::NQ, NR = Cfg::NR, CPW = kTcCpw;
  constexpr int kStages = Cfg::kStages;
  extern __shared__ __align__(128) uint8_t tc_smem[];
  __shared__ uint64_t full[kStages], empty[kStages], tfull, tempty, drain;
  __shared__ uint32_t tmem_base;
  __shared__ int fail, consumed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) lio::umma::tmem_alloc(&tmem_base, Cfg::kTmem);
  if (tid == 0) {
    for (int b = 0; b < kStages; b++) {
      lio::umma::mbar_init(&full[b], 1);
      lio::umma::mbar_init(&empty[b], 1);
    }
    lio::umma::mbar_init(&tfull, 1);
    lio::umma::mbar_init(&tempty, kTcEpiWarps);
    lio::umma::mbar_init(&drain, 1);
    lio::umma::fence_mbar_init();
    fail = 0;
    consumed = 0;
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  lio::umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  volatile int* vfail = &fail;
  int issued = 0;  // producer: stages issued

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
  } else if (warp == Cfg::kMma) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      // descriptors of the first A slice and of the stacked D of each stage; an
      // operand further into the stage adds its byte offset / 16 to the start
      // address field (bits 0-13: shared addresses stay below 2^18 bytes)
      const uint32_t smem0 = lio::umma::smem_u32(tc_smem);
      const uint64_t ad0 = lio::umma::smem_desc(smem0, 16u * kTcPoints, 128u);
      const uint64_t ad1 = lio::umma::smem_desc(smem0 + Cfg::kStage, 16u * kTcPoints, 128u);
      const uint64_t dd0 = lio::umma::smem_desc(smem0 + Cfg::kStageA, 16u * kTcTall, 128u);
      const uint64_t dd1 = lio::umma::smem_desc(smem0 + Cfg::kStage + Cfg::kStageA, 16u * kTcTall, 128u);
      static_assert(Cfg::kStages == 2, "two descriptor bases");
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
            const uint64_t ad = buf ? ad1 : ad0, dd = buf ? dd1 : dd0;
#pragma unroll
            for (int sp = 0; sp < NS; sp++) {
              // stacked D of this spin: K-major, 192 rows (LBO = 16 * 192 bytes between K halves)
              const uint64_t bd = dd + (uint64_t)((sp * kTcStepD) >> 4);
#pragma unroll
              for (int kp = 0; kp < KP; kp++)
#pragma unroll
                for (int s = 0; s < kSlices; s++)
                  lio::umma::mma_i8(tbase + (uint32_t)(((sp * KP + kp) * kSlices + s) * kTcFuncs),
                                    ad + (uint64_t)((kp * kTcStepA + s * kTcSliceA) >> 4), bd,
                                    lio::umma::idesc_i8(kTcPoints, (kSlices - s) * kTcFuncs),
                                    (kk > 0 || s > 0) ? 1u : 0u);
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
    const int row = quad * 32 + lane;  // this thread's point of the tile
    const int etid = tid;              // 0 .. 255
    const uint32_t lane_base = tbase + ((uint32_t)(quad * 32) << 16);
    // this warp's radial sums, [shell][NR][lane]: every thread reads only its own values
    double* wrad = reinterpret_cast<double*>(tc_smem + Cfg::kRad + (size_t)warp * Cfg::kWarpRad) + lane;
    const uint32_t wrad_s = lio::umma::smem_u32(wrad);
    // column group 1 -> 0 hand-off at the end of a tile: warp 4 + quad's radial area, [spin][lane][NQ]
    double* red = reinterpret_cast<double*>(tc_smem + Cfg::kRad + (size_t)(4 + quad) * Cfg::kWarpRad);
    double* tsa = reinterpret_cast<double*>(tc_smem + Cfg::kTab);  // 2^f_T per function, spin a
    double* tsb = tsa + fcap;                                        // spin b (NS = 2 only)
    bool lfail = false;
    int ucnt = 0;
    for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
      const int2 t = tiles[w];
      const GroupDev& G = groups[t.x];
      const int m = G.m, ldp = G.ldp, nft = G.nftc;
      const int p = t.y * kTcPoints + row;
      // per-function scales of this group (the previous tile's readers are past the last barrier)
      const int mt = nft * kTcFuncs;  // <= fcap: fcap covers the largest padded m
      for (int i = etid; i < mt; i += kTcEpiWarps * 32) {
        tsa[i] = i < m ? pow2(dexp_a[G.dexp_off + i]) : 0.0;
        if (NS == 2) tsb[i] = i < m ? pow2(dexp_b[G.dexp_off + i]) : 0.0;
      }
      double spx[NA];  // 2^(point exponent - 7(S+1)) per kind
#pragma unroll
      for (int a = 0; a < NA; a++) spx[a] = pow2(aexp[G.aexp_off + (long long)a * ldp + p] - 7 * (kSlices + 1));
      const double xp = px[G.pt_off + p], yp = py[G.pt_off + p], zp = pz[G.pt_off + p];
      double q[NS][NQ];
#pragma unroll
      for (int sp = 0; sp < NS; sp++)
#pragma unroll
        for (int k = 0; k < NQ; k++) q[sp][k] = 0.0;
      const bool narrow = G.m32 <= kTcNarrowK;
      const int* fsh = fn_sh + G.fn_off;
      const double* trad = rad + G.rad_off + (long long)t.y * G.nsimple * NR * kTcPoints + row;
      epi_sync_or(false);  // the scale table is complete
      for (int ft = 0; ft < nft; ft++) {
        const int i0 = ft * kTcFuncs;
        // ---- this warp's columns [w0, w0 + wlen) and the shells they touch (lane s holds shell s)
        const int w0 = i0 + colg * CPW, wlen = min(CPW, m - w0);
        int nsl = 0, sh_a = 0;
        double s_ax = 0.0, s_ay = 0.0, s_az = 0.0;
        int s_type = 0, s_fcol = 0;
        if (wlen > 0) {
          sh_a = fsh[w0];
          nsl = fsh[w0 + wlen - 1] - sh_a + 1;  // <= 16: one shell per function at most
          if (lane < nsl) {
            const ShellInfo si = sinfo[G.sf_off + sh_a + lane];
            s_ax = si.x;
            s_ay = si.y;
            s_az = si.z;
            s_type = si.type;
            s_fcol = si.fcol - w0;  // first component's column in the window (may be < 0)
          }
          // their radial sums at this thread's point, copied while the unit's MMAs run
          for (int s2 = 0; s2 < nsl; s2++)
#pragma unroll
            for (int k = 0; k < NR; k++)
              asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(wrad_s + (uint32_t)((s2 * NR + k) * 32 * 8)),
                           "l"(trad + ((long long)(sh_a + s2) * NR + k) * kTcPoints)
                           : "memory");
          asm volatile("cp.async.commit_group;" ::: "memory");
        }
        for (int pass = 0; pass < NP; pass++, ucnt++) {
          const int first = pass * KP;
          const int cb = colg * CPW;  // this warp's first column of the function tile
          // ---- the unit's accumulators -> G (FP64), parked in the TMEM columns after the levels
          double sc[NS][KP];
#pragma unroll
          for (int sp = 0; sp < NS; sp++)
#pragma unroll
            for (int kp = 0; kp < KP; kp++) sc[sp][kp] = spx[first + kp] * (sp == 0 ? tsa : tsb)[i0];
          bool ok = !lfail && !*vfail && lio::umma::mbar_wait(&tfull, ucnt & 1);
          ok = __all_sync(0xffffffffu, ok);
          lio::umma::fence_after_sync();
          const uint32_t gbase = lane_base + Cfg::kCols + (uint32_t)cb * Cfg::kGPer;  // this warp's columns
          if (ok && wlen > 0) {
#pragma unroll
            for (int h = 0; h < CPW / 8; h++) {
              double gh[8][NS][KP];
#pragma unroll
              for (int sp = 0; sp < NS; sp++)
#pragma unroll
                for (int kp = 0; kp < KP; kp++) {
                  int32_t lv[kSlices][8];
#pragma unroll
                  for (int l = 0; l < kSlices; l++)
                    lio::umma::tmem_ld8(lane_base + (uint32_t)(((sp * KP + kp) * kSlices + l) * kTcFuncs + cb + h * 8),
                                        lv[l]);
                  lio::umma::tmem_wait_ld();
#pragma unroll
                  for (int c = 0; c < 8; c++) gh[c][sp][kp] = level_sum(lv, c, narrow) * sc[sp][kp];
                }
              // 8 columns x NS x KP doubles: 8 * kGPer consecutive 32-bit TMEM columns
#pragma unroll
              for (int part = 0; part < (8 * (int)Cfg::kGPer) / 16; part++) {
                uint32_t v[16];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                  const int idx = part * 8 + e;  // double index within the block: c * NS * KP + sp * KP + kp
                  const int c = idx / (NS * KP), sk = idx % (NS * KP);
                  const double x = gh[c][sk / KP][sk % KP];
                  v[2 * e] = (uint32_t)__double2loint(x);
                  v[2 * e + 1] = (uint32_t)__double2hiint(x);
                }
                lio::umma::tmem_st16(gbase + (uint32_t)(h * 8 * Cfg::kGPer + part * 16), v);
              }
            }
            lio::umma::tmem_wait_st();
          } else if (!ok) {
            lfail = true;
            *vfail = 1;
          }
          // levels read: hand their columns back to the MMA issuer (G stays in the columns after them)
          lio::umma::fence_before_sync();
          __syncwarp();
          if (lane == 0 && ok) lio::umma::mbar_arrive(&tempty);
          if (!ok || wlen <= 0) continue;
          if (pass == 0) asm volatile("cp.async.wait_all;" ::: "memory");  // this thread's radial sums landed
          // ---- shell by shell over this warp's columns
#pragma unroll 1
          for (int s2 = 0; s2 < nsl; s2++) {
            const int type = __shfl_sync(0xffffffffu, s_type, s2);
            const int fcol = __shfl_sync(0xffffffffu, s_fcol, s2);
            ShellPoint spt;
            spt.r[0] = xp - __shfl_sync(0xffffffffu, s_ax, s2);
            spt.r[1] = yp - __shfl_sync(0xffffffffu, s_ay, s2);
            spt.r[2] = zp - __shfl_sync(0xffffffffu, s_az, s2);
            spt.t = wrad[(s2 * NR) * 32];
            spt.tg2 = GGA ? wrad[(s2 * NR + 1) * 32] : 0.0;
            spt.th4 = GGA ? wrad[(s2 * NR + 2) * 32] : 0.0;
            if (type == 0)
              shell_unit<0, GGA, NS, KP, NQ, Cfg::kGPer>(pass, gbase, fcol, wlen, spt, dnorm, q);
            else if (type == 1)
              shell_unit<1, GGA, NS, KP, NQ, Cfg::kGPer>(pass, gbase, fcol, wlen, spt, dnorm, q);
            else
              shell_unit<2, GGA, NS, KP, NQ, Cfg::kGPer>(pass, gbase, fcol, wlen, spt, dnorm, q);
          }
        }
      }
      // tile done: column group 1 hands its sums to column group 0, which writes them
      if (colg == 1) {
#pragma unroll
        for (int sp = 0; sp < NS; sp++)
#pragma unroll
          for (int k = 0; k < NQ; k++) red[(sp * 32 + lane) * NQ + k] = q[sp][k];
      }
      const bool anyfail = epi_sync_or(lfail || *vfail);
      if (anyfail) break;
      if (colg == 0) {
#pragma unroll
        for (int sp = 0; sp < NS; sp++) {
          double* dst = (sp == 0 ? part_a : part_b) + G.part_off;
#pragma unroll
          for (int k = 0; k < NQ; k++) {
            const double v = q[sp][k] + red[(sp * 32 + lane) * NQ + k];
            dst[(long long)k * ldp + p] = k == 0 ? v : 2.0 * v;  // the factor 2 of the derivative terms
          }
        }
      }
      epi_sync_or(false);  // the table and the reduction area are free again
    }
    asm volatile("cp.async.wait_all;" ::: "memory");  // nothing in flight into shared memory at exit
  }
  __syncthreads();  // every role done
  if (warp == Cfg::kProd && lane == 0) {
    // copies issued but never consumed (after a timeout) land before the CTA exits
    for (int k = consumed; k < issued; k++)
      if (!lio::umma::mbar_wait(&full[k % kStages], (k / kStages) & 1)) break;
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  if (tid == 0 && fail) atomicExch(err, 1);
  if (warp == 0) lio::umma::tmem_dealloc(tbase, Cfg::kTmem);
}
