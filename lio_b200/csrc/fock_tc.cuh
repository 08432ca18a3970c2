// Tensor-core form of the Kohn-Sham contraction (included by engine.cu inside
// its anonymous namespace, after density_tc.cuh).
//
// K_ij = sum_p F_ip f_p F_jp (i <= j) per spin, as C = A . B^T with the points
// as the reduction dimension:
//   A_ip = F_ip          = 2^(a_i) sum_s a_s[i][p] 128^-(s+1)  (per geometry, per function row)
//   B_jp = f_p F_jp      = 2^(b_j) sum_t b_t[j][p] 128^-(t+1)  (per solve and spin, per row)
// with the same int8 slices, level accumulators and level sum as the density
// contraction. A tile is 128 functions (i) x 32 functions (j); the S slices
// of a B tile are stacked along N, level-major with the spins interleaved (row
// (t * NS + spin) * 32 + j holds b_t[j] of that spin), so the MMAs of A slice s
// over rows [0, (S - s) * NS * 32) (at most 256 per MMA) land every product
// (s, t) of every spin on level s + t: TMEM column (l * NS + spin) * 32 + j.
// The spins share each read of the A slices: 8 MMAs per K step for two spins
// instead of 12, and a third less operand traffic from shared memory, which
// bounds this kernel. The A slices are built once per geometry; the B slices
// are cut inside the contraction kernel, a K step at a time, so they never go
// through HBM. The F values of the B operand come from the blocked basis, or,
// when an engine does not keep it (RAD), from each shell's radial sum times the
// function's monomial, as k_basis forms them.
#pragma once

constexpr int kFkRows = 128;  // UMMA M: functions i per tile
constexpr int kFkCols = 32;   // functions j per tile (output columns per level)
constexpr int kFkTall = kSlices * kFkCols;  // rows of one spin's stacked B operand
constexpr int kFkStages = 4;
constexpr int kFkSliceA = 32 * kFkRows;       // bytes of one A slice per 32-point K step
constexpr int kFkStepA = kSlices * kFkSliceA;  // all A slices of a K step (contiguous)
constexpr int kFkStepB = 32 * kFkTall;         // one spin's stacked B slices of a K step (contiguous)
template <int NS>
struct FkCfg {
  static constexpr int kStageA = kFkStepA;
  static constexpr int kStage = kStageA + NS * kFkStepB;
  static constexpr int kLevelRows = NS * kFkCols;           // B rows (and TMEM columns) per level
  static constexpr int kTallRows = kSlices * kLevelRows;    // rows of the stacked B operand
  static constexpr int kMaxLevels = 256 / kLevelRows;       // levels per MMA (N <= 256)
  // ring slot: the 32 F rows (or the radial sums of up to 32 shells) of a
  // 128-point tile, each padded to 1040 bytes so that 32 lanes reading 16 bytes
  // of 32 different rows hit distinct banks, then each spin's 128 factors, then
  // the points' x, y, z (RAD)
  static constexpr int kRowBytes = kTcPoints * 8 + 16;
  static constexpr int kFac = kFkCols * kRowBytes;
  static constexpr int kXyz = kFac + NS * kTcPoints * 8;
  static constexpr int kSlot = kXyz + 3 * kTcPoints * 8;
  static constexpr size_t kSmem = (size_t)kFkStages * kStage + 2 * (size_t)kSlot;
  static constexpr uint32_t kCols = NS * kSlices * kFkCols;
  static constexpr uint32_t kTmem = kCols <= 256 ? 256 : 512;
  // B slicers (4 per spin; the first four are also the epilogue), producer, MMA issuer
  static constexpr int kSlicers = 4 * NS;
  static constexpr int kProd = kSlicers, kMma = kSlicers + 1;
  static constexpr int kThreads = 32 * (kSlicers + 2);
};
static_assert(FkCfg<2>::kSmem <= 227 * 1024, "shared memory of the Kohn-Sham kernel");

// Rows of the A operand kept for 128-row tile I of a group of m functions:
// whole tiles 128, the last its functions rounded up to a core matrix (8 rows).
// The MMA still reads 128 rows (M = 128); with the shorter leading-dimension
// offset of the stored rows, rows past them read the next bytes of the same
// stage (the other K half, the next slice, the stage's B block), which feed
// only TMEM lanes of functions past m, never read out.
__host__ __device__ __forceinline__ int fk_tile_rows(int m, int I) {
  const int left = m - I * kFkRows;
  return left >= kFkRows ? kFkRows : ((left + 7) / 8) * 8;
}
static_assert(FkCfg<1>::kSlot % 128 == 0 && FkCfg<2>::kSlot % 128 == 0 && FkCfg<2>::kStage % 128 == 0,
              "ring slots and stages stay 128-byte aligned");

// Slices of the rows of v = F (A operand, per geometry) or v = f_s F (B
// operand, per solve, both spins at once), in two passes over the FP64 basis:
// pass 1 (row exponents) runs for both operands; pass 2 writes the A slices to
// HBM, while the B slices are cut by the Kohn-Sham kernel itself (in the TALL
// layout below, in shared memory).
//
// F(i, p) of a group and the values after it up to the end of its 128-point
// tile: from the function-major basis cache (nkb = 0) or from the blocked copy
// of the tensor-core density (nkb = its number of kinds; kind 0 is F)
__device__ __forceinline__ const double* f_row(const GroupDev& G, const double* basis, int i, int p, int nkb) {
  if (nkb == 0) return basis + G.bas_off + (long long)i * G.ldp + p;
  return basis + G.bb_off + (long long)((p >> 7) * G.nftc + (i >> 5)) * nkb * kTcChunk + (i & 31) * kTcPoints +
         (p & 127);
}

// F values without the blocked basis: a function's value at a point is its
// shell's contracted radial sum t (k_radial: per group and 128-point tile,
// [shell][nr][128 points], t first) times its monomial x^lx y^ly z^lz, times
// dnorm for the d xx, yy, zz components ((dnorm P) t, the order of k_basis).
struct RadialSource {
  const double* rad;
  const double* px;
  const double* py;
  const double* pz;
  const int* fn_sh;
  const int8_t* fn_cp;
  const int* fn_atom;
  const double* ax;
  const double* ay;
  const double* az;
  double dnorm;
  int nr;
};
// the per-function constants of that product (function i of group G, i < m):
// the monomial as up to two axes (x, y or z; -1 for none), the atom's
// coordinates along them, and the d normalisation. P = (r_1)(r_2) is the
// product k_basis forms (its factors of 1.0 are exact), so F is the same value.
struct RadialRow {
  double a1, a2, scale;
  int i1, i2, sh;
  __device__ __forceinline__ void load(const RadialSource& rs, const GroupDev& G, int i) {
    const int cp = rs.fn_cp[G.fn_off + i], c = cp & 15, atom = rs.fn_atom[G.fn_off + i];
    const double ax = rs.ax[atom], ay = rs.ay[atom], az = rs.az[atom];
    const int lx = c_comp_l[c][0], ly = c_comp_l[c][1], lz = c_comp_l[c][2];
    // the first and second axis of x^lx y^ly z^lz (lx + ly + lz <= 2)
    i1 = lx > 0 ? 0 : (ly > 0 ? 1 : (lz > 0 ? 2 : -1));
    i2 = lx == 2 ? 0 : (lx + ly == 2 ? 1 : (lx + ly + lz == 2 ? 2 : -1));
    a1 = i1 == 0 ? ax : (i1 == 1 ? ay : az);
    a2 = i2 == 0 ? ax : (i2 == 1 ? ay : az);
    scale = (cp & 16) ? rs.dnorm : 1.0;
    sh = rs.fn_sh[G.fn_off + i];
  }
  __device__ __forceinline__ double value(double x, double y, double z, double t) const {
    const double p1 = i1 < 0 ? 1.0 : (i1 == 0 ? x : (i1 == 1 ? y : z)) - a1;
    const double p2 = i2 < 0 ? 1.0 : (i2 == 0 ? x : (i2 == 1 ? y : z)) - a2;
    return scale * (p1 * p2) * t;
  }
};

// Pass 1, one warp per (group, row): the row's exponent per spin from
// max_p |v_p|. Rows at or beyond m get exponent 0 (their slices are zeros).
// The row is read a 128-point tile at a time, four consecutive points per lane
// (two 16-byte loads of F and of each spin's factors), two tiles in flight.
static_assert(kPointPad % kTcPoints == 0, "rows are read in whole 128-point tiles");
template <int NS, bool RAD>
__global__ void k_fock_rowexp(const int2* __restrict__ rows, int nrows, const GroupDev* __restrict__ groups,
                              const double* __restrict__ basis, const double* __restrict__ fac_a,
                              const double* __restrict__ fac_b, int16_t* __restrict__ expo_a,
                              int16_t* __restrict__ expo_b, int use_sl_b, int nkb, RadialSource rs) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nrows) return;  // whole warps only
  const int2 t = rows[warp];
  const GroupDev& G = groups[t.x];
  const int i = t.y, ntl = G.ldp / kTcPoints;
  double amax[NS];
#pragma unroll
  for (int sp = 0; sp < NS; sp++) amax[sp] = 0.0;
  if (i < G.m) {
    RadialRow rr{};
    if (RAD) rr.load(rs, G, i);
#pragma unroll 2
    for (int T = 0; T < ntl; T++) {
      const int p = T * kTcPoints + lane * 4;
      double2 v01, v23;
      if constexpr (RAD) {
        const double* tr = rs.rad + G.rad_off + ((long long)(T * G.nsimple + rr.sh) * rs.nr) * kTcPoints + lane * 4;
        const double2 t01 = *reinterpret_cast<const double2*>(tr), t23 = *reinterpret_cast<const double2*>(tr + 2);
        // only the coordinates along the monomial's axes (the row's, one per warp)
        const long long q = G.pt_off + p;
        double f1[4] = {1.0, 1.0, 1.0, 1.0}, f2[4] = {1.0, 1.0, 1.0, 1.0};
        auto axis = [&](int ax, double a, double (&f)[4]) {
          const double* c = (ax == 0 ? rs.px : (ax == 1 ? rs.py : rs.pz)) + q;
          const double2 c01 = *reinterpret_cast<const double2*>(c), c23 = *reinterpret_cast<const double2*>(c + 2);
          f[0] = c01.x - a;
          f[1] = c01.y - a;
          f[2] = c23.x - a;
          f[3] = c23.y - a;
        };
        if (rr.i1 >= 0) axis(rr.i1, rr.a1, f1);
        if (rr.i2 >= 0) axis(rr.i2, rr.a2, f2);
        // scale (r_1 r_2) t, as RadialRow::value
        v01 = make_double2(rr.scale * (f1[0] * f2[0]) * t01.x, rr.scale * (f1[1] * f2[1]) * t01.y);
        v23 = make_double2(rr.scale * (f1[2] * f2[2]) * t23.x, rr.scale * (f1[3] * f2[3]) * t23.y);
      } else {
        const double* Fi = f_row(G, basis, i, p, nkb);
        v01 = *reinterpret_cast<const double2*>(Fi);
        v23 = *reinterpret_cast<const double2*>(Fi + 2);
      }
#pragma unroll
      for (int sp = 0; sp < NS; sp++) {
        const double* fac = sp == 0 ? fac_a : fac_b;
        double f0 = 1.0, f1 = 1.0, f2 = 1.0, f3 = 1.0;
        if (fac) {
          const double2 a01 = *reinterpret_cast<const double2*>(fac + G.pt_off + p);
          const double2 a23 = *reinterpret_cast<const double2*>(fac + G.pt_off + p + 2);
          f0 = a01.x, f1 = a01.y, f2 = a23.x, f3 = a23.y;
        }
        amax[sp] = fmax(amax[sp], fmax(fmax(fabs(v01.x * f0), fabs(v01.y * f1)),
                                       fmax(fabs(v23.x * f2), fabs(v23.y * f3))));
      }
    }
  }
  const long long ebase = use_sl_b ? G.fbe_off : G.fae_off;
#pragma unroll
  for (int sp = 0; sp < NS; sp++) {
    double a = amax[sp];
    for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
    if (lane == 0) (sp == 0 ? expo_a : expo_b)[ebase + i] = (int16_t)slice_exponent(a);
  }
}

// Pass 2 for the A operand (per geometry): a CTA per 32-row piece of a
// 128-row tile (lane = row), each warp taking 16-point blocks, one 16-byte store
// per slice. Layout per row tile and 32-point K step: the S slices one after
// the other, each a 128-row x 32-byte K-major block (kFkStepA bytes, one bulk
// copy). The B operand's layout, per 32-row tile and K step one
// (S * 32)-row x 32-byte block whose row t * 32 + r holds slice t of row r, is
// written by the Kohn-Sham kernel's slicers in shared memory.
__global__ void __launch_bounds__(256) k_fock_aslices(const int2* __restrict__ rtiles,
                                                      const GroupDev* __restrict__ groups,
                                                      const double* __restrict__ basis,
                                                      const int16_t* __restrict__ expo, int8_t* __restrict__ sl,
                                                      int nkb) {
  const int2 t = rtiles[blockIdx.x];
  const GroupDev& G = groups[t.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = t.y + lane, ldp = G.ldp, nkp = ldp / 32;
  const bool valid = i < G.m;
  const double s42 = digit_scale(expo[G.fae_off + i]);
  const int tile = i / kFkRows, r = i % kFkRows;
  const int R = fk_tile_rows(G.m, tile);  // rows stored for this tile
  if (r >= R) return;                     // past them: not stored (no shuffles below)
  for (int b = warp; b < ldp / 16; b += blockDim.x / 32) {
    const int p0 = b * 16;
    const double* Fi = f_row(G, basis, valid ? i : 0, p0, nkb);  // 16 values within one 128-point tile
    uint32_t lo[16], hi[16];
#pragma unroll
    for (int k = 0; k < 16; k += 2) {
      const double2 v = valid ? *reinterpret_cast<const double2*>(Fi + k) : make_double2(0.0, 0.0);
      digits_m(v.x, s42, lo[k], hi[k]);
      digits_m(v.y, s42, lo[k + 1], hi[k + 1]);
    }
    int8_t* blk = sl + G.fa_off + (long long)tile * nkp * kFkStepA + (long long)(p0 >> 5) * kSlices * 32 * R;
#pragma unroll
    for (int s = 0; s < kSlices; s++) {
      uint32_t w[4];
#pragma unroll
      for (int k4 = 0; k4 < 4; k4++)
        w[k4] = pack_digits(digit_field(lo[4 * k4], hi[4 * k4], s), digit_field(lo[4 * k4 + 1], hi[4 * k4 + 1], s),
                            digit_field(lo[4 * k4 + 2], hi[4 * k4 + 2], s),
                            digit_field(lo[4 * k4 + 3], hi[4 * k4 + 3], s), s == 0);
      *reinterpret_cast<uint4*>(blk + s * 32 * R + lio::umma::kmajor_offset(r, p0 & 31, R)) =
          make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// CTA = (group, 128-row tile I, 32-column tile J) with some j >= some i.
// Warp roles:
//   warps 0 .. 4 NS - 1  B slicers: per stage each cuts the values f_p F_jp 2^-b_j
//                        of 8 rows j and 32 / NS points, every spin, into S
//                        digits (digits_m: one FP64 rounding, then integer
//                        fields) and stores them in the stage's stacked B
//                        block. Warps 0-3 are also the epilogue.
//   warp 4 NS            producer: per K step the A slices (one bulk copy); per
//                        128-point tile the F rows of J (kind 0 of the blocked
//                        basis, one bulk copy per existing row) and each spin's
//                        factors, into a two-slot ring
//   warp 4 NS + 1        MMA issuer: per stage NS x S MMAs
// A stage is ready when its A copy has landed (afull) and every slicer has
// stored and fenced its part (bready). After the last K step the epilogue
// combines the levels of each (i, j) with i <= j and adds K_ij into the packed
// accumulator(s) with FP64 atomics. Every wait is bounded; a timeout sets the
// error flag, and the producer lets its copies in flight land before exiting.
template <int NS, bool RAD>
__global__ void __launch_bounds__(FkCfg<NS>::kThreads, 1)
    k_fock_tc(const int4* __restrict__ tiles, const GroupDev* __restrict__ groups, const int* __restrict__ fn_glob,
              const int8_t* __restrict__ aslices, const int16_t* __restrict__ aexp, const double* __restrict__ bblk,
              int nkb, const double* __restrict__ fac_a, const double* __restrict__ fac_b,
              const int16_t* __restrict__ bexp_a, const int16_t* __restrict__ bexp_b, int M,
              double* __restrict__ K_a, double* __restrict__ K_b, int* __restrict__ err, RadialSource rs) {
  using Cfg = FkCfg<NS>;
  extern __shared__ __align__(128) uint8_t fk_smem[];
  __shared__ uint64_t afull[kFkStages], bready[kFkStages], empty[kFkStages], cfull[2], cempty[2], done;
  __shared__ uint32_t tmem_base;
  __shared__ int fail;
  const int4 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int I = t.y, J = t.z;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nsteps = G.ldp / 32;  // a multiple of 4: groups are padded to whole 128-point tiles
  uint8_t* ring = fk_smem + (size_t)kFkStages * Cfg::kStage;
  if (warp == 0) lio::umma::tmem_alloc(&tmem_base, Cfg::kTmem);
  if (tid == 0) {
    for (int s = 0; s < kFkStages; s++) {
      lio::umma::mbar_init(&afull[s], 1);
      lio::umma::mbar_init(&bready[s], Cfg::kSlicers);
      lio::umma::mbar_init(&empty[s], 1);
    }
    for (int c = 0; c < 2; c++) {
      lio::umma::mbar_init(&cfull[c], 1);
      lio::umma::mbar_init(&cempty[c], Cfg::kSlicers);
    }
    lio::umma::mbar_init(&done, 1);
    lio::umma::fence_mbar_init();
    fail = 0;
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  lio::umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  volatile int* vfail = &fail;
  if (warp == Cfg::kProd) {
    if (lane == 0) {
      const int8_t* A = aslices + G.fa_off + (long long)I * nsteps * kFkStepA;
      const int stepA = kSlices * 32 * fk_tile_rows(G.m, I);  // A bytes of a K step
      const int rows = min(kFkCols, G.m - J * kFkCols);  // rows of J that exist (from row 0 of the chunk)
      // RAD: the shells of those rows (consecutive), one radial row each
      const int sh0 = RAD ? rs.fn_sh[G.fn_off + J * kFkCols] : 0;
      const int nsh = RAD ? rs.fn_sh[G.fn_off + J * kFkCols + rows - 1] - sh0 + 1 : 0;
      int na = 0, nc = 0;  // A stages and F tiles issued
      for (int st = 0; st < nsteps && !*vfail; st++) {
        const int T = st >> 2;
        if ((st & 3) == 0) {
          const int c = T & 1;
          if (T >= 2 && !lio::umma::mbar_wait(&cempty[c], ((T >> 1) - 1) & 1)) {
            *vfail = 1;
            break;
          }
          uint8_t* slot = ring + c * Cfg::kSlot;
          if constexpr (RAD) {
            const double* tr = rs.rad + G.rad_off + ((long long)(T * G.nsimple + sh0) * rs.nr) * kTcPoints;
            lio::umma::mbar_expect_tx(&cfull[c], (uint32_t)((nsh + NS + 3) * kTcPoints * 8));
            for (int r = 0; r < nsh; r++)
              lio::umma::bulk_copy_g2s(slot + r * Cfg::kRowBytes, tr + (long long)r * rs.nr * kTcPoints,
                                       kTcPoints * 8, &cfull[c]);
            const double* xyz[3] = {rs.px, rs.py, rs.pz};
            for (int d3 = 0; d3 < 3; d3++)
              lio::umma::bulk_copy_g2s(slot + Cfg::kXyz + d3 * kTcPoints * 8, xyz[d3] + G.pt_off + T * kTcPoints,
                                       kTcPoints * 8, &cfull[c]);
          } else {
            const double* F = bblk + G.bb_off + (long long)(T * G.nftc + J) * nkb * kTcChunk;
            lio::umma::mbar_expect_tx(&cfull[c], (uint32_t)((rows + NS) * kTcPoints * 8));
            for (int r = 0; r < rows; r++)
              lio::umma::bulk_copy_g2s(slot + r * Cfg::kRowBytes, F + r * kTcPoints, kTcPoints * 8, &cfull[c]);
          }
          for (int sp = 0; sp < NS; sp++)
            lio::umma::bulk_copy_g2s(slot + Cfg::kFac + sp * kTcPoints * 8,
                                     (sp == 0 ? fac_a : fac_b) + G.pt_off + T * kTcPoints, kTcPoints * 8, &cfull[c]);
          nc = T + 1;
        }
        const int buf = st % kFkStages, use = st / kFkStages;
        if (use > 0 && !lio::umma::mbar_wait(&empty[buf], (use - 1) & 1)) {
          *vfail = 1;
          break;
        }
        lio::umma::mbar_expect_tx(&afull[buf], (uint32_t)stepA);
        lio::umma::bulk_copy_g2s(fk_smem + buf * Cfg::kStage, A + (long long)st * stepA, stepA, &afull[buf]);
        na = st + 1;
      }
      // copies in flight land before the CTA exits (each is the latest phase of its barrier)
      for (int k = max(0, na - kFkStages); k < na; k++)
        if (!lio::umma::mbar_wait(&afull[k % kFkStages], (k / kFkStages) & 1)) break;
      for (int T = max(0, nc - 2); T < nc; T++)
        if (!lio::umma::mbar_wait(&cfull[T & 1], (T >> 1) & 1)) break;
    }
  } else if (warp == Cfg::kMma) {
    if (lane == 0) {
      const uint32_t smem0 = lio::umma::smem_u32(fk_smem);
      const uint32_t R = (uint32_t)fk_tile_rows(G.m, I);  // A rows stored per K half
      for (int st = 0; st < nsteps; st++) {
        const int buf = st % kFkStages, use = st / kFkStages;
        if (*vfail || !lio::umma::mbar_wait(&afull[buf], use & 1) || !lio::umma::mbar_wait(&bready[buf], use & 1)) {
          *vfail = 1;
          break;
        }
        lio::umma::fence_after_sync();
        const uint32_t sa = smem0 + buf * Cfg::kStage;
        // stacked B: K-major, kTallRows rows (LBO = 16 * kTallRows bytes between K halves); the
        // rows of levels t0 .. start (t0 * kLevelRows / 8) core matrices in. At st = 0 the
        // MMAs of slice 0 (levels 0 .. S-1, disjoint columns) write every column first.
#pragma unroll
        for (int s = 0; s < kSlices; s++) {
          const uint64_t ad = lio::umma::smem_desc(sa + s * 32u * R, 16u * R, 128u);
#pragma unroll
          for (int t0 = 0; t0 < kSlices - s; t0 += Cfg::kMaxLevels) {
            const int nl = min(Cfg::kMaxLevels, kSlices - s - t0);
            const uint64_t bd = lio::umma::smem_desc(sa + Cfg::kStageA + (t0 * Cfg::kLevelRows / 8) * 128,
                                                     16u * Cfg::kTallRows, 128u);
            lio::umma::mma_i8(tbase + (uint32_t)((s + t0) * Cfg::kLevelRows), ad, bd,
                              lio::umma::idesc_i8(kFkRows, nl * Cfg::kLevelRows), (st > 0 || s > 0) ? 1u : 0u);
          }
        }
        lio::umma::commit(&empty[buf]);
      }
      lio::umma::commit(&done);
    }
  } else {
    // ---- B slicers: stage st holds points 32 st .. 32 st + 31 of the group
    {
      // lane = (row r8 of the warp's 8 rows, point group q): warp w takes rows 8 (w % 4) .. + 7
      // and PPT points per lane (pb ..), every spin from one read of F. Reads of F (16 bytes
      // per lane, rows 1040 bytes apart) and the digit stores (8 rows x 16 bytes of one core
      // matrix per instruction) are free of bank conflicts.
      constexpr int PPT = 8 / NS;
      const int r8 = lane & 7, q = lane >> 3;
      const int row = 8 * (warp & 3) + r8;
      const int pb = 4 * PPT * (warp >> 2) + PPT * q;  // first point of the lane within a K step
      const int j = J * kFkCols + row;
      const bool valid = j < G.m;  // rows past m are zeros (the ring holds stale rows there)
      RadialRow rr{};
      if (RAD && valid) {
        rr.load(rs, G, j);
        rr.sh -= rs.fn_sh[G.fn_off + J * kFkCols];  // its radial row in the ring slot
      }
      double s42[NS];
#pragma unroll
      for (int sp = 0; sp < NS; sp++)
        s42[sp] = valid ? digit_scale((sp == 0 ? bexp_a : bexp_b)[G.fbe_off + j]) : 1.0;
      // two K steps per iteration (nsteps is a multiple of 4, so both lie in one 128-point
      // tile): their independent digit work interleaves, which a warp needs to keep up with
      // the MMAs
      constexpr int SU = 2;
      for (int st = 0; st < nsteps; st += SU) {
        const int T = st >> 2, sub = st & 3, c = T & 1;
        bool ok = !*vfail;
        if (ok && sub == 0) ok = lio::umma::mbar_wait(&cfull[c], (T >> 1) & 1);
#pragma unroll
        for (int u = 0; u < SU; u++) {
          const int use = (st + u) / kFkStages;
          if (ok && use > 0) ok = lio::umma::mbar_wait(&empty[(st + u) % kFkStages], (use - 1) & 1);
        }
        if (!__all_sync(0xffffffffu, ok)) {
          *vfail = 1;
          break;
        }
        const uint8_t* slot = ring + c * Cfg::kSlot;
        uint32_t lo[SU][NS][PPT], hi[SU][NS][PPT];
#pragma unroll
        for (int u = 0; u < SU; u++) {
          const double* Fr =
              reinterpret_cast<const double*>(slot + (RAD ? rr.sh : row) * Cfg::kRowBytes) + (sub + u) * 32 + pb;
          const double* fr = reinterpret_cast<const double*>(slot + Cfg::kFac) + (sub + u) * 32 + pb;
          const double* xr = reinterpret_cast<const double*>(slot + Cfg::kXyz) + (sub + u) * 32 + pb;
#pragma unroll
          for (int k = 0; k < PPT; k += 2) {
            double2 v = *reinterpret_cast<const double2*>(Fr + k);
            if constexpr (RAD) {  // Fr holds the radial sums t: F = monomial x t
              const double2 x = *reinterpret_cast<const double2*>(xr + k);
              const double2 y = *reinterpret_cast<const double2*>(xr + kTcPoints + k);
              const double2 z = *reinterpret_cast<const double2*>(xr + 2 * kTcPoints + k);
              v = make_double2(rr.value(x.x, y.x, z.x, v.x), rr.value(x.y, y.y, z.y, v.y));
            }
#pragma unroll
            for (int sp = 0; sp < NS; sp++) {
              const double2 f = *reinterpret_cast<const double2*>(fr + sp * kTcPoints + k);
              digits_m(valid ? v.x * f.x : 0.0, s42[sp], lo[u][sp][k], hi[u][sp][k]);
              digits_m(valid ? v.y * f.y : 0.0, s42[sp], lo[u][sp][k + 1], hi[u][sp][k + 1]);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < SU; u++) {
          uint8_t* bst = fk_smem + ((st + u) % kFkStages) * Cfg::kStage + Cfg::kStageA;
#pragma unroll
          for (int sp = 0; sp < NS; sp++)
#pragma unroll
            for (int s = 0; s < kSlices; s++) {
              uint32_t w[PPT / 4];
#pragma unroll
              for (int h = 0; h < PPT / 4; h++)
                w[h] = pack_digits(digit_field(lo[u][sp][4 * h], hi[u][sp][4 * h], s),
                                   digit_field(lo[u][sp][4 * h + 1], hi[u][sp][4 * h + 1], s),
                                   digit_field(lo[u][sp][4 * h + 2], hi[u][sp][4 * h + 2], s),
                                   digit_field(lo[u][sp][4 * h + 3], hi[u][sp][4 * h + 3], s), s == 0);
              uint8_t* dst =
                  bst + lio::umma::kmajor_offset(s * Cfg::kLevelRows + sp * kFkCols + row, pb, Cfg::kTallRows);
              if (PPT == 8)
                *reinterpret_cast<uint2*>(dst) = make_uint2(w[0], w[PPT / 4 - 1]);
              else
                *reinterpret_cast<uint32_t*>(dst) = w[0];
            }
        }
        // generic-proxy stores -> visible to the MMAs (async proxy) once bready completes
        lio::umma::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
#pragma unroll
          for (int u = 0; u < SU; u++) lio::umma::mbar_arrive(&bready[(st + u) % kFkStages]);
          if (sub + SU - 1 == 3) lio::umma::mbar_arrive(&cempty[c]);
        }
      }
    }
  }
  if (warp < 4) {
    // ---- epilogue
    const int rrow = warp * 32 + lane;  // TMEM lane
    const int i = I * kFkRows + rrow;
    const bool ok = lio::umma::mbar_wait(&done, 0) && !*vfail;
    lio::umma::fence_after_sync();
    if (!ok) *vfail = 1;
    if (ok) {
      const int gi = i < G.m ? fn_glob[G.fn_off + i] : 0;
      const int ea = i < G.m ? aexp[G.fae_off + i] : 0;
      const uint32_t lane_base = tbase + ((uint32_t)(warp * 32) << 16);
      for (int sp = 0; sp < NS; sp++) {
        const int16_t* bexp = sp == 0 ? bexp_a : bexp_b;
        double* K = sp == 0 ? K_a : K_b;
        for (int c0 = 0; c0 < kFkCols; c0 += 8) {
          int32_t lv[kSlices][8];
#pragma unroll
          for (int l = 0; l < kSlices; l++)
            lio::umma::tmem_ld8(lane_base + (uint32_t)((l * NS + sp) * kFkCols + c0), lv[l]);
          lio::umma::tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 8; c++) {
            const int j = J * kFkCols + c0 + c;
            if (i >= G.m || j >= G.m || i > j) continue;
            // each level converted on its own (the reduction runs over all the
            // group's points, so level pairs need not fit int32), one rounding
            const double v = level_sum(lv, c, false) * pow2(ea + bexp[G.fbe_off + j] - 7 * (kSlices + 1));
            atomicAdd(K + G.pk_off + packed_index(gi, fn_glob[G.fn_off + j], G.pk_M), v);
          }
        }
      }
    }
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  if (tid == 0 && fail) atomicExch(err, 1);
  if (warp == 0) lio::umma::tmem_dealloc(tbase, Cfg::kTmem);
}
