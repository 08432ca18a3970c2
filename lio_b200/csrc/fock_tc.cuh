// Tensor-core form of the Kohn-Sham contraction (included by engine.cu inside
// its anonymous namespace, after density_tc.cuh).
//
// K_ij = sum_p F_ip f_p F_jp (i <= j) per spin, as C = A . B^T with the points
// as the reduction dimension:
//   A_ip = F_ip          = 2^(a_i) sum_s a_s[i][p] 128^-(s+1)  (per geometry, per function row)
//   B_jp = f_p F_jp      = 2^(b_j) sum_t b_t[j][p] 128^-(t+1)  (per solve and spin, per row)
// with the same int8 slices, level accumulators and level sum as the density
// contraction. A tile is 128 functions (i) x 32 functions (j); the S slices
// of a B tile are stacked along N (row t * 32 + j holds b_t[j]), so one MMA per
// A slice s (N = (S - s) * 32) lands every product (s, t) on level s + t.
// Both spins share the A slices and keep 2 x S level blocks in TMEM.
#pragma once

constexpr int kFkRows = 128;  // UMMA M: functions i per tile
constexpr int kFkCols = 32;   // functions j per tile (output columns per level)
constexpr int kFkTall = kSlices * kFkCols;  // rows of the stacked B operand
constexpr int kFkStages = 4;
constexpr int kFkSliceA = 32 * kFkRows;       // bytes of one A slice per 32-point K step
constexpr int kFkStepA = kSlices * kFkSliceA;  // all A slices of a K step (contiguous)
constexpr int kFkStepB = 32 * kFkTall;         // one spin's stacked B slices of a K step (contiguous)
template <int NS>
struct FkCfg {
  static constexpr int kStageA = kFkStepA;
  static constexpr int kStage = kStageA + NS * kFkStepB;
  static constexpr size_t kSmem = (size_t)kFkStages * kStage;
  static constexpr uint32_t kCols = NS * kSlices * kFkCols;
  static constexpr uint32_t kTmem = kCols <= 256 ? 256 : 512;
  static constexpr int kThreads = 32 * 6;  // 4 epilogue warps, producer, MMA issuer
};

// Slices of the rows of v = F (A operand, per geometry) or v = f_s F (B
// operand, per solve, both spins at once), in two passes over the FP64 basis.
//
// F(i, p) of a group and the values after it up to the end of its 128-point
// tile: from the function-major basis cache (nkb = 0) or from the blocked copy
// of the tensor-core density (nkb = its number of kinds; kind 0 is F)
__device__ __forceinline__ const double* f_row(const GroupDev& G, const double* basis, int i, int p, int nkb) {
  if (nkb == 0) return basis + G.bas_off + (long long)i * G.ldp + p;
  return basis + G.bb_off + (long long)((p >> 7) * G.nftc + (i >> 5)) * nkb * kTcChunk + (i & 31) * kTcPoints +
         (p & 127);
}

// Pass 1, one warp per (group, row): the row's exponent per spin from
// max_p |v_p|. Rows at or beyond m get exponent 0 (their slices are zeros).
// The row is read a 128-point tile at a time, four consecutive points per lane
// (two 16-byte loads of F and of each spin's factors), two tiles in flight.
static_assert(kPointPad % kTcPoints == 0, "rows are read in whole 128-point tiles");
template <int NS>
__global__ void k_fock_rowexp(const int2* __restrict__ rows, int nrows, const GroupDev* __restrict__ groups,
                              const double* __restrict__ basis, const double* __restrict__ fac_a,
                              const double* __restrict__ fac_b, int16_t* __restrict__ expo_a,
                              int16_t* __restrict__ expo_b, int use_sl_b, int nkb) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nrows) return;  // whole warps only
  const int2 t = rows[warp];
  const GroupDev& G = groups[t.x];
  const int i = t.y, ntl = G.ldp / kTcPoints;
  double amax[NS];
#pragma unroll
  for (int sp = 0; sp < NS; sp++) amax[sp] = 0.0;
  if (i < G.m) {
#pragma unroll 2
    for (int T = 0; T < ntl; T++) {
      const int p = T * kTcPoints + lane * 4;
      const double* Fi = f_row(G, basis, i, p, nkb);
      const double2 v01 = *reinterpret_cast<const double2*>(Fi);
      const double2 v23 = *reinterpret_cast<const double2*>(Fi + 2);
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

// Pass 2, a CTA per 32-row piece of a row tile (lane = row), each warp taking
// 16-point blocks: per spin and slice one 16-byte store. Layout per row tile
// (R rows) and 32-point K step: A (TALL = false): the S slices one after the
// other, each an R-row x 32-byte K-major block; B (TALL = true): one
// (S * R)-row x 32-byte block whose row t * R + r holds slice t of row r.
template <int R, bool TALL, int NS>
__global__ void __launch_bounds__(256) k_fock_slices(const int2* __restrict__ rtiles, const GroupDev* __restrict__ groups,
                                                     const double* __restrict__ basis,
                                                     const double* __restrict__ fac_a,
                                                     const double* __restrict__ fac_b,
                                                     const int16_t* __restrict__ expo_a,
                                                     const int16_t* __restrict__ expo_b, int8_t* __restrict__ sl_a,
                                                     int8_t* __restrict__ sl_b, int use_sl_b, int nkb) {
  constexpr int kStep = kSlices * 32 * R;  // bytes of one K step of a row tile (either layout)
  const int2 t = rtiles[blockIdx.x];
  const GroupDev& G = groups[t.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = t.y + lane, ldp = G.ldp, nkp = ldp / 32;
  const bool valid = i < G.m;
  const long long base = use_sl_b ? G.fb_off : G.fa_off;
  const long long ebase = use_sl_b ? G.fbe_off : G.fae_off;
  double sc[NS];
#pragma unroll
  for (int sp = 0; sp < NS; sp++) sc[sp] = pow2(-(int)(sp == 0 ? expo_a : expo_b)[ebase + i]);
  const int tile = i / R, r = i % R;
  for (int b = warp; b < ldp / 16; b += blockDim.x / 32) {
    const int p0 = b * 16;
    const double* Fi = f_row(G, basis, valid ? i : 0, p0, nkb);  // 16 values within one 128-point tile
    double F[16];
#pragma unroll
    for (int k = 0; k < 16; k += 2) {
      const double2 v = valid ? *reinterpret_cast<const double2*>(Fi + k) : make_double2(0.0, 0.0);
      F[k] = v.x;
      F[k + 1] = v.y;
    }
#pragma unroll
    for (int sp = 0; sp < NS; sp++) {
      const double* fac = sp == 0 ? fac_a : fac_b;
      int8_t* blk = (sp == 0 ? sl_a : sl_b) + base + ((long long)tile * nkp + (p0 >> 5)) * kStep;
      double x[16];
#pragma unroll
      for (int k = 0; k < 16; k++) x[k] = (fac ? F[k] * fac[G.pt_off + p0 + k] : F[k]) * sc[sp];
#pragma unroll
      for (int s = 0; s < kSlices; s++) {
        uint32_t w[4];
#pragma unroll
        for (int k4 = 0; k4 < 4; k4++) {
          uint32_t packed = 0;
#pragma unroll
          for (int k = 0; k < 4; k++) packed |= ((uint32_t)(uint8_t)next_digit(x[k4 * 4 + k])) << (8 * k);
          w[k4] = packed;
        }
        const uint32_t off = TALL ? lio::umma::kmajor_offset(s * R + r, p0 & 31, kSlices * R)
                                  : s * 32 * R + lio::umma::kmajor_offset(r, p0 & 31, R);
        *reinterpret_cast<uint4*>(blk + off) = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
  }
}

// CTA = (group, 128-row tile I, 32-column tile J) with some j >= some i.
// Warps 0-3: epilogue (TMEM lane = row i); warp 4: producer (bulk copies of
// one 32-point K step per stage, four-stage ring); warp 5: MMA issuer. After
// the last K step the epilogue combines the levels of each (i, j <= ...) and
// adds K_ij into the packed accumulator(s) with FP64 atomics.
template <int NS>
__global__ void __launch_bounds__(FkCfg<NS>::kThreads, 1)
    k_fock_tc(const int4* __restrict__ tiles, const GroupDev* __restrict__ groups, const int* __restrict__ fn_glob,
              const int8_t* __restrict__ aslices, const int16_t* __restrict__ aexp,
              const int8_t* __restrict__ bslices_a, const int16_t* __restrict__ bexp_a,
              const int8_t* __restrict__ bslices_b, const int16_t* __restrict__ bexp_b, int M,
              double* __restrict__ K_a, double* __restrict__ K_b, int* __restrict__ err) {
  using Cfg = FkCfg<NS>;
  extern __shared__ __align__(128) uint8_t fk_smem[];
  __shared__ uint64_t full[kFkStages], empty[kFkStages], done;
  __shared__ uint32_t tmem_base;
  __shared__ int fail;
  const int4 t = tiles[blockIdx.x];
  const GroupDev G = groups[t.x];
  const int I = t.y, J = t.z;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nsteps = G.ldp / 32;
  if (warp == 0) lio::umma::tmem_alloc(&tmem_base, Cfg::kTmem);
  if (tid == 0) {
    for (int s = 0; s < kFkStages; s++) {
      lio::umma::mbar_init(&full[s], 1);
      lio::umma::mbar_init(&empty[s], 1);
    }
    lio::umma::mbar_init(&done, 1);
    lio::umma::fence_mbar_init();
    fail = 0;
  }
  lio::umma::fence_before_sync();
  __syncthreads();
  lio::umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (warp == 4) {
    if (lane == 0) {
      const int8_t* A = aslices + G.fa_off + (long long)I * nsteps * kFkStepA;
      const int8_t* Ba = bslices_a + G.fb_off + (long long)J * nsteps * kFkStepB;
      const int8_t* Bb = NS == 2 ? bslices_b + G.fb_off + (long long)J * nsteps * kFkStepB : nullptr;
      for (int st = 0; st < nsteps; st++) {
        const int buf = st % kFkStages, use = st / kFkStages;
        if (use > 0 && !lio::umma::mbar_wait(&empty[buf], (use - 1) & 1)) {
          fail = 1;
          break;
        }
        uint8_t* stage = fk_smem + buf * Cfg::kStage;
        lio::umma::mbar_expect_tx(&full[buf], (uint32_t)Cfg::kStage);
        lio::umma::bulk_copy_g2s(stage, A + (long long)st * kFkStepA, kFkStepA, &full[buf]);
        for (int sp = 0; sp < NS; sp++)
          lio::umma::bulk_copy_g2s(stage + Cfg::kStageA + sp * kFkStepB, (sp == 0 ? Ba : Bb) + (long long)st * kFkStepB,
                                   kFkStepB, &full[buf]);
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      const uint32_t smem0 = lio::umma::smem_u32(fk_smem);
      for (int st = 0; st < nsteps; st++) {
        const int buf = st % kFkStages, use = st / kFkStages;
        if (!lio::umma::mbar_wait(&full[buf], use & 1)) {
          fail = 1;
          break;
        }
        lio::umma::fence_after_sync();
        const uint32_t sa = smem0 + buf * Cfg::kStage;
#pragma unroll
        for (int sp = 0; sp < NS; sp++) {
          // stacked B of this spin: K-major, 192 rows (LBO = 16 * 192 bytes between K halves)
          const uint64_t bd = lio::umma::smem_desc(sa + Cfg::kStageA + sp * kFkStepB, 16u * kFkTall, 128u);
#pragma unroll
          for (int s = 0; s < kSlices; s++)
            lio::umma::mma_i8(tbase + (uint32_t)((sp * kSlices + s) * kFkCols),
                              lio::umma::smem_desc(sa + s * kFkSliceA, 16u * kFkRows, 128u), bd,
                              lio::umma::idesc_i8(kFkRows, (kSlices - s) * kFkCols), (st > 0 || s > 0) ? 1u : 0u);
        }
        lio::umma::commit(&empty[buf]);
      }
      lio::umma::commit(&done);
    }
  } else {
    const int rrow = warp * 32 + lane;  // TMEM lane
    const int i = I * kFkRows + rrow;
    const bool ok = lio::umma::mbar_wait(&done, 0);
    lio::umma::fence_after_sync();
    if (!ok) fail = 1;
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
            lio::umma::tmem_ld8(lane_base + (uint32_t)((sp * kSlices + l) * kFkCols + c0), lv[l]);
          lio::umma::tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 8; c++) {
            const int j = J * kFkCols + c0 + c;
            if (i >= G.m || j >= G.m || i > j) continue;
            // each level converted on its own (the reduction runs over all the
            // group's points, so level pairs need not fit int32), one rounding
            const double v = level_sum(lv, c, false) * pow2(ea + bexp[G.fbe_off + j] - 7 * (kSlices + 1));
            atomicAdd(K + packed_index(gi, fn_glob[G.fn_off + j], M), v);
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
