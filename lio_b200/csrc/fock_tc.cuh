// Tensor-core form of the Kohn-Sham contraction (included by engine.cu inside
// its anonymous namespace, after density_tc.cuh).
//
// K_ij = sum_p F_ip f_p F_jp (i <= j) per spin, as C = A . B^T with the points
// as the reduction dimension:
//   A_ip = F_ip          = 2^(a_i) sum_s a_s[i][p] 128^-(s+1)  (per geometry, per function row)
//   B_jp = f_p F_jp      = 2^(b_j) sum_t b_t[j][p] 128^-(t+1)  (per solve and spin, per row)
// with the same int8 slices, level accumulators and exact int64 level sum as
// the density contraction. A tile is 128 functions (i) x 32 functions (j);
// both spins share the A slices and keep 2 x S level accumulators in TMEM.
#pragma once

constexpr int kFkRows = 128;  // UMMA M: functions i per tile
constexpr int kFkCols = 32;   // UMMA N: functions j per tile
constexpr int kFkStages = 4;
constexpr int kFkSliceA = 32 * kFkRows;  // bytes of one A slice per 32-point K step
constexpr int kFkSliceB = 32 * kFkCols;
template <int NS>
struct FkCfg {
  static constexpr int kStageA = kSlices * kFkSliceA;
  static constexpr int kStage = kStageA + NS * kSlices * kFkSliceB;
  static constexpr size_t kSmem = (size_t)kFkStages * kStage;
  static constexpr uint32_t kCols = NS * kSlices * kFkCols;
  static constexpr uint32_t kTmem = kCols <= 256 ? 256 : 512;
  static constexpr int kThreads = 32 * 6;  // 4 epilogue warps, producer, MMA issuer
};

// One warp per (group, row) of a padded slice block: the row's exponent from
// max_p |v_p| (v = F_rp, times fac_p when fac != nullptr), then its S slices,
// in the K-major interleaved layout of an R-row block (R = kFkRows for A,
// kFkCols for B). Rows at or beyond m are written as zeros.
template <int R>
__global__ void k_slice_fock(const int2* __restrict__ rows, int nrows, const GroupDev* __restrict__ groups,
                             const double* __restrict__ basis, const double* __restrict__ fac,
                             int8_t* __restrict__ slices, int16_t* __restrict__ expo, int use_sl_b) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nrows) return;  // whole warps only
  const int2 t = rows[warp];
  const GroupDev G = groups[t.x];
  const int i = t.y;
  const bool valid = i < G.m;
  const double* Fi = basis + G.bas_off + (long long)(valid ? i : 0) * G.ldp;
  double amax = 0.0;
  if (valid)
    for (int p = lane; p < G.ldp; p += 32) {
      double v = Fi[p];
      if (fac) v *= fac[G.pt_off + p];
      amax = fmax(amax, fabs(v));
    }
  for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  const int e = slice_exponent(amax);
  const long long base = use_sl_b ? G.fb_off : G.fa_off;
  const long long ebase = use_sl_b ? G.fbe_off : G.fae_off;
  if (lane == 0) expo[ebase + i] = (int16_t)e;
  const int tile = i / R, r = i % R;
  int8_t* dst = slices + base + (long long)tile * kSlices * R * G.ldp;
  for (int p = lane; p < G.ldp; p += 32) {
    double x = 0.0;
    if (valid) {
      double v = Fi[p];
      if (fac) v *= fac[G.pt_off + p];
      x = ldexp(v, -e);
    }
    const uint32_t off = lio::umma::kmajor_offset(r, p, R);
    for (int s = 0; s < kSlices; s++) {
      x *= 128.0;
      const double d = rint(x);
      x -= d;
      dst[(long long)s * R * G.ldp + off] = (int8_t)d;
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
      const int8_t* A = aslices + G.fa_off + (long long)I * kSlices * kFkRows * G.ldp;
      const int8_t* Ba = bslices_a + G.fb_off + (long long)J * kSlices * kFkCols * G.ldp;
      const int8_t* Bb = NS == 2 ? bslices_b + G.fb_off + (long long)J * kSlices * kFkCols * G.ldp : nullptr;
      for (int st = 0; st < nsteps; st++) {
        const int buf = st % kFkStages, use = st / kFkStages;
        if (use > 0 && !lio::umma::mbar_wait(&empty[buf], (use - 1) & 1)) {
          fail = 1;
          break;
        }
        uint8_t* stage = fk_smem + buf * Cfg::kStage;
        lio::umma::mbar_expect_tx(&full[buf], (uint32_t)Cfg::kStage);
        for (int s = 0; s < kSlices; s++)
          lio::umma::bulk_copy_g2s(stage + s * kFkSliceA, A + (long long)s * kFkRows * G.ldp + st * kFkSliceA,
                                   kFkSliceA, &full[buf]);
        for (int sp = 0; sp < NS; sp++) {
          const int8_t* B = sp == 0 ? Ba : Bb;
          for (int s = 0; s < kSlices; s++)
            lio::umma::bulk_copy_g2s(stage + Cfg::kStageA + (sp * kSlices + s) * kFkSliceB,
                                     B + (long long)s * kFkCols * G.ldp + st * kFkSliceB, kFkSliceB, &full[buf]);
        }
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      const uint32_t idesc = lio::umma::idesc_i8(kFkRows, kFkCols);
      const uint32_t smem0 = lio::umma::smem_u32(fk_smem);
      for (int st = 0; st < nsteps; st++) {
        const int buf = st % kFkStages, use = st / kFkStages;
        if (!lio::umma::mbar_wait(&full[buf], use & 1)) {
          fail = 1;
          break;
        }
        lio::umma::fence_after_sync();
        const uint64_t ad0 = lio::umma::smem_desc(smem0 + buf * Cfg::kStage, 16u * kFkRows, 128u);
        const uint64_t bd0 = lio::umma::smem_desc(smem0 + buf * Cfg::kStage + Cfg::kStageA, 16u * kFkCols, 128u);
        const uint32_t keep = st > 0 ? 1u : 0u;
#pragma unroll
        for (int sp = 0; sp < NS; sp++)
#pragma unroll
          for (int l = 0; l < kSlices; l++)
#pragma unroll
            for (int s = 0; s <= l; s++)
              lio::umma::mma_i8(tbase + (uint32_t)((sp * kSlices + l) * kFkCols),
                                ad0 + (uint64_t)((s * kFkSliceA) >> 4),
                                bd0 + (uint64_t)(((sp * kSlices + l - s) * kFkSliceB) >> 4), idesc,
                                s > 0 ? 1u : keep);
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
            long long V = 0;
#pragma unroll
            for (int l = 0; l < kSlices; l += 2) V = V * (1LL << 14) + (long long)(lv[l][c] * 128 + lv[l + 1][c]);
            const double v = (double)V * pow2(ea + bexp[G.fbe_off + j] - 7 * (kSlices + 1));
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
