// Tensor-core form of the XC nuclear forces (included by engine.cu inside its
// anonymous namespace, after density_tc.cuh).
//
// The reference's force loop (g2g/cpu/iteration.cpp:213-267, open shell
// 496-563) gives atom A, per spin,
//   F_A = -2 sum_p f_p sum_(i on A) G_i(p) grad F_i(p),   G_i(p) = sum_j P_ij F_j(p),
// with f_p = w_p v_xc(p) the factors of the build. G is the density
// contraction's F unit: the int8 Ozaki slices of F (A operand, per geometry)
// against the stacked slices of P (per solve and spin), both still resident
// after the build, so one unit of k_density_tc's MMAs per (128-point tile,
// 32-function tile, spin) gives G exactly as the density saw it. The epilogue
// forms f_p G_i(p) grad F_i(p) with the gradient chunks of the blocked basis
// and sums it over the tile's points per function; the sums go to the atoms
// with FP64 atomics.
//
// Unit = (group, point tile T, function tile ft, spin); persistent CTAs (two
// per SM) take units w, w + gridDim.x, ... Warps 0-3 epilogue (TMEM lane
// quadrant = 32 points each), warp 4 producer (bulk copies of one 32-function
// K step per stage: the F slices and the spin's stacked D slices, running
// ahead across units), warp 5 MMA issuer (S MMAs per K step into S x 32 level
// columns). One unit's levels take 192 TMEM columns; the epilogue hands them
// back (tempty) as soon as G is in registers, so the next unit's MMAs overlap
// its gradient dots. Every wait is bounded; a timeout sets the error flag and
// the CTA drains its copies and MMAs before it frees TMEM.
#pragma once

constexpr int kFtStages = 3;
struct FtCfg {
  static constexpr int kStage = kTcStepA + kTcStepD;  // F slices of a K step + one spin's stacked D slices
  static constexpr size_t kSmem = (size_t)kFtStages * kStage;
  static constexpr uint32_t kTmem = 256;  // S x 32 = 192 level columns
  static constexpr int kThreads = 32 * 6;
};

// Sums v[c][a] (8 columns x 3 axes, one value per lane) over the warp's 32
// lanes; lane c (0 <= c < 8) returns the sums of column c. Three halving
// exchange steps leave column (lane & 7) in each lane, two butterflies finish.
__device__ __forceinline__ void warp_column_sums(double (&v)[8][3], int lane, double (&out)[3]) {
#pragma unroll
  for (int a = 0; a < 3; a++) {
    double x4[4], x2[2];
#pragma unroll
    for (int j = 0; j < 4; j++) {  // step 4: keep columns with bit 2 equal to the lane's
      const bool hi = lane & 4;
      const double send = hi ? v[j][a] : v[j + 4][a], keep = hi ? v[j + 4][a] : v[j][a];
      x4[j] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {  // step 2
      const bool hi = lane & 2;
      const double send = hi ? x4[j] : x4[j + 2], keep = hi ? x4[j + 2] : x4[j];
      x2[j] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    const bool hi = lane & 1;  // step 1
    const double send = hi ? x2[0] : x2[1], keep = hi ? x2[1] : x2[0];
    double x = keep + __shfl_xor_sync(0xffffffffu, send, 1);
    x += __shfl_xor_sync(0xffffffffu, x, 8);
    x += __shfl_xor_sync(0xffffffffu, x, 16);
    out[a] = x;
  }
}

// named barrier over the four epilogue warps; returns the OR of `pred` over them
__device__ __forceinline__ bool ft_epi_sync_or(bool pred) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(out)
      : "r"((uint32_t)pred)
      : "memory");
  return out != 0;
}

__global__ void __launch_bounds__(FtCfg::kThreads, 2)
    k_force_tc(const int4* __restrict__ tiles, int ntiles, const GroupDev* __restrict__ groups, const int NA,
               const int8_t* __restrict__ aslices, const int16_t* __restrict__ aexp,
               const int8_t* __restrict__ dsl_a, const int16_t* __restrict__ dexp_a,
               const int8_t* __restrict__ dsl_b, const int16_t* __restrict__ dexp_b,
               const double* __restrict__ bblk, int nkb, const double* __restrict__ fac_a,
               const double* __restrict__ fac_b, const int* __restrict__ fn_atom, double* __restrict__ force,
               int* __restrict__ err) {
  extern __shared__ __align__(128) uint8_t ft_smem[];
  __shared__ uint64_t full[kFtStages], empty[kFtStages], tfull, tempty, drain;
  __shared__ uint32_t tmem_base;
  __shared__ int fail, consumed;
  __shared__ double part[4][kTcFuncs][3];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) lio::umma::tmem_alloc(&tmem_base, FtCfg::kTmem);
  if (tid == 0) {
    for (int s = 0; s < kFtStages; s++) {
      lio::umma::mbar_init(&full[s], 1);
      lio::umma::mbar_init(&empty[s], 1);
    }
    lio::umma::mbar_init(&tfull, 1);
    lio::umma::mbar_init(&tempty, 4);  // one arrival per epilogue warp
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
  int issued = 0;
  if (warp == 4) {
    if (lane == 0) {
      int cnt = 0;
      for (int w = blockIdx.x; w < ntiles && !*vfail; w += gridDim.x) {
        const int4 t = tiles[w];
        const GroupDev& G = groups[t.x];
        const int nks = G.m32 / 32;
        const int8_t* A = aslices + G.sl_off + (long long)t.y * NA * nks * kTcStepA;  // kind F: the first of NA
        const int8_t* D = (t.w == 0 ? dsl_a : dsl_b) + G.ds_off + (long long)t.z * nks * kTcStepD;
        {  // the unit's gradient chunks (its existing function rows) into L2 for the epilogue's loads
          const double* gch = bblk + G.bb_off + ((long long)(t.y * G.nftc + t.z) * nkb + 1) * kTcChunk;
          const uint32_t bytes = (uint32_t)min(kTcFuncs, G.m - t.z * kTcFuncs) * kTcPoints * 8;
          for (int a = 0; a < 3; a++) lio::umma::bulk_prefetch_l2(gch + (long long)a * kTcChunk, bytes);
        }
        for (int kk = 0; kk < nks; kk++, cnt++) {
          const int buf = cnt % kFtStages, use = cnt / kFtStages;
          if (use > 0 && (*vfail || !lio::umma::mbar_wait(&empty[buf], (use - 1) & 1))) {
            *vfail = 1;
            break;
          }
          uint8_t* stage = ft_smem + buf * FtCfg::kStage;
          lio::umma::mbar_expect_tx(&full[buf], (uint32_t)FtCfg::kStage);
          lio::umma::bulk_copy_g2s(stage, A + (long long)kk * kTcStepA, kTcStepA, &full[buf]);
          lio::umma::bulk_copy_g2s(stage + kTcStepA, D + (long long)kk * kTcStepD, kTcStepD, &full[buf]);
          issued = cnt + 1;
        }
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      const uint32_t smem0 = lio::umma::smem_u32(ft_smem);
      int cnt = 0, ucnt = 0;
      bool stop = false;
      for (int w = blockIdx.x; w < ntiles && !stop; w += gridDim.x, ucnt++) {
        const GroupDev& G = groups[tiles[w].x];
        const int nks = G.m32 / 32;
        // the previous unit's levels must have been read out of TMEM
        if (ucnt > 0 && (*vfail || !lio::umma::mbar_wait(&tempty, (ucnt - 1) & 1))) {
          stop = true;
          break;
        }
        lio::umma::fence_after_sync();
        for (int kk = 0; kk < nks; kk++, cnt++) {
          const int buf = cnt % kFtStages, use = cnt / kFtStages;
          if (*vfail || !lio::umma::mbar_wait(&full[buf], use & 1)) {
            stop = true;
            break;
          }
          consumed = cnt + 1;
          lio::umma::fence_after_sync();
          const uint32_t sa = smem0 + buf * FtCfg::kStage;
          // stacked D: K-major, 192 rows (LBO = 16 * 192 bytes between K halves)
          const uint64_t bd = lio::umma::smem_desc(sa + kTcStepA, 16u * kTcTall, 128u);
#pragma unroll
          for (int s = 0; s < kSlices; s++)
            lio::umma::mma_i8(tbase + (uint32_t)(s * kTcFuncs),
                              lio::umma::smem_desc(sa + s * kTcSliceA, 16u * kTcPoints, 128u), bd,
                              lio::umma::idesc_i8(kTcPoints, (kSlices - s) * kTcFuncs), (kk > 0 || s > 0) ? 1u : 0u);
          lio::umma::commit(&empty[buf]);
          if (kk == nks - 1) lio::umma::commit(&tfull);
        }
      }
      if (stop) *vfail = 1;
      // every MMA issued so far has completed once this arrives
      lio::umma::commit(&drain);
      if (!lio::umma::mbar_wait(&drain, 0)) *vfail = 1;
    }
  } else {
    const int row = warp * 32 + lane;  // TMEM lane = point of the tile
    const uint32_t lane_base = tbase + ((uint32_t)(warp * 32) << 16);
    int ucnt = 0;
    for (int w = blockIdx.x; w < ntiles; w += gridDim.x, ucnt++) {
      const int4 t = tiles[w];
      const GroupDev& G = groups[t.x];
      const int T = t.y, ft = t.z, sp = t.w;
      const int p = T * kTcPoints + row;
      const bool ok = !*vfail && lio::umma::mbar_wait(&tfull, ucnt & 1);
      // one decision for all four warps (the TMEM loads are warp-collective and
      // the warps meet at named barriers below)
      if (ft_epi_sync_or(!ok)) {
        *vfail = 1;
        break;
      }
      lio::umma::fence_after_sync();
      // G_i(p) = acc * 2^(e_p + f_T - 7(S+1)), f_T the exponent of the density
      // tile (one per 32 functions; columns past m have no slices, acc = 0); the
      // factor f_p joins the point scale
      const int16_t* dexp = sp == 0 ? dexp_a : dexp_b;
      const double fp = (sp == 0 ? fac_a : fac_b)[G.pt_off + p];
      const double spx =
          fp * pow2(aexp[G.aexp_off + p] - 7 * (kSlices + 1)) * pow2(dexp[G.dexp_off + ft * kTcFuncs]);
      const bool narrow = G.m32 <= kTcNarrowK;
      double g[kTcFuncs];
#pragma unroll
      for (int h = 0; h < kTcFuncs / 8; h++) {
        int32_t lv[kSlices][8];
#pragma unroll
        for (int l = 0; l < kSlices; l++) lio::umma::tmem_ld8(lane_base + (uint32_t)(l * kTcFuncs + h * 8), lv[l]);
        lio::umma::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 8; c++) g[h * 8 + c] = level_sum(lv, c, narrow) * spx;
      }
      // levels read: the next unit's MMAs may overwrite TMEM
      lio::umma::fence_before_sync();
      __syncwarp();
      if (lane == 0) lio::umma::mbar_arrive(&tempty);
      // f_p G_i(p) grad F_i(p), summed over the warp's points per function
      const double* gch = bblk + G.bb_off + ((long long)(T * G.nftc + ft) * nkb + 1) * kTcChunk + (p & 127);
#pragma unroll
      for (int h = 0; h < kTcFuncs / 8; h++) {
        double v[8][3];
#pragma unroll
        for (int c = 0; c < 8; c++) {
          const double* gi = gch + (h * 8 + c) * kTcPoints;
#pragma unroll
          for (int a = 0; a < 3; a++) v[c][a] = g[h * 8 + c] * gi[a * kTcChunk];
        }
        double cs[3];
        warp_column_sums(v, lane, cs);
        if (lane < 8)
#pragma unroll
          for (int a = 0; a < 3; a++) part[warp][h * 8 + lane][a] = cs[a];
      }
      // the four quadrants' sums per function, then one atomic per (function, axis)
      asm volatile("bar.sync 1, 128;" ::: "memory");
      if (tid < kTcFuncs * 3) {
        const int c = tid / 3, a = tid - 3 * c, i = ft * kTcFuncs + c;
        if (i < G.m) {
          const double s = (part[0][c][a] + part[1][c][a]) + (part[2][c][a] + part[3][c][a]);
          atomicAdd(&force[fn_atom[G.fn_off + i] * 3 + a], -2.0 * s);
        }
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");  // part is free again
    }
  }
  lio::umma::fence_before_sync();
  __syncthreads();  // every role done
  if (warp == 4 && lane == 0) {
    // copies issued but never consumed (after a timeout) land before the CTA exits
    for (int k = consumed; k < issued; k++)
      if (!lio::umma::mbar_wait(&full[k % kFtStages], (k / kFtStages) & 1)) break;
  }
  __syncthreads();
  if (tid == 0 && fail) atomicExch(err, 1);
  if (warp == 0) lio::umma::tmem_dealloc(tbase, FtCfg::kTmem);
}
