// One work item of the exact pair sums: a tile of 256*R targets against a
// contiguous range of sources, summed into one partial-sum slab.  Shared by
// the single-transform kernel (pairsum.cu) and the persistent batched kernel
// (batched.cu).
//
// Sources are staged in chunks of PAIR_CH doubles: whole 16-byte-aligned
// chunks by TMA bulk copies (cp.async.bulk + mbarrier, double-buffered), tails
// by plain loads.  F64 sums every pair in FP64.  MIXED sums a 256-source
// block in FP32 on the packed f32x2 pipe (pairs32x4) when the block lies at
// least near_dist from all of the warp's targets, and everything else in
// FP64; FP32 partials are folded into FP64 every PAIR_FOLD sources.
#pragma once

#include "common.cuh"
#include "pairs.cuh"

namespace shrk {

constexpr int PAIR_NT = 256;    // threads per CTA
constexpr int PAIR_CH = 1024;   // sources per staged chunk
constexpr int PAIR_FOLD = 16;   // sources per FP32 partial before the FP64 fold

// Shared memory of one CTA.
struct __align__(16) PairStage {
  double sbuf[2][PAIR_CH];      // staged source chunks
  float4 sm4[PAIR_CH / 2];      // MIXED: {SM, SM, DL, DL} per source pair
  uint64_t bar[2];              // one mbarrier per buffer
};

struct PairItem {
  const double* tgt;        // targets
  int64_t nt;
  const double* src;        // sources; SUB-block b of the bounds starts at src[b*SUB]
  int64_t s0, s1;           // source range of this item (s0 a multiple of PAIR_CH)
  int64_t tile0;            // first target of the tile
  double eta;
  double near_dist;         // MIXED: minimal gap of an FP32 block
  const double2* bounds;    // MIXED: (min, max) per SUB-block of src
  double* out_re;           // partial slab, indexed by target
  double* out_im;
  int* err;
  bool use_tma;             // src + s0 is 16-byte aligned
  long long wait_cycles;    // budget of each bulk-copy wait (clock cycles)
};

__device__ __forceinline__ void pair_stage_init(PairStage& st) {
  if (threadIdx.x == 0) {
    mbar_init(&st.bar[0], 1);
    mbar_init(&st.bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
}

// Sums one item.  phase / pending carry the mbarrier state across items.
// Returns false (uniformly across the CTA, after recording DEV_ERR_TIMEOUT
// and draining its own bulk copies) if a bulk copy never completed.
template <bool MIXED, int R>
__device__ __forceinline__ bool pair_item(const PairItem& a, PairStage& st, uint32_t& phase,
                                          uint32_t& pending) {
  constexpr int NT = PAIR_NT, CH = PAIR_CH, FOLD = PAIR_FOLD;
  static_assert(!MIXED || R % 2 == 0, "the packed far field takes targets in pairs");
  constexpr int WT = 32 * R, R2 = R / 2 > 0 ? R / 2 : 1;  // R2: packed pairs (MIXED only)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double eta = a.eta, eta2 = eta * eta;
  const float eta2f = (float)eta2;
  const u64 ETA2 = pk2(eta2f, eta2f);

  const int64_t wbase = a.tile0 + (int64_t)warp * WT;
  const double x0 = a.tgt[a.tile0];
  double x[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t idx = wbase + r * 32 + lane;
    x[r] = idx < a.nt ? a.tgt[idx] : x0;
  }
  const int64_t s0 = a.s0, s1 = a.s1;
  const int nchunks = (int)((s1 - s0 + CH - 1) / CH);

  double re64[R], iv64[R];
#pragma unroll
  for (int r = 0; r < R; ++r) re64[r] = iv64[r] = 0.0;
  // Range of this warp's targets: a source block is summed in FP32 only if
  // it lies at least near_dist from all of them.
  double wlo = 0.0, whi = 0.0;
  if (MIXED) {
    double mn = x[0], mx = x[0];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      mn = fmin(mn, x[r]);
      mx = fmax(mx, x[r]);
    }
    wlo = warp_min(mn);
    whi = warp_max(mx);
  }

  auto chunk_is_tma = [&](int k) -> bool {
    const int64_t cs = s0 + (int64_t)k * CH;
    return a.use_tma && k < nchunks && (s1 - cs) >= CH;
  };
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (chunk_is_tma(k)) {
        mbar_arrive_expect_tx(&st.bar[k], CH * 8);
        bulk_g2s(st.sbuf[k], a.src + s0 + (int64_t)k * CH, CH * 8, &st.bar[k]);
        pending |= 1u << k;
      }
    }
  }

  for (int k = 0; k < nchunks; ++k) {
    const int b = k & 1;
    const int64_t cs = s0 + (int64_t)k * CH;
    const int len = (int)min((int64_t)CH, s1 - cs);
    bool ok = true;
    if (chunk_is_tma(k)) {
      ok = mbar_wait(&st.bar[b], (phase >> b) & 1u, a.wait_cycles);
      if (ok) {  // a copy that did not land stays pending for the drain below
        phase ^= 1u << b;
        pending &= ~(1u << b);
      }
    } else {
      for (int i = tid; i < len; i += NT) st.sbuf[b][i] = a.src[cs + i];
    }
    if (!__syncthreads_and(ok)) {
      // A bulk copy never completed: record it, drain what thread 0 still
      // has in flight (bounded), and leave uniformly.
      if (tid == 0) {
        atomicExch(a.err, DEV_ERR_TIMEOUT);
        for (int q = 0; q < 2; ++q)
          if ((pending >> q) & 1u) mbar_wait(&st.bar[q], (phase >> q) & 1u, 200000000LL);
      }
      return false;
    }
    if (MIXED) {
      // Source pairs of each full 256-block: (s1, s2) = (src[k], src[k+128])
      // as {SM, SM, DL, DL} relative to the block's first source.  Pairing
      // sources half a block apart keeps e1 = d1^2+eta^2 and e2 well apart:
      // adjacent sorted sources give e1 e2 ~ a square, and the rounded
      // reciprocal of a near-square carries a small systematic error
      // (~2e-11 relative, measured) that adds up coherently at large p.
      for (int i = tid; i < (len / SUB) * (SUB / 2); i += NT) {
        const int blk = i / (SUB / 2) * SUB, kk = i % (SUB / 2);
        const double cb = st.sbuf[b][blk];
        const double v1 = st.sbuf[b][blk + kk], v2 = st.sbuf[b][blk + kk + SUB / 2];
        const float sm = (float)(v1 - cb), dl = (float)(v1 - v2);
        st.sm4[i] = make_float4(sm, sm, dl, dl);
      }
      __syncthreads();
    }

    for (int sub = 0; sub < len; sub += SUB) {
      const int slen = min(SUB, len - sub);
      bool far32 = false;
      if (MIXED && slen == SUB) {
        const double2 bd = a.bounds[(cs + sub) / SUB];
        const double gap = fmax(fmax(bd.x - whi, wlo - bd.y), 0.0);
        const double span = fmax(bd.y - wlo, whi - bd.x);
        far32 = gap >= a.near_dist && span <= 1e9;
      }
      if (MIXED && far32) {
        // Block-wide target offsets x - cb = TH + TL.
        const double cb = st.sbuf[b][sub];
        u64 TH[R2], TL[R2];
#pragma unroll
        for (int kk = 0; kk < R2; ++kk) {
          const double o0 = x[2 * kk] - cb, o1 = x[2 * kk + 1] - cb;
          const float h0 = (float)o0, h1 = (float)o1;
          TH[kk] = pk2(h0, h1);
          TL[kk] = pk2((float)(o0 - (double)h0), (float)(o1 - (double)h1));
        }
        const float4* sp = &st.sm4[sub / 2];
        const u64 ETA2_ = ETA2;
        for (int j = 0; j < SUB / 2; j += FOLD / 2) {
          u64 RE[R2], IV[R2];
#pragma unroll
          for (int kk = 0; kk < R2; ++kk) RE[kk] = IV[kk] = 0ull;
#pragma unroll
          for (int q = 0; q < FOLD / 2; ++q) {
            const float4 s4 = sp[j + q];
            const u64 SM = pk2(s4.x, s4.y), DL = pk2(s4.z, s4.w);
#pragma unroll
            for (int kk = 0; kk < R2; ++kk)
              pairs32x4(SM, DL, TH[kk], TL[kk], ETA2_, RE[kk], IV[kk]);
          }
          // FP32 partials of FOLD sources are folded into FP64 (negated),
          // with the reciprocal's mean error taken out.
          constexpr double CORR = 1.0 - RCP32_BIAS;
#pragma unroll
          for (int kk = 0; kk < R2; ++kk) {
            float r0, r1, v0, v1;
            upk2(RE[kk], r0, r1);
            upk2(IV[kk], v0, v1);
            re64[2 * kk] = fma(-(double)r0, CORR, re64[2 * kk]);
            re64[2 * kk + 1] = fma(-(double)r1, CORR, re64[2 * kk + 1]);
            iv64[2 * kk] = fma(-(double)v0, CORR, iv64[2 * kk]);
            iv64[2 * kk + 1] = fma(-(double)v1, CORR, iv64[2 * kk + 1]);
          }
        }
      } else {
        const double* sp = &st.sbuf[b][sub];
        int j = 0;
#pragma unroll 2
        for (; j + 2 <= slen; j += 2) {
          const double2 l2 = *reinterpret_cast<const double2*>(sp + j);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            pair64(x[r], l2.x, eta2, re64[r], iv64[r]);
            pair64(x[r], l2.y, eta2, re64[r], iv64[r]);
          }
        }
        if (j < slen) {
          const double l = sp[j];
#pragma unroll
          for (int r = 0; r < R; ++r) pair64(x[r], l, eta2, re64[r], iv64[r]);
        }
      }
    }
    __syncthreads();
    if (tid == 0 && chunk_is_tma(k + 2)) {
      fence_proxy_async();
      mbar_arrive_expect_tx(&st.bar[b], CH * 8);
      bulk_g2s(st.sbuf[b], a.src + s0 + (int64_t)(k + 2) * CH, CH * 8, &st.bar[b]);
      pending |= 1u << b;
    }
  }

#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t idx = wbase + r * 32 + lane;
    if (idx < a.nt) {
      a.out_re[idx] = re64[r];
      a.out_im[idx] = eta * iv64[r];
    }
  }
  return true;
}

}  // namespace shrk
