// FP32 operator apply of a uniform cell batch on the 5th-generation tensor cores.
//
// When every cell of a 3-D tensor batch has the same size, a constant mass and diffusion
// coefficient and a plain map (one dof per box mode, no coefficients, no expansions), all cells
// share one local operator: the nb x nb element matrix K_e of the sum-factorised kernel
// (accumulators.jl:1955-2013 evaluated once on the host from the same 1-D tables and
// quadrature).  The batch apply is then the GEMM Y_loc = X_loc K_e^T over the cells, M = 128
// cells per tile, K = N = nb padded to 128 (degree <= 4), followed by the scatter of the
// local results.
//
// Precision: FP32 inputs and element matrix are split into BF16 pieces, x = x_hi + x_lo and
// K = K_hi + K_lo, and the tile accumulates x_hi K_hi + x_lo K_hi + x_hi K_lo in FP32 (tensor
// memory): 24 tcgen05.mma kind::f16 (M 128, N 128, K 16) per tile, about 2^-16 relative
// accuracy of each product.  Only the FP32 levels of mixed-precision solves use it.
//
// Pipeline (persistent CTAs, 8 worker warps and 1 MMA warp, one barrier per step, two TMEM
// accumulators and two A buffers): step i issues the MMAs of tile i while the workers wait for
// tile i - 1, gather tile i + 1 (map + x -> BF16 hi/lo in the UMMA K-major core-matrix layout)
// into the buffer tile i - 1 has released, and scatter tile i - 1 (tcgen05.ld, atomicAdd).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tcgen05_ops.cuh"

namespace grico {
namespace dense {

constexpr int kM = 128;           // cells per tile
constexpr int kK = 128;           // local modes, padded (nb <= 128)
constexpr int kChunks = kK / 8;   // K chunks of 8 BF16 (16 bytes)
constexpr int kWorkers = 256;
constexpr int kThreads = kWorkers + 32;
constexpr uint32_t kPiece = uint32_t(kChunks) * kM * 16;  // one BF16 operand piece: 32 KB
constexpr size_t kSmem = 128 + 6 * size_t(kPiece);         // B hi, lo; A[2] hi, lo
constexpr uint32_t kTmemCols = 256;                         // two 128-column accumulators

// Element matrix K_e (row i = output mode, column j = input mode, both ix + N (iy + N iz)) to
// the B operand pieces: wp[((p * kChunks + j / 8) * kK + i) * 8 + j % 8], p = 0 (hi), 1 (lo),
// zero outside nb x nb
inline void pack_element_matrix(const double* Ke, int nb, __nv_bfloat16* wp) {
  for (int p = 0; p < 2; ++p)
    for (int c = 0; c < kChunks; ++c)
      for (int i = 0; i < kK; ++i)
        for (int e = 0; e < 8; ++e) {
          const int j = 8 * c + e;
          const float v = (i < nb && j < nb) ? float(Ke[size_t(i) * nb + j]) : 0.0f;
          const __nv_bfloat16 hi = __float2bfloat16(v);
          wp[((size_t(p) * kChunks + c) * kK + i) * 8 + e] = p == 0 ? hi : __float2bfloat16(v - __bfloat162float(hi));
        }
}

// y[map[c * nb + i]] += sum_j K_e[i][j] x[map[c * nb + j]] over the cells c of the batch (map
// entries -1 contribute nothing).  wp: pack_element_matrix output (64 KB).  err[0] is set when
// an mbarrier wait gives up.
__global__ void __launch_bounds__(kThreads) cell_apply_dense_tc(const int32_t* __restrict__ map, int64_t n_cells,
                                                               int nb, const __nv_bfloat16* __restrict__ wp,
                                                               const float* __restrict__ x, float* __restrict__ y,
                                                               int64_t n_vec, int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + 16);
  unsigned char* bsm = smem + 128;               // B hi, B lo
  unsigned char* asm_ = bsm + 2 * kPiece;        // A[buf][piece]
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  x += blockIdx.y * n_vec;
  y += blockIdx.y * n_vec;

  {
    const uint4* src = reinterpret_cast<const uint4*>(wp);
    uint4* dst = reinterpret_cast<uint4*>(bsm);
    for (int i = tid; i < int(2 * kPiece / 16); i += kThreads) dst[i] = src[i];
  }
  if (warp == 0) tc::tmem_alloc(tslot, kTmemCols);
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t b_s = tc::smem_u32(bsm), a_s = tc::smem_u32(asm_);
  const uint32_t idesc = tc::idesc_bf16(kM, kK);
  // every operand view: K-adjacent core matrices kM * 16 bytes apart, M- (N-) adjacent ones 128
  const uint64_t dsc0 = tc::smem_desc(0, kM * 16, 128);

  const int64_t tiles = (n_cells + kM - 1) / kM;
  const int64_t mine = tiles > blockIdx.x ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  uint32_t ph0 = 0, ph1 = 0;
  int pending = 0, fail = 0;

  // gather of local tile li into A buffer li & 1: thread (m = tid % 128, half = tid / 128) fills
  // chunks 8 half .. 8 half + 7 of cell m with BF16 hi and lo pieces
  auto gather = [&](int64_t li) {
    const int64_t cell = (blockIdx.x + li * gridDim.x) * kM + tid % kM;
    const int half = tid / kM;
    const bool act = cell < n_cells;
    unsigned char* abuf = asm_ + size_t(li & 1) * 2 * kPiece;
#pragma unroll 2
    for (int c = 8 * half; c < 8 * half + 8; ++c) {
      uint32_t hw[4], lw[4];
#pragma unroll
      for (int e = 0; e < 8; e += 2) {
        float v[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int j = 8 * c + e + u;
          int32_t d = -1;
          if (act && j < nb) d = __ldg(map + cell * nb + j);
          v[u] = d >= 0 ? x[d] : 0.0f;
        }
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[0], v[1]);
        const float2 hf = __bfloat1622float2(h2);
        const __nv_bfloat162 l2 = __floats2bfloat162_rn(v[0] - hf.x, v[1] - hf.y);
        hw[e / 2] = *reinterpret_cast<const uint32_t*>(&h2);
        lw[e / 2] = *reinterpret_cast<const uint32_t*>(&l2);
      }
      const size_t off = (size_t(c) * kM + tid % kM) * 16;
      *reinterpret_cast<uint4*>(abuf + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
      *reinterpret_cast<uint4*>(abuf + kPiece + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
  };

  if (mine > 0 && warp < 8) {
    gather(0);
    tc::fence_async_smem();
  }
  __syncthreads();
  for (int64_t i = 0; i <= mine; ++i) {
    if (warp == 8) {
      if (i < mine && lane == 0) {
        tc::fence_after_sync();
        const uint32_t acc = tmem + uint32_t((i & 1) * kK);
        const uint32_t ah = a_s + uint32_t(i & 1) * 2 * kPiece, al = ah + kPiece;
        const uint32_t bh = b_s, bl = b_s + kPiece;
#pragma unroll
        for (int s = 0; s < kChunks / 2; ++s) {
          const uint32_t ko = uint32_t(s) * 2 * kM * 16;  // two K chunks per MMA
          const uint64_t dah = dsc0 | uint64_t(((ah + ko) >> 4) & 0x3FFFu);
          const uint64_t dal = dsc0 | uint64_t(((al + ko) >> 4) & 0x3FFFu);
          const uint64_t dbh = dsc0 | uint64_t(((bh + ko) >> 4) & 0x3FFFu);
          const uint64_t dbl = dsc0 | uint64_t(((bl + ko) >> 4) & 0x3FFFu);
          tc::mma_bf16(acc, dah, dbh, idesc, s > 0 ? 1u : 0u);
          tc::mma_bf16(acc, dal, dbh, idesc, 1u);
          tc::mma_bf16(acc, dah, dbl, idesc, 1u);
        }
        tc::mma_commit(&bar[i & 1]);
      }
    } else {
      bool done = true;
      if (i > 0) {
        const int pb = int((i - 1) & 1);
        done = tc::mbar_wait(&bar[pb], pb ? ph1 : ph0);
        fail |= done ? 0 : 1;
        tc::fence_after_sync();
      }
      if (i + 1 < mine) gather(i + 1);  // into the buffer tile i - 1 has released
      if (i > 0) {
        // scatter of tile i - 1: warp w reads TMEM lanes (cells) 32 (w % 4) .. + 31 and the
        // columns (output modes) 64 (w / 4) .. + 63
        const int pb = int((i - 1) & 1), q = warp & 3;
        const int64_t cell = (blockIdx.x + (i - 1) * gridDim.x) * kM + 32 * q + lane;
        const bool act = done && cell < n_cells;
        for (int c0 = (warp >> 2) * 64; c0 < (warp >> 2) * 64 + 64; c0 += 16) {
          uint32_t r[16];
          __syncwarp();
          tc::tmem_ld16(tmem + (uint32_t(32 * q) << 16) + uint32_t(pb * kK + c0), r);
          if (act) {
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              const int j = c0 + e;
              if (j < nb) {
                const int32_t d = __ldg(map + cell * nb + j);
                if (d >= 0) atomicAdd(y + d, __uint_as_float(r[e]));
              }
            }
          }
        }
      }
      tc::fence_async_smem();  // the gathered tile is read by the tensor cores next step
    }
    tc::fence_before_sync();
    fail = __syncthreads_or(fail);
    if (i < mine) pending |= 1 << int(i & 1);
    if (fail) break;
    if (i > 0) {
      const int pb = int((i - 1) & 1);
      if (pb) ph1 ^= 1u;
      else ph0 ^= 1u;
      pending &= ~(1 << pb);
    }
  }
  if (fail) {
    if (tid == 0) atomicExch(err, 1);
    if (pending & 1) tc::mbar_wait(&bar[0], ph0);
    if (pending & 2) tc::mbar_wait(&bar[1], ph1);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}

}  // namespace dense
}  // namespace grico
