// Tensor-core MO contraction (sm_100a: tcgen05 + TMA).
//
// D[r][j] = sum_k A[r][k] Bt[j][k] for the rows r of basis values (value,
// gradient, Laplacian of every basis function at one position: one row per
// component) against the MO coefficients of one spin (Bt[j][k] = C[k][j]).
// This is the per-position product of MO_matrix_blas::updateLap
// (orbitals/MO_matrix_blas.h:411-491) batched over positions into one dense
// GEMM.  Precision: split TF32, A = A_hi + A_lo and B = B_hi + B_lo with
// every part rounded to TF32 (10+1 mantissa bits), D = A_hi B_hi + A_hi B_lo
// + A_lo B_hi accumulated in FP32 in tensor memory (relative error of a
// product ~2^-22, the FP32 level).
//
// One CTA of 128 threads computes a 128-row tile of D for all (<= 256)
// columns.  Thread 0 issues the TMA loads of the K chunks (32 FP32 = one
// 128-byte swizzle row) into a ring of shared-memory stages and the MMAs
// (tcgen05.mma.cta_group::1.kind::tf32, M = 128, N = bn); each stage is
// released by tcgen05.commit to its mbarrier.  The accumulators live in
// tensor memory (2 bn FP32 columns x 128 lanes: the high products and the
// cross terms apart); the four warps read their 32 lanes back with
// tcgen05.ld and add the two.  TMA sources are this GPU's own global memory
// only and no load uses cluster multicast.
//
// Every wait is bounded (iteration and time limit): on expiry the CTA
// records an error code in *err, stops issuing, and still frees its tensor
// memory before returning.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace qwg {

constexpr int TC_BM = 128;        // rows per CTA (UMMA M)
constexpr int TC_BK = 32;         // FP32 elements per K chunk (128 bytes)
constexpr int TC_THREADS = 128;
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;  // 2 s per wait at most

struct TcGemmArgs {
  int rows;      // valid rows of A and D
  int kchunks;   // padded K / 32
  int n;         // valid columns of D
  int bn;        // UMMA N: multiple of 16, 16..256, >= n
  int ldd;       // row stride of D (elements)
  int stages;    // shared-memory ring depth
  float* D;      // [rows][ldd]
  int* err;      // 0, or the code of the first expired wait
};

__device__ __forceinline__ uint32_t tc_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long tc_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void tc_mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void tc_mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc_smem(bar)), "r"(bytes) : "memory");
}

// Wait for the phase with the given parity to complete; false when the
// time limit expires first.
__device__ __forceinline__ bool tc_mbar_wait(uint64_t* bar, uint32_t parity) {
  const unsigned long long t0 = tc_now();
  for (uint32_t it = 0;; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(tc_smem(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255) == 255 && tc_now() - t0 > TC_WAIT_NS) return false;
  }
}

__device__ __forceinline__ void tc_tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          tc_smem(dst)),
      "l"(map), "r"(tc_smem(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major tile in the 128-byte swizzle
// layout: rows of 128 bytes, 8-row atoms 1024 bytes apart (stride byte
// offset), leading byte offset unused (1), descriptor version 1, layout 2.
__device__ __forceinline__ uint64_t tc_sdesc_sw128(const void* p) {
  const uint64_t a = tc_smem(p);
  return ((a & 0x3FFFFull) >> 4) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: D FP32, A and B TF32, both K-major, M x N.
__host__ __device__ constexpr uint32_t tc_idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc_smem(bar))
               : "memory");
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane (the warp
// reads its 32 lanes); complete after tcgen05.wait::ld.
__device__ __forceinline__ void tc_ld16(uint32_t addr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(addr));
}

// Split of an FP32 value into two TF32 parts (round to nearest, ties away):
// hi + lo reproduces v to ~2^-22 relative.
__device__ __forceinline__ void tc_split_tf32(float v, float& hi, float& lo) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(v));
  hi = __uint_as_float(h);
  uint32_t l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(v - hi));
  lo = __uint_as_float(l);
}

// Shared memory of one CTA: the stage ring (A_hi, A_lo: 128 x 32 FP32;
// B_hi, B_lo: bn x 32 FP32), 1024-byte aligned, then the mbarriers.
__host__ __device__ constexpr size_t tc_stage_bytes(int bn) { return 2 * (size_t)TC_BM * 128 + 2 * (size_t)bn * 128; }
__host__ __device__ constexpr size_t tc_smem_bytes(int bn, int stages) {
  return 1024 + (size_t)stages * tc_stage_bytes(bn) + 256;
}

#ifndef QWG_WALKERS_ONLY  // the GEMM kernel lives in the engine translation unit
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_mo_gemm_tf32x3(const __grid_constant__ CUtensorMap map_ahi, const __grid_constant__ CUtensorMap map_alo,
                     const __grid_constant__ CUtensorMap map_bhi, const __grid_constant__ CUtensorMap map_blo,
                     TcGemmArgs g) {
  extern __shared__ unsigned char tc_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)tc_raw + 1023) & ~(uintptr_t)1023);
  const size_t sb = tc_stage_bytes(g.bn);
  uint64_t* bars = (uint64_t*)(base + (size_t)g.stages * sb);
  uint64_t* full = bars;                 // [stages]: TMA bytes of the stage landed
  uint64_t* empty = bars + g.stages;     // [stages]: the MMAs reading the stage completed
  uint64_t* done = bars + 2 * g.stages;  // all MMAs completed
  uint32_t* tmem_slot = (uint32_t*)(done + 1);
  __shared__ int s_fail;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = blockIdx.x * TC_BM;
  // two accumulators: columns [0, bn) take A_hi B_hi, [bn, 2 bn) the cross
  // terms A_hi B_lo + A_lo B_hi (added in FP32 in the epilogue, so the small
  // terms do not lose bits against the large running sum)
  uint32_t ncols = 32;
  while ((int)ncols < 2 * g.bn) ncols <<= 1;

  if (threadIdx.x == 0) {
    s_fail = 0;
    for (int s = 0; s < g.stages; s++) {
      tc_mbar_init(full + s, 1);
      tc_mbar_init(empty + s, 1);
    }
    tc_mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0) {
    const uint32_t idesc = tc_idesc_tf32(TC_BM, g.bn);
    const uint32_t bytes = (uint32_t)sb;
    auto load = [&](int c, int slot) {
      unsigned char* st = base + (size_t)slot * sb;
      tc_mbar_expect_tx(full + slot, bytes);
      tc_tma_load_2d(st, &map_ahi, full + slot, c * TC_BK, row0);
      tc_tma_load_2d(st + TC_BM * 128, &map_alo, full + slot, c * TC_BK, row0);
      tc_tma_load_2d(st + 2 * TC_BM * 128, &map_bhi, full + slot, c * TC_BK, 0);
      tc_tma_load_2d(st + 2 * TC_BM * 128 + (size_t)g.bn * 128, &map_blo, full + slot, c * TC_BK, 0);
    };
    int fail = 0;
    for (int c = 0; c < g.stages && c < g.kchunks; c++) load(c, c);
    for (int cc = 0; cc < g.kchunks; cc++) {
      const int s = cc % g.stages;
      if (!tc_mbar_wait(full + s, (cc / g.stages) & 1)) { fail = 2; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      unsigned char* st = base + (size_t)s * sb;
      const uint64_t ahi = tc_sdesc_sw128(st), alo = tc_sdesc_sw128(st + TC_BM * 128);
      const uint64_t bhi = tc_sdesc_sw128(st + 2 * TC_BM * 128);
      const uint64_t blo = tc_sdesc_sw128(st + 2 * TC_BM * 128 + (size_t)g.bn * 128);
#pragma unroll
      for (int k = 0; k < 4; k++) {  // UMMA K = 8 TF32 = 32 bytes: advance the start address by 2 x 16 B
        const uint64_t o = 2ull * k;
        const uint32_t acc = (cc > 0 || k > 0) ? 1u : 0u;
        tc_mma_tf32(tmem, ahi + o, bhi + o, idesc, acc);
        tc_mma_tf32(tmem + (uint32_t)g.bn, ahi + o, blo + o, idesc, acc);
        tc_mma_tf32(tmem + (uint32_t)g.bn, alo + o, bhi + o, idesc, 1u);
      }
      tc_commit(empty + s);
      // refill the stage of the previous chunk once its MMAs completed (the
      // tensor pipe meanwhile works on this chunk's)
      const int p = cc - 1, nxt = cc - 1 + g.stages;
      if (p >= 0 && nxt < g.kchunks) {
        const int ps = p % g.stages;
        if (!tc_mbar_wait(empty + ps, (p / g.stages) & 1)) { fail = 1; break; }
        load(nxt, ps);
      }
    }
    // the completion barrier tracks every MMA this thread issued, also
    // after a failed wait (then it guards the release of tensor memory)
    tc_commit(done);
    s_fail = fail;
  }
  __syncthreads();
  const bool bad = s_fail != 0 || !tc_mbar_wait(done, 0);
  const int fail = __syncthreads_or(bad) ? (s_fail ? s_fail : 3) : 0;
  if (fail) {
    if (threadIdx.x == 0) atomicCAS(g.err, 0, fail);
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int r = row0 + warp * 32 + lane;
    for (int c0 = 0; c0 < g.bn; c0 += 16) {
      uint32_t v[16], w[16];
      const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      tc_ld16(addr, v);
      tc_ld16(addr + (uint32_t)g.bn, w);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (r < g.rows) {
        float* d = g.D + (size_t)r * g.ldd;
#pragma unroll
        for (int j = 0; j < 16; j++)
          if (c0 + j < g.n) d[c0 + j] = __uint_as_float(v[j]) + __uint_as_float(w[j]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    // after a failed load wait the MMAs already issued may still run: wait
    // (bounded) for their completion barrier before freeing the columns
    if (fail == 1 || fail == 2) (void)tc_mbar_wait(done, 0);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}
#endif  // QWG_WALKERS_ONLY

}  // namespace qwg
