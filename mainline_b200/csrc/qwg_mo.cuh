// Batched MO evaluation at arbitrary positions (MO_matrix::updateLap for a
// list of positions, orbitals/MO_matrix.h:101-118): value, gradient and
// Laplacian of every orbital of one spin.
//
// FP64 contexts: one warp per position evaluates the basis and contracts it
// with the MO coefficients on CUDA cores (mo_lap_warp), as the walker
// kernels do.  Mixed-precision contexts: one warp per position writes the
// position's five basis rows (value, d/dx, d/dy, d/dz, Laplacian) as split
// TF32 pairs into the A operand of the tensor-core GEMM (qwg_tc.cuh), which
// contracts all positions with the coefficients in one launch.
#pragma once

#include "qwg_kernels.cuh"
#include "qwg_tc.cuh"

namespace qwg {

// FP64 reference path: out[p][m][5] for p < npos, m < nmo.
template <typename Real>
__global__ void __launch_bounds__(128) k_mo_rows_cuda(const __grid_constant__ DevSys<Real> S, const Real* moc_s,
                                                      const double* pos, int npos, int nmo, Real* bas_scratch,
                                                      Real* out_scratch, double* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = blockIdx.x * 4 + warp;
  if (p >= npos) return;
  double x = pos[3 * p], y = pos[3 * p + 1], z = pos[3 * p + 2];
  if (S.periodic) wrap_pos(S, x, y, z);
  Real* bas = bas_scratch + (size_t)p * S.nbasis * 5;
  Real* o = out_scratch + (size_t)p * S.mstride * 5;
  mo_lap_warp<Real, 2, true>(S, moc_s, x, y, z, nmo, bas, o, lane);
  for (int i = lane; i < nmo * 5; i += 32) out[(size_t)p * nmo * 5 + i] = double(o[i]);
}

// Basis rows of npos positions into the split-TF32 A operand:
// a_hi/a_lo[(p * 5 + c) * kpad + f] for component c of basis function f
// (zero for nbasis <= f < kpad).  bas_scratch: [npos][nbasis][5] doubles.
template <typename Real>
__global__ void __launch_bounds__(128) k_basis_rows_tf32(const __grid_constant__ DevSys<Real> S, const double* pos,
                                                         int npos, int kpad, double* bas_scratch, float* a_hi,
                                                         float* a_lo) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = blockIdx.x * 4 + warp;
  if (p >= npos) return;
  double x = pos[3 * p], y = pos[3 * p + 1], z = pos[3 * p + 2];
  if (S.periodic) wrap_pos(S, x, y, z);
  double* bas = bas_scratch + (size_t)p * S.nbasis * 5;
  basis_lap_warp<double, 2, true>(S, x, y, z, bas, lane);
  for (int idx = lane; idx < 5 * kpad; idx += 32) {
    const int c = idx / kpad, f = idx - c * kpad;
    const double v = f < S.nbasis ? bas[(size_t)f * 5 + c] : 0.0;
    // high part: v rounded to TF32; low part: the FP64 remainder rounded to
    // TF32 (it also carries the FP32 rounding of v)
    uint32_t h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(float(v)));
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(float(v - double(__uint_as_float(h)))));
    const size_t at = ((size_t)p * 5 + c) * kpad + f;
    a_hi[at] = __uint_as_float(h);
    a_lo[at] = __uint_as_float(l);
  }
}

}  // namespace qwg
