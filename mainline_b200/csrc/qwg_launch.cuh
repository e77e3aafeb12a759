// Launch entry of the walker kernels, one explicit instantiation per
// (working precision, orbital capacity) compiled in its own translation unit
// (qwg_walkers.cu built once per pair) so the kernel families build in
// parallel.
#pragma once
#include <cuda_runtime.h>

#include "qwg_kernels.cuh"

namespace qwg {

// Launches k_walkers<Real, MM, mode, has_tb> over nwalk walkers: wpc warps
// (walkers) per CTA, smem bytes of dynamic shared memory.  MM: 8/16/32
// shared-memory walkers, 0 HBM-resident walkers, -1 HBM-resident walkers with
// complex orbitals.
template <typename Real, int MM>
cudaError_t launch_walker_kernels(const DevSys<Real>& S, const WLayout& L, const StepParams& P, const EvalIO& io,
                                  int mode, int nwalk, int wpc, size_t smem, cudaStream_t stream);

#define QWG_WALKER_FAMILY(R, MM)                                                                              \
  extern template cudaError_t launch_walker_kernels<R, MM>(const DevSys<R>&, const WLayout&, const StepParams&, \
                                                           const EvalIO&, int, int, int, size_t, cudaStream_t);
QWG_WALKER_FAMILY(double, 8)
QWG_WALKER_FAMILY(double, 16)
QWG_WALKER_FAMILY(double, 32)
QWG_WALKER_FAMILY(double, 0)
QWG_WALKER_FAMILY(float, 8)
QWG_WALKER_FAMILY(float, 16)
QWG_WALKER_FAMILY(float, 32)
QWG_WALKER_FAMILY(float, 0)
QWG_WALKER_FAMILY(double, -1)
QWG_WALKER_FAMILY(float, -1)
#undef QWG_WALKER_FAMILY

}  // namespace qwg
