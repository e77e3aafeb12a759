// One walker-kernel family: compiled once per (QWG_REAL, QWG_MM) pair by the
// build (e.g. -DQWG_REAL=float -DQWG_MM=32).
#include <map>
#include <mutex>

#define QWG_WALKERS_ONLY
#include "qwg_launch.cuh"

#if !defined(QWG_REAL) || !defined(QWG_MM)
#error "qwg_walkers.cu is compiled with -DQWG_REAL=<double|float> -DQWG_MM=<8|16|32|0|-1>"
#endif

namespace qwg {
namespace {

// Raise a kernel's dynamic shared-memory limit once to the largest size any
// context asked for (never during a stream capture: callers make a plain
// launch of every kernel before capturing it).
template <class K>
cudaError_t ensure_smem_attr(K kern, size_t bytes) {
  static std::mutex mu;
  static std::map<const void*, size_t> done;
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = done[(const void*)kern];
  if (bytes > have) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    have = bytes;
  }
  return cudaSuccess;
}

// compiled variants: with/without e-e-n terms; the local-energy kernels also
// per molecule / periodic cell (the others check at run time)
template <typename Real, int MM, int MODE, bool XL>
auto pick_kernel(const DevSys<Real>& S) {
  constexpr bool SPLIT_PER = MODE == KM_ELOC || MODE == KM_ELOC_TM;
  constexpr int P0 = SPLIT_PER ? 0 : 2, P1 = SPLIT_PER ? 1 : 2;
  return S.periodic ? (S.has_tb ? k_walkers<Real, MM, MODE, true, P1, XL> : k_walkers<Real, MM, MODE, false, P1, XL>)
                    : (S.has_tb ? k_walkers<Real, MM, MODE, true, P0, XL> : k_walkers<Real, MM, MODE, false, P0, XL>);
}

template <typename Real, int MM, int MODE>
cudaError_t launch_mode(const DevSys<Real>& S, const WLayout& L, const StepParams& P, const EvalIO& io, int nwalk,
                        int wpc, size_t smem, cudaStream_t stream) {
  // the FP32 HBM-resident kernels without the F/G-shell and CUTOFF_MO code
  // for the decks that have neither
  auto kern = pick_kernel<Real, MM, MODE, (MM <= 0)>(S);
  if constexpr (MM == 0 && sizeof(Real) == 4)
    if (!S.xl) kern = pick_kernel<Real, MM, MODE, false>(S);
  cudaError_t e = ensure_smem_attr(kern, smem);
  if (e != cudaSuccess) return e;
  if (nwalk <= 0) return cudaSuccess;  // attribute set only (before a stream capture)
  const int grid = (nwalk + wpc - 1) / wpc;
  kern<<<grid, 32 * wpc, smem, stream>>>(S, L, P, io);
  return cudaGetLastError();
}

}  // namespace

template <typename Real, int MM>
cudaError_t launch_walker_kernels(const DevSys<Real>& S, const WLayout& L, const StepParams& P, const EvalIO& io,
                                  int mode, int nwalk, int wpc, size_t smem, cudaStream_t stream) {
  if (mode == KM_EVAL) return launch_mode<Real, MM, KM_EVAL>(S, L, P, io, nwalk, wpc, smem, stream);
  if (mode == KM_RATIO) return launch_mode<Real, MM, KM_RATIO>(S, L, P, io, nwalk, wpc, smem, stream);
  if (mode == KM_SWEEP) return launch_mode<Real, MM, KM_SWEEP>(S, L, P, io, nwalk, wpc, smem, stream);
  if (mode == KM_ELOC) return launch_mode<Real, MM, KM_ELOC>(S, L, P, io, nwalk, wpc, smem, stream);
  if (mode == KM_TMOVE) return launch_mode<Real, MM, KM_TMOVE>(S, L, P, io, nwalk, wpc, smem, stream);
  if (mode == KM_ELOC_TM) return launch_mode<Real, MM, KM_ELOC_TM>(S, L, P, io, nwalk, wpc, smem, stream);
  return launch_mode<Real, MM, KM_STEPS>(S, L, P, io, nwalk, wpc, smem, stream);
}

template cudaError_t launch_walker_kernels<QWG_REAL, QWG_MM>(const DevSys<QWG_REAL>&, const WLayout&,
                                                             const StepParams&, const EvalIO&, int, int, int, size_t,
                                                             cudaStream_t);

}  // namespace qwg
