// Register-FFT local part of H*psi, FP32 (complex64) instantiation.
#include "fftpath.cuh"

namespace pspw {

// Square planes up to 96 (the FP64 plane and its density accumulator must fit
// in 227 KB of shared memory) and any z length with a register split.
bool fast_supported(int n1, int n2, int n3) {
  return n1 == n2 && n1 <= 96 && nsplit_for(n1).n1 > 0 && nsplit_for(n3).n1 > 0;
}

template int local_fast<float>(pspw_cell *, const FastGeo &, const float2 *, int, float2 *, int,
                               int, int, const ScratchPlan *, const RecArg<float2, float> &);

template int rho_fast<float>(pspw_cell *, const FastGeo &, const float2 *, int, int, int,
                            const double *, double *);

}  // namespace pspw
