// Register-FFT local part of H*psi, FP64 (complex128) instantiation.
#include "fftpath.cuh"

namespace pspw {

template int local_fast<double>(pspw_cell *, const FastGeo &, const double2 *, int, double2 *,
                                int, int, int, const ScratchPlan *,
                                const RecArg<double2, double> &);

template int rho_fast<double>(pspw_cell *, const FastGeo &, const double2 *, int, int, int,
                            const double *, double *);

}  // namespace pspw
