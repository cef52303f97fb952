// Tensor-core (tcgen05, 3xTF32) projector GEMMs of the FP32 H*psi.
#pragma once

#include "engine.h"

namespace pspw {

// True when the cell's projectors fit the tensor-core kernels (one species,
// at most 256 atoms).
bool nl_tc_usable(const pspw_cell *c);

// wp[b*nproj + a*L + lm] = WNL(lm) sum_G conj(EIGR(G,a)) PKG_A(lm,G) psi_b(G)
// for the first ngw G of nb bands.  `part` holds max_split * 2*nb*nproj
// floats (null: the cell's workspace).
int nl_tc_project(pspw_cell *c, const float2 *psi, int ld, int ngw, int nb, float2 *wp,
                  float *part, int max_split);

// out = a*(out + sum_{a,lm} EIGR PKG_A wp) + b*in + g*xm2 on the first ngw G.
int nl_tc_backproject(pspw_cell *c, const float2 *wp, int ngw, int nb, float2 *out, int ldo,
                      const float2 *in, int ldi, const float2 *xm2, int ldx, float a, float b,
                      float g);

}  // namespace pspw
