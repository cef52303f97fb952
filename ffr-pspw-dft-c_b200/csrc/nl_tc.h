// Tensor-core (tcgen05, 3xTF32) projector GEMMs of the FP32 H*psi.
#pragma once

#include "engine.h"

namespace pspw {

// True when the cell's projectors fit the tensor-core kernels (every species
// with projectors: 1..256 atoms, at most 4 projectors per atom) and the
// kernels are selected.  The kernels run once per such species.
bool nl_tc_usable(const pspw_cell *c);

// Builds the EIGR operand tiles of a cell whose projectors fit the kernels
// (no-op otherwise).  Called once at cell creation.
int nl_tc_prepare(pspw_cell *c);
// The same tiles from a given EIGR copy (FP32, [nat][ngw]) into new buffers.
int nl_tc_build_tiles(pspw_cell *c, const float2 *eigr32, float **etp, float **etb);

// Bytes of the projection operand tiles for nb bands.
size_t nl_tc_wtile_bytes(const pspw_cell *c, int nb);

// Scratch of nl_tc_project from the cell's workspaces: partial sums (at most
// *max_split slices) and the projection operand tiles.
int nl_tc_reserve(pspw_cell *c, int ngw, int nb, float **part, int *max_split, float **wt);

// Projections of nb bands (first ngw G) into the operand tiles `wt`:
// W(a,lm,b) = WNL(lm) sum_G conj(EIGR(G,a)) PKG_A(lm,G) psi_b(G).
int nl_tc_project(pspw_cell *c, const float2 *psi, int ld, int ngw, int nb, float *part,
                  int max_split, float *wt);

// out = a*(out + sum_{a,lm} EIGR PKG_A W) + b*in + g*xm2 on the first ngw G;
// with pre, out already holds a*(H_loc psi) + b*in + g*xm2 and the kernel
// adds a * sum EIGR PKG_A W.
int nl_tc_backproject(pspw_cell *c, const float *wt, int ngw, int nb, float2 *out, int ldo,
                      const float2 *in, int ldi, const float2 *xm2, int ldx, float a, float b,
                      float g, bool pre = false);

// Runs one bounded device-side barrier wait on the cell stream and returns
// the cell's status after it: PSPW_ERR_TIMEOUT when the barrier is never
// completed (complete == 0), PSPW_OK otherwise.
int nl_tc_wait_check(pspw_cell *c, int complete);

}  // namespace pspw
