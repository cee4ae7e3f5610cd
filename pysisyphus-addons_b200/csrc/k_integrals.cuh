// Launch interfaces of the integral kernels (k_integrals.cu).
#pragma once

#include "pa_internal.h"

namespace pa {

// Arguments of the density-folding kernel for one class of sorted unit slots.
struct BraPrepArgs {
  int slot0 = 0, slot_end = 0;            // slots [slot0, slot_end) of this class
  const double* slot_Q = nullptr;         // slot -> Schwarz value of the unit's pair
  const double* qmax_aux = nullptr;       // device scalar: max aux Schwarz value
  double thresh = 0.0;
  const int* sorted_unit = nullptr;       // slot -> unit
  int nd = 0;                             // number of densities
  const double* dens = nullptr;           // density (d, i, j) at d*sd + i*si + j*sj
  long long sd = 0, si = 0, sj = 0;
  double4* slot_pP = nullptr;             // slot -> (p, P)
  double* G = nullptr;                    // G blocks: [z][slot in class][tuv][dw]
  long long g_base = 0;                   // offset of this class's first slot
  int dw = 8;                             // density chunk width (multiple of 8, <= 40)
  int n_class = 0;                        // slots in this class (stride of z)
  // QVL screening (null otherwise): per pair (center, extent) and
  // (zeta_a + zeta_b)^(1/4), copied to the unit's slot
  const double4* pair_qvl = nullptr;
  const double* pair_den = nullptr;
  double4* slot_qvl = nullptr;
  double* slot_den = nullptr;
};

size_t schwarz_bra_smem(int lab);
int launch_bra_prep(const DevBasis& B, const int2* pair_ab, UnitArrays U, const BraPrepArgs& a,
                    int lab, cudaStream_t s);

}  // namespace pa
