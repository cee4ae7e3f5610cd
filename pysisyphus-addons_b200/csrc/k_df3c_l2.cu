// Class kernels of the three-center contraction with L_ab = 2 (la + lb),
// every L_aux and tile-shape variant.
#include "k_df3c_impl.cuh"

PA_DF3C_ROW(2)
