// Launch interface of the sTDDFT ("std") tensor kernels (k_std.cu).
#pragma once

#include "pa_internal.h"

namespace pa {

struct StdArgs {
  DevBasis B;                        // orbital basis
  DevBasis X;                        // auxiliary basis
  DeviceTables dt;
  int boys_mode = 1;
  double thresh = 0.0;               // Schwarz threshold on Q_ab * Q_c
  const int2* pair_ab = nullptr;     // pair -> (a, b), a >= b
  const int* pair_unit0 = nullptr;   // pair -> first bra unit
  const double4* unit_pP = nullptr;  // unit -> (p, P)
  const double* esph = nullptr;      // E_sph blocks
  const long long* unit_esph = nullptr;
  const double* Qab = nullptr;       // pair -> Schwarz value
  const double* Qc = nullptr;        // aux shell -> Schwarz value
};

// Tt[P + naux * mu] = (mu mu|P) for surviving (a, a, c); other entries untouched
// (std/intor.f90:66-111).
int launch_std_df1c(const StdArgs& a, double* Tt, cudaStream_t s);

// Half-transformed, value-screened blocks of intor_df2c_mo (std/intor.f90:207-261)
// for the auxiliary shells [c0, c1): W[((k - k0) * nmos + p) * nbf + nu] =
// sum_a skip2(sum_(i in a) C[i, p] skip1((a b|k))) for nu in shell b, k in
// [k0, k1) the functions of the shells. mo is C (nbf x nmos, column-major).
int launch_std_df2c_half(const StdArgs& a, int c0, int c1, int k0, int nmos, const double* mo,
                         double* W, cudaStream_t s);

// Raw[(k0 + kk) + naux * (p(p+1)/2 + q)] = Res[(kk * nmos + p) + nk * nmos * q], q <= p.
int launch_std_pack(const double* Res, int nk, int nmos, int k0, int naux, double* Raw,
                    cudaStream_t s);

// out[kp * nshells_aux + c] = ||(ab|c)||_2 for pair rec_pair[kp] (kp < npairs)
// and every auxiliary shell c.
int launch_std_block_norms(const StdArgs& a, const int* rec_pair, int npairs, double* out, cudaStream_t s);

// out[i + rows * j] = in[j + cols * i] (out: rows x cols, column-major).
int launch_transpose(const double* in, int rows, int cols, double* out, cudaStream_t s);

}  // namespace pa
