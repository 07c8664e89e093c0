// complex64 matvec passes specialised for a cubic box n^3 on a (2n)^3 grid
// (compiled apart from the general kernels so the two build in parallel).
#include "matvec_impl.cuh"

namespace dda {
template <>
bool mv_cube_set<float>(int L, int p3var, MvSet<float>& o) {
  if (p3var == 1) {
    // the register-tensor variant, compiled for the power-of-two lengths
    switch (L) {
      case 32: mv_cube_fill<float, 32, 1>(o); return true;
      case 64: mv_cube_fill<float, 64, 1>(o); return true;
      case 128: mv_cube_fill<float, 128, 1>(o); return true;
      case 256: mv_cube_fill<float, 256, 1>(o); return true;
      case 512: mv_cube_fill<float, 512, 1>(o); return true;
    }
    return false;
  }
  if (p3var == 2) {
    // radix-8 plan, tensor product through shared memory (the complex128
    // default), compiled for the power-of-two lengths
    switch (L) {
      case 64: mv_cube_fill<float, 64, 2>(o); return true;
      case 128: mv_cube_fill<float, 128, 2>(o); return true;
      case 256: mv_cube_fill<float, 256, 2>(o); return true;
    }
    return false;
  }
  if (p3var != 0) return false;
  switch (L) {
#define DDA_K(n) case n: mv_cube_fill<float, n, 0>(o); return true;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  }
  return false;
}
}  // namespace dda
