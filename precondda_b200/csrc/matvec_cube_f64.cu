// complex128 matvec passes specialised for a cubic box n^3 on a (2n)^3 grid
// (compiled apart from the general kernels so the two build in parallel).
#include "matvec_impl.cuh"

namespace dda {
template <>
bool mv_cube_set<double>(int L, int p3var, MvSet<double>& o) {
  if (p3var != 2) return false;
  switch (L) {
#define DDA_K(n) case n: mv_cube_fill<double, n, 2>(o); return true;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  }
  return false;
}
}  // namespace dda
