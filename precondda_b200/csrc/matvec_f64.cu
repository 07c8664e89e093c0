// complex128 instantiations of the matvec passes
#include "matvec_impl.cuh"

namespace dda {
template <>
bool mv_general_set<double>(int Lx, int Ly, int Lz, int p3var, MvSet<double>& out) {
  return mv_general_set_impl<double>(Lx, Ly, Lz, p3var, out);
}
template <>
cudaError_t launch_matvec<double>(Ctx& ctx, const Geo& g, const PassCfg& pc, InstState* st, const int* act, int nb,
                                 int in_id, int out_id, int mode, int cond, double gscale, cudaStream_t s,
                                 const MvFuse& fz) {
  return launch_matvec_impl<double>(ctx, g, pc, st, act, nb, in_id, out_id, mode, cond, gscale, s, fz);
}
template <>
cudaError_t launch_amul<double>(Ctx& ctx, const Geo& g, const PassCfg& pc, InstState* st, const int* act, int nb,
                               int in_id, int mid_id, int out_id, int mode, int cond, double gscale, double pscale,
                               cudaStream_t s, const MvFuse& fz) {
  return launch_amul_impl<double>(ctx, g, pc, st, act, nb, in_id, mid_id, out_id, mode, cond, gscale, pscale, s,
                                  fz);
}
template <>
cudaError_t launch_matvec_tw<double>(const Geo& g, const PassCfg& pc, InstState* st, const void* twx, const void* twy,
                                   const void* twz, int in_id, int out_id, int mode, double gscale, cudaStream_t s) {
  typedef typename CT<double>::T C;
  return launch_matvec_tw_impl<double>(g, pc, st, (const C*)twx, (const C*)twy, (const C*)twz, in_id, out_id, mode,
                                     gscale, s);
}
}  // namespace dda
