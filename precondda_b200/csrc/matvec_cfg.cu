// Tile shapes of the five matvec passes (see matvec_impl.cuh).
#include "matvec_impl.cuh"

namespace dda {

PassCfg make_pass_cfg(const Geo& g, bool dbl) {
  return dbl ? make_pass_cfg_impl<double>(g) : make_pass_cfg_impl<float>(g);
}

}  // namespace dda
