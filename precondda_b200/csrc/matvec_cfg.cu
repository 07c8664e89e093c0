// Tile shapes of the five matvec passes (see matvec_impl.cuh).
#include "matvec_impl.cuh"

#include <cstdlib>
#include <mutex>
#include <set>
#include <utility>

namespace dda {

bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("DDA_NO_PDL");
    return !(e && *e == '1');
  }();
  return on;
}

bool fused_zy_enabled(bool inverse) {
  const char* e = getenv("DDA_NO_FUSED_ZY");
  if (e && *e == '1') return false;
  if (inverse) {
    e = getenv("DDA_NO_FUSED_INV");
    if (e && *e == '1') return false;
  }
  return true;
}

bool p3_pipe_enabled() {
  const char* e = getenv("DDA_NO_P3PIPE");
  return !(e && *e == '1');
}

int device_sms() {
  static std::mutex mu;
  static int sms[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  std::lock_guard<std::mutex> lk(mu);
  if (!sms[dev]) {
    int v = 0;
    sms[dev] = (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0) ? v : 148;
  }
  return sms[dev];
}

cudaError_t mv_prepare(const void* const* ks, int n) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  for (int i = 0; i < n; ++i) {
    if (!ks[i] || done.count({dev, ks[i]})) continue;
    if ((e = cudaFuncSetAttribute(ks[i], cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024))) return e;
    if ((e = cudaFuncSetAttribute(ks[i], cudaFuncAttributePreferredSharedMemoryCarveout, 100))) return e;
    done.insert({dev, ks[i]});
  }
  return cudaSuccess;
}

PassCfg make_pass_cfg(const Geo& g, bool dbl) {
  return dbl ? make_pass_cfg_impl<double>(g) : make_pass_cfg_impl<float>(g);
}

}  // namespace dda
