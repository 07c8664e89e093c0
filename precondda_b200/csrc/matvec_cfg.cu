// Tile shapes of the five matvec passes (see matvec_impl.cuh).
#include "matvec_impl.cuh"

#include <algorithm>
#include <cstdlib>
#include <map>
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

double mixed_sweep_target(double inner_tol, double tol, double relres) {
  static const double f = [] {
    const char* e = getenv("DDA_SWEEP_SAFETY");
    const double v = e ? atof(e) : 0.0;
    return (v > 0.0 && v < 1.0) ? v : 0.8;
  }();
  if (!(relres > 0.0)) return inner_tol;
  return std::max(inner_tol, std::min(0.5, f * tol / relres));
}

double mixed_inner_ratio(double ratio) {
  static const double r = [] {
    const char* e = getenv("DDA_INNER_RATIO");
    return e ? atof(e) : -1.0;
  }();
  if (r >= 0.0) return r;
  return ratio == 0.0 ? 0.0 : std::max(ratio, 1000.0);
}

bool ma_fuse_enabled() {
  const char* e = getenv("DDA_NO_MA_FUSE");   // read per call: tests switch it between captures
  return !(e && *e == '1');
}

int mv_split_ways(int nb) {
  static const int k = [] {
    const char* e = getenv("DDA_MV_SPLIT");
    const int v = e ? atoi(e) : 1;
    return v < 1 ? 1 : (v > Ctx::kMaxSplit ? Ctx::kMaxSplit : v);
  }();
  return nb < k ? nb : k;
}

namespace {
std::mutex g_pdl_mu;
std::set<cudaStream_t> g_no_pdl;
}  // namespace

bool stream_pdl(cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_pdl_mu);
  return g_no_pdl.empty() || !g_no_pdl.count(s);
}

void set_stream_pdl(cudaStream_t s, bool on) {
  std::lock_guard<std::mutex> lk(g_pdl_mu);
  if (on) g_no_pdl.erase(s);
  else g_no_pdl.insert(s);
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

bool prefetch_forced() {
  const char* e = getenv("DDA_PREFETCH");
  return e && *e == '1';
}

int resident_ctas(const void* k, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<const void*, std::pair<int, size_t>>, int> cache;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_pair(k, std::make_pair(threads, smem));
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (!k || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem) != cudaSuccess || n < 1) n = 1;
  cache[key] = n;
  return n;
}

bool z_pair_forced() {
  const char* e = getenv("DDA_ZPAIR");
  return e && *e == '1';
}

bool y_pair_forced() {
  const char* e = getenv("DDA_YPAIR");
  return e && *e == '1';
}

bool p3_pair_forced() {
  const char* e = getenv("DDA_P3PAIR");
  return e && *e == '1';
}

bool p3_pipe_forced() {
  const char* e = getenv("DDA_P3PIPE");
  return e && *e == '1';
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

// ---------------------------------------------------------------------------
// Launch tuning table: per (dtype, box, FFT lengths, batch-width class) the
// launch variant an autotuner measured fastest (DDA_TUNE_* flags).  Looked
// up at every matvec launch; absent entries mean the defaults.
// ---------------------------------------------------------------------------
namespace {
struct TuneKey {
  int dtype, nx, ny, nz, Lx, Ly, Lz, nbc;
  bool operator<(const TuneKey& o) const {
    const int a[8] = {dtype, nx, ny, nz, Lx, Ly, Lz, nbc};
    const int b[8] = {o.dtype, o.nx, o.ny, o.nz, o.Lx, o.Ly, o.Lz, o.nbc};
    for (int i = 0; i < 8; ++i)
      if (a[i] != b[i]) return a[i] < b[i];
    return false;
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tune;
TuneKey tune_key(int dtype, const Geo& g, int nb) {
  return TuneKey{dtype, g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz, nb_class(nb)};
}
}  // namespace

int nb_class(int nb) { return nb <= 1 ? 1 : nb <= 3 ? 2 : nb <= 7 ? 4 : nb <= 15 ? 8 : 16; }

int tune_flags(int dtype, const Geo& g, int nb) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (g_tune.empty()) return 0;
  auto it = g_tune.find(tune_key(dtype, g, nb));
  return it == g_tune.end() ? 0 : it->second;
}

void tune_set(int dtype, const Geo& g, int nb, int flags) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (flags < 0) g_tune.erase(tune_key(dtype, g, nb));
  else g_tune[tune_key(dtype, g, nb)] = flags;
}

bool tune_get(int dtype, const Geo& g, int nb, int* flags) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(tune_key(dtype, g, nb));
  if (it == g_tune.end()) return false;
  *flags = it->second;
  return true;
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
