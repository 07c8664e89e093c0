// Allocation-free A.x: dda_matvec_noalloc.
//
// Some callers cannot allocate device memory at the point where they need the
// DDA product: code that is recording work into a CUDA graph (cudaMalloc is
// not a capturable operation), real-time or serving loops whose latency
// budget forbids allocator calls, and hosts whose device memory is owned by
// another framework's pool that forbids raw cudaMalloc.  This entry point
// computes the same product as dda_matvec without any allocation: the
// transform scratch (the T1/T2 buffers of the five passes), the per-call
// state block and the FFT twiddle tables all live in one file-scope
// __device__ array of DDA_NOALLOC_SCRATCH_BYTES (64 MiB), which every GPU
// that loads this library holds until the process exits.
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress (with that device current) and remembers it; make
// that first call before any stream capture.  Every call shares the one
// array and leaves its contents behind for the next call; the state block and
// twiddles are rewritten on every call, and the transform passes overwrite
// every scratch element they read, so nothing has to start at zero.  Calls
// that overlap on the GPU (different streams, or different host threads
// without ordering) race on the array and must not be issued.
#include <cstring>
#include <mutex>

#include "../../include/dda_b200.h"
#include "dda_host.h"
#include "fft_sizes.h"

namespace {

constexpr size_t kScratchBytes = DDA_NOALLOC_SCRATCH_BYTES;
constexpr size_t kStateOff = 0;          // InstState (< 4 KiB)
constexpr size_t kTwOff = 4096;          // 3 twiddle tables of <= 512 double2
constexpr size_t kTwStride = 512 * 16;
constexpr size_t kDataOff = 32768;       // T1 then T2

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_base[kMaxDevices] = {};

// Device address of the scratch array on the current device.
int scratch_base(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { dda::set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  if (dev < 0 || dev >= kMaxDevices) { dda::set_error("device index out of range"); return DDA_ERR_ARG; }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_base[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      dda::set_error(std::string("cudaGetSymbolAddress of the scratch array failed: ") + cudaGetErrorString(e));
      return DDA_ERR_CUDA;
    }
    g_base[dev] = p;
  }
  *out = g_base[dev];
  return DDA_OK;
}

// Twiddles exp(-2 pi i j/L), the same values the context tables hold.
void twiddle_host(int L, bool dbl, unsigned char* dst) {
  const long double tau = 6.283185307179586476925286766559005768L;
  for (int j = 0; j < L; ++j) {
    const long double a = tau * (long double)j / (long double)L;
    const double c = (double)cosl(a), s = (double)-sinl(a);
    if (dbl) {
      double2 v = make_double2(c, s);
      std::memcpy(dst + (size_t)j * 16, &v, 16);
    } else {
      float2 v = make_float2((float)c, (float)s);
      std::memcpy(dst + (size_t)j * 8, &v, 8);
    }
  }
}

}  // namespace

extern "C" int dda_matvec_noalloc(int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, const void* ghat,
                                  double gscale, const void* inv_alpha, int mode, const void* x, void* y,
                                  const void* b, void* stream) {
  using namespace dda;
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("bad dtype"); return DDA_ERR_ARG; }
  if (!ghat || !inv_alpha || !x || !y || (mode == DDA_MV_RESIDUAL && !b)) {
    set_error("null argument");
    return DDA_ERR_ARG;
  }
  if (mode < 0 || mode > 3) { set_error("bad matvec mode"); return DDA_ERR_ARG; }
  if (x == y) { set_error("x and y must not alias"); return DDA_ERR_ARG; }
  if (nx < 1 || ny < 1 || nz < 1 || Lx < 2 * nx || Ly < 2 * ny || Lz < 2 * nz || !fft_size_compiled(Lx) ||
      !fft_size_compiled(Ly) || !fft_size_compiled(Lz) || (dtype == DDA_C128 && 3 * std::max(Lx, std::max(Ly, Lz)) > 3072)) {
    set_error("dda_matvec_noalloc: bad box or FFT lengths");
    return DDA_ERR_BAD_SHAPE;
  }
  const size_t esz = dtype == DDA_C128 ? 16 : 8;
  const size_t t1n = (size_t)nx * ny * Lz * 3, t2n = (size_t)nx * Ly * Lz * 3;
  const size_t need = (t1n + t2n) * esz;
  if (need > kScratchBytes - kDataOff) {
    set_error("dda_matvec_noalloc: problem needs " + std::to_string(need) + " bytes of transform scratch, more than " +
              "the " + std::to_string(kScratchBytes - kDataOff) + " the static buffer holds; use dda_matvec");
    return DDA_ERR_BAD_SHAPE;
  }
  void* base = nullptr;
  int rc = scratch_base(&base);
  if (rc) return rc;
  unsigned char* B = (unsigned char*)base;
  cudaStream_t s = (cudaStream_t)stream;
  Geo g;
  g.nx = nx; g.ny = ny; g.nz = nz; g.Lx = Lx; g.Ly = Ly; g.Lz = Lz;
  g.hx = Lx / 2 + 1; g.hy = Ly / 2 + 1; g.hz = Lz / 2 + 1;
  g.nsite = (long long)nx * ny * nz;
  // twiddle tables (host-staged copies; no device allocation)
  static thread_local unsigned char tw_host[3][kTwStride];
  const int Ls[3] = {Lx, Ly, Lz};
  for (int a = 0; a < 3; ++a) {
    twiddle_host(Ls[a], dtype == DDA_C128, tw_host[a]);
    cudaError_t e = cudaMemcpyAsync(B + kTwOff + a * kTwStride, tw_host[a], (size_t)Ls[a] * esz,
                                    cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  }
  InstState S;
  std::memset(&S, 0, sizeof(S));
  S.vec[V_R] = (void*)x;
  S.vec[V_RHAT] = y;
  S.vec[V_B] = (void*)b;
  S.ghat = ghat;
  S.inva = inv_alpha;
  S.t1 = B + kDataOff;
  S.t2 = B + kDataOff + t1n * esz;
  S.active = 1;
  cudaError_t e = cudaMemcpyAsync(B + kStateOff, &S, sizeof(S), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  const PassCfg pc = make_pass_cfg(g, dtype == DDA_C128);
  InstState* st = (InstState*)(B + kStateOff);
  const void* twx = B + kTwOff, *twy = B + kTwOff + kTwStride, *twz = B + kTwOff + 2 * kTwStride;
  e = dtype == DDA_C128 ? launch_matvec_tw<double>(g, pc, st, twx, twy, twz, V_R, V_RHAT, mode, gscale, s)
                        : launch_matvec_tw<float>(g, pc, st, twx, twy, twz, V_R, V_RHAT, mode, gscale, s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}
