// Allocation-free A.x: dda_matvec_noalloc.
//
// Some callers cannot allocate device memory at the point where they need the
// DDA product: serving or real-time loops whose latency budget forbids
// allocator calls (cudaMalloc may synchronise the whole device and takes an
// unbounded time), and host applications whose device memory belongs to
// another framework's caching pool, which must not be bypassed by raw
// cudaMalloc calls.  This entry point computes the same product as dda_matvec
// without any allocation: the transform scratch (the T1/T2 buffers of the
// five passes), the per-call state block and the FFT twiddle tables all live
// in one file-scope __device__ array of DDA_NOALLOC_SCRATCH_BYTES (64 MiB),
// which every GPU that loads this library holds until the process exits.
//
// Set-up: the first call on each device (with that device current) looks up
// the array's device address with cudaGetSymbolAddress and writes the twiddle
// tables of every compiled FFT length into it with one synchronous host to
// device copy; make that first call before any stream capture.  After that a
// call only enqueues kernels: a one-thread kernel that takes the state block
// by value and stores it into the array, then the five matvec passes.  Every
// call shares the one array and leaves its contents behind for the next call;
// the state block is rewritten by every call and the transform passes
// overwrite every scratch element they read, so nothing has to start at zero.
// Calls that overlap on the GPU (different streams, or different host threads
// without ordering) race on the array and must not be issued.
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/dda_b200.h"
#include "dda_host.h"
#include "fft_sizes.h"

namespace {

// Array layout: [state block | twiddle tables | T1 | T2].
constexpr size_t kScratchBytes = DDA_NOALLOC_SCRATCH_BYTES;
constexpr size_t kStateOff = 0;
constexpr size_t kTwOff = 4096;
// Sum of the compiled FFT lengths: each length has a complex64 table
// (8 bytes per entry) followed by a complex128 one (16 bytes per entry).
constexpr int kMaxL = 512;
constexpr int kSumL = 0
#define DDA_SUM(n) + n
    DDA_FFT_SIZES(DDA_SUM)
#undef DDA_SUM
    ;
constexpr size_t kTwBytes = (size_t)kSumL * 24;
constexpr size_t kDataOff = (kTwOff + kTwBytes + 4095) / 4096 * 4096;
static_assert(sizeof(dda::InstState) <= kTwOff, "state block overlaps the twiddle tables");
static_assert(kTwOff + kTwBytes <= kDataOff, "twiddle tables overlap the transform scratch");
static_assert(kDataOff < kScratchBytes, "no room for transform scratch");
static_assert(kDataOff % 256 == 0, "transform scratch must stay 256-byte aligned");
#define DDA_MAXL(n) static_assert(n <= kMaxL, "compiled FFT length above the table bound");
DDA_FFT_SIZES(DDA_MAXL)
#undef DDA_MAXL

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Byte offset of length L's complex64 table inside the twiddle region (the
// complex128 table follows it at + 8 L); -1 for a length not compiled.
long long tw_offset(int L) {
  long long off = 0;
#define DDA_OFF(n)                 \
  if (L == n) return off;          \
  off += 24LL * n;
  DDA_FFT_SIZES(DDA_OFF)
#undef DDA_OFF
  return -1;
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_base[kMaxDevices] = {};

// Twiddles exp(-2 pi i j/L) from extended-precision cos/sin, the same values
// the context tables of the allocating entry points hold.
void twiddle_host(int L, unsigned char* dst64, unsigned char* dst128) {
  const long double tau = 6.283185307179586476925286766559005768L;
  for (int j = 0; j < L; ++j) {
    const long double a = tau * (long double)j / (long double)L;
    const double c = (double)cosl(a), s = (double)-sinl(a);
    const double2 v = make_double2(c, s);
    const float2 f = make_float2((float)c, (float)s);
    std::memcpy(dst128 + (size_t)j * 16, &v, 16);
    std::memcpy(dst64 + (size_t)j * 8, &f, 8);
  }
}

// Device address of the scratch array on the current device; the first call
// per device also writes the twiddle tables (synchronous copy).
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
    std::vector<unsigned char> tw(kTwBytes);
#define DDA_TW(n) twiddle_host(n, tw.data() + tw_offset(n), tw.data() + tw_offset(n) + 8 * n);
    DDA_FFT_SIZES(DDA_TW)
#undef DDA_TW
    e = cudaMemcpy((unsigned char*)p + kTwOff, tw.data(), kTwBytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      dda::set_error(std::string("twiddle table set-up failed: ") + cudaGetErrorString(e));
      return DDA_ERR_CUDA;
    }
    g_base[dev] = p;
  }
  *out = g_base[dev];
  return DDA_OK;
}

// Stores the call's state block (a kernel parameter, so the values travel
// with the launch) into the scratch array.
__global__ void k_noalloc_state(dda::InstState S, dda::InstState* dst) { *dst = S; }

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
      !fft_size_compiled(Ly) || !fft_size_compiled(Lz)) {
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
  InstState* st = (InstState*)(B + kStateOff);
  k_noalloc_state<<<1, 1, 0, s>>>(S, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  const PassCfg pc = make_pass_cfg(g, dtype == DDA_C128);
  const size_t dsel = dtype == DDA_C128 ? 1 : 0;
  auto tw = [&](int L) -> const void* { return B + kTwOff + tw_offset(L) + dsel * 8 * L; };
  e = dtype == DDA_C128 ? launch_matvec_tw<double>(g, pc, st, tw(Lx), tw(Ly), tw(Lz), V_R, V_RHAT, mode, gscale, s)
                        : launch_matvec_tw<float>(g, pc, st, tw(Lx), tw(Ly), tw(Lz), V_R, V_RHAT, mode, gscale, s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}
