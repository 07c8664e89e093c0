// CPU emulation prelude for running the reference's CUDA-C kernel strings
// (TEST INFRASTRUCTURE ONLY).  Kernel bodies are compiled unchanged as C++;
// this header supplies what they use from CUDA/CuPy: thread and block
// indices, complex<T>, __shared__, __syncthreads.  Blocks run one after the
// other; threads of a block run as cooperative fibers so that a barrier
// switches to the next thread (see fibers.cpp).
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstddef>

template <class T> using complex = std::complex<T>;
using std::conj;
using std::exp;
using std::max;
using std::min;
using std::sqrt;

namespace refshim {
struct Idx { unsigned x, y, z; };
extern Idx g_thread, g_block, g_bdim, g_gdim;
void sync();
}  // namespace refshim

#define threadIdx refshim::g_thread
#define blockIdx refshim::g_block
#define blockDim refshim::g_bdim
#define gridDim refshim::g_gdim
#define __global__
#define __device__
#define __shared__ static
#define __syncthreads() refshim::sync()
