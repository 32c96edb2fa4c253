// Coulomb energy without any device allocation.
//
// pbgpu_energy computes the Coulomb term sum_{i<j} q_i q_j / r_ij / eps_in over
// the charged atoms with scratch it allocates per call (a compacted copy of the
// charged atoms and one partial sum per block).  Some callers cannot allocate
// device memory at all: code that runs inside another library's enqueue or
// plugin callback, where allocating is not permitted, or a process whose device
// memory is owned entirely by a pool allocator it must not go around.  For them,
// pbgpu_coulomb_energy_static computes the same quantity from caller-owned
// input and output buffers, with its scratch in the fixed arrays below:
//
//   g_atoms     kStaticMaxAtoms double4 (x, y, z, q)  = 4 MiB
//   g_partials  kStaticBlocks doubles                  = 4 KiB
//   g_ticket    one counter for the last-block reduction
//
// Every GPU that loads this library holds these 4 MiB until the process exits.
// All calls share them: two calls whose work overlaps on the GPU (different
// streams, or different host threads) race and must be serialised by the
// caller.  The arrays keep the last call's contents; each call rewrites the
// atom copy and the partials before reading them, and the last block resets the
// counter to zero after use.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "pbgpu_internal.cuh"

namespace pbgpu {

constexpr int64_t kStaticMaxAtoms = 131072;
constexpr int kStaticBlocks = 512;
constexpr int kStaticThreads = 256;

static __device__ __align__(256) double4 g_atoms[kStaticMaxAtoms];
static __device__ __align__(256) double g_partials[kStaticBlocks];
static __device__ __align__(256) unsigned int g_ticket;

// Device addresses of the arrays, looked up once per device with that device
// current (in host code the symbols are only host-side stand-ins).  They are
// addresses in the device's primary context, the one the CUDA runtime uses;
// the cache is never invalidated, so after cudaDeviceReset (which unloads the
// module) or from another context the cached addresses would be stale: the
// entry point is for processes that keep the primary context for their life.
struct StaticScratch {
  double4* atoms = nullptr;
  double* partials = nullptr;
  unsigned int* ticket = nullptr;
  bool ready = false;
};
static StaticScratch g_scratch[64];
static std::mutex g_scratch_mu;

// Atom copy with charges below the reference's threshold (|q| <= 1e-5,
// src/pb_class.cpp:2829-2834) set to zero, so they drop out of the sum.
__global__ void k_static_copy(const double* __restrict__ in, int64_t n, double4* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double q = in[4 * i + 3];
    out[i] = make_double4(in[4 * i], in[4 * i + 1], in[4 * i + 2], fabs(q) > 1.e-5 ? q : 0.0);
  }
}

__device__ __forceinline__ double rsqrt_nr_static(double x) {
  double y = (double)rsqrtf((float)x);
  y = y * (1.5 - 0.5 * x * y * y);
  y = y * (1.5 - 0.5 * x * y * y);
  return y;
}

// Pairs i < j in tiles staged in shared memory; block partials into the static
// array, the last block to finish sums them in block order and writes the
// energy to the caller's output.
__global__ void __launch_bounds__(kStaticThreads) k_static_coulomb(const double4* __restrict__ atoms, int64_t m,
                                                                   double inv_eps_in, double* __restrict__ partials,
                                                                   unsigned int* __restrict__ ticket,
                                                                   double* __restrict__ out) {
  __shared__ double4 tile[kStaticThreads];
  __shared__ double red[kStaticThreads / 32];
  __shared__ bool last;
  double acc = 0.0;
  for (int64_t base = blockIdx.x * (int64_t)kStaticThreads; base < m; base += (int64_t)gridDim.x * kStaticThreads) {
    const int64_t i = base + threadIdx.x;
    const double4 P = i < m ? atoms[i] : make_double4(0, 0, 0, 0);
    double s = 0.0;
    for (int64_t a0 = base; a0 < m; a0 += kStaticThreads) {
      __syncthreads();
      if (a0 + threadIdx.x < m) tile[threadIdx.x] = atoms[a0 + threadIdx.x];
      __syncthreads();
      // an uncharged row adds nothing: it skips its pairs (a zero charge on
      // top of a charged atom would otherwise give 0 * inf), but still takes
      // part in every tile load and barrier of the block
      if (P.w == 0.0) continue;
      const int lim = (int)min((int64_t)kStaticThreads, m - a0);
      for (int j = 0; j < lim; ++j) {
        if (a0 + j <= i) continue;
        const double4 A = tile[j];
        if (A.w == 0.0) continue;
        const double dx = P.x - A.x, dy = P.y - A.y, dz = P.z - A.z;
        s += A.w * rsqrt_nr_static(dx * dx + dy * dy + dz * dz);
      }
    }
    if (i < m && P.w != 0.0) acc += P.w * s;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < kStaticThreads / 32; ++w) b += red[w];
    partials[blockIdx.x] = b;
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) t += __ldcg(partials + b);
    *out = t * inv_eps_in;
    *ticket = 0;
  }
}

}  // namespace pbgpu

using namespace pbgpu;

extern "C" int pbgpu_coulomb_energy_static(const double* atoms, int64_t n_atoms, double e_in, double T,
                                           double* out_energy, void* cuda_stream) {
  if (!atoms || !out_energy || n_atoms < 0 || !(e_in > 0) || !(T > 0)) return PBGPU_ERR_ARG;
  if (n_atoms > kStaticMaxAtoms) {
    std::fprintf(stderr, "pbgpu_coulomb_energy_static: %lld atoms exceed the fixed scratch of %lld atoms\n",
                 (long long)n_atoms, (long long)kStaticMaxAtoms);
    return PBGPU_ERR_CAPACITY;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return PBGPU_ERR_CUDA;
  }
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  StaticScratch& S = g_scratch[dev];
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!S.ready) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_atoms) != cudaSuccess) return PBGPU_ERR_CUDA;
      S.atoms = static_cast<double4*>(p);
      if (cudaGetSymbolAddress(&p, g_partials) != cudaSuccess) return PBGPU_ERR_CUDA;
      S.partials = static_cast<double*>(p);
      if (cudaGetSymbolAddress(&p, g_ticket) != cudaSuccess) return PBGPU_ERR_CUDA;
      S.ticket = static_cast<unsigned int*>(p);
      S.ready = true;
    }
  }
  // eps_in in the reference's units (src/pb_class.cpp:1800)
  const double e_0 = 8.85418781762e-12, kb = 1.380649e-23, e = 1.602176634e-19, Angs = 1e-10;
  const double eps_in = 4.0 * kPi * e_0 * e_in * kb * T * Angs / (e * e);
  if (n_atoms < 2) {
    // no pair: the energy is zero, written on the stream like any other result
    // (all-zero bytes are +0.0); nothing here waits for the stream
    return cudaMemsetAsync(out_energy, 0, sizeof(double), stream) == cudaSuccess ? PBGPU_OK : PBGPU_ERR_CUDA;
  }
  if (cudaMemsetAsync(S.ticket, 0, sizeof(unsigned int), stream) != cudaSuccess) return PBGPU_ERR_CUDA;
  k_static_copy<<<kStaticBlocks, kStaticThreads, 0, stream>>>(atoms, n_atoms, S.atoms);
  int64_t blocks = (n_atoms + kStaticThreads - 1) / kStaticThreads;
  if (blocks > kStaticBlocks) blocks = kStaticBlocks;
  k_static_coulomb<<<(int)blocks, kStaticThreads, 0, stream>>>(S.atoms, n_atoms, 1.0 / eps_in, S.partials, S.ticket,
                                                               out_energy);
  if (cudaGetLastError() != cudaSuccess) return PBGPU_ERR_CUDA;
  return PBGPU_OK;
}
