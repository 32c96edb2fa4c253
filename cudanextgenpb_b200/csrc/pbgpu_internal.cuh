// Internal declarations of libpbgpu: the context, device buffers and the
// device-side helpers shared by the kernels.  B200 (sm_100a) only.
#pragma once
#include <cuda_runtime.h>

#include <utility>
#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pbgpu.h"

namespace pbgpu {

constexpr int kRootLog = 19;
constexpr int32_t kRoot = 1 << kRootLog;
constexpr int kMaxRow = 96;         // distinct columns a matrix row may hold
constexpr int kMaxIncidence = 160;  // (octant, corner) incidences of one node
constexpr uint64_t kEmptyKey = ~0ull;

// ---------------------------------------------------------------------------
// Device bytes held per context: a buffer charges the counter that is current
// on this thread when it allocates (AcctScope, set at every API entry) and
// credits the same counter when it frees.
inline thread_local int64_t* tl_acct = nullptr;

struct AcctScope {
  int64_t* prev;
  explicit AcctScope(int64_t* a) : prev(tl_acct) { tl_acct = a; }
  ~AcctScope() { tl_acct = prev; }
};

// Stream-ordered allocation.  Inside an API call on a context (StreamScope,
// set with the accounting scope) buffers come from a per-device pool on the
// stream the call works on, and go back to the pool on that stream: growing
// a buffer then waits for nothing but that stream.  A cudaFree would wait for
// the whole device -- every other context's work and a running batch kernel
// -- which serialised contexts that are reused for systems of varying sizes.
// Outside such a scope, and while the stream is being captured into a graph,
// buffers use cudaMalloc / cudaFree.
inline thread_local cudaStream_t tl_stream = nullptr;
inline thread_local bool tl_pooled = false;

// Pool blocks a context's buffers released inside one of its API calls,
// kept for reuse by later allocations of the same context on the same stream
// instead of going back to the pool: the mesh build and the set-up allocate
// and free hundreds of temporaries per request, and a pool allocation costs
// microseconds (tens while several contexts allocate at once).  Reuse on the
// stream the block was freed on is ordered as the pool's own reuse is.  A
// cached block counts as freed in the context's byte count, as memory the
// pool caches does; at most kMaxBytes are kept, and flush() returns them to
// the pool (when the context is destroyed, or when an allocation finds the
// device full).
struct BlockCache {
  struct Blk {
    void* p;
    size_t bytes;
  };
  static constexpr size_t kMaxBlocks = 512;
  static constexpr size_t kMaxBytes = size_t(128) << 20;
  cudaStream_t s = nullptr;  // the context's stream
  int64_t* acct = nullptr;   // the context's byte count (identifies the owner)
  std::vector<Blk> blks;
  size_t bytes = 0;
  // the smallest cached block of want .. 2 want (+ 64 KiB) bytes, or null
  void* take(size_t want, size_t* got) {
    int best = -1;
    for (size_t i = 0; i < blks.size(); ++i)
      if (blks[i].bytes >= want && blks[i].bytes <= 2 * want + 65536 &&
          (best < 0 || blks[i].bytes < blks[best].bytes))
        best = (int)i;
    if (best < 0) return nullptr;
    void* q = blks[best].p;
    *got = blks[best].bytes;
    bytes -= *got;
    blks[best] = blks.back();
    blks.pop_back();
    return q;
  }
  bool put(void* q, size_t nb) {
    if (blks.size() >= kMaxBlocks || bytes + nb > kMaxBytes) return false;
    blks.push_back(Blk{q, nb});
    bytes += nb;
    return true;
  }
  void flush() {
    for (const Blk& b : blks) cudaFreeAsync(b.p, s);
    blks.clear();
    bytes = 0;
  }
};
inline thread_local BlockCache* tl_cache = nullptr;

struct StreamScope {
  cudaStream_t prev;
  bool prev_pooled;
  BlockCache* prev_cache;
  explicit StreamScope(cudaStream_t s, BlockCache* cache = nullptr)
      : prev(tl_stream), prev_pooled(tl_pooled), prev_cache(tl_cache) {
    tl_stream = s;
    tl_pooled = true;
    tl_cache = cache;
  }
  ~StreamScope() {
    tl_stream = prev;
    tl_pooled = prev_pooled;
    tl_cache = prev_cache;
  }
};

// The library's memory pool on the current device (created on first use;
// freed memory stays in it for reuse until pool_trim); null if the device has
// no memory pools.
cudaMemPool_t device_pool();
// Returns the unused memory of the current device's pool to the device.
void pool_trim();

inline bool stream_capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
    cudaGetLastError();
    return true;  // unknown: take the plain path
  }
  return st != cudaStreamCaptureStatusNone;
}

// Device buffer owned by a context.
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  size_t nbytes = 0;  // the block's size (a cached block may exceed n * sizeof(T))
  int64_t* acct = nullptr;
  cudaStream_t s = nullptr;  // stream of a pool allocation
  bool pooled = false;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) {
      const bool kept = pooled && acct && tl_cache && tl_cache->s == s && tl_cache->acct == acct &&
                        tl_cache->put(p, nbytes);
      if (!kept) {
        if (pooled)
          cudaFreeAsync(p, s);
        else
          cudaFree(p);
      }
      if (acct) *acct -= (int64_t)nbytes;
    }
    p = nullptr;
    n = 0;
    nbytes = 0;
    acct = nullptr;
    s = nullptr;
    pooled = false;
  }
  cudaError_t alloc(size_t count) {
    if (count <= n && p) return cudaSuccess;
    release();
    if (count == 0) return cudaSuccess;
    const size_t bytes = count * sizeof(T);
    cudaError_t e;
    cudaMemPool_t pool = (tl_pooled && !stream_capturing(tl_stream)) ? device_pool() : nullptr;
    if (pool) {
      BlockCache* bc = (tl_acct && tl_cache && tl_cache->s == tl_stream && tl_cache->acct == tl_acct) ? tl_cache : nullptr;
      size_t got = 0;
      void* q = bc ? bc->take(bytes, &got) : nullptr;
      if (q) {
        p = reinterpret_cast<T*>(q);
        pooled = true;
        s = tl_stream;
        n = got / sizeof(T);
        nbytes = got;
        acct = tl_acct;
        *acct += (int64_t)got;
        return cudaSuccess;
      }
      e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), bytes, pool, tl_stream);
      if (e == cudaErrorMemoryAllocation && bc && bc->bytes) {  // the cache's blocks first
        cudaGetLastError();
        bc->flush();
        e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), bytes, pool, tl_stream);
      }
      if (e == cudaSuccess) {
        pooled = true;
        s = tl_stream;
      }
    } else {
      e = cudaMalloc(&p, bytes);
      if (e == cudaErrorMemoryAllocation) {  // memory cached in the pool is not cudaMalloc's
        cudaGetLastError();
        pool_trim();
        e = cudaMalloc(&p, bytes);
      }
    }
    if (e == cudaSuccess) {
      n = count;
      nbytes = bytes;
      acct = tl_acct;
      if (acct) *acct += (int64_t)bytes;
    } else {
      p = nullptr;
    }
    return e;
  }
  T* get() const { return p; }
  void swap(DBuf& o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
    std::swap(nbytes, o.nbytes);
    std::swap(acct, o.acct);
    std::swap(s, o.s);
    std::swap(pooled, o.pooled);
  }
};

struct Rays {
  int64_t n = 0;          // rays with crossings
  int64_t nc = 0;         // crossings
  int64_t cap = 0;        // hash capacity (power of two)
  int cap_log = 0;
  DBuf<uint64_t> keys;    // key of each ray (ascending)
  DBuf<uint64_t> hkeys;   // open-addressing table of ray keys
  DBuf<int32_t> hval;     // ray index of each slot
  DBuf<int64_t> ptr;
  DBuf<double> inters;
  DBuf<double> normals;
};

// Krylov scalars kept on the device (one struct, updated by the last block of
// each reducing kernel).
struct KrylovScalars {
  double rz, rz_new, pq, alpha, beta, omega, rho, rr, bb, ss, ts, tt, rv;
  double tol2;            // tol^2 * ||b||^2
  double r1, b1, tol1;    // ||r||_1, ||b||_1, tol_w ||b||_1 + tol (LIS conv_cond 2)
  int conv;               // 2: stop on the 1-norm rule, else on the 2-norm rule
  int ru;                 // FP32 CG with reliable updates: 1 while an FP64 residual is due
  int fold;               // 1 from that FP64 residual until the next p-update has folded d into x
  int reliable;           // reliable updates on (the FP64 residual decides convergence)
  double rr_ref, delta2;  // ||r||^2 at the last FP64 residual; update when rr < delta2 rr_ref
  int iter, max_iter, done, status, s_conv;
  unsigned int ticket[8]; // last-block tickets, one per reducing kernel
  unsigned long long wait_ns;  // limit of each bounded wait of the staged SpMV (0: give up at once)
};

// Element j of the SELL row in lane `lane` of a slice that starts at element
// `base` and has width W (columns), height C and column-group width G: the
// first W - W % G columns are stored in groups of G lane-interleaved (a
// thread loads a group with one vector load, a warp's loads of one group are
// contiguous), the last W % G columns one per lane.  The assembly pads W to a
// multiple of G, so the tail is empty for its matrices.
__host__ __device__ __forceinline__ int64_t sell_elem(int64_t base, int W, int C, int G, int lane, int j) {
  const int Wg = W - W % G;
  if (j < Wg) return base + (int64_t)(j / G) * G * C + (int64_t)lane * G + j % G;
  return base + (int64_t)Wg * C + (int64_t)(j - Wg) * C + lane;
}

// Scratch slots of a context: one per stage-local buffer.
enum ScratchSlot {
  kScMkOvf, kScMkFlags, kScMkSel, kScMkNsel,
  kScDenCnt, kScDenK0, kScDenK1, kScDenV0, kScDenV1,
  kScAsmOvf, kScAsmK0, kScAsmK1, kScAsmId0, kScAsmElems, kScAsmNnz, kScAsmCond, kScAsmKd, kScAsmFr,
  kScAsmCols, kScAsmVals, kScAsmRhs, kScAsmUcnt,
  kScKrBad, kScKrRh32, kScKrV32, kScKrS32, kScKrT32, kScKrPh32, kScKrSh32,
  kScEnPhi, kScEnQ, kScEnAcc, kScEnUsed, kScEnSlotRay, kScEnSel, kScEnNsel, kScEnNextra, kScEnXp, kScEnXd,
  kScEnP, kScEnD, kScEnXk, kScEnXk2, kScEnXi, kScEnXi2, kScPfAtoms, kScPfPart, kScPfOut,
  kScInOctXyz, kScInOctLvl, kScInNodeXyz, kScInHangNp, kScInHangPar, kScInErr,
  kScratchSlots
};

struct Context;

// Small device-to-host reads (counts, totals, flags, block partials) go
// through the context's pinned scratch and wait for its stream.  A copy into
// pageable memory is staged by the driver through buffers that the threads of
// the process share, which serialised the set-up of requests running on
// concurrent worker contexts.  Larger reads copy directly.
constexpr size_t kReadbackBytes = 65536;
inline cudaError_t readback(Context* c, void* dst, const void* src, size_t bytes);

// A typed view of one scratch slot with DBuf's alloc() / get() interface.
template <typename T>
struct Scratch {
  DBuf<uint8_t>* slot;
  T* p = nullptr;
  Scratch(Context* c, int which);
  cudaError_t alloc(size_t count) {
    const cudaError_t e = slot->alloc(count * sizeof(T) > 0 ? count * sizeof(T) : 1);
    p = reinterpret_cast<T*>(slot->get());
    return e;
  }
  T* get() const { return p; }
  void release() {
    slot->release();
    p = nullptr;
  }
};

struct Context {
  int64_t dev_bytes = 0;     // device memory held by this context's buffers
  BlockCache blk_cache;      // blocks its buffers released, for reuse on its stream
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t evc[2] = {nullptr, nullptr};  // ends of the two Krylov chunks in flight
  double stage_ms[6] = {0, 0, 0, 0, 0, 0};

  // ---- mesh
  int64_t n_oct = 0, n = 0, nh = 0;
  double lo[3] = {0, 0, 0}, len[3] = {0, 0, 0}, tol = 0;
  DBuf<int4> oct;            // x, y, z, level
  DBuf<uint64_t> oct_key;    // Morton key of the lower corner
  DBuf<int32_t> oct_nodes;   // 8 per octant
  DBuf<int4> node_xyz;       // x, y, z, boundary flag
  DBuf<int4> hang_par;       // 4 parents, -1 padded
  DBuf<int8_t> hang_np;
  bool have_mesh = false;

  Rays rays[3];
  bool have_rays[3] = {false, false, false};

  // ---- atoms
  int64_t na = 0;
  DBuf<double4> atoms;       // x, y, z, q
  bool have_atoms = false;

  // ---- model
  pbgpu_model model{};
  double eps_in = 0, eps_out = 0, k2 = 0, kappa = 0;
  bool have_model = false;

  // ---- markers
  DBuf<uint8_t> inside;      // per node
  DBuf<double> eps, react;   // per node
  DBuf<uint8_t> marker;      // per octant: 0 in, 1 border, 2 out
  DBuf<double> react_cell;   // per octant (Stern layer)
  DBuf<int32_t> border;      // border octants, ascending
  DBuf<int32_t> border_pos;  // octant -> border position or -1
  DBuf<double> frac;         // 12 per border octant
  int64_t nb = 0;
  bool have_markers = false;

  // ---- incidence (node -> (octant, corner))
  DBuf<int64_t> inc_ptr;
  DBuf<uint32_t> inc;
  bool have_incidence = false;

  // ---- density
  DBuf<double> vol_patch, rho;
  DBuf<int32_t> atom_oct;    // octant of each atom or -1
  bool have_density = false;

  // ---- system in SELL-C-sigma (rows permuted; vectors live in SELL order)
  int C = 32, sigma = 2048, G = 1;
  int spmv_cols = 16;        // staged SpMV chunk width (8, 12 or 16 columns)
  int64_t n_slices = 0, nnz = 0, sell_len = 0;
  DBuf<int64_t> slice_ptr;   // element offset of each slice
  DBuf<int32_t> slice_w;     // width (multiple of 4) of each slice
  DBuf<int32_t> perm;        // SELL position -> node
  DBuf<int32_t> iperm;       // node -> SELL position
  DBuf<int32_t> scol;        // column (SELL numbering)
  DBuf<double> sval;
  DBuf<float> sval32;        // fp32 copy for the mixed-precision inner solve
  DBuf<double> b;            // right-hand side (SELL order)
  DBuf<double> dinv;         // 1 / diagonal (SELL order)
  DBuf<int32_t> rowlen;      // per node
  DBuf<uint8_t> dirichlet;   // per node
  DBuf<double> gval;         // Dirichlet value per node
  bool have_system = false;

  // ---- solve
  DBuf<double> x, r, p, q, z, rh, v, s, t, ph, sh;   // fp64 work vectors (SELL order)
  DBuf<float> x32, r32, p32, q32, b32, dinv32, z32; // fp32 inner vectors
  DBuf<double> ones;         // the "no preconditioner" diagonal
  DBuf<float> ones32;
  DBuf<float> bjinv;         // block-Jacobi inverse blocks (node order)
  // many right-hand sides: n_pad x kp blocks (row-major), per-column scalars
  DBuf<double> mr_b, mr_x, mr_r, mr_p, mr_q, mr_scal, mr_part, mr_q_dev;
  DBuf<int> mr_int;
  bool bj_ready = false;     // bjinv belongs to the current system
  DBuf<double> partials;     // block partial sums
  DBuf<KrylovScalars> ks;
  KrylovScalars* ks_host = nullptr;   // pinned mirror
  void* rb_host = nullptr;            // pinned scratch of small device-to-host reads (readback)
  DBuf<double> phi;          // node order
  bool have_phi = false;
  int sm_count = 148;
  double wait_s = 1.0;       // limit of each bounded device-side wait (pbgpu_set_wait_limit)

  // ---- energy scratch
  DBuf<double4> elem_a;      // element position + coefficient
  DBuf<double4> elem_b;      // element normal (triangle vertices)
  DBuf<int32_t> elem_cnt;
  DBuf<double> energy_part;

  // ---- scratch for CUB
  DBuf<uint8_t> tmp;

  // ---- per-stage scratch, kept between calls (grow-only) so a repeated
  // stage neither allocates nor frees device memory (cudaFree synchronises
  // the device and large cudaMalloc calls take milliseconds)
  DBuf<uint8_t> scratch[kScratchSlots];

  // ---- measurement
  bool profiling = false;
  int64_t launches = 0;       // kernels launched (CUB device algorithms count their kernels)
  int64_t spmv_launches = 0;
  double spmv_ms = 0.0;
  double spmv_bytes = 0.0;
  int64_t krylov_iters = 0;
  int64_t energy_points = 0;  // surface points of the last energy call
  int64_t energy_pairs = 0;   // point x charged-atom pairs evaluated

  int fail(int code, const std::string& msg) {
    err = msg;
    return code;
  }
};

inline cudaError_t readback(Context* c, void* dst, const void* src, size_t bytes) {
  if (!c->rb_host || bytes > kReadbackBytes) {
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
    return e != cudaSuccess ? e : cudaStreamSynchronize(c->stream);
  }
  cudaError_t e = cudaMemcpyAsync(c->rb_host, src, bytes, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) std::memcpy(dst, c->rb_host, bytes);
  return e;
}

template <typename T>
Scratch<T>::Scratch(Context* c, int which) : slot(&c->scratch[which]) {}

int cuda_fail(Context* c, cudaError_t e, const char* what);


#define PBGPU_STR2(x) #x
#define PBGPU_STR(x) PBGPU_STR2(x)
#define PBGPU_CUDA(ctx, expr)                                                                            \
  do {                                                                                                   \
    cudaError_t _e = (expr);                                                                             \
    if (_e != cudaSuccess) return ::pbgpu::cuda_fail((ctx), _e, __FILE__ ":" PBGPU_STR(__LINE__) " " #expr); \
  } while (0)

// After a kernel launch: count it and check the launch.
#define PBGPU_LAUNCHED(ctx)                          \
  do {                                               \
    (ctx)->launches += 1;                            \
    PBGPU_CUDA(ctx, cudaGetLastError());             \
  } while (0)

// Kernels launched by one CUB device-wide call (CUB of CUDA 12.9): scans and
// flagged selects run an init kernel and a sweep kernel; a radix sort of 64-bit
// keys runs one single-tile kernel for small inputs, otherwise a histogram, an
// exclusive-sum and one onesweep pass per 8 key bits.
constexpr int kCubScanLaunches = 2;
constexpr int kCubSelectLaunches = 2;
inline int cub_radix_launches(int64_t n, int bits) { return n <= 3584 ? 1 : 2 + (bits + 7) / 8; }

// ---------------------------------------------------------------------------
// Device helpers.

// lo + len * (i * 2^-19) with one rounding per operation, never contracted.
__device__ __forceinline__ double coord(double lo, double len, int32_t i) {
  return __dadd_rn(lo, __dmul_rn(len, (double)i * 0x1p-19));
}

// Morton key of integer octree coordinates (x in the lowest bit).
// x^{-1/2}: the FP32 hardware estimate refined by Newton-Raphson steps
// y <- y (3 - x y^2) / 2, each squaring the relative error: one step
// (~2.4e-7 -> ~1e-13) for the surface-point x atom pairs, whose kernel is
// FP64-pipe bound and whose energies are held to 1e-10; two (-> below double
// rounding) for the Coulomb sum, compared at 1e-12.
__device__ __forceinline__ double rsqrt_nr1(double x) {
  const double y = (double)rsqrtf((float)x);
  return y * (1.5 - 0.5 * x * y * y);
}

__device__ __forceinline__ double rsqrt_nr(double x) {
  double y = (double)rsqrtf((float)x);
  y = y * (1.5 - 0.5 * x * y * y);
  y = y * (1.5 - 0.5 * x * y * y);
  return y;
}

__device__ __forceinline__ uint64_t spread3(uint64_t v) {
  v &= 0x1fffffULL;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}

__device__ __forceinline__ uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

// Point coordinates run 0 .. 2^kRootLog (kRootLog + 1 bits): a Morton code
// of a point uses 3 (kRootLog + 1) bits, a ray key 2 (kRootLog + 1).
constexpr int kMortonBits = 3 * (kRootLog + 1);
constexpr int kRayKeyBits = 2 * (kRootLog + 1);
static_assert(kRootLog + 1 <= 20, "ray keys hold 20 bits per coordinate");

__device__ __forceinline__ uint64_t ray_key(int32_t a, int32_t b) {
  return ((uint64_t)(uint32_t)a << 20) | (uint64_t)(uint32_t)b;
}

__device__ __forceinline__ uint64_t hash_slot(uint64_t key, int cap_log) {
  return (key * 0x9E3779B97F4A7C15ull) >> (64 - cap_log);
}

// Ray index of `key` or -1.
__device__ __forceinline__ int32_t ray_find(const uint64_t* __restrict__ hk, const int32_t* __restrict__ hv,
                                            int64_t cap, int cap_log, uint64_t key) {
  if (cap == 0) return -1;
  uint64_t s = hash_slot(key, cap_log);
  for (int64_t probe = 0; probe < cap; ++probe) {
    const uint64_t k = hk[s];
    if (k == key) return hv[s];
    if (k == kEmptyKey) return -1;
    s = (s + 1) & (uint64_t)(cap - 1);
  }
  return -1;
}

struct RayView {
  const uint64_t* hk;
  const int32_t* hv;
  const int64_t* ptr;
  const double* inters;
  const double* normals;
  const uint64_t* keys;
  int64_t cap;
  int cap_log;
};

inline RayView ray_view(const Rays& r) {
  return RayView{r.hkeys.get(), r.hval.get(), r.ptr.get(), r.inters.get(), r.normals.get(), r.keys.get(),
                 r.cap, r.cap_log};
}

// Which axis edge e runs along, and its two corners (reference edge table,
// include/pb_class.h:190-207).
__device__ __constant__ static const int8_t d_edge_nodes[24] = {0, 1, 1, 3, 2, 3, 0, 2, 4, 5, 5, 7,
                                                                  6, 7, 4, 6, 0, 4, 1, 5, 3, 7, 2, 6};
__device__ __constant__ static const int8_t d_edge_axis[12] = {0, 1, 0, 1, 0, 1, 0, 1, 2, 2, 2, 2};

// Edges meeting at corner c: the edge along axis a is the one whose corner
// pair is (c with bit a cleared, c with bit a set).
__device__ __forceinline__ int edge_of(int c, int axis) {
  // edges along x: 0 (0-1), 2 (2-3), 4 (4-5), 6 (6-7): 2 * (c >> 1)
  // edges along y: 3 (0-2), 1 (1-3), 7 (4-6), 5 (5-7): by the x and z bits
  // edges along z: 8 (0-4), 9 (1-5), 11 (2-6), 10 (3-7): 8 + Gray code of (x, y)
  if (axis == 0) return c & 6;
  if (axis == 1) return 3 + 4 * ((c >> 2) & 1) - 2 * (c & 1);
  const int t = c & 3;
  return 8 + (t ^ (t >> 1));
}

__device__ __forceinline__ double wha(double e1, double e2, double f) { return 1.0 / (f / e1 + (1 - f) / e2); }

// physical constants of the reference (include/pb_class.h:47-54)
constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Stage entry points (implemented per .cu file).
int build_ray_hash_from(Context* c, int axis, const uint64_t* d_keys);
int run_markers(Context* c);
int build_incidence(Context* c);
int run_density(Context* c);
int run_assemble(Context* c, const pbgpu_sell_opts* o);
int run_solve(Context* c, const pbgpu_solver_opts* o, pbgpu_solve_stats* st);
int run_phi_atoms(Context* c, double* out);
int run_energy(Context* c, int fast, pbgpu_energy_out* out);
// surface points of the energy integrals, merged per crossing (k_energy.cu)
struct SurfacePoints {
  const double4* P;  // V, F
  const double4* D;  // sum of coef * N (ionic)
  int64_t n;
};
int surface_points(Context* c, int fast, bool ionic, SurfacePoints* out);
int run_pot_field(Context* c, int fast, int calc_potential_term, int calc_field_term, double* per_atom,
                  pbgpu_pot_field_out* out);
int run_rhs(Context* c);
bool tuned_layout(int64_t n, pbgpu_sell_opts* sell, int* cols);
int run_solve_charges(Context* c, int k, const double* charges, const pbgpu_solver_opts* opts, int fast,
                      pbgpu_energy_out* energies, pbgpu_solve_stats* stats);
int export_system(Context* c, int64_t* nnz, int64_t* row_ptr, int32_t* col, double* val, double* rhs);

// scratch for CUB temporaries
cudaError_t ensure_tmp(Context* c, size_t bytes);
}  // namespace pbgpu
struct pbgpu_batch;
namespace pbgpu {
// persistent kernels a batch has launched (k_batch.cu)
int64_t batch_launch_count(const pbgpu_batch* b);
// Morton keys of the octants' lower corners
void launch_oct_keys(const int4* oct, int64_t n_oct, uint64_t* key, cudaStream_t s);

inline int grid_for(int64_t n, int block) { return (int)((n + block - 1) / block); }

}  // namespace pbgpu

struct pbgpu_ctx {
  pbgpu::Context c;
};
