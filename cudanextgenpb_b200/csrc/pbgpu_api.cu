// extern "C" entry points of libpbgpu (include/pbgpu.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "pbgpu_internal.cuh"

namespace pbgpu {

int cuda_fail(Context* c, cudaError_t e, const char* what) {
  c->err = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a sticky-free error so the context stays usable
  return e == cudaErrorMemoryAllocation ? PBGPU_ERR_OOM : PBGPU_ERR_CUDA;
}

cudaError_t ensure_tmp(Context* c, size_t bytes) { return c->tmp.alloc(bytes > 0 ? bytes : 1); }

// One pool per device, kept for the life of the process.  Its release
// threshold is unlimited, so memory that a context frees stays cached for the
// next allocation on that device instead of going back at every
// synchronisation; pool_trim hands the unused part back (when a context is
// destroyed).
static std::mutex g_pool_mu;
static std::map<int, cudaMemPool_t> g_pools;

cudaMemPool_t device_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pools.find(dev);
  if (it != g_pools.end()) return it->second;
  cudaMemPool_t pool = nullptr;
  int supported = 0;
  if (cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, dev) == cudaSuccess && supported) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
      uint64_t threshold = UINT64_MAX;
      // Contexts on different streams share the pool.  By default the driver
      // may hand one stream memory another stream freed and make the first
      // wait for the second (internal dependencies), which chains concurrent
      // requests together; here memory moves between streams only once its
      // free is known to be complete.  PBGPU_POOL_CROSS_STREAM=1 restores the
      // driver's default.
      const char* cross = std::getenv("PBGPU_POOL_CROSS_STREAM");
      int reuse = (cross && cross[0] == '1') ? 1 : 0;
      if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold) != cudaSuccess ||
          cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &reuse) != cudaSuccess ||
          cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowOpportunistic, &reuse) != cudaSuccess) {
        cudaMemPoolDestroy(pool);
        pool = nullptr;
      }
    } else {
      pool = nullptr;
    }
  }
  cudaGetLastError();
  g_pools[dev] = pool;
  return pool;
}

void pool_trim() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) pool = it->second;
  }
  if (pool && cudaMemPoolTrimTo(pool, 0) != cudaSuccess) cudaGetLastError();
}

template <typename T>
static int upload(Context* c, DBuf<T>& d, const T* h, size_t count) {
  PBGPU_CUDA(c, d.alloc(count > 0 ? count : 1));
  if (count) PBGPU_CUDA(c, cudaMemcpyAsync(d.get(), h, count * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  return PBGPU_OK;
}

static void invalidate_from_mesh(Context* c) {
  c->have_markers = c->have_incidence = c->have_density = c->have_system = c->have_phi = false;
}

// Stage timing with CUDA events on the context stream.
struct StageTimer {
  Context* c;
  int idx;
  cudaEvent_t a = nullptr, b = nullptr;
  bool ok = false;
  StageTimer(Context* ctx, int i) : c(ctx), idx(i) {
    ok = cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess &&
         cudaEventRecord(a, c->stream) == cudaSuccess;
    if (!ok) cudaGetLastError();  // timing only: leave no error behind
  }
  ~StageTimer() {
    float ms = 0;
    if (ok && cudaEventRecord(b, c->stream) == cudaSuccess && cudaEventSynchronize(b) == cudaSuccess &&
        cudaEventElapsedTime(&ms, a, b) == cudaSuccess)
      c->stage_ms[idx] = ms;
    else
      cudaGetLastError();
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

int build_ray_hash_from(Context* c, int axis, const uint64_t* d_keys);

}  // namespace pbgpu

using namespace pbgpu;

#define CTX_CHECK(ctx) \
  if (!(ctx)) return PBGPU_ERR_ARG;
// Select the context's device and clear a non-sticky error that an earlier
// runtime call of this thread left behind (reported on stderr when PBGPU_DEBUG
// is set), so it is not blamed on this call's launches.
#define SET_DEVICE(C)                                                                         \
  AcctScope _acct(&(C)->dev_bytes);                                                           \
  StreamScope _sscope((C)->stream, &(C)->blk_cache);                                         \
  do {                                                                                        \
    cudaError_t _e = cudaSetDevice((C)->device);                                              \
    if (_e != cudaSuccess) return cuda_fail((C), _e, "cudaSetDevice");                        \
    const cudaError_t _stale = cudaGetLastError();                                            \
    if (_stale != cudaSuccess && std::getenv("PBGPU_DEBUG"))                                  \
      std::fprintf(stderr, "pbgpu: stale error before %s: %s\n", __func__, cudaGetErrorString(_stale)); \
  } while (0)

extern "C" {

int pbgpu_version(void) { return 1; }

int pbgpu_ctx_create(pbgpu_ctx** out, int device, void* cuda_stream) {
  if (!out) return PBGPU_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return PBGPU_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return PBGPU_ERR_ARG;
  pbgpu_ctx* h = new (std::nothrow) pbgpu_ctx();
  if (!h) return PBGPU_ERR_OOM;
  Context* c = &h->c;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete h;
    return PBGPU_ERR_CUDA;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->sm_count = prop.multiProcessorCount;
  if (cuda_stream) {
    c->stream = static_cast<cudaStream_t>(cuda_stream);
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete h;
      return PBGPU_ERR_CUDA;
    }
    c->own_stream = true;
  }
  c->blk_cache.s = c->stream;
  c->blk_cache.acct = &c->dev_bytes;
  if (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->evc[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->evc[1], cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost(&c->ks_host, 2 * sizeof(KrylovScalars)) != cudaSuccess ||
      cudaMallocHost(&c->rb_host, kReadbackBytes) != cudaSuccess) {
    pbgpu_ctx_destroy(h);
    return PBGPU_ERR_CUDA;
  }
  *out = h;
  return PBGPU_OK;
}

void pbgpu_ctx_destroy(pbgpu_ctx* h) {
  if (!h) return;
  Context* c = &h->c;
  cudaSetDevice(c->device);
  cudaStream_t st = c->stream;
  const bool own = c->own_stream;
  if (st) cudaStreamSynchronize(st);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (cudaEvent_t e : c->evc)
    if (e) cudaEventDestroy(e);
  if (c->ks_host) cudaFreeHost(c->ks_host);
  if (c->rb_host) cudaFreeHost(c->rb_host);
  c->blk_cache.flush();  // the cached blocks back to the pool, on the context's stream
  delete h;  // DBuf destructors free device memory (pool buffers on the stream)
  if (st) cudaStreamSynchronize(st);
  if (own && st) cudaStreamDestroy(st);
  pool_trim();
}

const char* pbgpu_last_error(const pbgpu_ctx* h) { return h ? h->c.err.c_str() : "null context"; }

void* pbgpu_ctx_stream(const pbgpu_ctx* h) { return h ? static_cast<void*>(h->c.stream) : nullptr; }

// ---- input packing and checks on the device (the host only copies)
enum { kErrLevel, kErrNodeId, kErrNodeXyz, kErrHangNp, kErrHangPar, kErrRayPtr, kErrRayKey, kNumInputErr };

__global__ void k_pack_octants(int64_t no, const int32_t* __restrict__ xyz, const int8_t* __restrict__ lvl,
                               int4* __restrict__ oct, int* __restrict__ err) {
  const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= no) return;
  const int lv = lvl[o];
  if (lv < 0 || lv > 18) err[kErrLevel] = 1;
  oct[o] = make_int4(xyz[3 * o], xyz[3 * o + 1], xyz[3 * o + 2], lv);
}

__global__ void k_check_ids(int64_t m, const int32_t* __restrict__ ids, int64_t lim, int* __restrict__ err) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < m && (ids[t] < 0 || ids[t] >= lim)) err[kErrNodeId] = 1;
}

__global__ void k_pack_nodes(int64_t n, const int32_t* __restrict__ xyz, int4* __restrict__ nodes,
                             int* __restrict__ err) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p[3], flag = 0;
  for (int a = 0; a < 3; ++a) {
    p[a] = xyz[3 * i + a];
    if (p[a] < 0 || p[a] > kRoot) err[kErrNodeXyz] = 1;
    if (p[a] == 0 || p[a] == kRoot) flag = 1;
  }
  nodes[i] = make_int4(p[0], p[1], p[2], flag);
}

__global__ void k_pack_hanging(int64_t nh, const int8_t* __restrict__ np_in, const int32_t* __restrict__ par_in,
                               int64_t n, int4* __restrict__ par, int8_t* __restrict__ np_out,
                               int* __restrict__ err) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= nh) return;
  const int np = np_in[j];
  if (np != 2 && np != 4) err[kErrHangNp] = 1;
  int32_t q[4];
  for (int k = 0; k < 4; ++k) {
    q[k] = k < np ? par_in[4 * j + k] : par_in[4 * j];
    if (q[k] < 0 || q[k] >= n) err[kErrHangPar] = 1;
  }
  par[j] = make_int4(q[0], q[1], q[2], q[3]);
  np_out[j] = (int8_t)np;
}

__global__ void k_check_rays(int64_t nr, const uint64_t* __restrict__ keys, const int64_t* __restrict__ ptr,
                             int* __restrict__ err) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= nr) return;
  if (ptr[j + 1] < ptr[j]) err[kErrRayPtr] = 1;
  if (j && keys[j] <= keys[j - 1]) err[kErrRayKey] = 1;
}

static const char* kInputErrMsg[kNumInputErr] = {
    "set_mesh: octant level out of range", "set_mesh: bad node id", "set_mesh: node coordinate out of range",
    "set_mesh: hanging node needs 2 or 4 parents", "set_mesh: hanging parent is not an independent node",
    "set_rays: ptr not ascending", "set_rays: keys not strictly ascending"};

// Waits for the stream and reports the first input check that failed.
static int input_errors(Context* c, const int* d_err) {
  int h[kNumInputErr];
  PBGPU_CUDA(c, readback(c, h, d_err, sizeof(h)));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int k = 0; k < kNumInputErr; ++k)
    if (h[k]) return c->fail(PBGPU_ERR_ARG, kInputErrMsg[k]);
  return PBGPU_OK;
}

int pbgpu_set_mesh(pbgpu_ctx* h, const pbgpu_mesh* m) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!m || m->n_oct <= 0 || m->n_nodes <= 0 || !m->oct_xyz || !m->oct_level || !m->oct_nodes || !m->node_xyz)
    return c->fail(PBGPU_ERR_ARG, "set_mesh: empty or null mesh arrays");
  if (m->n_hang > 0 && (!m->hang_np || !m->hang_par)) return c->fail(PBGPU_ERR_ARG, "set_mesh: null hanging arrays");
  if (m->n_nodes + m->n_hang >= (int64_t(1) << 31)) return c->fail(PBGPU_ERR_ARG, "set_mesh: too many nodes");
  for (int a = 0; a < 3; ++a)
    if (!(m->hi[a] > m->lo[a])) return c->fail(PBGPU_ERR_ARG, "set_mesh: empty domain box");
  SET_DEVICE(c);
  const int64_t no = m->n_oct, n = m->n_nodes, nh = m->n_hang;
  // the host copies the caller's arrays as they are; packing to int4 and the
  // range checks run on the device, and the mesh is dropped if a check fails
  invalidate_from_mesh(c);
  c->have_mesh = false;
  c->n_oct = no;
  c->n = n;
  c->nh = nh;
  for (int a = 0; a < 3; ++a) {
    c->lo[a] = m->lo[a];
    c->len[a] = m->hi[a] - m->lo[a];
  }
  c->tol = m->locate_tol;
  Scratch<int32_t> oxyz(c, kScInOctXyz), nxyz(c, kScInNodeXyz), hpar(c, kScInHangPar);
  Scratch<int8_t> olvl(c, kScInOctLvl), hnp(c, kScInHangNp);
  Scratch<int> err(c, kScInErr);
  PBGPU_CUDA(c, err.alloc(kNumInputErr));
  PBGPU_CUDA(c, cudaMemsetAsync(err.get(), 0, kNumInputErr * sizeof(int), c->stream));
  PBGPU_CUDA(c, oxyz.alloc(3 * no));
  PBGPU_CUDA(c, olvl.alloc(no));
  PBGPU_CUDA(c, nxyz.alloc(3 * n));
  PBGPU_CUDA(c, c->oct.alloc(no));
  PBGPU_CUDA(c, c->oct_nodes.alloc(8 * no));
  PBGPU_CUDA(c, c->node_xyz.alloc(n));
  PBGPU_CUDA(c, c->hang_par.alloc(nh > 0 ? nh : 1));
  PBGPU_CUDA(c, c->hang_np.alloc(nh > 0 ? nh : 1));
  auto h2d = [&](void* d, const void* src, size_t bytes) {
    return cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, c->stream);
  };
  PBGPU_CUDA(c, h2d(oxyz.get(), m->oct_xyz, 3 * no * sizeof(int32_t)));
  PBGPU_CUDA(c, h2d(olvl.get(), m->oct_level, no));
  PBGPU_CUDA(c, h2d(c->oct_nodes.get(), m->oct_nodes, 8 * no * sizeof(int32_t)));
  PBGPU_CUDA(c, h2d(nxyz.get(), m->node_xyz, 3 * n * sizeof(int32_t)));
  k_pack_octants<<<grid_for(no, 256), 256, 0, c->stream>>>(no, oxyz.get(), olvl.get(), c->oct.get(), err.get());
  PBGPU_LAUNCHED(c);
  k_check_ids<<<grid_for(8 * no, 256), 256, 0, c->stream>>>(8 * no, c->oct_nodes.get(), n + nh, err.get());
  PBGPU_LAUNCHED(c);
  k_pack_nodes<<<grid_for(n, 256), 256, 0, c->stream>>>(n, nxyz.get(), c->node_xyz.get(), err.get());
  PBGPU_LAUNCHED(c);
  if (nh > 0) {
    PBGPU_CUDA(c, hpar.alloc(4 * nh));
    PBGPU_CUDA(c, hnp.alloc(nh));
    PBGPU_CUDA(c, h2d(hpar.get(), m->hang_par, 4 * nh * sizeof(int32_t)));
    PBGPU_CUDA(c, h2d(hnp.get(), m->hang_np, nh));
    k_pack_hanging<<<grid_for(nh, 256), 256, 0, c->stream>>>(nh, hnp.get(), hpar.get(), n, c->hang_par.get(),
                                                             c->hang_np.get(), err.get());
    PBGPU_LAUNCHED(c);
  }
  PBGPU_CUDA(c, c->oct_key.alloc(no));
  launch_oct_keys(c->oct.get(), no, c->oct_key.get(), c->stream);
  PBGPU_LAUNCHED(c);
  const int st = input_errors(c, err.get());
  if (st != PBGPU_OK) return st;
  c->have_mesh = true;
  return PBGPU_OK;
}

int pbgpu_set_rays(pbgpu_ctx* h, int axis, const pbgpu_rays* r) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (axis < 0 || axis > 2 || !r || r->n_rays < 0) return c->fail(PBGPU_ERR_ARG, "set_rays: bad axis or table");
  if (r->n_rays > 0 && (!r->keys || !r->ptr || !r->inters || !r->normals))
    return c->fail(PBGPU_ERR_ARG, "set_rays: null arrays");
  if (r->n_rays >= (int64_t(1) << 31)) return c->fail(PBGPU_ERR_ARG, "set_rays: too many rays");
  SET_DEVICE(c);
  const int64_t nr = r->n_rays;
  const int64_t nc = nr > 0 ? r->ptr[nr] : 0;
  if (nr > 0 && (r->ptr[0] != 0 || nc < 0)) return c->fail(PBGPU_ERR_ARG, "set_rays: ptr[0] must be 0");
  Rays& R = c->rays[axis];
  c->have_rays[axis] = false;
  R.n = nr;
  int st;
  if ((st = upload(c, R.ptr, r->ptr, nr + 1)) != PBGPU_OK) return st;
  if ((st = upload(c, R.inters, r->inters, nc)) != PBGPU_OK) return st;
  if ((st = upload(c, R.normals, r->normals, 3 * nc)) != PBGPU_OK) return st;
  R.nc = nc;
  if ((st = upload(c, R.keys, r->keys, nr)) != PBGPU_OK) return st;
  if (nr > 0) {
    // ascending offsets and strictly ascending keys, checked on the device
    Scratch<int> err(c, kScInErr);
    PBGPU_CUDA(c, err.alloc(kNumInputErr));
    PBGPU_CUDA(c, cudaMemsetAsync(err.get(), 0, kNumInputErr * sizeof(int), c->stream));
    k_check_rays<<<grid_for(nr, 256), 256, 0, c->stream>>>(nr, R.keys.get(), R.ptr.get(), err.get());
    PBGPU_LAUNCHED(c);
    if ((st = input_errors(c, err.get())) != PBGPU_OK) return st;
  }
  if ((st = build_ray_hash_from(c, axis, R.keys.get())) != PBGPU_OK) return st;
  c->have_rays[axis] = true;
  c->have_markers = c->have_system = c->have_phi = false;
  return PBGPU_OK;
}

int pbgpu_set_atoms(pbgpu_ctx* h, int64_t na, const double* pos, const double* q) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (na < 0 || (na > 0 && (!pos || !q))) return c->fail(PBGPU_ERR_ARG, "set_atoms: bad arrays");
  if (na >= (int64_t(1) << 27)) return c->fail(PBGPU_ERR_ARG, "set_atoms: too many atoms");
  SET_DEVICE(c);
  std::vector<double4> a(na > 0 ? na : 1);
  for (int64_t i = 0; i < na; ++i) a[i] = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], q[i]);
  int st = upload(c, c->atoms, a.data(), na);
  if (st != PBGPU_OK) return st;
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  c->na = na;
  c->have_atoms = true;
  c->have_density = c->have_system = c->have_phi = false;
  return PBGPU_OK;
}

int pbgpu_set_model(pbgpu_ctx* h, const pbgpu_model* m) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!m) return c->fail(PBGPU_ERR_ARG, "set_model: null");
  if (!(m->e_in > 0) || !(m->e_out > 0) || !(m->T > 0) || m->ionic_strength < 0)
    return c->fail(PBGPU_ERR_ARG, "set_model: dielectric constants and T must be positive, ionic strength >= 0");
  if (m->bc_type < 0 || m->bc_type > 3) return c->fail(PBGPU_ERR_ARG, "set_model: bc_type must be 0..3");
  c->model = *m;
  // physical constants and scalings of src/pb_class.cpp:1800-1806 (same
  // evaluation order)
  const double e_0 = 8.85418781762e-12, kb = 1.380649e-23, e = 1.602176634e-19, N_av = 6.022e23, Angs = 1e-10;
  c->eps_in = 4.0 * kPi * e_0 * m->e_in * kb * m->T * Angs / (e * e);
  c->eps_out = 4.0 * kPi * e_0 * m->e_out * kb * m->T * Angs / (e * e);
  const double C_0 = 1.0e3 * N_av * m->ionic_strength;
  c->k2 = 2.0 * C_0 * Angs * Angs * e * e / (e_0 * m->e_out * kb * m->T);
  c->kappa = std::sqrt(c->k2);
  c->have_model = true;
  c->have_markers = c->have_system = c->have_phi = false;
  return PBGPU_OK;
}

int pbgpu_create_markers(pbgpu_ctx* h) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!c->have_mesh || !c->have_model || !c->have_rays[0] || !c->have_rays[1] || !c->have_rays[2])
    return c->fail(PBGPU_ERR_STATE, "create_markers: mesh, model and the 3 ray tables are required");
  SET_DEVICE(c);
  StageTimer t(c, 0);
  c->have_system = c->have_phi = false;
  return run_markers(c);
}

int pbgpu_create_density_map(pbgpu_ctx* h) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!c->have_mesh || !c->have_atoms) return c->fail(PBGPU_ERR_STATE, "create_density_map: mesh and atoms are required");
  SET_DEVICE(c);
  StageTimer t(c, 1);
  c->have_system = c->have_phi = false;
  return run_density(c);
}

int pbgpu_assemble(pbgpu_ctx* h, const pbgpu_sell_opts* o) {
  CTX_CHECK(h);
  Context* c = &h->c;
  SET_DEVICE(c);
  StageTimer t(c, 2);
  pbgpu_sell_opts tuned;
  int cols = 0;
  if (!o && c->have_mesh && tuned_layout(c->n, &tuned, &cols)) {  // pbgpu_autotune ran for this size class
    c->spmv_cols = cols ? cols : c->spmv_cols;
    return run_assemble(c, &tuned);
  }
  return run_assemble(c, o);
}

int pbgpu_solve(pbgpu_ctx* h, const pbgpu_solver_opts* o, pbgpu_solve_stats* st) {
  CTX_CHECK(h);
  Context* c = &h->c;
  SET_DEVICE(c);
  StageTimer t(c, 3);
  return run_solve(c, o, st);
}

int pbgpu_phi_on_atoms(pbgpu_ctx* h, double* out) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!out && c->na > 0) return c->fail(PBGPU_ERR_ARG, "phi_on_atoms: null output");
  SET_DEVICE(c);
  StageTimer t(c, 4);
  return run_phi_atoms(c, out);
}

int pbgpu_energy(pbgpu_ctx* h, int fast, pbgpu_energy_out* out) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!out) return c->fail(PBGPU_ERR_ARG, "energy: null output");
  SET_DEVICE(c);
  StageTimer t(c, 5);
  return run_energy(c, fast, out);
}

// pot_field / pot_field_fast; its device time adds to the energy stage.
int pbgpu_pot_field(pbgpu_ctx* h, int fast, int calc_potential_term, int calc_field_term, double* per_atom,
                    pbgpu_pot_field_out* out) {
  CTX_CHECK(h);
  Context* c = &h->c;
  SET_DEVICE(c);
  StageTimer t(c, 5);
  return run_pot_field(c, fast, calc_potential_term, calc_field_term, per_atom, out);
}

int pbgpu_solve_charges(pbgpu_ctx* h, int k, const double* charges, const pbgpu_solver_opts* o, int fast,
                        pbgpu_energy_out* energies, pbgpu_solve_stats* stats) {
  CTX_CHECK(h);
  Context* c = &h->c;
  SET_DEVICE(c);
  StageTimer t(c, 3);
  return run_solve_charges(c, k, charges, o, fast, energies, stats);
}

void pbgpu_default_solver_opts(pbgpu_solver_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->method = PBGPU_BICGSTAB;
  o->precond = PBGPU_PRECOND_JACOBI;
  o->precision = PBGPU_FP64;
  o->tol = 1e-6;
  o->max_iter = 10000;
  o->inner_tol = 1e-5;
  o->max_outer = 50;
  o->check_every = 16;
  o->conv_cond = 0;
  o->tol_w = 1.0;
}

int pbgpu_parse_lis_options(const char* options, pbgpu_solver_opts* out) {
  if (!out) return PBGPU_ERR_ARG;
  pbgpu_default_solver_opts(out);
  // LIS defaults (-i bicg is LIS's own default solver; NextGenPB passes -i)
  if (!options) return PBGPU_OK;
  std::istringstream in(options);
  std::vector<std::string> tok;
  for (std::string t; in >> t;) tok.push_back(t);
  for (size_t i = 0; i < tok.size(); ++i) {
    const std::string& k = tok[i];
    const bool has = i + 1 < tok.size();
    if ((k == "-i" || k == "-solver") && has) {
      const std::string v = tok[++i];
      if (v == "cg" || v == "1" || v == "cr" || v == "5")
        out->method = PBGPU_CG;
      else if (v == "cgs" || v == "3")
        out->method = PBGPU_CGS;
      else
        out->method = PBGPU_BICGSTAB;  // bicg, bicgstab, bicgsafe, gmres, ...
    } else if ((k == "-p" || k == "-precon") && has) {
      const std::string v = tok[++i];
      if (v == "none" || v == "0")
        out->precond = PBGPU_PRECOND_NONE;
      else if (v == "jacobi" || v == "1")
        out->precond = PBGPU_PRECOND_JACOBI;
      else
        out->precond = PBGPU_PRECOND_BLOCK_JACOBI;
    } else if (k == "-tol" && has) {
      const double t = std::strtod(tok[++i].c_str(), nullptr);
      if (!(t > 0)) return PBGPU_ERR_ARG;
      out->tol = t;
    } else if (k == "-conv_cond" && has) {
      const long m = std::strtol(tok[++i].c_str(), nullptr, 10);
      if (m < 0 || m > 2) return PBGPU_ERR_ARG;
      out->conv_cond = (int)m;
    } else if (k == "-tol_w" && has) {
      const double t = std::strtod(tok[++i].c_str(), nullptr);
      if (!(t >= 0)) return PBGPU_ERR_ARG;
      out->tol_w = t;
    } else if (k == "-maxiter" && has) {
      const long m = std::strtol(tok[++i].c_str(), nullptr, 10);
      if (m <= 0) return PBGPU_ERR_ARG;
      out->max_iter = (int)m;
    } else if (k == "-f" && has) {
      const std::string v = tok[++i];
      if (v == "mixed" || v == "float" || v == "quad") out->precision = v == "quad" ? PBGPU_FP64 : PBGPU_MIXED;
    } else if (has && k.size() > 1 && k[0] == '-' && tok[i + 1][0] != '-') {
      ++i;  // other LIS options (-print, -conv_cond, -tol_w, -ssor_omega ...) take one value
    }
  }
  return PBGPU_OK;
}

int pbgpu_get_node_coeffs(pbgpu_ctx* h, double* eps, double* react) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!c->have_markers) return c->fail(PBGPU_ERR_STATE, "get_node_coeffs: create_markers has not run");
  SET_DEVICE(c);
  if (eps) PBGPU_CUDA(c, cudaMemcpyAsync(eps, c->eps.get(), c->n * 8, cudaMemcpyDeviceToHost, c->stream));
  if (react) PBGPU_CUDA(c, cudaMemcpyAsync(react, c->react.get(), c->n * 8, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  return PBGPU_OK;
}

int pbgpu_get_markers(pbgpu_ctx* h, double* marker, int64_t* n_border, int32_t* border) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!c->have_markers) return c->fail(PBGPU_ERR_STATE, "get_markers: create_markers has not run");
  SET_DEVICE(c);
  if (n_border) *n_border = c->nb;
  if (marker) {
    std::vector<uint8_t> m(c->n_oct);
    PBGPU_CUDA(c, cudaMemcpyAsync(m.data(), c->marker.get(), c->n_oct, cudaMemcpyDeviceToHost, c->stream));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int64_t o = 0; o < c->n_oct; ++o) marker[o] = m[o] == 0 ? 0.0 : (m[o] == 1 ? 0.5 : 1.0);
  }
  if (border && c->nb)
    PBGPU_CUDA(c, cudaMemcpyAsync(border, c->border.get(), c->nb * 4, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  return PBGPU_OK;
}

int pbgpu_get_fractions(pbgpu_ctx* h, double* frac) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!c->have_markers) return c->fail(PBGPU_ERR_STATE, "get_fractions: create_markers has not run");
  if (!frac) return c->fail(PBGPU_ERR_ARG, "get_fractions: null output");
  SET_DEVICE(c);
  if (c->nb) PBGPU_CUDA(c, cudaMemcpyAsync(frac, c->frac.get(), 12 * c->nb * 8, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  return PBGPU_OK;
}

int pbgpu_get_density(pbgpu_ctx* h, double* rho, double* vol_patch) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!c->have_density) return c->fail(PBGPU_ERR_STATE, "get_density: create_density_map has not run");
  SET_DEVICE(c);
  if (rho) PBGPU_CUDA(c, cudaMemcpyAsync(rho, c->rho.get(), c->n * 8, cudaMemcpyDeviceToHost, c->stream));
  if (vol_patch) PBGPU_CUDA(c, cudaMemcpyAsync(vol_patch, c->vol_patch.get(), c->n * 8, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  return PBGPU_OK;
}

int pbgpu_get_system(pbgpu_ctx* h, int64_t* nnz, int64_t* row_ptr, int32_t* col, double* val, double* rhs) {
  CTX_CHECK(h);
  Context* c = &h->c;
  SET_DEVICE(c);
  return export_system(c, nnz, row_ptr, col, val, rhs);
}

int pbgpu_get_phi(pbgpu_ctx* h, double* phi) {
  CTX_CHECK(h);
  Context* c = &h->c;
  if (!c->have_phi) return c->fail(PBGPU_ERR_STATE, "get_phi: solve has not run");
  if (!phi) return c->fail(PBGPU_ERR_ARG, "get_phi: null output");
  SET_DEVICE(c);
  PBGPU_CUDA(c, cudaMemcpyAsync(phi, c->phi.get(), c->n * 8, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  return PBGPU_OK;
}

int pbgpu_get_stage_ms(pbgpu_ctx* h, double ms[6]) {
  CTX_CHECK(h);
  if (!ms) return PBGPU_ERR_ARG;
  for (int i = 0; i < 6; ++i) ms[i] = h->c.stage_ms[i];
  return PBGPU_OK;
}

int pbgpu_set_profiling(pbgpu_ctx* h, int on) {
  CTX_CHECK(h);
  h->c.profiling = on != 0;
  return PBGPU_OK;
}

int pbgpu_set_wait_limit(pbgpu_ctx* h, double seconds) {
  CTX_CHECK(h);
  if (!(seconds >= 0.0) || seconds > 60.0) return h->c.fail(PBGPU_ERR_ARG, "set_wait_limit: seconds must be in [0, 60]");
  h->c.wait_s = seconds;
  return PBGPU_OK;
}

int pbgpu_get_counters(pbgpu_ctx* h, pbgpu_counters* out) {
  CTX_CHECK(h);
  if (!out) return PBGPU_ERR_ARG;
  const Context& c = h->c;
  out->launches = c.launches;
  out->spmv_launches = c.spmv_launches;
  out->spmv_ms = c.spmv_ms;
  out->spmv_bytes = c.spmv_bytes;
  out->krylov_iterations = c.krylov_iters;
  out->energy_points = c.energy_points;
  out->energy_pairs = c.energy_pairs;
  out->device_bytes = c.dev_bytes;
  return PBGPU_OK;
}

int pbgpu_reset_counters(pbgpu_ctx* h) {
  CTX_CHECK(h);
  Context& c = h->c;
  c.launches = c.spmv_launches = c.krylov_iters = c.energy_pairs = 0;
  c.spmv_ms = 0.0;
  return PBGPU_OK;
}

}  // extern "C"
