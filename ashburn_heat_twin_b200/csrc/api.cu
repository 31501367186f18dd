// C ABI of the B200 live solver (include/ahx.h): handle lifetime, host images, stepping, asynchronous read-back,
// diagnostics and budgets over the kernels of step_exact.cu / step_fast.cu / aux.cu.
//
// Device model: one CUDA stream per handle runs everything that touches the state, in submission order (the
// reference's single WebGPU queue, solver.js:401-427). Read-back runs its two small kernels on that stream and copies
// on a second stream, so a read never stalls stepping (solver.js:439-471). Host images are staged through a ring of
// pinned buffers so an upload between steps does not wait for the GPU (the reference's queue.writeBuffer).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ahx.h"
#include "handle.h"
#include "launch.h"

using namespace ahx;

namespace {

thread_local std::string g_err;

}  // namespace

ahx_status ahx::fail(ahx_status st, const std::string& msg) {
  g_err = msg;
  return st;
}

void ahx::set_last_error(const std::string& m) { g_err = m; }

// mark the handle lost on a CUDA error; returns AHX_EDEVICE with the message
ahx_status ahx::cuda_fail(ahx_handle* h, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (h) {
    h->lost = true;
    h->lost_msg = m;
  }
  return fail(AHX_EDEVICE, "live solver: CUDA error (" + m + ")");
}

#define AHX_CUDA(h, call)                                   \
  do {                                                      \
    cudaError_t e__ = (call);                               \
    if (e__ != cudaSuccess) return cuda_fail(h, e__, #call); \
  } while (0)

ahx_status ahx::check(ahx_handle* h) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  if (h->destroyed) return fail(AHX_EDESTROYED, "live solver: destroyed");
  if (h->lost) return fail(AHX_EDEVICE, "live solver: CUDA device lost (" + h->lost_msg + ")");
  if (h->batch_lost.load()) return fail(AHX_EDEVICE, "live solver: CUDA device lost (a batched step failed)");
  return AHX_OK;
}

// the view of the handle's state for a step that reads buffer `parity`
DomainView ahx::view_at(ahx_handle* h, int parity) {
  DomainView D;
  D.params = h->d_params;
  D.colv = h->d_colv;
  D.ktop = h->d_ktop;
  D.fA = h->f[parity];
  D.fB = h->f[1 - parity];
  D.gA = h->g[parity];
  D.gB = h->g[1 - parity];
  D.dbg = h->d_dbg;
  D.budget = h->d_budget;
  D.sacc = h->accum_on ? h->d_sacc : nullptr;
  D.facc = h->accum_on ? h->d_facc : nullptr;
  D.err = h->d_err;
  D.tick = h->d_tick;
  D.tick_blocks = 0;
  D.pf = h->prefetch ? 1 : 0;
  D.nx = h->dims.nx;
  D.ny = h->dims.ny;
  D.nz = h->dims.nz;
  D.px = h->px;
  const bool slab = h->nyg > 0;
  D.jg0 = slab ? h->jg0 : 0;
  D.nyg = slab ? h->nyg : h->dims.ny;
  D.jlo = slab ? h->jlo : 0;
  D.jhi = slab ? h->jhi : h->dims.ny;
  D.jbase = 0;
  D.strip = strip_width(h->esize, h->dims.nx);
  D.ps = h->ps;
  D.qs = h->qs;
  set_offsets(D, h->esize, h->esize_g);
  set_pointers(D, h->esize, h->esize_g);
  return D;
}

namespace {

size_t nxy(const ahx_handle* h) { return (size_t)h->dims.nx * h->dims.ny; }
size_t ncells(const ahx_handle* h) { return nxy(h) * h->dims.nz; }
size_t params_bytes(const ahx_handle* h) { return 64 + 16 * (size_t)h->dims.nz; }

DomainView view(ahx_handle* h) { return view_at(h, h->parity); }

}  // namespace

StepLaunch ahx::solo_launch(const ahx_handle* h, int parity) {
  StepLaunch L;
  L.precision = h->dims.precision;
  L.mode = 0;
  L.budget = false;
  L.block_y = h->block_y;
  L.zslab = h->zslab;
  L.minb = h->minb;
  L.pairs = h->pairs;
  L.tma_ty = (h->pairs ? h->pmaps_ok : h->maps_ok) ? h->tma_ty : 0;
  L.tma_depth = h->tma_depth;
  L.maps = stage_maps(h, L, parity);
  return L;
}

const TmaMaps* ahx::stage_maps(const ahx_handle* h, const StepLaunch& L, int parity) {
  if (!L.tma_ty) return nullptr;
  const int t = L.tma_ty == 8 ? 1 : 0;
  return L.pairs ? &h->pmaps[t][parity] : &h->maps[t][parity];
}

uint64_t ahx::solo_launch_key(const ahx_handle* h) {
  const StepLaunch L = solo_launch(h, 0);
  uint64_t k = 1469598103934665603ull;
  const int v[] = {L.precision, L.block_y, L.zslab, L.minb, (int)L.pairs, L.tma_ty, L.tma_depth,
                   h->jg0, h->nyg, h->jlo, h->jhi, h->dims.arith, (int)h->prefetch};
  for (int x : v) k = (k ^ (uint64_t)(uint32_t)x) * 1099511628211ull;
  return k | 1;   // never 0, the "no graph" key
}

cudaError_t ahx::solo_step(ahx_handle* h, int parity, cudaStream_t s) {
  const StepLaunch L = solo_launch(h, parity);
  const DomainView D = view_at(h, parity);
  return h->dims.arith == AHX_ARITH_FAST ? fast::launch_step(D, L, s) : exact::launch_step(D, L, s);
}

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
  });
  return fn;
}

// 4-D tensor map [q][z][y][x] over one population buffer with a box of width x TY x 1 x 1
bool encode_map(ahx_handle* h, void* buf, int nq, int width, int ty, CUtensorMap* out) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const int es = h->esize;
  const CUtensorMapDataType dt = es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                 : es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                           : CU_TENSOR_MAP_DATA_TYPE_UINT16;
  const cuuint64_t dims[4] = {(cuuint64_t)h->dims.nx, (cuuint64_t)h->dims.ny, (cuuint64_t)h->dims.nz, (cuuint64_t)nq};
  const cuuint64_t strides[3] = {(cuuint64_t)h->px * es, (cuuint64_t)h->ps * es, (cuuint64_t)h->qs * es};
  const cuuint32_t box[4] = {(cuuint32_t)width, (cuuint32_t)ty, 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return fn(out, dt, 4, buf, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the four maps (f wide / narrow, g wide / narrow) of a state (f, g) for blocks of 32 x ty columns
bool make_maps(ahx_handle* h, void* f, void* g, int ty, TmaMaps* M) {
  const int H = 16 / h->esize;
  return encode_map(h, f, 19, 32 + 2 * H, ty, &M->fw) && encode_map(h, f, 19, 32, ty, &M->fn) &&
         encode_map(h, g, 7, 32 + 2 * H, ty, &M->gw) && encode_map(h, g, 7, 32, ty, &M->gn);
}

// 4-D tensor map [q][level pair][y][x] of 32-bit words over a level-paired 16-bit population buffer (word (t, j, i)
// holds the levels 2t and 2t + 1 of column (i, j)), with a box of width x TY x 1 x 1 words
bool encode_pair_map(ahx_handle* h, void* buf, int nq, int width, int ty, CUtensorMap* out) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)h->dims.nx, (cuuint64_t)h->dims.ny, (cuuint64_t)((h->dims.nz + 1) / 2),
                              (cuuint64_t)nq};
  // row: px words; level pair: ps words; population plane: qs 16-bit elements
  const cuuint64_t strides[3] = {(cuuint64_t)h->px * 4, (cuuint64_t)h->ps * 4, (cuuint64_t)h->qs * 2};
  const cuuint32_t box[4] = {(cuuint32_t)width, (cuuint32_t)ty, 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return fn(out, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, buf, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the four word maps of a level-paired state for the staged paired step (wide boxes: 4 words of halo on each side)
bool make_pair_maps(ahx_handle* h, void* f, void* g, int ty, TmaMaps* M) {
  return encode_pair_map(h, f, 19, 40, ty, &M->fw) && encode_pair_map(h, f, 19, 32, ty, &M->fn) &&
         encode_pair_map(h, g, 7, 40, ty, &M->gw) && encode_pair_map(h, g, 7, 32, ty, &M->gn);
}

// a staged copy that ran out of time leaves its block's cells unstepped: report it (the state is not usable)
ahx_status check_kernel_error(ahx_handle* h) {
  int e = 0;
  if (cudaMemcpy(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return cuda_fail(h, cudaGetLastError(), "error word read");
  if (e != 0) {
    h->lost = true;
    h->lost_msg = "a TMA stage of the step kernel did not arrive within its time bound";
    return fail(AHX_ETIMEOUT, "live solver: " + h->lost_msg);
  }
  return AHX_OK;
}

// copy a host image to device memory in stream order without blocking the host on the GPU
ahx_status upload(ahx_handle* h, void* dst, const void* src, size_t bytes) {
  UploadSlot& u = h->up[h->up_next];
  h->up_next = (h->up_next + 1) % kUploadSlots;
  if (u.used) AHX_CUDA(h, cudaEventSynchronize(u.ev));
  if (u.bytes < bytes) {
    if (u.h) cudaFreeHost(u.h);
    u.h = nullptr;
    u.bytes = 0;
    if (cudaMallocHost(&u.h, bytes) != cudaSuccess) return fail(AHX_ENOMEM, "live solver: pinned allocation failed");
    u.bytes = bytes;
  }
  std::memcpy(u.h, src, bytes);
  AHX_CUDA(h, cudaMemcpyAsync(dst, u.h, bytes, cudaMemcpyHostToDevice, h->s_step));
  AHX_CUDA(h, cudaEventRecord(u.ev, h->s_step));
  u.used = true;
  return AHX_OK;
}

ahx_status ensure_dbg(ahx_handle* h) {
  if (h->d_dbg) return AHX_OK;
  const size_t bytes = (size_t)h->ps * h->dims.nz * sizeof(float4);
  if (cudaMalloc(&h->d_dbg, bytes) != cudaSuccess) {
    h->d_dbg = nullptr;
    cudaGetLastError();
    return fail(AHX_ENOMEM, "live solver: debug buffer allocation failed");
  }
  AHX_CUDA(h, cudaMemsetAsync(h->d_dbg, 0, bytes, h->s_step));
  return AHX_OK;
}

void free_all(ahx_handle* h) {
  cudaSetDevice(h->dev);
  if (h->s_step) cudaStreamSynchronize(h->s_step);
  if (h->s_copy) cudaStreamSynchronize(h->s_copy);
  for (auto& g : h->graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  for (int p = 0; p < 2; ++p) {
    if (h->f[p]) cudaFree(h->f[p]);
    if (h->g[p]) cudaFree(h->g[p]);
    h->f[p] = h->g[p] = nullptr;
  }
  void* devs[] = {h->d_params, h->d_colv, h->d_ktop, h->d_oldk, h->d_dbg, h->d_budget, h->d_stats, h->d_err,
                  h->d_tick, h->d_sacc, h->d_facc};
  for (void* p : devs)
    if (p) cudaFree(p);
  h->d_params = nullptr;
  h->d_colv = nullptr;
  h->d_ktop = h->d_oldk = nullptr;
  h->d_dbg = nullptr;
  h->d_budget = nullptr;
  h->d_sacc = h->d_facc = nullptr;
  h->d_stats = nullptr;
  h->d_err = nullptr;
  h->d_tick = nullptr;
  for (auto& r : h->reads) {
    if (r.d_surf) cudaFree(r.d_surf);
    if (r.d_vol) cudaFree(r.d_vol);
    if (r.d_tmax) cudaFree(r.d_tmax);
    if (r.h_surf) cudaFreeHost(r.h_surf);
    if (r.h_vol) cudaFreeHost(r.h_vol);
    if (r.h_tmax) cudaFreeHost(r.h_tmax);
    if (r.ev_kernels) cudaEventDestroy(r.ev_kernels);
    if (r.ev_done) cudaEventDestroy(r.ev_done);
    r = ReadSlot{};
  }
  for (auto& u : h->up) {
    if (u.h) cudaFreeHost(u.h);
    if (u.ev) cudaEventDestroy(u.ev);
    u = UploadSlot{};
  }
  for (auto& f : h->fences) cudaEventDestroy(f.ev);
  h->fences.clear();
  if (h->s_step) cudaStreamDestroy(h->s_step);
  if (h->s_copy) cudaStreamDestroy(h->s_copy);
  h->s_step = h->s_copy = nullptr;
}

}  // namespace

// bounded wait on an event; the handle lock is not held while waiting
ahx_status ahx::wait_event(ahx_handle* h, cudaEvent_t ev, int timeout_ms) {
  const auto t0 = std::chrono::steady_clock::now();
  int spin = 0;
  for (;;) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return AHX_OK;
    if (e != cudaErrorNotReady) return cuda_fail(h, e, "cudaEventQuery");
    if (timeout_ms >= 0) {
      const auto ms =
          std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
      if (ms >= timeout_ms) return fail(AHX_ETIMEOUT, "live solver: timed out waiting for the GPU");
    }
    if (++spin < 200) std::this_thread::yield();
    else std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

extern "C" {

const char* ahx_last_error(void) { return g_err.c_str(); }

ahx_status ahx_create(const ahx_dims* dims, ahx_handle** out) {
  if (!dims || !out) return fail(AHX_EINVAL, "live solver: null argument");
  *out = nullptr;
  if (dims->nx < 2 || dims->ny < 2 || dims->nz < 2)
    return fail(AHX_EINVAL, "live solver: grid must be at least 2 x 2 x 2");
  const int esize = element_bytes(dims->precision);
  if (!esize) return fail(AHX_EINVAL, "live solver: unknown precision");
  if (dims->arith != AHX_ARITH_EXACT && dims->arith != AHX_ARITH_FAST)
    return fail(AHX_EINVAL, "live solver: unknown arithmetic variant");
  const int align = 128 / esize;   // x rows start on 128-byte boundaries
  const int px = (dims->nx + align - 1) / align * align;
  const uint64_t ps = (uint64_t)px * dims->ny;
  // a level-paired (16-bit) population plane holds nz rounded up to even levels (lvl)
  const bool paired = esize == 2 || element_bytes_g(dims->precision) == 2;
  const uint64_t qs = ps * (uint64_t)(paired ? dims->nz + (dims->nz & 1) : dims->nz);
  if (19 * qs >= (1ull << 32))
    return fail(AHX_EINVAL, "live solver: grid too large for one handle (19 population planes must index in 32 bits)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AHX_EDEVICE, "live solver: no CUDA device is available");
  }
  int dev = dims->device_ordinal;
  if (dev < 0) cudaGetDevice(&dev);
  if (dev >= ndev) return fail(AHX_EINVAL, "live solver: device ordinal out of range");
  ahx_handle* h = new ahx_handle();
  h->dev = dev;
  h->dims = *dims;
  h->dims.device_ordinal = dev;
  h->esize = esize;
  h->esize_g = element_bytes_g(dims->precision);
  h->px = px;
  h->ps = (uint32_t)ps;
  h->qs = (uint32_t)qs;
  h->zslab = 0;
  cudaDeviceProp prop;
  if (cudaSetDevice(dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    delete h;
    return fail(AHX_EDEVICE, "live solver: cannot use CUDA device");
  }
  std::strncpy(h->name, prop.name, sizeof(h->name) - 1);
  auto bail = [&](ahx_status st, const std::string& m) {
    free_all(h);
    delete h;
    cudaGetLastError();
    return fail(st, m);
  };
  if (cudaStreamCreateWithFlags(&h->s_step, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->s_copy, cudaStreamNonBlocking) != cudaSuccess)
    return bail(AHX_EDEVICE, "live solver: stream creation failed");
  const size_t fbytes = 19 * qs * esize, gbytes = 7 * qs * (size_t)element_bytes_g(dims->precision);
  const size_t NXY = (size_t)dims->nx * dims->ny;
  for (int p = 0; p < 2; ++p) {
    if (cudaMalloc(&h->f[p], fbytes) != cudaSuccess || cudaMalloc(&h->g[p], gbytes) != cudaSuccess)
      return bail(AHX_ENOMEM, "live solver: buffer allocation failed (out of memory). Try a coarser grid.");
    cudaMemsetAsync(h->f[p], 0, fbytes, h->s_step);
    cudaMemsetAsync(h->g[p], 0, gbytes, h->s_step);
  }
  if (cudaMalloc(&h->d_params, 64 + 16 * (size_t)dims->nz) != cudaSuccess ||
      cudaMalloc(&h->d_colv, NXY * sizeof(uint4)) != cudaSuccess ||
      cudaMalloc(&h->d_ktop, NXY * 4) != cudaSuccess || cudaMalloc(&h->d_oldk, NXY * 4) != cudaSuccess ||
      cudaMalloc(&h->d_budget, (size_t)kBudgetSlots * kBudgetStride * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->d_stats, sizeof(StatsScratch)) != cudaSuccess ||
      cudaMalloc(&h->d_err, sizeof(int)) != cudaSuccess || cudaMalloc(&h->d_tick, 4 * sizeof(uint32_t)) != cudaSuccess)
    return bail(AHX_ENOMEM, "live solver: buffer allocation failed (out of memory)");
  cudaMemsetAsync(h->d_err, 0, sizeof(int), h->s_step);
  cudaMemsetAsync(h->d_tick, 0, 4 * sizeof(uint32_t), h->s_step);
  // the staged kernel stages f and g with one element size and rounds to nearest
  // staged boxes are single levels of 4- and 8-byte planes
  h->maps_ok = h->esize == h->esize_g && h->esize != 2 && dims->precision != AHX_FP16_SR;
  for (int t = 0; t < 2 && h->maps_ok; ++t)
    for (int p = 0; p < 2; ++p) h->maps_ok = h->maps_ok && make_maps(h, h->f[p], h->g[p], t ? 8 : 4, &h->maps[t][p]);
  // the staged paired step reads level-paired f and g (the 16-bit storages)
  h->pmaps_ok = h->esize == 2 && h->esize_g == 2;
  for (int t = 0; t < 2 && h->pmaps_ok; ++t)
    for (int p = 0; p < 2; ++p)
      h->pmaps_ok = h->pmaps_ok && make_pair_maps(h, h->f[p], h->g[p], t ? 8 : 4, &h->pmaps[t][p]);
  cudaMemsetAsync(h->d_params, 0, 64 + 16 * (size_t)dims->nz, h->s_step);
  cudaMemsetAsync(h->d_colv, 0, NXY * sizeof(uint4), h->s_step);
  cudaMemsetAsync(h->d_ktop, 0, NXY * 4, h->s_step);
  cudaMemsetAsync(h->d_budget, 0, (size_t)kBudgetSlots * kBudgetStride * sizeof(double), h->s_step);
  const size_t volw = ((size_t)dims->nz * NXY + 3) / 4;
  for (auto& r : h->reads) {
    if (cudaMalloc(&r.d_surf, 3 * NXY * 4) != cudaSuccess || cudaMalloc(&r.d_vol, volw * 4) != cudaSuccess ||
        cudaMalloc(&r.d_tmax, 4) != cudaSuccess || cudaMallocHost(&r.h_surf, 3 * NXY * 4) != cudaSuccess ||
        cudaMallocHost(&r.h_vol, volw * 4) != cudaSuccess || cudaMallocHost(&r.h_tmax, 4) != cudaSuccess ||
        cudaEventCreateWithFlags(&r.ev_kernels, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&r.ev_done, cudaEventDisableTiming) != cudaSuccess)
      return bail(AHX_ENOMEM, "live solver: read-back buffer allocation failed");
  }
  for (auto& u : h->up)
    if (cudaEventCreateWithFlags(&u.ev, cudaEventDisableTiming) != cudaSuccess)
      return bail(AHX_EDEVICE, "live solver: event creation failed");
  if (cudaStreamSynchronize(h->s_step) != cudaSuccess) return bail(AHX_EDEVICE, "live solver: initialisation failed");
  *out = h;
  return AHX_OK;
}

ahx_status ahx_destroy(ahx_handle* h) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  {
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->destroyed) return AHX_OK;
    if (h->batch_refs > 0)
      return fail(AHX_EINVAL, "live solver: the handle belongs to a batch; destroy the batch first");
    h->destroyed = true;
    free_all(h);
  }
  // the handle object itself stays allocated so later calls report "destroyed" instead of touching freed memory
  return AHX_OK;
}

ahx_status ahx_get_info(ahx_handle* h, ahx_info_out* out) {
  if (!h || !out) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  std::memset(out, 0, sizeof(*out));
  out->nx = h->dims.nx;
  out->ny = h->dims.ny;
  out->nz = h->dims.nz;
  out->px = h->px;
  out->precision = h->dims.precision;
  out->arith = h->dims.arith;
  out->parity = h->parity;
  out->device_ordinal = h->dev;
  out->steps = h->steps;
  out->state_bytes = 2ull * h->qs * (19ull * h->esize + 7ull * h->esize_g);
  out->bytes_per_cell = 2ull * (19ull * h->esize + 7ull * h->esize_g);
  std::snprintf(out->device_name, sizeof(out->device_name), "%s", h->name);
  if (h->destroyed) return fail(AHX_EDESTROYED, "live solver: destroyed");
  return AHX_OK;
}

ahx_status ahx_set_params(ahx_handle* h, const void* params, size_t bytes) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (!params || bytes != params_bytes(h))
    return fail(AHX_EINVAL, "live solver: parameter block must be 64 + 16*nz bytes");
  AHX_CUDA(h, cudaSetDevice(h->dev));
  return upload(h, h->d_params, params, bytes);
}

ahx_status ahx_set_columns(ahx_handle* h, const uint32_t* colv) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (!colv) return fail(AHX_EINVAL, "live solver: null column records");
  for (size_t c = 0; c < nxy(h); ++c)
    if (colv[4 * c] > kMaxLevel || colv[4 * c + 1] > kMaxLevel)
      return fail(AHX_EINVAL, "live solver: column record with kt or ktop out of range");
  AHX_CUDA(h, cudaSetDevice(h->dev));
  return upload(h, h->d_colv, colv, nxy(h) * sizeof(uint4));
}

ahx_status ahx_set_ktop(ahx_handle* h, const uint32_t* ktop, const uint32_t* old_ktop) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (!ktop) return fail(AHX_EINVAL, "live solver: null ktop");
  for (size_t c = 0; c < nxy(h); ++c)
    if (ktop[c] > kMaxLevel || (old_ktop && old_ktop[c] > kMaxLevel))
      return fail(AHX_EINVAL, "live solver: ktop out of range");
  AHX_CUDA(h, cudaSetDevice(h->dev));
  if (ahx_status st = upload(h, h->d_ktop, ktop, nxy(h) * 4)) return st;
  if (old_ktop) {
    if (ahx_status st = upload(h, h->d_oldk, old_ktop, nxy(h) * 4)) return st;
    DomainView D = view(h);
    AHX_CUDA(h, launch_reinit(D, h->dims.precision, h->d_oldk, h->f[h->parity], h->g[h->parity], h->s_step));
  }
  return AHX_OK;
}

ahx_status ahx_init_flow(ahx_handle* h) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  AHX_CUDA(h, cudaSetDevice(h->dev));
  DomainView D = view(h);
  AHX_CUDA(h, launch_init(D, h->dims.precision, h->f[0], h->f[1], h->s_step));
  // a re-initialised flow continues like a fresh handle: the stochastic-rounding step counter restarts too
  AHX_CUDA(h, cudaMemsetAsync(h->d_tick, 0, 2 * sizeof(uint32_t), h->s_step));
  return AHX_OK;
}

ahx_status ahx_clear_heat(ahx_handle* h) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  AHX_CUDA(h, cudaSetDevice(h->dev));
  for (int p = 0; p < 2; ++p) AHX_CUDA(h, cudaMemsetAsync(h->g[p], 0, 7ull * h->qs * h->esize_g, h->s_step));
  return AHX_OK;
}

ahx_status ahx_set_parity(ahx_handle* h, int parity) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (parity != 0 && parity != 1) return fail(AHX_EINVAL, "live solver: parity must be 0 or 1");
  h->parity = parity;
  return AHX_OK;
}


// two plain steps starting at parity p, captured once per launch set-up and replayed (launch gaps matter for small
// grids, where a step takes tens of microseconds)
static ahx_status step_graph(ahx_handle* h, const StepLaunch& L0, int p, cudaGraphExec_t* out) {
  const uint64_t key = solo_launch_key(h);
  if (h->graph[p] && h->graph_key[p] == key) {
    *out = h->graph[p];
    return AHX_OK;
  }
  if (h->graph[p]) cudaGraphExecDestroy(h->graph[p]);
  h->graph[p] = nullptr;
  h->graph_key[p] = 0;
  cudaGraph_t g = nullptr;
  AHX_CUDA(h, cudaStreamBeginCapture(h->s_step, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < 2 && e == cudaSuccess; ++s) e = solo_step(h, p ^ s, h->s_step);
  const cudaError_t e2 = cudaStreamEndCapture(h->s_step, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cuda_fail(h, e != cudaSuccess ? e : e2, "step graph capture");
  }
  const cudaError_t e3 = cudaGraphInstantiate(&h->graph[p], g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) {
    h->graph[p] = nullptr;
    return cuda_fail(h, e3, "step graph instantiate");
  }
  h->graph_key[p] = key;
  *out = h->graph[p];
  return AHX_OK;
}

// the launch set-up of this handle's steps (mode and tensor maps are per step)
static StepLaunch step_launch(const ahx_handle* h) {
  StepLaunch L = solo_launch(h, h->parity);
  L.budget = h->budget_on || h->accum_on;
  return L;
}

// whether n steps in this mode replay the two-step graph
static bool graph_steps(const ahx_handle* h, int n, int mode) {
  return mode == AHX_MODE_NONE && !(h->budget_on || h->accum_on) && n >= 2;
}

ahx_status ahx_step(ahx_handle* h, int n, int mode) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (n < 0 || mode < 0 || mode > 2) return fail(AHX_EINVAL, "live solver: bad step count or mode");
  AHX_CUDA(h, cudaSetDevice(h->dev));
  if (mode != AHX_MODE_NONE)
    if (ahx_status st = ensure_dbg(h)) return st;
  StepLaunch L = step_launch(h);
  int s = 0;
  if (graph_steps(h, n, mode)) {
    // pairs of plain steps from the captured graph of the current parity
    cudaGraphExec_t g = nullptr;
    if (ahx_status st = step_graph(h, L, h->parity, &g)) return st;
    for (; s + 2 <= n; s += 2) {
      AHX_CUDA(h, cudaGraphLaunch(g, h->s_step));
      h->steps += 2;
    }
  }
  for (; s < n; ++s) {
    L.mode = (mode == AHX_MODE_ACC) ? 2 : ((mode == AHX_MODE_OUT && s == n - 1) ? 1 : 0);
    L.maps = stage_maps(h, L, h->parity);
    DomainView D = view(h);
    const cudaError_t e = h->dims.arith == AHX_ARITH_FAST ? fast::launch_step(D, L, h->s_step)
                                                            : exact::launch_step(D, L, h->s_step);
    if (e != cudaSuccess) return cuda_fail(h, e, "step launch");
    h->parity ^= 1;
    ++h->steps;
    if (h->accum_on) ++h->accum_steps;
  }
  return AHX_OK;
}

ahx_status ahx_time_steps(ahx_handle* h, int n, int mode, int timeout_ms, float* ms) {
  if (!h || !ms) return fail(AHX_EINVAL, "live solver: null argument");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  {
    std::lock_guard<std::mutex> lk(h->mu);
    if (ahx_status st = check(h)) return st;
    AHX_CUDA(h, cudaSetDevice(h->dev));
    if (n < 0 || mode < 0 || mode > 2) return fail(AHX_EINVAL, "live solver: bad step count or mode");
    if (graph_steps(h, n, mode)) {   // capture outside the timed region
      cudaGraphExec_t g = nullptr;
      if (ahx_status st = step_graph(h, step_launch(h), h->parity, &g)) return st;
    }
    AHX_CUDA(h, cudaEventCreate(&e0));
    AHX_CUDA(h, cudaEventCreate(&e1));
    AHX_CUDA(h, cudaEventRecord(e0, h->s_step));
  }
  ahx_status st = ahx_step(h, n, mode);
  if (st == AHX_OK) {
    std::lock_guard<std::mutex> lk(h->mu);
    const cudaError_t e = cudaEventRecord(e1, h->s_step);
    if (e != cudaSuccess) st = cuda_fail(h, e, "cudaEventRecord");
  }
  if (st == AHX_OK) st = wait_event(h, e1, timeout_ms);
  if (st == AHX_OK) {
    const cudaError_t e = cudaEventElapsedTime(ms, e0, e1);
    if (e != cudaSuccess) st = cuda_fail(h, e, "cudaEventElapsedTime");
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st == AHX_OK) {
    std::lock_guard<std::mutex> lk(h->mu);
    st = check_kernel_error(h);
  }
  return st;
}

ahx_status ahx_sync(ahx_handle* h, int timeout_ms) {
  cudaEvent_t ev = nullptr;
  {
    if (!h) return fail(AHX_EINVAL, "live solver: null handle");
    std::lock_guard<std::mutex> lk(h->mu);
    if (ahx_status st = check(h)) return st;
    AHX_CUDA(h, cudaSetDevice(h->dev));
    AHX_CUDA(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    AHX_CUDA(h, cudaEventRecord(ev, h->s_step));
  }
  ahx_status st = wait_event(h, ev, timeout_ms);
  cudaEventDestroy(ev);
  if (st == AHX_OK) {
    std::lock_guard<std::mutex> lk(h->mu);
    st = check_kernel_error(h);
  }
  return st;
}

ahx_status ahx_fence(ahx_handle* h, uint64_t* ticket) {
  if (!h || !ticket) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  AHX_CUDA(h, cudaSetDevice(h->dev));
  // bound the number of outstanding fences: retire the oldest ones that already passed
  if (h->fences.size() > 256) {
    std::vector<Fence> keep;
    for (auto& f : h->fences) {
      if (cudaEventQuery(f.ev) == cudaSuccess) cudaEventDestroy(f.ev);
      else keep.push_back(f);
    }
    cudaGetLastError();
    h->fences.swap(keep);
  }
  Fence f;
  f.ticket = ++h->next_fence;
  AHX_CUDA(h, cudaEventCreateWithFlags(&f.ev, cudaEventDisableTiming));
  AHX_CUDA(h, cudaEventRecord(f.ev, h->s_step));
  h->fences.push_back(f);
  *ticket = f.ticket;
  return AHX_OK;
}

ahx_status ahx_fence_query(ahx_handle* h, uint64_t ticket, int* done) {
  if (!h || !done) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  *done = 1;   // unknown or retired tickets have passed
  for (size_t a = 0; a < h->fences.size(); ++a) {
    if (h->fences[a].ticket != ticket) continue;
    const cudaError_t e = cudaEventQuery(h->fences[a].ev);
    if (e == cudaErrorNotReady) {
      *done = 0;
    } else if (e != cudaSuccess) {
      return cuda_fail(h, e, "cudaEventQuery");
    } else {
      cudaEventDestroy(h->fences[a].ev);
      h->fences.erase(h->fences.begin() + a);
    }
    break;
  }
  return AHX_OK;
}

ahx_status ahx_read_submit(ahx_handle* h, float conv, float volscale, int nzv, int want_vol, int want_wind,
                           uint64_t* ticket) {
  if (!h || !ticket) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (nzv < 0 || nzv > h->dims.nz) return fail(AHX_EINVAL, "live solver: nzv out of range");
  ReadSlot* r = nullptr;
  for (auto& s : h->reads)
    if (!s.busy) {
      r = &s;
      break;
    }
  if (!r) return fail(AHX_EBUSY, "live solver: too many reads in flight");
  AHX_CUDA(h, cudaSetDevice(h->dev));
  const size_t NXY = nxy(h);
  DomainView D = view(h);
  AHX_CUDA(h, cudaMemsetAsync(r->d_tmax, 0, 4, h->s_step));
  AHX_CUDA(h, launch_surf(D, h->dims.precision, conv, r->d_surf, h->s_step));
  AHX_CUDA(h, launch_vol(D, h->dims.precision, nzv, volscale, r->d_vol, r->d_tmax, h->s_step));
  AHX_CUDA(h, cudaEventRecord(r->ev_kernels, h->s_step));
  AHX_CUDA(h, cudaStreamWaitEvent(h->s_copy, r->ev_kernels, 0));
  AHX_CUDA(h, cudaMemcpyAsync(r->h_surf, r->d_surf, (want_wind ? 3 : 1) * NXY * 4, cudaMemcpyDeviceToHost,
                              h->s_copy));
  if (want_vol && nzv > 0)
    AHX_CUDA(h, cudaMemcpyAsync(r->h_vol, r->d_vol, (size_t)nzv * NXY, cudaMemcpyDeviceToHost, h->s_copy));
  AHX_CUDA(h, cudaMemcpyAsync(r->h_tmax, r->d_tmax, 4, cudaMemcpyDeviceToHost, h->s_copy));
  AHX_CUDA(h, cudaEventRecord(r->ev_done, h->s_copy));
  r->busy = true;
  r->ticket = ++h->next_read;
  r->nzv = nzv;
  r->want_vol = want_vol;
  r->want_wind = want_wind;
  *ticket = r->ticket;
  return AHX_OK;
}

ahx_status ahx_read_wait(ahx_handle* h, uint64_t ticket, int timeout_ms, float* surf, float* u, float* v,
                         uint8_t* vol, float* theta_max) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  ReadSlot* r = nullptr;
  cudaEvent_t ev;
  {
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->destroyed) return fail(AHX_EDESTROYED, "live solver: read failed (solver destroyed)");
    for (auto& s : h->reads)
      if (s.busy && s.ticket == ticket) r = &s;
    if (!r) return fail(AHX_EINVAL, "live solver: unknown read ticket");
    ev = r->ev_done;
  }
  if (ahx_status st = wait_event(h, ev, timeout_ms)) return st;
  std::lock_guard<std::mutex> lk(h->mu);
  if (h->destroyed) return fail(AHX_EDESTROYED, "live solver: read failed (solver destroyed)");
  const size_t NXY = nxy(h);
  if (surf) std::memcpy(surf, r->h_surf, NXY * 4);
  if (r->want_wind) {
    if (u) std::memcpy(u, r->h_surf + NXY, NXY * 4);
    if (v) std::memcpy(v, r->h_surf + 2 * NXY, NXY * 4);
  }
  if (vol && r->want_vol) std::memcpy(vol, r->h_vol, (size_t)r->nzv * NXY);
  if (theta_max) std::memcpy(theta_max, r->h_tmax, 4);
  r->busy = false;
  return AHX_OK;
}

static ahx_status state_io(ahx_handle* h, void* f, void* g, bool is_f64, bool to_host) {
  AHX_CUDA(h, cudaSetDevice(h->dev));
  const size_t N = ncells(h);
  const size_t eb = is_f64 ? 8 : 4;
  void* stage = nullptr;
  if (cudaMalloc(&stage, N * eb) != cudaSuccess) {
    cudaGetLastError();
    return fail(AHX_ENOMEM, "live solver: staging allocation failed");
  }
  DomainView D = view(h);
  ahx_status st = AHX_OK;
  for (int pass = 0; pass < 2 && st == AHX_OK; ++pass) {
    void* host = pass == 0 ? f : g;
    if (!host) continue;
    const int nq = pass == 0 ? 19 : 7;
    void* dev_state = pass == 0 ? h->f[h->parity] : h->g[h->parity];
    for (int q = 0; q < nq; ++q) {
      char* hp = static_cast<char*>(host) + (size_t)q * N * eb;
      cudaError_t e;
      if (to_host) {
        e = launch_export_plane(D, h->dims.precision, dev_state, stage, is_f64, q, pass == 1, h->s_step);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hp, stage, N * eb, cudaMemcpyDeviceToHost, h->s_step);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->s_step);
      } else {
        e = cudaMemcpyAsync(stage, hp, N * eb, cudaMemcpyHostToDevice, h->s_step);
        if (e == cudaSuccess)
          e = launch_import_plane(D, h->dims.precision, stage, is_f64, dev_state, q, pass == 1, h->s_step);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->s_step);
      }
      if (e != cudaSuccess) {
        st = cuda_fail(h, e, "state copy");
        break;
      }
    }
  }
  cudaFree(stage);
  return st;
}

ahx_status ahx_read_state(ahx_handle* h, float* f, float* g) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  return state_io(h, f, g, false, true);
}

ahx_status ahx_write_state(ahx_handle* h, const float* f, const float* g) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  return state_io(h, const_cast<float*>(f), const_cast<float*>(g), false, false);
}

ahx_status ahx_read_state_f64(ahx_handle* h, double* f, double* g) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  return state_io(h, f, g, true, true);
}

ahx_status ahx_write_state_f64(ahx_handle* h, const double* f, const double* g) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  return state_io(h, const_cast<double*>(f), const_cast<double*>(g), true, false);
}

ahx_status ahx_read_dbg(ahx_handle* h, float* dbg4) {
  if (!h || !dbg4) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  AHX_CUDA(h, cudaSetDevice(h->dev));
  if (ahx_status st = ensure_dbg(h)) return st;
  const size_t rows = (size_t)h->dims.ny * h->dims.nz;
  AHX_CUDA(h, cudaMemcpy2DAsync(dbg4, (size_t)h->dims.nx * 16, h->d_dbg, (size_t)h->px * 16,
                                (size_t)h->dims.nx * 16, rows, cudaMemcpyDeviceToHost, h->s_step));
  AHX_CUDA(h, cudaStreamSynchronize(h->s_step));
  return AHX_OK;
}

ahx_status ahx_clear_dbg(ahx_handle* h) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  AHX_CUDA(h, cudaSetDevice(h->dev));
  if (ahx_status st = ensure_dbg(h)) return st;
  AHX_CUDA(h, cudaMemsetAsync(h->d_dbg, 0, (size_t)h->ps * h->dims.nz * sizeof(float4), h->s_step));
  return AHX_OK;
}

ahx_status ahx_stats(ahx_handle* h, ahx_stats_out* out) {
  if (!h || !out) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  AHX_CUDA(h, cudaSetDevice(h->dev));
  AHX_CUDA(h, cudaMemsetAsync(h->d_stats, 0, sizeof(StatsScratch), h->s_step));
  DomainView D = view(h);
  AHX_CUDA(h, launch_stats(D, h->dims.precision, h->d_stats, h->s_step));
  StatsScratch s;
  AHX_CUDA(h, cudaMemcpyAsync(&s, h->d_stats, sizeof(s), cudaMemcpyDeviceToHost, h->s_step));
  AHX_CUDA(h, cudaStreamSynchronize(h->s_step));
  std::memset(out, 0, sizeof(*out));
  out->sum_theta = s.sum[0];
  out->sum_ke = s.sum[1];
  out->sum_rho_dev = s.sum[2];
  out->count = s.sum[3];
  std::memcpy(&out->theta_max, &s.tmax_bits, 4);
  std::memcpy(&out->umax, &s.umax_bits, 4);
  out->non_finite = s.non_finite;
  return AHX_OK;
}

ahx_status ahx_budget_enable(ahx_handle* h, int on) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  h->budget_on = on != 0;
  return AHX_OK;
}

ahx_status ahx_budget_read(ahx_handle* h, ahx_budget_out* out, int reset) {
  if (!h || !out) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  AHX_CUDA(h, cudaSetDevice(h->dev));
  std::vector<double> b((size_t)kBudgetSlots * kBudgetStride);
  AHX_CUDA(h, cudaMemcpyAsync(b.data(), h->d_budget, b.size() * sizeof(double), cudaMemcpyDeviceToHost, h->s_step));
  if (reset) AHX_CUDA(h, cudaMemsetAsync(h->d_budget, 0, b.size() * sizeof(double), h->s_step));
  AHX_CUDA(h, cudaStreamSynchronize(h->s_step));
  double acc[11] = {0};
  for (int s = 0; s < kBudgetSlots; ++s)
    for (int a = 0; a < 11; ++a) acc[a] += b[(size_t)s * kBudgetStride + a];
  std::memset(out, 0, sizeof(*out));
  out->theta_sum = acc[0];
  out->src_sum = acc[1];
  for (int a = 0; a < 4; ++a) {
    out->face_theta_u[a] = acc[2 + a];
    out->face_u[a] = acc[6 + a];
  }
  out->cells = acc[10];
  return AHX_OK;
}

size_t face_doubles(const ahx_handle* h) {
  return 2 * (2 * (size_t)h->dims.ny * h->dims.nz + 2 * (size_t)h->dims.nx * h->dims.nz);
}

ahx_status ahx_accum_enable(ahx_handle* h, int on) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  AHX_CUDA(h, cudaSetDevice(h->dev));
  if (on && !h->d_sacc) {
    if (cudaMalloc(&h->d_sacc, 3 * nxy(h) * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->d_facc, face_doubles(h) * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      if (h->d_sacc) cudaFree(h->d_sacc);
      h->d_sacc = nullptr;
      return fail(AHX_ENOMEM, "live solver: accumulator allocation failed");
    }
    AHX_CUDA(h, cudaMemsetAsync(h->d_sacc, 0, 3 * nxy(h) * sizeof(double), h->s_step));
    AHX_CUDA(h, cudaMemsetAsync(h->d_facc, 0, face_doubles(h) * sizeof(double), h->s_step));
    h->accum_steps = 0;
  }
  h->accum_on = on != 0;
  return AHX_OK;
}

ahx_status ahx_accum_read(ahx_handle* h, double* surf3, double* faces, int64_t* steps, int reset) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (!h->d_sacc) return fail(AHX_EINVAL, "live solver: accumulators were never enabled");
  AHX_CUDA(h, cudaSetDevice(h->dev));
  if (surf3)
    AHX_CUDA(h, cudaMemcpyAsync(surf3, h->d_sacc, 3 * nxy(h) * sizeof(double), cudaMemcpyDeviceToHost, h->s_step));
  if (faces)
    AHX_CUDA(h, cudaMemcpyAsync(faces, h->d_facc, face_doubles(h) * sizeof(double), cudaMemcpyDeviceToHost,
                                h->s_step));
  if (reset) {
    AHX_CUDA(h, cudaMemsetAsync(h->d_sacc, 0, 3 * nxy(h) * sizeof(double), h->s_step));
    AHX_CUDA(h, cudaMemsetAsync(h->d_facc, 0, face_doubles(h) * sizeof(double), h->s_step));
  }
  AHX_CUDA(h, cudaStreamSynchronize(h->s_step));
  if (steps) *steps = h->accum_steps;
  if (reset) h->accum_steps = 0;
  return AHX_OK;
}

ahx_status ahx_set_slab(ahx_handle* h, int jg0, int nyg, int jlo, int jhi) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  const int ny = h->dims.ny;
  if (nyg < ny || jg0 < 0 || jg0 + ny > nyg || jlo < 0 || jhi > ny || jlo >= jhi)
    return fail(AHX_EINVAL, "live solver: bad slab (need 0 <= jg0, jg0 + ny <= nyg, 0 <= jlo < jhi <= ny)");
  if (h->batch_refs > 0) return fail(AHX_EINVAL, "live solver: a batch member cannot become a slab");
  h->jg0 = jg0;
  h->nyg = nyg;
  h->jlo = jlo;
  h->jhi = jhi;
  // the staged kernels update whole row blocks: slabs use the plain kernels
  h->maps_ok = false;
  h->pmaps_ok = false;
  h->tma_ty = h->tma_depth = 0;
  return AHX_OK;
}

ahx_status ahx_row_bytes(ahx_handle* h, size_t* bytes) {
  if (!h || !bytes) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  const size_t per = (size_t)h->dims.nz * h->dims.nx;
  *bytes = ((19 * per * h->esize + 15) & ~(size_t)15) + 7 * per * h->esize_g;   // f part padded to 16 bytes
  return AHX_OK;
}

static ahx_status row_copy(ahx_handle* h, int j, void* buf, int to_buffer) {
  if (!h || !buf) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (j < 0 || j >= h->dims.ny) return fail(AHX_EINVAL, "live solver: row out of range");
  AHX_CUDA(h, cudaSetDevice(h->dev));
  const DomainView D = view(h);
  AHX_CUDA(h, launch_row_copy(D, h->dims.precision, j, buf, to_buffer, h->s_step));
  return AHX_OK;
}

ahx_status ahx_row_pack(ahx_handle* h, int j, void* dst_device) { return row_copy(h, j, dst_device, 1); }
ahx_status ahx_row_unpack(ahx_handle* h, int j, const void* src_device) {
  return row_copy(h, j, const_cast<void*>(src_device), 0);
}

ahx_status ahx_halo_bytes(ahx_handle* h, size_t* bytes) {
  if (!h || !bytes) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  const size_t per = (size_t)h->dims.nz * h->dims.nx;
  *bytes = ((5 * per * h->esize + 15) & ~(size_t)15) + per * h->esize_g;   // f part padded to 16 bytes
  return AHX_OK;
}

static ahx_status halo_copy(ahx_handle* h, int j, int dir, int next, void* buf, int to_buffer) {
  if (!h || !buf) return fail(AHX_EINVAL, "live solver: null argument");
  if (dir != 1 && dir != -1) return fail(AHX_EINVAL, "live solver: halo direction must be +1 or -1");
  if ((reinterpret_cast<uintptr_t>(buf) & 15) != 0) return fail(AHX_EINVAL, "live solver: halo buffer not 16-byte aligned");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (j < 0 || j >= h->dims.ny) return fail(AHX_EINVAL, "live solver: row out of range");
  AHX_CUDA(h, cudaSetDevice(h->dev));
  const DomainView D = view(h);
  AHX_CUDA(h, launch_halo_copy(D, h->dims.precision, j, dir, next, buf, to_buffer, h->s_step));
  return AHX_OK;
}

ahx_status ahx_halo_pack(ahx_handle* h, int j, int dir, int next, void* dst_device) {
  return halo_copy(h, j, dir, next ? 1 : 0, dst_device, 1);
}
ahx_status ahx_halo_unpack(ahx_handle* h, int j, int dir, const void* src_device) {
  return halo_copy(h, j, dir, 0, const_cast<void*>(src_device), 0);
}

ahx_status ahx_step_rows(ahx_handle* h, int j0, int j1, int advance) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  const int lo = h->nyg > 0 ? h->jlo : 0, hi = h->nyg > 0 ? h->jhi : h->dims.ny;
  if (j0 < lo || j1 > hi || j0 > j1) return fail(AHX_EINVAL, "live solver: rows outside the updated range");
  if (h->dims.precision == AHX_FP16_SR)
    return fail(AHX_EINVAL, "live solver: a stochastic-rounding state steps whole (its dithers count the step's blocks)");
  if (h->budget_on || h->accum_on)
    return fail(AHX_EINVAL, "live solver: budgets and accumulators are taken over whole steps");
  AHX_CUDA(h, cudaSetDevice(h->dev));
  if (j1 > j0) {
    StepLaunch L = solo_launch(h, h->parity);
    L.tma_ty = 0;
    L.maps = nullptr;
    DomainView D = view(h);
    D.jlo = j0;
    D.jhi = j1;
    D.jbase = j0;
    AHX_CUDA(h, h->dims.arith == AHX_ARITH_FAST ? fast::launch_step(D, L, h->s_step) : exact::launch_step(D, L, h->s_step));
  }
  if (advance) {
    h->parity ^= 1;
    ++h->steps;
  }
  return AHX_OK;
}

ahx_status ahx_set_launch(ahx_handle* h, int block_y, int zslab) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  const bool pf = block_y >= 10000;   // next-level L2 prefetch: 10000 + the plain or paired encoding
  if (pf) {
    if (h->dims.arith != AHX_ARITH_FAST) return fail(AHX_EINVAL, "live solver: the L2 prefetch needs the FMA build");
    block_y -= 10000;
  }
  const bool pairs = block_y >= 2000;   // paired levels: 2000 + the plain encoding
  if (pairs) {
    if (h->dims.arith != AHX_ARITH_FAST || h->dims.precision == AHX_FP64)
      return fail(AHX_EINVAL, "live solver: paired levels need the FMA build and f32 arithmetic");
    block_y -= 2000;
  }
  if (block_y >= 1000 && pairs) {
    // staged paired step of the 16-bit storages: 2000 + 1000 + 100 x depth + rows (4 with depth 2-4, or 8 with
    // depth 2-3)
    const int ty = block_y % 100, dp = (block_y / 100) % 10;
    if (!((ty == 4 && dp >= 2 && dp <= 4) || (ty == 8 && dp >= 2 && dp <= 3)) || zslab < 0)
      return fail(AHX_EINVAL, "live solver: bad staged paired launch shape");
    if (!h->pmaps_ok)
      return fail(AHX_EINVAL, "live solver: the staged paired step needs a whole-domain 16-bit state (FP16, BF16 or "
                              "FP16 with stochastic rounding)");
    if (pf) return fail(AHX_EINVAL, "live solver: the staged paired step has no prefetch variant");
    h->tma_ty = ty;
    h->tma_depth = dp;
    h->block_y = ty;
    h->minb = 0;
    h->pairs = true;
    h->prefetch = false;
  } else if (block_y >= 1000) {   // staged kernel: 1000 + 100 x depth + rows (4 with depth 2-4, or 8 with depth 2-3)
    const int ty = block_y % 100, dp = (block_y / 100) % 10;
    if (!((ty == 4 && dp >= 2 && dp <= 4) || (ty == 8 && dp >= 2 && dp <= 3)) || zslab < 0)
      return fail(AHX_EINVAL, "live solver: bad staged launch shape");
    if (!h->maps_ok) return fail(AHX_EINVAL, "live solver: tensor maps unavailable for the staged kernel");
    if (pf) return fail(AHX_EINVAL, "live solver: the staged kernel has no prefetch variant");
    h->tma_ty = ty;
    h->tma_depth = dp;
    h->block_y = ty;
    h->minb = 0;
    h->pairs = false;
    h->prefetch = false;
  } else {
    const int by = block_y % 100, mb = block_y / 100;
    if (by < 0 || by > 8 || zslab < 0 || (mb != 0 && (mb < 4 || mb > 6) && mb != 8) || (mb && by != 4))
      return fail(AHX_EINVAL, "live solver: bad launch shape");
    if (block_y || pairs || pf) {
      h->block_y = by ? by : 4;
      h->minb = mb;
      h->tma_ty = 0;
      h->tma_depth = 0;
      h->pairs = pairs;
      h->prefetch = pf;
    }
  }
  if (zslab) h->zslab = zslab;
  return AHX_OK;
}

ahx_status ahx_autotune(ahx_handle* h, int steps_per_trial, int* best_block_y, int* best_zslab, float* best_ms) {
  if (!h) return fail(AHX_EINVAL, "live solver: null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (ahx_status st = check(h)) return st;
  if (steps_per_trial < 1) steps_per_trial = 4;
  AHX_CUDA(h, cudaSetDevice(h->dev));
  // trials ping-pong between the two state buffers, so they would advance the state: run them on a copy
  const size_t fbytes = 19ull * h->qs * h->esize, gbytes = 7ull * h->qs * h->esize_g;
  void *f0 = nullptr, *f1 = nullptr, *g0 = nullptr, *g1 = nullptr;
  if (cudaMalloc(&f0, fbytes) != cudaSuccess || cudaMalloc(&f1, fbytes) != cudaSuccess ||
      cudaMalloc(&g0, gbytes) != cudaSuccess || cudaMalloc(&g1, gbytes) != cudaSuccess) {
    cudaFree(f0);
    cudaFree(f1);
    cudaFree(g0);
    cudaFree(g1);
    cudaGetLastError();
    return fail(AHX_ENOMEM, "live solver: autotune needs a second copy of the state");
  }
  AHX_CUDA(h, cudaMemcpyAsync(f0, h->f[h->parity], fbytes, cudaMemcpyDeviceToDevice, h->s_step));
  AHX_CUDA(h, cudaMemcpyAsync(g0, h->g[h->parity], gbytes, cudaMemcpyDeviceToDevice, h->s_step));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  struct Shape {
    int by, minb, ty, depth;
    bool pairs;
  };
  std::vector<Shape> shapes = {{2, 0, 0, 0, false}, {4, 0, 0, 0, false}, {8, 0, 0, 0, false},
                               {4, 4, 0, 0, false}, {4, 5, 0, 0, false}, {4, 6, 0, 0, false},
                               {4, 8, 0, 0, false}};
  if (h->dims.arith == AHX_ARITH_FAST && h->dims.precision != AHX_FP64)
    for (Shape sh : {Shape{4, 4, 0, 0, true}, Shape{4, 5, 0, 0, true}, Shape{4, 6, 0, 0, true},
                     Shape{4, 8, 0, 0, true}})
      shapes.push_back(sh);
  // The TMA-staged kernels are not candidates. The single-level one never won a trial (16-20 against 26.6 GLUPS on
  // 600x600x64) and an early build of it once stopped with a misaligned-address error whose cause was not found; the
  // staged paired step of the 16-bit storages runs 0.76-0.81 of the plain paired step's rate there (27.6-29.1 against
  // 36.1 GLUPS when measured: half the resident warps, a block barrier per level pair). Both stay reachable only
  // through explicit ahx_set_launch values.
  // thin slabs put more blocks in flight on small grids, where one 6-level wave leaves the SMs latency-bound
  std::vector<int> zss = {h->dims.nz, 32, 16, 12, 8, 6, 4, 3, 2};
  DomainView D = view(h);
  D.dbg = nullptr;
  D.tick = h->d_tick + 2;   // trials advance a scratch step counter, not the handle's
  StepLaunch L;
  L.precision = h->dims.precision;
  L.mode = 0;
  L.budget = false;
  ahx_status st = AHX_OK;
  // one trial: a warm-up round, then steps_per_trial timed steps (ms per step)
  auto trial = [&](const Shape& sh, int zs, int pf, float* out) -> ahx_status {
    L.block_y = sh.by;
    L.minb = sh.minb;
    L.pairs = sh.pairs;
    L.tma_ty = sh.ty;
    L.tma_depth = sh.depth;
    L.zslab = zs;
    D.pf = pf;
    float ms = 0;
    for (int rep = 0; rep < 2; ++rep) {   // rep 0 warms up
      cudaEventRecord(e0, h->s_step);
      for (int s = 0; s < steps_per_trial; ++s) {
        D.fA = (s & 1) ? f1 : f0;
        D.fB = (s & 1) ? f0 : f1;
        D.gA = (s & 1) ? g1 : g0;
        D.gB = (s & 1) ? g0 : g1;
        set_pointers(D, h->esize, h->esize_g);
        L.maps = nullptr;
        const cudaError_t e = h->dims.arith == AHX_ARITH_FAST ? fast::launch_step(D, L, h->s_step)
                                                                : exact::launch_step(D, L, h->s_step);
        if (e != cudaSuccess) return cuda_fail(h, e, "autotune launch");
        // each trial launch completes before the next is queued, so an error is charged to the shape that made it
        const cudaError_t e2 = cudaStreamSynchronize(h->s_step);
        if (e2 != cudaSuccess) {
          char what[112];
          std::snprintf(what, sizeof(what),
                        "autotune trial (rows %d, variant %d, staged %d/%d, paired %d, zslab %d, prefetch %d)", sh.by,
                        sh.minb, sh.ty, sh.depth, (int)sh.pairs, zs, pf);
          return cuda_fail(h, e2, what);
        }
      }
      cudaEventRecord(e1, h->s_step);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&ms, e0, e1);
    }
    *out = ms / steps_per_trial;
    return AHX_OK;
  };
  struct Cand {
    Shape sh;
    int zs, pf;
    float ms;
  };
  std::vector<Cand> res;
  for (const Shape& sh : shapes) {
    for (int zs : zss) {
      if (zs > h->dims.nz) continue;
      if (sh.ty && zs < 16) continue;   // the staged kernel needs a few levels per block to fill its pipeline
      float ms = 0;
      if ((st = trial(sh, zs, 0, &ms)) != AHX_OK) break;
      res.push_back(Cand{sh, zs, 0, ms});
    }
    if (st != AHX_OK) break;
  }
  // the next-level L2 prefetch (FMA build, plain kernel) on the three fastest plain candidates: it helps grids whose
  // steps are latency-bound and costs issue slots where the step already streams near the copy bandwidth
  if (st == AHX_OK && h->dims.arith == AHX_ARITH_FAST) {
    std::vector<Cand> top;
    for (const Cand& c : res)
      if (!c.sh.ty) top.push_back(c);
    std::sort(top.begin(), top.end(), [](const Cand& a, const Cand& b) { return a.ms < b.ms; });
    if (top.size() > 3) top.resize(3);
    for (const Cand& c : top) {
      float ms = 0;
      if ((st = trial(c.sh, c.zs, 1, &ms)) != AHX_OK) break;
      res.push_back(Cand{c.sh, c.zs, 1, ms});
    }
  }
  float best = 1e30f;
  int bby = h->block_y, bzs = h->zslab, bmb = h->minb, bty = h->tma_ty, bdp = h->tma_depth, bpf = h->prefetch;
  bool bpr = h->pairs;
  for (const Cand& c : res)
    if (c.ms < best) {
      best = c.ms;
      bby = c.sh.by;
      bzs = c.zs;
      bmb = c.sh.minb;
      bty = c.sh.ty;
      bdp = c.sh.depth;
      bpr = c.sh.pairs;
      bpf = c.pf;
    }
  if (st == AHX_OK) st = check_kernel_error(h);
  cudaStreamSynchronize(h->s_step);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(f0);
  cudaFree(f1);
  cudaFree(g0);
  cudaFree(g1);
  if (st != AHX_OK) return st;
  h->block_y = bby;
  h->zslab = bzs;
  h->minb = bmb;
  h->tma_ty = bty;
  h->tma_depth = bdp;
  h->pairs = bpr;
  h->prefetch = bpf != 0;
  // the ahx_set_launch encoding: variant x 100 + block_y (+ 2000 for paired levels, + 10000 for the L2 prefetch),
  // or 1000 + 100 x depth + rows for a staged kernel (+ 2000 for the staged paired step)
  if (best_block_y)
    *best_block_y = bty ? (bpr ? 2000 : 0) + 1000 + 100 * bdp + bty
                        : (bpf ? 10000 : 0) + (bpr ? 2000 : 0) + bmb * 100 + bby;
  if (best_zslab) *best_zslab = bzs;
  if (best_ms) *best_ms = best;
  return AHX_OK;
}

}  // extern "C"
