// N-API addon over libahx.so (include/ahx.h): what a Node host loads to drive the live solver's CUDA backend in place
// of WebGPU. One JS function per C-ABI operation the reference's solver.js performs on its device (parameter block,
// column records, ktop plane, init / clear / parity, steps, read-back, state and diagnostics hooks; solver.js:137-578).
//
// Threading: the C ABI is thread-safe per handle. Calls that only queue device work (uploads, steps, read submission)
// run on the JS thread and return at once. The two waits the reference expresses as promises become async work on
// libuv's thread pool: step(n) resolves when the fence recorded after its steps has passed (solver.js:401-405,
// queue.onSubmittedWorkDone), read() resolves when its read-back has arrived in host memory (solver.js:439-471,
// mapAsync), with the result arrays allocated on the JS thread beforehand and filled by the worker. Errors reject with
// the library's message (ahx_last_error); a lost device rejects every later call, as the reference's lost device does.
//
// Build: node-gyp rebuild (binding.gyp links ../libahx.so). The exact C-ABI calls of each operation are listed in
// call_sequences.json.
#include <node_api.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>

#include "ahx.h"

namespace {

// ---------------------------------------------------------------- small helpers

napi_value undefined(napi_env env) {
  napi_value u;
  napi_get_undefined(env, &u);
  return u;
}

napi_value throw_error(napi_env env, const std::string& msg) {
  napi_throw_error(env, nullptr, msg.c_str());
  return nullptr;
}

// a C-ABI status as a JS exception carrying ahx_last_error()
napi_value throw_status(napi_env env, ahx_status st) {
  return throw_error(env, std::string(ahx_last_error()) + " (status " + std::to_string((int)st) + ")");
}

#define AHX_JS(env, call)                              \
  do {                                                 \
    const ahx_status st_ = (call);                     \
    if (st_ != AHX_OK) return throw_status(env, st_);  \
  } while (0)

#define NAPI_JS(env, call)                                                      \
  do {                                                                          \
    if ((call) != napi_ok) return throw_error(env, "ahx_napi: N-API call failed"); \
  } while (0)

struct Args {
  size_t argc = 8;
  napi_value argv[8];
};

bool get_args(napi_env env, napi_callback_info info, Args& a, size_t need) {
  if (napi_get_cb_info(env, info, &a.argc, a.argv, nullptr, nullptr) != napi_ok) return false;
  return a.argc >= need;
}

ahx_handle* handle_of(napi_env env, napi_value v) {
  void* p = nullptr;
  if (napi_get_value_external(env, v, &p) != napi_ok) return nullptr;
  return static_cast<ahx_handle*>(p);
}

int32_t i32(napi_env env, napi_value v, int32_t dflt = 0) {
  int32_t x = dflt;
  napi_get_value_int32(env, v, &x);
  return x;
}

double f64(napi_env env, napi_value v, double dflt = 0) {
  double x = dflt;
  napi_get_value_double(env, v, &x);
  return x;
}

bool is_nullish(napi_env env, napi_value v) {
  napi_valuetype t;
  napi_typeof(env, v, &t);
  return t == napi_null || t == napi_undefined;
}

// the bytes of a typed array, a DataView-free ArrayBuffer, or null
bool bytes_of(napi_env env, napi_value v, void** data, size_t* len) {
  bool is = false;
  napi_is_typedarray(env, v, &is);
  if (is) {
    napi_typedarray_type t;
    size_t n = 0, off = 0;
    napi_value ab;
    void* d = nullptr;
    if (napi_get_typedarray_info(env, v, &t, &n, &d, &ab, &off) != napi_ok) return false;
    size_t es = 1;
    switch (t) {
      case napi_int16_array:
      case napi_uint16_array: es = 2; break;
      case napi_int32_array:
      case napi_uint32_array:
      case napi_float32_array: es = 4; break;
      case napi_float64_array:
      case napi_bigint64_array:
      case napi_biguint64_array: es = 8; break;
      default: es = 1;
    }
    *data = d;
    *len = n * es;
    return true;
  }
  napi_is_arraybuffer(env, v, &is);
  if (is) return napi_get_arraybuffer_info(env, v, data, len) == napi_ok;
  return false;
}

// a new typed array of n elements over a fresh ArrayBuffer; *data points at its storage
napi_value new_typed(napi_env env, napi_typedarray_type t, size_t n, size_t es, void** data) {
  napi_value ab, ta;
  if (napi_create_arraybuffer(env, n * es, data, &ab) != napi_ok) return nullptr;
  if (napi_create_typedarray(env, t, n, ab, 0, &ta) != napi_ok) return nullptr;
  return ta;
}

void finalize_handle(napi_env, void* data, void*) { ahx_destroy(static_cast<ahx_handle*>(data)); }

// ---------------------------------------------------------------- lifetime

// create(nx, ny, nz, precision, device, arith) -> external handle (solver.js:137-196 device part)
napi_value Create(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 3)) return throw_error(env, "ahx_napi.create(nx, ny, nz, precision, device, arith)");
  ahx_dims d{};
  d.nx = i32(env, a.argv[0]);
  d.ny = i32(env, a.argv[1]);
  d.nz = i32(env, a.argv[2]);
  d.precision = a.argc > 3 ? i32(env, a.argv[3]) : AHX_FP32;
  d.device_ordinal = a.argc > 4 ? i32(env, a.argv[4], -1) : -1;
  d.arith = a.argc > 5 ? i32(env, a.argv[5]) : AHX_ARITH_FAST;
  ahx_handle* h = nullptr;
  AHX_JS(env, ahx_create(&d, &h));
  napi_value ext;
  NAPI_JS(env, napi_create_external(env, h, finalize_handle, nullptr, &ext));
  return ext;
}

napi_value Destroy(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.destroy(h)");
  AHX_JS(env, ahx_destroy(handle_of(env, a.argv[0])));
  return undefined(env);
}

napi_value Info(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.info(h)");
  ahx_info_out o{};
  AHX_JS(env, ahx_get_info(handle_of(env, a.argv[0]), &o));
  napi_value r, v;
  NAPI_JS(env, napi_create_object(env, &r));
  const std::pair<const char*, double> num[] = {{"nx", (double)o.nx},         {"ny", (double)o.ny},
                                                {"nz", (double)o.nz},         {"px", (double)o.px},
                                                {"precision", (double)o.precision}, {"arith", (double)o.arith},
                                                {"parity", (double)o.parity}, {"device", (double)o.device_ordinal},
                                                {"steps", (double)o.steps},   {"stateBytes", (double)o.state_bytes},
                                                {"bytesPerCell", (double)o.bytes_per_cell}};
  for (const auto& kv : num) {
    NAPI_JS(env, napi_create_double(env, kv.second, &v));
    NAPI_JS(env, napi_set_named_property(env, r, kv.first, v));
  }
  NAPI_JS(env, napi_create_string_utf8(env, o.device_name, NAPI_AUTO_LENGTH, &v));
  NAPI_JS(env, napi_set_named_property(env, r, "deviceName", v));
  return r;
}

// ---------------------------------------------------------------- host images (solver.js:225-242, 323-376)

napi_value SetParams(napi_env env, napi_callback_info info) {
  Args a;
  void* d = nullptr;
  size_t n = 0;
  if (!get_args(env, info, a, 2) || !bytes_of(env, a.argv[1], &d, &n))
    return throw_error(env, "ahx_napi.setParams(h, bytes)");
  AHX_JS(env, ahx_set_params(handle_of(env, a.argv[0]), d, n));
  return undefined(env);
}

napi_value SetColumns(napi_env env, napi_callback_info info) {
  Args a;
  void* d = nullptr;
  size_t n = 0;
  if (!get_args(env, info, a, 2) || !bytes_of(env, a.argv[1], &d, &n))
    return throw_error(env, "ahx_napi.setColumns(h, Uint32Array)");
  ahx_handle* h = handle_of(env, a.argv[0]);
  ahx_info_out o{};
  AHX_JS(env, ahx_get_info(h, &o));
  if (n != (size_t)o.nx * o.ny * 16) return throw_error(env, "ahx_napi.setColumns: expected 16 bytes per column");
  AHX_JS(env, ahx_set_columns(h, static_cast<const uint32_t*>(d)));
  return undefined(env);
}

// setKtop(h, ktop, oldKtop | null): cells that turned from solid to fluid are re-initialised when oldKtop is given
napi_value SetKtop(napi_env env, napi_callback_info info) {
  Args a;
  void *k = nullptr, *old = nullptr;
  size_t nk = 0, no = 0;
  if (!get_args(env, info, a, 2) || !bytes_of(env, a.argv[1], &k, &nk))
    return throw_error(env, "ahx_napi.setKtop(h, Uint32Array, Uint32Array | null)");
  if (a.argc > 2 && !is_nullish(env, a.argv[2]) && !bytes_of(env, a.argv[2], &old, &no))
    return throw_error(env, "ahx_napi.setKtop: oldKtop must be a Uint32Array or null");
  ahx_handle* h = handle_of(env, a.argv[0]);
  ahx_info_out o{};
  AHX_JS(env, ahx_get_info(h, &o));
  const size_t want = (size_t)o.nx * o.ny * 4;
  if (nk != want || (old && no != want)) return throw_error(env, "ahx_napi.setKtop: expected 4 bytes per column");
  AHX_JS(env, ahx_set_ktop(h, static_cast<const uint32_t*>(k), static_cast<const uint32_t*>(old)));
  return undefined(env);
}

napi_value InitFlow(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.initFlow(h)");
  AHX_JS(env, ahx_init_flow(handle_of(env, a.argv[0])));
  return undefined(env);
}

napi_value ClearHeat(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.clearHeat(h)");
  AHX_JS(env, ahx_clear_heat(handle_of(env, a.argv[0])));
  return undefined(env);
}

napi_value SetParity(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 2)) return throw_error(env, "ahx_napi.setParity(h, p)");
  AHX_JS(env, ahx_set_parity(handle_of(env, a.argv[0]), i32(env, a.argv[1])));
  return undefined(env);
}

// ---------------------------------------------------------------- stepping (solver.js:401-427)

struct StepWork {
  napi_async_work work = nullptr;
  napi_deferred deferred = nullptr;
  ahx_handle* h = nullptr;
  uint64_t fence = 0;
  ahx_status status = AHX_OK;
  std::string err;
};

void step_execute(napi_env, void* data) {
  StepWork* w = static_cast<StepWork*>(data);
  for (int spin = 0;; ++spin) {
    int done = 0;
    w->status = ahx_fence_query(w->h, w->fence, &done);
    if (w->status != AHX_OK) {
      w->err = ahx_last_error();
      return;
    }
    if (done) return;
    if (spin < 64) std::this_thread::yield();
    else std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

void step_complete(napi_env env, napi_status, void* data) {
  StepWork* w = static_cast<StepWork*>(data);
  if (w->status == AHX_OK) {
    napi_resolve_deferred(env, w->deferred, undefined(env));
  } else {
    napi_value msg, e;
    napi_create_string_utf8(env, w->err.c_str(), NAPI_AUTO_LENGTH, &msg);
    napi_create_error(env, nullptr, msg, &e);
    napi_reject_deferred(env, w->deferred, e);
  }
  napi_delete_async_work(env, w->work);
  delete w;
}

// step(h, n, mode) -> Promise resolved when the n steps have run (mode 0 none, 1 out, 2 acc)
napi_value Step(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 2)) return throw_error(env, "ahx_napi.step(h, n, mode)");
  ahx_handle* h = handle_of(env, a.argv[0]);
  const int n = i32(env, a.argv[1]);
  const int mode = a.argc > 2 ? i32(env, a.argv[2]) : AHX_MODE_NONE;
  napi_value promise;
  StepWork* w = new StepWork;
  w->h = h;
  if (napi_create_promise(env, &w->deferred, &promise) != napi_ok) {
    delete w;
    return throw_error(env, "ahx_napi.step: cannot create a promise");
  }
  ahx_status st = n > 0 ? ahx_step(h, n, mode) : AHX_OK;
  if (st == AHX_OK) st = ahx_fence(h, &w->fence);
  if (st != AHX_OK) {
    napi_value msg, e;
    napi_create_string_utf8(env, ahx_last_error(), NAPI_AUTO_LENGTH, &msg);
    napi_create_error(env, nullptr, msg, &e);
    napi_reject_deferred(env, w->deferred, e);
    delete w;
    return promise;
  }
  napi_value name;
  napi_create_string_utf8(env, "ahx_step", NAPI_AUTO_LENGTH, &name);
  napi_create_async_work(env, nullptr, name, step_execute, step_complete, w, &w->work);
  napi_queue_async_work(env, w->work);
  return promise;
}

// sync(h, timeoutMs): wait for all queued work on the JS thread (the benchmark's and destroy()'s waits)
napi_value Sync(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.sync(h, timeoutMs)");
  AHX_JS(env, ahx_sync(handle_of(env, a.argv[0]), a.argc > 1 ? i32(env, a.argv[1], -1) : -1));
  return undefined(env);
}

// ---------------------------------------------------------------- read-back (solver.js:439-471)

struct ReadWork {
  napi_async_work work = nullptr;
  napi_deferred deferred = nullptr;
  ahx_handle* h = nullptr;
  uint64_t ticket = 0;
  float* surf = nullptr;
  float* u = nullptr;
  float* v = nullptr;
  uint8_t* vol = nullptr;
  float theta_max = 0;
  napi_ref result = nullptr;   // the result object with its arrays, kept alive until completion
  ahx_status status = AHX_OK;
  std::string err;
};

void read_execute(napi_env, void* data) {
  ReadWork* w = static_cast<ReadWork*>(data);
  w->status = ahx_read_wait(w->h, w->ticket, -1, w->surf, w->u, w->v, w->vol, &w->theta_max);
  if (w->status != AHX_OK) w->err = ahx_last_error();
}

void read_complete(napi_env env, napi_status, void* data) {
  ReadWork* w = static_cast<ReadWork*>(data);
  napi_value r;
  napi_get_reference_value(env, w->result, &r);
  if (w->status == AHX_OK) {
    napi_value t;
    napi_create_double(env, (double)w->theta_max, &t);
    napi_set_named_property(env, r, "thetaMax", t);
    napi_resolve_deferred(env, w->deferred, r);
  } else {
    napi_value msg, e;
    napi_create_string_utf8(env, w->err.c_str(), NAPI_AUTO_LENGTH, &msg);
    napi_create_error(env, nullptr, msg, &e);
    napi_reject_deferred(env, w->deferred, e);
  }
  napi_delete_reference(env, w->result);
  napi_delete_async_work(env, w->work);
  delete w;
}

// read(h, conv, volscale, nzv, wantVol, wantWind) -> Promise<{surf, u, v, vol, thetaMax}>; the state read is the one
// the steps queued before this call leave (later steps do not change it)
napi_value Read(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 6)) return throw_error(env, "ahx_napi.read(h, conv, volscale, nzv, wantVol, wantWind)");
  ahx_handle* h = handle_of(env, a.argv[0]);
  const float conv = (float)f64(env, a.argv[1]), volscale = (float)f64(env, a.argv[2]);
  const int nzv = i32(env, a.argv[3]);
  bool want_vol = false, want_wind = false;
  napi_get_value_bool(env, a.argv[4], &want_vol);
  napi_get_value_bool(env, a.argv[5], &want_wind);
  ahx_info_out o{};
  AHX_JS(env, ahx_get_info(h, &o));
  const size_t NXY = (size_t)o.nx * o.ny;
  ReadWork* w = new ReadWork;
  w->h = h;
  napi_value r, arr, nul;
  napi_get_null(env, &nul);
  NAPI_JS(env, napi_create_object(env, &r));
  void* p = nullptr;
  arr = new_typed(env, napi_float32_array, NXY, 4, &p);
  w->surf = static_cast<float*>(p);
  napi_set_named_property(env, r, "surf", arr);
  if (want_wind) {
    arr = new_typed(env, napi_float32_array, NXY, 4, &p);
    w->u = static_cast<float*>(p);
    napi_set_named_property(env, r, "u", arr);
    arr = new_typed(env, napi_float32_array, NXY, 4, &p);
    w->v = static_cast<float*>(p);
    napi_set_named_property(env, r, "v", arr);
  } else {
    napi_set_named_property(env, r, "u", nul);
    napi_set_named_property(env, r, "v", nul);
  }
  if (want_vol) {
    arr = new_typed(env, napi_uint8_array, (size_t)nzv * NXY, 1, &p);
    w->vol = static_cast<uint8_t*>(p);
    napi_set_named_property(env, r, "vol", arr);
  } else {
    napi_set_named_property(env, r, "vol", nul);
  }
  napi_create_reference(env, r, 1, &w->result);
  napi_value promise;
  napi_create_promise(env, &w->deferred, &promise);
  const ahx_status st = ahx_read_submit(h, conv, volscale, nzv, want_vol ? 1 : 0, want_wind ? 1 : 0, &w->ticket);
  if (st != AHX_OK) {
    napi_value msg, e;
    napi_create_string_utf8(env, ahx_last_error(), NAPI_AUTO_LENGTH, &msg);
    napi_create_error(env, nullptr, msg, &e);
    napi_reject_deferred(env, w->deferred, e);
    napi_delete_reference(env, w->result);
    delete w;
    return promise;
  }
  napi_value name;
  napi_create_string_utf8(env, "ahx_read", NAPI_AUTO_LENGTH, &name);
  napi_create_async_work(env, nullptr, name, read_execute, read_complete, w, &w->work);
  napi_queue_async_work(env, w->work);
  return promise;
}

// ---------------------------------------------------------------- validation hooks (solver.js:496-578)

napi_value ReadState(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.readState(h)");
  ahx_handle* h = handle_of(env, a.argv[0]);
  ahx_info_out o{};
  AHX_JS(env, ahx_get_info(h, &o));
  const size_t N = (size_t)o.nx * o.ny * o.nz;
  void *pf = nullptr, *pg = nullptr;
  napi_value f = new_typed(env, napi_float32_array, 19 * N, 4, &pf);
  napi_value g = new_typed(env, napi_float32_array, 7 * N, 4, &pg);
  if (!f || !g) return throw_error(env, "ahx_napi.readState: out of memory");
  AHX_JS(env, ahx_read_state(h, static_cast<float*>(pf), static_cast<float*>(pg)));
  napi_value r;
  NAPI_JS(env, napi_create_object(env, &r));
  napi_set_named_property(env, r, "f", f);
  napi_set_named_property(env, r, "g", g);
  return r;
}

napi_value WriteState(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 3)) return throw_error(env, "ahx_napi.writeState(h, f | null, g | null)");
  ahx_handle* h = handle_of(env, a.argv[0]);
  ahx_info_out o{};
  AHX_JS(env, ahx_get_info(h, &o));
  const size_t N = (size_t)o.nx * o.ny * o.nz;
  void *pf = nullptr, *pg = nullptr;
  size_t nf = 0, ng = 0;
  if (!is_nullish(env, a.argv[1]) && (!bytes_of(env, a.argv[1], &pf, &nf) || nf != 19 * N * 4))
    return throw_error(env, "ahx_napi.writeState: f must be a Float32Array of 19 N values");
  if (!is_nullish(env, a.argv[2]) && (!bytes_of(env, a.argv[2], &pg, &ng) || ng != 7 * N * 4))
    return throw_error(env, "ahx_napi.writeState: g must be a Float32Array of 7 N values");
  AHX_JS(env, ahx_write_state(h, static_cast<const float*>(pf), static_cast<const float*>(pg)));
  return undefined(env);
}

napi_value ReadDbg(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.readDbg(h)");
  ahx_handle* h = handle_of(env, a.argv[0]);
  ahx_info_out o{};
  AHX_JS(env, ahx_get_info(h, &o));
  void* p = nullptr;
  napi_value d = new_typed(env, napi_float32_array, 4 * (size_t)o.nx * o.ny * o.nz, 4, &p);
  if (!d) return throw_error(env, "ahx_napi.readDbg: out of memory");
  AHX_JS(env, ahx_read_dbg(h, static_cast<float*>(p)));
  return d;
}

napi_value ClearDbg(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.clearDbg(h)");
  AHX_JS(env, ahx_clear_dbg(handle_of(env, a.argv[0])));
  return undefined(env);
}

napi_value Stats(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.stats(h)");
  ahx_stats_out s{};
  AHX_JS(env, ahx_stats(handle_of(env, a.argv[0]), &s));
  napi_value r, v;
  NAPI_JS(env, napi_create_object(env, &r));
  const std::pair<const char*, double> num[] = {{"sumTheta", s.sum_theta},       {"sumKE", s.sum_ke},
                                                {"sumRhoDev", s.sum_rho_dev},    {"count", s.count},
                                                {"thetaMax", (double)s.theta_max}, {"umax", (double)s.umax},
                                                {"nonFinite", (double)s.non_finite}};
  for (const auto& kv : num) {
    NAPI_JS(env, napi_create_double(env, kv.second, &v));
    NAPI_JS(env, napi_set_named_property(env, r, kv.first, v));
  }
  return r;
}

// timeSteps(h, n) -> device milliseconds of n steps (the benchmark, solver.js:474-483)
napi_value TimeSteps(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 2)) return throw_error(env, "ahx_napi.timeSteps(h, n)");
  float ms = 0;
  AHX_JS(env, ahx_time_steps(handle_of(env, a.argv[0]), i32(env, a.argv[1]), AHX_MODE_NONE, -1, &ms));
  napi_value v;
  NAPI_JS(env, napi_create_double(env, (double)ms, &v));
  return v;
}

napi_value Autotune(napi_env env, napi_callback_info info) {
  Args a;
  if (!get_args(env, info, a, 1)) return throw_error(env, "ahx_napi.autotune(h, stepsPerTrial)");
  int by = 0, zs = 0;
  float ms = 0;
  AHX_JS(env, ahx_autotune(handle_of(env, a.argv[0]), a.argc > 1 ? i32(env, a.argv[1], 3) : 3, &by, &zs, &ms));
  napi_value r, v;
  NAPI_JS(env, napi_create_object(env, &r));
  napi_create_int32(env, by, &v);
  napi_set_named_property(env, r, "blockY", v);
  napi_create_int32(env, zs, &v);
  napi_set_named_property(env, r, "zslab", v);
  napi_create_double(env, (double)ms, &v);
  napi_set_named_property(env, r, "ms", v);
  return r;
}

napi_value LastError(napi_env env, napi_callback_info) {
  napi_value v;
  napi_create_string_utf8(env, ahx_last_error(), NAPI_AUTO_LENGTH, &v);
  return v;
}

}  // namespace

NAPI_MODULE_INIT() {
  const napi_property_descriptor props[] = {
      {"create", nullptr, Create, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"destroy", nullptr, Destroy, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"info", nullptr, Info, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setParams", nullptr, SetParams, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setColumns", nullptr, SetColumns, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setKtop", nullptr, SetKtop, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"initFlow", nullptr, InitFlow, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"clearHeat", nullptr, ClearHeat, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setParity", nullptr, SetParity, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"step", nullptr, Step, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"sync", nullptr, Sync, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"read", nullptr, Read, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"readState", nullptr, ReadState, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"writeState", nullptr, WriteState, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"readDbg", nullptr, ReadDbg, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"clearDbg", nullptr, ClearDbg, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"stats", nullptr, Stats, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"timeSteps", nullptr, TimeSteps, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"autotune", nullptr, Autotune, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"lastError", nullptr, LastError, nullptr, nullptr, nullptr, napi_default, nullptr},
  };
  napi_define_properties(env, exports, sizeof(props) / sizeof(props[0]), props);
  return exports;
}
