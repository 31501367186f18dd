// The live solver's domain builder on the GPU (ahx_static_* / ahx_domain_build, include/ahx.h): the 10 m static
// planes decoded on the device once, block-aggregated to the solver spacing once per spacing, and per request the
// exact-overlap campus raster, the build_domain rules and the packed column records.
//
// Reference: js/live/domain.js, loadStatic10 row-delta decode (:41-52) and checksums (:60-62), aggregate (:89-118),
// rasterizeCampuses (:124-160), buildDomain (:166-190); the column record of js/live/solver.js:359-376. Every
// floating-point result is formed with the operations and in the order of those functions (double precision, no
// contraction: this unit is compiled with -fmad=false), so the images equal the host restatement bit for bit:
//   - aggregate: integer block sums (exact in any order); the drag-coefficient block sum sequentially, block row outer
//     and column inner, one thread per coarse cell;
//   - campus raster: one thread per coarse cell walks the campuses and their halls in list order, so a cell's overlap
//     sum and its heat accumulate in the reference's order;
//   - reductions (minimum dem, maximum ktop, counts) are order-independent (min / max / integer sums).
// North-up [row][col] with row 0 at the north edge, as domain.js; the packed records are in solver orientation (row
// j = 0 at the south edge), as solver.js uploads them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "ahx.h"
#include "launch.h"

namespace {

constexpr double kSceneX0 = -2995.0, kSceneZ0 = -2995.0;   // domain.js:7-8

struct Agg {
  int r = 0, nx = 0, ny = 0;
  double dx = 0;
  double* dem = nullptr;     // block mean of the 10 m dem (m)
  double* frac = nullptr;    // building cover fraction
  double* hmean = nullptr;   // area-weighted mean building height (m)
  double* dcarea = nullptr;  // operational data-center roof area (m^2)
  double* cd = nullptr;      // block mean drag coefficient
  double cd_tab[256];
};

}  // namespace

struct ahx_static {
  std::mutex mu;
  int dev = 0, nrows = 0, ncols = 0;
  bool destroyed = false;
  int32_t* dem = nullptr;      // cm
  uint8_t* lc = nullptr;
  uint8_t* frac25 = nullptr;
  uint16_t* hmean = nullptr;   // cm
  uint8_t* dca4 = nullptr;
  std::vector<Agg> aggs;       // per spacing (same cd table)
  cudaStream_t s = nullptr;
  // scratch of a build, grown on demand and kept (a build allocates nothing once it has run at a size)
  size_t cap_cells = 0, cap_halls = 0, cap_campus = 0;
  double *d_area = nullptr, *d_heat = nullptr, *d_flux = nullptr, *d_min = nullptr;
  void* d_halls = nullptr;
  uint4* d_colv = nullptr;
  uint32_t* d_ktop = nullptr;
  int* d_kmax = nullptr;
  unsigned long long* d_nb = nullptr;
};

namespace {

ahx_status fail(ahx_status st, const std::string& m) {
  ahx::set_last_error(m);
  return st;
}

#define DCUDA(call)                                                                                 \
  do {                                                                                              \
    const cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) {                                                                        \
      cudaGetLastError();                                                                           \
      return fail(AHX_EDEVICE, std::string("live solver: domain builder: ") + cudaGetErrorString(e_)); \
    }                                                                                               \
  } while (0)

// row-wise prefix sum of the int16 first differences (low byte plane, high byte plane), one thread per row
__global__ void decode_dem_kernel(const uint8_t* lo, const uint8_t* hi, int nrows, int ncols, int32_t* dem) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  int32_t acc = 0;
  for (int c = 0; c < ncols; ++c) {
    const size_t k = (size_t)row * ncols + c;
    const int d = (int)(int16_t)(uint16_t)(lo[k] | (hi[k] << 8));
    acc += d;
    dem[k] = acc;
  }
}

// integer sums of the five planes (the reference's checksums)
__global__ void checksum_kernel(const int32_t* dem, const uint8_t* lc, const uint8_t* frac25, const uint16_t* hmean,
                                const uint8_t* dca4, size_t n, unsigned long long* out) {
  long long s[5] = {0, 0, 0, 0, 0};
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    s[0] += dem[k];
    s[1] += lc[k];
    s[2] += frac25[k];
    s[3] += hmean[k];
    s[4] += dca4[k];
  }
  for (int a = 0; a < 5; ++a) atomicAdd(out + a, (unsigned long long)s[a]);   // two's complement: exact for signed
}

// domain.js:89-118 for one coarse cell
__global__ void aggregate_kernel(const int32_t* dem, const uint8_t* lc, const uint8_t* frac25, const uint16_t* hmean,
                                 const uint8_t* dca4, int ncols, int r, int nx, int ny, const double* cd_tab,
                                 double* o_dem, double* o_frac, double* o_hmean, double* o_dcarea, double* o_cd) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (c >= nx || row >= ny) return;
  long long sd = 0, sc = 0, sh = 0, sa = 0;
  double scd = 0.0;
  for (int a = 0; a < r; ++a)
    for (int b = 0; b < r; ++b) {
      const size_t k = (size_t)(row * r + a) * ncols + (c * r + b);
      sd += dem[k];
      sc += frac25[k];
      sh += (long long)frac25[k] * hmean[k];
      sa += dca4[k];
      scd = scd + cd_tab[lc[k]];
    }
  const size_t o = (size_t)row * nx + c;
  const double rr = (double)(r * r);
  o_dem[o] = (double)sd / (100.0 * rr);
  o_frac[o] = (double)sc / (25.0 * rr);
  o_hmean[o] = sc > 0 ? (double)sh / (double)(sc > 1 ? sc : 1) / 100.0 : 0.0;
  o_dcarea[o] = (double)(4 * sa);
  o_cd[o] = scd / rr;
}

// minimum of a double array and maximum / sums of the build results in one block
__global__ void min_kernel(const double* v, int n, double* out) {
  __shared__ double s[256];
  double m = INFINITY;
  for (int k = threadIdx.x; k < n; k += blockDim.x) m = fmin(m, v[k]);
  s[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] = fmin(s[threadIdx.x], s[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

struct Hall {
  double x0, x1, z0, z1;   // clipped to the box
  int c0, c1, r0, r1;      // cell range
  int campus;
};

// domain.js:124-160 for one coarse cell: the campuses in list order, their halls in list order
__global__ void campus_kernel(const Hall* halls, int nhalls, const double* flux, int ncampus, int nx, int ny,
                              double dx, double* new_area, double* heat_w) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (c >= nx || row >= ny) return;
  const double cellA = dx * dx;
  double area = 0.0, heat = 0.0;
  int h = 0;
  for (int cp = 0; cp < ncampus; ++cp) {
    double per = 0.0;
    bool touched = false;
    for (; h < nhalls && halls[h].campus == cp; ++h) {
      const Hall H = halls[h];
      if (row < H.r0 || row > H.r1 || c < H.c0 || c > H.c1) continue;
      const double oz = fmin(H.z1, kSceneZ0 + (double)(row + 1) * dx) - fmax(H.z0, kSceneZ0 + (double)row * dx);
      if (oz <= 0.0) continue;
      const double ox = fmin(H.x1, kSceneX0 + (double)(c + 1) * dx) - fmax(H.x0, kSceneX0 + (double)c * dx);
      if (ox <= 0.0) continue;
      per = per + ox * oz;
      touched = true;
    }
    if (touched) {
      const double a = fmin(per, cellA);
      area = area + a;
      heat = heat + a * flux[cp];
    }
  }
  const size_t o = (size_t)row * nx + c;
  new_area[o] = fmin(area, cellA);
  heat_w[o] = heat;
}

// domain.js:166-190 per cell (north-up) and solver.js:359-376 column record (solver orientation)
__global__ void build_kernel(const double* dem, const double* frac, const double* hmean, const double* cd,
                             const double* dcarea, const double* new_area, const double* heat_w, int nx, int ny,
                             double dx, double zbase, double extra_h, double flux_existing, double kq, uint4* colv,
                             uint32_t* ktop_s, int* ktop_max, unsigned long long* nb_cells) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (c >= nx || row >= ny) return;
  const size_t o = (size_t)row * nx + c;
  double f = frac[o], hm = hmean[o];
  const double na = new_area[o];
  if (na > 0.0) {
    f = fmax(f, na / (dx * dx));
    hm = fmax(hm, extra_h);
  }
  const double ktd = ceil((dem[o] - zbase) / dx - 0.5);
  const int kt = ktd > 1.0 ? (int)ktd : 1;
  const int nb = f >= 0.5 ? (int)rint(hm / dx) : 0;
  const int kp = kt + nb;
  const double W = dcarea[o] * flux_existing + heat_w[o];
  const float q = (float)(W * kq);
  const float cdf = (float)cd[o];
  const size_t s = (size_t)(ny - 1 - row) * nx + c;   // solver orientation: row 0 north -> j = ny - 1
  colv[s] = make_uint4((uint32_t)kt, (uint32_t)kp, __float_as_uint(cdf), __float_as_uint(q));
  ktop_s[s] = (uint32_t)kp;
  atomicMax(ktop_max, kp);
  if (nb) atomicAdd(nb_cells, (unsigned long long)nb);
}

}  // namespace

extern "C" {

ahx_status ahx_static_create(int device_ordinal, int nrows, int ncols, const uint8_t* raw, size_t raw_bytes,
                             const size_t* offsets, ahx_static** out) {
  if (!raw || !offsets || !out) return fail(AHX_EINVAL, "live solver: null argument");
  *out = nullptr;
  if (nrows < 1 || ncols < 1 || nrows > 65536 || ncols > 65536)
    return fail(AHX_EINVAL, "live solver: bad static plane size");
  const size_t n = (size_t)nrows * ncols;
  // dem: two byte planes; lc, frac25, dca4: one byte; hmean: u16 little-endian
  const size_t need[5] = {2 * n, n, n, 2 * n, n};
  for (int p = 0; p < 5; ++p)
    if (offsets[p] > raw_bytes || need[p] > raw_bytes - offsets[p])
      return fail(AHX_EINVAL, "live solver: static plane outside the raw buffer");
  int dev = device_ordinal;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return fail(AHX_EDEVICE, "live solver: no CUDA device");
  if (cudaSetDevice(dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(AHX_EDEVICE, "live solver: cannot use CUDA device " + std::to_string(dev));
  }
  ahx_static* S = new ahx_static;
  S->dev = dev;
  S->nrows = nrows;
  S->ncols = ncols;
  uint8_t *lo = nullptr, *hi = nullptr;
  auto bail = [&](const char* what) {
    cudaGetLastError();
    cudaFree(lo);
    cudaFree(hi);
    cudaFree(S->dem);
    cudaFree(S->lc);
    cudaFree(S->frac25);
    cudaFree(S->hmean);
    cudaFree(S->dca4);
    if (S->s) cudaStreamDestroy(S->s);
    delete S;
    return fail(AHX_ENOMEM, std::string("live solver: domain builder: ") + what);
  };
  if (cudaStreamCreateWithFlags(&S->s, cudaStreamNonBlocking) != cudaSuccess) return bail("stream");
  if (cudaMalloc(&lo, n) != cudaSuccess || cudaMalloc(&hi, n) != cudaSuccess ||
      cudaMalloc(&S->dem, n * 4) != cudaSuccess || cudaMalloc(&S->lc, n) != cudaSuccess ||
      cudaMalloc(&S->frac25, n) != cudaSuccess || cudaMalloc(&S->hmean, n * 2) != cudaSuccess ||
      cudaMalloc(&S->dca4, n) != cudaSuccess)
    return bail("allocation failed");
  if (cudaMemcpy(lo, raw + offsets[0], n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(hi, raw + offsets[0] + n, n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(S->lc, raw + offsets[1], n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(S->frac25, raw + offsets[2], n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(S->hmean, raw + offsets[3], n * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(S->dca4, raw + offsets[4], n, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail("upload failed");
  decode_dem_kernel<<<(nrows + 127) / 128, 128, 0, S->s>>>(lo, hi, nrows, ncols, S->dem);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(S->s) != cudaSuccess) return bail("dem decode");
  cudaFree(lo);
  cudaFree(hi);
  *out = S;
  return AHX_OK;
}

ahx_status ahx_static_checksums(ahx_static* S, int64_t* sums) {
  if (!S || !sums) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->destroyed) return fail(AHX_EDESTROYED, "live solver: static planes destroyed");
  DCUDA(cudaSetDevice(S->dev));
  unsigned long long* d = nullptr;
  DCUDA(cudaMalloc(&d, 5 * sizeof(unsigned long long)));
  cudaMemsetAsync(d, 0, 5 * sizeof(unsigned long long), S->s);
  checksum_kernel<<<148, 256, 0, S->s>>>(S->dem, S->lc, S->frac25, S->hmean, S->dca4, (size_t)S->nrows * S->ncols,
                                         d);
  unsigned long long h[5];
  const cudaError_t e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, S->s);
  const cudaError_t e2 = cudaStreamSynchronize(S->s);
  cudaFree(d);
  DCUDA(e);
  DCUDA(e2);
  for (int a = 0; a < 5; ++a) sums[a] = (int64_t)h[a];
  return AHX_OK;
}

ahx_status ahx_domain_build(ahx_static* S, const ahx_domain_spec* sp, ahx_domain_out* out, uint32_t* colv,
                            uint32_t* ktop, double* heat_w, double* new_area) {
  if (!S || !sp || !out) return fail(AHX_EINVAL, "live solver: null argument");
  if (!sp->cd_table) return fail(AHX_EINVAL, "live solver: drag-coefficient table missing");
  const int r = (int)std::lround(sp->dx / 10.0);
  if (r < 1 || std::fabs(r * 10.0 - sp->dx) > 1e-9 || S->ncols % r || S->nrows % r)
    return fail(AHX_EINVAL, "live solver: dx must be a multiple of 10 m dividing the box");
  if (sp->ncampus < 0 || (sp->ncampus > 0 && (!sp->campus_mw || !sp->campus_flux || !sp->hall_count || !sp->halls)))
    return fail(AHX_EINVAL, "live solver: bad campus list");
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->destroyed) return fail(AHX_EDESTROYED, "live solver: static planes destroyed");
  DCUDA(cudaSetDevice(S->dev));
  const int nx = S->ncols / r, ny = S->nrows / r;
  const size_t NXY = (size_t)nx * ny;
  // the aggregate of this spacing (and drag table), made once
  Agg* A = nullptr;
  for (Agg& g : S->aggs)
    if (g.r == r && g.dx == sp->dx && std::memcmp(g.cd_tab, sp->cd_table, sizeof(g.cd_tab)) == 0) A = &g;
  if (!A) {
    Agg g;
    g.r = r;
    g.nx = nx;
    g.ny = ny;
    g.dx = sp->dx;
    std::memcpy(g.cd_tab, sp->cd_table, sizeof(g.cd_tab));
    double* tab = nullptr;
    if (cudaMalloc(&g.dem, NXY * 8) != cudaSuccess || cudaMalloc(&g.frac, NXY * 8) != cudaSuccess ||
        cudaMalloc(&g.hmean, NXY * 8) != cudaSuccess || cudaMalloc(&g.dcarea, NXY * 8) != cudaSuccess ||
        cudaMalloc(&g.cd, NXY * 8) != cudaSuccess || cudaMalloc(&tab, 256 * 8) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(g.dem);
      cudaFree(g.frac);
      cudaFree(g.hmean);
      cudaFree(g.dcarea);
      cudaFree(g.cd);
      cudaFree(tab);
      return fail(AHX_ENOMEM, "live solver: domain builder: aggregate allocation failed");
    }
    cudaMemcpyAsync(tab, g.cd_tab, 256 * 8, cudaMemcpyHostToDevice, S->s);
    const dim3 b(32, 8), gr((nx + 31) / 32, (ny + 7) / 8);
    aggregate_kernel<<<gr, b, 0, S->s>>>(S->dem, S->lc, S->frac25, S->hmean, S->dca4, S->ncols, r, nx, ny, tab,
                                         g.dem, g.frac, g.hmean, g.dcarea, g.cd);
    const cudaError_t e = cudaGetLastError();
    const cudaError_t e2 = cudaStreamSynchronize(S->s);
    cudaFree(tab);
    DCUDA(e);
    DCUDA(e2);
    S->aggs.push_back(g);
    A = &S->aggs.back();
  }
  // halls clipped to the box with their cell ranges (domain.js:131-144), campus heat flux per unit hall area
  std::vector<Hall> halls;
  std::vector<double> flux((size_t)std::max(sp->ncampus, 1), 0.0);
  const double X1 = kSceneX0 + nx * sp->dx, Z1 = kSceneZ0 + ny * sp->dx;
  int hi = 0;
  for (int cp = 0; cp < sp->ncampus; ++cp) {
    double total = 0.0;
    for (int t = 0; t < sp->hall_count[cp]; ++t, ++hi) {
      const double* h = sp->halls + 4 * (size_t)hi;
      const double xa = std::fmin(h[0], h[2]), xb = std::fmax(h[0], h[2]);
      const double za = std::fmin(h[1], h[3]), zb = std::fmax(h[1], h[3]);
      if (!(xb > xa && zb > za)) continue;
      total += (xb - xa) * (zb - za);
      Hall H;
      H.x0 = std::fmax(xa, kSceneX0);
      H.x1 = std::fmin(xb, X1);
      H.z0 = std::fmax(za, kSceneZ0);
      H.z1 = std::fmin(zb, Z1);
      if (H.x1 <= H.x0 || H.z1 <= H.z0) continue;
      H.c0 = std::max(0, (int)std::floor((H.x0 - kSceneX0) / sp->dx));
      H.c1 = std::min(nx - 1, (int)std::floor((H.x1 - kSceneX0) / sp->dx));
      H.r0 = std::max(0, (int)std::floor((H.z0 - kSceneZ0) / sp->dx));
      H.r1 = std::min(ny - 1, (int)std::floor((H.z1 - kSceneZ0) / sp->dx));
      H.campus = cp;
      halls.push_back(H);
    }
    const double mw = std::fmax(0.0, sp->campus_mw[cp]);
    flux[cp] = total > 0 ? mw * 1e6 / total : 0.0;
    sp->campus_flux[cp] = flux[cp];
  }
  // device scratch of a build: raster, packed outputs, reductions (kept on the static object)
  if (S->cap_cells < NXY || S->cap_halls < std::max<size_t>(1, halls.size()) || S->cap_campus < flux.size() ||
      !S->d_min) {
    cudaFree(S->d_area);
    cudaFree(S->d_heat);
    cudaFree(S->d_flux);
    cudaFree(S->d_min);
    cudaFree(S->d_halls);
    cudaFree(S->d_colv);
    cudaFree(S->d_ktop);
    cudaFree(S->d_kmax);
    cudaFree(S->d_nb);
    S->d_area = S->d_heat = S->d_flux = S->d_min = nullptr;
    S->d_halls = nullptr;
    S->d_colv = nullptr;
    S->d_ktop = nullptr;
    S->d_kmax = nullptr;
    S->d_nb = nullptr;
    S->cap_cells = std::max(S->cap_cells, NXY);
    S->cap_halls = std::max(S->cap_halls, std::max<size_t>(16, halls.size()));
    S->cap_campus = std::max(S->cap_campus, std::max<size_t>(16, flux.size()));
    if (cudaMalloc(&S->d_area, S->cap_cells * 8) != cudaSuccess || cudaMalloc(&S->d_heat, S->cap_cells * 8) != cudaSuccess ||
        cudaMalloc(&S->d_flux, S->cap_campus * 8) != cudaSuccess || cudaMalloc(&S->d_min, 8) != cudaSuccess ||
        cudaMalloc(&S->d_halls, S->cap_halls * sizeof(Hall)) != cudaSuccess ||
        cudaMalloc(&S->d_colv, S->cap_cells * 16) != cudaSuccess || cudaMalloc(&S->d_ktop, S->cap_cells * 4) != cudaSuccess ||
        cudaMalloc(&S->d_kmax, 4) != cudaSuccess || cudaMalloc(&S->d_nb, 8) != cudaSuccess) {
      cudaGetLastError();
      S->cap_cells = S->cap_halls = S->cap_campus = 0;
      return fail(AHX_ENOMEM, "live solver: domain builder: allocation failed");
    }
  }
  double *d_area = S->d_area, *d_heat = S->d_heat, *d_flux = S->d_flux, *d_min = S->d_min;
  Hall* d_halls = static_cast<Hall*>(S->d_halls);
  uint4* d_colv = S->d_colv;
  uint32_t* d_ktop = S->d_ktop;
  int* d_kmax = S->d_kmax;
  unsigned long long* d_nb = S->d_nb;
  ahx_status st = AHX_OK;
  const dim3 b(32, 8), gr((nx + 31) / 32, (ny + 7) / 8);
  double mn = 0;
  int kmax = 0;
  unsigned long long nbc = 0;
  cudaError_t e = cudaSuccess;
  do {
    if ((e = cudaMemcpyAsync(d_flux, flux.data(), flux.size() * 8, cudaMemcpyHostToDevice, S->s)) != cudaSuccess) break;
    if (!halls.empty() && (e = cudaMemcpyAsync(d_halls, halls.data(), halls.size() * sizeof(Hall),
                                               cudaMemcpyHostToDevice, S->s)) != cudaSuccess)
      break;
    campus_kernel<<<gr, b, 0, S->s>>>(d_halls, (int)halls.size(), d_flux, sp->ncampus, nx, ny, sp->dx, d_area, d_heat);
    min_kernel<<<1, 256, 0, S->s>>>(A->dem, (int)NXY, d_min);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    if ((e = cudaMemcpyAsync(&mn, d_min, 8, cudaMemcpyDeviceToHost, S->s)) != cudaSuccess) break;
    if ((e = cudaStreamSynchronize(S->s)) != cudaSuccess) break;
    const double zbase = std::floor(mn) - sp->dx;   // domain.js:169
    cudaMemsetAsync(d_kmax, 0, 4, S->s);
    cudaMemsetAsync(d_nb, 0, 8, S->s);
    build_kernel<<<gr, b, 0, S->s>>>(A->dem, A->frac, A->hmean, A->cd, A->dcarea, d_area, d_heat, nx, ny, sp->dx,
                                     zbase, sp->extra_height, sp->flux_existing, sp->kq, d_colv, d_ktop, d_kmax, d_nb);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    if ((e = cudaMemcpyAsync(&kmax, d_kmax, 4, cudaMemcpyDeviceToHost, S->s)) != cudaSuccess) break;
    if ((e = cudaMemcpyAsync(&nbc, d_nb, 8, cudaMemcpyDeviceToHost, S->s)) != cudaSuccess) break;
    if (colv && (e = cudaMemcpyAsync(colv, d_colv, NXY * 16, cudaMemcpyDeviceToHost, S->s)) != cudaSuccess) break;
    if (ktop && (e = cudaMemcpyAsync(ktop, d_ktop, NXY * 4, cudaMemcpyDeviceToHost, S->s)) != cudaSuccess) break;
    if (heat_w && (e = cudaMemcpyAsync(heat_w, d_heat, NXY * 8, cudaMemcpyDeviceToHost, S->s)) != cudaSuccess) break;
    if (new_area && (e = cudaMemcpyAsync(new_area, d_area, NXY * 8, cudaMemcpyDeviceToHost, S->s)) != cudaSuccess)
      break;
    if ((e = cudaStreamSynchronize(S->s)) != cudaSuccess) break;
    std::memset(out, 0, sizeof(*out));
    out->nx = nx;
    out->ny = ny;
    int nz = std::max((int)std::floor(sp->heightM / sp->dx + 0.5), sp->nz_min);   // Math.round, domain.js:181
    if (kmax >= nz - 8) nz = kmax + 9;
    out->nz = nz;
    out->ktop_max = kmax;
    out->zbase = zbase;
    out->nb_cells = (int64_t)nbc;
  } while (false);
  if (e != cudaSuccess) {
    cudaGetLastError();
    st = fail(AHX_EDEVICE, std::string("live solver: domain builder: ") + cudaGetErrorString(e));
  }
  return st;
}

ahx_status ahx_static_destroy(ahx_static* S) {
  if (!S) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->destroyed) return AHX_OK;
  cudaSetDevice(S->dev);
  cudaStreamSynchronize(S->s);
  for (Agg& g : S->aggs) {
    cudaFree(g.dem);
    cudaFree(g.frac);
    cudaFree(g.hmean);
    cudaFree(g.dcarea);
    cudaFree(g.cd);
  }
  S->aggs.clear();
  cudaFree(S->d_area);
  cudaFree(S->d_heat);
  cudaFree(S->d_flux);
  cudaFree(S->d_min);
  cudaFree(S->d_halls);
  cudaFree(S->d_colv);
  cudaFree(S->d_ktop);
  cudaFree(S->d_kmax);
  cudaFree(S->d_nb);
  cudaFree(S->dem);
  cudaFree(S->lc);
  cudaFree(S->frac25);
  cudaFree(S->hmean);
  cudaFree(S->dca4);
  cudaStreamDestroy(S->s);
  cudaGetLastError();
  S->destroyed = true;   // the object stays, so later calls report "destroyed"
  return AHX_OK;
}

}  // extern "C"
