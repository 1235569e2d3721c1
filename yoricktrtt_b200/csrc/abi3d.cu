// abi3d.cu -- C ABI of the 3D projectors: the drop-in trtt_PB3D/CB3D(_cubic)
// symbols, the batched host-buffer entry point and the native plan API.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <new>
#include <string>
#include <algorithm>
#include <utility>
#include <vector>

#include "host3d.h"
#include "kernels.h"
#include "runtime.h"
#include "trtt_b200.h"

using namespace trtt;


// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
struct trtt_b200_plan3d {
  Params3D P;
  int device = 0;
  long nviews = 0;
  int nt = 1;
  int band_rows = 0, warps = 16;
  int pull = 0;  // 1: atomic-free band kernel (closed-form model, nu <= 512)
  int tc = 0;    // 1: tensor-core band kernel (closed-form model)
  int cols = 1;  // 2: column-pair band kernel (closed-form model)
  bool factorized = true;
  DevBuf views, cum, gate_ptr, entries, pairs, scratch, err;
  std::vector<View3D> hviews;
  // view groups related by turns of the grid (closed-form model, factorised
  // views): index 0 singles, 1 pairs (half turns), 2 quads (quarter turns)
  int sym = 2;            // group kernels when they apply: 2 (interleaved member profiles), 1; 0 never
  bool grouped = false;   // groups were found (some group has 2 or 4 views)
  int ngroups[3] = {0, 0, 0};
  DevBuf groups[3];
  int gband[3] = {64, 32, 32};  // direct: band rows per group size
  int gutile4 = 0, gminb4 = 1;  // direct, quads: cells per u tile (0: up to 256), CTAs per SM
  long back_chunk_bytes = 32L << 20;  // transpose: detector bytes per launch
  // persistent weighted least-squares launch
  int wls_rows = 32, wls_ctas = 1, wls_extra = 0;
  long long wls_wait_ns = 2000000000LL;
  DevBuf resid, wls_parts, wls_queue;
};

static int group_size_of(int idx) { return idx == 2 ? 4 : idx + 1; }

// Group kernels apply: closed-form model, every view factorised, one gate,
// the whole scan in one call.
static bool use_groups(const trtt_b200_plan3d *pl, long view0, long nview)
{
  return pl->sym && pl->grouped && pl->factorized && pl->P.model == MODEL_CUBIC && pl->nt == 1 &&
         !pl->pull && !pl->tc && pl->cols == 1 && view0 == 0 && nview == pl->nviews &&
         pl->nviews <= 65535;
}

static int upload_gates(trtt_b200_plan3d *pl, const std::vector<std::vector<GateEntry>> &lists)
{
  std::vector<int> ptr(lists.size() + 1, 0);
  std::vector<GateEntry> ent;
  for (size_t g = 0; g < lists.size(); ++g) {
    ptr[g] = (int)ent.size();
    ent.insert(ent.end(), lists[g].begin(), lists[g].end());
  }
  ptr[lists.size()] = (int)ent.size();
  TRTT_CK(pl->gate_ptr.ensure(sizeof(int) * ptr.size()));
  TRTT_CK(pl->entries.ensure(sizeof(GateEntry) * (ent.empty() ? 1 : ent.size())));
  TRTT_CK(cudaMemcpy(pl->gate_ptr.p, ptr.data(), sizeof(int) * ptr.size(), cudaMemcpyHostToDevice));
  if (!ent.empty())
    TRTT_CK(cudaMemcpy(pl->entries.p, ent.data(), sizeof(GateEntry) * ent.size(), cudaMemcpyHostToDevice));
  // the same weights by view, for the transpose that walks each view once
  std::vector<GatePair> pairs(std::max<long>(1, pl->nviews), GatePair{-1, -1, 0.f, 0.f});
  for (size_t g = 0; g < lists.size(); ++g)
    for (const GateEntry &e : lists[g]) {
      GatePair &q = pairs[e.view];
      if (q.g0 < 0) {
        q.g0 = (int)g;
        q.w0 = e.w;
      } else {
        q.g1 = (int)g;
        q.w1 = e.w;
      }
    }
  TRTT_CK(pl->pairs.ensure(sizeof(GatePair) * pairs.size()));
  TRTT_CK(cudaMemcpy(pl->pairs.p, pairs.data(), sizeof(GatePair) * pairs.size(), cudaMemcpyHostToDevice));
  return 0;
}

extern "C" int trtt_b200_plan3d_create(trtt_b200_plan3d **plan, int geometry,
                                       long nx, long ny, long nz, double s_scl,
                                       int s_deg, const double *cum_footprint,
                                       long size_footprint, double step_footprint,
                                       const double *coord_footprint, long nu,
                                       long nv, double u_scl, double v_scl,
                                       long nviews, const double *xos,
                                       const double *xsd)
{
  clear_error();
  if (!plan) return fail("plan3d_create: null plan pointer");
  *plan = nullptr;
  const int g = geom_code(geometry);
  if (g < 0) return fail("plan3d_create: geometry must be 3 (parallel), 4 (cone) or 5 (fan)");
  if (const char *why = check_sizes3d(nx, ny, nz, nu, nv, nviews))
    return fail(std::string("plan3d_create: ") + why);
  if (!xos || !xsd) return fail("plan3d_create: null xos/xsd");
  if (cum_footprint && (size_footprint < 1 || !coord_footprint || !(step_footprint > 0)))
    return fail("plan3d_create: invalid footprint table");
  trtt_b200_plan3d *pl = new (std::nothrow) trtt_b200_plan3d();
  if (!pl) return fail("plan3d_create: out of host memory");
  cudaGetDevice(&pl->device);
  if (cum_footprint) {
    cudaError_t e = pl->cum.ensure(sizeof(double) * size_footprint);
    if (e == cudaSuccess)
      e = cudaMemcpy(pl->cum.p, cum_footprint, sizeof(double) * size_footprint, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      delete pl;
      return fail_cuda(e, "plan3d_create(footprint)");
    }
  }
  pl->P = make_params(g, nx, ny, nz, s_scl, s_deg, cum_footprint ? pl->cum.as<double>() : nullptr,
                      size_footprint, step_footprint, cum_footprint ? coord_footprint[0] : 0.0,
                      nu, nv, u_scl, v_scl);
  pl->nviews = nviews;
  pl->hviews.resize(nviews);
  for (long v = 0; v < nviews; ++v) {
    make_view3d(pl->P, xos + 12 * v, xsd + 12 * v, pl->hviews[v]);
    if (!pl->hviews[v].factorized) pl->factorized = false;
  }
  choose_band(pl->P.nu, pl->P.nv, pl->band_rows, pl->warps);
  if (pl->factorized && !cum_footprint) {
    std::vector<int> lists[3];
    find_view_groups(nx, ny, nviews, xos, xsd, lists);
    pl->grouped = !lists[1].empty() || !lists[2].empty();
    for (int q = 0; q < 3 && pl->grouped; ++q) {
      pl->ngroups[q] = (int)(lists[q].size() / 4);
      if (lists[q].empty()) continue;
      cudaError_t eg = pl->groups[q].ensure(sizeof(int) * lists[q].size());
      if (eg == cudaSuccess)
        eg = cudaMemcpy(pl->groups[q].p, lists[q].data(), sizeof(int) * lists[q].size(),
                        cudaMemcpyHostToDevice);
      if (eg != cudaSuccess) {
        delete pl;
        return fail_cuda(eg, "plan3d_create(groups)");
      }
    }
  }
  cudaError_t e = pl->views.ensure(sizeof(View3D) * nviews);
  if (e == cudaSuccess)
    e = cudaMemcpy(pl->views.p, pl->hviews.data(), sizeof(View3D) * nviews, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = pl->err.ensure(sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(pl->err.p, 0, sizeof(int));
  if (e != cudaSuccess) {
    delete pl;
    return fail_cuda(e, "plan3d_create(upload)");
  }
  std::vector<std::vector<GateEntry>> lists(1);
  for (long v = 0; v < nviews; ++v) lists[0].push_back(GateEntry{(int)v, 1.0f});
  if (upload_gates(pl, lists)) {
    delete pl;
    return -1;
  }
  *plan = pl;
  return 0;
}

extern "C" int trtt_b200_plan3d_set_gates(trtt_b200_plan3d *pl, long nt, const double *t_index)
{
  clear_error();
  if (!pl || !t_index) return fail("plan3d_set_gates: null argument");
  if (nt < 1 || nt > 65535) return fail("plan3d_set_gates: nt must be in [1, 65535]");
  std::vector<std::vector<GateEntry>> lists(nt);
  for (long v = 0; v < pl->nviews; ++v) {
    const double t = t_index[v];
    if (!(t >= 0.0 && t <= (double)nt))
      return fail("plan3d_set_gates: t_index must lie in [0, nt] (Ytrtt_3D_projectors.i:289-292)");
    const double f = std::floor(t), c = std::ceil(t);
    const double pe = t - f;
    const int g0 = (int)((long)f % nt), g1 = (int)((long)c % nt);
    View3D &V = pl->hviews[v];
    V.g0 = g0;
    V.g1 = g1;
    V.w0 = (float)(1.0 - pe);
    V.w1 = (float)pe;
    if (g0 != g1) {
      lists[g0].push_back(GateEntry{(int)v, (float)(1.0 - pe)});
      lists[g1].push_back(GateEntry{(int)v, (float)pe});
    } else {
      // both interpolation indices equal: Yorick's repeated-index
      // assignment keeps the second (weight pe) write
      lists[g0].push_back(GateEntry{(int)v, (float)pe});
      V.w0 = (float)((1.0 - pe) + pe);
      V.w1 = 0.0f;
    }
  }
  TRTT_CK(cudaMemcpy(pl->views.p, pl->hviews.data(), sizeof(View3D) * pl->nviews, cudaMemcpyHostToDevice));
  pl->nt = (int)nt;
  pl->P.nt = (int)nt;
  return upload_gates(pl, lists);
}

extern "C" int trtt_b200_plan3d_set_tiles(trtt_b200_plan3d *pl, int band_rows, int warps)
{
  clear_error();
  if (!pl) return fail("plan3d_set_tiles: null plan");
  if (band_rows == 0 && warps == 0) {  // defaults
    pl->pull = 0;
    pl->tc = 0;
    choose_band(pl->P.nu, pl->P.nv, pl->band_rows, pl->warps);
    return 0;
  }
  if (band_rows == TRTT_B200_TILES_PULL) {  // atomic-free band kernel
    pl->pull = 1;
    pl->tc = 0;
    return 0;
  }
  if (band_rows == TRTT_B200_TILES_TENSOR) {  // tensor-core band kernel
    if (fwd3d_tc_band_rows((int)pl->P.nu, (int)pl->P.nv) <= 0)
      return fail("plan3d_set_tiles: detector too wide for the tensor-core band kernel");
    pl->pull = 0;
    pl->tc = 1;
    if (pl->band_rows <= 0) choose_band(pl->P.nu, pl->P.nv, pl->band_rows, pl->warps);
    return 0;
  }
  pl->pull = 0;
  pl->tc = 0;
  if (warps > 0) {
    if (warps < 2 || warps > 16) return fail("plan3d_set_tiles: warps must be in [2, 16]");
    pl->warps = warps;
  }
  if (band_rows < 0) {
    pl->band_rows = 0;
  } else if (band_rows > 0) {
    const long smem = (long)band_fast_smem(pl->P.nu, band_rows, pl->warps);
    if (smem > 227L * 1024) return fail("plan3d_set_tiles: band does not fit in shared memory");
    pl->band_rows = band_rows > pl->P.nv ? pl->P.nv : band_rows;
  }
  return 0;
}

extern "C" int trtt_b200_plan3d_set_columns(trtt_b200_plan3d *pl, int cols)
{
  clear_error();
  if (!pl) return fail("plan3d_set_columns: null plan");
  if (cols != 1 && cols != 2) return fail("plan3d_set_columns: cols must be 1 or 2");
  if (cols == 2 && pl->band_rows > 0) {
    const long smem = 4L * ((long)pl->band_rows * pl->P.nu + 2L * pl->warps * pl->P.nu + 2L * pl->warps * pl->band_rows);
    if (smem > 227L * 1024) return fail("plan3d_set_columns: band does not fit in shared memory");
  }
  pl->cols = cols;
  return 0;
}

extern "C" int trtt_b200_plan3d_set_symmetry(trtt_b200_plan3d *pl, int on)
{
  clear_error();
  if (!pl) return fail("plan3d_set_symmetry: null plan");
  if (on < 0 || on > 2) return fail("plan3d_set_symmetry: mode must be 0, 1 or 2");
  pl->sym = on;
  return 0;
}

extern "C" int trtt_b200_plan3d_groups(const trtt_b200_plan3d *pl, long *counts)
{
  clear_error();
  if (!pl || !counts) return fail("plan3d_groups: null argument");
  for (int q = 0; q < 3; ++q) counts[q] = pl->grouped ? pl->ngroups[q] : 0;
  if (!pl->grouped) counts[0] = pl->factorized && pl->P.model == MODEL_CUBIC ? pl->nviews : 0;
  return 0;
}

extern "C" int trtt_b200_plan3d_set_group_tiles(trtt_b200_plan3d *pl, int band_rows4, int band_rows2,
                                                int band_rows1, long back_chunk_bytes)
{
  clear_error();
  if (!pl) return fail("plan3d_set_group_tiles: null plan");
  const int req[3] = {band_rows1, band_rows2, band_rows4};
  const int usplit = (pl->P.nu + 255) / 256;
  const int utile = (pl->P.nu + usplit - 1) / usplit;
  for (int q = 0; q < 3; ++q) {
    if (req[q] == 0) continue;
    if (req[q] < 2) return fail("plan3d_set_group_tiles: band rows must be >= 2");
    const int r = std::min(req[q], pl->P.nv);
    const int G = group_size_of(q), minb = G == 4 ? pl->gminb4 : 2;
    if (group_fwd_smem(G, r, utile, group_fwd_warps(G, r, utile, minb)) > 227u * 1024u)
      return fail("plan3d_set_group_tiles: band does not fit in shared memory");
  }
  for (int q = 0; q < 3; ++q)
    if (req[q]) pl->gband[q] = req[q];
  if (back_chunk_bytes < 0) return fail("plan3d_set_group_tiles: negative chunk size");
  if (back_chunk_bytes) pl->back_chunk_bytes = back_chunk_bytes;
  return 0;
}

extern "C" int trtt_b200_plan3d_set_persistent(trtt_b200_plan3d *pl, int band_rows, int ctas_per_sm,
                                               double wait_seconds, int extra_wait)
{
  clear_error();
  if (!pl) return fail("plan3d_set_persistent: null plan");
  if (band_rows < 0 || (band_rows > 0 && band_rows < 2))
    return fail("plan3d_set_persistent: band rows must be 0 (keep) or >= 2");
  if (ctas_per_sm < 0 || ctas_per_sm > 2) return fail("plan3d_set_persistent: CTAs per SM must be 0, 1 or 2");
  if (!(wait_seconds >= 0.0) || wait_seconds > 60.0)
    return fail("plan3d_set_persistent: wait limit must be in [0, 60] s (0 keeps)");
  if (extra_wait < 0) return fail("plan3d_set_persistent: negative extra wait");
  if (band_rows) {
    const int r = std::min(band_rows, pl->P.nv);
    if (wls_smem(pl->P.nu, r) > 227u * 1024u) return fail("plan3d_set_persistent: band does not fit in shared memory");
    pl->wls_rows = band_rows;
  }
  if (ctas_per_sm) pl->wls_ctas = ctas_per_sm;
  if (wait_seconds > 0.0) pl->wls_wait_ns = (long long)(wait_seconds * 1e9);
  pl->wls_extra = extra_wait;
  return 0;
}

extern "C" int trtt_b200_plan3d_wls_grad(trtt_b200_plan3d *pl, const float *vol, const float *y,
                                         const float *w, float *grad, double *cost, void *stream)
{
  clear_error();
  if (!pl || !vol || !y || !grad || !cost) return fail("plan3d_wls_grad: null argument");
  if (!pl->factorized || pl->P.model != MODEL_CUBIC)
    return fail("plan3d_wls_grad: needs the closed-form model and column-factorised views");
  cudaStream_t st = (cudaStream_t)stream;
  const Params3D &P = pl->P;
  int dev = 0, sms = 0, coop = 0;
  TRTT_CK(cudaGetDevice(&dev));
  TRTT_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  TRTT_CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop) return fail("plan3d_wls_grad: the device has no cooperative launch");
  WlsLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.P = P;
  L.views = pl->views.as<View3D>();
  L.nviews = (int)pl->nviews;
  L.gate_ptr = pl->gate_ptr.as<int>();
  L.entries = pl->entries.as<GateEntry>();
  L.ngates = pl->nt;
  L.pairs = pl->nt > 1 ? pl->pairs.as<GatePair>() : nullptr;
  L.vol = vol;
  L.gate_stride = (long)P.nx * P.ny * P.nz;
  L.y = y;
  L.w = w;
  L.grad = grad;
  L.cost = cost;
  L.band_rows = std::min(pl->wls_rows, P.nv);
  L.ctas_per_sm = pl->wls_ctas;
  L.extra_wait = pl->wls_extra;
  L.wait_ns = pl->wls_wait_ns;
  L.err = pl->err.as<int>();
  const long nbands = (P.nv + L.band_rows - 1) / L.band_rows;
  TRTT_CK(pl->resid.ensure(sizeof(float) * (size_t)pl->nviews * P.nu * P.nv));
  TRTT_CK(pl->wls_parts.ensure(sizeof(double) * (size_t)(pl->nviews * nbands)));
  TRTT_CK(pl->wls_queue.ensure(sizeof(unsigned) * 2));
  TRTT_CK(cudaMemsetAsync(pl->wls_queue.p, 0, sizeof(unsigned) * 2, st));
  L.resid = pl->resid.as<float>();
  L.cost_parts = pl->wls_parts.as<double>();
  L.queue = pl->wls_queue.as<unsigned>();
  TRTT_CK(launch_wls_persistent(L, sms, st));
  count_launch();
  return 0;
}

extern "C" int trtt_b200_plan3d_set_group_shape(trtt_b200_plan3d *pl, int band_rows4, int utile4,
                                                int ctas_per_sm4)
{
  clear_error();
  if (!pl) return fail("plan3d_set_group_shape: null plan");
  if (band_rows4 < 0 || band_rows4 == 1) return fail("plan3d_set_group_shape: band rows must be 0 (keep) or >= 2");
  if (utile4 < 0 || utile4 > 256 || (utile4 > 0 && utile4 < 32))
    return fail("plan3d_set_group_shape: u tile must be 0 (automatic) or in [32, 256]");
  if (ctas_per_sm4 < 0 || ctas_per_sm4 > 2) return fail("plan3d_set_group_shape: CTAs per SM must be 0, 1 or 2");
  const int rows = std::min(band_rows4 ? band_rows4 : pl->gband[2], pl->P.nv);
  const int umax = utile4 > 0 ? utile4 : 256;
  const int usplit = (pl->P.nu + umax - 1) / umax, ut = (pl->P.nu + usplit - 1) / usplit;
  const int cpsm = ctas_per_sm4 ? ctas_per_sm4 : pl->gminb4;
  const size_t smem = group_fwd_smem(4, rows, ut, group_fwd_warps(4, rows, ut, cpsm));
  if (smem > (cpsm == 2 ? 113u : 227u) * 1024u)
    return fail("plan3d_set_group_shape: the quad band does not fit in shared memory at that occupancy");
  if (band_rows4) pl->gband[2] = band_rows4;
  pl->gutile4 = utile4;
  if (ctas_per_sm4) pl->gminb4 = ctas_per_sm4;
  return 0;
}

extern "C" int trtt_b200_plan3d_factorized(const trtt_b200_plan3d *pl)
{
  return pl && pl->factorized ? 1 : 0;
}

extern "C" int trtt_b200_plan3d_shape(const trtt_b200_plan3d *pl, long *shape)
{
  clear_error();
  if (!pl || !shape) return fail("plan3d_shape: null argument");
  shape[0] = pl->P.nx;
  shape[1] = pl->P.ny;
  shape[2] = pl->P.nz;
  shape[3] = pl->P.nu;
  shape[4] = pl->P.nv;
  shape[5] = pl->nviews;
  shape[6] = pl->nt;
  return 0;
}

static int plan_run(trtt_b200_plan3d *pl, const float *src, float *dst, long view0,
                    long nview, int layout, void *stream, bool forward)
{
  clear_error();
  if (!pl || !src || !dst) return fail("plan3d: null argument");
  if (view0 < 0 || nview < 0 || view0 + nview > pl->nviews) return fail("plan3d: view range out of bounds");
  if (layout != TRTT_B200_LAYOUT_XYZ && layout != TRTT_B200_LAYOUT_COLUMNS)
    return fail("plan3d: unknown volume layout");
  if (nview == 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  const Params3D &P = pl->P;
  const long nvox = (long)P.nx * P.ny * P.nz;
  const long npix = (long)P.nu * P.nv;
  const float *volc = forward ? src : nullptr;
  float *volo = forward ? nullptr : dst;
  if (layout == TRTT_B200_LAYOUT_XYZ) {
    TRTT_CK(pl->scratch.ensure(sizeof(float) * nvox * pl->nt));
    if (forward) {
      TRTT_CK(xyz_f32_to_col_f32(src, pl->scratch.as<float>(), P.nx, P.ny, P.nz, pl->nt, st));
      count_launch();
      volc = pl->scratch.as<float>();
    } else {
      TRTT_CK(cudaMemsetAsync(pl->scratch.p, 0, sizeof(float) * nvox * pl->nt, st));
      volo = pl->scratch.as<float>();
    }
  }
  if (forward && use_groups(pl, view0, nview)) {
    for (int q = 2; q >= 0; --q) {
      if (!pl->ngroups[q]) continue;
      const int G = group_size_of(q);
      GroupFwdLaunch L;
      L.P = P;
      L.views = pl->views.as<View3D>();
      L.groups = pl->groups[q].as<int>();
      L.ngroups = pl->ngroups[q];
      L.vol = volc;
      L.sino = dst;
      L.sino_view_stride = npix;
      L.band_rows = std::min(pl->gband[q], P.nv);
      const int umax = (G == 4 && pl->gutile4 > 0) ? pl->gutile4 : 256;
      L.usplit = (P.nu + umax - 1) / umax;
      L.utile = (P.nu + L.usplit - 1) / L.usplit;
      L.interleave = pl->sym == 2 ? 1 : 0;
      L.minb = G == 4 ? pl->gminb4 : 2;
      L.warps = group_fwd_warps(G, L.band_rows, L.utile, L.minb);
      L.err = pl->err.as<int>();
      TRTT_CK(launch_fwd3d_group(L, G, st));
      count_launch();
    }
  } else if (!forward && use_groups(pl, view0, nview)) {
    for (int q = 2; q >= 0; --q) {
      if (!pl->ngroups[q]) continue;
      const int G = group_size_of(q);
      GroupBackLaunch L;
      L.P = P;
      L.views = pl->views.as<View3D>();
      L.groups = pl->groups[q].as<int>();
      L.norbits = group_orbits(G, P.nx, P.ny);
      L.sino = src;
      L.sino_view_stride = npix;
      L.vol = volo;
      L.vec4 = (P.nu % 4 == 0 && ((uintptr_t)src & 15) == 0) ? 1 : 0;
      L.err = pl->err.as<int>();
      // groups per launch: the launch's detector images stay in L2 while
      // every orbit walks them
      const long per_group = (long)G * npix * (long)sizeof(float);
      const int chunk = (int)std::max<long>(1, pl->back_chunk_bytes / per_group);
      for (int g0 = 0; g0 < pl->ngroups[q]; g0 += chunk) {
        L.g_lo = g0;
        L.g_hi = std::min(g0 + chunk, pl->ngroups[q]);
        TRTT_CK(launch_back3d_group(L, G, st));
        count_launch();
      }
    }
    if (layout == TRTT_B200_LAYOUT_XYZ) {
      TRTT_CK(col_f32_add_to_xyz_f32(volo, dst, P.nx, P.ny, P.nz, pl->nt, st));
      count_launch();
    }
  } else if (forward) {
    Fwd3DLaunch L;
    L.P = P;
    L.views = pl->views.as<View3D>() + view0;
    L.nviews = (int)nview;
    L.vol = volc;
    L.gate_stride = nvox;
    L.sino = dst;
    L.sino_view_stride = npix;
    L.band_rows = pl->factorized ? pl->band_rows : 0;
    L.warps = pl->warps;
    L.pull = pl->pull;
    L.tc = pl->tc;
    L.cols = pl->cols;
    L.err = pl->err.as<int>();
    TRTT_CK(launch_fwd3d(L, st));
    count_launch();
  } else {
    Back3DLaunch L;
    L.P = P;
    L.views = pl->views.as<View3D>();
    L.gate_ptr = pl->gate_ptr.as<int>();
    L.entries = pl->entries.as<GateEntry>();
    L.ngates = pl->nt;
    L.view_lo = (int)view0;
    L.view_hi = (int)(view0 + nview);
    L.sino = src;
    L.sino_view_stride = npix;
    L.vol = volo;
    L.gate_stride = nvox;
    L.factorized = pl->factorized ? 1 : 0;
    L.pairs = pl->nt > 1 ? pl->pairs.as<GatePair>() : nullptr;
    L.err = pl->err.as<int>();
    TRTT_CK(launch_back3d(L, st));
    count_launch();
    if (layout == TRTT_B200_LAYOUT_XYZ) {
      TRTT_CK(col_f32_add_to_xyz_f32(volo, dst, P.nx, P.ny, P.nz, pl->nt, st));
      count_launch();
    }
  }
  return 0;
}

extern "C" int trtt_b200_plan3d_forward(trtt_b200_plan3d *pl, const float *vol, float *sino,
                                        long view0, long nview, int layout, void *stream)
{
  return plan_run(pl, vol, sino, view0, nview, layout, stream, true);
}

extern "C" int trtt_b200_plan3d_backward(trtt_b200_plan3d *pl, const float *sino, float *vol,
                                         long view0, long nview, int layout, void *stream)
{
  return plan_run(pl, sino, vol, view0, nview, layout, stream, false);
}

extern "C" int trtt_b200_plan3d_status(trtt_b200_plan3d *pl, void *stream)
{
  clear_error();
  if (!pl) return fail("plan3d_status: null plan");
  int h = 0;
  TRTT_CK(cudaStreamSynchronize((cudaStream_t)stream));
  TRTT_CK(cudaMemcpy(&h, pl->err.p, sizeof(int), cudaMemcpyDeviceToHost));
  TRTT_CK(cudaMemset(pl->err.p, 0, sizeof(int)));
  if (h & TRTT_ERR_SOURCE_PLANE) return fail("a voxel lies in the source plane (wk == 0)");
  if (h & TRTT_ERR_STALL) return fail("a bounded device wait ran out (persistent launch stalled)");
  if (h) return fail("device error flag set");
  return 0;
}

extern "C" int trtt_b200_plan3d_destroy(trtt_b200_plan3d *pl)
{
  if (!pl) return 0;
  pl->views.release();
  pl->cum.release();
  pl->gate_ptr.release();
  pl->entries.release();
  pl->pairs.release();
  for (auto &gb : pl->groups) gb.release();
  pl->resid.release();
  pl->wls_parts.release();
  pl->wls_queue.release();
  pl->scratch.release();
  pl->err.release();
  delete pl;
  return 0;
}

// ---------------------------------------------------------------------------
// Host-buffer entry points (drop-in and batched)
// ---------------------------------------------------------------------------
namespace {

// One call of a 3D projector on host double* arrays for `nviews` views:
// out += H in (job 0) or out += H^T in (job != 0), reference layouts.
// View chunks of the host-buffer pipeline, as boundaries (chunks + 1
// entries).  Only one copy per call cannot overlap a kernel: the read-back
// of the direct projection's last chunk and the upload of the transpose's
// first chunk.  The direct projection therefore runs full chunks and ends
// with a chunk of one wave of CTAs (`tail` views); the transpose starts with
// `head` views and grows its chunks by half each time (each upload hides
// behind the previous chunk's kernel) up to `full` views.  At most `cap`
// chunks (the event pool).
std::vector<long> fwd_chunks(long nviews, long full, long tail, int cap)
{
  std::vector<long> b{0};
  tail = std::max<long>(1, std::min(tail, nviews));
  const long mid = nviews - tail;
  if (mid > 0) {
    const long n = std::min<long>(std::max<long>(1, (mid + full - 1) / full), cap - 1);
    for (long c = 0; c < n; ++c) b.push_back(b.back() + mid / n + (c < mid % n ? 1 : 0));
  }
  b.push_back(nviews);
  return b;
}

std::vector<long> back_chunks(long nviews, long head, long full, int cap)
{
  std::vector<long> b{0};
  double size = (double)std::max<long>(1, head);
  while (b.back() < nviews) {
    long c = std::min<long>((long)size, nviews - b.back());
    if ((int)b.size() == cap) c = nviews - b.back();
    b.push_back(b.back() + c);
    size = std::min<double>(size * 1.5, (double)std::max<long>(1, full));
  }
  return b;
}

// Runs [first, last) of consecutive view indices among the members of
// groups [g0, g1) of a list of groups of G views (4 ints per group).
void member_runs(const std::vector<int> &list, int G, long g0, long g1,
                 std::vector<std::pair<long, long>> &runs)
{
  std::vector<long> v;
  for (long g = g0; g < g1; ++g)
    for (int m = 0; m < G; ++m) v.push_back(list[4 * g + m]);
  std::sort(v.begin(), v.end());
  runs.clear();
  for (size_t t = 0; t < v.size();) {
    size_t e = t + 1;
    while (e < v.size() && v[e] == v[e - 1] + 1) ++e;
    runs.push_back({v[t], v[e - 1] + 1});
    t = e;
  }
}

// Host-buffer projection of a grouped scan (closed-form model, factorised
// views, groups found by find_view_groups): the group kernels run in chunks
// of groups; the forward reads each chunk's views back while later chunks
// are projected, the transpose projects each chunk as soon as its views are
// on the device.  `out64` already receives `out` (or zeros) on the copy
// stream, ordered after ev[0].
int host3d_grouped(DropIn &D, const Params3D &P, double *out, const double *in,
                   const std::vector<int> (&lists)[3], long nviews, int job,
                   const std::function<cudaError_t(cudaStream_t)> &out_to_device, bool in_early)
{
  cudaStream_t st = D.stream, cp = D.copy, ks2 = D.stream2;
  const long nx = P.nx, ny = P.ny, nz = P.nz, nu = P.nu, nv = P.nv;
  const long nvox = nx * ny * nz, nview_px = nu * nv, npix = nview_px * nviews;
  // group lists on the device, one after the other
  long total = 0, offs[3];
  for (int q = 0; q < 3; ++q) {
    offs[q] = total;
    total += (long)lists[q].size();
  }
  TRTT_CK(D.grp.ensure(sizeof(int) * std::max<long>(1, total)));
  for (int q = 0; q < 3; ++q)
    if (!lists[q].empty())
      TRTT_CK(cudaMemcpyAsync(D.grp.as<int>() + offs[q], lists[q].data(), sizeof(int) * lists[q].size(),
                              cudaMemcpyHostToDevice, st));
  const int usplit = (int)((nu + 255) / 256), utile = (int)((nu + usplit - 1) / usplit);
  std::vector<std::pair<long, long>> runs;
  int ev = 2;
  if (job == 0) {
    if (in_early)  // started on the copy stream before the grouping
      TRTT_CK(cudaStreamWaitEvent(st, D.ev[DropIn::kEvIn], 0));
    else
      TRTT_CK(upload_host(D, D.in64.p, in, sizeof(double) * nvox, st));
    TRTT_CK(out_to_device(cp));
    TRTT_CK(xyz_f64_to_col_f32(D.in64.as<double>(), D.vol32.as<float>(), (int)nx, (int)ny, (int)nz, 1, st));
    TRTT_CK(cudaMemsetAsync(D.det32.p, 0, sizeof(float) * npix, st));
    TRTT_CK(cudaEventRecord(D.ev[DropIn::kEvents - 2], st));
    TRTT_CK(cudaStreamWaitEvent(ks2, D.ev[DropIn::kEvents - 2], 0));
    int unit = 0;
    for (int q = 2; q >= 0; --q) {
      const long n = (long)lists[q].size() / 4;
      if (!n) continue;
      const int G = q == 2 ? 4 : q + 1;
      GroupFwdLaunch L;
      L.P = P;
      L.views = D.geom.as<View3D>();
      L.vol = D.vol32.as<float>();
      L.sino = D.det32.as<float>();
      L.sino_view_stride = nview_px;
      L.band_rows = (int)std::min<long>(G == 1 ? 64 : 32, nv);
      L.usplit = usplit;
      L.utile = utile;
      L.interleave = 1;
      L.minb = G == 4 ? 1 : 2;
      L.warps = group_fwd_warps(G, L.band_rows, utile, L.minb);
      L.err = D.err.as<int>();
      const long bands = (nv + L.band_rows - 1) / L.band_rows;
      const long per_wave = (long)D.sms * (G == 4 ? 1 : 2);
      // chunks of at most ~84 MB of FP64 output (1.5 ms of read-back at
      // ~57 GB/s), so that the read-back of the last full chunk hides behind
      // the last, one-wave chunk (measured at 256^3 -> 360 x 512^2: chunks of
      // 10 quads 39.4 ms per call, of 15 quads 40.1-42.3 ms)
      const long per_chunk = std::max<long>(1, std::min<long>((n + 5) / 6, 84000000L / (G * nview_px * 8)));
      const std::vector<long> cb = fwd_chunks(n, per_chunk, std::max<long>(1, per_wave / (bands * usplit)), 12);
      for (size_t c = 0; c + 1 < cb.size(); ++c, ++unit) {
        cudaStream_t ks = (unit & 1) ? ks2 : st;
        L.groups = D.grp.as<int>() + offs[q] + 4 * cb[c];
        L.ngroups = (int)(cb[c + 1] - cb[c]);
        TRTT_CK(launch_fwd3d_group(L, G, ks));
        TRTT_CK(cudaEventRecord(D.ev[ev], ks));
        TRTT_CK(cudaStreamWaitEvent(cp, D.ev[ev], 0));
        ++ev;
        count_launch();
        member_runs(lists[q], G, cb[c], cb[c + 1], runs);
        for (const auto &r : runs) {
          const long off = r.first * nview_px, cnt = (r.second - r.first) * nview_px;
          TRTT_CK(f32_add_to_f64(D.det32.as<float>() + off, D.out64.as<double>() + off, cnt, cp));
          TRTT_CK(cudaMemcpyAsync(out + off, D.out64.as<double>() + off, sizeof(double) * cnt,
                                  cudaMemcpyDeviceToHost, cp));
          count_launch();
        }
      }
    }
    TRTT_CK(cudaEventRecord(D.ev[DropIn::kEvents - 1], ks2));
    TRTT_CK(cudaStreamWaitEvent(st, D.ev[DropIn::kEvents - 1], 0));
    TRTT_CK(cudaEventRecord(D.ev[1], cp));
    TRTT_CK(cudaStreamWaitEvent(st, D.ev[1], 0));
    TRTT_CK(cudaStreamSynchronize(st));
    return 0;
  }
  // transpose: views arrive in chunks of groups on the copy stream
  TRTT_CK(cudaMemsetAsync(D.vol32.p, 0, sizeof(float) * nvox, st));
  for (int q = 2; q >= 0; --q) {
    const long n = (long)lists[q].size() / 4;
    if (!n) continue;
    const int G = q == 2 ? 4 : q + 1;
    GroupBackLaunch L;
    L.P = P;
    L.views = D.geom.as<View3D>();
    L.groups = D.grp.as<int>() + offs[q];
    L.norbits = group_orbits(G, (int)nx, (int)ny);
    L.sino = D.det32.as<float>();
    L.sino_view_stride = nview_px;
    L.vol = D.vol32.as<float>();
    L.vec4 = (nu % 4 == 0) ? 1 : 0;  // det32 comes from cudaMalloc
    L.err = D.err.as<int>();
    const std::vector<long> cb = back_chunks(n, std::max<long>(1, n / 32), (n + 5) / 6, 10);
    for (size_t c = 0; c + 1 < cb.size(); ++c) {
      member_runs(lists[q], G, cb[c], cb[c + 1], runs);
      for (const auto &r : runs) {
        const long off = r.first * nview_px, cnt = (r.second - r.first) * nview_px;
        TRTT_CK(upload_host(D, D.in64.as<double>() + off, in + off, sizeof(double) * cnt, cp));
        TRTT_CK(f64_to_f32(D.in64.as<double>() + off, D.det32.as<float>() + off, cnt, cp));
        count_launch();
      }
      TRTT_CK(cudaEventRecord(D.ev[ev], cp));
      TRTT_CK(cudaStreamWaitEvent(st, D.ev[ev], 0));
      ++ev;
      L.g_lo = (int)cb[c];
      L.g_hi = (int)cb[c + 1];
      TRTT_CK(launch_back3d_group(L, G, st));
      count_launch();
    }
  }
  TRTT_CK(out_to_device(cp));
  TRTT_CK(cudaEventRecord(D.ev[1], cp));
  return 1;  // continue with the common tail (error check, out += volume)
}

int host3d(int geom, double *out, const double *in, long nx, long ny, long nz,
           double s_scl, int s_deg, const double *cum, long size, double step,
           const double *coord, long nu, long nv, double u_scl, double v_scl,
           long nviews, const double *xos, const double *xsd, int job,
           bool accumulate = true)
{
  clear_error();
  if (!out || !in || !xos || !xsd) return fail("null array argument");
  if (!dim_ok(nx) || !dim_ok(ny) || !dim_ok(nz) || !dim_ok(nu) || !dim_ok(nv) || !dim_ok(nviews))
    return fail("dimensions must be in [1, 2^30)");
  if (cum && (size < 1 || !coord)) return fail("invalid footprint table");
  DropIn &D = dropin();
  std::lock_guard<std::mutex> lock(D.mu);
  TRTT_CK(D.init());
  TRTT_CK(cudaSetDevice(D.device));
  cudaStream_t st = D.stream;
  const long nvox = nx * ny * nz;
  const long npix = nu * nv * nviews;
  const long nin = job == 0 ? nvox : npix, nout = job == 0 ? npix : nvox;
  // footprint table
  const double *cum_dev = nullptr;
  if (cum) {
    TRTT_CK(D.aux.ensure(sizeof(double) * size));
    TRTT_CK(cudaMemcpyAsync(D.aux.p, cum, sizeof(double) * size, cudaMemcpyHostToDevice, st));
    cum_dev = D.aux.as<double>();
  }
  Params3D P = make_params(geom, nx, ny, nz, s_scl, s_deg, cum_dev, size, step,
                           cum ? coord[0] : 0.0, nu, nv, u_scl, v_scl);
  std::vector<View3D> hv(nviews);
  bool fact = true;
  for (long v = 0; v < nviews; ++v) {
    make_view3d(P, xos + 12 * v, xsd + 12 * v, hv[v]);
    fact = fact && hv[v].factorized;
  }
  TRTT_CK(D.geom.ensure(sizeof(View3D) * nviews));
  TRTT_CK(cudaMemcpyAsync(D.geom.p, hv.data(), sizeof(View3D) * nviews, cudaMemcpyHostToDevice, st));
  TRTT_CK(D.err.ensure(sizeof(int)));
  TRTT_CK(cudaMemsetAsync(D.err.p, 0, sizeof(int), st));
  TRTT_CK(D.in64.ensure(sizeof(double) * nin));
  TRTT_CK(D.out64.ensure(sizeof(double) * nout));
  TRTT_CK(D.vol32.ensure(sizeof(float) * nvox));
  TRTT_CK(D.det32.ensure(sizeof(float) * npix));
  cudaStream_t cp = D.copy;
  // The copy stream brings `out` to the device while the kernels run (it is
  // only read there: the host array is written after the error check); with
  // accumulate == false the device copy starts from zeros instead and `out`
  // is only written.  Either must not start before the previous call's
  // read-back of out64 is done.
  TRTT_CK(cudaEventRecord(D.ev[0], st));
  TRTT_CK(cudaStreamWaitEvent(cp, D.ev[0], 0));
  // a transpose accumulated into a pageable host volume (a Yorick caller's
  // array) is added into `out` on the host at the end (download_add)
  // instead of taking `out` to the device and back
  const bool host_add = job == 1 && accumulate && sizeof(double) * nout >= (4u << 20) && host_pageable(out);
  auto out_to_device = [&](cudaStream_t s) -> cudaError_t {
    if (host_add) return cudaSuccess;
    if (accumulate) return cudaMemcpyAsync(D.out64.p, out, sizeof(double) * nout, cudaMemcpyHostToDevice, s);
    return cudaMemsetAsync(D.out64.p, 0, sizeof(double) * nout, s);
  };
  // the factorised closed-form direct projection starts from the volume:
  // its upload overlaps the view grouping and the source-plane check below
  const bool in_early = job == 0 && fact && !cum;
  if (in_early) {
    TRTT_CK(upload_host(D, D.in64.p, in, sizeof(double) * nin, cp));
    TRTT_CK(cudaEventRecord(D.ev[DropIn::kEvIn], cp));
  }
  std::vector<int> glists[3];
  bool grouped = false;
  if (fact && !cum && nviews <= 65535) {
    find_view_groups(nx, ny, nviews, xos, xsd, glists);
    grouped = !glists[1].empty() || !glists[2].empty();
  }
  if (grouped && job == 0) {
    // the source-plane pre-check of the per-view path below, then the group
    // kernels
    TRTT_CK(launch_check_columns(P, D.geom.as<View3D>(), (int)nviews, D.err.as<int>(), st));
    count_launch();
    int herr = 0;
    TRTT_CK(cudaMemcpyAsync(&herr, D.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TRTT_CK(cudaStreamSynchronize(st));
    if (herr & TRTT_ERR_SOURCE_PLANE) {
      TRTT_CK(cudaStreamSynchronize(cp));  // the early upload still reads `in`
      std::fprintf(stderr, "trtt_b200: a voxel lies in the source plane (wk == 0); out left unchanged\n");
      return fail("a voxel lies in the source plane (wk == 0)");
    }
    return host3d_grouped(D, P, out, in, glists, nviews, job, out_to_device, in_early);
  }
  if (grouped) {
    const int r = host3d_grouped(D, P, out, in, glists, nviews, job, out_to_device, in_early);
    if (r < 0) return r;
  } else if (job == 0 && fact) {
    // Column-factorised views: the only failure (a voxel in the source
    // plane) is a property of the column geometry, so it is checked first;
    // the projection then runs in view chunks (fwd_chunks) and each chunk's
    // result is added into `out` and read back while the next chunk is
    // projected.
    TRTT_CK(launch_check_columns(P, D.geom.as<View3D>(), (int)nviews, D.err.as<int>(), st));
    count_launch();
    int herr = 0;
    TRTT_CK(cudaMemcpyAsync(&herr, D.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TRTT_CK(cudaStreamSynchronize(st));
    if (herr & TRTT_ERR_SOURCE_PLANE) {
      TRTT_CK(cudaStreamSynchronize(cp));  // the early upload still reads `in`
      std::fprintf(stderr, "trtt_b200: a voxel lies in the source plane (wk == 0); out left unchanged\n");
      return fail("a voxel lies in the source plane (wk == 0)");
    }
    if (in_early)
      TRTT_CK(cudaStreamWaitEvent(st, D.ev[DropIn::kEvIn], 0));
    else
      TRTT_CK(upload_host(D, D.in64.p, in, sizeof(double) * nin, st));
    TRTT_CK(out_to_device(cp));
    TRTT_CK(xyz_f64_to_col_f32(D.in64.as<double>(), D.vol32.as<float>(), (int)nx, (int)ny, (int)nz, 1, st));
    TRTT_CK(cudaMemsetAsync(D.det32.p, 0, sizeof(float) * npix, st));
    Fwd3DLaunch L;
    L.P = P;
    L.vol = D.vol32.as<float>();
    L.gate_stride = nvox;
    L.sino_view_stride = nu * nv;
    int rows = 0, warps = 16;
    choose_band((int)nu, (int)nv, rows, warps);
    L.band_rows = rows;
    L.warps = warps;
    L.err = D.err.as<int>();
    const long bands = (nv + rows - 1) / rows;
    const std::vector<long> cb = fwd_chunks(nviews, (nviews + 5) / 6, std::max<long>(1, 2L * D.sms / bands),
                                            DropIn::kChunks);
    // chunks alternate between two kernel streams (they write disjoint
    // views), so that the last, partly filled wave of CTAs of one chunk
    // overlaps the start of the next
    cudaStream_t ks2 = D.stream2;
    TRTT_CK(cudaEventRecord(D.ev[DropIn::kEvents - 2], st));
    TRTT_CK(cudaStreamWaitEvent(ks2, D.ev[DropIn::kEvents - 2], 0));
    for (size_t c = 0; c + 1 < cb.size(); ++c) {
      const long v0 = cb[c], v1 = cb[c + 1];
      const long off = v0 * nu * nv, cnt = (v1 - v0) * nu * nv;
      cudaStream_t ks = (c & 1) ? ks2 : st;
      L.views = D.geom.as<View3D>() + v0;
      L.nviews = (int)(v1 - v0);
      L.sino = D.det32.as<float>() + off;
      TRTT_CK(launch_fwd3d(L, ks));
      TRTT_CK(cudaEventRecord(D.ev[2 + c], ks));
      TRTT_CK(cudaStreamWaitEvent(cp, D.ev[2 + c], 0));
      TRTT_CK(f32_add_to_f64(D.det32.as<float>() + off, D.out64.as<double>() + off, cnt, cp));
      TRTT_CK(cudaMemcpyAsync(out + off, D.out64.as<double>() + off, sizeof(double) * cnt,
                              cudaMemcpyDeviceToHost, cp));
      count_launch(3);
    }
    TRTT_CK(cudaEventRecord(D.ev[DropIn::kEvents - 1], ks2));
    TRTT_CK(cudaStreamWaitEvent(st, D.ev[DropIn::kEvents - 1], 0));
    TRTT_CK(cudaEventRecord(D.ev[1], cp));
    TRTT_CK(cudaStreamWaitEvent(st, D.ev[1], 0));
    TRTT_CK(cudaStreamSynchronize(st));
    return 0;
  } else if (job == 0) {
    TRTT_CK(upload_host(D, D.in64.p, in, sizeof(double) * nin, st));
    TRTT_CK(out_to_device(cp));
    TRTT_CK(cudaEventRecord(D.ev[1], cp));
    TRTT_CK(xyz_f64_to_col_f32(D.in64.as<double>(), D.vol32.as<float>(), (int)nx, (int)ny, (int)nz, 1, st));
    TRTT_CK(cudaMemsetAsync(D.det32.p, 0, sizeof(float) * npix, st));
    Fwd3DLaunch L;
    L.P = P;
    L.views = D.geom.as<View3D>();
    L.nviews = (int)nviews;
    L.vol = D.vol32.as<float>();
    L.gate_stride = nvox;
    L.sino = D.det32.as<float>();
    L.sino_view_stride = nu * nv;
    int rows = 0, warps = 16;
    choose_band((int)nu, (int)nv, rows, warps);
    L.band_rows = fact ? rows : 0;
    L.warps = warps;
    L.err = D.err.as<int>();
    TRTT_CK(launch_fwd3d(L, st));
    count_launch(2);
  } else {
    TRTT_CK(cudaMemsetAsync(D.vol32.p, 0, sizeof(float) * nvox, st));
    std::vector<int> gp = {0, (int)nviews};
    std::vector<GateEntry> ge(nviews);
    for (long v = 0; v < nviews; ++v) ge[v] = GateEntry{(int)v, 1.0f};
    TRTT_CK(D.gates.ensure(sizeof(int) * 2 + sizeof(GateEntry) * nviews + 16));
    int *gp_dev = D.gates.as<int>();
    GateEntry *ge_dev = reinterpret_cast<GateEntry *>(D.gates.as<char>() + 16);
    TRTT_CK(cudaMemcpyAsync(gp_dev, gp.data(), sizeof(int) * 2, cudaMemcpyHostToDevice, st));
    TRTT_CK(cudaMemcpyAsync(ge_dev, ge.data(), sizeof(GateEntry) * nviews, cudaMemcpyHostToDevice, st));
    Back3DLaunch L;
    L.P = P;
    L.views = D.geom.as<View3D>();
    L.gate_ptr = gp_dev;
    L.entries = ge_dev;
    L.ngates = 1;
    L.sino_view_stride = nu * nv;
    L.vol = D.vol32.as<float>();
    L.gate_stride = nvox;
    L.factorized = fact ? 1 : 0;
    L.err = D.err.as<int>();
    // the detector stack arrives in view chunks (back_chunks) on the copy
    // stream; each chunk is projected back (accumulating into the volume)
    // as soon as it is on the device, while the next chunk is copied
    const std::vector<long> cb = back_chunks(nviews, std::max<long>(1, nviews / 32), (nviews + 5) / 6,
                                             DropIn::kChunks);
    for (size_t c = 0; c + 1 < cb.size(); ++c) {
      const long v0 = cb[c], v1 = cb[c + 1];
      const long off = v0 * nu * nv, cnt = (v1 - v0) * nu * nv;
      TRTT_CK(upload_host(D, D.in64.as<double>() + off, in + off, sizeof(double) * cnt, cp));
      TRTT_CK(f64_to_f32(D.in64.as<double>() + off, D.det32.as<float>() + off, cnt, cp));
      TRTT_CK(cudaEventRecord(D.ev[2 + c], cp));
      TRTT_CK(cudaStreamWaitEvent(st, D.ev[2 + c], 0));
      L.view_lo = (int)v0;
      L.view_hi = (int)v1;
      L.sino = D.det32.as<float>() + off;  // the kernel reads sino[view - view_lo]
      TRTT_CK(launch_back3d(L, st));
      count_launch(2);
    }
    TRTT_CK(out_to_device(cp));
    TRTT_CK(cudaEventRecord(D.ev[1], cp));
  }
  TRTT_CK(cudaStreamWaitEvent(st, D.ev[1], 0));
  int herr = 0;
  TRTT_CK(cudaMemcpyAsync(&herr, D.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  if (herr & TRTT_ERR_SOURCE_PLANE) {
    std::fprintf(stderr, "trtt_b200: a voxel lies in the source plane (wk == 0); out left unchanged\n");
    return fail("a voxel lies in the source plane (wk == 0)");
  }
  if (host_add) {
    // out += result on the host: the volume comes back in FP32 (half the
    // bytes of the FP64 round trip, and no upload of `out`) through the
    // pinned staging ring, and host threads make the same FP64 additions
    TRTT_CK(D.xyz32.ensure(sizeof(float) * nvox));
    TRTT_CK(cudaMemsetAsync(D.xyz32.p, 0, sizeof(float) * nvox, st));
    TRTT_CK(col_f32_add_to_xyz_f32(D.vol32.as<float>(), D.xyz32.as<float>(), (int)nx, (int)ny, (int)nz, 1, st));
    count_launch();
    TRTT_CK(download_add(D, out, D.xyz32.as<float>(), nvox, st));
    return 0;
  }
  // out += result (FP64 accumulation on the device; out64 holds out already)
  if (job == 0) {
    TRTT_CK(f32_add_to_f64(D.det32.as<float>(), D.out64.as<double>(), npix, st));
  } else {
    TRTT_CK(col_f32_add_to_xyz_f64(D.vol32.as<float>(), D.out64.as<double>(), (int)nx, (int)ny, (int)nz, 1, st));
  }
  count_launch();
  TRTT_CK(cudaMemcpyAsync(out, D.out64.p, sizeof(double) * nout, cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  return 0;
}

}  // namespace

extern "C" {

int trtt_PB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
              int s_deg, double *footprint, double *cum_footprint,
              long size_footprint, double step_footprint, double *coord_footprint,
              long nu, long nv, double u_scl, double v_scl, double *xos,
              double *xsd, int job)
{
  (void)footprint;
  if (!cum_footprint) return fail("trtt_PB3D: null cum_footprint");
  return host3d(GEOM_PARALLEL, out, in, nx, ny, nz, s_scl, s_deg, cum_footprint,
                size_footprint, step_footprint, coord_footprint, nu, nv, u_scl, v_scl,
                1, xos, xsd, job);
}

int trtt_CB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
              int s_deg, double *footprint, double *cum_footprint,
              long size_footprint, double step_footprint, double *coord_footprint,
              long nu, long nv, double u_scl, double v_scl, double *xos,
              double *xsd, int job)
{
  (void)footprint;
  if (!cum_footprint) return fail("trtt_CB3D: null cum_footprint");
  return host3d(GEOM_CONE, out, in, nx, ny, nz, s_scl, s_deg, cum_footprint,
                size_footprint, step_footprint, coord_footprint, nu, nv, u_scl, v_scl,
                1, xos, xsd, job);
}

int trtt_PB3D_cubic(double *out, double *in, long nx, long ny, long nz,
                    double s_scl, int s_deg, long nu, long nv, double u_scl,
                    double v_scl, double *xos, double *xsd, int job)
{
  return host3d(GEOM_PARALLEL, out, in, nx, ny, nz, s_scl, s_deg, nullptr, 0, 1.0,
                nullptr, nu, nv, u_scl, v_scl, 1, xos, xsd, job);
}

int trtt_CB3D_cubic(double *out, double *in, long nx, long ny, long nz,
                    double s_scl, int s_deg, long nu, long nv, double u_scl,
                    double v_scl, double *xos, double *xsd, int job)
{
  return host3d(GEOM_CONE, out, in, nx, ny, nz, s_scl, s_deg, nullptr, 0, 1.0,
                nullptr, nu, nv, u_scl, v_scl, 1, xos, xsd, job);
}

int trtt_b200_cb3d_batch(double *out, const double *in, long nx, long ny, long nz,
                         double s_scl, int s_deg, const double *cum_footprint,
                         long size_footprint, double step_footprint,
                         const double *coord_footprint, long nu, long nv,
                         double u_scl, double v_scl, long nviews,
                         const double *xos, const double *xsd, int geometry,
                         int job)
{
  const int g = geom_code(geometry);
  if (g < 0) return fail("cb3d_batch: geometry must be 3, 4 or 5");
  return host3d(g, out, in, nx, ny, nz, s_scl, s_deg, cum_footprint, size_footprint,
                step_footprint, coord_footprint, nu, nv, u_scl, v_scl, nviews, xos, xsd,
                job);
}

int trtt_b200_cb3d_batch_ex(double *out, const double *in, long nx, long ny, long nz,
                            double s_scl, int s_deg, const double *cum_footprint,
                            long size_footprint, double step_footprint,
                            const double *coord_footprint, long nu, long nv,
                            double u_scl, double v_scl, long nviews,
                            const double *xos, const double *xsd, int geometry,
                            int job, int accumulate)
{
  const int g = geom_code(geometry);
  if (g < 0) return fail("cb3d_batch_ex: geometry must be 3, 4 or 5");
  return host3d(g, out, in, nx, ny, nz, s_scl, s_deg, cum_footprint, size_footprint,
                step_footprint, coord_footprint, nu, nv, u_scl, v_scl, nviews, xos, xsd,
                job, accumulate != 0);
}

}  // extern "C"
