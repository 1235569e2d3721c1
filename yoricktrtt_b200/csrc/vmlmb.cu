// vmlmb.cu -- native VMLM-B + TV reconstruction on a 3D projector plan.
//
// Minimises f(x) = 1/2 (Hx - y)' W (Hx - y) + mu TV(S x) under
// lower <= x <= upper (the cost of Tomography_3D/Ytrtt3D_optim.i:128-234,
// minimised by OptimPack's VMLM-B at Tomography_3D/Ytrtt3D_optim.i:663),
// with the rules of yoricktrtt_b200/recon.py vmlmb (L-BFGS on the free
// variables, projected Armijo backtracking with safeguarded quadratic steps,
// stop on |f_k - f_k+1| <= frtol max(|f_k|, |f_k+1|)).  Everything but the
// branch decisions stays on the device: vector updates are fused kernels,
// inner products are FP64 accumulators, the two-loop recursion applies its
// coefficients as device scalars, and the host reads back a handful of
// doubles per iteration.  The iterate is kept in the kernels' column layout
// for the whole solve (TV and the B-spline sampling are symmetric under the
// axis permutation).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <mutex>
#include <vector>

#include "kernels.h"
#include "runtime.h"
#include "trtt_b200.h"

namespace {

constexpr int kThreads = 256;

unsigned blocks_for(long n)
{
  long b = (n + kThreads - 1) / kThreads;
  if (b > 148L * 8) b = 148L * 8;
  return (unsigned)(b > 0 ? b : 1);
}

__device__ __forceinline__ void block_add(double v, double *out)
{
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < kThreads / 32 ? red[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(out, v);
  }
}

#define GRID_LOOP(i, n) for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long)gridDim.x * blockDim.x)

// free = not blocked by an active bound, pg = g free; acc[0] += pg.pg, acc[1] += x.x
__global__ void k_free_pg(const float *__restrict__ x, const float *__restrict__ g, float *__restrict__ fr,
                          float *__restrict__ pg, long n, float lo, float hi, int has_lo, int has_hi,
                          double *__restrict__ acc)
{
  double a0 = 0.0, a1 = 0.0;
  GRID_LOOP(i, n) {
    const float xi = x[i], gi = g[i];
    const bool blk = (has_lo && xi <= lo && gi > 0.f) || (has_hi && xi >= hi && gi < 0.f);
    const float f = blk ? 0.f : 1.f;
    const float p = __fmul_rn(gi, f);
    fr[i] = f;
    pg[i] = p;
    a0 += (double)p * (double)p;
    a1 += (double)xi * (double)xi;
  }
  block_add(a0, acc);
  block_add(a1, acc + 1);
}

// acc += sum (a m)(b m) with m the free mask (m may be null: unmasked)
__global__ void k_mdot(const float *__restrict__ a, const float *__restrict__ b, const float *__restrict__ m,
                       long n, double *__restrict__ acc)
{
  double s = 0.0;
  GRID_LOOP(i, n) {
    float ai = a[i], bi = b[i];
    if (m) {
      ai = __fmul_rn(ai, m[i]);
      bi = __fmul_rn(bi, m[i]);
    }
    s += (double)ai * (double)bi;
  }
  block_add(s, acc);
}

// q -= (float)(num / den) * (y m)
__global__ void k_axpy1(float *__restrict__ q, const float *__restrict__ y, const float *__restrict__ m, long n,
                        const double *__restrict__ num, double den)
{
  const float c = (float)(*num / den);
  GRID_LOOP(i, n) q[i] = __fsub_rn(q[i], __fmul_rn(c, __fmul_rn(y[i], m[i])));
}

// q *= (float)(sy / yy)
__global__ void k_scale(float *__restrict__ q, long n, double sy, const double *__restrict__ yy)
{
  const float c = (float)(sy / *yy);
  GRID_LOOP(i, n) q[i] = __fmul_rn(q[i], c);
}

// q += (float)(na / sy - nb / sy) * (s m)
__global__ void k_axpy2(float *__restrict__ q, const float *__restrict__ s, const float *__restrict__ m, long n,
                        const double *__restrict__ na, const double *__restrict__ nb, double sy)
{
  const float c = (float)(*na / sy - *nb / sy);
  GRID_LOOP(i, n) q[i] = __fadd_rn(q[i], __fmul_rn(c, __fmul_rn(s[i], m[i])));
}

// d = -(q m); acc += g.d
__global__ void k_dir(float *__restrict__ d, const float *__restrict__ q, const float *__restrict__ m,
                      const float *__restrict__ g, long n, double *__restrict__ acc)
{
  double s = 0.0;
  GRID_LOOP(i, n) {
    const float v = m ? -__fmul_rn(q[i], m[i]) : -q[i];
    d[i] = v;
    s += (double)g[i] * (double)v;
  }
  block_add(s, acc);
}

// xt = clip(x + alpha d), step = xt - x, acc += g.step
__global__ void k_trial(const float *__restrict__ x, const float *__restrict__ d, const float *__restrict__ g,
                        float *__restrict__ xt, float *__restrict__ step, long n, float alpha, float lo, float hi,
                        int has_lo, int has_hi, double *__restrict__ acc)
{
  double s = 0.0;
  GRID_LOOP(i, n) {
    float v = __fadd_rn(x[i], __fmul_rn(alpha, d[i]));
    if (has_lo) v = fmaxf(v, lo);
    if (has_hi) v = fminf(v, hi);
    const float st = __fsub_rn(v, x[i]);
    xt[i] = v;
    step[i] = st;
    s += (double)g[i] * (double)st;
  }
  block_add(s, acc);
}

// y = gt - g, acc += s.y
__global__ void k_pair(const float *__restrict__ gt, const float *__restrict__ g, const float *__restrict__ s,
                       float *__restrict__ y, long n, double *__restrict__ acc)
{
  double a = 0.0;
  GRID_LOOP(i, n) {
    const float v = __fsub_rn(gt[i], g[i]);
    y[i] = v;
    a += (double)s[i] * (double)v;
  }
  block_add(a, acc);
}

__global__ void k_add(float *__restrict__ a, const float *__restrict__ b, long n)
{
  GRID_LOOP(i, n) a[i] = __fadd_rn(a[i], b[i]);
}

// device scalar slots
enum {
  kF = 0,        // objective of the last evaluation
  kGStep = 1,    // g . (xt - x) of the last trial
  kPg = 2,       // |pg|^2
  kX = 3,        // |x|^2
  kGD = 4,       // g . d
  kCand = 5,     // s . y of the candidate pair (full space)
  kPairs = 8,    // free-space s . y of the pending pairs (up to 33)
  kNumA = 48,    // two-loop numerators s . q (up to 33)
  kNumB = 88,    // two-loop numerators y . q (up to 33)
  kYY = 121,     // y . y of the newest used pair
  kJunk = 127,
  kSlots = 128
};

// Work buffers are kept between calls with the same sizes (a reconstruction
// loop over many samples then allocates once) and freed when the sizes
// change; the last set is held until the process exits.
struct Workspace {
  std::mutex mu;
  int device = -1;
  long n = 0, m = 0;
  int mem = 0;
  std::vector<float *> bufs;
  double *acc = nullptr;
  void release()
  {
    for (float *p : bufs) cudaFree(p);
    bufs.clear();
    if (acc) cudaFree(acc);
    acc = nullptr;
    n = m = 0;
    mem = 0;
  }
};
Workspace &workspace()
{
  static Workspace *ws = new Workspace;  // never destroyed: the CUDA context may be gone at exit
  return *ws;
}

struct Solver {
  trtt_b200_plan3d *plan;
  cudaStream_t st;
  long n, m;
  long tx, ty, tz;  // dims handed to the TV / spline kernels (fastest first)
  const float *y, *w;
  double mu, eps;
  Workspace *ws = nullptr;
  size_t next = 0;  // next buffer of the workspace to hand out
  bool oom = false;
  float *hx, *wr, *z, *tmp, *gz, *sg;
  long nviews;
  double *acc = nullptr;  // device scalars (kSlots)
  // view sharding: this rank's data term is summed over `world` ranks by
  // `allreduce` (one FP32 gradient and one FP64 objective per evaluation);
  // the regulariser is added by rank 0 only, before the sum
  int rank = 0, world = 1;
  trtt_b200_allreduce_fn allreduce = nullptr;
  void *ctx = nullptr;

  // in-place sum over the ranks of `count` device values (dtype 0: FP32,
  // 1: FP64); a no-op on one rank
  int reduce(void *buf, long count, int dtype)
  {
    if (world <= 1) return 0;
    if (allreduce(ctx, buf, count, dtype, st) != 0) return trtt::fail("recon3d: all-reduce failed");
    return 0;
  }

  // hand out the workspace's buffers in a fixed order; allocate on first use
  float *alloc(long count)
  {
    if (next < ws->bufs.size()) return ws->bufs[next++];
    float *p = nullptr;
    if (cudaMalloc(&p, sizeof(float) * count) != cudaSuccess) {
      oom = true;
      return nullptr;
    }
    ws->bufs.push_back(p);
    ++next;
    return p;
  }

  // f(x) and g = grad f(x); f is read back (synchronises)
  int eval(const float *x, float *g, double *f, double *extra_dev = nullptr, double *extra = nullptr)
  {
    TRTT_CK(cudaMemsetAsync(acc + kF, 0, sizeof(double), st));
    TRTT_CK(cudaMemsetAsync(hx, 0, sizeof(float) * m, st));
    if (trtt_b200_plan3d_forward(plan, x, hx, 0, nviews, TRTT_B200_LAYOUT_COLUMNS, st) != 0) return -1;
    if (trtt_b200_wls_residual(hx, y, w, wr, m, acc + kF, st) != 0) return -1;
    TRTT_CK(cudaMemsetAsync(g, 0, sizeof(float) * n, st));
    if (trtt_b200_plan3d_backward(plan, wr, g, 0, nviews, TRTT_B200_LAYOUT_COLUMNS, st) != 0) return -1;
    if (mu > 0 && rank == 0) {
      if (trtt_b200_spline_sample(x, z, tmp, tx, ty, tz, st) != 0) return -1;
      TRTT_CK(cudaMemsetAsync(gz, 0, sizeof(float) * n, st));
      if (trtt_b200_tv(z, tx, ty, tz, eps, mu, gz, acc + kF, st) != 0) return -1;
      if (trtt_b200_spline_sample(gz, sg, tmp, tx, ty, tz, st) != 0) return -1;
      k_add<<<blocks_for(n), kThreads, 0, st>>>(g, sg, n);
      trtt::count_launch();
    }
    if (reduce(g, n, 0) != 0 || reduce(acc + kF, 1, 1) != 0) return -1;
    if (extra_dev && reduce(extra_dev, 1, 1) != 0) return -1;
    double h[1];
    TRTT_CK(cudaMemcpyAsync(h, acc + kF, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (extra_dev) TRTT_CK(cudaMemcpyAsync(extra, extra_dev, sizeof(double), cudaMemcpyDeviceToHost, st));
    TRTT_CK(cudaStreamSynchronize(st));
    *f = h[0];
    if (extra_dev) *extra /= (double)world;  // the ranks' copies of a replicated value
    return 0;
  }
};

}  // namespace

extern "C" int trtt_b200_recon3d_sharded(trtt_b200_plan3d *plan, const float *y, const float *w, float *x,
                                         int layout, double mu, double eps, double lower, double upper,
                                         int mem, int maxiter, double frtol, double *f_hist, double *t_hist,
                                         trtt_b200_vmlmb_info *info, void *stream, int rank, int world,
                                         trtt_b200_allreduce_fn allreduce, void *ctx)
{
  using namespace trtt;
  clear_error();
  if (!plan || !y || !x || !info) return fail("recon3d: null argument");
  if (world < 1 || rank < 0 || rank >= world) return fail("recon3d: invalid rank / world");
  if (world > 1 && !allreduce) return fail("recon3d: several ranks need an all-reduce hook");
  if (layout != TRTT_B200_LAYOUT_XYZ && layout != TRTT_B200_LAYOUT_COLUMNS)
    return fail("recon3d: unknown volume layout");
  if (mem < 1 || mem > 32 || maxiter < 0 || !(frtol >= 0) || mu < 0 || !(eps > 0))
    return fail("recon3d: bad solver parameters");
  long shape[7];
  if (trtt_b200_plan3d_shape(plan, shape) != 0) return -1;
  const long nx = shape[0], ny = shape[1], nz = shape[2], nu = shape[3], nv = shape[4], nviews = shape[5];
  if (shape[6] != 1) return fail("recon3d: gated (4D) plans are not supported");
  const auto t_start = std::chrono::steady_clock::now();
  auto seconds = [&]() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  };

  Workspace &W = workspace();
  std::lock_guard<std::mutex> lock(W.mu);
  int dev = 0;
  TRTT_CK(cudaGetDevice(&dev));
  if (W.device != dev || W.n != nx * ny * nz || W.m != nviews * nu * nv || W.mem != mem) {
    if (W.device >= 0 && W.device != dev) {  // free the other device's buffers there
      TRTT_CK(cudaSetDevice(W.device));
      W.release();
      TRTT_CK(cudaSetDevice(dev));
    } else {
      W.release();
    }
    W.device = dev;
    W.n = nx * ny * nz;
    W.m = nviews * nu * nv;
    W.mem = mem;
  }
  Solver S;
  S.ws = &W;
  S.plan = plan;
  S.st = static_cast<cudaStream_t>(stream);
  S.n = nx * ny * nz;
  S.m = nviews * nu * nv;
  S.tx = nz; S.ty = nx; S.tz = ny;  // column layout [j][i][k]: k fastest
  S.nviews = nviews;
  S.y = y;
  S.w = w;
  S.mu = mu;
  S.eps = eps;
  S.rank = rank;
  S.world = world;
  S.allreduce = allreduce;
  S.ctx = ctx;
  if (!W.acc) TRTT_CK(cudaMalloc(&W.acc, sizeof(double) * kSlots));
  S.acc = W.acc;
  const long n = S.n;
  S.hx = S.alloc(S.m);
  S.wr = S.alloc(S.m);
  S.z = S.alloc(n);
  S.tmp = S.alloc(n);
  S.gz = S.alloc(n);
  S.sg = S.alloc(n);
  float *xc = S.alloc(n), *g = S.alloc(n), *xt = S.alloc(n), *gt = S.alloc(n), *d = S.alloc(n),
        *q = S.alloc(n), *fr = S.alloc(n), *pg = S.alloc(n);
  std::vector<float *> Sb(mem + 1), Yb(mem + 1);
  for (int k = 0; k <= mem; ++k) {
    Sb[k] = S.alloc(n);
    Yb[k] = S.alloc(n);
  }
  if (S.oom) {
    cudaGetLastError();
    W.release();
    return fail("recon3d: out of device memory");
  }
  cudaStream_t st = S.st;
  const unsigned B = blocks_for(n);
  const bool has_lo = std::isfinite(lower), has_hi = std::isfinite(upper);
  const float flo = has_lo ? (float)lower : 0.f, fhi = has_hi ? (float)upper : 0.f;

  // start: x in the column layout, clipped to the box
  if (layout == TRTT_B200_LAYOUT_XYZ) {
    TRTT_CK(xyz_f32_to_col_f32(x, xt, (int)nx, (int)ny, (int)nz, 1, st));
    count_launch();
  } else {
    TRTT_CK(cudaMemcpyAsync(xt, x, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
  }
  TRTT_CK(cudaMemsetAsync(d, 0, sizeof(float) * n, st));
  k_trial<<<B, kThreads, 0, st>>>(xt, d, d, xc, q, n, 0.f, flo, fhi, has_lo, has_hi, S.acc + kJunk);
  count_launch();
  double f;
  if (S.eval(xc, g, &f) != 0) return -1;
  info->evaluations = 1;
  info->iterations = 0;
  info->converged = 0;
  info->f_first = f;
  if (f_hist) f_hist[0] = f;
  if (t_hist) t_hist[0] = 0.0;

  std::vector<int> ring;  // slots of the stored pairs, oldest first
  int cand = -1;          // slot of the last step's pair (not yet tested)
  std::vector<int> freeslots;
  for (int k = 0; k <= mem; ++k) freeslots.push_back(k);
  double *A = S.acc;
  for (int it = 1; it <= maxiter; ++it) {
    // free variables, projected gradient, one read-back of all scalars
    std::vector<int> pend = ring;
    if (cand >= 0) pend.push_back(cand);
    const int np = (int)pend.size();
    TRTT_CK(cudaMemsetAsync(A + kPg, 0, sizeof(double) * 2, st));
    TRTT_CK(cudaMemsetAsync(A + kPairs, 0, sizeof(double) * (np > 0 ? np : 1), st));
    k_free_pg<<<B, kThreads, 0, st>>>(xc, g, fr, pg, n, flo, fhi, has_lo, has_hi, A + kPg);
    count_launch();
    for (int k = 0; k < np; ++k) {
      k_mdot<<<B, kThreads, 0, st>>>(Sb[pend[k]], Yb[pend[k]], fr, n, A + kPairs + k);
      count_launch();
    }
    // sharded: every rank holds the same vectors; the scalars the host
    // branches on are averaged over the ranks so that all ranks take the
    // same decisions
    if (S.reduce(A + kPg, kPairs + np - kPg, 1) != 0) return -1;
    std::vector<double> h(kPairs + np);
    TRTT_CK(cudaMemcpyAsync(h.data(), A, sizeof(double) * (kPairs + np), cudaMemcpyDeviceToHost, st));
    TRTT_CK(cudaStreamSynchronize(st));
    for (int k = kPg; k < kPairs + np; ++k) h[k] /= (double)world;
    const double pgn = std::sqrt(h[kPg]), xn = std::sqrt(h[kX]);
    std::vector<double> syf(h.begin() + kPairs, h.end());
    if (cand >= 0) {
      if (h[kCand] > 0.0) {
        ring.push_back(cand);
      } else {
        freeslots.push_back(cand);
        pend.pop_back();
        syf.pop_back();
      }
      cand = -1;
      if ((int)ring.size() > mem) {
        freeslots.push_back(ring.front());
        ring.erase(ring.begin());
        pend.erase(pend.begin());
        syf.erase(syf.begin());
      }
    }
    if (pgn == 0.0) {
      info->converged = 2;
      break;
    }
    // two-loop recursion on the free subspace, coefficients on the device
    TRTT_CK(cudaMemcpyAsync(q, pg, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    std::vector<int> used;  // indices into pend, newest first
    const int SA = kNumA, SB = kNumB;
    TRTT_CK(cudaMemsetAsync(A + SA, 0, sizeof(double) * (kYY + 1 - SA), st));
    for (int k = (int)pend.size() - 1; k >= 0; --k) {
      if (syf[k] <= 0.0) continue;
      const int u = (int)used.size();
      k_mdot<<<B, kThreads, 0, st>>>(Sb[pend[k]], q, fr, n, A + SA + u);
      k_axpy1<<<B, kThreads, 0, st>>>(q, Yb[pend[k]], fr, n, A + SA + u, syf[k]);
      count_launch(2);
      used.push_back(k);
    }
    double alpha;
    bool have_dir = false;
    if (!used.empty()) {
      const int k0 = used[0];
      k_mdot<<<B, kThreads, 0, st>>>(Yb[pend[k0]], Yb[pend[k0]], fr, n, A + kYY);
      k_scale<<<B, kThreads, 0, st>>>(q, n, syf[k0], A + kYY);
      count_launch(2);
      for (int u = (int)used.size() - 1; u >= 0; --u) {
        const int k = used[u];
        k_mdot<<<B, kThreads, 0, st>>>(Yb[pend[k]], q, fr, n, A + SB + u);
        k_axpy2<<<B, kThreads, 0, st>>>(q, Sb[pend[k]], fr, n, A + SA + u, A + SB + u, syf[k]);
        count_launch(2);
      }
      TRTT_CK(cudaMemsetAsync(A + kGD, 0, sizeof(double), st));
      k_dir<<<B, kThreads, 0, st>>>(d, q, fr, g, n, A + kGD);
      count_launch();
      alpha = 1.0;
      have_dir = true;
    } else {
      TRTT_CK(cudaMemsetAsync(A + kGD, 0, sizeof(double), st));
      k_dir<<<B, kThreads, 0, st>>>(d, pg, nullptr, g, n, A + kGD);
      count_launch();
      alpha = (xn > 0 ? 0.1 * xn : 1.0) / pgn;
    }
    double gd;
    if (S.reduce(A + kGD, 1, 1) != 0) return -1;
    TRTT_CK(cudaMemcpyAsync(&gd, A + kGD, sizeof(double), cudaMemcpyDeviceToHost, st));
    TRTT_CK(cudaStreamSynchronize(st));
    gd /= (double)world;
    if (gd >= 0.0 && have_dir) {  // not a descent direction: restart with the gradient
      for (int s : ring) freeslots.push_back(s);
      ring.clear();
      TRTT_CK(cudaMemsetAsync(A + kGD, 0, sizeof(double), st));
      k_dir<<<B, kThreads, 0, st>>>(d, pg, nullptr, g, n, A + kGD);
      count_launch();
      alpha = (xn > 0 ? 0.1 * xn : 1.0) / pgn;
      if (S.reduce(A + kGD, 1, 1) != 0) return -1;
      TRTT_CK(cudaMemcpyAsync(&gd, A + kGD, sizeof(double), cudaMemcpyDeviceToHost, st));
      TRTT_CK(cudaStreamSynchronize(st));
      gd /= (double)world;
    }
    // the step of this iteration goes to a free slot (it becomes the candidate pair)
    const int slot = freeslots.back();
    freeslots.pop_back();
    double ft = 0.0;
    bool ok = false;
    for (int bt = 0; bt < 30; ++bt) {
      TRTT_CK(cudaMemsetAsync(A + kGStep, 0, sizeof(double), st));
      k_trial<<<B, kThreads, 0, st>>>(xc, d, g, xt, Sb[slot], n, (float)alpha, flo, fhi, has_lo, has_hi,
                                      A + kGStep);
      count_launch();
      double gs = 0.0;
      if (S.eval(xt, gt, &ft, A + kGStep, &gs) != 0) return -1;
      info->evaluations += 1;
      if (ft <= f + 1e-4 * gs) {
        ok = true;
        break;
      }
      const double denom = 2.0 * (ft - f - gd * alpha);
      const double aq = denom > 0 ? -gd * alpha * alpha / denom : 0.5 * alpha;
      alpha = std::min(std::max(aq, 0.1 * alpha), 0.5 * alpha);
    }
    if (!ok) {
      freeslots.push_back(slot);
      info->converged = -1;
      break;
    }
    // candidate pair (s = step, y = gt - g); its s'y is tested next iteration
    TRTT_CK(cudaMemsetAsync(A + kCand, 0, sizeof(double), st));
    k_pair<<<B, kThreads, 0, st>>>(gt, g, Sb[slot], Yb[slot], n, A + kCand);
    count_launch();
    cand = slot;
    const double fprev = f;
    std::swap(xc, xt);
    std::swap(g, gt);
    f = ft;
    info->iterations = it;
    if (f_hist) f_hist[it] = f;
    if (t_hist) t_hist[it] = seconds();
    if (std::fabs(fprev - f) <= frtol * std::max(std::fabs(fprev), std::fabs(f))) {
      info->converged = 1;
      break;
    }
  }
  info->f_last = f;
  if (layout == TRTT_B200_LAYOUT_XYZ) {
    TRTT_CK(cudaMemsetAsync(x, 0, sizeof(float) * n, st));
    TRTT_CK(col_f32_add_to_xyz_f32(xc, x, (int)nx, (int)ny, (int)nz, 1, st));
    count_launch();
  } else {
    TRTT_CK(cudaMemcpyAsync(x, xc, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
  }
  TRTT_CK(cudaStreamSynchronize(st));
  info->seconds = seconds();
  return 0;
}

extern "C" int trtt_b200_recon3d(trtt_b200_plan3d *plan, const float *y, const float *w, float *x, int layout,
                                 double mu, double eps, double lower, double upper, int mem, int maxiter,
                                 double frtol, double *f_hist, double *t_hist, trtt_b200_vmlmb_info *info,
                                 void *stream)
{
  return trtt_b200_recon3d_sharded(plan, y, w, x, layout, mu, eps, lower, upper, mem, maxiter, frtol,
                                   f_hist, t_hist, info, stream, 0, 1, nullptr, nullptr);
}
