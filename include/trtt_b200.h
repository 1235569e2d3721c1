/*
 * trtt_b200.h -- C ABI of libtrtt_b200, the B200 (sm_100a) implementation of
 * the TRTT forward/back projector pair.
 *
 * Two layers:
 *
 * 1. Drop-in layer.  Exactly the symbols, signatures, argument meanings and
 *    return codes of the reference TRTT plugins, so the codger-generated
 *    Yorick wrappers (plugin/ywrap.c, tomography-LongFessler-model/ywrap.c)
 *    link against this library unchanged.  Arrays are host double* in the
 *    reference layouts; every projector ACCUMULATES into `out` (the caller
 *    zeroes it), except the Long-Fessler routines whose `clr` flag clears the
 *    destination first, as in the reference.  Return value 0 = TRTT_SUCCESS,
 *    -1 = TRTT_FAILURE (plugin/trtt_common.h:131,140).  Each call copies its
 *    inputs to the GPU, computes in FP32 there, and adds the result into
 *    `out` before returning (synchronous, like the reference).  On failure
 *    `out` is left unchanged and trtt_b200_last_error() says why.
 *
 * 2. Native layer (prefix trtt_b200_).  Device pointers, FP32 data, many
 *    views per launch, caller-supplied CUDA stream; this is the performance
 *    path (a plan holds the per-view geometry on the device).
 *
 * There is no CPU fallback: without a usable CUDA device every entry point
 * returns -1.
 */
#ifndef TRTT_B200_H
#define TRTT_B200_H 1

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Drop-in layer (reference interfaces)                                      */
/* ------------------------------------------------------------------------ */

/* Replaces trtt_mvmult, plugin/trtt_common.h:267 (plugin/trtt_common.c:62-69):
 * out[i[k]-1] += a[k] * in[j[k]-1] for k < number (1-based COO). */
int trtt_mvmult(double *out, double *in, long number, double *a, long *i, long *j);

/* Replace plugin/trtt_2D_projectors.h:72-82 (plugin/trtt_2D_projectors.c:186-536,
 * plugin/trtt_2D_projectors_cubic.c:209-398). job 0 = direct (out: nv cells),
 * job != 0 = transpose (out: nx*ny pixels). */
int trtt_PB2D(double *out, double *in, long nx, long ny, double s_scl, int s_deg,
              double *footprint, double *cum_footprint, long size_footprint,
              double step_footprint, double *coord_footprint, long nv,
              double v_scl, double *xos, double *xsd, int job);
int trtt_FB2D(double *out, double *in, long nx, long ny, double s_scl, int s_deg,
              double *footprint, double *cum_footprint, long size_footprint,
              double step_footprint, double *coord_footprint, long nv,
              double v_scl, double *xos, double *xsd, int job);
int trtt_PB2D_cubic(double *out, double *in, long nx, long ny, double s_scl,
                    int s_deg, long nv, double v_scl, double *xos, double *xsd,
                    int job);
int trtt_FB2D_cubic(double *out, double *in, long nx, long ny, double s_scl,
                    int s_deg, long nv, double v_scl, double *xos, double *xsd,
                    int job);
/* Column (i,j) of the 2D system matrix: out[nv] += H(:, i + j*nx)
 * (plugin/trtt_2D_projectors.c:393-536). */
int trtt_PB2D_sparser(double *out, long i, long j, long nx, long ny, double s_scl,
                      int s_deg, double *footprint, double *cum_footprint,
                      long size_footprint, double step_footprint,
                      double *coord_footprint, long nv, double v_scl,
                      double *xos, double *xsd);
int trtt_FB2D_sparser(double *out, long i, long j, long nx, long ny, double s_scl,
                      int s_deg, double *footprint, double *cum_footprint,
                      long size_footprint, double step_footprint,
                      double *coord_footprint, long nv, double v_scl,
                      double *xos, double *xsd);

/* Replace plugin/trtt_3D_projectors.h:299,359,423 and
 * plugin/trtt_3D_projectors_cubic.h:299,363 (plugin/trtt_3D_projectors.c:959-1338,
 * plugin/trtt_3D_projectors_cubic.c:506-778).  Volume in[/out] is
 * [k][j][i] (nx fastest), detector [v][u] (nu fastest). */
int trtt_PB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
              int s_deg, double *footprint, double *cum_footprint,
              long size_footprint, double step_footprint, double *coord_footprint,
              long nu, long nv, double u_scl, double v_scl, double *xos,
              double *xsd, int job);
int trtt_CB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
              int s_deg, double *footprint, double *cum_footprint,
              long size_footprint, double step_footprint, double *coord_footprint,
              long nu, long nv, double u_scl, double v_scl, double *xos,
              double *xsd, int job);
int trtt_DD_PB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
                 long nu, long nv, double u_scl, double v_scl, double *xos,
                 double *xsd, int job);
/* Replaces the reference's trtt_DD_CB3D, commented out and unfinished in
 * plugin/trtt_3D_projectors.c:1340-1434 (same arguments as trtt_DD_PB3D):
 * cone-beam distance-driven footprint completed with its intent (the voxel
 * section through the centre, perpendicular to x or y, projected from the
 * source through its four corners; its bounding detector rectangle clamped
 * like trtt_DD_PB3D; weight s^3 magn^2 delta_u delta_v spread over the
 * rectangle; the transpose is the adjoint).  FP64; 0 or -1 (a voxel centre
 * in the source plane, out unchanged). */
int trtt_DD_CB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
                 long nu, long nv, double u_scl, double v_scl, double *xos,
                 double *xsd, int job);
/* trtt_DD_CB3D over nviews views at once (xos/xsd: nviews*12 coefficients;
 * out/in: nviews detector images of nv x nu doubles, view-major). */
int trtt_b200_dd_cb3d(double *out, const double *in, long nx, long ny, long nz, double s_scl,
                      long nu, long nv, double u_scl, double v_scl, long nviews,
                      const double *xos, const double *xsd, int job);
int trtt_PB3D_cubic(double *out, double *in, long nx, long ny, long nz,
                    double s_scl, int s_deg, long nu, long nv, double u_scl,
                    double v_scl, double *xos, double *xsd, int job);
int trtt_CB3D_cubic(double *out, double *in, long nx, long ny, long nz,
                    double s_scl, int s_deg, long nu, long nv, double u_scl,
                    double v_scl, double *xos, double *xsd, int job);

/* Long-Fessler separable-footprint fan-beam model.  The parameter block has
 * the layout of struct _lf2d_parameters
 * (tomography-LongFessler-model/LongFessler2D.h:16-28). */
typedef struct {
  double pixelSize;
  double pixelStep;
  double voxelSize;
  double sourceDistance;
  double detectorDistance;
  double objectOffset1, objectOffset2;
  long objectDimension1, objectDimension2;
  long detectorDimension;
} trtt_b200_lf2d_parameters;

/* Replace tomography-LongFessler-model/LongFessler2D.h:30-70 and the
 * sparsers declared in tomography-LongFessler-model/ywrap.c:57-77
 * (LongFessler2D.c:41-681).  void return, as in the reference; a failure
 * is reported by trtt_b200_last_error() and leaves the destination
 * unchanged. */
void lf2d_direct(const void *p, double beta, double detectorOffset,
                 const double voxel[], double pixel[], int clr);
void lf2d_line_integ_direct(const void *p, double beta, double detectorOffset,
                            const double voxel[], double pixel[], int clr);
void lf2d_adjoint(const void *p, double beta, double detectorOffset,
                  const double pixel[], double voxel[], int clr);
void lf2d_line_integ_adjoint(const void *p, double beta, double detectorOffset,
                             const double pixel[], double voxel[], int clr);
void lf2d_sparser(const void *p, double beta, double detectorOffset, long i1,
                  long i2, double pixel[], int clr);
void lf2d_line_integ_sparser(const void *p, double beta, double detectorOffset,
                             long i1, long i2, double pixel[], int clr);

/* ------------------------------------------------------------------------ */
/* Native layer                                                              */
/* ------------------------------------------------------------------------ */

/* Geometry codes (Ytrtt_common.i:70-77). */
#define TRTT_B200_PARALLEL_BEAM 3
#define TRTT_B200_CONE_BEAM 4
#define TRTT_B200_FAN_BEAM 5

/* Volume layouts accepted by the native 3D calls. */
#define TRTT_B200_LAYOUT_XYZ 0     /* [k][j][i], x fastest (reference) */
#define TRTT_B200_LAYOUT_COLUMNS 1 /* [j][i][k], z fastest (kernel order) */

/* Message describing the last failure of the calling thread ("" if none). */
const char *trtt_b200_last_error(void);

/* Library version string. */
const char *trtt_b200_version(void);

/* Number of kernel launches issued by this process so far (all entry
 * points, all devices). */
long trtt_b200_launch_count(void);

typedef struct trtt_b200_plan3d trtt_b200_plan3d;

/* Create a plan for `nviews` views of a 3D parallel or cone beam projector.
 * cum_footprint == NULL selects the closed-form cubic footprint
 * (trtt_*3D_cubic); otherwise the table footprint (trtt_*3D) with the given
 * table (copied).  xos/xsd are nviews*12 coefficients (host).  The plan
 * copies everything it needs to the current device. */
int trtt_b200_plan3d_create(trtt_b200_plan3d **plan, int geometry, long nx,
                            long ny, long nz, double s_scl, int s_deg,
                            const double *cum_footprint, long size_footprint,
                            double step_footprint, const double *coord_footprint,
                            long nu, long nv, double u_scl, double v_scl,
                            long nviews, const double *xos, const double *xsd);

/* 4D per-gate projection: view k projects the linear temporal interpolation
 * of gates floor(t_index[k]) and ceil(t_index[k]) (mod nt) with weights
 * 1-pe, pe (Ytrtt_3D_projectors.i:301-311); the transpose distributes with
 * the same weights, keeping the reference's handling of an integer
 * t_index (both indices equal: the later, zero-weight write wins,
 * Ytrtt_3D_projectors.i:369-371). */
int trtt_b200_plan3d_set_gates(trtt_b200_plan3d *plan, long nt,
                               const double *t_index);

/* sino[view-view0][nv][nu] += H_view vol for view in [view0, view0+nview).
 * vol holds nt volumes (nt = 1 unless gates were set) in `layout`. */
int trtt_b200_plan3d_forward(trtt_b200_plan3d *plan, const float *vol,
                             float *sino, long view0, long nview, int layout,
                             void *stream);

/* vol += sum_view H_view^T sino[view-view0] over [view0, view0+nview). */
int trtt_b200_plan3d_backward(trtt_b200_plan3d *plan, const float *sino,
                              float *vol, long view0, long nview, int layout,
                              void *stream);

/* Synchronise `stream`, then return 0 if no kernel of the plan has flagged
 * an error since the last call, -1 otherwise (flags are cleared). */
int trtt_b200_plan3d_status(trtt_b200_plan3d *plan, void *stream);

/* Direct-projector kernel selection.  (0, 0): defaults (band kernel with
 * shared-memory accumulation, automatic shape).  band_rows > 0: band kernel
 * with that many detector rows per CTA and `warps` warps per CTA (0 keeps
 * the current value).  band_rows == TRTT_B200_TILES_PULL: closed-form model,
 * atomic-free band kernel (each detector cell accumulated in registers by one
 * owning thread; nu <= 512).  band_rows == TRTT_B200_TILES_TENSOR: closed-form
 * model, band accumulated on the tensor cores (tcgen05 kind::tf32, each
 * value split into two TF32 parts; nu <= 1536, band height chosen from nu).
 * Its accumulation in tensor memory rounds toward zero: about 1.5e-5 relative
 * error at 256^3 -> 512^2 where the default kernels stay below 1e-6, so it is
 * never chosen automatically.  Other band_rows < 0: the per-voxel kernel. */
#define TRTT_B200_TILES_PULL (-2)
#define TRTT_B200_TILES_TENSOR (-3)

/* Host-only: the shared-memory plan of the tensor-core band kernel for an
 * nu-cell-wide detector, info[10] = {band rows, 128-cell u chunks, ring
 * groups, TMEM columns, A bytes and B bytes of one group, profile floats per
 * warp, dynamic shared memory, producer warps, columns per group}; -1 if nu
 * is too wide. */
int trtt_b200_fwd3d_tc_plan_info(int nu, long *info);
int trtt_b200_plan3d_set_tiles(trtt_b200_plan3d *plan, int band_rows, int warps);

/* Band kernel variant (closed-form model): cols = 1 one column at a time
 * (default), cols = 2 neighbouring columns in pairs, spread into the band
 * with one atomic per cell of the union of their footprints.  -1 if the
 * pair kernel's shared memory (band + 2 profiles per warp) does not fit. */
int trtt_b200_plan3d_set_columns(trtt_b200_plan3d *plan, int cols);

/* Weighted least-squares data term in one persistent launch.  No single
 * counterpart in the reference: it is the cost evaluation of its 4D
 * reconstruction (Tomography_4D/Ytrtt4D_optim.i:87-223) with the per-gate
 * projection of Ytrtt_3D_projectors.i:254-375.  For the plan's views (gates
 * set by plan3d_set_gates, else one volume):
 *   resid = W (H x - y), *cost = 1/2 sum W (H x - y)^2 (FP64, written),
 *   grad += H^T resid (per gate).
 * vol and grad: device, column layout (TRTT_B200_LAYOUT_COLUMNS), gates
 * stacked; y and w: device [view][nv][nu] (w NULL: unit weights); cost:
 * device, one double.  Closed-form model, column-factorised views (else
 * -1).  One cooperative launch of resident CTAs draws (view, band) items,
 * then (gate, column block) items from a device queue; a column item waits,
 * bounded by the plan's wait limit, for every band item; a wait that runs
 * out makes the next plan3d_status call fail ("bounded device wait ran
 * out") and the launch returns early.
 * Not synchronous: the results are ready when `stream` is. */
int trtt_b200_plan3d_wls_grad(trtt_b200_plan3d *plan, const float *vol, const float *y,
                              const float *w, float *grad, double *cost, void *stream);
/* Shape of the persistent launch: detector-row band height (0 keeps; 32 by
 * default), CTAs per SM (1: up to 128 registers per thread, 2: 64; 0
 * keeps), the bound of the device wait in seconds (0 keeps; 2 s by
 * default) and extra_wait, a test hook: column items also wait for
 * extra_wait band items that do not exist, so the bounded wait runs out. */
int trtt_b200_plan3d_set_persistent(trtt_b200_plan3d *plan, int band_rows, int ctas_per_sm,
                                    double wait_seconds, int extra_wait);

/* 1 if every view of the plan uses the column-factorised kernels. */
int trtt_b200_plan3d_factorized(const trtt_b200_plan3d *plan);

/* Orbit symmetry.  No counterpart in the reference.  At creation a plan of
 * the closed-form model whose views are all column-factorised groups its
 * views by turns of the volume grid about the z axis: {a, b1, b2, b3} when
 * view b_m sees voxel (i, j, k) where view a sees (R^m(i, j), k), R the
 * quarter turn (i, j) -> (n-1-j, i) of a square grid of even side (a
 * circular orbit of 4N views over 2 pi), else {a, b2} for the half turn (nx
 * or ny even), else {a}; xsd equal within 1e-10.  A whole-scan projection of
 * a one-gate plan then evaluates the footprints of each group's first view
 * once for all members (group kernels).  counts[0..2] = singles, pairs and
 * quads found (all-zero when the group kernels never apply to the plan).
 * set_symmetry(plan, 0) returns to the per-view kernels (results equal to
 * FP32 summation order); 2 (default) uses the group kernels with the member
 * profiles and bands of the direct projector interleaved per detector cell,
 * profiles updated by plain shared-memory loads and stores wherever the
 * voxels' first cells strictly increase along a column and band rows under
 * row locks (35.7 ms per 360 views at 256^3 -> 512^2); 1 the group kernels
 * with one profile per member and shared-memory atomics (87 ms). */
int trtt_b200_plan3d_groups(const trtt_b200_plan3d *plan, long *counts);
int trtt_b200_plan3d_set_symmetry(trtt_b200_plan3d *plan, int on);

/* Group-kernel shape: detector-row band heights of the direct kernel for
 * groups of 4, 2 and 1 views (0 keeps the current value; each in [2, nv]
 * and within shared memory) and the detector bytes the transpose covers per
 * launch (0 keeps; the images of one launch stay in L2 while every column
 * orbit walks them). */
int trtt_b200_plan3d_set_group_tiles(trtt_b200_plan3d *plan, int band_rows4, int band_rows2,
                                     int band_rows1, long back_chunk_bytes);
/* Shape of the direct kernel for groups of 4 views: band rows (0 keeps),
 * detector cells per u tile (0: up to 256; else 32..256) and CTAs per SM
 * (1: one CTA of 22 warps, or 16 where 22 warps' profiles do not fit in
 * shared memory; 2: two CTAs of 16 warps, 64 registers per thread; 0
 * keeps).  -1 if the CTA's shared memory does not fit at that occupancy. */
int trtt_b200_plan3d_set_group_shape(trtt_b200_plan3d *plan, int band_rows4, int utile4,
                                     int ctas_per_sm4);

/* shape[0..6] = nx, ny, nz, nu, nv, nviews, number of gates. */
int trtt_b200_plan3d_shape(const trtt_b200_plan3d *plan, long *shape);

int trtt_b200_plan3d_destroy(trtt_b200_plan3d *plan);

typedef struct trtt_b200_plan2d trtt_b200_plan2d;

/* 2D B-spline projector plan (trtt_PB2D/FB2D geometry and footprint
 * semantics, plugin/trtt_2D_projectors.c:186-383) for `nviews` views;
 * cum_footprint == NULL selects the closed-form cubic footprint
 * (trtt_PB2D_cubic/trtt_FB2D_cubic). */
int trtt_b200_plan2d_create(trtt_b200_plan2d **plan, int geometry, long nx, long ny,
                            double s_scl, int s_deg, const double *cum_footprint,
                            long size_footprint, double step_footprint,
                            const double *coord_footprint, long nv, double v_scl,
                            long nviews, const double *xos, const double *xsd);

/* Long-Fessler plan: `params` is a trtt_b200_lf2d_parameters block, one
 * (beta, detector offset) pair per view (LongFessler2D.c:41-470). */
int trtt_b200_plan2d_create_lf(trtt_b200_plan2d **plan, const void *params,
                               int line_integ, long nviews, const double *beta,
                               const double *offset);

/* sino[view][nv] += H img  /  img += H^T sino  (img is [j][i], nx fastest). */
int trtt_b200_plan2d_forward(trtt_b200_plan2d *plan, const float *img, float *sino,
                             void *stream);
int trtt_b200_plan2d_backward(trtt_b200_plan2d *plan, const float *sino, float *img,
                              void *stream);
int trtt_b200_plan2d_status(trtt_b200_plan2d *plan, void *stream);

/* GPU assembly of the per-view sparse system matrices as 1-based COO
 * triplets (the matrix the reference builds column by column with the
 * sparsers, Ytrtt_2D_projectors.i:212-369).  Device arrays of
 * nviews*nx*ny*max_cells entries; slot ((view*nx*ny)+pixel)*max_cells+l;
 * unused slots have row = col = 0. */
int trtt_b200_plan2d_assemble(trtt_b200_plan2d *plan, int max_cells, double *a,
                              long *rows, long *cols, void *stream);

/* y (+)= A x for a sparse matrix in compressed rows (device arrays, FP64,
 * 0-based column indices): the sparse-product mode of the 2D projectors
 * (the matrix of trtt_b200_plan2d_assemble once sorted into rows, for H or
 * for H^T), which the reference evaluates with trtt_mvmult
 * (plugin/trtt_common.c:62-69; Tomography_2D/Ytrtt2D_optim.i:320-387).
 * row_ptr has nrows + 1 entries; accumulate == 0 overwrites y.  Entries with
 * a column index outside [0, ncols) are skipped and flagged; asynchronous on
 * `stream`.  csr_status synchronises `stream` and returns -1 (clearing the
 * flag) if a product since the last call skipped an entry. */
int trtt_b200_csr_spmv(const long *row_ptr, const long *col, const double *val, long nrows,
                       long ncols, const double *x, double *y, int accumulate, void *stream);
int trtt_b200_csr_status(void *stream);

int trtt_b200_plan2d_destroy(trtt_b200_plan2d *plan);

/* Distance-driven 2D projector pair (the reference's Yorick evaluators
 * _trtt_single_distance_driven_{PB,FB}2D_projector, Ytrtt_2D_projectors.i:
 * 943-1245) on host FP64 arrays for `nviews` views, accumulating into out:
 * job 0: out(detector [view][nv]) += H in(image [ny][nx]); job 1:
 * out(image) += H^T in(detector).  xos / xsd are nviews*12 coefficients of
 * each view's (xos . xotilt) and xsd transforms, in millimetres (the
 * distance-driven evaluator does not fold in the pixel and cell transforms,
 * :868-880).  geometry: TRTT_B200_PARALLEL_BEAM, or TRTT_B200_FAN_BEAM /
 * TRTT_B200_CONE_BEAM (fan).  Returns -1 (out unchanged) if a fan-beam point
 * lies in the source plane, as the reference raises an error there. */
int trtt_b200_dd2d(double *out, const double *in, long nx, long ny, double s_scl, long nv,
                   double v_scl, long nviews, const double *xos, const double *xsd,
                   int geometry, int job);

/* Batched host-buffer entry point: the whole scan in one call.  Same
 * conventions as trtt_CB3D/trtt_CB3D_cubic (host double*, accumulate,
 * reference layouts) for `nviews` views: xos/xsd are nviews*12, the
 * detector array is [view][nv][nu].  job 0: out(detector) += H in(volume);
 * job != 0: out(volume) += H^T in(detector). */
int trtt_b200_cb3d_batch(double *out, const double *in, long nx, long ny,
                         long nz, double s_scl, int s_deg,
                         const double *cum_footprint, long size_footprint,
                         double step_footprint, const double *coord_footprint,
                         long nu, long nv, double u_scl, double v_scl,
                         long nviews, const double *xos, const double *xsd,
                         int geometry, int job);

/* Same call with a choice of accumulation: accumulate != 0 is
 * trtt_b200_cb3d_batch (out += ...); accumulate == 0 overwrites out with
 * the projection (out = H in / out = H^T in): the host array is only
 * written, so it need not be cleared nor copied to the device. */
int trtt_b200_cb3d_batch_ex(double *out, const double *in, long nx, long ny,
                            long nz, double s_scl, int s_deg,
                            const double *cum_footprint, long size_footprint,
                            double step_footprint, const double *coord_footprint,
                            long nu, long nv, double u_scl, double v_scl,
                            long nviews, const double *xos, const double *xsd,
                            int geometry, int job, int accumulate);

/* Reconstruction helpers (device pointers, FP32 data, FP64 scalars).  The
 * FP64 results are ADDED into *f_dev / *out_dev (device scalars), so several
 * terms can be summed before one read-back.
 * wls_residual: wr = w*(hx - y) (w may be NULL: unit weights) and
 *   f += 1/2 sum w (hx - y)^2, the data term of Tomography_3D/Ytrtt3D_optim.i:186-201.
 * dot: out += sum a*b accumulated in FP64.
 * tv: isotropic smoothed total variation of z ([nz][ny][nx], nz = 1 in 2D),
 *   f += mu * sum (sqrt(|grad z|^2 + eps^2) - eps), g += mu * dTV/dz.
 * spline_sample: z = S x, the cubic B-spline coefficients x sampled at the
 *   voxel centres (separable [1/6, 2/3, 1/6], zero outside); S is symmetric
 *   so the same call applies S^T.  tmp: scratch of the same size. */
int trtt_b200_wls_residual(const float *hx, const float *y, const float *w, float *wr, long n,
                           double *f_dev, void *stream);
int trtt_b200_dot(const float *a, const float *b, long n, double *out_dev, void *stream);
int trtt_b200_tv(const float *z, long nx, long ny, long nz, double eps, double mu, float *g,
                 double *f_dev, void *stream);
int trtt_b200_spline_sample(const float *x, float *z, float *tmp, long nx, long ny, long nz,
                            void *stream);

/* Native regularised reconstruction on a 3D plan (one volume, no gates):
 * minimise 1/2 (Hx - y)' W (Hx - y) + mu TV(S x) (w may be NULL: W = I;
 * TV and S as in trtt_b200_tv / trtt_b200_spline_sample) under
 * lower <= x <= upper (+-HUGE_VAL: no bound) by VMLM-B with `mem` pairs,
 * projected Armijo backtracking (at most 30 trials) and the stopping rule
 * |f_k - f_k+1| <= frtol max(|f_k|, |f_k+1|), at most maxiter iterations.
 * The cost is that of Tomography_3D/Ytrtt3D_optim.i:128-234, minimised
 * there by OptimPack's op_mnb (Tomography_3D/Ytrtt3D_optim.i:663).
 * x (device, `layout`) holds the start and receives the result; y, w are
 * device detector stacks [view][nv][nu].  f_hist / t_hist (host, may be
 * NULL) receive maxiter + 1 objective values / wall-clock seconds since the
 * start (entry k after iteration k).  info->converged: 1 stopping rule met,
 * 2 zero projected gradient, 0 iteration limit, -1 line search failed.
 * Work buffers (2 mem + 14 volumes and 2 detector stacks) are allocated on
 * the first call and kept for later calls with the same sizes on the same
 * device (a reconstruction loop over many data sets then allocates once);
 * a call with other sizes frees and reallocates them.  Calls are
 * serialised by a process-wide lock. */
typedef struct {
  int iterations, evaluations, converged;
  double f_first, f_last, seconds;
} trtt_b200_vmlmb_info;
int trtt_b200_recon3d(trtt_b200_plan3d *plan, const float *y, const float *w, float *x, int layout,
                      double mu, double eps, double lower, double upper, int mem, int maxiter,
                      double frtol, double *f_hist, double *t_hist, trtt_b200_vmlmb_info *info,
                      void *stream);

/* View-sharded reconstruction, the B200 form of the reference's MPY view
 * split (Tomography_3D/Ytrtt3D_optim.i:48-124): one process per GPU, each
 * with a plan of its own block of views (and its y, w); every rank runs the
 * same iteration on a resident copy of the volume.  Per evaluation the
 * ranks' data-term gradients (FP32 volume) and objectives (one FP64) are
 * summed by `allreduce` (the regulariser is added by rank 0 only); the
 * FP64 scalars the iteration branches on are averaged the same way, so all
 * ranks take the same decisions.  allreduce(ctx, buf, count, dtype, stream)
 * sums `count` device values in place over the ranks (dtype 0: float, 1:
 * double) ordered on `stream`, and returns 0 (non-zero: the solve fails
 * with -1).  world == 1 is trtt_b200_recon3d.  No counterpart in the
 * reference's C. */
typedef int (*trtt_b200_allreduce_fn)(void *ctx, void *buf, long count, int dtype, void *stream);
int trtt_b200_recon3d_sharded(trtt_b200_plan3d *plan, const float *y, const float *w, float *x,
                              int layout, double mu, double eps, double lower, double upper,
                              int mem, int maxiter, double frtol, double *f_hist, double *t_hist,
                              trtt_b200_vmlmb_info *info, void *stream, int rank, int world,
                              trtt_b200_allreduce_fn allreduce, void *ctx);

/* Allocation-free cone-beam direct projector.  No counterpart in the
 * reference (whose plugin allocates on the host per voxel).  For callers that
 * cannot call cudaMalloc: real-time or embedded hosts that forbid device
 * allocation after start-up (cudaMalloc may synchronise the device), and
 * frameworks whose device memory belongs to their own pool allocator.  Same
 * sizes accepted and same result as trtt_b200_plan3d_forward with the closed-form cubic footprint and
 * TRTT_B200_LAYOUT_COLUMNS: sino[view][nv][nu] += H_view vol_columns for
 * nviews cone-beam views (xos/xsd: host, nviews*12).  vol_columns and sino are
 * device arrays owned by the caller.  The per-view geometry lives in one
 * static device array of TRTT_B200_NOALLOC_MAX_VIEWS records (688,384 bytes,
 * held by every GPU that loads the library until exit); more views return -1.
 * Every call reuses that array, so calls overlapping on the GPU race; host
 * threads are serialised and the call returns after the projection has
 * completed (it waits for `stream`).  The first call on a device looks the array up
 * (cudaGetSymbolAddress): make it before any stream capture. */
#define TRTT_B200_NOALLOC_MAX_VIEWS 2048
int trtt_b200_cb3d_cubic_forward_noalloc(const float *vol_columns, float *sino,
                                         long nx, long ny, long nz, double s_scl,
                                         int s_deg, long nu, long nv, double u_scl,
                                         double v_scl, long nviews,
                                         const double *xos, const double *xsd,
                                         void *stream);

/* Learned warm start: building blocks of a 3D U-Net on the sm_100a tensor
 * cores.  No counterpart in the reference (its reconstructions start from
 * zero, Tomography_3D/Ytrtt3D_optim.i:663).  All arrays are device arrays.
 *
 * Activation layout: a batch of nb volumes of d x h x w voxels with C BF16
 * channels is stored "padded channels-last": nb (d+2)(h+2)(w+2) rows of C
 * values, row ((v (d+2) + z)(h+2) + y)(w+2) + x, interior z in 1..d, y in
 * 1..h, x in 1..w.  The one-voxel border must be zero; no call writes it.
 *
 * conv3_pack: FP32 weights w[cout][27][cin] (tap = 9 (dz+1) + 3 (dy+1) +
 *   (dx+1)) -> BF16 operand tiles.  transpose = 0: the forward operand
 *   (27 * roundup16(cout) * cin values); transpose = 1: the input-gradient
 *   operand (weights transposed and flipped, 27 * cin * roundup16(cout)).
 *   cin must be a multiple of 16.
 * conv3_forward: 3x3x3 convolution, zero padding, of the channels of x1
 *   (c1) followed by those of x2 (c2; x2 may be NULL with c2 = 0), c1, c2
 *   multiples of 16, into n output channels (multiple of 16, <= 256) with the
 *   packed weights of conv3_pack.  mode 0: y = act(conv + bias) as BF16
 *   [rows][n], act(v) = v > 0 ? v : slope v; mode 1: the same in FP32;
 *   mode 2: y[p] = resid[p] + conv[p][0] + bias[0] (FP32, one channel;
 *   resid and y padded FP32 [rows]); mode 3 (gradients): output channels
 *   [0, n1) go to y ([rows][n1]) and [n1, n) to y2 ([rows][n - n1]), BF16,
 *   added to the present values when accumulate != 0, no bias/activation.
 * conv3_wgrad: dw[cout][27][cin] = sum over rows of dy[row][co] *
 *   x[row + off(tap)][ci] (x = x1 channels then x2 channels), db[co] =
 *   sum dy[row][co] (db may be NULL).  cout in {16, 32, 48, 64}, cin =
 *   c1 + c2 a multiple of 16 with 3 cin <= 512.  scratch: device buffer of
 *   at least conv3_wgrad_scratch() bytes.
 * unet_resample: between a fine grid (d, h, w even) and the coarse grid
 *   (d/2, h/2, w/2), C channels (multiple of 8): mode 0 coarse = mean of the
 *   2x2x2 children, 1 children (+)= coarse / 8, 2 children = coarse (nearest
 *   upsampling), 3 coarse (+)= sum of children; (+)= when accumulate != 0.
 * unet_act_grad: g *= (y > 0 ? 1 : slope), rows x C BF16 values.
 * unet_pad_input: dense FP32 x[nb][d][h][w] -> xb ([rows][16] BF16,
 *   channel 0 = scale x) and xf ([rows] FP32 = scale x; may be NULL).
 * unet_unpad: padded FP32 [rows] -> dense FP32 times scale.
 * unet_mse: *loss += mean over voxels of (out - scale target)^2 (FP64) and,
 *   if dout is not NULL, dout[row][0] = its derivative (BF16 [rows][16]).
 * unet_add_output_grad: dout[row][0] += coef g for a dense FP32 g[nb][d][h][w]
 *   (an extra loss term on the network output).
 * adam: Adam step number `step` (>= 1) with decoupled-free L2 term
 *   weight_decay * w added to the gradient.
 * unet_status: -1 if a convolution kernel gave up waiting for its tensor-core
 *   work (bounded waits), then clears the flag; synchronises the stream. */
int trtt_b200_conv3_pack(const float *w, int cout, int cin, int transpose, void *wpack, void *stream);
/* Staging of trtt_b200_conv3_forward, process-wide: 0 copies each stage's
 * slab and weights into shared memory with 16-byte cp.async by all 128
 * threads; 1 loads them with TMA (2D tiled copies of the padded
 * channels-last activations, a bulk copy of the weights) issued by one
 * producer thread while one thread issues the MMAs on an mbarrier ring
 * (warp specialisation), one tile per CTA; 2 is the same in persistent
 * CTAs of 6 warps that walk many tiles with two tensor-memory accumulators,
 * the epilogue of one tile (4 warps) overlapping the copies and MMAs of the
 * next (needs 2 x 2 x n <= 512 tensor-memory columns; else 1).  All
 * compute the same MMAs in the same order (identical results).  Forward
 * pass of the 128^3 U-Net: 1.73 ms (0), 1.37 ms (1), 1.03 ms (2).  The
 * weight gradient follows the same switch: 0 stages with cp.async, any
 * other value with TMA and a producer / MMA-issuer pair (same MMAs; a
 * training step of the 128^3 U-Net 8.6 ms with 0, 5.4 ms with TMA).
 * Default (on < 0): 2 when the driver provides a tensor-map encoder, else
 * 0.  -1 when asked for TMA without one.  No counterpart in the reference. */
int trtt_b200_conv3_set_tma(int on);
int trtt_b200_conv3_forward(const void *x1, int c1, const void *x2, int c2, const void *wpack, int n,
                            const float *bias, int mode, float slope, void *y, void *y2, int n1,
                            int accumulate, const float *resid, int nb, int d, int h, int w,
                            void *stream);
size_t trtt_b200_conv3_wgrad_scratch(int cout, int cin, int nb, int d, int h, int w);
/* Shared-memory plan the convolution kernels use for a shape (host only, no
 * GPU needed; for checks of the staging arithmetic).  which = 0: forward /
 * input-gradient kernel with cin input and cout output channels, info[0..7]
 * = sub-tiles S, slab rows, chunk stride, stage bytes, stages, dynamic shared
 * memory, tensor-memory columns, tiles.  which = 1: weight gradient,
 * info[0..9] = rows per stage, A and B chunk strides, A and B region bytes,
 * stages, dynamic shared memory, tensor-memory columns, row chunks, stages
 * per chunk.  which = 0 and 1 describe the cp.async staging; which = 2 the
 * persistent TMA forward kernel (layout of 0), which = 3 the TMA weight
 * gradient (layout of 1). */
int trtt_b200_conv3_plan_info(int which, int cin, int cout, int nb, int d, int h, int w, long *info);
int trtt_b200_conv3_wgrad(const void *dy, int cout, const void *x1, int c1, const void *x2, int c2,
                          float *dw, float *db, void *scratch, size_t scratch_bytes, int nb, int d,
                          int h, int w, void *stream);
int trtt_b200_unet_resample(void *fine, void *coarse, int c, int nb, int d, int h, int w, int mode,
                            int accumulate, void *stream);
int trtt_b200_unet_act_grad(void *g, const void *y, long rows, int c, float slope, void *stream);
int trtt_b200_unet_pad_input(const float *x, void *xb, float *xf, float scale, int nb, int d, int h,
                             int w, void *stream);
int trtt_b200_unet_unpad(const float *xf, float *x, float scale, int nb, int d, int h, int w,
                         void *stream);
int trtt_b200_unet_mse(const float *out, const float *target, void *dout, float scale, double *loss,
                       int nb, int d, int h, int w, void *stream);
int trtt_b200_unet_add_output_grad(void *dout, const float *g, float coef, int nb, int d, int h, int w,
                                   void *stream);
int trtt_b200_adam(float *w, const float *g, float *m, float *v, long n, float lr, float b1, float b2,
                   float eps, int step, float weight_decay, void *stream);
int trtt_b200_unet_status(void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TRTT_B200_H */
