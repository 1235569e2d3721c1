/*
 * trtt_oracle.h -- FP64 CPU restatement of the TRTT projector plugin.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * B200 kernels: tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py may call it; the product (yoricktrtt_b200) never links or calls
 * it.  Every routine keeps the signature of the reference routine it
 * restates (prefix orc_ instead of trtt_/lf2d_), the same argument meaning,
 * the same accumulate-into-out semantics and the same 0/-1 return codes.
 *
 * The arithmetic follows the reference operation by operation (same
 * operand order, no fused multiply-add) so that, compiled with
 * -ffp-contract=off, results are bit-identical to the reference plugin built
 * from its own sources (oracle/_ref).  Pinned by tests/test_oracle_pin.py.
 */
#ifndef TRTT_ORACLE_H
#define TRTT_ORACLE_H 1

#ifdef __cplusplus
extern "C" {
#endif

/* plugin/trtt_common.c:62-69 */
int orc_mvmult(double *out, double *in, long number, double *a, long *i, long *j);

/* plugin/trtt_2D_projectors.c:186-383 (table footprint) */
int orc_PB2D(double *out, double *in, long nx, long ny, double s_scl, int s_deg,
             double *footprint, double *cum_footprint, long size_footprint,
             double step_footprint, double *coord_footprint, long nv,
             double v_scl, double *xos, double *xsd, int job);
int orc_FB2D(double *out, double *in, long nx, long ny, double s_scl, int s_deg,
             double *footprint, double *cum_footprint, long size_footprint,
             double step_footprint, double *coord_footprint, long nv,
             double v_scl, double *xos, double *xsd, int job);
/* plugin/trtt_2D_projectors.c:393-536 */
int orc_PB2D_sparser(double *out, long i, long j, long nx, long ny, double s_scl,
                     int s_deg, double *footprint, double *cum_footprint,
                     long size_footprint, double step_footprint,
                     double *coord_footprint, long nv, double v_scl,
                     double *xos, double *xsd);
int orc_FB2D_sparser(double *out, long i, long j, long nx, long ny, double s_scl,
                     int s_deg, double *footprint, double *cum_footprint,
                     long size_footprint, double step_footprint,
                     double *coord_footprint, long nv, double v_scl,
                     double *xos, double *xsd);
/* plugin/trtt_2D_projectors_cubic.c:209-398 (closed-form cubic footprint) */
int orc_PB2D_cubic(double *out, double *in, long nx, long ny, double s_scl,
                   int s_deg, long nv, double v_scl, double *xos, double *xsd,
                   int job);
int orc_FB2D_cubic(double *out, double *in, long nx, long ny, double s_scl,
                   int s_deg, long nv, double v_scl, double *xos, double *xsd,
                   int job);

/* plugin/trtt_3D_projectors.c:959-1338 */
int orc_PB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
             int s_deg, double *footprint, double *cum_footprint,
             long size_footprint, double step_footprint, double *coord_footprint,
             long nu, long nv, double u_scl, double v_scl, double *xos,
             double *xsd, int job);
int orc_CB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
             int s_deg, double *footprint, double *cum_footprint,
             long size_footprint, double step_footprint, double *coord_footprint,
             long nu, long nv, double u_scl, double v_scl, double *xos,
             double *xsd, int job);
int orc_DD_PB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
                long nu, long nv, double u_scl, double v_scl, double *xos,
                double *xsd, int job);
/* Cone-beam distance-driven pair: the reference's unfinished trtt_DD_CB3D
 * (plugin/trtt_3D_projectors.c:1340-1434) completed with its intent. */
int orc_DD_CB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
                long nu, long nv, double u_scl, double v_scl, double *xos,
                double *xsd, int job);
/* plugin/trtt_3D_projectors_cubic.c:506-778 */
int orc_PB3D_cubic(double *out, double *in, long nx, long ny, long nz,
                   double s_scl, int s_deg, long nu, long nv, double u_scl,
                   double v_scl, double *xos, double *xsd, int job);
int orc_CB3D_cubic(double *out, double *in, long nx, long ny, long nz,
                   double s_scl, int s_deg, long nu, long nv, double u_scl,
                   double v_scl, double *xos, double *xsd, int job);

/* tomography-LongFessler-model/LongFessler2D.h:16-28 (same field order) */
typedef struct {
  double pixelSize, pixelStep, voxelSize, sourceDistance, detectorDistance;
  double objectOffset1, objectOffset2;
  long objectDimension1, objectDimension2, detectorDimension;
} orc_lf2d_parameters;

/* tomography-LongFessler-model/LongFessler2D.c:41-681 */
void orc_lf2d_direct(const orc_lf2d_parameters *p, double beta, double offset,
                     const double voxel[], double pixel[], int clr);
void orc_lf2d_line_integ_direct(const orc_lf2d_parameters *p, double beta,
                                double offset, const double voxel[],
                                double pixel[], int clr);
void orc_lf2d_adjoint(const orc_lf2d_parameters *p, double beta, double offset,
                      const double pixel[], double voxel[], int clr);
void orc_lf2d_line_integ_adjoint(const orc_lf2d_parameters *p, double beta,
                                 double offset, const double pixel[],
                                 double voxel[], int clr);
void orc_lf2d_sparser(const orc_lf2d_parameters *p, double beta, double offset,
                      long i1, long i2, double pixel[], int clr);
void orc_lf2d_line_integ_sparser(const orc_lf2d_parameters *p, double beta,
                                 double offset, long i1, long i2,
                                 double pixel[], int clr);

/* Footprint table of a degree-DEG B-spline sampled on M points, restating
 * Ytrtt_tomobj.i:140-196 (_monodim_bspline + _cumsum).  Writes
 * footprint[m], cum[m], coord[m] and returns the sampling step. */
double orc_footprint_table(int deg, long m, double *footprint, double *cum,
                           double *coord);

#ifdef __cplusplus
}
#endif
#endif /* TRTT_ORACLE_H */
