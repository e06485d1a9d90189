/*
 * Stand-in for the einspline interface used by the reference's diagnostics.
 *
 * TEST INFRASTRUCTURE ONLY (linked into the oracle binary under oracle/_ref,
 * never into the product library).
 *
 * einspline (an external library, no version pinned by the reference: the
 * build links ${HOME}/einspline, weno/makefileGPU:4,7,13) is absent here.  Its
 * published algorithm is a tensor-product interpolating cubic B-spline; with
 * NATURAL boundary codes every grid line carries the natural cubic spline of
 * its samples (second derivative zero at both ends).  The reference only
 * evaluates the spline AT GRID NODES (PrintStats, weno/src/update.cpp:674-685;
 * the particle path that evaluates off-node is never called), where the
 * interpolant equals the data and each partial derivative equals the node
 * slope of the 1-D natural cubic spline along that axis.  This stand-in
 * computes exactly those node values and slopes, and refuses off-node
 * evaluation.
 */
#ifndef GKS_REFSHIM_BSPLINE_H
#define GKS_REFSHIM_BSPLINE_H

typedef enum { PERIODIC, DERIV1, DERIV2, FLAT, NATURAL, ANTIPERIODIC } bc_code;

typedef struct {
    bc_code lCode, rCode;
    double lVal, rVal;
} BCtype_d;

typedef struct {
    double start, end;
    int num;
    double delta, delta_inv;
} Ugrid;

typedef struct {
    int n[3];
    double start[3], delta[3];
    double *val;     /* node values, layout [i0][i1][i2] */
    double *grad[3]; /* node slopes along axis 0, 1, 2 */
} UBspline_3d_d;

UBspline_3d_d *create_UBspline_3d_d(Ugrid g0, Ugrid g1, Ugrid g2, BCtype_d bc0, BCtype_d bc1,
                                    BCtype_d bc2, double *data);
void eval_UBspline_3d_d(UBspline_3d_d *s, double x0, double x1, double x2, double *val);
void eval_UBspline_3d_d_vg(UBspline_3d_d *s, double x0, double x1, double x2, double *val,
                           double *grad);
void destroy_Bspline(void *s);

#endif
