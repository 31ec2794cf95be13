/*
 * rmhd2d_oracle.h -- CPU restatement of the reference's 2D resistive-MHD RK2
 * step.  TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path,
 * never linked into the product.  See rmhd2d_oracle.c for the reference
 * file:line each function restates.
 */
#ifndef RMHD2D_ORACLE_H
#define RMHD2D_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_BC_PERIODIC = 0, ORC_BC_SYMMETRIC = 1, ORC_BC_ZERO_GRADIENT = 2, ORC_BC_WALL = 3, ORC_BC_FLARE = 4 };

typedef struct {
    int nx, ny;               /* cells per direction, 3 ghost layers per side included */
    double dx, dy;
    double gamma;             /* gamma_mhd */
    double cfl;               /* CFL */
    double eps;               /* EPS regulariser */
    double eta;               /* scalar eta: resistive term when eta_table is NULL, and dt limit */
    const double *eta_table;  /* optional cell-centred eta, k = j + i*ny */
    int bc;                   /* x boundary: ORC_BC_PERIODIC, _SYMMETRIC, _ZERO_GRADIENT or _FLARE */
    int bc_y;                 /* y boundary, or -1 for the same as bc */
    int ct_contact;           /* 0: the step's CT with the stage-1 EMF; 1: CT-Contact EMF (orc_step_contact) */
} orc_params;

double orc_calc_dt(const orc_params *p, const double *U);
int orc_is_crashed(const orc_params *p, const double *U);
void orc_boundary(const orc_params *p, double *U);
size_t orc_work_doubles(int nx, int ny);
double orc_step(const orc_params *p, double *U, double *work);
double orc_step_contact(const orc_params *p, double *U, double *work);
size_t orc_contact_ct_work_doubles(int nx, int ny);
void orc_contact_ct(const orc_params *p, const double *Uold, const double *Fold, const double *Gold,
                    const double *Fnow, const double *Gnow, const double *bXOld, const double *bYOld, double dt,
                    double *U, double *work);
int orc_run(const orc_params *p, double *U, int nsteps, double *dts);
int orc_run_keep_stages(const orc_params *p, double *U, int nsteps, double *dts, double *Un, double *Ustar);

#ifdef __cplusplus
}
#endif
#endif
