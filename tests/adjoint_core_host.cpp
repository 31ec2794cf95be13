// Host build of the per-interface reverse-mode functions of the CUDA
// adjoint (resistivemhd_gpu_b200/csrc/adjoint_core.cuh), for the CPU
// dot-product tests in test_adjoint_core.py.
#include "../resistivemhd_gpu_b200/csrc/adjoint_core.cuh"

extern "C" {

void host_hlld_flux_adj(const double *L, const double *R, double gm, double eps, const double *fb, double *Lb,
                        double *Rb)
{
    for (int c = 0; c < 8; ++c) { Lb[c] = 0.0; Rb[c] = 0.0; }
    rmhd2d::adj::hlld_flux_adj(L, R, gm, eps, fb, Lb, Rb);
}

void host_basic_param(const double *c, double bn_next, double gm, double *q)
{
    rmhd2d::adj::basic_param(c, bn_next, gm, q);
}

void host_basic_param_adj(const double *c, double gm, const double *qb, double *cb)
{
    for (int k = 0; k < 8; ++k) cb[k] = 0.0;
    double q[8];
    rmhd2d::adj::basic_param(c, 0.3, gm, q);
    rmhd2d::adj::basic_param_adj(q, c[4], gm, qb, cb);
}

unsigned host_muscl_states(const double *q0, const double *q1, const double *q2, const double *q3, double eps,
                           double *L, double *R)
{
    return rmhd2d::adj::muscl_states(q0, q1, q2, q3, eps, L, R);
}

}
