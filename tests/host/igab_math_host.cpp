// Host build of the product's point mathematics (igab_math.cuh) for CPU tests.
#include <cstring>
#include "igab_math.cuh"

extern "C" void host_ge_point(const double *u, const double *par, double *r, double *D27)
{
    igab_ge_coef c = igab_ge_coef_from_par(par);
    igab_ge_point<double> P;
    igab_ge_eval(u, c, P);
    igab_ge_residual(P, r);
    double D[27][27];
    igab_ge_dense_tangent(P, D);
    memcpy(D27, D, sizeof(D));
}

extern "C" void host_bspline_p2(const double *kv6, double x, double *out9)
{
    double o[3][3];
    igab_bspline_p2(kv6, x, o);
    memcpy(out9, o, sizeof(o));
}

extern "C" void host_getime_point(const double *u90, const double *par, double *r, double *D27)
{
    igab_ge_coef c = igab_ge_coef_from_par(par);
    igab_getime_residual(u90, u90 + 30, u90 + 60, c, par[5], par[6], par[7], r);
    static double D[27][27];
    igab_getime_dense_tangent(u90, u90 + 30, u90 + 60, c, D);
    memcpy(D27, D, sizeof(D));
}
