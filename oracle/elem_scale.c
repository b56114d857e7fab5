/*
 * Per-element integrand scaling s_e for the reference's own CPU callbacks
 * (test infrastructure: the oracle of the adjoint tests, never shipped).
 *
 * The reference's residual and tangent loops call phys->residual
 * (src/snesiga_Residual.c:146) and phys->tangent (src/snesiga_Tangent.c:146)
 * once per Gauss point, 4x4x4 points per element, elements in x, y, z loop
 * order (src/snesiga_Residual.c:104-106).  Wrapping those two function
 * pointers with a call counter therefore knows the element index
 * e = count / 64 and can multiply the integrand output by s_e, which scales
 * the element's whole volume contribution -- without editing the reference.
 * The counter is reset before every callback by oracle_scale_reset().
 */
#include <stddef.h>
#include "iga.h"

static residual_ptr base_residual = NULL;
static tangent_ptr base_tangent = NULL;
static const double *scale = NULL;
static long n_elem = 0, n_call = 0, n_overflow = 0;
static int n_out = 30, n_tan = 900;

static double scale_of_call(void)
{
    long e = n_call++ / 64;
    if (e >= n_elem) {
        n_overflow++;
        return 1.0;
    }
    return scale[e];
}

static void scaled_residual(double *r, double *u, double *par)
{
    base_residual(r, u, par);
    double s = scale_of_call();
    for (int i = 0; i < n_out; i++) r[i] *= s;
}

static void scaled_tangent(double *t, double *u, double *par)
{
    base_tangent(t, u, par);
    double s = scale_of_call();
    for (int i = 0; i < n_tan; i++) t[i] *= s;
}

/* s: [n] element scales (kept by pointer); app: the IGA of a case */
void oracle_scale_install(void *app, const double *s, long n)
{
    Phys *p = ((IGA *)app)->phys;
    if (p->residual != scaled_residual) base_residual = p->residual;
    if (p->tangent != scaled_tangent) base_tangent = p->tangent;
    n_out = p->ndof * 10;
    n_tan = n_out * n_out;
    scale = s;
    n_elem = n;
    p->residual = scaled_residual;
    p->tangent = scaled_tangent;
    n_call = 0;
    n_overflow = 0;
}

void oracle_scale_remove(void *app)
{
    Phys *p = ((IGA *)app)->phys;
    if (p->residual == scaled_residual) p->residual = base_residual;
    if (p->tangent == scaled_tangent) p->tangent = base_tangent;
    scale = NULL;
    n_elem = 0;
}

void oracle_scale_reset(void) { n_call = 0; }

/* calls seen since the last reset, and calls past the last element (must be 0) */
long oracle_scale_calls(void) { return n_call; }
long oracle_scale_overflow(void) { return n_overflow; }
