/*
 * C ABI of libigap4_b200 (include/igab.h): context set-up on the host, the
 * boundary-condition tables, and the assembly entry points.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <vector>
#include "igab_internal.h"

static thread_local char g_err[512] = "";

void igab_set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

extern "C" const char *igab_last_error(void) { return g_err; }
extern "C" int igab_version(void) { return 100; }

#define ARG_CHECK(cond, msg)                   \
    do {                                       \
        if (!(cond)) {                         \
            igab_set_error("%s", msg);         \
            return IGAB_ERR_ARG;               \
        }                                      \
    } while (0)

igab_geom igab_ctx::geom() const
{
    igab_geom g;
    for (int d = 0; d < 3; d++) {
        g.ne[d] = ne[d];
        g.nb[d] = nb[d];
        g.tab[d] = d_tab[d];
        g.wh[d] = d_wh[d];
        g.xq[d] = d_xq[d];
    }
    g.ndof = ndof;
    g.rowptr = d_rowptr;
    g.coef = igab_ge_coef_from_par(par_mat);
    g.periodic = 0;
    for (int i = 0; i < 9; i++) {
        g.pp[i] = par_periodic[i];
        if (par_periodic[i] != 0.0) g.periodic = 1;
    }
    g.hist1 = d_hist;
    g.hist0 = d_hist ? d_hist + ndof : nullptr;
    g.rho = par_mat[5];
    g.cii = par_mat[6];
    g.dt = par_mat[7];
    g.phys = phys;
    g.escale = escale_on ? d_escale : nullptr;
    g.tw[0] = 0.25;
    g.tw[1] = 1.0 / 6.0;
    g.tw[2] = 0.125;
    g.tw[3] = 0.0;
    g.tmass = g.dt != 0.0 ? g.rho / (g.dt * g.dt) + g.cii / (2.0 * g.dt) : 0.0;
    return g;
}

/* ----------------------------------------------------------- host B-splines */

/* k-th derivative of the degree-p basis function i at x on knot vector kv
 * (nk knots).  Same conventions as mesh/nurbs/evalN.c:7-62: the last basis
 * function is 1 at the right end of a clamped knot vector, 0/0 terms of
 * repeated knots vanish, and derivatives come from the divided-difference
 * recursion of the lower-degree functions. */
static double bsp_eval(const double *kv, int nk, int k, int i, int p, double x)
{
    if (k == 0) {
        if (i == nk - p - 2 && fabs(x - kv[nk - 1]) < 1e-15 && fabs(kv[nk - 1] - kv[nk - 2]) < 1e-15) return 1.0;
        if (p == 0) return (x >= kv[i] && kv[i + 1] > x) ? 1.0 : 0.0;
        bool left_deg = kv[i + p] == kv[i], right_deg = kv[i + p + 1] == kv[i + 1];
        if (left_deg && right_deg) return 0.0;
        if (left_deg) return (kv[i + p + 1] - x) / (kv[i + p + 1] - kv[i + 1]) * bsp_eval(kv, nk, 0, i + 1, p - 1, x);
        if (right_deg) return (x - kv[i]) / (kv[i + p] - kv[i]) * bsp_eval(kv, nk, 0, i, p - 1, x);
        return (x - kv[i]) / (kv[i + p] - kv[i]) * bsp_eval(kv, nk, 0, i, p - 1, x) +
               (kv[i + p + 1] - x) / (kv[i + p + 1] - kv[i + 1]) * bsp_eval(kv, nk, 0, i + 1, p - 1, x);
    }
    if (k > p) return 0.0;
    double a[4][4];
    a[0][0] = 1.0;
    for (int r = 1; r <= k; r++) {
        double d0 = kv[i + p - r + 1] - kv[i];
        a[r][0] = (kv[i + p - r + 1] == kv[i]) ? 0.0 : a[r - 1][0] / d0;
        for (int c = 1; c < r; c++) {
            double dc = kv[i + p + c - r + 1] - kv[i + c];
            a[r][c] = (kv[i + p + c - r + 1] == kv[i + c]) ? 0.0 : (a[r - 1][c] - a[r - 1][c - 1]) / dc;
        }
        double dr = kv[i + p + 1] - kv[i + r];
        a[r][r] = (kv[i + p + 1] == kv[i + r]) ? 0.0 : -a[r - 1][r - 1] / dr;
    }
    double s = 0.0;
    for (int j = 0; j <= k; j++) s += a[k][j] * bsp_eval(kv, nk, 0, i + j, p - k, x);
    double f = 1.0;
    for (int j = p; j > p - k; j--) f *= j;
    return s * f;
}

/* 4-point Gauss-Legendre rule on [0,1], ascending nodes (closed form of the
 * roots of P4; src/quadrature.c:381-431 computes the same rule numerically). */
static void gauss4(double x[4], double w[4])
{
    long double s65 = sqrtl(6.0L / 5.0L);
    long double r_in = sqrtl(3.0L / 7.0L - 2.0L / 7.0L * s65);
    long double r_out = sqrtl(3.0L / 7.0L + 2.0L / 7.0L * s65);
    long double w_in = (18.0L + sqrtl(30.0L)) / 36.0L;
    long double w_out = (18.0L - sqrtl(30.0L)) / 36.0L;
    x[0] = (double)((1.0L - r_out) / 2.0L); w[0] = (double)(w_out / 2.0L);
    x[1] = (double)((1.0L - r_in) / 2.0L);  w[1] = (double)(w_in / 2.0L);
    x[2] = (double)((1.0L + r_in) / 2.0L);  w[2] = (double)(w_in / 2.0L);
    x[3] = (double)((1.0L + r_out) / 2.0L); w[3] = (double)(w_out / 2.0L);
}

/* face -> (in-face dir 0, in-face dir 1, normal dir), as the switch on
 * boun/2 in src/snesiga_Residual.c:191-228 */
static void face_dirs(int face, int &d0, int &d1, int &dn)
{
    switch (face / 2) {
    case 0: d0 = 1; d1 = 2; dn = 0; break;
    case 1: d0 = 0; d1 = 2; dn = 1; break;
    default: d0 = 0; d1 = 1; dn = 2; break;
    }
}

static long cp_of(const igab_ctx *c, int face, int b0, int b1, int layer)
{
    int p[3];
    int d0, d1, dn;
    face_dirs(face, d0, d1, dn);
    p[d0] = b0; p[d1] = b1; p[dn] = layer;
    return ((long)p[0] * c->nb[1] + p[1]) * c->nb[2] + p[2];
}

static int layer_of(const igab_ctx *c, int face, int slot)
{
    int d0, d1, dn;
    face_dirs(face, d0, d1, dn);
    return (face % 2 == 0) ? slot : c->nb[dn] - 1 - slot;
}

/* Dirichlet control values of one (face, order, dof): src/iga_dirichlet.c:7-80.
 * out[nb[d0] * nb[d1]] in (i over d0, j over d1) order. */
static void dirichlet_values(const igab_ctx *c, int face, int order, int idof, std::vector<double> &out)
{
    const int p = 2;
    int d0, d1, dn;
    face_dirs(face, d0, d1, dn);
    int dims[3] = {d0, d1, dn};
    const double *par = c->par_dirichlet;
    double par_[3] = {par[3 * idof + d0], par[3 * idof + d1], par[3 * idof + dn]};
    const std::vector<double> &kn = c->knots[dn];
    int nkn = (int)kn.size();
    double Z = (face % 2 == 0) ? kn[0] : kn[nkn - 1] - 1.e-15;
    std::vector<double> d1d[2];
    for (int b = 0; b < 2; b++) {
        const std::vector<double> &kv = c->knots[dims[b]];
        int nk = (int)kv.size();
        int nbas = c->nb[dims[b]];
        d1d[b].assign(nbas, 0.0);
        double W = kv[p];
        double vec[2] = {par_[b] * W, par_[b]};
        double m[4];
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) m[2 * i + j] = bsp_eval(kv.data(), nk, i, j, p, W);
        double idet = 1. / (-(m[1] * m[2]) + m[0] * m[3]);
        double inv[4] = {idet * m[3], idet * (-m[1]), idet * (-m[2]), idet * m[0]};
        d1d[b][0] = inv[0] * vec[0] + inv[1] * vec[1];
        d1d[b][1] = inv[2] * vec[0] + inv[3] * vec[1];
        for (int i = p; i < nbas; i++) d1d[b][i] = d1d[b][i - 1] + (kv[i + p] - kv[i]) / ((double)p) * par_[b];
    }
    int n0 = c->nb[d0], n1 = c->nb[d1];
    out.assign((size_t)n0 * n1, 0.0);
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++) out[(size_t)n1 * i + j] = d1d[0][i] + d1d[1][j] + par_[2] * Z;
    if (order == 1) {
        int ib1 = (face % 2 == 0) ? 1 : c->nb[dn] - 2;
        double mval = 0.0 / bsp_eval(kn.data(), nkn, 1, ib1, p, Z);
        for (auto &v : out) v += mval;
    }
}

/* rows and values of the Dirichlet INSERT pass, last writer wins
 * (src/snesiga_Residual.c:331-409 loop order) */
static int build_dirichlet(igab_ctx *c)
{
    /* with periodic directions the rows are owned dofs: the faces of periodic directions are
     * no boundaries, and along a periodic tangential direction the face has its owned points
     * only (nbasis = nelem, mesh/nurbs/nurbs_init.c:24-39) */
    long nbo[3];
    for (int d = 0; d < 3; d++) nbo[d] = c->periodic[d] ? c->ne[d] : c->nb[d];
    const long nown = 3 * nbo[0] * nbo[1] * nbo[2];
    std::vector<double> g(nown, 0.0);
    std::vector<char> is(nown, 0);
    std::vector<double> vals;
    for (int face = 0; face < 6; face++) {
        int d0, d1, dn;
        face_dirs(face, d0, d1, dn);
        if (c->periodic[dn]) continue;
        for (int order = 0; order < 2; order++)
            for (int idof = 0; idof < 3; idof++) {
                if (c->bc_type[6 * face + 3 * order + idof] != 0) continue;
                dirichlet_values(c, face, order, idof, vals);
                int layer = layer_of(c, face, order);
                for (int i = 0; i < nbo[d0]; i++)
                    for (int j = 0; j < nbo[d1]; j++) {
                        int xyz[3];
                        xyz[d0] = i;
                        xyz[d1] = j;
                        xyz[dn] = layer;
                        long r = 3 * (((long)xyz[0] * nbo[1] + xyz[1]) * nbo[2] + xyz[2]) + idof;
                        g[r] = vals[(size_t)c->nb[d1] * i + j];
                        is[r] = 1;
                    }
            }
    }
    std::vector<int> rows;
    std::vector<double> gv;
    for (long r = 0; r < nown; r++)
        if (is[r]) { rows.push_back((int)r); gv.push_back(g[r]); }
    if (c->per) {
        c->nd = 0;   /* the local-grid kernels apply none; the owned system does */
        c->dirichlet_dirty = false;
        return igab_periodic_set_dirichlet(c, rows, gv);
    }
    /* the Dirichlet row set depends only on bc_type; values change with par_dirichlet.
     * Existing buffers are refilled in place so captured graphs stay valid. */
    if ((long)rows.size() != c->nd || !c->d_drow) {
        if (c->d_drow) { cudaFree(c->d_drow); c->d_drow = nullptr; }
        if (c->d_dg) { cudaFree(c->d_dg); c->d_dg = nullptr; }
        c->nd = (long)rows.size();
        if (c->nd > 0) {
            IGAB_CUDA_TRY(cudaMalloc((void **)&c->d_drow, rows.size() * sizeof(int)));
            IGAB_CUDA_TRY(cudaMalloc((void **)&c->d_dg, gv.size() * sizeof(double)));
        }
    }
    if (c->nd > 0) {
        IGAB_CUDA_TRY(cudaMemcpy(c->d_drow, rows.data(), rows.size() * sizeof(int), cudaMemcpyHostToDevice));
        IGAB_CUDA_TRY(cudaMemcpy(c->d_dg, gv.data(), gv.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    c->dirichlet_dirty = false;
    return 0;
}

/* Neumann combos, surface points and the per-row gather lists */
static int build_neumann(igab_ctx *c)
{
    c->combos.clear();
    long off = 0;
    for (int face = 0; face < 6; face++) {
        int d0, d1, dn;
        face_dirs(face, d0, d1, dn);
        if (c->periodic[dn]) continue;   /* no boundary (mesh/nurbs/nurbs_init.c:24-27) */
        for (int order = 0; order < 2; order++)
            for (int idof = 0; idof < 3; idof++) {
                if (c->bc_type[6 * face + 3 * order + idof] != 1) continue;
                igab_ctx::combo cb;
                cb.face = face; cb.order = order; cb.dof = idof;
                cb.ne0 = c->ne[d0]; cb.ne1 = c->ne[d1];
                cb.offset = off;
                off += (long)cb.ne0 * cb.ne1 * 16;
                c->combos.push_back(cb);
            }
    }
    c->n_neu_points = off;
    /* gather entries (dof, combo, slot, b0, b1) */
    struct ent { int dof; int4 e; };
    std::vector<ent> ents;
    for (size_t k = 0; k < c->combos.size(); k++) {
        const auto &cb = c->combos[k];
        int d0, d1, dn;
        face_dirs(cb.face, d0, d1, dn);
        int nslot = cb.order == 0 ? 1 : 2;
        for (int s = 0; s < nslot; s++) {
            int layer = layer_of(c, cb.face, s);
            for (int b0 = 0; b0 < c->nb[d0]; b0++)
                for (int b1 = 0; b1 < c->nb[d1]; b1++) {
                    ent e;
                    e.dof = (int)(3 * cp_of(c, cb.face, b0, b1, layer) + cb.dof);
                    e.e = make_int4((int)k, s, b0, b1);
                    ents.push_back(e);
                }
        }
    }
    std::stable_sort(ents.begin(), ents.end(), [](const ent &a, const ent &b) { return a.dof < b.dof; });
    std::vector<int> row_dof, ptr;
    std::vector<int4> ev;
    for (size_t i = 0; i < ents.size(); i++) {
        if (i == 0 || ents[i].dof != ents[i - 1].dof) { row_dof.push_back(ents[i].dof); ptr.push_back((int)i); }
        ev.push_back(ents[i].e);
    }
    ptr.push_back((int)ents.size());
    c->n_neu_rows = (long)row_dof.size();
    std::vector<int> info(8 * std::max<size_t>(c->combos.size(), 1), 0);
    for (size_t k = 0; k < c->combos.size(); k++) {
        const auto &cb = c->combos[k];
        int d0, d1, dn;
        face_dirs(cb.face, d0, d1, dn);
        int *ci = &info[8 * k];
        ci[0] = cb.face; ci[1] = cb.order; ci[2] = cb.dof; ci[3] = cb.ne0; ci[4] = cb.ne1;
        ci[5] = (int)(cb.offset & 0xffffffffL); ci[6] = (int)(cb.offset >> 32);
        ci[7] = d0 | (d1 << 2);
    }
    double dnz[12];
    for (int face = 0; face < 6; face++) {
        int d0, d1, dn;
        face_dirs(face, d0, d1, dn);
        const std::vector<double> &kv = c->knots[dn];
        int nk = (int)kv.size();
        double z = (face % 2 == 0) ? kv[0] : kv[nk - 1];
        for (int s = 0; s < 2; s++) dnz[2 * face + s] = bsp_eval(kv.data(), nk, 1, layer_of(c, face, s), 2, z);
    }
    if (c->n_neu_rows > 0) {
        IGAB_CUDA_TRY(cudaMalloc((void **)&c->d_neu_row, row_dof.size() * sizeof(int)));
        IGAB_CUDA_TRY(cudaMalloc((void **)&c->d_neu_ptr, ptr.size() * sizeof(int)));
        IGAB_CUDA_TRY(cudaMalloc((void **)&c->d_neu_ent, ev.size() * sizeof(int4)));
        IGAB_CUDA_TRY(cudaMemcpy(c->d_neu_row, row_dof.data(), row_dof.size() * sizeof(int), cudaMemcpyHostToDevice));
        IGAB_CUDA_TRY(cudaMemcpy(c->d_neu_ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice));
        IGAB_CUDA_TRY(cudaMemcpy(c->d_neu_ent, ev.data(), ev.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    IGAB_CUDA_TRY(cudaMalloc((void **)&c->d_combo_info, info.size() * sizeof(int)));
    IGAB_CUDA_TRY(cudaMemcpy(c->d_combo_info, info.data(), info.size() * sizeof(int), cudaMemcpyHostToDevice));
    IGAB_CUDA_TRY(cudaMalloc((void **)&c->d_dnz, sizeof(dnz)));
    IGAB_CUDA_TRY(cudaMemcpy(c->d_dnz, dnz, sizeof(dnz), cudaMemcpyHostToDevice));
    if (c->n_neu_points > 0) {
        IGAB_CUDA_TRY(cudaMalloc((void **)&c->d_hval, (size_t)c->n_neu_points * sizeof(double)));
        IGAB_CUDA_TRY(cudaMemset(c->d_hval, 0, (size_t)c->n_neu_points * sizeof(double)));
    }
    c->neumann_nonzero = false;
    return 0;
}

static void free_ctx(igab_ctx *c)
{
    for (int d = 0; d < 3; d++) {
        cudaFree(c->d_tab[d]); cudaFree(c->d_wh[d]); cudaFree(c->d_xq[d]);
    }
    cudaFree(c->d_rowptr); cudaFree(c->d_drow); cudaFree(c->d_dg);
    cudaFree(c->d_hval); cudaFree(c->d_neu_row); cudaFree(c->d_neu_ptr); cudaFree(c->d_neu_ent);
    cudaFree(c->d_dnz); cudaFree(c->d_combo_info); cudaFree(c->d_hist);
    cudaFree(c->d_U); cudaFree(c->d_R); cudaFree(c->d_vals);
    cudaFree(c->d_escale); cudaFree(c->d_lam); cudaFree(c->d_status);
    cudaFree(c->d_dens_part); cudaFree(c->d_HH);
    igab_periodic_release(c);
    igab_krylov_release(c);
    igab_newton_release(c);
    igab_mg_release(c);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    for (int k = 0; k < 6; k++)
        if (c->ev[k]) cudaEventDestroy(c->ev[k]);
    for (int k = 0; k < IGAB_MAX_SLABS; k++)
        if (c->slab_ev[k]) cudaEventDestroy(c->slab_ev[k]);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" int igab_create(const igab_mesh_desc *desc, int device, igab_ctx **out)
{
    ARG_CHECK(desc && out, "igab_create: null argument");
    *out = nullptr;
    ARG_CHECK(desc->phys == IGAB_PHYS_GE || desc->phys == IGAB_PHYS_GETIME, "igab_create: unknown physics");
    ARG_CHECK(desc->knots, "igab_create: knots missing");
    for (int d = 0; d < 3; d++) ARG_CHECK(desc->nelem[d] >= 1, "igab_create: nelem must be >= 1");
    /* the reference reads bc_type as 0 (Dirichlet) or 1 (Neumann) only (include/bc.h:6) */
    for (int i = 0; i < 36; i++)
        ARG_CHECK(desc->bc_type[i] == 0 || desc->bc_type[i] == 1, "igab_create: bc_type entries must be 0 or 1");
    for (int d = 0; d < 3; d++) {
        ARG_CHECK(desc->bc_periodic[d] == 0 || desc->bc_periodic[d] == 1, "igab_create: bc_periodic entries must be 0 or 1");
        ARG_CHECK(!desc->bc_periodic[d] || desc->nelem[d] >= 3, "igab_create: a periodic direction needs nelem >= 3");
    }
    long ncp = 1;
    for (int d = 0; d < 3; d++) ncp *= desc->nelem[d] + 2;
    ARG_CHECK(3 * ncp < 2147483647L, "igab_create: dof count exceeds int32");
    /* CSR size: per direction the number of (i,j) pairs with |i-j| <= 2 */
    long nnz = 9;
    for (int d = 0; d < 3; d++) {
        long n = desc->nelem[d] + 2;
        long pairs = n + 2 * (n - 1 > 0 ? n - 1 : 0) + 2 * (n - 2 > 0 ? n - 2 : 0);
        nnz *= pairs;
    }
    ARG_CHECK(nnz < 2147483647L, "igab_create: nonzero count exceeds int32 (PETSc AIJ index range)");
    size_t koff = 0;
    for (int d = 0; d < 3; d++) {
        int nk = desc->nelem[d] + 5;
        for (int i = 1; i < nk; i++)
            ARG_CHECK(desc->knots[koff + i] >= desc->knots[koff + i - 1], "igab_create: knots must be nondecreasing");
        koff += (size_t)nk;
    }
    IGAB_CUDA_TRY(cudaSetDevice(device));
    igab_ctx *c = new igab_ctx();
    c->device = device;
    c->phys = desc->phys;
    c->torder = desc->phys == IGAB_PHYS_GE ? 0 : 2;
    koff = 0;
    for (int d = 0; d < 3; d++) {
        c->ne[d] = desc->nelem[d];
        c->nb[d] = desc->nelem[d] + 2;
        int nk = desc->nelem[d] + 5;
        c->knots[d].assign(desc->knots + koff, desc->knots + koff + nk);
        koff += (size_t)nk;
    }
    c->ncp = ncp;
    c->ndof = 3 * ncp;
    c->nnz = nnz;
    c->nel = (long)c->ne[0] * c->ne[1] * c->ne[2];
    memcpy(c->par_mat, desc->par_mat, sizeof(c->par_mat));
    memcpy(c->par_dirichlet, desc->par_dirichlet, sizeof(c->par_dirichlet));
    memcpy(c->par_periodic, desc->par_periodic, sizeof(c->par_periodic));
    memcpy(c->bc_type, desc->bc_type, sizeof(c->bc_type));
    for (int d = 0; d < 3; d++) c->periodic[d] = desc->bc_periodic[d];

    int rc = 0;
    cudaError_t ce = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) { igab_set_error("cudaStreamCreate: %s", cudaGetErrorString(ce)); delete c; return IGAB_ERR_CUDA; }
    c->own_stream = true;

    /* row pointer of the structured AIJ pattern (src/snesiga_init.c:341-359, one rank) */
    c->rowptr_h.assign((size_t)c->ndof + 1, 0);
    {
        long acc = 0, r = 0;
        for (int x = 0; x < c->nb[0]; x++) {
            int nx = std::min(x, 2) + 1 + std::min(c->nb[0] - 1 - x, 2);
            for (int y = 0; y < c->nb[1]; y++) {
                int ny = std::min(y, 2) + 1 + std::min(c->nb[1] - 1 - y, 2);
                for (int z = 0; z < c->nb[2]; z++) {
                    int nz = std::min(z, 2) + 1 + std::min(c->nb[2] - 1 - z, 2);
                    for (int k = 0; k < 3; k++) { c->rowptr_h[r++] = (int)acc; acc += 3L * nx * ny * nz; }
                }
            }
        }
        c->rowptr_h[r] = (int)acc;
        if (acc != nnz) { igab_set_error("internal: nnz mismatch"); free_ctx(c); return IGAB_ERR_ARG; }
    }
#define TRY(call)                                                            \
    do {                                                                     \
        cudaError_t _e = (call);                                             \
        if (_e != cudaSuccess) {                                             \
            igab_set_error("%s: %s", #call, cudaGetErrorString(_e));         \
            free_ctx(c);                                                     \
            return _e == cudaErrorMemoryAllocation ? IGAB_ERR_NOMEM : IGAB_ERR_CUDA; \
        }                                                                    \
    } while (0)
    TRY(cudaMalloc((void **)&c->d_status, sizeof(int)));
    TRY(cudaMemset(c->d_status, 0, sizeof(int)));
    TRY(cudaMalloc((void **)&c->d_rowptr, c->rowptr_h.size() * sizeof(int)));
    TRY(cudaMemcpy(c->d_rowptr, c->rowptr_h.data(), c->rowptr_h.size() * sizeof(int), cudaMemcpyHostToDevice));

    gauss4(c->gauss_x, c->gauss_w);
    double *dgx = nullptr, *dgw = nullptr, *dkv = nullptr;
    TRY(cudaMalloc((void **)&dgx, 4 * sizeof(double)));
    TRY(cudaMalloc((void **)&dgw, 4 * sizeof(double)));
    TRY(cudaMemcpy(dgx, c->gauss_x, 4 * sizeof(double), cudaMemcpyHostToDevice));
    TRY(cudaMemcpy(dgw, c->gauss_w, 4 * sizeof(double), cudaMemcpyHostToDevice));
    for (int d = 0; d < 3; d++) {
        TRY(cudaMalloc((void **)&c->d_tab[d], (size_t)c->ne[d] * IGAB_TAB1D * sizeof(double)));
        TRY(cudaMalloc((void **)&c->d_wh[d], (size_t)c->ne[d] * IGAB_NQ * sizeof(double)));
        TRY(cudaMalloc((void **)&c->d_xq[d], (size_t)c->ne[d] * IGAB_NQ * sizeof(double)));
        TRY(cudaMalloc((void **)&dkv, c->knots[d].size() * sizeof(double)));
        TRY(cudaMemcpy(dkv, c->knots[d].data(), c->knots[d].size() * sizeof(double), cudaMemcpyHostToDevice));
        rc = igab_launch_basis_tables(c, d, dkv, dgx, dgw);
        TRY(cudaStreamSynchronize(c->stream));
        cudaFree(dkv);
        dkv = nullptr;
        if (rc) { free_ctx(c); return rc; }
    }
    cudaFree(dgx);
    cudaFree(dgw);
    if (c->torder > 0) {
        TRY(cudaMalloc((void **)&c->d_hist, (size_t)c->torder * c->ndof * sizeof(double)));
        TRY(cudaMemset(c->d_hist, 0, (size_t)c->torder * c->ndof * sizeof(double)));
    }
#undef TRY
    if (c->periodic[0] || c->periodic[1] || c->periodic[2]) rc = igab_periodic_build(c);
    if (!rc) rc = build_dirichlet(c);
    if (!rc) rc = build_neumann(c);
    if (rc) { free_ctx(c); return rc; }
    *out = c;
    return 0;
}

extern "C" int igab_destroy(igab_ctx *ctx)
{
    if (!ctx) return 0;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_ctx(ctx);
    return 0;
}

extern "C" int igab_sizes(const igab_ctx *ctx, long *ndof, long *nnz, long *nelem_total)
{
    ARG_CHECK(ctx, "igab_sizes: null context");
    if (ndof) *ndof = igab_periodic_ndof(ctx);
    if (nnz) *nnz = igab_periodic_nnz(ctx);
    if (nelem_total) *nelem_total = ctx->nel;
    return 0;
}

extern "C" int igab_csr_pattern(igab_ctx *ctx, int *rowptr, int *cols)
{
    ARG_CHECK(ctx, "igab_csr_pattern: null context");
    if (ctx->per) {
        const std::vector<int> &rp = igab_periodic_rowptr(ctx), &cl = igab_periodic_cols(ctx);
        if (rowptr) memcpy(rowptr, rp.data(), rp.size() * sizeof(int));
        if (cols) memcpy(cols, cl.data(), cl.size() * sizeof(int));
        return 0;
    }
    if (rowptr) memcpy(rowptr, ctx->rowptr_h.data(), ctx->rowptr_h.size() * sizeof(int));
    if (cols) {
        IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
        int *dcols = nullptr;
        IGAB_CUDA_TRY(cudaMalloc((void **)&dcols, (size_t)ctx->nnz * sizeof(int)));
        int rc = igab_launch_csr_cols(ctx, dcols);
        if (!rc) {
            cudaError_t e = cudaMemcpyAsync(cols, dcols, (size_t)ctx->nnz * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) { igab_set_error("igab_csr_pattern: %s", cudaGetErrorString(e)); rc = IGAB_ERR_CUDA; }
        }
        cudaFree(dcols);
        return rc;
    }
    return 0;
}

extern "C" long igab_csr_offset(const igab_ctx *ctx, long row, long col)
{
    if (ctx && ctx->per) {
        const long n = igab_periodic_ndof(ctx);
        if (row < 0 || col < 0 || row >= n || col >= n) return -1;
        const std::vector<int> &rp = igab_periodic_rowptr(ctx), &cl = igab_periodic_cols(ctx);
        const int *b = cl.data() + rp[(size_t)row], *e = cl.data() + rp[(size_t)row + 1];
        const int *it = std::lower_bound(b, e, (int)col);
        return it != e && *it == col ? (long)(it - cl.data()) : -1;
    }
    if (!ctx || row < 0 || col < 0 || row >= ctx->ndof || col >= ctx->ndof) return -1;
    long cp = row / 3, cq = col / 3;
    int z = (int)(cp % ctx->nb[2]), y = (int)((cp / ctx->nb[2]) % ctx->nb[1]), x = (int)(cp / ((long)ctx->nb[2] * ctx->nb[1]));
    int cz = (int)(cq % ctx->nb[2]), cy = (int)((cq / ctx->nb[2]) % ctx->nb[1]), cx = (int)(cq / ((long)ctx->nb[2] * ctx->nb[1]));
    if (abs(cx - x) > 2 || abs(cy - y) > 2 || abs(cz - z) > 2) return -1;
    int x0 = std::max(x - 2, 0);
    int y0 = std::max(y - 2, 0), y1 = std::min(y + 2, ctx->nb[1] - 1);
    int z0 = std::max(z - 2, 0), z1 = std::min(z + 2, ctx->nb[2] - 1);
    int nyb = y1 - y0 + 1, nzb = z1 - z0 + 1;
    return ctx->rowptr_h[row] + (((long)(cx - x0) * nyb + (cy - y0)) * nzb + (cz - z0)) * 3 + col % 3;
}

extern "C" int igab_set_par_mat(igab_ctx *ctx, const double par_mat[9])
{
    ARG_CHECK(ctx && par_mat, "igab_set_par_mat: null argument");
    if (memcmp(ctx->par_mat, par_mat, sizeof(ctx->par_mat)) != 0) {
        ctx->param_version++;
        ctx->sched_version++;
    }
    memcpy(ctx->par_mat, par_mat, sizeof(ctx->par_mat));
    return 0;
}

extern "C" int igab_set_par_dirichlet(igab_ctx *ctx, const double par_dirichlet[9])
{
    ARG_CHECK(ctx && par_dirichlet, "igab_set_par_dirichlet: null argument");
    if (memcmp(ctx->par_dirichlet, par_dirichlet, sizeof(ctx->par_dirichlet)) != 0) {
        memcpy(ctx->par_dirichlet, par_dirichlet, sizeof(ctx->par_dirichlet));
        ctx->sched_version++;
        IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
        IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        return build_dirichlet(ctx);
    }
    return 0;
}

extern "C" int igab_set_par_periodic(igab_ctx *ctx, const double par_periodic[9])
{
    ARG_CHECK(ctx && par_periodic, "igab_set_par_periodic: null argument");
    if (memcmp(ctx->par_periodic, par_periodic, sizeof(ctx->par_periodic)) != 0) {
        ctx->param_version++;
        ctx->sched_version++;
    }
    memcpy(ctx->par_periodic, par_periodic, sizeof(ctx->par_periodic));
    return 0;
}

extern "C" int igab_neumann_points(const igab_ctx *ctx, long *n_points, double *xyz, int *meta)
{
    ARG_CHECK(ctx && n_points, "igab_neumann_points: null argument");
    *n_points = ctx->n_neu_points;
    if (!xyz && !meta) return 0;
    long k = 0;
    for (const auto &cb : ctx->combos) {
        int d0, d1, dn;
        face_dirs(cb.face, d0, d1, dn);
        const std::vector<double> &kn = ctx->knots[dn];
        double zq = (cb.face % 2 == 0) ? kn[0] : kn[kn.size() - 1];
        for (int e0 = 0; e0 < cb.ne0; e0++)
            for (int e1 = 0; e1 < cb.ne1; e1++)
                for (int q0 = 0; q0 < 4; q0++)
                    for (int q1 = 0; q1 < 4; q1++) {
                        if (xyz) {
                            double X0 = ctx->knots[d0][e0 + 2], X1 = ctx->knots[d0][e0 + 3];
                            double Y0 = ctx->knots[d1][e1 + 2], Y1 = ctx->knots[d1][e1 + 3];
                            double xi = ctx->gauss_x[q0], eta = ctx->gauss_x[q1];
                            double *p = xyz + 3 * k;
                            p[d0] = (-xi + 1.0) * X0 + xi * X1;
                            p[d1] = (-eta + 1.0) * Y0 + eta * Y1;
                            p[dn] = zq;
                        }
                        if (meta) { meta[3 * k] = cb.face; meta[3 * k + 1] = cb.order; meta[3 * k + 2] = cb.dof; }
                        k++;
                    }
    }
    return 0;
}

extern "C" int igab_set_neumann_values(igab_ctx *ctx, const double *values)
{
    ARG_CHECK(ctx, "igab_set_neumann_values: null context");
    if (ctx->n_neu_points == 0) return 0;
    ARG_CHECK(values, "igab_set_neumann_values: null values");
    bool nz = false;
    for (long i = 0; i < ctx->n_neu_points; i++)
        if (values[i] != 0.0) { nz = true; break; }
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    /* zeros are copied too while a captured graph (which always runs the Neumann kernel) exists */
    if (nz || ctx->graph_exec || ctx->nlg)
        IGAB_CUDA_TRY(cudaMemcpyAsync(ctx->d_hval, values, (size_t)ctx->n_neu_points * sizeof(double),
                                      cudaMemcpyHostToDevice, ctx->stream));
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->neumann_nonzero = nz;
    return 0;
}

extern "C" int igab_set_history(igab_ctx *ctx, int level, const double *U, int on_device)
{
    ARG_CHECK(ctx && U, "igab_set_history: null argument");
    ARG_CHECK(level >= 1 && level <= ctx->torder, "igab_set_history: level outside 1..torder");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    double *dst = ctx->d_hist + (size_t)(level - 1) * ctx->ndof;
    if (ctx->per) {   /* owned level -> local grid (ghosts from their owners) */
        const long n = igab_periodic_ndof(ctx);
        const double *src = U;
        double *tmp = nullptr;
        if (!on_device) {
            IGAB_CUDA_TRY(cudaMallocAsync((void **)&tmp, (size_t)n * sizeof(double), ctx->stream));
            IGAB_CUDA_TRY(cudaMemcpyAsync(tmp, U, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            src = tmp;
        }
        int rc = igab_periodic_gather(ctx, src, dst);
        if (tmp) IGAB_CUDA_TRY(cudaFreeAsync(tmp, ctx->stream));
        if (!on_device) IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        return rc;
    }
    IGAB_CUDA_TRY(cudaMemcpyAsync(dst, U, (size_t)ctx->ndof * sizeof(double),
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    return 0;
}


static int ensure_buffers(igab_ctx *ctx, int prec)
{
    if (!ctx->d_U) IGAB_CUDA_TRY(cudaMalloc((void **)&ctx->d_U, (size_t)ctx->ndof * sizeof(double)));
    if (!ctx->d_R) IGAB_CUDA_TRY(cudaMalloc((void **)&ctx->d_R, (size_t)ctx->ndof * sizeof(double)));
    if (prec >= 0) {
        size_t es = prec == IGAB_PREC_FP64 ? sizeof(double) : sizeof(float);
        size_t cur = ctx->vals_prec < 0 ? 0 : (ctx->vals_prec == IGAB_PREC_FP64 ? sizeof(double) : sizeof(float));
        if (cur < es) {
            cudaFree(ctx->d_vals);
            ctx->d_vals = nullptr;
            IGAB_CUDA_TRY(cudaMalloc(&ctx->d_vals, (size_t)ctx->nnz * es));
            ctx->vals_prec = prec;
        }
    }
    return 0;
}

extern "C" int igab_device_buffers(igab_ctx *ctx, double **U_dev, double **R_dev, void **vals_dev, int prec)
{
    ARG_CHECK(ctx, "igab_device_buffers: null context");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    int rc = ensure_buffers(ctx, vals_dev ? prec : -1);
    if (rc) return rc;
    if (U_dev) *U_dev = ctx->d_U;
    if (R_dev) *R_dev = ctx->d_R;
    if (vals_dev) *vals_dev = ctx->d_vals;
    return 0;
}

extern "C" int igab_upload(igab_ctx *ctx, const double *host, double *dev, long n)
{
    ARG_CHECK(ctx && host && dev && n >= 0, "igab_upload: bad argument");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    IGAB_CUDA_TRY(cudaMemcpyAsync(dev, host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return 0;
}

extern "C" int igab_download(igab_ctx *ctx, const double *dev, double *host, long n)
{
    ARG_CHECK(ctx && host && dev && n >= 0, "igab_download: bad argument");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    IGAB_CUDA_TRY(cudaMemcpyAsync(host, dev, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return 0;
}

extern "C" int igab_staging_bytes(const igab_ctx *ctx, size_t *bytes)
{
    ARG_CHECK(ctx && bytes, "igab_staging_bytes: null argument");
    size_t b = 0;
    if (ctx->d_U) b += (size_t)ctx->ndof * sizeof(double);
    if (ctx->d_R) b += (size_t)ctx->ndof * sizeof(double);
    if (ctx->d_vals) b += (size_t)ctx->nnz * (ctx->vals_prec == IGAB_PREC_FP64 ? sizeof(double) : sizeof(float));
    *bytes = b;
    return 0;
}

extern "C" int igab_residual_device(igab_ctx *ctx, const double *U_dev, double *R_dev)
{
    ARG_CHECK(ctx && U_dev && R_dev, "igab_residual_device: null argument");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    if (ctx->per) return igab_periodic_residual(ctx, U_dev, R_dev);
    return igab_launch_residual(ctx, U_dev, R_dev);
}

extern "C" int igab_residual(igab_ctx *ctx, const double *U_host, double *R_host)
{
    ARG_CHECK(ctx && U_host && R_host, "igab_residual: null argument");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    int rc = ensure_buffers(ctx, -1);
    if (rc) return rc;
    const long n = igab_periodic_ndof(ctx);   /* the owned dofs (all of them without periodic directions) */
    IGAB_CUDA_TRY(cudaMemcpyAsync(ctx->d_U, U_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    rc = igab_residual_device(ctx, ctx->d_U, ctx->d_R);
    if (rc) return rc;
    IGAB_CUDA_TRY(cudaMemcpyAsync(R_host, ctx->d_R, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (long i = 0; i < n; i++)
        if (!isfinite(R_host[i])) { igab_set_error("igab_residual: non-finite entry at %ld", i); return IGAB_ERR_NONFINITE; }
    return 0;
}

extern "C" int igab_tangent_device(igab_ctx *ctx, const double *U_dev, void *vals_dev, int prec)
{
    ARG_CHECK(ctx && U_dev && vals_dev, "igab_tangent_device: null argument");
    ARG_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_tangent_device: bad precision");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    if (ctx->per) return igab_periodic_tangent(ctx, U_dev, vals_dev, prec);
    return igab_launch_tangent(ctx, U_dev, vals_dev, prec);
}

extern "C" int igab_tangent(igab_ctx *ctx, const double *U_host, void *vals_host, int prec)
{
    ARG_CHECK(ctx && U_host && vals_host, "igab_tangent: null argument");
    ARG_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_tangent: bad precision");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    int rc = ensure_buffers(ctx, prec);
    if (rc) return rc;
    if (ctx->per) {   /* owned system: one pass, one download */
        const long n = igab_periodic_ndof(ctx), nnz = igab_periodic_nnz(ctx);
        const size_t es = prec == IGAB_PREC_FP64 ? sizeof(double) : sizeof(float);
        IGAB_CUDA_TRY(cudaMemcpyAsync(ctx->d_U, U_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        if ((rc = igab_periodic_tangent(ctx, ctx->d_U, ctx->d_vals, prec))) return rc;
        int fin = 1;
        if ((rc = igab_launch_check_finite(ctx, ctx->d_vals, nnz, prec, &fin))) return rc;
        IGAB_CUDA_TRY(cudaMemcpyAsync(vals_host, ctx->d_vals, (size_t)nnz * es, cudaMemcpyDeviceToHost, ctx->stream));
        IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if ((rc = igab_check_status(ctx))) return rc;
        if (!fin) { igab_set_error("igab_tangent: non-finite entry"); return IGAB_ERR_NONFINITE; }
        return 0;
    }
    if (!ctx->copy_stream) IGAB_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    IGAB_CUDA_TRY(cudaMemcpyAsync(ctx->d_U, U_host, (size_t)ctx->ndof * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    /* x-slab by x-slab: the rows a slab finishes are downloaded on the copy stream while
     * the next slabs are assembled (the values are the same as one whole-mesh pass) */
    long row_end[IGAB_MAX_SLABS];
    int nslab = 0;
    rc = igab_launch_tangent_slabs(ctx, ctx->d_U, ctx->d_vals, prec, row_end, &nslab);
    if (rc) return rc;
    const size_t es = prec == IGAB_PREC_FP64 ? sizeof(double) : sizeof(float);
    const int *rp = ctx->rowptr_h.data();
    long r0 = 0;
    for (int i = 0; i < nslab; i++) {
        IGAB_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, ctx->slab_ev[i], 0));
        const size_t off = (size_t)rp[r0] * es, len = (size_t)(rp[row_end[i]] - rp[r0]) * es;
        if (len)
            IGAB_CUDA_TRY(cudaMemcpyAsync((char *)vals_host + off, (const char *)ctx->d_vals + off, len,
                                          cudaMemcpyDeviceToHost, ctx->copy_stream));
        r0 = row_end[i];
    }
    int fin = 1;
    rc = igab_launch_check_finite(ctx, ctx->d_vals, ctx->nnz, prec, &fin);
    const cudaError_t ce = cudaStreamSynchronize(ctx->copy_stream);
    if (rc) return rc;
    IGAB_CUDA_TRY(ce);
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    rc = igab_check_status(ctx);
    if (rc) return rc;
    if (!fin) { igab_set_error("igab_tangent: non-finite entry"); return IGAB_ERR_NONFINITE; }
    return 0;
}

extern "C" int igab_dirichlet_rows(igab_ctx *ctx, long *n, int *rows)
{
    ARG_CHECK(ctx && n, "igab_dirichlet_rows: null argument");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    if (ctx->dirichlet_dirty) {
        int rc = build_dirichlet(ctx);
        if (rc) return rc;
    }
    if (ctx->per) return igab_periodic_dirichlet_rows(ctx, n, rows);
    *n = ctx->nd;
    if (rows && ctx->nd > 0) {
        IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        IGAB_CUDA_TRY(cudaMemcpy(rows, ctx->d_drow, (size_t)ctx->nd * sizeof(int), cudaMemcpyDeviceToHost));
    }
    return 0;
}

extern "C" int igab_history_jacobian_device(igab_ctx *ctx, const double *U_dev, void *vals_dev, int prec, int level)
{
    IGAB_NO_PERIODIC(ctx, "igab_history_jacobian_device");
    ARG_CHECK(ctx && U_dev && vals_dev, "igab_history_jacobian_device: null argument");
    ARG_CHECK(ctx->phys == IGAB_PHYS_GETIME, "igab_history_jacobian_device: needs the transient physics");
    ARG_CHECK(level == 1 || level == 2, "igab_history_jacobian_device: level must be 1 or 2");
    ARG_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_history_jacobian_device: bad precision");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    ctx->last_launches = 0;
    const size_t es = prec == IGAB_PREC_FP64 ? sizeof(double) : sizeof(float);
    IGAB_CUDA_TRY(cudaMemsetAsync(vals_dev, 0, (size_t)ctx->nnz * es, ctx->stream));
    int rc = igab_launch_tan_getime_level(ctx, U_dev, vals_dev, prec, level);
    if (!rc) rc = igab_launch_zero_csr_rows(ctx, vals_dev, prec);
    return rc;
}

extern "C" int igab_ndensity(const igab_ctx *ctx, int *n)
{
    ARG_CHECK(ctx && n, "igab_ndensity: null argument");
    *n = ctx->phys == IGAB_PHYS_GETIME ? 2 : 13;   /* phys/getime/init.c:14, phys/ge/init.c:14 */
    return 0;
}

extern "C" int igab_intdensity_device(igab_ctx *ctx, const double *U_dev, double *HH_dev)
{
    IGAB_NO_PERIODIC(ctx, "igab_intdensity_device");
    ARG_CHECK(ctx && U_dev && HH_dev, "igab_intdensity_device: null argument");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    return igab_launch_density(ctx, U_dev, HH_dev);
}

extern "C" int igab_intdensity(igab_ctx *ctx, const double *U_host, double *HH_host)
{
    IGAB_NO_PERIODIC(ctx, "igab_intdensity");
    ARG_CHECK(ctx && U_host && HH_host, "igab_intdensity: null argument");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    int rc = ensure_buffers(ctx, -1);
    if (rc) return rc;
    if (!ctx->d_HH) IGAB_CUDA_TRY(cudaMalloc((void **)&ctx->d_HH, 16 * sizeof(double)));
    int nd = 0;
    igab_ndensity(ctx, &nd);
    IGAB_CUDA_TRY(cudaMemcpyAsync(ctx->d_U, U_host, (size_t)ctx->ndof * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    rc = igab_intdensity_device(ctx, ctx->d_U, ctx->d_HH);
    if (rc) return rc;
    IGAB_CUDA_TRY(cudaMemcpyAsync(HH_host, ctx->d_HH, (size_t)nd * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < nd; i++)
        if (!isfinite(HH_host[i])) { igab_set_error("igab_intdensity: non-finite density %d", i); return IGAB_ERR_NONFINITE; }
    return 0;
}

extern "C" int igab_spmv_device(igab_ctx *ctx, const void *vals_dev, int prec, const double *x_dev, double *y_dev)
{
    IGAB_NO_PERIODIC(ctx, "igab_spmv_device");
    ARG_CHECK(ctx && vals_dev && x_dev && y_dev, "igab_spmv_device: null argument");
    ARG_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_spmv_device: bad precision");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    ctx->last_launches = 0;
    return igab_launch_spmv(ctx, vals_dev, prec, x_dev, y_dev);
}

extern "C" int igab_solve_device(igab_ctx *ctx, const void *vals_dev, int prec, const double *b_dev, double *x_dev,
                                 double rtol, double atol, int maxit, igab_solve_info *info)
{
    IGAB_NO_PERIODIC(ctx, "igab_solve_device");
    ARG_CHECK(ctx && vals_dev && b_dev && x_dev, "igab_solve_device: null argument");
    ARG_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_solve_device: bad precision");
    ARG_CHECK(maxit >= 1 && rtol >= 0.0 && atol >= 0.0, "igab_solve_device: bad tolerances");
    ARG_CHECK(ctx->stream != nullptr, "igab_solve_device: needs a non-default stream (igab_set_stream)");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    int its = 0, conv = 0;
    double rn = 0.0, bn = 0.0;
    int rc = igab_krylov_solve(ctx, vals_dev, prec, b_dev, x_dev, rtol, atol, maxit, &its, &conv, &rn, &bn);
    if (rc) return rc;
    if (info) {
        info->iterations = its;
        info->converged = conv;
        info->residual_norm = rn;
        info->rhs_norm = bn;
    }
    return 0;
}

extern "C" int igab_solve_mg_device(igab_ctx *ctx, int method, const void *vals_dev, int prec, const double *b_dev,
                                    double *x_dev, double rtol, double atol, int maxit, igab_solve_info *info)
{
    IGAB_NO_PERIODIC(ctx, "igab_solve_mg_device");
    ARG_CHECK(method == IGAB_KSP_MG_CG || method == IGAB_KSP_MG_GMRES, "igab_solve_mg_device: unknown method");
    ARG_CHECK(ctx && vals_dev && b_dev && x_dev, "igab_solve_mg_device: null argument");
    ARG_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_solve_mg_device: bad precision");
    ARG_CHECK(maxit >= 1 && rtol >= 0.0 && atol >= 0.0, "igab_solve_mg_device: bad tolerances");
    ARG_CHECK(ctx->stream != nullptr, "igab_solve_mg_device: needs a non-default stream (igab_set_stream)");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    int its = 0, conv = 0, brk = 0;
    double rn = 0.0, bn = 0.0;
    int rc = igab_mg_solve(ctx, method, vals_dev, prec, b_dev, x_dev, rtol, atol, maxit, &its, &conv, &rn, &bn, &brk);
    if (rc) return rc;
    if (info) {
        info->iterations = its;
        info->converged = conv;
        info->residual_norm = rn;
        info->rhs_norm = bn;
    }
    if (brk) {
        igab_set_error("igab_solve_mg_device: CG breakdown (the tangent is not positive definite)");
        return IGAB_ERR_UNSUPPORTED;
    }
    return 0;
}

extern "C" int igab_solve_mg_levels(igab_ctx *ctx, int *levels)
{
    ARG_CHECK(ctx && levels, "igab_solve_mg_levels: null argument");
    return igab_mg_levels(ctx, levels);
}

extern "C" int igab_set_stream(igab_ctx *ctx, void *cuda_stream)
{
    ARG_CHECK(ctx, "igab_set_stream: null context");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    if (ctx->own_stream && ctx->stream) {
        IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        cudaStreamDestroy(ctx->stream);
    }
    ctx->stream = (cudaStream_t)cuda_stream;
    ctx->own_stream = false;
    return 0;
}

/* after a stream synchronisation: report (and clear) a kernel's bounded-wait failure */
int igab_check_status(igab_ctx *ctx)
{
    int st = 0;
    IGAB_CUDA_TRY(cudaMemcpy(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) {
        IGAB_CUDA_TRY(cudaMemset(ctx->d_status, 0, sizeof(int)));
        igab_set_error("tensor-core tangent kernel: a completion wait gave up (status %d)", st);
        return IGAB_ERR_CUDA;
    }
    return 0;
}

extern "C" int igab_sync(igab_ctx *ctx)
{
    ARG_CHECK(ctx, "igab_sync: null context");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return igab_check_status(ctx);
}

extern "C" int igab_check_finite(igab_ctx *ctx, const void *dev, long n, int prec, int *all_finite)
{
    ARG_CHECK(ctx && dev && all_finite, "igab_check_finite: null argument");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    return igab_launch_check_finite(ctx, dev, n, prec, all_finite);
}

extern "C" int igab_set_tile(igab_ctx *ctx, int residual_tile, int tangent_tile)
{
    ARG_CHECK(ctx, "igab_set_tile: null context");
    ARG_CHECK(residual_tile == 0 || residual_tile == 2 || residual_tile == 4, "igab_set_tile: residual tile must be 2 or 4");
    ARG_CHECK(tangent_tile == 0 || tangent_tile == 2, "igab_set_tile: tangent tile must be 2");
    ctx->tile_res = residual_tile ? residual_tile : 2;
    ctx->tile_tan = tangent_tile ? tangent_tile : 2;
    ctx->sched_version++;
    return 0;
}

extern "C" int igab_last_launch_count(const igab_ctx *ctx, int *n)
{
    ARG_CHECK(ctx && n, "igab_last_launch_count: null argument");
    *n = ctx->last_launches;
    return 0;
}

extern "C" int igab_set_profiling(igab_ctx *ctx, int on)
{
    ARG_CHECK(ctx, "igab_set_profiling: null context");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    if (on && !ctx->ev[0])
        for (int k = 0; k < 6; k++) IGAB_CUDA_TRY(cudaEventCreate(&ctx->ev[k]));
    ctx->profiling = on != 0;
    ctx->ev_res = ctx->ev_tan = false;
    return 0;
}

extern "C" int igab_last_kernel_ms(igab_ctx *ctx, double ms[6])
{
    ARG_CHECK(ctx && ms, "igab_last_kernel_ms: null argument");
    for (int k = 0; k < 6; k++) ms[k] = 0.0;
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    float t = 0.f;
    if (ctx->ev_res) {
        IGAB_CUDA_TRY(cudaEventElapsedTime(&t, ctx->ev[0], ctx->ev[1])); ms[0] = t;
        IGAB_CUDA_TRY(cudaEventElapsedTime(&t, ctx->ev[1], ctx->ev[2])); ms[1] = t;
    }
    if (ctx->ev_tan) {
        IGAB_CUDA_TRY(cudaEventElapsedTime(&t, ctx->ev[3], ctx->ev[4])); ms[2] = t;
        IGAB_CUDA_TRY(cudaEventElapsedTime(&t, ctx->ev[4], ctx->ev[5])); ms[3] = t;
    }
    ms[4] = ctx->nvol_res;
    ms[5] = ctx->nvol_tan;
    return 0;
}

extern "C" int igab_fma_peak(int device, int prec, double *tflops)
{
    ARG_CHECK(tflops && (prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32), "igab_fma_peak: bad argument");
    IGAB_CUDA_TRY(cudaSetDevice(device));
    return igab_launch_fma_peak(prec, tflops);
}

extern "C" int igab_dmma_peak(int device, double *tflops)
{
    ARG_CHECK(tflops, "igab_dmma_peak: null argument");
    IGAB_CUDA_TRY(cudaSetDevice(device));
    return igab_launch_dmma_peak(tflops);
}

extern "C" int igab_set_option(igab_ctx *ctx, int option, int value)
{
    ARG_CHECK(ctx, "igab_set_option: null context");
    switch (option) {
    case IGAB_OPT_TANGENT_FP64_KERNEL:
        ARG_CHECK(value == 0 || value == 1, "igab_set_option: tangent kernel must be 0 or 1");
        ctx->tan_kernel = value;
        ctx->sched_version++;
        return 0;
    case IGAB_OPT_TANGENT_FP32_KERNEL:
        ARG_CHECK(value == 0 || value == 1, "igab_set_option: tangent kernel must be 0 or 1");
        ctx->tan32_kernel = value;
        ctx->sched_version++;
        return 0;
    case IGAB_OPT_COLOUR_ORDER:
        ARG_CHECK(value >= 0 && value <= 2, "igab_set_option: colour order must be 0, 1 or 2");
        ctx->colour_order = value;
        ctx->sched_version++;
        return 0;
    default:
        igab_set_error("igab_set_option: unknown option %d", option);
        return IGAB_ERR_ARG;
    }
}

extern "C" int igab_get_option(const igab_ctx *ctx, int option, int *value)
{
    ARG_CHECK(ctx && value, "igab_get_option: null argument");
    switch (option) {
    case IGAB_OPT_TANGENT_FP64_KERNEL: *value = ctx->tan_kernel; return 0;
    case IGAB_OPT_TANGENT_FP32_KERNEL: *value = ctx->tan32_kernel; return 0;
    case IGAB_OPT_COLOUR_ORDER: *value = ctx->colour_order; return 0;
    default:
        igab_set_error("igab_get_option: unknown option %d", option);
        return IGAB_ERR_ARG;
    }
}

extern "C" int igab_graph_destroy(igab_ctx *ctx)
{
    ARG_CHECK(ctx, "igab_graph_destroy: null context");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    if (ctx->graph_exec) { cudaGraphExecDestroy(ctx->graph_exec); ctx->graph_exec = nullptr; }
    if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
    return 0;
}

extern "C" int igab_graph_capture(igab_ctx *ctx, const double *U_dev, double *R_dev, void *vals_dev, int prec, int what)
{
    IGAB_NO_PERIODIC(ctx, "igab_graph_capture");
    ARG_CHECK(ctx && U_dev, "igab_graph_capture: null argument");
    ARG_CHECK(what >= 1 && what <= 3, "igab_graph_capture: what must be 1, 2 or 3");
    ARG_CHECK(!(what & 1) || R_dev, "igab_graph_capture: residual output missing");
    ARG_CHECK(!(what & 2) || vals_dev, "igab_graph_capture: tangent output missing");
    ARG_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_graph_capture: bad precision");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    int rc = igab_graph_destroy(ctx);
    if (rc) return rc;
    ARG_CHECK(ctx->stream != nullptr, "igab_graph_capture: the context stream must not be the legacy default stream");
    /* the graph always runs the Neumann kernel: zero values skipped by the last upload */
    if (!ctx->neumann_nonzero && ctx->d_hval)
        IGAB_CUDA_TRY(cudaMemsetAsync(ctx->d_hval, 0, (size_t)ctx->n_neu_points * sizeof(double), ctx->stream));
    /* one eager run first: kernel attributes are set outside the capture */
    const bool prof = ctx->profiling;
    ctx->profiling = false;
    ctx->force_neumann = true;
    if (what & 1) rc = igab_launch_residual(ctx, U_dev, R_dev);
    if (!rc && (what & 2)) rc = igab_launch_tangent(ctx, U_dev, vals_dev, prec);
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) { igab_set_error("igab_graph_capture: %s", cudaGetErrorString(e)); rc = IGAB_ERR_CUDA; }
    }
    if (!rc) {
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { igab_set_error("cudaStreamBeginCapture: %s", cudaGetErrorString(e)); rc = IGAB_ERR_CUDA; }
        else {
            int rc2 = 0;
            if (what & 1) rc2 = igab_launch_residual(ctx, U_dev, R_dev);
            if (!rc2 && (what & 2)) rc2 = igab_launch_tangent(ctx, U_dev, vals_dev, prec);
            cudaGraph_t gr = nullptr;
            e = cudaStreamEndCapture(ctx->stream, &gr);
            if (rc2) { rc = rc2; if (gr) cudaGraphDestroy(gr); }
            else if (e != cudaSuccess) { igab_set_error("cudaStreamEndCapture: %s", cudaGetErrorString(e)); rc = IGAB_ERR_CUDA; }
            else {
                ctx->graph = gr;
                e = cudaGraphInstantiate(&ctx->graph_exec, gr, 0);
                if (e != cudaSuccess) { igab_set_error("cudaGraphInstantiate: %s", cudaGetErrorString(e)); rc = IGAB_ERR_CUDA; }
            }
        }
    }
    ctx->profiling = prof;
    ctx->force_neumann = false;
    return rc;
}

extern "C" int igab_graph_launch(igab_ctx *ctx)
{
    ARG_CHECK(ctx && ctx->graph_exec, "igab_graph_launch: no captured graph");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    IGAB_CUDA_TRY(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    return 0;
}

/* ------------------------------------------------------------------ adjoint */

static int ensure_escale(igab_ctx *ctx)
{
    if (!ctx->d_escale) IGAB_CUDA_TRY(cudaMalloc((void **)&ctx->d_escale, (size_t)ctx->nel * sizeof(double)));
    return 0;
}

extern "C" int igab_set_element_log_scale(igab_ctx *ctx, const double *g, int on_device)
{
    ARG_CHECK(ctx, "igab_set_element_log_scale: null context");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    ctx->param_version++;
    ctx->sched_version++;
    if (!g) {
        ctx->escale_on = false;
        return 0;
    }
    int rc = ensure_escale(ctx);
    if (rc) return rc;
    double *dg = nullptr;
    if (on_device) {
        dg = const_cast<double *>(g);
    } else {
        IGAB_CUDA_TRY(cudaMallocAsync((void **)&dg, (size_t)ctx->nel * sizeof(double), ctx->stream));
        IGAB_CUDA_TRY(cudaMemcpyAsync(dg, g, (size_t)ctx->nel * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    }
    rc = igab_launch_exp_scale(ctx, dg);
    if (!on_device) cudaFreeAsync(dg, ctx->stream);
    if (rc) return rc;
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->escale_on = true;
    return 0;
}

extern "C" int igab_adjoint_forward(igab_ctx *ctx, const double *g_dev, const double *U_dev, double *R_dev,
                                    void *vals_dev, int prec)
{
    IGAB_NO_PERIODIC(ctx, "igab_adjoint_forward");
    ARG_CHECK(ctx && U_dev, "igab_adjoint_forward: null argument");
    ARG_CHECK(R_dev || vals_dev, "igab_adjoint_forward: nothing to compute");
    ARG_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_adjoint_forward: bad precision");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    int rc = 0;
    if (g_dev) {
        rc = ensure_escale(ctx);
        if (!rc) rc = igab_launch_exp_scale(ctx, g_dev);
        if (rc) return rc;
        ctx->escale_on = true;
        ctx->param_version++;
        ctx->sched_version++;
    }
    if (R_dev) rc = igab_launch_residual(ctx, U_dev, R_dev);
    if (!rc && vals_dev) rc = igab_launch_tangent(ctx, U_dev, vals_dev, prec);
    return rc;
}

extern "C" int igab_adjoint_backward(igab_ctx *ctx, const double *U_dev, const void *vals_dev, int prec,
                                     const double *lam_dev, double *KTlam_dev, double *grad_dev)
{
    IGAB_NO_PERIODIC(ctx, "igab_adjoint_backward");
    ARG_CHECK(ctx && lam_dev, "igab_adjoint_backward: null argument");
    ARG_CHECK(KTlam_dev || grad_dev, "igab_adjoint_backward: nothing to compute");
    ARG_CHECK(!KTlam_dev || vals_dev, "igab_adjoint_backward: K^T lam needs the tangent values");
    ARG_CHECK(!grad_dev || U_dev, "igab_adjoint_backward: dR/dg needs U");
    ARG_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_adjoint_backward: bad precision");
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    ctx->last_launches = 0;
    int rc = 0;
    if (KTlam_dev) rc = igab_launch_tangent_transpose(ctx, vals_dev, prec, lam_dev, KTlam_dev);
    if (!rc && grad_dev) {
        if (!ctx->d_lam) IGAB_CUDA_TRY(cudaMalloc((void **)&ctx->d_lam, (size_t)ctx->ndof * sizeof(double)));
        rc = igab_launch_adjoint_dRdg(ctx, U_dev, lam_dev, grad_dev);
    }
    return rc;
}
