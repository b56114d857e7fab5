/*
 * CPU restatement of IGAP4STANDARD's element assembly (test infrastructure:
 * the checker of the tests, never shipped, never the measured path).
 *
 * Written from the reference's algorithm, in this project's own code:
 *   gauss_rule      4-point Gauss-Legendre on [0,1] by Newton iteration on
 *                   P_4 (src/quadrature.c:381-431 computes the same rule)
 *   bspline_window  p=2 values/derivatives of an element's 3 functions with
 *                   the 1e-15 denominator guard (mesh/nurbs/eval_Bspline.c:64-74)
 *   bspline_any     k-th derivative of basis i anywhere, end-point rule of
 *                   mesh/nurbs/evalN.c:19-20, divided differences :31-48
 *   ge_energy       W of phys/ge/density.c:49 (hh[0]); its gradient and
 *                   Hessian come from hyper-dual arithmetic, independently
 *                   of the product's hand-derived chain rule
 *   assembly        src/snesiga_Residual.c:99-412 and src/snesiga_Tangent.c:99-272
 *                   (volume, Neumann, Dirichlet rows / rows+columns)
 * Parity pinned against the reference itself (oracle/_ref) and the committed
 * golden vectors under tests/golden/.
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

/* ------------------------------------------------------------ hyper-dual */
struct HD {
    double a, b, c, d;   /* a + b e1 + c e2 + d e1 e2 */
    HD(double x = 0) : a(x), b(0), c(0), d(0) {}
    HD(double a_, double b_, double c_, double d_) : a(a_), b(b_), c(c_), d(d_) {}
};
static inline HD operator+(HD x, HD y) { return HD(x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d); }
static inline HD operator-(HD x, HD y) { return HD(x.a - y.a, x.b - y.b, x.c - y.c, x.d - y.d); }
static inline HD operator*(HD x, HD y)
{
    return HD(x.a * y.a, x.a * y.b + x.b * y.a, x.a * y.c + x.c * y.a, x.a * y.d + x.b * y.c + x.c * y.b + x.d * y.a);
}
static inline HD operator*(double s, HD x) { return HD(s * x.a, s * x.b, s * x.c, s * x.d); }

/* energy density W(u) for 30 field components, par = par_mat */
template <typename T>
static T ge_energy(const T *u, const double *par)
{
    auto F = [&](int k, int J) { return u[10 * k + 1 + J] + T(k == J ? 1.0 : 0.0); };
    auto G = [&](int k, int I, int K) {
        int a = I < K ? I : K, b = I < K ? K : I;
        int c = a == 0 ? b : (a == 1 ? 2 + b : 5);
        return u[10 * k + 4 + c];
    };
    T E[3][3];
    for (int I = 0; I < 3; I++)
        for (int J = 0; J < 3; J++) {
            T s(0.0);
            for (int k = 0; k < 3; k++) s = s + F(k, I) * F(k, J);
            E[I][J] = 0.5 * (s - T(I == J ? 1.0 : 0.0));
        }
    T EK[3][3];   /* E_II,K = sum_k F_kI u_k,IK */
    for (int I = 0; I < 3; I++)
        for (int K = 0; K < 3; K++) {
            T s(0.0);
            for (int k = 0; k < 3; k++) s = s + F(k, I) * G(k, I, K);
            EK[I][K] = s;
        }
    const double s2 = 1.0 / std::sqrt(2.0), s3 = 1.0 / std::sqrt(3.0), s6 = 1.0 / std::sqrt(6.0);
    T vv = s3 * (E[0][0] + E[1][1] + E[2][2]);
    T va = s2 * (E[0][0] - E[1][1]);
    T vb = s6 * (E[0][0] + E[1][1] - 2.0 * E[2][2]);
    double r = par[0], cu = par[1];
    double q = 4.0 / 3.0 * r * (1.0 - cu);
    double den = r * r * (1.0 - 2.0 * cu) - r * q;
    double c36 = -q / (r * r * den), c37 = 2.0 * cu / den, c38 = -1.0 / (r * r * den);
    T sq = va * va + vb * vb;
    T W = c36 * (vb * (vb * vb - 3.0 * (va * va))) + c37 * sq + c38 * (sq * sq) + par[2] * (vv * vv) +
          par[3] * (E[0][1] * E[0][1] + E[0][2] * E[0][2] + E[1][2] * E[1][2]);
    T g(0.0);
    for (int K = 0; K < 3; K++) {
        T ga = s2 * (EK[0][K] - EK[1][K]);
        T gb = s6 * (EK[0][K] + EK[1][K] - 2.0 * EK[2][K]);
        g = g + ga * ga + gb * gb;
    }
    return W + (par[4] * par[4]) * g;
}

static void ge_point(const double *u, const double *par, double *r, double *D /* 900 or NULL */)
{
    HD x[30];
    for (int i = 0; i < 30; i++) x[i] = HD(u[i]);
    for (int i = 0; i < 30; i++) {
        r[i] = 0.0;
        if (i % 10 == 0) continue;
        x[i].b = 1.0;
        r[i] = ge_energy(x, par).b;
        x[i].b = 0.0;
    }
    if (!D) return;
    for (int i = 0; i < 900; i++) D[i] = 0.0;
    for (int i = 0; i < 30; i++) {
        if (i % 10 == 0) continue;
        for (int j = i; j < 30; j++) {
            if (j % 10 == 0) continue;
            x[i].b = 1.0;
            x[j].c = 1.0;
            double h = ge_energy(x, par).d;
            x[i].b = 0.0;
            x[j].c = 0.0;
            D[30 * i + j] = D[30 * j + i] = h;
        }
    }
}

/* ------------------------------------------------------------ quadrature */
static void gauss_rule(double x[4], double w[4])
{
    for (int i = 0; i < 4; i++) {
        double t = std::cos(M_PI * (i + 0.75) / 4.5);
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = t;
            for (int n = 2; n <= 4; n++) { double p2 = ((2 * n - 1) * t * p1 - (n - 1) * p0) / n; p0 = p1; p1 = p2; }
            double dp = 4.0 * (t * p1 - p0) / (t * t - 1.0);
            double dt = p1 / dp;
            t -= dt;
            if (std::fabs(dt) < 1e-17) break;
        }
        double p0 = 1.0, p1 = t;
        for (int n = 2; n <= 4; n++) { double p2 = ((2 * n - 1) * t * p1 - (n - 1) * p0) / n; p0 = p1; p1 = p2; }
        double dp = 4.0 * (t * p1 - p0) / (t * t - 1.0);
        x[3 - i] = 0.5 * (t + 1.0);
        w[3 - i] = 1.0 / ((1.0 - t * t) * dp * dp);   /* 2/((1-t^2) P'^2), halved for [0,1] */
    }
}

/* ------------------------------------------------------------ B-splines */
static void bspline_window(const double *kv, double x, double N[3][3])
{
    const double eps = 1e-15;
    double b0[5] = {0, 0, 1, 0, 0}, b1[4], d1[4];
    for (int i = 0; i < 4; i++) {
        double l = kv[i + 1] - kv[i] + eps, r = kv[i + 2] - kv[i + 1] + eps;
        b1[i] = (x - kv[i]) / l * b0[i] + (kv[i + 2] - x) / r * b0[i + 1];
        d1[i] = b0[i] / l - b0[i + 1] / r;
    }
    for (int i = 0; i < 3; i++) {
        double l = kv[i + 2] - kv[i] + eps, r = kv[i + 3] - kv[i + 1] + eps;
        N[i][0] = (x - kv[i]) / l * b1[i] + (kv[i + 3] - x) / r * b1[i + 1];
        N[i][1] = 2.0 * (b1[i] / l - b1[i + 1] / r);
        N[i][2] = 2.0 * (d1[i] / l - d1[i + 1] / r);
    }
}

static double bspline_any(const double *kv, int nk, int k, int i, int p, double x)
{
    if (k == 0) {
        if (i == nk - p - 2 && std::fabs(x - kv[nk - 1]) < 1e-15 && std::fabs(kv[nk - 1] - kv[nk - 2]) < 1e-15)
            return 1.0;
        if (p == 0) return (x >= kv[i] && x < kv[i + 1]) ? 1.0 : 0.0;
        double left = 0.0, right = 0.0;
        if (kv[i + p] != kv[i]) left = (x - kv[i]) / (kv[i + p] - kv[i]) * bspline_any(kv, nk, 0, i, p - 1, x);
        if (kv[i + p + 1] != kv[i + 1])
            right = (kv[i + p + 1] - x) / (kv[i + p + 1] - kv[i + 1]) * bspline_any(kv, nk, 0, i + 1, p - 1, x);
        return left + right;
    }
    if (k > p) return 0.0;
    /* k-th derivative = p!/(p-k)! sum_j a_kj N_{i+j,p-k}, a from divided differences */
    double a[3][3] = {{1.0}};
    for (int r = 1; r <= k; r++) {
        for (int c = 0; c <= r; c++) {
            double lo = c > 0 ? a[r - 1][c - 1] : 0.0, hi = c < r ? a[r - 1][c] : 0.0;
            double span = kv[i + p + c - r + 1] - kv[i + c];
            a[r][c] = span == 0.0 ? 0.0 : (hi - lo) / span;
        }
    }
    double s = 0.0;
    for (int j = 0; j <= k; j++) s += a[k][j] * bspline_any(kv, nk, 0, i + j, p - k, x);
    double f = 1.0;
    for (int j = 0; j < k; j++) f *= (p - j);
    return s * f;
}

/* ------------------------------------------------------------ case */
struct PortCase {
    int ne[3], nb[3];
    std::vector<double> kv[3];
    double par[9], pp[9], pd[9];
    int bc[36];
    std::vector<double> pn;
    long ndof;
};

static void face_dirs(int face, int &d0, int &d1, int &dn)
{
    if (face / 2 == 0) { d0 = 1; d1 = 2; dn = 0; }
    else if (face / 2 == 1) { d0 = 0; d1 = 2; dn = 1; }
    else { d0 = 0; d1 = 1; dn = 2; }
}

static long cp_index(const PortCase &c, int x, int y, int z) { return ((long)x * c.nb[1] + y) * c.nb[2] + z; }

static long face_cp(const PortCase &c, int face, int b0, int b1, int layer)
{
    int d0, d1, dn, p[3];
    face_dirs(face, d0, d1, dn);
    p[d0] = b0; p[d1] = b1; p[dn] = layer;
    return cp_index(c, p[0], p[1], p[2]);
}

/* default traction hook of the case builder */
static double traction(const PortCase &c, int face, int order, int dof, const double x[3])
{
    const double *pn = c.pn.data();
    return pn[6 * face + 3 * order + dof] * (1.0 + pn[36] * x[0] + pn[37] * x[1] + pn[38] * x[2]);
}

/* values of iga_dirichlet for (face, order, dof) in (i over d0, j over d1) order */
static std::vector<double> dirichlet_values(const PortCase &c, int face, int order, int dof)
{
    int d0, d1, dn;
    face_dirs(face, d0, d1, dn);
    int dims[2] = {d0, d1};
    double a[3] = {c.pd[3 * dof + d0], c.pd[3 * dof + d1], c.pd[3 * dof + dn]};
    const std::vector<double> &kn = c.kv[dn];
    double Z = (face % 2 == 0) ? kn.front() : kn.back() - 1e-15;
    std::vector<double> line[2];
    for (int b = 0; b < 2; b++) {
        const std::vector<double> &k = c.kv[dims[b]];
        int n = c.nb[dims[b]], nk = (int)k.size();
        line[b].resize(n);
        /* interpolate value a*W and slope a at the first element start with the first two functions */
        double W = k[2];
        double m00 = bspline_any(k.data(), nk, 0, 0, 2, W), m01 = bspline_any(k.data(), nk, 0, 1, 2, W);
        double m10 = bspline_any(k.data(), nk, 1, 0, 2, W), m11 = bspline_any(k.data(), nk, 1, 1, 2, W);
        double det = m00 * m11 - m01 * m10;
        double v0 = a[b] * W, v1 = a[b];
        line[b][0] = (m11 * v0 - m01 * v1) / det;
        line[b][1] = (-m10 * v0 + m00 * v1) / det;
        for (int i = 2; i < n; i++) line[b][i] = line[b][i - 1] + 0.5 * (k[i + 2] - k[i]) * a[b];
    }
    std::vector<double> out((size_t)c.nb[d0] * c.nb[d1]);
    for (int i = 0; i < c.nb[d0]; i++)
        for (int j = 0; j < c.nb[d1]; j++) out[(size_t)c.nb[d1] * i + j] = line[0][i] + line[1][j] + a[2] * Z;
    if (order == 1) {
        int ib = (face % 2 == 0) ? 1 : c.nb[dn] - 2;
        double m = 0.0 / bspline_any(kn.data(), (int)kn.size(), 1, ib, 2, Z);
        for (auto &v : out) v += m;
    }
    return out;
}

/* element loop shared by residual and tangent */
struct ElemBasis {
    double N[27][10];
    double w;
    double x[3];
};

static void element_points(const PortCase &c, int ex, int ey, int ez, std::vector<ElemBasis> &pts)
{
    double gx[4], gw[4];
    gauss_rule(gx, gw);
    int e[3] = {ex, ey, ez};
    double tab[3][4][3][3], X[3][4], h[3];
    for (int d = 0; d < 3; d++) {
        const double *k = c.kv[d].data() + e[d];
        double X0 = k[2], X1 = k[3];
        h[d] = X1 - X0;
        for (int q = 0; q < 4; q++) {
            X[d][q] = (1.0 - gx[q]) * X0 + gx[q] * X1;
            bspline_window(k, X[d][q], tab[d][q]);
        }
    }
    static const int KX[10] = {0, 1, 0, 0, 2, 1, 1, 0, 0, 0}, KY[10] = {0, 0, 1, 0, 0, 1, 0, 2, 1, 0},
                     KZ[10] = {0, 0, 0, 1, 0, 0, 1, 0, 1, 2};
    pts.resize(64);
    for (int qx = 0; qx < 4; qx++)
        for (int qy = 0; qy < 4; qy++)
            for (int qz = 0; qz < 4; qz++) {
                ElemBasis &P = pts[16 * qx + 4 * qy + qz];
                P.w = gw[qx] * gw[qy] * gw[qz] * h[0] * h[1] * h[2];
                P.x[0] = X[0][qx]; P.x[1] = X[1][qy]; P.x[2] = X[2][qz];
                for (int a = 0; a < 27; a++)
                    for (int al = 0; al < 10; al++)
                        P.N[a][al] = tab[0][qx][a / 9][KX[al]] * tab[1][qy][(a / 3) % 3][KY[al]] * tab[2][qz][a % 3][KZ[al]];
            }
}

static void field_at(const PortCase &c, const ElemBasis &P, const double *U, int ex, int ey, int ez, double u[30])
{
    for (int i = 0; i < 30; i++) u[i] = 0.0;
    for (int a = 0; a < 27; a++) {
        long cp = cp_index(c, ex + a / 9, ey + (a / 3) % 3, ez + a % 3);
        for (int k = 0; k < 3; k++)
            for (int al = 0; al < 10; al++) u[10 * k + al] += P.N[a][al] * U[3 * cp + k];
    }
    for (int k = 0; k < 3; k++) {
        for (int J = 0; J < 3; J++) {
            u[10 * k] += c.pp[3 * k + J] * P.x[J];
            u[10 * k + 1 + J] += c.pp[3 * k + J];
        }
    }
}

extern "C" {

void *port_case_create(const int nelem[3], const double *knots, const double par_mat[9], const int bc_type[36],
                       const double par_periodic[9], const double par_dirichlet[9], const double *par_neumann,
                       int n_par_neumann)
{
    PortCase *c = new PortCase();
    size_t o = 0;
    for (int d = 0; d < 3; d++) {
        c->ne[d] = nelem[d];
        c->nb[d] = nelem[d] + 2;
        c->kv[d].assign(knots + o, knots + o + nelem[d] + 5);
        o += (size_t)nelem[d] + 5;
    }
    memcpy(c->par, par_mat, sizeof(c->par));
    memcpy(c->pp, par_periodic, sizeof(c->pp));
    memcpy(c->pd, par_dirichlet, sizeof(c->pd));
    memcpy(c->bc, bc_type, sizeof(c->bc));
    c->pn.assign(n_par_neumann > 39 ? n_par_neumann : 39, 0.0);
    if (par_neumann) memcpy(c->pn.data(), par_neumann, (size_t)n_par_neumann * sizeof(double));
    c->ndof = 3L * c->nb[0] * c->nb[1] * c->nb[2];
    return c;
}

void port_case_destroy(void *h) { delete (PortCase *)h; }
long port_ndof(void *h) { return ((PortCase *)h)->ndof; }

void port_ge_point(const double *u, const double *par, double *r, double *D) { ge_point(u, par, r, D); }
void port_gauss(double *x, double *w) { gauss_rule(x, w); }
void port_bspline_window(const double *kv6, double x, double *out9)
{
    double N[3][3];
    bspline_window(kv6, x, N);
    memcpy(out9, N, sizeof(N));
}
double port_bspline_any(const double *kv, int nk, int k, int i, int p, double x) { return bspline_any(kv, nk, k, i, p, x); }

/* residual with all boundary terms */
void port_residual(void *h, const double *U, double *R)
{
    PortCase &c = *(PortCase *)h;
    for (long i = 0; i < c.ndof; i++) R[i] = 0.0;
    std::vector<ElemBasis> pts;
    for (int ex = 0; ex < c.ne[0]; ex++)
        for (int ey = 0; ey < c.ne[1]; ey++)
            for (int ez = 0; ez < c.ne[2]; ez++) {
                element_points(c, ex, ey, ez, pts);
                double val[81] = {0};
                for (auto &P : pts) {
                    double u[30], r[30];
                    field_at(c, P, U, ex, ey, ez, u);
                    ge_point(u, c.par, r, nullptr);
                    for (int a = 0; a < 27; a++)
                        for (int k = 0; k < 3; k++) {
                            double s = 0.0;
                            for (int al = 0; al < 10; al++) s += P.N[a][al] * r[10 * k + al];
                            val[3 * a + k] += P.w * s;
                        }
                }
                for (int a = 0; a < 27; a++)
                    for (int k = 0; k < 3; k++)
                        R[3 * cp_index(c, ex + a / 9, ey + (a / 3) % 3, ez + a % 3) + k] += val[3 * a + k];
            }
    /* Neumann: -int N h (order 0) and -int dN/dn h on the two face layers (order 1) */
    double gx[4], gw[4];
    gauss_rule(gx, gw);
    for (int face = 0; face < 6; face++) {
        int d0, d1, dn;
        face_dirs(face, d0, d1, dn);
        const std::vector<double> &kz = c.kv[dn];
        double zq = (face % 2 == 0) ? kz.front() : kz.back();
        int l0 = (face % 2 == 0) ? 0 : c.nb[dn] - 1, l1 = (face % 2 == 0) ? 1 : c.nb[dn] - 2;
        double dz0 = bspline_any(kz.data(), (int)kz.size(), 1, l0, 2, zq);
        double dz1 = bspline_any(kz.data(), (int)kz.size(), 1, l1, 2, zq);
        for (int order = 0; order < 2; order++)
            for (int dof = 0; dof < 3; dof++) {
                if (c.bc[6 * face + 3 * order + dof] != 1) continue;
                for (int e0 = 0; e0 < c.ne[d0]; e0++)
                    for (int e1 = 0; e1 < c.ne[d1]; e1++) {
                        const double *k0 = c.kv[d0].data(), *k1 = c.kv[d1].data();
                        double h0 = k0[e0 + 3] - k0[e0 + 2], h1 = k1[e1 + 3] - k1[e1 + 2];
                        for (int q0 = 0; q0 < 4; q0++)
                            for (int q1 = 0; q1 < 4; q1++) {
                                double x[3];
                                x[d0] = (1.0 - gx[q0]) * k0[e0 + 2] + gx[q0] * k0[e0 + 3];
                                x[d1] = (1.0 - gx[q1]) * k1[e1 + 2] + gx[q1] * k1[e1 + 3];
                                x[dn] = zq;
                                double tv = traction(c, face, order, dof, x);
                                double wt = gw[q0] * gw[q1] * h0 * h1;
                                for (int b0 = 0; b0 < 3; b0++)
                                    for (int b1 = 0; b1 < 3; b1++) {
                                        double n0 = bspline_any(k0, (int)c.kv[d0].size(), 0, e0 + b0, 2, x[d0]);
                                        double n1 = bspline_any(k1, (int)c.kv[d1].size(), 0, e1 + b1, 2, x[d1]);
                                        if (order == 0) {
                                            R[3 * face_cp(c, face, e0 + b0, e1 + b1, l0) + dof] -= wt * n0 * n1 * tv;
                                        } else {
                                            R[3 * face_cp(c, face, e0 + b0, e1 + b1, l0) + dof] -= wt * n0 * n1 * dz0 * tv;
                                            R[3 * face_cp(c, face, e0 + b0, e1 + b1, l1) + dof] -= wt * n0 * n1 * dz1 * tv;
                                        }
                                    }
                            }
                    }
            }
    }
    /* Dirichlet rows R = U - g, last write wins */
    for (int face = 0; face < 6; face++) {
        int d0, d1, dn;
        face_dirs(face, d0, d1, dn);
        for (int order = 0; order < 2; order++)
            for (int dof = 0; dof < 3; dof++) {
                if (c.bc[6 * face + 3 * order + dof] != 0) continue;
                std::vector<double> g = dirichlet_values(c, face, order, dof);
                int layer = (face % 2 == 0) ? order : c.nb[dn] - 1 - order;
                for (int i = 0; i < c.nb[d0]; i++)
                    for (int j = 0; j < c.nb[d1]; j++) {
                        long r = 3 * face_cp(c, face, i, j, layer) + dof;
                        R[r] = U[r] - g[(size_t)c.nb[d1] * i + j];
                    }
            }
    }
}

/* tangent: CSR with ascending columns (every pair of points with overlapping supports) */
long port_nnz(void *h)
{
    PortCase &c = *(PortCase *)h;
    long n = 9;
    for (int d = 0; d < 3; d++) {
        long m = c.nb[d];
        n *= m + 2 * (m > 1 ? m - 1 : 0) + 2 * (m > 2 ? m - 2 : 0);
    }
    return n;
}

void port_tangent(void *h, const double *U, int *rowptr, int *cols, double *vals)
{
    PortCase &c = *(PortCase *)h;
    /* pattern */
    long o = 0, r = 0;
    for (int x = 0; x < c.nb[0]; x++)
        for (int y = 0; y < c.nb[1]; y++)
            for (int z = 0; z < c.nb[2]; z++)
                for (int k = 0; k < 3; k++) {
                    rowptr[r++] = (int)o;
                    for (int cx = std::max(x - 2, 0); cx <= std::min(x + 2, c.nb[0] - 1); cx++)
                        for (int cy = std::max(y - 2, 0); cy <= std::min(y + 2, c.nb[1] - 1); cy++)
                            for (int cz = std::max(z - 2, 0); cz <= std::min(z + 2, c.nb[2] - 1); cz++)
                                for (int l = 0; l < 3; l++) { cols[o] = (int)(3 * cp_index(c, cx, cy, cz) + l); vals[o] = 0.0; o++; }
                }
    rowptr[r] = (int)o;
    auto find = [&](long row, long col) -> long {
        long lo = rowptr[row], hi = rowptr[row + 1];
        while (lo < hi) { long m = (lo + hi) / 2; if (cols[m] < col) lo = m + 1; else hi = m; }
        return lo;
    };
    std::vector<ElemBasis> pts;
    std::vector<double> Ke(81 * 81);
    for (int ex = 0; ex < c.ne[0]; ex++)
        for (int ey = 0; ey < c.ne[1]; ey++)
            for (int ez = 0; ez < c.ne[2]; ez++) {
                element_points(c, ex, ey, ez, pts);
                std::fill(Ke.begin(), Ke.end(), 0.0);
                for (auto &P : pts) {
                    double u[30], rr[30], D[900];
                    field_at(c, P, U, ex, ey, ez, u);
                    ge_point(u, c.par, rr, D);
                    /* DN[(k,al)][(b,l)] = sum_be D[k al][l be] N_b^be */
                    static double DN[30][81];
                    for (int ka = 0; ka < 30; ka++)
                        for (int b = 0; b < 27; b++)
                            for (int l = 0; l < 3; l++) {
                                double s = 0.0;
                                for (int be = 0; be < 10; be++) s += D[30 * ka + 10 * l + be] * P.N[b][be];
                                DN[ka][3 * b + l] = s;
                            }
                    for (int a = 0; a < 27; a++)
                        for (int k = 0; k < 3; k++)
                            for (int cc = 0; cc < 81; cc++) {
                                double s = 0.0;
                                for (int al = 0; al < 10; al++) s += P.N[a][al] * DN[10 * k + al][cc];
                                Ke[(3 * a + k) * 81 + cc] += P.w * s;
                            }
                }
                for (int a = 0; a < 27; a++) {
                    long ra = cp_index(c, ex + a / 9, ey + (a / 3) % 3, ez + a % 3);
                    for (int k = 0; k < 3; k++)
                        for (int b = 0; b < 27; b++) {
                            long cb = cp_index(c, ex + b / 9, ey + (b / 3) % 3, ez + b % 3);
                            for (int l = 0; l < 3; l++) vals[find(3 * ra + k, 3 * cb + l)] += Ke[(3 * a + k) * 81 + 3 * b + l];
                        }
                }
            }
    /* Dirichlet rows and columns zeroed, unit diagonal */
    std::vector<char> mask(c.ndof, 0);
    for (int face = 0; face < 6; face++) {
        int d0, d1, dn;
        face_dirs(face, d0, d1, dn);
        for (int order = 0; order < 2; order++)
            for (int dof = 0; dof < 3; dof++) {
                if (c.bc[6 * face + 3 * order + dof] != 0) continue;
                int layer = (face % 2 == 0) ? order : c.nb[dn] - 1 - order;
                for (int i = 0; i < c.nb[d0]; i++)
                    for (int j = 0; j < c.nb[d1]; j++) mask[3 * face_cp(c, face, i, j, layer) + dof] = 1;
            }
    }
    for (long row = 0; row < c.ndof; row++)
        for (long k = rowptr[row]; k < rowptr[row + 1]; k++) {
            if (mask[row] || mask[cols[k]]) vals[k] = (row == cols[k] && mask[row]) ? 1.0 : 0.0;
        }
}

} /* extern "C" */
