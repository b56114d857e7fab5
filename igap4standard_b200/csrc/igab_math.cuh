/*
 * igab_math.cuh -- point-level mathematics of the assembly path, shared by
 * the device kernels and the host set-up code (and compiled on the host by
 * the unit tests).
 *
 *  - 1-D quadratic B-spline values, first and second derivatives at a point
 *    inside an element, by the Cox-de Boor recursion with the reference's
 *    1e-15 denominator guard (mesh/nurbs/eval_Bspline.c:64-74).
 *  - The phys/ge strain-gradient energy and its first and second
 *    derivatives with respect to the 30 interpolated field components
 *    (3 displacement components x [value, 3 first, 6 second derivatives],
 *    component order of mesh/nurbs/eval_Bspline.c:82-91).
 *
 * The energy is the one of phys/ge/density.c:49 (hh[0]):
 *   W = c36 vb (vb^2 - 3 va^2) + c37 (va^2 + vb^2) + c38 (va^2 + vb^2)^2
 *     + p2 vvol^2 + p3 (E01^2 + E02^2 + E12^2) + p4^2 sum_K (ga_K^2 + gb_K^2)
 * with E the Green-Lagrange strain of F = I + grad u, vvol/va/vb its
 * volumetric and two deviatoric invariants (density.c:33-35), and ga_K, gb_K
 * the deviatoric parts of the strain gradient E_II,K (density.c:39-44).
 * Everything below is derived here from that energy, not taken from the
 * generated residual/tangent code.  With the 12 scalar variables
 *   v = (vvol, va, vb, E01, E02, E12, ga_0..2, gb_0..2)
 * each a quadratic function of the field components, W = Phi(v) and
 *   dW/du   = sum_v Phi_v grad v
 *   d2W/du2 = sum_{v,w} Phi_vw grad v grad w^T + sum_v Phi_v hess v,
 * where Phi_vw is diagonal except for the (va, vb) pair and sum_v Phi_v hess v
 * ("geometric" part) is the same 9x9 block for each displacement component.
 * The assembly kernels use this low-rank-plus-block form directly.
 */
#ifndef IGAB_MATH_CUH
#define IGAB_MATH_CUH

#ifdef __CUDACC__
#define IGAB_HD __host__ __device__ __forceinline__
#else
#define IGAB_HD inline

#endif

#define IGAB_INV_SQRT2 0.70710678118654752440
#define IGAB_INV_SQRT3 0.57735026918962576451
#define IGAB_INV_SQRT6 0.40824829046386301637
#define IGAB_MTOL 1.e-15

/* symmetric second-derivative component index: (I,K) -> 0..5 for xx,xy,xz,yy,yz,zz */
IGAB_HD int igab_idx6(int I, int K)
{
    int a = I < K ? I : K, b = I < K ? K : I;
    return a == 0 ? b : (a == 1 ? 2 + b : 5);
}

/* ------------------------------------------------------------------ basis */

/* 1-D p=2 B-spline functions 0..2 of the element whose 6-knot window is kv
 * (kv = knotVector + ielem), at x: out[l][k] = d^k N_l / dx^k.
 * Recursion and guard as mesh/nurbs/eval_Bspline.c:66-73. */
IGAB_HD void igab_bspline_p2(const double kv[6], double x, double out[3][3])
{
    double N0[5] = {0.0, 0.0, 1.0, 0.0, 0.0};
    double N1[4], D1[4];
    for (int i = 0; i < 4; i++) {
        double a = kv[i + 1] - kv[i] + IGAB_MTOL;
        double b = kv[i + 2] - kv[i + 1] + IGAB_MTOL;
        N1[i] = (x - kv[i]) / a * N0[i] + (kv[i + 2] - x) / b * N0[i + 1];
        D1[i] = 1.0 / a * N0[i] - 1.0 / b * N0[i + 1];
    }
    for (int i = 0; i < 3; i++) {
        double a = kv[i + 2] - kv[i] + IGAB_MTOL;
        double b = kv[i + 3] - kv[i + 1] + IGAB_MTOL;
        out[i][0] = (x - kv[i]) / a * N1[i] + (kv[i + 3] - x) / b * N1[i + 1];
        out[i][1] = 2.0 / a * N1[i] - 2.0 / b * N1[i + 1];
        out[i][2] = 2.0 / a * D1[i] - 2.0 / b * D1[i + 1];
    }
}

/* ------------------------------------------------------------- phys/ge */

/* material constants of the energy, from par_mat = {r, curv, e0, e345, le, ...}
 * (phys/ge/residual.c:36-38 give c36..c38 as functions of r and curv) */
typedef struct {
    double p2, p3, p4sq, c36, c37, c38;
} igab_ge_coef;

static inline igab_ge_coef igab_ge_coef_from_par(const double *par)
{
    igab_ge_coef c;
    double r = par[0], cu = par[1];
    double q = 1.3333333333333333 * r - 1.3333333333333333 * r * cu;
    double den = r * r - 2 * (r * r) * cu - r * q;
    c.c36 = -(q / ((r * r) * den));
    c.c37 = (2 * cu) / den;
    c.c38 = -(1 / ((r * r) * den));
    c.p2 = par[2];
    c.p3 = par[3];
    c.p4sq = par[4] * par[4];
    return c;
}

/* Point state: deformation gradient, second derivatives, the 12 energy
 * variables and the first/second derivatives of Phi. */
template <typename T>
struct igab_ge_point {
    T F[3][3];   /* F[k][J] = delta_kJ + du_k/dX_J */
    T G[3][6];   /* G[k][c] = d2u_k/dX_I dX_K, c = idx6(I,K) */
    T v[12];
    T d1[12];    /* Phi_v */
    T d2[12];    /* Phi_vv */
    T d2ab;      /* Phi_{va vb} */
    T sig[3];    /* dW/dE_II */
    T tau[3][3]; /* dW/dE_II,K */
};

/* u: 30 components of one field point (value comps unused by the energy) */
template <typename T>
IGAB_HD void igab_ge_eval(const T *u, const igab_ge_coef &c, igab_ge_point<T> &P)
{
    for (int k = 0; k < 3; k++) {
        for (int J = 0; J < 3; J++) P.F[k][J] = u[10 * k + 1 + J] + (k == J ? T(1) : T(0));
        for (int q = 0; q < 6; q++) P.G[k][q] = u[10 * k + 4 + q];
    }
    T E[3][3];
    for (int I = 0; I < 3; I++)
        for (int J = I; J < 3; J++) {
            T s = P.F[0][I] * P.F[0][J] + P.F[1][I] * P.F[1][J] + P.F[2][I] * P.F[2][J];
            E[I][J] = T(0.5) * (s - (I == J ? T(1) : T(0)));
        }
    T EK[3][3];
    for (int I = 0; I < 3; I++)
        for (int K = 0; K < 3; K++) {
            int q = igab_idx6(I, K);
            EK[I][K] = P.F[0][I] * P.G[0][q] + P.F[1][I] * P.G[1][q] + P.F[2][I] * P.G[2][q];
        }
    const T is2 = T(IGAB_INV_SQRT2), is3 = T(IGAB_INV_SQRT3), is6 = T(IGAB_INV_SQRT6);
    T vv = (E[0][0] + E[1][1] + E[2][2]) * is3;
    T va = (E[0][0] - E[1][1]) * is2;
    T vb = (E[0][0] + E[1][1] - T(2) * E[2][2]) * is6;
    P.v[0] = vv; P.v[1] = va; P.v[2] = vb;
    P.v[3] = E[0][1]; P.v[4] = E[0][2]; P.v[5] = E[1][2];
    for (int K = 0; K < 3; K++) {
        P.v[6 + K] = (EK[0][K] - EK[1][K]) * is2;
        P.v[9 + K] = (EK[0][K] + EK[1][K] - T(2) * EK[2][K]) * is6;
    }
    const T c36 = T(c.c36), c37 = T(c.c37), c38 = T(c.c38);
    const T p2 = T(c.p2), p3 = T(c.p3), p4sq = T(c.p4sq);
    T s2 = va * va + vb * vb;
    P.d1[0] = T(2) * p2 * vv;
    P.d1[1] = T(-6) * c36 * va * vb + T(2) * c37 * va + T(4) * c38 * s2 * va;
    P.d1[2] = T(3) * c36 * (vb * vb - va * va) + T(2) * c37 * vb + T(4) * c38 * s2 * vb;
    for (int i = 3; i < 6; i++) P.d1[i] = T(2) * p3 * P.v[i];
    for (int i = 6; i < 12; i++) P.d1[i] = T(2) * p4sq * P.v[i];
    P.d2[0] = T(2) * p2;
    P.d2[1] = T(-6) * c36 * vb + T(2) * c37 + T(4) * c38 * (T(3) * va * va + vb * vb);
    P.d2[2] = T(6) * c36 * vb + T(2) * c37 + T(4) * c38 * (va * va + T(3) * vb * vb);
    for (int i = 3; i < 6; i++) P.d2[i] = T(2) * p3;
    for (int i = 6; i < 12; i++) P.d2[i] = T(2) * p4sq;
    P.d2ab = T(-6) * c36 * va + T(8) * c38 * va * vb;
    P.sig[0] = P.d1[0] * is3 + P.d1[1] * is2 + P.d1[2] * is6;
    P.sig[1] = P.d1[0] * is3 - P.d1[1] * is2 + P.d1[2] * is6;
    P.sig[2] = P.d1[0] * is3 - T(2) * P.d1[2] * is6;
    for (int K = 0; K < 3; K++) {
        P.tau[0][K] = P.d1[6 + K] * is2 + P.d1[9 + K] * is6;
        P.tau[1][K] = -P.d1[6 + K] * is2 + P.d1[9 + K] * is6;
        P.tau[2][K] = T(-2) * P.d1[9 + K] * is6;
    }
}

/* dW/du for the 30 components (value components are zero) */
template <typename T>
IGAB_HD void igab_ge_residual(const igab_ge_point<T> &P, T *r)
{
    T S[3][3];
    S[0][0] = P.sig[0]; S[1][1] = P.sig[1]; S[2][2] = P.sig[2];
    S[0][1] = S[1][0] = T(0.5) * P.d1[3];
    S[0][2] = S[2][0] = T(0.5) * P.d1[4];
    S[1][2] = S[2][1] = T(0.5) * P.d1[5];
    for (int k = 0; k < 3; k++) {
        r[10 * k] = T(0);
        for (int I = 0; I < 3; I++) {
            T a = S[I][0] * P.F[k][0] + S[I][1] * P.F[k][1] + S[I][2] * P.F[k][2];
            for (int K = 0; K < 3; K++) a += P.tau[I][K] * P.G[k][igab_idx6(I, K)];
            r[10 * k + 1 + I] = a;
        }
        for (int I = 0; I < 3; I++)
            for (int K = I; K < 3; K++) {
                T a = P.tau[I][K] * P.F[k][I];
                if (I != K) a += P.tau[K][I] * P.F[k][K];
                r[10 * k + 4 + igab_idx6(I, K)] = a;
            }
    }
}

/* Gradient of energy variable v with respect to the 9 strain components
 * (3 first + 6 second derivatives) of displacement component k:
 * g[m], m = 0..2 -> d/d(du_k/dX_m), m = 3..8 -> d/d(second derivative m-3). */
template <typename T>
IGAB_HD void igab_ge_grad_var(const igab_ge_point<T> &P, int v, int k, T g[9])
{
    for (int m = 0; m < 9; m++) g[m] = T(0);
    const T is2 = T(IGAB_INV_SQRT2), is3 = T(IGAB_INV_SQRT3), is6 = T(IGAB_INV_SQRT6);
    const T *F = P.F[k];
    const T *G = P.G[k];
    switch (v) {
    case 0: g[0] = F[0] * is3; g[1] = F[1] * is3; g[2] = F[2] * is3; break;
    case 1: g[0] = F[0] * is2; g[1] = -F[1] * is2; break;
    case 2: g[0] = F[0] * is6; g[1] = F[1] * is6; g[2] = T(-2) * F[2] * is6; break;
    case 3: g[0] = T(0.5) * F[1]; g[1] = T(0.5) * F[0]; break;
    case 4: g[0] = T(0.5) * F[2]; g[2] = T(0.5) * F[0]; break;
    case 5: g[1] = T(0.5) * F[2]; g[2] = T(0.5) * F[1]; break;
    default:
        if (v < 9) {
            int K = v - 6;
            int q0 = igab_idx6(0, K), q1 = igab_idx6(1, K);
            g[0] = G[q0] * is2; g[1] = -G[q1] * is2;
            g[3 + q0] = F[0] * is2; g[3 + q1] = -F[1] * is2;
        } else {
            int K = v - 9;
            int q0 = igab_idx6(0, K), q1 = igab_idx6(1, K), q2 = igab_idx6(2, K);
            g[0] = G[q0] * is6; g[1] = G[q1] * is6; g[2] = T(-2) * G[q2] * is6;
            g[3 + q0] = F[0] * is6; g[3 + q1] = F[1] * is6; g[3 + q2] = T(-2) * F[2] * is6;
        }
    }
}

/* geometric block geo[m][n] (9x9, identical for every displacement component) */
template <typename T>
IGAB_HD void igab_ge_geo(const igab_ge_point<T> &P, T geo[9][9])
{
    for (int m = 0; m < 9; m++)
        for (int n = 0; n < 9; n++) geo[m][n] = T(0);
    for (int I = 0; I < 3; I++) geo[I][I] = P.sig[I];
    geo[0][1] = geo[1][0] = T(0.5) * P.d1[3];
    geo[0][2] = geo[2][0] = T(0.5) * P.d1[4];
    geo[1][2] = geo[2][1] = T(0.5) * P.d1[5];
    for (int I = 0; I < 3; I++)
        for (int K = 0; K < 3; K++) {
            int n = 3 + igab_idx6(I, K);
            geo[I][n] += P.tau[I][K];
            geo[n][I] += P.tau[I][K];
        }
}

/* dense d2W/du2 restricted to the 27 strain components, s = 9k + m */
template <typename T>
IGAB_HD void igab_ge_dense_tangent(const igab_ge_point<T> &P, T D[27][27])
{
    T g[12][27];
    for (int v = 0; v < 12; v++)
        for (int k = 0; k < 3; k++) igab_ge_grad_var(P, v, k, &g[v][9 * k]);
    T geo[9][9];
    igab_ge_geo(P, geo);
    for (int s = 0; s < 27; s++)
        for (int t = 0; t < 27; t++) {
            T a = P.d2ab * (g[1][s] * g[2][t] + g[2][s] * g[1][t]);
            for (int v = 0; v < 12; v++) a += P.d2[v] * g[v][s] * g[v][t];
            if (s / 9 == t / 9) a += geo[s % 9][t % 9];
            D[s][t] = a;
        }
}


/* ------------------------------------------------------------- Taylor arithmetic */

/* Truncated univariate Taylor polynomials c[0] + c[1] s + ... + c[N-1] s^(N-1).
 * Running the energy code on u(s) = m + s h with this type yields the Taylor
 * coefficients of dW/du (or of the point data) along the segment, which is how
 * the transient integrand below is formed. */
template <int N>
struct igab_tay {
    double c[N];
    IGAB_HD igab_tay() {}
    IGAB_HD igab_tay(double x)
    {
        c[0] = x;
        for (int i = 1; i < N; i++) c[i] = 0.0;
    }
};
template <int N>
IGAB_HD igab_tay<N> operator+(const igab_tay<N> &a, const igab_tay<N> &b)
{
    igab_tay<N> r;
    for (int i = 0; i < N; i++) r.c[i] = a.c[i] + b.c[i];
    return r;
}
template <int N>
IGAB_HD igab_tay<N> operator-(const igab_tay<N> &a, const igab_tay<N> &b)
{
    igab_tay<N> r;
    for (int i = 0; i < N; i++) r.c[i] = a.c[i] - b.c[i];
    return r;
}
template <int N>
IGAB_HD igab_tay<N> operator-(const igab_tay<N> &a)
{
    igab_tay<N> r;
    for (int i = 0; i < N; i++) r.c[i] = -a.c[i];
    return r;
}
template <int N>
IGAB_HD igab_tay<N> operator*(const igab_tay<N> &a, const igab_tay<N> &b)
{
    igab_tay<N> r;
    for (int i = 0; i < N; i++) {
        double t = 0.0;
        for (int j = 0; j <= i; j++) t += a.c[j] * b.c[i - j];
        r.c[i] = t;
    }
    return r;
}
template <int N>
IGAB_HD igab_tay<N> &operator+=(igab_tay<N> &a, const igab_tay<N> &b)
{
    a = a + b;
    return a;
}

/* ------------------------------------------------------------- phys/getime */

/* The transient integrand of phys/getime (torder = 2, U_hist levels: u at t_{n+1},
 * u1 at t_n, u0 at t_{n-1}; par = {.., rho = par[5], c = par[6], dt = par[7]}):
 *   value components:  c (u - u0) / (2 dt) + rho (u + u0 - 2 u1) / dt^2
 *   field derivatives: sum_{n=0..3} g_n / (n + 1),  g(s) = dW/du(m + s h) = sum g_n s^n,
 *                      m = (u0 + u1)/2, h = (u - u0)/2,
 * i.e. the average of dW/du over the segment from the mid-state of (t_{n-1}, t_n)
 * to that of (t_n, t_{n+1}), truncated after the cubic term of its Taylor series
 * (the expression phys/getime/residual.c:4127-4156 expands).  Its derivative is
 *   d r / d u = 1/2 (H_0/2 + H_1/3 + H_2/4) + diag(rho/dt^2 + c/(2 dt)) on values,
 * H(s) = d2W/du2(m + s h) = sum H_j s^j. */
template <typename T>
IGAB_HD void igab_getime_residual(const T *u, const T *u1, const T *u0, const igab_ge_coef &c,
                                  double rho, double cii, double dt, T *r)
{
    igab_tay<4> ut[30];
    for (int i = 0; i < 30; i++) {
        ut[i].c[0] = double((u0[i] + u1[i]) * T(0.5));
        ut[i].c[1] = double((u[i] - u0[i]) * T(0.5));
        ut[i].c[2] = 0.0;
        ut[i].c[3] = 0.0;
    }
    igab_ge_point<igab_tay<4>> P;
    igab_ge_eval(ut, c, P);
    igab_tay<4> rt[30];
    igab_ge_residual(P, rt);
    for (int i = 0; i < 30; i++) r[i] = T(rt[i].c[0] + rt[i].c[1] / 2.0 + rt[i].c[2] / 3.0 + rt[i].c[3] / 4.0);
    for (int k = 0; k < 3; k++)
        r[10 * k] = T(cii) * (u[10 * k] - u0[10 * k]) / T(2.0 * dt) +
                    T(rho) * (u[10 * k] + u0[10 * k] - T(2) * u1[10 * k]) / T(dt * dt);
}

/* dense getime tangent on the 27 field-derivative components (check path) */
template <typename T>
IGAB_HD void igab_getime_dense_tangent(const T *u, const T *u1, const T *u0, const igab_ge_coef &c, T D[27][27])
{
    igab_tay<3> ut[30];
    for (int i = 0; i < 30; i++) {
        ut[i].c[0] = double((u0[i] + u1[i]) * T(0.5));
        ut[i].c[1] = double((u[i] - u0[i]) * T(0.5));
        ut[i].c[2] = 0.0;
    }
    igab_ge_point<igab_tay<3>> P;
    igab_ge_eval(ut, c, P);
    igab_tay<3> H[27][27];
    igab_ge_dense_tangent(P, H);
    for (int s = 0; s < 27; s++)
        for (int t = 0; t < 27; t++) D[s][t] = T(0.5 * (H[s][t].c[0] / 2.0 + H[s][t].c[1] / 3.0 + H[s][t].c[2] / 4.0));
}
#endif
