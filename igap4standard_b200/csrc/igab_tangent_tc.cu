/*
 * FP32 tangent volume kernel on the 5th-generation tensor cores (tcgen05,
 * TF32 operands in shared memory, FP32 accumulators in tensor memory): the
 * tangent of the mixed-precision Newton path (FP32 Jacobian, FP64 residual).
 *
 * Per element (src/snesiga_Tangent.c:104-190), with the energy written as
 * W = Phi(v(u)) over 12 variables (igab_math.cuh):
 *   K_e = sum_q sum_v s_qv x_qv x_qv^T + blockdiag_k(Gamma),
 * where x_qv[3a+k] = sum_m dv'/du_{k,m}(q) N_a^m(q) uses the variables after the
 * per-point rotation that diagonalises Phi'' (its one 2x2 block), and
 * s_qv = w_q lambda_v(q).  With y = sqrt|s| x and the rows split by the sign
 * of s,  K_main = Y_+^T Y_+ - Y_-^T Y_-.  A Gram product Y^T Y needs only two
 * TF32 products per k-step for FP32 accuracy: with y = y_hi + y_lo (y_hi TF32, 2 y_lo the
 * FP32 remainder, which the MMA reads truncated to TF32: an error of 2^-21 |y|),
 *   E = Y_hi^T Y_hi + Y_hi^T (2 Y_lo),   Y^T Y = (E + E^T)/2 + O(2^-21),
 * so the symmetric part taken at read-out recovers the cross term Y_lo^T Y_hi.
 * (2 y_lo stored unrounded saves one conversion per operand value.)
 * The geometric block, identical for the three displacement components, is
 *   Gamma(a,b) = sum_q [grad N_a^T S grad N_b + grad N_a . (T H_b) + (T H_a) . grad N_b]
 * (geo = [[S, T], [T^T, 0]], S the 3x3 first-derivative block, T the coupling to the
 * second derivatives H): 27 x 27 entries, computed on the FP32 FMA pipe by sum
 * factorisation, three contractions (z, y, x) with the 1-D tables, intermediates in the
 * free operand stage at the element's start.  Its 15 derivative-pair terms share their
 * (x, y) derivative orders in 12 classes and their x orders in 5, so the z contraction
 * yields 12 partial sums per (qx, qy, az, bz), the y contraction 5 per (qx, ay, by, az, bz)
 * and the x contraction reads 5 per point (64^3: 55.3 -> 46.9 ms against one contraction
 * chain per term; built as six U / V operand rows per point it took twelve tcgen05 chunks
 * per element whose construction cost more than the whole contraction does: 59.7 ms).
 *
 * Work per CTA: a 2x2x2 tile of elements of one of the 8 colours (the scatter
 * is conflict-free within a colour).  Warps 0-8 build, warp 9 issues MMAs.
 * Per element the builders compute the sum-factorised field at the 64 Gauss
 * points (FP64), the point integrand (FP64, 64 threads) and sign buckets of
 * the 768 (point, variable) rows, then build chunks of 32 rows into one of three
 * shared-memory stages (TF32 hi/lo in the K-major layout of
 * igab_tc.cuh; element-matrix column c sits at operand row tc_pos(c), so that a
 * builder thread's 9 outputs are 1024 bytes apart; each thread evaluates its row's
 * coefficients itself, which took 46.7 -> 43.3 ms at 64^3 against a pre-pass by 96
 * threads that the other builders waited for) and hand each to the issuer through
 * an mbarrier, on which the issuer spins (no suspension: 43.3 -> 43.1 ms).  The issuer
 * runs 4 k-steps of one MMA each per chunk (M 128: Y_hi; N 192: the whole stage) and
 * commits to the stage's mbarrier, which frees the stage for the chunk three later
 * (three stages rather than two: 43.1 -> 42.8 ms); negative-curvature rows use the
 * negate-A form.  Even chunks hold Y_hi then 2 Y_lo, odd chunks 2 Y_lo then Y_hi, so the
 * 192 accumulator columns take Y_hi^T Y_hi and Y_hi^T 2 Y_lo alternately: each half
 * sums half of each product (about 100 accumulating MMAs, half the magnitude), and the
 * read-out adds the halves.  The FP32 accumulation sets the rowwise agreement with the
 * FP64 reference: 4.4e-6 / 3.0e-6 / 5.9e-6 on three parity cases (41.2 ms at 64^3).
 * Two N 96 MMAs per k-step into two accumulators by chunk parity gave 4.5e-6 / 3.1e-6 /
 * 6.0e-6 at 41.7 ms; one N 192 MMA with Y_hi^T Y_hi always in columns 0-95 gave 39.6 ms
 * but 6.9e-6 / 4.9e-6 / 8.6e-6 (each column one FP32 sum over the whole element), and
 * the 64^3 Newton solve with FP32 tangents then took 14 steps instead of 7 (6 instead
 * of 5 with the FP64 polish).  Positive and negative chunks alternate while both last,
 * so that the running sums stay near the final values.  Tensor memory: 256 columns per
 * CTA; at most two CTAs per SM.  Rows 81-127 of the M side (for odd chunks rows 96-127
 * lie in the next stage or behind the stages) and columns 81-95 / 177-191 of the N side
 * read data that only feed accumulator rows and columns that are never read.  At the
 * end of an element the builders sum the two halves into shared memory, release the
 * accumulator to the issuer, take the
 * symmetric part, add Gamma on the k1 = k2 blocks and read-modify-write the
 * 81 x 81 values into the FP32 CSR values.
 */
#include <cuda_runtime.h>
#include "igab_device.cuh"
#include "igab_tc.cuh"

namespace {

#define TCN_BLD 288            /* builder warps 0-8: one operand task per thread per chunk */
#define TCN_THR 320            /* + warp 9: the MMA issuer */
#define TC_BAR_BLD 1           /* named barrier of the builder warps */
#define TC_STAGE 24576         /* bytes per operand stage */
#define TC_NS 3                /* operand stages */
#define TC_MAIN_LO 12288       /* the second operand half (B rows 96-191): 2 Y_lo in even chunks,
                                  Y_hi in odd ones; each half 81 rows and 15 free */
#define TC_TMEM_COLS 256u
#define TC_COL_MAIN 0u         /* the 192-column element-matrix accumulator */

/* float point data per Gauss point */
#define TP_F 0      /* F[k][J], 9 */
#define TP_G 9      /* G[k][c], 18 */
#define TP_CS 27    /* rotation of the (va, vb) block */
#define TP_SN 28
#define TP_RS 29    /* sign(s) sqrt|s|, 12 */
#define TP_C 41     /* the geometric block's 15 term coefficients: w sig_I (3), w d1[3 + I] (3),
                       2 w tau[I][K] (9) */
#define TP_N 57

template <int TE>
struct tc_smem {
    static constexpr int TC = TE + 2;
    static constexpr int NCP = TC * TC * TC;
    unsigned char stage[TC_NS][TC_STAGE];   /* operand stages; at an element's start the interpolation
                                               temporaries (stage 1) and the geometric block's
                                               intermediates (stage 0), E staging at read-out */
    double U[NCP * 3];
    double tab[3][TE][IGAB_TAB1D];
    double wh[3][TE][IGAB_NQ];
    float4 tabf[3][TE][IGAB_NQ][3];     /* FP32 1-D tables [d][element][q][function], derivatives 0-2 in x, y, z */
    float pt[IGAB_NQ3][TP_N];
    unsigned short map[2][768];         /* bucket slot -> 12 q + v (positive, negative) */
    int cnt[2];
    int vcnt[12][2][2];                 /* rows per (variable, point warp, sign) */
    long rbase[81];                     /* CSR row bases of the element matrix (elem_row_base) */
    int rsx[81], rsy[81];
    unsigned long long full[TC_NS];     /* stage b written (288 builder arrivals) */
    unsigned long long done[TC_NS];     /* MMAs of the chunk in stage b completed (commit) */
    unsigned long long freed;           /* the element's accumulator read out (288 builder arrivals) */
    unsigned long long drain;           /* issuer: every MMA it issued has completed */
    float gam[27 * 27];                 /* the element's geometric block (sum-factorised, FP32) */
    int ckind[TC_NS];                   /* chunk in stage b: 0 positive rows, 1 negative rows,
                                           3 end of tile; + 4 on an element's first chunk */
    unsigned int tmem_base;
    int abort_flag;
};


/* spin (no suspension) until the phase with the given parity completes; bounded, abortable */
__device__ __forceinline__ bool tc_mbar_spin_abortable(unsigned long long *bar, uint32_t parity,
                                                       const volatile int *abort)
{
    const uint32_t a = tc_smem_u32(bar);
    for (long i = 0; i < 64 * TC_WAIT_POLLS; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 1023) == 1023 && *abort) return false;
    }
    return false;
}

/* eigen-rotation of [[a, b], [b, c]]: [[a,b],[b,c]] = l1 e1 e1^T + l2 e2 e2^T,
 * e1 = (cs, -sn), e2 = (sn, cs) (same convention as the FP64 tensor kernel) */
__device__ __forceinline__ void tc_sym2_eig(double a, double b, double c, double &cs, double &sn, double &l1,
                                            double &l2)
{
    if (b == 0.0) {
        cs = 1.0; sn = 0.0; l1 = a; l2 = c;
        return;
    }
    double zeta = (c - a) / (2.0 * b);
    double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
    cs = 1.0 / sqrt(1.0 + t * t);
    sn = t * cs;
    l1 = a - t * b;
    l2 = c + t * b;
}

/* gradient of rotated variable v with respect to the 9 strain components of
 * displacement component k (igab_ge_grad_var, then the (va, vb) rotation) */
__device__ __forceinline__ void tc_grad_var(const float *p, int v, int k, float g[9])
{
#pragma unroll
    for (int m = 0; m < 9; m++) g[m] = 0.f;
    const float is2 = (float)IGAB_INV_SQRT2, is3 = (float)IGAB_INV_SQRT3, is6 = (float)IGAB_INV_SQRT6;
    const float F0 = p[TP_F + 3 * k], F1 = p[TP_F + 3 * k + 1], F2 = p[TP_F + 3 * k + 2];
    const float *G = p + TP_G + 6 * k;
    if (v == 0) {
        g[0] = F0 * is3; g[1] = F1 * is3; g[2] = F2 * is3;
    } else if (v <= 2) {
        const float cs = p[TP_CS], sn = p[TP_SN];
        const float a0 = F0 * is2, a1 = -F1 * is2;                        /* va */
        const float b0 = F0 * is6, b1 = F1 * is6, b2 = -2.f * F2 * is6;   /* vb */
        if (v == 1) { g[0] = cs * a0 - sn * b0; g[1] = cs * a1 - sn * b1; g[2] = -sn * b2; }
        else        { g[0] = sn * a0 + cs * b0; g[1] = sn * a1 + cs * b1; g[2] = cs * b2; }
    } else if (v == 3) {
        g[0] = 0.5f * F1; g[1] = 0.5f * F0;
    } else if (v == 4) {
        g[0] = 0.5f * F2; g[2] = 0.5f * F0;
    } else if (v == 5) {
        g[1] = 0.5f * F2; g[2] = 0.5f * F1;
    } else if (v == 6) {   /* strain-gradient variables: constant indices keep g[] in registers */
        g[0] = G[0] * is2; g[1] = -G[1] * is2; g[3] = F0 * is2; g[4] = -F1 * is2;
    } else if (v == 7) {
        g[0] = G[1] * is2; g[1] = -G[3] * is2; g[4] = F0 * is2; g[6] = -F1 * is2;
    } else if (v == 8) {
        g[0] = G[2] * is2; g[1] = -G[4] * is2; g[5] = F0 * is2; g[7] = -F1 * is2;
    } else if (v == 9) {
        g[0] = G[0] * is6; g[1] = G[1] * is6; g[2] = -2.f * G[2] * is6;
        g[3] = F0 * is6; g[4] = F1 * is6; g[5] = -2.f * F2 * is6;
    } else if (v == 10) {
        g[0] = G[1] * is6; g[1] = G[3] * is6; g[2] = -2.f * G[4] * is6;
        g[4] = F0 * is6; g[6] = F1 * is6; g[7] = -2.f * F2 * is6;
    } else {
        g[0] = G[2] * is6; g[1] = G[4] * is6; g[2] = -2.f * G[5] * is6;
        g[5] = F0 * is6; g[7] = F1 * is6; g[8] = -2.f * F2 * is6;
    }
}

/* operand row of element-matrix column c = 3 a + k, a = 9 ax + g: 8 g + 3 k + ax, or
 * 72 + g for k = ax = 2 (a bijection of 0..80 onto 0..80) */
__device__ __forceinline__ int tc_pos(int c)
{
    const int a = c / 3, cb = 3 * (c % 3) + a / 9, g = a % 9;
    return cb < 8 ? 8 * g + cb : 72 + g;
}

/* y = hi + lo: hi rounded to TF32 (exact in the MMA), 2 lo = 2 (y - hi) stored as FP32
 * (exact); the MMA reads it truncated to TF32, an error of at most 2^-21 |y| */
__device__ __forceinline__ void st_pair(unsigned char *hi_base, unsigned char *lo_base, uint32_t off, float y)
{
    const float h = tc_tf32(y);
    *reinterpret_cast<float *>(hi_base + off) = h;
    *reinterpret_cast<float *>(lo_base + off) = 2.f * (y - h);
}

/* pipeline state of a thread, carried across the tiles its CTA processes: the
 * builders track the commits they wait for, the issuer the arrivals it waits for */
struct tc_state {
    uint32_t ph_done[TC_NS];   /* builders: parity of the next wait on done[b] */
    bool pend[TC_NS];          /* builders: a chunk in stage b whose completion is not yet waited for */
    uint32_t ph_full[TC_NS];   /* issuer: parity of the next wait on full[b] */
    uint32_t ph_free;      /* issuer: parity of the next wait on freed */
    uint32_t ph_drain;
    int gc;                /* chunks (with MMAs) so far */
    int nelem;             /* elements (issuer: started) so far */
    bool aborted;
    uint32_t tmem;
};

/* barriers and tensor memory of the CTA (all threads) */
template <int TE>
__device__ __forceinline__ void tc_setup(tc_smem<TE> &S, tc_state &Q)
{
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        for (int b = 0; b < TC_NS; b++) {
            tc_mbar_init(&S.full[b], TCN_BLD);
            tc_mbar_init(&S.done[b], 1);
        }
        tc_mbar_init(&S.freed, TCN_BLD);
        tc_mbar_init(&S.drain, 1);
        tc_fence_mbar_init();
        S.abort_flag = 0;
    }
    if (warp == 0) tc_alloc(&S.tmem_base, TC_TMEM_COLS);
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    Q.tmem = S.tmem_base;
    for (int b = 0; b < TC_NS; b++) {
        Q.ph_done[b] = Q.ph_full[b] = 0u;
        Q.pend[b] = false;
    }
    Q.ph_free = Q.ph_drain = 0u;
    Q.gc = 0;
    Q.nelem = 0;
    Q.aborted = false;
}

/* release (all threads): the issuer has drained its MMAs; free the tensor memory */
template <int TE>
__device__ __forceinline__ void tc_release(tc_smem<TE> &S, tc_state &Q, int *status)
{
    const int tid = threadIdx.x, warp = tid >> 5;
    tc_fence_before_sync();
    __syncthreads();
    if (tid == 0 && S.abort_flag) atomicOr(status, 1);
    if (warp == 0) {
        tc_fence_after_sync();
        tc_dealloc(Q.tmem, TC_TMEM_COLS);
    }
}

/* the issuer warp for one tile: wait for each built chunk and issue its MMAs.
 * An element's chunks accumulate in one tensor-memory accumulator of 192 columns
 * (A = the chunk's Y_hi half, B = the whole stage); negative-curvature chunks use the
 * negate-A form.
 * Before the first MMA of an element the issuer waits until the builders have
 * read the previous element's accumulator.  Ends
 * at the builders' end-of-tile chunk; before returning it waits (bounded) until
 * every MMA it issued has completed. */
template <int TE>
__device__ __forceinline__ void tc_issue(tc_smem<TE> &S, tc_state &Q)
{
    const int lane = threadIdx.x & 31;
    const volatile int *abort = &S.abort_flag;
    bool ok = !*abort;
    bool started = false;   /* the accumulator holds this element's sums */
    while (ok) {
        const int b = Q.gc % TC_NS;
        if (lane == 0) ok = tc_mbar_spin_abortable(&S.full[b], Q.ph_full[b], abort);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        Q.ph_full[b] ^= 1u;
        if (!ok) break;
        int ck = 0;
        if (lane == 0) ck = S.ckind[b];   /* read by the thread that observed the arrival */
        ck = __shfl_sync(0xffffffffu, ck, 0);
        if (ck == 3) break;
        if (ck & 4) {
            /* first chunk of an element: the previous element's accumulators must be read out */
            if (Q.nelem > 0) {
                if (lane == 0) ok = tc_mbar_wait_abortable(&S.freed, Q.ph_free, abort);
                ok = __shfl_sync(0xffffffffu, ok, 0);
                Q.ph_free ^= 1u;
                if (!ok) break;
            }
            Q.nelem++;
            started = false;
        }
        const int kind = ck & 3;
        const int odd = Q.gc & 1;   /* odd chunks: 2 Y_lo first, then Y_hi, in the stage */
        const uint32_t acc0 = started ? 1u : 0u;
        started = true;
        if (lane == 0) {
            tc_fence_after_sync();
            const uint32_t sb = tc_smem_u32(S.stage[b]);
            const uint32_t idm = kind == 0 ? tc_idesc_tf32(128, 192) : tc_idesc_tf32(128, 192, true);
            const uint32_t d = Q.tmem + TC_COL_MAIN;
            const uint32_t sa = sb + (odd ? (uint32_t)TC_MAIN_LO : 0u);
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                /* A: Y_hi; B: the whole stage, 192 rows (Y_hi | 2 Y_lo, or 2 Y_lo | Y_hi) */
                tc_mma_tf32(d, tc_sdesc(sa + kk * TC_KSTEP_BYTES), tc_sdesc(sb + kk * TC_KSTEP_BYTES), idm,
                            kk == 0 ? acc0 : 1u);
            }
            tc_commit(&S.done[b]);
        }
        __syncwarp();
        Q.gc++;
    }
    if (!ok && lane == 0) S.abort_flag = 1;
    /* drain: the commit tracks every MMA this thread issued */
    if (lane == 0) {
        tc_commit(&S.drain);
        if (!tc_mbar_wait(&S.drain, Q.ph_drain)) S.abort_flag = 1;
    }
    Q.ph_drain ^= 1u;
    __syncwarp();
}

/* Sum the two 96-column halves of the element's accumulator into shared memory
 * (FP32, round to nearest): element-matrix rows by warps 0-2 / 4-6 (TMEM lanes = rows
 * 0-95, columns 0-47 / 48-95).  used: the accumulator holds this element's sums (none:
 * zeros). */
__device__ __forceinline__ void tc_readout(uint32_t tmem, bool used, int warp, int lane, float *E)
{
    if (warp < 8) {
        if (warp == 3 || warp == 7) return;   /* lanes 96-127: rows beyond 80 */
        const int lb = 32 * (warp & 3), half = warp >> 2, row = lb + lane;
#pragma unroll 1
        for (int part = 0; part < 3; part++) {
            const int c0 = 48 * half + 16 * part;
            float s[16];
#pragma unroll
            for (int i = 0; i < 16; i++) s[i] = 0.f;
#pragma unroll
            for (int b = 0; b < 2; b++) {
                if (!used) continue;   /* warp-uniform */
                float v[16];
                tc_ld16(tmem + ((uint32_t)lb << 16) + TC_COL_MAIN + (uint32_t)b * 96u + (uint32_t)c0, v);
#pragma unroll
                for (int i = 0; i < 16; i++) s[i] += v[i];
            }
            if (row < 81)
#pragma unroll
                for (int i = 0; i < 16; i++)
                    if (c0 + i < 81) E[row * 81 + c0 + i] = s[i];
        }
    }
}

/* the builder warps (threads 0..287) for one tile of up to TE^3 elements */
template <int TE>
__device__ __forceinline__ void tc_tile(const igab_geom &g, const tile_t &Tl, const double *__restrict__ U,
                                        float *__restrict__ vals, tc_smem<TE> &S, tc_state &Q)
{
    constexpr int TC = TE + 2;
    constexpr int NCP = TC * TC * TC;
    constexpr int NEL = TE * TE * TE;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    /* local copies of the pipeline state (registers), written back at the end */
    uint32_t ph[TC_NS];
    bool pend[TC_NS];
#pragma unroll
    for (int b = 0; b < TC_NS; b++) {
        ph[b] = Q.ph_done[b];
        pend[b] = Q.pend[b];
    }
    double *SA = reinterpret_cast<double *>(S.stage[1]);   /* interpolation temporaries */
    double *SC = SA + 972;
    int gc = Q.gc;
    bool aborted = Q.aborted;
    const uint32_t tmem = Q.tmem;
    const volatile int *abort = &S.abort_flag;

    for (int idx = tid; idx < NCP * 3; idx += TCN_BLD) {
        int i = idx % 3, cp = idx / 3;
        int lz = cp % TC, ly = (cp / TC) % TC, lx = cp / (TC * TC);
        double v = 0.0;
        if (lx < Tl.nv[0] + 2 && ly < Tl.nv[1] + 2 && lz < Tl.nv[2] + 2)
            v = U[3 * cp_index(g, Tl.e0[0] + lx, Tl.e0[1] + ly, Tl.e0[2] + lz) + i];
        S.U[idx] = v;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_TAB1D; idx += TCN_BLD) {
        int d = idx / (TE * IGAB_TAB1D), r = idx % (TE * IGAB_TAB1D), le = r / IGAB_TAB1D, o = r % IGAB_TAB1D;
        double t = le < Tl.nv[d] ? g.tab[d][(long)(Tl.e0[d] + le) * IGAB_TAB1D + o] : 0.0;
        S.tab[d][le][o] = t;
        reinterpret_cast<float *>(S.tabf[d][le])[(o / 3) * 4 + o % 3] = (float)t;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_NQ; idx += TCN_BLD) {
        int d = idx / (TE * IGAB_NQ), r = idx % (TE * IGAB_NQ), le = r / IGAB_NQ, q = r % IGAB_NQ;
        S.wh[d][le][q] = le < Tl.nv[d] ? g.wh[d][(long)(Tl.e0[d] + le) * IGAB_NQ + q] : 0.0;
    }
    tc_bar_sync(TC_BAR_BLD, TCN_BLD);

    for (int le = 0; le < NEL && !aborted; le++) {
        const int lex = le / (TE * TE), ley = (le / TE) % TE, lez = le % TE;
        if (!(lex < Tl.nv[0] && ley < Tl.nv[1] && lez < Tl.nv[2])) continue;   /* block-uniform */
        const double *Bx = S.tab[0][lex];
        const double *By = S.tab[1][ley];
        const double *Bz = S.tab[2][lez];
        /* ---- field at the 64 Gauss points (sum-factorised: z, then y, then x) */
        for (int o = tid; o < 972; o += TCN_BLD) {
            int i = o % 3, kz = (o / 3) % 3, ay = (o / 9) % 3, ax = (o / 27) % 3, q = o / 81;
            const double *u0 = &S.U[(((lex + ax) * TC + (ley + ay)) * TC + lez) * 3 + i];
            SA[o] = Bz[q * 9 + kz] * u0[0] + Bz[q * 9 + 3 + kz] * u0[3] + Bz[q * 9 + 6 + kz] * u0[6];
        }
        tc_bar_sync(TC_BAR_BLD, TCN_BLD);
        for (int o = tid; o < 864; o += TCN_BLD) {
            int i = o % 3, kk = (o / 3) % 6, ax = (o / 18) % 3, qq = o / 54;
            int qyy = qq & 3, qzz = qq >> 2;
            const double *a0 = &SA[((qzz * 3 + ax) * 3) * 9 + kk_kz(kk) * 3 + i];
            SC[o] = By[qyy * 9 + kk_ky(kk)] * a0[0] + By[qyy * 9 + 3 + kk_ky(kk)] * a0[9] +
                     By[qyy * 9 + 6 + kk_ky(kk)] * a0[18];
        }
        tc_bar_sync(TC_BAR_BLD, TCN_BLD);
        /* ---- point integrand (FP64), rotated curvatures, sign masks; q = 16 qz + 4 qy + qx */
        unsigned pmask = 0, nmask = 0;
        if (tid < IGAB_NQ3) {
            const int qx = tid & 3, qy = (tid >> 2) & 3, qz = tid >> 4, qq = qy + 4 * qz;
            double u[30];
#pragma unroll
            for (int a = 0; a < 10; a++)
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    double s = 0.0;
#pragma unroll
                    for (int ax = 0; ax < 3; ax++)
                        s += Bx[qx * 9 + ax * 3 + a_kx(a)] * SC[((qq * 3 + ax) * 6 + a_kk(a)) * 3 + i];
                    u[10 * i + a] = s;
                }
            if (g.periodic) {
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int J = 0; J < 3; J++) u[10 * i + 1 + J] += g.pp[3 * i + J];
            }
            igab_ge_point<double> P;
            igab_ge_eval(u, g.coef, P);
            const double w = S.wh[0][lex][qx] * S.wh[1][ley][qy] * S.wh[2][lez][qz] *
                             elem_scale(g, Tl.e0[0] + lex, Tl.e0[1] + ley, Tl.e0[2] + lez);
            double cs, sn, l1, l2;
            tc_sym2_eig(P.d2[1], P.d2ab, P.d2[2], cs, sn, l1, l2);
            float *pt = S.pt[tid];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int J = 0; J < 3; J++) pt[TP_F + 3 * k + J] = (float)P.F[k][J];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int c = 0; c < 6; c++) pt[TP_G + 6 * k + c] = (float)P.G[k][c];
            pt[TP_CS] = (float)cs;
            pt[TP_SN] = (float)sn;
#pragma unroll
            for (int v = 0; v < 12; v++) {
                const double s = w * (v == 1 ? l1 : (v == 2 ? l2 : P.d2[v]));
                const float r = sqrtf(fabsf((float)s));   /* FP32: the operand rows are FP32 */
                pt[TP_RS + v] = s < 0.0 ? -r : r;
                if (s > 0.0) pmask |= 1u << v;
                if (s < 0.0) nmask |= 1u << v;
            }
#pragma unroll
            for (int I = 0; I < 3; I++) pt[TP_C + I] = (float)(w * P.sig[I]);
#pragma unroll
            for (int I = 0; I < 3; I++) pt[TP_C + 3 + I] = (float)(w * P.d1[3 + I]);
#pragma unroll
            for (int I = 0; I < 3; I++)
#pragma unroll
                for (int K = 0; K < 3; K++) pt[TP_C + 6 + 3 * I + K] = (float)(2.0 * w * P.tau[I][K]);
        }
        /* ---- sign buckets in variable-major order: the slot of row (q, v) counts the
         * bucket's rows of smaller variables, then the points before q with the same
         * sign for v (ballot ranks over the two point warps).  Consecutive slots then
         * share their variable, so the coefficient evaluation branches alike across a warp. */
        if (tid < IGAB_NQ3) {
#pragma unroll 1
            for (int v = 0; v < 12; v++) {
                const unsigned pb = __ballot_sync(0xffffffffu, (pmask >> v) & 1u);
                const unsigned nb = __ballot_sync(0xffffffffu, (nmask >> v) & 1u);
                if (lane == 0) {
                    S.vcnt[v][warp][0] = __popc(pb);
                    S.vcnt[v][warp][1] = __popc(nb);
                }
            }
        }
        tc_bar_sync(TC_BAR_BLD, TCN_BLD);
        if (tid < IGAB_NQ3) {
            const unsigned lt = (1u << lane) - 1u;
            int po = 0, no = 0;   /* rows of the smaller variables */
#pragma unroll 1
            for (int v = 0; v < 12; v++) {
                const unsigned pb = __ballot_sync(0xffffffffu, (pmask >> v) & 1u);
                const unsigned nb = __ballot_sync(0xffffffffu, (nmask >> v) & 1u);
                if ((pmask >> v) & 1u)
                    S.map[0][po + (warp ? S.vcnt[v][0][0] : 0) + __popc(pb & lt)] = (unsigned short)(12 * tid + v);
                if ((nmask >> v) & 1u)
                    S.map[1][no + (warp ? S.vcnt[v][0][1] : 0) + __popc(nb & lt)] = (unsigned short)(12 * tid + v);
                po += S.vcnt[v][0][0] + S.vcnt[v][1][0];
                no += S.vcnt[v][0][1] + S.vcnt[v][1][1];
            }
            if (tid == 0) {
                S.cnt[0] = po;
                S.cnt[1] = no;
            }
        }
        tc_bar_sync(TC_BAR_BLD, TCN_BLD);
        const int npos = S.cnt[0], nneg = S.cnt[1];
        const int cpos = (npos + TC_KC - 1) / TC_KC, cneg = (nneg + TC_KC - 1) / TC_KC;
        const int nch = cpos + cneg;

        /* ---- geometric block by sum factorisation (FP32 FMA pipe).  The 15 terms fall
         * into 12 classes h of equal (x, y) derivative orders, and those into 5 classes G of
         * equal x orders: the z contraction sums each class h (Zs), the y contraction each
         * class G (Ys), the x contraction the 5 G.  Intermediates in the free operand stage. */
        {
            float *Zs = reinterpret_cast<float *>(S.stage[0]);   /* [12 h][16 (qx, qy)][9 (az, bz)] */
            float *Ys = Zs + 12 * 144;                           /* [5 G][4 qx][81 (ay, by, az, bz)] */
            if (tid < 144) {
                const int qxy = tid / 9, az = (tid % 9) / 3, bz = tid % 3;
                float z[12];
#pragma unroll
                for (int h = 0; h < 12; h++) z[h] = 0.f;
#pragma unroll
                for (int qz = 0; qz < 4; qz++) {
                    const float4 na = S.tabf[2][lez][qz][az], nb = S.tabf[2][lez][qz][bz];
                    const float *c = S.pt[16 * qz + qxy] + TP_C;
                    const float z00 = na.x * nb.x, z11 = na.y * nb.y, z01 = na.x * nb.y, z12 = na.y * nb.z;
                    z[0] += c[0] * z00 + c[8] * z01;     /* t 0, 8 */
                    z[1] += c[1] * z00 + c[11] * z01;    /* t 1, 11 */
                    z[2] += c[2] * z11 + c[14] * z12;    /* t 2, 14 */
                    z[3] += c[3] * z00;
                    z[4] += c[4] * z01;
                    z[5] += c[5] * z01;
                    z[6] += c[6] * z00;
                    z[7] += c[7] * z00;
                    z[8] += c[9] * z00;
                    z[9] += c[10] * z00;
                    z[10] += c[12] * z11;
                    z[11] += c[13] * z11;
                }
#pragma unroll
                for (int h = 0; h < 12; h++) Zs[h * 144 + tid] = z[h];
            }
            tc_bar_sync(TC_BAR_BLD, TCN_BLD);
            for (int o = tid; o < 324; o += TCN_BLD) {
                const int qx = o / 81, ay = (o / 27) % 3, by = (o / 9) % 3, azbz = o % 9;
                float G[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int qy = 0; qy < 4; qy++) {
                    const float4 na = S.tabf[1][ley][qy][ay], nb = S.tabf[1][ley][qy][by];
                    const float *zs = Zs + (4 * qy + qx) * 9 + azbz;
                    const float y00 = na.x * nb.x, y11 = na.y * nb.y, y01 = na.x * nb.y, y10 = na.y * nb.x,
                                y12 = na.y * nb.z;
                    G[0] += y00 * zs[0 * 144] + y01 * zs[7 * 144];
                    G[1] += y11 * zs[1 * 144] + y00 * zs[2 * 144] + y10 * zs[5 * 144] + y12 * zs[9 * 144] +
                            y01 * zs[11 * 144];
                    G[2] += y01 * zs[3 * 144] + y00 * zs[4 * 144];
                    G[3] += y00 * zs[6 * 144];
                    G[4] += y11 * zs[8 * 144] + y00 * zs[10 * 144];
                }
#pragma unroll
                for (int c = 0; c < 5; c++) Ys[c * 324 + o] = G[c];
            }
            tc_bar_sync(TC_BAR_BLD, TCN_BLD);
            for (int o = tid; o < 729; o += TCN_BLD) {
                const int a = o / 27, b = o % 27;
                const int ax = a / 9, bx = b / 9;
                const int yo = (3 * ((a / 3) % 3) + (b / 3) % 3) * 9 + 3 * (a % 3) + b % 3;
                float s = 0.f;
#pragma unroll
                for (int qx = 0; qx < 4; qx++) {
                    const float4 na = S.tabf[0][lex][qx][ax], nb = S.tabf[0][lex][qx][bx];
                    const float *ys = Ys + qx * 81 + yo;
                    s += na.y * nb.y * ys[0] + na.x * nb.x * ys[324] + na.y * nb.x * ys[2 * 324] +
                         na.y * nb.z * ys[3 * 324] + na.x * nb.y * ys[4 * 324];
                }
                S.gam[o] = s;
            }
            tc_bar_sync(TC_BAR_BLD, TCN_BLD);
        }

        /* ---- chunk loop: chunk ch is built into stage gc % 3 while the tensor core
         * works on the previous chunks; the element accumulates in tensor memory */
        const int cmain = cpos + cneg;
        const int cmin = min(cpos, cneg);
        for (int ch = 0; ch < nch; ch++) {
            const int b = gc % TC_NS;
            /* positive and negative chunks alternate while both last, so that the running
             * sum in the accumulator stays near the final value */
            const int cbk = ch < 2 * cmin ? (ch & 1) : (cpos > cneg ? 0 : 1);
            const int cix = ch < 2 * cmin ? (ch >> 1) : cmin + (ch - 2 * cmin);
            unsigned char *st = S.stage[b];
            /* stage b holds chunk gc-3: one thread waits for its MMAs (their operand reads
             * are complete once the commit arrives); the barrier passes that on to the
             * other builders */
            bool ok = true;
            if (pend[b]) {
                if (tid == 0) ok = tc_mbar_wait_abortable(&S.done[b], ph[b], abort);
                ph[b] ^= 1u;
                pend[b] = false;
            }
            if (!tc_bar_and(TC_BAR_BLD, TCN_BLD, ok)) { aborted = true; break; }
            if (ch < cpos + cneg) {
                /* main rows: task (slot j, component k, ax) -> 9 outputs (ay, az), column
                 * c = 3 (9 ax + 3 ay + az) + k at operand row tc_pos(c): row 8 g + 3 k + ax
                 * for g = 3 ay + az, or 72 + g for k = ax = 2, so the 9 stores sit at
                 * off0 + g * step (+ adj at g = 8) */
                const int bucket = cbk;
                const int slot = cix * TC_KC + tid / 9;
                const int j = tid / 9, k = (tid / 3) % 3, ax = tid % 3, cb = 3 * k + ax;
                const uint32_t off0 = (uint32_t)((j >> 2) * TC_LBO + (j & 3) * 4) +
                                      (cb < 8 ? (uint32_t)cb * 16u : 9u * TC_SBO);
                const uint32_t step = cb < 8 ? (uint32_t)TC_SBO : 16u;
                const uint32_t adj8 = cb < 8 ? 0u : (uint32_t)(TC_SBO - 128);
                /* odd chunks put 2 Y_lo first: the MMA's 192 columns then take Y_hi^T Y_hi and
                 * Y_hi^T 2 Y_lo alternately, so each half of the accumulator sums half of each */
                unsigned char *hi = st + ((gc & 1) ? TC_MAIN_LO : 0), *lo = st + ((gc & 1) ? 0 : TC_MAIN_LO);
                if (slot < (bucket ? nneg : npos)) {
                    const int id = S.map[bucket][slot], q = id / 12, v = id - 12 * q;
                    const int qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
                    /* the row's coefficients r d v'/d u_{k,m}, m = 0..8 (variable-major slots: v is
                     * nearly uniform across a warp) and the 1-D tables as float4 loads */
                    const float *p = S.pt[q];
                    float gv[9];
                    tc_grad_var(p, v, k, gv);
                    const float r = fabsf(p[TP_RS + v]);
                    const float4 bxv = S.tabf[0][lex][qx][ax];
                    const float bx0 = r * bxv.x, bx1 = r * bxv.y, bx2 = r * bxv.z;
                    /* coefficients of By[ky] per kz: derivative m -> (kx, ky, kz) as eval_Bspline */
                    const float t00 = gv[0] * bx1 + gv[3] * bx2, t01 = gv[1] * bx0 + gv[4] * bx1, t02 = gv[6] * bx0;
                    const float t10 = gv[2] * bx0 + gv[5] * bx1, t11 = gv[7] * bx0;
                    const float t20 = gv[8] * bx0;
                    float bz[9];
#pragma unroll
                    for (int i = 0; i < 3; i++) {
                        const float4 b4 = S.tabf[2][lez][qz][i];
                        bz[3 * i] = b4.x;
                        bz[3 * i + 1] = b4.y;
                        bz[3 * i + 2] = b4.z;
                    }
#pragma unroll
                    for (int ay = 0; ay < 3; ay++) {
                        const float4 byv = S.tabf[1][ley][qy][ay];
                        const float cy0 = t00 * byv.x + t01 * byv.y + t02 * byv.z;
                        const float cy1 = t10 * byv.x + t11 * byv.y;
                        const float cy2 = t20 * byv.x;
#pragma unroll
                        for (int az = 0; az < 3; az++) {
                            const float y = cy0 * bz[3 * az] + cy1 * bz[3 * az + 1] + cy2 * bz[3 * az + 2];
                            const int gg = 3 * ay + az;
                            st_pair(hi, lo, off0 + (uint32_t)gg * step + (gg == 8 ? adj8 : 0u), y);
                        }
                    }
                } else {
#pragma unroll
                    for (int gg = 0; gg < 9; gg++) {
                        const uint32_t off = off0 + (uint32_t)gg * step + (gg == 8 ? adj8 : 0u);
                        *reinterpret_cast<float *>(hi + off) = 0.f;
                        *reinterpret_cast<float *>(lo + off) = 0.f;
                    }
                }
            }
            /* hand the chunk to the issuer */
            const int ck = cbk | (ch == 0 ? 4 : 0);
            if (tid == 0) S.ckind[b] = ck;
            tc_fence_proxy_async();
            tc_mbar_arrive(&S.full[b]);
            pend[b] = true;
            gc++;
        }
        if (aborted) break;

        /* ---- all chunks of the element done (older stage first), accumulators -> shared memory */
        for (int k = 0; k < TC_NS && !aborted; k++) {
            const int b = (gc + k) % TC_NS;   /* chunk gc-3, gc-2, gc-1 */
            if (!pend[b]) continue;
            const bool ok = tid == 0 ? tc_mbar_wait_abortable(&S.done[b], ph[b], abort) : true;
            ph[b] ^= 1u;
            pend[b] = false;
            if (!tc_bar_and(TC_BAR_BLD, TCN_BLD, ok)) aborted = true;
        }
        if (aborted) break;
        const bool used = cmain > 0;
        float *E = reinterpret_cast<float *>(&S.stage[0][0]);   /* [81][81] */
        tc_fence_after_sync();
        tc_readout(tmem, used, warp, lane, E);
        tc_fence_before_sync();
        if (cmain > 0) tc_mbar_arrive(&S.freed);   /* the issuer saw this element only through its chunks */
        if (tid >= 192 && tid < 192 + 81)
            elem_row_base(g, Tl.e0[0] + lex, Tl.e0[1] + ley, Tl.e0[2] + lez, tid - 192, S.rbase[tid - 192],
                          S.rsx[tid - 192], S.rsy[tid - 192]);
        tc_fence_before_sync();
        tc_bar_sync(TC_BAR_BLD, TCN_BLD);
        /* ---- symmetric part + Gamma on the k1 = k2 blocks, added into the CSR values
         * with fire-and-forget reductions (red.global.add): the tiles of one colour
         * touch disjoint entries and the elements of a tile are separated by a
         * barrier, so every entry still receives its additions in a fixed order.
         * Thread (k1, c2), 243 of them, walks the rows c1 = 3 a1 + k1: the column's
         * position terms and the Gamma test are per-thread constants.  E is indexed by
         * operand rows (tc_pos). */
        if (tid < 243) {
            const int k1 = tid / 81, c2 = tid % 81, a2 = c2 / 3;
            const int q2 = tc_pos(c2);
            const bool gam = k1 == c2 % 3;
            const int o2 = c2 / 27, p2 = (c2 / 9) % 3, z2 = c2 % 9;
#pragma unroll 1
            for (int ax1 = 0; ax1 < 3; ax1++) {
                const int cb = 3 * k1 + ax1, pb = cb < 8 ? cb : 72, ps = cb < 8 ? 8 : 1;
#pragma unroll 3
                for (int g1 = 0; g1 < 9; g1++) {
                    const int a1 = 9 * ax1 + g1, c1 = 3 * a1 + k1, q1 = pb + ps * g1;
                    float v = 0.5f * (E[q1 * 81 + q2] + E[q2 * 81 + q1]);
                    if (gam) v += 0.5f * (S.gam[a1 * 27 + a2] + S.gam[a2 * 27 + a1]);
                    atomicAdd(&vals[S.rbase[c1] + o2 * S.rsx[c1] + p2 * S.rsy[c1] + z2], v);
                }
            }
        }
        tc_bar_sync(TC_BAR_BLD, TCN_BLD);
    }
    /* end of tile for the issuer (also after an abort: it stops at the flag) */
    if (aborted && tid == 0) S.abort_flag = 1;
    if (!aborted) {
        const int b = gc % TC_NS;
        if (tid == 0) S.ckind[b] = 3;
        tc_mbar_arrive(&S.full[b]);
    }
#pragma unroll
    for (int b = 0; b < TC_NS; b++) {
        Q.ph_done[b] = ph[b];
        Q.pend[b] = pend[b];
    }
    Q.gc = gc;
    Q.aborted = aborted;
}

template <int TE>
__global__ void __launch_bounds__(TCN_THR, 2) k_tan_tc32(igab_geom g, const double *__restrict__ U,
                                                         float *__restrict__ vals, int colour, int tile0,
                                                         int *status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    tc_smem<TE> &S = *reinterpret_cast<tc_smem<TE> *>(smem_raw);
    tile_t Tl;
    if (!decode_tile(g, TE, colour, tile0 + (int)blockIdx.x, Tl)) return;   /* block-uniform, before any barrier */
    tc_state Q;
    tc_setup<TE>(S, Q);
    if (threadIdx.x < TCN_BLD) tc_tile<TE>(g, Tl, U, vals, S, Q);
    else tc_issue<TE>(S, Q);
    tc_release<TE>(S, Q, status);
}

/* FP32 tangent over the tiles of every instance of a batch: one CTA per work item.
 * Each CTA takes the next item of the colour-major list from the batch counter when
 * it starts (not by its block index), so every item it may wait for (an earlier colour
 * of its instance) belongs to a CTA that started before it: the bounded waits always
 * make progress.  Per CTA the code is the single-mesh kernel's (a persistent loop over
 * items measured 1.8x slower per element: register spills across the item loop). */
__global__ void __launch_bounds__(TCN_THR, 2) k_tan_tc32_batch(igab_batch_dev B, const double *__restrict__ U,
                                                               float *__restrict__ vals)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    tc_smem<2> &S = *reinterpret_cast<tc_smem<2> *>(smem_raw);
    __shared__ batch_slot sl;
    if (!batch_next(B, sl)) return;   /* block-uniform, before any barrier of the tile */
    tc_state Q;
    tc_setup<2>(S, Q);
    if (threadIdx.x < TCN_BLD) {
        tile_t Tl;
        decode_tile(sl.g, 2, sl.colour, sl.tile, Tl);
        tc_tile<2>(sl.g, Tl, U + B.dof_off[sl.inst], vals + B.nnz_off[sl.inst], S, Q);
    } else {
        tc_issue<2>(S, Q);
    }
    tc_release<2>(S, Q, B.status);
    batch_done(B, sl);
}

/* ---------------------------------------------------------------- self-test
 * One CTA: A (128 x 32) and B (96 x 32) of small exact values in the operand
 * layout, D = A B^T with M 128 / N 96 (4 k-steps) into columns 0-95 and, for
 * a narrow shape, A B[0:32]^T with M 128 / N 32 into columns 96-127 (first
 * k-step overwrite, then accumulate), and with negate-A on k-steps 2-3 into
 * columns 128-159.  out[128][160] receives columns 0-159. */
__global__ void __launch_bounds__(128) k_tc_selftest(float *out, int *status)
{
    __shared__ __align__(128) unsigned char sm[16384 + 12288];
    __shared__ unsigned long long bar;
    __shared__ unsigned int tbase;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char *A = sm, *B = sm + 16384;
    for (int idx = tid; idx < 128 * 32; idx += 128) {
        const int m = idx / 32, k = idx % 32;
        *reinterpret_cast<float *>(A + tc_off(m, k)) = (float)((m * 5 + k * 3) % 13 - 6) * 0.5f;
    }
    for (int idx = tid; idx < 96 * 32; idx += 128) {
        const int n = idx / 32, k = idx % 32;
        *reinterpret_cast<float *>(B + tc_off(n, k)) = (float)((n * 7 + k) % 11 - 5) * 0.25f;
    }
    if (tid == 0) {
        tc_mbar_init(&bar, 1);
        tc_fence_mbar_init();
    }
    if (warp == 0) tc_alloc(&tbase, 256);
    tc_fence_proxy_async();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tm = tbase;
    if (tid == 0) {
        const uint32_t sa = tc_smem_u32(A), sb = tc_smem_u32(B);
        for (int kk = 0; kk < 4; kk++)
            tc_mma_tf32(tm, tc_sdesc(sa + kk * TC_KSTEP_BYTES), tc_sdesc(sb + kk * TC_KSTEP_BYTES),
                        tc_idesc_tf32(128, 96), kk > 0);
        for (int kk = 0; kk < 4; kk++)
            tc_mma_tf32(tm + 96, tc_sdesc(sa + kk * TC_KSTEP_BYTES), tc_sdesc(sb + kk * TC_KSTEP_BYTES),
                        tc_idesc_tf32(128, 32), kk > 0);
        /* negate-A: columns 128-159 = A B[0:32]^T for k-steps 0-1 minus it for k-steps 2-3 */
        for (int kk = 0; kk < 4; kk++)
            tc_mma_tf32(tm + 128, tc_sdesc(sa + kk * TC_KSTEP_BYTES), tc_sdesc(sb + kk * TC_KSTEP_BYTES),
                        tc_idesc_tf32(128, 32, kk >= 2), kk > 0);
        tc_commit(&bar);
    }
    __syncthreads();
    if (tid == 0 && !tc_mbar_wait(&bar, 0)) atomicOr(status, 1);
    __syncthreads();
    tc_fence_after_sync();
    for (int part = 0; part < 10; part++) {
        float v[16];
        tc_ld16(tm + ((uint32_t)(32 * warp) << 16) + 16u * part, v);
        for (int i = 0; i < 16; i++) out[(32 * warp + lane) * 160 + 16 * part + i] = v[i];
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after_sync();
        tc_dealloc(tm, 256);
    }
}

/* ---------------------------------------------------------------- peak probe
 * One CTA per SM, one thread issues `reps` back-to-back tcgen05.mma kind::tf32
 * M 128 x N n x K 8 into one accumulator (operands: zeros in shared memory). */
template <int N>
__global__ void __launch_bounds__(128) k_tc_peak(int reps, int *status)
{
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ unsigned long long bar;
    __shared__ unsigned int tb;
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int i = tid; i < 49152 / 4; i += blockDim.x) reinterpret_cast<float *>(sm)[i] = 0.f;
    if (tid == 0) {
        tc_mbar_init(&bar, 1);
        tc_fence_mbar_init();
    }
    if (warp == 0) tc_alloc(&tb, 256);
    tc_fence_proxy_async();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tm = tb;
    if (tid == 0) {
        const uint32_t sa = tc_smem_u32(sm), sb = sa + 16384;
        for (int r = 0; r < reps; r++)
            tc_mma_tf32(tm, tc_sdesc(sa + (r & 3) * TC_KSTEP_BYTES), tc_sdesc(sb + (r & 3) * TC_KSTEP_BYTES),
                        tc_idesc_tf32(128, N), r > 0);
        tc_commit(&bar);
        if (!tc_mbar_wait(&bar, 0)) atomicOr(status, 1);
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after_sync();
        tc_dealloc(tm, 256);
    }
}

template <int N>
int tc_peak_run(int nsm, double *tflops)
{
    const int reps = 4096;
    const size_t smem = 200000;   /* one CTA per SM */
    int *st = nullptr;
    IGAB_CUDA_TRY(cudaMalloc((void **)&st, sizeof(int)));
    cudaError_t e = cudaMemset(st, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_tc_peak<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaEvent_t a = nullptr, b = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess) {
        k_tc_peak<N><<<nsm, 128, smem>>>(reps, st);   /* warm-up */
        cudaEventRecord(a);
        k_tc_peak<N><<<nsm, 128, smem>>>(reps, st);
        cudaEventRecord(b);
        e = cudaEventSynchronize(b);
    }
    float ms = 0.f;
    int hs = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    if (e == cudaSuccess) e = cudaMemcpy(&hs, st, sizeof(int), cudaMemcpyDeviceToHost);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(st);
    if (e != cudaSuccess) {
        igab_set_error("igab_tc_peak: %s", cudaGetErrorString(e));
        return IGAB_ERR_CUDA;
    }
    if (hs) {
        igab_set_error("igab_tc_peak: completion wait timed out");
        return IGAB_ERR_CUDA;
    }
    *tflops = 2.0 * 128 * N * 8 * (double)reps * nsm / (ms * 1e-3) / 1e12;
    return 0;
}

} /* namespace */

extern "C" int igab_tc_peak(int device, int n_cols, double *tflops)
{
    if (!tflops) {
        igab_set_error("igab_tc_peak: null output");
        return IGAB_ERR_ARG;
    }
    IGAB_CUDA_TRY(cudaSetDevice(device));
    int nsm = 0;
    IGAB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    switch (n_cols) {
    case 32: return tc_peak_run<32>(nsm, tflops);
    case 96: return tc_peak_run<96>(nsm, tflops);
    case 256: return tc_peak_run<256>(nsm, tflops);
    default:
        igab_set_error("igab_tc_peak: n_cols must be 32, 96 or 256");
        return IGAB_ERR_ARG;
    }
}

int igab_launch_tan_tc32(igab_ctx *c, const double *dU, float *dv, int tx0, int tx1)
{
    igab_geom g = c->geom();
    const size_t sm = sizeof(tc_smem<2>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_tc32<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_tc32<2>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    /* 256 tensor-memory columns per CTA: at most two CTAs may share an SM */
    int per_sm = 0;
    IGAB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tan_tc32<2>, TCN_THR, sm));
    if (per_sm > 2 || per_sm < 1) {
        igab_set_error("k_tan_tc32: %d CTAs per SM (needs 1 or 2 for its tensor memory)", per_sm);
        return IGAB_ERR_UNSUPPORTED;
    }
    for (int k = 0; k < 8; k++) {
        const int colour = igab_colour_at(c->colour_order, k);
        long first = 0;
        const long nblk = tiles_of_colour_in(g, 2, colour, tx0, tx1, &first);
        if (nblk == 0) continue;
        k_tan_tc32<2><<<(unsigned)nblk, TCN_THR, sm, c->stream>>>(g, dU, dv, colour, (int)first, c->d_status);
        c->last_launches++;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_launch_tan_tc32_batch(const igab_batch_dev &B, int grid, cudaStream_t st, const double *dU, float *dv)
{
    (void)grid;   /* one CTA per work item; the hardware keeps at most two per SM (tensor memory) */
    const size_t sm = sizeof(tc_smem<2>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_tc32_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_tc32_batch, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    if (B.nitems == 0) return 0;
    k_tan_tc32_batch<<<B.nitems, TCN_THR, sm, st>>>(B, dU, dv);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_batch_occupancy_tc32(int *per_sm)
{
    const size_t sm = sizeof(tc_smem<2>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_tc32_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_tc32_batch, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    IGAB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_tan_tc32_batch, TCN_THR, sm));
    if (*per_sm > 2) *per_sm = 2;   /* 256 tensor-memory columns per CTA */
    return 0;
}

extern "C" int igab_tc_selftest(int device, float *out_host)
{
    if (!out_host) {
        igab_set_error("igab_tc_selftest: null output");
        return IGAB_ERR_ARG;
    }
    IGAB_CUDA_TRY(cudaSetDevice(device));
    float *d_out = nullptr;
    int *d_st = nullptr;
    IGAB_CUDA_TRY(cudaMalloc((void **)&d_out, 128 * 160 * sizeof(float)));
    cudaError_t e = cudaMalloc((void **)&d_st, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d_st, 0, sizeof(int));
    if (e == cudaSuccess) {
        k_tc_selftest<<<1, 128>>>(d_out, d_st);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    int st = 0;
    if (e == cudaSuccess) e = cudaMemcpy(out_host, d_out, 128 * 160 * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&st, d_st, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_out);
    cudaFree(d_st);
    if (e != cudaSuccess) {
        igab_set_error("igab_tc_selftest: %s", cudaGetErrorString(e));
        return IGAB_ERR_CUDA;
    }
    if (st) {
        igab_set_error("igab_tc_selftest: tensor-core completion wait timed out");
        return IGAB_ERR_CUDA;
    }
    return 0;
}
