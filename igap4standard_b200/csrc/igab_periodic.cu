/*
 * The owned system of a mesh with periodic directions (one rank).
 *
 * Along a periodic direction the reference owns nelem control points
 * (mesh/nurbs/nurbs_init.c:39) and assembles on a local grid of nelem + 2 points whose
 * last two are ghosts of owned points 0 and 1: the halo it sends to itself
 * (mesh/nurbs/nurbs_init.c:156-199 with npart = 1, exchanged by
 * src/snesiga_Residual.c:54-74).  Element contributions to a ghost row or column land in
 * the owner's global index through globalIdx (src/snesiga_init.c:84-110), the AIJ pattern
 * is every pair of owned points that share an element (src/snesiga_Tangent.c:189, first
 * MatSetValues pass), and the Dirichlet rows of the remaining (non-periodic) faces are
 * inserted last (src/snesiga_Residual.c:331-409, src/snesiga_Tangent.c:202-272).
 *
 * Here the volume and Neumann kernels run unchanged on the local grid (the context's
 * nb, ndof, nnz); this file gathers the owned U into the local grid, adds every local
 * row / entry into its owner in a fixed order (ascending local index; host-built
 * preimage lists, so the result is bitwise repeatable), and applies the Dirichlet rows
 * and columns on the owned system.  The owned pattern is a tensor product per direction:
 * the owned neighbours of owned index x are the owners of the local neighbours (distance
 * <= 2) of x's local preimages.
 */
#include <algorithm>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "igab_internal.h"

struct igab_periodic {
    int nbo[3];                        /* owned control points per direction */
    long ncp = 0, ndof = 0, nnz = 0;
    std::vector<int> rowptr_h, cols_h; /* owned AIJ pattern */
    int *d_own = nullptr;              /* [local ndof] owned dof of every local dof */
    int *d_rf_ptr = nullptr, *d_rf_idx = nullptr;   /* local dofs of each owned dof */
    int *d_kf_ptr = nullptr, *d_kf_idx = nullptr;   /* local entries of each owned entry */
    int *d_rowptr = nullptr, *d_cols = nullptr;
    long nd = 0;                       /* owned Dirichlet rows and values */
    int *d_drow = nullptr;
    double *d_dg = nullptr;
    unsigned char *d_isd = nullptr;    /* [ndof] 1 on a Dirichlet row */
    double *d_Ul = nullptr, *d_Rl = nullptr;        /* local-grid U and R */
    void *d_Vl = nullptr;              /* local-grid tangent values (FP64 size) */
};

namespace {

#define PER_THREADS 256

__global__ void k_per_gather(long n, const int *__restrict__ own, const double *__restrict__ Uo,
                             double *__restrict__ Ul)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) Ul[i] = Uo[own[i]];
}

__global__ void k_per_fold_res(long n, const int *__restrict__ ptr, const int *__restrict__ idx,
                               const double *__restrict__ Rl, double *__restrict__ Ro)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = ptr[i]; k < ptr[i + 1]; k++) s += Rl[idx[k]];
    Ro[i] = s;
}

template <typename T>
__global__ void k_per_fold_tan(long n, const int *__restrict__ ptr, const int *__restrict__ idx,
                               const T *__restrict__ Vl, T *__restrict__ Vo)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = ptr[i]; k < ptr[i + 1]; k++) s += (double)Vl[idx[k]];
    Vo[i] = (T)s;
}

/* R = U - g on the owned Dirichlet rows */
__global__ void k_per_res_dirichlet(long nd, const int *__restrict__ rows, const double *__restrict__ g,
                                    const double *__restrict__ U, double *__restrict__ R)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < nd) R[rows[i]] = U[rows[i]] - g[i];
}

/* Dirichlet rows and columns zeroed, unit diagonal on the Dirichlet rows (MatZeroRowsColumns) */
template <typename T>
__global__ void k_per_tan_dirichlet(long nrow, const int *__restrict__ rowptr, const int *__restrict__ cols,
                                    const unsigned char *__restrict__ isd, T *__restrict__ V)
{
    const long r = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (r >= nrow) return;
    const bool rd = isd[r] != 0;
    for (int k = rowptr[r]; k < rowptr[r + 1]; k++) {
        const int c = cols[k];
        if (rd) V[k] = c == r ? T(1) : T(0);
        else if (isd[c]) V[k] = T(0);
    }
}

unsigned blocks(long n)
{
    return (unsigned)((n + PER_THREADS - 1) / PER_THREADS);
}

template <typename T>
int upload(T **d, const std::vector<T> &h)
{
    IGAB_CUDA_TRY(cudaMalloc((void **)d, std::max<size_t>(h.size(), 1) * sizeof(T)));
    if (!h.empty()) IGAB_CUDA_TRY(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
}

} /* namespace */

long igab_periodic_ndof(const igab_ctx *c) { return c->per ? c->per->ndof : c->ndof; }
long igab_periodic_nnz(const igab_ctx *c) { return c->per ? c->per->nnz : c->nnz; }
const std::vector<int> &igab_periodic_rowptr(const igab_ctx *c) { return c->per->rowptr_h; }
const std::vector<int> &igab_periodic_cols(const igab_ctx *c) { return c->per->cols_h; }

void igab_periodic_release(igab_ctx *c)
{
    igab_periodic *p = c->per;
    if (!p) return;
    for (void *q : {(void *)p->d_own, (void *)p->d_rf_ptr, (void *)p->d_rf_idx, (void *)p->d_kf_ptr,
                    (void *)p->d_kf_idx, (void *)p->d_rowptr, (void *)p->d_cols, (void *)p->d_drow,
                    (void *)p->d_dg, (void *)p->d_isd, (void *)p->d_Ul, (void *)p->d_Rl, p->d_Vl})
        cudaFree(q);
    delete p;
    c->per = nullptr;
}

int igab_periodic_build(igab_ctx *c)
{
    igab_periodic *p = new igab_periodic();
    c->per = p;
    int nb[3], nbo[3];
    for (int d = 0; d < 3; d++) {
        nb[d] = c->nb[d];
        nbo[d] = c->periodic[d] ? c->ne[d] : c->nb[d];
        p->nbo[d] = nbo[d];
    }
    /* per direction: owner of a local index, and the sorted owned neighbours of an owned index */
    auto own1 = [&](int d, int a) { return c->periodic[d] && a >= nbo[d] ? a - nbo[d] : a; };
    std::vector<std::vector<int>> S[3];
    for (int d = 0; d < 3; d++) {
        S[d].resize(nbo[d]);
        for (int x = 0; x < nbo[d]; x++) {
            std::vector<int> &s = S[d][x];
            for (int a = x; a < nb[d]; a += nbo[d]) {   /* local preimages of x */
                for (int b = std::max(0, a - 2); b <= std::min(nb[d] - 1, a + 2); b++) s.push_back(own1(d, b));
                if (!c->periodic[d]) break;
            }
            std::sort(s.begin(), s.end());
            s.erase(std::unique(s.begin(), s.end()), s.end());
        }
    }
    auto pos1 = [&](int d, int x, int y) {   /* position of owned y among the neighbours of owned x */
        const std::vector<int> &s = S[d][x];
        return (int)(std::lower_bound(s.begin(), s.end(), y) - s.begin());
    };
    p->ncp = (long)nbo[0] * nbo[1] * nbo[2];
    p->ndof = 3 * p->ncp;
    /* owned pattern: S_x(x) x S_y(y) x S_z(z) x 3 components, lexicographic */
    p->rowptr_h.assign((size_t)p->ndof + 1, 0);
    long nnz = 0;
    for (int x = 0; x < nbo[0]; x++)
        for (int y = 0; y < nbo[1]; y++)
            for (int z = 0; z < nbo[2]; z++) {
                const long len = 3L * (long)S[0][x].size() * (long)S[1][y].size() * (long)S[2][z].size();
                const long r0 = 3L * (((long)x * nbo[1] + y) * nbo[2] + z);
                for (int k = 0; k < 3; k++) {
                    p->rowptr_h[(size_t)r0 + k] = (int)nnz;
                    nnz += len;
                }
            }
    if (nnz >= 2147483647L) {
        igab_set_error("igab_create: nonzero count exceeds int32 (PETSc AIJ index range)");
        return IGAB_ERR_ARG;
    }
    p->rowptr_h[(size_t)p->ndof] = (int)nnz;
    p->nnz = nnz;
    p->cols_h.resize((size_t)nnz);
    for (int x = 0; x < nbo[0]; x++)
        for (int y = 0; y < nbo[1]; y++)
            for (int z = 0; z < nbo[2]; z++)
                for (int k = 0; k < 3; k++) {
                    long o = p->rowptr_h[(size_t)3 * (((long)x * nbo[1] + y) * nbo[2] + z) + k];
                    for (int cx : S[0][x])
                        for (int cy : S[1][y])
                            for (int cz : S[2][z])
                                for (int kc = 0; kc < 3; kc++)
                                    p->cols_h[(size_t)o++] = (int)(3 * (((long)cx * nbo[1] + cy) * nbo[2] + cz) + kc);
                }
    /* local -> owned maps: dofs, and every entry of the local structured pattern */
    const long nl = c->ndof;
    std::vector<int> own((size_t)nl), rcount((size_t)p->ndof + 1, 0);
    std::vector<int> ktgt((size_t)c->nnz);
    long e = 0;
    for (int ax = 0; ax < nb[0]; ax++)
        for (int ay = 0; ay < nb[1]; ay++)
            for (int az = 0; az < nb[2]; az++) {
                const int ox = own1(0, ax), oy = own1(1, ay), oz = own1(2, az);
                const long ocp = ((long)ox * nbo[1] + oy) * nbo[2] + oz;
                const long lcp = ((long)ax * nb[1] + ay) * nb[2] + az;
                for (int k = 0; k < 3; k++) {
                    own[(size_t)(3 * lcp + k)] = (int)(3 * ocp + k);
                    const long orow = 3 * ocp + k;
                    const long base = p->rowptr_h[(size_t)orow];
                    const long ny = (long)S[1][oy].size(), nz = (long)S[2][oz].size();
                    for (int bx = std::max(0, ax - 2); bx <= std::min(nb[0] - 1, ax + 2); bx++) {
                        const long ix = pos1(0, ox, own1(0, bx));
                        for (int by = std::max(0, ay - 2); by <= std::min(nb[1] - 1, ay + 2); by++) {
                            const long iy = pos1(1, oy, own1(1, by));
                            for (int bz = std::max(0, az - 2); bz <= std::min(nb[2] - 1, az + 2); bz++) {
                                const long iz = pos1(2, oz, own1(2, bz));
                                for (int kc = 0; kc < 3; kc++) {
                                    if (e >= c->nnz) {
                                        igab_set_error("internal: periodic fold map overruns the local pattern");
                                        return IGAB_ERR_ARG;
                                    }
                                    ktgt[(size_t)e++] = (int)(base + ((ix * ny + iy) * nz + iz) * 3 + kc);
                                }
                            }
                        }
                    }
                }
            }
    if (e != c->nnz) {
        igab_set_error("internal: periodic fold map covers %ld of %ld local entries", e, c->nnz);
        return IGAB_ERR_ARG;
    }
    /* preimage lists by counting sort (ascending local index within each target) */
    auto invert = [](const std::vector<int> &tgt, long ntgt, std::vector<int> &ptr, std::vector<int> &idx) {
        ptr.assign((size_t)ntgt + 1, 0);
        for (int t : tgt) ptr[(size_t)t + 1]++;
        for (long i = 0; i < ntgt; i++) ptr[(size_t)i + 1] += ptr[(size_t)i];
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        idx.resize(tgt.size());
        for (size_t k = 0; k < tgt.size(); k++) idx[(size_t)fill[(size_t)tgt[k]]++] = (int)k;
    };
    std::vector<int> rf_ptr, rf_idx, kf_ptr, kf_idx;
    invert(own, p->ndof, rf_ptr, rf_idx);
    invert(ktgt, p->nnz, kf_ptr, kf_idx);
    for (long i = 0; i < p->nnz; i++)
        if (kf_ptr[(size_t)i + 1] == kf_ptr[(size_t)i]) {
            igab_set_error("internal: owned entry %ld has no local preimage", i);
            return IGAB_ERR_ARG;
        }
    int rc = 0;
    if ((rc = upload(&p->d_own, own)) || (rc = upload(&p->d_rf_ptr, rf_ptr)) || (rc = upload(&p->d_rf_idx, rf_idx)) ||
        (rc = upload(&p->d_kf_ptr, kf_ptr)) || (rc = upload(&p->d_kf_idx, kf_idx)) ||
        (rc = upload(&p->d_rowptr, p->rowptr_h)) || (rc = upload(&p->d_cols, p->cols_h)))
        return rc;
    IGAB_CUDA_TRY(cudaMalloc((void **)&p->d_isd, (size_t)p->ndof));
    IGAB_CUDA_TRY(cudaMemset(p->d_isd, 0, (size_t)p->ndof));
    return 0;
}

int igab_periodic_set_dirichlet(igab_ctx *c, const std::vector<int> &rows, const std::vector<double> &g)
{
    igab_periodic *p = c->per;
    if ((long)rows.size() != p->nd || (!p->d_drow && !rows.empty())) {
        cudaFree(p->d_drow);
        cudaFree(p->d_dg);
        p->d_drow = nullptr;
        p->d_dg = nullptr;
        p->nd = (long)rows.size();
        if (p->nd > 0) {
            IGAB_CUDA_TRY(cudaMalloc((void **)&p->d_drow, rows.size() * sizeof(int)));
            IGAB_CUDA_TRY(cudaMalloc((void **)&p->d_dg, g.size() * sizeof(double)));
        }
    }
    std::vector<unsigned char> isd((size_t)p->ndof, 0);
    for (int r : rows) isd[(size_t)r] = 1;
    if (p->nd > 0) {
        IGAB_CUDA_TRY(cudaMemcpy(p->d_drow, rows.data(), rows.size() * sizeof(int), cudaMemcpyHostToDevice));
        IGAB_CUDA_TRY(cudaMemcpy(p->d_dg, g.data(), g.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    IGAB_CUDA_TRY(cudaMemcpy(p->d_isd, isd.data(), isd.size(), cudaMemcpyHostToDevice));
    return 0;
}

int igab_periodic_gather(igab_ctx *c, const double *U_own, double *U_loc)
{
    k_per_gather<<<blocks(c->ndof), PER_THREADS, 0, c->stream>>>(c->ndof, c->per->d_own, U_own, U_loc);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

static int ensure_local(igab_ctx *c, bool vals)
{
    igab_periodic *p = c->per;
    if (!p->d_Ul) IGAB_CUDA_TRY(cudaMalloc((void **)&p->d_Ul, (size_t)c->ndof * sizeof(double)));
    if (!p->d_Rl) IGAB_CUDA_TRY(cudaMalloc((void **)&p->d_Rl, (size_t)c->ndof * sizeof(double)));
    if (vals && !p->d_Vl) IGAB_CUDA_TRY(cudaMalloc(&p->d_Vl, (size_t)c->nnz * sizeof(double)));
    return 0;
}

int igab_periodic_residual(igab_ctx *c, const double *U_own, double *R_own)
{
    igab_periodic *p = c->per;
    int rc = ensure_local(c, false);
    if (rc) return rc;
    if ((rc = igab_periodic_gather(c, U_own, p->d_Ul))) return rc;
    if ((rc = igab_launch_residual(c, p->d_Ul, p->d_Rl))) return rc;   /* c->nd = 0: no local Dirichlet rows */
    int launches = c->last_launches + 1;
    k_per_fold_res<<<blocks(p->ndof), PER_THREADS, 0, c->stream>>>(p->ndof, p->d_rf_ptr, p->d_rf_idx, p->d_Rl, R_own);
    launches++;
    if (p->nd > 0) {
        k_per_res_dirichlet<<<blocks(p->nd), PER_THREADS, 0, c->stream>>>(p->nd, p->d_drow, p->d_dg, U_own, R_own);
        launches++;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    c->last_launches = launches;
    return 0;
}

int igab_periodic_tangent(igab_ctx *c, const double *U_own, void *V_own, int prec)
{
    igab_periodic *p = c->per;
    int rc = ensure_local(c, true);
    if (rc) return rc;
    if ((rc = igab_periodic_gather(c, U_own, p->d_Ul))) return rc;
    if ((rc = igab_launch_tangent(c, p->d_Ul, p->d_Vl, prec))) return rc;
    int launches = c->last_launches + 1;
    if (prec == IGAB_PREC_FP64) {
        k_per_fold_tan<double><<<blocks(p->nnz), PER_THREADS, 0, c->stream>>>(p->nnz, p->d_kf_ptr, p->d_kf_idx,
                                                                               (const double *)p->d_Vl, (double *)V_own);
        if (p->nd > 0)
            k_per_tan_dirichlet<double><<<blocks(p->ndof), PER_THREADS, 0, c->stream>>>(p->ndof, p->d_rowptr, p->d_cols,
                                                                                       p->d_isd, (double *)V_own);
    } else {
        k_per_fold_tan<float><<<blocks(p->nnz), PER_THREADS, 0, c->stream>>>(p->nnz, p->d_kf_ptr, p->d_kf_idx,
                                                                              (const float *)p->d_Vl, (float *)V_own);
        if (p->nd > 0)
            k_per_tan_dirichlet<float><<<blocks(p->ndof), PER_THREADS, 0, c->stream>>>(p->ndof, p->d_rowptr, p->d_cols,
                                                                                      p->d_isd, (float *)V_own);
    }
    launches += p->nd > 0 ? 2 : 1;
    IGAB_CUDA_TRY(cudaGetLastError());
    c->last_launches = launches;
    return 0;
}

int igab_periodic_dirichlet_rows(igab_ctx *c, long *n, int *rows)
{
    igab_periodic *p = c->per;
    *n = p->nd;
    if (rows && p->nd > 0) {
        IGAB_CUDA_TRY(cudaStreamSynchronize(c->stream));
        IGAB_CUDA_TRY(cudaMemcpy(rows, p->d_drow, (size_t)p->nd * sizeof(int), cudaMemcpyDeviceToHost));
    }
    return 0;
}
