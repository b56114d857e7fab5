/*
 * Batched assembly: many independent single-rank meshes (uneven sizes, their
 * own material constants and boundary tables) assembled by ONE persistent
 * launch per operator.
 *
 * The reference assembles one mesh per process (src/snesiga_Residual.c:13,
 * src/snesiga_Tangent.c:13); a batch is that loop over instances, each
 * instance exactly the single-mesh assembly of its own igab_ctx.  Unknowns of
 * instance i occupy U[dof_off[i] .. dof_off[i+1]) and its CSR values
 * vals[nnz_off[i] .. nnz_off[i+1]), in the instance's own numbering and AIJ
 * pattern.
 *
 * Schedule: the work list holds every (instance, colour, tile) of 2x2x2-element
 * tiles, colour-major (all colour-0 tiles of all instances, then colour 1,
 * ...), instances in natural order or largest first.  The persistent CTAs take
 * items from an atomic counter; a tile of colour c waits (bounded) until every
 * earlier colour of its instance is complete, so the read-modify-write
 * accumulation stays free of atomics and its per-entry order is the
 * single-mesh one: batched results equal the per-instance results bit for bit.
 * Colour-major order makes those waits rare: the colour-(c-1) tiles of an
 * instance were handed out a whole colour sweep earlier.
 */
#include <algorithm>
#include <numeric>
#include <vector>
#include <cuda_runtime.h>
#include "igab_device.cuh"

struct igab_batch {
    int device = 0, n = 0, nsm = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<igab_ctx *> inst;
    std::vector<long> dof_off, nnz_off;   /* n + 1 */
    long nel = 0;
    /* device work list and synchronisation */
    igab_geom *d_geoms = nullptr;
    int4 *d_items = nullptr;
    int nitems = 0;
    int *d_sync = nullptr;   /* counter, then done[8 n] */
    int *d_need = nullptr;
    long *d_dof_off = nullptr, *d_nnz_off = nullptr;
    int *d_status = nullptr;
    /* Dirichlet rows of all instances */
    long nd = 0;
    int *d_drow_g = nullptr, *d_dinst = nullptr, *d_drow_l = nullptr;
    double *d_dg = nullptr;
    /* schedule: CTAs per SM of the persistent kernels (0 = as many as fit), instance order */
    int ctas[3] = {0, 0, 0};
    int order = 0;
    int colour_order = 0;   /* igab_colour_order of the work list */
    /* colour-dependency wait: poll limit, and the test switch that makes it run out */
    long spin_limit = IGAB_BATCH_SPIN;
    int hold = 0;
    int last_launches = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
};

namespace {

void free_batch(igab_batch *b)
{
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_geoms); cudaFree(b->d_items); cudaFree(b->d_sync); cudaFree(b->d_need);
    cudaFree(b->d_dof_off); cudaFree(b->d_nnz_off); cudaFree(b->d_status);
    cudaFree(b->d_drow_g); cudaFree(b->d_dinst); cudaFree(b->d_drow_l); cudaFree(b->d_dg);
    for (igab_ctx *c : b->inst) igab_destroy(c);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

/* work list in the current orders; need[8 i + p] = tiles of instance i at sweep position p */
int build_items(igab_batch *b)
{
    std::vector<int> ord(b->n);
    std::iota(ord.begin(), ord.end(), 0);
    if (b->order == 1)
        std::stable_sort(ord.begin(), ord.end(), [b](int x, int y) { return b->inst[x]->nel > b->inst[y]->nel; });
    std::vector<int4> items;
    std::vector<int> need(8 * (size_t)b->n, 0);
    for (int p = 0; p < 8; p++) {
        const int c = igab_colour_at(b->colour_order, p);
        for (int i : ord) {
            const igab_geom g = b->inst[i]->geom();
            const long nt = tiles_of_colour(g, 2, c);
            need[8 * (size_t)i + p] = (int)nt;
            for (long t = 0; t < nt; t++) items.push_back(make_int4(i, p, (int)t, c));
        }
    }
    if (b->d_items && (int)items.size() != b->nitems) {
        igab_set_error("internal: batch work list changed size");
        return IGAB_ERR_ARG;
    }
    b->nitems = (int)items.size();
    if (!b->d_items) IGAB_CUDA_TRY(cudaMalloc((void **)&b->d_items, items.size() * sizeof(int4)));
    if (!b->d_need) IGAB_CUDA_TRY(cudaMalloc((void **)&b->d_need, need.size() * sizeof(int)));
    IGAB_CUDA_TRY(cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
    IGAB_CUDA_TRY(cudaMemcpy(b->d_need, need.data(), need.size() * sizeof(int), cudaMemcpyHostToDevice));
    return 0;
}

/* geometry / parameters and Dirichlet rows of every instance -> device (in place) */
int refresh(igab_batch *b)
{
    std::vector<igab_geom> geoms(b->n);
    for (int i = 0; i < b->n; i++) geoms[i] = b->inst[i]->geom();
    IGAB_CUDA_TRY(cudaMemcpy(b->d_geoms, geoms.data(), geoms.size() * sizeof(igab_geom), cudaMemcpyHostToDevice));
    std::vector<int> rg, ri, rl;
    std::vector<double> dg;
    for (int i = 0; i < b->n; i++) {
        igab_ctx *c = b->inst[i];
        if (c->nd <= 0) continue;
        std::vector<int> rows(c->nd);
        std::vector<double> vals(c->nd);
        IGAB_CUDA_TRY(cudaMemcpy(rows.data(), c->d_drow, c->nd * sizeof(int), cudaMemcpyDeviceToHost));
        IGAB_CUDA_TRY(cudaMemcpy(vals.data(), c->d_dg, c->nd * sizeof(double), cudaMemcpyDeviceToHost));
        for (long j = 0; j < c->nd; j++) {
            rg.push_back((int)(b->dof_off[i] + rows[j]));
            ri.push_back(i);
            rl.push_back(rows[j]);
            dg.push_back(vals[j]);
        }
    }
    if ((long)rg.size() != b->nd || (!b->d_drow_g && !rg.empty())) {
        cudaFree(b->d_drow_g); cudaFree(b->d_dinst); cudaFree(b->d_drow_l); cudaFree(b->d_dg);
        b->d_drow_g = b->d_dinst = b->d_drow_l = nullptr;
        b->d_dg = nullptr;
        b->nd = (long)rg.size();
        if (b->nd > 0) {
            IGAB_CUDA_TRY(cudaMalloc((void **)&b->d_drow_g, b->nd * sizeof(int)));
            IGAB_CUDA_TRY(cudaMalloc((void **)&b->d_dinst, b->nd * sizeof(int)));
            IGAB_CUDA_TRY(cudaMalloc((void **)&b->d_drow_l, b->nd * sizeof(int)));
            IGAB_CUDA_TRY(cudaMalloc((void **)&b->d_dg, b->nd * sizeof(double)));
        }
    }
    if (b->nd > 0) {
        IGAB_CUDA_TRY(cudaMemcpy(b->d_drow_g, rg.data(), rg.size() * sizeof(int), cudaMemcpyHostToDevice));
        IGAB_CUDA_TRY(cudaMemcpy(b->d_dinst, ri.data(), ri.size() * sizeof(int), cudaMemcpyHostToDevice));
        IGAB_CUDA_TRY(cudaMemcpy(b->d_drow_l, rl.data(), rl.size() * sizeof(int), cudaMemcpyHostToDevice));
        IGAB_CUDA_TRY(cudaMemcpy(b->d_dg, dg.data(), dg.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    return 0;
}

igab_batch_dev dev_view(const igab_batch *b)
{
    igab_batch_dev B;
    B.geoms = b->d_geoms;
    B.items = b->d_items;
    B.nitems = b->nitems;
    B.counter = b->d_sync;
    B.done = b->d_sync + 1;
    B.need = b->d_need;
    B.dof_off = b->d_dof_off;
    B.nnz_off = b->d_nnz_off;
    B.status = b->d_status;
    B.spin_limit = b->spin_limit;
    B.hold = b->hold;
    return B;
}

/* persistent grid: SM count x CTAs per SM (occupancy, capped by the schedule knob) */
int grid_of(const igab_batch *b, int what, int *grid)
{
    int per = 0, rc;
    if (what == 0) rc = igab_batch_occupancy_res(&per);
    else if (what == 1) rc = igab_batch_occupancy_dmma(&per);
    else rc = igab_batch_occupancy_tc32(&per);
    if (rc) return rc;
    if (per < 1) {
        igab_set_error("batch kernel %d does not fit on an SM", what);
        return IGAB_ERR_UNSUPPORTED;
    }
    if (b->ctas[what] > 0 && b->ctas[what] < per) per = b->ctas[what];
    *grid = per * b->nsm;
    return 0;
}

int reset_sync(igab_batch *b)
{
    IGAB_CUDA_TRY(cudaMemsetAsync(b->d_sync, 0, (1 + 8 * (size_t)b->n) * sizeof(int), b->stream));
    return 0;
}

int launch_residual(igab_batch *b, const double *dU, double *dR)
{
    int grid = 0, rc = grid_of(b, 0, &grid);
    if (rc) return rc;
    IGAB_CUDA_TRY(cudaMemsetAsync(dR, 0, (size_t)b->dof_off[b->n] * sizeof(double), b->stream));
    if ((rc = reset_sync(b))) return rc;
    if ((rc = igab_launch_res_batch(dev_view(b), grid, b->stream, dU, dR))) return rc;
    b->last_launches = 1;
    if (b->nd > 0) {
        /* R = U - g on the Dirichlet rows of every instance (src/snesiga_Residual.c:326-412) */
        if ((rc = igab_launch_res_dirichlet_rows(b->nd, b->d_drow_g, b->d_dg, dU, dR, b->stream))) return rc;
        b->last_launches++;
    }
    return 0;
}

int launch_tangent(igab_batch *b, const double *dU, void *dv, int prec)
{
    const int what = prec == IGAB_PREC_FP64 ? 1 : 2;
    int grid = 0, rc = grid_of(b, what, &grid);
    if (rc) return rc;
    const size_t es = prec == IGAB_PREC_FP64 ? sizeof(double) : sizeof(float);
    IGAB_CUDA_TRY(cudaMemsetAsync(dv, 0, (size_t)b->nnz_off[b->n] * es, b->stream));
    if ((rc = reset_sync(b))) return rc;
    if (prec == IGAB_PREC_FP64) rc = igab_launch_tan_dmma_batch(dev_view(b), grid, b->stream, dU, (double *)dv);
    else rc = igab_launch_tan_tc32_batch(dev_view(b), grid, b->stream, dU, (float *)dv);
    if (rc) return rc;
    b->last_launches = 1;
    if (b->nd > 0) {
        if ((rc = igab_launch_tan_dirichlet_batch(dev_view(b), b->nd, b->d_dinst, b->d_drow_l, dv, prec, b->stream)))
            return rc;
        b->last_launches++;
    }
    return 0;
}

int check_batch_status(igab_batch *b)
{
    int st = 0;
    IGAB_CUDA_TRY(cudaMemcpy(&st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) {
        IGAB_CUDA_TRY(cudaMemset(b->d_status, 0, sizeof(int)));
        igab_set_error("batched assembly: a bounded wait gave up (status %d: 1 tensor-core completion, "
                       "2 colour dependency)", st);
        return IGAB_ERR_CUDA;
    }
    return 0;
}

} /* namespace */

#define BATCH_CHECK(cond, msg)             \
    do {                                   \
        if (!(cond)) {                     \
            igab_set_error("%s", msg);     \
            return IGAB_ERR_ARG;           \
        }                                  \
    } while (0)

extern "C" int igab_batch_create(const igab_mesh_desc *descs, int n, int device, igab_batch **out)
{
    BATCH_CHECK(descs && n > 0 && out, "igab_batch_create: bad argument");
    *out = nullptr;
    for (int i = 0; i < n; i++)
        if (descs[i].phys != IGAB_PHYS_GE) {
            igab_set_error("igab_batch_create: instance %d: batched assembly is built for phys/ge only", i);
            return IGAB_ERR_UNSUPPORTED;
        }
    for (int i = 0; i < n; i++)
        if (descs[i].bc_periodic[0] || descs[i].bc_periodic[1] || descs[i].bc_periodic[2]) {
            igab_set_error("igab_batch_create: instance %d: batched assembly takes non-periodic meshes", i);
            return IGAB_ERR_UNSUPPORTED;
        }
    IGAB_CUDA_TRY(cudaSetDevice(device));
    igab_batch *b = new igab_batch;
    b->device = device;
    b->n = n;
    int rc = 0;
    cudaError_t ce = cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, device);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
        igab_set_error("igab_batch_create: %s", cudaGetErrorString(ce));
        delete b;
        return IGAB_ERR_CUDA;
    }
    b->own_stream = true;
    b->dof_off.assign(n + 1, 0);
    b->nnz_off.assign(n + 1, 0);
    for (int i = 0; i < n; i++) {
        igab_ctx *c = nullptr;
        if ((rc = igab_create(&descs[i], device, &c))) {
            free_batch(b);
            return rc;
        }
        /* every instance works on the batch stream (igab_create made one of its own) */
        if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
        c->stream = b->stream;
        c->own_stream = false;
        b->inst.push_back(c);
        b->dof_off[i + 1] = b->dof_off[i] + c->ndof;
        b->nnz_off[i + 1] = b->nnz_off[i] + c->nnz;
        b->nel += c->nel;
    }
#define BTRY(call)                                                                 \
    do {                                                                           \
        cudaError_t _e = (call);                                                   \
        if (_e != cudaSuccess) {                                                   \
            igab_set_error("igab_batch_create: %s: %s", #call, cudaGetErrorString(_e)); \
            free_batch(b);                                                         \
            return IGAB_ERR_CUDA;                                                  \
        }                                                                          \
    } while (0)
    BTRY(cudaMalloc((void **)&b->d_geoms, (size_t)n * sizeof(igab_geom)));
    BTRY(cudaMalloc((void **)&b->d_sync, (1 + 8 * (size_t)n) * sizeof(int)));
    BTRY(cudaMalloc((void **)&b->d_dof_off, (size_t)(n + 1) * sizeof(long)));
    BTRY(cudaMalloc((void **)&b->d_nnz_off, (size_t)(n + 1) * sizeof(long)));
    BTRY(cudaMalloc((void **)&b->d_status, sizeof(int)));
    BTRY(cudaMemset(b->d_status, 0, sizeof(int)));
    BTRY(cudaMemcpy(b->d_dof_off, b->dof_off.data(), (n + 1) * sizeof(long), cudaMemcpyHostToDevice));
    BTRY(cudaMemcpy(b->d_nnz_off, b->nnz_off.data(), (n + 1) * sizeof(long), cudaMemcpyHostToDevice));
#undef BTRY
    if ((rc = refresh(b)) || (rc = build_items(b))) {
        free_batch(b);
        return rc;
    }
    *out = b;
    return 0;
}

extern "C" int igab_batch_destroy(igab_batch *b)
{
    if (!b) return 0;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    /* the instances' streams are the batch stream: let free_batch destroy it once */
    free_batch(b);
    return 0;
}

extern "C" int igab_batch_sizes(const igab_batch *b, long *ndof, long *nnz, long *nelem, long *dof_offsets,
                                long *nnz_offsets)
{
    BATCH_CHECK(b, "igab_batch_sizes: null batch");
    if (ndof) *ndof = b->dof_off[b->n];
    if (nnz) *nnz = b->nnz_off[b->n];
    if (nelem) *nelem = b->nel;
    if (dof_offsets) std::copy(b->dof_off.begin(), b->dof_off.end(), dof_offsets);
    if (nnz_offsets) std::copy(b->nnz_off.begin(), b->nnz_off.end(), nnz_offsets);
    return 0;
}

extern "C" igab_ctx *igab_batch_instance(igab_batch *b, int i)
{
    if (!b || i < 0 || i >= b->n) return nullptr;
    return b->inst[i];
}

extern "C" int igab_batch_refresh(igab_batch *b)
{
    BATCH_CHECK(b, "igab_batch_refresh: null batch");
    IGAB_CUDA_TRY(cudaSetDevice(b->device));
    IGAB_CUDA_TRY(cudaStreamSynchronize(b->stream));
    return refresh(b);
}

extern "C" int igab_batch_set_stream(igab_batch *b, void *cuda_stream)
{
    BATCH_CHECK(b, "igab_batch_set_stream: null batch");
    IGAB_CUDA_TRY(cudaSetDevice(b->device));
    IGAB_CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (b->own_stream) cudaStreamDestroy(b->stream);
    b->stream = (cudaStream_t)cuda_stream;
    b->own_stream = false;
    for (igab_ctx *c : b->inst) c->stream = b->stream;
    return 0;
}

extern "C" int igab_batch_set_schedule(igab_batch *b, int ctas_res, int ctas_tan64, int ctas_tan32, int order)
{
    BATCH_CHECK(b, "igab_batch_set_schedule: null batch");
    BATCH_CHECK(ctas_res >= 0 && ctas_tan64 >= 0 && ctas_tan32 >= 0 && (order == 0 || order == 1),
                "igab_batch_set_schedule: bad argument");
    IGAB_CUDA_TRY(cudaSetDevice(b->device));
    IGAB_CUDA_TRY(cudaStreamSynchronize(b->stream));
    b->ctas[0] = ctas_res;
    b->ctas[1] = ctas_tan64;
    b->ctas[2] = ctas_tan32;
    if (order != b->order) {
        b->order = order;
        return build_items(b);
    }
    return 0;
}

extern "C" int igab_batch_set_colour_order(igab_batch *b, int colour_order)
{
    BATCH_CHECK(b, "igab_batch_set_colour_order: null batch");
    BATCH_CHECK(colour_order >= 0 && colour_order <= 2, "igab_batch_set_colour_order: order must be 0, 1 or 2");
    IGAB_CUDA_TRY(cudaSetDevice(b->device));
    IGAB_CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (colour_order != b->colour_order) {
        b->colour_order = colour_order;
        return build_items(b);
    }
    return 0;
}

extern "C" int igab_batch_get_colour_order(const igab_batch *b, int *colour_order)
{
    BATCH_CHECK(b && colour_order, "igab_batch_get_colour_order: null argument");
    *colour_order = b->colour_order;
    return 0;
}

extern "C" int igab_batch_get_schedule(const igab_batch *b, int *ctas_res, int *ctas_tan64, int *ctas_tan32,
                                       int *order)
{
    BATCH_CHECK(b, "igab_batch_get_schedule: null batch");
    if (ctas_res) *ctas_res = b->ctas[0];
    if (ctas_tan64) *ctas_tan64 = b->ctas[1];
    if (ctas_tan32) *ctas_tan32 = b->ctas[2];
    if (order) *order = b->order;
    return 0;
}

extern "C" int igab_batch_residual_device(igab_batch *b, const double *U_dev, double *R_dev)
{
    BATCH_CHECK(b && U_dev && R_dev, "igab_batch_residual_device: null argument");
    IGAB_CUDA_TRY(cudaSetDevice(b->device));
    return launch_residual(b, U_dev, R_dev);
}

extern "C" int igab_batch_tangent_device(igab_batch *b, const double *U_dev, void *vals_dev, int prec)
{
    BATCH_CHECK(b && U_dev && vals_dev, "igab_batch_tangent_device: null argument");
    BATCH_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_batch_tangent_device: bad precision");
    IGAB_CUDA_TRY(cudaSetDevice(b->device));
    return launch_tangent(b, U_dev, vals_dev, prec);
}

extern "C" int igab_batch_sync(igab_batch *b)
{
    BATCH_CHECK(b, "igab_batch_sync: null batch");
    IGAB_CUDA_TRY(cudaSetDevice(b->device));
    IGAB_CUDA_TRY(cudaStreamSynchronize(b->stream));
    return check_batch_status(b);
}

extern "C" int igab_batch_set_wait_limit(igab_batch *b, long polls, int unreachable)
{
    BATCH_CHECK(b && polls >= 0, "igab_batch_set_wait_limit: bad argument");
    b->spin_limit = polls > 0 ? polls : IGAB_BATCH_SPIN;
    b->hold = unreachable ? 1 : 0;
    return 0;
}

extern "C" int igab_batch_last_launch_count(const igab_batch *b, int *n)
{
    BATCH_CHECK(b && n, "igab_batch_last_launch_count: null argument");
    *n = b->last_launches;
    return 0;
}

/* one Newton iteration's assembly (residual, then tangent) captured once and replayed */
extern "C" int igab_batch_graph_capture(igab_batch *b, const double *U_dev, double *R_dev, void *vals_dev, int prec)
{
    BATCH_CHECK(b && U_dev && R_dev && vals_dev, "igab_batch_graph_capture: null argument");
    BATCH_CHECK(prec == IGAB_PREC_FP64 || prec == IGAB_PREC_FP32, "igab_batch_graph_capture: bad precision");
    IGAB_CUDA_TRY(cudaSetDevice(b->device));
    if (b->graph_exec) { cudaGraphExecDestroy(b->graph_exec); b->graph_exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    /* the launchers query occupancy and set kernel attributes: do that once before capture */
    int g0 = 0, g1 = 0, rc = grid_of(b, 0, &g0);
    if (!rc) rc = grid_of(b, prec == IGAB_PREC_FP64 ? 1 : 2, &g1);
    if (rc) return rc;
    IGAB_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    rc = launch_residual(b, U_dev, R_dev);
    if (!rc) rc = launch_tangent(b, U_dev, vals_dev, prec);
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
    if (rc) {
        if (gr) cudaGraphDestroy(gr);
        return rc;
    }
    if (e != cudaSuccess) {
        igab_set_error("igab_batch_graph_capture: %s", cudaGetErrorString(e));
        return IGAB_ERR_CUDA;
    }
    b->graph = gr;
    IGAB_CUDA_TRY(cudaGraphInstantiate(&b->graph_exec, b->graph, 0));
    return 0;
}

extern "C" int igab_batch_graph_launch(igab_batch *b)
{
    BATCH_CHECK(b && b->graph_exec, "igab_batch_graph_launch: nothing captured");
    IGAB_CUDA_TRY(cudaSetDevice(b->device));
    IGAB_CUDA_TRY(cudaGraphLaunch(b->graph_exec, b->stream));
    return 0;
}
