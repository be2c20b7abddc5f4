// api.cu -- the C ABI (include/bbmg_b200.h): handle, level hierarchy, setup
// and the solve drivers (stationary V-cycles, PCG, mixed precision).
//
// The solve routines follow src/solver/bbmg_class.f90: solve 604-639, cgsolve
// 643-703, mgsolve 707-728, cycle 732-776; the ILS wrapper around them follows
// src/solver/ils_class.f90:162-226 (init), 230-376 (setup), 674-822 (solve).
// One iteration of a solve is captured once into a CUDA graph and replayed;
// the host reads back one double per iteration for the convergence test.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bbmg_b200.h"
#include "hostcopy.cuh"
#include "setup.cuh"

using namespace bbmg;

namespace {

// slots of the handle's device scalars (dscal) and their pinned host mirror
constexpr int kScalRes0 = 0;    // max|r0|
constexpr int kScalRes = 1;     // max|r| of the last iteration
constexpr int kScalInfo = 2;    // setup: LU info (an int)
constexpr int kScalRhs = 3;     // max|rhs|
constexpr int kScalRes0L2 = 4;  // sum r0^2
constexpr int kScalRhsL2 = 5;   // sum rhs^2
constexpr int kScalTrue = 6;    // max|b - A x| at exit
constexpr int kScalTrueL2 = 7;  // sum (b - A x)^2 at exit
constexpr int kScalN = 16;
constexpr int kModes = 5;  // iteration graphs, see record_iteration

struct Level {
    Lay L;
    NbrOff nb;
    int npt = 27;       // stencil of the solve-phase operator planes
    bool fuse = true;   // periodic images can be written inside a GS colour
    // FP64
    double *opr27 = nullptr;   // 27 planes: the reference's operator
    double *oprS = nullptr;    // solve stencil planes (== opr27 when npt == 27)
    int nS = 0;                // planes allocated in oprS when it is not opr27
    double *c2f = nullptr, *f2c = nullptr, *oprc2f = nullptr;
    double *v = nullptr, *f = nullptr, *r = nullptr;
    // FP32 (mixed precision)
    float *oprS32 = nullptr, *c2f32 = nullptr;
    int n32 = 0;        // planes held in oprS32
    float *v32 = nullptr, *f32 = nullptr, *r32 = nullptr;
};

template <typename T> struct LvlPtr;
template <> struct LvlPtr<double> {
    static double *opr(Level &l) { return l.oprS; }
    static double *c2f(Level &l) { return l.c2f; }
    static double *v(Level &l) { return l.v; }
    static double *f(Level &l) { return l.f; }
    static double *r(Level &l) { return l.r; }
};
template <> struct LvlPtr<float> {
    static float *opr(Level &l) { return l.oprS32; }
    static float *c2f(Level &l) { return l.c2f32; }
    static float *v(Level &l) { return l.v32; }
    static float *f(Level &l) { return l.f32; }
    static float *r(Level &l) { return l.r32; }
};

}  // namespace

struct bbmg_handle {
    bbmg_grid grid{};
    bbmg_params prm{};
    int res_norm = BBMG_NORM_GUESS;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int nlvl = 0, nlvl_alloc = 0;
    std::vector<Level> lv;  // 1-based: lv[0] unused
    // coarsest dense problem
    int np = 0, lu_info = 0, npinned = 0;
    // coarse tail of the V-cycle in one cluster launch from level tail_n0
    // (0: every level runs pass by pass)
    int tail_n0 = 0;
    bool tail_off = false;        // cluster launch unavailable or not capturable: pass by pass
    int tail_blocks[2] = {0, 0};  // cluster size per precision (0 = not sized yet)
    size_t tail_smem_b = 0;
    int tail_mat_in_smem = 0;
    double *OP = nullptr, *LU = nullptr;
    int *piv = nullptr, *pinned = nullptr, *d_info = nullptr, *d_flag = nullptr;
    // Krylov / outer iteration vectors (level-1 layout)
    double *sol = nullptr, *pp = nullptr, *pp2 = nullptr, *Ap = nullptr;  // pp/pp2 alternate per iteration
    double *x2 = nullptr;  // second solution buffer of the mixed defect correction (alternates with lv[1].v)
    double *b1 = nullptr;  // pcg_bbox: the right-hand side (lv[1].f holds the CG residual during the solve)
    // first preconditioner stage (mixed PCG): the caller's function, its
    // context, the iterations that apply it (0 = all), the caller's dense
    // (no overlap) device arrays the residual is handed over in and the
    // stage's output comes back in, that output in the level layout and the
    // combined z
    bbmg_stage_fn stage_fn = nullptr;
    void *stage_ctx = nullptr;
    int stage_iters = 0;
    double *stage_r = nullptr, *stage_z = nullptr;
    double *z1 = nullptr, *zz = nullptr;

    CgScal *sc = nullptr;
    double *part = nullptr, *dscal = nullptr;  // reduction partials; scalars (kScal* slots)
    double *h_scal = nullptr;                  // pinned host mirror of dscal
    // staging for caller arrays
    double *d_opr_in = nullptr;
    size_t d_opr_in_n = 0;
    double *d_io = nullptr;  // one caller-shaped vector
    size_t io_n = 0;
    bool setup_done = false;
    int npt1 = 27;
    // graphs of one iteration: [mode] 0 = FP64 MG, 1 = FP64 PCG, 2 = mixed MG, 3 = mixed PCG,
    // 4 = mixed PCG after a first preconditioner stage;
    // graphs [mode][parity of the iteration] (the CG direction vectors alternate buffers)
    cudaGraphExec_t gexec[kModes][2] = {};
    int gkernels[kModes][2] = {};  // kernel nodes per graph
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long bytes = 0;
    std::string err;
    bbmg_info info{};
    unsigned l1_planes = 0;  // planes of the level-1 27-point storage the last scatter wrote (0: none yet)
    HostCopier copier;       // caller host arrays <-> device
};

static thread_local std::string g_create_err;

namespace bbmg {
// message for bbmg_last_error(NULL) from entry points without a handle
void set_create_error(const char *msg) { g_create_err = msg; }
}  // namespace bbmg

namespace {

int fail(bbmg_handle *h, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    else g_create_err = buf;
    return code;
}

#define CU(h, call)                                                                                  \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return fail((h), e_ == cudaErrorMemoryAllocation ? BBMG_NO_MEMORY : BBMG_CUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                          \
    } while (0)

template <typename T>
int dalloc(bbmg_handle *h, T **p, size_t n) {
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(h, BBMG_NO_MEMORY, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
    }
    h->bytes += (long long)(n * sizeof(T));
    e = cudaMemsetAsync(*p, 0, n * sizeof(T), h->stream);
    if (e != cudaSuccess) return fail(h, BBMG_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    return BBMG_OK;
}

void dfree(void *p) {
    if (p) cudaFree(p);
}

bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

inline int odiv(int n) { return n / 2 + n % 2; }  // bbmg_class.f90:147-151

void drop_graphs(bbmg_handle *h) {
    for (auto &gm : h->gexec)
        for (auto &g : gm)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
}

// ---------------------------------------------------------------------------
// V-cycle (bbmg_class.f90:732-776), recursive over levels
template <typename T> struct PrecIdx { static constexpr int value = sizeof(T) == 8 ? 0 : 1; };

// cycle(n) for n >= tail_n0 as one cooperative launch; returns BBMG_NOT_SETUP
// (nothing launched) when the levels do not qualify
template <typename T>
int vcycle_tail(bbmg_handle *h, int n) {
    using P = LvlPtr<T>;
    TailArgs<T> A{};
    A.n = h->nlvl - n + 1;
    if (A.n > kTailMax || A.n < 2) return BBMG_NOT_SETUP;
    for (int m = n; m <= h->nlvl; m++) {
        Level &l = h->lv[m];
        if (l.npt != 27 || !l.fuse) return BBMG_NOT_SETUP;
        TailLvl<T> &t = A.lv[m - n];
        t.L = l.L;
        for (int q = 0; q < 27; q++) {
            t.off[0].o[q] = l.nb.off[0][q];
            t.off[1].o[q] = l.nb.off[1][q];
        }
        t.opr = P::opr(l);
        t.v = P::v(l);
        t.f = P::f(l);
        t.r = P::r(l);
        t.c2f = m < h->nlvl ? P::c2f(l) : nullptr;
    }
    A.split = A.n - 1;
    for (int m = 0; m < A.n - 1; m++) {
        const Lay &L = A.lv[m].L;
        if ((long long)L.nx * L.ny * L.nz <= kTailBlockCells) { A.split = m; break; }
    }
    if (const char *env = getenv("BBMG_TAIL_SPLIT")) A.split = std::max(0, std::min(A.n - 1, atoi(env)));
    A.pre = h->prm.relax_pre;
    A.post = h->prm.relax_post;
    A.direct = h->prm.use_direct_solve;
    A.mat_in_smem = h->tail_mat_in_smem;
    A.LU = h->LU;
    A.piv = h->piv;
    A.pinned = h->pinned;
    int &blocks = h->tail_blocks[PrecIdx<T>::value];
    if (!blocks && tail_grid<T>(h->tail_smem_b, &blocks) != cudaSuccess) {
        cudaGetLastError();
        h->tail_off = true;  // no cluster of 8 fits: the levels run pass by pass
        return BBMG_NOT_SETUP;
    }
    CU(h, launch_vtail<T>(A, blocks, h->tail_smem_b, h->stream));
    return BBMG_OK;
}

template <typename T>
int vcycle(bbmg_handle *h, int n) {
    using P = LvlPtr<T>;
    cudaStream_t s = h->stream;
    if (n == h->tail_n0 && !h->tail_off && h->prm.ncycle == 1) {
        int st = vcycle_tail<T>(h, n);
        if (st != BBMG_NOT_SETUP) return st;
    }
    Level &l = h->lv[n];
    if (n == h->nlvl) {
        if (h->prm.use_direct_solve) {
            CU(h, launch_coarse_solve<T>(l.L, h->LU, h->piv, h->pinned, P::f(l), P::v(l), s));
        } else {
            CU(h, launch_relax_sweeps<T>(l.L, l.nb, l.npt, l.fuse, P::opr(l), P::v(l), P::f(l), 1,
                                         h->prm.relax_pre + h->prm.relax_post, s));
        }
        return BBMG_OK;
    }
    Level &c = h->lv[n + 1];
    CU(h, launch_relax_sweeps<T>(l.L, l.nb, l.npt, l.fuse, P::opr(l), P::v(l), P::f(l), 1, h->prm.relax_pre, s));
    const int dir = (h->prm.relax_pre & 1) ? -1 : 1;
    CU(h, launch_residual<T>(l.L, l.nb, l.npt, P::opr(l), P::v(l), P::f(l), P::r(l), s));
    CU(h, launch_restrict<T>(l.L, c.L, P::c2f(l), P::r(l), P::f(c), P::v(c), s));
    for (int i = 0; i < h->prm.ncycle; i++) {
        // every call of cycle(n+1) starts from v = 0 (bbmg_class.f90:739)
        if (i > 0) CU(h, cudaMemsetAsync(P::v(c), 0, sizeof(T) * c.L.plane, s));
        int st = vcycle<T>(h, n + 1);
        if (st) return st;
    }
    CU(h, launch_prolong<T>(l.L, c.L, P::c2f(l), P::v(c), P::v(l), s));
    CU(h, launch_relax_sweeps<T>(l.L, l.nb, l.npt, l.fuse, P::opr(l), P::v(l), P::f(l), dir, h->prm.relax_post, s));
    return BBMG_OK;
}

// One iteration of each solver, written once into a graph.  `par` selects
// which of the two CG direction buffers is the old one.
int record_iteration(bbmg_handle *h, int mode, int par) {
    cudaStream_t s = h->stream;
    Level &l1 = h->lv[1];
    const Lay &L = l1.L;
    double *pp_old = par ? h->pp2 : h->pp, *pp_new = par ? h->pp : h->pp2;
    int st = BBMG_OK;
    switch (mode) {
    case 0:  // FP64 mgsolve: cycle; residual; max|r| (bbmg_class.f90:716-722)
        if ((st = vcycle<double>(h, 1))) return st;
        CU(h, launch_residual<double>(L, l1.nb, l1.npt, l1.oprS, l1.v, l1.f, l1.r, s));
        CU(h, launch_maxabs<double>(L, l1.r, h->part, h->dscal + kScalRes, s));
        break;
    case 1:  // FP64 cgsolve body, v zeroed by the previous step; res lives in l1.f
        if ((st = vcycle<double>(h, 1))) return st;
        CU(h, launch_cg_rho<double>(L, l1.v, l1.f, h->part, h->sc, s));
        CU(h, launch_cg_pap_fused<double>(L, l1.nb, l1.npt, l1.oprS, l1.v, pp_old, pp_new, h->Ap, h->part, h->sc, s));
        CU(h, launch_cg_xr_fused<double>(L, h->sol, pp_new, l1.f, h->Ap, h->sc, nullptr, l1.v, h->part, h->dscal + kScalRes, s));
        break;
    case 2: {  // mixed defect correction: e = V32(r); x += e; r = b - A x (FP64); f32/v32 prepared
        double *x_old = par ? h->x2 : l1.v, *x_new = par ? l1.v : h->x2;
        CU(h, cudaMemsetAsync(l1.v32, 0, sizeof(float) * L.plane, s));
        if ((st = vcycle<float>(h, 1))) return st;
        CU(h, launch_defect_fused(L, l1.nb, l1.npt, l1.oprS, x_old, l1.v32, l1.f, x_new, l1.f32, h->part,
                                  h->dscal + kScalRes, s));
        break;
    }
    case 3:  // mixed PCG: FP64 Krylov vectors, FP32 V-cycle; f32/v32 prepared by the previous step.
             // The FP32 V-cycle is not an exactly symmetric, fixed operator (its rounding
             // depends on the residual it is given), so the direction update is the
             // flexible one, beta = -z.Ap_old / pap_old (FCG(1)), where the reference's
             // rho/rho_old (bbmg_class.f90:666-672) assumes a fixed SPD preconditioner
        if ((st = vcycle<float>(h, 1))) return st;
        CU(h, launch_fcg_rho<float>(L, l1.v32, l1.f, h->Ap, h->part, h->sc, s));
        CU(h, launch_cg_pap_fused<float>(L, l1.nb, l1.npt, l1.oprS, l1.v32, pp_old, pp_new, h->Ap, h->part, h->sc, s));
        CU(h, launch_cg_xr_fused<float>(L, h->sol, pp_new, l1.f, h->Ap, h->sc, l1.f32, l1.v32, h->part, h->dscal + kScalRes, s));
        break;
    case 4:  // mixed PCG with a first preconditioner stage: z1 = stage(res) is in place
             // (run before the graph); the V-cycle acts on the remaining residual
             // res - A z1 and z = z1 + V(res - A z1); flexible direction update
        CU(h, launch_residual<double>(L, l1.nb, l1.npt, l1.oprS, h->z1, l1.f, l1.r, s));
        CU(h, launch_round_f32(L, l1.r, l1.f32, s));
        if ((st = vcycle<float>(h, 1))) return st;
        CU(h, launch_fcg_z(L, h->z1, l1.v32, l1.f, h->Ap, h->zz, h->part, h->sc, s));
        CU(h, launch_cg_pap_fused<double>(L, l1.nb, l1.npt, l1.oprS, h->zz, pp_old, pp_new, h->Ap, h->part, h->sc, s));
        CU(h, launch_cg_xr_fused<float>(L, h->sol, pp_new, l1.f, h->Ap, h->sc, l1.f32, l1.v32, h->part, h->dscal + kScalRes, s));
        break;
    }
    CU(h, cudaMemcpyAsync(h->h_scal + kScalRes, h->dscal + kScalRes, sizeof(double), cudaMemcpyDeviceToHost, s));
    return BBMG_OK;
}

int get_graph(bbmg_handle *h, int mode, int par, cudaGraphExec_t *out) {
    if (h->gexec[mode][par]) {
        *out = h->gexec[mode][par];
        return BBMG_OK;
    }
    cudaGraph_t g = nullptr;
    CU(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int st = record_iteration(h, mode, par);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if ((st || e != cudaSuccess) && h->tail_n0 && !h->tail_off) {
        // a cluster launch that cannot be captured here: record the coarse
        // levels pass by pass instead
        if (g) cudaGraphDestroy(g);
        g = nullptr;
        cudaGetLastError();
        h->tail_off = true;
        drop_graphs(h);
        CU(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        st = record_iteration(h, mode, par);
        e = cudaStreamEndCapture(h->stream, &g);
    }
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return fail(h, BBMG_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    cudaGraphGetNodes(g, nodes.data(), &nn);
    int nk = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) nk++;
    }
    h->gkernels[mode][par] = nk;
    e = cudaGraphInstantiate(&h->gexec[mode][par], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(h, BBMG_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
    *out = h->gexec[mode][par];
    return BBMG_OK;
}

int sync_read(bbmg_handle *h, double *v, int slot) {
    CU(h, cudaStreamSynchronize(h->stream));
    *v = h->h_scal[slot];
    return BBMG_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

void bbmg_default_params(bbmg_params *p) {
    if (!p) return;
    p->method = BBMG_METHOD_PCG_BBOX;
    p->precision = BBMG_PREC_FP64;
    p->ncycle = 1;
    p->relax_pre = 2;
    p->relax_post = 2;
    p->ncell_coarsest = 300;
    p->use_direct_solve = 1;
    p->maxit = 100;
    p->rcvg = 1e-10;
    p->device = -1;
}

const char *bbmg_last_error(const bbmg_handle *h) { return h ? h->err.c_str() : g_create_err.c_str(); }

int bbmg_destroy(bbmg_handle *h) {
    if (!h) return BBMG_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graphs(h);
    for (size_t n = 1; n < h->lv.size(); n++) {
        Level &l = h->lv[n];
        if (l.oprS != l.opr27) dfree(l.oprS);
        dfree(l.opr27); dfree(l.c2f); dfree(l.f2c); dfree(l.oprc2f);
        dfree(l.v); dfree(l.f); dfree(l.r);
        dfree(l.oprS32); dfree(l.c2f32); dfree(l.v32); dfree(l.f32); dfree(l.r32);
    }
    dfree(h->OP); dfree(h->LU); dfree(h->piv); dfree(h->pinned); dfree(h->d_info); dfree(h->d_flag);
    dfree(h->sol); dfree(h->pp); dfree(h->pp2); dfree(h->Ap); dfree(h->x2); dfree(h->b1); dfree(h->sc); dfree(h->part);
    dfree(h->z1); dfree(h->zz);
    dfree(h->dscal);
    dfree(h->d_opr_in); dfree(h->d_io);
    if (h->h_scal) cudaFreeHost(h->h_scal);
    h->copier.release();
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return BBMG_OK;
}

int bbmg_create(const bbmg_grid *grid, const bbmg_params *params, bbmg_handle **out) {
    if (!out) return fail(nullptr, BBMG_BAD_ARGS, "null handle pointer");
    *out = nullptr;
    if (!grid) return fail(nullptr, BBMG_BAD_ARGS, "null grid");
    if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || grid->ghost < 0)
        return fail(nullptr, BBMG_BAD_ARGS, "grid sizes must be >= 1 and ghost >= 0 (got %d %d %d, ghost %d)",
                    grid->nx, grid->ny, grid->nz, grid->ghost);
    bbmg_params prm;
    bbmg_default_params(&prm);
    if (params) prm = *params;
    if (prm.method != BBMG_METHOD_BBOX && prm.method != BBMG_METHOD_PCG_BBOX)
        return fail(nullptr, BBMG_BAD_ARGS, "unknown method %d", prm.method);
    if (prm.precision != BBMG_PREC_FP64 && prm.precision != BBMG_PREC_MIXED)
        return fail(nullptr, BBMG_BAD_ARGS, "unknown precision %d", prm.precision);
    if (prm.ncycle < 1 || prm.relax_pre < 0 || prm.relax_post < 0 || prm.maxit < 0)
        return fail(nullptr, BBMG_BAD_ARGS, "invalid cycle parameters");

    bbmg_handle *h = new bbmg_handle();
    h->grid = *grid;
    h->prm = prm;
    int dev = prm.device;
    if (dev < 0) {
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            delete h;
            return fail(nullptr, BBMG_CUDA, "no CUDA device available");
        }
    }
    h->device = dev;
    if (cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        return fail(nullptr, BBMG_CUDA, "cannot select CUDA device %d", dev);
    }
    int st = BBMG_OK;
    auto bail = [&](int code) {
        g_create_err = h->err;
        bbmg_destroy(h);
        return code;
    };
    // a blocking stream: it waits for work the caller queued on the legacy
    // default stream (and the reverse), so device arrays a caller has just
    // written there are complete when setup/solve read them
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamDefault) != cudaSuccess) return bail(fail(h, BBMG_CUDA, "stream"));
    h->own_stream = true;
    if (coarse_solve_prepare() != cudaSuccess) return bail(fail(h, BBMG_CUDA, "coarse solve attributes"));

    // level hierarchy (bbmg_class.f90:231-341, initialize 584-589)
    int lx = 1, ly = 1, lz = 1;
    while (grid->nx > (1 << (lx - 1))) lx++;
    while (grid->ny > (1 << (ly - 1))) ly++;
    while (grid->nz > (1 << (lz - 1))) lz++;
    const int BIG = 1 << 30;
    int n1 = lx == 1 ? BIG : lx, n2 = ly == 1 ? BIG : ly, n3 = lz == 1 ? BIG : lz;
    int nl = std::min(n1, std::min(n2, n3));
    if (lx == 1 && ly == 1 && lz == 1) nl = 1;
    if (nl > 16) nl = 16;
    int nx = grid->nx, ny = grid->ny, nz = grid->nz;
    h->lv.resize(nl + 1);
    for (int n = 1; n <= nl; n++) {
        h->lv[n].L = make_lay(nx, ny, nz, grid->xper, grid->yper, grid->zper);
        nx = odiv(nx); ny = odiv(ny); nz = odiv(nz);
    }
    h->nlvl_alloc = nl;
    h->nlvl = nl;
    for (int n = 1; n <= nl; n++) {
        const Lay &L = h->lv[n].L;
        if ((long long)L.nx * L.ny * L.nz <= prm.ncell_coarsest) { h->nlvl = n; break; }
    }
    // direct problem size check
    {
        const Lay &Lc = h->lv[h->nlvl].L;
        long long np = (long long)Lc.nx * Lc.ny * Lc.nz;
        if (prm.use_direct_solve && np > 4096)
            return bail(fail(h, BBMG_BAD_ARGS, "coarsest level has %lld unknowns; the direct solve supports <= 4096", np));
        h->np = (int)np;
    }
    const bool mixed = prm.precision == BBMG_PREC_MIXED;
    for (int n = 1; n <= h->nlvl; n++) {
        Level &l = h->lv[n];
        const Lay &L = l.L;
        l.nb = make_nbr(L);
        l.fuse = !((L.xper && (L.nx & 1)) || (L.yper && (L.ny & 1)) || (L.zper && (L.nz & 1)));
        size_t P = (size_t)L.plane;
        if ((st = dalloc(h, &l.opr27, 27 * P))) return bail(st);
        if (n < h->nlvl) {
            if ((st = dalloc(h, &l.c2f, 8 * P))) return bail(st);
            if ((st = dalloc(h, &l.oprc2f, 27 * P))) return bail(st);
        }
        if (n > 1 && (st = dalloc(h, &l.f2c, 27 * P))) return bail(st);
        if ((st = dalloc(h, &l.v, P)) || (st = dalloc(h, &l.f, P)) || (st = dalloc(h, &l.r, P))) return bail(st);
        if (mixed) {
            if ((st = dalloc(h, &l.v32, P)) || (st = dalloc(h, &l.f32, P)) || (st = dalloc(h, &l.r32, P))) return bail(st);
            if (n < h->nlvl && (st = dalloc(h, &l.c2f32, 8 * P))) return bail(st);
        }
    }
    const Lay &L1 = h->lv[1].L;
    if ((st = dalloc(h, &h->OP, (size_t)h->np * h->np)) || (st = dalloc(h, &h->LU, (size_t)h->np * h->np)) ||
        (st = dalloc(h, &h->piv, (size_t)h->np)) || (st = dalloc(h, &h->pinned, (size_t)h->np)) ||
        (st = dalloc(h, &h->d_info, 1)) || (st = dalloc(h, &h->d_flag, 1)) ||
        (st = dalloc(h, &h->part, 2 * (size_t)kRedBlocks)) ||
        (st = dalloc(h, &h->dscal, kScalN)) || (st = dalloc(h, &h->sc, 1)))
        return bail(st);
    if (mixed && prm.method == BBMG_METHOD_BBOX && (st = dalloc(h, &h->x2, (size_t)L1.plane))) return bail(st);
    if (prm.method == BBMG_METHOD_PCG_BBOX) {
        if ((st = dalloc(h, &h->sol, (size_t)L1.plane)) || (st = dalloc(h, &h->pp, (size_t)L1.plane)) ||
            (st = dalloc(h, &h->pp2, (size_t)L1.plane)) || (st = dalloc(h, &h->Ap, (size_t)L1.plane)) ||
            (st = dalloc(h, &h->b1, (size_t)L1.plane)))
            return bail(st);
    }
    {
        // the coarse tail: the first level >= 2 at or below tail_cells cells
        // from which every level can be fused (27-point, periodic sizes even)
        long long tail_cells = kTailCells;
        if (const char *env = getenv("BBMG_TAIL_CELLS")) tail_cells = atoll(env);
        for (int n = 2; prm.ncycle == 1 && tail_cells > 0 && n < h->nlvl; n++) {
            const Lay &L = h->lv[n].L;
            if ((long long)L.nx * L.ny * L.nz > tail_cells || h->nlvl - n + 1 > kTailMax) continue;
            bool ok = true;
            for (int m = n; m <= h->nlvl; m++) ok = ok && h->lv[m].fuse;
            if (ok) { h->tail_n0 = n; break; }
        }
        if (h->tail_n0) h->tail_smem_b = tail_smem(h->np, &h->tail_mat_in_smem);
    }
    if (cudaMallocHost((void **)&h->h_scal, kScalN * sizeof(double)) != cudaSuccess) return bail(fail(h, BBMG_NO_MEMORY, "pinned host"));
    if (cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess)
        return bail(fail(h, BBMG_CUDA, "events"));
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(fail(h, BBMG_CUDA, "initialisation"));
    h->info.nlvl = h->nlvl;
    for (int n = 1; n <= h->nlvl && n <= 16; n++) {
        h->info.level_dims[n - 1][0] = h->lv[n].L.nx;
        h->info.level_dims[n - 1][1] = h->lv[n].L.ny;
        h->info.level_dims[n - 1][2] = h->lv[n].L.nz;
    }
    h->info.coarse_n = h->np;
    h->info.device_bytes = h->bytes;
    *out = h;
    return BBMG_OK;
}

int bbmg_set_stream(bbmg_handle *h, void *stream) {
    if (!h) return BBMG_BAD_ARGS;
    if (!h->own_stream && h->stream == (cudaStream_t)stream) return BBMG_OK;  // graphs stay valid
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    h->own_stream = false;
    h->stream = (cudaStream_t)stream;
    drop_graphs(h);
    return BBMG_OK;
}

int bbmg_set_convergence(bbmg_handle *h, int maxit, double rcvg) {
    if (!h || maxit < 0) return BBMG_BAD_ARGS;
    h->prm.maxit = maxit;
    h->prm.rcvg = rcvg;
    return BBMG_OK;
}

int bbmg_set_residual_norm(bbmg_handle *h, int norm) {
    if (!h) return BBMG_BAD_ARGS;
    if (norm != BBMG_NORM_GUESS && norm != BBMG_NORM_RHS) return fail(h, BBMG_BAD_ARGS, "unknown norm %d", norm);
    h->res_norm = norm;
    return BBMG_OK;
}

int bbmg_set_precond_stage(bbmg_handle *h, bbmg_stage_fn fn, void *ctx, int iters, double *r, double *z) {
    if (!h) return BBMG_BAD_ARGS;
    if (!fn) {
        h->stage_fn = nullptr;
        h->stage_ctx = nullptr;
        h->stage_r = h->stage_z = nullptr;
        return BBMG_OK;
    }
    if (iters < 0) return fail(h, BBMG_BAD_ARGS, "stage iterations must be >= 0");
    if (h->prm.method != BBMG_METHOD_PCG_BBOX || h->prm.precision != BBMG_PREC_MIXED)
        return fail(h, BBMG_BAD_ARGS, "a preconditioner stage needs a pcg_bbox handle in mixed precision");
    CU(h, cudaSetDevice(h->device));
    for (const void *p : {(const void *)r, (const void *)z}) {
        cudaPointerAttributes a;
        if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess ||
            !(a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == h->device))) {
            cudaGetLastError();
            return fail(h, BBMG_BAD_ARGS, "the stage's r and z must be device arrays of the handle's device");
        }
    }
    if (r == z) return fail(h, BBMG_BAD_ARGS, "the stage's r and z must be distinct arrays");
    if (!h->z1) {
        const Lay &L = h->lv[1].L;
        int st;
        if ((st = dalloc(h, &h->z1, (size_t)L.plane)) || (st = dalloc(h, &h->zz, (size_t)L.plane))) return st;
        h->info.device_bytes = h->bytes;
    }
    h->stage_fn = fn;
    h->stage_ctx = ctx;
    h->stage_iters = iters;
    h->stage_r = r;
    h->stage_z = z;
    return BBMG_OK;
}

int bbmg_setup(bbmg_handle *h, int nst, const int *stc, const double *opr) {
    if (!h) return BBMG_BAD_ARGS;
    if (nst < 1 || nst > 27 || !stc || !opr) return fail(h, BBMG_BAD_ARGS, "invalid stencil arguments");
    // bbmg only supports 3x3x3 operators (bbmg_class.f90:197)
    bool seven = true;
    for (int st = 0; st < nst; st++) {
        int a = stc[3 * st], b = stc[3 * st + 1], c = stc[3 * st + 2];
        if (a < -1 || a > 1 || b < -1 || b > 1 || c < -1 || c > 1)
            return fail(h, BBMG_BAD_ARGS, "stencil entry %d = (%d,%d,%d) lies outside 3x3x3", st, a, b, c);
        if (std::abs(a) + std::abs(b) + std::abs(c) > 1) seven = false;
    }
    CU(h, cudaSetDevice(h->device));
    cudaStream_t s = h->stream;
    CU(h, cudaEventRecord(h->ev0, s));
    const int g = h->grid.ghost;
    Level &l1 = h->lv[1];
    const Lay &L1 = l1.L;
    size_t ncaller = (size_t)(L1.nx + 2 * g) * (L1.ny + 2 * g) * (L1.nz + 2 * g);
    const double *src = opr;
    if (!is_device_ptr(opr)) {
        if (h->d_opr_in_n < ncaller * nst) {
            dfree(h->d_opr_in);
            h->d_opr_in = nullptr;
            int st = dalloc(h, &h->d_opr_in, ncaller * nst);
            if (st) return st;
            h->d_opr_in_n = ncaller * nst;
        }
        CU(h, h->copier.h2d(h->d_opr_in, opr, sizeof(double) * ncaller * nst, s));
        src = h->d_opr_in;
    }
    // ils scatter + identity overlap + periodic copy (ils_class.f90:247-256, bbmg_class.f90:937-950).
    // Only the planes the stencil touches (and the centre, which carries the
    // overlap's identity) are written; the other planes of the 27-point
    // level-1 storage are zeroed when the set of planes changes and then stay
    // zero, so the prolongation and A*P of level 1 skip them.
    unsigned smask = 1u << kCentre27;
    for (int st = 0; st < nst; st++) smask |= 1u << q27(stc[3 * st], stc[3 * st + 1], stc[3 * st + 2]);
    if (smask != h->l1_planes) {
        CU(h, cudaMemsetAsync(l1.opr27, 0, sizeof(double) * 27 * (size_t)L1.plane, s));
        // A*P of a 7-point level 1 writes only the slots such an operator
        // reaches; the others must read zero after a 27-point setup
        if (h->nlvl > 1) CU(h, cudaMemsetAsync(l1.oprc2f, 0, sizeof(double) * 27 * (size_t)L1.plane, s));
        h->l1_planes = smask;
    }
    CU(h, setup_scatter(L1, src, nst, g, stc, l1.opr27, smask, s));
    CU(h, wrap_planes_mask(L1, l1.opr27, smask, s));
    const bool mixed = h->prm.precision == BBMG_PREC_MIXED;
    // the mixed V-cycle's FP32 operators of the coarse levels (27 planes) are
    // written by the Galerkin product itself
    if (mixed) {
        for (int n = 2; n <= h->nlvl; n++) {
            Level &l = h->lv[n];
            if (l.oprS32 && l.n32 == 27) continue;
            if (l.oprS32) {
                dfree(l.oprS32);
                h->bytes -= (long long)((size_t)l.n32 * l.L.plane * sizeof(float));
                l.oprS32 = nullptr;
                drop_graphs(h);
            }
            int st = dalloc(h, &l.oprS32, (size_t)27 * l.L.plane);
            if (st) return st;
            l.n32 = 27;
        }
    }
    // hierarchy (bbmg_class.f90:952-959); in mixed precision the FP32 copies
    // of the prolongation weights and coarse operators come out of the same
    // kernels
    for (int n = 2; n <= h->nlvl; n++) {
        Level &F = h->lv[n - 1], &C = h->lv[n];
        const unsigned fmask = n == 2 ? smask : 0x7FFFFFFu;
        CU(h, setup_prolongation(F.L, F.opr27, F.c2f, fmask, s, mixed ? F.c2f32 : nullptr));
        CU(h, setup_restriction(F.L, C.L, F.c2f, C.f2c, s));
        CU(h, setup_operator(F.L, C.L, F.opr27, F.c2f, C.f2c, F.oprc2f, C.opr27, fmask, s, mixed ? C.oprS32 : nullptr));
    }
    // dense coarsest problem (bbmg_class.f90:961, 1307-1385)
    CU(h, setup_direct(h->lv[h->nlvl].L, h->lv[h->nlvl].opr27, h->OP, h->LU, h->piv, h->pinned, h->d_info, s));
    // solve-phase operator planes: a 7-point level-1 operator that is exactly
    // symmetric is stored as 4 planes (D, E, N, T), otherwise as 7; coarse
    // levels keep the 27 planes
    int sym = 0;
    if (seven) {
        const int one = 1;
        CU(h, cudaMemcpyAsync(h->d_flag, &one, sizeof(int), cudaMemcpyHostToDevice, s));
        CU(h, check_symmetric7(L1, l1.opr27, h->d_flag, s));
        CU(h, cudaMemcpyAsync(&sym, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(h, cudaStreamSynchronize(s));
    }
    const int npt1 = seven ? (sym ? 4 : 7) : 27;
    if (npt1 != h->npt1) drop_graphs(h);
    h->npt1 = npt1;
    for (int n = 1; n <= h->nlvl; n++) {
        Level &l = h->lv[n];
        size_t P = (size_t)l.L.plane;
        int npt = (n == 1) ? npt1 : 27;
        if (npt == 27) {
            if (l.oprS && l.oprS != l.opr27) {
                dfree(l.oprS);
                h->bytes -= (long long)((size_t)l.nS * P * sizeof(double));
                l.nS = 0;
            }
            l.oprS = l.opr27;
        } else {
            if (l.oprS == l.opr27) l.oprS = nullptr;
            if (l.oprS && l.nS != npt) {
                dfree(l.oprS);
                h->bytes -= (long long)((size_t)l.nS * P * sizeof(double));
                l.oprS = nullptr;
            }
            if (!l.oprS) {
                int st = dalloc(h, &l.oprS, (size_t)npt * P);
                if (st) return st;
                l.nS = npt;
            }
        }
        if (l.npt != npt) { l.npt = npt; drop_graphs(h); }
        if (mixed) {
            if (l.oprS32 && l.n32 != npt) {
                dfree(l.oprS32);
                h->bytes -= (long long)((size_t)l.n32 * P * sizeof(float));
                l.oprS32 = nullptr;
                drop_graphs(h);
            }
            if (!l.oprS32) {
                int st = dalloc(h, &l.oprS32, (size_t)npt * P);
                if (st) return st;
                l.n32 = npt;
            }
            // levels >= 2 and every c2f32 were written during the hierarchy
            if (n == 1 && npt == 27) CU(h, launch_to_f32(l.oprS, l.oprS32, 27LL * P, s));
        }
        if (npt < 27) {
            // the level-1 4- or 7-plane storage (and its FP32 copy) in one pass
            static const int sym4[4] = {13, 14, 16, 22};
            int slots[7];
            for (int q = 0; q < npt; q++) slots[q] = npt == 4 ? sym4[q] : k7to27(q);
            CU(h, setup_solve_planes(l.L, l.opr27, npt, slots, l.oprS, mixed ? l.oprS32 : nullptr, s));
        }
    }
    CU(h, cudaMemcpyAsync(h->h_scal + kScalInfo, h->d_info, sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(h, cudaEventRecord(h->ev1, s));
    CU(h, cudaStreamSynchronize(s));
    int info;
    memcpy(&info, h->h_scal + kScalInfo, sizeof(int));
    h->lu_info = info;
    std::vector<int> pin(h->np);
    CU(h, cudaMemcpy(pin.data(), h->pinned, sizeof(int) * h->np, cudaMemcpyDeviceToHost));
    h->npinned = 0;
    for (int v : pin) h->npinned += v;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->info.setup_ms = ms;
    h->info.coarse_pinned = h->npinned;
    h->info.device_bytes = h->bytes;
    h->info.level1_stencil = npt1;
    h->setup_done = true;
    return BBMG_OK;
}

int bbmg_solve(bbmg_handle *h, const double *rhs, double *sol, int *it_out, double *rerr_out) {
    if (!h) return BBMG_BAD_ARGS;
    if (!h->setup_done) return fail(h, BBMG_NOT_SETUP, "[bbmg solve] solver has not been setup");
    if (!rhs || !sol) return fail(h, BBMG_BAD_ARGS, "null rhs or sol");
    CU(h, cudaSetDevice(h->device));
    cudaStream_t s = h->stream;
    Level &l1 = h->lv[1];
    const Lay &L = l1.L;
    const int g = h->grid.ghost;
    const size_t ncaller = (size_t)(L.nx + 2 * g) * (L.ny + 2 * g) * (L.nz + 2 * g);
    const bool rhs_dev = is_device_ptr(rhs), sol_dev = is_device_ptr(sol);
    if ((!rhs_dev || !sol_dev) && h->io_n < ncaller) {
        dfree(h->d_io);
        h->d_io = nullptr;
        int st = dalloc(h, &h->d_io, ncaller);
        if (st) return st;
        h->io_n = ncaller;
    }
    const bool mixed = h->prm.precision == BBMG_PREC_MIXED;
    const bool krylov = h->prm.method == BBMG_METHOD_PCG_BBOX;
    int it = -1;
    double rerr = HUGE_VAL;
    CU(h, cudaEventRecord(h->ev0, s));
    // rhs/initial guess into the level-1 arrays; overlap zero, then periodic
    // images (bbmg_class.f90:611-624; ils_class.f90:693-700)
    CU(h, cudaMemsetAsync(l1.f, 0, sizeof(double) * L.plane, s));
    CU(h, cudaMemsetAsync(l1.v, 0, sizeof(double) * L.plane, s));
    const double *rsrc = rhs;
    if (!rhs_dev) {
        CU(h, h->copier.h2d(h->d_io, rhs, sizeof(double) * ncaller, s));
        rsrc = h->d_io;
    }
    CU(h, launch_from_caller<double>(L, rsrc, g, l1.f, s));
    const double *xsrc = sol;
    if (!sol_dev) {
        CU(h, h->copier.h2d(h->d_io, sol, sizeof(double) * ncaller, s));
        xsrc = h->d_io;
    }
    CU(h, launch_from_caller<double>(L, xsrc, g, l1.v, s));
    // initial residual (bbmg_class.f90:626-628)
    CU(h, launch_residual<double>(L, l1.nb, l1.npt, l1.oprS, l1.v, l1.f, l1.r, s));
    CU(h, launch_maxabs<double>(L, l1.r, h->part, h->dscal + kScalRes0, s));
    const bool by_rhs = h->res_norm == BBMG_NORM_RHS;
    if (by_rhs) {
        CU(h, launch_maxabs<double>(L, l1.f, h->part, h->dscal + kScalRhs, s));
        CU(h, launch_dot<double>(L, l1.f, l1.f, h->part, h->dscal + kScalRhsL2, s));
    }
    CU(h, launch_dot<double>(L, l1.r, l1.r, h->part, h->dscal + kScalRes0L2, s));
    CU(h, cudaMemcpyAsync(h->h_scal, h->dscal, sizeof(double) * kScalTrue, cudaMemcpyDeviceToHost, s));
    double res0 = 0.0;
    int st = sync_read(h, &res0, kScalRes0);
    if (st) return st;
    // denominator of rerr: the guess's own initial residual (the reference's
    // definition), or max|rhs|, the residual a zero guess would start from
    double rnorm = res0, rnorm2 = h->h_scal[kScalRes0L2];
    if (by_rhs && h->h_scal[kScalRhs] > 0.0) {
        rnorm = h->h_scal[kScalRhs];
        rnorm2 = h->h_scal[kScalRhsL2];
    }
    int status = BBMG_OK;
    int fallback_it = 0, stage_it = 0;
    double *xout = l1.v;
    // two copies-in, residual, max and sum of squares (two each) [, max and sum of squares of rhs]
    long long launches = by_rhs ? 10 : 6;
    if (res0 == 0.0) {
        it = 0;
        rerr = 0.0;
    } else if (!(res0 == res0) || std::isinf(res0)) {
        status = fail(h, BBMG_NONFINITE, "initial residual is not finite");
        it = 0;
        rerr = res0;
    } else {
        int mode = (mixed ? 2 : 0) + (krylov ? 1 : 0);
        // a first preconditioner stage (mixed PCG only)
        bool staged = krylov && mixed && h->stage_fn != nullptr;
        if (krylov) {
            // res = r, sol = v (bbmg_class.f90:652-653); res lives in l1.f, b is kept in b1
            CU(h, cudaMemcpyAsync(h->b1, l1.f, sizeof(double) * L.plane, cudaMemcpyDeviceToDevice, s));
            CU(h, cudaMemcpyAsync(l1.f, l1.r, sizeof(double) * L.plane, cudaMemcpyDeviceToDevice, s));
            CU(h, cudaMemcpyAsync(h->sol, l1.v, sizeof(double) * L.plane, cudaMemcpyDeviceToDevice, s));
            CU(h, cudaMemsetAsync(h->sc, 0, sizeof(CgScal), s));
            CU(h, cudaMemsetAsync(h->pp, 0, sizeof(double) * L.plane, s));
            CU(h, cudaMemsetAsync(h->pp2, 0, sizeof(double) * L.plane, s));
            // the first preconditioner call starts from v = 0 (bbmg_class.f90:659)
            if (mixed) {
                CU(h, launch_round_f32(L, l1.f, l1.f32, s));
                CU(h, cudaMemsetAsync(l1.v32, 0, sizeof(float) * L.plane, s));
            } else {
                CU(h, cudaMemsetAsync(l1.v, 0, sizeof(double) * L.plane, s));
            }
            launches += mixed ? 1 : 0;
            xout = h->sol;
            // the flexible update reads the previous A p (times beta = 0 at the first iteration)
            if (mixed) CU(h, cudaMemsetAsync(h->Ap, 0, sizeof(double) * L.plane, s));
        } else if (mixed) {
            CU(h, launch_round_f32(L, l1.r, l1.f32, s));
            CU(h, cudaMemsetAsync(l1.v32, 0, sizeof(float) * L.plane, s));
            launches += 1;
        }
        bool pingpong = krylov || mixed;
        std::vector<double> hist;
        hist.reserve(h->prm.maxit + 1);
        for (int n = 1; n <= h->prm.maxit; n++) {
            const int par = pingpong ? ((n - 1) & 1) : 0;
            if (mode == 2) xout = par ? l1.v : h->x2;  // the buffer this iteration writes
            if (staged) {
                mode = (h->stage_iters == 0 || n <= h->stage_iters) ? 4 : 3;
                if (mode == 4) {
                    // the first stage on the current residual, in the caller's dense layout
                    CU(h, launch_to_caller(L, l1.f, 0, h->stage_r, s));
                    const int rc = h->stage_fn(h->stage_ctx, h->stage_r, h->stage_z, (void *)s);
                    if (rc) return fail(h, BBMG_BAD_ARGS, "preconditioner stage returned %d at iteration %d", rc, n);
                    CU(h, cudaGetLastError());
                    CU(h, launch_from_caller<double>(L, h->stage_z, 0, h->z1, s));
                    launches += 2;
                    stage_it++;
                }
            }
            cudaGraphExec_t ge = nullptr;
            if ((st = get_graph(h, mode, par, &ge))) return st;
            CU(h, cudaGraphLaunch(ge, s));
            launches += h->gkernels[mode][par];
            double mr = 0.0;
            if ((st = sync_read(h, &mr, kScalRes))) return st;
            rerr = mr / rnorm;  // bbmg_class.f90:696,723 (rnorm = res0 there)
            it = n;
            hist.push_back(rerr);
            if (!(rerr == rerr) || std::isinf(rerr)) {
                status = fail(h, BBMG_NONFINITE, "residual became non-finite at iteration %d", n);
                break;
            }
            if (rerr <= h->prm.rcvg) break;
            // An FP32 V-cycle cannot resolve error components below its rounding
            // floor (high-contrast coefficients make them large): when the
            // residual drops by less than 10 % over three iterations, the rest
            // of the solve runs the plain FP64 method from the current iterate.
            if (mode >= 2 && n >= 4 && rerr > 0.9 * hist[n - 4]) {
                if (mode == 3 || mode == 4) {
                    // restart CG (beta = 0) with the FP64 V-cycle as preconditioner
                    CU(h, cudaMemsetAsync(l1.v, 0, sizeof(double) * L.plane, s));
                    CU(h, cudaMemsetAsync(h->sc, 0, sizeof(CgScal), s));
                    mode = 1;
                    staged = false;
                } else {
                    // mgsolve's cycles act on lvl(1)%v in place: move x there
                    if (xout != l1.v)
                        CU(h, cudaMemcpyAsync(l1.v, xout, sizeof(double) * L.plane, cudaMemcpyDeviceToDevice, s));
                    xout = l1.v;
                    mode = 0;
                    pingpong = false;
                }
                fallback_it = n;
            }
        }
        if (status == BBMG_OK && rerr > h->prm.rcvg) status = BBMG_MAXIT;
    }
    // the true FP64 residual of the returned solution: recomputed from b and
    // x, independent of the iteration's own residual (the CG recurrence)
    double true_res = 0.0, true_l2 = 0.0;
    const bool verify = res0 != 0.0 && status != BBMG_NONFINITE;
    if (verify) {
        double *bvec = krylov ? h->b1 : l1.f;
        double *rscr = krylov ? h->Ap : l1.r;
        // the CG solution is updated on the interior only: refresh its periodic images
        if (krylov && (L.xper || L.yper || L.zper)) CU(h, wrap_planes(L, xout, 1, s));
        CU(h, launch_residual<double>(L, l1.nb, l1.npt, l1.oprS, xout, bvec, rscr, s));
        CU(h, launch_maxabs<double>(L, rscr, h->part, h->dscal + kScalTrue, s));
        CU(h, launch_dot<double>(L, rscr, rscr, h->part, h->dscal + kScalTrueL2, s));
        CU(h, cudaMemcpyAsync(h->h_scal + kScalTrue, h->dscal + kScalTrue, 2 * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
        launches += 5 + ((krylov && (L.xper || L.yper || L.zper)) ? 1 : 0);
    }
    // solution out (ils_class.f90:782-788)
    if (sol_dev) {
        CU(h, launch_to_caller(L, xout, g, sol, s));
    } else {
        // d_io still holds the caller's sol (copied in last), so its overlap
        // layers go back unchanged
        CU(h, launch_to_caller(L, xout, g, h->d_io, s));
        CU(h, h->copier.d2h(sol, h->d_io, sizeof(double) * ncaller, s));
    }
    if (krylov && status != BBMG_NONFINITE)  // the reference puts the solution back into lvl(1)%v (702)
        CU(h, cudaMemcpyAsync(l1.v, h->sol, sizeof(double) * L.plane, cudaMemcpyDeviceToDevice, s));
    CU(h, cudaEventRecord(h->ev1, s));
    CU(h, cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    if (verify) {
        true_res = h->h_scal[kScalTrue];
        true_l2 = std::sqrt(h->h_scal[kScalTrueL2]);
    }
    h->info.solve_ms = ms;
    h->info.it = it;
    h->info.rerr = rerr;
    h->info.res0 = res0;
    h->info.true_res = verify ? true_res : (res0 == 0.0 ? 0.0 : res0);
    h->info.true_rerr = verify ? true_res / rnorm : (res0 == 0.0 ? 0.0 : rerr);
    h->info.l2_rerr = verify ? (rnorm2 > 0.0 ? true_l2 / std::sqrt(rnorm2) : 0.0) : (res0 == 0.0 ? 0.0 : rerr);
    h->info.status = status;
    h->info.launches = launches + 1;
    h->info.fallback_it = fallback_it;
    h->info.stage_it = stage_it;
    if (it_out) *it_out = it;
    if (rerr_out) *rerr_out = rerr;
    return status;
}

int bbmg_get_info(const bbmg_handle *h, bbmg_info *info) {
    if (!h || !info) return BBMG_BAD_ARGS;
    *info = h->info;
    return BBMG_OK;
}

// ---------------------------------------------------------------------------
// step-level access
static int array_of(bbmg_handle *h, int n, int which, int prec, void **p, int *nc, bool *is32) {
    if (n < 1 || n > h->nlvl) return fail(h, BBMG_BAD_ARGS, "level %d out of range", n);
    Level &l = h->lv[n];
    *is32 = prec == 1;
    switch (which) {
    case BBMG_ARR_OPR: *p = prec ? (void *)l.oprS32 : (void *)l.opr27; *nc = prec ? l.npt : 27; break;
    case BBMG_ARR_C2F: *p = prec ? (void *)l.c2f32 : (void *)l.c2f; *nc = 8; break;
    case BBMG_ARR_F2C: *p = prec ? nullptr : (void *)l.f2c; *nc = 27; break;
    case BBMG_ARR_OPRC2F: *p = prec ? nullptr : (void *)l.oprc2f; *nc = 27; break;
    case BBMG_ARR_V: *p = prec ? (void *)l.v32 : (void *)l.v; *nc = 1; break;
    case BBMG_ARR_F: *p = prec ? (void *)l.f32 : (void *)l.f; *nc = 1; break;
    case BBMG_ARR_R: *p = prec ? (void *)l.r32 : (void *)l.r; *nc = 1; break;
    default: return fail(h, BBMG_BAD_ARGS, "unknown array %d", which);
    }
    if (!*p) return fail(h, BBMG_BAD_ARGS, "array %d not held on level %d (prec %d)", which, n, prec);
    return BBMG_OK;
}

long long bbmg_debug_get(bbmg_handle *h, int n, int which, int prec, double *out) {
    if (!h) return -BBMG_BAD_ARGS;
    void *p; int nc; bool is32;
    int st = array_of(h, n, which, prec, &p, &nc, &is32);
    if (st) return -st;
    const Lay &L = h->lv[n].L;
    long long cells = (long long)(L.nx + 2) * (L.ny + 2) * (L.nz + 2);
    if (!out) return cells * nc;
    if (cudaSetDevice(h->device) != cudaSuccess) return -fail(h, BBMG_CUDA, "device");
    // the setup does not fill the overlap of these two (nothing reads it there)
    if (h->setup_done && which == BBMG_ARR_F2C && n > 1 && fill_overlap_f2c(L, (double *)p, h->stream) != cudaSuccess)
        return -fail(h, BBMG_CUDA, "overlap");
    if (h->setup_done && which == BBMG_ARR_OPRC2F && n < h->nlvl &&
        fill_overlap_oprc2f(L, (double *)p, h->stream) != cudaSuccess)
        return -fail(h, BBMG_CUDA, "overlap");
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return -fail(h, BBMG_CUDA, "sync");
    size_t es = is32 ? 4 : 8;
    std::vector<char> buf((size_t)nc * L.plane * es);
    if (cudaMemcpy(buf.data(), p, buf.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return -fail(h, BBMG_CUDA, "copy");
    long long t = 0;
    for (int k = -1; k <= L.nz; k++)
        for (int j = -1; j <= L.ny; j++)
            for (int i = -1; i <= L.nx; i++, t++) {
                long long id = L.idx(i, j, k);
                for (int q = 0; q < nc; q++) {
                    size_t e = (size_t)q * L.plane + id;
                    out[t * nc + q] = is32 ? (double)((float *)buf.data())[e] : ((double *)buf.data())[e];
                }
            }
    return cells * nc;
}

long long bbmg_debug_put(bbmg_handle *h, int n, int which, int prec, const double *in) {
    if (!h || !in) return -BBMG_BAD_ARGS;
    if (which != BBMG_ARR_V && which != BBMG_ARR_F && which != BBMG_ARR_R)
        return -fail(h, BBMG_BAD_ARGS, "only vectors can be written");
    void *p; int nc; bool is32;
    int st = array_of(h, n, which, prec, &p, &nc, &is32);
    if (st) return -st;
    const Lay &L = h->lv[n].L;
    if (cudaSetDevice(h->device) != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess)
        return -fail(h, BBMG_CUDA, "sync");
    size_t es = is32 ? 4 : 8;
    std::vector<char> buf((size_t)L.plane * es, 0);
    long long t = 0;
    for (int k = -1; k <= L.nz; k++)
        for (int j = -1; j <= L.ny; j++)
            for (int i = -1; i <= L.nx; i++, t++) {
                long long id = L.idx(i, j, k);
                if (is32) ((float *)buf.data())[id] = (float)in[t];
                else ((double *)buf.data())[id] = in[t];
            }
    if (cudaMemcpy(p, buf.data(), buf.size(), cudaMemcpyHostToDevice) != cudaSuccess) return -fail(h, BBMG_CUDA, "copy");
    return t;
}

}  // extern "C"

template <typename T>
static int debug_step_t(bbmg_handle *h, int step, int n, int arg) {
    using P = LvlPtr<T>;
    cudaStream_t s = h->stream;
    Level &l = h->lv[n];
    switch (step) {
    case BBMG_STEP_RELAX:
        CU(h, launch_relax<T>(l.L, l.nb, l.npt, l.fuse, P::opr(l), P::v(l), P::f(l), arg >= 0 ? 1 : -1, s));
        break;
    case BBMG_STEP_RESIDUAL:
        CU(h, launch_residual<T>(l.L, l.nb, l.npt, P::opr(l), P::v(l), P::f(l), P::r(l), s));
        break;
    case BBMG_STEP_RESTRICT:
        if (n >= h->nlvl) return fail(h, BBMG_BAD_ARGS, "no coarser level");
        CU(h, launch_restrict<T>(l.L, h->lv[n + 1].L, P::c2f(l), P::r(l), P::f(h->lv[n + 1]), P::v(h->lv[n + 1]), s));
        break;
    case BBMG_STEP_PROLONG:
        if (n >= h->nlvl) return fail(h, BBMG_BAD_ARGS, "no coarser level");
        CU(h, launch_prolong<T>(l.L, h->lv[n + 1].L, P::c2f(l), P::v(h->lv[n + 1]), P::v(l), s));
        break;
    case BBMG_STEP_CYCLE: {
        if (n > 1) CU(h, cudaMemsetAsync(P::v(l), 0, sizeof(T) * l.L.plane, s));
        int st = vcycle<T>(h, n);
        if (st) return st;
        break;
    }
    case BBMG_STEP_DIRECT: {
        Level &c = h->lv[h->nlvl];
        CU(h, launch_coarse_solve<T>(c.L, h->LU, h->piv, h->pinned, P::f(c), P::v(c), s));
        break;
    }
    default: return fail(h, BBMG_BAD_ARGS, "unknown step %d", step);
    }
    CU(h, cudaStreamSynchronize(s));
    return BBMG_OK;
}

extern "C" {

int bbmg_debug_step(bbmg_handle *h, int step, int n, int arg, int prec) {
    if (!h) return BBMG_BAD_ARGS;
    if (!h->setup_done) return fail(h, BBMG_NOT_SETUP, "not set up");
    if (n < 1 || n > h->nlvl) return fail(h, BBMG_BAD_ARGS, "level %d out of range", n);
    if (prec == 1 && h->prm.precision != BBMG_PREC_MIXED) return fail(h, BBMG_BAD_ARGS, "no FP32 copy (FP64 handle)");
    CU(h, cudaSetDevice(h->device));
    return prec == 1 ? debug_step_t<float>(h, step, n, arg) : debug_step_t<double>(h, step, n, arg);
}

int bbmg_profile_step(bbmg_handle *h, int step, int n, int arg, int prec, int reps, double *ms) {
    if (!h || !ms || reps < 1) return BBMG_BAD_ARGS;
    if (!h->setup_done) return fail(h, BBMG_NOT_SETUP, "not set up");
    if (n < 1 || n > h->nlvl) return fail(h, BBMG_BAD_ARGS, "level %d out of range", n);
    if (prec == 1 && h->prm.precision != BBMG_PREC_MIXED) return fail(h, BBMG_BAD_ARGS, "no FP32 copy (FP64 handle)");
    if (step != BBMG_STEP_RELAX && step != BBMG_STEP_RESIDUAL && step != BBMG_STEP_RESTRICT &&
        step != BBMG_STEP_PROLONG && step != BBMG_STEP_CYCLE)
        return fail(h, BBMG_BAD_ARGS, "step %d cannot be profiled", step);
    if ((step == BBMG_STEP_RESTRICT || step == BBMG_STEP_PROLONG) && n >= h->nlvl)
        return fail(h, BBMG_BAD_ARGS, "no coarser level");
    CU(h, cudaSetDevice(h->device));
    cudaStream_t s = h->stream;
    Level &l = h->lv[n];
    CU(h, cudaEventRecord(h->ev0, s));
    for (int r = 0; r < reps; r++) {
        cudaError_t e = cudaSuccess;
        if (step == BBMG_STEP_CYCLE) {  // cycle(n) as the solve runs it (the fused tail included)
            int st = prec == 1 ? vcycle<float>(h, n) : vcycle<double>(h, n);
            if (st) return st;
            continue;
        }
        if (prec == 1) {
            using P = LvlPtr<float>;
            if (step == BBMG_STEP_RELAX) e = launch_relax_sweeps<float>(l.L, l.nb, l.npt, l.fuse, P::opr(l), P::v(l), P::f(l), arg >= 0 ? 1 : -1, 1, s);
            else if (step == BBMG_STEP_RESIDUAL) e = launch_residual<float>(l.L, l.nb, l.npt, P::opr(l), P::v(l), P::f(l), P::r(l), s);
            else if (step == BBMG_STEP_RESTRICT) e = launch_restrict<float>(l.L, h->lv[n + 1].L, P::c2f(l), P::r(l), P::f(h->lv[n + 1]), P::v(h->lv[n + 1]), s);
            else e = launch_prolong<float>(l.L, h->lv[n + 1].L, P::c2f(l), P::v(h->lv[n + 1]), P::v(l), s);
        } else {
            using P = LvlPtr<double>;
            if (step == BBMG_STEP_RELAX) e = launch_relax_sweeps<double>(l.L, l.nb, l.npt, l.fuse, P::opr(l), P::v(l), P::f(l), arg >= 0 ? 1 : -1, 1, s);
            else if (step == BBMG_STEP_RESIDUAL) e = launch_residual<double>(l.L, l.nb, l.npt, P::opr(l), P::v(l), P::f(l), P::r(l), s);
            else if (step == BBMG_STEP_RESTRICT) e = launch_restrict<double>(l.L, h->lv[n + 1].L, P::c2f(l), P::r(l), P::f(h->lv[n + 1]), P::v(h->lv[n + 1]), s);
            else e = launch_prolong<double>(l.L, h->lv[n + 1].L, P::c2f(l), P::v(h->lv[n + 1]), P::v(l), s);
        }
        CU(h, e);
    }
    CU(h, cudaEventRecord(h->ev1, s));
    CU(h, cudaEventSynchronize(h->ev1));
    float t = 0.f;
    CU(h, cudaEventElapsedTime(&t, h->ev0, h->ev1));
    *ms = (double)t / reps;
    return BBMG_OK;
}

int bbmg_debug_direct(bbmg_handle *h, double *op, double *lu, int *piv, int *np) {
    if (!h) return BBMG_BAD_ARGS;
    if (np) *np = h->np;
    CU(h, cudaSetDevice(h->device));
    CU(h, cudaStreamSynchronize(h->stream));
    int n = h->np;
    std::vector<double> t((size_t)n * n);
    auto tr = [&](const double *d, double *o) -> int {
        CU(h, cudaMemcpy(t.data(), d, sizeof(double) * t.size(), cudaMemcpyDeviceToHost));
        for (int r = 0; r < n; r++)
            for (int c = 0; c < n; c++) o[(size_t)r * n + c] = t[(size_t)c * n + r];
        return BBMG_OK;
    };
    if (op) { int st = tr(h->OP, op); if (st) return st; }
    if (lu) { int st = tr(h->LU, lu); if (st) return st; }
    if (piv) CU(h, cudaMemcpy(piv, h->piv, sizeof(int) * n, cudaMemcpyDeviceToHost));
    return BBMG_OK;
}

}  // extern "C"
