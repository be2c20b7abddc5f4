// projection.cu -- the steps of the flow solvers' time loop around the
// pressure solve on the GPU (nga_projection.h): operator assembly, divergence
// and right-hand side, mean removal, pressure gradient and velocity
// correction; get_dmomdt, the sub-iteration updates and the flow statistics
// of the incompressible time loop.
//
// Every kernel is a single pass over the interior (or, for the whole-array
// updates, the padded array) in the caller's Fortran layout (i fastest): one
// thread per cell, consecutive threads on consecutive i, so every array
// access of a warp is one contiguous run.  The metrics are 1-D (a rectilinear
// pgrid) and stay in L1.  HBM traffic per cell, FP64: assembly 3 face
// densities in + 7 coefficients out (80 B); divergence 3 velocities in + div
// and rhs out (40 B); correction sol, 3 densities, 3 velocities and P in,
// 3 velocities and P out (96 B); mean removal 2 passes of 8 + 16 B;
// get_dmomdt U, V, W, P, visc in + 3 derivatives out (64 B, the neighbour
// planes from L1/L2); midpoint 72 B; explicit update 96 B; statistics 24 B.
//
// Arithmetic follows the reference's expressions term for term with
// __dadd_rn / __dmul_rn / __ddiv_rn (no contraction), so outputs equal the
// reference's bits; only shift_p's volume sum is reduced in a different
// (fixed) order.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/nga_projection.h"

namespace bbmg {
void set_create_error(const char *msg);  // api.cu
}

struct nga_proj {
    bbmg_grid g{};
    int device = 0;
    cudaStream_t stream = nullptr;
    // per direction (x, y, z): divp(0), divp(1) on the n cells; divu(-1),
    // divu(0) on the n+1 faces; cell sizes d (for the volume)
    double *dp0[3] = {nullptr, nullptr, nullptr}, *dp1[3] = {nullptr, nullptr, nullptr};
    double *du0[3] = {nullptr, nullptr, nullptr}, *du1[3] = {nullptr, nullptr, nullptr};
    double *d[3] = {nullptr, nullptr, nullptr};
    double *metrics = nullptr;  // one allocation holding all of the above
    double *part = nullptr;     // reduction partials + the mean
    double vol_total = 0.0;
    // momentum metrics per direction (two layers of the naive extension):
    // dxi on cells -1..n (index c+1), dxmi and the edge weights itm (of the
    // value at f-1) and itz (of the value at f) on faces 0..n
    const double *mom[3][10] = {};  // per direction, in momentum_metrics' order
    double *mmetrics = nullptr;
};

namespace {

constexpr int kRedBlocks = 148 * 8;
constexpr int kThreads = 256;

int pfail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    bbmg::set_create_error(buf);
    return code;
}

#define PCU(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return pfail(e_ == cudaErrorMemoryAllocation ? BBMG_NO_MEMORY : BBMG_CUDA, "%s: %s (%s:%d)", \
                         #call, cudaGetErrorString(e_), __FILE__, __LINE__);                             \
    } while (0)

bool on_device(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Padded-array geometry of the caller's arrays.
struct Pad {
    int nx, ny, nz, g;
    long long sy, sz;  // strides of j and k
    __host__ __device__ long long at(int i, int j, int k) const {
        return (long long)(k + g) * sz + (long long)(j + g) * sy + (i + g);
    }
};

Pad pad_of(const bbmg_grid &g) {
    Pad p;
    p.nx = g.nx; p.ny = g.ny; p.nz = g.nz; p.g = g.ghost;
    p.sy = g.nx + 2LL * g.ghost;
    p.sz = p.sy * (g.ny + 2LL * g.ghost);
    return p;
}

struct Metrics {
    const double *dp0x, *dp1x, *du0x, *du1x, *dx;
    const double *dp0y, *dp1y, *du0y, *du1y, *dy;
    const double *dp0z, *dp1z, *du0z, *du1z, *dz;
};

Metrics metrics_of(const nga_proj *p) {
    return {p->dp0[0], p->dp1[0], p->du0[0], p->du1[0], p->d[0], p->dp0[1], p->dp1[1], p->du0[1],
            p->du1[1], p->d[1],   p->dp0[2], p->dp1[2], p->du0[2], p->du1[2], p->d[2]};
}

__device__ __forceinline__ void cell_of(const Pad &P, long long t, int &i, int &j, int &k) {
    i = (int)(t % P.nx);
    const long long r = t / P.nx;
    j = (int)(r % P.ny);
    k = (int)(r / P.ny);
}

__device__ __forceinline__ double rho_at(const double *r, long long e) { return r ? r[e] : 1.0; }

// (a*b)/c, the reference's divp*divu/rho_face
__device__ __forceinline__ double mdv(double a, double b, double c) { return __ddiv_rn(__dmul_rn(a, b), c); }

// update_laplacian (tpns_class.f90:1565-1593), one cell per thread
__global__ void __launch_bounds__(kThreads) k_laplacian(Pad P, Metrics M, const double *__restrict__ rU,
                                                         const double *__restrict__ rV,
                                                         const double *__restrict__ rW, double *__restrict__ opr) {
    const long long n = (long long)P.nx * P.ny * P.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const long long e = P.at(i, j, k);
        const double rUp = rho_at(rU, e + 1), rUm = rho_at(rU, e);
        const double rVp = rho_at(rV, e + P.sy), rVm = rho_at(rV, e);
        const double rWp = rho_at(rW, e + P.sz), rWm = rho_at(rW, e);
        double o[7];
        o[0] = mdv(M.dp1x[i], M.du0x[i + 1], rUp);
        o[0] = __dadd_rn(o[0], mdv(M.dp0x[i], M.du1x[i], rUm));
        o[0] = __dadd_rn(o[0], mdv(M.dp1y[j], M.du0y[j + 1], rVp));
        o[0] = __dadd_rn(o[0], mdv(M.dp0y[j], M.du1y[j], rVm));
        o[0] = __dadd_rn(o[0], mdv(M.dp1z[k], M.du0z[k + 1], rWp));
        o[0] = __dadd_rn(o[0], mdv(M.dp0z[k], M.du1z[k], rWm));
        o[1] = mdv(M.dp1x[i], M.du1x[i + 1], rUp);
        o[2] = mdv(M.dp0x[i], M.du0x[i], rUm);
        o[3] = mdv(M.dp1y[j], M.du1y[j + 1], rVp);
        o[4] = mdv(M.dp0y[j], M.du0y[j], rVm);
        o[5] = mdv(M.dp1z[k], M.du1z[k + 1], rWp);
        o[6] = mdv(M.dp0z[k], M.du0z[k], rWm);
        // opr = -opr*vol, vol = dx*dy*dz (config_class.f90:108)
        const double vol = __dmul_rn(__dmul_rn(M.dx[i], M.dy[j]), M.dz[k]);
        double *out = opr + 7 * e;
#pragma unroll
        for (int q = 0; q < 7; q++) out[q] = __dmul_rn(-o[q], vol);
    }
}

// get_div (incomp_class.f90:1144-1159) and rhs = -vol*div*rho/dt
__global__ void __launch_bounds__(kThreads) k_divergence(Pad P, Metrics M, const double *__restrict__ U,
                                                          const double *__restrict__ V,
                                                          const double *__restrict__ W, double rho, double dt,
                                                          double *__restrict__ div, double *__restrict__ rhs) {
    const long long n = (long long)P.nx * P.ny * P.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const long long e = P.at(i, j, k);
        const double sx = __dadd_rn(__dmul_rn(M.dp0x[i], U[e]), __dmul_rn(M.dp1x[i], U[e + 1]));
        const double sy = __dadd_rn(__dmul_rn(M.dp0y[j], V[e]), __dmul_rn(M.dp1y[j], V[e + P.sy]));
        const double sz = __dadd_rn(__dmul_rn(M.dp0z[k], W[e]), __dmul_rn(M.dp1z[k], W[e + P.sz]));
        const double d = __dadd_rn(__dadd_rn(sx, sy), sz);
        if (div) div[e] = d;
        if (rhs) {
            const double vol = __dmul_rn(__dmul_rn(M.dx[i], M.dy[j]), M.dz[k]);
            rhs[e] = -__ddiv_rn(__dmul_rn(__dmul_rn(vol, d), rho), dt);
        }
    }
}

// block partial sums of vol*p (config_class.f90:196-214 with VF = 1), a fixed
// grid and a fixed per-thread order: the same bits on every call
__global__ void __launch_bounds__(kThreads) k_vol_sum(Pad P, Metrics M, const double *__restrict__ p,
                                                       double *__restrict__ part) {
    __shared__ double sh[kThreads];
    const long long n = (long long)P.nx * P.ny * P.nz;
    double s = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const double vol = __dmul_rn(__dmul_rn(M.dx[i], M.dy[j]), M.dz[k]);
        s = __dadd_rn(s, __dmul_rn(vol, p[P.at(i, j, k)]));
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + h]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// mean = (sum of the partials) / fluid_vol into part[kRedBlocks]
__global__ void __launch_bounds__(kThreads) k_vol_mean(double *__restrict__ part, double fluid_vol) {
    __shared__ double sh[kThreads];
    double s = 0.0;
    for (int b = threadIdx.x; b < kRedBlocks; b += kThreads) s = __dadd_rn(s, part[b]);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + h]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[kRedBlocks] = __ddiv_rn(sh[0], fluid_vol);
}

__global__ void __launch_bounds__(kThreads) k_shift(Pad P, const double *__restrict__ mean, double *__restrict__ p) {
    const long long n = (long long)P.nx * P.ny * P.nz;
    const double m = *mean;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const long long e = P.at(i, j, k);
        p[e] = __dsub_rn(p[e], m);
    }
}

// get_pgrad (incomp_class.f90:1163-1184): sum(divu_x(:,i) P(i-1:i)), ...
__global__ void __launch_bounds__(kThreads) k_pgrad(Pad P, Metrics M, const double *__restrict__ p,
                                                     double *__restrict__ gx, double *__restrict__ gy,
                                                     double *__restrict__ gz) {
    const long long n = (long long)P.nx * P.ny * P.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const long long e = P.at(i, j, k);
        const double pc = p[e];
        gx[e] = __dadd_rn(__dmul_rn(M.du0x[i], p[e - 1]), __dmul_rn(M.du1x[i], pc));
        gy[e] = __dadd_rn(__dmul_rn(M.du0y[j], p[e - P.sy]), __dmul_rn(M.du1y[j], pc));
        gz[e] = __dadd_rn(__dmul_rn(M.du0z[k], p[e - P.sz]), __dmul_rn(M.du1z[k], pc));
    }
}

// P += sol; U -= dt*gradx(sol)/rho_U; V, W likewise (falling_drop
// simulation.f90:308-313 with get_pgrad inlined)
__global__ void __launch_bounds__(kThreads) k_correct(Pad P, Metrics M, const double *__restrict__ s, double dt,
                                                       const double *__restrict__ rU, const double *__restrict__ rV,
                                                       const double *__restrict__ rW, double *__restrict__ pres,
                                                       double *__restrict__ U, double *__restrict__ V,
                                                       double *__restrict__ W) {
    const long long n = (long long)P.nx * P.ny * P.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const long long e = P.at(i, j, k);
        const double sc = s[e];
        const double gx = __dadd_rn(__dmul_rn(M.du0x[i], s[e - 1]), __dmul_rn(M.du1x[i], sc));
        const double gy = __dadd_rn(__dmul_rn(M.du0y[j], s[e - P.sy]), __dmul_rn(M.du1y[j], sc));
        const double gz = __dadd_rn(__dmul_rn(M.du0z[k], s[e - P.sz]), __dmul_rn(M.du1z[k], sc));
        if (pres) pres[e] = __dadd_rn(pres[e], sc);
        U[e] = __dsub_rn(U[e], __ddiv_rn(__dmul_rn(dt, gx), rho_at(rU, e)));
        V[e] = __dsub_rn(V[e], __ddiv_rn(__dmul_rn(dt, gy), rho_at(rV, e)));
        W[e] = __dsub_rn(W[e], __ddiv_rn(__dmul_rn(dt, gz), rho_at(rW, e)));
    }
}

__device__ __forceinline__ int wrap_coord(int per, int c, int n) {
    if (!per) return c;
    if (c < 0) return c + n * ((-c + n - 1) / n);
    if (c >= n) return c - n * (c / n);
    return c;
}

// cfg%sync on one rank: every overlap cell with a coordinate outside the
// interior of a periodic direction takes the value of the cell reached by
// wrapping those coordinates (the reference copies x, then y, then z over the
// full extent of the other directions, which amounts to the same).  Sources
// are never themselves periodic images, so one gather pass suffices.
struct SyncArrays {
    double *a[4];
    int n;
};

__global__ void __launch_bounds__(kThreads) k_sync(Pad P, int xper, int yper, int zper, SyncArrays A) {
    const long long ex = P.nx + 2LL * P.g, ey = P.ny + 2LL * P.g, ez = P.nz + 2LL * P.g;
    const long long n = ex * ey * ez;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % ex) - P.g;
        const long long r = t / ex;
        const int j = (int)(r % ey) - P.g, k = (int)(r / ey) - P.g;
        const int si = wrap_coord(xper, i, P.nx), sj = wrap_coord(yper, j, P.ny), sk = wrap_coord(zper, k, P.nz);
        if (si == i && sj == j && sk == k) continue;
        const long long d = P.at(i, j, k), s = P.at(si, sj, sk);
        for (int q = 0; q < A.n; q++) A.a[q][d] = A.a[q][s];
    }
}

unsigned grid_cells(long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    const long long cap = 148LL * 16;
    if (b > cap) b = cap;
    return (unsigned)(b < 1 ? 1 : b);
}

int sync_arrays(nga_proj *p, double *a0, double *a1, double *a2, double *a3) {
    const bbmg_grid &g = p->g;
    if (!(g.xper || g.yper || g.zper) || g.ghost == 0) return BBMG_OK;
    SyncArrays A{{a0, a1, a2, a3}, 0};
    double *all[4] = {a0, a1, a2, a3};
    for (double *x : all)
        if (x) A.a[A.n++] = x;
    if (A.n == 0) return BBMG_OK;
    const Pad P = pad_of(g);
    const long long n = (g.nx + 2LL * g.ghost) * (g.ny + 2LL * g.ghost) * (g.nz + 2LL * g.ghost);
    k_sync<<<grid_cells(n), kThreads, 0, p->stream>>>(P, g.xper, g.yper, g.zper, A);
    PCU(cudaGetLastError());
    return BBMG_OK;
}

// Metrics of one direction from its n+1 nodes (sgrid_class.f90:160-254 with
// the naive extension; incomp_class.f90:355-380 for divp/divu; the wall faces
// of a non-periodic direction get divu = 0, incomp_class.f90:529-563).
void axis_metrics(const double *x, int n, bool per, std::vector<double> &dp0, std::vector<double> &dp1,
                  std::vector<double> &du0, std::vector<double> &du1, std::vector<double> &d) {
    std::vector<double> xe(n + 3), xm(n + 2);
    for (int i = 0; i <= n; i++) xe[i + 1] = x[i];
    xe[0] = xe[1] - (xe[2] - xe[1]);
    xe[n + 2] = xe[n + 1] + (xe[n + 1] - xe[n]);
    for (int m = 0; m <= n + 1; m++) xm[m] = 0.5 * (xe[m] + xe[m + 1]);
    dp0.assign(n, 0.0); dp1.assign(n, 0.0); d.assign(n, 0.0);
    du0.assign(n + 1, 0.0); du1.assign(n + 1, 0.0);
    for (int c = 0; c < n; c++) {
        d[c] = xe[c + 2] - xe[c + 1];
        const double di = 1.0 / d[c];
        dp0[c] = di * -1.0;
        dp1[c] = di * 1.0;
    }
    for (int f = 0; f <= n; f++) {
        const bool wall = !per && (f == 0 || f == n);
        const double dmi = 1.0 / (xm[f + 1] - xm[f]);
        du0[f] = wall ? 0.0 : dmi * -1.0;
        du1[f] = wall ? 0.0 : dmi * 1.0;
    }
}

// Momentum metrics of one direction (incomp_class.f90:250-446 with the mesh of
// sgrid_class.f90:160-254 extended naively by two layers).
// Momentum metrics of one direction (q order): 0 dxi on cells -1..n (index
// c+1); on faces 0..n: 1 dxmi, 2/3 the interpolation weights itm (value at
// f-1) and itz (value at f); with walls at both ends of a non-periodic
// direction (cfg%VF = 0 outside the domain, as the channel example sets it)
// the adjust_metrics versions (incomp_class.f90:449-700): 4/5 interpolation
// weights and 6 gradient coefficient of a velocity component tangential to
// the direction at its faces -- [1,0], [0,1] and [-1,+1]/delta on the two
// wall faces -- and 7/8 the 1-D factors of the edge viscosity weights with the
// wall cell's entry zeroed.  Periodic directions: 4-8 equal 2, 3, 1, 2, 3.
constexpr int kMomQ = 10;  // 9: the centroid spacing xm(f) - xm(f-1) itself (cfg%dxm)
void momentum_metrics(const double *x, int n, bool walls, std::vector<double> (&m)[kMomQ]) {
    std::vector<double> xe(n + 5), xm(n + 4);  // nodes -2..n+2, cells -2..n+1 at index +2
    for (int i = 0; i <= n; i++) xe[i + 2] = x[i];
    for (int k = 1; k >= 0; k--) xe[k] = xe[k + 1] - (xe[3] - xe[2]);
    for (int k = n + 3; k <= n + 4; k++) xe[k] = xe[k - 1] + (xe[n + 2] - xe[n + 1]);
    for (int k = 0; k < n + 4; k++) xm[k] = 0.5 * (xe[k] + xe[k + 1]);
    m[0].assign(n + 2, 0.0);
    for (int c = -1; c <= n; c++) m[0][c + 1] = 1.0 / (xe[c + 3] - xe[c + 2]);
    for (int q = 1; q < kMomQ; q++) m[q].assign(n + 1, 0.0);
    for (int f = 0; f <= n; f++) {
        const double dmi = 1.0 / (xm[f + 2] - xm[f + 1]);
        const double itm = dmi * (xm[f + 2] - xe[f + 2]), itz = dmi * (xe[f + 2] - xm[f + 1]);
        m[1][f] = dmi;
        m[9][f] = xm[f + 2] - xm[f + 1];
        m[2][f] = m[4][f] = m[7][f] = itm;
        m[3][f] = m[5][f] = m[8][f] = itz;
        m[6][f] = dmi;
    }
    if (walls) {
        m[4][0] = 1.0; m[5][0] = 0.0;                   // [1,0]: the wall-side value
        m[6][0] = 1.0 / (xm[2] - xe[2]);                 // delta = xm(0) - x(0)
        m[4][n] = 0.0; m[5][n] = 1.0;                   // [0,1]
        m[6][n] = 1.0 / (xe[n + 2] - xm[n + 1]);         // delta = x(n) - xm(n-1)
        m[7][0] = 0.0;                                   // cell -1 is wall
        m[8][n] = 0.0;                                   // cell n is wall
    }
}

struct MomM {
    const double *di[3], *dmi[3], *itm[3], *itz[3];
    const double *vtm[3], *vtz[3], *gdm[3], *wtm[3], *wtz[3], *dm[3];
    int nf[3];    // faces per direction minus one (n)
    int walls[3]; // walls at both ends (non-periodic direction)
    // a face of the component normal to direction d lies on a wall
    __device__ __forceinline__ bool wall_face(int d, int f) const { return walls[d] && (f == 0 || f == nf[d]); }
    // umask/vmask/wmask > 0 at padded indices (i, j, k) of component c: a
    // wall or overlap face of its own direction, or a wall-cell row of another
    __device__ __forceinline__ bool masked(int c, int i, int j, int k) const {
        const int f[3] = {i, j, k};
        bool m = false;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (!walls[d]) continue;
            m = m || (d == c ? (f[d] <= 0 || f[d] >= nf[d]) : (f[d] < 0 || f[d] >= nf[d]));
        }
        return m;
    }
    // interpolation weights and gradient coefficients (-g, +g) along d at face f
    // of a component whose own face is a wall face (cw: both values masked,
    // interpolation unchanged, gradient zero) or not
    __device__ __forceinline__ void tang(int d, int f, bool cw, double &tm, double &tz, double &gm, double &gz) const {
        if (cw) {
            tm = itm[d][f]; tz = itz[d][f]; gm = 0.0; gz = 0.0;
        } else {
            tm = vtm[d][f]; tz = vtz[d][f]; gz = gdm[d][f]; gm = -gz;
        }
    }
};

__device__ __forceinline__ double pa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double pm(double a, double b) { return __dmul_rn(a, b); }
// sum(a(:)*b(:)) over two entries, in order
__device__ __forceinline__ double two(double a0, double b0, double a1, double b1) { return pa(pm(a0, b0), pm(a1, b1)); }
// sum(itp2d(:,:)*visc(..)) with the lower index (l) fastest, where itp2d =
// itp_l(st1)*itp_h(st2) (incomp_class.f90:277-288) divided by its own sum
// (adjust_metrics, incomp_class.f90:505-511), summed in the same order
__device__ __forceinline__ double visc_edge(double lm, double lz, double hm, double hz, double v_mm, double v_zm,
                                            double v_mz, double v_zz) {
    double w_mm = pm(lm, hm), w_zm = pm(lz, hm), w_mz = pm(lm, hz), w_zz = pm(lz, hz);
    const double s = pa(pa(pa(w_mm, w_zm), w_mz), w_zz);
    if (s > 0.0) {
        w_mm = __ddiv_rn(w_mm, s);
        w_zm = __ddiv_rn(w_zm, s);
        w_mz = __ddiv_rn(w_mz, s);
        w_zz = __ddiv_rn(w_zz, s);
    }
    double t = pm(w_mm, v_mm);
    t = pa(t, pm(w_zm, v_zm));
    t = pa(t, pm(w_mz, v_mz));
    return pa(t, pm(w_zz, v_zz));
}
// -rho (itp_a Qa) (itp_b Qb) + vi (grd_a Qa + grd_b Qb)
__device__ __forceinline__ double edge_flux(double rho, double am, double az, double qam, double qa0, double bm,
                                            double bz, double qbm, double qb0, double gam, double gaz, double gbm,
                                            double gbz, double vi) {
    const double a = two(am, qam, az, qa0), b = two(bm, qbm, bz, qb0);
    const double g = pa(two(gam, qam, gaz, qa0), two(gbm, qbm, gbz, qb0));
    return pa(-pm(pm(rho, a), b), pm(vi, g));
}

// The edge flux in the plane (d1, d2) at faces f1 (along d1) and f2 (along d2)
// for Qa = the component along d2 varying along d1 and Qb = the component along
// d1 varying along d2 (e.g. d1 = y, d2 = x: U along y, V along x), element o
// at the edge's upper corner; sa, sb the strides along d1 and d2; the
// viscosity weights with the lower of the two directions first.
__device__ __forceinline__ double edge_at(const MomM &M, double rho, int d1, int f1, int d2, int f2,
                                          const double *__restrict__ Qa, const double *__restrict__ Qb, long long o,
                                          long long sa, long long sb, double vi) {
    double am, az, gam, gaz, bm, bz, gbm, gbz;
    M.tang(d1, f1, M.wall_face(d2, f2), am, az, gam, gaz);
    M.tang(d2, f2, M.wall_face(d1, f1), bm, bz, gbm, gbz);
    return edge_flux(rho, am, az, Qa[o - sa], Qa[o], bm, bz, Qb[o - sb], Qb[o], gam, gaz, gbm, gbz, vi);
}

// get_dmomdt (incomp_class.f90:1021-1159), one thread per cell computing the
// three face derivatives there; every flux is recomputed by the threads that
// need it (the same bits each time) instead of being stored.  Terms and order
// follow the reference expression by expression.  Non-periodic directions have
// walls at both ends: the edge coefficients come from the adjusted metrics
// (MomM::tang, the wall-zeroed viscosity weights) and the derivative of the
// component normal to a wall is zero on the wall face (divu = 0 where umask > 0).
__global__ void __launch_bounds__(kThreads) k_dmomdt(Pad P, MomM M, const double *__restrict__ U,
                                                      const double *__restrict__ V, const double *__restrict__ W,
                                                      const double *__restrict__ Pr, double rho,
                                                      const double *__restrict__ visc, double visc0,
                                                      double *__restrict__ dU, double *__restrict__ dV,
                                                      double *__restrict__ dW) {
    const long long n = (long long)P.nx * P.ny * P.nz;
    const double c23 = 2.0 / 3.0;
    const long long sx = 1, sy = P.sy, sz = P.sz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const long long e = P.at(i, j, k);
        auto vs = [&](long long o) { return visc ? visc[o] : visc0; };
        // divergence at the cell at element o with cell indices (ci, cj, ck)
        auto divc = [&](long long o, int ci, int cj, int ck) {
            const double dx = M.di[0][ci + 1], dy = M.di[1][cj + 1], dz = M.di[2][ck + 1];
            const double a = two(-dx, U[o], dx, U[o + sx]);
            const double b = two(-dy, V[o], dy, V[o + sy]);
            const double c = two(-dz, W[o], dz, W[o + sz]);
            return pa(pa(a, b), c);
        };
        // normal flux of component Q along direction d at the cell at element o
        auto normal = [&](const double *Q, long long st, double dci, long long o, int ci, int cj, int ck) {
            const double q0 = Q[o], q1 = Q[o + st];
            const double s1 = two(0.5, q0, 0.5, q1);
            const double g = two(-dci, q0, dci, q1);
            const double vt = pm(vs(o), __dsub_rn(pa(g, g), pm(c23, divc(o, ci, cj, ck))));
            return __dsub_rn(pa(-pm(pm(rho, s1), s1), vt), Pr[o]);
        };
        // ---- rho U at x-face i
        {
            const double fxm = normal(U, sx, M.di[0][i], e - sx, i - 1, j, k);
            const double fx0 = normal(U, sx, M.di[0][i + 1], e, i, j, k);
            double fy[2], fz[2];
#pragma unroll
            for (int oy = 0; oy < 2; oy++) {  // xy edge (x-face i, y-face j+oy)
                const int f = j + oy;
                const long long o = e + oy * sy;
                const double vi = visc_edge(M.wtm[0][i], M.wtz[0][i], M.wtm[1][f], M.wtz[1][f], vs(o - sx - sy),
                                            vs(o - sy), vs(o - sx), vs(o));
                fy[oy] = edge_at(M, rho, 1, f, 0, i, U, V, o, sy, sx, vi);
            }
#pragma unroll
            for (int oz = 0; oz < 2; oz++) {  // xz edge (x-face i, z-face k+oz)
                const int f = k + oz;
                const long long o = e + oz * sz;
                const double vi = visc_edge(M.wtm[0][i], M.wtz[0][i], M.wtm[2][f], M.wtz[2][f], vs(o - sx - sz),
                                            vs(o - sz), vs(o - sx), vs(o));
                fz[oz] = edge_at(M, rho, 2, f, 0, i, U, W, o, sz, sx, vi);
            }
            const double dmx = M.dmi[0][i], dy = M.di[1][j + 1], dz = M.di[2][k + 1];
            dU[e] = M.wall_face(0, i) ? 0.0
                                      : pa(pa(two(-dmx, fxm, dmx, fx0), two(-dy, fy[0], dy, fy[1])),
                                           two(-dz, fz[0], dz, fz[1]));
        }
        // ---- rho V at y-face j
        {
            double fx[2], fz[2];
#pragma unroll
            for (int ox = 0; ox < 2; ox++) {  // xy edge (x-face i+ox, y-face j)
                const int f = i + ox;
                const long long o = e + ox * sx;
                const double vi = visc_edge(M.wtm[0][f], M.wtz[0][f], M.wtm[1][j], M.wtz[1][j], vs(o - sx - sy),
                                            vs(o - sy), vs(o - sx), vs(o));
                fx[ox] = edge_at(M, rho, 0, f, 1, j, V, U, o, sx, sy, vi);
            }
            const double fym = normal(V, sy, M.di[1][j], e - sy, i, j - 1, k);
            const double fy0 = normal(V, sy, M.di[1][j + 1], e, i, j, k);
#pragma unroll
            for (int oz = 0; oz < 2; oz++) {  // yz edge (y-face j, z-face k+oz)
                const int f = k + oz;
                const long long o = e + oz * sz;
                const double vi = visc_edge(M.wtm[1][j], M.wtz[1][j], M.wtm[2][f], M.wtz[2][f], vs(o - sy - sz),
                                            vs(o - sz), vs(o - sy), vs(o));
                fz[oz] = edge_at(M, rho, 2, f, 1, j, V, W, o, sz, sy, vi);
            }
            const double dx = M.di[0][i + 1], dmy = M.dmi[1][j], dz = M.di[2][k + 1];
            dV[e] = M.wall_face(1, j) ? 0.0
                                      : pa(pa(two(-dx, fx[0], dx, fx[1]), two(-dmy, fym, dmy, fy0)),
                                           two(-dz, fz[0], dz, fz[1]));
        }
        // ---- rho W at z-face k
        {
            double fx[2], fy[2];
#pragma unroll
            for (int ox = 0; ox < 2; ox++) {  // xz edge (x-face i+ox, z-face k)
                const int f = i + ox;
                const long long o = e + ox * sx;
                const double vi = visc_edge(M.wtm[0][f], M.wtz[0][f], M.wtm[2][k], M.wtz[2][k], vs(o - sx - sz),
                                            vs(o - sz), vs(o - sx), vs(o));
                fx[ox] = edge_at(M, rho, 0, f, 2, k, W, U, o, sx, sz, vi);
            }
#pragma unroll
            for (int oy = 0; oy < 2; oy++) {  // yz edge (y-face j+oy, z-face k)
                const int f = j + oy;
                const long long o = e + oy * sy;
                const double vi = visc_edge(M.wtm[1][f], M.wtz[1][f], M.wtm[2][k], M.wtz[2][k], vs(o - sy - sz),
                                            vs(o - sz), vs(o - sy), vs(o));
                fy[oy] = edge_at(M, rho, 1, f, 2, k, W, V, o, sy, sz, vi);
            }
            const double fzm = normal(W, sz, M.di[2][k], e - sz, i, j, k - 1);
            const double fz0 = normal(W, sz, M.di[2][k + 1], e, i, j, k);
            const double dx = M.di[0][i + 1], dy = M.di[1][j + 1], dmz = M.dmi[2][k];
            dW[e] = M.wall_face(2, k) ? 0.0
                                      : pa(pa(two(-dx, fx[0], dx, fx[1]), two(-dy, fy[0], dy, fy[1])),
                                           two(-dmz, fzm, dmz, fz0));
        }
    }
}

// ---------------------------------------------------------------------------
// The whole-array updates of a sub-iteration of the time loop (the hit
// example, simulation.f90:283-341): elementwise over the padded arrays, like
// the reference's array statements, so the overlap stays the periodic image.

struct Vel3 {
    double *a[3];
};
struct CVel3 {
    const double *a[3];
};

// U = 0.5*(U + Uold)
__global__ void __launch_bounds__(kThreads) k_midpoint(long long n, Vel3 U, CVel3 Uo) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; c++) U.a[c][t] = pm(0.5, pa(U.a[c][t], Uo.a[c][t]));
    }
}

// res = -2*(rho*U - rho*Uold) + dt*drhoUdt [+ (fa*(U - mean))/fb];
// U = 2*U - Uold + res/rho
__global__ void __launch_bounds__(kThreads) k_advance(long long n, double dt, double rho, Vel3 U, CVel3 Uo,
                                                      CVel3 dU, double fa, double fb, double m0, double m1,
                                                      double m2) {
    const double mean[3] = {m0, m1, m2};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const double u = U.a[c][t], uo = Uo.a[c][t];
            double r = pa(pm(-2.0, __dsub_rn(pm(rho, u), pm(rho, uo))), pm(dt, dU.a[c][t]));
            if (fa != 0.0) r = pa(r, __ddiv_rn(pm(fa, __dsub_rn(u, mean[c])), fb));
            U.a[c][t] = pa(__dsub_rn(pm(2.0, u), uo), __ddiv_rn(r, rho));
        }
    }
}

// The operator solve_implicit assembles for velocity component C
// (incomp_class.f90:1744-1910), one thread per cell (the component's face at
// the cell's lower side): rho + dt/2 (linearised convection) - dt/2
// (viscous terms), stencil order [0, +x, -x, +y, -y, +z, -z], written into the
// padded [k][j][i][7] array.  Per direction the two terms are summed upper
// then lower, x, y, z, as the reference does; the rows of the component's
// wall faces are rho alone (divu = 0 there).
template <int C>
__global__ void __launch_bounds__(kThreads) k_implicit_opr(Pad P, MomM M, const double *__restrict__ U,
                                                            const double *__restrict__ V,
                                                            const double *__restrict__ W,
                                                            const double *__restrict__ visc, double visc0, double rho,
                                                            double dt, double *__restrict__ opr) {
    const long long n = (long long)P.nx * P.ny * P.nz;
    const long long st[3] = {1, P.sy, P.sz};
    const double *Q[3] = {U, V, W};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const long long e = P.at(i, j, k);
        const int fi[3] = {i, j, k};
        double *out = opr + 7 * e;
        if (M.wall_face(C, fi[C])) {
            out[0] = rho;
#pragma unroll
            for (int q = 1; q < 7; q++) out[q] = 0.0;
            continue;
        }
        auto vs = [&](long long o) { return visc ? visc[o] : visc0; };
        double cd[6], vd[6], co[6], vo[6];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const long long sc = st[C], sd = st[d];
            if (d == C) {
                const double wn0 = 0.5, wnm = (M.walls[C] && fi[C] == 0) ? 0.0 : 0.5;  // cell f-1 a wall cell
                const double *q = Q[C];
                const double rp = pm(pm(rho, pa(pm(wn0, q[e]), pm(wn0, q[e + sc]))), 2.0);
                const double rm = pm(pm(rho, pa(pm(wnm, q[e - sc]), pm(wnm, q[e]))), 2.0);
                const double dup = M.dmi[C][fi[C]], dlo = pm(dup, -1.0);
                cd[2 * d] = pm(pm(dup, wn0), rp);
                cd[2 * d + 1] = pm(pm(dlo, wnm), rm);
                co[2 * d] = cd[2 * d];
                co[2 * d + 1] = cd[2 * d + 1];
                const double ci0 = M.di[C][fi[C] + 1], cim = M.di[C][fi[C]];
                const double fu = pm(__ddiv_rn(pm(dup, 4.0), 3.0), vs(e)), fl = pm(__ddiv_rn(pm(dlo, 4.0), 3.0), vs(e - sc));
                vd[2 * d] = pm(fu, pm(ci0, -1.0));
                vd[2 * d + 1] = pm(fl, pm(cim, 1.0));
                vo[2 * d] = pm(fu, pm(ci0, 1.0));
                vo[2 * d + 1] = pm(fl, pm(cim, -1.0));
            } else {
                const bool cw = M.wall_face(C, fi[C]);
                double am_u, az_u, gm_u, gz_u, am_l, az_l, gm_l, gz_l, bm_u, bz_u, bm_l, bz_l, g0, g1;
                M.tang(d, fi[d] + 1, cw, am_u, az_u, gm_u, gz_u);
                M.tang(d, fi[d], cw, am_l, az_l, gm_l, gz_l);
                M.tang(C, fi[C], M.wall_face(d, fi[d] + 1), bm_u, bz_u, g0, g1);
                M.tang(C, fi[C], M.wall_face(d, fi[d]), bm_l, bz_l, g0, g1);
                const double *q = Q[d];
                const double rp = pm(rho, pa(pm(bm_u, q[e - sc + sd]), pm(bz_u, q[e + sd])));
                const double rm = pm(rho, pa(pm(bm_l, q[e - sc]), pm(bz_l, q[e])));
                const double dup = M.di[d][fi[d] + 1], dlo = pm(dup, -1.0);
                cd[2 * d] = pm(pm(dup, am_u), rp);
                cd[2 * d + 1] = pm(pm(dlo, az_l), rm);
                co[2 * d] = pm(pm(dup, az_u), rp);
                co[2 * d + 1] = pm(pm(dlo, am_l), rm);
                // edge viscosities at (c-face, d-face + 1) and (c-face, d-face), lower direction first
                const int lo = C < d ? C : d, hi = C < d ? d : C;
                const long long sl = st[lo], sh = st[hi];
                double ve[2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int fd = fi[d] + (1 - u);
                    const int flo = lo == C ? fi[C] : fd, fhi = hi == C ? fi[C] : fd;
                    const long long o = e + (1 - u) * sd;
                    ve[u] = visc_edge(M.wtm[lo][flo], M.wtz[lo][flo], M.wtm[hi][fhi], M.wtz[hi][fhi], vs(o - sl - sh),
                                      vs(o - sh), vs(o - sl), vs(o));
                }
                vd[2 * d] = pm(pm(dup, ve[0]), gm_u);
                vd[2 * d + 1] = pm(pm(dlo, ve[1]), gz_l);
                vo[2 * d] = pm(pm(dup, ve[0]), gz_u);
                vo[2 * d + 1] = pm(pm(dlo, ve[1]), gm_l);
            }
        }
        double sc = cd[0], sv = vd[0];
#pragma unroll
        for (int q = 1; q < 6; q++) {
            sc = pa(sc, cd[q]);
            sv = pa(sv, vd[q]);
        }
        const double hd = pm(0.5, dt);
        out[0] = __dsub_rn(pa(rho, pm(hd, sc)), pm(hd, sv));
#pragma unroll
        for (int q = 0; q < 6; q++) out[q + 1] = __dsub_rn(pa(0.0, pm(hd, co[q])), pm(hd, vo[q]));
    }
}

// The explicit residual of a sub-iteration before an implicit solve (the
// channel example, simulation.f90:290-301): res = -2*(rho*U - rho*Uold) +
// dt*res, then, for the components in fmask, res = (res + fa) - fb where the
// face is not masked; whole padded arrays.
__global__ void __launch_bounds__(kThreads) k_mom_residual(Pad P, MomM M, double dt, double rho, CVel3 U, CVel3 Uo,
                                                           Vel3 R, int fmask, double a0, double b0, double a1,
                                                           double b1, double a2, double b2) {
    const long long ex = P.nx + 2LL * P.g, ey = P.ny + 2LL * P.g, ez = P.nz + 2LL * P.g, n = ex * ey * ez;
    const double fa[3] = {a0, a1, a2}, fb[3] = {b0, b1, b2};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % ex) - P.g;
        const long long r = t / ex;
        const int j = (int)(r % ey) - P.g, k = (int)(r / ey) - P.g;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double v = pa(pm(-2.0, __dsub_rn(pm(rho, U.a[c][t]), pm(rho, Uo.a[c][t]))), pm(dt, R.a[c][t]));
            if (((fmask >> c) & 1) && !M.masked(c, i, j, k)) v = __dsub_rn(pa(v, fa[c]), fb[c]);
            R.a[c][t] = v;
        }
    }
}

// U = 2*U - Uold + res after the implicit solve (simulation.f90:319-321)
__global__ void __launch_bounds__(kThreads) k_apply_residual(long long n, Vel3 U, CVel3 Uo, CVel3 R) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; c++) U.a[c][t] = pa(__dsub_rn(pm(2.0, U.a[c][t]), Uo.a[c][t]), R.a[c][t]);
    }
}

// Bulk velocities of the channel forcing (simulation.f90:280-298): per
// component c, sums over the unmasked interior faces of w*(2*U - Uold) and
// of w, with w = dxm(i)*dy(j)*dz(k) for U (dx*dym*dz for V, dx*dy*dzm for W);
// block partials in part[q*kRedBlocks + b], q = 2c (sum) and 2c+1 (volume).
constexpr int kBulk = 6;
__global__ void __launch_bounds__(kThreads) k_bulk(Pad P, Metrics Mp, MomM M, CVel3 U, CVel3 Uo,
                                                   double *__restrict__ part) {
    __shared__ double sh[kBulk][kThreads];
    double acc[kBulk];
#pragma unroll
    for (int q = 0; q < kBulk; q++) acc[q] = 0.0;
    const long long n = (long long)P.nx * P.ny * P.nz;
    const double *cellw[3] = {Mp.dx, Mp.dy, Mp.dz};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const long long e = P.at(i, j, k);
        const int f[3] = {i, j, k};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (M.masked(c, i, j, k)) continue;
            const double w0 = c == 0 ? M.dm[0][f[0]] : cellw[0][f[0]];
            const double w1 = c == 1 ? M.dm[1][f[1]] : cellw[1][f[1]];
            const double w2 = c == 2 ? M.dm[2][f[2]] : cellw[2][f[2]];
            const double w = pm(pm(w0, w1), w2);
            acc[2 * c] = pa(acc[2 * c], pm(w, __dsub_rn(pm(2.0, U.a[c][e]), Uo.a[c][e])));
            acc[2 * c + 1] = pa(acc[2 * c + 1], w);
        }
    }
#pragma unroll
    for (int q = 0; q < kBulk; q++) sh[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
#pragma unroll
            for (int q = 0; q < kBulk; q++) sh[q][threadIdx.x] = pa(sh[q][threadIdx.x], sh[q][threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x < kBulk) part[threadIdx.x * kRedBlocks + blockIdx.x] = sh[threadIdx.x][0];
}

__global__ void __launch_bounds__(kBulk * 32) k_bulk_final(double *__restrict__ part) {
    const int q = threadIdx.x / 32, l = threadIdx.x % 32;
    double s = 0.0;
    for (int b = l; b < kRedBlocks; b += 32) s = pa(s, part[q * kRedBlocks + b]);
    for (int o = 16; o > 0; o >>= 1) s = pa(s, __shfl_down_sync(0xffffffffu, s, o));
    if (l == 0) part[kBulk * kRedBlocks + q] = s;
}

// Flow statistics, block partials over the interior cells (fixed grid, fixed
// per-thread order): q 0-2 max|U|*dxmi (get_cfl, incomp_class.f90:1497-1540),
// 3-5 max 4*visc*dxi**2/rho, 6 sum 0.5*(Ui**2+Vi**2+Wi**2) with the
// interp_vel midpoints (incomp_class.f90:1188-1225), 7-9 sum vol*U
// (config_class.f90:196-214 with VF = 1).
constexpr int kStat = 10;

__global__ void __launch_bounds__(kThreads) k_stats(Pad P, Metrics Mp, MomM M, const double *__restrict__ U,
                                                    const double *__restrict__ V, const double *__restrict__ W,
                                                    const double *__restrict__ visc, double visc0, double rho,
                                                    double *__restrict__ part) {
    __shared__ double sh[kStat][kThreads];
    double acc[kStat];
#pragma unroll
    for (int q = 0; q < kStat; q++) acc[q] = 0.0;
    const long long n = (long long)P.nx * P.ny * P.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(P, t, i, j, k);
        const long long e = P.at(i, j, k);
        const double u = U[e], v = V[e], w = W[e];
        acc[0] = fmax(acc[0], pm(fabs(u), M.dmi[0][i]));
        acc[1] = fmax(acc[1], pm(fabs(v), M.dmi[1][j]));
        acc[2] = fmax(acc[2], pm(fabs(w), M.dmi[2][k]));
        const double vis = visc ? visc[e] : visc0;
        const double dxi = M.di[0][i + 1], dyi = M.di[1][j + 1], dzi = M.di[2][k + 1];
        acc[3] = fmax(acc[3], __ddiv_rn(pm(pm(4.0, vis), pm(dxi, dxi)), rho));
        acc[4] = fmax(acc[4], __ddiv_rn(pm(pm(4.0, vis), pm(dyi, dyi)), rho));
        acc[5] = fmax(acc[5], __ddiv_rn(pm(pm(4.0, vis), pm(dzi, dzi)), rho));
        const double ui = pa(pm(0.5, u), pm(0.5, U[e + 1]));
        const double vi = pa(pm(0.5, v), pm(0.5, V[e + P.sy]));
        const double wi = pa(pm(0.5, w), pm(0.5, W[e + P.sz]));
        acc[6] = pa(acc[6], pm(0.5, pa(pa(pm(ui, ui), pm(vi, vi)), pm(wi, wi))));
        const double vol = pm(pm(Mp.dx[i], Mp.dy[j]), Mp.dz[k]);
        acc[7] = pa(acc[7], pm(vol, u));
        acc[8] = pa(acc[8], pm(vol, v));
        acc[9] = pa(acc[9], pm(vol, w));
    }
#pragma unroll
    for (int q = 0; q < kStat; q++) sh[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
#pragma unroll
            for (int q = 0; q < kStat; q++)
                sh[q][threadIdx.x] = q < 6 ? fmax(sh[q][threadIdx.x], sh[q][threadIdx.x + h])
                                           : pa(sh[q][threadIdx.x], sh[q][threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x < kStat) part[threadIdx.x * kRedBlocks + blockIdx.x] = sh[threadIdx.x][0];
}

// final: maxima times dt, the kinetic energy, sums / fluid_vol, into
// part[kStat*kRedBlocks + q]; one warp per statistic
__global__ void __launch_bounds__(kStat * 32) k_stats_final(double *__restrict__ part, double dt, double fluid_vol) {
    const int q = threadIdx.x / 32, l = threadIdx.x % 32;
    double s = 0.0;
    for (int b = l; b < kRedBlocks; b += 32) s = q < 6 ? fmax(s, part[q * kRedBlocks + b]) : pa(s, part[q * kRedBlocks + b]);
    for (int o = 16; o > 0; o >>= 1) {
        const double x = __shfl_down_sync(0xffffffffu, s, o);
        s = q < 6 ? fmax(s, x) : pa(s, x);
    }
    if (l == 0) part[kStat * kRedBlocks + q] = q < 6 ? pm(s, dt) : (q == 6 ? s : __ddiv_rn(s, fluid_vol));
}

int check_dev(const void *a, const char *name) {
    if (!a) return pfail(BBMG_BAD_ARGS, "%s is NULL", name);
    if (!on_device(a)) return pfail(BBMG_BAD_ARGS, "%s is not a device pointer", name);
    return BBMG_OK;
}

int check_opt(const void *a, const char *name) {
    if (a && !on_device(a)) return pfail(BBMG_BAD_ARGS, "%s is not a device pointer", name);
    return BBMG_OK;
}

#define PCHK(x)                   \
    do {                          \
        int st_ = (x);            \
        if (st_ != BBMG_OK) return st_; \
    } while (0)

}  // namespace

extern "C" int nga_proj_create(const bbmg_grid *grid, const double *x, const double *y, const double *z, int device,
                               nga_proj **out) {
    if (!grid || !x || !y || !z || !out) return pfail(BBMG_BAD_ARGS, "null argument");
    *out = nullptr;
    const bbmg_grid g = *grid;
    if (g.nx < 1 || g.ny < 1 || g.nz < 1) return pfail(BBMG_BAD_ARGS, "grid sizes must be >= 1");
    if (g.ghost < 1) return pfail(BBMG_BAD_ARGS, "the projection steps need ghost >= 1 (got %d)", g.ghost);
    const double *xs[3] = {x, y, z};
    const int ns[3] = {g.nx, g.ny, g.nz}, pers[3] = {g.xper, g.yper, g.zper};
    for (int a = 0; a < 3; a++)
        for (int i = 0; i < ns[a]; i++)
            if (!(xs[a][i + 1] > xs[a][i])) return pfail(BBMG_BAD_ARGS, "nodes of direction %d must increase", a);
    if (device < 0) PCU(cudaGetDevice(&device));
    PCU(cudaSetDevice(device));
    nga_proj *p = new nga_proj;
    p->g = g;
    p->device = device;
    std::vector<double> host;
    size_t off[3][5];
    for (int a = 0; a < 3; a++) {
        std::vector<double> dp0, dp1, du0, du1, d;
        axis_metrics(xs[a], ns[a], pers[a] != 0, dp0, dp1, du0, du1, d);
        const std::vector<double> *parts[5] = {&dp0, &dp1, &du0, &du1, &d};
        for (int q = 0; q < 5; q++) {
            off[a][q] = host.size();
            host.insert(host.end(), parts[q]->begin(), parts[q]->end());
        }
    }
    cudaError_t e = cudaMalloc((void **)&p->metrics, host.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void **)&p->part, (kStat * kRedBlocks + kStat) * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(p->metrics, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaGetLastError();
        nga_proj_destroy(p);
        return pfail(e == cudaErrorMemoryAllocation ? BBMG_NO_MEMORY : BBMG_CUDA, "projection setup: %s",
                     cudaGetErrorString(e));
    }
    for (int a = 0; a < 3; a++) {
        p->dp0[a] = p->metrics + off[a][0];
        p->dp1[a] = p->metrics + off[a][1];
        p->du0[a] = p->metrics + off[a][2];
        p->du1[a] = p->metrics + off[a][3];
        p->d[a] = p->metrics + off[a][4];
    }
    {
        std::vector<double> mh;
        size_t mo[3][kMomQ];
        const int per[3] = {g.xper, g.yper, g.zper};
        for (int a = 0; a < 3; a++) {
            std::vector<double> m[kMomQ];
            momentum_metrics(xs[a], ns[a], !per[a], m);
            for (int q = 0; q < kMomQ; q++) {
                mo[a][q] = mh.size();
                mh.insert(mh.end(), m[q].begin(), m[q].end());
            }
        }
        cudaError_t e2 = cudaMalloc((void **)&p->mmetrics, mh.size() * sizeof(double));
        if (e2 == cudaSuccess) e2 = cudaMemcpy(p->mmetrics, mh.data(), mh.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e2 != cudaSuccess) {
            cudaGetLastError();
            nga_proj_destroy(p);
            return pfail(e2 == cudaErrorMemoryAllocation ? BBMG_NO_MEMORY : BBMG_CUDA, "momentum metrics: %s",
                         cudaGetErrorString(e2));
        }
        for (int a = 0; a < 3; a++)
            for (int q = 0; q < kMomQ; q++) p->mom[a][q] = p->mmetrics + mo[a][q];
    }
    // fluid_vol = vol_total = xL*yL*zL (sgrid_class.f90:260-263; config_class.f90:129)
    const double xL = x[g.nx] - x[0], yL = y[g.ny] - y[0], zL = z[g.nz] - z[0];
    p->vol_total = xL * yL * zL;
    *out = p;
    return BBMG_OK;
}

extern "C" int nga_proj_destroy(nga_proj *p) {
    if (!p) return BBMG_OK;
    cudaSetDevice(p->device);
    if (p->metrics) cudaFree(p->metrics);
    if (p->part) cudaFree(p->part);
    if (p->mmetrics) cudaFree(p->mmetrics);
    delete p;
    return BBMG_OK;
}

extern "C" int nga_proj_set_stream(nga_proj *p, void *stream) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    p->stream = (cudaStream_t)stream;
    return BBMG_OK;
}

extern "C" int nga_proj_laplacian(nga_proj *p, const double *rho_U, const double *rho_V, const double *rho_W,
                                  double *opr) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(opr, "opr"));
    PCHK(check_opt(rho_U, "rho_U"));
    PCHK(check_opt(rho_V, "rho_V"));
    PCHK(check_opt(rho_W, "rho_W"));
    PCU(cudaSetDevice(p->device));
    const Pad P = pad_of(p->g);
    const long long n = (long long)P.nx * P.ny * P.nz;
    k_laplacian<<<grid_cells(n), kThreads, 0, p->stream>>>(P, metrics_of(p), rho_U, rho_V, rho_W, opr);
    PCU(cudaGetLastError());
    return BBMG_OK;
}

extern "C" int nga_proj_divergence(nga_proj *p, const double *U, const double *V, const double *W, double rho,
                                   double dt, double *div, double *rhs) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_opt(div, "div"));
    PCHK(check_opt(rhs, "rhs"));
    if (!div && !rhs) return pfail(BBMG_BAD_ARGS, "div and rhs are both NULL");
    if (rhs && !(dt != 0.0)) return pfail(BBMG_BAD_ARGS, "dt must be nonzero");
    PCU(cudaSetDevice(p->device));
    const Pad P = pad_of(p->g);
    const long long n = (long long)P.nx * P.ny * P.nz;
    k_divergence<<<grid_cells(n), kThreads, 0, p->stream>>>(P, metrics_of(p), U, V, W, rho, dt, div, rhs);
    PCU(cudaGetLastError());
    // div is synchronised like get_div's cfg%sync; rhs is the solver's input,
    // which reads the interior only
    return sync_arrays(p, div, nullptr, nullptr, nullptr);
}

extern "C" int nga_proj_shift_p(nga_proj *p, double *pressure, double *mean) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(pressure, "pressure"));
    PCU(cudaSetDevice(p->device));
    const Pad P = pad_of(p->g);
    const long long n = (long long)P.nx * P.ny * P.nz;
    k_vol_sum<<<kRedBlocks, kThreads, 0, p->stream>>>(P, metrics_of(p), pressure, p->part);
    PCU(cudaGetLastError());
    k_vol_mean<<<1, kThreads, 0, p->stream>>>(p->part, p->vol_total);
    PCU(cudaGetLastError());
    k_shift<<<grid_cells(n), kThreads, 0, p->stream>>>(P, p->part + kRedBlocks, pressure);
    PCU(cudaGetLastError());
    PCHK(sync_arrays(p, pressure, nullptr, nullptr, nullptr));
    if (mean) {
        PCU(cudaMemcpyAsync(mean, p->part + kRedBlocks, sizeof(double), cudaMemcpyDefault, p->stream));
        PCU(cudaStreamSynchronize(p->stream));
    }
    return BBMG_OK;
}

extern "C" int nga_proj_pgrad(nga_proj *p, const double *P_, double *gx, double *gy, double *gz) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(P_, "P"));
    PCHK(check_dev(gx, "Pgradx"));
    PCHK(check_dev(gy, "Pgrady"));
    PCHK(check_dev(gz, "Pgradz"));
    PCU(cudaSetDevice(p->device));
    const Pad P = pad_of(p->g);
    const long long n = (long long)P.nx * P.ny * P.nz;
    k_pgrad<<<grid_cells(n), kThreads, 0, p->stream>>>(P, metrics_of(p), P_, gx, gy, gz);
    PCU(cudaGetLastError());
    return sync_arrays(p, gx, gy, gz, nullptr);
}

extern "C" int nga_proj_correct(nga_proj *p, const double *sol, double dt, const double *rho_U, const double *rho_V,
                                const double *rho_W, double *pres, double *U, double *V, double *W) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(sol, "sol"));
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_opt(rho_U, "rho_U"));
    PCHK(check_opt(rho_V, "rho_V"));
    PCHK(check_opt(rho_W, "rho_W"));
    PCHK(check_opt(pres, "P"));
    PCU(cudaSetDevice(p->device));
    const Pad P = pad_of(p->g);
    const long long n = (long long)P.nx * P.ny * P.nz;
    k_correct<<<grid_cells(n), kThreads, 0, p->stream>>>(P, metrics_of(p), sol, dt, rho_U, rho_V, rho_W, pres, U, V,
                                                         W);
    PCU(cudaGetLastError());
    return sync_arrays(p, U, V, W, pres);
}

namespace {
MomM momentum_of(const nga_proj *p) {
    MomM M;
    const int per[3] = {p->g.xper, p->g.yper, p->g.zper}, nn[3] = {p->g.nx, p->g.ny, p->g.nz};
    for (int a = 0; a < 3; a++) {
        M.di[a] = p->mom[a][0];
        M.dmi[a] = p->mom[a][1];
        M.itm[a] = p->mom[a][2];
        M.itz[a] = p->mom[a][3];
        M.vtm[a] = p->mom[a][4];
        M.vtz[a] = p->mom[a][5];
        M.gdm[a] = p->mom[a][6];
        M.wtm[a] = p->mom[a][7];
        M.wtz[a] = p->mom[a][8];
        M.dm[a] = p->mom[a][9];
        M.nf[a] = nn[a];
        M.walls[a] = per[a] ? 0 : 1;
    }
    return M;
}
}  // namespace

extern "C" int nga_proj_dmomdt(nga_proj *p, const double *U, const double *V, const double *W, const double *P_,
                               double rho, const double *visc, double visc0, double *dU, double *dV, double *dW) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_dev(P_, "P"));
    PCHK(check_opt(visc, "visc"));
    PCHK(check_dev(dU, "drhoUdt"));
    PCHK(check_dev(dV, "drhoVdt"));
    PCHK(check_dev(dW, "drhoWdt"));
    PCU(cudaSetDevice(p->device));
    const Pad P = pad_of(p->g);
    const long long n = (long long)P.nx * P.ny * P.nz;
    k_dmomdt<<<grid_cells(n), kThreads, 0, p->stream>>>(P, momentum_of(p), U, V, W, P_, rho, visc, visc0, dU, dV,
                                                         dW);
    PCU(cudaGetLastError());
    return sync_arrays(p, dU, dV, dW, nullptr);
}

namespace {
long long padded_size(const bbmg_grid &g) {
    return (g.nx + 2LL * g.ghost) * (g.ny + 2LL * g.ghost) * (g.nz + 2LL * g.ghost);
}
}  // namespace

extern "C" int nga_proj_midpoint(nga_proj *p, double *U, double *V, double *W, const double *Uold,
                                 const double *Vold, const double *Wold) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_dev(Uold, "Uold"));
    PCHK(check_dev(Vold, "Vold"));
    PCHK(check_dev(Wold, "Wold"));
    PCU(cudaSetDevice(p->device));
    const long long n = padded_size(p->g);
    k_midpoint<<<grid_cells(n), kThreads, 0, p->stream>>>(n, Vel3{{U, V, W}}, CVel3{{Uold, Vold, Wold}});
    PCU(cudaGetLastError());
    return BBMG_OK;
}

extern "C" int nga_proj_advance(nga_proj *p, double dt, double rho, double *U, double *V, double *W,
                                const double *Uold, const double *Vold, const double *Wold, const double *drhoUdt,
                                const double *drhoVdt, const double *drhoWdt, double force_a, double force_b,
                                const double *mean) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_dev(Uold, "Uold"));
    PCHK(check_dev(Vold, "Vold"));
    PCHK(check_dev(Wold, "Wold"));
    PCHK(check_dev(drhoUdt, "drhoUdt"));
    PCHK(check_dev(drhoVdt, "drhoVdt"));
    PCHK(check_dev(drhoWdt, "drhoWdt"));
    if (!(rho != 0.0)) return pfail(BBMG_BAD_ARGS, "rho must be non-zero");
    if (force_a != 0.0 && (!mean || !(force_b != 0.0)))
        return pfail(BBMG_BAD_ARGS, "forcing needs the mean velocity and a non-zero force_b");
    PCU(cudaSetDevice(p->device));
    const long long n = padded_size(p->g);
    const double m0 = force_a != 0.0 ? mean[0] : 0.0, m1 = force_a != 0.0 ? mean[1] : 0.0,
                 m2 = force_a != 0.0 ? mean[2] : 0.0;
    k_advance<<<grid_cells(n), kThreads, 0, p->stream>>>(n, dt, rho, Vel3{{U, V, W}}, CVel3{{Uold, Vold, Wold}},
                                                         CVel3{{drhoUdt, drhoVdt, drhoWdt}}, force_a, force_b, m0, m1,
                                                         m2);
    PCU(cudaGetLastError());
    return BBMG_OK;
}

extern "C" int nga_proj_flow_stats(nga_proj *p, const double *U, const double *V, const double *W,
                                   const double *visc, double visc0, double rho, double dt, double *out) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    if (!out) return pfail(BBMG_BAD_ARGS, "out is NULL");
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_opt(visc, "visc"));
    if (!(rho != 0.0)) return pfail(BBMG_BAD_ARGS, "rho must be non-zero");
    PCU(cudaSetDevice(p->device));
    const Pad P = pad_of(p->g);
    k_stats<<<kRedBlocks, kThreads, 0, p->stream>>>(P, metrics_of(p), momentum_of(p), U, V, W, visc, visc0, rho,
                                                    p->part);
    PCU(cudaGetLastError());
    k_stats_final<<<1, kStat * 32, 0, p->stream>>>(p->part, dt, p->vol_total);
    PCU(cudaGetLastError());
    PCU(cudaMemcpyAsync(out, p->part + kStat * kRedBlocks, kStat * sizeof(double), cudaMemcpyDefault, p->stream));
    PCU(cudaStreamSynchronize(p->stream));
    return BBMG_OK;
}

extern "C" int nga_proj_implicit_operator(nga_proj *p, int comp, double dt, double rho, const double *U,
                                          const double *V, const double *W, const double *visc, double visc0,
                                          double *opr) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    if (comp < 0 || comp > 2) return pfail(BBMG_BAD_ARGS, "comp must be 0 (U), 1 (V) or 2 (W), got %d", comp);
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_opt(visc, "visc"));
    PCHK(check_dev(opr, "opr"));
    PCU(cudaSetDevice(p->device));
    const Pad P = pad_of(p->g);
    const long long n = (long long)P.nx * P.ny * P.nz;
    const MomM M = momentum_of(p);
    if (comp == 0)
        k_implicit_opr<0><<<grid_cells(n), kThreads, 0, p->stream>>>(P, M, U, V, W, visc, visc0, rho, dt, opr);
    else if (comp == 1)
        k_implicit_opr<1><<<grid_cells(n), kThreads, 0, p->stream>>>(P, M, U, V, W, visc, visc0, rho, dt, opr);
    else
        k_implicit_opr<2><<<grid_cells(n), kThreads, 0, p->stream>>>(P, M, U, V, W, visc, visc0, rho, dt, opr);
    PCU(cudaGetLastError());
    return BBMG_OK;
}

extern "C" int nga_proj_mom_residual(nga_proj *p, double dt, double rho, const double *U, const double *V,
                                     const double *W, const double *Uold, const double *Vold, const double *Wold,
                                     double *resU, double *resV, double *resW, int force_mask, const double *force) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_dev(Uold, "Uold"));
    PCHK(check_dev(Vold, "Vold"));
    PCHK(check_dev(Wold, "Wold"));
    PCHK(check_dev(resU, "resU"));
    PCHK(check_dev(resV, "resV"));
    PCHK(check_dev(resW, "resW"));
    if (force_mask & ~7) return pfail(BBMG_BAD_ARGS, "force_mask holds bits 1 (U), 2 (V), 4 (W) only");
    if (force_mask && !force) return pfail(BBMG_BAD_ARGS, "force is NULL");
    PCU(cudaSetDevice(p->device));
    double f[6] = {0, 0, 0, 0, 0, 0};
    if (force_mask)
        for (int q = 0; q < 6; q++) f[q] = force[q];
    const long long n = padded_size(p->g);
    k_mom_residual<<<grid_cells(n), kThreads, 0, p->stream>>>(pad_of(p->g), momentum_of(p), dt, rho,
                                                              CVel3{{U, V, W}}, CVel3{{Uold, Vold, Wold}},
                                                              Vel3{{resU, resV, resW}}, force_mask, f[0], f[1], f[2],
                                                              f[3], f[4], f[5]);
    PCU(cudaGetLastError());
    return BBMG_OK;
}

extern "C" int nga_proj_apply_residual(nga_proj *p, double *U, double *V, double *W, const double *Uold,
                                       const double *Vold, const double *Wold, const double *resU,
                                       const double *resV, const double *resW) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_dev(Uold, "Uold"));
    PCHK(check_dev(Vold, "Vold"));
    PCHK(check_dev(Wold, "Wold"));
    PCHK(check_dev(resU, "resU"));
    PCHK(check_dev(resV, "resV"));
    PCHK(check_dev(resW, "resW"));
    PCU(cudaSetDevice(p->device));
    const long long n = padded_size(p->g);
    k_apply_residual<<<grid_cells(n), kThreads, 0, p->stream>>>(n, Vel3{{U, V, W}}, CVel3{{Uold, Vold, Wold}},
                                                                CVel3{{resU, resV, resW}});
    PCU(cudaGetLastError());
    return BBMG_OK;
}

extern "C" int nga_proj_bulk(nga_proj *p, const double *U, const double *V, const double *W, const double *Uold,
                             const double *Vold, const double *Wold, double *out) {
    if (!p) return pfail(BBMG_BAD_ARGS, "null projection handle");
    if (!out) return pfail(BBMG_BAD_ARGS, "out is NULL");
    PCHK(check_dev(U, "U"));
    PCHK(check_dev(V, "V"));
    PCHK(check_dev(W, "W"));
    PCHK(check_dev(Uold, "Uold"));
    PCHK(check_dev(Vold, "Vold"));
    PCHK(check_dev(Wold, "Wold"));
    PCU(cudaSetDevice(p->device));
    k_bulk<<<kRedBlocks, kThreads, 0, p->stream>>>(pad_of(p->g), metrics_of(p), momentum_of(p), CVel3{{U, V, W}},
                                                   CVel3{{Uold, Vold, Wold}}, p->part);
    PCU(cudaGetLastError());
    k_bulk_final<<<1, kBulk * 32, 0, p->stream>>>(p->part);
    PCU(cudaGetLastError());
    PCU(cudaMemcpyAsync(out, p->part + kBulk * kRedBlocks, kBulk * sizeof(double), cudaMemcpyDefault, p->stream));
    PCU(cudaStreamSynchronize(p->stream));
    return BBMG_OK;
}

