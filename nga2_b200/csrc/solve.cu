// solve.cu -- V-cycle kernels of the black-box multigrid (FP64 and FP32).
//
// Each kernel restates one solve-phase routine of src/solver/bbmg_class.f90.
// The FP64 instantiation (EXACT) evaluates every sum in the reference's
// column-major term order without FMA contraction, so it matches the oracle
// bit for bit; the FP32 instantiation is the fast V-cycle of the mixed
// precision solver and uses FMA.  Terms whose coefficient is structurally
// zero (the 20 unused slots of a 7-point operator, prolongation weights of the
// other parity classes) are skipped: adding +0.0 does not change a sum.
#include "setup.cuh"

namespace bbmg {

struct Off27 {
    int o[27];
};

static Off27 off_for(const NbrOff &nb, int par) {
    Off27 r;
    for (int q = 0; q < 27; q++) r.o[q] = nb.off[par][q];
    return r;
}


// Programmatic dependent launch: every solve-phase kernel lets the next kernel
// in the stream start launching as soon as all of its own blocks are running,
// then waits for its predecessor to finish (and its writes to be visible)
// before touching memory.  Semantics stay those of plain stream order; only
// the launch latency overlaps the previous kernel's tail.
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... KArgs, typename... Args>
static cudaError_t launch_k(void (*kern)(KArgs...), int grid, int block, size_t shm, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = shm;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

template <typename T, bool EXACT> struct Ops;
template <> struct Ops<double, true> {
    __device__ static __forceinline__ double mac(double s, double a, double b) { return __dadd_rn(s, __dmul_rn(a, b)); }
    __device__ static __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ static __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    __device__ static __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};
template <typename T> struct Ops<T, false> {
    __device__ static __forceinline__ T mac(T s, T a, T b) { return fma(a, b, s); }
    __device__ static __forceinline__ T add(T a, T b) { return a + b; }
    __device__ static __forceinline__ T sub(T a, T b) { return a - b; }
    __device__ static __forceinline__ T div(T a, T b) { return a / b; }
};
template <typename T> struct ExactOf { static constexpr bool value = sizeof(T) == 8; };

// ---------------------------------------------------------------------------
// One colour of the 8-colour Gauss-Seidel (bbmg_class.f90:872-885):
// A = (B - sum_{l != 0} opr(l) A(nbr)) / (opr(0) + eps) on the points
// i = px + 2a, j = py + 2b, k = pz + 2c.  With `fuse` the new value is also
// written into its periodic images (the vsync after the colour); that is only
// race-free when every periodic direction has an even size, otherwise the
// caller runs the overlap copy as a separate pass.
template <typename T, int NPT>
__global__ void __launch_bounds__(256) k_relax(Lay L, Off27 off, const T *__restrict__ opr, T *v,
                                                const T *__restrict__ f, int px, int py, int pz, int fuse) {
    pdl_entry();
    using O = Ops<T, ExactOf<T>::value>;
    const int na = (L.nx - px + 1) >> 1, nb = (L.ny - py + 1) >> 1, nc = (L.nz - pz + 1) >> 1;
    const long long total = (long long)na * nb * nc;
    for (long long t = gtid(); t < total; t += gstride()) {
        int a = (int)(t % na);
        long long rr = t / na;
        int b = (int)(rr % nb), c = (int)(rr / nb);
        int i = px + 2 * a, j = py + 2 * b, k = pz + 2 * c;
        long long id = L.idx(i, j, k);
        T s = T(0);
#pragma unroll
        for (int q = 0; q < Lay7<NPT>::terms; q++) {
            if (q == Lay7<NPT>::centre) continue;
            const int o = off.o[Lay7<NPT>::slot(q)];
            s = O::mac(s, opr[Lay7<NPT>::plane(q) * L.plane + id + (Lay7<NPT>::at_nbr(q) ? o : 0)], v[id + o]);
        }
        T d = opr[Lay7<NPT>::plane(Lay7<NPT>::centre) * L.plane + id];
        T val = O::div(O::sub(f[id], s), O::add(d, T(kEps)));
        v[id] = val;
        if (fuse && on_periodic_face(L, i, j, k)) write_images(L, v, i, j, k, val);
    }
}

// Residual r = f - sum_l opr(l) v(nbr) on the interior, periodic images
// written (bbmg_class.f90:831-844).  With f == nullptr the kernel returns the
// operator product itself (the PCG's Ap, bbmg_class.f90:676-683).
template <typename T, int NPT>
__global__ void __launch_bounds__(256) k_residual(Lay L, NbrOff nb, const T *__restrict__ opr,
                                                   const T *__restrict__ v, const T *__restrict__ f,
                                                   T *__restrict__ r) {
    pdl_entry();
    using O = Ops<T, ExactOf<T>::value>;
    const long long total = (long long)L.nx * L.ny * L.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        const int par = i & 1;
        long long id = L.idx(i, j, k);
        T s = T(0);
#pragma unroll
        for (int q = 0; q < Lay7<NPT>::terms; q++) {
            const int q27i = Lay7<NPT>::slot(q);
            const int o = par ? nb.off[1][q27i] : nb.off[0][q27i];
            s = O::mac(s, opr[Lay7<NPT>::plane(q) * L.plane + id + (Lay7<NPT>::at_nbr(q) ? o : 0)], v[id + o]);
        }
        T val = f ? O::sub(f[id], s) : s;
        r[id] = val;
        if (on_periodic_face(L, i, j, k)) write_images(L, r, i, j, k, val);
    }
}

// Restriction f_c = sum_r f2c(r) r_f(2c + r) (bbmg_class.f90:805-827), with
// f2c(r) = c2f((1-r)/2, 2c+r) (bbmg_class.f90:1218-1222) read straight from the
// fine prolongation weights.  Also zeroes the coarse correction v_c, the first
// statement of cycle(n+1) (bbmg_class.f90:739).
template <typename T>
__global__ void __launch_bounds__(256) k_restrict(Lay F, Lay C, const T *__restrict__ c2f,
                                                   const T *__restrict__ rF, T *__restrict__ fC,
                                                   T *__restrict__ vC) {
    pdl_entry();
    using O = Ops<T, ExactOf<T>::value>;
    const long long total = (long long)C.nx * C.ny * C.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int ci, cj, ck;
        interior_cell(C, t, ci, cj, ck);
        int fi = 2 * ci, fj = 2 * cj, fk = 2 * ck;
        int rk0 = -pmod(F.zper, fk - 1, F.nz), rk1 = pmod(F.zper, fk + 1, F.nz);
        int rj0 = -pmod(F.yper, fj - 1, F.ny), rj1 = pmod(F.yper, fj + 1, F.ny);
        int ri0 = -pmod(F.xper, fi - 1, F.nx), ri1 = pmod(F.xper, fi + 1, F.nx);
        T s = T(0);
        for (int rk = rk0; rk <= rk1; rk++)
            for (int rj = rj0; rj <= rj1; rj++)
                for (int ri = ri0; ri <= ri1; ri++) {
                    long long fid = F.idx(fi + ri, fj + rj, fk + rk);
                    s = O::mac(s, c2f[q8((1 - ri) / 2, (1 - rj) / 2, (1 - rk) / 2) * F.plane + fid], rF[fid]);
                }
        long long cid = C.idx(ci, cj, ck);
        fC[cid] = s;
        vC[cid] = T(0);
        if (on_periodic_face(C, ci, cj, ck)) {
            write_images(C, fC, ci, cj, ck, s);
            write_images(C, vC, ci, cj, ck, T(0));
        }
    }
}

// Prolongation and correction v_f += sum_p c2f(p) v_c((i+1)/2 + p)
// (bbmg_class.f90:779-801 then 770).  A fine point of parity class
// (n1,n2,n3) only carries weights p_d <= n_d.
template <typename T>
__global__ void __launch_bounds__(256) k_prolong(Lay F, Lay C, const T *__restrict__ c2f,
                                                  const T *__restrict__ vC, T *__restrict__ vF) {
    pdl_entry();
    using O = Ops<T, ExactOf<T>::value>;
    const long long total = (long long)F.nx * F.ny * F.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(F, t, i, j, k);
        const int n1 = i & 1, n2 = j & 1, n3 = k & 1;
        const int ci = i >> 1, cj = j >> 1, ck = k >> 1;
        long long id = F.idx(i, j, k);
        T e = T(0);
        for (int pk = 0; pk <= n3; pk++)
            for (int pj = 0; pj <= n2; pj++)
                for (int pi = 0; pi <= n1; pi++)
                    e = O::mac(e, c2f[q8(pi, pj, pk) * F.plane + id], vC[C.idx(ci + pi, cj + pj, ck + pk)]);
        T val = O::add(vF[id], e);
        vF[id] = val;
        if (on_periodic_face(F, i, j, k)) write_images(F, vF, i, j, k, val);
    }
}

// Coarsest level: gather f in lexicographic order, solve with the stored LU
// (FP64 always), scatter into v (bbmg_class.f90:891-927).  One block; the
// triangular solves run on one warp with the factors in shared memory when
// they fit.
template <typename T>
__global__ void k_coarse_solve(Lay L, const double *__restrict__ LU, const int *__restrict__ piv,
                               const int *__restrict__ pinned, const T *__restrict__ f, T *__restrict__ v,
                               int mat_in_smem) {
    pdl_entry();
    extern __shared__ double sm[];
    const int np = L.nx * L.ny * L.nz;
    double *x = sm;
    const double *A = mat_in_smem ? sm + np : LU;
    for (int ind = threadIdx.x; ind < np; ind += blockDim.x) {
        int i = ind % L.nx, j = (ind / L.nx) % L.ny, k = ind / (L.nx * L.ny);
        x[ind] = (double)f[L.idx(i, j, k)];
    }
    if (mat_in_smem)
        for (long long e = threadIdx.x; e < (long long)np * np; e += blockDim.x) sm[np + e] = LU[e];
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        if (lane == 0)
            for (int j = 0; j < np; j++) {
                int p = piv[j];
                if (p != j) { double t = x[j]; x[j] = x[p]; x[p] = t; }
            }
        __syncwarp();
        for (int kk = 0; kk < np; kk++) {
            double xk = x[kk];
            if (xk != 0.0)
                for (int i = kk + 1 + lane; i < np; i += 32)
                    x[i] = __dsub_rn(x[i], __dmul_rn(xk, A[(long long)kk * np + i]));
            __syncwarp();
        }
        for (int kk = np - 1; kk >= 0; kk--) {
            if (pinned[kk]) {
                if (lane == 0) x[kk] = 0.0;
                __syncwarp();
                continue;
            }
            double xk = x[kk];
            if (xk != 0.0) {
                xk = __ddiv_rn(xk, A[(long long)kk * np + kk]);
                __syncwarp();
                if (lane == 0) x[kk] = xk;
                for (int i = lane; i < kk; i += 32)
                    x[i] = __dsub_rn(x[i], __dmul_rn(xk, A[(long long)kk * np + i]));
            }
            __syncwarp();
        }
    }
    __syncthreads();
    for (int ind = threadIdx.x; ind < np; ind += blockDim.x) {
        int i = ind % L.nx, j = (ind / L.nx) % L.ny, k = ind / (L.nx * L.ny);
        T val = (T)x[ind];
        v[L.idx(i, j, k)] = val;
        if (on_periodic_face(L, i, j, k)) write_images(L, v, i, j, k, val);
    }
}

// ---------------------------------------------------------------------------
// Deterministic reductions: a fixed grid of kRedBlocks blocks, fixed tree.
template <int MODE>  // 0 = max with NaN propagation, 1 = sum
__device__ __forceinline__ double block_reduce(double v, double *sh) {
    const int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s) {
            double a = sh[tid], b = sh[tid + s];
            if (MODE == 0) sh[tid] = (a != a || b != b) ? (a + b) : fmax(a, b);
            else sh[tid] = a + b;
        }
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

template <typename T>
__global__ void __launch_bounds__(256) k_maxabs_part(Lay L, const T *__restrict__ x, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    const long long total = (long long)L.nx * L.ny * L.nz;
    double m = 0.0;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        double a = fabs((double)x[L.idx(i, j, k)]);
        m = (a != a || m != m) ? (a + m) : fmax(m, a);
    }
    m = block_reduce<0>(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

template <typename TA, typename TB>
__global__ void __launch_bounds__(256) k_dot_part(Lay L, const TA *__restrict__ a, const TB *__restrict__ b,
                                                   double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    const long long total = (long long)L.nx * L.ny * L.nz;
    double s = 0.0;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        long long id = L.idx(i, j, k);
        s = __dadd_rn(s, __dmul_rn((double)a[id], (double)b[id]));
    }
    s = block_reduce<1>(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_final(const double *__restrict__ part, int n, double *__restrict__ out) {
    pdl_entry();
    __shared__ double sh[256];
    double v = MODE == 0 ? 0.0 : 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        double a = part[t];
        if (MODE == 0) v = (a != a || v != v) ? (a + v) : fmax(v, a);
        else v = v + a;
    }
    v = block_reduce<MODE>(v, sh);
    if (threadIdx.x == 0) *out = v;
}

// ---------------------------------------------------------------------------
// caller arrays (Fortran, g overlap layers) <-> level interior
template <typename T>
__global__ void __launch_bounds__(256) k_from_caller(Lay L, const double *__restrict__ src, int g, T *__restrict__ dst) {
    pdl_entry();
    const long long total = (long long)L.nx * L.ny * L.nz;
    const long long sy = L.nx + 2 * g, sz = sy * (L.ny + 2 * g);
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        T val = (T)src[(k + g) * sz + (j + g) * sy + (i + g)];
        dst[L.idx(i, j, k)] = val;
        if (on_periodic_face(L, i, j, k)) write_images(L, dst, i, j, k, val);
    }
}

__global__ void __launch_bounds__(256) k_to_caller(Lay L, const double *__restrict__ src, int g, double *__restrict__ dst) {
    pdl_entry();
    const long long total = (long long)L.nx * L.ny * L.nz;
    const long long sy = L.nx + 2 * g, sz = sy * (L.ny + 2 * g);
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        dst[(k + g) * sz + (j + g) * sy + (i + g)] = src[L.idx(i, j, k)];
    }
}

__global__ void __launch_bounds__(256) k_to_f32(const double *__restrict__ src, float *__restrict__ dst, long long n) {
    pdl_entry();
    for (long long t = gtid(); t < n; t += gstride()) dst[t] = (float)src[t];
}

// ---------------------------------------------------------------------------
// launchers
#define BB_CHECK_LAUNCH() do { cudaError_t e_ = cudaGetLastError(); if (e_ != cudaSuccess) return e_; } while (0)

template <typename T>
cudaError_t launch_relax(const Lay &L, const NbrOff &nb, int npt, bool fuse, const T *opr, T *v, const T *f, int dir,
                         cudaStream_t s) {
    const bool per = L.xper || L.yper || L.zper;
    for (int c = 0; c < 8; c++) {
        int col = dir > 0 ? c : 7 - c;  // colours 1..8 forward, 8..1 backward
        int px = col & 1, py = (col >> 1) & 1, pz = (col >> 2) & 1;
        long long n = (long long)((L.nx - px + 1) >> 1) * ((L.ny - py + 1) >> 1) * ((L.nz - pz + 1) >> 1);
        if (n == 0) continue;
        Off27 off = off_for(nb, px);
        int g = grid_for(n, 256);
        if (npt == 4) launch_k(k_relax<T, 4>, g, 256, 0, s, L, off, opr, v, f, px, py, pz, fuse ? 1 : 0);
        else if (npt == 7) launch_k(k_relax<T, 7>, g, 256, 0, s, L, off, opr, v, f, px, py, pz, fuse ? 1 : 0);
        else launch_k(k_relax<T, 27>, g, 256, 0, s, L, off, opr, v, f, px, py, pz, fuse ? 1 : 0);
        BB_CHECK_LAUNCH();
        if (per && !fuse) {
            cudaError_t e = wrap_planes(L, v, 1, s);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_residual(const Lay &L, const NbrOff &nb, int npt, const T *opr, const T *v, const T *f, T *r,
                            cudaStream_t s) {
    long long n = (long long)L.nx * L.ny * L.nz;
    int g = grid_for(n, 256);
    if (npt == 4) launch_k(k_residual<T, 4>, g, 256, 0, s, L, nb, opr, v, f, r);
    else if (npt == 7) launch_k(k_residual<T, 7>, g, 256, 0, s, L, nb, opr, v, f, r);
    else launch_k(k_residual<T, 27>, g, 256, 0, s, L, nb, opr, v, f, r);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_restrict(const Lay &F, const Lay &C, const T *c2f, const T *rF, T *fC, T *vC, cudaStream_t s) {
    long long n = (long long)C.nx * C.ny * C.nz;
    launch_k(k_restrict<T>, grid_for(n, 256), 256, 0, s, F, C, c2f, rF, fC, vC);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_prolong(const Lay &F, const Lay &C, const T *c2f, const T *vC, T *vF, cudaStream_t s) {
    long long n = (long long)F.nx * F.ny * F.nz;
    launch_k(k_prolong<T>, grid_for(n, 256), 256, 0, s, F, C, c2f, vC, vF);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_coarse_solve(const Lay &L, const double *LU, const int *piv, const int *pinned, const T *f, T *v,
                                cudaStream_t s) {
    int np = L.nx * L.ny * L.nz;
    size_t mat = (size_t)np * np * sizeof(double), vec = (size_t)np * sizeof(double);
    int in_smem = (mat + vec) <= kCoarseSmem;
    size_t shm = vec + (in_smem ? mat : 0);
    launch_k(k_coarse_solve<T>, 1, 256, shm, s, L, LU, piv, pinned, f, v, in_smem);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}

cudaError_t coarse_solve_prepare() {
    cudaError_t e = cudaFuncSetAttribute(k_coarse_solve<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_coarse_solve<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmem);
}

template <typename T>
cudaError_t launch_maxabs(const Lay &L, const T *x, double *part, double *out, cudaStream_t s) {
    launch_k(k_maxabs_part<T>, kRedBlocks, 256, 0, s, L, x, part);
    BB_CHECK_LAUNCH();
    launch_k(k_final<0>, 1, 256, 0, s, part, kRedBlocks, out);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_dot(const Lay &L, const T *a, const T *b, double *part, double *out, cudaStream_t s) {
    launch_k(k_dot_part<T, T>, kRedBlocks, 256, 0, s, L, a, b, part);
    BB_CHECK_LAUNCH();
    launch_k(k_final<1>, 1, 256, 0, s, part, kRedBlocks, out);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_from_caller(const Lay &L, const double *src, int g, T *dst, cudaStream_t s) {
    long long n = (long long)L.nx * L.ny * L.nz;
    launch_k(k_from_caller<T>, grid_for(n, 256), 256, 0, s, L, src, g, dst);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}

cudaError_t launch_to_caller(const Lay &L, const double *src, int g, double *dst, cudaStream_t s) {
    long long n = (long long)L.nx * L.ny * L.nz;
    launch_k(k_to_caller, grid_for(n, 256), 256, 0, s, L, src, g, dst);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}

cudaError_t launch_to_f32(const double *src, float *dst, long long n, cudaStream_t s) {
    launch_k(k_to_f32, grid_for(n, 256), 256, 0, s, src, dst, n);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}


// ---------------------------------------------------------------------------
// PCG (bbmg_class.f90:643-703).  Scalars live on the device so an iteration
// needs no host round trip; only the convergence norm is copied back.
__global__ void k_cg_rho(const double *__restrict__ part, int n, CgScal *sc) {
    pdl_entry();
    __shared__ double sh[256];
    double v = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) v = v + part[t];
    v = block_reduce<1>(v, sh);
    if (threadIdx.x == 0) {
        sc->rho2 = sc->rho1;
        sc->rho1 = v;
        sc->iter += 1;
        sc->beta = sc->iter == 1 ? 0.0 : __ddiv_rn(sc->rho1, sc->rho2);
    }
}
__global__ void k_cg_pap(const double *__restrict__ part, int n, CgScal *sc) {
    pdl_entry();
    __shared__ double sh[256];
    double v = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) v = v + part[t];
    v = block_reduce<1>(v, sh);
    if (threadIdx.x == 0) {
        sc->pap = v;
        sc->alpha = __ddiv_rn(sc->rho1, v);
    }
}
// pp = zz + beta*pp, then the overlap copy of pp (bbmg_class.f90:674-676)
template <typename TZ>
__global__ void __launch_bounds__(256) k_cg_p(Lay L, const TZ *__restrict__ zz, double *__restrict__ pp,
                                               const CgScal *__restrict__ sc) {
    pdl_entry();
    const double beta = sc->beta;
    const long long total = (long long)L.nx * L.ny * L.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        long long id = L.idx(i, j, k);
        double val = __dadd_rn((double)zz[id], __dmul_rn(beta, pp[id]));
        pp[id] = val;
        if (on_periodic_face(L, i, j, k)) write_images(L, pp, i, j, k, val);
    }
}
// sol += alpha*pp; res -= alpha*Ap (bbmg_class.f90:688-692)
__global__ void __launch_bounds__(256) k_cg_xr(Lay L, double *__restrict__ sol, const double *__restrict__ pp,
                                                double *__restrict__ res, const double *__restrict__ Ap,
                                                const CgScal *__restrict__ sc) {
    pdl_entry();
    const double alpha = sc->alpha;
    const long long total = (long long)L.nx * L.ny * L.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        long long id = L.idx(i, j, k);
        sol[id] = __dadd_rn(sol[id], __dmul_rn(alpha, pp[id]));
        res[id] = __dsub_rn(res[id], __dmul_rn(alpha, Ap[id]));
    }
}

// mixed precision: FP64 residual -> FP32 right-hand side of the V-cycle
__global__ void __launch_bounds__(256) k_round_f32(Lay L, const double *__restrict__ r, float *__restrict__ f) {
    pdl_entry();
    const long long total = (long long)L.nx * L.ny * L.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        long long id = L.idx(i, j, k);
        f[id] = (float)r[id];
    }
}
// mixed precision: x += e (FP32 correction accumulated in FP64), images kept
__global__ void __launch_bounds__(256) k_add_correction(Lay L, double *__restrict__ x, const float *__restrict__ e) {
    pdl_entry();
    const long long total = (long long)L.nx * L.ny * L.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        long long id = L.idx(i, j, k);
        double val = x[id] + (double)e[id];
        x[id] = val;
        if (on_periodic_face(L, i, j, k)) write_images(L, x, i, j, k, val);
    }
}

template <typename TZ>
cudaError_t launch_cg_rho(const Lay &L, const TZ *zz, const double *res, double *part, CgScal *sc, cudaStream_t s) {
    launch_k(k_dot_part<TZ, double>, kRedBlocks, 256, 0, s, L, zz, res, part);
    BB_CHECK_LAUNCH();
    launch_k(k_cg_rho, 1, 256, 0, s, part, kRedBlocks, sc);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}
template <typename TZ>
cudaError_t launch_cg_p(const Lay &L, const TZ *zz, double *pp, const CgScal *sc, cudaStream_t s) {
    long long n = (long long)L.nx * L.ny * L.nz;
    launch_k(k_cg_p<TZ>, grid_for(n, 256), 256, 0, s, L, zz, pp, sc);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}
cudaError_t launch_cg_pap(const Lay &L, const double *pp, const double *Ap, double *part, CgScal *sc, cudaStream_t s) {
    launch_k(k_dot_part<double, double>, kRedBlocks, 256, 0, s, L, pp, Ap, part);
    BB_CHECK_LAUNCH();
    launch_k(k_cg_pap, 1, 256, 0, s, part, kRedBlocks, sc);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}
cudaError_t launch_cg_xr(const Lay &L, double *sol, const double *pp, double *res, const double *Ap, const CgScal *sc,
                         cudaStream_t s) {
    long long n = (long long)L.nx * L.ny * L.nz;
    launch_k(k_cg_xr, grid_for(n, 256), 256, 0, s, L, sol, pp, res, Ap, sc);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}
cudaError_t launch_round_f32(const Lay &L, const double *r, float *f, cudaStream_t s) {
    long long n = (long long)L.nx * L.ny * L.nz;
    launch_k(k_round_f32, grid_for(n, 256), 256, 0, s, L, r, f);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}
cudaError_t launch_add_correction(const Lay &L, double *x, const float *e, cudaStream_t s) {
    long long n = (long long)L.nx * L.ny * L.nz;
    launch_k(k_add_correction, grid_for(n, 256), 256, 0, s, L, x, e);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}
template cudaError_t launch_cg_rho<double>(const Lay &, const double *, const double *, double *, CgScal *, cudaStream_t);
template cudaError_t launch_cg_rho<float>(const Lay &, const float *, const double *, double *, CgScal *, cudaStream_t);
template cudaError_t launch_cg_p<double>(const Lay &, const double *, double *, const CgScal *, cudaStream_t);
template cudaError_t launch_cg_p<float>(const Lay &, const float *, double *, const CgScal *, cudaStream_t);


// ---------------------------------------------------------------------------
// Fused CG steps.  pp_new = zz + beta*pp_old on the own cell (with images) and
// Ap = A pp_new, the neighbours' pp_new formed on the fly from zz and pp_old
// (bit-identical to the stored value), plus the block partial of pp_new.Ap
// (bbmg_class.f90:674-687 in one pass).  pp_old and pp_new are distinct
// buffers.
template <typename TZ, int NPT>
__global__ void __launch_bounds__(256) k_cg_pap_fused(Lay L, NbrOff nb, const double *__restrict__ opr,
                                                       const TZ *__restrict__ zz, const double *__restrict__ pp_old,
                                                       double *__restrict__ pp_new, double *__restrict__ Ap,
                                                       const CgScal *__restrict__ sc, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    const double beta = sc->beta;
    const long long total = (long long)L.nx * L.ny * L.nz;
    double acc = 0.0;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        const int par = i & 1;
        const long long id = L.idx(i, j, k);
        double s = 0.0, pc = 0.0;
#pragma unroll
        for (int q = 0; q < Lay7<NPT>::terms; q++) {
            const int q27i = Lay7<NPT>::slot(q);
            const int o = par ? nb.off[1][q27i] : nb.off[0][q27i];
            const double pq = __dadd_rn((double)zz[id + o], __dmul_rn(beta, pp_old[id + o]));
            if (q == Lay7<NPT>::centre) pc = pq;
            s = __dadd_rn(s, __dmul_rn(opr[Lay7<NPT>::plane(q) * L.plane + id + (Lay7<NPT>::at_nbr(q) ? o : 0)], pq));
        }
        pp_new[id] = pc;
        if (on_periodic_face(L, i, j, k)) write_images(L, pp_new, i, j, k, pc);
        Ap[id] = s;
        acc = __dadd_rn(acc, __dmul_rn(pc, s));
    }
    acc = block_reduce<1>(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// sol += alpha*pp; res -= alpha*Ap; block partial of max|res|
// (bbmg_class.f90:688-695).  Also prepares the next preconditioner call: the
// FP32 right-hand side (mixed precision) and a zero correction vector
// (bbmg_class.f90:657-659), images included.
template <typename TV>
__global__ void __launch_bounds__(256) k_cg_xr_fused(Lay L, double *__restrict__ sol, const double *__restrict__ pp,
                                                      double *__restrict__ res, const double *__restrict__ Ap,
                                                      const CgScal *__restrict__ sc, float *__restrict__ f32,
                                                      TV *__restrict__ vzero, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    const double alpha = sc->alpha;
    const long long total = (long long)L.nx * L.ny * L.nz;
    double m = 0.0;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        const long long id = L.idx(i, j, k);
        sol[id] = __dadd_rn(sol[id], __dmul_rn(alpha, pp[id]));
        const double r = __dsub_rn(res[id], __dmul_rn(alpha, Ap[id]));
        res[id] = r;
        const double a = fabs(r);
        m = (a != a || m != m) ? (a + m) : fmax(m, a);
        if (f32) f32[id] = (float)r;
        vzero[id] = TV(0);
        if (on_periodic_face(L, i, j, k)) write_images(L, vzero, i, j, k, TV(0));
    }
    m = block_reduce<0>(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

template <typename TZ>
cudaError_t launch_cg_pap_fused(const Lay &L, const NbrOff &nb, int npt, const double *opr, const TZ *zz,
                                const double *pp_old, double *pp_new, double *Ap, double *part, CgScal *sc,
                                cudaStream_t s) {
    if (npt == 4) launch_k(k_cg_pap_fused<TZ, 4>, kRedBlocks, 256, 0, s, L, nb, opr, zz, pp_old, pp_new, Ap, sc, part);
    else if (npt == 7) launch_k(k_cg_pap_fused<TZ, 7>, kRedBlocks, 256, 0, s, L, nb, opr, zz, pp_old, pp_new, Ap, sc, part);
    else launch_k(k_cg_pap_fused<TZ, 27>, kRedBlocks, 256, 0, s, L, nb, opr, zz, pp_old, pp_new, Ap, sc, part);
    BB_CHECK_LAUNCH();
    launch_k(k_cg_pap, 1, 256, 0, s, part, kRedBlocks, sc);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}

template <typename TV>
cudaError_t launch_cg_xr_fused(const Lay &L, double *sol, const double *pp, double *res, const double *Ap,
                               const CgScal *sc, float *f32, TV *vzero, double *part, double *out, cudaStream_t s) {
    launch_k(k_cg_xr_fused<TV>, kRedBlocks, 256, 0, s, L, sol, pp, res, Ap, sc, f32, vzero, part);
    BB_CHECK_LAUNCH();
    launch_k(k_final<0>, 1, 256, 0, s, part, kRedBlocks, out);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}
template cudaError_t launch_cg_pap_fused<double>(const Lay &, const NbrOff &, int, const double *, const double *,
                                                 const double *, double *, double *, double *, CgScal *, cudaStream_t);
template cudaError_t launch_cg_pap_fused<float>(const Lay &, const NbrOff &, int, const double *, const float *,
                                                const double *, double *, double *, double *, CgScal *, cudaStream_t);
template cudaError_t launch_cg_xr_fused<double>(const Lay &, double *, const double *, double *, const double *,
                                                const CgScal *, float *, double *, double *, double *, cudaStream_t);
template cudaError_t launch_cg_xr_fused<float>(const Lay &, double *, const double *, double *, const double *,
                                               const CgScal *, float *, float *, double *, double *, cudaStream_t);

// ---------------------------------------------------------------------------
// 7-point operators: the colours of one Gauss-Seidel sweep only couple to
// colours of Hamming weight +-1 (weight = px+py+pz), so the 8-colour sweep in
// the reference's order equals four phases by weight (0,1,2,3 forward,
// 3,2,1,0 backward): the colours inside a phase never read each other.  A phase
// repeated back to back (the last of a forward sweep and the first of the
// following backward sweep) recomputes identical values and is skipped.  The
// result is bit-identical to the colour-by-colour sweep; one launch per phase.
struct PhaseCols {
    int n;             // colours in the phase (1..3)
    int col[3];        // colour index px + 2py + 4pz, ascending
    long long beg[4];  // prefix sums of the colour point counts
};

template <typename T, int NPT>
__global__ void __launch_bounds__(256) k_relax_phase7(Lay L, NbrOff nb, const T *__restrict__ opr, T *v,
                                                       const T *__restrict__ f, PhaseCols pc, int fuse) {
    pdl_entry();
    using O = Ops<T, ExactOf<T>::value>;
    const long long total = pc.beg[pc.n];
    for (long long t = gtid(); t < total; t += gstride()) {
        int c = 0;
        if (pc.n > 1 && t >= pc.beg[1]) c = (pc.n > 2 && t >= pc.beg[2]) ? 2 : 1;
        const int col = pc.col[c];
        const int px = col & 1, py = (col >> 1) & 1, pz = (col >> 2) & 1;
        const int na = (L.nx - px + 1) >> 1, nbb = (L.ny - py + 1) >> 1;
        const long long u = t - pc.beg[c];
        const int a = (int)(u % na);
        const long long rr = u / na;
        const int b = (int)(rr % nbb), cc = (int)(rr / nbb);
        const int i = px + 2 * a, j = py + 2 * b, k = pz + 2 * cc;
        const long long id = L.idx(i, j, k);
        T s = T(0);
#pragma unroll
        for (int q = 0; q < 7; q++) {
            if (q == kCentre7) continue;
            const int q27i = k7to27(q);
            const int o = px ? nb.off[1][q27i] : nb.off[0][q27i];
            s = O::mac(s, opr[Lay7<NPT>::plane(q) * L.plane + id + (Lay7<NPT>::at_nbr(q) ? o : 0)], v[id + o]);
        }
        const T d = opr[Lay7<NPT>::plane(kCentre7) * L.plane + id];
        const T val = O::div(O::sub(f[id], s), O::add(d, T(kEps)));
        v[id] = val;
        if (fuse && on_periodic_face(L, i, j, k)) write_images(L, v, i, j, k, val);
    }
}

static PhaseCols phase_cols(const Lay &L, int w) {
    PhaseCols p{};
    p.n = 0;
    p.beg[0] = 0;
    for (int col = 0; col < 8; col++) {
        if (__builtin_popcount(col) != w) continue;
        int px = col & 1, py = (col >> 1) & 1, pz = (col >> 2) & 1;
        long long cnt = (long long)((L.nx - px + 1) >> 1) * ((L.ny - py + 1) >> 1) * ((L.nz - pz + 1) >> 1);
        if (cnt == 0) continue;
        p.col[p.n] = col;
        p.beg[p.n + 1] = p.beg[p.n] + cnt;
        p.n++;
    }
    return p;
}

template <typename T>
cudaError_t launch_relax_sweeps(const Lay &L, const NbrOff &nb, int npt, bool fuse, const T *opr, T *v, const T *f,
                                int first_dir, int nsweeps, cudaStream_t s) {
    if (npt == 27 || !fuse) {
        int dir = first_dir;
        for (int i = 0; i < nsweeps; i++) {
            cudaError_t e = launch_relax<T>(L, nb, npt, fuse, opr, v, f, dir, s);
            if (e != cudaSuccess) return e;
            dir = -dir;
        }
        return cudaSuccess;
    }
    int dir = first_dir, last = -1;
    for (int i = 0; i < nsweeps; i++) {
        for (int p = 0; p < 4; p++) {
            int w = dir > 0 ? p : 3 - p;
            if (w == last) continue;  // identical recomputation
            last = w;
            PhaseCols pc = phase_cols(L, w);
            if (pc.n == 0) continue;
            if (npt == 4) launch_k(k_relax_phase7<T, 4>, grid_for(pc.beg[pc.n], 256), 256, 0, s, L, nb, opr, v, f, pc, 1);
            else launch_k(k_relax_phase7<T, 7>, grid_for(pc.beg[pc.n], 256), 256, 0, s, L, nb, opr, v, f, pc, 1);
            BB_CHECK_LAUNCH();
        }
        dir = -dir;
    }
    return cudaSuccess;
}
template cudaError_t launch_relax_sweeps<double>(const Lay &, const NbrOff &, int, bool, const double *, double *,
                                                 const double *, int, int, cudaStream_t);
template cudaError_t launch_relax_sweeps<float>(const Lay &, const NbrOff &, int, bool, const float *, float *,
                                                const float *, int, int, cudaStream_t);

// ---------------------------------------------------------------------------
// Mixed-precision defect correction step (the FP64 half of an mgsolve
// iteration, bbmg_class.f90:716-722 with the correction of 770): x_new = x + e
// on the own cell (images written), r = b - A (x + e) with the neighbours'
// x + e formed on the fly; r becomes the FP32 right-hand side of the next
// V-cycle, the FP32 correction is zeroed for it, and the block partial of
// max|r| is written.  x_old and x_new are distinct buffers.
template <int NPT>
__global__ void __launch_bounds__(256) k_defect_fused(Lay L, NbrOff nb, const double *__restrict__ opr,
                                                       const double *__restrict__ x_old, const float *__restrict__ e,
                                                       const double *__restrict__ b, double *__restrict__ x_new,
                                                       float *__restrict__ f32, float *__restrict__ v32,
                                                       double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    const long long total = (long long)L.nx * L.ny * L.nz;
    double m = 0.0;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        const int par = i & 1;
        const long long id = L.idx(i, j, k);
        double s = 0.0, xc = 0.0;
#pragma unroll
        for (int q = 0; q < Lay7<NPT>::terms; q++) {
            const int q27i = Lay7<NPT>::slot(q);
            const int o = par ? nb.off[1][q27i] : nb.off[0][q27i];
            const double xq = x_old[id + o] + (double)e[id + o];
            if (q == Lay7<NPT>::centre) xc = xq;
            s = fma(opr[Lay7<NPT>::plane(q) * L.plane + id + (Lay7<NPT>::at_nbr(q) ? o : 0)], xq, s);
        }
        const double r = b[id] - s;
        x_new[id] = xc;
        f32[id] = (float)r;
        v32[id] = 0.0f;
        if (on_periodic_face(L, i, j, k)) {
            write_images(L, x_new, i, j, k, xc);
            write_images(L, v32, i, j, k, 0.0f);
        }
        const double a = fabs(r);
        m = (a != a || m != m) ? (a + m) : fmax(m, a);
    }
    m = block_reduce<0>(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

cudaError_t launch_defect_fused(const Lay &L, const NbrOff &nb, int npt, const double *opr, const double *x_old,
                                const float *e, const double *b, double *x_new, float *f32, float *v32, double *part,
                                double *out, cudaStream_t s) {
    if (npt == 4) launch_k(k_defect_fused<4>, kRedBlocks, 256, 0, s, L, nb, opr, x_old, e, b, x_new, f32, v32, part);
    else if (npt == 7) launch_k(k_defect_fused<7>, kRedBlocks, 256, 0, s, L, nb, opr, x_old, e, b, x_new, f32, v32, part);
    else launch_k(k_defect_fused<27>, kRedBlocks, 256, 0, s, L, nb, opr, x_old, e, b, x_new, f32, v32, part);
    BB_CHECK_LAUNCH();
    launch_k(k_final<0>, 1, 256, 0, s, part, kRedBlocks, out);
    BB_CHECK_LAUNCH();
    return cudaSuccess;
}
#define BB_INST(T)                                                                                                   \
    template cudaError_t launch_relax<T>(const Lay &, const NbrOff &, int, bool, const T *, T *, const T *, int,     \
                                         cudaStream_t);                                                              \
    template cudaError_t launch_residual<T>(const Lay &, const NbrOff &, int, const T *, const T *, const T *, T *,  \
                                            cudaStream_t);                                                           \
    template cudaError_t launch_restrict<T>(const Lay &, const Lay &, const T *, const T *, T *, T *, cudaStream_t); \
    template cudaError_t launch_prolong<T>(const Lay &, const Lay &, const T *, const T *, T *, cudaStream_t);       \
    template cudaError_t launch_coarse_solve<T>(const Lay &, const double *, const int *, const int *, const T *,    \
                                                T *, cudaStream_t);                                                  \
    template cudaError_t launch_maxabs<T>(const Lay &, const T *, double *, double *, cudaStream_t);                \
    template cudaError_t launch_dot<T>(const Lay &, const T *, const T *, double *, double *, cudaStream_t);        \
    template cudaError_t launch_from_caller<T>(const Lay &, const double *, int, T *, cudaStream_t);
BB_INST(double)
BB_INST(float)

}  // namespace bbmg
