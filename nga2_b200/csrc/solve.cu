// solve.cu -- V-cycle kernels of the black-box multigrid (FP64 and FP32).
//
// Each kernel restates one solve-phase routine of src/solver/bbmg_class.f90.
// The FP64 instantiation evaluates every sum in the reference's column-major
// term order without FMA contraction, so it matches the oracle bit for bit;
// the FP32 instantiation is the fast V-cycle of the mixed precision solver and
// uses FMA.  Terms whose coefficient is structurally zero (the 20 unused slots
// of a 7-point operator, prolongation weights of the other parity classes) are
// skipped: adding +0.0 does not change a sum.
//
// Work mapping: a 2-D launch whose y dimension walks (j,k) rows and whose x
// dimension walks positions inside a row, so no thread divides a 64-bit
// linear index.  The Gauss-Seidel kernels give each thread VW consecutive
// points of one half-row (16-byte vector loads); neighbour offsets that are
// not a multiple of VW (the odd x-neighbour) fall back to scalar loads that
// hit the lines the aligned loads just brought in.
#include <cstdlib>

#include "setup.cuh"

namespace bbmg {

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
// The two halves, for kernels that first read data no kernel of the solve
// writes (the operator planes, written only by the setup, which ends with a
// stream synchronisation): those loads may start before the wait, while the
// predecessor (or the one before it, still running its own tail) finishes.
__device__ __forceinline__ void pdl_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// L2 prefetch of the line holding p (a hint; L2 is coherent, so it is safe
// for any operand, also one the predecessor is still writing)
__device__ __forceinline__ void pf_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

template <typename... KArgs, typename... Args>
static cudaError_t launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t shm, cudaStream_t s,
                            Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = shm;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

#define BB_CHECK_LAUNCH(call)                \
    do {                                     \
        cudaError_t e0_ = (call);            \
        if (e0_ != cudaSuccess) return e0_;  \
        cudaError_t e_ = cudaGetLastError(); \
        if (e_ != cudaSuccess) return e_;    \
    } while (0)

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
// launch geometry: x = chunks of a row, y = rows (grid-stride in both)
struct Geo {
    dim3 grid, block;
};
static Geo geo_rows(long long nchunks, long long nrows, long long cap_blocks = 148LL * 24) {
    int bx = 1;
    while (bx < nchunks && bx < 128) bx <<= 1;
    int by = 256 / bx;
    long long gx = (nchunks + bx - 1) / bx;
    if (gx < 1) gx = 1;
    long long gy = (nrows + by - 1) / by;
    long long cy = cap_blocks / gx;
    if (cy < 1) cy = 1;
    if (gy > cy) gy = cy;
    if (gy > 65535) gy = 65535;
    if (gy < 1) gy = 1;
    return {dim3((unsigned)gx, (unsigned)gy), dim3((unsigned)bx, (unsigned)by)};
}
// fixed geometry of the deterministic reductions on a level
static Geo geo_red(const Lay &L) { return geo_rows(L.nx, (long long)L.ny * L.nz, kRedBlocks); }

#define FOR_ROWS(nrows) for (int row = blockIdx.y * blockDim.y + threadIdx.y; row < (nrows); row += gridDim.y * blockDim.y)
#define FOR_CHUNKS(nch) for (int ch = blockIdx.x * blockDim.x + threadIdx.x; ch < (nch); ch += gridDim.x * blockDim.x)

// storage-order position t of a row -> x index (odd x first, then even x)
__device__ __forceinline__ int x_of(const Lay &L, int t) {
    const int nodd = L.nx >> 1;
    return t < nodd ? 2 * t + 1 : 2 * (t - nodd);
}

// VW consecutive values, one vector load when aligned
template <int VW, typename T> struct VecT;
template <> struct VecT<1, float> { using type = float; };
template <> struct VecT<2, float> { using type = float2; };
template <> struct VecT<4, float> { using type = float4; };
template <> struct VecT<1, double> { using type = double; };
template <> struct VecT<2, double> { using type = double2; };

template <int VW, typename T>
__device__ __forceinline__ void ldv(const T *p, bool aligned, T (&o)[VW]) {
    if (VW == 1 || !aligned) {
#pragma unroll
        for (int e = 0; e < VW; e++) o[e] = p[e];
    } else {
        using V = typename VecT<VW, T>::type;
        const V w = *reinterpret_cast<const V *>(p);
        const T *wp = reinterpret_cast<const T *>(&w);
#pragma unroll
        for (int e = 0; e < VW; e++) o[e] = wp[e];
    }
}
// aligned vector load marked evict-first in L1 and L2 (ld.global.cs): for
// operands read once per pass, so that they do not displace reused lines
template <int VW, typename T>
__device__ __forceinline__ void ldv_cs(const T *p, T (&o)[VW]) {
    if (VW == 1) {
        o[0] = __ldcs(p);
    } else {
        using V = typename VecT<VW, T>::type;
        const V w = __ldcs(reinterpret_cast<const V *>(p));
        const T *wp = reinterpret_cast<const T *>(&w);
#pragma unroll
        for (int e = 0; e < VW; e++) o[e] = wp[e];
    }
}
template <int VW, typename T>
__device__ __forceinline__ void stv(T *p, const T (&o)[VW]) {
    if (VW == 1) {
        p[0] = o[0];
    } else {
        using V = typename VecT<VW, T>::type;
        V w;
        T *wp = reinterpret_cast<T *>(&w);
#pragma unroll
        for (int e = 0; e < VW; e++) wp[e] = o[e];
        *reinterpret_cast<V *>(p) = w;
    }
}

// ---------------------------------------------------------------------------
// Gauss-Seidel update of VW points of colour (px,py,pz) starting at id0
// (bbmg_class.f90:876-880): A = (B - sum_{l != 0} opr(l) A(nbr)) / (opr(0)+eps).
template <typename T, int NPT, int VW>
__device__ __forceinline__ void gs_points(const Lay &L, const Off27 &off, const T *__restrict__ opr, T *v,
                                          const T *__restrict__ f, long long id0, int px, int j, int k, int a0,
                                          int fuse, bool cs = false) {
    using O = Ops<T, ExactOf<T>::value>;
    T s[VW];
#pragma unroll
    for (int e = 0; e < VW; e++) s[e] = T(0);
#pragma unroll
    for (int q = 0; q < Lay7<NPT>::terms; q++) {
        if (q == Lay7<NPT>::centre) continue;
        const int o = off.o[Lay7<NPT>::slot(q)];
        const bool al = (o % VW) == 0;
        T cv[VW], vv[VW];
        ldv<VW>(opr + (long long)Lay7<NPT>::plane(q) * L.plane + id0 + (Lay7<NPT>::at_nbr(q) ? o : 0),
                Lay7<NPT>::at_nbr(q) ? al : true, cv);
        ldv<VW>(v + id0 + o, al, vv);
#pragma unroll
        for (int e = 0; e < VW; e++) s[e] = O::mac(s[e], cv[e], vv[e]);
    }
    T dv[VW], fv[VW], out[VW];
    if (cs) {
        ldv_cs<VW>(opr + (long long)Lay7<NPT>::plane(Lay7<NPT>::centre) * L.plane + id0, dv);
        ldv_cs<VW>(f + id0, fv);
    } else {
        ldv<VW>(opr + (long long)Lay7<NPT>::plane(Lay7<NPT>::centre) * L.plane + id0, true, dv);
        ldv<VW>(f + id0, true, fv);
    }
#pragma unroll
    for (int e = 0; e < VW; e++) out[e] = O::div(O::sub(fv[e], s[e]), O::add(dv[e], T(kEps)));
    stv<VW>(v + id0, out);
    if (fuse) {
#pragma unroll
        for (int e = 0; e < VW; e++) {
            const int i = px + 2 * (a0 + e);
            if (on_periodic_face(L, i, j, k)) write_images(L, v, i, j, k, out[e]);
        }
    }
}

// One colour of the 8-colour Gauss-Seidel (bbmg_class.f90:872-885) on the
// points i = px + 2a, j = py + 2b, k = pz + 2c.  With `fuse` the new value is
// also written into its periodic images (the vsync after the colour); that is
// only race-free when every periodic direction has an even size, otherwise the
// caller runs the overlap copy as a separate pass.
template <typename T, int NPT, int VW>
__global__ void __launch_bounds__(256) k_relax(Lay L, Off27 off, const T *__restrict__ opr, T *v,
                                                const T *__restrict__ f, int px, int py, int pz, int fuse) {
    pdl_entry();
    const int na = (L.nx - px + 1) >> 1, nb = (L.ny - py + 1) >> 1, nc = (L.nz - pz + 1) >> 1;
    const int nrows = nb * nc, nch = na / VW;
    const long long hb = px ? 0 : L.B0;
    FOR_ROWS(nrows) {
        const int b = row % nb, c = row / nb;
        const int j = py + 2 * b, k = pz + 2 * c;
        const long long base = L.G + L.row(j, k) * L.P + hb;
        FOR_CHUNKS(nch) {
            gs_points<T, NPT, VW>(L, off, opr, v, f, base + (long long)ch * VW, px, j, k, ch * VW, fuse);
        }
    }
}

// 7-point operators: the colours of one sweep only couple to colours of
// Hamming weight +-1 (weight = px+py+pz), so the 8-colour sweep in the
// reference's order equals four phases by weight (0,1,2,3 forward, 3,2,1,0
// backward): the colours inside a phase never read each other.  A phase
// repeated back to back (the last of a forward sweep and the first of the
// following backward sweep) recomputes identical values and is skipped.  The
// result is bit-identical to the colour-by-colour sweep; one launch per
// phase, blockIdx.z = colour within the phase.
struct PhaseCols {
    int n;         // colours in the phase (1..3)
    int col[3];    // colour index px + 2py + 4pz, ascending
    Off27 off[2];  // neighbour offsets for even / odd x
};

// Block order (`ord`): bit 0 walks the rows from the last (k, j) to the first,
// bit 1 interleaves the phase's colours (consecutive blocks take the same rows
// of the different colours instead of one colour after the other), bit 2 loads
// the centre coefficient and f evict-first, bit 3 prefetches the first point
// group's operator lines into L2 before the wait for the predecessor.  The
// colours of a phase are independent and every point is written once, so the
// order changes no bits.
template <typename T, int NPT, int VW>
__global__ void __launch_bounds__(256) k_relax_phase7(Lay L, const T *__restrict__ opr, T *v,
                                                       const T *__restrict__ f, PhaseCols pc, int fuse, int ord) {
    pdl_launch();
    unsigned zc = blockIdx.z, yb = blockIdx.y;
    if (ord & 2) {
        const unsigned lin = blockIdx.y + gridDim.y * blockIdx.z;
        zc = lin % gridDim.z;
        yb = lin / gridDim.z;
    }
    const int col = pc.col[zc];
    const int px = col & 1, py = (col >> 1) & 1, pz = (col >> 2) & 1;
    const int na = (L.nx - px + 1) >> 1, nb = (L.ny - py + 1) >> 1, nc = (L.nz - pz + 1) >> 1;
    const int nrows = nb * nc, nch = na / VW;
    const long long hb = px ? 0 : L.B0;
    const Off27 &off = pc.off[px];
    const bool cs = (ord & 4) != 0;
    if (ord & 8) {  // the first point group's operator lines into L2 while the predecessor finishes
        const int r0 = yb * blockDim.y + threadIdx.y, ch = blockIdx.x * blockDim.x + threadIdx.x;
        if (r0 < nrows && ch < nch) {
            const int row = (ord & 1) ? nrows - 1 - r0 : r0;
            const long long id0 = L.G + L.row(py + 2 * (row % nb), pz + 2 * (row / nb)) * L.P + hb + (long long)ch * VW;
#pragma unroll
            for (int q = 0; q < Lay7<NPT>::terms; q++)
                pf_l2(opr + (long long)Lay7<NPT>::plane(q) * L.plane + id0 +
                      (Lay7<NPT>::at_nbr(q) ? off.o[Lay7<NPT>::slot(q)] : 0));
        }
    }
    pdl_wait();
    for (int r0 = yb * blockDim.y + threadIdx.y; r0 < nrows; r0 += gridDim.y * blockDim.y) {
        const int row = (ord & 1) ? nrows - 1 - r0 : r0;
        const int b = row % nb, c = row / nb;
        const int j = py + 2 * b, k = pz + 2 * c;
        const long long base = L.G + L.row(j, k) * L.P + hb;
        FOR_CHUNKS(nch) {
            gs_points<T, NPT, VW>(L, off, opr, v, f, base + (long long)ch * VW, px, j, k, ch * VW, fuse, cs);
        }
    }
}

// 16-byte asynchronous global -> shared copy (cp.async, L1 bypassed).
__device__ __forceinline__ void cp16(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

// One colour of the FP32 27-point Gauss-Seidel with its operands staged in
// shared memory: one warp per half-row of the colour.  It copies the 27
// coefficient planes and f at its points, and for each of the 9 rows
// (j+dy, k+dz) the v values of its own x-half (not for the row itself: v(i)
// is not read) and of the other x-half (from 4 elements before to 4 after,
// for the i-1 / i+1 neighbours), then updates its points term for term as
// gs_points does (column-major order, centre last): identical bits.
// Requires na (points per half-row) to be a multiple of 4.
template <typename T>
__global__ void __launch_bounds__(128) k_relax27_staged(Lay L, const T *__restrict__ opr, T *v,
                                                         const T *__restrict__ f, int px, int py, int pz,
                                                         int fuse, int na) {
    pdl_launch();
    extern __shared__ __align__(16) unsigned char smraw[];
    T *smf = reinterpret_cast<T *>(smraw);
    using O = Ops<T, ExactOf<T>::value>;
    constexpr int EPC = 16 / sizeof(T);  // elements per 16-byte copy
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = na + 8;
    T *S = smf + (size_t)warp * 46 * seg;
    // segments: 0..26 coefficient planes; 27 f; 28 + 2*(row) own half v, 29 + 2*(row) other half v,
    // row = (dy+1) + 3*(dz+1)
    const int nb = (L.ny - py + 1) >> 1, nc = (L.nz - pz + 1) >> 1;
    const int nrows = nb * nc;
    const long long hown = px ? 0 : L.B0, hoth = px ? L.B0 : 0;
    const long long P = L.plane;
    const int om = px ? 4 : 3, op = px ? 5 : 4;  // other-half index of i-1 / i+1 (slack 4)
    // the first row's coefficient planes before the wait for the predecessor
    int row = blockIdx.x * 4 + warp;
    if (row < nrows) {
        const long long r0 = L.G + L.row(py + 2 * (row % nb), pz + 2 * (row / nb)) * L.P;
        for (int e = lane * EPC; e < na; e += 32 * EPC) {
#pragma unroll
            for (int q = 0; q < 27; q++) cp16(S + q * seg + e, opr + q * P + r0 + hown + e);
        }
    }
    pdl_wait();
    for (bool first = true; row < nrows; row += gridDim.x * 4, first = false) {
        const int j = py + 2 * (row % nb), k = pz + 2 * (row / nb);
        const long long r0 = L.G + L.row(j, k) * L.P;
        __syncwarp();
        for (int e = lane * EPC; e < na; e += 32 * EPC) {
            if (!first) {
#pragma unroll
                for (int q = 0; q < 27; q++) cp16(S + q * seg + e, opr + q * P + r0 + hown + e);
            }
            cp16(S + 27 * seg + e, f + r0 + hown + e);
        }
#pragma unroll
        for (int rr = 0; rr < 9; rr++) {
            const int dy = rr % 3 - 1, dz = rr / 3 - 1;
            const long long rb = L.G + L.row(j + dy, k + dz) * L.P;
            for (int e = lane * EPC; e < seg; e += 32 * EPC) {
                if (rr != 4 && e < na) cp16(S + (28 + 2 * rr) * seg + e, v + rb + hown + e);
                cp16(S + (29 + 2 * rr) * seg + e, v + rb + hoth - 4 + e);
            }
        }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        __syncwarp();
        for (int a = lane; a < na; a += 32) {
            T sum = T(0);
#pragma unroll
            for (int q = 0; q < 27; q++) {
                if (q == 13) continue;
                const int dx = q % 3 - 1, rr = q / 3;  // rr = (dy+1) + 3 (dz+1)
                const T vv = dx == 0 ? S[(28 + 2 * rr) * seg + a]
                                         : S[(29 + 2 * rr) * seg + a + (dx < 0 ? om : op)];
                sum = O::mac(sum, S[q * seg + a], vv);
            }
            const T out = O::div(O::sub(S[27 * seg + a], sum), O::add(S[13 * seg + a], T(kEps)));
            v[r0 + hown + a] = out;
            const int i = px + 2 * a;
            if (fuse && on_periodic_face(L, i, j, k)) write_images(L, v, i, j, k, out);
        }
    }
}

// Residual of an FP32 27-point level with its operands staged as in
// k_relax27_staged: one warp per x-half of a (j,k) row (both halves of every
// row, so blockIdx/warp walk 2 * ny * nz jobs); here the row's own v is copied
// too and the centre term enters the sum in its column-major place, as in
// residual_point: identical bits.
template <typename T>
__global__ void __launch_bounds__(128) k_residual27_staged(Lay L, const T *__restrict__ opr,
                                                            const T *__restrict__ v, const T *__restrict__ f,
                                                            T *__restrict__ r, int na) {
    pdl_launch();
    extern __shared__ __align__(16) unsigned char smraw[];
    T *smf = reinterpret_cast<T *>(smraw);
    using O = Ops<T, ExactOf<T>::value>;
    constexpr int EPC = 16 / sizeof(T);  // elements per 16-byte copy
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = na + 8;
    T *S = smf + (size_t)warp * 46 * seg;
    const long long P = L.plane;
    const int njobs = 2 * L.ny * L.nz;
    // the first job's coefficient planes before the wait for the predecessor
    int job = blockIdx.x * 4 + warp;
    if (job < njobs) {
        const long long r0 = L.G + L.row((job >> 1) % L.ny, (job >> 1) / L.ny) * L.P + ((job & 1) ? 0 : L.B0);
        for (int e = lane * EPC; e < na; e += 32 * EPC) {
#pragma unroll
            for (int q = 0; q < 27; q++) cp16(S + q * seg + e, opr + q * P + r0 + e);
        }
    }
    pdl_wait();
    for (bool first = true; job < njobs; job += gridDim.x * 4, first = false) {
        const int px = job & 1, row = job >> 1;  // px = 1: odd-x half, 0: even-x half
        const int j = row % L.ny, k = row / L.ny;
        const long long hown = px ? 0 : L.B0, hoth = px ? L.B0 : 0;
        const int om = px ? 4 : 3, op = px ? 5 : 4;
        const long long r0 = L.G + L.row(j, k) * L.P;
        __syncwarp();
        for (int e = lane * EPC; e < na; e += 32 * EPC) {
            if (!first) {
#pragma unroll
                for (int q = 0; q < 27; q++) cp16(S + q * seg + e, opr + q * P + r0 + hown + e);
            }
            cp16(S + 27 * seg + e, f + r0 + hown + e);
        }
#pragma unroll
        for (int rr = 0; rr < 9; rr++) {
            const int dy = rr % 3 - 1, dz = rr / 3 - 1;
            const long long rb = L.G + L.row(j + dy, k + dz) * L.P;
            for (int e = lane * EPC; e < seg; e += 32 * EPC) {
                if (e < na) cp16(S + (28 + 2 * rr) * seg + e, v + rb + hown + e);
                cp16(S + (29 + 2 * rr) * seg + e, v + rb + hoth - 4 + e);
            }
        }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        __syncwarp();
        for (int a = lane; a < na; a += 32) {
            T sum = T(0);
#pragma unroll
            for (int q = 0; q < 27; q++) {
                const int dx = q % 3 - 1, rr = q / 3;
                const T vv = dx == 0 ? S[(28 + 2 * rr) * seg + a]
                                         : S[(29 + 2 * rr) * seg + a + (dx < 0 ? om : op)];
                sum = O::mac(sum, S[q * seg + a], vv);
            }
            const T out = O::sub(S[27 * seg + a], sum);
            r[r0 + hown + a] = out;
            const int i = px + 2 * a;
            if (on_periodic_face(L, i, j, k)) write_images(L, r, i, j, k, out);
        }
    }
}

// Residual r = f - sum_l opr(l) v(nbr) on the interior, periodic images
// written (bbmg_class.f90:831-844).  With f == nullptr the kernel returns the
// operator product itself.
template <typename T, int NPT>
__device__ __forceinline__ void residual_point(const Lay &L, const int *__restrict__ off0,
                                               const int *__restrict__ off1, const T *__restrict__ opr,
                                               const T *__restrict__ v, const T *__restrict__ f,
                                               T *__restrict__ r, int i, int j, int k) {
    using O = Ops<T, ExactOf<T>::value>;
    const int par = i & 1;
    const long long id = L.idx(i, j, k);
    T s = T(0);
#pragma unroll
    for (int q = 0; q < Lay7<NPT>::terms; q++) {
        const int q27i = Lay7<NPT>::slot(q);
        const int o = par ? off1[q27i] : off0[q27i];
        s = O::mac(s, opr[(long long)Lay7<NPT>::plane(q) * L.plane + id + (Lay7<NPT>::at_nbr(q) ? o : 0)], v[id + o]);
    }
    const T val = f ? O::sub(f[id], s) : s;
    r[id] = val;
    if (on_periodic_face(L, i, j, k)) write_images(L, r, i, j, k, val);
}

template <typename T, int NPT>
__global__ void __launch_bounds__(256) k_residual(Lay L, NbrOff nb, const T *__restrict__ opr,
                                                   const T *__restrict__ v, const T *__restrict__ f,
                                                   T *__restrict__ r) {
    pdl_entry();
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) residual_point<T, NPT>(L, nb.off[0], nb.off[1], opr, v, f, r, x_of(L, ch), j, k);
    }
}

// Residual of the FP32 symmetric 7-point level (planes D, E, N, T) with its
// operands staged in shared memory: one warp per (j,k) row; the 24 segments
// (both x-halves of D, E, N, T, f, v of the row, N and v of row j-1, v of row
// j+1, T and v of plane k-1, v of plane k+1) are copied with 16-byte cp.async,
// each from 4 elements before the half-row to 4 after it, so the i-1 / i+1
// neighbours (other half, overlap included) are on chip.  Same terms in the
// same order as residual_point: identical bits.
template <typename T>
__global__ void __launch_bounds__(128) k_residual_staged(Lay L, const T *__restrict__ opr,
                                                          const T *__restrict__ v, const T *__restrict__ f,
                                                          T *__restrict__ r, int na) {
    pdl_entry();
    extern __shared__ __align__(16) unsigned char smraw[];
    T *smf = reinterpret_cast<T *>(smraw);
    using O = Ops<T, ExactOf<T>::value>;
    constexpr int EPC = 16 / sizeof(T);  // elements per 16-byte copy
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = na + 8;
    T *S = smf + (size_t)warp * 24 * seg;
    const long long P = L.plane;
    const int nrows = L.ny * L.nz;
    for (int row = blockIdx.x * 4 + warp; row < nrows; row += gridDim.x * 4) {
        const int j = row % L.ny, k = row / L.ny;
        const long long r0 = L.G + L.row(j, k) * L.P;
        const long long rjm = L.G + L.row(j - 1, k) * L.P, rjp = L.G + L.row(j + 1, k) * L.P;
        const long long rkm = L.G + L.row(j, k - 1) * L.P, rkp = L.G + L.row(j, k + 1) * L.P;
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; h++) {  // h = 0: odd-x half (offset 0), h = 1: even-x half (offset B0)
            const long long hb = (h ? L.B0 : 0) - 4;
            const T *src[12] = {opr + r0 + hb,         opr + P + r0 + hb,     opr + 2 * P + r0 + hb,
                                    opr + 3 * P + r0 + hb, f + r0 + hb,           v + r0 + hb,
                                    opr + 2 * P + rjm + hb, v + rjm + hb,         v + rjp + hb,
                                    opr + 3 * P + rkm + hb, v + rkm + hb,         v + rkp + hb};
#pragma unroll
            for (int q = 0; q < 12; q++)
                for (int e = lane * EPC; e < seg; e += 32 * EPC) cp16(S + (h * 12 + q) * seg + e, src[q] + e);
        }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        __syncwarp();
        // segment q of half h at S[(12 h + q) seg + 4 + position]
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const T *Sh = S + h * 12 * seg + 4, *So = S + (1 - h) * 12 * seg + 4;
            // x-neighbours in the other half: odd point a (i = 2a+1) has i-1 at even a, i+1 at even a+1;
            // even point a (i = 2a) has i-1 at odd a-1, i+1 at odd a
            const int om = h ? -1 : 0, op = h ? 0 : 1;
            for (int a = lane; a < na; a += 32) {  // lane-strided: conflict-free shared loads
                T sum = T(0);
                sum = O::mac(sum, Sh[9 * seg + a], Sh[10 * seg + a]);          // B: T(k-1) v(k-1)
                sum = O::mac(sum, Sh[6 * seg + a], Sh[7 * seg + a]);           // S: N(j-1) v(j-1)
                sum = O::mac(sum, So[1 * seg + a + om], So[5 * seg + a + om]); // W: E(i-1) v(i-1)
                sum = O::mac(sum, Sh[0 * seg + a], Sh[5 * seg + a]);           // C: D v
                sum = O::mac(sum, Sh[1 * seg + a], So[5 * seg + a + op]);      // E: E(i) v(i+1)
                sum = O::mac(sum, Sh[2 * seg + a], Sh[8 * seg + a]);           // N: N(i) v(j+1)
                sum = O::mac(sum, Sh[3 * seg + a], Sh[11 * seg + a]);          // T: T(i) v(k+1)
                const T out = O::sub(Sh[4 * seg + a], sum);
                r[r0 + (h ? L.B0 : 0) + a] = out;
                const int i = h ? 2 * a : 2 * a + 1;
                if (on_periodic_face(L, i, j, k)) write_images(L, r, i, j, k, out);
            }
        }
    }
}

// Asynchronous global -> shared copy of 4, 8 or 16 bytes.
template <int BYTES>
__device__ __forceinline__ void cpa(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(BYTES) : "memory");
}

template <typename T>
struct MarchVec;
template <> struct MarchVec<float> { using V = float4; static constexpr int W = 4; };
template <> struct MarchVec<double> { using V = double2; static constexpr int W = 2; };

// VW consecutive shared-memory values, 16-byte aligned, as one vector load
template <typename T, int VW>
__device__ __forceinline__ void ldvec(T *dst, const T *src) {
    using V = typename MarchVec<T>::V;
    const V x = *reinterpret_cast<const V *>(src);
    if constexpr (VW == 4) {
        dst[0] = x.x; dst[1] = x.y; dst[2] = x.z; dst[3] = x.w;
    } else {
        dst[0] = x.x; dst[1] = x.y;
    }
}

// Residual of the symmetric 7-point level (planes D, E, N, T) by marching up
// the k columns.  A block owns TY consecutive (j) rows, both x-halves, of a
// chunk of k-planes; each thread owns VW = 16/sizeof(T) consecutive positions
// of one half-row.  Plane by plane, a three-slot ring of shared-memory stages
// is filled with cp.async one plane ahead of the computation: stage(k) holds
// D, E, N, T and f of plane k on the block's rows, N on row j0-1, and v of
// plane k+1 on rows j0-1 .. j0+TY (each half-row with its overlap positions -1
// and na).  The residual of plane k reads stage(k) and stage(k-1) (v of plane
// k and T of plane k-1), and v(k-1) from a register.  Every array is read from
// HBM once per block apart from the two halo rows and one extra plane per
// chunk: ~31 B per cell against the algorithm's 28.  Terms and order are
// residual_point's (B, S, W, C, E, N, T): the same bits.  Requires an even
// nx, na = nx/2 a multiple of VW and TH = na/VW in [4, 128]; the block of
// 2*TH*TY threads holds TY = floor(128/TH) rows.
template <typename T>
__global__ void __launch_bounds__(256) k_residual_march(Lay L, const T *__restrict__ opr, const T *__restrict__ v,
                                                         const T *__restrict__ f, T *__restrict__ r, int na,
                                                         int kchunk) {
    pdl_launch();
    using O = Ops<T, ExactOf<T>::value>;
    constexpr int VW = MarchVec<T>::W;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *sm = reinterpret_cast<T *>(smraw);
    const int TH = na / VW, TY = blockDim.x / (2 * TH);
    const int seg = na + 8;                  // position p of a half-row at index p + 4
    const int rows = 5 * TY + 1 + TY + 2;    // C[5][TY], NH, VT[TY+2]
    const int SS = rows * 2 * seg;           // elements per stage
    const int tid = threadIdx.x, c = tid % TH, h = (tid / TH) & 1, jj = tid / (2 * TH);
    const int j0 = blockIdx.x * TY, j = j0 + jj;
    const bool valid = j < L.ny;
    const int k0 = blockIdx.y * kchunk, k1 = min(L.nz, k0 + kchunk);
    if (k0 >= k1) return;  // uniform over the block
    const long long P = L.plane, hb = h ? L.B0 : 0;
    const int pos = c * VW;
    const int jt = min(j0 + TY, L.ny);  // row after the block's last valid row
    const bool lo_edge = h == 0 && c == 0, hi_edge = h == 1 && c == TH - 1;
    const int ovl = h == 0 ? -1 : na;   // overlap position of this half
    auto goff = [&](int jr, int kr) { return L.G + L.row(jr, kr) * L.P + hb; };
    // row `rr` of stage slot `sl`, this thread's half (hh = h) or the other
    auto srow = [&](int sl, int rr, int hh) { return sm + (size_t)sl * SS + (rr * 2 + hh) * seg + 4; };
    const int RC = 0, RNH = 5 * TY, RVT = 5 * TY + 1;  // first rows of C, NH, VT
    if (valid) {  // the first two stages' operator rows into L2 while the predecessor finishes
#pragma unroll
        for (int kp = k0 - 1; kp <= k0; kp++)
#pragma unroll
            for (int q = 0; q < 4; q++) pf_l2(opr + q * P + goff(j, kp) + pos);
    }
    pdl_wait();
    auto fill = [&](int sl, int kp) {
        if (valid) {
            const long long g = goff(j, kp) + pos;
#pragma unroll
            for (int q = 0; q < 4; q++) cpa<16>(srow(sl, RC + q * TY + jj, h) + pos, opr + q * P + g);
            cpa<16>(srow(sl, RC + 4 * TY + jj, h) + pos, f + g);
            cpa<16>(srow(sl, RVT + jj + 1, h) + pos, v + goff(j, kp + 1) + pos);
            if (lo_edge) cpa<sizeof(T)>(srow(sl, RC + TY + jj, 0) - 1, opr + P + goff(j, kp) - 1);
            if (lo_edge || hi_edge) cpa<sizeof(T)>(srow(sl, RVT + jj + 1, h) + ovl, v + goff(j, kp + 1) + ovl);
        }
        if (jj == 0) {  // row j0-1 (always a stored row: overlap or interior)
            cpa<16>(srow(sl, RNH, h) + pos, opr + 2 * P + goff(j0 - 1, kp) + pos);
            cpa<16>(srow(sl, RVT, h) + pos, v + goff(j0 - 1, kp + 1) + pos);
            if (lo_edge || hi_edge) cpa<sizeof(T)>(srow(sl, RVT, h) + ovl, v + goff(j0 - 1, kp + 1) + ovl);
        }
        if (jj == TY - 1) {
            cpa<16>(srow(sl, RVT + jt - j0 + 1, h) + pos, v + goff(jt, kp + 1) + pos);
            if (lo_edge || hi_edge)
                cpa<sizeof(T)>(srow(sl, RVT + jt - j0 + 1, h) + ovl, v + goff(jt, kp + 1) + ovl);
        }
    };
    auto commit = []() { asm volatile("cp.async.commit_group;" ::: "memory"); };
    T vm[VW];  // v(k-1) at the thread's positions
    if (valid) {
#pragma unroll
        for (int q = 0; q < VW; q++) vm[q] = v[goff(j, k0 - 1) + pos + q];
    }
    // stage(k) lives in slot (k - k0 + 1) % 3
    fill(0, k0 - 1);
    commit();
    fill(1, k0);
    commit();
    for (int k = k0; k < k1; k++) {
        const int sp = (k - k0) % 3, sc = (k - k0 + 1) % 3, sn = (k - k0 + 2) % 3;
        __syncthreads();  // slot sn (stage k-2) is no longer read
        if (k + 1 < k1) fill(sn, k + 1);
        commit();
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();  // stage k complete for every thread
        if (valid) {
            const int rs = 2 * seg;
            const T *Cc = srow(sc, RC, h);
            const T *Dk = Cc + (0 * TY + jj) * rs, *Ek = Cc + (1 * TY + jj) * rs;
            const T *Nk = Cc + (2 * TY + jj) * rs, *Tk = Cc + (3 * TY + jj) * rs, *Fk = Cc + (4 * TY + jj) * rs;
            const T *Eo = srow(sc, RC + TY + jj, 1 - h);                                // E(k), other half
            const T *Ns = jj ? srow(sc, RC + 2 * TY + jj - 1, h) : srow(sc, RNH, h);    // N(j-1, k)
            const T *Tm = srow(sp, RC + 3 * TY + jj, h);                                // T(k-1)
            const T *vS = srow(sp, RVT + jj, h), *vN = srow(sp, RVT + jj + 2, h);       // v(j-1,k), v(j+1,k)
            const T *vC = srow(sp, RVT + jj + 1, h), *vO = srow(sp, RVT + jj + 1, 1 - h);  // v(k): own, other half
            const T *vP = srow(sc, RVT + jj + 1, h);                                    // v(k+1)
            // vector reads of the thread's VW positions (conflict-free); the
            // other half's v and E also one position either side
            T tm[VW], ns[VW], vs[VW], dk[VW], vc[VW], ek[VW], nk[VW], vn[VW], tk[VW], vp[VW], fk[VW];
            T vo[VW + 2], eo[VW + 1];
            ldvec<T, VW>(tm, Tm + pos); ldvec<T, VW>(ns, Ns + pos); ldvec<T, VW>(vs, vS + pos);
            ldvec<T, VW>(dk, Dk + pos); ldvec<T, VW>(vc, vC + pos); ldvec<T, VW>(ek, Ek + pos);
            ldvec<T, VW>(nk, Nk + pos); ldvec<T, VW>(vn, vN + pos); ldvec<T, VW>(tk, Tk + pos);
            ldvec<T, VW>(vp, vP + pos); ldvec<T, VW>(fk, Fk + pos);
            ldvec<T, VW>(vo + 1, vO + pos); vo[0] = vO[pos - 1]; vo[VW + 1] = vO[pos + VW];
            ldvec<T, VW>(eo + 1, Eo + pos); eo[0] = Eo[pos - 1];
            T res[VW];
#pragma unroll
            for (int q = 0; q < VW; q++) {
                T s = T(0);
                s = O::mac(s, tm[q], vm[q]);                          // B: T(k-1) v(k-1)
                s = O::mac(s, ns[q], vs[q]);                          // S: N(j-1) v(j-1)
                // odd point (h = 0): i-1 at the other half's position a, i+1 at a+1;
                // even point (h = 1): i-1 at a-1, i+1 at a
                const T wcoef = h ? eo[q] : eo[q + 1], wval = h ? vo[q] : vo[q + 1];
                const T eval = h ? vo[q + 1] : vo[q + 2];
                s = O::mac(s, wcoef, wval);                           // W: E(i-1) v(i-1)
                s = O::mac(s, dk[q], vc[q]);                          // C: D v
                s = O::mac(s, ek[q], eval);                           // E: E(i) v(i+1)
                s = O::mac(s, nk[q], vn[q]);                          // N: N(i) v(j+1)
                s = O::mac(s, tk[q], vp[q]);                          // T: T(i) v(k+1)
                res[q] = O::sub(fk[q], s);
            }
            T *dst = r + goff(j, k) + pos;
            if constexpr (VW == 4)
                *reinterpret_cast<float4 *>(dst) = make_float4(res[0], res[1], res[2], res[3]);
            else
                *reinterpret_cast<double2 *>(dst) = make_double2(res[0], res[1]);
            if (L.xper || L.yper || L.zper) {
#pragma unroll
                for (int q = 0; q < VW; q++) {
                    const int i = h ? 2 * (pos + q) : 2 * (pos + q) + 1;
                    if (on_periodic_face(L, i, j, k)) write_images(L, r, i, j, k, res[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < VW; q++) vm[q] = vc[q];
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Restriction f_c = sum_r f2c(r) r_f(2c + r) (bbmg_class.f90:805-827), with
// f2c(r) = c2f((1-r)/2, 2c+r) (bbmg_class.f90:1218-1222) read straight from the
// fine prolongation weights.  Also zeroes the coarse correction v_c, the first
// statement of cycle(n+1) (bbmg_class.f90:739).
template <typename T>
__device__ __forceinline__ void restrict_point(const Lay &F, const Lay &C, const T *__restrict__ c2f,
                                               const T *__restrict__ rF, T *__restrict__ fC, T *__restrict__ vC,
                                               int ci, int cj, int ck) {
    using O = Ops<T, ExactOf<T>::value>;
    const int fi = 2 * ci, fj = 2 * cj, fk = 2 * ck;
    const int rk0 = -pmod(F.zper, fk - 1, F.nz), rk1 = pmod(F.zper, fk + 1, F.nz);
    const int rj0 = -pmod(F.yper, fj - 1, F.ny), rj1 = pmod(F.yper, fj + 1, F.ny);
    const int ri0 = -pmod(F.xper, fi - 1, F.nx), ri1 = pmod(F.xper, fi + 1, F.nx);
    // all 27 offsets unrolled, the ones outside [r0, r1] predicated off: the
    // loads issue together, the terms enter the sum in the same order
    T s = T(0);
#pragma unroll
    for (int rk = -1; rk <= 1; rk++)
#pragma unroll
        for (int rj = -1; rj <= 1; rj++)
#pragma unroll
            for (int ri = -1; ri <= 1; ri++) {
                if (rk < rk0 || rk > rk1 || rj < rj0 || rj > rj1 || ri < ri0 || ri > ri1) continue;
                const long long fid = F.idx(fi + ri, fj + rj, fk + rk);
                s = O::mac(s, c2f[(long long)q8((1 - ri) / 2, (1 - rj) / 2, (1 - rk) / 2) * F.plane + fid], rF[fid]);
            }
    const long long cid = C.idx(ci, cj, ck);
    fC[cid] = s;
    vC[cid] = T(0);
    if (on_periodic_face(C, ci, cj, ck)) {
        write_images(C, fC, ci, cj, ck, s);
        write_images(C, vC, ci, cj, ck, T(0));
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_restrict(Lay F, Lay C, const T *__restrict__ c2f,
                                                   const T *__restrict__ rF, T *__restrict__ fC,
                                                   T *__restrict__ vC) {
    pdl_entry();
    FOR_ROWS(C.ny * C.nz) {
        const int cj = row % C.ny, ck = row / C.ny;
        FOR_CHUNKS(C.nx) restrict_point<T>(F, C, c2f, rF, fC, vC, x_of(C, ch), cj, ck);
    }
}

// Prolongation and correction v_f += sum_p c2f(p) v_c((i+1)/2 + p)
// (bbmg_class.f90:779-801 then 770).  A fine point of parity class
// (n1,n2,n3) only carries weights p_d <= n_d.
template <typename T>
__device__ __forceinline__ void prolong_point(const Lay &F, const Lay &C, const T *__restrict__ c2f,
                                              const T *__restrict__ vC, T *__restrict__ vF, int i, int j, int k) {
    using O = Ops<T, ExactOf<T>::value>;
    const int n1 = i & 1, n2 = j & 1, n3 = k & 1, ci = i >> 1, cj = j >> 1, ck = k >> 1;
    const long long id = F.idx(i, j, k);
    T e = T(0);
#pragma unroll
    for (int pk = 0; pk <= 1; pk++)
#pragma unroll
        for (int pj = 0; pj <= 1; pj++)
#pragma unroll
            for (int pi = 0; pi <= 1; pi++) {
                if (pk > n3 || pj > n2 || pi > n1) continue;  // predicated: same terms, same order
                e = O::mac(e, c2f[(long long)q8(pi, pj, pk) * F.plane + id], vC[C.idx(ci + pi, cj + pj, ck + pk)]);
            }
    const T val = O::add(vF[id], e);
    vF[id] = val;
    if (on_periodic_face(F, i, j, k)) write_images(F, vF, i, j, k, val);
}

template <typename T>
__global__ void __launch_bounds__(256) k_prolong(Lay F, Lay C, const T *__restrict__ c2f,
                                                  const T *__restrict__ vC, T *__restrict__ vF) {
    pdl_entry();
    FOR_ROWS(F.ny * F.nz) {
        const int j = row % F.ny, k = row / F.ny;
        FOR_CHUNKS(F.nx) prolong_point<T>(F, C, c2f, vC, vF, x_of(F, ch), j, k);
    }
}

// Restriction of an FP32 level with an even x size into the next coarser one,
// operands staged in shared memory: one warp per coarse (cj,ck) row.  For each
// of the 9 fine rows (2cj+rj, 2ck+rk) it copies both x-halves of r_f and the
// three weight planes a coarse point reads there (even half: q8(0,pj,pk) for
// ri = 0; odd half: q8(0,pj,pk) for ri = +1 and q8(1,pj,pk) for ri = -1,
// pj = (1-rj)/2, pk = (1-rk)/2), each from 4 elements before the half-row to
// 4 after it.  Same terms in the same order as restrict_point.
template <typename T>
__global__ void __launch_bounds__(128) k_restrict_staged(Lay F, Lay C, const T *__restrict__ c2f,
                                                          const T *__restrict__ rF, T *__restrict__ fC,
                                                          T *__restrict__ vC, int na, int np) {
    pdl_launch();
    extern __shared__ __align__(16) unsigned char smraw[];
    T *smf = reinterpret_cast<T *>(smraw);
    using O = Ops<T, ExactOf<T>::value>;
    constexpr int EPC = 16 / sizeof(T);  // elements per 16-byte copy
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // a job is one of the np equal parts of a coarse row (np = 2 halves the
    // shared memory per warp, so twice the warps fit on an SM)
    const int nh = na / np, seg = nh + 8;
    T *S = smf + (size_t)warp * 45 * seg;
    const long long P = F.plane;
    const int nrows = C.ny * C.nz * np;
    // the weight segments of job `row` (written only by the setup)
    auto copy_w = [&](int row) {
        const int h0 = (row % np) * nh;
        row /= np;
        const int fj = 2 * (row % C.ny), fk = 2 * (row / C.ny);
        for (int rk = -1; rk <= 1; rk++)
            for (int rj = -1; rj <= 1; rj++) {
                const int b = 5 * ((rk + 1) * 3 + (rj + 1));
                const int pj = (1 - rj) / 2, pk = (1 - rk) / 2;
                const long long fr = F.G + F.row(fj + rj, fk + rk) * F.P - 4 + h0;
                for (int e = lane * EPC; e < seg; e += 32 * EPC) {
                    cp16(S + (b + 2) * seg + e, c2f + q8(0, pj, pk) * P + fr + F.B0 + e);  // ri = 0
                    cp16(S + (b + 3) * seg + e, c2f + q8(0, pj, pk) * P + fr + e);         // ri = +1
                    cp16(S + (b + 4) * seg + e, c2f + q8(1, pj, pk) * P + fr + e);         // ri = -1
                }
            }
    };
    int row = blockIdx.x * 4 + warp;
    if (row < nrows) copy_w(row);  // before the wait for the predecessor
    pdl_wait();
    for (bool first = true; row < nrows; row += gridDim.x * 4, first = false) {
        const int h0 = (row % np) * nh, crow = row / np;
        const int cj = crow % C.ny, ck = crow / C.ny;
        const int fj = 2 * cj, fk = 2 * ck;
        const int rk0 = -pmod(F.zper, fk - 1, F.nz), rk1 = pmod(F.zper, fk + 1, F.nz);
        const int rj0 = -pmod(F.yper, fj - 1, F.ny), rj1 = pmod(F.yper, fj + 1, F.ny);
        __syncwarp();
        if (!first) copy_w(row);
        for (int rk = -1; rk <= 1; rk++)
            for (int rj = -1; rj <= 1; rj++) {
                const int b = 5 * ((rk + 1) * 3 + (rj + 1));
                const long long fr = F.G + F.row(fj + rj, fk + rk) * F.P - 4 + h0;
                for (int e = lane * EPC; e < seg; e += 32 * EPC) {
                    cp16(S + (b + 0) * seg + e, rF + fr + e);         // r odd half
                    cp16(S + (b + 1) * seg + e, rF + fr + F.B0 + e);  // r even half
                }
            }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        __syncwarp();
        for (int c0 = lane; c0 < nh; c0 += 32) {  // lane-strided coarse points of the part
            {
                const int ci = h0 + c0;
                const int fi = 2 * ci;
                const int ri0 = -pmod(F.xper, fi - 1, F.nx), ri1 = pmod(F.xper, fi + 1, F.nx);
                T sum = T(0);
#pragma unroll
                for (int rk = -1; rk <= 1; rk++)
#pragma unroll
                    for (int rj = -1; rj <= 1; rj++)
#pragma unroll
                        for (int ri = -1; ri <= 1; ri++) {
                            if (rk < rk0 || rk > rk1 || rj < rj0 || rj > rj1 || ri < ri0 || ri > ri1) continue;
                            const T *Sb = S + 5 * ((rk + 1) * 3 + (rj + 1)) * seg + 4;
                            // fi = 2ci: even position ci; fi+1: odd ci; fi-1: odd ci-1
                            // (segment index relative to the part's start h0)
                            const T w = ri == 0 ? Sb[2 * seg + c0] : (ri > 0 ? Sb[3 * seg + c0] : Sb[4 * seg + c0 - 1]);
                            const T rv = ri == 0 ? Sb[seg + c0] : (ri > 0 ? Sb[c0] : Sb[c0 - 1]);
                            sum = O::mac(sum, w, rv);
                        }
                const long long cid = C.idx(ci, cj, ck);
                fC[cid] = sum;
                vC[cid] = T(0);
                if (on_periodic_face(C, ci, cj, ck)) {
                    write_images(C, fC, ci, cj, ck, sum);
                    write_images(C, vC, ci, cj, ck, T(0));
                }
            }
        }
    }
}

// Prolongation + correction of an FP32 level with an even x size, operands
// staged in shared memory: one warp per fine (j,k) row.  It copies both x-halves
// of v_f, the weight planes the row's parity class uses (q8(pi,pj,pk) with
// pj <= j&1, pk <= k&1; the even half only needs pi = 0) and both x-halves of
// the (up to four) coarse rows it interpolates from, then applies
// prolong_point's sum term for term.  Requires na = nx/2 (the coarse x size)
// to be a multiple of 8, so every copied segment is 16-byte aligned.
template <typename T>
__global__ void __launch_bounds__(128) k_prolong_staged(Lay F, Lay C, const T *__restrict__ c2f,
                                                         const T *__restrict__ vC, T *__restrict__ vF,
                                                         int na) {
    pdl_launch();
    extern __shared__ __align__(16) unsigned char smraw[];
    T *smf = reinterpret_cast<T *>(smraw);
    using O = Ops<T, ExactOf<T>::value>;
    constexpr int EPC = 16 / sizeof(T);  // elements per 16-byte copy
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = na + 8;
    T *S = smf + (size_t)warp * 22 * seg;
    // segments: 0,1 v_f odd/even half; 2 + 3*(pj+2pk) + {0: even pi=0, 1: odd pi=0, 2: odd pi=1};
    // 14 + 2*(pj+2pk) + {0: coarse odd half, 1: coarse even half}
    const long long P = F.plane;
    const int nrows = F.ny * F.nz;
    // the weight planes of fine row `row` (written only by the setup)
    auto copy_w = [&](int row) {
        const int j = row % F.ny, k = row / F.ny;
        const long long r0 = F.G + F.row(j, k) * F.P;
        for (int pk = 0; pk <= (k & 1); pk++)
            for (int pj = 0; pj <= (j & 1); pj++) {
                const int b = 2 + 3 * (pj + 2 * pk);
                for (int e = lane * EPC; e < na; e += 32 * EPC) {
                    cp16(S + b * seg + e, c2f + q8(0, pj, pk) * P + r0 + F.B0 + e);
                    cp16(S + (b + 1) * seg + e, c2f + q8(0, pj, pk) * P + r0 + e);
                    cp16(S + (b + 2) * seg + e, c2f + q8(1, pj, pk) * P + r0 + e);
                }
            }
    };
    int row = blockIdx.x * 4 + warp;
    if (row < nrows) copy_w(row);  // before the wait for the predecessor
    pdl_wait();
    for (bool first = true; row < nrows; row += gridDim.x * 4, first = false) {
        const int j = row % F.ny, k = row / F.ny;
        const int n2 = j & 1, n3 = k & 1, cj = j >> 1, ck = k >> 1;
        const long long r0 = F.G + F.row(j, k) * F.P;
        __syncwarp();
        if (!first) copy_w(row);
        for (int e = lane * EPC; e < na; e += 32 * EPC) {
            cp16(S + e, vF + r0 + e);
            cp16(S + seg + e, vF + r0 + F.B0 + e);
        }
        for (int pk = 0; pk <= n3; pk++)
            for (int pj = 0; pj <= n2; pj++) {
                const long long cr = C.G + C.row(cj + pj, ck + pk) * C.P;
                // coarse odd half: positions < C.nx/2; even half: <= C.nx/2 (overlap
                // included); both copied up to the next multiple of 4 above C.nx/2
                const int cb = 14 + 2 * (pj + 2 * pk), ccl = ((C.nx >> 1) + 4) & ~3;
                for (int e = lane * EPC; e < ccl; e += 32 * EPC) {
                    cp16(S + cb * seg + e, vC + cr + e);
                    cp16(S + (cb + 1) * seg + e, vC + cr + C.B0 + e);
                }
            }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; h++) {  // h = 0: odd-x fine points (n1 = 1), h = 1: even-x (n1 = 0)
            const int n1 = 1 - h;
            for (int a = lane; a < na; a += 32) {  // lane-strided: conflict-free shared loads
                const int i = h ? 2 * a : 2 * a + 1, ci = i >> 1;
                T ev = T(0);
#pragma unroll
                for (int pk = 0; pk <= 1; pk++)
#pragma unroll
                    for (int pj = 0; pj <= 1; pj++)
#pragma unroll
                        for (int pi = 0; pi <= 1; pi++) {
                            if (pk > n3 || pj > n2 || pi > n1) continue;
                            const int b = 2 + 3 * (pj + 2 * pk) + (h ? 0 : 1 + pi);
                            const int cx = ci + pi, cb = 14 + 2 * (pj + 2 * pk);
                            // coarse x-split: odd cx at odd-half position (cx-1)/2, even at even-half cx/2
                            const T vc = (cx & 1) ? S[cb * seg + ((cx - 1) >> 1)] : S[(cb + 1) * seg + (cx >> 1)];
                            ev = O::mac(ev, S[b * seg + a], vc);
                        }
                const T out = O::add(S[h * seg + a], ev);
                vF[r0 + (h ? F.B0 : 0) + a] = out;
                if (on_periodic_face(F, i, j, k)) write_images(F, vF, i, j, k, out);
            }
        }
    }
}

// Coarsest level: gather f in lexicographic order, solve with the stored LU
// (FP64 always), scatter into v (bbmg_class.f90:891-927).  One block; the
// triangular solves run on one warp with the factors in shared memory when
// they fit.
template <typename T>
__device__ __forceinline__ void coarse_solve_block(const Lay &L, const double *__restrict__ LU,
                                                   const int *__restrict__ piv, const int *__restrict__ pinned,
                                                   const T *__restrict__ f, T *__restrict__ v, int mat_in_smem,
                                                   double *sm) {
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

template <typename T>
__global__ void k_coarse_solve(Lay L, const double *__restrict__ LU, const int *__restrict__ piv,
                               const int *__restrict__ pinned, const T *__restrict__ f, T *__restrict__ v,
                               int mat_in_smem) {
    pdl_entry();
    extern __shared__ double sm[];
    coarse_solve_block<T>(L, LU, piv, pinned, f, v, mat_in_smem, sm);
}

// ---------------------------------------------------------------------------
// Deterministic reductions: a fixed grid per level, a fixed tree per block.
template <int MODE>  // 0 = max with NaN propagation, 1 = sum
__device__ __forceinline__ double block_reduce(double v, double *sh) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    sh[tid] = v;
    __syncthreads();
    for (int s = nt / 2; s > 0; s >>= 1) {
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
__device__ __forceinline__ bool block_leader() { return threadIdx.x == 0 && threadIdx.y == 0; }
__device__ __forceinline__ int block_id() { return blockIdx.y * gridDim.x + blockIdx.x; }
__device__ __forceinline__ double max_nan(double m, double a) { return (a != a || m != m) ? (a + m) : fmax(m, a); }

template <typename T>
__global__ void __launch_bounds__(256) k_maxabs_part(Lay L, const T *__restrict__ x, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    double m = 0.0;
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) m = max_nan(m, fabs((double)x[L.idx(x_of(L, ch), j, k)]));
    }
    m = block_reduce<0>(m, sh);
    if (block_leader()) part[block_id()] = m;
}

template <typename TA, typename TB>
__global__ void __launch_bounds__(256) k_dot_part(Lay L, const TA *__restrict__ a, const TB *__restrict__ b,
                                                   double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    double s = 0.0;
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) {
            const long long id = L.idx(x_of(L, ch), j, k);
            s = __dadd_rn(s, __dmul_rn((double)a[id], (double)b[id]));
        }
    }
    s = block_reduce<1>(s, sh);
    if (block_leader()) part[block_id()] = s;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_final(const double *__restrict__ part, int n, double *__restrict__ out) {
    pdl_entry();
    __shared__ double sh[256];
    double v = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        double a = part[t];
        v = MODE == 0 ? max_nan(v, a) : v + a;
    }
    v = block_reduce<MODE>(v, sh);
    if (threadIdx.x == 0) *out = v;
}

// ---------------------------------------------------------------------------
// caller arrays (Fortran, g overlap layers) <-> level interior
template <typename T>
__global__ void __launch_bounds__(256) k_from_caller(Lay L, const double *__restrict__ src, int g, T *__restrict__ dst) {
    pdl_entry();
    const long long sy = L.nx + 2 * g, sz = sy * (L.ny + 2 * g);
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) {
            const int i = ch;  // natural order: coalesced reads of the caller's row
            const T val = (T)src[(k + g) * sz + (j + g) * sy + (i + g)];
            dst[L.idx(i, j, k)] = val;
            if (on_periodic_face(L, i, j, k)) write_images(L, dst, i, j, k, val);
        }
    }
}

__global__ void __launch_bounds__(256) k_to_caller(Lay L, const double *__restrict__ src, int g, double *__restrict__ dst) {
    pdl_entry();
    const long long sy = L.nx + 2 * g, sz = sy * (L.ny + 2 * g);
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) {
            const int i = ch;
            dst[(k + g) * sz + (j + g) * sy + (i + g)] = src[L.idx(i, j, k)];
        }
    }
}

__global__ void __launch_bounds__(256) k_to_f32(const double *__restrict__ src, float *__restrict__ dst, long long n) {
    pdl_entry();
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        dst[t] = (float)src[t];
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

// Flexible CG, FCG(1) (Notay, SIAM J. Sci. Comput. 22 (2000) 1444-1460): the
// preconditioner may change from one iteration to the next (a learned first
// stage followed by the V-cycle, or the V-cycle alone), so the new direction
// is A-orthogonalised against the previous one explicitly:
// p = z - (z.Ap_old / p_old.Ap_old) p_old, i.e. beta = -z.Ap_old / pap_old,
// instead of the recurrence beta = rho/rho_old of bbmg_class.f90:666-672.
// With a fixed SPD preconditioner both give the same directions in exact
// arithmetic.  alpha = z.r / p.Ap is unchanged (r is orthogonal to p_old).
//
// k_fcg_z: z = z1 + e (z1 the first stage's output, absent when the stage is
// off; e the V-cycle correction of z1's residual) on the own cell with its
// periodic images, and the block partials of z.res (part[0..nb)) and
// z.Ap_old (part[nb..2nb)).
__global__ void __launch_bounds__(256) k_fcg_z(Lay L, const double *__restrict__ z1, const float *__restrict__ e,
                                                const double *__restrict__ res, const double *__restrict__ Ap,
                                                double *__restrict__ zz, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    double a = 0.0, b = 0.0;
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) {
            const int i = x_of(L, ch);
            const long long id = L.idx(i, j, k);
            const double z = z1 ? __dadd_rn(z1[id], (double)e[id]) : (double)e[id];
            zz[id] = z;
            if (on_periodic_face(L, i, j, k)) write_images(L, zz, i, j, k, z);
            a = __dadd_rn(a, __dmul_rn(z, res[id]));
            b = __dadd_rn(b, __dmul_rn(z, Ap[id]));
        }
    }
    a = block_reduce<1>(a, sh);
    b = block_reduce<1>(b, sh);
    if (block_leader()) {
        part[block_id()] = a;
        part[gridDim.x * gridDim.y + block_id()] = b;
    }
}
// rho = z.res, beta = -z.Ap_old / pap_old (0 at the first iteration)
__global__ void k_fcg_scal(const double *__restrict__ part, int n, CgScal *sc) {
    pdl_entry();
    __shared__ double sh[256];
    double a = 0.0, b = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        a = a + part[t];
        b = b + part[n + t];
    }
    a = block_reduce<1>(a, sh);
    b = block_reduce<1>(b, sh);
    if (threadIdx.x == 0) {
        sc->rho2 = sc->rho1;
        sc->rho1 = a;
        sc->iter += 1;
        sc->beta = sc->iter == 1 ? 0.0 : -__ddiv_rn(b, sc->pap);
    }
}

// pp_new = zz + beta*pp_old on the own cell (with images) and Ap = A pp_new,
// the neighbours' pp_new formed on the fly from zz and pp_old (bit-identical
// to the stored value), plus the block partial of pp_new.Ap
// (bbmg_class.f90:674-687 in one pass).  pp_old and pp_new are distinct.
template <typename TZ, int NPT>
__global__ void __launch_bounds__(256) k_cg_pap_fused(Lay L, NbrOff nb, const double *__restrict__ opr,
                                                       const TZ *__restrict__ zz, const double *__restrict__ pp_old,
                                                       double *__restrict__ pp_new, double *__restrict__ Ap,
                                                       const CgScal *__restrict__ sc, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    const double beta = sc->beta;
    double acc = 0.0;
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) {
            const int i = x_of(L, ch);
            const int par = i & 1;
            const long long id = L.idx(i, j, k);
            double s = 0.0, pc = 0.0;
#pragma unroll
            for (int q = 0; q < Lay7<NPT>::terms; q++) {
                const int q27i = Lay7<NPT>::slot(q);
                const int o = par ? nb.off[1][q27i] : nb.off[0][q27i];
                const double pq = __dadd_rn((double)zz[id + o], __dmul_rn(beta, pp_old[id + o]));
                if (q == Lay7<NPT>::centre) pc = pq;
                s = __dadd_rn(s, __dmul_rn(opr[(long long)Lay7<NPT>::plane(q) * L.plane + id +
                                               (Lay7<NPT>::at_nbr(q) ? o : 0)],
                                           pq));
            }
            pp_new[id] = pc;
            if (on_periodic_face(L, i, j, k)) write_images(L, pp_new, i, j, k, pc);
            Ap[id] = s;
            acc = __dadd_rn(acc, __dmul_rn(pc, s));
        }
    }
    acc = block_reduce<1>(acc, sh);
    if (block_leader()) part[block_id()] = acc;
}

// pp_new = zz + beta*pp_old and Ap = A pp_new with the block partial of
// pp_new . Ap, for the symmetric 7-point level-1 operator, by k-column
// marching (the structure of k_residual_march): a block of 2*TH*TY <= NT
// threads owns TY = floor(NT/(2 TH)) rows (both halves) of a chunk of
// k-planes, a thread VW = 2 consecutive positions of one half-row (TH = nx/4).
// A three-slot ring of cp.async stages, filled two planes ahead, holds for
// plane k D, E, N, T on the block's rows and N on row j0-1, and zz and pp_old
// of plane k+1 on rows j0-1 .. j0+TY with the overlap positions; from those
// the block forms the direction p of plane k+1 in a two-slot shared ring.
// Ap(k) reads p(k-1) and T(k-1) from registers, p(k) and p(k+1) from the
// ring.  Each point's arithmetic is k_cg_pap_fused's, so pp_new and Ap are
// the same bits; the partial sums group the products differently.
template <typename TZ, int NT>
__global__ void __launch_bounds__(NT) k_cg_pap_march(Lay L, const double *__restrict__ opr,
                                                      const TZ *__restrict__ zz, const double *__restrict__ pp_old,
                                                      double *__restrict__ pp_new, double *__restrict__ Ap,
                                                      const CgScal *__restrict__ sc, double *__restrict__ part,
                                                      int na, int kchunk) {
    pdl_launch();
    __shared__ double red[NT];
    extern __shared__ __align__(16) unsigned char smraw[];
    using O = Ops<double, true>;
    constexpr int VW = 2;
    const int TH = na / VW, TY = blockDim.x / (2 * TH);
    const int seg = na + 8;  // position p of a half-row at index p + 4
    const int rowsO = 4 * TY + 1, rowsV = TY + 2;
    const size_t bO = (size_t)rowsO * 2 * seg * sizeof(double), bZ = (size_t)rowsV * 2 * seg * sizeof(TZ);
    const size_t bP = (size_t)rowsV * 2 * seg * sizeof(double), bS = bO + bZ + bP;
    auto sO = [&](int sl, int rr, int hh) {
        return reinterpret_cast<double *>(smraw + sl * bS) + (rr * 2 + hh) * seg + 4;
    };
    auto sZ = [&](int sl, int rr, int hh) {
        return reinterpret_cast<TZ *>(smraw + sl * bS + bO) + (rr * 2 + hh) * seg + 4;
    };
    auto sP = [&](int sl, int rr, int hh) {
        return reinterpret_cast<double *>(smraw + sl * bS + bO + bZ) + (rr * 2 + hh) * seg + 4;
    };
    auto pR = [&](int sl, int rr, int hh) {
        return reinterpret_cast<double *>(smraw + 3 * bS + sl * bP) + (rr * 2 + hh) * seg + 4;
    };
    const int tid = threadIdx.x, c = tid % TH, h = (tid / TH) & 1, jj = tid / (2 * TH);
    const int j0 = blockIdx.x * TY, j = j0 + jj;
    const bool valid = j < L.ny;
    const int k0 = blockIdx.y * kchunk, k1 = min(L.nz, k0 + kchunk);
    const long long P = L.plane, hb = h ? L.B0 : 0;
    const int pos = c * VW;
    const int jt = min(j0 + TY, L.ny);
    const bool lo_edge = h == 0 && c == 0, hi_edge = h == 1 && c == TH - 1, edge = lo_edge || hi_edge;
    const int ovl = h == 0 ? -1 : na;
    auto goff = [&](int jr, int kr) { return L.G + L.row(jr, kr) * L.P + hb; };
    if (valid && k0 < k1) {  // the first stages' operator rows into L2 while the predecessor finishes
#pragma unroll
        for (int kp = k0 - 1; kp <= k0 + 1; kp++)
#pragma unroll
            for (int q = 0; q < 4; q++) pf_l2(opr + q * P + goff(j, kp) + pos);
    }
    pdl_wait();
    const double beta = sc->beta;  // written by the predecessor: after the wait
    auto commit = []() { asm volatile("cp.async.commit_group;" ::: "memory"); };
    // zz and pp_old of plane kp on row jr into tile row rr of slot sl
    auto fill_v = [&](int sl, int rr, int jr, int kp) {
        const long long g = goff(jr, kp);
        cpa<VW * sizeof(TZ)>(sZ(sl, rr, h) + pos, zz + g + pos);
        cpa<16>(sP(sl, rr, h) + pos, pp_old + g + pos);
        if (edge) {
            cpa<sizeof(TZ)>(sZ(sl, rr, h) + ovl, zz + g + ovl);
            cpa<8>(sP(sl, rr, h) + ovl, pp_old + g + ovl);
        }
    };
    auto fill = [&](int sl, int kp) {
        if (valid) {
            const long long g = goff(j, kp) + pos;
#pragma unroll
            for (int q = 0; q < 4; q++) cpa<16>(sO(sl, q * TY + jj, h) + pos, opr + q * P + g);
            if (lo_edge) cpa<8>(sO(sl, TY + jj, 0) - 1, opr + P + goff(j, kp) - 1);
            fill_v(sl, jj + 1, j, kp + 1);
        }
        if (jj == 0) {
            cpa<16>(sO(sl, 4 * TY, h) + pos, opr + 2 * P + goff(j0 - 1, kp) + pos);
            fill_v(sl, 0, j0 - 1, kp + 1);
        }
        if (jj == TY - 1) fill_v(sl, jt - j0 + 1, jt, kp + 1);
    };
    // p = zz + beta*pp_old for the tile positions this thread copied
    auto make_p_row = [&](int sl, int slot, int rr) {
        const TZ *z = sZ(sl, rr, h);
        const double *po = sP(sl, rr, h);
        double *pr = pR(slot, rr, h);
#pragma unroll
        for (int q = 0; q < VW; q++) pr[pos + q] = __dadd_rn((double)z[pos + q], __dmul_rn(beta, po[pos + q]));
        if (edge) pr[ovl] = __dadd_rn((double)z[ovl], __dmul_rn(beta, po[ovl]));
    };
    auto make_p = [&](int sl, int slot) {
        if (valid) make_p_row(sl, slot, jj + 1);
        if (jj == 0) make_p_row(sl, slot, 0);
        if (jj == TY - 1) make_p_row(sl, slot, jt - j0 + 1);
    };
    double acc = 0.0;
    if (k0 < k1) {
        double pm[VW] = {0.0, 0.0}, tm[VW] = {0.0, 0.0};
        if (valid) {
            const long long g = goff(j, k0 - 1) + pos;
#pragma unroll
            for (int q = 0; q < VW; q++) {
                pm[q] = __dadd_rn((double)zz[g + q], __dmul_rn(beta, pp_old[g + q]));
                tm[q] = opr[3 * P + g + q];
            }
        }
        // stage(k) lives in slot (k - k0 + 1) % 3, the direction of plane k in ring slot k & 1;
        // stages run two planes ahead of the computation
        fill(0, k0 - 1);
        commit();
        fill(1, k0);
        commit();
        if (k0 + 1 < k1) fill(2, k0 + 1);
        commit();
        asm volatile("cp.async.wait_group 2;" ::: "memory");
        __syncthreads();
        make_p(0, k0 & 1);
        for (int k = k0; k < k1; k++) {
            const int scur = (k - k0 + 1) % 3, sfree = (k - k0) % 3;
            __syncthreads();  // stage(k-1) and p(k-1) are no longer read
            if (k + 2 < k1) fill(sfree, k + 2);
            commit();
            asm volatile("cp.async.wait_group 2;" ::: "memory");
            __syncthreads();  // stage(k) complete for every thread
            make_p(scur, (k + 1) & 1);
            __syncthreads();  // p(k+1) complete
            if (valid) {
                double dk[VW], ek[VW], nk[VW], tk[VW], ns[VW], pc[VW], ps[VW], pn[VW], pp[VW];
                double po[VW + 2], eo[VW + 1];
                ldvec<double, VW>(dk, sO(scur, jj, h) + pos);
                ldvec<double, VW>(ek, sO(scur, TY + jj, h) + pos);
                ldvec<double, VW>(nk, sO(scur, 2 * TY + jj, h) + pos);
                ldvec<double, VW>(tk, sO(scur, 3 * TY + jj, h) + pos);
                ldvec<double, VW>(ns, (jj ? sO(scur, 2 * TY + jj - 1, h) : sO(scur, 4 * TY, h)) + pos);
                const double *Eo = sO(scur, TY + jj, 1 - h);
                ldvec<double, VW>(eo + 1, Eo + pos);
                eo[0] = Eo[pos - 1];
                ldvec<double, VW>(pc, pR(k & 1, jj + 1, h) + pos);
                ldvec<double, VW>(ps, pR(k & 1, jj, h) + pos);
                ldvec<double, VW>(pn, pR(k & 1, jj + 2, h) + pos);
                ldvec<double, VW>(pp, pR((k + 1) & 1, jj + 1, h) + pos);
                const double *Po = pR(k & 1, jj + 1, 1 - h);
                ldvec<double, VW>(po + 1, Po + pos);
                po[0] = Po[pos - 1];
                po[VW + 1] = Po[pos + VW];
                double out[VW];
#pragma unroll
                for (int q = 0; q < VW; q++) {
                    const double wcoef = h ? eo[q] : eo[q + 1], wval = h ? po[q] : po[q + 1];
                    const double eval = h ? po[q + 1] : po[q + 2];
                    double s = 0.0;
                    s = O::mac(s, tm[q], pm[q]);   // B
                    s = O::mac(s, ns[q], ps[q]);   // S
                    s = O::mac(s, wcoef, wval);    // W
                    s = O::mac(s, dk[q], pc[q]);   // C
                    s = O::mac(s, ek[q], eval);    // E
                    s = O::mac(s, nk[q], pn[q]);   // N
                    s = O::mac(s, tk[q], pp[q]);   // T
                    out[q] = s;
                    acc = __dadd_rn(acc, __dmul_rn(pc[q], s));
                }
                const long long g = goff(j, k) + pos;
                *reinterpret_cast<double2 *>(pp_new + g) = make_double2(pc[0], pc[1]);
                *reinterpret_cast<double2 *>(Ap + g) = make_double2(out[0], out[1]);
                if (L.xper || L.yper || L.zper) {
#pragma unroll
                    for (int q = 0; q < VW; q++) {
                        const int i = h ? 2 * (pos + q) : 2 * (pos + q) + 1;
                        if (on_periodic_face(L, i, j, k)) write_images(L, pp_new, i, j, k, pc[q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < VW; q++) {
                    tm[q] = tk[q];
                    pm[q] = pc[q];
                }
            }
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    // block partial (fixed tree over NT slots; threads beyond the block add 0)
    red[tid] = acc;
    for (int t2 = blockDim.x + tid; t2 < NT; t2 += blockDim.x) red[t2] = 0.0;
    __syncthreads();
    for (int s2 = NT / 2; s2 > 0; s2 >>= 1) {
        if (tid < s2) red[tid] = red[tid] + red[tid + s2];
        __syncthreads();
    }
    if (tid == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = red[0];
}

// Streaming kernels over the interior two positions at a time (16-byte
// double2 accesses): thread t takes chunk t % CH of half-row (t / CH) % 2 of
// row t / (2 CH), CH = nx/4, grid-stride over a fixed grid, so consecutive
// threads touch consecutive 16-byte words and every block's partial is
// accumulated in a fixed order.  Requires nx a multiple of 4.
template <typename T>
struct Pair;
template <> struct Pair<double> { using V = double2; };
template <> struct Pair<float> { using V = float2; };

__device__ __forceinline__ long long pair_base(const Lay &L, long long t, int CH, int &j, int &k, int &hh, int &c) {
    c = (int)(t % CH);
    const long long r2 = t / CH;
    hh = (int)(r2 & 1);
    const long long row = r2 >> 1;
    j = (int)(row % L.ny);
    k = (int)(row / L.ny);
    return L.G + L.row(j, k) * L.P + (hh ? L.B0 : 0) + 2 * c;
}

// block partials of sum a*b (the CG's rho = r . z, bbmg_class.f90:662)
template <typename TA>
__global__ void __launch_bounds__(256) k_dot2_part(Lay L, const TA *__restrict__ a, const double *__restrict__ b,
                                                    double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    const int CH = L.nx >> 2;
    const long long total = (long long)L.ny * L.nz * 2 * CH;
    double s = 0.0;
    const long long st = gstride();
    // four chunks' loads in flight per thread; the sum still runs in chunk order
    for (long long t0 = gtid(); t0 < total; t0 += 4 * st) {
        typename Pair<TA>::V x[4];
        double2 y[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const long long t = t0 + u * st;
            if (t < total) {
                int j, k, hh, c;
                const long long e = pair_base(L, t, CH, j, k, hh, c);
                x[u] = *reinterpret_cast<const typename Pair<TA>::V *>(a + e);
                y[u] = *reinterpret_cast<const double2 *>(b + e);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (t0 + u * st < total) {
                s = __dadd_rn(s, __dmul_rn((double)x[u].x, y[u].x));
                s = __dadd_rn(s, __dmul_rn((double)x[u].y, y[u].y));
            }
        }
    }
    s = block_reduce<1>(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// The flexible CG's two dots in one pass, two positions at a time: block
// partials of a.b (rho = z.res) into part[0..nb) and of a.c (z.Ap_old) into
// part[nb..2nb), the sums in k_dot2_part's order.
template <typename TA>
__global__ void __launch_bounds__(256) k_dot2_flex_part(Lay L, const TA *__restrict__ a, const double *__restrict__ b,
                                                         const double *__restrict__ c, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    const int CH = L.nx >> 2;
    const long long total = (long long)L.ny * L.nz * 2 * CH;
    double s = 0.0, t2 = 0.0;
    const long long st = gstride();
    for (long long t0 = gtid(); t0 < total; t0 += 4 * st) {
        typename Pair<TA>::V x[4];
        double2 y[4], z[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const long long t = t0 + u * st;
            if (t < total) {
                int j, k, hh, cc;
                const long long e = pair_base(L, t, CH, j, k, hh, cc);
                x[u] = *reinterpret_cast<const typename Pair<TA>::V *>(a + e);
                y[u] = *reinterpret_cast<const double2 *>(b + e);
                z[u] = *reinterpret_cast<const double2 *>(c + e);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (t0 + u * st < total) {
                s = __dadd_rn(s, __dmul_rn((double)x[u].x, y[u].x));
                s = __dadd_rn(s, __dmul_rn((double)x[u].y, y[u].y));
                t2 = __dadd_rn(t2, __dmul_rn((double)x[u].x, z[u].x));
                t2 = __dadd_rn(t2, __dmul_rn((double)x[u].y, z[u].y));
            }
        }
    }
    s = block_reduce<1>(s, sh);
    t2 = block_reduce<1>(t2, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
        part[gridDim.x + blockIdx.x] = t2;
    }
}
// the same for any nx, one cell per thread
template <typename TA>
__global__ void __launch_bounds__(256) k_dot_flex_part(Lay L, const TA *__restrict__ a, const double *__restrict__ b,
                                                        const double *__restrict__ c, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    double s = 0.0, t2 = 0.0;
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) {
            const long long id = L.idx(x_of(L, ch), j, k);
            s = __dadd_rn(s, __dmul_rn((double)a[id], b[id]));
            t2 = __dadd_rn(t2, __dmul_rn((double)a[id], c[id]));
        }
    }
    s = block_reduce<1>(s, sh);
    t2 = block_reduce<1>(t2, sh);
    if (block_leader()) {
        part[block_id()] = s;
        part[gridDim.x * gridDim.y + block_id()] = t2;
    }
}

// k_cg_xr_fused two positions at a time (same per-point arithmetic)
template <typename TV>
__global__ void __launch_bounds__(256) k_cg_xr2(Lay L, double *__restrict__ sol, const double *__restrict__ pp,
                                                 double *__restrict__ res, const double *__restrict__ Ap,
                                                 const CgScal *__restrict__ sc, float *__restrict__ f32,
                                                 TV *__restrict__ vzero, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    const double alpha = sc->alpha;
    const int CH = L.nx >> 2;
    const long long total = (long long)L.ny * L.nz * 2 * CH;
    const bool per = L.xper || L.yper || L.zper;
    double m = 0.0;
    for (long long t = gtid(); t < total; t += gstride()) {
        int j, k, hh, c;
        const long long e = pair_base(L, t, CH, j, k, hh, c);
        double2 x = *reinterpret_cast<const double2 *>(sol + e);
        const double2 p = *reinterpret_cast<const double2 *>(pp + e);
        double2 r = *reinterpret_cast<const double2 *>(res + e);
        const double2 a = *reinterpret_cast<const double2 *>(Ap + e);
        x.x = __dadd_rn(x.x, __dmul_rn(alpha, p.x));
        x.y = __dadd_rn(x.y, __dmul_rn(alpha, p.y));
        r.x = __dsub_rn(r.x, __dmul_rn(alpha, a.x));
        r.y = __dsub_rn(r.y, __dmul_rn(alpha, a.y));
        *reinterpret_cast<double2 *>(sol + e) = x;
        *reinterpret_cast<double2 *>(res + e) = r;
        m = max_nan(m, fabs(r.x));
        m = max_nan(m, fabs(r.y));
        if (f32) *reinterpret_cast<float2 *>(f32 + e) = make_float2((float)r.x, (float)r.y);
        typename Pair<TV>::V z;
        z.x = TV(0);
        z.y = TV(0);
        *reinterpret_cast<typename Pair<TV>::V *>(vzero + e) = z;
        if (per) {
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int i = hh ? 2 * (2 * c + q) : 2 * (2 * c + q) + 1;
                if (on_periodic_face(L, i, j, k)) write_images(L, vzero, i, j, k, TV(0));
            }
        }
    }
    m = block_reduce<0>(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

static unsigned pair_grid(const Lay &L) {
    const long long total = (long long)L.ny * L.nz * 2 * (L.nx >> 2);
    long long b = (total + 255) / 256;
    if (b > kRedBlocks) b = kRedBlocks;
    return (unsigned)(b < 1 ? 1 : b);
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
    double m = 0.0;
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) {
            const int i = x_of(L, ch);
            const long long id = L.idx(i, j, k);
            sol[id] = __dadd_rn(sol[id], __dmul_rn(alpha, pp[id]));
            const double r = __dsub_rn(res[id], __dmul_rn(alpha, Ap[id]));
            res[id] = r;
            m = max_nan(m, fabs(r));
            if (f32) f32[id] = (float)r;
            vzero[id] = TV(0);
            if (on_periodic_face(L, i, j, k)) write_images(L, vzero, i, j, k, TV(0));
        }
    }
    m = block_reduce<0>(m, sh);
    if (block_leader()) part[block_id()] = m;
}

// mixed precision: FP64 residual -> FP32 right-hand side of the V-cycle
__global__ void __launch_bounds__(256) k_round_f32(Lay L, const double *__restrict__ r, float *__restrict__ f) {
    pdl_entry();
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) {
            const long long id = L.idx(x_of(L, ch), j, k);
            f[id] = (float)r[id];
        }
    }
}

// Mixed-precision defect correction step (the FP64 half of an mgsolve
// iteration, bbmg_class.f90:716-722 with the correction of 770): x_new = x + e
// on the own cell (images written), r = b - A (x + e) with the neighbours'
// x + e formed on the fly; r becomes the FP32 right-hand side of the next
// V-cycle and the block partial of max|r| is written.  x_old and x_new are
// distinct buffers; e is only read (its neighbours are needed by other
// threads), so it is zeroed for the next V-cycle by a separate memset.
template <int NPT>
__global__ void __launch_bounds__(256) k_defect_fused(Lay L, NbrOff nb, const double *__restrict__ opr,
                                                       const double *__restrict__ x_old, const float *__restrict__ e,
                                                       const double *__restrict__ b, double *__restrict__ x_new,
                                                       float *__restrict__ f32, double *__restrict__ part) {
    pdl_entry();
    __shared__ double sh[256];
    double m = 0.0;
    FOR_ROWS(L.ny * L.nz) {
        const int j = row % L.ny, k = row / L.ny;
        FOR_CHUNKS(L.nx) {
            const int i = x_of(L, ch);
            const int par = i & 1;
            const long long id = L.idx(i, j, k);
            double s = 0.0, xc = 0.0;
#pragma unroll
            for (int q = 0; q < Lay7<NPT>::terms; q++) {
                const int q27i = Lay7<NPT>::slot(q);
                const int o = par ? nb.off[1][q27i] : nb.off[0][q27i];
                const double xq = x_old[id + o] + (double)e[id + o];
                if (q == Lay7<NPT>::centre) xc = xq;
                s = fma(opr[(long long)Lay7<NPT>::plane(q) * L.plane + id + (Lay7<NPT>::at_nbr(q) ? o : 0)], xq, s);
            }
            const double r = b[id] - s;
            x_new[id] = xc;
            f32[id] = (float)r;
            if (on_periodic_face(L, i, j, k)) write_images(L, x_new, i, j, k, xc);
            m = max_nan(m, fabs(r));
        }
    }
    m = block_reduce<0>(m, sh);
    if (block_leader()) part[block_id()] = m;
}

// ---------------------------------------------------------------------------
// launchers
template <typename T> static int vw_for(int n);
template <> int vw_for<float>(int n) { return (n % 4 == 0) ? 4 : ((n % 2 == 0) ? 2 : 1); }
template <> int vw_for<double>(int n) { return (n % 2 == 0) ? 2 : 1; }
template <typename T> struct VwMax { static constexpr int value = sizeof(T) == 4 ? 4 : 2; };

// the shared-memory-staged FP32 kernels (27-point colours, level-1 residual,
// restriction, prolongation)
// serve levels whose half-rows hold a multiple of 4 points (nx even), unless
// BBMG_NO_STAGED is set (then the register kernels run: same bits)
static bool use_staged(const Lay &L) {
    static const bool off = getenv("BBMG_NO_STAGED") != nullptr;
    return !off && !(L.nx & 1) && (L.nx >> 1) % 4 == 0;
}

// k-chunks for a k-marching kernel over `jtiles` row tiles: the count in
// [1, min(nz, 16)] that maximises the fill of the resident slots (waves of
// SMs x blocks per SM) times kc/(kc+1) for chunks of kc planes (each chunk
// reads one plane more); the smallest among near-ties; 0 if no block fits.
static int march_chunks(const void *kern, int nt, size_t smem, int jtiles, int nz) {
    int oc = 0, nsm = 148, dev = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oc, kern, nt, smem) != cudaSuccess || oc < 1) return 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long slots = (long long)nsm * oc;
    int best = 1;
    double beff = 0.0;
    for (int n = 1; n <= nz && n <= 16; n++) {
        const long long tot = (long long)jtiles * n, waves = (tot + slots - 1) / slots;
        const int kc = (nz + n - 1) / n;
        const double eff = (double)tot / (double)(waves * slots) * kc / (kc + 1.0);
        if (eff > beff + 0.01) {
            beff = eff;
            best = n;
        }
    }
    return best;
}

template <typename T, int NPT>
static cudaError_t launch_colour(const Lay &L, const Off27 &off, const T *opr, T *v, const T *f, int px, int py,
                                 int pz, int fuse, cudaStream_t s) {
    const int na = (L.nx - px + 1) >> 1;
    if constexpr (NPT == 27) {
        const size_t smem = sizeof(T) * 46 * (size_t)(na + 8) * 4;
        if (use_staged(L) && smem <= 200 * 1024) {
            static bool attr = false;
            if (!attr && smem > 48 * 1024) {
                cudaError_t e = cudaFuncSetAttribute(k_relax27_staged<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     200 * 1024);
                if (e != cudaSuccess) return e;
                attr = true;
            }
            const long long nrows = (long long)((L.ny - py + 1) >> 1) * ((L.nz - pz + 1) >> 1);
            long long gx = (nrows + 3) / 4;
            if (gx > 148LL * 8) gx = 148LL * 8;
            BB_CHECK_LAUNCH((launch_k(k_relax27_staged<T>, dim3((unsigned)gx), dim3(128), smem, s, L, opr, v, f, px,
                                      py, pz, fuse, na)));
            return cudaSuccess;
        }
    }
    const long long nrows = (long long)((L.ny - py + 1) >> 1) * ((L.nz - pz + 1) >> 1);
    const int vw = vw_for<T>(na);
    const Geo g = geo_rows(na / vw, nrows);
    if (vw == VwMax<T>::value)
        BB_CHECK_LAUNCH((launch_k(k_relax<T, NPT, VwMax<T>::value>, g.grid, g.block, 0, s, L, off, opr, v, f, px, py, pz, fuse)));
    else if (vw == 2)
        BB_CHECK_LAUNCH((launch_k(k_relax<T, NPT, 2>, g.grid, g.block, 0, s, L, off, opr, v, f, px, py, pz, fuse)));
    else
        BB_CHECK_LAUNCH((launch_k(k_relax<T, NPT, 1>, g.grid, g.block, 0, s, L, off, opr, v, f, px, py, pz, fuse)));
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_relax(const Lay &L, const NbrOff &nb, int npt, bool fuse, const T *opr, T *v, const T *f, int dir,
                         cudaStream_t s, bool skip_first) {
    const bool per = L.xper || L.yper || L.zper;
    for (int c = skip_first ? 1 : 0; c < 8; c++) {
        int col = dir > 0 ? c : 7 - c;  // colours 1..8 forward, 8..1 backward
        int px = col & 1, py = (col >> 1) & 1, pz = (col >> 2) & 1;
        long long n = (long long)((L.nx - px + 1) >> 1) * ((L.ny - py + 1) >> 1) * ((L.nz - pz + 1) >> 1);
        if (n == 0) continue;
        Off27 off = off_for(nb, px);
        cudaError_t e;
        if (npt == 4) e = launch_colour<T, 4>(L, off, opr, v, f, px, py, pz, fuse ? 1 : 0, s);
        else if (npt == 7) e = launch_colour<T, 7>(L, off, opr, v, f, px, py, pz, fuse ? 1 : 0, s);
        else e = launch_colour<T, 27>(L, off, opr, v, f, px, py, pz, fuse ? 1 : 0, s);
        if (e != cudaSuccess) return e;
        if (per && !fuse) {
            e = wrap_planes(L, v, 1, s);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

static PhaseCols phase_cols(const Lay &L, const NbrOff &nb, int w, int vw_cap, int &vw, long long &rows,
                            int &chunks) {
    PhaseCols p{};
    p.n = 0;
    p.off[0] = off_for(nb, 0);
    p.off[1] = off_for(nb, 1);
    vw = vw_cap;
    rows = 0;
    int na_max = 0;
    for (int col = 0; col < 8; col++) {
        if (__builtin_popcount(col) != w) continue;
        int px = col & 1, py = (col >> 1) & 1, pz = (col >> 2) & 1;
        int na = (L.nx - px + 1) >> 1;
        long long nr = (long long)((L.ny - py + 1) >> 1) * ((L.nz - pz + 1) >> 1);
        if (na == 0 || nr == 0) continue;
        p.col[p.n++] = col;
        while (vw > 1 && na % vw) vw >>= 1;
        if (nr > rows) rows = nr;
        if (na > na_max) na_max = na;
    }
    chunks = na_max / vw;
    return p;
}


// Block order of the colour phases (bits as in k_relax_phase7; BBMG_PHASE_ORD
// overrides).  Default 15: alternate launches walk the rows in opposite
// directions, so a phase starts on the rows whose lines the previous phase
// left in L2; colours interleaved; centre coefficient and f evict-first;
// operator lines prefetched before the wait.  Measured at 256^3 (FP32 level-1
// sweep): 0.174 ms in the plain order, 0.162 with bits 0-2; bit 3 adds 1.3 %
// to the whole solve (37.6 -> 38.1 solves/s).
static int phase_order_env() {
    static int o = -1;
    if (o < 0) {
        const char *e = getenv("BBMG_PHASE_ORD");
        o = e ? (atoi(e) & 15) : 15;
    }
    return o;
}

template <typename T, int NPT>
static cudaError_t launch_phase(const Lay &L, const PhaseCols &pc, int vw, long long rows, int chunks, const T *opr,
                                T *v, const T *f, int ord, cudaStream_t s) {
    Geo g = geo_rows(chunks, rows, 148LL * 24 / (pc.n > 0 ? pc.n : 1));
    g.grid.z = pc.n;
    if (vw == VwMax<T>::value)
        BB_CHECK_LAUNCH((launch_k(k_relax_phase7<T, NPT, VwMax<T>::value>, g.grid, g.block, 0, s, L, opr, v, f, pc, 1, ord)));
    else if (vw == 2)
        BB_CHECK_LAUNCH((launch_k(k_relax_phase7<T, NPT, 2>, g.grid, g.block, 0, s, L, opr, v, f, pc, 1, ord)));
    else
        BB_CHECK_LAUNCH((launch_k(k_relax_phase7<T, NPT, 1>, g.grid, g.block, 0, s, L, opr, v, f, pc, 1, ord)));
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_relax_sweeps(const Lay &L, const NbrOff &nb, int npt, bool fuse, const T *opr, T *v, const T *f,
                                int first_dir, int nsweeps, cudaStream_t s) {
    if (npt == 27 || !fuse) {
        int dir = first_dir;
        for (int i = 0; i < nsweeps; i++) {
            // the first colour of a sweep after the opposite sweep is the colour
            // that sweep ended with: the reference's update (rhs minus the
            // neighbours' sum, over the centre) reads only the other colours,
            // so recomputing it gives the same bits and is skipped
            cudaError_t e = launch_relax<T>(L, nb, npt, fuse, opr, v, f, dir, s, i > 0);
            if (e != cudaSuccess) return e;
            dir = -dir;
        }
        return cudaSuccess;
    }
    int dir = first_dir, last = -1, nl = 0;
    const int oenv = phase_order_env();
    for (int i = 0; i < nsweeps; i++) {
        for (int p = 0; p < 4; p++) {
            int w = dir > 0 ? p : 3 - p;
            if (w == last) continue;  // identical recomputation
            last = w;
            int vw, chunks;
            long long rows;
            PhaseCols pc = phase_cols(L, nb, w, VwMax<T>::value, vw, rows, chunks);
            if (pc.n == 0) continue;
            // bit 0 of the setting: every other launch walks the rows backwards
            const int ord = (oenv & ~1) | ((oenv & 1) & nl++);
            cudaError_t e = npt == 4 ? launch_phase<T, 4>(L, pc, vw, rows, chunks, opr, v, f, ord, s)
                                     : launch_phase<T, 7>(L, pc, vw, rows, chunks, opr, v, f, ord, s);
            if (e != cudaSuccess) return e;
        }
        dir = -dir;
    }
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_residual(const Lay &L, const NbrOff &nb, int npt, const T *opr, const T *v, const T *f, T *r,
                            cudaStream_t s) {
    const int na = L.nx >> 1;
    // symmetric 7-point level: column marching (both precisions, same bits as
    // the register kernel)
    if (f && npt == 4 && use_staged(L)) {
        constexpr int VW = MarchVec<T>::W;
        const int TH = na / VW;
        if (!(L.nx & 1) && na % VW == 0 && TH >= 4 && TH <= 128) {
            const int TY = 128 / TH, seg = na + 8, nthr = 2 * TH * TY;
            const size_t smem = sizeof(T) * (size_t)seg * 2 * (5 * TY + 1 + TY + 2) * 3;
            static bool attr[2] = {false, false};
            if (smem <= 200 * 1024 && !attr[sizeof(T) == 8]) {
                if (cudaFuncSetAttribute(k_residual_march<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) ==
                    cudaSuccess)
                    attr[sizeof(T) == 8] = true;
            }
            if (smem <= 200 * 1024 && attr[sizeof(T) == 8]) {
                const int jtiles = (L.ny + TY - 1) / TY;
                int nch = march_chunks((const void *)k_residual_march<T>, nthr, smem, jtiles, L.nz);
                if (nch < 1) nch = 1;
                const int kchunk = (L.nz + nch - 1) / nch;
                nch = (L.nz + kchunk - 1) / kchunk;
                BB_CHECK_LAUNCH((launch_k(k_residual_march<T>, dim3(jtiles, nch), dim3(nthr), smem, s, L, opr, v, f,
                                          r, na, kchunk)));
                return cudaSuccess;
            }
        }
    }
    // measured at 256^3: staged wins for 27-point levels in both precisions and
    // ties on the FP32 7-point level; the FP64 7-point segments need 104 KB of
    // shared memory per block (two blocks per SM) and lose to the register kernel
    if (f && use_staged(L) && (npt == 27 || (npt == 4 && sizeof(T) == 4))) {
        const int nseg = npt == 27 ? 46 : 24;
        const size_t smem = sizeof(T) * nseg * (size_t)(na + 8) * 4;
        auto kern = npt == 27 ? k_residual27_staged<T> : k_residual_staged<T>;
        if (smem <= 200 * 1024) {
            static bool attr[2] = {false, false};
            if (!attr[npt == 27] && smem > 48 * 1024) {
                cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
                if (e != cudaSuccess) return e;
                attr[npt == 27] = true;
            }
            const long long jobs = npt == 27 ? 2LL * L.ny * L.nz : (long long)L.ny * L.nz;
            long long gx = (jobs + 3) / 4;
            if (gx > 148LL * 16) gx = 148LL * 16;
            BB_CHECK_LAUNCH((launch_k(kern, dim3((unsigned)gx), dim3(128), smem, s, L, opr, v, f, r, na)));
            return cudaSuccess;
        }
    }
    const Geo g = geo_rows(L.nx, (long long)L.ny * L.nz);
    if (npt == 4) BB_CHECK_LAUNCH((launch_k(k_residual<T, 4>, g.grid, g.block, 0, s, L, nb, opr, v, f, r)));
    else if (npt == 7) BB_CHECK_LAUNCH((launch_k(k_residual<T, 7>, g.grid, g.block, 0, s, L, nb, opr, v, f, r)));
    else BB_CHECK_LAUNCH((launch_k(k_residual<T, 27>, g.grid, g.block, 0, s, L, nb, opr, v, f, r)));
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_restrict(const Lay &F, const Lay &C, const T *c2f, const T *rF, T *fC, T *vC, cudaStream_t s) {
    const int na = F.nx >> 1;
    // coarse rows of 128 or more points in two parts (16-byte aligned starts)
    const int np = (na >= 128 && na % 8 == 0) ? 2 : 1;
    const size_t smem = sizeof(T) * 45 * (size_t)(na / np + 8) * 4;
    // FP64 segments fill up to 196 KB per block (one block per SM): slower than
    // the register kernel at 256^3, so the staged restriction is FP32 only
    if (sizeof(T) == 4 && use_staged(F) && C.nx == na && smem <= 200 * 1024) {
        static bool attr = false;
        if (!attr && smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k_restrict_staged<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 200 * 1024);
            if (e != cudaSuccess) return e;
            attr = true;
        }
        long long gx = ((long long)C.ny * C.nz * np + 3) / 4;
        if (gx > 148LL * 16) gx = 148LL * 16;
        BB_CHECK_LAUNCH((launch_k(k_restrict_staged<T>, dim3((unsigned)gx), dim3(128), smem, s, F, C, c2f, rF, fC, vC,
                                  na, np)));
        return cudaSuccess;
    }
    const Geo g = geo_rows(C.nx, (long long)C.ny * C.nz);
    BB_CHECK_LAUNCH((launch_k(k_restrict<T>, g.grid, g.block, 0, s, F, C, c2f, rF, fC, vC)));
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_prolong(const Lay &F, const Lay &C, const T *c2f, const T *vC, T *vF, cudaStream_t s) {
    const int na = F.nx >> 1;
    const size_t smem = sizeof(T) * 22 * (size_t)(na + 8) * 4;
    // coarse half-rows (x size nx/2, overlap included) fit in na + 8 elements
    if (use_staged(F) && C.nx == na && (C.nx % 8) == 0 && smem <= 200 * 1024) {
        static bool attr = false;
        if (!attr && smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k_prolong_staged<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 200 * 1024);
            if (e != cudaSuccess) return e;
            attr = true;
        }
        long long gx = ((long long)F.ny * F.nz + 3) / 4;
        if (gx > 148LL * 16) gx = 148LL * 16;
        BB_CHECK_LAUNCH((launch_k(k_prolong_staged<T>, dim3((unsigned)gx), dim3(128), smem, s, F, C, c2f, vC, vF, na)));
        return cudaSuccess;
    }
    const Geo g = geo_rows(F.nx, (long long)F.ny * F.nz);
    BB_CHECK_LAUNCH((launch_k(k_prolong<T>, g.grid, g.block, 0, s, F, C, c2f, vC, vF)));
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_coarse_solve(const Lay &L, const double *LU, const int *piv, const int *pinned, const T *f, T *v,
                                cudaStream_t s) {
    int np = L.nx * L.ny * L.nz;
    size_t mat = (size_t)np * np * sizeof(double), vec = (size_t)np * sizeof(double);
    int in_smem = (mat + vec) <= kCoarseSmem;
    size_t shm = vec + (in_smem ? mat : 0);
    BB_CHECK_LAUNCH((launch_k(k_coarse_solve<T>, dim3(1), dim3(256), shm, s, L, LU, piv, pinned, f, v, in_smem)));
    return cudaSuccess;
}

cudaError_t coarse_solve_prepare() {
    cudaError_t e = cudaFuncSetAttribute(k_coarse_solve<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kCoarseSmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_coarse_solve<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmem);
}

template <typename T>
cudaError_t launch_maxabs(const Lay &L, const T *x, double *part, double *out, cudaStream_t s) {
    const Geo g = geo_red(L);
    BB_CHECK_LAUNCH((launch_k(k_maxabs_part<T>, g.grid, g.block, 0, s, L, x, part)));
    BB_CHECK_LAUNCH((launch_k(k_final<0>, dim3(1), dim3(256), 0, s, (const double *)part, (int)(g.grid.x * g.grid.y), out)));
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_dot(const Lay &L, const T *a, const T *b, double *part, double *out, cudaStream_t s) {
    const Geo g = geo_red(L);
    BB_CHECK_LAUNCH((launch_k(k_dot_part<T, T>, g.grid, g.block, 0, s, L, a, b, part)));
    BB_CHECK_LAUNCH((launch_k(k_final<1>, dim3(1), dim3(256), 0, s, (const double *)part, (int)(g.grid.x * g.grid.y), out)));
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_from_caller(const Lay &L, const double *src, int g, T *dst, cudaStream_t s) {
    const Geo gg = geo_rows(L.nx, (long long)L.ny * L.nz);
    BB_CHECK_LAUNCH((launch_k(k_from_caller<T>, gg.grid, gg.block, 0, s, L, src, g, dst)));
    return cudaSuccess;
}

cudaError_t launch_to_caller(const Lay &L, const double *src, int g, double *dst, cudaStream_t s) {
    const Geo gg = geo_rows(L.nx, (long long)L.ny * L.nz);
    BB_CHECK_LAUNCH((launch_k(k_to_caller, gg.grid, gg.block, 0, s, L, src, g, dst)));
    return cudaSuccess;
}

cudaError_t launch_to_f32(const double *src, float *dst, long long n, cudaStream_t s) {
    BB_CHECK_LAUNCH((launch_k(k_to_f32, dim3(grid_for(n, 256)), dim3(256), 0, s, src, dst, n)));
    return cudaSuccess;
}

template <typename TZ>
cudaError_t launch_cg_rho(const Lay &L, const TZ *zz, const double *res, double *part, CgScal *sc, cudaStream_t s) {
    if (use_staged(L)) {  // nx a multiple of 8: two positions per thread
        const unsigned nb2 = pair_grid(L);
        BB_CHECK_LAUNCH((launch_k(k_dot2_part<TZ>, dim3(nb2), dim3(256), 0, s, L, zz, res, part)));
        BB_CHECK_LAUNCH((launch_k(k_cg_rho, dim3(1), dim3(256), 0, s, (const double *)part, (int)nb2, sc)));
        return cudaSuccess;
    }
    const Geo g = geo_red(L);
    BB_CHECK_LAUNCH((launch_k(k_dot_part<TZ, double>, g.grid, g.block, 0, s, L, zz, res, part)));
    BB_CHECK_LAUNCH((launch_k(k_cg_rho, dim3(1), dim3(256), 0, s, (const double *)part, (int)(g.grid.x * g.grid.y), sc)));
    return cudaSuccess;
}

// flexible CG scalars: rho = zz.res and beta = -zz.Ap_old / pap_old
template <typename TZ>
cudaError_t launch_fcg_rho(const Lay &L, const TZ *zz, const double *res, const double *Ap, double *part, CgScal *sc,
                           cudaStream_t s) {
    if (use_staged(L)) {  // nx a multiple of 8: two positions per thread
        const unsigned nb2 = pair_grid(L);
        BB_CHECK_LAUNCH((launch_k(k_dot2_flex_part<TZ>, dim3(nb2), dim3(256), 0, s, L, zz, res, Ap, part)));
        BB_CHECK_LAUNCH((launch_k(k_fcg_scal, dim3(1), dim3(256), 0, s, (const double *)part, (int)nb2, sc)));
        return cudaSuccess;
    }
    const Geo g = geo_red(L);
    BB_CHECK_LAUNCH((launch_k(k_dot_flex_part<TZ>, g.grid, g.block, 0, s, L, zz, res, Ap, part)));
    BB_CHECK_LAUNCH((launch_k(k_fcg_scal, dim3(1), dim3(256), 0, s, (const double *)part, (int)(g.grid.x * g.grid.y), sc)));
    return cudaSuccess;
}

template <typename TZ>
cudaError_t launch_cg_pap_fused(const Lay &L, const NbrOff &nb, int npt, const double *opr, const TZ *zz,
                                const double *pp_old, double *pp_new, double *Ap, double *part, CgScal *sc,
                                cudaStream_t s) {
    const CgScal *csc = sc;
    if (npt == 4 && use_staged(L)) {
        // symmetric 7-point level: k-column marching
        const int na = L.nx >> 1, TH = na / 2;
        constexpr int NT = 512;
        if (!(L.nx & 1) && (na & 1) == 0 && TH >= 4 && 2 * TH <= NT) {
            const int TY = NT / (2 * TH), seg = na + 8, nthr = 2 * TH * TY;
            const size_t smem = (size_t)seg * 2 *
                                (3 * ((4 * TY + 1) * sizeof(double) + (TY + 2) * sizeof(TZ) + (TY + 2) * sizeof(double)) +
                                 2 * (TY + 2) * sizeof(double));
            constexpr size_t kMaxSmem = 220 * 1024;  // + 4 KB static: under the 227 KB a block may hold
            static bool attr = false;
            if (!attr && smem <= kMaxSmem &&
                cudaFuncSetAttribute(k_cg_pap_march<TZ, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem) ==
                    cudaSuccess)
                attr = true;
            if (attr && smem <= kMaxSmem) {
                const int jtiles = (L.ny + TY - 1) / TY;
                const int nch = march_chunks((const void *)k_cg_pap_march<TZ, NT>, nthr, smem, jtiles, L.nz);
                if (nch > 0 && jtiles * nch <= kRedBlocks) {
                    const int kchunk = (L.nz + nch - 1) / nch, nb2 = (L.nz + kchunk - 1) / kchunk;
                    BB_CHECK_LAUNCH((launch_k(k_cg_pap_march<TZ, NT>, dim3(jtiles, nb2), dim3(nthr), smem, s, L, opr, zz,
                                              pp_old, pp_new, Ap, csc, part, na, kchunk)));
                    BB_CHECK_LAUNCH((launch_k(k_cg_pap, dim3(1), dim3(256), 0, s, (const double *)part, jtiles * nb2, sc)));
                    return cudaSuccess;
                }
            }
        }
    }
    const Geo g = geo_red(L);
    if (npt == 4)
        BB_CHECK_LAUNCH((launch_k(k_cg_pap_fused<TZ, 4>, g.grid, g.block, 0, s, L, nb, opr, zz, pp_old, pp_new, Ap, csc, part)));
    else if (npt == 7)
        BB_CHECK_LAUNCH((launch_k(k_cg_pap_fused<TZ, 7>, g.grid, g.block, 0, s, L, nb, opr, zz, pp_old, pp_new, Ap, csc, part)));
    else
        BB_CHECK_LAUNCH((launch_k(k_cg_pap_fused<TZ, 27>, g.grid, g.block, 0, s, L, nb, opr, zz, pp_old, pp_new, Ap, csc, part)));
    BB_CHECK_LAUNCH((launch_k(k_cg_pap, dim3(1), dim3(256), 0, s, (const double *)part, (int)(g.grid.x * g.grid.y), sc)));
    return cudaSuccess;
}

template <typename TV>
cudaError_t launch_cg_xr_fused(const Lay &L, double *sol, const double *pp, double *res, const double *Ap,
                               const CgScal *sc, float *f32, TV *vzero, double *part, double *out, cudaStream_t s) {
    if (use_staged(L)) {  // nx a multiple of 8: two positions per thread
        const unsigned nb2 = pair_grid(L);
        BB_CHECK_LAUNCH((launch_k(k_cg_xr2<TV>, dim3(nb2), dim3(256), 0, s, L, sol, pp, res, Ap, sc, f32, vzero, part)));
        BB_CHECK_LAUNCH((launch_k(k_final<0>, dim3(1), dim3(256), 0, s, (const double *)part, (int)nb2, out)));
        return cudaSuccess;
    }
    const Geo g = geo_red(L);
    BB_CHECK_LAUNCH((launch_k(k_cg_xr_fused<TV>, g.grid, g.block, 0, s, L, sol, pp, res, Ap, sc, f32, vzero, part)));
    BB_CHECK_LAUNCH((launch_k(k_final<0>, dim3(1), dim3(256), 0, s, (const double *)part, (int)(g.grid.x * g.grid.y), out)));
    return cudaSuccess;
}

cudaError_t launch_fcg_z(const Lay &L, const double *z1, const float *e, const double *res, const double *Ap,
                         double *zz, double *part, CgScal *sc, cudaStream_t s) {
    const Geo g = geo_rows(L.nx, (long long)L.ny * L.nz, kRedBlocks / 2);  // 2 partials per block
    const int nb = (int)(g.grid.x * g.grid.y);
    BB_CHECK_LAUNCH((launch_k(k_fcg_z, g.grid, g.block, 0, s, L, z1, e, res, Ap, zz, part)));
    BB_CHECK_LAUNCH((launch_k(k_fcg_scal, dim3(1), dim3(256), 0, s, (const double *)part, nb, sc)));
    return cudaSuccess;
}

cudaError_t launch_round_f32(const Lay &L, const double *r, float *f, cudaStream_t s) {
    const Geo g = geo_rows(L.nx, (long long)L.ny * L.nz);
    BB_CHECK_LAUNCH((launch_k(k_round_f32, g.grid, g.block, 0, s, L, r, f)));
    return cudaSuccess;
}

cudaError_t launch_defect_fused(const Lay &L, const NbrOff &nb, int npt, const double *opr, const double *x_old,
                                const float *e, const double *b, double *x_new, float *f32, double *part,
                                double *out, cudaStream_t s) {
    const Geo g = geo_red(L);
    if (npt == 4)
        BB_CHECK_LAUNCH((launch_k(k_defect_fused<4>, g.grid, g.block, 0, s, L, nb, opr, x_old, e, b, x_new, f32, part)));
    else if (npt == 7)
        BB_CHECK_LAUNCH((launch_k(k_defect_fused<7>, g.grid, g.block, 0, s, L, nb, opr, x_old, e, b, x_new, f32, part)));
    else
        BB_CHECK_LAUNCH((launch_k(k_defect_fused<27>, g.grid, g.block, 0, s, L, nb, opr, x_old, e, b, x_new, f32, part)));
    BB_CHECK_LAUNCH((launch_k(k_final<0>, dim3(1), dim3(256), 0, s, (const double *)part, (int)(g.grid.x * g.grid.y), out)));
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// The coarse tail of the V-cycle in one launch.  On levels of at most a few
// hundred thousand cells a colour pass, residual, restriction or prolongation
// is a few microseconds of work but a full kernel launch (about 35 launches
// per level and cycle).  This kernel runs cycle(n0) (bbmg_class.f90:732-776)
// for every level n0..nlvl inside one thread-block cluster: the passes are
// separated by the cluster's hardware barrier, whose release/acquire
// semantics make each pass's global-memory writes visible to the next.  A
// cluster is scheduled as a unit, so no block can wait on one that is not
// running, and no barrier can outlive its kernel.  Each pass calls the same
// per-point functions as the single-pass kernels, so FP64 results stay
// bit-identical.
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// The passes of the tail, over the threads [tid, nth) of either the whole
// cluster (CL: a cluster barrier after each pass) or block 0 alone.
template <bool CL>
__device__ __forceinline__ void pass_sync() {
    if (CL) cluster_sync_all();
    else __syncthreads();
}

// skip: leave out the first colour (the one the opposite sweep before ended
// with; recomputing it gives the same bits).  The loop keeps its fixed start:
// with a runtime start ptxas gave the tail kernel half the registers (64
// against 127) and its passes ran ~40 % slower.
template <bool CL, typename T>
__device__ void tail_relax(const TailLvl<T> &l, int dir, int tid, int nth, bool skip) {
    for (int c = 0; c < 8; c++) {
        if (c == 0 && skip) continue;
        const int col = dir > 0 ? c : 7 - c;  // colours 1..8 forward, 8..1 backward
        const int px = col & 1, py = (col >> 1) & 1, pz = (col >> 2) & 1;
        const Lay &L = l.L;
        const int na = (L.nx - px + 1) >> 1, nb = (L.ny - py + 1) >> 1, nc = (L.nz - pz + 1) >> 1;
        const int n = na * nb * nc;
        if (n == 0) continue;
        const long long hb = px ? 0 : L.B0;
        for (int it = tid; it < n; it += nth) {
            const int a = it % na, row = it / na;
            const int j = py + 2 * (row % nb), k = pz + 2 * (row / nb);
            gs_points<T, 27, 1>(L, l.off[px], l.opr, l.v, l.f, L.G + L.row(j, k) * L.P + hb + a, px, j, k, a, 1);
        }
        pass_sync<CL>();
    }
}

// pre-smoothing, residual and restriction of level l into c (bbmg_class.f90:750-763)
template <bool CL, typename T>
__device__ void tail_down(const TailArgs<T> &A, const TailLvl<T> &l, const TailLvl<T> &c, int tid, int nth) {
    int dir = 1;
    for (int i = 0; i < A.pre; i++, dir = -dir) {
        tail_relax<CL>(l, dir, tid, nth, i > 0);
    }
    const Lay &L = l.L;
    for (int it = tid; it < L.nx * L.ny * L.nz; it += nth) {
        const int i = it % L.nx, row = it / L.nx;
        residual_point<T, 27>(L, l.off[0].o, l.off[1].o, l.opr, l.v, l.f, l.r, i, row % L.ny, row / L.ny);
    }
    pass_sync<CL>();
    const Lay &C = c.L;
    for (int it = tid; it < C.nx * C.ny * C.nz; it += nth) {
        const int i = it % C.nx, row = it / C.nx;
        restrict_point<T>(L, C, l.c2f, l.r, c.f, c.v, i, row % C.ny, row / C.ny);
    }
    pass_sync<CL>();
}

// prolongation + correction into l from c, post-smoothing (bbmg_class.f90:766-775)
template <bool CL, typename T>
__device__ void tail_up(const TailArgs<T> &A, const TailLvl<T> &l, const TailLvl<T> &c, int tid, int nth) {
    const Lay &F = l.L;
    for (int it = tid; it < F.nx * F.ny * F.nz; it += nth) {
        const int i = it % F.nx, row = it / F.nx;
        prolong_point<T>(F, c.L, l.c2f, c.v, l.v, i, row % F.ny, row / F.ny);
    }
    pass_sync<CL>();
    int dir = (A.pre & 1) ? -1 : 1;
    for (int i = 0; i < A.post; i++, dir = -dir) {
        tail_relax<CL>(l, dir, tid, nth, i > 0);
    }
}

// coarsest level (bbmg_class.f90:741-748): block 0 solves with the stored LU
template <bool CL, typename T>
__device__ void tail_coarsest(const TailArgs<T> &A, double *sm, int tid, int nth) {
    const TailLvl<T> &lc = A.lv[A.n - 1];
    if (A.direct) {
        if (blockIdx.x == 0) coarse_solve_block<T>(lc.L, A.LU, A.piv, A.pinned, lc.f, lc.v, A.mat_in_smem, sm);
        pass_sync<CL>();
        return;
    }
    int dir = 1;
    for (int i = 0; i < A.pre + A.post; i++, dir = -dir) {
        tail_relax<CL>(lc, dir, tid, nth, i > 0);
    }
}

// The launch is one cluster.  Levels [0, A.split) run on every block of it;
// when A.split < A.n - 1 the levels [A.split, A.n) -- a few thousand cells or
// fewer -- run inside block 0 with block-wide barriers while the other blocks
// wait at one cluster barrier; otherwise only the coarsest level is left.
template <typename T>
__global__ void __launch_bounds__(kTailThreads) k_vtail(const __grid_constant__ TailArgs<T> A) {
    extern __shared__ double sm[];
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    for (int n = 0; n < A.split; n++) tail_down<true>(A, A.lv[n], A.lv[n + 1], tid, nth);
    if (A.split < A.n - 1) {
        if (blockIdx.x == 0) {
            const int t = threadIdx.x, nt = blockDim.x;
            for (int n = A.split; n + 1 < A.n; n++) tail_down<false>(A, A.lv[n], A.lv[n + 1], t, nt);
            tail_coarsest<false>(A, sm, t, nt);
            for (int n = A.n - 2; n >= A.split; n--) tail_up<false>(A, A.lv[n], A.lv[n + 1], t, nt);
        }
        cluster_sync_all();
    } else {
        tail_coarsest<true>(A, sm, tid, nth);
    }
    for (int n = A.split - 1; n >= 0; n--) tail_up<true>(A, A.lv[n], A.lv[n + 1], tid, nth);
}

size_t tail_smem(int np, int *mat_in_smem) {
    const size_t full = sizeof(double) * ((size_t)np + (size_t)np * np);
    *mat_in_smem = full <= kTailSmemMax ? 1 : 0;
    return *mat_in_smem ? full : sizeof(double) * (size_t)np;
}

static cudaLaunchConfig_t tail_cfg(int cl, size_t smem, cudaStream_t s, cudaLaunchAttribute *at) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3(kTailThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

// The largest cluster (16 blocks, else 8) the device can schedule for k_vtail.
template <typename T>
cudaError_t tail_grid(size_t smem, int *blocks) {
    cudaError_t e = cudaFuncSetAttribute(k_vtail<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess && smem > 48 * 1024)
        e = cudaFuncSetAttribute(k_vtail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    for (int cl = kTailClusterMax; cl >= 8; cl /= 2) {
        cudaLaunchAttribute at[1];
        cudaLaunchConfig_t cfg = tail_cfg(cl, smem, nullptr, at);
        int nc = 0;
        if (cudaOccupancyMaxActiveClusters(&nc, k_vtail<T>, &cfg) == cudaSuccess && nc >= 1) {
            *blocks = cl;
            return cudaSuccess;
        }
        cudaGetLastError();
    }
    return cudaErrorLaunchOutOfResources;
}

template <typename T>
cudaError_t launch_vtail(const TailArgs<T> &A, int blocks, size_t smem, cudaStream_t s) {
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = tail_cfg(blocks, smem, s, at);
    BB_CHECK_LAUNCH(cudaLaunchKernelEx(&cfg, k_vtail<T>, A));
    return cudaSuccess;
}

template cudaError_t tail_grid<double>(size_t, int *);
template cudaError_t tail_grid<float>(size_t, int *);
template cudaError_t launch_vtail<double>(const TailArgs<double> &, int, size_t, cudaStream_t);
template cudaError_t launch_vtail<float>(const TailArgs<float> &, int, size_t, cudaStream_t);

#define BB_INST(T)                                                                                                   \
    template cudaError_t launch_relax<T>(const Lay &, const NbrOff &, int, bool, const T *, T *, const T *, int,     \
                                         cudaStream_t, bool);                                                        \
    template cudaError_t launch_relax_sweeps<T>(const Lay &, const NbrOff &, int, bool, const T *, T *, const T *,   \
                                                int, int, cudaStream_t);                                             \
    template cudaError_t launch_residual<T>(const Lay &, const NbrOff &, int, const T *, const T *, const T *, T *,  \
                                            cudaStream_t);                                                           \
    template cudaError_t launch_restrict<T>(const Lay &, const Lay &, const T *, const T *, T *, T *, cudaStream_t); \
    template cudaError_t launch_prolong<T>(const Lay &, const Lay &, const T *, const T *, T *, cudaStream_t);       \
    template cudaError_t launch_coarse_solve<T>(const Lay &, const double *, const int *, const int *, const T *,    \
                                                T *, cudaStream_t);                                                  \
    template cudaError_t launch_maxabs<T>(const Lay &, const T *, double *, double *, cudaStream_t);                \
    template cudaError_t launch_dot<T>(const Lay &, const T *, const T *, double *, double *, cudaStream_t);        \
    template cudaError_t launch_from_caller<T>(const Lay &, const double *, int, T *, cudaStream_t);                 \
    template cudaError_t launch_cg_rho<T>(const Lay &, const T *, const double *, double *, CgScal *, cudaStream_t); \
    template cudaError_t launch_fcg_rho<T>(const Lay &, const T *, const double *, const double *, double *, CgScal *, \
                                           cudaStream_t);                                                            \
    template cudaError_t launch_cg_pap_fused<T>(const Lay &, const NbrOff &, int, const double *, const T *,         \
                                                const double *, double *, double *, double *, CgScal *,             \
                                                cudaStream_t);                                                       \
    template cudaError_t launch_cg_xr_fused<T>(const Lay &, double *, const double *, double *, const double *,      \
                                               const CgScal *, float *, T *, double *, double *, cudaStream_t);
BB_INST(double)
BB_INST(float)

}  // namespace bbmg
