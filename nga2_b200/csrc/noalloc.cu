// noalloc.cu -- residual check that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a flow solver whose device memory is
// handed out by its own pool allocator (every byte it may touch is reserved up
// front, so the CUDA allocator must not be called behind its back), and a time
// loop that must not allocate because cudaMalloc/cudaFree can synchronise the
// device.  bbmg_residual_norm_noalloc gives those callers the solver's residual
// check on their own arrays without allocating: its only scratch is the
// file-scope array below.  CUDA places it in a GPU's memory when it loads this
// library's device code on that GPU -- with CUDA's default lazy module loading
// that happens at the first call on the GPU, which can synchronise the device,
// so a caller makes one warm-up call before its time loop or any stream
// capture -- and the GPU holds it until the process exits.
//
// The scratch holds one partial pair (max|r|, max|b|) per k-plane of the
// grid, so a call accepts at most kNoAllocMaxPlanes planes and rejects larger
// grids.  Every call writes each slot it reads before reading it, so nothing
// needs clearing between calls.  All calls share the one array: calls whose
// kernels overlap on the GPU (different streams, or different host threads)
// race on it and must be serialised by the caller.
#include <cmath>
#include <cstdio>

#include "../../include/bbmg_b200.h"
#include "common.cuh"

namespace bbmg {
void set_create_error(const char *msg);  // api.cu
}

namespace {

constexpr int kNoAllocMaxPlanes = 8192;  // 2 doubles per plane: 128 KiB
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxPlanes];

// In host code the array's name is only a host-side stand-in, not a device
// address: every call looks up the address on the current device with
// cudaGetSymbolAddress (a table lookup once the module is loaded), so no
// address outlives a device reset or a new primary context.

int noalloc_fail(int code, const char *msg) {
    bbmg::set_create_error(msg);  // reported by bbmg_last_error(NULL)
    return code;
}

struct TermTable {
    int nterm;          // stencil slots present, in the reference's column-major order
    int dx[27], dy[27], dz[27];
    int first[28];      // entries of term t: st_list[first[t] .. first[t+1])
    int st_list[27];    // caller stencil entries, in stencil order
};

__device__ __forceinline__ double max_nan(double m, double a) { return (a != a || m != m) ? (a + m) : fmax(m, a); }

// One block per k-plane: r = rhs - A sol over the plane's interior (the
// operator scattered from the caller's stencil as bbmg_setup does, neighbours
// outside a non-periodic direction are zero, periodic ones wrap), block maxima
// of |r| and |rhs| into scratch[2k], scratch[2k+1].
__global__ void __launch_bounds__(256) k_noalloc_partials(bbmg_grid g, TermTable tt, const double *__restrict__ opr,
                                                           const double *__restrict__ rhs,
                                                           const double *__restrict__ sol,
                                                           double *__restrict__ scratch) {
    __shared__ double shr[256], shb[256];
    const int k = blockIdx.x;
    const int gh = g.ghost, nst = tt.first[tt.nterm];
    const long long sy = g.nx + 2 * gh, sz = sy * (g.ny + 2 * gh);
    double mr = 0.0, mb = 0.0;
    const int ncell = g.nx * g.ny;
    for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
        const int i = c % g.nx, j = c / g.nx;
        const long long e = (long long)(k + gh) * sz + (long long)(j + gh) * sy + (i + gh);
        double s = 0.0;
        for (int t = 0; t < tt.nterm; t++) {
            int i2 = i + tt.dx[t], j2 = j + tt.dy[t], k2 = k + tt.dz[t];
            bool zero = false;
            if (i2 < 0 || i2 >= g.nx) { if (g.xper) i2 = (i2 + g.nx) % g.nx; else zero = true; }
            if (j2 < 0 || j2 >= g.ny) { if (g.yper) j2 = (j2 + g.ny) % g.ny; else zero = true; }
            if (k2 < 0 || k2 >= g.nz) { if (g.zper) k2 = (k2 + g.nz) % g.nz; else zero = true; }
            double coef = 0.0;
            for (int q = tt.first[t]; q < tt.first[t + 1]; q++) coef = __dadd_rn(coef, opr[e * nst + tt.st_list[q]]);
            const double v = zero ? 0.0 : sol[(long long)(k2 + gh) * sz + (long long)(j2 + gh) * sy + (i2 + gh)];
            s = __dadd_rn(s, __dmul_rn(coef, v));
        }
        const double b = rhs[e];
        mr = max_nan(mr, fabs(__dsub_rn(b, s)));
        mb = max_nan(mb, fabs(b));
    }
    shr[threadIdx.x] = mr;
    shb[threadIdx.x] = mb;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            shr[threadIdx.x] = max_nan(shr[threadIdx.x], shr[threadIdx.x + h]);
            shb[threadIdx.x] = max_nan(shb[threadIdx.x], shb[threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scratch[2 * k] = shr[0];
        scratch[2 * k + 1] = shb[0];
    }
}

// out = {max|r|, max|rhs|, max|r| / max|rhs|} from the first nz partial pairs.
__global__ void __launch_bounds__(256) k_noalloc_final(int nz, const double *__restrict__ scratch,
                                                        double *__restrict__ out) {
    __shared__ double shr[256], shb[256];
    double mr = 0.0, mb = 0.0;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        mr = max_nan(mr, scratch[2 * k]);
        mb = max_nan(mb, scratch[2 * k + 1]);
    }
    shr[threadIdx.x] = mr;
    shb[threadIdx.x] = mb;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            shr[threadIdx.x] = max_nan(shr[threadIdx.x], shr[threadIdx.x + h]);
            shb[threadIdx.x] = max_nan(shb[threadIdx.x], shb[threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = shr[0];
        out[1] = shb[0];
        // a zero rhs: 0 for a zero residual (what a zero-guess solve reports), +inf otherwise
        out[2] = shb[0] > 0.0 ? __ddiv_rn(shr[0], shb[0]) : (shr[0] == 0.0 ? 0.0 : HUGE_VAL);
    }
}

// device memory of device `dev` (managed memory is reachable from any device)
bool on_device(const void *p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
}

}  // namespace

extern "C" int bbmg_residual_norm_noalloc(const bbmg_grid *grid, int nst, const int *stc, const double *opr,
                                          const double *rhs, const double *sol, double *out, void *stream) {
    if (!grid || !stc || !opr || !rhs || !sol || !out) return noalloc_fail(BBMG_BAD_ARGS, "null argument");
    const bbmg_grid g = *grid;
    if (g.nx < 1 || g.ny < 1 || g.nz < 1 || g.ghost < 0) return noalloc_fail(BBMG_BAD_ARGS, "grid sizes must be >= 1");
    if (g.nz > kNoAllocMaxPlanes) {
        char m[160];
        snprintf(m, sizeof m, "nz = %d exceeds the %d k-planes the allocation-free scratch holds", g.nz,
                 kNoAllocMaxPlanes);
        return noalloc_fail(BBMG_BAD_ARGS, m);
    }
    if ((long long)g.nx * g.ny > (1LL << 30)) return noalloc_fail(BBMG_BAD_ARGS, "nx*ny exceeds 2^30 cells per plane");
    if (nst < 1 || nst > 27) return noalloc_fail(BBMG_BAD_ARGS, "nst must be 1..27");
    // stencil terms in the reference's column-major slot order (the 27-point
    // scatter of ils_class.f90:247-256), entries of one slot in stencil order
    TermTable tt{};
    int slot_of[27];
    for (int st = 0; st < nst; st++) {
        int a = stc[3 * st], b = stc[3 * st + 1], c = stc[3 * st + 2];
        if (a < -1 || a > 1 || b < -1 || b > 1 || c < -1 || c > 1)
            return noalloc_fail(BBMG_BAD_ARGS, "stencil entry outside 3x3x3");
        slot_of[st] = bbmg::q27(a, b, c);
    }
    int cnt = 0;
    for (int q = 0; q < 27; q++) {
        int first = cnt;
        for (int st = 0; st < nst; st++)
            if (slot_of[st] == q) tt.st_list[cnt++] = st;
        if (cnt > first) {
            tt.dx[tt.nterm] = q % 3 - 1;
            tt.dy[tt.nterm] = (q / 3) % 3 - 1;
            tt.dz[tt.nterm] = q / 9 - 1;
            tt.first[tt.nterm] = first;
            tt.nterm++;
        }
    }
    tt.first[tt.nterm] = cnt;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return noalloc_fail(BBMG_CUDA, "no current CUDA device");
    }
    if (!on_device(opr, dev) || !on_device(rhs, dev) || !on_device(sol, dev) || !on_device(out, dev))
        return noalloc_fail(BBMG_BAD_ARGS, "opr, rhs, sol and out must be memory of the current device");
    // the scratch array's address on this device (the current one)
    double *scratch = nullptr;
    {
        cudaError_t e = cudaGetSymbolAddress((void **)&scratch, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            char m[160];
            snprintf(m, sizeof m, "cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return noalloc_fail(BBMG_CUDA, m);
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    k_noalloc_partials<<<g.nz, 256, 0, s>>>(g, tt, opr, rhs, sol, scratch);
    k_noalloc_final<<<1, 256, 0, s>>>(g.nz, scratch, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(BBMG_CUDA, cudaGetErrorString(e));
    return BBMG_OK;
}
