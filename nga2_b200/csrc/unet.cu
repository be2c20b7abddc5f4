// unet.cu -- kernels of the learned initial guess (a small 3-D U-Net).
//
// No counterpart in the reference (NGA2 starts each pressure solve from the
// previous pressure).  The 3x3x3 convolutions are implicit GEMMs on the
// tensor cores: M = voxels, N = output channels, K = 27 taps x input
// channels, BF16 operands, FP32 accumulation (mma.sync m16n8k16).  A warp owns
// 16 consecutive voxels and all output channels; its A fragments are the
// tap-shifted input rows (periodic wrap), its B fragments the packed weights.
// The weight gradient is a reduction over voxels done on the CUDA cores with
// shared-memory staging; everything else is elementwise.
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdlib>

#include "../../include/bbmg_b200.h"
#include "../../include/bbmg_learned.h"

namespace {

typedef __nv_bfloat16 bf16;

struct Act {
    bf16 *p;
    int n, d, h, w, c, ld;
    int nvox;
};

Act act_of(const nn_act *a) {
    Act r;
    r.p = (bf16 *)a->data;
    r.n = a->n; r.d = a->d; r.h = a->h; r.w = a->w; r.c = a->c; r.ld = a->ld;
    r.nvox = a->n * a->d * a->h * a->w;
    return r;
}

bool bad_act(const nn_act *a) {
    return !a || !a->data || a->n < 1 || a->d < 1 || a->h < 1 || a->w < 1 || a->c < 1 || a->ld < a->c ||
           (a->ld & 1) || (long long)a->n * a->d * a->h * a->w * a->ld >= (1LL << 31);
}

int done(cudaError_t e) { return e == cudaSuccess ? BBMG_OK : BBMG_CUDA; }

__device__ __forceinline__ void decode(const Act &a, int v, int &n, int &d, int &h, int &w) {
    w = v % a.w;
    int r = v / a.w;
    h = r % a.h;
    r /= a.h;
    d = r % a.d;
    n = r / a.d;
}
__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }
__device__ __forceinline__ int vox(const Act &a, int n, int d, int h, int w) {
    return ((n * a.d + d) * a.h + h) * a.w + w;
}

__device__ __forceinline__ uint32_t ld32(const bf16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

__device__ __forceinline__ void mma16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// ---------------------------------------------------------------------------
// Convolution as implicit GEMM.  wt is [27][cout][cin] (K contiguous per
// output channel, the layout of the mma B operand).  NT = cout / 8.
template <int NT>
__global__ void __launch_bounds__(128) k_conv3(Act x, const bf16 *__restrict__ wt, const float *__restrict__ bias,
                                                Act y, int relu) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int v0 = (blockIdx.x * 4 + warp) * 16;
    if (v0 >= x.nvox) return;
    const int cin = x.c;
    const int r0 = v0 + g, r1 = v0 + g + 8;
    const int q0 = min(r0, x.nvox - 1), q1 = min(r1, x.nvox - 1);
    int n0, d0, h0, w0, n1, d1, h1, w1;
    decode(x, q0, n0, d0, h0, w0);
    decode(x, q1, n1, d1, h1, w1);
    float acc[NT][4];
#pragma unroll
    for (int i = 0; i < NT; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    for (int tap = 0; tap < 27; tap++) {
        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
        const int s0 = vox(x, n0, wrapi(d0 + dz, x.d), wrapi(h0 + dy, x.h), wrapi(w0 + dx, x.w));
        const int s1 = vox(x, n1, wrapi(d1 + dz, x.d), wrapi(h1 + dy, x.h), wrapi(w1 + dx, x.w));
        const bf16 *xa = x.p + (long long)s0 * x.ld + 2 * t;
        const bf16 *xb = x.p + (long long)s1 * x.ld + 2 * t;
        const bf16 *wtap = wt + (long long)tap * (NT * 8) * cin + (long long)g * cin + 2 * t;
        for (int c0 = 0; c0 < cin; c0 += 16) {
            const uint32_t a0 = ld32(xa + c0), a1 = ld32(xb + c0), a2 = ld32(xa + c0 + 8), a3 = ld32(xb + c0 + 8);
#pragma unroll
            for (int nt = 0; nt < NT; nt++) {
                const bf16 *wp = wtap + (long long)nt * 8 * cin + c0;
                mma16816(acc[nt], a0, a1, a2, a3, __ldg(reinterpret_cast<const unsigned int *>(wp)),
                         __ldg(reinterpret_cast<const unsigned int *>(wp + 8)));
            }
        }
    }
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
        const int col = nt * 8 + 2 * t;
        const float b0 = bias ? bias[col] : 0.f, b1 = bias ? bias[col + 1] : 0.f;
        float o0 = acc[nt][0] + b0, o1 = acc[nt][1] + b1, o2 = acc[nt][2] + b0, o3 = acc[nt][3] + b1;
        if (relu) {
            o0 = fmaxf(o0, 0.f); o1 = fmaxf(o1, 0.f); o2 = fmaxf(o2, 0.f); o3 = fmaxf(o3, 0.f);
        }
        if (r0 < y.nvox)
            *reinterpret_cast<__nv_bfloat162 *>(y.p + (long long)r0 * y.ld + col) = __floats2bfloat162_rn(o0, o1);
        if (r1 < y.nvox)
            *reinterpret_cast<__nv_bfloat162 *>(y.p + (long long)r1 * y.ld + col) = __floats2bfloat162_rn(o2, o3);
    }
}

// ---------------------------------------------------------------------------
// The same convolution on the fifth-generation tensor cores (tcgen05), for
// grids whose rows hold a multiple of 128 voxels.  One CTA computes a tile of
// 128 consecutive voxels of one (n, d, h) row against all output channels:
//   * the 9 input rows (d+dz, h+dy) of the tile with their x-halo (130 voxels,
//     periodic wrap) are staged once in shared memory in the K-major canonical
//     layout of the MMA (no swizzle): for each group of 8 channels, the 130
//     voxels' 16-byte chunks one after another.  A tap (dz, dy, dx) is then
//     just a descriptor whose start address is shifted by dx chunks;
//   * the packed weights [tap][cout][cin] are staged as [tap][K-chunk][group of
//     8 channels][cout][16 bytes];
//   * one thread issues 27 x cin/16 tcgen05.mma (M = 128, N = cout, K = 16,
//     BF16 x BF16 -> FP32) into a TMEM accumulator of cout columns, then
//     tcgen05.commit arrives on an mbarrier;
//   * the four warps read their 32 TMEM lanes (= 32 voxels) with tcgen05.ld,
//     add the bias, apply the ReLU and store BF16 rows.
// The mbarrier wait is bounded: a wait that runs out raises *err, the CTA still
// frees its TMEM and returns.
constexpr unsigned kTcSpinLimit = 1u << 22;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cpa16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// shared-memory matrix descriptor: K-major, no swizzle (addresses and offsets in bytes)
__device__ __forceinline__ uint64_t umma_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major, M = 128
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

template <int N>
__global__ void __launch_bounds__(128, 1) k_conv3_tc(Act x, const bf16 *__restrict__ wt, const float *__restrict__ bias,
                                                     Act y, int relu, int *err) {
    extern __shared__ __align__(128) unsigned char smtc[];
    constexpr int kCols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));  // TMEM columns (power of 2)
    unsigned *tmem_slot = reinterpret_cast<unsigned *>(smtc);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smtc + 8);
    const int cin = x.c, kg = cin >> 3, kc = cin >> 4;
    unsigned char *A = smtc + 128;                               // [9][kg][130][16 B]
    unsigned char *B = A + (size_t)9 * kg * 130 * 16;          // [27][kc][2][N][16 B]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_per_row = x.w >> 7;
    const int tile = blockIdx.x;
    const int w0 = (tile % tiles_per_row) << 7;
    int rowid = tile / tiles_per_row;  // (n, d, h) row
    const int h = rowid % x.h;
    rowid /= x.h;
    const int d = rowid % x.d, n = rowid / x.d;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
    // stage the weights: chunk (tap, c, g, o) <- wt[tap][o][16c + 8g .. +8]
    const int nw = 27 * kc * 2 * N;
    for (int e = tid; e < nw; e += 128) {
        const int o = e % N, r = e / N, g = r & 1, c = (r >> 1) % kc, tap = (r >> 1) / kc;
        cpa16(B + (size_t)e * 16, wt + ((size_t)tap * N + o) * cin + c * 16 + g * 8);
    }
    // stage the 9 input rows with their x-halo
    const int na = 9 * kg * 130;
    for (int e = tid; e < na; e += 128) {
        const int vv = e % 130, r = e / 130, g = r % kg, rr = r / kg;
        const int dz = rr / 3 - 1, dy = rr % 3 - 1;
        const int dd = wrapi(d + dz, x.d), hh = wrapi(h + dy, x.h), ww = wrapi(w0 - 1 + vv, x.w);
        cpa16(A + (size_t)e * 16, x.p + (size_t)vox(x, n, dd, hh, ww) * x.ld + g * 8);
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *reinterpret_cast<volatile unsigned *>(tmem_slot);

    if (tid == 0) {
        const unsigned abase = smem_u32(A), bbase = smem_u32(B);
        const uint32_t idesc = umma_idesc_bf16(N);
        int first = 1;
        for (int rr = 0; rr < 9; rr++)
            for (int dx = 0; dx < 3; dx++)
                for (int c = 0; c < kc; c++) {
                    const int tap = rr * 3 + dx;
                    const uint64_t ad = umma_desc(abase + ((rr * kg + 2 * c) * 130 + dx) * 16, 130 * 16, 128);
                    const uint64_t bd = umma_desc(bbase + ((tap * kc + c) * 2) * N * 16, N * 16, 128);
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
                        ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(first ? 0 : 1), "r"(0));
                    first = 0;
                }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                     : "memory");
    }
    // wait for the accumulator (bounded)
    unsigned done = 0, spins = 0;
    while (!done) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(smem_u32(mbar)) : "memory");
        if (!done && ++spins > kTcSpinLimit) {
            if (lane == 0) atomicExch(err, 1);
            break;
        }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (done) {
        const int m = warp * 32 + lane;  // TMEM lane = tile row = voxel
        const long long v = (long long)vox(x, n, d, h, w0 + m);
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 16) {
            unsigned r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            __nv_bfloat162 o2[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                float a = __uint_as_float(r[2 * q]) + (bias ? bias[c0 + 2 * q] : 0.f);
                float b = __uint_as_float(r[2 * q + 1]) + (bias ? bias[c0 + 2 * q + 1] : 0.f);
                if (relu) { a = fmaxf(a, 0.f); b = fmaxf(b, 0.f); }
                o2[q] = __floats2bfloat162_rn(a, b);
            }
            uint4 *dst = reinterpret_cast<uint4 *>(y.p + v * y.ld + c0);
            dst[0] = *reinterpret_cast<uint4 *>(&o2[0]);
            dst[1] = *reinterpret_cast<uint4 *>(&o2[4]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

int *tc_err_flag() {
    static int *flag = nullptr;
    if (!flag && cudaMalloc(&flag, sizeof(int)) == cudaSuccess) cudaMemset(flag, 0, sizeof(int));
    return flag;
}

bool tc_eligible(const Act &x, const Act &y) {
    static const bool off = getenv("BBMG_NO_TCGEN05") != nullptr;
    if (off || x.w % 128 || x.c % 16 || (y.c != 16 && y.c != 32 && y.c != 48 && y.c != 64)) return false;
    if (x.ld % 8 || y.ld % 8 || (reinterpret_cast<uintptr_t>(x.p) & 15) || (reinterpret_cast<uintptr_t>(y.p) & 15))
        return false;
    const size_t smem = 128 + (size_t)9 * (x.c / 8) * 130 * 16 + (size_t)27 * x.c * y.c * 2;
    return smem <= 200 * 1024;
}

template <int N>
int launch_conv_tc(const Act &x, const bf16 *wt, const float *bias, const Act &y, int relu, cudaStream_t s) {
    const size_t smem = 128 + (size_t)9 * (x.c / 8) * 130 * 16 + (size_t)27 * x.c * N * 2;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_conv3_tc<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
            return BBMG_CUDA;
        attr = true;
    }
    int *err = tc_err_flag();
    if (!err) return BBMG_NO_MEMORY;
    const int tiles = (x.nvox >> 7);
    k_conv3_tc<N><<<tiles, 128, smem, s>>>(x, wt, bias, y, relu, err);
    return done(cudaGetLastError());
}

int launch_conv(const Act &x, const bf16 *wt, const float *bias, const Act &y, int relu, cudaStream_t s) {
    const int blocks = (x.nvox + 63) / 64;
    // rows of a multiple of 128 voxels: the tcgen05 kernel
    if (tc_eligible(x, y)) {
        switch (y.c) {
        case 16: return launch_conv_tc<16>(x, wt, bias, y, relu, s);
        case 32: return launch_conv_tc<32>(x, wt, bias, y, relu, s);
        case 48: return launch_conv_tc<48>(x, wt, bias, y, relu, s);
        case 64: return launch_conv_tc<64>(x, wt, bias, y, relu, s);
        }
    }
    // output widths of the U-Net: 16/32/64/128 forward; the data gradients
    // of the concatenated decoder inputs add 48/96/192
    if (y.c % 8) return BBMG_BAD_ARGS;
    switch (y.c / 8) {
    case 2: k_conv3<2><<<blocks, 128, 0, s>>>(x, wt, bias, y, relu); break;
    case 4: k_conv3<4><<<blocks, 128, 0, s>>>(x, wt, bias, y, relu); break;
    case 6: k_conv3<6><<<blocks, 128, 0, s>>>(x, wt, bias, y, relu); break;
    case 8: k_conv3<8><<<blocks, 128, 0, s>>>(x, wt, bias, y, relu); break;
    case 12: k_conv3<12><<<blocks, 128, 0, s>>>(x, wt, bias, y, relu); break;
    case 16: k_conv3<16><<<blocks, 128, 0, s>>>(x, wt, bias, y, relu); break;
    case 24: k_conv3<24><<<blocks, 128, 0, s>>>(x, wt, bias, y, relu); break;
    default: return BBMG_BAD_ARGS;
    }
    return done(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Weight gradient: dw[tap][ci][co] += sum_v x(v + tap, ci) dy(v, co).  Block
// (tap, voxel chunk); each step stages VB voxels of dy and of the tap-shifted
// x in shared memory, every thread accumulates its (ci, co) pairs.
constexpr int kWgVB = 16;
__global__ void __launch_bounds__(256) k_wgrad(Act x, Act gy, float *__restrict__ dw, float *__restrict__ db,
                                                int vchunk) {
    extern __shared__ float sm[];
    const int cin = x.c, cout = gy.c, tap = blockIdx.y;
    float *sx = sm;                      // [kWgVB][cin]
    float *sg = sm + kWgVB * cin;        // [kWgVB][cout]
    const int npair = cin * cout;
    constexpr int kMaxPairs = 24;        // pairs per thread; blockIdx.z selects a range of 24*256 pairs
    const int pbase = blockIdx.z * kMaxPairs * 256;
    float acc[kMaxPairs];
#pragma unroll
    for (int q = 0; q < kMaxPairs; q++) acc[q] = 0.f;
    float accb = 0.f;
    const int dz = tap / 9 - 1, dyy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const int vbeg = blockIdx.x * vchunk, vend = min(vbeg + vchunk, gy.nvox);
    for (int vb = vbeg; vb < vend; vb += kWgVB) {
        __syncthreads();
        for (int e = threadIdx.x; e < kWgVB * cin; e += blockDim.x) {
            const int k = e / cin, c = e % cin, v = vb + k;
            float val = 0.f;
            if (v < vend) {
                int n, d, h, w;
                decode(gy, v, n, d, h, w);
                const int s = vox(x, n, wrapi(d + dz, x.d), wrapi(h + dyy, x.h), wrapi(w + dx, x.w));
                val = __bfloat162float(x.p[(long long)s * x.ld + c]);
            }
            sx[e] = val;
        }
        for (int e = threadIdx.x; e < kWgVB * cout; e += blockDim.x) {
            const int k = e / cout, c = e % cout, v = vb + k;
            sg[e] = v < vend ? __bfloat162float(gy.p[(long long)v * gy.ld + c]) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kMaxPairs; q++) {
            const int p = pbase + threadIdx.x + q * blockDim.x;
            if (p < npair) {
                const int ci = p / cout, co = p % cout;
                float a = acc[q];
#pragma unroll
                for (int k = 0; k < kWgVB; k++) a = fmaf(sx[k * cin + ci], sg[k * cout + co], a);
                acc[q] = a;
            }
        }
        if (db && tap == 13 && blockIdx.z == 0 && threadIdx.x < cout)
            for (int k = 0; k < kWgVB; k++) accb += sg[k * cout + threadIdx.x];
    }
#pragma unroll
    for (int q = 0; q < kMaxPairs; q++) {
        const int p = pbase + threadIdx.x + q * blockDim.x;
        if (p < npair) atomicAdd(&dw[(long long)tap * npair + p], acc[q]);
    }
    if (db && tap == 13 && blockIdx.z == 0 && threadIdx.x < cout) atomicAdd(&db[threadIdx.x], accb);
}

// ---------------------------------------------------------------------------
__global__ void k_pack(const float *__restrict__ w, int cin, int cout, bf16 *__restrict__ wt, bf16 *__restrict__ wd) {
    const long long n = 27LL * cin * cout;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int tap = (int)(e / (cin * cout)), r = (int)(e % (cin * cout)), ci = r / cout, co = r % cout;
        const bf16 v = __float2bfloat16(w[e]);
        wt[((long long)tap * cout + co) * cin + ci] = v;               // forward: [tap][co][ci]
        wd[((long long)(26 - tap) * cin + ci) * cout + co] = v;        // backward: [26-tap][ci][co]
    }
}

__global__ void k_relu_bwd(Act dy, Act y) {
    const long long n = (long long)dy.nvox * dy.c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(e / dy.c), c = (int)(e % dy.c);
        if (!(__bfloat162float(y.p[(long long)v * y.ld + c]) > 0.f)) dy.p[(long long)v * dy.ld + c] = __float2bfloat16(0.f);
    }
}

// y (half size) = mean of the 8 children of x
__global__ void k_pool2(Act x, Act y) {
    const long long n = (long long)y.nvox * y.c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(e / y.c), c = (int)(e % y.c);
        int nn, d, h, w;
        decode(y, v, nn, d, h, w);
        float s = 0.f;
        for (int q = 0; q < 8; q++)
            s += __bfloat162float(x.p[(long long)vox(x, nn, 2 * d + (q >> 2), 2 * h + ((q >> 1) & 1), 2 * w + (q & 1)) * x.ld + c]);
        y.p[(long long)v * y.ld + c] = __float2bfloat16(0.125f * s);
    }
}
// dx (twice the size of dy) = dy(parent) / 8, or dx += that (accumulate: the
// pooled tensor is also a skip connection whose gradient is already in dx)
__global__ void k_pool2_bwd(Act dy, Act dx, int accumulate) {
    const long long n = (long long)dx.nvox * dx.c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(e / dx.c), c = (int)(e % dx.c);
        int nn, d, h, w;
        decode(dx, v, nn, d, h, w);
        float g = 0.125f * __bfloat162float(dy.p[(long long)vox(dy, nn, d >> 1, h >> 1, w >> 1) * dy.ld + c]);
        bf16 *o = dx.p + (long long)v * dx.ld + c;
        if (accumulate) g += __bfloat162float(*o);
        *o = __float2bfloat16(g);
    }
}
// y (twice the size of x) = x(parent)
__global__ void k_up2(Act x, Act y) {
    const long long n = (long long)y.nvox * y.c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(e / y.c), c = (int)(e % y.c);
        int nn, d, h, w;
        decode(y, v, nn, d, h, w);
        y.p[(long long)v * y.ld + c] = x.p[(long long)vox(x, nn, d >> 1, h >> 1, w >> 1) * x.ld + c];
    }
}
// dx (half the size of dy) = sum of the 8 children of dy
__global__ void k_up2_bwd(Act dy, Act dx) {
    const long long n = (long long)dx.nvox * dx.c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(e / dx.c), c = (int)(e % dx.c);
        int nn, d, h, w;
        decode(dx, v, nn, d, h, w);
        float s = 0.f;
        for (int q = 0; q < 8; q++)
            s += __bfloat162float(dy.p[(long long)vox(dy, nn, 2 * d + (q >> 2), 2 * h + ((q >> 1) & 1), 2 * w + (q & 1)) * dy.ld + c]);
        dx.p[(long long)v * dx.ld + c] = __float2bfloat16(s);
    }
}

struct Fields {
    const double *f[NN_MAX_FIELDS];
    double s[NN_MAX_FIELDS];
    int nf;
};

// pool = 1: the fields are on x's grid.  pool = 2: they are on the grid twice
// as fine and each voxel gets the mean of its 8 children (FP64 sum).
__global__ void k_embed(Fields fs, Act x, int pool) {
    const long long n = (long long)x.nvox * x.c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(e / x.c), c = (int)(e % x.c);
        float val = 0.f;
        if (c < fs.nf) {
            if (pool == 1) {
                val = (float)(fs.s[c] * fs.f[c][v]);
            } else {
                int nn, d, h, w;
                decode(x, v, nn, d, h, w);
                const int D = 2 * x.d, H = 2 * x.h, W = 2 * x.w;
                const double *f = fs.f[c] + (long long)nn * D * H * W;
                double sum = 0.0;
#pragma unroll
                for (int q = 0; q < 8; q++)
                    sum += f[((long long)(2 * d + (q >> 2)) * H + (2 * h + ((q >> 1) & 1))) * W + 2 * w + (q & 1)];
                val = (float)(fs.s[c] * 0.125 * sum);
            }
        }
        x.p[(long long)v * x.ld + c] = __float2bfloat16(val);
    }
}

__global__ void k_head(Act x, const float *__restrict__ w, const float *__restrict__ b, float *__restrict__ out) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < x.nvox; v += gridDim.x * blockDim.x) {
        float s = b[0];
        for (int c = 0; c < x.c; c++) s = fmaf(__bfloat162float(x.p[(long long)v * x.ld + c]), w[c], s);
        out[v] = s;
    }
}

__global__ void k_head_bwd(Act x, const float *__restrict__ w, const float *__restrict__ dout, Act dx,
                           float *__restrict__ dw, float *__restrict__ db) {
    __shared__ float sw[128], sb;
    if (threadIdx.x < 128) sw[threadIdx.x] = 0.f;
    if (threadIdx.x == 0) sb = 0.f;
    __syncthreads();
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < x.nvox; v += gridDim.x * blockDim.x) {
        const float g = dout[v];
        for (int c = 0; c < x.c; c++) {
            dx.p[(long long)v * dx.ld + c] = __float2bfloat16(g * w[c]);
            atomicAdd(&sw[c], g * __bfloat162float(x.p[(long long)v * x.ld + c]));
        }
        atomicAdd(&sb, g);
    }
    __syncthreads();
    if (threadIdx.x < x.c) atomicAdd(&dw[threadIdx.x], sw[threadIdx.x]);
    if (threadIdx.x == 0) atomicAdd(db, sb);
}

__global__ void k_mse(const float *__restrict__ pred, const double *__restrict__ tgt, double scale, long long n,
                      float *__restrict__ grad, double *loss) {
    __shared__ double sh[256];
    double s = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const double d = (double)pred[v] - scale * tgt[v];
        grad[v] = (float)(2.0 * d / (double)n);
        s += d * d;
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, sh[0]);
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const float gg = g[e];
        const float mm = b1 * m[e] + (1.f - b1) * gg;
        const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
        m[e] = mm;
        v[e] = vv;
        w[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

// out = base + scale * pred, pred given on the same grid (up = 1) or on a grid
// half as fine (up = 2), then interpolated trilinearly between cell centres
// (weights 3/4 and 1/4 per direction, periodic wrap).
__global__ void k_apply(const double *__restrict__ base, const float *__restrict__ pred, double scale, int nb, int d,
                        int h, int w, int up, double *__restrict__ out) {
    const int D = d * up, H = h * up, W = w * up;
    const long long n = (long long)nb * D * H * W;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        double v;
        if (up == 1) {
            v = (double)pred[e];
        } else {
            const int i = (int)(e % W), j = (int)((e / W) % H), k = (int)((e / ((long long)W * H)) % D);
            const int b = (int)(e / ((long long)W * H * D));
            const int i0 = i >> 1, j0 = j >> 1, k0 = k >> 1;
            const int i1 = wrapi(i0 + ((i & 1) ? 1 : -1), w), j1 = wrapi(j0 + ((j & 1) ? 1 : -1), h),
                      k1 = wrapi(k0 + ((k & 1) ? 1 : -1), d);
            const float *pb = pred + (long long)b * d * h * w;
            float acc = 0.f;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int kk = (q & 4) ? k1 : k0, jj = (q & 2) ? j1 : j0, ii = (q & 1) ? i1 : i0;
                const float wq = ((q & 4) ? 0.25f : 0.75f) * ((q & 2) ? 0.25f : 0.75f) * ((q & 1) ? 0.25f : 0.75f);
                acc = fmaf(wq, pb[((long long)kk * h + jj) * w + ii], acc);
            }
            v = (double)acc;
        }
        out[e] = (base ? base[e] : 0.0) + scale * v;
    }
}

int grid_elems(long long n) {
    long long g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

// ===========================================================================
extern "C" {

int nn_conv3(const nn_act *x, const void *wt, const float *bias, const nn_act *y, int relu, void *stream) {
    if (bad_act(x) || bad_act(y) || !wt || x->c % 16 || y->c % 16 || x->n != y->n || x->d != y->d ||
        x->h != y->h || x->w != y->w)
        return BBMG_BAD_ARGS;
    return launch_conv(act_of(x), (const bf16 *)wt, bias, act_of(y), relu, (cudaStream_t)stream);
}

int nn_conv3_dgrad(const nn_act *dy, const void *wd, const nn_act *dx, void *stream) {
    // conv of dy with the [tap'][ci][co] packing: input channels = cout of the
    // forward, output channels = its cin; with taps mirrored this is the
    // transposed convolution.
    if (bad_act(dy) || bad_act(dx) || !wd || dy->c % 16 || dx->c % 16 || dy->n != dx->n || dy->d != dx->d ||
        dy->h != dx->h || dy->w != dx->w)
        return BBMG_BAD_ARGS;
    return launch_conv(act_of(dy), (const bf16 *)wd, nullptr, act_of(dx), 0, (cudaStream_t)stream);
}

int nn_conv3_wgrad(const nn_act *x, const nn_act *dy, float *dw, float *db, void *stream) {
    if (bad_act(x) || bad_act(dy) || !dw || x->n != dy->n || x->d != dy->d || x->h != dy->h || x->w != dy->w ||
        dy->c > 256)
        return BBMG_BAD_ARGS;
    const Act ax = act_of(x), ag = act_of(dy);
    const int chunks = 148 * 4 / 27 + 1;
    int vchunk = (ag.nvox + chunks - 1) / chunks;
    vchunk = (vchunk + kWgVB - 1) / kWgVB * kWgVB;
    const int nchunk = (ag.nvox + vchunk - 1) / vchunk;
    const size_t shm = sizeof(float) * kWgVB * (ax.c + ag.c);
    const int nz = (ax.c * ag.c + 24 * 256 - 1) / (24 * 256);
    k_wgrad<<<dim3(nchunk, 27, nz), 256, shm, (cudaStream_t)stream>>>(ax, ag, dw, db, vchunk);
    return done(cudaGetLastError());
}

int nn_tc_error(void) {
    int *flag = tc_err_flag();
    if (!flag) return BBMG_NO_MEMORY;
    int v = 0;
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(&v, flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return BBMG_CUDA;
    if (v) cudaMemset(flag, 0, sizeof(int));
    return v ? BBMG_CUDA : BBMG_OK;
}

int nn_pack_weights(const float *w, int cin, int cout, void *wt, void *wd, void *stream) {
    if (!w || !wt || !wd || cin < 1 || cout < 1) return BBMG_BAD_ARGS;
    k_pack<<<grid_elems(27LL * cin * cout), 256, 0, (cudaStream_t)stream>>>(w, cin, cout, (bf16 *)wt, (bf16 *)wd);
    return done(cudaGetLastError());
}

int nn_relu_bwd(const nn_act *dy, const nn_act *y, void *stream) {
    if (bad_act(dy) || bad_act(y) || dy->c != y->c) return BBMG_BAD_ARGS;
    const Act a = act_of(dy);
    k_relu_bwd<<<grid_elems((long long)a.nvox * a.c), 256, 0, (cudaStream_t)stream>>>(a, act_of(y));
    return done(cudaGetLastError());
}

static bool halves(const nn_act *big, const nn_act *small) {
    return big->n == small->n && big->d == 2 * small->d && big->h == 2 * small->h && big->w == 2 * small->w &&
           big->c == small->c;
}

int nn_pool2(const nn_act *x, const nn_act *y, void *stream) {
    if (bad_act(x) || bad_act(y) || !halves(x, y)) return BBMG_BAD_ARGS;
    const Act b = act_of(y);
    k_pool2<<<grid_elems((long long)b.nvox * b.c), 256, 0, (cudaStream_t)stream>>>(act_of(x), b);
    return done(cudaGetLastError());
}
int nn_pool2_bwd(const nn_act *dy, const nn_act *dx, int accumulate, void *stream) {
    if (bad_act(dy) || bad_act(dx) || !halves(dx, dy)) return BBMG_BAD_ARGS;
    const Act b = act_of(dx);
    k_pool2_bwd<<<grid_elems((long long)b.nvox * b.c), 256, 0, (cudaStream_t)stream>>>(act_of(dy), b, accumulate);
    return done(cudaGetLastError());
}
int nn_up2(const nn_act *x, const nn_act *y, void *stream) {
    if (bad_act(x) || bad_act(y) || !halves(y, x)) return BBMG_BAD_ARGS;
    const Act b = act_of(y);
    k_up2<<<grid_elems((long long)b.nvox * b.c), 256, 0, (cudaStream_t)stream>>>(act_of(x), b);
    return done(cudaGetLastError());
}
int nn_up2_bwd(const nn_act *dy, const nn_act *dx, void *stream) {
    if (bad_act(dy) || bad_act(dx) || !halves(dy, dx)) return BBMG_BAD_ARGS;
    const Act b = act_of(dx);
    k_up2_bwd<<<grid_elems((long long)b.nvox * b.c), 256, 0, (cudaStream_t)stream>>>(act_of(dy), b);
    return done(cudaGetLastError());
}

int nn_embed(int nf, const double *const *fields, const double *scales, int pool, const nn_act *x, void *stream) {
    if (bad_act(x) || nf < 1 || nf > NN_MAX_FIELDS || nf > x->c || !fields || !scales || (pool != 1 && pool != 2))
        return BBMG_BAD_ARGS;
    Fields fs{};
    fs.nf = nf;
    for (int i = 0; i < nf; i++) {
        if (!fields[i]) return BBMG_BAD_ARGS;
        fs.f[i] = fields[i];
        fs.s[i] = scales[i];
    }
    const Act a = act_of(x);
    k_embed<<<grid_elems((long long)a.nvox * a.c), 256, 0, (cudaStream_t)stream>>>(fs, a, pool);
    return done(cudaGetLastError());
}

int nn_head(const nn_act *x, const float *w, const float *b, float *out, void *stream) {
    if (bad_act(x) || !w || !b || !out) return BBMG_BAD_ARGS;
    const Act a = act_of(x);
    k_head<<<grid_elems(a.nvox), 256, 0, (cudaStream_t)stream>>>(a, w, b, out);
    return done(cudaGetLastError());
}

int nn_head_bwd(const nn_act *x, const float *w, const float *dout, const nn_act *dx, float *dw, float *db,
                void *stream) {
    if (bad_act(x) || bad_act(dx) || !w || !dout || !dw || !db || x->c > 128 || dx->c != x->c) return BBMG_BAD_ARGS;
    const Act a = act_of(x);
    k_head_bwd<<<grid_elems(a.nvox), 256, 0, (cudaStream_t)stream>>>(a, w, dout, act_of(dx), dw, db);
    return done(cudaGetLastError());
}

int nn_mse(const float *pred, const double *target, double scale, long long nvox, float *grad, double *loss,
           void *stream) {
    if (!pred || !target || !grad || !loss || nvox < 1) return BBMG_BAD_ARGS;
    k_mse<<<grid_elems(nvox), 256, 0, (cudaStream_t)stream>>>(pred, target, scale, nvox, grad, loss);
    return done(cudaGetLastError());
}

int nn_adam(float *w, const float *g, float *m, float *v, long long n, float lr, float b1, float b2, float eps,
            int t, void *stream) {
    if (!w || !g || !m || !v || n < 1 || t < 1) return BBMG_BAD_ARGS;
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    k_adam<<<grid_elems(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return done(cudaGetLastError());
}

int nn_apply(const double *base, const float *pred, double scale, int nb, int d, int h, int w, int up, double *out,
             void *stream) {
    if (!pred || !out || nb < 1 || d < 1 || h < 1 || w < 1 || (up != 1 && up != 2) ||
        (long long)nb * d * h * w * up * up * up >= (1LL << 40))
        return BBMG_BAD_ARGS;
    const long long n = (long long)nb * d * h * w * up * up * up;
    k_apply<<<grid_elems(n), 256, 0, (cudaStream_t)stream>>>(base, pred, scale, nb, d, h, w, up, out);
    return done(cudaGetLastError());
}

}  // extern "C"
