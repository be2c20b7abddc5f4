// unet.cu -- kernels of the learned initial guess (a small 3-D U-Net).
//
// No counterpart in the reference (NGA2 starts each pressure solve from the
// previous pressure).  The 3x3x3 convolutions (forward and data gradient) are
// implicit GEMMs on the tensor cores: M = voxels, N = output channels, K = 27
// taps x input channels, BF16 operands, FP32 accumulation.  Grids of whole
// 128-voxel tiles run on tcgen05 (k_conv3_tcg: TMEM accumulator, cp.async
// stage ring, one thread issuing the MMAs); other sizes on mma.sync m16n8k16
// (k_conv3: a warp owns 16 consecutive voxels and all output channels, its A
// fragments the tap-shifted input rows with periodic wrap, its B fragments the
// packed weights).  The weight gradient, a contraction over voxels, runs on
// mma.sync with ldmatrix.trans fragments (k_wgrad_mma); everything else is
// elementwise.
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
// The same convolution on the fifth-generation tensor cores (tcgen05): an
// implicit GEMM with M = 128 consecutive voxels per CTA (one or more (h, w)
// rows, or part of one), N = all output channels, K = 27 taps x cin.
//   * K is walked in units of 16 channels (of one tap, or of one input row
//     for three taps, below); a few units form a pipeline stage.  A stage holds the A tile (the 128 voxels' tap-shifted
//     input channels, periodic wrap: thread m copies voxel m's two 16-byte
//     chunks per step) and the B tile (the packed weights [tap][cout][cin] of
//     those steps), both in the K-major no-swizzle canonical layout of the
//     MMA: per 8-channel group, rows of 16 bytes one after another (A:
//     [step][group][voxel][16 B], B: [step][group][cout][16 B]).
//   * S stages (template parameter, 2 by default) form a ring filled with
//     cp.async S-1 stages ahead; one
//     thread issues the tcgen05.mma (M = 128, N = cout, K = 16, BF16 x BF16 ->
//     FP32 in TMEM) of a stage and commits them to that stage's mbarrier; a
//     stage is refilled once its mbarrier shows the MMAs reading it are done.
//   * after the last stage the four warps read their 32 TMEM lanes (= 32
//     voxels) with tcgen05.ld, add the bias, apply the ReLU, store BF16.
// Every mbarrier wait is bounded: a wait that runs out raises *err (read by
// nn_tc_error), and the CTA then drains its copies, frees its TMEM and
// returns without writing.
constexpr unsigned kTcSpinLimit = 1u << 22;
constexpr int kTgS = 4;   // pipeline stages (the default of TgCfg; the launcher picks 2)

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

// bounded wait for the completion of phase `parity` of an mbarrier
__device__ __forceinline__ bool mbar_wait(const uint64_t *mb, unsigned parity) {
    for (unsigned spins = 0; spins < kTcSpinLimit; spins++) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(smem_u32(mb)), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Two tilings.  ROW (rows of a multiple of 128 voxels): a tile is 128
// consecutive voxels of one (n, d, h) row, and a K unit is one (dz, dy) input
// row with its x-halo (130 voxels) for 16 channels: it is staged once and
// serves the three dx taps through descriptors shifted by one 16-byte row
// (three MMAs per unit).  Otherwise a tile is 128 consecutive voxels of the
// grid (several rows when w < 128) and a K unit is one tap's 16 channels of
// the 128 voxels (one MMA).
template <int N, bool ROW, int S = kTgS>
struct TgCfg {
    static constexpr int kCols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));  // TMEM columns
    static constexpr int VOX = ROW ? 130 : 128;         // A rows staged per unit
    static constexpr int TAPS = ROW ? 3 : 1;            // MMAs (taps) per unit
    static constexpr int KU = ROW ? 2 : 4;              // units per stage
    static constexpr int A_UNIT = 2 * VOX * 16;         // bytes: [group][voxel][16 B]
    static constexpr int B_UNIT = TAPS * 2 * N * 16;    // bytes: [tap][group][cout][16 B]
    static constexpr int A_BYTES = KU * A_UNIT;
    static constexpr int B_BYTES = KU * B_UNIT;
    static constexpr size_t SMEM = 128 + (size_t)S * (A_BYTES + B_BYTES);
};

template <int N, bool ROW, int S>
__global__ void __launch_bounds__(128) k_conv3_tcg(Act x, const bf16 *__restrict__ wt, const float *__restrict__ bias,
                                                    Act y, int relu, int *err) {
    using Cfg = TgCfg<N, ROW, S>;
    extern __shared__ __align__(128) unsigned char smtc[];
    unsigned *tmem_slot = reinterpret_cast<unsigned *>(smtc);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smtc + 16);  // S barriers
    unsigned char *A = smtc + 128;
    unsigned char *B = A + (size_t)S * Cfg::A_BYTES;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int cin = x.c, kpt = cin >> 4;                 // 16-channel blocks
    const int nu = (ROW ? 9 : 27) * kpt;                 // K units
    const int nK = (nu + Cfg::KU - 1) / Cfg::KU;         // stages
    int v0;              // first voxel of the tile
    int vn[3], vd[3], vh[3], vw[3];
    const int ag = tid & 1;  // A copies: chunk e = (voxel e/2, group e%2), e = tid + 128 r
    if constexpr (ROW) {
        const int tiles_per_row = x.w >> 7;
        const int w0 = (blockIdx.x % tiles_per_row) << 7;
        int rowid = blockIdx.x / tiles_per_row;
        const int h = rowid % x.h;
        rowid /= x.h;
        const int d = rowid % x.d, n = rowid / x.d;
        v0 = vox(x, n, d, h, w0);
#pragma unroll
        for (int u = 0; u < 3; u++) {  // halo voxel (tid>>1) + 64u of the row, x-wrapped
            vn[u] = n; vd[u] = d; vh[u] = h;
            vw[u] = wrapi(w0 - 1 + (tid >> 1) + 64 * u, x.w);
        }
    } else {
        v0 = blockIdx.x * 128;
#pragma unroll
        for (int u = 0; u < 2; u++) decode(x, v0 + (tid >> 1) + 64 * u, vn[u], vd[u], vh[u], vw[u]);
    }

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(Cfg::kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0)
        for (int s = 0; s < S; s++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar + s)));

    // stage `chunk` (units chunk*KU ..) into ring slot `s`
    auto load = [&](int chunk, int s) {
        unsigned char *As = A + (size_t)s * Cfg::A_BYTES, *Bs = B + (size_t)s * Cfg::B_BYTES;
#pragma unroll
        for (int j = 0; j < Cfg::KU; j++) {
            const int un = chunk * Cfg::KU + j;
            if (un >= nu) break;
            int dz, dy, dx0, cb;  // the unit's row (and tap) and channel block
            if constexpr (ROW) {
                const int rr = un / kpt;
                cb = un - rr * kpt;
                dz = rr / 3 - 1; dy = rr % 3 - 1; dx0 = 0;
            } else {
                const int tap = un / kpt;
                cb = un - tap * kpt;
                dz = tap / 9 - 1; dy = (tap / 3) % 3 - 1; dx0 = tap % 3 - 1;
            }
#pragma unroll
            for (int u = 0; u < (ROW ? 3 : 2); u++) {
                const int vv = (tid >> 1) + 64 * u;  // A row of this copy
                if (ROW && vv >= Cfg::VOX) break;
                const bf16 *src = x.p +
                                  (long long)vox(x, vn[u], wrapi(vd[u] + dz, x.d), wrapi(vh[u] + dy, x.h),
                                                 ROW ? vw[u] : wrapi(vw[u] + dx0, x.w)) * x.ld + cb * 16 + ag * 8;
                cpa16(As + (size_t)j * Cfg::A_UNIT + ((size_t)ag * Cfg::VOX + vv) * 16, src);
            }
            for (int e = tid; e < Cfg::TAPS * 2 * N; e += 128) {
                const int t3 = e / (2 * N), r2 = e - t3 * 2 * N, g = r2 / N, o = r2 - g * N;
                const int tap = ROW ? (dz + 1) * 9 + (dy + 1) * 3 + t3 : (dz + 1) * 9 + (dy + 1) * 3 + dx0 + 1;
                cpa16(Bs + (size_t)j * Cfg::B_UNIT + ((size_t)(t3 * 2 + g) * N + o) * 16,
                      wt + ((long long)tap * N + o) * cin + cb * 16 + g * 8);
            }
        }
    };
    auto commit_group = []() { asm volatile("cp.async.commit_group;" ::: "memory"); };

#pragma unroll 1
    for (int p = 0; p < S - 1; p++) {
        if (p < nK) load(p, p);
        commit_group();
    }
    __syncthreads();  // barrier inits and the TMEM address are visible
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *reinterpret_cast<volatile unsigned *>(tmem_slot);
    const uint32_t idesc = umma_idesc_bf16(N);
    bool ok = true;
#pragma unroll 1
    for (int k = 0; k < nK; k++) {
        const int s = k % S;
        asm volatile("cp.async.wait_group %0;" ::"n"(S - 2) : "memory");  // stage k has landed
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");          // visible to the tensor core
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned as = smem_u32(A + (size_t)s * Cfg::A_BYTES), bs = smem_u32(B + (size_t)s * Cfg::B_BYTES);
#pragma unroll 1
            for (int j = 0; j < Cfg::KU; j++) {
                const int un = k * Cfg::KU + j;
                if (un >= nu) break;
#pragma unroll
                for (int t3 = 0; t3 < Cfg::TAPS; t3++) {
                    // ROW: tap dx = t3 - 1 reads the halo row shifted by t3 voxels
                    const uint64_t ad = umma_desc(as + j * Cfg::A_UNIT + t3 * 16, Cfg::VOX * 16, 128);
                    const uint64_t bd = umma_desc(bs + j * Cfg::B_UNIT + t3 * 2 * N * 16, N * 16, 128);
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
                        ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"((un > 0 || t3 > 0) ? 1 : 0), "r"(0));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(mbar + s)) : "memory");
        }
        const int nk = k + S - 1;  // the stage to fill next, in the slot stage k-1 used
        if (nk < nK) {
            if (k >= 1) {
                const bool done = mbar_wait(mbar + nk % S, ((k - 1) / S) & 1);
                if (__syncthreads_or(!done)) {
                    ok = false;
                    break;
                }
            }
            load(nk, nk % S);
        }
        commit_group();
    }
    bool done = false;
    if (ok) done = mbar_wait(mbar + (nK - 1) % S, ((nK - 1) / S) & 1);
    if (__syncthreads_or(!done)) {
        done = false;
        if (tid == 0) atomicExch(err, 1);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (done) {
        const long long v = v0 + tid;  // TMEM lane = tile row = voxel
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::kCols));
}

int *tc_err_flag() {
    static int *flag = nullptr;
    if (!flag && cudaMalloc(&flag, sizeof(int)) == cudaSuccess) cudaMemset(flag, 0, sizeof(int));
    return flag;
}

// the tcgen05 path: whole 128-voxel tiles, 16-byte aligned channel rows, and
// an output width the kernel is instantiated for
bool tc_eligible(const Act &x, const Act &y) {
    static const bool off = getenv("BBMG_NO_TCGEN05") != nullptr;
    if (off || x.nvox % 128 || x.c % 16) return false;
    if (y.c != 16 && y.c != 32 && y.c != 48 && y.c != 64 && y.c != 96 && y.c != 128 && y.c != 192) return false;
    return !(x.ld % 8 || y.ld % 8 || (reinterpret_cast<uintptr_t>(x.p) & 15) || (reinterpret_cast<uintptr_t>(y.p) & 15));
}

template <int N, bool ROW, int S>
int launch_conv_tc_t(const Act &x, const bf16 *wt, const float *bias, const Act &y, int relu, cudaStream_t s) {
    using Cfg = TgCfg<N, ROW, S>;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_conv3_tcg<N, ROW, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM) !=
            cudaSuccess)
            return BBMG_CUDA;
        attr = true;
    }
    int *err = tc_err_flag();
    if (!err) return BBMG_NO_MEMORY;
    k_conv3_tcg<N, ROW, S><<<x.nvox / 128, 128, Cfg::SMEM, s>>>(x, wt, bias, y, relu, err);
    return done(cudaGetLastError());
}

// ring depth S (BBMG_TC_STAGES = 2, 3 or 4): with 2 stages a CTA needs half
// the shared memory of 4 and about twice as many CTAs share an SM; measured
// at 128^3 the forward pass took 3.66 ms with 2 stages, 3.72 with 3, 3.79
// with 4
template <int N, bool ROW>
int launch_conv_tc_s(const Act &x, const bf16 *wt, const float *bias, const Act &y, int relu, cudaStream_t s) {
    static int st = -1;
    if (st < 0) {
        const char *e = getenv("BBMG_TC_STAGES");
        st = e ? atoi(e) : 2;
    }
    if (st == 2) return launch_conv_tc_t<N, ROW, 2>(x, wt, bias, y, relu, s);
    if (st == 3) return launch_conv_tc_t<N, ROW, 3>(x, wt, bias, y, relu, s);
    return launch_conv_tc_t<N, ROW, 4>(x, wt, bias, y, relu, s);
}

template <int N>
int launch_conv_tc(const Act &x, const bf16 *wt, const float *bias, const Act &y, int relu, cudaStream_t s) {
    static const bool no_rows = getenv("BBMG_NO_TC_ROWS") != nullptr;
    return (x.w % 128 == 0 && !no_rows) ? launch_conv_tc_s<N, true>(x, wt, bias, y, relu, s)
                                        : launch_conv_tc_s<N, false>(x, wt, bias, y, relu, s);
}

int launch_conv(const Act &x, const bf16 *wt, const float *bias, const Act &y, int relu, cudaStream_t s) {
    const int blocks = (x.nvox + 63) / 64;
    // whole 128-voxel tiles: the tcgen05 kernel
    if (tc_eligible(x, y)) {
        switch (y.c) {
        case 16: return launch_conv_tc<16>(x, wt, bias, y, relu, s);
        case 32: return launch_conv_tc<32>(x, wt, bias, y, relu, s);
        case 48: return launch_conv_tc<48>(x, wt, bias, y, relu, s);
        case 64: return launch_conv_tc<64>(x, wt, bias, y, relu, s);
        case 96: return launch_conv_tc<96>(x, wt, bias, y, relu, s);
        case 128: return launch_conv_tc<128>(x, wt, bias, y, relu, s);
        case 192: return launch_conv_tc<192>(x, wt, bias, y, relu, s);
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

// Weight gradient on the tensor cores: for one tap, dW[ci][co] = sum over
// voxels v of x(v + tap, ci) dy(v, co) is a GEMM with M = ci, N = co and the
// voxels as K (mma.sync m16n8k16, BF16 products, FP32 accumulation).  A CTA
// takes one tap, a chunk of voxels and a group of up to kWgTiles output tiles
// (16 ci x 8 co); per stage it copies kst voxels' channels (a multiple of 128:
// tap-shifted x with periodic wrap, and dy) as rows of 16-byte chunks into
// shared memory, its 8 warps take 16 of the voxels at a time as K steps, and
// ldmatrix.trans turns
// the channels-last rows into the A (ci x voxel) and B (voxel x co)
// fragments.  The warps' partial sums meet in shared memory and go to dw with
// one atomicAdd per output and CTA; the bias gradient (tap 13, tile group 0)
// is the column sum of dy.  Rows are padded by 16 bytes, so the eight rows an
// ldmatrix reads fall in distinct banks.
constexpr int kWgTiles = 8;   // output tiles (16 x 8) per CTA

__device__ __forceinline__ void ldsm_x4_t(unsigned &r0, unsigned &r1, unsigned &r2, unsigned &r3, const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2_t(unsigned &r0, unsigned &r1, const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(smem_u32(p)));
}

__global__ void __launch_bounds__(256) k_wgrad_mma(Act x, Act gy, float *__restrict__ dw, float *__restrict__ db,
                                                    int vchunk, int kst) {
    extern __shared__ __align__(16) unsigned char smw[];
    const int cin = x.c, cout = gy.c, tap = blockIdx.y;
    const int xs = cin * 2 + 16, gs = cout * 2 + 16;  // padded row strides (bytes)
    unsigned char *SX = smw;                                     // [kst][xs]
    unsigned char *SG = SX + (size_t)kst * xs;                   // [kst][gs]
    float *red = reinterpret_cast<float *>(SG + (size_t)kst * gs);  // [kWgTiles][128]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
    const int nt = cout >> 3, ntiles = (cin >> 4) * nt;
    const int tile0 = blockIdx.z * kWgTiles, ntl = min(kWgTiles, ntiles - tile0);
    const int dz = tap / 9 - 1, dyy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const int vbeg = blockIdx.x * vchunk, vend = min(vbeg + vchunk, gy.nvox);
    const bool bias = db && tap == 13 && blockIdx.z == 0;
    float acc[kWgTiles][4];
#pragma unroll
    for (int q = 0; q < kWgTiles; q++) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = 0.f;
    float accb = 0.f;
    for (int e = tid; e < kWgTiles * 128; e += 256) red[e] = 0.f;
    const int cx = cin >> 3, cg = cout >> 3;  // 16-byte chunks per voxel
    for (int vb = vbeg; vb < vend; vb += kst) {
        __syncthreads();  // the previous stage is consumed
        for (int kb = 0; kb < kst; kb += 128) {
            const int k = kb + (tid & 127), half = tid >> 7, v = vb + k;  // two threads per voxel
            const bool in = v < vend;
            long long src = 0;
            if (in) {
                int n, d, h, w;
                decode(gy, v, n, d, h, w);
                src = (long long)vox(x, n, wrapi(d + dz, x.d), wrapi(h + dyy, x.h), wrapi(w + dx, x.w)) * x.ld;
            }
            const uint4 zero = make_uint4(0, 0, 0, 0);
            for (int c = half; c < cx; c += 2)
                *reinterpret_cast<uint4 *>(SX + (size_t)k * xs + c * 16) =
                    in ? *reinterpret_cast<const uint4 *>(x.p + src + c * 8) : zero;
            for (int c = half; c < cg; c += 2)
                *reinterpret_cast<uint4 *>(SG + (size_t)k * gs + c * 16) =
                    in ? *reinterpret_cast<const uint4 *>(gy.p + (long long)v * gy.ld + c * 8) : zero;
        }
        __syncthreads();
        for (int k0 = warp * 16; k0 < kst; k0 += 128) {  // this warp's K steps: voxels k0 .. k0+15
#pragma unroll
            for (int q = 0; q < kWgTiles; q++) {
                if (q >= ntl) break;
                const int tile = tile0 + q, mb = (tile / nt) * 16, nb = (tile % nt) * 8;
                unsigned a0, a1, a2, a3, b0, b1;
                const int mi = lane >> 3, r = lane & 7;
                ldsm_x4_t(a0, a1, a2, a3, SX + (size_t)(k0 + r + (mi >= 2 ? 8 : 0)) * xs + (mb + (mi & 1) * 8) * 2);
                ldsm_x2_t(b0, b1, SG + (size_t)(k0 + r + ((lane >> 3) & 1) * 8) * gs + nb * 2);
                mma16816(acc[q], a0, a1, a2, a3, b0, b1);
            }
        }
        if (bias && tid < cout) {
            for (int k = 0; k < kst; k++)
                accb += __bfloat162float(reinterpret_cast<const bf16 *>(SG + (size_t)k * gs)[tid]);
        }
    }
    // the 8 warps' partial tiles -> shared memory -> dw
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kWgTiles; q++) {
        if (q >= ntl) break;
        // D fragment: rows g / g+8, columns 2 t4, 2 t4 + 1 of the 16 x 8 tile
        atomicAdd(&red[q * 128 + g * 8 + 2 * t4], acc[q][0]);
        atomicAdd(&red[q * 128 + g * 8 + 2 * t4 + 1], acc[q][1]);
        atomicAdd(&red[q * 128 + (g + 8) * 8 + 2 * t4], acc[q][2]);
        atomicAdd(&red[q * 128 + (g + 8) * 8 + 2 * t4 + 1], acc[q][3]);
    }
    __syncthreads();
    for (int e = tid; e < ntl * 128; e += 256) {
        const int q = e >> 7, m = (e >> 3) & 15, nn = e & 7;
        const int tile = tile0 + q, ci = (tile / nt) * 16 + m, co = (tile % nt) * 8 + nn;
        atomicAdd(&dw[((long long)tap * cin + ci) * cout + co], red[e]);
    }
    if (bias && tid < cout) atomicAdd(&db[tid], accb);
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
// the same, 8 channels (16 bytes) per thread, for 16-byte aligned views
__global__ void k_up2_v8(Act x, Act y) {
    const int g8 = y.c >> 3;
    const long long n = (long long)y.nvox * g8;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(e / g8), c = 8 * (int)(e - (long long)v * g8);
        int nn, d, h, w;
        decode(y, v, nn, d, h, w);
        *reinterpret_cast<uint4 *>(y.p + (long long)v * y.ld + c) =
            *reinterpret_cast<const uint4 *>(x.p + (long long)vox(x, nn, d >> 1, h >> 1, w >> 1) * x.ld + c);
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
    static const bool no_mma = getenv("BBMG_NO_WGRAD_MMA") != nullptr;
    // tensor cores: channel counts in whole tiles and 16-byte aligned channel rows
    if (!no_mma && ax.c % 16 == 0 && ag.c % 8 == 0 && ax.ld % 8 == 0 && ag.ld % 8 == 0 &&
        !(reinterpret_cast<uintptr_t>(ax.p) & 15) && !(reinterpret_cast<uintptr_t>(ag.p) & 15)) {
        const int ntiles = (ax.c / 16) * (ag.c / 8), groups = (ntiles + kWgTiles - 1) / kWgTiles;
        // voxels per stage: 128 x (1..4), up to ~64 KB of staged rows
        const size_t row = (size_t)(ax.c * 2 + 16 + ag.c * 2 + 16);
        int kst = 128;
        while (kst < 512 && (size_t)(2 * kst) * row <= 64 * 1024) kst *= 2;
        const size_t smem = (size_t)kst * row + sizeof(float) * kWgTiles * 128;
        static int attr_set = 0;
        if (smem > 48 * 1024 && !attr_set) {
            if (cudaFuncSetAttribute(k_wgrad_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
                return BBMG_CUDA;
            attr_set = 1;
        }
        // about eight CTAs per SM in all: voxel chunks of whole stages
        int nchunk = (148 * 8 + 27 * groups - 1) / (27 * groups);
        int vchunk = (ag.nvox + nchunk - 1) / nchunk;
        vchunk = (vchunk + kst - 1) / kst * kst;
        nchunk = (ag.nvox + vchunk - 1) / vchunk;
        k_wgrad_mma<<<dim3(nchunk, 27, groups), 256, smem, (cudaStream_t)stream>>>(ax, ag, dw, db, vchunk, kst);
        return done(cudaGetLastError());
    }
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
    const Act a = act_of(x), b = act_of(y);
    const bool v8 = b.c % 8 == 0 && a.ld % 8 == 0 && b.ld % 8 == 0 && !(reinterpret_cast<uintptr_t>(a.p) & 15) &&
                    !(reinterpret_cast<uintptr_t>(b.p) & 15);
    if (v8)
        k_up2_v8<<<grid_elems((long long)b.nvox * (b.c >> 3)), 256, 0, (cudaStream_t)stream>>>(a, b);
    else
        k_up2<<<grid_elems((long long)b.nvox * b.c), 256, 0, (cudaStream_t)stream>>>(a, b);
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
