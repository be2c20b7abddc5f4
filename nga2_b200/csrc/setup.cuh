// setup.cuh -- launchers of the setup and solve kernels.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace bbmg {

// setup.cu (FP64)
// `wmask`/`mask`: 27-bit sets of operator planes (q27 slots); the scatter
// writes only the planes in wmask (the others hold zeros already), the
// prolongation and A*P skip planes outside mask (known to be all zero);
// the scatter's stc is the caller's stencil in host memory
cudaError_t setup_scatter(const Lay &L, const double *src, int nst, int g, const int *stc, double *opr, unsigned wmask,
                          cudaStream_t s);
cudaError_t wrap_planes(const Lay &L, double *a, int nplanes, cudaStream_t s);
cudaError_t wrap_planes_mask(const Lay &L, double *a, unsigned mask, cudaStream_t s);
cudaError_t wrap_planes(const Lay &L, float *a, int nplanes, cudaStream_t s);
// c2f32 / oprC32, if given, receive the FP32 copies of the prolongation
// weights and of the coarse operator (the mixed-precision V-cycle's arrays)
cudaError_t setup_prolongation(const Lay &L, const double *opr, double *c2f, unsigned mask, cudaStream_t s,
                               float *c2f32 = nullptr);
cudaError_t setup_restriction(const Lay &F, const Lay &C, const double *c2f, double *f2c, cudaStream_t s);
cudaError_t setup_operator(const Lay &F, const Lay &C, const double *oprF, const double *c2f, const double *f2c,
                           double *oprc2f, double *oprC, unsigned mask, cudaStream_t s, float *oprC32 = nullptr);
// the overlap of f2c and of A P (oprc2f) as the reference holds it (zero in
// non-periodic directions, the periodic image otherwise); the setup leaves it
// unfilled where nothing reads it, so it is filled before a read-out
cudaError_t fill_overlap_f2c(const Lay &C, double *f2c, cudaStream_t s);
cudaError_t fill_overlap_oprc2f(const Lay &F, double *oprc2f, cudaStream_t s);
// plane q of oprS (and of oprS32, if given) = plane slots[q] of the 27-plane opr, npt <= 7
cudaError_t setup_solve_planes(const Lay &L, const double *opr, int npt, const int *slots, double *oprS,
                               float *oprS32, cudaStream_t s);
cudaError_t check_symmetric7(const Lay &L, const double *opr, int *flag, cudaStream_t s);
cudaError_t setup_direct(const Lay &L, const double *opr, double *OP, double *LU, int *piv, int *pinned, int *info,
                         cudaStream_t s);

// solve.cu
template <typename T>
cudaError_t launch_relax(const Lay &L, const NbrOff &nb, int npt, bool fuse, const T *opr, T *v, const T *f, int dir,
                         cudaStream_t s, bool skip_first = false);
// `nsweeps` alternating sweeps starting with `first_dir` (the relax loops of
// cycle, bbmg_class.f90:754-758 and 772-775)
template <typename T>
cudaError_t launch_relax_sweeps(const Lay &L, const NbrOff &nb, int npt, bool fuse, const T *opr, T *v, const T *f,
                                int first_dir, int nsweeps, cudaStream_t s);
template <typename T>
cudaError_t launch_residual(const Lay &L, const NbrOff &nb, int npt, const T *opr, const T *v, const T *f, T *r,
                            cudaStream_t s);
template <typename T>
cudaError_t launch_restrict(const Lay &F, const Lay &C, const T *c2f, const T *rF, T *fC, T *vC, cudaStream_t s);
template <typename T>
cudaError_t launch_prolong(const Lay &F, const Lay &C, const T *c2f, const T *vC, T *vF, cudaStream_t s);
constexpr size_t kCoarseSmem = 200 * 1024;  // factors of up to 158 unknowns stay on chip
cudaError_t coarse_solve_prepare();  // per device, before the first coarse solve
template <typename T>
cudaError_t launch_coarse_solve(const Lay &L, const double *LU, const int *piv, const int *pinned, const T *f, T *v,
                                cudaStream_t s);

// the coarse tail of the V-cycle in one launch of one thread-block cluster
// (levels n0..nlvl, 27-point operators, V-cycle only)
struct Off27 {
    int o[27];
};
template <typename T>
struct TailLvl {
    Lay L;
    Off27 off[2];          // neighbour offsets for even / odd x
    const T *opr;          // 27 coefficient planes
    T *v, *f, *r;
    const T *c2f;          // prolongation weights of this level (to the next coarser one)
};
constexpr int kTailMax = 8;            // levels in one launch (kernel parameters stay under 4 KB)
constexpr int kTailThreads = 512;
constexpr int kTailClusterMax = 16;    // blocks of the cluster (non-portable size; 8 if refused)
constexpr long long kTailCells = 512;  // first fused level: at most 8^3 cells.  Larger levels run
                                       // faster as staged passes in the iteration's CUDA graph
                                       // (measured: fused from 32^3 27.8 ms per 256^3 mixed solve,
                                       // from 16^3 27.4, from 8^3 27.0)
constexpr size_t kTailSmemMax = 100 * 1024;
constexpr long long kTailBlockCells = 4096;  // levels this small run inside one block
template <typename T>
struct TailArgs {
    TailLvl<T> lv[kTailMax];
    int n;                 // levels in lv; lv[n-1] is the coarsest
    int split;             // levels >= split (when split < n-1) run inside one block
    int pre, post, direct, mat_in_smem;
    const double *LU;
    const int *piv, *pinned;
};
size_t tail_smem(int np, int *mat_in_smem);
template <typename T>
cudaError_t tail_grid(size_t smem, int *blocks);
template <typename T>
cudaError_t launch_vtail(const TailArgs<T> &A, int blocks, size_t smem, cudaStream_t s);
// reductions (deterministic two-pass) into a device double
constexpr int kRedBlocks = 1184;  // 8 blocks of 256 threads per SM on 148 SMs
template <typename T>
cudaError_t launch_maxabs(const Lay &L, const T *x, double *part, double *out, cudaStream_t s);
template <typename T>
cudaError_t launch_dot(const Lay &L, const T *a, const T *b, double *part, double *out, cudaStream_t s);

// PCG scalars (device resident)
struct CgScal {
    double rho1, rho2, pap, alpha, beta;
    int iter, pad;
};
template <typename TZ>
cudaError_t launch_cg_rho(const Lay &L, const TZ *zz, const double *res, double *part, CgScal *sc, cudaStream_t s);
template <typename TZ>
cudaError_t launch_fcg_rho(const Lay &L, const TZ *zz, const double *res, const double *Ap, double *part, CgScal *sc,
                           cudaStream_t s);
template <typename TZ>
cudaError_t launch_cg_pap_fused(const Lay &L, const NbrOff &nb, int npt, const double *opr, const TZ *zz,
                                const double *pp_old, double *pp_new, double *Ap, double *part, CgScal *sc,
                                cudaStream_t s);
template <typename TV>
cudaError_t launch_cg_xr_fused(const Lay &L, double *sol, const double *pp, double *res, const double *Ap,
                               const CgScal *sc, float *f32, TV *vzero, double *part, double *out, cudaStream_t s);
cudaError_t launch_defect_fused(const Lay &L, const NbrOff &nb, int npt, const double *opr, const double *x_old,
                                const float *e, const double *b, double *x_new, float *f32, double *part,
                                double *out, cudaStream_t s);
cudaError_t launch_round_f32(const Lay &L, const double *r, float *f, cudaStream_t s);
// flexible CG: zz = z1 + e (z1 may be null), rho = zz.res, beta = -zz.Ap_old / pap_old
cudaError_t launch_fcg_z(const Lay &L, const double *z1, const float *e, const double *res, const double *Ap,
                         double *zz, double *part, CgScal *sc, cudaStream_t s);

// caller I/O: Fortran arrays with g overlap layers <-> level interior
template <typename T>
cudaError_t launch_from_caller(const Lay &L, const double *src, int g, T *dst, cudaStream_t s);
cudaError_t launch_to_caller(const Lay &L, const double *src, int g, double *dst, cudaStream_t s);
// FP64 level arrays <-> FP32 copies (planes)
cudaError_t launch_to_f32(const double *src, float *dst, long long n, cudaStream_t s);

}  // namespace bbmg
