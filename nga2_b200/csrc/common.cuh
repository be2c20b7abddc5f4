// common.cuh -- shared device helpers of the bbmg kernels.
#pragma once
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>

#include "layout.cuh"

namespace bbmg {

constexpr double kEps = DBL_EPSILON;  // epsilon(1.0_WP), bbmg_class.f90:880,1005

// 27-point stencil slot of offset (li,lj,lk), the reference's column-major
// order of opr(-1:1,-1:1,-1:1) (li fastest).
BB_HD int q27(int li, int lj, int lk) { return (li + 1) + 3 * (lj + 1) + 9 * (lk + 1); }
__host__ __device__ constexpr int q27h(int li, int lj, int lk) { return (li + 1) + 3 * (lj + 1) + 9 * (lk + 1); }
// prolongation slot of c2f(pi,pj,pk)
BB_HD int q8(int pi, int pj, int pk) { return pi + 2 * pj + 4 * pk; }

// The 7 offsets of a 7-point stencil in the same column-major order; the
// level-1 operator of NGA2's pressure solve uses only these (incomp_class.f90:
// 758-764) and is then stored as 7 planes in this order.
__host__ __device__ constexpr int s7x(int q) { return q == 2 ? -1 : (q == 4 ? 1 : 0); }
__host__ __device__ constexpr int s7y(int q) { return q == 1 ? -1 : (q == 5 ? 1 : 0); }
__host__ __device__ constexpr int s7z(int q) { return q == 0 ? -1 : (q == 6 ? 1 : 0); }
constexpr int kCentre7 = 3;
constexpr int kCentre27 = 13;
// 27-slot index of each 7-point slot: 4, 10, 12, 13, 14, 16, 22
__host__ __device__ constexpr int k7to27(int q) {
    return q27h(s7x(q), s7y(q), s7z(q));
}

template <int NPT> struct Sten;
template <> struct Sten<27> {
    static constexpr int centre = kCentre27;
    BB_HD static int dx(int q) { return q % 3 - 1; }
    BB_HD static int dy(int q) { return (q / 3) % 3 - 1; }
    BB_HD static int dz(int q) { return q / 9 - 1; }
};
template <> struct Sten<7> {
    static constexpr int centre = kCentre7;
    BB_HD static int dx(int q) { return s7x(q); }
    BB_HD static int dy(int q) { return s7y(q); }
    BB_HD static int dz(int q) { return s7z(q); }
};

// Solve-phase stencil layouts.  NPT = 27: the full 3x3x3 operator, 27 planes.
// NPT = 7: a 7-point operator, 7 planes in the column-major term order.
// NPT = 4: a symmetric 7-point operator, planes D, E, N, T; the west, south
// and bottom coefficients of a cell are the east, north and top ones of its
// neighbour (used only when the operator is exactly symmetric, so the values
// are bit-identical).  terms() is the number of stencil terms summed.
template <int NPT> struct Lay7 {
    static constexpr int terms = NPT == 27 ? 27 : 7;
    static constexpr int centre = NPT == 27 ? kCentre27 : kCentre7;
    // 27-slot of term q (for the neighbour offset table)
    BB_HD static int slot(int q) { return NPT == 27 ? q : k7to27(q); }
    // coefficient plane of term q
    BB_HD static int plane(int q) { return NPT == 4 ? (q < 3 ? 3 - q : q - 3) : q; }
    // true if term q's coefficient is stored at the neighbour cell
    BB_HD static bool at_nbr(int q) { return NPT == 4 && q < 3; }
};

// Element offsets of the 27 neighbours of a cell, for a cell of even x
// (off[0]) or odd x (off[1]).  In the x-split layout the offset of a
// neighbour only depends on the parity of i.
struct NbrOff {
    int off[2][27];
};

inline NbrOff make_nbr(const Lay &L) {
    NbrOff n;
    for (int par = 0; par < 2; par++) {
        int i = par ? 1 : 2;  // any interior-safe representative
        for (int q = 0; q < 27; q++) {
            int dx = q % 3 - 1, dy = (q / 3) % 3 - 1, dz = q / 9 - 1;
            n.off[par][q] = (int)(L.idx(i + dx, 1 + dy, 1 + dz) - L.idx(i, 1, 1));
        }
    }
    return n;
}

// Arithmetic that the reference's parity demands: no contraction into FMA in
// the FP64 path (EXACT), ordinary FMA in the FP32 path.
template <bool EXACT> struct Arith;
template <> struct Arith<true> {
    __device__ static __forceinline__ double mac(double s, double a, double b) { return __dadd_rn(s, __dmul_rn(a, b)); }
    __device__ static __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ static __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ static __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};
template <> struct Arith<false> {
    template <typename T> __device__ static __forceinline__ T mac(T s, T a, T b) { return fma(a, b, s); }
    template <typename T> __device__ static __forceinline__ T mul(T a, T b) { return a * b; }
    template <typename T> __device__ static __forceinline__ T add(T a, T b) { return a + b; }
    template <typename T> __device__ static __forceinline__ T sub(T a, T b) { return a - b; }
};

// Interior enumeration in storage order: the first nx/2 values of t within a
// row are the odd x (consecutive in memory), the rest the even x.
BB_HD void interior_cell(const Lay &L, long long t, int &i, int &j, int &k) {
    int nodd = L.nx >> 1;
    int ti = (int)(t % L.nx);
    long long r = t / L.nx;
    j = (int)(r % L.ny);
    k = (int)(r / L.ny);
    i = ti < nodd ? 2 * ti + 1 : 2 * (ti - nodd);
}

// Enumeration of every cell including the overlap, i, j, k in [-1, n].
BB_HD void any_cell(const Lay &L, long long t, int &i, int &j, int &k) {
    int n = L.nx + 2;
    int odd_max = (L.nx & 1) ? L.nx : L.nx - 1;
    int nodd = (odd_max + 3) / 2;  // -1, 1, 3, .., odd_max
    int ti = (int)(t % n);
    long long r = t / n;
    j = (int)(r % (L.ny + 2)) - 1;
    k = (int)(r / (L.ny + 2)) - 1;
    i = ti < nodd ? 2 * ti - 1 : 2 * (ti - nodd);
}

// Enumeration of the overlap shell only: the planes k = -1 and k = nz, then
// the rows j = -1 and j = ny of the interior planes, then the cells i = -1
// and i = nx of the interior rows.
BB_HD long long shell_cells(const Lay &L) {
    return 2LL * (L.nx + 2) * (L.ny + 2) + 2LL * (L.nx + 2) * L.nz + 2LL * L.ny * L.nz;
}
BB_HD void shell_cell(const Lay &L, long long t, int &i, int &j, int &k) {
    const long long A = (long long)(L.nx + 2) * (L.ny + 2);
    if (t < 2 * A) {
        k = t < A ? -1 : L.nz;
        const long long r = t % A;
        i = (int)(r % (L.nx + 2)) - 1;
        j = (int)(r / (L.nx + 2)) - 1;
        return;
    }
    t -= 2 * A;
    const long long B = (long long)(L.nx + 2) * L.nz;
    if (t < 2 * B) {
        j = t < B ? -1 : L.ny;
        const long long r = t % B;
        i = (int)(r % (L.nx + 2)) - 1;
        k = (int)(r / (L.nx + 2));
        return;
    }
    t -= 2 * B;
    const long long C = (long long)L.ny * L.nz;
    i = t < C ? -1 : L.nx;
    const long long r = t % C;
    j = (int)(r % L.ny);
    k = (int)(r / L.ny);
}

// Write `val` into every periodic image of interior cell (i,j,k) held in the
// overlap, reproducing the reference's vsync after a write of the interior
// (bbmg_class.f90:1388-1554 on one rank).
template <typename T>
__device__ __forceinline__ void write_images(const Lay &L, T *arr, int i, int j, int k, T val) {
    int xs[3], ys[3], zs[3];
    int nxs = 0, nys = 0, nzs = 0;
    xs[nxs++] = i;
    if (L.xper) { if (i == 0) xs[nxs++] = L.nx; if (i == L.nx - 1) xs[nxs++] = -1; }
    ys[nys++] = j;
    if (L.yper) { if (j == 0) ys[nys++] = L.ny; if (j == L.ny - 1) ys[nys++] = -1; }
    zs[nzs++] = k;
    if (L.zper) { if (k == 0) zs[nzs++] = L.nz; if (k == L.nz - 1) zs[nzs++] = -1; }
    if (nxs + nys + nzs == 3) return;
    for (int c = 0; c < nzs; c++)
        for (int b = 0; b < nys; b++)
            for (int a = 0; a < nxs; a++) {
                if (a == 0 && b == 0 && c == 0) continue;
                arr[L.idx(xs[a], ys[b], zs[c])] = val;
            }
}

__device__ __forceinline__ bool on_periodic_face(const Lay &L, int i, int j, int k) {
    return (L.xper && (i == 0 || i == L.nx - 1)) || (L.yper && (j == 0 || j == L.ny - 1)) ||
           (L.zper && (k == 0 || k == L.nz - 1));
}

// grid-stride helpers
__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long gstride() { return (long long)gridDim.x * blockDim.x; }

inline int grid_for(long long n, int block, int maxblocks = 148 * 32) {
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > maxblocks) g = maxblocks;
    return (int)g;
}

}  // namespace bbmg
