// layout.cuh -- HBM layout of one multigrid level.
//
// A level of nx*ny*nz cells carries the reference's one-cell overlap (0-based
// interior i in [0,nx), overlap at -1 and nx).  Each (j,k) row is stored with
// its x-parities split: odd i first (i = 2a+1 at position a, so the low
// overlap i = -1 sits at position -1, the last slot of the previous row), then
// even i from the row offset B0 (i = 2a at B0 + a).  A Gauss-Seidel colour
// (bbmg_class.f90:872-883) touches one x-parity of every other row, which in
// this layout is one contiguous half-row: loads are fully coalesced and no
// sector is fetched for the other colour.  Coarse point c sits over fine point
// 2c (bbmg_class.f90:794,820), i.e. at the start of the fine even half.
//
// Operator coefficients and prolongation weights are structure-of-arrays:
// plane q of a level is the same layout at q * plane elements.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define BB_HD __host__ __device__ __forceinline__
#else
#define BB_HD inline
#endif

namespace bbmg {

struct Lay {
    int nx, ny, nz;      // interior cells
    int xper, yper, zper;
    int P;               // row pitch (elements)
    int B0;              // offset of the even half within a row
    long long G;         // guard before row 0 (holds position -1 of row 0)
    long long plane;     // elements per array (multiple of 32)

    BB_HD long long row(int j, int k) const { return (long long)(k + 1) * (ny + 2) + (j + 1); }
    // odd i -> (i-1)/2 (i = -1 -> -1), even i -> B0 + i/2
    BB_HD long long idx(int i, int j, int k) const {
        int p = (i & 1) ? ((i - 1) >> 1) : (B0 + (i >> 1));
        return G + row(j, k) * P + p;
    }
};

inline int align_up(int v, int a) { return (v + a - 1) / a * a; }

inline Lay make_lay(int nx, int ny, int nz, int xper, int yper, int zper) {
    Lay L;
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.xper = xper; L.yper = yper; L.zper = zper;
    int a = nx >= 32 ? 32 : 8;
    int odd_max = (nx & 1) ? nx : nx - 1;   // largest odd i in [-1, nx]
    int even_max = (nx & 1) ? nx - 1 : nx;  // largest even i in [0, nx]
    int a1 = odd_max >= 1 ? (odd_max - 1) / 2 : -1;
    int a0 = even_max / 2;
    L.B0 = align_up(a1 + 1, a);
    L.P = align_up(L.B0 + a0 + 2, a);       // keeps P-1 free for the next row's i=-1
    L.G = 32;
    long long n = L.G + (long long)(ny + 2) * (nz + 2) * L.P + 32;
    L.plane = (n + 31) / 32 * 32;
    return L;
}

// 0-based interior index i <-> the reference's 1-based index i+1.
// Parity used by the prolongation (bbmg_class.f90:155-181): 0 when the fine
// point coincides with a coarse point, 1 when it lies between two.
BB_HD int pmod(int per, int i, int n) {
    int fi = i + 1;  // Fortran index, >= 0 wherever it is evaluated
    if (per) return 1 - ((((fi + n - 1) % n) + 1) % 2);
    return 1 - (fi % 2);
}

// wrap a 0-based index in [-1, n] into the interior for periodic directions
BB_HD int wrap(int per, int i, int n) {
    if (!per) return i;
    if (i < 0) return i + n;
    if (i >= n) return i - n;
    return i;
}

}  // namespace bbmg
