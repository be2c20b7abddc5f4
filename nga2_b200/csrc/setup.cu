// setup.cu -- operator setup of the black-box multigrid on the GPU (FP64).
//
// Every kernel restates one routine of src/solver/bbmg_class.f90 for one
// rank; the loop nests that accumulate into a coefficient keep the
// reference's order so that the FP64 results match the oracle bit for bit.
// The grid-wide work is data parallel per cell: each output cell is written
// by exactly one thread, so no atomics and no ordering between threads are
// needed.
#include "setup.cuh"

namespace bbmg {

// ---------------------------------------------------------------------------
// Level-1 operator: ils scatter of the caller's nst-point stencil into the
// 27-point layout (ils_class.f90:247-256), identity in the overlap
// (bbmg_class.f90:937-949).  src is (nst, nx+2g, ny+2g, nz+2g) Fortran order.
// caller stencil entries of each q27 slot
struct ScatterMap {
    signed char slot[27];  // q27 slot of caller entry st
    signed char one[27];   // DIRECT form: the caller entry of slot q, -1 if none
};

// Each slot's value is the sum of the caller's entries that map to it, in
// stencil order, built one slot at a time so the sums stay in registers.
// DIRECT: every slot has at most one entry (the usual stencil), so slot q is
// 0 + src[one[q]] and the loads do not depend on a search.
template <bool DIRECT>
__global__ void __launch_bounds__(128, 8) k_scatter_operator(Lay L, const double *__restrict__ src, int nst, int g,
                                                             ScatterMap map, double *__restrict__ opr,
                                                             unsigned wmask) {
    __shared__ int qst[27];
    if (!DIRECT) {
        if (threadIdx.x == 0) {
#pragma unroll
            for (int st = 0; st < 27; st++) qst[st] = map.slot[st];
        }
        __syncthreads();
    }
    long long total = (long long)(L.nx + 2) * (L.ny + 2) * (L.nz + 2);
    const long long sx = nst, sy = sx * (L.nx + 2 * g), sz = sy * (L.ny + 2 * g);
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        any_cell(L, t, i, j, k);
        long long id = L.idx(i, j, k);
        bool interior = i >= 0 && i < L.nx && j >= 0 && j < L.ny && k >= 0 && k < L.nz;
        const double *s = src + (long long)(k + g) * sz + (long long)(j + g) * sy + (long long)(i + g) * sx;
#pragma unroll
        for (int q = 0; q < 27; q++) {
            if (!((wmask >> q) & 1u)) continue;
            double o = 0.0;
            if (interior) {
                if (DIRECT) {
                    if (map.one[q] >= 0) o = __dadd_rn(o, s[map.one[q]]);
                } else {
#pragma unroll 1
                    for (int st = 0; st < nst; st++)
                        if (qst[st] == q) o = __dadd_rn(o, s[st]);
                }
            } else if (q == kCentre27) {
                o = 1.0;
            }
            opr[q * L.plane + id] = o;
        }
    }
}

// ---------------------------------------------------------------------------
// Periodic copy of the overlap for nplanes planes (msync / vsync on one rank,
// bbmg_class.f90:1388-1724).  The reference copies x, then y, then z over the
// full extent of the other directions; the result is that every overlap cell
// with a coordinate outside the interior of a periodic direction holds the
// value of the cell obtained by wrapping those coordinates.  The sources are
// never themselves periodic images, so one gather pass reproduces it.
// Only the overlap shell is visited (2 ((nx+2)(ny+2) + (nx+2) nz + ny nz)
// cells), and only the planes in `mask`.
__global__ void k_wrap(Lay L, double *__restrict__ a, unsigned mask) {
    const long long total = shell_cells(L);
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        shell_cell(L, t, i, j, k);
        int si = wrap(L.xper, i, L.nx), sj = wrap(L.yper, j, L.ny), sk = wrap(L.zper, k, L.nz);
        if (si == i && sj == j && sk == k) continue;
        long long d = L.idx(i, j, k), s = L.idx(si, sj, sk);
        // all loads before the stores: the image is interior and the
        // destination is not, but the compiler cannot know, and a load after
        // each store would wait out the previous store's latency
        double v[27];
#pragma unroll
        for (int q = 0; q < 27; q++)
            if ((mask >> q) & 1u) v[q] = a[q * L.plane + s];
#pragma unroll
        for (int q = 0; q < 27; q++)
            if ((mask >> q) & 1u) a[q * L.plane + d] = v[q];
    }
}
__global__ void k_wrap_f(Lay L, float *__restrict__ a, int nplanes) {
    const long long total = shell_cells(L);
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        shell_cell(L, t, i, j, k);
        int si = wrap(L.xper, i, L.nx), sj = wrap(L.yper, j, L.ny), sk = wrap(L.zper, k, L.nz);
        if (si == i && sj == j && sk == k) continue;
        long long d = L.idx(i, j, k), s = L.idx(si, sj, sk);
        float v[27];  // loads first, as in k_wrap
#pragma unroll
        for (int q = 0; q < 27; q++)
            if (q < nplanes) v[q] = a[q * L.plane + s];
#pragma unroll
        for (int q = 0; q < 27; q++)
            if (q < nplanes) a[q * L.plane + d] = v[q];
    }
}
// The overlap shell after a kernel that wrote the interior: a shell cell that
// lies outside in a non-periodic direction is zero, any other takes its
// periodic image (an interior cell).  The same values as zeroing the shell
// and then running k_wrap on every plane, in one pass; a32, if given,
// receives the FP32 copy of what is written.
__global__ void k_fill_shell(Lay L, double *__restrict__ a, int nplanes, float *__restrict__ a32) {
    const long long total = shell_cells(L);
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        shell_cell(L, t, i, j, k);
        const bool out = (!L.xper && (i < 0 || i >= L.nx)) || (!L.yper && (j < 0 || j >= L.ny)) ||
                         (!L.zper && (k < 0 || k >= L.nz));
        const long long d = L.idx(i, j, k);
        if (out) {
            for (int q = 0; q < nplanes; q++) a[q * L.plane + d] = 0.0;
            if (a32)
                for (int q = 0; q < nplanes; q++) a32[q * L.plane + d] = 0.0f;
            continue;
        }
        const long long s = L.idx(wrap(L.xper, i, L.nx), wrap(L.yper, j, L.ny), wrap(L.zper, k, L.nz));
        double v[27];  // all loads before the stores, as in k_wrap
#pragma unroll
        for (int q = 0; q < 27; q++)
            if (q < nplanes) v[q] = a[q * L.plane + s];
#pragma unroll
        for (int q = 0; q < 27; q++)
            if (q < nplanes) a[q * L.plane + d] = v[q];
        if (a32) {
#pragma unroll
            for (int q = 0; q < 27; q++)
                if (q < nplanes) a32[q * L.plane + d] = (float)v[q];
        }
    }
}

// Solve-phase planes of a level that keeps fewer than 27 (the level-1 4- or
// 7-point storage): plane q of oprS is plane slot[q] of the 27-plane opr;
// oprS32, if given, receives the FP32 copy.  Every element of the arrays
// (guards and padding included), as a plane-by-plane copy.
struct PlaneSlots {
    int n;
    int slot[7];
};
__global__ void k_solve_planes(long long P, const double *__restrict__ opr, PlaneSlots ps, double *__restrict__ oprS,
                               float *__restrict__ oprS32) {
    for (long long t = gtid(); t < P; t += gstride()) {
        for (int q = 0; q < ps.n; q++) {
            const double v = opr[(long long)ps.slot[q] * P + t];
            oprS[q * P + t] = v;
            if (oprS32) oprS32[q * P + t] = (float)v;
        }
    }
}


__device__ __forceinline__ double sgn_clamp(double a) {
    // sign(max(abs(a),epsilon(1.0_WP)),a)
    return copysign(fmax(fabs(a), kEps), a);
}

// ---------------------------------------------------------------------------
// Prolongation, sweep 1: identity and 1-D lines with Shapira lumping
// (bbmg_class.f90:978-1051).  Every cell including the overlap.
__global__ void k_prolong_sweep1(Lay L, const double *__restrict__ opr, double *__restrict__ c2f, unsigned mask) {
    const double ratio = 10.0;
    long long total = (long long)(L.nx + 2) * (L.ny + 2) * (L.nz + 2);
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        any_cell(L, t, i, j, k);
        long long id = L.idx(i, j, k);
        int n1 = pmod(L.xper, i, L.nx), n2 = pmod(L.yper, j, L.ny), n3 = pmod(L.zper, k, L.nz);
        // c2f(0,0,0) and the one line weight (slot sx); every other weight is zero.
        // Scalars rather than an array indexed at run time, so nothing goes to local memory.
        double c0 = 0.0, cx = 0.0;
        int sx = -1;
        int sum = n1 + n2 + n3;
        if (sum == 0) {
            c0 = 1.0;
        } else if (sum == 1) {
            double m = 0.0, z = 0.0, p = 0.0;  // opr1d(-1), opr1d(0), opr1d(+1)
            // unrolled: the loads of all planes can be in flight together
#pragma unroll
            for (int q = 0; q < 27; q++) {
                if (!((mask >> q) & 1u)) continue;  // an all-zero plane adds only zeros
                int li = q % 3 - 1, lj = (q / 3) % 3 - 1, lk = q / 9 - 1;
                int l = n1 ? li : (n2 ? lj : lk);
                int ax = n1 ? q27(li, 0, 0) : (n2 ? q27(0, lj, 0) : q27(0, 0, lk));
                double a = opr[q * L.plane + id];
                if (__dmul_rn(ratio, fabs(opr[ax * L.plane + id])) >= fabs(a)) {
                    if (l < 0) m = __dadd_rn(m, a);
                    else if (l == 0) z = __dadd_rn(z, a);
                    else p = __dadd_rn(p, a);
                } else {
                    z = __dadd_rn(z, a);
                }
            }
            z = sgn_clamp(z);
            c0 = -m / z;
            cx = -p / z;
            sx = n1 ? q8(1, 0, 0) : (n2 ? q8(0, 1, 0) : q8(0, 0, 1));
        }
#pragma unroll
        for (int s = 0; s < 8; s++) c2f[s * L.plane + id] = s == 0 ? c0 : (s == sx ? cx : 0.0);
    }
}

// Prolongation, sweep 2: 2-D faces (bbmg_class.f90:1052-1160).  Reads the
// line weights of the in-plane neighbours written by sweep 1.  AXN is the
// plane normal (0: yz-plane, 1: zx-plane, 2: xy-plane); PA is the in-plane
// axis of the reference's inner loop, PB that of its outer loop.
// zinit: the cell's weights start from the zeros sweep 1 would have written
// (it skipped the cell); c2f32, if given, receives the FP32 copy.
template <int AXN>
__device__ __forceinline__ void face_weights(const Lay &L, const double *__restrict__ opr, double *__restrict__ c2f,
                                             int i, int j, int k, unsigned mask, bool zinit = false,
                                             float *__restrict__ c2f32 = nullptr) {
    constexpr int PA = AXN == 0 ? 1 : 0;
    constexpr int PB = AXN == 2 ? 1 : 2;
    const double ratio = 10.0;
    const int ia[3] = {i, j, k};
    const int na[3] = {L.nx, L.ny, L.nz};
    if (ia[PA] == -1 || ia[PA] == na[PA] || ia[PB] == -1 || ia[PB] == na[PB]) return;
    const long long id = L.idx(i, j, k);
    // opr2d(a,b) at (a+1) + 3(b+1).  The loops are unrolled so every index
    // into o2 and c is a compile-time constant: both stay in registers.
    double o2[9];
#pragma unroll
    for (int e = 0; e < 9; e++) o2[e] = 0.0;
#pragma unroll
    for (int q = 0; q < 27; q++) {
        if (!((mask >> q) & 1u)) continue;  // an all-zero plane adds only zeros
        const int l[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
        const int la = l[PA], lb = l[PB];
        int lr[3] = {l[0], l[1], l[2]};
        lr[AXN] = 0;
        const double a = opr[q * L.plane + id];
        const int e1 = (la + 1) + 3 * (lb + 1);
        if (__dmul_rn(ratio, fabs(opr[q27(lr[0], lr[1], lr[2]) * L.plane + id])) >= fabs(a))
            o2[e1] = __dadd_rn(o2[e1], a);
        else
            o2[4] = __dadd_rn(o2[4], a);
    }
    const double o00 = sgn_clamp(o2[4]);
    double c[8];
#pragma unroll
    for (int t = 0; t < 8; t++) c[t] = zinit ? 0.0 : c2f[t * L.plane + id];
#pragma unroll
    for (int lb = -1; lb <= 1; lb++)
#pragma unroll
        for (int la = -1; la <= 1; la++) {
            if (la == 0 && lb == 0) continue;
            int off[3] = {0, 0, 0};
            off[PA] = la; off[PB] = lb;
            const long long nid = L.idx(i + off[0], j + off[1], k + off[2]);
            const double w = o2[(la + 1) + 3 * (lb + 1)] / o00;
#pragma unroll
            for (int qb = 0; qb <= 1 - abs(lb); qb++)
#pragma unroll
                for (int qa = 0; qa <= 1 - abs(la); qa++) {
                    int s3[3] = {0, 0, 0}, p3[3] = {0, 0, 0};
                    s3[PA] = (la + 1) / 2 + qa; s3[PB] = (lb + 1) / 2 + qb;
                    p3[PA] = qa; p3[PB] = qb;
                    const int so = q8(s3[0], s3[1], s3[2]);
                    const double cn = c2f[q8(p3[0], p3[1], p3[2]) * L.plane + nid];
                    c[so] = __dsub_rn(c[so], __dmul_rn(w, cn));
                }
        }
#pragma unroll
    for (int t = 0; t < 8; t++) c2f[t * L.plane + id] = c[t];
    if (c2f32) {
#pragma unroll
        for (int t = 0; t < 8; t++) c2f32[t * L.plane + id] = (float)c[t];
    }
}

__global__ void k_prolong_sweep2(Lay L, const double *__restrict__ opr, double *__restrict__ c2f, unsigned mask) {
    long long total = (long long)(L.nx + 2) * (L.ny + 2) * (L.nz + 2);
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        any_cell(L, t, i, j, k);
        int n1 = pmod(L.xper, i, L.nx), n2 = pmod(L.yper, j, L.ny), n3 = pmod(L.zper, k, L.nz);
        if (n1 + n2 + n3 != 2) continue;
        if (n1 == 0) face_weights<0>(L, opr, c2f, i, j, k, mask);
        else if (n2 == 0) face_weights<1>(L, opr, c2f, i, j, k, mask);
        else face_weights<2>(L, opr, c2f, i, j, k, mask);
    }
}

// Prolongation, sweep 3: cube centres, interior only (bbmg_class.f90:1161-1194).
__device__ __forceinline__ void cube_weights(const Lay &L, const double *__restrict__ opr, double *__restrict__ c2f,
                                             int i, int j, int k, unsigned mask, bool zinit = false,
                                             float *__restrict__ c2f32 = nullptr) {
        long long id = L.idx(i, j, k);
        double d = sgn_clamp(opr[kCentre27 * L.plane + id]);
        double c[8];
#pragma unroll
        for (int s = 0; s < 8; s++) c[s] = zinit ? 0.0 : c2f[s * L.plane + id];
        // unrolled: every index into c is a compile-time constant (registers)
#pragma unroll 27
        for (int q = 0; q < 27; q++) {
            if (q == kCentre27 || !((mask >> q) & 1u)) continue;  // an all-zero plane subtracts only zeros
            const int li = q % 3 - 1, lj = (q / 3) % 3 - 1, lk = q / 9 - 1;
            const int ni = li ? 1 : 2, nj = lj ? 1 : 2, nk = lk ? 1 : 2;  // prolongation weights per direction
            long long nid = L.idx(i + li, j + lj, k + lk);
            double w = opr[q * L.plane + id] / d;
#pragma unroll 2
            for (int pk = 0; pk < nk; pk++)
#pragma unroll 2
                for (int pj = 0; pj < nj; pj++)
#pragma unroll 2
                    for (int pi = 0; pi < ni; pi++) {
                        int so = q8((li + 1) / 2 + pi, (lj + 1) / 2 + pj, (lk + 1) / 2 + pk);
                        c[so] = __dsub_rn(c[so], __dmul_rn(w, c2f[q8(pi, pj, pk) * L.plane + nid]));
                    }
        }
#pragma unroll
        for (int s = 0; s < 8; s++) c2f[s * L.plane + id] = c[s];
        if (c2f32) {
#pragma unroll
            for (int s = 0; s < 8; s++) c2f32[s * L.plane + id] = (float)c[s];
        }
}

__global__ void k_prolong_sweep3(Lay L, const double *__restrict__ opr, double *__restrict__ c2f, unsigned mask) {
    long long total = (long long)L.nx * L.ny * L.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int i, j, k;
        interior_cell(L, t, i, j, k);
        int n1 = pmod(L.xper, i, L.nx), n2 = pmod(L.yper, j, L.ny), n3 = pmod(L.zper, k, L.nz);
        if (n1 + n2 + n3 != 3) continue;
        cube_weights(L, opr, c2f, i, j, k, mask);
    }
}

// ---------------------------------------------------------------------------
// Even levels (nx, ny, nz all even).  There pmod(i) is the parity of i for
// every i in [-1, n], periodic or not, so a cell's parity class (i, j, k mod
// 2) fixes which prolongation sweep writes it and, in the Galerkin products,
// every loop bound and accumulator slot.  The kernels below enumerate only
// the cells a sweep updates, and give each parity class its own unrolled code
// with the accumulators in registers; every sum keeps the reference's order,
// so the results are the same bits as the generic kernels above (which serve
// the odd-sized levels).

// Sweep 1 on an even level, where a cell's parity class never changes: only
// the point cells (three even indices) and the line cells (one odd index),
// one class per blockIdx.y (0 points, 1 + AX lines along AX), each writing
// the planes that can be nonzero (0, and the line's plane sx); the other
// planes of these cells hold the zeros of the allocation.  The face and cube
// cells are left to sweeps 2 and 3 (or, with an index -1, hold zeros or their
// periodic image, written by the overlap copy).  c2f32, if given, receives the
// FP32 copy.  Each class enumerates (nx/2+1)(ny/2+1)(nz/2+1) cells: an odd
// index runs over -1, 1, .., n-1, an even one over 0, 2, .., n.
template <int AX>
__device__ __forceinline__ void line_weights(const Lay &L, const double *__restrict__ opr, double *__restrict__ c2f,
                                             float *__restrict__ c2f32, unsigned mask, long long id) {
    const double ratio = 10.0;
    double m = 0.0, z = 0.0, p = 0.0;  // opr1d(-1), opr1d(0), opr1d(+1)
#pragma unroll
    for (int q = 0; q < 27; q++) {
        if (!((mask >> q) & 1u)) continue;  // an all-zero plane adds only zeros
        const int li = q % 3 - 1, lj = (q / 3) % 3 - 1, lk = q / 9 - 1;
        const int l = AX == 0 ? li : (AX == 1 ? lj : lk);
        const int ax = AX == 0 ? q27(li, 0, 0) : (AX == 1 ? q27(0, lj, 0) : q27(0, 0, lk));
        const double a = opr[q * L.plane + id];
        if (__dmul_rn(ratio, fabs(opr[ax * L.plane + id])) >= fabs(a)) {
            if (l < 0) m = __dadd_rn(m, a);
            else if (l == 0) z = __dadd_rn(z, a);
            else p = __dadd_rn(p, a);
        } else {
            z = __dadd_rn(z, a);
        }
    }
    z = sgn_clamp(z);
    const double c0 = -m / z, cx = -p / z;
    constexpr int sx = AX == 0 ? 1 : (AX == 1 ? 2 : 4);
    c2f[id] = c0;
    c2f[sx * L.plane + id] = cx;
    if (c2f32) {
        c2f32[id] = (float)c0;
        c2f32[sx * L.plane + id] = (float)cx;
    }
}

__global__ void k_prolong_sweep1_even(Lay L, const double *__restrict__ opr, double *__restrict__ c2f,
                                      unsigned mask, float *__restrict__ c2f32) {
    const int cls = blockIdx.y;
    const long long ax = L.nx / 2 + 1, ay = L.ny / 2 + 1, total = ax * ay * (L.nz / 2 + 1);
    for (long long t = gtid(); t < total; t += gstride()) {
        const long long u = t / ax;
        const int a = (int)(t % ax), b = (int)(u % ay), c = (int)(u / ay);
        const int i = 2 * a - (cls == 1), j = 2 * b - (cls == 2), k = 2 * c - (cls == 3);
        const long long id = L.idx(i, j, k);
        switch (cls) {
            case 0:
                c2f[id] = 1.0;
                if (c2f32) c2f32[id] = 1.0f;
                break;
            case 1: line_weights<0>(L, opr, c2f, c2f32, mask, id); break;
            case 2: line_weights<1>(L, opr, c2f, c2f32, mask, id); break;
            default: line_weights<2>(L, opr, c2f, c2f32, mask, id); break;
        }
    }
}

// Sweep 2, face cells only: the normal index even in [0, n] (the overlap n
// included), the two in-plane indices odd and interior -- the cells of
// k_prolong_sweep2 that face_weights does not skip.
__global__ void k_prolong_sweep2_even(Lay L, const double *__restrict__ opr, double *__restrict__ c2f,
                                      unsigned mask, float *__restrict__ c2f32) {
    const long long hx = L.nx / 2, hy = L.ny / 2, hz = L.nz / 2;
    const long long n0 = (hx + 1) * hy * hz, n1 = hx * (hy + 1) * hz, n2 = hx * hy * (hz + 1);
    for (long long t = gtid(); t < n0 + n1 + n2; t += gstride()) {
        if (t < n0) {
            const long long u = t / (hx + 1);
            face_weights<0>(L, opr, c2f, (int)(2 * (t % (hx + 1))), (int)(2 * (u % hy) + 1), (int)(2 * (u / hy) + 1),
                            mask, true, c2f32);
        } else if (t < n0 + n1) {
            const long long v = t - n0, u = v / hx;
            face_weights<1>(L, opr, c2f, (int)(2 * (v % hx) + 1), (int)(2 * (u % (hy + 1))), (int)(2 * (u / (hy + 1)) + 1),
                            mask, true, c2f32);
        } else {
            const long long v = t - n0 - n1, u = v / hx;
            face_weights<2>(L, opr, c2f, (int)(2 * (v % hx) + 1), (int)(2 * (u % hy) + 1), (int)(2 * (u / hy)), mask,
                            true, c2f32);
        }
    }
}

// Sweep 3, the interior cells with three odd indices only.
__global__ void k_prolong_sweep3_even(Lay L, const double *__restrict__ opr, double *__restrict__ c2f,
                                      unsigned mask, float *__restrict__ c2f32) {
    const long long hx = L.nx / 2, hy = L.ny / 2, hz = L.nz / 2;
    for (long long t = gtid(); t < hx * hy * hz; t += gstride()) {
        const long long u = t / hx;
        cube_weights(L, opr, c2f, (int)(2 * (t % hx) + 1), (int)(2 * (u % hy) + 1), (int)(2 * (u / hy) + 1), mask, true,
                     c2f32);
    }
}

// A P at one fine cell of parity class (PX, PY, PZ), ap_cell's loops with
// compile-time bounds (the parity of a neighbour at offset l is that of the
// cell plus |l|).  SEVEN: the operator has only the centre and the six face
// planes.  Slots with s = -1 in a direction of odd parity are never reached
// and never read by R (A P); they are not written (the array is zeroed when
// allocated and stays zero there).  With SEVEN a slot is reached only if at
// most one of its components is nonzero in a direction of even parity (one
// face neighbour moves one index); the others hold zero (the array is zeroed
// whenever the level-1 stencil changes) and are not written either.
template <int PX, int PY, int PZ, bool SEVEN>
__device__ __forceinline__ void ap_fast(const Lay &F, const double *__restrict__ opr, const double *__restrict__ c2f,
                                        double *__restrict__ oprc2f, unsigned mask, int fi, int fj, int fk) {
    const long long id = F.idx(fi, fj, fk);
    double acc[27];
#pragma unroll
    for (int q = 0; q < 27; q++) acc[q] = 0.0;
#pragma unroll
    for (int q = 0; q < 27; q++) {
        const int li = q % 3 - 1, lj = (q / 3) % 3 - 1, lk = q / 9 - 1;
        if (SEVEN && (li != 0) + (lj != 0) + (lk != 0) > 1) continue;
        if (!((mask >> q) & 1u)) continue;  // an all-zero plane adds only zeros
        const int pxl = (PX + (li & 1)) & 1, pyl = (PY + (lj & 1)) & 1, pzl = (PZ + (lk & 1)) & 1;
        const double o = opr[q * F.plane + id];
        const long long nid = F.idx(fi + li, fj + lj, fk + lk);
#pragma unroll 2
        for (int pk = 0; pk <= pzl; pk++)
#pragma unroll 2
            for (int pj = 0; pj <= pyl; pj++)
#pragma unroll 2
                for (int pi = 0; pi <= pxl; pi++) {
                    const int si = pi + (1 - PX) * min(li, 0) + (1 - pxl) * max(li, 0);
                    const int sj = pj + (1 - PY) * min(lj, 0) + (1 - pyl) * max(lj, 0);
                    const int sk = pk + (1 - PZ) * min(lk, 0) + (1 - pzl) * max(lk, 0);
                    const int so = q27(si, sj, sk);
                    acc[so] = __dadd_rn(acc[so], __dmul_rn(o, c2f[q8(pi, pj, pk) * F.plane + nid]));
                }
    }
#pragma unroll
    for (int q = 0; q < 27; q++) {
        const int sx = q % 3 - 1, sy = (q / 3) % 3 - 1, sz = q / 9 - 1;
        if ((PX && sx < 0) || (PY && sy < 0) || (PZ && sz < 0)) continue;
        if (SEVEN && (!PX && sx != 0) + (!PY && sy != 0) + (!PZ && sz != 0) > 1) continue;
        oprc2f[q * F.plane + id] = acc[q];
    }
}

// One parity class per blockIdx.y: the blocks of a class are dispatched
// together, so an SM runs one class's code at a time (the eight unrolled
// classes together overflow the instruction cache).  Within a class, t runs
// over the cells i = 2a + PX, j = 2b + PY, k = 2c + PZ (a fastest).
template <bool SEVEN>
__global__ void __launch_bounds__(128) k_rap_ap_even(Lay F, const double *__restrict__ opr,
                                                     const double *__restrict__ c2f, double *__restrict__ oprc2f,
                                                     unsigned mask) {
    const int cls = blockIdx.y;
    const int px = cls & 1, py = (cls >> 1) & 1, pz = cls >> 2;
    const long long hx = F.nx / 2, hy = F.ny / 2, total = hx * hy * (F.nz / 2);
    for (long long t = gtid(); t < total; t += gstride()) {
        const long long u = t / hx;
        const int fi = (int)(2 * (t % hx)) + px, fj = (int)(2 * (u % hy)) + py, fk = (int)(2 * (u / hy)) + pz;
        switch (cls) {
            case 0: ap_fast<0, 0, 0, SEVEN>(F, opr, c2f, oprc2f, mask, fi, fj, fk); break;
            case 1: ap_fast<1, 0, 0, SEVEN>(F, opr, c2f, oprc2f, mask, fi, fj, fk); break;
            case 2: ap_fast<0, 1, 0, SEVEN>(F, opr, c2f, oprc2f, mask, fi, fj, fk); break;
            case 3: ap_fast<1, 1, 0, SEVEN>(F, opr, c2f, oprc2f, mask, fi, fj, fk); break;
            case 4: ap_fast<0, 0, 1, SEVEN>(F, opr, c2f, oprc2f, mask, fi, fj, fk); break;
            case 5: ap_fast<1, 0, 1, SEVEN>(F, opr, c2f, oprc2f, mask, fi, fj, fk); break;
            case 6: ap_fast<0, 1, 1, SEVEN>(F, opr, c2f, oprc2f, mask, fi, fj, fk); break;
            default: ap_fast<1, 1, 1, SEVEN>(F, opr, c2f, oprc2f, mask, fi, fj, fk); break;
        }
    }
}

// R (A P) at one coarse cell, the 9 output slots with z offset SK.  The fine
// centre 2c is even, so the fine offsets r run over -1..1 and the A P slots l
// from -1 + |r| to 1 in every direction; for given r and SK the z slot of A P
// is lk = SK - (rk - 1) / 2.  Each output slot's contributions come in the
// reference's (rk, rj, ri) order, a subsequence of k_rap_rap's loop.  A fine
// cell in the overlap is read at its periodic image (the value the overlap
// copy would hold there; in a non-periodic direction the overlap of A P is
// never written and stays zero), so A P's overlap is not filled during the
// setup.
template <int SK, bool SEVEN>
__device__ __forceinline__ void rap_fast(const Lay &F, const Lay &C, const double *__restrict__ f2c,
                                         const double *__restrict__ oprc2f, double *__restrict__ oprc,
                                         float *__restrict__ oprc32, int ci, int cj, int ck) {
    const int fi = 2 * ci, fj = 2 * cj, fk = 2 * ck;
    const long long cid = C.idx(ci, cj, ck);
    double acc[9];
#pragma unroll
    for (int q = 0; q < 9; q++) acc[q] = 0.0;
#pragma unroll
    for (int rk = -1; rk <= 1; rk++) {
        const int lk = SK - (rk - 1) / 2;  // (r-1)/2 truncates toward zero, as Fortran's integer division
        if (lk < -1 + (rk & 1) || lk > 1) continue;
#pragma unroll
        for (int rj = -1; rj <= 1; rj++)
#pragma unroll
            for (int ri = -1; ri <= 1; ri++) {
                const double w = f2c[q27(ri, rj, rk) * C.plane + cid];
                const long long nid = F.idx(wrap(F.xper, fi + ri, F.nx), wrap(F.yper, fj + rj, F.ny),
                                            wrap(F.zper, fk + rk, F.nz));
#pragma unroll
                for (int lj = -1; lj <= 1; lj++) {
                    if (lj < -1 + (rj & 1)) continue;
#pragma unroll
                    for (int li = -1; li <= 1; li++) {
                        if (li < -1 + (ri & 1)) continue;
                        // a 7-point fine operator leaves this slot of A P zero
                        // (fine parity is even where r = 0): adding w * 0 to a
                        // sum that starts at +0 changes no bit
                        if (SEVEN && (ri == 0 && li != 0) + (rj == 0 && lj != 0) + (rk == 0 && lk != 0) > 1) continue;
                        const int so = ((ri - 1) / 2 + li + 1) + 3 * ((rj - 1) / 2 + lj + 1);
                        acc[so] = __dadd_rn(acc[so], __dmul_rn(w, oprc2f[q27(li, lj, lk) * F.plane + nid]));
                    }
                }
            }
    }
#pragma unroll
    for (int q = 0; q < 9; q++) oprc[(q + 9 * (SK + 1)) * C.plane + cid] = acc[q];
    if (oprc32) {
#pragma unroll
        for (int q = 0; q < 9; q++) oprc32[(q + 9 * (SK + 1)) * C.plane + cid] = (float)acc[q];
    }
}

// One warp per 32 consecutive coarse cells and one z slot: warp w takes the
// slot SK = w % 3 - 1 of the cells 32 (w / 3) .. + 31.  oprc32, if given,
// receives the FP32 copy.  SEVEN: the fine operator is 7-point.
template <bool SEVEN>
__global__ void __launch_bounds__(128) k_rap_rap_even(Lay F, Lay C, const double *__restrict__ f2c,
                                                      const double *__restrict__ oprc2f, double *__restrict__ oprc,
                                                      float *__restrict__ oprc32) {
    const long long total = (long long)C.nx * C.ny * C.nz;
    const long long nw = 3 * ((total + 31) / 32);
    const int lane = threadIdx.x & 31;
    for (long long w = gtid() >> 5; w < nw; w += gstride() >> 5) {
        const long long t = (w / 3) * 32 + lane;
        if (t >= total) continue;
        int ci, cj, ck;
        interior_cell(C, t, ci, cj, ck);
        switch ((int)(w % 3)) {
            case 0: rap_fast<-1, SEVEN>(F, C, f2c, oprc2f, oprc, oprc32, ci, cj, ck); break;
            case 1: rap_fast<0, SEVEN>(F, C, f2c, oprc2f, oprc, oprc32, ci, cj, ck); break;
            default: rap_fast<1, SEVEN>(F, C, f2c, oprc2f, oprc, oprc32, ci, cj, ck); break;
        }
    }
}

static bool even_level(const Lay &L) { return !(L.nx & 1) && !(L.ny & 1) && !(L.nz & 1); }

// BBMG_GENERIC_SETUP=1 keeps the generic kernels on every level (for timing)
static bool fast_setup() {
    static int f = -1;
    if (f < 0) {
        const char *e = getenv("BBMG_GENERIC_SETUP");
        f = (e && atoi(e)) ? 0 : 1;
    }
    return f == 1;
}

// Restriction weights of a coarse cell on an even fine level: every offset
// r runs over -1..1 (unrolled), so all 27 weights are written.
__global__ void k_restriction_weights_even(Lay F, Lay C, const double *__restrict__ c2f, double *__restrict__ f2c) {
    const long long total = (long long)C.nx * C.ny * C.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int ci, cj, ck;
        interior_cell(C, t, ci, cj, ck);
        const int fi = 2 * ci, fj = 2 * cj, fk = 2 * ck;
        const long long cid = C.idx(ci, cj, ck);
#pragma unroll
        for (int rk = -1; rk <= 1; rk++)
#pragma unroll
            for (int rj = -1; rj <= 1; rj++)
#pragma unroll
                for (int ri = -1; ri <= 1; ri++)
                    f2c[q27(ri, rj, rk) * C.plane + cid] =
                        c2f[q8((1 - ri) / 2, (1 - rj) / 2, (1 - rk) / 2) * F.plane + F.idx(fi + ri, fj + rj, fk + rk)];
    }
}

// ---------------------------------------------------------------------------
// Restriction weights f2c(r, c) = c2f((1-r)/2, 2c+r) over the parity ranges
// (bbmg_class.f90:1201-1231).  F is the fine level, C the coarse one; f2c is
// zero beforehand.
__global__ void k_restriction_weights(Lay F, Lay C, const double *__restrict__ c2f, double *__restrict__ f2c) {
    long long total = (long long)C.nx * C.ny * C.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int ci, cj, ck;
        interior_cell(C, t, ci, cj, ck);
        int fi = 2 * ci, fj = 2 * cj, fk = 2 * ck;
        long long cid = C.idx(ci, cj, ck);
        int rk0 = -pmod(F.zper, fk - 1, F.nz), rk1 = pmod(F.zper, fk + 1, F.nz);
        int rj0 = -pmod(F.yper, fj - 1, F.ny), rj1 = pmod(F.yper, fj + 1, F.ny);
        int ri0 = -pmod(F.xper, fi - 1, F.nx), ri1 = pmod(F.xper, fi + 1, F.nx);
        for (int rk = rk0; rk <= rk1; rk++)
            for (int rj = rj0; rj <= rj1; rj++)
                for (int ri = ri0; ri <= ri1; ri++) {
                    int pi = (1 - ri) / 2, pj = (1 - rj) / 2, pk = (1 - rk) / 2;
                    f2c[q27(ri, rj, rk) * C.plane + cid] =
                        c2f[q8(pi, pj, pk) * F.plane + F.idx(fi + ri, fj + rj, fk + rk)];
                }
    }
}

// ---------------------------------------------------------------------------
// Galerkin operator, part 1: oprc2f = A P at one fine interior cell
// (bbmg_class.f90:1245-1271), the 27 sums in the reference's order.  The
// accumulators are indexed at run time, so they live in shared memory (slot q
// at acc[q * AS]: with AS the block's thread count a warp's accesses fall in
// distinct banks), not in a per-thread local array that spills to L2.
__device__ __forceinline__ void ap_cell(const Lay &F, const double *__restrict__ opr, const double *__restrict__ c2f,
                                        unsigned mask, int fi, int fj, int fk, double *acc, int AS) {
    const long long id = F.idx(fi, fj, fk);
    const int px0 = pmod(F.xper, fi, F.nx), py0 = pmod(F.yper, fj, F.ny), pz0 = pmod(F.zper, fk, F.nz);
#pragma unroll
    for (int q = 0; q < 27; q++) acc[q * AS] = 0.0;
#pragma unroll 1
    for (int q = 0; q < 27; q++) {
        if (!((mask >> q) & 1u)) continue;  // an all-zero plane adds only zeros
        int li = q % 3 - 1, lj = (q / 3) % 3 - 1, lk = q / 9 - 1;
        int pxl = pmod(F.xper, fi + li, F.nx), pyl = pmod(F.yper, fj + lj, F.ny), pzl = pmod(F.zper, fk + lk, F.nz);
        double o = opr[q * F.plane + id];
        long long nid = F.idx(fi + li, fj + lj, fk + lk);
        for (int pk = 0; pk <= pzl; pk++)
            for (int pj = 0; pj <= pyl; pj++)
                for (int pi = 0; pi <= pxl; pi++) {
                    int si = pi + (1 - px0) * min(li, 0) + (1 - pxl) * max(li, 0);
                    int sj = pj + (1 - py0) * min(lj, 0) + (1 - pyl) * max(lj, 0);
                    int sk = pk + (1 - pz0) * min(lk, 0) + (1 - pzl) * max(lk, 0);
                    int so = q27(si, sj, sk);
                    acc[so * AS] = __dadd_rn(acc[so * AS], __dmul_rn(o, c2f[q8(pi, pj, pk) * F.plane + nid]));
                }
    }
}

// oprc2f = A P on the whole fine interior.
__global__ void k_rap_ap(Lay F, const double *__restrict__ opr, const double *__restrict__ c2f,
                         double *__restrict__ oprc2f, unsigned mask) {
    extern __shared__ double rap_sm[];
    double *acc = rap_sm + threadIdx.x;
    const int AS = blockDim.x;
    long long total = (long long)F.nx * F.ny * F.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int fi, fj, fk;
        interior_cell(F, t, fi, fj, fk);
        ap_cell(F, opr, c2f, mask, fi, fj, fk, acc, AS);
        const long long id = F.idx(fi, fj, fk);
#pragma unroll
        for (int q = 0; q < 27; q++) oprc2f[q * F.plane + id] = acc[q * AS];
    }
}

// Galerkin operator, part 2: A_c = R (A P) on the coarse interior
// (bbmg_class.f90:1274-1300), accumulators in shared memory as in k_rap_ap.
// opr_c is zero beforehand.
__global__ void k_rap_rap(Lay F, Lay C, const double *__restrict__ f2c, const double *__restrict__ oprc2f,
                          double *__restrict__ oprc) {
    extern __shared__ double rap_sm[];
    double *acc = rap_sm + threadIdx.x;
    const int AS = blockDim.x;
    long long total = (long long)C.nx * C.ny * C.nz;
    for (long long t = gtid(); t < total; t += gstride()) {
        int ci, cj, ck;
        interior_cell(C, t, ci, cj, ck);
        int fi = 2 * ci, fj = 2 * cj, fk = 2 * ck;
        long long cid = C.idx(ci, cj, ck);
#pragma unroll
        for (int q = 0; q < 27; q++) acc[q * AS] = 0.0;
        int rk0 = -pmod(F.zper, fk - 1, F.nz), rk1 = pmod(F.zper, fk + 1, F.nz);
        int rj0 = -pmod(F.yper, fj - 1, F.ny), rj1 = pmod(F.yper, fj + 1, F.ny);
        int ri0 = -pmod(F.xper, fi - 1, F.nx), ri1 = pmod(F.xper, fi + 1, F.nx);
#pragma unroll 1
        for (int rk = rk0; rk <= rk1; rk++)
#pragma unroll 1
            for (int rj = rj0; rj <= rj1; rj++)
#pragma unroll 1
                for (int ri = ri0; ri <= ri1; ri++) {
                    double w = f2c[q27(ri, rj, rk) * C.plane + cid];
                    long long nid = F.idx(fi + ri, fj + rj, fk + rk);
                    int lk0 = -1 + pmod(F.zper, fk + rk, F.nz);
                    int lj0 = -1 + pmod(F.yper, fj + rj, F.ny);
                    int li0 = -1 + pmod(F.xper, fi + ri, F.nx);
                    for (int lk = lk0; lk <= 1; lk++)
                        for (int lj = lj0; lj <= 1; lj++)
                            for (int li = li0; li <= 1; li++) {
                                // (r-1)/2 truncates toward zero, as Fortran's integer division
                                int so = q27((ri - 1) / 2 + li, (rj - 1) / 2 + lj, (rk - 1) / 2 + lk);
                                acc[so * AS] = __dadd_rn(acc[so * AS], __dmul_rn(w, oprc2f[q27(li, lj, lk) * F.plane + nid]));
                            }
                }
#pragma unroll
        for (int q = 0; q < 27; q++) oprc[q * C.plane + cid] = acc[q * AS];
    }
}

// ---------------------------------------------------------------------------
// Dense coarsest matrix (bbmg_class.f90:1307-1385): column-major np x np.
// Thread `ind1` owns row ind1, so its accumulations keep the loop order.
__global__ void k_dense_operator(Lay L, const double *__restrict__ opr, double *__restrict__ OP) {
    int np = L.nx * L.ny * L.nz;
    for (int ind1 = threadIdx.x + blockIdx.x * blockDim.x; ind1 < np; ind1 += blockDim.x * gridDim.x) {
        int i1 = ind1 % L.nx, j1 = (ind1 / L.nx) % L.ny, k1 = ind1 / (L.nx * L.ny);
        long long id = L.idx(i1, j1, k1);
        for (int c = 0; c < np; c++) OP[(long long)c * np + ind1] = 0.0;
        for (int sk = -1; sk <= 1; sk++) {
            int k2 = k1 + sk;
            if (k2 == L.nz) { if (!L.zper) continue; k2 = 0; }
            if (k2 == -1) { if (!L.zper) continue; k2 = L.nz - 1; }
            for (int sj = -1; sj <= 1; sj++) {
                int j2 = j1 + sj;
                if (j2 == L.ny) { if (!L.yper) continue; j2 = 0; }
                if (j2 == -1) { if (!L.yper) continue; j2 = L.ny - 1; }
                for (int si = -1; si <= 1; si++) {
                    int i2 = i1 + si;
                    if (i2 == L.nx) { if (!L.xper) continue; i2 = 0; }
                    if (i2 == -1) { if (!L.xper) continue; i2 = L.nx - 1; }
                    int ind2 = i2 + j2 * L.nx + k2 * L.nx * L.ny;
                    long long e = (long long)ind2 * np + ind1;
                    OP[e] = __dadd_rn(OP[e], opr[q27(si, sj, sk) * L.plane + id]);
                }
            }
        }
    }
}

// Unblocked LU with row partial pivoting on a column-major n x n matrix, one
// thread block (the DGESV factorisation of bbmg_class.f90:912-913, done once
// per setup because the reference's per-call factorisation is deterministic).
// Pivot: the first row holding the largest magnitude.  Then marks the
// unknowns whose pivot is below 1000*n*eps*max|pivot| (a singular coarsest
// matrix); the solve sets those to zero.
// The factorisation of k_lu on A (global or shared memory), one block; sval
// and sidx hold blockDim.x entries.
__device__ __forceinline__ void lu_block(double *A, int n, int *__restrict__ piv, int *__restrict__ pinned,
                                         int *__restrict__ info_out, double *sval, int *sidx, int &s_info) {
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) s_info = 0;
    __syncthreads();
    for (int j = 0; j < n; j++) {
        // argmax |A(i,j)|, i >= j; ties -> smallest index
        double best = -1.0;
        int bi = n;
        for (int i = j + tid; i < n; i += nt) {
            double a = fabs(A[(long long)j * n + i]);
            if (a > best || (a == best && i < bi)) { best = a; bi = i; }
        }
        // the largest value with the smallest index among equals: a total
        // order, so any reduction order gives the same pivot.  Within each
        // warp by shuffles, then over the warps' winners by every thread.
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double a = __shfl_down_sync(0xffffffffu, best, o);
            const int ia = __shfl_down_sync(0xffffffffu, bi, o);
            if (a > best || (a == best && ia < bi)) { best = a; bi = ia; }
        }
        if ((tid & 31) == 0) { sval[tid >> 5] = best; sidx[tid >> 5] = bi; }
        __syncthreads();
        best = sval[0];
        bi = sidx[0];
        for (int w = 1; w < (nt + 31) / 32; w++) {
            const double a = sval[w];
            const int ia = sidx[w];
            if (a > best || (a == best && ia < bi)) { best = a; bi = ia; }
        }
        int p = bi;
        if (p >= n) p = j;
        __syncthreads();
        double pv = A[(long long)j * n + p];
        if (tid == 0) piv[j] = p;
        if (pv != 0.0) {
            if (p != j)
                for (int c = tid; c < n; c += nt) {
                    double x = A[(long long)c * n + j];
                    A[(long long)c * n + j] = A[(long long)c * n + p];
                    A[(long long)c * n + p] = x;
                }
            __syncthreads();
            double d = A[(long long)j * n + j];
            for (int i = j + 1 + tid; i < n; i += nt) A[(long long)j * n + i] = A[(long long)j * n + i] / d;
        } else if (tid == 0 && s_info == 0) {
            s_info = j + 1;
        }
        __syncthreads();
        long long m = (long long)(n - j - 1) * (n - j - 1);
        for (long long e = tid; e < m; e += nt) {
            int c = j + 1 + (int)(e / (n - j - 1));
            int i = j + 1 + (int)(e % (n - j - 1));
            A[(long long)c * n + i] = __dsub_rn(A[(long long)c * n + i], __dmul_rn(A[(long long)j * n + i], A[(long long)c * n + j]));
        }
        __syncthreads();
    }
    // pin round-off pivots
    double umax = 0.0;
    for (int k = tid; k < n; k += nt) umax = fmax(umax, fabs(A[(long long)k * n + k]));
    sval[tid] = umax;
    __syncthreads();
    for (int s = nt / 2; s > 0; s >>= 1) {
        if (tid < s) sval[tid] = fmax(sval[tid], sval[tid + s]);
        __syncthreads();
    }
    // round-off pivots of a singular (periodic / all-Neumann) coarsest matrix
    // reach ~1e-14 of the largest once density contrasts of 1e3 enter the
    // Galerkin operators, while genuine pivots stay above ~1e-3 of it: pin
    // within three decades of the round-off level n*eps*max|pivot|
    double tol = 1000.0 * (double)n * kEps * sval[0];
    for (int k = tid; k < n; k += nt) pinned[k] = fabs(A[(long long)k * n + k]) <= tol ? 1 : 0;
    if (tid == 0) *info_out = s_info;
}

__global__ void k_lu(double *__restrict__ A, int n, int *__restrict__ piv, int *__restrict__ pinned,
                     int *__restrict__ info_out) {
    __shared__ double sval[1024];
    __shared__ int sidx[1024];
    __shared__ int s_info;
    lu_block(A, n, piv, pinned, info_out, sval, sidx, s_info);
}

// The same factorisation with the matrix held in shared memory (n*n*8 bytes
// plus blockDim.x * 12): the per-column barriers then wait on shared-memory
// traffic instead of global-memory round trips.
__global__ void k_lu_smem(double *__restrict__ A, int n, int *__restrict__ piv, int *__restrict__ pinned,
                          int *__restrict__ info_out) {
    extern __shared__ __align__(16) unsigned char lu_sm[];
    double *M = reinterpret_cast<double *>(lu_sm);
    double *sval = M + (size_t)n * n;
    int *sidx = reinterpret_cast<int *>(sval + blockDim.x);
    __shared__ int s_info;
    const long long nn = (long long)n * n;
    for (long long e = threadIdx.x; e < nn; e += blockDim.x) M[e] = A[e];
    __syncthreads();
    lu_block(M, n, piv, pinned, info_out, sval, sidx, s_info);
    __syncthreads();
    for (long long e = threadIdx.x; e < nn; e += blockDim.x) A[e] = M[e];
}

// ---------------------------------------------------------------------------
// Exact symmetry of a 7-point level-1 operator: west(c) == east(c - x) etc.
// for every interior cell whose neighbour is interior or a periodic image
// (a coupling to a non-periodic overlap cell multiplies a zero value either
// way).  Clears *flag on the first mismatch.
// rows (j,k) on the y dimension of the grid, i on x: no 64-bit index division;
// one flag update per warp that saw a mismatch
__global__ void k_check_sym7(Lay L, const double *__restrict__ opr, int *flag) {
    for (int row = blockIdx.y * blockDim.y + threadIdx.y; row < L.ny * L.nz; row += gridDim.y * blockDim.y) {
        const int j = row % L.ny, k = row / L.ny;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.nx; i += gridDim.x * blockDim.x) {
            const long long id = L.idx(i, j, k);
            bool ok = true;
            if (i > 0 || L.xper) ok = ok && opr[q27(-1, 0, 0) * L.plane + id] == opr[q27(1, 0, 0) * L.plane + L.idx(i - 1, j, k)];
            if (j > 0 || L.yper) ok = ok && opr[q27(0, -1, 0) * L.plane + id] == opr[q27(0, 1, 0) * L.plane + L.idx(i, j - 1, k)];
            if (k > 0 || L.zper) ok = ok && opr[q27(0, 0, -1) * L.plane + id] == opr[q27(0, 0, 1) * L.plane + L.idx(i, j, k - 1)];
            if (!ok) atomicAnd(flag, 0);
        }
    }
}

// ---------------------------------------------------------------------------
// host launchers
#define BB_LAUNCH_CHECK() do { cudaError_t e_ = cudaGetLastError(); if (e_ != cudaSuccess) return e_; } while (0)

cudaError_t setup_scatter(const Lay &L, const double *src, int nst, int g, const int *stc, double *opr, unsigned wmask,
                          cudaStream_t s) {
    ScatterMap map;
    int cnt[27] = {0};
    for (int q = 0; q < 27; q++) map.one[q] = -1;
    for (int st = 0; st < 27; st++) map.slot[st] = -1;
    for (int st = 0; st < nst; st++) {
        const int q = q27h(stc[3 * st], stc[3 * st + 1], stc[3 * st + 2]);
        map.slot[st] = (signed char)q;
        map.one[q] = (signed char)st;
        cnt[q]++;
    }
    bool direct = true;
    for (int q = 0; q < 27; q++) direct = direct && cnt[q] <= 1;
    long long n = (long long)(L.nx + 2) * (L.ny + 2) * (L.nz + 2);
    if (direct)
        k_scatter_operator<true><<<grid_for(n, 128), 128, 0, s>>>(L, src, nst, g, map, opr, wmask);
    else
        k_scatter_operator<false><<<grid_for(n, 128), 128, 0, s>>>(L, src, nst, g, map, opr, wmask);
    BB_LAUNCH_CHECK();
    return cudaSuccess;
}

cudaError_t wrap_planes_mask(const Lay &L, double *a, unsigned mask, cudaStream_t s) {
    if (!(L.xper || L.yper || L.zper)) return cudaSuccess;
    k_wrap<<<grid_for(shell_cells(L), 256), 256, 0, s>>>(L, a, mask);
    BB_LAUNCH_CHECK();
    return cudaSuccess;
}

cudaError_t wrap_planes(const Lay &L, double *a, int nplanes, cudaStream_t s) {
    return wrap_planes_mask(L, a, nplanes >= 32 ? ~0u : ((1u << nplanes) - 1u), s);
}

cudaError_t wrap_planes(const Lay &L, float *a, int nplanes, cudaStream_t s) {
    if (!(L.xper || L.yper || L.zper)) return cudaSuccess;
    k_wrap_f<<<grid_for(shell_cells(L), 256), 256, 0, s>>>(L, a, nplanes);
    BB_LAUNCH_CHECK();
    return cudaSuccess;
}

cudaError_t setup_prolongation(const Lay &L, const double *opr, double *c2f, unsigned mask, cudaStream_t s,
                               float *c2f32) {
    long long na = (long long)(L.nx + 2) * (L.ny + 2) * (L.nz + 2);
    long long ni = (long long)L.nx * L.ny * L.nz;
    cudaError_t e;
    if (even_level(L) && fast_setup()) {
        const long long np = (long long)(L.nx / 2 + 1) * (L.ny / 2 + 1) * (L.nz / 2 + 1);
        k_prolong_sweep1_even<<<dim3((unsigned)grid_for(np, 128, 148 * 8), 4), 128, 0, s>>>(L, opr, c2f, mask, c2f32);
        BB_LAUNCH_CHECK();
        const long long hx = L.nx / 2, hy = L.ny / 2, hz = L.nz / 2;
        const long long nf = (hx + 1) * hy * hz + hx * (hy + 1) * hz + hx * hy * (hz + 1);
        k_prolong_sweep2_even<<<grid_for(nf, 128), 128, 0, s>>>(L, opr, c2f, mask, c2f32);
        BB_LAUNCH_CHECK();
        k_prolong_sweep3_even<<<grid_for(hx * hy * hz, 128), 128, 0, s>>>(L, opr, c2f, mask, c2f32);
        BB_LAUNCH_CHECK();
        if ((e = wrap_planes(L, c2f, 8, s)) != cudaSuccess) return e;
        return c2f32 ? wrap_planes(L, c2f32, 8, s) : cudaSuccess;
    }
    k_prolong_sweep1<<<grid_for(na, 128), 128, 0, s>>>(L, opr, c2f, mask);
    BB_LAUNCH_CHECK();
    k_prolong_sweep2<<<grid_for(na, 128), 128, 0, s>>>(L, opr, c2f, mask);
    BB_LAUNCH_CHECK();
    k_prolong_sweep3<<<grid_for(ni, 128), 128, 0, s>>>(L, opr, c2f, mask);
    BB_LAUNCH_CHECK();
    if ((e = wrap_planes(L, c2f, 8, s)) != cudaSuccess) return e;
    return c2f32 ? launch_to_f32(c2f, c2f32, 8LL * L.plane, s) : cudaSuccess;
}

// The overlap of f2c is read by nothing in the setup or the solve (the
// Galerkin product reads the weights of interior coarse cells only); it is
// filled when the array is read out (fill_overlap_f2c).
cudaError_t setup_restriction(const Lay &F, const Lay &C, const double *c2f, double *f2c, cudaStream_t s) {
    long long n = (long long)C.nx * C.ny * C.nz;
    if (even_level(F) && fast_setup()) {
        // every interior weight is written; the overlap is zero since the
        // allocation or its periodic image (written at read-out)
        k_restriction_weights_even<<<grid_for(n, 128), 128, 0, s>>>(F, C, c2f, f2c);
        BB_LAUNCH_CHECK();
        return cudaSuccess;
    }
    cudaError_t e = cudaMemsetAsync(f2c, 0, sizeof(double) * 27 * C.plane, s);
    if (e != cudaSuccess) return e;
    k_restriction_weights<<<grid_for(n, 128), 128, 0, s>>>(F, C, c2f, f2c);
    BB_LAUNCH_CHECK();
    return cudaSuccess;
}

cudaError_t fill_overlap_f2c(const Lay &C, double *f2c, cudaStream_t s) { return wrap_planes(C, f2c, 27, s); }

cudaError_t fill_overlap_oprc2f(const Lay &F, double *oprc2f, cudaStream_t s) {
    k_fill_shell<<<grid_for(shell_cells(F), 256), 256, 0, s>>>(F, oprc2f, 27, nullptr);
    BB_LAUNCH_CHECK();
    return cudaSuccess;
}

cudaError_t setup_operator(const Lay &F, const Lay &C, const double *oprF, const double *c2f, const double *f2c,
                           double *oprc2f, double *oprC, unsigned mask, cudaStream_t s, float *oprC32) {
    // the products are written on every interior cell; the overlap is zero
    // (non-periodic) or the periodic image
    constexpr int nt = 128;
    constexpr size_t smem = 27 * nt * sizeof(double);  // 27 accumulators per thread
    long long nf = (long long)F.nx * F.ny * F.nz;
    const bool fast = even_level(F) && fast_setup();
    // the centre and the six face planes only
    const unsigned seven = (1u << q27h(0, 0, 0)) | (1u << q27h(-1, 0, 0)) | (1u << q27h(1, 0, 0)) |
                           (1u << q27h(0, -1, 0)) | (1u << q27h(0, 1, 0)) | (1u << q27h(0, 0, -1)) |
                           (1u << q27h(0, 0, 1));
    const bool fast7 = fast && !(mask & ~seven);
    const dim3 gap((unsigned)grid_for(nf / 8, nt, 148 * 4), 8);  // one class per blockIdx.y
    if (fast7)
        k_rap_ap_even<true><<<gap, nt, 0, s>>>(F, oprF, c2f, oprc2f, mask);
    else if (fast)
        k_rap_ap_even<false><<<gap, nt, 0, s>>>(F, oprF, c2f, oprc2f, mask);
    else
        k_rap_ap<<<grid_for(nf, nt), nt, smem, s>>>(F, oprF, c2f, oprc2f, mask);
    BB_LAUNCH_CHECK();
    if (!fast) {  // k_rap_rap reads A P in the overlap
        k_fill_shell<<<grid_for(shell_cells(F), 256), 256, 0, s>>>(F, oprc2f, 27, nullptr);
        BB_LAUNCH_CHECK();
    }
    long long nc = (long long)C.nx * C.ny * C.nz;
    if (fast) {
        if (fast7)
            k_rap_rap_even<true><<<grid_for(3 * ((nc + 31) / 32) * 32, nt), nt, 0, s>>>(F, C, f2c, oprc2f, oprC, oprC32);
        else
            k_rap_rap_even<false><<<grid_for(3 * ((nc + 31) / 32) * 32, nt), nt, 0, s>>>(F, C, f2c, oprc2f, oprC, oprC32);
        BB_LAUNCH_CHECK();
        k_fill_shell<<<grid_for(shell_cells(C), 256), 256, 0, s>>>(C, oprC, 27, oprC32);
        BB_LAUNCH_CHECK();
        return cudaSuccess;
    }
    k_rap_rap<<<grid_for(nc, nt), nt, smem, s>>>(F, C, f2c, oprc2f, oprC);
    BB_LAUNCH_CHECK();
    k_fill_shell<<<grid_for(shell_cells(C), 256), 256, 0, s>>>(C, oprC, 27, nullptr);
    BB_LAUNCH_CHECK();
    return oprC32 ? launch_to_f32(oprC, oprC32, 27LL * C.plane, s) : cudaSuccess;
}

cudaError_t setup_solve_planes(const Lay &L, const double *opr, int npt, const int *slots, double *oprS,
                               float *oprS32, cudaStream_t s) {
    PlaneSlots ps{};
    ps.n = npt;
    for (int q = 0; q < npt; q++) ps.slot[q] = slots[q];
    k_solve_planes<<<grid_for(L.plane, 256), 256, 0, s>>>(L.plane, opr, ps, oprS, oprS32);
    BB_LAUNCH_CHECK();
    return cudaSuccess;
}

cudaError_t check_symmetric7(const Lay &L, const double *opr, int *flag, cudaStream_t s) {
    const int bx = L.nx >= 64 ? 64 : 32, by = 256 / bx;
    const int gx = (L.nx + bx - 1) / bx;
    long long gy = ((long long)L.ny * L.nz + by - 1) / by;
    if (gy > 65535) gy = 65535;
    k_check_sym7<<<dim3(gx, (unsigned)gy), dim3(bx, by), 0, s>>>(L, opr, flag);
    BB_LAUNCH_CHECK();
    return cudaSuccess;
}

cudaError_t setup_direct(const Lay &L, const double *opr, double *OP, double *LU, int *piv, int *pinned, int *info,
                         cudaStream_t s) {
    int np = L.nx * L.ny * L.nz;
    k_dense_operator<<<(np + 127) / 128, 128, 0, s>>>(L, opr, OP);
    BB_LAUNCH_CHECK();
    cudaError_t e = cudaMemcpyAsync(LU, OP, sizeof(double) * (size_t)np * np, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    constexpr int kLuThreads = 256;
    const size_t lu_smem = (size_t)np * np * sizeof(double) + kLuThreads * (sizeof(double) + sizeof(int));
    if (lu_smem <= 200 * 1024) {
        static bool attr = false;
        if (!attr) {
            e = cudaFuncSetAttribute(k_lu_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            if (e != cudaSuccess) return e;
            attr = true;
        }
        k_lu_smem<<<1, kLuThreads, lu_smem, s>>>(LU, np, piv, pinned, info);
    } else {
        k_lu<<<1, 1024, 0, s>>>(LU, np, piv, pinned, info);
    }
    BB_LAUNCH_CHECK();
    return cudaSuccess;
}

}  // namespace bbmg
