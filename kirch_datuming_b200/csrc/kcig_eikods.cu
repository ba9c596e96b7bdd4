// First-arrival traveltime tables on the GPU, the role of eikods2d
// (src/eikods2d.cpp:149-765, SERECKIRCH/src/eikods.cpp:66-211,
// SERECKIRCH/src/neighbors.cpp): for each source, the time T, its first
// derivatives with respect to the source position (tdl1 in the relative
// coordinate, tds1 in the source coordinate) and the branch-aware spatial
// gradients (gradz, gradx).
//
// eikods2d marches the front with a binary heap (fast marching).  Here every
// source's grid is solved by Gauss-Seidel sweeps in the four diagonal
// orderings, repeated until four consecutive sweeps change nothing, with the
// same local problem: the same constant-slowness box around the source
// (neighbors.cpp:418-484), the same first/second-order upwind quadratic in
// double precision (neighbors.cpp:106-188, 271-302) and the same rounding of
// every operation (explicit round-to-nearest intrinsics, no contraction).  For
// order 1 the update is monotone and the converged sweeps reach exactly the
// marching result; for order 2 the marching result also depends on the order
// in which the heap accepts points, and the two differ by up to ~2.5e-4 s at a
// fraction of the points.  The derivative recursion of eikods.cpp:119-211
// (each point from its upwind neighbours, in order of increasing time) is
// solved the same way: sweeps until nothing changes give exactly the ordered
// result.
//
// Execution: one CTA per source.  Step k of a sweep updates anti-diagonal k
// (local row r at local column k - r); a point's upwind neighbours (one and two
// samples back along each axis) lie on diagonals k-1 and k-2, its downwind
// neighbours on k+1 and k+2.  Diagonals k-2 .. k+D sit in a shared-memory ring
// indexed by row; diagonal k+D is fetched from global memory with cp.async
// while step k computes, so a step costs one barrier and no global-memory
// round trip.  Thread t owns rows t, t + blockDim, ...  A point whose inputs
// did not change since its previous evaluation is skipped (a per-point stamp
// of the sweep of its last change), which changes no result.  There is no
// wait other than the barriers and every loop has a fixed bound.
//
// Cost: a step gathers one anti-diagonal, one cache line per row, so the
// passes run at about one L1 wavefront per row and step (400 sources of the
// 601 x 1601 salt model in 83 ms for the time, 182 ms with tdl1/tds1).
#include <float.h>
#include <math.h>

#include <vector>

#include "kcig_common.h"

namespace kcig {
namespace {

constexpr float kFar = FLT_MAX;  // not yet reached (neighbors.cpp:423-426)

struct EikSource {
    int st0, en0, st1, en1;  // constant-slowness box, inclusive and clamped to the grid
    int ic;                  // box centre (its slowness is the box's)
    float xs0, xs1, xs2;     // source minus origin: depth, lateral, third axis
};

struct EikArgs {
    const float *vv;    // slowness squared [nx][nz]
    const double *dw;   // derivative of vv along axis l [nx][nz]
    const EikSource *src;
    float *T, *dl1, *ds1;  // [nsrc][nx][nz]
    int *status;           // set to 1 when a source has no fixed point within max_iter
    int *iters;            // [nsrc] sweeps the traveltime pass took (0: no fixed point)
    unsigned *stamp;       // [nsrc][nx][nz] 1 + the sweep of a point's last change (0: none)
    int nz, nx, order, l, max_iter;
    float d0, d1, d2;  // sampling: depth, lateral, third axis
    float rdx0, rdx1;  // 1 / d^2 rounded to float (neighbors.cpp:19-30)
};

__device__ __forceinline__ void cp_async4(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// one axis of the local problem (neighbors.cpp struct Upd)
struct Upd {
    double stencil, value, delta;
};

// neighbors.cpp:106-160 for one axis, with stencil() (:271-276): the
// smaller neighbour, or the second-order one-sided value when the sample two
// steps further is not larger
__device__ __forceinline__ void upd_axis(Upd &x, float a, float b, float a2, float b2, float rdx, int order)
{
    const float m = (a < b) ? a : b;
    const double v = (double)m;
    x.value = x.stencil = v;
    x.delta = (double)rdx;
    if (order > 1) {
        // a2 / b2 are kFar where the sample two steps away is outside the grid
        // or not reached, which fails the comparisons exactly as the marching
        // code's bounds and status checks do
        const float t2 = (a < b) ? a2 : b2;
        if ((a < b && a >= a2) || (a > b && b >= b2)) {
            x.stencil = __ddiv_rn(__dsub_rn(__dmul_rn(4.0, v), (double)t2), 3.0);
            x.delta = __dmul_rn(x.delta, 2.25);
        }
    }
}

// neighbors.cpp:278-302 updaten(): root of sum_j delta_j (t - stencil_j)^2 =
// v1 over the first m axes in increasing order of value; false if not causal
__device__ __forceinline__ bool upd_solve(int m, const Upd &p, const Upd &q, double v1, float &res)
{
    double A = __dadd_rn(0.0, p.delta);
    double B = __dadd_rn(0.0, __dmul_rn(p.stencil, p.delta));
    double C = __dadd_rn(0.0, __dmul_rn(__dmul_rn(p.stencil, p.stencil), p.delta));
    if (m > 1) {
        A = __dadd_rn(A, q.delta);
        B = __dadd_rn(B, __dmul_rn(q.stencil, q.delta));
        C = __dadd_rn(C, __dmul_rn(__dmul_rn(q.stencil, q.stencil), q.delta));
    }
    B = __ddiv_rn(B, A);
    const double discr = __dadd_rn(__dmul_rn(B, B), __ddiv_rn(__dsub_rn(v1, C), A));
    if (discr < 0.0) return false;
    const double t = __dadd_rn(B, __dsqrt_rn(discr));
    if (t <= (m > 1 ? q.value : p.value)) return false;
    res = __double2float_rn(t);
    return true;
}

// neighbors.cpp:106-188 qsolve() on a 2-D grid (the third axis never contributes)
__device__ __forceinline__ float qsolve2d(float zm, float zp, float zm2, float zp2, float xm, float xp, float xm2,
                                          float xp2, float vv, float rdx0, float rdx1, int order)
{
    Upd x0, x1;
    upd_axis(x0, zm, zp, zm2, zp2, rdx0, order);
    upd_axis(x1, xm, xp, xm2, xp2, rdx1, order);
    // the marching code sorts the three axes by value; with the third axis at
    // FLT_MAX the first two keep their order unless x1 < x0
    const bool swap = !(x0.value <= x1.value);
    Upd p, q;  // selected field by field: no address of a local is taken
    p.stencil = swap ? x1.stencil : x0.stencil;
    p.value = swap ? x1.value : x0.value;
    p.delta = swap ? x1.delta : x0.delta;
    q.stencil = swap ? x0.stencil : x1.stencil;
    q.value = swap ? x0.value : x1.value;
    q.delta = swap ? x0.delta : x1.delta;
    const double v1 = (double)vv;
    float res;
    if (q.value < (double)kFar) {
        if (upd_solve(2, p, q, v1, res) || upd_solve(1, p, q, v1, res)) return res;
    } else if (p.value < (double)kFar) {
        if (upd_solve(1, p, q, v1, res)) return res;
    }
    return kFar;
}

// ------------------------------------------------------------- kernels --

__global__ void k_slowness2(const float *__restrict__ vel, float *__restrict__ vv, size_t n, int is_slowness2)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = vel[i];
    // eikods2d.cpp:325-335: v = 1 / (v * v) with the product in float
    vv[i] = is_slowness2 ? v : __double2float_rn(__ddiv_rn(1.0, (double)__fmul_rn(v, v)));
}

// derivative of slowness squared along axis l (eikods.cpp:197-204)
__global__ void k_dw(const float *__restrict__ vv, double *__restrict__ dw, int nz, int nx, int l, float dl)
{
    const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i0 >= (size_t)nz * nx) return;
    const int ii = l == 0 ? (int)(i0 % nz) : (int)(i0 / nz), n = l == 0 ? nz : nx;
    const size_t s = l == 0 ? 1 : (size_t)nz;
    const double den = __dmul_rn(2.0, (double)dl);
    double w;
    if (0 < ii && ii < n - 1) {
        w = __ddiv_rn((double)__fsub_rn(vv[i0 + s], vv[i0 - s]), den);
    } else if (ii == 0) {
        const double u = __dadd_rn(-(double)vv[i0 + 2 * s], __dmul_rn(4.0, (double)vv[i0 + s]));
        w = __ddiv_rn(__dsub_rn(u, __dmul_rn(3.0, (double)vv[i0])), den);
    } else {
        const double u = __dsub_rn(__dmul_rn(3.0, (double)vv[i0]), __dmul_rn(4.0, (double)vv[i0 - s]));
        w = __ddiv_rn(__dadd_rn(u, (double)vv[i0 - 2 * s]), den);
    }
    dw[i0] = w;
}

// Sweeps of one source per CTA.  MODE 0: traveltime; MODE 1: the source
// derivative recursion on the final traveltime.  S: ring slots (a power of
// two), D: prefetch distance in diagonals (S >= D + 3), ROWS: rows per thread
// (blockDim * ROWS >= nz); a thread's rows of one step are independent and
// their branch-free updates interleave.
template <int MODE, int S, int D, int ROWS>
__global__ void __launch_bounds__(ROWS == 1 ? 1024 : 512) k_eik_sweep(EikArgs a)
{
    static_assert((S & (S - 1)) == 0 && S >= D + 3 && D >= 3, "ring too small");
    extern __shared__ __align__(16) unsigned char eik_smem[];
    const int nz = a.nz, nx = a.nx, NR = nz + 4;  // ring rows -2 .. nz+1
    float *RT = reinterpret_cast<float *>(eik_smem);            // [S][NR] traveltime
    unsigned *RS = reinterpret_cast<unsigned *>(RT + S * NR);   // [S][NR] change stamps
    float *RL = reinterpret_cast<float *>(RS + S * NR);         // [S][NR] tdl1 (MODE 1)
    double *RW = reinterpret_cast<double *>(RL + S * NR);       // [S][NR] dw (MODE 1); offset 12*S*NR bytes
    const int js = blockIdx.x;
    const size_t nzx = (size_t)nz * nx;
    float *T = a.T + (size_t)js * nzx;
    float *DL = MODE == 1 ? a.dl1 + (size_t)js * nzx : nullptr;
    float *DS = MODE == 1 ? a.ds1 + (size_t)js * nzx : nullptr;
    unsigned *ST = a.stamp + (size_t)js * nzx;
    const EikSource sc = a.src[js];
    const int nthr = blockDim.x, tid = threadIdx.x;

    // pad rows stay constant for the whole kernel
    for (int q = tid; q < S * 4; q += nthr) {
        const int slot = q >> 2, pr = q & 3, row = pr < 2 ? pr : nz + pr;
        RT[slot * NR + row] = kFar;
        RS[slot * NR + row] = 0u;
        if (MODE == 1) {
            RL[slot * NR + row] = 0.0f;
            RW[slot * NR + row] = 0.0;
        }
    }
    if (MODE == 0) {
        // initial state: nothing reached, the box at straight-ray times
        // (neighbors.cpp:418-484)
        for (size_t i = tid; i < nzx; i += nthr) T[i] = kFar;
        __syncthreads();
        const double v1 = (double)a.vv[sc.ic];
        const int bz = sc.en0 - sc.st0 + 1, nb = bz * (sc.en1 - sc.st1 + 1);
        for (int q = tid; q < nb; q += nthr) {
            const int iz = sc.st0 + q % bz, iy = sc.st1 + q / bz;
            const double e0 = (double)__fsub_rn(sc.xs0, __fmul_rn((float)iz, a.d0));
            const double e1 = (double)__fsub_rn(sc.xs1, __fmul_rn((float)iy, a.d1));
            const double e2 = (double)__fsub_rn(sc.xs2, __fmul_rn(0.0f, a.d2));
            double d2 = __dadd_rn(0.0, __dmul_rn(e0, e0));
            d2 = __dadd_rn(d2, __dmul_rn(e1, e1));
            d2 = __dadd_rn(d2, __dmul_rn(e2, e2));
            T[(size_t)iy * nz + iz] = __fsqrt_rn(__double2float_rn(__dmul_rn(v1, d2)));
        }
    }
    __syncthreads();

    const int ndiag = nz + nx - 1;
    int quiet = 0, nsweep = 0;
    for (int sweep = 0; sweep < 4 * a.max_iter; sweep++) {
        const int dir = sweep & 3;
        const bool fz = (dir & 1) == 0, fx = (dir & 2) == 0;
        const int sz = fz ? 1 : -1, sx = fx ? 1 : -1;
        // diagonal kk of this sweep into its ring slot (async where inside the grid)
        auto fetch = [&](int kk) {
            const int slot = kk & (S - 1);
#pragma unroll
            for (int qr = 0; qr < ROWS; qr++) {
                const int r = tid + qr * nthr;
                if (r >= nz) continue;
                const int c = kk - r;
                const int ri = slot * NR + r + 2;
                if (c >= 0 && c < nx) {
                    const size_t i = (size_t)(fx ? c : nx - 1 - c) * nz + (fz ? r : nz - 1 - r);
                    cp_async4(RT + ri, T + i);
                    cp_async4(RS + ri, ST + i);
                    if (MODE == 1) {
                        cp_async4(RL + ri, DL + i);
                        cp_async8(RW + ri, a.dw + i);
                    }
                } else {
                    RT[ri] = kFar;
                    RS[ri] = 0u;
                    if (MODE == 1) {
                        RL[ri] = 0.0f;
                        RW[ri] = 0.0;
                    }
                }
            }
        };
        for (int r = tid; r < nz; r += nthr) {  // diagonals -2 and -1
            RT[(S - 2) * NR + r + 2] = kFar;
            RT[(S - 1) * NR + r + 2] = kFar;
            RS[(S - 2) * NR + r + 2] = 0u;
            RS[(S - 1) * NR + r + 2] = 0u;
            if (MODE == 1) {
                RL[(S - 2) * NR + r + 2] = 0.0f;
                RL[(S - 1) * NR + r + 2] = 0.0f;
            }
        }
        for (int kk = 0; kk < D; kk++) {
            fetch(kk);
            cp_commit();
        }
        cp_wait<D - 3>();
        __syncthreads();
        bool changed = false;
        for (int k = 0; k < ndiag; k++) {
            fetch(k + D);
            cp_commit();
            const int s0 = k & (S - 1);
#pragma unroll
            for (int qr = 0; qr < ROWS; qr++) {
                const int r0 = tid + qr * nthr, c0 = k - r0;
                const bool act = r0 < nz && c0 >= 0 && c0 < nx;
                // inactive rows compute on a valid point and store nothing
                const int r = act ? r0 : 0, c = act ? c0 : 0;
                const int iz = fz ? r : nz - 1 - r, ix = fx ? c : nx - 1 - c;
                const size_t i = (size_t)ix * nz + iz;
                const int R = r + 2;
                // physical neighbours: z -/+ one and two samples, x -/+ one and two
                const float t0 = RT[s0 * NR + R];
                const float zm = RT[((k - sz) & (S - 1)) * NR + R - sz];
                const float zp = RT[((k + sz) & (S - 1)) * NR + R + sz];
                const float zm2 = RT[((k - 2 * sz) & (S - 1)) * NR + R - 2 * sz];
                const float zp2 = RT[((k + 2 * sz) & (S - 1)) * NR + R + 2 * sz];
                const float xm = RT[((k - sx) & (S - 1)) * NR + R];
                const float xp = RT[((k + sx) & (S - 1)) * NR + R];
                const float xm2 = RT[((k - 2 * sx) & (S - 1)) * NR + R];
                const float xp2 = RT[((k + 2 * sx) & (S - 1)) * NR + R];
                // A point whose inputs did not change since its evaluation in
                // the previous sweep would come out the same: it is skipped.
                // Its inputs are the neighbours one step away (both passes)
                // and two steps away (traveltime pass); stamps >= sweep mark
                // a change in the previous sweep or earlier in this one.
                const unsigned szm = RS[((k - sz) & (S - 1)) * NR + R - sz];
                const unsigned szp = RS[((k + sz) & (S - 1)) * NR + R + sz];
                const unsigned sxm = RS[((k - sx) & (S - 1)) * NR + R];
                const unsigned sxp = RS[((k + sx) & (S - 1)) * NR + R];
                unsigned snew = max(max(szm, szp), max(sxm, sxp));
                if (MODE == 0) {
                    const unsigned szm2 = RS[((k - 2 * sz) & (S - 1)) * NR + R - 2 * sz];
                    const unsigned szp2 = RS[((k + 2 * sz) & (S - 1)) * NR + R + 2 * sz];
                    const unsigned sxm2 = RS[((k - 2 * sx) & (S - 1)) * NR + R];
                    const unsigned sxp2 = RS[((k + 2 * sx) & (S - 1)) * NR + R];
                    snew = max(snew, max(max(szm2, szp2), max(sxm2, sxp2)));
                }
                const bool need = act && (sweep == 0 || snew >= (unsigned)sweep);
                if (!need) continue;
                if (MODE == 0) {
                    const bool in_box = iz >= sc.st0 && iz <= sc.en0 && ix >= sc.st1 && ix <= sc.en1;
                    if (in_box) continue;
                    const float q = qsolve2d(zm, zp, zm2, zp2, xm, xp, xm2, xp2, a.vv[i], a.rdx0, a.rdx1, a.order);
                    if (q < t0) {
                        RT[s0 * NR + R] = q;
                        T[i] = q;
                        RS[s0 * NR + R] = (unsigned)sweep + 1u;
                        ST[i] = (unsigned)sweep + 1u;
                        changed = true;
                    }
                } else {
                    // eikods.cpp:149-211 (eikods_dt1) for point i, branch-free
                    const float lzm = RL[((k - sz) & (S - 1)) * NR + R - sz];
                    const float lzp = RL[((k + sz) & (S - 1)) * NR + R + sz];
                    const float lxm = RL[((k - sx) & (S - 1)) * NR + R];
                    const float lxp = RL[((k + sx) & (S - 1)) * NR + R];
                    double rhs = 0.0, den = 0.0, dt = 0.0;
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        const int ii = j == 0 ? iz : ix, n = j == 0 ? nz : nx;
                        const float ta = j == 0 ? zm : xm, tb = j == 0 ? zp : xp;
                        const float ta2 = j == 0 ? zm2 : xm2, tb2 = j == 0 ? zp2 : xp2;
                        const float la = j == 0 ? lzm : lxm, lb = j == 0 ? lzp : lxp;
                        const float dj = j == 0 ? a.d0 : a.d1;
                        const bool use_b = ii == 0 || (ii != n - 1 && ta > tb);
                        const float t1 = use_b ? tb : ta, l1 = use_b ? lb : la;
                        const bool up = t1 < t0;
                        const float dd = __fmul_rn(dj, dj);
                        const float e = __fsub_rn(t0, t1);
                        const double term = (double)__fdiv_rn(__fmul_rn(e, l1), dd);
                        const double dterm = (double)__fdiv_rn(e, dd);
                        rhs = up ? __dadd_rn(rhs, term) : rhs;
                        den = up ? __dadd_rn(den, dterm) : den;
                        if (a.l == j) {
                            const float t2 = use_b ? tb2 : ta2;
                            const bool three = use_b ? (ii < n - 2 && t1 > tb2) : (ii > 1 && t1 > ta2);
                            const double num3 =
                                use_b ? __dsub_rn(__dadd_rn(-(double)t2, __dmul_rn(4.0, (double)t1)),
                                                  __dmul_rn(3.0, (double)t0))
                                      : __dadd_rn(__dsub_rn(__dmul_rn(3.0, (double)t0), __dmul_rn(4.0, (double)t1)),
                                                  (double)t2);
                            const double d3 = __ddiv_rn(num3, __dmul_rn(2.0, (double)dj));
                            const double d2p = (double)__fdiv_rn(use_b ? __fsub_rn(t1, t0) : __fsub_rn(t0, t1), dj);
                            dt = up ? (three ? d3 : d2p) : dt;
                        }
                    }
                    const double w = RW[s0 * NR + R];
                    const bool has = den != 0.0;
                    const float nl0 = __double2float_rn(__ddiv_rn(__dadd_rn(__dmul_rn(0.5, w), rhs), den));
                    const float nl = has ? nl0 : 0.0f;
                    const float ns = has ? __double2float_rn(__dsub_rn((double)nl0, dt)) : 0.0f;
                    // tds1 follows tdl1 (dt is fixed by the final time), so
                    // after the first visit only a change of tdl1 is news
                    const float ol = RL[s0 * NR + R];
                    if (sweep == 0 || nl != ol) {
                        RL[s0 * NR + R] = nl;
                        DL[i] = nl;
                        DS[i] = ns;
                    }
                    if (nl != ol) {
                        RS[s0 * NR + R] = (unsigned)sweep + 1u;
                        ST[i] = (unsigned)sweep + 1u;
                        changed = true;
                    }
                }
            }
            cp_wait<D - 3>();
            __syncthreads();
        }
        cp_wait<0>();
        const bool any = __syncthreads_or(changed);
        quiet = any ? 0 : quiet + 1;
        // four quiet sweeps in a row (one of each ordering): a fixed point
        if (quiet >= 4) {
            nsweep = sweep + 1;
            break;
        }
    }
    if (tid == 0) {
        if (nsweep == 0) atomicExch(a.status, 1);
        if (MODE == 0) a.iters[js] = nsweep;
    }
}

// launch of one pass: one row per thread up to 1024 rows, else four
template <int MODE, int S, int D>
int launch_sweep(const EikArgs &a, int nshot, cudaStream_t st)
{
    const int nz = a.nz, rows = nz <= 1024 ? 1 : 4;
    const size_t smem =
        (size_t)S * (nz + 4) * (MODE == 0 ? 2 * sizeof(float) : 3 * sizeof(float) + sizeof(double));
    const int threads = (((nz + rows - 1) / rows + 31) / 32) * 32;
    if (rows == 1) {
        KCIG_TRY(set_dyn_smem((const void *)k_eik_sweep<MODE, S, D, 1>, (int)smem));
        k_eik_sweep<MODE, S, D, 1><<<nshot, threads, smem, st>>>(a);
    } else {
        KCIG_TRY(set_dyn_smem((const void *)k_eik_sweep<MODE, S, D, 4>, (int)smem));
        k_eik_sweep<MODE, S, D, 4><<<nshot, threads, smem, st>>>(a);
    }
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

// branch-aware spatial gradient along one axis (eikods2d.cpp:30-68)
__device__ __forceinline__ float upwind_grad(const float *t, size_t i0, int ii, int n, size_t s, float dd)
{
    const size_t a = i0 - s, b = i0 + s;
    size_t i1;
    if (ii == 0) i1 = b;
    else if (ii != n - 1 && t[b] < t[a]) i1 = b;
    else i1 = a;
    if (!(t[i1] < t[i0])) return 0.0f;
    const float two_d = __fmul_rn(2.0f, dd);
    if (i1 == b) {
        if (ii < n - 2 && t[i1 + s] < t[i1]) {
            const float u = __fadd_rn(-t[i1 + s], __fmul_rn(4.0f, t[i1]));
            return __fdiv_rn(__fsub_rn(u, __fmul_rn(3.0f, t[i0])), two_d);
        }
        return __fdiv_rn(__fsub_rn(t[i1], t[i0]), dd);
    }
    if (ii > 1 && t[i1 - s] < t[i1]) {
        const float u = __fsub_rn(__fmul_rn(3.0f, t[i0]), __fmul_rn(4.0f, t[i1]));
        return __fdiv_rn(__fadd_rn(u, t[i1 - s]), two_d);
    }
    return __fdiv_rn(__fsub_rn(t[i0], t[i1]), dd);
}

__global__ void k_upwind_grads(const float *__restrict__ T, float *__restrict__ gz, float *__restrict__ gx, int nz,
                               int nx, float dz, float dx)
{
    const size_t nzx = (size_t)nz * nx;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nzx) return;
    const float *t = T + (size_t)blockIdx.y * nzx;
    const size_t o = (size_t)blockIdx.y * nzx + i;
    const int iz = (int)(i % nz), ix = (int)(i / nz);
    if (gz) gz[o] = upwind_grad(t, i, iz, nz, 1, dz);
    if (gx) gx[o] = upwind_grad(t, i, ix, nx, (size_t)nz, dx);
}

// host side of neighbors.cpp:428-445: the box around the source, in the
// reference's own float arithmetic
EikSource source_box(float s0, float s1, float s2, float o0, float o1, float o2, float d0, float d1, int nz, int nx,
                     int b0, int b1)
{
    const float xs[3] = {s0 - o0, s1 - o1, s2 - o2};
    const float d[2] = {d0, d1};
    const int n[2] = {nz, nx}, b[2] = {b0, b1};
    int st[3], en[3];
    for (int j = 0; j < 2; j++) {
        const int is = (int)(xs[j] / d[j] + 0.5);
        st[j] = is - b[j];
        en[j] = is + b[j];
        st[j] = st[j] < 0 ? 0 : (st[j] >= n[j] ? n[j] - 1 : st[j]);
        en[j] = en[j] < 0 ? 0 : (en[j] >= n[j] ? n[j] - 1 : en[j]);
    }
    st[2] = en[2] = 0;  // a 2-D grid: the third axis clamps to its one sample
    EikSource e;
    e.st0 = st[0];
    e.en0 = en[0];
    e.st1 = st[1];
    e.en1 = en[1];
    e.ic = (st[0] + en[0]) / 2 + n[0] * ((st[1] + en[1]) / 2 + n[1] * (st[2] + en[2]) / 2);
    e.xs0 = xs[0];
    e.xs1 = xs[1];
    e.xs2 = xs[2];
    return e;
}

struct DevBuf {
    void *p = nullptr;
    cudaStream_t st = nullptr;
    ~DevBuf()
    {
        if (p) cudaFreeAsync(p, st);
    }
};

}  // namespace
}  // namespace kcig

using namespace kcig;

extern "C" int kcig_eikods(const float *vel, int nz, int nx, float o1, float o2, float d1, float d2, float o3,
                           float d3, const float *shots, int nshot, const kcig_eikods_opts *opt, float *time,
                           float *tdl1, float *tds1, float *gradz, float *gradx, int *iters, void *stream)
{
    if (!vel || !time || !shots || !opt || nz < 3 || nx < 3 || nshot < 1 || !(d1 > 0.0f) || !(d2 > 0.0f))
        return set_error(KCIG_ERR_ARG, "kcig_eikods: bad arguments");
    if (opt->order != 1 && opt->order != 2) return set_error(KCIG_ERR_ARG, "kcig_eikods: order must be 1 or 2");
    if (opt->l != 0 && opt->l != 1) return set_error(KCIG_ERR_ARG, "kcig_eikods: l must be 0 or 1");
    if ((tdl1 == nullptr) != (tds1 == nullptr))
        return set_error(KCIG_ERR_ARG, "kcig_eikods: tdl1 and tds1 go together");
    // the rings hold 16 (time) and 8 (derivative pass) diagonals of nz + 4 rows
    if (nz > 1400) return set_error(KCIG_ERR_ARG, "kcig_eikods: nz=%d above 1400", nz);
    const int max_iter = opt->max_iter > 0 ? opt->max_iter : 256;
    const int b0 = opt->b1 < 1 ? 1 : opt->b1, b1 = opt->b2 < 1 ? 1 : opt->b2;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nzx = (size_t)nz * nx;

    std::vector<EikSource> hs(nshot);
    for (int j = 0; j < nshot; j++)
        hs[j] = source_box(shots[3 * j], shots[3 * j + 1], shots[3 * j + 2], o1, o2, o3, d1, d2, nz, nx, b0, b1);

    DevBuf bvv, bdw, bsrc, bstat, bit, bstamp;
    bvv.st = bdw.st = bsrc.st = bstat.st = bit.st = bstamp.st = st;
    KCIG_CUDA(cudaMallocAsync(&bvv.p, nzx * sizeof(float), st));
    KCIG_CUDA(cudaMallocAsync(&bsrc.p, nshot * sizeof(EikSource), st));
    KCIG_CUDA(cudaMallocAsync(&bstat.p, sizeof(int), st));
    KCIG_CUDA(cudaMallocAsync(&bit.p, nshot * sizeof(int), st));
    KCIG_CUDA(cudaMallocAsync(&bstamp.p, (size_t)nshot * nzx * sizeof(unsigned), st));
    KCIG_CUDA(cudaMemsetAsync(bstamp.p, 0, (size_t)nshot * nzx * sizeof(unsigned), st));
    if (tdl1) KCIG_CUDA(cudaMallocAsync(&bdw.p, nzx * sizeof(double), st));
    KCIG_CUDA(cudaMemcpyAsync(bsrc.p, hs.data(), nshot * sizeof(EikSource), cudaMemcpyHostToDevice, st));
    KCIG_CUDA(cudaMemsetAsync(bstat.p, 0, sizeof(int), st));

    EikArgs a;
    a.vv = (const float *)bvv.p;
    a.dw = (const double *)bdw.p;
    a.src = (const EikSource *)bsrc.p;
    a.T = time;
    a.dl1 = tdl1;
    a.ds1 = tds1;
    a.status = (int *)bstat.p;
    a.iters = (int *)bit.p;
    a.stamp = (unsigned *)bstamp.p;
    a.nz = nz;
    a.nx = nx;
    a.order = opt->order;
    a.l = opt->l;
    a.max_iter = max_iter;
    a.d0 = d1;
    a.d1 = d2;
    a.d2 = d3;
    a.rdx0 = (float)(1. / (d1 * d1));
    a.rdx1 = (float)(1. / (d2 * d2));

    const unsigned g1 = (unsigned)((nzx + 255) / 256);
    k_slowness2<<<g1, 256, 0, st>>>(vel, (float *)bvv.p, nzx, opt->vel_is_slowness2);
    KCIG_TRY((launch_sweep<0, 16, 8>(a, nshot, st)));
    if (tdl1) {
        k_dw<<<g1, 256, 0, st>>>((const float *)bvv.p, (double *)bdw.p, nz, nx, opt->l, opt->l == 0 ? d1 : d2);
        KCIG_CUDA(cudaMemsetAsync(tdl1, 0, (size_t)nshot * nzx * sizeof(float), st));
        KCIG_CUDA(cudaMemsetAsync(tds1, 0, (size_t)nshot * nzx * sizeof(float), st));
        KCIG_CUDA(cudaMemsetAsync(bstamp.p, 0, (size_t)nshot * nzx * sizeof(unsigned), st));
        KCIG_TRY((launch_sweep<1, 8, 5>(a, nshot, st)));
    }
    if (gradz || gradx) {
        k_upwind_grads<<<dim3(g1, nshot), 256, 0, st>>>(time, gradz, gradx, nz, nx, d1, d2);
        KCIG_CUDA(cudaGetLastError());
    }
    int status = 0;
    std::vector<int> hit(nshot);
    KCIG_CUDA(cudaMemcpyAsync(&status, bstat.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    KCIG_CUDA(cudaMemcpyAsync(hit.data(), bit.p, nshot * sizeof(int), cudaMemcpyDeviceToHost, st));
    KCIG_CUDA(cudaStreamSynchronize(st));
    if (iters)
        for (int j = 0; j < nshot; j++) iters[j] = hit[j];
    if (status)
        return set_error(KCIG_ERR_DEVICE, "kcig_eikods: sweeps found no fixed point within max_iter=%d", max_iter);
    return KCIG_OK;
}

// fixed-geometry entry point: sources at depth zsrc and lateral positions
// p0 + k*dp (shotgen's float arithmetic), order 2, derivative = tds1
extern "C" int kcig_eikonal_tables(const float *vel, int nz, int nx, float dz, float dx, float z0, float x0, int npos,
                                   float p0, float dp, float zsrc, int b1, int b2, int iterations, float *time,
                                   float *deriv, void *stream)
{
    if (npos < 1) return set_error(KCIG_ERR_ARG, "kcig_eikonal_tables: npos < 1");
    std::vector<float> shots(3 * (size_t)npos);
    for (int j = 0; j < npos; j++) {
        shots[3 * j] = zsrc;
        shots[3 * j + 1] = p0 + (float)j * dp;
        shots[3 * j + 2] = 0.0f;
    }
    kcig_eikods_opts o;
    o.order = 2;
    o.b1 = b1;
    o.b2 = b2;
    o.l = 1;
    o.vel_is_slowness2 = 0;
    o.max_iter = iterations;
    float *dl1 = nullptr;
    if (deriv) {
        cudaError_t e = cudaMallocAsync((void **)&dl1, (size_t)npos * nz * nx * sizeof(float), (cudaStream_t)stream);
        if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync(tdl1)");
    }
    const int rc = kcig_eikods(vel, nz, nx, z0, x0, dz, dx, 0.0f, 1.0f, shots.data(), npos, &o, time, dl1, deriv,
                               nullptr, nullptr, nullptr, stream);
    if (dl1) cudaFreeAsync(dl1, (cudaStream_t)stream);
    return rc;
}
