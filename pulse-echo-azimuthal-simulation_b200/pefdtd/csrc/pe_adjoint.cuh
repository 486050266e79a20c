// Discrete adjoint (reverse-time) step of the label-indexed elastic FDTD.
//
// The forward step n maps (v^{n-1}, s^{n-1}) to (v^n, s^n):
//   g   = D v^{n-1}                       strains (order-2..8 staggered taps)
//   s^n = d s^{n-1} + dt C(M g) + src     stress (half-cell moves M, 6x6 C)
//   v^n = d (v^{n-1} + dt_h G(s^n) / rho_face)
// and the recorded samples are linear in (v^n, s^n). These kernels apply the
// exact transpose of that map, in reverse order, to the adjoint state
// (lv, ls) = dJ/d(v^n, s^n), and accumulate dJ/dC per material:
//   k_adj_inject    lv or ls += trace adjoint at the receiver cells
//   k_adj_vel_u     u = d dt_h lv / rho_face              (per component)
//   k_adj_vel       ls += G^T u                           (gathers), then
//                   w[p][J] = sum over stresses I at position p of
//                   C_IJ dt ls_I, for the 18 moved (p, J), once per cell
//   k_adj_strain    g = D v^{n-1}                         (same taps as forward)
//   k_adj_stress    dJ/dC[m] += dt ls (x) (M g); t = M^T C^T (dt ls);
//                   then ls = d ls
//   k_adj_velfin    lv = d lv + D^T t
// Every transpose is a gather that evaluates the forward guard at the forward
// cell it reads from, so the boundaries transpose exactly and no result
// depends on thread order except the per-material gradient sums (f64
// atomics after warp aggregation). The reference's own adjoint is the
// order-2, cell-density, undamped vendor/ringfwi/elastic3d.py:348-463; this
// one is the adjoint of the full production scheme.
#pragma once
#include "pe_kernels_pair.cuh"

namespace pe {

template <typename T>
struct AdjArgs {
    T *lv[3];          // adjoint of v
    T *ls[6];          // adjoint of s
    const T *vp[3];    // forward v at the start of the step (v^{n-1})
    T *u[3];           // scratch: scaled velocity adjoint
    T *g[6];           // scratch: forward strains
    T *t[6];           // scratch: strain adjoint
    T *w[18];          // scratch: C^T (dt ls) per moved (position, strain)
    const uint16_t *lab;
    const T *c21;      // (n_mat, C21_STRIDE)
    const T *rho;
    const float *rinv;  // (n_mat,) RN32(1 / rho) (FP32 solves), or null
    const float *dz, *dy, *dx, *dvol;
    int nz, ny, nx;
    long long sy, sz;
    T c[4];
    int nc;
    T inv_h, dt, dt_h;
    double *grad;      // (grad_rep, n_mat, 21) dJ/dC, upper triangle row major
    int grad_rep;      // replicas of the table the atomic sums spread over (>= 1)
    int n_mat;
};

__device__ __forceinline__ bool gF(int x, int j, int n) { return x >= j && x < n - j - 1; }
__device__ __forceinline__ bool gB(int x, int j, int n) { return x >= j + 1 && x < n - j; }

template <typename T>
__device__ __forceinline__ float adj_damp(const AdjArgs<T> &A, int iz, int iy, int ix, long long idx)
{
    float d = 1.0f;
    if (A.dz) {
        d = A.dz[iz] * A.dy[iy];
        d = d * A.dx[ix];
    }
    if (A.dvol) d = A.dz ? d * A.dvol[idx] : A.dvol[idx];
    return d;
}

// transpose of the forward derivative along one axis, at position y of an
// axis of length n; f(o) reads the operand at y + o. A tap whose forward cell
// y + o does not exist reads the operand at y instead (always in the grid)
// and contributes c * 0, which leaves the sum unchanged bit for bit: every
// load is independent of the guards, so the gathers of a cell overlap.
// G: evaluate the guards (false where the caller has established that every
// tap of the cell along this axis exists: adj_block_inside, adj_inside_x,
// adj_inside_yz).
template <typename T, bool G = true, typename F>
__device__ __forceinline__ T DfT(const F &f, int y, int n, const T c[4], int nc)
{
    T a = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (j < nc) {
            const bool p1 = !G || gF(y - j - 1, j, n), p2 = !G || gF(y + j, j, n);
            const T v1 = f(p1 ? -j - 1 : 0), v2 = f(p2 ? j : 0);
            a += c[j] * (p1 ? v1 : T(0));
            a -= c[j] * (p2 ? v2 : T(0));
        }
    }
    return a;
}
template <typename T, bool G = true, typename F>
__device__ __forceinline__ T DbT(const F &f, int y, int n, const T c[4], int nc)
{
    T a = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (j < nc) {
            const bool p1 = !G || gB(y - j, j, n), p2 = !G || gB(y + j + 1, j, n);
            const T v1 = f(p1 ? -j : 0), v2 = f(p2 ? j + 1 : 0);
            a += c[j] * (p1 ? v1 : T(0));
            a -= c[j] * (p2 ? v2 : T(0));
        }
    }
    return a;
}

template <typename T>
__device__ __forceinline__ void cell_of(const AdjArgs<T> &A, long long i, int &iz, int &iy, int &ix)
{
    ix = (int)(i % A.nx);
    iy = (int)((i / A.nx) % A.ny);
    iz = (int)(i / ((long long)A.nx * A.ny));
}

// Cell of this thread in the adjoint kernels' launches: 32 x 8 blocks over
// (x tiles, y tiles, z planes), so that a warp is 32 consecutive cells of a
// row and the coordinates come from the launch indices (no 64-bit division
// per cell). False for the threads past the grid's x / y edge.
constexpr int ADJ_BX = 32, ADJ_BY = 8;
template <typename T>
__device__ __forceinline__ bool adj_cell(const AdjArgs<T> &A, long long &i, int &iz, int &iy, int &ix)
{
    ix = blockIdx.x * ADJ_BX + threadIdx.x;
    iy = blockIdx.y * ADJ_BY + threadIdx.y;
    iz = blockIdx.z;
    i = ((long long)iz * A.ny + iy) * A.nx + ix;
    return ix < A.nx && iy < A.ny;
}

// Every cell of this block lies at least ADJ_MARGIN_LO cells from the low
// faces and ADJ_MARGIN_HI from the high ones. Then every guard of the kernels
// below holds at every cell of the block: the transposed taps (DfT / DbT:
// forward cells y - 2j - 1 ... y + 2j + 1 with j <= 3, guards true for
// 7 <= y <= n - 8), the forward strains (4 <= y <= n - 5) and the moves and
// their transposes (2 <= y <= n - 3). Such blocks run the unguarded
// instantiations, whose arithmetic is the guarded one with every guard true.
constexpr int ADJ_MARGIN_LO = 7, ADJ_MARGIN_HI = 8;
template <typename T>
__device__ __forceinline__ bool adj_block_inside(const AdjArgs<T> &A)
{
    const int x0 = blockIdx.x * ADJ_BX, y0 = blockIdx.y * ADJ_BY, z = blockIdx.z;
    return x0 >= ADJ_MARGIN_LO && x0 + ADJ_BX - 1 <= A.nx - ADJ_MARGIN_HI && y0 >= ADJ_MARGIN_LO &&
           y0 + ADJ_BY - 1 <= A.ny - ADJ_MARGIN_HI && z >= ADJ_MARGIN_LO && z <= A.nz - ADJ_MARGIN_HI;
}

// The same test split by axis, for k_adj_strain and k_adj_velfin: a block inside
// along x (adj_inside_x) runs with the x guards compiled out (GX = false), a
// block inside along y and z (adj_inside_yz) with the y / z guards compiled
// out (GYZ = false); most blocks that miss the margins do so along one axis.
template <typename T>
__device__ __forceinline__ bool adj_inside_x(const AdjArgs<T> &A)
{
    const int x0 = blockIdx.x * ADJ_BX;
    return x0 >= ADJ_MARGIN_LO && x0 + ADJ_BX - 1 <= A.nx - ADJ_MARGIN_HI;
}
template <typename T>
__device__ __forceinline__ bool adj_inside_yz(const AdjArgs<T> &A)
{
    const int y0 = blockIdx.y * ADJ_BY, z = blockIdx.z;
    return y0 >= ADJ_MARGIN_LO && y0 + ADJ_BY - 1 <= A.ny - ADJ_MARGIN_HI && z >= ADJ_MARGIN_LO &&
           z <= A.nz - ADJ_MARGIN_HI;
}
// f<T, GX, GYZ>(args...) for this block's classification (block-uniform)
#define ADJ_DISPATCH(A, f, ...)                                          \
    do {                                                                 \
        const bool in_x_ = adj_inside_x(A), in_yz_ = adj_inside_yz(A);   \
        if (in_x_ && in_yz_) f<T, false, false>(__VA_ARGS__);            \
        else if (in_x_) f<T, false, true>(__VA_ARGS__);                  \
        else if (in_yz_) f<T, true, false>(__VA_ARGS__);                 \
        else f<T, true, true>(__VA_ARGS__);                              \
    } while (0)

// ---------------------------------------------------------------- receivers
// entries: cells[k] sorted, pos[k] = caller position; w and grp in caller order
template <typename T>
__global__ void k_adj_inject(AdjArgs<T> A, const long long *cells, const int *pos, const T *w,
                             const int *grp, int n_ent, const T *res_row, int kind, int damped)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_ent) return;
    const long long q = cells[k];
    const int e = pos[k];
    const T val = res_row[grp[e]] * w[e];
    if (kind == 0) {
        T f = -val / T(3);
        if (damped) {
            int iz, iy, ix;
            cell_of(A, q, iz, iy, ix);
            f = f * (T)adj_damp(A, iz, iy, ix, q);
        }
        atomicAdd(A.ls[0] + q, f);
        atomicAdd(A.ls[1] + q, f);
        atomicAdd(A.ls[2] + q, f);
    } else {
        atomicAdd(A.lv[kind - 1] + q, val);
    }
}

// ---------------------------------------------------------------- velocity transpose
// a / b rounded as the division; in FP32 through the reciprocal table
// (div_face_rcp: exact, without the float32 divide's slow path for the tiny
// adjoint values ahead of the back-propagating front)
template <typename T>
__device__ __forceinline__ T adj_div(T a, T b, T r0, const float *rinv, int m)
{
    return a / b;
}
template <>
__device__ __forceinline__ float adj_div<float>(float a, float b, float r0, const float *rinv, int m)
{
    return rinv ? div_face_rcp(a, b, b == r0, __ldg(rinv + m)) : a / b;
}

template <typename T>
__global__ void k_adj_vel_u(AdjArgs<T> A)
{
    long long i;
    int iz, iy, ix;
    if (!adj_cell(A, i, iz, iy, ix)) return;
    const int m0 = A.lab[i] & LAB_MAT;
    const T r0 = A.rho[m0];
    const T rvx = ix < A.nx - 1 ? T(0.5) * (r0 + A.rho[A.lab[i + 1] & LAB_MAT]) : r0;
    const T rvy = iy < A.ny - 1 ? T(0.5) * (r0 + A.rho[A.lab[i + A.sy] & LAB_MAT]) : r0;
    const T rvz = iz < A.nz - 1 ? T(0.5) * (r0 + A.rho[A.lab[i + A.sz] & LAB_MAT]) : r0;
    const T s = (T)adj_damp(A, iz, iy, ix, i) * A.dt_h;
    A.u[0][i] = adj_div(s * A.lv[0][i], rvx, r0, A.rinv, m0);
    A.u[1][i] = adj_div(s * A.lv[1][i], rvy, r0, A.rinv, m0);
    A.u[2][i] = adj_div(s * A.lv[2][i], rvz, r0, A.rinv, m0);
}

// index of the moved (position p, strain J) pairs, p != position of J:
// J = 0..5 in order, p ascending, three per strain
__host__ __device__ constexpr int adj_widx(int J, int p)
{
    return 3 * J + (p - (p > (J < 3 ? 0 : J - 2) ? 1 : 0));
}

// w[p][J](x) = sum over I at position p of C_IJ(x) * (dt * ls_I(x)), I
// ascending, for the moved pairs: the values the stress transpose gathers
// from the forward cells of each move tap. ls: the cell's ls after the
// velocity transpose, as k_adj_vel has just stored it.
template <typename T>
__device__ __forceinline__ void adj_w_cell(const AdjArgs<T> &A, long long i, const T (&ls)[6])
{
    const int VP[6] = {0, 0, 0, 1, 2, 3};
    const T *Cx = A.c21 + (long long)(A.lab[i] & LAB_MAT) * C21_STRIDE;
    T e[6];
#pragma unroll
    for (int I = 0; I < 6; ++I) e[I] = A.dt * ls[I];
#pragma unroll
    for (int J = 0; J < 6; ++J)
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            if (p == VP[J]) continue;
            T W = 0;
#pragma unroll
            for (int I = 0; I < 6; ++I)
                if (VP[I] == p) W += Cx[c21_slot(I, J)] * e[I];
            A.w[adj_widx(J, p)][i] = W;
        }
}

template <typename T, bool GX, bool GYZ>
__device__ __forceinline__ void adj_vel_cell(const AdjArgs<T> &A, long long i, int iz, int iy, int ix)
{
    const long long sy = A.sy, sz = A.sz;
    const T *ux = A.u[0] + i, *uy = A.u[1] + i, *uz = A.u[2] + i;
    auto X = [&](const T *p) { return [p](int o) { return p[o]; }; };
    auto Y = [&](const T *p) { return [p, sy](int o) { return p[o * sy]; }; };
    auto Z = [&](const T *p) { return [p, sz](int o) { return p[o * sz]; }; };
    T ls[6];
    ls[0] = A.ls[0][i] + DfT<T, GX>(X(ux), ix, A.nx, A.c, A.nc);
    ls[1] = A.ls[1][i] + DfT<T, GYZ>(Y(uy), iy, A.ny, A.c, A.nc);
    ls[2] = A.ls[2][i] + DfT<T, GYZ>(Z(uz), iz, A.nz, A.c, A.nc);
    ls[3] = A.ls[3][i] + (DbT<T, GYZ>(Z(uy), iz, A.nz, A.c, A.nc) + DbT<T, GYZ>(Y(uz), iy, A.ny, A.c, A.nc));
    ls[4] = A.ls[4][i] + (DbT<T, GYZ>(Z(ux), iz, A.nz, A.c, A.nc) + DbT<T, GX>(X(uz), ix, A.nx, A.c, A.nc));
    ls[5] = A.ls[5][i] + (DbT<T, GYZ>(Y(ux), iy, A.ny, A.c, A.nc) + DbT<T, GX>(X(uy), ix, A.nx, A.c, A.nc));
#pragma unroll
    for (int I = 0; I < 6; ++I) A.ls[I][i] = ls[I];
    adj_w_cell(A, i, ls);   // this cell's ls is final for the step until k_adj_stress damps it
}
// eight 256-thread blocks per SM in FP32 (32 registers, no spills; the
// stiffness columns formed at the end would otherwise take it to 40)
template <typename T>
__global__ void __launch_bounds__(ADJ_BX * ADJ_BY, sizeof(T) == 4 ? 8 : 4) k_adj_vel(AdjArgs<T> A)
{
    long long i;
    int iz, iy, ix;
    if (!adj_cell(A, i, iz, iy, ix)) return;
    // two instantiations (all guards or none): the four of ADJ_DISPATCH
    // measured slower here (more registers)
    if (adj_inside_x(A) && adj_inside_yz(A)) adj_vel_cell<T, false, false>(A, i, iz, iy, ix);
    else adj_vel_cell<T, true, true>(A, i, iz, iy, ix);
}

// ---------------------------------------------------------------- strains of v^{n-1}
template <typename T, bool GX, bool GYZ>
__device__ __forceinline__ void adj_strain_cell(const AdjArgs<T> &A, long long i, int iz, int iy, int ix)
{
    const long long sy = A.sy, sz = A.sz;
    const T *vx = A.vp[0], *vy = A.vp[1], *vz = A.vp[2];
    T a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
    // a skipped tap reads the cell itself twice: its difference is +0 and
    // fmac(a, c, +0) == a bit for bit, so the loads need not wait on guards
    auto d = [&](const T *f, bool ok, long long hi, long long lo) -> T {
        return f[ok ? i + hi : i] - f[ok ? i + lo : i];
    };
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (j < A.nc) {
            const T cj = A.c[j];
            const bool bx = !GX || gB(ix, j, A.nx), by = !GYZ || gB(iy, j, A.ny), bz = !GYZ || gB(iz, j, A.nz);
            const bool fx = !GX || gF(ix, j, A.nx), fy = !GYZ || gF(iy, j, A.ny), fz = !GYZ || gF(iz, j, A.nz);
            a1 = fmac(a1, cj, d(vx, bx, j, -(j + 1)));
            a2 = fmac(a2, cj, d(vy, by, j * sy, -(j + 1) * sy));
            a3 = fmac(a3, cj, d(vz, bz, j * sz, -(j + 1) * sz));
            a4 = fmac(a4, cj, d(vz, fy, (j + 1) * sy, -j * sy));
            a4 = fmac(a4, cj, d(vy, fz, (j + 1) * sz, -j * sz));
            a5 = fmac(a5, cj, d(vz, fx, j + 1, -j));
            a5 = fmac(a5, cj, d(vx, fz, (j + 1) * sz, -j * sz));
            a6 = fmac(a6, cj, d(vy, fx, j + 1, -j));
            a6 = fmac(a6, cj, d(vx, fy, (j + 1) * sy, -j * sy));
        }
    }
    const T ih = A.inv_h;
    A.g[0][i] = a1 * ih; A.g[1][i] = a2 * ih; A.g[2][i] = a3 * ih;
    A.g[3][i] = a4 * ih; A.g[4][i] = a5 * ih; A.g[5][i] = a6 * ih;
}
template <typename T>
__global__ void k_adj_strain(AdjArgs<T> A)
{
    long long i;
    int iz, iy, ix;
    if (!adj_cell(A, i, iz, iy, ix)) return;
    ADJ_DISPATCH(A, adj_strain_cell, A, i, iz, iy, ix);
}

// move guard at forward cell (z, y, x) for offsets d (exactly the forward's)
__device__ __forceinline__ bool move_ok(int z, int y, int x, int dz, int dy, int dx, int nz, int ny, int nx)
{
    if (z < 0 || z >= nz || y < 0 || y >= ny || x < 0 || x >= nx) return false;
    if (dz > 0 && z > nz - 2) return false;
    if (dz < 0 && z < 1) return false;
    if (dy > 0 && y > ny - 2) return false;
    if (dy < 0 && y < 1) return false;
    if (dx > 0 && x > nx - 2) return false;
    if (dx < 0 && x < 1) return false;
    return true;
}

// ---------------------------------------------------------------- stress transpose
constexpr int ADJ_STRESS_WARPS = ADJ_BY;   // k_adj_stress blocks: one warp per row of the 32 x 8 tile
static_assert(ADJ_BX == 32, "a warp is one row of an adjoint block");

// strain J moved to position P at cell i (the forward's half-cell move,
// same tap order). The taps are loaded unconditionally, from the cell itself
// where the move is off the grid, and masked afterwards: no load waits on a
// guard, so the gathers of a cell are all in flight together.
template <typename T, int P, int J, bool G>
__device__ __forceinline__ T adj_q(const AdjArgs<T> &A, long long i, int iz, int iy, int ix)
{
    constexpr int S = vpos(J);
    constexpr int DZ = pos_z(P) - pos_z(S), DY = pos_y(P) - pos_y(S), DX = pos_x(P) - pos_x(S);
    if constexpr (DZ == 0 && DY == 0 && DX == 0) {
        return A.g[J][i];
    } else {
        const bool ok = !G || move_ok(iz, iy, ix, DZ, DY, DX, A.nz, A.ny, A.nx);
        const T *g = A.g[J];
        T acc = 0;
#pragma unroll
        for (int a0 = (DZ < 0 ? -1 : 0); a0 <= (DZ > 0 ? 1 : 0); ++a0)
#pragma unroll
            for (int a1 = (DY < 0 ? -1 : 0); a1 <= (DY > 0 ? 1 : 0); ++a1)
#pragma unroll
                for (int a2 = (DX < 0 ? -1 : 0); a2 <= (DX > 0 ? 1 : 0); ++a2)
                    acc += g[ok ? i + a0 * A.sz + a1 * A.sy + a2 : i];
        return ok ? acc * T(0.25) : T(0);
    }
}

// strain adjoint t_J, the contribution of position P: the direct term (P the
// position of J) or the transposed move of W[P][J] gathered from the forward
// cells x = i - o of every tap offset o (guards evaluated at x, loads
// unconditional as in adj_q)
template <typename T, int J, int P, bool G>
__device__ __forceinline__ void adj_t(const AdjArgs<T> &A, long long i, int iz, int iy, int ix, const T *Cm,
                                      const T (&e)[6], T &acc)
{
    constexpr int S = vpos(J);
    constexpr int DZ = pos_z(P) - pos_z(S), DY = pos_y(P) - pos_y(S), DX = pos_x(P) - pos_x(S);
    if constexpr (DZ == 0 && DY == 0 && DX == 0) {
#pragma unroll
        for (int I = 0; I < 6; ++I)
            if (vpos(I) == P) acc += Cm[c21_slot(I, J)] * e[I];
    } else {
        const T *w = A.w[adj_widx(J, P)];
#pragma unroll
        for (int a0 = (DZ < 0 ? -1 : 0); a0 <= (DZ > 0 ? 1 : 0); ++a0)
#pragma unroll
            for (int a1 = (DY < 0 ? -1 : 0); a1 <= (DY > 0 ? 1 : 0); ++a1)
#pragma unroll
                for (int a2 = (DX < 0 ? -1 : 0); a2 <= (DX > 0 ? 1 : 0); ++a2) {
                    const bool ok = !G || move_ok(iz - a0, iy - a1, ix - a2, DZ, DY, DX, A.nz, A.ny, A.nx);
                    const T v = w[ok ? i - a0 * A.sz - a1 * A.sy - a2 : i];
                    acc += T(0.25) * (ok ? v : T(0));
                }
    }
}

template <typename T, int J, bool G>
__device__ __forceinline__ T adj_tJ(const AdjArgs<T> &A, long long i, int iz, int iy, int ix, const T *Cm,
                                    const T (&e)[6])
{
    T acc = 0;
    adj_t<T, J, 0, G>(A, i, iz, iy, ix, Cm, e, acc);
    adj_t<T, J, 1, G>(A, i, iz, iy, ix, Cm, e, acc);
    adj_t<T, J, 2, G>(A, i, iz, iy, ix, Cm, e, acc);
    adj_t<T, J, 3, G>(A, i, iz, iy, ix, Cm, e, acc);
    return acc;
}

template <typename T, int P, bool G>
__device__ __forceinline__ void adj_qrow(const AdjArgs<T> &A, long long i, int iz, int iy, int ix, T (&q)[6])
{
    q[0] = adj_q<T, P, 0, G>(A, i, iz, iy, ix);
    q[1] = adj_q<T, P, 1, G>(A, i, iz, iy, ix);
    q[2] = adj_q<T, P, 2, G>(A, i, iz, iy, ix);
    q[3] = adj_q<T, P, 3, G>(A, i, iz, iy, ix);
    q[4] = adj_q<T, P, 4, G>(A, i, iz, iy, ix);
    q[5] = adj_q<T, P, 5, G>(A, i, iz, iy, ix);
}

// the cell's 21 gradient terms into its row of the warp's reduction tile
template <typename T, bool G>
__device__ __forceinline__ bool adj_grad_terms(const AdjArgs<T> &A, long long i, int iz, int iy, int ix,
                                               const T (&e)[6], T *row)
{
    // moved strains at this cell, q[p][J]
    T q[4][6];
    adj_qrow<T, 0, G>(A, i, iz, iy, ix, q[0]);
    adj_qrow<T, 1, G>(A, i, iz, iy, ix, q[1]);
    adj_qrow<T, 2, G>(A, i, iz, iy, ix, q[2]);
    adj_qrow<T, 3, G>(A, i, iz, iy, ix, q[3]);
    // dJ/dC_IJ for I <= J: e_I q[p(I)][J] + e_J q[p(J)][I]  (I != J),
    // formed in the solve's precision (in FP32 one rounding of the
    // cell's term, as its fields carry) and summed over cells in f64
    bool any = false;
#pragma unroll
    for (int I = 0; I < 6; ++I)
#pragma unroll
        for (int J = I; J < 6; ++J) {
            T v = e[I] * q[vpos(I)][J];
            if (J != I) v += e[J] * q[vpos(J)][I];
            row[c21_slot(I, J)] = v;
            any = any || v != T(0);
        }
    return any;
}

// strain adjoint t_J: direct term plus transposed moves of
// W[p][J](x) = sum_{I at p} C_IJ(x) e_I(x) from the forward cells x
template <typename T, bool G>
__device__ __forceinline__ void adj_strain_adjoint(const AdjArgs<T> &A, long long i, int iz, int iy, int ix,
                                                   const T *Cm, const T (&e)[6])
{
    A.t[0][i] = adj_tJ<T, 0, G>(A, i, iz, iy, ix, Cm, e);
    A.t[1][i] = adj_tJ<T, 1, G>(A, i, iz, iy, ix, Cm, e);
    A.t[2][i] = adj_tJ<T, 2, G>(A, i, iz, iy, ix, Cm, e);
    A.t[3][i] = adj_tJ<T, 3, G>(A, i, iz, iy, ix, Cm, e);
    A.t[4][i] = adj_tJ<T, 4, G>(A, i, iz, iy, ix, Cm, e);
    A.t[5][i] = adj_tJ<T, 5, G>(A, i, iz, iy, ix, Cm, e);
}

template <typename T>
__global__ void __launch_bounds__(ADJ_STRESS_WARPS * 32) k_adj_stress(AdjArgs<T> A)
{
    long long i;
    int iz, iy, ix;
    const bool live = adj_cell(A, i, iz, iy, ix);
    // Per-material gradient, summed per warp: every lane writes its 21 terms
    // to its row of the warp's 32 x 21 tile in shared memory (zero where the
    // cell is off the grid), then for each distinct material of the warp
    // lanes 0..20 each add up one column over the lanes of that material and
    // issue the 21 f64 atomics together. Writing the terms out as they are
    // formed keeps them out of registers during the gathers that follow.
    // Warps add into one of grad_rep replicas of the table (by warp index),
    // so that the warps of a large single-material region (the couplant) do
    // not all serialise on the same 21 addresses. The tile holds the terms in
    // the solve's precision (each is one rounding in T) and the column sums
    // convert them to f64 as they add them, exactly: in FP32 this halves the
    // tile (21.5 KB per block) and leaves that much more of the SM's unified
    // L1 to the gathers. Tile rows are 21 elements apart (odd): row stores and
    // column loads are free of bank conflicts.
    __shared__ T red[ADJ_STRESS_WARPS][32][21];
    __shared__ int rmat[ADJ_STRESS_WARPS][32];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.y;
    int m = -1;
    bool any = false;
    T e[6];
    const bool inside = adj_block_inside(A);   // block-uniform
    if (live) {
        m = A.lab[i] & LAB_MAT;
#pragma unroll
        for (int I = 0; I < 6; ++I) e[I] = A.dt * A.ls[I][i];
        any = inside ? adj_grad_terms<T, false>(A, i, iz, iy, ix, e, red[warp][lane])
                     : adj_grad_terms<T, true>(A, i, iz, iy, ix, e, red[warp][lane]);
    } else {
#pragma unroll
        for (int k = 0; k < 21; ++k) red[warp][lane][k] = T(0);
    }
    rmat[warp][lane] = m;
    __syncwarp();
    double *gtab = A.grad;
    if (A.grad_rep > 1)
        gtab += (long long)(((blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x * ADJ_BY + blockIdx.x * ADJ_BY + warp) %
                            (unsigned)A.grad_rep) * A.n_mat * 21;
    // lanes whose 21 terms are all zero (no overlap of the adjoint stress
    // and the forward strain at the cell) add nothing and sit out
    unsigned remaining = __ballot_sync(full, live && any);
    const int my = live && any ? m : -1;
    while (remaining) {
        const int src = __ffs(remaining) - 1;
        const int mm = __shfl_sync(full, my, src);
        remaining &= ~__ballot_sync(full, my == mm);
        if (lane < 21) {
            double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;   // four chains, for latency
#pragma unroll
            for (int r = 0; r < 32; r += 4) {
                v0 += rmat[warp][r] == mm ? (double)red[warp][r][lane] : 0.0;
                v1 += rmat[warp][r + 1] == mm ? (double)red[warp][r + 1][lane] : 0.0;
                v2 += rmat[warp][r + 2] == mm ? (double)red[warp][r + 2][lane] : 0.0;
                v3 += rmat[warp][r + 3] == mm ? (double)red[warp][r + 3][lane] : 0.0;
            }
            atomicAdd(gtab + (long long)mm * 21 + lane, (v0 + v1) + (v2 + v3));
        }
    }
    if (!live) return;
    const T *Cm = A.c21 + (long long)m * C21_STRIDE;
    if (inside) adj_strain_adjoint<T, false>(A, i, iz, iy, ix, Cm, e);
    else adj_strain_adjoint<T, true>(A, i, iz, iy, ix, Cm, e);
    // the step's last use of ls at this cell (k_adj_vel formed w from it, and only
    // this thread reads it here): apply the deferred damping, ls = d ls (the
    // transpose of the forward s^{n-1} * d)
    const T d = (T)adj_damp(A, iz, iy, ix, i);
#pragma unroll
    for (int I = 0; I < 6; ++I) A.ls[I][i] = d * A.ls[I][i];
}

// grad += sum of the replicas, which are left zero
__global__ void k_grad_fold(double *rep, int nrep, long long len, double *grad)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= len) return;
    double s = 0.0;
    for (int r = 0; r < nrep; ++r) {
        s += rep[(long long)r * len + i];
        rep[(long long)r * len + i] = 0.0;
    }
    grad[i] += s;
}

template <typename T, bool GX, bool GYZ>
__device__ __forceinline__ void adj_velfin_cell(const AdjArgs<T> &A, long long i, int iz, int iy, int ix)
{
    const long long sy = A.sy, sz = A.sz;
    auto X = [&](const T *p) { return [p](int o) { return p[o]; }; };
    auto Y = [&](const T *p) { return [p, sy](int o) { return p[o * sy]; }; };
    auto Z = [&](const T *p) { return [p, sz](int o) { return p[o * sz]; }; };
    const T *t1 = A.t[0] + i, *t2 = A.t[1] + i, *t3 = A.t[2] + i;
    const T *t4 = A.t[3] + i, *t5 = A.t[4] + i, *t6 = A.t[5] + i;
    const T d = (T)adj_damp(A, iz, iy, ix, i);
    const T ih = A.inv_h;
    const T gx = DbT<T, GX>(X(t1), ix, A.nx, A.c, A.nc) + DfT<T, GYZ>(Z(t5), iz, A.nz, A.c, A.nc) +
                 DfT<T, GYZ>(Y(t6), iy, A.ny, A.c, A.nc);
    const T gy = DbT<T, GYZ>(Y(t2), iy, A.ny, A.c, A.nc) + DfT<T, GYZ>(Z(t4), iz, A.nz, A.c, A.nc) +
                 DfT<T, GX>(X(t6), ix, A.nx, A.c, A.nc);
    const T gz = DbT<T, GYZ>(Z(t3), iz, A.nz, A.c, A.nc) + DfT<T, GYZ>(Y(t4), iy, A.ny, A.c, A.nc) +
                 DfT<T, GX>(X(t5), ix, A.nx, A.c, A.nc);
    A.lv[0][i] = d * A.lv[0][i] + ih * gx;
    A.lv[1][i] = d * A.lv[1][i] + ih * gy;
    A.lv[2][i] = d * A.lv[2][i] + ih * gz;
}
template <typename T>
__global__ void k_adj_velfin(AdjArgs<T> A)
{
    long long i;
    int iz, iy, ix;
    if (!adj_cell(A, i, iz, iy, ix)) return;
    ADJ_DISPATCH(A, adj_velfin_cell, A, i, iz, iy, ix);
}

#undef ADJ_DISPATCH

}  // namespace pe
