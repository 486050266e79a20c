// Shared-memory tiled step kernels (the default path).
//
// Same arithmetic, term order and explicit FMA placement as the simple
// kernels in pe_kernels.cuh (and the oracle); only the data movement differs.
// Each block marches z over a 32 x 16 column tile and never consumes a global
// value in the plane iteration that requested it:
//  - the xy stencil taps and every per-cell operand of a plane (the other
//    fields of the cell, the damping volume) are copied into shared memory
//    by cp.async two planes ahead (three slots, zero-filled off the grid);
//  - the z taps come from per-thread register rings refilled one plane ahead,
//    and labels are prefetched one plane ahead into registers;
//  - the per-material stiffness / density table sits in shared memory.
// In k_stress_t the 512 threads are the strain columns of the tile including
// a one-column halo, so every strain value the half-cell moves need is
// computed once per block; the inner 30 x 14 threads update the stress.
// Tiles whose every tap lies inside the grid run without x/y guards.
#pragma once
#include "pe_kernels.cuh"

namespace pe {

// ---------------------------------------------------------------- cp.async
template <int BYTES>
__device__ __forceinline__ void cp_async_el(void *smem, const void *gmem, bool ok)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = ok ? BYTES : 0;   // src-size 0: zero-fill, no global read
    if constexpr (BYTES == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

constexpr int TB_X = 32, TB_Y = 16, TB_N = TB_X * TB_Y;  // block = thread tile
constexpr int TS_OX = TB_X - 2, TS_OY = TB_Y - 2;       // stress outputs per block
constexpr int T_H = 4;                                  // tap reach
constexpr int T_W = TB_X + 2 * T_H, T_HT = TB_Y + 2 * T_H, T_SZ = T_W * T_HT;  // 40 x 24
constexpr int T_SLOTS = 3;
constexpr int V_FIELDS = 5;  // s1, s2, s4, s5, s6 carry xy taps in the velocity update
// largest table kept in shared memory (rows of C21_STRIDE values)
constexpr int SMEM_TABLE_MAX = 1024;

// per-slot layouts (elements of T)
constexpr int S_VT = 3 * T_SZ;            // stress: v tile
constexpr int S_SC = 7 * TB_N;            // stress: s1..s6 + damping of the output cells
constexpr int V_ST = V_FIELDS * T_SZ;     // velocity: s tile
constexpr int V_VC = 4 * TB_N;            // velocity: vx, vy, vz + damping of the cells

template <typename T>
__host__ __device__ constexpr bool table_in_smem(int n_mat)
{
    return sizeof(T) == 4 && n_mat <= SMEM_TABLE_MAX;
}
template <typename T>
__host__ __device__ constexpr size_t stress_tiled_smem(int n_mat)
{
    return sizeof(T) * ((size_t)T_SLOTS * (S_VT + S_SC) + (size_t)3 * 6 * TB_N +
                        (table_in_smem<T>(n_mat) ? (size_t)n_mat * C21_STRIDE : 0));
}
template <typename T>
__host__ __device__ constexpr size_t velocity_tiled_smem(int n_mat)
{
    return sizeof(T) * ((size_t)T_SLOTS * (V_ST + V_VC) + (table_in_smem<T>(n_mat) ? (size_t)n_mat : 0));
}

template <typename T>
__device__ __forceinline__ void load_c21(const T *Cr, bool shared, T Cm[24])
{
    if constexpr (sizeof(T) == 4) {
        const float4 *p = reinterpret_cast<const float4 *>(Cr);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float4 u = shared ? p[k] : __ldg(p + k);
            Cm[4 * k] = u.x; Cm[4 * k + 1] = u.y; Cm[4 * k + 2] = u.z; Cm[4 * k + 3] = u.w;
        }
    } else {
        const double2 *p = reinterpret_cast<const double2 *>(Cr);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const double2 u = __ldg(p + k);
            Cm[2 * k] = u.x; Cm[2 * k + 1] = u.y;
        }
    }
}

// The (up to) two positions of a 40 x 24 tile plane this thread copies, with
// their in-plane global offsets and whether they lie inside the grid.
struct TileLanes {
    int p0, p1;          // tile positions (p1 < 0: none)
    int g0, g1;          // iy * sy + ix, or 0 when outside
    bool ok0, ok1;
};

__device__ __forceinline__ TileLanes tile_lanes(int tid, int ox, int oy, int nx, int ny, long long sy)
{
    TileLanes L;
    L.p0 = tid;
    L.p1 = tid + TB_N < T_SZ ? tid + TB_N : -1;
    {
        const int hy = L.p0 / T_W, hx = L.p0 - hy * T_W;
        const int iy = oy + hy, ix = ox + hx;
        L.ok0 = ix >= 0 && ix < nx && iy >= 0 && iy < ny;
        L.g0 = L.ok0 ? (int)(iy * sy + ix) : 0;
    }
    if (L.p1 >= 0) {
        const int hy = L.p1 / T_W, hx = L.p1 - hy * T_W;
        const int iy = oy + hy, ix = ox + hx;
        L.ok1 = ix >= 0 && ix < nx && iy >= 0 && iy < ny;
        L.g1 = L.ok1 ? (int)(iy * sy + ix) : 0;
    } else {
        L.ok1 = false;
        L.g1 = 0;
    }
    return L;
}

template <typename T>
__device__ __forceinline__ void tile_copy(T *dst, const T *plane, const TileLanes &L, bool zok)
{
    cp_async_el<sizeof(T)>(dst + L.p0, plane + L.g0, zok && L.ok0);
    if (L.p1 >= 0) cp_async_el<sizeof(T)>(dst + L.p1, plane + L.g1, zok && L.ok1);
}

// ---------------------------------------------------------------- stress
template <typename T, bool EDGE>
__device__ __forceinline__ void stress_tiled_run(const StepArgs<T> &A, T *slots, T *gs,
                                                 const T *tab, bool tab_smem)
{
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TB_X + tx;
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long sy = A.sy, sz = A.sz;
    const int X0 = blockIdx.x * TS_OX - 1, Y0 = blockIdx.y * TS_OY - 1;
    const int gx = X0 + tx, gy = Y0 + ty;
    const bool col_ok = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
    const int col = col_ok ? (int)(gy * sy + gx) : 0;
    const int zb = blockIdx.z * A.zc;
    const int ze = min(zb + A.zc, nz);
    const T *vx = A.v[0], *vy = A.v[1], *vz = A.v[2];
    const long long n = *A.step + A.k;
    const T wn = A.n_src ? A.wavelet[n] : T(0);
    const bool has_dvol = A.dvol != nullptr;
    T *const vt_base = slots;                          // [3][S_VT]
    T *const sc_base = slots + (size_t)T_SLOTS * S_VT; // [3][S_SC]
    const TileLanes L = tile_lanes(tid, X0 - T_H, Y0 - T_H, nx, ny, sy);

    // group i: v tile of plane i+2 and the output cells' s / damping of plane i+1
    auto issue = [&](int qv, int qs) {
        {
            T *dst = vt_base + (size_t)((qv + 3) % 3) * S_VT;
            const bool zok = qv >= 0 && qv < nz;
            const long long po = zok ? (long long)qv * sz : 0;
            tile_copy(dst, vx + po, L, zok);
            tile_copy(dst + T_SZ, vy + po, L, zok);
            tile_copy(dst + 2 * T_SZ, vz + po, L, zok);
        }
        if (qs >= zb && qs < ze) {
            T *dst = sc_base + (size_t)((qs + 3) % 3) * S_SC + tid;
            const long long po = (long long)qs * sz + col;
#pragma unroll
            for (int I = 0; I < 6; ++I) cp_async_el<sizeof(T)>(dst + I * TB_N, A.s[I] + po, col_ok);
            if (has_dvol) cp_async_el<4>(reinterpret_cast<float *>(dst + 6 * TB_N), A.dvol + po, col_ok);
        }
        cp_async_commit();
    };
    auto ldcol = [&](const T *f, int q) -> T {
        return (col_ok && q >= 0 && q < nz) ? ldg(f + (long long)q * sz + col) : T(0);
    };

    const int q0 = zb - 1;
    T rz[8], ry[8], rx[8];   // rz[k] <-> plane q-4+k (Dbz taps), ry/rx[k] <-> q-3+k (Dfz)
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        rz[k] = ldcol(vz, q0 - 4 + k);
        ry[k] = ldcol(vy, q0 - 3 + k);
        rx[k] = ldcol(vx, q0 - 3 + k);
    }
    bool xb[4], xf[4], yb[4], yf[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        xb[j] = !EDGE || (gx >= j + 1 && gx < nx - j);
        xf[j] = !EDGE || (gx >= j && gx < nx - j - 1);
        yb[j] = !EDGE || (gy >= j + 1 && gy < ny - j);
        yf[j] = !EDGE || (gy >= j && gy < ny - j - 1);
    }
    const bool xlo = !EDGE || gx >= 1, xhi = !EDGE || gx <= nx - 2;
    const bool ylo = !EDGE || gy >= 1, yhi = !EDGE || gy <= ny - 2;
    const bool is_out = tx >= 1 && tx <= TS_OX && ty >= 1 && ty <= TS_OY && gx < nx && gy < ny;
    float dyx = 1.0f, dxx = 1.0f;
    if (A.dz && is_out) { dyx = A.dy[gy]; dxx = A.dx[gx]; }
    const int tc = (ty + T_H) * T_W + tx + T_H;
    uint16_t lab_next = (is_out && zb < nz) ? A.lab[(long long)zb * sz + col] : 0;

    issue(q0, -1);
    issue(q0 + 1, q0);
    for (int q = q0; q <= ze; ++q) {
        cp_async_wait<1>();
        __syncthreads();
        issue(q + 2, q + 1);
        const T nzv = ldcol(vz, q + 4), nyv = ldcol(vy, q + 5), nxv = ldcol(vx, q + 5);
        const int z = q - 1;
        const uint16_t lab = lab_next;
        if (is_out && z >= zb && q < ze) lab_next = A.lab[(long long)q * sz + col];
        // ---------- strains at plane q, this column
        {
            const T *t = vt_base + (size_t)((q + 3) % 3) * S_VT + tc;
            const T *tvx = t, *tvy = t + T_SZ, *tvz = t + 2 * T_SZ;
            T a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (j < A.nc) {
                    const T cj = A.c[j];
                    const bool zbj = q >= j + 1 && q < nz - j, zfj = q >= j && q < nz - j - 1;
                    if (xb[j]) a1 = fmac(a1, cj, tvx[j] - tvx[-(j + 1)]);
                    if (yb[j]) a2 = fmac(a2, cj, tvy[j * T_W] - tvy[-(j + 1) * T_W]);
                    if (zbj) a3 = fmac(a3, cj, rz[4 + j] - rz[3 - j]);
                    if (yf[j]) a4 = fmac(a4, cj, tvz[(j + 1) * T_W] - tvz[-j * T_W]);
                    if (zfj) a4 = fmac(a4, cj, ry[4 + j] - ry[3 - j]);
                    if (xf[j]) a5 = fmac(a5, cj, tvz[j + 1] - tvz[-j]);
                    if (zfj) a5 = fmac(a5, cj, rx[4 + j] - rx[3 - j]);
                    if (xf[j]) a6 = fmac(a6, cj, tvy[j + 1] - tvy[-j]);
                    if (yf[j]) a6 = fmac(a6, cj, tvx[(j + 1) * T_W] - tvx[-j * T_W]);
                }
            }
            const T ih = A.inv_h;
            T *g = gs + (size_t)((q + 3) % 3) * 6 * TB_N + tid;
            g[0 * TB_N] = a1 * ih; g[1 * TB_N] = a2 * ih; g[2 * TB_N] = a3 * ih;
            g[3 * TB_N] = a4 * ih; g[4 * TB_N] = a5 * ih; g[5 * TB_N] = a6 * ih;
        }
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            rz[k] = rz[k + 1];
            ry[k] = ry[k + 1];
            rx[k] = rx[k + 1];
        }
        rz[7] = nzv;
        ry[7] = nyv;
        rx[7] = nxv;
        __syncthreads();
        // ---------- stress at plane z = q - 1
        if (z >= zb && is_out) {
            const T *gm = gs + (size_t)((q + 1) % 3) * 6 * TB_N + tid;   // plane z-1
            const T *g0 = gs + (size_t)((q + 2) % 3) * 6 * TB_N + tid;   // plane z
            const T *gp = gs + (size_t)(q % 3) * 6 * TB_N + tid;         // plane z+1
            auto G = [&](int J, int dz, int dy, int dx) -> T {
                const T *b = dz < 0 ? gm : (dz > 0 ? gp : g0);
                return b[J * TB_N + dy * TB_X + dx];
            };
            const bool zlo = z >= 1, zhi = z <= nz - 2;
            T q0v[6], q1v[6], q2v[6], q3v[6];
            qrow<0>(G, zlo, zhi, ylo, yhi, xlo, xhi, q0v);
            qrow<1>(G, zlo, zhi, ylo, yhi, xlo, xhi, q1v);
            qrow<2>(G, zlo, zhi, ylo, yhi, xlo, xhi, q2v);
            qrow<3>(G, zlo, zhi, ylo, yhi, xlo, xhi, q3v);
            const T *sc = sc_base + (size_t)((z + 3) % 3) * S_SC + tid;
            T Cm[24];
            load_c21(tab + (size_t)(lab & LAB_MAT) * C21_STRIDE, tab_smem, Cm);
            float d = 1.0f;
            if (A.dz) {
                d = A.dz[z] * dyx;
                d = d * dxx;
            }
            if (has_dvol) {
                const float dv = reinterpret_cast<const float *>(sc + 6 * TB_N)[0];
                d = A.dz ? d * dv : dv;
            }
            const T dmp = (T)d;
            T acc[6];
            acc[0] = row_dot(Cm, 0, q0v);
            acc[1] = row_dot(Cm, 1, q0v);
            acc[2] = row_dot(Cm, 2, q0v);
            acc[3] = row_dot(Cm, 3, q1v);
            acc[4] = row_dot(Cm, 4, q2v);
            acc[5] = row_dot(Cm, 5, q3v);
            T sv[6];
#pragma unroll
            for (int I = 0; I < 6; ++I) {
                const T s = sc[I * TB_N] * dmp;
                sv[I] = fmac(s, A.dt, acc[I]);
            }
            const long long idx = (long long)z * sz + col;
            if (lab & LAB_SRC) {
                const int e = lower_bound_ll(A.src_idx, A.n_src, idx);
                if (e < A.n_src && A.src_idx[e] == idx) {
                    const T add = wn * A.src_w[e];
                    sv[0] = sv[0] + add;
                    sv[1] = sv[1] + add;
                    sv[2] = sv[2] + add;
                }
            }
#pragma unroll
            for (int I = 0; I < 6; ++I) A.s[I][idx] = sv[I];
            if ((lab & LAB_REC) && A.rec_kind == 0) {
                T a = sv[0], b = sv[1], c = sv[2];
                if (A.rec_damped) { a = a * dmp; b = b * dmp; c = c * dmp; }
                T t = a + b;
                t = t + c;
                record_cell(A, idx, -t / T(3));
            }
        }
    }
    cp_async_wait<0>();
}

template <typename T>
__global__ void __launch_bounds__(TB_N, 1) k_stress_t(const StepArgs<T> A, int n_mat)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *slots = reinterpret_cast<T *>(smem_raw);
    T *gs = slots + (size_t)T_SLOTS * (S_VT + S_SC);
    T *tsm = gs + (size_t)3 * 6 * TB_N;
    const bool tab_smem = table_in_smem<T>(n_mat);
    if (tab_smem) {
        const int tid = threadIdx.y * TB_X + threadIdx.x;
        for (int i = tid; i < n_mat * C21_STRIDE; i += TB_N) tsm[i] = A.c21[i];
        // made visible by the first barrier of the march
    }
    const T *tab = tab_smem ? tsm : A.c21;
    const int X0 = blockIdx.x * TS_OX - 1, Y0 = blockIdx.y * TS_OY - 1;
    const bool inner = X0 - T_H >= 0 && X0 + TB_X - 1 + T_H < A.nx && Y0 - T_H >= 0 &&
                       Y0 + TB_Y - 1 + T_H < A.ny;
    if (inner) stress_tiled_run<T, false>(A, slots, gs, tab, tab_smem);
    else stress_tiled_run<T, true>(A, slots, gs, tab, tab_smem);
}

// ---------------------------------------------------------------- velocity
template <typename T, bool EDGE>
__device__ __forceinline__ void velocity_tiled_run(const StepArgs<T> &A, T *slots,
                                                   const T *rho_tab)
{
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TB_X + tx;
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long sy = A.sy, sz = A.sz;
    const int x0 = blockIdx.x * TB_X, y0 = blockIdx.y * TB_Y;
    const int ix = x0 + tx, iy = y0 + ty;
    const bool out_ok = ix < nx && iy < ny;
    const int col = out_ok ? (int)(iy * sy + ix) : 0;
    const int zb = blockIdx.z * A.zc;
    const int ze = min(zb + A.zc, nz);
    const T *s3 = A.s[2], *s4 = A.s[3], *s5 = A.s[4];
    const T *tf[V_FIELDS] = {A.s[0], A.s[1], A.s[3], A.s[4], A.s[5]};
    const bool has_dvol = A.dvol != nullptr;
    const TileLanes L = tile_lanes(tid, x0 - T_H, y0 - T_H, nx, ny, sy);

    // group z: s tile and the cells' v / damping of plane z
    auto issue = [&](int z) {
        T *dst = slots + (size_t)((z + 3) % 3) * (V_ST + V_VC);
        const bool zok = z >= zb && z < ze;
        const long long po = zok ? (long long)z * sz : 0;
#pragma unroll
        for (int f = 0; f < V_FIELDS; ++f) tile_copy(dst + f * T_SZ, tf[f] + po, L, zok);
        T *vc = dst + V_ST + tid;
#pragma unroll
        for (int c = 0; c < 3; ++c) cp_async_el<sizeof(T)>(vc + c * TB_N, A.v[c] + po + col, zok && out_ok);
        if (has_dvol)
            cp_async_el<4>(reinterpret_cast<float *>(vc + 3 * TB_N), A.dvol + po + col, zok && out_ok);
        cp_async_commit();
    };
    auto ldcol = [&](const T *f, int z) -> T {
        return (out_ok && z >= 0 && z < nz) ? ldg(f + (long long)z * sz + col) : T(0);
    };
    auto ldlab = [&](long long i, bool ok) -> uint16_t { return ok ? A.lab[i] : (uint16_t)0; };

    T r3[8], r4[8], r5[8];   // r3[k] <-> z-3+k (s3 forward taps), r4/r5[k] <-> z-4+k
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        r3[k] = ldcol(s3, zb - 3 + k);
        r4[k] = ldcol(s4, zb - 4 + k);
        r5[k] = ldcol(s5, zb - 4 + k);
    }
    bool xb[4], xf[4], yb[4], yf[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        xb[j] = !EDGE || (ix >= j + 1 && ix < nx - j);
        xf[j] = !EDGE || (ix >= j && ix < nx - j - 1);
        yb[j] = !EDGE || (iy >= j + 1 && iy < ny - j);
        yf[j] = !EDGE || (iy >= j && iy < ny - j - 1);
    }
    const bool xin = ix < nx - 1, yin = iy < ny - 1;
    float dyx = 1.0f, dxx = 1.0f;
    if (A.dz && out_ok) { dyx = A.dy[iy]; dxx = A.dx[ix]; }
    const int tc = (ty + T_H) * T_W + tx + T_H;
    // labels: own cell at z and z+1, +x / +y neighbours at z (prefetched a plane ahead)
    long long cz = (long long)zb * sz + col;
    uint16_t lab_c = ldlab(cz, out_ok && zb < nz);
    uint16_t lab_z = ldlab(cz + sz, out_ok && zb + 1 < nz);
    uint16_t lab_x = ldlab(cz + 1, out_ok && xin && zb < nz);
    uint16_t lab_y = ldlab(cz + sy, out_ok && yin && zb < nz);

    issue(zb);
    issue(zb + 1);
    for (int z = zb; z < ze; ++z) {
        cp_async_wait<1>();
        __syncthreads();
        issue(z + 2);
        const T n3 = ldcol(s3, z + 5), n4 = ldcol(s4, z + 4), n5 = ldcol(s5, z + 4);
        const long long cn = (long long)(z + 1) * sz + col;
        const uint16_t nlab_z = ldlab(cn + sz, out_ok && z + 2 < nz);
        const uint16_t nlab_x = ldlab(cn + 1, out_ok && xin && z + 1 < nz);
        const uint16_t nlab_y = ldlab(cn + sy, out_ok && yin && z + 1 < nz);
        const T *slot = slots + (size_t)((z + 3) % 3) * (V_ST + V_VC);
        const T *t = slot + tc;
        const T *t1 = t, *t2 = t + T_SZ, *t4 = t + 2 * T_SZ, *t5 = t + 3 * T_SZ, *t6 = t + 4 * T_SZ;
        T ax = 0, ay = 0, az = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (j < A.nc) {
                const T cj = A.c[j];
                if (xf[j]) ax = fmac(ax, cj, t1[j + 1] - t1[-j]);
                if (xb[j]) {
                    ay = fmac(ay, cj, t6[j] - t6[-(j + 1)]);
                    az = fmac(az, cj, t5[j] - t5[-(j + 1)]);
                }
                if (yf[j]) ay = fmac(ay, cj, t2[(j + 1) * T_W] - t2[-j * T_W]);
                if (yb[j]) {
                    ax = fmac(ax, cj, t6[j * T_W] - t6[-(j + 1) * T_W]);
                    az = fmac(az, cj, t4[j * T_W] - t4[-(j + 1) * T_W]);
                }
                if (z >= j && z < nz - j - 1) az = fmac(az, cj, r3[4 + j] - r3[3 - j]);
                if (z >= j + 1 && z < nz - j) {
                    ax = fmac(ax, cj, r5[4 + j] - r5[3 - j]);
                    ay = fmac(ay, cj, r4[4 + j] - r4[3 - j]);
                }
            }
        }
        if (out_ok) {
            const T r0 = rho_tab[lab_c & LAB_MAT];
            const T rvx = xin ? T(0.5) * (r0 + rho_tab[lab_x & LAB_MAT]) : r0;
            const T rvy = yin ? T(0.5) * (r0 + rho_tab[lab_y & LAB_MAT]) : r0;
            const T rvz = (z < nz - 1) ? T(0.5) * (r0 + rho_tab[lab_z & LAB_MAT]) : r0;
            const T *vc = slot + V_ST + tid;
            float d = 1.0f;
            if (A.dz) {
                d = A.dz[z] * dyx;
                d = d * dxx;
            }
            if (has_dvol) {
                const float dv = reinterpret_cast<const float *>(vc + 3 * TB_N)[0];
                d = A.dz ? d * dv : dv;
            }
            const T dmp = (T)d;
            T ux = A.dt_h * ax, uy = A.dt_h * ay, uz = A.dt_h * az;
            ux = div_face(ux, rvx);
            uy = div_face(uy, rvy);
            uz = div_face(uz, rvz);
            const T vxn = (vc[0] + ux) * dmp;
            const T vyn = (vc[TB_N] + uy) * dmp;
            const T vzn = (vc[2 * TB_N] + uz) * dmp;
            const long long idx = (long long)z * sz + col;
            A.v[0][idx] = vxn;
            A.v[1][idx] = vyn;
            A.v[2][idx] = vzn;
            if ((lab_c & LAB_REC) && A.rec_kind != 0)
                record_cell(A, idx, A.rec_kind == 1 ? vxn : (A.rec_kind == 2 ? vyn : vzn));
        }
        lab_c = lab_z;
        lab_z = nlab_z;
        lab_x = nlab_x;
        lab_y = nlab_y;
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            r3[k] = r3[k + 1];
            r4[k] = r4[k + 1];
            r5[k] = r5[k + 1];
        }
        r3[7] = n3;
        r4[7] = n4;
        r5[7] = n5;
    }
    cp_async_wait<0>();
}

template <typename T>
__global__ void __launch_bounds__(TB_N, 1) k_velocity_t(const StepArgs<T> A, int n_mat)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *slots = reinterpret_cast<T *>(smem_raw);
    T *rsm = slots + (size_t)T_SLOTS * (V_ST + V_VC);
    const bool tab_smem = table_in_smem<T>(n_mat);
    if (tab_smem) {
        const int tid = threadIdx.y * TB_X + threadIdx.x;
        for (int i = tid; i < n_mat; i += TB_N) rsm[i] = A.rho[i];
    }
    const T *rho_tab = tab_smem ? rsm : A.rho;
    const int x0 = blockIdx.x * TB_X, y0 = blockIdx.y * TB_Y;
    const bool inner = x0 - T_H >= 0 && x0 + TB_X - 1 + T_H < A.nx && y0 - T_H >= 0 &&
                       y0 + TB_Y - 1 + T_H < A.ny;
    if (inner) velocity_tiled_run<T, false>(A, slots, rho_tab);
    else velocity_tiled_run<T, true>(A, slots, rho_tab);
}

}  // namespace pe
