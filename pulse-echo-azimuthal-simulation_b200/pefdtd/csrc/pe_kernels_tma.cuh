// TMA-fed step kernels (the default path on grids whose rows are 16-byte
// multiples).
//
// Same block geometry, arithmetic, term order and explicit FMA placement as
// pe_kernels_tiled.cuh; the difference is who moves the data. One elected
// thread per block issues, per plane, a handful of cp.async.bulk.tensor box
// loads (tile planes with their stencil halo, and the per-cell operands) into
// one of three shared-memory slots, each tracked by an mbarrier with the
// transaction byte count; the other threads only wait on that mbarrier. No
// per-thread address arithmetic is spent on staging. Every wait is bounded:
// a wait that exceeds its limit records PE_ERR_TIMEOUT in a device status
// word and the block carries on (its results are then discarded by the host),
// so no launch can hang.
//
// Box x-origins are multiples of 4 elements (16 bytes): the velocity tile
// starts at x0 - 4 with x0 a multiple of 32; the stress tiles start at the
// multiple of 4 at or below the first needed column and the threads index
// them with the block's offset from it.
#pragma once
#include <cuda.h>

#include "pe_kernels_tiled.cuh"

namespace pe {

constexpr unsigned long long MBAR_SPIN_LIMIT = 1ull << 22;  // try_wait polls before giving up
constexpr int STATUS_TIMEOUT = 5;

// tensor maps of one launch (passed by value as a grid constant)
struct alignas(64) TmapsStress {
    CUtensorMap vt[3];   // vx, vy, vz: box 44 x 24 x 1
    CUtensorMap sc[6];   // s1..s6: box 36 x 16 x 1
    CUtensorMap dv;      // damping volume (f32): box 36 x 16 x 1
};
struct alignas(64) TmapsVelocity {
    CUtensorMap st[5];   // s1, s2, s4, s5, s6: box 40 x 24 x 1
    CUtensorMap vc[3];   // vx, vy, vz: box 32 x 16 x 1
    CUtensorMap dv;      // damping volume (f32): box 32 x 16 x 1
};

constexpr int KS_VW = 44, KS_VH = 24, KS_VSZ = KS_VW * KS_VH;   // stress v tile
constexpr int KS_SW = 36, KS_SH = 16, KS_SSZ = KS_SW * KS_SH;   // stress s centres
constexpr int KV_SW = 40, KV_SH = 24, KV_SSZ = KV_SW * KV_SH;   // velocity s tile
constexpr int KV_CW = 32, KV_CH = 16, KV_CSZ = KV_CW * KV_CH;   // velocity centres

// slot sizes in elements of T (each box padded to 128 bytes)
template <typename T>
__host__ __device__ constexpr int pad128(int elems)
{
    return (int)(((size_t)elems * sizeof(T) + 127) / 128 * 128 / sizeof(T));
}
template <typename T>
__host__ __device__ constexpr int ks_slot_v() { return 3 * pad128<T>(KS_VSZ); }
template <typename T>
__host__ __device__ constexpr int ks_slot_s() { return 6 * pad128<T>(KS_SSZ) + pad128<T>(KS_SSZ); }
template <typename T>
__host__ __device__ constexpr int kv_slot() { return 5 * pad128<T>(KV_SSZ) + 4 * pad128<T>(KV_CSZ); }

template <typename T>
__host__ __device__ constexpr size_t stress_tma_smem(int n_mat)
{
    return 128 + sizeof(T) * (3 * (size_t)(ks_slot_v<T>() + ks_slot_s<T>()) + (size_t)3 * 6 * TB_N +
                              (table_in_smem<T>(n_mat) ? (size_t)n_mat * C21_STRIDE : 0));
}
template <typename T>
__host__ __device__ constexpr size_t velocity_tma_smem(int n_mat)
{
    return 128 + sizeof(T) * (3 * (size_t)kv_slot<T>() + (table_in_smem<T>(n_mat) ? (size_t)n_mat : 0));
}

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait; on timeout record the status and return false
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, int *status)
{
    for (unsigned long long it = 0; it < MBAR_SPIN_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (status) atomicExch(status, STATUS_TIMEOUT);
    return false;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

__device__ __forceinline__ int floor4(int x) { return x & ~3; }

// ---------------------------------------------------------------- strains (one column)
// NC: compile-time tap count (0 = runtime A.nc); ZIN: every z tap inside the grid;
// EDGE: x / y guards needed.
template <typename T, int NC, bool ZIN, bool EDGE>
__device__ __forceinline__ void strain_column(const StepArgs<T> &A, int q, const T *tvx, const T *tvy,
                                              const T *tvz, int W, const T rz[8], const T ry[8],
                                              const T rx[8], const bool xb[4], const bool xf[4],
                                              const bool yb[4], const bool yf[4], T g[6])
{
    T a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
    const int nz = A.nz;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (NC ? j < NC : j < A.nc) {
            const T cj = A.c[j];
            const bool zbj = ZIN || (q >= j + 1 && q < nz - j);
            const bool zfj = ZIN || (q >= j && q < nz - j - 1);
            if (!EDGE || xb[j]) a1 = fmac(a1, cj, tvx[j] - tvx[-(j + 1)]);
            if (!EDGE || yb[j]) a2 = fmac(a2, cj, tvy[j * W] - tvy[-(j + 1) * W]);
            if (zbj) a3 = fmac(a3, cj, rz[4 + j] - rz[3 - j]);
            if (!EDGE || yf[j]) a4 = fmac(a4, cj, tvz[(j + 1) * W] - tvz[-j * W]);
            if (zfj) a4 = fmac(a4, cj, ry[4 + j] - ry[3 - j]);
            if (!EDGE || xf[j]) a5 = fmac(a5, cj, tvz[j + 1] - tvz[-j]);
            if (zfj) a5 = fmac(a5, cj, rx[4 + j] - rx[3 - j]);
            if (!EDGE || xf[j]) a6 = fmac(a6, cj, tvy[j + 1] - tvy[-j]);
            if (!EDGE || yf[j]) a6 = fmac(a6, cj, tvx[(j + 1) * W] - tvx[-j * W]);
        }
    }
    const T ih = A.inv_h;
    g[0] = a1 * ih; g[1] = a2 * ih; g[2] = a3 * ih;
    g[3] = a4 * ih; g[4] = a5 * ih; g[5] = a6 * ih;
}

// ---------------------------------------------------------------- stress
template <typename T, int NC, bool EDGE>
__device__ __forceinline__ void stress_tma_run(const TmapsStress &M, const StepArgs<T> &A, T *vslots,
                                               T *sslots, T *gs, unsigned long long *bars,
                                               const T *tab, bool tab_smem, bool has_dvol,
                                               int bx, int by, int bz)
{
    constexpr int PV = pad128<T>(KS_VSZ), PS = pad128<T>(KS_SSZ);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TB_X + tx;
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long sy = A.sy, sz = A.sz;
    const int X0 = bx * TS_OX - 1, Y0 = by * TS_OY - 1;
    const int gx = X0 + tx, gy = Y0 + ty;
    const bool col_ok = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
    const int col = col_ok ? (int)(gy * sy + gx) : 0;
    const int zb = bz * A.zc;
    const int ze = min(zb + A.zc, nz);
    const long long n = *A.step + A.k;
    const T wn = A.n_src ? A.wavelet[n] : T(0);
    const int xv = floor4(X0 - T_H), xs = floor4(X0 + 1);   // box x-origins
    const int q0 = zb - 1;
    const bool leader = tid == 0;
    const unsigned bytes_v = 3u * KS_VSZ * sizeof(T);
    const unsigned bytes_s = 6u * KS_SSZ * sizeof(T) + (has_dvol ? KS_SSZ * 4u : 0u);

    // plane p = q0 + i of the v tiles shares a barrier with s centres of plane p - 1
    auto issue = [&](int i) {
        const int p = q0 + i;
        if (!leader || p > ze) return;
        const int slot = i % 3;
        unsigned long long *bar = bars + slot;
        const int ps = p - 1;
        const bool with_s = ps >= zb && ps < ze;
        fence_proxy_async();
        mbar_expect_tx(bar, bytes_v + (with_s ? bytes_s : 0u));
        T *dv = vslots + (size_t)slot * 3 * PV;
#pragma unroll
        for (int f = 0; f < 3; ++f) tma_load_3d(dv + f * PV, &M.vt[f], xv, Y0 - T_H, p, bar);
        if (with_s) {
            T *ds = sslots + (size_t)(((ps - zb) % 3 + 3) % 3) * 7 * PS;
#pragma unroll
            for (int f = 0; f < 6; ++f) tma_load_3d(ds + f * PS, &M.sc[f], xs, Y0, ps, bar);
            if (has_dvol) tma_load_3d(ds + 6 * PS, &M.dv, xs, Y0, ps, bar);
        }
    };
    // column loads for the z rings: running pointers, one plane ahead
    const T *pz = A.v[2] + col, *py = A.v[1] + col, *px = A.v[0] + col;
    auto ldcol = [&](const T *f, int q) -> T {
        return (col_ok && q >= 0 && q < nz) ? ldg(f + (long long)q * sz) : T(0);
    };
    T rz[8], ry[8], rx[8];   // rz[k] <-> plane q-4+k, ry/rx[k] <-> q-3+k
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        rz[k] = ldcol(pz, q0 - 4 + k);
        ry[k] = ldcol(py, q0 - 3 + k);
        rx[k] = ldcol(px, q0 - 3 + k);
    }
    bool xb[4], xf[4], yb[4], yf[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        xb[j] = gx >= j + 1 && gx < nx - j;
        xf[j] = gx >= j && gx < nx - j - 1;
        yb[j] = gy >= j + 1 && gy < ny - j;
        yf[j] = gy >= j && gy < ny - j - 1;
    }
    const bool xlo = !EDGE || gx >= 1, xhi = !EDGE || gx <= nx - 2;
    const bool ylo = !EDGE || gy >= 1, yhi = !EDGE || gy <= ny - 2;
    const bool is_out = tx >= 1 && tx <= TS_OX && ty >= 1 && ty <= TS_OY && gx < nx && gy < ny;
    float dyx = 1.0f, dxx = 1.0f;
    if (A.dz && is_out) { dyx = A.dy[gy]; dxx = A.dx[gx]; }
    const int tcv = (ty + T_H) * KS_VW + (gx - xv);   // this column in a v tile
    const int tcs = ty * KS_SW + (gx - xs);           // this cell in an s centre box
    uint16_t lab_next = (is_out && zb < nz) ? A.lab[(long long)zb * sz + col] : 0;
    int *status = A.status;

    issue(0);
    issue(1);
    const int n_it = ze - q0 + 1;
    for (int i = 0; i < n_it; ++i) {
        const int q = q0 + i;
        mbar_wait(bars + i % 3, (unsigned)(i / 3) & 1u, status);
        __syncthreads();   // also: every thread is done with the slot refilled below
        issue(i + 2);
        const T nzv = ldcol(pz, q + 4), nyv = ldcol(py, q + 5), nxv = ldcol(px, q + 5);
        const int z = q - 1;
        const uint16_t lab = lab_next;
        if (is_out && z >= zb && q < ze) lab_next = A.lab[(long long)q * sz + col];
        {
            const T *t = vslots + (size_t)(i % 3) * 3 * PV + tcv;
            T g[6];
            const bool zin = q >= T_H && q <= nz - 1 - T_H;
            if (zin) strain_column<T, NC, true, EDGE>(A, q, t, t + PV, t + 2 * PV, KS_VW, rz, ry, rx, xb, xf, yb, yf, g);
            else strain_column<T, NC, false, EDGE>(A, q, t, t + PV, t + 2 * PV, KS_VW, rz, ry, rx, xb, xf, yb, yf, g);
            T *gw = gs + (size_t)(i % 3) * 6 * TB_N + tid;
#pragma unroll
            for (int J = 0; J < 6; ++J) gw[J * TB_N] = g[J];
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
        if (z >= zb && is_out) {
            // strain planes z-1, z, z+1 were written at iterations i-2, i-1, i
            const T *gm = gs + (size_t)((i + 1) % 3) * 6 * TB_N + tid;
            const T *g0 = gs + (size_t)((i + 2) % 3) * 6 * TB_N + tid;
            const T *gp = gs + (size_t)(i % 3) * 6 * TB_N + tid;
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
            const T *sc = sslots + (size_t)((z - zb) % 3) * 7 * PS + tcs;
            T Cm[24];
            load_c21(tab + (size_t)(lab & LAB_MAT) * C21_STRIDE, tab_smem, Cm);
            float d = 1.0f;
            if (A.dz) {
                d = A.dz[z] * dyx;
                d = d * dxx;
            }
            if (has_dvol) {
                const float dvv = reinterpret_cast<const float *>(sslots + (size_t)((z - zb) % 3) * 7 * PS + 6 * PS)[tcs];
                d = A.dz ? d * dvv : dvv;
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
                const T s = sc[I * PS] * dmp;
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
}

// One block's share of a stress launch: tile (bx, by), z-chunk bz. The
// material table is (re)loaded into shared memory when load_table is set; the
// caller guarantees the block is between barriers (no copy in flight).
template <typename T>
__device__ __forceinline__ void stress_tma_block(const TmapsStress &M, const StepArgs<T> &A, int n_mat,
                                                 unsigned char *smem, int bx, int by, int bz,
                                                 bool load_table)
{
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem);
    T *vslots = reinterpret_cast<T *>(smem + 128);
    T *sslots = vslots + 3 * (size_t)ks_slot_v<T>();
    T *gs = sslots + 3 * (size_t)ks_slot_s<T>();
    T *tsm = gs + (size_t)3 * 6 * TB_N;
    const int tid = threadIdx.y * TB_X + threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < 3; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    const bool tab_smem = table_in_smem<T>(n_mat);
    if (tab_smem && load_table)
        for (int i = tid; i < n_mat * C21_STRIDE; i += TB_N) tsm[i] = A.c21[i];
    __syncthreads();
    const T *tab = tab_smem ? tsm : A.c21;
    const bool has_dvol = A.dvol != nullptr;
    const int X0 = bx * TS_OX - 1, Y0 = by * TS_OY - 1;
    const bool inner = X0 - T_H >= 0 && X0 + TB_X - 1 + T_H < A.nx && Y0 - T_H >= 0 &&
                       Y0 + TB_Y - 1 + T_H < A.ny;
    if (A.nc == 4) {
        if (inner) stress_tma_run<T, 4, false>(M, A, vslots, sslots, gs, bars, tab, tab_smem, has_dvol, bx, by, bz);
        else stress_tma_run<T, 4, true>(M, A, vslots, sslots, gs, bars, tab, tab_smem, has_dvol, bx, by, bz);
    } else {
        stress_tma_run<T, 0, true>(M, A, vslots, sslots, gs, bars, tab, tab_smem, has_dvol, bx, by, bz);
    }
}

template <typename T>
__global__ void __launch_bounds__(TB_N, 1) k_stress_tma(const __grid_constant__ TmapsStress M,
                                                        const StepArgs<T> A, int n_mat)
{
    extern __shared__ __align__(128) unsigned char smem_tma[];
    stress_tma_block<T>(M, A, n_mat, smem_tma, blockIdx.x, blockIdx.y, blockIdx.z, true);
}

// ---------------------------------------------------------------- velocity
template <typename T, int NC, bool ZIN, bool EDGE>
__device__ __forceinline__ void vel_taps(const StepArgs<T> &A, int z, const T *t1, const T *t2,
                                         const T *t4, const T *t5, const T *t6, const T r3[8],
                                         const T r4[8], const T r5[8], const bool xb[4],
                                         const bool xf[4], const bool yb[4], const bool yf[4],
                                         T &ax, T &ay, T &az)
{
    constexpr int W = KV_SW;
    const int nz = A.nz;
    ax = 0; ay = 0; az = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (NC ? j < NC : j < A.nc) {
            const T cj = A.c[j];
            if (!EDGE || xf[j]) ax = fmac(ax, cj, t1[j + 1] - t1[-j]);
            if (!EDGE || xb[j]) {
                ay = fmac(ay, cj, t6[j] - t6[-(j + 1)]);
                az = fmac(az, cj, t5[j] - t5[-(j + 1)]);
            }
            if (!EDGE || yf[j]) ay = fmac(ay, cj, t2[(j + 1) * W] - t2[-j * W]);
            if (!EDGE || yb[j]) {
                ax = fmac(ax, cj, t6[j * W] - t6[-(j + 1) * W]);
                az = fmac(az, cj, t4[j * W] - t4[-(j + 1) * W]);
            }
            if (ZIN || (z >= j && z < nz - j - 1)) az = fmac(az, cj, r3[4 + j] - r3[3 - j]);
            if (ZIN || (z >= j + 1 && z < nz - j)) {
                ax = fmac(ax, cj, r5[4 + j] - r5[3 - j]);
                ay = fmac(ay, cj, r4[4 + j] - r4[3 - j]);
            }
        }
    }
}

template <typename T, int NC, bool EDGE>
__device__ __forceinline__ void velocity_tma_run(const TmapsVelocity &M, const StepArgs<T> &A, T *slots,
                                                 unsigned long long *bars, const T *rho_tab,
                                                 bool has_dvol, int bx, int by, int bz)
{
    constexpr int PT = pad128<T>(KV_SSZ), PC = pad128<T>(KV_CSZ), SL = kv_slot<T>();
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TB_X + tx;
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long sy = A.sy, sz = A.sz;
    const int x0 = bx * TB_X, y0 = by * TB_Y;
    const int ix = x0 + tx, iy = y0 + ty;
    const bool out_ok = ix < nx && iy < ny;
    const int col = out_ok ? (int)(iy * sy + ix) : 0;
    const int zb = bz * A.zc;
    const int ze = min(zb + A.zc, nz);
    const bool leader = tid == 0;
    const unsigned bytes = 5u * KV_SSZ * sizeof(T) + 3u * KV_CSZ * sizeof(T) + (has_dvol ? KV_CSZ * 4u : 0u);

    auto issue = [&](int i) {
        const int z = zb + i;
        if (!leader || z >= ze) return;
        unsigned long long *bar = bars + i % 3;
        T *d = slots + (size_t)(i % 3) * SL;
        fence_proxy_async();
        mbar_expect_tx(bar, bytes);
#pragma unroll
        for (int f = 0; f < 5; ++f) tma_load_3d(d + f * PT, &M.st[f], x0 - T_H, y0 - T_H, z, bar);
#pragma unroll
        for (int c = 0; c < 3; ++c) tma_load_3d(d + 5 * PT + c * PC, &M.vc[c], x0, y0, z, bar);
        if (has_dvol) tma_load_3d(d + 5 * PT + 3 * PC, &M.dv, x0, y0, z, bar);
    };
    const T *p3 = A.s[2] + col, *p4 = A.s[3] + col, *p5 = A.s[4] + col;
    auto ldcol = [&](const T *f, int z) -> T {
        return (out_ok && z >= 0 && z < nz) ? ldg(f + (long long)z * sz) : T(0);
    };
    auto ldlab = [&](long long i, bool ok) -> uint16_t { return ok ? A.lab[i] : (uint16_t)0; };

    T r3[8], r4[8], r5[8];   // r3[k] <-> z-3+k, r4/r5[k] <-> z-4+k
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        r3[k] = ldcol(p3, zb - 3 + k);
        r4[k] = ldcol(p4, zb - 4 + k);
        r5[k] = ldcol(p5, zb - 4 + k);
    }
    bool xb[4], xf[4], yb[4], yf[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        xb[j] = ix >= j + 1 && ix < nx - j;
        xf[j] = ix >= j && ix < nx - j - 1;
        yb[j] = iy >= j + 1 && iy < ny - j;
        yf[j] = iy >= j && iy < ny - j - 1;
    }
    const bool xin = ix < nx - 1, yin = iy < ny - 1;
    float dyx = 1.0f, dxx = 1.0f;
    if (A.dz && out_ok) { dyx = A.dy[iy]; dxx = A.dx[ix]; }
    const int tc = (ty + T_H) * KV_SW + tx + T_H;
    const int cc = ty * KV_CW + tx;
    long long cz = (long long)zb * sz + col;
    uint16_t lab_c = ldlab(cz, out_ok && zb < nz);
    uint16_t lab_z = ldlab(cz + sz, out_ok && zb + 1 < nz);
    uint16_t lab_x = ldlab(cz + 1, out_ok && xin && zb < nz);
    uint16_t lab_y = ldlab(cz + sy, out_ok && yin && zb < nz);
    int *status = A.status;

    issue(0);
    issue(1);
    for (int i = 0; i < ze - zb; ++i) {
        const int z = zb + i;
        mbar_wait(bars + i % 3, (unsigned)(i / 3) & 1u, status);
        __syncthreads();
        issue(i + 2);
        const T n3 = ldcol(p3, z + 5), n4 = ldcol(p4, z + 4), n5 = ldcol(p5, z + 4);
        const long long cn = (long long)(z + 1) * sz + col;
        const uint16_t nlab_z = ldlab(cn + sz, out_ok && z + 2 < nz);
        const uint16_t nlab_x = ldlab(cn + 1, out_ok && xin && z + 1 < nz);
        const uint16_t nlab_y = ldlab(cn + sy, out_ok && yin && z + 1 < nz);
        const T *slot = slots + (size_t)(i % 3) * SL;
        const T *t = slot + tc;
        T ax, ay, az;
        const bool zin = z >= T_H && z <= nz - 1 - T_H;
        if (zin) vel_taps<T, NC, true, EDGE>(A, z, t, t + PT, t + 2 * PT, t + 3 * PT, t + 4 * PT, r3, r4, r5, xb, xf, yb, yf, ax, ay, az);
        else vel_taps<T, NC, false, EDGE>(A, z, t, t + PT, t + 2 * PT, t + 3 * PT, t + 4 * PT, r3, r4, r5, xb, xf, yb, yf, ax, ay, az);
        if (out_ok) {
            const T r0 = rho_tab[lab_c & LAB_MAT];
            const T rvx = xin ? T(0.5) * (r0 + rho_tab[lab_x & LAB_MAT]) : r0;
            const T rvy = yin ? T(0.5) * (r0 + rho_tab[lab_y & LAB_MAT]) : r0;
            const T rvz = (z < nz - 1) ? T(0.5) * (r0 + rho_tab[lab_z & LAB_MAT]) : r0;
            const T *vc = slot + 5 * PT + cc;
            float d = 1.0f;
            if (A.dz) {
                d = A.dz[z] * dyx;
                d = d * dxx;
            }
            if (has_dvol) {
                const float dvv = reinterpret_cast<const float *>(slot + 5 * PT + 3 * PC)[cc];
                d = A.dz ? d * dvv : dvv;
            }
            const T dmp = (T)d;
            T ux = A.dt_h * ax, uy = A.dt_h * ay, uz = A.dt_h * az;
            ux = div_face(ux, rvx);
            uy = div_face(uy, rvy);
            uz = div_face(uz, rvz);
            const T vxn = (vc[0] + ux) * dmp;
            const T vyn = (vc[PC] + uy) * dmp;
            const T vzn = (vc[2 * PC] + uz) * dmp;
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
}

template <typename T>
__device__ __forceinline__ void velocity_tma_block(const TmapsVelocity &M, const StepArgs<T> &A, int n_mat,
                                                   unsigned char *smem, int bx, int by, int bz,
                                                   bool load_table)
{
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem);
    T *slots = reinterpret_cast<T *>(smem + 128);
    T *rsm = slots + 3 * (size_t)kv_slot<T>();
    const int tid = threadIdx.y * TB_X + threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < 3; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    const bool tab_smem = table_in_smem<T>(n_mat);
    if (tab_smem && load_table)
        for (int i = tid; i < n_mat; i += TB_N) rsm[i] = A.rho[i];
    __syncthreads();
    const T *rho_tab = tab_smem ? rsm : A.rho;
    const bool has_dvol = A.dvol != nullptr;
    const int x0 = bx * TB_X, y0 = by * TB_Y;
    const bool inner = x0 - T_H >= 0 && x0 + TB_X - 1 + T_H < A.nx && y0 - T_H >= 0 &&
                       y0 + TB_Y - 1 + T_H < A.ny;
    if (A.nc == 4) {
        if (inner) velocity_tma_run<T, 4, false>(M, A, slots, bars, rho_tab, has_dvol, bx, by, bz);
        else velocity_tma_run<T, 4, true>(M, A, slots, bars, rho_tab, has_dvol, bx, by, bz);
    } else {
        velocity_tma_run<T, 0, true>(M, A, slots, bars, rho_tab, has_dvol, bx, by, bz);
    }
}

template <typename T>
__global__ void __launch_bounds__(TB_N, 1) k_velocity_tma(const __grid_constant__ TmapsVelocity M,
                                                          const StepArgs<T> A, int n_mat)
{
    extern __shared__ __align__(128) unsigned char smem_tma[];
    velocity_tma_block<T>(M, A, n_mat, smem_tma, blockIdx.x, blockIdx.y, blockIdx.z, true);
}

// ---------------------------------------------------------------- batches
// A batch of solves of any grid sizes advances one step per launch pair. Work
// items (solve, tile x, tile y, z-chunk) are listed solve by solve; each
// resident block walks a contiguous run of items, re-staging the solve's
// arguments and material table only when the solve changes.
struct BatchItem {
    int solve, bx, by, bz;
};

template <typename T>
__device__ __forceinline__ void copy_args(StepArgs<T> *dst, const StepArgs<T> *src, int k)
{
    const int tid = threadIdx.y * TB_X + threadIdx.x;
    const int nw = (int)(sizeof(StepArgs<T>) / 4);
    for (int i = tid; i < nw; i += TB_N)
        reinterpret_cast<int *>(dst)[i] = reinterpret_cast<const int *>(src)[i];
    __syncthreads();
    if (tid == 0) dst->k = k;
}

template <typename T>
__global__ void __launch_bounds__(TB_N, 1)
    k_stress_tma_batch(const StepArgs<T> *__restrict__ descs, const TmapsStress *__restrict__ maps,
                       const int *__restrict__ n_mats, const BatchItem *__restrict__ items, int n_items,
                       int k)
{
    extern __shared__ __align__(128) unsigned char smem_tma[];
    __shared__ __align__(16) StepArgs<T> As;
    const int per = (n_items + gridDim.x - 1) / gridDim.x;
    const int i0 = blockIdx.x * per, i1 = min(n_items, i0 + per);
    int cur = -1;
    for (int it = i0; it < i1; ++it) {
        const BatchItem w = items[it];
        __syncthreads();   // the previous item is finished by every thread
        const bool fresh = w.solve != cur;
        if (fresh) copy_args(&As, descs + w.solve, k);
        __syncthreads();
        stress_tma_block<T>(maps[w.solve], As, n_mats[w.solve], smem_tma, w.bx, w.by, w.bz, fresh);
        cur = w.solve;
    }
}

template <typename T>
__global__ void __launch_bounds__(TB_N, 1)
    k_velocity_tma_batch(const StepArgs<T> *__restrict__ descs, const TmapsVelocity *__restrict__ maps,
                         const int *__restrict__ n_mats, const BatchItem *__restrict__ items, int n_items,
                         int k)
{
    extern __shared__ __align__(128) unsigned char smem_tma[];
    __shared__ __align__(16) StepArgs<T> As;
    const int per = (n_items + gridDim.x - 1) / gridDim.x;
    const int i0 = blockIdx.x * per, i1 = min(n_items, i0 + per);
    int cur = -1;
    for (int it = i0; it < i1; ++it) {
        const BatchItem w = items[it];
        __syncthreads();
        const bool fresh = w.solve != cur;
        if (fresh) copy_args(&As, descs + w.solve, k);
        __syncthreads();
        velocity_tma_block<T>(maps[w.solve], As, n_mats[w.solve], smem_tma, w.bx, w.by, w.bz, fresh);
        cur = w.solve;
    }
}

}  // namespace pe
