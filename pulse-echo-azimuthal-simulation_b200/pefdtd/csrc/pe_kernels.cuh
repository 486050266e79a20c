// Label-indexed anisotropic elastic staggered-grid FDTD step kernels for
// sm_100a (B200).
//
// One time step is two launches:
//   k_stress    strains of v (9 staggered derivatives) computed into a
//               rolling 3-plane shared-memory ring while the block marches z,
//               half-cell moves out of that ring, the 6x6 label-indexed
//               stiffness product, deferred damping, source injection and
//               (for pressure) receiver sampling.  Replaces the reference's
//               strains_zp + stress_lab_u + source scatter
//               (sim/core/fdtd.py:1102-1177, :594-689, :1798-1800).
//   k_velocity  the velocity update with in-kernel face density from the
//               label-indexed density table, damping and (for vx/vy/vz)
//               receiver sampling.  Replaces vel_zp and the receiver gather
//               (sim/core/fdtd.py:1179-1257, :1806-1813).
//
// Arithmetic contract: every expression keeps the reference's term order
// (j-ascending taps, per-component interleaving, z-major move taps,
// J-ascending stiffness rows, deferred damping) and the file is compiled
// with -fmad=false, so the only fused multiply-adds are the explicit fmac()
// calls. The CPU oracle (oracle/fdtd_oracle_impl.h, fma_mode 1) places the
// same FMAs, which makes these kernels bit-exact against it.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pe {

constexpr uint16_t LAB_SRC = 0x8000;  // cell receives the source
constexpr uint16_t LAB_REC = 0x4000;  // cell is sampled by a receiver
constexpr uint16_t LAB_MAT = 0x3FFF;  // material index bits

constexpr int C21_STRIDE = 24;        // table row: 21 constants + pad

__device__ __forceinline__ float fmac(float a, float b, float c) { return __fmaf_rn(b, c, a); }
__device__ __forceinline__ double fmac(double a, double b, double c) { return __fma_rn(b, c, a); }

template <typename T>
struct StepArgs {
    T *v[3];
    T *s[6];
    const uint16_t *lab;     // material | flags
    const T *c21;            // (n_mat, C21_STRIDE)
    const T *rho;            // (n_mat,)
    const float *rinv;       // (n_mat,) RN32(1 / rho) (FP32 solves), or null
    const float *dz, *dy, *dx;  // sponge tapers or null
    const float *dvol;          // damping volume or null
    int nz, ny, nx;
    long long sy, sz;
    T c[4];
    int nc;
    T inv_h, dt, dt_h;
    // source
    const long long *src_idx;  // sorted, unique
    const T *src_w;
    int n_src;
    const T *wavelet;
    // receivers
    const long long *rec_cell;  // sorted cell of each entry
    const int *rec_pos;         // entry position in caller order
    int n_rec;
    T *rec_val;                 // (chunk, n_rec) sampled values of this chunk
    int rec_kind;               // 0 pressure, 1 vx, 2 vy, 3 vz
    int rec_damped;
    // time
    const long long *step;      // device: global index of chunk step 0
    int k;                      // step within the chunk
    int zc;                     // planes per z-march
    int *status;                // device status word (bounded waits record timeouts)
    int dense;                  // per-cell media: the table row of cell i is i (untiled kernels)
};

// ---------------------------------------------------------------- helpers
template <typename T>
__device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// a / b for b > 0 (a face density), rounded as the plain division: a zero
// numerator returns itself (+0 / b = +0, -0 / b = -0) without dividing.
// Before the wavefront arrives most of the grid is zero, and profiling shows
// zero numerators otherwise taking the division's slow path.
template <typename T>
__device__ __forceinline__ T div_face(T a, T b)
{
    T q = a;
    if (a != T(0)) {
        asm volatile("" ::: "memory");   // keeps the division inside the branch
        q = a / b;
    }
    return q;
}

__device__ __forceinline__ int lower_bound_ll(const long long *a, int n, long long key)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

template <typename T>
__device__ __forceinline__ float damp_at(const StepArgs<T> &A, int iz, int iy, int ix,
                                         long long idx)
{
    float d = 1.0f;
    if (A.dz) {
        d = A.dz[iz] * A.dy[iy];
        d = d * A.dx[ix];
    }
    if (A.dvol) d = A.dz ? d * A.dvol[idx] : A.dvol[idx];
    return d;
}

// upper-triangle slot of (I, J) in a row of 21
__host__ __device__ constexpr int c21_slot(int I, int J)
{
    return I <= J ? (I * (13 - I)) / 2 + (J - I) : (J * (13 - J)) / 2 + (I - J);
}

// staggered position offsets (z, y, x) of position p: c, yz, xz, xy
__host__ __device__ constexpr int pos_z(int p) { return (p == 1 || p == 2) ? 1 : 0; }
__host__ __device__ constexpr int pos_y(int p) { return (p == 1 || p == 3) ? 1 : 0; }
__host__ __device__ constexpr int pos_x(int p) { return (p == 2 || p == 3) ? 1 : 0; }
// position of strain / stress component J: g1..g3 at c, g4 yz, g5 xz, g6 xy
__host__ __device__ constexpr int vpos(int J) { return J < 3 ? 0 : J - 2; }

// ---------------------------------------------------------------- strains
// Nine staggered derivatives of v at one cell, term order of
// sim/core/fdtd.py:1141-1162; loads go through the read-only cache.
template <typename T>
__device__ __forceinline__ void strains_cell(const StepArgs<T> &A, int iz, int iy, int ix,
                                             T g[6])
{
    const long long sy = A.sy, sz = A.sz;
    const long long idx = iz * sz + iy * sy + ix;
    const T *vx = A.v[0], *vy = A.v[1], *vz = A.v[2];
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    T a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (j < A.nc) {
            const T cj = A.c[j];
            if (ix >= j + 1 && ix < nx - j)
                a1 = fmac(a1, cj, ldg(vx + idx + j) - ldg(vx + idx - (j + 1)));
            if (iy >= j + 1 && iy < ny - j)
                a2 = fmac(a2, cj, ldg(vy + idx + j * sy) - ldg(vy + idx - (j + 1) * sy));
            if (iz >= j + 1 && iz < nz - j)
                a3 = fmac(a3, cj, ldg(vz + idx + j * sz) - ldg(vz + idx - (j + 1) * sz));
            if (iy >= j && iy < ny - j - 1)
                a4 = fmac(a4, cj, ldg(vz + idx + (j + 1) * sy) - ldg(vz + idx - j * sy));
            if (iz >= j && iz < nz - j - 1)
                a4 = fmac(a4, cj, ldg(vy + idx + (j + 1) * sz) - ldg(vy + idx - j * sz));
            if (ix >= j && ix < nx - j - 1)
                a5 = fmac(a5, cj, ldg(vz + idx + (j + 1)) - ldg(vz + idx - j));
            if (iz >= j && iz < nz - j - 1)
                a5 = fmac(a5, cj, ldg(vx + idx + (j + 1) * sz) - ldg(vx + idx - j * sz));
            if (ix >= j && ix < nx - j - 1)
                a6 = fmac(a6, cj, ldg(vy + idx + (j + 1)) - ldg(vy + idx - j));
            if (iy >= j && iy < ny - j - 1)
                a6 = fmac(a6, cj, ldg(vx + idx + (j + 1) * sy) - ldg(vx + idx - j * sy));
        }
    }
    const T ih = A.inv_h;
    g[0] = a1 * ih; g[1] = a2 * ih; g[2] = a3 * ih;
    g[3] = a4 * ih; g[4] = a5 * ih; g[5] = a6 * ih;
}

// ---------------------------------------------------------------- moves
// Strain J moved to position P (sim/core/fdtd.py:612-633): 4 taps over the
// two axes whose half-cell offsets differ, summed z-major, times 1/4; zero
// where a needed neighbour is off the grid. G(J, dz, dy, dx) reads the ring.
template <int P, int J, typename T, typename GF>
__device__ __forceinline__ T qval(const GF &G, bool zlo, bool zhi, bool ylo, bool yhi, bool xlo,
                                  bool xhi)
{
    constexpr int S = vpos(J);
    constexpr int DZ = pos_z(P) - pos_z(S), DY = pos_y(P) - pos_y(S), DX = pos_x(P) - pos_x(S);
    if constexpr (DZ == 0 && DY == 0 && DX == 0) {
        return G(J, 0, 0, 0);
    } else {
        bool ok = true;
        if constexpr (DZ > 0) ok = ok && zhi;
        if constexpr (DZ < 0) ok = ok && zlo;
        if constexpr (DY > 0) ok = ok && yhi;
        if constexpr (DY < 0) ok = ok && ylo;
        if constexpr (DX > 0) ok = ok && xhi;
        if constexpr (DX < 0) ok = ok && xlo;
        constexpr int LZ = DZ < 0 ? -1 : 0, HZ = DZ > 0 ? 1 : 0;
        constexpr int LY = DY < 0 ? -1 : 0, HY = DY > 0 ? 1 : 0;
        constexpr int LX = DX < 0 ? -1 : 0, HX = DX > 0 ? 1 : 0;
        T acc = 0;
        bool first = true;
#pragma unroll
        for (int a0 = LZ; a0 <= HZ; ++a0)
#pragma unroll
            for (int a1 = LY; a1 <= HY; ++a1)
#pragma unroll
                for (int a2 = LX; a2 <= HX; ++a2) {
                    const T t = G(J, a0, a1, a2);
                    acc = first ? t : acc + t;
                    first = false;
                }
        return ok ? acc * T(0.25) : T(0);
    }
}

template <int P, typename T, typename GF>
__device__ __forceinline__ void qrow(const GF &G, bool zlo, bool zhi, bool ylo, bool yhi,
                                     bool xlo, bool xhi, T q[6])
{
    q[0] = qval<P, 0, T>(G, zlo, zhi, ylo, yhi, xlo, xhi);
    q[1] = qval<P, 1, T>(G, zlo, zhi, ylo, yhi, xlo, xhi);
    q[2] = qval<P, 2, T>(G, zlo, zhi, ylo, yhi, xlo, xhi);
    q[3] = qval<P, 3, T>(G, zlo, zhi, ylo, yhi, xlo, xhi);
    q[4] = qval<P, 4, T>(G, zlo, zhi, ylo, yhi, xlo, xhi);
    q[5] = qval<P, 5, T>(G, zlo, zhi, ylo, yhi, xlo, xhi);
}

template <typename T>
__device__ __forceinline__ T row_dot(const T *Cr, int I, const T q[6])
{
    T acc = 0;
#pragma unroll
    for (int J = 0; J < 6; ++J) acc = fmac(acc, Cr[c21_slot(I, J)], q[J]);
    return acc;
}

// ---------------------------------------------------------------- receivers
template <typename T>
__device__ __forceinline__ void record_cell(const StepArgs<T> &A, long long idx, T val)
{
    int e = lower_bound_ll(A.rec_cell, A.n_rec, idx);
    T *out = A.rec_val + (long long)A.k * A.n_rec;
    for (; e < A.n_rec && A.rec_cell[e] == idx; ++e) out[A.rec_pos[e]] = val;
}

// ---------------------------------------------------------------- stress
template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX *TY) k_stress(const StepArgs<T> A)
{
    constexpr int GX = TX + 2, GY = TY + 2, NG = GX * GY;
    __shared__ T gsm[3][6][NG];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * A.zc;
    const int ze = min(zb + A.zc, A.nz);
    const long long n = *A.step + A.k;
    const T wn = A.n_src ? A.wavelet[n] : T(0);

    auto gplane = [&](int q) {
        const int slot = (q + 3) % 3;
        for (int t = tid; t < NG; t += TX * TY) {
            const int lx = t % GX, ly = t / GX;
            const int ix = x0 - 1 + lx, iy = y0 - 1 + ly;
            T g[6] = {0, 0, 0, 0, 0, 0};
            if (q >= 0 && q < A.nz && ix >= 0 && ix < A.nx && iy >= 0 && iy < A.ny)
                strains_cell(A, q, iy, ix, g);
#pragma unroll
            for (int J = 0; J < 6; ++J) gsm[slot][J][t] = g[J];
        }
    };

    gplane(zb - 1);
    gplane(zb);
    const int ix = x0 + tx, iy = y0 + ty;
    const int lc = (ty + 1) * GX + (tx + 1);
    for (int z = zb; z < ze; ++z) {
        gplane(z + 1);
        __syncthreads();
        if (ix < A.nx && iy < A.ny) {
            const int sm = (z + 2) % 3, s0 = z % 3, sp = (z + 1) % 3;
            auto G = [&](int J, int dz, int dy, int dx) -> T {
                const int slot = dz < 0 ? sm : (dz > 0 ? sp : s0);
                return gsm[slot][J][lc + dy * GX + dx];
            };
            const bool zlo = z >= 1, zhi = z <= A.nz - 2;
            const bool ylo = iy >= 1, yhi = iy <= A.ny - 2;
            const bool xlo = ix >= 1, xhi = ix <= A.nx - 2;
            T q0[6], q1[6], q2[6], q3[6];
            qrow<0>(G, zlo, zhi, ylo, yhi, xlo, xhi, q0);
            qrow<1>(G, zlo, zhi, ylo, yhi, xlo, xhi, q1);
            qrow<2>(G, zlo, zhi, ylo, yhi, xlo, xhi, q2);
            qrow<3>(G, zlo, zhi, ylo, yhi, xlo, xhi, q3);

            const long long idx = z * A.sz + iy * A.sy + ix;
            const uint16_t lab = A.lab[idx];
            const T *Cr = A.c21 + (A.dense ? idx : (long long)(lab & LAB_MAT)) * C21_STRIDE;
            T Cm[21];
#pragma unroll
            for (int k = 0; k < 21; ++k) Cm[k] = ldg(Cr + k);
            const T dmp = (T)damp_at(A, z, iy, ix, idx);
            T acc[6];
            acc[0] = row_dot(Cm, 0, q0);
            acc[1] = row_dot(Cm, 1, q0);
            acc[2] = row_dot(Cm, 2, q0);
            acc[3] = row_dot(Cm, 3, q1);
            acc[4] = row_dot(Cm, 4, q2);
            acc[5] = row_dot(Cm, 5, q3);
            T sv[6];
#pragma unroll
            for (int I = 0; I < 6; ++I) {
                const T s = A.s[I][idx] * dmp;
                sv[I] = fmac(s, A.dt, acc[I]);
            }
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
        __syncthreads();
    }
}

// ---------------------------------------------------------------- velocity
template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX *TY) k_velocity(const StepArgs<T> A)
{
    const int ix = blockIdx.x * TX + threadIdx.x;
    const int iy = blockIdx.y * TY + threadIdx.y;
    if (ix >= A.nx || iy >= A.ny) return;
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const int zb = blockIdx.z * A.zc;
    const int ze = min(zb + A.zc, nz);
    const long long sy = A.sy, sz = A.sz;
    const long long base = iy * sy + ix;
    const T *s1 = A.s[0], *s2 = A.s[1], *s3 = A.s[2], *s4 = A.s[3], *s5 = A.s[4], *s6 = A.s[5];

    // z-rings of the three fields with z taps: slot k holds plane iz - 4 + k
    T r3[9], r4[9], r5[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int z = zb - 4 + k;
        const bool ok = z >= 0 && z < nz;
        const long long p = base + z * sz;
        r3[k] = ok ? ldg(s3 + p) : T(0);
        r4[k] = ok ? ldg(s4 + p) : T(0);
        r5[k] = ok ? ldg(s5 + p) : T(0);
    }
    for (int iz = zb; iz < ze; ++iz) {
        const long long idx = base + iz * sz;
        T ax = 0, ay = 0, az = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (j < A.nc) {
                const T cj = A.c[j];
                if (ix >= j && ix < nx - j - 1)
                    ax = fmac(ax, cj, ldg(s1 + idx + (j + 1)) - ldg(s1 + idx - j));
                if (ix >= j + 1 && ix < nx - j) {
                    ay = fmac(ay, cj, ldg(s6 + idx + j) - ldg(s6 + idx - (j + 1)));
                    az = fmac(az, cj, ldg(s5 + idx + j) - ldg(s5 + idx - (j + 1)));
                }
                if (iy >= j && iy < ny - j - 1)
                    ay = fmac(ay, cj, ldg(s2 + idx + (j + 1) * sy) - ldg(s2 + idx - j * sy));
                if (iy >= j + 1 && iy < ny - j) {
                    ax = fmac(ax, cj, ldg(s6 + idx + j * sy) - ldg(s6 + idx - (j + 1) * sy));
                    az = fmac(az, cj, ldg(s4 + idx + j * sy) - ldg(s4 + idx - (j + 1) * sy));
                }
                if (iz >= j && iz < nz - j - 1) az = fmac(az, cj, r3[5 + j] - r3[4 - j]);
                if (iz >= j + 1 && iz < nz - j) {
                    ax = fmac(ax, cj, r5[4 + j] - r5[3 - j]);
                    ay = fmac(ay, cj, r4[4 + j] - r4[3 - j]);
                }
            }
        }
        const uint16_t lab = A.lab[idx];
        // density of a cell: its table row (the cell itself for per-cell media)
        auto rho_at = [&](long long q) -> T {
            return ldg(A.rho + (A.dense ? q : (long long)(A.lab[q] & LAB_MAT)));
        };
        const T r0 = rho_at(idx);
        const T rvx = (ix < nx - 1) ? T(0.5) * (r0 + rho_at(idx + 1)) : r0;
        const T rvy = (iy < ny - 1) ? T(0.5) * (r0 + rho_at(idx + sy)) : r0;
        const T rvz = (iz < nz - 1) ? T(0.5) * (r0 + rho_at(idx + sz)) : r0;
        const T dmp = (T)damp_at(A, iz, iy, ix, idx);
        T tx = A.dt_h * ax, ty = A.dt_h * ay, tz = A.dt_h * az;
        tx = div_face(tx, rvx); ty = div_face(ty, rvy); tz = div_face(tz, rvz);
        const T vx = (A.v[0][idx] + tx) * dmp;
        const T vy = (A.v[1][idx] + ty) * dmp;
        const T vz = (A.v[2][idx] + tz) * dmp;
        A.v[0][idx] = vx;
        A.v[1][idx] = vy;
        A.v[2][idx] = vz;
        if ((lab & LAB_REC) && A.rec_kind != 0)
            record_cell(A, idx, A.rec_kind == 1 ? vx : (A.rec_kind == 2 ? vy : vz));
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            r3[k] = r3[k + 1];
            r4[k] = r4[k + 1];
            r5[k] = r5[k + 1];
        }
        const int zn = iz + 5;
        const bool ok = zn < nz;
        const long long p = base + zn * sz;
        r3[8] = ok ? ldg(s3 + p) : T(0);
        r4[8] = ok ? ldg(s4 + p) : T(0);
        r5[8] = ok ? ldg(s5 + p) : T(0);
    }
}

// ---------------------------------------------------------------- chunk epilogue
// trace[n][g] = sum over the group's entries, in caller order, of val * w,
// for the chunk's steps; then the step counter advances by the chunk length.
template <typename T>
__global__ void k_reduce_traces(const T *rec_val, const T *rec_w, const long long *grp_off,
                                int n_groups, int n_rec, int n_steps, const long long *step,
                                T *traces)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_steps * n_groups) return;
    const int k = t / n_groups, g = t % n_groups;
    const T *val = rec_val + (long long)k * n_rec;
    T acc = 0;
    for (long long e = grp_off[g]; e < grp_off[g + 1]; ++e) {
        const T prod = val[e] * rec_w[e];
        acc = acc + prod;
    }
    traces[(*step + k) * n_groups + g] = acc;
}

__global__ void k_step_set(long long *step, long long value) { *step = value; }
__global__ void k_step_advance(long long *step, long long by) { *step += by; }

// ---------------------------------------------------------------- setup kernels
// copy material indices into the solver's flagged label volume, counting any
// index >= n_mat
__global__ void k_labels_copy(const uint16_t *in, uint16_t *out, long long n, int n_mat,
                              unsigned long long *n_bad)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint16_t m = in[i];
    if (m >= n_mat) atomicAdd(n_bad, 1ULL);
    out[i] = m < n_mat ? m : 0;
}

__global__ void k_labels_flag(uint16_t *lab, const long long *cells, int n, uint16_t flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) lab[cells[i]] = lab[cells[i]] | flag;
}

template <typename T>
__global__ void k_c36_to_c21(const T *c36, T *c21, int n_mat)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_mat) return;
    for (int I = 0; I < 6; ++I)
        for (int J = I; J < 6; ++J) c21[m * C21_STRIDE + c21_slot(I, J)] = c36[m * 36 + I * 6 + J];
    for (int k = 21; k < C21_STRIDE; ++k) c21[m * C21_STRIDE + k] = T(0);
}

}  // namespace pe
