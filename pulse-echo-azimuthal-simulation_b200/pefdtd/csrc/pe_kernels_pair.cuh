// Pair-column FP32 step kernels (the default FP32 path on grids whose rows
// are 16-byte multiples).
//
// Arithmetic, term order and explicit FMA placement are those of the
// one-column kernels (pe_kernels_tma.cuh, pe_kernels.cuh), so the results are
// bit-identical to them and to the oracle. What changes is the number of
// instructions spent per operand, which is what bounds the one-column
// kernels: every thread owns two x-adjacent cells, so
//  - each stencil tap read from shared memory is one 64-bit load serving
//    both cells, and the x taps of a row (10 values) are five such loads;
//  - the half-cell moves read strain rows as 64-bit pairs (42 loads per pair
//    of cells instead of 156 scalar loads);
//  - the stiffness product runs column by column (J outer), reading column J
//    of a material from a (n_mat, 36) table (shared memory when two blocks'
//    copies fit, else through L1) with one 128-bit and one 64-bit load per
//    cell, which keeps the register footprint within 128 registers;
//  - tiles whose every tap lies inside the grid run an unguarded body; the
//    others zero the coefficients of skipped taps instead of branching.
// Data movement is the TMA scheme of the one-column kernels: one elected
// thread issues cp.async.bulk.tensor box loads two planes ahead into three
// mbarrier-tracked slots; z taps come from per-thread register rings.
// Every mbarrier wait is bounded (status word, no hang).
//
// Blocks: 256 threads = 16 lanes along x (two columns each) x 16 rows, two
// blocks per SM, so that one block's barrier and memory waits overlap the
// other's work.
//   k_stress_pair    strain tile 32 x 16 columns, the inner 30 x 14 are
//                    updated; replaces strains_zp + stress_lab_u + the source
//                    scatter (sim/core/fdtd.py:1102-1177, :594-689,
//                    :1798-1800).
//   k_velocity_pair  32 x 16 cells; replaces vel_zp and the receiver gather
//                    (sim/core/fdtd.py:1179-1257, :1806-1813).
#pragma once
#include "pe_kernels_tma.cuh"

namespace pe {

constexpr int PR_LX = 16;                                         // lanes along x, two columns each
// stress: two 256-thread blocks per SM (16 rows of strain columns)
constexpr int PS_ROWS = 16, PS_N = PR_LX * PS_ROWS;
constexpr int PS_OX = 30, PS_OY = PS_ROWS - 2;                    // updated cells per block
constexpr int PS_VW = 44, PS_VH = PS_ROWS + 8, PS_VSZ = PS_VW * PS_VH;   // v box: 1056 floats (4224 B)
constexpr int PS_SW = 36, PS_SH = PS_OY, PS_SSZ = PS_SW * PS_SH;  // cell box: 504 floats
constexpr int PS_SSZP = 512;                                      // ... padded to 128 B
constexpr int PS_GW = 32, PS_GOFF = 8, PS_GST = 2 * PS_GOFF + PS_GW * PS_ROWS;   // strain plane: pad, 32 x 16, pad
constexpr int PS_VSLOT = 3 * PS_VSZ;
constexpr int PS_SSLOT = 6 * PS_SSZP;
// Strain ring: the update of plane z reads g4 and g5 at planes z - 1 and z,
// the other four components at z and z + 1 (the half-cell moves,
// sim/core/fdtd.py:612-633). While it runs, the strains of plane z + 2 are
// written; with four planes for g4, g5 and three for the others they never
// overwrite what the update reads, so one block barrier per plane suffices.
__host__ __device__ constexpr int ring_planes(int J) { return (J == 3 || J == 4) ? 4 : 3; }
__host__ __device__ constexpr int ring_base(int J)   // first plane of component J, in planes
{
    return J < 3 ? 3 * J : (J == 5 ? 9 : (J == 3 ? 12 : 16));
}
constexpr int PS_RING = 20;   // strain planes held
// shared memory of a stress block: mbarriers (v, cell slot 0, cell slot 1),
// one v slot, two cell slots, the strain ring, then the material table
constexpr size_t PS_SMEM_FIXED = 128 + sizeof(float) * ((size_t)PS_VSLOT + 2 * (size_t)PS_SSLOT + (size_t)PS_RING * PS_GST);
constexpr int TAB36 = 36;   // material: columns J as [C0J..C3J] at 4J, then [C4J, C5J] at 24 + 2J
// velocity
// two velocity blocks of 256 threads share an SM, so that one block's
// barrier waits overlap the other's work
constexpr int PV_ROWS = 16, PV_N = PR_LX * PV_ROWS;
constexpr int PV_OX = 32, PV_OY = PV_ROWS;
constexpr int PV_TW = 40, PV_TH = PV_OY + 8, PV_TSZ = PV_TW * PV_TH;   // s box with halo: 3840 B
constexpr int PV_CSZ = PV_OX * PV_OY;                             // cell box: 4096 B
constexpr int PV_SLOT = 5 * PV_TSZ + 4 * PV_CSZ;

struct alignas(64) TmapsPairStress {
    CUtensorMap vt[3];   // vx, vy, vz: box 44 x 40
    CUtensorMap sc[6];   // s1..s6: box 36 x 30
    CUtensorMap dv;      // damping volume: box 36 x 30
};
struct alignas(64) TmapsPairVelocity {
    CUtensorMap st[5];   // s1, s2, s4, s5, s6: box 40 x 40
    CUtensorMap vc[3];   // vx, vy, vz: box 32 x 32
    CUtensorMap dv;      // damping volume: box 32 x 32
};

// the table goes to shared memory when two blocks with it still fit an
// SM's 228 KB (1 KB of each block's share is reserved), else it is read
// through L1
__host__ __device__ constexpr bool pair_tab_in_smem(int n_mat)
{
    return 2 * (PS_SMEM_FIXED + (size_t)n_mat * TAB36 * sizeof(float) + 1024) <= 233472;
}
__host__ __device__ constexpr size_t stress_pair_smem(int n_mat)
{
    return PS_SMEM_FIXED + (pair_tab_in_smem(n_mat) ? (size_t)n_mat * TAB36 * sizeof(float) : 0);
}
__host__ __device__ constexpr bool pair_rho_in_smem(int n_mat) { return n_mat <= 8192; }
__host__ __device__ constexpr size_t velocity_pair_smem(int n_mat)
{
    return 128 + sizeof(float) * (3 * (size_t)PV_SLOT + (pair_rho_in_smem(n_mat) ? (size_t)n_mat : 0));
}

__device__ __forceinline__ float2 lds2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float2 ldg2(const float *p) { return __ldg(reinterpret_cast<const float2 *>(p)); }
__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void stg2(float *p, float a, float b)
{
    *reinterpret_cast<float2 *>(p) = make_float2(a, b);
}
__device__ __forceinline__ float pick(float2 v, int c) { return c ? v.y : v.x; }
// Paired FP32 arithmetic (sm_100: one FADD2 / FMUL2 / FFMA2 instruction does
// the operation on both lanes of a 64-bit register pair, each lane rounded to
// nearest exactly as the scalar instruction). A thread's two cells share the
// y and z offsets of every tap, so their y / z taps, the half-cell moves
// without an x component and the update expressions run as one paired
// instruction per operation; per lane the operations, their order and the
// fused multiply-adds are those of the scalar code, so results are unchanged
// bit for bit.
__device__ __forceinline__ unsigned long long u64_of(float2 v)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
    return r;
}
__device__ __forceinline__ float2 f2_of(unsigned long long r)
{
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(u64_of(a)), "l"(u64_of(b)));
    return f2_of(r);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(u64_of(a)), "l"(u64_of(b)));
    return f2_of(r);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(u64_of(a)), "l"(u64_of(b)));
    return f2_of(r);
}
// fmac2(a, b, c) = b * c + a per lane, one rounding (fmac's argument order)
__device__ __forceinline__ float2 fmac2(float2 a, float2 b, float2 c)
{
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(u64_of(b)), "l"(u64_of(c)), "l"(u64_of(a)));
    return f2_of(r);
}

// streaming column loads for the z rings: read once, kept out of L1 so that
// L1 holds the material table
__device__ __forceinline__ float2 ldg2_stream(const float *p)
{
    float2 v;
    asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}
// the same column loads where other blocks of the same launch write the
// field (the persistent batch kernel): cached in L2 only, the point where
// the grid barrier makes other blocks' writes visible
__device__ __forceinline__ float2 ldcg2(const float *p)
{
    float2 v;
    asm volatile("ld.global.cg.v2.f32 {%0, %1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "l"(p) : "memory");
    return v;
}
template <bool COH>
__device__ __forceinline__ float2 ld2_column(const float *p)
{
    if constexpr (COH) return ldcg2(p);
    else return ldg2_stream(p);
}

// ======================================================================== stress
// Tap limits near the grid faces. The reference skips a tap whose reach
// leaves the grid (sim/core/fdtd.py:1141-1162, :1215-1236): tap j of a
// backward difference along x at column x exists iff j < min(x, nx - x), of
// a forward difference iff j < min(x + 1, nx - x - 1). The guarded bodies
// multiply instead of branching: a skipped tap gets the coefficient 0, and
// fma(0, d, a) == a bit for bit for finite d, because an accumulator that
// starts at +0 is never -0.
struct TapLimits {
    int xb[2], xf[2], yb, yf;
};
__device__ __forceinline__ int lim_b(int i, int n) { return min(i, n - i); }
__device__ __forceinline__ int lim_f(int i, int n) { return min(i + 1, n - i - 1); }
template <bool G>
__device__ __forceinline__ float tapc(float cj, int j, int lim) { return (!G || j < lim) ? cj : 0.0f; }

// strain of both columns at plane q; cv = this thread's cell 0 in the vx box;
// the z rings hold both columns' values as lane pairs
template <int NC, bool G>
__device__ __forceinline__ void pair_strain(const StepArgs<float> &A, int q, const float *cv,
                                            const float2 (&rz)[8], const float2 (&ry)[8],
                                            const float2 (&rx)[8], const TapLimits &tl,
                                            float2 (&g)[6])
{
    constexpr int W = PS_VW;
    const float *tvx = cv, *tvy = cv + PS_VSZ, *tvz = cv + 2 * PS_VSZ;
    float X[10], Y[10], Z[10];   // centre rows, columns (cell 0) - 4 .. + 5
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const float2 a = lds2(tvx + 2 * k - 4), b = lds2(tvy + 2 * k - 4), c = lds2(tvz + 2 * k - 4);
        X[2 * k] = a.x; X[2 * k + 1] = a.y;
        Y[2 * k] = b.x; Y[2 * k + 1] = b.y;
        Z[2 * k] = c.x; Z[2 * k + 1] = c.y;
    }
    float2 a1 = bc2(0.f), a2 = bc2(0.f), a3 = bc2(0.f), a4 = bc2(0.f), a5 = bc2(0.f), a6 = bc2(0.f);
    const int nz = A.nz;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (NC ? j < NC : j < A.nc) {
            const float cj = A.c[j];
            const float czb = tapc<G>(cj, j, lim_b(q, nz)), czf = tapc<G>(cj, j, lim_f(q, nz));
            const float cyb = tapc<G>(cj, j, tl.yb), cyf = tapc<G>(cj, j, tl.yf);
            const float cxb0 = tapc<G>(cj, j, tl.xb[0]), cxb1 = tapc<G>(cj, j, tl.xb[1]);
            const float cxf0 = tapc<G>(cj, j, tl.xf[0]), cxf1 = tapc<G>(cj, j, tl.xf[1]);
            const float2 yp = lds2(tvy + j * W), ym = lds2(tvy - (j + 1) * W);     // Dby vy
            const float2 zp = lds2(tvz + (j + 1) * W), zm = lds2(tvz - j * W);     // Dfy vz
            const float2 xp = lds2(tvx + (j + 1) * W), xm = lds2(tvx - j * W);     // Dfy vx
            // per lane: a1 x; a2 y; a3 z; a4 y, z; a5 x, z; a6 x, y. The x
            // taps' differences are per lane (their operands straddle the
            // lanes' 64-bit pairs), their fused multiply-adds paired
            const float2 cxb = make_float2(cxb0, cxb1), cxf = make_float2(cxf0, cxf1);
            a1 = fmac2(a1, cxb, make_float2(X[4 + j] - X[3 - j], X[5 + j] - X[4 - j]));
            a2 = fmac2(a2, bc2(cyb), sub2(yp, ym));
            a3 = fmac2(a3, bc2(czb), sub2(rz[4 + j], rz[3 - j]));
            a4 = fmac2(a4, bc2(cyf), sub2(zp, zm));
            a4 = fmac2(a4, bc2(czf), sub2(ry[4 + j], ry[3 - j]));
            a5 = fmac2(a5, cxf, make_float2(Z[5 + j] - Z[4 - j], Z[6 + j] - Z[5 - j]));
            a5 = fmac2(a5, bc2(czf), sub2(rx[4 + j], rx[3 - j]));
            a6 = fmac2(a6, cxf, make_float2(Y[5 + j] - Y[4 - j], Y[6 + j] - Y[5 - j]));
            a6 = fmac2(a6, bc2(cyf), sub2(xp, xm));
        }
    }
    const float2 ih = bc2(A.inv_h);
    g[0] = mul2(a1, ih); g[1] = mul2(a2, ih); g[2] = mul2(a3, ih);
    g[3] = mul2(a4, ih); g[4] = mul2(a5, ih); g[5] = mul2(a6, ih);
}

// strain J at (dz, dy) and column offset dx in -1..2 from cell 0. pl[0]:
// the 4-plane ring slot of plane z - 1, pl[1] of z (both at this thread's
// cell 0, component offsets added here); pl[2]: the 3-plane ring slot of
// z, pl[3] of z + 1.
// address of the lane pair (cell 0, cell 1) of strain J at (dz, dy), column
// offset 0
__device__ __forceinline__ const float *gptr(const float *const (&pl)[4], int J, int dz, int dy)
{
    const float *b = (J == 3 || J == 4) ? pl[dz + 1] : pl[dz + 2];
    return b + ring_base(J) * PS_GST + dy * PS_GW;
}
__device__ __forceinline__ float gval(const float *const (&pl)[4], int J, int dz, int dy, int dx)
{
    const float *b = (J == 3 || J == 4) ? pl[dz + 1] : pl[dz + 2];
    const float *p = b + ring_base(J) * PS_GST + dy * PS_GW + (dx & ~1);
    const float2 v = lds2(p);
    return (dx & 1) ? v.y : v.x;
}

struct MoveGuards {
    bool zlo, zhi, ylo, yhi, xlo[2], xhi[2];
};

// strain J moved to position P (sim/core/fdtd.py:612-633) for both cells:
// 4 taps summed z-major, times 1/4, zero where a needed neighbour is off
// the grid; the term order of qval() in pe_kernels.cuh. A move without an x
// component reads the same column offsets for both cells (one 64-bit load
// per tap, paired sums); the others combine lanes per cell.
template <int P, int J, bool G>
__device__ __forceinline__ void qpair(const float *const (&pl)[4], const MoveGuards &mg, float2 &q)
{
    constexpr int S = vpos(J);
    constexpr int DZ = pos_z(P) - pos_z(S), DY = pos_y(P) - pos_y(S), DX = pos_x(P) - pos_x(S);
    constexpr int LZ = DZ < 0 ? -1 : 0, HZ = DZ > 0 ? 1 : 0;
    constexpr int LY = DY < 0 ? -1 : 0, HY = DY > 0 ? 1 : 0;
    if constexpr (DZ == 0 && DY == 0 && DX == 0) {
        q = lds2(gptr(pl, J, 0, 0));
    } else if constexpr (DX == 0) {
        float2 acc = bc2(0.f);
        bool first = true;
#pragma unroll
        for (int a0 = LZ; a0 <= HZ; ++a0)
#pragma unroll
            for (int a1 = LY; a1 <= HY; ++a1) {
                const float2 t = lds2(gptr(pl, J, a0, a1));
                acc = first ? t : add2(acc, t);
                first = false;
            }
        bool ok = true;
        if constexpr (G) {
            if constexpr (DZ > 0) ok = ok && mg.zhi;
            if constexpr (DZ < 0) ok = ok && mg.zlo;
            if constexpr (DY > 0) ok = ok && mg.yhi;
            if constexpr (DY < 0) ok = ok && mg.ylo;
        }
        q = ok ? mul2(acc, bc2(0.25f)) : bc2(0.0f);
    } else {
        constexpr int LX = DX < 0 ? -1 : 0, HX = DX > 0 ? 1 : 0;
        float r[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            float acc = 0.f;
            bool first = true;
#pragma unroll
            for (int a0 = LZ; a0 <= HZ; ++a0)
#pragma unroll
                for (int a1 = LY; a1 <= HY; ++a1)
#pragma unroll
                    for (int a2 = LX; a2 <= HX; ++a2) {
                        const float t = gval(pl, J, a0, a1, c + a2);
                        acc = first ? t : acc + t;
                        first = false;
                    }
            if constexpr (G) {
                bool ok = true;
                if constexpr (DZ > 0) ok = ok && mg.zhi;
                if constexpr (DZ < 0) ok = ok && mg.zlo;
                if constexpr (DY > 0) ok = ok && mg.yhi;
                if constexpr (DY < 0) ok = ok && mg.ylo;
                if constexpr (DX > 0) ok = ok && mg.xhi[c];
                if constexpr (DX < 0) ok = ok && mg.xlo[c];
                r[c] = ok ? acc * 0.25f : 0.0f;
            } else {
                r[c] = acc * 0.25f;
            }
        }
        q = make_float2(r[0], r[1]);
    }
}

// column J of the stiffness product: acc[I] = fmac(acc[I], C[I][J], q_J at
// the position of stress I), J ascending as in row_dot(). TS: the table is
// in shared memory (else global, through the read-only cache). The two cells
// hold different materials, so these run per lane.
template <int J, bool G, bool TS>
__device__ __forceinline__ void stiff_column(const float *const (&pl)[4], const MoveGuards &mg,
                                             const float *const (&crow)[2], float2 (&acc)[6])
{
    float2 q0, q1, q2, q3;
    qpair<0, J, G>(pl, mg, q0);
    qpair<1, J, G>(pl, mg, q1);
    qpair<2, J, G>(pl, mg, q2);
    qpair<3, J, G>(pl, mg, q3);
    {
        const float4 a = TS ? lds4(crow[0] + 4 * J) : ldg4(crow[0] + 4 * J);
        const float2 b = TS ? lds2(crow[0] + 24 + 2 * J) : ldg2(crow[0] + 24 + 2 * J);
        acc[0].x = fmac(acc[0].x, a.x, q0.x);
        acc[1].x = fmac(acc[1].x, a.y, q0.x);
        acc[2].x = fmac(acc[2].x, a.z, q0.x);
        acc[3].x = fmac(acc[3].x, a.w, q1.x);
        acc[4].x = fmac(acc[4].x, b.x, q2.x);
        acc[5].x = fmac(acc[5].x, b.y, q3.x);
    }
    {
        const float4 a = TS ? lds4(crow[1] + 4 * J) : ldg4(crow[1] + 4 * J);
        const float2 b = TS ? lds2(crow[1] + 24 + 2 * J) : ldg2(crow[1] + 24 + 2 * J);
        acc[0].y = fmac(acc[0].y, a.x, q0.y);
        acc[1].y = fmac(acc[1].y, a.y, q0.y);
        acc[2].y = fmac(acc[2].y, a.z, q0.y);
        acc[3].y = fmac(acc[3].y, a.w, q1.y);
        acc[4].y = fmac(acc[4].y, b.x, q2.y);
        acc[5].y = fmac(acc[5].y, b.y, q3.y);
    }
}

template <bool G, bool TS>
__device__ __forceinline__ void stiff_all(const float *const (&pl)[4], const MoveGuards &mg,
                                          const float *const (&crow)[2], float2 (&acc)[6])
{
#pragma unroll
    for (int I = 0; I < 6; ++I) acc[I] = bc2(0.f);
    stiff_column<0, G, TS>(pl, mg, crow, acc);
    stiff_column<1, G, TS>(pl, mg, crow, acc);
    stiff_column<2, G, TS>(pl, mg, crow, acc);
    stiff_column<3, G, TS>(pl, mg, crow, acc);
    stiff_column<4, G, TS>(pl, mg, crow, acc);
    stiff_column<5, G, TS>(pl, mg, crow, acc);
}

// mbarrier phase counters of a block, carried across its marches
struct PairPhases {
    int v, s;   // v loads / cell-box loads issued (and waited) so far
};

// Row of the strain tile a stress thread computes. Warps 0..6 take rows
// 1..14 (the updated rows), two each; warp 7 takes the halo rows 0 and 15,
// whose strains are only read by neighbours, so it skips the update phase
// as a whole instead of leaving half of two warps idle there.
static_assert(PS_N == 256 && PS_ROWS == 16, "pair_row assumes 8 warps of two 16-lane rows");
__device__ __forceinline__ int pair_row(int tid)
{
    const int w = tid >> 5, h = (tid >> 4) & 1;
    return w < 7 ? 2 * w + 1 + h : (h ? PS_ROWS - 1 : 0);
}

// Every x / y tap of strain tile (bx, by) lies inside the grid (then no x or
// y guard can bind: every tap limit is at least T_H and every neighbour
// exists).
__device__ __forceinline__ bool pair_tile_inside(const StepArgs<float> &A, int bx, int by)
{
    const int S0 = bx * PS_OX - 2, S0y = by * PS_OY - 1;
    return S0 - T_H >= 0 && S0 + PS_GW - 1 + T_H < A.nx && S0y - T_H >= 0 && S0y + PS_ROWS - 1 + T_H < A.ny;
}

// One z-march of a block over strain tile (bx, by), updating planes
// [zb, ze). tab: the (n_mat, 36) table (shared memory when TS). Pipeline per
// iteration (strain plane q, update plane z = q - 1):
//   wait v(q) | strains of q | (warp 7: wait cell boxes of z) | block
//   barrier | issue v(q + 1) and the cell boxes of z + 1 | updates of plane z
// Every warp waits on the v mbarrier itself; warp 7 (halo rows, nothing to
// update) alone waits for the cell boxes. One v slot suffices (its refill
// overlaps the update phase); the cell boxes alternate between two slots and
// are issued a plane ahead. The caller synchronises the block before a march
// that follows another. TIN: pair_tile_inside(A, bx, by) holds, and the
// x / y limits and guards are compile-time constants.
template <int NC, bool TS, bool TIN, bool COH = false>
__device__ __forceinline__ void stress_pair_march(const TmapsPairStress &M, const StepArgs<float> &A,
                                                  const float *tab, unsigned char *smem, int bx, int by,
                                                  int zb, int ze, PairPhases &ph)
{
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem);
    float *vslot = reinterpret_cast<float *>(smem + 128);
    float *sslots = vslot + PS_VSLOT;
    float *gs = sslots + 2 * PS_SSLOT;
    const int tid = threadIdx.x;
    (void)tab;
    const int l = tid & (PR_LX - 1), r = pair_row(tid);
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long sy = A.sy, sz = A.sz;
    const int S0 = bx * PS_OX - 2, S0y = by * PS_OY - 1;   // first strain column / row (S0 even)
    const int gx0 = S0 + 2 * l, gy = S0y + r;
    const bool pair_ok = TIN || (gx0 >= 0 && gx0 < nx && gy >= 0 && gy < ny);   // nx even: both columns
    const int col = pair_ok ? (int)(gy * sy + gx0) : 0;
    const long long n = *A.step + A.k;
    const float wn = A.n_src ? A.wavelet[n] : 0.f;
    const int xv = floor4(S0 - T_H), xs = floor4(S0);    // box x-origins (16-byte multiples)
    const int q0 = zb - 1;
    const bool has_dvol = A.dvol != nullptr;
    const unsigned bytes_s = 6u * PS_SSZ * 4u;
    const unsigned bytes_v = 3u * PS_VSZ * 4u;
    const int v0 = ph.v, s0 = ph.s;   // phase counts at the start of this march

    auto issue_v = [&](int q) {   // v boxes of plane q (q0 <= q <= ze)
        fence_proxy_async();
        mbar_expect_tx(bars, bytes_v);
#pragma unroll
        for (int f = 0; f < 3; ++f) tma_load_3d(vslot + f * PS_VSZ, &M.vt[f], xv, S0y - T_H, q, bars);
    };
    auto issue_s = [&](int z) {   // cell boxes of plane z (zb <= z < ze)
        const int k = (s0 + z - zb) & 1;
        unsigned long long *bar = bars + 1 + k;
        float *ds = sslots + k * PS_SSLOT;
        fence_proxy_async();
        mbar_expect_tx(bar, bytes_s);
#pragma unroll
        for (int f = 0; f < 6; ++f) tma_load_3d(ds + f * PS_SSZP, &M.sc[f], xs, S0y + 1, z, bar);
    };

    // z rings (rz[c][k] <-> plane q-4+k, ry/rx[c][k] <-> q-3+k), one plane ahead
    const float *pz = A.v[2] + col, *py = A.v[1] + col, *px = A.v[0] + col;
    auto ld2col = [&](const float *f, int q) -> float2 {
        return (pair_ok && q >= 0 && q < nz) ? ld2_column<COH>(f + (long long)q * sz) : make_float2(0.f, 0.f);
    };
    float2 rz[8], ry[8], rx[8];   // lane pairs (cell 0, cell 1)
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        rz[k] = ld2col(pz, q0 - 4 + k);
        ry[k] = ld2col(py, q0 - 3 + k);
        rx[k] = ld2col(px, q0 - 3 + k);
    }
    TapLimits tl;
    MoveGuards mg;
    if constexpr (TIN) {
        tl.xb[0] = tl.xb[1] = tl.xf[0] = tl.xf[1] = tl.yb = tl.yf = T_H;
        mg.xlo[0] = mg.xlo[1] = mg.xhi[0] = mg.xhi[1] = mg.ylo = mg.yhi = true;
    } else {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int x = gx0 + c;
            tl.xb[c] = lim_b(x, nx);
            tl.xf[c] = lim_f(x, nx);
            mg.xlo[c] = x >= 1;
            mg.xhi[c] = x <= nx - 2;
        }
        tl.yb = lim_b(gy, ny);
        tl.yf = lim_f(gy, ny);
        mg.ylo = gy >= 1;
        mg.yhi = gy <= ny - 2;
    }
    // updated cells: inner 30 x 14 of the strain tile, inside the grid
    const bool row_out = r >= 1 && r <= PS_OY && (TIN || gy < ny);
    bool out_c[2];
    out_c[0] = row_out && l >= 1 && (TIN || (gx0 >= 0 && gx0 < nx));
    out_c[1] = row_out && l <= PR_LX - 2 && (TIN || (gx0 + 1 >= 0 && gx0 + 1 < nx));
    const bool any_out = out_c[0] || out_c[1];
    float dyx = 1.0f, dxx[2] = {1.0f, 1.0f};
    if (A.dz && any_out) {
        dyx = A.dy[gy];
        dxx[0] = A.dx[gx0];
        dxx[1] = A.dx[gx0 + 1];
    }
    // a warp's two rows both past the last grid row: no strain of theirs is
    // read by an updated cell, so the warp skips the strain work (warp-uniform;
    // the lower of the warp's rows is pair_row of its first thread)
    const bool warp_rows_in = TIN || S0y + pair_row(tid & ~31) < ny;
    const int cv = (r + T_H) * PS_VW + (S0 - xv) + 2 * l;   // cell 0 in a v box (even)
    const int cs = (r - 1) * PS_SW + (S0 - xs) + 2 * l;     // cell 0 in a cell box (even)
    const int cg = PS_GOFF + r * PS_GW + 2 * l;              // cell 0 in a strain plane
    const uint32_t *lab32 = reinterpret_cast<const uint32_t *>(A.lab);
    auto ldlab = [&](int z) -> uint32_t {
        return (any_out && z >= zb && z < ze) ? __ldg(lab32 + (((long long)z * sz + col) >> 1)) : 0u;
    };
    uint32_t lab_next = 0u;
    int *status = A.status;

    if (tid == 0) {
        issue_v(q0);
        issue_s(zb);
        if (zb + 1 < ze) issue_s(zb + 1);
    }
    const int n_it = ze - q0 + 1;
    int r3 = (q0 + 3) % 3;   // plane q modulo 3 (q >= -1), kept by increment
    for (int i = 0; i < n_it; ++i) {
        const int q = q0 + i;
        mbar_wait(bars, (unsigned)(v0 + i) & 1u, status);   // v(q) landed
        const float2 nzv = ld2col(pz, q + 4), nyv = ld2col(py, q + 5), nxv = ld2col(px, q + 5);
        const int z = q - 1;
        const uint32_t lab2 = lab_next;
        lab_next = ldlab(q);
        const bool fast = NC == 4 && TIN && q >= T_H && q <= nz - 1 - T_H;
        if (warp_rows_in) {
            const float *tv = vslot + cv;
            float2 g[6];
            if (fast) pair_strain<NC, false>(A, q, tv, rz, ry, rx, tl, g);
            else pair_strain<NC, true>(A, q, tv, rz, ry, rx, tl, g);
            const int s4 = q & 3;   // ring slots of plane q: r3 and q mod 4
#pragma unroll
            for (int J = 0; J < 6; ++J)
                *reinterpret_cast<float2 *>(gs + (ring_base(J) + (ring_planes(J) == 4 ? s4 : r3)) * PS_GST + cg) = g[J];
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
        // the cell boxes of plane z (issued a plane earlier): warp 7, which
        // has no cell to update, waits for them before the block barrier,
        // and the barrier orders every other warp's reads after that wait
        const int us = s0 + z - zb;   // cell-box load index of plane z
        if ((tid >> 5) == 7 && z >= zb) mbar_wait(bars + 1 + (us & 1), (unsigned)(us >> 1) & 1u, status);
        __syncthreads();   // strains of q written; the v slot is free; the updates of z - 1 are done
        if (tid == 7 * 32) {   // warp 7: idle while the others update
            if (q + 1 <= ze) issue_v(q + 1);
            if (q >= zb + 2 && q < ze) issue_s(q);   // plane z + 1, into the slot plane z - 1 used
        }
        if (z >= zb && any_out) {
            // strain planes z - 1, z, z + 1 were written at iterations i - 2, i - 1, i
            const int zr3 = r3 == 0 ? 2 : r3 - 1;   // plane z modulo 3
            const float *const pl[4] = {gs + ((z - 1) & 3) * PS_GST + cg, gs + (z & 3) * PS_GST + cg,
                                        gs + zr3 * PS_GST + cg, gs + r3 * PS_GST + cg};
            mg.zlo = z >= 1;
            mg.zhi = z <= nz - 2;
            const uint16_t lab[2] = {(uint16_t)(lab2 & 0xFFFFu), (uint16_t)(lab2 >> 16)};
            const float *const crow[2] = {tab + (lab[0] & LAB_MAT) * TAB36, tab + (lab[1] & LAB_MAT) * TAB36};
            float2 acc[6];
            if (fast) stiff_all<false, TS>(pl, mg, crow, acc);
            else stiff_all<true, TS>(pl, mg, crow, acc);
            const float *sc = sslots + (us & 1) * PS_SSLOT + cs;
            float dmp[2];
            {
                const float dz = A.dz ? A.dz[z] : 1.0f;
                float2 dvv = make_float2(1.0f, 1.0f);
                if (has_dvol) dvv = ldg2(A.dvol + (long long)z * sz + col);
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    float d = 1.0f;
                    if (A.dz) {
                        d = dz * dyx;
                        d = d * dxx[c];
                    }
                    if (has_dvol) d = A.dz ? d * pick(dvv, c) : pick(dvv, c);
                    dmp[c] = d;
                }
            }
            // s = fmac(s_old * damp, dt, acc) per lane
            const float2 dmp2 = make_float2(dmp[0], dmp[1]), dt2 = bc2(A.dt);
            float sv[6][2];
#pragma unroll
            for (int I = 0; I < 6; ++I) {
                const float2 v = fmac2(mul2(lds2(sc + I * PS_SSZP), dmp2), dt2, acc[I]);
                sv[I][0] = v.x;
                sv[I][1] = v.y;
            }
            const long long idx0 = (long long)z * sz + col;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                if (out_c[c] && (lab[c] & LAB_SRC)) {
                    const long long idx = idx0 + c;
                    const int e = lower_bound_ll(A.src_idx, A.n_src, idx);
                    if (e < A.n_src && A.src_idx[e] == idx) {
                        const float add = wn * A.src_w[e];
                        sv[0][c] = sv[0][c] + add;
                        sv[1][c] = sv[1][c] + add;
                        sv[2][c] = sv[2][c] + add;
                    }
                }
            }
            if (out_c[0] && out_c[1]) {
#pragma unroll
                for (int I = 0; I < 6; ++I) stg2(A.s[I] + idx0, sv[I][0], sv[I][1]);
            } else {
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    if (out_c[c]) {
#pragma unroll
                        for (int I = 0; I < 6; ++I) A.s[I][idx0 + c] = sv[I][c];
                    }
            }
            if (A.rec_kind == 0) {
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    if (out_c[c] && (lab[c] & LAB_REC)) {
                        float a = sv[0][c], b = sv[1][c], e = sv[2][c];
                        if (A.rec_damped) { a = a * dmp[c]; b = b * dmp[c]; e = e * dmp[c]; }
                        float t = a + b;
                        t = t + e;
                        record_cell(A, idx0 + c, -t / 3.0f);
                    }
                }
            }
        }
        r3 = r3 == 2 ? 0 : r3 + 1;
    }
    ph.v = v0 + n_it;
    ph.s = s0 + (ze - zb);
}

// Stage the (n_mat, 36) table into shared memory (16-byte copies).
__device__ __forceinline__ void stage_table(float *dst, const float *src, int n_mat)
{
    const float4 *s4 = reinterpret_cast<const float4 *>(src);
    float4 *d4 = reinterpret_cast<float4 *>(dst);
    for (int i = threadIdx.x; i < n_mat * (TAB36 / 4); i += blockDim.x) d4[i] = __ldg(s4 + i);
}

// zero the strain planes' pads (read only by cells that are not updated)
__device__ __forceinline__ void stress_pair_zero_pads(unsigned char *smem)
{
    float *gs = reinterpret_cast<float *>(smem + 128) + PS_VSLOT + 2 * PS_SSLOT;
    for (int i = threadIdx.x; i < PS_RING * 2 * PS_GOFF; i += blockDim.x) {
        const int p = i / (2 * PS_GOFF), k = i % (2 * PS_GOFF);
        gs[p * PS_GST + (k < PS_GOFF ? k : PS_GST - 2 * PS_GOFF + k)] = 0.f;
    }
}

__device__ __forceinline__ void stress_pair_init(unsigned char *smem)
{
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem);
    float *gs = reinterpret_cast<float *>(smem + 128) + PS_VSLOT + 2 * PS_SSLOT;
    if (threadIdx.x == 0) {
        for (int s = 0; s < 3; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    // zero the strain planes' pads (read only by cells that are not updated)
    for (int i = threadIdx.x; i < PS_RING * 2 * PS_GOFF; i += blockDim.x) {
        const int p = i / (2 * PS_GOFF), k = i % (2 * PS_GOFF);
        gs[p * PS_GST + (k < PS_GOFF ? k : PS_GST - 2 * PS_GOFF + k)] = 0.f;
    }
}

// Tile k (k < tx * ty) of a launch whose interior tiles (those whose every
// tap lies inside the grid) are bx in [1, bxh], by in [1, byh]: interior
// tiles first (row-major), then the others (row-major). Blocks resident on
// an SM together then mostly run the same instantiation of the march, which
// keeps the instruction cache warm (3.7 % faster for the stress kernel on
// disk_prod than row-major order). A bijection of [0, tx * ty).
__device__ __forceinline__ void interior_first(int bxh, int byh, int tx, int ty, int k, int &bx, int &by)
{
    int nix = min(tx - 1, bxh), niy = min(ty - 1, byh);
    if (nix <= 0 || niy <= 0) nix = niy = 0;
    const int ni = nix * niy;
    if (k < ni) {
        bx = 1 + k % nix;
        by = 1 + k / nix;
        return;
    }
    int e = k - ni;
    if (ni == 0 || e < tx) {
        bx = e % tx;
        by = e / tx;
        return;
    }
    e -= tx;
    const int w = tx - nix, mid = niy * w;
    if (e < mid) {
        const int c = e % w;
        bx = c < 1 ? c : c + nix;
        by = 1 + e / w;
        return;
    }
    e -= mid;
    bx = e % tx;
    by = 1 + niy + e / tx;
}
// last interior stress tile along x / y (pair_tile_inside), or <= 0
__host__ __device__ constexpr int pair_last_inside_x(int nx) { return nx < 34 ? 0 : (nx - 34) / PS_OX; }
__host__ __device__ constexpr int pair_last_inside_y(int ny) { return ny < 19 ? 0 : (ny - 19) / PS_OY; }

// Launch grid: (tiles x, tiles y, z-chunks of A.zc planes). Blocks that run
// at the same time march the same planes of neighbouring tiles, so the tile
// halos they share are read from DRAM once and from L2 after that.
template <int NC, bool TS>
__global__ void __launch_bounds__(PS_N, 2) k_stress_pair(const __grid_constant__ TmapsPairStress M,
                                                         const StepArgs<float> A,
                                                         const float *__restrict__ tab36, int n_mat)
{
    extern __shared__ __align__(128) unsigned char smem_pair[];
    float *tsm = reinterpret_cast<float *>(smem_pair + PS_SMEM_FIXED);
    stress_pair_init(smem_pair);
    if (TS) stage_table(tsm, tab36, n_mat);
    __syncthreads();
    const int zb = blockIdx.z * A.zc, ze = min(zb + A.zc, A.nz);
    PairPhases ph{0, 0};
    int bx, by;
    interior_first(pair_last_inside_x(A.nx), pair_last_inside_y(A.ny), gridDim.x, gridDim.y,
                   blockIdx.x + gridDim.x * blockIdx.y, bx, by);
    if (pair_tile_inside(A, bx, by))
        stress_pair_march<NC, TS, true>(M, A, TS ? tsm : tab36, smem_pair, bx, by, zb, ze, ph);
    else
        stress_pair_march<NC, TS, false>(M, A, TS ? tsm : tab36, smem_pair, bx, by, zb, ze, ph);
}

// ====================================================================== velocity
// a / b in float32 with IEEE round-to-nearest, for a face density b > 0 (the
// reference divides, sim/core/fdtd.py:1237-1244). The float32 division's
// slow path for tiny numerators (which fill a shell ahead of the wavefront)
// otherwise costs a third of the velocity kernel. When b is the cell's own
// density, y = RN32(1 / b) is at hand and Markstein's theorem gives the
// correctly rounded quotient: with y within half an ulp of 1 / b and q1
// within one ulp of a / b, r = a - b q1 is exact (one FMA) and RN(q1 + r y)
// is RN(a / b), while nothing underflows (2^-100 <= |a| <= 2^100 here).
// q1 comes from one correction of q0 = RN(a y) (which alone is only within
// two ulps): q1 = RN(q0 + (a - b q0) y) is within half an ulp plus 2^-47
// relative. Smaller numerators are scaled by 2^64 first (exact), and the
// scaled quotient scaled back, which is exact while the result is a normal
// float32 (|scaled quotient| >= 2^-62; the subnormal grid continues the
// lowest binade's spacing, so the boundary itself is safe). A subnormal
// result is |a| 2^149 / b rounded to an integer (ties to even) in units of
// 2^-149: A = |a| 2^149 is an integer below 2^49, a candidate n comes from
// the correctly rounded A / b, and the exact remainder A - b n (one FMA:
// it is a multiple of ulp(b) below 2 b) moves n by at most one. Mixed-density
// faces and non-finite or huge numerators divide in float64 and round once
// more, which is exact (53 >= 2 * 24 + 2 bits, Figueroa's theorem; a
// subnormal midpoint survives the float64 quotient unchanged). Zero
// numerators return themselves (the sign of zero kept).
__device__ __forceinline__ float markstein(float a, float b, float y)
{
    const float q0 = a * y;
    const float q1 = fmaf(fmaf(-b, q0, a), y, q0);
    return fmaf(fmaf(-b, q1, a), y, q1);
}
// 0 < |a| < 2^-100, y = RN32(1 / b)
__device__ __forceinline__ float div_face_tiny(float a, float b, float y)
{
    const float qs = markstein(a * 0x1p64f, b, y);
    if (fabsf(qs) >= 0x1p-62f) return qs * 0x1p-64f;
    const float A = fabsf(a) * 0x1p100f * 0x1p49f;
    float n = markstein(A, b, y);          // below 2^23 + 1: the result is subnormal
    n = (n + 0x1p23f) - 0x1p23f;           // nearest integer, ties to even
    const float R = fmaf(-b, n, A), hb = 0.5f * b;
    const bool odd = (__float2int_rz(n) & 1) != 0;
    if (R > hb || (R == hb && odd)) n += 1.0f;
    else if (R < -hb || (R == -hb && odd)) n -= 1.0f;
    return copysignf(n * 0x1p-100f * 0x1p-49f, a);
}
__device__ __forceinline__ float div_face_rcp(float a, float b, bool own, float y)
{
    const float aa = fabsf(a);
    if (own && aa >= 0x1p-100f && aa <= 0x1p100f) return markstein(a, b, y);
    if (a == 0.0f) return a;
    if (own && aa < 0x1p-100f) return div_face_tiny(a, b, y);
    return (float)((double)a / (double)b);
}

// reciprocal densities RN32(1 / rho), correctly rounded (IEEE division)
__global__ void k_rho_inv(const float *rho, float *rinv, int n_mat)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < n_mat) rinv[m] = 1.0f / rho[m];
}

template <int NC, bool G>
__device__ __forceinline__ void pair_vel_taps(const StepArgs<float> &A, int z, const float *t1,
                                              const float *t2, const float *t4, const float *t5,
                                              const float *t6, const float2 (&r3)[8],
                                              const float2 (&r4)[8], const float2 (&r5)[8],
                                              const TapLimits &tl, float2 &ax, float2 &ay,
                                              float2 &az)
{
    constexpr int W = PV_TW;
    float S1[10], S5[10], S6[10];   // centre rows, columns (cell 0) - 4 .. + 5
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const float2 a = lds2(t1 + 2 * k - 4), b = lds2(t5 + 2 * k - 4), c = lds2(t6 + 2 * k - 4);
        S1[2 * k] = a.x; S1[2 * k + 1] = a.y;
        S5[2 * k] = b.x; S5[2 * k + 1] = b.y;
        S6[2 * k] = c.x; S6[2 * k + 1] = c.y;
    }
    const int nz = A.nz;
    ax = ay = az = bc2(0.f);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (NC ? j < NC : j < A.nc) {
            const float cj = A.c[j];
            const float2 p2 = lds2(t2 + (j + 1) * W), m2 = lds2(t2 - j * W);         // Dfy s2
            const float2 p6 = lds2(t6 + j * W), m6 = lds2(t6 - (j + 1) * W);         // Dby s6
            const float2 p4 = lds2(t4 + j * W), m4 = lds2(t4 - (j + 1) * W);         // Dby s4
            const float czf = tapc<G>(cj, j, lim_f(z, nz)), czb = tapc<G>(cj, j, lim_b(z, nz));
            const float cyf = tapc<G>(cj, j, tl.yf), cyb = tapc<G>(cj, j, tl.yb);
            const float cxb0 = tapc<G>(cj, j, tl.xb[0]), cxb1 = tapc<G>(cj, j, tl.xb[1]);
            const float cxf0 = tapc<G>(cj, j, tl.xf[0]), cxf1 = tapc<G>(cj, j, tl.xf[1]);
            // per lane: x taps, then y, then z, for each of ax, ay, az (x-tap
            // differences per lane, their fused multiply-adds paired)
            const float2 cxb = make_float2(cxb0, cxb1), cxf = make_float2(cxf0, cxf1);
            ax = fmac2(ax, cxf, make_float2(S1[5 + j] - S1[4 - j], S1[6 + j] - S1[5 - j]));
            ay = fmac2(ay, cxb, make_float2(S6[4 + j] - S6[3 - j], S6[5 + j] - S6[4 - j]));
            az = fmac2(az, cxb, make_float2(S5[4 + j] - S5[3 - j], S5[5 + j] - S5[4 - j]));
            ay = fmac2(ay, bc2(cyf), sub2(p2, m2));
            ax = fmac2(ax, bc2(cyb), sub2(p6, m6));
            az = fmac2(az, bc2(cyb), sub2(p4, m4));
            az = fmac2(az, bc2(czf), sub2(r3[4 + j], r3[3 - j]));
            ax = fmac2(ax, bc2(czb), sub2(r5[4 + j], r5[3 - j]));
            ay = fmac2(ay, bc2(czb), sub2(r4[4 + j], r4[3 - j]));
        }
    }
}

// Every x / y tap of velocity tile (bx, by), and every face-density
// neighbour, lies inside the grid.
__device__ __forceinline__ bool pair_vtile_inside(const StepArgs<float> &A, int bx, int by)
{
    const int x0 = bx * PV_OX, y0 = by * PV_OY;
    return x0 - T_H >= 0 && x0 + PV_OX - 1 + T_H < A.nx && y0 - T_H >= 0 && y0 + PV_OY - 1 + T_H < A.ny;
}

// One z-march of a block over cell tile (bx, by), planes [zb, ze); it0 as
// in stress_pair_march. TIN: pair_vtile_inside(A, bx, by) holds, and the
// x / y limits and neighbour tests are compile-time constants.
// bars_at: the three mbarriers (default: the first bytes of smem; the
// persistent batch kernel keeps separate ones for each phase)
template <int NC, bool TIN, bool COH = false>
__device__ __forceinline__ int velocity_pair_march(const TmapsPairVelocity &M, const StepArgs<float> &A,
                                                   const float *rho_tab, unsigned char *smem, int bx,
                                                   int by, int zb, int ze, int it0,
                                                   unsigned long long *bars_at = nullptr)
{
    unsigned long long *bars = bars_at ? bars_at : reinterpret_cast<unsigned long long *>(smem);
    float *slots = reinterpret_cast<float *>(smem + 128);
    const int tid = threadIdx.x;
    const int l = tid & (PR_LX - 1), r = tid >> 4;
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long sy = A.sy, sz = A.sz;
    const int x0 = bx * PV_OX, y0 = by * PV_OY;
    const int ix = x0 + 2 * l, iy = y0 + r;
    const bool out_ok = TIN || (ix < nx && iy < ny);   // nx even: both cells
    const int col = out_ok ? (int)(iy * sy + ix) : 0;
    const bool has_dvol = A.dvol != nullptr;
    const unsigned bytes = (5u * PV_TSZ + 3u * PV_CSZ + (has_dvol ? (unsigned)PV_CSZ : 0u)) * 4u;

    auto issue = [&](int i) {
        const int z = zb + i;
        if (tid != 0 || z >= ze) return;
        const int sl = (it0 + i) % 3;
        unsigned long long *bar = bars + sl;
        float *d = slots + sl * PV_SLOT;
        fence_proxy_async();
        mbar_expect_tx(bar, bytes);
#pragma unroll
        for (int f = 0; f < 5; ++f) tma_load_3d(d + f * PV_TSZ, &M.st[f], x0 - T_H, y0 - T_H, z, bar);
#pragma unroll
        for (int c = 0; c < 3; ++c) tma_load_3d(d + 5 * PV_TSZ + c * PV_CSZ, &M.vc[c], x0, y0, z, bar);
        if (has_dvol) tma_load_3d(d + 5 * PV_TSZ + 3 * PV_CSZ, &M.dv, x0, y0, z, bar);
    };
    const float *p3 = A.s[2] + col, *p4 = A.s[3] + col, *p5 = A.s[4] + col;
    auto ld2col = [&](const float *f, int z) -> float2 {
        return (out_ok && z >= 0 && z < nz) ? ld2_column<COH>(f + (long long)z * sz) : make_float2(0.f, 0.f);
    };
    float2 r3[8], r4[8], r5[8];   // lane pairs: r3[k] <-> z-3+k, r4/r5[k] <-> z-4+k
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        r3[k] = ld2col(p3, zb - 3 + k);
        r4[k] = ld2col(p4, zb - 4 + k);
        r5[k] = ld2col(p5, zb - 4 + k);
    }
    TapLimits tl;
    if constexpr (TIN) {
        tl.xb[0] = tl.xb[1] = tl.xf[0] = tl.xf[1] = tl.yb = tl.yf = T_H;
    } else {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            tl.xb[c] = lim_b(ix + c, nx);
            tl.xf[c] = lim_f(ix + c, nx);
        }
        tl.yb = lim_b(iy, ny);
        tl.yf = lim_f(iy, ny);
    }
    const bool xin1 = TIN || ix + 1 < nx - 1;   // cell 1 has a +x neighbour (cell 0 always does)
    const bool yin = TIN || iy < ny - 1;
    float dyx = 1.0f, dxx[2] = {1.0f, 1.0f};
    if (A.dz && out_ok) {
        dyx = A.dy[iy];
        dxx[0] = A.dx[ix];
        dxx[1] = A.dx[ix + 1];
    }
    const int tc = (r + T_H) * PV_TW + 2 * l + T_H;
    const int cc = r * PV_OX + 2 * l;
    const uint32_t *lab32 = reinterpret_cast<const uint32_t *>(A.lab);
    // labels of plane z: the pair, cell x+2, and the pair at y+1
    auto ldlabs = [&](int z, uint32_t &pr, uint16_t &px2, uint32_t &py) {
        pr = 0u; px2 = 0; py = 0u;
        if (out_ok && z < nz) {
            const long long b = (long long)z * sz + col;
            pr = __ldg(lab32 + (b >> 1));
            if (xin1) px2 = A.lab[b + 2];
            if (yin) py = __ldg(lab32 + ((b + sy) >> 1));
        }
    };
    uint32_t lab_c, lab_y, nlab_c, nlab_y;
    uint16_t lab_x2, nlab_x2;
    ldlabs(zb, lab_c, lab_x2, lab_y);
    ldlabs(zb + 1, nlab_c, nlab_x2, nlab_y);
    int *status = A.status;

    issue(0);
    issue(1);
    for (int i = 0; i < ze - zb; ++i) {
        const int z = zb + i;
        const int g = it0 + i, sl = g % 3;
        if (tid < 32) mbar_wait(bars + sl, (unsigned)(g / 3) & 1u, status);
        __syncthreads();   // slot g landed (observed by warp 0); slot g + 2 is free
        issue(i + 2);
        const float2 n3 = ld2col(p3, z + 5), n4 = ld2col(p4, z + 4), n5 = ld2col(p5, z + 4);
        uint32_t mlab_c, mlab_y;
        uint16_t mlab_x2;
        ldlabs(z + 2, mlab_c, mlab_x2, mlab_y);
        const float *slot = slots + sl * PV_SLOT;
        const float *t = slot + tc;
        float2 ax, ay, az;
        const bool fast = NC == 4 && TIN && z >= T_H && z <= nz - 1 - T_H;
        if (fast) pair_vel_taps<NC, false>(A, z, t, t + PV_TSZ, t + 2 * PV_TSZ, t + 3 * PV_TSZ, t + 4 * PV_TSZ, r3, r4, r5, tl, ax, ay, az);
        else pair_vel_taps<NC, true>(A, z, t, t + PV_TSZ, t + 2 * PV_TSZ, t + 3 * PV_TSZ, t + 4 * PV_TSZ, r3, r4, r5, tl, ax, ay, az);
        if (out_ok) {
            const uint16_t lc[2] = {(uint16_t)(lab_c & 0xFFFFu), (uint16_t)(lab_c >> 16)};
            const uint16_t lyv[2] = {(uint16_t)(lab_y & 0xFFFFu), (uint16_t)(lab_y >> 16)};
            const uint16_t lzv[2] = {(uint16_t)(nlab_c & 0xFFFFu), (uint16_t)(nlab_c >> 16)};
            const uint16_t lxv[2] = {lc[1], lab_x2};
            const float *vc = slot + 5 * PV_TSZ + cc;
            float dmp[2];
            {
                const float dz = A.dz ? A.dz[z] : 1.0f;
                float2 dvv = make_float2(1.0f, 1.0f);
                if (has_dvol) dvv = lds2(vc + 3 * PV_CSZ);
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    float d = 1.0f;
                    if (A.dz) {
                        d = dz * dyx;
                        d = d * dxx[c];
                    }
                    if (has_dvol) d = A.dz ? d * pick(dvv, c) : pick(dvv, c);
                    dmp[c] = d;
                }
            }
            const float2 vo[3] = {lds2(vc), lds2(vc + PV_CSZ), lds2(vc + 2 * PV_CSZ)};
            // the six face divisions: Markstein quotients for all of them
            // (independent chains, lane pairs), then the exact fallback for
            // the lanes whose numerator or face rules that out (div_face_rcp)
            float r0[2], rn[2][3];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const bool xin = c == 0 ? true : xin1;
                r0[c] = rho_tab[lc[c] & LAB_MAT];
                rn[c][0] = xin ? rho_tab[lxv[c] & LAB_MAT] : 0.f;
                rn[c][1] = yin ? rho_tab[lyv[c] & LAB_MAT] : 0.f;
                rn[c][2] = (z < nz - 1) ? rho_tab[lzv[c] & LAB_MAT] : 0.f;
            }
            const bool has_nb[2][3] = {{true, yin, z < nz - 1}, {xin1, yin, z < nz - 1}};
            const float2 r02 = make_float2(r0[0], r0[1]);
            const float2 y2 = make_float2(__ldg(A.rinv + (lc[0] & LAB_MAT)), __ldg(A.rinv + (lc[1] & LAB_MAT)));
            const float2 a2[3] = {ax, ay, az};
            float2 u[3], rv[3], q[3];
            bool fine = true;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                // face density 0.5 (rho0 + rho1), or the cell's own at the last slice
                const float2 h = mul2(bc2(0.5f), add2(r02, make_float2(rn[0][d], rn[1][d])));
                rv[d] = make_float2(has_nb[0][d] ? h.x : r0[0], has_nb[1][d] ? h.y : r0[1]);
                u[d] = mul2(bc2(A.dt_h), a2[d]);
                // markstein(u, rv, y) per lane: q0 = u y, two corrections
                const float2 nb = make_float2(-rv[d].x, -rv[d].y);
                const float2 q0 = mul2(u[d], y2);
                const float2 q1 = fmac2(q0, fmac2(u[d], nb, q0), y2);
                q[d] = fmac2(q1, fmac2(u[d], nb, q1), y2);
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const float au = fabsf(c ? u[d].y : u[d].x);
                    fine = fine && (c ? rv[d].y : rv[d].x) == r0[c] && au >= 0x1p-100f && au <= 0x1p100f;
                }
            }
            if (!fine) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    q[d].x = div_face_rcp(u[d].x, rv[d].x, rv[d].x == r0[0], y2.x);
                    q[d].y = div_face_rcp(u[d].y, rv[d].y, rv[d].y == r0[1], y2.y);
                }
            }
            const float2 dmp2 = make_float2(dmp[0], dmp[1]);
            float vn[3][2];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float2 v = mul2(add2(vo[d], q[d]), dmp2);
                vn[d][0] = v.x;
                vn[d][1] = v.y;
            }
            const long long idx = (long long)z * sz + col;
            stg2(A.v[0] + idx, vn[0][0], vn[0][1]);
            stg2(A.v[1] + idx, vn[1][0], vn[1][1]);
            stg2(A.v[2] + idx, vn[2][0], vn[2][1]);
            if (A.rec_kind != 0) {
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    if (lc[c] & LAB_REC)
                        record_cell(A, idx + c, A.rec_kind == 1 ? vn[0][c] : (A.rec_kind == 2 ? vn[1][c] : vn[2][c]));
            }
        }
        lab_c = nlab_c; lab_x2 = nlab_x2; lab_y = nlab_y;
        nlab_c = mlab_c; nlab_x2 = mlab_x2; nlab_y = mlab_y;
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
    return ze - zb;
}

template <int NC>
__global__ void __launch_bounds__(PV_N, 2) k_velocity_pair(const __grid_constant__ TmapsPairVelocity M,
                                                           const StepArgs<float> A, int n_mat)
{
    extern __shared__ __align__(128) unsigned char smem_pair[];
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_pair);
    float *rsm = reinterpret_cast<float *>(smem_pair + 128) + 3 * PV_SLOT;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < 3; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    const bool rho_smem = pair_rho_in_smem(n_mat);
    if (rho_smem)
        for (int i = tid; i < n_mat; i += PV_N) rsm[i] = A.rho[i];
    __syncthreads();
    const float *rho_tab = rho_smem ? rsm : A.rho;
    const int zb = blockIdx.z * A.zc, ze = min(zb + A.zc, A.nz);
    int bx, by;
    interior_first(A.nx < 36 ? 0 : (A.nx - 36) / PV_OX, A.ny < 20 ? 0 : (A.ny - 20) / PV_OY, gridDim.x,
                   gridDim.y, blockIdx.x + gridDim.x * blockIdx.y, bx, by);
    if (pair_vtile_inside(A, bx, by))
        velocity_pair_march<NC, true>(M, A, rho_tab, smem_pair, bx, by, zb, ze, 0);
    else
        velocity_pair_march<NC, false>(M, A, rho_tab, smem_pair, bx, by, zb, ze, 0);
}

// ---------------------------------------------------------------- batches
// Many solves (any grid sizes) advance one step per launch pair. Work items
// (solve, tile x, tile y, z-chunk) are listed solve by solve and chunk-major
// within a solve, so blocks that run together march the same planes of
// neighbouring tiles; each resident block walks a contiguous run of items,
// re-staging the solve's arguments and tables only when the solve changes.
// All solves of a pair batch have rows of 16-byte multiples.
template <int NC, bool TS>
__global__ void __launch_bounds__(PS_N, 2)
    k_stress_pair_batch(const StepArgs<float> *__restrict__ descs, const TmapsPairStress *__restrict__ maps,
                        const float *const *__restrict__ tabs, const int *__restrict__ n_mats,
                        const BatchItem *__restrict__ items, int n_items, int k)
{
    extern __shared__ __align__(128) unsigned char smem_pair[];
    __shared__ __align__(16) StepArgs<float> As;
    float *tsm = reinterpret_cast<float *>(smem_pair + PS_SMEM_FIXED);
    stress_pair_init(smem_pair);
    const int per = (n_items + gridDim.x - 1) / gridDim.x;
    const int i0 = blockIdx.x * per, i1 = min(n_items, i0 + per);
    int cur = -1;
    PairPhases ph{0, 0};
    for (int it = i0; it < i1; ++it) {
        const BatchItem w = items[it];
        __syncthreads();   // the previous march is finished by every thread
        const bool fresh = w.solve != cur;
        if (fresh) {
            copy_args(&As, descs + w.solve, k);
            if (TS) stage_table(tsm, tabs[w.solve], n_mats[w.solve]);
        }
        __syncthreads();
        const int zb = w.bz * As.zc, ze = min(zb + As.zc, As.nz);
        const float *tab = TS ? tsm : tabs[w.solve];
        if (pair_tile_inside(As, w.bx, w.by))
            stress_pair_march<NC, TS, true>(maps[w.solve], As, tab, smem_pair, w.bx, w.by, zb, ze, ph);
        else
            stress_pair_march<NC, TS, false>(maps[w.solve], As, tab, smem_pair, w.bx, w.by, zb, ze, ph);
        cur = w.solve;
    }
}

template <int NC>
__global__ void __launch_bounds__(PV_N, 2)
    k_velocity_pair_batch(const StepArgs<float> *__restrict__ descs, const TmapsPairVelocity *__restrict__ maps,
                          const int *__restrict__ n_mats, const BatchItem *__restrict__ items, int n_items,
                          int k)
{
    extern __shared__ __align__(128) unsigned char smem_pair[];
    __shared__ __align__(16) StepArgs<float> As;
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_pair);
    float *rsm = reinterpret_cast<float *>(smem_pair + 128) + 3 * PV_SLOT;
    if (threadIdx.x == 0) {
        for (int s = 0; s < 3; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    const int per = (n_items + gridDim.x - 1) / gridDim.x;
    const int i0 = blockIdx.x * per, i1 = min(n_items, i0 + per);
    int cur = -1, it0 = 0;
    for (int it = i0; it < i1; ++it) {
        const BatchItem w = items[it];
        __syncthreads();
        const bool fresh = w.solve != cur;
        if (fresh) {
            copy_args(&As, descs + w.solve, k);
            for (int i = threadIdx.x; i < n_mats[w.solve]; i += PV_N) rsm[i] = As.rho[i];
        }
        __syncthreads();
        const int zb = w.bz * As.zc, ze = min(zb + As.zc, As.nz);
        if (pair_vtile_inside(As, w.bx, w.by))
            it0 += velocity_pair_march<NC, true>(maps[w.solve], As, rsm, smem_pair, w.bx, w.by, zb, ze, it0);
        else
            it0 += velocity_pair_march<NC, false>(maps[w.solve], As, rsm, smem_pair, w.bx, w.by, zb, ze, it0);
        cur = w.solve;
    }
}

// ---------------------------------------------------------------- persistent batches
// One launch advances every batched solve by nk steps: the blocks (all
// resident: a cooperative launch) alternate a stress phase and a velocity
// phase over the same work items as k_stress_pair_batch /
// k_velocity_pair_batch, separated by grid-wide barriers. Differences from
// the per-step launches, each needed because other blocks of the same launch
// write the fields a block reads:
//  - the z-ring column loads are L2-coherent (ld.global.cg) instead of the
//    read-only path;
//  - after each barrier every thread fences the async proxy, so the TMA
//    boxes it issues read what the barrier made visible;
//  - the two phases keep separate mbarriers (stress: bytes 0-23, velocity:
//    bytes 64-87 of shared memory) and share the data region after them, so
//    the strain ring's zero pads, the stiffness table and the density table
//    are restaged at the start of each phase.
// The arithmetic is the per-step kernels': results are bit-identical.
constexpr unsigned long long GRID_SPIN_LIMIT = 1ull << 24;   // barrier polls (64 ns sleeps) before giving up

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }

// Bounded grid-wide barrier: a block's writes, a fence, its arrival; then
// poll (acquire) until `target` blocks have arrived, at most GRID_SPIN_LIMIT
// polls, after which it records STATUS_TIMEOUT in the status word and goes
// on (the results are then invalid; nothing hangs).
__device__ __forceinline__ void grid_barrier(unsigned *count, unsigned target, int *status)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        fence_proxy_async_global();
        __threadfence();
        atomicAdd(count, 1u);
        unsigned long long it = 0;
        while (ld_acquire_u32(count) < target) {
            if (++it >= GRID_SPIN_LIMIT) {
                if (status) atomicExch(status, STATUS_TIMEOUT);
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
    fence_proxy_async_global();
}

__host__ __device__ constexpr size_t persistent_pair_smem(size_t smem_s, size_t smem_v)
{
    return smem_s > smem_v ? smem_s : smem_v;
}

template <int NC, bool TS>
__global__ void __launch_bounds__(PS_N, 2)
    k_pair_batch_persistent(const StepArgs<float> *__restrict__ descs, const TmapsPairStress *__restrict__ smaps,
                            const TmapsPairVelocity *__restrict__ vmaps, const float *const *__restrict__ tabs,
                            const int *__restrict__ n_mats, const BatchItem *__restrict__ items_s, int n_s,
                            const BatchItem *__restrict__ items_v, int n_v, int nk, unsigned *bar, int *status)
{
    extern __shared__ __align__(128) unsigned char smem_pair[];
    __shared__ __align__(16) StepArgs<float> As;
    unsigned long long *vbars = reinterpret_cast<unsigned long long *>(smem_pair) + 8;
    float *tsm = reinterpret_cast<float *>(smem_pair + PS_SMEM_FIXED);
    float *rsm = reinterpret_cast<float *>(smem_pair + 128) + 3 * PV_SLOT;
    stress_pair_init(smem_pair);
    if (threadIdx.x == 0) {
        for (int b = 0; b < 3; ++b) mbar_init(vbars + b, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const int per_s = (n_s + gridDim.x - 1) / gridDim.x, i0s = blockIdx.x * per_s, i1s = min(n_s, i0s + per_s);
    const int per_v = (n_v + gridDim.x - 1) / gridDim.x, i0v = blockIdx.x * per_v, i1v = min(n_v, i0v + per_v);
    PairPhases ph{0, 0};
    int it0 = 0;
    unsigned nbar = 0;
    for (int k = 0; k < nk; ++k) {
        int cur = -1;
        for (int it = i0s; it < i1s; ++it) {
            const BatchItem w = items_s[it];
            __syncthreads();   // the previous march is finished by every thread
            if (w.solve != cur) {
                copy_args(&As, descs + w.solve, k);
                if (TS) stage_table(tsm, tabs[w.solve], n_mats[w.solve]);
            }
            __syncthreads();
            const int zb = w.bz * As.zc, ze = min(zb + As.zc, As.nz);
            const float *tab = TS ? tsm : tabs[w.solve];
            if (pair_tile_inside(As, w.bx, w.by))
                stress_pair_march<NC, TS, true, true>(smaps[w.solve], As, tab, smem_pair, w.bx, w.by, zb, ze, ph);
            else
                stress_pair_march<NC, TS, false, true>(smaps[w.solve], As, tab, smem_pair, w.bx, w.by, zb, ze, ph);
            cur = w.solve;
        }
        grid_barrier(bar, ++nbar * gridDim.x, status);
        cur = -1;
        for (int it = i0v; it < i1v; ++it) {
            const BatchItem w = items_v[it];
            __syncthreads();
            if (w.solve != cur) {
                copy_args(&As, descs + w.solve, k);
                for (int i = threadIdx.x; i < n_mats[w.solve]; i += PV_N) rsm[i] = As.rho[i];
            }
            __syncthreads();
            const int zb = w.bz * As.zc, ze = min(zb + As.zc, As.nz);
            if (pair_vtile_inside(As, w.bx, w.by))
                it0 += velocity_pair_march<NC, true, true>(vmaps[w.solve], As, rsm, smem_pair, w.bx, w.by, zb, ze,
                                                           it0, vbars);
            else
                it0 += velocity_pair_march<NC, false, true>(vmaps[w.solve], As, rsm, smem_pair, w.bx, w.by, zb, ze,
                                                            it0, vbars);
            cur = w.solve;
        }
        grid_barrier(bar, ++nbar * gridDim.x, status);
        stress_pair_zero_pads(smem_pair);   // the velocity slots overwrote them
    }
}

// (n_mat, 36) column-split stiffness from the (n_mat, 24) upper-triangle
// rows, with C[I][J] as row_dot() reads it: tab[m][4J + I] for I < 4,
// tab[m][24 + 2J + I - 4] for I = 4, 5
__global__ void k_c21_to_tab36(const float *c21, float *tab, int n_mat)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_mat) return;
    for (int J = 0; J < 6; ++J)
        for (int I = 0; I < 6; ++I)
            tab[m * TAB36 + (I < 4 ? 4 * J + I : 24 + 2 * J + I - 4)] = c21[m * C21_STRIDE + c21_slot(I, J)];
}

}  // namespace pe
