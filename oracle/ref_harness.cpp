// TEST INFRASTRUCTURE ONLY — runs the reference's own CUDA-C kernel sources
// (Jerome-Graves/pulse-echo-azimuthal-simulation, sim/core/fdtd.py) on the
// host CPU, so the C oracle and the CUDA product path can be pinned against
// the reference's own update arithmetic without a GPU.
//
// The kernel bodies are NOT in this file: oracle/build_ref.py imports the
// reference module where it lies and writes its source strings into
// oracle/_ref/ref_kernels.inc (git-ignored), which is #included below after
// the CUDA built-ins have been mapped onto a sequential thread emulation.
// None of the included kernels uses shared memory or __syncthreads, and no
// kernel reads a buffer it writes at another cell, so running the threads of
// a launch one after another is exact.
//
// What IS in this file is a restatement of the two host drivers that launch
// those kernels:
//   ref_labels_forward  sim/core/fdtd.py:1741-1816 (forward_fused_labels loop:
//                       z-slabs of strains_zp + stress_lab_u, source, vel_zp,
//                       receiver gather)
//   ref_dense_forward   sim/core/fdtd.py:875-921 (forward_fused loop: strains,
//                       stress_acc, source, vel_update, damping, record)
// Launch shapes follow the reference (:1784-1797, :878-880).
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
struct emu_dim3 {
    unsigned x, y, z;
};
thread_local emu_dim3 blockIdx, blockDim, threadIdx;
}  // namespace

#define __global__
#define __device__
#define __forceinline__ inline
#define __restrict__ __restrict

#include "_ref/ref_kernels.inc"

namespace {

template <typename F>
void launch2d(unsigned gx, unsigned gy, unsigned bx, F &&f)
{
#pragma omp parallel for schedule(static)
    for (long b = 0; b < (long)gx * gy; ++b) {
        blockIdx = {(unsigned)(b % gx), (unsigned)(b / gx), 0};
        blockDim = {bx, 1, 1};
        for (unsigned t = 0; t < bx; ++t) {
            threadIdx = {t, 0, 0};
            f();
        }
    }
}

template <typename F>
void launch1d(long nblocks, unsigned bx, F &&f)
{
#pragma omp parallel for schedule(static)
    for (long b = 0; b < nblocks; ++b) {
        blockIdx = {(unsigned)b, 0, 0};
        blockDim = {bx, 1, 1};
        for (unsigned t = 0; t < bx; ++t) {
            threadIdx = {t, 0, 0};
            f();
        }
    }
}

// sf[I][s_idx] += wn * s_w  (CuPy gather, add, scatter: a repeated cell keeps
// its last entry) — sim/core/fdtd.py:1798-1800
void add_source(float *s[6], const int64_t *s_idx, const float *s_w, int n_src, float wn)
{
    std::vector<float> tmp((size_t)n_src * 3);
    for (int k = 0; k < n_src; ++k) {
        float add = wn * s_w[k];
        for (int I = 0; I < 3; ++I) tmp[(size_t)k * 3 + I] = s[I][s_idx[k]] + add;
    }
    for (int k = 0; k < n_src; ++k)
        for (int I = 0; I < 3; ++I) s[I][s_idx[k]] = tmp[(size_t)k * 3 + I];
}

// (val * r_w).sum() per receiver group, summed in list order —
// sim/core/fdtd.py:1806-1813 (pressure from pre-damp stress) and :914-918
void record(float *out, int n_groups, const int64_t *r_off, const int64_t *r_idx,
            const float *r_w, int kind, float *const s[6], float *const v[3],
            const float *damp, int damped)
{
    for (int r = 0; r < n_groups; ++r) {
        float acc = 0.f;
        for (int64_t k = r_off[r]; k < r_off[r + 1]; ++k) {
            long q = (long)r_idx[k];
            float val;
            if (kind == 0) {
                float a = s[0][q], b = s[1][q], c = s[2][q];
                if (damped && damp) {
                    float d = damp[q];
                    a = a * d; b = b * d; c = c * d;
                }
                float t = a + b;
                t = t + c;
                val = -t / 3.0f;
            } else {
                val = v[kind - 1][q];
            }
            float prod = val * r_w[k];
            acc = acc + prod;
        }
        out[r] = acc;
    }
}

}  // namespace

extern "C" int ref_abi_version(void) { return 1; }

// Label path. mats: uint8 material index (lab + 1), Ct: (n_mat, 36) f32,
// act: 36 flags, rho_t: (n_mat,), damp: combined f32 volume or NULL.
extern "C" int ref_labels_forward(int nz, int ny, int nx, const uint8_t *mats,
                                  const float *Ct, const int32_t *act, const float *rho_t,
                                  const float *damp, const float *coeffs, int nc,
                                  float inv_h, float dt, float dt_h, int slab,
                                  const int64_t *s_idx, const float *s_w, int n_src,
                                  const float *wavelet, int nt, int n_groups,
                                  const int64_t *r_off, const int64_t *r_idx,
                                  const float *r_w, int record_kind, float *rec_out,
                                  float *state_out, int n_threads)
{
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    if (nc < 1 || nc > 4 || slab < 1) return 1;
    const long ncell = (long)nz * ny * nx;
    std::vector<float> store((size_t)9 * ncell, 0.f);
    float *v[3], *s[6];
    for (int i = 0; i < 3; ++i) v[i] = store.data() + (size_t)i * ncell;
    for (int i = 0; i < 6; ++i) s[i] = store.data() + (size_t)(3 + i) * ncell;
    std::vector<float> gbuf((size_t)6 * (slab + 2) * ny * nx, 0.f);
    float *g[6];
    for (int i = 0; i < 6; ++i) g[i] = gbuf.data() + (size_t)i * (slab + 2) * ny * nx;
    static const float one_damp = 0.f;
    const float *damp_arg = damp ? damp : &one_damp;
    const int use_damp = damp ? 1 : 0;
    const unsigned tpb = 256, tpbc = 128;
    const unsigned gcx = (unsigned)((nx + tpbc - 1) / tpbc);

    for (int n = 0; n < nt; ++n) {
        for (int z0 = 0; z0 < nz; z0 += slab) {
            int z1 = z0 + slab < nz ? z0 + slab : nz;
            int zg0 = z0 - 1 > 0 ? z0 - 1 : 0;
            int zg1 = z1 + 1 < nz ? z1 + 1 : nz;
            launch2d(gcx, (unsigned)ny, tpbc, [&] {
                strains_zp(v[0], v[1], v[2], g[0], g[1], g[2], g[3], g[4], g[5], coeffs, nc,
                           inv_h, nz, ny, nx, zg0, zg1);
            });
            long ncr = (long)(z1 - z0) * ny * nx;
            launch1d((ncr + tpb - 1) / tpb, tpb, [&] {
                stress_lab_u(g[0], g[1], g[2], g[3], g[4], g[5], s[0], s[1], s[2], s[3], s[4],
                             s[5], mats, Ct, act, damp_arg, use_damp, dt, nz, ny, nx, z0, z1,
                             zg0);
            });
        }
        add_source(s, s_idx, s_w, n_src, wavelet[n]);
        launch2d(gcx, (unsigned)ny, tpbc, [&] {
            vel_zp(s[0], s[1], s[2], s[3], s[4], s[5], v[0], v[1], v[2], mats, rho_t, damp_arg,
                   use_damp, coeffs, nc, dt_h, nz, ny, nx);
        });
        record(rec_out + (size_t)n * n_groups, n_groups, r_off, r_idx, r_w, record_kind, s, v,
               damp, 0);
    }
    if (state_out) std::memcpy(state_out, store.data(), sizeof(float) * 9 * ncell);
    return 0;
}

// Dense path. Cflat: (36, nz, ny, nx) f32, act: 36 flags, rv*: face densities
// (f32 volumes), damp: combined f32 volume or NULL.
extern "C" int ref_dense_forward(int nz, int ny, int nx, const float *Cflat,
                                 const int32_t *act, const float *rvx, const float *rvy,
                                 const float *rvz, const float *damp, const float *coeffs,
                                 int nc, float inv_h, float dt, float dt_h,
                                 const int64_t *s_idx, const float *s_w, int n_src,
                                 const float *wavelet, int nt, int n_groups,
                                 const int64_t *r_off, const int64_t *r_idx,
                                 const float *r_w, int record_kind, float *rec_out,
                                 float *state_out, int n_threads)
{
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    if (nc < 1) return 1;
    const long ncell = (long)nz * ny * nx;
    std::vector<float> store((size_t)15 * ncell, 0.f);
    float *v[3], *s[6], *g[6];
    for (int i = 0; i < 3; ++i) v[i] = store.data() + (size_t)i * ncell;
    for (int i = 0; i < 6; ++i) s[i] = store.data() + (size_t)(3 + i) * ncell;
    for (int i = 0; i < 6; ++i) g[i] = store.data() + (size_t)(9 + i) * ncell;
    const unsigned tpb = 256;
    const long blocks = (ncell + tpb - 1) / tpb;

    for (int n = 0; n < nt; ++n) {
        launch1d(blocks, tpb, [&] {
            strains(v[0], v[1], v[2], g[0], g[1], g[2], g[3], g[4], g[5], coeffs, nc, inv_h, nz,
                    ny, nx);
        });
        launch1d(blocks, tpb, [&] {
            stress_acc(g[0], g[1], g[2], g[3], g[4], g[5], s[0], s[1], s[2], s[3], s[4], s[5],
                       Cflat, act, dt, nz, ny, nx);
        });
        add_source(s, s_idx, s_w, n_src, wavelet[n]);
        launch1d(blocks, tpb, [&] {
            vel_update(s[0], s[1], s[2], s[3], s[4], s[5], v[0], v[1], v[2], rvx, rvy, rvz,
                       coeffs, nc, dt_h, nz, ny, nx);
        });
        if (damp) {
#pragma omp parallel for schedule(static)
            for (long i = 0; i < ncell; ++i) {
                float d = damp[i];
                v[0][i] *= d; v[1][i] *= d; v[2][i] *= d;
                for (int I = 0; I < 6; ++I) s[I][i] *= d;
            }
        }
        record(rec_out + (size_t)n * n_groups, n_groups, r_off, r_idx, r_w, record_kind, s, v,
               nullptr, 0);
    }
    if (state_out) std::memcpy(state_out, store.data(), sizeof(float) * 9 * ncell);
    return 0;
}
