// Power-diagram (Laguerre) labelling of a cylinder on the device.
//
// Same arithmetic as the reference's exact labeller
// (sim/core/specimen.py:298-337): per grid point, in float64,
//   d = ((x - sx)^2 + (y - sy)^2) - w  +  (z - sz)^2
// minimised over ALL seeds, first index on ties, -1 where x^2 + y^2 > R2
// (R2 is the caller's R**2, so the inside test matches bit for bit).
// Compiled with -fmad=false so no product is fused into a sum, as in NumPy.
// One thread per cell; seeds are staged through shared memory in tiles.
#include <atomic>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "pefdtd.h"

namespace {

constexpr int SEED_TILE = 256;

__global__ void k_label_cylinder(const double *__restrict__ xs, const double *__restrict__ ys,
                                 const double *__restrict__ zs, int nx, int ny, int nz, double R2,
                                 const double *__restrict__ seeds, const double *__restrict__ w,
                                 int ns, int32_t *__restrict__ out)
{
    __shared__ double sh[SEED_TILE][4];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)nx * ny * nz;
    const bool live = i < n;
    int ix = 0, iy = 0, iz = 0;
    if (live) {
        ix = (int)(i % nx);
        iy = (int)((i / nx) % ny);
        iz = (int)(i / ((long long)nx * ny));
    }
    const double x = live ? xs[ix] : 0.0, y = live ? ys[iy] : 0.0, z = live ? zs[iz] : 0.0;
    const bool inside = live && (x * x + y * y <= R2);
    double best = 0.0;
    int arg = -1;
    for (int t0 = 0; t0 < ns; t0 += SEED_TILE) {
        const int nt = min(SEED_TILE, ns - t0);
        __syncthreads();
        for (int k = threadIdx.x; k < nt; k += blockDim.x) {
            sh[k][0] = seeds[(t0 + k) * 3 + 0];
            sh[k][1] = seeds[(t0 + k) * 3 + 1];
            sh[k][2] = seeds[(t0 + k) * 3 + 2];
            sh[k][3] = w[t0 + k];
        }
        __syncthreads();
        if (inside) {
            for (int k = 0; k < nt; ++k) {
                const double dx = x - sh[k][0], dy = y - sh[k][1], dz = z - sh[k][2];
                double d = dx * dx + dy * dy;
                d = d - sh[k][3];
                d = d + dz * dz;
                if (arg < 0 || d < best) {
                    best = d;
                    arg = t0 + k;
                }
            }
        }
    }
    if (live) out[i] = inside ? arg : -1;
}

// Solver grid of a specimen rotated by -rot about z, resampled by nearest
// neighbour (reference sim/core/rotation_test.py:60-137, restated in
// pefdtd/specimen.py rotated_grid): the core cell (k, j, i) samples the
// specimen label at
//   gi = rint((ca*u_i - sa*u_j) / h_spec + c),  gj = rint((sa*u_i + ca*u_j) / h_spec + c),
//   gz = trunc(clip(((k + 0.5)*h) / h_spec, 0, nz_s - 1)),
// u_i = (i + 0.5)*h - D/2, c = (nx_s - 1)/2, or -1 where (gi, gj) leaves
// the specimen; every expression in the NumPy evaluation order, float64,
// no fused multiply-add (-fmad=false), rint rounding half to even as
// np.rint. The core sits at offset m in each axis of the output, whose
// other cells the host fills with -1.
__global__ void k_rotated_grid(const int32_t *__restrict__ lab_xyz, int nx_s, int nz_s, int nd, int ndz,
                               double h, double h_spec, double half_d, double ca, double sa, double c_off,
                               int m, int nxo, int32_t *__restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)nd * nd * ndz;
    if (t >= n) return;
    const int i = (int)(t % nd);
    const int j = (int)((t / nd) % nd);
    const int k = (int)(t / ((long long)nd * nd));
    const double ui = ((double)i + 0.5) * h - half_d;
    const double uj = ((double)j + 0.5) * h - half_d;
    const double xr = ca * ui - sa * uj;
    const double yr = sa * ui + ca * uj;
    const long long gi = (long long)rint(xr / h_spec + c_off);
    const long long gj = (long long)rint(yr / h_spec + c_off);
    double tz = ((double)k + 0.5) * h / h_spec;
    tz = fmin(fmax(tz, 0.0), (double)(nz_s - 1));
    const int gz = (int)tz;
    int32_t v = -1;
    if (gi >= 0 && gi < nx_s && gj >= 0 && gj < nx_s) v = lab_xyz[(gi * nx_s + gj) * nz_s + gz];
    out[((long long)(m + k) * nxo + (m + j)) * nxo + (m + i)] = v;
}

thread_local std::string g_err_spec;

}  // namespace

extern "C" int pe_rotated_grid(const int32_t *labels_dev, int nx_s, int nz_s, double h_spec, double h,
                               int nd, int ndz, double cos_a, double sin_a, int m, int32_t *out_dev,
                               void *stream)
{
    if (!labels_dev || !out_dev || nx_s < 1 || nz_s < 1 || nd < 1 || ndz < 1 || m < 0 || !(h > 0) ||
        !(h_spec > 0))
        return PE_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    const long long nxo = nd + 2LL * m, nzo = ndz + 2LL * m;
    cudaError_t e = cudaMemsetAsync(out_dev, 0xFF, sizeof(int32_t) * (size_t)(nzo * nxo * nxo), st);
    if (e == cudaSuccess) {
        const double D = nx_s * h_spec;
        const long long n = (long long)nd * nd * ndz;
        k_rotated_grid<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(labels_dev, nx_s, nz_s, nd, ndz, h, h_spec,
                                                                   D / 2.0, cos_a, sin_a, (nx_s - 1) / 2.0, m,
                                                                   (int)nxo, out_dev);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? PE_OK : PE_ERR_CUDA;
}

extern "C" int pe_label_cylinder(const double *xs, int nx, const double *ys, int ny,
                                 const double *zs, int nz, double R2, const double *seeds,
                                 const double *weights, int ns, int32_t *out_dev, void *stream)
{
    if (!xs || !ys || !zs || !seeds || !out_dev || nx < 1 || ny < 1 || nz < 1 || ns < 1)
        return PE_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    double *d = nullptr;
    const size_t nb = sizeof(double) * ((size_t)nx + ny + nz + 4 * (size_t)ns);
    if (cudaMalloc(&d, nb) != cudaSuccess) return PE_ERR_NOMEM;
    double *dx = d, *dy = dx + nx, *dz = dy + ny, *ds = dz + nz, *dw = ds + 3 * (size_t)ns;
    cudaError_t e = cudaMemcpyAsync(dx, xs, sizeof(double) * nx, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dy, ys, sizeof(double) * ny, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dz, zs, sizeof(double) * nz, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds, seeds, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if (weights) e = cudaMemcpyAsync(dw, weights, sizeof(double) * ns, cudaMemcpyHostToDevice, st);
        else e = cudaMemsetAsync(dw, 0, sizeof(double) * ns, st);
    }
    if (e == cudaSuccess) {
        const long long n = (long long)nx * ny * nz;
        k_label_cylinder<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dx, dy, dz, nx, ny, nz, R2, ds,
                                                                     dw, ns, out_dev);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    return e == cudaSuccess ? PE_OK : PE_ERR_CUDA;
}

// ------------------------------------------------------------------------------
// Allocation-free variant of the labeller, for callers that may not allocate
// device memory at all: a host application whose framework has reserved the
// whole device pool for its own caching allocator, or a pipeline stage that
// must not pay cudaMalloc/cudaFree's implicit device synchronisation in the
// middle of an acquisition loop. The grid coordinates, seeds and weights that
// pe_label_cylinder stages in a fresh cudaMalloc buffer are staged instead in
// this file-scope device array. Every device that loads the library holds
// the array (PE_NOALLOC_SCRATCH_BYTES) until the process exits.
//
// Contract:
//  - limits: nx + ny + nz <= PE_NOALLOC_MAX_COORDS, ns <= PE_NOALLOC_MAX_SEEDS;
//    larger requests return PE_ERR_INVALID with a message and touch nothing;
//  - the first call on a device looks the array up (cudaGetSymbolAddress,
//    with that device current) and caches the address; make that first call
//    before any stream capture on the device;
//  - all calls on a device share the one array and every call overwrites
//    it (the weights are zeroed when none are given): calls that can overlap
//    on the GPU (different streams, different host threads) race and must be
//    serialised by the caller;
//  - no cudaMalloc, cudaFree or other allocating routine is called.
// ------------------------------------------------------------------------------
namespace {

constexpr int NOALLOC_MAX_COORDS = PE_NOALLOC_MAX_COORDS;
constexpr int NOALLOC_MAX_SEEDS = PE_NOALLOC_MAX_SEEDS;
constexpr size_t NOALLOC_DOUBLES = (size_t)NOALLOC_MAX_COORDS + 4 * (size_t)NOALLOC_MAX_SEEDS;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];
static_assert(sizeof(g_noalloc_scratch) == PE_NOALLOC_SCRATCH_BYTES,
              "the array must be exactly the size the header documents");

// per-device address of the array, looked up once; atomic, so that first
// calls from several host threads do not race on the cache (they may each
// look it up, and all store the same address)
constexpr int NOALLOC_MAX_DEVICES = 64;
std::atomic<double *> g_noalloc_ptr[NOALLOC_MAX_DEVICES];

thread_local std::string g_noalloc_err;

int noalloc_fail(int code, const std::string &msg)
{
    g_noalloc_err = msg;
    return code;
}

}  // namespace

extern "C" const char *pe_label_cylinder_noalloc_error(void) { return g_noalloc_err.c_str(); }

extern "C" int pe_label_cylinder_noalloc(const double *xs, int nx, const double *ys, int ny,
                                         const double *zs, int nz, double R2, const double *seeds,
                                         const double *weights, int ns, int32_t *out_dev, void *stream)
{
    if (!xs || !ys || !zs || !seeds || !out_dev || nx < 1 || ny < 1 || nz < 1 || ns < 1)
        return noalloc_fail(PE_ERR_INVALID, "null pointer or empty axis / seed list");
    if ((long long)nx + ny + nz > NOALLOC_MAX_COORDS)
        return noalloc_fail(PE_ERR_INVALID, "nx + ny + nz = " + std::to_string((long long)nx + ny + nz) +
                                                " exceeds the allocation-free limit of " +
                                                std::to_string(NOALLOC_MAX_COORDS));
    if (ns > NOALLOC_MAX_SEEDS)
        return noalloc_fail(PE_ERR_INVALID, std::to_string(ns) + " seeds exceed the allocation-free limit of " +
                                                std::to_string(NOALLOC_MAX_SEEDS));
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return noalloc_fail(PE_ERR_CUDA, "no usable current device");
    double *d = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!d) {
        const cudaError_t e = cudaGetSymbolAddress((void **)&d, g_noalloc_scratch);
        if (e != cudaSuccess || !d)
            return noalloc_fail(PE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev].store(d, std::memory_order_release);
    }
    cudaStream_t st = (cudaStream_t)stream;
    double *dx = d, *dy = dx + nx, *dz = dy + ny, *ds = d + NOALLOC_MAX_COORDS, *dw = ds + 3 * (size_t)ns;
    cudaError_t e = cudaMemcpyAsync(dx, xs, sizeof(double) * nx, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dy, ys, sizeof(double) * ny, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dz, zs, sizeof(double) * nz, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds, seeds, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if (weights) e = cudaMemcpyAsync(dw, weights, sizeof(double) * ns, cudaMemcpyHostToDevice, st);
        else e = cudaMemsetAsync(dw, 0, sizeof(double) * ns, st);
    }
    if (e == cudaSuccess) {
        const long long n = (long long)nx * ny * nz;
        k_label_cylinder<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dx, dy, dz, nx, ny, nz, R2, ds, dw,
                                                                     ns, out_dev);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return noalloc_fail(PE_ERR_CUDA, std::string("labelling failed: ") + cudaGetErrorString(e));
    return PE_OK;
}
