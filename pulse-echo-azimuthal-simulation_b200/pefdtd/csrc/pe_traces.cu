// Batched trace post-processing on the device, in float64: the Hilbert
// envelope, the high-pass / mean detrend, the windowed envelope pick and the
// sweep driver's per-trace analysis.
//
//   envelope  |x + i H(x)|, H as scipy.signal.hilbert defines it (FFT of
//             length N, spectrum weights 1, 2, .., 2, 1): the imaginary part
//             is the circular convolution of x with the discrete Hilbert
//             kernel, whose closed form is
//               N even: g[m] = (2/N) cot(pi m / N) for odd m, 0 for even m
//               N odd:  g[m] = (cot(pi m / N) - (-1)^m / sin(pi m / N)) / N
//             (g[0] = 0). Used by pick_peak (sim/core/fdtd.py:976) and the
//             sweep analysis (sim/pipeline/sweep_runner.py:210).
//   detrend   filtfilt(b, a, x) with odd padding (scipy's default, the
//             reference's detrend_hp, sim/core/fdtd.py:943-948), or x - mean.
//   pick      argmax of the envelope in [lo, hi), edge flag and parabolic
//             refinement (sim/core/fdtd.py:977-984).
//   analyse   E1 / arrival / coda level / stability tail
//             (sim/pipeline/sweep_runner.py:209-225).
//
// A batch is `batch` traces packed back to back: trace i is samples
// off[i] .. off[i+1]-1. Window bounds, time steps and filter coefficients are
// computed on the host exactly as the reference's Python computes them.
#include <cmath>
#include <cstdint>
#include <algorithm>
#include <initializer_list>
#include <mutex>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "pefdtd.h"

namespace {

constexpr int ENV_T = 128;               // threads per envelope block
constexpr int ENV_R = 4;                 // outputs per thread (strided by ENV_T)
constexpr int ENV_TILE = ENV_T * ENV_R;  // outputs per block
constexpr int ENV_KC = 512;              // input samples staged per pass
constexpr int RED_T = 256;               // threads per reduction block
constexpr int FILT_MAX = 8;              // filter taps (order <= 7)
constexpr int PAD_MAX = 3 * FILT_MAX;    // scipy's default padlen bound

template <typename T>
__device__ __forceinline__ double rd(const T *p, long long i) { return (double)p[i]; }

// Discrete Hilbert kernel tap g[j mod N].
__device__ double hilbert_tap(long long j, long long N)
{
    long long m = j % N;
    if (m < 0) m += N;
    if (m == 0) return 0.0;
    double s, c;
    sincospi((double)m / (double)N, &s, &c);
    if ((N & 1) == 0) return (m & 1) ? (2.0 / (double)N) * (c / s) : 0.0;
    return ((c - ((m & 1) ? -1.0 : 1.0)) / s) / (double)N;
}

// One block: ENV_TILE outputs of one trace; the whole trace is swept in
// ENV_KC-sample passes, the kernel taps a pass needs staged beside them.
template <typename T>
__global__ void __launch_bounds__(ENV_T) k_envelope(const T *__restrict__ x, const long long *__restrict__ off,
                                                    const long long *__restrict__ tiles, double *__restrict__ env)
{
    __shared__ double xs[ENV_KC];
    __shared__ double gs[ENV_TILE + ENV_KC - 1];
    const long long tr = tiles[2 * blockIdx.x], n0 = tiles[2 * blockIdx.x + 1];
    const long long base = off[tr], N = off[tr + 1] - base;
    const int t = threadIdx.x;
    double acc[ENV_R];
#pragma unroll
    for (int r = 0; r < ENV_R; ++r) acc[r] = 0.0;
    for (long long k0 = 0; k0 < N; k0 += ENV_KC) {
        __syncthreads();
        for (int i = t; i < ENV_KC; i += ENV_T) xs[i] = (k0 + i < N) ? rd(x, base + k0 + i) : 0.0;
        // gs[u] = g[n0 - k0 - (ENV_KC - 1) + u]: output n0 + t + ENV_T r and
        // input k0 + kk meet at u = t + ENV_T r - kk + ENV_KC - 1
        const long long j0 = n0 - k0 - (ENV_KC - 1);
        for (int u = t; u < ENV_TILE + ENV_KC - 1; u += ENV_T) gs[u] = hilbert_tap(j0 + u, N);
        __syncthreads();
        const int kmax = (int)((N - k0) < ENV_KC ? (N - k0) : ENV_KC);
        const double *gp = gs + t + ENV_KC - 1;
#pragma unroll 4
        for (int kk = 0; kk < kmax; ++kk) {
            const double xv = xs[kk];
#pragma unroll
            for (int r = 0; r < ENV_R; ++r) acc[r] = fma(xv, gp[r * ENV_T - kk], acc[r]);
        }
    }
#pragma unroll
    for (int r = 0; r < ENV_R; ++r) {
        const long long n = n0 + t + (long long)ENV_T * r;
        if (n < N) env[base + n] = hypot(rd(x, base + n), acc[r]);
    }
}

struct Filt {
    double b[FILT_MAX], a[FILT_MAX], zi[FILT_MAX];
    int n;       // taps (len(b) == len(a)); the state has n - 1 entries
    int padlen;  // odd-extension length at each end
};

// scipy.signal.lfilter's transposed direct form II, one sample:
//   y = z0 + b0 x;  z_k = (z_{k+1} + x b_{k+1}) - y a_{k+1};  z_last = x b_n - y a_n
// (every product rounded separately: the file is built without contraction).
__device__ __forceinline__ double lfilter_step(const Filt &F, double *z, double xv)
{
    const double y = z[0] + F.b[0] * xv;
    for (int k = 0; k < F.n - 2; ++k) z[k] = (z[k + 1] + xv * F.b[k + 1]) - y * F.a[k + 1];
    z[F.n - 2] = xv * F.b[F.n - 1] - y * F.a[F.n - 1];
    return y;
}

// filtfilt with odd padding, one thread per trace. The forward pass keeps
// the samples of the trace in `out` and the right padding in registers;
// the backward pass then overwrites `out` in place (each sample is read
// before it is written), never needing the left padding's outputs.
template <typename T>
__global__ void k_filtfilt(const T *__restrict__ x, const long long *__restrict__ off, int batch, Filt F,
                           double *__restrict__ out)
{
    const int tr = blockIdx.x * blockDim.x + threadIdx.x;
    if (tr >= batch) return;
    const long long base = off[tr], N = off[tr + 1] - base;
    const int p = F.padlen;
    const double x0 = rd(x, base), xl = rd(x, base + N - 1);
    double z[FILT_MAX], tail[PAD_MAX];
    // ext[e] = 2 x[0] - x[p - e] (e < p); x[e - p]; 2 x[N-1] - x[N-2-(e-N-p)] (e >= N + p)
    const double e0 = p > 0 ? 2.0 * x0 - rd(x, base + p) : x0;
    for (int k = 0; k < F.n - 1; ++k) z[k] = F.zi[k] * e0;
    for (int e = 0; e < p; ++e) lfilter_step(F, z, 2.0 * x0 - rd(x, base + p - e));
    for (long long i = 0; i < N; ++i) out[base + i] = lfilter_step(F, z, rd(x, base + i));
    for (int j = 0; j < p; ++j) tail[j] = lfilter_step(F, z, 2.0 * xl - rd(x, base + N - 2 - j));
    const double y0 = p > 0 ? tail[p - 1] : out[base + N - 1];
    for (int k = 0; k < F.n - 1; ++k) z[k] = F.zi[k] * y0;
    for (int j = p - 1; j >= 0; --j) lfilter_step(F, z, tail[j]);
    for (long long i = N - 1; i >= 0; --i) out[base + i] = lfilter_step(F, z, out[base + i]);
}

// Block-wide reductions (RED_T threads).
struct ArgMax {
    double v;
    long long i;
};

// a beats b: NaN first (numpy's argmax returns the first NaN), then the
// larger value, then the lower index.
__device__ __forceinline__ bool beats(const ArgMax &a, const ArgMax &b)
{
    if (a.i < 0) return false;
    if (b.i < 0) return true;
    const bool na = a.v != a.v, nb = b.v != b.v;
    if (na != nb) return na;
    if (!na && a.v != b.v) return a.v > b.v;
    return a.i < b.i;
}

__device__ ArgMax block_argmax(ArgMax m)
{
    __shared__ double sv[RED_T / 32];
    __shared__ long long si[RED_T / 32];
    for (int o = 16; o > 0; o >>= 1) {
        ArgMax q{__shfl_down_sync(0xffffffffu, m.v, o), __shfl_down_sync(0xffffffffu, m.i, o)};
        if (beats(q, m)) m = q;
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        sv[w] = m.v;
        si[w] = m.i;
    }
    __syncthreads();
    ArgMax r{sv[0], si[0]};
    for (int k = 1; k < RED_T / 32; ++k) {
        ArgMax q{sv[k], si[k]};
        if (beats(q, r)) r = q;
    }
    return r;
}

__device__ double block_sum(double s)
{
    __shared__ double sh[RED_T / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = s;
    __syncthreads();
    double r = 0.0;
    for (int k = 0; k < RED_T / 32; ++k) r += sh[k];
    return r;
}

// max with NaN propagation (numpy's max)
__device__ __forceinline__ double nanmax2(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }

__device__ double block_max(double m)
{
    __shared__ double sh[RED_T / 32];
    for (int o = 16; o > 0; o >>= 1) m = nanmax2(m, __shfl_down_sync(0xffffffffu, m, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = m;
    __syncthreads();
    double r = sh[0];
    for (int k = 1; k < RED_T / 32; ++k) r = nanmax2(r, sh[k]);
    return r;
}

__device__ ArgMax window_argmax(const double *e, long long lo, long long hi)
{
    ArgMax m{0.0, -1};
    for (long long i = lo + threadIdx.x; i < hi; i += RED_T) {
        ArgMax q{e[i], i};
        if (beats(q, m)) m = q;
    }
    return block_argmax(m);
}

template <typename T>
__global__ void __launch_bounds__(RED_T) k_demean(const T *__restrict__ x, const long long *__restrict__ off,
                                                  double *__restrict__ out)
{
    const long long base = off[blockIdx.x], N = off[blockIdx.x + 1] - base;
    double s = 0.0;
    for (long long i = threadIdx.x; i < N; i += RED_T) s += rd(x, base + i);
    const double mean = block_sum(s) / (double)N;
    for (long long i = threadIdx.x; i < N; i += RED_T) out[base + i] = rd(x, base + i) - mean;
}

// win (lo, hi) per trace, hi > lo + 2 (the host settles the other case);
// out (t, peak, ok) per trace.
__global__ void __launch_bounds__(RED_T) k_pick(const double *__restrict__ env, const long long *__restrict__ off,
                                                const long long *__restrict__ win, const double *__restrict__ dt,
                                                double *__restrict__ out)
{
    const int tr = blockIdx.x;
    const long long base = off[tr], n = off[tr + 1] - base;
    const long long lo = win[2 * tr], hi = win[2 * tr + 1];
    const double *e = env + base;
    const ArgMax m = window_argmax(e, lo, hi);
    if (threadIdx.x != 0) return;
    const long long k = m.i - lo;
    const bool ok = 0 < k && k < (hi - lo - 1);
    double kk = (double)m.i;
    if (0 < m.i && m.i < n - 1) {
        const double y0 = e[m.i - 1], y1 = e[m.i], y2 = e[m.i + 1];
        const double d = (y0 - 2.0 * y1) + y2;
        kk = kk + (fabs(d) > 1e-30 ? (0.5 * (y0 - y2)) / d : 0.0);
    }
    out[3 * tr] = kk * dt[tr];
    out[3 * tr + 1] = m.v;
    out[3 * tr + 2] = ok ? 1.0 : 0.0;
}

// win (a, b, lo, hi) per trace with b > a; tf (dt, fs); out (E1, t1, coda, tail).
template <typename T>
__global__ void __launch_bounds__(RED_T) k_analyse(const T *__restrict__ x, const double *__restrict__ env,
                                                   const long long *__restrict__ off,
                                                   const long long *__restrict__ win, const double *__restrict__ tf,
                                                   double *__restrict__ out)
{
    const int tr = blockIdx.x;
    const long long base = off[tr], n = off[tr + 1] - base;
    const long long a = win[4 * tr], b = win[4 * tr + 1], lo = win[4 * tr + 2], hi = win[4 * tr + 3];
    const double dt = tf[2 * tr], fs = tf[2 * tr + 1];
    const double *e = env + base;
    const ArgMax m = window_argmax(e, a, b);
    const double E1 = m.v, t1 = (double)m.i * dt;
    double s = 0.0;
    for (long long i = lo + threadIdx.x; i < hi; i += RED_T) s += e[i] * e[i];
    const double ss = block_sum(s);
    const long long k_tail = (long long)((t1 + 3e-6) * fs);
    const bool have_tail = k_tail < n - 8;
    double mx = 0.0;
    if (have_tail)
        for (long long i = k_tail + threadIdx.x; i < n; i += RED_T) mx = nanmax2(mx, fabs(rd(x, base + i)));
    mx = block_max(mx);
    if (threadIdx.x != 0) return;
    const double mean = ss / (double)(hi > lo ? hi - lo : 0);
    out[4 * tr] = E1;
    out[4 * tr + 1] = t1;
    out[4 * tr + 2] = 20.0 * log10(sqrt(mean) / E1 + 1e-30);
    out[4 * tr + 3] = have_tail ? mx / (E1 > 1e-30 ? E1 : 1e-30) : NAN;
}

// Device copies of a call's small host arrays (offsets, windows, time
// steps) go to one grow-only buffer per device, held (mutex) for the whole
// call: every entry point synchronises its stream before returning, so the
// next call may reuse the buffer, and after the first calls on a device no
// call allocates or frees device memory (cudaFree would also synchronise
// the device).
struct StageArea {
    std::mutex mu;
    char *p = nullptr;
    size_t cap = 0;
};
constexpr int STAGE_DEVICES = 64;

struct Staged {
    std::unique_lock<std::mutex> lock;
};

cudaError_t stage(Staged &s, cudaStream_t st, std::initializer_list<std::pair<const void *, size_t>> parts,
                  std::vector<void *> &dst)
{
    static StageArea areas[STAGE_DEVICES];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= STAGE_DEVICES) return cudaErrorInvalidDevice;
    StageArea &a = areas[dev];
    s.lock = std::unique_lock<std::mutex>(a.mu);
    size_t total = 0;
    for (auto &q : parts) total += (q.second + 255) & ~size_t(255);
    if (total > a.cap) {
        // grow geometrically, so that a run of ever larger calls reallocates
        // (and synchronises the device in cudaFree) only O(log) times
        const size_t want = std::max(total, std::max(a.cap * 2, (size_t)1 << 16));
        if (a.p) cudaFree(a.p);
        a.p = nullptr;
        a.cap = 0;
        e = cudaMalloc(&a.p, want);
        if (e != cudaSuccess) {
            a.p = nullptr;
            return e;
        }
        a.cap = want;
    }
    size_t at = 0;
    for (auto &q : parts) {
        dst.push_back(a.p + at);
        if (q.second) {
            e = cudaMemcpyAsync(a.p + at, q.first, q.second, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return e;
        }
        at += (q.second + 255) & ~size_t(255);
    }
    return cudaSuccess;
}

bool valid_offsets(const int64_t *off, int batch, long long min_len)
{
    if (!off || batch < 1 || off[0] != 0) return false;
    for (int i = 0; i < batch; ++i)
        if (off[i + 1] - off[i] < min_len) return false;
    return true;
}

int finish(cudaError_t e, cudaStream_t st)
{
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? PE_OK : PE_ERR_CUDA;
}

}  // namespace

extern "C" int pe_trace_envelope(const void *x_dev, int32_t dtype, const int64_t *off, int32_t batch,
                                 double *env_dev, void *stream)
{
    if (!x_dev || !env_dev || (dtype != PE_F32 && dtype != PE_F64) || !valid_offsets(off, batch, 1))
        return PE_ERR_INVALID;
    std::vector<long long> tiles;
    for (int i = 0; i < batch; ++i)
        for (long long n0 = 0; n0 < off[i + 1] - off[i]; n0 += ENV_TILE) {
            tiles.push_back(i);
            tiles.push_back(n0);
        }
    if (tiles.size() / 2 > 0x7fffffffULL) return PE_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    Staged s;
    std::vector<void *> d;
    cudaError_t e = stage(s, st, {{off, sizeof(int64_t) * (batch + 1)}, {tiles.data(), sizeof(long long) * tiles.size()}}, d);
    if (e == cudaSuccess) {
        const unsigned nb = (unsigned)(tiles.size() / 2);
        const long long *doff = (const long long *)d[0], *dtl = (const long long *)d[1];
        if (dtype == PE_F32) k_envelope<float><<<nb, ENV_T, 0, st>>>((const float *)x_dev, doff, dtl, env_dev);
        else k_envelope<double><<<nb, ENV_T, 0, st>>>((const double *)x_dev, doff, dtl, env_dev);
    }
    return finish(e, st);
}

extern "C" int pe_trace_detrend(const void *x_dev, int32_t dtype, const int64_t *off, int32_t batch,
                                const double *b, const double *a, int32_t n_ab, const double *zi, int32_t padlen,
                                double *out_dev, void *stream)
{
    if (!x_dev || !out_dev || (dtype != PE_F32 && dtype != PE_F64)) return PE_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    if (n_ab == 0) {
        if (!valid_offsets(off, batch, 1)) return PE_ERR_INVALID;
        Staged s;
        std::vector<void *> d;
        cudaError_t e = stage(s, st, {{off, sizeof(int64_t) * (batch + 1)}}, d);
        if (e == cudaSuccess) {
            const long long *doff = (const long long *)d[0];
            if (dtype == PE_F32) k_demean<float><<<batch, RED_T, 0, st>>>((const float *)x_dev, doff, out_dev);
            else k_demean<double><<<batch, RED_T, 0, st>>>((const double *)x_dev, doff, out_dev);
        }
        return finish(e, st);
    }
    if (!b || !a || !zi || n_ab < 2 || n_ab > FILT_MAX || padlen < 0 || padlen > PAD_MAX ||
        !valid_offsets(off, batch, (long long)padlen + 1))
        return PE_ERR_INVALID;
    Filt F{};
    for (int k = 0; k < n_ab; ++k) {
        F.b[k] = b[k];
        F.a[k] = a[k];
    }
    for (int k = 0; k < n_ab - 1; ++k) F.zi[k] = zi[k];
    F.n = n_ab;
    F.padlen = padlen;
    Staged s;
    std::vector<void *> d;
    cudaError_t e = stage(s, st, {{off, sizeof(int64_t) * (batch + 1)}}, d);
    if (e == cudaSuccess) {
        const long long *doff = (const long long *)d[0];
        const unsigned nb = (unsigned)((batch + 63) / 64);
        if (dtype == PE_F32) k_filtfilt<float><<<nb, 64, 0, st>>>((const float *)x_dev, doff, batch, F, out_dev);
        else k_filtfilt<double><<<nb, 64, 0, st>>>((const double *)x_dev, doff, batch, F, out_dev);
    }
    return finish(e, st);
}

extern "C" int pe_trace_pick(const double *env_dev, const int64_t *off, int32_t batch, const int64_t *win,
                             const double *dt, double *out_dev, void *stream)
{
    if (!env_dev || !win || !dt || !out_dev || !valid_offsets(off, batch, 1)) return PE_ERR_INVALID;
    for (int i = 0; i < batch; ++i)
        if (win[2 * i] < 0 || win[2 * i + 1] > off[i + 1] - off[i] || win[2 * i + 1] <= win[2 * i] + 2)
            return PE_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    Staged s;
    std::vector<void *> d;
    cudaError_t e = stage(s, st,
                          {{off, sizeof(int64_t) * (batch + 1)}, {win, sizeof(int64_t) * 2 * batch},
                           {dt, sizeof(double) * batch}},
                          d);
    if (e == cudaSuccess)
        k_pick<<<batch, RED_T, 0, st>>>(env_dev, (const long long *)d[0], (const long long *)d[1],
                                        (const double *)d[2], out_dev);
    return finish(e, st);
}

extern "C" int pe_trace_analyse(const void *x_dev, int32_t dtype, const double *env_dev, const int64_t *off,
                                int32_t batch, const int64_t *win, const double *dt_fs, double *out_dev,
                                void *stream)
{
    if (!x_dev || !env_dev || !win || !dt_fs || !out_dev || (dtype != PE_F32 && dtype != PE_F64) ||
        !valid_offsets(off, batch, 1))
        return PE_ERR_INVALID;
    for (int i = 0; i < batch; ++i) {
        const int64_t n = off[i + 1] - off[i];
        const int64_t *w = win + 4 * i;
        if (w[0] < 0 || w[1] > n || w[1] <= w[0] || w[2] < 0 || w[3] > n) return PE_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    Staged s;
    std::vector<void *> d;
    cudaError_t e = stage(s, st,
                          {{off, sizeof(int64_t) * (batch + 1)}, {win, sizeof(int64_t) * 4 * batch},
                           {dt_fs, sizeof(double) * 2 * batch}},
                          d);
    if (e == cudaSuccess) {
        const long long *doff = (const long long *)d[0], *dwin = (const long long *)d[1];
        const double *dtf = (const double *)d[2];
        if (dtype == PE_F32)
            k_analyse<float><<<batch, RED_T, 0, st>>>((const float *)x_dev, env_dev, doff, dwin, dtf, out_dev);
        else
            k_analyse<double><<<batch, RED_T, 0, st>>>((const double *)x_dev, env_dev, doff, dwin, dtf, out_dev);
    }
    return finish(e, st);
}
