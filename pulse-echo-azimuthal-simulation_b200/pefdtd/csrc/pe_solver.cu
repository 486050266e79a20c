// C ABI and runtime of the B200 FDTD solver (include/pefdtd.h).
//
// The runtime owns everything a solve needs besides the nine state fields:
// the flagged label volume, tables, damping, probe lists, the receiver
// sample buffer of one chunk and a device step counter. A chunk of
// `chunk_steps` steps (stress + velocity launch per step, then one trace
// reduction and a counter advance) is captured once as a CUDA graph and
// replayed; the kernels read the global step from the device counter, so the
// same graph serves every chunk. This is the reference's Python step loop
// (sim/core/fdtd.py:1786-1816) moved onto the device.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "pe_kernels.cuh"
#include "pe_kernels_tiled.cuh"
#include "pe_kernels_tma.cuh"
#include "pe_kernels_pair.cuh"
#include "pe_adjoint.cuh"
#include "pefdtd.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define PE_CUDA(expr)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(e_ == cudaErrorMemoryAllocation ? PE_ERR_NOMEM : PE_ERR_CUDA,      \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));               \
    } while (0)

// Device buffers of solvers, batches and the host entry come from a
// per-device cache: a freed buffer is kept and handed out again for a request
// of the same size (rounded to 256 bytes), so that creating and destroying
// solves of the same shapes allocates and frees nothing after the first
// time. cudaMalloc and cudaFree synchronise the device, and cudaFree of a
// large buffer can stall for much longer. At most POOL_KEEP bytes are kept
// per device (beyond that a freed buffer goes back to the driver);
// pe_release_cached_memory empties the cache. Buffers are returned only
// after the work using them has finished (their owners synchronise first).
constexpr int POOL_DEVICES = 64;
constexpr size_t POOL_KEEP = (size_t)8 << 30;
struct DevPool {
    std::mutex mu;
    std::unordered_map<void *, size_t> live;   // handed out: size
    std::multimap<size_t, void *> idle;        // kept for reuse
    size_t idle_bytes = 0;
};
DevPool g_pool[POOL_DEVICES];

DevPool *pool_of_current()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= POOL_DEVICES) return nullptr;
    return &g_pool[dev];
}

template <typename P>
int dev_alloc(P **p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    bytes = (bytes + 255) & ~size_t(255);
    DevPool *pool = pool_of_current();
    if (pool) {
        std::lock_guard<std::mutex> g(pool->mu);
        auto it = pool->idle.find(bytes);
        if (it != pool->idle.end()) {
            *p = (P *)it->second;
            pool->idle_bytes -= bytes;
            pool->idle.erase(it);
            pool->live[(void *)*p] = bytes;
            return PE_OK;
        }
    }
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(PE_ERR_NOMEM, std::string("cudaMalloc(") + std::to_string(bytes) +
                                      "): " + cudaGetErrorString(e));
    }
    if (pool) {
        std::lock_guard<std::mutex> g(pool->mu);
        pool->live[(void *)*p] = bytes;
    }
    return PE_OK;
}

// return a dev_alloc buffer to the cache of the device it came from (the
// current device's cache is searched first, then the others)
void dev_free(void *p)
{
    if (!p) return;
    DevPool *cur = pool_of_current();
    for (int d = -1; d < POOL_DEVICES; ++d) {
        DevPool *pool = d < 0 ? cur : &g_pool[d];
        if (!pool || (d >= 0 && pool == cur)) continue;
        std::lock_guard<std::mutex> g(pool->mu);
        auto it = pool->live.find(p);
        if (it == pool->live.end()) continue;
        const size_t bytes = it->second;
        pool->live.erase(it);
        if (pool->idle_bytes + bytes <= POOL_KEEP) {
            pool->idle.emplace(bytes, p);
            pool->idle_bytes += bytes;
        } else {
            cudaFree(p);
        }
        return;
    }
    cudaFree(p);
}

void pool_release_all()
{
    for (DevPool &pool : g_pool) {
        std::lock_guard<std::mutex> g(pool.mu);
        for (auto &kv : pool.idle) cudaFree(kv.second);
        pool.idle.clear();
        pool.idle_bytes = 0;
    }
}

int dtype_size(int dtype) { return dtype == PE_F64 ? 8 : 4; }

struct TileShape {
    int tx, ty;
};

}  // namespace

struct PeSolver {
    PeConfig cfg{};
    long long ncell = 0;
    int esize = 4;
    // device buffers owned by the solver
    uint16_t *lab = nullptr;
    void *c21 = nullptr, *rho = nullptr;
    float *dz = nullptr, *dy = nullptr, *dx = nullptr, *dvol = nullptr;
    long long *src_idx = nullptr;
    void *src_w = nullptr;
    int n_src = 0;
    long long *rec_cell = nullptr;
    int *rec_pos = nullptr;
    void *rec_w = nullptr;
    long long *grp_off = nullptr;
    int *ent_group = nullptr;   // group of each receiver entry (caller order)
    int n_rec = 0, n_groups = 0;
    void *rec_val = nullptr;
    void *wavelet = nullptr;
    long long nt_wav = 0;
    long long *step = nullptr;
    // execution
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t gexec = nullptr;
    PeState gstate{};
    void *gtraces = nullptr;
    int chunk = 200;
    int tx = 32, ty = 8;        // simple-kernel tile
    int variant = PE_KERNEL_TILED;
    int zc_s = 0, zc_v = 0;     // planes per z-march of the stress / velocity launches
    long long launches = 0;
    int *status = nullptr;      // device status word
    bool tma = false;           // TMA-fed kernels in use for the current state
    bool tma_capable = false;   // grid rows are 16-byte multiples and the driver encodes maps
    PeState mstate{};           // state the tensor maps were encoded for
    bool maps_ok = false;
    pe::TmapsStress ms{};
    pe::TmapsVelocity mv{};
    // FP32 pair-column kernels (the default where the grid allows them)
    float *tab36 = nullptr;     // (n_mat, 36) column-split stiffness
    float *rinv = nullptr;      // (n_mat,) reciprocal densities (FP32 pair velocity kernel)
    double *grad_rep = nullptr; // (nrep, n_mat, 21) replicas the adjoint's gradient sums spread over
    int nrep = 0;
    bool pair_capable = false;  // FP32, rows of 16-byte multiples, maps encodable, smem fits
    bool pair = false;          // pair kernels in use for the current state
    bool solo = false;          // in a batch: fills the GPU alone, so runs its own launches
    int zc_ps = 0, zc_pv = 0;   // planes per z-march of the pair launches
    pe::TmapsPairStress mps{};
    pe::TmapsPairVelocity mpv{};

    ~PeSolver()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        if (stream) cudaStreamDestroy(stream);
        void *bufs[] = {lab, c21, rho, dz, dy, dx, dvol, src_idx, src_w, rec_cell,
                        rec_pos, rec_w, grp_off, rec_val, wavelet, step, status, ent_group, tab36, rinv, grad_rep};
        for (void *b : bufs)
            if (b) dev_free(b);
    }
};

namespace {

template <typename T>
pe::StepArgs<T> make_args(const PeSolver *S, const PeState *st, int k)
{
    pe::StepArgs<T> A{};
    for (int i = 0; i < 3; ++i) A.v[i] = (T *)st->v[i];
    for (int i = 0; i < 6; ++i) A.s[i] = (T *)st->s[i];
    A.lab = S->lab;
    A.c21 = (const T *)S->c21;
    A.rho = (const T *)S->rho;
    A.rinv = S->rinv;
    A.dz = S->dz;
    A.dy = S->dy;
    A.dx = S->dx;
    A.dvol = S->dvol;
    A.nz = S->cfg.nz;
    A.ny = S->cfg.ny;
    A.nx = S->cfg.nx;
    A.sy = S->cfg.nx;
    A.sz = (long long)S->cfg.nx * S->cfg.ny;
    for (int j = 0; j < 4; ++j) A.c[j] = j < S->cfg.n_coeffs ? (T)S->cfg.coeffs[j] : T(0);
    A.nc = S->cfg.n_coeffs;
    A.inv_h = (T)(1.0 / S->cfg.h);
    A.dt = (T)S->cfg.dt;
    A.dt_h = (T)(S->cfg.dt / S->cfg.h);
    A.src_idx = S->src_idx;
    A.src_w = (const T *)S->src_w;
    A.n_src = S->n_src;
    A.wavelet = (const T *)S->wavelet;
    A.rec_cell = S->rec_cell;
    A.rec_pos = S->rec_pos;
    A.n_rec = S->n_rec;
    A.rec_val = (T *)S->rec_val;
    A.rec_kind = S->cfg.record;
    A.rec_damped = S->cfg.damped_record;
    A.step = S->step;
    A.k = k;
    A.zc = S->zc_s;
    A.status = S->status;
    A.dense = S->variant == PE_KERNEL_DENSE;
    return A;
}

template <typename T, int TX, int TY>
void launch_simple_stress(pe::StepArgs<T> A, int zc, cudaStream_t st)
{
    A.zc = zc;
    dim3 grid((A.nx + TX - 1) / TX, (A.ny + TY - 1) / TY, (A.nz + zc - 1) / zc);
    pe::k_stress<T, TX, TY><<<grid, dim3(TX, TY, 1), 0, st>>>(A);
}
template <typename T, int TX, int TY>
void launch_simple_velocity(pe::StepArgs<T> A, int zc, cudaStream_t st)
{
    A.zc = zc;
    dim3 grid((A.nx + TX - 1) / TX, (A.ny + TY - 1) / TY, (A.nz + zc - 1) / zc);
    pe::k_velocity<T, TX, TY><<<grid, dim3(TX, TY, 1), 0, st>>>(A);
}

template <typename T>
void launch_stress(const PeSolver *S, const pe::StepArgs<T> &A0, cudaStream_t st)
{
    if (S->variant == PE_KERNEL_SIMPLE || S->variant == PE_KERNEL_DENSE) {
        if (S->ty == 8) launch_simple_stress<T, 32, 8>(A0, S->zc_s, st);
        else launch_simple_stress<T, 32, 4>(A0, S->zc_s, st);
        return;
    }
    pe::StepArgs<T> A = A0;
    if constexpr (std::is_same<T, float>::value) {
        if (S->pair) {
            A.zc = S->zc_ps;
            // stress tiles update columns [30 bx - 1, 30 bx + 29)
            dim3 grid((A.nx + pe::PS_OX) / pe::PS_OX, (A.ny + pe::PS_OY - 1) / pe::PS_OY, (A.nz + A.zc - 1) / A.zc);
            const int nm = S->cfg.n_mat;
            const size_t sm = pe::stress_pair_smem(nm);
            const bool ts = pe::pair_tab_in_smem(nm);
            if (A.nc == 4 && ts) pe::k_stress_pair<4, true><<<grid, pe::PS_N, sm, st>>>(S->mps, A, S->tab36, nm);
            else if (A.nc == 4) pe::k_stress_pair<4, false><<<grid, pe::PS_N, sm, st>>>(S->mps, A, S->tab36, nm);
            else if (ts) pe::k_stress_pair<0, true><<<grid, pe::PS_N, sm, st>>>(S->mps, A, S->tab36, nm);
            else pe::k_stress_pair<0, false><<<grid, pe::PS_N, sm, st>>>(S->mps, A, S->tab36, nm);
            return;
        }
    }
    A.zc = S->zc_s;
    dim3 grid((A.nx + pe::TS_OX - 1) / pe::TS_OX, (A.ny + pe::TS_OY - 1) / pe::TS_OY,
              (A.nz + A.zc - 1) / A.zc);
    if (S->tma) {
        pe::k_stress_tma<T><<<grid, dim3(pe::TB_X, pe::TB_Y, 1), pe::stress_tma_smem<T>(S->cfg.n_mat), st>>>(
            S->ms, A, S->cfg.n_mat);
        return;
    }
    pe::k_stress_t<T><<<grid, dim3(pe::TB_X, pe::TB_Y, 1), pe::stress_tiled_smem<T>(S->cfg.n_mat), st>>>(
        A, S->cfg.n_mat);
}

template <typename T>
void launch_velocity(const PeSolver *S, const pe::StepArgs<T> &A0, cudaStream_t st)
{
    if (S->variant == PE_KERNEL_SIMPLE || S->variant == PE_KERNEL_DENSE) {
        if (S->ty == 8) launch_simple_velocity<T, 32, 8>(A0, S->zc_v, st);
        else launch_simple_velocity<T, 32, 4>(A0, S->zc_v, st);
        return;
    }
    pe::StepArgs<T> A = A0;
    if constexpr (std::is_same<T, float>::value) {
        if (S->pair) {
            A.zc = S->zc_pv;
            dim3 grid((A.nx + pe::PV_OX - 1) / pe::PV_OX, (A.ny + pe::PV_OY - 1) / pe::PV_OY, (A.nz + A.zc - 1) / A.zc);
            const size_t sm = pe::velocity_pair_smem(S->cfg.n_mat);
            if (A.nc == 4)
                pe::k_velocity_pair<4><<<grid, pe::PV_N, sm, st>>>(S->mpv, A, S->cfg.n_mat);
            else
                pe::k_velocity_pair<0><<<grid, pe::PV_N, sm, st>>>(S->mpv, A, S->cfg.n_mat);
            return;
        }
    }
    A.zc = S->zc_v;
    dim3 grid((A.nx + pe::TB_X - 1) / pe::TB_X, (A.ny + pe::TB_Y - 1) / pe::TB_Y,
              (A.nz + A.zc - 1) / A.zc);
    if (S->tma) {
        pe::k_velocity_tma<T><<<grid, dim3(pe::TB_X, pe::TB_Y, 1), pe::velocity_tma_smem<T>(S->cfg.n_mat),
                                 st>>>(S->mv, A, S->cfg.n_mat);
        return;
    }
    pe::k_velocity_t<T><<<grid, dim3(pe::TB_X, pe::TB_Y, 1), pe::velocity_tiled_smem<T>(S->cfg.n_mat),
                          st>>>(A, S->cfg.n_mat);
}

template <typename T>
int launch_chunk_t(PeSolver *S, const PeState *st, void *traces, int len)
{
    for (int k = 0; k < len; ++k) {
        pe::StepArgs<T> A = make_args<T>(S, st, k);
        launch_stress<T>(S, A, S->stream);
        launch_velocity<T>(S, A, S->stream);
        S->launches += 2;
    }
    if (S->n_groups > 0) {
        const int nthr = len * S->n_groups;
        pe::k_reduce_traces<T><<<(nthr + 127) / 128, 128, 0, S->stream>>>(
            (const T *)S->rec_val, (const T *)S->rec_w, S->grp_off, S->n_groups, S->n_rec, len,
            S->step, (T *)traces);
        S->launches += 1;
    }
    pe::k_step_advance<<<1, 1, 0, S->stream>>>(S->step, len);
    S->launches += 1;
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

int launch_chunk(PeSolver *S, const PeState *st, void *traces, int len)
{
    return S->cfg.dtype == PE_F64 ? launch_chunk_t<double>(S, st, traces, len)
                                  : launch_chunk_t<float>(S, st, traces, len);
}

bool same_state(const PeState &a, const PeState &b)
{
    for (int i = 0; i < 3; ++i)
        if (a.v[i] != b.v[i]) return false;
    for (int i = 0; i < 6; ++i)
        if (a.s[i] != b.s[i]) return false;
    return true;
}

// Planes per z-march: the split of nz into chunks that minimises
// waves x (planes per chunk + per-chunk start-up planes), where a wave is
// one block on every SM slot the occupancy allows.
int pick_zchunk(int nz, long long tiles, int slots, int startup)
{
    int best_zc = nz;
    double best = 1e300;
    for (int nch = 1; nch <= nz; ++nch) {
        const int zc = (nz + nch - 1) / nch;
        const int real = (nz + zc - 1) / zc;
        if (zc < 4 && nch > 1) break;
        const long long blocks = tiles * real;
        const long long waves = (blocks + slots - 1) / slots;
        const double cost = (double)waves * (zc + startup);
        if (cost < best - 1e-9) {
            best = cost;
            best_zc = zc;
        }
    }
    return best_zc;
}

template <typename K>
int occupancy_slots(K kernel, int threads, size_t smem)
{
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess || per < 1)
        per = 1;
    return nsm * per;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 3-D map (x fastest) of one (nz, ny, nx) field with a (bw, bh, 1) box;
// out-of-grid box elements read as zero
int encode_box(CUtensorMap *m, const void *base, CUtensorMapDataType dt, int es, const PeConfig &c,
               int bw, int bh)
{
    const cuuint64_t dims[3] = {(cuuint64_t)c.nx, (cuuint64_t)c.ny, (cuuint64_t)c.nz};
    const cuuint64_t strides[2] = {(cuuint64_t)c.nx * es, (cuuint64_t)c.nx * c.ny * es};
    const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode_fn()(m, dt, 3, const_cast<void *>(base), dims, strides, box, estr,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(PE_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return PE_OK;
}

template <typename T>
int configure_kernels(PeSolver *S)
{
    const PeConfig &c = S->cfg;
    if (S->variant == PE_KERNEL_SIMPLE || S->variant == PE_KERNEL_DENSE) {
        const long long tiles = (long long)((c.nx + S->tx - 1) / S->tx) * ((c.ny + S->ty - 1) / S->ty);
        const int slots = occupancy_slots(pe::k_stress<T, 32, 8>, 32 * S->ty, 0);
        S->zc_s = c.z_chunk > 0 ? c.z_chunk : pick_zchunk(c.nz, tiles, slots, 2);
        S->zc_v = c.z_chunk > 0 ? c.z_chunk : pick_zchunk(c.nz, tiles, slots, 2);
        return PE_OK;
    }
    // allow every launch up to the device's opt-in shared memory per block
    int dev = 0, optin = 0;
    PE_CUDA(cudaGetDevice(&dev));
    PE_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t need_s = pe::stress_tiled_smem<T>(c.n_mat), need_v = pe::velocity_tiled_smem<T>(c.n_mat);
    if (need_s > (size_t)optin || need_v > (size_t)optin)
        return fail(PE_ERR_UNSUPPORTED, "tiled kernels need " + std::to_string(need_s) +
                                            " B of shared memory per block; device offers " +
                                            std::to_string(optin));
    PE_CUDA(cudaFuncSetAttribute(pe::k_stress_t<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    PE_CUDA(cudaFuncSetAttribute(pe::k_velocity_t<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    const long long ts = (long long)((c.nx + pe::TS_OX - 1) / pe::TS_OX) * ((c.ny + pe::TS_OY - 1) / pe::TS_OY);
    const long long tv = (long long)((c.nx + pe::TB_X - 1) / pe::TB_X) * ((c.ny + pe::TB_Y - 1) / pe::TB_Y);
    int ss = occupancy_slots(pe::k_stress_t<T>, pe::TB_X * pe::TB_Y, need_s);
    int sv = occupancy_slots(pe::k_velocity_t<T>, pe::TB_X * pe::TB_Y, need_v);
    // TMA path: rows must be whole 16-byte units (box x-origins are multiples of 4 elements)
    const size_t tms = pe::stress_tma_smem<T>(c.n_mat), tmv = pe::velocity_tma_smem<T>(c.n_mat);
    S->tma_capable = c.nx % 4 == 0 && tms <= (size_t)optin && tmv <= (size_t)optin &&
                     encode_fn() != nullptr;
    if (S->tma_capable) {
        PE_CUDA(cudaFuncSetAttribute(pe::k_stress_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        PE_CUDA(cudaFuncSetAttribute(pe::k_velocity_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        ss = occupancy_slots(pe::k_stress_tma<T>, pe::TB_X * pe::TB_Y, tms);
        sv = occupancy_slots(pe::k_velocity_tma<T>, pe::TB_X * pe::TB_Y, tmv);
    }
    S->zc_s = c.z_chunk > 0 ? c.z_chunk : pick_zchunk(c.nz, ts, ss, 4);
    S->zc_v = c.z_chunk > 0 ? c.z_chunk : pick_zchunk(c.nz, tv, sv, 3);
    if constexpr (std::is_same<T, float>::value) {
        const size_t ps = pe::stress_pair_smem(c.n_mat), pv = pe::velocity_pair_smem(c.n_mat);
        S->pair_capable = S->variant == PE_KERNEL_TILED && c.nx % 4 == 0 && ps <= (size_t)optin &&
                          pv <= (size_t)optin && encode_fn() != nullptr;
        if (S->pair_capable) {
            // the attribute belongs to the kernel, not to this solve: allow the
            // device maximum so that solves with other table sizes can coexist
            PE_CUDA(cudaFuncSetAttribute(pe::k_stress_pair<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            PE_CUDA(cudaFuncSetAttribute(pe::k_stress_pair<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            PE_CUDA(cudaFuncSetAttribute(pe::k_stress_pair<0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            PE_CUDA(cudaFuncSetAttribute(pe::k_stress_pair<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            PE_CUDA(cudaFuncSetAttribute(pe::k_velocity_pair<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            PE_CUDA(cudaFuncSetAttribute(pe::k_velocity_pair<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            const long long tps = (long long)((c.nx + pe::PS_OX) / pe::PS_OX) * ((c.ny + pe::PS_OY - 1) / pe::PS_OY);
            const long long tpv = (long long)((c.nx + pe::PV_OX - 1) / pe::PV_OX) * ((c.ny + pe::PV_OY - 1) / pe::PV_OY);
            const int sps = occupancy_slots(pe::k_stress_pair<4, true>, pe::PS_N, ps);
            const int spv = occupancy_slots(pe::k_velocity_pair<4>, pe::PV_N, pv);
            S->zc_ps = c.z_chunk > 0 ? c.z_chunk : pick_zchunk(c.nz, tps, sps, 3);
            S->zc_pv = c.z_chunk > 0 ? c.z_chunk : pick_zchunk(c.nz, tpv, spv, 2);
        }
    }
    return PE_OK;
}

// Tensor maps of the nine fields (and the damping volume) for the TMA
// kernels; re-encoded whenever the caller's state buffers change. Falls back
// to the cp.async kernels when a buffer is not 16-byte aligned.
int ensure_maps(PeSolver *S, const PeState *st)
{
    if (!S->tma_capable && !S->pair_capable) {
        S->tma = false;
        S->pair = false;
        return PE_OK;
    }
    if (S->maps_ok && same_state(S->mstate, *st)) return PE_OK;
    const PeConfig &c = S->cfg;
    const int es = S->esize;
    bool aligned = !S->dvol || ((uintptr_t)S->dvol % 16) == 0;
    for (int i = 0; i < 3; ++i) aligned = aligned && ((uintptr_t)st->v[i] % 16) == 0;
    for (int i = 0; i < 6; ++i) aligned = aligned && ((uintptr_t)st->s[i] % 16) == 0;
    S->mstate = *st;
    S->maps_ok = true;
    S->tma = aligned && S->tma_capable;
    S->pair = aligned && S->pair_capable;
    if (!aligned) return PE_OK;
    const CUtensorMapDataType dt = es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    int rc;
    if (S->pair) {
        for (int f = 0; f < 3; ++f)
            if ((rc = encode_box(&S->mps.vt[f], st->v[f], dt, es, c, pe::PS_VW, pe::PS_VH))) return rc;
        for (int f = 0; f < 6; ++f)
            if ((rc = encode_box(&S->mps.sc[f], st->s[f], dt, es, c, pe::PS_SW, pe::PS_SH))) return rc;
        const int pvf[5] = {0, 1, 3, 4, 5};
        for (int f = 0; f < 5; ++f)
            if ((rc = encode_box(&S->mpv.st[f], st->s[pvf[f]], dt, es, c, pe::PV_TW, pe::PV_TH))) return rc;
        for (int f = 0; f < 3; ++f)
            if ((rc = encode_box(&S->mpv.vc[f], st->v[f], dt, es, c, pe::PV_OX, pe::PV_OY))) return rc;
        if (S->dvol) {
            if ((rc = encode_box(&S->mps.dv, S->dvol, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, c, pe::PS_SW, pe::PS_SH))) return rc;
            if ((rc = encode_box(&S->mpv.dv, S->dvol, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, c, pe::PV_OX, pe::PV_OY))) return rc;
        } else {
            std::memset(&S->mps.dv, 0, sizeof(S->mps.dv));
            std::memset(&S->mpv.dv, 0, sizeof(S->mpv.dv));
        }
    }
    if (!S->tma) return PE_OK;
    for (int f = 0; f < 3; ++f)
        if ((rc = encode_box(&S->ms.vt[f], st->v[f], dt, es, c, pe::KS_VW, pe::KS_VH))) return rc;
    for (int f = 0; f < 6; ++f)
        if ((rc = encode_box(&S->ms.sc[f], st->s[f], dt, es, c, pe::KS_SW, pe::KS_SH))) return rc;
    const int vf[5] = {0, 1, 3, 4, 5};
    for (int f = 0; f < 5; ++f)
        if ((rc = encode_box(&S->mv.st[f], st->s[vf[f]], dt, es, c, pe::KV_SW, pe::KV_SH))) return rc;
    for (int f = 0; f < 3; ++f)
        if ((rc = encode_box(&S->mv.vc[f], st->v[f], dt, es, c, pe::KV_CW, pe::KV_CH))) return rc;
    if (S->dvol) {
        if ((rc = encode_box(&S->ms.dv, S->dvol, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, c, pe::KS_SW, pe::KS_SH))) return rc;
        if ((rc = encode_box(&S->mv.dv, S->dvol, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, c, pe::KV_CW, pe::KV_CH))) return rc;
    } else {
        std::memset(&S->ms.dv, 0, sizeof(S->ms.dv));
        std::memset(&S->mv.dv, 0, sizeof(S->mv.dv));
    }
    return PE_OK;
}

}  // namespace

extern "C" {

int pe_abi_version(void) { return PE_ABI_VERSION; }

const char *pe_last_error(void) { return g_err.c_str(); }

int pe_solver_create(const PeConfig *cfg, const PeMedium *md, const PeProbe *pr, PeSolver **out)
{
    if (!cfg || !md || !pr || !out) return fail(PE_ERR_INVALID, "null argument");
    *out = nullptr;
    const PeConfig &c = *cfg;
    if (c.nz < 1 || c.ny < 1 || c.nx < 1)
        return fail(PE_ERR_INVALID, "grid dimensions must be positive");
    if ((long long)c.ny * c.nx >= (1LL << 31))
        return fail(PE_ERR_UNSUPPORTED, "an xy plane must hold fewer than 2^31 cells");
    if (c.n_coeffs < 1 || c.n_coeffs > 4)
        return fail(PE_ERR_INVALID,
                    "supports order <= 8 (" + std::to_string(c.n_coeffs) +
                        " coefficients given): the kernels carry +/-4 taps per axis");
    if (c.dtype != PE_F32 && c.dtype != PE_F64) return fail(PE_ERR_INVALID, "dtype must be F32 or F64");
    if (c.record < 0 || c.record > 3) return fail(PE_ERR_INVALID, "record must be 0..3");
    const bool dense = c.variant == PE_KERNEL_DENSE;
    if (dense && (long long)c.n_mat != (long long)c.nz * c.ny * c.nx)
        return fail(PE_ERR_INVALID, "per-cell media (PE_KERNEL_DENSE) need one table row per cell: n_mat = " +
                                        std::to_string((long long)c.nz * c.ny * c.nx));
    if (!dense && (c.n_mat < 1 || c.n_mat > PE_MAX_MATERIALS))
        return fail(PE_ERR_INVALID, "n_mat must lie in [1, " + std::to_string(PE_MAX_MATERIALS) + "]");
    if (!(c.h > 0) || !(c.dt > 0)) return fail(PE_ERR_INVALID, "h and dt must be positive");
    if ((!dense && !md->labels_dev) || !md->ctab || !md->rho)
        return fail(PE_ERR_INVALID, "labels_dev, ctab and rho are required");
    const bool any_sp = md->sponge_z || md->sponge_y || md->sponge_x;
    const bool all_sp = md->sponge_z && md->sponge_y && md->sponge_x;
    if (any_sp && !all_sp) return fail(PE_ERR_INVALID, "give all three sponge profiles or none");
    if (pr->n_src < 0 || pr->n_groups < 0) return fail(PE_ERR_INVALID, "negative probe sizes");
    if (pr->n_src > 0 && (!pr->src_idx || !pr->src_w)) return fail(PE_ERR_INVALID, "source arrays missing");
    if (pr->n_groups > 0 && (!pr->rec_off || !pr->rec_idx || !pr->rec_w))
        return fail(PE_ERR_INVALID, "receiver arrays missing");

    std::unique_ptr<PeSolver> S(new PeSolver());
    S->cfg = c;
    S->ncell = (long long)c.nz * c.ny * c.nx;
    S->esize = dtype_size(c.dtype);
    S->chunk = c.chunk_steps > 0 ? c.chunk_steps : 200;
    if (c.variant != PE_KERNEL_TILED && c.variant != PE_KERNEL_SIMPLE && c.variant != PE_KERNEL_COLUMN &&
        c.variant != PE_KERNEL_DENSE)
        return fail(PE_ERR_INVALID, "variant must be PE_KERNEL_TILED, PE_KERNEL_SIMPLE, PE_KERNEL_COLUMN "
                                    "or PE_KERNEL_DENSE");
    S->variant = c.variant;
    if (c.tile_x > 0 && c.tile_y > 0) {
        const TileShape ok[] = {{32, 8}, {32, 4}};
        bool found = false;
        for (auto t : ok) found |= (t.tx == c.tile_x && t.ty == c.tile_y);
        if (!found || (S->variant != PE_KERNEL_SIMPLE && S->variant != PE_KERNEL_DENSE))
            return fail(PE_ERR_UNSUPPORTED, "tile shape not compiled in for this kernel variant");
        S->tx = c.tile_x;
        S->ty = c.tile_y;
    }
    {
        int rc0 = c.dtype == PE_F64 ? configure_kernels<double>(S.get()) : configure_kernels<float>(S.get());
        if (rc0) return rc0;
    }
    const long long ncell = S->ncell;
    const int es = S->esize;

    // ---- probe lists (host side: validate, dedupe, sort)
    std::vector<long long> sidx;
    std::vector<char> swb;
    {
        std::map<long long, int> last;  // cell -> last entry
        for (int k = 0; k < pr->n_src; ++k) {
            const long long q = pr->src_idx[k];
            if (q < 0 || q >= ncell)
                return fail(PE_ERR_INVALID, "source cell index " + std::to_string(q) + " outside the grid");
            last[q] = k;
        }
        for (auto &kv : last) {
            sidx.push_back(kv.first);
            const char *w = (const char *)pr->src_w + (size_t)kv.second * es;
            swb.insert(swb.end(), w, w + es);
        }
    }
    S->n_src = (int)sidx.size();
    std::vector<long long> roff, rcell_sorted;
    std::vector<int> rpos_sorted;
    S->n_groups = pr->n_groups;
    long long n_rec = 0;
    if (pr->n_groups > 0) {
        if (pr->rec_off[0] != 0) return fail(PE_ERR_INVALID, "rec_off[0] must be 0");
        for (int g = 0; g < pr->n_groups; ++g)
            if (pr->rec_off[g + 1] < pr->rec_off[g]) return fail(PE_ERR_INVALID, "rec_off must be non-decreasing");
        n_rec = pr->rec_off[pr->n_groups];
        if (n_rec > (1LL << 30)) return fail(PE_ERR_INVALID, "too many receiver entries");
        std::vector<std::pair<long long, int>> ent((size_t)n_rec);
        for (long long e = 0; e < n_rec; ++e) {
            const long long q = pr->rec_idx[e];
            if (q < 0 || q >= ncell)
                return fail(PE_ERR_INVALID, "receiver cell index " + std::to_string(q) + " outside the grid");
            ent[(size_t)e] = {q, (int)e};
        }
        std::sort(ent.begin(), ent.end());
        for (auto &p : ent) {
            rcell_sorted.push_back(p.first);
            rpos_sorted.push_back(p.second);
        }
        roff.assign(pr->rec_off, pr->rec_off + pr->n_groups + 1);
    }
    S->n_rec = (int)n_rec;

    PE_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    PE_CUDA(cudaEventCreateWithFlags(&S->ev_in, cudaEventDisableTiming));
    PE_CUDA(cudaEventCreateWithFlags(&S->ev_out, cudaEventDisableTiming));
    cudaStream_t st = S->stream;

    int rc;
    if ((rc = dev_alloc(&S->lab, sizeof(uint16_t) * ncell))) return rc;
    if ((rc = dev_alloc(&S->c21, (size_t)es * pe::C21_STRIDE * c.n_mat))) return rc;
    if ((rc = dev_alloc(&S->rho, (size_t)es * c.n_mat))) return rc;
    if ((rc = dev_alloc(&S->step, sizeof(long long)))) return rc;
    if ((rc = dev_alloc(&S->status, sizeof(int)))) return rc;
    PE_CUDA(cudaMemsetAsync(S->status, 0, sizeof(int), st));

    // labels: copy + range check, then mark source / receiver cells (per-cell
    // media: no material bits, only the flags)
    if (dense) PE_CUDA(cudaMemsetAsync(S->lab, 0, sizeof(uint16_t) * ncell, st));
    unsigned long long *nbad = nullptr;
    if ((rc = dev_alloc(&nbad, sizeof(unsigned long long)))) return rc;
    PE_CUDA(cudaMemsetAsync(nbad, 0, sizeof(unsigned long long), st));
    if (!dense)
        pe::k_labels_copy<<<(unsigned)((ncell + 255) / 256), 256, 0, st>>>(md->labels_dev, S->lab, ncell,
                                                                           c.n_mat, nbad);
    unsigned long long bad = 0;
    PE_CUDA(cudaMemcpyAsync(&bad, nbad, sizeof(bad), cudaMemcpyDeviceToHost, st));
    PE_CUDA(cudaStreamSynchronize(st));
    dev_free(nbad);
    if (bad)
        return fail(PE_ERR_INVALID, std::to_string(bad) + " cells carry a material index >= n_mat (" +
                                        std::to_string(c.n_mat) + "): label has no table row");

    // tables
    {
        void *c36 = nullptr;
        if ((rc = dev_alloc(&c36, (size_t)es * 36 * c.n_mat))) return rc;
        PE_CUDA(cudaMemcpyAsync(c36, md->ctab, (size_t)es * 36 * c.n_mat, cudaMemcpyHostToDevice, st));
        if (c.dtype == PE_F64)
            pe::k_c36_to_c21<double><<<(c.n_mat + 127) / 128, 128, 0, st>>>((const double *)c36, (double *)S->c21, c.n_mat);
        else
            pe::k_c36_to_c21<float><<<(c.n_mat + 127) / 128, 128, 0, st>>>((const float *)c36, (float *)S->c21, c.n_mat);
        PE_CUDA(cudaMemcpyAsync(S->rho, md->rho, (size_t)es * c.n_mat, cudaMemcpyHostToDevice, st));
        if (c.dtype == PE_F32 && !dense) {   // the pair kernels' tables
            if ((rc = dev_alloc(&S->tab36, sizeof(float) * pe::TAB36 * c.n_mat))) return rc;
            pe::k_c21_to_tab36<<<(c.n_mat + 127) / 128, 128, 0, st>>>((const float *)S->c21, S->tab36, c.n_mat);
            if ((rc = dev_alloc(&S->rinv, sizeof(float) * c.n_mat))) return rc;
            pe::k_rho_inv<<<(c.n_mat + 127) / 128, 128, 0, st>>>((const float *)S->rho, S->rinv, c.n_mat);
        }
        PE_CUDA(cudaStreamSynchronize(st));
        dev_free(c36);
    }
    if (all_sp) {
        if ((rc = dev_alloc(&S->dz, sizeof(float) * c.nz))) return rc;
        if ((rc = dev_alloc(&S->dy, sizeof(float) * c.ny))) return rc;
        if ((rc = dev_alloc(&S->dx, sizeof(float) * c.nx))) return rc;
        PE_CUDA(cudaMemcpyAsync(S->dz, md->sponge_z, sizeof(float) * c.nz, cudaMemcpyHostToDevice, st));
        PE_CUDA(cudaMemcpyAsync(S->dy, md->sponge_y, sizeof(float) * c.ny, cudaMemcpyHostToDevice, st));
        PE_CUDA(cudaMemcpyAsync(S->dx, md->sponge_x, sizeof(float) * c.nx, cudaMemcpyHostToDevice, st));
    }
    if (md->damp_volume_dev) {
        if ((rc = dev_alloc(&S->dvol, sizeof(float) * ncell))) return rc;
        PE_CUDA(cudaMemcpyAsync(S->dvol, md->damp_volume_dev, sizeof(float) * ncell, cudaMemcpyDeviceToDevice, st));
    }
    // probe
    if ((rc = dev_alloc(&S->src_idx, sizeof(long long) * std::max<size_t>(1, sidx.size())))) return rc;
    if ((rc = dev_alloc(&S->src_w, (size_t)es * std::max<size_t>(1, sidx.size())))) return rc;
    if (!sidx.empty()) {
        PE_CUDA(cudaMemcpyAsync(S->src_idx, sidx.data(), sizeof(long long) * sidx.size(), cudaMemcpyHostToDevice, st));
        PE_CUDA(cudaMemcpyAsync(S->src_w, swb.data(), swb.size(), cudaMemcpyHostToDevice, st));
        pe::k_labels_flag<<<(S->n_src + 127) / 128, 128, 0, st>>>(S->lab, S->src_idx, S->n_src, pe::LAB_SRC);
    }
    const size_t nr = (size_t)std::max<long long>(1, n_rec);
    if ((rc = dev_alloc(&S->rec_cell, sizeof(long long) * nr))) return rc;
    if ((rc = dev_alloc(&S->rec_pos, sizeof(int) * nr))) return rc;
    if ((rc = dev_alloc(&S->rec_w, (size_t)es * nr))) return rc;
    if ((rc = dev_alloc(&S->grp_off, sizeof(long long) * (S->n_groups + 1)))) return rc;
    if ((rc = dev_alloc(&S->rec_val, (size_t)es * nr * S->chunk))) return rc;
    PE_CUDA(cudaMemsetAsync(S->rec_val, 0, (size_t)es * nr * S->chunk, st));
    if (n_rec > 0) {
        PE_CUDA(cudaMemcpyAsync(S->rec_cell, rcell_sorted.data(), sizeof(long long) * n_rec, cudaMemcpyHostToDevice, st));
        PE_CUDA(cudaMemcpyAsync(S->rec_pos, rpos_sorted.data(), sizeof(int) * n_rec, cudaMemcpyHostToDevice, st));
        PE_CUDA(cudaMemcpyAsync(S->rec_w, pr->rec_w, (size_t)es * n_rec, cudaMemcpyHostToDevice, st));
        pe::k_labels_flag<<<(unsigned)((n_rec + 127) / 128), 128, 0, st>>>(S->lab, S->rec_cell, (int)n_rec, pe::LAB_REC);
    }
    if (S->n_groups > 0)
        PE_CUDA(cudaMemcpyAsync(S->grp_off, roff.data(), sizeof(long long) * (S->n_groups + 1), cudaMemcpyHostToDevice, st));
    {
        std::vector<int> eg((size_t)std::max<long long>(1, n_rec), 0);
        for (int g = 0; g < S->n_groups; ++g)
            for (long long e = roff[g]; e < roff[g + 1]; ++e) eg[(size_t)e] = g;
        if ((rc = dev_alloc(&S->ent_group, sizeof(int) * eg.size()))) return rc;
        PE_CUDA(cudaMemcpyAsync(S->ent_group, eg.data(), sizeof(int) * eg.size(), cudaMemcpyHostToDevice, st));
        PE_CUDA(cudaStreamSynchronize(st));
    }
    PE_CUDA(cudaStreamSynchronize(st));
    PE_CUDA(cudaGetLastError());
    *out = S.release();
    return PE_OK;
}

int pe_solver_set_wavelet(PeSolver *S, const void *wavelet, int64_t nt)
{
    if (!S || (nt > 0 && !wavelet) || nt < 0) return fail(PE_ERR_INVALID, "bad wavelet");
    if (S->wavelet) {
        dev_free(S->wavelet);
        S->wavelet = nullptr;
    }
    int rc = dev_alloc(&S->wavelet, (size_t)S->esize * std::max<int64_t>(1, nt));
    if (rc) return rc;
    if (nt > 0)
        PE_CUDA(cudaMemcpyAsync(S->wavelet, wavelet, (size_t)S->esize * nt, cudaMemcpyHostToDevice, S->stream));
    PE_CUDA(cudaStreamSynchronize(S->stream));
    S->nt_wav = nt;
    return PE_OK;
}

int pe_solver_run(PeSolver *S, const PeState *state, void *traces, int64_t b, int64_t e, void *stream)
{
    if (!S || !state) return fail(PE_ERR_INVALID, "null argument");
    if (b < 0 || e < b) return fail(PE_ERR_INVALID, "need 0 <= step_begin <= step_end");
    if (e > S->nt_wav && S->n_src > 0)
        return fail(PE_ERR_INVALID, "step_end " + std::to_string(e) + " beyond the wavelet (" +
                                        std::to_string(S->nt_wav) + " samples)");
    if (S->n_groups > 0 && !traces) return fail(PE_ERR_INVALID, "traces buffer required");
    for (int i = 0; i < 3; ++i)
        if (!state->v[i]) return fail(PE_ERR_INVALID, "state field missing");
    for (int i = 0; i < 6; ++i)
        if (!state->s[i]) return fail(PE_ERR_INVALID, "state field missing");
    S->launches = 0;
    {
        const int rc0 = ensure_maps(S, state);
        if (rc0) return rc0;
    }
    if (e == b) return PE_OK;
    cudaStream_t user = (cudaStream_t)stream;
    PE_CUDA(cudaEventRecord(S->ev_in, user));
    PE_CUDA(cudaStreamWaitEvent(S->stream, S->ev_in, 0));
    pe::k_step_set<<<1, 1, 0, S->stream>>>(S->step, b);
    S->launches += 1;
    int64_t n = b;
    while (n < e) {
        const int len = (int)std::min<int64_t>(S->chunk, e - n);
        if (len == S->chunk) {
            if (!S->gexec || !same_state(S->gstate, *state) || S->gtraces != traces) {
                if (S->gexec) {
                    cudaGraphExecDestroy(S->gexec);
                    S->gexec = nullptr;
                }
                cudaGraph_t g = nullptr;
                PE_CUDA(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
                const long long before = S->launches;
                int rc = launch_chunk(S, state, traces, len);
                cudaError_t ce = cudaStreamEndCapture(S->stream, &g);
                if (rc) return rc;
                if (ce != cudaSuccess) return fail(PE_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
                S->launches = before;
                ce = cudaGraphInstantiate(&S->gexec, g, 0);
                cudaGraphDestroy(g);
                if (ce != cudaSuccess) return fail(PE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
                S->gstate = *state;
                S->gtraces = traces;
            }
            PE_CUDA(cudaGraphLaunch(S->gexec, S->stream));
            S->launches += 2LL * len + (S->n_groups > 0 ? 1 : 0) + 1;
        } else {
            int rc = launch_chunk(S, state, traces, len);
            if (rc) return rc;
        }
        n += len;
    }
    PE_CUDA(cudaEventRecord(S->ev_out, S->stream));
    PE_CUDA(cudaStreamWaitEvent(user, S->ev_out, 0));
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

int64_t pe_solver_launch_count(const PeSolver *S) { return S ? S->launches : -1; }

}  // extern "C"

namespace {

// grad: the table the step's gradient sums go to (adj->grad, or the
// solver's replicas when nrep > 1)
template <typename T>
int adjoint_step_t(PeSolver *S, const PeAdjoint *adj, int64_t n, const void *residual, cudaStream_t st,
                   double *grad, int nrep)
{
    const PeConfig &c = S->cfg;
    pe::AdjArgs<T> A{};
    const long long ncell = S->ncell;
    for (int i = 0; i < 3; ++i) {
        A.lv[i] = (T *)adj->lv[i];
        A.vp[i] = (const T *)adj->v_prev[i];
        A.u[i] = (T *)adj->scratch + (size_t)i * ncell;
    }
    for (int i = 0; i < 6; ++i) {
        A.ls[i] = (T *)adj->ls[i];
        A.g[i] = (T *)adj->scratch + (size_t)(3 + i) * ncell;
        A.t[i] = (T *)adj->scratch + (size_t)(9 + i) * ncell;
    }
    for (int k = 0; k < 18; ++k) A.w[k] = (T *)adj->scratch + (size_t)(15 + k) * ncell;
    A.lab = S->lab;
    A.c21 = (const T *)S->c21;
    A.rho = (const T *)S->rho;
    A.rinv = S->rinv;
    A.dz = S->dz;
    A.dy = S->dy;
    A.dx = S->dx;
    A.dvol = S->dvol;
    A.nz = c.nz;
    A.ny = c.ny;
    A.nx = c.nx;
    A.sy = c.nx;
    A.sz = (long long)c.nx * c.ny;
    for (int j = 0; j < 4; ++j) A.c[j] = j < c.n_coeffs ? (T)c.coeffs[j] : T(0);
    A.nc = c.n_coeffs;
    A.inv_h = (T)(1.0 / c.h);
    A.dt = (T)c.dt;
    A.dt_h = (T)(c.dt / c.h);
    A.grad = grad;
    A.grad_rep = nrep;
    A.n_mat = c.n_mat;
    if (c.nz > 65535) return fail(PE_ERR_UNSUPPORTED, "the adjoint launches one block row per z plane (nz <= 65535)");
    if (S->n_rec > 0 && residual) {
        const T *row = (const T *)residual + (size_t)n * S->n_groups;
        pe::k_adj_inject<T><<<(S->n_rec + 127) / 128, 128, 0, st>>>(A, S->rec_cell, S->rec_pos, (const T *)S->rec_w,
                                                                     S->ent_group, S->n_rec, row, c.record,
                                                                     c.damped_record);
    }
    // cell kernels: 32 x 8 blocks over (x tiles, y tiles, z planes)
    const dim3 ab(pe::ADJ_BX, pe::ADJ_BY, 1);
    const dim3 ag((unsigned)((c.nx + pe::ADJ_BX - 1) / pe::ADJ_BX), (unsigned)((c.ny + pe::ADJ_BY - 1) / pe::ADJ_BY),
                  (unsigned)c.nz);
    pe::k_adj_vel_u<T><<<ag, ab, 0, st>>>(A);
    pe::k_adj_vel<T><<<ag, ab, 0, st>>>(A);
    pe::k_adj_strain<T><<<ag, ab, 0, st>>>(A);
    pe::k_adj_stress<T><<<ag, ab, 0, st>>>(A);
    pe::k_adj_velfin<T><<<ag, ab, 0, st>>>(A);
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

}  // namespace

extern "C" {

int pe_solver_adjoint_step(PeSolver *S, const PeAdjoint *adj, int64_t n, const void *residual, void *stream)
{
    if (!S || !adj || !adj->scratch || !adj->grad) return fail(PE_ERR_INVALID, "null adjoint argument");
    if (S->variant == PE_KERNEL_DENSE)
        return fail(PE_ERR_UNSUPPORTED, "the adjoint runs on material tables, not per-cell media");
    for (int i = 0; i < 3; ++i)
        if (!adj->lv[i] || !adj->v_prev[i]) return fail(PE_ERR_INVALID, "adjoint velocity buffers missing");
    for (int i = 0; i < 6; ++i)
        if (!adj->ls[i]) return fail(PE_ERR_INVALID, "adjoint stress buffers missing");
    if (n < 0) return fail(PE_ERR_INVALID, "negative step");
    cudaStream_t st = (cudaStream_t)stream;
    return S->cfg.dtype == PE_F64 ? adjoint_step_t<double>(S, adj, n, residual, st, adj->grad, 1)
                                  : adjoint_step_t<float>(S, adj, n, residual, st, adj->grad, 1);
}

int pe_solver_adjoint_segment(PeSolver *S, const PeState *state, const PeAdjoint *adj0, void *v_hist,
                              int64_t a, int64_t b, const void *residual, void *stream)
{
    if (!S || !state || !adj0 || !v_hist || !adj0->scratch || !adj0->grad)
        return fail(PE_ERR_INVALID, "null adjoint argument");
    if (S->variant == PE_KERNEL_DENSE)
        return fail(PE_ERR_UNSUPPORTED, "the adjoint runs on material tables, not per-cell media");
    for (int i = 0; i < 3; ++i)
        if (!adj0->lv[i] || !state->v[i]) return fail(PE_ERR_INVALID, "adjoint velocity buffers missing");
    for (int i = 0; i < 6; ++i)
        if (!adj0->ls[i] || !state->s[i]) return fail(PE_ERR_INVALID, "adjoint stress buffers missing");
    if (a < 0 || b <= a) return fail(PE_ERR_INVALID, "need 0 <= step_begin < step_end");
    if (S->n_src > 0 && b > S->nt_wav) return fail(PE_ERR_INVALID, "step_end beyond the wavelet");
    int rc = ensure_maps(S, state);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t fb = (size_t)S->esize * (size_t)S->ncell;   // bytes of one field
    char *hist = (char *)v_hist;
    // recompute the segment, keeping v before every step
    for (int64_t n = a; n < b; ++n) {
        for (int c = 0; c < 3; ++c)
            PE_CUDA(cudaMemcpyAsync(hist + ((size_t)(n - a) * 3 + c) * fb, state->v[c], fb,
                                    cudaMemcpyDeviceToDevice, st));
        pe::k_step_set<<<1, 1, 0, st>>>(S->step, n);
        if (S->cfg.dtype == PE_F64) {
            pe::StepArgs<double> A = make_args<double>(S, state, 0);
            launch_stress<double>(S, A, st);
            launch_velocity<double>(S, A, st);
        } else {
            pe::StepArgs<float> A = make_args<float>(S, state, 0);
            launch_stress<float>(S, A, st);
            launch_velocity<float>(S, A, st);
        }
    }
    PE_CUDA(cudaGetLastError());
    // then the adjoint steps backwards through it, the gradient sums spread
    // over replicas of the table (allocated zero on the first segment, left
    // zero by the fold)
    const long long glen = (long long)S->cfg.n_mat * 21;
    if (!S->grad_rep) {
        const int nrep = (int)std::max(1LL, std::min(64LL, (64LL << 20) / (glen * 8)));
        if ((rc = dev_alloc(&S->grad_rep, sizeof(double) * (size_t)(glen * nrep)))) return rc;
        PE_CUDA(cudaMemsetAsync(S->grad_rep, 0, sizeof(double) * (size_t)(glen * nrep), st));
        S->nrep = nrep;
    }
    PeAdjoint adj = *adj0;
    for (int64_t n = b - 1; n >= a; --n) {
        for (int c = 0; c < 3; ++c) adj.v_prev[c] = hist + ((size_t)(n - a) * 3 + c) * fb;
        rc = S->cfg.dtype == PE_F64 ? adjoint_step_t<double>(S, &adj, n, residual, st, S->grad_rep, S->nrep)
                                    : adjoint_step_t<float>(S, &adj, n, residual, st, S->grad_rep, S->nrep);
        if (rc) {
            // the replicas hold partial sums of this segment: clear them, so
            // that a later segment's fold starts from zero as it assumes
            cudaMemsetAsync(S->grad_rep, 0, sizeof(double) * (size_t)(glen * S->nrep), st);
            return rc;
        }
    }
    pe::k_grad_fold<<<(unsigned)((glen + 255) / 256), 256, 0, st>>>(S->grad_rep, S->nrep, glen, adj0->grad);
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

int pe_solver_status(PeSolver *S)
{
    if (!S) return fail(PE_ERR_INVALID, "null solver");
    int st = 0;
    PE_CUDA(cudaStreamSynchronize(S->stream));
    PE_CUDA(cudaMemcpy(&st, S->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) {
        PE_CUDA(cudaMemset(S->status, 0, sizeof(int)));
        return fail(st == PE_ERR_TIMEOUT ? PE_ERR_TIMEOUT : PE_ERR_CUDA,
                    "a bounded device-side wait gave up; the results of the affected steps are invalid");
    }
    return PE_OK;
}

int pe_solver_profile(PeSolver *S, const PeState *state, int n_steps, float *ms_out, void *stream)
{
    if (!S || !state || !ms_out || n_steps < 1) return fail(PE_ERR_INVALID, "bad profile request");
    if (S->n_src > 0 && S->nt_wav < n_steps) return fail(PE_ERR_INVALID, "wavelet shorter than n_steps");
    cudaStream_t user = (cudaStream_t)stream;
    cudaEvent_t ev[3];
    for (auto &e : ev) PE_CUDA(cudaEventCreate(&e));
    PE_CUDA(cudaEventRecord(S->ev_in, user));
    PE_CUDA(cudaStreamWaitEvent(S->stream, S->ev_in, 0));
    {
        const int rc0 = ensure_maps(S, state);
        if (rc0) return rc0;
    }
    pe::k_step_set<<<1, 1, 0, S->stream>>>(S->step, 0);
    float tot_s = 0.f, tot_v = 0.f;
    const int saved_chunk = S->chunk;
    for (int n = 0; n < n_steps; ++n) {
        // one step at a time with events around each kernel (no graph)
        PE_CUDA(cudaEventRecord(ev[0], S->stream));
        if (S->cfg.dtype == PE_F64) {
            pe::StepArgs<double> A = make_args<double>(S, state, 0);
            launch_stress<double>(S, A, S->stream);
            PE_CUDA(cudaEventRecord(ev[1], S->stream));
            launch_velocity<double>(S, A, S->stream);
        } else {
            pe::StepArgs<float> A = make_args<float>(S, state, 0);
            launch_stress<float>(S, A, S->stream);
            PE_CUDA(cudaEventRecord(ev[1], S->stream));
            launch_velocity<float>(S, A, S->stream);
        }
        PE_CUDA(cudaEventRecord(ev[2], S->stream));
        pe::k_step_advance<<<1, 1, 0, S->stream>>>(S->step, 1);
        PE_CUDA(cudaEventSynchronize(ev[2]));
        float a = 0.f, b = 0.f;
        PE_CUDA(cudaEventElapsedTime(&a, ev[0], ev[1]));
        PE_CUDA(cudaEventElapsedTime(&b, ev[1], ev[2]));
        tot_s += a;
        tot_v += b;
    }
    S->chunk = saved_chunk;
    for (auto &e : ev) cudaEventDestroy(e);
    PE_CUDA(cudaEventRecord(S->ev_out, S->stream));
    PE_CUDA(cudaStreamWaitEvent(user, S->ev_out, 0));
    ms_out[0] = tot_s / n_steps;
    ms_out[1] = tot_v / n_steps;
    return PE_OK;
}

int pe_solver_destroy(PeSolver *S)
{
    if (S) {
        // the solve's buffers go back to the cache for reuse: every stream's
        // work on them (runs, adjoint segments on the caller's stream) must
        // be finished first, as cudaFree's implicit synchronisation ensured
        cudaDeviceSynchronize();
        delete S;
    }
    return PE_OK;
}

}  // extern "C"

namespace {

// Device buffers of pe_forward_host kept between calls, per device
// (grow-only): a call of the same or a smaller size allocates and frees
// nothing, and so does not pay cudaMalloc / cudaFree (whose synchronisation
// and mapping of a 377 MB state dominate a short call). Released by
// pe_release_cached_memory.
struct HostEntryBufs {
    std::mutex mu;
    void *lab = nullptr, *dvol = nullptr, *fields = nullptr, *traces = nullptr;
    size_t c_lab = 0, c_dvol = 0, c_fields = 0, c_traces = 0;
    cudaStream_t st = nullptr;
};
constexpr int HOST_ENTRY_DEVICES = 64;
HostEntryBufs g_host_bufs[HOST_ENTRY_DEVICES];

int grow(void **p, size_t *cap, size_t need)
{
    if (need <= *cap) return PE_OK;
    if (*p) dev_free(*p);
    *p = nullptr;
    *cap = 0;
    const int rc = dev_alloc(p, need);
    if (rc == PE_OK) *cap = need;
    return rc;
}

}  // namespace

extern "C" {

int pe_forward_host(const PeConfig *cfg, const uint16_t *labels_host, const float *damp_host,
                    const PeMedium *medium, const PeProbe *probe, const void *wavelet_host,
                    int64_t nt, void *traces_host)
{
    if (!cfg || !labels_host || !medium || !probe || (nt > 0 && !traces_host))
        return fail(PE_ERR_INVALID, "null argument");
    const long long ncell = (long long)cfg->nz * cfg->ny * cfg->nx;
    if (ncell <= 0) return fail(PE_ERR_INVALID, "grid dimensions must be positive");
    const int es = dtype_size(cfg->dtype);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= HOST_ENTRY_DEVICES)
        return fail(PE_ERR_CUDA, "no usable current device");
    HostEntryBufs &H = g_host_bufs[dev];
    std::lock_guard<std::mutex> guard(H.mu);   // calls on one device share the buffers: one at a time
    PeSolver *S = nullptr;
    int rc = PE_OK;
    PeMedium md = *medium;
    PeState state{};
    const size_t tr_bytes = (size_t)es * (size_t)std::max<int64_t>(1, nt) * std::max(1, probe->n_groups);
    do {
        if ((rc = grow(&H.lab, &H.c_lab, sizeof(uint16_t) * ncell))) break;
        if (damp_host && (rc = grow(&H.dvol, &H.c_dvol, sizeof(float) * ncell))) break;
        if ((rc = grow(&H.fields, &H.c_fields, (size_t)es * 9 * ncell))) break;
        if ((rc = grow(&H.traces, &H.c_traces, tr_bytes))) break;
        cudaError_t ce = cudaSuccess;
        if (!H.st) ce = cudaStreamCreateWithFlags(&H.st, cudaStreamNonBlocking);
        cudaStream_t st = H.st;
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(H.lab, labels_host, sizeof(uint16_t) * ncell, cudaMemcpyHostToDevice, st);
        if (ce == cudaSuccess && damp_host)
            ce = cudaMemcpyAsync(H.dvol, damp_host, sizeof(float) * ncell, cudaMemcpyHostToDevice, st);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(H.fields, 0, (size_t)es * 9 * ncell, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) {
            rc = fail(PE_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(ce));
            break;
        }
        md.labels_dev = (const uint16_t *)H.lab;
        md.damp_volume_dev = damp_host ? (const float *)H.dvol : nullptr;
        if ((rc = pe_solver_create(cfg, &md, probe, &S))) break;
        if ((rc = pe_solver_set_wavelet(S, wavelet_host, nt))) break;
        for (int i = 0; i < 3; ++i) state.v[i] = (char *)H.fields + (size_t)es * i * ncell;
        for (int i = 0; i < 6; ++i) state.s[i] = (char *)H.fields + (size_t)es * (3 + i) * ncell;
        if ((rc = pe_solver_run(S, &state, H.traces, 0, nt, st))) break;
        if (probe->n_groups > 0 && nt > 0) {
            ce = cudaMemcpyAsync(traces_host, H.traces, (size_t)es * nt * probe->n_groups, cudaMemcpyDeviceToHost, st);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
            if (ce != cudaSuccess) {
                rc = fail(PE_ERR_CUDA, std::string("download: ") + cudaGetErrorString(ce));
                break;
            }
        }
    } while (0);
    if (H.st) cudaStreamSynchronize(H.st);
    if (S) pe_solver_destroy(S);
    return rc;
}

void pe_release_cached_memory(void)
{
    for (HostEntryBufs &H : g_host_bufs) {
        std::lock_guard<std::mutex> guard(H.mu);
        if (H.st) cudaStreamSynchronize(H.st);
        void *bufs[] = {H.lab, H.dvol, H.fields, H.traces};
        for (void *b : bufs)
            if (b) dev_free(b);
        H.lab = H.dvol = H.fields = H.traces = nullptr;
        H.c_lab = H.c_dvol = H.c_fields = H.c_traces = 0;
        if (H.st) cudaStreamDestroy(H.st);
        H.st = nullptr;
    }
    pool_release_all();
}

}  // extern "C"

// ===================================================================== batches
// A batch advances many independent solves (any grid sizes, one dtype) with
// one stress and one velocity launch per step for all of them, replayed as
// captured CUDA graphs of `chunk` steps. Each solve keeps its own solver-owned
// buffers (a PeSolver); the batch owns the shared step counter and status
// word, the per-solve argument blocks and tensor maps in device memory, and
// the work-item lists.
struct PeBatch {
    std::vector<PeSolver *> solves;
    int dtype = PE_F32, esize = 4;
    long long *step = nullptr;
    int *status = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    void *descs = nullptr;
    pe::TmapsStress *maps_s = nullptr;
    pe::TmapsVelocity *maps_v = nullptr;
    int *nmats = nullptr;
    pe::BatchItem *items_s = nullptr, *items_v = nullptr;
    int n_items_s = 0, n_items_v = 0;
    int grid_s = 1, grid_v = 1;
    size_t smem_s = 0, smem_v = 0;
    int z_chunk = 0, chunk = 200;
    std::vector<PeState> states;
    std::vector<void *> traces;
    bool uploaded = false;
    cudaGraphExec_t gexec = nullptr;
    long long launches = 0;
    long long graph_launches = 0;   // kernels in one captured chunk
    bool tma_batch = true;          // the batched TMA kernels fit this batch
    // FP32 batches of solves whose rows are 16-byte multiples run the
    // pair-column kernels
    bool pair_batch = false;
    bool pair_ts = false;           // every batched table fits shared memory
    bool pair_nc4 = true;           // every batched solve has four coefficients
    pe::TmapsPairStress *pmaps_s = nullptr;
    pe::TmapsPairVelocity *pmaps_v = nullptr;
    const float **tabs = nullptr;
    // persistent mode: one cooperative launch per graph chunk runs every step
    // of the batched pair solves (k_pair_batch_persistent)
    bool persistent = false;
    unsigned *bar = nullptr;        // grid barrier counter, zeroed before each launch
    int grid_p = 1;
    size_t smem_p = 0;

    ~PeBatch()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (stream) cudaStreamSynchronize(stream);
        for (PeSolver *s : solves) pe_solver_destroy(s);
        void *bufs[] = {step, status, descs, maps_s, maps_v, nmats, items_s, items_v, pmaps_s, pmaps_v, tabs, bar};
        for (void *b : bufs)
            if (b) dev_free(b);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// Whether solve S runs inside the batched TMA launches (else its own pair).
bool batched(const PeBatch *B, const PeSolver *S)
{
    return B->pair_batch ? (S->pair_capable && !S->solo) : (B->tma_batch && S->tma_capable);
}

// Pair-kernel layout of an FP32 batch: work items, grids and shared memory.
int batch_layout_pair(PeBatch *B, int nsm, int optin, std::vector<pe::BatchItem> &is,
                      std::vector<pe::BatchItem> &iv)
{
    int max_mat = 1;
    B->pair_nc4 = true;
    // a solve whose own launches fill every SM at least twice runs them
    // inside the batch's graph; the shared persistent launches are for the
    // solves too small to fill the GPU alone
    for (PeSolver *S : B->solves) {
        const PeConfig &c = S->cfg;
        const long long tiles = (long long)((c.nx + pe::PS_OX) / pe::PS_OX) * ((c.ny + pe::PS_OY - 1) / pe::PS_OY);
        const long long blocks = tiles * ((c.nz + S->zc_ps - 1) / std::max(1, S->zc_ps));
        S->solo = S->pair_capable && S->zc_ps > 0 && blocks >= 2LL * nsm;
        if (S->pair_capable && !S->solo) {
            max_mat = std::max(max_mat, S->cfg.n_mat);
            B->pair_nc4 = B->pair_nc4 && S->cfg.n_coeffs == 4;
        }
    }
    cudaFuncAttributes fa{};
    PE_CUDA(cudaFuncGetAttributes(&fa, pe::k_stress_pair_batch<4, true>));
    const size_t dyn_s = (size_t)optin - fa.sharedSizeBytes;
    B->pair_ts = pe::pair_tab_in_smem(max_mat) &&
                 pe::PS_SMEM_FIXED + (size_t)max_mat * pe::TAB36 * sizeof(float) <= dyn_s;
    B->smem_s = pe::PS_SMEM_FIXED + (B->pair_ts ? (size_t)max_mat * pe::TAB36 * sizeof(float) : 0);
    B->smem_v = 128 + sizeof(float) * (3 * (size_t)pe::PV_SLOT + (size_t)max_mat);
    PE_CUDA(cudaFuncGetAttributes(&fa, pe::k_velocity_pair_batch<4>));
    if (B->smem_v > (size_t)optin - fa.sharedSizeBytes) return fail(PE_ERR_UNSUPPORTED, "density table too large");
    // per-kernel attributes: the largest dynamic size any batch may use
    auto setattr = [&](const void *f) {
        cudaFuncAttributes a{};
        cudaError_t e = cudaFuncGetAttributes(&a, f);
        if (e != cudaSuccess) return e;
        return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)a.sharedSizeBytes);
    };
    PE_CUDA(setattr((const void *)pe::k_stress_pair_batch<4, true>));
    PE_CUDA(setattr((const void *)pe::k_stress_pair_batch<4, false>));
    PE_CUDA(setattr((const void *)pe::k_stress_pair_batch<0, true>));
    PE_CUDA(setattr((const void *)pe::k_stress_pair_batch<0, false>));
    PE_CUDA(setattr((const void *)pe::k_velocity_pair_batch<4>));
    PE_CUDA(setattr((const void *)pe::k_velocity_pair_batch<0>));
    PE_CUDA(setattr((const void *)pe::k_pair_batch_persistent<4, true>));
    PE_CUDA(setattr((const void *)pe::k_pair_batch_persistent<4, false>));
    PE_CUDA(setattr((const void *)pe::k_pair_batch_persistent<0, true>));
    PE_CUDA(setattr((const void *)pe::k_pair_batch_persistent<0, false>));
    B->smem_p = pe::persistent_pair_smem(B->smem_s, B->smem_v);
    for (int s = 0; s < (int)B->solves.size(); ++s) {
        PeSolver *S = B->solves[s];
        if (!batched(B, S)) continue;
        const PeConfig &c = S->cfg;
        const int zc = S->zc_s;
        const int nzc = (c.nz + zc - 1) / zc;
        for (int bz = 0; bz < nzc; ++bz) {
            for (int by = 0; by < (c.ny + pe::PS_OY - 1) / pe::PS_OY; ++by)
                for (int bx = 0; bx < (c.nx + pe::PS_OX) / pe::PS_OX; ++bx) is.push_back({s, bx, by, bz});
            for (int by = 0; by < (c.ny + pe::PV_OY - 1) / pe::PV_OY; ++by)
                for (int bx = 0; bx < (c.nx + pe::PV_OX - 1) / pe::PV_OX; ++bx) iv.push_back({s, bx, by, bz});
        }
    }
    int per_v = 1, per_s = 1, per_p = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_v, pe::k_velocity_pair_batch<4>, pe::PV_N, B->smem_v);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_s, pe::k_stress_pair_batch<4, true>, pe::PS_N, B->smem_s);
    B->grid_s = std::max(1, std::min((int)is.size(), nsm * std::max(1, per_s)));
    B->grid_v = std::max(1, std::min((int)iv.size(), nsm * std::max(1, per_v)));
    // the persistent kernel's blocks must all be resident at once (its grid
    // barriers wait for every block): at most the occupancy times the SMs
    PE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_p, pe::k_pair_batch_persistent<4, true>, pe::PS_N,
                                                          B->smem_p));
    B->grid_p = std::max(1, std::min((int)std::max(is.size(), iv.size()), nsm * std::max(1, per_p)));
    return PE_OK;
}

template <typename T>
int batch_layout(PeBatch *B)
{
    std::vector<pe::BatchItem> is, iv;
    int max_mat = 1;
    for (int s = 0; s < (int)B->solves.size(); ++s) {
        const PeConfig &c = B->solves[s]->cfg;
        if (B->solves[s]->tma_capable) max_mat = std::max(max_mat, c.n_mat);
        const int target = c.z_chunk > 0 ? c.z_chunk : (B->z_chunk > 0 ? B->z_chunk : 40);
        const int nch = std::max(1, (c.nz + target - 1) / target);
        const int zc = (c.nz + nch - 1) / nch;
        B->solves[s]->zc_s = zc;
        B->solves[s]->zc_v = zc;
    }
    int dev = 0, optin = 0, nsm = 148;
    PE_CUDA(cudaGetDevice(&dev));
    PE_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    PE_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    B->pair_batch = false;
    if constexpr (std::is_same<T, float>::value) {
        bool any = false;
        for (PeSolver *S : B->solves) any = any || S->pair_capable;
        if (any) {
            B->pair_batch = true;
            int rc0 = batch_layout_pair(B, nsm, optin, is, iv);
            if (rc0 == PE_ERR_UNSUPPORTED) {
                B->pair_batch = false;
                is.clear();
                iv.clear();
            } else if (rc0) {
                return rc0;
            }
        }
    }
    if (!B->pair_batch) {
    B->smem_s = pe::stress_tma_smem<T>(max_mat);
    B->smem_v = pe::velocity_tma_smem<T>(max_mat);
    cudaFuncAttributes fa_s{}, fa_v{};
    PE_CUDA(cudaFuncGetAttributes(&fa_s, pe::k_stress_tma_batch<T>));
    PE_CUDA(cudaFuncGetAttributes(&fa_v, pe::k_velocity_tma_batch<T>));
    const int dyn_s = optin - (int)fa_s.sharedSizeBytes, dyn_v = optin - (int)fa_v.sharedSizeBytes;
    // when the batched kernels' tiles and tables do not fit (FP64 tiles with
    // large tables), every solve runs its own launches instead
    B->tma_batch = B->smem_s <= (size_t)dyn_s && B->smem_v <= (size_t)dyn_v;
    int per_s = 1, per_v = 1;
    if (B->tma_batch) {
        PE_CUDA(cudaFuncSetAttribute(pe::k_stress_tma_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_s));
        PE_CUDA(cudaFuncSetAttribute(pe::k_velocity_tma_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_v));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_s, pe::k_stress_tma_batch<T>, pe::TB_N, B->smem_s);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_v, pe::k_velocity_tma_batch<T>, pe::TB_N, B->smem_v);
    }
    for (int s = 0; s < (int)B->solves.size(); ++s) {
        if (!batched(B, B->solves[s])) continue;   // launched on its own
        const PeConfig &c = B->solves[s]->cfg;
        const int zc = B->solves[s]->zc_s;
        const int nzc = (c.nz + zc - 1) / zc;
        for (int bz = 0; bz < nzc; ++bz) {
            for (int by = 0; by < (c.ny + pe::TS_OY - 1) / pe::TS_OY; ++by)
                for (int bx = 0; bx < (c.nx + pe::TS_OX - 1) / pe::TS_OX; ++bx) is.push_back({s, bx, by, bz});
            for (int by = 0; by < (c.ny + pe::TB_Y - 1) / pe::TB_Y; ++by)
                for (int bx = 0; bx < (c.nx + pe::TB_X - 1) / pe::TB_X; ++bx) iv.push_back({s, bx, by, bz});
        }
    }
    B->grid_s = std::max(1, std::min((int)is.size(), nsm * std::max(1, per_s)));
    B->grid_v = std::max(1, std::min((int)iv.size(), nsm * std::max(1, per_v)));
    }
    B->n_items_s = (int)is.size();
    B->n_items_v = (int)iv.size();
    if (B->items_s) dev_free(B->items_s);
    if (B->items_v) dev_free(B->items_v);
    B->items_s = B->items_v = nullptr;
    int rc;
    if ((rc = dev_alloc(&B->items_s, sizeof(pe::BatchItem) * is.size()))) return rc;
    if ((rc = dev_alloc(&B->items_v, sizeof(pe::BatchItem) * iv.size()))) return rc;
    PE_CUDA(cudaMemcpy(B->items_s, is.data(), sizeof(pe::BatchItem) * is.size(), cudaMemcpyHostToDevice));
    PE_CUDA(cudaMemcpy(B->items_v, iv.data(), sizeof(pe::BatchItem) * iv.size(), cudaMemcpyHostToDevice));
    if (B->gexec) {
        cudaGraphExecDestroy(B->gexec);
        B->gexec = nullptr;
    }
    return PE_OK;
}

template <typename T>
int batch_upload(PeBatch *B, const PeState *states, void *const *traces)
{
    const int n = (int)B->solves.size();
    bool same = B->uploaded && (int)B->states.size() == n;
    for (int s = 0; same && s < n; ++s) same = same_state(B->states[s], states[s]) && B->traces[s] == traces[s];
    if (same) return PE_OK;
    std::vector<pe::StepArgs<T>> descs(n);
    std::vector<pe::TmapsStress> ms(n);
    std::vector<pe::TmapsVelocity> mv(n);
    std::vector<pe::TmapsPairStress> pms(n);
    std::vector<pe::TmapsPairVelocity> pmv(n);
    std::vector<const float *> tabs(n, nullptr);
    for (int s = 0; s < n; ++s) {
        PeSolver *S = B->solves[s];
        int rc = ensure_maps(S, &states[s]);
        if (rc) return rc;
        if (batched(B, S) && !(B->pair_batch ? S->pair : S->tma))
            return fail(PE_ERR_UNSUPPORTED, "batched solves need 16-byte aligned state buffers");
        descs[s] = make_args<T>(S, &states[s], 0);
        descs[s].step = B->step;
        descs[s].status = B->status;
        descs[s].zc = S->zc_s;
        ms[s] = S->ms;
        mv[s] = S->mv;
        pms[s] = S->mps;
        pmv[s] = S->mpv;
        tabs[s] = S->tab36;
    }
    PE_CUDA(cudaMemcpy(B->descs, descs.data(), sizeof(pe::StepArgs<T>) * n, cudaMemcpyHostToDevice));
    PE_CUDA(cudaMemcpy(B->maps_s, ms.data(), sizeof(pe::TmapsStress) * n, cudaMemcpyHostToDevice));
    PE_CUDA(cudaMemcpy(B->maps_v, mv.data(), sizeof(pe::TmapsVelocity) * n, cudaMemcpyHostToDevice));
    PE_CUDA(cudaMemcpy(B->pmaps_s, pms.data(), sizeof(pe::TmapsPairStress) * n, cudaMemcpyHostToDevice));
    PE_CUDA(cudaMemcpy(B->pmaps_v, pmv.data(), sizeof(pe::TmapsPairVelocity) * n, cudaMemcpyHostToDevice));
    PE_CUDA(cudaMemcpy(B->tabs, tabs.data(), sizeof(const float *) * n, cudaMemcpyHostToDevice));
    B->states.assign(states, states + n);
    B->traces.assign(traces, traces + n);
    B->uploaded = true;
    if (B->gexec) {
        cudaGraphExecDestroy(B->gexec);
        B->gexec = nullptr;
    }
    return PE_OK;
}

// the persistent batch kernel over `len` steps (a cooperative launch: the
// runtime refuses it rather than leave any block unresident)
int launch_pair_persistent(PeBatch *B, int len)
{
    PE_CUDA(cudaMemsetAsync(B->bar, 0, sizeof(unsigned), B->stream));
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)B->grid_p, 1, 1);
    lc.blockDim = dim3(pe::PS_N, 1, 1);
    lc.dynamicSmemBytes = B->smem_p;
    lc.stream = B->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    const pe::StepArgs<float> *d = (const pe::StepArgs<float> *)B->descs;
    const float *const *tabs = B->tabs;
    const pe::TmapsPairStress *ms = B->pmaps_s;
    const pe::TmapsPairVelocity *mv = B->pmaps_v;
    const int *nm = B->nmats;
    const pe::BatchItem *is = B->items_s, *iv = B->items_v;
    const int ns = B->n_items_s, nv = B->n_items_v;
    cudaError_t e;
    if (B->pair_nc4 && B->pair_ts)
        e = cudaLaunchKernelEx(&lc, pe::k_pair_batch_persistent<4, true>, d, ms, mv, tabs, nm, is, ns, iv, nv, len, B->bar, B->status);
    else if (B->pair_nc4)
        e = cudaLaunchKernelEx(&lc, pe::k_pair_batch_persistent<4, false>, d, ms, mv, tabs, nm, is, ns, iv, nv, len, B->bar, B->status);
    else if (B->pair_ts)
        e = cudaLaunchKernelEx(&lc, pe::k_pair_batch_persistent<0, true>, d, ms, mv, tabs, nm, is, ns, iv, nv, len, B->bar, B->status);
    else
        e = cudaLaunchKernelEx(&lc, pe::k_pair_batch_persistent<0, false>, d, ms, mv, tabs, nm, is, ns, iv, nv, len, B->bar, B->status);
    if (e != cudaSuccess) return fail(PE_ERR_CUDA, std::string("persistent batch launch: ") + cudaGetErrorString(e));
    B->launches += 1;
    return PE_OK;
}

template <typename T>
int batch_chunk(PeBatch *B, int len)
{
    const dim3 block(pe::TB_X, pe::TB_Y, 1);
    if constexpr (std::is_same<T, float>::value) {
        if (B->pair_batch && B->persistent && B->n_items_s > 0) {
            const int rc = launch_pair_persistent(B, len);
            if (rc) return rc;
        }
    }
    for (int k = 0; k < len; ++k) {
        if constexpr (std::is_same<T, float>::value) {
            if (B->pair_batch && !B->persistent && B->n_items_s > 0) {
                const pe::StepArgs<float> *d = (const pe::StepArgs<float> *)B->descs;
                const int ns = B->n_items_s, nv = B->n_items_v;
                if (B->pair_nc4 && B->pair_ts)
                    pe::k_stress_pair_batch<4, true><<<B->grid_s, pe::PS_N, B->smem_s, B->stream>>>(d, B->pmaps_s, B->tabs, B->nmats, B->items_s, ns, k);
                else if (B->pair_nc4)
                    pe::k_stress_pair_batch<4, false><<<B->grid_s, pe::PS_N, B->smem_s, B->stream>>>(d, B->pmaps_s, B->tabs, B->nmats, B->items_s, ns, k);
                else if (B->pair_ts)
                    pe::k_stress_pair_batch<0, true><<<B->grid_s, pe::PS_N, B->smem_s, B->stream>>>(d, B->pmaps_s, B->tabs, B->nmats, B->items_s, ns, k);
                else
                    pe::k_stress_pair_batch<0, false><<<B->grid_s, pe::PS_N, B->smem_s, B->stream>>>(d, B->pmaps_s, B->tabs, B->nmats, B->items_s, ns, k);
                if (B->pair_nc4)
                    pe::k_velocity_pair_batch<4><<<B->grid_v, pe::PV_N, B->smem_v, B->stream>>>(d, B->pmaps_v, B->nmats, B->items_v, nv, k);
                else
                    pe::k_velocity_pair_batch<0><<<B->grid_v, pe::PV_N, B->smem_v, B->stream>>>(d, B->pmaps_v, B->nmats, B->items_v, nv, k);
                B->launches += 2;
            }
        }
        if (!B->pair_batch && B->n_items_s > 0) {
            pe::k_stress_tma_batch<T><<<B->grid_s, block, B->smem_s, B->stream>>>(
                (const pe::StepArgs<T> *)B->descs, B->maps_s, B->nmats, B->items_s, B->n_items_s, k);
            pe::k_velocity_tma_batch<T><<<B->grid_v, block, B->smem_v, B->stream>>>(
                (const pe::StepArgs<T> *)B->descs, B->maps_v, B->nmats, B->items_v, B->n_items_v, k);
            B->launches += 2;
        }
        // solves outside the batched launches (rows not whole 16-byte
        // units, or tiles too large) run their own kernel pair each, on the
        // same stream and step counter
        for (int s = 0; s < (int)B->solves.size(); ++s) {
            PeSolver *S = B->solves[s];
            if (batched(B, S)) continue;
            pe::StepArgs<T> A = make_args<T>(S, &B->states[s], k);
            A.step = B->step;
            A.status = B->status;
            launch_stress<T>(S, A, B->stream);
            launch_velocity<T>(S, A, B->stream);
            B->launches += 2;
        }
    }
    for (int s = 0; s < (int)B->solves.size(); ++s) {
        PeSolver *S = B->solves[s];
        if (S->n_groups <= 0) continue;
        const int nthr = len * S->n_groups;
        pe::k_reduce_traces<T><<<(nthr + 127) / 128, 128, 0, B->stream>>>(
            (const T *)S->rec_val, (const T *)S->rec_w, S->grp_off, S->n_groups, S->n_rec, len, B->step,
            (T *)B->traces[s]);
        B->launches += 1;
    }
    pe::k_step_advance<<<1, 1, 0, B->stream>>>(B->step, len);
    B->launches += 1;
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

template <typename T>
int batch_run_t(PeBatch *B, const PeState *states, void *const *traces, int64_t b, int64_t e, cudaStream_t user)
{
    int rc = batch_upload<T>(B, states, traces);
    if (rc) return rc;
    PE_CUDA(cudaEventRecord(B->ev_in, user));
    PE_CUDA(cudaStreamWaitEvent(B->stream, B->ev_in, 0));
    pe::k_step_set<<<1, 1, 0, B->stream>>>(B->step, b);
    B->launches += 1;
    for (int64_t n = b; n < e;) {
        const int len = (int)std::min<int64_t>(B->chunk, e - n);
        if (len == B->chunk) {
            if (!B->gexec) {
                cudaGraph_t g = nullptr;
                PE_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
                const long long before = B->launches;
                rc = batch_chunk<T>(B, len);
                cudaError_t ce = cudaStreamEndCapture(B->stream, &g);
                if (rc) return rc;
                if (ce != cudaSuccess) return fail(PE_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(ce));
                B->graph_launches = B->launches - before;
                B->launches = before;
                ce = cudaGraphInstantiate(&B->gexec, g, 0);
                cudaGraphDestroy(g);
                if (ce != cudaSuccess) return fail(PE_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ce));
            }
            PE_CUDA(cudaGraphLaunch(B->gexec, B->stream));
            B->launches += B->graph_launches;
        } else if ((rc = batch_chunk<T>(B, len))) {
            return rc;
        }
        n += len;
    }
    PE_CUDA(cudaEventRecord(B->ev_out, B->stream));
    PE_CUDA(cudaStreamWaitEvent(user, B->ev_out, 0));
    return PE_OK;
}

}  // namespace

extern "C" {

int pe_batch_create(int n, const PeConfig *cfgs, const PeMedium *media, const PeProbe *probes,
                    PeBatch **out)
{
    if (n < 1 || !cfgs || !media || !probes || !out) return fail(PE_ERR_INVALID, "bad batch arguments");
    *out = nullptr;
    std::unique_ptr<PeBatch> B(new PeBatch());
    B->dtype = cfgs[0].dtype;
    B->esize = dtype_size(B->dtype);
    for (int s = 0; s < n; ++s) {
        if (cfgs[s].dtype != B->dtype) return fail(PE_ERR_INVALID, "all solves of a batch share one dtype");
        if (cfgs[s].variant != PE_KERNEL_TILED)
            return fail(PE_ERR_UNSUPPORTED, "batches run the tiled kernels");
        PeSolver *S = nullptr;
        int rc = pe_solver_create(&cfgs[s], &media[s], &probes[s], &S);
        if (rc) return fail(rc, "solve " + std::to_string(s) + ": " + g_err);
        B->solves.push_back(S);
    }
    B->chunk = cfgs[0].chunk_steps > 0 ? cfgs[0].chunk_steps : 200;
    int rc;
    if ((rc = dev_alloc(&B->step, sizeof(long long)))) return rc;
    if ((rc = dev_alloc(&B->status, sizeof(int)))) return rc;
    PE_CUDA(cudaMemset(B->status, 0, sizeof(int)));
    if ((rc = dev_alloc(&B->bar, sizeof(unsigned)))) return rc;
    const size_t ds = B->dtype == PE_F64 ? sizeof(pe::StepArgs<double>) : sizeof(pe::StepArgs<float>);
    if ((rc = dev_alloc(&B->descs, ds * n))) return rc;
    if ((rc = dev_alloc(&B->maps_s, sizeof(pe::TmapsStress) * n))) return rc;
    if ((rc = dev_alloc(&B->maps_v, sizeof(pe::TmapsVelocity) * n))) return rc;
    if ((rc = dev_alloc(&B->nmats, sizeof(int) * n))) return rc;
    if ((rc = dev_alloc(&B->pmaps_s, sizeof(pe::TmapsPairStress) * n))) return rc;
    if ((rc = dev_alloc(&B->pmaps_v, sizeof(pe::TmapsPairVelocity) * n))) return rc;
    if ((rc = dev_alloc(&B->tabs, sizeof(const float *) * n))) return rc;
    std::vector<int> nm(n);
    for (int s = 0; s < n; ++s) nm[s] = cfgs[s].n_mat;
    PE_CUDA(cudaMemcpy(B->nmats, nm.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    PE_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    PE_CUDA(cudaEventCreateWithFlags(&B->ev_in, cudaEventDisableTiming));
    PE_CUDA(cudaEventCreateWithFlags(&B->ev_out, cudaEventDisableTiming));
    rc = B->dtype == PE_F64 ? batch_layout<double>(B.get()) : batch_layout<float>(B.get());
    if (rc) return rc;
    *out = B.release();
    return PE_OK;
}

int pe_batch_schedule(PeBatch *B, int z_chunk, int chunk_steps)
{
    if (!B || z_chunk < 0 || chunk_steps < 0) return fail(PE_ERR_INVALID, "bad schedule");
    B->z_chunk = z_chunk;
    if (chunk_steps > 0) B->chunk = chunk_steps;
    for (PeSolver *S : B->solves) S->cfg.z_chunk = 0;
    B->uploaded = false;
    return B->dtype == PE_F64 ? batch_layout<double>(B) : batch_layout<float>(B);
}

int pe_batch_set_persistent(PeBatch *B, int on)
{
    if (!B) return fail(PE_ERR_INVALID, "null batch");
    if (on && !B->pair_batch)
        return fail(PE_ERR_UNSUPPORTED, "the persistent kernel runs FP32 batches of pair-column solves");
    if (B->persistent != (on != 0)) {
        B->persistent = on != 0;
        if (B->gexec) {
            cudaGraphExecDestroy(B->gexec);
            B->gexec = nullptr;
        }
    }
    return PE_OK;
}

int pe_batch_set_wavelet(PeBatch *B, int i, const void *wavelet, int64_t nt)
{
    if (!B || i < 0 || i >= (int)B->solves.size()) return fail(PE_ERR_INVALID, "bad solve index");
    return pe_solver_set_wavelet(B->solves[i], wavelet, nt);
}

int pe_batch_run(PeBatch *B, const PeState *states, void *const *traces, int64_t b, int64_t e, void *stream)
{
    if (!B || !states || !traces) return fail(PE_ERR_INVALID, "null argument");
    if (b < 0 || e < b) return fail(PE_ERR_INVALID, "need 0 <= step_begin <= step_end");
    for (int s = 0; s < (int)B->solves.size(); ++s) {
        PeSolver *S = B->solves[s];
        if (S->n_src > 0 && e > S->nt_wav) return fail(PE_ERR_INVALID, "solve " + std::to_string(s) + ": wavelet shorter than step_end");
        if (S->n_groups > 0 && !traces[s]) return fail(PE_ERR_INVALID, "solve " + std::to_string(s) + ": traces buffer required");
    }
    B->launches = 0;
    if (e == b) return PE_OK;
    return B->dtype == PE_F64 ? batch_run_t<double>(B, states, traces, b, e, (cudaStream_t)stream)
                              : batch_run_t<float>(B, states, traces, b, e, (cudaStream_t)stream);
}

int pe_batch_status(PeBatch *B)
{
    if (!B) return fail(PE_ERR_INVALID, "null batch");
    int st = 0;
    PE_CUDA(cudaStreamSynchronize(B->stream));
    PE_CUDA(cudaMemcpy(&st, B->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) {
        PE_CUDA(cudaMemset(B->status, 0, sizeof(int)));
        return fail(PE_ERR_TIMEOUT, "a bounded device-side wait gave up; the batch results are invalid");
    }
    return PE_OK;
}

int64_t pe_batch_launch_count(const PeBatch *B) { return B ? B->launches : -1; }

int pe_batch_destroy(PeBatch *B)
{
    delete B;
    return PE_OK;
}

}  // extern "C"
