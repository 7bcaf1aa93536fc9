// Host side of libpyfwi_b200: plans, workspace layout, the time-loop
// schedules, and the C ABI declared in include/pyfwi_b200.h.
//
// The reference drives its kernels from Python, one pyopencl launch per
// kernel, step and shot (PyFWI src/PyFWI/wave_propagation.py:625-856).  Here a
// plan runs every step of a batch of shots with one fused launch per step,
// all enqueued on the caller's stream (optionally replayed as a CUDA graph).
#include "pyfwi_b200.h"
#include "kernels.cuh"
#include "persist_kernels.cuh"
#include "stream_kernels.cuh"
#include "tile_tma.cuh"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace pyfwi;

namespace {

// NVTX range over a scope: the phases of a call show as named ranges in a
// profiler's timeline (no cost without a profiler attached).
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};


thread_local std::string g_err;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(x)                                                                               \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) return fail(PYFWI_E_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

#define CKL()                                                                                      \
    do {                                                                                           \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess) return fail(PYFWI_E_CUDA, "kernel launch: %s", cudaGetErrorString(e_)); \
    } while (0)

constexpr size_t ALIGN = 256;
size_t up(size_t x, size_t a = ALIGN) { return (x + a - 1) / a * a; }

// kernel variants: 0..2 tile kernels with 16 / 8 / 32 rows per tile,
// 3..5 streaming kernels whose CTAs span 128 / 64 / 256 columns, 6..7 the
// 16-row tile kernels whose adjoint CTAs carry 2 / 4 shots each (the
// forward step of 6..7 is variant 0's), 8..10 the tile kernels of 16 / 8 /
// 32 rows with the forward tile staged by TMA box copies (the adjoint of
// 8..10 is that of 0..2), 11 the 16-row tile kernels whose adjoint copies
// the tile's gradient accumulators into shared memory at its start
constexpr int TILE_TZ[] = {16, 8, 32, 0, 0, 0, 16, 16, 16, 8, 32, 16};
constexpr int STREAM_W[] = {0, 0, 0, 128, 64, 256, 0, 0, 0, 0, 0, 0};
constexpr int ADJ_NS[] = {1, 1, 1, 1, 1, 1, 2, 4, 1, 1, 1, 1};
constexpr int FWD_TMA[] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 0};
constexpr int ADJ_PREFETCH[] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1};
constexpr int N_TILES = 12;
constexpr int FWD_PF = 4, ADJ_PF = 2;  // rows the streaming kernels fetch ahead
constexpr size_t ERR_OFF = 128;         // byte offset of the device error word in the header
constexpr size_t CHECK_OFF = 192;       // byte offset of the frame-check counter (uint64) in the header
constexpr size_t BAR_OFF = 224;         // byte offset of the persistent kernels' grid barrier (2 x uint32)

// cuTensorMapEncodeTiled, resolved through the runtime so the library does
// not link the driver API directly
typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

}  // namespace

// Lets the static-scratch entry point (static_scratch.cu) report through
// pyfwi_last_error(); hidden from the library's exported symbols.
__attribute__((visibility("hidden"))) void pyfwi_set_error(const char *msg) { g_err = msg; }

struct pyfwi_plan {
    pyfwi_geometry geom;
    pyfwi_options opt;
    std::vector<int32_t> srcx, srcz, chp;
    std::vector<float> src_vals;  // [n_inj][4] host copy of the last forward's wavelet
    Grid g;
    Coef k;
    Lines lines;
    int R, tz, st_w, ftma, atz, ast_w, ans, apf, chunk_opt, nacc, G, ngroups, seg, M, n_inj;  // a*: adjoint step variant
    bool exact_adj = false;  // PYFWI_ADJOINT_EXACT
    bool persist = false;    // time loops as persistent kernels (options.persist, where the layout allows)
    bool overlap = false;    // recompute of segment m-1 on a second stream beside the adjoint of segment m
    int qd = 0;              // the segment store holds the imaging's differences of each state (options.store_diffs):
                             // 1 in FP32, 2 in 24 bits (FP24 snapshots); 0 the states
    cudaStream_t side = nullptr;          // that second stream (created on first use)
    std::vector<cudaEvent_t> ovev;        // its events: [2m] recompute of m done, [2m+1] adjoint of m done
    int fwd_cap = 0, adj_cap = 0;  // co-resident CTAs of the persistent kernels on this device
    long long state;  // floats per state (5 planes)
    // workspace offsets in bytes
    size_t o_hdr, o_src, o_red, o_mat, o_dampx, o_dampz, o_work, o_adj, o_gacc, o_store, o_store16, o_store8, total;
    long long launches = 0;
    bool model_set = false, fwd_valid = false;
    // per-kernel event timing (pyfwi_profile_enable)
    bool profiling = false;
    struct Ev {
        cudaEvent_t a, b;
        int kind;
        double cells;
    };
    std::vector<Ev> events;
    size_t ev_used = 0;
    double prof_ms[3] = {0, 0, 0}, prof_cells[3] = {0, 0, 0};
    long long prof_n[3] = {0, 0, 0};
    void *ws_initialised = nullptr;
    // CUDA-graph replay of whole calls (options.graph)
    struct GraphCache {
        cudaGraphExec_t exec = nullptr;
        std::vector<uintptr_t> key;
        long long launches = 0;
    } gfwd, ggrad, gmis;
    cudaStream_t cap = nullptr;  // capture stream (the caller's may be the legacy default stream)
    // tensor maps of the workspace (rows of `pitch` floats), per box shape
    struct TMap {
        void *ws = nullptr;
        int w = 0, h = 0;
        alignas(64) CUtensorMap map;
    } tmaps[6];
    int tmap_next = 0;
};

// The static-scratch entry point clears its array before every call: the
// plan must then initialise that workspace again (zero frames, source cells)
// in pyfwi_set_model.  Hidden from the library's exported symbols.
__attribute__((visibility("hidden"))) void pyfwi_plan_workspace_cleared(pyfwi_plan *p) { p->ws_initialised = nullptr; }

// Trace dimensions of a plan for the static-scratch entry point; hidden from
// the library's exported symbols.
__attribute__((visibility("hidden"))) void pyfwi_plan_trace_dims(const pyfwi_plan *p, int *nt_ext, int *ns, int *nr)
{
    *nt_ext = p->geom.nt_ext;
    *ns = p->geom.ns;
    *nr = p->geom.nr;
}

namespace {

int check_ws(const pyfwi_plan *p, void *ws, size_t bytes)
{
    if (!ws) return fail(PYFWI_E_WORKSPACE, "workspace is NULL");
    if (bytes < p->total) return fail(PYFWI_E_WORKSPACE, "workspace has %zu bytes, plan needs %zu", bytes, p->total);
    if (reinterpret_cast<uintptr_t>(ws) % ALIGN) return fail(PYFWI_E_WORKSPACE, "workspace not 256-byte aligned");
    return PYFWI_OK;
}

template <typename T>
T *at(void *ws, size_t off)
{
    return reinterpret_cast<T *>(static_cast<char *>(ws) + off);
}

// ---- kernel dispatch ------------------------------------------------------
template <int R, int TZ>
int launch_fwd(pyfwi_plan *p, const StepArgs &a, int nslots, cudaStream_t s, bool reverse)
{
    dim3 grid((p->g.tnx + TX - 1) / TX, (p->g.tnz + TZ - 1) / TZ, nslots);
    if (!reverse) {
        size_t sm = FwdShape<R, TZ>::FLOATS * sizeof(float), sm_q = sm + 4 * sizeof(float);
        static bool attr = false;
        if (!attr) {
            CK(cudaFuncSetAttribute(fwd_step<R, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            CK(cudaFuncSetAttribute(fwd_step24<R, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            CK(cudaFuncSetAttribute(fwd_step<R, TZ, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_q));
            CK(cudaFuncSetAttribute(fwd_step<R, TZ, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_q));
            attr = true;
        }
        if (a.snap8)  // 24-bit snapshots written by their own instance (keeps the others' registers)
            fwd_step24<R, TZ><<<grid, NTHREADS, sm, s>>>(a);
        else if (a.qout && a.qout8)  // difference sets, also by their own instances
            fwd_step<R, TZ, 2><<<grid, NTHREADS, sm_q, s>>>(a);
        else if (a.qout)
            fwd_step<R, TZ, 1><<<grid, NTHREADS, sm_q, s>>>(a);
        else
            fwd_step<R, TZ><<<grid, NTHREADS, sm, s>>>(a);
    } else {
        size_t sm = RevShape<R, TZ>::FLOATS * sizeof(float);
        static bool attr = false;
        if (!attr) {
            CK(cudaFuncSetAttribute(rev_step<R, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            attr = true;
        }
        rev_step<R, TZ><<<grid, NTHREADS, sm, s>>>(a);
    }
    p->launches++;
    CKL();
    return PYFWI_OK;
}

// Adds the residual row of this step to the input adjoint state, in place
// (Adj_injSrc, elastic_surface.cl:48-71), before the step kernel reads it.
int launch_inject(pyfwi_plan *p, const AdjArgs &a, int nslots, cudaStream_t s)
{
    if (a.inj_row < 0) return PYFWI_OK;
    // one CTA per shot: receivers of different lines on one cell then add in line order
    inject_kernel<<<dim3(1, nslots), 256, 0, s>>>(p->g, const_cast<float *>(a.in), a.in_stride, a.shot0, a.inj_row,
                                                  a.res[0], a.res[1], a.res[2], a.res[3], a.res[4], p->lines, a.ns,
                                                  a.nr, 0);
    p->launches++;
    CKL();
    return PYFWI_OK;
}

template <int R, int TZ, bool E, int NS, bool NARROW>
int launch_adj_t(pyfwi_plan *p, const AdjArgs &a, int nslots, cudaStream_t s)
{
    int rc = launch_inject(p, a, nslots, s);
    if (rc) return rc;
    dim3 grid((p->g.tnx + TX - 1) / TX, (p->g.tnz + TZ - 1) / TZ, (nslots + NS - 1) / NS);
    size_t sm = adj_smem_floats<R, TZ, E, NS>() * sizeof(float);
    // one shot per CTA on FP32 or BF16 states: adj_step (with the
    // accumulators prefetched: variant 11); else adj_step_ns
    constexpr bool own = NS == 1 && !NARROW;
    const bool pf = own && !E && p->apf;
    const size_t sm_pf = sm + 3 * TZ * TX * sizeof(float);
    static bool attr = false;
    if (!attr) {
        if constexpr (own) {
            CK(cudaFuncSetAttribute(adj_step<R, TZ, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            if constexpr (!E)
                CK(cudaFuncSetAttribute(adj_step<R, TZ, E, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm_pf));
        } else {
            CK(cudaFuncSetAttribute(adj_step_ns<R, TZ, E, NS, NARROW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sm));
        }
        attr = true;
    }
    AdjArgs b = a;
    b.nslots = nslots;
    if constexpr (own && !E) {
        if (p->qd) {  // difference sets in the segment store (FP32) or the snapshot store (24 bits)
            static bool attr_q = false;
            if (!attr_q) {
                CK(cudaFuncSetAttribute(adj_step<R, TZ, E, false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm));
                CK(cudaFuncSetAttribute(adj_step<R, TZ, E, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm));
                attr_q = true;
            }
            if (p->qd == 2)
                adj_step<R, TZ, E, false, 2><<<grid, NTHREADS, sm, s>>>(b);
            else
                adj_step<R, TZ, E, false, 1><<<grid, NTHREADS, sm, s>>>(b);
            p->launches++;
            CKL();
            return PYFWI_OK;
        }
        if (pf) {
            adj_step<R, TZ, E, true><<<grid, NTHREADS, sm_pf, s>>>(b);
            p->launches++;
            CKL();
            return PYFWI_OK;
        }
    }
    if constexpr (own)
        adj_step<R, TZ, E><<<grid, NTHREADS, sm, s>>>(b);
    else
        adj_step_ns<R, TZ, E, NS, NARROW><<<grid, NTHREADS, sm, s>>>(b);
    p->launches++;
    CKL();
    return PYFWI_OK;
}

template <int R, int TZ, int NS>
int launch_adj_ns(pyfwi_plan *p, const AdjArgs &a, int nslots, cudaStream_t s)
{
    return p->nacc == 6 ? launch_adj_t<R, TZ, true, NS, false>(p, a, nslots, s)
                        : launch_adj_t<R, TZ, false, NS, false>(p, a, nslots, s);
}

template <int R, int TZ>
int launch_adj(pyfwi_plan *p, const AdjArgs &a, int nslots, cudaStream_t s)
{
    if (a.fwd8 && !p->qd) {  // 24-bit snapshots: the 16-row kernel, one shot per CTA (the plan picks no other)
        if (TZ != 16 || p->ans != 1) return fail(PYFWI_E_INVALID, "snapshots are imaged by adjoint variant 0 only");
        return p->nacc == 6 ? launch_adj_t<R, 16, true, 1, true>(p, a, nslots, s)
                            : launch_adj_t<R, 16, false, 1, true>(p, a, nslots, s);
    }
    if (TZ == 16 && p->ans == 2) return launch_adj_ns<R, TZ, 2>(p, a, nslots, s);
    if (TZ == 16 && p->ans == 4) return launch_adj_ns<R, TZ, 4>(p, a, nslots, s);
    return launch_adj_ns<R, TZ, 1>(p, a, nslots, s);
}

// ---- persistent kernels ----------------------------------------------------
// Co-resident CTAs of `kern` with `smem` bytes of shared memory on the
// current device (the most a cooperative launch may have).
int coresident(const void *kern, size_t smem, int *out)
{
    int dev = 0, sms = 0, per = 0, coop = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return fail(PYFWI_E_CUDA, "the device does not support cooperative launches");
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, NTHREADS, smem));
    if (per < 1) return fail(PYFWI_E_CUDA, "a persistent kernel does not fit on an SM");
    *out = per * sms;
    return PYFWI_OK;
}

template <int R, int TZ>
int launch_fwd_persist(pyfwi_plan *p, const FwdPersistArgs &a, cudaStream_t s)
{
    const size_t sm = FwdShape<R, TZ>::FLOATS * sizeof(float);
    const void *kern = reinterpret_cast<const void *>(fwd_persist<R, TZ>);
    if (!p->fwd_cap) {
        CK(cudaFuncSetAttribute(fwd_persist<R, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        int rc = coresident(kern, sm, &p->fwd_cap);
        if (rc) return rc;
    }
    const int nwork = a.ntx * a.ntz * a.nslots;
    void *args[] = {const_cast<FwdPersistArgs *>(&a)};
    CK(cudaLaunchCooperativeKernel(kern, dim3(std::min(nwork, p->fwd_cap)), dim3(NTHREADS), args, sm, s));
    p->launches++;
    return PYFWI_OK;
}

template <int R, int TZ, bool E>
int launch_adj_persist_t(pyfwi_plan *p, const AdjPersistArgs &a, cudaStream_t s)
{
    const size_t sm = AdjShape<R, TZ>::FLOATS * sizeof(float);
    const void *kern = reinterpret_cast<const void *>(adj_persist<R, TZ, E>);
    if (!p->adj_cap) {
        CK(cudaFuncSetAttribute(adj_persist<R, TZ, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        int rc = coresident(kern, sm, &p->adj_cap);
        if (rc) return rc;
    }
    const int nwork = a.ntx * a.ntz * a.a.nslots;
    void *args[] = {const_cast<AdjPersistArgs *>(&a)};
    CK(cudaLaunchCooperativeKernel(kern, dim3(std::min(nwork, p->adj_cap)), dim3(NTHREADS), args, sm, s));
    p->launches++;
    return PYFWI_OK;
}

// Gradient accumulator slots the adjoint kernel writes for a launch of
// `nslots` shots: one per CTA shot group of the tile kernel, one per shot
// for the others.
int acc_slots(const pyfwi_plan *p, int nslots)
{
    const int ns = (!p->exact_adj && !p->ast_w) ? p->ans : 1;
    return (nslots + ns - 1) / ns;
}

// Event pair around one step launch when profiling (kind 0 fwd, 1 adj, 2 rev).
struct ProfileScope {
    pyfwi_plan *p;
    cudaStream_t s;
    pyfwi_plan::Ev *ev = nullptr;
    ProfileScope(pyfwi_plan *p_, cudaStream_t s_, int kind, int nslots) : p(p_), s(s_)
    {
        if (!p->profiling) return;
        if (p->ev_used == p->events.size()) {
            pyfwi_plan::Ev e{};
            if (cudaEventCreate(&e.a) != cudaSuccess || cudaEventCreate(&e.b) != cudaSuccess) return;
            p->events.push_back(e);
        }
        ev = &p->events[p->ev_used++];
        ev->kind = kind;
        ev->cells = (double)p->g.tnz * p->g.tnx * nslots;
        cudaEventRecord(ev->a, s);
    }
    ~ProfileScope()
    {
        if (ev) cudaEventRecord(ev->b, s);
    }
};

// Rows per CTA of the streaming kernels: the option, or enough row chunks
// to give about eight CTAs of 128 threads per SM over the launch.
int stream_chunk(const pyfwi_plan *p, int nslots, int T)
{
    if (p->chunk_opt > 0) return std::min(p->chunk_opt, p->g.tnz);
    const int stripes = (p->g.tnx + (T - 2 * p->R) - 1) / (T - 2 * p->R);
    const long long target = 148LL * 8 * 128 / T;
    long long per_chunk = (long long)stripes * nslots;
    int nchunks = (int)std::max(1LL, (target + per_chunk - 1) / per_chunk);
    int chunk = (p->g.tnz + nchunks - 1) / nchunks;
    return std::max(chunk, std::min(p->g.tnz, 8 * p->R));
}

// The workspace as a 2-D tensor of rows of `pitch` floats with a box of
// W x H (W x 1 for the streaming kernels, whole tiles for the TMA tile
// kernel); encoded once per workspace and box, a few kept.
int workspace_map(pyfwi_plan *p, const float *ws, int W, CUtensorMap *out, int H = 1)
{
    for (auto &m : p->tmaps)
        if (m.ws == ws && m.w == W && m.h == H) {
            *out = m.map;
            return PYFWI_OK;
        }
    pyfwi_plan::TMap *slot = &p->tmaps[p->tmap_next];
    p->tmap_next = (p->tmap_next + 1) % (int)(sizeof p->tmaps / sizeof p->tmaps[0]);
    static EncodeTiled encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn)
            return fail(PYFWI_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        encode = reinterpret_cast<EncodeTiled>(fn);
    }
    const size_t row = (size_t)p->g.pitch * sizeof(float);
    cuuint64_t dims[2] = {(cuuint64_t)p->g.pitch, (cuuint64_t)(p->total / row)};
    cuuint64_t strides[1] = {(cuuint64_t)row};
    cuuint32_t box[2] = {(cuuint32_t)W, (cuuint32_t)H}, estr[2] = {1, 1};
    CUresult r = encode(&slot->map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(ws), dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(PYFWI_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    slot->ws = const_cast<float *>(ws);
    slot->w = W;
    slot->h = H;
    *out = slot->map;
    return PYFWI_OK;
}

template <int R, int TZ>
int launch_fwd_tma(pyfwi_plan *p, const StepArgs &a, int nslots, cudaStream_t s, const float *ws)
{
    using S = FwdShape<R, TZ>;
    FwdTmaArgs t;
    memset(&t, 0, sizeof t);
    t.a = a;
    t.a.tbase = ws;
    t.a.err = at<int>(const_cast<float *>(ws), ERR_OFF);
    int rc = workspace_map(p, ws, S::SW, &t.ms, S::HT);
    if (!rc) rc = workspace_map(p, ws, S::VW, &t.mv, S::HV);
    if (!rc) rc = workspace_map(p, ws, TX, &t.mt, TZ);
    if (rc) return rc;
    dim3 grid((p->g.tnx + TX - 1) / TX, (p->g.tnz + TZ - 1) / TZ, nslots);
    const size_t sm = FwdTmaShape<R, TZ>::BYTES;
    static bool attr = false;
    if (!attr) {
        CK(cudaFuncSetAttribute(fwd_tma<R, TZ, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        CK(cudaFuncSetAttribute(fwd_tma<R, TZ, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        attr = true;
    }
    if (a.snap8)
        fwd_tma<R, TZ, true><<<grid, NTHREADS, sm, s>>>(t);
    else
        fwd_tma<R, TZ, false><<<grid, NTHREADS, sm, s>>>(t);
    p->launches++;
    CKL();
    return PYFWI_OK;
}

template <int R, int W>
int launch_fwd_stream(pyfwi_plan *p, StepArgs a, int nslots, cudaStream_t s, const float *ws)
{
    using S = FwdRing<R, W, FWD_PF>;
    a.chunk = stream_chunk(p, nslots, S::T);
    a.tbase = ws;
    a.err = reinterpret_cast<int *>(const_cast<char *>(reinterpret_cast<const char *>(ws)) + ERR_OFF);
    int rc = workspace_map(p, ws, W, &a.tmap);
    if (rc) return rc;
    const int iw = S::T - 2 * R;
    dim3 grid((p->g.tnx + iw - 1) / iw, (p->g.tnz + a.chunk - 1) / a.chunk, nslots);
    static bool attr = false;
    if (!attr) {
        CK(cudaFuncSetAttribute(fwd_stream<R, W, FWD_PF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::BYTES));
        attr = true;
    }
    fwd_stream<R, W, FWD_PF><<<grid, S::T, S::BYTES, s>>>(a);
    p->launches++;
    CKL();
    return PYFWI_OK;
}

template <int R, int W, bool E>
int launch_adj_stream_t(pyfwi_plan *p, AdjArgs a, int nslots, cudaStream_t s, const float *ws)
{
    using S = AdjRing<R, W, ADJ_PF, E>;
    int rc = launch_inject(p, a, nslots, s);
    if (rc) return rc;
    a.chunk = stream_chunk(p, nslots, S::T);
    a.tbase = ws;
    a.err = reinterpret_cast<int *>(const_cast<char *>(reinterpret_cast<const char *>(ws)) + ERR_OFF);
    rc = workspace_map(p, ws, W, &a.tmap);
    if (rc) return rc;
    const int iw = S::T - 2 * R;
    dim3 grid((p->g.tnx + iw - 1) / iw, (p->g.tnz + a.chunk - 1) / a.chunk, nslots);
    static bool attr = false;
    if (!attr) {
        CK(cudaFuncSetAttribute(adj_stream<R, W, ADJ_PF, E>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)S::BYTES));
        attr = true;
    }
    adj_stream<R, W, ADJ_PF, E><<<grid, S::T, S::BYTES, s>>>(a);
    p->launches++;
    CKL();
    return PYFWI_OK;
}

template <int R, int W>
int launch_adj_stream(pyfwi_plan *p, const AdjArgs &a, int nslots, cudaStream_t s, const float *ws)
{
    return p->nacc == 6 ? launch_adj_stream_t<R, W, true>(p, a, nslots, s, ws)
                        : launch_adj_stream_t<R, W, false>(p, a, nslots, s, ws);
}

int step_fwd(pyfwi_plan *p, const StepArgs &a, int nslots, cudaStream_t s, bool reverse, const float *ws)
{
    ProfileScope prof(p, s, reverse ? 2 : 0, nslots);
    if (p->st_w && !reverse) {
#define CASE(R_, W_) \
    if (p->R == R_ && p->st_w == W_) return launch_fwd_stream<R_, W_>(p, a, nslots, s, ws);
        CASE(2, 128) CASE(2, 64) CASE(2, 256) CASE(4, 128) CASE(4, 64) CASE(4, 256)
#undef CASE
    }
    const int tz = p->tz ? p->tz : 16;  // reverse steps always use the tile kernel
    if (p->ftma && !reverse) {
#define CASE(R_, TZ_) \
    if (p->R == R_ && tz == TZ_) return launch_fwd_tma<R_, TZ_>(p, a, nslots, s, ws);
        CASE(2, 16) CASE(2, 8) CASE(2, 32) CASE(4, 16) CASE(4, 8) CASE(4, 32)
#undef CASE
    }
#define CASE(R_, TZ_) \
    if (p->R == R_ && tz == TZ_) return launch_fwd<R_, TZ_>(p, a, nslots, s, reverse);
    CASE(2, 16) CASE(2, 8) CASE(2, 32) CASE(4, 16) CASE(4, 8) CASE(4, 32)
#undef CASE
    return fail(PYFWI_E_INVALID, "no kernel for half order %d, tile rows %d", p->R, tz);
}

int step_adj(pyfwi_plan *p, const AdjArgs &a, int nslots, cudaStream_t s, const float *ws)
{
    ProfileScope prof(p, s, 1, nslots);
    if (p->ast_w) {
#define CASE(R_, W_) \
    if (p->R == R_ && p->ast_w == W_) return launch_adj_stream<R_, W_>(p, a, nslots, s, ws);
        CASE(2, 128) CASE(2, 64) CASE(2, 256) CASE(4, 128) CASE(4, 64) CASE(4, 256)
#undef CASE
    }
#define CASE(R_, TZ_) \
    if (p->R == R_ && p->atz == TZ_) return launch_adj<R_, TZ_>(p, a, nslots, s);
    CASE(2, 16) CASE(2, 8) CASE(2, 32) CASE(4, 16) CASE(4, 8) CASE(4, 32)
#undef CASE
    return fail(PYFWI_E_INVALID, "no kernel for half order %d, tile rows %d", p->R, p->atz);
}

int grid_blocks(long long n)
{
    long long b = (n + 255) / 256;
    return (int)(b < PYFWI_REDUCE_SLOTS ? (b < 1 ? 1 : b) : PYFWI_REDUCE_SLOTS);
}

// ---- state addressing -------------------------------------------------------
struct Buf {
    float *base;       // state of slot 0
    long long stride;  // floats between slots
};

// Snapshots narrower than FP32 (BF16, or 24 bits: a BF16 plane plus a byte
// plane) hold the states of the segment being imaged.
bool bf16_snaps(const pyfwi_plan *p)
{
    return p->opt.checkpoint == PYFWI_CKPT_EXACT &&
           (p->opt.snapshot == PYFWI_SNAP_BF16 || p->opt.snapshot == PYFWI_SNAP_FP24);
}

bool fp24_snaps(const pyfwi_plan *p) { return bf16_snaps(p) && p->opt.snapshot == PYFWI_SNAP_FP24; }

// exact mode, per slot of the store: M restart states S_0, S_seg, ...
// S_{(M-1)seg}, then (FP32 snapshots) the seg states of the segment being
// imaged.  With BF16 snapshots the segment states live in the BF16 store and
// the FP32 chain that produces them runs in the two work states; with
// difference sets (p->qd) slot k of the segment holds the imaging's
// differences of S_{t_lo+k+1} instead of the state, and the chain runs in the
// work states as well.
// With overlap the segment states take two buffers: segment m uses buffer
// m % 2, so the recompute of segment m - 1 can fill one while the adjoint of
// segment m reads the other.
long long store_stride(const pyfwi_plan *p)
{
    return (long long)(p->M + (bf16_snaps(p) ? 0 : p->seg * (p->overlap ? 2 : 1))) * p->state;
}

// Stored state k (S_{t_lo+k+1}) of segment m, FP32 snapshots (or its
// difference set).
Buf seg_state(pyfwi_plan *p, void *ws, int m, int k)
{
    const int buf = p->overlap ? (m & 1) : 0;
    return {at<float>(ws, p->o_store) + (long long)(p->M + buf * p->seg + k) * p->state, store_stride(p)};
}

// exact mode: where state S_s of the current group lives during a pass
Buf exact_state(pyfwi_plan *p, void *ws, int s)
{
    float *store = at<float>(ws, p->o_store);
    float *work = at<float>(ws, p->o_work);
    long long sstride = store_stride(p);
    if (s == 0) return {store, sstride};
    if (p->M > 1 && s % p->seg == 0 && s / p->seg <= p->M - 1) return {store + (long long)(s / p->seg) * p->state, sstride};
    if (s > (p->M - 1) * p->seg && !bf16_snaps(p) && !p->qd)
        return seg_state(p, ws, p->M - 1, s - (p->M - 1) * p->seg - 1);
    return {work + (long long)(s & 1) * p->state, 2 * p->state};
}

// BF16 snapshot k (state S_{t_lo+k+1} of the segment being imaged)
__nv_bfloat16 *snap_at(pyfwi_plan *p, void *ws, int k)
{
    return at<__nv_bfloat16>(ws, p->o_store16) + (long long)k * p->state;
}

// its byte planes (24-bit snapshots; NULL for BF16)
unsigned char *snap8_at(pyfwi_plan *p, void *ws, int k)
{
    return fp24_snaps(p) ? at<unsigned char>(ws, p->o_store8) + (long long)k * p->state : nullptr;
}

StepArgs base_step(pyfwi_plan *p, void *ws)
{
    StepArgs a;
    memset(&a, 0, sizeof a);
    a.g = p->g;
    a.k = p->k;
    a.mat = at<float>(ws, p->o_mat);
    a.dampx = at<float>(ws, p->o_dampx);
    a.dampz = at<float>(ws, p->o_dampz);
    a.srcx = at<int>(ws, p->o_src);
    a.srcz = at<int>(ws, p->o_src) + p->geom.ns;
    a.rec_row = -1;
    a.lines = p->lines;
    a.nr = p->geom.nr;
    a.ns = p->geom.ns;
    a.trace_plane = (long long)p->geom.nt_ext * p->geom.ns * p->geom.nr;
    // the imaging domain (Grad, elastic.cl:470): difference sets cover it
    a.qlo = p->geom.npml + p->R;
    a.qhi_z = p->g.tnz - p->R - p->geom.npml;
    a.qhi_x = p->g.tnx - p->R - p->geom.npml;
    return a;
}

// A source sample whose four components are zero adds nothing (x + 0 = x,
// up to the sign of a zero), so its step skips the add and the forward
// kernel's barrier after it; the reference adds it (elastic_surface.cl:23-28).
bool src_adds(const float4 &v) { return v.x != 0.f || v.y != 0.f || v.z != 0.f || v.w != 0.f; }

float4 src_at(const pyfwi_plan *p, int inj)
{
    if (inj < 0 || inj >= (int)(p->src_vals.size() / 4)) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float *v = &p->src_vals[4 * (size_t)inj];
    return make_float4(v[0], v[1], v[2], v[3]);
}

// The persistent kernels run this call's time loops: the plan allows them
// and the stream is not being captured by the caller (cooperative launches
// stay out of the caller's graphs).
bool use_persist(const pyfwi_plan *p, cudaStream_t st)
{
    if (!p->persist) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone;
}

unsigned *barrier_words(void *ws) { return at<unsigned>(ws, BAR_OFF); }

// The forward pass of a group as persistent launches of up to
// PERSIST_CHUNK steps (layout: every step stored in FP32, M == 1).
int persist_pass(pyfwi_plan *p, void *ws, int s0, int n, float *traces, cudaStream_t st)
{
    const pyfwi_geometry &G = p->geom;
    StepArgs a = base_step(p, ws);
    a.shot0 = s0;
    a.traces = traces;
    FwdPersistArgs pa;
    memset(&pa, 0, sizeof pa);
    pa.a = a;
    pa.store = at<float>(ws, p->o_store);
    pa.sstride = store_stride(p);
    pa.state = p->state;
    pa.dt_scale = G.dt_scale;
    pa.nt_ext = G.nt_ext;
    pa.record = traces != nullptr;
    pa.nslots = n;
    pa.ntx = (p->g.tnx + TX - 1) / TX;
    pa.ntz = (p->g.tnz + p->tz - 1) / p->tz;
    pa.bar = barrier_words(ws);
    pa.err = at<int>(ws, ERR_OFF);
    pa.limit_ns = BARRIER_WAIT_NS;
    for (int t0 = 0; t0 < G.nt; t0 += PERSIST_CHUNK) {
        pa.t0 = t0;
        pa.t1 = std::min(t0 + PERSIST_CHUNK, G.nt);
        pa.k0 = t0 / G.dt_scale;
        pa.nk = (pa.t1 - 1) / G.dt_scale - pa.k0 + 1;
        for (int q = 0; q < pa.nk; ++q) pa.wav[q] = src_at(p, pa.k0 + q);
        CK(cudaMemsetAsync(pa.bar, 0, 2 * sizeof(unsigned), st));
        ProfileScope prof(p, st, 0, n * (pa.t1 - t0));
        int rc = PYFWI_E_INVALID;
#define CASE(R_, TZ_) \
    if (p->R == R_ && p->tz == TZ_) rc = launch_fwd_persist<R_, TZ_>(p, pa, st);
        CASE(2, 16) CASE(2, 8) CASE(2, 32) CASE(4, 16) CASE(4, 8) CASE(4, 32)
#undef CASE
        if (rc) return rc;
    }
    return PYFWI_OK;
}

int inj_row_of(const pyfwi_plan *p, int t);

// The adjoint steps nt-1 .. 1 of a group as one persistent launch (the first
// step's residual is injected by its own launch, as in adjoint_iter).
int persist_backward(pyfwi_plan *p, void *ws, AdjArgs &a, int n, cudaStream_t st)
{
    const pyfwi_geometry &G = p->geom;
    float *adj = at<float>(ws, p->o_adj);
    a.nslots = n;
    a.in = adj;
    a.in_stride = a.out_stride = 2 * p->state;
    a.inj_row = inj_row_of(p, G.nt - 1);
    int rc = launch_inject(p, a, n, st);
    if (rc) return rc;
    if (G.nt < 2) return PYFWI_OK;
    AdjPersistArgs pa;
    memset(&pa, 0, sizeof pa);
    pa.a = a;
    pa.a.fwd_stride = store_stride(p);  // S_{t+1} of slot q sits q store strides on
    pa.adj = adj;
    pa.store = at<float>(ws, p->o_store);
    pa.sstride = store_stride(p);
    pa.state = p->state;
    pa.t_hi = G.nt;
    pa.t_lo = 1;
    pa.ping0 = 0;
    pa.nt = G.nt;
    pa.nt_ext = G.nt_ext;
    pa.dt_scale = G.dt_scale;
    pa.ntx = (p->g.tnx + TX - 1) / TX;
    pa.ntz = (p->g.tnz + p->atz - 1) / p->atz;
    pa.bar = barrier_words(ws);
    pa.err = at<int>(ws, ERR_OFF);
    pa.limit_ns = BARRIER_WAIT_NS;
    CK(cudaMemsetAsync(pa.bar, 0, 2 * sizeof(unsigned), st));
    ProfileScope prof(p, st, 1, n * (G.nt - 1));
    rc = PYFWI_E_INVALID;
#define CASE(R_, TZ_)                                                                                          \
    if (p->R == R_ && p->atz == TZ_)                                                                           \
        rc = p->nacc == 6 ? launch_adj_persist_t<R_, TZ_, true>(p, pa, st) : launch_adj_persist_t<R_, TZ_, false>(p, pa, st);
    CASE(2, 16) CASE(2, 8) CASE(2, 32) CASE(4, 16) CASE(4, 8) CASE(4, 32)
#undef CASE
    return rc;
}

// One forward pass of a group (exact mode), optionally recording traces.
Buf work_state(pyfwi_plan *p, void *ws, int w)
{
    return {at<float>(ws, p->o_work) + (long long)w * p->state, 2 * p->state};
}

// Difference sets (p->qd): forward step t of segment m (first step t_lo)
// writes the velocity planes of S_{t+1} into slot t - t_lo and the stress
// planes of its input S_t into slot t - t_lo - 1; the stress planes of S_{t_lo}
// belong to the segment before, which computes them from its last state.
void set_diffs(pyfwi_plan *p, void *ws, StepArgs &a, int m, int t, int t_lo)
{
    a.qout = a.qin = nullptr;
    a.qout8 = a.qin8 = nullptr;
    if (!p->qd || t < t_lo) return;
    a.snap = nullptr;  // the difference sets take the snapshots' place
    a.snap8 = nullptr;
    if (p->qd == 2) {  // 24 bits: the BF16 and byte planes of the snapshot store
        a.qout = snap_at(p, ws, t - t_lo);
        a.qout8 = snap8_at(p, ws, t - t_lo);
        a.qin = t > t_lo ? snap_at(p, ws, t - t_lo - 1) : nullptr;
        a.qin8 = t > t_lo ? snap8_at(p, ws, t - t_lo - 1) : nullptr;
        a.q_stride = (long long)p->seg * p->state;
        return;
    }
    a.qout = seg_state(p, ws, m, t - t_lo).base;
    a.qin = t > t_lo ? seg_state(p, ws, m, t - t_lo - 1).base : nullptr;
    a.q_stride = store_stride(p);
}

// The stress planes of the last state S_{t_hi} of segment m (in a work
// state after the segment's steps), into its last slot.
int last_diffs(pyfwi_plan *p, void *ws, int m, int t_hi, int n, cudaStream_t st)
{
    const Buf s = work_state(p, ws, t_hi & 1);
    const int t_lo = m * p->seg, k = t_hi - 1 - t_lo;
    dim3 grid((p->g.tnx + 255) / 256, p->g.tnz, n);
    const int npml = p->geom.npml;
    if (p->qd == 2) {
        void *q = snap_at(p, ws, k);
        unsigned char *q8 = snap8_at(p, ws, k);
        const long long qs = (long long)p->seg * p->state;
        if (p->R == 4)
            qstress_kernel<4, 2><<<grid, 256, 0, st>>>(p->g, p->k, s.base, s.stride, q, q8, qs, npml);
        else
            qstress_kernel<2, 2><<<grid, 256, 0, st>>>(p->g, p->k, s.base, s.stride, q, q8, qs, npml);
    } else {
        float *q = seg_state(p, ws, m, k).base;
        if (p->R == 4)
            qstress_kernel<4, 1><<<grid, 256, 0, st>>>(p->g, p->k, s.base, s.stride, q, nullptr, store_stride(p), npml);
        else
            qstress_kernel<2, 1><<<grid, 256, 0, st>>>(p->g, p->k, s.base, s.stride, q, nullptr, store_stride(p), npml);
    }
    p->launches++;
    CKL();
    return PYFWI_OK;
}

int exact_pass(pyfwi_plan *p, void *ws, int s0, int n, float *traces, cudaStream_t st)
{
    Buf z = exact_state(p, ws, 0);
    for (int q = 0; q < n; ++q) CK(cudaMemsetAsync(z.base + q * z.stride, 0, p->state * sizeof(float), st));
    if (use_persist(p, st)) return persist_pass(p, ws, s0, n, traces, st);
    StepArgs a = base_step(p, ws);
    a.shot0 = s0;
    a.traces = traces;
    for (int t = 0; t < p->geom.nt; ++t) {
        Buf in = exact_state(p, ws, t), out = exact_state(p, ws, t + 1);
        a.in = in.base;
        a.in_stride = in.stride;
        a.out = out.base;
        a.out_stride = out.stride;
        bool inj = t % p->geom.dt_scale == 0;
        int k = t / p->geom.dt_scale;
        a.src = src_at(p, k);
        a.add_src = inj && src_adds(a.src);
        a.rec_row = (inj && traces && k < p->geom.nt_ext) ? k : -1;
        const int last_lo = (p->M - 1) * p->seg;
        a.snap = bf16_snaps(p) && t >= last_lo ? snap_at(p, ws, t - last_lo) : nullptr;
        a.snap8 = a.snap ? snap8_at(p, ws, t - last_lo) : nullptr;
        a.snap_stride = (long long)p->seg * p->state;
        set_diffs(p, ws, a, p->M - 1, t, last_lo);
        int rc = step_fwd(p, a, n, st, false, at<float>(ws, 0));
        if (rc) return rc;
    }
    if (p->qd) return last_diffs(p, ws, p->M - 1, p->geom.nt, n, st);
    return PYFWI_OK;
}

// reverse mode: checkpoint slot k of the group
Buf chp_state(pyfwi_plan *p, void *ws, int s0, int k)
{
    float *store = at<float>(ws, p->o_store);
    long long stride = (long long)p->chp.size() * p->state;
    return {store + (long long)s0 * stride + (long long)k * p->state, stride};
}

int reverse_pass(pyfwi_plan *p, void *ws, int s0, int n, float *traces, cudaStream_t st)
{
    // states stored after the steps listed in chp (wave_propagation.py:710-727)
    Buf cur = work_state(p, ws, 0);
    for (int q = 0; q < n; ++q) CK(cudaMemsetAsync(cur.base + q * cur.stride, 0, p->state * sizeof(float), st));
    int wcur = 0;  // work buffer holding the current state (-1: a checkpoint slot)
    size_t kc = 0;
    StepArgs a = base_step(p, ws);
    a.shot0 = s0;
    a.traces = traces;
    for (int t = 0; t < p->geom.nt; ++t) {
        Buf out;
        int wnext;
        if (kc < p->chp.size() && p->chp[kc] == t) {
            out = chp_state(p, ws, s0, (int)kc);
            ++kc;
            wnext = -1;
        } else {
            wnext = wcur == 0 ? 1 : 0;
            out = work_state(p, ws, wnext);
        }
        a.in = cur.base;
        a.in_stride = cur.stride;
        a.out = out.base;
        a.out_stride = out.stride;
        bool inj = t % p->geom.dt_scale == 0;
        int k = t / p->geom.dt_scale;
        a.src = src_at(p, k);
        a.add_src = inj && src_adds(a.src);
        a.rec_row = (inj && traces && k < p->geom.nt_ext) ? k : -1;
        int rc = step_fwd(p, a, n, st, false, at<float>(ws, 0));
        if (rc) return rc;
        cur = out;
        wcur = wnext;
    }
    return PYFWI_OK;
}

AdjArgs base_adj(pyfwi_plan *p, void *ws, const float *const *res)
{
    AdjArgs a;
    memset(&a, 0, sizeof a);
    a.g = p->g;
    a.k = p->k;
    a.mat = at<float>(ws, p->o_mat);
    a.dampx = at<float>(ws, p->o_dampx);
    a.dampz = at<float>(ws, p->o_dampz);
    a.npml = p->geom.npml;
    a.gacc = at<float>(ws, p->o_gacc);
    a.gacc_stride = (long long)p->nacc * p->g.plane;
    for (int c = 0; c < 5; ++c) a.res[c] = res ? res[c] : nullptr;
    a.nr = p->geom.nr;
    a.ns = p->geom.ns;
    a.lines = p->lines;
    return a;
}

// backward iteration t of the reference loop (wave_propagation.py:814-848)
// Residual row injected before backward step t (wave_propagation.py:814-824):
// t_src starts at nt_ext and steps down at every injection step, the row is
// t_src - 1 read with numpy's negative-index wrap; -1 if t injects nothing.
int inj_row_of(const pyfwi_plan *p, int t)
{
    const int d = p->geom.dt_scale;
    if (t < 0 || t % d) return -1;
    int row = p->geom.nt_ext - 1 - ((p->geom.nt - 1) / d - t / d);
    if (row < 0) row += p->geom.nt_ext;
    return row;
}

int adjoint_iter(pyfwi_plan *p, void *ws, AdjArgs &a, int t, int &t_src, int &ping, float *adj, int n, cudaStream_t st)
{
    if (t % p->geom.dt_scale == 0) t_src -= 1;
    // the tile kernel adds the residual of the next step (t - 1; step 0 never
    // runs) to its own output, so only the first backward step injects into
    // its input with a separate launch
    const bool epilogue = p->ast_w == 0;
    a.inj_row = (!epilogue || t == p->geom.nt - 1) ? inj_row_of(p, t) : -1;
    a.epi_row = epilogue && t - 1 >= 1 ? inj_row_of(p, t - 1) : -1;
    a.in = adj + (long long)ping * p->state;
    a.out = adj + (long long)(1 - ping) * p->state;
    a.in_stride = a.out_stride = 2 * p->state;
    int rc = step_adj(p, a, n, st, at<float>(ws, 0));
    ping = 1 - ping;
    return rc;
}

// Recompute of segment m (steps [t_lo, t_hi)) from its restart state into
// its segment buffer, on stream `st`.
int recompute_segment(pyfwi_plan *p, void *ws, int s0, int n, int m, cudaStream_t st)
{
    const pyfwi_geometry &G = p->geom;
    const int t_lo = m * p->seg, t_hi = std::min((m + 1) * p->seg, G.nt);
    StepArgs f = base_step(p, ws);
    f.shot0 = s0;
    Range range("pyfwi recompute segment");
    for (int t = t_lo; t < t_hi; ++t) {
        Buf in = t > t_lo ? seg_state(p, ws, m, t - t_lo - 1) : exact_state(p, ws, t), out = seg_state(p, ws, m, t - t_lo);
        if (p->qd) {  // the states in the work states, their differences in the segment
            if (t > t_lo) in = work_state(p, ws, t & 1);
            out = work_state(p, ws, (t + 1) & 1);
        }
        set_diffs(p, ws, f, m, t, t_lo);
        f.in = in.base;
        f.in_stride = in.stride;
        f.out = out.base;
        f.out_stride = out.stride;
        f.src = src_at(p, t / G.dt_scale);
        f.add_src = t % G.dt_scale == 0 && src_adds(f.src);
        f.rec_row = -1;
        int rc = step_fwd(p, f, n, st, false, at<float>(ws, 0));
        if (rc) return rc;
    }
    if (p->qd) return last_diffs(p, ws, m, t_hi, n, st);
    return PYFWI_OK;
}

// The exact-checkpoint backward pass of a group with the recompute of
// segment m - 1 on the plan's second stream while the adjoint of segment m
// runs on `st`: segment buffers alternate (m % 2); the recompute of m - 1
// waits for the adjoint of m + 1 to release its buffer, the adjoint of m for
// the recompute of m.  The results are those of the one-stream schedule.
int overlap_backward(pyfwi_plan *p, void *ws, AdjArgs &a, int s0, int n, int &t_src, int &ping, float *adj,
                     cudaStream_t st)
{
    const pyfwi_geometry &G = p->geom;
    if (!p->side) CK(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
    if ((int)p->ovev.size() < 2 * p->M + 1) {
        for (int q = (int)p->ovev.size(); q < 2 * p->M + 1; ++q) {
            cudaEvent_t e;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            p->ovev.push_back(e);
        }
    }
    cudaEvent_t start = p->ovev[2 * p->M];
    CK(cudaEventRecord(start, st));  // the side stream starts after everything queued so far
    CK(cudaStreamWaitEvent(p->side, start, 0));
    int rc;
    for (int m = p->M - 1; m >= 0; --m) {
        const int t_lo = m * p->seg, t_hi = std::min((m + 1) * p->seg, G.nt);
        if (m >= 1) {  // the recompute of segment m - 1, once the adjoint of m + 1 is done with its buffer
            if (m + 1 <= p->M - 1) CK(cudaStreamWaitEvent(p->side, p->ovev[2 * (m + 1) + 1], 0));
            rc = recompute_segment(p, ws, s0, n, m - 1, p->side);
            if (rc) return rc;
            CK(cudaEventRecord(p->ovev[2 * (m - 1)], p->side));
        }
        if (m < p->M - 1) CK(cudaStreamWaitEvent(st, p->ovev[2 * m], 0));
        Range range("pyfwi adjoint segment");
        for (int t = t_hi - 1; t >= std::max(t_lo, 1); --t) {
            a.fwd = seg_state(p, ws, m, t - t_lo).base;
            a.fwd_stride = store_stride(p);
            rc = adjoint_iter(p, ws, a, t, t_src, ping, adj, n, st);
            if (rc) return rc;
        }
        CK(cudaEventRecord(p->ovev[2 * m + 1], st));
    }
    return PYFWI_OK;
}

template <int R, int TZ>
int launch_exact(pyfwi_plan *p, const ExactArgs &a, int nslots, cudaStream_t s)
{
    dim3 grid((p->g.tnx + TX - 1) / TX, (p->g.tnz + TZ - 1) / TZ, nslots);
    const size_t sm = ExactShape<R, TZ>::FLOATS * sizeof(float);
    const int bf = a.s1h != nullptr;
    auto kern = bf ? exact_adj_step<R, TZ, true> : exact_adj_step<R, TZ, false>;
    static bool attr[2] = {false, false};
    if (!attr[bf]) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        attr[bf] = true;
    }
    kern<<<grid, NTHREADS, sm, s>>>(a);
    p->launches++;
    CKL();
    return PYFWI_OK;
}

// The exact adjoint of one group (exact checkpoints): for t = nt-1 .. 0 the
// transposed step from L_{t+1} to L_t with S_{t+1} and S_t from the segment
// store (FP32) or the BF16 snapshots, then the trace adjoint of step t.
int exact_backward(pyfwi_plan *p, void *ws, const float *const *residual, int s0, int n, cudaStream_t st)
{
    const pyfwi_geometry &G = p->geom;
    float *adj = at<float>(ws, p->o_adj);
    float *store = at<float>(ws, p->o_store);
    const long long sstride = store_stride(p);
    StepArgs f = base_step(p, ws);
    f.shot0 = s0;
    ExactArgs e;
    memset(&e, 0, sizeof e);
    e.g = p->g;
    e.k = p->k;
    e.mat = at<float>(ws, p->o_mat);
    e.dampx = at<float>(ws, p->o_dampx);
    e.dampz = at<float>(ws, p->o_dampz);
    e.gacc = at<float>(ws, p->o_gacc);
    e.gacc_stride = (long long)p->nacc * p->g.plane;
    e.shot0 = s0;
    e.srcx = at<int>(ws, p->o_src);
    e.srcz = at<int>(ws, p->o_src) + G.ns;
    e.in_stride = e.out_stride = 2 * p->state;
    e.s1_stride = e.s0_stride = sstride;
    int ping = 0, rc;
    for (int m = p->M - 1; m >= 0; --m) {
        const int t_lo = m * p->seg, t_hi = std::min((m + 1) * p->seg, G.nt);
        if (m < p->M - 1) {  // recompute segment m from its restart state
            for (int t = t_lo; t < t_hi; ++t) {
                Buf in = exact_state(p, ws, t), out;
                if (bf16_snaps(p)) {  // FP32 chain in the work states, BF16 copies into the snapshots
                    out = work_state(p, ws, (t + 1) & 1);
                    if (t > t_lo) in = work_state(p, ws, t & 1);
                    f.snap = snap_at(p, ws, t - t_lo);
                    f.snap8 = snap8_at(p, ws, t - t_lo);
                    f.snap_stride = (long long)p->seg * p->state;
                } else {
                    out = {store + (long long)(p->M + t - t_lo) * p->state, sstride};
                    if (t > t_lo) in = {store + (long long)(p->M + t - t_lo - 1) * p->state, sstride};
                }
                f.in = in.base;
                f.in_stride = in.stride;
                f.out = out.base;
                f.out_stride = out.stride;
                f.src = src_at(p, t / G.dt_scale);
                f.add_src = t % G.dt_scale == 0 && src_adds(f.src);
                f.rec_row = -1;
                rc = step_fwd(p, f, n, st, false, at<float>(ws, 0));
                if (rc) return rc;
            }
        }
        for (int t = t_hi - 1; t >= t_lo; --t) {
            if (bf16_snaps(p)) {
                // snapshot k holds S_{t_lo+k+1}; S_{t_lo} is the FP32 restart state
                e.s1h = snap_at(p, ws, t - t_lo);
                e.s1b = snap8_at(p, ws, t - t_lo);
                e.s1_stride = (long long)p->seg * p->state;
                e.s0h = t > t_lo ? snap_at(p, ws, t - t_lo - 1) : nullptr;
                e.s0b = t > t_lo ? snap8_at(p, ws, t - t_lo - 1) : nullptr;
                Buf s_t = exact_state(p, ws, t_lo);
                e.s0 = t > t_lo ? nullptr : s_t.base;
                e.s0_stride = t > t_lo ? e.s1_stride : s_t.stride;
            } else {
                Buf s_t = t > t_lo ? Buf{store + (long long)(p->M + t - t_lo - 1) * p->state, sstride}
                                   : exact_state(p, ws, t);
                e.s1 = store + (long long)(p->M + t - t_lo) * p->state;
                e.s0 = s_t.base;
                e.s0_stride = s_t.stride;
            }
            e.add_src = t % G.dt_scale == 0;
            e.src = src_at(p, t / G.dt_scale);
            e.in = adj + (long long)ping * p->state;
            e.out = adj + (long long)(1 - ping) * p->state;
            {
                ProfileScope prof(p, st, 1, n);
#define CASE(R_) \
    if (p->R == R_) rc = launch_exact<R_, 16>(p, e, n, st);
                rc = PYFWI_E_INVALID;
                CASE(2) CASE(4)
#undef CASE
                if (rc) return rc;
            }
            const int row = t / G.dt_scale;
            if (t % G.dt_scale == 0 && row < G.nt_ext) {
                inject_kernel<<<dim3(1, n), 256, 0, st>>>(p->g, e.out, 2 * p->state, s0, row, residual[0], residual[1],
                                                          residual[2], residual[3], residual[4], p->lines, G.ns, G.nr,
                                                          1);
                p->launches++;
                CKL();
            }
            ping = 1 - ping;
        }
    }
    return PYFWI_OK;
}

// Everything pyfwi_gradient enqueues (host state is updated by the caller).
// The fused misfit evaluation (pyfwi_misfit_gradient): per shot group,
// forward with traces, then the L2 residual of the group's traces, then the
// group's adjoint, so a layout of several groups models each group once.
struct Misfit {
    float *traces;        // [5][nt_ext][ns*nr] modelled traces (written)
    const float *obs[5];  // observed traces per field (nullable)
    float *res[5];        // adjoint sources (written where used)
    int mean_stress;      // the stress keys hold (txx + tzz) / 2
    double *misfit;
    double *partials;     // PYFWI_REDUCE_SLOTS block sums (workspace)
};

int misfit_group(pyfwi_plan *p, const Misfit &mf, int s0, int n, cudaStream_t st)
{
    const pyfwi_geometry &G = p->geom;
    MisfitArgs m;
    m.traces = mf.traces;
    for (int c = 0; c < 5; ++c) {
        m.obs[c] = mf.obs[c];
        m.res[c] = mf.res[c];
    }
    m.nt = G.nt_ext;
    m.ncol = (long long)G.ns * G.nr;
    m.col0 = (long long)s0 * G.nr;
    m.ncols = (long long)n * G.nr;
    m.plane = (long long)G.nt_ext * G.ns * G.nr;
    m.mean_stress = mf.mean_stress;
    m.exact = p->exact_adj;
    m.partials = mf.partials;
    const int nb = grid_blocks(m.nt * m.ncols);
    misfit_kernel<<<nb, 256, 0, st>>>(m);
    CKL();
    sum_partials_kernel<<<1, 32, 0, st>>>(mf.partials, nb, mf.misfit);
    p->launches += 2;
    CKL();
    return PYFWI_OK;
}

int gradient_enqueue(pyfwi_plan *p, void *ws, const float *const *residual, int32_t param, float *grad, float *raw,
                     cudaStream_t st, const Misfit *mf = nullptr)
{
    int rc;
    const pyfwi_geometry &G = p->geom;
    float *gacc = at<float>(ws, p->o_gacc);
    float *adj = at<float>(ws, p->o_adj);
    CK(cudaMemsetAsync(gacc, 0, (size_t)p->nacc * p->g.plane * p->G * sizeof(float), st));
    if (mf) {
        residual = mf->res;
        CK(cudaMemsetAsync(mf->traces, 0, 5 * (size_t)G.nt_ext * G.ns * G.nr * sizeof(float), st));
        CK(cudaMemsetAsync(mf->misfit, 0, sizeof(double), st));
    }
    AdjArgs a = base_adj(p, ws, residual);

    for (int grp = 0; grp < p->ngroups; ++grp) {
        Range range("pyfwi shot group: forward, residual, adjoint");
        int s0 = grp * p->G, n = std::min(p->G, G.ns - s0);
        a.shot0 = s0;
        if (mf) {  // model this group, then its residual
            rc = p->opt.checkpoint == PYFWI_CKPT_EXACT ? exact_pass(p, ws, s0, n, mf->traces, st)
                                                         : reverse_pass(p, ws, s0, n, mf->traces, st);
            if (rc) return rc;
            rc = misfit_group(p, *mf, s0, n, st);
            if (rc) return rc;
        } else if (p->opt.checkpoint == PYFWI_CKPT_EXACT && (p->ngroups > 1 || !p->fwd_valid)) {
            rc = exact_pass(p, ws, s0, n, nullptr, st);  // the states of this group are gone
            if (rc) return rc;
        }
        for (int q = 0; q < n; ++q) CK(cudaMemsetAsync(adj + 2 * q * p->state, 0, p->state * sizeof(float), st));
        int ping = 0, t_src = G.nt_ext;
        if (p->exact_adj) {
            const float *zero[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
            rc = exact_backward(p, ws, residual ? residual : zero, s0, n, st);
            if (rc) return rc;
        } else if (p->opt.checkpoint == PYFWI_CKPT_EXACT && use_persist(p, st)) {
            rc = persist_backward(p, ws, a, n, st);  // M == 1: every step stored
            if (rc) return rc;
        } else if (p->opt.checkpoint == PYFWI_CKPT_EXACT && p->overlap) {
            rc = overlap_backward(p, ws, a, s0, n, t_src, ping, adj, st);
            if (rc) return rc;
        } else if (p->opt.checkpoint == PYFWI_CKPT_EXACT) {
            StepArgs f = base_step(p, ws);
            f.shot0 = s0;
            for (int m = p->M - 1; m >= 0; --m) {
                int t_lo = m * p->seg, t_hi = std::min((m + 1) * p->seg, G.nt);
                if (m < p->M - 1 && p->qd) {
                    rc = recompute_segment(p, ws, s0, n, m, st);
                    if (rc) return rc;
                } else if (m < p->M - 1) {  // recompute segment m from its restart state
                    Range range("pyfwi recompute segment");
                    for (int t = t_lo; t < t_hi; ++t) {
                        Buf in = exact_state(p, ws, t), out;
                        if (bf16_snaps(p)) {
                            out = work_state(p, ws, (t + 1) & 1);
                            if (t > t_lo) in = work_state(p, ws, t & 1);
                            f.snap = snap_at(p, ws, t - t_lo);
                            f.snap8 = snap8_at(p, ws, t - t_lo);
                            f.snap_stride = (long long)p->seg * p->state;
                        } else {
                            out = seg_state(p, ws, m, t - t_lo);
                            if (t > t_lo) in = seg_state(p, ws, m, t - t_lo - 1);
                        }
                        f.in = in.base;
                        f.in_stride = in.stride;
                        f.out = out.base;
                        f.out_stride = out.stride;
                        bool inj = t % G.dt_scale == 0;
                        f.src = src_at(p, t / G.dt_scale);
                        f.add_src = inj && src_adds(f.src);
                        f.rec_row = -1;
                        rc = step_fwd(p, f, n, st, false, at<float>(ws, 0));
                        if (rc) return rc;
                    }
                }
                Range range("pyfwi adjoint segment");
                for (int t = t_hi - 1; t >= std::max(t_lo, 1); --t) {
                    // forward state after step t: S_{t+1}
                    if (bf16_snaps(p)) {
                        a.fwd = nullptr;
                        a.fwd16 = snap_at(p, ws, t - t_lo);
                        a.fwd8 = snap8_at(p, ws, t - t_lo);
                        a.fwd_stride = (long long)p->seg * p->state;
                    } else {
                        a.fwd = seg_state(p, ws, m, t - t_lo).base;
                        a.fwd_stride = store_stride(p);
                    }
                    rc = adjoint_iter(p, ws, a, t, t_src, ping, adj, n, st);
                    if (rc) return rc;
                }
            }
        } else {
            // reference chpr < 100 scheme (wave_propagation.py:761-812)
            int nchp = (int)p->chp.size(), chpc = nchp - 1, wlast = 1;
            Buf cur = {nullptr, 0};
            StepArgs f = base_step(p, ws);
            f.shot0 = s0;
            for (int t = G.nt - 1; t > 0; --t) {
                int kk = chpc >= 0 ? chpc : chpc + nchp;
                if (t == p->chp[kk]) {
                    cur = chp_state(p, ws, s0, kk);
                    chpc -= 1;
                } else {
                    if (!cur.base) return fail(PYFWI_E_STATE, "reverse schedule has no starting checkpoint");
                    int w = 1 - wlast;
                    Buf out = work_state(p, ws, w);
                    f.in = cur.base;
                    f.in_stride = cur.stride;
                    f.out = out.base;
                    f.out_stride = out.stride;
                    rc = step_fwd(p, f, n, st, true, at<float>(ws, 0));
                    if (rc) return rc;
                    cur = out;
                    wlast = w;
                }
                a.fwd = cur.base;
                a.fwd_stride = cur.stride;
                rc = adjoint_iter(p, ws, a, t, t_src, ping, adj, n, st);
                if (rc) return rc;
            }
        }
    }

    const long long nplane = (long long)p->nacc * p->g.plane;
    if (acc_slots(p, p->G) > 1) {
        reduce_slots_kernel<<<grid_blocks(nplane), 256, 0, st>>>(gacc, nplane, acc_slots(p, p->G), nplane);
        p->launches++;
        CKL();
    }
    if (raw) {
        if (p->nacc < 6)
            CK(cudaMemsetAsync(raw, 0, 6 * (size_t)p->g.tnz * p->g.tnx * sizeof(float), st));
        raw_out_kernel<<<grid_blocks((long long)p->nacc * p->g.tnz * p->g.tnx), 256, 0, st>>>(p->g, gacc, p->nacc, raw);
        p->launches++;
        CKL();
    }
    if (p->exact_adj) {
        const long long nm = (long long)G.nz * G.nx;
        exact_post_kernel<<<grid_blocks(nm), 256, 0, st>>>(p->g, G.nz, G.nx, G.npml, gacc, at<float>(ws, p->o_mat),
                                                           param == PYFWI_PARAM_DV ? 1 : 0, grad);
        p->launches++;
        CKL();
        return PYFWI_OK;
    }
    PostArgs pa;
    pa.g = p->g;
    pa.nz = G.nz;
    pa.nx = G.nx;
    pa.npml = G.npml;
    pa.r0 = G.mask_row0;
    pa.r1 = G.mask_row1;
    pa.c0 = G.mask_col0;
    pa.c1 = G.mask_col1;
    pa.energy = p->nacc == 6;
    pa.param = param;
    pa.gacc = gacc;
    pa.mat = at<float>(ws, p->o_mat);
    pa.fmax_bits = at<int>(ws, p->o_hdr) + 4;
    pa.out = grad;
    CK(cudaMemsetAsync(pa.fmax_bits, 0, 3 * sizeof(int), st));
    long long nm = (long long)G.nz * G.nx;
    factor_max_kernel<<<grid_blocks(nm), 256, 0, st>>>(pa);
    p->launches++;
    CKL();
    post_kernel<<<grid_blocks(nm), 256, 0, st>>>(pa);
    p->launches++;
    CKL();
    return PYFWI_OK;
}

int forward_enqueue(pyfwi_plan *p, void *ws, float *traces, cudaStream_t st)
{
    if (traces)
        CK(cudaMemsetAsync(traces, 0, 5 * (size_t)p->geom.nt_ext * p->geom.ns * p->geom.nr * sizeof(float), st));
    for (int grp = 0; grp < p->ngroups; ++grp) {
        Range range("pyfwi shot group: forward");
        int s0 = grp * p->G, n = std::min(p->G, p->geom.ns - s0);
        int rc = p->opt.checkpoint == PYFWI_CKPT_EXACT ? exact_pass(p, ws, s0, n, traces, st)
                                                         : reverse_pass(p, ws, s0, n, traces, st);
        if (rc) return rc;
    }
    return PYFWI_OK;
}

// Kernel launches of one pyfwi_forward (backward false) or one gradient
// call (backward true), from the layout: per shot group nt forward steps,
// and for a gradient the recomputed steps, nt adjoint steps and a few more.
long long call_launches(const pyfwi_plan *p, bool backward)
{
    const long long nt = p->geom.nt, per = backward ? 2 * nt + (long long)(p->M - 1) * p->seg + p->M + 16 : nt + 4;
    return (long long)p->ngroups * per;
}

// Replay `enqueue` as a CUDA graph: captured once per distinct key (the
// pointers and values the launches bake in) on the plan's own stream, then
// launched on the caller's stream.  A caller stream that is being captured
// already (the caller builds its own graph) gets the launches directly, and
// so does a call of more than PYFWI_GRAPH_MAX_LAUNCHES launches (a graph of
// millions of nodes exhausts host memory while it is captured; its launches
// are long enough that issuing them costs little).
template <typename F>
int run_graph(pyfwi_plan *p, pyfwi_plan::GraphCache &c, const std::vector<uintptr_t> &key, cudaStream_t st,
              long long launches, F enqueue)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone || launches > PYFWI_GRAPH_MAX_LAUNCHES) return enqueue(st);
    if (!c.exec || c.key != key) {
        if (c.exec) {
            cudaGraphExecDestroy(c.exec);
            c.exec = nullptr;
        }
        if (!p->cap) CK(cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking));
        const long long l0 = p->launches;
        CK(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue(p->cap);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(p->cap, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return fail(PYFWI_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&c.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            c.exec = nullptr;
            return fail(PYFWI_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        }
        c.key = key;
        c.launches = p->launches - l0;
        p->launches = l0;
    }
    CK(cudaGraphLaunch(c.exec, st));
    p->launches += c.launches;
    return PYFWI_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char *pyfwi_last_error(void) { return g_err.c_str(); }

int pyfwi_abi_version(void) { return PYFWI_ABI_VERSION; }

int pyfwi_tile_count(int32_t half_order) { return (half_order == 2 || half_order == 4) ? N_TILES : 0; }

int pyfwi_plan_create(const pyfwi_geometry *geom, const int32_t *srcx, const int32_t *srcz, const pyfwi_options *opt,
                      pyfwi_plan **out)
{
    if (!geom || !srcx || !srcz || !opt || !out) return fail(PYFWI_E_INVALID, "NULL argument");
    *out = nullptr;
    const pyfwi_geometry &G = *geom;
    if (G.half_order != 2 && G.half_order != 4) return fail(PYFWI_E_INVALID, "half_order must be 2 or 4");
    if (G.nz < 1 || G.nx < 1 || G.npml < 0 || G.nt < 1 || G.nt_ext < 1 || G.dt_scale < 1 || G.ns < 1 || G.nr < 1)
        return fail(PYFWI_E_INVALID, "bad grid/time/shot sizes");
    if (G.n_lines < 1 || G.n_lines > 3) return fail(PYFWI_E_INVALID, "n_lines must be 1..3");
    const int tnz = G.nz + 2 * G.npml, tnx = G.nx + 2 * G.npml;
    for (int l = 0; l < G.n_lines; ++l) {
        const pyfwi_rec_line &L = G.lines[l];
        if (L.count < 0 || L.slot0 < 0 || L.slot0 + L.count > G.nr) return fail(PYFWI_E_INVALID, "line %d slots", l);
        if ((L.drow == 0) == (L.dcol == 0) || L.drow < 0 || L.dcol < 0)
            return fail(PYFWI_E_INVALID, "line %d: exactly one of drow, dcol must be positive", l);
    }
    for (int s = 0; s < G.ns; ++s)
        if (srcx[s] < 0 || srcx[s] >= tnx || srcz[s] < 0 || srcz[s] >= tnz)
            return fail(PYFWI_E_INVALID, "source %d at (%d, %d) is outside the %dx%d grid", s, srcz[s], srcx[s], tnz, tnx);
    if (opt->checkpoint != PYFWI_CKPT_EXACT && opt->checkpoint != PYFWI_CKPT_REVERSE)
        return fail(PYFWI_E_INVALID, "unknown checkpoint mode");
    if (opt->checkpoint == PYFWI_CKPT_REVERSE) {
        if (opt->nchp < 1 || !opt->chp) return fail(PYFWI_E_INVALID, "reverse mode needs a checkpoint list");
        for (int q = 0; q < opt->nchp; ++q)
            if (opt->chp[q] < 0 || opt->chp[q] >= G.nt || (q && opt->chp[q] <= opt->chp[q - 1]))
                return fail(PYFWI_E_INVALID, "checkpoint steps must be increasing and inside [0, nt)");
        if (opt->chp[opt->nchp - 1] != G.nt - 1) return fail(PYFWI_E_INVALID, "last checkpoint must be step nt-1");
    }
    if (opt->snapshot != PYFWI_SNAP_FP32 && opt->snapshot != PYFWI_SNAP_BF16 && opt->snapshot != PYFWI_SNAP_FP24)
        return fail(PYFWI_E_INVALID, "unknown snapshot format");
    if (opt->snapshot != PYFWI_SNAP_FP32 && opt->checkpoint != PYFWI_CKPT_EXACT)
        return fail(PYFWI_E_INVALID, "bf16 and 24-bit snapshots need the exact checkpoint mode");
    if (opt->tile < 0 || opt->tile >= N_TILES) return fail(PYFWI_E_INVALID, "tile variant out of range");
    if (opt->adj_tile < 0 || opt->adj_tile > N_TILES) return fail(PYFWI_E_INVALID, "adj_tile out of range");
    if (opt->adjoint != PYFWI_ADJOINT_REFERENCE && opt->adjoint != PYFWI_ADJOINT_EXACT)
        return fail(PYFWI_E_INVALID, "unknown adjoint kind");
    if (opt->adjoint == PYFWI_ADJOINT_EXACT && (opt->checkpoint != PYFWI_CKPT_EXACT || opt->energy))
        return fail(PYFWI_E_INVALID, "the exact adjoint needs exact checkpoints and no energy terms");
    if (opt->chunk < 0) return fail(PYFWI_E_INVALID, "chunk must be >= 0");

    pyfwi_plan *p = new pyfwi_plan();
    p->geom = G;
    p->opt = *opt;
    p->srcx.assign(srcx, srcx + G.ns);
    p->srcz.assign(srcz, srcz + G.ns);
    if (opt->checkpoint == PYFWI_CKPT_REVERSE) p->chp.assign(opt->chp, opt->chp + opt->nchp);
    p->opt.chp = nullptr;
    p->R = G.half_order;
    p->tz = TILE_TZ[opt->tile];
    p->st_w = STREAM_W[opt->tile];
    p->ftma = FWD_TMA[opt->tile];
    const int av = opt->adj_tile ? opt->adj_tile - 1 : opt->tile;
    p->atz = TILE_TZ[av];
    p->ast_w = STREAM_W[av];
    p->ans = ADJ_NS[av];
    p->apf = ADJ_PREFETCH[av] && !opt->energy;
    if (opt->snapshot != PYFWI_SNAP_FP32 && opt->checkpoint == PYFWI_CKPT_EXACT) {
        // snapshots are read by the 16-row tile adjoint kernel with one shot per CTA
        p->ast_w = 0;
        p->atz = TILE_TZ[0];
        p->ans = 1;
    }
    p->chunk_opt = opt->chunk;
    p->nacc = opt->energy ? 6 : 3;
    p->exact_adj = opt->adjoint == PYFWI_ADJOINT_EXACT;
    p->g.tnz = tnz;
    p->g.tnx = tnx;
    p->g.pitch = (int)up((size_t)tnx + 2 * XO, 32);
    p->g.rows = tnz + 2 * ZO;
    p->g.plane = (long long)p->g.pitch * p->g.rows;
    p->state = 5 * p->g.plane;
    for (int q = 0; q < 4; ++q) {
        p->k.cx[q] = G.c[q] / G.dh;
        p->k.cz[q] = G.c[q] / G.dh;
    }
    p->k.dt = G.dt;
    memset(&p->lines, 0, sizeof p->lines);
    p->lines.n = G.n_lines;
    for (int l = 0; l < G.n_lines; ++l) {
        const pyfwi_rec_line &L = G.lines[l];
        p->lines.row0[l] = L.row0;
        p->lines.col0[l] = L.col0;
        p->lines.drow[l] = L.drow;
        p->lines.dcol[l] = L.dcol;
        p->lines.count[l] = L.count;
        p->lines.slot0[l] = L.slot0;
        p->lines.vzx[l] = L.vz_from_vx;
    }
    p->G = opt->shot_batch > 0 && opt->shot_batch < G.ns ? opt->shot_batch : G.ns;
    p->ngroups = (G.ns + p->G - 1) / p->G;
    p->seg = opt->segment > 0 && opt->segment < G.nt ? opt->segment : G.nt;
    p->M = (G.nt + p->seg - 1) / p->seg;
    p->n_inj = (G.nt + G.dt_scale - 1) / G.dt_scale;
    // persistent time loops: every step stored in FP32 (one segment), tile
    // kernels with one shot per adjoint CTA, the reference adjoint
    p->persist = opt->persist && opt->checkpoint == PYFWI_CKPT_EXACT && p->M == 1 &&
                 opt->snapshot == PYFWI_SNAP_FP32 && !p->exact_adj && !p->st_w && !p->ftma && !p->ast_w &&
                 p->ans == 1;
    if (p->persist) p->opt.graph = 0;  // a few launches per call: nothing to replay
    // recompute beside the adjoint: exact checkpoints in FP32 with recompute
    // segments, the reference adjoint
    p->overlap = opt->overlap && opt->checkpoint == PYFWI_CKPT_EXACT && p->M > 1 && opt->snapshot == PYFWI_SNAP_FP32 &&
                 !p->exact_adj;
    // difference sets in the segment store: exact checkpoints in FP32, the
    // reference adjoint without energy terms, the plain tile kernels
    const bool qd = opt->store_diffs && opt->checkpoint == PYFWI_CKPT_EXACT &&
                    (opt->snapshot == PYFWI_SNAP_FP32 || opt->snapshot == PYFWI_SNAP_FP24) && !p->exact_adj &&
                    p->nacc == 3 && !p->persist && !p->st_w && !p->ftma && !p->ast_w && p->ans == 1 && !p->apf &&
                    G.npml + p->R >= 4;  // whole 4-column groups are written: the imaged columns end 3 short of tnx
    p->qd = qd ? (opt->snapshot == PYFWI_SNAP_FP24 ? 2 : 1) : 0;

    const size_t pf = (size_t)p->g.plane * sizeof(float), sb = (size_t)p->state * sizeof(float);
    // regions holding planes start on a row of the workspace (a multiple of
    // the row bytes and of ALIGN), so every plane is a run of whole rows of
    // the workspace tensor the streaming kernels copy from
    const size_t rowb = (size_t)p->g.pitch * sizeof(float), ra = rowb % ALIGN ? rowb * 2 : rowb;
    auto upr = [ra](size_t x) { return (x + ra - 1) / ra * ra; };
    size_t o = 0;
    p->o_hdr = o;
    o += ALIGN;
    p->o_src = o;
    o += up(2 * (size_t)G.ns * sizeof(int));
    p->o_red = o;
    o += up(PYFWI_REDUCE_SLOTS * sizeof(double));
    o = upr(o);
    p->o_mat = o;
    o += up(4 * pf);
    p->o_dampx = o;
    o += up((size_t)p->g.pitch * sizeof(float));
    p->o_dampz = o;
    o += up((size_t)p->g.rows * sizeof(float));
    o = upr(o);
    p->o_work = o;
    o += up(2 * sb * p->G);
    o = upr(o);
    p->o_adj = o;
    o += up(2 * sb * p->G);
    o = upr(o);
    p->o_gacc = o;
    o += up((size_t)p->nacc * pf * p->G);
    o = upr(o);
    p->o_store = o;
    if (opt->checkpoint == PYFWI_CKPT_EXACT)
        o += up((size_t)store_stride(p) * sizeof(float) * p->G);
    else
        o += up(p->chp.size() * sb * G.ns);
    o = upr(o);
    p->o_store16 = o;
    if (bf16_snaps(p)) o += up((size_t)p->seg * p->state * sizeof(__nv_bfloat16) * p->G);
    p->o_store8 = o;
    if (fp24_snaps(p)) o += up((size_t)p->seg * p->state * p->G);
    p->total = o;
    *out = p;
    return PYFWI_OK;
}

int pyfwi_plan_destroy(pyfwi_plan *plan)
{
    if (plan) {
        for (auto &e : plan->events) {
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
        if (plan->gfwd.exec) cudaGraphExecDestroy(plan->gfwd.exec);
        if (plan->ggrad.exec) cudaGraphExecDestroy(plan->ggrad.exec);
        if (plan->gmis.exec) cudaGraphExecDestroy(plan->gmis.exec);
        if (plan->cap) cudaStreamDestroy(plan->cap);
        for (auto e : plan->ovev) cudaEventDestroy(e);
        if (plan->side) cudaStreamDestroy(plan->side);
    }
    delete plan;
    return PYFWI_OK;
}

int pyfwi_profile_enable(pyfwi_plan *p, int32_t enable)
{
    if (!p) return fail(PYFWI_E_INVALID, "NULL plan");
    p->profiling = enable != 0;
    return PYFWI_OK;
}

int pyfwi_profile_read(pyfwi_plan *p, int32_t kind, int64_t *launches, double *ms, double *cells)
{
    if (!p || !launches || !ms || !cells) return fail(PYFWI_E_INVALID, "NULL argument");
    if (kind < 0 || kind > 2) return fail(PYFWI_E_INVALID, "kind must be 0, 1 or 2");
    // fold every pending event pair into the per-kind totals
    for (size_t q = 0; q < p->ev_used; ++q) {
        auto &e = p->events[q];
        CK(cudaEventSynchronize(e.b));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, e.a, e.b));
        p->prof_n[e.kind] += 1;
        p->prof_ms[e.kind] += t;
        p->prof_cells[e.kind] += e.cells;
    }
    p->ev_used = 0;
    *launches = p->prof_n[kind];
    *ms = p->prof_ms[kind];
    *cells = p->prof_cells[kind];
    p->prof_n[kind] = 0;
    p->prof_ms[kind] = 0.0;
    p->prof_cells[kind] = 0.0;
    return PYFWI_OK;
}

int pyfwi_workspace_size(const pyfwi_plan *p, size_t *bytes)
{
    if (!p || !bytes) return fail(PYFWI_E_INVALID, "NULL argument");
    *bytes = p->total;
    return PYFWI_OK;
}

int pyfwi_launch_count(const pyfwi_plan *p, int64_t *count)
{
    if (!p || !count) return fail(PYFWI_E_INVALID, "NULL argument");
    *count = p->launches;
    return PYFWI_OK;
}

int pyfwi_plan_flags(const pyfwi_plan *p, int32_t *flags)
{
    if (!p || !flags) return fail(PYFWI_E_INVALID, "NULL argument");
    *flags = (p->persist ? 1 : 0) | (p->overlap ? 2 : 0) | (p->qd ? 4 : 0);
    return PYFWI_OK;
}

int pyfwi_device_error(pyfwi_plan *p, void *ws, size_t bytes, int32_t *code, void *stream)
{
    if (!p || !code) return fail(PYFWI_E_INVALID, "NULL argument");
    int rc = check_ws(p, ws, bytes);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int32_t v = 0;
    int *word = at<int>(ws, ERR_OFF);
    CK(cudaMemcpyAsync(&v, word, sizeof v, cudaMemcpyDeviceToHost, st));
    CK(cudaMemsetAsync(word, 0, sizeof v, st));
    CK(cudaStreamSynchronize(st));
    *code = v;
    if (v)
        return fail(PYFWI_E_TIMEOUT, "device error word %d: %s", v,
                    v == 3 ? "a persistent kernel gave up at a grid barrier" : "a streaming kernel stopped early");
    return PYFWI_OK;
}

int pyfwi_checkpoint_states(pyfwi_plan *p, void *ws, size_t bytes, float *out, void *stream)
{
    if (!p || !out) return fail(PYFWI_E_INVALID, "NULL argument");
    int rc = check_ws(p, ws, bytes);
    if (rc) return rc;
    if (p->opt.checkpoint != PYFWI_CKPT_REVERSE)
        return fail(PYFWI_E_STATE, "only reverse-mode plans keep the checkpoint states");
    if (!p->fwd_valid) return fail(PYFWI_E_STATE, "pyfwi_checkpoint_states needs a pyfwi_forward first");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Grid &g = p->g;
    // store: per shot, per checkpoint, one state of 5 planes (chp_state)
    const long long nplanes = (long long)p->geom.ns * (long long)p->chp.size() * 5;
    const float *store = at<float>(ws, p->o_store);
    const long long cells = (long long)g.tnz * g.tnx;
    for (long long q = 0; q < nplanes; ++q)
        CK(cudaMemcpy2DAsync(out + q * cells, (size_t)g.tnx * sizeof(float),
                             store + q * g.plane + (long long)ZO * g.pitch + XO, (size_t)g.pitch * sizeof(float),
                             (size_t)g.tnx * sizeof(float), (size_t)g.tnz, cudaMemcpyDeviceToDevice, st));
    return PYFWI_OK;
}

int pyfwi_frame_check(pyfwi_plan *p, void *ws, size_t bytes, int64_t *nonzero, void *stream)
{
    if (!p || !nonzero) return fail(PYFWI_E_INVALID, "NULL argument");
    int rc = check_ws(p, ws, bytes);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto *cnt = at<unsigned long long>(ws, CHECK_OFF);
    CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st));
    const long long G5 = 5LL * p->G;
    long long store_planes = p->opt.checkpoint == PYFWI_CKPT_EXACT
                                 ? store_stride(p) / p->g.plane * p->G
                                 : (long long)p->chp.size() * 5 * p->geom.ns;
    const struct {
        size_t off;
        long long planes;
    } regions[] = {{p->o_mat, 4}, {p->o_work, 2 * G5}, {p->o_adj, 2 * G5}, {p->o_gacc, (long long)p->nacc * p->G},
                   {p->o_store, store_planes}};
    for (const auto &r : regions) {
        if (r.planes <= 0) continue;
        frame_check_kernel<<<4 * 148, 256, 0, st>>>(at<float>(ws, r.off), r.planes, p->g, cnt);
        CKL();
    }
    unsigned long long v = 0;
    CK(cudaMemcpyAsync(&v, cnt, sizeof v, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *nonzero = (int64_t)v;
    return PYFWI_OK;
}

int pyfwi_wait_selftest(pyfwi_plan *p, void *ws, size_t bytes, int64_t limit_ns, void *stream)
{
    if (!p) return fail(PYFWI_E_INVALID, "NULL plan");
    if (limit_ns < 1000 || limit_ns > 10000000000LL) return fail(PYFWI_E_INVALID, "limit_ns outside [1e3, 1e10]");
    int rc = check_ws(p, ws, bytes);
    if (rc) return rc;
    wait_selftest_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(at<int>(ws, ERR_OFF),
                                                                          (unsigned long long)limit_ns);
    CKL();
    return PYFWI_OK;
}

int pyfwi_barrier_selftest(pyfwi_plan *p, void *ws, size_t bytes, int64_t limit_ns, void *stream)
{
    if (!p) return fail(PYFWI_E_INVALID, "NULL plan");
    int rc = check_ws(p, ws, bytes);
    if (rc) return rc;
    if (limit_ns < 1000 || limit_ns > 10000000000LL) return fail(PYFWI_E_INVALID, "limit_ns out of range");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CK(cudaMemsetAsync(barrier_words(ws), 0, 2 * sizeof(unsigned), st));
    barrier_selftest_kernel<<<2, 32, 0, st>>>(barrier_words(ws), at<int>(ws, ERR_OFF), (unsigned long long)limit_ns);
    p->launches++;
    CKL();
    return PYFWI_OK;
}

int pyfwi_set_model(pyfwi_plan *p, void *ws, size_t bytes, const float *vp, const float *vs, const float *rho,
                    const float *damp_x, const float *damp_z, void *stream)
{
    if (!p || !vp || !vs || !rho || !damp_x || !damp_z) return fail(PYFWI_E_INVALID, "NULL argument");
    int rc = check_ws(p, ws, bytes);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (p->ws_initialised != ws) {
        // frames and padding of every plane must read as zero; the source
        // cells are constant for the plan (later calls copy nothing from the
        // host, so they may be captured in a CUDA graph)
        CK(cudaMemsetAsync(ws, 0, p->total, st));
        CK(cudaMemcpyAsync(at<int>(ws, p->o_src), p->srcx.data(), p->geom.ns * sizeof(int), cudaMemcpyHostToDevice,
                           st));
        CK(cudaMemcpyAsync(at<int>(ws, p->o_src) + p->geom.ns, p->srcz.data(), p->geom.ns * sizeof(int),
                           cudaMemcpyHostToDevice, st));
        p->ws_initialised = ws;
    }
    int *vmax = at<int>(ws, p->o_hdr);
    CK(cudaMemsetAsync(vmax, 0, sizeof(int), st));
    long long nm = (long long)p->geom.nz * p->geom.nx;
    vp_max_kernel<<<grid_blocks(nm), 256, 0, st>>>(vp, nm, vmax);
    p->launches++;
    CKL();
    model_kernel<<<grid_blocks((long long)p->g.tnz * p->g.tnx), 256, 0, st>>>(p->g, p->geom.nz, p->geom.nx, p->geom.npml,
                                                                              vp, vs, rho, at<float>(ws, p->o_mat));
    p->launches++;
    CKL();
    damp_kernel<<<grid_blocks(p->g.pitch + p->g.rows), 256, 0, st>>>(p->g, damp_x, damp_z, vmax,
                                                                    at<float>(ws, p->o_dampx), at<float>(ws, p->o_dampz));
    p->launches++;
    CKL();
    p->model_set = true;
    p->fwd_valid = false;
    return PYFWI_OK;
}

int pyfwi_forward(pyfwi_plan *p, void *ws, size_t bytes, const float *src_vals, int32_t n_src, float *traces,
                  void *stream)
{
    if (!p || (n_src > 0 && !src_vals) || n_src < 0) return fail(PYFWI_E_INVALID, "bad argument");
    int rc = check_ws(p, ws, bytes);
    if (rc) return rc;
    if (!p->model_set) return fail(PYFWI_E_STATE, "pyfwi_set_model must come first");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    p->src_vals.assign(src_vals, src_vals + 4 * (size_t)n_src);
    std::vector<uintptr_t> key = {reinterpret_cast<uintptr_t>(ws), reinterpret_cast<uintptr_t>(traces)};
    for (float v : p->src_vals) {
        uint32_t b;
        memcpy(&b, &v, 4);
        key.push_back(b);
    }
    rc = p->opt.graph && !p->profiling
             ? run_graph(p, p->gfwd, key, st, call_launches(p, false), [&](cudaStream_t s) { return forward_enqueue(p, ws, traces, s); })
             : forward_enqueue(p, ws, traces, st);
    if (rc) return rc;
    p->fwd_valid = true;
    return PYFWI_OK;
}

int pyfwi_gradient(pyfwi_plan *p, void *ws, size_t bytes, const float *const *residual, int32_t param, float *grad,
                   float *raw, void *stream)
{
    if (!p || !grad || (param != PYFWI_PARAM_LMD && param != PYFWI_PARAM_DV)) return fail(PYFWI_E_INVALID, "bad argument");
    int rc = check_ws(p, ws, bytes);
    if (rc) return rc;
    if (!p->fwd_valid) return fail(PYFWI_E_STATE, "pyfwi_gradient needs a pyfwi_forward of the current model first");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<uintptr_t> key = {reinterpret_cast<uintptr_t>(ws), reinterpret_cast<uintptr_t>(grad),
                                  reinterpret_cast<uintptr_t>(raw), (uintptr_t)param, (uintptr_t)p->fwd_valid};
    for (int c = 0; c < 5; ++c) key.push_back(reinterpret_cast<uintptr_t>(residual ? residual[c] : nullptr));
    for (float v : p->src_vals) {
        uint32_t b;
        memcpy(&b, &v, 4);
        key.push_back(b);
    }
    rc = p->opt.graph && !p->profiling
             ? run_graph(p, p->ggrad, key, st, call_launches(p, true),
                         [&](cudaStream_t s) { return gradient_enqueue(p, ws, residual, param, grad, raw, s); })
             : gradient_enqueue(p, ws, residual, param, grad, raw, st);
    if (rc) return rc;
    if (p->opt.checkpoint == PYFWI_CKPT_EXACT && p->M > 1) p->fwd_valid = false;  // last segment overwritten
    if (p->opt.checkpoint == PYFWI_CKPT_EXACT && p->ngroups > 1) p->fwd_valid = true;  // passes were redone anyway
    return PYFWI_OK;
}

int pyfwi_misfit_gradient(pyfwi_plan *p, void *ws, size_t bytes, const float *src_vals, int32_t n_src,
                          const float *const *observed, int32_t mean_stress, float *const *adjoint_source,
                          int32_t param, float *traces, float *grad, double *misfit, void *stream)
{
    if (!p || !observed || !adjoint_source || !traces || !grad || !misfit || (n_src > 0 && !src_vals) || n_src < 0 ||
        (param != PYFWI_PARAM_LMD && param != PYFWI_PARAM_DV))
        return fail(PYFWI_E_INVALID, "bad argument");
    int rc = check_ws(p, ws, bytes);
    if (rc) return rc;
    if (!p->model_set) return fail(PYFWI_E_STATE, "pyfwi_set_model must come first");
    Misfit mf;
    mf.traces = traces;
    mf.mean_stress = mean_stress != 0;
    mf.misfit = misfit;
    mf.partials = at<double>(ws, p->o_red);
    bool any = false;
    for (int c = 0; c < 5; ++c) {
        mf.obs[c] = observed[c];
        mf.res[c] = adjoint_source[c];
        if (observed[c] && !adjoint_source[c]) return fail(PYFWI_E_INVALID, "field %d observed but no adjoint buffer", c);
        any = any || observed[c];
    }
    if (!any) return fail(PYFWI_E_INVALID, "no observed field");
    if (mf.mean_stress && ((observed[TXX] && !adjoint_source[TZZ]) || (observed[TZZ] && !adjoint_source[TXX])))
        return fail(PYFWI_E_INVALID, "mean_stress needs adjoint buffers for both stress fields");
    p->src_vals.assign(src_vals, src_vals + 4 * (size_t)n_src);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<uintptr_t> key = {reinterpret_cast<uintptr_t>(ws), reinterpret_cast<uintptr_t>(traces),
                                  reinterpret_cast<uintptr_t>(grad), reinterpret_cast<uintptr_t>(misfit),
                                  (uintptr_t)param, (uintptr_t)mf.mean_stress, (uintptr_t)p->fwd_valid};
    for (int c = 0; c < 5; ++c) {
        key.push_back(reinterpret_cast<uintptr_t>(observed[c]));
        key.push_back(reinterpret_cast<uintptr_t>(adjoint_source[c]));
    }
    for (float v : p->src_vals) {
        uint32_t b;
        memcpy(&b, &v, 4);
        key.push_back(b);
    }
    rc = p->opt.graph && !p->profiling
             ? run_graph(p, p->gmis, key, st, call_launches(p, true),
                         [&](cudaStream_t s) { return gradient_enqueue(p, ws, nullptr, param, grad, nullptr, s, &mf); })
             : gradient_enqueue(p, ws, nullptr, param, grad, nullptr, st, &mf);
    if (rc) return rc;
    // the last group's states are in the store: a pyfwi_gradient may follow
    // without another forward only if there is one group and nothing was recomputed
    p->fwd_valid = p->ngroups == 1 && (p->opt.checkpoint != PYFWI_CKPT_EXACT || p->M == 1);
    return PYFWI_OK;
}

int pyfwi_l2_residual(const float *est, const float *obs, float *res, int64_t n, double *scratch, double *misfit,
                      void *stream)
{
    if (!est || !obs || !res || !scratch || !misfit || n < 0) return fail(PYFWI_E_INVALID, "bad argument");
    if (n == 0) return PYFWI_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nb = grid_blocks(n);
    l2_kernel<<<nb, 256, 0, st>>>(est, obs, res, n, scratch);
    CKL();
    sum_partials_kernel<<<1, 32, 0, st>>>(scratch, nb, misfit);
    CKL();
    return PYFWI_OK;
}

int pyfwi_smooth(const float *in, float *out, float *tmp, int32_t n, int32_t nz, int32_t nx, const double *weights,
                 int32_t radius, void *stream)
{
    if (!in || !out || !tmp || !weights || n < 0 || nz < 1 || nx < 1) return fail(PYFWI_E_INVALID, "bad argument");
    if (radius < 0 || radius > SMOOTH_MAX_RADIUS)
        return fail(PYFWI_E_INVALID, "smoothing radius %d outside [0, %d]", radius, SMOOTH_MAX_RADIUS);
    if (n == 0) return PYFWI_OK;
    if (tmp == in || tmp == out) return fail(PYFWI_E_INVALID, "tmp must not alias in or out");
    SmoothWeights w;
    memset(&w, 0, sizeof w);
    for (int k = 0; k <= 2 * radius; ++k) w.w[k] = weights[k];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long total = (long long)n * nz * nx;
    smooth_kernel<<<grid_blocks(total), 256, 0, st>>>(in, tmp, n, nz, nx, 0, radius, w);
    CKL();
    smooth_kernel<<<grid_blocks(total), 256, 0, st>>>(tmp, out, n, nz, nx, 1, radius, w);
    CKL();
    return PYFWI_OK;
}

int pyfwi_mean2(const float *a, const float *b, float *out, int64_t n, void *stream)
{
    if (!a || !b || !out || n < 0) return fail(PYFWI_E_INVALID, "bad argument");
    if (n == 0) return PYFWI_OK;
    mean2_kernel<<<grid_blocks(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(a, b, out, n);
    CKL();
    return PYFWI_OK;
}

}  // extern "C"
