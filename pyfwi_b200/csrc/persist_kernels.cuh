// Persistent step kernels for small surveys.
//
// A survey whose padded grid and shots fill only a fraction of the GPU (a
// few hundred tiles per step) spends most of a step launching it: each step
// kernel runs for a few microseconds.  The persistent kernels run a whole
// run of consecutive steps in one cooperative launch instead -- the
// reference's per-step, per-shot loops (wave_propagation.py:639-733 forward,
// :740-848 backward) become one loop inside the kernel: every CTA takes the
// (tile, shot) items of a step in turn, through the same tile code as the
// step kernels (fwd_tile, adj_tile), then all CTAs meet at a grid barrier
// before the next step.
//
// The grid barrier is a counter and a generation word in the workspace
// header, reset by the host before each launch.  The waiting thread of each
// CTA spins with a bound on the global timer: past it the kernel sets the
// workspace error word to 3 and every CTA leaves (later waits give up at once
// when they see the word); pyfwi_device_error reports it.  A cooperative
// launch puts every CTA on the GPU at once, so the bound is only a guard.
//
// Memory visibility: a step reads what other CTAs wrote in the step before,
// so those reads go through L2 (cp.async.cg staging, ld.global.cg), never
// through the read-only data path; the barrier's release/acquire pair at GPU
// scope orders the writes before the reads.
#pragma once

#include "stream_kernels.cuh"

namespace pyfwi {

constexpr int PERSIST_CHUNK = 512;                          // forward steps per launch (their source samples travel as parameters)
constexpr unsigned long long BARRIER_WAIT_NS = 1000000000ull;  // give up on a grid barrier after one second

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_relaxed_gpu(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// `expected` CTAs (all of the launch) meet here.  bar[0]: CTAs arrived,
// bar[1]: barrier generation.  False when the wait gave up (error word set,
// here or by another CTA): the caller then leaves the kernel.
__device__ __forceinline__ bool grid_sync(unsigned *bar, unsigned expected, int *err, unsigned long long limit_ns)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        const unsigned gen = ld_acquire_gpu(bar + 1);
        __threadfence();  // this CTA's writes of the step before it arrives
        if (atomicAdd(bar, 1u) == expected - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            st_release_gpu(bar + 1, gen + 1);
        } else {
            const unsigned long long t0 = global_ns();
            while (ld_acquire_gpu(bar + 1) == gen) {
                if (ld_relaxed_gpu(err) != 0) {
                    good = 0;
                    break;
                }
                if (global_ns() - t0 > limit_ns) {
                    atomicCAS(err, 0, 3);
                    good = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// The forward steps [t0, t1) of one shot group in the layout that stores
// every step in FP32: S_0 = store (zero), S_t = store + t * state, slots
// `sstride` apart.  Injection k (step k * dt_scale) adds wav[k - k0]
// (zero past the wavelet, filled in by the host); traces are recorded when
// `record` is set.
struct FwdPersistArgs {
    StepArgs a;        // constant fields; in / out / source / trace row are set per step here
    float *store;
    long long sstride, state;
    int t0, t1;
    int dt_scale, nt_ext, record;
    int nslots, ntx, ntz;
    unsigned *bar;     // [2] in the workspace header
    int *err;          // workspace error word
    unsigned long long limit_ns;
    int k0, nk;
    float4 wav[PERSIST_CHUNK];
};

template <int R, int TZ>
__global__ void __launch_bounds__(NTHREADS) fwd_persist(const __grid_constant__ FwdPersistArgs p)
{
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4);
    const int per_slot = p.ntx * p.ntz, nwork = per_slot * p.nslots;
    for (int t = p.t0; t < p.t1; ++t) {
        StepVar v;
        v.in = p.store + (long long)t * p.state;
        v.out = p.store + (long long)(t + 1) * p.state;
        v.in_stride = v.out_stride = p.sstride;
        const int k = t / p.dt_scale;
        v.add_src = t % p.dt_scale == 0;
        v.src = (v.add_src && k - p.k0 < p.nk) ? p.wav[k - p.k0] : make_float4(0.f, 0.f, 0.f, 0.f);
        v.rec_row = (v.add_src && p.record && k < p.nt_ext) ? k : -1;
        v.snap = nullptr;
        v.snap8 = nullptr;
        for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
            const int slot = w / per_slot, r = w - slot * per_slot, by = r / p.ntx, bx = r - by * p.ntx;
            fwd_tile<R, TZ, false>(p.a, v, bx, by, slot, sm);
            __syncthreads();  // shared memory is reused by the next tile
        }
        if (t + 1 < p.t1 && !grid_sync(p.bar, gridDim.x, p.err, p.limit_ns)) return;
    }
}

// The adjoint steps t = t_hi - 1 .. t_lo (t_lo >= 1) of one shot group,
// imaging S_{t+1} = store + (t + 1) * state (every step stored in FP32); the
// adjoint states alternate between adj and adj + state (slots 2 * state
// apart), starting from adj + ping0 * state.  The first step's residual is
// in its input already; each step adds the next one's (inj_row_of).
struct AdjPersistArgs {
    AdjArgs a;         // constant fields (a.nslots set)
    float *adj;
    const float *store;
    long long sstride, state;
    int t_hi, t_lo, ping0;
    int nt, nt_ext, dt_scale;
    int ntx, ntz;
    unsigned *bar;
    int *err;
    unsigned long long limit_ns;
};

// Residual row injected before backward step t (wave_propagation.py:814-824;
// the host's inj_row_of): -1 when t injects nothing.
__device__ __forceinline__ int inj_row_dev(int t, int nt, int nt_ext, int d)
{
    if (t < 0 || t % d) return -1;
    int row = nt_ext - 1 - ((nt - 1) / d - t / d);
    if (row < 0) row += nt_ext;
    return row;
}

template <int R, int TZ, bool ENERGY>
__global__ void __launch_bounds__(NTHREADS) adj_persist(const __grid_constant__ AdjPersistArgs p)
{
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4);
    const int per_slot = p.ntx * p.ntz, nwork = per_slot * p.a.nslots;
    int ping = p.ping0;
    for (int t = p.t_hi - 1; t >= p.t_lo; --t) {
        AdjVar v;
        v.in = p.adj + (long long)ping * p.state;
        v.out = p.adj + (long long)(1 - ping) * p.state;
        v.fwd = p.store + (long long)(t + 1) * p.state;
        v.fwd16 = nullptr;
        v.fwd8 = nullptr;
        v.epi_row = t - 1 >= 1 ? inj_row_dev(t - 1, p.nt, p.nt_ext, p.dt_scale) : -1;
        for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
            const int slot = w / per_slot, r = w - slot * per_slot, by = r / p.ntx, bx = r - by * p.ntx;
            adj_tile<R, TZ, ENERGY, 1, false, true>(p.a, v, bx, by, slot, sm);
            __syncthreads();
        }
        ping = 1 - ping;
        if (t > p.t_lo && !grid_sync(p.bar, gridDim.x, p.err, p.limit_ns)) return;
    }
}

// Failure-path self test of the grid barrier: the CTAs of this launch wait
// for one CTA more than there are, so the wait runs out after `limit_ns` and
// sets the error word to 3, as a persistent kernel's would.
__global__ void barrier_selftest_kernel(unsigned *bar, int *err, unsigned long long limit_ns)
{
    grid_sync(bar, gridDim.x + 1, err, limit_ns);
}

}  // namespace pyfwi
