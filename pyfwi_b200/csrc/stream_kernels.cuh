// Streaming ("z-marching") variants of the step kernels, fed by TMA.
//
// A CTA of T = W - 2R threads owns W grid columns of one shot (T - 2R of
// them are written; the columns at either side are recomputed by the
// neighbouring CTA) and marches down a chunk of rows.  Input rows arrive in
// shared-memory row rings through TMA bulk tensor copies
// (cp.async.bulk.tensor, one W-float row of one field per copy, the copies
// of a row spread over the lanes of warp 0) PF rows ahead of use; completion is tracked by one mbarrier per
// in-flight row.  z-neighbours are read from the rings, x-neighbours from
// the same ring rows; the velocities the forward step computes (and the
// adjoint stresses of the adjoint step) live in register windows and one
// shared row ring.
//
// The workspace is one 2-D tensor for the TMA unit: rows of `pitch` floats,
// every plane starting on a row boundary, so plane row r of the plane at
// pointer p is tensor row (p - base) / pitch + r + ZO.  Rows and columns
// outside that tensor arrive as zeros.  Every wait on an mbarrier is bounded;
// a wait that gives up sets the workspace error word and the CTA stops at its
// next barrier.
//
// Same arithmetic, edge rules and source handling as the tile kernels in
// kernels.cuh.  The adjoint residual is added by inject_kernel into the
// input adjoint state before the step.
#pragma once

#include <cuda.h>

#include "kernels.cuh"

namespace pyfwi {

// ---- TMA / mbarrier primitives ---------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// One box (W floats x 1 row) of the workspace tensor at (x, y) into shared memory.
__device__ __forceinline__ void tma_row(float *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

constexpr unsigned long long WAIT_NS = 1000000000ull;  // give up on a copy after one second

__device__ __forceinline__ unsigned mbar_try(uint64_t *bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return done;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// Wait for phase `parity` of `bar`; false (and the error word set to 1) if
// it does not complete within `limit_ns` of the global timer.
__device__ __forceinline__ bool mbar_wait_for(uint64_t *bar, unsigned parity, int *err, unsigned long long limit_ns)
{
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try(bar, parity))
        if (global_ns() - t0 > limit_ns) {
            atomicExch(err, 1);
            return false;
        }
    return true;
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int *err)
{
    return mbar_wait_for(bar, parity, err, WAIT_NS);
}

// The bounded wait on an mbarrier nothing arrives at: one thread waits
// `limit_ns` and gives up as a streaming kernel does, so the timeout path
// and the host's handling of the error word can be exercised on purpose.
__global__ void wait_selftest_kernel(int *err, unsigned long long limit_ns)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_wait_for(&bar, 0, err, limit_ns);
}

// Tensor row of plane row r of the plane starting at p.
__device__ __forceinline__ int trow(const float *p, const float *base, int pitch, int r)
{
    return (int)((p - base) / pitch) + r + ZO;
}

// Non-negative ring index of row r for a ring of n rows.
__device__ __forceinline__ int ring(int r, int n) { return (r % n + n) % n; }

// z-differences down column `col` of a ring whose rows r-R .. r+R start at
// the offsets o[0..2R] (o[R] is row r).
template <int R>
__device__ __forceinline__ float ofwd(const float *rg, const int (&o)[2 * R + 1], int col, const float *c)
{
    float v = c[0] * (rg[o[R + 1] + col] - rg[o[R] + col]);
    v = fmaf(c[1], rg[o[R + 2] + col] - rg[o[R - 1] + col], v);
    if (R == 4) {
        v = fmaf(c[2], rg[o[R + 3] + col] - rg[o[R - 2] + col], v);
        v = fmaf(c[3], rg[o[R + 4] + col] - rg[o[R - 3] + col], v);
    }
    return v;
}

template <int R>
__device__ __forceinline__ float obwd(const float *rg, const int (&o)[2 * R + 1], int col, const float *c)
{
    float v = c[0] * (rg[o[R] + col] - rg[o[R - 1] + col]);
    v = fmaf(c[1], rg[o[R + 1] + col] - rg[o[R - 2] + col], v);
    if (R == 4) {
        v = fmaf(c[2], rg[o[R + 2] + col] - rg[o[R - 3] + col], v);
        v = fmaf(c[3], rg[o[R + 3] + col] - rg[o[R - 4] + col], v);
    }
    return v;
}

// Offsets (in floats) of rows r-R .. r+R in a ring of n rows of width w.
template <int R>
__device__ __forceinline__ void ring_rows(int (&o)[2 * R + 1], int r, int n, int w)
{
    int s = ring(r - R, n);
#pragma unroll
    for (int q = 0; q < 2 * R + 1; ++q) {
        o[q] = s * w;
        s = (s + 1 == n) ? 0 : s + 1;
    }
}

// Adjoint residual injection (Adj_injSrc, elastic_surface.cl:48-71,
// elastic.cl:316-363): adds this step's residual row to the five adjoint
// fields at every receiver, in place.  One CTA per shot (blockIdx.y); the
// lines are walked in order so two receivers on one cell add in turn.
// transpose != 0: the exact adjoint of the recording, where a line whose vz
// trace records vx (crosswell) sends its vz residual to the vx field.
__global__ void inject_kernel(Grid g, float *adj, long long stride, int shot0, int row, const float *r0,
                              const float *r1, const float *r2, const float *r3, const float *r4, Lines L, int ns,
                              int nr, int transpose)
{
    const float *res[5] = {r0, r1, r2, r3, r4};
    const int slot = blockIdx.y, shot = shot0 + slot;
    float *st = adj + slot * stride;
    for (int l = 0; l < L.n; ++l) {
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.count[l]; k += gridDim.x * blockDim.x) {
            const int i = L.row0[l] + k * L.drow[l], j = L.col0[l] + k * L.dcol[l];
            if (i < 0 || i >= g.tnz || j < 0 || j >= g.tnx) continue;
            const long long o = (long long)row * ns * nr + (long long)shot * nr + L.slot0[l] + k;
            const long long c = cell_off(g, i, j);
            for (int f = 0; f < 5; ++f) {
                const int to = (transpose && f == VZ && L.vzx[l]) ? VX : f;
                if (res[f]) st[to * g.plane + c] += __ldg(res[f] + o);
            }
        }
        __syncthreads();
    }
}

// After an abandoned wait: wait (bounded) for the copies still in flight so
// that none lands in shared memory after the CTA has left.  `abort_at` is
// 0 on the normal path (nothing is outstanding then), else 1 + the first
// iteration not consumed.
__device__ __forceinline__ void drain(uint64_t *bar, int nb, int kb, int ke, int pf, int abort_at, int *err)
{
    if (!abort_at) return;
    mbar_wait(bar + nb, 0, err);  // the prologue rows
    const int first = abort_at - 1, n = ke - kb;
    for (int it = first; it < min(first + pf, n); ++it) mbar_wait(bar + it % nb, (it / nb) & 1, err);
}

// Shared-memory layout common to both ring kernels: the mbarriers in the
// first 128 bytes, then 128-byte aligned rings of W-float rows (W is 64 or
// 128, so every row is a 128-byte aligned TMA destination).
constexpr int BAR_BYTES = 128;

// ---------------------------------------------------------------------------
// forward step (elastic.cl:155-308, coeff = +1)
// ---------------------------------------------------------------------------
template <int R, int W, int PFW>
struct FwdRing {
    static constexpr int T = W - 2 * R;         // threads = computed columns
    static constexpr int NT = 2 * R + 1 + PFW;  // stress rows k-R .. k+R+PF
    static constexpr int NQ = PFW + 1;          // pointwise rows
    static constexpr int NB = PFW + 1;          // mbarriers for rows in flight (+1 prologue)
    static constexpr int FLOATS = 3 * NT * W + 5 * NQ * W + 2 * (R + 1) * T;
    static constexpr size_t BYTES = BAR_BYTES + FLOATS * sizeof(float);
    static constexpr unsigned TX = 8u * W * sizeof(float);  // bytes landing per iteration
};

template <int R, int W, int PFW>
__global__ void __launch_bounds__(W - 2 * R) fwd_stream(const __grid_constant__ StepArgs a)
{
    using S = FwdRing<R, W, PFW>;
    // the x coordinate of every copy, blockIdx.x * (W - 4R) - 2R + XO, is a multiple of 4 floats
    static_assert((W - 4 * R) % 4 == 0 && (XO - 2 * R) % 4 == 0 && W <= 256, "TMA x alignment");
    static_assert(S::NB + 1 <= (BAR_BYTES - 8) / 8, "mbarriers exceed their area");
    constexpr int T = S::T, IW = T - 2 * R, NT = S::NT, NQ = S::NQ, NB = S::NB, WL = 2 * R + 1, NV = R + 1;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);  // [NB + 1], the last one for the prologue
    float *s_t = reinterpret_cast<float *>(smem + BAR_BYTES);  // [3][NT][W] txx, tzz, txz
    float *s_q = s_t + 3 * NT * W;                             // [5][NQ][W] vx, vz, b (row k), lam, mu (row k-R)
    float *s_v = s_q + 5 * NQ * W;                             // [2][NV][T] new velocities rows k-R .. k
    int &s_abort = *reinterpret_cast<int *>(smem + BAR_BYTES - sizeof(int));

    const Grid &g = a.g;
    const int t = threadIdx.x, slot = blockIdx.z, shot = a.shot0 + slot;
    const int c0 = blockIdx.x * IW - R, j = c0 + t;  // this thread's column, ring column t + R
    const int z0 = blockIdx.y * a.chunk, z1 = min(z0 + a.chunk, g.tnz);
    const int kb = z0 - R, ke = z1 + R;
    const long long P = g.plane;
    const float *in = a.in + slot * a.in_stride;
    float *out = a.out + slot * a.out_stride;
    const float dt = a.k.dt;
    const int si = a.add_src ? a.srcz[shot] : -(1 << 30), sj = a.srcx[shot];
    const float dxj = (j + XO >= 0 && j + XO < g.pitch) ? __ldg(a.dampx + j + XO) : 0.f;
    const bool inner = t >= R && t < T - R && j < g.tnx;
    const int x0 = c0 - R + XO;  // tensor column of ring column 0 (a multiple of 4)

    if (t == 0) {
        for (int b = 0; b <= NB; ++b) mbar_init(bar + b, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        // every TMA destination must be 128-byte aligned: refuse to copy otherwise
        s_abort = (smem_u32(smem) & 127) != 0;
        if (s_abort) atomicExch(a.err, 2);
        // after an earlier failure the results are void: stop at once
        if (*reinterpret_cast<volatile int *>(a.err)) s_abort = 1;
    }
    __syncthreads();
    if (s_abort) return;

    // rows iteration m consumes: stress row m+R, vx/vz/b row m, lam/mu row m-R;
    // issued by the lanes of warp 0, one row copy per lane
    auto issue = [&](int m) {
        uint64_t *bm = bar + (m - kb) % NB;
        if (t == 0) mbar_expect_tx(bm, S::TX);
        __syncwarp();
        const int q = t;
        if (q < 8) {
            float *dst;
            const float *src;
            int row;
            if (q < 3) {
                dst = s_t + (q * NT + ring(m + R, NT)) * W;
                src = in + (TXX + q) * P;
                row = m + R;
            } else if (q < 6) {
                const int f = q - 3;
                dst = s_q + (f * NQ + ring(m, NQ)) * W;
                src = f == 2 ? a.mat + 2 * P : in + (VX + f) * P;
                row = m;
            } else {
                const int f = q - 6;
                dst = s_q + ((3 + f) * NQ + ring(m - R, NQ)) * W;
                src = a.mat + f * P;
                row = m - R;
            }
            tma_row(dst, &a.tmap, x0, trow(src, a.tbase, g.pitch, row), bm);
        }
    };
    if (t < 32) {
        uint64_t *bp = bar + NB;  // stress rows kb-R .. kb+R-1
        if (t == 0) mbar_expect_tx(bp, 3u * 2 * R * W * sizeof(float));
        __syncwarp();
        for (int q = t; q < 6 * R; q += 32) {
            const int r = kb - R + q / 3, f = q % 3;
            tma_row(s_t + (f * NT + ring(r, NT)) * W, &a.tmap, x0, trow(in + (TXX + f) * P, a.tbase, g.pitch, r), bp);
        }
        for (int m = kb; m < min(kb + PFW, ke); ++m) issue(m);
    }
    if (!mbar_wait(bar + NB, 0, a.err)) s_abort = 1;
    __syncthreads();
    // the step adds the source to the stresses of every row it reads
    // (elastic_surface.cl:23-28): patch the ring once, before first use
    bool src_done = !(si >= kb - R && si < ke + R);

    float wvx[WL], wvz[WL];
#pragma unroll
    for (int q = 0; q < WL; ++q) wvx[q] = wvz[q] = 0.f;
    const float *txx_r = s_t, *tzz_r = s_t + NT * W, *txz_r = s_t + 2 * NT * W;
    const int rc = t + R;

    for (int k = kb; k < ke; ++k) {
        const int it = k - kb;
        if (!mbar_wait(bar + it % NB, (it / NB) & 1, a.err)) s_abort = 1;
        __syncthreads();
        if (s_abort) {
            s_abort = it + 1;  // iterations 0 .. it-1 were consumed (every thread writes the same)
            break;
        }
        if (t < 32 && k + PFW < ke) issue(k + PFW);
        if (!src_done && k + R >= si) {  // CTA-uniform: row si is resident and not read yet
            src_done = true;
            const int cs = sj - (c0 - R);
            if (t == 0 && cs >= 0 && cs < W) {
                const int st = ring(si, NT);
                s_t[(0 * NT + st) * W + cs] += a.src.z;
                s_t[(1 * NT + st) * W + cs] += a.src.w;
                // order these generic writes before a later TMA reuses the slot
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            }
            __syncthreads();
        }
        int o[2 * R + 1];
        ring_rows<R>(o, k, NT, W);
        const int qk = ring(k, NQ) * W;

        // velocities at (k, j): update_velx / update_velz
        float vx = s_q[0 * NQ * W + qk + rc], vz = s_q[1 * NQ * W + qk + rc];
        if (k == si && j == sj) {
            vx += a.src.x;
            vz += a.src.y;
        }
        if (in_domain(g, R, k, j)) {
            const float b = s_q[2 * NQ * W + qk + rc];
            const float d = dxj + __ldg(a.dampz + k + ZO);
            vx = vx + dt * (b * (dbwd<R>(txx_r + o[R], rc, 1, a.k.cx) + obwd<R>(txz_r, o, rc, a.k.cz)));
            vx = vx + dt * (-d * vx);
            vz = vz + dt * (b * (ofwd<R>(tzz_r, o, rc, a.k.cz) + dfwd<R>(txz_r + o[R], rc, 1, a.k.cx)));
            vz = vz + dt * (-d * vz);
        }
        shift(wvx, vx);
        shift(wvz, vz);
        const int kv = ring(k, NV);
        s_v[(0 * NV + kv) * T + t] = vx;
        s_v[(1 * NV + kv) * T + t] = vz;
        __syncthreads();

        // stresses at (i, j), i = k - R: update_tauz / update_tauxz
        const int i = k - R;
        if (i >= z0 && inner) {
            const int oi = o[0], qi = ring(i, NQ) * W;
            float txx = txx_r[oi + rc], tzz = tzz_r[oi + rc], txz = txz_r[oi + rc];
            const long long co = cell_off(g, i, j);
            if (in_domain(g, R, i, j)) {
                const int iv = ring(i, NV);
                const float lam = s_q[3 * NQ * W + qi + rc], mu = s_q[4 * NQ * W + qi + rc];
                const float d = dxj + __ldg(a.dampz + i + ZO);
                const float *rvx = s_v + (0 * NV + iv) * T, *rvz = s_v + (1 * NV + iv) * T;
                float dxp_vx = dfwd<R>(rvx, t, 1, a.k.cx), dzm_vz = wbwd<R>(wvz, a.k.cz);
                float dxm_vz = dbwd<R>(rvz, t, 1, a.k.cx), dzp_vx = wfwd<R>(wvx, a.k.cz);
                normal_pair_fwd(lam, mu, dxp_vx, dzm_vz, d, dt, txx, tzz);
                txz = txz + dt * (mu * (dxm_vz + dzp_vx));
                txz = txz + dt * (-d * txz);
            }
            out[VX * P + co] = wvx[R];
            out[VZ * P + co] = wvz[R];
            out[TXX * P + co] = txx;
            out[TZZ * P + co] = tzz;
            out[TXZ * P + co] = txz;
            if (a.snap)
                write_snap(a.snap + slot * a.snap_stride, a.snap8 ? a.snap8 + slot * a.snap_stride : nullptr, P, co,
                           wvx[R], wvz[R], txx, tzz, txz);
            if (a.rec_row >= 0) record_cell(a, a.rec_row, in, shot, i, j);
        }
    }
    drain(bar, NB, kb, ke, PFW, s_abort, a.err);
}

// ---------------------------------------------------------------------------
// adjoint step + imaging (Adj_update_tau, Adj_update_v, Grad); the residual
// is already in the input state (inject_kernel)
// ---------------------------------------------------------------------------
template <int R, int W, int PFW, bool ENERGY>
struct AdjRing {
    static constexpr int T = W - 2 * R;
    static constexpr int NA = 2 * R + 1 + PFW;  // adjoint velocity + buoyancy rows k-R .. k+R+PF
    static constexpr int NQ = PFW + 1;          // pointwise rows
    static constexpr int NF = 2 * R + 1 + PFW;  // forward rows k-2R .. k+PF
    static constexpr int NG = ENERGY ? 6 : 3;
    static constexpr int NP = R + 1;
    static constexpr int NB = PFW + 1;
    static constexpr int FLOATS = 3 * NA * W + 5 * NQ * W + 5 * NF * W + NG * NQ * W + 3 * NP * T;
    static constexpr size_t BYTES = BAR_BYTES + FLOATS * sizeof(float);
    static constexpr unsigned TX = (13u + NG) * W * sizeof(float);
};

template <int R, int W, int PFW, bool ENERGY>
__global__ void __launch_bounds__(W - 2 * R) adj_stream(const __grid_constant__ AdjArgs a)
{
    using S = AdjRing<R, W, PFW, ENERGY>;
    // the x coordinate of every copy, blockIdx.x * (W - 4R) - 2R + XO, is a multiple of 4 floats
    static_assert((W - 4 * R) % 4 == 0 && (XO - 2 * R) % 4 == 0 && W <= 256, "TMA x alignment");
    static_assert(S::NB + 1 <= (BAR_BYTES - 8) / 8, "mbarriers exceed their area");
    constexpr int T = S::T, IW = T - 2 * R, NA = S::NA, NQ = S::NQ, NF = S::NF, NG = S::NG, NB = S::NB,
                  WL = 2 * R + 1, NP = S::NP;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    float *s_a = reinterpret_cast<float *>(smem + BAR_BYTES);  // [3][NA][W]  Avx, Avz, b
    float *s_q = s_a + 3 * NA * W;                             // [5][NQ][W]  Atx, Atz, Atxz, lam, mu (row k)
    float *s_f = s_q + 5 * NQ * W;                             // [5][NF][W]  forward vx, vz, txx, tzz, txz
    float *s_g = s_f + 5 * NF * W;                             // [NG][NQ][W] accumulators (row k-R)
    float *s_p = s_g + NG * NQ * W;  // [3][NP][T]  (lam+2mu)Atx, lam Atz, mu Atxz rows k-R .. k
    int &s_abort = *reinterpret_cast<int *>(smem + BAR_BYTES - sizeof(int));

    const Grid &g = a.g;
    const int t = threadIdx.x, slot = blockIdx.z;
    const int c0 = blockIdx.x * IW - R, j = c0 + t;
    const int z0 = blockIdx.y * a.chunk, z1 = min(z0 + a.chunk, g.tnz);
    const int kb = z0 - R, ke = z1 + R;
    const long long P = g.plane;
    const float *in = a.in + slot * a.in_stride;
    float *out = a.out + slot * a.out_stride;
    const float *F = a.fwd + slot * a.fwd_stride;
    float *G = a.gacc + slot * a.gacc_stride;
    const float dt = a.k.dt;
    const float dxj = (j + XO >= 0 && j + XO < g.pitch) ? __ldg(a.dampx + j + XO) : 0.f;
    const bool inner = t >= R && t < T - R && j < g.tnx;
    const int glo = a.npml + R;
    const bool gcol = inner && j >= glo && j <= g.tnx - R - a.npml;
    const int x0 = c0 - R + XO;

    if (t == 0) {
        for (int b = 0; b <= NB; ++b) mbar_init(bar + b, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        // every TMA destination must be 128-byte aligned: refuse to copy otherwise
        s_abort = (smem_u32(smem) & 127) != 0;
        if (s_abort) atomicExch(a.err, 2);
        // after an earlier failure the results are void: stop at once
        if (*reinterpret_cast<volatile int *>(a.err)) s_abort = 1;
    }
    __syncthreads();
    if (s_abort) return;

    // rows iteration m consumes: adjoint velocities + b row m+R, adjoint
    // stresses + lam/mu row m, forward state row m, accumulators row m-R
    // issued by the lanes of warp 0, one row copy per lane
    auto issue = [&](int m) {
        uint64_t *bm = bar + (m - kb) % NB;
        if (t == 0) mbar_expect_tx(bm, S::TX);
        __syncwarp();
        const int q = t;
        if (q < 13 + NG) {
            float *dst;
            const float *src;
            int row = m;
            if (q < 3) {  // adjoint velocities and buoyancy, row m+R
                dst = s_a + (q * NA + ring(m + R, NA)) * W;
                src = q == 2 ? a.mat + 2 * P : in + (VX + q) * P;
                row = m + R;
            } else if (q < 8) {  // adjoint stresses, lam, mu, row m
                const int f = q - 3;
                dst = s_q + (f * NQ + ring(m, NQ)) * W;
                src = f < 3 ? in + (TXX + f) * P : a.mat + (f - 3) * P;
            } else if (q < 13) {  // forward state, row m
                const int f = q - 8;
                dst = s_f + (f * NF + ring(m, NF)) * W;
                src = F + f * P;
            } else {  // accumulators, row m-R
                const int f = q - 13;
                dst = s_g + (f * NQ + ring(m - R, NQ)) * W;
                src = G + f * P;
                row = m - R;
            }
            tma_row(dst, &a.tmap, x0, trow(src, a.tbase, g.pitch, row), bm);
        }
    };
    if (t < 32) {
        uint64_t *bp = bar + NB;  // adjoint velocity + b rows kb-R .. kb+R-1
        if (t == 0) mbar_expect_tx(bp, 3u * 2 * R * W * sizeof(float));
        __syncwarp();
        for (int q = t; q < 6 * R; q += 32) {
            const int r = kb - R + q / 3, f = q % 3;
            tma_row(s_a + (f * NA + ring(r, NA)) * W, &a.tmap, x0,
                    trow(f == 2 ? a.mat + 2 * P : in + (VX + f) * P, a.tbase, g.pitch, r), bp);
        }
        for (int m = kb; m < min(kb + PFW, ke); ++m) issue(m);
    }
    if (!mbar_wait(bar + NB, 0, a.err)) s_abort = 1;
    __syncthreads();

    float wpl[WL], wpm[WL], wpu[WL];         // lam*Atx, (lam+2mu)*Atz, mu*Atxz rows k-2R .. k
    float atx_d[NP], atz_d[NP], atxz_d[NP];  // new adjoint stresses rows k-R .. k
#pragma unroll
    for (int q = 0; q < WL; ++q) wpl[q] = wpm[q] = wpu[q] = 0.f;
#pragma unroll
    for (int q = 0; q < NP; ++q) atx_d[q] = atz_d[q] = atxz_d[q] = 0.f;
    const float *avx_r = s_a, *avz_r = s_a + NA * W, *b_r = s_a + 2 * NA * W;
    const int rc = t + R;

    for (int k = kb; k < ke; ++k) {
        const int it = k - kb;
        if (!mbar_wait(bar + it % NB, (it / NB) & 1, a.err)) s_abort = 1;
        __syncthreads();
        if (s_abort) {
            s_abort = it + 1;  // iterations 0 .. it-1 were consumed (every thread writes the same)
            break;
        }
        if (t < 32 && k + PFW < ke) issue(k + PFW);
        int oa[2 * R + 1];
        ring_rows<R>(oa, k, NA, W);
        const int qk = ring(k, NQ) * W;

        // adjoint stresses at (k, j) for every column of the CTA (Adj_update_tau)
        float atx = s_q[0 * NQ * W + qk + rc], atz = s_q[1 * NQ * W + qk + rc], atxz = s_q[2 * NQ * W + qk + rc];
        if (in_domain(g, R, k, j)) {
            const float dk = __ldg(a.dampz + k + ZO);
            // x differences of Av*b on row k, z differences down ring column rc
            const float dxp_avx = dfwd_p<R>(avx_r + oa[R], b_r + oa[R], rc, 1, a.k.cx);
            const float dxm_avz = dbwd_p<R>(avz_r + oa[R], b_r + oa[R], rc, 1, a.k.cx);
#define AB_(f, d) (f[oa[R + (d)] + rc] * b_r[oa[R + (d)] + rc])
            float dzm_avz = a.k.cz[0] * (AB_(avz_r, 0) - AB_(avz_r, -1));
            dzm_avz = fmaf(a.k.cz[1], AB_(avz_r, 1) - AB_(avz_r, -2), dzm_avz);
            float dzp_avx = a.k.cz[0] * (AB_(avx_r, 1) - AB_(avx_r, 0));
            dzp_avx = fmaf(a.k.cz[1], AB_(avx_r, 2) - AB_(avx_r, -1), dzp_avx);
            if constexpr (R == 4) {
                dzm_avz = fmaf(a.k.cz[2], AB_(avz_r, 2) - AB_(avz_r, -3), dzm_avz);
                dzm_avz = fmaf(a.k.cz[3], AB_(avz_r, 3) - AB_(avz_r, -4), dzm_avz);
                dzp_avx = fmaf(a.k.cz[2], AB_(avx_r, 3) - AB_(avx_r, -2), dzp_avx);
                dzp_avx = fmaf(a.k.cz[3], AB_(avx_r, 4) - AB_(avx_r, -3), dzp_avx);
            }
#undef AB_
            atx = atx + (-dt) * (dxj * atx + dxp_avx);
            atz = atz + (-dt) * (dk * atz + dzm_avz);
            atxz = atxz + (-dt) * ((dxj + dk) * atxz + (dzp_avx + dxm_avz));
        }
        {
            const float lam = s_q[3 * NQ * W + qk + rc], mu = s_q[4 * NQ * W + qk + rc];
            const float l2m = lam + 2.f * mu;
            const int kp = ring(k, NP);
            s_p[(0 * NP + kp) * T + t] = l2m * atx;
            s_p[(1 * NP + kp) * T + t] = lam * atz;
            s_p[(2 * NP + kp) * T + t] = mu * atxz;
            shift(wpl, lam * atx);
            shift(wpm, l2m * atz);
            shift(wpu, mu * atxz);
            shift(atx_d, atx);
            shift(atz_d, atz);
            shift(atxz_d, atxz);
        }
        __syncthreads();

        // adjoint velocities (Adj_update_v) and imaging (Grad) at (i, j)
        const int i = k - R;
        if (i >= z0 && inner) {
            const long long co = cell_off(g, i, j);
            const int ai = oa[0];
            float avx = avx_r[ai + rc], avz = avz_r[ai + rc];
            if (in_domain(g, R, i, j)) {
                const int ip = ring(i, NP);
                const float di = __ldg(a.dampz + i + ZO);
                float sx = dbwd<R>(s_p + (0 * NP + ip) * T, t, 1, a.k.cx) +
                           dbwd<R>(s_p + (1 * NP + ip) * T, t, 1, a.k.cx) + wbwd<R>(wpu, a.k.cz);
                float sz = wfwd<R>(wpl, a.k.cz) + wfwd<R>(wpm, a.k.cz) +
                           dfwd<R>(s_p + (2 * NP + ip) * T, t, 1, a.k.cx);
                avx = avx + (-dt) * ((2.f * dxj + di) * avx + sx);
                avz = avz + (-dt) * ((dxj + 2.f * di) * avz + sz);
            }
            const float atx0 = atx_d[0], atz0 = atz_d[0], atxz0 = atxz_d[0];
            out[VX * P + co] = avx;
            out[VZ * P + co] = avz;
            out[TXX * P + co] = atx0;
            out[TZZ * P + co] = atz0;
            out[TXZ * P + co] = atxz0;
            if (gcol && i >= glo && i <= g.tnz - R - a.npml) {
                int of[2 * R + 1];
                ring_rows<R>(of, i, NF, W);
                const int fi = of[R], gi = ring(i, NQ) * W;
                const float *fvx = s_f, *fvz = s_f + NF * W, *ftx = s_f + 2 * NF * W, *ftz = s_f + 3 * NF * W,
                            *ftxz = s_f + 4 * NF * W;
                // DzpVx is formed from vz, as the reference does (elastic.cl:485)
                float dzp_vx = ofwd<R>(fvz, of, rc, a.k.cz), dzm_vz = obwd<R>(fvz, of, rc, a.k.cz);
                float dxm_vz = dbwd<R>(fvz + fi, rc, 1, a.k.cx), dxp_vx = dfwd<R>(fvx + fi, rc, 1, a.k.cx);
                float dzp_tz = ofwd<R>(ftz, of, rc, a.k.cz), dxm_tx = dbwd<R>(ftx + fi, rc, 1, a.k.cx);
                float dxp_txz = dfwd<R>(ftxz + fi, rc, 1, a.k.cx), dzm_txz = obwd<R>(ftxz, of, rc, a.k.cz);
                const float b = b_r[ai + rc];
                float gmu = s_g[0 * NQ * W + gi + rc], glam = s_g[1 * NQ * W + gi + rc],
                      grho = s_g[2 * NQ * W + gi + rc];
                gmu += 2.f * dt * (atx0 * dxp_vx + atz0 * dzm_vz) + dt * atxz0 * (dzp_vx + dxm_vz);
                glam += dt * (atx0 + atz0) * (dxp_vx + dzm_vz);
                grho += -(dt * (b * b)) * (avx * (dxm_tx + dzm_txz) + avz * (dzp_tz + dxp_txz));
                G[0 * P + co] = gmu;
                G[1 * P + co] = glam;
                G[2 * P + co] = grho;
                if constexpr (ENERGY) {
                    const float dt2 = dt * dt, vx = fvx[fi + rc], vz = fvz[fi + rc], tx = ftx[fi + rc],
                                tz = ftz[fi + rc], txz = ftxz[fi + rc];
                    G[3 * P + co] = s_g[3 * NQ * W + gi + rc] +
                                    (4.f * dt2 * (tx * tx * dxp_vx * dxp_vx + tz * tz * dzm_vz * dzm_vz) +
                                     dt2 * txz * txz * (dzp_vx * dzp_vx + dxm_vz * dxm_vz));
                    G[4 * P + co] = s_g[4 * NQ * W + gi + rc] +
                                    dt2 * (tx * tx + tz * tz) * (dxp_vx * dxp_vx + dzm_vz * dzm_vz);
                    G[5 * P + co] = s_g[5 * NQ * W + gi + rc] +
                                    dt2 * (vx * vx * (dxm_tx * dxm_tx + dzm_txz * dzm_txz) +
                                           vz * vz * (dzp_tz * dzp_tz + dxp_txz * dxp_txz));
                }
            }
        }
    }
    drain(bar, NB, kb, ke, PFW, s_abort, a.err);
}

}  // namespace pyfwi
