// Forward step fed by the Tensor Memory Accelerator.
//
// The same tile step as fwd_step (elastic.cl:155-308, coeff = +1: source
// add, velocities on the tile and a ring, stresses on the tile, traces from
// the input state), with the haloed tile staged by eight 2-D TMA box copies
// (cp.async.bulk.tensor, no multicast: this GPU's own workspace) instead of
// ~3000 16-byte cp.async copies issued by every thread: the three stresses
// (SW x HT box, rows i0-2R ..), the two velocities and the buoyancy (VW x HV,
// rows i0-R ..) and lam, mu (TX x TZ).  One thread issues the copies; every
// thread waits on the mbarrier with the one-second bound of the streaming
// kernels (error word 1, a drain of the copies in flight, then leave).
//
// The tensor maps cover the workspace as rows of `pitch` floats, so a box
// runs over whole rows of one plane: rows past the last allocated row read
// as zero (the map's fill), columns past the pitch likewise; rows past a
// plane's zero frame fall into the next plane, but only cells outside the
// update domain are computed from them and those are never stored changed
// (the frame is eight rows, the stencil reaches four).  Every box starts on a
// column that is a multiple of 4 floats (16 bytes): j0 - 8 + XO = j0,
// j0 - 4 + XO, j0 + XO with j0 a multiple of 64.
#pragma once

#include "stream_kernels.cuh"

namespace pyfwi {

struct FwdTmaArgs {
    StepArgs a;                  // a.tbase: workspace base (row 0 of the maps); a.err: error word
    alignas(64) CUtensorMap ms;  // box SW x HT: stresses
    alignas(64) CUtensorMap mv;  // box VW x HV: velocities, buoyancy
    alignas(64) CUtensorMap mt;  // box TX x TZ: lam, mu
};

template <int R, int TZ>
struct FwdTmaShape {
    using S = FwdShape<R, TZ>;
    static constexpr size_t BYTES = BAR_BYTES + S::FLOATS * sizeof(float);
    static constexpr unsigned TXB = S::FLOATS * sizeof(float);  // bytes the eight boxes land
    static_assert((S::HT * S::SW * 4) % 128 == 0 && (S::HV * S::VW * 4) % 128 == 0 && (TZ * TX * 4) % 128 == 0,
                  "every box lands 128-byte aligned");
};

template <int R, int TZ, bool W24>
__global__ void __launch_bounds__(NTHREADS) fwd_tma(const __grid_constant__ FwdTmaArgs t)
{
    using S = FwdShape<R, TZ>;
    constexpr int SW = S::SW, VW = S::VW, HT = S::HT, HV = S::HV;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    int &s_abort = *reinterpret_cast<int *>(smem + BAR_BYTES - sizeof(int));
    float *sm = reinterpret_cast<float *>(smem + BAR_BYTES);
    const StepArgs &a = t.a;
    const Grid &g = a.g;
    const long long P = g.plane;
    const int slot = blockIdx.z, j0 = blockIdx.x * TX, i0 = blockIdx.y * TZ;
    const float *in = a.in + slot * a.in_stride;

    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        // every TMA destination must be 128-byte aligned: refuse to copy otherwise
        s_abort = (smem_u32(smem) & 127) != 0;
        if (s_abort) atomicExch(a.err, 2);
        // after an earlier failure the results are void: stop at once
        if (*reinterpret_cast<volatile int *>(a.err)) s_abort = 1;
        if (!s_abort) {
            float *s_txx = sm, *s_tzz = s_txx + HT * SW, *s_txz = s_tzz + HT * SW;
            float *s_vx = s_txz + HT * SW, *s_vz = s_vx + HV * VW, *s_b = s_vz + HV * VW;
            float *s_lam = s_b + HV * VW, *s_mu = s_lam + TZ * TX;
            mbar_expect_tx(bar, FwdTmaShape<R, TZ>::TXB);
            const int xs = j0 - 8 + XO, xv = j0 - 4 + XO, xt = j0 + XO;
            tma_row(s_txx, &t.ms, xs, trow(in + TXX * P, a.tbase, g.pitch, i0 - 2 * R), bar);
            tma_row(s_tzz, &t.ms, xs, trow(in + TZZ * P, a.tbase, g.pitch, i0 - 2 * R), bar);
            tma_row(s_txz, &t.ms, xs, trow(in + TXZ * P, a.tbase, g.pitch, i0 - 2 * R), bar);
            tma_row(s_vx, &t.mv, xv, trow(in + VX * P, a.tbase, g.pitch, i0 - R), bar);
            tma_row(s_vz, &t.mv, xv, trow(in + VZ * P, a.tbase, g.pitch, i0 - R), bar);
            tma_row(s_b, &t.mv, xv, trow(a.mat + 2 * P, a.tbase, g.pitch, i0 - R), bar);
            tma_row(s_lam, &t.mt, xt, trow(a.mat, a.tbase, g.pitch, i0), bar);
            tma_row(s_mu, &t.mt, xt, trow(a.mat + P, a.tbase, g.pitch, i0), bar);
        }
    }
    __syncthreads();
    if (s_abort) return;
    if (!mbar_wait(bar, 0, a.err)) s_abort = 1;
    __syncthreads();
    if (s_abort) {
        if (threadIdx.x == 0) mbar_wait(bar, 0, a.err);  // the copies in flight land before the CTA leaves
        return;
    }
    fwd_tile<R, TZ, W24, StepArgs, true>(a, a, blockIdx.x, blockIdx.y, slot, sm);
}

}  // namespace pyfwi
